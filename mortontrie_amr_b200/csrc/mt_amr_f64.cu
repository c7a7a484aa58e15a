// FP64 instantiation of the multi-level phases.  Built with --fmad=false so
// every phase keeps the reference's rounding (bit-for-bit parity).
#include "mt_amr_phases.cuh"

namespace mt {
template struct AmrOps<double>;
}
