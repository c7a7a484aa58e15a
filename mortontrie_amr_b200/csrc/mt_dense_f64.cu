// FP64 instantiation of the dense uniform path.  Built with --fmad=false so
// the collision keeps the reference's rounding (bit-for-bit parity).
#include "mt_dense.cuh"

namespace mt {
template struct DenseOps<double>;
}
