// Reduced-precision instantiations of the multi-level phases: FP32
// arithmetic on populations stored as f - s_q (the level's storage shift) in
// FP32, FP16 or BF16.
#include "mt_amr_phases.cuh"

namespace mt {
template struct AmrOps<float>;
template struct AmrOps<__half>;
template struct AmrOps<__nv_bfloat16>;
}
