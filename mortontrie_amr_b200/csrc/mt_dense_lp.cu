// Reduced-precision instantiations of the dense uniform path: FP32 arithmetic
// on populations stored as f - w_q in FP32, FP16 or BF16.
#include "mt_dense.cuh"

namespace mt {
template struct DenseOps<float>;
template struct DenseOps<__half>;
template struct DenseOps<__nv_bfloat16>;
}
