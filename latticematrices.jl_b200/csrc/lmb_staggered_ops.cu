// lmb_staggered_ops.cu -- staggered / HISQ apply and D^+D CG drivers (FP64,
// FP32 and int16 storage).
#include "lmb_op_staggered.cuh"

namespace lmb {
LMB_OP_INSTANCES(, StaggeredPolicy)
}  // namespace lmb
