// lmb_dist_s.cu -- apply, timing and D^+D CG drivers of the sharded
// Wilson / Wilson-clover and staggered / HISQ operators with FP32 iterated
// fields (one precision per translation unit keeps the builds in parallel).
#include "lmb_op_dist.cuh"

namespace lmb {
LMB_OP_INSTANCE(, DistWilsonPolicy, PREC_SINGLE, PREC_SINGLE)
LMB_OP_INSTANCE(, DistStaggeredPolicy, PREC_SINGLE, PREC_SINGLE)
}  // namespace lmb
