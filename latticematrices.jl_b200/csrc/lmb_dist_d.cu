// lmb_dist_d.cu -- apply, timing and D^+D CG drivers of the sharded
// Wilson / Wilson-clover and staggered / HISQ operators with FP64 iterated
// fields (one precision per translation unit keeps the builds in parallel).
#include "lmb_op_dist.cuh"

namespace lmb {
LMB_OP_INSTANCE(, DistWilsonPolicy, PREC_DOUBLE, PREC_DOUBLE)
LMB_OP_INSTANCE(, DistStaggeredPolicy, PREC_DOUBLE, PREC_DOUBLE)
}  // namespace lmb
