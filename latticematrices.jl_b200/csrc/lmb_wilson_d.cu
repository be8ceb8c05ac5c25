// lmb_wilson_d.cu -- Wilson / Wilson-clover apply and D^+D CG drivers with
// FP64 iterated fields (one precision per translation unit keeps the
// stencil instantiations of a build in parallel).
#include "lmb_op_wilson.cuh"

namespace lmb {
LMB_OP_INSTANCE(, WilsonPolicy, PREC_DOUBLE, PREC_DOUBLE)
}  // namespace lmb
