// lmb_wilson_h.cu -- Wilson / Wilson-clover apply and D^+D CG drivers with
// int16 storage iterated fields (one precision per translation unit keeps the
// stencil instantiations of a build in parallel).
#include "lmb_op_wilson.cuh"

namespace lmb {
LMB_OP_INSTANCE(, WilsonPolicy, PREC_HALF, PREC_SINGLE)
}  // namespace lmb
