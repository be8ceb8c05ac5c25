// lmb_wilson_s.cu -- Wilson / Wilson-clover apply and D^+D CG drivers with
// FP32 storage iterated fields (one precision per translation unit keeps the
// stencil instantiations of a build in parallel).
#include "lmb_op_wilson.cuh"

namespace lmb {
LMB_OP_INSTANCE(, WilsonPolicy, PREC_SINGLE, PREC_SINGLE)
}  // namespace lmb
