// lmb_dw_ops.cu -- domain-wall (5D) apply and D5^+D5 CG drivers (FP64, FP32
// and int16 storage).
#include "lmb_op_dw.cuh"

namespace lmb {
LMB_OP_INSTANCES(, DWPolicy)
}  // namespace lmb
