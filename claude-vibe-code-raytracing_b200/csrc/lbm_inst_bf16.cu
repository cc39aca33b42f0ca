// Kernel instantiation for population storage type __nv_bfloat16.
#include "lbm_ops.cuh"

namespace lbm {
OpsBase *make_ops_bf16() {
  static Ops<__nv_bfloat16> ops;
  return &ops;
}
}  // namespace lbm
