// Kernel instantiation for population storage type __half.
#include "lbm_ops.cuh"

namespace lbm {
OpsBase *make_ops_f16() {
  static Ops<__half> ops;
  return &ops;
}
}  // namespace lbm
