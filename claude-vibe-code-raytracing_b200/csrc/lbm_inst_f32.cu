// Kernel instantiation for population storage type float.
#include "lbm_ops.cuh"

namespace lbm {
OpsBase *make_ops_f32() {
  static Ops<float> ops;
  return &ops;
}
}  // namespace lbm
