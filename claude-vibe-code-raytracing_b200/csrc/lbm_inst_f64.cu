// Kernel instantiation for population storage type double.
#include "lbm_ops.cuh"

namespace lbm {
OpsBase *make_ops_f64() {
  static Ops<double> ops;
  return &ops;
}
}  // namespace lbm
