// y-direction kernels for chunk sizes 13 (see lmc_ykernels.cuh).
#include "lmc_ykernels.cuh"

namespace lmc {
template struct YL<13, double2>;
template struct YL<13, float2>;
}  // namespace lmc
