// y-direction kernels for chunk sizes 17 (see lmc_ykernels.cuh).
#include "lmc_ykernels.cuh"

namespace lmc {
template struct YL<17, double2>;
template struct YL<17, float2>;
}  // namespace lmc
