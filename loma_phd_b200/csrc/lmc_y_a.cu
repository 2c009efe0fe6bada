// y-direction kernels for chunk sizes 4, 5 (see lmc_ykernels.cuh).
#include "lmc_ykernels.cuh"

namespace lmc {
template struct YL<4, double2>;
template struct YL<4, float2>;
template struct YL<5, double2>;
template struct YL<5, float2>;
}  // namespace lmc
