// y-direction kernels for chunk sizes 7, 9 (see lmc_ykernels.cuh).
#include "lmc_ykernels.cuh"

namespace lmc {
template struct YL<7, double2>;
template struct YL<7, float2>;
template struct YL<9, double2>;
template struct YL<9, float2>;
}  // namespace lmc
