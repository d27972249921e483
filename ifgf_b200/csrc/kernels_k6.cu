// Matvec kernels instantiated for one kernel plug-in (K_HELMHOLTZ_DK).
#include "mult_kernels.cuh"

namespace ifgf
{
IFGF_INSTANTIATE_KIND(K_HELMHOLTZ_DK)
} // namespace ifgf
