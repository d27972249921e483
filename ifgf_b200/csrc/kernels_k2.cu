// Matvec kernels instantiated for one kernel plug-in (K_MODHELMHOLTZ).
#include "mult_kernels.cuh"

namespace ifgf
{
IFGF_INSTANTIATE_KIND(K_MODHELMHOLTZ)
} // namespace ifgf
