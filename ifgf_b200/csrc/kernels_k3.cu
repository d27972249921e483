// Matvec kernels instantiated for one kernel plug-in (K_GRADHELMHOLTZ).
#include "mult_kernels.cuh"

namespace ifgf
{
IFGF_INSTANTIATE_KIND(K_GRADHELMHOLTZ)
} // namespace ifgf
