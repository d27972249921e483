// Matvec kernels instantiated for one kernel plug-in (K_LAPLACE).
#include "mult_kernels.cuh"

namespace ifgf
{
IFGF_INSTANTIATE_KIND(K_LAPLACE)
} // namespace ifgf
