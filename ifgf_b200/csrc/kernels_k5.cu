// Matvec kernels instantiated for one kernel plug-in (K_COMBINEDFIELD).
#include "mult_kernels.cuh"

namespace ifgf
{
IFGF_INSTANTIATE_KIND(K_COMBINEDFIELD)
} // namespace ifgf
