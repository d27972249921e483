// Matvec kernels instantiated for one kernel plug-in (K_COMBINEDFIELD_DK).
#include "mult_kernels.cuh"

namespace ifgf
{
IFGF_INSTANTIATE_KIND(K_COMBINEDFIELD_DK)
} // namespace ifgf
