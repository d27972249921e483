// Matvec kernels instantiated for one kernel plug-in (K_DOUBLELAYER).
#include "mult_kernels.cuh"

namespace ifgf
{
IFGF_INSTANTIATE_KIND(K_DOUBLELAYER)
} // namespace ifgf
