// Fixed device scratch for ifgf_mult_device_noalloc.
//
// Some callers cannot allocate device memory at the moment they apply the
// operator: solvers embedded in frameworks whose memory pool has reserved the
// whole device (a cudaMalloc there fails or takes memory the pool counts on),
// or real-time loops that must not stall on the implicit device
// synchronisation of cudaMalloc / cudaFree.  For them the matvec can run with
// its per-call scratch (sorted densities, coarse nodal values, fine
// coefficients, near-field sums) in the file-scope array below instead of the
// buffers the operator allocated at init.
//
// The array is NOALLOC_SCRATCH_BYTES (64 MiB) on every GPU that loads this
// library, held until the process exits.  Every call shares it and it keeps
// the last call's contents, so calls whose GPU work overlaps (two streams, two
// threads, two operators) race; serialise them.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "common.hpp"

namespace ifgf
{

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(64) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch on the current device.  The address is
// looked up once per device, with that device current, on the first call made
// on that device; make that first call before any stream capture begins.  In
// host code the symbol itself is only a host-side stand-in, never a device
// address, so kernels must receive the looked-up pointer.
void* noalloc_scratch(size_t* bytes)
{
    constexpr int MAX_DEVICES = 64;
    static std::mutex mu;
    static void* addr[MAX_DEVICES] = {};
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        throw Error(2, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= MAX_DEVICES)
        throw Error(1, "device ordinal out of range for the no-allocation scratch");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev])
    {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            throw Error(2, std::string("cudaGetSymbolAddress(no-allocation scratch): ") +
                               cudaGetErrorString(e));
        addr[dev] = p;
    }
    *bytes = NOALLOC_SCRATCH_BYTES;
    return addr[dev];
}

} // namespace ifgf
