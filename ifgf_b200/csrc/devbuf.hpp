// Owning device buffer and the CUDA status check shared by the host-side
// translation units that hold device tables.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "common.hpp"

namespace ifgf
{

// C-ABI status codes carried by Error
static constexpr int ERR_INVALID = 1, ERR_CUDA = 2, ERR_STATE = 3, ERR_OOM = 4, ERR_TIMEOUT = 5;

#define IFGF_CUDA(x)                                                                          \
    do                                                                                         \
    {                                                                                          \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            throw Error(ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));           \
    } while (0)

template <typename T> struct DevBuf
{
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n)
    {
        o.p = nullptr;
        o.n = 0;
    }
    DevBuf& operator=(DevBuf&& o) noexcept
    {
        if (this != &o)
        {
            release();
            p = o.p;
            n = o.n;
            o.p = nullptr;
            o.n = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t count)
    {
        release();
        if (count == 0)
            return;
        cudaError_t e = cudaMalloc((void**)&p, count * sizeof(T));
        if (e != cudaSuccess)
        {
            cudaGetLastError();
            p = nullptr;
            throw Error(ERR_OOM, "cudaMalloc(" + std::to_string(count * sizeof(T)) +
                                     " bytes) failed: " + cudaGetErrorString(e));
        }
        n = count;
    }
    void upload(const T* h, size_t count)
    {
        alloc(count);
        if (count)
            IFGF_CUDA(cudaMemcpy(p, h, count * sizeof(T), cudaMemcpyHostToDevice));
    }
    void upload(const std::vector<T>& v) { upload(v.data(), v.size()); }
    std::vector<T> download() const
    {
        std::vector<T> v(n);
        if (n)
            IFGF_CUDA(cudaMemcpy(v.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost));
        return v;
    }
    void zero()
    {
        if (n)
            IFGF_CUDA(cudaMemset(p, 0, n * sizeof(T)));
    }
    void release()
    {
        if (p)
            cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

} // namespace ifgf
