// Basis images of the tensor-core upward transfer (declared in mult.hpp,
// kernel uptc_image_kernel in upward_tc.cuh).
#include "mult_kernels.cuh"

namespace ifgf
{

namespace
{
template <int N0, int N1, int N2>
void image_pass(const int2* fe_list, int fe_pad, const UpGeo32* geo32, int up_pad, int nslots,
                const long long* off, unsigned char* img, long long* sizes, bool meta_only)
{
    const unsigned rows = (unsigned)nslots * 8u;
    if (rows == 0)
        return;
    uptc_image_kernel<N0, N1, N2><<<rows, 128>>>(fe_list, fe_pad, geo32, up_pad, off, img, sizes,
                                                 meta_only);
    IFGF_CHECK_LAUNCH();
    IFGF_CHECK(cudaDeviceSynchronize());
}

template <typename F> bool by_shape(const int* lo, F&& f)
{
    if (lo[0] == 2 && lo[1] == 5 && lo[2] == 5)
    {
        f(std::integral_constant<int, 2>{}, std::integral_constant<int, 5>{});
        return true;
    }
    if (lo[0] == 3 && lo[1] == 6 && lo[2] == 6)
    {
        f(std::integral_constant<int, 3>{}, std::integral_constant<int, 6>{});
        return true;
    }
    return false;
}
} // namespace

bool upward_tc_image_sizes(const int* lo, const int2* fe_list, int fe_pad, int up_pad, int nslots,
                           long long* d_sizes)
{
    return by_shape(lo, [&](auto a, auto b) {
        image_pass<decltype(a)::value, decltype(b)::value, decltype(b)::value>(
            fe_list, fe_pad, nullptr, up_pad, nslots, nullptr, nullptr, d_sizes, false);
    });
}

bool upward_tc_image_fill(const int* lo, const int2* fe_list, int fe_pad, const UpGeo32* geo32,
                          int up_pad, int nslots, const long long* d_off, unsigned char* img,
                          bool meta_only)
{
    return by_shape(lo, [&](auto a, auto b) {
        image_pass<decltype(a)::value, decltype(b)::value, decltype(b)::value>(
            fe_list, fe_pad, geo32, up_pad, nslots, d_off, img, nullptr, meta_only);
    });
}

} // namespace ifgf
