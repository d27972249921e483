// Device-side numerics of the IFGF matvec: complex arithmetic, interpolation
// coordinates, cone lookups, Chebyshev evaluation and the six kernel plug-ins.
#pragma once

#include <cuda_runtime.h>

#include "common.hpp"

namespace ifgf
{

template <typename R> struct cplx
{
    R re, im;
};

template <typename R> __device__ __forceinline__ cplx<R> cmake(R a, R b) { return {a, b}; }
template <typename R> __device__ __forceinline__ cplx<R> cadd(cplx<R> a, cplx<R> b)
{
    return {a.re + b.re, a.im + b.im};
}
template <typename R> __device__ __forceinline__ cplx<R> cmul(cplx<R> a, cplx<R> b)
{
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename R> __device__ __forceinline__ cplx<R> cscale(cplx<R> a, R s)
{
    return {a.re * s, a.im * s};
}
// acc += a * b
template <typename R> __device__ __forceinline__ void cfma(cplx<R>& acc, cplx<R> a, cplx<R> b)
{
    acc.re = fma(a.re, b.re, fma(-a.im, b.im, acc.re));
    acc.im = fma(a.re, b.im, fma(a.im, b.re, acc.im));
}

constexpr double INV4PI = 1.0 / (4.0 * 3.14159265358979323846);
constexpr double DPI = 3.14159265358979323846;

// Wavenumber and plug-in switches shared by all kernels of one operator.
struct KParams
{
    double kr, ki; // k = kr + i ki (real kernels use kr)
    int dx;        // GradHelmholtz derivative direction, -1 = plain single layer
};

// e^{-k d} for complex k: e^{-kr d} (cos(ki d), -sin(ki d))
__device__ __forceinline__ cplx<double> exp_mk(const KParams& p, double d)
{
    double s, c;
    sincos(-p.ki * d, &s, &c);
    const double m = exp(-p.kr * d);
    return {m * c, m * s};
}
// e^{i k d} for real k
__device__ __forceinline__ cplx<double> exp_ik(double k, double d)
{
    double s, c;
    sincos(k * d, &s, &c);
    return {c, s};
}

// ---------------------------------------------------------------------------
// Interpolation coordinates (util.hpp:96-116, 156-171)
// ---------------------------------------------------------------------------
// (s, theta, phi) of x relative to the centre xc of a box of side H.  Angles
// are clamped into [0, pi] / [-pi, pi], the range of the C library's atan2,
// so that a device atan2 rounding past +-pi cannot push a point out of the
// interpolation domain.
__device__ __forceinline__ void cart_to_interp(double p0, double p1, double p2, double H,
                                               double* s)
{
    const double a = p0 * p0 + p1 * p1;
    s[2] = fmin(fmax(atan2(p1, p0), -DPI), DPI);
    s[1] = fmin(fmax(atan2(sqrt(a), p2), 0.0), DPI);
    s[0] = H / sqrt(a + p2 * p2);
}

__device__ __forceinline__ void interp_to_cart(const double* s, const double* xc, double H,
                                               double* x)
{
    const double r = H / s[0];
    double st, ct, sp, cp;
    sincos(s[1], &st, &ct);
    sincos(s[2], &sp, &cp);
    x[0] = xc[0] + r * cp * st;
    x[1] = xc[1] + r * sp * st;
    x[2] = xc[2] + r * ct;
}

// ConeDomain::elementForPoint (cone_domain.hpp:232-256): element id or -1
// when the point lies outside the interpolation domain.
__device__ __forceinline__ int element_for_point(const double* s, const double* dmin,
                                                 const double* dmax, const double* h,
                                                 const int* n)
{
    double d2 = 0;
#pragma unroll
    for (int k = 0; k < 3; k++)
    {
        if (dmin[k] > s[k])
        {
            const double a = dmin[k] - s[k];
            d2 += a * a;
        }
        else if (s[k] > dmax[k])
        {
            const double a = s[k] - dmax[k];
            d2 += a * a;
        }
    }
    if (d2 > 0)
        return -1;
    int id = 0, stride = 1;
#pragma unroll
    for (int j = 0; j < 3; j++)
    {
        int q = (int)floor((s[j] - dmin[j]) / h[j]);
        q = min(max(q, 0), n[j] - 1);
        id += q * stride;
        stride *= n[j];
    }
    return id;
}

// ConeDomain::transformBackwards (cone_domain.hpp:173-184)
__device__ __forceinline__ void to_local(int el, const double* s, const double* dmin,
                                         const double* h, const int* n, double* loc)
{
    int i0 = el % n[0];
    int r = el / n[0];
    int i1 = r % n[1];
    int i2 = r / n[1];
    const int idx[3] = {i0, i1, i2};
#pragma unroll
    for (int d = 0; d < 3; d++)
    {
        const double a = 0.5 * h[d];
        const double b = dmin[d] + ((double)idx[d] + 0.5) * h[d];
        loc[d] = (s[d] - b) / a;
    }
}

// ConeDomain::transform (cone_domain.hpp:145-158)
__device__ __forceinline__ void from_local(int el, const double* loc, const double* dmin,
                                           const double* h, const int* n, double* s)
{
    int i0 = el % n[0];
    int r = el / n[0];
    int i1 = r % n[1];
    int i2 = r / n[1];
    const int idx[3] = {i0, i1, i2};
#pragma unroll
    for (int d = 0; d < 3; d++)
    {
        const double a = 0.5 * h[d];
        const double b = dmin[d] + ((double)idx[d] + 0.5) * h[d];
        s[d] = loc[d] * a + b;
    }
}

// Tensor-product Chebyshev series sum_{ijk} c[i + n0 (j + n1 k)] T_i(x0)
// T_j(x1) T_k(x2) (the function ClenshawEvaluator computes,
// chebinterp.hpp:252-346), with T evaluated by the three-term recurrence.
template <int MAXN>
__device__ __forceinline__ cplx<double> cheb_eval3(const double2* __restrict__ c,
                                                   const double* x, const int* n)
{
    double t0[MAXN], t1[MAXN], t2[MAXN];
    const double* xs[3] = {x, x + 1, x + 2};
    double* ts[3] = {t0, t1, t2};
#pragma unroll
    for (int d = 0; d < 3; d++)
    {
        double* t = ts[d];
        const double xv = *xs[d];
        t[0] = 1.0;
        if (n[d] > 1)
            t[1] = xv;
        for (int i = 2; i < n[d]; i++)
            t[i] = 2.0 * xv * t[i - 1] - t[i - 2];
    }
    double ar = 0, ai = 0;
    int q = 0;
    for (int k = 0; k < n[2]; k++)
    {
        double br = 0, bi = 0;
        for (int j = 0; j < n[1]; j++)
        {
            double cr = 0, ci = 0;
            for (int i = 0; i < n[0]; i++, q++)
            {
                const double2 v = __ldg(c + q);
                cr = fma(v.x, t0[i], cr);
                ci = fma(v.y, t0[i], ci);
            }
            br = fma(cr, t1[j], br);
            bi = fma(ci, t1[j], bi);
        }
        ar = fma(br, t2[k], ar);
        ai = fma(bi, t2[k], ai);
    }
    return {ar, ai};
}

// ---------------------------------------------------------------------------
// Kernel plug-ins.  x = x_src - y_tgt throughout, as in the reference's
// evaluateKernel loops (e.g. helmholtz_ifgf.hpp:104-111).
// ---------------------------------------------------------------------------
template <int KIND> struct Plugin;

// laplace_ifgf.hpp
template <> struct Plugin<K_LAPLACE>
{
    static constexpr bool needs_normals = false;
    __device__ static cplx<double> kernel(const double* x, const double*, const KParams&)
    {
        const double d = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        return {(d == 0) ? 0.0 : INV4PI / d, 0.0};
    }
    __device__ static cplx<double> cf(const double* x, const KParams&)
    {
        const double d2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        return {(1.0 / sqrt(d2)) * INV4PI, 0.0};
    }
    __device__ static cplx<double> transfer(double d2, double dp2, const KParams&)
    {
        return {sqrt(dp2) / sqrt(d2), 0.0};
    }
    // w * G(y, x)/G(y, xc) with a = x - y
    __device__ static cplx<double> factored(const double* a, const double*, cplx<double> w,
                                            const double*, double dc, const KParams&)
    {
        const double d = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        return {(d == 0) ? 0.0 : w.re * dc / d, 0.0};
    }
};

// helmholtz_ifgf.hpp (real k)
template <> struct Plugin<K_HELMHOLTZ>
{
    static constexpr bool needs_normals = false;
    __device__ static cplx<double> kernel(const double* x, const double*, const KParams& p)
    {
        const double d = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        if (d == 0)
            return {0.0, 0.0};
        const cplx<double> e = exp_ik(p.kr, d);
        const double f = INV4PI / d;
        return {e.re * f, e.im * f};
    }
    __device__ static cplx<double> cf(const double* x, const KParams& p)
    {
        const double d2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        const double id = 1.0 / sqrt(d2);
        const double d = d2 * id;
        return cscale(exp_ik(p.kr, d), id * INV4PI);
    }
    __device__ static cplx<double> transfer(double d2, double dp2, const KParams& p)
    {
        const double d = sqrt(d2), dp = sqrt(dp2);
        return cscale(exp_ik(p.kr, d - dp), dp / d);
    }
    __device__ static cplx<double> factored(const double* a, const double*, cplx<double> w,
                                            const double*, double dc, const KParams& p)
    {
        const double d = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        return cmul(w, cscale(exp_ik(p.kr, d - dc), dc / d));
    }
};

// modified_helmholtz_ifgf.hpp (complex k, kernel e^{-kd}/(4 pi d))
template <> struct Plugin<K_MODHELMHOLTZ>
{
    static constexpr bool needs_normals = false;
    __device__ static cplx<double> kernel(const double* x, const double*, const KParams& p)
    {
        const double d = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        if (d == 0)
            return {0.0, 0.0};
        return cscale(exp_mk(p, d), INV4PI / d);
    }
    __device__ static cplx<double> cf(const double* x, const KParams& p)
    {
        const double d2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        const double id = 1.0 / sqrt(d2);
        return cscale(exp_mk(p, d2 * id), id * INV4PI);
    }
    __device__ static cplx<double> transfer(double d2, double dp2, const KParams& p)
    {
        const double d = sqrt(d2), dp = sqrt(dp2);
        return cscale(exp_mk(p, d - dp), dp / d);
    }
    __device__ static cplx<double> factored(const double* a, const double*, cplx<double> w,
                                            const double*, double dc, const KParams& p)
    {
        const double d = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        if (d == 0)
            return {0.0, 0.0};
        return cmul(w, cscale(exp_mk(p, d - dc), dc / d));
    }
};

// grad_helmholtz_ifgf.hpp (complex k, derivative along dx, or plain if -1)
template <> struct Plugin<K_GRADHELMHOLTZ>
{
    static constexpr bool needs_normals = false;
    __device__ static cplx<double> kernel(const double* x, const double*, const KParams& p)
    {
        const double d = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        if (d < 1e-12)
            return {0.0, 0.0};
        const cplx<double> e = exp_mk(p, d);
        if (p.dx < 0)
            return cscale(e, INV4PI / d);
        // -(1/4pi) (1/d^2) e^{-kd} (-k - 1/d) x[dx]
        const cplx<double> m = {-p.kr - 1.0 / d, -p.ki};
        return cscale(cmul(e, m), -INV4PI * (1.0 / (d * d)) * x[p.dx]);
    }
    __device__ static cplx<double> cf(const double* x, const KParams& p)
    {
        const double d2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        const double id = 1.0 / sqrt(d2);
        return cscale(exp_mk(p, d2 * id), id * INV4PI);
    }
    __device__ static cplx<double> transfer(double d2, double dp2, const KParams& p)
    {
        const double invd = d2 > 1e-12 ? 1.0 / sqrt(d2) : 0.0;
        const double dp = sqrt(dp2), d = d2 * invd;
        return cscale(exp_mk(p, d - dp), dp * invd);
    }
    __device__ static cplx<double> factored(const double* a, const double*, cplx<double> w,
                                            const double*, double dc, const KParams& p)
    {
        const double d2 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
        const double id = d2 > 1e-12 ? 1.0 / sqrt(d2) : 0.0;
        const double d = d2 * id;
        const cplx<double> e = cmul(w, exp_mk(p, d - dc));
        if (p.dx < 0)
            return cscale(e, dc * id);
        const double ww = -(1.0 / d2) * dc * a[p.dx];
        const cplx<double> m = {-p.kr - id, -p.ki};
        return cscale(cmul(e, m), ww);
    }
};

// double_layer_helmholtz_ifgf.hpp (complex k, source normals)
template <> struct Plugin<K_DOUBLELAYER>
{
    static constexpr bool needs_normals = true;
    __device__ static cplx<double> kernel(const double* x, const double* n, const KParams& p)
    {
        const double d = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        if (d < 1e-12)
            return {0.0, 0.0};
        const double xn = x[0] * n[0] + x[1] * n[1] + x[2] * n[2];
        const cplx<double> m = {-p.kr - 1.0 / d, -p.ki};
        return cscale(cmul(exp_mk(p, d), m), -INV4PI * (1.0 / (d * d)) * xn);
    }
    __device__ static cplx<double> cf(const double* x, const KParams& p)
    {
        const double d2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        const double id = 1.0 / sqrt(d2);
        return cscale(exp_mk(p, d2 * id), id * INV4PI);
    }
    __device__ static cplx<double> transfer(double d2, double dp2, const KParams& p)
    {
        const double invd = 1.0 / sqrt(d2);
        const double dp = sqrt(dp2), d = d2 * invd;
        return cscale(exp_mk(p, d - dp), dp * invd);
    }
    __device__ static cplx<double> factored(const double* a, const double* n, cplx<double> w,
                                            const double*, double dc, const KParams& p)
    {
        const double d2 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
        const double id = d2 > 1e-12 ? 1.0 / sqrt(d2) : 0.0;
        const double d = d2 * id;
        const double ww = -(1.0 / d2) * dc * (a[0] * n[0] + a[1] * n[1] + a[2] * n[2]);
        const cplx<double> m = {-p.kr - id, -p.ki};
        return cscale(cmul(cmul(w, exp_mk(p, d - dc)), m), ww);
    }
};

// combined_field_helmholtz_ifgf.hpp (real kappa, source normals)
template <> struct Plugin<K_COMBINEDFIELD>
{
    static constexpr bool needs_normals = true;
    __device__ static cplx<double> kernel(const double* x, const double* n, const KParams& p)
    {
        const double kap = p.kr;
        const double d2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        const double invd = d2 < 1e-14 ? 0.0 : 1.0 / sqrt(d2);
        const double d = d2 * invd;
        const double nxy = -(n[0] * x[0] + n[1] * x[1] + n[2] * x[2]);
        double s, c;
        sincos(kap * d, &s, &c);
        const double f = INV4PI * invd * invd * invd;
        return {f * (c * nxy + s * kap * (d * nxy + d2)), f * (-c * kap * (d * nxy + d2) + s * nxy)};
    }
    __device__ static cplx<double> cf(const double* x, const KParams& p)
    {
        const double d2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        const double id = 1.0 / sqrt(d2);
        return cscale(exp_ik(p.kr, d2 * id), id * INV4PI);
    }
    __device__ static cplx<double> transfer(double d2, double dp2, const KParams& p)
    {
        const double invd = 1.0 / sqrt(d2);
        const double dp = sqrt(dp2), d = d2 * invd;
        return cscale(exp_ik(p.kr, d - dp), dp * invd);
    }
    __device__ static cplx<double> factored(const double* a, const double* n, cplx<double> w,
                                            const double*, double dc, const KParams& p)
    {
        // z = y - x = -a
        const double d2 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
        if (!(d2 > 1e-14))
            return {0.0, 0.0};
        const double kap = p.kr;
        const double nxy = -(a[0] * n[0] + a[1] * n[1] + a[2] * n[2]);
        const double id = 1.0 / sqrt(d2);
        const double d = d2 * id;
        double s, c;
        sincos(kap * (d - dc), &s, &c);
        const double f = dc / (d2 * d);
        const double A = w.re * c - w.im * s, B = w.re * s + w.im * c;
        return {f * (A * nxy + B * kap * (d * nxy + d2)), f * (-A * kap * (d * nxy + d2) + B * nxy)};
    }
};

} // namespace ifgf
