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
    // kr and ki split into two floats each (hi + lo), for the mixed pipeline
    float krh, krl, kih, kil;
};

inline KParams make_kparams(double kr, double ki, int dx)
{
    KParams p;
    p.kr = kr;
    p.ki = ki;
    p.dx = dx;
    p.krh = (float)kr;
    p.krl = (float)(kr - (double)p.krh);
    p.kih = (float)ki;
    p.kil = (float)(ki - (double)p.kih);
    return p;
}

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
// when the point lies outside the interpolation domain.  hinv = 1 / width:
// floor((s - min) * hinv) equals the reference's floor((s - min) / h) except
// within one rounding of an element boundary.
__device__ __forceinline__ int element_for_point(const double* s, const double* dmin,
                                                 const double* dmax, const double* hinv,
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
        int q = (int)floor((s[j] - dmin[j]) * hinv[j]);
        q = min(max(q, 0), n[j] - 1);
        id += q * stride;
        stride *= n[j];
    }
    return id;
}

// ConeDomain::transformBackwards (cone_domain.hpp:173-184), with the division
// by the half width replaced by a multiplication with 2 / width
__device__ __forceinline__ void to_local(int el, const double* s, const double* dmin,
                                         const double* h, const double* hinv, const int* n,
                                         double* loc)
{
    int i0 = el % n[0];
    int r = el / n[0];
    int i1 = r % n[1];
    int i2 = r / n[1];
    const int idx[3] = {i0, i1, i2};
#pragma unroll
    for (int d = 0; d < 3; d++)
    {
        const double a2 = 2.0 * hinv[d]; // 1 / (h / 2)
        const double b = dmin[d] + ((double)idx[d] + 0.5) * h[d];
        loc[d] = (s[d] - b) * a2;
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

// d/dk of the Helmholtz kernel, i e^{ikr} / (4 pi).  Centred factor
// e^{ik r_c} / (4 pi) (no 1/r_c: the factored kernel i e^{ik(r - r_c)} is then
// as smooth in the cone coordinates as the Helmholtz one), centre shift
// e^{ik(r - r_p)}.
template <> struct Plugin<K_HELMHOLTZ_DK>
{
    static constexpr bool needs_normals = false;
    __device__ static cplx<double> kernel(const double* x, const double*, const KParams& p)
    {
        const double d = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        if (d == 0)
            return {0.0, 0.0};
        const cplx<double> e = exp_ik(p.kr, d);
        return {-e.im * INV4PI, e.re * INV4PI};
    }
    __device__ static cplx<double> cf(const double* x, const KParams& p)
    {
        const double d = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        return cscale(exp_ik(p.kr, d), INV4PI);
    }
    __device__ static cplx<double> transfer(double d2, double dp2, const KParams& p)
    {
        return exp_ik(p.kr, sqrt(d2) - sqrt(dp2));
    }
    __device__ static cplx<double> factored(const double* a, const double*, cplx<double> w,
                                            const double*, double dc, const KParams& p)
    {
        const double d = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        const cplx<double> v = cmul(w, exp_ik(p.kr, d - dc));
        return {-v.im, v.re};
    }
};

// d/dkappa of the combined-field kernel e^{i kap d} / (4 pi d^3)
// (nxy (1 - i kap d) - i kap d^2):  e^{i kap d} / (4 pi d) (kap (nxy + d) - i),
// nxy = -n . x.  Centred factor and centre shift as for K_HELMHOLTZ_DK.
template <> struct Plugin<K_COMBINEDFIELD_DK>
{
    static constexpr bool needs_normals = true;
    __device__ static cplx<double> kernel(const double* x, const double* n, const KParams& p)
    {
        const double kap = p.kr;
        const double d2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        if (d2 < 1e-14)
            return {0.0, 0.0};
        const double invd = 1.0 / sqrt(d2);
        const double d = d2 * invd;
        const double nxy = -(n[0] * x[0] + n[1] * x[1] + n[2] * x[2]);
        const cplx<double> e = exp_ik(kap, d);
        const double f = INV4PI * invd;
        const double g = kap * (nxy + d); // (g - i) e
        return {f * (g * e.re + e.im), f * (g * e.im - e.re)};
    }
    __device__ static cplx<double> cf(const double* x, const KParams& p)
    {
        const double d = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        return cscale(exp_ik(p.kr, d), INV4PI);
    }
    __device__ static cplx<double> transfer(double d2, double dp2, const KParams& p)
    {
        return exp_ik(p.kr, sqrt(d2) - sqrt(dp2));
    }
    __device__ static cplx<double> factored(const double* a, const double* n, cplx<double> w,
                                            const double*, double dc, const KParams& p)
    {
        const double d2 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
        if (!(d2 > 1e-14))
            return {0.0, 0.0};
        const double kap = p.kr;
        const double nxy = -(a[0] * n[0] + a[1] * n[1] + a[2] * n[2]);
        const double invd = 1.0 / sqrt(d2);
        const double d = d2 * invd;
        const cplx<double> v = cmul(w, exp_ik(kap, d - dc));
        const double g = kap * (nxy + d);
        return {invd * (g * v.re + v.im), invd * (g * v.im - v.re)};
    }
};

// ===========================================================================
// Mixed precision: FP32 arithmetic on coordinates relative to a nearby box
// centre, with the phase k*r formed and reduced modulo 2 pi in FP64 and the
// reduced angle (|r| <= pi) fed to the FP32 sine/cosine unit.
// ===========================================================================
constexpr float INV4PIF = (float)INV4PI;

// (cos(k r), sin(k r)) with k r and its reduction in FP64
__device__ __forceinline__ cplx<float> phase_sc(double k, double r)
{
    const double th = k * r;
    const double n = rint(th * (1.0 / (2.0 * DPI)));
    const float red = (float)fma(-n, 2.0 * DPI, th);
    float s, c;
    __sincosf(red, &s, &c);
    return {c, s};
}

// (cos(k r), sin(k r)) for an FP32 distance r, with k r formed and reduced
// modulo 2 pi in double-float arithmetic: k = kh + kl (two floats, made on the
// host), the product k r as an unevaluated float pair (exact through FMA) and
// 2 pi as a three-float sum (Cody-Waite), so the reduced angle carries the
// accuracy of an FP64 reduction without leaving the FP32 pipes.
__device__ __forceinline__ cplx<float> phase_sc_ff(float kh, float kl, float r)
{
    const float th = kh * r;
    const float tl = fmaf(kh, r, -th) + kl * r;
    constexpr float C1 = 6.2831854820251465f;      // float(2 pi)
    constexpr float C2 = -1.7484555314695172e-07f; // float(2 pi - C1)
    constexpr float C3 = -6.8604980400235275e-15f; // float(2 pi - C1 - C2)
    const float n = rintf(th * 0.15915493667125702f);
    float red = fmaf(-n, C1, th);
    red = fmaf(-n, C2, red);
    red = fmaf(-n, C3, red) + tl;
    float s, c;
    __sincosf(red, &s, &c);
    return {c, s};
}

// e^{-k r} for complex k (FP64 distance): e^{-kr r} (cos(ki r), -sin(ki r))
__device__ __forceinline__ cplx<float> exp_mk_f(const KParams& p, double r)
{
    const cplx<float> e = phase_sc(-p.ki, r);
    const float m = __expf((float)(-p.kr * r));
    return {m * e.re, m * e.im};
}
__device__ __forceinline__ cplx<float> exp_ik_f(double k, double r) { return phase_sc(k, r); }

// the same for an FP32 distance (double-float phase)
__device__ __forceinline__ cplx<float> exp_ik_ff(const KParams& p, float r)
{
    return phase_sc_ff(p.krh, p.krl, r);
}
__device__ __forceinline__ cplx<float> exp_mk_ff(const KParams& p, float r)
{
    const cplx<float> e = phase_sc_ff(-p.kih, -p.kil, r);
    const float m = __expf(-p.krh * r);
    return {m * e.re, m * e.im};
}

template <typename R> __device__ __forceinline__ void cfmaf(cplx<R>& acc, cplx<R> a, cplx<R> b)
{
    acc.re = fmaf(a.re, b.re, fmaf(-a.im, b.im, acc.re));
    acc.im = fmaf(a.re, b.im, fmaf(a.im, b.re, acc.im));
}

template <int KIND> struct PluginF;

// Near field: kernel(x, n) with x = x_src - y_tgt in FP32.  Kernels with
// normals take x and n in FP64 (kernel_d): for neighbouring points of a
// surface x.n is O(|x|^2) and would cancel in FP32, so x.n and |x|^2 are
// formed in FP64 and only the rest in FP32.
//
// Leaf sampling: factored(a, aa, b, n, w, dc) = w G(y, x)/G(y, xc) with
// a = x - xc, aa = |a|^2, b = y - xc (FP32) and dc = |b|; the difference
// d - dc is formed as (aa - 2 a.b) / (d + dc), free of cancellation.
__device__ __forceinline__ void factored_geom(const float* a, float aa, const float* b, float dc,
                                              float& inv, float& d, float& dd, float& d2)
{
    const float v0 = a[0] - b[0], v1 = a[1] - b[1], v2 = a[2] - b[2];
    d2 = v0 * v0 + v1 * v1 + v2 * v2;
    inv = rsqrtf(d2);
    d = d2 * inv;
    const float ab = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    dd = __fdividef(fmaf(-2.f, ab, aa), d + dc);
}

template <> struct PluginF<K_LAPLACE>
{
    static constexpr bool needs_normals = false;
    __device__ static cplx<float> kernel(const float* x, const float*, const KParams&)
    {
        const float d2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        return {d2 == 0.f ? 0.f : INV4PIF * rsqrtf(d2), 0.f};
    }
    __device__ static cplx<float> factored(const float* a, float, const float* b, const float*,
                                           cplx<float> w, float dc, const KParams&)
    {
        const float v0 = a[0] - b[0], v1 = a[1] - b[1], v2 = a[2] - b[2];
        const float d2 = v0 * v0 + v1 * v1 + v2 * v2;
        return {d2 == 0.f ? 0.f : w.re * dc * rsqrtf(d2), 0.f};
    }
};

template <> struct PluginF<K_HELMHOLTZ>
{
    static constexpr bool needs_normals = false;
    __device__ static cplx<float> kernel(const float* x, const float*, const KParams& p)
    {
        const float d2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        if (d2 == 0.f)
            return {0.f, 0.f};
        const float inv = rsqrtf(d2);
        const cplx<float> e = exp_ik_ff(p, d2 * inv);
        const float f = inv * INV4PIF;
        return {e.re * f, e.im * f};
    }
    __device__ static cplx<float> factored(const float* a, float aa, const float* b, const float*,
                                           cplx<float> w, float dc, const KParams& p)
    {
        float inv, d, dd, d2;
        factored_geom(a, aa, b, dc, inv, d, dd, d2);
        const cplx<float> e = exp_ik_ff(p, dd);
        const float f = dc * inv;
        return {f * (w.re * e.re - w.im * e.im), f * (w.re * e.im + w.im * e.re)};
    }
};

template <> struct PluginF<K_MODHELMHOLTZ>
{
    static constexpr bool needs_normals = false;
    __device__ static cplx<float> kernel(const float* x, const float*, const KParams& p)
    {
        const float d2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        if (d2 == 0.f)
            return {0.f, 0.f};
        const float inv = rsqrtf(d2);
        const cplx<float> e = exp_mk_ff(p, d2 * inv);
        const float f = inv * INV4PIF;
        return {e.re * f, e.im * f};
    }
    __device__ static cplx<float> factored(const float* a, float aa, const float* b, const float*,
                                           cplx<float> w, float dc, const KParams& p)
    {
        float inv, d, dd, d2;
        factored_geom(a, aa, b, dc, inv, d, dd, d2);
        if (d2 == 0.f)
            return {0.f, 0.f};
        const cplx<float> e = exp_mk_ff(p, dd);
        const float f = dc * inv;
        return {f * (w.re * e.re - w.im * e.im), f * (w.re * e.im + w.im * e.re)};
    }
};

template <> struct PluginF<K_GRADHELMHOLTZ>
{
    static constexpr bool needs_normals = false;
    __device__ static cplx<float> kernel(const float* x, const float*, const KParams& p)
    {
        const float d2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        if (!(d2 >= 1e-24f))
            return {0.f, 0.f};
        const float inv = rsqrtf(d2), d = d2 * inv;
        const cplx<float> e = exp_mk_ff(p, d);
        if (p.dx < 0)
            return {e.re * inv * INV4PIF, e.im * inv * INV4PIF};
        // -(1/4pi) (1/d^2) e^{-kd} (-k - 1/d) x[dx]
        const float mr = -p.krh - inv, mi = -p.kih;
        const float s = -INV4PIF * inv * inv * x[p.dx];
        return {s * (e.re * mr - e.im * mi), s * (e.re * mi + e.im * mr)};
    }
    __device__ static cplx<float> factored(const float* a, float aa, const float* b, const float*,
                                           cplx<float> w, float dc, const KParams& p)
    {
        float inv, d, dd, d2;
        factored_geom(a, aa, b, dc, inv, d, dd, d2);
        if (!(d2 > 1e-12f))
            inv = 0.f;
        const cplx<float> e = exp_mk_ff(p, dd);
        const cplx<float> we = {w.re * e.re - w.im * e.im, w.re * e.im + w.im * e.re};
        if (p.dx < 0)
            return {we.re * dc * inv, we.im * dc * inv};
        const float ww = -(inv * inv) * dc * (a[p.dx] - b[p.dx]);
        const float mr = -p.krh - inv, mi = -p.kih;
        return {ww * (we.re * mr - we.im * mi), ww * (we.re * mi + we.im * mr)};
    }
};

template <> struct PluginF<K_DOUBLELAYER>
{
    static constexpr bool needs_normals = true;
    __device__ static cplx<float> kernel_d(const double* x, const double* n, const KParams& p)
    {
        const double d2d = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        if (!(d2d >= 1e-24))
            return {0.f, 0.f};
        const float xn = (float)(x[0] * n[0] + x[1] * n[1] + x[2] * n[2]);
        const float d2 = (float)d2d;
        const float inv = rsqrtf(d2), d = d2 * inv;
        const cplx<float> e = exp_mk_ff(p, d);
        const float mr = -p.krh - inv, mi = -p.kih;
        const float s = -INV4PIF * inv * inv * xn;
        return {s * (e.re * mr - e.im * mi), s * (e.re * mi + e.im * mr)};
    }
    __device__ static cplx<float> factored(const float* a, float aa, const float* b, const float* n,
                                           cplx<float> w, float dc, const KParams& p)
    {
        float inv, d, dd, d2;
        factored_geom(a, aa, b, dc, inv, d, dd, d2);
        if (!(d2 > 1e-12f))
            inv = 0.f;
        const float an = (a[0] - b[0]) * n[0] + (a[1] - b[1]) * n[1] + (a[2] - b[2]) * n[2];
        const float ww = -(inv * inv) * dc * an;
        const cplx<float> e = exp_mk_ff(p, dd);
        const cplx<float> we = {w.re * e.re - w.im * e.im, w.re * e.im + w.im * e.re};
        const float mr = -p.krh - inv, mi = -p.kih;
        return {ww * (we.re * mr - we.im * mi), ww * (we.re * mi + we.im * mr)};
    }
};

template <> struct PluginF<K_COMBINEDFIELD>
{
    static constexpr bool needs_normals = true;
    __device__ static cplx<float> kernel_d(const double* x, const double* n, const KParams& p)
    {
        const double d2d = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        if (!(d2d >= 1e-14))
            return {0.f, 0.f};
        const float kap = p.krh;
        const float nxy = (float)-(n[0] * x[0] + n[1] * x[1] + n[2] * x[2]);
        const float d2 = (float)d2d;
        const float inv = rsqrtf(d2), d = d2 * inv;
        const cplx<float> e = exp_ik_ff(p, d);
        const float f = INV4PIF * inv * inv * inv;
        return {f * (e.re * nxy + e.im * kap * (d * nxy + d2)),
                f * (-e.re * kap * (d * nxy + d2) + e.im * nxy)};
    }
    __device__ static cplx<float> factored(const float* a, float aa, const float* b, const float* n,
                                           cplx<float> w, float dc, const KParams& p)
    {
        float inv, d, dd, d2;
        factored_geom(a, aa, b, dc, inv, d, dd, d2);
        if (!(d2 > 1e-14f))
            return {0.f, 0.f};
        const float kap = p.krh;
        // z = y - x = b - a
        const float nxy = (b[0] - a[0]) * n[0] + (b[1] - a[1]) * n[1] + (b[2] - a[2]) * n[2];
        const cplx<float> e = exp_ik_ff(p, dd);
        const float f = dc * inv * inv * inv;
        const float A = w.re * e.re - w.im * e.im, B = w.re * e.im + w.im * e.re;
        return {f * (A * nxy + B * kap * (d * nxy + d2)), f * (-A * kap * (d * nxy + d2) + B * nxy)};
    }
};

template <> struct PluginF<K_HELMHOLTZ_DK>
{
    static constexpr bool needs_normals = false;
    __device__ static cplx<float> kernel(const float* x, const float*, const KParams& p)
    {
        const float d2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        if (d2 == 0.f)
            return {0.f, 0.f};
        const cplx<float> e = exp_ik_ff(p, d2 * rsqrtf(d2));
        return {-e.im * INV4PIF, e.re * INV4PIF};
    }
    __device__ static cplx<float> factored(const float* a, float aa, const float* b, const float*,
                                           cplx<float> w, float dc, const KParams& p)
    {
        float inv, d, dd, d2;
        factored_geom(a, aa, b, dc, inv, d, dd, d2);
        const cplx<float> e = exp_ik_ff(p, dd);
        return {-(w.re * e.im + w.im * e.re), w.re * e.re - w.im * e.im};
    }
};
template <> struct PluginF<K_COMBINEDFIELD_DK>
{
    static constexpr bool needs_normals = true;
    __device__ static cplx<float> kernel_d(const double* x, const double* n, const KParams& p)
    {
        const double d2d = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        if (!(d2d >= 1e-14))
            return {0.f, 0.f};
        const float kap = p.krh;
        const float nxy = (float)-(n[0] * x[0] + n[1] * x[1] + n[2] * x[2]);
        const float d2 = (float)d2d;
        const float inv = rsqrtf(d2), d = d2 * inv;
        const cplx<float> e = exp_ik_ff(p, d);
        const float f = INV4PIF * inv, g = kap * (nxy + d);
        return {f * (g * e.re + e.im), f * (g * e.im - e.re)};
    }
    __device__ static cplx<float> factored(const float* a, float aa, const float* b, const float* n,
                                           cplx<float> w, float dc, const KParams& p)
    {
        float inv, d, dd, d2;
        factored_geom(a, aa, b, dc, inv, d, dd, d2);
        if (!(d2 > 1e-14f))
            return {0.f, 0.f};
        const float kap = p.krh;
        // z = y - x = b - a, nxy = z . n
        const float nxy = (b[0] - a[0]) * n[0] + (b[1] - a[1]) * n[1] + (b[2] - a[2]) * n[2];
        const cplx<float> e = exp_ik_ff(p, dd);
        const float vr = w.re * e.re - w.im * e.im, vi = w.re * e.im + w.im * e.re;
        const float g = kap * (nxy + d);
        return {inv * (g * vr + vi), inv * (g * vi - vr)};
    }
};


// Centred factor CF(y - xc) and centre-shift factor G(y, xc)/G(y, pxc) in
// mixed precision: distances in FP64 (d2 given), phases reduced in FP64.
template <int KIND>
__device__ __forceinline__ cplx<float> cf_mixed(double d2, const KParams& p)
{
    const double d = sqrt(d2);
    if (KIND == K_HELMHOLTZ_DK || KIND == K_COMBINEDFIELD_DK)
    {
        const cplx<float> e = exp_ik_f(p.kr, d);
        return {e.re * INV4PIF, e.im * INV4PIF};
    }
    const float id = rsqrtf((float)d2) * INV4PIF;
    if (KIND == K_LAPLACE)
        return {id, 0.f};
    if (KIND == K_HELMHOLTZ || KIND == K_COMBINEDFIELD)
    {
        const cplx<float> e = exp_ik_f(p.kr, d);
        return {e.re * id, e.im * id};
    }
    const cplx<float> e = exp_mk_f(p, d);
    return {e.re * id, e.im * id};
}

template <int KIND>
__device__ __forceinline__ cplx<float> transfer_mixed(double d2, double dp2, const KParams& p)
{
    const double d = sqrt(d2), dp = sqrt(dp2);
    if (KIND == K_HELMHOLTZ_DK || KIND == K_COMBINEDFIELD_DK)
        return exp_ik_f(p.kr, d - dp);
    const float ratio = __fdividef((float)dp, (float)d);
    if (KIND == K_LAPLACE)
        return {ratio, 0.f};
    if (KIND == K_HELMHOLTZ || KIND == K_COMBINEDFIELD)
    {
        const cplx<float> e = exp_ik_f(p.kr, d - dp);
        return {e.re * ratio, e.im * ratio};
    }
    const cplx<float> e = exp_mk_f(p, d - dp);
    return {e.re * ratio, e.im * ratio};
}

// The same factor from a tabulated delta = d - d_parent (FP64 difference
// rounded to FP32) and ratio = d_parent / d: the distance tables of
// multi-wavenumber batches, which serve every wavenumber of the batch.
template <int KIND>
__device__ __forceinline__ cplx<float> transfer_delta(float delta, float ratio, const KParams& p)
{
    if (KIND == K_HELMHOLTZ_DK || KIND == K_COMBINEDFIELD_DK)
        return exp_ik_ff(p, delta);
    if (KIND == K_LAPLACE)
        return {ratio, 0.f};
    const cplx<float> e = (KIND == K_HELMHOLTZ || KIND == K_COMBINEDFIELD) ? exp_ik_ff(p, delta)
                                                                          : exp_mk_ff(p, delta);
    return {e.re * ratio, e.im * ratio};
}

// FP32 coordinates: (s, theta, phi) from an FP32 difference vector
__device__ __forceinline__ void cart_to_interp_f(float p0, float p1, float p2, float H, float* s)
{
    const float a = p0 * p0 + p1 * p1;
    s[2] = fminf(fmaxf(atan2f(p1, p0), -(float)DPI), (float)DPI);
    s[1] = fminf(fmaxf(atan2f(sqrtf(a), p2), 0.f), (float)DPI);
    s[0] = H * rsqrtf(a + p2 * p2);
}


// FP32 cone-lookup parameters of one level, made once per CTA in shared
// memory so that the far-field lookups read no level data from global memory.
struct LookupF
{
    float lo[3], hi[3], hinv[3], top[3]; // domain, 1 / fine width, nf - 1
    int nf[3];
};

__device__ __forceinline__ void make_lookupf(const LevelGeom& G, LookupF& L)
{
#pragma unroll
    for (int d = 0; d < 3; d++)
    {
        L.lo[d] = (float)G.dmin[d];
        L.hi[d] = (float)G.dmax[d];
        L.hinv[d] = (float)G.hfi[d];
        L.top[d] = (float)(G.nf[d] - 1);
        L.nf[d] = G.nf[d];
    }
}

// fine_lookup_mixed with the level's FP32 parameters at hand: with
// t = (s - lo) / h the element index is q = floor(t) (clamped) and the local
// coordinate 2 (t - q) - 1, the same quantities as (s - centre) / (h / 2).
// The FP64 fallback (outside the FP32 domain or an inactive cone) is that of
// fine_lookup_mixed.
__device__ __forceinline__ int fine_lookup_fast(const LookupF& L, const LevelGeom& G,
                                                const int* __restrict__ fm, const double* p,
                                                double H, float* loc, unsigned long long* err)
{
    float sf[3];
    cart_to_interp_f((float)p[0], (float)p[1], (float)p[2], (float)H, sf);
    bool inside = true;
    int id = 0, stride = 1;
    float fr[3];
#pragma unroll
    for (int j = 0; j < 3; j++)
    {
        inside = inside && sf[j] >= L.lo[j] && sf[j] <= L.hi[j];
        const float t = (sf[j] - L.lo[j]) * L.hinv[j];
        const float q = fminf(fmaxf(floorf(t), 0.f), L.top[j]);
        fr[j] = t - q;
        id += __float2int_rz(q) * stride;
        stride *= L.nf[j];
    }
    if (inside)
    {
        const int gf = fm[id];
        if (gf >= 0)
        {
#pragma unroll
            for (int d = 0; d < 3; d++)
                loc[d] = fmaf(2.f, fr[d], -1.f);
            return gf;
        }
    }
    double s[3], ld[3];
    cart_to_interp(p[0], p[1], p[2], H, s);
    const int fe = element_for_point(s, G.dmin, G.dmax, G.hfi, G.nf);
    if (fe < 0)
        return -1;
    const int gf = fm[fe];
    if (gf < 0)
    {
        atomicAdd(err, 1ull);
        return -1;
    }
    to_local(fe, s, G.dmin, G.hf, G.hfi, G.nf, ld);
    loc[0] = (float)ld[0];
    loc[1] = (float)ld[1];
    loc[2] = (float)ld[2];
    return gf;
}

} // namespace ifgf
