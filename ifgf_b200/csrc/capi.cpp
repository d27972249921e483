// extern "C" entry points of libifgf_b200.so (declared in include/ifgf_b200.h).
#include "../../include/ifgf_b200.h"

#include <algorithm>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "operator.hpp"

namespace ifgf
{
void* noalloc_scratch(size_t* bytes); // noalloc.cu
void bounded_wait_selftest(double limit_ms, double* waited_ms); // operator.cu
}

struct ifgf_operator
{
    ifgf::Operator op;
    template <typename... A> explicit ifgf_operator(A&&... a) : op(std::forward<A>(a)...) {}
};

namespace
{
thread_local std::string g_last_error;

template <typename F> int guarded(F&& f)
{
    try
    {
        g_last_error.clear();
        f();
        return IFGF_OK;
    }
    catch (const ifgf::Error& e)
    {
        g_last_error = e.what();
        return e.code;
    }
    catch (const std::bad_alloc&)
    {
        g_last_error = "host allocation failed";
        return IFGF_ERR_OOM;
    }
    catch (const std::exception& e)
    {
        g_last_error = e.what();
        return IFGF_ERR_INTERNAL;
    }
    catch (...)
    {
        g_last_error = "unknown error";
        return IFGF_ERR_INTERNAL;
    }
}

int null_handle()
{
    g_last_error = "null operator handle";
    return IFGF_ERR_INVALID_ARG;
}
} // namespace

extern "C"
{
    int ifgf_create(int kind, double k_re, double k_im, long leaf_size, long order, long n_elem,
                    double tol, ifgf_operator** out)
    {
        if (!out)
            return null_handle();
        *out = nullptr;
        return guarded([&] { *out = new ifgf_operator(kind, k_re, k_im, leaf_size, order, n_elem, tol); });
    }

    int ifgf_set_dx(ifgf_operator* h, int dx)
    {
        if (!h)
            return null_handle();
        return guarded([&] { h->op.set_dx(dx); });
    }

    int ifgf_set_wavenumber(ifgf_operator* h, double k_re, double k_im)
    {
        if (!h)
            return null_handle();
        return guarded([&] { h->op.set_wavenumber(k_re, k_im); });
    }

    int ifgf_set_shard(ifgf_operator* h, int rank, int nranks)
    {
        if (!h)
            return null_handle();
        return guarded([&] { h->op.set_shard(rank, nranks); });
    }

    int ifgf_shard_boxes(const ifgf_operator* h, int* level, long* boxes, long cap, long* n)
    {
        if (!h)
            return null_handle();
        return guarded([&] {
            const std::vector<int64_t> b = h->op.shard_boxes();
            if (level)
                *level = h->op.shard_level();
            if (n)
                *n = (long)b.size();
            for (long i = 0; boxes && i < cap && i < (long)b.size(); i++)
                boxes[i] = (long)b[i];
        });
    }

    int ifgf_set_precision(ifgf_operator* h, int mode)
    {
        if (!h)
            return null_handle();
        return guarded([&] { h->op.set_precision(mode); });
    }

    int ifgf_set_upward_path(ifgf_operator* h, int path)
    {
        if (!h)
            return null_handle();
        return guarded([&] { h->op.set_upward_path(path); });
    }

    int ifgf_set_far_plan(ifgf_operator* h, int enable)
    {
        if (!h)
            return null_handle();
        return guarded([&] { h->op.set_far_plan(enable != 0); });
    }

    int ifgf_bounded_wait_selftest(double limit_ms, double* waited_ms)
    {
        return guarded([&] { ifgf::bounded_wait_selftest(limit_ms, waited_ms); });
    }

    int ifgf_init(ifgf_operator* h, const double* srcs, long n_src, const double* tgts, long n_tgt,
                  const double* normals, ifgf_cutoff_fn cutoff, void* user)
    {
        if (!h)
            return null_handle();
        return guarded([&] {
            std::function<bool(double)> cf;
            if (cutoff)
                cf = [cutoff, user](double d) { return cutoff(d, user) != 0; };
            h->op.init(srcs, n_src, tgts, n_tgt, normals, cf);
        });
    }

    int ifgf_init_plan_only(ifgf_operator* h, const double* srcs, long n_src, const double* tgts,
                            long n_tgt, ifgf_cutoff_fn cutoff, void* user)
    {
        if (!h)
            return null_handle();
        return guarded([&] {
            std::function<bool(double)> cf;
            if (cutoff)
                cf = [cutoff, user](double d) { return cutoff(d, user) != 0; };
            h->op.init(srcs, n_src, tgts, n_tgt, nullptr, cf, true);
        });
    }

    int ifgf_mult(ifgf_operator* h, const void* w, void* u)
    {
        if (!h)
            return null_handle();
        return guarded([&] { h->op.mult_host(w, u, 1); });
    }

    int ifgf_mult_batch(ifgf_operator* h, const void* w, void* u, long batch)
    {
        if (!h)
            return null_handle();
        return guarded([&] { h->op.mult_host(w, u, batch); });
    }

    int ifgf_mult_batch_device(ifgf_operator* h, const void* d_w, void* d_u, long batch,
                               void* stream)
    {
        if (!h)
            return null_handle();
        return guarded([&] { h->op.mult_batch_device(d_w, d_u, batch, stream); });
    }

    int ifgf_mult_wavenumbers(ifgf_operator* h, const double* k, long n_k, const void* w,
                              void* u)
    {
        if (!h)
            return null_handle();
        return guarded([&] { h->op.mult_wavenumbers_host(k, n_k, w, u); });
    }

    int ifgf_mult_wavenumbers_device(ifgf_operator* h, const double* k, long n_k,
                                     const void* d_w, void* d_u, void* stream)
    {
        if (!h)
            return null_handle();
        return guarded([&] { h->op.mult_wavenumbers_device(k, n_k, d_w, d_u, stream); });
    }

    int ifgf_mult_device(ifgf_operator* h, const void* d_w, void* d_u, void* stream)
    {
        if (!h)
            return null_handle();
        return guarded([&] { h->op.mult_device(d_w, d_u, stream); });
    }

    int ifgf_direct_eval(ifgf_operator* h, const void* w, const long* tidx, long nt, void* out)
    {
        if (!h)
            return null_handle();
        return guarded([&] {
            std::vector<int64_t> t(tidx, tidx + (tidx ? nt : 0));
            h->op.direct_eval(w, t.data(), nt, out);
        });
    }

    int ifgf_direct_eval_dk(ifgf_operator* h, const void* w, const long* tidx, long nt,
                            void* out)
    {
        if (!h)
            return null_handle();
        return guarded([&] {
            std::vector<int64_t> t(tidx, tidx + (tidx ? nt : 0));
            h->op.direct_eval(w, t.data(), nt, out, true);
        });
    }

    int ifgf_mult_adjoint(ifgf_operator* h, const void* w, void* u, long batch)
    {
        if (!h)
            return null_handle();
        return guarded([&] { h->op.mult_adjoint_host(w, u, batch); });
    }

    int ifgf_mult_adjoint_device(ifgf_operator* h, const void* d_w, void* d_u, void* stream)
    {
        if (!h)
            return null_handle();
        return guarded([&] { h->op.mult_adjoint_device(d_w, d_u, stream); });
    }

    int ifgf_mult_dk(ifgf_operator* h, const void* w, void* u, long batch)
    {
        if (!h)
            return null_handle();
        return guarded([&] { h->op.mult_dk_host(w, u, batch); });
    }

    int ifgf_mult_dk_device(ifgf_operator* h, const void* d_w, void* d_u, void* stream)
    {
        if (!h)
            return null_handle();
        return guarded([&] { h->op.mult_dk_device(d_w, d_u, stream); });
    }

    int ifgf_set_profiling(ifgf_operator* h, int on)
    {
        if (!h)
            return null_handle();
        return guarded([&] { h->op.set_profiling(on != 0); });
    }

    int ifgf_mult_device_noalloc(ifgf_operator* h, const void* d_w, void* d_u, void* stream)
    {
        if (!h)
            return null_handle();
        return guarded([&] {
            size_t bytes = 0;
            void* scratch = ifgf::noalloc_scratch(&bytes);
            h->op.mult_device_external_scratch(d_w, d_u, stream, scratch, bytes);
        });
    }

    int ifgf_num_sources(const ifgf_operator* h, long* n)
    {
        if (!h || !n)
            return null_handle();
        *n = (long)h->op.n_src();
        return IFGF_OK;
    }

    int ifgf_num_targets(const ifgf_operator* h, long* n)
    {
        if (!h || !n)
            return null_handle();
        *n = (long)h->op.n_tgt();
        return IFGF_OK;
    }

    int ifgf_stats_json(const ifgf_operator* h, char* buf, long cap, long* needed)
    {
        if (!h)
            return null_handle();
        return guarded([&] {
            const std::string s = h->op.stats_json();
            if (needed)
                *needed = (long)s.size() + 1;
            if (buf && cap > 0)
            {
                const size_t n = std::min<size_t>(s.size(), (size_t)cap - 1);
                std::memcpy(buf, s.data(), n);
                buf[n] = 0;
            }
        });
    }

    static const ifgf::Tree& tree_of(const ifgf_operator* h, int which)
    {
        if (which != 0 && which != 1)
            throw ifgf::Error(IFGF_ERR_INVALID_ARG, "which must be 0 (sources) or 1 (targets)");
        if (!h->op.planned())
            throw ifgf::Error(IFGF_ERR_STATE, "operator not initialised");
        return which == 0 ? h->op.plan().src : h->op.plan().tgt;
    }

    int ifgf_tree_levels(const ifgf_operator* h, int which, int* levels)
    {
        if (!h || !levels)
            return null_handle();
        return guarded([&] { *levels = tree_of(h, which).num_levels(); });
    }

    int ifgf_tree_num_boxes(const ifgf_operator* h, int which, int level, long* n)
    {
        if (!h || !n)
            return null_handle();
        return guarded([&] {
            const auto& t = tree_of(h, which);
            if (level < 0 || level >= t.num_levels())
                throw ifgf::Error(IFGF_ERR_INVALID_ARG, "level out of range");
            *n = (long)t.levels[level].size();
        });
    }

    int ifgf_tree_permutation(const ifgf_operator* h, int which, long* perm)
    {
        if (!h || !perm)
            return null_handle();
        return guarded([&] {
            const auto& t = tree_of(h, which);
            for (size_t i = 0; i < t.perm.size(); i++)
                perm[i] = (long)t.perm[i];
        });
    }

    int ifgf_tree_boxes(const ifgf_operator* h, int which, int level, long* ints, double* bbox)
    {
        if (!h)
            return null_handle();
        return guarded([&] {
            const auto& t = tree_of(h, which);
            if (level < 0 || level >= t.num_levels())
                throw ifgf::Error(IFGF_ERR_INVALID_ARG, "level out of range");
            const auto& L = t.levels[level];
            for (size_t b = 0; b < L.size(); b++)
            {
                if (ints)
                {
                    long* q = ints + 12 * b;
                    q[0] = (long)L.first[b];
                    q[1] = (long)L.last[b];
                    q[2] = L.parent[b];
                    q[3] = L.leaf[b];
                    for (int j = 0; j < 8; j++)
                        q[4 + j] = L.child[8 * b + j];
                }
                if (bbox)
                    for (int d = 0; d < 3; d++)
                    {
                        bbox[6 * b + d] = L.bbmin[3 * b + d];
                        bbox[6 * b + 3 + d] = L.bbmax[3 * b + d];
                    }
            }
        });
    }

    int ifgf_box_list(const ifgf_operator* h, int level, long box, int far, long* out, long cap,
                      long* n)
    {
        if (!h)
            return null_handle();
        return guarded([&] {
            const auto& t = tree_of(h, 0);
            if (level < 0 || level >= t.num_levels() || box < 0 || box >= (long)t.levels[level].size())
                throw ifgf::Error(IFGF_ERR_INVALID_ARG, "box out of range");
            const auto& P = h->op.plan();
            const ifgf::PairLists& pl = far ? P.far : P.near;
            const int64_t sg = t.level_off[level] + box;
            const long cnt = (long)pl.count(sg);
            if (n)
                *n = cnt;
            const auto& T = P.tgt;
            for (long i = 0; out && i < cnt && i < cap; i++)
            {
                const int64_t g = pl.begin(sg)[i];
                int lev = (int)(std::upper_bound(T.level_off.begin(), T.level_off.end(), g) -
                                T.level_off.begin()) - 1;
                const int64_t b = g - T.level_off[lev];
                out[2 * i] = (long)T.levels[lev].first[b];
                out[2 * i + 1] = (long)T.levels[lev].last[b];
            }
        });
    }

    int ifgf_box_cones(const ifgf_operator* h, int level, long box, int step, long* out, long cap,
                       long* n)
    {
        if (!h)
            return null_handle();
        return guarded([&] {
            if (!h->op.initialized())
                throw ifgf::Error(IFGF_ERR_STATE, "operator not initialised");
            auto v = h->op.box_cones(level, box, step);
            if (n)
                *n = (long)v.size();
            for (long i = 0; out && i < (long)v.size() && i < cap; i++)
                out[i] = (long)v[i];
        });
    }

    int ifgf_level_grid(const ifgf_operator* h, int level, int step, long* n)
    {
        if (!h || !n)
            return null_handle();
        return guarded([&] {
            int64_t v[3];
            h->op.level_grid(level, step, v);
            for (int d = 0; d < 3; d++)
                n[d] = (long)v[d];
        });
    }

    int ifgf_orders(const ifgf_operator* h, int step, int* order)
    {
        if (!h || !order)
            return null_handle();
        return guarded([&] { h->op.orders(step, order); });
    }

    int ifgf_destroy(ifgf_operator* h)
    {
        return guarded([&] { delete h; });
    }

    const char* ifgf_last_error(void) { return g_last_error.c_str(); }
}
