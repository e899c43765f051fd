// host.cpp -- the C ABI (include/ndlgpu.h): validation, view canonicalisation,
// planning and launch.  Host-only C++17.
//
// Every entry point validates its arguments completely before the first CUDA
// call, so an error return means nothing was enqueued (the reference checks
// with assert() only, processing/convolution.h:59,112 and image/core.h:557).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "internal.h"

namespace ndlgpu {

static thread_local std::string t_last_error;
static std::atomic<uint64_t> g_launches{0};

void count_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

ndlgpu_status set_error(ndlgpu_status s, const std::string& msg)
{
    t_last_error = msg;
    return s;
}

static ndlgpu_status fail(ndlgpu_status s, const std::string& msg)
{
    t_last_error = msg;
    return s;
}

static ndlgpu_status cuda_fail(cudaError_t e, const char* what)
{
    if (e == cudaErrorMemoryAllocation) return fail(NDLGPU_ERR_OUT_OF_MEMORY, std::string(what) + ": out of device memory");
    return fail(NDLGPU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// Views
// ---------------------------------------------------------------------------

static ndlgpu_status check_view(const ndlgpu_view* v, const char* name, bool device_data)
{
    if (!v) return fail(NDLGPU_ERR_INVALID_ARGUMENT, std::string(name) + " is NULL");
    if (v->rank < 1 || v->rank > kMaxRank)
        return fail(NDLGPU_ERR_INVALID_ARGUMENT, std::string(name) + ": rank must be 1..8");
    if (!dtype_valid(v->dtype)) return fail(NDLGPU_ERR_UNSUPPORTED_DTYPE, std::string(name) + ": unknown dtype");
    __int128 span = 0;
    bool empty = false;
    for (int i = 0; i < v->rank; i++) {
        if (v->extent[i] < 0) return fail(NDLGPU_ERR_INVALID_ARGUMENT, std::string(name) + ": negative extent");
        if (v->extent[i] == 0) empty = true;
        if (v->extent[i] > 0x7fffffffLL)
            return fail(NDLGPU_ERR_INDEX_OVERFLOW, std::string(name) + ": extent exceeds 2^31-1");
        const __int128 s = v->stride[i] < 0 ? -(__int128)v->stride[i] : (__int128)v->stride[i];
        span += s * (__int128)(v->extent[i] > 0 ? v->extent[i] - 1 : 0);
    }
    if (span > ((__int128)1 << 62)) return fail(NDLGPU_ERR_INDEX_OVERFLOW, std::string(name) + ": view spans more than 2^62 elements");
    if (!empty && device_data && !v->data) return fail(NDLGPU_ERR_INVALID_ARGUMENT, std::string(name) + ": data is NULL");
    return NDLGPU_OK;
}

static int64_t view_count(const ndlgpu_view* v)
{
    int64_t n = 1;
    for (int i = 0; i < v->rank; i++) n *= v->extent[i];
    return n;
}

// Byte range [lo, hi) covered by a view.
static void view_bytes(const ndlgpu_view* v, intptr_t* lo, intptr_t* hi)
{
    const int es = dtype_size(v->dtype);
    int64_t mn = 0, mx = 0;
    for (int i = 0; i < v->rank; i++) {
        const int64_t d = v->stride[i] * (v->extent[i] - 1);
        if (d < 0) mn += d; else mx += d;
    }
    *lo = (intptr_t)v->data + (intptr_t)mn * es;
    *hi = (intptr_t)v->data + (intptr_t)mx * es + es;
}

// dst must not write one address twice: with axes sorted by |stride|, each
// axis must step over everything the faster axes cover.
static ndlgpu_status check_no_self_overlap(const ndlgpu_view* dst)
{
    std::vector<std::pair<int64_t, int64_t>> ax;
    for (int i = 0; i < dst->rank; i++)
        if (dst->extent[i] > 1) ax.push_back({dst->stride[i] < 0 ? -dst->stride[i] : dst->stride[i], dst->extent[i]});
    std::sort(ax.begin(), ax.end());
    int64_t covered = 1;
    for (auto& a : ax) {
        if (a.first < covered) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "dst view overlaps itself (a stride is smaller than the span of the faster axes)");
        covered = a.first * a.second;
    }
    return NDLGPU_OK;
}

static ndlgpu_status check_pair(const ndlgpu_view* src, const ndlgpu_view* dst)
{
    if (src->rank != dst->rank) return fail(NDLGPU_ERR_EXTENT_MISMATCH, "src and dst ranks differ");
    for (int i = 0; i < src->rank; i++)
        if (src->extent[i] != dst->extent[i])
            return fail(NDLGPU_ERR_EXTENT_MISMATCH, "dst.extent() != src.extent() (convolution.h:59) on axis " + std::to_string(i));
    if (view_count(src) == 0) return NDLGPU_OK;
    intptr_t a0, a1, b0, b1;
    view_bytes(src, &a0, &a1);
    view_bytes(dst, &b0, &b1);
    if (a0 < b1 && b0 < a1) return fail(NDLGPU_ERR_ALIASING, "src and dst memory overlap (in-place convolution is not supported)");
    return check_no_self_overlap(dst);
}

// ---------------------------------------------------------------------------
// Canonical problem
// ---------------------------------------------------------------------------

struct CAxis {
    int64_t n, ss, ds;
    int logical;
};

struct CPass {
    int axis;                 // canonical axis index
    std::vector<int> off;     // nonzero taps, summation order
    std::vector<double> w;
};

struct Canon {
    const char* src;
    char* dst;
    int sdt, ddt;
    std::vector<CAxis> ax;
    std::vector<CPass> passes;
    int64_t total;
};

// Input pass description (logical axis).
struct LPass {
    int axis;
    int center;
    std::vector<double> taps;
};

static ndlgpu_status canonicalise(const ndlgpu_view* src, const ndlgpu_view* dst,
                                  const std::vector<LPass>& lp, int border, Canon* out, bool keep_zero = false)
{
    const int R = src->rank;
    if (border < NDLGPU_CLAMP || border > NDLGPU_REFLECT) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "unknown border mode");
    Canon c;
    c.src = (const char*)src->data;
    c.dst = (char*)dst->data;
    c.sdt = src->dtype;
    c.ddt = dst->dtype;
    c.total = view_count(src);
    const int ses = dtype_size(c.sdt), des = dtype_size(c.ddt);

    // passes, with the one-period rule for Wrap/Reflect (mathHelpers.h:23-24
    // wrap/reflect once; a larger offset would index outside the image)
    std::vector<CPass> passes;
    for (const LPass& p : lp) {
        if (p.axis < 0 || p.axis >= R) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "pass axis out of range");
        if (p.taps.empty()) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "a pass has no taps");
        if ((int)p.taps.size() > kMaxTaps) return fail(NDLGPU_ERR_TOO_MANY_TAPS, "a pass has more than 255 taps");
        CPass cp;
        cp.axis = p.axis;
        for (int k = 0; k < (int)p.taps.size(); k++) {
            if (p.taps[k] == 0.0 && !keep_zero) continue;   // image/detail.h:171-172
            const int o = k - p.center;
            if (border != NDLGPU_CLAMP && c.total > 0 && (o > src->extent[p.axis] || o < -src->extent[p.axis]))
                return fail(NDLGPU_ERR_RADIUS_EXCEEDS_EXTENT,
                            "tap offset " + std::to_string(o) + " exceeds the extent " + std::to_string(src->extent[p.axis]) +
                                " of axis " + std::to_string(p.axis) + " (Wrap/Reflect map one period only)");
            cp.off.push_back(o);
            cp.w.push_back(p.taps[k]);
        }
        passes.push_back(cp);
    }
    if (c.total == 0) {
        *out = c;
        return NDLGPU_OK;
    }

    // flip negative source strides (the border maps are symmetric under
    // reversal, so only the tap offsets change sign; summation order kept)
    std::vector<CAxis> ax(R);
    std::vector<bool> has_pass(R, false);
    for (auto& p : passes) has_pass[p.axis] = true;
    for (int i = 0; i < R; i++) {
        CAxis a{src->extent[i], src->stride[i], dst->stride[i], i};
        if (a.ss < 0) {
            c.src += (intptr_t)(a.n - 1) * a.ss * ses;
            c.dst += (intptr_t)(a.n - 1) * a.ds * des;
            a.ss = -a.ss;
            a.ds = -a.ds;
            for (auto& p : passes)
                if (p.axis == i)
                    for (auto& o : p.off) o = -o;
        }
        ax[i] = a;
    }
    // drop extent-1 axes without passes; order by source stride
    std::vector<int> keep;
    for (int i = 0; i < R; i++)
        if (ax[i].n > 1 || has_pass[i]) keep.push_back(i);
    if (keep.empty()) keep.push_back(0);
    std::stable_sort(keep.begin(), keep.end(), [&](int a, int b) { return ax[a].ss < ax[b].ss; });
    std::vector<int> pos(R, -1);
    for (int k = 0; k < (int)keep.size(); k++) {
        c.ax.push_back(ax[keep[k]]);
        pos[keep[k]] = k;
    }
    for (auto& p : passes) p.axis = pos[p.axis];
    c.passes = passes;
    *out = c;
    return NDLGPU_OK;
}

// ---------------------------------------------------------------------------
// Arithmetic selection
// ---------------------------------------------------------------------------

static double max_abs_of(int dt)
{
    switch (dt) {
    case NDLGPU_U8: return 255;
    case NDLGPU_I8: return 128;
    case NDLGPU_U16: return 65535;
    case NDLGPU_I16: return 32768;
    default: return -1;   // not eligible for the int32 path
    }
}

// Smallest shift s <= 20 with every weight an integer multiple of 2^-s and
// |numerator| < 2^20; -1 if none (the taps are not all dyadic).
static int dyadic_shift(const std::vector<double>& w, std::vector<int32_t>* num)
{
    for (int s = 0; s <= 20; s++) {
        bool ok = true;
        const double scale = std::ldexp(1.0, s);
        for (double x : w) {
            const double y = x * scale;   // exact (power-of-two scale)
            if (!(std::fabs(y) < 1048576.0) || y != std::floor(y)) { ok = false; break; }
        }
        if (ok) {
            if (num) {
                num->clear();
                for (double x : w) num->push_back((int32_t)(x * scale));
            }
            return s;
        }
    }
    return -1;
}

// Integer path eligibility: integral src and dst, all taps dyadic and every
// partial sum bounded by 2^31 (so the reference's double sums are exact too).
static bool int_path_ok(const Canon& c, int compose)
{
    if (!dtype_integral(c.ddt)) return false;
    double in_max = max_abs_of(c.sdt);
    if (in_max < 0) return false;
    if (compose == NDLGPU_CAST_EACH && c.passes.size() > 1 && max_abs_of(c.ddt) < 0) return false;
    double bound = in_max;
    int shift = 0;
    for (size_t i = 0; i < c.passes.size(); i++) {
        std::vector<int32_t> m;
        const int s = dyadic_shift(c.passes[i].w, &m);
        if (s < 0) return false;
        double sum = 0;
        for (int32_t v : m) sum += std::fabs((double)v);
        if (compose == NDLGPU_CAST_EACH) {
            const double b = (i == 0 ? in_max : max_abs_of(c.ddt)) * sum;
            if (!(b < 2147483647.0)) return false;
        } else {
            bound *= sum;
            shift += s;
        }
    }
    if (compose != NDLGPU_CAST_EACH && !(bound < 2147483647.0 && shift <= 30)) return false;
    return true;
}

static Acc pick_acc(const Canon& c, int compose, int precision)
{
    const bool intok = int_path_ok(c, compose);
    if (precision == NDLGPU_PREC_EXACT) return intok ? Acc::I32 : Acc::F64;
    if (precision == NDLGPU_PREC_FP32) return Acc::F32;
    if (dtype_integral(c.ddt)) return intok ? Acc::I32 : Acc::F64;
    if (c.ddt == NDLGPU_F64 || c.sdt == NDLGPU_F64) return Acc::F64;
    return Acc::F32;
}

// ---------------------------------------------------------------------------
// Workspace
// ---------------------------------------------------------------------------

struct Scratch {
    void* base = nullptr;
    bool owned = false;
    cudaStream_t stream = nullptr;
    ~Scratch()
    {
        if (owned && base) cudaFreeAsync(base, stream);
    }
};

static size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

// The library's own stream-ordered pool for scratch the caller did not
// provide, one per device: it keeps up to 2 GiB cached between calls (the
// device's default pool returns everything at each synchronisation, so every
// call would map its scratch anew); the process's other pools are untouched.
static cudaError_t scratch_pool(cudaMemPool_t* out)
{
    static std::mutex mu;
    static std::vector<cudaMemPool_t> pools;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    if ((int)pools.size() <= dev) pools.resize(dev + 1, nullptr);
    if (!pools[dev]) {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool;
        e = cudaMemPoolCreate(&pool, &props);
        if (e != cudaSuccess) return e;
        uint64_t keep = 2ull << 30;
        e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) return e;
        pools[dev] = pool;
    }
    *out = pools[dev];
    return cudaSuccess;
}

static ndlgpu_status get_scratch(size_t need, void* ws, size_t ws_bytes, cudaStream_t s, Scratch* sc)
{
    if (need == 0) return NDLGPU_OK;
    if (ws) {
        if (ws_bytes < need)
            return fail(NDLGPU_ERR_WORKSPACE, "workspace of " + std::to_string(ws_bytes) + " bytes is smaller than the " +
                                                  std::to_string(need) + " bytes required");
        sc->base = ws;
        return NDLGPU_OK;
    }
    cudaMemPool_t pool = nullptr;
    cudaError_t e = scratch_pool(&pool);
    if (e != cudaSuccess) return cuda_fail(e, "scratch memory pool");
    e = cudaMallocFromPoolAsync(&sc->base, need, pool, s);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocFromPoolAsync(workspace)");
    sc->owned = true;
    sc->stream = s;
    return NDLGPU_OK;
}

// ---------------------------------------------------------------------------
// Generic pass chain
// ---------------------------------------------------------------------------

static void fill_div(GenericPassParams& p)
{
    for (int i = 0; i < p.rank; i++) p.div[i].init((uint32_t)p.n[i]);
}

// One pass between two canonical buffers (strides given per canonical axis),
// split into launches of < 2^31 outputs along the slowest non-pass axis.
static ndlgpu_status run_generic_pass(Acc acc, const Canon& c, const CPass& pass,
                                      const char* in, int in_dt, const std::vector<int64_t>& in_st,
                                      char* out, int out_dt, const std::vector<int64_t>& out_st,
                                      int border, int store_mode, int shift, const std::vector<int32_t>& num,
                                      cudaStream_t s, bool transpose = false)
{
    const int R = (int)c.ax.size();
    // float storage with FP32 sums and dense taps: the tiled pass kernels
    if (!transpose && acc == Acc::F32 && store_mode == STORE_CAST && R <= kTiledRank && !pass.off.empty() &&
        (int)pass.off.size() <= kMaxTaps) {
        TiledPassParams t;
        std::memset(&t, 0, sizeof(t));
        std::vector<std::pair<int, double>> tw;
        for (size_t i = 0; i < pass.off.size(); i++) tw.push_back({pass.off[i], pass.w[i]});
        std::sort(tw.begin(), tw.end());
        t.src = in;
        t.dst = out;
        t.src_dtype = in_dt;
        t.dst_dtype = out_dt;
        t.rank = R;
        t.axis = pass.axis;
        t.border = border;
        t.ntap = (int)tw.size();
        t.omin = tw.front().first;
        t.omax = tw.back().first;
        for (int k = 0; k < t.ntap; k++) t.w[k] = (float)tw[k].second;
        for (int i = 0; i < R; i++) {
            t.n[i] = c.ax[i].n;
            t.ss[i] = in_st[i];
            t.ds[i] = out_st[i];
        }
        t.rows = c.total / c.ax[0].n;
        if (tiled_pass_supported(t)) {
            cudaError_t e = launch_tiled_pass(t, s);
            if (e != cudaSuccess) return cuda_fail(e, "tiled pass");
            return NDLGPU_OK;
        }
    }
    GenericPassParams p;
    std::memset(&p, 0, sizeof(p));
    p.src_dtype = in_dt;
    p.dst_dtype = out_dt;
    p.rank = R;
    p.axis = pass.axis;
    p.ntap = (int)pass.off.size();
    p.border = border;
    p.store_mode = store_mode;
    p.shift = shift;
    for (int t = 0; t < p.ntap; t++) {
        p.off[t] = pass.off[t];
        p.wd[t] = pass.w[t];
        p.wf[t] = (float)pass.w[t];
        p.wi[t] = num.empty() ? 0 : num[t];
    }
    for (int i = 0; i < R; i++) {
        p.n[i] = c.ax[i].n;
        p.ss[i] = in_st[i];
        p.ds[i] = out_st[i];
    }
    // chunking axis: slowest axis that is not the pass axis
    int cax = -1;
    for (int i = R - 1; i >= 0; i--)
        if (i != pass.axis) { cax = i; break; }
    int64_t per = c.total;
    int64_t chunk_n = 1;
    if (c.total >= (int64_t(1) << 31)) {
        if (cax < 0) return fail(NDLGPU_ERR_INDEX_OVERFLOW, "a single 1-D pass of 2^31 or more elements is not supported");
        per = c.total / c.ax[cax].n;
        chunk_n = std::max<int64_t>(1, ((int64_t(1) << 31) - 1) / per);
        if (per >= (int64_t(1) << 31)) return fail(NDLGPU_ERR_INDEX_OVERFLOW, "view too large for the general kernel");
    }
    const int ies = dtype_size(in_dt), oes = dtype_size(out_dt);
    if (chunk_n == 1 && c.total < (int64_t(1) << 31)) {
        p.src = in;
        p.dst = out;
        p.total = (uint32_t)c.total;
        fill_div(p);
        cudaError_t e = transpose ? launch_pass_adjoint(acc, p, s) : launch_generic_pass(acc, p, s);
        if (e != cudaSuccess) return cuda_fail(e, "generic pass");
        return NDLGPU_OK;
    }
    for (int64_t b = 0; b < c.ax[cax].n; b += chunk_n) {
        const int64_t m = std::min<int64_t>(chunk_n, c.ax[cax].n - b);
        p.n[cax] = m;
        p.src = in + (intptr_t)b * in_st[cax] * ies;
        p.dst = out + (intptr_t)b * out_st[cax] * oes;
        p.total = (uint32_t)(per * m);
        fill_div(p);
        if (transpose) return fail(NDLGPU_ERR_INDEX_OVERFLOW, "adjoint views of 2^31 or more elements are not supported");
        cudaError_t e = launch_generic_pass(acc, p, s);
        if (e != cudaSuccess) return cuda_fail(e, "generic pass");
    }
    return NDLGPU_OK;
}

static std::vector<int64_t> contiguous_strides(const Canon& c)
{
    std::vector<int64_t> st(c.ax.size());
    int64_t m = 1;
    for (size_t i = 0; i < c.ax.size(); i++) {
        st[i] = m;
        m *= c.ax[i].n;
    }
    return st;
}

struct Plan {
    Acc acc;
    bool fused = false;
    FusedParams fp;
    int nscratch = 0;       // intermediate buffers for the generic chain
    int scratch_dtype = 0;
};

// Effective weights of a transposed 1-D pass at the positions within r = K/2
// of either end of an axis of extent M: for position j, window entry m (the
// zero-padded input at j - r + m) collects every tap w_k whose forward read
// of that input lands on j after the border map (map(i + o_k) == j).  The
// transposed pass elsewhere is the plain flipped correlation.
// Zone rows for a transposed pass whose window is W wide (centred) and whose
// real taps reach r: rows e < r hold positions 0..r-1, rows r..2r-1 hold
// positions M-r..M-1; entry m weighs the zero-padded input at j - W/2 + m.
static void zone_rows(int64_t M, int border, const std::vector<std::pair<int, double>>& taps, int W, int r,
                      std::vector<float>* out)
{
    out->assign((size_t)2 * r * W, 0.f);
    for (int e = 0; e < 2 * r; e++) {
        const int64_t j = (e < r) ? e : (M - r + (e - r));
        if (j < 0 || j >= M) continue;
        for (int m = 0; m < W; m++) {
            const int64_t i = j - W / 2 + m;
            if (i < 0 || i >= M) continue;
            double acc = 0;
            for (const auto& t : taps) {
                int64_t pos = i + t.first;
                if (pos < 0 || pos >= M) {
                    if (border == NDLGPU_WRAP) pos = pos < 0 ? pos + M : pos - M;
                    else if (border == NDLGPU_REFLECT) pos = pos < 0 ? -pos - 1 : 2 * M - pos - 1;
                    else pos = pos < 0 ? 0 : M - 1;
                }
                if (pos == j) acc += t.second;
            }
            (*out)[(size_t)e * W + m] = (float)acc;
        }
    }
}

static void zone_table(int64_t M, int border, const std::vector<std::pair<int, double>>& taps, int K,
                       float (*tab)[17])
{
    const int r = K / 2;
    for (int e = 0; e < 16; e++)
        for (int m = 0; m < 17; m++) tab[e][m] = 0.f;
    for (int e = 0; e < 2 * r && e < 16; e++) {
        const int64_t j = (e < r) ? e : (M - r + (e - r));
        if (j < 0 || j >= M) continue;
        double acc[17] = {0};
        for (int m = 0; m < K; m++) {
            const int64_t i = j - r + m;
            if (i < 0 || i >= M) continue;
            for (const auto& t : taps) {
                int64_t pos = i + t.first;
                if (pos < 0 || pos >= M) {
                    if (border == NDLGPU_WRAP) pos = pos < 0 ? pos + M : pos - M;
                    else if (border == NDLGPU_REFLECT) pos = pos < 0 ? -pos - 1 : 2 * M - pos - 1;
                    else pos = pos < 0 ? 0 : M - 1;
                }
                if (pos == j) acc[m] += t.second;
            }
        }
        for (int m = 0; m < K; m++) tab[e][m] = (float)acc[m];
    }
}

// Fused-kernel eligibility and parameters.  adj: the transposed chain (the
// input gradient), run by the float fused kernel only.
static bool plan_fused(const Canon& c, Acc acc, int compose, int border, FusedParams* fp, int adj = 0)
{
    if (acc != Acc::F32 && acc != Acc::I32) return false;
    if (c.passes.empty() || c.passes.size() > 3) return false;
    if (compose == NDLGPU_CAST_EACH && c.passes.size() > 1) {
        // per-pass DstT rounding is the identity only for f32 results
        if (!(acc == Acc::F32 && c.ddt == NDLGPU_F32)) return false;
    }
    const int R = (int)c.ax.size();
    int kx = 1, ky = 1, kz = 1;
    int role[3] = {0, -1, -1};   // canonical axis of X, Y, Z
    std::vector<bool> used(R, false);
    used[0] = true;
    std::vector<const CPass*> by_axis(R, nullptr);
    for (auto& p : c.passes) {
        if (by_axis[p.axis]) return false;   // two passes on one axis
        by_axis[p.axis] = &p;
    }
    // tap lists must be dense, odd and centred (offsets -K/2 .. K/2) in
    // either direction; the order does not matter for F32/I32 sums
    auto dense = [&](const CPass* p, int* K) {
        if (!p) { *K = 1; return true; }
        std::vector<int> o = p->off;
        std::sort(o.begin(), o.end());
        const int k = (int)o.size();
        if (k % 2 == 0 || k > 37) return false;
        for (int i = 0; i < k; i++)
            if (o[i] != i - k / 2) return false;
        *K = k;
        return true;
    };
    std::vector<int> others;
    for (int i = 1; i < R; i++)
        if (by_axis[i]) others.push_back(i);
    if (others.size() > 2) return false;
    for (int i = 1; i < R && others.size() < 2; i++)
        if (!by_axis[i] && std::find(others.begin(), others.end(), i) == others.end()) others.push_back(i);
    std::sort(others.begin(), others.end());
    // integer path: when the destination is contiguous along a non-X pass
    // axis (a transposed output), make that axis Y and stage the stores
    bool tstore = false;
    if (acc == Acc::I32 && !adj && others.size() == 2) {
        auto ads = [&](int i) { return c.ax[i].ds < 0 ? -c.ax[i].ds : c.ax[i].ds; };
        const int64_t dx0 = c.ax[0].ds < 0 ? -c.ax[0].ds : c.ax[0].ds;
        if (dx0 != 1) {
            if (ads(others[1]) == 1) std::swap(others[0], others[1]);
            tstore = ads(others[0]) == 1;
        }
    }
    if (others.size() >= 1) role[1] = others[0];
    if (others.size() >= 2) role[2] = others[1];
    for (int r = 0; r < 3; r++)
        if (role[r] >= 0) used[role[r]] = true;
    if (!dense(by_axis[0], &kx)) return false;
    if (role[1] >= 0 && !dense(by_axis[role[1]], &ky)) return false;
    if (role[2] >= 0 && !dense(by_axis[role[2]], &kz)) return false;
    const bool v2 = (acc == Acc::F32) && fused2_supported(c.sdt, c.ddt, kx, ky, kz, adj);
    if (adj && !v2) return false;
    const bool u8shape = acc == Acc::I32 && !adj && fused_u8_shape(c.sdt, c.ddt, kx, ky, kz);
    if (!v2 && !fused_supported(acc, c.sdt, c.ddt, kx, ky, kz) && !u8shape) return false;

    FusedParams& p = *fp;
    std::memset(&p, 0, sizeof(p));
    p.src = c.src;
    p.dst = c.dst;
    p.src_dtype = c.sdt;
    p.dst_dtype = c.ddt;
    p.border = border;
    p.store_mode = (dtype_integral(c.ddt) && c.passes.size() > 1 && compose == NDLGPU_ROUND_ONCE) ? STORE_ROUND : STORE_CAST;
    auto geo = [&](int r, int* n, int64_t* s, int64_t* d) {
        if (role[r] < 0) { *n = 1; *s = 0; *d = 0; return; }
        *n = (int)c.ax[role[r]].n;
        *s = c.ax[role[r]].ss;
        *d = c.ax[role[r]].ds;
    };
    geo(0, &p.nx, &p.sx, &p.dx);
    geo(1, &p.ny, &p.sy, &p.dy);
    geo(2, &p.nz, &p.sz, &p.dz);
    // remaining axes must merge into one affine batch axis
    int64_t nb = 1, sb = 0, db = 0;
    for (int i = 0; i < R; i++) {
        if (used[i]) continue;
        if (nb == 1) { nb = c.ax[i].n; sb = c.ax[i].ss; db = c.ax[i].ds; continue; }
        if (c.ax[i].ss != sb * nb || c.ax[i].ds != db * nb) return false;
        nb *= c.ax[i].n;
    }
    if (nb > 0x7fffffffLL) return false;
    p.nbatch = (int)nb;
    p.sb = sb;
    p.db = db;
    p.kx = kx; p.ky = ky; p.kz = kz;
    p.cx = kx / 2; p.cy = ky / 2; p.cz = kz / 2;
    // weights in ascending offset order
    auto fill = [&](const CPass* cp, int K, float* wf, int32_t* wi, int* shift) {
        if (!cp) { wf[0] = 1.0f; wi[0] = 1; return; }
        std::vector<std::pair<int, double>> t;
        for (size_t i = 0; i < cp->off.size(); i++) t.push_back({cp->off[i], cp->w[i]});
        std::sort(t.begin(), t.end());
        std::vector<double> w;
        for (auto& x : t) w.push_back(x.second);
        for (int k = 0; k < K; k++) wf[k] = (float)w[k];
        if (acc == Acc::I32) {
            std::vector<int32_t> m;
            *shift += dyadic_shift(w, &m);
            for (int k = 0; k < K; k++) wi[k] = m[k];
        }
    };
    int shift = 0;
    fill(by_axis[0], kx, p.wxf, p.wxi, &shift);
    fill(role[1] >= 0 ? by_axis[role[1]] : nullptr, ky, p.wyf, p.wyi, &shift);
    fill(role[2] >= 0 ? by_axis[role[2]] : nullptr, kz, p.wzf, p.wzi, &shift);
    p.shift = shift;
    if (adj) {
        // transposed passes: flipped taps; Clamp/Reflect read zeros outside
        // the image and fold the border through the zone tables
        p.adj = 1;
        p.zero_pad = (border != NDLGPU_WRAP) ? 1 : 0;
        auto flip = [](float* w, int K) { std::reverse(w, w + K); };
        flip(p.wxf, kx);
        flip(p.wyf, ky);
        flip(p.wzf, kz);
        auto sorted = [&](const CPass* cp) {
            std::vector<std::pair<int, double>> t;
            if (cp)
                for (size_t i = 0; i < cp->off.size(); i++) t.push_back({cp->off[i], cp->w[i]});
            else
                t.push_back({0, 1.0});
            std::sort(t.begin(), t.end());
            return t;
        };
        if (p.zero_pad) {
            if (kx > 17 || ky > 17 || kz > 17) return false;
            zone_table(p.nx, border, sorted(by_axis[0]), kx, p.zx);
            zone_table(p.ny, border, sorted(role[1] >= 0 ? by_axis[role[1]] : nullptr), ky, p.zy);
            zone_table(p.nz, border, sorted(role[2] >= 0 ? by_axis[role[2]] : nullptr), kz, p.zz);
        }
    }
    for (int k = 0; k < 40; k++) {
        p.wx2[k] = make_float2(k < kx ? p.wxf[k] : 0.f, k < kx ? p.wxf[k] : 0.f);
        p.wy2[k] = make_float2(k < ky ? p.wyf[k] : 0.f, k < ky ? p.wyf[k] : 0.f);
        p.wz2[k] = make_float2(k < kz ? p.wzf[k] : 0.f, k < kz ? p.wzf[k] : 0.f);
    }
    // 32-bit in-plane offsets in the kernels
    const int ses = dtype_size(c.sdt), des = dtype_size(c.ddt);
    if ((__int128)(p.ny - 1) * (p.sy < 0 ? -p.sy : p.sy) + (__int128)(p.nx - 1) * (p.sx < 0 ? -p.sx : p.sx) >= ((__int128)1 << 31))
        return false;
    // vector paths: 16-byte aligned source rows, 4-element aligned output rows
    auto al = [](const void* ptr, int64_t bytes) { return ((uintptr_t)ptr % (uintptr_t)bytes) == 0; };
    p.vec_ld = (p.sx == 1 && al(p.src, 16) && (p.sy * ses) % 16 == 0 && (p.sz * ses) % 16 == 0 &&
                (p.sb * ses) % 16 == 0) ? 1 : 0;
    p.vec_st = (p.dx == 1 && al(p.dst, 4 * des) && (p.dy % 4) == 0 && (p.dz % 4) == 0 && (p.db % 4) == 0) ? 1 : 0;
    p.vec_st = v2 ? p.vec_st : 0;
    p.tstore = tstore ? 1 : 0;
    // a shape only the packed uint8 kernel compiles must also meet its bounds
    if (u8shape && !fused_supported(acc, c.sdt, c.ddt, kx, ky, kz) && !fused_u8_supported(p)) return false;
    // Z chunk of the integer kernel (64 x 32 tiles, two resident CTAs per SM);
    // the float kernel picks its own at launch
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long tiles = (long long)((p.nx + 63) / 64) * ((p.ny + 31) / 32) * p.nbatch;
    const int chunks = pick_zchunks(tiles, 2LL * sms, p.nz, kz - 1);
    p.zchunk = std::max(1, (p.nz + chunks - 1) / chunks);
    return true;
}

static ndlgpu_status plan(const Canon& c, int compose, int precision, int border, Plan* pl)
{
    pl->acc = pick_acc(c, compose, precision);
    pl->fused = plan_fused(c, pl->acc, compose, border, &pl->fp);
    if (pl->fused || c.passes.size() <= 1) {
        pl->nscratch = 0;
        return NDLGPU_OK;
    }
    pl->nscratch = c.passes.size() == 2 ? 1 : 2;
    if (compose == NDLGPU_CAST_EACH) pl->scratch_dtype = c.ddt;
    else pl->scratch_dtype = acc_dtype(pl->acc);
    return NDLGPU_OK;
}

static size_t plan_workspace(const Canon& c, const Plan& pl)
{
    if (pl.nscratch == 0) return 0;
    return (size_t)pl.nscratch * align_up((size_t)c.total * dtype_size(pl.scratch_dtype));
}

static ndlgpu_status execute(const Canon& c, const Plan& pl, int compose, int border, void* ws, size_t ws_bytes,
                             cudaStream_t s)
{
    if (c.total == 0) return NDLGPU_OK;
    if (pl.fused) {
        const FusedParams& f = pl.fp;
        cudaError_t e;
        if (pl.acc == Acc::F32 && !f.adj && !f.tstore && fwd3_supported(f.src_dtype, f.dst_dtype, f.kx, f.ky, f.kz))
            e = launch_fwd3(f, s);
        else if (pl.acc == Acc::F32 && fused2_supported(f.src_dtype, f.dst_dtype, f.kx, f.ky, f.kz))
            e = launch_fused2(f, s);
        else if (pl.acc == Acc::I32 && fused_u8_supported(f))
            e = launch_fused_u8(f, s);
        else
            e = launch_fused(pl.acc, f, s);
        if (e != cudaSuccess) return cuda_fail(e, "fused kernel");
        return NDLGPU_OK;
    }
    const int R = (int)c.ax.size();
    std::vector<int64_t> sst(R), dst_st(R);
    for (int i = 0; i < R; i++) {
        sst[i] = c.ax[i].ss;
        dst_st[i] = c.ax[i].ds;
    }
    const size_t need = plan_workspace(c, pl);
    Scratch sc;
    ndlgpu_status st = get_scratch(need, ws, ws_bytes, s, &sc);
    if (st != NDLGPU_OK) return st;
    char* buf[2] = {nullptr, nullptr};
    if (pl.nscratch >= 1) buf[0] = (char*)sc.base;
    if (pl.nscratch >= 2) buf[1] = (char*)sc.base + align_up((size_t)c.total * dtype_size(pl.scratch_dtype));
    const std::vector<int64_t> cst = contiguous_strides(c);

    const int np = (int)c.passes.size();
    if (np == 0) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "no passes");
    const bool integral_dst = dtype_integral(c.ddt);
    const char* in = c.src;
    int in_dt = c.sdt;
    std::vector<int64_t> in_st = sst;
    for (int p = 0; p < np; p++) {
        const bool last = (p == np - 1);
        char* out = last ? c.dst : buf[p % 2];
        const int out_dt = last ? c.ddt : pl.scratch_dtype;
        const std::vector<int64_t>& out_st = last ? dst_st : cst;
        int mode;
        int shift = 0;
        std::vector<int32_t> num;
        if (pl.acc == Acc::I32) {
            shift = dyadic_shift(c.passes[p].w, &num);
        }
        if (compose == NDLGPU_CAST_EACH || np == 1) {
            mode = STORE_CAST;
        } else if (!last) {
            mode = (pl.acc == Acc::I32) ? STORE_RAW : STORE_CAST;
        } else {
            mode = integral_dst ? STORE_ROUND : STORE_CAST;
        }
        if (pl.acc == Acc::I32 && compose != NDLGPU_CAST_EACH && np > 1) {
            // raw integer sums carry the scale until the last pass
            if (!last) shift = 0;
            else {
                shift = 0;
                for (int q = 0; q < np; q++) shift += dyadic_shift(c.passes[q].w, nullptr);
            }
        }
        ndlgpu_status r = run_generic_pass(pl.acc, c, c.passes[p], in, in_dt, in_st, out, out_dt, out_st, border,
                                           mode, shift, num, s);
        if (r != NDLGPU_OK) return r;
        in = out;
        in_dt = out_dt;
        in_st = out_st;
    }
    return NDLGPU_OK;
}

// ---------------------------------------------------------------------------
// Gaussian weights: processing/convolution.h:116-126 with the radius rule
// _kernelSize(sigma) = _ceil(3.0f * sigma) of mathHelpers.h:17-18.
// ---------------------------------------------------------------------------

static int kernel_size(double sigma)
{
    const double num = 3.0f * sigma;
    const int t = static_cast<int>(num);
    return (static_cast<double>(t) == num) ? t : t + ((num > 0) ? 1 : 0);
}

static std::vector<double> gaussian_taps(double sigma)
{
    const int radius = kernel_size(sigma);
    const int width = 2 * radius + 1;
    std::vector<double> w((size_t)width);
    double wsum = 0;
    for (int i = 0; i < width; i++) {
        const double d = i - radius;
        w[i] = std::exp(-(d * d) / (2 * sigma * sigma));
        wsum += w[i];
    }
    for (auto& x : w) x /= wsum;
    return w;
}

// ---------------------------------------------------------------------------
// Shared front end of the pass-chain entry points
// ---------------------------------------------------------------------------

static ndlgpu_status prepare(const ndlgpu_view* src, const ndlgpu_view* dst, const std::vector<LPass>& lp,
                             int border, int compose, int precision, Canon* c, Plan* pl)
{
    ndlgpu_status st;
    if ((st = check_view(src, "src", true)) != NDLGPU_OK) return st;
    if ((st = check_view(dst, "dst", true)) != NDLGPU_OK) return st;
    if ((st = check_pair(src, dst)) != NDLGPU_OK) return st;
    if (compose != NDLGPU_ROUND_ONCE && compose != NDLGPU_CAST_EACH)
        return fail(NDLGPU_ERR_INVALID_ARGUMENT, "unknown compose mode");
    if (precision < NDLGPU_PREC_AUTO || precision > NDLGPU_PREC_EXACT)
        return fail(NDLGPU_ERR_INVALID_ARGUMENT, "unknown precision");
    if (lp.empty()) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "at least one pass is required");
    if ((st = canonicalise(src, dst, lp, border, c)) != NDLGPU_OK) return st;
    if (c->total == 0) return NDLGPU_OK;
    return plan(*c, compose, precision, border, pl);
}

static ndlgpu_status lpasses_from(int npass, const ndlgpu_axis_kernel* passes, std::vector<LPass>* out)
{
    if (npass < 1 || !passes) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "npass must be >= 1 and passes non-NULL");
    for (int i = 0; i < npass; i++) {
        const ndlgpu_axis_kernel& k = passes[i];
        if (k.ntaps < 1 || !k.taps) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "a pass has no taps");
        if (k.ntaps > kMaxTaps) return fail(NDLGPU_ERR_TOO_MANY_TAPS, "a pass has more than 255 taps");
        if (k.reserved != 0) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "ndlgpu_axis_kernel.reserved must be 0");
        LPass lp;
        lp.axis = k.axis;
        lp.center = k.center;
        lp.taps.assign(k.taps, k.taps + k.ntaps);
        out->push_back(lp);
    }
    return NDLGPU_OK;
}

static ndlgpu_status gaussian_passes(const ndlgpu_view* src, const double* sigma, bool per_axis,
                                     std::vector<LPass>* out)
{
    if (!src || src->rank < 1 || src->rank > kMaxRank) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "bad src view");
    for (int a = 0; a < src->rank; a++) {
        const double s = per_axis ? sigma[a] : sigma[0];
        if (per_axis && s == 0.0) continue;
        if (!(s > 0) || !std::isfinite(s)) return fail(NDLGPU_ERR_BAD_SIGMA, "sigma must be positive and finite (convolution.h:112)");
        LPass lp;
        lp.axis = a;
        lp.taps = gaussian_taps(s);
        lp.center = (int)lp.taps.size() / 2;
        if ((int)lp.taps.size() > kMaxTaps) return fail(NDLGPU_ERR_TOO_MANY_TAPS, "sigma too large (more than 255 taps)");
        out->push_back(lp);
    }
    if (out->empty()) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "every sigma is zero");
    return NDLGPU_OK;
}

// ---------------------------------------------------------------------------
// Host reading of a kernel view (ndlgpu_convolve's kernel is host memory)
// ---------------------------------------------------------------------------

static double host_value(const ndlgpu_view* k, int64_t off)
{
    const char* b = (const char*)k->data;
    switch (k->dtype) {
    case NDLGPU_U8: return ((const uint8_t*)b)[off];
    case NDLGPU_I8: return ((const int8_t*)b)[off];
    case NDLGPU_U16: return ((const uint16_t*)b)[off];
    case NDLGPU_I16: return ((const int16_t*)b)[off];
    case NDLGPU_I32: return ((const int32_t*)b)[off];
    case NDLGPU_U32: return ((const uint32_t*)b)[off];
    case NDLGPU_I64: return (double)((const int64_t*)b)[off];
    case NDLGPU_U64: return (double)((const uint64_t*)b)[off];
    case NDLGPU_F32: return ((const float*)b)[off];
    case NDLGPU_F64: return ((const double*)b)[off];
    case NDLGPU_F16: {
        uint16_t h = ((const uint16_t*)b)[off];
        const int e = (h >> 10) & 31, m = h & 1023;
        const double sgn = (h & 0x8000) ? -1.0 : 1.0;
        if (e == 0) return sgn * std::ldexp((double)m, -24);
        if (e == 31) return m ? NAN : sgn * INFINITY;
        return sgn * std::ldexp((double)(m | 1024), e - 25);
    }
    default: {
        uint32_t u = (uint32_t)((const uint16_t*)b)[off] << 16;
        float f;
        std::memcpy(&f, &u, 4);
        return f;
    }
    }
}


// ---------------------------------------------------------------------------
// Adjoint (input and tap gradients of a ROUND_ONCE pass chain)
// ---------------------------------------------------------------------------

struct AdjPlan {
    Acc acc;
    int R;
    int64_t total;
    std::vector<CPass> fwd;        // forward passes (zero taps skipped)
    std::vector<CPass> all;        // every tap, original order (tap gradients)
    int nF = 0, nB = 0;
    unsigned nblocks = 0;
    int maxk = 0;
    size_t elem_bytes = 0;
};

static bool float_dtype(int dt) { return dt == NDLGPU_F32 || dt == NDLGPU_F64 || dt == NDLGPU_F16 || dt == NDLGPU_BF16; }

static ndlgpu_status adjoint_prepare(const ndlgpu_view* g, const ndlgpu_view* x, const ndlgpu_view* gx, int npass,
                                     const ndlgpu_axis_kernel* passes, int border, bool want_taps, int tdt,
                                     AdjPlan* ap)
{
    ndlgpu_status st;
    if ((st = check_view(g, "grad_out", true)) != NDLGPU_OK) return st;
    if (x && (st = check_view(x, "src", true)) != NDLGPU_OK) return st;
    if (gx && (st = check_view(gx, "grad_src", true)) != NDLGPU_OK) return st;
    if (want_taps && !x) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "tap gradients need the forward input (src)");
    if (want_taps && tdt != NDLGPU_F32 && tdt != NDLGPU_F64)
        return fail(NDLGPU_ERR_UNSUPPORTED_DTYPE, "grad_taps must be F32 or F64");
    if (!float_dtype(g->dtype) || (x && !float_dtype(x->dtype)) || (gx && !float_dtype(gx->dtype)))
        return fail(NDLGPU_ERR_UNSUPPORTED_DTYPE, "the adjoint takes floating-point images");
    if (border < NDLGPU_CLAMP || border > NDLGPU_REFLECT) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "unknown border mode");
    if (x && (st = check_pair(x, g)) != NDLGPU_OK) return st;
    if (gx && (st = check_pair(g, gx)) != NDLGPU_OK) return st;
    if (gx && x) {
        intptr_t a0, a1, b0, b1;
        view_bytes(x, &a0, &a1);
        view_bytes(gx, &b0, &b1);
        if (view_count(x) > 0 && a0 < b1 && b0 < a1) return fail(NDLGPU_ERR_ALIASING, "src and grad_src overlap");
    }
    std::vector<LPass> lp;
    if ((st = lpasses_from(npass, passes, &lp)) != NDLGPU_OK) return st;
    ap->R = g->rank;
    ap->total = view_count(g);
    bool f64 = g->dtype == NDLGPU_F64 || (x && x->dtype == NDLGPU_F64) || (gx && gx->dtype == NDLGPU_F64);
    ap->acc = f64 ? Acc::F64 : Acc::F32;
    for (const LPass& p : lp) {
        if (p.axis < 0 || p.axis >= ap->R) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "pass axis out of range");
        CPass f, a;
        f.axis = a.axis = p.axis;
        for (int k = 0; k < (int)p.taps.size(); k++) {
            const int o = k - p.center;
            if (border != NDLGPU_CLAMP && ap->total > 0 && (o > g->extent[p.axis] || o < -g->extent[p.axis]))
                return fail(NDLGPU_ERR_RADIUS_EXCEEDS_EXTENT, "tap offset exceeds the extent (Wrap/Reflect map one period only)");
            a.off.push_back(o);
            a.w.push_back(p.taps[k]);
            if (p.taps[k] != 0.0) {
                f.off.push_back(o);
                f.w.push_back(p.taps[k]);
            }
        }
        ap->maxk = std::max(ap->maxk, (int)a.off.size());
        ap->fwd.push_back(f);
        ap->all.push_back(a);
    }
    if (ap->total >= (int64_t(1) << 31))
        return fail(NDLGPU_ERR_INDEX_OVERFLOW, "the adjoint supports images of fewer than 2^31 elements");
    const int n = (int)lp.size();
    ap->nF = want_taps ? n - 1 : 0;
    ap->nB = (n > 1) ? std::min(2, n - 1) : 0;
    ap->elem_bytes = align_up((size_t)ap->total * dtype_size(acc_dtype(ap->acc)));
    ap->nblocks = want_taps && ap->total > 0 ? tap_grad_blocks((uint32_t)ap->total) : 0;
    return NDLGPU_OK;
}

static size_t adjoint_workspace(const AdjPlan& ap)
{
    if (ap.total == 0) return 0;
    return (size_t)(ap.nF + ap.nB) * ap.elem_bytes + align_up((size_t)ap.nblocks * ap.maxk * sizeof(double));
}

// Fused input gradient (float types, up to three dense odd-tap passes on
// distinct axes): the transposed chain in one kernel.
static bool plan_fused_adjoint(const ndlgpu_view* g, const ndlgpu_view* gx, int npass,
                               const ndlgpu_axis_kernel* passes, int border, FusedParams* fp)
{
    if (!float_dtype(g->dtype) || !float_dtype(gx->dtype) || g->dtype == NDLGPU_F64 || gx->dtype == NDLGPU_F64)
        return false;
    std::vector<LPass> lp;
    const std::string keep = t_last_error;
    if (lpasses_from(npass, passes, &lp) != NDLGPU_OK) { t_last_error = keep; return false; }
    for (auto& p : lp)
        for (double w : p.taps)
            if (w == 0.0) return false;    // every tap must be present in the fused tap window
    Canon c;
    if (canonicalise(g, gx, lp, border, &c) != NDLGPU_OK || c.total == 0) { t_last_error = keep; return false; }
    return plan_fused(c, Acc::F32, NDLGPU_ROUND_ONCE, border, fp, 1);
}

// Fused tap gradients: three dense odd-tap passes on distinct axes, X and G
// of one float type.  Returns false (and leaves no error) when not eligible.
struct FusedTap {
    TapFusedParams tp;
    TapFinalMap map;
    long long ncta = 0;
};

static bool plan_fused_tapgrad(const ndlgpu_view* g, const ndlgpu_view* x, int npass,
                               const ndlgpu_axis_kernel* passes, int border, FusedTap* ft)
{
    if (!x || x->dtype != g->dtype) return false;
    if (x->dtype != NDLGPU_F32 && x->dtype != NDLGPU_BF16 && x->dtype != NDLGPU_F16) return false;
    // three passes (volumes), or two (images: the planes the kernel streams
    // are then an axis without a pass, run as a one-tap unit pass whose
    // gradient is not reported)
    if (npass != 3 && npass != 2) return false;
    const std::string keep = t_last_error;
    std::vector<LPass> lp;
    if (lpasses_from(npass, passes, &lp) != NDLGPU_OK) { t_last_error = keep; return false; }
    Canon c;
    if (canonicalise(x, g, lp, border, &c, true) != NDLGPU_OK || c.total == 0) { t_last_error = keep; return false; }
    const int R = (int)c.ax.size();
    std::vector<int> pass_of(R, -1);
    for (int i = 0; i < npass; i++) {
        if (pass_of[c.passes[i].axis] >= 0) return false;
        pass_of[c.passes[i].axis] = i;
    }
    if (pass_of[0] < 0) return false;
    std::vector<int> others;
    for (int i = 1; i < R; i++)
        if (pass_of[i] >= 0) others.push_back(i);
    if ((int)others.size() != npass - 1) return false;
    // images: Z is the first axis without a pass (-1: a single plane)
    int zrole = npass == 3 ? others[1] : -1;
    if (npass == 2)
        for (int i = 1; i < R && zrole < 0; i++)
            if (pass_of[i] < 0) zrole = i;
    const int role[3] = {0, others[0], zrole};
    int K[3] = {1, 1, 1};
    for (int r = 0; r < 3; r++) {
        if (role[r] < 0 || pass_of[role[r]] < 0) continue;   // the unit pass
        std::vector<int> o = c.passes[pass_of[role[r]]].off;
        std::sort(o.begin(), o.end());
        const int k = (int)o.size();
        if (k % 2 == 0 || k > 17) return false;
        for (int i = 0; i < k; i++)
            if (o[i] != i - k / 2) return false;
        K[r] = k;
    }
    if (!tapgrad_supported(x->dtype, K[0], K[1], K[2])) return false;
    TapFusedParams& p = ft->tp;
    std::memset(&p, 0, sizeof(p));
    p.x = c.src;
    p.g = c.dst;
    p.x_dtype = x->dtype;
    p.border = border;
    p.zero_pad = border != NDLGPU_WRAP;
    const CAxis& ax0 = c.ax[role[0]];
    const CAxis& ay = c.ax[role[1]];
    const CAxis unit{1, 0, 0, -1};
    const CAxis& az = role[2] >= 0 ? c.ax[role[2]] : unit;
    p.nx = (int)ax0.n; p.ny = (int)ay.n; p.nz = (int)az.n;
    p.sx = ax0.ss; p.sy = ay.ss; p.sz = az.ss;
    p.gxs = ax0.ds; p.gy = ay.ds; p.gz = az.ds;
    int64_t nb = 1, sb = 0, gb = 0;
    for (int i = 0; i < R; i++) {
        if (i == role[0] || i == role[1] || i == role[2]) continue;
        if (nb == 1) { nb = c.ax[i].n; sb = c.ax[i].ss; gb = c.ax[i].ds; continue; }
        if (c.ax[i].ss != sb * nb || c.ax[i].ds != gb * nb) return false;
        nb *= c.ax[i].n;
    }
    if (nb > 0x7fffffffLL) return false;
    p.nbatch = (int)nb;
    p.sb = sb;
    p.gb = gb;
    if ((__int128)(p.ny - 1) * p.sy + (__int128)(p.nx - 1) * p.sx >= ((__int128)1 << 31)) return false;
    p.kx = K[0]; p.ky = K[1]; p.kz = K[2];
    const int es = dtype_size(x->dtype);
    auto al = [](const void* ptr, int64_t bytes) { return ((uintptr_t)ptr % (uintptr_t)bytes) == 0; };
    p.vec_ld = (p.sx == 1 && al(p.x, 16) && (p.sy * es) % 16 == 0 && (p.sz * es) % 16 == 0 && (p.sb * es) % 16 == 0);
    p.vec_g = (p.gxs == 1 && al(p.g, 4 * es) && p.gy % 4 == 0 && p.gz % 4 == 0 && p.gb % 4 == 0);
    // taps ascending by canonical offset; output slot of each: the original
    // pass and tap index (offsets were negated on axes flipped above)
    size_t base[3] = {0, 0, 0};
    {
        size_t off = 0;
        for (int i = 0; i < npass; i++) { base[i] = off; off += (size_t)passes[i].ntaps; }
    }
    float* wdst[3] = {p.wxf, p.wyf, p.wzf};
    int t = 0;
    for (int r = 0; r < 3; r++) {
        if (role[r] < 0 || pass_of[role[r]] < 0) {
            // the unit pass of an image: weight 1, gradient discarded
            wdst[r][0] = 1.f;
            ft->map.dst[t++] = -1;
            continue;
        }
        const int pi = pass_of[role[r]];
        const CPass& cp = c.passes[pi];
        const int la = passes[pi].axis;
        const bool flipped = x->stride[la] < 0;
        std::vector<std::pair<int, double>> tw;
        for (size_t i = 0; i < cp.off.size(); i++) tw.push_back({cp.off[i], cp.w[i]});
        std::sort(tw.begin(), tw.end());
        for (int k = 0; k < K[r]; k++) {
            wdst[r][k] = (float)tw[k].second;
            const int o_orig = flipped ? -tw[k].first : tw[k].first;
            const int k_orig = o_orig + passes[pi].center;
            if (k_orig < 0 || k_orig >= passes[pi].ntaps) return false;
            ft->map.dst[t++] = (int)base[pi] + k_orig;
        }
    }
    for (int k = 0; k < 40; k++) {
        const float wx = k < p.kx ? p.wxf[k] : 0.f, wy = k < p.ky ? p.wyf[k] : 0.f;
        const float wz = k < p.kz ? p.wzf[p.kz - 1 - k] : 0.f;
        p.wx2[k] = make_float2(wx, wx);
        p.wy2[k] = make_float2(wy, wy);
        p.wzr2[k] = make_float2(wz, wz);
    }
    p.zchunk = tapgrad_zchunk(p.nx, p.ny, p.nz, p.nbatch, p.kz);
    ft->ncta = tapgrad_ctas(p);
    return true;
}

static ndlgpu_status adjoint_execute(const ndlgpu_view* g, const ndlgpu_view* x, const ndlgpu_view* gx,
                                     int border, void* grad_taps, int tdt, const AdjPlan& ap, void* ws,
                                     size_t ws_bytes, cudaStream_t s, const FusedParams* fused_gx = nullptr,
                                     FusedTap* fused_tap = nullptr)
{
    if (ap.total == 0) return NDLGPU_OK;
    if (fused_gx && !grad_taps) {
        cudaError_t e = launch_fused2(*fused_gx, s);
        if (e != cudaSuccess) return cuda_fail(e, "fused adjoint");
        return NDLGPU_OK;
    }
    if (fused_tap && grad_taps && (fused_gx || !gx)) {
        const size_t need = align_up((size_t)fused_tap->ncta * (fused_tap->tp.kx + fused_tap->tp.ky + fused_tap->tp.kz) *
                                     sizeof(double));
        Scratch sc;
        ndlgpu_status st = get_scratch(need, ws, ws_bytes, s, &sc);
        if (st != NDLGPU_OK) return st;
        fused_tap->tp.partial = (double*)sc.base;
        cudaError_t e = launch_tapgrad(fused_tap->tp, grad_taps, tdt, fused_tap->map, s);
        if (e != cudaSuccess) return cuda_fail(e, "fused tap gradients");
        if (fused_gx) {
            e = launch_fused2(*fused_gx, s);
            if (e != cudaSuccess) return cuda_fail(e, "fused adjoint");
        }
        return NDLGPU_OK;
    }
    Scratch sc;
    ndlgpu_status st = get_scratch(adjoint_workspace(ap), ws, ws_bytes, s, &sc);
    if (st != NDLGPU_OK) return st;
    const int n = (int)ap.fwd.size();
    const int adt = acc_dtype(ap.acc);
    Canon geo;   // logical axis order, no flips: the general kernels take any strides
    geo.total = ap.total;
    for (int i = 0; i < ap.R; i++) geo.ax.push_back(CAxis{g->extent[i], 0, 0, i});
    std::vector<int64_t> cst = contiguous_strides(geo);
    auto strides_of = [&](const ndlgpu_view* v) {
        std::vector<int64_t> r(ap.R);
        for (int i = 0; i < ap.R; i++) r[i] = v->stride[i];
        return r;
    };
    char* base = (char*)sc.base;
    std::vector<char*> F(ap.nF), B(ap.nB);
    for (int i = 0; i < ap.nF; i++) F[i] = base + (size_t)i * ap.elem_bytes;
    for (int i = 0; i < ap.nB; i++) B[i] = base + (size_t)(ap.nF + i) * ap.elem_bytes;
    double* partial = (double*)(base + (size_t)(ap.nF + ap.nB) * ap.elem_bytes);
    const std::vector<int32_t> none;

    // forward intermediates (inputs of passes 1..n-1)
    std::vector<const char*> in_ptr(n, nullptr);
    std::vector<int> in_dt(n, adt);
    std::vector<std::vector<int64_t>> in_st(n, cst);
    if (grad_taps) {
        in_ptr[0] = (const char*)x->data;
        in_dt[0] = x->dtype;
        in_st[0] = strides_of(x);
        for (int p = 0; p + 1 < n; p++) {
            st = run_generic_pass(ap.acc, geo, ap.fwd[p], in_ptr[p], in_dt[p], in_st[p], F[p], adt, cst, border,
                                  STORE_CAST, 0, none, s);
            if (st != NDLGPU_OK) return st;
            in_ptr[p + 1] = F[p];
        }
    }
    // backward sweep
    const char* gcur = (const char*)g->data;
    int gdt = g->dtype;
    std::vector<int64_t> gst = strides_of(g);
    size_t tap_off = 0;
    std::vector<size_t> tap_base(n, 0);
    for (int p = 0; p < n; p++) { tap_base[p] = tap_off; tap_off += ap.all[p].off.size(); }
    const int tes = (tdt == NDLGPU_F64) ? 8 : 4;
    for (int p = n - 1; p >= 0; p--) {
        if (grad_taps) {
            TapGradParams tp;
            std::memset(&tp, 0, sizeof(tp));
            tp.g = gcur;
            tp.x = in_ptr[p];
            tp.partial = partial;
            tp.g_dtype = gdt;
            tp.x_dtype = in_dt[p];
            tp.rank = ap.R;
            tp.axis = ap.all[p].axis;
            tp.ntap = (int)ap.all[p].off.size();
            tp.border = border;
            tp.total = (uint32_t)ap.total;
            for (int i = 0; i < ap.R; i++) {
                tp.n[i] = g->extent[i];
                tp.gs[i] = gst[i];
                tp.xs[i] = in_st[p][i];
                tp.div[i].init((uint32_t)g->extent[i]);
            }
            for (int t = 0; t < tp.ntap; t++) tp.off[t] = ap.all[p].off[t];
            cudaError_t e = launch_tap_grad(ap.acc, tp, ap.nblocks, (char*)grad_taps + tap_base[p] * tes, tdt, s);
            if (e != cudaSuccess) return cuda_fail(e, "tap gradient");
        }
        char* gnext;
        int ndt;
        std::vector<int64_t> nst;
        if (p > 0) {
            // the intermediates alternate between the nB = min(2, n - 1)
            // buffers, the first pass (p = n - 1) writing B[0]
            gnext = B[(n - 1 - p) % 2];
            ndt = adt;
            nst = cst;
        } else if (gx) {
            gnext = (char*)gx->data;
            ndt = gx->dtype;
            nst = strides_of(gx);
        } else {
            break;
        }
        st = run_generic_pass(ap.acc, geo, ap.fwd[p], gcur, gdt, gst, gnext, ndt, nst, border, STORE_CAST, 0, none, s,
                              true);
        if (st != NDLGPU_OK) return st;
        gcur = gnext;
        gdt = ndt;
        gst = nst;
    }
    return NDLGPU_OK;
}


// ---------------------------------------------------------------------------
// Batched form
// ---------------------------------------------------------------------------

struct BatchHost {
    int dtype = -1;
    std::vector<BatchDesc> descs;
    std::vector<float> zones;
    std::vector<int64_t> elems;
    int cfg = -1;
    BatchLaunch L{};
    int nitems = 0;
    bool planned = false;
    BatchDesc* d_descs = nullptr;
    int4* d_items = nullptr;
    float* d_zones = nullptr;
    int* d_counter = nullptr;
    float* d_scratch = nullptr;
    size_t counter_ints = 0;
    cudaGraphExec_t gexec = nullptr;
    cudaGraph_t graph = nullptr;
    void release()
    {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        gexec = nullptr;
        graph = nullptr;
        if (d_descs) cudaFree(d_descs);
        if (d_items) cudaFree(d_items);
        if (d_zones) cudaFree(d_zones);
        if (d_counter) cudaFree(d_counter);
        if (d_scratch) cudaFree(d_scratch);
        d_scratch = nullptr;
        d_descs = nullptr;
        d_items = nullptr;
        d_zones = nullptr;
        d_counter = nullptr;
        planned = false;
    }
};

static ndlgpu_status batch_add(BatchHost* b, const ndlgpu_view* src, const ndlgpu_view* dst, int npass,
                               const ndlgpu_axis_kernel* passes, int border, int adjoint)
{
    ndlgpu_status st;
    if ((st = check_view(src, "src", true)) != NDLGPU_OK) return st;
    if ((st = check_view(dst, "dst", true)) != NDLGPU_OK) return st;
    if ((st = check_pair(src, dst)) != NDLGPU_OK) return st;
    if (src->dtype != dst->dtype || (src->dtype != NDLGPU_F32 && src->dtype != NDLGPU_BF16 && src->dtype != NDLGPU_F16))
        return fail(NDLGPU_ERR_UNSUPPORTED_DTYPE, "batched instances are F32, BF16 or F16, src and dst alike");
    if (b->dtype >= 0 && b->dtype != src->dtype)
        return fail(NDLGPU_ERR_UNSUPPORTED_DTYPE, "all instances of a batch share one storage type");
    if (border < NDLGPU_CLAMP || border > NDLGPU_REFLECT) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "unknown border mode");
    if (adjoint != 0 && adjoint != 1) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "adjoint must be 0 or 1");
    if (npass > 3) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "a batched instance has at most three passes");
    std::vector<LPass> lp;
    if ((st = lpasses_from(npass, passes, &lp)) != NDLGPU_OK) return st;
    Canon c;
    if ((st = canonicalise(src, dst, lp, border, &c, true)) != NDLGPU_OK) return st;
    if (c.total == 0) return NDLGPU_OK;
    const int R = (int)c.ax.size();
    std::vector<const CPass*> by_axis(R, nullptr);
    for (auto& p : c.passes) {
        if (by_axis[p.axis]) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "two passes on one axis of a batched instance");
        by_axis[p.axis] = &p;
    }
    std::vector<int> others;
    for (int i = 1; i < R; i++)
        if (by_axis[i]) others.push_back(i);
    for (int i = 1; i < R && others.size() < 2; i++)
        if (!by_axis[i] && std::find(others.begin(), others.end(), i) == others.end()) others.push_back(i);
    std::sort(others.begin(), others.end());
    int role[3] = {0, others.size() > 0 ? others[0] : -1, others.size() > 1 ? others[1] : -1};
    BatchDesc d;
    std::memset(&d, 0, sizeof(d));
    d.src = c.src;
    d.dst = c.dst;
    d.border = border;
    d.zero_pad = (adjoint && border != NDLGPU_WRAP) ? 1 : 0;
    d.zone_x = d.zone_y = d.zone_z = -1;
    int* nn[3] = {&d.nx, &d.ny, &d.nz};
    long long* ss[3] = {&d.sx, &d.sy, &d.sz};
    long long* ds[3] = {&d.dx, &d.dy, &d.dz};
    int* bb[3] = {&d.bx, &d.by, &d.bz};
    int* rr[3] = {&d.rx, &d.ry, &d.rz};
    float* ww[3] = {d.wx, d.wy, d.wz};
    int* zz[3] = {&d.zone_x, &d.zone_y, &d.zone_z};
    bool has_pass[3] = {false, false, false};
    for (int r = 0; r < 3; r++) {
        if (role[r] < 0) { *nn[r] = 1; *ss[r] = 0; *ds[r] = 0; *bb[r] = 1; *rr[r] = 0; ww[r][0] = 1.f; continue; }
        const CAxis& a = c.ax[role[r]];
        if (a.n > 0x7fffffffLL) return fail(NDLGPU_ERR_INDEX_OVERFLOW, "extent too large");
        *nn[r] = (int)a.n;
        *ss[r] = a.ss;
        *ds[r] = a.ds;
        const CPass* cp = by_axis[role[r]];
        if (!cp) { *bb[r] = 1; *rr[r] = 0; ww[r][0] = 1.f; continue; }
        std::vector<std::pair<int, double>> t;
        for (size_t i = 0; i < cp->off.size(); i++) t.push_back({cp->off[i], cp->w[i]});
        std::sort(t.begin(), t.end());
        const int K = (int)t.size();
        for (int i = 0; i < K; i++)
            if (K % 2 == 0 || t[i].first != i - K / 2)
                return fail(NDLGPU_ERR_INVALID_ARGUMENT, "batched passes need odd, centred tap lists");
        const int B = batch_bucket(K);
        if (B < 0 || K > kBatchMaxTaps) return fail(NDLGPU_ERR_TOO_MANY_TAPS, "batched passes have at most 37 taps");
        if (K / 2 > a.n && border != NDLGPU_CLAMP)
            return fail(NDLGPU_ERR_RADIUS_EXCEEDS_EXTENT, "a Wrap/Reflect pass's radius exceeds its axis extent");
        has_pass[r] = true;
        *bb[r] = B;
        *rr[r] = K / 2;
        const int pad = (B - K) / 2;
        for (int m = 0; m < B; m++) ww[r][m] = 0.f;
        for (int k = 0; k < K; k++) ww[r][pad + k] = (float)t[k].second;
        if (adjoint) std::reverse(ww[r], ww[r] + B);
        if (d.zero_pad && K > 1) {
            std::vector<float> rows;
            zone_rows(a.n, border, t, B, K / 2, &rows);
            *zz[r] = (int)b->zones.size();
            b->zones.insert(b->zones.end(), rows.begin(), rows.end());
        }
    }
    d.nphase = 0;
    for (int r = 0; r < 3; r++)
        if (has_pass[r]) d.pax[d.nphase++] = r;
    if (d.nphase == 0) d.pax[d.nphase++] = 0;   // no pass: one identity X pass (a copy)
    d.scr[0] = d.scr[1] = -1;
    int64_t nb = 1, sb = 0, db = 0;
    for (int i = 0; i < R; i++) {
        if (i == role[0] || i == role[1] || i == role[2]) continue;
        if (nb == 1) { nb = c.ax[i].n; sb = c.ax[i].ss; db = c.ax[i].ds; continue; }
        if (c.ax[i].ss != sb * nb || c.ax[i].ds != db * nb)
            return fail(NDLGPU_ERR_INVALID_ARGUMENT, "the untouched axes of a batched instance must merge into one");
        nb *= c.ax[i].n;
    }
    if (nb > 0x7fffffffLL) return fail(NDLGPU_ERR_INDEX_OVERFLOW, "batch axis too large");
    d.nb = (int)nb;
    d.sb = sb;
    d.db = db;
    const int es = dtype_size(src->dtype);
    auto al = [](const void* ptr, int64_t bytes) { return ((uintptr_t)ptr % (uintptr_t)bytes) == 0; };
    d.vec_ld = (d.sx == 1 && al(d.src, 16) && (d.sy * es) % 16 == 0 && (d.sz * es) % 16 == 0 && (d.sb * es) % 16 == 0);
    d.vec_st = (d.dx == 1 && al(d.dst, 2 * es) && d.dy % 2 == 0 && d.dz % 2 == 0 && d.db % 2 == 0);
    b->dtype = src->dtype;
    b->descs.push_back(d);
    b->elems.push_back(c.total);
    b->planned = false;
    return NDLGPU_OK;
}

static ndlgpu_status batch_plan(BatchHost* b, int cfg)
{
    if (cfg < 0) cfg = 0;
    if (cfg >= batch_tile_configs()) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "unknown tile configuration");
    b->release();
    int kout, warps, nt;
    batch_tile_info(cfg, &kout, &warps, &nt);
    const double target = (double)batch_item_outputs(cfg);
    if (b->dtype < 0) b->dtype = NDLGPU_F32;
    // f32 scratch between phases: per instance, one buffer per intermediate,
    // each 256-byte aligned (an L1 line never spans two instances' buffers)
    long long off = 0;
    int bmax = 1;
    for (auto& d : b->descs) {
        const long long el = (long long)((d.nx + 3) / 4 * 4) * d.ny * d.nz * d.nb;   // rows padded to 4 floats
        bmax = std::max(bmax, std::max(d.by, d.bz));
        const long long al = (el + 63) / 64 * 64;
        d.scr[0] = d.scr[1] = -1;
        for (int p = 0; p + 1 < d.nphase; p++) { d.scr[p] = off; off += al; }
    }
    // work items: (instance, phase, first unit, units); rows for the X pass,
    // (64-column block, line, 64-output segment) units for Y and Z
    struct It { int4 v; int phase; double cost; };
    std::vector<It> items;
    const int seg = batch_col_unit();
    for (size_t i = 0; i < b->descs.size(); i++) {
        BatchDesc& d = b->descs[i];
        for (int p = 0; p < d.nphase; p++) {
            const int a = d.pax[p];
            const int B = a == 0 ? d.bx : (a == 1 ? d.by : d.bz);
            long long units, per;
            double unit_out;
            if (a == 0) {
                units = (long long)d.nb * d.nz * d.ny;
                unit_out = d.nx;
            } else {
                const long long n = a == 1 ? d.ny : d.nz;
                const long long lines = (long long)d.nb * (a == 1 ? d.nz : d.ny);
                units = (long long)((d.nx + 63) / 64) * lines * ((n + seg - 1) / seg);
                unit_out = 64.0 * std::min<long long>(n, seg);
            }
            // X: rows shared by the warps of a CTA; Y/Z: whole-CTA units
            per = a == 0 ? std::max<long long>(warps, (long long)std::llround(target / unit_out / warps) * warps)
                         : std::max<long long>(1, (long long)std::llround(target / unit_out));
            int cnt = 0;
            for (long long u = 0; u < units; u += per) {
                const long long k = std::min(per, units - u);
                if (u > 0x7fffffffLL) return fail(NDLGPU_ERR_INDEX_OVERFLOW, "batch instance too large");
                items.push_back({make_int4((int)i, p, (int)u, (int)k), p, (double)k * unit_out * (B + 4)});
                cnt++;
            }
            d.nitems[p] = cnt;
        }
    }
    std::stable_sort(items.begin(), items.end(), [](const It& a, const It& c) {
        return a.phase != c.phase ? a.phase < c.phase : a.cost > c.cost;
    });
    std::vector<int4> iv;
    for (auto& it : items) iv.push_back(it.v);
    b->nitems = (int)iv.size();
    b->cfg = cfg;
    b->L = BatchLaunch{};
    b->L.nitems = b->nitems;
    b->L.stage_bytes = batch_stage_bytes(bmax);
    cudaError_t e = batch_prepare(b->dtype, cfg, &b->L);
    if (e != cudaSuccess) return cuda_fail(e, "batch kernel set-up");
    const size_t nd = std::max<size_t>(1, b->descs.size()), ni = std::max<size_t>(1, iv.size()),
                 nz = std::max<size_t>(1, b->zones.size());
    b->counter_ints = 2 + 3 * nd;
    if ((e = cudaMalloc(&b->d_descs, nd * sizeof(BatchDesc))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_items, ni * sizeof(int4))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_zones, nz * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_counter, b->counter_ints * sizeof(int))) != cudaSuccess ||
        (off > 0 && (e = cudaMalloc(&b->d_scratch, (size_t)off * sizeof(float))) != cudaSuccess)) {
        b->release();
        return cuda_fail(e, "batch tables");
    }
    if (!b->descs.empty())
        e = cudaMemcpy(b->d_descs, b->descs.data(), b->descs.size() * sizeof(BatchDesc), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !iv.empty())
        e = cudaMemcpy(b->d_items, iv.data(), iv.size() * sizeof(int4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !b->zones.empty())
        e = cudaMemcpy(b->d_zones, b->zones.data(), b->zones.size() * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        b->release();
        return cuda_fail(e, "batch table upload");
    }
    b->L.descs = b->d_descs;
    b->L.items = b->d_items;
    b->L.zones = b->d_zones;
    b->L.counter = b->d_counter;
    b->L.scratch = b->d_scratch;
    b->planned = true;
    return NDLGPU_OK;
}

static ndlgpu_status batch_enqueue(BatchHost* b, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(b->d_counter, 0, b->counter_ints * sizeof(int), s);
    if (e != cudaSuccess) return cuda_fail(e, "batch counter reset");
    if (b->nitems == 0) return NDLGPU_OK;
    e = launch_batch(b->dtype, b->cfg, b->L, s);
    if (e != cudaSuccess) return cuda_fail(e, "batch launch");
    return NDLGPU_OK;
}

}  // namespace ndlgpu

using namespace ndlgpu;

struct ndlgpu_batch : ndlgpu::BatchHost {};

extern "C" {

const char* ndlgpu_version(void) { return "ndlgpu 0.1.0 (sm_100a)"; }

const char* ndlgpu_status_string(ndlgpu_status s)
{
    switch (s) {
    case NDLGPU_OK: return "ok";
    case NDLGPU_ERR_INVALID_ARGUMENT: return "invalid argument";
    case NDLGPU_ERR_UNSUPPORTED_DTYPE: return "unsupported dtype";
    case NDLGPU_ERR_EXTENT_MISMATCH: return "extent mismatch";
    case NDLGPU_ERR_RADIUS_EXCEEDS_EXTENT: return "kernel radius exceeds extent";
    case NDLGPU_ERR_ALIASING: return "src and dst overlap";
    case NDLGPU_ERR_INDEX_OVERFLOW: return "index overflow";
    case NDLGPU_ERR_BAD_SIGMA: return "bad sigma";
    case NDLGPU_ERR_WORKSPACE: return "workspace too small";
    case NDLGPU_ERR_CUDA: return "CUDA error";
    case NDLGPU_ERR_OUT_OF_MEMORY: return "out of device memory";
    case NDLGPU_ERR_TOO_MANY_TAPS: return "too many taps";
    case NDLGPU_ERR_DEVICE_CHECK: return "device guard fired";
    }
    return "unknown status";
}

const char* ndlgpu_last_error(void) { return t_last_error.c_str(); }

ndlgpu_status ndlgpu_convolve_axes_workspace_size(const ndlgpu_view* src, const ndlgpu_view* dst, int npass,
                                                  const ndlgpu_axis_kernel* passes, int border, int compose,
                                                  int precision, size_t* bytes)
{
    t_last_error.clear();
    if (!bytes) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "bytes is NULL");
    *bytes = 0;
    std::vector<LPass> lp;
    ndlgpu_status st = lpasses_from(npass, passes, &lp);
    if (st != NDLGPU_OK) return st;
    Canon c;
    Plan pl;
    st = prepare(src, dst, lp, border, compose, precision, &c, &pl);
    if (st != NDLGPU_OK || c.total == 0) return st;
    *bytes = plan_workspace(c, pl);
    return NDLGPU_OK;
}

ndlgpu_status ndlgpu_convolve_axes(const ndlgpu_view* src, const ndlgpu_view* dst, int npass,
                                   const ndlgpu_axis_kernel* passes, int border, int compose, int precision,
                                   void* workspace, size_t workspace_bytes, void* stream)
{
    t_last_error.clear();
    std::vector<LPass> lp;
    ndlgpu_status st = lpasses_from(npass, passes, &lp);
    if (st != NDLGPU_OK) return st;
    Canon c;
    Plan pl;
    st = prepare(src, dst, lp, border, compose, precision, &c, &pl);
    if (st != NDLGPU_OK || c.total == 0) return st;
    return execute(c, pl, compose, border, workspace, workspace_bytes, (cudaStream_t)stream);
}

// The route a gaussian_blur takes; the workspace query and the call both
// ask this, so that the scratch reported is the scratch used.
enum class GaussRoute { Planned, Exact2D, Exact3D };

static GaussRoute gauss_route(const ndlgpu_view* src, const ndlgpu_view* dst, const std::vector<LPass>& lp,
                              const Plan& pl)
{
    // an integer-numerator fused plan is already bit-exact and needs no scratch
    if (pl.fused && pl.acc == Acc::I32) return GaussRoute::Planned;
    const bool isrc = src->dtype == NDLGPU_U8 || src->dtype == NDLGPU_U16 || src->dtype == NDLGPU_I16;
    if (!isrc || !(dtype_integral(dst->dtype) || dst->dtype == NDLGPU_F64)) return GaussRoute::Planned;
    if (src->rank != (int)lp.size() || (lp.size() != 2 && lp.size() != 3)) return GaussRoute::Planned;
    for (size_t i = 0; i < lp.size(); i++)
        if (lp[i].axis != (int)i) return GaussRoute::Planned;
    if (lp[0].taps.size() > 61 || lp[1].taps.size() > 61) return GaussRoute::Planned;
    if (src->extent[0] > 0x7fffffffLL || src->extent[1] > 0x7fffffffLL) return GaussRoute::Planned;
    if (lp.size() == 2) return GaussRoute::Exact2D;
    if (lp[2].taps.size() > 128 || src->extent[2] > 65535) return GaussRoute::Planned;
    if (view_count(src) >= (int64_t(1) << 31)) return GaussRoute::Planned;
    return GaussRoute::Exact3D;
}

static size_t gauss_workspace(const ndlgpu_view* src, const ndlgpu_view* dst, const std::vector<LPass>& lp,
                              const Canon& c, const Plan& pl)
{
    switch (gauss_route(src, dst, lp, pl)) {
    case GaussRoute::Exact2D: return 0;
    case GaussRoute::Exact3D: return align_up((size_t)view_count(src) * sizeof(double));
    default: return plan_workspace(c, pl);
    }
}

ndlgpu_status ndlgpu_gaussian_blur_workspace_size(const ndlgpu_view* src, const ndlgpu_view* dst, double sigma,
                                                  int border, size_t* bytes)
{
    t_last_error.clear();
    if (!bytes) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "bytes is NULL");
    *bytes = 0;
    std::vector<LPass> lp;
    ndlgpu_status st = gaussian_passes(src, &sigma, false, &lp);
    if (st != NDLGPU_OK) return st;
    Canon c;
    Plan pl;
    st = prepare(src, dst, lp, border, NDLGPU_ROUND_ONCE, NDLGPU_PREC_AUTO, &c, &pl);
    if (st != NDLGPU_OK || c.total == 0) return st;
    *bytes = gauss_workspace(src, dst, lp, c, pl);
    return NDLGPU_OK;
}

// 2-D integral images (at most 16 bits) blurred into an integral or f64
// image: the reference's double arithmetic in one fused kernel
// (gauss_exact.cu).  False when not eligible.
static ndlgpu_status gauss3d_exact(const ndlgpu_view* src, const ndlgpu_view* dst, const std::vector<LPass>& lp,
                                   int border, void* ws, size_t ws_bytes, cudaStream_t s, bool* done);

static bool gauss2d_exact(const ndlgpu_view* src, const ndlgpu_view* dst, const std::vector<LPass>& lp, int border,
                          cudaStream_t s, cudaError_t* err)
{
    if (src->rank != 2 || lp.size() != 2) return false;
    if (src->dtype != NDLGPU_U8 && src->dtype != NDLGPU_U16 && src->dtype != NDLGPU_I16) return false;
    if (!(dtype_integral(dst->dtype) || dst->dtype == NDLGPU_F64)) return false;
    if (lp[0].axis != 0 || lp[1].axis != 1) return false;
    const int kx = (int)lp[0].taps.size(), ky = (int)lp[1].taps.size();
    if (kx > 61 || ky > 61) return false;
    if (src->extent[0] > 0x7fffffffLL || src->extent[1] > 0x7fffffffLL) return false;
    GaussExactParams p;
    std::memset(&p, 0, sizeof(p));
    p.src = static_cast<const char*>(src->data);
    p.dst = static_cast<char*>(dst->data);
    p.sdt = src->dtype;
    p.ddt = dst->dtype;
    p.des = dtype_size(dst->dtype);
    p.nx = (int)src->extent[0];
    p.ny = (int)src->extent[1];
    p.nb = 1;
    p.sx = src->stride[0];
    p.sy = src->stride[1];
    p.dx = dst->stride[0];
    p.dy = dst->stride[1];
    p.kx = kx;
    p.ky = ky;
    p.cx = lp[0].center;
    p.cy = lp[1].center;
    p.border = border;
    p.store_mode = STORE_ROUND;
    for (int k = 0; k < kx; k++) p.wx[k] = lp[0].taps[k];
    for (int k = 0; k < ky; k++) p.wy[k] = lp[1].taps[k];
    *err = launch_gauss2d_exact(p, s);
    return true;
}

// 3-D integral volumes (at most 16 bits) blurred into an integral or f64
// volume: every z plane through the fused exact x/y kernel into a double
// image (bufB of the reference's gaussian_blur), then the z pass in the
// same double arithmetic with the one final round.  *done = false when not
// eligible.
static ndlgpu_status gauss3d_exact(const ndlgpu_view* src, const ndlgpu_view* dst, const std::vector<LPass>& lp,
                                   int border, void* ws, size_t ws_bytes, cudaStream_t s, bool* done)
{
    *done = false;
    if (src->rank != 3 || lp.size() != 3) return NDLGPU_OK;
    if (src->dtype != NDLGPU_U8 && src->dtype != NDLGPU_U16 && src->dtype != NDLGPU_I16) return NDLGPU_OK;
    if (!(dtype_integral(dst->dtype) || dst->dtype == NDLGPU_F64)) return NDLGPU_OK;
    if (lp[0].axis != 0 || lp[1].axis != 1 || lp[2].axis != 2) return NDLGPU_OK;
    const int kx = (int)lp[0].taps.size(), ky = (int)lp[1].taps.size();
    if (kx > 61 || ky > 61 || lp[2].taps.size() > 128 || src->extent[2] > 65535) return NDLGPU_OK;
    const int64_t count = view_count(src);
    if (count >= (int64_t(1) << 31)) return NDLGPU_OK;
    Scratch sc;
    ndlgpu_status st = get_scratch(align_up((size_t)count * sizeof(double)), ws, ws_bytes, s, &sc);
    if (st != NDLGPU_OK) return st;
    const int64_t nx = src->extent[0], ny = src->extent[1];
    GaussExactParams p;
    std::memset(&p, 0, sizeof(p));
    p.src = static_cast<const char*>(src->data);
    p.dst = static_cast<char*>(sc.base);
    p.sdt = src->dtype;
    p.ddt = NDLGPU_F64;
    p.des = 8;
    p.nx = (int)nx;
    p.ny = (int)ny;
    p.nb = (int)src->extent[2];
    p.sx = src->stride[0];
    p.sy = src->stride[1];
    p.sb = src->stride[2];
    p.dx = 1;
    p.dy = nx;
    p.db = nx * ny;
    p.kx = kx;
    p.ky = ky;
    p.cx = lp[0].center;
    p.cy = lp[1].center;
    p.border = border;
    p.store_mode = STORE_CAST;         // double intermediate: no rounding
    for (int k = 0; k < kx; k++) p.wx[k] = lp[0].taps[k];
    for (int k = 0; k < ky; k++) p.wy[k] = lp[1].taps[k];
    cudaError_t e = launch_gauss2d_exact(p, s);
    if (e != cudaSuccess) return cuda_fail(e, "exact x/y gaussian");
    // the z pass over the double volume, rounded and cast
    GaussZExactParams z;
    std::memset(&z, 0, sizeof(z));
    z.src = static_cast<const double*>(sc.base);
    z.dst = static_cast<char*>(dst->data);
    z.ddt = dst->dtype;
    z.nx = (int)nx;
    z.ny = (int)ny;
    z.nz = (int)src->extent[2];
    z.dx = dst->stride[0];
    z.dy = dst->stride[1];
    z.dz = dst->stride[2];
    z.kz = (int)lp[2].taps.size();
    z.cz = lp[2].center;
    z.border = border;
    for (int k = 0; k < z.kz; k++) z.wz[k] = lp[2].taps[k];
    e = launch_gauss_z_exact(z, s);
    if (e != cudaSuccess) return cuda_fail(e, "exact z gaussian");
    *done = true;
    return NDLGPU_OK;
}

ndlgpu_status ndlgpu_gaussian_blur(const ndlgpu_view* src, const ndlgpu_view* dst, double sigma, int border,
                                   void* workspace, size_t workspace_bytes, void* stream)
{
    t_last_error.clear();
    std::vector<LPass> lp;
    ndlgpu_status st = gaussian_passes(src, &sigma, false, &lp);
    if (st != NDLGPU_OK) return st;
    Canon c;
    Plan pl;
    st = prepare(src, dst, lp, border, NDLGPU_ROUND_ONCE, NDLGPU_PREC_AUTO, &c, &pl);
    if (st != NDLGPU_OK || c.total == 0) return st;
    const GaussRoute route = gauss_route(src, dst, lp, pl);
    cudaError_t e = cudaSuccess;
    if (route == GaussRoute::Exact2D && gauss2d_exact(src, dst, lp, border, (cudaStream_t)stream, &e))
        return e == cudaSuccess ? NDLGPU_OK : cuda_fail(e, "exact 2-D gaussian");
    bool done = false;
    if (route == GaussRoute::Exact3D)
        st = gauss3d_exact(src, dst, lp, border, workspace, workspace_bytes, (cudaStream_t)stream, &done);
    if (st != NDLGPU_OK || done) return st;
    return execute(c, pl, NDLGPU_ROUND_ONCE, border, workspace, workspace_bytes, (cudaStream_t)stream);
}

ndlgpu_status ndlgpu_gaussian_blur_axes(const ndlgpu_view* src, const ndlgpu_view* dst, const double* sigma_per_axis,
                                        int border, void* workspace, size_t workspace_bytes, void* stream)
{
    t_last_error.clear();
    if (!sigma_per_axis) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "sigma_per_axis is NULL");
    std::vector<LPass> lp;
    ndlgpu_status st = gaussian_passes(src, sigma_per_axis, true, &lp);
    if (st != NDLGPU_OK) return st;
    Canon c;
    Plan pl;
    st = prepare(src, dst, lp, border, NDLGPU_ROUND_ONCE, NDLGPU_PREC_AUTO, &c, &pl);
    if (st != NDLGPU_OK || c.total == 0) return st;
    const GaussRoute route = gauss_route(src, dst, lp, pl);
    cudaError_t e = cudaSuccess;
    if (route == GaussRoute::Exact2D && gauss2d_exact(src, dst, lp, border, (cudaStream_t)stream, &e))
        return e == cudaSuccess ? NDLGPU_OK : cuda_fail(e, "exact 2-D gaussian");
    bool done = false;
    if (route == GaussRoute::Exact3D)
        st = gauss3d_exact(src, dst, lp, border, workspace, workspace_bytes, (cudaStream_t)stream, &done);
    if (st != NDLGPU_OK || done) return st;
    return execute(c, pl, NDLGPU_ROUND_ONCE, border, workspace, workspace_bytes, (cudaStream_t)stream);
}

ndlgpu_status ndlgpu_convolve_ex(const ndlgpu_view* src, const ndlgpu_view* dst, const ndlgpu_view* kernel,
                                 int border, int precision, void* stream)
{
    t_last_error.clear();
    ndlgpu_status st;
    if ((st = check_view(src, "src", true)) != NDLGPU_OK) return st;
    if ((st = check_view(dst, "dst", true)) != NDLGPU_OK) return st;
    if ((st = check_view(kernel, "kernel", false)) != NDLGPU_OK) return st;
    if ((st = check_pair(src, dst)) != NDLGPU_OK) return st;
    if (kernel->rank != src->rank) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "kernel rank must equal image rank");
    if (border < NDLGPU_CLAMP || border > NDLGPU_REFLECT) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "unknown border mode");
    if (precision < NDLGPU_PREC_AUTO || precision > NDLGPU_PREC_EXACT)
        return fail(NDLGPU_ERR_INVALID_ARGUMENT, "unknown precision");
    const int R = src->rank;
    int64_t kn = view_count(kernel);
    if (kn == 0) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "kernel is empty");
    if (!kernel->data) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "kernel data is NULL");
    int wide = -1, nwide = 0;
    for (int i = 0; i < R; i++)
        if (kernel->extent[i] > 1) { wide = i; nwide++; }
    if (nwide <= 1) {
        // a {1,..,K,..,1} kernel: one separable pass (convolution.h:132-139)
        const int axis = wide < 0 ? 0 : wide;
        LPass lp;
        lp.axis = axis;
        lp.center = (int)(kernel->extent[axis] / 2);   // image/detail.h:161
        if (kernel->extent[axis] > kMaxTaps) return fail(NDLGPU_ERR_TOO_MANY_TAPS, "kernel has more than 255 taps");
        for (int64_t k = 0; k < kernel->extent[axis]; k++) lp.taps.push_back(host_value(kernel, k * kernel->stride[axis]));
        Canon c;
        Plan pl;
        st = prepare(src, dst, {lp}, border, NDLGPU_CAST_EACH, precision, &c, &pl);
        if (st != NDLGPU_OK || c.total == 0) return st;
        return execute(c, pl, NDLGPU_CAST_EACH, border, nullptr, 0, (cudaStream_t)stream);
    }
    // general N-D kernel: nonzero taps in coordinates() order (axis 0 fastest,
    // image/detail.h:127-143, :164-174), centre K/2 per axis
    if (view_count(src) == 0) return NDLGPU_OK;
    std::vector<int32_t> off;
    std::vector<double> w;
    std::vector<int64_t> kc(R, 0);
    for (int64_t t = 0; t < kn; t++) {
        int64_t ko = 0;
        for (int i = 0; i < R; i++) ko += kc[i] * kernel->stride[i];
        const double v = host_value(kernel, ko);
        if (v != 0.0) {
            for (int i = 0; i < R; i++) {
                const int64_t o = kc[i] - kernel->extent[i] / 2;
                if (border != NDLGPU_CLAMP && (o > src->extent[i] || o < -src->extent[i]))
                    return fail(NDLGPU_ERR_RADIUS_EXCEEDS_EXTENT, "kernel radius exceeds the image extent (Wrap/Reflect)");
                off.push_back((int32_t)o);
            }
            w.push_back(v);
        }
        for (int i = 0; i < R; i++) {
            if (++kc[i] < kernel->extent[i]) break;
            kc[i] = 0;
        }
    }
    if ((int64_t)w.size() > NDLGPU_MAX_ND_TAPS) return fail(NDLGPU_ERR_TOO_MANY_TAPS, "more than 4096 nonzero kernel taps");
    if (view_count(src) >= (int64_t(1) << 31))
        return fail(NDLGPU_ERR_INDEX_OVERFLOW, "N-D kernels support images of fewer than 2^31 elements");
    Acc acc = Acc::F64;
    if (precision == NDLGPU_PREC_FP32) acc = Acc::F32;
    else if (precision == NDLGPU_PREC_AUTO && !dtype_integral(dst->dtype) && dst->dtype != NDLGPU_F64 &&
             src->dtype != NDLGPU_F64)
        acc = Acc::F32;
    // integral sources of up to 16 bits with a 2-D / 3-D kernel of up to 9
    // taps per axis, exact double arithmetic: the tiled exact stencil
    // (stencil.cu; zero taps included, which leaves integral sums unchanged)
    if (acc == Acc::F64 && (src->dtype == NDLGPU_U8 || src->dtype == NDLGPU_U16 || src->dtype == NDLGPU_I16) &&
        (R == 2 || R == 3)) {
        bool fits = true;
        for (int i = 0; i < R; i++) fits = fits && kernel->extent[i] <= kStencilMaxTaps;
        if (fits) {
            StencilParams sp;
            std::memset(&sp, 0, sizeof(sp));
            sp.srcc = static_cast<const char*>(src->data);
            sp.dstc = static_cast<char*>(dst->data);
            sp.sdt = src->dtype;
            sp.ddt = dst->dtype;
            sp.nx = (int)src->extent[0];
            sp.ny = (int)src->extent[1];
            sp.nz = R == 3 ? (int)src->extent[2] : 1;
            sp.nb = 1;
            sp.sx = src->stride[0];
            sp.sy = src->stride[1];
            sp.sz = R == 3 ? src->stride[2] : 0;
            sp.dx = dst->stride[0];
            sp.dy = dst->stride[1];
            sp.dz = R == 3 ? dst->stride[2] : 0;
            sp.kx = (int)kernel->extent[0];
            sp.ky = (int)kernel->extent[1];
            sp.kz = R == 3 ? (int)kernel->extent[2] : 1;
            sp.cx = sp.kx / 2;
            sp.cy = sp.ky / 2;
            sp.cz = sp.kz / 2;
            sp.border = border;
            // every tap, zeros included, in coordinates() order
            int t = 0;
            for (int z = 0; z < sp.kz; z++)
                for (int y = 0; y < sp.ky; y++)
                    for (int x = 0; x < sp.kx; x++) {
                        int64_t ko = x * kernel->stride[0] + y * kernel->stride[1];
                        if (R == 3) ko += z * kernel->stride[2];
                        sp.wd[t++] = host_value(kernel, ko);
                    }
            cudaError_t e = launch_stencil_exact(sp, (cudaStream_t)stream);
            return e == cudaSuccess ? NDLGPU_OK : cuda_fail(e, "exact stencil launch");
        }
    }
    // f32 images with a dense 2-D / 3-D kernel of up to 9 taps per axis: the
    // tiled stencil (stencil.cu)
    if (acc == Acc::F32 && src->dtype == NDLGPU_F32 && dst->dtype == NDLGPU_F32 && (R == 2 || R == 3) &&
        (int64_t)w.size() == kn) {
        bool fits = true;
        for (int i = 0; i < R; i++) fits = fits && kernel->extent[i] <= kStencilMaxTaps;
        if (fits) {
            StencilParams sp;
            std::memset(&sp, 0, sizeof(sp));
            sp.src = static_cast<const float*>(src->data);
            sp.dst = static_cast<float*>(dst->data);
            sp.nx = (int)src->extent[0];
            sp.ny = (int)src->extent[1];
            sp.nz = R == 3 ? (int)src->extent[2] : 1;
            sp.nb = 1;
            sp.sx = src->stride[0];
            sp.sy = src->stride[1];
            sp.sz = R == 3 ? src->stride[2] : 0;
            sp.dx = dst->stride[0];
            sp.dy = dst->stride[1];
            sp.dz = R == 3 ? dst->stride[2] : 0;
            sp.kx = (int)kernel->extent[0];
            sp.ky = (int)kernel->extent[1];
            sp.kz = R == 3 ? (int)kernel->extent[2] : 1;
            sp.cx = sp.kx / 2;
            sp.cy = sp.ky / 2;
            sp.cz = sp.kz / 2;
            sp.border = border;
            for (size_t t = 0; t < w.size(); t++) sp.w[t] = (float)w[t];
            cudaError_t e = launch_stencil(sp, (cudaStream_t)stream);
            return e == cudaSuccess ? NDLGPU_OK : cuda_fail(e, "stencil launch");
        }
    }
    GenericNdParams p;
    std::memset(&p, 0, sizeof(p));
    p.src = (const char*)src->data;
    p.dst = (char*)dst->data;
    p.src_dtype = src->dtype;
    p.dst_dtype = dst->dtype;
    p.rank = R;
    p.ntap = (int)w.size();
    p.border = border;
    p.store_mode = STORE_CAST;
    p.total = (uint32_t)view_count(src);
    for (int i = 0; i < R; i++) {
        p.n[i] = src->extent[i];
        p.ss[i] = src->stride[i];
        p.ds[i] = dst->stride[i];
        p.div[i].init((uint32_t)src->extent[i]);
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (w.empty()) {
        // every tap is zero: convolve() writes DstT(0) everywhere
        w.push_back(0.0);
        for (int i = 0; i < R; i++) off.push_back(0);
        p.ntap = 0;
    }
    const size_t ob = align_up(off.size() * sizeof(int32_t));
    Scratch sc;
    st = get_scratch(ob + w.size() * sizeof(double), nullptr, 0, s, &sc);
    if (st != NDLGPU_OK) return st;
    cudaError_t e = cudaMemcpyAsync(sc.base, off.data(), off.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync((char*)sc.base + ob, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "tap upload");
    p.tap_off = (const int32_t*)sc.base;
    p.tap_w = (const double*)((char*)sc.base + ob);
    e = launch_generic_nd(acc, p, s);
    if (e != cudaSuccess) return cuda_fail(e, "N-D kernel");
    // the pageable-memory copies above completed staging before returning;
    // the scratch is released stream-ordered after the kernel
    return NDLGPU_OK;
}

ndlgpu_status ndlgpu_gradient(const ndlgpu_view* src, const ndlgpu_view* dst, int border, void* stream)
{
    // ndl::gradient (processing/convolution.h:359-388): for every axis a,
    // convolve(src, dst.slice(0, a), kernel {-0.5, 0, +0.5} along a)
    t_last_error.clear();
    ndlgpu_status st;
    if ((st = check_view(src, "src", true)) != NDLGPU_OK) return st;
    if ((st = check_view(dst, "dst", true)) != NDLGPU_OK) return st;
    if (border < NDLGPU_CLAMP || border > NDLGPU_REFLECT) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "unknown border mode");
    const int R = src->rank;
    if (dst->rank != R + 1)
        return fail(NDLGPU_ERR_INVALID_ARGUMENT, "gradient dst must have one more axis than src (a leading component axis)");
    if (dst->extent[0] != R) return fail(NDLGPU_ERR_EXTENT_MISMATCH, "gradient dst's leading extent must equal src's rank");
    for (int d = 0; d < R; d++)
        if (dst->extent[d + 1] != src->extent[d])
            return fail(NDLGPU_ERR_EXTENT_MISMATCH, "gradient dst's extents after the first must equal src's");
    if (view_count(src) == 0) return NDLGPU_OK;
    for (int a = 0; a < R; a++) {
        ndlgpu_view slice{};
        slice.data = static_cast<char*>(dst->data) + (ptrdiff_t)a * dst->stride[0] * dtype_size(dst->dtype);
        slice.dtype = dst->dtype;
        slice.rank = R;
        for (int d = 0; d < R; d++) {
            slice.extent[d] = dst->extent[d + 1];
            slice.stride[d] = dst->stride[d + 1];
        }
        if ((st = check_pair(src, &slice)) != NDLGPU_OK) return st;
    }
    // one pass over the source for ranks 1..3 (gradient.cu)
    GradParams gp{};
    gp.src = static_cast<const char*>(src->data);
    gp.dst = static_cast<char*>(dst->data);
    gp.sdt = src->dtype;
    gp.ddt = dst->dtype;
    gp.rank = R;
    gp.border = border;
    bool fits = R <= 3;
    for (int d = 0; d < R && fits; d++) {
        if (src->extent[d] > 0x7fffffffLL) fits = false;
        gp.ext[d] = (int)src->extent[d];
        gp.sstr[d] = src->stride[d];
        gp.dstr[d + 1] = dst->stride[d + 1];
    }
    gp.dstr[0] = dst->stride[0];
    if (fits && gradient_supported(gp)) {
        cudaError_t e = launch_gradient(gp, (cudaStream_t)stream);
        return e == cudaSuccess ? NDLGPU_OK : cuda_fail(e, "gradient launch");
    }
    // any rank: one convolve() pass per axis, as the reference runs it
    for (int a = 0; a < R; a++) {
        ndlgpu_view slice{};
        slice.data = static_cast<char*>(dst->data) + (ptrdiff_t)a * dst->stride[0] * dtype_size(dst->dtype);
        slice.dtype = dst->dtype;
        slice.rank = R;
        for (int d = 0; d < R; d++) {
            slice.extent[d] = dst->extent[d + 1];
            slice.stride[d] = dst->stride[d + 1];
        }
        if ((st = check_pair(src, &slice)) != NDLGPU_OK) return st;
        LPass lp;
        lp.axis = a;
        lp.center = 1;
        lp.taps = {-0.5, 0.0, 0.5};
        Canon c;
        Plan pl;
        st = prepare(src, &slice, {lp}, border, NDLGPU_CAST_EACH, NDLGPU_PREC_AUTO, &c, &pl);
        if (st != NDLGPU_OK) return st;
        if (c.total == 0) continue;
        if ((st = execute(c, pl, NDLGPU_CAST_EACH, border, nullptr, 0, (cudaStream_t)stream)) != NDLGPU_OK) return st;
    }
    return NDLGPU_OK;
}

// Blur of one level (gaussian_blur(src, dst, sigma, Reflect)) through the
// pass-chain planner.
static ndlgpu_status blur_level(const ndlgpu_view* src, const ndlgpu_view* dst, double sigma, cudaStream_t s)
{
    std::vector<LPass> lp;
    ndlgpu_status st = gaussian_passes(src, &sigma, false, &lp);
    if (st != NDLGPU_OK) return st;
    Canon c;
    Plan pl;
    st = prepare(src, dst, lp, NDLGPU_REFLECT, NDLGPU_ROUND_ONCE, NDLGPU_PREC_AUTO, &c, &pl);
    if (st != NDLGPU_OK || c.total == 0) return st;
    return execute(c, pl, NDLGPU_ROUND_ONCE, NDLGPU_REFLECT, nullptr, 0, s);
}

// Source types that convert to float exactly (the fused kernel's loads).
static bool float_exact_dtype(int dt)
{
    return dt == NDLGPU_U8 || dt == NDLGPU_I8 || dt == NDLGPU_U16 || dt == NDLGPU_I16 || dt == NDLGPU_F32 ||
           dt == NDLGPU_F16 || dt == NDLGPU_BF16;
}

ndlgpu_status ndlgpu_dog_scale_space(const ndlgpu_view* src, int num_scales, double sigma0, const ndlgpu_view* levels,
                                     const ndlgpu_view* dogs, void* stream)
{
    // ndl::detect_keypoints' scale space (processing/feature_detection.h:101-122)
    t_last_error.clear();
    ndlgpu_status st;
    if ((st = check_view(src, "src", true)) != NDLGPU_OK) return st;
    if (num_scales < 4 || num_scales > kDogMaxScales)
        return fail(NDLGPU_ERR_INVALID_ARGUMENT, "num_scales must be 4.." + std::to_string(kDogMaxScales) +
                                                     " (feature_detection.h:95 asserts >= 4)");
    if (!(sigma0 > 0) || !std::isfinite(sigma0))
        return fail(NDLGPU_ERR_BAD_SIGMA, "sigma0 must be positive and finite (feature_detection.h:96)");
    if (!dogs) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "dogs is NULL");
    const int ns = num_scales;
    std::vector<const ndlgpu_view*> outs;
    for (int i = 0; i < ns - 1; i++) outs.push_back(&dogs[i]);
    if (levels)
        for (int i = 0; i < ns; i++) outs.push_back(&levels[i]);
    for (size_t i = 0; i < outs.size(); i++) {
        const ndlgpu_view* o = outs[i];
        if ((st = check_view(o, (int)i < ns - 1 ? "dogs[i]" : "levels[i]", true)) != NDLGPU_OK) return st;
        if (o->dtype != NDLGPU_F32 && o->dtype != NDLGPU_F64)
            return fail(NDLGPU_ERR_UNSUPPORTED_DTYPE, "levels and dogs must be F32 or F64 images");
        if ((st = check_pair(src, o)) != NDLGPU_OK) return st;
    }
    if (view_count(src) == 0) return NDLGPU_OK;
    for (size_t i = 0; i < outs.size(); i++)
        for (size_t j = i + 1; j < outs.size(); j++) {
            intptr_t a0, a1, b0, b1;
            view_bytes(outs[i], &a0, &a1);
            view_bytes(outs[j], &b0, &b1);
            if (a0 < b1 && b0 < a1) return fail(NDLGPU_ERR_ALIASING, "two output images overlap");
        }
    // sigma_i = sigma0 * 2^(i / (num_scales - 3)), radius ceil(3 sigma_i)
    std::vector<double> sig(ns);
    int rmax = 0;
    for (int i = 0; i < ns; i++) {
        sig[i] = sigma0 * std::pow(2.0, (double)i / (ns - 3));
        if (2 * kernel_size(sig[i]) + 1 > kMaxTaps) return fail(NDLGPU_ERR_TOO_MANY_TAPS, "sigma too large (more than 255 taps)");
        rmax = std::max(rmax, kernel_size(sig[i]));
    }
    for (int a = 0; a < src->rank; a++)
        if (rmax > src->extent[a])
            return fail(NDLGPU_ERR_RADIUS_EXCEEDS_EXTENT, "the largest level's radius " + std::to_string(rmax) +
                                                               " exceeds extent " + std::to_string(src->extent[a]) +
                                                               " (Reflect maps one period, mathHelpers.h:24)");
    const cudaStream_t s = (cudaStream_t)stream;
    bool all_f32 = true;
    for (const ndlgpu_view* o : outs) all_f32 = all_f32 && o->dtype == NDLGPU_F32;
    if (src->rank == 2 && all_f32 && ns <= kDogMaxLevels && rmax <= kDogMaxRadius && float_exact_dtype(src->dtype)) {
        // one pass over the source (dog.cu)
        DogParams p{};
        p.src = static_cast<const char*>(src->data);
        p.sdt = src->dtype;
        p.nx = (int)src->extent[0];
        p.ny = (int)src->extent[1];
        p.sx = src->stride[0];
        p.sy = src->stride[1];
        p.ns = ns;
        p.R = rmax;
        for (int i = 0; i < ns; i++) {
            const std::vector<double> w = gaussian_taps(sig[i]);
            p.r[i] = (int)w.size() / 2;
            for (size_t k = 0; k < w.size(); k++) p.w2[i][k] = make_float2((float)w[k], (float)w[k]);
            // pair stores need x stride 1 and 8-byte aligned pairs on every row
            auto pairs_ok = [](const ndlgpu_view& v) {
                return v.stride[0] == 1 && reinterpret_cast<uintptr_t>(v.data) % 8 == 0 && v.stride[1] % 2 == 0;
            };
            if (levels) {
                p.lv[i] = static_cast<float*>(levels[i].data);
                p.lx[i] = levels[i].stride[0];
                p.ly[i] = levels[i].stride[1];
                p.lvec[i] = pairs_ok(levels[i]);
            }
            if (i > 0) {
                p.dg[i - 1] = static_cast<float*>(dogs[i - 1].data);
                p.gx[i - 1] = dogs[i - 1].stride[0];
                p.gy[i - 1] = dogs[i - 1].stride[1];
                p.gvec[i - 1] = pairs_ok(dogs[i - 1]);
            }
        }
        cudaError_t e = launch_dog2d(p, s);
        return e == cudaSuccess ? NDLGPU_OK : cuda_fail(e, "dog launch");
    }
    // any rank and type: one gaussian_blur per level, then the differences in
    // double.  Levels go to the caller's level images when they have the
    // differences' precision, else to two stream-ordered scratch images.
    bool any_f64 = false;
    for (int i = 0; i < ns - 1; i++) any_f64 = any_f64 || dogs[i].dtype == NDLGPU_F64;
    const int ldt = any_f64 ? NDLGPU_F64 : NDLGPU_F32;
    const int64_t count = view_count(src);
    Scratch sc;
    const bool own = !levels || levels[0].dtype != ldt;
    for (int i = 0; levels && i < ns && !own; i++)
        if (levels[i].dtype != ldt) return fail(NDLGPU_ERR_UNSUPPORTED_DTYPE, "level images must share one dtype");
    ndlgpu_view tmp[2];
    if (own) {
        const size_t one = align_up((size_t)count * dtype_size(ldt));
        if ((st = get_scratch(2 * one, nullptr, 0, s, &sc)) != NDLGPU_OK) return st;
        for (int b = 0; b < 2; b++) {
            tmp[b] = ndlgpu_view{};
            tmp[b].data = static_cast<char*>(sc.base) + b * one;
            tmp[b].dtype = ldt;
            tmp[b].rank = src->rank;
            int64_t stv = 1;
            for (int a = 0; a < src->rank; a++) {
                tmp[b].extent[a] = src->extent[a];
                tmp[b].stride[a] = stv;
                stv *= src->extent[a];
            }
        }
    }
    const ndlgpu_view* prev = nullptr;
    for (int i = 0; i < ns; i++) {
        const ndlgpu_view* cur = own ? &tmp[i & 1] : &levels[i];
        if ((st = blur_level(src, cur, sig[i], s)) != NDLGPU_OK) return st;
        if (own && levels && (st = blur_level(src, &levels[i], sig[i], s)) != NDLGPU_OK) return st;
        if (prev) {
            const ndlgpu_view& d = dogs[i - 1];
            SubParams sp{};
            sp.a = static_cast<const char*>(cur->data);
            sp.b = static_cast<const char*>(prev->data);
            sp.dst = static_cast<char*>(d.data);
            sp.adt = cur->dtype;
            sp.bdt = prev->dtype;
            sp.ddt = d.dtype;
            sp.rank = src->rank;
            sp.total = count;
            for (int a = 0; a < src->rank; a++) {
                sp.ext[a] = src->extent[a];
                sp.as[a] = cur->stride[a];
                sp.bs[a] = prev->stride[a];
                sp.ds[a] = d.stride[a];
            }
            cudaError_t e = launch_sub(sp, s);
            if (e != cudaSuccess) return cuda_fail(e, "dog difference launch");
        }
        prev = cur;
    }
    return NDLGPU_OK;
}

static ndlgpu_status box_prepare(const ndlgpu_view* src, const ndlgpu_view* dst, int radius, int border, BoxParams* p)
{
    ndlgpu_status st;
    if ((st = check_view(src, "src", true)) != NDLGPU_OK) return st;
    if ((st = check_view(dst, "dst", true)) != NDLGPU_OK) return st;
    if ((st = check_pair(src, dst)) != NDLGPU_OK) return st;
    if (radius < 1) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "radius must be > 0 (summed_area_table.h:306)");
    if (border < NDLGPU_CLAMP || border > NDLGPU_REFLECT) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "unknown border mode");
    *p = BoxParams{};
    p->rank = src->rank;
    p->radius = radius;
    p->border = border;
    p->npad = 1;
    p->total = view_count(src);
    p->area = 1.0;
    __int128 npad = 1;
    for (int a = 0; a < src->rank; a++) {
        if (border != NDLGPU_CLAMP && radius > src->extent[a] && src->extent[a] > 0)
            return fail(NDLGPU_ERR_RADIUS_EXCEEDS_EXTENT, "Wrap/Reflect map one period: radius must not exceed extent " +
                                                               std::to_string(src->extent[a]) + " (mathHelpers.h:23-24)");
        p->ext[a] = (int)src->extent[a];
        p->sstr[a] = src->stride[a];
        p->dstr[a] = dst->stride[a];
        p->pext[a] = src->extent[a] + 2 * (int64_t)radius;
        p->pst[a] = (int64_t)npad;
        npad *= p->pext[a];
        p->area *= (2 * radius + 1);
    }
    if (npad > ((__int128)1 << 40)) return fail(NDLGPU_ERR_INDEX_OVERFLOW, "padded summed-area table too large");
    p->npad = (int64_t)npad;
    p->src = static_cast<const char*>(src->data);
    p->dst = static_cast<char*>(dst->data);
    p->sdt = src->dtype;
    p->ddt = dst->dtype;
    return NDLGPU_OK;
}

ndlgpu_status ndlgpu_box_blur_workspace_size(const ndlgpu_view* src, const ndlgpu_view* dst, int radius, int border,
                                             size_t* bytes)
{
    t_last_error.clear();
    if (!bytes) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "bytes is NULL");
    BoxParams p;
    ndlgpu_status st = box_prepare(src, dst, radius, border, &p);
    if (st != NDLGPU_OK) return st;
    *bytes = p.total == 0 ? 0 : align_up((size_t)p.npad * sizeof(double));
    return NDLGPU_OK;
}

ndlgpu_status ndlgpu_box_blur(const ndlgpu_view* src, const ndlgpu_view* dst, int radius, int border, void* workspace,
                              size_t workspace_bytes, void* stream)
{
    // ndl::box_blur (processing/summed_area_table.h:300-339)
    t_last_error.clear();
    BoxParams p;
    ndlgpu_status st = box_prepare(src, dst, radius, border, &p);
    if (st != NDLGPU_OK || p.total == 0) return st;
    Scratch sc;
    const cudaStream_t s = (cudaStream_t)stream;
    if ((st = get_scratch(align_up((size_t)p.npad * sizeof(double)), workspace, workspace_bytes, s, &sc)) != NDLGPU_OK)
        return st;
    p.table = static_cast<double*>(sc.base);
    cudaError_t e = launch_box_blur(p, s);
    return e == cudaSuccess ? NDLGPU_OK : cuda_fail(e, "box_blur launch");
}

ndlgpu_status ndlgpu_downsample(const ndlgpu_view* src, const ndlgpu_view* dst, int factor, int channel_axis,
                                int border, void* stream)
{
    // ndl::downsample (processing/convolution.h:241-305); `border` is accepted
    // and unused, as in the reference (:262)
    (void)border;
    t_last_error.clear();
    ndlgpu_status st;
    if ((st = check_view(src, "src", true)) != NDLGPU_OK) return st;
    if ((st = check_view(dst, "dst", true)) != NDLGPU_OK) return st;
    if (factor < 2) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "factor must be > 1 (convolution.h:265)");
    if (src->rank < 2) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "downsample needs a channel axis and at least one other");
    if (channel_axis < 0 || channel_axis >= src->rank) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "channel_axis out of range");
    if (dst->rank != src->rank) return fail(NDLGPU_ERR_EXTENT_MISMATCH, "src and dst ranks differ");
    DownParams p{};
    p.rank = src->rank;
    p.channel = channel_axis;
    p.factor = factor;
    p.total = 1;
    for (int a = 0; a < src->rank; a++) {
        const int64_t oe = (a == channel_axis || src->extent[a] == 0) ? src->extent[a] : (src->extent[a] - 1) / factor + 1;
        if (dst->extent[a] != oe)
            return fail(NDLGPU_ERR_EXTENT_MISMATCH, "dst extent on axis " + std::to_string(a) + " must be " +
                                                        std::to_string(oe) + " ((extent - 1) / factor + 1, convolution.h:268-269)");
        p.ext[a] = (int)src->extent[a];
        p.oext[a] = (int)oe;
        p.sstr[a] = src->stride[a];
        p.dstr[a] = dst->stride[a];
        p.total *= oe;
    }
    if (p.total == 0) return NDLGPU_OK;
    if (p.total > 0xffffffffLL) return fail(NDLGPU_ERR_INDEX_OVERFLOW, "downsample writes at most 2^32-1 outputs per call");
    for (int a = 0; a < src->rank; a++) {
        p.odiv[a].init((uint32_t)p.oext[a]);
        if (a != channel_axis) p.sub[p.nsub++] = a;
    }
    intptr_t a0, a1, b0, b1;
    view_bytes(src, &a0, &a1);
    view_bytes(dst, &b0, &b1);
    if (a0 < b1 && b0 < a1) return fail(NDLGPU_ERR_ALIASING, "src and dst memory overlap");
    if ((st = check_no_self_overlap(dst)) != NDLGPU_OK) return st;
    p.src = static_cast<const char*>(src->data);
    p.dst = static_cast<char*>(dst->data);
    p.sdt = src->dtype;
    p.ddt = dst->dtype;
    cudaError_t e = launch_downsample(p, (cudaStream_t)stream);
    return e == cudaSuccess ? NDLGPU_OK : cuda_fail(e, "downsample launch");
}

ndlgpu_status ndlgpu_convolve(const ndlgpu_view* src, const ndlgpu_view* dst, const ndlgpu_view* kernel, int border,
                              void* stream)
{
    return ndlgpu_convolve_ex(src, dst, kernel, border, NDLGPU_PREC_AUTO, stream);
}

ndlgpu_status ndlgpu_convolve_axes_adjoint_workspace_size(const ndlgpu_view* grad_out, const ndlgpu_view* src,
                                                          const ndlgpu_view* grad_src, int npass,
                                                          const ndlgpu_axis_kernel* passes, int border,
                                                          int grad_taps_dtype, size_t* bytes)
{
    t_last_error.clear();
    if (!bytes) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "bytes is NULL");
    *bytes = 0;
    AdjPlan ap;
    ndlgpu_status st = adjoint_prepare(grad_out, src, grad_src, npass, passes, border, src != nullptr,
                                       grad_taps_dtype, &ap);
    if (st != NDLGPU_OK) return st;
    size_t need = adjoint_workspace(ap);
    FusedTap ft;
    if (src && ap.total > 0 && plan_fused_tapgrad(grad_out, src, npass, passes, border, &ft))
        need = std::max(need, align_up((size_t)ft.ncta * (ft.tp.kx + ft.tp.ky + ft.tp.kz) * sizeof(double)));
    *bytes = need;
    return NDLGPU_OK;
}

ndlgpu_status ndlgpu_convolve_axes_adjoint(const ndlgpu_view* grad_out, const ndlgpu_view* src,
                                           const ndlgpu_view* grad_src, int npass, const ndlgpu_axis_kernel* passes,
                                           int border, void* grad_taps, int grad_taps_dtype, void* workspace,
                                           size_t workspace_bytes, void* stream)
{
    t_last_error.clear();
    if (!grad_src && !grad_taps) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "nothing to compute: grad_src and grad_taps are NULL");
    AdjPlan ap;
    ndlgpu_status st = adjoint_prepare(grad_out, src, grad_src, npass, passes, border, grad_taps != nullptr,
                                       grad_taps_dtype, &ap);
    if (st != NDLGPU_OK) return st;
    FusedParams fp;
    const bool fused = grad_src && ap.total > 0 && plan_fused_adjoint(grad_out, grad_src, npass, passes, border, &fp);
    FusedTap ft;
    const bool ftap = grad_taps && ap.total > 0 && plan_fused_tapgrad(grad_out, src, npass, passes, border, &ft);
    return adjoint_execute(grad_out, src, grad_src, border, grad_taps, grad_taps_dtype, ap, workspace,
                           workspace_bytes, (cudaStream_t)stream, fused ? &fp : nullptr, ftap ? &ft : nullptr);
}

ndlgpu_status ndlgpu_batch_create(ndlgpu_batch** out)
{
    t_last_error.clear();
    if (!out) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = new ndlgpu_batch();
    return NDLGPU_OK;
}

ndlgpu_status ndlgpu_batch_add(ndlgpu_batch* b, const ndlgpu_view* src, const ndlgpu_view* dst, int npass,
                               const ndlgpu_axis_kernel* passes, int border, int adjoint)
{
    t_last_error.clear();
    if (!b) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "batch is NULL");
    return batch_add(b, src, dst, npass, passes, border, adjoint);
}

ndlgpu_status ndlgpu_batch_plan(ndlgpu_batch* b, int tile_config)
{
    t_last_error.clear();
    if (!b) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "batch is NULL");
    return batch_plan(b, tile_config);
}

ndlgpu_status ndlgpu_batch_launch(ndlgpu_batch* b, void* stream)
{
    t_last_error.clear();
    if (!b || !b->planned) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "batch is NULL or not planned");
    return batch_enqueue(b, (cudaStream_t)stream);
}

ndlgpu_status ndlgpu_batch_graph_launch(ndlgpu_batch* b, void* stream)
{
    t_last_error.clear();
    if (!b || !b->planned) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "batch is NULL or not planned");
    cudaStream_t s = (cudaStream_t)stream;
    if (!b->gexec) {
        if (!s) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "graph capture needs a non-default stream");
        cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
        ndlgpu_status st = batch_enqueue(b, s);
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(s, &g);
        if (st != NDLGPU_OK) { if (g) cudaGraphDestroy(g); return st; }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&b->gexec, g, 0);
        if (e != cudaSuccess) { cudaGraphDestroy(g); return cuda_fail(e, "cudaGraphInstantiate"); }
        b->graph = g;
    }
    cudaError_t e = cudaGraphLaunch(b->gexec, s);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
    return NDLGPU_OK;
}

ndlgpu_status ndlgpu_batch_destroy(ndlgpu_batch* b)
{
    t_last_error.clear();
    if (!b) return NDLGPU_OK;
    b->release();
    delete b;
    return NDLGPU_OK;
}

int ndlgpu_batch_tile_configs(void) { return batch_tile_configs(); }

ndlgpu_status ndlgpu_batch_tile_config_info(int index, int* tile_x, int* tile_y, int* threads)
{
    t_last_error.clear();
    if (index < 0 || index >= batch_tile_configs() || !tile_x || !tile_y || !threads)
        return fail(NDLGPU_ERR_INVALID_ARGUMENT, "bad tile configuration index or NULL output");
    batch_tile_info(index, tile_x, tile_y, threads);
    return NDLGPU_OK;
}

ndlgpu_status ndlgpu_batch_info(const ndlgpu_batch* b, int* instances, int* items, int64_t* elements)
{
    t_last_error.clear();
    if (!b) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "batch is NULL");
    if (instances) *instances = (int)b->descs.size();
    if (items) *items = b->nitems;
    if (elements) {
        int64_t n = 0;
        for (int64_t v : b->elems) n += v;
        *elements = n;
    }
    return NDLGPU_OK;
}

uint64_t ndlgpu_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

ndlgpu_status ndlgpu_test_wait_timeouts(int spin_limit, int unreachable)
{
    t_last_error.clear();
    if (spin_limit < 0) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "spin_limit must be >= 0");
    const bool on = spin_limit > 0 || unreachable != 0;
    cudaError_t e = set_tma_wait_test(on && spin_limit > 0 ? spin_limit : (1 << 22), on && unreachable ? 16u : 0u);
    if (e == cudaSuccess)
        e = set_fwd3_wait_test(on && spin_limit > 0 ? spin_limit : (1 << 22), on && unreachable ? 16u : 0u);

    if (e == cudaSuccess)
        e = set_batch_wait_test(on && spin_limit > 0 ? spin_limit : (1 << 22), on && unreachable ? 1 : 0);
    if (e != cudaSuccess) return cuda_fail(e, "wait test controls");
    return NDLGPU_OK;
}

ndlgpu_status ndlgpu_device_status(void* stream, int32_t* code)
{
    t_last_error.clear();
    if (!code) return fail(NDLGPU_ERR_INVALID_ARGUMENT, "code is NULL");
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    e = read_device_status((cudaStream_t)stream, code);
    if (e != cudaSuccess) return cuda_fail(e, "guard read");
    return NDLGPU_OK;
}

}  // extern "C"
