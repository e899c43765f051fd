// pass_tiled.cu -- one 1-D pass of any width (runtime taps) along one axis,
// FP32 accumulation, float storage (f32 / bf16 / f16 in and out): the pass
// kernels of the plain path for the widths the fused kernels do not compile
// (wide Gaussians, uneven per-axis widths, ranks above 3).
//
// The tile (outputs plus the tap window) is staged in shared memory with its
// coordinates border-mapped (Clamp / Wrap / Reflect, mathHelpers.h:23-25),
// then every thread sums its outputs from a sliding register window, taps in
// ascending order (no tap past the kernel is ever multiplied, so non-finite
// samples behave as in the reference's sum):
//   along x (the contiguous axis): 8 rows x 256 outputs per CTA, a warp per
//     row, lane l outputs 4l .. 4l+3 and 128+4l .. 128+4l+3, four taps per
//     step from two 16-byte chunks per output block;
//   along another axis: 64 columns x 64 outputs per CTA, a thread a column
//     pair (packed FP32 pairs) and 8 outputs along the axis, one new row per
//     tap.
// Both kernels are persistent: a CTA walks its tiles with two staging
// buffers, cp.async loading the next tile's rows while the current one is
// summed.  Taps are the pass's dense offsets omin .. omin+K-1 in ascending
// order.
#include <algorithm>
#include <atomic>

#include "dtype.cuh"

namespace ndlgpu {
namespace {

constexpr int NT = 256;
constexpr int XO = 256;     // x pass: outputs per row
constexpr int XR = 8;       // x pass: rows per CTA
constexpr int SC = 64;      // strided pass: columns per CTA
constexpr int SO = 64;      // strided pass: outputs along the axis per CTA

template <class T> __device__ __forceinline__ float ldf(const T* p);
template <> __device__ __forceinline__ float ldf<float>(const float* p) { return *p; }
template <> __device__ __forceinline__ float ldf<__nv_bfloat16>(const __nv_bfloat16* p) { return __bfloat162float(*p); }
template <> __device__ __forceinline__ float ldf<__half>(const __half* p) { return __half2float(*p); }
template <class T> __device__ __forceinline__ T stf(float v);
template <> __device__ __forceinline__ float stf<float>(float v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 stf<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ __half stf<__half>(float v) { return __float2half_rn(v); }

__device__ __forceinline__ int64_t bmap(int border, int64_t n, int64_t x) { return map_border(border, n, x); }

// Outer coordinates (every axis but x and the pass axis) of index o, as
// source and destination offsets (32-bit magic-number divisions).
__device__ __forceinline__ void outer_offsets(const TiledPassParams& p, int skip0, int skip1, uint32_t o, int64_t* so,
                                              int64_t* dof)
{
    int64_t s = 0, d = 0;
#pragma unroll
    for (int i = 0; i < kTiledRank; i++) {
        if (i >= p.rank || i == skip0 || i == skip1) continue;
        const uint32_t q = p.dv[i].div(o);
        const int64_t c = (int64_t)(o - q * p.dv[i].d);
        o = q;
        s += c * p.ss[i];
        d += c * p.ds[i];
    }
    *so = s;
    *dof = d;
}

__device__ __forceinline__ void cp_async16(float* smem, const float* gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(float* smem, const float* gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(float* smem, const float* gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// x pass: the window of row `row` from x0 + omin, Lr floats (the outputs'
// XO + K - 1 plus the chunk the last step reads past it), staged so that
// srow[j] holds the input at x0 + omin + j.  Global reads are 16-byte chunks
// aligned down from x0 + omin (rem = the offset into the first chunk); chunks
// wholly inside a contiguous f32 row load as float4, the rest (the row's ends,
// strided or 16-bit rows) element by element with their coordinates mapped.
__host__ __device__ constexpr int x_window(int K) { return (XO + K + 4 + 3) & ~3; }
__host__ __device__ constexpr int x_pitch(int K) { return x_window(K) + 8; }

// Four taps on four outputs from an 8-float register window (chunks A, B).
__device__ __forceinline__ void taps4(float (&a)[4], const float4 A, const float4 B, const float4 w)
{
    const float win[8] = {A.x, A.y, A.z, A.w, B.x, B.y, B.z, B.w};
    const float wq[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
        for (int m = 0; m < 4; m++) a[m] = fmaf(wq[q], win[m + q], a[m]);
}

// The last r (1..3) taps: the same window, taps 0 .. r-1 only.
__device__ __forceinline__ void taps_tail(float (&a)[4], const float4 A, const float4 B, const float4 w, int r)
{
    const float win[8] = {A.x, A.y, A.z, A.w, B.x, B.y, B.z, B.w};
    const float wq[3] = {w.x, w.y, w.z};
#pragma unroll
    for (int q = 0; q < 3; q++) {
        if (q >= r) break;
#pragma unroll
        for (int m = 0; m < 4; m++) a[m] = fmaf(wq[q], win[m + q], a[m]);
    }
}

struct XTile {
    uint32_t row;
    int64_t x0, so, dof;
};

__device__ __forceinline__ XTile x_tile(const TiledPassParams& p, uint32_t t, int warp)
{
    XTile r;
    const uint32_t rb = p.dtx.div(t), tx = t - rb * p.dtx.d;
    r.x0 = (int64_t)tx * XO;
    r.row = rb * XR + warp;
    r.so = r.dof = 0;
    if (r.row < (uint32_t)p.rows) outer_offsets(p, 0, -1, r.row, &r.so, &r.dof);
    return r;
}

// The window of one row into srow (see x_window): whole 16-byte chunks of a
// contiguous f32 row by cp.async (16, 8 or 4 bytes at a time, as the
// window's offset rem into its first chunk allows), every other element by a
// border-mapped load.
template <class Tin>
__device__ __forceinline__ void x_stage(const TiledPassParams& p, const XTile& tl, float* srow, int lane)
{
    if (tl.row >= (uint32_t)p.rows) return;
    const int L = x_window(p.ntap);
    const Tin* src = reinterpret_cast<const Tin*>(p.src) + tl.so;
    // coordinates fit 32 bits (extents below 2^30)
    const int n0i = (int)p.n[0];
    const int gs = (int)tl.x0 + p.omin;
    const int xs = gs & ~3;
    const int rem = gs - xs;
    const int nv = (L + rem + 3) >> 2;
    // chunks va .. vb-1 lie wholly inside [0, n0)
    int va = 0, vb = 0;
    if constexpr (sizeof(Tin) == 4) {
        if (p.ss[0] == 1 && (reinterpret_cast<uintptr_t>(src) & 15) == 0) {
            va = min(nv, xs >= 0 ? 0 : -xs >> 2);
            vb = max(va, min(nv, (n0i - xs) >> 2));
        }
        const float* s4 = reinterpret_cast<const float*>(src) + xs;
#pragma unroll 3
        for (int v = va + lane; v < vb; v += 32) {
            const float* g = s4 + 4 * v;
            float* d = srow + 4 * v - rem;
            if (rem == 0) {
                cp_async16(d, g);
            } else if (rem == 2) {
                cp_async8(d, g);
                cp_async8(d + 2, g + 2);
            } else {
#pragma unroll
                for (int k = 0; k < 4; k++) cp_async4(d + k, g + k);
            }
        }
    }
    const int nlead = 4 * va, nrest = nlead + 4 * (nv - vb);
    for (int i = lane; i < nrest; i += 32) {
        const int e = i < nlead ? i : 4 * vb + (i - nlead);
        int x = xs + e;
        if (x < 0 || x >= n0i) x = (x >= n0i + p.omax || x < p.omin) ? n0i - 1 : map_border32(p.border, n0i, x);
        srow[e - rem] = ldf<Tin>(src + (int64_t)x * p.ss[0]);
    }
}

template <class Tout>
__device__ __forceinline__ void x_sum_store(const TiledPassParams& p, const XTile& tl, const float* srow,
                                            const float* s_w, int lane)
{
    if (tl.row >= (uint32_t)p.rows) return;
    const int K = p.ntap;
    const int64_t n0 = p.n[0];
    // lane l: outputs 4l .. 4l+3 and 128+4l .. 128+4l+3 (16-byte lane stride:
    // conflict-free window reads); a sliding window of two chunks per block
    const float* b0 = srow + 4 * lane;
    const float* b1 = b0 + XO / 2;
    float a0[4] = {0.f, 0.f, 0.f, 0.f}, a1[4] = {0.f, 0.f, 0.f, 0.f};
    float4 A0 = *reinterpret_cast<const float4*>(b0), A1 = *reinterpret_cast<const float4*>(b1);
    const int S = K >> 2;
#pragma unroll 2
    for (int s = 0; s < S; s++) {
        const float4 B0 = *reinterpret_cast<const float4*>(b0 + 4 * s + 4);
        const float4 B1 = *reinterpret_cast<const float4*>(b1 + 4 * s + 4);
        const float4 w = *reinterpret_cast<const float4*>(s_w + 4 * s);
        taps4(a0, A0, B0, w);
        taps4(a1, A1, B1, w);
        A0 = B0;
        A1 = B1;
    }
    if (K & 3) {
        const float4 B0 = *reinterpret_cast<const float4*>(b0 + 4 * S + 4);
        const float4 B1 = *reinterpret_cast<const float4*>(b1 + 4 * S + 4);
        const float4 w = *reinterpret_cast<const float4*>(s_w + 4 * S);
        taps_tail(a0, A0, B0, w, K & 3);
        taps_tail(a1, A1, B1, w, K & 3);
    }
    Tout* dst = reinterpret_cast<Tout*>(p.dst) + tl.dof;
    bool vst = false;
    if constexpr (sizeof(Tout) == 4) vst = p.ds[0] == 1 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const float* a = h ? a1 : a0;
        const int64_t xb = tl.x0 + 4 * lane + h * (XO / 2);
        if constexpr (sizeof(Tout) == 4) {
            if (vst && xb + 4 <= n0) {
                *reinterpret_cast<float4*>(reinterpret_cast<float*>(dst) + xb) = make_float4(a[0], a[1], a[2], a[3]);
                continue;
            }
        }
#pragma unroll
        for (int m = 0; m < 4; m++)
            if (xb + m < n0) dst[(xb + m) * p.ds[0]] = stf<Tout>(a[m]);
    }
}

// Persistent CTAs walk the tiles (8 rows x 256 outputs) with two staging
// buffers: the windows of the next tile load while the current one is summed.
template <class Tin, class Tout>
__global__ void __launch_bounds__(NT) k_tpass_x(const __grid_constant__ TiledPassParams p, uint32_t ntiles)
{
    extern __shared__ __align__(16) float sm_x[];
    const int K = p.ntap;
    const int P = x_pitch(K);
    float* s_w = sm_x + 2 * XR * P;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int K4 = (K + 3) & ~3;
    for (int i = tid; i < K4; i += NT) s_w[i] = i < K ? p.w[i] : 0.f;
    uint32_t t = blockIdx.x;
    if (t >= ntiles) return;
    __syncthreads();   // the taps visible; from here each warp works on its own rows
    XTile cur = x_tile(p, t, warp);
    x_stage<Tin>(p, cur, sm_x + warp * P + 4, lane);
    cp_async_commit();
    for (int i = 0; t < ntiles; i++) {
        const uint32_t tn = t + gridDim.x;
        XTile nxt = cur;
        if (tn < ntiles) {
            // the warp's row of buffer i+1 was last read by tile i-1, before
            // the warp barrier that ended its step
            nxt = x_tile(p, tn, warp);
            x_stage<Tin>(p, nxt, sm_x + (((i + 1) & 1) * XR + warp) * P + 4, lane);
        }
        cp_async_commit();
        cp_async_wait<1>();
        __syncwarp();   // tile i's window (every lane's copies) visible to the warp
        x_sum_store<Tout>(p, cur, sm_x + ((i & 1) * XR + warp) * P + 4, s_w, lane);
        __syncwarp();   // every lane is done with the warp's row of buffer i & 1
        cur = nxt;
        t = tn;
    }
    cp_async_wait<0>();
}

// Strided pass (any axis but x): SO + K - 1 staged rows along the axis of 64
// columns; thread (cp, og) sums the column pair 2cp, 2cp+1 (packed FP32
// pairs) for the 8 outputs 8og .. 8og+7 from a sliding window of 8 rows,
// one new row per tap.  Persistent CTAs walk the tiles with two staging
// buffers: the rows of the next tile load (cp.async, 16-byte chunks) while
// the current one is summed.
__host__ __device__ constexpr int s_rows(int K) { return SO + K - 1; }

struct STile {
    int64_t x0, y0, so, dof;
};

__device__ __forceinline__ STile s_tile(const TiledPassParams& p, uint32_t t)
{
    STile r;
    const uint32_t q = p.dtx.div(t), tx = t - q * p.dtx.d;
    const uint32_t o = p.dta.div(q), ta = q - o * p.dta.d;
    r.x0 = (int64_t)tx * SC;
    r.y0 = (int64_t)ta * SO;
    outer_offsets(p, 0, p.axis, o, &r.so, &r.dof);
    return r;
}

// Rows r = 0 .. nr-1 of a tile into buf: axis coordinate y0 + omin + r,
// border-mapped; columns x0 .. x0+63 (past n0: zero, never stored).  Whole
// 16-byte chunks of contiguous f32 rows go by cp.async, the rest by loads.
template <class Tin>
__device__ __forceinline__ void s_stage(const TiledPassParams& p, const STile& tl, float* buf, int nr)
{
    const int tid = threadIdx.x;
    const int a = p.axis;
    const int64_t n0 = p.n[0], na = p.n[a];
    const Tin* src = reinterpret_cast<const Tin*>(p.src) + tl.so;
    const int64_t ys = tl.y0 + p.omin;
    bool vec = false;
    if constexpr (sizeof(Tin) == 4)
        vec = p.ss[0] == 1 && tl.x0 + SC <= n0 && (p.ss[a] & 3) == 0 &&
              (reinterpret_cast<uintptr_t>(src + tl.x0) & 15) == 0;
    if (vec) {
        // a thread keeps one 16-byte column chunk, rows tid/16 + 16i
        const int c4 = tid & 15;
        const float* sp = reinterpret_cast<const float*>(src) + tl.x0 + 4 * c4;
#pragma unroll 4
        for (int r = tid >> 4; r < nr; r += NT / 16) {
            int64_t y = ys + r;
            if (y < 0 || y >= na) y = (y >= na + p.omax || y < p.omin) ? na - 1 : bmap(p.border, na, y);
            cp_async16(buf + r * SC + 4 * c4, sp + y * p.ss[a]);
        }
    } else {
        const int c = tid & (SC - 1);
        const int64_t x = tl.x0 + c;
        const Tin* sp = src + x * p.ss[0];
#pragma unroll 4
        for (int r = tid / SC; r < nr; r += NT / SC) {
            float v = 0.f;
            if (x < n0) {
                int64_t y = ys + r;
                if (y < 0 || y >= na) y = (y >= na + p.omax || y < p.omin) ? na - 1 : bmap(p.border, na, y);
                v = ldf<Tin>(sp + y * p.ss[a]);
            }
            buf[r * SC + c] = v;
        }
    }
}

template <class Tout>
__device__ __forceinline__ void s_sum_store(const TiledPassParams& p, const STile& tl, const float* buf,
                                            const float2* s_w2)
{
    const int K = p.ntap;
    const int tid = threadIdx.x;
    const int a = p.axis;
    const int64_t n0 = p.n[0], na = p.n[a];
    const int cp = tid & 31, og = tid >> 5;
    const float* col = buf + (8 * og) * SC + 2 * cp;
    float2 acc[8], win[8];
#pragma unroll
    for (int j = 0; j < 8; j++) acc[j] = make_float2(0.f, 0.f);
#pragma unroll
    for (int j = 0; j < 7; j++) win[j] = *reinterpret_cast<const float2*>(col + j * SC);
    const int K8 = K & ~7;
    for (int t0 = 0; t0 < K8; t0 += 8) {
#pragma unroll
        for (int u = 0; u < 8; u += 2) {
            const float4 w = *reinterpret_cast<const float4*>(s_w2 + t0 + u);     // taps t0+u, t0+u+1
            win[(u + 7) & 7] = *reinterpret_cast<const float2*>(col + (t0 + u + 7) * SC);
#pragma unroll
            for (int j = 0; j < 8; j++) acc[j] = __ffma2_rn(win[(u + j) & 7], make_float2(w.x, w.y), acc[j]);
            win[(u + 8) & 7] = *reinterpret_cast<const float2*>(col + (t0 + u + 8) * SC);
#pragma unroll
            for (int j = 0; j < 8; j++) acc[j] = __ffma2_rn(win[(u + 1 + j) & 7], make_float2(w.z, w.w), acc[j]);
        }
    }
    // the last K mod 8 taps (t0 = K8, a multiple of 8: the same slots)
#pragma unroll
    for (int u = 0; u < 7; u++) {
        if (K8 + u >= K) break;
        win[(u + 7) & 7] = *reinterpret_cast<const float2*>(col + (K8 + u + 7) * SC);
        const float2 w = s_w2[K8 + u];
#pragma unroll
        for (int j = 0; j < 8; j++) acc[j] = __ffma2_rn(win[(u + j) & 7], w, acc[j]);
    }
    Tout* dst = reinterpret_cast<Tout*>(p.dst) + tl.dof;
    const int64_t xa = tl.x0 + 2 * cp;
    const int64_t ya = tl.y0 + 8 * og;
    const int nj = na - ya < 8 ? (int)(na - ya) : 8;
    if (nj <= 0) return;
    bool vst = false;
    if constexpr (sizeof(Tout) == 4)
        vst = p.ds[0] == 1 && (p.ds[a] & 1) == 0 && (reinterpret_cast<uintptr_t>(dst + tl.x0) & 7) == 0 &&
              xa + 2 <= n0;
    Tout* d = dst + xa * p.ds[0] + ya * p.ds[a];
    const int64_t dsa = p.ds[a];
    if constexpr (sizeof(Tout) == 4) {
        if (vst) {
#pragma unroll
            for (int j = 0; j < 8; j++)
                if (j < nj) *reinterpret_cast<float2*>(reinterpret_cast<float*>(d) + j * dsa) = acc[j];
            return;
        }
    }
    const int64_t ds0 = p.ds[0];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        if (j >= nj) break;
        if (xa < n0) d[j * dsa] = stf<Tout>(acc[j].x);
        if (xa + 1 < n0) d[j * dsa + ds0] = stf<Tout>(acc[j].y);
    }
}

template <class Tin, class Tout>
__global__ void __launch_bounds__(NT, 4) k_tpass_s(const __grid_constant__ TiledPassParams p, uint32_t ntiles)
{
    extern __shared__ __align__(16) float sm_s[];
    const int K = p.ntap;
    const int nr = s_rows(K);
    float2* s_w2 = reinterpret_cast<float2*>(sm_s + 2 * nr * SC);     // (w, w) pairs
    const int tid = threadIdx.x;
    for (int i = tid; i < ((K + 1) & ~1); i += NT) s_w2[i] = i < K ? make_float2(p.w[i], p.w[i]) : make_float2(0.f, 0.f);
    uint32_t t = blockIdx.x;
    if (t >= ntiles) return;
    STile cur = s_tile(p, t);
    s_stage<Tin>(p, cur, sm_s, nr);
    cp_async_commit();
    for (int i = 0; t < ntiles; i++) {
        const uint32_t tn = t + gridDim.x;
        STile nxt = cur;
        if (tn < ntiles) {
            // the buffer of tile i+1 was last read by tile i-1, before the
            // barrier that ended its step
            nxt = s_tile(p, tn);
            s_stage<Tin>(p, nxt, sm_s + ((i + 1) & 1) * nr * SC, nr);
        }
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();   // tile i's rows (every thread's copies) and the taps visible
        s_sum_store<Tout>(p, cur, sm_s + (i & 1) * nr * SC, s_w2);
        __syncthreads();   // every thread is done with buffer i & 1
        cur = nxt;
        t = tn;
    }
    cp_async_wait<0>();
}

// The SM count of the current device (cached per device).
int sm_count()
{
    static std::atomic<int> cache[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    int n = cache[dev].load(std::memory_order_relaxed);
    if (n == 0) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = 148;
        cache[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}

// The persistent grid of a pass kernel (as many CTAs as fit at once, at most
// one per tile) and its dynamic shared-memory opt-in, each looked up once per
// kernel and tap count: the plain path launches these passes once per call,
// and the queries would otherwise cost host time on every launch.
template <class Kern>
cudaError_t persistent_grid(Kern kern, size_t smem, int K, int64_t ntiles, int64_t* grid)
{
    static std::atomic<int> smem_set{0};
    static std::atomic<int> per_sm_k[kMaxTaps + 1];
    if (smem > 48 * 1024 && (int)smem > smem_set.load(std::memory_order_relaxed)) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        int cur = smem_set.load(std::memory_order_relaxed);
        while ((int)smem > cur && !smem_set.compare_exchange_weak(cur, (int)smem)) {
        }
    }
    const int k = K < 0 ? 0 : (K > kMaxTaps ? kMaxTaps : K);
    int per_sm = per_sm_k[k].load(std::memory_order_relaxed);
    if (per_sm == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem) != cudaSuccess || per_sm < 1)
            per_sm = 1;
        per_sm_k[k].store(per_sm, std::memory_order_relaxed);
    }
    *grid = std::min<int64_t>(ntiles, (int64_t)sm_count() * per_sm);
    return cudaSuccess;
}

template <class Tin, class Tout>
cudaError_t launch_t(const TiledPassParams& p_in, cudaStream_t s)
{
    TiledPassParams p = p_in;
    for (int i = 0; i < p.rank; i++) p.dv[i].init((uint32_t)p.n[i]);
    p.dtx.init((uint32_t)((p.n[0] + (p.axis == 0 ? XO : SC) - 1) / (p.axis == 0 ? XO : SC)));
    const int K = p.ntap;
    if (p.axis == 0) {
        const size_t smem = (2 * (size_t)XR * x_pitch(K) + ((K + 3) & ~3)) * sizeof(float);
        const int64_t ntx = (p.n[0] + XO - 1) / XO;
        const int64_t ntiles = ntx * ((p.rows + XR - 1) / XR);
        if (ntiles > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
        auto kern = k_tpass_x<Tin, Tout>;
        int64_t grid = 0;
        cudaError_t e = persistent_grid(kern, smem, K, ntiles, &grid);
        if (e != cudaSuccess) return e;
        kern<<<(unsigned)grid, NT, smem, s>>>(p, (uint32_t)ntiles);
    } else {
        const size_t smem = 2 * (size_t)s_rows(K) * SC * sizeof(float) + (size_t)((K + 1) & ~1) * sizeof(float2);
        const int64_t ntx = (p.n[0] + SC - 1) / SC, nta = (p.n[p.axis] + SO - 1) / SO;
        const int64_t outer = p.rows / p.n[p.axis];
        const int64_t ntiles = ntx * nta * outer;
        if (ntiles > 0x7fffffffLL || ntx * nta > 0xffffffffLL) return cudaErrorInvalidConfiguration;
        p.dta.init((uint32_t)nta);
        auto kern = k_tpass_s<Tin, Tout>;
        int64_t grid = 0;
        cudaError_t e = persistent_grid(kern, smem, K, ntiles, &grid);
        if (e != cudaSuccess) return e;
        kern<<<(unsigned)grid, NT, smem, s>>>(p, (uint32_t)ntiles);
    }
    count_launch();
    return cudaGetLastError();
}

bool float_type(int dt) { return dt == NDLGPU_F32 || dt == NDLGPU_BF16 || dt == NDLGPU_F16; }

template <class Tin>
cudaError_t launch_in(const TiledPassParams& p, cudaStream_t s)
{
    switch (p.dst_dtype) {
    case NDLGPU_F32: return launch_t<Tin, float>(p, s);
    case NDLGPU_BF16: return launch_t<Tin, __nv_bfloat16>(p, s);
    default: return launch_t<Tin, __half>(p, s);
    }
}

}  // namespace

bool tiled_pass_supported(const TiledPassParams& p)
{
    if (!float_type(p.src_dtype) || !float_type(p.dst_dtype)) return false;
    if (p.rank < 1 || p.rank > kTiledRank || p.axis < 0 || p.axis >= p.rank) return false;
    if (p.ntap < 1 || p.ntap > kMaxTaps || p.omax - p.omin + 1 != p.ntap) return false;
    if (p.rows < 1 || p.rows >= (1LL << 31)) return false;
    for (int i = 0; i < p.rank; i++)
        if (p.n[i] >= (1LL << 30)) return false;
    // tiles of 256 (x pass) or 64 (other axes) contiguous columns: short x
    // extents (a channel axis) keep the general kernel
    if (p.n[0] < (p.axis == 0 ? 16 : 32)) return false;
    // the staged window of the widest kernel must fit one CTA's shared memory
    const size_t smx = (2 * (size_t)XR * x_pitch(p.ntap) + p.ntap + 3) * 4;
    const size_t sms = 2 * (size_t)s_rows(p.ntap) * SC * 4 + (size_t)(p.ntap + 1) * 8;
    if (smx > 200 * 1024 || sms > 200 * 1024) return false;
    return true;
}

cudaError_t launch_tiled_pass(const TiledPassParams& p, cudaStream_t s)
{
    if (!tiled_pass_supported(p)) return cudaErrorNotSupported;
    switch (p.src_dtype) {
    case NDLGPU_F32: return launch_in<float>(p, s);
    case NDLGPU_BF16: return launch_in<__nv_bfloat16>(p, s);
    default: return launch_in<__half>(p, s);
    }
}

}  // namespace ndlgpu
