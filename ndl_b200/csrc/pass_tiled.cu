// pass_tiled.cu -- one 1-D pass of any width (runtime taps) along one axis,
// FP32 accumulation, float storage (f32 / bf16 / f16 in and out): the pass
// kernels of the plain path for the widths the fused kernels do not compile
// (wide Gaussians, uneven per-axis widths, ranks above 3).
//
// The tile (outputs plus the tap window) is staged in shared memory with its
// coordinates border-mapped (Clamp / Wrap / Reflect, mathHelpers.h:23-25),
// then every thread sums four outputs, four taps at a time from a register
// window, and the last K mod 4 taps one by one (no tap past the kernel is
// ever read, so non-finite samples behave as in the reference's sum):
//   along x (the contiguous axis): 8 rows x 128 outputs per CTA, a warp per
//     row, lane l outputs 4l .. 4l+3;
//   along another axis: 64 columns x 32 outputs per CTA, a thread a column
//     pair (packed FP32 pairs) and 4 outputs along the axis.
// Taps are the pass's dense offsets omin .. omin+K-1 in ascending order.
#include "dtype.cuh"

namespace ndlgpu {
namespace {

constexpr int NT = 256;
constexpr int XO = 128;     // x pass: outputs per row
constexpr int XR = 8;       // x pass: rows per CTA
constexpr int SC = 64;      // strided pass: columns per CTA
constexpr int SO = 32;      // strided pass: outputs along the axis per CTA

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

template <class Tin, class Tout>
__global__ void __launch_bounds__(NT) k_tpass_x(const __grid_constant__ TiledPassParams p)
{
    extern __shared__ __align__(16) float sm_x[];
    const int K = p.ntap;
    const int pitch = (XO + K + 3 + 3) & ~3;       // the last lane's window reads up to XO + K + 2
    float* s_w = sm_x + XR * pitch;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t n0 = p.n[0];
    const uint32_t rb = p.dtx.div(blockIdx.x), tx = blockIdx.x - rb * p.dtx.d;
    const int64_t x0 = (int64_t)tx * XO;
    const uint32_t nrows = (uint32_t)p.rows;
    for (int i = tid; i < K; i += NT) s_w[i] = p.w[i];
    const uint32_t row = rb * XR + warp;
    int64_t so = 0, dof = 0;
    if (row < nrows) outer_offsets(p, 0, -1, row, &so, &dof);
    const Tin* src = reinterpret_cast<const Tin*>(p.src) + so;
    float* srow = sm_x + warp * pitch;
    // rows wholly inside the image, 16-byte aligned f32: float4 loads
    const int nvec = (XO + K - 1 + 3) >> 2;
    bool vec = false;
    if constexpr (sizeof(Tin) == 4)
        vec = p.ss[0] == 1 && x0 + p.omin >= 0 && x0 + p.omin + 4 * nvec <= n0 &&
              (reinterpret_cast<uintptr_t>(src + x0 + p.omin) & 15) == 0;
    if (row < nrows && vec) {
        const float4* v4 = reinterpret_cast<const float4*>(src + x0 + p.omin);
#pragma unroll 2
        for (int v = lane; v < nvec; v += 32) *reinterpret_cast<float4*>(srow + 4 * v) = v4[v];
    } else if (row < nrows) {
        // unrolled so that the loads of several iterations are in flight at once
#pragma unroll 4
        for (int j = lane; j < pitch; j += 32) {
            float v = 0.f;
            if (j < XO + K - 1) {
                int64_t x = x0 + p.omin + j;
                if (x < 0 || x >= n0) x = (x >= n0 + p.omax || x < p.omin) ? n0 - 1 : bmap(p.border, n0, x);
                v = ldf<Tin>(src + x * p.ss[0]);
            }
            srow[j] = v;
        }
    }
    __syncthreads();
    if (row >= nrows) return;
    float a[4] = {0.f, 0.f, 0.f, 0.f};
    const float* wr = srow + 4 * lane;
    const int K4 = K & ~3;
    for (int t = 0; t < K4; t += 4) {
        const float4 v0 = *reinterpret_cast<const float4*>(wr + t);
        const float4 v1 = *reinterpret_cast<const float4*>(wr + t + 4);
        const float4 w = *reinterpret_cast<const float4*>(s_w + t);
        const float win[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
        const float wq[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int q = 0; q < 4; q++)
#pragma unroll
            for (int m = 0; m < 4; m++) a[m] = fmaf(wq[q], win[m + q], a[m]);
    }
    for (int t = K4; t < K; t++) {
        const float w = s_w[t];
#pragma unroll
        for (int m = 0; m < 4; m++) a[m] = fmaf(w, wr[m + t], a[m]);
    }
    Tout* dst = reinterpret_cast<Tout*>(p.dst) + dof;
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const int64_t x = x0 + 4 * lane + m;
        if (x < n0) dst[x * p.ds[0]] = stf<Tout>(a[m]);
    }
}

template <class Tin, class Tout>
__global__ void __launch_bounds__(NT) k_tpass_s(const __grid_constant__ TiledPassParams p)
{
    extern __shared__ __align__(16) float sm_s[];
    const int K = p.ntap;
    const int nr = SO + K - 1;                       // staged rows along the axis
    float* s_w = sm_s + nr * SC;
    const int tid = threadIdx.x;
    const int a = p.axis;
    const int64_t n0 = p.n[0], na = p.n[a];
    const uint32_t ta = p.dtx.div(blockIdx.x), tx = blockIdx.x - ta * p.dtx.d;
    const int64_t x0 = (int64_t)tx * SC, y0 = (int64_t)ta * SO;
    int64_t so = 0, dof = 0;
    outer_offsets(p, 0, a, blockIdx.y, &so, &dof);
    const Tin* src = reinterpret_cast<const Tin*>(p.src) + so;
    for (int i = tid; i < K; i += NT) s_w[i] = p.w[i];
    // staged rows r = 0 .. nr-1: axis coordinate y0 + omin + r, border-mapped;
    // columns x0 .. x0+63 (past n0: zero, never stored)
    // rows of 64 columns inside the image, 16-byte aligned f32: float4 loads
    bool vec = false;
    if constexpr (sizeof(Tin) == 4)
        vec = p.ss[0] == 1 && x0 + SC <= n0 && (p.ss[a] & 3) == 0 && (reinterpret_cast<uintptr_t>(src + x0) & 15) == 0;
    if (vec) {
#pragma unroll 4
        for (int i = tid; i < nr * (SC / 4); i += NT) {
            const int r = i / (SC / 4), c4 = i - (i / (SC / 4)) * (SC / 4);
            int64_t y = y0 + p.omin + r;
            if (y < 0 || y >= na) y = (y >= na + p.omax || y < p.omin) ? na - 1 : bmap(p.border, na, y);
            *reinterpret_cast<float4*>(sm_s + r * SC + 4 * c4) =
                *reinterpret_cast<const float4*>(src + x0 + 4 * c4 + y * p.ss[a]);
        }
    } else
    // (unrolled so that the loads of several iterations are in flight at once)
#pragma unroll 8
    for (int i = tid; i < nr * SC; i += NT) {
        const int r = i / SC, c = i - (i / SC) * SC;
        float v = 0.f;
        const int64_t x = x0 + c;
        if (x < n0) {
            int64_t y = y0 + p.omin + r;
            if (y < 0 || y >= na) y = (y >= na + p.omax || y < p.omin) ? na - 1 : bmap(p.border, na, y);
            v = ldf<Tin>(src + x * p.ss[0] + y * p.ss[a]);
        }
        sm_s[i] = v;
    }
    __syncthreads();
    const int cp = tid & 31, og = tid >> 5;
    float2 acc[4] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    const float* col = sm_s + (4 * og) * SC + 2 * cp;
    const int K4 = K & ~3;
    for (int t = 0; t < K4; t += 4) {
        float2 rows[7];
#pragma unroll
        for (int j = 0; j < 7; j++) rows[j] = *reinterpret_cast<const float2*>(col + (t + j) * SC);
        const float4 w = *reinterpret_cast<const float4*>(s_w + t);
        const float wq[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int q = 0; q < 4; q++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[j] = __ffma2_rn(rows[j + q], make_float2(wq[q], wq[q]), acc[j]);
    }
    for (int t = K4; t < K; t++) {
        const float w = s_w[t];
#pragma unroll
        for (int j = 0; j < 4; j++)
            acc[j] = __ffma2_rn(*reinterpret_cast<const float2*>(col + (t + j) * SC), make_float2(w, w), acc[j]);
    }
    Tout* dst = reinterpret_cast<Tout*>(p.dst) + dof;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int64_t y = y0 + 4 * og + j;
        if (y >= na) continue;
        const int64_t xa = x0 + 2 * cp;
        if (xa < n0) dst[xa * p.ds[0] + y * p.ds[a]] = stf<Tout>(acc[j].x);
        if (xa + 1 < n0) dst[(xa + 1) * p.ds[0] + y * p.ds[a]] = stf<Tout>(acc[j].y);
    }
}

template <class Tin, class Tout>
cudaError_t launch_t(const TiledPassParams& p_in, cudaStream_t s)
{
    TiledPassParams p = p_in;
    for (int i = 0; i < p.rank; i++) p.dv[i].init((uint32_t)p.n[i]);
    p.dtx.init((uint32_t)((p.n[0] + (p.axis == 0 ? XO : SC) - 1) / (p.axis == 0 ? XO : SC)));
    const int K = p.ntap;
    if (p.axis == 0) {
        const int pitch = (XO + K + 3 + 3) & ~3;
        const size_t smem = ((size_t)XR * pitch + ((K + 3) & ~3)) * sizeof(float);
        const int64_t ntx = (p.n[0] + XO - 1) / XO;
        const int64_t nb = ntx * ((p.rows + XR - 1) / XR);
        if (nb > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k_tpass_x<Tin, Tout>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem);
            if (e != cudaSuccess) return e;
        }
        k_tpass_x<Tin, Tout><<<(unsigned)nb, NT, smem, s>>>(p);
    } else {
        const size_t smem = ((size_t)(SO + K - 1) * SC + ((K + 3) & ~3)) * sizeof(float);
        const int64_t ntx = (p.n[0] + SC - 1) / SC, nta = (p.n[p.axis] + SO - 1) / SO;
        const int64_t outer = p.rows / p.n[p.axis];
        if (ntx * nta > 0x7fffffffLL || outer > 65535) return cudaErrorInvalidConfiguration;
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k_tpass_s<Tin, Tout>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem);
            if (e != cudaSuccess) return e;
        }
        k_tpass_s<Tin, Tout><<<dim3((unsigned)(ntx * nta), (unsigned)outer), NT, smem, s>>>(p);
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
        if (p.n[i] >= (1LL << 31)) return false;
    // tiles of 128 (x pass) or 64 (other axes) contiguous columns: short x
    // extents (a channel axis) keep the general kernel
    if (p.n[0] < (p.axis == 0 ? 16 : 32)) return false;
    // the staged window of the widest kernel must fit one CTA's shared memory
    const size_t smx = ((size_t)XR * ((XO + p.ntap + 6) & ~3) + p.ntap + 3) * 4;
    const size_t sms = ((size_t)(SO + p.ntap - 1) * SC + p.ntap + 3) * 4;
    if (smx > 200 * 1024 || sms > 200 * 1024) return false;
    if (p.axis != 0 && p.rows / p.n[p.axis] > 65535) return false;
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
