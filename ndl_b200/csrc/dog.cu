// dog.cu -- the Difference-of-Gaussians scale space of ndl::detect_keypoints
// (processing/feature_detection.h:101-122): num_scales Gaussian levels of one
// image, sigma_i = sigma0 * 2^(i / (num_scales - 3)), each a gaussian_blur()
// with Reflect borders (convolution.h:107-186), and the differences of
// consecutive levels.
//
// k_dog2d (2-D images, FP32 results): one read of the source per tile, every
// level and difference from it.  A CTA owns 64 x 32 outputs.  It loads the
// tile with the largest level's halo once (Reflect-mapped, converted to
// float) into shared memory, then per level runs the X pass over the rows
// that level's Y pass needs (one unit = 2 rows x 4 outputs as packed FP32
// pairs; lanes of a warp take consecutive rows, conflict-free on the odd
// pitch), then the Y pass (2 columns x DTY/8 rows per thread, packed), keeps the
// level in registers and writes level - previous level.  Both passes keep
// their sample window in slots indexed by tap mod 4 (a tap loop unrolled by
// 4, the last K mod 4 taps guarded), so no value is ever moved between
// registers.  The
// source is read once instead of num_scales times, and no level goes through
// HBM unless the caller asks for it.
//
// k_sub_nd: dst = a - b elementwise in double for any rank, dtype and
// strides (the differences of the per-level path for other ranks and for
// FP64 results).
#include <type_traits>

#include "dtype.cuh"

namespace ndlgpu {
namespace {

constexpr int DTX = 64;     // outputs per tile along x
constexpr int DTY = 32;     // outputs per tile along y
constexpr int DNT = 256;    // threads: Y pass = 32 column pairs x 8 row groups
constexpr int RPT = DTY / (DNT / 32);   // Y-pass rows per thread (window slots)
constexpr int XP = DTX + 4; // pitch of the X-pass buffer (float4 row stores spread over the banks)

// Reflect (mathHelpers.h:24) for the coordinates an output inside the image
// can reach (radius <= extent); coordinates only reached by the discarded
// outputs of a partial tile are clamped into the image.
__device__ __forceinline__ int reflect_tile(int x, int n)
{
    int m = x < 0 ? -x - 1 : (x >= n ? 2 * n - x - 1 : x);
    return m < 0 ? 0 : (m >= n ? n - 1 : m);
}

template <class T> __device__ __forceinline__ float src_f(const T* p, int64_t i);
template <> __device__ __forceinline__ float src_f<float>(const float* p, int64_t i) { return __ldg(p + i); }
template <> __device__ __forceinline__ float src_f<uint8_t>(const uint8_t* p, int64_t i) { return (float)__ldg(p + i); }
template <> __device__ __forceinline__ float src_f<__half>(const __half* p, int64_t i) { return __half2float(__ldg(p + i)); }
template <> __device__ __forceinline__ float src_f<__nv_bfloat16>(const __nv_bfloat16* p, int64_t i)
{
    return __bfloat162float(__ldg(p + i));
}

// Stores of one output pair (columns ox, ox+1 of row oy).
__device__ __forceinline__ void store_pair(float* base, int64_t sx, int64_t sy, int vec, int ox, int oy, int nx,
                                           float2 v)
{
    float* q = base + (int64_t)ox * sx + (int64_t)oy * sy;
    if (vec && ox + 1 < nx) {
        *reinterpret_cast<float2*>(q) = v;
    } else {
        if (ox < nx) q[0] = v.x;
        if (ox + 1 < nx) q[sx] = v.y;
    }
}

// T: the source type (void: any exact-in-float type through load_as).
template <class T>
__global__ void __launch_bounds__(DNT, 2) k_dog2d(const __grid_constant__ DogParams p)
{
    extern __shared__ __align__(16) float sm[];
    const int R = p.R;
    const int SW = DTX + 2 * R;         // source tile width
    const int SP = SW | 1;              // odd pitch
    const int SH = DTY + 2 * R;         // source tile height
    float* s_src = sm;
    float* s_x = sm + ((SH * SP + 3) & ~3);
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int x0 = blockIdx.x * DTX;
    const int y0 = blockIdx.y * DTY;

    // the tile with the largest halo, Reflect-mapped, as float
    for (int r = warp; r < SH; r += DNT / 32) {
        const int64_t rowoff = (int64_t)reflect_tile(y0 - R + r, p.ny) * p.sy;
        for (int c = lane; c < SW; c += 32) {
            const int64_t i = rowoff + (int64_t)reflect_tile(x0 - R + c, p.nx) * p.sx;
            float v;
            if constexpr (std::is_void<T>::value) v = load_as<float>(p.src, p.sdt, i);
            else v = src_f<T>(reinterpret_cast<const T*>(p.src), i);
            s_src[r * SP + c] = v;
        }
    }
    __syncthreads();

    // Y-pass outputs of this thread: columns cx, cx+1 of rows ry .. ry+RPT-1
    const int cx = 2 * lane;
    const int ry = RPT * warp;
    const int ox = x0 + cx;
    float2 prev[RPT];
#pragma unroll
    for (int j = 0; j < RPT; j++) prev[j] = make_float2(0.f, 0.f);

    for (int s = 0; s < p.ns; s++) {
        const int r = p.r[s];
        const int K = 2 * r + 1;
        const int H = DTY / 2 + r;     // X-pass rows come in pairs (i, i + H)
        const float2* w2 = p.w2[s];
        // X pass: unit u = rows (i, i+H) x columns 4g .. 4g+3, packed as
        // (row i, row i+H) pairs; lanes take consecutive i (odd pitch: no
        // bank conflicts).  Window slot m holds column offset k+m (mod 4), so
        // the window never moves.
        for (int u = tid; u < H * (DTX / 4); u += DNT) {
            const int g = u / H, i = u - g * H;
            const float* s0 = s_src + (i + R - r) * SP + 4 * g + (R - r);
            const float* s1 = s0 + H * SP;
            float2 wv[4];
            wv[0] = make_float2(s0[0], s1[0]);
            wv[1] = make_float2(s0[1], s1[1]);
            wv[2] = make_float2(s0[2], s1[2]);
            wv[3] = make_float2(0.f, 0.f);
            float2 a[4] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f),
                           make_float2(0.f, 0.f)};
            int k = 0;
            for (; k + 4 <= K; k += 4) {
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    wv[(q + 3) & 3] = make_float2(s0[k + q + 3], s1[k + q + 3]);
                    const float2 wk = w2[k + q];
#pragma unroll
                    for (int m = 0; m < 4; m++) a[m] = __ffma2_rn(wv[(q + m) & 3], wk, a[m]);
                }
            }
            // the last K mod 4 taps, the same slots
#pragma unroll
            for (int q = 0; q < 3; q++) {
                if (k + q < K) {
                    wv[(q + 3) & 3] = make_float2(s0[k + q + 3], s1[k + q + 3]);
                    const float2 wk = w2[k + q];
#pragma unroll
                    for (int m = 0; m < 4; m++) a[m] = __ffma2_rn(wv[(q + m) & 3], wk, a[m]);
                }
            }
            *reinterpret_cast<float4*>(s_x + i * XP + 4 * g) = make_float4(a[0].x, a[1].x, a[2].x, a[3].x);
            *reinterpret_cast<float4*>(s_x + (i + H) * XP + 4 * g) = make_float4(a[0].y, a[1].y, a[2].y, a[3].y);
        }
        __syncthreads();
        // Y pass: (column cx, column cx+1) pairs down rows ry .. ry+RPT-1,
        // window slot m holding row k+m (mod RPT)
        float2 cur[RPT];
#pragma unroll
        for (int j = 0; j < RPT; j++) cur[j] = make_float2(0.f, 0.f);
        {
            const float* xp = s_x + ry * XP + cx;
            float2 v[RPT];
#pragma unroll
            for (int j = 0; j + 1 < RPT; j++) v[j] = *reinterpret_cast<const float2*>(xp + j * XP);
            v[RPT - 1] = make_float2(0.f, 0.f);
            int k = 0;
            for (; k + RPT <= K; k += RPT) {
#pragma unroll
                for (int q = 0; q < RPT; q++) {
                    v[(q + RPT - 1) % RPT] = *reinterpret_cast<const float2*>(xp + (k + q + RPT - 1) * XP);
                    const float2 wk = w2[k + q];
#pragma unroll
                    for (int j = 0; j < RPT; j++) cur[j] = __ffma2_rn(v[(q + j) % RPT], wk, cur[j]);
                }
            }
#pragma unroll
            for (int q = 0; q + 1 < RPT; q++) {
                if (k + q < K) {
                    v[(q + RPT - 1) % RPT] = *reinterpret_cast<const float2*>(xp + (k + q + RPT - 1) * XP);
                    const float2 wk = w2[k + q];
#pragma unroll
                    for (int j = 0; j < RPT; j++) cur[j] = __ffma2_rn(v[(q + j) % RPT], wk, cur[j]);
                }
            }
        }
        __syncthreads();    // the next level's X pass reuses s_x
        if (ox < p.nx) {
            float* lv = p.lv[s];
            float* dg = s > 0 ? p.dg[s - 1] : nullptr;
#pragma unroll
            for (int j = 0; j < RPT; j++) {
                const int oy = y0 + ry + j;
                if (oy >= p.ny) break;
                if (lv) store_pair(lv, p.lx[s], p.ly[s], p.lvec[s], ox, oy, p.nx, cur[j]);
                if (dg)
                    store_pair(dg, p.gx[s - 1], p.gy[s - 1], p.gvec[s - 1], ox, oy, p.nx,
                               make_float2(cur[j].x - prev[j].x, cur[j].y - prev[j].y));
            }
        }
#pragma unroll
        for (int j = 0; j < RPT; j++) prev[j] = cur[j];
    }
}

__global__ void __launch_bounds__(256) k_sub_nd(const SubParams p)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.total; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t rem = i, oa = 0, ob = 0, od = 0;
        for (int d = 0; d < p.rank; d++) {
            const int64_t c = rem % p.ext[d];
            rem /= p.ext[d];
            oa += c * p.as[d];
            ob += c * p.bs[d];
            od += c * p.ds[d];
        }
        const double v = load_as<double>(p.a, p.adt, oa) - load_as<double>(p.b, p.bdt, ob);
        store_from(p.dst, p.ddt, od, v, STORE_CAST);
    }
}

}  // namespace

size_t dog2d_smem_bytes(int R)
{
    const int SW = DTX + 2 * R, SP = SW | 1, SH = DTY + 2 * R;
    return (size_t)(((SH * SP + 3) & ~3) + SH * XP) * sizeof(float);
}

cudaError_t launch_dog2d(const DogParams& p, cudaStream_t s)
{
    const size_t smem = dog2d_smem_bytes(p.R);
    static size_t configured = 0;
    if (smem > configured) {
        cudaError_t e = cudaSuccess;
        for (const void* k : {(const void*)k_dog2d<float>, (const void*)k_dog2d<uint8_t>, (const void*)k_dog2d<__half>,
                              (const void*)k_dog2d<__nv_bfloat16>, (const void*)k_dog2d<void>})
            if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = smem;
    }
    const dim3 grid((unsigned)((p.nx + DTX - 1) / DTX), (unsigned)((p.ny + DTY - 1) / DTY));
    if (grid.y > 65535) return cudaErrorInvalidConfiguration;
    switch (p.sdt) {
    case NDLGPU_F32: k_dog2d<float><<<grid, DNT, smem, s>>>(p); break;
    case NDLGPU_U8: k_dog2d<uint8_t><<<grid, DNT, smem, s>>>(p); break;
    case NDLGPU_F16: k_dog2d<__half><<<grid, DNT, smem, s>>>(p); break;
    case NDLGPU_BF16: k_dog2d<__nv_bfloat16><<<grid, DNT, smem, s>>>(p); break;
    default: k_dog2d<void><<<grid, DNT, smem, s>>>(p); break;
    }
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_sub(const SubParams& p, cudaStream_t s)
{
    if (p.total == 0) return cudaSuccess;
    const int64_t blocks = (p.total + 255) / 256;
    const unsigned g = (unsigned)(blocks < 148 * 16 ? blocks : 148 * 16);
    k_sub_nd<<<g, 256, 0, s>>>(p);
    count_launch();
    return cudaGetLastError();
}

}  // namespace ndlgpu
