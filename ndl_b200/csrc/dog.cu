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
// that level's Y pass needs (one unit = 4 outputs from a rolling register
// window; lanes of a warp take consecutive rows, conflict-free on the odd
// pitch), then the Y pass (8 rows per thread, rolling window down a column),
// keeps the level in registers and writes level - previous level.  The
// source is read once instead of num_scales times, and no level goes through
// HBM unless the caller asks for it.
//
// k_sub_nd: dst = a - b elementwise in double for any rank, dtype and
// strides (the differences of the per-level path for other ranks and for
// FP64 results).
#include "dtype.cuh"

namespace ndlgpu {
namespace {

constexpr int DTX = 64;     // outputs per tile along x
constexpr int DTY = 32;     // outputs per tile along y
constexpr int DNT = 256;    // threads: Y pass = 64 columns x 4 groups of 8 rows
constexpr int XP = DTX + 4; // pitch of the X-pass buffer (float4 row stores spread over the banks)

// Reflect (mathHelpers.h:24) for the coordinates an output inside the image
// can reach (radius <= extent); coordinates only reached by the discarded
// outputs of a partial tile are clamped into the image.
__device__ __forceinline__ int reflect_tile(int x, int n)
{
    int m = x < 0 ? -x - 1 : (x >= n ? 2 * n - x - 1 : x);
    return m < 0 ? 0 : (m >= n ? n - 1 : m);
}

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
    const int x0 = blockIdx.x * DTX;
    const int y0 = blockIdx.y * DTY;

    for (int i = tid; i < SH * SW; i += DNT) {
        const int r = i / SW, c = i - r * SW;
        const int gy = reflect_tile(y0 - R + r, p.ny);
        const int gx = reflect_tile(x0 - R + c, p.nx);
        s_src[r * SP + c] = load_as<float>(p.src, p.sdt, (int64_t)gx * p.sx + (int64_t)gy * p.sy);
    }
    __syncthreads();

    const int tx = tid & (DTX - 1);
    const int tg = tid / DTX;
    const int ox = x0 + tx;
    float prev[8];
#pragma unroll
    for (int j = 0; j < 8; j++) prev[j] = 0.f;

    for (int s = 0; s < p.ns; s++) {
        const int r = p.r[s];
        const int K = 2 * r + 1;
        const int rows = DTY + 2 * r;
        const float* w = p.w[s];
        // X pass: unit u = (row u % rows, columns 4g .. 4g+3 with g = u / rows)
        for (int u = tid; u < rows * (DTX / 4); u += DNT) {
            const int g = u / rows, row = u - g * rows;
            const float* sp = s_src + (row + R - r) * SP + 4 * g + (R - r);
            float v0 = sp[0], v1 = sp[1], v2 = sp[2];
            float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll 4
            for (int k = 0; k < K; k++) {
                const float v3 = sp[k + 3];
                const float wk = w[k];
                a0 = fmaf(v0, wk, a0);
                a1 = fmaf(v1, wk, a1);
                a2 = fmaf(v2, wk, a2);
                a3 = fmaf(v3, wk, a3);
                v0 = v1;
                v1 = v2;
                v2 = v3;
            }
            *reinterpret_cast<float4*>(s_x + row * XP + 4 * g) = make_float4(a0, a1, a2, a3);
        }
        __syncthreads();
        // Y pass: rows 8tg .. 8tg+7 of column tx
        float cur[8];
        {
            const float* xp = s_x + 8 * tg * XP + tx;
            float v[8];
#pragma unroll
            for (int j = 0; j < 7; j++) v[j] = xp[j * XP];
#pragma unroll
            for (int j = 0; j < 8; j++) cur[j] = 0.f;
#pragma unroll 2
            for (int k = 0; k < K; k++) {
                v[7] = xp[(k + 7) * XP];
                const float wk = w[k];
#pragma unroll
                for (int j = 0; j < 8; j++) cur[j] = fmaf(v[j], wk, cur[j]);
#pragma unroll
                for (int j = 0; j < 7; j++) v[j] = v[j + 1];
            }
        }
        __syncthreads();    // the next level's X pass reuses s_x
        if (ox < p.nx) {
            float* lv = p.lv[s];
            float* dg = s > 0 ? p.dg[s - 1] : nullptr;
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const int oy = y0 + 8 * tg + j;
                if (oy >= p.ny) break;
                if (lv) lv[(int64_t)ox * p.lx[s] + (int64_t)oy * p.ly[s]] = cur[j];
                if (dg) dg[(int64_t)ox * p.gx[s - 1] + (int64_t)oy * p.gy[s - 1]] = cur[j] - prev[j];
            }
        }
#pragma unroll
        for (int j = 0; j < 8; j++) prev[j] = cur[j];
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
        cudaError_t e = cudaFuncSetAttribute(k_dog2d, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = smem;
    }
    const dim3 grid((unsigned)((p.nx + DTX - 1) / DTX), (unsigned)((p.ny + DTY - 1) / DTY));
    if (grid.y > 65535) return cudaErrorInvalidConfiguration;
    k_dog2d<<<grid, DNT, smem, s>>>(p);
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
