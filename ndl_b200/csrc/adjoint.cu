// adjoint.cu -- general adjoint kernels (no reference counterpart: ndl has no
// gradients).  For one forward pass y[i] = sum_k w[k] * x[map(i + o_k)]
// along an axis of extent M (border map per mathHelpers.h:23-25):
//
//   input gradient  gx[j] = sum over (i, k) with map(i + o_k) == j of w[k] g[i]
//   tap gradient    dw[k] = sum_i g[i] * x[map(i + o_k)]
//
// The input gradient is written as a gather per output j: the in-range term
// i = j - o_k, plus the out-of-range positions that the border folds onto j
// --  Clamp: every position < 0 onto j = 0 and every position > M-1 onto
// j = M-1; Wrap: positions j - M and j + M; Reflect: positions -j-1 and
// 2M-1-j (the mirror images of j).  Tap gradients reduce in two fixed-order
// stages (per-block partials in double, then a per-tap sum over blocks), so
// results are bitwise reproducible run to run.
#include "dtype.cuh"

namespace ndlgpu {

namespace {

template <class A> __device__ __forceinline__ A adj_mac(A acc, A g, double w);
template <> __device__ __forceinline__ double adj_mac<double>(double acc, double g, double w) { return fma(g, w, acc); }
template <> __device__ __forceinline__ float adj_mac<float>(float acc, float g, double w) { return fmaf(g, (float)w, acc); }

// Transposed 1-D pass; p.src holds g (the gradient at the pass output),
// p.dst receives gx.  Offsets o_k = p.off[t], weights p.wd[t].
template <class A>
__global__ void __launch_bounds__(256) k_pass_adjoint(const __grid_constant__ GenericPassParams p)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < p.total; idx += stride) {
        uint32_t rem = idx;
        int64_t so = 0, dof = 0, j = 0;
#pragma unroll
        for (int i = 0; i < kMaxRank; i++) {
            if (i < p.rank) {
                const uint32_t q = p.div[i].div(rem);
                const int64_t c = (int64_t)(rem - q * p.div[i].d);
                rem = q;
                if (i == p.axis) j = c;
                else so += c * p.ss[i];
                dof += c * p.ds[i];
            }
        }
        const int64_t M = p.n[p.axis];
        const int64_t sa = p.ss[p.axis];
        A acc = A(0);
        for (int t = 0; t < p.ntap; t++) {
            const int64_t o = p.off[t];
            const double w = p.wd[t];
            // in range: position j reached from i = j - o
            int64_t i = j - o;
            if (i >= 0 && i < M) acc = adj_mac<A>(acc, load_as<A>(p.src, p.src_dtype, so + i * sa), w);
            if (p.border == NDLGPU_WRAP) {
                i = j - o + M;     // position j + M wraps to j
                if (i >= 0 && i < M) acc = adj_mac<A>(acc, load_as<A>(p.src, p.src_dtype, so + i * sa), w);
                i = j - o - M;     // position j - M wraps to j
                if (i >= 0 && i < M) acc = adj_mac<A>(acc, load_as<A>(p.src, p.src_dtype, so + i * sa), w);
            } else if (p.border == NDLGPU_REFLECT) {
                i = -j - 1 - o;    // position -j-1 reflects to j
                if (i >= 0 && i < M) acc = adj_mac<A>(acc, load_as<A>(p.src, p.src_dtype, so + i * sa), w);
                i = 2 * M - 1 - j - o;   // position 2M-1-j reflects to j
                if (i >= 0 && i < M) acc = adj_mac<A>(acc, load_as<A>(p.src, p.src_dtype, so + i * sa), w);
            } else {
                // Clamp: all positions < 0 land on 0, all > M-1 on M-1
                if (j == 0 && o < 0) {
                    const int64_t hi = (-o < M ? -o : M);
                    for (int64_t u = 0; u < hi; u++)
                        acc = adj_mac<A>(acc, load_as<A>(p.src, p.src_dtype, so + u * sa), w);
                }
                if (j == M - 1 && o > 0) {
                    const int64_t lo = (M - o > 0 ? M - o : 0);
                    for (int64_t u = lo; u < M; u++)
                        acc = adj_mac<A>(acc, load_as<A>(p.src, p.src_dtype, so + u * sa), w);
                }
            }
        }
        store_from(p.dst, p.dst_dtype, dof, acc, STORE_CAST);
    }
}

constexpr int kTapChunk = 8;

// Stage 1: per-block partial sums of dw[k] = sum_i g[i] x[map(i + o_k)],
// taps in chunks of 8; partial[block * ntap + t] (double).
template <class A>
__global__ void __launch_bounds__(256) k_tap_grad_partial(const __grid_constant__ TapGradParams p)
{
    __shared__ double s_red[8][kTapChunk];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t M = p.n[p.axis];
    for (int t0 = 0; t0 < p.ntap; t0 += kTapChunk) {
        A acc[kTapChunk];
#pragma unroll
        for (int c = 0; c < kTapChunk; c++) acc[c] = A(0);
        for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < p.total; idx += gridDim.x * blockDim.x) {
            uint32_t rem = idx;
            int64_t go = 0, xo = 0, ca = 0;
#pragma unroll
            for (int i = 0; i < kMaxRank; i++) {
                if (i < p.rank) {
                    const uint32_t q = p.div[i].div(rem);
                    const int64_t c = (int64_t)(rem - q * p.div[i].d);
                    rem = q;
                    go += c * p.gs[i];
                    if (i == p.axis) ca = c;
                    else xo += c * p.xs[i];
                }
            }
            const A g = load_as<A>(p.g, p.g_dtype, go);
#pragma unroll
            for (int c = 0; c < kTapChunk; c++) {
                if (t0 + c < p.ntap) {
                    const int64_t xi = map_border(p.border, M, ca + p.off[t0 + c]);
                    acc[c] += g * load_as<A>(p.x, p.x_dtype, xo + xi * p.xs[p.axis]);
                }
            }
        }
        // fixed-order block reduction in double
#pragma unroll
        for (int c = 0; c < kTapChunk; c++) {
            double v = (double)acc[c];
            for (int s = 16; s > 0; s >>= 1) v += __shfl_down_sync(0xffffffffu, v, s);
            if (lane == 0) s_red[warp][c] = v;
        }
        __syncthreads();
        if (threadIdx.x < kTapChunk && t0 + threadIdx.x < p.ntap) {
            double v = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += s_red[w][threadIdx.x];
            p.partial[(int64_t)blockIdx.x * p.ntap + t0 + threadIdx.x] = v;
        }
        __syncthreads();
    }
}

// Stage 2: dw[t] = sum over blocks in block order.
__global__ void k_tap_grad_final(const double* partial, int nblocks, int ntap, void* out, int out_dtype)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntap) return;
    double v = 0;
    for (int b = 0; b < nblocks; b++) v += partial[(int64_t)b * ntap + t];
    if (out_dtype == NDLGPU_F64) ((double*)out)[t] = v;
    else ((float*)out)[t] = (float)v;
}

unsigned grid_cap(uint32_t total, int per_sm)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = (uint64_t(total) + 255) / 256;
    const uint64_t cap = uint64_t(sms) * per_sm;
    return (unsigned)(want < cap ? (want ? want : 1) : cap);
}

}  // namespace

cudaError_t launch_pass_adjoint(Acc acc, const GenericPassParams& p, cudaStream_t s)
{
    if (p.total == 0) return cudaSuccess;
    const unsigned g = grid_cap(p.total, 8);
    if (acc == Acc::F64) k_pass_adjoint<double><<<g, 256, 0, s>>>(p);
    else k_pass_adjoint<float><<<g, 256, 0, s>>>(p);
    count_launch();
    return cudaGetLastError();
}

unsigned tap_grad_blocks(uint32_t total) { return grid_cap(total, 2); }

cudaError_t launch_tap_grad(Acc acc, const TapGradParams& p, unsigned nblocks, void* out, int out_dtype,
                            cudaStream_t s)
{
    if (p.total == 0 || p.ntap == 0) return cudaSuccess;
    if (acc == Acc::F64) k_tap_grad_partial<double><<<nblocks, 256, 0, s>>>(p);
    else k_tap_grad_partial<float><<<nblocks, 256, 0, s>>>(p);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_tap_grad_final<<<(p.ntap + 127) / 128, 128, 0, s>>>(p.partial, (int)nblocks, p.ntap, out, out_dtype);
    count_launch(2);
    return cudaGetLastError();
}

}  // namespace ndlgpu
