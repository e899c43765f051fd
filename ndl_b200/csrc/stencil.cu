// stencil.cu -- ndl::convolve (processing/convolution.h:52-71) with a full
// (non-separable) 2-D or 3-D kernel of up to 9 taps per axis: f32 image and
// result with FP32 accumulation (k_stencil), and integral sources of up to
// 16 bits into any type with the reference's exact double sequence
// (k_stencil_exact).  The general kernel remains the path for other types
// and for f32 kernels with zero taps, whose skipped terms matter for
// non-finite samples.
//
// A CTA owns a TX x TY x TZ output box (64 x 64 x 1 for images, 32 x 16 x 8
// for volumes; 256 threads, units of 4 consecutive outputs along x).  The
// box and its halo are loaded once into shared memory with each coordinate
// border-mapped per axis (mathHelpers.h:23-25); every kernel row then feeds
// the thread's 4 outputs from a register window of kx + 3 samples.  Taps are
// summed in the kernel's coordinates() order (x fastest, then y, then z).
#include "dtype.cuh"

namespace ndlgpu {
namespace {

// The border map for the coordinates an output inside the image reaches
// (the host checks the radius against the extent); positions only the
// discarded outputs of a partial box reach are clamped into the image.
__device__ __forceinline__ int tile_map(int border, int n, int x)
{
    const int m = map_border32(border, n, x);
    return m < 0 ? 0 : (m >= n ? n - 1 : m);
}

// KX: the kernel's x extent (compile time: the row window and its taps
// unroll); y and z extents at run time.
template <int KX>
__global__ void __launch_bounds__(256) k_stencil(const __grid_constant__ StencilParams p)
{
    extern __shared__ __align__(16) float s_t[];
    const int SX = p.tx + p.kx - 1, SY = p.ty + p.ky - 1, SZ = p.tz + p.kz - 1;
    const int bx = blockIdx.x % p.gx, rest = blockIdx.x / p.gx;
    const int by = rest % p.gy, bz = rest / p.gy;
    const int x0 = bx * p.tx, y0 = by * p.ty, z0 = bz * p.tz;
    const float* src = p.src + (int64_t)blockIdx.y * p.sb;
    float* dst = p.dst + (int64_t)blockIdx.y * p.db;
    // rows of the box by warp, columns by lane: one row offset per row
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const bool xin = x0 - p.cx >= 0 && x0 - p.cx + SX <= p.nx;   // no column of the box needs a border map
    const float* xsrc = src + (int64_t)(x0 - p.cx) * p.sx;
    for (int rr = warp; rr < SY * SZ; rr += nwarp) {
        const int r = rr % SY, q = rr / SY;
        const int64_t rowoff = (int64_t)tile_map(p.border, p.ny, y0 - p.cy + r) * p.sy +
                               (int64_t)tile_map(p.border, p.nz, z0 - p.cz + q) * p.sz;
        if (xin) {
            for (int c = lane; c < SX; c += 32) s_t[rr * SX + c] = __ldg(xsrc + rowoff + (int64_t)c * p.sx);
        } else {
            for (int c = lane; c < SX; c += 32)
                s_t[rr * SX + c] = __ldg(src + rowoff + (int64_t)tile_map(p.border, p.nx, x0 - p.cx + c) * p.sx);
        }
    }
    __syncthreads();
    // units of 4 outputs: column group g, row ry, plane rz (box sides are
    // powers of two: shifts and masks)
    const int units = (p.tx >> 2) * p.ty * p.tz;
    for (int u = threadIdx.x; u < units; u += blockDim.x) {
        const int g = u & ((p.tx >> 2) - 1);
        const int ry = (u >> p.lgx) & (p.ty - 1);
        const int rz = u >> (p.lgx + p.lgy);
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        int wi = 0;
        for (int dz = 0; dz < p.kz; dz++) {
            for (int dy = 0; dy < p.ky; dy++) {
                const float* row = s_t + ((rz + dz) * SY + (ry + dy)) * SX + 4 * g;
                float win[KX + 3];
#pragma unroll
                for (int j = 0; j < KX + 3; j++) win[j] = row[j];
#pragma unroll
                for (int k = 0; k < KX; k++) {
                    const float wk = p.w[wi + k];
#pragma unroll
                    for (int m = 0; m < 4; m++) acc[m] = fmaf(win[m + k], wk, acc[m]);
                }
                wi += KX;
            }
        }
        const int oy = y0 + ry, oz = z0 + rz;
        if (oy >= p.ny || oz >= p.nz) continue;
        float* orow = dst + (int64_t)oy * p.dy + (int64_t)oz * p.dz;
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const int ox = x0 + 4 * g + m;
            if (ox < p.nx) orow[(int64_t)ox * p.dx] = acc[m];
        }
    }
}

// The exact form for integral sources of at most 16 bits (exact in the float
// shared tile): per output, total = total + double(x) * double(w) in the
// kernel's coordinates() order, each product and sum rounded as the
// reference's double arithmetic rounds them (convolution.h:66-68), then
// DstT's static_cast (truncation for integral DstT, :69).  Zero taps are
// summed too: with integral samples every such term is +-0 and leaves a
// finite total unchanged, so the result equals the reference's, which skips
// them.
template <class T, int KX>
__global__ void __launch_bounds__(256) k_stencil_exact(const __grid_constant__ StencilParams p)
{
    extern __shared__ __align__(16) float s_t[];
    const int SX = p.tx + p.kx - 1, SY = p.ty + p.ky - 1, SZ = p.tz + p.kz - 1;
    const int bx = blockIdx.x % p.gx, rest = blockIdx.x / p.gx;
    const int by = rest % p.gy, bz = rest / p.gy;
    const int x0 = bx * p.tx, y0 = by * p.ty, z0 = bz * p.tz;
    const T* src = reinterpret_cast<const T*>(p.srcc);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int rr = warp; rr < SY * SZ; rr += nwarp) {
        const int r = rr % SY, q = rr / SY;
        const int64_t rowoff = (int64_t)tile_map(p.border, p.ny, y0 - p.cy + r) * p.sy +
                               (int64_t)tile_map(p.border, p.nz, z0 - p.cz + q) * p.sz;
        for (int c = lane; c < SX; c += 32)
            s_t[rr * SX + c] = (float)__ldg(src + rowoff + (int64_t)tile_map(p.border, p.nx, x0 - p.cx + c) * p.sx);
    }
    __syncthreads();
    const int units = (p.tx >> 2) * p.ty * p.tz;
    for (int u = threadIdx.x; u < units; u += blockDim.x) {
        const int g = u & ((p.tx >> 2) - 1);
        const int ry = (u >> p.lgx) & (p.ty - 1);
        const int rz = u >> (p.lgx + p.lgy);
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        int wi = 0;
        for (int dz = 0; dz < p.kz; dz++) {
            for (int dy = 0; dy < p.ky; dy++) {
                const float* row = s_t + ((rz + dz) * SY + (ry + dy)) * SX + 4 * g;
                float win[KX + 3];
#pragma unroll
                for (int j = 0; j < KX + 3; j++) win[j] = row[j];
#pragma unroll
                for (int k = 0; k < KX; k++) {
                    const double wk = p.wd[wi + k];
#pragma unroll
                    for (int m = 0; m < 4; m++) acc[m] = __dadd_rn(acc[m], __dmul_rn((double)win[m + k], wk));
                }
                wi += KX;
            }
        }
        const int oy = y0 + ry, oz = z0 + rz;
        if (oy >= p.ny || oz >= p.nz) continue;
        const int64_t orow = (int64_t)oy * p.dy + (int64_t)oz * p.dz;
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const int ox = x0 + 4 * g + m;
            if (ox < p.nx) store_from(p.dstc, p.ddt, orow + (int64_t)ox * p.dx, acc[m], STORE_CAST);
        }
    }
}

}  // namespace

namespace {
// Output box and grid of one launch; false when the grid does not fit.
bool stencil_box(StencilParams& p, long long* blocks, size_t* smem)
{
    if (p.nz == 1 && p.kz == 1) {
        p.tx = 64; p.ty = 64; p.tz = 1; p.lgx = 4; p.lgy = 6;
    } else {
        p.tx = 32; p.ty = 16; p.tz = 8; p.lgx = 3; p.lgy = 4;
    }
    p.gx = (p.nx + p.tx - 1) / p.tx;
    p.gy = (p.ny + p.ty - 1) / p.ty;
    const long long gz = (p.nz + p.tz - 1) / p.tz;
    *blocks = (long long)p.gx * p.gy * gz;
    *smem = (size_t)(p.tx + p.kx - 1) * (p.ty + p.ky - 1) * (p.tz + p.kz - 1) * sizeof(float);
    return *blocks <= 0x7fffffffLL && p.nb <= 65535 && p.kx >= 1 && p.kx <= kStencilMaxTaps;
}
}  // namespace

cudaError_t launch_stencil_exact(StencilParams p, cudaStream_t s)
{
    long long blocks;
    size_t smem;
    if (!stencil_box(p, &blocks, &smem)) return cudaErrorInvalidConfiguration;
    using Fn = void (*)(StencilParams);
#define NDLGPU_SE(T) {k_stencil_exact<T, 1>, k_stencil_exact<T, 2>, k_stencil_exact<T, 3>, k_stencil_exact<T, 4>, \
                      k_stencil_exact<T, 5>, k_stencil_exact<T, 6>, k_stencil_exact<T, 7>, k_stencil_exact<T, 8>, \
                      k_stencil_exact<T, 9>}
    static const Fn fu8[kStencilMaxTaps] = NDLGPU_SE(uint8_t);
    static const Fn fu16[kStencilMaxTaps] = NDLGPU_SE(uint16_t);
    static const Fn fi16[kStencilMaxTaps] = NDLGPU_SE(int16_t);
#undef NDLGPU_SE
    const Fn* fns = p.sdt == NDLGPU_U8 ? fu8 : (p.sdt == NDLGPU_U16 ? fu16 : (p.sdt == NDLGPU_I16 ? fi16 : nullptr));
    if (!fns) return cudaErrorInvalidValue;
    static bool configured = false;
    if (!configured) {
        for (const Fn* t : {fu8, fu16, fi16})
            for (int i = 0; i < kStencilMaxTaps; i++) {
                cudaError_t e = cudaFuncSetAttribute(t[i], cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
                if (e != cudaSuccess) return e;
            }
        configured = true;
    }
    fns[p.kx - 1]<<<dim3((unsigned)blocks, (unsigned)p.nb), 256, smem, s>>>(p);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_stencil(StencilParams p, cudaStream_t s)
{
    // boxes of 4096 outputs (16 per thread) amortise the halo and the load
    // latency of each box
    if (p.nz == 1 && p.kz == 1) {
        p.tx = 64; p.ty = 64; p.tz = 1; p.lgx = 4; p.lgy = 6;
    } else {
        p.tx = 32; p.ty = 16; p.tz = 8; p.lgx = 3; p.lgy = 4;
    }
    p.gx = (p.nx + p.tx - 1) / p.tx;
    p.gy = (p.ny + p.ty - 1) / p.ty;
    const long long gz = (p.nz + p.tz - 1) / p.tz;
    const long long blocks = (long long)p.gx * p.gy * gz;
    if (blocks > 0x7fffffffLL || p.nb > 65535) return cudaErrorInvalidConfiguration;
    const size_t smem = (size_t)(p.tx + p.kx - 1) * (p.ty + p.ky - 1) * (p.tz + p.kz - 1) * sizeof(float);
    using Fn = void (*)(StencilParams);
    static const Fn fns[kStencilMaxTaps] = {k_stencil<1>, k_stencil<2>, k_stencil<3>, k_stencil<4>, k_stencil<5>,
                                            k_stencil<6>, k_stencil<7>, k_stencil<8>, k_stencil<9>};
    if (p.kx < 1 || p.kx > kStencilMaxTaps) return cudaErrorInvalidValue;
    static bool configured = false;
    if (!configured) {
        for (Fn f : fns) {
            cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
            if (e != cudaSuccess) return e;
        }
        configured = true;
    }
    fns[p.kx - 1]<<<dim3((unsigned)blocks, (unsigned)p.nb), 256, smem, s>>>(p);
    count_launch();
    return cudaGetLastError();
}

}  // namespace ndlgpu
