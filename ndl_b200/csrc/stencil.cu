// stencil.cu -- ndl::convolve (processing/convolution.h:52-71) with a full
// (non-separable) 2-D or 3-D kernel of up to 9 taps per axis, f32 image and
// result, FP32 accumulation (the general kernel's double sequence remains
// the path for integral and f64 data and for kernels with zero taps, whose
// skipped terms matter for non-finite samples).
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

}  // namespace

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
