// gauss_exact.cu -- ndl::gaussian_blur (processing/convolution.h:107-186) of
// a 2-D integral image (sources of up to 16 bits, exact in float) in one
// pass over it, with the reference's own double arithmetic: pass 0 along x
// into double, pass 1 along y in double, each sum `total = total + x * w` in
// tap order with every product and sum rounded (convolution.h:66-68, no
// contraction), then std::round and DstT's cast (:180-185).  The reference
// runs the two passes through two full double images; here a CTA loads its
// 64 x 32 output box with the y and x halos once (each coordinate
// border-mapped, mathHelpers.h:23-25), runs the x pass over the rows the y
// pass needs into a double tile, and the y pass from it, so the results are
// the reference's bit for bit with one read of the source and one write.
#include "dtype.cuh"

namespace ndlgpu {
namespace {

constexpr int GX = 64, GY = 32, GNT = 256;

__device__ __forceinline__ int gmap(int border, int n, int x)
{
    const int m = map_border32(border, n, x);
    return m < 0 ? 0 : (m >= n ? n - 1 : m);
}

template <class T>
__global__ void __launch_bounds__(GNT) k_gauss2d_exact(const __grid_constant__ GaussExactParams p)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int SW = GX + p.kx - 1, SH = GY + p.ky - 1;
    double* s_x = reinterpret_cast<double*>(smem);                  // SH x GX
    float* s_src = reinterpret_cast<float*>(smem + (size_t)SH * GX * sizeof(double));   // SH x SW
    const int x0 = blockIdx.x * GX, y0 = blockIdx.y * GY;
    const T* src = reinterpret_cast<const T*>(p.src) + (int64_t)blockIdx.z * p.sb;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = warp; r < SH; r += GNT / 32) {
        const int64_t rowoff = (int64_t)gmap(p.border, p.ny, y0 - p.cy + r) * p.sy;
        for (int c = lane; c < SW; c += 32)
            s_src[r * SW + c] = (float)__ldg(src + rowoff + (int64_t)gmap(p.border, p.nx, x0 - p.cx + c) * p.sx);
    }
    __syncthreads();
    // x pass over every row the y pass reads; units of 4 consecutive
    // outputs, whose 4 sums are independent chains (the sum of one output
    // is a chain of dependent double additions)
    for (int i = threadIdx.x; i < SH * (GX / 4); i += GNT) {
        const int r = i / (GX / 4), c = 4 * (i - r * (GX / 4));
        const float* row = s_src + r * SW + c;
        double t[4] = {0.0, 0.0, 0.0, 0.0};
        float v0 = row[0], v1 = row[1], v2 = row[2];
        for (int k = 0; k < p.kx; k++) {
            const float v3 = row[k + 3];     // column c + kx + 2 < SW at most
            const double wk = p.wx[k];
            t[0] = __dadd_rn(t[0], __dmul_rn((double)v0, wk));
            t[1] = __dadd_rn(t[1], __dmul_rn((double)v1, wk));
            t[2] = __dadd_rn(t[2], __dmul_rn((double)v2, wk));
            t[3] = __dadd_rn(t[3], __dmul_rn((double)v3, wk));
            v0 = v1;
            v1 = v2;
            v2 = v3;
        }
        double* xo = s_x + r * GX + c;
        xo[0] = t[0];
        xo[1] = t[1];
        xo[2] = t[2];
        xo[3] = t[3];
    }
    __syncthreads();
    // y pass, round, cast: each thread sums 4 outputs of a row GX/4 apart,
    // so that a warp's shared-memory reads are consecutive doubles
    char* dst = p.dst + (int64_t)blockIdx.z * p.db * p.des;
    for (int i = threadIdx.x; i < GY * (GX / 4); i += GNT) {
        const int r = i / (GX / 4), c = i - r * (GX / 4);
        const int oy = y0 + r;
        if (oy >= p.ny) continue;
        double t[4] = {0.0, 0.0, 0.0, 0.0};
        for (int k = 0; k < p.ky; k++) {
            const double* xr = s_x + (r + k) * GX + c;
            const double wk = p.wy[k];
#pragma unroll
            for (int m = 0; m < 4; m++) t[m] = __dadd_rn(t[m], __dmul_rn(xr[m * (GX / 4)], wk));
        }
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const int ox = x0 + c + m * (GX / 4);
            if (ox < p.nx) store_from(dst, p.ddt, (int64_t)ox * p.dx + (int64_t)oy * p.dy, t[m], p.store_mode);
        }
    }
}

// The z pass of a 3-D integral gaussian over the double volume the x/y
// kernel wrote (the reference's bufB): each thread owns one (x, y) column
// and ZC consecutive outputs along z, ZC independent chains over a sliding
// register window of the column (border-mapped per plane), then the final
// round and DstT's cast.  Consecutive threads read consecutive x of a
// plane; the planes a chunk shares with its neighbours stay in L2.
constexpr int ZC = 8, ZNT = 256;

__global__ void __launch_bounds__(ZNT) k_gauss_z_exact(const __grid_constant__ GaussZExactParams p)
{
    const int64_t plane = (int64_t)p.nx * p.ny;
    const int64_t xy = (int64_t)blockIdx.x * ZNT + threadIdx.x;
    if (xy >= plane) return;
    const int z0 = blockIdx.y * ZC;
    const double* col = p.src + xy;
    double t[ZC], v[ZC];
#pragma unroll
    for (int m = 0; m < ZC; m++) t[m] = 0.0;
#pragma unroll
    for (int m = 0; m < ZC - 1; m++) v[m] = col[plane * gmap(p.border, p.nz, z0 - p.cz + m)];
    for (int k = 0; k < p.kz; k++) {
        v[ZC - 1] = col[plane * gmap(p.border, p.nz, z0 - p.cz + k + ZC - 1)];
        const double wk = p.wz[k];
#pragma unroll
        for (int m = 0; m < ZC; m++) t[m] = __dadd_rn(t[m], __dmul_rn(v[m], wk));
#pragma unroll
        for (int m = 0; m < ZC - 1; m++) v[m] = v[m + 1];
    }
    const int x = (int)(xy % p.nx), y = (int)(xy / p.nx);
    const int64_t o = (int64_t)x * p.dx + (int64_t)y * p.dy;
#pragma unroll
    for (int m = 0; m < ZC; m++)
        if (z0 + m < p.nz) store_from(p.dst, p.ddt, o + (int64_t)(z0 + m) * p.dz, t[m], STORE_ROUND);
}

}  // namespace

size_t gauss2d_exact_smem(int kx, int ky)
{
    const int SW = GX + kx - 1, SH = GY + ky - 1;
    return (size_t)SH * GX * sizeof(double) + (size_t)SH * SW * sizeof(float);
}

cudaError_t launch_gauss2d_exact(const GaussExactParams& p, cudaStream_t s)
{
    const size_t smem = gauss2d_exact_smem(p.kx, p.ky);
    if (smem > 200 * 1024 || p.nb > 65535) return cudaErrorInvalidConfiguration;
    static size_t configured = 0;
    if (smem > configured) {
        for (auto f : {k_gauss2d_exact<uint8_t>, k_gauss2d_exact<uint16_t>, k_gauss2d_exact<int16_t>}) {
            cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        configured = smem;
    }
    const dim3 grid((unsigned)((p.nx + GX - 1) / GX), (unsigned)((p.ny + GY - 1) / GY), (unsigned)p.nb);
    if (grid.y > 65535) return cudaErrorInvalidConfiguration;
    switch (p.sdt) {
    case NDLGPU_U8: k_gauss2d_exact<uint8_t><<<grid, GNT, smem, s>>>(p); break;
    case NDLGPU_U16: k_gauss2d_exact<uint16_t><<<grid, GNT, smem, s>>>(p); break;
    case NDLGPU_I16: k_gauss2d_exact<int16_t><<<grid, GNT, smem, s>>>(p); break;
    default: return cudaErrorInvalidValue;
    }
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_gauss_z_exact(const GaussZExactParams& p, cudaStream_t s)
{
    const int64_t plane = (int64_t)p.nx * p.ny;
    const int64_t gx = (plane + ZNT - 1) / ZNT, gy = (p.nz + ZC - 1) / ZC;
    if (gx > 0x7fffffff || gy > 65535 || p.kz > 128) return cudaErrorInvalidConfiguration;
    k_gauss_z_exact<<<dim3((unsigned)gx, (unsigned)gy), ZNT, 0, s>>>(p);
    count_launch();
    return cudaGetLastError();
}

}  // namespace ndlgpu
