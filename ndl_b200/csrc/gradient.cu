// gradient.cu -- ndl::gradient (processing/convolution.h:359-388) in one
// pass over the source.
//
// The reference runs one convolve() per axis with the taps {-0.5, 0, +0.5}
// (zero centre tap skipped), each into dst.slice(0, axis).  Here one thread
// takes one voxel: it reads the 2*DIM axis neighbours (border-mapped like
// every other pass, mathHelpers.h:23-25) and writes the DIM central
// differences, so the source is read once (neighbours from L1/L2) and the DIM
// components of a voxel are written together.  The arithmetic is the
// reference's own: double products (exact: a weight of +-0.5), a double sum
// in tap order, then the DstT cast (truncation for integral DstT).
#include <type_traits>

#include "dtype.cuh"

namespace ndlgpu {
namespace {

template <int DIM>
__global__ void __launch_bounds__(256) k_gradient(const GradParams p)
{
    int c[3];
    c[0] = blockIdx.x * blockDim.x + threadIdx.x;
    c[1] = blockIdx.y;
    c[2] = blockIdx.z;
    if (c[0] >= p.ext[0]) return;
    int64_t sb = 0, db = 0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        sb += (int64_t)c[d] * p.sstr[d];
        db += (int64_t)c[d] * p.dstr[d + 1];
    }
#pragma unroll
    for (int a = 0; a < DIM; a++) {
        const int n = p.ext[a];
        const int lo = c[a] > 0 ? c[a] - 1 : map_border32(p.border, n, c[a] - 1);
        const int hi = c[a] + 1 < n ? c[a] + 1 : map_border32(p.border, n, c[a] + 1);
        const double v0 = load_as<double>(p.src, p.sdt, sb + (int64_t)(lo - c[a]) * p.sstr[a]);
        const double v1 = load_as<double>(p.src, p.sdt, sb + (int64_t)(hi - c[a]) * p.sstr[a]);
        double t = 0.0;
        t += v0 * -0.5;
        t += v1 * 0.5;
        store_from(p.dst, p.ddt, db + (int64_t)a * p.dstr[0], t, STORE_CAST);
    }
}

// Typed form of the same pass for the common storage pairs: plain loads
// through the read-only path and typed stores, the same double arithmetic.
template <class Ti, class To, int DIM>
__global__ void __launch_bounds__(256) k_gradient_t(const GradParams p)
{
    int c[3];
    c[0] = blockIdx.x * blockDim.x + threadIdx.x;
    c[1] = blockIdx.y;
    c[2] = blockIdx.z;
    if (c[0] >= p.ext[0]) return;
    const Ti* src = reinterpret_cast<const Ti*>(p.src);
    To* dst = reinterpret_cast<To*>(p.dst);
    int64_t sb = 0, db = 0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        sb += (int64_t)c[d] * p.sstr[d];
        db += (int64_t)c[d] * p.dstr[d + 1];
    }
#pragma unroll
    for (int a = 0; a < DIM; a++) {
        const int n = p.ext[a];
        const int lo = c[a] > 0 ? c[a] - 1 : map_border32(p.border, n, c[a] - 1);
        const int hi = c[a] + 1 < n ? c[a] + 1 : map_border32(p.border, n, c[a] + 1);
        const double v0 = (double)__ldg(src + sb + (int64_t)(lo - c[a]) * p.sstr[a]);
        const double v1 = (double)__ldg(src + sb + (int64_t)(hi - c[a]) * p.sstr[a]);
        double t = 0.0;
        t += v0 * -0.5;
        t += v1 * 0.5;
        if constexpr (std::is_same_v<To, float>) dst[db + (int64_t)a * p.dstr[0]] = __double2float_rn(t);
        else if constexpr (std::is_same_v<To, double>) dst[db + (int64_t)a * p.dstr[0]] = t;
        else store_from(p.dst, p.ddt, db + (int64_t)a * p.dstr[0], t, STORE_CAST);
    }
}

// f32 -> f32 with a contiguous source (x stride 1, rows 16-byte aligned) and
// the default destination layout (components innermost): 4 voxels of a row
// per thread from float4 loads of the row and its y/z neighbours, written as
// DIM float4 (the 4 x DIM components are contiguous).  nx % 4 == 0.
template <int DIM>
__global__ void __launch_bounds__(256) k_gradient_v4(const GradParams p)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;      // quad of the row
    const int x = 4 * q;
    const int y = blockIdx.y, z = blockIdx.z;
    if (x >= p.ext[0]) return;
    const float* src = reinterpret_cast<const float*>(p.src);
    float* dst = reinterpret_cast<float*>(p.dst);
    const int64_t row = (DIM > 1 ? (int64_t)y * p.sstr[1] : 0) + (DIM > 2 ? (int64_t)z * p.sstr[2] : 0);
    auto ld4 = [&](int64_t off) { return __ldg(reinterpret_cast<const float4*>(src + off)); };
    auto diff = [](float a, float b) {    // (b - a) / 2 as the reference sums it: double, then the cast
        double t = 0.0;
        t += (double)a * -0.5;
        t += (double)b * 0.5;
        return __double2float_rn(t);
    };
    const int nx = p.ext[0];
    const float4 m = ld4(row + x);
    const float xl = __ldg(src + row + (x > 0 ? x - 1 : map_border32(p.border, nx, -1)));
    const float xr = __ldg(src + row + (x + 4 < nx ? x + 4 : map_border32(p.border, nx, x + 4)));
    float g[3][4];
    g[0][0] = diff(xl, m.y);
    g[0][1] = diff(m.x, m.z);
    g[0][2] = diff(m.y, m.w);
    g[0][3] = diff(m.z, xr);
#pragma unroll
    for (int a = 1; a < DIM; a++) {
        const int c = a == 1 ? y : z, n = p.ext[a];
        const int lo = c > 0 ? c - 1 : map_border32(p.border, n, c - 1);
        const int hi = c + 1 < n ? c + 1 : map_border32(p.border, n, c + 1);
        const float4 u = ld4(row + (int64_t)(lo - c) * p.sstr[a] + x);
        const float4 v = ld4(row + (int64_t)(hi - c) * p.sstr[a] + x);
        g[a][0] = diff(u.x, v.x);
        g[a][1] = diff(u.y, v.y);
        g[a][2] = diff(u.z, v.z);
        g[a][3] = diff(u.w, v.w);
    }
    float o[4 * DIM];
#pragma unroll
    for (int e = 0; e < 4; e++)
#pragma unroll
        for (int a = 0; a < DIM; a++) o[DIM * e + a] = g[a][e];
    float* out = dst + (DIM > 1 ? (int64_t)y * p.dstr[2] : 0) + (DIM > 2 ? (int64_t)z * p.dstr[3] : 0) +
                 (int64_t)x * DIM;
#pragma unroll
    for (int v = 0; v < DIM; v++)
        *reinterpret_cast<float4*>(out + 4 * v) = make_float4(o[4 * v], o[4 * v + 1], o[4 * v + 2], o[4 * v + 3]);
}

template <class Ti, class To>
void launch_typed(const GradParams& p, dim3 grid, cudaStream_t s)
{
    switch (p.rank) {
    case 1: k_gradient_t<Ti, To, 1><<<grid, 256, 0, s>>>(p); break;
    case 2: k_gradient_t<Ti, To, 2><<<grid, 256, 0, s>>>(p); break;
    default: k_gradient_t<Ti, To, 3><<<grid, 256, 0, s>>>(p); break;
    }
}

}  // namespace

bool gradient_supported(const GradParams& p)
{
    if (p.rank < 1 || p.rank > 3) return false;
    for (int d = 1; d < p.rank; d++)
        if (p.ext[d] > 65535) return false;
    return true;
}

cudaError_t launch_gradient(const GradParams& p, cudaStream_t s)
{
    const dim3 grid((unsigned)((p.ext[0] + 255) / 256), p.rank > 1 ? (unsigned)p.ext[1] : 1u,
                    p.rank > 2 ? (unsigned)p.ext[2] : 1u);
    bool v4 = p.sdt == NDLGPU_F32 && p.ddt == NDLGPU_F32 && p.sstr[0] == 1 && p.ext[0] % 4 == 0 &&
              p.dstr[0] == 1 && p.dstr[1] == p.rank && (reinterpret_cast<uintptr_t>(p.src) & 15) == 0 &&
              (reinterpret_cast<uintptr_t>(p.dst) & 15) == 0;
    for (int d = 1; d < p.rank; d++) v4 = v4 && (p.sstr[d] & 3) == 0 && (p.dstr[d + 1] & 3) == 0;
    if (v4) {
        const dim3 g4((unsigned)((p.ext[0] / 4 + 255) / 256), grid.y, grid.z);
        switch (p.rank) {
        case 1: k_gradient_v4<1><<<g4, 256, 0, s>>>(p); break;
        case 2: k_gradient_v4<2><<<g4, 256, 0, s>>>(p); break;
        default: k_gradient_v4<3><<<g4, 256, 0, s>>>(p); break;
        }
    } else if (p.sdt == NDLGPU_F32 && p.ddt == NDLGPU_F32) launch_typed<float, float>(p, grid, s);
    else if (p.sdt == NDLGPU_F64 && p.ddt == NDLGPU_F64) launch_typed<double, double>(p, grid, s);
    else if (p.sdt == NDLGPU_U8 && p.ddt == NDLGPU_F32) launch_typed<uint8_t, float>(p, grid, s);
    else if (p.sdt == NDLGPU_U8) launch_typed<uint8_t, int16_t>(p, grid, s);     // integral DstT: store_from
    else {
        switch (p.rank) {
        case 1: k_gradient<1><<<grid, 256, 0, s>>>(p); break;
        case 2: k_gradient<2><<<grid, 256, 0, s>>>(p); break;
        default: k_gradient<3><<<grid, 256, 0, s>>>(p); break;
        }
    }
    count_launch();
    return cudaGetLastError();
}

}  // namespace ndlgpu
