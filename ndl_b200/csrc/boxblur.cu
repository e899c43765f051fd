// boxblur.cu -- ndl::box_blur (processing/summed_area_table.h:300-339): the
// (2r+1)^DIM box average through a summed-area table, computed as the
// reference computes it so that every result is the reference's bit for bit.
//
//   k_box_pad_scan0: one thread per padded axis-0 fiber.  The padded image
//     (extent + 2r per axis) is never stored: the thread reads the source at
//     the border-mapped position p - r (:319-322) and writes the running sum
//     along axis 0 straight into the double table.
//   k_box_scan: one thread per fiber of axis a >= 1, the running sum from
//     index 0 upward in place (:74-87); consecutive threads take consecutive
//     axis-0 positions, so every step is one coalesced row of the table.
//   k_box_query: one thread per output, rectangle_sum() over [c, c + 2r]
//     (:117-137): the 2^DIM corners in the reference's mask order, corners
//     off the table's low edge skipped, then sum / (2r+1)^DIM and DstT's
//     static_cast (truncation for integral types).
// Each running sum is sequential along its fiber, as the reference's is, so
// floating-point tables round exactly as the reference's do.
#include <type_traits>

#include "dtype.cuh"

namespace ndlgpu {
namespace {

__device__ __forceinline__ int box_map(int border, int n, int x)
{
    if (border == NDLGPU_WRAP) return x < 0 ? x + n : (x >= n ? x - n : x);
    if (border == NDLGPU_REFLECT) return x < 0 ? -x - 1 : (x >= n ? 2 * n - x - 1 : x);
    return x < 0 ? 0 : (x >= n ? n - 1 : x);
}

template <class T> __device__ __forceinline__ double box_ld(const BoxParams& p, int64_t i)
{
    if constexpr (std::is_void<T>::value) return load_as<double>(p.src, p.sdt, i);
    else return (double)__ldg(reinterpret_cast<const T*>(p.src) + i);
}

// T: the source type (void: any type through load_as).
template <class T>
__global__ void __launch_bounds__(256) k_box_pad_scan0(const __grid_constant__ BoxParams p)
{
    const int64_t nfib = p.npad / p.pext[0];
    for (int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; f < nfib; f += (int64_t)gridDim.x * blockDim.x) {
        int64_t rem = f, soff = 0, toff = 0;
        for (int a = 1; a < p.rank; a++) {
            const int64_t c = rem % p.pext[a];
            rem /= p.pext[a];
            soff += (int64_t)box_map(p.border, p.ext[a], (int)c - p.radius) * p.sstr[a];
            toff += c * p.pst[a];
        }
        double running = 0.0;
        const int n0 = (int)p.pext[0];
#pragma unroll 4
        for (int k = 0; k < n0; k++) {
            const int64_t i = soff + (int64_t)box_map(p.border, p.ext[0], k - p.radius) * p.sstr[0];
            running = running + box_ld<T>(p, i);
            p.table[toff + k] = running;
        }
    }
}

__global__ void __launch_bounds__(256) k_box_scan(const __grid_constant__ BoxParams p, int axis)
{
    const int64_t nfib = p.npad / p.pext[axis];
    const int64_t st = p.pst[axis];
    for (int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; f < nfib; f += (int64_t)gridDim.x * blockDim.x) {
        // fiber index -> padded coordinates of every axis but `axis`, axis 0 fastest
        int64_t rem = f, off = 0;
        for (int a = 0; a < p.rank; a++) {
            if (a == axis) continue;
            const int64_t c = rem % p.pext[a];
            rem /= p.pext[a];
            off += c * p.pst[a];
        }
        double running = 0.0;
        const int64_t n = p.pext[axis];
#pragma unroll 4
        for (int64_t k = 0; k < n; k++) {
            running = running + p.table[off + k * st];
            p.table[off + k * st] = running;
        }
    }
}

__global__ void __launch_bounds__(256) k_box_query(const __grid_constant__ BoxParams p)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.total; i += (int64_t)gridDim.x * blockDim.x) {
        int c[kMaxRank];
        int64_t rem = i, doff = 0;
        for (int a = 0; a < p.rank; a++) {
            c[a] = (int)(rem % p.ext[a]);
            rem /= p.ext[a];
            doff += (int64_t)c[a] * p.dstr[a];
        }
        double total = 0.0;
        const int corners = 1 << p.rank;
        for (int mask = 0; mask < corners; mask++) {
            int sign = 1;
            bool oob = false;
            int64_t off = 0;
            for (int a = 0; a < p.rank; a++) {
                const bool low = (mask >> a) & 1;
                const int q = low ? c[a] - 1 : c[a] + 2 * p.radius;
                if (low) sign = -sign;
                if (q < 0) {
                    oob = true;
                    break;
                }
                off += (int64_t)q * p.pst[a];
            }
            if (oob) continue;
            total = total + sign * p.table[off];
        }
        store_from(p.dst, p.ddt, doff, total / p.area, STORE_CAST);
    }
}

unsigned grid_of(int64_t n)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t blocks = (n + 255) / 256;
    const int64_t cap = (int64_t)sms * 16;
    return (unsigned)(blocks < cap ? (blocks > 0 ? blocks : 1) : cap);
}

}  // namespace

cudaError_t launch_box_blur(const BoxParams& p, cudaStream_t s)
{
    const unsigned g0 = grid_of(p.npad / p.pext[0]);
    switch (p.sdt) {
    case NDLGPU_U8: k_box_pad_scan0<uint8_t><<<g0, 256, 0, s>>>(p); break;
    case NDLGPU_F32: k_box_pad_scan0<float><<<g0, 256, 0, s>>>(p); break;
    case NDLGPU_F64: k_box_pad_scan0<double><<<g0, 256, 0, s>>>(p); break;
    default: k_box_pad_scan0<void><<<g0, 256, 0, s>>>(p); break;
    }
    count_launch();
    for (int a = 1; a < p.rank; a++) {
        k_box_scan<<<grid_of(p.npad / p.pext[a]), 256, 0, s>>>(p, a);
        count_launch();
    }
    k_box_query<<<grid_of(p.total), 256, 0, s>>>(p);
    count_launch();
    return cudaGetLastError();
}

}  // namespace ndlgpu
