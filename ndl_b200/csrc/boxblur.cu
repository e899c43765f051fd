// boxblur.cu -- ndl::box_blur (processing/summed_area_table.h:300-339): the
// (2r+1)^DIM box average through a summed-area table, computed as the
// reference computes it so that every result is the reference's bit for bit.
//
//   k_box_pad_scan0: 32 padded axis-0 fibers per warp.  The padded image
//     (extent + 2r per axis) is never stored: the source is read at the
//     border-mapped position p - r (:319-322), staged through a shared tile
//     so that loads and stores stay coalesced, and each lane writes its
//     fiber's running sum along axis 0 straight into the double table.
//   k_box_scan: one thread per fiber of axis a >= 1, the running sum from
//     index 0 upward in place (:74-87); consecutive threads take consecutive
//     axis-0 positions, so every step is one coalesced row of the table.
//   k_box_query: one thread per output, rectangle_sum() over [c, c + 2r]
//     (:117-137): the 2^DIM corners in the reference's mask order, corners
//     off the table's low edge skipped, then sum / (2r+1)^DIM and DstT's
//     static_cast (truncation for integral types).
// Each running sum is sequential along its fiber, as the reference's is, so
// floating-point tables round exactly as the reference's do.
#include <algorithm>
#include <type_traits>

#include "dtype.cuh"

namespace ndlgpu {
namespace {

constexpr int kBatch = 32;   // fiber elements loaded ahead of their running sums

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

// T: the source type (void: any type through load_as).  One warp per CTA
// and 32 fibers per warp: each 32-column chunk is read row by row with
// coalesced loads into a shared tile, every lane then runs its own fiber's
// sequential sum over the chunk, and the tile goes back to the table row by
// row, again coalesced.
template <class T>
__global__ void __launch_bounds__(32) k_box_pad_scan0(const __grid_constant__ BoxParams p)
{
    __shared__ double tile[32][33];
    __shared__ int64_t s_toff[32];       // table offsets of the warp's 32 fibers
    const int lane = threadIdx.x;
    const int64_t nfib = p.npad / p.pext[0];
    const int n0 = (int)p.pext[0];
    for (int64_t f0 = (int64_t)blockIdx.x * 32; f0 < nfib; f0 += (int64_t)gridDim.x * 32) {
        // this lane's fiber: source offset of its border-mapped row, table offset
        int64_t soff = 0, toff = 0;
        if (f0 + lane < nfib) {
            int64_t rem = f0 + lane;
            for (int a = 1; a < p.rank; a++) {
                const int64_t c = rem % p.pext[a];
                rem /= p.pext[a];
                soff += (int64_t)box_map(p.border, p.ext[a], (int)c - p.radius) * p.sstr[a];
                toff += c * p.pst[a];
            }
        }
        __syncwarp();
        s_toff[lane] = toff;
        __syncwarp();
        const int rows = nfib - f0 < 32 ? (int)(nfib - f0) : 32;
        using Raw = typename std::conditional<std::is_void<T>::value, double, T>::type;
        // chunk k0's raw values of rows r = 0..31 at column k0 + lane, loaded
        // one chunk ahead of the scan so the loads overlap it
        Raw v[32];
        auto load_chunk = [&](int k0) {
            const int k = k0 + lane;
            const bool kin = k < n0;
            const int64_t xoff = kin ? (int64_t)box_map(p.border, p.ext[0], k - p.radius) * p.sstr[0] : 0;
#pragma unroll
            for (int r = 0; r < 32; r++) {
                const int64_t so = __shfl_sync(0xffffffffu, soff, r);
                if (r < rows && kin) {
                    if constexpr (std::is_void<T>::value) v[r] = load_as<double>(p.src, p.sdt, so + xoff);
                    else v[r] = __ldg(reinterpret_cast<const T*>(p.src) + so + xoff);
                } else {
                    v[r] = Raw(0);
                }
            }
        };
        load_chunk(0);
        double running = 0.0;
        for (int k0 = 0; k0 < n0; k0 += 32) {
#pragma unroll
            for (int r = 0; r < 32; r++) tile[r][lane] = (double)v[r];
            __syncwarp();
            if (k0 + 32 < n0) load_chunk(k0 + 32);
            const int cnt = min(32, n0 - k0);
            if (cnt == 32) {
                // a full chunk: every shared read ahead of the sum chain
                double t[32];
#pragma unroll
                for (int j = 0; j < 32; j++) t[j] = tile[lane][j];
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    running = running + t[j];
                    tile[lane][j] = running;
                }
            } else {
                for (int j = 0; j < cnt; j++) {
                    running = running + tile[lane][j];
                    tile[lane][j] = running;
                }
            }
            __syncwarp();
            const int k = k0 + lane;
#pragma unroll 8
            for (int r = 0; r < 32; r++)
                if (r < rows && k < n0) p.table[s_toff[r] + k] = tile[r][lane];
            __syncwarp();
        }
    }
}

__device__ __forceinline__ void cp_async_el(void* smem, const void* gmem, int bytes)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    if (bytes == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}

constexpr int kRing = 4;   // chunks in flight per warp (row scan, 4- and 8-byte sources)

// The row scan for f32 and f64 sources: the same chunks as k_box_pad_scan0,
// but each chunk arrives by cp.async into a ring of kRing shared tiles, so
// several chunks' loads are in flight while the warp sums an earlier one.
template <class T>
__global__ void __launch_bounds__(32) k_box_pad_scan0_async(const __grid_constant__ BoxParams p)
{
    static_assert(sizeof(T) == 4 || sizeof(T) == 8, "cp.async element copies of 4 or 8 bytes");
    __shared__ T raw[kRing][32][33];
    __shared__ double tile[32][33];
    __shared__ int64_t s_soff[32], s_toff[32];
    const int lane = threadIdx.x;
    const int64_t nfib = p.npad / p.pext[0];
    const int n0 = (int)p.pext[0];
    const int nchunk = (n0 + 31) / 32;
    const T* src = reinterpret_cast<const T*>(p.src);
    for (int64_t f0 = (int64_t)blockIdx.x * 32; f0 < nfib; f0 += (int64_t)gridDim.x * 32) {
        int64_t soff = 0, toff = 0;
        if (f0 + lane < nfib) {
            int64_t rem = f0 + lane;
            for (int a = 1; a < p.rank; a++) {
                const int64_t c = rem % p.pext[a];
                rem /= p.pext[a];
                soff += (int64_t)box_map(p.border, p.ext[a], (int)c - p.radius) * p.sstr[a];
                toff += c * p.pst[a];
            }
        }
        __syncwarp();
        s_soff[lane] = soff;
        s_toff[lane] = toff;
        __syncwarp();
        const int rows = nfib - f0 < 32 ? (int)(nfib - f0) : 32;
        auto issue = [&](int c) {
            if (c < nchunk) {
                T (*b)[33] = raw[c % kRing];
                const int k = c * 32 + lane;
                const bool kin = k < n0;
                const int64_t xoff = kin ? (int64_t)box_map(p.border, p.ext[0], k - p.radius) * p.sstr[0] : 0;
#pragma unroll 8
                for (int r = 0; r < 32; r++) {
                    if (r < rows && kin) cp_async_el(&b[r][lane], src + s_soff[r] + xoff, (int)sizeof(T));
                    else b[r][lane] = T(0);
                }
            }
            asm volatile("cp.async.commit_group;\n" ::: "memory");
        };
#pragma unroll
        for (int c = 0; c < kRing - 1; c++) issue(c);
        double running = 0.0;
        for (int c = 0; c < nchunk; c++) {
            asm volatile("cp.async.wait_group %0;\n" ::"n"(kRing - 2) : "memory");
            __syncwarp();                  // chunk c visible to every lane; chunk c-1's tile reads done
            issue(c + kRing - 1);
            const T (*b)[33] = raw[c % kRing];
            const int k0 = c * 32;
            const int cnt = min(32, n0 - k0);
            if (cnt == 32) {
                double t[32];
#pragma unroll
                for (int j = 0; j < 32; j++) t[j] = (double)b[lane][j];
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    running = running + t[j];
                    tile[lane][j] = running;
                }
            } else {
                for (int j = 0; j < cnt; j++) {
                    running = running + (double)b[lane][j];
                    tile[lane][j] = running;
                }
            }
            __syncwarp();
            const int k = k0 + lane;
#pragma unroll 8
            for (int r = 0; r < 32; r++)
                if (r < rows && k < n0) p.table[s_toff[r] + k] = tile[r][lane];
            __syncwarp();
        }
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncwarp();
    }
}

__global__ void __launch_bounds__(32) k_box_scan(const __grid_constant__ BoxParams p, int axis)
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
        double* t = p.table + off;
        int64_t k = 0;
        for (; k + kBatch <= n; k += kBatch) {
            double v[kBatch];
#pragma unroll
            for (int j = 0; j < kBatch; j++) v[j] = t[(k + j) * st];
#pragma unroll
            for (int j = 0; j < kBatch; j++) {
                running = running + v[j];
                t[(k + j) * st] = running;
            }
        }
        for (; k < n; k++) {
            running = running + t[k * st];
            t[k * st] = running;
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

// Ranks 1-3 with the y and z extents within the grid limits: x from the
// thread index, y and z from the block indices (no index division), the
// corner loop unrolled.
template <int RANK>
__global__ void __launch_bounds__(256) k_box_query_r(const __grid_constant__ BoxParams p)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= p.ext[0]) return;
    int c[3] = {x, RANK > 1 ? (int)blockIdx.y : 0, RANK > 2 ? (int)blockIdx.z : 0};
    int64_t doff = 0;
#pragma unroll
    for (int a = 0; a < RANK; a++) doff += (int64_t)c[a] * p.dstr[a];
    double total = 0.0;
#pragma unroll
    for (int mask = 0; mask < (1 << RANK); mask++) {
        int sign = 1;
        bool oob = false;
        int64_t off = 0;
#pragma unroll
        for (int a = 0; a < RANK; a++) {
            const bool low = (mask >> a) & 1;
            const int q = low ? c[a] - 1 : c[a] + 2 * p.radius;
            if (low) sign = -sign;
            oob = oob || q < 0;
            off += (int64_t)q * p.pst[a];
        }
        if (!oob) total = total + sign * p.table[off];
    }
    store_from(p.dst, p.ddt, doff, total / p.area, STORE_CAST);
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
    // the scans: one warp per CTA, so that the few hundred warps of a 2-D
    // table spread over every SM instead of filling a handful
    const int64_t f0 = p.npad / p.pext[0];
    const unsigned g0 = (unsigned)std::min<int64_t>((f0 + 31) / 32, 1 << 20);
    switch (p.sdt) {
    case NDLGPU_U8: k_box_pad_scan0<uint8_t><<<g0, 32, 0, s>>>(p); break;
    case NDLGPU_F32: k_box_pad_scan0_async<float><<<g0, 32, 0, s>>>(p); break;
    case NDLGPU_F64: k_box_pad_scan0_async<double><<<g0, 32, 0, s>>>(p); break;
    default: k_box_pad_scan0<void><<<g0, 32, 0, s>>>(p); break;
    }
    count_launch();
    for (int a = 1; a < p.rank; a++) {
        const int64_t fa = p.npad / p.pext[a];
        k_box_scan<<<(unsigned)std::min<int64_t>((fa + 31) / 32, 1 << 20), 32, 0, s>>>(p, a);
        count_launch();
    }
    const bool fits = p.rank <= 3 && (p.rank < 2 || p.ext[1] <= 65535) && (p.rank < 3 || p.ext[2] <= 65535);
    if (fits) {
        const dim3 g((unsigned)((p.ext[0] + 255) / 256), p.rank > 1 ? (unsigned)p.ext[1] : 1u,
                     p.rank > 2 ? (unsigned)p.ext[2] : 1u);
        if (p.rank == 1) k_box_query_r<1><<<g, 256, 0, s>>>(p);
        else if (p.rank == 2) k_box_query_r<2><<<g, 256, 0, s>>>(p);
        else k_box_query_r<3><<<g, 256, 0, s>>>(p);
    } else {
        k_box_query<<<grid_of(p.total), 256, 0, s>>>(p);
    }
    count_launch();
    return cudaGetLastError();
}

}  // namespace ndlgpu
