// downsample.cu -- ndl::downsample (processing/convolution.h:241-305): every
// axis but the channel axis shrinks by `factor`, each output the average of
// its non-overlapping source block.
//
// A few consecutive outputs per thread.  The block is walked in the reference's odometer
// order (the lowest non-channel axis fastest, :283-292) with a double sum, so
// the result is the reference's bit for bit: the sum over the block divided
// by its element count (a short last block along an axis averages only the
// samples that exist, :273-277), then std::round for integral types (:295).
// An HBM-bound gather: every source element is read once and the outputs are
// 1/factor^(DIM-1) of it; consecutive threads take consecutive outputs along
// the fastest output axis, so a warp reads contiguous runs of the source.
#include <type_traits>

#include "dtype.cuh"

namespace ndlgpu {
namespace {

template <class T> __device__ __forceinline__ T ld_src(const char* b, int64_t i)
{
    return __ldg(reinterpret_cast<const T*>(b) + i);
}

// A run of kRun consecutive outputs per thread; the first output's 32-bit
// index is split with precomputed multiplicative inverses (outputs < 2^32,
// checked on the host) and the rest step the coordinates.  RANK > 0
// fixes the rank at compile time (per-axis arrays stay in registers); 0 takes
// it from p.rank.  The block is summed with its first non-channel axis
// innermost and the others as an odometer, the reference's order.  Integer
// types add exactly in 64-bit integers (every partial sum of the reference's
// double accumulation is an exact integer below 2^53, so the value is the
// same); floating types add in double in that order.  T = void reads any
// type through load_as.
constexpr int kRun = 4;     // consecutive outputs per thread (one index split per run)

template <class T, int RANK>
__global__ void __launch_bounds__(256) k_downsample(const __grid_constant__ DownParams p)
{
    constexpr int NR = RANK > 0 ? RANK : kMaxRank;
    const int rank = RANK > 0 ? RANK : p.rank;
    const uint32_t total = (uint32_t)p.total;
    const int a0 = p.channel == 0 ? 1 : 0;           // innermost block axis
    const int64_t s0 = p.sstr[a0];
    using Acc = typename std::conditional<std::is_integral<T>::value, long long, double>::type;
    const uint32_t step = gridDim.x * blockDim.x * kRun;
    for (uint32_t i0 = (blockIdx.x * blockDim.x + threadIdx.x) * kRun; i0 < total; i0 += step) {
        // output coordinates of the first output of this run
        int oc[NR];
        uint32_t rem = i0;
#pragma unroll
        for (int d = 0; d < NR; d++) {
            if (d >= rank) break;
            const uint32_t q = p.odiv[d].div(rem);
            oc[d] = (int)(rem - q * (uint32_t)p.oext[d]);
            rem = q;
        }
        const uint32_t iend = min(total, i0 + kRun);
        for (uint32_t i = i0; i < iend; i++) {
            int n[NR];
            int64_t doff = 0, off = 0;
            int count = 1, n0 = 1;
#pragma unroll
            for (int d = 0; d < NR; d++) {
                if (d >= rank) break;
                doff += (int64_t)oc[d] * p.dstr[d];
                if (d == p.channel) {
                    off += (int64_t)oc[d] * p.sstr[d];
                    n[d] = 1;
                } else {
                    const int lo = oc[d] * p.factor;
                    off += (int64_t)lo * p.sstr[d];
                    n[d] = min(lo + p.factor, p.ext[d]) - lo;
                    count *= n[d];
                }
                if (d == a0) n0 = n[d];
            }
            int c[NR];
#pragma unroll
            for (int d = 0; d < NR; d++) c[d] = 0;
            Acc sum = 0;
            for (;;) {
                for (int t = 0; t < n0; t++) {
                    if constexpr (std::is_void<T>::value) sum += load_as<double>(p.src, p.sdt, off + t * s0);
                    else sum += (Acc)ld_src<T>(p.src, off + t * s0);
                }
                bool carry = true;              // odometer over the other block axes
#pragma unroll
                for (int d = 0; d < NR; d++) {
                    if (d < rank && carry && d != p.channel && d != a0) {
                        if (++c[d] < n[d]) {
                            off += p.sstr[d];
                            carry = false;
                        } else {
                            off -= (int64_t)(n[d] - 1) * p.sstr[d];
                            c[d] = 0;
                        }
                    }
                }
                if (carry) break;
            }
            // sum / count; a power-of-two count divides exactly as a product
            // with its reciprocal (the same correctly rounded quotient)
            double avg;
            if ((count & (count - 1)) == 0)
                avg = (double)sum * __longlong_as_double((long long)(1023 - (__ffs(count) - 1)) << 52);
            else
                avg = (double)sum / (double)count;
            store_from(p.dst, p.ddt, doff, avg, STORE_ROUND);
            // next output: axis 0 fastest
            bool carry = true;
#pragma unroll
            for (int d = 0; d < NR; d++) {
                if (d < rank && carry) {
                    if (++oc[d] < p.oext[d]) carry = false;
                    else oc[d] = 0;
                }
            }
        }
    }
}

template <int RANK>
cudaError_t launch_typed(const DownParams& p, unsigned g, cudaStream_t s)
{
    switch (p.sdt) {
    case NDLGPU_U8: k_downsample<uint8_t, RANK><<<g, 256, 0, s>>>(p); break;
    case NDLGPU_U16: k_downsample<uint16_t, RANK><<<g, 256, 0, s>>>(p); break;
    case NDLGPU_I16: k_downsample<int16_t, RANK><<<g, 256, 0, s>>>(p); break;
    case NDLGPU_I32: k_downsample<int32_t, RANK><<<g, 256, 0, s>>>(p); break;
    case NDLGPU_F32: k_downsample<float, RANK><<<g, 256, 0, s>>>(p); break;
    case NDLGPU_F64: k_downsample<double, RANK><<<g, 256, 0, s>>>(p); break;
    default: k_downsample<void, RANK><<<g, 256, 0, s>>>(p); break;
    }
    count_launch();
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_downsample(const DownParams& p, cudaStream_t s)
{
    if (p.total == 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (p.total > 0xffffffffLL) return cudaErrorInvalidValue;
    const int64_t blocks = (p.total + 256 * kRun - 1) / (256 * kRun);
    const int64_t cap = (int64_t)sms * 8;
    const unsigned g = (unsigned)(blocks < cap ? blocks : cap);
    switch (p.rank) {
    case 2: return launch_typed<2>(p, g, s);
    case 3: return launch_typed<3>(p, g, s);
    case 4: return launch_typed<4>(p, g, s);
    default: return launch_typed<0>(p, g, s);
    }
}

}  // namespace ndlgpu
