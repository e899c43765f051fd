// downsample.cu -- ndl::downsample (processing/convolution.h:241-305): every
// axis but the channel axis shrinks by `factor`, each output the average of
// its non-overlapping source block.
//
// One thread per output.  The block is walked in the reference's odometer
// order (the lowest non-channel axis fastest, :283-292) with a double sum, so
// the result is the reference's bit for bit: the sum over the block divided
// by its element count (a short last block along an axis averages only the
// samples that exist, :273-277), then std::round for integral types (:295).
// An HBM-bound gather: every source element is read once and the outputs are
// 1/factor^(DIM-1) of it; consecutive threads take consecutive outputs along
// the fastest output axis, so a warp reads contiguous runs of the source.
#include "dtype.cuh"

namespace ndlgpu {
namespace {

__global__ void __launch_bounds__(256) k_downsample(const DownParams p)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.total; i += (int64_t)gridDim.x * blockDim.x) {
        int lo[kMaxRank], hi[kMaxRank], c[kMaxRank];
        int64_t rem = i, doff = 0, base = 0;
        int count = 1;
        for (int d = 0; d < p.rank; d++) {
            const int oc = (int)(rem % p.oext[d]);
            rem /= p.oext[d];
            doff += (int64_t)oc * p.dstr[d];
            if (d == p.channel) {
                lo[d] = oc;
                hi[d] = oc + 1;
            } else {
                lo[d] = oc * p.factor;
                hi[d] = min(lo[d] + p.factor, p.ext[d]);
                count *= hi[d] - lo[d];
            }
            c[d] = lo[d];
            base += (int64_t)lo[d] * p.sstr[d];
        }
        double sum = 0.0;
        int64_t off = base;
        for (int k = 0; k < count; k++) {
            sum += load_as<double>(p.src, p.sdt, off);
            for (int d = 0; d < p.rank; d++) {
                if (d == p.channel) continue;
                if (++c[d] < hi[d]) {
                    off += p.sstr[d];
                    break;
                }
                off -= (int64_t)(hi[d] - 1 - lo[d]) * p.sstr[d];
                c[d] = lo[d];
            }
        }
        store_from(p.dst, p.ddt, doff, sum / (double)count, STORE_ROUND);
    }
}

}  // namespace

cudaError_t launch_downsample(const DownParams& p, cudaStream_t s)
{
    if (p.total == 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t blocks = (p.total + 255) / 256;
    const int64_t cap = (int64_t)sms * 8;
    k_downsample<<<(unsigned)(blocks < cap ? blocks : cap), 256, 0, s>>>(p);
    count_launch();
    return cudaGetLastError();
}

}  // namespace ndlgpu
