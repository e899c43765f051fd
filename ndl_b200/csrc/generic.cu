// generic.cu -- general kernels: one 1-D pass, or a full N-D kernel, over any
// strided view and any element type.  These carry the exact arithmetic modes
// (the reference's double sequence, integer dyadic sums) and every shape the
// fused kernels do not take; one thread computes one output element.
//
// Arithmetic follows processing/convolution.h:64-69: for each output
// coordinate, total = 0, then for each included tap in kernel order
// total += double(src[mapped]) * double(w), then the DstT cast.  The border
// map is applied per axis as image/detail.h:178-194 does.
#include "dtype.cuh"

namespace ndlgpu {

namespace {

__device__ int32_t g_guard_generic;

template <class A>
struct Mac;

// The reference's sequence: product rounded, then sum rounded (no fused
// multiply-add: x86-64 g++ without -march contracts nothing).
template <>
struct Mac<double> {
    __device__ static __forceinline__ double step(double acc, double x, const GenericPassParams& p, int t)
    {
        return __dadd_rn(acc, __dmul_rn(x, p.wd[t]));
    }
};
template <>
struct Mac<float> {
    __device__ static __forceinline__ float step(float acc, float x, const GenericPassParams& p, int t)
    {
        return fmaf(x, p.wf[t], acc);
    }
};
template <>
struct Mac<int32_t> {
    __device__ static __forceinline__ int32_t step(int32_t acc, int32_t x, const GenericPassParams& p, int t)
    {
        return acc + x * p.wi[t];
    }
};

template <class A>
__device__ __forceinline__ void store_acc(const GenericPassParams& p, int64_t i, A acc);
template <>
__device__ __forceinline__ void store_acc<double>(const GenericPassParams& p, int64_t i, double acc)
{
    store_from(p.dst, p.dst_dtype, i, acc, p.store_mode);
}
template <>
__device__ __forceinline__ void store_acc<float>(const GenericPassParams& p, int64_t i, float acc)
{
    store_from(p.dst, p.dst_dtype, i, acc, p.store_mode);
}
template <>
__device__ __forceinline__ void store_acc<int32_t>(const GenericPassParams& p, int64_t i, int32_t acc)
{
    store_from(p.dst, p.dst_dtype, i, acc, p.store_mode, p.shift);
}

template <class A>
__global__ void __launch_bounds__(256) k_generic_pass(const __grid_constant__ GenericPassParams p)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < p.total; idx += stride) {
        uint32_t rem = idx;
        int64_t so = 0, dof = 0, ca = 0;
#pragma unroll
        for (int i = 0; i < kMaxRank; i++) {
            if (i < p.rank) {
                const uint32_t q = p.div[i].div(rem);
                const int64_t c = (int64_t)(rem - q * p.div[i].d);
                rem = q;
                if (i == p.axis) ca = c;
                else so += c * p.ss[i];
                dof += c * p.ds[i];
            }
        }
        const int64_t M = p.n[p.axis];
        const int64_t sa = p.ss[p.axis];
        A acc = A(0);
        for (int t = 0; t < p.ntap; t++) {
            const int64_t x = map_border(p.border, M, ca + p.off[t]);
            acc = Mac<A>::step(acc, load_as<A>(p.src, p.src_dtype, so + x * sa), p, t);
        }
        store_acc<A>(p, dof, acc);
    }
}

template <class A>
__device__ __forceinline__ A nd_step(A acc, A x, double w);
template <>
__device__ __forceinline__ double nd_step<double>(double acc, double x, double w)
{
    return __dadd_rn(acc, __dmul_rn(x, w));
}
template <>
__device__ __forceinline__ float nd_step<float>(float acc, float x, double w)
{
    return fmaf(x, (float)w, acc);
}

// General N-D kernel (convolve() with a non-separable kernel): every axis of
// every tap is border-mapped (image/detail.h:182-192), taps in kernel
// coordinates() order (image/detail.h:171).
template <class A>
__global__ void __launch_bounds__(256) k_generic_nd(const __grid_constant__ GenericNdParams p)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < p.total; idx += stride) {
        uint32_t rem = idx;
        int64_t c[kMaxRank];
        int64_t dof = 0;
#pragma unroll
        for (int i = 0; i < kMaxRank; i++) {
            c[i] = 0;
            if (i < p.rank) {
                const uint32_t q = p.div[i].div(rem);
                c[i] = (int64_t)(rem - q * p.div[i].d);
                rem = q;
                dof += c[i] * p.ds[i];
            }
        }
        A acc = A(0);
        for (int t = 0; t < p.ntap; t++) {
            int64_t so = 0;
            const int32_t* o = p.tap_off + (int64_t)t * p.rank;
#pragma unroll
            for (int i = 0; i < kMaxRank; i++)
                if (i < p.rank) so += map_border(p.border, p.n[i], c[i] + o[i]) * p.ss[i];
            acc = nd_step<A>(acc, load_as<A>(p.src, p.src_dtype, so), p.tap_w[t]);
        }
        store_from(p.dst, p.dst_dtype, dof, acc, p.store_mode);
    }
}

unsigned grid_for(uint32_t total)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = (uint64_t(total) + 255) / 256;
    const uint64_t cap = uint64_t(sms) * 8;
    return (unsigned)(want < cap ? (want ? want : 1) : cap);
}

}  // namespace

cudaError_t launch_generic_pass(Acc acc, const GenericPassParams& p, cudaStream_t s)
{
    if (p.total == 0) return cudaSuccess;
    const unsigned g = grid_for(p.total);
    switch (acc) {
    case Acc::F64: k_generic_pass<double><<<g, 256, 0, s>>>(p); break;
    case Acc::F32: k_generic_pass<float><<<g, 256, 0, s>>>(p); break;
    default: k_generic_pass<int32_t><<<g, 256, 0, s>>>(p); break;
    }
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_generic_nd(Acc acc, const GenericNdParams& p, cudaStream_t s)
{
    if (p.total == 0) return cudaSuccess;
    const unsigned g = grid_for(p.total);
    if (acc == Acc::F32) k_generic_nd<float><<<g, 256, 0, s>>>(p);
    else k_generic_nd<double><<<g, 256, 0, s>>>(p);
    count_launch();
    return cudaGetLastError();
}

cudaError_t read_guard_generic(int32_t* v)
{
    int32_t zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(v, g_guard_generic, sizeof(int32_t));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(g_guard_generic, &zero, sizeof(int32_t));
}

}  // namespace ndlgpu

namespace ndlgpu {
cudaError_t read_device_status(cudaStream_t, int32_t* code)
{
    int32_t a = 0, b = 0, c = 0, d = 0;
    cudaError_t e = read_guard_generic(&a);
    if (e == cudaSuccess) e = read_guard_fused(&b);
    if (e == cudaSuccess) e = read_guard_batch(&c);
    if (e == cudaSuccess) e = read_guard_fwd3(&d);
    *code = a | b | c | d;
    return e;
}
}  // namespace ndlgpu
