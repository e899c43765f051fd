// fused.cu -- fused separable forward: up to three 1-D passes in one kernel,
// so the volume crosses HBM once in and once out (the reference instead runs
// DIM full passes through two double buffers, processing/convolution.h:151-169).
//
// Geometry (host canonicalises every view to this): X = the axis with the
// smallest source stride, Y and Z = the other pass axes, batch = the rest
// merged into one affine axis.  A CTA owns a TX x TY column tile of one batch
// item and streams a chunk of Z planes (2.5-D blocking):
//   1. plane zi (border-mapped along Z) + X/Y halos -> shared memory, loaded
//      through registers one plane ahead of the compute;
//   2. X pass along shared-memory rows (register sliding window);
//   3. Y pass down shared-memory columns into 8 outputs per thread;
//   4. Z pass from a KZ-deep per-thread register queue of Y-pass results.
// Border maps (Clamp/Wrap/Reflect, mathHelpers.h:23-25) are applied to the
// load coordinates only, so the pass arithmetic never branches on the border.
//
// Arithmetic: Acc::F32 (fmaf, float storage types) or Acc::I32 (dyadic
// integer numerators, exact; result = acc / 2^shift rounded per store mode).
#include "dtype.cuh"

namespace ndlgpu {

namespace {

constexpr int TX = 64;   // tile columns (X)
constexpr int TY = 32;   // tile rows (Y)
constexpr int NT = 256;  // threads: 16 column groups of 4 x 16 row pairs

template <class A> struct V4;
template <> struct V4<float> { using T = float4; };
template <> struct V4<int32_t> { using T = int4; };

template <class A> __device__ __forceinline__ A mac(A acc, A x, A w);
template <> __device__ __forceinline__ float mac<float>(float acc, float x, float w) { return fmaf(x, w, acc); }
template <> __device__ __forceinline__ int32_t mac<int32_t>(int32_t acc, int32_t x, int32_t w) { return acc + x * w; }

template <class A> __device__ __forceinline__ A wx(const FusedParams& p, int k);
template <> __device__ __forceinline__ float wx<float>(const FusedParams& p, int k) { return p.wxf[k]; }
template <> __device__ __forceinline__ int32_t wx<int32_t>(const FusedParams& p, int k) { return p.wxi[k]; }
template <class A> __device__ __forceinline__ A wy(const FusedParams& p, int k);
template <> __device__ __forceinline__ float wy<float>(const FusedParams& p, int k) { return p.wyf[k]; }
template <> __device__ __forceinline__ int32_t wy<int32_t>(const FusedParams& p, int k) { return p.wyi[k]; }
template <class A> __device__ __forceinline__ A wz(const FusedParams& p, int k);
template <> __device__ __forceinline__ float wz<float>(const FusedParams& p, int k) { return p.wzf[k]; }
template <> __device__ __forceinline__ int32_t wz<int32_t>(const FusedParams& p, int k) { return p.wzi[k]; }

template <class T, class A> __device__ __forceinline__ A to_acc(T v);
template <> __device__ __forceinline__ float to_acc<float, float>(float v) { return v; }
template <> __device__ __forceinline__ float to_acc<__nv_bfloat16, float>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <> __device__ __forceinline__ float to_acc<__half, float>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float to_acc<uint8_t, float>(uint8_t v) { return (float)v; }
template <> __device__ __forceinline__ int32_t to_acc<uint8_t, int32_t>(uint8_t v) { return v; }
template <> __device__ __forceinline__ int32_t to_acc<int8_t, int32_t>(int8_t v) { return v; }
template <> __device__ __forceinline__ int32_t to_acc<uint16_t, int32_t>(uint16_t v) { return v; }
template <> __device__ __forceinline__ int32_t to_acc<int16_t, int32_t>(int16_t v) { return v; }

// Final conversion of one output to the destination type.
template <class T> __device__ __forceinline__ T from_f32(float v);
template <> __device__ __forceinline__ float from_f32<float>(float v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 from_f32<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ __half from_f32<__half>(float v) { return __float2half_rn(v); }

template <class T>
__device__ __forceinline__ T out_cast(float v, const FusedParams&) { return from_f32<T>(v); }
template <class T>
__device__ __forceinline__ T out_cast(int32_t v, const FusedParams& p)
{
    // dyadic integer sum -> DstT, exactly as the double reference would
    // round (ROUND) or truncate (CAST) the same value
    return (T)(long long)int_scaled(v, p.shift, p.store_mode);
}

template <class Tin, class Tout, class A, int KX, int KY, int KZ, bool TS>
__global__ void __launch_bounds__(NT, 1) k_fused(const __grid_constant__ FusedParams p)
{
    constexpr int ROWS = TY + KY - 1;
    constexpr int COLS = TX + KX - 1;
    constexpr int NV = (KX + 3 + 3) / 4;          // 4-wide loads per X window
    constexpr int PITCH = ((60 + 4 * NV > COLS ? 60 + 4 * NV : COLS) + 3) / 4 * 4 + 4;
    constexpr int NLD = (ROWS * COLS + NT - 1) / NT;
    using VA = typename V4<A>::T;

    __shared__ __align__(16) A s_in[ROWS][PITCH];
    __shared__ __align__(16) A s_x[ROWS][TX];
    // output plane staged x-major (destination contiguous along Y)
    __shared__ __align__(16) Tout s_o[TS ? TX : 1][TS ? TY + 4 : 1];

    const int tid = threadIdx.x;
    const int ntx = (p.nx + TX - 1) / TX;
    const int nty = (p.ny + TY - 1) / TY;
    const int tile = blockIdx.x % (ntx * nty);
    const int bat = blockIdx.x / (ntx * nty);
    const int x0 = (tile % ntx) * TX;
    const int y0 = (tile / ntx) * TY;
    const int zs = blockIdx.y * p.zchunk;
    const int ze = min(p.nz, zs + p.zchunk);
    if (zs >= ze) return;

    const Tin* src = reinterpret_cast<const Tin*>(p.src) + (int64_t)bat * p.sb;
    Tout* dst = reinterpret_cast<Tout*>(p.dst) + (int64_t)bat * p.db;

    const int cx = KX / 2, cy = KY / 2, cz = KZ / 2;
    const int hz = KZ - 1 - cz;
    const bool inner = (x0 - cx >= 0) && (x0 - cx + COLS <= p.nx) &&
                       (y0 - cy >= 0) && (y0 - cy + ROWS <= p.ny);

    // Per-thread load slots: element i = tid + j*NT of the ROWS x COLS tile.
    int32_t loff[NLD];
#pragma unroll
    for (int j = 0; j < NLD; j++) {
        const int i = tid + j * NT;
        const int r = i / COLS;
        const int c = i - r * COLS;
        int y = y0 - cy + r, x = x0 - cx + c;
        if (!inner) {
            // columns/rows past the last needed halo (partial edge tiles)
            // feed no output: any in-range address will do
            y = (y >= p.ny + KY - 1 - cy) ? p.ny - 1 : map_border32(p.border, p.ny, y);
            x = (x >= p.nx + KX - 1 - cx) ? p.nx - 1 : map_border32(p.border, p.nx, x);
        }
        loff[j] = (i < ROWS * COLS) ? (int32_t)(y * p.sy + x * p.sx) : 0;
    }

    A stage[NLD];
    // copies of the parameters the plane loads read (a lambda reading the
    // __grid_constant__ parameters through a reference would make generic loads)
    const int l_border = p.border, l_nz = p.nz;
    const int64_t l_sz = p.sz;
    auto fetch = [&](int zi) {
        const int zm = map_border32(l_border, l_nz, zi);
        const Tin* pl = src + (int64_t)zm * l_sz;
#pragma unroll
        for (int j = 0; j < NLD; j++)
            if (tid + j * NT < ROWS * COLS) stage[j] = to_acc<Tin, A>(pl[loff[j]]);
    };

    const int gx = tid & 15;   // column group: x = 4*gx .. 4*gx+3
    const int gy = tid >> 4;   // row pair: y = 2*gy, 2*gy+1

    A q[KZ][8];
#pragma unroll
    for (int k = 0; k < KZ; k++)
#pragma unroll
        for (int e = 0; e < 8; e++) q[k][e] = A(0);

    const int zin0 = zs - cz;
    const int zin1 = ze - 1 + hz;
    fetch(zin0);
    int filled = 0;
    for (int zi = zin0; zi <= zin1; zi++) {
        // staged plane -> shared memory
#pragma unroll
        for (int j = 0; j < NLD; j++) {
            const int i = tid + j * NT;
            if (i < ROWS * COLS) {
                const int r = i / COLS;
                s_in[r][i - r * COLS] = stage[j];
            }
        }
        __syncthreads();
        if (zi < zin1) fetch(zi + 1);   // in flight during this plane's compute

        // X pass: rows 0..ROWS-1, 4 outputs per unit
        for (int u = tid; u < ROWS * 16; u += NT) {
            const int r = u >> 4, g = u & 15;
            A acc[4] = {A(0), A(0), A(0), A(0)};
#pragma unroll
            for (int v = 0; v < NV; v++) {
                const VA w4 = *reinterpret_cast<const VA*>(&s_in[r][4 * g + 4 * v]);
                const A win[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int j = 4 * v + e;
#pragma unroll
                    for (int m = 0; m < 4; m++) {
                        const int k = j - m;
                        if (k >= 0 && k < KX) acc[m] = mac<A>(acc[m], win[e], wx<A>(p, k));
                    }
                }
            }
            VA o;
            o.x = acc[0]; o.y = acc[1]; o.z = acc[2]; o.w = acc[3];
            *reinterpret_cast<VA*>(&s_x[r][4 * g]) = o;
        }
        __syncthreads();

        // Y pass: rows 2gy, 2gy+1 of the tile, columns 4gx..4gx+3
        A yv[8];
#pragma unroll
        for (int e = 0; e < 8; e++) yv[e] = A(0);
#pragma unroll
        for (int j = 0; j < KY + 1; j++) {
            const VA v = *reinterpret_cast<const VA*>(&s_x[2 * gy + j][4 * gx]);
            const A c4[4] = {v.x, v.y, v.z, v.w};
            if (j < KY) {
#pragma unroll
                for (int m = 0; m < 4; m++) yv[m] = mac<A>(yv[m], c4[m], wy<A>(p, j));
            }
            if (j >= 1) {
#pragma unroll
                for (int m = 0; m < 4; m++) yv[4 + m] = mac<A>(yv[4 + m], c4[m], wy<A>(p, j - 1));
            }
        }

        // Z queue
#pragma unroll
        for (int k = 0; k + 1 < KZ; k++)
#pragma unroll
            for (int e = 0; e < 8; e++) q[k][e] = q[k + 1][e];
#pragma unroll
        for (int e = 0; e < 8; e++) q[KZ - 1][e] = yv[e];
        filled++;
        if (filled >= KZ) {
            const int zo = zi - hz;
            A out[8];
#pragma unroll
            for (int e = 0; e < 8; e++) {
                A a = A(0);
#pragma unroll
                for (int k = 0; k < KZ; k++) a = mac<A>(a, q[k][e], wz<A>(p, k));
                out[e] = a;
            }
            if constexpr (TS) {
#pragma unroll
                for (int h = 0; h < 2; h++)
#pragma unroll
                    for (int m = 0; m < 4; m++) s_o[4 * gx + m][2 * gy + h] = out_cast<Tout>(out[4 * h + m], p);
                __syncthreads();
                // consecutive threads walk Y: each warp writes one contiguous run
                Tout* pl = dst + (int64_t)zo * p.dz;
                for (int t = tid; t < TX * TY; t += NT) {
                    const int xl = t / TY, yl = t - (t / TY) * TY;
                    if (x0 + xl < p.nx && y0 + yl < p.ny)
                        pl[(int64_t)(x0 + xl) * p.dx + (int64_t)(y0 + yl) * p.dy] = s_o[xl][yl];
                }
            } else {
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int y = y0 + 2 * gy + h;
                    if (y >= p.ny) continue;
                    const int xb = x0 + 4 * gx;
                    Tout* row = dst + (int64_t)zo * p.dz + (int64_t)y * p.dy;
#pragma unroll
                    for (int m = 0; m < 4; m++)
                        if (xb + m < p.nx) row[(int64_t)(xb + m) * p.dx] = out_cast<Tout>(out[4 * h + m], p);
                }
            }
        }
    }
}

using LaunchFn = cudaError_t (*)(const FusedParams&, cudaStream_t);

template <class Tin, class Tout, class A, int KX, int KY, int KZ>
cudaError_t launch_one(const FusedParams& p, cudaStream_t s)
{
    const int ntx = (p.nx + TX - 1) / TX;
    const int nty = (p.ny + TY - 1) / TY;
    const long long gx = (long long)ntx * nty * p.nbatch;
    const int gz = (p.nz + p.zchunk - 1) / p.zchunk;
    if (gx > 0x7fffffffLL || gz > 65535) return cudaErrorInvalidConfiguration;
    if (p.tstore) k_fused<Tin, Tout, A, KX, KY, KZ, true><<<dim3((unsigned)gx, (unsigned)gz), NT, 0, s>>>(p);
    else k_fused<Tin, Tout, A, KX, KY, KZ, false><<<dim3((unsigned)gx, (unsigned)gz), NT, 0, s>>>(p);
    count_launch();
    return cudaGetLastError();
}

struct Variant {
    Acc acc;
    int sdt, ddt, kx, ky, kz;
    LaunchFn fn;
};

// Compiled variants (tap counts per axis; 1 = no pass along that axis).
const Variant kVariants[] = {
    // 3-D FP32, 9 taps per axis (random-kernel forward)
    {Acc::F32, NDLGPU_F32, NDLGPU_F32, 9, 9, 9, &launch_one<float, float, float, 9, 9, 9>},
    // 2-D FP32 Gaussian sigma = 2 (13 taps)
    {Acc::F32, NDLGPU_F32, NDLGPU_F32, 13, 13, 1, &launch_one<float, float, float, 13, 13, 1>},
    // 3-D uint8 binomial [1,4,6,4,1]/16 (exact integer path)
    {Acc::I32, NDLGPU_U8, NDLGPU_U8, 5, 5, 5, &launch_one<uint8_t, uint8_t, int32_t, 5, 5, 5>},
    // 4-D video sigma = (2.5, 2.5, -, 1.5): 17 x 17 x 11 taps, bf16 / f16 / f32 storage
    {Acc::F32, NDLGPU_BF16, NDLGPU_BF16, 17, 17, 11, &launch_one<__nv_bfloat16, __nv_bfloat16, float, 17, 17, 11>},
    {Acc::F32, NDLGPU_F16, NDLGPU_F16, 17, 17, 11, &launch_one<__half, __half, float, 17, 17, 11>},
    {Acc::F32, NDLGPU_F32, NDLGPU_F32, 17, 17, 11, &launch_one<float, float, float, 17, 17, 11>},
};

const Variant* find_variant(Acc acc, int sdt, int ddt, int kx, int ky, int kz)
{
    for (const Variant& v : kVariants)
        if (v.acc == acc && v.sdt == sdt && v.ddt == ddt && v.kx == kx && v.ky == ky && v.kz == kz) return &v;
    return nullptr;
}

}  // namespace

bool fused_supported(Acc acc, int sdt, int ddt, int kx, int ky, int kz)
{
    return find_variant(acc, sdt, ddt, kx, ky, kz) != nullptr;
}

cudaError_t launch_fused(Acc acc, const FusedParams& p, cudaStream_t s)
{
    const Variant* v = find_variant(acc, p.src_dtype, p.dst_dtype, p.kx, p.ky, p.kz);
    if (!v) return cudaErrorNotSupported;
    if (p.nx <= 0 || p.ny <= 0 || p.nz <= 0 || p.nbatch <= 0) return cudaSuccess;
    return v->fn(p, s);
}

}  // namespace ndlgpu
