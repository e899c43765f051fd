// batch.cu -- the batched form: many instances of uneven extents, tap counts
// and border modes in one persistent launch (no reference counterpart).
//
// Every CTA of a persistent grid (SMs x resident CTAs) takes work items
// (instance, XY tile, Z chunk, batch index) from an atomic counter over a
// table the host sorted by decreasing cost, so the uneven items balance over
// the SMs.  An item runs the 2.5-D scheme of the fused kernels with the tap
// widths of its instance chosen at run time from the compiled widths
// {1,3,5,9,...,37} (zero-padded taps):
//   load  : plane (border-mapped, or zero outside the image for the adjoint
//           with Clamp/Reflect) with X/Y halos, cp.async, one plane ahead;
//   X pass: 4 outputs per unit over all halo rows;
//   Y pass: 2 outputs per thread into the newest slot of a shared-memory
//           ring of Y-pass planes;
//   Z pass: 2 outputs per thread from the ring.
// The adjoint (transposed chain) reads flipped taps; positions within the
// real tap radius of a border take effective weights from per-instance
// tables (the fold of the out-of-range taps, built on the host).
#include "dtype.cuh"

namespace ndlgpu {
namespace {

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

template <class T> __device__ __forceinline__ float to_f(T v);
template <> __device__ __forceinline__ float to_f<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <> __device__ __forceinline__ float to_f<__half>(__half v) { return __half2float(v); }
template <class T> __device__ __forceinline__ T from_f(float v);
template <> __device__ __forceinline__ float from_f<float>(float v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ __half from_f<__half>(float v) { return __float2half_rn(v); }

__device__ __forceinline__ void lds4(const float* p, float* v)
{
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void lds4(const __nv_bfloat16* p, float* v)
{
    const uint2 t = *reinterpret_cast<const uint2*>(p);
    v[0] = __uint_as_float(t.x << 16); v[1] = __uint_as_float(t.x & 0xffff0000u);
    v[2] = __uint_as_float(t.y << 16); v[3] = __uint_as_float(t.y & 0xffff0000u);
}
__device__ __forceinline__ void lds4(const __half* p, float* v)
{
    const uint2 t = *reinterpret_cast<const uint2*>(p);
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&t.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&t.y));
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

__device__ __forceinline__ int zone_row(int j, int n, int r)
{
    if (j < r) return j;
    if (j >= n - r) return r + (j - (n - r));
    return -1;
}

// X pass with a compiled width B (taps at offsets -B/2..B/2).
template <class T, int TX, int B>
__device__ __forceinline__ void xpass(const T* sb, float* s_x, const float* s_w, int rows, int pitch, int nt,
                                      const BatchDesc& d, const float* zones, int x0)
{
    constexpr int EPC = 16 / (int)sizeof(T);
    constexpr int CB = B / 2;
    constexpr int D = (EPC - CB % EPC) % EPC;
    constexpr int WOFF = D % 4;
    constexpr int WBASE = (D / 4) * 4;
    constexpr int NV = (WOFF + B + 3 + 3) / 4;
    constexpr int G = TX / 4;
    for (int u = threadIdx.x; u < rows * G; u += nt) {
        const int r = u / G, g = u - (u / G) * G;
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        const T* rowp = sb + r * pitch + 4 * g + WBASE;
#pragma unroll
        for (int v = 0; v < NV; v++) {
            float val[4];
            lds4(rowp + 4 * v, val);
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int pos = 4 * v + e - WOFF;
#pragma unroll
                for (int m = 0; m < 4; m++) {
                    const int k = pos - m;
                    if (k >= 0 && k < B) acc[m] = fmaf(val[e], s_w[k], acc[m]);
                }
            }
        }
        if (d.zone_x >= 0) {
            const int xg0 = x0 + 4 * g;
            if (xg0 < d.rx || xg0 + 3 >= d.nx - d.rx) {
#pragma unroll
                for (int m = 0; m < 4; m++) {
                    const int e = zone_row(xg0 + m, d.nx, d.rx);
                    if (e < 0) continue;
                    const float* zw = zones + d.zone_x + e * B;
                    float a = 0.f;
#pragma unroll
                    for (int v = 0; v < NV; v++) {
                        float val[4];
                        lds4(rowp + 4 * v, val);
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            const int k = 4 * v + q - WOFF - m;
                            if (k >= 0 && k < B) a = fmaf(val[q], __ldg(zw + k), a);
                        }
                    }
                    acc[m] = a;
                }
            }
        }
        *reinterpret_cast<float4*>(s_x + r * TX + 4 * g) = make_float4(acc[0], acc[1], acc[2], acc[3]);
    }
}

// Y pass with a compiled width B: outputs (2tx, 2tx+1) of row ty.
template <int TX, int B>
__device__ __forceinline__ void ypass(const float* s_x, const float* s_w, int ty, int tx2, const BatchDesc& d,
                                      const float* zones, int y0, float (&yv)[2])
{
    float a0 = 0.f, a1 = 0.f;
#pragma unroll
    for (int k = 0; k < B; k++) {
        const float2 v = *reinterpret_cast<const float2*>(s_x + (ty + k) * TX + 2 * tx2);
        const float w = s_w[k];
        a0 = fmaf(v.x, w, a0);
        a1 = fmaf(v.y, w, a1);
    }
    if (d.zone_y >= 0) {
        const int e = zone_row(y0 + ty, d.ny, d.ry);
        if (e >= 0) {
            const float* zw = zones + d.zone_y + e * B;
            a0 = a1 = 0.f;
#pragma unroll
            for (int k = 0; k < B; k++) {
                const float2 v = *reinterpret_cast<const float2*>(s_x + (ty + k) * TX + 2 * tx2);
                const float w = __ldg(zw + k);
                a0 = fmaf(v.x, w, a0);
                a1 = fmaf(v.y, w, a1);
            }
        }
    }
    yv[0] = a0;
    yv[1] = a1;
}

// Z pass with a compiled width B from the ring (plane p at slot p mod ring).
template <int TX, int TY, int B>
__device__ __forceinline__ void zpass(const float* s_ring, int ring, int newest, const float* s_w, int pos,
                                      const BatchDesc& d, const float* zones, int zo, float (&out)[2])
{
    float a0 = 0.f, a1 = 0.f;
    const int e = (d.zone_z >= 0) ? zone_row(zo, d.nz, d.rz) : -1;
    const float* zw = (e >= 0) ? zones + d.zone_z + e * B : nullptr;
#pragma unroll
    for (int k = 0; k < B; k++) {
        int sl = newest - (B - 1) + k;
        sl = sl < 0 ? sl + ring : sl;
        const float2 v = *reinterpret_cast<const float2*>(s_ring + (size_t)sl * (TX * TY) + pos);
        const float w = zw ? __ldg(zw + k) : s_w[k];
        a0 = fmaf(v.x, w, a0);
        a1 = fmaf(v.y, w, a1);
    }
    out[0] = a0;
    out[1] = a1;
}

#define NDLGPU_BUCKETS(M) M(1) M(3) M(5) M(9) M(13) M(17) M(21) M(25) M(29) M(33) M(37)

template <class T, int TX, int TY>
__global__ void __launch_bounds__(TX * TY / 2) k_batch(const BatchDesc* __restrict__ descs,
                                                      const int4* __restrict__ items, int nitems,
                                                      int* __restrict__ counter, const float* __restrict__ zones,
                                                      int rows_max, int ring)
{
    constexpr int NT = TX * TY / 2;
    constexpr int EPC = 16 / (int)sizeof(T);
    constexpr int PITCH = TX + 48;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const size_t stage_elems = (size_t)rows_max * PITCH;
    T* s_in = reinterpret_cast<T*>(smem_raw);
    const size_t x_off = ((2 * stage_elems * sizeof(T)) + 15) / 16 * 16;
    float* s_x = reinterpret_cast<float*>(smem_raw + x_off);
    const size_t ring_off = x_off + (size_t)rows_max * TX * 4;
    float* s_ring = reinterpret_cast<float*>(smem_raw + ring_off);
    const size_t w_off = ring_off + (size_t)ring * TX * TY * 4;
    float* s_w = reinterpret_cast<float*>(smem_raw + w_off);     // [3][40]
    int* s_item = reinterpret_cast<int*>(smem_raw + w_off + 3 * 40 * 4);

    const int tid = threadIdx.x;
    const int tx2 = tid % (TX / 2), ty = tid / (TX / 2);

    for (;;) {
        if (tid == 0) *s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int it = *s_item;
        if (it >= nitems) break;
        const int4 item = items[it];
        const BatchDesc& d = descs[item.x];
        for (int i = tid; i < 3 * 40; i += NT) {
            const int a = i / 40, k = i - a * 40;
            const float* src = a == 0 ? d.wx : (a == 1 ? d.wy : d.wz);
            const int B = a == 0 ? d.bx : (a == 1 ? d.by : d.bz);
            s_w[i] = k < B ? src[k] : 0.f;
        }
        const int x0 = (item.y % d.ntx) * TX;
        const int y0 = (item.y / d.ntx) * TY;
        const int zs = item.z * d.zchunk;
        const int ze = min(d.nz, zs + d.zchunk);
        const T* src = reinterpret_cast<const T*>(d.src) + (int64_t)item.w * d.sb;
        T* dst = reinterpret_cast<T*>(d.dst) + (int64_t)item.w * d.db;
        const int cbx = d.bx / 2, cby = d.by / 2, cbz = d.bz / 2;
        const int rows = TY + d.by - 1;
        const int D = (EPC - cbx % EPC) % EPC;
        const int gx0 = x0 - cbx - D;
        const int nch = (TX + d.bx - 1 + D + EPC - 1) / EPC;
        const int zin0 = zs - cbz;
        const int nplanes = (ze - 1 + (d.bz - 1 - cbz)) - zin0 + 1;

        auto issue = [&](int zi, int stage) {
            T* sb = s_in + stage * stage_elems;
            const bool zplane = d.zero_pad && (zi < 0 || zi >= d.nz);
            // planes beyond the real tap radius feed only zero-padded taps:
            // any plane inside the image will do (the padded radius can
            // exceed the extent, where the border map is not defined)
            const int zm = zplane ? 0
                         : (zi < -d.rz || zi >= d.nz + d.rz) ? (zi < 0 ? 0 : d.nz - 1)
                                                             : map_border32(d.border, d.nz, zi);
            const T* pl = src + (int64_t)zm * d.sz;
            for (int t = tid; t < rows * nch; t += NT) {
                const int r = t / nch, q = t - (t / nch) * nch;
                T* sd = sb + r * PITCH + q * EPC;
                int y = y0 - cby + r;
                const bool zrow = zplane || (d.zero_pad && (y < 0 || y >= d.ny));
                if (zrow) {
#pragma unroll
                    for (int e = 0; e < EPC; e++) sd[e] = from_f<T>(0.f);
                    continue;
                }
                y = (y < -d.ry || y >= d.ny + d.ry) ? d.ny - 1 : map_border32(d.border, d.ny, y);
                const T* row = pl + (int64_t)y * d.sy;
                const int cx0 = gx0 + q * EPC;
                if (d.vec_ld && cx0 >= 0 && cx0 + EPC <= d.nx) {
                    cp_async16(sd, row + cx0);
                } else {
#pragma unroll
                    for (int e = 0; e < EPC; e++) {
                        int x = cx0 + e;
                        if (d.zero_pad && (x < 0 || x >= d.nx)) { sd[e] = from_f<T>(0.f); continue; }
                        x = (x < -d.rx || x >= d.nx + d.rx) ? d.nx - 1 : map_border32(d.border, d.nx, x);
                        if constexpr (sizeof(T) == 4) cp_async4(sd + e, row + (int64_t)x * d.sx);
                        else sd[e] = row[(int64_t)x * d.sx];
                    }
                }
            }
        };

        __syncthreads();      // s_w ready; previous item's stages and ring are free
        issue(zin0, 0);
        cp_async_commit();
        int newest = -1;
        for (int n = 0; n < nplanes; n++) {
            cp_async_wait_all();
            __syncthreads();
            if (n + 1 < nplanes) issue(zin0 + n + 1, (n + 1) & 1);
            cp_async_commit();
            const T* sb = s_in + (n & 1) * stage_elems;
            switch (d.bx) {
#define NDLGPU_XC(B) case B: xpass<T, TX, B>(sb, s_x, s_w, rows, PITCH, NT, d, zones, x0); break;
                NDLGPU_BUCKETS(NDLGPU_XC)
#undef NDLGPU_XC
            default: break;
            }
            __syncthreads();
            float yv[2] = {0.f, 0.f};
            switch (d.by) {
#define NDLGPU_YC(B) case B: ypass<TX, B>(s_x, s_w + 40, ty, tx2, d, zones, y0, yv); break;
                NDLGPU_BUCKETS(NDLGPU_YC)
#undef NDLGPU_YC
            default: break;
            }
            newest = (newest + 1 == ring) ? 0 : newest + 1;
            *reinterpret_cast<float2*>(s_ring + (size_t)newest * (TX * TY) + ty * TX + 2 * tx2) = make_float2(yv[0], yv[1]);
            // the ring slot of each position is private to its thread: no barrier
            if (n >= d.bz - 1) {
                const int zo = zin0 + n - (d.bz - 1 - cbz);
                float out[2] = {0.f, 0.f};
                switch (d.bz) {
#define NDLGPU_ZC(B) case B: zpass<TX, TY, B>(s_ring, ring, newest, s_w + 80, ty * TX + 2 * tx2, d, zones, zo, out); break;
                    NDLGPU_BUCKETS(NDLGPU_ZC)
#undef NDLGPU_ZC
                default: break;
                }
                const int xg = x0 + 2 * tx2, yg = y0 + ty;
                if (yg < d.ny) {
                    T* rowo = dst + (int64_t)zo * d.dz + (int64_t)yg * d.dy;
                    if (d.vec_st && xg + 2 <= d.nx) {
                        if constexpr (sizeof(T) == 4) {
                            *reinterpret_cast<float2*>(rowo + xg) = make_float2(out[0], out[1]);
                        } else {
                            T pair[2] = {from_f<T>(out[0]), from_f<T>(out[1])};
                            *reinterpret_cast<uint32_t*>(rowo + xg) = *reinterpret_cast<uint32_t*>(pair);
                        }
                    } else {
                        if (xg < d.nx) rowo[(int64_t)xg * d.dx] = from_f<T>(out[0]);
                        if (xg + 1 < d.nx) rowo[(int64_t)(xg + 1) * d.dx] = from_f<T>(out[1]);
                    }
                }
            }
        }
        cp_async_wait_all();
        __syncthreads();      // everyone done with s_item, s_w, stages and ring
    }
}

template <class T, int TX, int TY>
size_t smem_bytes(int rows_max, int ring)
{
    const size_t stage = (size_t)rows_max * (TX + 48) * sizeof(T);
    const size_t x_off = (2 * stage + 15) / 16 * 16;
    return x_off + (size_t)rows_max * TX * 4 + (size_t)ring * TX * TY * 4 + 3 * 40 * 4 + 16;
}

template <class T, int TX, int TY>
cudaError_t prepare_b(BatchLaunch* L)
{
    const size_t smem = smem_bytes<T, TX, TY>(L->rows_max, L->ring);
    if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
    cudaError_t e = cudaFuncSetAttribute(k_batch<T, TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch<T, TX, TY>, TX * TY / 2, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int dev = 0, sms = 148;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    L->grid = sms * per_sm;
    L->smem = smem;
    return cudaSuccess;
}

template <class T, int TX, int TY>
cudaError_t launch_b(const BatchLaunch& L, cudaStream_t s)
{
    k_batch<T, TX, TY><<<L.grid, TX * TY / 2, L.smem, s>>>(L.descs, L.items, L.nitems, L.counter, L.zones,
                                                           L.rows_max, L.ring);
    count_launch();
    return cudaGetLastError();
}

struct TileCfg {
    int tx, ty;
};
const TileCfg kTiles[] = {{32, 16}, {64, 16}, {32, 32}, {64, 8}};

template <class T>
cudaError_t prepare_t(int cfg, BatchLaunch* L)
{
    switch (cfg) {
    case 0: return prepare_b<T, 32, 16>(L);
    case 1: return prepare_b<T, 64, 16>(L);
    case 2: return prepare_b<T, 32, 32>(L);
    case 3: return prepare_b<T, 64, 8>(L);
    default: return cudaErrorInvalidValue;
    }
}

template <class T>
cudaError_t launch_t(int cfg, const BatchLaunch& L, cudaStream_t s)
{
    switch (cfg) {
    case 0: return launch_b<T, 32, 16>(L, s);
    case 1: return launch_b<T, 64, 16>(L, s);
    case 2: return launch_b<T, 32, 32>(L, s);
    case 3: return launch_b<T, 64, 8>(L, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

int batch_tile_configs() { return (int)(sizeof(kTiles) / sizeof(kTiles[0])); }

void batch_tile_info(int i, int* tx, int* ty, int* nt)
{
    *tx = kTiles[i].tx;
    *ty = kTiles[i].ty;
    *nt = kTiles[i].tx * kTiles[i].ty / 2;
}

int batch_bucket(int k)
{
    const int b[] = {1, 3, 5, 9, 13, 17, 21, 25, 29, 33, 37};
    for (int v : b)
        if (k <= v) return v;
    return -1;
}

size_t batch_smem(int dtype, int cfg, int rows_max, int ring)
{
    const int es = dtype == NDLGPU_F32 ? 4 : 2;
    const int tx = kTiles[cfg].tx, ty = kTiles[cfg].ty;
    const size_t stage = (size_t)rows_max * (tx + 48) * es;
    const size_t x_off = (2 * stage + 15) / 16 * 16;
    return x_off + (size_t)rows_max * tx * 4 + (size_t)ring * tx * ty * 4 + 3 * 40 * 4 + 16;
}

cudaError_t batch_prepare(int dtype, int cfg, BatchLaunch* L)
{
    switch (dtype) {
    case NDLGPU_F32: return prepare_t<float>(cfg, L);
    case NDLGPU_BF16: return prepare_t<__nv_bfloat16>(cfg, L);
    case NDLGPU_F16: return prepare_t<__half>(cfg, L);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_batch(int dtype, int cfg, const BatchLaunch& L, cudaStream_t s)
{
    switch (dtype) {
    case NDLGPU_F32: return launch_t<float>(cfg, L, s);
    case NDLGPU_BF16: return launch_t<__nv_bfloat16>(cfg, L, s);
    case NDLGPU_F16: return launch_t<__half>(cfg, L, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace ndlgpu
