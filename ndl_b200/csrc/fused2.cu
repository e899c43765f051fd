// fused2.cu -- fused separable forward for float storage (f32 / bf16 / f16
// in, FP32 accumulation): up to three 1-D passes, one HBM read and one write
// per element.
//
// A CTA owns a TX x TY column tile of one batch item and streams a chunk of Z
// planes (2.5-D blocking):
//   load  : plane zi (border-mapped along Z) with its X/Y halos goes to a
//           3-stage shared-memory ring by cp.async, two planes ahead of the
//           compute.  Rows are border-mapped as whole rows; the columns that
//           fall outside [0, nx) and ragged 16-byte chunks are copied element
//           by element from their border-mapped column.
//   X pass: shared-memory rows, 4 outputs per thread-unit from a register
//           window (taps as compile-time offsets).
//   Y pass: 4 columns x 2 rows of outputs per thread.
//   Z pass: a KZ-deep register queue per thread; the slot of the newest plane
//           rotates, and the queue is read through a compile-time slot
//           dispatch so that no value is ever moved.
// Border maps are Clamp / Wrap / Reflect of mathHelpers.h:23-25, applied to
// load coordinates only.
//
// The adjoint with Clamp/Reflect reads zero outside the image.  Where the
// source rows are 16-byte aligned, its planes come in through the copy engine
// instead: one 4-D tensor-map box (cp.async.bulk.tensor) per plane, issued by
// one thread and completed on an mbarrier; the engine's out-of-bounds zero
// fill is exactly that zero padding, so no element-copy table is needed.
// Every mbarrier wait is bounded: on timeout the CTA sets bit 1 of the guard
// word and returns.
#include <algorithm>
#include <cstring>
#include <utility>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "dtype.cuh"

namespace ndlgpu {

namespace {

constexpr int TX = 64;
constexpr int STAGES = 3;

template <class T> __device__ __forceinline__ float to_f(T v);
template <> __device__ __forceinline__ float to_f<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <> __device__ __forceinline__ float to_f<__half>(__half v) { return __half2float(v); }

template <class T> __device__ __forceinline__ T from_f(float v);
template <> __device__ __forceinline__ float from_f<float>(float v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ __half from_f<__half>(float v) { return __float2half_rn(v); }

// 4 consecutive shared-memory elements (aligned to 4 elements) as floats.
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
    const __half2 a = *reinterpret_cast<const __half2*>(&t.x);
    const __half2 b = *reinterpret_cast<const __half2*>(&t.y);
    const float2 fa = __half22float2(a), fb = __half22float2(b);
    v[0] = fa.x; v[1] = fa.y; v[2] = fb.x; v[3] = fb.y;
}

// 4 consecutive outputs to global memory (aligned when vec is set).
__device__ __forceinline__ void stg4(float* p, const float* v) { *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]); }
__device__ __forceinline__ void stg4(__nv_bfloat16* p, const float* v)
{
    __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]), b = __floats2bfloat162_rn(v[2], v[3]);
    uint2 t;
    t.x = *reinterpret_cast<uint32_t*>(&a);
    t.y = *reinterpret_cast<uint32_t*>(&b);
    *reinterpret_cast<uint2*>(p) = t;
}
__device__ __forceinline__ void stg4(__half* p, const float* v)
{
    __half2 a = __floats2half2_rn(v[0], v[1]), b = __floats2half2_rn(v[2], v[3]);
    uint2 t;
    t.x = *reinterpret_cast<uint32_t*>(&a);
    t.y = *reinterpret_cast<uint32_t*>(&b);
    *reinterpret_cast<uint2*>(p) = t;
}

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
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ int32_t g_guard_fused;

constexpr int kTmaSpins = 1 << 22;   // bound on the mbarrier polls for one plane
// Test controls (ndlgpu_test_wait_timeouts): the poll bound of a plane wait,
// and extra bytes every plane load announces to its mbarrier but never
// delivers, so that the wait runs out without anything faulting.
__device__ int g_tma_wait_spins = kTmaSpins;
__device__ unsigned g_tma_tx_bias = 0;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void mbar_complete_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.complete_tx.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// orders this thread's earlier generic-proxy shared-memory accesses before
// the copy engine's writes that it issues next
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
// one box of a 4-D tensor map into shared memory, completing on bar
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, "
        "%6}], [%2];\n" ::"r"(smem_u32(dst)),
        "l"(map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}

template <class Tin, int KX, int KY, int TY_>
struct Geo {
    static constexpr int TY = TY_;
    static constexpr int NT = 8 * TY;                           // 16 column groups x TY/2 row pairs
    static constexpr int EPC = 16 / (int)sizeof(Tin);          // elements per 16-byte chunk
    static constexpr int CX = KX / 2;
    static constexpr int CY = KY / 2;
    static constexpr int D = (EPC - CX % EPC) % EPC;          // smem column of global x0 - CX
    static constexpr int ROWS = TY + KY - 1;
    static constexpr int NCH = (TX + KX - 1 + D + EPC - 1) / EPC;
    static constexpr int NV = (D % 4 + KX + 3 + 3) / 4;        // 4-wide loads per X window
    static constexpr int WBASE = (D / 4) * 4;                   // first loaded column of a window
    static constexpr int WOFF = D % 4;                          // window offset inside it
    // elements per shared row: the loaded chunks, and every column an X
    // window reads (the last window may read past the loaded chunks)
    static constexpr int WEND = 60 + WBASE + 4 * NV;
    static constexpr int PITCH = (NCH * EPC > WEND ? NCH * EPC : (WEND + EPC - 1) / EPC * EPC);
    static constexpr int NTASK = (ROWS * NCH + NT - 1) / NT;
    static constexpr int NXU = (ROWS * 16 + NT - 1) / NT;       // X-pass units per thread
    static constexpr size_t STAGE_BYTES = (size_t)ROWS * PITCH * sizeof(Tin);
    static constexpr size_t IN_BYTES = (size_t)STAGES * STAGE_BYTES;
    static constexpr size_t X_BYTES = (size_t)ROWS * TX * sizeof(float);
    // element-copy table: border columns and ragged chunks, built once per CTA
    static constexpr int MAXEL = ROWS * PITCH;
    static constexpr size_t TAB_BYTES = (size_t)MAXEL * 8;
    static constexpr size_t SMEM = IN_BYTES + X_BYTES + TAB_BYTES + 16 + 128;   // + alignment slack
};

// Output plane sum of the Z queue for the newest slot S: tap k reads slot
// (S + 1 + k) mod KZ (the queue holds the last KZ planes in ring order).
template <int KZ, int S>
__device__ __forceinline__ void zstep(float2 (&q)[KZ][4], const float2 (&yv)[4], float2 (&out)[4],
                                      const float2 (&wz)[KZ])
{
#pragma unroll
    for (int e = 0; e < 4; e++) q[S][e] = yv[e];
#pragma unroll
    for (int e = 0; e < 4; e++) {
        float2 a = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < KZ; k++) a = __ffma2_rn(q[(S + 1 + k) % KZ][e], wz[k], a);
        out[e] = a;
    }
}

// Row of the effective-weight table for position j of an axis of extent n
// with zone radius r, or -1 outside the zones.
__device__ __forceinline__ int zone_row(int j, int n, int r)
{
    if (j < r) return j;
    if (j >= n - r) return r + (j - (n - r));
    return -1;
}

template <int KZ>
__device__ __forceinline__ void zdispatch(int slot, float2 (&q)[KZ][4], const float2 (&yv)[4], float2 (&out)[4],
                                          const float2 (&wz)[KZ])
{
#define NDLGPU_ZCASE(S) \
    case S:             \
        if constexpr (S < KZ) zstep<KZ, (S < KZ ? S : 0)>(q, yv, out, wz); \
        break;
    switch (slot) {
        NDLGPU_ZCASE(0) NDLGPU_ZCASE(1) NDLGPU_ZCASE(2) NDLGPU_ZCASE(3) NDLGPU_ZCASE(4) NDLGPU_ZCASE(5)
        NDLGPU_ZCASE(6) NDLGPU_ZCASE(7) NDLGPU_ZCASE(8) NDLGPU_ZCASE(9) NDLGPU_ZCASE(10) NDLGPU_ZCASE(11)
        NDLGPU_ZCASE(12) NDLGPU_ZCASE(13) NDLGPU_ZCASE(14) NDLGPU_ZCASE(15) NDLGPU_ZCASE(16) NDLGPU_ZCASE(17)
        NDLGPU_ZCASE(18) NDLGPU_ZCASE(19) NDLGPU_ZCASE(20) NDLGPU_ZCASE(21) NDLGPU_ZCASE(22) NDLGPU_ZCASE(23)
        NDLGPU_ZCASE(24) NDLGPU_ZCASE(25) NDLGPU_ZCASE(26) NDLGPU_ZCASE(27) NDLGPU_ZCASE(28) NDLGPU_ZCASE(29)
        NDLGPU_ZCASE(30) NDLGPU_ZCASE(31) NDLGPU_ZCASE(32) NDLGPU_ZCASE(33) NDLGPU_ZCASE(34) NDLGPU_ZCASE(35)
        NDLGPU_ZCASE(36)
    default: break;
    }
#undef NDLGPU_ZCASE
}

// CTAs per SM: the adjoint's border-zone paths and deep Z queues need more
// registers (13 planes fit 3 CTAs; 15 planes measured faster at 2).
template <int TY, bool ADJ, int KZ>
struct Occ {
    static constexpr int value = TY <= 16 ? (KZ > 13 ? 2 : (KZ > 11 ? 3 : ((ADJ && KZ > 9) ? 3 : 4))) : 2;
};

// TMA: plane loads through the tensor map (adjoint with zero padding only).
template <class Tin, class Tout, int KX, int KY, int KZ, int TY, bool ADJ, bool TMA>
__global__ void __launch_bounds__(8 * TY, (Occ<TY, ADJ, KZ>::value))
    k_fused2(const __grid_constant__ FusedParams p, const __grid_constant__ CUtensorMap tmap)
{
    using G = Geo<Tin, KX, KY, TY>;
    constexpr int NT = G::NT;
    static_assert(!TMA || ADJ, "the copy-engine loader serves the zero-padded adjoint");
    static_assert(!TMA || G::STAGE_BYTES % 128 == 0, "plane stages stay 128-byte aligned for the copy engine");
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    __shared__ uint64_t s_bar[STAGES];
    unsigned char* smem_raw = smem_dyn + ((128u - (smem_u32(smem_dyn) & 127u)) & 127u);
    Tin* s_in = reinterpret_cast<Tin*>(smem_raw);
    float* s_x = reinterpret_cast<float*>(smem_raw + G::IN_BYTES);
    int2* s_tab = reinterpret_cast<int2*>(smem_raw + G::IN_BYTES + G::X_BYTES);
    int* s_ntab = reinterpret_cast<int*>(smem_raw + G::IN_BYTES + G::X_BYTES + G::TAB_BYTES);

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

    constexpr int CZ = KZ / 2;
    constexpr int HZ = KZ - 1 - CZ;
    const int gx0 = x0 - G::CX - G::D;    // global column of shared column 0 (multiple of EPC)

    // Loader set-up, once per CTA.  Chunk t = tid + j*NT covers shared row
    // r = t / NCH, columns [q*EPC, (q+1)*EPC).  A chunk lying inside [0, nx)
    // on a 16-byte aligned row is one 16-byte copy (offsets kept in
    // registers); every other element goes to a shared table of (shared
    // offset, in-plane global offset) pairs with its column border-mapped.
    const bool zp = ADJ && p.zero_pad;   // adjoint, Clamp/Reflect: zero outside the image
    unsigned tx_bias = 0;
    int wait_spins = kTmaSpins;
    if constexpr (TMA) {
        tx_bias = g_tma_tx_bias;
        wait_spins = g_tma_wait_spins;
    }
    if (tid == 0) {
        *s_ntab = 0;
        if constexpr (TMA) {
            for (int st = 0; st < STAGES; st++) mbar_init(&s_bar[st], 1);
            fence_mbar_init();
        }
    }
    __syncthreads();
    int32_t goff[G::NTASK];
    int32_t soff[G::NTASK];
#pragma unroll
    for (int j = 0; j < G::NTASK; j++) {
        const int t = tid + j * NT;
        goff[j] = -1;
        soff[j] = 0;
        if constexpr (TMA) continue;
        if (t >= G::ROWS * G::NCH) continue;
        const int r = t / G::NCH;
        const int q = t - r * G::NCH;
        int y = y0 - G::CY + r;
        const int cx0 = gx0 + q * G::EPC;
        if (zp && (y < 0 || y >= p.ny)) {
            // a row outside the image: zero in every stage, never copied
            for (int e = 0; e < G::EPC; e++)
                for (int st = 0; st < STAGES; st++) s_in[st * (G::ROWS * G::PITCH) + r * G::PITCH + q * G::EPC + e] = Tin(0.f);
            continue;
        }
        y = (y >= p.ny + KY - 1 - G::CY) ? p.ny - 1 : map_border32(p.border, p.ny, y);
        const int32_t rowoff = (int32_t)(y * p.sy);
        if (p.vec_ld && cx0 >= 0 && cx0 + G::EPC <= p.nx) {
            goff[j] = rowoff + cx0;
            soff[j] = r * G::PITCH + q * G::EPC;
        } else {
            for (int e = 0; e < G::EPC; e++) {
                int x = cx0 + e;
                if (zp && (x < 0 || x >= p.nx)) {
                    for (int st = 0; st < STAGES; st++) s_in[st * (G::ROWS * G::PITCH) + r * G::PITCH + q * G::EPC + e] = Tin(0.f);
                    continue;
                }
                x = (x >= p.nx + KX - 1 - G::CX || x < -G::CX) ? p.nx - 1 : map_border32(p.border, p.nx, x);
                const int slot_i = atomicAdd(s_ntab, 1);
                s_tab[slot_i] = make_int2(r * G::PITCH + q * G::EPC + e, rowoff + (int32_t)(x * p.sx));
            }
        }
    }
    __syncthreads();
    const int ntab = *s_ntab;

    // copies of the parameters the plane loads read (a lambda reading the
    // __grid_constant__ parameters through a reference would make generic loads)
    const int l_border = p.border, l_nz = p.nz, l_tpos0 = p.tma_pos[0], l_tpos1 = p.tma_pos[1];
    const int64_t l_sz = p.sz;
    auto issue = [&](int zi, int stage) {
        Tin* sb = s_in + stage * (G::ROWS * G::PITCH);
        if constexpr (TMA) {
            // one box: rows y0-CY.., columns gx0.. of plane zi; the planes,
            // rows and columns outside the image come back zero-filled
            if (tid == 0) {
                const int yc = y0 - G::CY;
                auto coord = [&](int d) { return l_tpos0 == d ? yc : (l_tpos1 == d ? zi : bat); };
                fence_proxy_async();
                mbar_expect_tx(&s_bar[stage], (unsigned)G::STAGE_BYTES + tx_bias);
                tma_load_4d(sb, &tmap, &s_bar[stage], gx0, coord(0), coord(1), coord(2));
            }
            return;
        }
        if (zp && (zi < 0 || zi >= l_nz)) {
            // a plane outside the image: zero what the copies would fill
#pragma unroll
            for (int j = 0; j < G::NTASK; j++)
                if (goff[j] >= 0) *reinterpret_cast<uint4*>(sb + soff[j]) = make_uint4(0u, 0u, 0u, 0u);
            for (int i = tid; i < ntab; i += NT) sb[s_tab[i].x] = Tin(0.f);
            return;
        }
        const int zm = map_border32(l_border, l_nz, zi);
        const Tin* pl = src + (int64_t)zm * l_sz;
#pragma unroll
        for (int j = 0; j < G::NTASK; j++)
            if (goff[j] >= 0) cp_async16(sb + soff[j], pl + goff[j]);
        for (int i = tid; i < ntab; i += NT) {
            const int2 e = s_tab[i];
            if constexpr (sizeof(Tin) == 4) cp_async4(sb + e.x, pl + e.y);
            else sb[e.x] = pl[e.y];
        }
    };

    const int zin0 = zs - CZ;
    const int zin1 = ze - 1 + HZ;
    const int nplanes = zin1 - zin0 + 1;
#pragma unroll
    for (int s = 0; s < STAGES - 1; s++) {
        if (s < nplanes) issue(zin0 + s, s);
        cp_async_commit();
    }

    const int gx = tid & 15;
    const int gy = tid >> 4;
    float2 q[KZ][4];
#pragma unroll
    for (int k = 0; k < KZ; k++)
#pragma unroll
        for (int e = 0; e < 4; e++) q[k][e] = make_float2(0.f, 0.f);

    // adjoint zone rows of this thread's two rows, and whether the tile has
    // zone columns (both plane-invariant)
    int ey[2] = {-1, -1};
    if (zp) {
#pragma unroll
        for (int h = 0; h < 2; h++) ey[h] = zone_row(y0 + 2 * gy + h, p.ny, G::CY);
    }
    const bool yzone = ey[0] >= 0 || ey[1] >= 0;
    const bool xzone_tile = zp && (x0 < G::CX || x0 + TX > p.nx - G::CX);
    int slot = 0;
    unsigned phase = 0;                  // mbarrier parity of the current pass over the ring
    int stage = 0;                       // ring stage of plane n
    int stage_next = STAGES - 1;         // ring stage of plane n + STAGES - 1
    // output rows of this thread: row offsets and, per plane, a running
    // plane pointer (the first output plane is input plane KZ - 1)
    const int xb = x0 + 4 * gx;
    int64_t rowoff[2];
#pragma unroll
    for (int h = 0; h < 2; h++) rowoff[h] = (int64_t)(y0 + 2 * gy + h) * p.dy;
    Tout* oplane = dst + (int64_t)(zin0 + KZ - 1 - HZ) * p.dz;
    for (int n = 0; n < nplanes; n++) {
        if constexpr (TMA) {
            bool ok = false;
            for (int i = 0; i < wait_spins && !ok; i++) ok = mbar_try_wait(&s_bar[stage], phase);
            // plane n visible; every thread is past the X pass of plane n-1
            if (__syncthreads_or(!ok)) {
                if (tid == 0) {
                    atomicOr(&g_guard_fused, 2);
                    // planes n .. n+STAGES-2 may still be landing in this
                    // CTA's ring: retire the announced surplus (test control)
                    // and wait, bounded, for each before the CTA lets go of
                    // its shared memory.  Plane m sits in stage m % STAGES
                    // with parity (m / STAGES) & 1.
                    for (int m = n; m < min(n + STAGES - 1, nplanes); m++) {
                        uint64_t* bar = &s_bar[m % STAGES];
                        if (tx_bias) mbar_complete_tx(bar, tx_bias);
                        const unsigned par = (unsigned)(m / STAGES) & 1u;
                        for (int i = 0; i < kTmaSpins && !mbar_try_wait(bar, par); i++) {
                        }
                    }
                }
                return;
            }
            if (stage + 1 == STAGES) phase ^= 1u;
        } else {
            cp_async_wait<STAGES - 2>();
            __syncthreads();    // plane n visible; every thread is past the X pass of plane n-1
        }
        if (n + STAGES - 1 < nplanes) issue(zin0 + n + STAGES - 1, stage_next);
        cp_async_commit();
        stage_next = (stage_next + 1 == STAGES) ? 0 : stage_next + 1;

        const Tin* sb = s_in + stage * (G::ROWS * G::PITCH);
        // X pass: ROWS x 16 units of 4 outputs; unit i of this thread is row
        // gy + i * NT/16, column group gx
#pragma unroll
        for (int i = 0; i < G::NXU; i++) {
            if (G::NXU * NT != G::ROWS * 16 && gy + i * (NT / 16) >= G::ROWS) break;
            const int r = gy + i * (NT / 16), g = gx;
            float win[G::NV * 4];
#pragma unroll
            for (int v = 0; v < G::NV; v++) lds4(sb + r * G::PITCH + 4 * g + G::WBASE + 4 * v, win + 4 * v);
            float acc[4];
#pragma unroll
            for (int m = 0; m < 4; m++) {
                float a = 0.f;
#pragma unroll
                for (int k = 0; k < KX; k++) a = fmaf(win[G::WOFF + m + k], p.wxf[k], a);
                acc[m] = a;
            }
            *reinterpret_cast<float4*>(s_x + r * TX + 4 * g) = make_float4(acc[0], acc[1], acc[2], acc[3]);
        }
        if (xzone_tile) {
            // adjoint border columns: effective weights (a separate pass keeps
            // the main X pass free of these registers)
            __syncthreads();
            const int zlo = max(0, G::CX - x0);                 // columns x0 .. x0+zlo-1 are left-zone
            const int zr0 = max(0, p.nx - G::CX - x0);          // columns from zr0 on are right-zone
            const int nl = min(zlo, TX), nr = max(0, TX - zr0);
            for (int t = tid; t < G::ROWS * (nl + nr); t += NT) {
                const int r = t / (nl + nr), ci = t - r * (nl + nr);
                const int col = ci < nl ? ci : zr0 + (ci - nl);
                const int e = zone_row(x0 + col, p.nx, G::CX);
                if (e < 0 || col >= TX) continue;
                float a = 0.f;
#pragma unroll
                for (int k = 0; k < KX; k++)
                    a = fmaf(to_f<Tin>(sb[r * G::PITCH + G::D + col + k]), p.zx[e][k], a);
                s_x[r * TX + col] = a;
            }
        }
        __syncthreads();
        // Y pass (packed pairs of columns): rows 2gy and 2gy+1
        float2 yv[4] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
#pragma unroll
        for (int j = 0; j < KY + 1; j++) {
            const float4 v = *reinterpret_cast<const float4*>(s_x + (2 * gy + j) * TX + 4 * gx);
            const float2 lo = make_float2(v.x, v.y), hi = make_float2(v.z, v.w);
            if (j < KY) {
                yv[0] = __ffma2_rn(lo, p.wy2[j], yv[0]);
                yv[1] = __ffma2_rn(hi, p.wy2[j], yv[1]);
            }
            if (j >= 1) {
                yv[2] = __ffma2_rn(lo, p.wy2[j - 1], yv[2]);
                yv[3] = __ffma2_rn(hi, p.wy2[j - 1], yv[3]);
            }
        }
        if (yzone) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int e = ey[h];
                if (e < 0) continue;
                float2 a0 = make_float2(0.f, 0.f), a1 = make_float2(0.f, 0.f);
#pragma unroll
                for (int j = 0; j < KY; j++) {
                    const float4 v = *reinterpret_cast<const float4*>(s_x + (2 * gy + h + j) * TX + 4 * gx);
                    const float w = p.zy[e][j];
                    a0 = __ffma2_rn(make_float2(v.x, v.y), make_float2(w, w), a0);
                    a1 = __ffma2_rn(make_float2(v.z, v.w), make_float2(w, w), a1);
                }
                yv[2 * h] = a0;
                yv[2 * h + 1] = a1;
            }
        }
        // Z pass
        float2 out2[4];
        if constexpr (ADJ) {
            // shift-register queue (one copy of the border-plane path)
#pragma unroll
            for (int k = 0; k + 1 < KZ; k++)
#pragma unroll
                for (int e = 0; e < 4; e++) q[k][e] = q[k + 1][e];
#pragma unroll
            for (int e = 0; e < 4; e++) q[KZ - 1][e] = yv[e];
            const int ez = zp ? zone_row(zin0 + n - HZ, p.nz, CZ) : -1;
            if (ez < 0) {
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    float2 a = make_float2(0.f, 0.f);
#pragma unroll
                    for (int k = 0; k < KZ; k++) a = __ffma2_rn(q[k][e], p.wz2[k], a);
                    out2[e] = a;
                }
            } else {
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    float2 a = make_float2(0.f, 0.f);
#pragma unroll
                    for (int k = 0; k < KZ; k++) {
                        const float w = p.zz[ez][k];
                        a = __ffma2_rn(q[k][e], make_float2(w, w), a);
                    }
                    out2[e] = a;
                }
            }
        } else {
            // the Z taps in registers for the step (a reference to the
            // __grid_constant__ parameters would make generic loads)
            float2 wz[KZ];
#pragma unroll
            for (int k = 0; k < KZ; k++) wz[k] = p.wz2[k];
            zdispatch<KZ>(slot, q, yv, out2, wz);
            slot = (slot + 1 == KZ) ? 0 : slot + 1;
        }
        const float out[8] = {out2[0].x, out2[0].y, out2[1].x, out2[1].y, out2[2].x, out2[2].y, out2[3].x, out2[3].y};
        stage = (stage + 1 == STAGES) ? 0 : stage + 1;
        if (n >= KZ - 1) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int y = y0 + 2 * gy + h;
                if (y >= p.ny) continue;
                Tout* row = oplane + rowoff[h];
                if (p.vec_st && xb + 4 <= p.nx) {
                    stg4(row + xb, out + 4 * h);
                } else {
#pragma unroll
                    for (int m = 0; m < 4; m++)
                        if (xb + m < p.nx) row[(int64_t)(xb + m) * p.dx] = from_f<Tout>(out[4 * h + m]);
                }
            }
            oplane += p.dz;
        }
    }
    cp_async_wait<0>();
}

using LaunchFn = cudaError_t (*)(const FusedParams&, cudaStream_t);

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }();
    return fn;
}

template <class T> constexpr CUtensorMapDataType tma_type();
template <> constexpr CUtensorMapDataType tma_type<float>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT32; }
template <> constexpr CUtensorMapDataType tma_type<__nv_bfloat16>() { return CU_TENSOR_MAP_DATA_TYPE_BFLOAT16; }
template <> constexpr CUtensorMapDataType tma_type<__half>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT16; }

// A 4-D tiled map of the source -- x, then y, z and batch in increasing
// stride order -- with a box of boxx columns x boxy rows of one plane, for
// the adjoint with Clamp/Reflect (its zero padding is the copy engine's
// fill); p.tma_pos gets the map dimension (0..2 after x) of y, z and batch.
// False where the plane loads keep the cp.async path: the forward (a
// border-mapped halo would have to be rewritten in every border tile), Wrap,
// unaligned, non-unit-stride or negative-stride sources, or an encode failure.
template <class Tin>
bool plane_map(FusedParams& p, int boxx, int boxy, CUtensorMap* m)
{
    if (!p.adj || !p.zero_pad || !p.vec_ld || p.sx != 1) return false;
    if (reinterpret_cast<uintptr_t>(p.src) % 16 != 0) return false;
    // a partial last column tile has most of its box outside the image, and
    // such boxes measured 7-13x slower than the cp.async loads (e.g. a
    // 72-wide volume: 380 us against 46 us): whole tiles only
    if (p.nx % TX != 0) return false;
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    const int64_t es = (int64_t)sizeof(Tin);
    struct Dim {
        int64_t n, s;
        int role;
    } d[3] = {{p.ny, p.sy, 0}, {p.nz, p.sz, 1}, {p.nbatch, p.sb, 2}};
    int64_t span = es * p.nx;
    for (const Dim& e : d) {
        if (e.n <= 1) continue;
        if (e.s <= 0 || (e.s * es) % 16 != 0) return false;
        span = std::max(span, e.s * es * e.n);
    }
    span = (span + 15) / 16 * 16;
    for (Dim& e : d)
        if (e.n <= 1) e.s = span / es;   // never stepped: any valid stride
    std::stable_sort(d, d + 3, [](const Dim& a, const Dim& b) { return a.s < b.s; });
    cuuint64_t gdim[4] = {(cuuint64_t)p.nx, 0, 0, 0};
    cuuint64_t gstr[3];
    cuuint32_t box[4] = {(cuuint32_t)boxx, 1, 1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    for (int i = 0; i < 3; i++) {
        gdim[i + 1] = (cuuint64_t)d[i].n;
        gstr[i] = (cuuint64_t)(d[i].s * es);
        if (gstr[i] >= (1ull << 40)) return false;
        p.tma_pos[d[i].role] = i;
        if (d[i].role == 0) box[i + 1] = (cuuint32_t)boxy;
    }
    std::memset(m, 0, sizeof(*m));
    const CUresult r = enc(m, tma_type<Tin>(), 4, const_cast<char*>(p.src), gdim, gstr, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

template <class Tin, class Tout, int KX, int KY, int KZ, int TY, bool ADJ>
cudaError_t launch2(const FusedParams& p, cudaStream_t s)
{
    using G = Geo<Tin, KX, KY, TY>;
    static_assert(G::PITCH <= 256 && G::ROWS <= 256, "tensor-map boxes hold at most 256 per dimension");
    static_assert(G::PITCH * sizeof(Tin) % 16 == 0, "box rows are whole 16-byte units");
    static bool configured[2] = {false, false};
    FusedParams pp = p;
    CUtensorMap tmap;
    std::memset(&tmap, 0, sizeof(tmap));
    bool tma = false;
    auto kern = k_fused2<Tin, Tout, KX, KY, KZ, TY, ADJ, false>;
    // the copy engine writes 128-byte aligned stages: geometries whose plane
    // stage is not a multiple of 128 bytes keep cp.async
    if constexpr (ADJ && G::STAGE_BYTES % 128 == 0) {
        tma = plane_map<Tin>(pp, G::PITCH, G::ROWS, &tmap);
        if (tma) kern = k_fused2<Tin, Tout, KX, KY, KZ, TY, ADJ, true>;
    }
    if (!configured[tma]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM);
        if (e != cudaSuccess) return e;
        configured[tma] = true;
    }
    const int ntx = (p.nx + TX - 1) / TX;
    const int nty = (p.ny + TY - 1) / TY;
    const long long gx = (long long)ntx * nty * p.nbatch;
    // Z chunks: about one full wave of resident CTAs, chunks of >= 4*KZ planes
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long slots = (long long)sms * Occ<TY, ADJ, KZ>::value;
    const int chunks = pick_zchunks(gx, slots, p.nz, KZ - 1);
    pp.zchunk = max(1, (p.nz + chunks - 1) / chunks);
    const int gz = (p.nz + pp.zchunk - 1) / pp.zchunk;
    if (gx > 0x7fffffffLL || gz > 65535) return cudaErrorInvalidConfiguration;
    kern<<<dim3((unsigned)gx, (unsigned)gz), G::NT, G::SMEM, s>>>(pp, tmap);
    count_launch();
    return cudaGetLastError();
}

struct Variant2 {
    int adj, sdt, ddt, kx, ky, kz;
    LaunchFn fn;
};

#define NDLGPU_V2(A, TI, TO, DI, DO, KX_, KY_, KZ_, TY_) \
    {A, DI, DO, KX_, KY_, KZ_, &launch2<TI, TO, KX_, KY_, KZ_, TY_, (A != 0)>}
const Variant2 kVariants2[] = {
    // small learnable filters (3 taps per axis) and gaussian_blur of volumes:
    // one width per radius 1..9 (sigma 0.5 .. 3)
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 3, 3, 3, 16),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 3, 3, 1, 24),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 5, 5, 5, 16),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 7, 7, 7, 16),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 11, 11, 11, 16),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 13, 13, 13, 16),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 15, 15, 15, 16),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 17, 17, 17, 16),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 19, 19, 19, 16),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 9, 9, 9, 16),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 13, 13, 1, 16),
    // gaussian_blur of 2-D images: every width from radius 2 to 12 (sigma 0.5 to 4);
    // 16-row tiles (4 CTAs per SM) up to 17 taps, 24-row tiles beyond (measured)
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 5, 5, 1, 16),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 7, 7, 1, 16),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 9, 9, 1, 16),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 11, 11, 1, 16),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 15, 15, 1, 16),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 17, 17, 1, 16),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 19, 19, 1, 24),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 21, 21, 1, 24),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 23, 23, 1, 24),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 25, 25, 1, 24),
    NDLGPU_V2(0, float, float, NDLGPU_F32, NDLGPU_F32, 17, 17, 11, 16),
    NDLGPU_V2(0, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 17, 17, 11, 16),
    // 16-bit storage: gaussian_blur of volumes (5..13 taps) and images (5..25 taps)
    NDLGPU_V2(0, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 5, 5, 5, 16),
    NDLGPU_V2(0, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 7, 7, 7, 16),
    NDLGPU_V2(0, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 9, 9, 9, 16),
    NDLGPU_V2(0, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 11, 11, 11, 16),
    NDLGPU_V2(0, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 13, 13, 13, 16),
    NDLGPU_V2(0, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 5, 5, 1, 16),
    NDLGPU_V2(0, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 7, 7, 1, 16),
    NDLGPU_V2(0, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 9, 9, 1, 16),
    NDLGPU_V2(0, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 11, 11, 1, 16),
    NDLGPU_V2(0, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 13, 13, 1, 16),
    NDLGPU_V2(0, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 15, 15, 1, 16),
    NDLGPU_V2(0, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 17, 17, 1, 16),
    NDLGPU_V2(0, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 19, 19, 1, 24),
    NDLGPU_V2(0, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 21, 21, 1, 24),
    NDLGPU_V2(0, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 23, 23, 1, 24),
    NDLGPU_V2(0, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 25, 25, 1, 24),
    NDLGPU_V2(0, __half, __half, NDLGPU_F16, NDLGPU_F16, 5, 5, 5, 16),
    NDLGPU_V2(0, __half, __half, NDLGPU_F16, NDLGPU_F16, 7, 7, 7, 16),
    NDLGPU_V2(0, __half, __half, NDLGPU_F16, NDLGPU_F16, 9, 9, 9, 16),
    NDLGPU_V2(0, __half, __half, NDLGPU_F16, NDLGPU_F16, 11, 11, 11, 16),
    NDLGPU_V2(0, __half, __half, NDLGPU_F16, NDLGPU_F16, 13, 13, 13, 16),
    NDLGPU_V2(0, __half, __half, NDLGPU_F16, NDLGPU_F16, 5, 5, 1, 16),
    NDLGPU_V2(0, __half, __half, NDLGPU_F16, NDLGPU_F16, 7, 7, 1, 16),
    NDLGPU_V2(0, __half, __half, NDLGPU_F16, NDLGPU_F16, 9, 9, 1, 16),
    NDLGPU_V2(0, __half, __half, NDLGPU_F16, NDLGPU_F16, 11, 11, 1, 16),
    NDLGPU_V2(0, __half, __half, NDLGPU_F16, NDLGPU_F16, 13, 13, 1, 16),
    NDLGPU_V2(0, __half, __half, NDLGPU_F16, NDLGPU_F16, 15, 15, 1, 16),
    NDLGPU_V2(0, __half, __half, NDLGPU_F16, NDLGPU_F16, 17, 17, 1, 16),
    NDLGPU_V2(0, __half, __half, NDLGPU_F16, NDLGPU_F16, 19, 19, 1, 24),
    NDLGPU_V2(0, __half, __half, NDLGPU_F16, NDLGPU_F16, 21, 21, 1, 24),
    NDLGPU_V2(0, __half, __half, NDLGPU_F16, NDLGPU_F16, 23, 23, 1, 24),
    NDLGPU_V2(0, __half, __half, NDLGPU_F16, NDLGPU_F16, 25, 25, 1, 24),
    NDLGPU_V2(0, __half, __half, NDLGPU_F16, NDLGPU_F16, 17, 17, 11, 16),
    NDLGPU_V2(1, float, float, NDLGPU_F32, NDLGPU_F32, 9, 9, 9, 16),
    // input gradients of small filters (3-13 taps per axis on volumes, 3-17 on images)
    NDLGPU_V2(1, float, float, NDLGPU_F32, NDLGPU_F32, 3, 3, 3, 16),
    NDLGPU_V2(1, float, float, NDLGPU_F32, NDLGPU_F32, 5, 5, 5, 16),
    NDLGPU_V2(1, float, float, NDLGPU_F32, NDLGPU_F32, 7, 7, 7, 16),
    NDLGPU_V2(1, float, float, NDLGPU_F32, NDLGPU_F32, 11, 11, 11, 16),
    NDLGPU_V2(1, float, float, NDLGPU_F32, NDLGPU_F32, 13, 13, 13, 16),
    NDLGPU_V2(1, float, float, NDLGPU_F32, NDLGPU_F32, 3, 3, 1, 24),
    NDLGPU_V2(1, float, float, NDLGPU_F32, NDLGPU_F32, 5, 5, 1, 24),
    NDLGPU_V2(1, float, float, NDLGPU_F32, NDLGPU_F32, 7, 7, 1, 24),
    NDLGPU_V2(1, float, float, NDLGPU_F32, NDLGPU_F32, 9, 9, 1, 24),
    NDLGPU_V2(1, float, float, NDLGPU_F32, NDLGPU_F32, 11, 11, 1, 24),
    NDLGPU_V2(1, float, float, NDLGPU_F32, NDLGPU_F32, 15, 15, 1, 24),
    NDLGPU_V2(1, float, float, NDLGPU_F32, NDLGPU_F32, 17, 17, 1, 24),
    NDLGPU_V2(1, float, float, NDLGPU_F32, NDLGPU_F32, 13, 13, 1, 24),
    NDLGPU_V2(1, float, float, NDLGPU_F32, NDLGPU_F32, 17, 17, 11, 16),
    NDLGPU_V2(1, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 17, 17, 11, 16),
    NDLGPU_V2(1, __half, __half, NDLGPU_F16, NDLGPU_F16, 17, 17, 11, 16),
    // 16-bit input gradients of small volume filters
    NDLGPU_V2(1, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 3, 3, 3, 16),
    NDLGPU_V2(1, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 5, 5, 5, 16),
    NDLGPU_V2(1, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 7, 7, 7, 16),
    NDLGPU_V2(1, __nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 9, 9, 9, 16),
    NDLGPU_V2(1, __half, __half, NDLGPU_F16, NDLGPU_F16, 3, 3, 3, 16),
    NDLGPU_V2(1, __half, __half, NDLGPU_F16, NDLGPU_F16, 5, 5, 5, 16),
    NDLGPU_V2(1, __half, __half, NDLGPU_F16, NDLGPU_F16, 7, 7, 7, 16),
    NDLGPU_V2(1, __half, __half, NDLGPU_F16, NDLGPU_F16, 9, 9, 9, 16),
};
#undef NDLGPU_V2

}  // namespace

bool fused2_supported(int sdt, int ddt, int kx, int ky, int kz, int adj)
{
    for (const Variant2& v : kVariants2)
        if (v.adj == adj && v.sdt == sdt && v.ddt == ddt && v.kx == kx && v.ky == ky && v.kz == kz) return true;
    return false;
}

cudaError_t set_tma_wait_test(int spins, unsigned tx_bias)
{
    cudaError_t e = cudaMemcpyToSymbol(g_tma_wait_spins, &spins, sizeof(int));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(g_tma_tx_bias, &tx_bias, sizeof(unsigned));
}

cudaError_t read_guard_fused(int32_t* v)
{
    int32_t zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(v, g_guard_fused, sizeof(int32_t));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(g_guard_fused, &zero, sizeof(int32_t));
}

cudaError_t launch_fused2(const FusedParams& p, cudaStream_t s)
{
    for (const Variant2& v : kVariants2)
        if (v.adj == (p.adj ? 1 : 0) && v.sdt == p.src_dtype && v.ddt == p.dst_dtype && v.kx == p.kx &&
            v.ky == p.ky && v.kz == p.kz) {
            if (p.nx <= 0 || p.ny <= 0 || p.nz <= 0 || p.nbatch <= 0) return cudaSuccess;
            return v.fn(p, s);
        }
    return cudaErrorNotSupported;
}

}  // namespace ndlgpu
