// fwd3.cu -- fused separable forward of a volume (three 1-D passes) for
// float storage (f32 / bf16 / f16 in and out, FP32 accumulation): one HBM
// read and one write per element.
//
// A CTA owns a 64 x 16 column tile of one batch item and streams a chunk of
// Z planes (2.5-D blocking).  The passes run Y first, so that every pass is
// a packed pair of FP32 multiply-adds and the X pass computes no halo rows:
//   load  : plane zi (border-mapped along Z) with its X/Y halos goes to a
//           3-stage shared-memory ring two planes ahead of the compute.
//           Where the rows are 16-byte aligned, the tile width divides the
//           extent and the border is Clamp or Reflect, one thread issues one
//           tensor-map box per plane (cp.async.bulk.tensor, no multicast)
//           completing on an mbarrier; the halo elements outside the image
//           (zero-filled by the copy engine) are then rewritten from their
//           border-mapped source inside the box.  Otherwise (Wrap, ragged
//           or unaligned rows) cp.async: rows border-mapped as whole rows,
//           the columns outside [0, nx) and ragged 16-byte chunks element by
//           element from their border-mapped column.
//   Y pass: 4 rows x 1 column pair per unit, pairs of adjacent columns
//           packed; results go to shared memory with the rows of a pair
//           interleaved (element (r, c) at [r/2][c][r%2]).
//   X pass: 2 rows x 4 columns per thread from that interleaved tile, the
//           two rows packed.
//   Z pass: a KZ-deep register queue of those row pairs; the slot of the
//           newest plane rotates and is read through a compile-time slot
//           dispatch, so that no value is ever moved.
// Border maps are Clamp / Wrap / Reflect of mathHelpers.h:23-25, applied to
// load coordinates only.  Taps are summed in the same order as the
// reference's per-axis convolve (processing/convolution.h:64-70), in FP32.
// Every mbarrier wait is bounded: on timeout the CTA sets bit 1 of its guard
// word, lets its copies in flight land (bounded) and returns.
#include <algorithm>
#include <cstring>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "dtype.cuh"

namespace ndlgpu {
namespace {

constexpr int TX = 64;
constexpr int TY = 16;
constexpr int NT = 128;
constexpr int STAGES = 3;

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

__device__ int32_t g_guard_fwd3;                     // bit 1: a plane wait ran past its bound
constexpr int kSpins3 = 1 << 22;                      // bound on the mbarrier polls for one plane
// Test controls (ndlgpu_test_wait_timeouts), as for the other tensor-map
// plane loads: the poll bound, and bytes announced but never delivered.
__device__ int g_wait_spins3 = kSpins3;
__device__ unsigned g_tx_bias3 = 0;

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
__device__ __forceinline__ void mbar_complete_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.complete_tx.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
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
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, "
        "%6}], [%2];\n" ::"r"(smem_u32(dst)),
        "l"(map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}

// two adjacent shared-memory elements as a float pair
__device__ __forceinline__ float2 lds2(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ float2 lds2(const __nv_bfloat16* p)
{
    const unsigned t = *reinterpret_cast<const unsigned*>(p);
    return make_float2(__uint_as_float(t << 16), __uint_as_float(t & 0xffff0000u));
}
__device__ __forceinline__ float2 lds2(const __half* p)
{
    return __half22float2(*reinterpret_cast<const __half2*>(p));
}

template <class T> __device__ __forceinline__ T from_f(float v);
template <> __device__ __forceinline__ float from_f<float>(float v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ __half from_f<__half>(float v) { return __float2half_rn(v); }

__device__ __forceinline__ void stg4(float* p, float a, float b, float c, float d)
{
    *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
}
__device__ __forceinline__ void stg4(__nv_bfloat16* p, float a, float b, float c, float d)
{
    __nv_bfloat162 u = __floats2bfloat162_rn(a, b), v = __floats2bfloat162_rn(c, d);
    uint2 t;
    t.x = *reinterpret_cast<unsigned*>(&u);
    t.y = *reinterpret_cast<unsigned*>(&v);
    *reinterpret_cast<uint2*>(p) = t;
}
__device__ __forceinline__ void stg4(__half* p, float a, float b, float c, float d)
{
    __half2 u = __floats2half2_rn(a, b), v = __floats2half2_rn(c, d);
    uint2 t;
    t.x = *reinterpret_cast<unsigned*>(&u);
    t.y = *reinterpret_cast<unsigned*>(&v);
    *reinterpret_cast<uint2*>(p) = t;
}

template <class Tin, int KX, int KY>
struct G3 {
    static constexpr int EPC = 16 / (int)sizeof(Tin);        // elements per 16-byte chunk
    static constexpr int CX = KX / 2;
    static constexpr int CY = KY / 2;
    static constexpr int HX = (CX + 1) & ~1;                  // Y-pass halo columns per side (even)
    static constexpr int WO = HX - CX;                        // X window offset (0 or 1 column)
    static constexpr int YC = TX + 2 * HX;                    // Y-pass columns
    static constexpr int YCP = YC / 2;                        // ... in pairs
    static_assert(NT == 128 && TY == 16 && YCP >= 32 && 4 * (YCP - 32) <= NT, "Y-pass unit mapping");
    static constexpr int D = (EPC - HX % EPC) % EPC;          // ring column of global x0 - HX
    static constexpr int ROWS = TY + KY - 1;
    static constexpr int NCH = (D + YC + EPC - 1) / EPC;      // 16-byte chunks per ring row
    static constexpr int PITCH = NCH * EPC + (sizeof(Tin) == 4 ? 4 : 8);   // + a bank shift per row
    static constexpr int NTASK = (ROWS * NCH + NT - 1) / NT;
    // floats per interleaved row pair, = 4 (mod 32): the two row pairs a
    // quarter-warp of the X pass reads then fall on disjoint banks
    static constexpr int YPITCH = 2 * YC + ((4 - (2 * YC) % 32) + 32) % 32;
    static constexpr int NW = (WO + 3 + KX + 1) / 2;          // float4 loads per X window
    static constexpr size_t STAGE = (size_t)ROWS * PITCH;      // elements per ring stage
    static constexpr bool TMA_OK = (STAGE * sizeof(Tin)) % 128 == 0 && PITCH <= 256 && ROWS <= 256;
    static constexpr size_t IN_BYTES = STAGES * STAGE * sizeof(Tin);
    static constexpr size_t Y_BYTES = (size_t)(TY / 2) * YPITCH * 4;
    static constexpr int MAXEL = ROWS * NCH * EPC;            // table bound: every ring element once
    static constexpr size_t TAB_BYTES = (size_t)MAXEL * 8;
    static constexpr size_t SMEM = IN_BYTES + Y_BYTES + TAB_BYTES + 16 + 128;   // + alignment slack
};

// Loads one plane (border-mapped along Z) into a ring stage by cp.async:
// the 16-byte chunks this thread owns, then its share of the element table.
template <class Tin, int NTASK, size_t STAGE>
struct PlaneLoader3 {
    const Tin* src;
    Tin* s_in;
    const int2* s_tab;
    int ntab, tid, border, nz;
    int64_t sz;
    int32_t goff[NTASK];
    unsigned sadr[NTASK];

    __device__ __forceinline__ void issue(int zi, int stage) const
    {
        const unsigned sbo = (unsigned)(stage * STAGE * sizeof(Tin));
        const int zm = map_border32(border, nz, zi);
        const Tin* pl = src + (int64_t)zm * sz;
#pragma unroll
        for (int j = 0; j < NTASK; j++)
            if (goff[j] >= 0)
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sadr[j] + sbo), "l"(pl + goff[j])
                             : "memory");
        for (int i = tid; i < ntab; i += NT) {
            const int2 e = s_tab[i];
            if constexpr (sizeof(Tin) == 4) cp_async4(s_in + stage * STAGE + e.x, pl + e.y);
            else s_in[stage * STAGE + e.x] = pl[e.y];
        }
    }
};

// Output plane of the Z queue for the newest slot S: tap k reads slot
// (S + 1 + k) mod KZ (the queue holds the last KZ planes in ring order).
template <int KZ, int S>
__device__ __forceinline__ void zstep3(float2 (&q)[KZ][4], const float2 (&xv)[4], float2 (&out)[4],
                                       const float2 (&wz)[KZ])
{
#pragma unroll
    for (int e = 0; e < 4; e++) q[S][e] = xv[e];
#pragma unroll
    for (int e = 0; e < 4; e++) {
        float2 a = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < KZ; k++) a = __ffma2_rn(q[(S + 1 + k) % KZ][e], wz[k], a);
        out[e] = a;
    }
}

template <int KZ>
__device__ __forceinline__ void zdispatch3(int slot, float2 (&q)[KZ][4], const float2 (&xv)[4], float2 (&out)[4],
                                           const float2 (&wz)[KZ])
{
#define NDLGPU_Z3(S)                                                              \
    case S:                                                                       \
        if constexpr (S < KZ) zstep3<KZ, (S < KZ ? S : 0)>(q, xv, out, wz);       \
        break;
    switch (slot) {
        NDLGPU_Z3(0) NDLGPU_Z3(1) NDLGPU_Z3(2) NDLGPU_Z3(3) NDLGPU_Z3(4) NDLGPU_Z3(5) NDLGPU_Z3(6)
        NDLGPU_Z3(7) NDLGPU_Z3(8) NDLGPU_Z3(9) NDLGPU_Z3(10) NDLGPU_Z3(11) NDLGPU_Z3(12) NDLGPU_Z3(13)
        NDLGPU_Z3(14) NDLGPU_Z3(15) NDLGPU_Z3(16) NDLGPU_Z3(17) NDLGPU_Z3(18)
    default: break;
    }
#undef NDLGPU_Z3
}

// CTAs per SM: the Z queue holds 8 KZ registers per thread.
template <int KZ>
struct Occ3 {
    static constexpr int value = KZ > 13 ? 2 : (KZ > 9 ? 3 : 4);
};

template <class Tin, class Tout, int KX, int KY, int KZ, bool TMA>
__global__ void __launch_bounds__(NT, Occ3<KZ>::value)
    k_fwd3(const __grid_constant__ FusedParams p, const __grid_constant__ CUtensorMap tmap)
{
    using G = G3<Tin, KX, KY>;
    extern __shared__ __align__(128) unsigned char smem3_raw[];
    __shared__ uint64_t s_bar[STAGES];
    unsigned char* smem3 = smem3_raw + ((128u - (smem_u32(smem3_raw) & 127u)) & 127u);
    Tin* s_in = reinterpret_cast<Tin*>(smem3);
    float* s_y = reinterpret_cast<float*>(smem3 + G::IN_BYTES);
    int2* s_tab = reinterpret_cast<int2*>(smem3 + G::IN_BYTES + G::Y_BYTES);
    int* s_ntab = reinterpret_cast<int*>(smem3 + G::IN_BYTES + G::Y_BYTES + G::TAB_BYTES);

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
    const int gx0 = x0 - G::HX - G::D;   // global column of ring column 0 (a multiple of EPC)

    if (tid == 0) {
        *s_ntab = 0;
        if constexpr (TMA) {
            for (int st = 0; st < STAGES; st++) mbar_init(&s_bar[st], 1);
            fence_mbar_init();
        }
    }
    __syncthreads();
    PlaneLoader3<Tin, G::NTASK, G::STAGE> ld;
    ld.src = src;
    ld.s_in = s_in;
    ld.s_tab = s_tab;
    ld.tid = tid;
    ld.border = p.border;
    ld.nz = p.nz;
    ld.sz = p.sz;
    if constexpr (TMA) {
        // ring elements outside the image that a kept output reads get
        // their border-mapped source inside the box (always an element of
        // the image, so one pass serves the corners)
        const bool ytile = y0 < G::CY || y0 + TY + G::CY > p.ny;
        const bool xtile = x0 < G::HX || x0 + TX + G::HX > p.nx;
        if (ytile || xtile) {
            for (int i = tid; i < G::ROWS * G::YC; i += NT) {
                const int r = i / G::YC, c = G::D + (i - (i / G::YC) * G::YC);
                const int y = y0 - G::CY + r, x = gx0 + c;
                if (y >= 0 && y < p.ny && x >= 0 && x < p.nx) continue;
                if (y >= p.ny + G::CY || x < -G::CX || x >= p.nx + G::CX) continue;   // read by no kept output
                const int ys = map_border32(p.border, p.ny, y), xs = map_border32(p.border, p.nx, x);
                const int slot_i = atomicAdd(s_ntab, 1);
                s_tab[slot_i] = make_int2(r * G::PITCH + c, (ys - (y0 - G::CY)) * G::PITCH + (xs - gx0));
            }
        }
    } else {
        // Chunk t = tid + j*NT covers ring row t / NCH, columns
        // [q*EPC, (q+1)*EPC).  A chunk inside [0, nx) on a 16-byte aligned
        // row is one 16-byte copy (offsets kept in registers); every other
        // element goes to a shared table of (ring offset, in-plane source
        // offset) pairs with its column border-mapped.
        const unsigned s_in_u = smem_u32(s_in);
#pragma unroll
        for (int j = 0; j < G::NTASK; j++) {
            const int t = tid + j * NT;
            ld.goff[j] = -1;
            ld.sadr[j] = s_in_u;
            if (t >= G::ROWS * G::NCH) continue;
            const int r = t / G::NCH;
            const int q = t - r * G::NCH;
            int y = y0 - G::CY + r;
            const int cx0 = gx0 + q * G::EPC;
            // rows past the last tile row are never read by a kept output
            y = (y >= p.ny + G::CY) ? p.ny - 1 : map_border32(p.border, p.ny, y);
            const int32_t rowoff = (int32_t)(y * p.sy);
            if (p.vec_ld && cx0 >= 0 && cx0 + G::EPC <= p.nx) {
                ld.goff[j] = rowoff + cx0;
                ld.sadr[j] = s_in_u + (unsigned)((r * G::PITCH + q * G::EPC) * (int)sizeof(Tin));
            } else {
                for (int e = 0; e < G::EPC; e++) {
                    int x = cx0 + e;
                    x = (x >= p.nx + G::CX || x < -G::CX) ? p.nx - 1 : map_border32(p.border, p.nx, x);
                    const int slot_i = atomicAdd(s_ntab, 1);
                    s_tab[slot_i] = make_int2(r * G::PITCH + q * G::EPC + e, rowoff + (int32_t)(x * p.sx));
                }
            }
        }
    }
    __syncthreads();
    const int ntab = *s_ntab;   // table entries: copies (cp.async) or halo fix-ups (tensor map)
    ld.ntab = ntab;

    const int zin0 = zs - CZ;
    const int zin1 = ze - 1 + HZ;
    const int nplanes = zin1 - zin0 + 1;
    const int tpos0 = p.tma_pos[0], tpos1 = p.tma_pos[1];
    unsigned tx_bias = 0;
    int wait_spins = kSpins3;
    if constexpr (TMA) {
        tx_bias = g_tx_bias3;
        wait_spins = g_wait_spins3;
    }
    auto issue_tma = [&](int zi, int st) {
        const int zc = map_border32(ld.border, ld.nz, zi);
        const int yc = y0 - G::CY;
        const int c1 = tpos0 == 0 ? yc : (tpos1 == 0 ? zc : bat);
        const int c2 = tpos0 == 1 ? yc : (tpos1 == 1 ? zc : bat);
        const int c3 = tpos0 == 2 ? yc : (tpos1 == 2 ? zc : bat);
        fence_proxy_async();
        mbar_expect_tx(&s_bar[st], (unsigned)(G::STAGE * sizeof(Tin)) + tx_bias);
        tma_load_4d(s_in + st * G::STAGE, &tmap, &s_bar[st], gx0, c1, c2, c3);
    };
#pragma unroll
    for (int s = 0; s < STAGES - 1; s++) {
        if constexpr (TMA) {
            if (tid == 0 && s < nplanes) issue_tma(zin0 + s, s);
        } else {
            if (s < nplanes) ld.issue(zin0 + s, s);
            cp_async_commit();
        }
    }

    // X/Z role of this thread: lane l of warp w has columns 4 xg.. with
    // xg = 4 w + (l & 3) and row pair xr = 2 (l >> 3) + ((l >> 2) & 1); each
    // quarter-warp reads 4 column groups of 2 row pairs (conflict-free with
    // the interleaved pitch)
    const int xg = ((tid >> 5) << 2) | (tid & 3);
    const int xr = (((tid & 31) >> 3) << 1) | ((tid >> 2) & 1);
    float2 q[KZ][4];
#pragma unroll
    for (int k = 0; k < KZ; k++)
#pragma unroll
        for (int e = 0; e < 4; e++) q[k][e] = make_float2(0.f, 0.f);
    int slot = 0;
    int stage = 0;
    int stage_next = STAGES - 1;
    unsigned phase = 0;   // mbarrier parity of the current pass over the ring
    const int xb = x0 + 4 * xg;
    const int ya = y0 + 2 * xr;
    const bool row0 = ya < p.ny, row1 = ya + 1 < p.ny;
    const bool vst = p.vec_st && xb + 4 <= p.nx;
    Tout* orow0 = dst + (int64_t)ya * p.dy + (int64_t)xb * p.dx;
    Tout* orow1 = orow0 + p.dy;
    int64_t oz = (int64_t)(zin0 + KZ - 1 - HZ) * p.dz;

    for (int n = 0; n < nplanes; n++) {
        if constexpr (TMA) {
            bool ok = false;
            for (int i = 0; i < wait_spins && !ok; i++) ok = mbar_try_wait(&s_bar[stage], phase);
            // plane n visible; every thread is past the X pass of plane n-1
            if (__syncthreads_or(!ok)) {
                if (tid == 0) {
                    atomicOr(&g_guard_fwd3, 2);
                    // planes n .. n+STAGES-2 may still be landing in this
                    // CTA's ring: retire the announced surplus (test
                    // control) and wait, bounded, for each before the CTA
                    // lets go of its shared memory.  Plane m sits in stage
                    // m % STAGES with parity (m / STAGES) & 1.
                    for (int m = n; m < min(n + STAGES - 1, nplanes); m++) {
                        uint64_t* bar = &s_bar[m % STAGES];
                        if (tx_bias) mbar_complete_tx(bar, tx_bias);
                        const unsigned par = (unsigned)(m / STAGES) & 1u;
                        for (int i = 0; i < kSpins3 && !mbar_try_wait(bar, par); i++) {
                        }
                    }
                }
                return;
            }
            if (stage + 1 == STAGES) phase ^= 1u;
            if (tid == 0 && n + STAGES - 1 < nplanes) issue_tma(zin0 + n + STAGES - 1, stage_next);
            if (ntab > 0) {
                // border halo: border-mapped sources inside the box
                Tin* sbf = s_in + stage * G::STAGE;
                for (int i = tid; i < ntab; i += NT) {
                    const int2 e = s_tab[i];
                    sbf[e.x] = sbf[e.y];
                }
                __syncthreads();
            }
        } else {
            cp_async_wait<STAGES - 2>();
            __syncthreads();    // plane n visible; every thread is past the X pass of plane n-1
            if (n + STAGES - 1 < nplanes) ld.issue(zin0 + n + STAGES - 1, stage_next);
            cp_async_commit();
        }
        stage_next = (stage_next + 1 == STAGES) ? 0 : stage_next + 1;

        // Y pass: first sweep, warp w = row quad w, lane = column pair (the
        // first 64 of the YC columns); second sweep, the last 2 HX columns'
        // pairs, by the first 4 HX threads
        const Tin* sb = s_in + stage * G::STAGE + G::D;
#pragma unroll
        for (int i = 0; i < 2; i++) {
            if (i == 1 && tid >= 4 * (G::YCP - 32)) break;
            const int rq = i == 0 ? (tid >> 5) : (tid & 3);
            const int cp = i == 0 ? (tid & 31) : 32 + (tid >> 2);
            const Tin* col = sb + (4 * rq) * G::PITCH + 2 * cp;
            float2 a[4] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f),
                           make_float2(0.f, 0.f)};
#pragma unroll
            for (int j = 0; j < KY + 3; j++) {
                const float2 v = lds2(col + j * G::PITCH);
#pragma unroll
                for (int r = 0; r < 4; r++)
                    if (j - r >= 0 && j - r < KY) a[r] = __ffma2_rn(v, p.wy2[j - r], a[r]);
            }
            float* yo = s_y + (2 * rq) * G::YPITCH + 4 * cp;
            *reinterpret_cast<float4*>(yo) = make_float4(a[0].x, a[1].x, a[0].y, a[1].y);
            *reinterpret_cast<float4*>(yo + G::YPITCH) = make_float4(a[2].x, a[3].x, a[2].y, a[3].y);
        }
        __syncthreads();
        // X pass: rows 2xr, 2xr+1 packed, output columns 4xg .. 4xg+3
        float2 xv[4];
        {
            const float* wrow = s_y + xr * G::YPITCH + 8 * xg;
            float2 win[2 * G::NW];
#pragma unroll
            for (int v = 0; v < G::NW; v++) {
                const float4 t = *reinterpret_cast<const float4*>(wrow + 4 * v);
                win[2 * v] = make_float2(t.x, t.y);
                win[2 * v + 1] = make_float2(t.z, t.w);
            }
#pragma unroll
            for (int m = 0; m < 4; m++) {
                float2 a = make_float2(0.f, 0.f);
#pragma unroll
                for (int k = 0; k < KX; k++) a = __ffma2_rn(win[G::WO + m + k], p.wx2[k], a);
                xv[m] = a;
            }
        }
        // Z pass (the taps in registers for the step)
        float2 o[4];
        {
            float2 wz[KZ];
#pragma unroll
            for (int k = 0; k < KZ; k++) wz[k] = p.wz2[k];
            zdispatch3<KZ>(slot, q, xv, o, wz);
            slot = (slot + 1 == KZ) ? 0 : slot + 1;
        }
        stage = (stage + 1 == STAGES) ? 0 : stage + 1;
        if (n >= KZ - 1) {
            if (vst) {
                if (row0) stg4(orow0 + oz, o[0].x, o[1].x, o[2].x, o[3].x);
                if (row1) stg4(orow1 + oz, o[0].y, o[1].y, o[2].y, o[3].y);
            } else {
                const float v0[4] = {o[0].x, o[1].x, o[2].x, o[3].x};
                const float v1[4] = {o[0].y, o[1].y, o[2].y, o[3].y};
#pragma unroll
                for (int m = 0; m < 4; m++) {
                    if (xb + m >= p.nx) break;
                    if (row0) orow0[oz + (int64_t)m * p.dx] = from_f<Tout>(v0[m]);
                    if (row1) orow1[oz + (int64_t)m * p.dx] = from_f<Tout>(v1[m]);
                }
            }
            oz += p.dz;
        }
    }
    if constexpr (!TMA) cp_async_wait<0>();
}

using LaunchFn3 = cudaError_t (*)(const FusedParams&, cudaStream_t);

PFN_cuTensorMapEncodeTiled_v12000 encoder3()
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

template <class T> constexpr CUtensorMapDataType tma_type3();
template <> constexpr CUtensorMapDataType tma_type3<float>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT32; }
template <> constexpr CUtensorMapDataType tma_type3<__nv_bfloat16>() { return CU_TENSOR_MAP_DATA_TYPE_BFLOAT16; }
template <> constexpr CUtensorMapDataType tma_type3<__half>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT16; }

// A 4-D tiled map of the source -- x, then y, z and batch in increasing
// stride order -- with a box of boxx columns x boxy rows of one plane;
// p.tma_pos gets the map dimension (0..2 after x) of y, z and batch.  False
// where the plane loads keep cp.async: Wrap (its halo comes from the far
// side of the image, outside the box), a tile width that does not divide the
// extent (boxes mostly outside the image measured 7-13x slower), unaligned,
// non-unit-stride or negative-stride sources.
template <class Tin>
bool plane_map3(FusedParams& p, int boxx, int boxy, CUtensorMap* m)
{
    if (p.adj || !p.vec_ld || p.sx != 1 || p.nx % TX != 0 || p.border == NDLGPU_WRAP) return false;
    if (reinterpret_cast<uintptr_t>(p.src) % 16 != 0) return false;
    PFN_cuTensorMapEncodeTiled_v12000 enc = encoder3();
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
    const CUresult r = enc(m, tma_type3<Tin>(), 4, const_cast<char*>(p.src), gdim, gstr, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

template <class Tin, class Tout, int KX, int KY, int KZ>
cudaError_t launch3(const FusedParams& p, cudaStream_t s)
{
    using G = G3<Tin, KX, KY>;
    static_assert(G::SMEM <= 227 * 1024, "shared memory");
    static bool configured[2] = {false, false};
    FusedParams pp = p;
    CUtensorMap tmap;
    std::memset(&tmap, 0, sizeof(tmap));
    bool tma = false;
    auto kern = k_fwd3<Tin, Tout, KX, KY, KZ, false>;
    if constexpr (G::TMA_OK) {
        tma = plane_map3<Tin>(pp, G::PITCH, G::ROWS, &tmap);
        if (tma) kern = k_fwd3<Tin, Tout, KX, KY, KZ, true>;
    }
    if (!configured[tma]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM);
        if (e != cudaSuccess) return e;
        configured[tma] = true;
    }
    const int ntx = (p.nx + TX - 1) / TX;
    const int nty = (p.ny + TY - 1) / TY;
    const long long gx = (long long)ntx * nty * p.nbatch;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long slots = (long long)sms * Occ3<KZ>::value;
    const int chunks = pick_zchunks(gx, slots, p.nz, KZ - 1);
    pp.zchunk = max(1, (p.nz + chunks - 1) / chunks);
    const int gz = (p.nz + pp.zchunk - 1) / pp.zchunk;
    if (gx > 0x7fffffffLL || gz > 65535) return cudaErrorInvalidConfiguration;
    kern<<<dim3((unsigned)gx, (unsigned)gz), NT, G::SMEM, s>>>(pp, tmap);
    count_launch();
    return cudaGetLastError();
}

struct Variant3 {
    int sdt, ddt, kx, ky, kz;
    LaunchFn3 fn;
};

#define NDLGPU_V3(TI, TO, DI, DO, KX_, KY_, KZ_) {DI, DO, KX_, KY_, KZ_, &launch3<TI, TO, KX_, KY_, KZ_>}
const Variant3 kVariants3[] = {
    // learnable filters and gaussian_blur of volumes (one width per radius
    // 1..9), the 4-D video (17 x 17 x 11), 16-bit storage
    NDLGPU_V3(float, float, NDLGPU_F32, NDLGPU_F32, 9, 9, 9),
    NDLGPU_V3(float, float, NDLGPU_F32, NDLGPU_F32, 3, 3, 3),
    NDLGPU_V3(float, float, NDLGPU_F32, NDLGPU_F32, 5, 5, 5),
    NDLGPU_V3(float, float, NDLGPU_F32, NDLGPU_F32, 7, 7, 7),
    NDLGPU_V3(float, float, NDLGPU_F32, NDLGPU_F32, 11, 11, 11),
    NDLGPU_V3(float, float, NDLGPU_F32, NDLGPU_F32, 13, 13, 13),
    NDLGPU_V3(float, float, NDLGPU_F32, NDLGPU_F32, 15, 15, 15),
    NDLGPU_V3(float, float, NDLGPU_F32, NDLGPU_F32, 17, 17, 17),
    NDLGPU_V3(float, float, NDLGPU_F32, NDLGPU_F32, 19, 19, 19),
    NDLGPU_V3(float, float, NDLGPU_F32, NDLGPU_F32, 17, 17, 11),
    NDLGPU_V3(__nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 17, 17, 11),
    NDLGPU_V3(__half, __half, NDLGPU_F16, NDLGPU_F16, 17, 17, 11),
    NDLGPU_V3(__nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 5, 5, 5),
    NDLGPU_V3(__nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 7, 7, 7),
    NDLGPU_V3(__nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 9, 9, 9),
    NDLGPU_V3(__nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 11, 11, 11),
    NDLGPU_V3(__nv_bfloat16, __nv_bfloat16, NDLGPU_BF16, NDLGPU_BF16, 13, 13, 13),
    NDLGPU_V3(__half, __half, NDLGPU_F16, NDLGPU_F16, 5, 5, 5),
    NDLGPU_V3(__half, __half, NDLGPU_F16, NDLGPU_F16, 7, 7, 7),
    NDLGPU_V3(__half, __half, NDLGPU_F16, NDLGPU_F16, 9, 9, 9),
    NDLGPU_V3(__half, __half, NDLGPU_F16, NDLGPU_F16, 11, 11, 11),
    NDLGPU_V3(__half, __half, NDLGPU_F16, NDLGPU_F16, 13, 13, 13),
};
#undef NDLGPU_V3

}  // namespace

cudaError_t read_guard_fwd3(int32_t* v)
{
    int32_t zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(v, g_guard_fwd3, sizeof(int32_t));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(g_guard_fwd3, &zero, sizeof(int32_t));
}

cudaError_t set_fwd3_wait_test(int spins, unsigned tx_bias)
{
    cudaError_t e = cudaMemcpyToSymbol(g_wait_spins3, &spins, sizeof(int));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(g_tx_bias3, &tx_bias, sizeof(unsigned));
}

bool fwd3_supported(int sdt, int ddt, int kx, int ky, int kz)
{
    for (const Variant3& v : kVariants3)
        if (v.sdt == sdt && v.ddt == ddt && v.kx == kx && v.ky == ky && v.kz == kz) return true;
    return false;
}

cudaError_t launch_fwd3(const FusedParams& p, cudaStream_t s)
{
    if (p.adj) return cudaErrorNotSupported;
    for (const Variant3& v : kVariants3)
        if (v.sdt == p.src_dtype && v.ddt == p.dst_dtype && v.kx == p.kx && v.ky == p.ky && v.kz == p.kz) {
            if (p.nx <= 0 || p.ny <= 0 || p.nz <= 0 || p.nbatch <= 0) return cudaSuccess;
            return v.fn(p, s);
        }
    return cudaErrorNotSupported;
}

}  // namespace ndlgpu
