// fused_u8.cu -- fused separable forward of a uint8 volume with dyadic
// integer taps (the exact integer path: every sum an integer numerator, one
// rounding at the end), packed two values to a 32-bit word.
//
// A CTA owns a 64 x 32 column tile of one batch item and streams its Z chunk
// (2.5-D blocking):
//   load  : plane zi (border-mapped along Z) with its X/Y halos: whole rows
//           border-mapped, 16-byte cp.async chunks of the bytes x0-16 ..
//           x0+79, element copies for the columns outside [0, nx) (their
//           border-mapped source) and ragged chunks; 3-stage ring.
//   Y pass: 4 columns x 1 row pair per unit from the raw bytes; the bytes
//           are widened to 16-bit lanes (two per word) and multiplied by the
//           integer taps with one 32-bit multiply-add per word; results go to
//           shared memory as words holding the two rows of a pair.
//   X pass: 4 columns x 1 row pair per thread, the same packed arithmetic
//           (a word is the row pair of one column, so every tap reads an
//           aligned word).
//   Z pass: the X-pass row pairs as packed FP32 pairs of integers in a
//           KZ-deep register queue (the slot of the newest plane rotates;
//           compile-time slot dispatch), packed FP32 multiply-adds (every
//           sum an integer below 2^23, exact), starting from the rounding's
//           half unit.
//   store : round (or truncate) the numerator once, as the reference's
//           double result would be (one FP32 multiply-add rounded down onto
//           the integer grid of [2^23, 2^24)), and stage the bytes in shared
//           memory so that 16-byte stores run along the destination's
//           contiguous axis (X, or Y for a transposed destination).
// The packed lanes hold the Y sums and the X-of-Y sums, both below 2^16 by
// the host's bound; the taps are non-negative.  Border maps are Clamp / Wrap
// / Reflect of mathHelpers.h:23-25 on load coordinates only.
#include "dtype.cuh"

namespace ndlgpu {
namespace {

constexpr int TX = 64;
constexpr int TY = 32;
constexpr int NT = 256;
constexpr int STAGES = 3;
constexpr int RP = 96;           // ring row: bytes x0-16 .. x0+79 (6 chunks)
constexpr int NCH = RP / 16;
constexpr int YW = 18;           // Y-pass words per row pair: columns x0-4 .. x0+67
constexpr int YP = 4 * YW + 4;   // ... row-pair pitch in words (+ a bank shift)

__device__ __forceinline__ void cp_async16(unsigned saddr, const void* gmem)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <int KY>
struct GU8 {
    static constexpr int CY = KY / 2;
    static constexpr int ROWS = TY + KY - 1;
    static constexpr int STAGE = ROWS * RP;                    // bytes per ring stage
    static constexpr int NTASK = (ROWS * NCH + NT - 1) / NT;
    static constexpr int MAXEL = ROWS * RP;                     // element-copy bound
    static constexpr size_t RING_B = (size_t)STAGES * STAGE;
    static constexpr size_t Y_B = (size_t)(TY / 2) * YP * 4;
    static constexpr size_t O_B = (size_t)(TX + 4) * TY;      // staged bytes (row pitch TX + 4 or TY)
    static constexpr size_t TAB_B = (size_t)MAXEL * 8;
    static constexpr size_t SMEM = RING_B + Y_B + O_B + TAB_B + 16;
};

// bytes b0 b1 of a word -> 16-bit lanes (lo), bytes b2 b3 -> (hi)
__device__ __forceinline__ unsigned lo16(unsigned w) { return __byte_perm(w, 0u, 0x4140); }
__device__ __forceinline__ unsigned hi16(unsigned w) { return __byte_perm(w, 0u, 0x4342); }

// The Z queue: q[s][m] holds the X-pass values of column 4g + m, rows 2rp
// and 2rp+1 (a packed FP32 pair), of the plane in slot s; the newest plane is
// in slot S and tap k reads slot (S + 1 + k) % KZ.  The values and every Z
// sum are integers below 2^23 (the host's bound), exact in FP32; the taps are
// the integer numerators as FP32 pairs (wz2).
// The sums start from a0 (the rounding's half unit, an integer).
template <int KZ, int S>
__device__ __forceinline__ void zstep_u8(float2 (&q)[KZ][4], const float2 (&xv)[4], float2 (&o)[4],
                                         const FusedParams& p, float2 a0)
{
#pragma unroll
    for (int m = 0; m < 4; m++) q[S][m] = xv[m];
#pragma unroll
    for (int m = 0; m < 4; m++) {
        float2 a = a0;
#pragma unroll
        for (int k = 0; k < KZ; k++) a = __ffma2_rn(q[(S + 1 + k) % KZ][m], p.wz2[k], a);
        o[m] = a;
    }
}

template <int KZ>
__device__ __forceinline__ void zdispatch_u8(int slot, float2 (&q)[KZ][4], const float2 (&xv)[4], float2 (&o)[4],
                                             const FusedParams& p, float2 a0)
{
#define NDLGPU_ZU8(S) \
    case S: if constexpr (S < KZ) zstep_u8<KZ, (S < KZ ? S : 0)>(q, xv, o, p, a0); break;
    switch (slot) {
        NDLGPU_ZU8(0) NDLGPU_ZU8(1) NDLGPU_ZU8(2) NDLGPU_ZU8(3) NDLGPU_ZU8(4) NDLGPU_ZU8(5) NDLGPU_ZU8(6)
        NDLGPU_ZU8(7) NDLGPU_ZU8(8)
    default: break;
    }
#undef NDLGPU_ZU8
}

// A packed 16-bit lane as an FP32 integer: exponent bits of 2^23 over the
// lane, minus 2^23 (exact).
__device__ __forceinline__ float2 lanes_to_f2(unsigned w)
{
    const float2 b = make_float2(__uint_as_float(__byte_perm(w, 0x4B000000u, 0x7610)),
                                 __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7632)));
    return __fadd2_rn(b, make_float2(-8388608.f, -8388608.f));
}

template <int KX, int KY, int KZ, bool TS>
__global__ void __launch_bounds__(NT, 2) k_fused_u8(const __grid_constant__ FusedParams p)
{
    using G = GU8<KY>;
    constexpr int CX = KX / 2;
    static_assert(CX <= 4 && KZ <= 9, "window and queue bounds");
    extern __shared__ __align__(16) unsigned char su8_raw[];
    unsigned char* s_in = su8_raw;
    unsigned* s_y = reinterpret_cast<unsigned*>(su8_raw + G::RING_B);
    unsigned char* s_o = su8_raw + G::RING_B + G::Y_B;
    int2* s_tab = reinterpret_cast<int2*>(su8_raw + G::RING_B + G::Y_B + G::O_B);
    __shared__ int s_ntab;

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
    const unsigned char* src = reinterpret_cast<const unsigned char*>(p.src) + (int64_t)bat * p.sb;
    unsigned char* dst = reinterpret_cast<unsigned char*>(p.dst) + (int64_t)bat * p.db;
    constexpr int CZ = KZ / 2;
    constexpr int HZ = KZ - 1 - CZ;

    // Loader set-up, once per CTA: chunk t = tid + j*NT covers ring row
    // t / NCH (image row y0 - CY + r, border-mapped), bytes [16q, 16q+16) of
    // x0 - 16 ..; a chunk inside [0, nx) is one 16-byte copy, every other
    // byte a table entry with its column border-mapped.
    if (tid == 0) s_ntab = 0;
    __syncthreads();
    int32_t goff[G::NTASK];
    unsigned sadr[G::NTASK];
    const unsigned s_in_u = (unsigned)__cvta_generic_to_shared(s_in);
#pragma unroll
    for (int j = 0; j < G::NTASK; j++) {
        const int t = tid + j * NT;
        goff[j] = -1;
        sadr[j] = s_in_u;
        if (t >= G::ROWS * NCH) continue;
        const int r = t / NCH, q = t - (t / NCH) * NCH;
        int y = y0 - G::CY + r;
        y = (y >= p.ny + G::CY) ? p.ny - 1 : map_border32(p.border, p.ny, y);
        const int32_t rowoff = (int32_t)(y * p.sy);
        const int cx0 = x0 - 16 + 16 * q;
        if (cx0 >= 0 && cx0 + 16 <= p.nx) {
            goff[j] = rowoff + cx0;
            sadr[j] = s_in_u + (unsigned)(r * RP + 16 * q);
        } else {
            for (int e = 0; e < 16; e++) {
                int x = cx0 + e;
                // bytes no kept output reads take any in-range source
                x = (x < -CX || x >= p.nx + CX) ? p.nx - 1 : map_border32(p.border, p.nx, x);
                s_tab[atomicAdd(&s_ntab, 1)] = make_int2(r * RP + 16 * q + e, rowoff + x);
            }
        }
    }
    __syncthreads();
    const int ntab = s_ntab;
    const int l_border = p.border, l_nz = p.nz;
    const int64_t l_sz = p.sz;
    // A plane's element copies: the first NEL per thread are loaded into
    // registers when the plane is issued and stored into its stage after the
    // current plane's compute (the load latency hides behind it); any beyond
    // (ragged extents only) are copied at once.
    constexpr int NEL = 3;
    unsigned ev[NEL];
    auto issue = [&](int zi, int st, bool now) {
        const int zm = map_border32(l_border, l_nz, zi);
        const unsigned char* pl = src + (int64_t)zm * l_sz;
        const unsigned sbo = (unsigned)(st * G::STAGE);
#pragma unroll
        for (int j = 0; j < G::NTASK; j++)
            if (goff[j] >= 0) cp_async16(sadr[j] + sbo, pl + goff[j]);
        unsigned char* sb = s_in + st * G::STAGE;
#pragma unroll
        for (int j = 0; j < NEL; j++)
            if (tid + j * NT < ntab) ev[j] = pl[s_tab[tid + j * NT].y];
        if (now) {
#pragma unroll
            for (int j = 0; j < NEL; j++)
                if (tid + j * NT < ntab) sb[s_tab[tid + j * NT].x] = (unsigned char)ev[j];
        }
        for (int i = tid + NEL * NT; i < ntab; i += NT) {
            const int2 e = s_tab[i];
            sb[e.x] = pl[e.y];
        }
    };
    auto commit_el = [&](int st) {
        unsigned char* sb = s_in + st * G::STAGE;
#pragma unroll
        for (int j = 0; j < NEL; j++)
            if (tid + j * NT < ntab) sb[s_tab[tid + j * NT].x] = (unsigned char)ev[j];
    };

    const int zin0 = zs - CZ, zin1 = ze - 1 + HZ;
    const int nplanes = zin1 - zin0 + 1;
#pragma unroll
    for (int s = 0; s < STAGES - 1; s++) {
        if (s < nplanes) issue(zin0 + s, s, true);
        cp_async_commit();
    }

    // X/Z role: column group g (columns 4g .. 4g+3), row pair rp
    // (a warp holds 16 row pairs x 2 column groups: the X-pass window loads
    // and the staged byte stores then fall on distinct banks)
    const int rp = tid & 15, g = tid >> 4;
    float2 q[KZ][4];
#pragma unroll
    for (int s = 0; s < KZ; s++)
#pragma unroll
        for (int m = 0; m < 4; m++) q[s][m] = make_float2(0.f, 0.f);
    int slot = 0;
    int stage = 0, stage_next = STAGES - 1;
    // one rounding of the numerator S: floor((S + h) / 2^shift), h = 2^(shift-1)
    // (round) or 0 (truncate).  The Z sums start from h, and the FP32
    // multiply-add (S + h) * 2^-shift + 2^23 rounded down lands on the integer
    // grid of [2^23, 2^24): the low byte of its bits is the result byte.
    const float rscale = __uint_as_float((unsigned)(127 - p.shift) << 23);
    const float rhalf = p.store_mode == STORE_ROUND && p.shift > 0 ? (float)(1 << (p.shift - 1)) : 0.f;
    const float2 rscale2 = make_float2(rscale, rscale), rbias2 = make_float2(8388608.f, 8388608.f);
    const float2 zinit = make_float2(rhalf, rhalf);

    for (int n = 0; n < nplanes; n++) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();   // plane n visible; every thread is past plane n-1
        const bool pending = n + STAGES - 1 < nplanes;
        const int st_pending = stage_next;
        if (pending) issue(zin0 + n + STAGES - 1, stage_next, false);
        cp_async_commit();
        stage_next = (stage_next + 1 == STAGES) ? 0 : stage_next + 1;
        const unsigned char* sb = s_in + stage * G::STAGE;
        stage = (stage + 1 == STAGES) ? 0 : stage + 1;

        // Y pass: word w (columns x0-4+4w ..), rows 2yp, 2yp+1.  Thread tid
        // takes the inner word 1 + (tid & 15) of row pair tid >> 4 (a warp
        // reads two row pairs' 64 inner bytes: no bank conflict); the last
        // warp also takes the two halo words of every row pair as half units
        // (the two columns of each that the X pass reads).
        {
            const int yp = tid >> 4, w = 1 + (tid & 15);
            const unsigned char* col = sb + (2 * yp) * RP + 12 + 4 * w;
            unsigned a0l = 0, a0h = 0, a1l = 0, a1h = 0;   // rows 2yp / 2yp+1, columns (0,1) / (2,3)
#pragma unroll
            for (int j = 0; j < KY + 1; j++) {
                const unsigned wd = *reinterpret_cast<const unsigned*>(col + j * RP);
                const unsigned l = lo16(wd), h = hi16(wd);
                if (j < KY) {
                    a0l += l * (unsigned)p.wyi[j];
                    a0h += h * (unsigned)p.wyi[j];
                }
                if (j >= 1) {
                    a1l += l * (unsigned)p.wyi[j - 1];
                    a1h += h * (unsigned)p.wyi[j - 1];
                }
            }
            // words (row 2yp, row 2yp+1) of columns 0..3
            uint4 o;
            o.x = __byte_perm(a0l, a1l, 0x5410);
            o.y = __byte_perm(a0l, a1l, 0x7632);
            o.z = __byte_perm(a0h, a1h, 0x5410);
            o.w = __byte_perm(a0h, a1h, 0x7632);
            *reinterpret_cast<uint4*>(s_y + yp * YP + 4 * w) = o;
        }
        if (tid >= NT - 32) {
            // halo unit h: row pair h >> 1; word 0 (columns x0-2, x0-1: the
            // high lanes) or word YW-1 (columns x0+64, x0+65: the low lanes)
            const int h = tid - (NT - 32), yp = h >> 1;
            const bool right = (h & 1) != 0;
            const int w = right ? YW - 1 : 0;
            const unsigned sel = right ? 0x4140u : 0x4342u;
            const unsigned char* col = sb + (2 * yp) * RP + 12 + 4 * w;
            unsigned a0 = 0, a1 = 0;
#pragma unroll
            for (int j = 0; j < KY + 1; j++) {
                const unsigned lane = __byte_perm(*reinterpret_cast<const unsigned*>(col + j * RP), 0u, sel);
                if (j < KY) a0 += lane * (unsigned)p.wyi[j];
                if (j >= 1) a1 += lane * (unsigned)p.wyi[j - 1];
            }
            *reinterpret_cast<uint2*>(s_y + yp * YP + 4 * w + (right ? 0 : 2)) =
                make_uint2(__byte_perm(a0, a1, 0x5410), __byte_perm(a0, a1, 0x7632));
        }
        __syncthreads();

        // X pass: columns 4g .. 4g+3 of row pair rp; window of Y-pass words
        // 4g .. 4g+11 (columns x0-4+4g ..)
        float2 xv[4];
        {
            const unsigned* wr = s_y + rp * YP + 4 * g;
            unsigned win[12];
#pragma unroll
            for (int v = 0; v < 3; v++) {
                const uint4 t = *reinterpret_cast<const uint4*>(wr + 4 * v);
                win[4 * v] = t.x; win[4 * v + 1] = t.y; win[4 * v + 2] = t.z; win[4 * v + 3] = t.w;
            }
#pragma unroll
            for (int m = 0; m < 4; m++) {
                unsigned a = 0;
#pragma unroll
                for (int k = 0; k < KX; k++) a += win[m + 4 - CX + k] * (unsigned)p.wxi[k];
                xv[m] = lanes_to_f2(a);
            }
        }
        float2 o[4];
        zdispatch_u8<KZ>(slot, q, xv, o, p, zinit);
        slot = (slot + 1 == KZ) ? 0 : slot + 1;
        if (n >= KZ - 1) {
            unsigned ob[4][2];   // column m: rows 2rp, 2rp+1; the result in the low byte
#pragma unroll
            for (int m = 0; m < 4; m++) {
                const float2 r = __ffma2_rd(o[m], rscale2, rbias2);
                ob[m][0] = __float_as_uint(r.x);
                ob[m][1] = __float_as_uint(r.y);
            }
            if constexpr (TS) {
                // staged x-major: the destination is contiguous along Y
#pragma unroll
                for (int m = 0; m < 4; m++) {
                    const unsigned short v2 = (unsigned short)__byte_perm(ob[m][0], ob[m][1], 0x0040);
                    *reinterpret_cast<unsigned short*>(s_o + (4 * g + m) * TY + 2 * rp) = v2;
                }
            } else {
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const unsigned v4 = __byte_perm(__byte_perm(ob[0][h], ob[1][h], 0x0040),
                                                    __byte_perm(ob[2][h], ob[3][h], 0x0040), 0x5410);
                    *reinterpret_cast<unsigned*>(s_o + (2 * rp + h) * (TX + 4) + 4 * g) = v4;
                }
            }
        }
        __syncthreads();
        if (n >= KZ - 1) {
            const int zo = zin0 + n - HZ;
            unsigned char* pl = dst + (int64_t)zo * p.dz;
            if constexpr (TS) {
                if (tid < TX * TY / 16) {
                    // 16 bytes along Y (the destination's contiguous axis)
                    const int xl = tid >> 1, yl = 16 * (tid & 1);
                    const int xa = x0 + xl, ya = y0 + yl;
                    const uint4 v = *reinterpret_cast<const uint4*>(s_o + xl * TY + yl);
                    unsigned char* d = pl + (int64_t)xa * p.dx + ya;
                    if (xa < p.nx && ya + 16 <= p.ny && p.vec_st) {
                        *reinterpret_cast<uint4*>(d) = v;
                    } else if (xa < p.nx) {
                        const unsigned char* bv = reinterpret_cast<const unsigned char*>(&v);
                        for (int e = 0; e < 16 && ya + e < p.ny; e++) d[e] = bv[e];
                    }
                }
            } else {
                // 4 bytes along X per word, two words per thread
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int wd = tid + h * NT;
                    const int yl = wd >> 4, xl = 4 * (wd & 15);
                    const int xa = x0 + xl, ya = y0 + yl;
                    const unsigned v = *reinterpret_cast<const unsigned*>(s_o + yl * (TX + 4) + xl);
                    unsigned char* d = pl + (int64_t)ya * p.dy + xa;
                    if (ya < p.ny && xa + 4 <= p.nx && p.vec_st) {
                        *reinterpret_cast<unsigned*>(d) = v;
                    } else if (ya < p.ny) {
                        for (int e = 0; e < 4 && xa + e < p.nx; e++) d[e] = (unsigned char)(v >> (8 * e));
                    }
                }
            }
        }
        // the issued plane's element bytes into its stage (read two planes on)
        if (pending) commit_el(st_pending);
    }
    cp_async_wait<0>();
}

using LaunchU8 = cudaError_t (*)(const FusedParams&, cudaStream_t);

template <int KX, int KY, int KZ>
cudaError_t launch_u8(const FusedParams& p_in, cudaStream_t s)
{
    using G = GU8<KY>;
    static_assert(G::SMEM <= 113 * 1024, "two CTAs per SM");
    static bool configured[2] = {false, false};
    FusedParams p = p_in;
    // the Z taps' integer numerators as FP32 pairs (exact below 2^24)
    for (int k = 0; k < 40; k++) {
        const float w = k < p.kz ? (float)p.wzi[k] : 0.f;
        p.wz2[k] = make_float2(w, w);
    }
    // 16-byte stores along Y for a transposed destination, 4-byte ones along X
    // otherwise
    const auto al16 = [](int64_t v) { return v % 16 == 0; };
    const bool dst16 = reinterpret_cast<uintptr_t>(p.dst) % 16 == 0 && al16(p.dz) && al16(p.db);
    const bool dst4 = reinterpret_cast<uintptr_t>(p.dst) % 4 == 0 && p.dy % 4 == 0 && p.dz % 4 == 0 && p.db % 4 == 0;
    p.vec_st = p.tstore ? (dst16 && al16(p.dx)) : dst4;
    auto kern = p.tstore ? k_fused_u8<KX, KY, KZ, true> : k_fused_u8<KX, KY, KZ, false>;
    if (!configured[p.tstore ? 1 : 0]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM);
        if (e != cudaSuccess) return e;
        configured[p.tstore ? 1 : 0] = true;
    }
    const long long gx = (long long)((p.nx + TX - 1) / TX) * ((p.ny + TY - 1) / TY) * p.nbatch;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int chunks = pick_zchunks(gx, 2LL * sms, p.nz, KZ - 1);
    p.zchunk = std::max(1, (p.nz + chunks - 1) / chunks);
    const int gz = (p.nz + p.zchunk - 1) / p.zchunk;
    if (gx > 0x7fffffffLL || gz > 65535) return cudaErrorInvalidConfiguration;
    kern<<<dim3((unsigned)gx, (unsigned)gz), NT, G::SMEM, s>>>(p);
    count_launch();
    return cudaGetLastError();
}

struct VariantU8 {
    int kx, ky, kz;
    LaunchU8 fn;
};
const VariantU8 kVariantsU8[] = {
    {5, 5, 5, &launch_u8<5, 5, 5>},   // binomial [1,4,6,4,1]/16 per axis
    {3, 3, 3, &launch_u8<3, 3, 3>},   // [1,2,1]/4 per axis
};

long long tap_sum(const int32_t* w, int k)
{
    long long s = 0;
    for (int i = 0; i < k; i++) s += w[i];
    return s;
}

}  // namespace

bool fused_u8_shape(int sdt, int ddt, int kx, int ky, int kz)
{
    if (sdt != NDLGPU_U8 || ddt != NDLGPU_U8) return false;
    for (const VariantU8& v : kVariantsU8)
        if (v.kx == kx && v.ky == ky && v.kz == kz) return true;
    return false;
}

bool fused_u8_supported(const FusedParams& p)
{
    if (p.src_dtype != NDLGPU_U8 || p.dst_dtype != NDLGPU_U8 || p.adj) return false;
    if (p.store_mode != STORE_ROUND && p.store_mode != STORE_CAST) return false;
    if (p.sx != 1 || !p.vec_ld || p.shift < 0 || p.shift > 30) return false;
    if (!p.tstore && p.dx != 1) return false;
    if (p.tstore && p.dy != 1) return false;
    bool found = false;
    for (const VariantU8& v : kVariantsU8)
        if (v.kx == p.kx && v.ky == p.ky && v.kz == p.kz) found = true;
    if (!found) return false;
    for (int k = 0; k < p.kx; k++) if (p.wxi[k] < 0) return false;
    for (int k = 0; k < p.ky; k++) if (p.wyi[k] < 0) return false;
    for (int k = 0; k < p.kz; k++) if (p.wzi[k] < 0) return false;
    // packed lanes: the Y sums and the X-of-Y sums of bytes stay below 2^16;
    // the Z sums plus the rounding's half unit (FP32 integers) below 2^23
    const long long sy = tap_sum(p.wyi, p.ky), sx = tap_sum(p.wxi, p.kx), sz = tap_sum(p.wzi, p.kz);
    if (255 * sy >= 65536 || 255 * sy * sx >= 65536) return false;
    const long long half = p.shift > 0 ? 1LL << (p.shift - 1) : 0;
    if (255 * sy * sx * sz + half >= (1LL << 23)) return false;
    return true;
}

cudaError_t launch_fused_u8(const FusedParams& p, cudaStream_t s)
{
    if (!fused_u8_supported(p)) return cudaErrorNotSupported;
    if (p.nx <= 0 || p.ny <= 0 || p.nz <= 0 || p.nbatch <= 0) return cudaSuccess;
    for (const VariantU8& v : kVariantsU8)
        if (v.kx == p.kx && v.ky == p.ky && v.kz == p.kz) return v.fn(p, s);
    return cudaErrorNotSupported;
}

}  // namespace ndlgpu
