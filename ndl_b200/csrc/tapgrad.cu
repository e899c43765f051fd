// tapgrad.cu -- fused tap gradients of a three-pass separable chain (no
// reference counterpart: ndl has no gradients).
//
// For Y = Pz(Py(Px X)) and L = sum(G * Y), with P_a = sum_k w_a[k] S_a^k
// (S_a^k: the border-mapped shift by o_k = k - K/2 along axis a), and the
// passes and shifts along different axes commuting:
//   dL/dwz[k] = < G,        S_z^k (Py Px X) >
//   dL/dwy[k] = < Pz^T G,   S_y^k (Px X) >
//   dL/dwx[k] = < Pz^T G,   S_x^k (Py X) >
// One kernel streams Z: a CTA owns a 64 x 16 tile and, per plane c, has the X
// tile of plane c with border-mapped X/Y halos in shared memory (cp.async
// ring), computes Px X (halo rows), Py X (halo columns) and Py Px X, and keeps
// the G values of planes c-r..c+r in a per-thread register queue for Pz^T G
// and the Z correlations.  Pz^T near the Z borders (Clamp / Reflect, G read as
// zero outside the image) folds the out-of-range taps back with coefficients
// computed on the fly; Wrap reads G wrapped.  Per-thread sums are reduced per
// CTA in a fixed order, then over CTAs in a fixed order (deterministic).
#include "dtype.cuh"

namespace ndlgpu {
namespace {

constexpr int TX = 64;
constexpr int TY = 16;
constexpr int NT = 256;   // 16 column groups of 4 x 16 rows
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

template <class T> __device__ __forceinline__ float to_f(T v);
template <> __device__ __forceinline__ float to_f<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <> __device__ __forceinline__ float to_f<__half>(__half v) { return __half2float(v); }

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

template <class T, int KX, int KY>
struct TGeo {
    static constexpr int EPC = 16 / (int)sizeof(T);
    static constexpr int CX = KX / 2;
    static constexpr int CY = KY / 2;
    static constexpr int D = (EPC - CX % EPC) % EPC;       // shared column of global x0 - CX
    static constexpr int WBASE = (D / 4) * 4;               // first column of a 4-aligned window
    static constexpr int WOFF = D % 4;                      // window offset inside it
    static constexpr int ROWS = TY + KY - 1;
    static constexpr int XC = TX + KX - 1;                 // columns of Py X the taps need
    static constexpr int XCP = (WOFF + XC + 3) / 4 * 4;    // columns computed, from shared column WBASE
    static_assert(TY % 4 == 0, "the Y-pass units cover 4 rows");
    static constexpr int NCH = (XC + D + EPC - 1) / EPC;
    static constexpr int NV = (WOFF + KX + 3 + 3) / 4;
    static constexpr int WEND0 = 60 + WBASE + 4 * NV;      // columns an X window reads
    static constexpr int WEND = WEND0 > WBASE + XCP ? WEND0 : WBASE + XCP;   // and the Py X pass
    static constexpr int PITCH = (NCH * EPC > WEND ? NCH * EPC : (WEND + EPC - 1) / EPC * EPC);
    static constexpr int NTASK = (ROWS * NCH + NT - 1) / NT;
    static constexpr int NXU = ROWS * 16;                  // X-pass units: 1 row x 4 columns
    static constexpr int NQ = XCP / 4;
    static constexpr int NU = NXU + (TY / 4) * NQ;         // + Y-pass units: 4 rows x 4 columns
    static constexpr int NUR = (NU + NT - 1) / NT;          // unit rounds per thread
    static_assert((TY / 4) * NQ <= NT, "one Y unit per thread at most");
    static constexpr size_t IN_BYTES = (size_t)STAGES * ROWS * PITCH * sizeof(T);
    static constexpr size_t X1_BYTES = (size_t)ROWS * TX * 4;
    static constexpr size_t X1Y_BYTES = (size_t)(TY * XCP + 16) * 4;   // the last windows read past the end
    static constexpr size_t TAB_BYTES = (size_t)ROWS * PITCH * 8;
    static constexpr size_t RED_BYTES = (size_t)(NT / 32) * 64 * 8;
    static constexpr size_t SMEM = IN_BYTES + X1_BYTES + X1Y_BYTES + TAB_BYTES + RED_BYTES + 16;
};

__device__ __forceinline__ int bmap(int border, int M, int x) { return map_border32(border, M, x); }

// The G queue is a shift register: gq[m] holds plane c - r + m (window
// position m), gq[KZ-1] the newest.  One copy of the code serves every plane
// (a rotating-slot dispatch would replicate the border-plane paths KZ times).

// (Pz^T G)(plane c) from the window; border planes (Clamp / Reflect, G zero
// outside the image) collect, for window plane z_m, every tap k whose
// forward read map(z_m + o_k) lands on c.
template <int KZ>
__device__ __forceinline__ void zt_apply(const float (&gq)[KZ][4], float (&g2)[4], const TapFusedParams& p, int c,
                                         bool border_plane)
{
    constexpr int R = KZ / 2;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        float a = 0.f;
#pragma unroll
        for (int m = 0; m < KZ; m++) a = fmaf(gq[m][e], p.wzf[KZ - 1 - m], a);
        g2[e] = a;
    }
    if (border_plane) {
#pragma unroll
        for (int e = 0; e < 4; e++) g2[e] = 0.f;
#pragma unroll
        for (int m = 0; m < KZ; m++) {
            const int z = c - R + m;
            float coef = 0.f;
            if (z >= 0 && z < p.nz) {
                for (int k = 0; k < KZ; k++)
                    if (map_border32(p.border, p.nz, z + k - R) == c) coef += p.wzf[k];
            }
#pragma unroll
            for (int e = 0; e < 4; e++) g2[e] = fmaf(gq[m][e], coef, g2[e]);
        }
    }
}

// dwz[k] += X2(plane c) . G(planes z with map(z + o_k) == c).
template <int KZ>
__device__ __forceinline__ void zt_taps(const float (&gq)[KZ][4], const float (&x2)[4], float (&dwz)[KZ],
                                        const TapFusedParams& p, int c, bool border_plane)
{
    constexpr int R = KZ / 2;
    float dd[KZ];
#pragma unroll
    for (int m = 0; m < KZ; m++)
        dd[m] = fmaf(x2[0], gq[m][0], fmaf(x2[1], gq[m][1], fmaf(x2[2], gq[m][2], x2[3] * gq[m][3])));
    if (border_plane) {
#pragma unroll
        for (int k = 0; k < KZ; k++) {
            float a = 0.f;
            for (int m = 0; m < KZ; m++) {
                const int z = c - R + m;
                if (z >= 0 && z < p.nz && map_border32(p.border, p.nz, z + k - R) == c) a += dd[m];
            }
            dwz[k] += a;
        }
    } else {
#pragma unroll
        for (int k = 0; k < KZ; k++) dwz[k] += dd[KZ - 1 - k];
    }
}

template <class T, int KX, int KY, int KZ>
__global__ void __launch_bounds__(NT, 2) k_tapgrad(const __grid_constant__ TapFusedParams p)
{
    using G = TGeo<T, KX, KY>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* s_in = reinterpret_cast<T*>(smem_raw);
    float* s_x1 = reinterpret_cast<float*>(smem_raw + G::IN_BYTES);
    float* s_x1y = reinterpret_cast<float*>(smem_raw + G::IN_BYTES + G::X1_BYTES);
    int2* s_tab = reinterpret_cast<int2*>(smem_raw + G::IN_BYTES + G::X1_BYTES + G::X1Y_BYTES);
    double* s_red = reinterpret_cast<double*>(smem_raw + G::IN_BYTES + G::X1_BYTES + G::X1Y_BYTES + G::TAB_BYTES);
    int* s_ntab = reinterpret_cast<int*>(smem_raw + G::IN_BYTES + G::X1_BYTES + G::X1Y_BYTES + G::TAB_BYTES +
                                         G::RED_BYTES);

    const int tid = threadIdx.x;
    __builtin_assume(tid < NT);
    const int ntx = (p.nx + TX - 1) / TX;
    const int nty = (p.ny + TY - 1) / TY;
    const int tile = blockIdx.x % (ntx * nty);
    const int bat = blockIdx.x / (ntx * nty);
    const int x0 = (tile % ntx) * TX;
    const int y0 = (tile / ntx) * TY;
    const int zs = blockIdx.y * p.zchunk;
    const int ze = min(p.nz, zs + p.zchunk);
    const T* xs = reinterpret_cast<const T*>(p.x) + (int64_t)bat * p.sb;
    const T* gs = reinterpret_cast<const T*>(p.g) + (int64_t)bat * p.gb;
    constexpr int RZ = KZ / 2;

    float dwx[KX], dwy[KY], dwz[KZ];
#pragma unroll
    for (int k = 0; k < KX; k++) dwx[k] = 0.f;
#pragma unroll
    for (int k = 0; k < KY; k++) dwy[k] = 0.f;
#pragma unroll
    for (int k = 0; k < KZ; k++) dwz[k] = 0.f;

    if (zs < ze) {
        // X loader set-up (border-mapped halos, as the forward)
        const int gx0 = x0 - G::CX - G::D;   // global column of shared column 0 (16-byte aligned)
        if (tid == 0) *s_ntab = 0;
        __syncthreads();
        int32_t goff[G::NTASK];
        int32_t soff[G::NTASK];
#pragma unroll
        for (int j = 0; j < G::NTASK; j++) {
            const int t = tid + j * NT;
            goff[j] = -1;
            soff[j] = 0;
            if (t >= G::ROWS * G::NCH) continue;
            const int r = t / G::NCH;
            const int q = t - r * G::NCH;
            int y = y0 - G::CY + r;
            y = (y >= p.ny + KY - 1 - G::CY) ? p.ny - 1 : bmap(p.border, p.ny, y);
            const int32_t rowoff = (int32_t)(y * p.sy);
            const int cx0 = gx0 + q * G::EPC;
            if (p.vec_ld && cx0 >= 0 && cx0 + G::EPC <= p.nx) {
                goff[j] = rowoff + cx0;
                soff[j] = r * G::PITCH + q * G::EPC;
            } else {
                for (int e = 0; e < G::EPC; e++) {
                    int x = cx0 + e;
                    x = (x >= p.nx + KX - 1 - G::CX || x < -G::CX) ? p.nx - 1 : bmap(p.border, p.nx, x);
                    const int si = atomicAdd(s_ntab, 1);
                    s_tab[si] = make_int2(r * G::PITCH + q * G::EPC + e, rowoff + (int32_t)(x * p.sx));
                }
            }
        }
        __syncthreads();
        const int ntab = *s_ntab;
        auto issue = [&](int zi, int stage) {
            const T* pl = xs + (int64_t)zi * p.sz;
            T* sb = s_in + stage * (G::ROWS * G::PITCH);
#pragma unroll
            for (int j = 0; j < G::NTASK; j++)
                if (goff[j] >= 0) cp_async16(sb + soff[j], pl + goff[j]);
            for (int i = tid; i < ntab; i += NT) {
                const int2 e = s_tab[i];
                if constexpr (sizeof(T) == 4) cp_async4(sb + e.x, pl + e.y);
                else sb[e.x] = pl[e.y];
            }
        };

        // G of this thread's 4 positions: (x0+4gx .. +3, y0+gy)
        const int gxq = tid & 15, gyq = tid >> 4;
        const int xg = x0 + 4 * gxq, yg = y0 + gyq;
        const T* grow = gs + (int64_t)yg * p.gy;
        auto gload = [&](int zi, float (&v)[4]) {
#pragma unroll
            for (int e = 0; e < 4; e++) v[e] = 0.f;
            if (yg >= p.ny) return;
            if (zi < 0 || zi >= p.nz) {
                if (p.zero_pad) return;
                zi = bmap(p.border, p.nz, zi);
            }
            const T* row = grow + (int64_t)zi * p.gz;
            if (p.vec_g && xg + 4 <= p.nx) {
                lds4(row + xg, v);   // 16- or 8-byte aligned global load
            } else {
#pragma unroll
                for (int e = 0; e < 4; e++)
                    if (xg + e < p.nx) v[e] = to_f<T>(row[(int64_t)(xg + e) * p.gxs]);
            }
        };

        float gq[KZ][4];
#pragma unroll
        for (int m = 0; m < KZ; m++)
#pragma unroll
            for (int e = 0; e < 4; e++) gq[m][e] = 0.f;
        // queue prologue: planes zs - r .. zs + r - 1 into window positions 1 .. KZ-1
        // (the shift at the first plane moves them to 0 .. KZ-2)
#pragma unroll
        for (int m = 1; m < KZ; m++) {
            float v[4];
            gload(zs - RZ + m - 1, v);
#pragma unroll
            for (int e = 0; e < 4; e++) gq[m][e] = v[e];
        }
        const bool valid_all = (yg < p.ny) && (xg + 4 <= p.nx);
        const int nplanes = ze - zs;
#pragma unroll
        for (int s = 0; s < STAGES - 1; s++) {
            if (s < nplanes) issue(zs + s, s);
            cp_async_commit();
        }
        float gn[4];
        gload(zs + RZ, gn);
        // this thread's Y unit (if any): v2 = u - NXU for its first u >= NXU
        int y_rg = 0, y_qq = 0;
        {
            const int v2 = tid + ((G::NXU - tid + NT - 1) / NT) * NT - G::NXU;
            y_rg = v2 / G::NQ;
            y_qq = v2 - y_rg * G::NQ;
        }
        int stage = 0, stage_next = STAGES - 1;
        for (int n = 0; n < nplanes; n++) {
            const int c = zs + n;
            cp_async_wait<STAGES - 2>();
            __syncthreads();
            if (n + STAGES - 1 < nplanes) issue(zs + n + STAGES - 1, stage_next);
            cp_async_commit();
            stage_next = (stage_next + 1 == STAGES) ? 0 : stage_next + 1;
            const T* sb = s_in + stage * (G::ROWS * G::PITCH);
            // X pass (Px X on all ROWS) and Y pass of the raw tile (Py X on
            // all XC columns).  Unit u = tid + i * NT of this thread: an X
            // unit (row (tid >> 4) + i * NT/16, column group tid & 15) while
            // u < NXU, then at most one Y unit (indices set up before the loop)
#pragma unroll
            for (int i = 0; i < G::NUR; i++) {
                const int u = tid + i * NT;
                if (u >= G::NU) break;
                if (u < G::NXU) {
                    const int r = (tid >> 4) + i * (NT / 16), g = tid & 15;
                    float win[G::NV * 4];
#pragma unroll
                    for (int v = 0; v < G::NV; v++) lds4(sb + r * G::PITCH + 4 * g + G::WBASE + 4 * v, win + 4 * v);
                    float a[4];
#pragma unroll
                    for (int m = 0; m < 4; m++) {
                        float s = 0.f;
#pragma unroll
                        for (int k = 0; k < KX; k++) s = fmaf(win[G::WOFF + m + k], p.wxf[k], s);
                        a[m] = s;
                    }
                    *reinterpret_cast<float4*>(s_x1 + r * TX + 4 * g) = make_float4(a[0], a[1], a[2], a[3]);
                } else {
                    // Py X: 4 rows x 4 columns, each loaded row feeding up to
                    // 4 outputs (packed FMA over column pairs)
                    const int rg = y_rg, qq = y_qq;
                    const T* col = sb + (4 * rg) * G::PITCH + G::WBASE + 4 * qq;
                    float2 a[4][2];
#pragma unroll
                    for (int h = 0; h < 4; h++) a[h][0] = a[h][1] = make_float2(0.f, 0.f);
#pragma unroll
                    for (int j = 0; j < KY + 3; j++) {
                        float t[4];
                        lds4(col + j * G::PITCH, t);
                        const float2 lo = make_float2(t[0], t[1]), hi = make_float2(t[2], t[3]);
#pragma unroll
                        for (int h = 0; h < 4; h++) {
                            const int k = j - h;
                            if (k >= 0 && k < KY) {
                                a[h][0] = __ffma2_rn(lo, p.wy2[k], a[h][0]);
                                a[h][1] = __ffma2_rn(hi, p.wy2[k], a[h][1]);
                            }
                        }
                    }
#pragma unroll
                    for (int h = 0; h < 4; h++)
                        *reinterpret_cast<float4*>(s_x1y + (4 * rg + h) * G::XCP + 4 * qq) =
                            make_float4(a[h][0].x, a[h][0].y, a[h][1].x, a[h][1].y);
                }
            }
            __syncthreads();
            // shift the G window and append plane c + r; then Pz^T G at plane c
#pragma unroll
            for (int m = 0; m + 1 < KZ; m++)
#pragma unroll
                for (int e = 0; e < 4; e++) gq[m][e] = gq[m + 1][e];
#pragma unroll
            for (int e = 0; e < 4; e++) gq[KZ - 1][e] = gn[e];
            const bool border_plane = p.zero_pad && (c < RZ || c >= p.nz - RZ);
            float g2[4];
            zt_apply<KZ>(gq, g2, p, c, border_plane);
            if (n + 1 < nplanes) gload(c + 1 + RZ, gn);
            // Y pass of Px X -> X2, and dwy
            float x2[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 0; k < KY; k++) {
                const float4 v = *reinterpret_cast<const float4*>(s_x1 + (gyq + k) * TX + 4 * gxq);
                x2[0] = fmaf(v.x, p.wyf[k], x2[0]); x2[1] = fmaf(v.y, p.wyf[k], x2[1]);
                x2[2] = fmaf(v.z, p.wyf[k], x2[2]); x2[3] = fmaf(v.w, p.wyf[k], x2[3]);
                dwy[k] = fmaf(g2[0], v.x, fmaf(g2[1], v.y, fmaf(g2[2], v.z, fmaf(g2[3], v.w, dwy[k]))));
            }
            // dwx from Py X
            {
                float win[G::NV * 4];
#pragma unroll
                for (int v = 0; v < G::NV; v++) lds4(s_x1y + gyq * G::XCP + 4 * gxq + 4 * v, win + 4 * v);
#pragma unroll
                for (int k = 0; k < KX; k++)
                    dwx[k] = fmaf(g2[0], win[G::WOFF + k], fmaf(g2[1], win[G::WOFF + k + 1],
                                  fmaf(g2[2], win[G::WOFF + k + 2], fmaf(g2[3], win[G::WOFF + k + 3], dwx[k]))));
            }
            // positions outside the image carry g2 = 0 but x2 from mapped
            // loads: zero x2 there so that dwz sees no contribution
            if (!valid_all) {
#pragma unroll
                for (int e = 0; e < 4; e++)
                    if (yg >= p.ny || xg + e >= p.nx) x2[e] = 0.f;
            }
            zt_taps<KZ>(gq, x2, dwz, p, c, border_plane);
            stage = (stage + 1 == STAGES) ? 0 : stage + 1;
        }
        cp_async_wait<0>();
    }

    // CTA reduction in a fixed order: warp shuffles, then warps in order
    const int warp = tid >> 5, lane = tid & 31;
    auto red = [&](float v, int idx) {
        double d = (double)v;
        for (int s = 16; s > 0; s >>= 1) d += __shfl_down_sync(0xffffffffu, d, s);
        if (lane == 0) s_red[warp * 64 + idx] = d;
    };
#pragma unroll
    for (int k = 0; k < KX; k++) red(dwx[k], k);
#pragma unroll
    for (int k = 0; k < KY; k++) red(dwy[k], KX + k);
#pragma unroll
    for (int k = 0; k < KZ; k++) red(dwz[k], KX + KY + k);
    __syncthreads();
    const int ntap = KX + KY + KZ;
    if (tid < ntap) {
        double a = 0.0;
        for (int w = 0; w < NT / 32; w++) a += s_red[w * 64 + tid];
        const long long cta = (long long)blockIdx.y * gridDim.x + blockIdx.x;
        p.partial[cta * ntap + tid] = a;
    }
}

// Sum of the per-CTA partials; out[map[t]] = sum_t.  One warp per tap: lane
// l adds CTAs l, l+32, ... in order, then a fixed shuffle tree (the same
// order on every run).
__global__ void k_tapgrad_final(const double* partial, int ncta, int ntap, TapFinalMap mp, void* out, int out_dtype)
{
    const int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= ntap) return;
    double a = 0.0;
    for (int c = lane; c < ncta; c += 32) a += partial[(long long)c * ntap + t];
    for (int s = 16; s > 0; s >>= 1) a += __shfl_down_sync(0xffffffffu, a, s);
    if (lane == 0) {
        const int o = mp.dst[t];
        if (o < 0) return;                 // an image's unit pass: not reported
        if (out_dtype == NDLGPU_F64) ((double*)out)[o] = a;
        else ((float*)out)[o] = (float)a;
    }
}

template <class T, int KX, int KY, int KZ>
cudaError_t launch_tg(const TapFusedParams& p, void* out, int out_dtype, const TapFinalMap& mp, cudaStream_t s)
{
    using G = TGeo<T, KX, KY>;
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(k_tapgrad<T, KX, KY, KZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)G::SMEM);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    const int ntx = (p.nx + TX - 1) / TX;
    const int nty = (p.ny + TY - 1) / TY;
    const long long gx = (long long)ntx * nty * p.nbatch;
    const int gz = (p.nz + p.zchunk - 1) / p.zchunk;
    if (gx > 0x7fffffffLL || gz > 65535) return cudaErrorInvalidConfiguration;
    k_tapgrad<T, KX, KY, KZ><<<dim3((unsigned)gx, (unsigned)gz), NT, G::SMEM, s>>>(p);
    const int ntap = KX + KY + KZ;
    k_tapgrad_final<<<(ntap + 7) / 8, 256, 0, s>>>(p.partial, (int)(gx * gz), ntap, mp, out, out_dtype);
    count_launch(2);
    return cudaGetLastError();
}

using TgFn = cudaError_t (*)(const TapFusedParams&, void*, int, const TapFinalMap&, cudaStream_t);
struct TgVariant {
    int dt, kx, ky, kz;
    TgFn fn;
};
const TgVariant kTg[] = {
    // images (two passes and a unit pass across the planes)
    {NDLGPU_F32, 3, 3, 1, &launch_tg<float, 3, 3, 1>},
    {NDLGPU_F32, 5, 5, 1, &launch_tg<float, 5, 5, 1>},
    {NDLGPU_F32, 7, 7, 1, &launch_tg<float, 7, 7, 1>},
    {NDLGPU_F32, 9, 9, 1, &launch_tg<float, 9, 9, 1>},
    {NDLGPU_F32, 11, 11, 1, &launch_tg<float, 11, 11, 1>},
    {NDLGPU_F32, 13, 13, 1, &launch_tg<float, 13, 13, 1>},
    {NDLGPU_F32, 3, 3, 3, &launch_tg<float, 3, 3, 3>},
    {NDLGPU_F32, 5, 5, 5, &launch_tg<float, 5, 5, 5>},
    {NDLGPU_F32, 7, 7, 7, &launch_tg<float, 7, 7, 7>},
    {NDLGPU_F32, 11, 11, 11, &launch_tg<float, 11, 11, 11>},
    {NDLGPU_F32, 13, 13, 13, &launch_tg<float, 13, 13, 13>},
    {NDLGPU_F32, 9, 9, 9, &launch_tg<float, 9, 9, 9>},
    {NDLGPU_F32, 17, 17, 9, &launch_tg<float, 17, 17, 9>},
    {NDLGPU_F32, 17, 17, 11, &launch_tg<float, 17, 17, 11>},
    // 16-bit small volume filters
    {NDLGPU_BF16, 3, 3, 3, &launch_tg<__nv_bfloat16, 3, 3, 3>},
    {NDLGPU_BF16, 5, 5, 5, &launch_tg<__nv_bfloat16, 5, 5, 5>},
    {NDLGPU_BF16, 7, 7, 7, &launch_tg<__nv_bfloat16, 7, 7, 7>},
    {NDLGPU_BF16, 9, 9, 9, &launch_tg<__nv_bfloat16, 9, 9, 9>},
    {NDLGPU_F16, 3, 3, 3, &launch_tg<__half, 3, 3, 3>},
    {NDLGPU_F16, 5, 5, 5, &launch_tg<__half, 5, 5, 5>},
    {NDLGPU_F16, 7, 7, 7, &launch_tg<__half, 7, 7, 7>},
    {NDLGPU_F16, 9, 9, 9, &launch_tg<__half, 9, 9, 9>},
    {NDLGPU_BF16, 17, 17, 11, &launch_tg<__nv_bfloat16, 17, 17, 11>},
    {NDLGPU_F16, 17, 17, 11, &launch_tg<__half, 17, 17, 11>},
};

}  // namespace

bool tapgrad_supported(int dt, int kx, int ky, int kz)
{
    for (const TgVariant& v : kTg)
        if (v.dt == dt && v.kx == kx && v.ky == ky && v.kz == kz) return true;
    return false;
}

// Number of CTAs the launch will use (the partial-sum buffer holds
// ncta * (kx + ky + kz) doubles).
long long tapgrad_ctas(const TapFusedParams& p)
{
    const long long ntx = (p.nx + TX - 1) / TX, nty = (p.ny + TY - 1) / TY;
    return ntx * nty * p.nbatch * ((p.nz + p.zchunk - 1) / p.zchunk);
}

int tapgrad_zchunk(int nx, int ny, int nz, int nbatch, int kz)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long tiles = (long long)((nx + TX - 1) / TX) * ((ny + TY - 1) / TY) * nbatch;
    const long long slots = 2LL * sms;
    const int chunks = pick_zchunks(tiles, slots, nz, kz - 1);
    const int zc = (nz + chunks - 1) / chunks;
    return zc < 1 ? 1 : zc;
}

cudaError_t launch_tapgrad(const TapFusedParams& p, void* out, int out_dtype, const TapFinalMap& mp, cudaStream_t s)
{
    for (const TgVariant& v : kTg)
        if (v.dt == p.x_dtype && v.kx == p.kx && v.ky == p.ky && v.kz == p.kz) return v.fn(p, out, out_dtype, mp, s);
    return cudaErrorNotSupported;
}

}  // namespace ndlgpu
