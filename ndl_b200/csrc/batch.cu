// batch.cu -- the batched form: many instances of uneven extents, tap counts
// and border modes in one persistent launch (no reference counterpart).
//
// Every instance runs its passes one axis at a time (X, then Y, then Z:
// those it has) as phases of one persistent launch.  A phase reads the
// instance's source (first phase) or the f32 scratch the previous phase
// wrote, and writes the next scratch buffer or the destination (last phase),
// so every pass sees the whole axis and no halo is ever recomputed -- the
// right trade for the wide kernels of this form (up to 37 taps per axis),
// where a fused 2.5-D tile would redo the X pass over 36 halo rows and hold
// a 37-plane ring per tile.
//
// Work items (instance, phase, first unit, units) sit in a table sorted by
// phase, then by decreasing cost; CTAs of a persistent grid take them from an
// atomic counter.  An item of phase p waits (bounded, on a per-instance
// counter) until every item of phase p-1 of its instance has finished: those
// items were handed out earlier to running CTAs and wait on nothing later,
// so the wait always ends.  A wait that runs past its bound sets an error
// flag and drops the item instead of hanging.
//
//   row pass (X, the contiguous axis): a warp takes one row at a time, in
//     128-output segments staged with their halo in a per-warp shared
//     buffer; each lane computes 4 outputs from a register window.
//   column pass (Y or Z): a warp takes 64 consecutive columns (2 per lane)
//     of one line and slides along the axis in blocks of P outputs, each
//     block read as a register window of P + B - 1 column pairs (L1-cached
//     global loads) and accumulated with packed FP32 FMA.
//
// Tap widths are bucketed to compiled widths {1,3,5,9,...,37} (zero padded,
// centred).  Forward and the adjoint's Wrap read border-mapped samples; the
// adjoint with Clamp/Reflect reads zeros outside the image and gives the r
// positions at each end of an axis host-built effective weights (the fold of
// the out-of-range taps).
#include <type_traits>

#include "dtype.cuh"

namespace ndlgpu {
namespace {

__device__ int32_t g_guard_batch;   // bit 2: a phase wait ran past its bound

constexpr int kSeg = 128;        // row-pass outputs per warp segment
constexpr int kColS = 64;        // column-pass outputs per unit along the axis
constexpr int kMaxSpins = 1 << 22;
// Test controls (ndlgpu_test_wait_timeouts): the bound of a phase wait, and
// extra predecessor items a wait asks for that never arrive.
__device__ int g_batch_wait_spins = kMaxSpins;
__device__ int g_batch_need_bias = 0;

template <class T> __device__ __forceinline__ float to_f(T v);
template <> __device__ __forceinline__ float to_f<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <> __device__ __forceinline__ float to_f<__half>(__half v) { return __half2float(v); }
template <class T> __device__ __forceinline__ T from_f(float v);
template <> __device__ __forceinline__ float from_f<float>(float v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ __half from_f<__half>(float v) { return __float2half_rn(v); }

__device__ __forceinline__ int zone_row(int j, int n, int r)
{
    if (j < r) return j;
    if (j >= n - r) return r + (j - (n - r));
    return -1;
}

// Sample coordinate read for axis position x (extent n, real radius r), or -1
// for a zero sample.  Positions beyond the real radius feed only zero-padded
// taps, so any in-range sample will do there.
__device__ __forceinline__ int sample_at(int x, int n, int r, int border, int zero_pad)
{
    if (x >= 0 && x < n) return x;
    if (zero_pad) return -1;
    if (x < -r) return 0;
    if (x >= n + r) return n - 1;
    return map_border32(border, n, x);
}

struct View {
    const void* p;
    long long s[4];   // element strides of x, y, z, batch
};

template <class T>
__device__ __forceinline__ void store1(void* out, bool f32, long long i, float v)
{
    if (f32) reinterpret_cast<float*>(out)[i] = v;
    else reinterpret_cast<T*>(out)[i] = from_f<T>(v);
}

// Loads of one element / an aligned pair as floats: the instance's source
// through the read-only path, the scratch of an earlier phase with a
// coherent L1-cached load (a scratch buffer is only read after every write
// to it has finished, and each instance's buffer is 256-byte aligned, so no
// SM can hold a stale line of it).
template <bool RO, class TI>
__device__ __forceinline__ float ldf(const TI* p)
{
    if constexpr (RO) return to_f<TI>(__ldg(p));
    else return to_f<TI>(__ldca(p));
}
template <bool RO>
__device__ __forceinline__ float2 ld2f(const float* p)
{
    if constexpr (RO) return __ldg(reinterpret_cast<const float2*>(p));
    else return __ldca(reinterpret_cast<const float2*>(p));
}
template <bool RO, class H>
__device__ __forceinline__ float2 ld2f(const H* p)
{
    const unsigned int u = RO ? __ldg(reinterpret_cast<const unsigned int*>(p))
                              : __ldca(reinterpret_cast<const unsigned int*>(p));
    if constexpr (std::is_same_v<H, __nv_bfloat16>)
        return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xffff0000u));
    else
        return __half22float2(*reinterpret_cast<const __half2*>(&u));
}

// Row pass of rows [row0, row0 + nrows) (row = (b * nz + z) * ny + y).
// FIRST: the input is the instance's source (storage type T), else the f32
// scratch of the previous phase.
template <bool FIRST, class T, int B>
__device__ void row_pass(const BatchDesc& d, const View& in, const View& out, bool out_f32, const float* s_w,
                         const float* __restrict__ zones, int row0, int nrows, float* s_buf)
{
    using TI = std::conditional_t<FIRST, T, float>;
    constexpr int R = B / 2;
    constexpr int NV = (B + 3 + 3) / 4;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const bool zoned = d.zero_pad && d.zone_x >= 0;
    const TI* ip = reinterpret_cast<const TI*>(in.p);
    const long long sx = in.s[0];
    for (int rr = row0 + warp; rr < row0 + nrows; rr += nw) {
        const int y = rr % d.ny;
        const int t = rr / d.ny;
        const int z = t % d.nz;
        const int b = t / d.nz;
        const TI* irow = ip + b * in.s[3] + z * in.s[2] + y * in.s[1];
        const long long obase = b * out.s[3] + z * out.s[2] + y * out.s[1];
        for (int x0 = 0; x0 < d.nx; x0 += kSeg) {
            if (x0 - R >= 0 && x0 + kSeg + B - 1 - R <= d.nx) {
                const TI* q = irow + (long long)(x0 - R) * sx;
                for (int i = lane; i < kSeg + B - 1; i += 32) s_buf[i] = ldf<FIRST>(q + (long long)i * sx);
            } else {
                for (int i = lane; i < kSeg + B - 1; i += 32) {
                    const int c = sample_at(x0 - R + i, d.nx, d.rx, d.border, d.zero_pad);
                    s_buf[i] = c < 0 ? 0.f : ldf<FIRST>(irow + (long long)c * sx);
                }
            }
            __syncwarp();
            // window element i = 4v + e feeds outputs m with tap k = i - m
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int v = 0; v < NV; v++) {
                const float4 q = *reinterpret_cast<const float4*>(s_buf + 4 * lane + 4 * v);
                const float val[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
                for (int e = 0; e < 4; e++)
#pragma unroll
                    for (int m = 0; m < 4; m++) {
                        const int k = 4 * v + e - m;
                        if (k >= 0 && k < B) acc[m] = fmaf(val[e], s_w[k], acc[m]);
                    }
            }
            const int xo = x0 + 4 * lane;
            if (zoned && (xo < d.rx || xo + 3 >= d.nx - d.rx)) {
#pragma unroll
                for (int m = 0; m < 4; m++) {
                    const int e = zone_row(xo + m, d.nx, d.rx);
                    if (e < 0) continue;
                    const float* zw = zones + d.zone_x + e * B;
                    float a = 0.f;
                    for (int k = 0; k < B; k++) a = fmaf(s_buf[4 * lane + m + k], __ldg(zw + k), a);
                    acc[m] = a;
                }
            }
            __syncwarp();
            if (xo < d.nx) {
                if (out_f32 && xo + 4 <= d.nx && ((obase + xo) & 3) == 0) {
                    *reinterpret_cast<float4*>(reinterpret_cast<float*>(const_cast<void*>(out.p)) + obase + xo) =
                        make_float4(acc[0], acc[1], acc[2], acc[3]);
                } else {
#pragma unroll
                    for (int m = 0; m < 4; m++)
                        if (xo + m < d.nx)
                            store1<T>(const_cast<void*>(out.p), out_f32, obase + (long long)(xo + m) * out.s[0], acc[m]);
                }
            }
        }
    }
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// 4 consecutive staged elements as floats.
__device__ __forceinline__ float4 lds4f(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ float4 lds4f(const __nv_bfloat16* p)
{
    const uint2 t = *reinterpret_cast<const uint2*>(p);
    return make_float4(__uint_as_float(t.x << 16), __uint_as_float(t.x & 0xffff0000u), __uint_as_float(t.y << 16),
                       __uint_as_float(t.y & 0xffff0000u));
}
__device__ __forceinline__ float4 lds4f(const __half* p)
{
    const uint2 t = *reinterpret_cast<const uint2*>(p);
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&t.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&t.y));
    return make_float4(a.x, a.y, b.x, b.y);
}

// Column pass along axis a (1 = Y, 2 = Z) of units [u0, u0 + nu): unit =
// ((xb * lines) + line) * nseg + seg; a line fixes the other two
// coordinates, xb a block of 64 columns, seg a run of kColS outputs.  The
// CTA stages the unit's kColS + B - 1 axis rows x 64 columns in shared
// memory (16-byte cp.async where rows are aligned, element copies at ragged
// edges; zero rows for the adjoint outside the image), the next unit's copy
// in flight while it computes the current one; each thread then computes 4
// rows x 4 columns (packed FMA over column pairs).
template <bool FIRST, class T, int B>
__device__ void col_pass(const BatchDesc& d, int a, const View& in, const View& out, bool out_f32,
                         const float2* s_w2, const float2* s_zw2, int u0, int nu, unsigned char* s_stage,
                         int stage_bytes)
{
    using TI = std::conditional_t<FIRST, T, float>;
    constexpr int R = B / 2;
    constexpr int EPC = 16 / (int)sizeof(TI);
    constexpr int CPR = 64 / EPC;                 // 16-byte chunks per staged row
    constexpr int ROWS = kColS + B - 1;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int n = a == 1 ? d.ny : d.nz;
    const int r = a == 1 ? d.ry : d.rz;
    const int zone = a == 1 ? d.zone_y : d.zone_z;
    const int no = a == 1 ? d.nz : d.ny;
    const long long in_sa = a == 1 ? in.s[1] : in.s[2], in_so = a == 1 ? in.s[2] : in.s[1];
    const long long out_sa = a == 1 ? out.s[1] : out.s[2], out_so = a == 1 ? out.s[2] : out.s[1];
    const long long sx = in.s[0];
    const int lines = d.nb * no;
    const int nseg = (n + kColS - 1) / kColS;
    const bool zoned = d.zero_pad && zone >= 0;
    // columns a 16-byte copy may cover: the scratch pitch (rows padded to 4
    // floats), or the extent for a source
    const int xlim = FIRST ? d.nx : (d.nx + 3) / 4 * 4;
    const TI* ip = reinterpret_cast<const TI*>(in.p);
    const bool vrow = sx == 1 && ((in_sa * (long long)sizeof(TI)) & 15) == 0 && ((in_so * (long long)sizeof(TI)) & 15) == 0 &&
                      ((in.s[3] * (long long)sizeof(TI)) & 15) == 0 && ((reinterpret_cast<uintptr_t>(ip) & 15) == 0);

    auto issue = [&](int u, TI* st) {
        const int seg = u % nseg;
        const int t = u / nseg;
        const int line = t % lines;
        const int xb = t / lines;
        const int o = line % no, b = line / no;
        const TI* base = ip + b * in.s[3] + o * in_so + (long long)(xb * 64) * sx;
        const int j0 = seg * kColS;
        for (int c = tid; c < ROWS * CPR; c += nt) {
            const int rr = c / CPR, q = c - (c / CPR) * CPR;
            TI* sd = st + rr * 64 + q * EPC;
            const int jm = sample_at(j0 - R + rr, n, r, d.border, d.zero_pad);
            const int x = xb * 64 + q * EPC;
            if (jm < 0 || x >= d.nx) {
                *reinterpret_cast<uint4*>(sd) = make_uint4(0u, 0u, 0u, 0u);
                continue;
            }
            const TI* src = base + (long long)jm * in_sa + (long long)(q * EPC) * sx;
            if (vrow && x + EPC <= xlim) {
                cp_async16(sd, src);
            } else {
#pragma unroll
                for (int e = 0; e < EPC; e++) sd[e] = (x + e < d.nx) ? src[(long long)e * sx] : TI(0.f);
            }
        }
    };

    TI* stage0 = reinterpret_cast<TI*>(s_stage);
    TI* stage1 = reinterpret_cast<TI*>(s_stage + stage_bytes);
    const int tx = tid & 15, ty = tid >> 4;     // columns 4tx.., rows 4ty.. (256 threads)
    if (nu > 0) issue(u0, stage0);
    cp_async_commit();
    for (int k = 0; k < nu; k++) {
        if (k + 1 < nu) issue(u0 + k + 1, (k & 1) ? stage0 : stage1);
        cp_async_commit();
        cp_async_wait1();
        __syncthreads();
        const TI* st = (k & 1) ? stage1 : stage0;
        const int u = u0 + k;
        const int seg = u % nseg;
        const int t = u / nseg;
        const int line = t % lines;
        const int xb = t / lines;
        const int o = line % no, b = line / no;
        const int j0 = seg * kColS + 4 * ty;
        const int j1 = min(n, (seg + 1) * kColS);
        const int x = xb * 64 + 4 * tx;
        if (j0 < j1 && x < d.nx) {
            float2 acc[4][2];
#pragma unroll
            for (int h = 0; h < 4; h++) acc[h][0] = acc[h][1] = make_float2(0.f, 0.f);
            const TI* rowp = st + (4 * ty) * 64 + 4 * tx;
            if (!zoned) {
#pragma unroll
                for (int i = 0; i < B + 3; i++) {
                    const float4 v = lds4f(rowp + i * 64);
                    const float2 lo = make_float2(v.x, v.y), hi = make_float2(v.z, v.w);
#pragma unroll
                    for (int h = 0; h < 4; h++) {
                        const int kk = i - h;
                        if (kk >= 0 && kk < B) {
                            acc[h][0] = __ffma2_rn(lo, s_w2[kk], acc[h][0]);
                            acc[h][1] = __ffma2_rn(hi, s_w2[kk], acc[h][1]);
                        }
                    }
                }
            } else {
                // adjoint, Clamp/Reflect: each row takes its own weight row --
                // the effective weights within the real radius of an axis end,
                // the flipped taps elsewhere (row 2r of the staged table)
                const float2* wr[4];
#pragma unroll
                for (int h = 0; h < 4; h++) {
                    const int e = zone_row(j0 + h, n, r);
                    wr[h] = s_zw2 + (e < 0 || j0 + h >= n ? 2 * r : e) * B;
                }
#pragma unroll
                for (int i = 0; i < B + 3; i++) {
                    const float4 v = lds4f(rowp + i * 64);
                    const float2 lo = make_float2(v.x, v.y), hi = make_float2(v.z, v.w);
#pragma unroll
                    for (int h = 0; h < 4; h++) {
                        const int kk = i - h;
                        if (kk >= 0 && kk < B) {
                            const float2 w = wr[h][kk];
                            acc[h][0] = __ffma2_rn(lo, w, acc[h][0]);
                            acc[h][1] = __ffma2_rn(hi, w, acc[h][1]);
                        }
                    }
                }
            }
            const long long obase = b * out.s[3] + o * out_so;
#pragma unroll
            for (int h = 0; h < 4; h++) {
                const int j = j0 + h;
                if (j >= j1) break;
                const long long oi = obase + (long long)j * out_sa + (long long)x * out.s[0];
                if (out_f32) {
                    // scratch rows are padded to 4 floats: the whole quad fits
                    *reinterpret_cast<float4*>(reinterpret_cast<float*>(const_cast<void*>(out.p)) + oi) =
                        make_float4(acc[h][0].x, acc[h][0].y, acc[h][1].x, acc[h][1].y);
                } else {
                    const float vals[4] = {acc[h][0].x, acc[h][0].y, acc[h][1].x, acc[h][1].y};
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        if (x + c < d.nx) store1<T>(const_cast<void*>(out.p), false, oi + (long long)c * out.s[0], vals[c]);
                }
            }
        }
        __syncthreads();   // the stage is refilled by the next iteration's copy
    }
    cp_async_wait0();
}

#define NDLGPU_BUCKETS(M) M(1) M(3) M(5) M(9) M(13) M(17) M(21) M(25) M(29) M(33) M(37)

template <bool FIRST, class T>
__device__ __forceinline__ void run_phase(const BatchDesc& d, int axis, int B, const View& in, const View& out,
                                          bool out_f32, const float* s_w, const float2* s_w2,
                                          const float* zones, const float2* s_zw2, int u0, int nu, float* s_buf,
                                          unsigned char* s_stage, int stage_bytes)
{
    if (axis == 0) {
        switch (B) {
#define NDLGPU_RC(BB) case BB: row_pass<FIRST, T, BB>(d, in, out, out_f32, s_w, zones, u0, nu, s_buf); break;
            NDLGPU_BUCKETS(NDLGPU_RC)
#undef NDLGPU_RC
        default: break;
        }
    } else {
        switch (B) {
#define NDLGPU_CC(BB) case BB: col_pass<FIRST, T, BB>(d, axis, in, out, out_f32, s_w2, s_zw2, u0, nu, s_stage, stage_bytes); break;
            NDLGPU_BUCKETS(NDLGPU_CC)
#undef NDLGPU_CC
        default: break;
        }
    }
}

constexpr int kMaxWarps = 8;
constexpr int kBufFloats = kSeg + 4 * ((kBatchMaxTaps + 6) / 4) + 4;

template <class T>
__global__ void __launch_bounds__(256, 3) k_batch(const BatchDesc* __restrict__ descs, const int4* __restrict__ items,
                                                 int nitems, int* __restrict__ counter,
                                                 const float* __restrict__ zones, float* __restrict__ scratch,
                                                 int stage_bytes)
{
    extern __shared__ __align__(16) unsigned char s_stage[];   // two column-pass stages
    __shared__ __align__(16) BatchDesc s_d;
    __shared__ __align__(16) float s_w[kBatchMaxTaps + 3];
    __shared__ __align__(16) float2 s_w2[kBatchMaxTaps + 3];
    // column passes of the adjoint with Clamp/Reflect: rows 0..2r-1 the
    // effective weights of the border positions, row 2r the flipped taps
    __shared__ __align__(16) float2 s_zw2[(kBatchMaxTaps + 1) * kBatchMaxTaps];
    __shared__ __align__(16) float s_buf[kMaxWarps][kBufFloats];
    __shared__ int s_item, s_skip;
    const int tid = threadIdx.x;
    int* work = counter;
    int* err = counter + 1;
    int* done = counter + 2;

    for (;;) {
        if (tid == 0) *(&s_item) = atomicAdd(work, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= nitems) break;
        const int4 item = items[it];
        {
            const int* src = reinterpret_cast<const int*>(descs + item.x);
            int* dstp = reinterpret_cast<int*>(&s_d);
            for (int i = tid; i < (int)(sizeof(BatchDesc) / 4); i += blockDim.x) dstp[i] = src[i];
        }
        const int phase = item.y;
        if (tid == 0) {
            s_skip = 0;
            if (phase > 0) {
                volatile int* dn = done + 3 * item.x + phase - 1;
                const int need = descs[item.x].nitems[phase - 1] + g_batch_need_bias;
                const int max_spins = g_batch_wait_spins;
                int spins = 0;
                while (*dn < need) {
                    __nanosleep(200);
                    if (++spins > max_spins) {
                        atomicExch(err, 1);
                        atomicOr(&g_guard_batch, 4);
                        s_skip = 1;
                        break;
                    }
                }
                __threadfence();
            }
        }
        __syncthreads();
        const BatchDesc& d = s_d;
        const int axis = d.pax[phase];
        const int B = axis == 0 ? d.bx : (axis == 1 ? d.by : d.bz);
        const float* wsrc = axis == 0 ? d.wx : (axis == 1 ? d.wy : d.wz);
        for (int i = tid; i < B; i += blockDim.x) {
            s_w[i] = wsrc[i];
            s_w2[i] = make_float2(wsrc[i], wsrc[i]);
        }
        const int zoff = axis == 0 ? d.zone_x : (axis == 1 ? d.zone_y : d.zone_z);
        if (axis != 0 && d.zero_pad && zoff >= 0) {
            const int rz2 = 2 * (axis == 1 ? d.ry : d.rz);
            for (int i = tid; i < (rz2 + 1) * B; i += blockDim.x) {
                const float w = i < rz2 * B ? zones[zoff + i] : wsrc[i - rz2 * B];
                s_zw2[i] = make_float2(w, w);
            }
        }
        __syncthreads();
        if (!s_skip) {
            // scratch layout: rows padded to a multiple of 4 floats
            const long long px = (d.nx + 3) / 4 * 4;
            const long long c1 = px, c2 = px * d.ny, c3 = px * d.ny * d.nz;
            View in, out;
            const bool first = phase == 0, last = phase == d.nphase - 1;
            if (first) {
                in.p = d.src;
                in.s[0] = d.sx; in.s[1] = d.sy; in.s[2] = d.sz; in.s[3] = d.sb;
            } else {
                in.p = scratch + d.scr[phase - 1];
                in.s[0] = 1; in.s[1] = c1; in.s[2] = c2; in.s[3] = c3;
            }
            if (last) {
                out.p = d.dst;
                out.s[0] = d.dx; out.s[1] = d.dy; out.s[2] = d.dz; out.s[3] = d.db;
            } else {
                out.p = scratch + d.scr[phase];
                out.s[0] = 1; out.s[1] = c1; out.s[2] = c2; out.s[3] = c3;
            }
            float* buf = s_buf[(tid >> 5) & (kMaxWarps - 1)];
            if (first)
                run_phase<true, T>(d, axis, B, in, out, !last, s_w, s_w2, zones, s_zw2, item.z, item.w, buf, s_stage, stage_bytes);
            else
                run_phase<false, T>(d, axis, B, in, out, !last, s_w, s_w2, zones, s_zw2, item.z, item.w, buf, s_stage, stage_bytes);
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) atomicAdd(done + 3 * item.x + phase, 1);
    }
}

template <class T>
cudaError_t prepare_b(int warps, BatchLaunch* L)
{
    if (warps != 8) return cudaErrorInvalidConfiguration;   // the column pass maps 16 x 16 threads
    const size_t smem = 2 * (size_t)L->stage_bytes;
    cudaError_t e = cudaFuncSetAttribute(k_batch<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch<T>, 32 * warps, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int dev = 0, sms = 148;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    L->grid = sms * per_sm;
    L->threads = 32 * warps;
    L->smem = smem;
    return cudaSuccess;
}

template <class T>
cudaError_t launch_b(const BatchLaunch& L, cudaStream_t s)
{
    k_batch<T><<<L.grid, L.threads, L.smem, s>>>(L.descs, L.items, L.nitems, L.counter, L.zones, L.scratch,
                                                 L.stage_bytes);
    count_launch();
    return cudaGetLastError();
}

// Tile configurations: warps per CTA, and the target number of outputs per
// work item (larger items: less scheduling, coarser balance).
struct TileCfg {
    int kout, warps;
};
const TileCfg kTiles[] = {{16, 8}, {64, 8}, {4, 8}, {256, 8}};

}  // namespace

int batch_tile_configs() { return (int)(sizeof(kTiles) / sizeof(kTiles[0])); }

void batch_tile_info(int i, int* tx, int* ty, int* nt)
{
    *tx = kTiles[i].kout;
    *ty = kTiles[i].warps;
    *nt = 32 * kTiles[i].warps;
}

int batch_item_outputs(int cfg) { return 1024 * kTiles[cfg].kout; }
int batch_row_segment() { return kSeg; }
int batch_col_unit() { return kColS; }

// Bytes of one column-pass stage for the widest taps B of a batch.
int batch_stage_bytes(int bmax) { return (kColS + bmax - 1) * 64 * 4; }

int batch_bucket(int k)
{
    const int b[] = {1, 3, 5, 9, 13, 17, 21, 25, 29, 33, 37};
    for (int v : b)
        if (k <= v) return v;
    return -1;
}

cudaError_t batch_prepare(int dtype, int cfg, BatchLaunch* L)
{
    const int w = kTiles[cfg].warps;
    switch (dtype) {
    case NDLGPU_F32: return prepare_b<float>(w, L);
    case NDLGPU_BF16: return prepare_b<__nv_bfloat16>(w, L);
    case NDLGPU_F16: return prepare_b<__half>(w, L);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t set_batch_wait_test(int spins, int need_bias)
{
    cudaError_t e = cudaMemcpyToSymbol(g_batch_wait_spins, &spins, sizeof(int));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(g_batch_need_bias, &need_bias, sizeof(int));
}

cudaError_t read_guard_batch(int32_t* v)
{
    int32_t zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(v, g_guard_batch, sizeof(int32_t));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(g_guard_batch, &zero, sizeof(int32_t));
}

cudaError_t launch_batch(int dtype, int cfg, const BatchLaunch& L, cudaStream_t s)
{
    (void)cfg;
    switch (dtype) {
    case NDLGPU_F32: return launch_b<float>(L, s);
    case NDLGPU_BF16: return launch_b<__nv_bfloat16>(L, s);
    case NDLGPU_F16: return launch_b<__half>(L, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace ndlgpu
