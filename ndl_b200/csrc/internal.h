// internal.h -- types shared by the host planner (host.cpp) and the kernel
// launchers (*.cu).  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/ndlgpu.h"

namespace ndlgpu {

constexpr int kMaxRank = NDLGPU_MAX_RANK;
constexpr int kMaxTaps = NDLGPU_MAX_TAPS;

// How a pass accumulates.
//   F32: FP32 fused multiply-add (float storage types).
//   F64: the reference's exact sequence, total = total + x*w with the
//        product and the sum each rounded (convolution.h:66-68).
//   I32: integer numerators of dyadic taps (w = m / 2^shift); exact.
enum class Acc : int { F32 = 0, F64 = 1, I32 = 2 };

// How an accumulator becomes DstT.
//   CAST : static_cast<DstT> -- truncation toward zero for integral DstT
//          (convolution.h:69); round-to-nearest for float DstT.
//   ROUND: std::round (half away from zero) first for integral DstT
//          (convolution.h:184).
//   RAW  : the accumulator itself, into a scratch buffer of the Acc type.
enum StoreMode : int { STORE_CAST = 0, STORE_ROUND = 1, STORE_RAW = 2 };

inline bool dtype_valid(int dt) { return dt >= NDLGPU_U8 && dt <= NDLGPU_BF16; }
inline bool dtype_integral(int dt) { return dt >= NDLGPU_U8 && dt <= NDLGPU_U64; }
inline int dtype_size(int dt)
{
    switch (dt) {
    case NDLGPU_U8: case NDLGPU_I8: return 1;
    case NDLGPU_U16: case NDLGPU_I16: case NDLGPU_F16: case NDLGPU_BF16: return 2;
    case NDLGPU_I32: case NDLGPU_U32: case NDLGPU_F32: return 4;
    default: return 8;
    }
}
inline int acc_dtype(Acc a)
{
    return a == Acc::F32 ? NDLGPU_F32 : (a == Acc::F64 ? NDLGPU_F64 : NDLGPU_I32);
}

// Unsigned 32-bit division by an invariant divisor with a multiply-high
// (Granlund & Montgomery, "Division by Invariant Integers using
// Multiplication", PLDI 1994, sec. 4): q = (mulhi(m, n) + n) >> l, evaluated
// without overflow as (t + ((n - t) >> 1)) >> (l - 1).
struct FastDiv {
    uint32_t d;
    uint32_t m;
    uint32_t l;
    void init(uint32_t div)
    {
        d = div;
        l = 0;
        while (l < 32 && (uint64_t(1) << l) < div) l++;
        m = (l == 0) ? 0u : uint32_t(((uint64_t(1) << 32) * ((uint64_t(1) << l) - div)) / div + 1);
    }
#ifdef __CUDACC__
    __device__ __forceinline__ uint32_t div(uint32_t n) const
    {
        if (l == 0) return n;
        uint32_t t = __umulhi(m, n);
        return (t + ((n - t) >> 1)) >> (l - 1);
    }
#endif
    uint32_t div_host(uint32_t n) const
    {
        if (l == 0) return n;
        uint32_t t = uint32_t((uint64_t(m) * n) >> 32);
        return (t + ((n - t) >> 1)) >> (l - 1);
    }
};

// One 1-D pass of the general kernel over a canonical geometry.
struct GenericPassParams {
    const char* src;
    char* dst;
    int src_dtype;
    int dst_dtype;
    int rank;
    int axis;
    int ntap;
    int border;
    int store_mode;
    int shift;            // Acc::I32: result = acc / 2^shift
    uint32_t total;       // outputs in this launch (< 2^32)
    int64_t n[kMaxRank];
    int64_t ss[kMaxRank]; // source strides (elements)
    int64_t ds[kMaxRank]; // destination strides (elements)
    FastDiv div[kMaxRank];
    int off[kMaxTaps];    // tap offsets, in summation order
    double wd[kMaxTaps];
    float wf[kMaxTaps];
    int32_t wi[kMaxTaps];
};

// One pass of any width along one axis, FP32 accumulation, float storage
// (pass_tiled.cu): canonical axes (0 = x, contiguous in neither necessarily),
// dense taps at offsets omin .. omax in ascending order.
constexpr int kTiledRank = 4;
struct TiledPassParams {
    const char* src;
    char* dst;
    int src_dtype, dst_dtype;
    int rank, axis, border;
    int ntap, omin, omax;
    int64_t rows;                 // product of the extents of every axis but 0
    int64_t n[kTiledRank], ss[kTiledRank], ds[kTiledRank];
    FastDiv dv[kTiledRank];       // dividers of the extents, of the tile count along x,
    FastDiv dtx;                  // and (strided pass) of the tile count along the axis
    FastDiv dta;
    float w[kMaxTaps];
};
bool tiled_pass_supported(const TiledPassParams& p);
cudaError_t launch_tiled_pass(const TiledPassParams& p, cudaStream_t s);

// The general N-D kernel (non-separable convolve()): taps live in device
// memory as ntap records of rank int32 offsets plus a double weight.
struct GenericNdParams {
    const char* src;
    char* dst;
    const int32_t* tap_off;  // ntap * rank
    const double* tap_w;     // ntap
    int src_dtype;
    int dst_dtype;
    int rank;
    int ntap;
    int border;
    int store_mode;
    uint32_t total;
    int64_t n[kMaxRank];
    int64_t ss[kMaxRank];
    int64_t ds[kMaxRank];
    FastDiv div[kMaxRank];
};

cudaError_t launch_generic_pass(Acc acc, const GenericPassParams& p, cudaStream_t s);
// Transposed pass: p.src = gradient at the pass output, p.dst = input gradient.
cudaError_t launch_pass_adjoint(Acc acc, const GenericPassParams& p, cudaStream_t s);

// Tap gradients of one pass: dw[t] = sum_i g[i] * x[map(i + off[t])].
struct TapGradParams {
    const char* g;
    const char* x;
    double* partial;      // [nblocks][ntap]
    int g_dtype;
    int x_dtype;
    int rank;
    int axis;
    int ntap;
    int border;
    uint32_t total;
    int64_t n[kMaxRank];
    int64_t gs[kMaxRank];
    int64_t xs[kMaxRank];
    FastDiv div[kMaxRank];
    int off[kMaxTaps];
};
unsigned tap_grad_blocks(uint32_t total);
cudaError_t launch_tap_grad(Acc acc, const TapGradParams& p, unsigned nblocks, void* out, int out_dtype,
                            cudaStream_t s);
cudaError_t launch_generic_nd(Acc acc, const GenericNdParams& p, cudaStream_t s);

// ---------------------------------------------------------------------------
// Fused separable forward (up to three pass axes, one HBM read + one write).
// Axis roles: X = canonical axis 0 (smallest source stride), Y and Z = the
// other pass axes (or extent-1 placeholders), batch = everything else.
struct FusedParams {
    const char* src;
    char* dst;
    int src_dtype;
    int dst_dtype;
    int border;
    int store_mode;
    int nx, ny, nz;
    int64_t sx, sy, sz;   // source strides (sx == 1 on the vector path)
    int64_t dx, dy, dz;   // destination strides
    int nbatch;           // product of batch extents (batch axes merged)
    int64_t sb, db;       // batch strides (merged batch must be affine)
    int kx, ky, kz;       // taps per axis (1 = no pass)
    int cx, cy, cz;       // centre = -(offset of tap 0)
    int shift;            // Acc::I32 total shift
    int zchunk;           // output planes per CTA along Z
    int vec_ld;           // source rows 16-byte aligned with sx == 1
    int vec_st;           // destination rows 4-element aligned with dx == 1
    int tstore;           // destination contiguous along Y: stores staged through shared memory
    // adjoint (input gradient): transposed passes.  zero_pad: out-of-range
    // samples read as 0 (Clamp/Reflect; Wrap keeps wrapped loads), and the
    // r = K/2 positions at each end of an axis use the effective weights
    // z?[e][k] over their K-wide window instead of the flipped taps (rows
    // e < r: positions 0..r-1; rows r..2r-1: positions n-r..n-1).
    int adj;
    int zero_pad;
    float zx[16][17], zy[16][17], zz[16][17];
    float wxf[64], wyf[64], wzf[64];
    int32_t wxi[64], wyi[64], wzi[64];
    float2 wx2[40], wy2[40], wz2[40];  // (w, w) pairs of the taps (packed FP32 FMA)
    int tma_pos[3];       // tensor-map dimension of y, z and batch (set at launch)
};

// Returns cudaErrorNotSupported when no compiled variant matches.
cudaError_t launch_fused(Acc acc, const FusedParams& p, cudaStream_t s);
bool fused_supported(Acc acc, int src_dtype, int dst_dtype, int kx, int ky, int kz);
// Float-storage fused kernel with asynchronous loads (fused2.cu).
cudaError_t launch_fused2(const FusedParams& p, cudaStream_t s);
bool fused2_supported(int src_dtype, int dst_dtype, int kx, int ky, int kz, int adj = 0);
// Fused forward of a uint8 volume with non-negative dyadic integer taps,
// two values packed per 32-bit word (fused_u8.cu): the compiled tap counts,
// and whether a planned launch qualifies (taps, bounds, layout).
bool fused_u8_shape(int sdt, int ddt, int kx, int ky, int kz);
bool fused_u8_supported(const FusedParams& p);
cudaError_t launch_fused_u8(const FusedParams& p, cudaStream_t s);
// Fused forward of a volume, Y pass first with every pass packed (fwd3.cu).
cudaError_t launch_fwd3(const FusedParams& p, cudaStream_t s);
bool fwd3_supported(int src_dtype, int dst_dtype, int kx, int ky, int kz);
// Reads and clears its guard word (bit 1: a tensor-map plane wait timed out),
// and sets the test controls of those waits (1 << 22 and 0: normal).
cudaError_t read_guard_fwd3(int32_t* v);
cudaError_t set_fwd3_wait_test(int spins, unsigned tx_bias);
// Reads and clears the fused kernels' guard word (bit 1: a plane load timed out).
cudaError_t read_guard_fused(int32_t* v);
// Test control of the tensor-map plane waits: poll bound and announced
// surplus bytes (kTmaSpins and 0 restore normal operation).
cudaError_t set_tma_wait_test(int spins, unsigned tx_bias);

// Sets the per-thread message ndlgpu_last_error() returns; returns s.
ndlgpu_status set_error(ndlgpu_status s, const std::string& msg);

// Number of Z chunks per tile column for a streaming kernel: minimises
// waves x (planes per chunk + halo planes), a wave being `slots` resident CTAs.
inline int pick_zchunks(long long tiles, long long slots, int nz, int halo)
{
    int best = 1;
    double best_t = 1e300;
    for (int c = 1; c <= 64 && c <= nz; c++) {
        const long long ctas = tiles * c;
        const long long waves = (ctas + slots - 1) / slots;
        const double t = (double)waves * ((double)((nz + c - 1) / c) + halo);
        if (t < best_t * 0.999) { best_t = t; best = c; }
    }
    return best;
}

// Process-wide count of kernel launches (ndlgpu_kernel_launches).
void count_launch(unsigned n = 1);

// Fused tap gradients of a three-pass chain (tapgrad.cu).  X strides
// (sx..sb) and G strides (gxs..gb) per canonical role; taps in ascending
// offset order (forward orientation), every tap present.
struct TapFusedParams {
    const char* x;
    const char* g;
    double* partial;      // [ncta][kx + ky + kz]
    int x_dtype;
    int border;
    int zero_pad;         // Clamp / Reflect: G read as zero outside the image
    int nx, ny, nz, nbatch;
    int64_t sx, sy, sz, sb;
    int64_t gxs, gy, gz, gb;
    int kx, ky, kz;
    int zchunk;
    int vec_ld;           // X rows 16-byte aligned, sx == 1
    int vec_g;            // G rows 4-element aligned, gxs == 1
    float wxf[64], wyf[64], wzf[64];
    // (w, w) pairs for packed FP32 FMA: X and Y taps, and the Z taps in
    // reverse order (window position m of Pz^T G weighs tap kz-1-m)
    float2 wx2[40], wy2[40], wzr2[40];
};
// Output slot of each canonical tap (x taps, then y, then z).
struct TapFinalMap {
    int dst[64];
};
bool tapgrad_supported(int dt, int kx, int ky, int kz);
long long tapgrad_ctas(const TapFusedParams& p);
int tapgrad_zchunk(int nx, int ny, int nz, int nbatch, int kz);
cudaError_t launch_tapgrad(const TapFusedParams& p, void* out, int out_dtype, const TapFinalMap& mp, cudaStream_t s);


// gradient (gradient.cu): all DIM central differences of a voxel in one pass.
struct GradParams {
    const char* src;
    char* dst;
    int sdt, ddt;
    int rank;                 // 1..3
    int border;
    int ext[3];
    int64_t sstr[3];          // source strides, elements
    int64_t dstr[4];          // destination strides: [0] the component axis
};
bool gradient_supported(const GradParams& p);
cudaError_t launch_gradient(const GradParams& p, cudaStream_t s);

// Difference-of-Gaussians scale space (dog.cu).
constexpr int kDogMaxLevels = 16;      // fused kernel; the per-level path takes up to kDogMaxScales
constexpr int kDogMaxScales = 64;
constexpr int kDogMaxRadius = 48;
struct DogParams {
    const char* src;
    int sdt;
    int nx, ny;
    int64_t sx, sy;                        // source strides, elements
    int ns;                                // levels
    int R;                                 // largest radius
    int r[kDogMaxLevels];
    float2 w2[kDogMaxLevels][2 * kDogMaxRadius + 1];   // (w, w) pairs of each level's taps
    float* lv[kDogMaxLevels];              // level outputs (NULL: not written)
    int64_t lx[kDogMaxLevels], ly[kDogMaxLevels];
    int lvec[kDogMaxLevels];               // x stride 1, 8-byte aligned rows: pair stores
    float* dg[kDogMaxLevels - 1];          // difference outputs
    int64_t gx[kDogMaxLevels - 1], gy[kDogMaxLevels - 1];
    int gvec[kDogMaxLevels - 1];
};
size_t dog2d_smem_bytes(int R);
cudaError_t launch_dog2d(const DogParams& p, cudaStream_t s);
struct SubParams {                         // dst = a - b in double, any rank
    const char* a;
    const char* b;
    char* dst;
    int adt, bdt, ddt;
    int rank;
    int64_t total;
    int64_t ext[kMaxRank], as[kMaxRank], bs[kMaxRank], ds[kMaxRank];
};
cudaError_t launch_sub(const SubParams& p, cudaStream_t s);

// downsample (downsample.cu): block averages, every axis but the channel axis.
struct DownParams {
    const char* src;
    char* dst;
    int sdt, ddt;
    int rank;
    int channel;
    int factor;
    int ext[kMaxRank];                     // source extents
    int oext[kMaxRank];                    // output extents
    int64_t sstr[kMaxRank], dstr[kMaxRank];
    int64_t total;                         // outputs (< 2^32)
    FastDiv odiv[kMaxRank];                // divisions by oext
    int nsub;                              // non-channel axes, ascending
    int sub[kMaxRank];
};
cudaError_t launch_downsample(const DownParams& p, cudaStream_t s);

// box_blur (boxblur.cu): the reference's summed-area-table arithmetic.
struct BoxParams {
    const char* src;
    char* dst;
    int sdt, ddt;
    int rank;
    int radius;
    int border;
    int ext[kMaxRank];
    int64_t sstr[kMaxRank], dstr[kMaxRank];
    int64_t pext[kMaxRank], pst[kMaxRank];   // padded extents and the table's strides
    int64_t npad;                            // table elements
    int64_t total;                           // outputs
    double area;                             // (2r+1)^DIM
    double* table;
};
cudaError_t launch_box_blur(const BoxParams& p, cudaStream_t s);

// gaussian_blur of 2-D integral images in the reference's double arithmetic
// (gauss_exact.cu).
struct GaussExactParams {
    const char* src;
    char* dst;
    int sdt, ddt, des;                     // des: destination element bytes
    int nx, ny, nb;                        // image extents, batch count
    int64_t sx, sy, sb, dx, dy, db;
    int kx, ky, cx, cy;
    int border;
    int store_mode;                        // STORE_ROUND (two passes) or STORE_CAST
    double wx[128], wy[128];
};
size_t gauss2d_exact_smem(int kx, int ky);
cudaError_t launch_gauss2d_exact(const GaussExactParams& p, cudaStream_t s);
// The exact z pass of a 3-D integral gaussian over a contiguous double
// volume (x fastest), rounded and cast into dst.
struct GaussZExactParams {
    const double* src;
    char* dst;
    int ddt;
    int nx, ny, nz;
    int64_t dx, dy, dz;
    int kz, cz;
    int border;
    double wz[128];
};
cudaError_t launch_gauss_z_exact(const GaussZExactParams& p, cudaStream_t s);

// Full 2-D / 3-D kernels on f32 images (stencil.cu).
constexpr int kStencilMaxTaps = 9;
struct StencilParams {
    const float* src;                      // f32 path (FP32 accumulation)
    float* dst;
    const char* srcc;                      // exact path: any <= 16-bit integral source,
    char* dstc;                            // any destination type
    int sdt, ddt;
    int nx, ny, nz, nb;                    // image extents (nz = 1 for images), batch count
    int64_t sx, sy, sz, sb, dx, dy, dz, db;
    int kx, ky, kz, cx, cy, cz;            // kernel extents and centres (K/2)
    int border;
    int tx, ty, tz, gx, gy;                // output box and grid (set at launch)
    int lgx, lgy;                          // log2(tx / 4), log2(ty)
    float w[kStencilMaxTaps * kStencilMaxTaps * kStencilMaxTaps];   // coordinates() order
    double wd[kStencilMaxTaps * kStencilMaxTaps * kStencilMaxTaps];  // the same taps, exact path
};
cudaError_t launch_stencil(StencilParams p, cudaStream_t s);
// The reference's own double sequence (bit-exact) for integral sources.
cudaError_t launch_stencil_exact(StencilParams p, cudaStream_t s);

// Batched form (batch.cu): one persistent launch over a table of instances.
constexpr int kBatchMaxTaps = 37;
struct BatchDesc {
    const void* src;
    void* dst;
    int nx, ny, nz, nb;
    long long sx, sy, sz, sb, dx, dy, dz, db;
    int bx, by, bz;           // compiled tap widths (odd; 1 = a single tap)
    int rx, ry, rz;           // radii of the real taps
    int border, zero_pad, vec_ld, vec_st;
    int nphase;               // passes of this instance, one axis each
    int pax[3];               // axis of each phase (0 = X, 1 = Y, 2 = Z), ascending
    int nitems[3];            // work items of each phase (dependency counts)
    int pad0;
    long long scr[2];         // element offsets of the f32 scratch after phases 0 and 1 (-1: none)
    int zone_x, zone_y, zone_z;   // offsets into the zone-table array (-1: none)
    float wx[kBatchMaxTaps], wy[kBatchMaxTaps], wz[kBatchMaxTaps];
};
struct BatchLaunch {
    const BatchDesc* descs;
    const int4* items;        // (instance, phase, first unit, units)
    int nitems;
    int* counter;             // [0] next item, [1] error flag, [2 + 3 i + p] finished items
    const float* zones;
    float* scratch;
    int grid;
    int threads;
    int stage_bytes;          // one column-pass stage (two are resident)
    size_t smem;
};
int batch_tile_configs();
void batch_tile_info(int i, int* tx, int* ty, int* nt);
int batch_bucket(int k);
int batch_item_outputs(int cfg);   // target outputs per work item
int batch_row_segment();           // row-pass outputs per warp segment
int batch_col_unit();              // column-pass outputs per unit along the axis
int batch_stage_bytes(int bmax);   // one column-pass stage for the widest taps
// Sets the kernel attributes and the persistent grid (no stream work).
cudaError_t batch_prepare(int dtype, int cfg, BatchLaunch* L);
cudaError_t launch_batch(int dtype, int cfg, const BatchLaunch& L, cudaStream_t s);
// Reads and clears the batched kernel's guard word (bit 2: a phase wait timed out).
cudaError_t read_guard_batch(int32_t* v);
// Test control of the batched phase waits: poll bound and extra
// predecessor items asked for (1 << 22 and 0 restore normal operation).
cudaError_t set_batch_wait_test(int spins, int need_bias);

// Device guard word.
cudaError_t read_device_status(cudaStream_t s, int32_t* code);

}  // namespace ndlgpu
