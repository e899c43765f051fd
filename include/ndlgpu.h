/*
 * ndlgpu.h -- C ABI of the B200 separable-convolution library (libndlgpu.so).
 *
 * Drop-in boundary for ndl's convolution hot path.  Every entry point below
 * replaces one reference interface; the citation is given per function
 * (paths relative to the ndl source tree).  The reference is a header-only
 * C++17 template library, so its "interface" is the template signature; the
 * C++ overloads in ndlgpu_dropin.h rebuild exactly those signatures on top of
 * this ABI.
 *
 * Conventions
 *   - Plain C: no C++ or torch types cross this boundary.  Status codes, never
 *     exceptions.  ndlgpu_last_error() gives a per-thread detail message.
 *   - Images are views {data, dtype, rank, extent[], stride[]} in ndl axis
 *     order (axis 0 fastest for a default layout, image/core.h:858-864),
 *     strides signed and in ELEMENTS -- exactly the triple an ndl::Image<T,DIM>
 *     carries after view()/slice()/swap_axes()/mirror() (image/core.h:50-972),
 *     with `data` = &image.at({0,..,0}).  Image data lives in device memory.
 *   - All work is asynchronous on the given CUDA stream (a cudaStream_t passed
 *     as void*; NULL = legacy default stream).  Host arrays given as arguments
 *     (kernels, sigmas, tap lists) are copied before the call returns.
 *   - Validation happens on the host, before any CUDA call: a call that
 *     returns an error has enqueued nothing.
 */
#ifndef NDLGPU_H
#define NDLGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define NDLGPU_API __attribute__((visibility("default")))
#else
#define NDLGPU_API
#endif

#define NDLGPU_MAX_RANK 8
/* Largest number of taps of one 1-D axis kernel (the fused kernels handle up
 * to 37 taps per axis, sigma = 6; longer kernels run the general kernels). */
#define NDLGPU_MAX_TAPS 255
/* Largest number of nonzero taps of a full N-D kernel given to
 * ndlgpu_convolve() (the non-separable general path). */
#define NDLGPU_MAX_ND_TAPS 4096

typedef enum ndlgpu_status {
    NDLGPU_OK = 0,
    NDLGPU_ERR_INVALID_ARGUMENT = 1,     /* null pointer, rank, axis, negative extent, ... */
    NDLGPU_ERR_UNSUPPORTED_DTYPE = 2,
    NDLGPU_ERR_EXTENT_MISMATCH = 3,      /* dst.extent != src.extent (convolution.h:59) */
    NDLGPU_ERR_RADIUS_EXCEEDS_EXTENT = 4,/* Wrap/Reflect tap beyond one period (mathHelpers.h:23-24) */
    NDLGPU_ERR_ALIASING = 5,             /* src and dst memory ranges overlap */
    NDLGPU_ERR_INDEX_OVERFLOW = 6,       /* a view spans more than 2^62 elements */
    NDLGPU_ERR_BAD_SIGMA = 7,            /* sigma <= 0 or not finite (convolution.h:112) */
    NDLGPU_ERR_WORKSPACE = 8,            /* caller workspace smaller than required */
    NDLGPU_ERR_CUDA = 9,                 /* a CUDA runtime call failed */
    NDLGPU_ERR_OUT_OF_MEMORY = 10,
    NDLGPU_ERR_TOO_MANY_TAPS = 11,
    NDLGPU_ERR_DEVICE_CHECK = 12         /* a kernel's own guard fired (see ndlgpu_device_status) */
} ndlgpu_status;

/* Element types.  bf16/f16 have no ndl counterpart (ndl accepts any
 * arithmetic T, convolution.h:57-58); they are storage formats here. */
typedef enum ndlgpu_dtype {
    NDLGPU_U8 = 0, NDLGPU_I8 = 1, NDLGPU_U16 = 2, NDLGPU_I16 = 3,
    NDLGPU_I32 = 4, NDLGPU_U32 = 5, NDLGPU_I64 = 6, NDLGPU_U64 = 7,
    NDLGPU_F32 = 8, NDLGPU_F64 = 9, NDLGPU_F16 = 10, NDLGPU_BF16 = 11
} ndlgpu_dtype;

/* Same order as ndl::BorderMode (image/border_mode.h:14-19). */
typedef enum ndlgpu_border {
    NDLGPU_CLAMP = 0, NDLGPU_WRAP = 1, NDLGPU_REFLECT = 2
} ndlgpu_border;

/* How a chain of 1-D passes turns into DstT.
 *  ROUND_ONCE: gaussian_blur()'s structure (convolution.h:148-185): passes
 *    accumulate without intermediate rounding; one final conversion, which
 *    is std::round (half away from zero) for integral DstT.  A single pass
 *    is a plain convolve() (truncating cast), as gaussian_blur()'s DIM==1
 *    branch (convolution.h:141-146).
 *  CAST_EACH: every pass is a complete convolve() into DstT (truncating for
 *    integral DstT, convolution.h:69) -- the chain a caller gets by calling
 *    convolve() once per axis. */
typedef enum ndlgpu_compose {
    NDLGPU_ROUND_ONCE = 0, NDLGPU_CAST_EACH = 1
} ndlgpu_compose;

/* Arithmetic.  AUTO: integral DstT and f64 data are computed bit-exactly
 * (integer arithmetic when every tap is a dyadic fraction, otherwise the
 * reference's own double sequence: each tap multiplied then added in
 * convolve()'s tap order, convolution.h:66-68); f32/f16/bf16 DstT accumulate
 * in FP32.  FP32: force FP32 accumulation.  EXACT: force the bit-exact
 * double sequence for every type (slower). */
typedef enum ndlgpu_precision {
    NDLGPU_PREC_AUTO = 0, NDLGPU_PREC_FP32 = 1, NDLGPU_PREC_EXACT = 2
} ndlgpu_precision;

typedef struct ndlgpu_view {
    void* data;                         /* &at({0,...,0}) */
    int32_t dtype;                      /* ndlgpu_dtype */
    int32_t rank;                       /* 1..NDLGPU_MAX_RANK */
    int64_t extent[NDLGPU_MAX_RANK];
    int64_t stride[NDLGPU_MAX_RANK];    /* elements, signed */
} ndlgpu_view;

/* One 1-D pass: taps[k] weighs the sample at offset k - center along `axis`
 * (ndl centres kernels at K/2, image/detail.h:155-163; zero taps are
 * skipped, image/detail.h:171-172).  taps is host memory. */
typedef struct ndlgpu_axis_kernel {
    int32_t axis;
    int32_t ntaps;
    int32_t center;
    int32_t reserved;                   /* must be 0 */
    const double* taps;
} ndlgpu_axis_kernel;

/* ---- library information ------------------------------------------------ */
NDLGPU_API const char* ndlgpu_version(void);
NDLGPU_API const char* ndlgpu_status_string(ndlgpu_status s);
/* Detail of the last error returned on this host thread ("" if none). */
NDLGPU_API const char* ndlgpu_last_error(void);

/* ---- forward ------------------------------------------------------------ */

/* ndl::convolve(src, dst, kernel, border)  -- processing/convolution.h:52-71.
 * `kernel` is a HOST view of any dtype and the image's rank (each value is
 * converted to double, convolution.h:68).  A kernel whose extent exceeds 1
 * along one axis only is run by the separable kernels; any other kernel by
 * the general N-D kernel.  Integral DstT truncates toward zero; arithmetic
 * per ndlgpu_precision AUTO. */
NDLGPU_API ndlgpu_status ndlgpu_convolve(const ndlgpu_view* src, const ndlgpu_view* dst,
                              const ndlgpu_view* kernel, int border, void* stream);

/* As ndlgpu_convolve with an explicit precision. */
NDLGPU_API ndlgpu_status ndlgpu_convolve_ex(const ndlgpu_view* src, const ndlgpu_view* dst,
                                 const ndlgpu_view* kernel, int border, int precision,
                                 void* stream);

/* ndl::gradient(src, dst, border)  -- processing/convolution.h:359-388.
 * dst has rank(src) + 1 axes, a leading component axis of extent rank(src)
 * and then src's extents ({DIM, ...}); dst.slice(0, a) receives the central
 * difference along axis a, i.e. convolve() with the {-0.5, 0, +0.5} taps
 * along that axis (zero centre tap skipped, truncation for integral DstT).
 * The reference's default border is Reflect. */
NDLGPU_API ndlgpu_status ndlgpu_gradient(const ndlgpu_view* src, const ndlgpu_view* dst, int border, void* stream);

/* ndl::box_blur(src, dst, radius, border) -- processing/summed_area_table.h:300-339.
 * The (2 radius + 1)^DIM box average through a summed-area table in double,
 * built and queried exactly as the reference does (border-mapped padding,
 * sequential running sums per axis, inclusion-exclusion over the 2^DIM
 * corners, then sum / (2r+1)^DIM and DstT's static_cast), so the results
 * equal the reference's bit for bit.  radius > 0; Wrap/Reflect need radius
 * <= every extent.  The table (8 bytes per element of the padded extent)
 * lives in `workspace` (at least ndlgpu_box_blur_workspace_size() bytes) or,
 * with workspace NULL, in stream-ordered scratch. */
NDLGPU_API ndlgpu_status ndlgpu_box_blur(const ndlgpu_view* src, const ndlgpu_view* dst, int radius, int border,
                                         void* workspace, size_t workspace_bytes, void* stream);
NDLGPU_API ndlgpu_status ndlgpu_box_blur_workspace_size(const ndlgpu_view* src, const ndlgpu_view* dst, int radius,
                                                        int border, size_t* bytes);

/* ndl::downsample(src, factor, channelAxis, border) -- processing/convolution.h:241-305.
 * Every axis but channel_axis shrinks to (extent - 1) / factor + 1 (dst must
 * have those extents; the reference returns a new image of them); each
 * output is the average of its non-overlapping factor-wide source block (a
 * short last block averages the samples that exist), summed in double in the
 * reference's block order and then std::round-ed for integral dst types, so
 * the results equal the reference's bit for bit when dst has src's type.
 * factor > 1; rank >= 2; `border` is accepted and unused, as in the
 * reference. */
NDLGPU_API ndlgpu_status ndlgpu_downsample(const ndlgpu_view* src, const ndlgpu_view* dst, int factor,
                                           int channel_axis, int border, void* stream);

/* The Difference-of-Gaussians scale space of ndl::detect_keypoints
 * (processing/feature_detection.h:101-122): num_scales (4..64) levels,
 * level i = gaussian_blur(src as double, sigma_i, Reflect) with
 * sigma_i = sigma0 * 2^(i / (num_scales - 3)), and num_scales - 1 differences
 * dogs[i] = level[i+1] - level[i].  `dogs` points to num_scales - 1 views,
 * `levels` to num_scales views or is NULL; all are F32 or F64 images of src's
 * extent that overlap neither src nor each other.  2-D images with F32
 * outputs (up to 16 levels, radius <= 48, sources exact in float) run one
 * kernel that reads the source once and writes every output (FP32
 * accumulation); other cases run one blur per level plus a difference pass
 * (FP64 outputs get the reference's exact double sequence) with
 * stream-ordered scratch for the levels the caller does not take. */
NDLGPU_API ndlgpu_status ndlgpu_dog_scale_space(const ndlgpu_view* src, int num_scales, double sigma0,
                                                const ndlgpu_view* levels, const ndlgpu_view* dogs, void* stream);

/* ndl::gaussian_blur(src, dst, sigma, border) -- processing/convolution.h:107-186.
 * Radius ceil(3*sigma) (mathHelpers.h:17-18), weights exp(-d^2/(2 sigma^2))
 * normalised in double on the host (convolution.h:116-126), one pass per
 * axis, one final rounding for integral DstT.  `workspace` may be NULL (the
 * library then allocates stream-ordered scratch) or at least the size
 * reported by ndlgpu_gaussian_blur_workspace_size(). */
NDLGPU_API ndlgpu_status ndlgpu_gaussian_blur(const ndlgpu_view* src, const ndlgpu_view* dst,
                                   double sigma, int border,
                                   void* workspace, size_t workspace_bytes, void* stream);
NDLGPU_API ndlgpu_status ndlgpu_gaussian_blur_workspace_size(const ndlgpu_view* src, const ndlgpu_view* dst,
                                                  double sigma, int border, size_t* bytes);

/* gaussian_blur() generalised to one sigma per axis (sigma[a] == 0 leaves
 * axis a untouched).  Same weights, structure and rounding as
 * ndlgpu_gaussian_blur; passes run in axis order. */
NDLGPU_API ndlgpu_status ndlgpu_gaussian_blur_axes(const ndlgpu_view* src, const ndlgpu_view* dst,
                                        const double* sigma_per_axis, int border,
                                        void* workspace, size_t workspace_bytes, void* stream);

/* A chain of 1-D passes (each a convolve() with a {1,..,K,..,1} kernel, the
 * kernel gaussian_blur() builds at convolution.h:132-139) applied in order,
 * composed per `compose` (ndlgpu_compose) with arithmetic per `precision`. */
NDLGPU_API ndlgpu_status ndlgpu_convolve_axes(const ndlgpu_view* src, const ndlgpu_view* dst,
                                   int npass, const ndlgpu_axis_kernel* passes,
                                   int border, int compose, int precision,
                                   void* workspace, size_t workspace_bytes, void* stream);
NDLGPU_API ndlgpu_status ndlgpu_convolve_axes_workspace_size(const ndlgpu_view* src, const ndlgpu_view* dst,
                                                  int npass, const ndlgpu_axis_kernel* passes,
                                                  int border, int compose, int precision,
                                                  size_t* bytes);

/* ---- adjoint (no reference counterpart: the reference has no gradients) --
 * For Y = P_n(...P_1(X)) (ROUND_ONCE composition, float types) and
 * L = sum(grad_out * Y):
 *   grad_src  (may be NULL)  <- dL/dX, the border-aware transpose: Clamp folds
 *             out-of-range taps onto the edge samples, Reflect onto their
 *             mirror images, Wrap onto the opposite end.
 *   grad_taps (may be NULL)  <- dL/dw for every tap of every pass, back to
 *             back in pass order (sum of ntaps values, dtype grad_taps_dtype
 *             F32 or F64, device memory).  Needs `src` (the forward input).
 * Deterministic: tap gradients are reduced in a fixed two-stage order. */
NDLGPU_API ndlgpu_status ndlgpu_convolve_axes_adjoint(const ndlgpu_view* grad_out, const ndlgpu_view* src,
                                           const ndlgpu_view* grad_src,
                                           int npass, const ndlgpu_axis_kernel* passes, int border,
                                           void* grad_taps, int grad_taps_dtype,
                                           void* workspace, size_t workspace_bytes, void* stream);
NDLGPU_API ndlgpu_status ndlgpu_convolve_axes_adjoint_workspace_size(const ndlgpu_view* grad_out, const ndlgpu_view* src,
                                                          const ndlgpu_view* grad_src,
                                                          int npass, const ndlgpu_axis_kernel* passes,
                                                          int border, int grad_taps_dtype, size_t* bytes);

/* ---- batched form (no reference counterpart) ------------------------------
 * Many images and volumes of uneven extents, tap counts and border modes in
 * ONE persistent launch.  Each instance is a chain of at most three 1-D
 * passes on distinct axes of one view (its other axes are left untouched),
 * with odd, centred tap lists of at most 37 taps, composed like
 * gaussian_blur() with FP32 accumulation; `adjoint` = 1 runs the transposed
 * chain (the input gradient of that instance).  All instances of a batch share
 * one storage type, F32, BF16 or F16 (src and dst alike).  Taps are padded
 * to compiled widths {1,3,5,9,...,37} with zero weights; inputs are assumed
 * finite (a padded zero tap multiplies its sample).
 * The launch runs every instance's passes one axis at a time, with FP32
 * intermediates in device scratch the plan allocates; Wrap/Reflect passes
 * need their radius within the axis extent (as the reference's one-period
 * border maps do).
 * Workflow: create, add instances, plan (uploads the instance table and the
 * work list, ordered by pass and cost, and allocates the scratch), then
 * launch or graph_launch as often as needed; the instance views keep their
 * addresses between launches.  A graph_launch captures the launch into a CUDA
 * graph on first use and replays it afterwards.  tile_config selects one of
 * ndlgpu_batch_tile_configs() work-item configurations (-1: the default);
 * ndlgpu_batch_tile_config_info reports for each the target outputs per work
 * item in units of 1024 (tile_x), the warps per CTA (tile_y) and the threads
 * per CTA. */
typedef struct ndlgpu_batch ndlgpu_batch;
NDLGPU_API ndlgpu_status ndlgpu_batch_create(ndlgpu_batch** out);
NDLGPU_API ndlgpu_status ndlgpu_batch_add(ndlgpu_batch* b, const ndlgpu_view* src, const ndlgpu_view* dst,
                                          int npass, const ndlgpu_axis_kernel* passes, int border, int adjoint);
NDLGPU_API ndlgpu_status ndlgpu_batch_plan(ndlgpu_batch* b, int tile_config);
NDLGPU_API ndlgpu_status ndlgpu_batch_launch(ndlgpu_batch* b, void* stream);
NDLGPU_API ndlgpu_status ndlgpu_batch_graph_launch(ndlgpu_batch* b, void* stream);
NDLGPU_API ndlgpu_status ndlgpu_batch_destroy(ndlgpu_batch* b);
NDLGPU_API int ndlgpu_batch_tile_configs(void);
NDLGPU_API ndlgpu_status ndlgpu_batch_tile_config_info(int index, int* tile_x, int* tile_y, int* threads);
/* Instances, work items and total output elements of a planned batch. */
NDLGPU_API ndlgpu_status ndlgpu_batch_info(const ndlgpu_batch* b, int* instances, int* items, int64_t* elements);

/* ---- allocation-free gaussian_blur ---------------------------------------
 * No counterpart in the reference.  Some callers cannot allocate device
 * memory: plugins hosted by an application that owns the GPU's memory pool
 * and forbids allocations behind its back, real-time loops that must never
 * reach the allocator (cudaMalloc can synchronise the device and takes an
 * unbounded time), and code held to a static memory budget.  This entry point
 * is ndlgpu_gaussian_blur with its scratch taken from a fixed device array
 * inside libndlgpu.so, so it calls no allocating routine; the caller still
 * passes src and dst.
 *   - The array is NDLGPU_NOALLOC_SCRATCH_BYTES (16 MiB); every GPU that loads
 *     the library holds it until the process exits.  A blur whose scratch
 *     (ndlgpu_gaussian_blur_workspace_size) exceeds it returns
 *     NDLGPU_ERR_WORKSPACE and enqueues nothing.
 *   - The first call on a device looks up the array's device address with the
 *     device current; make that first call before any stream capture.
 *   - All calls share the one array: calls that overlap on the GPU (other
 *     streams, other host threads) race.  The blur writes every scratch
 *     element before reading it, so the array needs no clearing between
 *     calls. */
#define NDLGPU_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
NDLGPU_API ndlgpu_status ndlgpu_gaussian_blur_noalloc(const ndlgpu_view* src, const ndlgpu_view* dst,
                                                      double sigma, int border, void* stream);

/* ---- instrumentation ---------------------------------------------------- */
/* Number of CUDA kernels this library has launched in this process (all
 * devices, all threads); no reference counterpart. */
NDLGPU_API uint64_t ndlgpu_kernel_launches(void);

/* ---- device guard word -------------------------------------------------- */
/* Reads (and clears) the library's device-side guard words on the current
 * device after synchronising `stream`: 0 if no kernel guard fired.  Bit 1: a
 * fused adjoint plane load did not complete within its bounded wait; bit 2: a
 * batched phase wait ran past its bound (the work item was dropped); other
 * bits are reserved. */
NDLGPU_API ndlgpu_status ndlgpu_device_status(void* stream, int32_t* code);

/* Test control of the bounded device waits on the current device; no
 * reference counterpart.  spin_limit > 0 bounds every tensor-map plane wait
 * and batched phase wait to that many polls; unreachable != 0 makes each of
 * those waits ask for more than ever arrives (plane loads announce 16 bytes
 * they never deliver, phase waits one predecessor item too many), so that
 * they run out: the kernel then sets its guard bit, lets its own copies in
 * flight land (bounded) and returns, and ndlgpu_device_status reports it.
 * Nothing faults.  ndlgpu_test_wait_timeouts(0, 0) restores normal
 * operation. */
NDLGPU_API ndlgpu_status ndlgpu_test_wait_timeouts(int spin_limit, int unreachable);

#ifdef __cplusplus
}
#endif

#endif /* NDLGPU_H */
