/*
 * ndl_oracle.c -- CPU restatement of ndl's separable-convolution path, in FP64.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load this library, and
 * only as the checker.  The product path (libndlgpu.so) never calls it.
 *
 * Every function follows the reference algorithm it cites (paths relative to
 * the ndl source tree):
 *   border maps          mathHelpers.h:23-25, image/detail.h:178-194
 *   kernel centre / taps image/detail.h:155-174  (centre K/2, zero taps skipped,
 *                        taps visited in coordinates() order = axis 0 fastest,
 *                        image/detail.h:127-143)
 *   convolve()           processing/convolution.h:52-71 (double accumulation,
 *                        total += double(src) * double(w) in tap order)
 *   gaussian weights     processing/convolution.h:116-126, mathHelpers.h:17-18
 *   final casts          processing/convolution.h:69 (static_cast, truncation
 *                        for integral types) and :180-185 (std::round, half
 *                        away from zero, for integral types)
 *
 * Views are {pointer, extent[], stride[]} in ndl axis order (axis 0 fastest
 * for a default layout, image/core.h:858-864), strides signed and in elements.
 * The adjoint and tap-gradient functions have no reference counterpart; they
 * are the literal transposes of the forward sum, written as scatters, so that
 * they are correct by construction.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORA_MAXDIM 8

enum { ORA_CLAMP = 0, ORA_WRAP = 1, ORA_REFLECT = 2 };

/* dtype codes shared with include/ndlgpu.h */
enum {
    ORA_U8 = 0, ORA_I8 = 1, ORA_U16 = 2, ORA_I16 = 3, ORA_I32 = 4, ORA_U32 = 5,
    ORA_I64 = 6, ORA_U64 = 7, ORA_F32 = 8, ORA_F64 = 9, ORA_F16 = 10, ORA_BF16 = 11
};

/* store modes: how the double total becomes DstT */
enum { ORA_STORE_CAST = 0 /* convolve(): static_cast, truncates integers */,
       ORA_STORE_ROUND = 1 /* gaussian_blur(): std::round then cast for integers */ };

/* mathHelpers.h:23-25 via detail.h:185-190.  One reflection / one wrap only;
 * callers guarantee |offset| <= M for Wrap and Reflect. */
static inline int64_t ora_map(int border, int64_t M, int64_t x)
{
    switch (border) {
    case ORA_WRAP:    return (x < 0) ? (x + M) : ((x >= M) ? (x - M) : x);
    case ORA_REFLECT: return (x < 0) ? (-x - 1) : ((x >= M) ? (2 * M - x - 1) : x);
    default:          return (x < 0) ? 0 : ((x >= M) ? (M - 1) : x);
    }
}

int ora_border_map(int border, int64_t M, int64_t x) { return (int)ora_map(border, M, x); }

/* Advance a coordinate in coordinates() order (axis 0 fastest). */
static inline int ora_next(int dim, const int64_t* ext, int64_t* c)
{
    for (int i = 0; i < dim; i++) {
        if (++c[i] < ext[i]) return 1;
        c[i] = 0;
    }
    return 0;
}

static inline int64_t ora_count(int dim, const int64_t* ext)
{
    int64_t n = 1;
    for (int i = 0; i < dim; i++) n *= ext[i];
    return n;
}

/*
 * convolve(): processing/convolution.h:52-71.  N-D kernel `kern` of extent
 * kext (contiguous, axis 0 fastest); taps with weight 0 are skipped
 * (detail.h:171-172); every axis of every tap goes through the border map
 * (detail.h:182-192).  Writes the double total (before the DstT cast).
 */
int ora_convolve(int dim, const double* src, const int64_t* ext, const int64_t* sstr,
                 double* dst, const int64_t* dstr,
                 const double* kern, const int64_t* kext, int border)
{
    if (dim < 1 || dim > ORA_MAXDIM) return -1;
    int64_t nk = ora_count(dim, kext);
    int64_t* tapc = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nk * dim + 1));
    double* tapw = (double*)malloc(sizeof(double) * (size_t)(nk + 1));
    int64_t ntap = 0;
    int64_t kc[ORA_MAXDIM] = {0};
    int64_t center[ORA_MAXDIM];
    for (int i = 0; i < dim; i++) center[i] = kext[i] / 2;   /* detail.h:161 */
    for (int64_t t = 0; t < nk; t++) {
        int64_t off = 0, mul = 1;
        for (int i = 0; i < dim; i++) { off += kc[i] * mul; mul *= kext[i]; }
        if (kern[off] != 0.0) {
            for (int i = 0; i < dim; i++) tapc[ntap * dim + i] = kc[i] - center[i];
            tapw[ntap] = kern[off];
            ntap++;
        }
        ora_next(dim, kext, kc);
    }
    int64_t n = ora_count(dim, ext);
    int64_t c[ORA_MAXDIM] = {0};
    for (int64_t e = 0; e < n; e++) {
        double total = 0.0;
        for (int64_t t = 0; t < ntap; t++) {
            int64_t so = 0;
            for (int i = 0; i < dim; i++)
                so += ora_map(border, ext[i], c[i] + tapc[t * dim + i]) * sstr[i];
            total += src[so] * tapw[t];
        }
        int64_t d = 0;
        for (int i = 0; i < dim; i++) d += c[i] * dstr[i];
        dst[d] = total;
        ora_next(dim, ext, c);
    }
    free(tapc);
    free(tapw);
    return 0;
}

/*
 * One 1-D pass along `axis` with taps w[0..K-1] at offsets k - center: the
 * same sum convolve() forms for a {1,..,K,..,1} kernel (convolution.h:132-139
 * builds exactly that kernel; extent-1 axes contribute offset 0).
 */
int ora_axis_pass(int dim, const double* src, const int64_t* ext, const int64_t* sstr,
                  double* dst, const int64_t* dstr,
                  int axis, int K, int center, const double* w, int border)
{
    if (dim < 1 || dim > ORA_MAXDIM || axis < 0 || axis >= dim) return -1;
    int64_t n = ora_count(dim, ext);
    int64_t c[ORA_MAXDIM] = {0};
    const int64_t M = ext[axis];
    for (int64_t e = 0; e < n; e++) {
        int64_t base = 0, d = 0;
        for (int i = 0; i < dim; i++) {
            if (i != axis) base += c[i] * sstr[i];
            d += c[i] * dstr[i];
        }
        double total = 0.0;
        for (int k = 0; k < K; k++) {
            if (w[k] == 0.0) continue;
            int64_t x = ora_map(border, M, c[axis] + k - center);
            total += src[base + x * sstr[axis]] * w[k];
        }
        dst[d] = total;
        ora_next(dim, ext, c);
    }
    return 0;
}

/*
 * Adjoint of ora_axis_pass with respect to its input: the literal transpose of
 * the forward sum.  For every output position i and tap k the forward pass
 * read x[map(i + k - c)] with weight w[k]; the adjoint scatters w[k] * g[i]
 * back to that position.  gx is accumulated into (caller zeroes it).
 */
int ora_axis_pass_adjoint(int dim, const double* g, const int64_t* ext, const int64_t* gstr,
                          double* gx, const int64_t* xstr,
                          int axis, int K, int center, const double* w, int border)
{
    if (dim < 1 || dim > ORA_MAXDIM || axis < 0 || axis >= dim) return -1;
    int64_t n = ora_count(dim, ext);
    int64_t c[ORA_MAXDIM] = {0};
    const int64_t M = ext[axis];
    for (int64_t e = 0; e < n; e++) {
        int64_t gb = 0, xb = 0;
        for (int i = 0; i < dim; i++) {
            gb += c[i] * gstr[i];
            if (i != axis) xb += c[i] * xstr[i];
        }
        double gv = g[gb];
        for (int k = 0; k < K; k++) {
            if (w[k] == 0.0) continue;
            int64_t x = ora_map(border, M, c[axis] + k - center);
            gx[xb + x * xstr[axis]] += w[k] * gv;
        }
        ora_next(dim, ext, c);
    }
    return 0;
}

/*
 * Gradient of L = sum(g * pass(x)) with respect to the taps of one 1-D pass:
 * dL/dw[k] = sum_i g[i] * x[map(i + k - c)].  Accumulated in double.
 */
int ora_axis_tap_grad(int dim, const double* g, const int64_t* ext, const int64_t* gstr,
                      const double* x, const int64_t* xstr,
                      int axis, int K, int center, int border, double* out)
{
    if (dim < 1 || dim > ORA_MAXDIM || axis < 0 || axis >= dim) return -1;
    int64_t n = ora_count(dim, ext);
    int64_t c[ORA_MAXDIM] = {0};
    const int64_t M = ext[axis];
    for (int k = 0; k < K; k++) out[k] = 0.0;
    for (int64_t e = 0; e < n; e++) {
        int64_t gb = 0, xb = 0;
        for (int i = 0; i < dim; i++) {
            gb += c[i] * gstr[i];
            if (i != axis) xb += c[i] * xstr[i];
        }
        double gv = g[gb];
        for (int k = 0; k < K; k++) {
            int64_t p = ora_map(border, M, c[axis] + k - center);
            out[k] += gv * x[xb + p * xstr[axis]];
        }
        ora_next(dim, ext, c);
    }
    return 0;
}

/* _kernelSize(sigma) = _ceil(3.0f * sigma): mathHelpers.h:17-18.  Note the
 * float literal: 3.0f * sigma is evaluated in double (sigma is double), and
 * _ceil truncates then bumps positive non-integers by one. */
int ora_gaussian_radius(double sigma)
{
    double num = 3.0f * sigma;
    int t = (int)num;
    return ((double)t == num) ? t : t + ((num > 0) ? 1 : 0);
}

/* Normalised Gaussian taps: processing/convolution.h:116-126.  w has room for
 * 2*radius+1 values; returns the width. */
int ora_gaussian_weights(double sigma, double* w)
{
    int radius = ora_gaussian_radius(sigma);
    int width = 2 * radius + 1;
    double wsum = 0;
    for (int i = 0; i < width; i++) {
        double d = i - radius;
        w[i] = exp(-(d * d) / (2 * sigma * sigma));
        wsum += w[i];
    }
    for (int i = 0; i < width; i++) w[i] /= wsum;
    return width;
}

/* IEEE binary16 / bfloat16 encode from double, round to nearest even
 * (decode is exact and done by the caller). */
static uint16_t ora_f32_to_bf16(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u && (u & 0x007fffffu)) return (uint16_t)((u >> 16) | 0x40);
    uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;
    return (uint16_t)(u >> 16);
}

/* Integral casts.  The reference's static_cast<DstT>(double) is undefined out
 * of range; x86-64 g++ truncates toward zero into a 32- or 64-bit register and
 * keeps the low bits.  In range, all choices agree. */
static int64_t ora_trunc_i64(double v)
{
    if (!(v > -9.2233720368547758e18 && v < 9.2233720368547758e18)) return INT64_MIN;
    return (int64_t)v;
}

/*
 * Casts the double totals to DstT (convolution.h:69 for ORA_STORE_CAST,
 * convolution.h:184 for ORA_STORE_ROUND).  Float targets round to nearest.
 */
int ora_cast(const double* v, int64_t n, int dtype, int mode, void* out)
{
    for (int64_t i = 0; i < n; i++) {
        double x = v[i];
        int is_int = dtype <= ORA_U64;
        if (is_int && mode == ORA_STORE_ROUND) x = round(x);
        switch (dtype) {
        case ORA_U8:  ((uint8_t*)out)[i] = (uint8_t)ora_trunc_i64(x); break;
        case ORA_I8:  ((int8_t*)out)[i] = (int8_t)(uint8_t)ora_trunc_i64(x); break;
        case ORA_U16: ((uint16_t*)out)[i] = (uint16_t)ora_trunc_i64(x); break;
        case ORA_I16: ((int16_t*)out)[i] = (int16_t)(uint16_t)ora_trunc_i64(x); break;
        case ORA_I32: ((int32_t*)out)[i] = (int32_t)(uint32_t)ora_trunc_i64(x); break;
        case ORA_U32: ((uint32_t*)out)[i] = (uint32_t)ora_trunc_i64(x); break;
        case ORA_I64: ((int64_t*)out)[i] = ora_trunc_i64(x); break;
        case ORA_U64: ((uint64_t*)out)[i] = (x >= 9.2233720368547758e18)
                          ? (uint64_t)ora_trunc_i64(x - 9.2233720368547758e18) + 0x8000000000000000ull
                          : (uint64_t)ora_trunc_i64(x); break;
        case ORA_F32: ((float*)out)[i] = (float)x; break;
        case ORA_F64: ((double*)out)[i] = x; break;
        case ORA_F16: {
            /* round to nearest even through the C compiler's _Float16 */
            _Float16 h = (_Float16)x;
            memcpy((uint16_t*)out + i, &h, 2);
            break;
        }
        case ORA_BF16: {
            /* double -> float is exact for every value that survives to bf16
             * except in rare double-rounding cases; decode via float first
             * exactly like a float32 pipeline storing bf16 would. */
            ((uint16_t*)out)[i] = ora_f32_to_bf16((float)x);
            break;
        }
        default: return -1;
        }
    }
    return 0;
}

/*
 * downsample(src, factor, channelAxis) -- processing/convolution.h:241-305.
 * Output extent: ext[a] on the channel axis, (ext[a] - 1) / factor + 1 on
 * every other.  Each output is the double sum of its block -- source indices
 * [o*factor, min(o*factor + factor, ext)) per non-channel axis -- walked as
 * the reference's odometer walks it (the lowest non-channel axis fastest,
 * :283-292), divided by the block's element count (:294).  The final cast
 * (std::round for integral T) is ora_cast's.  out is contiguous, axis 0
 * fastest.
 */
int ora_downsample(int dim, const double* src, const int64_t* ext, const int64_t* sstr, int factor, int channel,
                   double* out)
{
    if (dim < 2 || dim > 16 || factor < 2 || channel < 0 || channel >= dim) return -1;
    int64_t oext[16], oc[16], lo[16], hi[16], c[16];
    for (int a = 0; a < dim; a++) {
        oext[a] = (a == channel) ? ext[a] : (ext[a] - 1) / factor + 1;
        oc[a] = 0;
    }
    const int64_t n = ora_count(dim, oext);
    for (int64_t i = 0; i < n; i++) {
        int64_t count = 1;
        for (int a = 0; a < dim; a++) {
            if (a == channel) {
                lo[a] = oc[a];
                hi[a] = oc[a] + 1;
            } else {
                lo[a] = oc[a] * factor;
                hi[a] = lo[a] + factor < ext[a] ? lo[a] + factor : ext[a];
                count *= hi[a] - lo[a];
            }
            c[a] = lo[a];
        }
        double sum = 0;
        for (int64_t k = 0; k < count; k++) {
            int64_t off = 0;
            for (int a = 0; a < dim; a++) off += c[a] * sstr[a];
            sum += src[off];
            for (int a = 0; a < dim; a++) {
                if (a == channel) continue;
                if (++c[a] < hi[a]) break;
                c[a] = lo[a];
            }
        }
        out[i] = sum / (double)count;
        ora_next(dim, oext, oc);
    }
    return 0;
}

/*
 * box_blur(src, dst, radius, border) -- processing/summed_area_table.h:300-339.
 * 1. A padded copy of extent ext + 2r per axis, each position p holding the
 *    source value at the border-mapped p - r (:319-322).
 * 2. Its summed-area table in double (:48-88): the values, then one running
 *    sum per axis in axis order, each fiber summed from index 0 upward.
 * 3. Per output, rectangle_sum() over [c, c + 2r] (:117-137): the 2^DIM
 *    corners in mask order (bit i set: corner0[i] - 1 on axis i, sign
 *    flipped), corners with a negative coordinate skipped, each term
 *    sign * table added to the running total; then total / (2r+1)^DIM.
 * Writes the double quotients (the DstT static_cast is ora_cast's).
 * src is read through strides; out is contiguous (axis 0 fastest).
 */
int ora_box_blur(int dim, const double* src, const int64_t* ext, const int64_t* sstr, int radius, int border,
                 double* out)
{
    if (dim < 1 || dim > 16 || radius < 1) return -1;
    int64_t pext[16], pst[16], c[16];
    int64_t np = 1;
    for (int a = 0; a < dim; a++) {
        pext[a] = ext[a] + 2 * radius;
        pst[a] = np;
        np *= pext[a];
    }
    double* t = (double*)malloc((size_t)np * sizeof(double));
    if (!t) return -2;
    for (int a = 0; a < dim; a++) c[a] = 0;
    for (int64_t i = 0; i < np; i++) {
        int64_t off = 0;
        for (int a = 0; a < dim; a++) off += ora_map(border, ext[a], c[a] - radius) * sstr[a];
        t[i] = src[off];
        ora_next(dim, pext, c);
    }
    for (int axis = 0; axis < dim; axis++) {
        for (int a = 0; a < dim; a++) c[a] = 0;
        for (int64_t i = 0; i < np; i++) {
            if (c[axis] == 0) {
                int64_t off = 0;
                for (int a = 0; a < dim; a++) off += c[a] * pst[a];
                double running = 0.0;
                for (int64_t k = 0; k < pext[axis]; k++) {
                    running = running + t[off + k * pst[axis]];
                    t[off + k * pst[axis]] = running;
                }
            }
            ora_next(dim, pext, c);
        }
    }
    double area = 1.0;
    for (int a = 0; a < dim; a++) area *= (2 * radius + 1);
    const int64_t n = ora_count(dim, ext);
    for (int a = 0; a < dim; a++) c[a] = 0;
    for (int64_t i = 0; i < n; i++) {
        double total = 0.0;
        for (int mask = 0; mask < (1 << dim); mask++) {
            int sign = 1, oob = 0;
            int64_t off = 0;
            for (int a = 0; a < dim; a++) {
                const int low = (mask >> a) & 1;
                const int64_t q = low ? c[a] - 1 : c[a] + 2 * radius;
                if (low) sign = -sign;
                if (q < 0) { oob = 1; break; }
                off += q * pst[a];
            }
            if (oob) continue;
            total = total + sign * t[off];
        }
        out[i] = total / area;
        ora_next(dim, ext, c);
    }
    free(t);
    return 0;
}
