// ref_shim.cpp -- C entry points over the UNMODIFIED ndl reference.
//
// TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline).  Compiled by
// oracle/build_oracle.py against the reference's own headers into
// oracle/_ref/libndlref.so; nothing here re-implements the reference's
// arithmetic.  Every numeric result comes from ndl::convolve() /
// ndl::gaussian_blur() (processing/convolution.h:52-71, :107-186).
//
// Arbitrary {pointer, extent, stride} views reach ndl::convolve() through
// ndl's own extension point: convolve() is templated on any type exposing the
// minimal interface extent()/at()/coordinates() (image/detail.h:48-57), so
// StridedView below is such a type whose at() is the same signed-stride dot
// product Image::at() computes (image/core.h:557-558).  ref_view_probe() runs
// the reference's real Image view builders (view/swap_axes/mirror,
// image/core.h:647-757) so the host-side view arithmetic can be pinned to it.
// ref_detect_keypoints() runs ndl::detect_keypoints() itself, whose keypoints
// carry the Difference-of-Gaussians values (processing/feature_detection.h).
#include <ndl/image.h>
#include <ndl/processing/convolution.h>
#include <ndl/processing/feature_detection.h>
#include <ndl/processing/summed_area_table.h>

#include <array>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>

namespace {

template <class T, int DIM>
struct StridedView {
    using value_type = T;
    T* p;
    std::array<int, DIM> ext;
    std::array<int, DIM> str;
    const std::array<int, DIM>& extent() const { return ext; }
    const std::array<int, DIM>& stride() const { return str; }
    T& at(const std::array<int, DIM>& c) const
    {
        long long o = 0;
        for (int i = 0; i < DIM; i++) o += (long long)c[i] * str[i];
        return p[o];
    }
    std::vector<std::array<int, DIM>> coordinates() const { return ndl::detail::coordinatesOf(ext); }
    // the rank-(DIM-1) view at `index` along axis d, as Image::slice()
    // builds it (image/core.h:709-712, :814-823); ndl::gradient() uses it
    template <int D = DIM, std::enable_if_t<(D > 1), int> = 0>
    StridedView<T, DIM - 1> slice(int d, int index) const
    {
        StridedView<T, DIM - 1> v;
        v.p = p + (long long)index * str[d];
        for (int i = 0, j = 0; i < DIM; i++) {
            if (i == d) continue;
            v.ext[j] = ext[i];
            v.str[j] = str[i];
            j++;
        }
        return v;
    }
};

template <class T, int DIM>
StridedView<T, DIM> make_view(void* p, const int* ext, const int* str)
{
    StridedView<T, DIM> v;
    v.p = static_cast<T*>(p);
    for (int i = 0; i < DIM; i++) { v.ext[i] = ext[i]; v.str[i] = str[i]; }
    return v;
}

ndl::BorderMode to_border(int b)
{
    return b == 1 ? ndl::BorderMode::Wrap : (b == 2 ? ndl::BorderMode::Reflect : ndl::BorderMode::Clamp);
}

// dtype codes shared with include/ndlgpu.h
enum { U8 = 0, I8 = 1, U16 = 2, I16 = 3, I32 = 4, U32 = 5, I64 = 6, U64 = 7, F32 = 8, F64 = 9 };

template <class F>
int dispatch_type(int code, F&& f)
{
    switch (code) {
    case U8: return f((uint8_t)0);
    case I8: return f((int8_t)0);
    case U16: return f((uint16_t)0);
    case I16: return f((int16_t)0);
    case I32: return f((int32_t)0);
    case U32: return f((uint32_t)0);
    case F32: return f((float)0);
    case F64: return f((double)0);
    default: return -2;
    }
}

template <class F>
int dispatch_dim(int dim, F&& f)
{
    switch (dim) {
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    case 3: return f(std::integral_constant<int, 3>{});
    case 4: return f(std::integral_constant<int, 4>{});
    default: return -3;
    }
}

// Builds the {1,..,K,..,1} axis kernel exactly as gaussian_blur's
// buildAxisKernel does (processing/convolution.h:132-139), over caller storage.
template <int DIM>
ndl::Image<double, DIM> axis_kernel(int axis, int K, const double* w, std::vector<double>& store)
{
    store.assign((size_t)K, 0.0);
    std::array<int, DIM> kext;
    for (int i = 0; i < DIM; i++) kext[i] = (i == axis) ? K : 1;
    ndl::Image<double, DIM> k(store.data(), kext);
    std::array<int, DIM> kc{};
    for (int i = 0; i < K; i++) { kc[axis] = i; k.at(kc) = w[i]; }
    return k;
}

}  // namespace

extern "C" {

// ndl::per_channel(src, dst, channelAxis, fn) (image/kernels.h:78-87) with fn
// = gaussian_blur(s, d, sigma, border) on every channel slice, on contiguous
// images (axis 0 fastest) of one type.
int ref_per_channel_blur(int dim, int tsrc, void* src, const int* ext, int channel_axis, double sigma, int border,
                         void* dst)
{
    return dispatch_dim(dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        if constexpr (DIM < 2) {
            return -4;
        } else {
            return dispatch_type(tsrc, [&](auto s) {
                using S = decltype(s);
                std::array<int, DIM> e;
                for (int i = 0; i < DIM; i++) e[i] = ext[i];
                ndl::Image<S, DIM> in(static_cast<S*>(src), e);
                ndl::Image<S, DIM> out(static_cast<S*>(dst), e);
                const ndl::BorderMode b = to_border(border);
                ndl::per_channel(in, out, channel_axis, [&](auto si, auto di) { ndl::gaussian_blur(si, di, sigma, b); });
                return 0;
            });
        }
    });
}

// ndl::box_blur(src, dst, radius, border) (processing/summed_area_table.h:300-339).
int ref_box_blur(int dim, int tsrc, void* src, const int* ext, const int* sstr, int tdst, void* dst, const int* dstr,
                 int radius, int border)
{
    return dispatch_dim(dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        return dispatch_type(tsrc, [&](auto s) {
            using S = decltype(s);
            return dispatch_type(tdst, [&](auto d) {
                using Dt = decltype(d);
                auto sv = make_view<S, DIM>(src, ext, sstr);
                auto dv = make_view<Dt, DIM>(dst, ext, dstr);
                ndl::box_blur(sv, dv, radius, to_border(border));
                return 0;
            });
        });
    });
}

// ndl::downsample(src, factor, channelAxis) (processing/convolution.h:241-305)
// on a contiguous image (axis 0 fastest); its result, of src's type, is
// copied to dst (contiguous).
int ref_downsample(int dim, int tsrc, void* src, const int* ext, int factor, int channel_axis, void* dst)
{
    return dispatch_dim(dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        if constexpr (DIM < 2) {
            return -4;
        } else {
            return dispatch_type(tsrc, [&](auto s) {
                using S = decltype(s);
                std::array<int, DIM> e;
                for (int i = 0; i < DIM; i++) e[i] = ext[i];
                ndl::Image<S, DIM> img(static_cast<S*>(src), e);
                auto out = ndl::downsample(img, factor, channel_axis);
                S* o = static_cast<S*>(dst);
                size_t k = 0;
                for (const auto& c : out.coordinates()) o[k++] = out.at(c);
                return 0;
            });
        }
    });
}

// ndl::detect_keypoints(src, num_scales, sigma0, threshold) on a contiguous
// double image (axis 0 fastest).  Writes up to max_n keypoints -- position
// (dim ints each), scale and response -- and returns their count, or -1 when
// there are more than max_n.
int ref_detect_keypoints(int dim, double* src, const int* ext, int num_scales, double sigma0, double threshold,
                         int* pos, double* scale, double* response, int max_n)
{
    return dispatch_dim(dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        std::array<int, DIM> e;
        for (int i = 0; i < DIM; i++) e[i] = ext[i];
        ndl::Image<double, DIM> img(src, e);
        const auto kps = ndl::detect_keypoints(img, num_scales, sigma0, threshold);
        if ((int)kps.size() > max_n) return -1;
        for (size_t k = 0; k < kps.size(); k++) {
            for (int i = 0; i < DIM; i++) pos[k * DIM + i] = kps[k].position[i];
            scale[k] = kps[k].scale;
            response[k] = kps[k].response;
        }
        return (int)kps.size();
    });
}

// ndl::gradient(src, dst, border) (processing/convolution.h:359-388): dst of
// extent {dim, ext...} with strides dstr[0..dim].
int ref_gradient(int dim, int tsrc, void* src, const int* ext, const int* sstr, int tdst, void* dst, const int* dstr,
                 int border)
{
    return dispatch_dim(dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        return dispatch_type(tsrc, [&](auto s) {
            using S = decltype(s);
            return dispatch_type(tdst, [&](auto d) {
                using Dt = decltype(d);
                auto sv = make_view<S, DIM>(src, ext, sstr);
                int dext[DIM + 1];
                dext[0] = DIM;
                for (int i = 0; i < DIM; i++) dext[i + 1] = ext[i];
                auto dv = make_view<Dt, DIM + 1>(dst, dext, dstr);
                ndl::gradient(sv, dv, to_border(border));
                return 0;
            });
        });
    });
}

// ndl::convolve(src, dst, kernel, border) on arbitrary strided views; kernel
// is a contiguous double array of extent kext (axis 0 fastest).
int ref_convolve(int dim, int tsrc, void* src, const int* ext, const int* sstr,
                 int tdst, void* dst, const int* dstr,
                 const double* kern, const int* kext, int border)
{
    return dispatch_dim(dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        return dispatch_type(tsrc, [&](auto s) {
            using S = decltype(s);
            return dispatch_type(tdst, [&](auto d) {
                using Dt = decltype(d);
                auto sv = make_view<S, DIM>(src, ext, sstr);
                auto dv = make_view<Dt, DIM>(dst, ext, dstr);
                std::array<int, DIM> ke;
                for (int i = 0; i < DIM; i++) ke[i] = kext[i];
                ndl::Image<double, DIM> k(const_cast<double*>(kern), ke);
                ndl::convolve(sv, dv, k, to_border(border));
                return 0;
            });
        });
    });
}

// ndl::gaussian_blur(src, dst, sigma, border).
int ref_gaussian_blur(int dim, int tsrc, void* src, const int* ext, const int* sstr,
                      int tdst, void* dst, const int* dstr, double sigma, int border)
{
    return dispatch_dim(dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        return dispatch_type(tsrc, [&](auto s) {
            using S = decltype(s);
            return dispatch_type(tdst, [&](auto d) {
                using Dt = decltype(d);
                auto sv = make_view<S, DIM>(src, ext, sstr);
                auto dv = make_view<Dt, DIM>(dst, ext, dstr);
                ndl::gaussian_blur(sv, dv, sigma, to_border(border));
                return 0;
            });
        });
    });
}

// Per-axis composition of reference convolve() calls.
//   mode 0 ("round once"): the structure of gaussian_blur
//     (processing/convolution.h:148-185) with caller-given 1-D kernels:
//     first pass src -> double buffer, further passes double -> double, final
//     std::round for integral DstT (plain cast otherwise).  A single pass
//     calls convolve() straight into dst, as gaussian_blur's DIM==1 branch
//     does (:141-146).
//   mode 1 ("cast each pass"): every pass is a complete convolve() into a
//     DstT buffer (truncating for integral DstT), the chain a caller gets by
//     calling convolve() once per axis.
// taps holds the npass kernels back to back; centres are K/2.
int ref_compose(int dim, int tsrc, void* src, const int* ext, const int* sstr,
                int tdst, void* dst, const int* dstr,
                int npass, const int* axes, const int* ntaps, const double* taps,
                int mode, int border)
{
    if (npass < 1) return -4;
    return dispatch_dim(dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        return dispatch_type(tsrc, [&](auto s) {
            using S = decltype(s);
            return dispatch_type(tdst, [&](auto d) {
                using Dt = decltype(d);
                auto sv = make_view<S, DIM>(src, ext, sstr);
                auto dv = make_view<Dt, DIM>(dst, ext, dstr);
                const ndl::BorderMode bm = to_border(border);
                std::array<int, DIM> e;
                for (int i = 0; i < DIM; i++) e[i] = ext[i];
                std::vector<const double*> w((size_t)npass);
                {
                    size_t off = 0;
                    for (int p = 0; p < npass; p++) { w[p] = taps + off; off += (size_t)ntaps[p]; }
                }
                std::vector<double> kstore;
                if (npass == 1) {
                    ndl::convolve(sv, dv, axis_kernel<DIM>(axes[0], ntaps[0], w[0], kstore), bm);
                    return 0;
                }
                if (mode == 1) {
                    std::vector<Dt> a(ndl::Image<Dt, DIM>::size(e)), b(a.size());
                    ndl::Image<Dt, DIM> ia(a.data(), e), ib(b.data(), e);
                    ndl::convolve(sv, ia, axis_kernel<DIM>(axes[0], ntaps[0], w[0], kstore), bm);
                    ndl::Image<Dt, DIM>* cur = &ia;
                    ndl::Image<Dt, DIM>* oth = &ib;
                    for (int p = 1; p < npass - 1; p++) {
                        ndl::convolve(*cur, *oth, axis_kernel<DIM>(axes[p], ntaps[p], w[p], kstore), bm);
                        std::swap(cur, oth);
                    }
                    ndl::convolve(*cur, dv, axis_kernel<DIM>(axes[npass - 1], ntaps[npass - 1], w[npass - 1], kstore), bm);
                    return 0;
                }
                std::vector<double> a(ndl::Image<double, DIM>::size(e)), b(a.size());
                ndl::Image<double, DIM> ia(a.data(), e), ib(b.data(), e);
                ndl::convolve(sv, ia, axis_kernel<DIM>(axes[0], ntaps[0], w[0], kstore), bm);
                ndl::Image<double, DIM>* cur = &ia;
                ndl::Image<double, DIM>* oth = &ib;
                for (int p = 1; p < npass; p++) {
                    ndl::convolve(*cur, *oth, axis_kernel<DIM>(axes[p], ntaps[p], w[p], kstore), bm);
                    std::swap(cur, oth);
                }
                for (const auto& c : cur->coordinates()) {
                    double v = cur->at(c);
                    dv.at(c) = static_cast<Dt>(std::is_integral<Dt>::value ? std::round(v) : v);
                }
                return 0;
            });
        });
    });
}

// Applies a chain of reference view builders to a contiguous Image of
// base_ext and reports the resulting view: element offset of &at({0,..})
// from the buffer start, extent and stride.  ops: triples {code, a, b}
// with code 1 = swap_axes(a,b), 2 = mirror(a), 3 = view with
// start[a] / end / step given in the following op triples {4, start, end},
// {5, step, 0} for axis a (other axes full range, step 1).
int ref_view_probe(int dim, const int* base_ext, const int* ops, int nops,
                   long long* offset_out, int* ext_out, int* str_out)
{
    return dispatch_dim(dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        std::array<int, DIM> e;
        for (int i = 0; i < DIM; i++) e[i] = base_ext[i];
        std::vector<char> buf(ndl::Image<char, DIM>::size(e));
        // Image's operator= copies element values (image/core.h:253), so
        // each builder's result is kept by copy construction instead.
        std::vector<ndl::Image<char, DIM>> chain;
        chain.emplace_back(buf.data(), e);
        for (int o = 0; o < nops; o++) {
            const ndl::Image<char, DIM>& img = chain.back();
            int code = ops[3 * o], a = ops[3 * o + 1], b = ops[3 * o + 2];
            if (code == 1) chain.push_back(img.swap_axes(a, b));
            else if (code == 2) chain.push_back(img.mirror(a));
            else if (code == 3) {
                if (o + 2 >= nops || ops[3 * (o + 1)] != 4 || ops[3 * (o + 2)] != 5) return -5;
                std::vector<int> st(DIM, 0), en(DIM, -1), sp(DIM, 1);
                st[a] = ops[3 * (o + 1) + 1];
                en[a] = ops[3 * (o + 1) + 2];
                sp[a] = ops[3 * (o + 2) + 1];
                // view() takes initializer lists; expanded per DIM.
                if constexpr (DIM == 1) chain.push_back(img.view({st[0]}, {en[0]}, {sp[0]}));
                if constexpr (DIM == 2) chain.push_back(img.view({st[0], st[1]}, {en[0], en[1]}, {sp[0], sp[1]}));
                if constexpr (DIM == 3) chain.push_back(img.view({st[0], st[1], st[2]}, {en[0], en[1], en[2]}, {sp[0], sp[1], sp[2]}));
                if constexpr (DIM == 4) chain.push_back(img.view({st[0], st[1], st[2], st[3]}, {en[0], en[1], en[2], en[3]}, {sp[0], sp[1], sp[2], sp[3]}));
                o += 2;
            } else return -6;
        }
        const ndl::Image<char, DIM>& img = chain.back();
        std::array<int, DIM> z{};
        *offset_out = (long long)(&img.at(z) - buf.data());
        for (int i = 0; i < DIM; i++) { ext_out[i] = img.extent()[i]; str_out[i] = img.stride()[i]; }
        return 0;
    });
}

}  // extern "C"
