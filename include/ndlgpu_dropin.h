/*
 * ndlgpu_dropin.h -- C++17 drop-in overloads of ndl's convolution calls,
 * forwarding to the C ABI of libndlgpu.so (ndlgpu.h).
 *
 * The reference's interface is a pair of function templates over any type
 * with the minimal image interface (image/detail.h:48-57):
 *
 *   template<class SrcImageT, class DstImageT, class KernelT>
 *   void ndl::convolve(const SrcImageT&, DstImageT&, const KernelT&, BorderMode = Clamp);
 *                                                   -- processing/convolution.h:52-53
 *   template<class SrcImageT, class DstImageT>
 *   void ndl::gaussian_blur(const SrcImageT&, DstImageT&, double sigma, BorderMode = Clamp);
 *                                                   -- processing/convolution.h:107-108
 *   template<class SrcImageT, class DstImageT>
 *   void ndl::gradient(const SrcImageT&, DstImageT&, BorderMode = Reflect);
 *                                                   -- processing/convolution.h:359-360
 *
 * ndlgpu::convolve / ndlgpu::gaussian_blur / ndlgpu::gradient take the same arguments (plus an
 * optional CUDA stream) where src and dst are views of DEVICE memory: any type
 * with extent(), stride() and at() returning a reference -- an ndl::Image<T,DIM>
 * constructed over a device pointer, or any view derived from it by
 * view()/slice()/swap_axes()/mirror() (image/core.h:647-757).  The view's
 * address arithmetic is done on the host (&at({0,..})); no element is read or
 * written by the host.  The kernel is a HOST image of any arithmetic type
 * (converted to double as convolution.h:68 does).
 *
 * Where the reference asserts (dst.extent() == src.extent(), sigma > 0), these
 * overloads throw ndlgpu::error with the library's status and message, before
 * any GPU work is queued.  Calls are asynchronous on `stream`.
 */
#ifndef NDLGPU_DROPIN_H
#define NDLGPU_DROPIN_H

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>

#include "ndlgpu.h"

namespace ndlgpu {

class error : public std::runtime_error {
public:
    error(ndlgpu_status s, const std::string& msg) : std::runtime_error(msg), status_(s) {}
    ndlgpu_status status() const { return status_; }

private:
    ndlgpu_status status_;
};

template <class T> struct dtype_of;
template <> struct dtype_of<uint8_t> { static constexpr int value = NDLGPU_U8; };
template <> struct dtype_of<int8_t> { static constexpr int value = NDLGPU_I8; };
template <> struct dtype_of<uint16_t> { static constexpr int value = NDLGPU_U16; };
template <> struct dtype_of<int16_t> { static constexpr int value = NDLGPU_I16; };
template <> struct dtype_of<int32_t> { static constexpr int value = NDLGPU_I32; };
template <> struct dtype_of<uint32_t> { static constexpr int value = NDLGPU_U32; };
template <> struct dtype_of<int64_t> { static constexpr int value = NDLGPU_I64; };
template <> struct dtype_of<uint64_t> { static constexpr int value = NDLGPU_U64; };
template <> struct dtype_of<float> { static constexpr int value = NDLGPU_F32; };
template <> struct dtype_of<double> { static constexpr int value = NDLGPU_F64; };

namespace detail {

inline void check(ndlgpu_status s)
{
    if (s != NDLGPU_OK) throw error(s, std::string("ndlgpu: ") + ndlgpu_status_string(s) + ": " + ndlgpu_last_error());
}

template <class ImageT>
constexpr int rank_of()
{
    return (int)std::tuple_size<std::decay_t<decltype(std::declval<const ImageT&>().extent())>>::value;
}

// {pointer, extent, stride} of an Image-like view: data = &at({0,..,0}).
template <class ImageT>
ndlgpu_view view_of(const ImageT& img)
{
    using T = std::remove_cv_t<typename ImageT::value_type>;
    constexpr int DIM = rank_of<ImageT>();
    static_assert(DIM >= 1 && DIM <= NDLGPU_MAX_RANK, "rank must be 1..8");
    ndlgpu_view v{};
    const auto ext = img.extent();
    const auto str = img.stride();
    std::array<int, DIM> zero{};
    bool empty = false;
    for (int i = 0; i < DIM; i++) {
        v.extent[i] = ext[i];
        v.stride[i] = str[i];
        if (ext[i] == 0) empty = true;
    }
    v.data = empty ? nullptr : const_cast<void*>(static_cast<const void*>(&img.at(zero)));
    v.dtype = dtype_of<T>::value;
    v.rank = DIM;
    return v;
}

}  // namespace detail

/// ndl::convolve on device memory (processing/convolution.h:52-71).
template <class SrcImageT, class DstImageT, class KernelT, class BorderT = int>
void convolve(const SrcImageT& src, DstImageT& dst, const KernelT& kernel, BorderT border = BorderT(0),
              void* stream = nullptr)
{
    const ndlgpu_view s = detail::view_of(src);
    const ndlgpu_view d = detail::view_of(dst);
    const ndlgpu_view k = detail::view_of(kernel);   // host memory
    detail::check(ndlgpu_convolve(&s, &d, &k, static_cast<int>(border), stream));
}

/// ndl::gradient on device memory (processing/convolution.h:359-388): dst has
/// a leading component axis of extent DIM; dst.slice(0, a) gets the central
/// difference along axis a.  The reference's default border is Reflect (2).
template <class SrcImageT, class DstImageT, class BorderT = int>
void gradient(const SrcImageT& src, DstImageT& dst, BorderT border = BorderT(NDLGPU_REFLECT), void* stream = nullptr)
{
    const ndlgpu_view s = detail::view_of(src);
    const ndlgpu_view d = detail::view_of(dst);
    detail::check(ndlgpu_gradient(&s, &d, static_cast<int>(border), stream));
}

/// ndl::gaussian_blur on device memory (processing/convolution.h:107-186).
/// The library allocates its scratch stream-ordered unless a workspace is
/// given (see ndlgpu_gaussian_blur_workspace_size).
template <class SrcImageT, class DstImageT, class BorderT = int>
void gaussian_blur(const SrcImageT& src, DstImageT& dst, double sigma, BorderT border = BorderT(0),
                   void* stream = nullptr, void* workspace = nullptr, size_t workspace_bytes = 0)
{
    const ndlgpu_view s = detail::view_of(src);
    const ndlgpu_view d = detail::view_of(dst);
    detail::check(ndlgpu_gaussian_blur(&s, &d, sigma, static_cast<int>(border), workspace, workspace_bytes, stream));
}

/// ndl::box_blur on device memory (processing/summed_area_table.h:300-339):
/// the (2 radius + 1)^DIM box average through the reference's own
/// summed-area-table arithmetic (bit-exact).  Scratch as for gaussian_blur
/// (see ndlgpu_box_blur_workspace_size).
template <class SrcImageT, class DstImageT, class BorderT = int>
void box_blur(const SrcImageT& src, DstImageT& dst, int radius, BorderT border = BorderT(0), void* stream = nullptr,
              void* workspace = nullptr, size_t workspace_bytes = 0)
{
    const ndlgpu_view s = detail::view_of(src);
    const ndlgpu_view d = detail::view_of(dst);
    detail::check(ndlgpu_box_blur(&s, &d, radius, static_cast<int>(border), workspace, workspace_bytes, stream));
}

/// ndl::downsample on device memory (processing/convolution.h:241-305).  The
/// reference returns a new image; here the caller passes dst with the
/// decimated extents ((extent - 1) / factor + 1 on every axis but
/// channelAxis).  Bit-exact block averages.
template <class SrcImageT, class DstImageT, class BorderT = int>
void downsample(const SrcImageT& src, DstImageT& dst, int factor, int channelAxis = 0, BorderT border = BorderT(0),
                void* stream = nullptr)
{
    const ndlgpu_view s = detail::view_of(src);
    const ndlgpu_view d = detail::view_of(dst);
    detail::check(ndlgpu_downsample(&s, &d, factor, channelAxis, static_cast<int>(border), stream));
}

}  // namespace ndlgpu

#endif /* NDLGPU_DROPIN_H */
