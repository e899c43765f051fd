// dropin_check.cpp -- the C++ drop-in overloads (include/ndlgpu_dropin.h)
// against the reference's own ndl::gaussian_blur / ndl::convolve, on the same
// inputs and the same ndl::Image views.  Built by oracle/build_oracle.py into
// oracle/_ref/dropin_check (it includes the reference headers, so it is test
// infrastructure); run by tests/test_gpu_dropin.py.  Prints one line per check
// and exits non-zero on any failure.
#include <ndl/image.h>
#include <ndl/processing/convolution.h>
#include <ndl/processing/summed_area_table.h>

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "ndlgpu_dropin.h"

static int failures = 0;
static void report(const char* what, bool ok, double metric)
{
    std::printf("%-60s %s (%.3g)\n", what, ok ? "Pass" : "Fail", metric);
    if (!ok) failures++;
}

template <class T>
static T* upload(const std::vector<T>& h)
{
    T* d = nullptr;
    cudaMalloc(&d, h.size() * sizeof(T));
    cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
    return d;
}

int main()
{
    std::mt19937_64 rng(20261203);
    // 1. gaussian_blur, float 512x512, sigma 2, Clamp (the CPU-runnable configuration)
    {
        const int W = 512, H = 512;
        std::vector<float> in((size_t)W * H), ref((size_t)W * H), got((size_t)W * H);
        std::uniform_real_distribution<float> u(0.f, 1.f);
        for (auto& v : in) v = u(rng);
        ndl::Image<float, 2> hin(in.data(), {W, H}), href(ref.data(), {W, H});
        ndl::gaussian_blur(hin, href, 2.0, ndl::BorderMode::Clamp);
        float* din = upload(in);
        float* dout = upload(got);
        ndl::Image<float, 2> gin(din, {W, H}), gout(dout, {W, H});
        ndlgpu::gaussian_blur(gin, gout, 2.0, ndl::BorderMode::Clamp);
        cudaMemcpy(got.data(), dout, got.size() * sizeof(float), cudaMemcpyDeviceToHost);
        double worst = 0;
        for (size_t i = 0; i < got.size(); i++) worst = std::max(worst, std::fabs((double)got[i] - ref[i]) / std::fabs((double)ref[i]));
        report("gaussian_blur f32 512^2 sigma 2 Clamp, max rel err <= 1e-6", worst <= 1e-6, worst);
        cudaFree(din);
        cudaFree(dout);
    }
    // 2. uint8 64^3 seen through swap_axes(0,2).mirror(1): gaussian_blur (Wrap)
    //    and a per-axis convolve() with an integer kernel, bit-exact
    {
        const int N = 64;
        std::vector<uint8_t> base((size_t)N * N * N);
        for (auto& v : base) v = (uint8_t)(rng() & 255);
        ndl::Image<uint8_t, 3> hb(base.data(), {N, N, N});
        auto hview = hb.swap_axes(0, 2).mirror(1);
        uint8_t* db = upload(base);
        ndl::Image<uint8_t, 3> gb(db, {N, N, N});
        auto gview = gb.swap_axes(0, 2).mirror(1);
        for (auto border : {ndl::BorderMode::Clamp, ndl::BorderMode::Wrap, ndl::BorderMode::Reflect}) {
            ndl::OwnedImage<uint8_t, 3> ref(hview.extent());
            ndl::gaussian_blur(hview, ref, 1.3, border);
            std::vector<uint8_t> got((size_t)N * N * N, 0);
            uint8_t* dout = upload(got);
            ndl::Image<uint8_t, 3> gout(dout, hview.extent());
            ndlgpu::gaussian_blur(gview, gout, 1.3, border);
            cudaMemcpy(got.data(), dout, got.size(), cudaMemcpyDeviceToHost);
            size_t bad = 0;
            size_t i = 0;
            for (const auto& c : ref.coordinates()) bad += (got[i++] != ref.at(c));
            report("gaussian_blur u8 view swap_axes(0,2).mirror(1), bit-exact", bad == 0, (double)bad);
            // one convolve() pass along axis 1 with an int kernel {1,2,1}: truncation
            ndl::OwnedImage<int, 3> k({1, 3, 1});
            k.at({0, 0, 0}) = 1;
            k.at({0, 1, 0}) = 2;
            k.at({0, 2, 0}) = 1;
            ndl::OwnedImage<uint8_t, 3> ref2(hview.extent());
            ndl::convolve(hview, ref2, k, border);
            ndlgpu::convolve(gview, gout, k, border);
            cudaMemcpy(got.data(), dout, got.size(), cudaMemcpyDeviceToHost);
            bad = 0;
            i = 0;
            for (const auto& c : ref2.coordinates()) bad += (got[i++] != ref2.at(c));
            report("convolve u8 view, int {1,2,1} kernel on axis 1, bit-exact", bad == 0, (double)bad);
            cudaFree(dout);
        }
        cudaFree(db);
    }
    // 3. gradient (default border Reflect) of a float view and of uint8 into
    //    int16, against ndl::gradient itself, bit-exact
    {
        const int NX = 40, NY = 33, NZ = 27;
        std::vector<float> fb((size_t)NX * NY * NZ);
        std::normal_distribution<float> nd(0.f, 1.f);
        for (auto& v : fb) v = nd(rng);
        ndl::Image<float, 3> hf(fb.data(), {NX, NY, NZ});
        auto hv = hf.swap_axes(0, 2).mirror(1);
        float* df = upload(fb);
        ndl::Image<float, 3> gf(df, {NX, NY, NZ});
        auto gv = gf.swap_axes(0, 2).mirror(1);
        const auto e3 = hv.extent();
        ndl::OwnedImage<float, 4> ref({3, e3[0], e3[1], e3[2]});
        ndl::gradient(hv, ref);
        std::vector<float> got((size_t)3 * NX * NY * NZ, 0.f);
        float* dg = upload(got);
        ndl::Image<float, 4> gg(dg, {3, e3[0], e3[1], e3[2]});
        ndlgpu::gradient(gv, gg);
        cudaMemcpy(got.data(), dg, got.size() * sizeof(float), cudaMemcpyDeviceToHost);
        size_t bad = 0, i = 0;
        for (const auto& c : ref.coordinates()) bad += (got[i++] != ref.at(c));
        report("gradient f32 view swap_axes(0,2).mirror(1), bit-exact", bad == 0, (double)bad);
        std::vector<uint8_t> ub((size_t)NX * NY * NZ);
        for (auto& v : ub) v = (uint8_t)(rng() & 255);
        ndl::Image<uint8_t, 3> hu(ub.data(), {NX, NY, NZ});
        uint8_t* du = upload(ub);
        ndl::Image<uint8_t, 3> gu(du, {NX, NY, NZ});
        ndl::OwnedImage<int16_t, 4> ref16({3, NX, NY, NZ});
        ndl::gradient(hu, ref16, ndl::BorderMode::Clamp);
        std::vector<int16_t> got16((size_t)3 * NX * NY * NZ, 0);
        int16_t* d16 = upload(got16);
        ndl::Image<int16_t, 4> g16(d16, {3, NX, NY, NZ});
        ndlgpu::gradient(gu, g16, ndl::BorderMode::Clamp);
        cudaMemcpy(got16.data(), d16, got16.size() * sizeof(int16_t), cudaMemcpyDeviceToHost);
        bad = 0;
        i = 0;
        for (const auto& c : ref16.coordinates()) bad += (got16[i++] != ref16.at(c));
        report("gradient u8 -> int16 Clamp (truncation), bit-exact", bad == 0, (double)bad);
        cudaFree(df);
        cudaFree(dg);
        cudaFree(du);
        cudaFree(d16);
    }
    // 4. box_blur (float view, Reflect) and downsample (uint8 colour image),
    //    against ndl::box_blur and ndl::downsample themselves, bit-exact
    {
        const int NX = 70, NY = 45;
        std::vector<float> fb((size_t)NX * NY);
        std::uniform_real_distribution<float> u(0.f, 1.f);
        for (auto& v : fb) v = u(rng);
        ndl::Image<float, 2> hf(fb.data(), {NX, NY});
        auto hv = hf.swap_axes(0, 1).mirror(0);
        ndl::OwnedImage<float, 2> ref(hv.extent());
        ndl::box_blur(hv, ref, 3, ndl::BorderMode::Reflect);
        float* df = upload(fb);
        ndl::Image<float, 2> gf(df, {NX, NY});
        auto gv = gf.swap_axes(0, 1).mirror(0);
        std::vector<float> got((size_t)NX * NY, 0.f);
        float* dg = upload(got);
        ndl::Image<float, 2> gg(dg, hv.extent());
        ndlgpu::box_blur(gv, gg, 3, ndl::BorderMode::Reflect);
        cudaMemcpy(got.data(), dg, got.size() * sizeof(float), cudaMemcpyDeviceToHost);
        size_t bad = 0, i = 0;
        for (const auto& c : ref.coordinates()) bad += (got[i++] != ref.at(c));
        report("box_blur f32 view swap_axes(0,1).mirror(0) Reflect r=3, bit-exact", bad == 0, (double)bad);

        const int W = 37, H = 23;
        std::vector<uint8_t> rgb((size_t)3 * W * H);
        for (auto& v : rgb) v = (uint8_t)(rng() & 255);
        ndl::Image<uint8_t, 3> hc(rgb.data(), {3, W, H});
        auto small = ndl::downsample(hc, 3);
        uint8_t* dc = upload(rgb);
        ndl::Image<uint8_t, 3> gc(dc, {3, W, H});
        const auto es = small.extent();
        std::vector<uint8_t> got8((size_t)es[0] * es[1] * es[2], 0);
        uint8_t* ds = upload(got8);
        ndl::Image<uint8_t, 3> gs(ds, es);
        ndlgpu::downsample(gc, gs, 3);
        cudaMemcpy(got8.data(), ds, got8.size(), cudaMemcpyDeviceToHost);
        bad = 0;
        i = 0;
        for (const auto& c : small.coordinates()) bad += (got8[i++] != small.at(c));
        report("downsample u8 {3, 37, 23} by 3, bit-exact", bad == 0, (double)bad);
        cudaFree(df);
        cudaFree(dg);
        cudaFree(dc);
        cudaFree(ds);
    }
    // 5. the reference asserts on mismatched extents; the drop-in throws
    {
        float* d = nullptr;
        cudaMalloc(&d, 64 * sizeof(float));
        ndl::Image<float, 2> a(d, {4, 4}), b(d + 32, {4, 5});
        bool threw = false;
        try {
            ndlgpu::gaussian_blur(a, b, 1.0, ndl::BorderMode::Clamp);
        } catch (const ndlgpu::error& e) {
            threw = e.status() == NDLGPU_ERR_EXTENT_MISMATCH;
        }
        report("mismatched extents throw ndlgpu::error(EXTENT_MISMATCH)", threw, 0);
        cudaFree(d);
    }
    cudaError_t e = cudaDeviceSynchronize();
    report("no CUDA error", e == cudaSuccess, (double)e);
    std::printf(failures ? "DROPIN FAIL\n" : "DROPIN OK\n");
    return failures ? 1 : 0;
}
