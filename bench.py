"""Benchmark: 3-D separable convolution forward + adjoint on B200.

One step = the forward chain Y = Cz(Cy(Cx X)) and its adjoint (dL/dX and all
27 tap gradients of L = sum(W * Y)) over a batch of 192^3 float32 volumes:
per-axis 9-tap kernels (N(0,1) taps, each normalised to unit L1 norm),
border Reflect, X and W ~ N(0,1) from a seed.  The batch (8 volumes, an
untouched fourth axis) makes the inputs 226 MB each -- larger than the 126 MB
L2 -- so every step streams from HBM.

Printed on rank 0: one JSON line with the headline throughput (Gvoxel/s of
fwd+adjoint), the roofline of the dominant kernel, the end-to-end number
through the C ABI with host buffers, the CPU baseline (the compiled ndl
reference, single-threaded) and the other forms (uint8 bit-exact volume,
bf16/f16/f32 video, 2-D gaussian, the batched uneven launch).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gvoxel/s & % HBM peak, 3-D separable conv fwd+adjoint, FP32 plain vs batched BF16"
EDGE, NTAP, BATCH = 192, 9, 8
SEED = 20261203


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def make_taps(seed=SEED):
    rng = np.random.default_rng(seed)
    out = []
    for ax in range(3):
        w = rng.standard_normal(NTAP)
        out.append((ax, w / np.abs(w).sum()))
    return out


# ---------------------------------------------------------------------------
# clocks during the timed region (NVML sampler thread)
# ---------------------------------------------------------------------------

class ClockSampler:
    REASONS = {
        0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
        0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
    }

    def __init__(self, index):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        while not self._stop.is_set():
            self.sample()
            time.sleep(0.02)

    def sample(self):
        if self.nv is None:
            return
        try:
            self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
            mask = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            for bit, name in self.REASONS.items():
                if mask & bit and name != "gpu_idle":
                    self.reasons.add(name)
        except Exception:
            pass

    def __enter__(self):
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self.t.join()
        if not self.samples:
            self.sample()

    def result(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def run_gpu(args):
    import torch
    import torch.distributed as dist

    import ndl_b200 as n
    from ndl_b200 import BorderMode, Image, abi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)
    lib = abi.load()
    hbm, peak_src = peaks()
    passes = make_taps()
    stream = torch.cuda.current_stream()

    # workload: BATCH volumes of EDGE^3 (numpy shape (B, z, y, x))
    g = torch.Generator(device=dev)
    g.manual_seed(SEED + rank)
    shape = (BATCH, EDGE, EDGE, EDGE)
    X = torch.randn(shape, generator=g, device=dev, dtype=torch.float32)
    W = torch.randn(shape, generator=g, device=dev, dtype=torch.float32)
    Y = torch.empty_like(X)
    GX = torch.empty_like(X)
    taps = torch.zeros(3 * NTAP, dtype=torch.float32, device=dev)
    xi, wi, yi, gi = (Image.from_tensor(t) for t in (X, W, Y, GX))
    ws_f = n.convolve_axes_workspace_size(xi, yi, passes, BorderMode.Reflect)
    ws = torch.empty(max(1, ws_f), dtype=torch.uint8, device=dev)
    import ctypes
    arr, keep = abi.make_passes(passes)
    gv, xv, gxv = wi.abi_view(), xi.abi_view(), gi.abi_view()
    nb = ctypes.c_size_t(0)
    abi.check(lib.ndlgpu_convolve_axes_adjoint_workspace_size(ctypes.byref(gv), ctypes.byref(xv), ctypes.byref(gxv),
                                                              3, arr, BorderMode.Reflect, abi.F32, ctypes.byref(nb)))
    wsa = torch.empty(max(1, nb.value), dtype=torch.uint8, device=dev)

    def fwd():
        n.convolve_axes(xi, yi, passes, BorderMode.Reflect, workspace=ws, stream=stream)

    def adj():
        n.convolve_axes_adjoint(wi, xi, gi, passes, BorderMode.Reflect, taps, workspace=wsa, stream=stream)

    voxels = BATCH * EDGE ** 3
    K, Wm = args.steps, max(3, args.warmup)
    for _ in range(Wm):
        if args.only != "adj":
            fwd()
        if args.only != "fwd":
            adj()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    l0 = lib.ndlgpu_kernel_launches()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(dev.index)
    with sampler:
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        for k in range(K):
            ev[k][0].record(stream)
            if args.only != "adj":
                fwd()
            ev[k][1].record(stream)
            if args.only != "fwd":
                adj()
            ev[k][2].record(stream)
        t_end.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches = lib.ndlgpu_kernel_launches() - l0
    total_ms = t_start.elapsed_time(t_end)
    fwd_ms = sum(e[0].elapsed_time(e[1]) for e in ev) / K
    adj_ms = sum(e[1].elapsed_time(e[2]) for e in ev) / K
    fwd_ms, adj_ms = max(fwd_ms, 1e-9), max(adj_ms, 1e-9)
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_step = total_ms / K
    value = world * voxels / (ms_step * 1e-3) / 1e9

    fwd_gbs = 8.0 * voxels / (fwd_ms * 1e-3) / 1e9
    adj_gbs = 12.0 * voxels / (adj_ms * 1e-3) / 1e9

    # The three kernels of a step, each timed alone (CUDA events on the
    # launching stream): the forward, dL/dX alone (grad_taps NULL) and the
    # tap gradients alone (grad_src NULL).  Each moves 8 algorithmic bytes
    # per voxel: one f32 volume read and one written (forward, dL/dX), or two
    # f32 volumes read (tap gradients; the per-CTA partial sums are < 1 MB).
    kern = {}
    if not args.only:
        calls = {
            "k_fwd3 forward": fwd,
            "k_fused2 adjoint dL/dX": lambda: n.convolve_axes_adjoint(wi, xi, gi, passes, BorderMode.Reflect, None,
                                                                   workspace=wsa, stream=stream),
            "k_tapgrad tap gradients": lambda: n.convolve_axes_adjoint(wi, xi, None, passes, BorderMode.Reflect,
                                                                    taps, workspace=wsa, stream=stream),
        }
        for name, fn in calls.items():
            ms = time_call(fn, max(3, min(K, 20)), stream=stream)
            gbs = 8.0 * voxels / (ms * 1e-3) / 1e9
            kern[name] = {"ms": round(ms, 4), "gbs": round(gbs, 1), "frac_of_measured_hbm": round(gbs / hbm, 4)}
    if kern:
        name = max(kern, key=lambda k: kern[k]["ms"])
        traffic, tsrc = profiled_traffic(name)
        roofline = {"bound": "hbm", "achieved": kern[name]["gbs"], "peak": hbm, "unit": "GB/s",
                    "frac": round(kern[name]["gbs"] / hbm, 4), "traffic": traffic, "kernel": name,
                    "algorithmic_bytes_per_launch": 8 * voxels, "peak_source": peak_src, "traffic_source": tsrc}
    else:
        dom_ms, dom_gbs = (adj_ms, adj_gbs) if adj_ms >= fwd_ms else (fwd_ms, fwd_gbs)
        roofline = {"bound": "hbm", "achieved": round(dom_gbs, 1), "peak": hbm, "unit": "GB/s",
                    "frac": round(dom_gbs / hbm, 4), "traffic": None,
                    "kernel": "adjoint call" if adj_ms >= fwd_ms else "forward call", "peak_source": peak_src}

    # End to end through the C ABI with host (pinned) buffers.  Every step
    # copies its inputs X, W host->device and its results Y, dL/dX and the
    # taps device->host.  Steps are pipelined the way a serving loop runs
    # them: the upload of step k+1, the kernels of step k and the read-back
    # of step k-1 overlap on three streams (two device buffer sets), so the
    # sustained rate is set by the slower PCIe direction, not by their sum.
    e2e = None
    if not args.skip_e2e:
        hX = torch.empty(shape, dtype=torch.float32, pin_memory=True)
        hW = torch.empty(shape, dtype=torch.float32, pin_memory=True)
        hX.copy_(X)
        hW.copy_(W)
        hY = torch.empty_like(hX, pin_memory=True)
        hG = torch.empty_like(hX, pin_memory=True)
        htaps = torch.empty(3 * NTAP, dtype=torch.float32, pin_memory=True)
        ke = max(3, min(K, 24))   # steps timed: pipeline fill and drain amortised over them
        sets = [(X, W, Y, GX, taps, xi, wi, yi, gi)]
        X2, W2, Y2, G2 = (torch.empty_like(X) for _ in range(4))
        t2 = torch.zeros_like(taps)
        sets.append((X2, W2, Y2, G2, t2) + tuple(Image.from_tensor(t) for t in (X2, W2, Y2, G2)))
        s_up, s_cmp, s_dn = torch.cuda.Stream(dev), torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        ev_up = [torch.cuda.Event() for _ in range(2)]
        ev_cmp = [torch.cuda.Event() for _ in range(2)]
        ev_dn = [torch.cuda.Event() for _ in range(2)]
        for e in ev_cmp + ev_dn:
            e.record(stream)

        def e2e_step(k):
            b = k & 1
            dX, dW, dY, dG, dT, ix, iw, iy, ig = sets[b]
            with torch.cuda.stream(s_up):
                s_up.wait_event(ev_cmp[b])          # inputs of step k-2 consumed
                dX.copy_(hX, non_blocking=True)
                dW.copy_(hW, non_blocking=True)
                ev_up[b].record(s_up)
            s_cmp.wait_event(ev_up[b])
            s_cmp.wait_event(ev_dn[b])              # results of step k-2 read back
            n.convolve_axes(ix, iy, passes, BorderMode.Reflect, workspace=ws, stream=s_cmp)
            n.convolve_axes_adjoint(iw, ix, ig, passes, BorderMode.Reflect, dT, workspace=wsa, stream=s_cmp)
            ev_cmp[b].record(s_cmp)
            with torch.cuda.stream(s_dn):
                s_dn.wait_event(ev_cmp[b])
                hY.copy_(dY, non_blocking=True)
                hG.copy_(dG, non_blocking=True)
                htaps.copy_(dT, non_blocking=True)
                ev_dn[b].record(s_dn)

        for k in range(2):
            e2e_step(k)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s_up)
        for k in range(ke):
            e2e_step(k)
        s_up.wait_stream(s_dn)
        b.record(s_up)
        torch.cuda.synchronize()
        ems = a.elapsed_time(b) / ke
        if world > 1:
            t = torch.tensor([ems], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        e2e = {"value": round(world * voxels / (ems * 1e-3) / 1e9, 3), "unit": "Gvoxel/s",
               "h2d_bytes_per_step": 2 * X.numel() * 4, "d2h_bytes_per_step": 2 * X.numel() * 4 + 3 * NTAP * 4,
               "ms_per_step": round(ems, 3), "steps": ke,
               "pipeline": "upload k+1 / kernels k / read-back k-1 on three streams, two device buffer sets"}
        del sets, X2, W2, Y2, G2, t2

    # the batched form sharded: config 4's 512 uneven instances partitioned
    # across the ranks by cost (ndl_b200/shard.py), each rank one persistent
    # launch of its share; the job's time is the max over ranks (no
    # data-path collective)
    sharded = None
    if not args.skip_forms:
        sharded = sharded_config4(world, rank, dev, hbm)

    forms = {}
    if rank == 0 and not args.skip_forms:
        forms = other_forms(args, hbm)

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        cpu = cpu_baseline_sample()

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Gvoxel/s", "n_gpus": world, "steps": K, "warmup": Wm,
        "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded N(0,1) volumes and taps)",
        "config": step_config(world),
        "forward": {"ms": round(fwd_ms, 4), "gvoxel_s": round(voxels / fwd_ms / 1e6, 2),
                    "gbs": round(fwd_gbs, 1), "frac_of_measured_hbm": round(fwd_gbs / hbm, 4)},
        "adjoint": {"ms": round(adj_ms, 4), "gvoxel_s": round(voxels / adj_ms / 1e6, 2),
                    "gbs": round(adj_gbs, 1), "frac_of_measured_hbm": round(adj_gbs / hbm, 4)},
        "kernels": kern, "roofline": roofline, "e2e": e2e, "gpu_launches": int(launches), "clocks": sampler.result(),
        "cpu_baseline": cpu, "forms": forms, "sharded_config4": sharded,
    }
    print(json.dumps(line))


PROFILE_OF = {
    "k_fwd3 forward": "k_fwd3_fwd_f32_9x9x9_8x192cube.md",
    "k_fused2 adjoint dL/dX": "k_fused2_adj_f32_9x9x9_8x192cube.md",
    "k_tapgrad tap gradients": "k_tapgrad_f32_9x9x9_8x192cube.md",
}


def profiled_traffic(kernel):
    """DRAM bytes (read + write) of one launch of `kernel`, from the
    committed ncu summary of the same workload (the line
    'traffic_bytes_per_launch: N'), or (None, why)."""
    name = PROFILE_OF.get(kernel)
    if name is None:
        return None, "no ncu summary for this kernel"
    path = os.path.join(ROOT, "profiles", name)
    try:
        with open(path) as f:
            for line in f:
                if line.strip().startswith("traffic_bytes_per_launch:"):
                    return int(line.split(":", 1)[1].strip()), "profiles/" + name + " (ncu dram__bytes_read+write)"
    except OSError:
        pass
    return None, "profiles/" + name + " missing"


def time_call(fn, iters, warm=3, stream=None):
    """Average device time of fn() over iters calls (CUDA events on the
    launching stream, after warm untimed calls, synchronised on both sides)."""
    import torch
    st = stream if stream is not None else torch.cuda.current_stream()
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(iters):
        fn()
    b.record(st)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / iters


def fp64_blur_reference(v, sigmas):
    """FP64 reference of gaussian_blur_axes with Reflect borders, in plain
    PyTorch on the GPU: for each ndl axis with a sigma, the Gaussian taps of
    ndl's formula (radius ceil(3 sigma), exp(-d^2 / (2 sigma^2)) normalised,
    computed in double) applied as a correlation over the symmetric-reflect
    extended axis (ndl's Reflect duplicates the edge sample)."""
    import math

    import torch

    import ndl_b200 as n
    x = v.double()
    nd = x.dim()
    for ax, sg in enumerate(sigmas):
        if sg <= 0:
            continue
        r = n.gaussian_radius(sg)
        w = [math.exp(-(d * d) / (2.0 * sg * sg)) for d in range(-r, r + 1)]
        tot = sum(w)
        w = [t / tot for t in w]
        dim = nd - 1 - ax                          # ndl axis 0 is the last torch dim
        m = x.shape[dim]
        idx = torch.arange(-r, m + r, device=x.device)
        idx = torch.where(idx < 0, -idx - 1, torch.where(idx >= m, 2 * m - idx - 1, idx))
        ext = x.index_select(dim, idx)
        acc = torch.zeros_like(x)
        for k in range(2 * r + 1):
            acc += w[k] * ext.narrow(dim, k, m)
        x = acc
    return x


def video_error(dt, seed=SEED):
    """Error of the configuration-5 blur in storage type dt against an FP64
    reference (plain PyTorch in double on the same decoded inputs), on a
    96 x 3 x 128 x 128 (t, c, y, x) crop with the same value distribution;
    data and taps are positive, so the stencil magnitude is the exact
    result."""
    import torch

    import ndl_b200 as n
    from ndl_b200 import BorderMode, Image

    g = torch.Generator(device="cuda")
    g.manual_seed(seed + 5)
    v = torch.rand((96, 3, 128, 128), generator=g, device="cuda")
    v[torch.rand(v.shape, generator=g, device="cuda") < 0.01] = 1.0
    v = v.to(dt)
    o = Image.empty(Image.from_tensor(v).extent(), dt)
    sig = (2.5, 2.5, 0.0, 1.5)
    n.gaussian_blur_axes(Image.from_tensor(v), o, list(sig), BorderMode.Reflect)
    ref = fp64_blur_reference(v.float(), sig)
    got = o.tensor().double()
    rel = ((got - ref).abs() / ref.abs().clamp_min(1e-30)).cpu().numpy()
    return {"max_rel": float("%.3g" % rel.max()), "rms_rel": float("%.3g" % np.sqrt((rel ** 2).mean())),
            "sample": "96x3x128x128 crop, same distribution, vs an FP64 PyTorch reference"}


def dog_fma_per_pixel(num_scales, sigma0, tile_rows=32):
    """FMAs per output pixel of the fused scale-space kernel: each level's X
    pass covers the tile rows plus that level's halo, then its Y pass."""
    import ndl_b200 as n
    total = 0.0
    for i in range(num_scales):
        r = n.gaussian_radius(sigma0 * 2.0 ** (i / (num_scales - 3)))
        total += (2 * r + 1) * ((tile_rows + 2 * r) / tile_rows + 1.0)
    return total


def dog_form(g, it, hbm):
    """Difference-of-Gaussians scale space (feature_detection.h:101-122) of a
    4096^2 f32 image, 5 levels from sigma0 = 1.6, Reflect: 20 algorithmic
    bytes per pixel (read 4, write four 4-byte differences), timed beside the
    same five levels as five gaussian_blur calls."""
    import torch

    import ndl_b200 as n
    from ndl_b200 import BorderMode, Image

    x = torch.rand((4096, 4096), generator=g, device="cuda") * 255.0
    s = Image.from_tensor(x)
    dogs = [Image.empty(s.extent(), torch.float32) for _ in range(4)]
    ms = time_call(lambda: n.dog_scale_space(s, 5, 1.6, dogs=dogs), it)
    levels = [Image.empty(s.extent(), torch.float32) for _ in range(5)]
    sig = [1.6 * 2.0 ** (i / 2) for i in range(5)]

    def five_blurs():
        for i in range(5):
            n.gaussian_blur(s, levels[i], sig[i], BorderMode.Reflect)

    ms5 = time_call(five_blurs, max(3, it // 4))
    px = x.numel()
    fma = dog_fma_per_pixel(5, 1.6)
    return {"ms": round(ms, 4), "mpix_s": round(px / ms / 1e3, 1), "gbs": round(20.0 * px / ms / 1e6, 1),
            "frac_of_measured_hbm": round(20.0 * px / ms / 1e6 / hbm, 4),
            "fp32_tflops": round(2.0 * fma * px / ms / 1e9, 2), "fma_per_pixel": round(fma, 1),
            "five_gaussian_blur_calls_ms": round(ms5, 4)}


def other_forms(args, hbm):
    """The other workloads (configurations 1, 2, 4 and 5 and the further forms), timed briefly (each > L2)."""
    import torch

    import ndl_b200 as n
    from ndl_b200 import BorderMode, Image

    out = {}
    it = max(5, min(args.steps, 20))
    sel = getattr(args, "form", "") or ""

    def want(key):
        return not sel or key.startswith(sel) or sel.startswith(key)

    g = torch.Generator(device="cuda")
    g.manual_seed(SEED)
    if want("u8_binomial"):
        u8_form(n, g, it, hbm, out)
    if want("gradient"):
        gradient_form(n, g, it, hbm, out)
    if want("gaussian_blur"):
        gaussian_forms(n, g, it, hbm, out)
    if want("convolve_full5x5"):
        stencil_form(n, g, it, hbm, out)
    if want("learnable_3tap"):
        learnable_form(n, g, it, out)
    if want("dog"):
        out["dog_f32_4096^2_5scales"] = dog_form(g, it, hbm)
    if want("downsample"):
        downsample_form(n, g, it, hbm, out)
    if want("box_blur"):
        box_blur_form(n, g, it, hbm, out)
    if want("video"):
        video_forms(n, g, it, hbm, out, sel)
    if want("batched"):
        # config 4: 512 uneven instances, one persistent launch (graph replay),
        # FP32 and BF16 storage, forward and adjoint; against the plain
        # per-call FP32 path on the same instances
        out.update(batched_forms(hbm))
    if want("gauss2d"):
        gauss2d_form(n, g, out)
    torch.cuda.empty_cache()
    return out


def u8_form(n, g, it, hbm, out):
    import torch
    from ndl_b200 import BorderMode, Image
    # config 2: uint8 256^3 through swap_axes(0,2).mirror(1), binomial, Wrap (x4 volumes > L2)
    base = torch.randint(0, 256, (4, 256, 256, 256), generator=g, device="cuda", dtype=torch.uint8)
    src = Image.from_tensor(base).swap_axes(0, 2).mirror(1)
    dst = Image.empty(src.extent(), torch.uint8)
    w = [1 / 16, 4 / 16, 6 / 16, 4 / 16, 1 / 16]
    passes = [(0, w), (1, w), (2, w)]
    ms = time_call(lambda: n.convolve_axes(src, dst, passes, BorderMode.Wrap), it)
    vox = base.numel()
    out["u8_binomial_256^3_view_x4"] = {"ms": round(ms, 4), "gvoxel_s": round(vox / ms / 1e6, 2),
                                        "gbs": round(2.0 * vox / ms / 1e6, 1),
                                        "frac_of_measured_hbm": round(2.0 * vox / ms / 1e6 / hbm, 4),
                                        "exact": "bit-exact integer path"}
    del base, src, dst


def gradient_form(n, g, it, hbm, out):
    import torch
    from ndl_b200 import BorderMode, Image
    # gradient (convolution.h:359-388): 256^3 f32 -> {3, 256^3} central
    # differences, Reflect; 16 algorithmic bytes per voxel (read 4, write 12)
    x = torch.randn((256, 256, 256), generator=g, device="cuda")
    s = Image.from_tensor(x)
    o = Image.empty([3, 256, 256, 256], torch.float32)
    ms = time_call(lambda: n.gradient(s, o, BorderMode.Reflect), it)
    vox = x.numel()
    out["gradient_f32_256^3"] = {"ms": round(ms, 4), "gvoxel_s": round(vox / ms / 1e6, 2),
                                 "gbs": round(16.0 * vox / ms / 1e6, 1),
                                 "frac_of_measured_hbm": round(16.0 * vox / ms / 1e6 / hbm, 4)}
    del x, s, o


def gaussian_forms(n, g, it, hbm, out):
    import torch
    from ndl_b200 import BorderMode, Image
    # gaussian_blur of a 256^3 f32 volume (one sigma on every axis, Reflect)
    # at sigma 1, 2 and 3: the fused 3-pass kernels of 7, 13 and 19 taps; at
    # sigma 4 and 6 (25 and 37 taps): three tiled passes through f32 scratch
    x = torch.rand((256, 256, 256), generator=g, device="cuda")
    s = Image.from_tensor(x)
    o = Image.empty(s.extent(), torch.float32)
    for sg in (1.0, 2.0, 3.0, 4.0, 6.0):
        ms = time_call(lambda: n.gaussian_blur(s, o, sg, BorderMode.Reflect), it)
        out["gaussian_blur_f32_256^3_sigma%g" % sg] = {
            "ms": round(ms, 4), "gvoxel_s": round(x.numel() / ms / 1e6, 2), "gbs": round(8.0 * x.numel() / ms / 1e6, 1),
            "frac_of_measured_hbm": round(8.0 * x.numel() / ms / 1e6 / hbm, 4)}
    del x, s, o


def stencil_form(n, g, it, hbm, out):
    import torch
    from ndl_b200 import BorderMode, Image
    # convolve() with a full (non-separable) 5x5 kernel on a 4096^2 f32 image
    x = torch.rand((4096, 4096), generator=g, device="cuda")
    s = Image.from_tensor(x)
    o = Image.empty(s.extent(), torch.float32)
    ker = np.random.default_rng(SEED).random((5, 5)) + 0.1
    ms = time_call(lambda: n.convolve(s, o, ker, BorderMode.Reflect), it)
    out["convolve_full5x5_f32_4096^2"] = {"ms": round(ms, 4), "gpixel_s": round(x.numel() / ms / 1e6, 2),
                                          "gbs": round(8.0 * x.numel() / ms / 1e6, 1),
                                          "frac_of_measured_hbm": round(8.0 * x.numel() / ms / 1e6 / hbm, 4)}
    del x, s, o


def learnable_form(n, g, it, out):
    import torch
    from ndl_b200 import BorderMode, Image
    # a learnable 3-tap-per-axis separable filter on eight 192^3 f32 volumes:
    # forward, dL/dX and the 9 tap gradients of one training step
    X = torch.randn((8, 192, 192, 192), generator=g, device="cuda")
    W = torch.randn_like(X)
    Y, GX = torch.empty_like(X), torch.empty_like(X)
    T = torch.zeros(9, device="cuda")
    xi, wi, yi, gi = (Image.from_tensor(t) for t in (X, W, Y, GX))
    taps3 = [(a, np.random.default_rng(SEED + a).standard_normal(3)) for a in range(3)]

    def small_step():
        n.convolve_axes(xi, yi, taps3, BorderMode.Reflect)
        n.convolve_axes_adjoint(wi, xi, gi, taps3, BorderMode.Reflect, T)

    ms = time_call(small_step, it)
    out["learnable_3tap_step_f32_8x192^3"] = {"ms": round(ms, 4), "gvoxel_s": round(X.numel() / ms / 1e6, 2),
                                              "note": "forward + dL/dX + 9 tap gradients"}
    del X, W, Y, GX, xi, wi, yi, gi


def downsample_form(n, g, it, hbm, out):
    import torch
    from ndl_b200 import Image
    # downsample (convolution.h:241-305): a {3, 15360, 8640} uint8 colour
    # image (channel axis 0, 398 MB) by 2; algorithmic bytes = source + result
    x = torch.randint(0, 256, (8640, 15360, 3), generator=g, device="cuda", dtype=torch.uint8)
    s = Image.from_tensor(x)
    o = Image.empty([3, 7680, 4320], torch.uint8)
    ms = time_call(lambda: n.downsample(s, 2, 0, dst=o), it)
    nb = x.numel() * 1.25
    out["downsample_u8_rgb_15360x8640_f2"] = {"ms": round(ms, 4), "gbs": round(nb / ms / 1e6, 1),
                                              "frac_of_measured_hbm": round(nb / ms / 1e6 / hbm, 4),
                                              "exact": "bit-exact block averages"}
    del x, s, o


def box_blur_form(n, g, it, hbm, out):
    import torch
    from ndl_b200 import BorderMode, Image
    # box_blur (summed_area_table.h:300-339): 4096^2 f32, radius 8, Clamp,
    # the reference's double summed-area table (bit-exact)
    x = torch.rand((4096, 4096), generator=g, device="cuda")
    s = Image.from_tensor(x)
    o = Image.empty(s.extent(), torch.float32)
    ws = torch.empty(n.box_blur_workspace_size(s, o, 8), dtype=torch.uint8, device="cuda")
    ms = time_call(lambda: n.box_blur(s, o, 8, BorderMode.Clamp, workspace=ws), it)
    out["box_blur_f32_4096^2_r8"] = {"ms": round(ms, 4), "mpix_s": round(x.numel() / ms / 1e3, 1),
                                     "gbs": round(8.0 * x.numel() / ms / 1e6, 1),
                                     "frac_of_measured_hbm": round(8.0 * x.numel() / ms / 1e6 / hbm, 4),
                                     "exact": "bit-exact (the reference's double summed-area table, 8 B/element "
                                              "scratch written and re-read per axis)"}
    del x, s, o, ws


def video_forms(n, g, it, hbm, out, sel=""):
    import torch
    from ndl_b200 import BorderMode, Image
    from ndl_b200.convolution import gaussian_taps
    # config 5: 4-D video 1024x1024x3x96, sigma (2.5, 2.5, -, 1.5), Reflect:
    # the forward (gaussian_blur_axes) and the input gradient of the same chain
    for name, dt in (("video_bf16", torch.bfloat16), ("video_f16", torch.float16), ("video_f32", torch.float32)):
        if sel and not (name.startswith(sel) or sel.startswith(name)):
            continue
        v = torch.rand((96, 3, 1024, 1024), generator=g, device="cuda", dtype=torch.float32)
        salt = torch.rand(v.shape, generator=g, device="cuda") < 0.01
        v[salt] = 1.0
        v = v.to(dt)
        s = Image.from_tensor(v)
        o = Image.empty(s.extent(), dt)
        ms = time_call(lambda: n.gaussian_blur_axes(s, o, [2.5, 2.5, 0.0, 1.5], BorderMode.Reflect), max(3, it // 4))
        vox = v.numel()
        es = v.element_size()
        out[name] = {"ms": round(ms, 3), "gvoxel_s": round(vox / ms / 1e6, 2), "gbs": round(2.0 * es * vox / ms / 1e6, 1),
                     "frac_of_measured_hbm": round(2.0 * es * vox / ms / 1e6 / hbm, 4)}
        passes = [(0, gaussian_taps(2.5)), (1, gaussian_taps(2.5)), (3, gaussian_taps(1.5))]
        ga = Image.empty(s.extent(), dt)
        ms = time_call(lambda: n.convolve_axes_adjoint(s, None, ga, passes, BorderMode.Reflect), max(3, it // 4))
        out[name + "_adjoint"] = {"ms": round(ms, 3), "gvoxel_s": round(vox / ms / 1e6, 2),
                                  "gbs": round(2.0 * es * vox / ms / 1e6, 1),
                                  "frac_of_measured_hbm": round(2.0 * es * vox / ms / 1e6 / hbm, 4)}
        del v, s, o, salt, ga
        if not sel:
            out[name]["error_vs_fp64"] = video_error(dt)


def gauss2d_form(n, g, out):
    import torch
    from ndl_b200 import BorderMode, Image
    # config 1: 2-D 512^2 gaussian sigma 2 (L2-resident; launch-bound)
    im = torch.rand((512, 512), generator=g, device="cuda")
    s = Image.from_tensor(im)
    o = Image.empty(s.extent(), torch.float32)
    ms = time_call(lambda: n.gaussian_blur(s, o, 2.0, BorderMode.Clamp), 50)
    out["gauss2d_512_f32"] = {"ms": round(ms, 4), "gvoxel_s": round(im.numel() / ms / 1e6, 3),
                              "note": "2 MB, L2-resident and launch-bound"}


def sharded_config4(world, rank, dev, hbm, reps=10):
    """Config 4 (FP32 forward) partitioned over `world` ranks by cost; every
    rank times its own batched launch (graph replay, CUDA events) and the
    job's time is the max over ranks."""
    import torch

    from ndl_b200 import Image
    from ndl_b200.batch import Batch
    from ndl_b200.shard import instance_cost, job_time_ms, partition

    inst = config4_instances()
    costs = [instance_cost(sh, [len(w) for _, w in passes]) for sh, passes, _ in inst]
    mine = partition(costs, world)[rank]
    g = torch.Generator(device=dev)
    g.manual_seed(SEED + 7)
    b = Batch()
    keep = []
    for i in mine:
        sh, passes, border = inst[i]
        x = torch.rand(sh, generator=g, device=dev)
        y = torch.empty_like(x)
        b.add(Image.from_tensor(x), Image.from_tensor(y), passes, border)
        keep += [x, y]
    b.plan()
    # graph capture needs a stream other than the legacy default one
    stream = torch.cuda.Stream(dev)
    torch.cuda.synchronize(dev)
    for _ in range(3):
        b.graph_launch(stream)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        b.graph_launch(stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = job_time_ms(e0.elapsed_time(e1) / reps, device=dev)
    b.close()
    elems = sum(int(np.prod(sh)) for sh, _, _ in inst)
    return {"ms": round(ms, 4), "gvoxel_s": round(elems / ms / 1e6, 2), "instances": len(inst),
            "ranks": world, "instances_this_rank": len(mine),
            "note": "instances partitioned by cost (elements x taps) with no data-path collective; "
                    "job time = max over ranks"}


def config4_instances(seed=SEED):
    """512 instances: 256 2-D images with sides log-uniform in [64, 2048] and
    256 3-D volumes with sides log-uniform in [32, 160]; per axis a Gaussian
    sigma uniform in [0.5, 6] (radius ceil(3 sigma)); border uniform over
    Clamp/Wrap/Reflect; values uniform [0, 1)."""
    from ndl_b200.convolution import gaussian_taps
    rng = np.random.default_rng(seed)
    inst = []
    for i in range(512):
        if i < 256:
            shape = tuple(int(round(v)) for v in np.exp(rng.uniform(np.log(64), np.log(2048), 2)))
        else:
            shape = tuple(int(round(v)) for v in np.exp(rng.uniform(np.log(32), np.log(160), 3)))
        border = int(rng.integers(0, 3))
        passes = [(ax, gaussian_taps(float(rng.uniform(0.5, 6.0)))) for ax in range(len(shape))]
        inst.append((shape, passes, border))
    return inst


def batched_forms(hbm, count=512, tile=None, plain=True):
    """Config 4 in one persistent launch per direction (graph replay):
    the first `count` instances, tiles from the autotuner unless `tile`
    names a configuration."""
    import torch

    import ndl_b200 as n
    from ndl_b200 import Image
    from ndl_b200.autotune import best_tile_config
    from ndl_b200.batch import Batch

    res = {}
    inst = config4_instances()[:count]
    elems = sum(int(np.prod(sh)) for sh, _, _ in inst)
    g = torch.Generator(device="cuda")
    g.manual_seed(SEED)
    stream = torch.cuda.Stream()
    for name, dt in (("f32", torch.float32), ("bf16", torch.bfloat16)):
        xs = [torch.rand(sh, generator=g, device="cuda", dtype=torch.float32).to(dt) for sh, _, _ in inst]
        ys = [torch.empty_like(x) for x in xs]
        gs = [torch.empty_like(x) for x in xs]
        xi = [Image.from_tensor(x) for x in xs]
        yi = [Image.from_tensor(y) for y in ys]
        gi = [Image.from_tensor(v) for v in gs]
        fwd, adj = Batch(), Batch()
        for (sh, passes, border), a, b, c in zip(inst, xi, yi, gi):
            fwd.add(a, b, passes, border)
            adj.add(b, c, passes, border, adjoint=True)
        if tile is None:
            cfg_f, _ = best_tile_config(fwd)
            cfg_a, _ = best_tile_config(adj)
        else:
            fwd.plan(tile)
            adj.plan(tile)
            cfg_f = cfg_a = tile
        for tag, b in (("fwd", fwd), ("adj", adj)):
            with torch.cuda.stream(stream):
                for _ in range(3):
                    b.graph_launch(stream)
                stream.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(5):
                    b.graph_launch(stream)
                e1.record(stream)
                stream.synchronize()
            ms = e0.elapsed_time(e1) / 5
            es = xs[0].element_size()
            res["batched_%s_%s" % (name, tag)] = {
                "ms": round(ms, 3), "gvoxel_s": round(elems / ms / 1e6, 2),
                "gbs": round(2.0 * es * elems / ms / 1e6, 1),
                "frac_of_measured_hbm": round(2.0 * es * elems / ms / 1e6 / hbm, 4),
                "instances": len(inst), "elements": elems, "tile_config": cfg_f if tag == "fwd" else cfg_a}
        if name == "f32" and plain:
            # the plain path: one convolve_axes call per instance (FP32)
            def plain():
                for (sh, passes, border), a, b in zip(inst, xi, yi):
                    n.convolve_axes(a, b, passes, border)
            ms = time_call(plain, 3, warm=3)
            res["plain_f32_fwd_per_call"] = {"ms": round(ms, 3), "gvoxel_s": round(elems / ms / 1e6, 2),
                                             "instances": len(inst), "elements": elems}
        fwd.close()
        adj.close()
        del xs, ys, gs, xi, yi, gi
        torch.cuda.empty_cache()
    return res


# ---------------------------------------------------------------------------
# CPU baseline: the compiled ndl reference (forward) and the FP64 port (the
# reference has no adjoint)
# ---------------------------------------------------------------------------

def step_config(world):
    """The workload of one step, the same for both arms (per GPU / replica)."""
    return {"workload": "config 3: %d volumes of %d^3 f32 per step, per-axis 9-tap L1-normalised N(0,1) "
                        "kernels, Reflect; forward + adjoint (dL/dX and 27 tap gradients of sum(W*Y))"
                        % (BATCH, EDGE),
            "voxels_per_step": BATCH * EDGE ** 3, "l2": "inputs larger than L2 (226 MB per tensor)",
            "parallelism": "replicas%d" % world}


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def cpu_sample(depth, seed=SEED):
    """One bounded sample: a 192 x 192 x depth f32 volume, forward through
    the reference (or the port when the reference is absent) + FP64 port
    adjoint.  Returns (voxels, seconds, kind)."""
    from oracle import oracle as O
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((depth, EDGE, EDGE)).astype(np.float32)
    wv = rng.standard_normal((depth, EDGE, EDGE)).astype(np.float32)
    passes = make_taps()
    t0 = time.perf_counter()
    if O.have_reference():
        O.ref_compose(x, passes, O.REFLECT, np.float32)
        kind = "reference"
    else:
        O.compose(x, passes, O.REFLECT, O.F32)
        kind = "port"
    O.compose_adjoint(wv, x, passes, O.REFLECT)
    return x.size, time.perf_counter() - t0, kind


def cpu_baseline_sample(volumes=5):
    """About 10 s of single-thread CPU work: `volumes` 192^3 f32 volumes of
    the headline step (5 of the 8 a GPU step processes)."""
    vox, sec, kind = 0, 0.0, "reference"
    for i in range(volumes):
        v, s, kind = cpu_sample(EDGE, SEED + i)
        vox += v
        sec += s
    return {"value": round(vox / sec / 1e9, 6), "unit": "Gvoxel/s", "cores": 1, "kind": kind,
            "sample": "%d f32 volumes of 192^3 (of the 8 per step), single thread: forward = ndl convolve() x3 "
                      "(compiled reference, -O3) + adjoint = FP64 oracle port (ndl has no adjoint); %.1f s; %s"
                      % (volumes, sec, _cpu_model())}


def run_reference(args):
    """--impl reference: the reference's own CPU path on the host cores, on
    the GPU arm's step (BATCH volumes of 192^3): one volume per thread, the
    volumes in parallel (ndl's convolve() is single-threaded and re-entrant,
    processing/convolution.h:64-70; the oracle's C loops release the GIL).
    The inputs are made once, outside the timing.  Each step runs every
    volume whole when K + W steps of that fit in about 150 s; otherwise each
    step runs the same z-slab depth of every volume (rotating through it),
    the depth chosen from the first warm-up step so the run stays bounded."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle as O
    threads = min(os.cpu_count() or 1, BATCH)
    K, Wm = args.steps, max(3, args.warmup)
    ex = ThreadPoolExecutor(threads)
    passes = make_taps()
    vols = []
    for i in range(BATCH):
        rng = np.random.default_rng(SEED + i)
        vols.append((rng.standard_normal((EDGE, EDGE, EDGE)).astype(np.float32),
                     rng.standard_normal((EDGE, EDGE, EDGE)).astype(np.float32)))
    kind = "reference" if O.have_reference() else "port"

    def one(i, z0, depth):
        x = np.ascontiguousarray(vols[i][0][z0:z0 + depth])
        w = np.ascontiguousarray(vols[i][1][z0:z0 + depth])
        if kind == "reference":
            O.ref_compose(x, passes, O.REFLECT, np.float32)
        else:
            O.compose(x, passes, O.REFLECT, O.F32)
        O.compose_adjoint(w, x, passes, O.REFLECT)
        return x.size

    def step(k, depth):
        z0 = (k * depth) % (EDGE - depth + 1)
        t0 = time.perf_counter()
        vox = sum(ex.map(lambda i: one(i, z0, depth), range(BATCH)))
        return vox, time.perf_counter() - t0

    _, t_full = step(0, EDGE)
    depth = EDGE
    if t_full * (K + Wm) > 150.0:
        depth = max(16, min(EDGE, int(EDGE * 150.0 / (t_full * (K + Wm)))))
    for k in range(1, Wm):
        step(k, depth)
    vox, sec = 0, 0.0
    for k in range(K):
        v, t = step(k, depth)
        vox += v
        sec += t
    ex.shutdown()
    value = vox / sec / 1e9
    what = ("the GPU arm's %d volumes of 192^3 f32" % BATCH if depth == EDGE else
            "a %d-plane z-slab of each of the GPU arm's %d volumes of 192^3 f32 (rotating; whole volumes take "
            "%.1f s a step)" % (depth, BATCH, t_full))
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": "Gvoxel/s", "n_gpus": world,
            "steps": K, "warmup": Wm, "ms_per_step": round(1e3 * sec / K, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": step_config(world),
            "cpu_baseline": {"value": round(value, 6), "unit": "Gvoxel/s", "cores": threads, "kind": kind,
                             "sample": "every step %s, one volume per thread on %d threads: forward = ndl "
                                       "convolve() x3 (compiled reference) + adjoint = FP64 oracle port (ndl has "
                                       "no adjoint); inputs made before the timing; %s" % (what, threads,
                                                                                          _cpu_model())},
            "e2e": {"value": round(value, 6), "unit": "Gvoxel/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ndlgpu", choices=["ndlgpu", "reference"])
    ap.add_argument("--skip-forms", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--batched-only", type=int, default=0, metavar="N",
                    help="run only the batched form on the first N config-4 instances (profiling)")
    ap.add_argument("--batched-tile", type=int, default=None, help="tile configuration instead of the autotuner")
    ap.add_argument("--only", default="", choices=["", "fwd", "adj"],
                    help="time only one half of the step (for profiling captures)")
    ap.add_argument("--form", default="",
                    help="run only the other form(s) whose name starts with this (e.g. video_bf16, gradient, "
                         "u8_binomial, convolve_full5x5): for profiling captures; prints their timings")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.form:
        hbm, _ = peaks()
        print(json.dumps(other_forms(args, hbm)))
    elif args.batched_only:
        hbm, _ = peaks()
        print(json.dumps(batched_forms(hbm, args.batched_only, args.batched_tile, plain=False)))
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
