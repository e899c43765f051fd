"""Element-wise parity with the FP64 oracle at the workloads' full shapes.

* Configuration 3 -- the benchmark's own launch: eight 192^3 f32 volumes,
  the benchmark's 9-tap L1-normalised N(0,1) kernels, Reflect.  The forward,
  dL/dX and all 27 tap gradients against ``O.compose_total`` /
  ``O.compose_adjoint`` on every voxel of every volume (the oracle runs one
  volume per thread; its C loops release the GIL).
* Configuration 5 -- 1024 x 1024 x 3 x 96 video, BF16 and FP16 storage,
  sigma (2.5, 2.5, -, 1.5), Reflect: whole output t-planes at both t-borders
  and in the middle, forward and dL/dX, against FP64.  The x/y passes of
  every input plane those outputs read come from the oracle on that plane
  (plane-local, exact); the t pass is the oracle's own 1-D pass applied to
  unit vectors (the 96 x 96 matrix P with the border map built in), so
  out[t] = sum_s P[t, s] XY[s] and gx[t] = sum_s P[s, t] XY^T[s].
* Configuration 4 -- the 512 uneven instances in one batched launch: a
  stratified subset of 16 (8 images, 8 volumes, smallest to largest) against
  the oracle's composition.

Bounds are relative to the stencil magnitude (the same chain on |x| and
|w|): FP32 1e-6 (forward) and 2e-6 (dL/dX), tap gradients 2e-5 of their
magnitude sums, 16-bit storage 4e-3.
"""
import concurrent.futures as cf

import numpy as np
import pytest
import torch

import ndl_b200 as n
from ndl_b200 import BorderMode, Image
from ndl_b200.batch import Batch
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _pool():
    return cf.ThreadPoolExecutor(max_workers=8)


def _bound_check(got, ref, mag, tol, what):
    err = np.abs(np.asarray(got, np.float64) - ref)
    bound = tol * mag + 1e-30
    bad = err > bound
    assert not bad.any(), "%s: %d mismatches, worst err/bound %.3g" % (what, int(bad.sum()), float((err / bound).max()))


def test_config3_full_batch_elementwise():
    import bench
    g = torch.Generator(device=DEV)
    g.manual_seed(31)
    shape = (8, 192, 192, 192)
    X = torch.randn(shape, generator=g, device=DEV)
    W = torch.randn(shape, generator=g, device=DEV)
    passes = bench.make_taps()
    xi, wi = Image.from_tensor(X), Image.from_tensor(W)
    Y = torch.empty_like(X)
    GX = torch.empty_like(X)
    taps = torch.zeros(27, dtype=torch.float64, device=DEV)
    n.convolve_axes(xi, Image.from_tensor(Y), passes, BorderMode.Reflect)
    n.convolve_axes_adjoint(wi, xi, Image.from_tensor(GX), passes, BorderMode.Reflect, taps)
    torch.cuda.synchronize()
    xh, wh, yh, gxh = X.cpu().numpy(), W.cpu().numpy(), Y.cpu().numpy(), GX.cpu().numpy()
    apasses = [(a, np.abs(w)) for a, w in passes]

    def one(b):
        x = xh[b].astype(np.float64)
        w = wh[b].astype(np.float64)
        ref = O.compose_total(x, passes, O.REFLECT)
        mag = O.compose_total(np.abs(x), apasses, O.REFLECT)
        _bound_check(yh[b], ref, mag, 1e-6, "forward, volume %d" % b)
        gref, tref = O.compose_adjoint(w, x, passes, O.REFLECT)
        gmag, tmag = O.compose_adjoint(np.abs(w), np.abs(x), apasses, O.REFLECT)
        _bound_check(gxh[b], gref, gmag, 2e-6, "dL/dX, volume %d" % b)
        return np.concatenate(tref), np.concatenate(tmag)

    with _pool() as ex:
        parts = list(ex.map(one, range(8)))
    tref = np.sum([p[0] for p in parts], axis=0)
    tmag = np.sum([p[1] for p in parts], axis=0)
    _bound_check(taps.cpu().numpy(), tref, tmag, 2e-5, "tap gradients")


def _t_matrix(w, nt, border):
    """P[t, s]: the oracle's 1-D pass along t applied to the unit vectors."""
    P = np.zeros((nt, nt))
    for s in range(nt):
        e = np.zeros(nt)
        e[s] = 1.0
        P[:, s] = O.axis_pass_total(e, 0, w, border)
    return P


@pytest.mark.parametrize("tdt", [torch.bfloat16, torch.float16])
def test_config5_video_full_elementwise_vs_fp64(tdt):
    g = torch.Generator(device=DEV)
    g.manual_seed(51)
    shape = (96, 3, 1024, 1024)       # (t, c, y, x): ndl axes x, y, c, t
    v = torch.rand(shape, generator=g, device=DEV)
    salt = torch.rand(shape, generator=g, device=DEV) < 0.01
    v = torch.where(salt, torch.ones_like(v), v).to(tdt)
    gr = (torch.rand(shape, generator=g, device=DEV) - 0.5).to(tdt)
    wxy, wt = O.gaussian_weights(2.5), O.gaussian_weights(1.5)
    passes = [(0, wxy), (1, wxy), (3, wt)]
    out = Image.empty(Image.from_tensor(v).extent(), tdt)
    gx = Image.empty(Image.from_tensor(v).extent(), tdt)
    n.convolve_axes(Image.from_tensor(v), out, passes, BorderMode.Reflect)
    n.convolve_axes_adjoint(Image.from_tensor(gr), None, gx, passes, BorderMode.Reflect)
    torch.cuda.synchronize()
    T = [0, 1, 2, 3, 4, 5, 47, 48, 90, 91, 92, 93, 94, 95]
    P = _t_matrix(wt, 96, O.REFLECT)
    need_f = sorted({s for t in T for s in np.nonzero(P[t])[0]})
    need_a = sorted({s for t in T for s in np.nonzero(P[:, t])[0]})
    vf = v.float().cpu().numpy()
    gf = gr.float().cpu().numpy()

    def xy(s):                                    # forward x/y passes of input plane s
        pl = vf[s].astype(np.float64)
        return O.axis_pass_total(O.axis_pass_total(pl, 0, wxy, O.REFLECT), 1, wxy, O.REFLECT)

    def xyt(s):                                   # their transpose on gradient plane s, and its magnitude
        pl = gf[s].astype(np.float64)
        a = O.axis_pass_adjoint(O.axis_pass_adjoint(pl, 1, wxy, O.REFLECT), 0, wxy, O.REFLECT)
        m = O.axis_pass_adjoint(O.axis_pass_adjoint(np.abs(pl), 1, wxy, O.REFLECT), 0, wxy, O.REFLECT)
        return a, m

    with _pool() as ex:
        XY = dict(zip(need_f, ex.map(xy, need_f)))
        XYT = dict(zip(need_a, ex.map(xyt, need_a)))
    got_f = out.tensor().float().cpu().numpy()
    got_a = gx.tensor().float().cpu().numpy()
    for t in T:
        ref = sum(P[t, s] * XY[s] for s in need_f if P[t, s] != 0.0)
        # inputs in [0, 1] and positive taps: the magnitude is the output
        _bound_check(got_f[t], ref, np.abs(ref), 4e-3, "video forward, t=%d" % t)
        gref = sum(P[s, t] * XYT[s][0] for s in need_a if P[s, t] != 0.0)
        gmag = sum(P[s, t] * XYT[s][1] for s in need_a if P[s, t] != 0.0)
        _bound_check(got_a[t], gref, gmag, 4e-3, "video dL/dX, t=%d" % t)


def test_config4_stratified_subset_vs_oracle():
    import bench
    inst = bench.config4_instances()
    g = torch.Generator(device=DEV)
    g.manual_seed(41)
    xs = [torch.rand(sh, generator=g, device=DEV) for sh, _, _ in inst]
    b = Batch()
    outs = []
    for (sh, passes, border), x in zip(inst, xs):
        o = Image.empty(Image.from_tensor(x).extent(), torch.float32)
        b.add(Image.from_tensor(x), o, passes, border)
        outs.append(o)
    b.plan()
    b.launch()
    torch.cuda.synchronize()
    # 8 images and 8 volumes, evenly spread over their size order
    pick = []
    for lo, hi in ((0, 256), (256, 512)):
        order = sorted(range(lo, hi), key=lambda i: int(np.prod(inst[i][0])))
        pick += [order[int(round(j * (len(order) - 1) / 7))] for j in range(8)]

    def one(i):
        sh, passes, border = inst[i]
        x = xs[i].cpu().numpy().astype(np.float64)
        ref = O.compose_total(x, passes, border)
        # values in [0, 1), positive Gaussian taps: the magnitude is the output
        _bound_check(outs[i].tensor().cpu().numpy(), ref, np.abs(ref), 1e-6,
                     "instance %d %s border %d" % (i, sh, border))

    with _pool() as ex:
        list(ex.map(one, pick))
    b.close()
