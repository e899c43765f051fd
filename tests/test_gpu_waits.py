"""Bounded device waits that run out, without any fault.

The tensor-map plane loads of the fused forward and adjoint and the phase
waits of the batched form poll a bounded number of times; when the bound is reached the
kernel sets a guard bit, lets its own copies in flight land and returns, and
ndlgpu_device_status reports the bit.  ndlgpu_test_wait_timeouts makes those
waits ask for more than ever arrives (an mbarrier announced 16 bytes more
than the copy delivers; a phase wait one predecessor item too many) with a
short poll bound, so the timeout path runs; then normal operation is restored
and the same call is checked against the FP64 oracle.
"""
import ctypes

import numpy as np
import pytest
import torch

import ndl_b200 as n
from ndl_b200 import Image, abi
from ndl_b200.batch import Batch
from oracle import oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.sets_guards]


def _status():
    code = ctypes.c_int32(-1)
    abi.check(abi.load().ndlgpu_device_status(None, ctypes.byref(code)))
    return code.value


def _controls(spins, unreachable):
    abi.check(abi.load().ndlgpu_test_wait_timeouts(spins, unreachable))


def _passes(rng, k=9):
    out = []
    for ax in range(3):
        w = rng.standard_normal(k)
        out.append((ax, w / np.abs(w).sum()))
    return out


def test_tensor_map_plane_wait_runs_out_and_reports():
    rng = np.random.default_rng(3)
    # rows of 64 elements: whole 64-column tiles, so the plane loads go
    # through the tensor map
    g = rng.standard_normal((40, 48, 64)).astype(np.float32)
    passes = _passes(rng)
    gi = Image.from_tensor(torch.from_numpy(g).cuda())
    gx = Image.empty(gi.extent(), torch.float32)
    assert _status() == 0
    _controls(64, 1)
    try:
        n.convolve_axes_adjoint(gi, None, gx, passes, n.BorderMode.Reflect)
        code = _status()
    finally:
        _controls(0, 0)
    assert code & 2, code
    # normal operation again: the same call is right and fires nothing
    n.convolve_axes_adjoint(gi, None, gx, passes, n.BorderMode.Reflect)
    torch.cuda.synchronize()
    assert _status() == 0
    ref = g.astype(np.float64)
    for ax, w in passes[::-1]:
        ref = O.axis_pass_adjoint(ref, ax, w, O.REFLECT)
    err = np.abs(gx.tensor().cpu().numpy() - ref).max() / np.abs(ref).max()
    assert err <= 1e-5, err


def test_forward_plane_wait_runs_out_and_reports():
    # the forward's tensor-map plane loads (64-wide rows, Reflect)
    rng = np.random.default_rng(6)
    x = rng.standard_normal((24, 32, 64)).astype(np.float32)
    passes = _passes(rng)
    xi = Image.from_tensor(torch.from_numpy(x).cuda())
    y = Image.empty(xi.extent(), torch.float32)
    assert _status() == 0
    _controls(64, 1)
    try:
        n.convolve_axes(xi, y, passes, n.BorderMode.Reflect)
        code = _status()
    finally:
        _controls(0, 0)
    assert code & 2, code
    n.convolve_axes(xi, y, passes, n.BorderMode.Reflect)
    torch.cuda.synchronize()
    assert _status() == 0
    ref = O.compose_total(x.astype(np.float64), passes, O.REFLECT)
    mag = O.compose_total(np.abs(x).astype(np.float64), [(a, np.abs(w)) for a, w in passes], O.REFLECT)
    assert (np.abs(y.tensor().cpu().numpy() - ref) <= 1e-6 * mag + 1e-30).all()


def test_batched_phase_wait_runs_out_and_reports():
    rng = np.random.default_rng(4)
    shapes = [(20, 24, 30), (17, 33, 25)]
    xs = [rng.random(s).astype(np.float32) for s in shapes]
    passes = [[(ax, O.gaussian_weights(1.0 + 0.5 * ax)) for ax in range(3)] for _ in shapes]
    b = Batch()
    outs = []
    for x, p in zip(xs, passes):
        src = Image.from_tensor(torch.from_numpy(x).cuda())
        dst = Image.empty(src.extent(), torch.float32)
        b.add(src, dst, p, O.CLAMP, adjoint=False)
        outs.append(dst)
    b.plan()
    assert _status() == 0
    _controls(1000, 1)
    try:
        b.launch()
        code = _status()
    finally:
        _controls(0, 0)
    assert code & 4, code
    b.launch()
    torch.cuda.synchronize()
    assert _status() == 0
    for x, p, dst in zip(xs, passes, outs):
        ref = O.compose_total(x.astype(np.float64), p, O.CLAMP)
        mag = O.compose_total(np.abs(x).astype(np.float64), [(a, np.abs(w)) for a, w in p], O.CLAMP)
        err = np.abs(dst.tensor().cpu().numpy() - ref)
        assert (err <= 1e-6 * mag + 1e-30).all()
