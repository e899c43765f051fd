"""bench.py's FP64 PyTorch blur reference (used to state the 16-bit video
error) against the FP64 oracle, on the CPU: the same taps, borders and
summation up to FP64 rounding."""
import numpy as np
import torch

import bench
from oracle import oracle as O


def test_fp64_blur_reference_matches_oracle():
    rng = np.random.default_rng(3)
    x = rng.random((5, 3, 20, 24))
    sig = (2.5, 2.5, 0.0, 1.5)
    got = bench.fp64_blur_reference(torch.from_numpy(x), sig).numpy()
    ref = O.compose_total(x, [(ax, O.gaussian_weights(s)) for ax, s in enumerate(sig) if s > 0], O.REFLECT)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
