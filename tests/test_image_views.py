"""ndl_b200.Image's view arithmetic against the reference's own Image view
builders (image/core.h:647-757, run through oracle/_ref)."""
import pytest
import torch

from ndl_b200 import Image
from oracle import oracle as O

needs_ref = pytest.mark.skipif(not O.have_reference(), reason="compiled reference not present")


def _probe_ours(base_ext, ops):
    n = 1
    for e in base_ext:
        n *= e
    img = Image(torch.zeros(n, dtype=torch.uint8), 0, base_ext, [0] * len(base_ext))
    st, m = [], 1
    for e in base_ext:
        st.append(m)
        m *= e
    img = Image(img._storage, 0, base_ext, st)
    for op in ops:
        if op[0] == "swap":
            img = img.swap_axes(op[1], op[2])
        elif op[0] == "mirror":
            img = img.mirror(op[1])
        else:
            _, ax, s, e, step = op
            start = [0] * img.dim
            end = [-1] * img.dim
            stp = [1] * img.dim
            start[ax], end[ax], stp[ax] = s, e, step
            img = img.view(start, end, stp)
    return img._offset, img.extent(), img.stride()


CASES = [
    ([64, 64, 64], [("swap", 0, 2), ("mirror", 1)]),
    ([10, 7], [("mirror", 0), ("mirror", 0)]),
    ([10, 7, 5], [("view", 0, 1, 8, 3), ("swap", 0, 1)]),
    ([10, 7, 5], [("view", 1, 0, -1, -2), ("mirror", 2)]),
    ([9, 8, 7, 6], [("swap", 1, 3), ("view", 2, 2, 5, -1), ("mirror", 0)]),
    ([13], [("view", 0, 2, 12, 5)]),
    ([13], [("view", 0, 2, 12, -5)]),
]


@needs_ref
@pytest.mark.parametrize("base,ops", CASES)
def test_views_match_reference(base, ops):
    assert _probe_ours(base, ops) == tuple(O.ref_view_probe(base, ops))


def test_config2_view_strides():
    # swap_axes(0,2).mirror(1) of a contiguous 64^3 gives strides {4096,-64,1}
    off, ext, st = _probe_ours([64, 64, 64], [("swap", 0, 2), ("mirror", 1)])
    assert st == [4096, -64, 1] and off == 63 * 64 and ext == [64, 64, 64]


def test_tensor_roundtrip_of_mirrored_view():
    t = torch.arange(24, dtype=torch.float32).reshape(2, 3, 4)
    img = Image.from_tensor(t)
    v = img.swap_axes(0, 2).mirror(1)
    ref = t.permute(2, 1, 0).flip(1)
    assert torch.equal(v.tensor(), ref)
