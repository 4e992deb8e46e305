"""Host-array copies (the drop-in entry points' transfers): the first large
copy of a context goes through pageable memory, later ones through the
context's pinned chunk buffers and host threads; both must move every byte,
for sizes that are not multiples of a chunk or of a host task, and the
transforms must give bitwise the same results either way."""
import numpy as np
import pytest

import oracle as O
from conftest import wrt

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nbytes", [(1 << 20) + 7, (9 << 20) + 12345, 3 << 20])
def test_round_trip_through_both_paths(ctx, nbytes):
    rng = np.random.default_rng(nbytes)
    buf = wrt.DeviceBuffer(ctx, nbytes)
    for k in range(3):  # pageable first, then the pinned pipeline
        a = rng.integers(0, 256, nbytes, dtype=np.uint8)
        buf.upload(a)
        b = np.empty_like(a)
        buf.download(b)
        assert np.array_equal(a, b), k
    buf.close()


def test_transforms_repeat_bitwise(ctx):
    n = 96  # FP64 volume 7 MB, rays 4.7 MB
    vol = np.random.default_rng(5).standard_normal((n, n, n)) * 0.1
    first = ctx.ray_grid(vol, n, 96, 64)
    second = ctx.ray_grid(vol, n, 96, 64)
    assert np.array_equal(first, second)
    R = np.random.default_rng(6).standard_normal((128, 64, 32))  # 2.1 MB
    a1 = ctx.radon3d_adjoint(R, 64)
    a2 = ctx.radon3d_adjoint(R, 64)
    assert np.array_equal(a1, a2)
    # the FP64 volume is rounded to FP32 on the host, through a temporary
    # array on a context's first large copy and while staged afterwards: the
    # same FP32 values either way
    p1 = ctx.radon_grid(vol, 8, 4, 9, sampler=O.TRILINEAR)
    p2 = ctx.radon_grid(vol, 8, 4, 9, sampler=O.TRILINEAR)
    assert np.array_equal(p1, p2)
