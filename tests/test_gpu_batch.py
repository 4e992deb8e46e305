"""Batched forward transforms (wrt_radon_forward_batch): many volumes of
uneven edge lengths, each with its own sphere grid and shift count, in one
launch of the persistent staged kernel through a captured CUDA graph.

Every request's result must be bitwise identical to the same request run
alone (wrt_radon_forward_device), and within the FP32 tolerance of the FP64
oracle (radon_grid/src/integral.c:26-58 with the trilinear sampler)."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2, rel_max, wrt
from wrt_b200.phantom import ellipsoid_phantom

pytestmark = pytest.mark.gpu

TOL_L2 = 1e-5

# (n, nphi, ntheta, nshift, half_extent): uneven sizes and grids
BATCH = [
    (12, 8, 4, 9, 0),
    (17, 10, 5, 12, 17),
    (24, 12, 6, 10, 24),
    (33, 6, 3, 16, 33),
    (48, 8, 4, 7, 48),
    (20, 16, 8, 5, 0),
]


def _setup(ctx, spec, seed0):
    reqs, keep = [], []
    for k, (n, nphi, ntheta, nshift, L) in enumerate(spec):
        vol = ellipsoid_phantom(n, 4 + k, seed0 + k)
        v = wrt.Volume(ctx, n)
        v.upload(vol)
        g = wrt.Grid(ctx, nphi, ntheta, nshift)
        out = wrt.DeviceBuffer(ctx, g.nplanes * 8)
        reqs.append((v, g, out.ptr, L))
        keep.append((vol, v, g, out, (nshift, nphi, ntheta), L))
    return reqs, keep


def _download(out, shape):
    return out.download(np.empty(shape))


def test_batch_matches_alone_bitwise_and_oracle(ctx):
    reqs, keep = _setup(ctx, BATCH, 700)
    wrt.radon_forward_batch(ctx, reqs)
    ctx.synchronize()
    batched = [_download(out, shape) for (_, _, _, out, shape, _) in keep]
    for (vol, v, g, out, shape, L), got in zip(keep, batched):
        wrt.radon_forward_device(ctx, v, g, out.ptr, sampler=wrt.TRILINEAR, half_extent=L,
                                 kernel=wrt.KERNEL_STAGED)
        alone = _download(out, shape)
        assert np.array_equal(got, alone)
        ref = O.radon_forward(vol, shape[1], shape[2], shape[0], sampler=O.TRILINEAR,
                              half_extent=L or None)
        assert rel_l2(got, ref) < TOL_L2
        assert rel_max(got, ref) < 1e-4


def test_graph_replay_with_new_compositions(ctx):
    reqs, keep = _setup(ctx, BATCH, 900)
    # three launches of the same captured graph with different request sets
    for subset in ([0, 1, 2, 3, 4, 5], [5, 3], [2]):
        wrt.radon_forward_batch(ctx, [reqs[i] for i in subset])
        ctx.synchronize()
        for i in subset:
            vol, v, g, out, shape, L = keep[i]
            got = _download(out, shape)
            ref = O.radon_forward(vol, shape[1], shape[2], shape[0], sampler=O.TRILINEAR,
                                  half_extent=L or None)
            assert rel_l2(got, ref) < TOL_L2, (subset, i)


def test_batch_of_one_equals_single_request(ctx):
    reqs, keep = _setup(ctx, BATCH[2:3], 77)
    vol, v, g, out, shape, L = keep[0]
    wrt.radon_forward_batch(ctx, reqs)
    ctx.synchronize()
    a = _download(out, shape)
    wrt.radon_forward_device(ctx, v, g, out.ptr, sampler=wrt.TRILINEAR, half_extent=L,
                             kernel=wrt.KERNEL_STAGED)
    assert np.array_equal(a, _download(out, shape))


def test_batch_rejects_bad_requests(ctx):
    v = wrt.Volume(ctx, 3)  # too small for the staged kernel
    v.upload(np.zeros((3, 3, 3)))
    g = wrt.Grid(ctx, 4, 2, 3)
    out = wrt.DeviceBuffer(ctx, g.nplanes * 8)
    with pytest.raises(wrt.WrtError):
        wrt.radon_forward_batch(ctx, [(v, g, out.ptr, 0)])
    with pytest.raises(wrt.WrtError):
        wrt.radon_forward_batch(ctx, [(v, g, 0, 0)])
    wrt.radon_forward_batch(ctx, [])  # empty batch: nothing to do
