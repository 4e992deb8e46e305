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


# ----------------------------------------------------------- BF16 storage
def test_bf16_volume_matches_oracle_on_rounded_values(ctx):
    n, grid, L = 40, (12, 6, 14), 40
    vol = ellipsoid_phantom(n, 8, 4040)
    v16 = wrt.Volume(ctx, n, storage=wrt.STORAGE_BF16)
    v16.upload(vol)
    v32 = wrt.Volume(ctx, n)
    v32.upload(vol)
    g = wrt.Grid(ctx, *grid)
    out = wrt.DeviceBuffer(ctx, g.nplanes * 8)
    shape = (grid[2], grid[0], grid[1])
    wrt.radon_forward_device(ctx, v16, g, out.ptr, sampler=wrt.TRILINEAR, half_extent=L)
    got16 = out.download(np.empty(shape))
    # exact parity with the FP64 oracle on the values the volume holds
    ref16 = O.radon_forward(wrt.round_bf16(vol), *grid, sampler=O.TRILINEAR, half_extent=L)
    assert rel_l2(got16, ref16) < TOL_L2
    assert rel_max(got16, ref16) < 1e-4
    # against the unrounded volume the error is the storage rounding (bf16: 8 bits)
    ref = O.radon_forward(vol, *grid, sampler=O.TRILINEAR, half_extent=L)
    assert rel_l2(got16, ref) < 4e-3
    # half the device memory of the FP32 layouts, once the layer pairs exist
    wrt.radon_forward_device(ctx, v32, g, out.ptr, sampler=wrt.TRILINEAR, half_extent=L)
    assert v16.nbytes * 2 <= v32.nbytes + 64
    # BF16 volumes are sampled by the staged kernel only
    with pytest.raises(wrt.WrtError):
        wrt.radon_forward_device(ctx, v16, g, out.ptr, sampler=wrt.NEAREST)


def test_batch_mixes_fp32_and_bf16_volumes(ctx):
    reqs, outs = [], []
    for k, (n, storage) in enumerate([(24, wrt.STORAGE_F32), (30, wrt.STORAGE_BF16),
                                       (36, wrt.STORAGE_BF16)]):
        vol = ellipsoid_phantom(n, 5, 60 + k)
        v = wrt.Volume(ctx, n, storage=storage)
        v.upload(vol)
        g = wrt.Grid(ctx, 8, 4, 9)
        out = wrt.DeviceBuffer(ctx, g.nplanes * 8)
        reqs.append((v, g, out.ptr, n))
        outs.append((vol, storage, out))
    wrt.radon_forward_batch(ctx, reqs)
    ctx.synchronize()
    for vol, storage, out in outs:
        got = out.download(np.empty((9, 8, 4)))
        held = wrt.round_bf16(vol) if storage == wrt.STORAGE_BF16 else vol.astype(np.float32)
        ref = O.radon_forward(held.astype(np.float64), 8, 4, 9, sampler=O.TRILINEAR,
                              half_extent=vol.shape[0])
        assert rel_l2(got, ref) < TOL_L2
