"""Parity of the CUDA library against the FP64 oracle (small sizes).

Tolerances: the trilinear paths compute in FP32 with compensated sums and must
stay within relative L2 error 1e-5 of the FP64 oracle; the nearest sampler
uses the reference's cell choice exactly (guard band re-evaluated in FP64), so
its only error is FP32 storage of the volume values.
"""
import numpy as np
import pytest

import oracle as O
from conftest import wrt, rel_l2, rel_max

from wrt_b200.phantom import ellipsoid_phantom, layer_frames

pytestmark = pytest.mark.gpu

TOL_L2 = 1e-5


@pytest.fixture(scope="module")
def vol24():
    return ellipsoid_phantom(24, 8, 1000)


@pytest.fixture(scope="module")
def volrand():
    return np.random.default_rng(7).standard_normal((20, 20, 20))


def test_gauss_legendre_bit_identical(ctx):
    for n in (1, 2, 3, 7, 32, 64, 96, 128):
        x, w = ctx.gauss_legendre(n)
        xo, wo = O.gauss_legendre(n)
        assert np.array_equal(x, xo) and np.array_equal(w, wo), n


def test_radon_grid_init_matches_oracle(ctx):
    phi, th, w, s = ctx.radon_grid_init(64, 32, 129)
    po, to, wo, so = O.radon_grid(64, 32, 129)
    for a, b in ((phi, po), (th, to), (w, wo), (s, so)):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("sampler", [O.NEAREST, O.TRILINEAR])
def test_radon_grid_phantom(ctx, vol24, sampler):
    got = ctx.radon_grid(vol24, 16, 8, 12, sampler=sampler)
    ref = O.radon_forward(vol24, 16, 8, 12, sampler=sampler)
    assert rel_l2(got, ref) < TOL_L2
    assert rel_max(got, ref) < 1e-4


@pytest.mark.parametrize("sampler", [O.NEAREST, O.TRILINEAR])
def test_radon_grid_random_volume(ctx, volrand, sampler):
    """Non-zero faces: exercises the cube cut-off and the guard band."""
    got = ctx.radon_grid(volrand, 8, 6, 9, sampler=sampler)
    ref = O.radon_forward(volrand, 8, 6, 9, sampler=sampler)
    assert rel_l2(got, ref) < TOL_L2


def test_radon_grid_half_extent(ctx, vol24):
    got = ctx.radon_grid(vol24, 12, 6, 10, sampler=O.TRILINEAR, half_extent=24)
    ref = O.radon_forward(vol24, 12, 6, 10, sampler=O.TRILINEAR, half_extent=24)
    assert rel_l2(got, ref) < TOL_L2


def test_ray_grid_reference_frame(ctx, vol24, volrand):
    for v in (vol24, volrand):
        n = v.shape[0]
        got = ctx.ray_grid(v, n, 15, 16)
        ref = O.ray_forward(v, n, 15, 16)
        assert rel_l2(got, ref) < TOL_L2


def test_ray_grid_rotated_frames(ctx, vol24):
    for F in layer_frames(3, 5)[1:]:
        got = ctx.ray_grid(vol24, 24, 15, 16, frame=F)
        ref = O.ray_forward(vol24, 24, 15, 16, frame=F)
        assert rel_l2(got, ref) < TOL_L2


def test_reduction_coupled(ctx, vol24):
    rays = O.ray_forward(vol24, 24, 20, 16)
    got = ctx.radon_reduction(rays, 20, 6)
    ref = O.reduction_forward(rays, 20, 6)
    assert rel_l2(got, ref) < TOL_L2


def test_reduction_decoupled(ctx, vol24):
    rays = O.ray_forward(vol24, 24, 16, 16)
    got = ctx.radon_reduction(rays, 31, 8)
    ref = O.reduction_forward(rays, 31, 8)
    assert rel_l2(got, ref) < TOL_L2


def test_adjoint(ctx):
    R = np.random.default_rng(3).standard_normal((17, 12, 6))
    got = ctx.radon3d_adjoint(R, 10)
    ref = O.adjoint_forward(R, 10)
    assert rel_l2(got, ref) < TOL_L2


@pytest.mark.parametrize("sampler", [O.NEAREST, O.TRILINEAR])
def test_transpose_inner_product(ctx, vol24, sampler):
    g = np.random.default_rng(11).standard_normal((10, 12, 6))
    Rf = ctx.radon_grid(vol24, 12, 6, 10, sampler=sampler)
    RTg = ctx.radon_transpose(g, 24, sampler=sampler)
    lhs, rhs = float((Rf * g).sum()), float((vol24 * RTg).sum())
    assert abs(lhs - rhs) <= 1e-6 * max(abs(lhs), abs(rhs))
    ref = O.radon_transpose(g, 24, sampler=sampler)
    assert rel_l2(RTg, ref) < TOL_L2


# ----------------------------------------------------------- staged kernel
STAGED_CASES = [
    (24, (16, 8, 12), 0),     # one tile, the reference's lattice [-2n, 2n)^2
    (24, (12, 6, 10), 24),    # lattice [-n, n)^2 (the benchmark's definition)
    (33, (9, 7, 13), 0),      # odd n: z = 0 is a node (guard-band rows)
    (64, (16, 8, 20), 64),
    (200, (6, 4, 7), 200),    # several y-tiles
]


@pytest.mark.parametrize("n,grid,L", STAGED_CASES)
def test_staged_matches_oracle(ctx, n, grid, L):
    vol = ellipsoid_phantom(n, 8, 2000 + n)
    got = ctx.radon_grid(vol, *grid, sampler=O.TRILINEAR, half_extent=L, kernel=wrt.KERNEL_STAGED)
    ref = O.radon_forward(vol, *grid, sampler=O.TRILINEAR, half_extent=L)
    assert rel_l2(got, ref) < TOL_L2
    assert rel_max(got, ref) < 1e-4


def test_staged_random_volume_nonzero_faces(ctx, volrand):
    got = ctx.radon_grid(volrand, 8, 6, 9, sampler=O.TRILINEAR, kernel=wrt.KERNEL_STAGED)
    ref = O.radon_forward(volrand, 8, 6, 9, sampler=O.TRILINEAR)
    assert rel_l2(got, ref) < TOL_L2


def test_staged_is_bitwise_deterministic(ctx, vol24):
    a = ctx.radon_grid(vol24, 16, 8, 12, sampler=O.TRILINEAR, kernel=wrt.KERNEL_STAGED)
    b = ctx.radon_grid(vol24, 16, 8, 12, sampler=O.TRILINEAR, kernel=wrt.KERNEL_STAGED)
    assert np.array_equal(a, b)


def test_staged_agrees_with_plain(ctx):
    vol = ellipsoid_phantom(48, 10, 4242)
    a = ctx.radon_grid(vol, 24, 12, 33, sampler=O.TRILINEAR, half_extent=48, kernel=wrt.KERNEL_STAGED)
    b = ctx.radon_grid(vol, 24, 12, 33, sampler=O.TRILINEAR, half_extent=48, kernel=wrt.KERNEL_PLAIN)
    assert rel_l2(a, b) < 2e-6


# The reference's default sampler (zero_interp) through the staged kernel: one
# FP32 value per cell of a z-layer in shared memory, the reference's lattice
# [-2n, 2n)^2 unless stated.
NEAREST_CASES = [
    (24, (16, 8, 12), 0),
    (33, (9, 7, 13), 0),      # odd n: z = 0 is a cell boundary (guard-band rows)
    (64, (16, 8, 20), 64),
    (224, (4, 3, 5), 0),      # two y-tiles
]


@pytest.mark.parametrize("n,grid,L", NEAREST_CASES)
def test_staged_nearest_matches_oracle_and_plain(ctx, n, grid, L):
    vol = ellipsoid_phantom(n, 8, 2100 + n)
    got = ctx.radon_grid(vol, *grid, sampler=O.NEAREST, half_extent=L, kernel=wrt.KERNEL_STAGED)
    ref = O.radon_forward(vol, *grid, sampler=O.NEAREST, half_extent=L)
    assert rel_l2(got, ref) < TOL_L2
    assert rel_max(got, ref) < 1e-4
    # the plain kernel takes the same FP32 samples (or the same FP64 ones in the
    # guard band) and sums them in other groups: FP32 rounding of the partial sums
    plain = ctx.radon_grid(vol, *grid, sampler=O.NEAREST, half_extent=L, kernel=wrt.KERNEL_PLAIN)
    assert rel_l2(got, plain) < 1e-6


@pytest.mark.parametrize("sampler,L", [(O.NEAREST, 72), (O.TRILINEAR, 96)])
def test_staged_lattice_beyond_the_reference_extent(ctx, vol24, sampler, L):
    """Lattices wider than the reference's [-2n, 2n)^2 (up to 8n is accepted):
    the rows leave the cube further out, the row indices still fit the tables."""
    got = ctx.radon_grid(vol24, 8, 4, 6, sampler=sampler, half_extent=L,
                         kernel=wrt.KERNEL_STAGED)
    ref = O.radon_forward(vol24, 8, 4, 6, sampler=sampler, half_extent=L)
    assert rel_l2(got, ref) < TOL_L2


def test_ray_tiles_at_ragged_grid_sizes(ctx, vol24):
    """Shift and angle counts that are not multiples of a warp's tile (16 x 2
    in the reference frame, 2 x 16 in rotated ones)."""
    F = layer_frames(2, 77)[1]
    for nshift, nphi in ((15, 17), (33, 3), (2, 1)):
        for fr in (None, F):
            got = ctx.ray_grid(vol24, 24, nshift, nphi, frame=fr)
            ref = O.ray_forward(vol24, 24, nshift, nphi, frame=fr)
            assert rel_l2(got, ref) < TOL_L2, (nshift, nphi, fr is None)


def test_staged_nearest_random_volume_nonzero_faces(ctx, volrand):
    got = ctx.radon_grid(volrand, 8, 6, 9, sampler=O.NEAREST, kernel=wrt.KERNEL_STAGED)
    ref = O.radon_forward(volrand, 8, 6, 9, sampler=O.NEAREST)
    assert rel_l2(got, ref) < TOL_L2


def test_staged_nearest_is_the_default_and_deterministic(ctx, vol24):
    a = ctx.radon_grid(vol24, 16, 8, 12, sampler=O.NEAREST)
    b = ctx.radon_grid(vol24, 16, 8, 12, sampler=O.NEAREST, kernel=wrt.KERNEL_STAGED)
    assert np.array_equal(a, b)


def test_every_staged_tile_configuration_matches_oracle(ctx):
    vol = ellipsoid_phantom(40, 8, 515)
    ref = O.radon_forward(vol, 10, 6, 15, sampler=O.TRILINEAR, half_extent=40)
    try:
        for k, shape in enumerate(wrt.plane_kernel_configs()):
            wrt.set_plane_kernel_config(ctx, k)
            got = ctx.radon_grid(vol, 10, 6, 15, sampler=O.TRILINEAR, half_extent=40,
                                 kernel=wrt.KERNEL_STAGED)
            assert rel_l2(got, ref) < TOL_L2, shape
    finally:
        wrt.set_plane_kernel_config(ctx, -1)


def test_autotuner_picks_a_configuration(ctx):
    vol = wrt.Volume(ctx, 32)
    vol.upload(ellipsoid_phantom(32, 6, 9))
    grid = wrt.Grid(ctx, 12, 6, 16)
    out = wrt.DeviceBuffer(ctx, grid.nplanes * 8)
    best, ms = wrt.tune_plane_kernel(ctx, vol, grid, out.ptr, half_extent=32)
    assert 0 <= best < len(wrt.plane_kernel_configs()) and ms > 0
    wrt.set_plane_kernel_config(ctx, -1)
    out.close(); grid.close(); vol.close()


