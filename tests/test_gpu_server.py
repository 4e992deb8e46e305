"""The serving loop (wrt_server): continuous batching of forward and adjoint
requests under an HBM budget.

Checked here: every served result equals the library's single-request result
(bitwise) and the FP64 oracle (FP32 tolerance); a request gives the same
result alone and in a mix of concurrent requests; admission waits for memory
instead of failing when the budget is tight; requests that can never fit are
refused; requests arriving while others run are batched and overlap them."""
import threading

import numpy as np
import pytest

import oracle as O
from conftest import rel_l2, wrt
from wrt_b200.phantom import ellipsoid_phantom

pytestmark = pytest.mark.gpu

TOL_L2 = 1e-5
WAIT_MS = 120_000  # a request that takes longer fails the test instead of hanging it


def _forward_direct(ctx, vol, nphi, ntheta, nshift, L):
    v = wrt.Volume(ctx, vol.shape[0])
    v.upload(vol.astype(np.float32))
    g = wrt.Grid(ctx, nphi, ntheta, nshift)
    out = wrt.DeviceBuffer(ctx, g.nplanes * 8)
    wrt.radon_forward_device(ctx, v, g, out.ptr, sampler=wrt.TRILINEAR, half_extent=L,
                             kernel=wrt.KERNEL_STAGED)
    res = out.download(np.empty((nshift, nphi, ntheta)))
    out.close(); g.close(); v.close()
    return res


def _mixed_requests(rng, count):
    reqs = []
    for k in range(count):
        n = int(rng.choice([12, 16, 20, 24, 32]))
        nth = int(rng.integers(3, 8))
        if rng.random() < 0.75:
            vol = ellipsoid_phantom(n, 4, 5000 + k).astype(np.float32)
            reqs.append(("fwd", vol, 2 * nth, nth, int(rng.integers(5, 14)), int(rng.choice([0, n]))))
        else:
            radon = rng.standard_normal((int(rng.integers(5, 14)), 2 * nth, nth))
            reqs.append(("adj", radon, n))
    return reqs


def _submit(srv, r):
    if r[0] == "fwd":
        _, vol, nphi, nth, ns, L = r
        out = np.zeros((ns, nphi, nth))
        return srv.submit_forward(vol, nphi, nth, ns, out, half_extent=L), out
    _, radon, n = r
    out = np.zeros((n, n, n))
    return srv.submit_adjoint(radon, n, out), out


def test_served_results_equal_direct_and_oracle(ctx):
    vol = ellipsoid_phantom(24, 6, 321).astype(np.float32)
    radon = np.random.default_rng(5).standard_normal((11, 12, 6))
    with wrt.Server(0, budget_bytes=1 << 30) as srv:
        f_out = np.zeros((10, 12, 6))
        a_out = np.zeros((20, 20, 20))
        ids = [srv.submit_forward(vol, 12, 6, 10, f_out, half_extent=24),
               srv.submit_adjoint(radon, 20, a_out)]
        for i in ids:
            assert srv.wait(i, WAIT_MS).status == 0
    assert np.array_equal(f_out, _forward_direct(ctx, vol, 12, 6, 10, 24))
    ref = O.radon_forward(vol.astype(np.float64), 12, 6, 10, sampler=O.TRILINEAR, half_extent=24)
    assert rel_l2(f_out, ref) < TOL_L2
    assert np.array_equal(a_out, ctx.radon3d_adjoint(radon, 20))
    assert rel_l2(a_out, O.adjoint_forward(radon, 20)) < TOL_L2


def test_same_result_alone_and_in_the_mix():
    rng = np.random.default_rng(2024)
    mix = _mixed_requests(rng, 40)
    probe_f = ("fwd", ellipsoid_phantom(28, 7, 99).astype(np.float32), 10, 5, 9, 28)
    probe_a = ("adj", rng.standard_normal((9, 10, 5)), 18)
    with wrt.Server(0, budget_bytes=1 << 30, max_batch=16, max_inflight=2) as srv:
        alone = []
        for r in (probe_f, probe_a):
            rid, out = _submit(srv, r)
            assert srv.wait(rid, WAIT_MS).status == 0
            alone.append(out)
        # the same two requests among 40 others, submitted from 4 threads
        results, lock = {}, threading.Lock()

        def worker(items):
            for key, r in items:
                rid, out = _submit(srv, r)
                with lock:
                    results[key] = (rid, out)

        items = [(("mix", k), r) for k, r in enumerate(mix)]
        items.insert(13, (("probe", 0), probe_f))
        items.insert(29, (("probe", 1), probe_a))
        threads = [threading.Thread(target=worker, args=(items[k::4],)) for k in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        infos = {key: srv.wait(rid, WAIT_MS) for key, (rid, _) in results.items()}
        assert all(i.status == 0 for i in infos.values())
        for k in range(2):
            assert np.array_equal(results[("probe", k)][1], alone[k])
        # batching happened: fewer launches than requests
        st = srv.stats()
        assert st.completed == 44 and st.failed == 0
        assert st.launches < 44
        assert max(i.batch_size for i in infos.values()) > 1
    # spot-check a few mixed results against the oracle
    for k in (0, 1, 2, 3):
        r = mix[k]
        out = results[("mix", k)][1]
        if r[0] == "fwd":
            _, vol, nphi, nth, ns, L = r
            ref = O.radon_forward(vol.astype(np.float64), nphi, nth, ns, sampler=O.TRILINEAR,
                                  half_extent=L or None)
        else:
            _, radon, n = r
            ref = O.adjoint_forward(radon, n)
        assert rel_l2(out, ref) < TOL_L2


def test_tight_budget_admits_as_memory_frees():
    # each 32^3 forward request with a 16x8x16 grid needs ~0.4 MB of state:
    # a 1.5 MB budget holds only three at a time, all must still complete
    vols = [ellipsoid_phantom(32, 5, 7000 + k).astype(np.float32) for k in range(12)]
    with wrt.Server(0, budget_bytes=3 << 19, max_batch=8, max_inflight=2) as srv:
        outs, ids = [], []
        for v in vols:
            out = np.zeros((16, 16, 8))
            ids.append(srv.submit_forward(v, 16, 8, 16, out, half_extent=32))
            outs.append(out)
        infos = [srv.wait(i, WAIT_MS) for i in ids]
        st = srv.stats()
    assert all(i.status == 0 for i in infos)
    assert st.bytes_peak <= 3 << 19
    assert st.launches >= 3  # could not all be admitted at once
    ref = O.radon_forward(vols[5].astype(np.float64), 16, 8, 16, sampler=O.TRILINEAR, half_extent=32)
    assert rel_l2(outs[5], ref) < TOL_L2


def test_request_larger_than_budget_is_refused():
    with wrt.Server(0, budget_bytes=1 << 20) as srv:
        vol = np.zeros((64, 64, 64), np.float32)
        with pytest.raises(wrt.WrtError) as e:
            srv.submit_forward(vol, 8, 4, 8, np.zeros((8, 8, 4)))
        assert e.value.status == 3  # WRT_ERR_BUDGET


def test_requests_arriving_during_a_launch_overlap_it():
    big = ellipsoid_phantom(128, 8, 1).astype(np.float32)
    small = [ellipsoid_phantom(24, 4, 300 + k).astype(np.float32) for k in range(6)]
    outs = [np.zeros((8, 8, 4)) for _ in small]
    with wrt.Server(0, budget_bytes=1 << 30, max_batch=8, max_inflight=2) as srv:
        out0 = np.zeros((128, 64, 32))
        first = srv.submit_forward(big, 64, 32, 128, out0, half_extent=128)
        # submitted microseconds later, while the first launch runs
        later = [srv.submit_forward(v, 8, 4, 8, o, half_extent=24) for v, o in zip(small, outs)]
        i0 = srv.wait(first, WAIT_MS)
        infos = [srv.wait(i, WAIT_MS) for i in later]
    assert i0.status == 0 and all(i.status == 0 for i in infos)
    # the later requests were admitted and launched before the first one finished
    assert min(i.start_ms for i in infos) < i0.done_ms
    assert max(i.batch_size for i in infos) > 1


def test_served_ray_and_reduction_equal_direct_alone_and_in_the_mix(ctx):
    """The ray transform and the ray-to-Radon reduction as served requests
    (WRT_OP_RAY, WRT_OP_REDUCE): bitwise the direct entry points' results, in
    a batch of their own and among concurrent forward / adjoint requests; and
    the ray_grid -> radon_reduction chain within the FP32 tolerance of the
    oracle."""
    n, nsr, nphi, nshift, ntheta = 24, 20, 12, 16, 6
    vol = ellipsoid_phantom(n, 6, 808).astype(np.float32)
    frame = np.array([[0.36, 0.48, -0.8], [-0.8, 0.6, 0.0], [0.48, 0.64, 0.6]])
    rays_direct = ctx.ray_grid(vol.astype(np.float64), n, nsr, nphi)
    rays_frame = ctx.ray_grid(vol.astype(np.float64), n, nsr, nphi, frame=frame)
    radon_direct = ctx.radon_reduction(rays_direct, nshift, ntheta)
    assert rel_l2(rays_direct, O.ray_forward(vol.astype(np.float64), n, nsr, nphi)) < TOL_L2
    assert rel_l2(radon_direct, O.reduction_forward(rays_direct, nshift, ntheta)) < TOL_L2
    rng = np.random.default_rng(77)
    with wrt.Server(0, budget_bytes=1 << 30, max_batch=16, max_inflight=2) as srv:
        def three():
            r0, r1, r2 = (np.zeros((n, nsr, nphi)), np.zeros((n, nsr, nphi)),
                          np.zeros((nshift, nphi, ntheta)))
            ids = [srv.submit_ray(vol, n, nsr, nphi, r0),
                   srv.submit_ray(vol, n, nsr, nphi, r1, frame=frame),
                   srv.submit_reduce(rays_direct, nshift, ntheta, r2)]
            return ids, (r0, r1, r2)
        ids, outs = three()
        for i in ids:
            assert srv.wait(i, WAIT_MS).status == 0
        for got, ref in zip(outs, (rays_direct, rays_frame, radon_direct)):
            assert np.array_equal(got, ref)
        # again, among 30 forward / adjoint requests submitted at the same time
        mixed = [_submit(srv, r) for r in _mixed_requests(rng, 15)]
        ids, outs = three()
        mixed += [_submit(srv, r) for r in _mixed_requests(rng, 15)]
        infos = [srv.wait(i, WAIT_MS) for i in ids] + [srv.wait(i, WAIT_MS) for i, _ in mixed]
        assert all(i.status == 0 for i in infos)
        assert max(i.batch_size for i in infos) > 1
        for got, ref in zip(outs, (rays_direct, rays_frame, radon_direct)):
            assert np.array_equal(got, ref)
