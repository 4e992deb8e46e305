"""wrt_radon3d_adjoint_static: the backprojection for callers that cannot
allocate device memory (their device memory belongs to their own allocator,
or allocation is forbidden on their latency-critical path).  It must give the
same volume as the allocating wrt_radon3d_adjoint -- bit for bit, since both
build their tables with the same host code -- call after call, without the
context acquiring any device memory, and agree with the FP64 oracle within the
tolerance of every FP32 path.  Sizes exactly at each limit of its fixed
working memory run; sizes one past a limit are refused.  Collected last on
purpose: it is a separate entry point with its own working memory inside the
library."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from conftest import rel_l2, wrt

pytestmark = pytest.mark.gpu

TOL_L2 = 1e-5


def static_adjoint():
    f = wrt.lib().wrt_radon3d_adjoint_static
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
    f.restype = C.c_int
    return f


def _run(ctx, radon, n, din, dout):
    nshift, nphi, ntheta = radon.shape
    din.upload(radon)
    ctx.check(static_adjoint()(ctx.handle, din.ptr, nphi, ntheta, nshift, n, dout.ptr),
              "static adjoint")
    return dout.download(np.empty((n, n, n)))


def test_static_adjoint_matches_allocating_adjoint_on_two_calls():
    nshift, nphi, ntheta, n = 33, 24, 12, 20
    rng = np.random.default_rng(123)
    with wrt.Context(0) as ctx:
        din = wrt.DeviceBuffer(ctx, nshift * nphi * ntheta * 8)
        dout = wrt.DeviceBuffer(ctx, n ** 3 * 8)
        for call in range(2):
            radon = rng.standard_normal((nshift, nphi, ntheta))
            held = ctx.bytes_in_use
            got = _run(ctx, radon, n, din, dout)
            assert ctx.bytes_in_use == held  # the call acquired no device memory
            ref = ctx.radon3d_adjoint(radon, n)
            assert np.array_equal(got, ref), (call, rel_l2(got, ref))
            exact = O.adjoint_forward(radon, n)
            assert rel_l2(got, exact) < TOL_L2, call
        din.close()
        dout.close()


@pytest.mark.parametrize("nphi,ntheta,nshift", [(128, 128, 16), (8, 16, 2048), (16, 1024, 16)])
def test_static_adjoint_at_the_limits_of_its_memory(nphi, ntheta, nshift):
    n = 12
    rng = np.random.default_rng(nphi + ntheta + nshift)
    radon = rng.standard_normal((nshift, nphi, ntheta))
    with wrt.Context(0) as ctx:
        din = wrt.DeviceBuffer(ctx, radon.nbytes)
        dout = wrt.DeviceBuffer(ctx, n ** 3 * 8)
        got = _run(ctx, radon, n, din, dout)
        ref = ctx.radon3d_adjoint(radon, n)
        assert np.array_equal(got, ref), rel_l2(got, ref)
        din.close()
        dout.close()


@pytest.mark.parametrize("nphi,ntheta,nshift,what", [
    (128, 129, 16, "directions"),      # 16512 > 16384 directions
    (1, 1025, 3, "latitudes"),         # ntheta > 1024
    (1, 1, 2049, "shifts"),            # nshift > 2048
    (128, 128, 17, "spline samples"),  # 278528 > 262144 samples
])
def test_static_adjoint_rejects_sizes_beyond_its_memory(nphi, ntheta, nshift, what):
    with wrt.Context(0) as ctx:
        dummy = wrt.DeviceBuffer(ctx, 1024)
        st = static_adjoint()(ctx.handle, dummy.ptr, nphi, ntheta, nshift, 8, dummy.ptr)
        assert st == 1, what
        msg = wrt.lib().wrt_ctx_last_error(ctx.handle).decode()
        assert "exceeds the static working memory" in msg, what
        dummy.close()
