"""wrt_radon3d_adjoint_static: the backprojection for callers that cannot
allocate device memory (their device memory belongs to their own allocator,
or allocation is forbidden on their latency-critical path).  It must give the
same volume as the allocating wrt_radon3d_adjoint, call after call, without
the context acquiring any device memory.  Collected last on purpose: it is a
separate entry point with its own working memory inside the library."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2, wrt

pytestmark = pytest.mark.gpu

TOL_L2 = 1e-5


def static_adjoint():
    f = wrt.lib().wrt_radon3d_adjoint_static
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
    f.restype = C.c_int
    return f


def test_static_adjoint_matches_allocating_adjoint_on_two_calls():
    nshift, nphi, ntheta, n = 33, 24, 12, 20
    rng = np.random.default_rng(123)
    with wrt.Context(0) as ctx:
        din = wrt.DeviceBuffer(ctx, nshift * nphi * ntheta * 8)
        dout = wrt.DeviceBuffer(ctx, n ** 3 * 8)
        held = ctx.bytes_in_use
        for call in range(2):
            radon = rng.standard_normal((nshift, nphi, ntheta))
            din.upload(radon)
            ctx.check(static_adjoint()(ctx.handle, din.ptr, nphi, ntheta, nshift, n, dout.ptr),
                      f"static adjoint, call {call}")
            got = dout.download(np.empty((n, n, n)))
            assert ctx.bytes_in_use == held  # the call acquired no device memory
            ref = ctx.radon3d_adjoint(radon, n)
            assert rel_l2(got, ref) < TOL_L2, call
        din.close()
        dout.close()


def test_static_adjoint_rejects_sizes_beyond_its_memory():
    with wrt.Context(0) as ctx:
        dummy = wrt.DeviceBuffer(ctx, 1024)
        # 128 x 128 directions exceeds the 16384-direction limit
        st = static_adjoint()(ctx.handle, dummy.ptr, 128, 129, 16, 8, dummy.ptr)
        assert st == 1
        msg = wrt.lib().wrt_ctx_last_error(ctx.handle).decode()
        assert "exceeds the static working memory" in msg
        dummy.close()
