"""Python binding of libwrt (the B200 grid-sampled Radon / ray transform
library) through its C ABI (include/wrt.h).

The binding mirrors the reference's four programs, one call each:

=====================  ===========================================  ==========
call                   reference program (loop nest)                 output
=====================  ===========================================  ==========
``radon_grid``         radon_grid/src/radon_grid.c:229-264           [s][phi][theta]
``ray_grid``           ray_grid/src/ray_grid.c:225-262               [z][s][phi]
``radon_reduction``    radon_reduction/reduction.c:195-235           [s][phi][theta]
``radon3d_adjoint``    backprojection/C/src/radon3d_ajoint.c:221-260 [z][x][y]
=====================  ===========================================  ==========

Volumes are ``v[ix][iy][iz]`` arrays, as the reference's text files order
them.  There is no CPU fallback: every call runs the CUDA library, and a
missing library or device raises ``WrtError``.
"""
from __future__ import annotations

import atexit
import ctypes as C
import weakref
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "lib" / "libwrt.so"

NEAREST, TRILINEAR = 0, 1
STORAGE_F32, STORAGE_BF16 = 0, 1
KERNEL_AUTO, KERNEL_PLAIN, KERNEL_STAGED = 0, 1, 2

STATUS = {
    0: "ok", 1: "invalid argument", 2: "out of memory", 3: "over budget", 4: "CUDA error",
    5: "no device", 6: "timeout", 7: "queue full", 8: "not found", 9: "cancelled", 10: "internal",
}


class WrtError(RuntimeError):
    def __init__(self, status: int, message: str = ""):
        self.status = status
        super().__init__(f"wrt status {status} ({STATUS.get(status, '?')}): {message}")


class PlaneOpts(C.Structure):
    _fields_ = [("sampler", C.c_int), ("half_extent", C.c_int), ("kernel", C.c_int),
                ("reserved", C.c_int * 5)]


class ForwardReq(C.Structure):
    _fields_ = [("volume", C.c_void_p), ("grid", C.c_void_p), ("half_extent", C.c_int),
                ("reserved", C.c_int), ("dev_out", C.c_void_p)]


OP_FORWARD, OP_ADJOINT, OP_RAY, OP_REDUCE = 0, 1, 2, 3
FUNCTION_EXP_BUMP, FUNCTION_SINE_BUMPS = 0, 1


class Function(C.Structure):
    """An analytic test function (wrt_function): FUNCTION_EXP_BUMP with
    p = (cx, cy, cz, R2, eps), or FUNCTION_SINE_BUMPS with p = (cx, cy, cz,
    amplitude, rin, rout) per ball."""
    _fields_ = [("kind", C.c_int), ("count", C.c_int), ("p", C.c_double * 48)]


def exp_bump(center=(0.2, 0.0, 0.0), R2=0.5, eps=1e-2) -> Function:
    """The reference's exponential_bump.c (its constants by default)."""
    f = Function()
    f.kind, f.count = FUNCTION_EXP_BUMP, 1
    for k, v in enumerate([*center, R2, eps]):
        f.p[k] = v
    return f


def sine_bumps(balls=((0.0, 0.2, 0.0, 1.0, 0.4, 0.6), (-0.5, 0.0, 0.0, 0.6, 0.3, 0.45),
                      (0.0, 0.2, 0.5, 0.3, 0.4, 0.6))) -> Function:
    """The reference's sinusoidal_bump.c (its three balls by default):
    each ball (cx, cy, cz, amplitude, rin, rout)."""
    f = Function()
    f.kind, f.count = FUNCTION_SINE_BUMPS, len(balls)
    for b, ball in enumerate(balls):
        for k, v in enumerate(ball):
            f.p[6 * b + k] = v
    return f


class Request(C.Structure):
    _fields_ = [("op", C.c_int), ("ngrid", C.c_int), ("nphi", C.c_int), ("ntheta", C.c_int),
                ("nshift", C.c_int), ("half_extent", C.c_int), ("volume", C.c_void_p),
                ("radon", C.c_void_p), ("out", C.c_void_p), ("tag", C.c_uint64),
                ("nslices", C.c_int), ("nshift_ray", C.c_int), ("rays", C.c_void_p),
                ("frame", C.c_void_p)]


class RequestInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("batch_size", C.c_int), ("tag", C.c_uint64),
                ("submit_ms", C.c_double), ("start_ms", C.c_double), ("done_ms", C.c_double)]


class ServerOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("max_batch", C.c_int), ("max_inflight", C.c_int),
                ("queue_capacity", C.c_int), ("hbm_budget", C.c_size_t),
                ("reserved", C.c_int * 8)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("launches", C.c_uint64), ("budget", C.c_size_t), ("bytes_in_use", C.c_size_t),
                ("bytes_peak", C.c_size_t), ("queued", C.c_size_t), ("in_flight", C.c_size_t),
                ("grid_shapes", C.c_size_t)]


_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_vp, _i, _sz = C.c_void_p, C.c_int, C.c_size_t

_lib = None
# contexts and servers still open; closed in order at interpreter exit, while
# this module is intact (objects left to the garbage collector at shutdown
# would otherwise be finalised in no particular order)
_live = weakref.WeakSet()


def lib() -> C.CDLL:
    """Load libwrt.so (built by ``make -C wrt-project_b200``); raise if absent."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise WrtError(5, f"{LIB_PATH} is missing: build it with `make -C {HERE}`")
        L = C.CDLL(str(LIB_PATH))
        L.wrt_status_string.restype = C.c_char_p
        L.wrt_status_string.argtypes = [_i]
        L.wrt_abi_version.restype = _i
        L.wrt_ctx_create.argtypes = [_i, _sz, C.POINTER(_vp)]
        L.wrt_ctx_destroy.argtypes = [_vp]
        L.wrt_ctx_last_error.argtypes = [_vp]
        L.wrt_ctx_last_error.restype = C.c_char_p
        L.wrt_ctx_synchronize.argtypes = [_vp]
        L.wrt_ctx_bytes_in_use.argtypes = [_vp]
        L.wrt_ctx_bytes_in_use.restype = _sz
        L.wrt_ctx_launch_count.argtypes = [_vp]
        L.wrt_ctx_launch_count.restype = C.c_uint64
        L.wrt_ctx_stream.argtypes = [_vp]
        L.wrt_ctx_stream.restype = _vp
        L.wrt_gauss_legendre.argtypes = [_vp, _i, _dp, _dp]
        L.wrt_radon_grid_init.argtypes = [_vp, _i, _i, _i, _dp, _dp, _dp, _dp]
        L.wrt_radon_grid.argtypes = [_vp, _dp, _i, _i, _i, _i, C.POINTER(PlaneOpts), _dp]
        L.wrt_ray_grid.argtypes = [_vp, _dp, _i, _i, _i, _i, _vp, _dp]
        L.wrt_radon_reduction.argtypes = [_vp, _dp, _i, _i, _i, _i, _i, _dp]
        L.wrt_radon3d_adjoint.argtypes = [_vp, _dp, _i, _i, _i, _i, _dp]
        L.wrt_radon_transpose.argtypes = [_vp, _dp, _i, _i, _i, _i, C.POINTER(PlaneOpts), _dp]
        L.wrt_spectral_laplacian.argtypes = [_vp, _dp, _i, C.c_double, _dp]
        L.wrt_radon_analytic.argtypes = [_vp, C.POINTER(Function), _i, _i, _i, _i, _dp]
        L.wrt_fourier_slice_inversion.argtypes = [_vp, _dp, _i, _i, _i, C.c_double, _i, _i, _dp]
        L.wrt_ray_analytic.argtypes = [_vp, C.POINTER(Function), _i, _i, _i, _dp]
        L.wrt_spectral_laplacian_device.argtypes = [_vp, _vp, _i, C.c_double, _vp]
        L.wrt_volume_create.argtypes = [_vp, _i, C.POINTER(_vp)]
        L.wrt_volume_create_storage.argtypes = [_vp, _i, _i, C.POINTER(_vp)]
        L.wrt_volume_bytes.argtypes = [_vp]
        L.wrt_volume_bytes.restype = _sz
        L.wrt_volume_upload.argtypes = [_vp, _vp, _vp]
        L.wrt_volume_upload_device.argtypes = [_vp, _vp]
        L.wrt_volume_destroy.argtypes = [_vp]
        L.wrt_grid_create.argtypes = [_vp, _i, _i, _i, C.POINTER(_vp)]
        L.wrt_grid_destroy.argtypes = [_vp]
        L.wrt_radon_forward_device.argtypes = [_vp, _vp, _vp, C.POINTER(PlaneOpts), _vp]
        L.wrt_ray_forward_device.argtypes = [_vp, _vp, _vp, _i, _i, _i, _vp]
        L.wrt_radon_reduction_device.argtypes = [_vp, _vp, _i, _i, _vp, _vp]
        L.wrt_radon3d_adjoint_device.argtypes = [_vp, _vp, _vp, _i, _vp]
        L.wrt_radon3d_adjoint_static.argtypes = [_vp, _vp, _i, _i, _i, _i, _vp]
        L.wrt_ctx_timer_start.argtypes = [_vp]
        L.wrt_ctx_timer_stop.argtypes = [_vp, C.POINTER(C.c_float)]
        L.wrt_ctx_flush_l2.argtypes = [_vp]
        L.wrt_ctx_count_samples.argtypes = [_vp, _i]
        L.wrt_ctx_sample_count.argtypes = [_vp, C.POINTER(C.c_uint64)]
        L.wrt_measure_smem_bandwidth.argtypes = [_vp, C.POINTER(C.c_double)]
        L.wrt_device_alloc.argtypes = [_vp, _sz, C.POINTER(_vp)]
        L.wrt_device_free.argtypes = [_vp, _vp]
        L.wrt_host_alloc_pinned.argtypes = [_vp, _sz, C.POINTER(_vp)]
        L.wrt_host_free_pinned.argtypes = [_vp, _vp]
        L.wrt_copy_to_device.argtypes = [_vp, _vp, _vp, _sz]
        L.wrt_copy_to_host.argtypes = [_vp, _vp, _vp, _sz]
        L.wrt_tune_plane_kernel.argtypes = [_vp, _vp, _vp, C.POINTER(PlaneOpts), _vp,
                                            C.POINTER(_i), C.POINTER(C.c_float)]
        L.wrt_plane_kernel_config_describe.argtypes = [_i, C.POINTER(_i), C.POINTER(_i),
                                                       C.POINTER(_i)]
        L.wrt_ctx_set_plane_kernel_config.argtypes = [_vp, _i]
        L.wrt_radon_forward_batch.argtypes = [_vp, C.POINTER(ForwardReq), _i]
        L.wrt_server_create.argtypes = [C.POINTER(ServerOpts), C.POINTER(_vp)]
        L.wrt_server_submit.argtypes = [_vp, C.POINTER(Request), C.POINTER(C.c_uint64)]
        L.wrt_server_wait.argtypes = [_vp, C.c_uint64, _i, C.POINTER(RequestInfo)]
        L.wrt_server_get_stats.argtypes = [_vp, C.POINTER(ServerStats)]
        L.wrt_server_destroy.argtypes = [_vp]
        _lib = L
    return _lib


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _cube(a, dtype=np.float64) -> np.ndarray:
    """A C-contiguous n x n x n volume; anything else raises ValueError (the
    library reads n^3 values from the pointer it is given)."""
    v = np.ascontiguousarray(a, dtype=dtype)
    if v.ndim != 3 or not v.shape[0] == v.shape[1] == v.shape[2]:
        raise ValueError(f"volume must be an n x n x n array, got shape {v.shape}")
    return v


def _require(cond: bool, message: str):
    """Argument check that stays on under ``python -O`` (unlike assert): a
    wrong size here would let the library read or write past a buffer."""
    if not cond:
        raise ValueError(message)


def _out_array(out, count: int, what: str):
    _require(isinstance(out, np.ndarray) and out.flags.c_contiguous and out.dtype == np.float64
             and out.size == count, f"{what}: out must be a C-contiguous float64 array of "
                                    f"{count} values")


def plane_opts(sampler=NEAREST, half_extent=0, kernel=KERNEL_AUTO) -> PlaneOpts:
    o = PlaneOpts()
    o.sampler, o.half_extent, o.kernel = int(sampler), int(half_extent or 0), int(kernel)
    return o


class Context:
    """A libwrt context on one CUDA device (its own stream, budget, counters)."""

    def __init__(self, device: int = 0, budget_bytes: int = 0):
        self._h = _vp()
        self._children = weakref.WeakSet()  # resources created in this context
        st = lib().wrt_ctx_create(int(device), int(budget_bytes), C.byref(self._h))
        if st:
            raise WrtError(st, "wrt_ctx_create")
        _live.add(self)

    # -- plumbing
    @property
    def handle(self):
        return self._h

    def _adopt(self, obj):
        self._children.add(obj)

    def close(self):
        """Destroy the context; resources still open in it are closed first
        (the C library requires that order)."""
        if self._h:
            for c in list(self._children):
                c.close()
            lib().wrt_ctx_destroy(self._h)
            self._h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, st: int, what: str):
        if st:
            msg = lib().wrt_ctx_last_error(self._h)
            raise WrtError(st, f"{what}: {msg.decode() if msg else ''}")

    @property
    def launches(self) -> int:
        return int(lib().wrt_ctx_launch_count(self._h))

    @property
    def bytes_in_use(self) -> int:
        return int(lib().wrt_ctx_bytes_in_use(self._h))

    def synchronize(self):
        self.check(lib().wrt_ctx_synchronize(self._h), "synchronize")

    # -- measurement
    def timer_start(self):
        self.check(lib().wrt_ctx_timer_start(self._h), "timer_start")

    def timer_stop(self) -> float:
        ms = C.c_float()
        self.check(lib().wrt_ctx_timer_stop(self._h, C.byref(ms)), "timer_stop")
        return float(ms.value)

    def flush_l2(self):
        self.check(lib().wrt_ctx_flush_l2(self._h), "flush_l2")

    def count_samples(self, on: bool):
        self.check(lib().wrt_ctx_count_samples(self._h, int(bool(on))), "count_samples")

    def sample_count(self) -> int:
        v = C.c_uint64()
        self.check(lib().wrt_ctx_sample_count(self._h, C.byref(v)), "sample_count")
        return int(v.value)

    def smem_bandwidth(self) -> float:
        v = C.c_double()
        self.check(lib().wrt_measure_smem_bandwidth(self._h, C.byref(v)), "smem_bandwidth")
        return float(v.value)

    # -- grids
    def gauss_legendre(self, n: int):
        x, w = np.empty(n), np.empty(n)
        self.check(lib().wrt_gauss_legendre(self._h, n, x, w), "gauss_legendre")
        return x, w

    def radon_grid_init(self, nphi: int, ntheta: int, nshift: int):
        phi, th, w, s = np.empty(nphi), np.empty(ntheta), np.empty(ntheta), np.empty(nshift)
        self.check(lib().wrt_radon_grid_init(self._h, nphi, ntheta, nshift, phi, th, w, s),
                   "radon_grid_init")
        return phi, th, w, s

    # -- drop-in transforms
    def radon_grid(self, volume, nphi, ntheta, nshift, sampler=NEAREST, half_extent=0,
                   kernel=KERNEL_AUTO) -> np.ndarray:
        v = _cube(volume)
        n = v.shape[0]
        out = np.empty((nshift, nphi, ntheta))
        o = plane_opts(sampler, half_extent, kernel)
        self.check(lib().wrt_radon_grid(self._h, v, n, nphi, ntheta, nshift, C.byref(o), out),
                   "radon_grid")
        return out

    def ray_grid(self, volume, nslices, nshift, nphi, frame=None) -> np.ndarray:
        v = _cube(volume)
        out = np.empty((nslices, nshift, nphi))
        f = None if frame is None else _f64(frame).reshape(9)
        fp = None if f is None else f.ctypes.data_as(_vp)
        self.check(lib().wrt_ray_grid(self._h, v, v.shape[0], nslices, nshift, nphi, fp, out),
                   "ray_grid")
        return out

    def radon_reduction(self, rays, nshift, ntheta) -> np.ndarray:
        r = _f64(rays)
        ngrid, nsr, nphi = r.shape
        out = np.empty((nshift, nphi, ntheta))
        self.check(lib().wrt_radon_reduction(self._h, r, ngrid, nsr, nphi, nshift, ntheta, out),
                   "radon_reduction")
        return out

    def radon3d_adjoint(self, radon, ngrid) -> np.ndarray:
        R = _f64(radon)
        nshift, nphi, ntheta = R.shape
        out = np.empty((ngrid, ngrid, ngrid))
        self.check(lib().wrt_radon3d_adjoint(self._h, R, nphi, ntheta, nshift, ngrid, out),
                   "radon3d_adjoint")
        return out

    def fourier_slice_inversion(self, radon, ngrid, rsupp=1.0, padding=4) -> np.ndarray:
        """f on the ngrid^3 points -1 + 2l/ngrid ([ix][iy][iz]) from Radon data
        [s][phi][theta] via the Fourier slice theorem (rtft3d.m +
        nfft_reconstruct_3d.m, exact nonuniform sum)."""
        R = _f64(radon)
        nshift, nphi, ntheta = R.shape
        out = np.empty((ngrid, ngrid, ngrid))
        self.check(lib().wrt_fourier_slice_inversion(self._h, R, nphi, ntheta, nshift,
                                                     float(rsupp), int(padding), int(ngrid), out),
                   "fourier_slice_inversion")
        return out

    def radon_analytic(self, function, ngrid, nphi, ntheta, nshift) -> np.ndarray:
        """radon_analytic: plane integrals [s][phi][theta] of an analytic
        function (Function) on the reference's lattice for grid density ngrid."""
        out = np.empty((nshift, nphi, ntheta))
        self.check(lib().wrt_radon_analytic(self._h, C.byref(function), int(ngrid), int(nphi),
                                            int(ntheta), int(nshift), out), "radon_analytic")
        return out

    def ray_analytic(self, function, ngrid, nshift, nphi) -> np.ndarray:
        """ray_analytic: ray integrals [z][s][phi] on ngrid z-slices."""
        out = np.empty((ngrid, nshift, nphi))
        self.check(lib().wrt_ray_analytic(self._h, C.byref(function), int(ngrid), int(nshift),
                                          int(nphi), out), "ray_analytic")
        return out

    def spectral_laplacian(self, volume, period=2.0) -> np.ndarray:
        """ifftn(-(2 pi/period)^2 |k|^2 fftn(volume)) of an n^3 array
        (laplace3dfft.m), FP64 FFTs on the device."""
        v = _cube(volume)
        n = v.shape[0]
        out = np.empty_like(v)
        self.check(lib().wrt_spectral_laplacian(self._h, v, n, float(period), out),
                   "spectral_laplacian")
        return out

    def backprojection_inversion(self, radon, ngrid) -> np.ndarray:
        """The reference's backprojection inversion of Radon data on the
        Gauss-uniform sphere grid: f = -1/(8 pi^2) * Laplacian of the
        backprojection (cell-centred ngrid^3 grid on [-1, 1]^3, [iz][ix][iy])."""
        return self.spectral_laplacian(self.radon3d_adjoint(radon, ngrid), 2.0) * (
            -1.0 / (8.0 * np.pi ** 2))

    def radon_transpose(self, g, ngrid, sampler=TRILINEAR, half_extent=0) -> np.ndarray:
        g = _f64(g)
        nshift, nphi, ntheta = g.shape
        out = np.empty((ngrid, ngrid, ngrid))
        o = plane_opts(sampler, half_extent)
        self.check(lib().wrt_radon_transpose(self._h, g, ngrid, nphi, ntheta, nshift, C.byref(o),
                                             out), "radon_transpose")
        return out


class DeviceBuffer:
    """Caller-owned device memory (wrt_device_alloc), counted in the budget."""

    def __init__(self, ctx: Context, nbytes: int):
        self.ctx, self.nbytes, self._p = ctx, int(nbytes), _vp()
        ctx.check(lib().wrt_device_alloc(ctx.handle, self.nbytes, C.byref(self._p)), "device_alloc")
        ctx._adopt(self)

    @property
    def ptr(self) -> int:
        return int(self._p.value)

    def upload(self, host: np.ndarray):
        a = np.ascontiguousarray(host)
        _require(a.nbytes <= self.nbytes, f"upload of {a.nbytes} bytes into a {self.nbytes}-byte buffer")
        self.ctx.check(lib().wrt_copy_to_device(self.ctx.handle, self._p, a.ctypes.data_as(_vp),
                                                a.nbytes), "copy_to_device")

    def download(self, out: np.ndarray) -> np.ndarray:
        _require(isinstance(out, np.ndarray) and out.flags.c_contiguous and out.nbytes <= self.nbytes,
                 f"download needs a C-contiguous array of at most {self.nbytes} bytes")
        self.ctx.check(lib().wrt_copy_to_host(self.ctx.handle, out.ctypes.data_as(_vp), self._p,
                                              out.nbytes), "copy_to_host")
        return out

    def close(self):
        if self._p:
            if self.ctx.handle:
                lib().wrt_device_free(self.ctx.handle, self._p)
            self._p = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PinnedArray:
    """A numpy array over page-locked host memory (wrt_host_alloc_pinned)."""

    def __init__(self, ctx: Context, shape, dtype=np.float64):
        self.ctx, self._p = ctx, _vp()
        dt = np.dtype(dtype)
        nbytes = int(np.prod(shape)) * dt.itemsize
        ctx.check(lib().wrt_host_alloc_pinned(ctx.handle, nbytes, C.byref(self._p)), "pinned")
        ctx._adopt(self)
        buf = (C.c_char * nbytes).from_address(self._p.value)
        self.array = np.frombuffer(buf, dtype=dt).reshape(shape)

    def close(self):
        if self._p:
            self.array = None
            if self.ctx.handle:
                lib().wrt_host_free_pinned(self.ctx.handle, self._p)
            self._p = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Volume:
    """A volume resident on the device (wrt_volume); storage STORAGE_F32 or
    STORAGE_BF16 (values rounded to bfloat16, half the device memory)."""

    def __init__(self, ctx: Context, n: int, storage: int = STORAGE_F32):
        self.ctx, self.n, self._h = ctx, int(n), _vp()
        self.storage = int(storage)
        ctx.check(lib().wrt_volume_create_storage(ctx.handle, self.n, self.storage,
                                                  C.byref(self._h)), "volume_create")
        ctx._adopt(self)

    @property
    def nbytes(self) -> int:
        return int(lib().wrt_volume_bytes(self._h))

    @property
    def handle(self):
        return self._h

    def upload(self, data):
        a = np.ascontiguousarray(data)
        if a.shape != (self.n,) * 3:
            raise ValueError(f"volume must be {(self.n,) * 3}, got {a.shape}")
        if a.dtype == np.float32:
            st = lib().wrt_volume_upload(self._h, None, a.ctypes.data_as(_vp))
        else:
            a = a.astype(np.float64, copy=False)
            st = lib().wrt_volume_upload(self._h, a.ctypes.data_as(_vp), None)
        self.ctx.check(st, "volume_upload")

    def close(self):
        if self._h:
            if self.ctx.handle:
                lib().wrt_volume_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Grid:
    """A Gauss-uniform sphere grid with its tables resident on the device."""

    def __init__(self, ctx: Context, nphi: int, ntheta: int, nshift: int):
        self.ctx, self._h = ctx, _vp()
        self.nphi, self.ntheta, self.nshift = int(nphi), int(ntheta), int(nshift)
        ctx.check(lib().wrt_grid_create(ctx.handle, self.nphi, self.ntheta, self.nshift,
                                        C.byref(self._h)), "grid_create")
        ctx._adopt(self)

    @property
    def handle(self):
        return self._h

    @property
    def nplanes(self) -> int:
        return self.nphi * self.ntheta * self.nshift

    def close(self):
        if self._h:
            if self.ctx.handle:
                lib().wrt_grid_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def radon_forward_device(ctx: Context, vol: Volume, grid: Grid, dev_out: int, sampler=TRILINEAR,
                         half_extent=0, kernel=KERNEL_AUTO):
    """Plane integrals of a resident volume into device memory at ``dev_out``."""
    o = plane_opts(sampler, half_extent, kernel)
    ctx.check(lib().wrt_radon_forward_device(ctx.handle, vol.handle, grid.handle, C.byref(o),
                                             _vp(dev_out)), "radon_forward_device")


def ray_forward_device(ctx: Context, vol: Volume, nslices: int, nshift: int, nphi: int,
                       dev_out: int, frame=None):
    """Ray integrals of a resident volume into device memory at ``dev_out``
    ([iz][is][iphi] doubles); asynchronous on the context's stream."""
    f = None if frame is None else _f64(frame).reshape(9)
    fp = None if f is None else f.ctypes.data_as(_vp)
    ctx.check(lib().wrt_ray_forward_device(ctx.handle, vol.handle, fp, int(nslices), int(nshift),
                                           int(nphi), _vp(dev_out)), "ray_forward_device")


def radon_reduction_device(ctx: Context, dev_rays: int, ngrid: int, nshift_ray: int, grid: Grid,
                           dev_out: int):
    """Radon data on ``grid`` from device ray data [iz][is_ray][grid.nphi]."""
    ctx.check(lib().wrt_radon_reduction_device(ctx.handle, _vp(dev_rays), int(ngrid),
                                               int(nshift_ray), grid.handle, _vp(dev_out)),
              "radon_reduction_device")


def radon3d_adjoint_device(ctx: Context, dev_radon: int, grid: Grid, ngrid: int, dev_out: int):
    """Backprojection of device Radon data on ``grid`` to ngrid^3 voxels."""
    ctx.check(lib().wrt_radon3d_adjoint_device(ctx.handle, _vp(dev_radon), grid.handle,
                                               int(ngrid), _vp(dev_out)), "radon3d_adjoint_device")


def radon3d_adjoint_static(ctx: Context, dev_radon: int, nphi: int, ntheta: int, nshift: int,
                           ngrid: int, dev_out: int):
    """The backprojection with no device allocation (fixed working memory)."""
    ctx.check(lib().wrt_radon3d_adjoint_static(ctx.handle, _vp(dev_radon), int(nphi), int(ntheta),
                                               int(nshift), int(ngrid), _vp(dev_out)),
              "radon3d_adjoint_static")


def plane_kernel_configs():
    """Tile shapes of the staged plane kernel: list of (threads, rows per
    group, shifts per lane)."""
    out = []
    for k in range(lib().wrt_plane_kernel_config_count()):
        t, g, s = _i(), _i(), _i()
        lib().wrt_plane_kernel_config_describe(k, C.byref(t), C.byref(g), C.byref(s))
        out.append((t.value, g.value, s.value))
    return out


def set_plane_kernel_config(ctx: Context, index: int):
    ctx.check(lib().wrt_ctx_set_plane_kernel_config(ctx.handle, int(index)), "set config")


def tune_plane_kernel(ctx: Context, vol: Volume, grid: Grid, dev_out: int, sampler=TRILINEAR,
                      half_extent=0):
    """Run the autotuner on this request; returns (best index, ms per launch)."""
    o = plane_opts(sampler, half_extent, KERNEL_STAGED)
    best, ms = _i(), C.c_float()
    ctx.check(lib().wrt_tune_plane_kernel(ctx.handle, vol.handle, grid.handle, C.byref(o),
                                          _vp(dev_out), C.byref(best), C.byref(ms)), "tune")
    return best.value, float(ms.value)


def radon_forward_batch(ctx: Context, requests):
    """One launch for many forward requests.  ``requests``: sequence of
    (Volume, Grid, dev_out pointer, half_extent) tuples; asynchronous on the
    context's stream (trilinear sampler, staged kernel)."""
    arr = (ForwardReq * max(1, len(requests)))()
    for k, (vol, grid, dev_out, half_extent) in enumerate(requests):
        arr[k].volume = vol.handle.value
        arr[k].grid = grid.handle.value
        arr[k].half_extent = int(half_extent or 0)
        arr[k].dev_out = int(dev_out)
    ctx.check(lib().wrt_radon_forward_batch(ctx.handle, arr, len(requests)), "radon_forward_batch")


class Server:
    """The serving loop (wrt_server): submit forward / adjoint requests from
    host arrays, wait for them by id.  The arrays passed to ``submit`` are kept
    alive here until the request has been waited for."""

    def __init__(self, device: int = 0, max_batch: int = 0, max_inflight: int = 0,
                 budget_bytes: int = 0, queue_capacity: int = 0):
        o = ServerOpts()
        o.device, o.max_batch, o.max_inflight = int(device), int(max_batch), int(max_inflight)
        o.queue_capacity, o.hbm_budget = int(queue_capacity), int(budget_bytes)
        self._h = _vp()
        st = lib().wrt_server_create(C.byref(o), C.byref(self._h))
        if st:
            raise WrtError(st, "wrt_server_create")
        self._keep = {}
        _live.add(self)

    def submit_forward(self, volume, nphi, ntheta, nshift, out, half_extent=0, tag=0) -> int:
        """volume: float32 [n][n][n]; out: float64 [nshift][nphi][ntheta]."""
        v = _cube(volume, np.float32)
        _out_array(out, nshift * nphi * ntheta, "submit_forward")
        r = Request(OP_FORWARD, v.shape[0], nphi, ntheta, nshift, int(half_extent),
                    v.ctypes.data, None, out.ctypes.data, int(tag))
        return self._submit(r, (v, out))

    def submit_adjoint(self, radon, ngrid, out, tag=0) -> int:
        """radon: float64 [nshift][nphi][ntheta]; out: float64 [n][n][n] ([iz][ix][iy])."""
        g = np.ascontiguousarray(radon, dtype=np.float64)
        _require(g.ndim == 3, f"radon data must be [nshift][nphi][ntheta], got shape {g.shape}")
        nshift, nphi, ntheta = g.shape
        _out_array(out, int(ngrid) ** 3, "submit_adjoint")
        r = Request(OP_ADJOINT, int(ngrid), nphi, ntheta, nshift, 0, None, g.ctypes.data,
                    out.ctypes.data, int(tag))
        return self._submit(r, (g, out))

    def submit_ray(self, volume, nslices, nshift, nphi, out, frame=None, tag=0) -> int:
        """volume: float32 [n][n][n]; out: float64 [nslices][nshift][nphi]
        (ray_grid's order); frame: None (z-slices) or a 3x3 rotation."""
        v = _cube(volume, np.float32)
        _out_array(out, nslices * nshift * nphi, "submit_ray")
        f = None if frame is None else _f64(frame).reshape(9)
        r = Request(op=OP_RAY, ngrid=v.shape[0], nphi=int(nphi), ntheta=1, nshift=int(nshift),
                    volume=v.ctypes.data, out=out.ctypes.data, tag=int(tag),
                    nslices=int(nslices), frame=None if f is None else f.ctypes.data)
        return self._submit(r, (v, out, f))

    def submit_reduce(self, rays, nshift, ntheta, out, tag=0) -> int:
        """rays: float64 [ngrid][nshift_ray][nphi]; out: float64
        [nshift][nphi][ntheta] on the Gauss-uniform sphere grid."""
        g = np.ascontiguousarray(rays, dtype=np.float64)
        _require(g.ndim == 3, f"ray data must be [ngrid][nshift_ray][nphi], got shape {g.shape}")
        ngrid, nsr, nphi = g.shape
        _out_array(out, nshift * nphi * ntheta, "submit_reduce")
        r = Request(op=OP_REDUCE, ngrid=ngrid, nphi=nphi, ntheta=int(ntheta), nshift=int(nshift),
                    out=out.ctypes.data, tag=int(tag), nshift_ray=nsr, rays=g.ctypes.data)
        return self._submit(r, (g, out))

    def _submit(self, r, keep) -> int:
        rid = C.c_uint64()
        st = lib().wrt_server_submit(self._h, C.byref(r), C.byref(rid))
        if st:
            raise WrtError(st, "wrt_server_submit")
        self._keep[rid.value] = keep
        return rid.value

    def wait(self, rid: int, timeout_ms: int = -1) -> RequestInfo:
        info = RequestInfo()
        st = lib().wrt_server_wait(self._h, int(rid), int(timeout_ms), C.byref(info))
        if st == 6:  # still running
            raise TimeoutError(rid)
        self._keep.pop(rid, None)
        if st:
            raise WrtError(st, f"request {rid}")
        return info

    def stats(self) -> ServerStats:
        s = ServerStats()
        lib().wrt_server_get_stats(self._h, C.byref(s))
        return s

    def close(self):
        if self._h:
            lib().wrt_server_destroy(self._h)
            self._h = _vp()
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _close_all():
    """Servers first (their threads use their own contexts), then contexts
    (each closes its resources before itself)."""
    objs = sorted(list(_live), key=lambda o: not isinstance(o, Server))
    for o in objs:
        try:
            o.close()
        except Exception:
            pass


atexit.register(_close_all)


def round_bf16(a) -> np.ndarray:
    """Values rounded to bfloat16 (round to nearest even), as float64: what a
    STORAGE_BF16 volume holds."""
    x = np.ascontiguousarray(a, dtype=np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)
