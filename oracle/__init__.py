"""Python access to the oracle -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package.  It loads

* ``liboracle.so`` -- the FP64 C restatement of the reference hot path
  (``wrt_oracle.c``), and
* ``_ref/libref_*.so`` -- the reference's own hot-path sources compiled
  unmodified (present only where the reference tree was available at build
  time; the files travel with the repository snapshot otherwise).

Array layouts follow ``wrt_oracle.h``: volumes ``[ix][iy][iz]``, Radon data
``[shift][phi][theta]``, rays ``[z][shift][phi]``, adjoint ``[iz][ix][iy]``.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
NEAREST, TRILINEAR = 0, 1

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i, _d = C.c_int, C.c_double


def _load(path: Path):
    if not path.exists():
        raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
    return C.CDLL(str(path))


def _nthreads(n: int | None) -> int:
    return int(n) if n else (os.cpu_count() or 1)


class _Lib:
    _orc = None

    @classmethod
    def orc(cls):
        if cls._orc is None:
            L = _load(HERE / "liboracle.so")
            L.orc_radon_grid_init.argtypes = [_i, _i, _i, _dp, _dp, _dp, _dp]
            L.orc_ray_grid_init.argtypes = [_i, _i, _dp, _dp]
            L.orc_gauss_legendre.argtypes = [_i, _dp, _dp]
            L.orc_zero_interp.argtypes = [_dp, _i, _d, _d, _d]
            L.orc_zero_interp.restype = _d
            L.orc_trilinear.argtypes = [_dp, _i, _d, _d, _d]
            L.orc_trilinear.restype = _d
            L.orc_plane_integral.argtypes = [_dp, _i, _d, _d, _d, _i, _i]
            L.orc_plane_integral.restype = _d
            L.orc_radon_forward.argtypes = [_dp, _i, _i, _i, _i, _i, _i, _dp, _i]
            L.orc_radon_planes.argtypes = [_dp, _i, _i, _dp, _dp, _dp, _i, _i, _dp, _i]
            L.orc_ray_transform.argtypes = [_dp, _i, _d, _d, _d, C.c_void_p]
            L.orc_ray_transform.restype = _d
            L.orc_ray_forward.argtypes = [_dp, _i, _i, _i, _i, C.c_void_p, _dp, _i]
            L.orc_reduction_forward.argtypes = [_dp, _i, _i, _i, _i, _i, _dp, _i]
            L.orc_reduction_planes.argtypes = [_dp, _i, _i, _i, _i, _i, _i, _ip, _ip, _ip, _dp, _i]
            L.orc_adjoint_forward.argtypes = [_dp, _i, _i, _i, _i, _dp, _i]
            L.orc_adjoint_points.argtypes = [_dp, _i, _i, _i, _i, _dp, _dp, _dp, _dp, _i]
            L.orc_radon_transpose.argtypes = [_dp, _i, _i, _i, _i, _i, _i, _dp]
            cls._orc = L
        return cls._orc


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


# ----------------------------------------------------------------- restatement
def radon_grid(nphi: int, ntheta: int, nshift: int):
    """(phi, theta, theta_weights, shift) as radon_grid_init builds them."""
    phi, th, w, s = (np.empty(k) for k in (nphi, ntheta, ntheta, nshift))
    _Lib.orc().orc_radon_grid_init(nphi, ntheta, nshift, phi, th, w, s)
    return phi, th, w, s


def ray_grid(nshift: int, nphi: int):
    s, phi = np.empty(nshift), np.empty(nphi)
    _Lib.orc().orc_ray_grid_init(nshift, nphi, s, phi)
    return s, phi


def gauss_legendre(n: int):
    x, w = np.empty(n), np.empty(n)
    _Lib.orc().orc_gauss_legendre(n, x, w)
    return x, w


def trilinear(vol, x, y, z) -> float:
    v = _f64(vol)
    return _Lib.orc().orc_trilinear(v, v.shape[0], x, y, z)


def zero_interp(vol, x, y, z) -> float:
    v = _f64(vol)
    return _Lib.orc().orc_zero_interp(v, v.shape[0], x, y, z)


def plane_integral(vol, phi, theta, shift, sampler=NEAREST, half_extent=None) -> float:
    v = _f64(vol)
    n = v.shape[0]
    L = 2 * n if not half_extent else half_extent
    return _Lib.orc().orc_plane_integral(v, n, phi, theta, shift, sampler, L)


def radon_forward(vol, nphi, ntheta, nshift, sampler=NEAREST, half_extent=None, nthreads=None):
    v = _f64(vol)
    n = v.shape[0]
    L = 2 * n if not half_extent else half_extent
    out = np.empty((nshift, nphi, ntheta))
    _Lib.orc().orc_radon_forward(v, n, nphi, ntheta, nshift, sampler, L, out, _nthreads(nthreads))
    return out


def radon_planes(vol, phi, theta, shift, sampler=NEAREST, half_extent=None, nthreads=None):
    v = _f64(vol)
    n = v.shape[0]
    L = 2 * n if not half_extent else half_extent
    phi, theta, shift = _f64(phi), _f64(theta), _f64(shift)
    out = np.empty(phi.shape[0])
    _Lib.orc().orc_radon_planes(v, n, phi.shape[0], phi, theta, shift, sampler, L, out,
                                _nthreads(nthreads))
    return out


def _frame_ptr(frame):
    if frame is None:
        return None, None
    f = _f64(frame).reshape(9)
    return f, f.ctypes.data_as(C.c_void_p)


def ray_transform(vol, z, s, phi, frame=None) -> float:
    v = _f64(vol)
    keep, fp = _frame_ptr(frame)
    return _Lib.orc().orc_ray_transform(v, v.shape[0], z, s, phi, fp)


def ray_forward(vol, nslices, nshift, nphi, frame=None, nthreads=None):
    v = _f64(vol)
    keep, fp = _frame_ptr(frame)
    out = np.empty((nslices, nshift, nphi))
    _Lib.orc().orc_ray_forward(v, v.shape[0], nslices, nshift, nphi, fp, out, _nthreads(nthreads))
    return out


def reduction_forward(rays, nshift, ntheta, nthreads=None):
    """rays: [ngrid][nshift_ray][nphi] (file order); Radon grid (nshift, nphi, ntheta)."""
    r = _f64(rays)
    ngrid, nsr, nphi = r.shape
    out = np.empty((nshift, nphi, ntheta))
    _Lib.orc().orc_reduction_forward(r, ngrid, nsr, nphi, nshift, ntheta, out, _nthreads(nthreads))
    return out


def reduction_planes(rays, nshift, ntheta, idx_s, idx_phi, idx_theta, nthreads=None):
    r = _f64(rays)
    ngrid, nsr, nphi = r.shape
    a, b, c = (np.ascontiguousarray(q, dtype=np.int32) for q in (idx_s, idx_phi, idx_theta))
    out = np.empty(a.shape[0])
    _Lib.orc().orc_reduction_planes(r, ngrid, nsr, nphi, nshift, ntheta, a.shape[0], a, b, c, out,
                                    _nthreads(nthreads))
    return out


def adjoint_forward(radon, n, nthreads=None):
    R = _f64(radon)
    nshift, nphi, ntheta = R.shape
    out = np.empty((n, n, n))
    _Lib.orc().orc_adjoint_forward(R, nphi, ntheta, nshift, n, out, _nthreads(nthreads))
    return out


def adjoint_points(radon, x, y, z, nthreads=None):
    R = _f64(radon)
    nshift, nphi, ntheta = R.shape
    x, y, z = _f64(x), _f64(y), _f64(z)
    out = np.empty(x.shape[0])
    _Lib.orc().orc_adjoint_points(R, nphi, ntheta, nshift, x.shape[0], x, y, z, out,
                                  _nthreads(nthreads))
    return out


def radon_transpose(g, n, sampler=TRILINEAR, half_extent=None):
    g = _f64(g)
    nshift, nphi, ntheta = g.shape
    L = 2 * n if not half_extent else half_extent
    out = np.zeros((n, n, n))
    _Lib.orc().orc_radon_transpose(g, n, nphi, ntheta, nshift, sampler, L, out)
    return out


def spectral_laplacian(u, period=2.0):
    """radon_inversion/backprojection/laplace3dfft.m:1-25 in numpy: the real part
    of ifftn(U * fftn(u)), U = -(2 pi / period)^2 (k1^2 + k2^2 + k3^2) with the
    FFT-order frequencies k = i (i <= n/2) or i - n (laplace3dfft.m:9-15)."""
    u = _f64(u)
    n = u.shape[0]
    k = np.array([i if i <= n // 2 else i - n for i in range(n)], dtype=np.float64)
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    U = -(2.0 * np.pi / period) ** 2 * k2
    return np.real(np.fft.ifftn(U * np.fft.fftn(u)))


def fourier_slice_inversion(radon, ngrid, rsupp=1.0, padding=4, points=None):
    """The Fourier-slice inversion (radon_inversion/rtft3d.m +
    nfft_reconstruct_3d.m) in FP64 numpy with physical frequencies and an
    exact nonuniform sum: F(nu_k w) = ds sum_j R(s_j) e^{-2 pi i nu_k s_j},
    s_j = -rsupp + j ds, ds = 2 rsupp/(nshift-1), ntotal = padding floor(1/ds),
    nu_k = k dnu, dnu = 1/(ntotal ds), k in [-ntotal/2, ntotal/2), and
    f(y) = Re 1/2 sum_{w,k} dnu dphi w_theta nu_k^2 F(nu_k w) e^{2 pi i nu_k w.y}
    at `points` (M x 3), default the grid -1 + 2l/ngrid, order [ix][iy][iz]."""
    R = _f64(radon)
    nshift, nphi, ntheta = R.shape
    phi, theta, w, _ = radon_grid(nphi, ntheta, nshift)
    ds = 2.0 * rsupp / (nshift - 1)
    ntotal = padding * int(np.floor(1.0 / ds))
    dnu = 1.0 / (ntotal * ds)
    k = np.arange(-(ntotal // 2), ntotal - ntotal // 2)
    nu = k * dnu
    s = -rsupp + ds * np.arange(nshift)
    lines = R.reshape(nshift, nphi * ntheta).T                           # [d][j]
    F = ds * lines @ np.exp(-2j * np.pi * np.outer(s, nu))               # [d][k]
    wd = (2 * np.pi / nphi) * np.tile(w, nphi)                           # d = ip*ntheta + it
    C = 0.5 * dnu * wd[:, None] * nu[None, :] ** 2 * F
    st, ct = np.sin(theta)[None, :], np.cos(theta)[None, :]
    om = np.stack([(st * np.cos(phi)[:, None]).ravel(), (st * np.sin(phi)[:, None]).ravel(),
                   np.repeat(ct, nphi, 0).ravel()], 1)                   # [d][3], d = ip*ntheta + it
    grid = points is None
    if grid:
        g = -1.0 + 2.0 * np.arange(ngrid) / ngrid
        X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
        points = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    out = np.zeros(points.shape[0])
    for d in range(om.shape[0]):
        u = points @ om[d]                                               # [M]
        out += np.real(np.exp(2j * np.pi * np.outer(u, nu)) @ C[d])
    return out.reshape((ngrid,) * 3) if grid else out


# ------------------------------------------------- the reference, compiled here
class Reference:
    """The reference's own hot-path code (oracle/_ref), via small drivers."""

    def __init__(self):
        d = HERE / "_ref"
        self.radon = _load(d / "libref_radon_grid.so")
        self.radon.refdrv_radon_grid_init.argtypes = [_i, _i, _i, _dp, _dp, _dp]
        self.radon.refdrv_plane_integrals.argtypes = [_dp, _i, _i, _dp, _dp, _dp, _dp, _i]
        self.radon.refdrv_samplers.argtypes = [_dp, _i, _i, _dp, _dp, _dp, _dp, _dp]
        self.ray = _load(d / "libref_ray_grid.so")
        self.ray.refdrv_ray_forward.argtypes = [_dp, _i, _i, _i, _i, _dp, _i]
        self.ray.refdrv_rays.argtypes = [_dp, _i, _i, _dp, _dp, _dp, _dp, _i]
        self.red = _load(d / "libref_reduction.so")
        self.red.refdrv_reduction_planes.argtypes = [_dp, _i, _i, _i, _i, _i, _ip, _ip, _ip, _dp, _i]
        self.adj = _load(d / "libref_adjoint.so")
        self.adj.refdrv_adjoint_points.argtypes = [_dp, _i, _i, _i, _i, _dp, _dp, _dp, _dp, _i]
        self.adj.refdrv_grid.argtypes = [_i, _i, _i, _dp, _dp, _dp, _dp]

    @staticmethod
    def available() -> bool:
        return (HERE / "_ref" / "libref_radon_grid.so").exists()

    @staticmethod
    def analytic(kind: str, family: str):
        """The reference's radon_analytic ('plane') or ray_analytic ('ray')
        integrator compiled with its example function `family` ('exp':
        exponential_bump.c, 'sine': sinusoidal_bump.c)."""
        name = {"plane": "radon_analytic", "ray": "ray_analytic"}[kind]
        L = _load(HERE / "_ref" / f"libref_{name}_{family}.so")
        if kind == "plane":
            L.refdrv_analytic_planes.argtypes = [_i, _i, _dp, _dp, _dp, _dp, _i]
        else:
            L.refdrv_analytic_rays.argtypes = [_i, _i, _dp, _dp, _dp, _dp, _i]
        L.refdrv_analytic_values.argtypes = [_i, _dp, _dp, _dp, _dp]
        return L

    def analytic_planes(self, family, ngrid, phi, theta, shift, nthreads=None):
        L = self.analytic("plane", family)
        phi, theta, shift = _f64(phi), _f64(theta), _f64(shift)
        out = np.empty(phi.shape[0])
        L.refdrv_analytic_planes(ngrid, phi.shape[0], phi, theta, shift, out, _nthreads(nthreads))
        return out

    def analytic_rays(self, family, ngrid, z, shift, phi, nthreads=None):
        L = self.analytic("ray", family)
        z, shift, phi = _f64(z), _f64(shift), _f64(phi)
        out = np.empty(z.shape[0])
        L.refdrv_analytic_rays(ngrid, z.shape[0], z, shift, phi, out, _nthreads(nthreads))
        return out

    def analytic_values(self, family, x, y, z):
        L = self.analytic("plane", family)
        x, y, z = _f64(x), _f64(y), _f64(z)
        out = np.empty(x.shape[0])
        L.refdrv_analytic_values(x.shape[0], x, y, z, out)
        return out

    def radon_grid(self, nphi, ntheta, nshift):
        phi, th, s = np.empty(nphi), np.empty(ntheta), np.empty(nshift)
        self.radon.refdrv_radon_grid_init(nphi, ntheta, nshift, phi, th, s)
        return phi, th, s

    def adjoint_grid(self, nphi, ntheta, nshift):
        phi, th, w, s = np.empty(nphi), np.empty(ntheta), np.empty(ntheta), np.empty(nshift)
        self.adj.refdrv_grid(nphi, ntheta, nshift, phi, th, w, s)
        return phi, th, w, s

    def plane_integrals(self, vol, phi, theta, shift, nthreads=None):
        v = _f64(vol)
        phi, theta, shift = _f64(phi), _f64(theta), _f64(shift)
        out = np.empty(phi.shape[0])
        self.radon.refdrv_plane_integrals(v, v.shape[0], phi.shape[0], phi, theta, shift, out,
                                          _nthreads(nthreads))
        return out

    def samplers(self, vol, x, y, z):
        v = _f64(vol)
        x, y, z = _f64(x), _f64(y), _f64(z)
        a, b = np.empty(x.shape[0]), np.empty(x.shape[0])
        self.radon.refdrv_samplers(v, v.shape[0], x.shape[0], x, y, z, a, b)
        return a, b

    def ray_forward(self, vol, nslices, nshift, nphi, nthreads=None):
        v = _f64(vol)
        out = np.empty((nslices, nshift, nphi))
        self.ray.refdrv_ray_forward(v, v.shape[0], nslices, nshift, nphi, out, _nthreads(nthreads))
        return out

    def rays(self, vol, z, s, phi, nthreads=None):
        v = _f64(vol)
        z, s, phi = _f64(z), _f64(s), _f64(phi)
        out = np.empty(z.shape[0])
        self.ray.refdrv_rays(v, v.shape[0], z.shape[0], z, s, phi, out, _nthreads(nthreads))
        return out

    def reduction_planes(self, rays, ntheta, idx_s, idx_phi, idx_theta, nthreads=None):
        r = _f64(rays)
        ngrid, nshift, nphi = r.shape
        a, b, c = (np.ascontiguousarray(q, dtype=np.int32) for q in (idx_s, idx_phi, idx_theta))
        out = np.empty(a.shape[0])
        self.red.refdrv_reduction_planes(r, ngrid, nshift, nphi, ntheta, a.shape[0], a, b, c, out,
                                         _nthreads(nthreads))
        return out

    def adjoint_points(self, radon, x, y, z, nthreads=None):
        R = _f64(radon)
        nshift, nphi, ntheta = R.shape
        x, y, z = _f64(x), _f64(y), _f64(z)
        out = np.empty(x.shape[0])
        self.adj.refdrv_adjoint_points(R, nphi, ntheta, nshift, x.shape[0], x, y, z, out,
                                       _nthreads(nthreads))
        return out
