// k_fourier.cu -- inversion of 3D Radon data through the Fourier slice
// theorem, the reference's main reconstruction route (radon_inversion/
// rtft3d.m: 1D Fourier transform of every projection along the shift;
// nfft_reconstruct_3d.m: the inverse 3D Fourier integral at the grid points by
// an adjoint NFFT).
//
// With F(nu w) = int Rf(s, w) e^{-2 pi i nu s} ds = fhat(nu w),
//   f(y) = 1/2 int_{S^2} int_R F(nu w) e^{2 pi i nu w.y} nu^2 dnu dw,
// discretised as the reference sets it up: shifts s_j = -rsupp + j ds,
// ds = 2 rsupp/(nshift - 1), zero padding to ntotal = padding floor(1/ds)
// points, frequencies nu_k = k dnu, dnu = 1/(ntotal ds), k in [-ntotal/2,
// ntotal/2), directions w on the Gauss-uniform sphere grid with weights
// dphi w_theta, and the Jacobian weight 1/2 ds dnu dphi w_theta nu_k^2 per node
// (rtft3d.m:41-49, 96-101).  Differences from the scripts, which this file
// fixes: nodes are physical frequencies nu_k w (the scripts use the index k),
// the values keep the frequency order of their nodes (the scripts pair
// fftshift-ed values with FFT-ordered nodes) and the phase factor
// e^{2 pi i nu_k rsupp} uses each node's own frequency; the inverse integral
// is the exact sum over the nodes (an adjoint NFFT approximates it) and no
// zero-valued stabilisation nodes are needed for an exact sum.
//
// Kernels: slice_ft_kernel -- per direction, the DFT of its zero-padded line
// for k = 0 .. ntotal/2 in FP64, times the node weights (real data:
// F(-nu w) = conj F(nu w), so with the 1/2 of the double cover the pair
// (k, -k) adds Re(F e) dnu dphi w_theta nu^2 once; for even ntotal the
// unpaired node -ntotal/2 half of that); fourier_sum_kernel -- per voxel, the sum over directions and
// frequencies of Re(c_{d,k} e^{2 pi i k dnu w_d.y}), with the phase rotated
// by one complex multiply per frequency and re-anchored with sincospi every
// 32 frequencies (FP32; the anchor phase from an FP64 fraction of a turn).
#include <math.h>

#include <vector>

#include "wrt_internal.cuh"

namespace {

constexpr int kAnchor = 32;       // frequencies between exact phase anchors
constexpr int kFsDirChunk = 64;   // directions staged in shared memory at once

// c[d][k] (k = 0 .. K, K = ntotal/2): weighted Fourier coefficients of
// direction d's line radon[is][d] (stride ndir), float2 (re, im).
__global__ void slice_ft_kernel(const double *__restrict__ radon, int ndir, int nshift,
                                double ds, double rsupp, int ntotal, double dnu,
                                const double *__restrict__ wdir /* [ndir] dphi w_theta */,
                                float2 *__restrict__ c) {
  const int K = ntotal / 2;
  const long long total = (long long)ndir * (K + 1);
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(idx % (K + 1)), d = (int)(idx / (K + 1));
    // sum_j R_j e^{-2 pi i k j / ntotal}, exact phases by sincospi of k j / (ntotal/2)
    double re = 0.0, im = 0.0;
    for (int j = 0; j < nshift; ++j) {
      const long long kj = ((long long)k * j) % ntotal;  // exact turn count
      double sn, cs;
      sincospi(-2.0 * (double)kj / (double)ntotal, &sn, &cs);
      const double r = radon[(size_t)j * ndir + d];
      re += r * cs;
      im += r * sn;
    }
    // e^{2 pi i nu_k rsupp}: the line starts at s = -rsupp
    const double nu = k * dnu;
    double sn, cs;
    sincospi(2.0 * nu * rsupp, &sn, &cs);
    const double fr = ds * (re * cs - im * sn), fi = ds * (re * sn + im * cs);
    // 1/2 ds dnu dphi w nu^2 per node (ds already in F); the (k, -k) pair's
    // real parts are equal, the node -K has no partner
    const double w =
        (k == 0 ? 0.0 : (k == K && !(ntotal & 1) ? 0.5 : 1.0)) * dnu * wdir[d] * nu * nu;
    c[idx] = make_float2((float)(w * fr), (float)(w * fi));
  }
}

// One thread per voxel y = (-1 + 2 ix/n, -1 + 2 iy/n, -1 + 2 iz/n), order
// [ix][iy][iz]; dirs[d] = (w_x, w_y, w_z) FP64.
__global__ void __launch_bounds__(256)
    fourier_sum_kernel(const float2 *__restrict__ c, const double *__restrict__ dirs, int ndir,
                       int K, double dnu, int n, double *__restrict__ out) {
  __shared__ float2 sc[kFsDirChunk * 33];  // coefficients of a chunk, kAnchor+1 at a time
  __shared__ double sw[kFsDirChunk * 3];
  const long long nvox = (long long)n * n * n;
  const long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const bool active = v < nvox;
  const int iz = (int)(v % n), iy = (int)((v / n) % n), ix = (int)(v / ((long long)n * n));
  const double y0 = -1.0 + 2.0 * ix / n, y1 = -1.0 + 2.0 * iy / n, y2 = -1.0 + 2.0 * iz / n;
  double acc = 0.0;
  for (int d0 = 0; d0 < ndir; d0 += kFsDirChunk) {
    const int nd = min(kFsDirChunk, ndir - d0);
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * nd; i += blockDim.x) sw[i] = dirs[3 * (size_t)d0 + i];
    for (int k0 = 1; k0 <= K; k0 += kAnchor) {
      const int nk = min(kAnchor, K + 1 - k0);
      __syncthreads();
      for (int i = threadIdx.x; i < nd * nk; i += blockDim.x) {
        const int dd = i / nk, kk = i % nk;
        sc[dd * 33 + kk] = c[(size_t)(d0 + dd) * (K + 1) + k0 + kk];
      }
      __syncthreads();
      if (active) {
        float part = 0.0f;
        for (int dd = 0; dd < nd; ++dd) {
          // turns per frequency step, and the anchor phase at k0, exactly reduced
          const double u = sw[3 * dd] * y0 + sw[3 * dd + 1] * y1 + sw[3 * dd + 2] * y2;
          const double step = dnu * u;
          const double a = step * k0;
          float s1, c1, sa, ca;
          sincospif((float)(2.0 * (step - rint(step))), &s1, &c1);
          sincospif((float)(2.0 * (a - rint(a))), &sa, &ca);
          float zr = ca, zi = sa;
          for (int kk = 0; kk < nk; ++kk) {
            const float2 q = sc[dd * 33 + kk];
            part = fmaf(q.x, zr, fmaf(-q.y, zi, part));
            const float tr = zr * c1 - zi * s1;
            zi = fmaf(zr, s1, zi * c1);
            zr = tr;
          }
        }
        acc += (double)part;
      }
    }
  }
  if (active) out[v] = acc;
}

}  // namespace

extern "C" int wrt_fourier_slice_inversion(wrt_ctx *ctx, const double *radon, int nphi, int ntheta,
                                           int nshift, double rsupp, int padding, int ngrid,
                                           double *out) {
  if (!ctx || !radon || !out || nphi < 1 || ntheta < 1 || nshift < 3 || !(rsupp > 0.0) ||
      padding < 1 || padding > 64 || ngrid < 2 || ngrid > 1024)
    return ctx ? wrt::fail(ctx, WRT_ERR_INVALID_ARGUMENT, "fourier_slice_inversion: bad arguments")
               : WRT_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return wrt::cuda_fail(ctx, e, "cudaSetDevice");
  // the reference's discretisation (rtft3d.m:41-46)
  const double ds = 2.0 * rsupp / (nshift - 1);
  // the frequency count in FP64 first: a tiny rsupp would overflow the int
  const double nfreq = padding * floor(1.0 / ds);
  if (!(nfreq >= 2.0))
    return wrt::fail(ctx, WRT_ERR_INVALID_ARGUMENT, "fourier_slice_inversion: too few frequencies");
  if (nfreq > (double)(1 << 24))
    return wrt::fail(ctx, WRT_ERR_INVALID_ARGUMENT,
                     "fourier_slice_inversion: %.0f padded shifts (at most %d)", nfreq, 1 << 24);
  const int ntotal = (int)nfreq;
  const double dnu = 1.0 / (ntotal * ds);
  const int K = ntotal / 2, ndir = nphi * ntheta;
  // sphere grid (GL nodes on the GPU) and per-direction weights / unit vectors
  std::vector<double> phi(nphi), theta(ntheta), w(ntheta), shift(nshift);
  int st = wrt::sphere_grid(ctx, nphi, ntheta, nshift, phi.data(), theta.data(), w.data(),
                            shift.data());
  if (st) return st;
  std::vector<double> tab(4 * (size_t)ndir);  // dirs[3*ndir], then weights[ndir]
  const double dphi = 2 * M_PI / nphi;
  for (int ip = 0; ip < nphi; ++ip)
    for (int it = 0; it < ntheta; ++it) {
      const int d = ip * ntheta + it;
      tab[3 * d] = sin(theta[it]) * cos(phi[ip]);
      tab[3 * d + 1] = sin(theta[it]) * sin(phi[ip]);
      tab[3 * d + 2] = cos(theta[it]);
      tab[3 * (size_t)ndir + d] = dphi * w[it];
    }
  const size_t nin = (size_t)nshift * ndir, nout = (size_t)ngrid * ngrid * ngrid;
  void *din = nullptr, *dtab = nullptr, *dc = nullptr, *dout = nullptr;
  st = wrt::ws_get(ctx, wrt::WS_IN, sizeof(double) * nin, &din);
  if (!st) st = wrt::ws_get(ctx, wrt::WS_TABLE, sizeof(double) * tab.size(), &dtab);
  if (!st) st = wrt::ws_get(ctx, wrt::WS_LINES, sizeof(float2) * (size_t)ndir * (K + 1), &dc);
  if (!st) st = wrt::ws_get(ctx, wrt::WS_OUT, sizeof(double) * nout, &dout);
  if (st) return st;
  e = cudaMemcpyAsync(din, radon, sizeof(double) * nin, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dtab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice,
                        ctx->stream);
  if (e != cudaSuccess) return wrt::cuda_fail(ctx, e, "fourier_slice_inversion input");
  const double *d_dirs = static_cast<const double *>(dtab);
  slice_ft_kernel<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(
      static_cast<const double *>(din), ndir, nshift, ds, rsupp, ntotal, dnu, d_dirs + 3 * ndir,
      static_cast<float2 *>(dc));
  ctx->launches++;
  st = wrt::check_launch(ctx, "slice_ft_kernel");
  if (st) return st;
  fourier_sum_kernel<<<(unsigned)((nout + 255) / 256), 256, 0, ctx->stream>>>(
      static_cast<const float2 *>(dc), d_dirs, ndir, K, dnu, ngrid, static_cast<double *>(dout));
  ctx->launches++;
  st = wrt::check_launch(ctx, "fourier_sum_kernel");
  if (st) return st;
  e = cudaMemcpyAsync(out, dout, sizeof(double) * nout, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? WRT_OK : wrt::cuda_fail(ctx, e, "fourier_slice_inversion result");
}
