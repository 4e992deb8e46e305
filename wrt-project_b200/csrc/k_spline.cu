// k_spline.cu -- natural cubic splines in the shift variable, the ray-to-Radon
// reduction (radon_reduction/slicing.c:5-119) and the backprojection adjoint
// (radon_inversion/backprojection/C/src/integral.c:6-24, interp.c:5-28).
//
// The reference builds a GSL natural cubic spline of a whole data line for
// every single evaluation (slicing.c:45-61, backprojection interp.c:41-45).
// A line's spline depends only on that line, so here it is built once:
// spline_prep_kernel solves the natural-spline tridiagonal system of every
// line (uniform knots s_i = -1 + i h, h = 2/(ns-1), end conditions M_0 =
// M_{ns-1} = 0) in FP64 and stores one float4 per knot interval (the record
// forms are described in spline_dev.cuh); an evaluation is one 16-byte load
// and the same piecewise cubic as the reference's spline.
#include <vector>

#include "spline_dev.cuh"
#include "wrt_internal.cuh"

namespace {

// One thread per line.  src element k of line L is at src[L*line_stride_a +
// (L / lines_per_group)*... ] -- simplified by the two-level indexing below:
//   line L = (outer, inner), element e at
//   src[outer*so + e*se + inner*si].
// cp[i] / den[i]: forward-elimination coefficients of the (line-independent)
// tridiagonal matrix, computed on the host.
__global__ void spline_prep_kernel(const double *__restrict__ src, int nlines, int ninner,
                                   long long so, long long se, long long si, int ns, double h,
                                   const double *__restrict__ cp, const double *__restrict__ den,
                                   double *__restrict__ scratch, float4 *__restrict__ out,
                                   const double4 *__restrict__ weights) {
  const int L = blockIdx.x * blockDim.x + threadIdx.x;
  if (L >= nlines) return;
  const int outer = L / ninner, inner = L % ninner;
  // adjoint lines (weights given): centred power form scaled by the
  // direction's quadrature weight dphi * w_theta; reduction lines: values and
  // curvatures
  if (weights)
    wrtd::spline_line_centred(src + outer * so + inner * si, se, ns, h, cp, den,
                              scratch + (size_t)L * ns, out + (size_t)L * (ns - 1), weights[L].w);
  else
    wrtd::spline_line(src + outer * so + inner * si, se, ns, h, cp, den, scratch + (size_t)L * ns,
                      out + (size_t)L * (ns - 1));
}

// Reduction: one thread per Radon sample (wrtd::reduction_one), a warp on
// consecutive shifts (wrtd::reduction_sample_of).
__global__ void __launch_bounds__(256)
    reduction_kernel(const float4 *__restrict__ lines /* [iz][iphi][ns_ray-1] */, int ngrid,
                     int ns_ray, int nphi, const double *__restrict__ shift, int nshift,
                     const double *__restrict__ cs /* [ntheta][2] cos, sin */, int ntheta,
                     double *__restrict__ out, unsigned long long *counter) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nshift * nphi * ntheta) return;
  const long long k = wrtd::reduction_sample_of(t, nshift, nphi, ntheta);
  int evaluated = 0;
  out[k] = wrtd::reduction_one(lines, ngrid, ns_ray, nphi, shift, cs, ntheta, k, &evaluated);
  if (counter) atomicAdd(counter, (unsigned long long)evaluated);
}

// Adjoint: one warp per voxel block of wrtd::adjoint_block (8 x 4 columns of
// V voxels), output order [iz][ix][iy]; one launch per kAdjDirsPerLaunch
// directions, their constants in the parameter space.
template <int V>
__global__ void __launch_bounds__(256, V == 4 ? 3 : 2)
    adjoint_kernel(const float4 *__restrict__ lines /* [d][ns-1] */, int ns, int dbeg, int nd,
                   const __grid_constant__ wrtd::AdjDirs dirs, int n, double *__restrict__ out) {
  const long long w = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (w >= wrtd::adjoint_warps(n)) return;
  wrtd::adjoint_block<V>(lines, ns, dbeg, nd, dirs, n, w, threadIdx.x & 31, out);
}

// Natural splines of nlines lines into the context's workspace (records in
// WS_LINES); asynchronous on the context's stream.
int prep_lines(wrt_ctx *ctx, const double *d_src, int nlines, int ninner, long long so,
               long long se, long long si, int ns, float4 **d_lines,
               const double4 *d_weights) {
  // line-independent elimination coefficients for the uniform-knot system
  // h M_{i-1} + 4h M_i + h M_{i+1} = rhs (divided by h: M_{i-1} + 4 M_i + M_{i+1})
  const double h = 2.0 / (ns - 1);
  std::vector<double> coef(2 * (size_t)ns, 0.0);
  wrt::spline_coefficients(ns, coef.data(), coef.data() + ns);
  void *d_coef = nullptr, *d_scratch = nullptr, *lines = nullptr;
  int st = wrt::ws_get(ctx, wrt::WS_COEF, sizeof(double) * coef.size(), &d_coef);
  if (!st) st = wrt::ws_get(ctx, wrt::WS_SPLINE, sizeof(double) * (size_t)nlines * ns, &d_scratch);
  if (!st) st = wrt::ws_get(ctx, wrt::WS_LINES, sizeof(float4) * (size_t)nlines * (ns - 1), &lines);
  if (st) return st;
  // a copy from pageable memory returns once the data is staged
  cudaError_t e = cudaMemcpyAsync(d_coef, coef.data(), sizeof(double) * coef.size(),
                                  cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) return wrt::cuda_fail(ctx, e, "spline coefficients");
  const double *dc = static_cast<const double *>(d_coef);
  *d_lines = static_cast<float4 *>(lines);
  spline_prep_kernel<<<(nlines + 127) / 128, 128, 0, ctx->stream>>>(
      d_src, nlines, ninner, so, se, si, ns, h, dc, dc + ns, static_cast<double *>(d_scratch),
      *d_lines, d_weights);
  ctx->launches++;
  return wrt::check_launch(ctx, "spline_prep_kernel");
}

}  // namespace

namespace wrt {

// Launchers over caller-provided device memory (used by the allocation-free
// adjoint entry point): spline preparation of the nphi*ntheta lines of a
// Radon data set ([nshift][nphi][ntheta]) and the adjoint proper.
cudaError_t launch_adjoint_lines(cudaStream_t stream, const double *d_radon, int ndir, int nshift,
                                 const double *d_cp, const double *d_den, double *d_scratch,
                                 float4 *d_lines, const double4 *d_dirw) {
  spline_prep_kernel<<<(ndir + 127) / 128, 128, 0, stream>>>(
      d_radon, ndir, ndir, 0, (long long)ndir, 1, nshift, 2.0 / (nshift - 1), d_cp, d_den,
      d_scratch, d_lines, d_dirw);
  return cudaGetLastError();
}

cudaError_t launch_adjoint(cudaStream_t stream, const float4 *d_lines, int ndir, int nshift,
                           const double4 *h_dirw, int n, double *d_out, uint64_t *launches) {
  // parameters of one launch, filled on the host (the launch copies them)
  static thread_local wrtd::AdjDirs dirs;
  const int V = wrtd::adjoint_vox(n);
  const unsigned blocks = (unsigned)((wrtd::adjoint_warps(n) + 7) / 8);
  for (int d0 = 0; d0 < ndir; d0 += wrtd::kAdjDirsPerLaunch) {
    const int nd = ndir - d0 < wrtd::kAdjDirsPerLaunch ? ndir - d0 : wrtd::kAdjDirsPerLaunch;
    for (int j = 0; j < nd; ++j) {
      const double4 g = h_dirw[d0 + j];
      dirs.g[j][0] = g.x;
      dirs.g[j][1] = g.y;
      dirs.g[j][2] = g.z;
      wrtd::adjoint_header(g.x, n, nshift, V, &dirs.hd[j]);
    }
    if (V == 8)
      adjoint_kernel<8><<<blocks, 256, 0, stream>>>(d_lines, nshift, d0, nd, dirs, n, d_out);
    else
      adjoint_kernel<4><<<blocks, 256, 0, stream>>>(d_lines, nshift, d0, nd, dirs, n, d_out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (launches) ++*launches;
  }
  return cudaSuccess;
}

int reduction_forward(wrt_ctx *ctx, const double *d_rays, int ngrid, int nshift_ray, int nphi,
                      const double *d_shift, int nshift, const double *d_cs, int ntheta,
                      double *d_out) {
  // lines (iz, iphi): element is at d_rays[(iz*ns_ray + is)*nphi + iphi]
  float4 *d_lines = nullptr;
  int st = prep_lines(ctx, d_rays, ngrid * nphi, nphi, (long long)nshift_ray * nphi, nphi, 1,
                      nshift_ray, &d_lines, nullptr);
  if (st) return st;
  const long long total = (long long)nshift * nphi * ntheta;
  const long long blocks = (total + 255) / 256;
  reduction_kernel<<<(unsigned)blocks, 256, 0, ctx->stream>>>(
      d_lines, ngrid, nshift_ray, nphi, d_shift, nshift, d_cs, ntheta, d_out, ctx->d_counter);
  ctx->launches++;
  return check_launch(ctx, "reduction_kernel");
}

int adjoint_forward(wrt_ctx *ctx, const double *d_radon, int nphi, int ntheta, int nshift,
                    const double4 *d_dirw, const double4 *h_dirw, int n, double *d_out) {
  // lines (iphi, itheta): element is at d_radon[(is*nphi + iphi)*ntheta + itheta]
  float4 *d_lines = nullptr;
  const int ndir = nphi * ntheta;
  int st = prep_lines(ctx, d_radon, ndir, ndir, 0, (long long)ndir, 1, nshift, &d_lines, d_dirw);
  if (st) return st;
  cudaError_t e = launch_adjoint(ctx->stream, d_lines, ndir, nshift, h_dirw, n, d_out,
                                 &ctx->launches);
  return e == cudaSuccess ? WRT_OK : cuda_fail(ctx, e, "adjoint_kernel");
}

}  // namespace wrt
