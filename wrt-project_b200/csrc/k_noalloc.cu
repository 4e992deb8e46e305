// k_noalloc.cu -- the adjoint (backprojection) without any device allocation.
//
// wrt_radon3d_adjoint allocates its working memory (spline tables, direction
// table, Gauss-Legendre nodes) with cudaMalloc on every call.  Some callers
// cannot allow that: programs that hand all device memory to their own
// allocator or reserve it up front (a cudaMalloc then fails, or fragments the
// reservation), and latency-critical pipelines that forbid allocation after
// start-up because cudaMalloc/cudaFree synchronise the whole device and stall
// every other stream.  wrt_radon3d_adjoint_static serves them: the caller
// passes device input and output buffers, and all working memory lives in one
// file-scope __device__ array of fixed size (kScratchBytes below), which every
// GPU that loads this library holds until the process exits.
//
// Limits (checked, WRT_ERR_INVALID_ARGUMENT with a message otherwise):
//   nphi * ntheta <= 16384 directions, ntheta <= 1024, 3 <= nshift <= 2048,
//   nphi * ntheta * nshift <= 262144 spline samples.
// The scratch array is shared by every call on a device and keeps the last
// call's contents; every call writes all of it that it reads before reading,
// so nothing has to start at zero.  Calls whose GPU work overlaps (different
// streams, or different host threads) race on the array: order them.
#include <math.h>

#include <mutex>

#include "wrt_internal.cuh"

namespace wrt {
int launch_gl_nodes(cudaStream_t stream, int n, double *d_x, double *d_w);
int launch_adjoint_lines(cudaStream_t stream, const double *d_radon, int ndir, int nshift,
                         const double *d_cp, const double *d_den, double *d_scratch,
                         float4 *d_lines, const double4 *d_dirw);
int launch_adjoint(cudaStream_t stream, const float4 *d_lines, int ndir, int ntheta, int nshift,
                   const double4 *d_dirw, int n, double *d_out);
}  // namespace wrt

namespace {

constexpr int kMaxDirs = 16384, kMaxTheta = 1024, kMaxShift = 2048;
constexpr long long kMaxEntries = 262144;  // nphi * ntheta * nshift

constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kOffX = 0;
constexpr size_t kOffW = align256(kOffX + sizeof(double) * kMaxTheta);
constexpr size_t kOffCp = align256(kOffW + sizeof(double) * kMaxTheta);
constexpr size_t kOffDen = align256(kOffCp + sizeof(double) * kMaxShift);
constexpr size_t kOffDirw = align256(kOffDen + sizeof(double) * kMaxShift);
constexpr size_t kOffM = align256(kOffDirw + sizeof(double4) * kMaxDirs);
constexpr size_t kOffLines = align256(kOffM + sizeof(double) * kMaxEntries);
constexpr size_t kScratchBytes = align256(kOffLines + sizeof(float4) * kMaxEntries);

// The working memory (about 6.6 MB).  In host code this name is a host-side
// stand-in, not a device address: host code must use the address returned by
// cudaGetSymbolAddress (scratch_base below).
static __device__ __align__(256) unsigned char g_adjoint_scratch[kScratchBytes];

// Line-independent elimination coefficients of the uniform-knot natural
// spline system M_{i-1} + 4 M_i + M_{i+1} = rhs_i (same values as the host
// computation in k_spline.cu).
__global__ void spline_coef_kernel(int ns, double *cp, double *den) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  cp[0] = 0.0;
  den[0] = 1.0;
  cp[ns - 1] = 0.0;
  den[ns - 1] = 1.0;
  for (int i = 1; i + 1 < ns; ++i) {
    den[i] = 4.0 - (i > 1 ? cp[i - 1] : 0.0);
    cp[i] = 1.0 / den[i];
  }
}

// dirw[ip*ntheta + it] = (sin t cos p, sin t sin p, cos t, dphi * w_t),
// t = acos(GL node), p = 2 pi ip / nphi
// (backprojection/C/src/init.c:222-245 and integral.c:11-18).
__global__ void direction_weights_kernel(int nphi, int ntheta, const double *x, const double *w,
                                         double4 *dirw) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= nphi * ntheta) return;
  const int ip = d / ntheta, it = d - ip * ntheta;
  const double dphi = (2 * WRT_PI) / nphi;
  const double p = dphi * ip, t = acos(x[it]);
  dirw[d] = make_double4(sin(t) * cos(p), sin(t) * sin(p), cos(t), dphi * w[it]);
}

std::mutex g_setup_mutex;
void *g_scratch_base[64] = {nullptr};

// Device address of the scratch array for the current device; looked up once
// per device, with that device current.
int scratch_base(wrt_ctx *ctx, unsigned char **base) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (ctx->device < 0 || ctx->device >= 64)
    return wrt::fail(ctx, WRT_ERR_INVALID_ARGUMENT, "device ordinal out of range");
  if (!g_scratch_base[ctx->device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_adjoint_scratch);
    if (e != cudaSuccess || !p) return wrt::cuda_fail(ctx, e, "cudaGetSymbolAddress(adjoint scratch)");
    g_scratch_base[ctx->device] = p;
  }
  *base = static_cast<unsigned char *>(g_scratch_base[ctx->device]);
  return WRT_OK;
}

}  // namespace

extern "C" int wrt_radon3d_adjoint_static(wrt_ctx *ctx, const double *d_radon, int nphi,
                                          int ntheta, int nshift, int ngrid, double *d_out) {
  if (!ctx) return WRT_ERR_INVALID_ARGUMENT;
  if (!d_radon || !d_out || nphi < 1 || ntheta < 1 || nshift < 3 || ngrid < 1 || ngrid > 4096)
    return wrt::fail(ctx, WRT_ERR_INVALID_ARGUMENT, "radon3d_adjoint_static: bad arguments");
  const long long ndir = (long long)nphi * ntheta;
  if (ndir > kMaxDirs || ntheta > kMaxTheta || nshift > kMaxShift || ndir * nshift > kMaxEntries)
    return wrt::fail(ctx, WRT_ERR_INVALID_ARGUMENT,
                     "radon3d_adjoint_static: nphi=%d ntheta=%d nshift=%d exceeds the static "
                     "working memory (nphi*ntheta <= %d, ntheta <= %d, nshift <= %d, "
                     "nphi*ntheta*nshift <= %lld)",
                     nphi, ntheta, nshift, kMaxDirs, kMaxTheta, kMaxShift, kMaxEntries);
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return wrt::cuda_fail(ctx, e, "cudaSetDevice");
  unsigned char *base = nullptr;
  int st = scratch_base(ctx, &base);
  if (st) return st;
  double *x = reinterpret_cast<double *>(base + kOffX);
  double *w = reinterpret_cast<double *>(base + kOffW);
  double *cp = reinterpret_cast<double *>(base + kOffCp);
  double *den = reinterpret_cast<double *>(base + kOffDen);
  double4 *dirw = reinterpret_cast<double4 *>(base + kOffDirw);
  double *M = reinterpret_cast<double *>(base + kOffM);
  float4 *lines = reinterpret_cast<float4 *>(base + kOffLines);
  cudaStream_t s = ctx->stream;
  st = wrt::launch_gl_nodes(s, ntheta, x, w);
  if (!st) {
    spline_coef_kernel<<<1, 1, 0, s>>>(nshift, cp, den);
    direction_weights_kernel<<<(int)((ndir + 127) / 128), 128, 0, s>>>(nphi, ntheta, x, w, dirw);
    st = cudaGetLastError() == cudaSuccess ? WRT_OK : WRT_ERR_CUDA;
  }
  if (!st) st = wrt::launch_adjoint_lines(s, d_radon, (int)ndir, nshift, cp, den, M, lines, dirw);
  if (!st) st = wrt::launch_adjoint(s, lines, (int)ndir, ntheta, nshift, dirw, ngrid, d_out);
  ctx->launches += 5;
  if (st) return wrt::fail(ctx, WRT_ERR_CUDA, "radon3d_adjoint_static: launch failed");
  return WRT_OK;
}
