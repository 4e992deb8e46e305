// k_noalloc.cu -- the adjoint (backprojection) without any device allocation.
//
// wrt_radon3d_adjoint allocates its working memory (spline tables, direction
// table) with cudaMalloc on every call.  Some callers cannot allow that:
// programs that hand all device memory to their own allocator or reserve it
// up front (a cudaMalloc then fails, or fragments the reservation), and
// latency-critical pipelines that forbid allocation after start-up because
// cudaMalloc/cudaFree synchronise the whole device and stall every other
// stream.  wrt_radon3d_adjoint_static serves them: the caller passes device
// input and output buffers, and all working memory lives in one file-scope
// __device__ array of fixed size (kScratchBytes below), which every GPU that
// loads this library holds until the process exits.
//
// Limits (checked, WRT_ERR_INVALID_ARGUMENT with a message otherwise):
//   nphi * ntheta <= 16384 directions, ntheta <= 1024, 3 <= nshift <= 2048,
//   nphi * ntheta * nshift <= 262144 spline samples.
// The small tables (direction weights, spline elimination coefficients) are
// computed on the host by the same code as wrt_radon3d_adjoint's, Gauss-
// Legendre nodes included, and copied into the array from host memory, so the
// two entry points give bitwise the same volume.  The array is shared by every
// call on a device and keeps the last call's contents; every call writes all
// of it that it reads before reading, so nothing has to start at zero.  Calls
// whose GPU work overlaps (different streams, or different host threads) race
// on the array: order them.
#include <math.h>

#include <mutex>
#include <vector>

#include "wrt_internal.cuh"

namespace wrt {
cudaError_t launch_adjoint_lines(cudaStream_t stream, const double *d_radon, int ndir, int nshift,
                                 const double *d_cp, const double *d_den, double *d_scratch,
                                 float4 *d_lines, const double4 *d_dirw);
}  // namespace wrt

namespace {

constexpr int kMaxDirs = 16384, kMaxTheta = 1024, kMaxShift = 2048;
constexpr long long kMaxEntries = 262144;  // nphi * ntheta * nshift

constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kOffCp = 0;
constexpr size_t kOffDen = align256(kOffCp + sizeof(double) * kMaxShift);
constexpr size_t kOffDirw = align256(kOffDen + sizeof(double) * kMaxShift);
constexpr size_t kOffM = align256(kOffDirw + sizeof(double4) * kMaxDirs);
constexpr size_t kOffLines = align256(kOffM + sizeof(double) * kMaxEntries);
constexpr size_t kScratchBytes = align256(kOffLines + sizeof(float4) * kMaxEntries);

// The working memory (about 6.8 MB).  In host code this name is a host-side
// stand-in, not a device address: host code must use the address returned by
// cudaGetSymbolAddress (scratch_base below).
static __device__ __align__(256) unsigned char g_adjoint_scratch[kScratchBytes];

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

namespace wrt {
// Forgets the cached address of the scratch array on a device.  Called when a
// context is created: a device reset before it would have moved the array.
void noalloc_forget_device(int device) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (device >= 0 && device < 64) g_scratch_base[device] = nullptr;
}
}  // namespace wrt

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
  double *cp = reinterpret_cast<double *>(base + kOffCp);
  double *den = reinterpret_cast<double *>(base + kOffDen);
  double4 *dirw = reinterpret_cast<double4 *>(base + kOffDirw);
  double *M = reinterpret_cast<double *>(base + kOffM);
  float4 *lines = reinterpret_cast<float4 *>(base + kOffLines);
  // host tables: the sphere grid (radon_grid/src/init.c:165-189, GL nodes by
  // the GPU generator's own code), the direction weights and the natural
  // spline elimination coefficients, exactly as wrt_radon3d_adjoint builds them
  std::vector<double> x(ntheta), w(ntheta), theta(ntheta), phi(nphi);
  wrt::gauss_legendre_host(ntheta, x.data(), w.data());
  for (int i = 0; i < ntheta; ++i) theta[i] = acos(x[i]);
  const double dphi = (2 * M_PI) / nphi;
  for (int i = 0; i < nphi; ++i) phi[i] = dphi * i;
  std::vector<double4> h_dirw((size_t)ndir);
  wrt::adjoint_directions(nphi, ntheta, nshift, phi.data(), theta.data(), w.data(), h_dirw.data());
  std::vector<double> coef(2 * (size_t)nshift);
  double *h_cp = coef.data(), *h_den = coef.data() + nshift;
  wrt::spline_coefficients(nshift, h_cp, h_den);
  // copies from pageable host memory return once the data is staged, so the
  // vectors may go out of scope before the copies land
  cudaStream_t s = ctx->stream;
  e = cudaMemcpyAsync(dirw, h_dirw.data(), sizeof(double4) * (size_t)ndir,
                      cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(cp, h_cp, sizeof(double) * nshift, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(den, h_den, sizeof(double) * nshift, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return wrt::cuda_fail(ctx, e, "radon3d_adjoint_static: table upload");
  e = wrt::launch_adjoint_lines(s, d_radon, (int)ndir, nshift, cp, den, M, lines, dirw);
  if (e != cudaSuccess) return wrt::cuda_fail(ctx, e, "radon3d_adjoint_static: spline_prep_kernel");
  ctx->launches++;
  e = wrt::launch_adjoint(s, lines, (int)ndir, nshift, h_dirw.data(), ngrid, d_out,
                          &ctx->launches);
  if (e != cudaSuccess) return wrt::cuda_fail(ctx, e, "radon3d_adjoint_static: adjoint_kernel");
  return WRT_OK;
}
