// wrt_internal.cuh -- shared declarations of libwrt (not part of the ABI).
//
// Numerics contract of every volume sampler in this library
// ---------------------------------------------------------
// The reference samples in FP64 with two discontinuous rules:
//   * zero_interp (radon_grid/src/interp.c:63-87): value of the cell
//     floor((x+1)/(2/n)), clamped to n-1;
//   * cube_trilinear_interp (radon_grid/src/interp.c:25-60): cell index from
//     (int)((x+1)/delta) but fraction from fmod(x+1, delta)/delta, which
//     disagree when x+1 sits within one rounding of a multiple of delta, plus
//     the upper-boundary clamp, plus the |x| > 1 cut-off.
// Lattice points produced by the reference's own grids often sit exactly on
// such boundaries (axis-aligned directions, z-slices on grid nodes), so an
// FP32 sampler alone would pick different cells there.  Every kernel here
// therefore computes the cell coordinate q = (x+1)/delta in FP32 and, when
// frac(q) lies within a guard band g of 0 or 1 (g is several times the
// worst FP32 error of q), re-evaluates that one sample with the reference's
// FP64 arithmetic (exact_* below: same operations in the same order, no
// fused multiply-add).  Outside the band FP32 and FP64 select the same cell
// and the trilinear value is continuous, so the FP32 result differs from the
// reference only by rounding.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include <unordered_map>
#include <utility>
#include <vector>

#include "../../include/wrt.h"

#define WRT_PI 3.14159265358979323846

// ---------------------------------------------------------------- host side
namespace wrt {
struct HostPool;  // host threads of the staged copies (hostcopy.cu)
}

struct wrt_ctx {
  int device = 0;
  size_t budget = 0;      // 0 = unlimited
  size_t in_use = 0;      // bytes held through ctx_alloc
  uint64_t launches = 0;  // kernels launched through this context
  cudaStream_t stream = nullptr;
  int sm_count = 0;
  char err[512] = {0};
  // measurement helpers (api.cu)
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  void *flush_buf = nullptr;
  size_t flush_bytes = 0;
  unsigned long long *d_counter = nullptr;  // non-null while counting samples
  std::unordered_map<void *, size_t> user_allocs;  // wrt_device_alloc sizes
  // staged plane kernel (k_staged.cu): request descriptors, item counter and
  // the work-item lists of the geometries seen so far
  void *staged_req = nullptr;
  size_t staged_req_bytes = 0;
  int *staged_next = nullptr;
  void *staged_cache = nullptr;
  int staged_config = -1;  // tile configuration (-1: default), set by the autotuner
  void *batch_slot = nullptr;  // BatchSlot of wrt_radon_forward_batch (batch.cu)
  // grow-only working buffers, one per role (wrt::ws_get), freed with the
  // context: warm calls of the same or smaller sizes allocate nothing
  void *ws[8] = {};
  size_t ws_bytes[8] = {};
  void *fft_plans = nullptr;  // spectral Laplacian plans (k_laplace.cu)
  // the volume and sphere grid of the last drop-in (host-array) call, kept
  // for the next call of the same sizes
  wrt_volume *dropin_vol = nullptr;
  wrt_grid *dropin_grid = nullptr;
  // host-array copies (hostcopy.cu): two pinned chunk buffers, the events
  // that end their DMA, and the host threads that fill and drain them
  void *pin[2] = {};
  cudaEvent_t pin_ev[2] = {};
  wrt::HostPool *host_pool = nullptr;
  unsigned long long large_copies = 0;  // host-array copies of 1 MB or more so far
};

namespace wrt {

// status helpers (api.cu)
int fail(wrt_ctx *ctx, int status, const char *fmt, ...);
int cuda_fail(wrt_ctx *ctx, cudaError_t e, const char *what);
int ctx_alloc(wrt_ctx *ctx, void **p, size_t bytes);
void ctx_free(wrt_ctx *ctx, void *p, size_t bytes);
int check_launch(wrt_ctx *ctx, const char *what);
// Working buffer of a role, at least `bytes` long (grown after the context's
// stream has drained; contents are not kept).
enum WsRole { WS_STAGE, WS_IN, WS_OUT, WS_LINES, WS_SPLINE, WS_COEF, WS_TABLE, WS_FFT, WS_ROLES };
int ws_get(wrt_ctx *ctx, int role, size_t bytes, void **p);
// Copies between caller (pageable) host arrays and the device, through the
// context's pinned chunk buffers and host threads (hostcopy.cu): the upload
// returns once the caller's array has been read (the DMA may still run, in
// stream order); the download returns with the data in place.
int h2d_staged(wrt_ctx *ctx, void *dst, const void *src, size_t bytes, const char *what);
// FP64 host values rounded to FP32 (to nearest) while they are staged.
int h2d_staged_rounded(wrt_ctx *ctx, float *dst, const double *src, size_t count,
                       const char *what);
int d2h_staged_sync(wrt_ctx *ctx, void *dst, const void *src, size_t bytes, const char *what);
void pinned_release(wrt_ctx *ctx);
void host_pool_destroy(HostPool *p);

// Host-side FP64 geometry, computed with the host libm exactly as the
// reference computes it (radon_grid/src/integral.c:10-36).
void plane_directions(int nphi, const double *phi, int ntheta, const double *theta,
                      double *dir9 /* [nphi*ntheta][9]: normal, v1, v2 */);
// Sphere grid (phi, theta, theta weights, shift) with GL nodes from the GPU.
int sphere_grid(wrt_ctx *ctx, int nphi, int ntheta, int nshift, double *phi,
                double *theta, double *theta_w, double *shift);
int gauss_legendre_device(wrt_ctx *ctx, int n, double *x_host, double *w_host);
// The same nodes computed on the host (bit-identical to the GPU's).
void gauss_legendre_host(int n, double *x, double *w);
// Backprojection direction table [nphi*ntheta]: (omega / h, dphi * w_theta),
// h = 2/(nshift-1).
void adjoint_directions(int nphi, int ntheta, int nshift, const double *phi, const double *theta,
                        const double *theta_w, double4 *dirw);

// Volume preparation kernels (k_volume.cu).
// d_stats[0]: largest |x|^2 of a non-zero node, d_stats[1]: max |v| (float bits)
int volume_from_f32(wrt_ctx *ctx, const float *d_src, int n, float *d_vol,
                    unsigned int *d_stats);
int volume_pairs(wrt_ctx *ctx, const float *d_vol, int n, float2 *d_pairs, int pitch);
// Cell octets: 2 (n-1)^3 float4, the eight corners of every cell.
int volume_octets(wrt_ctx *ctx, const float *d_vol, int n, float4 *d_oct);
// BF16 storage: values rounded to bfloat16 (nearest even); statistics of the
// rounded values; layer pairs as bf16x2.
int volume_to_bf16(wrt_ctx *ctx, const float *d_vol, int n, __nv_bfloat16 *d_vol16,
                   unsigned int *d_stats);
int volume_pairs_bf16(wrt_ctx *ctx, const __nv_bfloat16 *d_vol16, int n,
                      __nv_bfloat162 *d_pairs, int pitch);

// Plane kernels (k_plane.cu).
struct PlaneJob {
  const float *vol;      // n^3 floats, v[ix][iy][iz]
  const float2 *pairs;   // layer pairs [iz][iy][pitch] (staged kernel) or null
  int n, pitch;
  const double *dir;     // [ndir][9] FP64 directions
  const double *shift;   // [nshift] FP64 shifts
  int ndir, nshift;
  int L;                 // lattice half extent
  int sampler;
  const unsigned int *r2bits;  // device: largest |x|^2 of a non-zero node (float bits)
  double margin;         // crop radius = sqrt(r2) + margin (>= the sampler's reach)
  double *out;           // [nshift][ndir]
  unsigned long long *counter;  // optional: samples evaluated
  const float4 *oct;    // cell octets of the volume (rotated frames), or null
};
int plane_forward_plain(wrt_ctx *ctx, const PlaneJob &job);
// z-major copy layers[iz][iy][ix] of an FP32 volume (the nearest sampler's
// staged cell layers).
int volume_layers(wrt_ctx *ctx, const float *d_vol, int n, float *d_layers);
int plane_transpose(wrt_ctx *ctx, const PlaneJob &job, const double *d_g, double *d_vol64);

// Staged plane kernel (k_staged.cu).
struct StagedReq {
  const void *pairs;       // layer pairs [iz][y][pitch2]: float2 (FP32) or bf16x2 (BF16 storage)
  const void *vol;         // reference layout, for guard-band samples: float or bf16
  const double *dir;       // [ndir][9] FP64 directions
  const float *dir32;      // [ndir][8]: normal, v1, v2.x, v2.y (unscaled) FP32
  const double *shift;     // [nshift]
  const float *shift32;    // [nshift]
  unsigned long long *acc; // [nshift][ndir] fixed-point accumulators (the output buffer)
  int n, pitch2, qpitch, tile_h, ndir, nshift, L;
  int storage;             // wrt_storage of pairs / vol
  int nearest;             // 1: zero_interp on the n^3 cells; pairs = z-major cell layers
                           // [iz][y][pitch2] (FP32), cells of tile_h rows staged per item
  float guard, crop_r2;
  double scale;            // fixed-point scale 2^k
};
struct StagedItem {
  int req, layer, tile, dir0, ndir;
};
struct StagedConfig {
  int threads, group, shifts_per_lane;
};
extern const StagedConfig kStagedConfigs[];
extern const int kNumStagedConfigs;
int staged_smem_bytes(int n, int *tile_h, int *qpitch);
// The nearest sampler's tile: tile_h cell rows of (n + 4) FP32 cells, pitch
// qpitch floats; bytes of the tile or -1.
int staged_smem_bytes_nearest(int n, int *tile_h, int *qpitch);
// Guard band (in cells) of the staged kernel's x / y cell fractions.  Cell
// coordinates are held relative to the centre cell C = (n-1)/2 (rounded
// down); q' = fma(j, du, q0') with q0' and du rounded once from FP64, so
// |q' - q'_exact| <= 0.5 ulp(q0') + |j| |du| 2^-24 + 0.5 ulp(q') where
// |q0'| <= sqrt(crop_r2) h + 1 (the row's j = 0 point lies in the crop
// ball), |q'| <= h + 3 for every sample evaluated, |du| < 1/2 and |j| <= L.
// The band is twice that bound, so every sample whose exact coordinate is on
// a cell boundary (where the reference's cell index and fraction can
// disagree) or on a cube face lies inside it.  Host and device compute it
// alike (the batched path sets it on the device from the volume statistics).
__host__ __device__ inline float staged_guard(int n, int L, float crop_r2, bool nearest = false) {
  const double h = 0.5 * (nearest ? n : n - 1);  // cells per unit length
  const double ulp = 1.0 / 8388608.0;  // 2^-23 relative
  const double bound = 0.5 * ulp * (sqrt((double)crop_r2) * h + 1.0) +
                       0.5 * ulp * (h + 3.0) + 0.5 * ulp * 0.5 * L;
  return (float)(2.0 * bound) + 1e-7f;
}
constexpr int kStagedDirChunk = 512;  // directions per work item
// Staged tile budget (bytes of dynamic shared memory): 227 KB per CTA minus
// the per-warp row tables and guard-band queues (kStagedWarpSmemQuads float4
// per warp, 48 KB at 1024 threads) and a few static words.
constexpr int kStagedSmemMax = 168 * 1024;
constexpr int kStagedWarpSmemQuads = 96;
int plane_staged_launch(wrt_ctx *ctx, cudaStream_t stream, const StagedReq *d_reqs,
                        const StagedItem *d_items, const int *d_nitems, int max_smem,
                        int *d_next);
// The nearest sampler's staged launch (one request; default tile shape).
int plane_staged_launch_nearest(wrt_ctx *ctx, cudaStream_t stream, const StagedReq *d_reqs,
                                const StagedItem *d_items, const int *d_nitems, int max_smem,
                                int *d_next);
int plane_finalize(wrt_ctx *ctx, double *out, long long count, double factor);
// Work items of one request (layer x y-tile x direction chunk) with their
// estimated cost (staged voxels inside the crop radius x directions x weight).
void staged_items_costed(int req, int n, int tile_h, float crop_r2, int ndir, int dir_chunk,
                         double weight, std::vector<std::pair<double, StagedItem>> &out,
                         bool nearest = false);
void staged_items(int req, int n, int tile_h, float crop_r2, int ndir, int dir_chunk,
                  std::vector<StagedItem> &out, bool nearest = false);
int staged_items_cached(wrt_ctx *ctx, int n, int tile_h, float crop_r2, int ndir,
                        StagedItem **d_items, const int **d_nitems, int *nitems,
                        bool nearest = false);
int staged_scratch(wrt_ctx *ctx, size_t req_bytes);
void staged_release(wrt_ctx *ctx);

// Ray kernels (k_ray.cu).
struct RayJob {
  const float *vol;
  int n;
  int nslices, nshift, nphi;
  const double *trig;   // [nphi][4]: cos phi, sin phi, cos(phi+pi/2), sin(phi+pi/2)
  const double *shift;  // [nshift]
  double frame[9];      // row-major rotation of the sample points (has_frame)
  int has_frame;        // 0: the reference's z-slices
  const unsigned int *r2bits;
  double margin;
  double *out;          // [nslices][nshift][nphi]
  const float2 *pairs;  // layer pairs [n-1][n][pitch] of the volume, or null
  int pitch;
  unsigned long long *counter;  // optional: samples evaluated
  const float4 *oct;    // cell octets of the volume (rotated frames), or null
};
// Batches (batch.cu): many requests in one launch of a captured CUDA graph.
// The batch is one table in device memory (layout BatchLayout), uploaded by
// the graph's first node from a pinned host mirror; every kernel of the graph
// reads its work from the table, so one captured graph serves every batch.
constexpr int kBatchMaxFwd = 256;  // forward requests per batch
constexpr int kBatchMaxAdj = 256;  // adjoint requests per batch
struct FwdAux {                    // per forward request, beside its StagedReq
  const float *vol;                // FP32 volume, reference order
  float2 *pairs;                   // layer pairs (built in the launch when prep)
  unsigned int *stats;             // [0] r2 bits, [1] max |v| bits (computed when prep)
  long long nout;                  // nshift * ndir
  double factor;                   // delta^2 / scale, written by the launch
  int n, pitch, L, prep;           // prep: build stats and pairs in this launch
};
struct AdjReq {                    // one backprojection
  const double *radon;             // [is][iphi][itheta]
  const double4 *dirw;             // [ndir]: omega / h, dphi * w_theta (FP64)
  const double *cp, *den;          // spline elimination coefficients [nshift]
  double *scratch;                 // [ndir][nshift]
  float4 *lines;                   // [ndir][nshift - 1]
  double *out;                     // [iz][ix][iy]
  const double4 *h_dirw;           // host copy of dirw (launch parameters)
  int ndir, ntheta, nshift, n;
};
constexpr int kBatchMaxRay = 64;   // ray-transform requests per batch
constexpr int kBatchMaxRed = 64;   // reduction requests per batch
struct RedReq {                    // one ray-to-Radon reduction
  const double *rays;              // [iz][is][iphi]
  const double *coef;              // spline elimination coefficients: cp[ns_ray], den[ns_ray]
  double *scratch;                 // [ngrid*nphi][ns_ray]
  float4 *lines;                   // [ngrid*nphi][ns_ray - 1]
  const double *shift;             // [nshift]
  const double *cs;                // [ntheta][2]: cos, sin theta
  double *out;                     // [is][iphi][itheta]
  int ngrid, ns_ray, nphi, nshift, ntheta, pad;
};
struct BatchHeader {
  int nfwd, nadj, nitems, nray, nred, pad[3];
};
constexpr size_t batch_align(size_t x) { return (x + 255) & ~(size_t)255; }
struct BatchLayout {
  static constexpr size_t fwd = 256;
  static constexpr size_t aux = batch_align(fwd + sizeof(StagedReq) * kBatchMaxFwd);
  static constexpr size_t adj = batch_align(aux + sizeof(FwdAux) * kBatchMaxFwd);
  static constexpr size_t ray = batch_align(adj + sizeof(AdjReq) * kBatchMaxAdj);
  static constexpr size_t red = batch_align(ray + sizeof(RayJob) * kBatchMaxRay);
  static constexpr size_t items = batch_align(red + sizeof(RedReq) * kBatchMaxRed);
  static size_t bytes(size_t nitems) { return items + sizeof(StagedItem) * nitems; }
};
// Host-side description of one batch.
struct BatchBuilder {
  std::vector<StagedReq> fwd;
  std::vector<FwdAux> aux;
  std::vector<AdjReq> adj;
  std::vector<RayJob> ray;
  std::vector<RedReq> red;
  std::vector<std::pair<double, StagedItem>> items;  // cost, item
  void clear() {
    fwd.clear();
    aux.clear();
    adj.clear();
    ray.clear();
    red.clear();
    items.clear();
  }
};
// One reusable launch slot: pinned + device tables and the captured graph.
struct BatchSlot {
  wrt_ctx *ctx = nullptr;
  cudaStream_t stream = nullptr;
  char *h_table = nullptr, *d_table = nullptr;
  size_t cap = 0;  // table bytes
  int *d_next = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphNode_t copy_node = nullptr;
  cudaEvent_t done = nullptr;
  int config = -2;
  bool counting = false, launched = false;
};
// Adds a forward request (staged kernel) to the builder: its descriptor, its
// auxiliary record and its work items.  crop_items: crop radius^2 used to
// generate the items (3 covers the whole cube).
void batch_add_forward(BatchBuilder &b, const StagedReq &req, const FwdAux &aux,
                       float crop_items);
int batch_slot_init(wrt_ctx *ctx, BatchSlot *slot, cudaStream_t stream);
// Waits for the slot's previous launch, writes the table, launches the graph.
int batch_slot_launch(BatchSlot *slot, BatchBuilder &b);
void batch_slot_release(BatchSlot *slot);
// Fills a StagedReq / FwdAux pair for a volume already on the device.
void staged_request(int n, int pitch, int ndir, int nshift, int L, int storage,
                    const void *pairs, const void *vol, const double *dir, const float *dir32,
                    const double *shift, const float *shift32, double *out, StagedReq *r);

int ray_forward(wrt_ctx *ctx, const RayJob &job);
// Host tables of a ray job (ray_grid/src/init.c:163-176, integral.c:16-24):
// tab[0..nshift) the shifts, then [nphi][4] cos phi, sin phi, cos(phi+pi/2),
// sin(phi+pi/2).
void ray_tables(int nshift, int nphi, double *tab);
// Device tables of a grid: FP64 directions [ndir][9] and shifts [nshift].
void grid_tables(const wrt_grid *g, const double **dir, const double **shift);
// True when a 3x3 frame is the identity (the reference's z-slices).
bool identity_frame(const double *frame);
// Reach of the trilinear sampler around a lattice point (one cell diagonal).
double trilinear_margin(int n);
// Line-independent elimination coefficients of the natural cubic spline on
// ns uniform knots: cp[ns], den[ns].
void spline_coefficients(int ns, double *cp, double *den);

// Spectral Laplacian (k_laplace.cu) of an n^3 device volume into d_out, and
// the release of the context's FFT plans.
int spectral_laplacian(wrt_ctx *ctx, const double *d_in, int n, double period, double *d_out);
void laplace_release(wrt_ctx *ctx);

// Allocation-free backprojection (k_noalloc.cu): drops the cached device
// address of its working array on a device (a new context may follow a reset).
void noalloc_forget_device(int device);

// Shared-memory bandwidth microbenchmark (k_probe.cu).
int smem_bandwidth(wrt_ctx *ctx, double *bytes_per_s);

// Spline / reduction / adjoint kernels (k_spline.cu).
int reduction_forward(wrt_ctx *ctx, const double *d_rays, int ngrid, int nshift_ray,
                      int nphi, const double *d_shift, int nshift,
                      const double *d_cs /* [ntheta][2]: cos, sin theta */, int ntheta,
                      double *d_out);
// d_dirw / h_dirw: the same direction table [nphi*ntheta] (omega/h, dphi*w) on
// the device (spline weights) and on the host (per-launch constants).
int adjoint_forward(wrt_ctx *ctx, const double *d_radon, int nphi, int ntheta, int nshift,
                    const double4 *d_dirw, const double4 *h_dirw, int n, double *d_out);
// The backprojection launches over prepared adjoint lines [ndir][nshift-1] on a
// stream (one launch per kAdjDirsPerLaunch directions; *launches counts them).
cudaError_t launch_adjoint(cudaStream_t stream, const float4 *d_lines, int ndir, int nshift,
                           const double4 *h_dirw, int n, double *d_out, uint64_t *launches);

}  // namespace wrt

// ------------------------------------------ shared by host and device code
namespace wrt {

// Scale 2^k of the staged kernel's 64-bit fixed-point plane sums: |row sum|
// <= maxabs * 2L and |plane sum| <= maxabs * (2L+1)^2, so 2^k <= 2^61 / that
// bound keeps every sum below 2^61 in magnitude.  Written with frexp/ldexp
// only (exact on host and device), so a request gets the same scale whether
// the host or a kernel computes it.
__host__ __device__ inline double fixed_point_scale(float maxabs, int L) {
  if (!(maxabs > 0.0f) || !(maxabs <= 3.4e38f)) return 1.0;
  const double bound = (double)maxabs * (2.0 * L + 1.0) * (2.0 * L + 1.0);
  int e = 0;
  const double m = frexp(bound, &e);     // bound = m 2^e, m in [1/2, 1)
  const int lg = (m == 0.5) ? e - 1 : e;  // ceil(log2(bound))
  int k = 61 - lg;
  k = k < -200 ? -200 : (k > 200 ? 200 : k);
  return ldexp(1.0, k);
}

// Squared crop radius of the trilinear sampler for a volume whose non-zero
// nodes lie within sqrt(r2) of the origin: every lattice point farther than
// sqrt(r2) plus one cell diagonal of the node grid has eight zero corners.
// Correctly rounded operations only (same value on host and device).
__host__ __device__ inline float trilinear_crop_r2(float r2, int n) {
  const double h = 2.0 / (n - 1);
  const double rc = sqrt((double)r2) + (sqrt(3.0) * h + 1e-6);
  return (float)fmin(rc * rc * (1.0 + 1e-6), 3.0 + 1e-5);
}

// The same for the nearest sampler: a lattice point farther than sqrt(r2)
// plus the margin of the plain kernel's nearest crop (two cell diagonals of
// the cell grid and one of the node grid) lies in a zero cell.
__host__ __device__ inline float nearest_crop_r2(float r2, int n) {
  const double rc = sqrt((double)r2) + (sqrt(3.0) * (4.0 / n + 2.0 / (n - 1)) + 1e-6);
  return (float)fmin(rc * rc * (1.0 + 1e-6), 3.0 + 1e-5);
}

}  // namespace wrt

// ------------------------------------------------------------ device side
namespace wrtd {

// Reference arithmetic, FP64, no contraction (radon_grid/src/interp.c:3-60).
__device__ __forceinline__ double lin64(double t, double a, double b) {
  return __dadd_rn(__dmul_rn(__dsub_rn(1.0, t), a), __dmul_rn(t, b));
}

__device__ __forceinline__ float ldv(const float *v, int n, int ix, int iy, int iz) {
  return __ldg(v + ((size_t)ix * n + iy) * n + iz);
}
__device__ __forceinline__ float ldv(const __nv_bfloat16 *v, int n, int ix, int iy, int iz) {
  return __bfloat162float(__ldg(v + ((size_t)ix * n + iy) * n + iz));
}

// fmod(x, y) for x >= 0, y > 0 and x / y < 2^52: the exact remainder x - n y,
// n = trunc(x / y).  The quotient estimate from the rounded division is off
// by at most one; a single fused multiply-add then gives x - n y exactly
// (the true remainder is representable), so the result equals fmod's.
__device__ __forceinline__ double exact_rem(double x, double y) {
  double n = trunc(__ddiv_rn(x, y));
  double r = fma(-n, y, x);
  if (r < 0.0) {
    n -= 1.0;
    r = fma(-n, y, x);
  } else if (r >= y) {
    n += 1.0;
    r = fma(-n, y, x);
  }
  return r;
}

// cube_trilinear_interp, radon_grid/src/interp.c:25-60.
template <typename T>
static __device__ __noinline__ double exact_trilinear(const T *v, int n, double x, double y,
                                                      double z) {
  if ((fabs(x) > 1.0) || (fabs(y) > 1.0) || (fabs(z) > 1.0)) return 0.0;
  const double delta = __ddiv_rn(2.0, (double)(n - 1));
  const double x1 = __dadd_rn(x, 1.0), y1 = __dadd_rn(y, 1.0), z1 = __dadd_rn(z, 1.0);
  int ix = (int)__ddiv_rn(x1, delta), iy = (int)__ddiv_rn(y1, delta),
      iz = (int)__ddiv_rn(z1, delta);
  double cx = __ddiv_rn(exact_rem(x1, delta), delta), cy = __ddiv_rn(exact_rem(y1, delta), delta),
         cz = __ddiv_rn(exact_rem(z1, delta), delta);
  if (ix == n - 1) { ix -= 1; cx = 1.0; }
  if (iy == n - 1) { iy -= 1; cy = 1.0; }
  if (iz == n - 1) { iz -= 1; cz = 1.0; }
  double a0 = lin64(cx, ldv(v, n, ix, iy, iz), ldv(v, n, ix + 1, iy, iz));
  double a1 = lin64(cx, ldv(v, n, ix, iy + 1, iz), ldv(v, n, ix + 1, iy + 1, iz));
  double c0 = lin64(cy, a0, a1);
  double b0 = lin64(cx, ldv(v, n, ix, iy, iz + 1), ldv(v, n, ix + 1, iy, iz + 1));
  double b1 = lin64(cx, ldv(v, n, ix, iy + 1, iz + 1), ldv(v, n, ix + 1, iy + 1, iz + 1));
  double c1 = lin64(cy, b0, b1);
  return lin64(cz, c0, c1);
}

// zero_interp, radon_grid/src/interp.c:63-87.
static __device__ __noinline__ double exact_nearest(const float *v, int n, double x, double y,
                                             double z) {
  if ((fabs(x) > 1.0) || (fabs(y) > 1.0) || (fabs(z) > 1.0)) return 0.0;
  const double delta = __ddiv_rn(2.0, (double)n);
  int ix = (int)__ddiv_rn(__dadd_rn(x, 1.0), delta), iy = (int)__ddiv_rn(__dadd_rn(y, 1.0), delta),
      iz = (int)__ddiv_rn(__dadd_rn(z, 1.0), delta);
  if (ix == n) ix -= 1;
  if (iy == n) iy -= 1;
  if (iz == n) iz -= 1;
  return (double)ldv(v, n, ix, iy, iz);
}

// FP32 fast path.  q* are cell coordinates ((x+1)/delta for the sampler's
// delta).  Returns false when the sample must be re-evaluated exactly.
__device__ __forceinline__ bool in_band(float q, float g) {
  float f = q - floorf(q);
  return (f < g) | (f > 1.0f - g);
}

__device__ __forceinline__ float lerp32(float t, float a, float b) { return fmaf(t, b - a, a); }

// Trilinear from the reference-layout volume at FP32 cell coordinates known
// to be outside the guard band and inside [0, n-1].
__device__ __forceinline__ float tri32(const float *__restrict__ v, int n, float qx, float qy,
                                       float qz) {
  float fx = floorf(qx), fy = floorf(qy), fz = floorf(qz);
  float tx = qx - fx, ty = qy - fy, tz = qz - fz;
  const float *p = v + ((size_t)(int)fx * n + (int)fy) * n + (int)fz;
  const size_t sx = (size_t)n * n;
  float c000 = __ldg(p), c001 = __ldg(p + 1), c010 = __ldg(p + n), c011 = __ldg(p + n + 1);
  float c100 = __ldg(p + sx), c101 = __ldg(p + sx + 1), c110 = __ldg(p + sx + n),
        c111 = __ldg(p + sx + n + 1);
  float a0 = lerp32(tx, c000, c100), a1 = lerp32(tx, c010, c110);
  float b0 = lerp32(tx, c001, c101), b1 = lerp32(tx, c011, c111);
  float e0 = lerp32(ty, a0, a1), e1 = lerp32(ty, b0, b1);
  return lerp32(tz, e0, e1);
}

// Squared radius of node (ix, iy, iz) of the node grid x_i = -1 + 2 i/(n-1)
// (radon_grid/src/init.c:120-124), widened by 1e-6 relative, as the volume
// statistics record it (explicit roundings: the same value in every kernel).
__device__ __forceinline__ float node_r2(int ix, int iy, int iz, int n) {
  const double h = 2.0 / (n - 1);
  const double x = __dadd_rn(-1.0, __dmul_rn(h, (double)ix));
  const double y = __dadd_rn(-1.0, __dmul_rn(h, (double)iy));
  const double z = __dadd_rn(-1.0, __dmul_rn(h, (double)iz));
  const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
  return __fmul_rn((float)r2, 1.0f + 1e-6f);
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

}  // namespace wrtd
