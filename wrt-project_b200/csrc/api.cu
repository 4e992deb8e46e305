// api.cu -- the C ABI of libwrt (include/wrt.h).
//
// Each drop-in entry point replaces one reference program's loop nest:
//   wrt_radon_grid       radon_grid/src/radon_grid.c:229-264
//   wrt_ray_grid         ray_grid/src/ray_grid.c:225-262
//   wrt_radon_reduction  radon_reduction/reduction.c:195-235
//   wrt_radon3d_adjoint  radon_inversion/backprojection/C/src/radon3d_ajoint.c:221-260
// Host buffers in, host buffers out; errors come back as wrt_status codes with
// a message in wrt_ctx_last_error (the reference perror()s and exits).
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <new>
#include <vector>

#include "wrt_internal.cuh"

struct wrt_volume {
  wrt_ctx *ctx = nullptr;
  int n = 0;
  float *d_vol = nullptr;          // n^3, v[ix][iy][iz]
  unsigned int *d_stats = nullptr; // [0] largest |x|^2 of a non-zero node, [1] max |v| (float bits)
  float r2 = 3.0f, maxabs = 0.0f;  // host copies of d_stats, read at upload
  float2 *d_pairs = nullptr;       // layer pairs for the staged kernel (built on first use)
  int pitch = 0;
  size_t vol_bytes = 0, pair_bytes = 0;
  bool pairs_valid = false;
  int storage = WRT_STORAGE_F32;        // BF16: d_vol16 / d_pairs16 replace d_vol / d_pairs
  __nv_bfloat16 *d_vol16 = nullptr;     // n^3 bf16 values, v[ix][iy][iz]
  __nv_bfloat162 *d_pairs16 = nullptr;  // layer pairs as bf16x2
  float4 *d_oct = nullptr;              // cell octets (ray transforms in rotated frames)
  size_t oct_bytes = 0;
  bool oct_valid = false;
  float *d_layers = nullptr;            // z-major copy [iz][iy][ix] (nearest sampler)
  bool layers_valid = false;
};

struct wrt_grid {
  wrt_ctx *ctx = nullptr;
  int nphi = 0, ntheta = 0, nshift = 0;
  std::vector<double> phi, theta, w, shift;
  double *d_dir = nullptr;    // [nphi*ntheta][9]
  double *d_shift = nullptr;  // [nshift]
  float *d_dir32 = nullptr;   // [nphi*ntheta][8]
  float *d_shift32 = nullptr; // [nshift]
  double *d_cs = nullptr;     // [ntheta][2]: cos, sin theta (reduction, slicing.c:104-105)
  double4 *d_dirw = nullptr;  // [nphi*ntheta]: omega / h, dphi * w_theta (backprojection)
  std::vector<double4> dirw;  // host copy of d_dirw
  size_t bytes = 0;
};

namespace wrt {

int fail(wrt_ctx *ctx, int status, const char *fmt, ...) {
  if (ctx) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(ctx->err, sizeof(ctx->err), fmt, ap);
    va_end(ap);
  }
  return status;
}

int cuda_fail(wrt_ctx *ctx, cudaError_t e, const char *what) {
  return fail(ctx, WRT_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

int ctx_alloc(wrt_ctx *ctx, void **p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) return WRT_OK;
  if (ctx->budget && ctx->in_use + bytes > ctx->budget)
    return fail(ctx, WRT_ERR_BUDGET, "device budget: %zu bytes in use + %zu requested > %zu",
                ctx->in_use, bytes, ctx->budget);
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(ctx, WRT_ERR_OUT_OF_MEMORY, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  }
  ctx->in_use += bytes;
  return WRT_OK;
}

void ctx_free(wrt_ctx *ctx, void *p, size_t bytes) {
  if (!p) return;
  cudaFree(p);
  ctx->in_use -= bytes;
}

int check_launch(wrt_ctx *ctx, const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, what);
  return WRT_OK;
}

void ray_tables(int nshift, int nphi, double *tab) {
  double *shift = tab, *trig = tab + nshift;
  const double dshift = 2.0 / (nshift - 1);
  for (int i = 0; i < nshift; ++i) shift[i] = (-1.0) + i * dshift;
  const double dphi = (2 * M_PI) / nphi;
  for (int i = 0; i < nphi; ++i) {
    const double phi = dphi * i;
    trig[4 * i + 0] = cos(phi);
    trig[4 * i + 1] = sin(phi);
    trig[4 * i + 2] = cos(phi + M_PI / 2);
    trig[4 * i + 3] = sin(phi + M_PI / 2);
  }
}

double trilinear_margin(int n) { return sqrt(3.0) * (2.0 / (n - 1)) + 1e-6; }

void grid_tables(const wrt_grid *g, const double **dir, const double **shift) {
  *dir = g->d_dir;
  *shift = g->d_shift;
}

bool identity_frame(const double *f) {
  return !f || (f[0] == 1.0 && f[4] == 1.0 && f[8] == 1.0 && f[1] == 0.0 && f[2] == 0.0 &&
                f[3] == 0.0 && f[5] == 0.0 && f[6] == 0.0 && f[7] == 0.0);
}

void spline_coefficients(int ns, double *cp, double *den) {
  for (int i = 0; i < ns; ++i) {
    cp[i] = 0.0;
    den[i] = 1.0;
  }
  for (int i = 1; i + 1 < ns; ++i) {
    den[i] = 4.0 - (i > 1 ? cp[i - 1] : 0.0);
    cp[i] = 1.0 / den[i];
  }
}

int ws_get(wrt_ctx *ctx, int role, size_t bytes, void **p) {
  if (role < 0 || role >= WS_ROLES) return fail(ctx, WRT_ERR_INTERNAL, "workspace role %d", role);
  if (bytes <= ctx->ws_bytes[role] && ctx->ws[role]) {
    *p = ctx->ws[role];
    return WRT_OK;
  }
  if (ctx->ws[role]) {  // work queued on the stream may still read the old buffer
    cudaStreamSynchronize(ctx->stream);
    ctx_free(ctx, ctx->ws[role], ctx->ws_bytes[role]);
    ctx->ws[role] = nullptr;
    ctx->ws_bytes[role] = 0;
  }
  const size_t want = (bytes + (1 << 16) - 1) & ~(size_t)((1 << 16) - 1);
  int st = ctx_alloc(ctx, &ctx->ws[role], want);
  if (st) return st;
  ctx->ws_bytes[role] = want;
  *p = ctx->ws[role];
  return WRT_OK;
}

}  // namespace wrt

using namespace wrt;

namespace {

// RAII device buffer owned by a context.
struct DevBuf {
  wrt_ctx *ctx;
  void *p = nullptr;
  size_t bytes = 0;
  explicit DevBuf(wrt_ctx *c) : ctx(c) {}
  int alloc(size_t b) {
    bytes = b;
    return ctx_alloc(ctx, &p, b);
  }
  ~DevBuf() {
    if (p) ctx_free(ctx, p, bytes);
  }
  template <typename T>
  T *as() const {
    return static_cast<T *>(p);
  }
};

int h2d(wrt_ctx *ctx, void *dst, const void *src, size_t bytes, const char *what) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
  return e == cudaSuccess ? WRT_OK : cuda_fail(ctx, e, what);
}

int d2h_sync(wrt_ctx *ctx, void *dst, const void *src, size_t bytes, const char *what) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? WRT_OK : cuda_fail(ctx, e, what);
}

int set_device(wrt_ctx *ctx) {
  cudaError_t e = cudaSetDevice(ctx->device);
  return e == cudaSuccess ? WRT_OK : cuda_fail(ctx, e, "cudaSetDevice");
}

// Reach of a sampler around a lattice point: every node whose value can enter
// the sample lies within this distance (trilinear: one cell diagonal of the
// node grid; nearest: cell 2/n plus the offset between cell and node grids).
double sampler_margin(int n, int sampler) {
  if (sampler == WRT_SAMPLER_TRILINEAR) return trilinear_margin(n);
  const double h = 2.0 / (n - 1);
  return sqrt(3.0) * (4.0 / n + h) + 1e-6;
}

bool valid_plane_opts(const wrt_plane_opts *o, int n) {
  if (!o) return true;
  if (o->sampler != WRT_SAMPLER_NEAREST && o->sampler != WRT_SAMPLER_TRILINEAR) return false;
  if (o->half_extent < 0 || o->half_extent > 8 * n) return false;
  if (o->kernel < WRT_KERNEL_AUTO || o->kernel > WRT_KERNEL_STAGED) return false;
  return true;
}

}  // namespace

extern "C" {

const char *wrt_status_string(int s) {
  switch (s) {
    case WRT_OK: return "ok";
    case WRT_ERR_INVALID_ARGUMENT: return "invalid argument";
    case WRT_ERR_OUT_OF_MEMORY: return "out of memory";
    case WRT_ERR_BUDGET: return "over the device-memory budget";
    case WRT_ERR_CUDA: return "CUDA error";
    case WRT_ERR_NO_DEVICE: return "no usable CUDA device";
    case WRT_ERR_TIMEOUT: return "timed out";
    case WRT_ERR_QUEUE_FULL: return "queue full";
    case WRT_ERR_NOT_FOUND: return "not found";
    case WRT_ERR_CANCELLED: return "cancelled";
    case WRT_ERR_INTERNAL: return "internal error";
    default: return "unknown status";
  }
}

int wrt_abi_version(void) { return WRT_ABI_VERSION; }

int wrt_ctx_create(int device, size_t budget, wrt_ctx **out) {
  if (!out) return WRT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return WRT_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count) return WRT_ERR_INVALID_ARGUMENT;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return WRT_ERR_NO_DEVICE;
  if (prop.major < 10) return WRT_ERR_NO_DEVICE;  // built for sm_100a only
  wrt_ctx *ctx = new (std::nothrow) wrt_ctx();
  if (!ctx) return WRT_ERR_OUT_OF_MEMORY;
  ctx->device = device;
  ctx->budget = budget;
  ctx->sm_count = prop.multiProcessorCount;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return WRT_ERR_CUDA;
  }
  noalloc_forget_device(device);
  *out = ctx;
  return WRT_OK;
}

int wrt_ctx_destroy(wrt_ctx *ctx) {
  if (!ctx) return WRT_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
  if (ctx->ev_stop) cudaEventDestroy(ctx->ev_stop);
  ctx_free(ctx, ctx->flush_buf, ctx->flush_bytes);
  ctx_free(ctx, ctx->d_counter, sizeof(unsigned long long));
  for (auto &kv : ctx->user_allocs) cudaFree(kv.first);
  if (ctx->batch_slot) {
    BatchSlot *s = static_cast<BatchSlot *>(ctx->batch_slot);
    batch_slot_release(s);
    delete s;
    ctx->batch_slot = nullptr;
  }
  staged_release(ctx);
  if (ctx->dropin_vol) wrt_volume_destroy(ctx->dropin_vol);
  if (ctx->dropin_grid) wrt_grid_destroy(ctx->dropin_grid);
  laplace_release(ctx);
  for (int r = 0; r < WS_ROLES; ++r) ctx_free(ctx, ctx->ws[r], ctx->ws_bytes[r]);
  pinned_release(ctx);
  host_pool_destroy(ctx->host_pool);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return WRT_OK;
}

const char *wrt_ctx_last_error(const wrt_ctx *ctx) { return ctx ? ctx->err : "no context"; }

int wrt_ctx_synchronize(wrt_ctx *ctx) {
  if (!ctx) return WRT_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? WRT_OK : cuda_fail(ctx, e, "synchronize");
}

size_t wrt_ctx_bytes_in_use(const wrt_ctx *ctx) { return ctx ? ctx->in_use : 0; }

int wrt_ctx_timer_start(wrt_ctx *ctx) {
  if (!ctx) return WRT_ERR_INVALID_ARGUMENT;
  if (!ctx->ev_start && (cudaEventCreate(&ctx->ev_start) != cudaSuccess ||
                         cudaEventCreate(&ctx->ev_stop) != cudaSuccess))
    return fail(ctx, WRT_ERR_CUDA, "timer events");
  cudaError_t e = cudaEventRecord(ctx->ev_start, ctx->stream);
  return e == cudaSuccess ? WRT_OK : cuda_fail(ctx, e, "timer start");
}

int wrt_ctx_timer_stop(wrt_ctx *ctx, float *ms) {
  if (!ctx || !ms || !ctx->ev_start) return WRT_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaEventRecord(ctx->ev_stop, ctx->stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(ctx->ev_stop);
  if (e == cudaSuccess) e = cudaEventElapsedTime(ms, ctx->ev_start, ctx->ev_stop);
  return e == cudaSuccess ? WRT_OK : cuda_fail(ctx, e, "timer stop");
}

int wrt_ctx_flush_l2(wrt_ctx *ctx) {
  if (!ctx) return WRT_ERR_INVALID_ARGUMENT;
  if (!ctx->flush_buf) {
    int l2 = 0;
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, ctx->device);
    const size_t bytes = 2 * (size_t)(l2 > 0 ? l2 : (128 << 20));
    int st = ctx_alloc(ctx, &ctx->flush_buf, bytes);
    if (st) return st;
    ctx->flush_bytes = bytes;
  }
  cudaError_t e = cudaMemsetAsync(ctx->flush_buf, ctx->launches & 0xff, ctx->flush_bytes, ctx->stream);
  return e == cudaSuccess ? WRT_OK : cuda_fail(ctx, e, "flush l2");
}

int wrt_ctx_count_samples(wrt_ctx *ctx, int on) {
  if (!ctx) return WRT_ERR_INVALID_ARGUMENT;
  if (on && !ctx->d_counter) {
    int st = ctx_alloc(ctx, (void **)&ctx->d_counter, sizeof(unsigned long long));
    if (st) return st;
    cudaError_t e = cudaMemsetAsync(ctx->d_counter, 0, sizeof(unsigned long long), ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "sample counter");
  } else if (!on && ctx->d_counter) {
    cudaStreamSynchronize(ctx->stream);
    ctx_free(ctx, ctx->d_counter, sizeof(unsigned long long));
    ctx->d_counter = nullptr;
  }
  return WRT_OK;
}

int wrt_ctx_sample_count(wrt_ctx *ctx, uint64_t *count) {
  if (!ctx || !count) return WRT_ERR_INVALID_ARGUMENT;
  *count = 0;
  if (!ctx->d_counter) return WRT_OK;
  unsigned long long v = 0;
  int st = d2h_sync(ctx, &v, ctx->d_counter, sizeof(v), "sample count");
  if (!st) *count = v;
  return st;
}

int wrt_device_alloc(wrt_ctx *ctx, size_t bytes, void **dev_ptr) {
  if (!ctx || !dev_ptr || bytes == 0) return WRT_ERR_INVALID_ARGUMENT;
  int st = set_device(ctx);
  if (!st) st = ctx_alloc(ctx, dev_ptr, bytes);
  if (!st) ctx->user_allocs[*dev_ptr] = bytes;
  return st;
}

int wrt_device_free(wrt_ctx *ctx, void *p) {
  if (!ctx || !p) return WRT_ERR_INVALID_ARGUMENT;
  auto it = ctx->user_allocs.find(p);
  if (it == ctx->user_allocs.end()) return fail(ctx, WRT_ERR_NOT_FOUND, "unknown device pointer");
  cudaStreamSynchronize(ctx->stream);
  ctx_free(ctx, p, it->second);
  ctx->user_allocs.erase(it);
  return WRT_OK;
}

int wrt_host_alloc_pinned(wrt_ctx *ctx, size_t bytes, void **host_ptr) {
  if (!ctx || !host_ptr || bytes == 0) return WRT_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaMallocHost(host_ptr, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, WRT_ERR_OUT_OF_MEMORY, "cudaMallocHost(%zu)", bytes);
  }
  return WRT_OK;
}

int wrt_host_free_pinned(wrt_ctx *ctx, void *host_ptr) {
  if (!ctx || !host_ptr) return WRT_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaFreeHost(host_ptr);
  return e == cudaSuccess ? WRT_OK : cuda_fail(ctx, e, "cudaFreeHost");
}

int wrt_copy_to_device(wrt_ctx *ctx, void *dst, const void *src, size_t bytes) {
  if (!ctx || !dst || !src) return WRT_ERR_INVALID_ARGUMENT;
  return h2d_staged(ctx, dst, src, bytes, "copy to device");
}

int wrt_copy_to_host(wrt_ctx *ctx, void *dst, const void *src, size_t bytes) {
  if (!ctx || !dst || !src) return WRT_ERR_INVALID_ARGUMENT;
  return d2h_staged_sync(ctx, dst, src, bytes, "copy to host");
}

int wrt_measure_smem_bandwidth(wrt_ctx *ctx, double *bytes_per_s) {
  if (!ctx || !bytes_per_s) return WRT_ERR_INVALID_ARGUMENT;
  int st = set_device(ctx);
  return st ? st : smem_bandwidth(ctx, bytes_per_s);
}
uint64_t wrt_ctx_launch_count(const wrt_ctx *ctx) { return ctx ? ctx->launches : 0; }
void *wrt_ctx_stream(wrt_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int wrt_gauss_legendre(wrt_ctx *ctx, int n, double *x, double *w) {
  if (!ctx || !x || !w) return WRT_ERR_INVALID_ARGUMENT;
  int st = set_device(ctx);
  return st ? st : gauss_legendre_device(ctx, n, x, w);
}

int wrt_radon_grid_init(wrt_ctx *ctx, int nphi, int ntheta, int nshift, double *phi,
                        double *theta, double *theta_w, double *shift) {
  if (!ctx || !phi || !theta || !shift) return WRT_ERR_INVALID_ARGUMENT;
  int st = set_device(ctx);
  return st ? st : sphere_grid(ctx, nphi, ntheta, nshift, phi, theta, theta_w, shift);
}

// ------------------------------------------------------------ resident objects
int wrt_volume_create(wrt_ctx *ctx, int n, wrt_volume **out) {
  return wrt_volume_create_storage(ctx, n, WRT_STORAGE_F32, out);
}

int wrt_volume_create_storage(wrt_ctx *ctx, int n, int storage, wrt_volume **out) {
  if (!ctx || !out || n < 2 || n > 2048) return WRT_ERR_INVALID_ARGUMENT;
  if (storage != WRT_STORAGE_F32 && storage != WRT_STORAGE_BF16) return WRT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int st = set_device(ctx);
  if (st) return st;
  wrt_volume *v = new (std::nothrow) wrt_volume();
  if (!v) return WRT_ERR_OUT_OF_MEMORY;
  v->ctx = ctx;
  v->n = n;
  v->storage = storage;
  const size_t count = (size_t)n * n * n;
  if (storage == WRT_STORAGE_BF16) {
    v->vol_bytes = sizeof(__nv_bfloat16) * count;
    st = ctx_alloc(ctx, (void **)&v->d_vol16, v->vol_bytes);
  } else {
    v->vol_bytes = sizeof(float) * count;
    st = ctx_alloc(ctx, (void **)&v->d_vol, v->vol_bytes);
  }
  if (!st) st = ctx_alloc(ctx, (void **)&v->d_stats, 2 * sizeof(unsigned int));
  if (st) {
    wrt_volume_destroy(v);
    return st;
  }
  *out = v;
  return WRT_OK;
}

namespace {
// Waits for the upload and copies the volume statistics to the host.
int volume_finish_upload(wrt_volume *v) {
  wrt_ctx *ctx = v->ctx;
  unsigned int stats[2] = {0, 0};
  int st = d2h_sync(ctx, stats, v->d_stats, sizeof(stats), "volume statistics");
  if (st) return st;
  memcpy(&v->r2, &stats[0], sizeof(float));
  memcpy(&v->maxabs, &stats[1], sizeof(float));
  v->pairs_valid = false;
  v->oct_valid = false;
  v->layers_valid = false;
  return WRT_OK;
}

int volume_ensure_layers(wrt_volume *v) {
  if (v->layers_valid) return WRT_OK;
  if (!v->d_layers) {
    int st = ctx_alloc(v->ctx, (void **)&v->d_layers, v->vol_bytes);
    if (st) return st;
  }
  int st = volume_layers(v->ctx, v->d_vol, v->n, v->d_layers);
  if (!st) v->layers_valid = true;
  return st;
}

int volume_ensure_octets(wrt_volume *v) {
  if (v->oct_valid) return WRT_OK;
  wrt_ctx *ctx = v->ctx;
  if (!v->d_oct) {
    const size_t m = (size_t)(v->n - 1);
    v->oct_bytes = 2 * sizeof(float4) * m * m * m;
    int st = ctx_alloc(ctx, (void **)&v->d_oct, v->oct_bytes);
    if (st) return st;
  }
  int st = volume_octets(ctx, v->d_vol, v->n, v->d_oct);
  if (!st) v->oct_valid = true;
  return st;
}

int volume_ensure_pairs(wrt_volume *v) {
  if (v->pairs_valid) return WRT_OK;
  wrt_ctx *ctx = v->ctx;
  const bool bf16 = v->storage == WRT_STORAGE_BF16;
  if (!v->d_pairs && !v->d_pairs16) {
    v->pitch = v->n + (v->n & 1);
    v->pair_bytes = (bf16 ? sizeof(__nv_bfloat162) : sizeof(float2)) * (size_t)(v->n - 1) * v->n *
                    v->pitch;
    int st = bf16 ? ctx_alloc(ctx, (void **)&v->d_pairs16, v->pair_bytes)
                  : ctx_alloc(ctx, (void **)&v->d_pairs, v->pair_bytes);
    if (st) return st;
  }
  int st = bf16 ? volume_pairs_bf16(ctx, v->d_vol16, v->n, v->d_pairs16, v->pitch)
                : volume_pairs(ctx, v->d_vol, v->n, v->d_pairs, v->pitch);
  if (!st) v->pairs_valid = true;
  return st;
}
}  // namespace

int wrt_volume_upload(wrt_volume *v, const double *f64, const float *f32) {
  if (!v || ((f64 == nullptr) == (f32 == nullptr))) return WRT_ERR_INVALID_ARGUMENT;
  wrt_ctx *ctx = v->ctx;
  int st = set_device(ctx);
  if (st) return st;
  const size_t count = (size_t)v->n * v->n * v->n;
  const bool bf16 = v->storage == WRT_STORAGE_BF16;
  // staging (and the FP32 copy a BF16 volume is rounded from) in the context's
  // workspace; the upload waits for the statistics, so the buffers are free
  // again when it returns.  FP64 values are rounded to FP32 on the host while
  // they are staged (to nearest, as the device conversion would), so the
  // device receives FP32 either way.
  const size_t in_bytes = count * sizeof(float);
  void *stage = nullptr, *vol32 = nullptr;
  st = ws_get(ctx, WS_STAGE, in_bytes, &stage);
  if (!st && bf16) st = ws_get(ctx, WS_IN, count * sizeof(float), &vol32);
  float *dst = bf16 ? static_cast<float *>(vol32) : v->d_vol;
  if (!st)
    st = f64 ? h2d_staged_rounded(ctx, static_cast<float *>(stage), f64, count, "volume upload")
             : h2d_staged(ctx, stage, f32, in_bytes, "volume upload");
  if (!st) st = volume_from_f32(ctx, static_cast<float *>(stage), v->n, dst, v->d_stats);
  if (!st && bf16) st = volume_to_bf16(ctx, dst, v->n, v->d_vol16, v->d_stats);
  if (!st) st = volume_finish_upload(v);
  return st;
}

int wrt_volume_upload_device(wrt_volume *v, const float *dev_f32) {
  if (!v || !dev_f32) return WRT_ERR_INVALID_ARGUMENT;
  int st = set_device(v->ctx);
  if (st) return st;
  st = v->storage == WRT_STORAGE_BF16 ? volume_to_bf16(v->ctx, dev_f32, v->n, v->d_vol16, v->d_stats)
                                      : volume_from_f32(v->ctx, dev_f32, v->n, v->d_vol, v->d_stats);
  if (!st) st = volume_finish_upload(v);
  return st;
}

size_t wrt_volume_bytes(const wrt_volume *v) {
  return v ? v->vol_bytes + v->pair_bytes + v->oct_bytes + (v->d_layers ? v->vol_bytes : 0) +
                 2 * sizeof(unsigned int)
           : 0;
}

int wrt_volume_destroy(wrt_volume *v) {
  if (!v) return WRT_ERR_INVALID_ARGUMENT;
  wrt_ctx *ctx = v->ctx;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ctx_free(ctx, v->d_vol, v->vol_bytes);
  ctx_free(ctx, v->d_vol16, v->vol_bytes);
  ctx_free(ctx, v->d_stats, 2 * sizeof(unsigned int));
  ctx_free(ctx, v->d_pairs, v->pair_bytes);
  ctx_free(ctx, v->d_pairs16, v->pair_bytes);
  ctx_free(ctx, v->d_oct, v->oct_bytes);
  ctx_free(ctx, v->d_layers, v->d_layers ? v->vol_bytes : 0);
  delete v;
  return WRT_OK;
}

int wrt_grid_create(wrt_ctx *ctx, int nphi, int ntheta, int nshift, wrt_grid **out) {
  if (!ctx || !out || nphi < 1 || ntheta < 1 || nshift < 2 || (long long)nphi * ntheta > (1 << 26))
    return WRT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int st = set_device(ctx);
  if (st) return st;
  wrt_grid *g = new (std::nothrow) wrt_grid();
  if (!g) return WRT_ERR_OUT_OF_MEMORY;
  g->ctx = ctx;
  g->nphi = nphi;
  g->ntheta = ntheta;
  g->nshift = nshift;
  g->phi.resize(nphi);
  g->theta.resize(ntheta);
  g->w.resize(ntheta);
  g->shift.resize(nshift);
  st = sphere_grid(ctx, nphi, ntheta, nshift, g->phi.data(), g->theta.data(), g->w.data(),
                   g->shift.data());
  const size_t ndir = (size_t)nphi * ntheta;
  std::vector<double> dir(ndir * 9);
  std::vector<float> dir32(ndir * 8), shift32(nshift);
  if (!st) {
    plane_directions(nphi, g->phi.data(), ntheta, g->theta.data(), dir.data());
    for (size_t d = 0; d < ndir; ++d)
      for (int k = 0; k < 8; ++k) dir32[8 * d + k] = (float)dir[9 * d + k];
    for (int i = 0; i < nshift; ++i) shift32[i] = (float)g->shift[i];
    st = ctx_alloc(ctx, (void **)&g->d_dir, sizeof(double) * dir.size());
  }
  if (!st) st = ctx_alloc(ctx, (void **)&g->d_shift, sizeof(double) * nshift);
  if (!st) st = ctx_alloc(ctx, (void **)&g->d_dir32, sizeof(float) * dir32.size());
  if (!st) st = ctx_alloc(ctx, (void **)&g->d_shift32, sizeof(float) * nshift);
  std::vector<double> cs(2 * (size_t)ntheta);
  std::vector<double4> &dirw = g->dirw;
  dirw.resize(ndir);
  if (!st) {
    for (int i = 0; i < ntheta; ++i) {
      cs[2 * i] = cos(g->theta[i]);  // slicing.c:104-105 evaluate cos/sin(p_theta)
      cs[2 * i + 1] = sin(g->theta[i]);
    }
    adjoint_directions(nphi, ntheta, nshift, g->phi.data(), g->theta.data(), g->w.data(),
                       dirw.data());
    st = ctx_alloc(ctx, (void **)&g->d_cs, sizeof(double) * cs.size());
  }
  if (!st) st = ctx_alloc(ctx, (void **)&g->d_dirw, sizeof(double4) * ndir);
  if (!st) st = h2d(ctx, g->d_dir, dir.data(), sizeof(double) * dir.size(), "grid upload");
  if (!st) st = h2d(ctx, g->d_shift, g->shift.data(), sizeof(double) * nshift, "grid upload");
  if (!st) st = h2d(ctx, g->d_dir32, dir32.data(), sizeof(float) * dir32.size(), "grid upload");
  if (!st) st = h2d(ctx, g->d_shift32, shift32.data(), sizeof(float) * nshift, "grid upload");
  if (!st) st = h2d(ctx, g->d_cs, cs.data(), sizeof(double) * cs.size(), "grid upload");
  if (!st) st = h2d(ctx, g->d_dirw, dirw.data(), sizeof(double4) * ndir, "grid upload");
  if (!st) {
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) st = cuda_fail(ctx, e, "grid upload");
  }
  if (st) {
    wrt_grid_destroy(g);
    return st;
  }
  *out = g;
  return WRT_OK;
}

int wrt_grid_destroy(wrt_grid *g) {
  if (!g) return WRT_ERR_INVALID_ARGUMENT;
  cudaSetDevice(g->ctx->device);
  cudaStreamSynchronize(g->ctx->stream);
  const size_t ndir = (size_t)g->nphi * g->ntheta;
  ctx_free(g->ctx, g->d_dir, sizeof(double) * 9 * ndir);
  ctx_free(g->ctx, g->d_shift, sizeof(double) * g->nshift);
  ctx_free(g->ctx, g->d_dir32, sizeof(float) * 8 * ndir);
  ctx_free(g->ctx, g->d_shift32, sizeof(float) * g->nshift);
  ctx_free(g->ctx, g->d_cs, sizeof(double) * 2 * g->ntheta);
  ctx_free(g->ctx, g->d_dirw, sizeof(double4) * ndir);
  delete g;
  return WRT_OK;
}

namespace {

// Staged-kernel launch of one request; see k_staged.cu.  Trilinear: the
// volume's layer pairs; nearest: its z-major cell layers (FP32 storage).
int radon_forward_staged(wrt_ctx *ctx, wrt_volume *vol, const wrt_grid *grid, int L,
                         double *dev_out, bool nearest) {
  int st = nearest ? volume_ensure_layers(vol) : volume_ensure_pairs(vol);
  if (st) return st;
  const int n = vol->n;
  int th = 0, qp = 0;
  const int smem =
      nearest ? staged_smem_bytes_nearest(n, &th, &qp) : staged_smem_bytes(n, &th, &qp);
  StagedReq r = {};
  const bool bf16 = vol->storage == WRT_STORAGE_BF16;
  r.pairs = nearest ? (const void *)vol->d_layers
                    : bf16 ? (const void *)vol->d_pairs16 : (const void *)vol->d_pairs;
  r.vol = bf16 ? (const void *)vol->d_vol16 : (const void *)vol->d_vol;
  r.storage = vol->storage;
  r.nearest = nearest ? 1 : 0;
  r.dir = grid->d_dir;
  r.dir32 = grid->d_dir32;
  r.shift = grid->d_shift;
  r.shift32 = grid->d_shift32;
  r.acc = reinterpret_cast<unsigned long long *>(dev_out);
  r.n = n;
  r.pitch2 = nearest ? n : vol->pitch;
  r.qpitch = qp;
  r.tile_h = th;
  r.ndir = grid->nphi * grid->ntheta;
  r.nshift = grid->nshift;
  r.L = L;
  r.crop_r2 = nearest ? nearest_crop_r2(vol->r2, n) : trilinear_crop_r2(vol->r2, n);
  r.guard = staged_guard(n, L, r.crop_r2, nearest);
  r.scale = fixed_point_scale(vol->maxabs, L);
  StagedItem *d_items = nullptr;
  const int *d_nitems = nullptr;
  int nitems = 0;
  st = staged_items_cached(ctx, n, th, r.crop_r2, r.ndir, &d_items, &d_nitems, &nitems, nearest);
  if (st) return st;
  st = staged_scratch(ctx, sizeof(StagedReq));
  if (st) return st;
  st = h2d(ctx, ctx->staged_req, &r, sizeof(r), "staged request");
  if (st) return st;
  const size_t nout = (size_t)r.ndir * r.nshift;
  cudaError_t e = cudaMemsetAsync(dev_out, 0, sizeof(double) * nout, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "staged output reset");
  if (nitems > 0) {
    st = (nearest ? plane_staged_launch_nearest : plane_staged_launch)(
        ctx, ctx->stream, (const StagedReq *)ctx->staged_req, d_items, d_nitems, smem,
        ctx->staged_next);
    if (st) return st;
  }
  const double delta = 1.0 / n;
  return plane_finalize(ctx, dev_out, (long long)nout, delta * delta / r.scale);
}

}  // namespace

int wrt_radon_forward_device(wrt_ctx *ctx, const wrt_volume *cvol, const wrt_grid *grid,
                             const wrt_plane_opts *opts, double *dev_out) {
  wrt_volume *vol = const_cast<wrt_volume *>(cvol);
  if (!ctx || !vol || !grid || !dev_out || vol->ctx != ctx || grid->ctx != ctx)
    return WRT_ERR_INVALID_ARGUMENT;
  if (!valid_plane_opts(opts, vol->n))
    return fail(ctx, WRT_ERR_INVALID_ARGUMENT, "invalid plane options");
  int st = set_device(ctx);
  if (st) return st;
  wrt_plane_opts o = {};
  if (opts) o = *opts;
  const int L = o.half_extent ? o.half_extent : 2 * vol->n;
  int th = 0, qp = 0;
  const bool nearest = o.sampler == WRT_SAMPLER_NEAREST;
  const bool staged_ok =
      vol->n >= 4 && (nearest ? vol->storage == WRT_STORAGE_F32 &&
                                    staged_smem_bytes_nearest(vol->n, &th, &qp) > 0
                              : staged_smem_bytes(vol->n, &th, &qp) > 0);
  if (vol->storage == WRT_STORAGE_BF16 && (o.kernel == WRT_KERNEL_PLAIN || nearest || !staged_ok))
    return fail(ctx, WRT_ERR_INVALID_ARGUMENT,
                "BF16 volumes are sampled by the staged kernel (trilinear sampler) only");
  if (o.kernel == WRT_KERNEL_STAGED && !staged_ok)
    return fail(ctx, WRT_ERR_INVALID_ARGUMENT, "staged kernel: volume edge below 4");
  if (o.kernel != WRT_KERNEL_PLAIN && staged_ok)
    return radon_forward_staged(ctx, vol, grid, L, dev_out, nearest);
  PlaneJob job = {};
  job.vol = vol->d_vol;
  job.n = vol->n;
  job.dir = grid->d_dir;
  job.shift = grid->d_shift;
  job.ndir = grid->nphi * grid->ntheta;
  job.nshift = grid->nshift;
  job.L = L;
  job.sampler = o.sampler;
  job.r2bits = vol->d_stats;
  job.margin = sampler_margin(vol->n, o.sampler);
  job.out = dev_out;
  job.counter = ctx->d_counter;
  return plane_forward_plain(ctx, job);
}

int wrt_radon_forward_batch(wrt_ctx *ctx, const wrt_forward_req *reqs, int nreq) {
  if (!ctx || (nreq > 0 && !reqs) || nreq < 0) return WRT_ERR_INVALID_ARGUMENT;
  if (nreq > kBatchMaxFwd)
    return fail(ctx, WRT_ERR_INVALID_ARGUMENT, "batch: at most %d requests", kBatchMaxFwd);
  int st = set_device(ctx);
  if (st) return st;
  if (nreq == 0) return WRT_OK;
  BatchBuilder b;
  for (int r = 0; r < nreq; ++r) {
    wrt_volume *vol = const_cast<wrt_volume *>(reqs[r].volume);
    const wrt_grid *grid = reqs[r].grid;
    if (!vol || !grid || !reqs[r].dev_out || vol->ctx != ctx || grid->ctx != ctx)
      return fail(ctx, WRT_ERR_INVALID_ARGUMENT, "batch request %d: bad volume, grid or output", r);
    const int n = vol->n;
    int th = 0, qp = 0;
    if (n < 4 || staged_smem_bytes(n, &th, &qp) <= 0)
      return fail(ctx, WRT_ERR_INVALID_ARGUMENT, "batch request %d: volume edge %d unsupported", r, n);
    if (reqs[r].half_extent < 0 || reqs[r].half_extent > 8 * n)
      return fail(ctx, WRT_ERR_INVALID_ARGUMENT, "batch request %d: bad half extent", r);
    st = volume_ensure_pairs(vol);
    if (st) return st;
    const int L = reqs[r].half_extent ? reqs[r].half_extent : 2 * n;
    StagedReq q;
    const bool bf16 = vol->storage == WRT_STORAGE_BF16;
    staged_request(n, vol->pitch, grid->nphi * grid->ntheta, grid->nshift, L, vol->storage,
                   bf16 ? (const void *)vol->d_pairs16 : (const void *)vol->d_pairs,
                   bf16 ? (const void *)vol->d_vol16 : (const void *)vol->d_vol, grid->d_dir,
                   grid->d_dir32, grid->d_shift, grid->d_shift32, reqs[r].dev_out, &q);
    FwdAux a = {};
    a.vol = vol->d_vol;
    a.pairs = vol->d_pairs;
    a.stats = vol->d_stats;
    a.nout = (long long)q.ndir * q.nshift;
    a.n = n;
    a.pitch = vol->pitch;
    a.L = L;
    a.prep = 0;
    batch_add_forward(b, q, a, trilinear_crop_r2(vol->r2, n));
  }
  if (!ctx->batch_slot) {
    BatchSlot *s = new (std::nothrow) BatchSlot();
    if (!s) return WRT_ERR_OUT_OF_MEMORY;
    st = batch_slot_init(ctx, s, ctx->stream);
    if (st) {
      batch_slot_release(s);
      delete s;
      return st;
    }
    ctx->batch_slot = s;
  }
  return batch_slot_launch(static_cast<BatchSlot *>(ctx->batch_slot), b);
}

int wrt_plane_kernel_config_count(void) { return kNumStagedConfigs; }

int wrt_plane_kernel_config_describe(int index, int *threads, int *rows_per_group,
                                     int *shifts_per_lane) {
  if (index < 0 || index >= kNumStagedConfigs) return WRT_ERR_INVALID_ARGUMENT;
  if (threads) *threads = kStagedConfigs[index].threads;
  if (rows_per_group) *rows_per_group = kStagedConfigs[index].group;
  if (shifts_per_lane) *shifts_per_lane = kStagedConfigs[index].shifts_per_lane;
  return WRT_OK;
}

int wrt_ctx_set_plane_kernel_config(wrt_ctx *ctx, int index) {
  if (!ctx || index < -1 || index >= kNumStagedConfigs) return WRT_ERR_INVALID_ARGUMENT;
  ctx->staged_config = index;
  return WRT_OK;
}

int wrt_tune_plane_kernel(wrt_ctx *ctx, const wrt_volume *vol, const wrt_grid *grid,
                          const wrt_plane_opts *opts, double *dev_out, int *best,
                          float *best_ms) {
  if (!ctx || !vol || !grid || !dev_out) return WRT_ERR_INVALID_ARGUMENT;
  wrt_plane_opts o = {};
  if (opts) o = *opts;
  o.kernel = WRT_KERNEL_STAGED;
  cudaEvent_t a, b;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess)
    return fail(ctx, WRT_ERR_CUDA, "tuner events");
  int st = WRT_OK, best_i = -1;
  float best_t = 0.0f;
  for (int c = 0; c < kNumStagedConfigs && !st; ++c) {
    ctx->staged_config = c;
    st = wrt_radon_forward_device(ctx, vol, grid, &o, dev_out);  // warm-up
    float tmin = 0.0f;
    for (int rep = 0; rep < 3 && !st; ++rep) {
      cudaEventRecord(a, ctx->stream);
      st = wrt_radon_forward_device(ctx, vol, grid, &o, dev_out);
      cudaEventRecord(b, ctx->stream);
      if (!st && cudaEventSynchronize(b) != cudaSuccess) st = fail(ctx, WRT_ERR_CUDA, "tuner sync");
      float ms = 0.0f;
      if (!st) cudaEventElapsedTime(&ms, a, b);
      if (rep == 0 || ms < tmin) tmin = ms;
    }
    if (!st && (best_i < 0 || tmin < best_t)) {
      best_i = c;
      best_t = tmin;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  ctx->staged_config = st ? -1 : best_i;
  if (!st) {
    if (best) *best = best_i;
    if (best_ms) *best_ms = best_t;
  }
  return st;
}

// -------------------------------------------------------- drop-in, host I/O
}  // extern "C"

namespace {

// The drop-in entry points keep the volume and the sphere grid of their last
// call in the context and their buffers in its workspace, so a warm call of
// the same sizes allocates no device memory.
int dropin_volume(wrt_ctx *ctx, int n, const double *host, wrt_volume **out) {
  if (ctx->dropin_vol && ctx->dropin_vol->n != n) {
    wrt_volume_destroy(ctx->dropin_vol);
    ctx->dropin_vol = nullptr;
  }
  int st = WRT_OK;
  if (!ctx->dropin_vol) st = wrt_volume_create(ctx, n, &ctx->dropin_vol);
  if (!st) st = wrt_volume_upload(ctx->dropin_vol, host, nullptr);
  *out = ctx->dropin_vol;
  return st;
}

int dropin_grid(wrt_ctx *ctx, int nphi, int ntheta, int nshift, wrt_grid **out) {
  wrt_grid *g = ctx->dropin_grid;
  if (g && (g->nphi != nphi || g->ntheta != ntheta || g->nshift != nshift)) {
    wrt_grid_destroy(g);
    ctx->dropin_grid = g = nullptr;
  }
  int st = WRT_OK;
  if (!g) st = wrt_grid_create(ctx, nphi, ntheta, nshift, &ctx->dropin_grid);
  *out = ctx->dropin_grid;
  return st;
}

}  // namespace

extern "C" {

int wrt_radon_grid(wrt_ctx *ctx, const double *volume, int n, int nphi, int ntheta, int nshift,
                   const wrt_plane_opts *opts, double *out) {
  if (!ctx || !volume || !out || n < 2 || nphi < 1 || ntheta < 1 || nshift < 2)
    return ctx ? fail(ctx, WRT_ERR_INVALID_ARGUMENT, "radon_grid: bad arguments")
               : WRT_ERR_INVALID_ARGUMENT;
  if (!valid_plane_opts(opts, n)) return fail(ctx, WRT_ERR_INVALID_ARGUMENT, "invalid plane options");
  int st = set_device(ctx);
  if (st) return st;
  wrt_volume *vol = nullptr;
  wrt_grid *grid = nullptr;
  void *dout = nullptr;
  const size_t nout = (size_t)nphi * ntheta * nshift;
  st = dropin_volume(ctx, n, volume, &vol);
  if (!st) st = dropin_grid(ctx, nphi, ntheta, nshift, &grid);
  if (!st) st = ws_get(ctx, WS_OUT, sizeof(double) * nout, &dout);
  if (!st) st = wrt_radon_forward_device(ctx, vol, grid, opts, static_cast<double *>(dout));
  if (!st) st = d2h_staged_sync(ctx, out, dout, sizeof(double) * nout, "radon_grid result");
  return st;
}

int wrt_radon_transpose(wrt_ctx *ctx, const double *g, int n, int nphi, int ntheta, int nshift,
                        const wrt_plane_opts *opts, double *out_volume) {
  if (!ctx || !g || !out_volume || n < 2 || nphi < 1 || ntheta < 1 || nshift < 2)
    return ctx ? fail(ctx, WRT_ERR_INVALID_ARGUMENT, "radon_transpose: bad arguments")
               : WRT_ERR_INVALID_ARGUMENT;
  if (!valid_plane_opts(opts, n)) return fail(ctx, WRT_ERR_INVALID_ARGUMENT, "invalid plane options");
  wrt_plane_opts o = {};
  if (opts) o = *opts;
  wrt_grid *grid = nullptr;
  int st = wrt_grid_create(ctx, nphi, ntheta, nshift, &grid);
  DevBuf dg(ctx), dvol(ctx), dvol32(ctx);
  const size_t nplanes = (size_t)nphi * ntheta * nshift, nvox = (size_t)n * n * n;
  if (!st) st = dg.alloc(sizeof(double) * nplanes);
  if (!st) st = dvol.alloc(sizeof(double) * nvox);
  if (!st) st = h2d(ctx, dg.p, g, sizeof(double) * nplanes, "transpose input");
  if (!st) {
    cudaError_t e = cudaMemsetAsync(dvol.p, 0, sizeof(double) * nvox, ctx->stream);
    if (e != cudaSuccess) st = cuda_fail(ctx, e, "transpose zero");
  }
  if (!st) {
    PlaneJob job = {};
    job.n = n;
    job.dir = grid->d_dir;
    job.shift = grid->d_shift;
    job.ndir = nphi * ntheta;
    job.nshift = nshift;
    job.L = o.half_extent ? o.half_extent : 2 * n;
    job.sampler = o.sampler;
    job.r2bits = nullptr;  // no volume: the whole cube
    job.margin = 0.0;
    st = plane_transpose(ctx, job, dg.as<double>(), dvol.as<double>());
  }
  if (!st) st = d2h_staged_sync(ctx, out_volume, dvol.p, sizeof(double) * nvox, "transpose result");
  if (grid) wrt_grid_destroy(grid);
  return st;
}

int wrt_ray_forward_device(wrt_ctx *ctx, const wrt_volume *cvol, const double *frame,
                           int nslices, int nshift, int nphi, double *dev_out) {
  wrt_volume *vol = const_cast<wrt_volume *>(cvol);
  if (!ctx || !vol || !dev_out || vol->ctx != ctx || nslices < 2 || nshift < 2 || nphi < 1)
    return ctx ? fail(ctx, WRT_ERR_INVALID_ARGUMENT, "ray_forward_device: bad arguments")
               : WRT_ERR_INVALID_ARGUMENT;
  if (vol->storage != WRT_STORAGE_F32)
    return fail(ctx, WRT_ERR_INVALID_ARGUMENT, "ray transform: FP32 volumes only");
  int st = set_device(ctx);
  if (st) return st;
  const int n = vol->n;
  std::vector<double> tab((size_t)nshift + 4 * (size_t)nphi);
  ray_tables(nshift, nphi, tab.data());
  const bool identity = identity_frame(frame);
  void *dtab = nullptr;
  st = ws_get(ctx, WS_TABLE, sizeof(double) * tab.size(), &dtab);
  // a copy from pageable memory returns once the data is staged
  if (!st) st = h2d(ctx, dtab, tab.data(), sizeof(double) * tab.size(), "ray grid");
  // samples read the cell octets (one 32-byte sector each; built once per
  // volume); in the reference frame the guard-band-free groups do, and single
  // samples read the layer pairs (built once) as before
  if (!st && identity) st = volume_ensure_pairs(vol);
  if (!st) st = volume_ensure_octets(vol);
  if (st) return st;
  RayJob job = {};
  job.vol = vol->d_vol;
  job.n = n;
  job.nslices = nslices;
  job.nshift = nshift;
  job.nphi = nphi;
  job.shift = static_cast<const double *>(dtab);
  job.trig = static_cast<const double *>(dtab) + nshift;
  job.has_frame = identity ? 0 : 1;
  if (!identity)
    for (int k = 0; k < 9; ++k) job.frame[k] = frame[k];
  job.r2bits = vol->d_stats;
  job.margin = sampler_margin(n, WRT_SAMPLER_TRILINEAR);
  job.out = dev_out;
  job.counter = ctx->d_counter;
  if (identity) {
    job.pairs = vol->d_pairs;
    job.pitch = vol->pitch;
  }
  job.oct = vol->d_oct;
  return ray_forward(ctx, job);
}

int wrt_ray_grid(wrt_ctx *ctx, const double *volume, int n, int nslices, int nshift, int nphi,
                 const double *frame, double *out) {
  if (!ctx || !volume || !out || n < 2 || nslices < 2 || nshift < 2 || nphi < 1)
    return ctx ? fail(ctx, WRT_ERR_INVALID_ARGUMENT, "ray_grid: bad arguments")
               : WRT_ERR_INVALID_ARGUMENT;
  int st = set_device(ctx);
  if (st) return st;
  wrt_volume *vol = nullptr;
  void *dout = nullptr;
  const size_t nout = (size_t)nslices * nshift * nphi;
  st = dropin_volume(ctx, n, volume, &vol);
  if (!st) st = ws_get(ctx, WS_OUT, sizeof(double) * nout, &dout);
  if (!st) st = wrt_ray_forward_device(ctx, vol, frame, nslices, nshift, nphi,
                                       static_cast<double *>(dout));
  if (!st) st = d2h_staged_sync(ctx, out, dout, sizeof(double) * nout, "ray_grid result");
  return st;
}

int wrt_radon_reduction_device(wrt_ctx *ctx, const double *dev_rays, int ngrid, int nshift_ray,
                               const wrt_grid *grid, double *dev_out) {
  if (!ctx || !dev_rays || !grid || !dev_out || grid->ctx != ctx || ngrid < 3 || nshift_ray < 3)
    return ctx ? fail(ctx, WRT_ERR_INVALID_ARGUMENT, "radon_reduction_device: bad arguments")
               : WRT_ERR_INVALID_ARGUMENT;
  int st = set_device(ctx);
  if (st) return st;
  return reduction_forward(ctx, dev_rays, ngrid, nshift_ray, grid->nphi, grid->d_shift,
                           grid->nshift, grid->d_cs, grid->ntheta, dev_out);
}

int wrt_radon_reduction(wrt_ctx *ctx, const double *rays, int ngrid, int nshift_ray, int nphi,
                        int nshift, int ntheta, double *out) {
  if (!ctx || !rays || !out || ngrid < 3 || nshift_ray < 3 || nphi < 1 || nshift < 2 || ntheta < 1)
    return ctx ? fail(ctx, WRT_ERR_INVALID_ARGUMENT, "radon_reduction: bad arguments")
               : WRT_ERR_INVALID_ARGUMENT;
  int st = set_device(ctx);
  if (st) return st;
  wrt_grid *grid = nullptr;
  void *din = nullptr, *dout = nullptr;
  const size_t nin = (size_t)ngrid * nshift_ray * nphi, nout = (size_t)nshift * nphi * ntheta;
  st = dropin_grid(ctx, nphi, ntheta, nshift, &grid);
  if (!st) st = ws_get(ctx, WS_IN, sizeof(double) * nin, &din);
  if (!st) st = ws_get(ctx, WS_OUT, sizeof(double) * nout, &dout);
  if (!st) st = h2d_staged(ctx, din, rays, sizeof(double) * nin, "reduction input");
  if (!st)
    st = wrt_radon_reduction_device(ctx, static_cast<const double *>(din), ngrid, nshift_ray, grid,
                                    static_cast<double *>(dout));
  if (!st) st = d2h_staged_sync(ctx, out, dout, sizeof(double) * nout, "reduction result");
  return st;
}

int wrt_radon3d_adjoint_device(wrt_ctx *ctx, const double *dev_radon, const wrt_grid *grid,
                               int ngrid, double *dev_out) {
  if (!ctx || !dev_radon || !grid || !dev_out || grid->ctx != ctx || ngrid < 1 || ngrid > 4096 ||
      grid->nshift < 3)
    return ctx ? fail(ctx, WRT_ERR_INVALID_ARGUMENT, "radon3d_adjoint_device: bad arguments")
               : WRT_ERR_INVALID_ARGUMENT;
  int st = set_device(ctx);
  if (st) return st;
  return adjoint_forward(ctx, dev_radon, grid->nphi, grid->ntheta, grid->nshift, grid->d_dirw,
                         grid->dirw.data(), ngrid, dev_out);
}

int wrt_radon3d_adjoint(wrt_ctx *ctx, const double *radon, int nphi, int ntheta, int nshift,
                        int ngrid, double *out) {
  if (!ctx || !radon || !out || ngrid < 1 || ngrid > 4096 || nphi < 1 || ntheta < 1 || nshift < 3)
    return ctx ? fail(ctx, WRT_ERR_INVALID_ARGUMENT, "radon3d_adjoint: bad arguments")
               : WRT_ERR_INVALID_ARGUMENT;
  int st = set_device(ctx);
  if (st) return st;
  wrt_grid *grid = nullptr;
  void *din = nullptr, *dout = nullptr;
  const size_t nin = (size_t)nshift * nphi * ntheta, nout = (size_t)ngrid * ngrid * ngrid;
  st = dropin_grid(ctx, nphi, ntheta, nshift, &grid);
  if (!st) st = ws_get(ctx, WS_IN, sizeof(double) * nin, &din);
  if (!st) st = ws_get(ctx, WS_OUT, sizeof(double) * nout, &dout);
  if (!st) st = h2d_staged(ctx, din, radon, sizeof(double) * nin, "adjoint input");
  if (!st)
    st = wrt_radon3d_adjoint_device(ctx, static_cast<const double *>(din), grid, ngrid,
                                    static_cast<double *>(dout));
  if (!st) st = d2h_staged_sync(ctx, out, dout, sizeof(double) * nout, "adjoint result");
  return st;
}

}  // extern "C"
