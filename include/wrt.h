/* wrt.h -- C ABI of the B200 (sm_100a) grid-sampled 3D Radon / ray transform
 * library (libwrt.so).
 *
 * The reference (devhliu/wrt-project) has no library API: its hot path is
 * four command-line programs whose inner functions are
 *   plane_integral     radon_grid/src/integral.c:26
 *   ray_transform      ray_grid/src/integral.c:11
 *   radon_reduction    radon_reduction/slicing.c:80  (+ ray_interpolate :5)
 *   radon3d_adjoint    radon_inversion/backprojection/C/src/integral.c:6
 * each driven by an OpenMP loop nest over the whole output grid.  The entry
 * points below replace one such program's loop nest each (host buffers in,
 * host buffers out, same array orders as the programs' text files), plus
 * device-resident objects for serving.  Every call returns a wrt_status; no
 * call exits the process.  There is no CPU fallback: without a usable CUDA
 * device the calls fail with WRT_ERR_NO_DEVICE.  The drop-in entry points
 * keep their device buffers in the context between calls: a warm call of the
 * same or smaller sizes allocates no device memory.
 *
 * Array orders (flat, row-major):
 *   volume  v[ix][iy][iz]          (radon_grid/src/init.c:120-124)
 *   radon   R[is][iphi][itheta]    (radon_grid/src/radon_grid.c:248-258)
 *   rays    P[iz][is][iphi]        (ray_grid/src/ray_grid.c:246-255)
 *   adjoint A[iz][ix][iy]          (backprojection/C/src/radon3d_ajoint.c:240-254)
 *
 * Threading: a wrt_ctx is used by one host thread at a time.  A wrt_server
 * owns its own dispatcher and completion threads; wrt_server_submit/wait may
 * be called from any thread.
 */
#ifndef WRT_H
#define WRT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WRT_ABI_VERSION 2

typedef enum wrt_status {
  WRT_OK = 0,
  WRT_ERR_INVALID_ARGUMENT = 1, /* sizes, pointers or options out of range */
  WRT_ERR_OUT_OF_MEMORY = 2,    /* a device or pinned allocation failed */
  WRT_ERR_BUDGET = 3,           /* the request does not fit the HBM budget */
  WRT_ERR_CUDA = 4,             /* a CUDA runtime call failed */
  WRT_ERR_NO_DEVICE = 5,        /* no usable sm_100 device */
  WRT_ERR_TIMEOUT = 6,          /* a bounded wait ran out */
  WRT_ERR_QUEUE_FULL = 7,       /* the server's arrival queue is full */
  WRT_ERR_NOT_FOUND = 8,        /* unknown request id */
  WRT_ERR_CANCELLED = 9,        /* the request was cancelled */
  WRT_ERR_INTERNAL = 10
} wrt_status;

typedef enum wrt_sampler {
  WRT_SAMPLER_NEAREST = 0,   /* zero_interp, radon_grid/src/interp.c:63 (reference default) */
  WRT_SAMPLER_TRILINEAR = 1  /* cube_trilinear_interp, radon_grid/src/interp.c:25 */
} wrt_sampler;

typedef enum wrt_kernel {
  WRT_KERNEL_AUTO = 0,   /* the staged kernel (both samplers; volumes of edge >= 4),
                            else the plain one */
  WRT_KERNEL_PLAIN = 1,  /* one warp per plane, gathers through L1 */
  WRT_KERNEL_STAGED = 2  /* volume layers staged in shared memory, persistent CTAs:
                            trilinear from the layer pairs (FP32 or BF16 storage),
                            nearest from the z-major cell layers (FP32 storage) */
} wrt_kernel;

/* Options of the plane-integral transform.  Zero-initialised options give the
 * reference's radon_grid exactly: nearest sampler, lattice [-2n, 2n)^2 with
 * step 1/n (radon_grid/src/integral.c:38-44). */
typedef struct wrt_plane_opts {
  int sampler;     /* wrt_sampler */
  int half_extent; /* lattice indices i, j in [-L, L); 0 means L = 2n */
  int kernel;      /* wrt_kernel */
  int reserved[5];
} wrt_plane_opts;

typedef struct wrt_ctx wrt_ctx;
typedef struct wrt_volume wrt_volume;
typedef struct wrt_grid wrt_grid;

/* ---------------------------------------------------------------- context */
const char *wrt_status_string(int status);
int wrt_abi_version(void);
/* device: CUDA ordinal.  hbm_budget_bytes: cap on the device memory this
 * context may hold (0 = no cap beyond what the device has). */
int wrt_ctx_create(int device, size_t hbm_budget_bytes, wrt_ctx **out);
int wrt_ctx_destroy(wrt_ctx *ctx);
const char *wrt_ctx_last_error(const wrt_ctx *ctx);
int wrt_ctx_synchronize(wrt_ctx *ctx);
/* Bytes of device memory the context currently holds. */
size_t wrt_ctx_bytes_in_use(const wrt_ctx *ctx);
/* Number of this library's kernels launched by the context so far. */
uint64_t wrt_ctx_launch_count(const wrt_ctx *ctx);

/* ------------------------------------------------------------ sphere grid */
/* n-point Gauss-Legendre nodes (ascending) and weights on [-1,1], computed in
 * FP64 by Newton's method on the GPU.  Replaces gsl_integration_glfixed_*
 * (radon_grid/src/init.c:180-187). */
int wrt_gauss_legendre(wrt_ctx *ctx, int n, double *x, double *w);
/* The Gauss-uniform Radon grid of radon_grid_init (radon_grid/src/init.c:165)
 * with the latitude weights of backprojection/C/src/init.c:222-249.
 * theta_w may be NULL. */
int wrt_radon_grid_init(wrt_ctx *ctx, int nphi, int ntheta, int nshift, double *phi,
                        double *theta, double *theta_w, double *shift);

/* ------------------------------------------- drop-in transforms, host I/O */
/* radon_grid: out[is][iphi][itheta] = plane integral over the plane
 * (shift[is], phi[iphi], theta[itheta]).  Replaces radon_grid.c:229-264 with
 * plane_integral (radon_grid/src/integral.c:26-58).  opts may be NULL. */
int wrt_radon_grid(wrt_ctx *ctx, const double *volume, int ngrid, int nphi, int ntheta,
                   int nshift, const wrt_plane_opts *opts, double *out);

/* ray_grid: out[iz][is][iphi] = ray integral (ray_grid/src/integral.c:11-50,
 * loop nest ray_grid/src/ray_grid.c:225-262).  frame: NULL for the
 * reference's z-slices, else a row-major 3x3 rotation applied to every
 * sample point (layer-by-layer scheme about another axis). */
int wrt_ray_grid(wrt_ctx *ctx, const double *volume, int ngrid, int nslices, int nshift,
                 int nphi, const double *frame, double *out);

/* radon_reduction: rays in[iz][is_ray][iphi] (iz < ngrid, the z-slices) to
 * Radon data out[is][iphi][itheta] (radon_reduction/slicing.c:5-119, loop
 * nest reduction.c:195-235).  nshift == nshift_ray is the reference; a
 * different nshift samples the Radon shifts independently of the ray offsets. */
int wrt_radon_reduction(wrt_ctx *ctx, const double *rays, int ngrid, int nshift_ray,
                        int nphi, int nshift, int ntheta, double *out);

/* radon3d_grid (backprojection): out[iz][ix][iy] at the cell centres
 * (radon_inversion/backprojection/C/src/integral.c:6-24 with interp.c:5-28,
 * loop nest radon3d_ajoint.c:221-260). */
int wrt_radon3d_adjoint(wrt_ctx *ctx, const double *radon, int nphi, int ntheta,
                        int nshift, int ngrid, double *out);

/* The backprojection of wrt_radon3d_adjoint without allocating any device
 * memory.  No counterpart in the reference.  For callers that cannot call
 * cudaMalloc: programs that give all device memory to their own allocator or
 * reserve it up front, and latency-critical pipelines that forbid allocation
 * after start-up (cudaMalloc/cudaFree synchronise the device).  d_radon
 * (nshift*nphi*ntheta doubles, order [is][iphi][itheta]) and d_out (ngrid^3
 * doubles, order [iz][ix][iy]) are device buffers owned by the caller; the
 * working memory is one fixed ~6.8 MB array inside the library, held by every
 * GPU that loads the library until the process exits.  Limits: nphi*ntheta
 * <= 16384, ntheta <= 1024, 3 <= nshift <= 2048, nphi*ntheta*nshift <=
 * 262144; larger sizes return WRT_ERR_INVALID_ARGUMENT with a message.  The
 * first call on a device looks up the array's device address (make that first
 * call before any stream capture); creating a context forgets it again, so
 * after a device reset create new contexts before calling.  Asynchronous on
 * the context's stream.
 * Every call shares the array: calls whose GPU work overlaps (other streams,
 * other contexts on the same device) race and must be ordered by the caller. */
int wrt_radon3d_adjoint_static(wrt_ctx *ctx, const double *d_radon, int nphi, int ntheta,
                               int nshift, int ngrid, double *d_out);

/* Exact transpose of wrt_radon_grid with the same options: out_volume (n^3,
 * v[ix][iy][iz] order) = R^T g.  No counterpart in the reference; it makes
 * the adjoint identity <R f, g> = <f, R^T g> testable. */
int wrt_radon_transpose(wrt_ctx *ctx, const double *g, int ngrid, int nphi, int ntheta,
                        int nshift, const wrt_plane_opts *opts, double *out_volume);

/* Spectral Laplacian of an n^3 volume (any axis order, row-major) sampled on
 * a periodic cell of length `period` per axis: out = ifftn(U * fftn(in)),
 * U = -(2 pi / period)^2 (k1^2 + k2^2 + k3^2), k the FFT-order frequencies
 * (i for i <= n/2, i - n above); the result is real.  The step after the
 * backprojection in the reference's inversion (f = -1/(8 pi^2) * Laplacian of
 * the backprojection), radon_inversion/backprojection/laplace3dfft.m:1-25.
 * Host arrays in and out; FP64 FFTs on the device. */
int wrt_spectral_laplacian(wrt_ctx *ctx, const double *in, int n, double period, double *out);
/* The same on device buffers of n^3 doubles, asynchronous on the context's
 * stream (FFT plans and the spectrum live in the context). */
int wrt_spectral_laplacian_device(wrt_ctx *ctx, const double *dev_in, int n, double period,
                                  double *dev_out);

/* Inversion of Radon data R[is][iphi][itheta] on the Gauss-uniform sphere
 * grid (shifts uniform on [-rsupp, rsupp]) through the Fourier slice theorem:
 * the 1D Fourier transform of every projection along the shift, zero-padded
 * to padding * floor(1/ds) points (ds = 2 rsupp/(nshift - 1)), and the inverse
 * 3D Fourier integral in spherical coordinates, 1/2 sum nu^2 dnu dphi w_theta,
 * evaluated exactly at the ngrid^3 points -1 + 2 l/ngrid of [-1, 1)^3, order
 * [ix][iy][iz].  The reference's route is radon_inversion/rtft3d.m followed by
 * nfft_reconstruct_3d.m (an adjoint NFFT); here nodes carry physical
 * frequencies and the nonuniform sum is exact. */
int wrt_fourier_slice_inversion(wrt_ctx *ctx, const double *radon, int nphi, int ntheta,
                                int nshift, double rsupp, int padding, int ngrid, double *out);

/* ------------------------------------------- analytic test functions */
/* The reference's analytic-function programs (radon_analytic, ray_analytic)
 * integrate a function compiled into the binary; its two example files are
 * the families below, with their constants as parameters here. */
typedef enum wrt_function_kind {
  /* exp(-1 / (R2 - |x - c|^2)) where |x - c|^2 < R2 - eps, else 0
   * (radon_analytic/examples-test-functions/exponential_bump.c: c = (0.2, 0, 0),
   * R2 = 0.5, eps = 1e-2); p = {cx, cy, cz, R2, eps} */
  WRT_FUNCTION_EXP_BUMP = 0,
  /* sum of `count` balls, each amplitude inside rin, a sine transition
   * amplitude/(20 pi) (-sin 6t/3 + 3 sin 4t - 15 sin 2t + 20 t), t = pi (r - rout)/
   * (rout - rin), between rin and rout, 0 beyond (.../sinusoidal_bump.c);
   * p = {cx, cy, cz, amplitude, rin, rout} per ball */
  WRT_FUNCTION_SINE_BUMPS = 1
} wrt_function_kind;
#define WRT_FUNCTION_MAX_BALLS 8
typedef struct wrt_function {
  int kind;   /* wrt_function_kind */
  int count;  /* sine bumps: balls, 1..WRT_FUNCTION_MAX_BALLS */
  double p[6 * WRT_FUNCTION_MAX_BALLS];
} wrt_function;

/* radon_analytic: out[is][iphi][itheta] = plane integral of f over the
 * reference's lattice (radon_analytic/src/integral.c:25-57: points
 * s n + delta (i v1 + j v2), i, j in [-2n, 2n), delta = 1/(n - 1), weight
 * delta^2) on the Gauss-uniform sphere grid; loop nest
 * radon_analytic/src/radon_analytic.c:244-262. */
int wrt_radon_analytic(wrt_ctx *ctx, const wrt_function *f, int ngrid, int nphi, int ntheta,
                       int nshift, double *out);
/* ray_analytic: out[iz][is][iphi] = ray integral of f on z-slice
 * z = -1 + 2 iz/(n - 1), iz < n (ray_analytic/integral.c:10-48, loop nest
 * ray_analytic/ray_analytic.c:254-272). */
int wrt_ray_analytic(wrt_ctx *ctx, const wrt_function *f, int ngrid, int nshift, int nphi,
                     double *out);

/* ------------------------------------------------ device-resident objects */
typedef enum wrt_storage {
  WRT_STORAGE_F32 = 0, /* FP32 node values (default) */
  WRT_STORAGE_BF16 = 1 /* bfloat16 node values, FP32 arithmetic: half the device memory */
} wrt_storage;

/* A volume held on the device in the layouts the kernels read. */
int wrt_volume_create(wrt_ctx *ctx, int ngrid, wrt_volume **out);
/* The same with a storage precision (wrt_storage).  A BF16 volume rounds each
 * value to bfloat16 (nearest even) on upload; the trilinear sampler of the
 * staged kernel (single, batched) interpolates the rounded values in FP32,
 * the guard-band samples in FP64.  No counterpart in the reference (FP64). */
int wrt_volume_create_storage(wrt_ctx *ctx, int ngrid, int storage, wrt_volume **out);
/* Device bytes the volume holds (values, layer pairs once built, statistics). */
size_t wrt_volume_bytes(const wrt_volume *vol);
/* Upload from host memory (exactly one of f64 / f32 non-NULL), ordered on
 * the context's stream.  Pinned host memory makes the copy asynchronous. */
int wrt_volume_upload(wrt_volume *vol, const double *host_f64, const float *host_f32);
/* Upload from a device buffer of n^3 floats in v[ix][iy][iz] order. */
int wrt_volume_upload_device(wrt_volume *vol, const float *dev_f32);
int wrt_volume_destroy(wrt_volume *vol);

/* A sphere grid with its direction tables resident on the device. */
int wrt_grid_create(wrt_ctx *ctx, int nphi, int ntheta, int nshift, wrt_grid **out);
int wrt_grid_destroy(wrt_grid *grid);

/* Plane integrals of a resident volume into a device buffer of
 * nshift*nphi*ntheta doubles (same order as wrt_radon_grid).  Asynchronous on
 * the context's stream. */
int wrt_radon_forward_device(wrt_ctx *ctx, const wrt_volume *vol, const wrt_grid *grid,
                             const wrt_plane_opts *opts, double *dev_out);

/* Ray integrals of a resident FP32 volume into a device buffer of
 * nslices*nshift*nphi doubles, order [iz][is][iphi] as wrt_ray_grid.  frame:
 * NULL (the reference's z-slices) or a row-major 3x3 rotation in host memory.
 * Asynchronous on the context's stream; small tables and the volume's layer
 * pairs live in the context (no allocation once warm).  Device-resident form of
 * ray_grid/src/ray_grid.c:225-262 with ray_transform (integral.c:11-50). */
int wrt_ray_forward_device(wrt_ctx *ctx, const wrt_volume *vol, const double *frame,
                           int nslices, int nshift, int nphi, double *dev_out);

/* Reduction of device ray data dev_rays[iz][is_ray][iphi] (ngrid z-slices,
 * nshift_ray offsets, grid->nphi angles) to Radon data on a resident sphere
 * grid, dev_out[is][iphi][itheta] (nshift * nphi * ntheta doubles of the
 * grid).  Asynchronous; spline working memory lives in the context.
 * Device-resident form of radon_reduction/reduction.c:195-235 with
 * radon_reduction and ray_interpolate (slicing.c:5-119). */
int wrt_radon_reduction_device(wrt_ctx *ctx, const double *dev_rays, int ngrid, int nshift_ray,
                               const wrt_grid *grid, double *dev_out);

/* Backprojection of device Radon data dev_radon[is][iphi][itheta] on a
 * resident sphere grid into dev_out, ngrid^3 doubles [iz][ix][iy].
 * Asynchronous; spline working memory lives in the context.  Device-resident
 * form of backprojection/C/src/radon3d_ajoint.c:221-260 with radon3d_adjoint
 * (integral.c:6-24). */
int wrt_radon3d_adjoint_device(wrt_ctx *ctx, const double *dev_radon, const wrt_grid *grid,
                               int ngrid, double *dev_out);

/* One request of a batch: the plane integrals of a resident volume on a
 * resident sphere grid (trilinear sampler, lattice [-L, L)^2 with step 1/n,
 * L = half_extent or 2n when 0) into dev_out, nshift*nphi*ntheta doubles in
 * the order of wrt_radon_grid. */
typedef struct wrt_forward_req {
  const wrt_volume *volume;
  const wrt_grid *grid;
  int half_extent;
  int reserved;
  double *dev_out;
} wrt_forward_req;

/* Up to 256 forward requests (volumes of any edge length, each with its own
 * sphere grid) in ONE launch of the persistent staged kernel: the work items
 * of all requests are ordered by cost and shared by all SMs.  The launch
 * sequence (table upload, output reset, request set-up, plane kernel,
 * finalize) is a CUDA graph captured once per context and replayed with a new
 * request table.  Asynchronous on the context's stream.  Each result is
 * bitwise identical to what wrt_radon_forward_device gives for the same
 * request alone.  Batch transforms of the reference's loop nest
 * radon_grid/src/radon_grid.c:229-264, one per request. */
int wrt_radon_forward_batch(wrt_ctx *ctx, const wrt_forward_req *reqs, int nreq);

/* The context's CUDA stream (cudaStream_t), for callers that order their own
 * work against the library's. */
void *wrt_ctx_stream(wrt_ctx *ctx);

/* Autotuner of the staged plane kernel's tile shape (CTA size, lattice rows
 * walked together per warp, shifts enumerated per lane): runs every
 * configuration on this request (dev_out receives the result), times each
 * with CUDA events and keeps the fastest in the context.  *best / *best_ms
 * (either may be NULL) receive the chosen index and its time per launch. */
int wrt_tune_plane_kernel(wrt_ctx *ctx, const wrt_volume *vol, const wrt_grid *grid,
                          const wrt_plane_opts *opts, double *dev_out, int *best,
                          float *best_ms);
/* Number of tile configurations; their shapes; force one (-1: default). */
int wrt_plane_kernel_config_count(void);
int wrt_plane_kernel_config_describe(int index, int *threads, int *rows_per_group,
                                     int *shifts_per_lane);
int wrt_ctx_set_plane_kernel_config(wrt_ctx *ctx, int index);

/* Caller-owned device and pinned host memory, counted against the context's
 * budget (device) and released with the matching free. */
int wrt_device_alloc(wrt_ctx *ctx, size_t bytes, void **dev_ptr);
int wrt_device_free(wrt_ctx *ctx, void *dev_ptr);
int wrt_host_alloc_pinned(wrt_ctx *ctx, size_t bytes, void **host_ptr);
int wrt_host_free_pinned(wrt_ctx *ctx, void *host_ptr);
/* Copies ordered on the context's stream; the host array may be pageable.
 * The host-to-device copy returns once the host array has been read (the
 * transfer completes in stream order); the device-to-host copy waits. */
int wrt_copy_to_device(wrt_ctx *ctx, void *dev_dst, const void *host_src, size_t bytes);
int wrt_copy_to_host(wrt_ctx *ctx, void *host_dst, const void *dev_src, size_t bytes);

/* ---------------------------------------------------------------- serving */
/* A request loop for many callers: a wrt_server keeps its device context, the
 * sphere-grid tables of the shapes it has seen and one arena of device memory
 * (its HBM budget, reserved at creation) resident, admits queued requests in
 * arrival order as launch slots and memory free up, and runs each admitted
 * set as ONE batch launch (the graph of wrt_radon_forward_batch, plus the
 * backprojections).  With max_inflight >= 2 a batch is formed and queued
 * while the previous one runs (continuous batching).  A request's result is
 * bitwise the same whatever batch it runs in.  No counterpart in the
 * reference, whose programs answer one request per process run. */
typedef struct wrt_server wrt_server;

typedef enum wrt_op {
  WRT_OP_FORWARD = 0, /* plane integrals, trilinear sampler (radon_grid/src/integral.c:26) */
  WRT_OP_ADJOINT = 1, /* backprojection (radon_inversion/backprojection/C/src/integral.c:6) */
  WRT_OP_RAY = 2,     /* layer-by-layer ray integrals (ray_grid/src/integral.c:11) */
  WRT_OP_REDUCE = 3   /* ray data to Radon data (radon_reduction/slicing.c:80) */
} wrt_op;

typedef struct wrt_request {
  int op;              /* wrt_op */
  int ngrid;           /* n: edge of the input (forward, ray) or output (adjoint) volume;
                          reduce: z-slices of the ray data */
  int nphi, ntheta, nshift; /* sphere grid (forward, adjoint, reduce); ray: nphi angles and
                               nshift offsets per layer (ntheta unused) */
  int half_extent;     /* forward: lattice [-L, L)^2 with step 1/n; 0 means L = 2n */
  const float *volume; /* forward and ray input: n^3 FP32 values, v[ix][iy][iz] */
  const double *radon; /* adjoint input: nshift*nphi*ntheta values, [is][iphi][itheta] */
  double *out;         /* result: forward and reduce [is][iphi][itheta]; adjoint
                          [iz][ix][iy]; ray [iz][is][iphi] */
  uint64_t tag;        /* the caller's, returned in wrt_request_info */
  int nslices;         /* ray: layers (z-slices) */
  int nshift_ray;      /* reduce: offsets per ray line of the input */
  const double *rays;  /* reduce input: ngrid*nshift_ray*nphi values, [iz][is][iphi] */
  const double *frame; /* ray: NULL (the reference's z-slices) or a row-major 3x3 rotation of
                          the sample points, read at submission */
} wrt_request;

typedef struct wrt_request_info {
  int status;          /* wrt_status of the request */
  int batch_size;      /* requests in the launch that ran it */
  uint64_t tag;
  double submit_ms, start_ms, done_ms; /* server clock: submission, launch, result in out */
} wrt_request_info;

typedef struct wrt_server_opts {
  int device;          /* CUDA ordinal */
  int max_batch;       /* requests per launch (0: 64; at most 256 forward + 256 adjoint
                          + 64 ray + 64 reduce) */
  int max_inflight;    /* launches on the device at once (0: 2; at most 8) */
  int queue_capacity;  /* requests waiting for admission (0: 65536) */
  size_t hbm_budget;   /* device memory for request state and grid tables
                          (0: 60 GiB or 3/4 of the free memory, whichever is less) */
  int reserved[8];
} wrt_server_opts;

typedef struct wrt_server_stats {
  uint64_t submitted, completed, failed, launches;
  size_t budget, bytes_in_use, bytes_peak;
  size_t queued, in_flight, grid_shapes;
} wrt_server_stats;

/* opts may be NULL (defaults). */
int wrt_server_create(const wrt_server_opts *opts, wrt_server **out);
/* Queues a request (copied; the buffers it points to must stay valid until
 * wrt_server_wait returns for it).  Host buffers in pinned memory
 * (wrt_host_alloc_pinned) are copied asynchronously; pageable ones are copied
 * synchronously by the server's threads.  Returns WRT_ERR_QUEUE_FULL when the
 * queue is full, WRT_ERR_BUDGET when the request can never fit the budget. */
int wrt_server_submit(wrt_server *srv, const wrt_request *req, uint64_t *id);
/* Waits up to timeout_ms (< 0: without limit, 0: poll) for a request; on
 * completion fills info (may be NULL), forgets the id and returns the
 * request's status; WRT_ERR_TIMEOUT if it is still running.  Each id is
 * waited for once (a second wait returns WRT_ERR_NOT_FOUND); a request never
 * waited for keeps its record until wrt_server_destroy. */
int wrt_server_wait(wrt_server *srv, uint64_t id, int timeout_ms, wrt_request_info *info);
int wrt_server_get_stats(wrt_server *srv, wrt_server_stats *stats);
/* Finishes the launches in flight, cancels queued requests
 * (WRT_ERR_CANCELLED) and releases everything. */
int wrt_server_destroy(wrt_server *srv);

/* ------------------------------------------------------------ measurement */
/* CUDA-event timer on the context's stream: start records an event, stop
 * records a second one, waits for it and returns the elapsed milliseconds. */
int wrt_ctx_timer_start(wrt_ctx *ctx);
int wrt_ctx_timer_stop(wrt_ctx *ctx, float *ms);
/* Overwrite a device buffer larger than the L2 cache (evicts the volume). */
int wrt_ctx_flush_l2(wrt_ctx *ctx);
/* When on, the plane and ray kernels count the lattice samples they evaluate
 * (one atomic per plane or ray) and the reduction kernel the slice samples
 * (three spline evaluations each).  wrt_ctx_sample_count waits for the stream and returns
 * the running total. */
int wrt_ctx_count_samples(wrt_ctx *ctx, int on);
int wrt_ctx_sample_count(wrt_ctx *ctx, uint64_t *count);
/* Shared-memory read bandwidth of the whole device (bytes/s), measured by a
 * conflict-free 16-byte-per-lane load loop on every SM: the ceiling of the
 * gather kernels, whose samples read 32 bytes of staged volume each. */
int wrt_measure_smem_bandwidth(wrt_ctx *ctx, double *bytes_per_s);

#ifdef __cplusplus
}
#endif
#endif /* WRT_H */
