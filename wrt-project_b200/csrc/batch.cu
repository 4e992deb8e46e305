// batch.cu -- many transform requests in one launch of a captured CUDA graph.
//
// The reference runs one transform per program invocation (radon_grid.c,
// radon3d_ajoint.c); a batch here holds up to kBatchMaxFwd plane-integral
// requests (volumes of any edge length, each with its own sphere grid and
// shifts) and kBatchMaxAdj backprojections.  All of it is described by one
// table in device memory (BatchLayout):
//
//   header | StagedReq[kBatchMaxFwd] | FwdAux[kBatchMaxFwd] | AdjReq[kBatchMaxAdj] |
//   RayJob[kBatchMaxRay] | RedReq[kBatchMaxRed] | items
//
// and executed by one graph, captured once per slot and replayed for every
// batch (only the size of its first node, the table upload, changes):
//
//   table H2D -> reset (outputs, statistics) -> volume prep (statistics and
//   layer pairs of freshly uploaded volumes) -> request prep (crop radius,
//   fixed-point scale) -> persistent staged plane kernel over the work items
//   of every forward request, largest first -> finalize (fixed point to FP64)
//   -> spline prep of every backprojection's lines -> every ray of the ray
//   requests -> spline prep of the reduction requests' ray lines -> every
//   Radon sample of the reduction requests;
//
// then, on the same stream, each backprojection's launches (its direction
// constants are launch parameters, which a graph replayed unchanged cannot
// carry).
//
// Every kernel has a fixed grid and reads its work from the table, which is
// what lets one captured graph serve batches of any composition.  A request's
// result is bitwise the same alone or in any batch: the plane sums are
// order-independent fixed-point integers, the backprojection of a voxel is one
// thread's sequential sum by the same kernel as a single request's, and a ray
// or a reduced Radon sample is one thread's sum by the single kernel's body.
#include <string.h>

#include <algorithm>
#include <vector>

#include "ray_dev.cuh"
#include "spline_dev.cuh"
#include "wrt_internal.cuh"

namespace {

using wrt::AdjReq;
using wrt::BatchHeader;
using wrt::BatchLayout;
using wrt::FwdAux;
using wrt::RayJob;
using wrt::RedReq;
using wrt::StagedReq;

__device__ __forceinline__ const BatchHeader *hdr(const char *t) {
  return reinterpret_cast<const BatchHeader *>(t);
}
__device__ __forceinline__ StagedReq *fwd_tab(char *t) {
  return reinterpret_cast<StagedReq *>(t + BatchLayout::fwd);
}
__device__ __forceinline__ FwdAux *aux_tab(char *t) {
  return reinterpret_cast<FwdAux *>(t + BatchLayout::aux);
}
__device__ __forceinline__ const AdjReq *adj_tab(const char *t) {
  return reinterpret_cast<const AdjReq *>(t + BatchLayout::adj);
}
__device__ __forceinline__ const RayJob *ray_tab(const char *t) {
  return reinterpret_cast<const RayJob *>(t + BatchLayout::ray);
}
__device__ __forceinline__ const RedReq *red_tab(const char *t) {
  return reinterpret_cast<const RedReq *>(t + BatchLayout::red);
}
// First index of request r's work for grid thread (or warp) g when the work
// of consecutive requests is numbered consecutively from `first` and dealt
// out round-robin over `nth` threads: small requests then leave no thread idle.
__device__ __forceinline__ long long dealt_first(long long g, long long first, long long nth) {
  long long k = g - first % nth;
  return k < 0 ? k + nth : k;
}

// Zero every forward output (the fixed-point accumulators) and the statistics
// of the volumes prepared in this launch.
__global__ void batch_reset_kernel(char *t) {
  const int nf = hdr(t)->nfwd;
  const StagedReq *F = fwd_tab(t);
  FwdAux *A = aux_tab(t);
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  for (int r = 0; r < nf; ++r) {
    unsigned long long *acc = F[r].acc;
    for (long long k = tid; k < A[r].nout; k += nth) acc[k] = 0ull;
    if (A[r].prep && tid < 2) A[r].stats[tid] = 0u;
  }
}

// Statistics (largest node radius^2 of a non-zero node, max |v|) and layer
// pairs of the volumes uploaded for this launch (same rules as k_volume.cu).
__global__ void batch_volume_kernel(char *t) {
  const int nf = hdr(t)->nfwd;
  const FwdAux *A = aux_tab(t);
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  for (int r = 0; r < nf; ++r) {
    if (!A[r].prep) continue;
    const int n = A[r].n, pitch = A[r].pitch;
    const float *v = A[r].vol;
    const long long total = (long long)n * n * n;
    float local = 0.0f, amax = 0.0f;
    for (long long k = tid; k < total; k += nth) {
      const float x = v[k];
      amax = fmaxf(amax, fabsf(x));
      if (x != 0.0f) {
        const int iz = (int)(k % n), iy = (int)((k / n) % n), ix = (int)(k / ((long long)n * n));
        local = fmaxf(local, wrtd::node_r2(ix, iy, iz, n));
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      local = fmaxf(local, __shfl_xor_sync(0xffffffffu, local, o));
      amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    }
    if ((threadIdx.x & 31) == 0) {
      if (local > 0.0f) atomicMax(A[r].stats, __float_as_uint(local));
      if (amax > 0.0f) atomicMax(A[r].stats + 1, __float_as_uint(amax));
    }
    float2 *pairs = A[r].pairs;
    const long long npairs = (long long)(n - 1) * n * pitch;
    for (long long k = tid; k < npairs; k += nth) {
      const int ix = (int)(k % pitch), iy = (int)((k / pitch) % n),
                iz = (int)(k / ((long long)pitch * n));
      float2 p = make_float2(0.0f, 0.0f);
      if (ix < n) {
        const float *q = v + ((size_t)ix * n + iy) * n + iz;
        p = make_float2(q[0], q[1]);
      }
      pairs[k] = p;
    }
  }
}

// Crop radius and fixed-point scale of every forward request from its
// volume's statistics (the same functions the host uses).
__global__ void batch_request_kernel(char *t) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= hdr(t)->nfwd) return;
  StagedReq *F = fwd_tab(t);
  FwdAux *A = aux_tab(t);
  const float r2 = __uint_as_float(A[r].stats[0]);
  const float maxabs = __uint_as_float(A[r].stats[1]);
  const int n = A[r].n;
  F[r].crop_r2 = wrt::trilinear_crop_r2(r2, n);
  F[r].guard = wrt::staged_guard(n, A[r].L, F[r].crop_r2);
  F[r].scale = wrt::fixed_point_scale(maxabs, A[r].L);
  const double delta = 1.0 / n;
  A[r].factor = delta * delta / F[r].scale;
}

// Fixed-point accumulators to FP64 plane integrals, in place.
__global__ void batch_finalize_kernel(char *t) {
  const int nf = hdr(t)->nfwd;
  const StagedReq *F = fwd_tab(t);
  const FwdAux *A = aux_tab(t);
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  for (int r = 0; r < nf; ++r) {
    double *out = reinterpret_cast<double *>(F[r].acc);
    const double f = A[r].factor;
    for (long long k = tid; k < A[r].nout; k += nth)
      out[k] = (double)reinterpret_cast<const long long *>(out)[k] * f;
  }
}

// Natural splines of every backprojection's lines (one thread per line).
__global__ void batch_spline_kernel(const char *t) {
  const int na = hdr(t)->nadj;
  const AdjReq *J = adj_tab(t);
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  for (int r = 0; r < na; ++r) {
    const int ns = J[r].nshift, nd = J[r].ndir;
    for (long long L = tid; L < nd; L += nth)
      wrtd::spline_line_centred(J[r].radon + L, nd, ns, 2.0 / (ns - 1), J[r].cp, J[r].den,
                                J[r].scratch + (size_t)L * ns, J[r].lines + (size_t)L * (ns - 1),
                                J[r].dirw[L].w);  // the direction's quadrature weight
  }
}

// Every ray of every ray-transform request (ray_grid/src/integral.c:11-50):
// consecutive threads take consecutive rays (32 shifts of one layer and angle).
__global__ void __launch_bounds__(256) batch_ray_kernel(const char *t) {
  const int nr = hdr(t)->nray;
  const RayJob *R = ray_tab(t);
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  long long first = 0;
  for (int r = 0; r < nr; ++r) {
    const RayJob &job = R[r];
    const long long total = (long long)job.nslices * job.nshift * job.nphi;
    const float g = wrtd::ray_guard(job.n);
    for (long long k = dealt_first(tid, first, nth); k < total; k += nth) {
      if (job.has_frame)
        wrtd::ray_one<true>(job, k, g);
      else
        wrtd::ray_one<false>(job, k, g);
    }
    first += total;
  }
}

// Natural splines of every reduction request's ray lines (one thread per line).
__global__ void batch_red_spline_kernel(const char *t) {
  const int nr = hdr(t)->nred;
  const RedReq *Q = red_tab(t);
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  for (int r = 0; r < nr; ++r) {
    const RedReq &q = Q[r];
    const int ns = q.ns_ray, nlines = q.ngrid * q.nphi;
    // line (iz, iphi): element is at rays[(iz*ns + is)*nphi + iphi]
    for (long long L = tid; L < nlines; L += nth) {
      const int outer = (int)(L / q.nphi), inner = (int)(L % q.nphi);
      wrtd::spline_line(q.rays + (size_t)outer * ns * q.nphi + inner, q.nphi, ns, 2.0 / (ns - 1),
                        q.coef, q.coef + ns, q.scratch + (size_t)L * ns,
                        q.lines + (size_t)L * (ns - 1));
    }
  }
}

// Every Radon sample of every reduction request (radon_reduction/slicing.c:80).
__global__ void __launch_bounds__(256) batch_reduction_kernel(const char *t) {
  const int nr = hdr(t)->nred;
  const RedReq *Q = red_tab(t);
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  long long first = 0;
  for (int r = 0; r < nr; ++r) {
    const RedReq &q = Q[r];
    const long long total = (long long)q.nshift * q.nphi * q.ntheta;
    for (long long t = dealt_first(tid, first, nth); t < total; t += nth) {
      const long long k = wrtd::reduction_sample_of(t, q.nshift, q.nphi, q.ntheta);
      int evaluated = 0;
      q.out[k] = wrtd::reduction_one(q.lines, q.ngrid, q.ns_ray, q.nphi, q.shift, q.cs, q.ntheta, k,
                                     &evaluated);
    }
    first += total;
  }
}

constexpr int kBatchKernels = 9;  // kernels per graph launch

}  // namespace

namespace wrt {

void staged_request(int n, int pitch, int ndir, int nshift, int L, int storage,
                    const void *pairs, const void *vol, const double *dir, const float *dir32,
                    const double *shift, const float *shift32, double *out, StagedReq *r) {
  int th = 0, qp = 0;
  staged_smem_bytes(n, &th, &qp);
  memset(r, 0, sizeof(*r));
  r->pairs = pairs;
  r->vol = vol;
  r->dir = dir;
  r->dir32 = dir32;
  r->shift = shift;
  r->shift32 = shift32;
  r->acc = reinterpret_cast<unsigned long long *>(out);
  r->n = n;
  r->pitch2 = pitch;
  r->qpitch = qp;
  r->tile_h = th;
  r->ndir = ndir;
  r->nshift = nshift;
  r->L = L;
  r->storage = storage;
  r->crop_r2 = 3.0f + 1e-5f;  // set from the volume statistics by the launch
  r->guard = staged_guard(n, L, r->crop_r2);
  r->scale = 1.0;
}

void batch_add_forward(BatchBuilder &b, const StagedReq &req, const FwdAux &aux,
                       float crop_items) {
  const int index = (int)b.fwd.size();
  b.fwd.push_back(req);
  b.aux.push_back(aux);
  staged_items_costed(index, req.n, req.tile_h, crop_items, req.ndir, kStagedDirChunk,
                      (double)req.nshift, b.items);
}

int batch_slot_init(wrt_ctx *ctx, BatchSlot *s, cudaStream_t stream) {
  s->ctx = ctx;
  s->stream = stream;
  cudaError_t e = cudaEventCreateWithFlags(&s->done, cudaEventDisableTiming);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch event");
  return ctx_alloc(ctx, (void **)&s->d_next, sizeof(int));
}

namespace {

void drop_graph(BatchSlot *s) {
  if (s->exec) cudaGraphExecDestroy(s->exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  s->exec = nullptr;
  s->graph = nullptr;
  s->copy_node = nullptr;
}

int ensure_capacity(BatchSlot *s, size_t bytes) {
  if (bytes <= s->cap) return WRT_OK;
  wrt_ctx *ctx = s->ctx;
  if (s->launched) cudaEventSynchronize(s->done);
  drop_graph(s);
  if (s->h_table) cudaFreeHost(s->h_table);
  s->h_table = nullptr;
  ctx_free(ctx, s->d_table, s->cap);
  s->d_table = nullptr;
  s->cap = 0;
  size_t cap = 1 << 20;
  while (cap < bytes) cap <<= 1;
  cudaError_t e = cudaMallocHost((void **)&s->h_table, cap);
  if (e != cudaSuccess) {
    cudaGetLastError();
    s->h_table = nullptr;
    return fail(ctx, WRT_ERR_OUT_OF_MEMORY, "batch table: cudaMallocHost(%zu)", cap);
  }
  int st = ctx_alloc(ctx, (void **)&s->d_table, cap);
  if (st) return st;
  s->cap = cap;
  return WRT_OK;
}

int capture(BatchSlot *s) {
  wrt_ctx *ctx = s->ctx;
  drop_graph(s);
  const uint64_t launches = ctx->launches;
  const int g = ctx->sm_count * 4;
  cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch capture begin");
  int st = WRT_OK;
  e = cudaMemcpyAsync(s->d_table, s->h_table, s->cap, cudaMemcpyHostToDevice, s->stream);
  if (e != cudaSuccess) st = cuda_fail(ctx, e, "batch table upload");
  if (!st) {
    batch_reset_kernel<<<g, 256, 0, s->stream>>>(s->d_table);
    batch_volume_kernel<<<g, 256, 0, s->stream>>>(s->d_table);
    batch_request_kernel<<<(kBatchMaxFwd + 127) / 128, 128, 0, s->stream>>>(s->d_table);
    st = plane_staged_launch(ctx, s->stream,
                             reinterpret_cast<const StagedReq *>(s->d_table + BatchLayout::fwd),
                             reinterpret_cast<const StagedItem *>(s->d_table + BatchLayout::items),
                             &reinterpret_cast<const BatchHeader *>(s->d_table)->nitems,
                             kStagedSmemMax, s->d_next);
  }
  if (!st) {
    batch_finalize_kernel<<<g, 256, 0, s->stream>>>(s->d_table);
    batch_spline_kernel<<<g, 128, 0, s->stream>>>(s->d_table);
    batch_ray_kernel<<<g, 256, 0, s->stream>>>(s->d_table);
    batch_red_spline_kernel<<<g, 128, 0, s->stream>>>(s->d_table);
    batch_reduction_kernel<<<g, 256, 0, s->stream>>>(s->d_table);
    e = cudaGetLastError();
    if (e != cudaSuccess) st = cuda_fail(ctx, e, "batch kernels");
  }
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(s->stream, &graph);
  ctx->launches = launches;
  if (st) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch capture end");
  s->graph = graph;
  size_t nnodes = 0;
  cudaGraphGetNodes(graph, nullptr, &nnodes);
  std::vector<cudaGraphNode_t> nodes(nnodes);
  cudaGraphGetNodes(graph, nodes.data(), &nnodes);
  for (auto nd : nodes) {
    cudaGraphNodeType ty;
    if (cudaGraphNodeGetType(nd, &ty) == cudaSuccess && ty == cudaGraphNodeTypeMemcpy) {
      s->copy_node = nd;
      break;
    }
  }
  if (!s->copy_node) return fail(ctx, WRT_ERR_INTERNAL, "batch graph: no table upload node");
  e = cudaGraphInstantiate(&s->exec, graph, 0);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch graph instantiate");
  s->config = ctx->staged_config;
  s->counting = ctx->d_counter != nullptr;
  return WRT_OK;
}

}  // namespace

int batch_slot_launch(BatchSlot *s, BatchBuilder &b) {
  wrt_ctx *ctx = s->ctx;
  if ((int)b.fwd.size() > kBatchMaxFwd || (int)b.adj.size() > kBatchMaxAdj ||
      (int)b.ray.size() > kBatchMaxRay || (int)b.red.size() > kBatchMaxRed)
    return fail(ctx, WRT_ERR_INVALID_ARGUMENT,
                "batch: more than %d forward, %d adjoint, %d ray or %d reduction requests",
                kBatchMaxFwd, kBatchMaxAdj, kBatchMaxRay, kBatchMaxRed);
  // the previous launch of this slot must have consumed the host table
  if (s->launched) {
    cudaError_t e = cudaEventSynchronize(s->done);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch slot wait");
  }
  const size_t bytes = BatchLayout::bytes(b.items.size());
  int st = ensure_capacity(s, bytes);
  if (st) return st;
  if (!s->exec || s->config != ctx->staged_config || s->counting != (ctx->d_counter != nullptr)) {
    st = capture(s);
    if (st) return st;
  }
  std::stable_sort(b.items.begin(), b.items.end(),
                   [](const std::pair<double, StagedItem> &x,
                      const std::pair<double, StagedItem> &y) { return x.first > y.first; });
  BatchHeader h = {};
  h.nfwd = (int)b.fwd.size();
  h.nadj = (int)b.adj.size();
  h.nitems = (int)b.items.size();
  h.nray = (int)b.ray.size();
  h.nred = (int)b.red.size();
  memset(s->h_table, 0, BatchLayout::items);
  memcpy(s->h_table, &h, sizeof(h));
  if (!b.fwd.empty()) {
    memcpy(s->h_table + BatchLayout::fwd, b.fwd.data(), sizeof(StagedReq) * b.fwd.size());
    memcpy(s->h_table + BatchLayout::aux, b.aux.data(), sizeof(FwdAux) * b.aux.size());
  }
  if (!b.adj.empty())
    memcpy(s->h_table + BatchLayout::adj, b.adj.data(), sizeof(AdjReq) * b.adj.size());
  if (!b.ray.empty())
    memcpy(s->h_table + BatchLayout::ray, b.ray.data(), sizeof(RayJob) * b.ray.size());
  if (!b.red.empty())
    memcpy(s->h_table + BatchLayout::red, b.red.data(), sizeof(RedReq) * b.red.size());
  StagedItem *items = reinterpret_cast<StagedItem *>(s->h_table + BatchLayout::items);
  for (size_t i = 0; i < b.items.size(); ++i) items[i] = b.items[i].second;
  cudaError_t e = cudaGraphExecMemcpyNodeSetParams1D(s->exec, s->copy_node, s->d_table,
                                                     s->h_table, bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch table size");
  e = cudaGraphLaunch(s->exec, s->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch graph launch");
  e = cudaEventRecord(s->done, s->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch event");
  s->launched = true;
  ctx->launches += kBatchKernels;
  // the backprojections, behind the graph (which built their spline lines):
  // their direction constants travel as launch parameters
  for (const AdjReq &j : b.adj) {
    e = launch_adjoint(s->stream, j.lines, j.ndir, j.nshift, j.h_dirw, j.n, j.out, &ctx->launches);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch adjoint_kernel");
  }
  return WRT_OK;
}

void batch_slot_release(BatchSlot *s) {
  if (!s->ctx) return;
  if (s->launched) cudaEventSynchronize(s->done);
  drop_graph(s);
  if (s->h_table) cudaFreeHost(s->h_table);
  ctx_free(s->ctx, s->d_table, s->cap);
  ctx_free(s->ctx, s->d_next, sizeof(int));
  if (s->done) cudaEventDestroy(s->done);
  *s = BatchSlot();
}

}  // namespace wrt
