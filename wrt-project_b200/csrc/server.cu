// server.cu -- the serving loop: continuous batching of transform requests.
//
// The reference answers one request per process run (a CLI invocation that
// reads text, transforms, writes text).  A wrt_server instead keeps a device
// context, the sphere-grid tables of the shapes it has seen and one arena of
// device memory (its HBM budget, reserved at start-up) resident, and runs two
// threads:
//
//   dispatcher  admits queued requests in arrival order while a launch slot is
//               free and the arena has room for their state, uploads their
//               inputs, and launches them together as ONE batch graph
//               (batch.cu: a persistent plane kernel over every forward
//               request's work items, then the backprojections);
//   completer   waits for launches in order, copies results to the callers'
//               buffers, releases their memory and wakes waiters.
//
// With max_inflight >= 2 a new batch is formed and queued on its own stream
// while the previous one runs: requests that arrive while others are on the
// GPU are admitted as slots and memory free up, and consecutive launches
// overlap on the device (the next graph's kernels start on SMs the previous
// persistent kernel has left).  A request's result does not depend on its
// batch: the plane sums are order-independent fixed-point integers and a
// voxel's backprojection is one thread's sequential sum.
#include <math.h>
#include <string.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "arena.h"
#include "wrt_internal.cuh"

namespace {

using wrt::Arena;
using Clock = std::chrono::steady_clock;

size_t al(size_t b) { return Arena::round_up(b); }

// Device tables of one sphere-grid shape, in one arena block.
struct GridTables {
  size_t off = 0, bytes = 0;
  double *dir = nullptr;     // [ndir][9]
  float *dir32 = nullptr;    // [ndir][8]
  double *shift = nullptr;   // [nshift]
  float *shift32 = nullptr;  // [nshift]
  double4 *dirw = nullptr;   // [ndir]
  std::vector<double4> h_dirw;  // host copy (backprojection launch parameters)
  double *cp = nullptr, *den = nullptr;  // [nshift]
  double *cs = nullptr;      // [ntheta][2]: cos, sin theta (reduction)
  int nphi = 0, ntheta = 0, nshift = 0;
  int refs = 0;
  uint64_t last_use = 0;
};

struct Request {
  uint64_t id = 0;
  wrt_request req = {};
  int status = WRT_OK;
  bool done = false;
  int batch_size = 0;
  double t_submit = 0, t_start = 0, t_done = 0;
  size_t off = 0, bytes = 0;  // arena block
  bool has_block = false;
  GridTables *grid = nullptr;
  bool out_pinned = false;
  // device pointers inside the block
  void *d_in = nullptr;
  double *d_out = nullptr;
  size_t in_bytes = 0, out_bytes = 0;
  // ray and reduce requests: small host tables uploaded beside the input
  // (ray: shifts and trig; reduce: spline coefficients) and the ray frame
  std::vector<double> tab;
  void *d_tab = nullptr;
  double frame[9] = {};
  bool has_frame = false;
};

struct Slot {
  wrt::BatchSlot batch;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  bool busy = false;
  std::vector<Request *> reqs;
};

}  // namespace

struct wrt_server {
  wrt_ctx *ctx = nullptr;
  wrt_server_opts opts = {};
  char *arena_base = nullptr;
  Arena arena;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Request *> arrivals;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  std::map<std::tuple<int, int, int>, GridTables> grids;
  std::vector<std::unique_ptr<Slot>> slots;
  std::deque<Slot *> inflight;
  std::thread dispatcher, completer;
  cudaStream_t copy_stream = nullptr;
  bool stop = false;
  uint64_t next_id = 1, use_clock = 0;
  wrt_server_stats stats = {};
  Clock::time_point t0;
  double now_ms() const {
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
  }
};

namespace {

// ---------------------------------------------------------------- sizes
size_t forward_pitch(int n) { return (size_t)n + (n & 1); }

size_t ray_table_len(const wrt_request &r) { return (size_t)r.nshift + 4 * (size_t)r.nphi; }

size_t request_bytes(const wrt_request &r) {
  const size_t nplanes = (size_t)r.nphi * r.ntheta * r.nshift;
  const size_t n = (size_t)r.ngrid;
  const size_t vol_state = al(4 * n * n * n) + al(8 * (n - 1) * n * forward_pitch((int)n)) + al(8);
  if (r.op == WRT_OP_FORWARD) return vol_state + al(8 * nplanes);
  if (r.op == WRT_OP_RAY)
    return vol_state + al(8 * ray_table_len(r)) +
           al(8 * (size_t)r.nslices * r.nshift * r.nphi);
  if (r.op == WRT_OP_REDUCE) {
    const size_t nlines = n * r.nphi, nsr = (size_t)r.nshift_ray;
    return al(8 * nlines * nsr) + al(16 * nsr) + al(8 * nlines * nsr) +
           al(16 * nlines * (nsr - 1)) + al(8 * nplanes);
  }
  const size_t ndir = (size_t)r.nphi * r.ntheta;
  return al(8 * nplanes) + al(8 * ndir * r.nshift) + al(16 * ndir * (r.nshift - 1)) +
         al(8 * n * n * n);
}

size_t grid_bytes(int nphi, int ntheta, int nshift) {
  const size_t ndir = (size_t)nphi * ntheta;
  return al(72 * ndir) + al(32 * ndir) + al(8 * (size_t)nshift) + al(4 * (size_t)nshift) +
         al(32 * ndir) + 2 * al(8 * (size_t)nshift) + al(16 * (size_t)ntheta);
}

// ---------------------------------------------------------------- grids
int make_grid(wrt_server *s, GridTables &g) {
  wrt_ctx *ctx = s->ctx;
  const int nphi = g.nphi, ntheta = g.ntheta, nshift = g.nshift;
  const size_t ndir = (size_t)nphi * ntheta;
  std::vector<double> phi(nphi), theta(ntheta), w(ntheta), shift(nshift);
  int st = wrt::sphere_grid(ctx, nphi, ntheta, nshift, phi.data(), theta.data(), w.data(),
                            shift.data());
  if (st) return st;
  std::vector<double> dir(ndir * 9);
  std::vector<float> dir32(ndir * 8), shift32(nshift);
  wrt::plane_directions(nphi, phi.data(), ntheta, theta.data(), dir.data());
  for (size_t d = 0; d < ndir; ++d)
    for (int k = 0; k < 8; ++k) dir32[8 * d + k] = (float)dir[9 * d + k];
  for (int i = 0; i < nshift; ++i) shift32[i] = (float)shift[i];
  // backprojection weights (backprojection/C/src/integral.c:11-18) and the
  // natural-spline elimination coefficients
  std::vector<double4> &dirw = g.h_dirw;
  dirw.resize(ndir);
  wrt::adjoint_directions(nphi, ntheta, nshift, phi.data(), theta.data(), w.data(), dirw.data());
  std::vector<double> cp(nshift), den(nshift);
  wrt::spline_coefficients(nshift, cp.data(), den.data());
  std::vector<double> cs(2 * (size_t)ntheta);
  for (int i = 0; i < ntheta; ++i) {
    cs[2 * i] = cos(theta[i]);  // slicing.c:104-105 evaluate cos/sin(p_theta)
    cs[2 * i + 1] = sin(theta[i]);
  }
  char *b = s->arena_base + g.off;
  size_t o = 0;
  auto place = [&](size_t bytes) {
    char *p = b + o;
    o += al(bytes);
    return p;
  };
  g.dir = reinterpret_cast<double *>(place(72 * ndir));
  g.dir32 = reinterpret_cast<float *>(place(32 * ndir));
  g.shift = reinterpret_cast<double *>(place(8 * (size_t)nshift));
  g.shift32 = reinterpret_cast<float *>(place(4 * (size_t)nshift));
  g.dirw = reinterpret_cast<double4 *>(place(32 * ndir));
  g.cp = reinterpret_cast<double *>(place(8 * (size_t)nshift));
  g.den = reinterpret_cast<double *>(place(8 * (size_t)nshift));
  g.cs = reinterpret_cast<double *>(place(16 * (size_t)ntheta));
  struct {
    void *dst;
    const void *src;
    size_t bytes;
  } copies[] = {{g.dir, dir.data(), 72 * ndir},          {g.dir32, dir32.data(), 32 * ndir},
                {g.shift, shift.data(), 8 * (size_t)nshift}, {g.shift32, shift32.data(), 4 * (size_t)nshift},
                {g.dirw, dirw.data(), 32 * ndir},         {g.cp, cp.data(), 8 * (size_t)nshift},
                {g.den, den.data(), 8 * (size_t)nshift},  {g.cs, cs.data(), 16 * (size_t)ntheta}};
  for (auto &c : copies) {
    cudaError_t e = cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return wrt::cuda_fail(ctx, e, "server grid tables");
  }
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? WRT_OK : wrt::cuda_fail(ctx, e, "server grid tables");
}

// Drops the tables of shapes no admitted request uses.  Caller holds s->mu.
void evict_unused_grids(wrt_server *s) {
  for (auto it = s->grids.begin(); it != s->grids.end();) {
    if (it->second.refs == 0) {
      s->arena.release(it->second.off);
      it = s->grids.erase(it);
    } else {
      ++it;
    }
  }
}

// Grid tables for a request, created on first use.  Caller holds s->mu.
// Returns nullptr when the arena has no room (after evicting unused shapes).
GridTables *acquire_grid(wrt_server *s, const wrt_request &r, int *status) {
  const auto key = std::make_tuple(r.nphi, r.ntheta, r.nshift);
  auto it = s->grids.find(key);
  if (it == s->grids.end()) {
    const size_t bytes = grid_bytes(r.nphi, r.ntheta, r.nshift);
    size_t off = 0;
    if (!s->arena.alloc(bytes, &off)) {
      evict_unused_grids(s);
      if (!s->arena.alloc(bytes, &off)) return nullptr;
    }
    GridTables g;
    g.off = off;
    g.bytes = bytes;
    g.nphi = r.nphi;
    g.ntheta = r.ntheta;
    g.nshift = r.nshift;
    *status = make_grid(s, g);
    if (*status) {
      s->arena.release(off);
      return nullptr;
    }
    it = s->grids.emplace(key, g).first;
  }
  it->second.refs++;
  it->second.last_use = ++s->use_clock;
  return &it->second;
}

// Reserves a request's state in the arena.  Caller holds s->mu.
bool reserve(wrt_server *s, Request *q, int *status) {
  *status = WRT_OK;
  const bool needs_grid = q->req.op != WRT_OP_RAY;
  GridTables *g = needs_grid ? acquire_grid(s, q->req, status) : nullptr;
  if (needs_grid && !g) return false;
  const size_t bytes = request_bytes(q->req);
  size_t off = 0;
  if (!s->arena.alloc(bytes, &off)) {
    if (g) g->refs--;
    evict_unused_grids(s);
    g = needs_grid ? acquire_grid(s, q->req, status) : nullptr;
    if (needs_grid && !g) return false;
    if (!s->arena.alloc(bytes, &off)) {
      if (g) g->refs--;
      return false;
    }
  }
  q->grid = g;
  q->off = off;
  q->bytes = bytes;
  q->has_block = true;
  const wrt_request &r = q->req;
  const size_t nplanes = (size_t)r.nphi * r.ntheta * r.nshift;
  const size_t n = (size_t)r.ngrid;
  char *b = s->arena_base + off;
  const size_t vol_state = al(4 * n * n * n) + al(8 * (n - 1) * n * forward_pitch((int)n)) + al(8);
  if (r.op == WRT_OP_FORWARD) {
    q->d_in = b;  // volume, then pairs, stats, output
    q->in_bytes = 4 * n * n * n;
    q->out_bytes = 8 * nplanes;
    q->d_out = reinterpret_cast<double *>(b + vol_state);
  } else if (r.op == WRT_OP_RAY) {
    q->d_in = b;  // volume, then pairs, stats, tables, output
    q->in_bytes = 4 * n * n * n;
    q->d_tab = b + vol_state;
    q->tab.resize(ray_table_len(r));
    wrt::ray_tables(r.nshift, r.nphi, q->tab.data());
    q->out_bytes = 8 * (size_t)r.nslices * r.nshift * r.nphi;
    q->d_out = reinterpret_cast<double *>(b + vol_state + al(8 * ray_table_len(r)));
  } else if (r.op == WRT_OP_REDUCE) {
    const size_t nlines = n * r.nphi, nsr = (size_t)r.nshift_ray;
    q->d_in = b;  // ray data, then spline coefficients, scratch, lines, output
    q->in_bytes = 8 * nlines * nsr;
    q->d_tab = b + al(8 * nlines * nsr);
    q->tab.resize(2 * nsr);
    wrt::spline_coefficients((int)nsr, q->tab.data(), q->tab.data() + nsr);
    q->out_bytes = 8 * nplanes;
    q->d_out = reinterpret_cast<double *>(b + al(8 * nlines * nsr) + al(16 * nsr) +
                                          al(8 * nlines * nsr) + al(16 * nlines * (nsr - 1)));
  } else {
    const size_t ndir = (size_t)r.nphi * r.ntheta;
    q->d_in = b;  // radon data, then spline scratch, lines, output
    q->in_bytes = 8 * nplanes;
    q->out_bytes = 8 * n * n * n;
    q->d_out = reinterpret_cast<double *>(b + al(8 * nplanes) + al(8 * ndir * r.nshift) +
                                          al(16 * ndir * (r.nshift - 1)));
  }
  return true;
}

void unreserve(wrt_server *s, Request *q) {
  if (q->has_block) s->arena.release(q->off);
  q->has_block = false;
  if (q->grid) q->grid->refs--;
  q->grid = nullptr;
}

bool is_pinned(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Adds an admitted request to the batch being built.
void add_to_batch(wrt_server *s, Request *q, wrt::BatchBuilder &b) {
  const wrt_request &r = q->req;
  const GridTables *g = q->grid;
  const int n = r.ngrid;
  const int ndir = r.nphi * r.ntheta;
  char *base = static_cast<char *>(q->d_in);
  if (r.op == WRT_OP_RAY) {
    // the volume is prepared (statistics, layer pairs) by the batch's volume
    // kernel through a forward entry with no planes and no work items
    const size_t nn = (size_t)n;
    float *vol = reinterpret_cast<float *>(base);
    float2 *pairs = reinterpret_cast<float2 *>(base + al(4 * nn * nn * nn));
    unsigned int *stats = reinterpret_cast<unsigned int *>(
        base + al(4 * nn * nn * nn) + al(8 * (nn - 1) * nn * forward_pitch(n)));
    wrt::StagedReq sr;
    wrt::staged_request(n, (int)forward_pitch(n), 0, 0, 2 * n, WRT_STORAGE_F32, pairs, vol,
                        nullptr, nullptr, nullptr, nullptr, nullptr, &sr);
    wrt::FwdAux a = {};
    a.vol = vol;
    a.pairs = pairs;
    a.stats = stats;
    a.nout = 0;
    a.n = n;
    a.pitch = (int)forward_pitch(n);
    a.L = 2 * n;
    a.prep = 1;
    b.fwd.push_back(sr);
    b.aux.push_back(a);
    wrt::RayJob job = {};
    job.vol = vol;
    job.n = n;
    job.nslices = r.nslices;
    job.nshift = r.nshift;
    job.nphi = r.nphi;
    job.shift = static_cast<const double *>(q->d_tab);
    job.trig = static_cast<const double *>(q->d_tab) + r.nshift;
    job.has_frame = q->has_frame ? 1 : 0;
    for (int k = 0; k < 9; ++k) job.frame[k] = q->frame[k];
    job.r2bits = stats;
    job.margin = wrt::trilinear_margin(n);
    job.out = q->d_out;
    if (!q->has_frame) {  // z-slices read the layer pairs
      job.pairs = pairs;
      job.pitch = (int)forward_pitch(n);
    }
    b.ray.push_back(job);
    return;
  }
  if (r.op == WRT_OP_REDUCE) {
    const size_t nlines = (size_t)n * r.nphi, nsr = (size_t)r.nshift_ray;
    wrt::RedReq rq = {};
    rq.rays = reinterpret_cast<const double *>(base);
    rq.coef = static_cast<const double *>(q->d_tab);
    rq.scratch = reinterpret_cast<double *>(base + al(8 * nlines * nsr) + al(16 * nsr));
    rq.lines = reinterpret_cast<float4 *>(base + al(8 * nlines * nsr) + al(16 * nsr) +
                                          al(8 * nlines * nsr));
    rq.shift = g->shift;
    rq.cs = g->cs;
    rq.out = q->d_out;
    rq.ngrid = n;
    rq.ns_ray = (int)nsr;
    rq.nphi = r.nphi;
    rq.nshift = r.nshift;
    rq.ntheta = r.ntheta;
    b.red.push_back(rq);
    return;
  }
  if (r.op == WRT_OP_FORWARD) {
    const size_t nn = (size_t)n;
    float *vol = reinterpret_cast<float *>(base);
    float2 *pairs = reinterpret_cast<float2 *>(base + al(4 * nn * nn * nn));
    unsigned int *stats = reinterpret_cast<unsigned int *>(
        base + al(4 * nn * nn * nn) + al(8 * (nn - 1) * nn * forward_pitch(n)));
    const int L = r.half_extent ? r.half_extent : 2 * n;
    wrt::StagedReq sr;
    wrt::staged_request(n, (int)forward_pitch(n), ndir, r.nshift, L, WRT_STORAGE_F32, pairs,
                        vol, g->dir, g->dir32, g->shift, g->shift32, q->d_out, &sr);
    wrt::FwdAux a = {};
    a.vol = vol;
    a.pairs = pairs;
    a.stats = stats;
    a.nout = (long long)ndir * r.nshift;
    a.n = n;
    a.pitch = (int)forward_pitch(n);
    a.L = L;
    a.prep = 1;
    wrt::batch_add_forward(b, sr, a, 3.0f + 1e-5f);
  } else {
    const size_t nplanes = (size_t)ndir * r.nshift;
    wrt::AdjReq j = {};
    j.radon = reinterpret_cast<const double *>(base);
    j.scratch = reinterpret_cast<double *>(base + al(8 * nplanes));
    j.lines = reinterpret_cast<float4 *>(base + al(8 * nplanes) + al(8 * (size_t)ndir * r.nshift));
    j.out = q->d_out;
    j.dirw = g->dirw;
    j.h_dirw = g->h_dirw.data();
    j.cp = g->cp;
    j.den = g->den;
    j.ndir = ndir;
    j.ntheta = r.ntheta;
    j.nshift = r.nshift;
    j.n = n;
    b.adj.push_back(j);
  }
}

void finish(wrt_server *s, Request *q, int status, double t) {
  q->status = status;
  q->done = true;
  q->t_done = t;
  unreserve(s, q);
  if (status == WRT_OK) s->stats.completed++;
  else s->stats.failed++;
}

void dispatch_loop(wrt_server *s) {
  cudaSetDevice(s->ctx->device);
  wrt::BatchBuilder b;
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    Slot *slot = nullptr;
    s->cv.wait(lk, [&] {
      if (s->stop) return true;
      if (s->arrivals.empty()) return false;
      for (auto &sl : s->slots)
        if (!sl->busy) return true;
      return false;
    });
    if (s->stop) break;
    for (auto &sl : s->slots)
      if (!sl->busy) {
        slot = sl.get();
        break;
      }
    // ---- admit in arrival order while memory allows
    std::vector<Request *> batch;
    const int max_batch = s->opts.max_batch;
    int nfwd = 0, nadj = 0, nray = 0, nred = 0;  // forward slots include ray volumes
    while (!s->arrivals.empty() && (int)batch.size() < max_batch) {
      Request *q = s->arrivals.front();
      const int op = q->req.op;
      if (((op == WRT_OP_FORWARD || op == WRT_OP_RAY) && nfwd >= wrt::kBatchMaxFwd) ||
          (op == WRT_OP_ADJOINT && nadj >= wrt::kBatchMaxAdj) ||
          (op == WRT_OP_RAY && nray >= wrt::kBatchMaxRay) ||
          (op == WRT_OP_REDUCE && nred >= wrt::kBatchMaxRed))
        break;
      int st = WRT_OK;
      if (!reserve(s, q, &st)) {
        if (st == WRT_OK && (!batch.empty() || !s->inflight.empty())) break;  // wait for memory
        s->arrivals.pop_front();
        finish(s, q, st ? st : WRT_ERR_BUDGET, s->now_ms());
        continue;
      }
      s->arrivals.pop_front();
      if (op == WRT_OP_FORWARD || op == WRT_OP_RAY) ++nfwd;
      if (op == WRT_OP_ADJOINT) ++nadj;
      if (op == WRT_OP_RAY) ++nray;
      if (op == WRT_OP_REDUCE) ++nred;
      batch.push_back(q);
    }
    if (batch.empty()) {
      s->cv.notify_all();  // failed requests wake their waiters
      if (!s->arrivals.empty()) s->cv.wait(lk);  // memory is held by launches in flight
      continue;
    }
    slot->busy = true;
    const double t_start = s->now_ms();
    lk.unlock();
    // ---- upload inputs, launch the batch graph, queue pinned result copies
    int st = WRT_OK;
    b.clear();
    for (Request *q : batch) {
      q->t_start = t_start;
      q->batch_size = (int)batch.size();
      q->out_pinned = is_pinned(q->req.out);
      const int op = q->req.op;
      const void *src = (op == WRT_OP_FORWARD || op == WRT_OP_RAY) ? (const void *)q->req.volume
                        : op == WRT_OP_REDUCE                     ? (const void *)q->req.rays
                                                                  : (const void *)q->req.radon;
      cudaError_t e = cudaMemcpyAsync(q->d_in, src, q->in_bytes, cudaMemcpyHostToDevice,
                                      slot->stream);
      // small tables from pageable memory: staged before the call returns
      if (e == cudaSuccess && !q->tab.empty())
        e = cudaMemcpyAsync(q->d_tab, q->tab.data(), sizeof(double) * q->tab.size(),
                            cudaMemcpyHostToDevice, slot->stream);
      if (e != cudaSuccess && !st) st = wrt::cuda_fail(s->ctx, e, "server input upload");
      add_to_batch(s, q, b);
    }
    if (!st) st = wrt::batch_slot_launch(&slot->batch, b);
    if (!st) {
      for (Request *q : batch)
        if (q->out_pinned) {
          cudaError_t e = cudaMemcpyAsync(q->req.out, q->d_out, q->out_bytes,
                                          cudaMemcpyDeviceToHost, slot->stream);
          if (e != cudaSuccess && !st) st = wrt::cuda_fail(s->ctx, e, "server result copy");
        }
      cudaError_t e = cudaEventRecord(slot->ev, slot->stream);
      if (e != cudaSuccess && !st) st = wrt::cuda_fail(s->ctx, e, "server event");
    }
    lk.lock();
    if (st) {
      const double t = s->now_ms();
      for (Request *q : batch) finish(s, q, st, t);
      slot->busy = false;
      s->cv.notify_all();
      continue;
    }
    slot->reqs = batch;
    s->stats.launches++;
    s->inflight.push_back(slot);
    s->cv.notify_all();
  }
  // cancel what never got admitted
  const double t = s->now_ms();
  while (!s->arrivals.empty()) {
    Request *q = s->arrivals.front();
    s->arrivals.pop_front();
    finish(s, q, WRT_ERR_CANCELLED, t);
  }
  s->cv.notify_all();
}

void complete_loop(wrt_server *s) {
  cudaSetDevice(s->ctx->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    s->cv.wait(lk, [&] { return !s->inflight.empty() || s->stop; });
    if (s->inflight.empty()) {
      if (s->stop) break;
      continue;
    }
    Slot *slot = s->inflight.front();
    lk.unlock();
    int st = WRT_OK;
    cudaError_t e = cudaEventSynchronize(slot->ev);
    if (e != cudaSuccess) st = WRT_ERR_CUDA;
    std::vector<int> per(slot->reqs.size(), st);
    if (!st) {
      for (size_t k = 0; k < slot->reqs.size(); ++k) {
        Request *q = slot->reqs[k];
        if (q->out_pinned) continue;
        e = cudaMemcpyAsync(q->req.out, q->d_out, q->out_bytes, cudaMemcpyDeviceToHost,
                            s->copy_stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->copy_stream);
        if (e != cudaSuccess) per[k] = WRT_ERR_CUDA;
      }
    }
    const double t = s->now_ms();
    lk.lock();
    for (size_t k = 0; k < slot->reqs.size(); ++k) finish(s, slot->reqs[k], per[k], t);
    slot->reqs.clear();
    slot->busy = false;
    s->inflight.pop_front();
    s->cv.notify_all();
  }
}

}  // namespace

// ------------------------------------------------------------------ C ABI
extern "C" {

int wrt_server_create(const wrt_server_opts *opts, wrt_server **out) {
  if (!out) return WRT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  wrt_server_opts o = {};
  if (opts) o = *opts;
  if (o.max_batch <= 0) o.max_batch = 64;
  const int most = wrt::kBatchMaxFwd + wrt::kBatchMaxAdj + wrt::kBatchMaxRed;
  if (o.max_batch > most) o.max_batch = most;
  if (o.max_inflight <= 0) o.max_inflight = 2;
  if (o.max_inflight > 8) o.max_inflight = 8;
  if (o.queue_capacity <= 0) o.queue_capacity = 1 << 16;
  wrt_ctx *ctx = nullptr;
  int st = wrt_ctx_create(o.device, 0, &ctx);
  if (st) return st;
  wrt_server *s = new (std::nothrow) wrt_server();
  if (!s) {
    wrt_ctx_destroy(ctx);
    return WRT_ERR_OUT_OF_MEMORY;
  }
  s->ctx = ctx;
  s->t0 = Clock::now();
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  size_t budget = o.hbm_budget;
  if (budget == 0) {
    budget = (size_t)60 << 30;
    if (budget > free_b / 4 * 3) budget = free_b / 4 * 3;
  }
  o.hbm_budget = budget;
  s->opts = o;
  cudaError_t e = cudaMalloc((void **)&s->arena_base, budget);
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete s;
    wrt_ctx_destroy(ctx);
    return WRT_ERR_OUT_OF_MEMORY;
  }
  s->arena.reset(budget);
  s->stats.budget = budget;
  st = cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking) == cudaSuccess
           ? WRT_OK : WRT_ERR_CUDA;
  for (int k = 0; k < o.max_inflight && !st; ++k) {
    auto sl = std::make_unique<Slot>();
    if (cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&sl->ev, cudaEventDisableTiming) != cudaSuccess) {
      st = WRT_ERR_CUDA;
      break;
    }
    st = wrt::batch_slot_init(ctx, &sl->batch, sl->stream);
    s->slots.push_back(std::move(sl));
  }
  if (st) {
    s->stop = true;
    wrt_server_destroy(s);
    return st;
  }
  s->dispatcher = std::thread(dispatch_loop, s);
  s->completer = std::thread(complete_loop, s);
  *out = s;
  return WRT_OK;
}

int wrt_server_submit(wrt_server *s, const wrt_request *r, uint64_t *id) {
  if (!s || !r || !id) return WRT_ERR_INVALID_ARGUMENT;
  *id = 0;
  if (r->op < WRT_OP_FORWARD || r->op > WRT_OP_REDUCE) return WRT_ERR_INVALID_ARGUMENT;
  if (r->nphi < 1 || (r->op != WRT_OP_RAY && r->ntheta < 1) || !r->out)
    return WRT_ERR_INVALID_ARGUMENT;
  if ((long long)r->nphi * (r->op == WRT_OP_RAY ? 1 : r->ntheta) > (1 << 24))
    return WRT_ERR_INVALID_ARGUMENT;
  if (r->op == WRT_OP_RAY) {
    if (!r->volume || r->ngrid < 4 || r->ngrid > 2048 || r->nslices < 2 || r->nshift < 2 ||
        (long long)r->nslices * r->nshift * r->nphi > (1LL << 34))
      return WRT_ERR_INVALID_ARGUMENT;
  } else if (r->op == WRT_OP_REDUCE) {
    if (!r->rays || r->ngrid < 3 || r->ngrid > 4096 || r->nshift_ray < 3 || r->nshift < 2)
      return WRT_ERR_INVALID_ARGUMENT;
  } else if (r->op == WRT_OP_FORWARD) {
    int th = 0, qp = 0;
    if (!r->volume || r->ngrid < 4 || r->ngrid > 2048 || r->nshift < 2 ||
        wrt::staged_smem_bytes(r->ngrid, &th, &qp) <= 0 || r->half_extent < 0 ||
        r->half_extent > 8 * r->ngrid)
      return WRT_ERR_INVALID_ARGUMENT;
  } else {
    if (!r->radon || r->ngrid < 1 || r->ngrid > 2048 || r->nshift < 3) return WRT_ERR_INVALID_ARGUMENT;
  }
  const size_t need = request_bytes(*r) +
                      (r->op == WRT_OP_RAY ? 0 : grid_bytes(r->nphi, r->ntheta, r->nshift));
  auto q = std::make_unique<Request>();
  q->req = *r;
  if (r->op == WRT_OP_RAY && r->frame && !wrt::identity_frame(r->frame)) {
    q->has_frame = true;
    memcpy(q->frame, r->frame, sizeof(q->frame));
  }
  q->req.frame = nullptr;  // read here; the caller's array may go away
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return WRT_ERR_CANCELLED;
  if (need > s->arena.capacity()) return WRT_ERR_BUDGET;
  if ((int)s->arrivals.size() >= s->opts.queue_capacity) return WRT_ERR_QUEUE_FULL;
  q->id = s->next_id++;
  q->t_submit = s->now_ms();
  *id = q->id;
  s->arrivals.push_back(q.get());
  s->reqs.emplace(q->id, std::move(q));
  s->stats.submitted++;
  s->cv.notify_all();
  return WRT_OK;
}

int wrt_server_wait(wrt_server *s, uint64_t id, int timeout_ms, wrt_request_info *info) {
  if (!s) return WRT_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return WRT_ERR_NOT_FOUND;
  Request *q = it->second.get();
  auto ready = [&] { return q->done; };
  if (timeout_ms < 0) s->cv.wait(lk, ready);
  else if (!s->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return WRT_ERR_TIMEOUT;
  if (info) {
    info->status = q->status;
    info->batch_size = q->batch_size;
    info->tag = q->req.tag;
    info->submit_ms = q->t_submit;
    info->start_ms = q->t_start;
    info->done_ms = q->t_done;
  }
  const int st = q->status;
  s->reqs.erase(it);
  return st;
}

int wrt_server_get_stats(wrt_server *s, wrt_server_stats *out) {
  if (!s || !out) return WRT_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  out->bytes_in_use = s->arena.used();
  out->bytes_peak = s->arena.peak();
  out->queued = s->arrivals.size();
  out->in_flight = s->inflight.size();
  out->grid_shapes = s->grids.size();
  return WRT_OK;
}

int wrt_server_destroy(wrt_server *s) {
  if (!s) return WRT_ERR_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv.notify_all();
  }
  if (s->dispatcher.joinable()) s->dispatcher.join();
  if (s->completer.joinable()) s->completer.join();
  cudaSetDevice(s->ctx->device);
  for (auto &sl : s->slots) {
    if (sl->stream) cudaStreamSynchronize(sl->stream);
    wrt::batch_slot_release(&sl->batch);
    if (sl->ev) cudaEventDestroy(sl->ev);
    if (sl->stream) cudaStreamDestroy(sl->stream);
  }
  s->slots.clear();
  if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
  if (s->arena_base) cudaFree(s->arena_base);
  wrt_ctx_destroy(s->ctx);
  delete s;
  return WRT_OK;
}

}  // extern "C"
