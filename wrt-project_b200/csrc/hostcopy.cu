// hostcopy.cu -- copies between the caller's (pageable) host arrays and the
// device for the host-array entry points: through two pinned chunk buffers
// per context, the host side of each chunk spread over a small pool of host
// threads, so the DMA of one chunk overlaps the host copy of the next.  A
// pageable cudaMemcpyAsync stages through the driver's buffers with one host
// thread; the drop-in calls move 8-17 MB each way at 128^3, which at that
// rate costs more than their kernels.  FP64 volumes are rounded to FP32 on
// the host while they are staged (round to nearest, as the device conversion
// does), which halves their upload.
#include <string.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

#include "wrt_internal.cuh"

namespace wrt {

namespace {
constexpr size_t kChunk = 4u << 20;     // bytes per pinned chunk buffer
constexpr size_t kPiece = 256u << 10;   // bytes per host task
constexpr size_t kStagedMin = 1u << 20; // smaller copies go straight through
}  // namespace

// A fixed set of worker threads; run() hands out task indices [0, count) of
// one job to them and to the calling thread and returns when every task has
// finished and no worker still holds the job.  Workers take the job only
// under the lock, while it is posted, so a worker that wakes late never sees
// a finished one.  One run() at a time (a context is used by one thread).
struct HostJob {
  void (*fn)(void *, int);
  void *arg;
  int count;
  std::atomic<int> next{0}, finished{0};
  int active = 0;  // workers holding the job (under the pool's lock)
};

struct HostPool {
  std::vector<std::thread> workers;
  std::mutex m;
  std::condition_variable wake, done;
  HostJob *job = nullptr;
  unsigned long generation = 0;
  bool stop = false;

  void work(HostJob *j) {
    for (;;) {
      const int i = j->next.fetch_add(1);
      if (i >= j->count) return;
      j->fn(j->arg, i);
      if (j->finished.fetch_add(1) + 1 == j->count) {
        std::lock_guard<std::mutex> g(m);
        done.notify_all();
      }
    }
  }
  void loop() {
    unsigned long seen = 0;
    for (;;) {
      HostJob *j;
      {
        std::unique_lock<std::mutex> l(m);
        wake.wait(l, [&] { return stop || (job && generation != seen); });
        if (stop) return;
        seen = generation;
        j = job;
        ++j->active;
      }
      work(j);
      std::lock_guard<std::mutex> g(m);
      if (--j->active == 0) done.notify_all();
    }
  }
  void run(int n, void (*f)(void *, int), void *a) {
    if (n <= 0) return;
    HostJob j;
    j.fn = f;
    j.arg = a;
    j.count = n;
    {
      std::lock_guard<std::mutex> g(m);
      job = &j;
      ++generation;
    }
    wake.notify_all();
    work(&j);
    std::unique_lock<std::mutex> l(m);
    done.wait(l, [&] { return j.finished.load() == n && j.active == 0; });
    job = nullptr;
  }
};

void host_pool_destroy(HostPool *p) {
  if (!p) return;
  {
    std::lock_guard<std::mutex> g(p->m);
    p->stop = true;
  }
  p->wake.notify_all();
  for (auto &t : p->workers) t.join();
  delete p;
}

namespace {

HostPool *pool_of(wrt_ctx *ctx) {
  if (!ctx->host_pool) {
    HostPool *p = new (std::nothrow) HostPool();
    if (!p) return nullptr;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned nw = std::min(15u, hw > 1 ? hw - 1 : 0u);  // plus the caller
    try {
      for (unsigned k = 0; k < nw; ++k) p->workers.emplace_back([p] { p->loop(); });
    } catch (...) {
      host_pool_destroy(p);
      return nullptr;
    }
    ctx->host_pool = p;
  }
  return ctx->host_pool;
}

// The first large copy of a context goes through pageable memory: pinning the
// chunk buffers and starting the threads costs ~5-20 ms once, more than
// they save on one transfer (a program that runs one transform); from the
// second on, the pinned pipeline.
bool use_pageable(wrt_ctx *ctx) { return ctx->large_copies++ == 0; }

// two pinned chunk buffers and the events that mark the end of their DMA
int ensure_pinned(wrt_ctx *ctx) {
  if (ctx->pin[0]) return WRT_OK;
  for (int b = 0; b < 2; ++b) {
    cudaError_t e = cudaHostAlloc(&ctx->pin[b], kChunk, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->pin_ev[b], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->pin_ev[b], ctx->stream);
    if (e != cudaSuccess) {
      pinned_release(ctx);
      return cuda_fail(ctx, e, "pinned staging buffers");
    }
  }
  return WRT_OK;
}

struct CopyJob {
  char *dst;
  const char *src;
  size_t bytes;
};
void copy_piece(void *a, int i) {
  const CopyJob &j = *static_cast<const CopyJob *>(a);
  const size_t off = (size_t)i * kPiece;
  memcpy(j.dst + off, j.src + off, std::min(kPiece, j.bytes - off));
}
struct RoundJob {
  float *dst;
  const double *src;
  size_t count;
};
void round_piece(void *a, int i) {
  const RoundJob &j = *static_cast<const RoundJob *>(a);
  const size_t per = kPiece / sizeof(float);
  const size_t b = (size_t)i * per, e = std::min(j.count, b + per);
  for (size_t k = b; k < e; ++k) j.dst[k] = (float)j.src[k];
}

int pieces(size_t bytes) { return (int)((bytes + kPiece - 1) / kPiece); }

void host_copy(HostPool *p, void *dst, const void *src, size_t bytes) {
  CopyJob j{static_cast<char *>(dst), static_cast<const char *>(src), bytes};
  if (p) p->run(pieces(bytes), copy_piece, &j);
  else memcpy(dst, src, bytes);
}

}  // namespace

void pinned_release(wrt_ctx *ctx) {
  for (int b = 0; b < 2; ++b) {
    if (ctx->pin_ev[b]) {
      cudaEventSynchronize(ctx->pin_ev[b]);
      cudaEventDestroy(ctx->pin_ev[b]);
      ctx->pin_ev[b] = nullptr;
    }
    if (ctx->pin[b]) cudaFreeHost(ctx->pin[b]);
    ctx->pin[b] = nullptr;
  }
}

int h2d_staged(wrt_ctx *ctx, void *dst, const void *src, size_t bytes, const char *what) {
  if (bytes < kStagedMin || use_pageable(ctx)) {
    const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
    return e == cudaSuccess ? WRT_OK : cuda_fail(ctx, e, what);
  }
  int st = ensure_pinned(ctx);
  if (st) return st;
  HostPool *p = pool_of(ctx);
  for (size_t off = 0, c = 0; off < bytes; off += kChunk, ++c) {
    const size_t len = std::min(kChunk, bytes - off);
    const int b = (int)(c & 1);
    cudaError_t e = cudaEventSynchronize(ctx->pin_ev[b]);  // its previous DMA is done
    if (e != cudaSuccess) return cuda_fail(ctx, e, what);
    host_copy(p, ctx->pin[b], static_cast<const char *>(src) + off, len);
    e = cudaMemcpyAsync(static_cast<char *>(dst) + off, ctx->pin[b], len, cudaMemcpyHostToDevice,
                        ctx->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->pin_ev[b], ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, what);
  }
  return WRT_OK;
}

int h2d_staged_rounded(wrt_ctx *ctx, float *dst, const double *src, size_t count,
                       const char *what) {
  if (use_pageable(ctx)) {
    // rounded into a temporary host array, then one pageable copy (which
    // returns once the data is staged)
    std::vector<float> tmp;
    try {
      tmp.resize(count);
    } catch (...) {
      return fail(ctx, WRT_ERR_OUT_OF_MEMORY, "%s: host buffer", what);
    }
    for (size_t k = 0; k < count; ++k) tmp[k] = (float)src[k];
    const cudaError_t e = cudaMemcpyAsync(dst, tmp.data(), count * sizeof(float),
                                          cudaMemcpyHostToDevice, ctx->stream);
    return e == cudaSuccess ? WRT_OK : cuda_fail(ctx, e, what);
  }
  int st = ensure_pinned(ctx);
  if (st) return st;
  HostPool *p = pool_of(ctx);
  const size_t per = kChunk / sizeof(float);  // values per chunk
  for (size_t off = 0, c = 0; off < count; off += per, ++c) {
    const size_t len = std::min(per, count - off);
    const int b = (int)(c & 1);
    cudaError_t e = cudaEventSynchronize(ctx->pin_ev[b]);
    if (e != cudaSuccess) return cuda_fail(ctx, e, what);
    RoundJob j{static_cast<float *>(ctx->pin[b]), src + off, len};
    if (p) p->run(pieces(len * sizeof(float)), round_piece, &j);
    else
      for (size_t k = 0; k < len; ++k) j.dst[k] = (float)j.src[k];
    e = cudaMemcpyAsync(dst + off, ctx->pin[b], len * sizeof(float), cudaMemcpyHostToDevice,
                        ctx->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->pin_ev[b], ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, what);
  }
  return WRT_OK;
}

int d2h_staged_sync(wrt_ctx *ctx, void *dst, const void *src, size_t bytes, const char *what) {
  if (bytes < kStagedMin || use_pageable(ctx)) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? WRT_OK : cuda_fail(ctx, e, what);
  }
  int st = ensure_pinned(ctx);
  if (st) return st;
  HostPool *p = pool_of(ctx);
  const size_t nch = (bytes + kChunk - 1) / kChunk;
  auto issue = [&](size_t c) {
    const size_t off = c * kChunk, len = std::min(kChunk, bytes - off);
    const int b = (int)(c & 1);
    cudaError_t e = cudaMemcpyAsync(ctx->pin[b], static_cast<const char *>(src) + off, len,
                                    cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->pin_ev[b], ctx->stream);
    return e;
  };
  cudaError_t e = issue(0);
  if (e == cudaSuccess && nch > 1) e = issue(1);
  for (size_t c = 0; c < nch && e == cudaSuccess; ++c) {
    const int b = (int)(c & 1);
    e = cudaEventSynchronize(ctx->pin_ev[b]);
    if (e != cudaSuccess) break;
    const size_t off = c * kChunk, len = std::min(kChunk, bytes - off);
    host_copy(p, static_cast<char *>(dst) + off, ctx->pin[b], len);
    if (c + 2 < nch) e = issue(c + 2);  // buffer b is free again
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? WRT_OK : cuda_fail(ctx, e, what);
}

}  // namespace wrt
