// k_probe.cu -- shared-memory bandwidth microbenchmark.
//
// The plane and ray kernels are gathers: every trilinear sample reads eight
// staged voxel values (32 bytes) from on-chip memory, so their ceiling is the
// SM's shared-memory / L1 data bandwidth, not HBM.  This kernel measures that
// ceiling on the device at hand: every warp reads 16 bytes per lane from
// shared memory with consecutive lanes on consecutive 16-byte words (no bank
// conflicts), many times, on every SM.
#include "wrt_internal.cuh"

namespace {

constexpr int kWords = 4096;  // float4 words of shared memory per block (64 KB)
constexpr int kUnroll = 16;

__global__ void __launch_bounds__(1024) smem_read_kernel(int iters, float *sink) {
  extern __shared__ float4 buf[];
  for (int i = threadIdx.x; i < kWords; i += blockDim.x)
    buf[i] = make_float4((float)i, (float)(i + 1), (float)(i + 2), (float)(i + 3));
  __syncthreads();
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  const int warp_base = (threadIdx.x & ~31) * 2;
  const int lane = threadIdx.x & 31;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int w = (warp_base + (it * kUnroll + u) * 32 + lane) & (kWords - 1);
      const float4 v = buf[w];
      acc.x += v.x;
      acc.y += v.y;
      acc.z += v.z;
      acc.w += v.w;
    }
  }
  if (acc.x + acc.y + acc.z + acc.w == -1.0f) sink[threadIdx.x] = acc.x;  // keep the loads
}

}  // namespace

namespace wrt {

int smem_bandwidth(wrt_ctx *ctx, double *bytes_per_s) {
  const int threads = 1024, blocks = 2 * ctx->sm_count, iters = 2048;
  const size_t smem = sizeof(float4) * kWords;
  cudaError_t e = cudaFuncSetAttribute(smem_read_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "smem probe attribute");
  float *sink = nullptr;
  int st = ctx_alloc(ctx, (void **)&sink, sizeof(float) * threads);
  if (st) return st;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double best = 0.0;
  for (int rep = 0; rep < 4 && !st; ++rep) {
    cudaEventRecord(a, ctx->stream);
    smem_read_kernel<<<blocks, threads, smem, ctx->stream>>>(iters, sink);
    ctx->launches++;
    cudaEventRecord(b, ctx->stream);
    st = check_launch(ctx, "smem_read_kernel");
    if (st) break;
    e = cudaEventSynchronize(b);
    if (e != cudaSuccess) {
      st = cuda_fail(ctx, e, "smem probe");
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    const double bytes = (double)blocks * threads * iters * kUnroll * sizeof(float4);
    if (rep > 0 && ms > 0.f) best = fmax(best, bytes / (ms * 1e-3));
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  ctx_free(ctx, sink, sizeof(float) * threads);
  if (!st) *bytes_per_s = best;
  return st;
}

}  // namespace wrt
