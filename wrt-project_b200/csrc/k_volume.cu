// k_volume.cu -- volume preparation.
//
// Input: the reference's node-sampled volume v[ix][iy][iz] (radon_grid/src/
// init.c:120-124), FP64 or FP32.  Output:
//   * d_vol    FP32 copy in the same order (gathers of the plain kernels and
//              the guard-band re-evaluation);
//   * stats[1] the largest |value| (float bits), which sizes the fixed-point
//              accumulators of the staged kernel;
//   * stats[0] the largest squared radius |x|^2 of a non-zero node, as the
//              bit pattern of a non-negative float (monotone under integer
//              max).  Every lattice sample farther than sqrt(r2) + sqrt(3)
//              delta from the origin has only zero corners, so it contributes
//              exactly 0; the kernels skip those samples.  This is exact for
//              any input, not an assumption about the support.
//   * d_pairs  layer pairs for the staged plane kernel: pairs[iz][iy][ix] =
//              (v[ix][iy][iz], v[ix][iy][iz+1]) for iz in [0, n-2], rows
//              padded to `pitch` elements so every row starts 16-byte aligned;
//   * d_oct    cell octets for ray transforms in rotated layer frames: cell
//              (ix, iy, iz), ix, iy, iz in [0, n-2], holds its eight corners
//              as two float4, (v(x,y,z), v(x,y,z+1), v(x,y+1,z), v(x,y+1,z+1))
//              at x = ix and at x = ix + 1, one 32-byte sector per sample.
#include "wrt_internal.cuh"

namespace {

template <typename T>
__global__ void volume_convert_kernel(const T *__restrict__ src, int n, float *__restrict__ dst,
                                      unsigned int *__restrict__ stats) {
  const size_t total = (size_t)n * n * n;
  float local = 0.0f, amax = 0.0f;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total;
       k += (size_t)gridDim.x * blockDim.x) {
    float v = (float)src[k];
    dst[k] = v;
    amax = fmaxf(amax, fabsf(v));
    if (v != 0.0f) {
      const int iz = (int)(k % n), iy = (int)((k / n) % n), ix = (int)(k / ((size_t)n * n));
      local = fmaxf(local, wrtd::node_r2(ix, iy, iz, n));
    }
  }
  // warp max, one atomic per warp
  for (int o = 16; o > 0; o >>= 1) {
    local = fmaxf(local, __shfl_xor_sync(0xffffffffu, local, o));
    amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  }
  if ((threadIdx.x & 31) == 0) {
    if (local > 0.0f) atomicMax(stats, __float_as_uint(local));
    if (amax > 0.0f) atomicMax(stats + 1, __float_as_uint(amax));
  }
}

// oct[2c], oct[2c+1]: corners of cell c = (iz*(n-1) + iy)*(n-1) + ix (x
// fastest: the cells a layer's rays cross side by side are neighbours).
// Threads run over z fastest, so the volume reads coalesce; each thread
// writes its cell's whole 32-byte sector.
__global__ void volume_octets_kernel(const float *__restrict__ v, int n, float4 *__restrict__ oct) {
  const size_t m = (size_t)(n - 1), total = m * m * m;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total;
       k += (size_t)gridDim.x * blockDim.x) {
    const int iz = (int)(k % m), iy = (int)((k / m) % m), ix = (int)(k / (m * m));
    const size_t c = ((size_t)iz * m + iy) * m + ix;
    const float *q = v + ((size_t)ix * n + iy) * n + iz;
    const size_t sx = (size_t)n * n;
    oct[2 * c] = make_float4(q[0], q[1], q[n], q[n + 1]);
    oct[2 * c + 1] = make_float4(q[sx], q[sx + 1], q[sx + n], q[sx + n + 1]);
  }
}

// pairs[iz][iy][ix] = (v[ix][iy][iz], v[ix][iy][iz+1]); one thread per output.
__global__ void volume_pairs_kernel(const float *__restrict__ v, int n, float2 *__restrict__ pairs,
                                    int pitch) {
  const size_t total = (size_t)(n - 1) * n * pitch;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total;
       k += (size_t)gridDim.x * blockDim.x) {
    int ix = (int)(k % pitch), iy = (int)((k / pitch) % n), iz = (int)(k / ((size_t)pitch * n));
    float2 p = make_float2(0.0f, 0.0f);
    if (ix < n) {
      const float *q = v + ((size_t)ix * n + iy) * n + iz;
      p = make_float2(q[0], q[1]);
    }
    pairs[k] = p;
  }
}

// BF16 storage: each value rounded to bfloat16; statistics of the rounded values.
__global__ void volume_bf16_kernel(const float *__restrict__ src, int n,
                                   __nv_bfloat16 *__restrict__ dst, unsigned int *__restrict__ stats) {
  const size_t total = (size_t)n * n * n;
  float local = 0.0f, amax = 0.0f;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total;
       k += (size_t)gridDim.x * blockDim.x) {
    const __nv_bfloat16 b = __float2bfloat16_rn(src[k]);
    dst[k] = b;
    const float v = __bfloat162float(b);
    amax = fmaxf(amax, fabsf(v));
    if (v != 0.0f) {
      const int iz = (int)(k % n), iy = (int)((k / n) % n), ix = (int)(k / ((size_t)n * n));
      local = fmaxf(local, wrtd::node_r2(ix, iy, iz, n));
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    local = fmaxf(local, __shfl_xor_sync(0xffffffffu, local, o));
    amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  }
  if ((threadIdx.x & 31) == 0) {
    if (local > 0.0f) atomicMax(stats, __float_as_uint(local));
    if (amax > 0.0f) atomicMax(stats + 1, __float_as_uint(amax));
  }
}

__global__ void volume_pairs_bf16_kernel(const __nv_bfloat16 *__restrict__ v, int n,
                                         __nv_bfloat162 *__restrict__ pairs, int pitch) {
  const size_t total = (size_t)(n - 1) * n * pitch;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total;
       k += (size_t)gridDim.x * blockDim.x) {
    int ix = (int)(k % pitch), iy = (int)((k / pitch) % n), iz = (int)(k / ((size_t)pitch * n));
    __nv_bfloat162 p = __floats2bfloat162_rn(0.0f, 0.0f);
    if (ix < n) {
      const __nv_bfloat16 *q = v + ((size_t)ix * n + iy) * n + iz;
      p.x = q[0];
      p.y = q[1];
    }
    pairs[k] = p;
  }
}

template <typename T>
int convert(wrt_ctx *ctx, const T *d_src, int n, float *d_vol, unsigned int *d_stats) {
  cudaError_t e = cudaMemsetAsync(d_stats, 0, 2 * sizeof(unsigned int), ctx->stream);
  if (e != cudaSuccess) return wrt::cuda_fail(ctx, e, "volume stats reset");
  int blocks = ctx->sm_count * 8;
  volume_convert_kernel<T><<<blocks, 256, 0, ctx->stream>>>(d_src, n, d_vol, d_stats);
  ctx->launches++;
  return wrt::check_launch(ctx, "volume_convert_kernel");
}

}  // namespace

namespace wrt {

int volume_from_f32(wrt_ctx *ctx, const float *d_src, int n, float *d_vol,
                    unsigned int *d_r2bits) {
  return convert(ctx, d_src, n, d_vol, d_r2bits);
}

int volume_to_bf16(wrt_ctx *ctx, const float *d_vol, int n, __nv_bfloat16 *d_vol16,
                   unsigned int *d_stats) {
  cudaError_t e = cudaMemsetAsync(d_stats, 0, 2 * sizeof(unsigned int), ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "volume stats reset");
  volume_bf16_kernel<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(d_vol, n, d_vol16, d_stats);
  ctx->launches++;
  return check_launch(ctx, "volume_bf16_kernel");
}

int volume_pairs_bf16(wrt_ctx *ctx, const __nv_bfloat16 *d_vol16, int n,
                      __nv_bfloat162 *d_pairs, int pitch) {
  volume_pairs_bf16_kernel<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(d_vol16, n, d_pairs, pitch);
  ctx->launches++;
  return check_launch(ctx, "volume_pairs_bf16_kernel");
}

int volume_octets(wrt_ctx *ctx, const float *d_vol, int n, float4 *d_oct) {
  volume_octets_kernel<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(d_vol, n, d_oct);
  ctx->launches++;
  return check_launch(ctx, "volume_octets_kernel");
}

int volume_pairs(wrt_ctx *ctx, const float *d_vol, int n, float2 *d_pairs, int pitch) {
  int blocks = ctx->sm_count * 8;
  volume_pairs_kernel<<<blocks, 256, 0, ctx->stream>>>(d_vol, n, d_pairs, pitch);
  ctx->launches++;
  return check_launch(ctx, "volume_pairs_kernel");
}

}  // namespace wrt
