// k_ray.cu -- layer-by-layer ray integrals (ray_grid/src/integral.c:11-50);
// the per-ray body is in ray_dev.cuh.
#include "ray_dev.cuh"

namespace {

template <bool FRAME>
__global__ void __launch_bounds__(256) ray_kernel(wrt::RayJob job, float guard) {
  const long long ray = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (ray >= (long long)job.nslices * job.nshift * job.nphi) return;
  wrtd::ray_one<FRAME>(job, ray, guard);
}

}  // namespace

namespace wrt {

int ray_forward(wrt_ctx *ctx, const RayJob &job) {
  const long long nrays = (long long)job.nslices * job.nshift * job.nphi;
  if (nrays == 0) return WRT_OK;
  const long long blocks = (nrays + 255) / 256;
  if (blocks > 0x7fffffffLL) return fail(ctx, WRT_ERR_INVALID_ARGUMENT, "too many rays");
  const float g = wrtd::ray_guard(job.n);
  if (job.has_frame)
    ray_kernel<true><<<(unsigned)blocks, 256, 0, ctx->stream>>>(job, g);
  else
    ray_kernel<false><<<(unsigned)blocks, 256, 0, ctx->stream>>>(job, g);
  ctx->launches++;
  return check_launch(ctx, "ray_kernel");
}

}  // namespace wrt
