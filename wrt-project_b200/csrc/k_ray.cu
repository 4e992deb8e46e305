// k_ray.cu -- layer-by-layer ray integrals (ray_grid/src/integral.c:11-50);
// the per-ray body is in ray_dev.cuh.
#include "ray_dev.cuh"

namespace {

// A warp takes a tile of kShiftLanes consecutive shifts x 32 / kShiftLanes
// consecutive angles of one layer.  Parallel rays (shifts) read neighbouring
// cells at each sample, but their chords through the crop ball differ in
// length, so lanes idle at the ends; the rays of one shift at neighbouring
// angles have the same chord.  Measured at 128^3 (128 layers x 128 shifts x
// 128 angles): the reference frame, whose rays read the layer's octets
// row by row, 1.09 ms with 16 shifts x 2 angles (1.11 with 32 x 1, 1.25 with
// 8 x 4); a rotated frame 0.60 ms with 2 x 16 (0.82 with 32 x 1, 0.63 with
// 4 x 8).  Each ray is the same computation whichever lane takes it.
template <bool FRAME>
constexpr int kShiftLanes = FRAME ? 2 : 16;

template <bool FRAME>
__global__ void __launch_bounds__(256) ray_kernel(wrt::RayJob job, float guard) {
  constexpr int kS = kShiftLanes<FRAME>, kA = 32 / kS;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = (int)(t & 31);
  const long long tile = t >> 5;
  const long long ts_n = (job.nshift + kS - 1) / kS, tp_n = (job.nphi + kA - 1) / kA;
  const long long iz = tile / (ts_n * tp_n), rem = tile % (ts_n * tp_n);
  const long long is = (rem % ts_n) * kS + lane % kS, ip = (rem / ts_n) * kA + lane / kS;
  if (iz >= job.nslices || is >= job.nshift || ip >= job.nphi) return;
  wrtd::ray_one<FRAME>(job, (iz * job.nphi + ip) * job.nshift + is, guard);
}

}  // namespace

namespace wrt {

int ray_forward(wrt_ctx *ctx, const RayJob &job) {
  const long long nrays = (long long)job.nslices * job.nshift * job.nphi;
  if (nrays == 0) return WRT_OK;
  // one warp per tile
  const int kS = job.has_frame ? kShiftLanes<true> : kShiftLanes<false>, kA = 32 / kS;
  const long long tiles =
      (long long)job.nslices * ((job.nshift + kS - 1) / kS) * ((job.nphi + kA - 1) / kA);
  const long long blocks = (tiles + 7) / 8;
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
