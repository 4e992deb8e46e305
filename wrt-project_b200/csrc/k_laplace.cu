// k_laplace.cu -- spectral Laplacian of a volume, the step after the
// backprojection in the reference's inversion (radon_inversion/backprojection/
// laplace3dfft.m:1-25):
//   output = ifftn(U .* fftn(u)),  U = -(2 pi / period)^2 (k1^2 + k2^2 + k3^2),
// k the FFT-order frequency of each axis (index i for i <= n/2, i - n above,
// laplace3dfft.m:9-15).  U is real and even in every axis, so the result is
// real: here a real-to-complex FP64 FFT (cuFFT), one kernel that multiplies
// the half spectrum by U / n^3, and the complex-to-real inverse.  Plans are
// made once per edge length and kept in the context.
#include <cufft.h>

#include "wrt_internal.cuh"

namespace {

__device__ __forceinline__ double fft_freq(int i, int n) { return (double)(i <= n / 2 ? i : i - n); }

// Half spectrum [n][n][n/2 + 1]; the last axis holds k3 = 0 .. n/2.
__global__ void laplace_spectrum_kernel(cufftDoubleComplex *__restrict__ Y, int n, double scale) {
  const long long nh = n / 2 + 1, total = (long long)n * n * nh;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int k3 = (int)(idx % nh), k2 = (int)((idx / nh) % n), k1 = (int)(idx / (nh * n));
    const double a = fft_freq(k1, n), b = fft_freq(k2, n), c = (double)k3;
    const double u = scale * (a * a + b * b + c * c);
    cufftDoubleComplex y = Y[idx];
    y.x *= u;
    y.y *= u;
    Y[idx] = y;
  }
}

struct LaplacePlans {
  int n = 0;
  cufftHandle fwd = 0, inv = 0;
};

const char *cufft_name(cufftResult r) {
  switch (r) {
    case CUFFT_SUCCESS: return "success";
    case CUFFT_ALLOC_FAILED: return "allocation failed";
    case CUFFT_INVALID_VALUE: return "invalid value";
    case CUFFT_EXEC_FAILED: return "execution failed";
    case CUFFT_SETUP_FAILED: return "setup failed";
    case CUFFT_INVALID_SIZE: return "invalid size";
    default: return "error";
  }
}

}  // namespace

namespace wrt {

void laplace_release(wrt_ctx *ctx) {
  LaplacePlans *p = static_cast<LaplacePlans *>(ctx->fft_plans);
  if (!p) return;
  if (p->n) {
    cufftDestroy(p->fwd);
    cufftDestroy(p->inv);
  }
  delete p;
  ctx->fft_plans = nullptr;
}

int spectral_laplacian(wrt_ctx *ctx, const double *d_in, int n, double period, double *d_out) {
  LaplacePlans *p = static_cast<LaplacePlans *>(ctx->fft_plans);
  if (!p) ctx->fft_plans = p = new LaplacePlans();
  if (p->n != n) {
    if (p->n) {
      cufftDestroy(p->fwd);
      cufftDestroy(p->inv);
      p->n = 0;
    }
    cufftResult r = cufftPlan3d(&p->fwd, n, n, n, CUFFT_D2Z);
    if (r == CUFFT_SUCCESS) {
      r = cufftPlan3d(&p->inv, n, n, n, CUFFT_Z2D);
      if (r != CUFFT_SUCCESS) cufftDestroy(p->fwd);
    }
    if (r != CUFFT_SUCCESS)
      return fail(ctx, r == CUFFT_ALLOC_FAILED ? WRT_ERR_OUT_OF_MEMORY : WRT_ERR_CUDA,
                  "spectral laplacian: cufftPlan3d(%d): %s", n, cufft_name(r));
    p->n = n;
  }
  void *spec = nullptr;
  const size_t bytes = sizeof(cufftDoubleComplex) * (size_t)n * n * (n / 2 + 1);
  int st = ws_get(ctx, WS_FFT, bytes, &spec);
  if (st) return st;
  cufftSetStream(p->fwd, ctx->stream);
  cufftSetStream(p->inv, ctx->stream);
  cufftDoubleComplex *Y = static_cast<cufftDoubleComplex *>(spec);
  // an out-of-place real-to-complex transform leaves its input as it was
  cufftResult r = cufftExecD2Z(p->fwd, const_cast<double *>(d_in), Y);
  if (r != CUFFT_SUCCESS)
    return fail(ctx, WRT_ERR_CUDA, "spectral laplacian: forward FFT: %s", cufft_name(r));
  const double two_pi_p = 2.0 * WRT_PI / period;
  const double scale = -(two_pi_p * two_pi_p) / ((double)n * n * n);  // inverse FFT is unnormalised
  laplace_spectrum_kernel<<<ctx->sm_count * 4, 256, 0, ctx->stream>>>(Y, n, scale);
  ctx->launches++;
  st = check_launch(ctx, "laplace_spectrum_kernel");
  if (st) return st;
  r = cufftExecZ2D(p->inv, Y, d_out);
  if (r != CUFFT_SUCCESS)
    return fail(ctx, WRT_ERR_CUDA, "spectral laplacian: inverse FFT: %s", cufft_name(r));
  return WRT_OK;
}

}  // namespace wrt

extern "C" {

int wrt_spectral_laplacian_device(wrt_ctx *ctx, const double *dev_in, int n, double period,
                                  double *dev_out) {
  if (!ctx || !dev_in || !dev_out || n < 2 || n > 2048 || !(period > 0.0))
    return ctx ? wrt::fail(ctx, WRT_ERR_INVALID_ARGUMENT, "spectral laplacian: bad arguments")
               : WRT_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return wrt::cuda_fail(ctx, e, "cudaSetDevice");
  return wrt::spectral_laplacian(ctx, dev_in, n, period, dev_out);
}

int wrt_spectral_laplacian(wrt_ctx *ctx, const double *in, int n, double period, double *out) {
  if (!ctx || !in || !out || n < 2 || n > 2048 || !(period > 0.0))
    return ctx ? wrt::fail(ctx, WRT_ERR_INVALID_ARGUMENT, "spectral laplacian: bad arguments")
               : WRT_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return wrt::cuda_fail(ctx, e, "cudaSetDevice");
  const size_t bytes = sizeof(double) * (size_t)n * n * n;
  void *din = nullptr, *dout = nullptr;
  int st = wrt::ws_get(ctx, wrt::WS_IN, bytes, &din);
  if (!st) st = wrt::ws_get(ctx, wrt::WS_OUT, bytes, &dout);
  if (st) return st;
  e = cudaMemcpyAsync(din, in, bytes, cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) return wrt::cuda_fail(ctx, e, "spectral laplacian input");
  st = wrt::spectral_laplacian(ctx, static_cast<const double *>(din), n, period,
                               static_cast<double *>(dout));
  if (st) return st;
  e = cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? WRT_OK : wrt::cuda_fail(ctx, e, "spectral laplacian result");
}

}  // extern "C"
