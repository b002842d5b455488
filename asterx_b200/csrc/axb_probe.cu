// FP64 throughput probe: the peak rates that bound the engine's
// instruction-bound kernels (the HBM peak alone does not), measured on the
// device the library runs on.  Not part of the reference; a measurement aid.
//
//   fma:  independent chains of x = x * a + b, 2 FLOP per fused multiply-add
//   div:  independent chains of x = a / x + b (IEEE double division, the
//         compiler's correctly rounded sequence), divisions per second
//   sqrt: independent chains of x = sqrt(x) + b, square roots per second
//   rsqrt: independent chains of x = rsqrt(x) + b
//
// Every chain's final value is stored, so no work is optimised away.  The
// grid is a multiple of the SM count with enough warps per SM to hide the
// pipeline latency.
#include <cuda_runtime.h>

#include "axb_internal.hxx"

namespace {

constexpr int kChains = 8;

template <int OP>
__global__ void __launch_bounds__(256) k_probe(double *out, double a, double b, int iters) {
  double x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c)
    x[c] = 1.0 + 1e-3 * (threadIdx.x + c);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) {
      if (OP == 0)
        x[c] = fma(x[c], a, b);
      else if (OP == 1)
        x[c] = a / x[c] + b;
      else if (OP == 2)
        x[c] = sqrt(x[c]) + b;
      else
        x[c] = rsqrt(x[c]) + b;
    }
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; ++c)
    s += x[c];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <int OP>
int time_probe(int sms, double *buf, int iters, double &ops_per_s) {
  const int blocks = sms * 8, threads = 256;
  cudaEvent_t e0, e1;
  AXB_CUDA_TRY(cudaEventCreate(&e0));
  AXB_CUDA_TRY(cudaEventCreate(&e1));
  // warm-up, then the timed launch
  k_probe<OP><<<blocks, threads>>>(buf, 0.999999, 1e-7, iters / 8);
  AXB_CUDA_TRY(cudaEventRecord(e0));
  k_probe<OP><<<blocks, threads>>>(buf, 0.999999, 1e-7, iters);
  AXB_CUDA_TRY(cudaEventRecord(e1));
  AXB_CUDA_TRY(cudaEventSynchronize(e1));
  float ms = 0;
  AXB_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ops_per_s = double(blocks) * threads * kChains * double(iters) / (ms * 1e-3);
  return AXB_OK;
}

} // namespace

// Measure the FP64 rates of the current device: out[0] = FMA TFLOP/s
// (2 FLOP per FMA), out[1] = divisions G/s, out[2] = square roots G/s,
// out[3] = reciprocal square roots G/s.  Synchronous; allocates a small
// result buffer for the duration of the call.
AXB_API int axb_probe_fp64(double out[4]) {
  if (!out)
    return AXB_ERR_ARG;
  int dev = 0, sms = 0;
  AXB_CUDA_TRY(cudaGetDevice(&dev));
  AXB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  double *buf = nullptr;
  AXB_CUDA_TRY(cudaMalloc(&buf, size_t(sms) * 8 * 256 * sizeof(double)));
  double r[4] = {0, 0, 0, 0};
  int rc = time_probe<0>(sms, buf, 1 << 16, r[0]);
  if (!rc)
    rc = time_probe<1>(sms, buf, 1 << 12, r[1]);
  if (!rc)
    rc = time_probe<2>(sms, buf, 1 << 12, r[2]);
  if (!rc)
    rc = time_probe<3>(sms, buf, 1 << 14, r[3]);
  cudaFree(buf);
  if (rc)
    return rc;
  out[0] = 2.0 * r[0] / 1e12;
  out[1] = r[1] / 1e9;
  out[2] = r[2] / 1e9;
  out[3] = r[3] / 1e9;
  return AXB_OK;
}
