// Pipe-throughput probes used as roofline denominators: FP32 FFMA, FP64 DFMA and SFU (MUFU.SIN)
// instruction rates of the whole GPU, measured with CUDA events around one launch of independent
// dependency chains (8 per thread, enough warps per SM to hide the latency).
#include <cuda_runtime.h>

#include "srs_internal.h"

namespace srs {
namespace {

constexpr int kChains = 8;

__global__ void ffma_probe(float *out, int iters, float a, float b) {
  float x[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) x[k] = threadIdx.x * 1e-3f + k;
  for (int i = 0; i < iters; ++i)
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = fmaf(x[k], a, b);
  float s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += x[k];
  if (s == 1.2345f) out[0] = s;  // keeps the chains alive; never true for the probe's inputs
}

__global__ void dfma_probe(double *out, int iters, double a, double b) {
  double x[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) x[k] = threadIdx.x * 1e-3 + k;
  for (int i = 0; i < iters; ++i)
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = fma(x[k], a, b);
  double s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += x[k];
  if (s == 1.2345) out[0] = s;
}

__global__ void mufu_probe(float *out, int iters) {
  float x[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) x[k] = threadIdx.x * 1e-3f + 0.1f * k;
  for (int i = 0; i < iters; ++i)
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = __sinf(x[k]);
  float s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += x[k];
  if (s == 1.2345f) out[0] = s;
}

}  // namespace
}  // namespace srs

using namespace srs;

extern "C" srs_status srs_measure_peak(int32_t kind, double *ops_per_s, void *stream) {
  clear_error();
  if (!ops_per_s || kind < 0 || kind > 2) return fail(SRS_ERR_INVALID, "kind must be 0 (fp32), 1 (fp64), 2 (sfu)");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int dev = 0, sms = 0;
  SRS_CUDA(cudaGetDevice(&dev));
  SRS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int threads = 256, blocks = sms * 8;
  const int iters = kind == 0 ? 4096 : kind == 1 ? 2048 : 1024;
  DeviceBuffer sink;
  SRS_CUDA(sink.alloc(64, s));
  cudaEvent_t e0, e1;
  SRS_CUDA(cudaEventCreate(&e0));
  SRS_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  for (int rep = 0; rep < 3; ++rep) {
    SRS_CUDA(cudaEventRecord(e0, s));
    if (kind == 0) ffma_probe<<<blocks, threads, 0, s>>>(sink.as<float>(), iters, 0.999f, 1e-3f);
    if (kind == 1) dfma_probe<<<blocks, threads, 0, s>>>(sink.as<double>(), iters, 0.999, 1e-3);
    if (kind == 2) mufu_probe<<<blocks, threads, 0, s>>>(sink.as<float>(), iters);
    SRS_CUDA(cudaGetLastError());
    SRS_CUDA(cudaEventRecord(e1, s));
    SRS_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    SRS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (rep > 0 && ms < best) best = ms;  // first launch warms up
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ops_per_s = (double)blocks * threads * iters * kChains / (best * 1e-3);
  return SRS_OK;
}
