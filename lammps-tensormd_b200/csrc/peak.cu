// peak.cu -- tmd_fp32_peak: the FP32 issue peak of this GPU, measured.
//
// The plain-form descriptor and force kernels are bound by FP32 FMA issue, so
// their roofline denominator is the rate at which the SMs retire packed FMAs.
// This kernel runs eight independent FFMA2 chains per thread (no memory
// traffic, no dependence stalls at 8+ warps per scheduler) on 2,048 threads
// per SM and is timed with CUDA events; FLOPs are counted as 2 per FMA.
#include <cuda_runtime.h>

#include <string>

#include "../../include/tmd_b200.h"

namespace tmd {
void set_last_error(const std::string &msg);
}

namespace {

constexpr int kChains = 8;
constexpr int kUnroll = 4;

__global__ void __launch_bounds__(256) k_ffma2_peak(int iters, float seed, float *sink) {
  float2 a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; k++)
    a[k] = make_float2(seed + 1e-7f * threadIdx.x + k, seed - k);
  const float2 m = make_float2(0.9999999f, 1.0000001f);
  const float2 c = make_float2(1e-7f, -1e-7f);
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int u = 0; u < kUnroll; u++)
#pragma unroll
      for (int k = 0; k < kChains; k++) a[k] = __ffma2_rn(a[k], m, c);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kChains; k++) s += a[k].x + a[k].y;
  if (s == 1234.5678f) sink[threadIdx.x] = s;  // keeps the chains live
}

int fail(int code, const std::string &m) {
  tmd::set_last_error(m);
  return code;
}

}  // namespace

extern "C" int tmd_fp32_peak(int device, int reps, double *tflops) {
  if (!tflops || reps < 1) return fail(TMD_ERR_ARG, "tmd_fp32_peak: bad argument");
  int prev = 0;
  cudaGetDevice(&prev);
  cudaError_t e = cudaSetDevice(device);
  int nsm = 0;
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float *sink = nullptr;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  if (e == cudaSuccess) e = cudaMalloc(&sink, 256 * sizeof(float));
  const int threads = 256, blocks = nsm * 8;  // 2,048 threads per SM
  const int iters = 16384;
  double best = 0.0;
  if (e == cudaSuccess) {
    k_ffma2_peak<<<blocks, threads, 0, st>>>(iters, 1.0f, sink);  // warm-up
    e = cudaGetLastError();
  }
  for (int r = 0; r < reps && e == cudaSuccess; r++) {
    cudaEventRecord(e0, st);
    k_ffma2_peak<<<blocks, threads, 0, st>>>(iters, 1.0f + r, sink);
    cudaEventRecord(e1, st);
    e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess && ms > 0.f) {
      const double flops = 4.0 * kChains * kUnroll * (double)iters * threads * blocks;
      const double tf = flops / (ms * 1e-3) / 1e12;
      if (tf > best) best = tf;
    }
  }
  if (sink) cudaFree(sink);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  cudaSetDevice(prev);
  if (e != cudaSuccess)
    return fail(TMD_ERR_CUDA, std::string("tmd_fp32_peak: ") + cudaGetErrorString(e));
  *tflops = best;
  return TMD_OK;
}
