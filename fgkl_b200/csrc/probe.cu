// FP32 FMA throughput probe: the denominator of the PairHMM kernels' FP32 roofline, measured on the
// device the library runs on (independent FMA chains, scalar FFMA and packed FFMA2 variants).
#include <cuda_runtime.h>

#include "../../include/fgkl_b200.h"

namespace {

constexpr int kChains = 8;

__global__ void fma_scalar(float* out, int iters, float m, float c) {
  float acc[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) acc[k] = threadIdx.x * 1e-3f + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) acc[k] = __fmaf_rn(acc[k], m, c);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += acc[k];
  if (s == 12345.678f) out[blockIdx.x] = s;  // keeps the chains live
}

__global__ void fma_packed(float* out, int iters, float m, float c) {
  float2 acc[kChains];
  const float2 mm = make_float2(m, m), cc = make_float2(c, c);
#pragma unroll
  for (int k = 0; k < kChains; ++k) acc[k] = make_float2(threadIdx.x * 1e-3f + k, k);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) acc[k] = __ffma2_rn(acc[k], mm, cc);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += acc[k].x + acc[k].y;
  if (s == 12345.678f) out[blockIdx.x] = s;
}

// Integer ALU throughput: independent chains of a bitwise XOR and a signed max, the two kinds of
// operation (LOP3, integer min/max) the ALU pipe issues alone.
__global__ void alu_chains(int* out, int iters, int x, int y) {
  int acc[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) acc[k] = static_cast<int>(threadIdx.x) * 7 + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) acc[k] = max(acc[k] ^ x, y);
  }
  int s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s ^= acc[k];
  if (s == 0x5a5a5a5a) out[blockIdx.x] = s;  // keeps the chains live
}

}  // namespace

extern "C" int fgkl_probe_int32_alu_gops(int32_t device, double* gops) {
  if (!gops) return FGKL_E_INVALID_ARGUMENT;
  if (cudaSetDevice(device) != cudaSuccess) return FGKL_E_NO_DEVICE;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int threads = 256, blocks = sms * 8, iters = 1 << 15;
  int* out = nullptr;
  if (cudaMalloc(&out, sizeof(int) * blocks) != cudaSuccess) return FGKL_E_CUDA;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double best = 0;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(a);
    alu_chains<<<blocks, threads>>>(out, iters, 0x1234567, -5);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    const double ops = 2.0 * kChains * iters * static_cast<double>(threads) * blocks;
    if (rep > 0 && ms > 0 && ops / (ms * 1e-3) / 1e9 > best) best = ops / (ms * 1e-3) / 1e9;
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  if (err != cudaSuccess) return FGKL_E_CUDA;
  *gops = best;
  return FGKL_OK;
}

extern "C" int fgkl_probe_fp32_tflops(int32_t device, double* scalar_tflops, double* packed_tflops, double* sm_clock_mhz) {
  if (cudaSetDevice(device) != cudaSuccess) return FGKL_E_NO_DEVICE;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int threads = 256, blocks = sms * 8, iters = 1 << 16;
  float* out = nullptr;
  if (cudaMalloc(&out, sizeof(float) * blocks) != cudaSuccess) return FGKL_E_CUDA;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double best[2] = {0, 0};
  for (int variant = 0; variant < 2; ++variant) {
    for (int rep = 0; rep < 4; ++rep) {
      cudaEventRecord(a);
      if (variant == 0)
        fma_scalar<<<blocks, threads>>>(out, iters, 0.999999f, 1e-7f);
      else
        fma_packed<<<blocks, threads>>>(out, iters, 0.999999f, 1e-7f);
      cudaEventRecord(b);
      cudaEventSynchronize(b);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      const double flops = 2.0 * kChains * iters * static_cast<double>(threads) * blocks * (variant ? 2 : 1);
      if (rep > 0 && ms > 0) best[variant] = best[variant] > flops / (ms * 1e-3) / 1e12 ? best[variant] : flops / (ms * 1e-3) / 1e12;
    }
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  if (err != cudaSuccess) return FGKL_E_CUDA;
  if (scalar_tflops) *scalar_tflops = best[0];
  if (packed_tflops) *packed_tflops = best[1];
  if (sm_clock_mhz) {
    int khz = 0;
    cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, device);
    *sm_clock_mhz = khz / 1000.0;
  }
  return FGKL_OK;
}
