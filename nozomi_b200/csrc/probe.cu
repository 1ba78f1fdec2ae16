// Device peak probe used by the benchmark to state the FP32 roofline it
// reports against: each thread runs 8 independent fused multiply-add chains.
#include "kernels.cuh"

namespace nz {

__global__ void __launch_bounds__(256) fma_probe_kernel(int iters, float seed, float* __restrict__ out) {
  float a[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = seed + float(threadIdx.x + i);
  const float m = 0.999999f, c = 1e-7f;
  for (int k = 0; k < iters; ++k) {
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = __fmaf_rn(a[i], m, c);
  }
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += a[i];
  if (s == 12345.678f) out[blockIdx.x] = s;  // keeps the chains live
}

}  // namespace nz

using namespace nz;

// FP32 FMA throughput probe: grid x 256 threads x iters x 8 FMAs (2 flops each).
extern "C" int nz_probe_fma(int grid, int iters, float* out, void* stream) {
  if (grid <= 0 || iters <= 0 || !out) return set_error(NZ_ERR_ARG, "nz_probe_fma: bad arguments");
  fma_probe_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(iters, 1.0f, out);
  return check_launch("fma_probe_kernel");
}
