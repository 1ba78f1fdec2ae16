/*
 * Oracle — TEST INFRASTRUCTURE ONLY.
 * Host stand-ins for the CUDA headers that the reference's kernel source
 * (simulation_toolkit/simulation_engine/sim3d_kernel.cu) includes, so that the
 * reference's own, template-substituted source compiles as C++ for the CPU
 * and its kernels run one emulated thread at a time (harness.cpp).
 * curand_normal / curand_uniform read injected tables instead of cuRAND.
 */
#pragma once
#include <math.h>
#include <stdint.h>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __shared__ static

struct oz_dim3 { unsigned x, y, z; };
extern thread_local oz_dim3 threadIdx;
extern thread_local oz_dim3 blockIdx;
extern thread_local oz_dim3 blockDim;
extern thread_local oz_dim3 gridDim;

static inline void __syncthreads() {}
static inline float atomicAdd(float* a, float v) { float o = *a; *a = o + v; return o; }

struct curandState { long long seed; int walker; int step; int k; int ku; };
void curand_init(unsigned long long seed, unsigned long long subsequence, unsigned long long offset,
                 curandState* state);
float curand_normal(curandState* state);
float curand_uniform(curandState* state);
