// Launch shim for the reference's own CUDA kernel source on the GPU.
//
// The reference drives its kernels through pycuda (DiffSim3d, diffsim3d.py:
// 236-261: block 1000, grid nspins/1000, default stream, one launch per
// waveform sample).  pycuda is not installed, so this file stands in for the
// launches only: it includes the reference's sim3d_kernel.cu after the
// reference's own %-template substitution (written by reference_gpu.py into
// baseline/_ref, never committed) and exposes C entry points that launch the
// unmodified kernels with the reference's launch shape.  It is a baseline
// harness, not part of the nozomi_b200 product.
#include NZ_REF_KERNEL_SOURCE

#include <cstdio>

static char g_err[256];

static int check(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return 0;
  std::snprintf(g_err, sizeof(g_err), "%s: %s", what, cudaGetErrorString(e));
  return 1;
}

extern "C" const char* refgpu_last_error(void) { return g_err; }
extern "C" int refgpu_nspins(void) { return nspins; }
extern "C" int refgpu_nspheres_per_seg(void) { return nspheres_per_seg; }

extern "C" int refgpu_initstates(int seed, int grid, int block, void* stream) {
  initstates<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(seed);
  return check("initstates");
}

extern "C" int refgpu_walk_multidir(float dt, float* spheres, int* segments, float* spins, float* spins0,
                                    float* phase, float G, float Garea, float* diffdir, int ndir, int grid,
                                    int block, void* stream) {
  randomWalk3d_phase_multidirr<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
      dt, spheres, segments, spins, spins0, phase, G, Garea, diffdir, ndir);
  return check("randomWalk3d_phase_multidirr");
}

extern "C" int refgpu_walk(float dt, float* spheres, int* segments, float* spins, float* spins0, float* sig,
                           int grid, int block, void* stream) {
  randomWalk3d<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(dt, spheres, segments, spins, spins0, sig);
  return check("randomWalk3d");
}
