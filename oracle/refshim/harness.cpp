/*
 * Oracle — TEST INFRASTRUCTURE ONLY.
 * Launch emulation for the reference's kernel source compiled for the CPU
 * (oracle/build.py links this file with the template-substituted
 * sim3d_kernel.cu).  A launch runs every (block, thread) of the grid, each as
 * an independent call; the walk and seeding kernels touch only their own
 * walker's slots, so threads may run in any order or in parallel.
 *
 * Draws: curand_normal returns normals[walker][step][k], k counting the
 * walker's draws within the launch's step, or, with ref_set_philox, component
 * k % 3 of the oracle's Philox draw k / 3 at (walker, step); curand_uniform returns
 * uniforms[walker][k] when a table is set, otherwise a splitmix64 hash of
 * (seed, walker, k).  An exhausted table returns 0 and raises a flag.
 */
#include "curand_kernel.h"
#include <stddef.h>
#include "../oz_rng.h"

thread_local oz_dim3 threadIdx, blockIdx, blockDim, gridDim;

static const float* g_normals = nullptr;
static int g_nsteps = 0, g_maxk = 0;
static int g_step = 0;
static const float* g_uniforms = nullptr;
static int g_nu = 0;
static volatile int g_exhausted = 0;
static int g_philox = 0;
static uint32_t g_k0 = 0, g_k1 = 0, g_stream = 0;

void curand_init(unsigned long long seed, unsigned long long subsequence, unsigned long long,
                 curandState* s) {
    s->seed = (long long)seed;
    s->walker = (int)subsequence;
    s->step = -1;
    s->k = 0;
    s->ku = 0;
}

float curand_normal(curandState* s) {
    if (s->step != g_step) { s->step = g_step; s->k = 0; }
    int k = s->k++;
    if (g_philox) {
        float n[3];
        oz_philox_normal3(g_k0, g_k1, g_stream, (uint32_t)s->walker, (uint32_t)g_step, (uint32_t)(k / 3),
                          &n[0], &n[1], &n[2]);
        return n[k % 3];
    }
    if (!g_normals || g_step < 0 || g_step >= g_nsteps || k >= g_maxk) { g_exhausted = 1; return 0.0f; }
    return g_normals[((size_t)s->walker * g_nsteps + g_step) * g_maxk + k];
}

static inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

float curand_uniform(curandState* s) {
    int k = s->ku++;
    if (g_uniforms) {
        if (k >= g_nu) { g_exhausted = 1; return 1.0f; }
        return g_uniforms[(size_t)s->walker * g_nu + k];
    }
    uint64_t h = splitmix64(splitmix64((uint64_t)s->seed) ^ ((uint64_t)(uint32_t)s->walker << 20) ^ (uint64_t)k);
    return (float)((h >> 40) + 1) * (1.0f / 16777216.0f); /* (0, 1] */
}

extern "C" {
void initstates(int seed);
void seedSpinsKernel(int nspin, int nstructures, float* spheres, int* sphere_counts, float* positions,
                     int n_struct_idx, int* struct_idxs, float Lx, float Ly, float Lz, unsigned int seed,
                     int* seeding_status);
void randomWalk3d(float dt, float* spheres, int* segmentList, float* spins, float* spins0, float* sig);
void randomWalk3d_phase(float dt, float* spheres, int* segmentList, float* spins, float* spins0,
                        float* phase_accumulated, float G, float G_area_at_this_time_step);
void randomWalk3d_phase_multidirr(float dt, float* spheres, int* segmentList, float* spins, float* spins0,
                                  float* phase_accumulated, float G, float G_area_at_this_time_step,
                                  float* diffdir, int ndiffdir);

void ref_set_normals(const float* table, int nsteps, int maxk) { g_normals = table; g_nsteps = nsteps; g_maxk = maxk; g_philox = 0; }
void ref_set_philox(unsigned k0, unsigned k1, unsigned stream) { g_philox = 1; g_k0 = k0; g_k1 = k1; g_stream = stream; }
void ref_set_uniforms(const float* table, int nu) { g_uniforms = table; g_nu = nu; }
int ref_exhausted(void) { return g_exhausted; }
void ref_clear_exhausted(void) { g_exhausted = 0; }

#define OZ_GRID_LOOP(CALL)                                                      \
    do {                                                                        \
        const long long total = (long long)grid * block;                        \
        _Pragma("omp parallel for schedule(static)")                            \
        for (long long t = 0; t < total; ++t) {                                 \
            blockDim.x = (unsigned)block; blockDim.y = blockDim.z = 1;          \
            gridDim.x = (unsigned)grid; gridDim.y = gridDim.z = 1;              \
            blockIdx.x = (unsigned)(t / block); blockIdx.y = blockIdx.z = 0;    \
            threadIdx.x = (unsigned)(t % block); threadIdx.y = threadIdx.z = 0; \
            CALL;                                                               \
        }                                                                       \
    } while (0)

void ref_run_initstates(int grid, int block, int seed) { OZ_GRID_LOOP(initstates(seed)); }

void ref_run_seed(int grid, int block, int nspin, int nstructures, float* spheres, int* counts, float* pos,
                  int nidx, int* idxs, float Lx, float Ly, float Lz, unsigned int seed, int* status) {
    OZ_GRID_LOOP(seedSpinsKernel(nspin, nstructures, spheres, counts, pos, nidx, idxs, Lx, Ly, Lz, seed, status));
}

void ref_run_walk(int grid, int block, int step, float dt, float* spheres, int* seg, float* spins,
                  float* spins0, float* sig) {
    g_step = step;
    OZ_GRID_LOOP(randomWalk3d(dt, spheres, seg, spins, spins0, sig));
}

void ref_run_walk_phase(int grid, int block, int step, float dt, float* spheres, int* seg, float* spins,
                        float* spins0, float* phase, float G, float Garea) {
    g_step = step;
    OZ_GRID_LOOP(randomWalk3d_phase(dt, spheres, seg, spins, spins0, phase, G, Garea));
}

void ref_run_walk_multidir(int grid, int block, int step, float dt, float* spheres, int* seg, float* spins,
                           float* spins0, float* phase, float G, float Garea, float* diffdir, int ndir) {
    g_step = step;
    OZ_GRID_LOOP(randomWalk3d_phase_multidirr(dt, spheres, seg, spins, spins0, phase, G, Garea, diffdir, ndir));
}
}
