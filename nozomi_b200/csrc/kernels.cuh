// Structures shared between the kernel files and the C entry points.
#pragma once
#include <cstdint>
#include "nozomi_b200.h"
#include "nz_common.cuh"

namespace nz {

// Devices a process can drive with per-device library state (function
// attributes, the static re-binning scratch).
constexpr int kMaxDevices = 64;

int set_error(int status, const char* fmt, ...);
int check_launch(const char* what);
// Host-side argument checks shared by the entry points (capi.cu): a packed
// state's four arrays present and 16-byte aligned (any, or none, when N is 0);
// a grid with at least one cell per axis.
int check_state(const nz_state* st, const char* who);
int check_grid(const nz_grid* g, const char* who);

// ---- plain walk (walk_plain.cu) ----
struct PlainArgs {
  Grid g;
  int nstructures, S, N;
  int ncell, n_items;  // checked by the bounds-checked build (n_items 0: unknown)
  const float* spheres;  // [5, S]: cx, cy, cz, r, structure id
  const int* cell_start;
  const int* cell_count;
  const int* cell_items;
  const float* D;        // [nstructures + 1]
  const float* T2;       // [nstructures + 1]
  float* spins;          // [3, N]
  float* spins0;         // [3, N]
  float* phase;          // [ndir, N]
  const float* diffdir;  // [3, ndir]
  int ndir;
  float* sig;            // [N]
  float* phi;            // [6, N]: Phi sums then Kahan compensations
  float dt, G, Garea;
  int step;
  Draws draws;
  int mode;
  int* label;
  int* n_iter;
  int* n_scatter;
  int* flags;
};
__global__ void walk_plain_kernel(const PlainArgs a);

// ---- fused walk (walk_fused.cu) ----
constexpr int kFusedThreads = 128;     // walkers per CTA of nz_walk_fused
constexpr int kFusedMaxThreads = 256;  // largest CTA of nz_walk_batch
constexpr int kMaxStageRecords = 12288;  // records a CTA of the staged batched walk holds in shared memory (192 KiB)
constexpr size_t kSmemPerSm = 228 * 1024;  // shared memory an SM can give its CTAs (sm_100)
#ifndef NZ_FUSED_MIN_BLOCKS
#define NZ_FUSED_MIN_BLOCKS 3
#endif
constexpr int kFusedMinBlocks = NZ_FUSED_MIN_BLOCKS;  // 256-thread CTAs per SM the register budget is sized for
#ifndef NZ_SCAN_UNROLL
#define NZ_SCAN_UNROLL 4
#endif
// list entries loaded together in the scan's first pass: 4 measured fastest
// on both the batched and the packed workloads (1, 2, 4, 8 tried)
constexpr int kScanUnroll = NZ_SCAN_UNROLL;
static_assert(32 % kScanUnroll == 0, "the scan unroll must divide 32");
constexpr int kMomentSteps = 256;  // steps per launch in NZ_MODE_MOMENTS (shared-memory staging)
// Internal mode bit (nz_walk_fused_moments only): at each step end the fused
// walk stores the walker's float displacement from its origin; a reduction
// kernel then forms the moments.
constexpr int kModeDisp = 32;

struct JobDev {
  Grid g;
  float idLx, idLy, idLz;  // 1 / cell edge (the fused walk's per-step cell)
  int nstructures;
  const float4* sph4;
  const int* sid;
  const int* cell_start;
  const int* cell_count;
  const float* D;
  const float* T2;
  const float* G;
  const float* Garea;
  int nsteps;
  float dt;
  uint32_t key0, key1, stream;
  int mode;
  float4* pos;
  float4* org;
  float4* phi;
  float4* comp;
  double* moments;
  float* disp;  // kModeDisp: per-step displacements [steps of the launch][3][nwalkers]
  int nwalkers;
  int step_offset;
  // near lists (null sph4, or null near_idx in index form: none)
  float near_margin;
  float near_cut;  // (near_margin - tol - 2 nm) / 1.02: the near test's bound on distance + reach
  const int* near_start;
  const int* near_count;
  const float4* near_sph4;
  const int* near_sid;
  // index form of the lists (nz_substrate.idx_bytes > 0)
  const void* idx;
  const void* near_idx;
  const float4* rec4;
  const int* rec_sid;
  const int* sid_start;
  int S;
  // checked by the bounds-checked build (list lengths 0: unknown)
  int ncell, n_items, near_items;
};

__host__ __device__ JobDev make_job(const nz_substrate& sub, const float* G, const float* Garea, int nsteps, float dt,
                                    const nz_draws& d, int mode, const nz_state& st, double* moments);
// lk: list kind, 0 (per-entry records), 2 or 4 (index lists of that width)
int launch_fused(int mode, int lk, const JobDev& single, const nz_job* jobs, const nz_item* items, int n_items,
                 int step0, int step1, int* queue, int grid, int threads, cudaStream_t st, int stage_cap = 0);
int occupancy_fused(int mode, int lk, int threads, int* blocks_per_sm, int stage_cap = 0);
__global__ void pack_kernel(nz_walkers wk, const uint32_t* ids, nz_state st);
__global__ void disp_moments_kernel(const float* __restrict__ disp, int N, double* __restrict__ out);
__global__ void unpack_kernel(nz_state st, nz_walkers wk, int by_id, int* bad);

// ---- ingest.cu ----
// *total = off[F - 1] + len[F - 1] (0 when F is 0): a list's size after its scan.
__global__ void offsets_total_kernel(const int* __restrict__ len, const int* __restrict__ off, int F,
                                     int* __restrict__ total);

// ---- cells.cu ----
__global__ void scan_kernel(const int* __restrict__ in, int* __restrict__ out, int n, int* __restrict__ total);
// Exclusive scan of n ints on stream st: one CTA up to kScanSingle ints,
// beyond that (with tile_sums and tile_offsets of scan_tiles(n) ints each)
// one CTA per kScanTile ints.
constexpr int kScanTile = 8192;
constexpr int kScanSingle = 32768;  // mirrored as SCAN_SINGLE_KEYS in nozomi_b200/_lib.py (launch counts)
int scan_tiles(int n);
int exclusive_scan(const int* in, int* out, int n, int* tile_sums, int* tile_offsets, cudaStream_t st);

}  // namespace nz
