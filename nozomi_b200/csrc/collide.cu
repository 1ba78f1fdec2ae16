// Collision detection of the substrate generator on a uniform grid: the work
// of collide_spheres_gpu (simulation_toolkit/substrate_generator/helper/
// CollisionDetection.py:10-62), which the reference does with a Python loop
// over grid blocks, a dense [K, K] overlap matrix per block and a
// torch.unique of the growing pair list after every block.
//
// Semantics kept from the reference:
//  * the grid: blocks of edge Lx/10, ceil(L/block) per axis (computed by the
//    caller in float32);
//  * membership: a sphere belongs to block (n, m, p) when every one of the
//    six boundary distances of set_segments (:65-115) is below 1 um, in
//    float32 and in the reference's operation order;
//  * a pair (a, b) of spheres of different fibres collides when
//    (r_a + r_b + buff) - |x_a - x_b| > 0 in float32 (intersect_block,
//    :52-63); it is reported once as (min, max), rows in lexicographic
//    order (torch.unique).
// The reference also tests pairs among the padding entries of its
// K-per-block table; those add pairs only for spheres that belong to no
// block (more than 1 um outside the grid), and which of those it tests
// depends on its sort's tie order.  Such spheres take part in no pair here.
//
// Work per block here: every pair of the block's members, once; a pair is
// emitted by the first block (lowest id) both spheres belong to, found from
// their two block ranges, so no deduplication pass is needed.
#include <cstdint>
#include "kernels.cuh"

namespace nz {

struct CollideGrid {
  float Lx, Ly, Lz;     // box (the reference's Lx, Ly, Lz)
  float dLx, dLy, dLz;  // block edges, Lx / nx in float32
  float hx, hy, hz;     // Lx / 2 in float32
  int nx, ny, nz;
};

// Blocks [lo, hi] of one axis whose two distances are both below 1 um,
// float32 as set_segments evaluates them: n*dL - r - x - L/2 and
// x - ((n+1)*dL + r - L/2).  Both are monotone in n (lo falls, hi rises), so
// a window around the sphere is scanned; empty when lo > hi.
__device__ __forceinline__ void block_range(float x, float r, float dL, float h, int nseg, int& lo, int& hi) {
  const float c = (x + h) / dL;
  int a = int(floorf(c - (r + 1.0f) / dL)) - 2;
  int b = int(ceilf(c + (r + 1.0f) / dL)) + 2;
  a = max(a, 0);
  b = min(b, nseg - 1);
  lo = 1;
  hi = 0;
  for (int n = a; n <= b; ++n) {
    const float t0 = float(n) * dL - r - x - h;
    const float t1 = x - (float(n + 1) * dL + r - h);
    if (t0 < 1.0f && t1 < 1.0f) {
      if (lo > hi) lo = n;
      hi = n;
    }
  }
}

__global__ void collide_count_kernel(const float* __restrict__ pos, const float* __restrict__ rad, int S, CollideGrid g,
                                     int* __restrict__ ranges, int* __restrict__ counts) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const float x = pos[3 * size_t(s)], y = pos[3 * size_t(s) + 1], z = pos[3 * size_t(s) + 2], r = rad[s];
  int x0, x1, y0, y1, z0, z1;
  block_range(x, r, g.dLx, g.hx, g.nx, x0, x1);
  block_range(y, r, g.dLy, g.hy, g.ny, y0, y1);
  block_range(z, r, g.dLz, g.hz, g.nz, z0, z1);
  int* rr = ranges + 6 * size_t(s);
  rr[0] = x0; rr[1] = x1; rr[2] = y0; rr[3] = y1; rr[4] = z0; rr[5] = z1;
  for (int p = z0; p <= z1; ++p)
    for (int m = y0; m <= y1; ++m)
      for (int n = x0; n <= x1; ++n) atomicAdd(counts + (size_t(p) * g.ny + m) * g.nx + n, 1);
}

__global__ void collide_fill_kernel(const int* __restrict__ ranges, int S, CollideGrid g,
                                    const int* __restrict__ offsets, int* __restrict__ cursor,
                                    int* __restrict__ items) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const int* rr = ranges + 6 * size_t(s);
  for (int p = rr[4]; p <= rr[5]; ++p)
    for (int m = rr[2]; m <= rr[3]; ++m)
      for (int n = rr[0]; n <= rr[1]; ++n) {
        const size_t c = (size_t(p) * g.ny + m) * g.nx + n;
        items[offsets[c] + atomicAdd(cursor + c, 1)] = s;
      }
}

// Every pair of one block's members; one CTA per block.  The pair is emitted
// by the block at the low corner of the two spheres' common block range.
__global__ void __launch_bounds__(256) collide_pairs_kernel(const float* __restrict__ pos,
                                                            const float* __restrict__ rad,
                                                            const float* __restrict__ fid,
                                                            const int* __restrict__ ranges, CollideGrid g,
                                                            const int* __restrict__ offsets,
                                                            const int* __restrict__ counts,
                                                            const int* __restrict__ items, float buff,
                                                            int2* __restrict__ pairs, int cap,
                                                            int* __restrict__ n_pairs) {
  const int c = blockIdx.x;
  const int k = counts[c];
  const int* it = items + offsets[c];
  const long long kk = 1ll * k * k;
  for (long long t = threadIdx.x; t < kk; t += blockDim.x) {
    const int i = int(t / k), j = int(t % k);
    if (i >= j) continue;
    const int a = it[i], b = it[j];
    if (fid[a] == fid[b]) continue;
    const float dx = pos[3 * size_t(a)] - pos[3 * size_t(b)];
    const float dy = pos[3 * size_t(a) + 1] - pos[3 * size_t(b) + 1];
    const float dz = pos[3 * size_t(a) + 2] - pos[3 * size_t(b) + 2];
    const float dm = sqrtf(dx * dx + dy * dy + dz * dz);
    if (!((rad[a] + rad[b]) + buff - dm > 0.0f)) continue;
    const int* ra = ranges + 6 * size_t(a);
    const int* rb = ranges + 6 * size_t(b);
    const int first = (max(ra[4], rb[4]) * g.ny + max(ra[2], rb[2])) * g.nx + max(ra[0], rb[0]);
    if (first != c) continue;
    const int slot = atomicAdd(n_pairs, 1);
    if (slot < cap) pairs[slot] = make_int2(min(a, b), max(a, b));
  }
}

// Lexicographic order of the pairs: a counting sort by the first index,
// then each first index's seconds sorted (a heapsort per first index).
__global__ void pair_hist_kernel(const int2* __restrict__ pairs, int n, int* __restrict__ hist) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) atomicAdd(hist + pairs[t].x, 1);
}

__global__ void pair_scatter_kernel(const int2* __restrict__ pairs, int n, const int* __restrict__ start,
                                    int* __restrict__ cursor, int2* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int2 p = pairs[t];
  out[start[p.x] + atomicAdd(cursor + p.x, 1)] = p;
}

__global__ void pair_bucket_sort_kernel(const int* __restrict__ start, const int* __restrict__ hist, int S,
                                        int2* __restrict__ out) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= S) return;
  int2* v = out + start[a];
  const int n = hist[a];
  for (int i = 1; i < n; ++i) {  // buckets hold a sphere's few collisions: insertion sort
    const int2 x = v[i];
    int j = i - 1;
    while (j >= 0 && v[j].y > x.y) {
      v[j + 1] = v[j];
      --j;
    }
    v[j + 1] = x;
  }
}

static inline size_t al256(size_t v) { return (v + 255) & ~size_t(255); }

static int check_collide_grid(const nz_grid* g, const char* who) {
  if (!g || g->nx <= 0 || g->ny <= 0 || g->nz <= 0 || !(g->dLx > 0.f) || !(g->dLy > 0.f) || !(g->dLz > 0.f))
    return set_error(NZ_ERR_ARG, "%s: grid needs nx, ny, nz > 0 and positive block edges", who);
  if (1ll * g->nx * g->ny * g->nz > (1 << 28)) return set_error(NZ_ERR_ARG, "%s: too many blocks", who);
  return NZ_OK;
}

static CollideGrid collide_grid(const nz_grid& g) {
  return CollideGrid{g.Lx, g.Ly, g.Lz, g.dLx, g.dLy, g.dLz, g.Lx / 2.0f, g.Ly / 2.0f, g.Lz / 2.0f, g.nx, g.ny, g.nz};
}

}  // namespace nz

using namespace nz;

extern "C" size_t nz_collide_scratch_bytes(int S, const nz_grid* grid) {
  if (S < 0 || !grid || grid->nx <= 0 || grid->ny <= 0 || grid->nz <= 0) return 0;
  const size_t ncell = size_t(grid->nx) * grid->ny * grid->nz;
  const size_t nmax = ncell > size_t(S) ? ncell : size_t(S);
  // block ranges; counts, offsets, cursor; scan tiles
  return al256(6 * size_t(S) * sizeof(int)) + 3 * al256(nmax * sizeof(int)) +
         2 * al256(size_t(scan_tiles(int(nmax))) * sizeof(int));
}

extern "C" int nz_collide_cells(const float* pos, const float* radii, int S, const nz_grid* grid, int* n_members,
                                void* scratch, size_t scratch_bytes, void* stream) {
  int rc = check_collide_grid(grid, "nz_collide_cells");
  if (rc) return rc;
  if (S < 0 || !n_members || (S > 0 && (!pos || !radii)))
    return set_error(NZ_ERR_ARG, "nz_collide_cells: bad arguments (S=%d)", S);
  const size_t need = nz_collide_scratch_bytes(S, grid);
  if (!scratch || scratch_bytes < need)
    return set_error(NZ_ERR_CAPACITY, "nz_collide_cells: scratch %zu bytes < %zu", scratch_bytes, need);
  const CollideGrid g = collide_grid(*grid);
  const int ncell = grid->nx * grid->ny * grid->nz;
  const size_t nmax = size_t(ncell) > size_t(S) ? size_t(ncell) : size_t(S);
  char* p = static_cast<char*>(scratch);
  int* ranges = reinterpret_cast<int*>(p);
  int* counts = reinterpret_cast<int*>(p + al256(6 * size_t(S) * sizeof(int)));
  int* offsets = counts + al256(nmax * sizeof(int)) / sizeof(int);
  int* cursor = offsets + al256(nmax * sizeof(int)) / sizeof(int);
  int* tile_sums = cursor + al256(nmax * sizeof(int)) / sizeof(int);
  int* tile_offsets = tile_sums + al256(size_t(scan_tiles(int(nmax))) * sizeof(int)) / sizeof(int);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(counts, 0, size_t(ncell) * sizeof(int), st) != cudaSuccess)
    return check_launch("nz_collide_cells memset");
  if (S > 0) {
    collide_count_kernel<<<(S + 255) / 256, 256, 0, st>>>(pos, radii, S, g, ranges, counts);
    rc = check_launch("collide_count_kernel");
    if (rc) return rc;
  }
  rc = exclusive_scan(counts, offsets, ncell, tile_sums, tile_offsets, st);
  if (rc) return rc;
  offsets_total_kernel<<<1, 1, 0, st>>>(counts, offsets, ncell, n_members);
  return check_launch("offsets_total_kernel");
}

extern "C" int nz_collide_pairs(const float* pos, const float* radii, const float* fiber_id, int S,
                                const nz_grid* grid, float buff, int* items, int n_members, int* pairs, int cap,
                                int* n_pairs, void* scratch, size_t scratch_bytes, void* stream) {
  int rc = check_collide_grid(grid, "nz_collide_pairs");
  if (rc) return rc;
  if (S < 0 || n_members < 0 || cap < 0 || !n_pairs || (S > 0 && (!pos || !radii || !fiber_id)) ||
      (n_members > 0 && !items) || (cap > 0 && !pairs))
    return set_error(NZ_ERR_ARG, "nz_collide_pairs: bad arguments (S=%d members=%d cap=%d)", S, n_members, cap);
  const size_t need = nz_collide_scratch_bytes(S, grid);
  if (!scratch || scratch_bytes < need)
    return set_error(NZ_ERR_CAPACITY, "nz_collide_pairs: scratch %zu bytes < %zu", scratch_bytes, need);
  const CollideGrid g = collide_grid(*grid);
  const int ncell = grid->nx * grid->ny * grid->nz;
  const size_t nmax = size_t(ncell) > size_t(S) ? size_t(ncell) : size_t(S);
  char* p = static_cast<char*>(scratch);
  int* ranges = reinterpret_cast<int*>(p);
  int* counts = reinterpret_cast<int*>(p + al256(6 * size_t(S) * sizeof(int)));
  int* offsets = counts + al256(nmax * sizeof(int)) / sizeof(int);
  int* cursor = offsets + al256(nmax * sizeof(int)) / sizeof(int);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(n_pairs, 0, sizeof(int), st) != cudaSuccess) return check_launch("nz_collide_pairs memset");
  if (S == 0 || n_members == 0) return NZ_OK;
  if (cudaMemsetAsync(cursor, 0, size_t(ncell) * sizeof(int), st) != cudaSuccess)
    return check_launch("nz_collide_pairs memset");
  collide_fill_kernel<<<(S + 255) / 256, 256, 0, st>>>(ranges, S, g, offsets, cursor, items);
  rc = check_launch("collide_fill_kernel");
  if (rc) return rc;
  collide_pairs_kernel<<<ncell, 256, 0, st>>>(pos, radii, fiber_id, ranges, g, offsets, counts, items, buff,
                                              reinterpret_cast<int2*>(pairs), cap, n_pairs);
  return check_launch("collide_pairs_kernel");
}

extern "C" size_t nz_pairs_sort_scratch_bytes(int S) {
  if (S < 0) return 0;
  return 3 * al256(size_t(S) * sizeof(int)) + 2 * al256(size_t(scan_tiles(S)) * sizeof(int));
}

extern "C" int nz_pairs_sort(const int* pairs, int n, int S, int* out, void* scratch, size_t scratch_bytes,
                             void* stream) {
  if (n < 0 || S < 0 || (n > 0 && (!pairs || !out || S == 0)))
    return set_error(NZ_ERR_ARG, "nz_pairs_sort: bad arguments (n=%d S=%d)", n, S);
  if (n == 0) return NZ_OK;
  const size_t need = nz_pairs_sort_scratch_bytes(S);
  if (!scratch || scratch_bytes < need)
    return set_error(NZ_ERR_CAPACITY, "nz_pairs_sort: scratch %zu bytes < %zu", scratch_bytes, need);
  char* p = static_cast<char*>(scratch);
  const size_t ns = al256(size_t(S) * sizeof(int));
  int* hist = reinterpret_cast<int*>(p);
  int* start = reinterpret_cast<int*>(p + ns);
  int* cursor = reinterpret_cast<int*>(p + 2 * ns);
  int* tile_sums = reinterpret_cast<int*>(p + 3 * ns);
  int* tile_offsets = reinterpret_cast<int*>(p + 3 * ns + al256(size_t(scan_tiles(S)) * sizeof(int)));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(hist, 0, size_t(S) * sizeof(int), st) != cudaSuccess ||
      cudaMemsetAsync(cursor, 0, size_t(S) * sizeof(int), st) != cudaSuccess)
    return check_launch("nz_pairs_sort memset");
  const int2* in = reinterpret_cast<const int2*>(pairs);
  int2* o = reinterpret_cast<int2*>(out);
  pair_hist_kernel<<<(n + 255) / 256, 256, 0, st>>>(in, n, hist);
  int rc = check_launch("pair_hist_kernel");
  if (rc) return rc;
  rc = exclusive_scan(hist, start, S, tile_sums, tile_offsets, st);
  if (rc) return rc;
  pair_scatter_kernel<<<(n + 255) / 256, 256, 0, st>>>(in, n, start, cursor, o);
  rc = check_launch("pair_scatter_kernel");
  if (rc) return rc;
  pair_bucket_sort_kernel<<<(S + 255) / 256, 256, 0, st>>>(start, hist, S, o);
  return check_launch("pair_bucket_sort_kernel");
}
