// Seeding, walker re-binning, signal and moment reductions.
#include <cstdint>
#include <mutex>
#include "kernels.cuh"

namespace nz {

// ---------------------------------------------------------------------------
// Seeding: seedSpinsKernel's acceptance rule (sim3d_kernel.cu:240-337) with
// the rounds of SimGeometry3D.gpu_seed (geometry.py:146-168) moved inside the
// kernel and bounded.  The label of a point is found from its cell's list:
// every sphere that contains a point of a cell is a member of that cell.
// ---------------------------------------------------------------------------
__global__ void seed_kernel(nz_substrate sub, const uint8_t* __restrict__ target, uint32_t id0, int N, uint32_t k0,
                            uint32_t k1, uint32_t stream, int max_rounds, float* __restrict__ spins,
                            int* __restrict__ label, int* __restrict__ n_unseeded) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= N) return;
  const Grid g{sub.grid.Lx, sub.grid.Ly, sub.grid.Lz, sub.grid.dLx, sub.grid.dLy, sub.grid.dLz,
               float(sub.grid.nx), float(sub.grid.ny), float(sub.grid.nz)};
  const int S = sub.S;
  const float* __restrict__ cx = sub.spheres;
  const float* __restrict__ rr = sub.spheres + 3 * S;
  const float* __restrict__ sphSID = sub.spheres + 4 * S;
  const int ns = sub.nstructures;
  for (int round = 0; round < max_rounds; ++round) {
    float u0, u1, u2;
    philox_uniform3(k0, k1, stream, id0 + uint32_t(w), uint32_t(round), u0, u1, u2);
    const float px = (u0 - 0.5f) * g.Lx;
    const float py = (u1 - 0.5f) * g.Ly;
    const float pz = (u2 - 0.5f) * g.Lz;
    const int cell = cell_of(g, px, py, pz);
    const int start = sub.cell_start[cell], count = sub.cell_count[cell];
    int lab = ns;
    for (int n = 0; n < count; ++n) {
      const int s = sub.cell_items[start + n];
      const float dx = px - cx[s], dy = py - cx[S + s], dz = pz - cx[2 * S + s];
      const int sid = int(sphSID[s]);
      if (dx * dx + dy * dy + dz * dz < rr[s] * rr[s] && sid < lab) lab = sid;
    }
    bool accept;
    if (lab < ns) accept = target[lab] != 0;
    else accept = target[ns] != 0 && px > -g.Lx / 2 && px < g.Lx / 2 && py > -g.Ly / 2 && py < g.Ly / 2 &&
                  pz > -g.Lz / 2 && pz < g.Lz / 2;
    if (accept) {
      spins[w] = px;
      spins[N + w] = py;
      spins[2 * N + w] = pz;
      if (label) label[w] = lab;
      return;
    }
  }
  if (label) label[w] = -1;
  atomicAdd(n_unseeded, 1);
}

// ---------------------------------------------------------------------------
// Re-binning: counting sort of the packed walker state by coarse cell.
// ---------------------------------------------------------------------------
struct BinGrid {
  Grid g;
  int cx, cy, cz;     // coarsening per axis
  int bx, by, bz;     // bins per axis
  int nlabels;        // > 0: key = label * nbins + bin (walkers of one structure together)
};

__device__ __forceinline__ int bin_of(const BinGrid& b, float x, float y, float z) {
  const int c = cell_of(b.g, x, y, z);
  const int nx = int(b.g.nLx), ny = int(b.g.nLy);
  const int ix = c % nx, iy = (c / nx) % ny, iz = c / (nx * ny);
  return ((iz / b.cz) * b.by + iy / b.cy) * b.bx + ix / b.cx;
}

__global__ void bin_count_kernel(const float4* __restrict__ pos, int N, BinGrid b, int* __restrict__ bins,
                                 int* __restrict__ hist) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= N) return;
  const float4 p = pos[w];
  int k = bin_of(b, p.x, p.y, p.z);
  if (b.nlabels > 0) {
    int label = __float_as_int(p.w);
    if (label < 0 || label >= b.nlabels) label = b.nlabels - 1;
    k += label * (b.bx * b.by * b.bz);
  }
  bins[w] = k;
  atomicAdd(hist + k, 1);
}

__global__ void bin_scatter_kernel(nz_state in, int N, const int* __restrict__ bins, int* __restrict__ cursor,
                                   nz_state out) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= N) return;
  const int slot = atomicAdd(cursor + bins[w], 1);
  reinterpret_cast<float4*>(out.pos)[slot] = reinterpret_cast<const float4*>(in.pos)[w];
  reinterpret_cast<float4*>(out.org)[slot] = reinterpret_cast<const float4*>(in.org)[w];
  reinterpret_cast<float4*>(out.phi)[slot] = reinterpret_cast<const float4*>(in.phi)[w];
  reinterpret_cast<float4*>(out.comp)[slot] = reinterpret_cast<const float4*>(in.comp)[w];
}

// ---------------------------------------------------------------------------
// Re-binning of many jobs in one pass: each thread finds its walker's job by a
// binary search over the jobs' walker offsets, then keys it as bin_count_kernel
// does, shifted into the job's key range.  The exclusive scan over the whole
// key space gives each key's first slot in the concatenation of all jobs'
// walkers; a job's walkers occupy [walker_offset, walker_offset + N) of it.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int job_of(const nz_sort_job* __restrict__ jobs, int n_jobs, int g) {
  int lo = 0, hi = n_jobs - 1;  // the last job whose walker_offset <= g
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&jobs[mid].walker_offset) <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ BinGrid bin_grid_of(const nz_grid& grid, int coarsen, int nlabels) {
  BinGrid b;
  b.g = Grid{grid.Lx, grid.Ly, grid.Lz, grid.dLx, grid.dLy, grid.dLz, float(grid.nx), float(grid.ny), float(grid.nz)};
  b.cx = b.cy = b.cz = coarsen;
  b.bx = (grid.nx + coarsen - 1) / coarsen;
  b.by = (grid.ny + coarsen - 1) / coarsen;
  b.bz = (grid.nz + coarsen - 1) / coarsen;
  b.nlabels = nlabels;
  return b;
}

__global__ void batch_bin_count_kernel(const nz_sort_job* __restrict__ jobs, int n_jobs, int total,
                                       int* __restrict__ bins, int* __restrict__ hist) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const int j = job_of(jobs, n_jobs, g);
  const nz_sort_job& J = jobs[j];
  const BinGrid b = bin_grid_of(J.grid, J.coarsen, J.nlabels);
  const float4 p = reinterpret_cast<const float4*>(J.in.pos)[g - J.walker_offset];
  int k = bin_of(b, p.x, p.y, p.z);
  if (b.nlabels > 0) {
    int label = __float_as_int(p.w);
    if (label < 0 || label >= b.nlabels) label = b.nlabels - 1;
    k += label * (b.bx * b.by * b.bz);
  }
  k += J.key_offset;
  bins[g] = k;
  atomicAdd(hist + k, 1);
}

__global__ void batch_bin_scatter_kernel(const nz_sort_job* __restrict__ jobs, int n_jobs, int total,
                                         const int* __restrict__ bins, int* __restrict__ cursor) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const int j = job_of(jobs, n_jobs, g);
  const nz_sort_job& J = jobs[j];
  const int w = g - J.walker_offset;
  const int slot = atomicAdd(cursor + bins[g], 1) - J.walker_offset;
  reinterpret_cast<float4*>(J.out.pos)[slot] = reinterpret_cast<const float4*>(J.in.pos)[w];
  reinterpret_cast<float4*>(J.out.org)[slot] = reinterpret_cast<const float4*>(J.in.org)[w];
  reinterpret_cast<float4*>(J.out.phi)[slot] = reinterpret_cast<const float4*>(J.in.phi)[w];
  reinterpret_cast<float4*>(J.out.comp)[slot] = reinterpret_cast<const float4*>(J.in.comp)[w];
}

// ---------------------------------------------------------------------------
// Signal: S[d][b] += sum_w exp(i amp[b] u_d . Phi_w); FP32 per walker, FP64
// block sums, one FP64 atomic per block and (d, b).
// ---------------------------------------------------------------------------
constexpr int kSigThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* s_red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) s_red[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < (blockDim.x >> 5) ? s_red[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  }
  return t;  // valid in thread 0
}

__global__ void __launch_bounds__(kSigThreads) signal_kernel(nz_state st, const float* __restrict__ dirs, int ndir,
                                                             const float* __restrict__ amp, int nb,
                                                             double* __restrict__ out) {
  __shared__ double s_red[32];
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  float px = 0.f, py = 0.f, pz = 0.f;
  const bool live = w < st.N;
  if (live) {
    const float4 f = reinterpret_cast<const float4*>(st.phi)[w];
    const float4 c = reinterpret_cast<const float4*>(st.comp)[w];
    px = f.x - c.x;
    py = f.y - c.y;
    pz = f.z - c.z;
  }
  for (int d = 0; d < ndir; ++d) {
    const float ph = px * __ldg(dirs + d) + py * __ldg(dirs + ndir + d) + pz * __ldg(dirs + 2 * ndir + d);
    for (int b = 0; b < nb; ++b) {
      float sn = 0.f, cs = 0.f;
      if (live) sincosf(__ldg(amp + b) * ph, &sn, &cs);
      const double re = block_sum(live ? double(cs) : 0.0, s_red);
      const double im = block_sum(live ? double(sn) : 0.0, s_red);
      if (threadIdx.x == 0) {
        atomicAdd(out + d * nb + b, re);
        atomicAdd(out + ndir * nb + d * nb + b, im);
      }
    }
  }
}

__global__ void __launch_bounds__(kSigThreads) signal_phase_kernel(const float* __restrict__ phase, int ndir, int N,
                                                                   const float* __restrict__ amp, int nb,
                                                                   double* __restrict__ out) {
  __shared__ double s_red[32];
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = w < N;
  for (int d = 0; d < ndir; ++d) {
    const float ph = live ? phase[size_t(d) * N + w] : 0.f;
    for (int b = 0; b < nb; ++b) {
      float sn = 0.f, cs = 0.f;
      if (live) sincosf(__ldg(amp + b) * ph, &sn, &cs);
      const double re = block_sum(live ? double(cs) : 0.0, s_red);
      const double im = block_sum(live ? double(sn) : 0.0, s_red);
      if (threadIdx.x == 0) {
        atomicAdd(out + d * nb + b, re);
        atomicAdd(out + ndir * nb + d * nb + b, im);
      }
    }
  }
}

__global__ void phase_from_phi_kernel(nz_state st, const float* __restrict__ dirs, int ndir, float* __restrict__ phase) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= st.N) return;
  const float4 f = reinterpret_cast<const float4*>(st.phi)[w];
  const float4 c = reinterpret_cast<const float4*>(st.comp)[w];
  const float px = f.x - c.x, py = f.y - c.y, pz = f.z - c.z;
  for (int d = 0; d < ndir; ++d)
    phase[size_t(d) * st.N + w] = px * dirs[d] + py * dirs[ndir + d] + pz * dirs[2 * ndir + d];
}

// computeDiffusionCoefficientsAndKurtosis's sums (sim3d_kernel.cu:193-200) in FP64.
__global__ void __launch_bounds__(256) moments_kernel(const float* __restrict__ spins, const float* __restrict__ spins0,
                                                      int N, double* __restrict__ out) {
  __shared__ double s_red[32];
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  double m[6] = {0, 0, 0, 0, 0, 0};
  if (w < N) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float d = spins[size_t(a) * N + w] - spins0[size_t(a) * N + w];
      const double d2 = double(d) * double(d);
      m[a] = d2;
      m[3 + a] = d2 * d2;
    }
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    const double t = block_sum(m[i], s_red);
    if (threadIdx.x == 0) atomicAdd(out + i, t);
  }
}

// The moments of every step of a fused launch from the displacements it
// stored: step blockIdx.y, walkers strided over blockIdx.x; each term is
// moments_kernel's (float displacement, squared and summed in FP64).
__global__ void __launch_bounds__(256) disp_moments_kernel(const float* __restrict__ disp, int N,
                                                           double* __restrict__ out) {
  __shared__ double s_red[32];
  const float* d = disp + size_t(blockIdx.y) * 3 * size_t(N);
  double m[6] = {0, 0, 0, 0, 0, 0};
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < N; w += gridDim.x * blockDim.x) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float v = d[size_t(a) * N + w];
      const double v2 = double(v) * double(v);
      m[a] += v2;
      m[3 + a] += v2 * v2;
    }
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    const double t = block_sum(m[i], s_red);
    if (threadIdx.x == 0) atomicAdd(out + size_t(blockIdx.y) * 6 + i, t);
  }
}

}  // namespace nz

using namespace nz;

extern "C" int nz_seed_range(const nz_substrate* sub, const uint8_t* target, uint32_t id0, int N, uint32_t key0,
                             uint32_t key1, uint32_t stream_id, int max_rounds, float* spins, int* label,
                             int* n_unseeded, void* stream) {
  if (!sub || !target || N < 0 || max_rounds <= 0 || (N > 0 && !spins) || !n_unseeded || !sub->cell_start ||
      !sub->cell_count || !sub->cell_items || (sub->S > 0 && !sub->spheres) ||
      uint64_t(id0) + uint64_t(N) > (uint64_t(1) << 32))
    return set_error(NZ_ERR_ARG, "nz_seed_range: bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(n_unseeded, 0, sizeof(int), st) != cudaSuccess) return check_launch("nz_seed memset");
  if (N == 0) return NZ_OK;
  seed_kernel<<<(N + 255) / 256, 256, 0, st>>>(*sub, target, id0, N, key0, key1, stream_id, max_rounds, spins,
                                                label, n_unseeded);
  return check_launch("seed_kernel");
}

extern "C" int nz_seed(const nz_substrate* sub, const uint8_t* target, int N, uint32_t key0, uint32_t key1,
                       uint32_t stream_id, int max_rounds, float* spins, int* label, int* n_unseeded, void* stream) {
  return nz_seed_range(sub, target, 0, N, key0, key1, stream_id, max_rounds, spins, label, n_unseeded, stream);
}

static inline size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

extern "C" size_t nz_sort_scratch_bytes(int N, int nbins) {
  if (N < 0 || nbins < 0) return 0;
  return align256(size_t(N) * sizeof(int)) + 2 * align256(size_t(nbins) * sizeof(int)) +
         2 * align256(size_t(scan_tiles(nbins)) * sizeof(int));
}

extern "C" int nz_state_sort_keyed(const nz_state* in, const nz_grid* grid, int coarsen, int nlabels, nz_state* out,
                                   void* scratch, size_t scratch_bytes, void* stream) {
  int rc = check_state(in, "nz_state_sort (in)");
  if (rc == NZ_OK) rc = check_state(out, "nz_state_sort (out)");
  if (rc == NZ_OK) rc = check_grid(grid, "nz_state_sort");
  if (rc) return rc;
  if (coarsen <= 0 || nlabels < 0 || in->N != out->N || !scratch)
    return set_error(NZ_ERR_ARG, "nz_state_sort: bad arguments");
  if (in->N > 0 && (in->pos == out->pos || in->org == out->org || in->phi == out->phi || in->comp == out->comp))
    return set_error(NZ_ERR_ARG, "nz_state_sort: in and out share an array (the sort is out of place)");
  BinGrid b;
  b.g = Grid{grid->Lx, grid->Ly, grid->Lz, grid->dLx, grid->dLy, grid->dLz, float(grid->nx), float(grid->ny),
             float(grid->nz)};
  b.cx = b.cy = b.cz = coarsen;
  b.bx = (grid->nx + coarsen - 1) / coarsen;
  b.by = (grid->ny + coarsen - 1) / coarsen;
  b.bz = (grid->nz + coarsen - 1) / coarsen;
  b.nlabels = nlabels;
  const long long nbins = 1ll * b.bx * b.by * b.bz * (nlabels > 0 ? nlabels : 1);
  if (nbins > (1 << 26)) return set_error(NZ_ERR_ARG, "nz_state_sort: %lld keys, coarsen more", nbins);
  const int N = in->N;
  const size_t need = nz_sort_scratch_bytes(N, int(nbins));
  if (scratch_bytes < need)
    return set_error(NZ_ERR_CAPACITY, "nz_state_sort: scratch %zu bytes < %zu", scratch_bytes, need);
  if (N == 0) return NZ_OK;
  char* p = static_cast<char*>(scratch);
  int* bins = reinterpret_cast<int*>(p);
  int* hist = reinterpret_cast<int*>(p + align256(size_t(N) * sizeof(int)));
  int* cursor = reinterpret_cast<int*>(p + align256(size_t(N) * sizeof(int)) + align256(size_t(nbins) * sizeof(int)));
  int* tile_sums = reinterpret_cast<int*>(reinterpret_cast<char*>(cursor) + align256(size_t(nbins) * sizeof(int)));
  int* tile_offsets = reinterpret_cast<int*>(reinterpret_cast<char*>(tile_sums) +
                                             align256(size_t(scan_tiles(int(nbins))) * sizeof(int)));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(hist, 0, size_t(nbins) * sizeof(int), st) != cudaSuccess) return check_launch("sort memset");
  bin_count_kernel<<<(N + 255) / 256, 256, 0, st>>>(reinterpret_cast<const float4*>(in->pos), N, b, bins, hist);
  rc = check_launch("bin_count_kernel");
  if (rc) return rc;
  rc = exclusive_scan(hist, cursor, int(nbins), tile_sums, tile_offsets, st);
  if (rc) return rc;
  bin_scatter_kernel<<<(N + 255) / 256, 256, 0, st>>>(*in, N, bins, cursor, *out);
  return check_launch("bin_scatter_kernel");
}

extern "C" long long nz_sort_job_keys(const nz_grid* grid, int coarsen, int nlabels) {
  if (!grid || grid->nx <= 0 || grid->ny <= 0 || grid->nz <= 0 || coarsen <= 0 || nlabels < 0) return -1;
  return 1ll * ((grid->nx + coarsen - 1) / coarsen) * ((grid->ny + coarsen - 1) / coarsen) *
         ((grid->nz + coarsen - 1) / coarsen) * (nlabels > 0 ? nlabels : 1);
}

extern "C" size_t nz_batch_sort_scratch_bytes(int total_walkers, int total_keys) {
  return nz_sort_scratch_bytes(total_walkers, total_keys);
}

extern "C" int nz_batch_sort(const nz_sort_job* jobs, int n_jobs, int total_walkers, int total_keys, void* scratch,
                             size_t scratch_bytes, void* stream) {
  if (n_jobs < 0 || total_walkers < 0 || total_keys < 0 || (n_jobs > 0 && !jobs) ||
      (total_walkers > 0 && (n_jobs == 0 || total_keys == 0)))
    return set_error(NZ_ERR_ARG, "nz_batch_sort: bad arguments (jobs=%d walkers=%d keys=%d)", n_jobs, total_walkers,
                     total_keys);
  if (total_walkers == 0) return NZ_OK;
  const size_t need = nz_sort_scratch_bytes(total_walkers, total_keys);
  if (!scratch || scratch_bytes < need)
    return set_error(NZ_ERR_CAPACITY, "nz_batch_sort: scratch %zu bytes < %zu", scratch_bytes, need);
  char* p = static_cast<char*>(scratch);
  const size_t nw = align256(size_t(total_walkers) * sizeof(int)), nk = align256(size_t(total_keys) * sizeof(int));
  int* bins = reinterpret_cast<int*>(p);
  int* hist = reinterpret_cast<int*>(p + nw);
  int* cursor = reinterpret_cast<int*>(p + nw + nk);
  int* tile_sums = reinterpret_cast<int*>(p + nw + 2 * nk);
  int* tile_offsets = reinterpret_cast<int*>(p + nw + 2 * nk + align256(size_t(scan_tiles(total_keys)) * sizeof(int)));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(hist, 0, size_t(total_keys) * sizeof(int), st) != cudaSuccess)
    return check_launch("nz_batch_sort memset");
  const unsigned blocks = unsigned((total_walkers + 255) / 256);
  batch_bin_count_kernel<<<blocks, 256, 0, st>>>(jobs, n_jobs, total_walkers, bins, hist);
  int rc = check_launch("batch_bin_count_kernel");
  if (rc) return rc;
  rc = exclusive_scan(hist, cursor, total_keys, tile_sums, tile_offsets, st);
  if (rc) return rc;
  batch_bin_scatter_kernel<<<blocks, 256, 0, st>>>(jobs, n_jobs, total_walkers, bins, cursor);
  return check_launch("batch_bin_scatter_kernel");
}

extern "C" int nz_state_sort(const nz_state* in, const nz_grid* grid, int coarsen, nz_state* out, void* scratch,
                             size_t scratch_bytes, void* stream) {
  return nz_state_sort_keyed(in, grid, coarsen, 0, out, scratch, scratch_bytes, stream);
}

extern "C" int nz_signal_phi(const nz_state* st, const float* dirs, int ndir, const float* amp, int nb, double* out,
                             void* stream) {
  const int rc = check_state(st, "nz_signal_phi");
  if (rc) return rc;
  if (!dirs || !amp || !out || ndir <= 0 || nb <= 0) return set_error(NZ_ERR_ARG, "nz_signal_phi: bad arguments");
  if (st->N == 0) return NZ_OK;
  signal_kernel<<<(st->N + kSigThreads - 1) / kSigThreads, kSigThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      *st, dirs, ndir, amp, nb, out);
  return check_launch("signal_kernel");
}

extern "C" int nz_signal_phase(const float* phase, int ndir, int N, const float* amp, int nb, double* out,
                               void* stream) {
  if (!phase || !amp || !out || ndir <= 0 || nb <= 0 || N < 0)
    return set_error(NZ_ERR_ARG, "nz_signal_phase: bad arguments");
  if (N == 0) return NZ_OK;
  signal_phase_kernel<<<(N + kSigThreads - 1) / kSigThreads, kSigThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      phase, ndir, N, amp, nb, out);
  return check_launch("signal_phase_kernel");
}

extern "C" int nz_phase_from_phi(const nz_state* st, const float* dirs, int ndir, float* phase, void* stream) {
  const int rc = check_state(st, "nz_phase_from_phi");
  if (rc) return rc;
  if (!dirs || (st->N > 0 && !phase) || ndir <= 0) return set_error(NZ_ERR_ARG, "nz_phase_from_phi: bad arguments");
  if (st->N == 0) return NZ_OK;
  phase_from_phi_kernel<<<(st->N + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(*st, dirs, ndir, phase);
  return check_launch("phase_from_phi_kernel");
}

extern "C" int nz_moments(const float* spins, const float* spins0, int N, double* out, void* stream) {
  if (!spins || !spins0 || !out || N < 0) return set_error(NZ_ERR_ARG, "nz_moments: bad arguments");
  if (N == 0) return NZ_OK;
  moments_kernel<<<(N + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(spins, spins0, N, out);
  return check_launch("moments_kernel");
}

// ---------------------------------------------------------------------------
// Re-binning without caller-provided scratch.  Some hosts cannot hand this
// library a device buffer: their memory manager reserves all device memory
// at start-up and forbids allocation afterwards, or an allocation's implicit
// synchronisation would stall their other streams.  For them the sort's
// scratch lives in a fixed device array of this file, one copy per GPU that
// loads the library, kept until the process exits.
// ---------------------------------------------------------------------------
namespace nz {
constexpr size_t kStaticSortScratch = size_t(16) << 20;  // 16 MiB per GPU
static __device__ __align__(256) unsigned char g_sort_scratch[kStaticSortScratch];

// Device address of g_sort_scratch on the current device, looked up once per
// device (the host-side name of a __device__ array is not a device address).
static int static_sort_scratch(void** out) {
  static std::mutex mu;
  static void* addr[kMaxDevices] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return check_launch("nz_state_sort_static: cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return set_error(NZ_ERR_ARG, "nz_state_sort_static: device %d out of range", dev);
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
    if (e != cudaSuccess)
      return set_error(NZ_ERR_CUDA, "nz_state_sort_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    addr[dev] = p;
  }
  *out = addr[dev];
  return NZ_OK;
}
}  // namespace nz

extern "C" size_t nz_state_sort_static_capacity(void) { return kStaticSortScratch; }

extern "C" int nz_state_sort_static(const nz_state* in, const nz_grid* grid, int coarsen, nz_state* out,
                                    void* stream) {
  int rc = check_grid(grid, "nz_state_sort_static");
  if (rc) return rc;
  if (!in || coarsen <= 0) return set_error(NZ_ERR_ARG, "nz_state_sort_static: bad arguments");
  const long long nbins = 1ll * ((grid->nx + coarsen - 1) / coarsen) * ((grid->ny + coarsen - 1) / coarsen) *
                          ((grid->nz + coarsen - 1) / coarsen);
  if (in->N < 0 || nbins > (1 << 26)) return set_error(NZ_ERR_ARG, "nz_state_sort_static: bad sizes");
  const size_t need = nz_sort_scratch_bytes(in->N, int(nbins));
  if (need > kStaticSortScratch)
    return set_error(NZ_ERR_CAPACITY,
                     "nz_state_sort_static: %d walkers and %lld bins need %zu bytes of scratch, more than the "
                     "fixed %zu; use nz_state_sort with a caller buffer or coarsen the bins",
                     in->N, nbins, need, kStaticSortScratch);
  void* scratch = nullptr;
  rc = static_sort_scratch(&scratch);
  if (rc != NZ_OK) return rc;
  return nz_state_sort(in, grid, coarsen, out, scratch, kStaticSortScratch, stream);
}
