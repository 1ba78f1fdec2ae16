// Uniform-grid cell lists on the GPU: the work of DiffSim3d.set_segments
// (simulation_toolkit/simulation_engine/diffsim3d.py:107-174), which the
// reference does on the host with a numpy loop over cells x spheres (twice) and
// an argsort per cell.
//
// Membership is the reference's predicate, in float64 and in its operation
// order (diffsim3d.py:128-141): sphere s belongs to cell (n, m, p) when all six
// boundary distances of its bounding box are below jump_tol.  The predicate is
// separable per axis and, per axis, monotone in the cell index, so each sphere
// enumerates only the box of cells it can belong to.
#include <cstdint>
#include "kernels.cuh"

namespace nz {

// in_segment's two terms on one axis for cell index n (diffsim3d.py:128-133).
__device__ __forceinline__ double seg_lo(double n, double dL, double r, double x, double L) {
  return __dsub_rn(__dsub_rn(__dsub_rn(__dmul_rn(n, dL), r), x), L / 2);
}
__device__ __forceinline__ double seg_hi(double n, double dL, double r, double x, double L) {
  return __dsub_rn(x, __dsub_rn(__dadd_rn(__dmul_rn(n + 1, dL), r), L / 2));
}

// Valid cell range [lo, hi] on one axis (empty when lo > hi).
__device__ __forceinline__ void axis_range(double x, double r, double L, int nseg, double tol, int& lo, int& hi) {
  const double dL = L / nseg;
  int a = int(floor((x - r + L / 2 - tol) / dL)) - 2;
  int b = int(ceil((tol + r + x + L / 2) / dL)) + 2;
  a = max(a, 0);
  b = min(b, nseg - 1);
  lo = 1;
  hi = 0;
  for (int n = a; n <= b; ++n) {
    const bool ok = seg_lo(double(n), dL, r, x, L) < tol && seg_hi(double(n), dL, r, x, L) < tol;
    if (ok) {
      if (lo > hi) lo = n;
      hi = n;
    }
  }
}

struct CellGeom {
  double Lx, Ly, Lz;
  int nx, ny, nz;
  double tol;
};

__global__ void cells_count_kernel(const double* __restrict__ sph, int S, CellGeom g, int* __restrict__ counts) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const double x = sph[s], y = sph[S + s], z = sph[2 * S + s], r = sph[3 * S + s];
  int x0, x1, y0, y1, z0, z1;
  axis_range(x, r, g.Lx, g.nx, g.tol, x0, x1);
  axis_range(y, r, g.Ly, g.ny, g.tol, y0, y1);
  axis_range(z, r, g.Lz, g.nz, g.tol, z0, z1);
  for (int p = z0; p <= z1; ++p)
    for (int m = y0; m <= y1; ++m)
      for (int n = x0; n <= x1; ++n) atomicAdd(counts + (size_t(p) * g.ny + m) * g.nx + n, 1);
}

__global__ void cells_fill_kernel(const double* __restrict__ sph, int S, CellGeom g, const int* __restrict__ offsets,
                                  int* __restrict__ cursor, int* __restrict__ items) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const double x = sph[s], y = sph[S + s], z = sph[2 * S + s], r = sph[3 * S + s];
  int x0, x1, y0, y1, z0, z1;
  axis_range(x, r, g.Lx, g.nx, g.tol, x0, x1);
  axis_range(y, r, g.Ly, g.ny, g.tol, y0, y1);
  axis_range(z, r, g.Lz, g.nz, g.tol, z0, z1);
  for (int p = z0; p <= z1; ++p)
    for (int m = y0; m <= y1; ++m)
      for (int n = x0; n <= x1; ++n) {
        const size_t c = (size_t(p) * g.ny + m) * g.nx + n;
        const int slot = atomicAdd(cursor + c, 1);
        items[offsets[c] + slot] = s;
      }
}

// Rounded membership, for the fused walk's near lists: a sphere is listed in
// a cell of its box-test window (in_segment < margin) only when the
// Euclidean distance from its centre to the cell's box is at most
// r + margin + 1e-4 um.  A walker in the cell (or within d of it) can touch
// or lie inside only spheres whose centre is within r + tol + reach + d of
// the box, and the fused walk takes the near list only while
// (d + reach) * 1.02 + tol + 2 nm <= margin, so these lists hold every
// sphere the walk can meet; the corners of the box test's window, about a
// third of its entries for cells small beside the spheres, are left out.
__device__ __forceinline__ bool within_round(double x, double y, double z, double r, const CellGeom& g, int n, int m,
                                             int p) {
  const double dLx = g.Lx / g.nx, dLy = g.Ly / g.ny, dLz = g.Lz / g.nz;
  const double x0 = n * dLx - g.Lx / 2, y0 = m * dLy - g.Ly / 2, z0 = p * dLz - g.Lz / 2;
  const double ex = fmax(fmax(x0 - x, 0.0), x - (x0 + dLx));
  const double ey = fmax(fmax(y0 - y, 0.0), y - (y0 + dLy));
  const double ez = fmax(fmax(z0 - z, 0.0), z - (z0 + dLz));
  const double R = r + g.tol + 1e-4;
  return ex * ex + ey * ey + ez * ez <= R * R;
}

__global__ void cells_count_round_kernel(const double* __restrict__ sph, int S, CellGeom g, int* __restrict__ counts) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const double x = sph[s], y = sph[S + s], z = sph[2 * S + s], r = sph[3 * S + s];
  int x0, x1, y0, y1, z0, z1;
  axis_range(x, r, g.Lx, g.nx, g.tol, x0, x1);
  axis_range(y, r, g.Ly, g.ny, g.tol, y0, y1);
  axis_range(z, r, g.Lz, g.nz, g.tol, z0, z1);
  for (int p = z0; p <= z1; ++p)
    for (int m = y0; m <= y1; ++m)
      for (int n = x0; n <= x1; ++n)
        if (within_round(x, y, z, r, g, n, m, p)) atomicAdd(counts + (size_t(p) * g.ny + m) * g.nx + n, 1);
}

__global__ void cells_fill_round_kernel(const double* __restrict__ sph, int S, CellGeom g,
                                        const int* __restrict__ offsets, int* __restrict__ cursor,
                                        int* __restrict__ items) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const double x = sph[s], y = sph[S + s], z = sph[2 * S + s], r = sph[3 * S + s];
  int x0, x1, y0, y1, z0, z1;
  axis_range(x, r, g.Lx, g.nx, g.tol, x0, x1);
  axis_range(y, r, g.Ly, g.ny, g.tol, y0, y1);
  axis_range(z, r, g.Lz, g.nz, g.tol, z0, z1);
  for (int p = z0; p <= z1; ++p)
    for (int m = y0; m <= y1; ++m)
      for (int n = x0; n <= x1; ++n) {
        if (!within_round(x, y, z, r, g, n, m, p)) continue;
        const size_t c = (size_t(p) * g.ny + m) * g.nx + n;
        const int slot = atomicAdd(cursor + c, 1);
        items[offsets[c] + slot] = s;
      }
}

// Heapsort of one cell's list (ascending sphere index), one thread per cell.
__global__ void cells_sort_kernel(const int* __restrict__ offsets, const int* __restrict__ counts, int ncell,
                                  int* __restrict__ items) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int* a = items + offsets[c];
  const int n = counts[c];
  auto sift = [&](int root, int end) {
    while (2 * root + 1 < end) {
      int child = 2 * root + 1;
      if (child + 1 < end && a[child] < a[child + 1]) child++;
      if (a[root] < a[child]) {
        const int t = a[root];
        a[root] = a[child];
        a[child] = t;
        root = child;
      } else {
        return;
      }
    }
  };
  for (int i = n / 2 - 1; i >= 0; --i) sift(i, n);
  for (int end = n - 1; end > 0; --end) {
    const int t = a[0];
    a[0] = a[end];
    a[end] = t;
    sift(0, end);
  }
}

// Orderable 64-bit key of a double (ascending keys = ascending values).
__device__ __forceinline__ unsigned long long okey(double v) {
  const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(v));
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

__device__ __forceinline__ double in_segment(const double* __restrict__ sph, int S, int s, const CellGeom& g, int n,
                                             int m, int p) {
  const double x = sph[s], y = sph[S + s], z = sph[2 * S + s], r = sph[3 * S + s];
  const double dLx = g.Lx / g.nx, dLy = g.Ly / g.ny, dLz = g.Lz / g.nz;
  double v = fmax(seg_lo(double(n), dLx, r, x, g.Lx), seg_hi(double(n), dLx, r, x, g.Lx));
  v = fmax(v, seg_lo(double(m), dLy, r, y, g.Ly));
  v = fmax(v, seg_hi(double(m), dLy, r, y, g.Ly));
  v = fmax(v, seg_lo(double(p), dLz, r, z, g.Lz));
  v = fmax(v, seg_hi(double(p), dLz, r, z, g.Lz));
  return v;
}

// Block-wide exclusive scan of one int per thread (blockDim.x == 256).
__device__ __forceinline__ int block_exclusive_scan(int v, int* s_warp, int& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int t = lane < 8 ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < 8) s_warp[lane] = t;
  }
  __syncthreads();
  total = s_warp[7];
  const int before = (wid > 0 ? s_warp[wid - 1] : 0) + x - v;
  __syncthreads();
  return before;
}

// The padded table: one 256-thread CTA per cell.  The K-th smallest
// (in_segment, index) is found by an 8-bit radix select over the orderable
// key, then the selected indices are written in ascending order.
__global__ void __launch_bounds__(256) segments_fill_kernel(const double* __restrict__ sph, int S, CellGeom g, int K,
                                                            int* __restrict__ segments) {
  __shared__ int hist[256];
  __shared__ int s_warp[8];
  __shared__ unsigned long long s_prefix;
  __shared__ int s_rank;
  const int c = blockIdx.x;
  const int n = c % g.nx, m = (c / g.nx) % g.ny, p = c / (g.nx * g.ny);
  int* out = segments + size_t(c) * K;
  if (K >= S) {  // every sphere is in every list
    for (int i = threadIdx.x; i < S; i += blockDim.x) out[i] = i;
    return;
  }
  if (threadIdx.x == 0) {
    s_prefix = 0ull;
    s_rank = K;  // 1-based rank of the K-th smallest key
  }
  unsigned long long mask = 0ull;
  for (int digit = 7; digit >= 0; --digit) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const unsigned long long prefix = s_prefix;
    for (int i = threadIdx.x; i < S; i += blockDim.x) {
      const unsigned long long k = okey(in_segment(sph, S, i, g, n, m, p));
      if ((k & mask) == prefix) atomicAdd(&hist[(k >> (8 * digit)) & 255ull], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int rank = s_rank, b = 0;
      while (b < 255 && hist[b] < rank) {
        rank -= hist[b];
        ++b;
      }
      s_rank = rank;
      s_prefix = prefix | (static_cast<unsigned long long>(b) << (8 * digit));
    }
    mask |= 255ull << (8 * digit);
    __syncthreads();
  }
  const unsigned long long T = s_prefix;  // key of the K-th smallest
  const int ties_needed = s_rank;         // how many keys equal to T are taken, lowest index first
  int written = 0, ties_seen = 0;
  for (int base = 0; base < S; base += blockDim.x) {
    const int i = base + threadIdx.x;
    int less = 0, tie = 0;
    if (i < S) {
      const unsigned long long k = okey(in_segment(sph, S, i, g, n, m, p));
      less = k < T;
      tie = k == T;
    }
    int tie_total;
    const int tie_before = block_exclusive_scan(tie, s_warp, tie_total);
    const int take = less || (tie && ties_seen + tie_before < ties_needed);
    int take_total;
    const int pos = block_exclusive_scan(take, s_warp, take_total);
    if (take && written + pos < K) out[written + pos] = i;
    written += take_total;
    ties_seen += tie_total;
  }
}

// Fused-walk list entries, three passes: (1) each entry gets its structure id
// and, parked in .x, its sphere index; (2) each cell's entries are sorted by
// (structure id, sphere index) with a heapsort in place; (3) each entry gets
// its sphere record.  Sorted by structure id, a walker labelled L may stop at
// the first entry of a higher structure.
__global__ void gather_ids_kernel(const float* __restrict__ spheres, int S, const int* __restrict__ items, int n,
                                  float4* __restrict__ sph4, int* __restrict__ sid) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int s = items[k];
  sid[k] = int(spheres[4 * S + s]);
  sph4[k].x = __int_as_float(s);
}

__global__ void gather_sort_kernel(const int* __restrict__ start, const int* __restrict__ count, int ncell,
                                   float4* __restrict__ sph4, int* __restrict__ sid) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const int base = start[c], n = count[c];
  auto key = [&](int i) {
    return (static_cast<unsigned long long>(static_cast<unsigned>(sid[base + i])) << 32) |
           static_cast<unsigned>(__float_as_int(sph4[base + i].x));
  };
  auto swap = [&](int i, int j) {
    const int t = sid[base + i];
    sid[base + i] = sid[base + j];
    sid[base + j] = t;
    const float u = sph4[base + i].x;
    sph4[base + i].x = sph4[base + j].x;
    sph4[base + j].x = u;
  };
  auto sift = [&](int root, int end) {
    while (2 * root + 1 < end) {
      int child = 2 * root + 1;
      if (child + 1 < end && key(child) < key(child + 1)) child++;
      if (key(root) < key(child)) {
        swap(root, child);
        root = child;
      } else {
        return;
      }
    }
  };
  for (int i = n / 2 - 1; i >= 0; --i) sift(i, n);
  for (int end = n - 1; end > 0; --end) {
    swap(0, end);
    sift(0, end);
  }
}

__global__ void gather_records_kernel(const float* __restrict__ spheres, int S, int n, float4* __restrict__ sph4) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int s = __float_as_int(sph4[k].x);
  sph4[k] = make_float4(spheres[s], spheres[S + s], spheres[2 * S + s], spheres[3 * S + s]);
}

// Index lists: each entry becomes its sphere's record index, then each
// cell's entries are sorted ascending (a heapsort per cell; one thread per
// cell).  Sphere order within the reference layout is usually already by
// structure, so the sort mostly finds its input in order.
template <typename T>
__global__ void index_fill_kernel(const int* __restrict__ items, int n, const int* __restrict__ perm,
                                  T* __restrict__ idx) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int s = items[k];
  idx[k] = T(perm ? perm[s] : s);
}

template <typename T>
__global__ void index_sort_kernel(const int* __restrict__ start, const int* __restrict__ count, int ncell,
                                  T* __restrict__ idx) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  T* a = idx + start[c];
  const int n = count[c];
  bool sorted = true;
  for (int i = 1; i < n && sorted; ++i) sorted = a[i - 1] <= a[i];
  if (sorted) return;
  auto sift = [&](int root, int end) {
    while (2 * root + 1 < end) {
      int child = 2 * root + 1;
      if (child + 1 < end && a[child] < a[child + 1]) child++;
      if (a[root] < a[child]) {
        const T t = a[root];
        a[root] = a[child];
        a[child] = t;
        root = child;
      } else {
        return;
      }
    }
  };
  for (int i = n / 2 - 1; i >= 0; --i) sift(i, n);
  for (int end = n - 1; end > 0; --end) {
    const T t = a[0];
    a[0] = a[end];
    a[end] = t;
    sift(0, end);
  }
}

// Exclusive scan of in[lo, hi) into out[lo, hi) by one CTA (1024 threads, 8
// items per thread per pass), starting from carry; returns the range's total
// (in every thread).
__device__ __forceinline__ int block_scan_range(const int* __restrict__ in, int* __restrict__ out, int lo, int hi,
                                                int carry) {
  constexpr int kItems = 8;
  __shared__ int s_warp[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int base = lo; base < hi; base += 1024 * kItems) {
    int v[kItems];
    int sum = 0;
    const int first = base + threadIdx.x * kItems;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      v[j] = (first + j < hi) ? in[first + j] : 0;
      sum += v[j];
    }
    int x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int t = s_warp[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += y;
      }
      s_warp[lane] = t;
    }
    __syncthreads();
    int run = carry + (wid > 0 ? s_warp[wid - 1] : 0) + x - sum;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      if (first + j < hi) out[first + j] = run;
      run += v[j];
    }
    carry += s_warp[31];
    __syncthreads();
  }
  return carry;
}

// Single-CTA exclusive scan of n ints.
__global__ void __launch_bounds__(1024) scan_kernel(const int* __restrict__ in, int* __restrict__ out, int n,
                                                    int* __restrict__ total) {
  const int t = block_scan_range(in, out, 0, n, 0);
  if (threadIdx.x == 0 && total) *total = t;
}

// Multi-CTA form for long arrays: each CTA sums one tile, one CTA scans the
// tile sums, each CTA then scans its tile from its offset.
__global__ void __launch_bounds__(1024) tile_sum_kernel(const int* __restrict__ in, int n, int* __restrict__ sums) {
  __shared__ int s_red[32];
  const int lo = blockIdx.x * kScanTile, hi = min(n, lo + kScanTile);
  int v = 0;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) v += in[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = s_red[threadIdx.x];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) sums[blockIdx.x] = v;
  }
}

__global__ void __launch_bounds__(1024) tile_scan_kernel(const int* __restrict__ in, int* __restrict__ out, int n,
                                                         const int* __restrict__ offsets) {
  const int lo = blockIdx.x * kScanTile, hi = min(n, lo + kScanTile);
  block_scan_range(in, out, lo, hi, offsets[blockIdx.x]);
}

int scan_tiles(int n) { return (n + kScanTile - 1) / kScanTile; }

int exclusive_scan(const int* in, int* out, int n, int* tile_sums, int* tile_offsets, cudaStream_t st) {
  if (n <= kScanSingle || !tile_sums || !tile_offsets) {
    scan_kernel<<<1, 1024, 0, st>>>(in, out, n, nullptr);
    return check_launch("scan_kernel");
  }
  const int tiles = scan_tiles(n);
  tile_sum_kernel<<<tiles, 1024, 0, st>>>(in, n, tile_sums);
  int rc = check_launch("tile_sum_kernel");
  if (rc) return rc;
  scan_kernel<<<1, 1024, 0, st>>>(tile_sums, tile_offsets, tiles, nullptr);
  rc = check_launch("scan_kernel");
  if (rc) return rc;
  tile_scan_kernel<<<tiles, 1024, 0, st>>>(in, out, n, tile_offsets);
  return check_launch("tile_scan_kernel");
}

}  // namespace nz

using namespace nz;

extern "C" int nz_cells_count(const double* spheres64, int S, double Lx, double Ly, double Lz, int nx, int ny, int nz_,
                              double jump_tol, int* counts, void* stream) {
  if (S < 0 || nx <= 0 || ny <= 0 || nz_ <= 0 || !counts || (S > 0 && !spheres64))
    return set_error(NZ_ERR_ARG, "nz_cells_count: bad arguments (S=%d grid=%dx%dx%d)", S, nx, ny, nz_);
  const size_t ncell = size_t(nx) * ny * nz_;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(counts, 0, ncell * sizeof(int), st) != cudaSuccess) return check_launch("nz_cells_count memset");
  if (S == 0) return NZ_OK;
  CellGeom g{Lx, Ly, Lz, nx, ny, nz_, jump_tol};
  cells_count_kernel<<<(S + 255) / 256, 256, 0, st>>>(spheres64, S, g, counts);
  return check_launch("cells_count_kernel");
}

extern "C" int nz_cells_count_round(const double* spheres64, int S, double Lx, double Ly, double Lz, int nx, int ny,
                                    int nz_, double margin, int* counts, void* stream) {
  if (S < 0 || nx <= 0 || ny <= 0 || nz_ <= 0 || !counts || (S > 0 && !spheres64) || !(margin >= 0.0))
    return set_error(NZ_ERR_ARG, "nz_cells_count_round: bad arguments (S=%d grid=%dx%dx%d)", S, nx, ny, nz_);
  const size_t ncell = size_t(nx) * ny * nz_;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(counts, 0, ncell * sizeof(int), st) != cudaSuccess)
    return check_launch("nz_cells_count_round memset");
  if (S == 0) return NZ_OK;
  CellGeom g{Lx, Ly, Lz, nx, ny, nz_, margin};
  cells_count_round_kernel<<<(S + 255) / 256, 256, 0, st>>>(spheres64, S, g, counts);
  return check_launch("cells_count_round_kernel");
}

extern "C" int nz_cells_fill_round(const double* spheres64, int S, double Lx, double Ly, double Lz, int nx, int ny,
                                   int nz_, double margin, const int* offsets, const int* counts, int* cursor,
                                   int* items, void* stream) {
  if (S < 0 || nx <= 0 || ny <= 0 || nz_ <= 0 || !offsets || !counts || !cursor || (S > 0 && !spheres64) ||
      !(margin >= 0.0))
    return set_error(NZ_ERR_ARG, "nz_cells_fill_round: bad arguments (S=%d grid=%dx%dx%d)", S, nx, ny, nz_);
  const size_t ncell = size_t(nx) * ny * nz_;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(cursor, 0, ncell * sizeof(int), st) != cudaSuccess)
    return check_launch("nz_cells_fill_round memset");
  if (S == 0) return NZ_OK;
  CellGeom g{Lx, Ly, Lz, nx, ny, nz_, margin};
  cells_fill_round_kernel<<<(S + 255) / 256, 256, 0, st>>>(spheres64, S, g, offsets, cursor, items);
  int rc = check_launch("cells_fill_round_kernel");
  if (rc != NZ_OK) return rc;
  cells_sort_kernel<<<unsigned((ncell + 127) / 128), 128, 0, st>>>(offsets, counts, int(ncell), items);
  return check_launch("cells_sort_kernel");
}

extern "C" int nz_exclusive_scan_i32(const int* in, int* out, int n, int* total, void* stream) {
  if (n < 0 || n > (1 << 26) || (n > 0 && (!in || !out)))
    return set_error(NZ_ERR_ARG, "nz_exclusive_scan_i32: bad arguments (n=%d)", n);
  scan_kernel<<<1, 1024, 0, static_cast<cudaStream_t>(stream)>>>(in, out, n, total);
  return check_launch("scan_kernel");
}

extern "C" int nz_cells_fill(const double* spheres64, int S, double Lx, double Ly, double Lz, int nx, int ny, int nz_,
                             double jump_tol, const int* offsets, const int* counts, int* cursor, int* items,
                             void* stream) {
  if (S < 0 || nx <= 0 || ny <= 0 || nz_ <= 0 || !offsets || !counts || !cursor || (S > 0 && !spheres64))
    return set_error(NZ_ERR_ARG, "nz_cells_fill: bad arguments (S=%d grid=%dx%dx%d)", S, nx, ny, nz_);
  const size_t ncell = size_t(nx) * ny * nz_;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(cursor, 0, ncell * sizeof(int), st) != cudaSuccess) return check_launch("nz_cells_fill memset");
  if (S == 0) return NZ_OK;
  CellGeom g{Lx, Ly, Lz, nx, ny, nz_, jump_tol};
  cells_fill_kernel<<<(S + 255) / 256, 256, 0, st>>>(spheres64, S, g, offsets, cursor, items);
  int rc = check_launch("cells_fill_kernel");
  if (rc != NZ_OK) return rc;
  cells_sort_kernel<<<unsigned((ncell + 127) / 128), 128, 0, st>>>(offsets, counts, int(ncell), items);
  return check_launch("cells_sort_kernel");
}

extern "C" int nz_segments_fill(const double* spheres64, int S, double Lx, double Ly, double Lz, int nx, int ny,
                                int nz_, int K, int* segments, void* stream) {
  if (S <= 0 || nx <= 0 || ny <= 0 || nz_ <= 0 || K <= 0 || K > S || !spheres64 || !segments)
    return set_error(NZ_ERR_ARG, "nz_segments_fill: bad arguments (S=%d K=%d)", S, K);
  const size_t ncell = size_t(nx) * ny * nz_;
  if (ncell > 0x7fffffffu) return set_error(NZ_ERR_ARG, "nz_segments_fill: too many cells");
  CellGeom g{Lx, Ly, Lz, nx, ny, nz_, 0.0};
  segments_fill_kernel<<<unsigned(ncell), 256, 0, static_cast<cudaStream_t>(stream)>>>(spheres64, S, g, K, segments);
  return check_launch("segments_fill_kernel");
}

extern "C" int nz_cells_gather(const float* spheres, int S, const int* items, int n_items, const int* cell_start,
                               const int* cell_count, int ncell, float* sph4, int* sid, void* stream) {
  if (S < 0 || n_items < 0 || ncell < 0 ||
      (n_items > 0 && (!spheres || !items || !sph4 || !sid || !cell_start || !cell_count)))
    return set_error(NZ_ERR_ARG, "nz_cells_gather: bad arguments");
  if (reinterpret_cast<uintptr_t>(sph4) % 16 != 0) return set_error(NZ_ERR_ARG, "nz_cells_gather: sph4 not 16-byte aligned");
  if (n_items == 0) return NZ_OK;
  if (ncell == 0) return set_error(NZ_ERR_ARG, "nz_cells_gather: %d items but no cells", n_items);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  float4* s4 = reinterpret_cast<float4*>(sph4);
  gather_ids_kernel<<<(n_items + 255) / 256, 256, 0, st>>>(spheres, S, items, n_items, s4, sid);
  int rc = check_launch("gather_ids_kernel");
  if (rc) return rc;
  gather_sort_kernel<<<(ncell + 127) / 128, 128, 0, st>>>(cell_start, cell_count, ncell, s4, sid);
  rc = check_launch("gather_sort_kernel");
  if (rc) return rc;
  gather_records_kernel<<<(n_items + 255) / 256, 256, 0, st>>>(spheres, S, n_items, s4);
  return check_launch("gather_records_kernel");
}

extern "C" int nz_cells_index(const int* items, int n_items, const int* perm, int S, const int* cell_start,
                              const int* cell_count, int ncell, void* idx, int idx_bytes, void* stream) {
  if (n_items < 0 || ncell < 0 || S < 0 || (idx_bytes != 2 && idx_bytes != 4) ||
      (n_items > 0 && (!items || !idx || !cell_start || !cell_count || ncell == 0)))
    return set_error(NZ_ERR_ARG, "nz_cells_index: bad arguments (items=%d cells=%d idx_bytes=%d)", n_items, ncell,
                     idx_bytes);
  if (idx_bytes == 2 && S > 65536)
    return set_error(NZ_ERR_ARG, "nz_cells_index: %d spheres do not fit 16-bit indices", S);
  if (n_items == 0) return NZ_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (idx_bytes == 2) {
    auto* p = static_cast<uint16_t*>(idx);
    index_fill_kernel<uint16_t><<<(n_items + 255) / 256, 256, 0, st>>>(items, n_items, perm, p);
    int rc = check_launch("index_fill_kernel");
    if (rc) return rc;
    index_sort_kernel<uint16_t><<<(ncell + 127) / 128, 128, 0, st>>>(cell_start, cell_count, ncell, p);
  } else {
    auto* p = static_cast<int*>(idx);
    index_fill_kernel<int><<<(n_items + 255) / 256, 256, 0, st>>>(items, n_items, perm, p);
    int rc = check_launch("index_fill_kernel");
    if (rc) return rc;
    index_sort_kernel<int><<<(ncell + 127) / 128, 128, 0, st>>>(cell_start, cell_count, ncell, p);
  }
  return check_launch("index_sort_kernel");
}
