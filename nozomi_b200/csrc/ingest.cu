// Substrate ingestion on the device: the simulation driver's reading of a
// substrate matrix (simulation_toolkit/utils/common_utils.py:41-55,
// split_matrix_to_list; utils/adjust_geometry.py:3-36, createBoundaryZ and
// create_pad), for substrates of 1e5-1e6 spheres.
//
// Input: the pickle's matrix, rows (x, y, z, r, fibre id) in float64, row
// major.  A fibre ends at a row whose z equals L/2 exactly; rows after the
// last such row belong to no fibre.  A fibre whose first sphere's (x, y)
// equals the last sphere's (x, y) of some fibre (the last such fibre in file
// order, as a dictionary built in order keeps it) continues through the z
// face: it gets that partner's last pad/2 rows shifted by -Lz before its own
// rows and the partner's first pad/2 rows shifted by +Lz after them, and the
// fibre id column of the result is its own ids (last pad/2, all, first
// pad/2), every fibre's ids truncated to integers.
//
// Three stages, with two host reads of a size in between:
//   nz_ingest_split  split rows and fibre count
//   nz_ingest_plan   partner of every fibre and output offsets
//   nz_ingest_write  the padded fibres (rows, as the reference returns them)
//                    and the walk's [5, S] sphere layout (x, y, z, r,
//                    structure = fibre index)
#include <cstdint>
#include "kernels.cuh"

namespace nz {

__global__ void split_flags_kernel(const double* __restrict__ rows, int M, double half, int* __restrict__ flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < M) flags[i] = rows[size_t(i) * 5 + 2] == half ? 1 : 0;
}

__global__ void split_ends_kernel(const int* __restrict__ flags, const int* __restrict__ pos, int M,
                                  int* __restrict__ ends, int* __restrict__ n_fibres) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  if (flags[i]) ends[pos[i]] = i;
  if (i == M - 1) *n_fibres = pos[i] + flags[i];
}

// Partner of every fibre: the last fibre j whose last row's (x, y) equals
// fibre k's first row's (x, y), or -1.  End keys are staged in shared memory
// a tile at a time.  Also each fibre's output length, and a count of padded
// fibres (or partners) shorter than pad / 2 rows, which the reference's
// create_pad cannot handle.
constexpr int kPartnerTile = 256;

__global__ void __launch_bounds__(kPartnerTile) partner_kernel(const double* __restrict__ rows,
                                                               const int* __restrict__ ends, int F, int pad,
                                                               int* __restrict__ partner, int* __restrict__ out_len,
                                                               int* __restrict__ n_bad) {
  __shared__ double s_x[kPartnerTile], s_y[kPartnerTile];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  double x = 0.0, y = 0.0;
  if (k < F) {
    const int s = k ? ends[k - 1] + 1 : 0;
    x = rows[size_t(s) * 5];
    y = rows[size_t(s) * 5 + 1];
  }
  int best = -1;
  for (int base = 0; base < F; base += kPartnerTile) {
    const int j = base + threadIdx.x;
    if (j < F) {
      const int e = ends[j];
      s_x[threadIdx.x] = rows[size_t(e) * 5];
      s_y[threadIdx.x] = rows[size_t(e) * 5 + 1];
    }
    __syncthreads();
    const int m = min(kPartnerTile, F - base);
    if (k < F)
      for (int t = 0; t < m; ++t)
        if (s_x[t] == x && s_y[t] == y) best = base + t;
    __syncthreads();
  }
  if (k >= F) return;
  partner[k] = best;
  const int n = ends[k] - (k ? ends[k - 1] + 1 : 0) + 1;
  out_len[k] = n + (best >= 0 ? pad : 0);
  if (best >= 0) {
    const int nj = ends[best] - (best ? ends[best - 1] + 1 : 0) + 1;
    if (n < pad / 2 || nj < pad / 2) atomicAdd(n_bad, 1);
  }
}

__global__ void offsets_total_kernel(const int* __restrict__ len, const int* __restrict__ off, int F,
                                     int* __restrict__ total) {
  *total = F ? off[F - 1] + len[F - 1] : 0;
}

__global__ void ingest_write_kernel(const double* __restrict__ rows, const int* __restrict__ ends, int F,
                                    const int* __restrict__ partner, const int* __restrict__ out_offset, int S,
                                    double Lz, int pad, double* __restrict__ out_rows, double* __restrict__ soa) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= S) return;
  int lo = 0, hi = F - 1;  // the fibre whose output range holds o
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (out_offset[mid] <= o) lo = mid;
    else hi = mid - 1;
  }
  const int k = lo;
  const int p = o - out_offset[k];
  const int s = k ? ends[k - 1] + 1 : 0;
  const int n = ends[k] - s + 1;
  const int j = partner[k];
  const int h = pad / 2;
  int src, own;  // row of x, y, z, r; row of the fibre id
  double dz = 0.0;
  if (j < 0) {
    src = own = s + p;
  } else {
    const int sj = j ? ends[j - 1] + 1 : 0;
    const int nj = ends[j] - sj + 1;
    if (p < h) {
      src = sj + nj - h + p;
      own = s + n - h + p;
      dz = -Lz;
    } else if (p < h + n) {
      src = own = s + p - h;
    } else {
      src = sj + (p - h - n);
      own = s + (p - h - n);
      dz = Lz;
    }
  }
  const double* r = rows + size_t(src) * 5;
  const double z = dz == 0.0 ? r[2] : (dz < 0.0 ? r[2] - Lz : r[2] + Lz);
  const double fid = trunc(rows[size_t(own) * 5 + 4]);
  double* w = out_rows + size_t(o) * 5;
  w[0] = r[0];
  w[1] = r[1];
  w[2] = z;
  w[3] = r[3];
  w[4] = fid;
  if (soa) {
    soa[o] = r[0];
    soa[size_t(S) + o] = r[1];
    soa[2 * size_t(S) + o] = z;
    soa[3 * size_t(S) + o] = r[3];
    soa[4 * size_t(S) + o] = double(k);
  }
}

static inline size_t align256i(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace nz

using namespace nz;

extern "C" size_t nz_ingest_scratch_bytes(int M) {
  if (M < 0) return 0;
  return 2 * align256i(size_t(M) * sizeof(int)) + 2 * align256i(size_t(scan_tiles(M)) * sizeof(int));
}

extern "C" int nz_ingest_split(const double* rows, int M, double L, int* ends, int* n_fibres, void* scratch,
                               size_t scratch_bytes, void* stream) {
  if (M < 0 || !n_fibres || (M > 0 && (!rows || !ends)))
    return set_error(NZ_ERR_ARG, "nz_ingest_split: bad arguments (M=%d)", M);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (M == 0) {
    if (cudaMemsetAsync(n_fibres, 0, sizeof(int), st) != cudaSuccess) return check_launch("nz_ingest_split memset");
    return NZ_OK;
  }
  const size_t need = nz_ingest_scratch_bytes(M);
  if (!scratch || scratch_bytes < need)
    return set_error(NZ_ERR_CAPACITY, "nz_ingest_split: scratch %zu bytes < %zu", scratch_bytes, need);
  char* p = static_cast<char*>(scratch);
  const size_t nm = align256i(size_t(M) * sizeof(int));
  int* flags = reinterpret_cast<int*>(p);
  int* pos = reinterpret_cast<int*>(p + nm);
  int* tile_sums = reinterpret_cast<int*>(p + 2 * nm);
  int* tile_offsets = reinterpret_cast<int*>(p + 2 * nm + align256i(size_t(scan_tiles(M)) * sizeof(int)));
  split_flags_kernel<<<(M + 255) / 256, 256, 0, st>>>(rows, M, L / 2, flags);
  int rc = check_launch("split_flags_kernel");
  if (rc) return rc;
  rc = exclusive_scan(flags, pos, M, tile_sums, tile_offsets, st);
  if (rc) return rc;
  split_ends_kernel<<<(M + 255) / 256, 256, 0, st>>>(flags, pos, M, ends, n_fibres);
  return check_launch("split_ends_kernel");
}

extern "C" int nz_ingest_plan(const double* rows, const int* ends, int F, int pad, int* partner, int* out_offset,
                              int* n_out, int* n_bad, void* scratch, size_t scratch_bytes, void* stream) {
  if (F < 0 || pad < 0 || pad % 2 || !n_out || !n_bad || (F > 0 && (!rows || !ends || !partner || !out_offset)))
    return set_error(NZ_ERR_ARG, "nz_ingest_plan: bad arguments (F=%d pad=%d)", F, pad);
  const size_t need = nz_ingest_scratch_bytes(F);
  if (F > 0 && (!scratch || scratch_bytes < need))
    return set_error(NZ_ERR_CAPACITY, "nz_ingest_plan: scratch %zu bytes < %zu", scratch_bytes, need);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(n_bad, 0, sizeof(int), st) != cudaSuccess) return check_launch("nz_ingest_plan memset");
  if (F == 0) {
    if (cudaMemsetAsync(n_out, 0, sizeof(int), st) != cudaSuccess) return check_launch("nz_ingest_plan memset");
    return NZ_OK;
  }
  char* p = static_cast<char*>(scratch);
  const size_t nf = align256i(size_t(F) * sizeof(int));
  int* len = reinterpret_cast<int*>(p);
  int* tile_sums = reinterpret_cast<int*>(p + 2 * nf);
  int* tile_offsets = reinterpret_cast<int*>(p + 2 * nf + align256i(size_t(scan_tiles(F)) * sizeof(int)));
  partner_kernel<<<(F + kPartnerTile - 1) / kPartnerTile, kPartnerTile, 0, st>>>(rows, ends, F, pad, partner, len,
                                                                                 n_bad);
  int rc = check_launch("partner_kernel");
  if (rc) return rc;
  rc = exclusive_scan(len, out_offset, F, tile_sums, tile_offsets, st);
  if (rc) return rc;
  offsets_total_kernel<<<1, 1, 0, st>>>(len, out_offset, F, n_out);
  return check_launch("offsets_total_kernel");
}

extern "C" int nz_ingest_write(const double* rows, const int* ends, int F, const int* partner, const int* out_offset,
                               int S, double Lz, int pad, double* out_rows, double* spheres, void* stream) {
  if (F < 0 || S < 0 || pad < 0 || pad % 2 ||
      (S > 0 && (F == 0 || !rows || !ends || !partner || !out_offset || !out_rows)))
    return set_error(NZ_ERR_ARG, "nz_ingest_write: bad arguments (F=%d S=%d pad=%d)", F, S, pad);
  if (S == 0) return NZ_OK;
  ingest_write_kernel<<<(S + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      rows, ends, F, partner, out_offset, S, Lz, pad, out_rows, spheres);
  return check_launch("ingest_write_kernel");
}
