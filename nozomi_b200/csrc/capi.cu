// C entry points of libnozomi_b200.so that are not next to their kernels:
// status handling, the plain step, packing and the fused / batched walks.
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include "kernels.cuh"

namespace nz {

static thread_local char g_last_error[512] = "";

int set_error(int status, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof g_last_error, fmt, ap);
  va_end(ap);
  return status;
}

int check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(NZ_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return NZ_OK;
}

static Grid to_grid(const nz_grid& g) {
  return Grid{g.Lx, g.Ly, g.Lz, g.dLx, g.dLy, g.dLz, float(g.nx), float(g.ny), float(g.nz)};
}

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace nz

using namespace nz;

extern "C" int nz_version(void) { return NZ_VERSION; }

extern "C" const char* nz_status_string(int status) {
  switch (status) {
    case NZ_OK: return "ok";
    case NZ_ERR_ARG: return "invalid argument";
    case NZ_ERR_CUDA: return "CUDA error";
    case NZ_ERR_CAPACITY: return "buffer too small";
    case NZ_ERR_UNSEEDED: return "walkers left unseeded";
    default: return "unknown status";
  }
}

extern "C" const char* nz_last_error(void) { return g_last_error; }

extern "C" int nz_device_sm_count(int* sms) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return check_launch("cudaGetDevice");
  if (cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return check_launch("cudaDeviceGetAttribute");
  return NZ_OK;
}

static int check_substrate(const nz_substrate* s, const char* who) {
  if (!s) return set_error(NZ_ERR_ARG, "%s: null substrate", who);
  if (s->grid.nx <= 0 || s->grid.ny <= 0 || s->grid.nz <= 0 || s->nstructures < 0 || s->S < 0 || !s->cell_start ||
      !s->cell_count || !s->D)
    return set_error(NZ_ERR_ARG, "%s: incomplete substrate", who);
  return NZ_OK;
}

extern "C" int nz_walk_step(const nz_substrate* sub, const nz_walkers* wk, int mode, float dt, float G, float Garea,
                            int step, const nz_draws* draws, void* stream) {
  int rc = check_substrate(sub, "nz_walk_step");
  if (rc) return rc;
  if (!wk || !draws || wk->N < 0 || !sub->cell_items || (sub->S > 0 && !sub->spheres))
    return set_error(NZ_ERR_ARG, "nz_walk_step: bad walkers or draws");
  if (mode & ~(NZ_MODE_SIG | NZ_MODE_PHASE | NZ_MODE_PHI)) return set_error(NZ_ERR_ARG, "nz_walk_step: mode %d", mode);
  if ((mode & NZ_MODE_PHASE) && wk->ndir <= 0) return set_error(NZ_ERR_ARG, "nz_walk_step: phase mode needs ndir > 0");
  if ((mode & NZ_MODE_SIG) && !sub->T2) return set_error(NZ_ERR_ARG, "nz_walk_step: sig mode needs T2");
  if (wk->N == 0) return NZ_OK;  // empty walker arrays may be null
  if (!wk->spins || !wk->spins0) return set_error(NZ_ERR_ARG, "nz_walk_step: null spins or spins0");
  if ((mode & NZ_MODE_PHASE) && (!wk->phase || !wk->diffdir))
    return set_error(NZ_ERR_ARG, "nz_walk_step: phase mode needs phase and diffdir");
  if ((mode & NZ_MODE_SIG) && !wk->sig) return set_error(NZ_ERR_ARG, "nz_walk_step: sig mode needs sig");
  if ((mode & NZ_MODE_PHI) && !wk->phi) return set_error(NZ_ERR_ARG, "nz_walk_step: phi mode needs phi");
  PlainArgs a;
  a.g = to_grid(sub->grid);
  a.nstructures = sub->nstructures;
  a.S = sub->S;
  a.N = wk->N;
  a.ncell = sub->grid.nx * sub->grid.ny * sub->grid.nz;
  a.n_items = sub->n_items;
  a.spheres = sub->spheres;
  a.cell_start = sub->cell_start;
  a.cell_count = sub->cell_count;
  a.cell_items = sub->cell_items;
  a.D = sub->D;
  a.T2 = sub->T2;
  a.spins = wk->spins;
  a.spins0 = wk->spins0;
  a.phase = wk->phase;
  a.diffdir = wk->diffdir;
  a.ndir = wk->ndir;
  a.sig = wk->sig;
  a.phi = wk->phi;
  a.dt = dt;
  a.G = G;
  a.Garea = Garea;
  a.step = step;
  a.draws = Draws{draws->table, draws->nsteps, draws->maxk, draws->key0, draws->key1, draws->stream};
  a.mode = mode;
  a.label = wk->label;
  a.n_iter = wk->n_iter;
  a.n_scatter = wk->n_scatter;
  a.flags = wk->flags;
  walk_plain_kernel<<<(wk->N + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(a);
  return check_launch("walk_plain_kernel");
}

int nz::check_state(const nz_state* st, const char* who) {
  if (!st || st->N < 0) return set_error(NZ_ERR_ARG, "%s: null state or negative N", who);
  if (st->N == 0) return NZ_OK;
  if (!st->pos || !st->org || !st->phi || !st->comp) return set_error(NZ_ERR_ARG, "%s: incomplete state", who);
  if (!aligned16(st->pos) || !aligned16(st->org) || !aligned16(st->phi) || !aligned16(st->comp))
    return set_error(NZ_ERR_ARG, "%s: state arrays must be 16-byte aligned", who);
  return NZ_OK;
}

int nz::check_grid(const nz_grid* g, const char* who) {
  if (!g || g->nx <= 0 || g->ny <= 0 || g->nz <= 0) return set_error(NZ_ERR_ARG, "%s: grid needs nx, ny, nz > 0", who);
  return NZ_OK;
}

extern "C" int nz_state_pack(const nz_walkers* wk, const uint32_t* walker_id, nz_state* st, void* stream) {
  int rc = check_state(st, "nz_state_pack");
  if (rc) return rc;
  if (!wk || wk->N != st->N || (st->N > 0 && (!wk->spins || !wk->spins0)))
    return set_error(NZ_ERR_ARG, "nz_state_pack: bad walkers");
  if (st->N == 0) return NZ_OK;
  pack_kernel<<<(st->N + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(*wk, walker_id, *st);
  return check_launch("pack_kernel");
}

extern "C" int nz_state_unpack(const nz_state* st, const nz_walkers* wk, void* stream) {
  int rc = check_state(st, "nz_state_unpack");
  if (rc) return rc;
  if (!wk || wk->N != st->N || (st->N > 0 && (!wk->spins || !wk->spins0)))
    return set_error(NZ_ERR_ARG, "nz_state_unpack: bad walkers");
  if (st->N == 0) return NZ_OK;
  unpack_kernel<<<(st->N + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(*st, *wk, 0, nullptr);
  return check_launch("unpack_kernel");
}

extern "C" int nz_state_unpack_by_id(const nz_state* st, const nz_walkers* wk, int* n_bad, void* stream) {
  int rc = check_state(st, "nz_state_unpack_by_id");
  if (rc) return rc;
  if (!wk || wk->N != st->N || (st->N > 0 && (!wk->spins || !wk->spins0)))
    return set_error(NZ_ERR_ARG, "nz_state_unpack_by_id: bad walkers");
  if (st->N == 0) return NZ_OK;
  unpack_kernel<<<(st->N + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(*st, *wk, 1, n_bad);
  return check_launch("unpack_kernel");
}

static int check_fused_sub(const nz_substrate* sub, const char* who) {
  int rc = check_substrate(sub, who);
  if (rc) return rc;
  if (sub->idx_bytes != 0) {
    if (sub->idx_bytes != 2 && sub->idx_bytes != 4)
      return set_error(NZ_ERR_ARG, "%s: idx_bytes %d is not 0, 2 or 4", who, sub->idx_bytes);
    if (sub->idx_bytes == 2 && sub->S > 65536)
      return set_error(NZ_ERR_ARG, "%s: %d spheres do not fit 16-bit indices", who, sub->S);
    if (!sub->cell_idx || !sub->rec4 || !sub->rec_sid || !sub->sid_start)
      return set_error(NZ_ERR_ARG, "%s: index lists need cell_idx, rec4, rec_sid and sid_start", who);
    if (!aligned16(sub->rec4)) return set_error(NZ_ERR_ARG, "%s: rec4 must be 16-byte aligned", who);
    if (sub->near_idx && (!sub->near_start || !sub->near_count || !(sub->near_margin > 0.0f)))
      return set_error(NZ_ERR_ARG, "%s: incomplete near lists", who);
    return NZ_OK;
  }
  if (!sub->cell_sph4 || !sub->cell_sid) return set_error(NZ_ERR_ARG, "%s: substrate lacks cell_sph4/cell_sid", who);
  if (!aligned16(sub->cell_sph4)) return set_error(NZ_ERR_ARG, "%s: cell_sph4 must be 16-byte aligned", who);
  if (sub->near_sph4) {
    if (!sub->near_start || !sub->near_count || !sub->near_sid || !(sub->near_margin > 0.0f))
      return set_error(NZ_ERR_ARG, "%s: incomplete near lists", who);
    if (!aligned16(sub->near_sph4)) return set_error(NZ_ERR_ARG, "%s: near_sph4 must be 16-byte aligned", who);
  }
  return NZ_OK;
}

// List kind of an nz_walk_batch launch from its mode bits.
static int batch_list_kind(int mode) {
  if ((mode & NZ_LIST_IDX16) && (mode & NZ_LIST_IDX32)) return -1;
  return (mode & NZ_LIST_IDX16) ? 2 : (mode & NZ_LIST_IDX32) ? 4 : 0;
}

extern "C" int nz_walk_fused(const nz_substrate* sub, const nz_state* st, int mode, float dt, const float* G,
                             const float* Garea, int step0, int step1, const nz_draws* draws, double* moments,
                             void* stream) {
  int rc = check_fused_sub(sub, "nz_walk_fused");
  if (rc) return rc;
  rc = check_state(st, "nz_walk_fused");
  if (rc) return rc;
  if (!draws || draws->table) return set_error(NZ_ERR_ARG, "nz_walk_fused: Philox draws only (table must be NULL)");
  if ((mode & NZ_MODE_PHI) && (!G || !Garea)) return set_error(NZ_ERR_ARG, "nz_walk_fused: phi mode needs G, Garea");
  if ((mode & NZ_MODE_SIG) && !sub->T2) return set_error(NZ_ERR_ARG, "nz_walk_fused: sig mode needs T2");
  if (mode & NZ_MODE_MOMENTS) {
    if (!moments) return set_error(NZ_ERR_ARG, "nz_walk_fused: moments mode needs moments");
    if (step1 - step0 > kMomentSteps)
      return set_error(NZ_ERR_ARG, "nz_walk_fused: moments mode runs at most %d steps per launch", kMomentSteps);
  }
  if (step0 < 0 || step1 < step0) return set_error(NZ_ERR_ARG, "nz_walk_fused: bad step range");
  if (st->N == 0 || step1 == step0) return NZ_OK;
  const JobDev j = make_job(*sub, G, Garea, step1, dt, *draws, mode, *st, moments);
  const int n_items = (st->N + kFusedThreads - 1) / kFusedThreads;
  return launch_fused(mode, sub->idx_bytes, j, nullptr, nullptr, n_items, step0, step1, nullptr, n_items,
                      kFusedThreads, static_cast<cudaStream_t>(stream));
}

extern "C" size_t nz_walk_fused_moments_scratch_bytes(int N, int nsteps) {
  return (N > 0 && nsteps > 0) ? size_t(N) * 3 * size_t(nsteps) * sizeof(float) : 0;
}

extern "C" int nz_walk_fused_moments(const nz_substrate* sub, const nz_state* st, int mode, float dt, const float* G,
                                     const float* Garea, int step0, int step1, const nz_draws* draws, float* scratch,
                                     size_t scratch_bytes, double* moments, void* stream) {
  int rc = check_fused_sub(sub, "nz_walk_fused_moments");
  if (rc) return rc;
  rc = check_state(st, "nz_walk_fused_moments");
  if (rc) return rc;
  if (!draws || draws->table)
    return set_error(NZ_ERR_ARG, "nz_walk_fused_moments: Philox draws only (table must be NULL)");
  if (mode & ~NZ_MODE_SIG) return set_error(NZ_ERR_ARG, "nz_walk_fused_moments: mode is 0 or NZ_MODE_SIG");
  if ((mode & NZ_MODE_SIG) && !sub->T2) return set_error(NZ_ERR_ARG, "nz_walk_fused_moments: sig mode needs T2");
  if (step0 < 0 || step1 < step0 || !moments) return set_error(NZ_ERR_ARG, "nz_walk_fused_moments: bad arguments");
  if (st->N == 0 || step1 == step0) return NZ_OK;
  const size_t need = nz_walk_fused_moments_scratch_bytes(st->N, step1 - step0);
  if (!scratch || scratch_bytes < need || (reinterpret_cast<uintptr_t>(scratch) & 3))
    return set_error(NZ_ERR_ARG, "nz_walk_fused_moments: scratch needs %zu bytes (4-byte aligned), got %zu", need,
                     scratch_bytes);
  if (step1 - step0 > 65535) return set_error(NZ_ERR_ARG, "nz_walk_fused_moments: at most 65535 steps per call");
  const cudaStream_t cs = static_cast<cudaStream_t>(stream);
  JobDev j = make_job(*sub, G, Garea, step1, dt, *draws, mode, *st, nullptr);
  j.disp = scratch;
  const int n_items = (st->N + kFusedThreads - 1) / kFusedThreads;
  rc = launch_fused(mode | kModeDisp, sub->idx_bytes, j, nullptr, nullptr, n_items, step0, step1, nullptr, n_items,
                    kFusedThreads, cs);
  if (rc) return rc;
  const int gx = min(64, (st->N + 255) / 256);
  disp_moments_kernel<<<dim3(gx, step1 - step0), 256, 0, cs>>>(scratch, st->N, moments + size_t(step0) * 6);
  return check_launch("disp_moments_kernel");
}

// nz_walk_batch with stage_records records of shared memory per CTA for
// staging (0: none).  A job is staged when its record array fits and starts on
// a 16-byte boundary (the kernel checks; other jobs read global memory).
static int walk_batch(const char* what, const nz_job* jobs, int n_jobs, const nz_item* items, int n_items, int mode,
                      int step0, int step1, int* queue, int grid, int threads, int stage_records, void* stream) {
  if (!jobs || n_jobs <= 0 || !items || n_items < 0 || step0 < 0 || step1 < step0 || grid < 0)
    return set_error(NZ_ERR_ARG, "%s: bad arguments", what);
  if (threads < 32 || threads > kFusedMaxThreads || threads % 32)
    return set_error(NZ_ERR_ARG, "%s: threads %d not a multiple of 32 in [32, %d]", what, threads, kFusedMaxThreads);
  if (grid > 0 && !queue) return set_error(NZ_ERR_ARG, "%s: a persistent grid needs a queue counter", what);
  if (mode & NZ_MODE_MOMENTS) return set_error(NZ_ERR_ARG, "%s: moments are per-substrate (nz_walk_fused)", what);
  const int lk = batch_list_kind(mode);
  if (lk < 0) return set_error(NZ_ERR_ARG, "%s: both list widths in mode %d", what, mode);
  if (stage_records < 0 || stage_records > kMaxStageRecords)
    return set_error(NZ_ERR_ARG, "%s: stage_records %d outside [0, %d]", what, stage_records, kMaxStageRecords);
  if (stage_records > 0 && lk == 0)
    return set_error(NZ_ERR_ARG, "%s: records are staged for index lists only (no NZ_LIST_IDX bit in mode)", what);
  if (n_items == 0 || step1 == step0) return NZ_OK;
  const JobDev unused{};
  return launch_fused(mode & ~(NZ_LIST_IDX16 | NZ_LIST_IDX32), lk, unused, jobs, items, n_items, step0, step1,
                      grid > 0 ? queue : nullptr, grid > 0 ? grid : n_items, threads,
                      static_cast<cudaStream_t>(stream), stage_records);
}

extern "C" int nz_walk_batch(const nz_job* jobs, int n_jobs, const nz_item* items, int n_items, int mode, int step0,
                             int step1, int* queue, int grid, int threads, void* stream) {
  return walk_batch("nz_walk_batch", jobs, n_jobs, items, n_items, mode, step0, step1, queue, grid, threads, 0,
                    stream);
}

extern "C" int nz_walk_batch_staged(const nz_job* jobs, int n_jobs, const nz_item* items, int n_items, int mode,
                                    int step0, int step1, int* queue, int grid, int threads, int stage_records,
                                    void* stream) {
  return walk_batch("nz_walk_batch_staged", jobs, n_jobs, items, n_items, mode, step0, step1, queue, grid, threads,
                    stage_records, stream);
}

extern "C" int nz_batch_occupancy(int mode, int threads, int* blocks_per_sm) {
  const int lk = batch_list_kind(mode);
  if (!blocks_per_sm || threads < 32 || threads > kFusedMaxThreads || lk < 0)
    return set_error(NZ_ERR_ARG, "nz_batch_occupancy: bad arguments");
  return occupancy_fused(mode & ~(NZ_LIST_IDX16 | NZ_LIST_IDX32), lk, threads, blocks_per_sm);
}

extern "C" int nz_batch_occupancy_staged(int mode, int threads, int stage_records, int* blocks_per_sm) {
  const int lk = batch_list_kind(mode);
  if (!blocks_per_sm || threads < 32 || threads > kFusedMaxThreads || lk <= 0 || stage_records < 0 ||
      stage_records > kMaxStageRecords)
    return set_error(NZ_ERR_ARG, "nz_batch_occupancy_staged: bad arguments");
  return occupancy_fused(mode & ~(NZ_LIST_IDX16 | NZ_LIST_IDX32), lk, threads, blocks_per_sm, stage_records);
}
