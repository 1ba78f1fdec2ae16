/*
 * nozomi_b200 — C ABI of the B200 spin random-walk library (libnozomi_b200.so).
 *
 * Every entry point takes device pointers, sizes and a cudaStream_t (passed as
 * void*, NULL = legacy default stream), enqueues its kernels on that stream and
 * returns a status: NZ_OK or an error code; nz_last_error() gives the message of
 * the calling thread's last failure.  No entry point allocates device memory or
 * synchronises the stream unless its comment says so; scratch buffers are
 * passed in by the caller.
 *
 * Each declaration names the reference interface it replaces (paths relative to
 * the nozomi source tree, simulation_toolkit/simulation_engine/...).  The
 * reference has no C ABI: its boundary is the Python object API of
 * DiffSim3d / DwiSim3d driving pycuda kernels, so the cited lines are those
 * methods and kernels.
 */
#ifndef NOZOMI_B200_H
#define NOZOMI_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NZ_VERSION 1

/* status codes */
#define NZ_OK 0
#define NZ_ERR_ARG 1        /* invalid argument (message in nz_last_error) */
#define NZ_ERR_CUDA 2       /* a CUDA launch or runtime call failed */
#define NZ_ERR_CAPACITY 3   /* a caller-provided buffer is too small */
#define NZ_ERR_UNSEEDED 4   /* seeding left walkers unplaced after its round limit */

/* walk modes (bit set) */
#define NZ_MODE_SIG 1       /* T2 weighting of sig[] (randomWalk3d) */
#define NZ_MODE_PHASE 2     /* per-direction phase[ndir][N] (randomWalk3d_phase_multidirr) */
#define NZ_MODE_PHI 4       /* Kahan 3-vector Phi = sum_n G_n p_n; phase_d = u_d . Phi */
#define NZ_MODE_MOMENTS 8   /* per-step displacement moments (fused walk only) */
#define NZ_MODE_TANGENT64 16 /* fused walk: a solve whose normalised discriminant sqterm/4a is below
                                1e-6 um^2 (a near-tangent ray) is recomputed in FP64 */

/* list format of every job of one nz_walk_batch launch (mode bits; none: the
 * per-entry record lists) */
#define NZ_LIST_IDX16 64    /* substrates with idx_bytes 2 */
#define NZ_LIST_IDX32 128   /* substrates with idx_bytes 4 */

/* per-walker flag bits */
#define NZ_FLAG_DRAWS_EXHAUSTED 1
#define NZ_FLAG_ITER_CAP 2
#define NZ_FLAG_UNSEEDED 4
#define NZ_FLAG_BOUNDS 8    /* bounds-checked build only: an index was out of range (the access was skipped) */
#define NZ_FLAG_STAGE_TIMEOUT 16 /* nz_walk_batch_staged: the copy of the substrate's records into shared
                                    memory did not complete in time; the records were read from global memory
                                    (the walk's result is unchanged) */

/* Box [-L/2, L/2]^3 and uniform cell grid: the reference kernel's template
 * constants Lx..Lz, dLx..dLz, nLx..nLz (sim3d_kernel.cu:17-28). */
typedef struct nz_grid {
    float Lx, Ly, Lz;
    float dLx, dLy, dLz;
    int nx, ny, nz;
} nz_grid;

/* A substrate on the device: spheres in the reference's SoA layout
 * (geometry.py:58-64, [5,S] = cx, cy, cz, r, structure id), compact cell lists
 * and the per-structure D and T2 (structure nstructures is the box,
 * diffsim3d.py:95-103). */
typedef struct nz_substrate {
    nz_grid grid;
    int nstructures;
    int S;
    const float* spheres;      /* [5, S] float32 */
    const int* cell_start;     /* [ncell] offset of each cell's list in cell_items */
    const int* cell_count;     /* [ncell] */
    const int* cell_items;     /* sphere indices, ascending within a cell */
    const float* cell_sph4;    /* [n_items][4] cx, cy, cz, r of each list entry, per cell ordered by
                                  (structure id, sphere index) (fused walk, nz_cells_gather) */
    const int* cell_sid;       /* [n_items] structure id of each list entry (fused walk) */
    const float* D;            /* [nstructures + 1] um^2/ms */
    const float* T2;           /* [nstructures + 1] ms */
    /* Optional near lists on the same grid, built with a smaller margin
     * near_margin (< the margin of the lists above): the fused walk scans them
     * for an iteration whose walker-to-cell distance plus reach fits inside
     * near_margin (then every sphere it can hit is in them and every sphere in
     * them is in the full list, so the result is the full list's), the full
     * lists otherwise.  near_sph4 == NULL: no near lists. */
    float near_margin;
    const int* near_start;
    const int* near_count;
    const float* near_sph4;
    const int* near_sid;
    /* Index form of the fused walk's lists (idx_bytes 2 or 4; 0: the
     * per-entry records above, which may then be NULL).  The spheres are put
     * in record order -- sorted by structure id, stable -- and rec4 holds
     * their (cx, cy, cz, r), rec_sid their structure ids; sid_start[k]
     * (k = 0 .. nstructures + 1) is the first record of a structure >= k
     * (sid_start[nstructures] = sid_start[nstructures + 1] = S).  A list
     * entry is a record index (uint16_t when idx_bytes is 2, int32 when 4),
     * ascending within a cell, laid out by the same cell_start / cell_count
     * (near_start / near_count for near_idx) as the record lists
     * (nz_cells_index).  Entries ascending by record are ascending by
     * structure, so a walker labelled L stops at the first record at or
     * beyond sid_start[L + 1]: no structure id is read per entry. */
    int idx_bytes;
    const void* cell_idx;
    const void* near_idx;
    const float* rec4;         /* [S][4], 16-byte aligned */
    const int* rec_sid;        /* [S] */
    const int* sid_start;      /* [nstructures + 2] */
    /* Entries of the cell lists and of the near lists (0: not given).  Only
     * the bounds-checked build reads them, to check every list range. */
    int n_items;
    int near_items;
} nz_substrate;

/* Source of the normal draws: an injected table normals[N][nsteps][maxk]
 * (k-th normal of a walker within a step; the reference's draw order), or,
 * with table == NULL, Philox4x32-10 at counter (walker, step, draw, stream)
 * under key (key0, key1). */
typedef struct nz_draws {
    const float* table;
    int nsteps, maxk;
    uint32_t key0, key1, stream;
} nz_draws;

/* Walkers in the reference's layout (diffsim3d.py:42-45, :62). */
typedef struct nz_walkers {
    int N;
    float* spins;          /* [3, N] */
    float* spins0;         /* [3, N] */
    float* phase;          /* [ndir, N] (NZ_MODE_PHASE) */
    const float* diffdir;  /* [3, ndir] (NZ_MODE_PHASE) */
    int ndir;
    float* sig;            /* [N] (NZ_MODE_SIG) */
    float* phi;            /* [6, N] Phi sums then compensations (NZ_MODE_PHI) */
    int* label;            /* [N] structure of the walker at its last iteration, or NULL */
    int* n_iter;           /* [N] accumulated collision-loop iterations, or NULL */
    int* n_scatter;        /* [N] accumulated scatterings (truncated jumps), or NULL */
    int* flags;            /* [N] NZ_FLAG_* bits, or NULL */
} nz_walkers;

/* Walkers packed for the fused walk: four float4 per walker,
 * pos = (x, y, z, label bits), org = (x0, y0, z0, walker id bits),
 * phi = (Phi_x, Phi_y, Phi_z, sig), comp = (Kahan x, y, z, flag bits). */
typedef struct nz_state {
    int N;
    float* pos;
    float* org;
    float* phi;
    float* comp;
} nz_state;

/* One job of the batched walk: a substrate, a protocol and a walker range. */
typedef struct nz_job {
    nz_substrate sub;
    const float* G;        /* [nsteps] unit-waveform phase increment per step */
    const float* Garea;    /* [nsteps] wrap correction per step */
    int nsteps;
    float dt;
    nz_draws draws;        /* Philox only (table must be NULL) */
    int mode;              /* NZ_MODE_PHI and/or NZ_MODE_SIG */
    nz_state state;
    double* moments;       /* [nsteps][6] (NZ_MODE_MOMENTS) or NULL */
    int step_offset;       /* this job runs steps [step0 + step_offset, step1 + step_offset) of a launch */
} nz_job;

/* A work item: walkers [first, first + count) of job `job`, count <= block size. */
typedef struct nz_item {
    int job;
    int first;
    int count;
} nz_item;

int nz_version(void);
const char* nz_status_string(int status);
const char* nz_last_error(void);
int nz_device_sm_count(int* sms);

/* ---- a1: cell lists — DiffSim3d.set_segments (diffsim3d.py:107-174) ---- */

/* Number of member spheres of every cell: in_segment < jump_tol, evaluated in
 * float64 in the reference's operation order (diffsim3d.py:128-141).
 * spheres64: [5, S] float64. counts: [nx*ny*nz]. */
int nz_cells_count(const double* spheres64, int S, double Lx, double Ly, double Lz, int nx, int ny, int nz,
                   double jump_tol, int* counts, void* stream);

/* Exclusive prefix sum of n ints (one block; n <= 1<<26); total receives the sum. */
int nz_exclusive_scan_i32(const int* in, int* out, int n, int* total, void* stream);

/* Member lists: items[offsets[c] ...] gets the counts[c] members of cell c in
 * ascending index order.  offsets = exclusive scan of counts (nz_cells_count);
 * cursor: scratch of nx*ny*nz ints. */
int nz_cells_fill(const double* spheres64, int S, double Lx, double Ly, double Lz, int nx, int ny, int nz,
                  double jump_tol, const int* offsets, const int* counts, int* cursor, int* items, void* stream);

/* The fused walk's near lists: nz_cells_count / nz_cells_fill with margin
 * `margin`, keeping of each sphere's cells only those whose box lies within
 * r + margin (+ 1e-4 um) of its centre (Euclidean), a subset of the box
 * test that still holds every sphere a walker near the cell can touch or lie
 * inside.  No reference counterpart (the reference has no near lists). */
int nz_cells_count_round(const double* spheres64, int S, double Lx, double Ly, double Lz, int nx, int ny, int nz,
                         double margin, int* counts, void* stream);
int nz_cells_fill_round(const double* spheres64, int S, double Lx, double Ly, double Lz, int nx, int ny, int nz,
                        double margin, const int* offsets, const int* counts, int* cursor, int* items, void* stream);

/* The reference's padded table (diffsim3d.py:144-168): K = the largest member
 * count; cell c's K entries at segments[c*K] are the K spheres of smallest
 * in_segment (ties by lower index), ascending by index. */
int nz_segments_fill(const double* spheres64, int S, double Lx, double Ly, double Lz, int nx, int ny, int nz,
                     int K, int* segments, void* stream);

/* List entries of the fused walk: the entries of cell c at
 * [cell_start[c], cell_start[c] + cell_count[c]) hold the sphere records
 * sph4 = (cx, cy, cz, r) and structure ids sid of that cell's members
 * (items), ordered by (structure id, sphere index). */
int nz_cells_gather(const float* spheres, int S, const int* items, int n_items, const int* cell_start,
                    const int* cell_count, int ncell, float* sph4, int* sid, void* stream);

/* Index lists of the fused walk: idx[k] = perm[items[k]] (perm: the record
 * index of every sphere, [S]; NULL = identity), then each cell's entries
 * sorted ascending.  idx_bytes 2 (uint16_t entries; needs S <= 65536) or 4
 * (int32). */
int nz_cells_index(const int* items, int n_items, const int* perm, int S, const int* cell_start,
                   const int* cell_count, int ncell, void* idx, int idx_bytes, void* stream);

/* ---- a12: substrate ingestion on the device — split_matrix_to_list
 * (utils/common_utils.py:41-55) and createBoundaryZ / create_pad
 * (utils/adjust_geometry.py:3-36), as the simulation driver applies them
 * (cli/simulation_main.py:37-54).  rows: the pickle's matrix [M][5]
 * (x, y, z, r, fibre id), float64, row major, on the device. ----
 *
 * Scratch of nz_ingest_split (M rows) and nz_ingest_plan (M = F fibres). */
size_t nz_ingest_scratch_bytes(int M);
/* Fibre k ends at row ends[k], the k-th row whose z equals L/2 exactly;
 * *n_fibres (one device int) = F.  ends: [M] ints. */
int nz_ingest_split(const double* rows, int M, double L, int* ends, int* n_fibres, void* scratch,
                    size_t scratch_bytes, void* stream);
/* partner[k]: the last fibre whose last row's (x, y) equals fibre k's first
 * row's (x, y), or -1; out_offset[k]: first output row of fibre k (its rows,
 * plus `pad` rows when it has a partner); *n_out = the output row count;
 * *n_bad = padded fibres where it or its partner has fewer than pad/2 rows
 * (the reference's create_pad fails on them).  partner, out_offset: [F]. */
int nz_ingest_plan(const double* rows, const int* ends, int F, int pad, int* partner, int* out_offset, int* n_out,
                   int* n_bad, void* scratch, size_t scratch_bytes, void* stream);
/* The padded fibres, concatenated: out_rows [S][5] as createBoundaryZ returns
 * them (partner rows shifted by -/+Lz, fibre ids truncated to integers), and,
 * when spheres is not NULL, the walk's [5, S] layout (x, y, z, r, fibre
 * index as the structure id). */
int nz_ingest_write(const double* rows, const int* ends, int F, const int* partner, const int* out_offset, int S,
                    double Lz, int pad, double* out_rows, double* spheres, void* stream);

/* ---- substrate-generator collision detection — collide_spheres_gpu
 * (substrate_generator/helper/CollisionDetection.py:10-62) on the grid of
 * blocks it builds: block edges Lx/10 (grid.dLx..dLz = Lx/nx.. in float32,
 * nx.. = ceil(L/(Lx/10)) per axis).  A sphere belongs to a block when all six
 * boundary distances of its set_segments (:65-115) are below 1 um (float32,
 * the reference's operation order).  A pair of spheres of different fibres
 * collides when (r_a + r_b + buff) - |x_a - x_b| > 0 in float32; each pair is
 * reported once, as (min, max).  Spheres that belong to no block take part
 * in no pair.  pos: [S][3] float32; radii, fiber_id: [S] float32. ----
 *
 * Scratch shared by nz_collide_cells and the nz_collide_pairs that follows it. */
size_t nz_collide_scratch_bytes(int S, const nz_grid* grid);
/* Block ranges and member counts; *n_members (one device int) = the total
 * number of (block, sphere) memberships, the size of nz_collide_pairs' items. */
int nz_collide_cells(const float* pos, const float* radii, int S, const nz_grid* grid, int* n_members,
                     void* scratch, size_t scratch_bytes, void* stream);
/* Every colliding pair, unordered, into pairs[cap][2]; *n_pairs = how many
 * there are (more than cap: call again with a larger buffer).  items:
 * n_members ints of scratch for the block lists. */
int nz_collide_pairs(const float* pos, const float* radii, const float* fiber_id, int S, const nz_grid* grid,
                     float buff, int* items, int n_members, int* pairs, int cap, int* n_pairs, void* scratch,
                     size_t scratch_bytes, void* stream);
/* Pairs [n][2] with entries in [0, S) into lexicographic order (out; the
 * order torch.unique gives the reference's rows). */
size_t nz_pairs_sort_scratch_bytes(int S);
int nz_pairs_sort(const int* pairs, int n, int S, int* out, void* scratch, size_t scratch_bytes, void* stream);

/* ---- a7: seeding — seedSpinsKernel (sim3d_kernel.cu:240-337) + SimGeometry3D.gpu_seed
 * (geometry.py:73-174).  target[k] != 0 marks structure k (k = nstructures is the
 * box) as a target.  A position is accepted when the first structure in id order
 * containing it is a target (the box only strictly inside).  Round r draws
 * Philox uniforms at (walker, r, 0, stream); at most max_rounds rounds, all in one
 * launch (no host round trips).  spins: [3,N]; label: [N] (-1 = unseeded);
 * n_unseeded: one device int.  Returns NZ_OK; check *n_unseeded on the host. */
int nz_seed(const nz_substrate* sub, const uint8_t* target, int N, uint32_t key0, uint32_t key1,
            uint32_t stream_id, int max_rounds, float* spins, int* label, int* n_unseeded, void* stream);

/* Walkers [id0, id0 + N) of the same seeding into slots [0, N): a shard of a
 * run sharded over processes seeds exactly its walkers of the unsharded run.
 * No reference counterpart (the reference runs one process per GPU with
 * independent seeds); nz_seed is this with id0 = 0.  id0 + N <= 2^32. */
int nz_seed_range(const nz_substrate* sub, const uint8_t* target, uint32_t id0, int N, uint32_t key0,
                  uint32_t key1, uint32_t stream_id, int max_rounds, float* spins, int* label, int* n_unseeded,
                  void* stream);

/* ---- a3/a4/a5: one time step of every walker, one launch —
 * randomWalk3d (sim3d_kernel.cu:340-522), randomWalk3d_phase (:524-717),
 * randomWalk3d_phase_multidirr (:719-943) as launched by DiffSim3d.step /
 * dwi_step / dwi_multidirections_step (diffsim3d.py:199-226). */
int nz_walk_step(const nz_substrate* sub, const nz_walkers* wk, int mode, float dt, float G, float Garea,
                 int step, const nz_draws* draws, void* stream);

/* ---- fused walk: steps [step0, step1) of every walker in one launch, state
 * in registers, G/Garea tables on the device (DwiSim3d.simulate_multi_directions'
 * loop, diffsim3d.py:246-261, moved onto the device). ---- */
int nz_state_pack(const nz_walkers* wk, const uint32_t* walker_id, nz_state* st, void* stream);
int nz_state_unpack(const nz_state* st, const nz_walkers* wk, void* stream);
/* Unpack in walker-id order: the walker whose id is i goes to column i of the
 * reference layout, undoing any re-binning (ids must be 0..N-1; others are
 * dropped and counted in *n_bad, a device int, when n_bad is not NULL). */
int nz_state_unpack_by_id(const nz_state* st, const nz_walkers* wk, int* n_bad, void* stream);

int nz_walk_fused(const nz_substrate* sub, const nz_state* st, int mode, float dt, const float* G,
                  const float* Garea, int step0, int step1, const nz_draws* draws, double* moments,
                  void* stream);

/* ---- a8: the narrow-pulse loop — randomWalk3d then
 * computeDiffusionCoefficientsAndKurtosis every step (simulation_main.py:91-118,
 * sim3d_kernel.cu:162-238) — as one fused launch plus one reduction.  The walk
 * (mode 0 or NZ_MODE_SIG) stores each walker's float displacement from its
 * origin at the end of every step into scratch ([step1-step0][3][N] floats,
 * nz_walk_fused_moments_scratch_bytes); a reduction kernel then adds, for each
 * step s, the FP64 sums of dx^2, dy^2, dz^2, dx^4, dy^4, dz^4 over walkers to
 * moments[s*6 .. s*6+5] (zeroed by the caller), the terms of nz_moments.  Any
 * number of steps per call (at most 65535); the scratch grows with them. */
size_t nz_walk_fused_moments_scratch_bytes(int N, int nsteps);
int nz_walk_fused_moments(const nz_substrate* sub, const nz_state* st, int mode, float dt, const float* G,
                          const float* Garea, int step0, int step1, const nz_draws* draws, float* scratch,
                          size_t scratch_bytes, double* moments, void* stream);

/* ---- batched persistent walk: every item of every job, steps [step0, step1)
 * of each job (clamped to its nsteps), CTAs pulling items from *queue (one
 * device int, zeroed by the caller) until none is left.  jobs and items are
 * device arrays; every job of one launch has mode `mode`.  grid = CTA count
 * (0 = one CTA per item, no queue); threads = walkers per CTA (a multiple of
 * 32 up to 256); an item holds at most `threads` walkers.  The batched form of
 * the fused walk: many substrates, protocols and walker sets in one launch.
 * mode may carry NZ_LIST_IDX16 or NZ_LIST_IDX32: every job's substrate then
 * has index lists of that width (otherwise every job's has record lists).
 * The device arrays are not read back for checking: the caller guarantees
 * 0 <= item.job < n_jobs, 1 <= item.count <= threads,
 * item.first + item.count <= that job's state.N, and the list format. */
int nz_walk_batch(const nz_job* jobs, int n_jobs, const nz_item* items, int n_items, int mode, int step0, int step1,
                  int* queue, int grid, int threads, void* stream);

/* CTAs of `threads` walkers of the batched walk in `mode` that fit on one SM
 * (the persistent grid is this times the SM count). */
int nz_batch_occupancy(int mode, int threads, int* blocks_per_sm);

/* nz_walk_batch with each job's sphere records staged in shared memory: a CTA
 * whose item belongs to a job of at most stage_records records (S) copies that
 * job's record array (S x 16 bytes) into its shared memory with one bulk copy
 * (cp.async.bulk, completing on an mbarrier) and reads every record of the
 * walk from there; the copy is reused by the CTA's next items of the same
 * job.  Jobs with more records, or whose record array does not start on a
 * 16-byte boundary, read global memory as in nz_walk_batch.  Index lists only
 * (mode carries NZ_LIST_IDX16 or NZ_LIST_IDX32); stage_records in
 * [0, 12288] (192 KiB per CTA; 0 is nz_walk_batch).  Results are bit-identical
 * to nz_walk_batch's.  Every wait for a copy is bounded: a copy that does not
 * complete in time is abandoned, the CTA reads global memory from then on and
 * its walkers of that item get NZ_FLAG_STAGE_TIMEOUT.  Replaces the same
 * gather as nz_walk_batch (reference: segmentList[idxSeg*K+n] in
 * randomWalk3d_phase_multidirr, sim3d_kernel.cu:767-783 and :801-841), with
 * the records in shared memory instead of L1/L2. */
int nz_walk_batch_staged(const nz_job* jobs, int n_jobs, const nz_item* items, int n_items, int mode, int step0,
                         int step1, int* queue, int grid, int threads, int stage_records, void* stream);

/* nz_batch_occupancy for nz_walk_batch_staged with stage_records records of
 * shared memory per CTA (index lists only). */
int nz_batch_occupancy_staged(int mode, int threads, int stage_records, int* blocks_per_sm);

/* ---- walker re-binning: a stable-key counting sort of the packed state by
 * cell, so that the walkers of one CTA share cells.  bins: bin per walker is
 * the cell of its position under `grid` coarsened by `coarsen` per axis;
 * scratch: nz_sort_scratch_bytes(N, nbins) bytes; out: a second state. ---- */
size_t nz_sort_scratch_bytes(int N, int nbins);
int nz_state_sort(const nz_state* in, const nz_grid* grid, int coarsen, nz_state* out, void* scratch,
                  size_t scratch_bytes, void* stream);
/* As nz_state_sort with the key (label, bin) when nlabels > 0: walkers of one
 * structure (label in pos.w; out-of-range labels count as nlabels - 1) are
 * contiguous, ordered by bin within.  Scratch: nz_sort_scratch_bytes(N,
 * nbins * nlabels). */
int nz_state_sort_keyed(const nz_state* in, const nz_grid* grid, int coarsen, int nlabels, nz_state* out,
                        void* scratch, size_t scratch_bytes, void* stream);

/* ---- the re-binning of many jobs at once (the batched walk's step between
 * chunks): one bin count, one scan and one scatter for every job of a chunk,
 * instead of a sort per job.  No reference counterpart (the reference runs
 * one substrate at a time and re-bins nothing).  Job j's walkers take keys
 * [key_offset, key_offset + nz_sort_job_keys(...)) of one key space, its
 * local key being nz_state_sort_keyed's; the walkers are counted and
 * scattered in one pass over all jobs' walkers, and job j's land in its own
 * out state.  walker_offset = the sum of N of the jobs before it. ---- */
typedef struct nz_sort_job {
    nz_state in;           /* the job's walkers (read) */
    nz_state out;          /* receives them re-binned: same N, no array shared with in */
    nz_grid grid;          /* the job's cell grid */
    int coarsen;           /* bins = cells coarsened by this factor per axis */
    int nlabels;           /* > 0: key (label, bin) as nz_state_sort_keyed; 0: bin */
    int walker_offset;
    int key_offset;
} nz_sort_job;

/* Keys of one job: bins, times nlabels when nlabels > 0; -1 for a bad grid. */
long long nz_sort_job_keys(const nz_grid* grid, int coarsen, int nlabels);
size_t nz_batch_sort_scratch_bytes(int total_walkers, int total_keys);
/* jobs: a device array of n_jobs descriptors, in walker_offset order, whose
 * walker_offset / key_offset are the running sums above (the caller
 * guarantees them; the device array is not read back for checking);
 * total_walkers / total_keys: the sums over all jobs. */
int nz_batch_sort(const nz_sort_job* jobs, int n_jobs, int total_walkers, int total_keys, void* scratch,
                  size_t scratch_bytes, void* stream);

/* Re-binning for callers that cannot allocate device memory (no counterpart in
 * the reference, which re-bins nothing).  Same result as nz_state_sort, but the
 * scratch is a fixed 16 MiB device array inside the library (one per GPU that
 * loads it, held until exit): no buffer is passed and nothing is allocated.
 * Fails with NZ_ERR_CAPACITY when nz_sort_scratch_bytes(N, nbins) exceeds
 * nz_state_sort_static_capacity().  The first call on a device looks up the
 * array's device address; make that first call before any stream capture.
 * All calls share the one array: calls that overlap on the GPU (other streams,
 * other threads) race and must be serialised by the caller. */
size_t nz_state_sort_static_capacity(void);
int nz_state_sort_static(const nz_state* in, const nz_grid* grid, int coarsen, nz_state* out, void* stream);

/* ---- a13: signal S[d][b] = sum_w exp(i * amp[b] * u_d . Phi_w) over walkers,
 * FP32 per walker, FP64 sums (the reference stops at per-spin phase,
 * diffsim3d.py:257-261).  dirs: [3, ndir]; amp: [nb]; out: [2][ndir][nb] doubles
 * (real then imaginary), accumulated into (zero it first). ---- */
int nz_signal_phi(const nz_state* st, const float* dirs, int ndir, const float* amp, int nb, double* out,
                  void* stream);

/* Signal from a per-direction phase array (the reference's phase_d layout,
 * [ndir, N] float): out[2][ndir][nb] += sums of cos / sin(amp[b] * phase). */
int nz_signal_phase(const float* phase, int ndir, int N, const float* amp, int nb, double* out, void* stream);

/* Per-direction phase from Phi: phase[d][w] = u_d . (Phi_w - comp_w), float. */
int nz_phase_from_phi(const nz_state* st, const float* dirs, int ndir, float* phase, void* stream);

/* ---- a8: displacement moments of one step —
 * computeDiffusionCoefficientsAndKurtosis (sim3d_kernel.cu:162-238) before its
 * divisions: out[6] += (sum dx^2, dy^2, dz^2, dx^4, dy^4, dz^4), FP64. ---- */
int nz_moments(const float* spins, const float* spins0, int N, double* out, void* stream);

/* ---- measurement aid (no reference counterpart): FP32 fused multiply-add
 * throughput of this GPU, grid x 256 threads x iters x 8 FMAs; the benchmark
 * divides its FP32 work by this peak. ---- */
int nz_probe_fma(int grid, int iters, float* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* NOZOMI_B200_H */
