/*
 * Oracle — TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs load
 * this library, and only as the checker or as the timed CPU baseline; the
 * product (nozomi_b200) never links, loads or calls it.
 *
 * CPU restatement of nozomi's Monte Carlo spin random walk
 * (simulation_toolkit/simulation_engine/sim3d_kernel.cu):
 *   sphere tests / ray-sphere fractions   sim3d_kernel.cu:72-160
 *   rejection seeding rule                sim3d_kernel.cu:240-337, geometry.py:73-174
 *   walk with T2 weighting                sim3d_kernel.cu:340-522
 *   walk with multi-direction phase       sim3d_kernel.cu:719-943
 *   displacement moments                  sim3d_kernel.cu:162-238
 * The single-precision walk evaluates the reference's expressions in source
 * order with IEEE rounding and no contraction (built with -ffp-contract=off),
 * so with the same draws it reproduces the reference bit for bit; the pin is
 * tests/test_oracle_pin.py against fixtures that the reference's own Python
 * driver and kernel source produced (tests/golden/make_golden.py).
 *
 * Walkers are independent, so the oracle runs walker by walker (all steps of
 * one walker, then the next), split over OpenMP threads.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "oz_rng.h"

#define OZ_API __attribute__((visibility("default")))

#define OZ_TOL ((float)1e-4) /* sim3d_kernel.cu:34 const float tol = 1e-4 */
#define OZ_BIG ((float)1e6)  /* sim3d_kernel.cu:35 someLargeNumber */

#define OZ_MIN(a, b) (((a) > (b)) ? (b) : (a)) /* sim3d_kernel.cu:7 */
#define OZ_MAX(a, b) (((a) < (b)) ? (b) : (a)) /* sim3d_kernel.cu:8 */

enum {
    OZ_MODE_SIG = 1,        /* T2 weighting of sig (randomWalk3d) */
    OZ_MODE_PHASE = 2,      /* per-direction phase (randomWalk3d_phase_multidirr) */
    OZ_MODE_PHI = 4,        /* Kahan 3-vector Phi = sum G_n p_n */
    OZ_MODE_TANGENT64 = 8,  /* FP64 near-tangent solves */
};
enum {
    OZ_FLAG_DRAWS_EXHAUSTED = 1, /* injected normal table ran out; the draw reads 0 */
    OZ_FLAG_ITER_CAP = 2,        /* a step ended at the 100-iteration cap */
    OZ_FLAG_UNSEEDED = 4,        /* seeding gave up after its round limit */
};
enum { OZ_RNG_INJECT = 0, OZ_RNG_PHILOX = 1 };

typedef struct oz_geom {
    int S;              /* spheres */
    int nstructures;    /* sphere structures; the box is structure nstructures */
    float Lx, Ly, Lz;   /* box, centred on the origin */
    float dLx, dLy, dLz;/* cell edge per axis */
    float nLx, nLy, nLz;/* cells per axis (float, like the reference's constants) */
    const float* spheres;   /* [5, S] SoA: cx, cy, cz, r, structure id */
    const int* cell_start;  /* [ncell] */
    const int* cell_count;  /* [ncell] */
    const int* cell_items;  /* sphere indices */
    const float* D;         /* [nstructures + 1] um^2/ms */
    const float* T2;        /* [nstructures + 1] ms */
} oz_geom;

typedef struct oz_rng {
    int kind;               /* OZ_RNG_INJECT or OZ_RNG_PHILOX */
    const float* normals;   /* injected: [N][nsteps][maxk], k-th normal of a walker's step */
    int nsteps, maxk;
    uint32_t key0, key1, stream;
    uint32_t id0;           /* Philox: walker w draws at counter id0 + w (a shard's first global id) */
} oz_rng;

static inline void oz_draw3(const oz_rng* rng, int w, int step, int draw,
                            float* n0, float* n1, float* n2, int* flags) {
    if (rng->kind == OZ_RNG_PHILOX) {
        oz_philox_normal3(rng->key0, rng->key1, rng->stream, rng->id0 + (uint32_t)w, (uint32_t)step,
                          (uint32_t)draw, n0, n1, n2);
        return;
    }
    float v[3];
    for (int i = 0; i < 3; ++i) {
        int k = 3 * draw + i;
        if (step < 0 || step >= rng->nsteps || k >= rng->maxk) {
            v[i] = 0.0f;
            if (flags) flags[w] |= OZ_FLAG_DRAWS_EXHAUSTED;
        } else {
            v[i] = rng->normals[((size_t)w * rng->nsteps + step) * rng->maxk + k];
        }
    }
    *n0 = v[0]; *n1 = v[1]; *n2 = v[2];
}

/* Full-FP64 ray-sphere fractions, used by the near-tangent precision form. */
static double oz_in_tol_f64(double dx, double dy, double dz, double r, double jx, double jy, double jz,
                            double tol) {
    if ((dx*dx + dy*dy + dz*dz - r*r) > 0) return 1e6;
    double a = jx*jx + jy*jy + jz*jz;
    double b = 2*(jx*dx + jy*dy + jz*dz);
    double c = dx*dx + dy*dy + dz*dz - (r-tol)*(r-tol);
    double sqterm = b*b - 4*a*c;
    if (sqterm < 0) return 0;
    sqterm = sqrt(sqterm);
    double q = -0.5*(b + sqterm);
    if (b < 0) q = -0.5*(b - sqterm);
    double fpos = q/a, fneg = c/q;
    return OZ_MAX(OZ_MAX(fpos, fneg), 0);
}

static double oz_out_tol_f64(double dx, double dy, double dz, double r, double jx, double jy, double jz,
                             double tol) {
    double a = jx*jx + jy*jy + jz*jz;
    double b = 2*(jx*dx + jy*dy + jz*dz);
    double c = dx*dx + dy*dy + dz*dz - (r+tol)*(r+tol);
    double sqterm = b*b - 4*a*c;
    if (sqterm < 0) return 1e6;
    sqterm = sqrt(sqterm);
    double q = -0.5*(b + sqterm);
    if (b < 0) q = -0.5*(b - sqterm);
    double fpos = q/a, fneg = c/q;
    if ((dx*dx + dy*dy + dz*dz - r*r) < 0) return OZ_MAX(fpos, fneg);
    if (fpos > 0 && fneg > 0) return OZ_MIN(fpos, fneg);
    else if ((fpos < 0 && fneg < 0) || (b > 0)) return 1e6;
    return 0;
}

/* Optional FP64 phase of the single-precision trajectory ([ndir, N], set by
 * oz_set_phase64 for the next oz_walk_f32 call; needs diffdir). */
static double* g_phase64 = NULL;

/* ---- single precision, the reference's arithmetic ---- */
#define REAL float
#define SFX(name) oz_##name##_f32
#define RSQRT sqrtf
#define RFLOOR floorf
#define REXP expf
#include "walk_step.inc"
#undef REAL
#undef SFX
#undef RSQRT
#undef RFLOOR
#undef REXP

/* ---- full double precision ---- */
#define REAL double
#define SFX(name) oz_##name##_f64
#define RSQRT sqrt
#define RFLOOR floor
#define REXP exp
#include "walk_step.inc"
#undef REAL
#undef SFX
#undef RSQRT
#undef RFLOOR
#undef REXP

static int oz_threads(int nthreads) {
#ifdef _OPENMP
    return nthreads > 0 ? nthreads : omp_get_max_threads();
#else
    (void)nthreads;
    return 1;
#endif
}

/*
 * Steps [step0, step0 + nsteps) for all N walkers.  G and Garea are indexed by
 * absolute step (the per-sample arguments of diffsim3d.py:252-255).  Any of
 * phase, sig, phi, label, n_iter, n_scatter, flags, work may be NULL when the
 * mode does not need them.  work (length 4, summed over walkers): iterations,
 * spheres within reach, solves within reach, unused.
 */
OZ_API int oz_walk_f32(const oz_geom* g, const oz_rng* rng, int mode, int N, int step0, int nsteps,
                       float dt, const float* G, const float* Garea,
                       float* spins, float* spins0, float* phase, const float* diffdir, int ndir,
                       float* sig, float* phi, int* label, int* n_iter, int* n_scatter, int* flags,
                       long long* work, int nthreads) {
    if (!g || !rng || N < 0 || nsteps < 0) return 1;
    const int nt = oz_threads(nthreads);
    long long acc0 = 0, acc1 = 0, acc2 = 0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64) reduction(+:acc0,acc1,acc2)
    for (int w = 0; w < N; ++w) {
        long long wk[4] = {0, 0, 0, 0};
        for (int s = step0; s < step0 + nsteps; ++s)
            oz_walker_step_f32(g, rng, mode, N, w, s, dt, G ? G[s] : 0.0f, Garea ? Garea[s] : 0.0f,
                               spins, spins0, phase, diffdir, ndir, sig, phi, label, n_iter, n_scatter,
                               flags, work ? wk : NULL, g_phase64);
        acc0 += wk[0]; acc1 += wk[1]; acc2 += wk[2];
    }
    if (work) { work[0] += acc0; work[1] += acc1; work[2] += acc2; }
    return 0;
}

OZ_API void oz_set_phase64(double* phase64) { g_phase64 = phase64; }

OZ_API int oz_walk_f64(const oz_geom* g, const oz_rng* rng, int mode, int N, int step0, int nsteps,
                       double dt, const double* G, const double* Garea,
                       double* spins, double* spins0, double* phase, const double* diffdir, int ndir,
                       double* sig, double* phi, int* label, int* n_iter, int* n_scatter, int* flags,
                       int nthreads) {
    if (!g || !rng || N < 0 || nsteps < 0) return 1;
    const int nt = oz_threads(nthreads);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64)
    for (int w = 0; w < N; ++w)
        for (int s = step0; s < step0 + nsteps; ++s)
            oz_walker_step_f64(g, rng, mode, N, w, s, dt, G ? G[s] : 0.0, Garea ? Garea[s] : 0.0,
                               spins, spins0, phase, diffdir, ndir, sig, phi, label, n_iter, n_scatter,
                               flags, NULL, NULL);
    return 0;
}

/*
 * Label of a point: the lowest structure id among the spheres of its cell list
 * that contain it, else nstructures (the box).  Shared by seeding.
 */
static int oz_label_of(const oz_geom* g, float px, float py, float pz) {
    const int S = g->S;
    const float *cx = g->spheres, *cy = cx + S, *cz = cx + 2*S, *rr = cx + 3*S, *sid = cx + 4*S;
    int idx = (int)(OZ_MIN(g->nLz-1, OZ_MAX(0, floorf((pz+g->Lz/2)/g->dLz)))*g->nLx*g->nLy +
                    OZ_MIN(g->nLy-1, OZ_MAX(0, floorf((py+g->Ly/2)/g->dLy)))*g->nLx +
                    OZ_MIN(g->nLx-1, OZ_MAX(0, floorf((px+g->Lx/2)/g->dLx))));
    int label = g->nstructures;
    const int* items = g->cell_items + g->cell_start[idx];
    for (int n = 0; n < g->cell_count[idx]; ++n) {
        int s = items[n];
        float dx = px - cx[s], dy = py - cy[s], dz = pz - cz[s];
        /* seedSpinsKernel's test (sim3d_kernel.cu:299) */
        if (dx*dx + dy*dy + dz*dz < rr[s]*rr[s] && (int)sid[s] < label) label = (int)sid[s];
    }
    return label;
}

/*
 * Rejection seeding (sim3d_kernel.cu:240-337, geometry.py:73-174).  A
 * position is accepted when the first structure, in id order with the box
 * last, that contains it is a target; the box counts only strictly inside.
 * target[k] != 0 marks structure k (k = nstructures is the box) as a target.
 * Positions are (u - 0.5) * L with Philox uniforms of round r at counter
 * (walker, r, 0, stream); at most max_rounds rounds.  Returns the number of
 * walkers left unseeded.
 */
OZ_API int oz_seed_range(const oz_geom* g, const unsigned char* target, uint32_t id0, int N, uint32_t key0,
                         uint32_t key1, uint32_t stream, int max_rounds, float* spins, int* label, int nthreads) {
    const int nt = oz_threads(nthreads);
    int unseeded = 0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 256) reduction(+:unseeded)
    for (int w = 0; w < N; ++w) {
        int ok = 0;
        for (int r = 0; r < max_rounds && !ok; ++r) {
            float u0, u1, u2;
            oz_philox_uniform3(key0, key1, stream, id0 + (uint32_t)w, (uint32_t)r, &u0, &u1, &u2);
            float px = (u0 - 0.5f) * g->Lx;
            float py = (u1 - 0.5f) * g->Ly;
            float pz = (u2 - 0.5f) * g->Lz;
            int lab = oz_label_of(g, px, py, pz);
            int accept;
            if (lab < g->nstructures) accept = target[lab] != 0;
            else accept = target[g->nstructures] &&
                          px > -g->Lx/2 && px < g->Lx/2 && py > -g->Ly/2 && py < g->Ly/2 &&
                          pz > -g->Lz/2 && pz < g->Lz/2;
            if (accept) {
                spins[w] = px; spins[N + w] = py; spins[2*N + w] = pz;
                if (label) label[w] = lab;
                ok = 1;
            }
        }
        if (!ok) {
            unseeded++;
            if (label) label[w] = -1;
        }
    }
    return unseeded;
}

/* Walkers [id0, id0 + N) of the same seeding: walker id0 + w lands in slot w,
 * so shards of a run seed exactly the walkers of the unsharded run. */
OZ_API int oz_seed(const oz_geom* g, const unsigned char* target, int N, uint32_t key0, uint32_t key1,
                   uint32_t stream, int max_rounds, float* spins, int* label, int nthreads) {
    return oz_seed_range(g, target, 0, N, key0, key1, stream, max_rounds, spins, label, nthreads);
}

/* Accept/reject of given positions under the seeding rule (pinned against the
 * reference's seedSpinsKernel). */
OZ_API void oz_seed_accept(const oz_geom* g, const unsigned char* target, int N, const float* pos,
                           unsigned char* accept) {
    for (int w = 0; w < N; ++w) {
        float px = pos[w], py = pos[N + w], pz = pos[2*N + w];
        int lab = oz_label_of(g, px, py, pz);
        if (lab < g->nstructures) accept[w] = target[lab] != 0;
        else accept[w] = target[g->nstructures] &&
                         px > -g->Lx/2 && px < g->Lx/2 && py > -g->Ly/2 && py < g->Ly/2 &&
                         pz > -g->Lz/2 && pz < g->Lz/2;
    }
}

/* One Philox4x32-10 block, in place: c[4] counter, (k0, k1) key. */
OZ_API void oz_philox_block(uint32_t* c, uint32_t k0, uint32_t k1) { oz_philox4x32_10(c, k0, k1); }

/* The Box-Muller pair of n word pairs: out[2i], out[2i+1] from (ua[i], ub[i]). */
OZ_API void oz_box_muller_pairs(const uint32_t* ua, const uint32_t* ub, int n, float* out) {
    for (int i = 0; i < n; ++i) oz_box_muller(ua[i], ub[i], out + 2 * i, out + 2 * i + 1);
}

/* Normals of draws [0, ndraw) of every walker at one step: out[w][d][3]. */
OZ_API void oz_philox_normals(uint32_t key0, uint32_t key1, uint32_t stream, int N, int step, int ndraw,
                              float* out) {
    for (int w = 0; w < N; ++w)
        for (int d = 0; d < ndraw; ++d) {
            float* o = out + ((size_t)w * ndraw + d) * 3;
            oz_philox_normal3(key0, key1, stream, (uint32_t)w, (uint32_t)step, (uint32_t)d, o, o + 1, o + 2);
        }
}

/* Sums of dx^2 and dx^4 per axis over walkers, in double
 * (computeDiffusionCoefficientsAndKurtosis, sim3d_kernel.cu:162-238, before
 * its division by 2tN and N).  out: [sx2, sy2, sz2, sx4, sy4, sz4]. */
OZ_API void oz_moments(int N, const float* spins, const float* spins0, double* out) {
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int w = 0; w < N; ++w)
        for (int a = 0; a < 3; ++a) {
            /* the displacement in float, as sim3d_kernel.cu:193-195 forms it */
            double d = (double)(spins[a*N + w] - spins0[a*N + w]);
            acc[a] += d*d;
            acc[3 + a] += d*d*d*d;
        }
    memcpy(out, acc, sizeof acc);
}

/*
 * Signal from the Kahan 3-vector Phi ([6, N]: sums then compensations):
 * S[d][b] = (1/N) sum_w exp(i * amp[b] * u_d . (Phi_w - comp_w)), in double.
 */
OZ_API void oz_signal_phi(int N, const float* phi, const double* dirs, int ndir, const double* amp, int nb,
                          double* re, double* im) {
    for (int i = 0; i < ndir * nb; ++i) { re[i] = 0; im[i] = 0; }
    for (int w = 0; w < N; ++w) {
        double px = (double)phi[w] - (double)phi[3*N + w];
        double py = (double)phi[N + w] - (double)phi[4*N + w];
        double pz = (double)phi[2*N + w] - (double)phi[5*N + w];
        for (int d = 0; d < ndir; ++d) {
            double ph = dirs[d]*px + dirs[ndir + d]*py + dirs[2*ndir + d]*pz;
            for (int b = 0; b < nb; ++b) {
                re[d*nb + b] += cos(amp[b]*ph);
                im[d*nb + b] += sin(amp[b]*ph);
            }
        }
    }
    for (int i = 0; i < ndir * nb; ++i) { re[i] /= N; im[i] /= N; }
}

/* Signal from a per-direction phase array [ndir, N] (double). */
OZ_API void oz_signal_phase(int N, const double* phase, int ndir, const double* amp, int nb,
                            double* re, double* im) {
    for (int i = 0; i < ndir * nb; ++i) { re[i] = 0; im[i] = 0; }
    for (int d = 0; d < ndir; ++d)
        for (int w = 0; w < N; ++w)
            for (int b = 0; b < nb; ++b) {
                re[d*nb + b] += cos(amp[b]*phase[(size_t)d*N + w]);
                im[d*nb + b] += sin(amp[b]*phase[(size_t)d*N + w]);
            }
    for (int i = 0; i < ndir * nb; ++i) { re[i] /= N; im[i] /= N; }
}

/*
 * Member cell lists (diffsim3d.py:128-141 predicate, float64, reference
 * operation order), sphere by sphere over the box of cells each sphere can
 * belong to.  Two calls: items == NULL fills count[ncell] and returns the
 * total; otherwise start[] (exclusive scan of count) is filled and items[]
 * receives each cell's members in ascending index order.
 */
static inline double oz_seg_lo(double n, double dL, double r, double x, double L) { return n*dL - r - x - L/2; }
static inline double oz_seg_hi(double n, double dL, double r, double x, double L) { return x - ((n+1)*dL + r - L/2); }

static void oz_axis_range(double x, double r, double L, int nseg, double tol, int* lo, int* hi) {
    double dL = L / nseg;
    int a = (int)floor((x - r + L/2 - tol) / dL) - 2;
    int b = (int)ceil((tol + r + x + L/2) / dL) + 2;
    if (a < 0) a = 0;
    if (b > nseg - 1) b = nseg - 1;
    *lo = 1; *hi = 0;
    for (int n = a; n <= b; ++n) {
        if (oz_seg_lo(n, dL, r, x, L) < tol && oz_seg_hi(n, dL, r, x, L) < tol) {
            if (*lo > *hi) *lo = n;
            *hi = n;
        }
    }
}

OZ_API long long oz_cells(const double* sph, int S, double Lx, double Ly, double Lz, int nx, int ny, int nz,
                          double tol, int* count, int* start, int* items) {
    const long long ncell = (long long)nx * ny * nz;
    if (!items) {
        memset(count, 0, sizeof(int) * ncell);
    } else {
        long long acc = 0;
        for (long long c = 0; c < ncell; ++c) { start[c] = (int)acc; acc += count[c]; }
        memset(count, 0, sizeof(int) * ncell);
    }
    long long total = 0;
    for (int s = 0; s < S; ++s) {
        double x = sph[s], y = sph[S + s], z = sph[2*S + s], r = sph[3*S + s];
        int x0, x1, y0, y1, z0, z1;
        oz_axis_range(x, r, Lx, nx, tol, &x0, &x1);
        oz_axis_range(y, r, Ly, ny, tol, &y0, &y1);
        oz_axis_range(z, r, Lz, nz, tol, &z0, &z1);
        for (int p = z0; p <= z1; ++p)
            for (int m = y0; m <= y1; ++m)
                for (int n = x0; n <= x1; ++n) {
                    long long c = ((long long)p * ny + m) * nx + n;
                    if (items) items[start[c] + count[c]] = s;
                    count[c]++;
                    total++;
                }
    }
    return total;
}

/*
 * The reference's padded cell table (diffsim3d.py:144-168): K = the largest
 * member count; cell c = p*nx*ny + m*nx + n gets, at seg[c*K], the K spheres
 * of smallest in_segment (ties to the lower index; numpy's unstable argsort
 * leaves them unspecified), ascending by index.  in_segment is the maximum of
 * six per-axis terms, so each axis's terms are computed once per (cell
 * column, sphere) and combined per cell.
 */
static inline int oz_heap_less(double va, int ia, double vb, int ib) { return va < vb || (va == vb && ia < ib); }

static void oz_heap_sift_down(double* hv, int* hi, int n, int i) {
    for (;;) {
        int l = 2*i + 1, r = l + 1, m = i;
        if (l < n && oz_heap_less(hv[m], hi[m], hv[l], hi[l])) m = l;
        if (r < n && oz_heap_less(hv[m], hi[m], hv[r], hi[r])) m = r;
        if (m == i) return;
        double tv = hv[i]; hv[i] = hv[m]; hv[m] = tv;
        int ti = hi[i]; hi[i] = hi[m]; hi[m] = ti;
        i = m;
    }
}

static void oz_heap_sift_up(double* hv, int* hi, int i) {
    while (i > 0) {
        int p = (i - 1) / 2;
        if (!oz_heap_less(hv[p], hi[p], hv[i], hi[i])) return;
        double tv = hv[i]; hv[i] = hv[p]; hv[p] = tv;
        int ti = hi[i]; hi[i] = hi[p]; hi[p] = ti;
        i = p;
    }
}

static int oz_cmp_int(const void* a, const void* b) { return (*(const int*)a > *(const int*)b) - (*(const int*)a < *(const int*)b); }

OZ_API int oz_segments(const double* sph, int S, double Lx, double Ly, double Lz, int nx, int ny, int nz, int K,
                       int* seg, int nthreads) {
    if (K <= 0 || K > S) return -1;
    const double dLx = Lx / nx, dLy = Ly / ny, dLz = Lz / nz;
    double* vx = (double*)malloc(sizeof(double) * (size_t)nx * S);
    double* vy = (double*)malloc(sizeof(double) * (size_t)ny * S);
    double* vz = (double*)malloc(sizeof(double) * (size_t)nz * S);
    if (!vx || !vy || !vz) { free(vx); free(vy); free(vz); return -2; }
    for (int s = 0; s < S; ++s) {
        const double x = sph[s], y = sph[S + s], z = sph[2*S + s], r = sph[3*S + s];
        for (int n = 0; n < nx; ++n) vx[(size_t)n*S + s] = OZ_MAX(oz_seg_lo(n, dLx, r, x, Lx), oz_seg_hi(n, dLx, r, x, Lx));
        for (int m = 0; m < ny; ++m) vy[(size_t)m*S + s] = OZ_MAX(oz_seg_lo(m, dLy, r, y, Ly), oz_seg_hi(m, dLy, r, y, Ly));
        for (int p = 0; p < nz; ++p) vz[(size_t)p*S + s] = OZ_MAX(oz_seg_lo(p, dLz, r, z, Lz), oz_seg_hi(p, dLz, r, z, Lz));
    }
    const long long ncell = (long long)nx * ny * nz;
    const int nt = oz_threads(nthreads);
#pragma omp parallel num_threads(nt)
    {
        double* hv = (double*)malloc(sizeof(double) * K);
        int* hi = (int*)malloc(sizeof(int) * K);
#pragma omp for schedule(dynamic, 64)
        for (long long c = 0; c < ncell; ++c) {
            const int n = (int)(c % nx), m = (int)((c / nx) % ny), p = (int)(c / ((long long)nx * ny));
            const double* ax = vx + (size_t)n*S;
            const double* ay = vy + (size_t)m*S;
            const double* az = vz + (size_t)p*S;
            int h = 0;
            for (int s = 0; s < S; ++s) {
                const double v = OZ_MAX(OZ_MAX(ax[s], ay[s]), az[s]);
                if (h < K) {
                    hv[h] = v; hi[h] = s; oz_heap_sift_up(hv, hi, h); ++h;
                } else if (oz_heap_less(v, s, hv[0], hi[0])) {
                    hv[0] = v; hi[0] = s; oz_heap_sift_down(hv, hi, K, 0);
                }
            }
            int* out = seg + c * K;
            memcpy(out, hi, sizeof(int) * K);
            qsort(out, K, sizeof(int), oz_cmp_int);
        }
        free(hv); free(hi);
    }
    free(vx); free(vy); free(vz);
    return 0;
}
