// Fused walk: many time steps per launch, walker state in registers.
//
// The collision rule is the reference's, unchanged
// (simulation_toolkit/simulation_engine/sim3d_kernel.cu:758-874): label, first
// draw, collision pass over the cell's spheres, advance, scatter or continue.
// What changes is how the work is organised:
//
//  * one thread per walker runs a whole range of steps; each lane moves to its
//    next step as soon as its current one ends, so lanes of a warp do not wait
//    for each other's extra collision iterations at every step;
//  * the reference's two passes over the cell list (label, then collisions)
//    are one pass under the label carried from the previous iteration; the
//    pass proves that label (some containing sphere of that structure, none of
//    a lower one) or the iteration is redone with the recomputed label, so the
//    result is the reference's;
//  * the list is scanned in two passes.  The first, predicated and over
//    every entry, marks the near spheres: a sphere whose (r + tol) ball lies
//    more than 2 % + 2 nm beyond this iteration's reach |j| * jump_remaining
//    neither contains the walker nor can lower the jump fraction (its root
//    exceeds jump_remaining), so it is dropped.  The second, over the near
//    spheres of a 32-entry chunk only, runs the reference's inside test and
//    the fractions, so a warp pays for the most near spheres of any lane
//    rather than for every entry twice;
//  * the near lists (the same cell grid with a smaller margin) serve every
//    iteration whose reach fits their margin; the full lists the rest;
//  * the cell list entries carry their sphere's (cx, cy, cz, r) and structure
//    id inline (one 16-byte and one 4-byte read-only load per entry; walkers
//    in the box read no structure id);
//  * each iteration has one draw site (the scatter draw of this step or the
//    first draw of the next), and the inside and outside fractions share one
//    instruction stream (step_either);
//  * phase is accrued as the 3-vector Phi = sum_n G_n p_n with Kahan
//    compensation, the wrap correction on the wrapped axis only; every
//    direction's phase is u_d . Phi (the reference's per-direction sums
//    regrouped; identical in exact arithmetic);
//  * draws are counter-based (Philox at walker, step, draw), so a walker's
//    trajectory does not depend on which thread, CTA or launch runs it.
#include <algorithm>
#include <cstdint>
#include <mutex>
#include "kernels.cuh"

namespace nz {

struct ScanOut {
  float fin, fout;
  bool any_in;
};

// One list entry: its sphere's record and a key.  Record lists (LK 0): the
// record inline, the key the structure id (-1 for a walker in the box, which
// reads none).  Index lists (LK 2 or 4): the key the record index, the record
// read from the substrate's record array.  In the bounds-checked build a
// record index outside [0, S) sets oob and reads nothing: the entry becomes
// a NaN record that is neither near nor containing, with a key that stops
// nothing.
// The records of a job staged in shared memory (staged batched walk only).
extern __shared__ __align__(16) float4 s_stage[];

template <int LK, bool SH>
__device__ __forceinline__ void entry(const void* __restrict__ list, const float4* __restrict__ rec,
                                      const int* __restrict__ sid, int k, bool box, int S, int& oob, int& key,
                                      float4& c) {
  if constexpr (LK == 0) {
    key = box ? -1 : __ldg(sid + k);
    c = __ldg(rec + k);
  } else {
    if constexpr (LK == 2) key = int(__ldg(static_cast<const unsigned short*>(list) + k));
    else key = __ldg(static_cast<const int*>(list) + k);
    if (kCheckBounds && (key < 0 || key >= S)) {
      oob = 1;
      key = -1;
      c = make_float4(__int_as_float(0x7fc00000), 0.f, 0.f, 0.f);
      return;
    }
    if constexpr (SH) c = s_stage[key];  // SH: the job's records were copied into s_stage
    else c = __ldg(rec + key);
  }
}

// One pass over a cell's list under assumed label L.  Returns false when the
// walker's label is not L (then nothing in `o` is used).  The entries of a
// cell are ordered by structure id: the pass ends at the first entry of a
// structure above L (the reference skips those spheres, :805-806).  In index
// form an entry's structure is compared through its record index: records
// [lo, hi) are structure L's, so key < hi is "structure <= L" and key < lo
// "structure < L".
template <int LK, bool T64, bool SH>
__device__ __forceinline__ bool scan_cell(const void* __restrict__ list, const float4* __restrict__ rec,
                                          const int* __restrict__ sid, int start, int count, int nstructures,
                                          int lo, int hi, float x, float y, float z, int L, float a, float jx,
                                          float jy, float jz, float reach, int S, int& oob, ScanOut& o) {
  o.fin = 0.0f;
  o.fout = kBig;
  o.any_in = false;
  bool found = false, lower = false, stop = false;
  // A walker in the box (label nstructures) has every entry below its label:
  // nothing to stop at and no structure to compare.
  const bool box = L >= nstructures;
  const float slack = kTol + reach * 1.02f + 2e-3f;
  for (int base = 0; base < count && !stop; base += 32) {
    const int m = min(32, count - base);
    // first pass: which entries are near, i.e. within (r + slack), a slack of
    // at least 2.1 nm that dwarfs the rounding of d2 and r*r, so that a far
    // sphere neither contains the walker nor lies within this iteration's
    // reach; predicated, one entry per load
    // kScanUnroll entries are loaded together, so that their loads (two
    // dependent ones each in index form) are in flight at once; entries past
    // the first of a higher structure are invalid too (keys ascend), so a
    // batch never marks one near
    uint32_t near_mask = 0u;
    for (int i0 = 0; i0 < m && !stop; i0 += kScanUnroll) {
      int key[kScanUnroll];
      float4 c[kScanUnroll];
#pragma unroll
      for (int u = 0; u < kScanUnroll; ++u) {
        if (kScanUnroll == 1 || i0 + u < m) {
          entry<LK, SH>(list, rec, sid, start + base + i0 + u, box, S, oob, key[u], c[u]);
        } else {  // past the chunk: a NaN record, never near, stops nothing
          key[u] = -1;
          c[u] = make_float4(__int_as_float(0x7fc00000), 0.f, 0.f, 0.f);
        }
      }
#pragma unroll
      for (int u = 0; u < kScanUnroll; ++u) {
        const bool valid = LK == 0 ? key[u] <= L : (box || key[u] < hi);
        stop |= !valid;
        const float dx = x - c[u].x, dy = y - c[u].y, dz = z - c[u].z;
        // a filter, not the reference's arithmetic: fused multiply-adds are
        // fine here (their rounding is far inside the slack)
        const float d2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, dz * dz));
        const float t = c[u].w + slack;
        near_mask |= (valid && d2 <= t * t) ? (1u << (i0 + u)) : 0u;
      }
    }
    // second pass, near entries only: the reference's inside test, then the
    // fraction of a containing sphere or of a lower structure's sphere
    while (near_mask) {
      const int i = __ffs(near_mask) - 1;
      near_mask &= near_mask - 1;
      int key;
      float4 c;
      entry<LK, SH>(list, rec, sid, start + base + i, box, S, oob, key, c);
      const bool below = LK == 0 ? key < L : (box || key < lo);
      const float dx = x - c.x, dy = y - c.y, dz = z - c.z;
      const float d2 = dx * dx + dy * dy + dz * dz;
      const bool inside = d2 - c.w * c.w < 0;
      lower |= inside && below;
      found |= inside && !below;
      if (inside || below) {
        const float f = step_either_t<T64>(inside, dx, dy, dz, c.w, a, jx, jy, jz);
        if (inside) {
          o.any_in = true;
          if (o.fin < f) o.fin = f;
        } else if (f < o.fout) {
          o.fout = f;
        }
      }
    }
  }
  return !(lower || (L < nstructures && !found));
}

// The reference's label pass (sim3d_kernel.cu:766-785): lowest structure id
// among the spheres containing the walker, nstructures if none.  In index
// form the entries ascend by structure, so the first containing one decides.
template <int LK, bool SH>
__device__ __forceinline__ int label_of(const void* __restrict__ list, const float4* __restrict__ rec,
                                        const int* __restrict__ sid, const int* __restrict__ rec_sid, int start,
                                        int count, int nstructures, float x, float y, float z, int S, int& oob) {
  int L = nstructures;
  for (int i = 0; i < count; ++i) {
    if constexpr (LK == 0) {
      const int s = __ldg(sid + start + i);
      if (s < L) {
        const float4 c = __ldg(rec + start + i);
        if (inside_test(x - c.x, y - c.y, z - c.z, c.w) < 0) L = s;
      }
    } else {
      int key;
      float4 c;
      entry<LK, SH>(list, rec, sid, start + i, false, S, oob, key, c);
      if (inside_test(x - c.x, y - c.y, z - c.z, c.w) < 0) return __ldg(rec_sid + key);
    }
  }
  return L;
}

// Records [lo, hi) of structure L in index form (hi = lo = S for the box).
__device__ __forceinline__ void label_bounds(const JobDev& J, int L, int& lo, int& hi) {
  if (L >= J.nstructures) {
    lo = hi = J.S;
  } else {
    lo = __ldg(J.sid_start + L);
    hi = __ldg(J.sid_start + L + 1);
  }
}

// Cell of the walker at the start of a step and the cell's low corner: the
// clamped floor of (x + L/2) times the reciprocal cell edge.  For a walker
// within a rounding error of a cell face this can be the neighbour of the
// reference's division-based cell (cell_of); the walk's result is the same
// with either: the near test measures the walker's distance to the cell taken
// here, and the full lists reach jump_tol beyond their cell, so both lists
// hold every sphere the iteration can touch or be inside.
__device__ __forceinline__ int step_cell(const JobDev& J, float x, float y, float z, float& lox, float& loy,
                                         float& loz) {
  const Grid& g = J.g;
  const float cz = ref_min(g.nLz - 1, ref_max(0, floorf((z + g.Lz / 2) * J.idLz)));
  const float cy = ref_min(g.nLy - 1, ref_max(0, floorf((y + g.Ly / 2) * J.idLy)));
  const float cx = ref_min(g.nLx - 1, ref_max(0, floorf((x + g.Lx / 2) * J.idLx)));
  lox = cx * g.dLx - g.Lx / 2;
  loy = cy * g.dLy - g.Ly / 2;
  loz = cz * g.dLz - g.Lz / 2;
  return int(cz * g.nLx * g.nLy + cy * g.nLx + cx);
}

// Start and count of cell `cell`'s list (the near list when near).  In the
// bounds-checked build a cell outside the grid, or a range outside the list,
// gives an empty list and sets oob.
__device__ __forceinline__ void cell_list(const JobDev& J, bool near, int cell, int& start, int& count, int& oob) {
  if (kCheckBounds && (cell < 0 || cell >= J.ncell)) {
    oob = 1;
    start = count = 0;
    return;
  }
  start = __ldg((near ? J.near_start : J.cell_start) + cell);
  count = __ldg((near ? J.near_count : J.cell_count) + cell);
  if (kCheckBounds) {
    const int n = near ? J.near_items : J.n_items;
    if (start < 0 || count < 0 || (n > 0 && start + count > n)) {
      oob = 1;
      start = count = 0;
    }
  }
}

// This iteration's reach |j| * jump_remaining, from the hardware reciprocal
// square root: within a few ulp of sqrtf, far inside the 2 % + 2 nm of slack
// of the only two uses (the near test and the first-pass filter), which
// decide what is scanned, never a result.
__device__ __forceinline__ float reach_of(float a, float jr) { return a * rsqrtf(fmaxf(a, 1e-30f)) * jr; }

// Draw `draw` of step s scaled by ds.
__device__ __forceinline__ void jump_of(const JobDev& J, uint32_t wid, int s, int draw, float ds, float& jx, float& jy,
                                        float& jz) {
  float n0, n1, n2;
  philox_normal3(J.key0, J.key1, J.stream, wid, uint32_t(s), uint32_t(draw), n0, n1, n2);
  jx = ds * n0;
  jy = ds * n1;
  jz = ds * n2;
}

// Steps [s0, s1) of walker w.  Registers hold position, label, Phi and its
// compensation and the step's jump; the origin (spins0) and the flag word stay
// in memory and are updated in place on the rare wrap / iteration-cap events
// (except with moments, which read the origin every step).
template <int MODE, int LK, bool SH>
__device__ __forceinline__ void walk_one(const JobDev& J, int w, int s0, int s1, double* s_mom) {
  constexpr bool kMom = (MODE & NZ_MODE_MOMENTS) != 0;
  constexpr bool kDisp = (MODE & kModeDisp) != 0;
  constexpr bool kOrig = kMom || kDisp;  // origin in registers
  const float4 P = J.pos[w];
  float x = P.x, y = P.y, z = P.z;
  int label = __float_as_int(P.w);
  const uint32_t wid = __float_as_uint(J.org[w].w);
  float fx = 0.f, fy = 0.f, fz = 0.f, sig = 1.f, kx = 0.f, ky = 0.f, kz = 0.f;
  if (MODE & (NZ_MODE_PHI | NZ_MODE_SIG)) {
    const float4 F = J.phi[w];
    fx = F.x; fy = F.y; fz = F.z; sig = F.w;
  }
  if (MODE & NZ_MODE_PHI) {
    const float4 C = J.comp[w];
    kx = C.x; ky = C.y; kz = C.z;
  }
  float x0 = 0.f, y0 = 0.f, z0 = 0.f;
  if (kOrig) {
    const float4 O = J.org[w];
    x0 = O.x; y0 = O.y; z0 = O.z;
  }
  if (label < 0 || label > J.nstructures) label = J.nstructures;
  int lo = 0, hi = 0;  // index form: structure `label`'s records
  if (LK) label_bounds(J, label, lo, hi);

  const float dt = J.dt;
  const bool has_near = (LK ? J.near_idx : static_cast<const void*>(J.near_sph4)) != nullptr;
  int s = s0;
  int niter = 0, draw = 0, cell = 0;
  // start and count of the step cell's primary list (the near list where
  // there is one), loaded as soon as the cell is known so that the load
  // overlaps the draw
  int pstart = 0, pcount = 0;
  float lox = 0.f, loy = 0.f, loz = 0.f;  // low corner of the step's cell
  float jr = 1.0f, jx = 0.0f, jy = 0.0f, jz = 0.0f;
  // ds depends on the label only; it is recomputed when the label at the
  // start of a step differs from the one it was computed for
  int ds_label = label;
  float ds = sqrtf(2 * __ldg(J.D + label) * dt);
  int oob = 0;  // bounds-checked build: an index was out of range
  if (s < s1) {
    cell = step_cell(J, x, y, z, lox, loy, loz);
    cell_list(J, has_near, cell, pstart, pcount, oob);
    jump_of(J, wid, s, 0, ds, jx, jy, jz);
    draw = 1;
  }
  while (s < s1) {
    niter++;
    float jc = jr;
    float a = jx * jx + jy * jy + jz * jz;
    float reach = reach_of(a, jr);
    // Near list when everything this iteration can touch lies within its
    // margin of the step's cell: distance from the walker to the cell plus
    // the reach, with 2 % + 2 nm of slack against rounding
    // ((dist + reach) * 1.02 + tol + 2 nm <= margin, as dist^2 <= t^2 with
    // t = near_cut - reach).
    bool near = false;
    if (has_near) {
      const float ex = fmaxf(0.f, fmaxf(lox - x, x - (lox + J.g.dLx)));
      const float ey = fmaxf(0.f, fmaxf(loy - y, y - (loy + J.g.dLy)));
      const float ez = fmaxf(0.f, fmaxf(loz - z, z - (loz + J.g.dLz)));
      const float t = J.near_cut - reach;
      near = t >= 0.f && ex * ex + ey * ey + ez * ez <= t * t;
    }
    const void* list = LK ? (near ? J.near_idx : J.idx) : nullptr;
    const float4* sph4 = LK ? J.rec4 : (near ? J.near_sph4 : J.sph4);
    const int* sidv = LK ? nullptr : (near ? J.near_sid : J.sid);
    int start = pstart, count = pcount;
    if (has_near && !near) cell_list(J, false, cell, start, count, oob);
    ScanOut r;
    constexpr bool kT64 = (MODE & NZ_MODE_TANGENT64) != 0;
    if (!scan_cell<LK, kT64, SH>(list, sph4, sidv, start, count, J.nstructures, lo, hi, x, y, z, label, a, jx, jy, jz,
                             reach, J.S, oob, r)) {
      label = label_of<LK, SH>(list, sph4, sidv, J.rec_sid, start, count, J.nstructures, x, y, z, J.S, oob);
      if (kCheckBounds && (label < 0 || label > J.nstructures)) {
        oob = 1;
        label = J.nstructures;
      }
      if (LK) label_bounds(J, label, lo, hi);
      if (niter == 1) {  // the first draw's length depends on the label
        ds = sqrtf(2 * __ldg(J.D + label) * dt);
        ds_label = label;
        jump_of(J, wid, s, 0, ds, jx, jy, jz);
        a = jx * jx + jy * jy + jz * jz;
        reach = reach_of(a, jr);
      }
      // the full list: the near one was chosen for the old reach
      int fs, fc;
      cell_list(J, false, cell, fs, fc, oob);
      scan_cell<LK, kT64, SH>(LK ? J.idx : nullptr, LK ? J.rec4 : J.sph4, LK ? nullptr : J.sid, fs, fc, J.nstructures, lo,
                          hi, x, y, z, label, a, jx, jy, jz, reach, J.S, oob, r);
    }
    jc = ref_min(jc, r.any_in ? r.fin : kBig);
    jc = ref_min(jc, r.fout);
    x += jc * jx;
    y += jc * jy;
    z += jc * jz;
    // the next draw: the scatter draw of this step, or the first draw of the
    // next one; every iteration ends with one or the other, so one call site
    // serves all lanes of the warp
    int next_step = s, next_draw = draw;
    if (jc < jr) {
      jr = sqrtf(ref_max(0, jr * jr - jc * jc));
      if (MODE & NZ_MODE_SIG) sig *= t2_decay(-jc * jc * dt / __ldg(J.T2 + label));
      draw++;
    } else {
      jr -= jc;
      if (MODE & NZ_MODE_SIG) sig *= t2_decay(-jc * dt / __ldg(J.T2 + label));
    }
    if (!((jr > kTol) && (niter < kMaxIter))) {
      if (niter >= kMaxIter && jr > kTol) {
        float4* c = J.comp + w;
        c->w = __int_as_float(__float_as_int(c->w) | kFlagIterCap);
      }
      if (MODE & NZ_MODE_PHI) {
        const float G = __ldg(J.G + s);
        kahan_add(fx, kx, G * x);
        kahan_add(fy, ky, G * y);
        kahan_add(fz, kz, G * z);
      }
      const float Lx = J.g.Lx, Ly = J.g.Ly, Lz = J.g.Lz;
      if (fabsf(x) > Lx / 2 || fabsf(y) > Ly / 2 || fabsf(z) > Lz / 2) {  // rare: a wrap
        const float Ga = (MODE & NZ_MODE_PHI) ? __ldg(J.Garea + s) : 0.0f;
        float4 O = kOrig ? make_float4(x0, y0, z0, 0.f) : J.org[w];
        if (x < -Lx / 2) {
          x += Lx; O.x += Lx;
          if (MODE & NZ_MODE_PHI) kahan_add(fx, kx, Lx * Ga);
        } else if (x > Lx / 2) {
          x -= Lx; O.x -= Lx;
          if (MODE & NZ_MODE_PHI) kahan_add(fx, kx, -(Lx * Ga));
        }
        if (y < -Ly / 2) {
          y += Ly; O.y += Ly;
          if (MODE & NZ_MODE_PHI) kahan_add(fy, ky, Ly * Ga);
        } else if (y > Ly / 2) {
          y -= Ly; O.y -= Ly;
          if (MODE & NZ_MODE_PHI) kahan_add(fy, ky, -(Ly * Ga));
        }
        if (z < -Lz / 2) {
          z += Lz; O.z += Lz;
          if (MODE & NZ_MODE_PHI) kahan_add(fz, kz, Lz * Ga);
        } else if (z > Lz / 2) {
          z -= Lz; O.z -= Lz;
          if (MODE & NZ_MODE_PHI) kahan_add(fz, kz, -(Lz * Ga));
        }
        if (kOrig) {
          x0 = O.x; y0 = O.y; z0 = O.z;
        } else {
          J.org[w] = O;
        }
      }
      if (kDisp) {  // coalesced across the warp's walkers of one step
        const size_t N = size_t(J.nwalkers);
        float* d = J.disp + size_t(s - s0) * 3 * N;
        d[w] = x - x0;
        d[N + w] = y - y0;
        d[2 * N + w] = z - z0;
      }
      if (kMom) {  // nz_moments' terms: float displacement, squared in FP64
        const double ex = double(x - x0), ey = double(y - y0), ez = double(z - z0);
        double* m = s_mom + 6 * (s - s0);
        const double ex2 = ex * ex, ey2 = ey * ey, ez2 = ez * ez;
        atomicAdd(m + 0, ex2);
        atomicAdd(m + 1, ey2);
        atomicAdd(m + 2, ez2);
        atomicAdd(m + 3, ex2 * ex2);
        atomicAdd(m + 4, ey2 * ey2);
        atomicAdd(m + 5, ez2 * ez2);
      }
      s++;
      niter = 0;
      jr = 1.0f;
      draw = 1;
      next_step = s;
      next_draw = 0;
      if (label != ds_label) {
        ds = sqrtf(2 * __ldg(J.D + label) * dt);
        ds_label = label;
      }
      cell = step_cell(J, x, y, z, lox, loy, loz);
      cell_list(J, has_near, cell, pstart, pcount, oob);
    }
    if (s < s1) jump_of(J, wid, next_step, next_draw, ds, jx, jy, jz);
  }
  J.pos[w] = make_float4(x, y, z, __int_as_float(label));
  if (kOrig) J.org[w] = make_float4(x0, y0, z0, __uint_as_float(wid));
  if (MODE & (NZ_MODE_PHI | NZ_MODE_SIG)) J.phi[w] = make_float4(fx, fy, fz, sig);
  if (MODE & NZ_MODE_PHI) {
    float4* c = J.comp + w;
    *c = make_float4(kx, ky, kz, c->w);
  }
  if (kCheckBounds && oob) {
    float4* c = J.comp + w;
    c->w = __int_as_float(__float_as_int(c->w) | kFlagBounds);
  }
}

// One work item: walkers [first, first + count) of job J, steps [step0, step1)
// clamped to the job's protocol.
template <int MODE, int LK, bool SH>
__device__ __forceinline__ void run_item(const JobDev& J, int first, int count, int step0, int step1, double* s_mom,
                                         int flags = 0) {
  const int s0 = step0 + J.step_offset, s1 = min(step1 + J.step_offset, J.nsteps);
  if (MODE & NZ_MODE_MOMENTS) {
    for (int i = threadIdx.x; i < kMomentSteps * 6; i += blockDim.x) s_mom[i] = 0.0;
    __syncthreads();
  }
  if (threadIdx.x < count && s0 < s1) {
    walk_one<MODE, LK, SH>(J, first + threadIdx.x, s0, s1, s_mom);
    if (flags) {
      float4* c = J.comp + first + threadIdx.x;
      c->w = __int_as_float(__float_as_int(c->w) | flags);
    }
  }
  if (MODE & NZ_MODE_MOMENTS) {
    __syncthreads();
    if (J.moments)
      for (int i = threadIdx.x; i < (s1 - s0) * 6; i += blockDim.x)
        atomicAdd(J.moments + size_t(s0) * 6 + i, s_mom[i]);
    __syncthreads();
  }
}

// Staging a job's records into shared memory: one bulk copy (the TMA unit's
// cp.async.bulk, global -> shared) completing on an mbarrier.  Sizes are
// multiples of 16 bytes and both addresses 16-byte aligned (the host checks
// the records' address; s_stage is 16-byte aligned).  Every wait is bounded.
constexpr int kStageSpin = 1 << 20;  // try_wait polls before a copy is given up on

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.b32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  for (int i = 0; i < kStageSpin; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// Thread 0 only.  The CTA's generic-proxy reads of the previous contents of
// s_stage ended at a barrier before this call; the proxy fence orders them
// before the bulk copy's writes.
__device__ __forceinline__ void stage_records(uint32_t bar, const float4* src, uint32_t bytes) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(s_stage)),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// Work items are CTAs' worth of walkers of one job.  SINGLE: one job passed by
// value, item i = walkers [i*T, i*T + T).  Otherwise jobs and items come from
// device arrays; with queue != null the grid is persistent and each CTA takes
// items from *queue until none is left.
// STAGE (batched, index lists): a job whose S records fit in stage_cap
// records is walked with its records in shared memory (s_stage, stage_cap *
// 16 bytes of dynamic shared memory); the copy is made when a CTA's item
// belongs to a job other than the one already staged.  Larger jobs read
// their records from global memory as without STAGE.  The records are the
// same bytes either way, so the walk's results are identical.
#ifdef NZ_FUSED_MAXNREG
#define NZ_FUSED_BOUNDS __maxnreg__(NZ_FUSED_MAXNREG)
#else
#define NZ_FUSED_BOUNDS __launch_bounds__(kFusedMaxThreads, kFusedMinBlocks)
#endif
template <int MODE, int LK, bool SINGLE, bool STAGE>
__global__ void NZ_FUSED_BOUNDS
    walk_fused_kernel(const __grid_constant__ JobDev single, const nz_job* __restrict__ jobs,
                      const nz_item* __restrict__ items, int n_items, int step0, int step1, int* queue,
                      int stage_cap) {
  static_assert(!STAGE || (!SINGLE && LK != 0), "staging is for batched index-list walks");
  __shared__ int s_item;
  __shared__ double s_mom[(MODE & NZ_MODE_MOMENTS) ? kMomentSteps * 6 : 1];
  __shared__ JobDev s_job;
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ const float4* s_staged;  // the records now in s_stage (thread 0's bookkeeping)
  __shared__ int s_use, s_broken, s_pending;
  uint32_t phase = 0;  // parity of the barrier phase the next copy completes
  if (STAGE) {
    if (threadIdx.x == 0) {
      mbar_init(smem_addr(&s_bar));
      s_staged = nullptr;
      s_broken = s_pending = 0;
    }
    __syncthreads();
  }
  int it = blockIdx.x;
  for (;;) {
    if (queue) {
      if (threadIdx.x == 0) s_item = atomicAdd(queue, 1);
      __syncthreads();
      it = s_item;
      __syncthreads();
    }
    if (it >= n_items) {
      // a copy given up on may still be writing s_stage: wait for it (bounded)
      // before the CTA's shared memory is released
      if (STAGE && threadIdx.x == 0 && s_pending) mbar_wait_bounded(smem_addr(&s_bar), phase);
      return;
    }
    if (SINGLE) {
      const int first = it * int(blockDim.x);
      const int count = min(int(blockDim.x), single.nwalkers - first);
      run_item<MODE, LK, false>(single, first, count, step0, step1, s_mom);
    } else {
      // every thread of the CTA works on the same job: its descriptor lives
      // in shared memory, not in each thread's registers
      const nz_item wi = items[it];
      if (threadIdx.x == 0) {
        const nz_job& a = jobs[wi.job];
        s_job = make_job(a.sub, a.G, a.Garea, a.nsteps, a.dt, a.draws, a.mode, a.state, a.moments);
        s_job.step_offset = a.step_offset;
        if (STAGE) {
          const float4* src = s_job.rec4;
          const int S = s_job.S;
          int use = 0;
          if (!s_broken && S > 0 && S <= stage_cap && (reinterpret_cast<uintptr_t>(src) & 15) == 0) {
            if (src == s_staged) {
              use = 1;
            } else {
              stage_records(smem_addr(&s_bar), src, uint32_t(S) * 16u);
              s_pending = 1;
              use = 2;
            }
          }
          s_use = use;
        }
      }
      __syncthreads();
      if (STAGE) {
        int use = s_use;
        int flags = 0;
        if (use == 2) {
          // every thread observes the copy's completion on the barrier
          const bool done = mbar_wait_bounded(smem_addr(&s_bar), phase);
          const int late = __syncthreads_or(!done);
          if (late) {  // walk from global memory; stage nothing more
            use = 0;
            flags = kFlagStageTimeout;
            if (threadIdx.x == 0) {
              s_broken = 1;
              s_staged = nullptr;
            }
          } else {
            phase ^= 1u;
            if (threadIdx.x == 0) {
              s_staged = s_job.rec4;
              s_pending = 0;
            }
          }
        }
        if (use) run_item<MODE, LK, true>(s_job, wi.first, wi.count, step0, step1, s_mom);
        else run_item<MODE, LK, false>(s_job, wi.first, wi.count, step0, step1, s_mom, flags);
      } else {
        run_item<MODE, LK, false>(s_job, wi.first, wi.count, step0, step1, s_mom);
      }
      __syncthreads();
    }
    if (!queue) {
      if (STAGE && threadIdx.x == 0 && s_pending) mbar_wait_bounded(smem_addr(&s_bar), phase);
      return;
    }
  }
}

// ---------------------------------------------------------------------------
// packing between the reference layout and the fused state
// ---------------------------------------------------------------------------
__global__ void pack_kernel(nz_walkers wk, const uint32_t* __restrict__ ids, nz_state st) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= wk.N) return;
  const int N = wk.N;
  const int label = wk.label ? wk.label[w] : -1;
  reinterpret_cast<float4*>(st.pos)[w] =
      make_float4(wk.spins[w], wk.spins[N + w], wk.spins[2 * N + w], __int_as_float(label));
  reinterpret_cast<float4*>(st.org)[w] =
      make_float4(wk.spins0[w], wk.spins0[N + w], wk.spins0[2 * N + w], __uint_as_float(ids ? ids[w] : uint32_t(w)));
  float4 f = make_float4(0.f, 0.f, 0.f, wk.sig ? wk.sig[w] : 1.0f);
  float4 c = make_float4(0.f, 0.f, 0.f, __int_as_float(wk.flags ? wk.flags[w] : 0));
  if (wk.phi) {
    f.x = wk.phi[w]; f.y = wk.phi[N + w]; f.z = wk.phi[2 * N + w];
    c.x = wk.phi[3 * N + w]; c.y = wk.phi[4 * N + w]; c.z = wk.phi[5 * N + w];
  }
  reinterpret_cast<float4*>(st.phi)[w] = f;
  reinterpret_cast<float4*>(st.comp)[w] = c;
}

// by_id: walker w of the state goes to the reference-layout slot of its
// walker id (ids outside [0, N) are dropped and counted in *bad).
__global__ void unpack_kernel(nz_state st, nz_walkers wk, int by_id, int* bad) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= wk.N) return;
  int w = slot;
  if (by_id) {
    w = __float_as_int(reinterpret_cast<const float4*>(st.org)[slot].w);
    if (w < 0 || w >= wk.N) {
      if (bad) atomicAdd(bad, 1);
      return;
    }
  }
  const int N = wk.N;
  const float4 p = reinterpret_cast<const float4*>(st.pos)[slot];
  const float4 o = reinterpret_cast<const float4*>(st.org)[slot];
  const float4 f = reinterpret_cast<const float4*>(st.phi)[slot];
  const float4 c = reinterpret_cast<const float4*>(st.comp)[slot];
  wk.spins[w] = p.x; wk.spins[N + w] = p.y; wk.spins[2 * N + w] = p.z;
  wk.spins0[w] = o.x; wk.spins0[N + w] = o.y; wk.spins0[2 * N + w] = o.z;
  if (wk.label) wk.label[w] = __float_as_int(p.w);
  if (wk.sig) wk.sig[w] = f.w;
  if (wk.flags) wk.flags[w] = __float_as_int(c.w);
  if (wk.phi) {
    wk.phi[w] = f.x; wk.phi[N + w] = f.y; wk.phi[2 * N + w] = f.z;
    wk.phi[3 * N + w] = c.x; wk.phi[4 * N + w] = c.y; wk.phi[5 * N + w] = c.z;
  }
}

__host__ __device__ JobDev make_job(const nz_substrate& sub, const float* G, const float* Garea, int nsteps, float dt,
                                    const nz_draws& d, int mode, const nz_state& st, double* moments) {
  JobDev j;
  j.nwalkers = st.N;
  j.step_offset = 0;
  j.g = Grid{sub.grid.Lx, sub.grid.Ly, sub.grid.Lz, sub.grid.dLx, sub.grid.dLy, sub.grid.dLz,
             float(sub.grid.nx), float(sub.grid.ny), float(sub.grid.nz)};
  j.idLx = 1.0f / sub.grid.dLx;
  j.idLy = 1.0f / sub.grid.dLy;
  j.idLz = 1.0f / sub.grid.dLz;
  j.nstructures = sub.nstructures;
  j.sph4 = reinterpret_cast<const float4*>(sub.cell_sph4);
  j.sid = sub.cell_sid;
  j.cell_start = sub.cell_start;
  j.cell_count = sub.cell_count;
  j.near_margin = sub.near_margin;
  j.near_cut = (sub.near_margin - kTol - 2e-3f) / 1.02f;
  j.near_start = sub.near_start;
  j.near_count = sub.near_count;
  j.near_sph4 = reinterpret_cast<const float4*>(sub.near_sph4);
  j.near_sid = sub.near_sid;
  j.idx = sub.idx_bytes ? sub.cell_idx : nullptr;
  j.near_idx = sub.idx_bytes ? sub.near_idx : nullptr;
  j.rec4 = reinterpret_cast<const float4*>(sub.rec4);
  j.rec_sid = sub.rec_sid;
  j.sid_start = sub.sid_start;
  j.S = sub.S;
  j.ncell = sub.grid.nx * sub.grid.ny * sub.grid.nz;
  j.n_items = sub.n_items;
  j.near_items = sub.near_items;
  j.D = sub.D;
  j.T2 = sub.T2;
  j.G = G;
  j.Garea = Garea;
  j.nsteps = nsteps;
  j.dt = dt;
  j.key0 = d.key0;
  j.key1 = d.key1;
  j.stream = d.stream;
  j.mode = mode;
  j.pos = reinterpret_cast<float4*>(st.pos);
  j.org = reinterpret_cast<float4*>(st.org);
  j.phi = reinterpret_cast<float4*>(st.phi);
  j.comp = reinterpret_cast<float4*>(st.comp);
  j.moments = moments;
  j.disp = nullptr;
  return j;
}

// Dynamic shared memory of the staged kernel for stage_cap records, after
// setting its attributes: the largest allowed size (once per device) and a
// carveout that leaves room for the CTAs the register budget allows at this
// CTA size, the rest staying L1.
template <int MODE, int LK>
size_t stage_setup(int stage_cap, int threads) {
  const size_t bytes = size_t(stage_cap) * 16;
  if (LK == 0 || stage_cap <= 0) return 0;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < kMaxDevices) {
    static std::once_flag once[kMaxDevices];
    std::call_once(once[dev], [] {
      cudaFuncSetAttribute(walk_fused_kernel<MODE, LK, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           kMaxStageRecords * 16);
    });
  }
  const int ctas = std::max(1, kFusedMinBlocks * kFusedMaxThreads / threads);
  const size_t need = size_t(ctas) * (bytes + 2048);
  const int pct = int(std::min<size_t>(100, (100 * need + kSmemPerSm - 1) / kSmemPerSm));
  cudaFuncSetAttribute(walk_fused_kernel<MODE, LK, false, true>, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
  return bytes;
}

template <int MODE, int LK>
void launch_mode(const JobDev& single, const nz_job* jobs, const nz_item* items, int n_items, int step0, int step1,
                 int* queue, int grid, int threads, int stage_cap, cudaStream_t st) {
  // the kernel keeps little in shared memory: prefer the whole carveout for
  // L1.  Function attributes belong to a device's context, so this is done
  // once per device (and once across threads).
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < kMaxDevices) {
    static std::once_flag once[kMaxDevices];
    std::call_once(once[dev], [] {
      cudaFuncSetAttribute(walk_fused_kernel<MODE, LK, false, false>, cudaFuncAttributePreferredSharedMemoryCarveout,
                           0);
      cudaFuncSetAttribute(walk_fused_kernel<MODE, LK, true, false>, cudaFuncAttributePreferredSharedMemoryCarveout,
                           0);
    });
  }
  if constexpr (LK != 0) {
    if (jobs && stage_cap > 0) {
      const size_t smem = stage_setup<MODE, LK>(stage_cap, threads);
      walk_fused_kernel<MODE, LK, false, true>
          <<<grid, threads, smem, st>>>(single, jobs, items, n_items, step0, step1, queue, stage_cap);
      return;
    }
  }
  if (jobs)
    walk_fused_kernel<MODE, LK, false, false>
        <<<grid, threads, 0, st>>>(single, jobs, items, n_items, step0, step1, queue, 0);
  else
    walk_fused_kernel<MODE, LK, true, false>
        <<<grid, threads, 0, st>>>(single, jobs, items, n_items, step0, step1, queue, 0);
}

template <int LK>
int launch_lk(int mode, const JobDev& single, const nz_job* jobs, const nz_item* items, int n_items, int step0,
              int step1, int* queue, int grid, int threads, int stage_cap, cudaStream_t st) {
#define NZ_LAUNCH(M) \
  launch_mode<(M), LK>(single, jobs, items, n_items, step0, step1, queue, grid, threads, stage_cap, st)
  switch (mode & (NZ_MODE_PHI | NZ_MODE_SIG | NZ_MODE_MOMENTS | NZ_MODE_TANGENT64 | kModeDisp)) {
    case NZ_MODE_PHI | NZ_MODE_TANGENT64: NZ_LAUNCH(NZ_MODE_PHI | NZ_MODE_TANGENT64); break;
    case NZ_MODE_PHI | NZ_MODE_SIG | NZ_MODE_TANGENT64: NZ_LAUNCH(NZ_MODE_PHI | NZ_MODE_SIG | NZ_MODE_TANGENT64); break;
    case NZ_MODE_PHI: NZ_LAUNCH(NZ_MODE_PHI); break;
    case NZ_MODE_SIG: NZ_LAUNCH(NZ_MODE_SIG); break;
    case NZ_MODE_PHI | NZ_MODE_SIG: NZ_LAUNCH(NZ_MODE_PHI | NZ_MODE_SIG); break;
    case NZ_MODE_SIG | NZ_MODE_MOMENTS: NZ_LAUNCH(NZ_MODE_SIG | NZ_MODE_MOMENTS); break;
    case NZ_MODE_MOMENTS: NZ_LAUNCH(NZ_MODE_MOMENTS); break;
    case NZ_MODE_SIG | kModeDisp: NZ_LAUNCH(NZ_MODE_SIG | kModeDisp); break;
    case kModeDisp: NZ_LAUNCH(kModeDisp); break;
    case 0: NZ_LAUNCH(0); break;
    default: return set_error(NZ_ERR_ARG, "fused walk: unsupported mode %d", mode);
  }
#undef NZ_LAUNCH
  return check_launch("walk_fused_kernel");
}

// jobs == null: the single job `single` with n_items CTAs of kFusedThreads walkers.
// stage_cap > 0 (batched index-list walks): stage the records of jobs of at
// most stage_cap records in shared memory.
int launch_fused(int mode, int lk, const JobDev& single, const nz_job* jobs, const nz_item* items, int n_items,
                 int step0, int step1, int* queue, int grid, int threads, cudaStream_t st, int stage_cap) {
  switch (lk) {
    case 0: return launch_lk<0>(mode, single, jobs, items, n_items, step0, step1, queue, grid, threads, 0, st);
    case 2:
      return launch_lk<2>(mode, single, jobs, items, n_items, step0, step1, queue, grid, threads, stage_cap, st);
    case 4:
      return launch_lk<4>(mode, single, jobs, items, n_items, step0, step1, queue, grid, threads, stage_cap, st);
    default: return set_error(NZ_ERR_ARG, "fused walk: list kind %d is not 0, 2 or 4", lk);
  }
}

template <int MODE, int LK>
cudaError_t occupancy_mode(int threads, int stage_cap, int* blocks_per_sm) {
  if constexpr (LK != 0) {
    if (stage_cap > 0) {
      const size_t smem = stage_setup<MODE, LK>(stage_cap, threads);
      return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, walk_fused_kernel<MODE, LK, false, true>,
                                                           threads, smem);
    }
  }
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, walk_fused_kernel<MODE, LK, false, false>,
                                                       threads, 0);
}

template <int LK>
cudaError_t occupancy_lk(int mode, int threads, int stage_cap, int* blocks_per_sm) {
  switch (mode & (NZ_MODE_PHI | NZ_MODE_SIG | NZ_MODE_MOMENTS)) {
    case NZ_MODE_PHI: return occupancy_mode<NZ_MODE_PHI, LK>(threads, stage_cap, blocks_per_sm);
    case NZ_MODE_SIG: return occupancy_mode<NZ_MODE_SIG, LK>(threads, stage_cap, blocks_per_sm);
    case NZ_MODE_PHI | NZ_MODE_SIG: return occupancy_mode<NZ_MODE_PHI | NZ_MODE_SIG, LK>(threads, stage_cap, blocks_per_sm);
    default: return cudaErrorInvalidValue;
  }
}

int occupancy_fused(int mode, int lk, int threads, int* blocks_per_sm, int stage_cap) {
  const int m = mode & (NZ_MODE_PHI | NZ_MODE_SIG | NZ_MODE_MOMENTS);
  if (m != NZ_MODE_PHI && m != NZ_MODE_SIG && m != (NZ_MODE_PHI | NZ_MODE_SIG))
    return set_error(NZ_ERR_ARG, "occupancy: unsupported batch mode %d", mode);
  cudaError_t e;
  switch (lk) {
    case 0: e = occupancy_lk<0>(mode, threads, 0, blocks_per_sm); break;
    case 2: e = occupancy_lk<2>(mode, threads, stage_cap, blocks_per_sm); break;
    case 4: e = occupancy_lk<4>(mode, threads, stage_cap, blocks_per_sm); break;
    default: return set_error(NZ_ERR_ARG, "occupancy: list kind %d is not 0, 2 or 4", lk);
  }
  if (e != cudaSuccess) return set_error(NZ_ERR_CUDA, "occupancy: %s", cudaGetErrorString(e));
  return NZ_OK;
}

}  // namespace nz
