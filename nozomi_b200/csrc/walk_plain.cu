// Plain walk kernel: one time step per launch, one thread per walker, walker
// state in HBM in the reference's layout (spins [3,N], spins0 [3,N],
// phase [ndir,N], sig [N]).  It is the drop-in for the reference's
// randomWalk3d (sim3d_kernel.cu:340-522), randomWalk3d_phase (:524-717) and
// randomWalk3d_phase_multidirr (:719-943) and the per-substrate baseline that
// the fused and batched paths are measured against.
//
// Differences from the reference kernel that do not change any result:
// a bounds guard (the reference needs N to be a multiple of its 1000-thread
// block), counter-based draws instead of a 48-byte cuRAND state per walker,
// compact cell lists (start, count) in place of the padded table (the padded
// table is the case start = c*K, count = K), runtime geometry instead of
// compile-time constants.
#include "kernels.cuh"

namespace nz {


__global__ void __launch_bounds__(256) walk_plain_kernel(const PlainArgs a) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= a.N) return;
  const int S = a.S, N = a.N;
  const float* __restrict__ cx = a.spheres;
  const float* __restrict__ cy = a.spheres + S;
  const float* __restrict__ cz = a.spheres + 2 * S;
  const float* __restrict__ rr = a.spheres + 3 * S;
  const float* __restrict__ sphSID = a.spheres + 4 * S;

  float x = a.spins[w], y = a.spins[N + w], z = a.spins[2 * N + w];
  int flags = a.flags ? a.flags[w] : 0;
  float sig = (a.mode & NZ_MODE_SIG) ? a.sig[w] : 1.0f;

  float ds = 0, jx = 0, jy = 0, jz = 0;
  float jump_current, jump_remaining = 1.0f;

  const int idxSeg = cell_of(a.g, x, y, z);
  int start = 0, count = 0;
  if (!kCheckBounds || (idxSeg >= 0 && idxSeg < a.ncell)) {
    start = __ldg(a.cell_start + idxSeg);
    count = __ldg(a.cell_count + idxSeg);
  } else {
    flags |= kFlagBounds;
  }
  if (kCheckBounds && (start < 0 || count < 0 || (a.n_items > 0 && start + count > a.n_items))) {
    flags |= kFlagBounds;
    start = count = 0;
  }
  const int* __restrict__ items = a.cell_items + start;

  int niter = 0, nscatter = 0, draw = 0;
  int spinSID = a.nstructures;
  while ((jump_remaining > kTol) && (niter < kMaxIter)) {
    niter++;
    jump_current = jump_remaining;

    // label: lowest structure id among the spheres containing the walker
    spinSID = a.nstructures;
    for (int n = 0; n < count; n++) {
      const int s = __ldg(items + n);
      if (kCheckBounds && (s < 0 || s >= S)) {
        flags |= kFlagBounds;
        continue;
      }
      const float sid = __ldg(sphSID + s);
      if (sid < spinSID) {
        const float isIn = inside_test(x - __ldg(cx + s), y - __ldg(cy + s), z - __ldg(cz + s), __ldg(rr + s));
        if (isIn < 0) spinSID = int(sid);
      }
    }
    if (kCheckBounds && (spinSID < 0 || spinSID > a.nstructures)) {
      flags |= kFlagBounds;
      spinSID = a.nstructures;
    }

    if (niter == 1) {
      float n0, n1, n2;
      draw3(a.draws, uint32_t(w), a.step, draw++, n0, n1, n2, flags);
      ds = sqrtf(2 * __ldg(a.D + spinSID) * a.dt);
      jx = ds * n0;
      jy = ds * n1;
      jz = ds * n2;
    }

    const float aa = jx * jx + jy * jy + jz * jz;
    float isInsideAny = 0;
    float furthest_fstep_in = 0;
    float closest_fstep_out = kBig;
    for (int n = 0; n < count; n++) {
      const int s = __ldg(items + n);
      if (kCheckBounds && (s < 0 || s >= S)) continue;  // flagged in the label pass
      const float sid = __ldg(sphSID + s);
      if (sid > spinSID) continue;
      const float dx = x - __ldg(cx + s), dy = y - __ldg(cy + s), dz = z - __ldg(cz + s);
      const float r = __ldg(rr + s);
      const float isIn = inside_test(dx, dy, dz, r);
      if (isIn < 0) {
        isInsideAny = 1;
        const float f = step_in(dx, dy, dz, r, aa, jx, jy, jz);
        if (furthest_fstep_in < f) furthest_fstep_in = f;
      } else if (sid < spinSID) {
        const float f = step_out(dx, dy, dz, r, aa, jx, jy, jz);
        if (f < closest_fstep_out) closest_fstep_out = f;
      }
    }

    jump_current = ref_min(jump_current, isInsideAny ? furthest_fstep_in : kBig);
    jump_current = ref_min(jump_current, closest_fstep_out);
    x += jump_current * jx;
    y += jump_current * jy;
    z += jump_current * jz;

    if (jump_current < jump_remaining) {
      jump_remaining = sqrtf(ref_max(0, jump_remaining * jump_remaining - jump_current * jump_current));
      if (a.mode & NZ_MODE_SIG) sig *= t2_decay(-jump_current * jump_current * a.dt / __ldg(a.T2 + spinSID));
      float n0, n1, n2;
      draw3(a.draws, uint32_t(w), a.step, draw++, n0, n1, n2, flags);
      jx = ds * n0;
      jy = ds * n1;
      jz = ds * n2;
      nscatter++;
    } else {
      jump_remaining -= jump_current;
      if (a.mode & NZ_MODE_SIG) sig *= t2_decay(-jump_current * a.dt / __ldg(a.T2 + spinSID));
    }
  }
  if (niter >= kMaxIter && jump_remaining > kTol) flags |= kFlagIterCap;

  // phase of every direction from the post-step, pre-wrap position
  const int nd = a.ndir;
  if (a.mode & NZ_MODE_PHASE) {
    for (int d = 0; d < nd; ++d) {
      const float proj = x * __ldg(a.diffdir + d) + y * __ldg(a.diffdir + nd + d) + z * __ldg(a.diffdir + 2 * nd + d);
      a.phase[w + size_t(d) * N] += proj * a.G;
    }
  }
  float fx = 0, fy = 0, fz = 0, kx = 0, ky = 0, kz = 0;
  if (a.mode & NZ_MODE_PHI) {
    fx = a.phi[w]; fy = a.phi[N + w]; fz = a.phi[2 * N + w];
    kx = a.phi[3 * N + w]; ky = a.phi[4 * N + w]; kz = a.phi[5 * N + w];
    kahan_add(fx, kx, a.G * x);
    kahan_add(fy, ky, a.G * y);
    kahan_add(fz, kz, a.G * z);
  }

  // periodic wrap; spins0 and phase follow the walker
  const float Lx = a.g.Lx, Ly = a.g.Ly, Lz = a.g.Lz;
  if (x < -Lx / 2) {
    x += Lx; a.spins0[w] += Lx;
    if (a.mode & NZ_MODE_PHASE) for (int d = 0; d < nd; ++d) a.phase[w + size_t(d) * N] += Lx * __ldg(a.diffdir + d) * a.Garea;
    if (a.mode & NZ_MODE_PHI) kahan_add(fx, kx, Lx * a.Garea);
  } else if (x > Lx / 2) {
    x -= Lx; a.spins0[w] -= Lx;
    if (a.mode & NZ_MODE_PHASE) for (int d = 0; d < nd; ++d) a.phase[w + size_t(d) * N] -= Lx * __ldg(a.diffdir + d) * a.Garea;
    if (a.mode & NZ_MODE_PHI) kahan_add(fx, kx, -(Lx * a.Garea));
  }
  if (y < -Ly / 2) {
    y += Ly; a.spins0[N + w] += Ly;
    if (a.mode & NZ_MODE_PHASE) for (int d = 0; d < nd; ++d) a.phase[w + size_t(d) * N] += Ly * __ldg(a.diffdir + nd + d) * a.Garea;
    if (a.mode & NZ_MODE_PHI) kahan_add(fy, ky, Ly * a.Garea);
  } else if (y > Ly / 2) {
    y -= Ly; a.spins0[N + w] -= Ly;
    if (a.mode & NZ_MODE_PHASE) for (int d = 0; d < nd; ++d) a.phase[w + size_t(d) * N] -= Ly * __ldg(a.diffdir + nd + d) * a.Garea;
    if (a.mode & NZ_MODE_PHI) kahan_add(fy, ky, -(Ly * a.Garea));
  }
  if (z < -Lz / 2) {
    z += Lz; a.spins0[2 * N + w] += Lz;
    if (a.mode & NZ_MODE_PHASE) for (int d = 0; d < nd; ++d) a.phase[w + size_t(d) * N] += Lz * __ldg(a.diffdir + 2 * nd + d) * a.Garea;
    if (a.mode & NZ_MODE_PHI) kahan_add(fz, kz, Lz * a.Garea);
  } else if (z > Lz / 2) {
    z -= Lz; a.spins0[2 * N + w] -= Lz;
    if (a.mode & NZ_MODE_PHASE) for (int d = 0; d < nd; ++d) a.phase[w + size_t(d) * N] -= Lz * __ldg(a.diffdir + 2 * nd + d) * a.Garea;
    if (a.mode & NZ_MODE_PHI) kahan_add(fz, kz, -(Lz * a.Garea));
  }

  a.spins[w] = x;
  a.spins[N + w] = y;
  a.spins[2 * N + w] = z;
  if (a.mode & NZ_MODE_SIG) a.sig[w] = sig;
  if (a.mode & NZ_MODE_PHI) {
    a.phi[w] = fx; a.phi[N + w] = fy; a.phi[2 * N + w] = fz;
    a.phi[3 * N + w] = kx; a.phi[4 * N + w] = ky; a.phi[5 * N + w] = kz;
  }
  if (a.label) a.label[w] = spinSID;
  if (a.n_iter) a.n_iter[w] += niter;
  if (a.n_scatter) a.n_scatter[w] += nscatter;
  if (a.flags) a.flags[w] = flags;
}

}  // namespace nz
