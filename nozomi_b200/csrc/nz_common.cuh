// Shared device code of the nozomi_b200 spin-walk library (sm_100a).
//
// The whole library is compiled with --fmad=false: an expression is rounded
// operation by operation in source order, as the reference kernel source
// reads, and a fused multiply-add appears only where __fmaf_rn is written.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace nz {

// Collision tolerance and "no hit" fraction of the reference kernel
// (simulation_toolkit/simulation_engine/sim3d_kernel.cu:34-35).
constexpr float kTol = 1e-4f;
constexpr float kBig = 1e6f;
constexpr int kMaxIter = 100;  // sim3d_kernel.cu:760

// Per-walker flag bits (the library's error/diagnostic word).
enum : int {
  kFlagDrawsExhausted = 1,  // injected normal table ran out; the draw read 0
  kFlagIterCap = 2,         // a step ended at the 100-iteration cap
  kFlagUnseeded = 4,        // seeding gave up after its round limit
  kFlagBounds = 8,          // bounds-checked build: an index was out of range and its access skipped
  kFlagStageTimeout = 16,   // staged walk: the record copy into shared memory did not complete in time;
                            // the walker read its records from global memory instead (results unchanged)
};

// The bounds-checked build (-DNZ_DEBUG_BOUNDS=1, libnozomi_b200_debug.so):
// cell indices, list ranges and sphere / record indices are checked before
// they are used; an index out of range sets kFlagBounds and its access is
// skipped.  Nothing traps.  The default build checks nothing.
#ifndef NZ_DEBUG_BOUNDS
#define NZ_DEBUG_BOUNDS 0
#endif
constexpr bool kCheckBounds = NZ_DEBUG_BOUNDS != 0;

// MIN / MAX exactly as the reference macros (sim3d_kernel.cu:7-8), NaN
// behaviour included.
__device__ __forceinline__ float ref_min(float a, float b) { return (a > b) ? b : a; }
__device__ __forceinline__ float ref_max(float a, float b) { return (a < b) ? b : a; }

// ---------------------------------------------------------------------------
// Counter-based draws.  Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11),
// Box-Muller on two 32-bit words, ln by the atanh series after splitting the
// binary exponent, sin/cos of |y| <= pi/4 by Taylor series.  Only IEEE
// single add/mul/fma/div/sqrt and integer operations: the same bits on any
// IEEE machine.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void philox4x32_10(uint32_t& c0, uint32_t& c1, uint32_t& c2, uint32_t& c3,
                                              uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int round = 0; round < 10; ++round) {
    const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
    const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

__device__ __forceinline__ float log_series(float x) {  // x in (0, 1], normal
  const uint32_t i = __float_as_uint(x);
  int e = int((i >> 23) & 0xffu) - 127;
  float m = __uint_as_float((i & 0x007fffffu) | 0x3f800000u);
  if (m > __uint_as_float(0x3fb504f3u)) {  // sqrt(2)
    m = m * 0.5f;
    e += 1;
  }
  const float s = (m - 1.0f) / (m + 1.0f);
  const float s2 = s * s;
  float p = __fmaf_rn(s2, __uint_as_float(0x3de38e39u), __uint_as_float(0x3e124925u));  // 1/9, 1/7
  p = __fmaf_rn(s2, p, __uint_as_float(0x3e4ccccdu));                                   // 1/5
  p = __fmaf_rn(s2, p, __uint_as_float(0x3eaaaaabu));                                   // 1/3
  p = __fmaf_rn(s2, p, 1.0f);
  const float lm = (2.0f * s) * p;
  return __fmaf_rn(__int2float_rn(e), __uint_as_float(0x3f317218u), lm);  // ln 2
}

__device__ __forceinline__ void box_muller(uint32_t ua, uint32_t ub, float& n0, float& n1) {
  const float u = __fmaf_rn(__uint2float_rn(ua), __uint_as_float(0x2f800000u), __uint_as_float(0x2f000000u));
  const float rad = sqrtf(-2.0f * log_series(u));
  const uint32_t q = ub >> 30;
  const float t = __fmaf_rn(__uint2float_rn(ub & 0x3fffffffu), __uint_as_float(0x30800000u), -0.5f);
  const float y = t * __uint_as_float(0x3fc90fdbu);  // pi/2
  const float y2 = y * y;
  float sp = __fmaf_rn(y2, __uint_as_float(0x3638ef1du), __uint_as_float(0xb9500d01u));  // 1/9!, -1/7!
  sp = __fmaf_rn(y2, sp, __uint_as_float(0x3c088889u));                                   // 1/5!
  sp = __fmaf_rn(y2, sp, __uint_as_float(0xbe2aaaabu));                                   // -1/3!
  const float sn = __fmaf_rn(y * y2, sp, y);
  float cp = __fmaf_rn(y2, __uint_as_float(0xb493f27eu), __uint_as_float(0x37d00d01u));  // -1/10!, 1/8!
  cp = __fmaf_rn(y2, cp, __uint_as_float(0xbab60b61u));                                   // -1/6!
  cp = __fmaf_rn(y2, cp, __uint_as_float(0x3d2aaaabu));                                   // 1/4!
  cp = __fmaf_rn(y2, cp, -0.5f);
  const float cs = __fmaf_rn(y2, cp, 1.0f);
  float c, s;
  switch (q) {
    case 0: c = cs; s = sn; break;
    case 1: c = -sn; s = cs; break;
    case 2: c = -cs; s = -sn; break;
    default: c = sn; s = -cs; break;
  }
  n0 = rad * c;
  n1 = rad * s;
}

// Three normals of draw `draw` of walker `walker` in time step `step`.
__device__ __forceinline__ void philox_normal3(uint32_t k0, uint32_t k1, uint32_t stream, uint32_t walker,
                                               uint32_t step, uint32_t draw, float& n0, float& n1,
                                               float& n2) {
  uint32_t c0 = walker, c1 = step, c2 = draw, c3 = stream;
  philox4x32_10(c0, c1, c2, c3, k0, k1);
  float unused;
  box_muller(c0, c1, n0, n1);
  box_muller(c2, c3, n2, unused);
}

// Three uniforms in [0, 1) (24-bit) for seeding round `round`.
__device__ __forceinline__ void philox_uniform3(uint32_t k0, uint32_t k1, uint32_t stream, uint32_t walker,
                                                uint32_t round, float& u0, float& u1, float& u2) {
  uint32_t c0 = walker, c1 = round, c2 = 0u, c3 = stream;
  philox4x32_10(c0, c1, c2, c3, k0, k1);
  const float s = __uint_as_float(0x33800000u);  // 2^-24
  u0 = __uint2float_rn(c0 >> 8) * s;
  u1 = __uint2float_rn(c1 >> 8) * s;
  u2 = __uint2float_rn(c2 >> 8) * s;
}

// Where a walk takes its normal draws from.
struct Draws {
  const float* table;  // injected: [N][nsteps][maxk], null for Philox
  int nsteps, maxk;
  uint32_t key0, key1, stream;
};

__device__ __forceinline__ void draw3(const Draws& d, uint32_t walker, int step, int draw, float& n0, float& n1,
                                      float& n2, int& flags) {
  if (d.table == nullptr) {
    philox_normal3(d.key0, d.key1, d.stream, walker, uint32_t(step), uint32_t(draw), n0, n1, n2);
    return;
  }
  float v[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const int k = 3 * draw + i;
    if (step < 0 || step >= d.nsteps || k >= d.maxk) {
      v[i] = 0.0f;
      flags |= kFlagDrawsExhausted;
    } else {
      v[i] = d.table[(size_t(walker) * d.nsteps + step) * d.maxk + k];
    }
  }
  n0 = v[0];
  n1 = v[1];
  n2 = v[2];
}

// ---------------------------------------------------------------------------
// Box and cell grid, as the reference kernel's template constants
// (sim3d_kernel.cu:11-28): floats, cell counts included.
// ---------------------------------------------------------------------------
struct Grid {
  float Lx, Ly, Lz;
  float dLx, dLy, dLz;
  float nLx, nLy, nLz;
};

// Cell of a position: clamped floor, idxSeg = iz*nx*ny + iy*nx + ix evaluated
// in float as sim3d_kernel.cu:754-756 does.
__device__ __forceinline__ int cell_of(const Grid& g, float x, float y, float z, float& fx, float& fy, float& fz) {
  fz = ref_min(g.nLz - 1, ref_max(0, floorf((z + g.Lz / 2) / g.dLz)));
  fy = ref_min(g.nLy - 1, ref_max(0, floorf((y + g.Ly / 2) / g.dLy)));
  fx = ref_min(g.nLx - 1, ref_max(0, floorf((x + g.Lx / 2) / g.dLx)));
  return int(fz * g.nLx * g.nLy + fy * g.nLx + fx);
}
__device__ __forceinline__ int cell_of(const Grid& g, float x, float y, float z) {
  float fx, fy, fz;
  return cell_of(g, x, y, z, fx, fy, fz);
}

// ---------------------------------------------------------------------------
// The reference's ray-sphere rule (sim3d_kernel.cu:72-160).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float inside_test(float dx, float dy, float dz, float r) {
  return dx * dx + dy * dy + dz * dz - r * r;
}

// Root pair of the stable quadratic.  The reference forms q in double and
// rounds it to float; -0.5f*(b +/- s) in float rounds to the same value
// (the double sum of two floats is exact unless one is below 2^-28 of the
// other, where both roundings return the larger; halving is exact).
__device__ __forceinline__ void roots(float a, float b, float c, float sq, float& fpos, float& fneg) {
  float q = -0.5f * (b + sq);
  if (b < 0) q = -0.5f * (b - sq);
  fpos = q / a;
  fneg = c / q;
}

// findStepSizeToSphereInsideTol for a walker known to be inside (the early
// "outside" return of :82-83 cannot fire).
__device__ __forceinline__ float step_in(float dx, float dy, float dz, float r, float a, float jx, float jy,
                                         float jz) {
  const float b = 2 * (jx * dx + jy * dy + jz * dz);
  const float c = dx * dx + dy * dy + dz * dz - (r - kTol) * (r - kTol);
  float sq = b * b - 4 * a * c;
  if (sq < 0) return 0;
  sq = sqrtf(sq);
  float fpos, fneg;
  roots(a, b, c, sq, fpos, fneg);
  return ref_max(ref_max(fpos, fneg), 0);
}

// findStepSizeToSphereOutsideTol for a walker known to be outside the sphere
// (the "inside" branch of :141-145 cannot fire).
__device__ __forceinline__ float step_out(float dx, float dy, float dz, float r, float a, float jx, float jy,
                                          float jz) {
  const float b = 2 * (jx * dx + jy * dy + jz * dz);
  const float c = dx * dx + dy * dy + dz * dz - (r + kTol) * (r + kTol);
  float sq = b * b - 4 * a * c;
  if (sq < 0) return kBig;
  sq = sqrtf(sq);
  float fpos, fneg;
  roots(a, b, c, sq, fpos, fneg);
  if (fpos > 0 && fneg > 0) return ref_min(fpos, fneg);
  else if ((fpos < 0 && fneg < 0) || (b > 0)) return kBig;
  return 0;
}

// step_in (inside) or step_out (outside) as one instruction stream: the two
// differ only in r -/+ tol and in how the roots are read, so lanes of a warp
// taking different sides share the arithmetic instead of running both
// branches.  Every operation is the one step_in / step_out performs, on the
// same operands, so the results are theirs bit for bit.
__device__ __forceinline__ float step_either(bool inside, float dx, float dy, float dz, float r, float a, float jx,
                                             float jy, float jz) {
  const float rt = inside ? r - kTol : r + kTol;
  const float b = 2 * (jx * dx + jy * dy + jz * dz);
  const float c = dx * dx + dy * dy + dz * dz - rt * rt;
  const float sq0 = b * b - 4 * a * c;
  const bool miss = sq0 < 0;
  const float sq = sqrtf(miss ? 0.0f : sq0);
  float fpos, fneg;
  roots(a, b, c, sq, fpos, fneg);
  float f;
  if (inside) {
    f = ref_max(ref_max(fpos, fneg), 0);
  } else if (fpos > 0 && fneg > 0) {
    f = ref_min(fpos, fneg);
  } else {
    f = ((fpos < 0 && fneg < 0) || (b > 0)) ? kBig : 0.0f;
  }
  return miss ? (inside ? 0.0f : kBig) : f;
}

// The T2 weight exp(x) of sim3d_kernel.cu:473/485 for a float argument,
// evaluated in double and rounded once to float: the correctly rounded value
// in all but rare double-rounding cases, so it agrees with any correctly
// rounding host expf and does not drift over many steps.
__device__ __forceinline__ float t2_decay(float x) { return float(exp(double(x))); }

// FP64 forms of the two fractions, for near-tangent rays (the chosen
// precision form): the same rule evaluated in double from the float inputs.
__device__ __forceinline__ double step_in_f64(double dx, double dy, double dz, double r, double jx, double jy,
                                              double jz) {
  const double tol = double(kTol);
  if ((dx * dx + dy * dy + dz * dz - r * r) > 0) return 1e6;  // the inside test, redone in double
  const double a = jx * jx + jy * jy + jz * jz;
  const double b = 2 * (jx * dx + jy * dy + jz * dz);
  const double c = dx * dx + dy * dy + dz * dz - (r - tol) * (r - tol);
  double sq = b * b - 4 * a * c;
  if (sq < 0) return 0;
  sq = sqrt(sq);
  double q = -0.5 * (b + sq);
  if (b < 0) q = -0.5 * (b - sq);
  const double fpos = q / a, fneg = c / q;
  const double m = (fpos < fneg) ? fneg : fpos;
  return (m < 0) ? 0 : m;
}
__device__ __forceinline__ double step_out_f64(double dx, double dy, double dz, double r, double jx, double jy,
                                               double jz) {
  const double tol = double(kTol);
  const double a = jx * jx + jy * jy + jz * jz;
  const double b = 2 * (jx * dx + jy * dy + jz * dz);
  const double c = dx * dx + dy * dy + dz * dz - (r + tol) * (r + tol);
  double sq = b * b - 4 * a * c;
  if (sq < 0) return 1e6;
  sq = sqrt(sq);
  double q = -0.5 * (b + sq);
  if (b < 0) q = -0.5 * (b - sq);
  const double fpos = q / a, fneg = c / q;
  if ((dx * dx + dy * dy + dz * dz - r * r) < 0) return (fpos < fneg) ? fneg : fpos;  // inside, in double
  if (fpos > 0 && fneg > 0) return (fpos > fneg) ? fneg : fpos;
  else if ((fpos < 0 && fneg < 0) || (b > 0)) return 1e6;
  return 0;
}

// The reference fractions with the near-tangent FP64 form when T64.
template <bool T64>
__device__ __forceinline__ float step_in_t(float dx, float dy, float dz, float r, float a, float jx, float jy,
                                           float jz) {
  if (T64) {
    const float b = 2 * (jx * dx + jy * dy + jz * dz);
    const float c = dx * dx + dy * dy + dz * dz - (r - kTol) * (r - kTol);
    const float sq = b * b - 4 * a * c;
    if (sq < __uint_as_float(0x368637bdu) * a) return float(step_in_f64(dx, dy, dz, r, jx, jy, jz));  // 4e-6
  }
  return step_in(dx, dy, dz, r, a, jx, jy, jz);
}
template <bool T64>
__device__ __forceinline__ float step_out_t(float dx, float dy, float dz, float r, float a, float jx, float jy,
                                            float jz) {
  if (T64) {
    const float b = 2 * (jx * dx + jy * dy + jz * dz);
    const float c = dx * dx + dy * dy + dz * dz - (r + kTol) * (r + kTol);
    const float sq = b * b - 4 * a * c;
    if (sq < __uint_as_float(0x368637bdu) * a) return float(step_out_f64(dx, dy, dz, r, jx, jy, jz));  // 4e-6
  }
  return step_out(dx, dy, dz, r, a, jx, jy, jz);
}

template <bool T64>
__device__ __forceinline__ float step_either_t(bool inside, float dx, float dy, float dz, float r, float a, float jx,
                                               float jy, float jz) {
  if (T64) {
    const float rt = inside ? r - kTol : r + kTol;
    const float b = 2 * (jx * dx + jy * dy + jz * dz);
    const float c = dx * dx + dy * dy + dz * dz - rt * rt;
    const float sq = b * b - 4 * a * c;
    if (sq < __uint_as_float(0x368637bdu) * a)  // 4e-6
      return float(inside ? step_in_f64(dx, dy, dz, r, jx, jy, jz) : step_out_f64(dx, dy, dz, r, jx, jy, jz));
  }
  return step_either(inside, dx, dy, dz, r, a, jx, jy, jz);
}

// Kahan-compensated accumulation.
__device__ __forceinline__ void kahan_add(float& sum, float& comp, float term) {
  const float yk = term - comp;
  const float t = sum + yk;
  comp = (t - sum) - yk;
  sum = t;
}

}  // namespace nz
