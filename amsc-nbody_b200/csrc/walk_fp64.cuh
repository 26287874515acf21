// walk_fp64.cuh -- FP64 interaction and acceptance test shared by the plain
// force walk, the frozen-structure replay and the adjoint walk, so all three
// take the same decisions on the same inputs.
#pragma once

#include "nbb_internal.cuh"

namespace nbb {

// barnes_hut.cu:56-80, the factor G m (d^2 + eps^2)^-3/2 with the
// reference's operation order.  The reference's 1.0 / sqrt(r2) is a
// correctly rounded division of 1, which is the correctly rounded reciprocal
// (__drcp_rn, a shorter sequence than the general division): the same bits
// for every input.  Returns false on a singular interaction.
__device__ __forceinline__ bool point_mass_factor(double d2, double m, double g, double soft2, double &f) {
  const double r2 = __dadd_rn(d2, soft2);
  const double inv = __drcp_rn(__dsqrt_rn(r2));
  const double inv3 = __dmul_rn(__dmul_rn(inv, inv), inv);
  f = __dmul_rn(__dmul_rn(g, m), inv3);
  return !(r2 <= 0.0);
}

// G m (d^2 + eps^2)^-3/2 d accumulated in the reference's order.  Returns
// false (and adds nothing) on a singular interaction.
__device__ __forceinline__ bool point_mass_fp64(double dx, double dy, double dz, double d2,
                                                double m, double g, double soft2, double &ax,
                                                double &ay, double &az) {
  double f;
  if (!point_mass_factor(d2, m, g, soft2, f)) return false;
  ax = __fma_rn(f, dx, ax);
  ay = __fma_rn(f, dy, ay);
  az = __fma_rn(f, dz, az);
  return true;
}

__device__ __forceinline__ double sqdist(double dx, double dy, double dz) {
  return __fma_rn(dz, dz, __fma_rn(dy, dy, __dmul_rn(dx, dx)));
}

// barnes_hut.cu:273-294: the acceptance test of target t at a node with
// records a = (com, mass), c = (crit, crit^2 band, box radius^2) and, at *bp,
// b = (centre, half size).  sqrt(d2) > crit is decided on d2 against crit^2
// outside a 2^-44 band and by the exact square root inside it; a node
// containing the target, or at zero distance, is never accepted.  Beyond the
// box radius (c.w: (max(crit, sqrt(3) h + |com - centre|) (1 + 2^-40))^2) no
// point of the cell lies, so the containment test can only fail there and b
// is read only inside it; the decisions are the reference's in every case.
// Returns the offset com - t and its square.
__device__ __forceinline__ bool accept_fp64(const double4 &a, const double4 *bp, const double4 &c,
                                            const double4 &t, double &dx, double &dy, double &dz,
                                            double &d2) {
  dx = __dsub_rn(a.x, t.x);
  dy = __dsub_rn(a.y, t.y);
  dz = __dsub_rn(a.z, t.z);
  d2 = sqdist(dx, dy, dz);
  bool accept = (d2 > c.z) ? true : (d2 < c.y) ? false : (__dsqrt_rn(d2) > c.x);
  if (accept && !(d2 > c.w)) {
    const double4 b = *bp;
    const bool contains = fabs(__dsub_rn(t.x, b.x)) <= b.w && fabs(__dsub_rn(t.y, b.y)) <= b.w &&
                          fabs(__dsub_rn(t.z, b.z)) <= b.w;
    accept = !contains && d2 > 0.0;
  }
  return accept;
}

}  // namespace nbb
