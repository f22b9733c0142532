// Slope limiter of the second-order uncollided flux solveFlux!
// (code/SolverCSD.jl:288-293, used at :295-386), shared by the standalone
// operator titus_limited_flux and the RK4 ("HighOrder") DLR kernel.
//
// The arithmetic uses the _rn intrinsics in the reference's evaluation order
// (no FMA contraction), so a face value is the same IEEE double as the FP64
// restatement of the loop body.
#pragma once
#include <cuda_runtime.h>

namespace titus_lim {

// minmod(x, y) = x < 0 ? clamp(y, x, 0) : clamp(y, 0, x), where Julia's
// clamp(v, lo, hi) is v > hi ? hi : (v < lo ? lo : v)  (SolverCSD.jl:288).
__device__ __forceinline__ double minmod(double x, double y) {
    const double lo = x < 0.0 ? x : 0.0;
    const double hi = x < 0.0 ? 0.0 : x;
    return y > hi ? hi : (y < lo ? lo : y);
}

// slopefit(l, c, r) = minmod(2 (r - c), minmod((r - l) / 2, 2 (c - l)))  (:290-293)
__device__ __forceinline__ double slopefit(double l, double c, double r) {
    const double tmp = minmod(__dmul_rn(0.5, __dsub_rn(r, l)), __dmul_rn(2.0, __dsub_rn(c, l)));
    return minmod(__dmul_rn(2.0, __dsub_rn(r, c)), tmp);
}

// Face values. F+(a) = phi_a + slopefit(phi_{a-1}, phi_a, phi_{a+1})/2 is the
// face between cells a and a+1 for a component >= 0; F-(a) = phi_a -
// slopefit(phi_{a-1}, phi_a, phi_{a+1})/2 the face between a-1 and a for a
// negative one. The reference's difference for cell i is F+(i) - F+(i-1)
// (s1..s4 = offsets -2..+1, :309-331) or F-(i+1) - F-(i) (offsets -1..+2,
// :333-355).
__device__ __forceinline__ double face_pos(double m1, double c, double p1) {
    return __dadd_rn(c, __dmul_rn(0.5, slopefit(m1, c, p1)));
}
__device__ __forceinline__ double face_neg(double m1, double c, double p1) {
    return __dsub_rn(c, __dmul_rn(0.5, slopefit(m1, c, p1)));
}
// (face after the centre) - (face before it) along one axis from the five
// values at offsets -2..+2 (only -2..+1 are read for pos, -1..+2 otherwise)
__device__ __forceinline__ double axis_diff(double m2, double m1, double c, double p1, double p2, bool pos) {
    return pos ? __dsub_rn(face_pos(m1, c, p1), face_pos(m2, m1, c))
               : __dsub_rn(face_neg(c, p1, p2), face_neg(m1, c, p1));
}

}  // namespace titus_lim
