// physics.cuh -- pointwise pieces of calRHS shared by every stage kernel.
//
// The expressions keep the association of the reference (nuosc_class.cpp):
//   ADV_FD  (:180-183)  factor*((x[-2] - x[+2]) - 8*(x[-1] - x[+1])) per axis
//   KO_FD   (:112-123)  eps*(x[-3] + x[+3] - 6*(x[-2] + x[+2]) + 15*(x[-1] + x[+1]) - 20*x[0])
//                       or eps*(x[-2] + x[+2] - 4*(x[-1] + x[+1]) + 6*x[0])
//   I-terms (:187-200)  commutator with H(v) = mu * sum_v' w (1 - v.v') (rho - rho-bar)
//   vacuum  (:280-287)  pmo * [H_vac, rho] with theta = 37 degrees
// so the FP64 path differs from the reference only by FMA contraction and the
// summation order of the velocity moments.
#pragma once
#include "internal.cuh"

namespace nuosc {

// s[0..6] hold the field at offsets -3..+3 along one axis.
template <typename T>
__device__ __forceinline__ T adv_axis(const T (&s)[7], T factor) {
    return factor * ((s[1] - s[5]) - T(8.0) * (s[2] - s[4]));
}
template <typename T, bool KO6>
__device__ __forceinline__ T ko_axis(const T (&s)[7], T eps) {
    if (KO6) return eps * (s[0] + s[6] - T(6) * (s[1] + s[5]) + T(15) * (s[2] + s[4]) - T(20) * s[3]);
    return eps * (s[1] + s[5] - T(4) * (s[2] + s[4]) + T(6) * s[3]);
}

// Moment contraction INP(m) = m0 - m1 vx - m2 vy - m3 vz (nuosc_class.cpp:187), in double.
__device__ __forceinline__ double inp(const double *m, double vx, double vy, double vz) {
    return m[0] - m[1] * vx - m[2] * vy - m[3] * vz;
}

// s/3 + t, with s the 3U-sized sum B + Y4 of the 12-pass step's last stage and
// t the small dt/6 k4.  q = s * (1/3) carries the rounded constant's relative
// error (3e-8 in float) on the whole sum -- a bias that would grow U by that
// much every step --; the exact remainder r = s - 3q (one fma) restores
// s/3 = q + r/3, and the small terms are summed before the one rounding at
// U's size.
template <typename T>
__device__ __forceinline__ T third_plus(T s, T t) {
    const T q = s * T(1.0 / 3.0);
    const T r = fma(-q, T(3), s);
    return q + fma(r, T(1.0 / 3.0), t);
}

// Self-interaction and vacuum terms for one flavour half.  `c` holds the
// centre values (ee, mm, emr, emi) or (bee, bmm, bemr, bemi); `a`, `b`, `e`
// are INP(emRm), INP(emIp), INP(eemm).  Adds into out[0..3] (which hold
// ADV+KO on entry, so the sum order is I + ADV + KO + vacuum as in the
// reference where the vacuum term comes last).
template <typename T>
__device__ __forceinline__ void commutator_half(const T (&c)[4], T a, T b, T e, const Coeffs &k, T (&out)[4],
                                                T (&adv)[4], T (&ko)[4]) {
    const T mu = T(k.mu), pmo = T(k.pmo), ct = T(k.ct), st = T(k.st);
    const T ee = c[0], mm = c[1], emr = c[2], emi = c[3];
    const T Iee = T(2) * mu * (emi * a + emr * b);
    const T Iemr = -mu * ((ee - mm) * b + e * emi);
    const T Iemi = mu * ((mm - ee) * a + e * emr);
    out[0] = Iee + adv[0] + ko[0] - pmo * T(2) * st * emi;
    out[1] = -Iee + adv[1] + ko[1] + pmo * T(2) * st * emi;
    out[2] = Iemr + adv[2] + ko[2] - pmo * T(2) * ct * emi;
    out[3] = Iemi + adv[3] + ko[3] + pmo * (T(2) * ct * emr + st * (ee - mm));
}

// Moment contributions of one velocity of one flavour half (nuosc_class.cpp:69-71):
// neutrinos enter with sign -1, antineutrinos with +1.
//   emRm += v4 w (bemr - emr), emIp += v4 w (bemi + emi), eemm += v4 w (bee - bmm - ee + mm)
template <bool BAR>
__device__ __forceinline__ void moment_terms(double ee, double mm, double emr, double emi, double &d0, double &d1,
                                             double &d2) {
    if (BAR) { d0 = emr; d1 = emi; d2 = ee - mm; }
    else { d0 = -emr; d1 = emi; d2 = mm - ee; }
}

__device__ __forceinline__ int wrap_index(int a, int n) {
    a %= n;
    return a < 0 ? a + n : a;
}

}  // namespace nuosc
