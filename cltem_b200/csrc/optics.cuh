// optics.cuh — the aberration function of the reference's probe and objective-lens kernels (device).
#pragma once

#include "misc.cuh"

namespace ms {

__device__ __forceinline__ double cModSq(double2 a) { return (a.x * a.x + a.y * a.y); }
__device__ __forceinline__ double2 cConj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cPow(double2 a, int n) {
    double2 temp = a;
    for (int j = 1; j < n; j++) temp = cmul(temp, a);
    return temp;
}
__device__ __forceinline__ double2 sc(double2 a, double s) { return make_double2(s * a.x, s * a.y); }
__device__ __forceinline__ double2 dv(double2 a, double s) { return make_double2(a.x / s, a.y / s); }

// the aberration function sum cchi (init_probe_wave_d.cl:83-100, ctem_image_d.cl:86-102)
__device__ __forceinline__ double cchi_of(const AberrD &A, double2 w) {
    double2 wc = cConj(w);
    double tC10 = 0.5 * A.C10 * cModSq(w);
    double2 tC12 = sc(cmul(A.C12, cPow(wc, 2)), 0.5);
    double2 tC21 = dv(cmul(A.C21, cmul(cPow(wc, 2), w)), 3.0);
    double2 tC23 = dv(cmul(A.C23, cPow(wc, 3)), 3.0);
    double tC30 = 0.25 * A.C30 * cModSq(w) * cModSq(w);
    double2 tC32 = sc(cmul(A.C32, cmul(cPow(wc, 3), w)), 0.25);
    double2 tC34 = sc(cmul(A.C34, cPow(wc, 4)), 0.25);
    double2 tC41 = sc(cmul(A.C41, cmul(cPow(wc, 3), cPow(w, 2))), 0.2);
    double2 tC43 = sc(cmul(A.C43, cmul(cPow(wc, 4), w)), 0.2);
    double2 tC45 = sc(cmul(A.C45, cPow(wc, 5)), 0.2);
    double tC50 = A.C50 * cModSq(w) * cModSq(w) * cModSq(w) / 6.0;
    double2 tC52 = dv(cmul(A.C52, cmul(cPow(wc, 4), cPow(w, 2))), 6.0);
    double2 tC54 = dv(cmul(A.C54, cmul(cPow(wc, 5), w)), 6.0);
    double2 tC56 = dv(cmul(A.C56, cPow(wc, 6)), 6.0);
    return tC10 + tC12.x + tC21.x + tC23.x + tC30 + tC32.x + tC34.x + tC41.x + tC43.x + tC45.x + tC50 + tC52.x + tC54.x + tC56.x;
}


}  // namespace ms
