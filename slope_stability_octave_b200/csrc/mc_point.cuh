// Per-point Mohr-Coulomb return mapping with consistent tangent (device functions).
//
// Algorithm of the reference's constitutive kernels
//   3D: +CONSTITUTIVE_PROBLEM/mex/constitutive_3D_kernel.h:101-410
//   2D: +CONSTITUTIVE_PROBLEM/mex/constitutive_2D_kernel.h:36-369
// (elastic-perfectly plastic Mohr-Coulomb, associated flow, implicit return onto the
// smooth face, the left / right edges or the apex; tangent from Miehe's closed form for
// eigen-projection derivatives).  Formulas and branch tests are kept in the reference's
// order so that the branch decision agrees with the reference's CPU code.
//
// 3D tangent symmetry: for associated flow the tangent is exactly symmetric (every term
// is a symmetric expression of (i, j)), so only the 21 entries with i <= j are evaluated
// and mirrored; the stored 6x6 matrix is identical to evaluating all 36.
#pragma once

#include <stdint.h>

namespace sg {

enum Branch : uint8_t { BR_ELASTIC = 0, BR_SMOOTH = 1, BR_LEFT = 2, BR_RIGHT = 3, BR_APEX = 4 };

__device__ __forceinline__ double unit3(int i) { return i < 3 ? 1.0 : 0.0; }
__device__ __forceinline__ double half_id(int i, int j) { return i != j ? 0.0 : (i < 3 ? 1.0 : 0.5); }

// d(T^2)_i / dE_j for the stress-representation tensor T (E engineering), entry (i, j).
__device__ __forceinline__ double dsq(const double t[6], int i, int j) {
    // symmetric in (i, j); callers use i <= j
    if (i > j) { int s = i; i = j; j = s; }
    switch (i * 6 + j) {
        case 0: return 2.0 * t[0];
        case 3: return t[3];
        case 5: return t[5];
        case 7: return 2.0 * t[1];
        case 9: return t[3];
        case 10: return t[4];
        case 14: return 2.0 * t[2];
        case 16: return t[4];
        case 17: return t[5];
        case 21: return 0.5 * (t[0] + t[1]);
        case 22: return 0.5 * t[5];
        case 23: return 0.5 * t[4];
        case 28: return 0.5 * (t[1] + t[2]);
        case 29: return 0.5 * t[3];
        case 35: return 0.5 * (t[0] + t[2]);
        default: return 0.0;
    }
}

__device__ __forceinline__ void sylvester(const double tsq[6], const double t[6], double bc_sum,
                                          double bc_prod, double scale, double P[6]) {
#pragma unroll
    for (int i = 0; i < 3; ++i) P[i] = scale * (tsq[i] - bc_sum * t[i] + bc_prod);
#pragma unroll
    for (int i = 3; i < 6; ++i) P[i] = scale * (tsq[i] - bc_sum * t[i]);
}

// Quantities shared by every branch: the stress-representation strain t, t^2, I1, the
// ordered principal strains e1 >= e2 >= e3 and the trial yield value.
struct MC3Pre {
    double t[6], tsq[6], I1, e1, e2, e3, f_tr;
};

__device__ __forceinline__ void mc3d_prefix(const double E[6], double c_bar, double sin_phi, double shear,
                                            double lame, MC3Pre &q) {
    const double sp = sin_phi;
    double *t = q.t, *tsq = q.tsq;
    t[0] = E[0];
    t[1] = E[1];
    t[2] = E[2];
    t[3] = 0.5 * E[3];
    t[4] = 0.5 * E[4];
    t[5] = 0.5 * E[5];
    tsq[0] = t[0] * t[0] + t[3] * t[3] + t[5] * t[5];
    tsq[1] = t[1] * t[1] + t[3] * t[3] + t[4] * t[4];
    tsq[2] = t[2] * t[2] + t[4] * t[4] + t[5] * t[5];
    tsq[3] = t[0] * t[3] + t[1] * t[3] + t[4] * t[5];
    tsq[4] = t[3] * t[5] + t[1] * t[4] + t[2] * t[4];
    tsq[5] = t[0] * t[5] + t[3] * t[4] + t[2] * t[5];
    const double I1 = t[0] + t[1] + t[2];
    const double I2 = t[0] * t[1] + t[0] * t[2] + t[1] * t[2] - t[3] * t[3] - t[4] * t[4] - t[5] * t[5];
    const double I3 = t[0] * t[1] * t[2] - t[2] * t[3] * t[3] - t[1] * t[5] * t[5] - t[0] * t[4] * t[4] +
                      2.0 * t[3] * t[4] * t[5];
    double Qv = (I1 * I1 - 3.0 * I2) / 9.0;
    if (Qv < 0.0) Qv = 0.0;
    const double Rv = (-2.0 * I1 * I1 * I1 + 9.0 * I1 * I2 - 27.0 * I3) / 54.0;
    const double rq = sqrt(Qv);
    double theta = 0.0;
    if (!(Qv < 1e-30)) {
        double c = Rv / (rq * Qv);
        c = fmin(fmax(c, -1.0), 1.0);
        theta = acos(c) / 3.0;
    }
    const double two_pi_3 = 2.0 * 3.14159265358979323846 / 3.0;
    const double e1 = -2.0 * rq * cos(theta + two_pi_3) + I1 / 3.0;
    const double e2 = -2.0 * rq * cos(theta - two_pi_3) + I1 / 3.0;
    const double e3 = -2.0 * rq * cos(theta) + I1 / 3.0;

    const double f_tr = 2.0 * shear * ((1.0 + sp) * e1 - (1.0 - sp) * e3) + 2.0 * lame * sp * I1 - c_bar;
    q.I1 = I1;
    q.e1 = e1;
    q.e2 = e2;
    q.e3 = e3;
    q.f_tr = f_tr;
}

// The branch the reference's kernel takes for this point (its tests, in its order).
__device__ __forceinline__ int mc3d_classify(const MC3Pre &q, double c_bar, double sp, double shear, double lame) {
    if (q.f_tr <= 0.0) return BR_ELASTIC;
    const double e1 = q.e1, e2 = q.e2, e3 = q.e3, I1 = q.I1;
    const double g_sl = (e1 - e2) / (1.0 + sp);
    const double g_sr = (e2 - e3) / (1.0 - sp);
    const double den_s = 4.0 * lame * sp * sp + 4.0 * shear * (1.0 + sp * sp);
    const double dl_s = q.f_tr / den_s;
    if (dl_s <= g_sl && dl_s <= g_sr) return BR_SMOOTH;
    if (g_sl < g_sr) {
        const double den_l = 4.0 * lame * sp * sp + shear * (1.0 + sp) * (1.0 + sp) +
                             2.0 * shear * (1.0 - sp) * (1.0 - sp);
        const double dl_l =
            (shear * ((1.0 + sp) * (e1 + e2) - 2.0 * (1.0 - sp) * e3) + 2.0 * lame * sp * I1 - c_bar) / den_l;
        const double g_la = (e1 + e2 - 2.0 * e3) / (3.0 - sp);
        if (dl_l >= g_sl && dl_l <= g_la) return BR_LEFT;
    }
    if (g_sl > g_sr) {
        const double den_r = 4.0 * lame * sp * sp + 2.0 * shear * (1.0 + sp) * (1.0 + sp) +
                             shear * (1.0 - sp) * (1.0 - sp);
        const double dl_r =
            (shear * (2.0 * (1.0 + sp) * e1 - (1.0 - sp) * (e2 + e3)) + 2.0 * lame * sp * I1 - c_bar) / den_r;
        const double g_ra = (2.0 * e1 - e2 - e3) / (3.0 + sp);
        if (dl_r >= g_sr && dl_r <= g_ra) return BR_RIGHT;
    }
    return BR_APEX;
}

// Stress (and tangent when WANT_DS) of branch `br` from the shared quantities; writes S[6] and
// ds[i + 6*j] (column-major).  The formulas are those of the reference's branch code.
template <bool WANT_DS>
__device__ __forceinline__ void mc3d_finish(const MC3Pre &q, int br, double c_bar, double sp, double shear,
                                            double lame, double S[6], double *ds) {
    const double *t = q.t, *tsq = q.tsq;
    const double I1 = q.I1, e1 = q.e1, e2 = q.e2, e3 = q.e3, f_tr = q.f_tr;
    if (br == BR_ELASTIC) {
        const double v = lame * I1, g2 = 2.0 * shear;
        S[0] = v + g2 * t[0];
        S[1] = v + g2 * t[1];
        S[2] = v + g2 * t[2];
        S[3] = g2 * t[3];
        S[4] = g2 * t[4];
        S[5] = g2 * t[5];
        if (WANT_DS) {
#pragma unroll
            for (int j = 0; j < 6; ++j)
#pragma unroll
                for (int i = 0; i < 6; ++i)
                    ds[i + 6 * j] = (i < 3 && j < 3 ? lame : 0.0) + (i == j ? (i < 3 ? g2 : shear) : 0.0);
        }
        return;
    }
    if (br == BR_SMOOTH) {
        const double den_s = 4.0 * lame * sp * sp + 4.0 * shear * (1.0 + sp * sp);
        const double dl_s = f_tr / den_s;
        const double k1 = 1.0 / ((e1 - e2) * (e1 - e3));
        const double k2 = 1.0 / ((e2 - e1) * (e2 - e3));
        const double k3 = 1.0 / ((e3 - e1) * (e3 - e2));
        double P1[6], P2[6], P3[6];
        sylvester(tsq, t, e2 + e3, e2 * e3, k1, P1);
        sylvester(tsq, t, e1 + e3, e1 * e3, k2, P2);
        sylvester(tsq, t, e1 + e2, e1 * e2, k3, P3);
        const double s1 = lame * I1 + 2.0 * shear * e1 - dl_s * (2.0 * lame * sp + 2.0 * shear * (1.0 + sp));
        const double s2 = lame * I1 + 2.0 * shear * e2 - dl_s * 2.0 * lame * sp;
        const double s3 = lame * I1 + 2.0 * shear * e3 - dl_s * (2.0 * lame * sp - 2.0 * shear * (1.0 - sp));
#pragma unroll
        for (int i = 0; i < 6; ++i) S[i] = s1 * P1[i] + s2 * P2[i] + s3 * P3[i];
        if (WANT_DS) {
            double n[6];
#pragma unroll
            for (int i = 0; i < 6; ++i)
                n[i] = 2.0 * shear * ((1.0 + sp) * P1[i] - (1.0 - sp) * P3[i]) + 2.0 * lame * sp * unit3(i);
            const double a1 = 2.0 * e1 - e2 - e3, b1 = e2 - e3;
            const double a2 = 2.0 * e2 - e1 - e3, b2 = e1 - e3;
            const double a3 = 2.0 * e3 - e1 - e2, b3 = e1 - e2;
            const double inv_den = 1.0 / den_s;
#pragma unroll
            for (int j = 0; j < 6; ++j)
#pragma unroll
                for (int i = 0; i <= j; ++i) {
                    const double hi = half_id(i, j), d = dsq(t, i, j);
                    const double q11 = P1[i] * P1[j], q22 = P2[i] * P2[j], q33 = P3[i] * P3[j];
                    const double d1 = k1 * (d - hi * (e2 + e3) - a1 * q11 - b1 * (q22 - q33));
                    const double d2 = k2 * (d - hi * (e1 + e3) - a2 * q22 - b2 * (q11 - q33));
                    const double d3 = k3 * (d - hi * (e1 + e2) - a3 * q33 - b3 * (q11 - q22));
                    const double v = s1 * d1 + s2 * d2 + s3 * d3 + lame * unit3(i) * unit3(j) +
                                     2.0 * shear * (q11 + q22 + q33) - n[i] * n[j] * inv_den;
                    ds[i + 6 * j] = v;
                    ds[j + 6 * i] = v;
                }
        }
        return;
    }
    if (br == BR_LEFT) {
        const double den_l = 4.0 * lame * sp * sp + shear * (1.0 + sp) * (1.0 + sp) +
                             2.0 * shear * (1.0 - sp) * (1.0 - sp);
        const double dl_l =
            (shear * ((1.0 + sp) * (e1 + e2) - 2.0 * (1.0 - sp) * e3) + 2.0 * lame * sp * I1 - c_bar) / den_l;
        {
            const double k3 = 1.0 / ((e3 - e1) * (e3 - e2));
            double P3[6], P12[6];
            sylvester(tsq, t, e1 + e2, e1 * e2, k3, P3);
#pragma unroll
            for (int i = 0; i < 6; ++i) P12[i] = unit3(i) - P3[i];
            const double s12 = lame * I1 + shear * (e1 + e2) - dl_l * (2.0 * lame * sp + shear * (1.0 + sp));
            const double s3 = lame * I1 + 2.0 * shear * e3 - dl_l * (2.0 * lame * sp - 2.0 * shear * (1.0 - sp));
#pragma unroll
            for (int i = 0; i < 6; ++i) S[i] = s12 * P12[i] + s3 * P3[i];
            if (WANT_DS) {
                double n[6];
#pragma unroll
                for (int i = 0; i < 6; ++i)
                    n[i] = shear * ((1.0 + sp) * P12[i] - 2.0 * (1.0 - sp) * P3[i]) + 2.0 * lame * sp * unit3(i);
                const double e12 = e1 + e2, inv_den = 1.0 / den_l;
#pragma unroll
                for (int j = 0; j < 6; ++j)
#pragma unroll
                    for (int i = 0; i <= j; ++i) {
                        const double hi = half_id(i, j), d = dsq(t, i, j);
                        const double q33 = P3[i] * P3[j], qpp = P12[i] * P12[j];
                        const double ct = P12[i] * t[j] + t[i] * P12[j];
                        const double cp = P12[i] * P3[j] + P3[i] * P12[j];
                        const double d3 = k3 * (d - hi * e12 - ct + e12 * qpp + (e12 - 2.0 * e3) * q33 + e3 * cp);
                        const double v = (s3 - s12) * d3 + lame * unit3(i) * unit3(j) + shear * (qpp + 2.0 * q33) -
                                         n[i] * n[j] * inv_den;
                        ds[i + 6 * j] = v;
                        ds[j + 6 * i] = v;
                    }
            }
            return;
        }
    }
    if (br == BR_RIGHT) {
        const double den_r = 4.0 * lame * sp * sp + 2.0 * shear * (1.0 + sp) * (1.0 + sp) +
                             shear * (1.0 - sp) * (1.0 - sp);
        const double dl_r =
            (shear * (2.0 * (1.0 + sp) * e1 - (1.0 - sp) * (e2 + e3)) + 2.0 * lame * sp * I1 - c_bar) / den_r;
        {
            const double k1 = 1.0 / ((e1 - e2) * (e1 - e3));
            double P1[6], P23[6];
            sylvester(tsq, t, e2 + e3, e2 * e3, k1, P1);
#pragma unroll
            for (int i = 0; i < 6; ++i) P23[i] = unit3(i) - P1[i];
            const double s1 = lame * I1 + 2.0 * shear * e1 - dl_r * (2.0 * lame * sp + 2.0 * shear * (1.0 + sp));
            const double s23 = lame * I1 + shear * (e2 + e3) - dl_r * (2.0 * lame * sp - shear * (1.0 - sp));
#pragma unroll
            for (int i = 0; i < 6; ++i) S[i] = s1 * P1[i] + s23 * P23[i];
            if (WANT_DS) {
                double n[6];
#pragma unroll
                for (int i = 0; i < 6; ++i)
                    n[i] = shear * (2.0 * (1.0 + sp) * P1[i] - (1.0 - sp) * P23[i]) + 2.0 * lame * sp * unit3(i);
                const double e23 = e2 + e3, inv_den = 1.0 / den_r;
#pragma unroll
                for (int j = 0; j < 6; ++j)
#pragma unroll
                    for (int i = 0; i <= j; ++i) {
                        const double hi = half_id(i, j), d = dsq(t, i, j);
                        const double q11 = P1[i] * P1[j], qmm = P23[i] * P23[j];
                        const double ct = P23[i] * t[j] + t[i] * P23[j];
                        const double cp = P23[i] * P1[j] + P1[i] * P23[j];
                        const double d1 = k1 * (d - hi * e23 - ct + e23 * qmm + (e23 - 2.0 * e1) * q11 + e1 * cp);
                        const double v = (s1 - s23) * d1 + lame * unit3(i) * unit3(j) + shear * (2.0 * q11 + qmm) -
                                         n[i] * n[j] * inv_den;
                        ds[i + 6 * j] = v;
                        ds[j + 6 * i] = v;
                    }
            }
            return;
        }
    }
    // apex
    const double sa = c_bar / (2.0 * sp);
    S[0] = sa;
    S[1] = sa;
    S[2] = sa;
    S[3] = 0.0;
    S[4] = 0.0;
    S[5] = 0.0;
    if (WANT_DS) {
#pragma unroll
        for (int k = 0; k < 36; ++k) ds[k] = 0.0;
    }
}

// Writes S[6]; when ds != nullptr writes the 6x6 tangent at ds[i + 6*j] (column-major).
template <bool WANT_DS>
__device__ __forceinline__ int mc3d_point(const double E[6], double c_bar, double sin_phi,
                                          double shear, double lame, double S[6], double *ds) {
    MC3Pre q;
    mc3d_prefix(E, c_bar, sin_phi, shear, lame, q);
    const int br = mc3d_classify(q, c_bar, sin_phi, shear, lame);
    mc3d_finish<WANT_DS>(q, br, c_bar, sin_phi, shear, lame, S, ds);
    return br;
}

// 2D plane-strain variant.  E = (e11, e22, g12); S = (s11, s22, s12, s33); ds 3x3 column-major.
template <bool WANT_DS>
__device__ __forceinline__ int mc2d_point(const double E[3], double c_bar, double sp, double shear,
                                          double lame, double S[4], double *ds) {
    const double tr = E[0] + E[1];
    const double rad = sqrt((E[0] - E[1]) * (E[0] - E[1]) + E[2] * E[2]);
    const double ua = 0.5 * (tr + rad), ub = 0.5 * (tr - rad), uc = 0.0;
    double pa0 = 1.0, pa1 = 1.0, pa2 = 0.0;
    if (rad != 0.0) {
        pa0 = (E[0] - ub) / rad;
        pa1 = (E[1] - ub) / rad;
        pa2 = 0.5 * E[2] / rad;
    }
    const double Pa[4] = {pa0, pa1, pa2, 0.0};
    const double Pb[4] = {1.0 - pa0, 1.0 - pa1, -pa2, 0.0};
    const double Pc[4] = {0.0, 0.0, 0.0, 1.0};
    // which of (a, b, c) sits at ordered positions 1, 2, 3
    int o1 = 0, o2 = 1, o3 = 2;
    double e1 = ua, e2 = ub, e3 = uc;
    if (ua >= uc && uc > ub) { o2 = 2; o3 = 1; e2 = uc; e3 = ub; }
    if (uc > ua) { o1 = 2; o2 = 0; o3 = 1; e1 = uc; e2 = ua; e3 = ub; }
    auto P = [&](int which, int i) { return which == 0 ? Pa[i] : (which == 1 ? Pb[i] : Pc[i]); };
    // Hessian of ua: Ha = (diag(1,1,1/2) - Pa Pa' - Pb Pb') / rad; Hb = -Ha; Hc = 0
    auto Hsgn = [&](int which) { return which == 0 ? 1.0 : (which == 1 ? -1.0 : 0.0); };
    auto Ha = [&](int i, int j) {
        if (rad == 0.0) return 0.0;
        const double dg = (i == j) ? (i < 2 ? 1.0 : 0.5) : 0.0;
        return (dg - Pa[j] * Pa[i] - Pb[j] * Pb[i]) * (1.0 / rad);
    };

    const double trE = e1 + e2 + e3;
    const double f_tr = 2.0 * shear * ((1.0 + sp) * e1 - (1.0 - sp) * e3) + 2.0 * lame * sp * trE - c_bar;
    const double g_sl = (e1 - e2) / (1.0 + sp);
    const double g_sr = (e2 - e3) / (1.0 - sp);
    const double g_la = (e1 + e2 - 2.0 * e3) / (3.0 - sp);
    const double g_ra = (2.0 * e1 - e2 - e3) / (3.0 + sp);
    const double den_s = 4.0 * lame * sp * sp + 2.0 * shear * (1.0 + sp) * (1.0 + sp) + 2.0 * shear * (1.0 - sp) * (1.0 - sp);
    const double den_l = 4.0 * lame * sp * sp + shear * (1.0 + sp) * (1.0 + sp) + 2.0 * shear * (1.0 - sp) * (1.0 - sp);
    const double den_r = 4.0 * lame * sp * sp + 2.0 * shear * (1.0 + sp) * (1.0 + sp) + shear * (1.0 - sp) * (1.0 - sp);
    const double dl_s = f_tr / den_s;
    const double dl_l = (shear * ((1.0 + sp) * (e1 + e2) - 2.0 * (1.0 - sp) * e3) + 2.0 * lame * sp * trE - c_bar) / den_l;
    const double dl_r = (shear * (2.0 * (1.0 + sp) * e1 - (1.0 - sp) * (e2 + e3)) + 2.0 * lame * sp * trE - c_bar) / den_r;

    int br;
    if (f_tr <= 0.0) br = BR_ELASTIC;
    else if (dl_s <= fmin(g_sl, g_sr)) br = BR_SMOOTH;
    else if (g_sl < g_sr && dl_l >= g_sl && dl_l <= g_la) br = BR_LEFT;
    else if (g_sl > g_sr && dl_r >= g_sr && dl_r <= g_ra) br = BR_RIGHT;
    else br = BR_APEX;

    if (br == BR_ELASTIC) {
        const double v = E[0] + E[1];
        S[0] = lame * v + 2.0 * shear * E[0];
        S[1] = lame * v + 2.0 * shear * E[1];
        S[2] = shear * E[2];
        S[3] = lame * v;
        if (WANT_DS) {
            ds[0] = lame + 2.0 * shear; ds[1] = lame; ds[2] = 0.0;
            ds[3] = lame; ds[4] = lame + 2.0 * shear; ds[5] = 0.0;
            ds[6] = 0.0; ds[7] = 0.0; ds[8] = shear;
        }
        return br;
    }
    if (br == BR_APEX) {
        const double sa = c_bar / (2.0 * sp);
        S[0] = sa; S[1] = sa; S[2] = 0.0; S[3] = sa;
        if (WANT_DS) {
#pragma unroll
            for (int k = 0; k < 9; ++k) ds[k] = 0.0;
        }
        return br;
    }
    // plastic, non-apex: stress = sum of weights * projections, tangent = weights * Hessians
    // + moduli * outer products - n n' / den
    double w1, w2, w3;          // stress weights of ordered projections 1, 2, 3
    double m1, m2, m3;          // tangent outer-product moduli (multiplying P_k P_k')
    double nc1, nc3, den;       // n = nc1 * P1 + nc3 * P3 (+ 2 lame sp iota)
    bool merge12 = false, merge23 = false;
    if (br == BR_SMOOTH) {
        w1 = lame * trE + 2.0 * shear * e1 - dl_s * (2.0 * lame * sp + 2.0 * shear * (1.0 + sp));
        w2 = lame * trE + 2.0 * shear * e2 - dl_s * (2.0 * lame * sp);
        w3 = lame * trE + 2.0 * shear * e3 - dl_s * (2.0 * lame * sp - 2.0 * shear * (1.0 - sp));
        m1 = m2 = m3 = 2.0 * shear;
        nc1 = 2.0 * shear * (1.0 + sp);
        nc3 = -2.0 * shear * (1.0 - sp);
        den = den_s;
    } else if (br == BR_LEFT) {
        w1 = w2 = lame * trE + shear * (e1 + e2) - dl_l * (2.0 * lame * sp + shear * (1.0 + sp));
        w3 = lame * trE + 2.0 * shear * e3 - dl_l * (2.0 * lame * sp - 2.0 * shear * (1.0 - sp));
        m1 = m2 = shear;
        m3 = 2.0 * shear;
        nc1 = shear * (1.0 + sp);
        nc3 = -2.0 * shear * (1.0 - sp);
        den = den_l;
        merge12 = true;
    } else {
        w1 = lame * trE + 2.0 * shear * e1 - dl_r * (2.0 * lame * sp + 2.0 * shear * (1.0 + sp));
        w2 = w3 = lame * trE + shear * (e2 + e3) - dl_r * (2.0 * lame * sp - shear * (1.0 - sp));
        m1 = 2.0 * shear;
        m2 = m3 = shear;
        nc1 = 2.0 * shear * (1.0 + sp);
        nc3 = -shear * (1.0 - sp);
        den = den_r;
        merge23 = true;
    }
    if (merge12) {
#pragma unroll
        for (int i = 0; i < 4; ++i) S[i] = w1 * (P(o1, i) + P(o2, i)) + w3 * P(o3, i);
    } else if (merge23) {
#pragma unroll
        for (int i = 0; i < 4; ++i) S[i] = w1 * P(o1, i) + w3 * (P(o2, i) + P(o3, i));
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) S[i] = w1 * P(o1, i) + w2 * P(o2, i) + w3 * P(o3, i);
    }
    if (WANT_DS) {
        double v1[3], v2[3], v3[3], nn[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            v1[i] = P(o1, i);
            v2[i] = P(o2, i);
            v3[i] = P(o3, i);
        }
        if (merge12) {
#pragma unroll
            for (int i = 0; i < 3; ++i) { v1[i] = v1[i] + v2[i]; }
        }
        if (merge23) {
#pragma unroll
            for (int i = 0; i < 3; ++i) { v3[i] = v2[i] + v3[i]; }
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) nn[i] = nc1 * v1[i] + nc3 * v3[i] + (i < 2 ? 2.0 * lame * sp : 0.0);
        const double s1 = Hsgn(o1), s2 = Hsgn(o2), s3 = Hsgn(o3);
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const double h = Ha(i, j);
                double hterm, oterm;
                if (merge12) {
                    hterm = w1 * ((s1 + s2) * h) + w3 * (s3 * h);
                    oterm = m1 * v1[i] * v1[j] + m3 * v3[i] * v3[j];
                } else if (merge23) {
                    hterm = w1 * (s1 * h) + w3 * ((s2 + s3) * h);
                    oterm = m1 * v1[i] * v1[j] + m3 * v3[i] * v3[j];
                } else {
                    hterm = w1 * (s1 * h) + w2 * (s2 * h) + w3 * (s3 * h);
                    oterm = m1 * v1[i] * v1[j] + m2 * v2[i] * v2[j] + m3 * v3[i] * v3[j];
                }
                const double vol = (i < 2 && j < 2) ? lame : 0.0;
                ds[i + 3 * j] = hterm + vol + oterm - (1.0 / den) * nn[i] * nn[j];
            }
    }
    return br;
}

// Davis strength reduction (+CONSTITUTIVE_PROBLEM/reduction.m:25-58), point-wise.
// Elastoplastic potential of the trial strain at one point (the integrand of the SSR direct
// method's energy): +CONSTITUTIVE_PROBLEM/potential_3D.m:36-123 (3D, E with engineering
// shears) and potential_2D.m:26-95 (2D, E = e11, e22, g12).  The branch tests and formulas
// follow those files, including their own eigenvalue formulas (R / sqrt(Q^3), Q > 0).
__device__ __forceinline__ double potential_branches(double e1, double e2, double e3, double f_tr, double den_s,
                                                     double c_bar, double sp, double shear, double bulk,
                                                     double lame) {
    const double g_sl = (e1 - e2) / (1.0 + sp);
    const double g_sr = (e2 - e3) / (1.0 - sp);
    const double g_la = (e1 + e2 - 2.0 * e3) / (3.0 - sp);
    const double g_ra = (2.0 * e1 - e2 - e3) / (3.0 + sp);
    const double den_l = 4.0 * lame * sp * sp + shear * (1.0 + sp) * (1.0 + sp) + 2.0 * shear * (1.0 - sp) * (1.0 - sp);
    const double den_r = 4.0 * lame * sp * sp + 2.0 * shear * (1.0 + sp) * (1.0 + sp) + shear * (1.0 - sp) * (1.0 - sp);
    const double den_a = 4.0 * bulk * sp * sp;
    const double tr = e1 + e2 + e3;
    const double el = 0.5 * lame * tr * tr;
    if (f_tr <= 0.0) return el + shear * (e1 * e1 + e2 * e2 + e3 * e3);
    const double l_s = f_tr / den_s;
    if (l_s <= fmin(g_sl, g_sr)) return el + shear * (e1 * e1 + e2 * e2 + e3 * e3) - 0.5 * den_s * l_s * l_s;
    const double l_l = (shear * ((1.0 + sp) * (e1 + e2) - 2.0 * (1.0 - sp) * e3) + 2.0 * lame * sp * tr - c_bar) / den_l;
    if (g_sl < g_sr && l_l >= g_sl && l_l <= g_la)
        return el + shear * (e3 * e3 + 0.5 * (e1 + e2) * (e1 + e2)) - 0.5 * den_l * l_l * l_l;
    const double l_r = (shear * (2.0 * (1.0 + sp) * e1 - (1.0 - sp) * (e2 + e3)) + 2.0 * lame * sp * tr - c_bar) / den_r;
    if (g_sl > g_sr && l_r >= g_sr && l_r <= g_ra)
        return el + shear * (e1 * e1 + 0.5 * (e2 + e3) * (e2 + e3)) - 0.5 * den_r * l_r * l_r;
    const double l_a = (2.0 * bulk * sp * tr - c_bar) / den_a;
    return 0.5 * bulk * tr * tr - 0.5 * den_a * l_a * l_a;
}

__device__ __forceinline__ double potential3d(const double E[6], double c_bar, double sp, double shear, double bulk,
                                              double lame) {
    const double t0 = E[0], t1 = E[1], t2 = E[2], t3 = 0.5 * E[3], t4 = 0.5 * E[4], t5 = 0.5 * E[5];
    const double I1 = t0 + t1 + t2;
    const double I2 = t0 * t1 + t0 * t2 + t1 * t2 - t3 * t3 - t4 * t4 - t5 * t5;
    const double I3 = t0 * t1 * t2 - t2 * t3 * t3 - t1 * t5 * t5 - t0 * t4 * t4 + 2.0 * t3 * t4 * t5;
    const double Q = fmax(0.0, (1.0 / 9.0) * (I1 * I1 - 3.0 * I2));
    const double R = (1.0 / 54.0) * (-2.0 * (I1 * I1 * I1) + 9.0 * (I1 * I2) - 27.0 * I3);
    const double th0 = Q > 0.0 ? R / sqrt(Q * Q * Q) : 0.0;
    const double th = acos(fmin(fmax(th0, -1.0), 1.0)) / 3.0;
    const double pi = 3.14159265358979323846, sq = sqrt(Q);
    const double e1 = -2.0 * sq * cos(th + 2.0 * pi / 3.0) + I1 / 3.0;
    const double e2 = -2.0 * sq * cos(th - 2.0 * pi / 3.0) + I1 / 3.0;
    const double e3 = -2.0 * sq * cos(th) + I1 / 3.0;
    const double f_tr = 2.0 * shear * ((1.0 + sp) * e1 - (1.0 - sp) * e3) + 2.0 * (lame * sp) * I1 - c_bar;
    const double den_s = 4.0 * lame * sp * sp + 4.0 * shear * (1.0 + sp * sp);
    return potential_branches(e1, e2, e3, f_tr, den_s, c_bar, sp, shear, bulk, lame);
}

__device__ __forceinline__ double potential2d(const double E[3], double c_bar, double sp, double shear, double bulk,
                                              double lame) {
    const double I1 = E[0] + E[1];
    const double I2 = sqrt((E[0] - E[1]) * (E[0] - E[1]) + E[2] * E[2]);
    const double a = (I1 + I2) / 2.0, b = (I1 - I2) / 2.0, c = 0.0;
    double e1 = a, e2 = b, e3 = c;
    if (a >= c && c > b) { e2 = c; e3 = b; }
    if (c > a) { e1 = c; e2 = a; e3 = b; }
    const double tr = e1 + e2 + e3;
    const double f_tr = 2.0 * shear * ((1.0 + sp) * e1 - (1.0 - sp) * e3) + 2.0 * lame * sp * tr - c_bar;
    const double den_s = 4.0 * lame * sp * sp + 2.0 * shear * (1.0 + sp) * (1.0 + sp) + 2.0 * shear * (1.0 - sp) * (1.0 - sp);
    return potential_branches(e1, e2, e3, f_tr, den_s, c_bar, sp, shear, bulk, lame);
}

__device__ __forceinline__ void davis_reduce(double c0, double phi, double psi, double lambda, char type,
                                             double &c_bar, double &sin_phi) {
    double beta, c_l, phi_l;
    if (type == 'A') {
        beta = cos(phi) * cos(psi) / (1.0 - sin(phi) * sin(psi));
        c_l = beta * c0 / lambda;
        phi_l = atan(beta * tan(phi) / lambda);
    } else if (type == 'B') {
        const double c1 = c0 / lambda;
        const double f1 = atan(tan(phi) / lambda);
        const double s1 = atan(tan(psi) / lambda);
        beta = cos(f1) * cos(s1) / (1.0 - sin(f1) * sin(s1));
        c_l = beta * c1;
        phi_l = atan(beta * tan(f1));
    } else {
        const double c1 = c0 / lambda;
        const double f1 = atan(tan(phi) / lambda);
        beta = (f1 > psi) ? cos(f1) * cos(psi) / (1.0 - sin(f1) * sin(psi)) : 1.0;
        c_l = beta * c1;
        phi_l = atan(beta * tan(f1));
    }
    c_bar = 2.0 * c_l * cos(phi_l);
    sin_phi = sin(phi_l);
}

}  // namespace sg
