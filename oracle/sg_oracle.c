/*
 * ORACLE -- test infrastructure only.  CPU restatement of the reference's hot-path
 * arithmetic, used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg as the checker.  Never linked into, or called by, the product library.
 *
 * Parity pin: this restatement is checked point-by-point against the reference's
 * own MEX sources compiled unchanged (oracle/Makefile `ref` target) and against
 * golden vectors generated from them (tests/golden/).
 *
 * Restated algorithms (file:line in Beremi/slope_stability_octave):
 *   mc3d_point   : +CONSTITUTIVE_PROBLEM/mex/constitutive_3D_kernel.h:101-410
 *                  (Mohr-Coulomb return mapping, associated flow, 5 branches;
 *                  eigen-projection derivatives after Miehe's closed form)
 *   mc2d_point   : +CONSTITUTIVE_PROBLEM/mex/constitutive_2D_kernel.h:36-369
 *   assemble_*   : +ASSEMBLY/mex/assemble_K_tangent_vals.c:77-171 and
 *                  assemble_K_tangent_vals_2D.c (element-local B'(wD)B summed into
 *                  a value vector through a 1-based scatter map, 0 = skip)
 *
 * Branch ids: 0 elastic, 1 smooth face, 2 left edge, 3 right edge, 4 apex.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.14159265358979323846

enum { BR_ELASTIC = 0, BR_SMOOTH = 1, BR_LEFT = 2, BR_RIGHT = 3, BR_APEX = 4 };

/* ---------------------------------------------------------------- 3D helpers */

/* Sylvester formula for the eigen-projection of eigenvalue a with the other two
 * eigenvalues b, c:  P_a = (T^2 - (b+c) T + b c I) / ((a-b)(a-c)).          */
static void sylvester(const double tsq[6], const double t[6], double bc_sum,
                      double bc_prod, double scale, double P[6])
{
    for (int i = 0; i < 3; ++i) P[i] = scale * (tsq[i] - bc_sum * t[i] + bc_prod);
    for (int i = 3; i < 6; ++i) P[i] = scale * (tsq[i] - bc_sum * t[i]);
}

/* d(T^2)_i / dE_j (E engineering, T tensor strain), column-major k = i + 6 j */
static void dsq_dE(const double t[6], double d[36])
{
    memset(d, 0, sizeof(double) * 36);
    d[0 + 6 * 0] = 2.0 * t[0];
    d[3 + 6 * 0] = t[3];
    d[5 + 6 * 0] = t[5];
    d[1 + 6 * 1] = 2.0 * t[1];
    d[3 + 6 * 1] = t[3];
    d[4 + 6 * 1] = t[4];
    d[2 + 6 * 2] = 2.0 * t[2];
    d[4 + 6 * 2] = t[4];
    d[5 + 6 * 2] = t[5];
    d[0 + 6 * 3] = t[3];
    d[1 + 6 * 3] = t[3];
    d[3 + 6 * 3] = 0.5 * (t[0] + t[1]);
    d[4 + 6 * 3] = 0.5 * t[5];
    d[5 + 6 * 3] = 0.5 * t[4];
    d[1 + 6 * 4] = t[4];
    d[2 + 6 * 4] = t[4];
    d[3 + 6 * 4] = 0.5 * t[5];
    d[4 + 6 * 4] = 0.5 * (t[1] + t[2]);
    d[5 + 6 * 4] = 0.5 * t[3];
    d[0 + 6 * 5] = t[5];
    d[2 + 6 * 5] = t[5];
    d[3 + 6 * 5] = 0.5 * t[4];
    d[4 + 6 * 5] = 0.5 * t[3];
    d[5 + 6 * 5] = 0.5 * (t[0] + t[2]);
}

static inline double unit_dev(int i) { return i < 3 ? 1.0 : 0.0; }
static inline double half_ident(int i, int j) { return i != j ? 0.0 : (i < 3 ? 1.0 : 0.5); }

/* Elastic tangent lame*iota(x)iota + 2*shear*diag(1,1,1,1/2,1/2,1/2). */
static void elastic_tangent3(double lame, double shear, double *DS)
{
    memset(DS, 0, sizeof(double) * 36);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) DS[i + 6 * j] = lame;
    for (int i = 0; i < 3; ++i) DS[i + 6 * i] = 2.0 * shear + lame;
    for (int i = 3; i < 6; ++i) DS[i + 6 * i] = shear;
}

int orc_mc3d_point(const double *E, double c_bar, double sin_phi, double shear,
                   double lame, double *S, double *DS)
{
    const double sp = sin_phi; /* associated flow: psi == phi */
    double t[6] = {E[0], E[1], E[2], 0.5 * E[3], 0.5 * E[4], 0.5 * E[5]};
    double tsq[6];
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

    /* principal values via the trigonometric (Lode-angle) solution */
    double Qv = (I1 * I1 - 3.0 * I2) / 9.0;
    if (Qv < 0.0) Qv = 0.0;
    const double Rv = (-2.0 * I1 * I1 * I1 + 9.0 * I1 * I2 - 27.0 * I3) / 54.0;
    const double rq = sqrt(Qv);
    double theta = 0.0;
    if (!(Qv < 1e-30)) {
        double c = Rv / (rq * Qv);
        if (c < -1.0) c = -1.0;
        if (c > 1.0) c = 1.0;
        theta = acos(c) / 3.0;
    }
    const double e1 = -2.0 * rq * cos(theta + 2.0 * ORC_PI / 3.0) + I1 / 3.0;
    const double e2 = -2.0 * rq * cos(theta - 2.0 * ORC_PI / 3.0) + I1 / 3.0;
    const double e3 = -2.0 * rq * cos(theta) + I1 / 3.0;

    const double f_tr = 2.0 * shear * ((1.0 + sin_phi) * e1 - (1.0 - sin_phi) * e3) +
                        2.0 * lame * sin_phi * I1 - c_bar;

    if (f_tr <= 0.0) {
        const double vol = lame * I1, g2 = 2.0 * shear;
        for (int i = 0; i < 3; ++i) S[i] = vol + g2 * t[i];
        for (int i = 3; i < 6; ++i) S[i] = g2 * t[i];
        if (DS) elastic_tangent3(lame, shear, DS);
        return BR_ELASTIC;
    }

    const double g_sl = (e1 - e2) / (1.0 + sp);
    const double g_sr = (e2 - e3) / (1.0 - sp);
    const double den_s = 4.0 * lame * sin_phi * sp + 4.0 * shear * (1.0 + sin_phi * sp);
    const double dl_s = f_tr / den_s;

    if (dl_s <= g_sl && dl_s <= g_sr) {
        /* ---- return onto the smooth face: three distinct projections ---- */
        const double k1 = 1.0 / ((e1 - e2) * (e1 - e3));
        const double k2 = 1.0 / ((e2 - e1) * (e2 - e3));
        const double k3 = 1.0 / ((e3 - e1) * (e3 - e2));
        double P[3][6];
        sylvester(tsq, t, e2 + e3, e2 * e3, k1, P[0]);
        sylvester(tsq, t, e1 + e3, e1 * e3, k2, P[1]);
        sylvester(tsq, t, e1 + e2, e1 * e2, k3, P[2]);
        const double s1 = lame * I1 + 2.0 * shear * e1 - dl_s * (2.0 * lame * sp + 2.0 * shear * (1.0 + sp));
        const double s2 = lame * I1 + 2.0 * shear * e2 - dl_s * 2.0 * lame * sp;
        const double s3 = lame * I1 + 2.0 * shear * e3 - dl_s * (2.0 * lame * sp - 2.0 * shear * (1.0 - sp));
        for (int i = 0; i < 6; ++i) S[i] = s1 * P[0][i] + s2 * P[1][i] + s3 * P[2][i];
        if (DS) {
            double dsq[36], nphi[6], npsi[6];
            dsq_dE(t, dsq);
            for (int i = 0; i < 6; ++i) {
                nphi[i] = 2.0 * shear * ((1.0 + sin_phi) * P[0][i] - (1.0 - sin_phi) * P[2][i]) +
                          2.0 * lame * sin_phi * unit_dev(i);
                npsi[i] = 2.0 * shear * ((1.0 + sp) * P[0][i] - (1.0 - sp) * P[2][i]) +
                          2.0 * lame * sp * unit_dev(i);
            }
            /* Miehe: dP_a/dE = k_a [dT^2 - (b+c) I - (2a-b-c) Pa(x)Pa - (b-c)(Pb(x)Pb - Pc(x)Pc)] */
            const double a1 = 2.0 * e1 - e2 - e3, b1 = e2 - e3;
            const double a2 = 2.0 * e2 - e1 - e3, b2 = e1 - e3;
            const double a3 = 2.0 * e3 - e1 - e2, b3 = e1 - e2;
            const double inv_den = 1.0 / den_s;
            for (int j = 0; j < 6; ++j) {
                for (int i = 0; i < 6; ++i) {
                    const int k = i + 6 * j;
                    const double hi = half_ident(i, j);
                    const double q11 = P[0][i] * P[0][j], q22 = P[1][i] * P[1][j], q33 = P[2][i] * P[2][j];
                    const double d1 = k1 * (dsq[k] - hi * (e2 + e3) - a1 * q11 - b1 * (q22 - q33));
                    const double d2 = k2 * (dsq[k] - hi * (e1 + e3) - a2 * q22 - b2 * (q11 - q33));
                    const double d3 = k3 * (dsq[k] - hi * (e1 + e2) - a3 * q33 - b3 * (q11 - q22));
                    DS[k] = s1 * d1 + s2 * d2 + s3 * d3 + lame * unit_dev(i) * unit_dev(j) +
                            2.0 * shear * (q11 + q22 + q33) - npsi[i] * nphi[j] * inv_den;
                }
            }
        }
        return BR_SMOOTH;
    }

    if (g_sl < g_sr) {
        /* ---- candidate: left edge (sigma_1 == sigma_2) ---- */
        const double den_l = 4.0 * lame * sin_phi * sp + shear * (1.0 + sin_phi) * (1.0 + sp) +
                             2.0 * shear * (1.0 - sin_phi) * (1.0 - sp);
        const double dl_l = (shear * ((1.0 + sin_phi) * (e1 + e2) - 2.0 * (1.0 - sin_phi) * e3) +
                             2.0 * lame * sin_phi * I1 - c_bar) / den_l;
        const double g_la = (e1 + e2 - 2.0 * e3) / (3.0 - sp);
        if (dl_l >= g_sl && dl_l <= g_la) {
            const double k3 = 1.0 / ((e3 - e1) * (e3 - e2));
            double P3[6], P12[6];
            sylvester(tsq, t, e1 + e2, e1 * e2, k3, P3);
            for (int i = 0; i < 6; ++i) P12[i] = unit_dev(i) - P3[i];
            const double s12 = lame * I1 + shear * (e1 + e2) - dl_l * (2.0 * lame * sp + shear * (1.0 + sp));
            const double s3 = lame * I1 + 2.0 * shear * e3 - dl_l * (2.0 * lame * sp - 2.0 * shear * (1.0 - sp));
            for (int i = 0; i < 6; ++i) S[i] = s12 * P12[i] + s3 * P3[i];
            if (DS) {
                double dsq[36], nphi[6], npsi[6];
                dsq_dE(t, dsq);
                const double e12 = e1 + e2;
                for (int i = 0; i < 6; ++i) {
                    nphi[i] = shear * ((1.0 + sin_phi) * P12[i] - 2.0 * (1.0 - sin_phi) * P3[i]) +
                              2.0 * lame * sin_phi * unit_dev(i);
                    npsi[i] = shear * ((1.0 + sp) * P12[i] - 2.0 * (1.0 - sp) * P3[i]) +
                              2.0 * lame * sp * unit_dev(i);
                }
                const double inv_den = 1.0 / den_l;
                for (int j = 0; j < 6; ++j) {
                    for (int i = 0; i < 6; ++i) {
                        const int k = i + 6 * j;
                        const double hi = half_ident(i, j);
                        const double q33 = P3[i] * P3[j];
                        const double qpp = P12[i] * P12[j];
                        const double cross_t = P12[i] * t[j] + t[i] * P12[j];
                        const double cross_p = P12[i] * P3[j] + P3[i] * P12[j];
                        const double d3 = k3 * (dsq[k] - hi * e12 - cross_t + e12 * qpp +
                                                (e12 - 2.0 * e3) * q33 + e3 * cross_p);
                        DS[k] = (s3 - s12) * d3 + lame * unit_dev(i) * unit_dev(j) +
                                shear * (qpp + 2.0 * q33) - npsi[i] * nphi[j] * inv_den;
                    }
                }
            }
            return BR_LEFT;
        }
    }

    if (g_sl > g_sr) {
        /* ---- candidate: right edge (sigma_2 == sigma_3) ---- */
        const double den_r = 4.0 * lame * sin_phi * sp + 2.0 * shear * (1.0 + sin_phi) * (1.0 + sp) +
                             shear * (1.0 - sin_phi) * (1.0 - sp);
        const double dl_r = (shear * (2.0 * (1.0 + sin_phi) * e1 - (1.0 - sin_phi) * (e2 + e3)) +
                             2.0 * lame * sin_phi * I1 - c_bar) / den_r;
        const double g_ra = (2.0 * e1 - e2 - e3) / (3.0 + sp);
        if (dl_r >= g_sr && dl_r <= g_ra) {
            const double k1 = 1.0 / ((e1 - e2) * (e1 - e3));
            double P1[6], P23[6];
            sylvester(tsq, t, e2 + e3, e2 * e3, k1, P1);
            for (int i = 0; i < 6; ++i) P23[i] = unit_dev(i) - P1[i];
            const double s1 = lame * I1 + 2.0 * shear * e1 - dl_r * (2.0 * lame * sp + 2.0 * shear * (1.0 + sp));
            const double s23 = lame * I1 + shear * (e2 + e3) - dl_r * (2.0 * lame * sp - shear * (1.0 - sp));
            for (int i = 0; i < 6; ++i) S[i] = s1 * P1[i] + s23 * P23[i];
            if (DS) {
                double dsq[36], nphi[6], npsi[6];
                dsq_dE(t, dsq);
                const double e23 = e2 + e3;
                for (int i = 0; i < 6; ++i) {
                    nphi[i] = shear * (2.0 * (1.0 + sin_phi) * P1[i] - (1.0 - sin_phi) * P23[i]) +
                              2.0 * lame * sin_phi * unit_dev(i);
                    npsi[i] = shear * (2.0 * (1.0 + sp) * P1[i] - (1.0 - sp) * P23[i]) +
                              2.0 * lame * sp * unit_dev(i);
                }
                const double inv_den = 1.0 / den_r;
                for (int j = 0; j < 6; ++j) {
                    for (int i = 0; i < 6; ++i) {
                        const int k = i + 6 * j;
                        const double hi = half_ident(i, j);
                        const double q11 = P1[i] * P1[j];
                        const double qmm = P23[i] * P23[j];
                        const double cross_t = P23[i] * t[j] + t[i] * P23[j];
                        const double cross_p = P23[i] * P1[j] + P1[i] * P23[j];
                        const double d1 = k1 * (dsq[k] - hi * e23 - cross_t + e23 * qmm +
                                                (e23 - 2.0 * e1) * q11 + e1 * cross_p);
                        DS[k] = (s1 - s23) * d1 + lame * unit_dev(i) * unit_dev(j) +
                                shear * (2.0 * q11 + qmm) - npsi[i] * nphi[j] * inv_den;
                    }
                }
            }
            return BR_RIGHT;
        }
    }

    /* ---- apex: hydrostatic stress c_bar / (2 sin phi), zero tangent ---- */
    {
        const double sa = c_bar / (2.0 * sin_phi);
        S[0] = S[1] = S[2] = sa;
        S[3] = S[4] = S[5] = 0.0;
        if (DS) memset(DS, 0, sizeof(double) * 36);
    }
    return BR_APEX;
}

/* ---------------------------------------------------------------- 2D */

static void outer3(const double *a, const double *b, double s, double *o)
{
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) o[i + 3 * j] = s * a[i] * b[j];
}

int orc_mc2d_point(const double *E, double c_bar, double sin_phi, double shear,
                   double bulk, double lame, double *S, double *DS)
{
    (void)bulk;
    /* in-plane eigenvalues of [e11, e12/2; e12/2, e22]; the out-of-plane value is 0 */
    const double tr = E[0] + E[1];
    const double rad = sqrt((E[0] - E[1]) * (E[0] - E[1]) + E[2] * E[2]);
    const double ua = 0.5 * (tr + rad), ub = 0.5 * (tr - rad), uc = 0.0;

    /* first derivatives (projections) and second derivatives of ua, ub */
    double Pa[4] = {1.0, 1.0, 0.0, 0.0};
    if (rad != 0.0) {
        Pa[0] = (E[0] - ub) / rad;
        Pa[1] = (E[1] - ub) / rad;
        Pa[2] = 0.5 * E[2] / rad;
    }
    const double Pb[4] = {1.0 - Pa[0], 1.0 - Pa[1], -Pa[2], 0.0};
    const double Pc[4] = {0.0, 0.0, 0.0, 1.0};
    double Ha[9] = {0}, Hb[9] = {0}, Hc[9] = {0};
    if (rad != 0.0) {
        const double inv = 1.0 / rad;
        const double one[3] = {1.0, 1.0, 0.5};
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                const double diag = (i == j) ? one[i] : 0.0;
                Ha[i + 3 * j] = (diag - Pa[j] * Pa[i] - Pb[j] * Pb[i]) * inv;
            }
        for (int k = 0; k < 9; ++k) Hb[k] = -Ha[k];
    }

    /* order e1 >= e2 >= e3 (same tie rules as the reference) */
    double e1 = ua, e2 = ub, e3 = uc;
    const double *p1 = Pa, *p2 = Pb, *p3 = Pc;
    const double *h1 = Ha, *h2 = Hb, *h3 = Hc;
    if (ua >= uc && uc > ub) {
        e2 = uc; e3 = ub;
        p2 = Pc; p3 = Pb;
        h2 = Hc; h3 = Hb;
    }
    if (uc > ua) {
        e1 = uc; e2 = ua; e3 = ub;
        p1 = Pc; p2 = Pa; p3 = Pb;
        h1 = Hc; h2 = Ha; h3 = Hb;
    }

    const double trE = e1 + e2 + e3;
    const double sp = sin_phi;
    const double f_tr = 2.0 * shear * ((1.0 + sp) * e1 - (1.0 - sp) * e3) + 2.0 * lame * sp * trE - c_bar;
    const double g_sl = (e1 - e2) / (1.0 + sp);
    const double g_sr = (e2 - e3) / (1.0 - sp);
    const double g_la = (e1 + e2 - 2.0 * e3) / (3.0 - sp);
    const double g_ra = (2.0 * e1 - e2 - e3) / (3.0 + sp);
    const double den_s = 4.0 * lame * sp * sp + 2.0 * shear * (1.0 + sp) * (1.0 + sp) +
                         2.0 * shear * (1.0 - sp) * (1.0 - sp);
    const double den_l = 4.0 * lame * sp * sp + shear * (1.0 + sp) * (1.0 + sp) +
                         2.0 * shear * (1.0 - sp) * (1.0 - sp);
    const double den_r = 4.0 * lame * sp * sp + 2.0 * shear * (1.0 + sp) * (1.0 + sp) +
                         shear * (1.0 - sp) * (1.0 - sp);
    const double dl_s = f_tr / den_s;
    const double dl_l = (shear * ((1.0 + sp) * (e1 + e2) - 2.0 * (1.0 - sp) * e3) + 2.0 * lame * sp * trE - c_bar) / den_l;
    const double dl_r = (shear * (2.0 * (1.0 + sp) * e1 - (1.0 - sp) * (e2 + e3)) + 2.0 * lame * sp * trE - c_bar) / den_r;

    int br;
    if (f_tr <= 0.0) br = BR_ELASTIC;
    else if (dl_s <= ((g_sl < g_sr) ? g_sl : g_sr)) br = BR_SMOOTH;
    else if (g_sl < g_sr && dl_l >= g_sl && dl_l <= g_la) br = BR_LEFT;
    else if (g_sl > g_sr && dl_r >= g_sr && dl_r <= g_ra) br = BR_RIGHT;
    else br = BR_APEX;

    static const double vol9[9] = {1, 1, 0, 1, 1, 0, 0, 0, 0};
    if (br == BR_ELASTIC) {
        const double v = E[0] + E[1];
        S[0] = lame * v + 2.0 * shear * E[0];
        S[1] = lame * v + 2.0 * shear * E[1];
        S[2] = shear * E[2];
        S[3] = lame * v;
        if (DS) {
            DS[0] = lame + 2.0 * shear; DS[1] = lame; DS[2] = 0.0;
            DS[3] = lame; DS[4] = lame + 2.0 * shear; DS[5] = 0.0;
            DS[6] = 0.0; DS[7] = 0.0; DS[8] = shear;
        }
        return br;
    }
    if (br == BR_SMOOTH) {
        const double s1 = lame * trE + 2.0 * shear * e1 - dl_s * (2.0 * lame * sp + 2.0 * shear * (1.0 + sp));
        const double s2 = lame * trE + 2.0 * shear * e2 - dl_s * (2.0 * lame * sp);
        const double s3 = lame * trE + 2.0 * shear * e3 - dl_s * (2.0 * lame * sp - 2.0 * shear * (1.0 - sp));
        for (int i = 0; i < 4; ++i) S[i] = s1 * p1[i] + s2 * p2[i] + s3 * p3[i];
        if (DS) {
            double n[3], o1[9], o2[9], o3[9], on[9];
            for (int i = 0; i < 3; ++i)
                n[i] = 2.0 * shear * (1.0 + sp) * p1[i] - 2.0 * shear * (1.0 - sp) * p3[i] + (i < 2 ? 2.0 * lame * sp : 0.0);
            outer3(p1, p1, 2.0 * shear, o1);
            outer3(p2, p2, 2.0 * shear, o2);
            outer3(p3, p3, 2.0 * shear, o3);
            outer3(n, n, 1.0 / den_s, on);
            for (int k = 0; k < 9; ++k)
                DS[k] = s1 * h1[k] + s2 * h2[k] + s3 * h3[k] + lame * vol9[k] + o1[k] + o2[k] + o3[k] - on[k];
        }
        return br;
    }
    if (br == BR_LEFT) {
        const double s12 = lame * trE + shear * (e1 + e2) - dl_l * (2.0 * lame * sp + shear * (1.0 + sp));
        const double s3 = lame * trE + 2.0 * shear * e3 - dl_l * (2.0 * lame * sp - 2.0 * shear * (1.0 - sp));
        for (int i = 0; i < 4; ++i) S[i] = s12 * (p1[i] + p2[i]) + s3 * p3[i];
        if (DS) {
            double p12[3], h12[9], n[3], o12[9], o3[9], on[9];
            for (int i = 0; i < 3; ++i) p12[i] = p1[i] + p2[i];
            for (int k = 0; k < 9; ++k) h12[k] = h1[k] + h2[k];
            for (int i = 0; i < 3; ++i)
                n[i] = shear * (1.0 + sp) * p12[i] - 2.0 * shear * (1.0 - sp) * p3[i] + (i < 2 ? 2.0 * lame * sp : 0.0);
            outer3(p12, p12, shear, o12);
            outer3(p3, p3, 2.0 * shear, o3);
            outer3(n, n, 1.0 / den_l, on);
            for (int k = 0; k < 9; ++k)
                DS[k] = s12 * h12[k] + s3 * h3[k] + lame * vol9[k] + o12[k] + o3[k] - on[k];
        }
        return br;
    }
    if (br == BR_RIGHT) {
        const double s1 = lame * trE + 2.0 * shear * e1 - dl_r * (2.0 * lame * sp + 2.0 * shear * (1.0 + sp));
        const double s23 = lame * trE + shear * (e2 + e3) - dl_r * (2.0 * lame * sp - shear * (1.0 - sp));
        for (int i = 0; i < 4; ++i) S[i] = s1 * p1[i] + s23 * (p2[i] + p3[i]);
        if (DS) {
            double p23[3], h23[9], n[3], o1[9], o23[9], on[9];
            for (int i = 0; i < 3; ++i) p23[i] = p2[i] + p3[i];
            for (int k = 0; k < 9; ++k) h23[k] = h2[k] + h3[k];
            for (int i = 0; i < 3; ++i)
                n[i] = 2.0 * shear * (1.0 + sp) * p1[i] - shear * (1.0 - sp) * p23[i] + (i < 2 ? 2.0 * lame * sp : 0.0);
            outer3(p1, p1, 2.0 * shear, o1);
            outer3(p23, p23, shear, o23);
            outer3(n, n, 1.0 / den_r, on);
            for (int k = 0; k < 9; ++k)
                DS[k] = s1 * h1[k] + s23 * h23[k] + lame * vol9[k] + o1[k] + o23[k] - on[k];
        }
        return br;
    }
    {
        const double sa = c_bar / (2.0 * sin_phi);
        S[0] = sa; S[1] = sa; S[2] = 0.0; S[3] = sa;
        if (DS) memset(DS, 0, sizeof(double) * 9);
    }
    return BR_APEX;
}

/* ------------------------------------------------------------ batch drivers */

void orc_constitutive3d(const double *E, const double *c_bar, const double *sin_phi,
                        const double *shear, const double *bulk, const double *lame,
                        int64_t n, double *S, double *DS, uint8_t *branch)
{
    (void)bulk;
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n; ++p) {
        int b = orc_mc3d_point(E + 6 * p, c_bar[p], sin_phi[p], shear[p], lame[p], S + 6 * p,
                               DS ? DS + 36 * p : NULL);
        if (branch) branch[p] = (uint8_t)b;
    }
}

void orc_constitutive2d(const double *E, const double *c_bar, const double *sin_phi,
                        const double *shear, const double *bulk, const double *lame,
                        int64_t n, double *S, double *DS, uint8_t *branch)
{
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n; ++p) {
        int b = orc_mc2d_point(E + 3 * p, c_bar[p], sin_phi[p], shear[p], bulk[p], lame[p],
                               S + 4 * p, DS ? DS + 9 * p : NULL);
        if (branch) branch[p] = (uint8_t)b;
    }
}

/* Davis-type strength reduction, +CONSTITUTIVE_PROBLEM/reduction.m:25-58. */
void orc_reduction(const double *c0, const double *phi, const double *psi, double lambda,
                   char davis, int64_t n, double *c_bar, double *sin_phi)
{
    for (int64_t p = 0; p < n; ++p) {
        double beta, c_l, phi_l;
        if (davis == 'A') {
            beta = cos(phi[p]) * cos(psi[p]) / (1.0 - sin(phi[p]) * sin(psi[p]));
            c_l = beta * c0[p] / lambda;
            phi_l = atan(beta * tan(phi[p]) / lambda);
        } else if (davis == 'B') {
            const double c1 = c0[p] / lambda;
            const double f1 = atan(tan(phi[p]) / lambda);
            const double s1 = atan(tan(psi[p]) / lambda);
            beta = cos(f1) * cos(s1) / (1.0 - sin(f1) * sin(s1));
            c_l = beta * c1;
            phi_l = atan(beta * tan(f1));
        } else {
            const double c1 = c0[p] / lambda;
            const double f1 = atan(tan(phi[p]) / lambda);
            beta = (f1 > psi[p]) ? cos(f1) * cos(psi[p]) / (1.0 - sin(f1) * sin(psi[p])) : 1.0;
            c_l = beta * c1;
            phi_l = atan(beta * tan(f1));
        }
        c_bar[p] = 2.0 * c_l * cos(phi_l);
        sin_phi[p] = sin(phi_l);
    }
}

/* -------------------------------------------------------- element assembly */

/* Local strain-displacement block for node i at one point: B[a][l], l = dim*i + comp.
 * 3D rows: e11, e22, e33, g12, g23, g13.  2D rows: e11, e22, g12.                  */
static void local_B(int dim, int n_p, const double *d1, const double *d2, const double *d3, double *B)
{
    const int ns = dim == 3 ? 6 : 3, nl = dim * n_p;
    memset(B, 0, sizeof(double) * (size_t)ns * nl);
    for (int i = 0; i < n_p; ++i) {
        if (dim == 3) {
            const int c = 3 * i;
            B[0 + ns * (c + 0)] = d1[i];
            B[1 + ns * (c + 1)] = d2[i];
            B[2 + ns * (c + 2)] = d3[i];
            B[3 + ns * (c + 0)] = d2[i];
            B[3 + ns * (c + 1)] = d1[i];
            B[4 + ns * (c + 1)] = d3[i];
            B[4 + ns * (c + 2)] = d2[i];
            B[5 + ns * (c + 0)] = d3[i];
            B[5 + ns * (c + 2)] = d1[i];
        } else {
            const int c = 2 * i;
            B[0 + ns * (c + 0)] = d1[i];
            B[1 + ns * (c + 1)] = d2[i];
            B[2 + ns * (c + 0)] = d2[i];
            B[2 + ns * (c + 1)] = d1[i];
        }
    }
}

/* V[map-1] += (sum_q B_q' (w_q D_q) B_q)  per element; V must be zeroed by caller. */
void orc_assemble(int dim, const double *DPhi1, const double *DPhi2, const double *DPhi3,
                  const double *DS, const double *W, const int64_t *smap, int n_p,
                  int64_t n_e, int n_q, double *V)
{
    const int ns = dim == 3 ? 6 : 3, nl = dim * n_p, nl2 = nl * nl;
    double *Ke = (double *)malloc(sizeof(double) * nl2);
    double *B = (double *)malloc(sizeof(double) * ns * nl);
    double *DB = (double *)malloc(sizeof(double) * ns * nl);
    for (int64_t e = 0; e < n_e; ++e) {
        memset(Ke, 0, sizeof(double) * nl2);
        for (int q = 0; q < n_q; ++q) {
            const int64_t g = e * n_q + q;
            local_B(dim, n_p, DPhi1 + g * n_p, DPhi2 + g * n_p, dim == 3 ? DPhi3 + g * n_p : NULL, B);
            const double *D = DS + g * ns * ns;
            for (int l = 0; l < nl; ++l)
                for (int a = 0; a < ns; ++a) {
                    double s = 0.0;
                    for (int b = 0; b < ns; ++b) s += W[g] * D[a + ns * b] * B[b + ns * l];
                    DB[a + ns * l] = s;
                }
            for (int c = 0; c < nl; ++c)
                for (int r = 0; r < nl; ++r) {
                    double s = 0.0;
                    for (int a = 0; a < ns; ++a) s += B[a + ns * r] * DB[a + ns * c];
                    Ke[r + nl * c] += s;
                }
        }
        const int64_t *m = smap + e * (int64_t)nl2;
        for (int k = 0; k < nl2; ++k)
            if (m[k] > 0) V[m[k] - 1] += Ke[k];
    }
    free(Ke);
    free(B);
    free(DB);
}
