/*
 * Oracle: plain-C FP64 restatement of PINY_MD's force path for flexible
 * water.  TEST INFRASTRUCTURE ONLY -- see piny_oracle.h.
 *
 * Build: gcc -O2 -ffp-contract=off (no FMA contraction, so the IEEE operation
 * order of every restated expression is the one PINY's gcc -O2 build uses on
 * x86-64, where doubles are not contracted either).
 */
#include "piny_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* NINT with SIMP_NINT: round half away from zero
 * (include/typ_defs/defines.h:96-97, SIMP_NINT set in
 * include/linux/standard_include.h). */
static inline double nint(double x)
{
    return (double)((int)((x) >= 0.0 ? ((x) + 0.5) : ((x)-0.5)));
}

/* ------------------------------------------------------------------------ */
/* Minimum image.                                                            */
/* period():      src/energy/control/period.c:27-114 (cubic branch :71-85,  */
/*                general branch :90-110)                                   */
/* period_pimd(): period.c:121-213, image shift from the mode-1 separation  */
/* ------------------------------------------------------------------------ */
static int is_cubic(const double *h)
{
    return h[1] == 0.0 && h[2] == 0.0 && h[3] == 0.0 && h[5] == 0.0 &&
           h[6] == 0.0 && h[7] == 0.0 && h[0] == h[4] && h[0] == h[8];
}

static void period_one(double *dx, double *dy, double *dz, const double *h,
                       const double *hi, int cubic)
{
    if (cubic) {
        double asx = *dx * hi[0], asy = *dy * hi[4], asz = *dz * hi[8];
        double sx = asx - nint(asx), sy = asy - nint(asy), sz = asz - nint(asz);
        *dx = sx * h[0];
        *dy = sy * h[4];
        *dz = sz * h[8];
    } else {
        double dxt = *dx, dyt = *dy, dzt = *dz;
        double asx = dxt * hi[0] + dyt * hi[3] + dzt * hi[6];
        double asy = dxt * hi[1] + dyt * hi[4] + dzt * hi[7];
        double asz = dxt * hi[2] + dyt * hi[5] + dzt * hi[8];
        double sx = asx - nint(asx), sy = asy - nint(asy), sz = asz - nint(asz);
        *dx = sx * h[0] + sy * h[3] + sz * h[6];
        *dy = sx * h[1] + sy * h[4] + sz * h[7];
        *dz = sx * h[2] + sy * h[5] + sz * h[8];
    }
}

static void period_pimd_one(double *dx, double *dy, double *dz, double dxs,
                            double dys, double dzs, const double *h,
                            const double *hi, int cubic)
{
    if (cubic) {
        double sx = -nint(dxs * hi[0]), sy = -nint(dys * hi[4]), sz = -nint(dzs * hi[8]);
        *dx += (sx * h[0]);
        *dy += (sy * h[4]);
        *dz += (sz * h[8]);
    } else {
        double asx = dxs * hi[0] + dys * hi[3] + dzs * hi[6];
        double asy = dxs * hi[1] + dys * hi[4] + dzs * hi[7];
        double asz = dxs * hi[2] + dys * hi[5] + dzs * hi[8];
        double sx = -nint(asx), sy = -nint(asy), sz = -nint(asz);
        *dx += (sx * h[0] + sy * h[3] + sz * h[6]);
        *dy += (sx * h[1] + sy * h[4] + sz * h[7]);
        *dz += (sx * h[2] + sy * h[5] + sz * h[8]);
    }
}

/* Inverse and determinant of the column-major cell, with the operation
 * order of gethinv's periodic branch (src/mathlib/mathlib.c:353-380). */
static double cell_inverse(const double *hm, double *hi)
{
    const double *h = hm - 1; /* 1-based view */
    double vol = (h[1] * (h[5] * h[9] - h[8] * h[6]) + h[4] * (h[8] * h[3] - h[2] * h[9]) +
                  h[7] * (h[2] * h[6] - h[5] * h[3]));
    hi[0] = (h[5] * h[9] - h[8] * h[6]) / vol;
    hi[4] = (h[1] * h[9] - h[7] * h[3]) / vol;
    hi[8] = (h[1] * h[5] - h[4] * h[2]) / vol;
    hi[3] = (h[7] * h[6] - h[4] * h[9]) / vol;
    hi[1] = (h[3] * h[8] - h[2] * h[9]) / vol;
    hi[6] = (h[4] * h[8] - h[7] * h[5]) / vol;
    hi[2] = (h[2] * h[6] - h[3] * h[5]) / vol;
    hi[7] = (h[7] * h[2] - h[8] * h[1]) / vol;
    hi[5] = (h[3] * h[4] - h[6] * h[1]) / vol;
    return vol;
}

/* ------------------------------------------------------------------------ */
/* PINY's erfc polynomial in t = 1/(1 + 0.3614 x)                           */
/* (src/interface/inter_params/spline_fit.c:314-398, the same coefficients  */
/*  appear in set_exclude.c:548-779 and energy_control_inter_real.c)        */
/* ------------------------------------------------------------------------ */
static const double EP = 0.3614;
static const double E1 = 0.2041422096422003, E2 = 0.1997535956961481;
static const double E3 = 0.2213176596405576, E4 = 0.03360430734640255;
static const double E5 = 0.4732592578721755, E6 = -0.509078520069735;
static const double E7 = 0.6772631491947646, E8 = -0.369912979092217;
static const double E9 = 0.06965131976970335;

static double gerfc_poly(double tt, double eee)
{
    return ((((((((E9 * tt + E8) * tt + E7) * tt + E6) * tt + E5) * tt + E4) * tt + E3) * tt + E2) * tt +
            E1) * tt * eee;
}

static double dgerfc_poly(double tt, double eee, double palp)
{
    double de1 = 1.0 * E1, de2 = 2.0 * E2, de3 = 3.0 * E3, de4 = 4.0 * E4, de5 = 5.0 * E5;
    double de6 = 6.0 * E6, de7 = 7.0 * E7, de8 = 8.0 * E8, de9 = 9.0 * E9;
    return ((((((((de9 * tt + de8) * tt + de7) * tt + de6) * tt + de5) * tt + de4) * tt + de3) * tt + de2) * tt +
            de1) * tt * tt * eee * palp;
}

/* ------------------------------------------------------------------------ */
/* spline_vdv (spline_fit.c:28-113) with vlj_bin (:149-177), vcoul_bin      */
/* (:314-398, periodic branch) and vnull_bin; itype 1 Coulomb, 2 LJ, 4 null */
/* ------------------------------------------------------------------------ */
void orc_spline_table(int nsplin, double rmin, double rmax, int itype,
                      double sig, double eps, double alp, double rheal,
                      int ishift, double *v, double *dv, double *dr_out,
                      double *dri_out)
{
    double dr = (rmax - rmin) / (double)(nsplin - 5);
    double dri = 1.0 / dr;
    double sig6 = sig * sig * sig * sig * sig * sig;
    double talp2 = 2.0 * alp * alp, palp = EP * alp;
    for (int i = 1; i <= nsplin; i++) {
        double r = dr * ((double)(i - 3)) + rmin;
        double sw = 1.0, dsw = 0.0;
        if (ishift == 2) {
            double rp = (r - rmax + rheal) / rheal;
            rp = rp < 1.0 ? rp : 1.0;
            rp = rp > 0.0 ? rp : 0.0;
            sw = 1.0 + rp * rp * (2.0 * rp - 3.0);
            dsw = -6.0 * (rp / rheal) * (rp - 1.0) / r;
        }
        double vnow = 0.0, dvnow = 0.0;
        if (itype == 2) {
            double r2 = r * r;
            double sig6r = sig6 / (r2 * r2 * r2);
            vnow = (eps * 4. * sig6r * (sig6r - 1.));
            dvnow = (eps * 24. * sig6r * (sig6r * 2. - 1.) / r2);
        } else if (itype == 1) {
            double r2 = r * r;
            double ralp = r * alp;
            double eee = exp(-ralp * ralp);
            double tt = 1.0 / (1.0 + EP * ralp);
            double gerfc = gerfc_poly(tt, eee);
            double dgerfc = dgerfc_poly(tt, eee, palp) + talp2 * gerfc * r;
            vnow = 1.0 * gerfc / r;
            dvnow = (gerfc / r2 + dgerfc / r) * 1.0 / r;
        }
        if (itype == 4) {
            v[i - 1] = 0.0;
            dv[i - 1] = 0.0;
        } else {
            v[i - 1] = vnow * sw;
            dv[i - 1] = dvnow * sw + vnow * dsw;
        }
    }
    if (ishift == 1) {
        double shift = v[nsplin - 3];
        for (int i = 0; i < nsplin; i++) v[i] -= shift;
    }
    *dr_out = dr;
    *dri_out = dri;
}

/* ------------------------------------------------------------------------ */
/* Ewald cutoff and k-sphere: calc_cutoff (set_cp_ewald.c:125-197),        */
/* countkvec3d (:304-427); the fill visits k in the same nested order.      */
/* ------------------------------------------------------------------------ */
double orc_ewald_ecut(int kmax, double deth)
{
    double rvol23 = pow(deth, -(2. / 3.));
    return M_PI * .5 * M_PI * (double)(kmax * kmax) * rvol23;
}

void orc_kmaxv(double ecut, const double *hi, int *kmaxv)
{
    for (int d = 0; d < 3; d++) {
        double d1 = hi[d], d2 = hi[d + 3], d3 = hi[d + 6];
        double tr = sqrt(d1 * d1 + d2 * d2 + d3 * d3);
        double temp = sqrt(ecut * .5) / (M_PI * tr);
        kmaxv[d] = (int)(2.0 * temp);
    }
}

static inline double ktry(double aka, double akb, double akc, const double *hi)
{
    const double tpi = 2.0 * M_PI;
    double xk = (aka * hi[0] + akb * hi[1] + akc * hi[2]) * tpi;
    double yk = (aka * hi[3] + akb * hi[4] + akc * hi[5]) * tpi;
    double zk = (aka * hi[6] + akb * hi[7] + akc * hi[8]) * tpi;
    return (xk * xk + yk * yk + zk * zk) * .5;
}

static int kvec_walk(double ecut, const int *kmaxv, const double *hi, int *ka_o, int *kb_o,
                     int *kc_o)
{
    int icount = 0, i, kamax = kmaxv[0];
    const double tpi = 2.0 * M_PI;
    for (i = 1; i <= kamax; ++i) {
        double aka = (double)i;
        double xk = aka * hi[0] * tpi, yk = aka * hi[3] * tpi, zk = aka * hi[6] * tpi;
        double tr = (xk * xk + yk * yk + zk * zk) * .5;
        if (tr > ecut * 4.) break;
    }
    kamax = i - 1;
    for (int ka = 0; ka <= kamax; ++ka) {
        double aka = (double)ka;
        int kbmin = -kmaxv[1];
        if (ka == 0) kbmin = 0;
        for (i = kbmin; i <= 0; ++i)
            if (ktry(aka, (double)i, 0.0, hi) <= ecut * 4.) break;
        kbmin = i;
        for (i = 1; i <= kmaxv[1]; ++i)
            if (ktry(aka, (double)i, 0.0, hi) > ecut * 4.) break;
        int kbmax = i - 1;
        for (int kb = kbmin; kb <= kbmax; ++kb) {
            double akb = (double)kb;
            int kcmin = -kmaxv[2];
            if (ka == 0 && kb == 0) kcmin = 1;
            for (i = kcmin; i <= 0; ++i)
                if (ktry(aka, akb, (double)i, hi) <= ecut * 4.) break;
            kcmin = i;
            for (i = 1; i <= kmaxv[2]; ++i)
                if (ktry(aka, akb, (double)i, hi) > ecut * 4.) break;
            int kcmax = i - 1;
            for (int kc = kcmin; kc <= kcmax; ++kc) {
                if (ka_o) {
                    ka_o[icount] = ka;
                    kb_o[icount] = kb;
                    kc_o[icount] = kc;
                }
                ++icount;
            }
        }
    }
    return icount;
}

int orc_kvec_count(double ecut, const int *kmaxv, const double *hi)
{
    return kvec_walk(ecut, kmaxv, hi, NULL, NULL, NULL);
}

int orc_kvec_fill(double ecut, const int *kmaxv, const double *hi, int *ka, int *kb, int *kc)
{
    return kvec_walk(ecut, kmaxv, hi, ka, kb, kc);
}

/* radixme (set_cp_ewald.c:815-1006), non-ESSL radix table 2^h 3^i 5^j:
 * the smallest allowed multiple-of-4 size >= 4*(k+1). */
static int radix_ok(int n)
{
    while (n % 2 == 0) n /= 2;
    while (n % 3 == 0) n /= 3;
    while (n % 5 == 0) n /= 5;
    return n == 1;
}

static int radix_up(int k)
{
    int n = (k + 1) * 4;
    while (!radix_ok(n)) n += 4;
    return n / 4 - 1;
}

/* set_pme_grid (set_cp_ewald.c:204-300) */
void orc_pme_grid(double ecut_now, double deth, const double *hi, const int *kmaxv, int kmax_pme,
                  int *ngrid)
{
    double rvol23 = pow(deth, -(2. / 3.));
    double ecut_pme = M_PI * .5 * M_PI * (double)(kmax_pme * kmax_pme) * rvol23;
    double ecut = ecut_pme > ecut_now ? ecut_pme : ecut_now;
    double temp[3];
    for (int d = 0; d < 3; d++) {
        double d1 = hi[d], d2 = hi[d + 3], d3 = hi[d + 6];
        double tr = sqrt(d1 * d1 + d2 * d2 + d3 * d3);
        temp[d] = sqrt(ecut * .5) / (M_PI * tr);
    }
    for (;;) {
        int go = 0;
        for (int d = 0; d < 3; d++) ngrid[d] = 4 * (radix_up((int)nint(temp[d])) + 1);
        for (int d = 0; d < 3; d++)
            if (ngrid[d] < 2 * (kmaxv[d] + 2)) { temp[d] += 1.0; go = 1; }
        if (!go) break;
    }
}

/* get_bspline_wght1d (set_cp_ewald.c:1288-1382) and set_pme_wght (:1136) */
static void bspline_weight_1d(int n_interp, int ngrid, double *bweight)
{
    double mn_k[64], uk[64], rn[64], rn1[64];
    for (int j = 1; j <= n_interp; j++) {
        rn[j] = (double)j;
        rn1[j] = j > 1 ? 1.0 / ((double)(j - 1)) : 0.0;
    }
    mn_k[1] = 1.0;
    uk[1] = 1.0;
    for (int k = 2; k <= n_interp; k++) { uk[k] = (double)k; mn_k[k] = 0.0; }
    for (int n = 3; n <= n_interp; n++) {
        for (int k = n; k >= 2; k--) mn_k[k] = (uk[k] * mn_k[k] + (rn[n] - uk[k]) * mn_k[k - 1]) * rn1[n];
        mn_k[1] = uk[1] * mn_k[1] * rn1[n];
    }
    double grid = (double)ngrid;
    double tpi_n = 2.0 * M_PI / grid;
    double tpi_n2 = 2.0 * M_PI * ((double)(n_interp - 1)) / grid;
    for (int m = 1; m <= ngrid; m++) {
        double br = 0.0, bi = 0.0;
        for (int k = 1; k <= n_interp - 1; k++) {
            double arg = tpi_n * ((double)((k - 1) * (m - 1)));
            br += cos(arg) * mn_k[k];
            bi += sin(arg) * mn_k[k];
        }
        double arg = tpi_n2 * ((double)(m - 1));
        double nr = cos(arg), ni = sin(arg);
        double denom = br * br + bi * bi;
        double tr = (nr * br + ni * bi) / denom;
        double ti = (ni * br - nr * bi) / denom;
        bweight[m - 1] = tr * tr + ti * ti;
    }
}

void orc_pme_bweight(int nk, const int *ka, const int *kb, const int *kc, const int *ngrid,
                     int n_interp, double *bw)
{
    double *wa = malloc(sizeof(double) * ngrid[0]);
    double *wb = malloc(sizeof(double) * ngrid[1]);
    double *wc = malloc(sizeof(double) * ngrid[2]);
    bspline_weight_1d(n_interp, ngrid[0], wa);
    bspline_weight_1d(n_interp, ngrid[1], wb);
    bspline_weight_1d(n_interp, ngrid[2], wc);
    for (int i = 0; i < nk; i++) {
        int a = ka[i] < 0 ? ka[i] + ngrid[0] : ka[i];
        int b = kb[i] < 0 ? kb[i] + ngrid[1] : kb[i];
        int c = kc[i] < 0 ? kc[i] + ngrid[2] : kc[i];
        bw[i] = wa[a] * wb[b] * wc[c];
    }
    free(wa); free(wb); free(wc);
}

/* Gauss-Legendre nodes/weights on [-1,1], ascending, by Newton iteration on
 * P_n (the 128-point rule splin_ecor uses, set_exclude.c:690). */
void orc_gauss_legendre(int n, double *node, double *weight)
{
    for (int i = 0; i < (n + 1) / 2; i++) {
        double x = cos(M_PI * (i + 0.75) / (n + 0.5)), pp = 0.0;
        for (int it = 0; it < 100; it++) {
            double p0 = 1.0, p1 = x;
            for (int k = 2; k <= n; k++) {
                double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            pp = n * (x * p1 - p0) / (x * x - 1.0);
            double dx = p1 / pp;
            x -= dx;
            if (fabs(dx) < 1e-16) break;
        }
        {
            double p0 = 1.0, p1 = x;
            for (int k = 2; k <= n; k++) {
                double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            pp = n * (x * p1 - p0) / (x * x - 1.0);
        }
        double w = 2.0 / ((1.0 - x * x) * pp * pp);
        node[i] = -x;
        node[n - 1 - i] = x;
        weight[i] = w;
        weight[n - 1 - i] = w;
    }
}

/* splin_ecor (src/interface/lists/set_exclude.c:548-779): -erf(alpha r)/r
 * on nsplin points from rmin = 0.1 to rmax, plus the finite-k correction
 * integrated with 128-point Gauss-Legendre between kcut and 15 alpha. */
void orc_ecor_table(int nsplin, double rmax, double alp, double ecut, double *cv0, double *cdv0,
                    double *dr_out, double *dri_out, double *self_erf)
{
    double rmin = 0.1;
    double dr = (rmax - rmin) / (double)(nsplin - 5), dri = 1.0 / dr;
    double alp2 = alp * alp, talp2 = 2.0 * alp * alp, palp = EP * alp;
    for (int i = 1; i <= nsplin; ++i) {
        double r12 = dr * (double)(i - 3) + rmin;
        double r12i = 1.0 / r12;
        double ralp = r12 * alp;
        double eee = exp(-ralp * ralp);
        double tt = 1.0 / (1.0 + EP * ralp);
        double temp = gerfc_poly(tt, eee);
        double gerf = 1.0 - temp;
        double dgerf = dgerfc_poly(tt, eee, palp) + talp2 * temp * r12;
        cv0[i - 1] = -gerf * r12i;
        double dvecor = -(dgerf * r12i - gerf / (r12 * r12));
        cdv0[i - 1] = -dvecor * r12i;
    }
    enum { NK = 128 };
    double anode[NK], weight[NK], know[NK], fknow[NK];
    orc_gauss_legendre(NK, anode, weight);
    double kcut = sqrt(2.0 * ecut);
    double arg = kcut / (2.0 * alp);
    double eee = exp(-arg * arg);
    double tt = 1.0 / (1.0 + EP * arg);
    *self_erf = 1.0 - gerfc_poly(tt, eee);
    double kmax = 15.0 * alp;
    if (kmax > kcut) {
        double dk = (kmax - kcut), pk = (kmax + kcut);
        for (int k = 0; k < NK; k++) {
            know[k] = 0.5 * (anode[k] * dk + pk);
            fknow[k] = (dk / M_PI) * exp(-0.25 * know[k] * know[k] / alp2) * weight[k];
        }
        for (int i = 1; i <= nsplin; ++i) {
            double r12 = dr * (double)(i - 3) + rmin;
            double chi = 0.0, dchi = 0.0;
            for (int k = 0; k < NK; k++) {
                double a = know[k] * r12;
                double j0 = (sin(a) / a);
                double j1 = (sin(a) / a - cos(a)) / a;
                chi += (fknow[k] * j0);
                dchi += (know[k] * fknow[k] * j1 / r12);
            }
            cv0[i - 1] += chi;
            cdv0[i - 1] += dchi;
        }
    }
    *dr_out = dr;
    *dri_out = dri;
}

/* bond_coef "power" (src/interface/intra_params/intra_coefs.c:120-160) and
 * the derivative coefficients (:183-190); inputs already in Hartree/Bohr^n */
void orc_bond_power(double c2, double c3, double c4, double *c, double *dc)
{
    for (int i = 0; i < 7; i++) c[i] = 0.0;
    c[2] = c2;
    c[3] = c3;
    c[4] = c4;
    dc[0] = 0.0;
    dc[1] = c[1];
    for (int i = 2; i < 7; i++) dc[i] = (double)i * c[i];
}

/* bend_coef "harm" (intra_coefs.c:240-276, derivatives :355-371):
 * 0.5 k (theta-theta0)^2 expanded in cos/sin to sixth order. */
void orc_bend_harm(double fk, double theta_0, double *c, double *s, double *dc, double *ds)
{
    const double cn1 = 49.0 / 72.0, cn2 = 3.0 / 4.0, cn3 = 3.0 / 40.0, cn4 = 1.0 / 180.0;
    const double cn5 = 3.0 / 2.0, cn6 = 3.0 / 5.0, cn7 = 1.0 / 10.0, cn8 = 4.0 / 15.0;
    const double cn9 = 8.0 / 45.0, cn10 = 3.0 / 10.0, cn11 = 1.0 / 30.0;
    double c2t = cos(2.0 * theta_0), c4t = cos(4.0 * theta_0), c6t = cos(6.0 * theta_0);
    double s2t = sin(2.0 * theta_0), s4t = sin(4.0 * theta_0), s6t = sin(6.0 * theta_0);
    c[0] = 0.5 * fk * (cn1 + cn2 * c2t + cn3 * c4t + cn4 * c6t);
    c[1] = 0.0;
    c[2] = 0.5 * fk * (-cn5 * c2t - cn6 * c4t - cn7 * c6t);
    c[3] = 0.0;
    c[4] = 0.5 * fk * (cn6 * c4t + cn8 * c6t);
    c[5] = 0.0;
    c[6] = 0.5 * fk * (-cn9 * c6t);
    s[0] = 0.0;
    s[1] = 0.0;
    s[2] = 0.5 * fk * (-cn5 * s2t + cn10 * s4t - cn11 * s6t);
    s[3] = 0.0;
    s[4] = 0.5 * fk * (-cn6 * s4t + cn9 * s6t);
    s[5] = 0.0;
    s[6] = 0.5 * fk * (-cn9 * s6t);
    dc[0] = 0.0;
    dc[1] = c[1];
    for (int i = 2; i < 7; i++) dc[i] = (double)i * c[i];
    ds[0] = 0.0;
    ds[1] = s[1];
    ds[2] = s[2];
    for (int i = 3; i < 7; i++) ds[i] = (double)(i - 1) * s[i];
}

/* get_clong (src/interface/inter_params/get_clong.c:27-118), swit branch;
 * c6 and cutoff are per pair type in PINY's upper-triangle order. */
double orc_clong(int natm, int ntyp, const int *atm_typ, const double *c6, const double *cutoff,
                 double rheal, int iswit)
{
    long *num = calloc((size_t)ntyp, sizeof(long));
    for (int i = 0; i < natm; i++) num[atm_typ[i]]++;
    int npair = ntyp * (ntyp + 1) / 2;
    double *cm = calloc((size_t)npair, sizeof(double));
    int ntype1 = ntyp + 1;
    for (int i = 1; i <= ntyp; i++) {
        for (int j = 1; j <= i; j++) {
            int idx = ((j - 1) * (2 * ntype1 - j)) / 2 + i - j + 1;
            if (j < i) cm[idx - 1] = (double)(num[i - 1] * num[j - 1]);
            else cm[idx - 1] = (double)((num[i - 1] * (num[i - 1] - 1)) / 2);
        }
    }
    double clong = 0.0, fpi = 4.0 * M_PI, fpi3 = 4.0 * M_PI / 3.0;
    for (int p = 0; p < npair; p++) {
        double rc = cutoff[p];
        if (!iswit) {
            clong -= fpi3 * c6[p] * cm[p] / pow(rc, 3.0);
        } else if (c6[p] > 0 && rc - rheal > 0) {
            double fact = (1.0 / (rheal * rheal)) * (1.0 / rc + 1.0 / (rc - rheal)) +
                          (2.0 / (rheal * rheal * rheal)) * log((rc - rheal) / rc);
            clong -= (fpi * c6[p] * cm[p] * fact);
        }
    }
    free(num);
    free(cm);
    return clong;
}

/* ------------------------------------------------------------------------ */
/* Pair type of two atoms (force_npol.c:585-599, npol_posdata_fetch)        */
/* ------------------------------------------------------------------------ */
static inline int pair_type(int ti, int tj, int ntyp)
{
    int i2 = ti + 1, i3 = tj + 1;
    int jj = i2 < i3 ? i2 : i3;
    int ii = i2 + i3 - jj;
    int kk = ((jj - 1) * ((ntyp + 1) * 2 - jj)) / 2;
    return kk + ii - jj; /* 0-based */
}

/* ------------------------------------------------------------------------ */
/* Verlet list (verlist_create.c:25-221 with vercreate_list_count_fill      */
/* :373-503): every non-excluded pair i > j whose bead-1 minimum-image      */
/* separation satisfies r^2 < cutskin^2 of its pair type.  Brute force;     */
/* PINY's link cells only enumerate candidates, the accepted set is this.   */
/* ------------------------------------------------------------------------ */
/* Rows i in [ilo, ihi) of the list below. */
long orc_verlist_rows(const orc_system *s, const double *x, const double *y, const double *z,
                      const double *xmod, const double *ymod, const double *zmod, const double *h,
                      const double *cutskin2, int ilo, int ihi, long cap, int *pi, int *pj)
{
    double hi[9];
    cell_inverse(h, hi);
    int cubic = is_cubic(h);
    long n = 0;
    char *ex = calloc((size_t)s->natm, 1);
    if (ilo < 1) ilo = 1;
    if (ihi > s->natm) ihi = s->natm;
    for (int i = ilo; i < ihi; i++) {
        for (int e = s->excl_off[i]; e < s->excl_off[i + 1]; e++) ex[s->excl_j[e]] = 1;
        for (int j = 0; j < i; j++) {
            if (ex[j]) continue;
            double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
            if (xmod)
                period_pimd_one(&dx, &dy, &dz, xmod[i] - xmod[j], ymod[i] - ymod[j], zmod[i] - zmod[j],
                                h, hi, cubic);
            else
                period_one(&dx, &dy, &dz, h, hi, cubic);
            double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < cutskin2[pair_type(s->atm_typ[i], s->atm_typ[j], s->ntyp)]) {
                if (n < cap) { pi[n] = i; pj[n] = j; }
                n++;
            }
        }
        for (int e = s->excl_off[i]; e < s->excl_off[i + 1]; e++) ex[s->excl_j[e]] = 0;
    }
    free(ex);
    return n;
}

long orc_verlist(const orc_system *s, const double *x, const double *y, const double *z,
                 const double *xmod, const double *ymod, const double *zmod, const double *h,
                 const double *hi_unused, const double *cutskin2, long cap, int *pi, int *pj)
{
    (void)hi_unused;
    return orc_verlist_rows(s, x, y, z, xmod, ymod, zmod, h, cutskin2, 1, s->natm, cap, pi, pj);
}

/* 4-point cubic of npol_vspl_fetch (force_npol.c:339-375); table is 0-based
 * storage of PINY's 1-based c0_data, k the 1-based knot index. */
static inline double vspl(const double *t, int k, double del)
{
    const double oneth = (1.0 / 3.0), onesi = (1.0 / 6.0);
    double c0 = t[k - 1], fp1 = t[k], fm1 = t[k - 2], fm2 = t[k - 3];
    double c1 = oneth * fp1 + 0.5 * c0 - fm1 + onesi * fm2;
    double c2 = 0.5 * fp1 - c0 + 0.5 * fm1;
    double c3 = onesi * fp1 - 0.5 * c0 + 0.5 * fm1 - onesi * fm2;
    return (c0 + del * (c1 + del * (c2 + del * c3)));
}

/* ------------------------------------------------------------------------ */
/* Plain complex 3D DFT used by the PME restatement (the sign convention    */
/* cancels between the two transforms; see ewald3d_pme.c:362 and :434).     */
/* ------------------------------------------------------------------------ */
static void dft1(double *re, double *im, int n, int stride, int sign, double *tr, double *ti,
                 const double *cs, const double *sn)
{
    for (int k = 0; k < n; k++) {
        double sr = 0.0, si = 0.0;
        for (int j = 0; j < n; j++) {
            int e = (int)(((long)j * k) % n);
            double c = cs[e], s = sign * sn[e];
            double xr = re[(long)j * stride], xi = im[(long)j * stride];
            sr += xr * c - xi * s;
            si += xr * s + xi * c;
        }
        tr[k] = sr;
        ti[k] = si;
    }
    for (int k = 0; k < n; k++) {
        re[(long)k * stride] = tr[k];
        im[(long)k * stride] = ti[k];
    }
}

static void fft1(double *re, double *im, int n, int stride, int sign, double *tr, double *ti,
                 const double *cs, const double *sn)
{
    if (n & (n - 1)) { dft1(re, im, n, stride, sign, tr, ti, cs, sn); return; }
    for (int k = 0; k < n; k++) { tr[k] = re[(long)k * stride]; ti[k] = im[(long)k * stride]; }
    for (int i = 1, j = 0; i < n; i++) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = tr[i]; tr[i] = tr[j]; tr[j] = t;
            t = ti[i]; ti[i] = ti[j]; ti[j] = t;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        int step = n / len;
        for (int i = 0; i < n; i += len) {
            for (int k = 0; k < len / 2; k++) {
                double c = cs[k * step], s = sign * sn[k * step];
                double ur = tr[i + k], ui = ti[i + k];
                double vr = tr[i + k + len / 2] * c - ti[i + k + len / 2] * s;
                double vi = tr[i + k + len / 2] * s + ti[i + k + len / 2] * c;
                tr[i + k] = ur + vr; ti[i + k] = ui + vi;
                tr[i + k + len / 2] = ur - vr; ti[i + k + len / 2] = ui - vi;
            }
        }
    }
    for (int k = 0; k < n; k++) { re[(long)k * stride] = tr[k]; im[(long)k * stride] = ti[k]; }
}

static void fft3(double *re, double *im, const int *N, int sign)
{
    int maxn = N[0] > N[1] ? N[0] : N[1];
    if (N[2] > maxn) maxn = N[2];
    double *tr = malloc(sizeof(double) * maxn), *ti = malloc(sizeof(double) * maxn);
    double *cs = malloc(sizeof(double) * maxn), *sn = malloc(sizeof(double) * maxn);
    int Na = N[0], Nb = N[1], Nc = N[2];
    for (int d = 0; d < 3; d++) {
        int n = N[d];
        for (int k = 0; k < n; k++) {
            cs[k] = cos(2.0 * M_PI * k / n);
            sn[k] = sin(2.0 * M_PI * k / n);
        }
        if (d == 0)
            for (long o = 0; o < (long)Nb * Nc; o++) fft1(re + o * Na, im + o * Na, Na, 1, sign, tr, ti, cs, sn);
        if (d == 1)
            for (int c = 0; c < Nc; c++)
                for (int a = 0; a < Na; a++) {
                    long o = (long)c * Na * Nb + a;
                    fft1(re + o, im + o, Nb, Na, sign, tr, ti, cs, sn);
                }
        if (d == 2)
            for (long o = 0; o < (long)Na * Nb; o++) fft1(re + o, im + o, Nc, Na * Nb, sign, tr, ti, cs, sn);
    }
    free(tr); free(ti); free(cs); free(sn);
}

/* ------------------------------------------------------------------------ */
/* PME for one bead: ewald3d_recip_pme_none (recip3d/ewald3d_pme.c:95-600)  */
/* ------------------------------------------------------------------------ */
static double pme_bead(const orc_system *s, const double *pos, const double *h, const double *hi,
                       double vol, double *f, double *pv)
{
    int Na = s->ngrid_a, Nb = s->ngrid_b, Nc = s->ngrid_c, n = s->n_interp;
    long G = (long)Na * Nb * Nc;
    double *re = calloc((size_t)G, sizeof(double)), *im = calloc((size_t)G, sizeof(double));
    double grid_a = Na, grid_b = Nb, grid_c = Nc;
    double mna[64], mnb[64], mnc[64], ua[64], ub[64], uc[64], dmna[64], dmnb[64], dmnc[64];
    int ga[64], gb[64], gc[64];
    double rn[64], rn1[64];
    for (int j = 1; j <= n; j++) { rn[j] = (double)j; rn1[j] = j > 1 ? 1.0 / ((double)(j - 1)) : 0.0; }

    /* scaled coordinates (:231-256) and B-splines (:274-338) */
    for (int pass = 0; pass < 2; pass++) {
        for (int iat = 0; iat < s->natm; iat++) {
            double q = s->charge[iat];
            if (q == 0.0) continue; /* PINY loops over ichrg only */
            const double *r = pos + 3 * (long)iat;
            double at = r[0] * hi[0] + r[1] * hi[3] + r[2] * hi[6];
            double bt = r[0] * hi[1] + r[1] * hi[4] + r[2] * hi[7];
            double ct = r[0] * hi[2] + r[1] * hi[5] + r[2] * hi[8];
            at = at - nint((at - 0.5));
            bt = bt - nint((bt - 0.5));
            ct = ct - nint((ct - 0.5));
            double xs = at * grid_a, ys = bt * grid_b, zs = ct * grid_c;
            int ia = (int)xs, ib = (int)ys, ic = (int)zs;
            double fa = xs - (double)ia, fb = ys - (double)ib, fc = zs - (double)ic;
            for (int j = 1; j <= n; j++) {
                ua[j] = fa + (double)(j - 1);
                ub[j] = fb + (double)(j - 1);
                uc[j] = fc + (double)(j - 1);
                int a = ia - (j - 2), b = ib - (j - 2), c = ic - (j - 2);
                a = a > 0 ? a : Na + a;
                b = b > 0 ? b : Nb + b;
                c = c > 0 ? c : Nc + c;
                ga[j] = a - 1;
                gb[j] = b - 1;
                gc[j] = c - 1;
            }
            mna[1] = 1.0 - fabs(ua[1] - 1.0); mnb[1] = 1.0 - fabs(ub[1] - 1.0); mnc[1] = 1.0 - fabs(uc[1] - 1.0);
            mna[2] = 1.0 - fabs(ua[2] - 1.0); mnb[2] = 1.0 - fabs(ub[2] - 1.0); mnc[2] = 1.0 - fabs(uc[2] - 1.0);
            for (int j = 3; j <= n; j++) mna[j] = mnb[j] = mnc[j] = 0.0;
            for (int m = 3; m <= n; m++) {
                for (int j = m; j >= 2; j--) {
                    double ta = (ua[j] * mna[j] + (rn[m] - ua[j]) * mna[j - 1]) * rn1[m];
                    double tb = (ub[j] * mnb[j] + (rn[m] - ub[j]) * mnb[j - 1]) * rn1[m];
                    double tc = (uc[j] * mnc[j] + (rn[m] - uc[j]) * mnc[j - 1]) * rn1[m];
                    mna[j] = ta; mnb[j] = tb; mnc[j] = tc;
                }
                mna[1] = ua[1] * mna[1] * rn1[m];
                mnb[1] = ub[1] * mnb[1] * rn1[m];
                mnc[1] = uc[1] * mnc[1] * rn1[m];
                if (m == n - 1) {
                    dmna[1] = mna[1]; dmnb[1] = mnb[1]; dmnc[1] = mnc[1];
                    for (int j = 2; j <= n; j++) {
                        dmna[j] = mna[j] - mna[j - 1];
                        dmnb[j] = mnb[j] - mnb[j - 1];
                        dmnc[j] = mnc[j] - mnc[j - 1];
                    }
                }
            }
            if (pass == 0) {
                /* spread (:340-357) */
                for (int jc = 1; jc <= n; jc++)
                    for (int jb = 1; jb <= n; jb++)
                        for (int ja = 1; ja <= n; ja++) {
                            long g = ((long)gc[jc] * Nb + gb[jb]) * Na + ga[ja];
                            re[g] += mna[ja] * mnb[jb] * mnc[jc] * q;
                        }
            } else {
                /* gather (:534-559) */
                double fx = 0.0, fy = 0.0, fz = 0.0;
                for (int jc = 1; jc <= n; jc++)
                    for (int jb = 1; jb <= n; jb++)
                        for (int ja = 1; ja <= n; ja++) {
                            long g = ((long)gc[jc] * Nb + gb[jb]) * Na + ga[ja];
                            double at2 = dmna[ja] * mnb[jb] * mnc[jc] * grid_a;
                            double bt2 = mna[ja] * dmnb[jb] * mnc[jc] * grid_b;
                            double ct2 = mna[ja] * mnb[jb] * dmnc[jc] * grid_c;
                            double qdx = at2 * hi[0] + bt2 * hi[1] + ct2 * hi[2];
                            double qdy = at2 * hi[3] + bt2 * hi[4] + ct2 * hi[5];
                            double qdz = at2 * hi[6] + bt2 * hi[7] + ct2 * hi[8];
                            double qn = re[g] * q;
                            fx -= (qdx * qn);
                            fy -= (qdy * qn);
                            fz -= (qdz * qn);
                        }
                f[3 * (long)iat] += fx;
                f[3 * (long)iat + 1] += fy;
                f[3 * (long)iat + 2] += fz;
            }
        }
        if (pass == 0) {
            int N[3] = {Na, Nb, Nc};
            fft3(re, im, N, +1);
            /* k-sphere energy, virial, convolution (:366-425) */
            double *tre = calloc((size_t)G, sizeof(double)), *tim = calloc((size_t)G, sizeof(double));
            double falp2 = 4.0 * s->alp_ewd * s->alp_ewd, tpi = 2.0 * M_PI, pivol = vol / (4.0 * M_PI);
            double vnow = 0.0, pt[9] = {0};
            for (int i = 0; i < s->nktot; i++) {
                double aka = tpi * ((double)s->kastr[i]), akb = tpi * ((double)s->kbstr[i]),
                       akc = tpi * ((double)s->kcstr[i]);
                double xk = (aka * hi[0] + akb * hi[1] + akc * hi[2]);
                double yk = (aka * hi[3] + akb * hi[4] + akc * hi[5]);
                double zk = (aka * hi[6] + akb * hi[7] + akc * hi[8]);
                double g2 = xk * xk + yk * yk + zk * zk;
                double preg = exp((-g2 / falp2)) / (g2 * pivol);
                double prep = -2.0 * preg * ((g2 / falp2) + 1.0) / g2;
                int a = ((s->kastr[i] % Na) + Na) % Na, b = ((s->kbstr[i] % Nb) + Nb) % Nb,
                    c = ((s->kcstr[i] % Nc) + Nc) % Nc;
                long g = ((long)c * Nb + b) * Na + a;
                double sr = re[g], si = im[g];
                double smag = (sr * sr + si * si) * s->bweight[i];
                vnow += (smag * preg);
                prep *= smag;
                pt[0] += prep * xk * xk;
                pt[4] += prep * yk * yk;
                pt[8] += prep * zk * zk;
                pt[1] += prep * xk * yk;
                pt[2] += prep * xk * zk;
                pt[5] += prep * yk * zk;
                double w = preg * s->bweight[i];
                tre[g] = sr * w;
                tim[g] = si * w;
                int am = (Na - a) % Na, bm = (Nb - b) % Nb, cm = (Nc - c) % Nc;
                long gm = ((long)cm * Nb + bm) * Na + am;
                tre[gm] = sr * w;
                tim[gm] = -(si * w);
            }
            pt[3] = pt[1];
            pt[6] = pt[2];
            pt[7] = pt[5];
            pt[0] += vnow;
            pt[4] += vnow;
            pt[8] += vnow;
            for (int i = 0; i < 9; i++) pv[i] += pt[i];
            fft3(tre, tim, N, -1);
            free(re);
            free(im);
            re = tre;
            im = tim;
            /* stash the energy in im[0]'s slot via the return path below */
            pv[9] = vnow;
        }
    }
    free(re);
    free(im);
    return pv[9];
}

/* ------------------------------------------------------------------------ */
/* One full evaluation over all beads: the sub-steps of energy_control_pimd */
/* (energy_control_pimd.c:91-111) with full inter/intra and no RESPA.       */
/* ------------------------------------------------------------------------ */
void orc_energy_force(const orc_system *s, int P, const double *pos_in, const double *xmod,
                      const double *h, long npairs, const int *pi, const int *pj,
                      int distribute_ghosts, double *force, orc_energies *e)
{
    double hi[9];
    double vol = cell_inverse(h, hi);
    int cubic = is_cubic(h);
    long natm = s->natm;
    memset(e, 0, sizeof(*e));
    double pv[10] = {0};
    double vreal_s = 0, vvdw_s = 0, vcoul_s = 0, vrecip_s = 0, vecor_s = 0, vbond_s = 0, vbend_s = 0;
    double *pos = malloc(sizeof(double) * 3 * natm);
    int npair_typ = s->ntyp * (s->ntyp + 1) / 2;
    (void)npair_typ;

    for (int b = 0; b < P; b++) {
        memcpy(pos, pos_in + 3 * natm * b, sizeof(double) * 3 * natm);
        double *f = force + 3 * natm * b;
        memset(f, 0, sizeof(double) * 3 * natm);

        /* get_ghost_pos (intra_con/ghost_control.c:28-69) */
        for (int g = 0; g < s->nghost; g++) {
            int gl = s->ghost_atom[g];
            double gx = 0.0, gy = 0.0, gz = 0.0;
            for (int c = 0; c < s->ghost_ncomp; c++) {
                int a = s->ghost_comp[g * s->ghost_ncomp + c];
                if (a < 0) continue;
                double cf = s->ghost_coef[g * s->ghost_ncomp + c];
                gx += cf * pos[3 * a];
                gy += cf * pos[3 * a + 1];
                gz += cf * pos[3 * a + 2];
            }
            pos[3 * gl] = gx; pos[3 * gl + 1] = gy; pos[3 * gl + 2] = gz;
        }

        /* real space: force_npol (force_npol.c:28-329) over the shared list */
        for (long p = 0; p < npairs; p++) {
            int i = pi[p], j = pj[p];
            double dx = pos[3 * i] - pos[3 * j], dy = pos[3 * i + 1] - pos[3 * j + 1],
                   dz = pos[3 * i + 2] - pos[3 * j + 2];
            if (P > 1)
                period_pimd_one(&dx, &dy, &dz, xmod[3 * i] - xmod[3 * j], xmod[3 * i + 1] - xmod[3 * j + 1],
                                xmod[3 * i + 2] - xmod[3 * j + 2], h, hi, cubic);
            else
                period_one(&dx, &dy, &dz, h, hi, cubic);
            double r = sqrt((dx * dx + dy * dy + dz * dz));
            int pt = pair_type(s->atm_typ[i], s->atm_typ[j], s->ntyp);
            if (!(r < s->cutoff[pt])) continue; /* npol_shave_skin (:1291-1390) */
            int u = s->inter_map[pt];
            double rmin = s->rmin_spl[u], dr = s->dr_spl[u], dri = s->dri_spl[u];
            int k = (int)(((r - rmin) * dri) + 0.5) + 3;
            k = k < s->nsplin - 2 ? k : s->nsplin - 2;
            k = k > 3 ? k : 3;
            double rsp = ((double)(k - 3)) * dr + rmin;
            double del = (r - rsp) * dri;
            long off = (long)u * s->nsplin;
            double q2 = s->charge[i] * s->charge[j];
            double vv = vspl(s->cv0 + off, k, del);
            double vc = q2 * vspl(s->cv0_c + off, k, del);
            double dvtemp = (q2 * vspl(s->cdv0_c + off, k, del) + vspl(s->cdv0 + off, k, del));
            double fx = dx * dvtemp, fy = dy * dvtemp, fz = dz * dvtemp;
            f[3 * i] += fx; f[3 * i + 1] += fy; f[3 * i + 2] += fz;
            f[3 * j] -= fx; f[3 * j + 1] -= fy; f[3 * j + 2] -= fz;
            vvdw_s += vv;
            vcoul_s += vc;
            vreal_s += vv + vc;
            pv[0] += dx * fx; pv[4] += dy * fy; pv[8] += dz * fz;
            pv[1] += dx * fy; pv[2] += dx * fz; pv[5] += dy * fz;
        }

        /* PME reciprocal space */
        if (s->nktot > 0) {
            double pvr[10] = {0};
            vrecip_s += pme_bead(s, pos, h, hi, vol, f, pvr);
            for (int c = 0; c < 9; c++) pv[c] += pvr[c];
        }

        /* Ewald exclusion correction: ecor (intra/ecorr.c:28-274) */
        for (int c = 0; c < s->necor; c++) {
            int a = s->ecor_j1[c], bb = s->ecor_j2[c];
            double dx = pos[3 * a] - pos[3 * bb], dy = pos[3 * a + 1] - pos[3 * bb + 1],
                   dz = pos[3 * a + 2] - pos[3 * bb + 2];
            double r = sqrt(dx * dx + dy * dy + dz * dz);
            int k = (int)(((r - s->ecor_rmin) * s->ecor_dri) + 0.5) + 3;
            k = k < s->ecor_nsplin - 2 ? k : s->ecor_nsplin - 2;
            k = k > 3 ? k : 3;
            double rsp = ((double)(k - 3)) * s->ecor_dr + s->ecor_rmin;
            double del = (r - rsp) * s->ecor_dri;
            double q12 = s->charge[a] * s->charge[bb];
            vecor_s += vspl(s->ecor_cv0, k, del) * q12;
            double dvt = vspl(s->ecor_cdv0, k, del) * q12;
            double fx = dx * dvt, fy = dy * dvt, fz = dz * dvt;
            f[3 * a] += fx; f[3 * a + 1] += fy; f[3 * a + 2] += fz;
            f[3 * bb] -= fx; f[3 * bb + 1] -= fy; f[3 * bb + 2] -= fz;
            pv[0] += dx * fx; pv[4] += dy * fy; pv[8] += dz * fz;
            pv[1] += dx * fy; pv[2] += dx * fz; pv[5] += dy * fz;
        }

        /* bonds: bond_both (intra/bond_both.c:29-420) */
        for (int c = 0; c < s->nbond; c++) {
            int a = s->bond_j1[c], bb = s->bond_j2[c], t = s->bond_typ[c];
            const double *cc = s->bond_c + 7 * t, *dc = s->bond_dc + 7 * t;
            double dx = pos[3 * a] - pos[3 * bb], dy = pos[3 * a + 1] - pos[3 * bb + 1],
                   dz = pos[3 * a + 2] - pos[3 * bb + 2];
            double r = sqrt(dx * dx + dy * dy + dz * dz);
            double rr0 = r - s->bond_eq[t];
            double v = (((((cc[6] * rr0 + cc[5]) * rr0 + cc[4]) * rr0 + cc[3]) * rr0 + cc[2]) * rr0 + cc[1]) * rr0 +
                       cc[0];
            double dv = ((((dc[6] * rr0 + dc[5]) * rr0 + dc[4]) * rr0 + dc[3]) * rr0 + dc[2]) * rr0 + dc[1];
            double pre = -dv / r;
            double fx = dx * pre, fy = dy * pre, fz = dz * pre;
            vbond_s += v;
            f[3 * a] += fx; f[3 * a + 1] += fy; f[3 * a + 2] += fz;
            f[3 * bb] -= fx; f[3 * bb + 1] -= fy; f[3 * bb + 2] -= fz;
            pv[0] += dx * fx; pv[4] += dy * fy; pv[8] += dz * fz;
            pv[1] += dx * fy; pv[2] += dx * fz; pv[5] += dy * fz;
        }

        /* bends: bend (intra/bend.c:28-440) */
        for (int c = 0; c < s->nbend; c++) {
            int a1 = s->bend_j1[c], a2 = s->bend_j2[c], a3 = s->bend_j3[c], t = s->bend_typ[c];
            const double *bc = s->bend_c + 7 * t, *bs = s->bend_s + 7 * t;
            const double *bdc = s->bend_dc + 7 * t, *bds = s->bend_ds + 7 * t;
            double x2 = pos[3 * a2], y2 = pos[3 * a2 + 1], z2 = pos[3 * a2 + 2];
            double dx12 = pos[3 * a1] - x2, dy12 = pos[3 * a1 + 1] - y2, dz12 = pos[3 * a1 + 2] - z2;
            double dx23 = pos[3 * a3] - x2, dy23 = pos[3 * a3 + 1] - y2, dz23 = pos[3 * a3 + 2] - z2;
            double r122i = 1.0 / (dx12 * dx12 + dy12 * dy12 + dz12 * dz12);
            double r12i = sqrt(r122i);
            double r322i = 1.0 / (dx23 * dx23 + dy23 * dy23 + dz23 * dz23);
            double r32i = sqrt(r322i);
            double rpmag = r12i * r32i;
            double cost = (dx12 * dx23 + dy12 * dy23 + dz12 * dz23) * rpmag;
            cost = (cost < 1.0 ? cost : 1.0);
            cost = (cost > -1.0 ? cost : -1.0);
            double sint = sqrt(1.0 - cost * cost);
            sint = (sint > 1.0e-8 ? sint : 1.0e-8);
            double cos122 = cost * r122i, cos322 = cost * r322i;
            double vbendc = ((((((bc[6] * cost + bc[5]) * cost + bc[4]) * cost + bc[3]) * cost + bc[2]) * cost +
                              bc[1]) * cost + bc[0]);
            double sisum = (((((bs[6] * sint + bs[5]) * sint + bs[4]) * sint + bs[3]) * sint + bs[2]) * sint);
            double vbends = sisum * cost + bs[1] * sint;
            vbend_s += vbendc + vbends;
            double dvbendc = (((((bdc[6] * cost + bdc[5]) * cost + bdc[4]) * cost + bdc[3]) * cost + bdc[2]) * cost +
                              bdc[1]);
            double dvbends = ((((bds[6] * sint + bds[5]) * sint + bds[4]) * sint + bds[3]) * sint + bds[2]);
            dvbends = dvbends * cost + bds[1];
            double pre = -(dvbendc + sisum - dvbends * cost / sint);
            double fx1 = (dx23 * rpmag - dx12 * cos122) * pre, fy1 = (dy23 * rpmag - dy12 * cos122) * pre,
                   fz1 = (dz23 * rpmag - dz12 * cos122) * pre;
            double fx3 = (dx12 * rpmag - dx23 * cos322) * pre, fy3 = (dy12 * rpmag - dy23 * cos322) * pre,
                   fz3 = (dz12 * rpmag - dz23 * cos322) * pre;
            double fx2 = -(fx1 + fx3), fy2 = -(fy1 + fy3), fz2 = -(fz1 + fz3);
            f[3 * a1] += fx1; f[3 * a1 + 1] += fy1; f[3 * a1 + 2] += fz1;
            f[3 * a2] += fx2; f[3 * a2 + 1] += fy2; f[3 * a2 + 2] += fz2;
            f[3 * a3] += fx3; f[3 * a3 + 1] += fy3; f[3 * a3 + 2] += fz3;
            pv[0] += dx12 * fx1 + dx23 * fx3; pv[4] += dy12 * fy1 + dy23 * fy3; pv[8] += dz12 * fz1 + dz23 * fz3;
            pv[1] += dx12 * fy1 + dx23 * fy3; pv[2] += dx12 * fz1 + dx23 * fz3; pv[5] += dy12 * fz1 + dy23 * fz3;
        }

        /* distrib_ghost_force (ghost_control.c:71-129) */
        if (distribute_ghosts) {
            for (int g = 0; g < s->nghost; g++) {
                int gl = s->ghost_atom[g];
                for (int c = 0; c < s->ghost_ncomp; c++) {
                    int a = s->ghost_comp[g * s->ghost_ncomp + c];
                    if (a < 0) continue;
                    double cf = s->ghost_coef[g * s->ghost_ncomp + c];
                    f[3 * a] += cf * f[3 * gl];
                    f[3 * a + 1] += cf * f[3 * gl + 1];
                    f[3 * a + 2] += cf * f[3 * gl + 2];
                }
                f[3 * gl] = f[3 * gl + 1] = f[3 * gl + 2] = 0.0;
            }
        }
    }
    free(pos);

    /* ewald3d_selfbgr (recip3d/ewald3d_self_bgr.c:28-80), once per call */
    double q2sum = 0.0, qsum = 0.0;
    for (long i = 0; i < natm; i++) { q2sum += s->charge[i] * s->charge[i]; qsum += s->charge[i]; }
    double vself = 0.0, vbgr = 0.0;
    if (s->nktot > 0) {
        vself = -q2sum * (s->alp_ewd) * (s->self_erf) / sqrt(M_PI);
        vbgr = -0.5 * qsum * qsum * M_PI / (s->alp_ewd * s->alp_ewd * vol);
    }
    /* long_range_corr (energy_control_inter_real.c:206-320), full step */
    double vlong = s->clong / vol;
    double amult = s->iswit_vdw ? 1.0 : 2.0;
    double pdiag = (s->clong / vol) * amult * (double)P;
    pv[0] += pdiag + vbgr * P;
    pv[4] += pdiag + vbgr * P;
    pv[8] += pdiag + vbgr * P;
    pv[3] = pv[1];
    pv[6] = pv[2];
    pv[7] = pv[5];

    double dP = (double)P;
    e->vreal = vreal_s / dP;
    e->vrecip = vrecip_s / dP;
    e->vecor = vecor_s / dP;
    e->vself = vself;
    e->vbgr = vbgr;
    e->vlong = vlong;
    e->vbond = vbond_s / dP;
    e->vbend = vbend_s / dP;
    e->vvdw = vvdw_s / dP + vlong;
    e->vcoul = vcoul_s / dP + (e->vrecip + vself + vbgr + e->vecor);
    e->vintert = e->vreal + vlong + (e->vrecip + vself + vbgr + e->vecor);
    e->vintrat = e->vbond + e->vbend;
    for (int c = 0; c < 9; c++) e->pvten[c] = pv[c];
}

/* ------------------------------------------------------------------------ */
/* RESPA split of the force at one level (orc_respa in piny_oracle.h).       */
/* force = PINY's weighted clatoms fx; forcet = the virial forces fxt,       */
/* written only at a full inter level (bead 1..P, unweighted).               */
/* ------------------------------------------------------------------------ */
static void add3(double *f, int a, double fx, double fy, double fz)
{
    f[3 * a] += fx; f[3 * a + 1] += fy; f[3 * a + 2] += fz;
}

static void distrib_ghosts(const orc_system *s, double *f)
{
    for (int g = 0; g < s->nghost; g++) {
        int gl = s->ghost_atom[g];
        for (int c = 0; c < s->ghost_ncomp; c++) {
            int a = s->ghost_comp[g * s->ghost_ncomp + c];
            if (a < 0) continue;
            double cf = s->ghost_coef[g * s->ghost_ncomp + c];
            add3(f, a, cf * f[3 * gl], cf * f[3 * gl + 1], cf * f[3 * gl + 2]);
        }
        f[3 * gl] = f[3 * gl + 1] = f[3 * gl + 2] = 0.0;
    }
}

void orc_respa_force(const orc_system *s, const orc_respa *r, int level, int P,
                     const double *pos_in, const double *xmod, const double *h,
                     long npairs, const int *pi, const int *pj,
                     int distribute_ghosts, double *force, double *forcet)
{
    const int full_inter = (level & ORC_FULL_INTER) != 0, res_inter = (level & ORC_RES_INTER) != 0;
    const int intra = (level & (ORC_FULL_INTRA | ORC_RES_INTRA)) != 0;
    double hi[9];
    double vol = cell_inverse(h, hi);
    int cubic = is_cubic(h);
    long natm = s->natm;
    double *pos = malloc(sizeof(double) * 3 * natm);
    double *tmp = malloc(sizeof(double) * 3 * natm);
    const double w_full = r->wght_ter, w_res = r->wght_ter_res, w_tra_res = r->wght_tra_res;
    const double rheal_resi = 1.0 / r->rheal_res;
    /* bond_both.c:156-161 */
    const double wfor_both = r->int_res_inter ? r->wght_ter_res : r->wght_ter;

    for (int b = 0; b < P; b++) {
        memcpy(pos, pos_in + 3 * natm * b, sizeof(double) * 3 * natm);
        double *f = force + 3 * natm * b;
        double *ft = full_inter ? forcet + 3 * natm * b : NULL;
        memset(f, 0, sizeof(double) * 3 * natm);
        if (ft) memset(ft, 0, sizeof(double) * 3 * natm);
        for (int g = 0; g < s->nghost; g++) {
            int gl = s->ghost_atom[g];
            double gx = 0.0, gy = 0.0, gz = 0.0;
            for (int c = 0; c < s->ghost_ncomp; c++) {
                int a = s->ghost_comp[g * s->ghost_ncomp + c];
                if (a < 0) continue;
                double cf = s->ghost_coef[g * s->ghost_ncomp + c];
                gx += cf * pos[3 * a];
                gy += cf * pos[3 * a + 1];
                gz += cf * pos[3 * a + 2];
            }
            pos[3 * gl] = gx; pos[3 * gl + 1] = gy; pos[3 * gl + 2] = gz;
        }

        /* real space (force_npol.c): shave at cutoff (full) or cutoff_res
         * (res only, npol_shave_skin :1309-1319), switch over the last
         * rheal_res before cutoff_res (:807-816), multiplier (:1030-1060) */
        if (full_inter || res_inter) {
            for (long p = 0; p < npairs; p++) {
                int i = pi[p], j = pj[p];
                double dx = pos[3 * i] - pos[3 * j], dy = pos[3 * i + 1] - pos[3 * j + 1],
                       dz = pos[3 * i + 2] - pos[3 * j + 2];
                if (P > 1)
                    period_pimd_one(&dx, &dy, &dz, xmod[3 * i] - xmod[3 * j], xmod[3 * i + 1] - xmod[3 * j + 1],
                                    xmod[3 * i + 2] - xmod[3 * j + 2], h, hi, cubic);
                else
                    period_one(&dx, &dy, &dz, h, hi, cubic);
                double rr = sqrt((dx * dx + dy * dy + dz * dz));
                int pt = pair_type(s->atm_typ[i], s->atm_typ[j], s->ntyp);
                double cut = full_inter ? s->cutoff[pt] : r->cutoff_res[pt];
                if (!(rr < cut)) continue;
                int u = s->inter_map[pt];
                double rmin = s->rmin_spl[u], dr = s->dr_spl[u], dri = s->dri_spl[u];
                int k = (int)(((rr - rmin) * dri) + 0.5) + 3;
                k = k < s->nsplin - 2 ? k : s->nsplin - 2;
                k = k > 3 ? k : 3;
                double rsp = ((double)(k - 3)) * dr + rmin;
                double del = (rr - rsp) * dri;
                long off = (long)u * s->nsplin;
                double q2 = s->charge[i] * s->charge[j];
                double dvtemp = (q2 * vspl(s->cdv0_c + off, k, del) + vspl(s->cdv0 + off, k, del));
                double fx = dx * dvtemp, fy = dy * dvtemp, fz = dz * dvtemp;
                double fmult = w_full;
                if (res_inter) {
                    double br = (rr - r->cutoff_res[pt] + r->rheal_res) * rheal_resi;
                    br = br > 0.0 ? br : 0.0;
                    br = br < 1.0 ? br : 1.0;
                    double swit = br * br * (br * 2.0 - 3.0) + 1.0;
                    fmult = full_inter ? (swit * w_res + (1.0 - swit) * w_full) : swit * w_res;
                }
                add3(f, i, fx * fmult, fy * fmult, fz * fmult);
                add3(f, j, -(fx * fmult), -(fy * fmult), -(fz * fmult));
                if (ft) {
                    add3(ft, i, fx, fy, fz);
                    add3(ft, j, -fx, -fy, -fz);
                }
            }
        }

        /* reciprocal space and the exclusion correction
         * (energy_control_inter_recip.c:184-214, :278-323): without the
         * reciprocal RESPA set at full steps only, x wght_ter (ewald3d_pme.c
         * forces x wght_now, ecorr.c:100 wfor); with it (one grid) PME at
         * every inner inter step x wght_ter_res, ecor from the RESPA table
         * x wght_ter_res (ecorr.c:103-106) or, at full steps, ecor_both
         * (ecorr.c:349-351, :497-505).  With the separate RESPA mesh
         * (:215-271): PME on that mesh (the RESPA k sphere, irespa = 1,
         * ewald3d_pme.c:204-216) x wght_ter_res at inner inter steps; at full
         * steps x (wght_ter_res - wght_ter) and the full-mesh PME x wght_ter,
         * both unweighted into the virial forces (ewald3d_pme.c:563-585) */
        const int kres = r->nktot_res > 0;
        if (kres && res_inter && r->pme_res_on) {
            if (s->nktot > 0) {
                orc_system sr = *s;
                sr.ngrid_a = r->ngrid_res[0];
                sr.ngrid_b = r->ngrid_res[1];
                sr.ngrid_c = r->ngrid_res[2];
                sr.n_interp = r->n_interp_res;
                sr.nktot = r->nktot_res;
                sr.kastr = r->kastr_res;
                sr.kbstr = r->kbstr_res;
                sr.kcstr = r->kcstr_res;
                sr.bweight = r->bweight_res;
                double pvr[10] = {0};
                memset(tmp, 0, sizeof(double) * 3 * natm);
                pme_bead(&sr, pos, h, hi, vol, tmp, pvr);
                const double wr = full_inter ? w_res - w_full : w_res;
                for (long a = 0; a < 3 * natm; a++) {
                    if (ft) ft[a] += tmp[a];
                    f[a] += tmp[a] * wr;
                }
                if (full_inter) {
                    double pvf[10] = {0};
                    memset(tmp, 0, sizeof(double) * 3 * natm);
                    pme_bead(s, pos, h, hi, vol, tmp, pvf);
                    for (long a = 0; a < 3 * natm; a++) {
                        ft[a] += tmp[a];
                        f[a] += tmp[a] * w_full;
                    }
                }
            }
        }
        if (kres && res_inter) {
            if (s->nktot > 0 && !r->pme_res_on) {
                double pvr[10] = {0};
                memset(tmp, 0, sizeof(double) * 3 * natm);
                pme_bead(s, pos, h, hi, vol, tmp, pvr);
                for (long a = 0; a < 3 * natm; a++) {
                    if (ft) ft[a] += tmp[a];
                    f[a] += tmp[a] * w_res;
                }
            }
            for (int c = 0; c < s->necor; c++) {
                int a = s->ecor_j1[c], bb = s->ecor_j2[c];
                double dx = pos[3 * a] - pos[3 * bb], dy = pos[3 * a + 1] - pos[3 * bb + 1],
                       dz = pos[3 * a + 2] - pos[3 * bb + 2];
                double rr = sqrt(dx * dx + dy * dy + dz * dz);
                int k = (int)(((rr - s->ecor_rmin) * s->ecor_dri) + 0.5) + 3;
                k = k < s->ecor_nsplin - 2 ? k : s->ecor_nsplin - 2;
                k = k > 3 ? k : 3;
                double rsp = ((double)(k - 3)) * s->ecor_dr + s->ecor_rmin;
                double del = (rr - rsp) * s->ecor_dri;
                double q12 = s->charge[a] * s->charge[bb];
                double dvr = vspl(r->ecor_cdv0_res, k, del) * q12;
                double g[3];
                if (full_inter) {
                    double dvt = vspl(s->ecor_cdv0, k, del) * q12;
                    double d[3] = {dx, dy, dz};
                    for (int e = 0; e < 3; e++) g[e] = w_full * (d[e] * dvt) + (w_res - w_full) * (d[e] * dvr);
                    add3(ft, a, dx * dvt, dy * dvt, dz * dvt);
                    add3(ft, bb, -(dx * dvt), -(dy * dvt), -(dz * dvt));
                } else {
                    g[0] = dx * dvr * w_res;
                    g[1] = dy * dvr * w_res;
                    g[2] = dz * dvr * w_res;
                }
                add3(f, a, g[0], g[1], g[2]);
                add3(f, bb, -g[0], -g[1], -g[2]);
            }
        } else if (full_inter) {
            if (s->nktot > 0) {
                double pvr[10] = {0};
                memset(tmp, 0, sizeof(double) * 3 * natm);
                pme_bead(s, pos, h, hi, vol, tmp, pvr);
                for (long a = 0; a < 3 * natm; a++) {
                    ft[a] += tmp[a];
                    f[a] += tmp[a] * w_full;
                }
            }
            for (int c = 0; c < s->necor; c++) {
                int a = s->ecor_j1[c], bb = s->ecor_j2[c];
                double dx = pos[3 * a] - pos[3 * bb], dy = pos[3 * a + 1] - pos[3 * bb + 1],
                       dz = pos[3 * a + 2] - pos[3 * bb + 2];
                double rr = sqrt(dx * dx + dy * dy + dz * dz);
                int k = (int)(((rr - s->ecor_rmin) * s->ecor_dri) + 0.5) + 3;
                k = k < s->ecor_nsplin - 2 ? k : s->ecor_nsplin - 2;
                k = k > 3 ? k : 3;
                double rsp = ((double)(k - 3)) * s->ecor_dr + s->ecor_rmin;
                double del = (rr - rsp) * s->ecor_dri;
                double q12 = s->charge[a] * s->charge[bb];
                double dvt = vspl(s->ecor_cdv0, k, del) * q12;
                double fx = dx * dvt, fy = dy * dvt, fz = dz * dvt;
                add3(ft, a, fx, fy, fz);
                add3(ft, bb, -fx, -fy, -fz);
                add3(f, a, fx * w_full, fy * w_full, fz * w_full);
                add3(f, bb, -(fx * w_full), -(fy * w_full), -(fz * w_full));
            }
        }

        if (intra) {
            /* bonds: bond_both at inter levels (bond_both.c:270-420), else
             * bond() with the res equilibrium when ires_bond (bond.c:113-118) */
            for (int c = 0; c < s->nbond; c++) {
                int a = s->bond_j1[c], bb = s->bond_j2[c], t = s->bond_typ[c];
                const double *dc = s->bond_dc + 7 * t;
                double dx = pos[3 * a] - pos[3 * bb], dy = pos[3 * a + 1] - pos[3 * bb + 1],
                       dz = pos[3 * a + 2] - pos[3 * bb + 2];
                double rr = sqrt(dx * dx + dy * dy + dz * dz);
                if (full_inter || res_inter) {
                    double rr0 = rr - s->bond_eq[t], rr0r = rr - r->bond_eq_res[t];
                    double dv = ((((dc[6] * rr0 + dc[5]) * rr0 + dc[4]) * rr0 + dc[3]) * rr0 + dc[2]) * rr0 + dc[1];
                    double dvr =
                        ((((dc[6] * rr0r + dc[5]) * rr0r + dc[4]) * rr0r + dc[3]) * rr0r + dc[2]) * rr0r + dc[1];
                    double pre = -dv / rr, prer = -dvr / rr;
                    double f1[3] = {dx * pre, dy * pre, dz * pre}, f2[3] = {dx * prer, dy * prer, dz * prer};
                    double fw[3];
                    for (int d = 0; d < 3; d++) fw[d] = w_tra_res * f2[d] + wfor_both * (f1[d] - f2[d]);
                    if (ft) {
                        add3(ft, a, f1[0], f1[1], f1[2]);
                        add3(ft, bb, -f1[0], -f1[1], -f1[2]);
                    }
                    add3(f, a, fw[0], fw[1], fw[2]);
                    add3(f, bb, -fw[0], -fw[1], -fw[2]);
                } else {
                    double rr0 = rr - (r->ires_bond ? r->bond_eq_res[t] : s->bond_eq[t]);
                    double dv = ((((dc[6] * rr0 + dc[5]) * rr0 + dc[4]) * rr0 + dc[3]) * rr0 + dc[2]) * rr0 + dc[1];
                    double pre = -dv / rr;
                    double fx = dx * pre * w_tra_res, fy = dy * pre * w_tra_res, fz = dz * pre * w_tra_res;
                    add3(f, a, fx, fy, fz);
                    add3(f, bb, -fx, -fy, -fz);
                }
            }
            /* bends x wght_tra_res (bend.c:144, :380-393) */
            for (int c = 0; c < s->nbend; c++) {
                int a1 = s->bend_j1[c], a2 = s->bend_j2[c], a3 = s->bend_j3[c], t = s->bend_typ[c];
                const double *bs = s->bend_s + 7 * t;
                const double *bdc = s->bend_dc + 7 * t, *bds = s->bend_ds + 7 * t;
                double x2 = pos[3 * a2], y2 = pos[3 * a2 + 1], z2 = pos[3 * a2 + 2];
                double dx12 = pos[3 * a1] - x2, dy12 = pos[3 * a1 + 1] - y2, dz12 = pos[3 * a1 + 2] - z2;
                double dx23 = pos[3 * a3] - x2, dy23 = pos[3 * a3 + 1] - y2, dz23 = pos[3 * a3 + 2] - z2;
                double r122i = 1.0 / (dx12 * dx12 + dy12 * dy12 + dz12 * dz12);
                double r12i = sqrt(r122i);
                double r322i = 1.0 / (dx23 * dx23 + dy23 * dy23 + dz23 * dz23);
                double r32i = sqrt(r322i);
                double rpmag = r12i * r32i;
                double cost = (dx12 * dx23 + dy12 * dy23 + dz12 * dz23) * rpmag;
                cost = (cost < 1.0 ? cost : 1.0);
                cost = (cost > -1.0 ? cost : -1.0);
                double sint = sqrt(1.0 - cost * cost);
                sint = (sint > 1.0e-8 ? sint : 1.0e-8);
                double cos122 = cost * r122i, cos322 = cost * r322i;
                double sisum = (((((bs[6] * sint + bs[5]) * sint + bs[4]) * sint + bs[3]) * sint + bs[2]) * sint);
                double dvbendc = (((((bdc[6] * cost + bdc[5]) * cost + bdc[4]) * cost + bdc[3]) * cost + bdc[2]) *
                                      cost + bdc[1]);
                double dvbends = ((((bds[6] * sint + bds[5]) * sint + bds[4]) * sint + bds[3]) * sint + bds[2]);
                dvbends = dvbends * cost + bds[1];
                double pre = -(dvbendc + sisum - dvbends * cost / sint);
                double g1[3] = {(dx23 * rpmag - dx12 * cos122) * pre, (dy23 * rpmag - dy12 * cos122) * pre,
                                (dz23 * rpmag - dz12 * cos122) * pre};
                double g3[3] = {(dx12 * rpmag - dx23 * cos322) * pre, (dy12 * rpmag - dy23 * cos322) * pre,
                                (dz12 * rpmag - dz23 * cos322) * pre};
                double g2[3] = {-(g1[0] + g3[0]), -(g1[1] + g3[1]), -(g1[2] + g3[2])};
                if (ft) {
                    add3(ft, a1, g1[0], g1[1], g1[2]);
                    add3(ft, a2, g2[0], g2[1], g2[2]);
                    add3(ft, a3, g3[0], g3[1], g3[2]);
                }
                add3(f, a1, g1[0] * w_tra_res, g1[1] * w_tra_res, g1[2] * w_tra_res);
                add3(f, a2, g2[0] * w_tra_res, g2[1] * w_tra_res, g2[2] * w_tra_res);
                add3(f, a3, g3[0] * w_tra_res, g3[1] * w_tra_res, g3[2] * w_tra_res);
            }
        }
        if (distribute_ghosts) {
            distrib_ghosts(s, f);
            if (ft) distrib_ghosts(s, ft);
        }
    }
    free(pos);
    free(tmp);
}

/* ------------------------------------------------------------------------ */
/* Verlet-list rebuild test.                                                 */
/* check_ver_list:  src/energy/inter/real_space/nbr_list_control.c:182-247 */
/* get_pimd_spread: src/energy/pimd/pimd_estimators.c:121-220 (bead 1 is   */
/*                  the reference, beads 2..P are compared with it)        */
/* get_cut_skin:    nbr_list_control.c:249-281 (plain cutskin only)         */
/* ------------------------------------------------------------------------ */
int orc_check_list(int natm, int nbeads, const double *pos, const double *x0,
                   double skin, double spread_ref, int ninter,
                   const double *cutoff, double *rmax, double *spread_now,
                   double *cutskin2)
{
    double r2max = 0.0, s2max = 0.0;
    for (int i = 0; i < natm; i++) {
        double dx = pos[3 * i] - x0[3 * i];
        double dy = pos[3 * i + 1] - x0[3 * i + 1];
        double dz = pos[3 * i + 2] - x0[3 * i + 2];
        double r2 = dx * dx + dy * dy + dz * dz;
        r2max = r2max > r2 ? r2max : r2;
    }
    for (int b = 1; b < nbeads; b++)
        for (int i = 0; i < natm; i++) {
            const double *p = pos + ((size_t)b * natm + i) * 3;
            double dx = p[0] - pos[3 * i];
            double dy = p[1] - pos[3 * i + 1];
            double dz = p[2] - pos[3 * i + 2];
            double r2 = dx * dx + dy * dy + dz * dz;
            s2max = s2max > r2 ? s2max : r2;
        }
    double rm = sqrt(r2max);
    double sp = nbeads > 1 ? sqrt(s2max) : 0.0;
    double dspread = 0.0;
    if (nbeads > 1) dspread = (sp - spread_ref) > 0.0 ? (sp - spread_ref) : 0.0;
    double skin2 = skin / 2.0 + dspread;
    if (rmax) *rmax = rm;
    if (spread_now) *spread_now = sp;
    if (cutskin2)
        for (int k = 0; k < ninter; k++) {
            double cs = cutoff[k] + skin + sp;
            cutskin2[k] = cs * cs;
        }
    return rm > skin2 ? 1 : 0;
}

/* --------------------------------------------------------------------------
 * Ring-polymer transforms, one (atom, direction) row of P beads at a time.
 * Staging: src/energy/pimd/transform_stg.c:31-85 (forces), :92-153 (modes),
 * :164-222 (positions), with rat1[ip] = (ip-1)/ip, rat2[ip] = 1/ip from
 * path_integral_init (transform_cnt.c:206-216); the loops and the grouping
 * of each update are PINY's, so the results are bit-identical to it.
 * Normal modes: transform_cnt.c:240-316 (modes: backward FFT, i.e.
 * e^{+2 pi i jk/P}, then /P), :321-410 (positions: forward FFT of the
 * Hermitian-completed modes), :415-489 (forces: backward FFT, x2 on the
 * paired modes).  PINY packs mode 1 = Re X_0, mode 2m = Re X_m,
 * mode 2m+1 = Im X_m (m = 1..P/2-1), mode P = Re X_{P/2}.  Here the DFTs are
 * direct sums, so they agree with PINY's FFT to rounding only.
 * ------------------------------------------------------------------------ */
static void orc_stage_row(int P, int what, double *v /* 1-based, v[1..P] */)
{
    double rat1[65], rat2[65];
    for (int ip = 2; ip <= P; ip++) {
        rat1[ip] = ((double)(ip - 1)) / ((double)(ip));
        rat2[ip] = 1.0 / ((double)(ip));
    }
    if (what == 0) {
        for (int ip = 2; ip <= P - 1; ip++) {
            double star = rat1[ip] * v[ip + 1] + rat2[ip] * v[1];
            v[ip] -= star;
        }
        double star = rat1[P] * v[1] + rat2[P] * v[1];
        v[P] -= star;
    } else if (what == 1) {
        v[P] += v[1];
        for (int ip = P - 1; ip >= 2; ip--) {
            double add = rat1[ip] * v[ip + 1] + v[1] * rat2[ip];
            v[ip] += add;
        }
    } else {
        for (int ip = 2; ip <= P; ip++) v[1] += v[ip];
        for (int ip = 2; ip <= P - 1; ip++) v[ip + 1] += (rat1[ip] * v[ip]);
    }
}

static void orc_mode_row(int P, int what, double *v /* 0-based, v[0..P-1] */)
{
    double out[64], cs[64], sn[64];
    const int np2 = P / 2;
    for (int m = 0; m < P; m++) {
        double a = 2.0 * M_PI * (double)m / (double)P;
        cs[m] = cos(a);
        sn[m] = sin(a);
    }
    if (what == 0 || what == 2) {
        for (int k = 0; k <= np2; k++) {
            double re = 0.0, im = 0.0;
            for (int j = 0; j < P; j++) {
                int m = (j * k) % P;
                re += v[j] * cs[m];
                im += v[j] * sn[m];
            }
            if (what == 0) {
                re /= P;
                im /= P;
            }
            double f2 = what == 2 ? 2.0 : 1.0;
            if (k == 0) out[0] = re;
            else if (k == np2) out[P - 1] = re;
            else {
                out[2 * k - 1] = re * f2;
                out[2 * k] = im * f2;
            }
        }
    } else {
        for (int j = 0; j < P; j++) {
            double s = v[0] + ((j & 1) ? -v[P - 1] : v[P - 1]);
            for (int k = 1; k < np2; k++) {
                int m = (j * k) % P;
                s += 2.0 * (v[2 * k - 1] * cs[m] + v[2 * k] * sn[m]);
            }
            out[j] = s;
        }
    }
    for (int j = 0; j < P; j++) v[j] = out[j];
}

int orc_pimd_transform(int natm, int nbeads, int kind, int what, double *x)
{
    if (natm < 1 || nbeads < 1 || nbeads > 64 || (kind != 1 && kind != 2) || what < 0 || what > 2) return -1;
    if (kind == 2 && (nbeads & (nbeads - 1))) return -1;
    if (nbeads == 1) return 0;
    const size_t stride = (size_t)natm * 3;
    double row[65];
    for (size_t t = 0; t < stride; t++) {
        for (int b = 0; b < nbeads; b++) row[b + 1] = x[b * stride + t];
        if (kind == 1) orc_stage_row(nbeads, what, row);
        else orc_mode_row(nbeads, what, row + 1);
        for (int b = 0; b < nbeads; b++) x[b * stride + t] = row[b + 1];
    }
    return 0;
}
