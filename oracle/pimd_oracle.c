/*
 * Oracle, part 2: PINY's path-integral MD bookkeeping around the force call.
 *
 * THIS IS TEST INFRASTRUCTURE (see piny_oracle.h).  Plain C, FP64, serial,
 * 0-based; bead arrays are [P][natm][3] (bead-major), chain arrays
 * [len_nhc][num_nhc].  Each routine cites the PINY source it restates.
 */
#include "piny_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* apply_NHC_par (src/integrate/md/int_NVT.c:144-353) on the velocities v
 * ([natm][3]) of one bead, with masses m ([natm]).  inhc[d*natm + i] is the
 * chain of coordinate d of atom i; chain num_nhc is the null chain (never
 * evolved, scale 1).  wdti[k] = Yoshida weight k times dti_nhc (PINY's
 * therm_info.wdti); x_nhc, v_nhc ([len_nhc][num_nhc]) are updated. */
void orc_nhc_apply(int natm, const int *inhc, const double *m, double *v, int num_nhc, int len_nhc,
                   int nres_nhc, int nyosh, const double *wdti, const double *mass_nhc, const double *gkt,
                   double *x_nhc, double *v_nhc)
{
    const int nc = num_nhc;
    double *kin = calloc((size_t)nc + 1, sizeof(double));
    double *sc = malloc(((size_t)nc + 1) * sizeof(double));
    double *f = malloc((size_t)len_nhc * (size_t)(nc > 0 ? nc : 1) * sizeof(double));
#define MN(c, k) mass_nhc[(size_t)(c) * nc + (k)]
#define GK(c, k) gkt[(size_t)(c) * nc + (k)]
#define XN(c, k) x_nhc[(size_t)(c) * nc + (k)]
#define VN(c, k) v_nhc[(size_t)(c) * nc + (k)]
#define FN(c, k) f[(size_t)(c) * nc + (k)]
    for (int d = 0; d < 3; d++)
        for (int i = 0; i < natm; i++) kin[inhc[d * natm + i]] += m[i] * v[3 * i + d] * v[3 * i + d];
    for (int k = 0; k <= nc; k++) sc[k] = 1.0;
    for (int k = 0; k < nc; k++) FN(0, k) = (kin[k] - GK(0, k)) / MN(0, k);
    for (int c = 0; c < len_nhc - 1; c++)
        for (int k = 0; k < nc; k++) FN(c + 1, k) = (MN(c, k) * VN(c, k) * VN(c, k) - GK(c + 1, k)) / MN(c + 1, k);
    const int L = len_nhc - 1; /* last link, 0-based */
    for (int r = 0; r < nres_nhc; r++)
        for (int y = 0; y < nyosh; y++) {
            const double w2 = wdti[y] / 2.0, w4 = wdti[y] / 4.0, w8 = wdti[y] / 8.0;
            for (int k = 0; k < nc; k++) VN(L, k) += FN(L, k) * w4;
            for (int c = L - 1; c >= 0; c--)
                for (int k = 0; k < nc; k++) {
                    double aa = exp(-w8 * VN(c + 1, k));
                    VN(c, k) = VN(c, k) * aa * aa + w4 * FN(c, k) * aa;
                }
            for (int k = 0; k < nc; k++) {
                double aa = exp(-w2 * VN(0, k));
                sc[k] *= aa;
                kin[k] *= aa * aa;
            }
            for (int c = 0; c <= L; c++)
                for (int k = 0; k < nc; k++) XN(c, k) += VN(c, k) * w2;
            for (int k = 0; k < nc; k++) FN(0, k) = (kin[k] - GK(0, k)) / MN(0, k);
            for (int c = 0; c < L; c++) {
                for (int k = 0; k < nc; k++) {
                    double aa = exp(-w8 * VN(c + 1, k));
                    VN(c, k) = VN(c, k) * aa * aa + w4 * FN(c, k) * aa;
                }
                for (int k = 0; k < nc; k++)
                    FN(c + 1, k) = (MN(c, k) * VN(c, k) * VN(c, k) - GK(c + 1, k)) / MN(c + 1, k);
            }
            for (int k = 0; k < nc; k++) VN(L, k) += FN(L, k) * w4;
        }
    for (int d = 0; d < 3; d++)
        for (int i = 0; i < natm; i++) v[3 * i + d] *= sc[inhc[d * natm + i]];
#undef MN
#undef GK
#undef XN
#undef VN
#undef FN
    free(kin);
    free(sc);
    free(f);
}

/* mode_energy_control (src/energy/pimd/pimd_estimators.c:31-110): harmonic
 * bead-coupling forces on the modes u, fm = -2 prekf veig u * wght, their
 * energy (returned; PINY's kin_harm) and pvten_mode_tot (9, row-major). */
double orc_pimd_springs(int natm, int P, const double *u, const double *prekf, const double *veig, double wght,
                        double *fm, double *pvten_mode_tot)
{
    double ake = 0.0, pv[9] = {0};
    for (int b = 0; b < P; b++)
        for (int i = 0; i < natm; i++) {
            const double *x = u + ((size_t)b * natm + i) * 3;
            double *g = fm + ((size_t)b * natm + i) * 3;
            double fk = prekf[i] * veig[b];
            ake += fk * (x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
            g[0] = -2.0 * fk * x[0];
            g[1] = -2.0 * fk * x[1];
            g[2] = -2.0 * fk * x[2];
            pv[0] += x[0] * g[0];
            pv[4] += x[1] * g[1];
            pv[8] += x[2] * g[2];
            pv[1] += x[0] * g[1];
            pv[2] += x[0] * g[2];
            pv[5] += x[1] * g[2];
            g[0] *= wght;
            g[1] *= wght;
            g[2] *= wght;
        }
    pv[3] = pv[1];
    pv[6] = pv[2];
    pv[7] = pv[5];
    if (pvten_mode_tot) memcpy(pvten_mode_tot, pv, sizeof pv);
    return ake;
}

/* The force post-processing of energy_control_pimd
 * (src/energy/control/energy_control_pimd.c:113-218) for a full step
 * without RESPA: bead forces f /= P, pvten and pvten_tot /= P, the centroid
 * virial correction of pimd_pvten_forc_corr (pimd_estimators.c:223-305; the
 * virial forces fxt equal the forces here), the force transform to modes
 * and the spring forces fm added.  x: bead positions, xmod: mode-1
 * positions.  Returns akvirx (PINY's 0.5 * akvirx). */
double orc_pimd_force_post(int natm, int P, int kind, double *f, const double *x, const double *xmod,
                           const double *fm, int nfree_atoms, double beta, double *pvten, double *pvten_tot)
{
    const size_t n3 = (size_t)natm * 3;
    for (size_t k = 0; k < (size_t)P * n3; k++) f[k] /= P;
    for (int k = 0; k < 9; k++) {
        pvten[k] /= P;
        pvten_tot[k] /= P;
    }
    double akvirx = 3.0 * (double)nfree_atoms / beta;
    /* PINY's pvten index order 1..9 = xx xy xz yx yy yz zx zy zz; the
     * correction runs only with more than one bead */
    for (int b = 0; b < (P > 1 ? P : 0); b++) {
        for (int i = 0; i < natm; i++) {
            const double *p = x + b * n3 + 3 * (size_t)i, *g = f + b * n3 + 3 * (size_t)i;
            double d[3] = {p[0] - xmod[3 * i], p[1] - xmod[3 * i + 1], p[2] - xmod[3 * i + 2]};
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) pvten[3 * r + c] -= d[r] * g[c];
        }
        for (int i = 0; i < natm; i++) {
            const double *p = x + b * n3 + 3 * (size_t)i, *g = f + b * n3 + 3 * (size_t)i;
            double d[3] = {p[0] - xmod[3 * i], p[1] - xmod[3 * i + 1], p[2] - xmod[3 * i + 2]};
            akvirx -= (d[0] * g[0] + d[1] * g[1] + d[2] * g[2]);
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) pvten_tot[3 * r + c] -= d[r] * g[c];
        }
    }
    if (P > 1) orc_pimd_transform(natm, P, kind, 2, f);
    for (size_t k = 0; k < (size_t)P * n3; k++) f[k] += fm[k];
    return 0.5 * akvirx;
}

/* energy_control_pimd's post-processing at one RESPA level
 * (energy_control_pimd.c:113-218, pimd_pvten_forc_corr pimd_estimators.c:
 * 223-305): forces / P; pvten corrected with the (weighted) forces f at
 * every level; at a full level (iget_full_inter and iget_full_intra) the
 * virial forces ft / P give akvirx and the pvten_tot correction; forces to
 * modes, springs added.  ft may be NULL when full is 0.  Returns 0.5 akvirx
 * (0 below the full level). */
double orc_pimd_force_post_respa(int natm, int P, int kind, double *f, double *ft, const double *x,
                                 const double *xmod, const double *fm, int nfree_atoms, double beta, int full,
                                 double *pvten, double *pvten_tot)
{
    const size_t n3 = (size_t)natm * 3;
    for (size_t k = 0; k < (size_t)P * n3; k++) f[k] /= P;
    if (full && ft)
        for (size_t k = 0; k < (size_t)P * n3; k++) ft[k] /= P;
    for (int k = 0; k < 9; k++) {
        pvten[k] /= P;
        pvten_tot[k] /= P;
    }
    double akvirx = full ? 3.0 * (double)nfree_atoms / beta : 0.0;
    for (int b = 0; b < (P > 1 ? P : 0); b++) {
        for (int i = 0; i < natm; i++) {
            const double *p = x + b * n3 + 3 * (size_t)i, *g = f + b * n3 + 3 * (size_t)i;
            double d[3] = {p[0] - xmod[3 * i], p[1] - xmod[3 * i + 1], p[2] - xmod[3 * i + 2]};
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) pvten[3 * r + c] -= d[r] * g[c];
        }
        if (!full) continue;
        for (int i = 0; i < natm; i++) {
            const double *p = x + b * n3 + 3 * (size_t)i, *g = ft + b * n3 + 3 * (size_t)i;
            double d[3] = {p[0] - xmod[3 * i], p[1] - xmod[3 * i + 1], p[2] - xmod[3 * i + 2]};
            akvirx -= (d[0] * g[0] + d[1] * g[1] + d[2] * g[2]);
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) pvten_tot[3 * r + c] -= d[r] * g[c];
        }
    }
    if (P > 1) orc_pimd_transform(natm, P, kind, 2, f);
    for (size_t k = 0; k < (size_t)P * n3; k++) f[k] += fm[k];
    return 0.5 * akvirx;
}
