/*
 * The PINY-side binding of libpinyb200: what a PINY maintainer adds to
 * src/energy/control/ to run the per-bead force sub-steps on the GPU.
 * Compiled here against PINY's own headers and linked with PINY's objects
 * and libpinyb200.so (make -C oracle ref-gpu) so the drop-in is exercised
 * on PINY's real CLASS / BONDED / GENERAL_DATA; the test driver
 * (ref_driver.c, mode gpu_dump) compares it with PINY's unmodified path.
 *
 *   gpu_force_init      PINY's set-up products (interact tables, exclusions,
 *                       Ewald k list and B-spline weights, ecor table, bond
 *                       and bend series, ghost definitions) -> one library
 *                       context for all beads of this CLASS.
 *   gpu_energy_control  in place of energy_control_inter_real,
 *                       energy_control_inter_recip and energy_control_intra
 *                       for all beads (energy_control_pimd.c:91-111,
 *                       energy_control.c:49-74): PINY's own list test
 *                       (get_pimd_spread, get_cut_skin, check_ver_list, as
 *                       nbr_list_control.c:32-118 calls them), a device
 *                       list build when it fires, then forces added to
 *                       fx/fy/fz and fxt/fyt/fzt, pvten_tot and stat_avg as
 *                       the three sub-steps add them.
 *
 * A non-zero return is a pinyb200 status; the caller prints
 * pinyb200_last_error and leaves through PINY's error convention.
 */
#include "standard_include.h"
#include "../typ_defs/typedefs_class.h"
#include "../typ_defs/typedefs_bnd.h"
#include "../typ_defs/typedefs_gen.h"
#include "../typ_defs/typedefs_cp.h"
#include "../typ_defs/typedefs_par.h"
#include "../typ_defs/typedefs_stat.h"
#include "pinyb200.h"

void get_pimd_spread(CLATOMS_INFO *, CLATOMS_POS *, double *, COMMUNICATE *);
void get_cut_skin(double *, double *, double *, double *, double *, double *, double, double, double, int);
void check_ver_list(CLATOMS_INFO *, CLATOMS_POS *, NBR_LIST *, INTERACT *, int *);

/* 1-based PINY array (allocated as ptr - 1) seen from element 0 */
#define ZB(p) ((p) + 1)

/* 0-based copy of a 1-based list of PINY atom / type numbers */
static int *minus_one(const int *one_based, int n)
{
    int *out = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; i++) out[i] = one_based[i + 1] - 1;
    return out;
}

/* [ntyp][7] series coefficients from PINY's seven per-type arrays */
static double *series7(double *const *cols, int ntyp)
{
    double *out = (double *)malloc(sizeof(double) * (size_t)(7 * (ntyp > 0 ? ntyp : 1)));
    for (int t = 0; t < ntyp; t++)
        for (int k = 0; k < 7; k++) out[7 * t + k] = cols[k][t + 1];
    return out;
}

int gpu_force_init(CLASS *class, BONDED *bonded, GENERAL_DATA *general_data, int mixed, pinyb200_ctx **ctx)
{
    CLATOMS_INFO *ci = &class->clatoms_info;
    ATOMMAPS *am = &class->atommaps;
    INTERACT *it = &class->interact;
    EXCL *ex = &bonded->excl;
    EWALD *ew = &general_data->ewald;
    PART_MESH *pm = &class->part_mesh;
    ECOR *ec = &bonded->ecor;
    BOND *bd = &bonded->bond;
    BEND *be = &bonded->bend;
    GHOST_ATOMS *gh = &class->ghost_atoms;
    const int n = ci->natm_tot;
    const int nter = am->natm_typ * (am->natm_typ + 1) / 2;
    pinyb200_system s;
    memset(&s, 0, sizeof(s));

    s.natm = n;
    s.ntyp = am->natm_typ;
    int *typ = minus_one(am->iatm_atm_typ, n);
    s.atm_typ = typ;
    s.charge = ZB(ci->q);
    /* real-space tables (control_inter_params.c:643-777) */
    int nuniq = 0;
    for (int k = 1; k <= nter; k++)
        if (it->inter_map_index[k] > nuniq) nuniq = it->inter_map_index[k];
    s.nsplin = it->nsplin;
    s.ninter_unique = nuniq;
    int *imap = minus_one(it->inter_map_index, nter);
    s.inter_map = imap;
    s.cutoff = ZB(it->cutoff);
    s.rmin_spl = ZB(it->rmin_spl);
    s.dr_spl = ZB(it->dr_spl);
    s.dri_spl = ZB(it->dri_spl);
    s.cv0 = ZB(it->cv0);
    s.cdv0 = ZB(it->cdv0);
    s.cv0_c = ci->nchrg > 0 ? ZB(it->cv0_c) : NULL;
    s.cdv0_c = ci->nchrg > 0 ? ZB(it->cdv0_c) : NULL;
    s.skin = it->skin;
    s.clong = it->clong;
    s.iswit_vdw = it->iswit_vdw;
    /* exclusions (set_exclude.c:30-396): num / j_off / j -> CSR, 0-based */
    int *eoff = (int *)malloc(sizeof(int) * (size_t)(n + 1));
    int *ej = (int *)malloc(sizeof(int) * (size_t)(ex->nlst > 0 ? ex->nlst : 1));
    eoff[0] = 0;
    for (int i = 0; i < n; i++) {
        const int num = ex->num[i + 1], off = ex->j_off[i + 1];
        for (int k = 0; k < num; k++) ej[eoff[i] + k] = ex->j[off + k + 1] - 1;
        eoff[i + 1] = eoff[i] + num;
    }
    s.excl_off = eoff;
    s.excl_j = ej;
    /* Ewald / PME (set_cp_ewald.c:204-586, 1136-1382) */
    s.alp_ewd = ew->alp_ewd;
    s.self_erf = ew->self_erf;
    s.nktot = pm->pme_on ? ew->nktot : 0;
    s.kastr = ZB(ew->kastr);
    s.kbstr = ZB(ew->kbstr);
    s.kcstr = ZB(ew->kcstr);
    if (pm->pme_on) {
        s.bweight = ZB(pm->bweight_tot);
        s.ngrid_a = pm->ngrid_a;
        s.ngrid_b = pm->ngrid_b;
        s.ngrid_c = pm->ngrid_c;
        s.n_interp = pm->n_interp;
    }
    /* excluded-pair Ewald correction (set_exclude.c:548-779) */
    int *e1 = NULL, *e2 = NULL;
    s.necor = ec->num;
    if (ec->num > 0) {
        e1 = minus_one(ec->j1, ec->num);
        e2 = minus_one(ec->j2, ec->num);
        s.ecor_j1 = e1;
        s.ecor_j2 = e2;
        s.ecor_nsplin = ec->nsplin;
        s.ecor_rmin = ec->rmin_spl;
        s.ecor_dr = ec->dr_spl;
        s.ecor_dri = ec->dri_spl;
        s.ecor_cv0 = ZB(ec->cv0);
        s.ecor_cdv0 = ZB(ec->cdv0);
    }
    /* power-series bonds (intra_coefs.c:95-122) */
    int *b1 = NULL, *b2 = NULL, *bt = NULL;
    double *bc = NULL, *bdc = NULL;
    s.nbond = bd->npow;
    if (bd->npow > 0) {
        b1 = minus_one(bd->j1_pow, bd->npow);
        b2 = minus_one(bd->j2_pow, bd->npow);
        bt = minus_one(bd->jtyp_pow, bd->npow);
        double *c[7] = {bd->c_0, bd->c_1, bd->c_2, bd->c_3, bd->c_4, bd->c_5, bd->c_6};
        double *dc[7] = {bd->dc_0, bd->dc_1, bd->dc_2, bd->dc_3, bd->dc_4, bd->dc_5, bd->dc_6};
        bc = series7(c, bd->ntyp_pow);
        bdc = series7(dc, bd->ntyp_pow);
        s.bond_j1 = b1;
        s.bond_j2 = b2;
        s.bond_typ = bt;
        s.nbond_typ = bd->ntyp_pow;
        s.bond_eq = ZB(bd->eq_pow);
        s.bond_c = bc;
        s.bond_dc = bdc;
    }
    /* cos/sin-series bends (intra_coefs.c:204-380) */
    int *a1 = NULL, *a2 = NULL, *a3 = NULL, *at = NULL;
    double *ac = NULL, *as = NULL, *adc = NULL, *ads = NULL;
    s.nbend = be->npow;
    if (be->npow > 0) {
        a1 = minus_one(be->j1_pow, be->npow);
        a2 = minus_one(be->j2_pow, be->npow);
        a3 = minus_one(be->j3_pow, be->npow);
        at = minus_one(be->jtyp_pow, be->npow);
        double *c[7] = {be->c_0, be->c_1, be->c_2, be->c_3, be->c_4, be->c_5, be->c_6};
        double *sn[7] = {be->s_0, be->s_1, be->s_2, be->s_3, be->s_4, be->s_5, be->s_6};
        double *dc[7] = {be->dc_0, be->dc_1, be->dc_2, be->dc_3, be->dc_4, be->dc_5, be->dc_6};
        double *ds[7] = {be->ds_0, be->ds_1, be->ds_2, be->ds_3, be->ds_4, be->ds_5, be->ds_6};
        ac = series7(c, be->ntyp_pow);
        as = series7(sn, be->ntyp_pow);
        adc = series7(dc, be->ntyp_pow);
        ads = series7(ds, be->ntyp_pow);
        s.bend_j1 = a1;
        s.bend_j2 = a2;
        s.bend_j3 = a3;
        s.bend_typ = at;
        s.nbend_typ = be->ntyp_pow;
        s.bend_c = ac;
        s.bend_s = as;
        s.bend_dc = adc;
        s.bend_ds = ads;
    }
    /* M sites (ghost_control.c:28-129) */
    int *ga = NULL, *gc = NULL;
    double *gcoef = NULL;
    s.nghost = gh->nghost_tot;
    if (gh->nghost_tot > 0) {
        const int ng = gh->nghost_tot, nc = gh->natm_comp_max;
        ga = minus_one(gh->ighost_map, ng);
        gc = (int *)malloc(sizeof(int) * (size_t)ng * nc);
        gcoef = (double *)malloc(sizeof(double) * (size_t)ng * nc);
        for (int g = 0; g < ng; g++)
            for (int c = 0; c < nc; c++) {
                const int has = c < gh->natm_comp[g + 1];
                gc[g * nc + c] = has ? gh->iatm_comp[c + 1][g + 1] - 1 : -1;
                gcoef[g * nc + c] = has ? gh->coef[c + 1][g + 1] : 0.0;
            }
        s.ghost_ncomp = nc;
        s.ghost_atom = ga;
        s.ghost_comp = gc;
        s.ghost_coef = gcoef;
    }
    const int rc = pinyb200_create(&s, ci->pi_beads_proc, mixed ? PINYB200_MIXED : PINYB200_FP64, ctx);
    void *tmp[] = {typ, imap, eoff, ej, e1, e2, b1, b2, bt, bc, bdc, a1, a2, a3, at, ac, as, adc, ads, ga, gc, gcoef};
    for (size_t k = 0; k < sizeof(tmp) / sizeof(tmp[0]); k++) free(tmp[k]);
    return rc;
}

/* natm x 3 copy of 1-based x/y/z */
static double *xyz_copy(const double *x, const double *y, const double *z, int n)
{
    double *a = (double *)malloc(sizeof(double) * (size_t)n * 3);
    for (int i = 0; i < n; i++) {
        a[3 * i] = x[i + 1];
        a[3 * i + 1] = y[i + 1];
        a[3 * i + 2] = z[i + 1];
    }
    return a;
}

/* The device Verlet list from bead 1, the mode-1 positions and PINY's
 * cutskin^2, and the reference positions PINY's next list test measures
 * displacements from (verlist_control.c:52-58). */
static int gpu_list(pinyb200_ctx *ctx, CLASS *class, GENERAL_DATA *general_data)
{
    CLATOMS_INFO *ci = &class->clatoms_info;
    CLATOMS_POS *p1 = &class->clatoms_pos[1];
    NBR_LIST *nl = &class->nbr_list;
    const int n = ci->natm_tot;
    double *x1 = xyz_copy(p1->x, p1->y, p1->z, n);
    double *xm = ci->pi_beads > 1 ? xyz_copy(ci->xmod, ci->ymod, ci->zmod, n) : NULL;
    long npairs = 0;
    const int rc = pinyb200_build_list(ctx, x1, xm, ZB(general_data->cell.hmat), ZB(class->interact.cutskin), &npairs);
    free(x1);
    free(xm);
    if (rc) return rc;
    for (int i = 1; i <= n; i++) {
        nl->x0[i] = p1->x[i];
        nl->y0[i] = p1->y[i];
        nl->z0[i] = p1->z[i];
    }
    return 0;
}

int gpu_energy_control(pinyb200_ctx *ctx, CLASS *class, BONDED *bonded, GENERAL_DATA *general_data, int first)
{
    (void)bonded;
    CLATOMS_INFO *ci = &class->clatoms_info;
    INTERACT *it = &class->interact;
    const int P = ci->pi_beads_proc, n = ci->natm_tot;
    /* PINY's list test, as nbr_list_control runs it */
    if (ci->pi_beads > 1) {
        get_pimd_spread(ci, class->clatoms_pos, &it->spread_now, &class->communicate);
        get_cut_skin(it->cutskin, it->cutskin_root, it->cutoff, it->cutskin_res, it->cutskin_root_res, it->cutoff_res,
                     it->skin, it->spread_now, it->brnch_root_skin, it->nter_typ);
    }
    int iflag = 1;
    if (!first) check_ver_list(ci, &class->clatoms_pos[1], &class->nbr_list, it, &iflag);
    else if (ci->pi_beads > 1) it->spread = it->spread_now;
    if (iflag) {
        int rc = gpu_list(ctx, class, general_data);
        if (rc) return rc;
        general_data->stat_avg.updates += 1.0;
    }
    /* forces of all beads; the virial forces receive the same sums */
    double **x = (double **)malloc(sizeof(double *) * 6 * (size_t)P);
    double **y = x + P, **z = x + 2 * P, **fx = x + 3 * P, **fy = x + 4 * P, **fz = x + 5 * P;
    double *f0 = (double *)malloc(sizeof(double) * (size_t)P * n * 3);
    for (int b = 0; b < P; b++) {
        CLATOMS_POS *cp = &class->clatoms_pos[b + 1];
        x[b] = cp->x;
        y[b] = cp->y;
        z[b] = cp->z;
        fx[b] = cp->fx;
        fy[b] = cp->fy;
        fz[b] = cp->fz;
        for (int i = 0; i < n; i++) {
            f0[((size_t)b * n + i) * 3 + 0] = cp->fx[i + 1];
            f0[((size_t)b * n + i) * 3 + 1] = cp->fy[i + 1];
            f0[((size_t)b * n + i) * 3 + 2] = cp->fz[i + 1];
        }
    }
    double pv0[9];
    for (int k = 0; k < 9; k++) pv0[k] = general_data->ptens.pvten_tot[k + 1];
    pinyb200_energies e;
    const int rc = pinyb200_piny_force(ctx, x, y, z, ci->pi_beads > 1 ? ci->xmod : NULL,
                                       ci->pi_beads > 1 ? ci->ymod : NULL, ci->pi_beads > 1 ? ci->zmod : NULL,
                                       general_data->cell.hmat, fx, fy, fz, general_data->ptens.pvten_tot, &e);
    if (rc == 0 && ci->pi_beads > 1)
        for (int b = 0; b < P; b++) {
            CLATOMS_POS *cp = &class->clatoms_pos[b + 1];
            for (int i = 0; i < n; i++) {
                cp->fxt[i + 1] += cp->fx[i + 1] - f0[((size_t)b * n + i) * 3 + 0];
                cp->fyt[i + 1] += cp->fy[i + 1] - f0[((size_t)b * n + i) * 3 + 1];
                cp->fzt[i + 1] += cp->fz[i + 1] - f0[((size_t)b * n + i) * 3 + 2];
            }
        }
    free(f0);
    free(x);
    if (rc) return rc;
    /* without RESPA PINY adds the same pressure tensor to pvten and pvten_tot */
    for (int k = 0; k < 9; k++) general_data->ptens.pvten[k + 1] += general_data->ptens.pvten_tot[k + 1] - pv0[k];
    /* energies as the three sub-steps book them (bead averages) */
    STAT_AVG *sa = &general_data->stat_avg;
    sa->vintert += e.vintert;
    sa->vintrat += e.vintrat;
    sa->vvdw += e.vvdw;
    sa->vcoul += e.vcoul;
    sa->vrecip += e.vrecip + e.vself + e.vbgr + e.vecor;
    sa->vlong += e.vlong;
    sa->vbondt += e.vbond;
    sa->vbendt += e.vbend;
    return 0;
}
