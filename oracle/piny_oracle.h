/*
 * Oracle: a plain-C, FP64, single-threaded restatement of PINY_MD's
 * per-bead force/energy path for flexible point-charge water.
 *
 * THIS IS TEST INFRASTRUCTURE.  It is the checker for the device path: only
 * the tests, the smoke check and the benchmark's CPU-baseline leg load it.
 * Nothing in the product links, imports or falls back to it.
 *
 * Every routine cites the PINY source (path relative to the PINY tree) whose
 * arithmetic it restates.  Indices are 0-based; arrays are plain C arrays in
 * PINY internal units (Bohr, Hartree).  The system description below carries
 * the same fields, in the same order, as the product's pinyb200_system in
 * include/pinyb200.h, so one host-side structure feeds both.
 *
 * Parity is pinned against PINY itself: oracle/_ref/piny_ref (PINY's own C
 * sources built by oracle/Makefile) dumps tables, lists, forces and energies
 * that tests/golden/ keeps as fixtures.
 */
#ifndef PINY_ORACLE_H
#define PINY_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_system {
    /* sites (atoms plus massless ghosts) */
    int natm;
    int ntyp;
    const int *atm_typ;        /* [natm] 0-based atom type                  */
    const double *charge;      /* [natm]                                    */

    /* real-space interaction tables (PINY INTERACT) */
    int nsplin;
    int ninter_unique;
    const int *inter_map;      /* [ntyp(ntyp+1)/2] pair type -> table index */
    const double *cutoff;      /* [npair] force cutoff                      */
    const double *rmin_spl;    /* [nuniq]                                   */
    const double *dr_spl;      /* [nuniq]                                   */
    const double *dri_spl;     /* [nuniq]                                   */
    const double *cv0;         /* [nuniq*nsplin] vdW energy table           */
    const double *cdv0;        /* [nuniq*nsplin] vdW -(1/r)dV/dr table      */
    const double *cv0_c;       /* [nuniq*nsplin] Ewald real-space energy    */
    const double *cdv0_c;      /* [nuniq*nsplin] Ewald real-space force     */
    double skin;
    double clong;              /* LJ tail constant, vlong = clong/vol       */
    int iswit_vdw;             /* 1: switched tables (shift_inter_pe swit)  */

    /* exclusions, CSR over atoms, every j < i */
    const int *excl_off;       /* [natm+1]                                  */
    const int *excl_j;         /* [nexcl]                                   */

    /* Ewald / PME */
    double alp_ewd;
    double self_erf;
    int nktot;
    const int *kastr;          /* [nktot] half-space k list                 */
    const int *kbstr;
    const int *kcstr;
    const double *bweight;     /* [nktot] |b_a b_b b_c|^2                   */
    int ngrid_a, ngrid_b, ngrid_c;
    int n_interp;

    /* Ewald exclusion correction (PINY ECOR) */
    int necor;
    const int *ecor_j1;
    const int *ecor_j2;
    int ecor_nsplin;
    double ecor_rmin;
    double ecor_dr;
    double ecor_dri;
    const double *ecor_cv0;
    const double *ecor_cdv0;

    /* power-series bonds (PINY BOND) */
    int nbond;
    const int *bond_j1;
    const int *bond_j2;
    const int *bond_typ;
    int nbond_typ;
    const double *bond_eq;     /* [ntyp]                                    */
    const double *bond_c;      /* [ntyp*7]  c_0..c_6                        */
    const double *bond_dc;     /* [ntyp*7]  dc_0..dc_6                      */

    /* cos/sin-series bends (PINY BEND) */
    int nbend;
    const int *bend_j1;
    const int *bend_j2;
    const int *bend_j3;
    const int *bend_typ;
    int nbend_typ;
    const double *bend_c;      /* [ntyp*7] */
    const double *bend_s;      /* [ntyp*7] */
    const double *bend_dc;     /* [ntyp*7] */
    const double *bend_ds;     /* [ntyp*7] */

    /* ghosts (PINY GHOST_ATOMS) */
    int nghost;
    int ghost_ncomp;           /* components per ghost (padded)             */
    const int *ghost_atom;     /* [nghost]                                  */
    const int *ghost_comp;     /* [nghost*ncomp], -1 = unused               */
    const double *ghost_coef;  /* [nghost*ncomp]                            */
} orc_system;

/* Energies and virial of one evaluation, bead-summed (PINY divides the
 * inter/intra energies by P; orc_energy_force reports both views). */
typedef struct orc_energies {
    double vreal;      /* real-space pairs, bead average                    */
    double vvdw;       /* vdW part of vreal + vlong                         */
    double vcoul;      /* Coulomb part of vreal + vrecip + self + bgr + ecor */
    double vrecip;     /* PME reciprocal, bead average                      */
    double vself, vbgr, vecor, vlong;
    double vbond, vbend;
    double vintert;    /* vreal + vlong + vrecip + vself + vbgr + vecor      */
    double vintrat;    /* vbond + vbend                                     */
    double pvten[9];   /* bead-summed pressure tensor (PINY pvten_tot)      */
} orc_energies;

/* RESPA split of the force (energy_control_initial.c:211-243 weights,
 * force_npol.c:805-816 / :1030-1060 switch and multipliers, bond_both.c,
 * bond.c, bend.c, ecorr.c, ewald3d_pme.c weights).  Level bits are the
 * energy_ctrl flags int_NVT_pimd sets (int_NVT_pimd.c:175-189). */
typedef struct orc_respa {
    double wght_ter, wght_ter_res, wght_tra_res;
    int int_res_ter;            /* energy_ctrl.int_res_ter                  */
    int int_res_inter;          /* intra_scr.int_res_inter (nres_ter > 1)   */
    int ires_bond;              /* bond() irespa: nres_tra*nres_tor > 1     */
    const double *cutoff_res;   /* [npair_typ] interact.cutoff_res (Bohr)   */
    double rheal_res;           /* interact.rheal_res (Bohr)                */
    const double *bond_eq_res;  /* [nbond_typ] bond.eq_pow_res              */
    int nktot_res;              /* ewald.nktot_res                          */
    const double *ecor_cdv0_res; /* [ecor_nsplin] ecor.cdv0_res             */
    /* PINY's separate RESPA PME mesh (part_mesh.pme_res_on): mesh, order,
     * RESPA k sphere and its B-spline weights (bweight_tot_res)           */
    int pme_res_on;
    int ngrid_res[3];
    int n_interp_res;
    const int *kastr_res, *kbstr_res, *kcstr_res;
    const double *bweight_res;
} orc_respa;
#define ORC_FULL_INTER 1
#define ORC_RES_INTER 2
#define ORC_FULL_INTRA 4
#define ORC_RES_INTRA 8
void orc_respa_force(const orc_system *s, const orc_respa *r, int level, int P,
                     const double *pos, const double *xmod, const double *h,
                     long npairs, const int *pi, const int *pj,
                     int distribute_ghosts, double *force, double *forcet);

/* ---- setup restatements -------------------------------------------------*/
void orc_spline_table(int nsplin, double rmin, double rmax, int itype,
                      double sig, double eps, double alp, double rheal,
                      int ishift, double *v, double *dv, double *dr,
                      double *dri);
double orc_ewald_ecut(int kmax, double deth);
void orc_kmaxv(double ecut, const double *hmati, int *kmaxv);
int orc_kvec_count(double ecut, const int *kmaxv, const double *hmati);
int orc_kvec_fill(double ecut, const int *kmaxv, const double *hmati,
                  int *ka, int *kb, int *kc);
void orc_pme_grid(double ecut, double deth, const double *hmati,
                  const int *kmaxv, int kmax_pme, int *ngrid);
void orc_pme_bweight(int nk, const int *ka, const int *kb, const int *kc,
                     const int *ngrid, int n_interp, double *bw);
void orc_ecor_table(int nsplin, double rmax, double alp, double ecut,
                    double *cv0, double *cdv0, double *dr, double *dri,
                    double *self_erf);
void orc_gauss_legendre(int n, double *node, double *weight);
void orc_bond_power(double c2, double c3, double c4, double *c, double *dc);
void orc_bend_harm(double fk, double theta0, double *c, double *s,
                   double *dc, double *ds);
double orc_clong(int natm, int ntyp, const int *atm_typ, const double *c6,
                 const double *cutoff, double rheal, int iswit);

/* ---- evaluation restatements --------------------------------------------*/
long orc_verlist(const orc_system *sys, const double *x, const double *y,
                 const double *z, const double *xmod, const double *ymod,
                 const double *zmod, const double *hmat, const double *hmati,
                 const double *cutskin2, long cap, int *pi, int *pj);
/* The rows i in [ilo, ihi) of the same list (checks of large boxes). */
long orc_verlist_rows(const orc_system *sys, const double *x, const double *y,
                      const double *z, const double *xmod, const double *ymod,
                      const double *zmod, const double *hmat,
                      const double *cutskin2, int ilo, int ihi, long cap,
                      int *pi, int *pj);

/* Verlet-list rebuild test: check_ver_list (nbr_list_control.c:182-247),
 * get_pimd_spread (pimd_estimators.c:121-220), get_cut_skin
 * (nbr_list_control.c:249-281).  pos: nbeads x natm x 3, x0: natm x 3 bead-1
 * positions at the last build.  Returns the rebuild flag. */
int orc_check_list(int natm, int nbeads, const double *pos, const double *x0,
                   double skin, double spread_ref, int ninter,
                   const double *cutoff, double *rmax, double *spread_now,
                   double *cutskin2);

/* Ring-polymer transforms, in place on x[P][natm][3] (bead-major).
 * kind 1 staging (transform_stg.c), 2 normal modes (transform_cnt.c);
 * what 0 positions -> modes, 1 modes -> positions, 2 forces -> mode forces. */
int orc_pimd_transform(int natm, int nbeads, int kind, int what, double *x);

/* PIMD bookkeeping around the force call (pimd_oracle.c). */
void orc_nhc_apply(int natm, const int *inhc, const double *m, double *v, int num_nhc, int len_nhc,
                   int nres_nhc, int nyosh, const double *wdti, const double *mass_nhc, const double *gkt,
                   double *x_nhc, double *v_nhc);
double orc_pimd_springs(int natm, int P, const double *u, const double *prekf, const double *veig, double wght,
                        double *fm, double *pvten_mode_tot);
double orc_pimd_force_post(int natm, int P, int kind, double *f, const double *x, const double *xmod,
                           const double *fm, int nfree_atoms, double beta, double *pvten, double *pvten_tot);

void orc_energy_force(const orc_system *sys, int nbeads, const double *pos,
                      const double *xmod, const double *hmat,
                      long npairs, const int *pi, const int *pj,
                      int distribute_ghosts, double *force,
                      orc_energies *e);

double orc_pimd_force_post_respa(int natm, int P, int kind, double *f, double *ft, const double *x,
                                 const double *xmod, const double *fm, int nfree_atoms, double beta, int full,
                                 double *pvten, double *pvten_tot);

#ifdef __cplusplus
}
#endif
#endif
