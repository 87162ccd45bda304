/*
 * pinyb200 -- B200-native force path for PINY_MD flexible point-charge water.
 *
 * C ABI: plain pointers and sizes, no CUDA or torch types.  Indices are
 * 0-based, arrays are in PINY internal units (Bohr, Hartree).  Every entry
 * point returns a pinyb200_status; none of them exits the process.
 *
 * The path replaces the three force sub-steps PINY's integrators reach
 * through energy_control()/energy_control_pimd():
 *   energy_control_inter_real   (src/energy/control/energy_control_inter_real.c:33)
 *   energy_control_inter_recip  (src/energy/control/energy_control_inter_recip.c:32)
 *   energy_control_intra        (src/energy/control/energy_control_intra.c:33)
 * as called from energy_control_pimd.c:91-111 and energy_control.c:49-74,
 * for all path-integral beads at once.
 */
#ifndef PINYB200_H
#define PINYB200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pinyb200_status {
    PINYB200_OK = 0,
    PINYB200_ERR_ARG = 1,            /* bad argument or inconsistent sizes      */
    PINYB200_ERR_CUDA = 2,           /* a CUDA runtime call failed              */
    PINYB200_ERR_NO_DEVICE = 3,      /* no usable GPU                           */
    PINYB200_ERR_LIST_OVERFLOW = 4,  /* Verlet list larger than its capacity    */
    PINYB200_ERR_CUTOFF = 5,         /* reserved (PINY only warns; not checked) */
    PINYB200_ERR_TIMEOUT = 6,        /* reserved (no kernel waits on another)   */
    PINYB200_ERR_NAN = 7,            /* non-finite energy (forces are written)  */
    PINYB200_ERR_UNSUPPORTED = 8,    /* option not built for this path          */
    PINYB200_ERR_STATE = 9           /* call order violated (e.g. no list yet)  */
} pinyb200_status;

enum {
    PINYB200_FP64 = 0,  /* every kernel in FP64                                */
    PINYB200_MIXED = 1  /* FP32 pair/PME arithmetic, FP64 force accumulation,  */
                        /* FP64 energies/virial and intramolecular terms      */
};

/* Flags for pinyb200_energy_force*(). */
enum {
    PINYB200_DISTRIB_GHOSTS = 1, /* apply distrib_ghost_force (ghost_control.c:71) */
    PINYB200_NO_ENERGY = 2,      /* skip energy/virial reductions                   */
    PINYB200_SITE_PAIRS = 4,     /* walk the site list instead of molecule pairs    */
    PINYB200_TUNE_AGAIN = 8,     /* pinyb200_autotune: ignore remembered results    */
    PINYB200_UPDATE_LIST = 16,   /* device list test and rebuild before the forces  */
    PINYB200_BATCH_BRANCHES = 32, /* batch call: one graph branch per box           */
    PINYB200_BATCH_KERNELS = 64   /* batch call: the multi-box kernels where they   */
                                  /* cover the boxes (branches otherwise), untimed  */
};

/*
 * Set-up data of one box: the products of PINY's input stage (parse()),
 * field by field.  PINY owns these arrays; pinyb200_create copies them.
 *   INTERACT       cv0/cdv0/cv0_c/cdv0_c, rmin_spl, dr_spl, dri_spl,
 *                  inter_map_index, cutoff   (include/typ_defs/typedefs_class.h:610)
 *   EXCL           num/j_off/j -> excl_off/excl_j (typedefs_bnd.h:449)
 *   EWALD          alp_ewd, self_erf, kastr/kbstr/kcstr (typedefs_gen.h:232)
 *   PART_MESH      bweight_tot, ngrid_*, n_interp (typedefs_class.h:790)
 *   ECOR, BOND, BEND, GHOST_ATOMS (typedefs_bnd.h:420, :21, :182;
 *                  typedefs_class.h:225)
 */
typedef struct pinyb200_system {
    int natm;
    int ntyp;
    const int *atm_typ;
    const double *charge;

    int nsplin;
    int ninter_unique;
    const int *inter_map;
    const double *cutoff;
    const double *rmin_spl;
    const double *dr_spl;
    const double *dri_spl;
    const double *cv0;
    const double *cdv0;
    const double *cv0_c;
    const double *cdv0_c;
    double skin;
    double clong;
    int iswit_vdw;

    const int *excl_off;
    const int *excl_j;

    double alp_ewd;
    double self_erf;
    int nktot;
    const int *kastr;
    const int *kbstr;
    const int *kcstr;
    const double *bweight;
    int ngrid_a, ngrid_b, ngrid_c;
    int n_interp;

    int necor;
    const int *ecor_j1;
    const int *ecor_j2;
    int ecor_nsplin;
    double ecor_rmin;
    double ecor_dr;
    double ecor_dri;
    const double *ecor_cv0;
    const double *ecor_cdv0;

    int nbond;
    const int *bond_j1;
    const int *bond_j2;
    const int *bond_typ;
    int nbond_typ;
    const double *bond_eq;
    const double *bond_c;
    const double *bond_dc;

    int nbend;
    const int *bend_j1;
    const int *bend_j2;
    const int *bend_j3;
    const int *bend_typ;
    int nbend_typ;
    const double *bend_c;
    const double *bend_s;
    const double *bend_dc;
    const double *bend_ds;

    int nghost;
    int ghost_ncomp;
    const int *ghost_atom;
    const int *ghost_comp;
    const double *ghost_coef;
} pinyb200_system;

/* Energy components with PINY's bead averaging
 * (energy_control_inter_real.c:141-183, energy_control_inter_recip.c:341-349,
 *  energy_control_intra.c:284-309).  pvten is the bead-summed PINY pvten_tot. */
typedef struct pinyb200_energies {
    double vreal, vvdw, vcoul, vrecip, vself, vbgr, vecor, vlong;
    double vbond, vbend, vintert, vintrat;
    double pvten[9];
} pinyb200_energies;

typedef struct pinyb200_ctx pinyb200_ctx;

/* Library version and the device it will use. */
int pinyb200_version(void);
int pinyb200_device_info(char *name, int len, int *sm_count);

/* Create a context for one box with nbeads path-integral beads (the
 * per-replica state PINY keeps in CLASS/BONDED/GENERAL_DATA).  One context
 * per CLASS; contexts are independent and may be driven from separate host
 * threads (python/piny/piny.pyx:426-436 runs replicas concurrently). */
int pinyb200_create(const pinyb200_system *sys, int nbeads, int precision,
                    pinyb200_ctx **out);
int pinyb200_destroy(pinyb200_ctx *ctx);

/*
 * Build the Verlet list from bead-1 positions: every non-excluded pair
 * i > j whose minimum-image separation has r^2 < cutskin2[pair type]
 * (verlist_control.c:30-128 -> verlist_create.c:25-221).  For PIMD the image
 * shift comes from xmod, the mode-1 positions (period_pimd, period.c:121);
 * pass xmod = NULL for classical runs.
 *   pos1, xmod : natm x 3 (AoS) host arrays;  hmat : 9, column-major;
 *   cutskin2   : ntyp(ntyp+1)/2 squared list radii (get_cut_skin,
 *                nbr_list_control.c:249-281).
 * Returns the number of pairs in *npairs.
 */
int pinyb200_build_list(pinyb200_ctx *ctx, const double *pos1,
                        const double *xmod, const double *hmat,
                        const double *cutskin2, long *npairs);

/* Copy the current list out as (i, j) pairs, i > j, in the device's order. */
int pinyb200_get_list(pinyb200_ctx *ctx, int *pi, int *pj, long cap,
                      long *npairs);

/*
 * How the molecule-pair list is enumerated, PINY's two list generators
 * (verlist_control.c:64-110):
 *   PINYB200_LIST_LNK   (default) link cells, as lnk_ver_update /
 *                       lnk_ver_gen_pad: molecules binned by their site-0
 *                       bead-1 position into cells at least half the
 *                       molecule reach wide; each home cell's molecules
 *                       meet the molecules of the 5 x 5 x 5 cells around
 *                       it.  Used when every cell axis holds >= 5 cells and
 *                       the 125 cells are at most 40 % of the box, else the
 *                       sweep runs.
 *   PINYB200_LIST_NOLST the all-pairs sweep, as nolst_ver_update /
 *                       nolst_ver_gen.
 * Both give the same pair set; a row's pairs come in neighbour-cell order
 * with cells and in index order with the sweep.  The method applies from
 * the next pinyb200_build_list (which plans the cells for its positions;
 * device rebuilds keep that plan and sweep when the molecules' reach has
 * outgrown it).  pinyb200_list_cells returns the plan of the current list:
 * cells[0..2] the cells along a, b, c (zeros when it swept) and cells[3] 1
 * when the cells built it.  Systems not made of molecules of <= 4
 * sites use the site sweep for either method.
 */
#define PINYB200_LIST_LNK 0
#define PINYB200_LIST_NOLST 1
int pinyb200_set_list_method(pinyb200_ctx *ctx, int method);
int pinyb200_list_cells(pinyb200_ctx *ctx, int *cells);

/*
 * Rebuild test of the current list for positions on the device, as PINY
 * runs it each step before the force call (nbr_list_control.c:63-110):
 *   *rmax       = max over atoms of |r(bead 1) - r(at the last build)|
 *                 (check_ver_list, nbr_list_control.c:182-247);
 *   *spread_now = max over beads > 1 and atoms of |r(bead) - r(bead 1)|
 *                 (get_pimd_spread, pimd_estimators.c:121-220; 0 for P = 1);
 *   *rebuild    = rmax > skin/2 + max(0, spread_now - spread_ref), where
 *                 spread_ref is PINY's interact.spread (the spread when the
 *                 list was last rebuilt; set it to spread_now on a rebuild);
 *   cutskin2    = (cutoff + skin + spread_now)^2 per type pair (get_cut_skin,
 *                 nbr_list_control.c:249-281), the radii for the next
 *                 pinyb200_build_list; may be NULL.
 * d_pos: nbeads x natm x 3 device array; stream as in
 * pinyb200_energy_force_device.  Any output pointer may be NULL.
 */
int pinyb200_check_list_device(pinyb200_ctx *ctx, const double *d_pos,
                               double spread_ref, int *rebuild, double *rmax,
                               double *spread_now, double *cutskin2,
                               void *stream);

/* Sizes of the current list: all pairs, the force-bearing ("active") pairs
 * the pair kernel walks (a charge product or a vdW table), and capacity. */
int pinyb200_list_info(pinyb200_ctx *ctx, long *npairs, long *nactive,
                       long *capacity);

/*
 * Pair count without allocation.  This entry point has no counterpart in
 * the reference: PINY sizes its list by counting inside verlist_create and
 * growing with realloc, which a caller that must not allocate device memory
 * cannot do.  Counts, for bead-1 positions already on the device, the pairs
 * pinyb200_build_list would hold (*npairs) and the force-bearing subset
 * (*nactive), with the same FP64 criterion, without touching the context's
 * list.  Arguments as in pinyb200_build_list, except:
 *   d_pos1, d_xmod : device arrays natm x 3 (d_xmod may be NULL);
 *   stream         : opaque CUDA stream handle, NULL = the context's stream;
 *                    the call returns after that stream is idle.
 * It calls no cudaMalloc/cudaFree: its scratch is one fixed device array per
 * GPU inside the library (4096 B + 8 B per atom of the limit: 528,384 B,
 * about 0.5 MiB), so
 *   - it accepts natm <= PINYB200_COUNT_MAX_ATOMS and at most
 *     PINYB200_COUNT_MAX_PAIR_TYPES pair types (ntyp(ntyp+1)/2), and returns
 *     PINYB200_ERR_ARG beyond them;
 *   - the first call on each GPU looks up the scratch address
 *     (cudaGetSymbolAddress, which may load the library's device code):
 *     make that first call before any stream capture begins;
 *   - calls on the same GPU share the scratch: calls that overlap in time
 *     (from several host threads, or on several streams) race and give
 *     wrong counts; serialise them.
 */
enum {
    PINYB200_COUNT_MAX_ATOMS = 65536,
    PINYB200_COUNT_MAX_PAIR_TYPES = 64
};
int pinyb200_count_list_device(pinyb200_ctx *ctx, const double *d_pos1,
                               const double *d_xmod, const double *hmat,
                               const double *cutskin2, long *npairs,
                               long *nactive, void *stream);

/*
 * One force/energy evaluation of all beads with host buffers.
 *   pos   : nbeads x natm x 3 host array (bead-major AoS), ghosts are
 *           recomputed from their components (get_ghost_pos);
 *   xmod  : natm x 3 mode-1 positions for the PIMD image, or NULL;
 *   force : nbeads x natm x 3 output, overwritten (not accumulated).
 */
int pinyb200_energy_force(pinyb200_ctx *ctx, const double *pos,
                          const double *xmod, const double *hmat, int flags,
                          double *force, pinyb200_energies *e);

/* Same, with device-resident pos / xmod / force (cudaMalloc'd by the
 * caller, same layouts).  The work is launched on the CUDA stream passed as
 * an opaque handle (NULL = the context's own stream); the call returns after
 * that stream is idle. */
int pinyb200_energy_force_device(pinyb200_ctx *ctx, const double *d_pos,
                                 const double *d_xmod, const double *hmat,
                                 int flags, double *d_force,
                                 pinyb200_energies *e, void *stream);

/*
 * PINY-layout drop-in for energy_control_inter_real + _inter_recip + _intra
 * over all beads.  x[ip], y[ip], z[ip] and fx[ip], fy[ip], fz[ip] are
 * PINY's 1-based per-bead arrays (clatoms_pos[ip+1].x etc., element 1 is the
 * first atom); xmod/ymod/zmod are clatoms_info.xmod etc. (1-based) or NULL;
 * hmat is cell.hmat (1-based).  Forces and pvten_tot (1-based, 9) are ADDED
 * to, as PINY's routines do; energies are returned in *e.  PINY also adds
 * every one of these forces to the virial forces fxt/fyt/fzt (force_npol,
 * the reciprocal sum, bond, bend, ecor); without RESPA they equal the forces
 * added here, so a PIMD shim adds the same values to fxt.
 */
int pinyb200_piny_force(pinyb200_ctx *ctx, double *const *x,
                        double *const *y, double *const *z, const double *xmod,
                        const double *ymod, const double *zmod,
                        const double *hmat, double *const *fx,
                        double *const *fy, double *const *fz,
                        double *pvten_tot, pinyb200_energies *e);

/*
 * RESPA split of the force (PINY's respa_steps_lrf / _intra / _pimd).
 * PINY's integrators nest RESPA loops and ask the force routines for one
 * level per inner step through four energy_ctrl flags (int_NVT_pimd.c:
 * 175-189); each term is weighted by the number of inner steps its impulse
 * spans (energy_control_initial.c:211-243).  pinyb200_set_respa stores the
 * split's set-up (NULL switches it off):
 *   wght_ter, wght_ter_res, wght_tra_res   for_scr.wght_* as
 *                  energy_control_initial sets them
 *   int_res_ter    energy_ctrl.int_res_ter (respa_steps_lrf given)
 *   int_res_inter  intra_scr.int_res_inter (nres_ter > 1): bond_both's
 *                  outer weight is wght_ter_res when set, else wght_ter
 *   ires_bond      energy_control_intra.c:116-119 (nres_tra*nres_tor > 1):
 *                  intra-only levels use the bonds' RESPA equilibria
 *   cutoff_res     interact.cutoff_res per pair type (npair_typ, Bohr)
 *   rheal_res      interact.rheal_res (Bohr), the switch width
 *   bond_eq_res    bond.eq_pow_res per bond type (nbond_typ, Bohr)
 *   nktot_res      ewald.nktot_res (> 0: ewald_respa_kmax given).  With
 *                  one PME grid (pme_res_on 0; PINY then demands
 *                  kmax_res = kmax) the reciprocal sum moves to the inner
 *                  inter level: PME x wght_ter_res at every RES_INTER level
 *                  (energy_control_inter_recip.c:184-213), the exclusion
 *                  correction at the inner level from ecor_cdv0_res x
 *                  wght_ter_res (ecorr.c:97-106) and at the outer level as
 *                  ecor_both, wght_ter F + (wght_ter_res - wght_ter) F_res
 *                  (ecorr.c:349-351, :497-505)
 *   pme_res_on     part_mesh.pme_res_on (ewald_respa_pme_opt on): the
 *                  RESPA reciprocal set on its own PME mesh
 *                  (energy_control_inter_recip.c:215-271, irespa = 1 in
 *                  ewald3d_pme.c:204-216): at inner inter levels PME on
 *                  that mesh x wght_ter_res; at the outer level PME on
 *                  the full mesh x wght_ter plus PME on the RESPA mesh x
 *                  (wght_ter_res - wght_ter), both added unweighted to the
 *                  virial forces (ewald3d_pme.c:563-585), the energy and
 *                  pvten_tot from the full mesh only
 *   ngrid_res, n_interp_res
 *                  part_mesh.ngrid_a_res/_b_res/_c_res, n_interp_res
 *   kastr_res, kbstr_res, kcstr_res
 *                  ewald.kastr_res... (nktot_res each): the RESPA k sphere
 *   bweight_res    part_mesh.bweight_tot_res (nktot_res)
 *   ecor_cdv0_res  ecor.cdv0_res (ecor_nsplin entries) when nktot_res > 0
 * pinyb200_respa_force_device evaluates one level, `level` being the OR of
 * the PINYB200_* flag bits below that PINY has set: one of
 *   RES_INTRA; FULL_INTRA|RES_INTRA; RES_INTER|FULL_INTRA|RES_INTRA (needs
 *   int_res_ter); FULL_INTER|FULL_INTRA with or without RES_INTRA, with
 *   RES_INTER exactly when int_res_ter (the levels int_NVT_pimd's loops
 *   and control_pimd's first force call produce).
 * d_force receives PINY's weighted forces fx: real-space pairs x the RESPA
 * multiplier (inner levels shave at cutoff_res; force_npol.c:805-816,
 * :1030-1060), PME and the exclusion correction x wght_ter at the outer
 * level only (nktot_res = 0; see above otherwise), bonds as bond_both /
 * bond, bends x wght_tra_res.  At the outer
 * level d_forcet (may be NULL) receives the unweighted forces PINY adds to
 * the virial forces fxt, and *e the energies and pvten_tot of
 * pinyb200_energy_force_device; at inner levels *e is zeroed (PINY books
 * energies at the outer step).  flags: PINYB200_DISTRIB_GHOSTS,
 * PINYB200_UPDATE_LIST.  The inner levels use the active site list shaved
 * at cutoff_res in place of PINY's separate RESPA Verlet list (pairs within
 * cutoff_res + skin + spread at the build); under the list's own validity
 * rule the two hold the same pairs inside cutoff_res.
 */
#define PINYB200_FULL_INTER 1
#define PINYB200_RES_INTER 2
#define PINYB200_FULL_INTRA 4
#define PINYB200_RES_INTRA 8
typedef struct pinyb200_respa {
    double wght_ter, wght_ter_res, wght_tra_res;
    int int_res_ter, int_res_inter, ires_bond;
    const double *cutoff_res;
    double rheal_res;
    const double *bond_eq_res;
    int nktot_res;
    int pme_res_on;
    const double *ecor_cdv0_res;
    int ngrid_res[3];
    int n_interp_res;
    const int *kastr_res, *kbstr_res, *kcstr_res;
    const double *bweight_res;
} pinyb200_respa;
int pinyb200_set_respa(pinyb200_ctx *ctx, const pinyb200_respa *r);
int pinyb200_respa_force_device(pinyb200_ctx *ctx, const double *d_pos,
                                const double *d_xmod, const double *hmat,
                                int level, int flags, double *d_force,
                                double *d_forcet, pinyb200_energies *e,
                                void *stream);
/* PINY-layout form (arrays as pinyb200_piny_force): forces ADDED to fx/fy/fz
 * and, at the outer level, the virial forces to fxt/fyt/fzt (may be NULL)
 * and pvten_tot; ghost forces are left on the ghost sites, as PINY's force
 * routines leave them for energy_control_final. */
int pinyb200_piny_force_respa(pinyb200_ctx *ctx, int level, double *const *x,
                              double *const *y, double *const *z,
                              const double *xmod, const double *ymod,
                              const double *zmod, const double *hmat,
                              double *const *fx, double *const *fy,
                              double *const *fz, double *const *fxt,
                              double *const *fyt, double *const *fzt,
                              double *pvten_tot, pinyb200_energies *e);

/*
 * Launch shapes and the autotuner.  A context runs with four choices:
 *   choice[0]  PME tile edge, 8 or 16 grid points (charges are binned per
 *              tile and bead; spread and gather run one block per tile)
 *   choice[1]  pair kernel: 0 molecule pairs (when the system is made of
 *              identical molecules of <= 4 sites; in MIXED, when all their
 *              site pairs share one cutoff and spline grid, with combined
 *              per-site-pair force and energy rows), 1 the site list,
 *              2 molecule pairs with PINY's per-table rows
 *   choice[2]  pair kernel grid cap, blocks per SM (1..64)
 *   choice[3]  1: PME on a second stream, concurrent with the pair kernel
 * pinyb200_autotune times every combination on the caller's inputs
 * (device positions as in pinyb200_energy_force_device; `reps` timed runs
 * each after one warm-up), keeps the fastest, returns it in choice[4] and
 * its device time in *best_ms, and remembers it for the rest of the process
 * for every context of the same shape (atoms, beads, mesh, order,
 * precision); later calls for that shape only apply it (*best_ms = -1)
 * unless flags holds PINYB200_TUNE_AGAIN.  Results do not depend on the
 * choice beyond floating-point summation order.  No counterpart in PINY,
 * whose force path has no launch shapes.
 */
int pinyb200_autotune(pinyb200_ctx *ctx, const double *d_pos,
                      const double *d_xmod, const double *hmat, int flags,
                      int reps, int *choice, float *best_ms);
int pinyb200_get_tuning(pinyb200_ctx *ctx, int *choice);
int pinyb200_set_tuning(pinyb200_ctx *ctx, const int *choice);

/*
 * Many independent boxes per call (the batched path).  A batch groups
 * contexts on one GPU (different sizes, bead counts and meshes are fine).
 * pinyb200_batch_energy_force_device evaluates every box, as
 * pinyb200_energy_force_device would one by one, from per-box device arrays
 * (d_xmod may be NULL, or hold NULL entries) and host cells, and writes
 * e[i] for box i (e may be NULL).  The work of one call is one CUDA graph
 * launch, captured on the first call and again whenever a device pointer, a
 * cell or the flags change, after one plain run of every box.  When every
 * box is MIXED with the molecule-pair kernel (q-TIP4P/F or q-SPC/Fw site
 * pattern), an orthorhombic cell and the compact PME path, and flags hold
 * neither PINYB200_UPDATE_LIST, PINYB200_SITE_PAIRS nor
 * PINYB200_BATCH_BRANCHES, the graph holds multi-box kernels: each phase
 * (staging, PME bin / spread / three FFT passes / gather, pair forces,
 * intramolecular terms, finishing) is one persistent launch per group of
 * boxes sharing its compile-time shape, walking every (box, bead, tile or
 * chunk) block of the group; the groups' PME chains, pair launches and the
 * intramolecular launch are parallel branches of the graph.  Otherwise
 * every box is a parallel branch of its own kernels.  Where the multi-box
 * kernels cover the boxes, the capture times both forms on the call's
 * inputs and keeps the faster, unless flags ask for one form
 * (PINYB200_BATCH_KERNELS or PINYB200_BATCH_BRANCHES).  The call returns when the work is done.  PINY's Python
 * driver reaches several replicas through one energy_control call per CLASS
 * (python/piny/piny.pyx:426-436); this entry point has no counterpart there.
 */
typedef struct pinyb200_batch pinyb200_batch;
int pinyb200_batch_create(pinyb200_ctx *const *ctx, int nbox,
                          pinyb200_batch **out);
int pinyb200_batch_destroy(pinyb200_batch *batch);
int pinyb200_batch_energy_force_device(pinyb200_batch *batch,
                                       const double *const *d_pos,
                                       const double *const *d_xmod,
                                       const double *const *hmat, int flags,
                                       double *const *d_force,
                                       pinyb200_energies *e, void *stream);
/* Device time of the last batch call (CUDA events around the graph launch). */
int pinyb200_batch_last_ms(pinyb200_batch *batch, float *ms);
/* How the last captured batch graph runs: *fused 1 for the multi-box
 * kernels, 0 for one branch per box; *launches its kernel launches. */
int pinyb200_batch_last_mode(pinyb200_batch *batch, int *fused, int *launches);
const char *pinyb200_batch_last_error(pinyb200_batch *batch);

/*
 * Parameter gradients (adjoint).  A tangent holds the derivative of the
 * set-up data with respect to one model parameter theta_k; NULL parts are
 * zero.  Array sizes as the matching pinyb200_system fields:
 *   dcharge      natm                  d charge
 *   dcv0, dcdv0  ninter_unique*nsplin  d vdW tables (cv0, cdv0)
 *   dghost_coef  nghost*ghost_ncomp    d ghost coefficients (moves the ghosts)
 *   dbond_eq     nbond_typ             d bond equilibrium length
 *   dbond_c      nbond_typ*7           d bond series c_0..c_6
 *   dbend_c/s/dc/ds  nbend_typ*7 each  d bend series (all four, or none)
 *   dclong       d clong (LJ tail, energy clong/volume)
 * pinyb200_grad_prepare copies up to 16 tangents to the device (it
 * allocates; call it when the parameters change).  pinyb200_grad then runs
 * one forward evaluation at d_pos / d_xmod / hmat (as
 * pinyb200_energy_force_device) and one adjoint pass, and returns for every
 * tangent
 *   dE[k] = d(vintert + vintrat) / d theta_k
 *   dF[k] = sum over beads and atoms of fbar . dF / d theta_k
 * where F are the forces with the ghost force distributed
 * (PINYB200_DISTRIB_GHOSTS) and fbar (device, nbeads x natm x 3, or NULL
 * for energy derivatives only) is the caller's upstream gradient, e.g.
 * 2 (F - F_target) for a force-matching loss.  Pair terms are recomputed
 * from the list, not stored.  No counterpart in PINY, which has no
 * parameter derivatives.
 */
typedef struct pinyb200_tangent {
    const double *dcharge;
    const double *dcv0, *dcdv0;
    const double *dghost_coef;
    const double *dbond_eq, *dbond_c;
    const double *dbend_c, *dbend_s, *dbend_dc, *dbend_ds;
    double dclong;
} pinyb200_tangent;
int pinyb200_grad_prepare(pinyb200_ctx *ctx, int ntan,
                          const pinyb200_tangent *tan);
int pinyb200_grad(pinyb200_ctx *ctx, const double *d_pos, const double *d_xmod,
                  const double *hmat, const double *d_fbar, double *dE,
                  double *dF, void *stream);

/* Milliseconds of the last evaluation, from CUDA events: 0 device work,
 * 1 pair forces, 2 PME, 3 intramolecular, 4 the whole host-buffer call of
 * pinyb200_energy_force (copies included).  PME runs on a second stream of
 * the context, concurrently with 1 and 3, so 1 + 2 + 3 may exceed 0. */
int pinyb200_last_timing(pinyb200_ctx *ctx, float *ms, int n);

/* Per-kernel timing, for measurement.  With on != 0 every later evaluation
 * of the context runs its kernels one after another on the context's
 * stream (PME not overlapped) with a CUDA event after each kernel;
 * pinyb200_kernel_times returns, for the last evaluation, the kernels in
 * launch order (names[i], static strings) and their milliseconds ms[i],
 * at most cap of them, their number in *count.  No counterpart in PINY
 * (its timer.c brackets whole routines on the host). */
int pinyb200_set_kernel_timing(pinyb200_ctx *ctx, int on);
int pinyb200_kernel_times(pinyb200_ctx *ctx, const char **names, float *ms, int cap, int *count);

/* FMA throughput of the current GPU in GFLOP/s (fp64 = 0: FP32, 1: FP64),
 * best of `reps` timed launches of a register-only probe: the ALU peak the
 * benchmark's roofline divides by.  No counterpart in PINY. */
int pinyb200_fma_peak(int fp64, int reps, double *gflops);

/*
 * PINY's per-step list update on the device: the rebuild test of
 * check_ver_list (nbr_list_control.c:182-247, with the PIMD spread) and,
 * when it fires, the list build of verlist_control (verlist_control.c:
 * 30-128) with get_cut_skin's cutskin^2 -- all enqueued on `stream`, no
 * host round trip, capturable in a CUDA graph (call it once outside a
 * capture first: that call sets up the device state).  d_pos: [P][natm][3]
 * with current ghost positions (PINY runs get_ghost_pos first); d_xmod: the
 * mode-1 positions (NULL for one bead).  The reference spread is kept on
 * the device (pinyb200_list_set_spread sets it; unset, the first call takes
 * the current spread).  The list must have been built once on the host
 * (pinyb200_build_list): device builds reuse its reservations (25 % slack);
 * a build that does not fit sets a sticky flag, the next evaluation returns
 * PINYB200_ERR_NAN and pinyb200_list_status PINYB200_ERR_LIST_OVERFLOW --
 * rebuild on the host then.  The same update runs inside
 * pinyb200_energy_force_device and the batch graph with
 * PINYB200_UPDATE_LIST, and inside every pinyb200_pimd_step.  No
 * counterpart call in PINY (it tests and rebuilds inside energy_control).
 */
typedef struct pinyb200_list_state {
    long rebuilds;           /* device rebuilds so far                       */
    int rebuilt_last;        /* the last update rebuilt                      */
    int overflow, mismatch;  /* sticky error flags                           */
    double rmax;             /* largest bead-1 displacement at the last test */
    double spread_now;       /* bead spread at the last test                 */
    double spread_ref;       /* bead spread of the current list              */
    long npairs, nactive;    /* site pairs (all, with a force) of the list   */
    long nmol_pairs;         /* molecule pairs of the list                   */
} pinyb200_list_state;

int pinyb200_update_list_device(pinyb200_ctx *ctx, const double *d_pos, const double *d_xmod,
                                const double *hmat, void *stream);
int pinyb200_list_set_spread(pinyb200_ctx *ctx, double spread_ref);
/* Reads the device state (waits for `stream`, NULL = the context's). */
int pinyb200_list_status(pinyb200_ctx *ctx, void *stream, pinyb200_list_state *out);

/* Ring-polymer transforms of PINY's PIMD integrators, in FP64, in place on
 * the device array d_x[nbeads][natm][3] (the bead-major layout of
 * pinyb200_energy_force_device), enqueued on `stream`.  No context needed.
 *   kind  PINYB200_STAGING      staging (pi_md_typ 1),
 *         PINYB200_NORMAL_MODES centroid normal modes (pi_md_typ 2);
 *   what  PINYB200_TO_MODES       positions -> modes
 *           (convert_pimd_mode_stag, transform_stg.c:92;
 *            convert_pimd_mode_cent, transform_cnt.c:240),
 *         PINYB200_TO_BEADS       modes -> positions
 *           (convert_pimd_pos_stag, transform_stg.c:164;
 *            convert_pimd_pos_cent, transform_cnt.c:321),
 *         PINYB200_FORCE_TO_MODES bead forces -> mode forces
 *           (convert_pimd_force_stag, transform_stg.c:31;
 *            convert_pimd_force_cent, transform_cnt.c:415).
 * Normal modes use PINY's packing: mode 1 = Re X_0, mode 2m = Re X_m,
 * mode 2m+1 = Im X_m, mode P = Re X_{P/2}, X_k = (1/P) sum_j x_j e^{2 pi i jk/P}.
 * Staging is bit-identical to PINY; normal modes agree to rounding.
 * nbeads 1 is a no-op (PINY skips it); else 2, 4, ..., 64. */
#define PINYB200_STAGING 1
#define PINYB200_NORMAL_MODES 2
#define PINYB200_TO_MODES 0
#define PINYB200_TO_BEADS 1
#define PINYB200_FORCE_TO_MODES 2
int pinyb200_pimd_transform(int natm, int nbeads, int kind, int what, double *d_x, void *stream);

/*
 * Path-integral MD around the force path, on the device, in FP64: PINY's
 * NVT ring-polymer step (int_NVT_pimd, src/integrate/pimd/int_NVT_pimd.c:
 * 142-217, with every RESPA count 1) as one call per step.
 *
 * A Nose-Hoover chain set is PINY's THERM_INFO (typedefs_class.h) for one
 * set of beads: the class set thermostats bead 1 (with the atom masses),
 * the bead set each of beads 2..P (with the bead masses; one chain state
 * per bead).  Chains are 0-based; chain num_nhc is the null chain.
 */
typedef struct pinyb200_nhc_set {
    int num_nhc;             /* chains (therm_info.num_nhc)                  */
    int len_nhc;             /* links per chain, 1..8                        */
    int nres_nhc;            /* RESPA steps of the chain operator            */
    int nyosh_nhc;           /* Yoshida-Suzuki stages, 1..9                  */
    const double *wdti;      /* [nyosh_nhc] stage weights x dti_nhc
                                (therm_info.wdti, from set_yosh)             */
    const int *inhc;         /* [3][natm] chain of each coordinate
                                (inhc_x, inhc_y, inhc_z)                    */
    const double *mass_nhc;  /* [len_nhc][num_nhc]                           */
    const double *gkt;       /* [len_nhc][num_nhc]                           */
} pinyb200_nhc_set;

typedef struct pinyb200_pimd_setup {
    int natm;                /* sites, ghosts included (as the force path)  */
    int nbeads;
    int kind;                /* PINYB200_STAGING or PINYB200_NORMAL_MODES    */
    const double *mass;      /* [natm] clatoms_info.mass                     */
    const double *bead_mass; /* [nbeads][natm] clatoms_pos[ip].mass          */
    const double *prekf;     /* [natm] clatoms_info.prekf                    */
    const double *path_eig;  /* [nbeads] clatoms_tran.path_eig (veig)        */
    double wght_pimd;        /* clatoms_info.wght_pimd (1 for NVT)           */
    double dt;               /* time step                                    */
    double beta;             /* BOLTZ / pi_temperature                       */
    int nfree_atoms;         /* natm - nghost - nfreeze (virial estimator)   */
    pinyb200_nhc_set class_nhc;
    pinyb200_nhc_set bead_nhc;
    /* RESPA (timeinfo.nres_ter, nres_tor, nres_tra, nres_pimd; 0 reads as 1)
     * and the level whose steps carry the chains (timeinfo.ix_respa, 1..5;
     * 0 reads as 1).  With a count above 1 the force context needs
     * pinyb200_set_respa; the chains' wdti must then be formed from PINY's
     * dt_nhc for ix_respa (int_NVT_pimd.c:96-125). */
    int nres_ter, nres_tor, nres_tra, nres_pimd;
    int ix_respa;
} pinyb200_pimd_setup;

typedef struct pinyb200_pimd_energies {
    pinyb200_energies force; /* the force path's, pvten = its bead sum        */
    double kin_harm;         /* sum of spring energies (stat_avg.kin_harm)    */
    double akvirx;           /* virial kinetic estimator (0.5 x PINY's sum)   */
    double pvten[9];         /* pvten / P with the centroid virial correction */
    double pvten_tot[9];     /* pvten_tot / P, likewise                       */
    double pvten_mode_tot[9];/* spring tensor (ptens.pvten_mode_tot)          */
} pinyb200_pimd_energies;

typedef struct pinyb200_pimd pinyb200_pimd;

/* Set up a step for one box; chain positions and velocities start at zero. */
int pinyb200_pimd_create(const pinyb200_pimd_setup *setup, pinyb200_pimd **out);
int pinyb200_pimd_destroy(pinyb200_pimd *pm);

/* Chain state, host arrays: set 0 (class) [len][num]; set 1 (bead)
 * [nbeads-1][len][num] for beads 2..P (therm_class / therm_bead[ip]). */
int pinyb200_pimd_set_nhc(pinyb200_pimd *pm, int set, const double *x_nhc, const double *v_nhc);
int pinyb200_pimd_get_nhc(pinyb200_pimd *pm, int set, double *x_nhc, double *v_nhc);

/* Mode forces of the bead positions d_x ([P][natm][3]): spring forces of
 * the modes (mode_energy_control, pimd_estimators.c:31), the force path
 * with the mode-1 image positions, and the post-processing of
 * energy_control_pimd.c:113-218 (bead forces / P, centroid virial
 * correction, forces to modes, springs added) into d_f.  With RESPA counts
 * above 1 the force path is asked for the outer level, as PINY's first
 * force call is (control_pimd.c:297-317).  Ghost positions in d_x are
 * recomputed (get_ghost_pos).  Work goes to `stream` (NULL: the
 * force context's own stream); the call blocks until it is done. */
int pinyb200_pimd_forces(pinyb200_pimd *pm, pinyb200_ctx *ctx, double *d_x, double *d_f,
                         const double *hmat, pinyb200_pimd_energies *e, void *stream);

/* One NVT step: chains and half kick (int_0_to_dt2_nvt_pimd,
 * int_0_to_dt2_pimd.c:34-190), positions to modes, drift, springs, modes
 * to positions, the device list update (pinyb200_update_list_device),
 * the forces as in pinyb200_pimd_forces, half kick and chains
 * (int_dt2_to_dt_nvt_pimd, int_dt2_to_dt_pimd.c).  With RESPA counts above
 * 1 the step is int_NVT_pimd's nested loops (int_NVT_pimd.c:142-223): every
 * inner step of dt / (nres_ter nres_tor nres_tra nres_pimd) kicks with the
 * current mode forces, the chains run at the inner steps that open / close
 * a loop of level <= ix_respa, positions go to modes at ir_pimd = 1 and back
 * at ir_pimd = nres_pimd, where the force path is asked for the level of
 * :175-189 (pinyb200_respa_force_device; the virial estimator from the
 * outer level's virial forces), and the other inner steps use the spring
 * forces alone.  d_x: bead positions, d_v: mode velocities, d_f: mode
 * forces of d_x on entry, of the new d_x on return (the outer level's
 * weighted forces with RESPA).  Energies are those of the outer level.
 * Blocks until done. */
int pinyb200_pimd_step(pinyb200_pimd *pm, pinyb200_ctx *ctx, double *d_x, double *d_v, double *d_f,
                       const double *hmat, pinyb200_pimd_energies *e, void *stream);

/* Last error text for this context (or the library if ctx is NULL). */
const char *pinyb200_last_error(pinyb200_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
