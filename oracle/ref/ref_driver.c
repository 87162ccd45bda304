/*
 * Test infrastructure only: a driver around PINY's own, unmodified CPU force
 * path.  It parses a PINY input directory exactly as PINY's main() does
 * (src/main/main.c:78-85) and then runs the four force sub-steps that
 * energy_control_pimd() runs before it transforms forces to modes
 * (src/energy/control/energy_control_pimd.c:91-111):
 *   energy_control_initial, energy_control_inter_real,
 *   energy_control_inter_recip, energy_control_intra.
 * The flags are set as PINYEmpirical does (python/piny/piny.pyx:185-188):
 * full inter and intra, no RESPA.
 *
 * Modes
 *   piny_ref dump  <dir> <input> <out.bin>           one evaluation, dump all
 *   piny_ref recip <dir> <input>                      print bead-1 PME energy
 *   piny_ref time  <dir> <input> <reps> <nbeads>      time <reps> evaluations
 *                                                     of the first <nbeads>
 *   piny_ref pimd  <typ> <in.bin> <out.bin>           PINY's ring-polymer
 *                 transforms (typ 1 staging, 2 normal modes) on given beads:
 *                 path_integral_init (transform_cnt.c:23), then
 *                 convert_pimd_mode_*, convert_pimd_pos_* on the modes, and
 *                 convert_pimd_force_* on given forces.  in.bin: int32 P,
 *                 natm, then doubles mass[natm], x[P][natm][3], f[P][natm][3].
 *   piny_ref nhc <in.bin> <out.bin>   apply_NHC_par (int_NVT.c:144) once on
 *                 given velocities and chains, weights from set_yosh
 *                 (int_utils.c:244).  in.bin: int32 natm, num_nhc, len_nhc,
 *                 nres_nhc, nyosh, inhc[3][natm] (1-based, num_nhc+1 null);
 *                 doubles dti, mass[natm], v[natm][3], mass_nhc, gkt, x_nhc,
 *                 v_nhc (each [len_nhc][num_nhc]).
 *   piny_ref io <dir> <input> <outdir> <binary 0|1>   after one evaluation,
 *                 PINY's restart dump (write_dump_file_pimd, output_pimd.c:786)
 *                 and configuration files (write_config_files_pimd, :1093)
 *                 into <outdir>, and <outdir>/state.bin with what they hold.
 *   piny_ref respa <dir> <input> <out.bin>   an input with RESPA keys
 *                 (respa_steps_lrf / _intra / _pimd, respa_rheal, res_dist,
 *                 eq_res): the four force sub-steps with the energy flags
 *                 int_NVT_pimd sets at each RESPA level (int_NVT_pimd.c:
 *                 175-189), then the full step dumped as in dump, plus per
 *                 level the raw forces (and at the full level the virial
 *                 forces fxt) and the RESPA set-up.
 *   piny_ref respa_time <dir> <input> <reps> <nbeads>   with a RESPA input:
 *                 time <reps> rounds of the four RESPA levels on the first
 *                 <nbeads> beads (one line "level L seconds" per call)
 *   piny_ref springs <in.bin> <out.bin>  mode_energy_control
 *                 (pimd_estimators.c:31) on modes u, then pimd_pvten_forc_corr
 *                 (pimd_estimators.c:223) on positions x with forces f (also
 *                 the virial forces).  in.bin: int32 P, natm, nfree_atoms
 *                 unused; doubles pi_temperature, wght, prekf[natm],
 *                 veig[P], u, x, f ([P][natm][3]), xmod[natm][3], pvten[9],
 *                 pvten_tot[9].
 *
 * The dump is a flat record file: for each record a 32-byte name, a one-byte
 * kind ('d' double, 'i' int32), 7 pad bytes, an int64 count, then the data.
 */
#include "standard_include.h"
#include "../typ_defs/typedefs_class.h"
#include "../typ_defs/typedefs_bnd.h"
#include "../typ_defs/typedefs_gen.h"
#include "../typ_defs/typedefs_cp.h"
#include "../typ_defs/typedefs_par.h"
#include "../typ_defs/typedefs_stat.h"
#include "../proto_defs/proto_parse_entry.h"
#include "../proto_defs/proto_energy_ctrl_entry.h"
#include "../proto_defs/proto_energy_ctrl_local.h"
#include "../proto_defs/proto_intra_con_entry.h"
#include "../proto_defs/proto_recip3d_entry.h"
#include <unistd.h>
#include <stdint.h>
#include <sys/time.h>

void Init_PINY(int argc, char *argv[], CLASS *class, GENERAL_DATA *general_data);

static FILE *g_out;

static void put(const char *name, char kind, const void *data, int64_t n)
{
    char hdr[40];
    memset(hdr, 0, sizeof(hdr));
    strncpy(hdr, name, 31);
    hdr[32] = kind;
    fwrite(hdr, 1, 40, g_out);
    fwrite(&n, sizeof(int64_t), 1, g_out);
    if (n > 0) fwrite(data, kind == 'd' ? 8 : kind == 'c' ? 1 : 4, (size_t)n, g_out);
}
static void putd(const char *name, const double *one_based, int64_t n) { put(name, 'd', one_based + 1, n); }
static void puti(const char *name, const int *one_based, int64_t n) { put(name, 'i', one_based + 1, n); }
static void put1d(const char *name, double v) { put(name, 'd', &v, 1); }
static void put1i(const char *name, int v) { put(name, 'i', &v, 1); }

static double now_s(void)
{
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

static CLASS class_;
static BONDED bonded_;
static GENERAL_DATA gd_;
static CP cp_;
static ANALYSIS analysis_;

static void setup(const char *dir, const char *input)
{
    if (chdir(dir) != 0) { fprintf(stderr, "piny_ref: cannot chdir to %s\n", dir); exit(2); }
    /* PINY writes its setup log to stdout; keep it out of ours. */
    fflush(stdout);
    int saved = dup(1);
    FILE *log = fopen("piny_setup.log", "w");
    if (log) dup2(fileno(log), 1);
    Init_PINY(0, NULL, &class_, &gd_);
    parse(&class_, &bonded_, &gd_, &cp_, &analysis_, (char *)input);
    fflush(stdout);
    if (log) { dup2(saved, 1); fclose(log); }
    close(saved);
    class_.energy_ctrl.iget_full_inter = 1;
    class_.energy_ctrl.iget_res_inter = 0;
    class_.energy_ctrl.iget_full_intra = 1;
    class_.energy_ctrl.iget_res_intra = 0;
}

static void evaluate(void)
{
    int ip;
    for (ip = 1; ip <= class_.clatoms_info.pi_beads_proc; ip++)
        get_ghost_pos(&class_.clatoms_info, &class_.clatoms_pos[ip], &class_.ghost_atoms);
    energy_control_initial(&class_, &bonded_, &gd_);
    energy_control_inter_real(&class_, &bonded_, &gd_);
    energy_control_inter_recip(&class_, &bonded_, &gd_);
    energy_control_intra(&class_, &bonded_, &gd_);
}

static void dump_all(const char *path)
{
    int i, ip;
    CLATOMS_INFO *ci = &class_.clatoms_info;
    int n = ci->natm_tot, P = ci->pi_beads;
    g_out = fopen(path, "wb");
    if (!g_out) { fprintf(stderr, "piny_ref: cannot open %s\n", path); exit(2); }

    put1i("natm_tot", n);
    put1i("pi_beads", P);
    put1i("nchrg", ci->nchrg);
    putd("q", ci->q, n);
    putd("mass", ci->mass, n);
    if (P > 1 && ci->xmod) {
        putd("xmod", ci->xmod, n); putd("ymod", ci->ymod, n); putd("zmod", ci->zmod, n);
    }
    CELL *cell = &gd_.cell;
    putd("hmat", cell->hmat, 9);
    putd("hmati", cell->hmati, 9);
    put1d("vol", cell->vol);
    put1i("iperd", cell->iperd);
    put1i("cubic_box_flag", cell->cubic_box_flag);
    put1i("intra_perds", cell->intra_perds);

    /* positions actually used and raw per-bead forces (M sites still loaded) */
    double *buf = (double *)malloc(sizeof(double) * (size_t)n * P * 3 + 8);
    for (ip = 1; ip <= P; ip++)
        for (i = 1; i <= n; i++) {
            size_t o = ((size_t)(ip - 1) * n + (i - 1)) * 3;
            buf[o] = class_.clatoms_pos[ip].x[i];
            buf[o + 1] = class_.clatoms_pos[ip].y[i];
            buf[o + 2] = class_.clatoms_pos[ip].z[i];
        }
    put("pos", 'd', buf, (int64_t)n * P * 3);
    for (ip = 1; ip <= P; ip++)
        for (i = 1; i <= n; i++) {
            size_t o = ((size_t)(ip - 1) * n + (i - 1)) * 3;
            buf[o] = class_.clatoms_pos[ip].fx[i];
            buf[o + 1] = class_.clatoms_pos[ip].fy[i];
            buf[o + 2] = class_.clatoms_pos[ip].fz[i];
        }
    put("force_raw", 'd', buf, (int64_t)n * P * 3);
    if (P > 1) {
        for (ip = 1; ip <= P; ip++)
            for (i = 1; i <= n; i++) {
                size_t o = ((size_t)(ip - 1) * n + (i - 1)) * 3;
                buf[o] = class_.clatoms_pos[ip].fxt[i];
                buf[o + 1] = class_.clatoms_pos[ip].fyt[i];
                buf[o + 2] = class_.clatoms_pos[ip].fzt[i];
            }
        put("forcet_raw", 'd', buf, (int64_t)n * P * 3);
    }
    /* forces after the M-site redistribution energy_control_final applies */
    for (ip = 1; ip <= P; ip++)
        distrib_ghost_force(ci, &class_.clatoms_pos[ip], &class_.ghost_atoms, 0);
    for (ip = 1; ip <= P; ip++)
        for (i = 1; i <= n; i++) {
            size_t o = ((size_t)(ip - 1) * n + (i - 1)) * 3;
            buf[o] = class_.clatoms_pos[ip].fx[i];
            buf[o + 1] = class_.clatoms_pos[ip].fy[i];
            buf[o + 2] = class_.clatoms_pos[ip].fz[i];
        }
    put("force", 'd', buf, (int64_t)n * P * 3);
    free(buf);

    STAT_AVG *sa = &gd_.stat_avg;
    put1d("vintert", sa->vintert);
    put1d("vintrat", sa->vintrat);
    put1d("vvdw", sa->vvdw);
    put1d("vcoul", sa->vcoul);
    put1d("vrecip", sa->vrecip);
    put1d("vlong", sa->vlong);
    put1d("vbondt", sa->vbondt);
    put1d("vbendt", sa->vbendt);
    putd("pvten", gd_.ptens.pvten, 9);
    putd("pvten_tot", gd_.ptens.pvten_tot, 9);

    /* interaction tables */
    ATOMMAPS *am = &class_.atommaps;
    INTERACT *it = &class_.interact;
    put1i("natm_typ", am->natm_typ);
    puti("iatm_atm_typ", am->iatm_atm_typ, n);
    int nter = am->natm_typ * (am->natm_typ + 1) / 2;
    int nuniq = 0;
    for (i = 1; i <= nter; i++) if (it->inter_map_index[i] > nuniq) nuniq = it->inter_map_index[i];
    put1i("nsplin", it->nsplin);
    put1i("ninter_unique", nuniq);
    puti("inter_map_index", it->inter_map_index, nter);
    putd("cutoff", it->cutoff, nter);
    putd("cutoff_res", it->cutoff_res, nter);
    putd("cutti", it->cutti, nter);
    putd("cutskin", it->cutskin, nter);
    putd("rmin_spl", it->rmin_spl, nuniq);
    putd("dr_spl", it->dr_spl, nuniq);
    putd("dri_spl", it->dri_spl, nuniq);
    putd("cv0", it->cv0, (int64_t)it->nsplin * nuniq);
    putd("cdv0", it->cdv0, (int64_t)it->nsplin * nuniq);
    if (ci->nchrg > 0) {
        putd("cv0_c", it->cv0_c, (int64_t)it->nsplin * nuniq);
        putd("cdv0_c", it->cdv0_c, (int64_t)it->nsplin * nuniq);
    }
    put1d("clong", it->clong);
    put1d("skin", it->skin);
    put1d("spread", it->spread);
    put1d("spread_now", it->spread_now);
    put1d("rheal_res", it->rheal_res);
    put1i("ishave_opt", it->ishave_opt);
    put1i("iswit_vdw", it->iswit_vdw);
    put1i("nlen", class_.for_scr.nlen);

    /* Verlet list as (i, j) pairs, i > j, in PINY's storage order */
    NBR_LIST *nl = &class_.nbr_list;
    put1i("iver", nl->iver);
    if (nl->iver == 1) {
        int64_t np = 0;
        for (i = 1; i <= n; i++) np += nl->verlist.nter[i];
        int *pairs = (int *)malloc(sizeof(int) * (size_t)(2 * np + 2));
        int64_t k = 0;
        for (i = 1; i <= n; i++) {
            int off = nl->verlist.jver_off[i];
            for (int j = 1; j <= nl->verlist.nter[i]; j++) {
                pairs[2 * k] = i;
                pairs[2 * k + 1] = nl->verlist.jter[off + j];
                k++;
            }
        }
        put("verlist_pairs", 'i', pairs, 2 * np);
        free(pairs);
    }

    /* exclusions */
    EXCL *ex = &bonded_.excl;
    put1i("excl_nlst", ex->nlst);
    puti("excl_num", ex->num, n);
    puti("excl_j_off", ex->j_off, n);
    puti("excl_j", ex->j, ex->nlst);

    /* Ewald / PME */
    EWALD *ew = &gd_.ewald;
    PART_MESH *pm = &class_.part_mesh;
    put1d("alp_ewd", ew->alp_ewd);
    put1d("self_erf", ew->self_erf);
    put1i("nktot", ew->nktot);
    puti("kastr", ew->kastr, ew->nktot);
    puti("kbstr", ew->kbstr, ew->nktot);
    puti("kcstr", ew->kcstr, ew->nktot);
    put1i("pme_on", pm->pme_on);
    if (pm->pme_on) {
        put1i("n_interp", pm->n_interp);
        put1i("ngrid_a", pm->ngrid_a);
        put1i("ngrid_b", pm->ngrid_b);
        put1i("ngrid_c", pm->ngrid_c);
        putd("bweight_tot", pm->bweight_tot, ew->nktot);
    }

    /* Ewald exclusion correction */
    ECOR *ec = &bonded_.ecor;
    put1i("ecor_num", ec->num);
    if (ec->num > 0) {
        puti("ecor_j1", ec->j1, ec->num);
        puti("ecor_j2", ec->j2, ec->num);
        put1i("ecor_nsplin", ec->nsplin);
        put1d("ecor_rmin_spl", ec->rmin_spl);
        put1d("ecor_rmax_spl", ec->rmax_spl);
        put1d("ecor_dr_spl", ec->dr_spl);
        put1d("ecor_dri_spl", ec->dri_spl);
        put1d("ecor_alp_ewd", ec->alp_ewd);
        put1d("ecor_ecut", ec->ecut);
        putd("ecor_cv0", ec->cv0, ec->nsplin);
        putd("ecor_cdv0", ec->cdv0, ec->nsplin);
    }

    /* bonds and bends (power series) */
    BOND *bd = &bonded_.bond;
    put1i("bond_npow", bd->npow);
    put1i("bond_ntyp_pow", bd->ntyp_pow);
    if (bd->npow > 0) {
        puti("bond_j1", bd->j1_pow, bd->npow);
        puti("bond_j2", bd->j2_pow, bd->npow);
        puti("bond_jtyp", bd->jtyp_pow, bd->npow);
        putd("bond_eq", bd->eq_pow, bd->ntyp_pow);
        putd("bond_c0", bd->c_0, bd->ntyp_pow); putd("bond_c1", bd->c_1, bd->ntyp_pow);
        putd("bond_c2", bd->c_2, bd->ntyp_pow); putd("bond_c3", bd->c_3, bd->ntyp_pow);
        putd("bond_c4", bd->c_4, bd->ntyp_pow); putd("bond_c5", bd->c_5, bd->ntyp_pow);
        putd("bond_c6", bd->c_6, bd->ntyp_pow);
        putd("bond_dc0", bd->dc_0, bd->ntyp_pow); putd("bond_dc1", bd->dc_1, bd->ntyp_pow);
        putd("bond_dc2", bd->dc_2, bd->ntyp_pow); putd("bond_dc3", bd->dc_3, bd->ntyp_pow);
        putd("bond_dc4", bd->dc_4, bd->ntyp_pow); putd("bond_dc5", bd->dc_5, bd->ntyp_pow);
        putd("bond_dc6", bd->dc_6, bd->ntyp_pow);
    }
    BEND *be = &bonded_.bend;
    put1i("bend_npow", be->npow);
    put1i("bend_ntyp_pow", be->ntyp_pow);
    if (be->npow > 0) {
        puti("bend_j1", be->j1_pow, be->npow);
        puti("bend_j2", be->j2_pow, be->npow);
        puti("bend_j3", be->j3_pow, be->npow);
        puti("bend_jtyp", be->jtyp_pow, be->npow);
        putd("bend_eq", be->eq_pow, be->ntyp_pow);
        putd("bend_c0", be->c_0, be->ntyp_pow); putd("bend_c1", be->c_1, be->ntyp_pow);
        putd("bend_c2", be->c_2, be->ntyp_pow); putd("bend_c3", be->c_3, be->ntyp_pow);
        putd("bend_c4", be->c_4, be->ntyp_pow); putd("bend_c5", be->c_5, be->ntyp_pow);
        putd("bend_c6", be->c_6, be->ntyp_pow);
        putd("bend_s0", be->s_0, be->ntyp_pow); putd("bend_s1", be->s_1, be->ntyp_pow);
        putd("bend_s2", be->s_2, be->ntyp_pow); putd("bend_s3", be->s_3, be->ntyp_pow);
        putd("bend_s4", be->s_4, be->ntyp_pow); putd("bend_s5", be->s_5, be->ntyp_pow);
        putd("bend_s6", be->s_6, be->ntyp_pow);
    }

    /* ghost (M site) definitions */
    GHOST_ATOMS *gh = &class_.ghost_atoms;
    put1i("nghost", gh->nghost_tot);
    if (gh->nghost_tot > 0) {
        puti("ighost_map", gh->ighost_map, gh->nghost_tot);
        puti("ghost_ncomp", gh->natm_comp, gh->nghost_tot);
        int nc = gh->natm_comp_max;
        put1i("ghost_ncomp_max", nc);
        for (int c = 1; c <= nc; c++) {
            char nm[32];
            snprintf(nm, sizeof nm, "ghost_iatm_%d", c);
            puti(nm, gh->iatm_comp[c], gh->nghost_tot);
            snprintf(nm, sizeof nm, "ghost_coef_%d", c);
            putd(nm, gh->coef[c], gh->nghost_tot);
        }
    }
    fclose(g_out);
}

void path_integral_init(CLATOMS_INFO *, CLATOMS_POS *, CLATOMS_TRAN *, GHOST_ATOMS *, SIMOPTS *, ATOMMAPS *,
                        COMMUNICATE *);
void convert_pimd_mode_cent(CLATOMS_INFO *, CLATOMS_POS *, CLATOMS_TRAN *);
void convert_pimd_pos_cent(CLATOMS_INFO *, CLATOMS_POS *, CLATOMS_TRAN *);
void convert_pimd_force_cent(CLATOMS_INFO *, CLATOMS_POS *, CLATOMS_TRAN *);
void convert_pimd_mode_stag(CLATOMS_INFO *, CLATOMS_POS *, CLATOMS_TRAN *);
void convert_pimd_pos_stag(CLATOMS_INFO *, CLATOMS_POS *, CLATOMS_TRAN *);
void convert_pimd_force_stag(CLATOMS_INFO *, CLATOMS_POS *, CLATOMS_TRAN *);

/* Bead-major [P][natm][3] <-> PINY's per-bead 1-based x/y/z (or fx/fy/fz). */
static void load_beads(CLATOMS_POS *cp, int P, int n, const double *a, int force)
{
    for (int b = 0; b < P; b++)
        for (int i = 0; i < n; i++) {
            double *x = force ? cp[b + 1].fx : cp[b + 1].x, *y = force ? cp[b + 1].fy : cp[b + 1].y,
                   *z = force ? cp[b + 1].fz : cp[b + 1].z;
            x[i + 1] = a[(b * n + i) * 3 + 0];
            y[i + 1] = a[(b * n + i) * 3 + 1];
            z[i + 1] = a[(b * n + i) * 3 + 2];
        }
}
static void store_beads(CLATOMS_POS *cp, int P, int n, double *a, int force)
{
    for (int b = 0; b < P; b++)
        for (int i = 0; i < n; i++) {
            const double *x = force ? cp[b + 1].fx : cp[b + 1].x, *y = force ? cp[b + 1].fy : cp[b + 1].y,
                         *z = force ? cp[b + 1].fz : cp[b + 1].z;
            a[(b * n + i) * 3 + 0] = x[i + 1];
            a[(b * n + i) * 3 + 1] = y[i + 1];
            a[(b * n + i) * 3 + 2] = z[i + 1];
        }
}

static int run_pimd(int typ, const char *inpath, const char *outpath)
{
    FILE *fi = fopen(inpath, "rb");
    int hdr[2];
    if (!fi || fread(hdr, sizeof(int), 2, fi) != 2) return 2;
    const int P = hdr[0], n = hdr[1];
    double *mass = malloc(sizeof(double) * n), *x = malloc(sizeof(double) * P * n * 3),
           *f = malloc(sizeof(double) * P * n * 3);
    if (fread(mass, sizeof(double), n, fi) != (size_t)n || fread(x, sizeof(double), (size_t)P * n * 3, fi) != (size_t)P * n * 3 ||
        fread(f, sizeof(double), (size_t)P * n * 3, fi) != (size_t)P * n * 3)
        return 2;
    fclose(fi);

    static CLATOMS_INFO info;
    static CLATOMS_TRAN tran;
    static GHOST_ATOMS ghost;
    static SIMOPTS sim;
    static ATOMMAPS maps;
    static COMMUNICATE comm;
    CLATOMS_POS *cp = calloc(P + 1, sizeof(CLATOMS_POS));
    info.pi_beads = P;
    info.pi_beads_proc = P;
    info.pi_beads_proc_st = 1;
    info.natm_tot = n;
    info.myatm_start = 1;
    info.myatm_end = n;
    info.gamma_adb = 1.0;
    info.pi_temperature = 300.0;
    info.mass = calloc(n + 1, sizeof(double));
    info.prekf = calloc(n + 1, sizeof(double));
    for (int i = 0; i < n; i++) info.mass[i + 1] = mass[i];
    for (int b = 1; b <= P; b++) {
        cp[b].mass = calloc(n + 1, sizeof(double));
        cp[b].x = calloc(n + 1, sizeof(double));
        cp[b].y = calloc(n + 1, sizeof(double));
        cp[b].z = calloc(n + 1, sizeof(double));
        cp[b].fx = calloc(n + 1, sizeof(double));
        cp[b].fy = calloc(n + 1, sizeof(double));
        cp[b].fz = calloc(n + 1, sizeof(double));
    }
    sim.pi_md_typ = typ;
    comm.np_beads = 1;
    path_integral_init(&info, cp, &tran, &ghost, &sim, &maps, &comm);

    g_out = fopen(outpath, "wb");
    if (!g_out) return 2;
    double *buf = malloc(sizeof(double) * P * n * 3);
    load_beads(cp, P, n, x, 0);
    if (typ == 2) convert_pimd_mode_cent(&info, cp, &tran);
    else convert_pimd_mode_stag(&info, cp, &tran);
    store_beads(cp, P, n, buf, 0);
    put("modes", 'd', buf, (int64_t)P * n * 3);
    if (typ == 2) convert_pimd_pos_cent(&info, cp, &tran);
    else convert_pimd_pos_stag(&info, cp, &tran);
    store_beads(cp, P, n, buf, 0);
    put("back", 'd', buf, (int64_t)P * n * 3);
    load_beads(cp, P, n, f, 1);
    if (typ == 2) convert_pimd_force_cent(&info, cp, &tran);
    else convert_pimd_force_stag(&info, cp, &tran);
    store_beads(cp, P, n, buf, 1);
    put("fmodes", 'd', buf, (int64_t)P * n * 3);
    putd("path_eig", tran.path_eig, P);
    for (int b = 0; b < P; b++)
        for (int i = 0; i < n; i++) buf[b * n + i] = cp[b + 1].mass[i + 1];
    put("bead_mass", 'd', buf, (int64_t)P * n);
    putd("prekf", info.prekf, n);
    if (typ == 1) {
        putd("rat1", tran.rat1_stag + 1, P - 1);
        putd("rat2", tran.rat2_stag + 1, P - 1);
    }
    fclose(g_out);
    return 0;
}

void apply_NHC_par(CLATOMS_INFO *, CLATOMS_POS *, THERM_INFO *, THERM_POS *, INT_SCR *, int, CLASS_COMM_FORC_PKG *);
void set_yosh(int, double, double *, double *, double *, double *, double *);
void mode_energy_control(CLASS *, GENERAL_DATA *);
void pimd_pvten_forc_corr(CLASS *, GENERAL_DATA *, double *);

static int read_all(FILE *f, void *p, size_t sz, size_t n) { return fread(p, sz, n, f) == n; }

/* 1-based [len][num] table from a 0-based row-major block */
static double **chain_table(int len, int num, const double *src)
{
    double **t = calloc(len + 1, sizeof(double *));
    for (int c = 1; c <= len; c++) {
        t[c] = calloc(num + 2, sizeof(double));
        if (src)
            for (int k = 1; k <= num; k++) t[c][k] = src[(size_t)(c - 1) * num + (k - 1)];
    }
    return t;
}
static void chain_dump(const char *name, double **t, int len, int num)
{
    double *buf = malloc(sizeof(double) * len * num);
    for (int c = 1; c <= len; c++)
        for (int k = 1; k <= num; k++) buf[(size_t)(c - 1) * num + (k - 1)] = t[c][k];
    put(name, 'd', buf, (int64_t)len * num);
    free(buf);
}

static int run_nhc(const char *inpath, const char *outpath)
{
    FILE *fi = fopen(inpath, "rb");
    int h[5];
    if (!fi || !read_all(fi, h, sizeof(int), 5)) return 2;
    const int n = h[0], num = h[1], len = h[2];
    int *inhc = malloc(sizeof(int) * 3 * n);
    double dti;
    double *m = malloc(sizeof(double) * n), *v = malloc(sizeof(double) * 3 * n);
    double *blk[4];
    if (!read_all(fi, inhc, sizeof(int), 3 * (size_t)n) || !read_all(fi, &dti, sizeof(double), 1) ||
        !read_all(fi, m, sizeof(double), n) || !read_all(fi, v, sizeof(double), 3 * (size_t)n))
        return 2;
    for (int k = 0; k < 4; k++) {
        blk[k] = malloc(sizeof(double) * len * num);
        if (!read_all(fi, blk[k], sizeof(double), (size_t)len * num)) return 2;
    }
    fclose(fi);

    static CLATOMS_INFO info;
    static CLATOMS_POS pos;
    static THERM_INFO ti;
    static THERM_POS tp;
    static INT_SCR scr;
    static CLASS_COMM_FORC_PKG pkg;
    info.natm_tot = n;
    info.myatm_start = 1;
    info.myatm_end = n;
    info.mass = calloc(n + 1, sizeof(double));
    pos.mass = calloc(n + 1, sizeof(double));
    pos.vx = calloc(n + 1, sizeof(double));
    pos.vy = calloc(n + 1, sizeof(double));
    pos.vz = calloc(n + 1, sizeof(double));
    for (int i = 0; i < n; i++) {
        info.mass[i + 1] = pos.mass[i + 1] = m[i];
        pos.vx[i + 1] = v[3 * i];
        pos.vy[i + 1] = v[3 * i + 1];
        pos.vz[i + 1] = v[3 * i + 2];
    }
    ti.num_nhc = num;
    ti.len_nhc = len;
    ti.nres_nhc = h[3];
    ti.nyosh_nhc = h[4];
    ti.mytherm_start = 1;
    ti.mytherm_end = num;
    ti.inhc_x = calloc(n + 1, sizeof(int));
    ti.inhc_y = calloc(n + 1, sizeof(int));
    ti.inhc_z = calloc(n + 1, sizeof(int));
    for (int i = 0; i < n; i++) {
        ti.inhc_x[i + 1] = inhc[i];
        ti.inhc_y[i + 1] = inhc[n + i];
        ti.inhc_z[i + 1] = inhc[2 * n + i];
    }
    ti.wdti = calloc(10, sizeof(double));
    ti.wdti2 = calloc(10, sizeof(double));
    ti.wdti4 = calloc(10, sizeof(double));
    ti.wdti8 = calloc(10, sizeof(double));
    ti.wdti16 = calloc(10, sizeof(double));
    set_yosh(ti.nyosh_nhc, dti, ti.wdti, ti.wdti2, ti.wdti4, ti.wdti8, ti.wdti16);
    ti.mass_nhc = chain_table(len, num, blk[0]);
    ti.gkt = chain_table(len, num, blk[1]);
    tp.x_nhc = chain_table(len, num, blk[2]);
    tp.v_nhc = chain_table(len, num, blk[3]);
    tp.f_nhc = chain_table(len, num, NULL);
    scr.atm_kin = calloc(num + 2, sizeof(double));
    scr.sc = calloc(num + 2, sizeof(double));
    scr.sc_temp = calloc(num + 2, sizeof(double));
    pkg.num_proc = 1;
    apply_NHC_par(&info, &pos, &ti, &tp, &scr, 2, &pkg);

    g_out = fopen(outpath, "wb");
    if (!g_out) return 2;
    for (int i = 0; i < n; i++) {
        v[3 * i] = pos.vx[i + 1];
        v[3 * i + 1] = pos.vy[i + 1];
        v[3 * i + 2] = pos.vz[i + 1];
    }
    put("v", 'd', v, 3 * (int64_t)n);
    chain_dump("x_nhc", tp.x_nhc, len, num);
    chain_dump("v_nhc", tp.v_nhc, len, num);
    putd("wdti", ti.wdti, ti.nyosh_nhc);
    fclose(g_out);
    return 0;
}

static int run_springs(const char *inpath, const char *outpath)
{
    FILE *fi = fopen(inpath, "rb");
    int h[3];
    double sc2[2];
    if (!fi || !read_all(fi, h, sizeof(int), 3) || !read_all(fi, sc2, sizeof(double), 2)) return 2;
    const int P = h[0], n = h[1];
    const size_t nb = (size_t)P * n * 3;
    double *prekf = malloc(sizeof(double) * n), *veig = malloc(sizeof(double) * P);
    double *u = malloc(sizeof(double) * nb), *x = malloc(sizeof(double) * nb), *f = malloc(sizeof(double) * nb);
    double *xm = malloc(sizeof(double) * 3 * n), pv[9], pvt[9];
    if (!read_all(fi, prekf, sizeof(double), n) || !read_all(fi, veig, sizeof(double), P) ||
        !read_all(fi, u, sizeof(double), nb) || !read_all(fi, x, sizeof(double), nb) ||
        !read_all(fi, f, sizeof(double), nb) || !read_all(fi, xm, sizeof(double), 3 * (size_t)n) ||
        !read_all(fi, pv, sizeof(double), 9) || !read_all(fi, pvt, sizeof(double), 9))
        return 2;
    fclose(fi);

    static CLASS cl;
    static GENERAL_DATA gd;
    CLATOMS_POS *cp = calloc(P + 1, sizeof(CLATOMS_POS));
    cl.clatoms_pos = cp;
    cl.clatoms_info.pi_beads = P;
    cl.clatoms_info.pi_beads_proc = P;
    cl.clatoms_info.pi_beads_proc_st = 1;
    cl.clatoms_info.natm_tot = n;
    cl.clatoms_info.myatm_start = 1;
    cl.clatoms_info.myatm_end = n;
    cl.clatoms_info.pi_temperature = sc2[0];
    cl.clatoms_info.wght_pimd = sc2[1];
    cl.clatoms_info.prekf = calloc(n + 1, sizeof(double));
    cl.clatoms_info.xmod = calloc(n + 1, sizeof(double));
    cl.clatoms_info.ymod = calloc(n + 1, sizeof(double));
    cl.clatoms_info.zmod = calloc(n + 1, sizeof(double));
    for (int i = 0; i < n; i++) {
        cl.clatoms_info.prekf[i + 1] = prekf[i];
        cl.clatoms_info.xmod[i + 1] = xm[3 * i];
        cl.clatoms_info.ymod[i + 1] = xm[3 * i + 1];
        cl.clatoms_info.zmod[i + 1] = xm[3 * i + 2];
    }
    cl.clatoms_tran.path_eig = calloc(P + 1, sizeof(double));
    for (int b = 0; b < P; b++) cl.clatoms_tran.path_eig[b + 1] = veig[b];
    cl.communicate.np_forc = 1;
    cl.energy_ctrl.iget_full_inter = 1;
    cl.energy_ctrl.iget_full_intra = 1;
    cl.ewd_scr.x = calloc(n + 1, sizeof(double));
    cl.ewd_scr.y = calloc(n + 1, sizeof(double));
    cl.ewd_scr.z = calloc(n + 1, sizeof(double));
    for (int b = 1; b <= P; b++) {
        cp[b].x = calloc(n + 1, sizeof(double));
        cp[b].y = calloc(n + 1, sizeof(double));
        cp[b].z = calloc(n + 1, sizeof(double));
        cp[b].fx = calloc(n + 1, sizeof(double));
        cp[b].fy = calloc(n + 1, sizeof(double));
        cp[b].fz = calloc(n + 1, sizeof(double));
        cp[b].fxt = cp[b].fx;
        cp[b].fyt = cp[b].fy;
        cp[b].fzt = cp[b].fz;
        cp[b].fxm = calloc(n + 1, sizeof(double));
        cp[b].fym = calloc(n + 1, sizeof(double));
        cp[b].fzm = calloc(n + 1, sizeof(double));
    }
    gd.ptens.pvten = calloc(10, sizeof(double));
    gd.ptens.pvten_tot = calloc(10, sizeof(double));
    gd.ptens.pvten_mode = calloc(10, sizeof(double));
    gd.ptens.pvten_mode_tot = calloc(10, sizeof(double));
    for (int k = 0; k < 9; k++) {
        gd.ptens.pvten[k + 1] = pv[k];
        gd.ptens.pvten_tot[k + 1] = pvt[k];
    }
    load_beads(cp, P, n, u, 0);
    mode_energy_control(&cl, &gd);
    load_beads(cp, P, n, x, 0);
    load_beads(cp, P, n, f, 1);
    double akvirx = 0.0;
    pimd_pvten_forc_corr(&cl, &gd, &akvirx);

    g_out = fopen(outpath, "wb");
    if (!g_out) return 2;
    double *buf = malloc(sizeof(double) * nb);
    for (int b = 0; b < P; b++)
        for (int i = 0; i < n; i++) {
            buf[((size_t)b * n + i) * 3 + 0] = cp[b + 1].fxm[i + 1];
            buf[((size_t)b * n + i) * 3 + 1] = cp[b + 1].fym[i + 1];
            buf[((size_t)b * n + i) * 3 + 2] = cp[b + 1].fzm[i + 1];
        }
    put("fm", 'd', buf, (int64_t)nb);
    put1d("kin_harm", gd.stat_avg.kin_harm);
    putd("pvten_mode_tot", gd.ptens.pvten_mode_tot, 9);
    putd("pvten", gd.ptens.pvten, 9);
    putd("pvten_tot", gd.ptens.pvten_tot, 9);
    put1d("akvirx", akvirx);
    fclose(g_out);
    return 0;
}

void write_dump_file_pimd(CLASS *, BONDED *, GENERAL_DATA *);
void write_config_files_pimd(CLASS *, BONDED *, GENERAL_DATA *);

/* absolute path of an output file that may not exist yet (setup chdirs) */
static char *resolve_out(const char *arg)
{
    char *outpath = realpath(arg, NULL);
    if (!outpath) {
        char *tmp = strdup(arg);
        char *slash = strrchr(tmp, '/');
        char *d = slash ? (*slash = 0, realpath(tmp[0] ? tmp : "/", NULL)) : realpath(".", NULL);
        const char *base = slash ? slash + 1 : arg;
        outpath = malloc(strlen(d) + strlen(base) + 2);
        sprintf(outpath, "%s/%s", d, base);
    }
    return outpath;
}

/* RESPA levels as int_NVT_pimd sets the flags (int_NVT_pimd.c:175-189):
 * iget_full_inter, iget_res_inter, iget_full_intra, iget_res_intra. */
static const int k_levels[4][4] = {{1, -1, 1, 1}, {0, 1, 1, 1}, {0, 0, 1, 1}, {0, 0, 0, 1}};

static void set_level(int l)
{
    class_.energy_ctrl.iget_full_inter = k_levels[l][0];
    class_.energy_ctrl.iget_res_inter = k_levels[l][1] < 0 ? gd_.timeinfo.int_res_ter : k_levels[l][1];
    class_.energy_ctrl.iget_full_intra = k_levels[l][2];
    class_.energy_ctrl.iget_res_intra = k_levels[l][3];
}

static void gather_forces(double *buf, int t)
{
    CLATOMS_INFO *ci = &class_.clatoms_info;
    int n = ci->natm_tot, P = ci->pi_beads;
    for (int ip = 1; ip <= P; ip++)
        for (int i = 1; i <= n; i++) {
            size_t o = ((size_t)(ip - 1) * n + (i - 1)) * 3;
            CLATOMS_POS *cp = &class_.clatoms_pos[ip];
            buf[o] = t ? cp->fxt[i] : cp->fx[i];
            buf[o + 1] = t ? cp->fyt[i] : cp->fy[i];
            buf[o + 2] = t ? cp->fzt[i] : cp->fz[i];
        }
}

static int run_respa_time(const char *dir, const char *input, int reps, int nb)
{
    setup(dir, input);
    CLATOMS_INFO *ci = &class_.clatoms_info;
    if (nb < 1 || nb > ci->pi_beads) nb = ci->pi_beads;
    ci->pi_beads_proc = nb;
    for (int l = 0; l < 4; l++) { /* warm-up */
        set_level(l);
        evaluate();
    }
    for (int r = 0; r < reps; r++)
        for (int l = 0; l < 4; l++) {
            set_level(l);
            double t0 = now_s();
            evaluate();
            printf("level %d %.6f s\n", l, now_s() - t0);
            fflush(stdout);
        }
    return 0;
}

static int run_respa(const char *dir, const char *input, const char *outpath)
{
    setup(dir, input);
    CLATOMS_INFO *ci = &class_.clatoms_info;
    const size_t nb = (size_t)ci->natm_tot * ci->pi_beads * 3;
    double *f[4], *ft = (double *)malloc(sizeof(double) * nb + 8);
    double e[4][2];
    for (int l = 0; l < 4; l++) {
        f[l] = (double *)malloc(sizeof(double) * nb + 8);
        set_level(l);
        evaluate();
        gather_forces(f[l], 0);
        if (l == 0 && ci->pi_beads > 1) gather_forces(ft, 1);
        e[l][0] = gd_.stat_avg.vintert;
        e[l][1] = gd_.stat_avg.vintrat;
    }
    set_level(0);
    evaluate();
    dump_all(outpath);
    g_out = fopen(outpath, "ab");
    if (!g_out) return 2;
    TIMEINFO *ti = &gd_.timeinfo;
    put1i("nres_ter", ti->nres_ter);
    put1i("nres_tor", ti->nres_tor);
    put1i("nres_tra", ti->nres_tra);
    put1i("nres_pimd", ti->nres_pimd);
    put1i("int_res_ter", ti->int_res_ter);
    put1i("int_res_tra", ti->int_res_tra);
    put1d("wght_ter", class_.for_scr.wght_ter);
    put1d("wght_ter_res", class_.for_scr.wght_ter_res);
    put1d("wght_tra", class_.for_scr.wght_tra);
    put1d("wght_tra_res", class_.for_scr.wght_tra_res);
    if (bonded_.bond.npow > 0) putd("bond_eq_res", bonded_.bond.eq_pow_res, bonded_.bond.ntyp_pow);
    put1i("nktot_res", gd_.ewald.nktot_res);
    put1i("pme_res_on", class_.part_mesh.pme_res_on);
    if (class_.part_mesh.pme_res_on && gd_.ewald.nktot_res > 0) {
        /* the separate RESPA PME grid: its mesh, order, k sphere and weights */
        const PART_MESH *pm = &class_.part_mesh;
        const int g3[3] = {pm->ngrid_a_res, pm->ngrid_b_res, pm->ngrid_c_res};
        put("ngrid_res", 'i', g3, 3);
        put1i("n_interp_res", pm->n_interp_res);
        put1i("kmax_pme_res", pm->kmax_pme_res);
        puti("kastr_res", gd_.ewald.kastr_res, gd_.ewald.nktot_res);
        puti("kbstr_res", gd_.ewald.kbstr_res, gd_.ewald.nktot_res);
        puti("kcstr_res", gd_.ewald.kcstr_res, gd_.ewald.nktot_res);
        putd("bweight_tot_res", pm->bweight_tot_res, gd_.ewald.nktot_res);
    }
    if (bonded_.ecor.num > 0 && bonded_.ecor.nktot_res > 0) {
        putd("ecor_cdv0_res", bonded_.ecor.cdv0_res, bonded_.ecor.nsplin);
        put1d("ecor_ecut_res", bonded_.ecor.ecut_res);
    }
    for (int l = 0; l < 4; l++) {
        char nm[32];
        snprintf(nm, sizeof nm, "L%d_force_raw", l);
        put(nm, 'd', f[l], (int64_t)nb);
        snprintf(nm, sizeof nm, "L%d_flags", l);
        int fl[4];
        set_level(l);
        fl[0] = class_.energy_ctrl.iget_full_inter;
        fl[1] = class_.energy_ctrl.iget_res_inter;
        fl[2] = class_.energy_ctrl.iget_full_intra;
        fl[3] = class_.energy_ctrl.iget_res_intra;
        put(nm, 'i', fl, 4);
        snprintf(nm, sizeof nm, "L%d_energies", l);
        put(nm, 'd', e[l], 2);
        free(f[l]);
    }
    if (ci->pi_beads > 1) put("L0_forcet_raw", 'd', ft, (int64_t)nb);
    free(ft);
    fclose(g_out);
    return 0;
}

static char *path_in(const char *dir, const char *name)
{
    char *p = malloc(strlen(dir) + strlen(name) + 2);
    sprintf(p, "%s/%s", dir, name);
    return p;
}

static int run_io(const char *dir, const char *input, const char *outdir_rel, int binary)
{
    char *outdir = realpath(outdir_rel, NULL);
    if (!outdir) return 2;
    setup(dir, input);
    evaluate();
    CLASS *cl = &class_;
    GENERAL_DATA *g = &gd_;
    const int P = cl->clatoms_info.pi_beads, n = cl->clatoms_info.natm_tot;
    g->filenames.dname = path_in(outdir, "dump");
    g->filenames.cpname = path_in(outdir, "conf_pos");
    g->filenames.cvname = path_in(outdir, "conf_vel");
    g->filenames.centname = path_in(outdir, "conf_cent");
    g->filenames.forcename = path_in(outdir, "conf_force");
    g->filenames.cpparname = path_in(outdir, "conf_par");
    g->filenames.iwrite_confp = g->filenames.iwrite_confv = g->filenames.iwrite_path_cent = 1;
    g->filenames.iwrite_atm_for = g->filenames.iwrite_par_confp = 1;
    g->filenames.low_lim_par = 2;
    g->filenames.high_lim_par = n < 6 ? n : 6;
    g->filenames.iwrite_conf_binary = binary;
    g->timeinfo.itime = 0;
    write_dump_file_pimd(cl, &bonded_, g);
    write_config_files_pimd(cl, &bonded_, g);

    g_out = fopen(path_in(outdir, "state.bin"), "wb");
    if (!g_out) return 2;
    double *buf = malloc(sizeof(double) * 3 * (size_t)n * P);
    const char *what[3] = {"pos", "vel", "fxt"};
    for (int w = 0; w < 3; w++) {
        for (int b = 0; b < P; b++)
            for (int i = 0; i < n; i++) {
                CLATOMS_POS *cp = &cl->clatoms_pos[b + 1];
                const double *x = w == 0 ? cp->x : w == 1 ? cp->vx : cp->fxt, *y = w == 0 ? cp->y : w == 1 ? cp->vy : cp->fyt,
                             *z = w == 0 ? cp->z : w == 1 ? cp->vz : cp->fzt;
                buf[((size_t)b * n + i) * 3 + 0] = x[i + 1];
                buf[((size_t)b * n + i) * 3 + 1] = y[i + 1];
                buf[((size_t)b * n + i) * 3 + 2] = z[i + 1];
            }
        put(what[w], 'd', buf, 3 * (int64_t)n * P);
    }
    putd("hmat", g->cell.hmat, 9);
    putd("hmat_ewd", g->cell.hmat_ewd, 9);
    putd("vgmat", g->par_rahman.vgmat, 9);
    put1d("x_lnv", g->baro.x_lnv);
    put1d("v_lnv", g->baro.v_lnv);
    put1d("dt", g->timeinfo.dt);
    put1d("t_ext", g->statepoint.t_ext);
    put1d("pext", g->statepoint.pext);
    put1d("stens_ext", g->statepoint.stens_ext);
    put1i("nfree", cl->clatoms_info.nfree);
    int ens[5] = {g->ensopts.nve, g->ensopts.nvt, g->ensopts.npt_i, g->ensopts.npt_f, g->ensopts.nst};
    put("ens", 'i', ens, 5);
    int fr[3] = {bonded_.bond_free.num, bonded_.bend_free.num, bonded_.tors_free.num};
    put("free", 'i', fr, 3);
    const int cn = cl->therm_info_class.num_nhc, cl_len = cl->therm_info_class.len_nhc;
    const int bn = cl->therm_info_bead.num_nhc, bl = cl->therm_info_bead.len_nhc;
    int nh[4] = {cn, cl_len, bn, bl};
    put("nhc_dims", 'i', nh, 4);
    double *v = malloc(sizeof(double) * ((size_t)cn * cl_len + (size_t)bn * bl * P + cl_len + 1));
    size_t k = 0;
    for (int j = 1; j <= cl_len; j++)
        for (int i = 1; i <= cn; i++) v[k++] = cl->therm_class.v_nhc[j][i];
    put("class_v_nhc", 'd', v, (int64_t)k);
    k = 0;
    for (int b = 2; b <= P; b++)
        for (int j = 1; j <= bl; j++)
            for (int i = 1; i <= bn; i++) v[k++] = cl->therm_bead[b].v_nhc[j][i];
    put("bead_v_nhc", 'd', v, (int64_t)k);
    putd("v_vol_nhc", g->baro.v_vol_nhc, cl_len);
    /* names: atom, residue, molecule type of each atom, then molecule numbers */
    char *names = malloc((size_t)n * 3 * 64 + 1);
    size_t off = 0;
    for (int i = 1; i <= n; i++)
        off += sprintf(names + off, "%s %s %s\n", cl->atommaps.atm_typ[cl->atommaps.iatm_atm_typ[i]],
                       cl->atommaps.res_typ[cl->atommaps.iatm_res_typ[i]],
                       cl->atommaps.mol_typ[cl->atommaps.iatm_mol_typ[i]]);
    put("names", 'c', names, (int64_t)off);
    puti("mol_num", cl->atommaps.iatm_mol_num, n);
    fclose(g_out);
    return 0;
}

#ifdef PINY_WITH_GPU
/* piny_ref_gpu gpu_dump <dir> <input> <out.bin> <mixed 0|1>: the same
 * evaluation as dump with the three force sub-steps replaced by the
 * libpinyb200 binding (energy_control_gpu.c), run twice -- a first call that
 * builds the device list, then PINY's own list test and a second evaluation
 * of the same positions -- and dumped after the second, with the device
 * list as gpu_pairs. */
#include "pinyb200.h"
int gpu_force_init(CLASS *, BONDED *, GENERAL_DATA *, int, pinyb200_ctx **);
int gpu_energy_control(pinyb200_ctx *, CLASS *, BONDED *, GENERAL_DATA *, int);

static int run_gpu_dump(const char *dir, const char *input, const char *outpath, int mixed)
{
    setup(dir, input);
    pinyb200_ctx *ctx = NULL;
    int rc = gpu_force_init(&class_, &bonded_, &gd_, mixed, &ctx);
    if (rc) {
        fprintf(stderr, "@@@ gpu_force_init: %s\n", pinyb200_last_error(ctx));
        return 3;
    }
    double updates0 = 0.0;
    for (int call = 0; call < 2; call++) {
        int ip;
        for (ip = 1; ip <= class_.clatoms_info.pi_beads_proc; ip++)
            get_ghost_pos(&class_.clatoms_info, &class_.clatoms_pos[ip], &class_.ghost_atoms);
        energy_control_initial(&class_, &bonded_, &gd_);
        if (call == 1) updates0 = gd_.stat_avg.updates;
        rc = gpu_energy_control(ctx, &class_, &bonded_, &gd_, call == 0);
        if (rc) {
            fprintf(stderr, "@@@ gpu_energy_control: %s\n", pinyb200_last_error(ctx));
            return 3;
        }
    }
    dump_all(outpath);
    /* device list (i > j, 1-based like verlist_pairs) and the second call's rebuilds */
    long np = 0, na = 0, cap = 0;
    pinyb200_list_info(ctx, &np, &na, &cap);
    int *pi = (int *)malloc(sizeof(int) * (size_t)(np + 1)), *pj = (int *)malloc(sizeof(int) * (size_t)(np + 1));
    long got = 0;
    pinyb200_get_list(ctx, pi, pj, np, &got);
    int *pairs = (int *)malloc(sizeof(int) * (size_t)(2 * got + 2));
    for (long k = 0; k < got; k++) {
        pairs[2 * k] = pi[k] + 1;
        pairs[2 * k + 1] = pj[k] + 1;
    }
    g_out = fopen(outpath, "ab");
    put("gpu_pairs", 'i', pairs, 2 * got);
    put1d("gpu_rebuilds_second_call", gd_.stat_avg.updates - updates0);
    fclose(g_out);
    free(pi);
    free(pj);
    free(pairs);
    pinyb200_destroy(ctx);
    return 0;
}
#endif

int main(int argc, char **argv)
{
#ifdef PINY_WITH_GPU
    if (argc == 6 && strcmp(argv[1], "gpu_dump") == 0)
        return run_gpu_dump(argv[2], argv[3], resolve_out(argv[4]), atoi(argv[5]));
#endif
    if (argc == 6 && strcmp(argv[1], "io") == 0) return run_io(argv[2], argv[3], argv[4], atoi(argv[5]));
    if (argc == 6 && strcmp(argv[1], "respa_time") == 0)
        return run_respa_time(argv[2], argv[3], atoi(argv[4]), atoi(argv[5]));
    if (argc == 5 && strcmp(argv[1], "respa") == 0) return run_respa(argv[2], argv[3], resolve_out(argv[4]));
    if (argc == 4 && strcmp(argv[1], "nhc") == 0) return run_nhc(argv[2], argv[3]);
    if (argc == 4 && strcmp(argv[1], "springs") == 0) return run_springs(argv[2], argv[3]);
    if (argc == 5 && strcmp(argv[1], "pimd") == 0) return run_pimd(atoi(argv[2]), argv[3], argv[4]);
    if (argc < 4) {
        fprintf(stderr, "usage: piny_ref dump|recip|time <dir> <input> [...]\n");
        return 2;
    }
    const char *mode = argv[1];
    char *outpath = NULL;
    if (strcmp(mode, "dump") == 0) {
        if (argc < 5) return 2;
        outpath = resolve_out(argv[4]);
    }
    setup(argv[2], argv[3]);

    if (strcmp(mode, "dump") == 0) {
        evaluate();
        dump_all(outpath);
        return 0;
    }
    if (strcmp(mode, "recip") == 0) {
        double vrecip = 0.0;
        int ip;
        for (ip = 1; ip <= class_.clatoms_info.pi_beads_proc; ip++)
            get_ghost_pos(&class_.clatoms_info, &class_.clatoms_pos[ip], &class_.ghost_atoms);
        class_.energy_ctrl.iget_pv_real_inter = 1;
        class_.energy_ctrl.iget_pe_real_inter = 1;
        ewald3d_recip_pme(&class_.clatoms_info, &class_.clatoms_pos[1], &gd_.cell, &gd_.ptens,
                          gd_.ewald.alp_ewd, gd_.ewald.nktot, gd_.ewald.kastr, gd_.ewald.kbstr,
                          gd_.ewald.kcstr, &class_.ewd_scr, &vrecip, class_.for_scr.wght_ter_res, 0,
                          &class_.part_mesh, 0, &class_.class_comm_forc_pkg,
                          class_.energy_ctrl.iget_pv_real_inter, &gd_.pme_fft_pkg, &class_.for_scr,
                          gd_.ewald.clus_corr_r, gd_.ewald.dclus_corr_r);
        printf("recip %.13g grid %d %d %d order %d alp %.10g\n", vrecip, class_.part_mesh.ngrid_a,
               class_.part_mesh.ngrid_b, class_.part_mesh.ngrid_c, class_.part_mesh.n_interp,
               gd_.ewald.alp_ewd / BOHR);
        return 0;
    }
    if (strcmp(mode, "time") == 0) {
        int reps = argc > 4 ? atoi(argv[4]) : 1;
        int nb = argc > 5 ? atoi(argv[5]) : class_.clatoms_info.pi_beads;
        if (nb < 1 || nb > class_.clatoms_info.pi_beads) nb = class_.clatoms_info.pi_beads;
        class_.clatoms_info.pi_beads_proc = nb;
        evaluate(); /* warm-up */
        for (int r = 0; r < reps; r++) {
            double t0 = now_s();
            evaluate();
            double t1 = now_s();
            printf("time %d beads %.6f s\n", nb, t1 - t0);
            fflush(stdout);
        }
        return 0;
    }
    fprintf(stderr, "piny_ref: unknown mode %s\n", mode);
    return 2;
}
