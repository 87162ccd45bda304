// C ABI of the pinyb200 library: context set-up, list build and the force
// evaluation that replaces PINY's energy_control_inter_real /
// energy_control_inter_recip / energy_control_intra for all beads.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

using namespace pinyb200;

namespace {

thread_local std::string g_lib_err;

int fail(pinyb200_ctx *c, int code, const std::string &msg)
{
    if (c) c->err = msg;
    else g_lib_err = msg;
    return code;
}

#define CK(call)                                                                               \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(c, PINYB200_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
cudaError_t upload(T **dst, const T *src, size_t n)
{
    *dst = nullptr;
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc((void **)dst, n * sizeof(T));
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice);
}

// Cell inverse with the operation order of gethinv (src/mathlib/mathlib.c:353).
Cell make_cell(const double *hm)
{
    Cell c;
    const double *h = hm - 1;
    double vol = (h[1] * (h[5] * h[9] - h[8] * h[6]) + h[4] * (h[8] * h[3] - h[2] * h[9]) +
                  h[7] * (h[2] * h[6] - h[5] * h[3]));
    c.hi[0] = (h[5] * h[9] - h[8] * h[6]) / vol;
    c.hi[4] = (h[1] * h[9] - h[7] * h[3]) / vol;
    c.hi[8] = (h[1] * h[5] - h[4] * h[2]) / vol;
    c.hi[3] = (h[7] * h[6] - h[4] * h[9]) / vol;
    c.hi[1] = (h[3] * h[8] - h[2] * h[9]) / vol;
    c.hi[6] = (h[4] * h[8] - h[7] * h[5]) / vol;
    c.hi[2] = (h[2] * h[6] - h[3] * h[5]) / vol;
    c.hi[7] = (h[7] * h[2] - h[8] * h[1]) / vol;
    c.hi[5] = (h[3] * h[4] - h[6] * h[1]) / vol;
    for (int i = 0; i < 9; i++) c.h[i] = hm[i];
    c.vol = vol;
    // cubic_box_flag: PINY sets it for an orthorhombic cell with equal edges
    c.cubic = (hm[1] == 0.0 && hm[2] == 0.0 && hm[3] == 0.0 && hm[5] == 0.0 && hm[6] == 0.0 && hm[7] == 0.0 &&
               hm[0] == hm[4] && hm[0] == hm[8]);
    return c;
}

// Interval coefficients of npol_vspl_fetch (force_npol.c:339-375) for knot
// k (1-based) of a table: c0 + del (c1 + del (c2 + del c3)).
void cubic_coefs(const double *t, int nsplin, std::vector<double> &out)
{
    // host code is built with -ffp-contract=off: these are PINY's roundings
    const double oneth = (1.0 / 3.0), onesi = (1.0 / 6.0);
    out.assign((size_t)4 * nsplin, 0.0);
    for (int k = 3; k <= nsplin - 1; k++) {
        const double c0 = t[k - 1], fp1 = t[k], fm1 = t[k - 2], fm2 = t[k - 3];
        out[4 * (size_t)(k - 1) + 0] = c0;
        out[4 * (size_t)(k - 1) + 1] = oneth * fp1 + 0.5 * c0 - fm1 + onesi * fm2;
        out[4 * (size_t)(k - 1) + 2] = 0.5 * fp1 - c0 + 0.5 * fm1;
        out[4 * (size_t)(k - 1) + 3] = onesi * fp1 - 0.5 * c0 + 0.5 * fm1 - onesi * fm2;
    }
}

void free_sys(DeviceSystem &s)
{
    void *ptrs[] = {s.atm_typ, s.charge, s.inter_map, s.cutoff, s.rmin, s.dr, s.dri, s.has_vdw, s.tab64, s.tab32,
                    s.excl_off, s.excl_j, s.ichrg, s.kvec, s.bweight, s.kmask, s.ecor_j1, s.ecor_j2, s.ecor_tab,
                    s.bond_j, s.bond_eq, s.bond_c, s.bond_dc, s.bend_j, s.bend_c, s.bend_s, s.bend_dc, s.bend_ds,
                    s.ghost_atom, s.ghost_comp, s.ghost_coef};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    s = DeviceSystem();
}

int check_system(pinyb200_ctx *c, const pinyb200_system *s, int nbeads)
{
    if (!s || s->natm <= 0 || s->ntyp <= 0 || !s->atm_typ || !s->charge)
        return fail(c, PINYB200_ERR_ARG, "system: natm/ntyp/atm_typ/charge required");
    if (nbeads != 1 && nbeads != 2 && nbeads != 4 && nbeads != 8 && nbeads != 16 && nbeads != 32 && nbeads != 64)
        return fail(c, PINYB200_ERR_UNSUPPORTED, "nbeads must be one of 1,2,4,8,16,32,64");
    if (s->nsplin < 8 || s->ninter_unique <= 0) return fail(c, PINYB200_ERR_ARG, "system: spline tables missing");
    for (int i = 0; i < s->natm; i++)
        if (s->atm_typ[i] < 0 || s->atm_typ[i] >= s->ntyp) return fail(c, PINYB200_ERR_ARG, "atm_typ out of range");
    const int npt = s->ntyp * (s->ntyp + 1) / 2;
    for (int p = 0; p < npt; p++)
        if (s->inter_map[p] < 0 || s->inter_map[p] >= s->ninter_unique)
            return fail(c, PINYB200_ERR_ARG, "inter_map out of range");
    for (int i = 0; i < s->excl_off[s->natm]; i++)
        if (s->excl_j[i] < 0 || s->excl_j[i] >= s->natm) return fail(c, PINYB200_ERR_ARG, "excl_j out of range");
    if (s->nktot > 0) {
        int N[3] = {s->ngrid_a, s->ngrid_b, s->ngrid_c};
        for (int d = 0; d < 3; d++)
            if (N[d] < s->n_interp || N[d] > 256) return fail(c, PINYB200_ERR_ARG, "PME grid size out of range");
        for (int i = 0; i < s->nktot; i++) {
            int k[3] = {s->kastr[i], s->kbstr[i], s->kcstr[i]};
            for (int d = 0; d < 3; d++)
                if (2 * abs(k[d]) >= N[d]) return fail(c, PINYB200_ERR_ARG, "k vector beyond the PME grid");
        }
    }
    for (int i = 0; i < s->nbond; i++)
        if (s->bond_j1[i] < 0 || s->bond_j1[i] >= s->natm || s->bond_j2[i] < 0 || s->bond_j2[i] >= s->natm ||
            s->bond_typ[i] < 0 || s->bond_typ[i] >= s->nbond_typ)
            return fail(c, PINYB200_ERR_ARG, "bond index out of range");
    for (int i = 0; i < s->nbend; i++)
        if (s->bend_j1[i] < 0 || s->bend_j1[i] >= s->natm || s->bend_j2[i] < 0 || s->bend_j2[i] >= s->natm ||
            s->bend_j3[i] < 0 || s->bend_j3[i] >= s->natm || s->bend_typ[i] < 0 || s->bend_typ[i] >= s->nbend_typ)
            return fail(c, PINYB200_ERR_ARG, "bend index out of range");
    for (int i = 0; i < s->necor; i++)
        if (s->ecor_j1[i] < 0 || s->ecor_j1[i] >= s->natm || s->ecor_j2[i] < 0 || s->ecor_j2[i] >= s->natm)
            return fail(c, PINYB200_ERR_ARG, "ecor index out of range");
    for (int g = 0; g < s->nghost; g++) {
        if (s->ghost_atom[g] < 0 || s->ghost_atom[g] >= s->natm) return fail(c, PINYB200_ERR_ARG, "ghost atom");
        for (int k = 0; k < s->ghost_ncomp; k++) {
            int a = s->ghost_comp[g * s->ghost_ncomp + k];
            if (a >= s->natm) return fail(c, PINYB200_ERR_ARG, "ghost component out of range");
        }
    }
    return PINYB200_OK;
}

}  // namespace

// Scratch of pinyb200_count_list_device: one fixed array per GPU, so that
// call allocates no device memory.  Byte layout:
//   [0, 16)                 totals (full, active) as two unsigned 64-bit
//                           integers; accumulated, so cleared by every call
//   [256, 256 + 8*MAXPT)    copy of cutskin2 (PINYB200_COUNT_MAX_PAIR_TYPES)
//   [4096, 4096 + 8*MAXAT)  per-atom counts [2][natm] (full, active); every
//                           entry is written by the count pass, none is read
//                           before it is written
static constexpr size_t kCountTotOff = 0;
static constexpr size_t kCountCutOff = 256;
static constexpr size_t kCountRowOff = 4096;
static constexpr size_t kCountScratchBytes = kCountRowOff + 2 * sizeof(int) * (size_t)PINYB200_COUNT_MAX_ATOMS;
static_assert(kCountCutOff + 8 * PINYB200_COUNT_MAX_PAIR_TYPES <= kCountRowOff, "count scratch layout");
static __device__ __align__(256) unsigned char g_count_scratch[kCountScratchBytes];

// Device address of g_count_scratch per GPU, looked up on the first call
// made with that GPU current.
static constexpr int kCountMaxDevices = 64;
static std::mutex g_count_mu;
static unsigned char *g_count_addr[kCountMaxDevices];

Cell pinyb200::cell_from_hmat(const double *hmat) { return make_cell(hmat); }
int pinyb200::record_error(pinyb200_ctx *c, int code, const std::string &msg) { return fail(c, code, msg); }
static int pme_tiles_setup(pinyb200_ctx *c, int T);
void pinyb200::table_coefs(const double *t, int nsplin, std::vector<double> &out) { cubic_coefs(t, nsplin, out); }
int pinyb200::pme_tiles_resize(pinyb200_ctx *c, int T)
{
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaStreamSynchronize(c->pme_stream));
    return pme_tiles_setup(c, T);
}

// Charge bins for the PME tiles of edge T: about twice the mean occupancy
// per (tile, bead); the rest goes to the overflow list, which can hold every
// charge.  Called at creation and by the autotuner.
static int pme_tiles_setup(pinyb200_ctx *c, int T)
{
    const int N[3] = {c->sys.ngrid[0], c->sys.ngrid[1], c->sys.ngrid[2]};
    for (int d = 0; d < 3; d++) c->pme_nt[d] = (N[d] + T - 1) / T;
    c->pme_tile = T;
    c->gen++;
    c->pme_ntile = c->pme_nt[0] * c->pme_nt[1] * c->pme_nt[2];
    const int mean = (c->sys.nchrg + c->pme_ntile - 1) / c->pme_ntile;
    c->pme_cap = (2 * mean + 32 + 31) / 32 * 32;
    if (c->d_pme_cnt) cudaFree(c->d_pme_cnt);
    if (c->d_pme_bin) cudaFree(c->d_pme_bin);
    c->d_pme_cnt = c->d_pme_bin = nullptr;
    CK(cudaMalloc(&c->d_pme_cnt, ((size_t)c->P * c->pme_ntile + 1) * sizeof(int)));
    CK(cudaMalloc(&c->d_pme_bin, (size_t)c->P * c->pme_ntile * c->pme_cap * sizeof(int)));
    return PINYB200_OK;
}

// PME mesh of one reciprocal set into the context's PME fields (sys.ngrid,
// k list, B-spline weights, k mask; grid, spectrum, filter, tiles, records,
// twiddles): the evaluation's mesh at creation, PINY's RESPA mesh into a
// PmeSet by way of pme_swap.
static int pme_alloc(pinyb200_ctx *c, int nbeads, const int *ngrid, int n_interp, int nktot, const int *kastr,
                     const int *kbstr, const int *kcstr, const double *bweight)
{
    DeviceSystem &d = c->sys;
    d.nktot = nktot;
    d.ngrid[0] = ngrid[0];
    d.ngrid[1] = ngrid[1];
    d.ngrid[2] = ngrid[2];
    d.n_interp = n_interp;
    if (nktot > 0) {
        std::vector<int> kv((size_t)3 * nktot);
        for (int i = 0; i < nktot; i++) {
            kv[3 * i] = kastr[i];
            kv[3 * i + 1] = kbstr[i];
            kv[3 * i + 2] = kcstr[i];
        }
        CK(upload(&d.kvec, kv.data(), kv.size()));
        CK(upload(&d.bweight, bweight, nktot));
        const int Na = ngrid[0], Nb = ngrid[1], Nc = ngrid[2];
        const size_t G = (size_t)Na * Nb * Nc;
        std::vector<int> mask(G, -1);
        for (int i = 0; i < nktot; i++) {
            int a = ((kastr[i] % Na) + Na) % Na, b = ((kbstr[i] % Nb) + Nb) % Nb, cc = ((kcstr[i] % Nc) + Nc) % Nc;
            mask[((size_t)cc * Nb + b) * Na + a] = i;
            int am = (Na - a) % Na, bm = (Nb - b) % Nb, cm = (Nc - cc) % Nc;
            mask[((size_t)cm * Nb + bm) * Na + am] = i;
        }
        CK(upload(&d.kmask, mask.data(), G));
        CK(cudaMalloc(&c->d_filter, G * (sizeof(double) + sizeof(float))));
        const bool f64 = c->precision == PINYB200_FP64;
        if (pme_plane_smem(Na, Nb, f64) > 220 * 1024 || pme_slab_smem(Na, Nc, f64) > 220 * 1024)
            return fail(c, PINYB200_ERR_UNSUPPORTED, "PME grid plane too large for shared memory");
        const size_t rsz = f64 ? sizeof(double) : sizeof(float);
        const size_t csz = f64 ? sizeof(double2) : sizeof(float2);
        CK(cudaMalloc(&c->d_grid, rsz * G * nbeads));
        CK(cudaMalloc(&c->d_spec, csz * (size_t)Nc * Nb * (Na / 2 + 1) * nbeads));
        // charge bins per grid tile and bead: 16^3 tiles, or 8^3 on small
        // meshes so that spread and gather still get enough blocks
        {
            const int rc2 = pme_tiles_setup(c, std::min(Na, std::min(Nb, Nc)) >= 32 ? 16 : 8);
            if (rc2) return rc2;
        }
        CK(cudaMalloc(&c->d_pme_ovf, (size_t)std::max(1, d.nchrg) * nbeads * sizeof(int)));
        // per (charge, bead) records: stencil origin and the six weight rows
        const int nip = n_interp <= 4 ? 4 : (n_interp <= 8 ? 8 : 12);
        const size_t nrec = (size_t)std::max(1, d.nchrg) * nbeads;
        CK(cudaMalloc(&c->d_pme_head, nrec * 4 * sizeof(int)));
        CK(cudaMalloc(&c->d_forceP, nrec * 3 * sizeof(double)));
        CK(cudaMalloc(&c->d_pme_w, nrec * 6 * nip * rsz));
        // twiddles exp(2 pi i m / N) per axis, 256 entries each
        std::vector<double> tw(2 * 256 * 3, 0.0);
        std::vector<float> tw32(tw.size());
        const int N3[3] = {Na, Nb, Nc};
        for (int ax = 0; ax < 3; ax++)
            for (int m = 0; m < N3[ax]; m++) {
                tw[2 * (256 * ax + m)] = cos(2.0 * M_PI * m / N3[ax]);
                tw[2 * (256 * ax + m) + 1] = sin(2.0 * M_PI * m / N3[ax]);
            }
        for (size_t i = 0; i < tw.size(); i++) tw32[i] = (float)tw[i];
        CK(upload(&c->d_twiddle64, tw.data(), tw.size()));
        CK(upload(&c->d_twiddle32, tw32.data(), tw32.size()));
    }
    c->filter_ok = false;
    return PINYB200_OK;
}

void pinyb200::pme_swap(pinyb200_ctx *c, PmeSet &p)
{
    using std::swap;
    DeviceSystem &d = c->sys;
    for (int k = 0; k < 3; k++) {
        swap(d.ngrid[k], p.ngrid[k]);
        swap(c->pme_nt[k], p.pme_nt[k]);
    }
    swap(d.n_interp, p.n_interp);
    swap(d.nktot, p.nktot);
    swap(d.kvec, p.kvec);
    swap(d.kmask, p.kmask);
    swap(d.bweight, p.bweight);
    swap(c->d_grid, p.d_grid);
    swap(c->d_spec, p.d_spec);
    swap(c->d_filter, p.d_filter);
    swap(c->d_forceP, p.d_forceP);
    swap(c->pme_tile, p.pme_tile);
    swap(c->pme_ntile, p.pme_ntile);
    swap(c->pme_cap, p.pme_cap);
    swap(c->d_pme_cnt, p.d_pme_cnt);
    swap(c->d_pme_bin, p.d_pme_bin);
    swap(c->d_pme_ovf, p.d_pme_ovf);
    swap(c->d_pme_head, p.d_pme_head);
    swap(c->d_pme_w, p.d_pme_w);
    swap(c->d_twiddle64, p.d_twiddle64);
    swap(c->d_twiddle32, p.d_twiddle32);
    swap(c->filter_ok, p.filter_ok);
    for (int k = 0; k < 9; k++) swap(c->filter_h[k], p.filter_h[k]);
}

// PINY's separate RESPA PME mesh into c->pme_res (replacing any earlier one).
int pinyb200::pme_res_setup(pinyb200_ctx *c, const int *ngrid, int n_interp, int nktot, const int *kastr,
                            const int *kbstr, const int *kcstr, const double *bweight)
{
    pme_res_free(c);
    PmeSet fresh;
    pme_swap(c, fresh);  // the context's PME fields are empty now
    int rc = pme_alloc(c, c->P, ngrid, n_interp, nktot, kastr, kbstr, kcstr, bweight);
    pme_swap(c, fresh);  // the new mesh into `fresh`, the evaluation's back
    c->pme_res = fresh;
    c->pme_res.on = rc == PINYB200_OK;
    if (rc) pme_res_free(c);
    return rc;
}

void pinyb200::pme_res_free(pinyb200_ctx *c)
{
    PmeSet &p = c->pme_res;
    void *ptrs[] = {p.kvec, p.kmask, p.bweight, p.d_grid, p.d_spec, p.d_filter, p.d_forceP, p.d_pme_cnt, p.d_pme_bin,
                    p.d_pme_ovf, p.d_pme_head, p.d_pme_w, p.d_twiddle64, p.d_twiddle32};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    p = PmeSet();
}

// Per-site-pair parameters of the MIXED molecule-pair kernel
// (mol_pair_mixed_kernel): for site pair (si, sj) of the uniform molecule
// with pair type p and table u = inter_map[p], its row offset u * nsplin + 2,
// charge product and which of the tables (Coulomb, vdW) it reads
// (force_npol.c:339-375).  Set only when every site pair shares the cutoff
// and the spline grid; otherwise mix_ok stays false and mol_pair_kernel runs.
static void mixed_setup(pinyb200_ctx *c, const pinyb200_system *s, int n0)
{
    const int NS = c->mol_ns;
    const size_t per = (size_t)s->nsplin;
    int p0 = -1;
    for (int si = 0; si < NS; si++)
        for (int sj = 0; sj < NS; sj++) {
            const int sp = si * NS + sj;
            const int ia = si < n0 ? si : 0, ja = sj < n0 ? sj : 0;
            const int ti = s->atm_typ[ia], tj = s->atm_typ[ja];
            const int i2 = ti + 1, i3 = tj + 1, jj = std::min(i2, i3), ii = i2 + i3 - jj;
            const int p = ((jj - 1) * ((s->ntyp + 1) * 2 - jj)) / 2 + ii - jj;
            if (p0 < 0) p0 = p;
            const int u = s->inter_map[p], u0 = s->inter_map[p0];
            if (s->cutoff[p] != s->cutoff[p0] || s->rmin_spl[u] != s->rmin_spl[u0] ||
                s->dri_spl[u] != s->dri_spl[u0] || s->dr_spl[u] != s->dr_spl[u0])
                return;  // not uniform: mol_pair_kernel
            bool vdw = false;
            for (size_t k = 0; k < per; k++)
                vdw |= s->cv0[(size_t)u * per + k] != 0.0 || s->cdv0[(size_t)u * per + k] != 0.0;
            const double q2 = s->charge[ia] * s->charge[ja];
            c->mix_eflag[sp] = (vdw ? 1 : 0) | (q2 != 0.0 ? 2 : 0);
            c->mix_q2[sp] = (float)q2;
            c->mix_toff[sp] = (int)((size_t)u * per + 2);  // knot k = nint(t) + 3, coefficients at k - 1
        }
    const int u0 = s->inter_map[p0];
    c->mix_rc2 = (float)(s->cutoff[p0] * s->cutoff[p0]);
    c->mix_dri = (float)s->dri_spl[u0];
    c->mix_rmd = (float)(s->rmin_spl[u0] * s->dri_spl[u0]);
    c->mix_tmax = (float)(s->nsplin - 5);
    // force and energy rows of each interval side by side, for the
    // evaluations with energies: [vdW, Coulomb][u][k][force, energy]
    {
        const size_t nu = (size_t)c->sys.nuniq;
        std::vector<double> cf, ce;
        std::vector<float> fe((size_t)2 * nu * per * 8, 0.0f);
        const double *tf[2] = {s->cdv0, s->cdv0_c}, *te[2] = {s->cv0, s->cv0_c};
        for (int kind = 0; kind < 2; kind++)
            for (size_t u = 0; u < nu; u++) {
                if (!tf[kind] || !te[kind]) continue;
                cubic_coefs(tf[kind] + u * per, s->nsplin, cf);
                cubic_coefs(te[kind] + u * per, s->nsplin, ce);
                float *dst = fe.data() + ((size_t)kind * nu + u) * per * 8;
                for (size_t k = 0; k < per; k++)
                    for (int e = 0; e < 4; e++) {
                        dst[8 * k + e] = (float)cf[4 * k + e];
                        dst[8 * k + 4 + e] = (float)ce[4 * k + e];
                    }
            }
        if (upload((float **)&c->d_tabfe, fe.data(), fe.size()) != cudaSuccess) return;
    }
    c->mix_ok = (size_t)c->sys.nuniq * per * 4 < (size_t)0x7fffffff;
    // one wave of resident blocks (5 per SM at its register count) serves
    // the grid-strided chunks best at the benchmark sizes
    if (c->mix_ok) c->pair_blocks_per_sm = 5;
}

extern "C" {

int pinyb200_version(void) { return 1; }

const char *pinyb200_last_error(pinyb200_ctx *ctx) { return ctx ? ctx->err.c_str() : g_lib_err.c_str(); }

int pinyb200_device_info(char *name, int len, int *sm_count)
{
    pinyb200_ctx *c = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return fail(c, PINYB200_ERR_NO_DEVICE, "no CUDA device");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    cudaDeviceProp p;
    CK(cudaGetDeviceProperties(&p, dev));
    if (name && len > 0) {
        strncpy(name, p.name, len - 1);
        name[len - 1] = 0;
    }
    if (sm_count) *sm_count = p.multiProcessorCount;
    return PINYB200_OK;
}

int pinyb200_destroy(pinyb200_ctx *c)
{
    if (!c) return PINYB200_OK;
    cudaSetDevice(c->device);
    pme_res_free(c);
    free_sys(c->sys);
    void *ptrs[] = {c->d_row, c->d_col, c->d_rowA, c->d_colA, c->d_count, c->d_tot, c->d_posT, c->d_forceT,
                    c->d_xmod, c->d_pos_aos, c->d_force_aos, c->d_acc, c->d_grid, c->d_spec, c->d_filter, c->d_twiddle64,
                    c->d_twiddle32, c->d_err, c->d_mstart, c->d_mcount, c->d_mrow, c->d_mj, c->d_mmask, c->d_chunk,
                    c->d_pme_cnt, c->d_pme_bin, c->d_pme_ovf, c->d_x0, c->d_forceP,
                    c->d_pme_head, c->d_pme_w, c->d_nchunk, c->d_ls, c->d_cs, c->d_mchunk, c->d_mmaskf,
                    c->d_reach, c->d_cut_res, c->d_bond_eq_res, c->d_forceW, c->d_forcet_aos, c->d_rowR,
                    c->d_colR, c->d_rtot, c->d_xm0, c->d_cs0, c->d_ecor_res_tab, c->d_cs_in, c->d_tabfe,
                    c->d_mcell, c->d_msf, c->d_ccnt, c->d_coff, c->d_cmol, c->d_cellok, c->d_ctot, c->d_ent, c->d_nent,
                    c->d_scan_part, c->d_reach_acc};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (cudaEvent_t e : c->kt_ev) cudaEventDestroy(e);
    if (c->eg_exec) cudaGraphExecDestroy(c->eg_exec);
    if (c->h_acc_pin) cudaFreeHost(c->h_acc_pin);
    for (int i = 0; i < 8; i++)
        if (c->ev[i]) cudaEventDestroy(c->ev[i]);
    for (void *p : c->grad.dev) cudaFree(p);
    c->grad.dev.clear();
    cudaEvent_t evx[4] = {c->ev_fork, c->ev_join, c->ev_pme[0], c->ev_pme[1]};
    for (cudaEvent_t ev : evx)
        if (ev) cudaEventDestroy(ev);
    if (c->pme_stream) cudaStreamDestroy(c->pme_stream);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return PINYB200_OK;
}

int pinyb200_create(const pinyb200_system *s, int nbeads, int precision, pinyb200_ctx **out)
{
    pinyb200_ctx *c = nullptr;
    if (!out) return fail(c, PINYB200_ERR_ARG, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(c, PINYB200_ERR_NO_DEVICE, "no CUDA device");
    int rc = check_system(nullptr, s, nbeads);
    if (rc) return rc;
    if (precision != PINYB200_FP64 && precision != PINYB200_MIXED)
        return fail(c, PINYB200_ERR_ARG, "precision must be PINYB200_FP64 or PINYB200_MIXED");
    c = new pinyb200_ctx();
    for (int i = 0; i < 8; i++) c->ev[i] = nullptr;
    CK(cudaGetDevice(&c->device));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, c->device));
    c->sm_count = prop.multiProcessorCount;
    c->precision = precision;
    c->P = nbeads;
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->pme_stream, cudaStreamNonBlocking));
    for (int i = 0; i < 8; i++) CK(cudaEventCreate(&c->ev[i]));
    CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
    for (int i = 0; i < 2; i++) CK(cudaEventCreate(&c->ev_pme[i]));

    DeviceSystem &d = c->sys;
    const int natm = s->natm;
    d.natm = natm;
    d.ntyp = s->ntyp;
    d.npair_typ = s->ntyp * (s->ntyp + 1) / 2;
    d.nsplin = s->nsplin;
    d.nuniq = s->ninter_unique;
    CK(upload(&d.atm_typ, s->atm_typ, natm));
    CK(upload(&d.charge, s->charge, natm));
    c->h_charge.assign(s->charge, s->charge + natm);
    c->h_cutoff.assign(s->cutoff, s->cutoff + s->ntyp * (s->ntyp + 1) / 2);
    c->skin = s->skin;
    c->nbond_typ = s->nbond_typ;
    c->nbend_typ = s->nbend_typ;
    CK(upload(&d.inter_map, s->inter_map, d.npair_typ));
    CK(upload(&d.cutoff, s->cutoff, d.npair_typ));
    CK(upload(&d.rmin, s->rmin_spl, d.nuniq));
    CK(upload(&d.dr, s->dr_spl, d.nuniq));
    CK(upload(&d.dri, s->dri_spl, d.nuniq));
    // tables -> interval coefficients, [kind][u][k]
    {
        const size_t per = (size_t)s->nsplin;
        std::vector<double> all((size_t)4 * 4 * d.nuniq * per, 0.0), tmp;
        std::vector<int> has_vdw(d.nuniq, 0);
        const double *tabs[4] = {s->cv0, s->cdv0, s->cv0_c, s->cdv0_c};
        for (int kind = 0; kind < 4; kind++)
            for (int u = 0; u < d.nuniq; u++) {
                const double *t = tabs[kind] + (size_t)u * per;
                if (kind <= 1)
                    for (size_t k = 0; k < per; k++)
                        if (t[k] != 0.0) has_vdw[u] = 1;
                cubic_coefs(t, s->nsplin, tmp);
                std::copy(tmp.begin(), tmp.end(), all.begin() + ((size_t)kind * d.nuniq + u) * per * 4);
            }
        CK(upload(&d.has_vdw, has_vdw.data(), d.nuniq));
        CK(upload((double **)&d.tab64, all.data(), all.size()));
        std::vector<float> f32(all.size());
        for (size_t i = 0; i < all.size(); i++) f32[i] = (float)all[i];
        CK(upload((float **)&d.tab32, f32.data(), f32.size()));
    }
    c->clong = s->clong;
    c->iswit_vdw = s->iswit_vdw;
    CK(upload(&d.excl_off, s->excl_off, natm + 1));
    CK(upload(&d.excl_j, s->excl_j, (size_t)s->excl_off[natm]));
    {
        std::vector<int> ich;
        for (int i = 0; i < natm; i++)
            if (s->charge[i] != 0.0) ich.push_back(i);
        d.nchrg = (int)ich.size();
        CK(upload(&d.ichrg, ich.data(), ich.size()));
    }
    c->alp_ewd = s->alp_ewd;
    c->self_erf = s->self_erf;
    {
        const int ng[3] = {s->ngrid_a, s->ngrid_b, s->ngrid_c};
        if (int rc = pme_alloc(c, nbeads, ng, s->n_interp, s->nktot, s->kastr, s->kbstr, s->kcstr, s->bweight)) {
            if (rc != PINYB200_ERR_UNSUPPORTED) return rc;
            const std::string msg = c->err;
            pinyb200_destroy(c);
            return fail(nullptr, rc, msg);
        }
    }
    d.necor = s->necor;
    if (s->necor > 0) {
        CK(upload(&d.ecor_j1, s->ecor_j1, s->necor));
        CK(upload(&d.ecor_j2, s->ecor_j2, s->necor));
        d.ecor_nsplin = s->ecor_nsplin;
        d.ecor_rmin = s->ecor_rmin;
        d.ecor_dr = s->ecor_dr;
        d.ecor_dri = s->ecor_dri;
        std::vector<double> a, b;
        cubic_coefs(s->ecor_cv0, s->ecor_nsplin, a);
        cubic_coefs(s->ecor_cdv0, s->ecor_nsplin, b);
        a.insert(a.end(), b.begin(), b.end());
        CK(upload((double **)&d.ecor_tab, a.data(), a.size()));
    }
    d.nbond = s->nbond;
    if (s->nbond > 0) {
        std::vector<int> bj((size_t)3 * s->nbond);
        for (int i = 0; i < s->nbond; i++) {
            bj[3 * i] = s->bond_j1[i];
            bj[3 * i + 1] = s->bond_j2[i];
            bj[3 * i + 2] = s->bond_typ[i];
        }
        CK(upload(&d.bond_j, bj.data(), bj.size()));
        CK(upload(&d.bond_eq, s->bond_eq, s->nbond_typ));
        CK(upload(&d.bond_c, s->bond_c, (size_t)7 * s->nbond_typ));
        CK(upload(&d.bond_dc, s->bond_dc, (size_t)7 * s->nbond_typ));
    }
    d.nbend = s->nbend;
    if (s->nbend > 0) {
        std::vector<int> bj((size_t)4 * s->nbend);
        for (int i = 0; i < s->nbend; i++) {
            bj[4 * i] = s->bend_j1[i];
            bj[4 * i + 1] = s->bend_j2[i];
            bj[4 * i + 2] = s->bend_j3[i];
            bj[4 * i + 3] = s->bend_typ[i];
        }
        CK(upload(&d.bend_j, bj.data(), bj.size()));
        CK(upload(&d.bend_c, s->bend_c, (size_t)7 * s->nbend_typ));
        CK(upload(&d.bend_s, s->bend_s, (size_t)7 * s->nbend_typ));
        CK(upload(&d.bend_dc, s->bend_dc, (size_t)7 * s->nbend_typ));
        CK(upload(&d.bend_ds, s->bend_ds, (size_t)7 * s->nbend_typ));
    }
    d.nghost = s->nghost;
    d.ghost_ncomp = s->ghost_ncomp;
    if (s->nghost > 0) {
        CK(upload(&d.ghost_atom, s->ghost_atom, s->nghost));
        CK(upload(&d.ghost_comp, s->ghost_comp, (size_t)s->nghost * s->ghost_ncomp));
        CK(upload(&d.ghost_coef, s->ghost_coef, (size_t)s->nghost * s->ghost_ncomp));
    }
    const size_t nb = (size_t)natm * 3 * nbeads;
    CK(cudaMalloc(&c->d_posT, nb * sizeof(double)));
    CK(cudaMalloc(&c->d_forceT, nb * sizeof(double)));
    CK(cudaMalloc(&c->d_pos_aos, nb * sizeof(double)));
    CK(cudaMalloc(&c->d_force_aos, nb * sizeof(double)));
    CK(cudaMalloc(&c->d_xmod, (size_t)natm * 3 * sizeof(double)));
    CK(cudaMalloc(&c->d_x0, (size_t)natm * 3 * sizeof(double)));
    CK(cudaMalloc(&c->d_acc, (size_t)nbeads * S_NSLOT * sizeof(double)));
    CK(cudaMalloc(&c->d_row, (size_t)(natm + 1) * sizeof(int)));
    CK(cudaMalloc(&c->d_rowA, (size_t)(natm + 1) * sizeof(int)));
    CK(cudaMalloc(&c->d_count, (size_t)2 * natm * sizeof(int)));
    CK(cudaMalloc(&c->d_tot, 8 * sizeof(long long)));  // list totals [4], chunk total, spare
    CK(cudaMalloc(&c->d_cs_in, (size_t)d.npair_typ * sizeof(double)));
    // molecules: connected components of the exclusion graph, each a run of
    // at most 4 consecutive sites (water); otherwise the site kernel is used
    {
        std::vector<int> root(natm);
        for (int i = 0; i < natm; i++) root[i] = i;
        auto find = [&](int x) {
            while (root[x] != x) x = root[x] = root[root[x]];
            return x;
        };
        for (int i = 0; i < natm; i++)
            for (int e = s->excl_off[i]; e < s->excl_off[i + 1]; e++) {
                int a = find(i), b = find(s->excl_j[e]);
                if (a != b) root[a < b ? b : a] = a < b ? a : b;
            }
        std::vector<int> mstart;
        bool ok = true;
        int maxn = 0;
        for (int i = 0; i < natm; i++) {
            if (i == 0 || find(i) != find(i - 1)) {
                if (find(i) != i) ok = false;  // not a new contiguous component
                mstart.push_back(i);
            }
        }
        mstart.push_back(natm);
        for (size_t m = 0; m + 1 < mstart.size(); m++) maxn = std::max(maxn, mstart[m + 1] - mstart[m]);
        // the molecule kernel also needs identical molecules (sizes, types, charges)
        for (size_t m = 1; ok && m + 1 < mstart.size(); m++) {
            const int n0 = mstart[1] - mstart[0], nm = mstart[m + 1] - mstart[m];
            if (nm != n0) ok = false;
            for (int k = 0; ok && k < nm; k++)
                if (s->atm_typ[mstart[m] + k] != s->atm_typ[k] || s->charge[mstart[m] + k] != s->charge[k]) ok = false;
        }
        // every pair inside a molecule must be excluded: the molecule lists
        // hold pairs of different molecules only
        for (size_t m = 0; ok && m + 1 < mstart.size(); m++)
            for (int i = mstart[m]; ok && i < mstart[m + 1]; i++)
                for (int j = mstart[m]; ok && j < i; j++) {
                    bool ex = false;
                    for (int e = s->excl_off[i]; e < s->excl_off[i + 1]; e++) ex |= s->excl_j[e] == j;
                    for (int e = s->excl_off[j]; e < s->excl_off[j + 1]; e++) ex |= s->excl_j[e] == i;
                    if (!ex) ok = false;
                }
        if (ok && maxn <= 4 && s->ntyp <= 8) {
            c->use_mol = true;
            c->nmol = (int)mstart.size() - 1;
            c->mol_ns = maxn <= 3 ? 3 : 4;
            CK(upload(&c->d_mstart, mstart.data(), mstart.size()));
            CK(cudaMalloc(&c->d_mcount, (size_t)c->nmol * sizeof(int)));
            CK(cudaMalloc(&c->d_mrow, (size_t)(c->nmol + 1) * sizeof(int)));
            CK(cudaMalloc(&c->d_msf, (size_t)c->nmol * sizeof(float4)));
            CK(cudaMalloc(&c->d_nent, sizeof(unsigned long long)));
            const int n0 = mstart[1];
            bool strided = true;
            for (size_t m = 0; m < mstart.size(); m++) strided &= mstart[m] == (int)m * n0;
            c->mol_stride = strided ? n0 : 0;
            if (strided && precision == PINYB200_MIXED) mixed_setup(c, s, n0);
        }
    }
    CK(cudaMalloc(&c->d_err, sizeof(int)));
    CK(cudaMemset(c->d_err, 0, sizeof(int)));
    // device-wide scans: tile sums for two arrays of up to max(natm + 1, 64^3) counts
    c->scan_part_cap = 2LL * scan_tiles(std::max(natm + 1, 1 << 18));
    CK(cudaMalloc(&c->d_scan_part, (size_t)c->scan_part_cap * sizeof(long long)));
    CK(cudaMalloc(&c->d_reach_acc, 4 * sizeof(unsigned long long)));
    CK(cudaMemset(c->d_reach_acc, 0, 4 * sizeof(unsigned long long)));
    *out = c;
    return PINYB200_OK;
}

int pinyb200_build_list(pinyb200_ctx *c, const double *pos1, const double *xmod, const double *hmat,
                        const double *cutskin2, long *npairs)
{
    if (!c || !pos1 || !hmat || !cutskin2) return fail(c, PINYB200_ERR_ARG, "build_list: NULL argument");
    CK(cudaSetDevice(c->device));
    c->gen++;  // the list arrays may move
    const int natm = c->sys.natm;
    Cell cell = make_cell(hmat);
    double *d_p1 = c->d_pos_aos;  // bead-1 positions in the staging buffer
    CK(cudaMemcpyAsync(d_p1, pos1, (size_t)natm * 3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const double *d_xm = nullptr;
    if (xmod) {
        CK(cudaMemcpyAsync(c->d_xmod, xmod, (size_t)natm * 3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        d_xm = c->d_xmod;
    }
    double *d_cs = c->d_cs_in;  // reserved at creation: no allocation per build
    CK(cudaMemcpyAsync(d_cs, cutskin2, c->sys.npair_typ * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    // grow like ver_list_mem_check (verlist_control.c:87-110), with slack
    // for lists that grow between host builds (device updates)
    auto grow_sites = [&](long long need) -> int {
        if (need <= c->list_cap && c->d_col) return PINYB200_OK;
        if (c->d_col) cudaFree(c->d_col);
        if (c->d_colA) cudaFree(c->d_colA);
        c->d_col = c->d_colA = nullptr;
        const long long cap = need + need / 4 + 1024;
        CK(cudaMalloc(&c->d_col, cap * sizeof(int)));
        CK(cudaMalloc(&c->d_colA, cap * sizeof(int)));
        c->list_cap = cap;
        return PINYB200_OK;
    };
    long long tot[4] = {0, 0, 0, 0};
    c->mol_ok = false;
    if (c->use_mol) {
        // molecule-pair list first; the site lists are expanded from its masks
        if (!c->d_reach) CK(cudaMalloc(&c->d_reach, sizeof(double)));
        if (int rc = mol_cells_plan(c, cell, d_p1, d_cs)) return rc;
        CK(cudaMemsetAsync(c->d_tot, 0, 4 * sizeof(long long), c->stream));
        CK(launch_mol_list(c, cell, d_p1, d_xm, d_cs, 0));
        CK(cudaMemcpyAsync(tot, c->d_tot, sizeof(tot), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (tot[2] > c->mlist_cap || !c->d_mj) {
            if (c->d_mj) cudaFree(c->d_mj);
            if (c->d_mmask) cudaFree(c->d_mmask);
            if (c->d_mmaskf) cudaFree(c->d_mmaskf);
            if (c->d_ent) cudaFree(c->d_ent);
            c->d_mj = nullptr;
            c->d_mmask = c->d_mmaskf = nullptr;
            c->d_ent = nullptr;
            c->ent_cap = 0;
            const long long cap = tot[2] + tot[2] / 4 + 1024;
            CK(cudaMalloc(&c->d_mj, cap * sizeof(int)));
            CK(cudaMalloc(&c->d_mmask, cap * sizeof(unsigned)));
            CK(cudaMalloc(&c->d_mmaskf, cap * sizeof(unsigned)));
            CK(cudaMalloc(&c->d_ent, cap * sizeof(int4)));
            c->mlist_cap = c->ent_cap = cap;
            // the count pass wrote its pairs into the freed buffer: the fill computes
            CK(cudaMemsetAsync(c->d_nent, 0xff, sizeof(unsigned long long), c->stream));
        }
        CK(launch_mol_list(c, cell, d_p1, d_xm, d_cs, 1));
        CK(launch_site_from_mol(c, 0));
        CK(cudaMemcpyAsync(tot, c->d_tot, sizeof(tot), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (tot[0] > 0x7fffffffLL) return fail(c, PINYB200_ERR_LIST_OVERFLOW, "Verlet list exceeds 2^31 pairs");
        if (int rc = grow_sites(tot[0])) return rc;
        CK(launch_site_from_mol(c, 1));
        c->nmp = tot[2];
        // the active site pairs of the masks are the active site list
        if (tot[3] == tot[1]) {
            std::vector<int> mrow(c->nmol + 1);
            CK(cudaMemcpy(mrow.data(), c->d_mrow, mrow.size() * sizeof(int), cudaMemcpyDeviceToHost));
            const int jpi = c->P >= 32 ? 1 : 32 / c->P;
            const int ch = PINYB200_MOL_CHUNK * jpi;
            std::vector<int> chunks;
            for (int m = 0; m < c->nmol; m++)
                for (int k = mrow[m]; k < mrow[m + 1]; k += ch) {
                    chunks.push_back(m);
                    chunks.push_back(k);
                    chunks.push_back(std::min(k + ch, mrow[m + 1]));
                }
            c->nchunk = (int)(chunks.size() / 3);
            if (!c->d_chunk || c->nchunk > c->chunk_cap) {
                if (c->d_chunk) cudaFree(c->d_chunk);
                c->d_chunk = nullptr;
                const long long cap = c->nchunk + c->nchunk / 4 + 256;
                CK(cudaMalloc(&c->d_chunk, (size_t)cap * 3 * sizeof(int)));
                c->chunk_cap = cap;
            }
            CK(cudaMemcpy(c->d_chunk, chunks.data(), chunks.size() * sizeof(int), cudaMemcpyHostToDevice));
            if (!c->d_nchunk) CK(cudaMalloc(&c->d_nchunk, sizeof(int)));
            CK(cudaMemcpy(c->d_nchunk, &c->nchunk, sizeof(int), cudaMemcpyHostToDevice));
            c->mol_ok = true;
        }
    } else {
        CK(launch_build_list(c, cell, d_p1, d_xm, d_cs, 0));
        CK(cudaMemcpyAsync(tot, c->d_tot, 2 * sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (tot[0] > 0x7fffffffLL) return fail(c, PINYB200_ERR_LIST_OVERFLOW, "Verlet list exceeds 2^31 pairs");
        if (int rc = grow_sites(tot[0])) return rc;
        CK(launch_build_list(c, cell, d_p1, d_xm, d_cs, 1));
    }
    // the rebuild test measures displacements from these positions
    CK(cudaMemcpyAsync(c->d_x0, d_p1, (size_t)natm * 3 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    // mode-1 positions and cutskin^2 of this build, for the RESPA list
    if (!c->d_xm0) CK(cudaMalloc(&c->d_xm0, (size_t)natm * 3 * sizeof(double)));
    if (!c->d_cs0) CK(cudaMalloc(&c->d_cs0, (size_t)c->sys.npair_typ * sizeof(double)));
    CK(launch_keep_build_state(c, nullptr, d_p1, d_xm, d_cs, c->stream));
    c->build_cell = cell;
    c->build_cell_ok = true;
    if (c->respa_on)
        if (int rc = respa_list_reserve(c, cell)) return rc;
    CK(cudaStreamSynchronize(c->stream));
    c->npairs = tot[0];
    c->nactive = tot[1];
    c->have_list = true;
    if (int rc = list_reset_flags(c)) return rc;
    if (npairs) *npairs = (long)tot[0];
    return PINYB200_OK;
}

int pinyb200_set_list_method(pinyb200_ctx *c, int method)
{
    if (!c) return fail(c, PINYB200_ERR_ARG, "NULL context");
    if (method != PINYB200_LIST_LNK && method != PINYB200_LIST_NOLST)
        return fail(c, PINYB200_ERR_ARG, "set_list_method: unknown method");
    c->list_method = method;
    return PINYB200_OK;
}

int pinyb200_list_cells(pinyb200_ctx *c, int *cells)
{
    if (!c || !cells) return fail(c, PINYB200_ERR_ARG, "list_cells: NULL argument");
    if (!c->have_list) return fail(c, PINYB200_ERR_STATE, "no list built yet");
    CK(cudaSetDevice(c->device));
    for (int d = 0; d < 3; d++) cells[d] = c->use_mol ? c->cell_n[d] : 0;
    cells[3] = 0;
    if (c->use_mol && c->cell_n[0] > 0) {
        CK(cudaStreamSynchronize(c->stream));
        CK(cudaMemcpy(&cells[3], c->d_cellok, sizeof(int), cudaMemcpyDeviceToHost));
    }
    return PINYB200_OK;
}

int pinyb200_get_list(pinyb200_ctx *c, int *pi, int *pj, long cap, long *npairs)
{
    if (!c) return fail(c, PINYB200_ERR_ARG, "NULL context");
    if (!c->have_list) return fail(c, PINYB200_ERR_STATE, "no list built yet");
    CK(cudaSetDevice(c->device));
    if (int rc = list_sync_counts(c)) return rc;
    if (npairs) *npairs = (long)c->npairs;
    if (!pi || !pj) return PINYB200_OK;
    if (cap < c->npairs) return fail(c, PINYB200_ERR_ARG, "get_list: capacity too small");
    CK(cudaSetDevice(c->device));
    std::vector<int> row(c->sys.natm + 1);
    CK(cudaMemcpy(row.data(), c->d_row, row.size() * sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(pj, c->d_col, c->npairs * sizeof(int), cudaMemcpyDeviceToHost));
    for (int i = 0; i < c->sys.natm; i++)
        for (int k = row[i]; k < row[i + 1]; k++) pi[k] = i;
    return PINYB200_OK;
}

// Device evaluation on inputs already in d_posT (and d_xmod for PIMD).
}  // extern "C"

// Everything one evaluation does on the device, enqueued on c->stream (PME
// forks to the context's PME stream and joins back); no host
// synchronisation, so it can be captured in a CUDA graph.  timing: record
// the phase events (not inside a graph); h_acc: where the per-bead energy
// sums [P][S_NSLOT] are copied (NULL: not copied).
int pinyb200::evaluate_enqueue(pinyb200_ctx *c, const Cell &cell, int flags, bool timing, double *h_acc,
                               double *respa_w)
{
    const bool energy = !(flags & PINYB200_NO_ENERGY);
    const size_t nb = (size_t)c->sys.natm * 3 * c->P;
    if (timing) CK(ev_rec(c->ev[0], c->stream));
    if (c->kt_n == 0) CK(kt_mark(c, nullptr));
    CK(launch_ghost_pos(c));
    CK(kt_mark(c, "ghost_pos"));
    CK(cudaMemsetAsync(c->d_forceT, 0, nb * sizeof(double), c->stream));
    CK(cudaMemsetAsync(c->d_acc, 0, (size_t)c->P * S_NSLOT * sizeof(double), c->stream));
    // the molecule extent bound the pair kernels' image test uses
    CK(launch_mol_extent(c));
    CK(kt_mark(c, "mol_extent"));
    if (timing) CK(ev_rec(c->ev[1], c->stream));
    // PME on its own stream, concurrently with the pair and intramolecular
    // kernels: it reads the positions, writes its own force buffer and adds
    // its energies and virial atomically
    CK(cudaEventRecord(c->ev_fork, c->stream));
    CK(cudaStreamWaitEvent(c->pme_stream, c->ev_fork, 0));
    {
        cudaStream_t main_stream = c->stream;
        if (c->pme_overlap && !c->kt_on) c->stream = c->pme_stream;
        cudaError_t perr = timing ? ev_rec(c->ev_pme[0], c->stream) : cudaSuccess;
        if (perr == cudaSuccess) perr = launch_pme(c, cell, energy);
        if (perr == cudaSuccess && timing) perr = ev_rec(c->ev_pme[1], c->stream);
        if (perr == cudaSuccess) perr = cudaEventRecord(c->ev_join, c->stream);
        c->stream = main_stream;
        CK(perr);
    }
    const bool ortho = cell.h[1] == 0.0 && cell.h[2] == 0.0 && cell.h[3] == 0.0 && cell.h[5] == 0.0 &&
                       cell.h[6] == 0.0 && cell.h[7] == 0.0;
    if (c->use_mol && c->mol_ok && ortho && c->pair_variant == 0 && !(flags & PINYB200_SITE_PAIRS) && c->mix_ok)
        CK(launch_mol_pair_mixed(c, cell, energy));
    else if (c->use_mol && c->mol_ok && ortho && c->pair_variant != 1 && !(flags & PINYB200_SITE_PAIRS))
        CK(launch_mol_pair(c, cell, energy));
    else CK(launch_pair(c, cell, energy));
    CK(kt_mark(c, "pair"));
    if (respa_w) {
        // RESPA outer level: the weighted pair forces from the plain ones
        // (so far the only forces in the buffer) and the switched pairs
        // inside cutoff_res: w_ter F + (w_ter_res - w_ter) swit F
        CK(launch_respa_scale_copy(c, c->r_wter, respa_w));
        if (c->r_int_res_ter) CK(launch_pair_respa(c, cell, 4, respa_w));
    }
    if (timing) CK(ev_rec(c->ev[2], c->stream));
    CK(launch_intra(c, cell, energy));
    CK(kt_mark(c, "intra (bond, bend, ecor)"));
    if (respa_w) {
        CK(launch_intra_respa(c, true, respa_w));
        CK(launch_ecor_weighted(c, c->r_wter, respa_w, c->r_kres ? 2 : 0));
    }
    if (timing) CK(ev_rec(c->ev[3], c->stream));
    CK(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
    CK(launch_pme_force_add(c));
    CK(kt_mark(c, "pme_force_add"));
    if (respa_w) {
        const bool mesh_res = c->r_kres && c->pme_res.on;
        CK(launch_pme_force_add_scaled(c, c->r_kres && !mesh_res ? c->r_wter_res : c->r_wter, respa_w));
        if (mesh_res) {
            // PINY's RESPA mesh at the outer step (energy_control_inter_recip.c:
            // 233-244): x (wght_ter_res - wght_ter) into the weighted forces and,
            // unweighted, into the virial forces; its energy is discarded
            pme_swap(c, c->pme_res);
            cudaError_t e = launch_pme(c, cell, false);
            if (e == cudaSuccess) e = launch_pme_force_add_scaled(c, c->r_wter_res - c->r_wter, respa_w);
            if (e == cudaSuccess) e = launch_pme_force_add(c);
            pme_swap(c, c->pme_res);
            CK(e);
        }
    }
    if (flags & PINYB200_DISTRIB_GHOSTS) {
        CK(launch_ghost_distrib(c));
        if (respa_w) CK(launch_ghost_distrib(c, respa_w));
    }
    if (timing) CK(ev_rec(c->ev[4], c->stream));
    if (energy && h_acc)
        CK(cudaMemcpyAsync(h_acc, c->d_acc, (size_t)c->P * S_NSLOT * sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream));
    return PINYB200_OK;
}

// Host bookkeeping of one evaluation from the per-bead sums acc[P][S_NSLOT]
// (energy_control_inter_real.c:141-183, energy_control_inter_recip.c:
// 341-349, energy_control_intra.c:284-309).
void pinyb200::evaluate_finish(pinyb200_ctx *c, const Cell &cell, int flags, const double *acc, pinyb200_energies *e)
{
    const bool energy = !(flags & PINYB200_NO_ENERGY);
    if (e) {
        memset(e, 0, sizeof(*e));
        if (energy) {
            // bead averages and constant terms as PINY books them
            const double P = (double)c->P;
            double s[S_NSLOT] = {0};
            for (int b = 0; b < c->P; b++)
                for (int k = 0; k < S_NSLOT; k++) s[k] += acc[(size_t)b * S_NSLOT + k];
            double q2 = 0, q1 = 0;
            for (double q : c->h_charge) { q2 += q * q; q1 += q; }
            const bool ewald = c->sys.nktot > 0 && c->sys.nchrg > 0;
            e->vself = ewald ? -q2 * c->alp_ewd * c->self_erf / sqrt(M_PI) : 0.0;
            e->vbgr = ewald ? -0.5 * q1 * q1 * M_PI / (c->alp_ewd * c->alp_ewd * cell.vol) : 0.0;
            e->vlong = c->clong / cell.vol;
            const double vvdw = s[S_VVDW] / P, vcoul = s[S_VCOUL] / P;
            e->vreal = vvdw + vcoul;
            e->vrecip = s[S_VRECIP] / P;
            e->vecor = s[S_VECOR] / P;
            e->vbond = s[S_VBOND] / P;
            e->vbend = s[S_VBEND] / P;
            e->vvdw = vvdw + e->vlong;
            e->vcoul = vcoul + e->vrecip + e->vself + e->vbgr + e->vecor;
            e->vintert = e->vreal + e->vlong + e->vrecip + e->vself + e->vbgr + e->vecor;
            e->vintrat = e->vbond + e->vbend;
            const double amult = c->iswit_vdw ? 1.0 : 2.0;
            const double diag = (c->clong / cell.vol) * amult * P + e->vbgr * P;
            e->pvten[0] = s[S_PXX] + diag;
            e->pvten[4] = s[S_PYY] + diag;
            e->pvten[8] = s[S_PZZ] + diag;
            e->pvten[1] = e->pvten[3] = s[S_PXY];
            e->pvten[2] = e->pvten[6] = s[S_PXZ];
            e->pvten[5] = e->pvten[7] = s[S_PYZ];
        }
    }
}

// mode-1 positions for a PIMD call without xmod: the bead centroid
__global__ void centroid_kernel(const double *__restrict__ posT, double *__restrict__ xm, int natm, int P)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)natm * 3) return;
    double s = 0.0;
    for (int b = 0; b < P; b++) s += posT[t * P + b];
    xm[t] = s / (double)P;
}

// One evaluation from device-resident positions to device-resident forces,
// enqueued on c->stream without host synchronisation (see evaluate_enqueue).
int pinyb200::enqueue_device(pinyb200_ctx *c, const double *d_pos, const double *d_xmod, const Cell &cell, int flags,
                             double *d_force, bool timing, double *h_acc)
{
    c->kt_n = 0;
    CK(kt_mark(c, nullptr));
    int rc = stage_positions(c, d_pos, d_xmod, cell, flags);
    if (rc) return rc;
    CK(kt_mark(c, "transpose_in"));
    rc = evaluate_enqueue(c, cell, flags, timing, h_acc);
    if (rc) return rc;
    CK(launch_transpose_out(c, d_force));
    CK(kt_mark(c, "transpose_out"));
    return PINYB200_OK;
}

// Positions into the internal [atom][xyz][bead] layout, the mode-1
// positions (given, or the bead centroid), and the device list update when
// flags ask for it; enqueued on c->stream.
int pinyb200::stage_positions(pinyb200_ctx *c, const double *d_pos, const double *d_xmod, const Cell &cell, int flags)
{
    CK(launch_transpose_in(c, d_pos));
    if (c->P > 1) {
        if (d_xmod == c->d_xmod) {
            // already in place
        } else if (d_xmod) {
            CK(cudaMemcpyAsync(c->d_xmod, d_xmod, (size_t)c->sys.natm * 3 * sizeof(double), cudaMemcpyDeviceToDevice,
                               c->stream));
        } else {
            const long long n = (long long)c->sys.natm * 3;
            centroid_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->d_posT, c->d_xmod, c->sys.natm, c->P);
            CK(cudaGetLastError());
        }
    }
    if (flags & PINYB200_UPDATE_LIST) {
        // PINY's list test (and rebuild) from these positions, on the device
        int rc = list_update_enqueue(c, d_pos, c->P > 1 ? c->d_xmod : nullptr, cell, c->stream);
        if (rc) return rc;
    }
    return PINYB200_OK;
}

// One evaluation enqueued through the context's cached CUDA graph.  A call
// whose key (pointers, stream, flags, cell, context generation) equals the
// previous call's replays one graph launch instead of ~15 kernel launches
// from the host: the first call with a key runs the work plainly (it sets
// kernel attributes and builds the influence function outside any
// capture), the second captures and launches it, later ones launch it.
// Per-kernel timing runs plainly.
static int run_eval_graph(pinyb200_ctx *c, const std::vector<double> &key, const std::function<int()> &body)
{
    if (c->kt_on || c->no_graph) return body();
    if (c->eg_exec && key == c->eg_key) {
        CK(cudaGraphLaunch(c->eg_exec, c->stream));
        return PINYB200_OK;
    }
    if (key != c->eg_seen) {
        c->eg_seen = key;
        return body();
    }
    if (c->eg_exec) cudaGraphExecDestroy(c->eg_exec);
    c->eg_exec = nullptr;
    c->eg_key.clear();
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = body();
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (ec != cudaSuccess) return fail(c, PINYB200_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
    const cudaError_t ei = cudaGraphInstantiate(&c->eg_exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        c->eg_exec = nullptr;
        return fail(c, PINYB200_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
    }
    c->eg_key = key;
    CK(cudaGraphLaunch(c->eg_exec, c->stream));
    return PINYB200_OK;
}

static std::vector<double> eval_key(pinyb200_ctx *c, int entry, const void *a, const void *b, const void *d,
                                    const double *hmat, int flags)
{
    std::vector<double> k = {(double)entry, (double)(uintptr_t)a, (double)(uintptr_t)b, (double)(uintptr_t)d,
                             (double)(uintptr_t)c->stream, (double)flags, (double)c->gen};
    for (int i = 0; i < 9; i++) k.push_back(hmat[i]);
    return k;
}

extern "C" {

int pinyb200_energy_force_device(pinyb200_ctx *c, const double *d_pos, const double *d_xmod, const double *hmat,
                                 int flags, double *d_force, pinyb200_energies *e, void *stream)
{
    if (!c || !d_pos || !hmat || !d_force) return fail(c, PINYB200_ERR_ARG, "energy_force_device: NULL argument");
    if (!c->have_list) return fail(c, PINYB200_ERR_STATE, "energy_force: build the Verlet list first");
    CK(cudaSetDevice(c->device));
    // launch on the caller's stream when one is given
    cudaStream_t own = c->stream;
    if (stream) c->stream = (cudaStream_t)stream;
    struct Restore {
        pinyb200_ctx *c;
        cudaStream_t s;
        ~Restore() { c->stream = s; }
    } restore{c, own};
    Cell cell = make_cell(hmat);
    const bool energy = !(flags & PINYB200_NO_ENERGY);
    if (energy && !c->h_acc_pin) CK(cudaMallocHost(&c->h_acc_pin, (size_t)c->P * S_NSLOT * sizeof(double)));
    double *acc = energy ? c->h_acc_pin : nullptr;  // pinned: the copy can sit in the graph
    int rc = run_eval_graph(c, eval_key(c, 1, d_pos, d_xmod, d_force, hmat, flags),
                            [&]() { return enqueue_device(c, d_pos, d_xmod, cell, flags, d_force, true, acc); });
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaEventElapsedTime(&c->last_ms[0], c->ev[0], c->ev[4]));
    CK(cudaEventElapsedTime(&c->last_ms[1], c->ev[1], c->ev[2]));
    CK(cudaEventElapsedTime(&c->last_ms[2], c->ev_pme[0], c->ev_pme[1]));
    CK(cudaEventElapsedTime(&c->last_ms[3], c->ev[2], c->ev[3]));
    evaluate_finish(c, cell, flags, acc, e);
    if (energy && e && !std::isfinite(e->vintert + e->vintrat))
        return fail(c, PINYB200_ERR_NAN, "non-finite energy: check the positions (forces were written)");
    return PINYB200_OK;
}

int pinyb200_energy_force(pinyb200_ctx *c, const double *pos, const double *xmod, const double *hmat, int flags,
                          double *force, pinyb200_energies *e)
{
    if (!c || !pos || !hmat || !force) return fail(c, PINYB200_ERR_ARG, "energy_force: NULL argument");
    if (!c->have_list) return fail(c, PINYB200_ERR_STATE, "energy_force: build the Verlet list first");
    CK(cudaSetDevice(c->device));
    const size_t nb = (size_t)c->sys.natm * 3 * c->P;
    CK(cudaEventRecord(c->ev[6], c->stream));
    CK(cudaMemcpyAsync(c->d_pos_aos, pos, nb * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (c->P > 1 && xmod)
        CK(cudaMemcpyAsync(c->d_xmod, xmod, (size_t)c->sys.natm * 3 * sizeof(double), cudaMemcpyHostToDevice,
                           c->stream));
    Cell cell = make_cell(hmat);
    // everything enqueued, one wait: the forces come back right behind the
    // evaluation; the device part replays the context's graph
    const bool energy = !(flags & PINYB200_NO_ENERGY);
    if (energy && !c->h_acc_pin) CK(cudaMallocHost(&c->h_acc_pin, (size_t)c->P * S_NSLOT * sizeof(double)));
    double *acc = energy ? c->h_acc_pin : nullptr;  // pinned: the copy is queued, not waited for
    int rc = run_eval_graph(c, eval_key(c, 2, c->d_pos_aos, xmod ? c->d_xmod : nullptr, c->d_force_aos, hmat, flags),
                            [&]() {
                                CK(launch_transpose_in(c, c->d_pos_aos));
                                if (c->P > 1 && !xmod) {
                                    const long long n = (long long)c->sys.natm * 3;
                                    centroid_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
                                        c->d_posT, c->d_xmod, c->sys.natm, c->P);
                                    CK(cudaGetLastError());
                                }
                                int r = evaluate_enqueue(c, cell, flags, true, acc);
                                if (r) return r;
                                CK(launch_transpose_out(c, c->d_force_aos));
                                return (int)PINYB200_OK;
                            });
    if (rc) return rc;
    CK(cudaMemcpyAsync(force, c->d_force_aos, nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaEventRecord(c->ev[7], c->stream));
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaEventElapsedTime(&c->last_ms[0], c->ev[0], c->ev[4]));
    CK(cudaEventElapsedTime(&c->last_ms[1], c->ev[1], c->ev[2]));
    CK(cudaEventElapsedTime(&c->last_ms[2], c->ev_pme[0], c->ev_pme[1]));
    CK(cudaEventElapsedTime(&c->last_ms[3], c->ev[2], c->ev[3]));
    CK(cudaEventElapsedTime(&c->last_ms[4], c->ev[6], c->ev[7]));
    evaluate_finish(c, cell, flags, acc, e);
    if (energy && e && !std::isfinite(e->vintert + e->vintrat))
        return fail(c, PINYB200_ERR_NAN, "non-finite energy: check the positions (forces were written)");
    return PINYB200_OK;
}

int pinyb200_piny_force(pinyb200_ctx *c, double *const *x, double *const *y, double *const *z, const double *xmod,
                        const double *ymod, const double *zmod, const double *hmat, double *const *fx,
                        double *const *fy, double *const *fz, double *pvten_tot, pinyb200_energies *e)
{
    if (!c || !x || !y || !z || !hmat || !fx || !fy || !fz) return fail(c, PINYB200_ERR_ARG, "piny_force: NULL");
    const int natm = c->sys.natm, P = c->P;
    std::vector<double> pos((size_t)P * natm * 3), frc(pos.size()), xm;
    for (int b = 0; b < P; b++)
        for (int i = 0; i < natm; i++) {
            pos[((size_t)b * natm + i) * 3 + 0] = x[b][i + 1];
            pos[((size_t)b * natm + i) * 3 + 1] = y[b][i + 1];
            pos[((size_t)b * natm + i) * 3 + 2] = z[b][i + 1];
        }
    if (P > 1 && xmod && ymod && zmod) {
        xm.resize((size_t)natm * 3);
        for (int i = 0; i < natm; i++) {
            xm[3 * i] = xmod[i + 1];
            xm[3 * i + 1] = ymod[i + 1];
            xm[3 * i + 2] = zmod[i + 1];
        }
    }
    double h[9];
    for (int k = 0; k < 9; k++) h[k] = hmat[k + 1];
    pinyb200_energies en;
    int rc = pinyb200_energy_force(c, pos.data(), xm.empty() ? nullptr : xm.data(), h, 0, frc.data(), &en);
    if (rc) return rc;
    for (int b = 0; b < P; b++)
        for (int i = 0; i < natm; i++) {
            fx[b][i + 1] += frc[((size_t)b * natm + i) * 3 + 0];
            fy[b][i + 1] += frc[((size_t)b * natm + i) * 3 + 1];
            fz[b][i + 1] += frc[((size_t)b * natm + i) * 3 + 2];
        }
    if (pvten_tot)
        for (int k = 0; k < 9; k++) pvten_tot[k + 1] += en.pvten[k];
    if (e) *e = en;
    return PINYB200_OK;
}

int pinyb200_count_list_device(pinyb200_ctx *c, const double *d_pos1, const double *d_xmod, const double *hmat,
                               const double *cutskin2, long *npairs, long *nactive, void *stream)
{
    if (!c || !d_pos1 || !hmat || !cutskin2) return fail(c, PINYB200_ERR_ARG, "count_list_device: NULL argument");
    if (c->sys.natm > PINYB200_COUNT_MAX_ATOMS)
        return fail(c, PINYB200_ERR_ARG,
                    "count_list_device: natm = " + std::to_string(c->sys.natm) +
                        " exceeds the fixed scratch limit PINYB200_COUNT_MAX_ATOMS = " +
                        std::to_string((int)PINYB200_COUNT_MAX_ATOMS) + "; use pinyb200_build_list");
    if (c->sys.npair_typ > PINYB200_COUNT_MAX_PAIR_TYPES)
        return fail(c, PINYB200_ERR_ARG,
                    "count_list_device: " + std::to_string(c->sys.npair_typ) +
                        " pair types exceed the fixed scratch limit PINYB200_COUNT_MAX_PAIR_TYPES = " +
                        std::to_string((int)PINYB200_COUNT_MAX_PAIR_TYPES));
    if (c->device < 0 || c->device >= kCountMaxDevices)
        return fail(c, PINYB200_ERR_UNSUPPORTED, "count_list_device: device ordinal beyond 63");
    CK(cudaSetDevice(c->device));
    unsigned char *base = nullptr;
    {
        // set-up, once per GPU, with that GPU current
        std::lock_guard<std::mutex> lock(g_count_mu);
        if (!g_count_addr[c->device]) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_count_scratch);
            if (e != cudaSuccess || !p)
                return fail(c, PINYB200_ERR_CUDA,
                            std::string("count_list_device: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_count_addr[c->device] = (unsigned char *)p;
        }
        base = g_count_addr[c->device];
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    unsigned long long *d_tot = (unsigned long long *)(base + kCountTotOff);
    double *d_cs = (double *)(base + kCountCutOff);
    int *d_cnt = (int *)(base + kCountRowOff);
    const Cell cell = make_cell(hmat);
    CK(cudaMemcpyAsync(d_cs, cutskin2, (size_t)c->sys.npair_typ * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(d_tot, 0, 2 * sizeof(unsigned long long), st));
    CK(launch_list_count(c, cell, d_pos1, d_xmod, d_cs, d_cnt, st));
    CK(launch_count_total(c, d_cnt, d_tot, st));
    unsigned long long tot[2] = {0, 0};
    CK(cudaMemcpyAsync(tot, d_tot, sizeof(tot), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (npairs) *npairs = (long)tot[0];
    if (nactive) *nactive = (long)tot[1];
    return PINYB200_OK;
}

int pinyb200_check_list_device(pinyb200_ctx *c, const double *d_pos, double spread_ref, int *rebuild,
                               double *rmax, double *spread_now, double *cutskin2, void *stream)
{
    if (!c || !d_pos) return fail(c, PINYB200_ERR_ARG, "check_list_device: NULL argument");
    if (!c->have_list) return fail(c, PINYB200_ERR_STATE, "check_list_device: no list built yet");
    CK(cudaSetDevice(c->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    unsigned long long *d_out = (unsigned long long *)(c->d_tot + 2);  // list totals slots, free after a build
    CK(cudaMemsetAsync(d_out, 0, 2 * sizeof(unsigned long long), st));
    CK(launch_list_check(c, d_pos, d_out, st));
    unsigned long long h[2];
    CK(cudaMemcpyAsync(h, d_out, sizeof(h), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double r2max, s2max;
    memcpy(&r2max, &h[0], sizeof(double));
    memcpy(&s2max, &h[1], sizeof(double));
    // check_ver_list (nbr_list_control.c:225-241) and get_cut_skin (:249-281)
    const double rm = sqrt(r2max);
    const double sp = c->P > 1 ? sqrt(s2max) : 0.0;
    double dspread = 0.0;
    if (c->P > 1) dspread = sp - spread_ref > 0.0 ? sp - spread_ref : 0.0;
    const double skin2 = c->skin / 2.0 + dspread;
    if (rebuild) *rebuild = rm > skin2 ? 1 : 0;
    if (rmax) *rmax = rm;
    if (spread_now) *spread_now = sp;
    if (cutskin2)
        for (int k = 0; k < c->sys.npair_typ; k++) {
            const double cs = c->h_cutoff[k] + c->skin + sp;
            cutskin2[k] = cs * cs;
        }
    return PINYB200_OK;
}

int pinyb200_list_info(pinyb200_ctx *c, long *npairs, long *nactive, long *capacity)
{
    if (!c) return fail(c, PINYB200_ERR_ARG, "list_info: NULL context");
    if (c->have_list) {
        CK(cudaSetDevice(c->device));
        if (int rc = list_sync_counts(c)) return rc;
    }
    if (npairs) *npairs = (long)c->npairs;
    if (nactive) *nactive = (long)c->nactive;
    if (capacity) *capacity = (long)c->list_cap;
    return c->have_list ? PINYB200_OK : fail(c, PINYB200_ERR_STATE, "no list built yet");
}

int pinyb200_set_kernel_timing(pinyb200_ctx *c, int on)
{
    if (!c) return fail(c, PINYB200_ERR_ARG, "set_kernel_timing: NULL");
    c->kt_on = on != 0;
    c->gen++;  // a captured graph holds no marks
    return PINYB200_OK;
}

int pinyb200_kernel_times(pinyb200_ctx *c, const char **names, float *ms, int cap, int *count)
{
    if (!c || !names || !ms || !count) return fail(c, PINYB200_ERR_ARG, "kernel_times: NULL");
    if (!c->kt_on) return fail(c, PINYB200_ERR_STATE, "kernel_times: per-kernel timing is off");
    CK(cudaSetDevice(c->device));
    *count = 0;
    for (int k = 1; k < c->kt_n && *count < cap; k++) {
        CK(cudaEventSynchronize(c->kt_ev[k]));
        CK(cudaEventElapsedTime(&ms[*count], c->kt_ev[k - 1], c->kt_ev[k]));
        names[*count] = c->kt_name[k];
        (*count)++;
    }
    return PINYB200_OK;
}

int pinyb200_last_timing(pinyb200_ctx *c, float *ms, int n)
{
    if (!c || !ms) return fail(c, PINYB200_ERR_ARG, "last_timing: NULL");
    for (int i = 0; i < n && i < 5; i++) ms[i] = c->last_ms[i];
    return PINYB200_OK;
}

}  // extern "C"
