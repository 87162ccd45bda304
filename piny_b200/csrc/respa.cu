// PINY's RESPA split of the force path (respa_steps_lrf / _intra / _pimd).
//
// int_NVT_pimd (int_NVT_pimd.c:142-223) nests inter, torsion, intra and bead
// RESPA loops and asks the force routines for one level per inner step
// through energy_ctrl's iget_full_inter / iget_res_inter / iget_full_intra /
// iget_res_intra (:175-189).  Each term carries the number of inner steps its
// impulse spans (energy_control_initial.c:211-243):
//   real space   outer level: x (swit wght_ter_res + (1 - swit) wght_ter),
//                or x wght_ter without inter RESPA; inner inter level:
//                shave at cutoff_res, x swit wght_ter_res (force_npol.c)
//   PME, ecor    outer level only, x wght_ter (energy_control_inter_recip.c)
//   bonds        inter levels: bond_both, wght_tra_res F_res + w (F - F_res);
//                intra levels: bond() x wght_tra_res at the RESPA equilibrium
//                when nres_tra nres_tor > 1 (energy_control_intra.c:116-140)
//   bends        x wght_tra_res at every intra level (bend.c)
// The outer level also yields the unweighted forces PINY adds to the virial
// forces fxt, its energies and pvten_tot: that is the plain evaluation, run
// into the context's force buffer, while the weighted forces go to a second
// buffer ([atom][xyz][bead] like the first).
#include <cmath>
#include <cstddef>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace pinyb200 {

// RESPA pair list (PINY's jter_res, verlist_create.c:409-491): the active
// pairs whose bead-1 separation at the list build lies within
// cutskin_res = min(cutoff_res + skin + spread, cutskin) (nbr_list_control.c:
// 265-275), i.e. cutoff_res plus the build's own cutskin - cutoff.  One warp
// per row i; separations as the list build forms them.
template <int FILL>
__global__ void __launch_bounds__(256) respa_list_kernel(const int *__restrict__ gate, int natm, int ntyp,
                                                         const double *__restrict__ pos1,
                                                         const double *__restrict__ xm, int use_xm, Cell cell,
                                                         const double *__restrict__ cs,
                                                         const double *__restrict__ cutoff,
                                                         const double *__restrict__ cut_res,
                                                         const int *__restrict__ atm_typ,
                                                         const int *__restrict__ rowA, const int *__restrict__ colA,
                                                         int *__restrict__ count, const int *__restrict__ rowR,
                                                         int *__restrict__ colR, long long cap)
{
    if (gate && *gate == 0) return;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < natm; i += nwarps) {
        const double xi = pos1[3 * i], yi = pos1[3 * i + 1], zi = pos1[3 * i + 2];
        double xmi = 0, ymi = 0, zmi = 0;
        if (use_xm) { xmi = xm[3 * i]; ymi = xm[3 * i + 1]; zmi = xm[3 * i + 2]; }
        const int ti = atm_typ[i];
        const int beg = rowA[i], end = rowA[i + 1];
        const long long w = FILL ? rowR[i] : 0;
        int n = 0;
        for (int jj0 = beg; jj0 < end; jj0 += 32) {
            const int jj = jj0 + lane;
            bool keep = false;
            int j = 0;
            if (jj < end) {
                j = colA[jj];
                double dx = __dsub_rn(xi, pos1[3 * j]);
                double dy = __dsub_rn(yi, pos1[3 * j + 1]);
                double dz = __dsub_rn(zi, pos1[3 * j + 2]);
                if (use_xm)
                    period_pimd_exact(dx, dy, dz, __dsub_rn(xmi, xm[3 * j]), __dsub_rn(ymi, xm[3 * j + 1]),
                                      __dsub_rn(zmi, xm[3 * j + 2]), cell);
                else
                    period_exact(dx, dy, dz, cell);
                const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                const int pt = pair_type(ti, atm_typ[j], ntyp);
                const double margin = fmax(sqrt(cs[pt]) - cutoff[pt], 0.0);
                const double cr = fmin(cut_res[pt] + margin, sqrt(cs[pt]));
                keep = r2 < cr * cr;
            }
            const unsigned b = __ballot_sync(0xffffffffu, keep);
            if (FILL && keep) {
                const long long p = w + n + __popc(b & ((1u << lane) - 1u));
                if (p < cap) colR[p] = j;
            }
            n += __popc(b);
        }
        if (!FILL && lane == 0) {
            count[i] = n;
        }
    }
}

__global__ void keep_build_state_kernel(const int *gate, const double *__restrict__ xm, double *__restrict__ xm0,
                                        long long n, const double *__restrict__ cs, double *__restrict__ cs0, int npt)
{
    if (gate && *gate == 0) return;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        xm0[i] = xm[i];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) cs0[i] = cs[i];
}

__global__ void scale_copy_kernel(const double *__restrict__ src, double w, double *__restrict__ dst, long long n)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) dst[t] = src[t] * w;
}

cudaError_t launch_keep_build_state(pinyb200_ctx *c, const int *gate, const double *d_pos1, const double *d_xm,
                                    const double *d_cs, cudaStream_t st)
{
    (void)d_pos1;  // bead-1 positions are kept in d_x0 by the list build itself
    if (!c->d_xm0 || !c->d_cs0) return cudaSuccess;
    const long long n = d_xm ? (long long)c->sys.natm * 3 : 0;
    keep_build_state_kernel<<<(unsigned)((n + 255) / 256 + 1), 256, 0, st>>>(gate, d_xm, c->d_xm0, n, d_cs, c->d_cs0,
                                                                             c->sys.npair_typ);
    return cudaGetLastError();
}

cudaError_t launch_respa_scale_copy(pinyb200_ctx *c, double w, double *target)
{
    const long long n = (long long)c->sys.natm * 3 * c->P;
    scale_copy_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->d_forceT, w, target, n);
    return cudaGetLastError();
}

// Count, scan and fill of the RESPA list on st (gated like a device build).
int respa_list_enqueue(pinyb200_ctx *c, const Cell &cell, const int *gate, cudaStream_t st)
{
    if (!c->respa_on || !c->d_rowR || !c->d_colR) return PINYB200_OK;
    const DeviceSystem &s = c->sys;
    const int threads = 256;
    const int blocks = (int)(((long long)s.natm * 32 + threads - 1) / threads);
    const bool use_xm = c->P > 1;
    respa_list_kernel<0><<<blocks, threads, 0, st>>>(gate, s.natm, s.ntyp, c->d_x0, c->d_xm0, use_xm, cell, c->d_cs0,
                                                     s.cutoff, c->d_cut_res, s.atm_typ, c->d_rowA, c->d_colA,
                                                     c->d_count, nullptr, nullptr, 0);
    cudaError_t e = launch_scan(c, gate, s.natm, 1, c->d_count, c->d_rowR, nullptr, c->d_rtot, st);
    if (e != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, cudaGetErrorString(e));
    respa_list_kernel<1><<<blocks, threads, 0, st>>>(gate, s.natm, s.ntyp, c->d_x0, c->d_xm0, use_xm, cell, c->d_cs0,
                                                     s.cutoff, c->d_cut_res, s.atm_typ, c->d_rowA, c->d_colA,
                                                     nullptr, c->d_rowR, c->d_colR, c->res_cap);
    e = cudaGetLastError();
    if (e != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, cudaGetErrorString(e));
    return PINYB200_OK;
}

// RESPA list storage for the current list capacity, and the list itself
// from the state of the last list build (host side, outside graphs).
int respa_list_reserve(pinyb200_ctx *c, const Cell &cell)
{
    if (!c->d_rowR) {
        cudaError_t e = cudaMalloc(&c->d_rowR, ((size_t)c->sys.natm + 1) * sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc(&c->d_rtot, 2 * sizeof(long long));
        if (e != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, cudaGetErrorString(e));
    }
    if (c->res_cap < c->list_cap || !c->d_colR) {
        if (c->d_colR) cudaFree(c->d_colR);
        c->d_colR = nullptr;
        c->res_cap = 0;
        cudaError_t e = cudaMalloc(&c->d_colR, (size_t)c->list_cap * sizeof(int));
        if (e != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, cudaGetErrorString(e));
        c->res_cap = c->list_cap;
    }
    return respa_list_enqueue(c, cell, nullptr, c->stream);
}

}  // namespace pinyb200

using namespace pinyb200;

namespace {

int check_level(pinyb200_ctx *c, int level)
{
    const int intra = PINYB200_FULL_INTRA | PINYB200_RES_INTRA;
    const int outer = PINYB200_FULL_INTER | PINYB200_FULL_INTRA | (c->r_int_res_ter ? PINYB200_RES_INTER : 0);
    // the outer level with or without RES_INTRA: PINY's first call sets it
    // only with intra RESPA (control_pimd.c:297-306); the forces agree
    const bool ok = level == PINYB200_RES_INTRA || level == intra ||
                    (level == (PINYB200_RES_INTER | intra) && c->r_int_res_ter) || level == outer ||
                    level == (outer | PINYB200_RES_INTRA);
    if (ok) return PINYB200_OK;
    return record_error(c, PINYB200_ERR_ARG,
                        "respa_force: level " + std::to_string(level) +
                            " is not one PINY's RESPA loops set (int_res_ter = " + std::to_string(c->r_int_res_ter) +
                            ")");
}

#define RK(x)                                                                          \
    do {                                                                               \
        cudaError_t e_ = (x);                                                          \
        if (e_ != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, cudaGetErrorString(e_)); \
    } while (0)

}  // namespace

// One level, enqueued on c->stream; the weighted forces end in c->d_forceW,
// the outer level's unweighted ones in c->d_forceT (and its per-bead sums
// are copied to h_acc).  The outer level is the plain evaluation with the
// weighted buffer formed alongside (evaluate_enqueue); the inner levels run
// only their own terms.
int pinyb200::respa_level_enqueue(pinyb200_ctx *c, const Cell &cell, int level, int flags, double *h_acc)
{
    if (level & PINYB200_FULL_INTER) return evaluate_enqueue(c, cell, flags, false, h_acc, c->d_forceW);
    const size_t nb = (size_t)c->sys.natm * 3 * c->P;
    const bool inter = level & PINYB200_RES_INTER;
    RK(launch_ghost_pos(c));
    RK(cudaMemsetAsync(c->d_forceW, 0, nb * sizeof(double), c->stream));
    if (inter) RK(launch_pair_respa(c, cell, 1, c->d_forceW));
    if (inter && c->r_kres) {
        // reciprocal-space RESPA: the reciprocal sum (on the one mesh, or
        // on PINY's separate RESPA mesh) and the exclusion correction
        // (RESPA table) belong to this level
        const bool mesh_res = c->pme_res.on;
        if (mesh_res) pme_swap(c, c->pme_res);
        cudaError_t e = launch_pme(c, cell, false);
        if (e == cudaSuccess) e = launch_pme_force_add_scaled(c, c->r_wter_res, c->d_forceW);
        if (mesh_res) pme_swap(c, c->pme_res);
        RK(e);
        RK(launch_ecor_weighted(c, c->r_wter_res, c->d_forceW, 1));
    }
    RK(launch_intra_respa(c, inter, c->d_forceW));
    if (flags & PINYB200_DISTRIB_GHOSTS) RK(launch_ghost_distrib(c, c->d_forceW));
    return PINYB200_OK;
}

namespace {

// The list update's sticky failure flags (a device rebuild that did not fit)
int check_list_flags(pinyb200_ctx *c)
{
    if (!c->d_ls) return PINYB200_OK;
    int fl[2] = {0, 0};
    RK(cudaMemcpy(fl, (const char *)c->d_ls + offsetof(ListState, overflow), sizeof(fl), cudaMemcpyDeviceToHost));
    if (fl[0] | fl[1])
        return record_error(c, PINYB200_ERR_LIST_OVERFLOW,
                            "respa_force: a device list rebuild exceeded the reserved list; rebuild on the host");
    return PINYB200_OK;
}

}  // namespace

extern "C" {

int pinyb200_set_respa(pinyb200_ctx *c, const pinyb200_respa *r)
{
    if (!c) return record_error(c, PINYB200_ERR_ARG, "set_respa: NULL context");
    RK(cudaSetDevice(c->device));
    if (!r) {
        c->respa_on = false;
        return PINYB200_OK;
    }
    const bool mesh_res = r->nktot_res > 0 && r->pme_res_on;
    if (mesh_res) {
        if (!r->kastr_res || !r->kbstr_res || !r->kcstr_res || !r->bweight_res)
            return record_error(c, PINYB200_ERR_ARG, "set_respa: RESPA PME mesh k vectors / weights missing");
        for (int d = 0; d < 3; d++)
            if (r->ngrid_res[d] < r->n_interp_res || r->ngrid_res[d] > 256)
                return record_error(c, PINYB200_ERR_ARG, "set_respa: RESPA PME mesh size out of range");
        if (r->n_interp_res < 4 || r->n_interp_res > 10)
            return record_error(c, PINYB200_ERR_UNSUPPORTED, "set_respa: RESPA PME order outside 4..10");
        for (int i = 0; i < r->nktot_res; i++) {
            const int k[3] = {r->kastr_res[i], r->kbstr_res[i], r->kcstr_res[i]};
            for (int d = 0; d < 3; d++)
                if (2 * abs(k[d]) >= r->ngrid_res[d])
                    return record_error(c, PINYB200_ERR_ARG, "set_respa: RESPA k vector beyond its PME mesh");
        }
    }
    if (r->nktot_res > 0 && c->sys.necor > 0 && !r->ecor_cdv0_res)
        return record_error(c, PINYB200_ERR_ARG, "set_respa: ecor_cdv0_res missing (nktot_res > 0)");
    if (!r->cutoff_res || (c->sys.nbond && !r->bond_eq_res))
        return record_error(c, PINYB200_ERR_ARG, "set_respa: cutoff_res / bond_eq_res missing");
    if (!(r->rheal_res > 0.0)) return record_error(c, PINYB200_ERR_ARG, "set_respa: rheal_res must be > 0");
    if (!(r->wght_ter >= 1.0 && r->wght_ter_res >= 1.0 && r->wght_tra_res >= 1.0))
        return record_error(c, PINYB200_ERR_ARG, "set_respa: RESPA weights are step counts (>= 1)");
    const int npt = c->sys.npair_typ;
    for (int k = 0; k < npt; k++)
        if (!(r->cutoff_res[k] > 0.0) || r->cutoff_res[k] > c->h_cutoff[k])
            return record_error(c, PINYB200_ERR_ARG, "set_respa: cutoff_res must lie in (0, cutoff]");
    if (!c->d_cut_res) RK(cudaMalloc(&c->d_cut_res, (size_t)npt * sizeof(double)));
    RK(cudaMemcpy(c->d_cut_res, r->cutoff_res, (size_t)npt * sizeof(double), cudaMemcpyHostToDevice));
    if (c->sys.nbond) {
        if (!c->d_bond_eq_res) RK(cudaMalloc(&c->d_bond_eq_res, (size_t)c->nbond_typ * sizeof(double)));
        RK(cudaMemcpy(c->d_bond_eq_res, r->bond_eq_res, (size_t)c->nbond_typ * sizeof(double),
                      cudaMemcpyHostToDevice));
    }
    if (!c->d_forceW) RK(cudaMalloc(&c->d_forceW, (size_t)c->sys.natm * 3 * c->P * sizeof(double)));
    c->r_kres = r->nktot_res > 0 ? 1 : 0;
    if (mesh_res && c->sys.nchrg > 0) {
        if (int rc = pme_res_setup(c, r->ngrid_res, r->n_interp_res, r->nktot_res, r->kastr_res, r->kbstr_res,
                                   r->kcstr_res, r->bweight_res))
            return rc;
    } else {
        pme_res_free(c);
    }
    if (c->r_kres && c->sys.necor > 0) {
        std::vector<double> coef;
        table_coefs(r->ecor_cdv0_res, c->sys.ecor_nsplin, coef);
        if (!c->d_ecor_res_tab) RK(cudaMalloc(&c->d_ecor_res_tab, coef.size() * sizeof(double)));
        RK(cudaMemcpy(c->d_ecor_res_tab, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    if (c->have_list && !c->build_cell_ok)
        return record_error(c, PINYB200_ERR_STATE, "set_respa: the list build state is missing");
    c->r_wter = r->wght_ter;
    c->r_wter_res = r->wght_ter_res;
    c->r_wtra_res = r->wght_tra_res;
    c->r_int_res_ter = r->int_res_ter ? 1 : 0;
    c->r_int_res_inter = r->int_res_inter ? 1 : 0;
    c->r_ires_bond = r->ires_bond ? 1 : 0;
    c->r_rheal = r->rheal_res;
    c->respa_on = true;
    c->gen++;  // captured graphs must pick up the RESPA list build
    if (c->have_list) {
        // the RESPA list of the current Verlet list, from its build state
        int rc = respa_list_reserve(c, c->build_cell);
        if (rc) return rc;
        RK(cudaStreamSynchronize(c->stream));
    }
    return PINYB200_OK;
}

int pinyb200_respa_force_device(pinyb200_ctx *c, const double *d_pos, const double *d_xmod, const double *hmat,
                                int level, int flags, double *d_force, double *d_forcet, pinyb200_energies *e,
                                void *stream)
{
    if (!c || !d_pos || !hmat || !d_force) return record_error(c, PINYB200_ERR_ARG, "respa_force: NULL argument");
    if (!c->have_list) return record_error(c, PINYB200_ERR_STATE, "respa_force: build the Verlet list first");
    if (!c->respa_on) return record_error(c, PINYB200_ERR_STATE, "respa_force: pinyb200_set_respa first");
    if (int rc = check_level(c, level)) return rc;
    RK(cudaSetDevice(c->device));
    cudaStream_t own = c->stream;
    if (stream) c->stream = (cudaStream_t)stream;
    struct Restore {
        pinyb200_ctx *c;
        cudaStream_t s;
        ~Restore() { c->stream = s; }
    } restore{c, own};
    const Cell cell = cell_from_hmat(hmat);
    const bool outer = level & PINYB200_FULL_INTER;
    const bool energy = outer && !(flags & PINYB200_NO_ENERGY);
    std::vector<double> acc(outer ? (size_t)c->P * S_NSLOT : 0);
    int rc = stage_positions(c, d_pos, d_xmod, cell, flags);
    if (rc) return rc;
    rc = respa_level_enqueue(c, cell, level, flags, outer ? acc.data() : nullptr);
    if (rc) return rc;
    RK(launch_transpose_out(c, d_force, c->d_forceW));
    if (outer && d_forcet) RK(launch_transpose_out(c, d_forcet, c->d_forceT));
    RK(cudaStreamSynchronize(c->stream));
    if (int rc2 = check_list_flags(c)) return rc2;
    if (e) {
        if (energy) {
            evaluate_finish(c, cell, flags, acc.data(), e);
            if (!std::isfinite(e->vintert + e->vintrat))
                return record_error(c, PINYB200_ERR_NAN, "non-finite energy: check the positions");
        } else {
            memset(e, 0, sizeof(*e));
        }
    }
    return PINYB200_OK;
}

int pinyb200_piny_force_respa(pinyb200_ctx *c, int level, double *const *x, double *const *y, double *const *z,
                              const double *xmod, const double *ymod, const double *zmod, const double *hmat,
                              double *const *fx, double *const *fy, double *const *fz, double *const *fxt,
                              double *const *fyt, double *const *fzt, double *pvten_tot, pinyb200_energies *e)
{
    if (!c || !x || !y || !z || !hmat || !fx || !fy || !fz)
        return record_error(c, PINYB200_ERR_ARG, "piny_force_respa: NULL argument");
    const int natm = c->sys.natm, P = c->P;
    const size_t nb = (size_t)P * natm * 3;
    std::vector<double> pos(nb), frc(nb), frt;
    for (int b = 0; b < P; b++)
        for (int i = 0; i < natm; i++) {
            pos[((size_t)b * natm + i) * 3 + 0] = x[b][i + 1];
            pos[((size_t)b * natm + i) * 3 + 1] = y[b][i + 1];
            pos[((size_t)b * natm + i) * 3 + 2] = z[b][i + 1];
        }
    RK(cudaSetDevice(c->device));
    const bool outer = level & PINYB200_FULL_INTER;
    const bool want_t = outer && fxt && fyt && fzt;
    if (want_t && !c->d_forcet_aos) RK(cudaMalloc(&c->d_forcet_aos, nb * sizeof(double)));
    double *d_xm = nullptr;
    if (P > 1 && xmod && ymod && zmod) {
        std::vector<double> xm((size_t)natm * 3);
        for (int i = 0; i < natm; i++) {
            xm[3 * i] = xmod[i + 1];
            xm[3 * i + 1] = ymod[i + 1];
            xm[3 * i + 2] = zmod[i + 1];
        }
        // the mode-1 positions go straight to the context's own buffer
        RK(cudaMemcpy(c->d_xmod, xm.data(), xm.size() * sizeof(double), cudaMemcpyHostToDevice));
        d_xm = c->d_xmod;
    }
    RK(cudaMemcpy(c->d_pos_aos, pos.data(), nb * sizeof(double), cudaMemcpyHostToDevice));
    double h[9];
    for (int k = 0; k < 9; k++) h[k] = hmat[k + 1];
    pinyb200_energies en;
    int rc = pinyb200_respa_force_device(c, c->d_pos_aos, d_xm, h, level, 0, c->d_force_aos,
                                         want_t ? c->d_forcet_aos : nullptr, &en, nullptr);
    if (rc) return rc;
    RK(cudaMemcpy(frc.data(), c->d_force_aos, nb * sizeof(double), cudaMemcpyDeviceToHost));
    if (want_t) {
        frt.resize(nb);
        RK(cudaMemcpy(frt.data(), c->d_forcet_aos, nb * sizeof(double), cudaMemcpyDeviceToHost));
    }
    for (int b = 0; b < P; b++)
        for (int i = 0; i < natm; i++) {
            const size_t o = ((size_t)b * natm + i) * 3;
            fx[b][i + 1] += frc[o];
            fy[b][i + 1] += frc[o + 1];
            fz[b][i + 1] += frc[o + 2];
            if (want_t) {
                fxt[b][i + 1] += frt[o];
                fyt[b][i + 1] += frt[o + 1];
                fzt[b][i + 1] += frt[o + 2];
            }
        }
    if (outer && pvten_tot)
        for (int k = 0; k < 9; k++) pvten_tot[k + 1] += en.pvten[k];
    if (e) *e = en;
    return PINYB200_OK;
}

}  // extern "C"
