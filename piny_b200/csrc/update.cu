// PINY's per-step Verlet list update entirely on the device: the rebuild
// test of check_ver_list (nbr_list_control.c:182-247) with the PIMD spread
// and get_cut_skin (:249-281), and, when the test fires, the list build of
// verlist_control (verlist_control.c:30-128) -- molecule-pair list, the
// site lists expanded from it, and the work chunks (or the site list alone
// for systems without such molecules) -- gated on the device flag, so a step needs no
// host round trip and can sit inside a CUDA graph.  The reserved capacities
// of the last host build bound the device builds; a build that would not
// fit sets a sticky flag, writes nothing past the reservation, and the pair
// kernel then poisons the energies (non-finite), so the next energy read
// fails loudly instead of a stale list being used.
#include <cstddef>

#include "common.cuh"

namespace pinyb200 {

__global__ void ls_begin_kernel(ListState *ls)
{
    ls->r2s2[0] = 0ull;
    ls->r2s2[1] = 0ull;
    ls->rebuild = 0;
}

// The decision, as pinyb200_check_list_device makes it on the host.
__global__ void ls_decide_kernel(ListState *ls, int P, double skin, int npt, const double *__restrict__ cutoff,
                                 double *__restrict__ cs)
{
    __shared__ int reb;
    __shared__ double sp_sh;
    if (threadIdx.x == 0) {
        const double rm = sqrt(__longlong_as_double((long long)ls->r2s2[0]));
        const double sp = P > 1 ? sqrt(__longlong_as_double((long long)ls->r2s2[1])) : 0.0;
        if (!ls->spread_set) {  // no reference yet: the current spread is it
            ls->spread_ref = sp;
            ls->spread_set = 1;
        }
        double dspread = 0.0;
        if (P > 1) dspread = sp - ls->spread_ref > 0.0 ? sp - ls->spread_ref : 0.0;
        const double skin2 = skin / 2.0 + dspread;
        reb = rm > skin2 ? 1 : 0;
        sp_sh = sp;
        ls->rmax = rm;
        ls->spread_now = sp;
        ls->rebuild = reb;
        if (reb) ls->spread_ref = sp;
    }
    __syncthreads();
    if (reb)
        for (int k = threadIdx.x; k < npt; k += blockDim.x) {
            const double c = cutoff[k] + skin + sp_sh;
            cs[k] = c * c;
        }
}

// Totals of the builds start from zero (the molecule fill adds into [3]).
__global__ void ls_prep_kernel(const int *gate, long long *tot, long long *chunk_tot)
{
    if (*gate == 0) return;
    for (int k = 0; k < 4; k++) tot[k] = 0;
    *chunk_tot = 0;
}

// Chunks per molecule row: rows cut into pieces of ch molecule pairs.
__global__ void ls_chunk_count_kernel(const int *gate, int nmol, const int *__restrict__ mrow, int ch,
                                      int *__restrict__ nch)
{
    if (*gate == 0) return;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < nmol; m += gridDim.x * blockDim.x)
        nch[m] = (mrow[m + 1] - mrow[m] + ch - 1) / ch;
}

__global__ void ls_chunk_fill_kernel(const int *gate, int nmol, const int *__restrict__ mrow, int ch,
                                     const int *__restrict__ nch, const int *__restrict__ crow,
                                     int *__restrict__ chunk, long long cap)
{
    if (*gate == 0) return;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < nmol; m += gridDim.x * blockDim.x) {
        const int r0 = mrow[m], r1 = mrow[m + 1];
        for (int q = 0; q < nch[m]; q++) {
            const long long idx = (long long)crow[m] + q;
            if (idx >= cap) break;
            const int b = r0 + q * ch;
            chunk[3 * idx] = m;
            chunk[3 * idx + 1] = b;
            chunk[3 * idx + 2] = b + ch < r1 ? b + ch : r1;
        }
    }
}

__global__ void ls_finish_kernel(const int *gate, ListState *ls, const long long *__restrict__ tot,
                                 const long long *__restrict__ chunk_tot, long long list_cap, long long mlist_cap,
                                 long long chunk_cap, int use_mol, int *__restrict__ nchunk)
{
    if (*gate == 0) return;
    ls->site_tot[0] = tot[0];
    ls->site_tot[1] = tot[1];
    int over = tot[0] > list_cap || tot[1] > list_cap;
    if (use_mol) {
        ls->mol_tot[0] = tot[2];
        ls->mol_tot[1] = tot[3];
        over |= tot[2] > mlist_cap || *chunk_tot > chunk_cap;
        if (tot[3] != tot[1]) ls->mismatch = 1;
        *nchunk = (int)(*chunk_tot < chunk_cap ? *chunk_tot : chunk_cap);
    }
    if (over) ls->overflow = 1;
    ls->rebuilds += 1;
}

// After an overflow the row pointers may reach past the reserved lists:
// empty every row so that no consumer reads beyond them.
__global__ void ls_clear_rows_kernel(const int *gate, const ListState *ls, int natm, int *row, int *rowA, int nmol,
                                     int *mrow)
{
    if (*gate == 0 || !ls->overflow) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= natm; i += gridDim.x * blockDim.x) {
        row[i] = 0;
        rowA[i] = 0;
    }
    if (mrow)
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= nmol; i += gridDim.x * blockDim.x) mrow[i] = 0;
}

__global__ void ls_copy_kernel(const int *gate, const double *__restrict__ src, double *__restrict__ dst, long long n)
{
    if (*gate == 0) return;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

int list_update_prepare(pinyb200_ctx *c)
{
    if (c->d_ls) return PINYB200_OK;
    cudaError_t e = cudaMalloc(&c->d_ls, sizeof(ListState));
    if (e == cudaSuccess) e = cudaMemset(c->d_ls, 0, sizeof(ListState));
    if (e == cudaSuccess) e = cudaMalloc(&c->d_cs, sizeof(double) * (size_t)c->sys.npair_typ);
    if (e == cudaSuccess && c->nmol > 0) e = cudaMalloc(&c->d_mchunk, sizeof(int) * (2 * (size_t)c->nmol + 1));
    if (e == cudaSuccess && c->use_mol && !c->d_reach) e = cudaMalloc(&c->d_reach, sizeof(double));
    if (e != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, std::string("list update: ") + cudaGetErrorString(e));
    return PINYB200_OK;
}

// Enqueue the update on st.  d_pos: [P][natm][3] with current ghost
// positions; d_xm: mode-1 positions (nullptr for one bead).
int list_update_enqueue(pinyb200_ctx *c, const double *d_pos, const double *d_xm, const Cell &cell, cudaStream_t st)
{
    int rc = list_update_prepare(c);
    if (rc) return rc;
    ListState *ls = c->d_ls;
    const int *gate = (const int *)((const char *)ls + offsetof(ListState, rebuild));
    long long *chunk_tot = (long long *)((char *)c->d_tot + 0) + 4;  // slot after the four list totals
    const int natm = c->sys.natm;
    cudaError_t e;
    ls_begin_kernel<<<1, 1, 0, st>>>(ls);
    if ((e = launch_list_check(c, d_pos, (unsigned long long *)((char *)ls + offsetof(ListState, r2s2)), st)) != cudaSuccess)
        return record_error(c, PINYB200_ERR_CUDA, cudaGetErrorString(e));
    ls_decide_kernel<<<1, 64, 0, st>>>(ls, c->P, c->skin, c->sys.npair_typ, c->sys.cutoff, c->d_cs);
    ls_prep_kernel<<<1, 1, 0, st>>>(gate, c->d_tot, chunk_tot);
    const double *xm = c->P > 1 ? d_xm : nullptr;
    const bool mol = c->use_mol && c->d_mj && c->d_chunk && c->d_nchunk;
    if (mol) {
        // molecule-pair list, the site lists expanded from its masks, chunks
        if ((e = launch_mol_list(c, cell, d_pos, xm, c->d_cs, 0, gate, st)) != cudaSuccess ||
            (e = launch_mol_list(c, cell, d_pos, xm, c->d_cs, 1, gate, st)) != cudaSuccess ||
            (e = launch_site_from_mol(c, 0, gate, st)) != cudaSuccess ||
            (e = launch_site_from_mol(c, 1, gate, st)) != cudaSuccess)
            return record_error(c, PINYB200_ERR_CUDA, cudaGetErrorString(e));
        const int jpi = c->P >= 32 ? 1 : 32 / c->P;
        const int ch = PINYB200_MOL_CHUNK * jpi;
        const int blocks = (c->nmol + 255) / 256;
        ls_chunk_count_kernel<<<blocks, 256, 0, st>>>(gate, c->nmol, c->d_mrow, ch, c->d_mchunk);
        if ((e = launch_scan(c, gate, c->nmol, 1, c->d_mchunk, c->d_mchunk + c->nmol, nullptr, chunk_tot, st)) !=
            cudaSuccess)
            return record_error(c, PINYB200_ERR_CUDA, cudaGetErrorString(e));
        ls_chunk_fill_kernel<<<blocks, 256, 0, st>>>(gate, c->nmol, c->d_mrow, ch, c->d_mchunk,
                                                     c->d_mchunk + c->nmol, c->d_chunk, c->chunk_cap);
    } else if ((e = launch_build_list(c, cell, d_pos, xm, c->d_cs, 0, gate, st)) != cudaSuccess ||
               (e = launch_build_list(c, cell, d_pos, xm, c->d_cs, 1, gate, st)) != cudaSuccess) {
        return record_error(c, PINYB200_ERR_CUDA, cudaGetErrorString(e));
    }
    ls_finish_kernel<<<1, 1, 0, st>>>(gate, ls, c->d_tot, chunk_tot, c->list_cap, c->mlist_cap, c->chunk_cap,
                                      mol ? 1 : 0, c->d_nchunk);
    ls_clear_rows_kernel<<<(natm + 256) / 256, 256, 0, st>>>(gate, ls, natm, c->d_row, c->d_rowA, c->nmol,
                                                              mol ? c->d_mrow : nullptr);
    const long long n = (long long)natm * 3;
    ls_copy_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(gate, d_pos, c->d_x0, n);
    if ((e = launch_keep_build_state(c, gate, d_pos, xm, c->d_cs, st)) != cudaSuccess)
        return record_error(c, PINYB200_ERR_CUDA, cudaGetErrorString(e));
    if (c->respa_on)
        if ((rc = respa_list_enqueue(c, cell, gate, st))) return rc;
    if ((e = cudaGetLastError()) != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, cudaGetErrorString(e));
    return PINYB200_OK;
}

// A host build replaces the list: clear the sticky flags of device builds.
int list_reset_flags(pinyb200_ctx *c)
{
    if (!c->d_ls) return PINYB200_OK;
    const int zero[2] = {0, 0};
    cudaError_t e = cudaMemcpy((char *)c->d_ls + offsetof(ListState, overflow), zero, sizeof(zero),
                               cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, cudaGetErrorString(e));
    return PINYB200_OK;
}

// Host copies of the list sizes after device rebuilds (waits for the
// context's stream).
int list_sync_counts(pinyb200_ctx *c)
{
    if (!c->d_ls) return PINYB200_OK;
    ListState h;
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = cudaMemcpy(&h, c->d_ls, sizeof(h), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, cudaGetErrorString(e));
    if (h.overflow) {  // the rows were emptied
        c->npairs = c->nactive = c->nmp = 0;
    } else if (h.rebuilds > 0) {
        c->npairs = h.site_tot[0];
        c->nactive = h.site_tot[1];
        c->nmp = h.mol_tot[0];
    }
    return PINYB200_OK;
}

}  // namespace pinyb200

using namespace pinyb200;

extern "C" {

int pinyb200_update_list_device(pinyb200_ctx *c, const double *d_pos, const double *d_xmod, const double *hmat,
                                void *stream)
{
    if (!c || !d_pos || !hmat) return record_error(c, PINYB200_ERR_ARG, "update_list_device: NULL argument");
    if (!c->have_list) return record_error(c, PINYB200_ERR_STATE, "update_list_device: build the list once first");
    if (c->P > 1 && !d_xmod) return record_error(c, PINYB200_ERR_ARG, "update_list_device: mode-1 positions needed");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, cudaGetErrorString(e));
    return list_update_enqueue(c, d_pos, d_xmod, cell_from_hmat(hmat), stream ? (cudaStream_t)stream : c->stream);
}

int pinyb200_list_set_spread(pinyb200_ctx *c, double spread_ref)
{
    if (!c) return record_error(c, PINYB200_ERR_ARG, "list_set_spread: NULL context");
    int rc = list_update_prepare(c);
    if (rc) return rc;
    const int one = 1;
    cudaError_t e = cudaMemcpy((char *)c->d_ls + offsetof(ListState, spread_ref), &spread_ref, sizeof(double),
                               cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy((char *)c->d_ls + offsetof(ListState, spread_set), &one, sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, cudaGetErrorString(e));
    return PINYB200_OK;
}

int pinyb200_list_status(pinyb200_ctx *c, void *stream, pinyb200_list_state *out)
{
    if (!c || !out) return record_error(c, PINYB200_ERR_ARG, "list_status: NULL argument");
    int rc = list_update_prepare(c);
    if (rc) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    ListState h;
    cudaError_t e = cudaMemcpyAsync(&h, c->d_ls, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, cudaGetErrorString(e));
    out->rebuilds = (long)h.rebuilds;
    out->rebuilt_last = h.rebuild;
    out->overflow = h.overflow;
    out->mismatch = h.mismatch;
    out->rmax = h.rmax;
    out->spread_now = h.spread_now;
    out->spread_ref = h.spread_ref;
    if (h.rebuilds > 0) {
        out->npairs = (long)h.site_tot[0];
        out->nactive = (long)h.site_tot[1];
        out->nmol_pairs = (long)h.mol_tot[0];
        // host copies follow the device list from here on
        c->npairs = h.site_tot[0];
        c->nactive = h.site_tot[1];
        c->nmp = h.mol_tot[0];
    } else {
        out->npairs = (long)c->npairs;
        out->nactive = (long)c->nactive;
        out->nmol_pairs = (long)c->nmp;
    }
    return (h.overflow || h.mismatch) ? record_error(c, PINYB200_ERR_LIST_OVERFLOW,
                                                     h.overflow ? "device list update: list outgrew its reservation"
                                                                : "device list update: molecule masks disagree")
                                      : PINYB200_OK;
}

}  // extern "C"
