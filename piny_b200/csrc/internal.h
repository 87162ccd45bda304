// Internal state and launchers of the pinyb200 library (not part of the ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/pinyb200.h"

namespace pinyb200 {

// Per-bead accumulator slots (FP64).
enum Slot {
    S_VVDW = 0,   // real-space vdW energy
    S_VCOUL,      // real-space Ewald energy
    S_VRECIP,     // PME reciprocal energy
    S_VECOR,      // Ewald exclusion correction
    S_VBOND,
    S_VBEND,
    S_PXX, S_PYY, S_PZZ, S_PXY, S_PXZ, S_PYZ,  // bead pressure tensor
    S_EXT = 15,   // bead 0 only: molecule extent bound of the evaluation (bits of a double >= 0)
    S_NSLOT = 16
};

// Cell passed by value to kernels: h column-major, hi = h^-1 (gethinv).
struct Cell {
    double h[9];
    double hi[9];
    double vol;
    int cubic;
};

// Table kinds in the coefficient arrays.
enum TabKind { T_CV0 = 0, T_CDV0 = 1, T_CV0C = 2, T_CDV0C = 3 };

// Molecule pairs per warp chunk of the molecule-pair kernel (per lane group
// when P < 32): the i sites are loaded and their forces flushed once per chunk.
#ifndef PINYB200_MOL_CHUNK
#define PINYB200_MOL_CHUNK 8
#endif

// Device state of the list update (pinyb200_update_list_device).
struct ListState {
    int rebuild;                   // this step's decision (gates the build kernels)
    int overflow;                  // a build needed more room than reserved (sticky)
    int mismatch;                  // molecule masks and active site list disagree (sticky)
    int spread_set;                // spread_ref holds a value
    double spread_ref;             // bead spread at the last build (PINY interact.spread)
    double spread_now, rmax;
    unsigned long long r2s2[2];    // max displacement^2, max spread^2 (bit patterns)
    long long rebuilds;            // builds done on the device
    long long site_tot[2];         // full, active site pairs of the last build
    long long mol_tot[2];          // molecule pairs, site pairs in their masks
};

struct DeviceSystem {
    int natm, ntyp, npair_typ, nsplin, nuniq;
    int *atm_typ = nullptr;
    double *charge = nullptr;
    int *inter_map = nullptr;       // [npair_typ]
    double *cutoff = nullptr;       // [npair_typ]
    double *rmin = nullptr, *dr = nullptr, *dri = nullptr;  // [nuniq]
    int *has_vdw = nullptr;         // [nuniq]
    double4 *tab64 = nullptr;       // [4][nuniq][nsplin] cubic coefficients
    float4 *tab32 = nullptr;
    int *excl_off = nullptr, *excl_j = nullptr;
    int nchrg;
    int *ichrg = nullptr;           // charged atoms
    // PME
    int ngrid[3];
    int n_interp;
    int nktot;
    int *kvec = nullptr;            // [nktot][3]
    double *bweight = nullptr;
    int *kmask = nullptr;           // [G] -> index into kvec or -1
    // ecor / bonds / bends / ghosts
    int necor, ecor_nsplin;
    int *ecor_j1 = nullptr, *ecor_j2 = nullptr;
    double ecor_rmin, ecor_dr, ecor_dri;
    double4 *ecor_tab = nullptr;    // [2][ecor_nsplin]  cv0, cdv0 coefficients
    int nbond;
    int *bond_j = nullptr;          // [nbond][3] j1, j2, typ
    double *bond_eq = nullptr, *bond_c = nullptr, *bond_dc = nullptr;
    int nbend;
    int *bend_j = nullptr;          // [nbend][4] j1, j2, j3, typ
    double *bend_c = nullptr, *bend_s = nullptr, *bend_dc = nullptr, *bend_ds = nullptr;
    int nghost, ghost_ncomp;
    int *ghost_atom = nullptr, *ghost_comp = nullptr;
    double *ghost_coef = nullptr;
};

// Parameter derivatives (tangent channels) for the adjoint.  Channel k
// holds the derivative of the set-up data with respect to one parameter;
// absent parts are NULL.
#define PINYB200_MAX_TAN 16
struct GradChan {
    const double *dq;        // [natm] d charge
    const void *ttab;        // [2][nuniq][nsplin] cubic coefficients of d cv0, d cdv0 (double4 / float4)
    const double *dcoef;     // [nghost][ncomp] d ghost coefficient
    double *w;               // [natm][3][P] d site position (ghost rows), filled on the device
    const double *bond_deq;  // [nbond_typ] d equilibrium length
    const double *bond_dc;   // [nbond_typ][7] d power-series coefficients
    const double *bend_c, *bend_s, *bend_dc, *bend_ds;  // [nbend_typ][7] d bend series
};
struct GradArgs {
    int K;
    GradChan ch[PINYB200_MAX_TAN];
    const double *uT;        // [natm][3][P] adjoint of the raw site forces
    double *gacc;            // [K][2] FP64 sums: energy derivative, force contraction
};
// host copies of the tangent data (owned by the context)
struct GradHost {
    int K = 0;
    std::vector<void *> dev;  // every device allocation of the tangents
    GradChan ch[PINYB200_MAX_TAN];
    double dq_dot_q[PINYB200_MAX_TAN];  // sum_i q_i dq_i
    double dq_sum[PINYB200_MAX_TAN];    // sum_i dq_i
    double dclong[PINYB200_MAX_TAN];
    double *d_u = nullptr;              // [natm][3][P]
    double *d_gacc = nullptr;           // [K][2]
    void *d_grid2 = nullptr;            // PME: dipole spread of u, then its convolution
};

cudaError_t launch_pme_adjoint(pinyb200_ctx *c, const Cell &cell, const GradArgs &g);
cudaError_t launch_grad_terms(pinyb200_ctx *c, const Cell &cell, const GradArgs &g, const double *d_fbar);

}  // namespace pinyb200

// State of one PME mesh.  The evaluation's mesh lives in the context's own
// fields (sys.ngrid..., d_grid...); PINY's separate RESPA mesh (pme_res_on)
// is held here and swapped into those fields while its kernels are
// enqueued (pme_swap), so every PME launcher serves both.
struct PmeSet {
    bool on = false;
    int ngrid[3] = {0, 0, 0}, n_interp = 0, nktot = 0;
    int *kvec = nullptr, *kmask = nullptr;
    double *bweight = nullptr;
    void *d_grid = nullptr, *d_spec = nullptr, *d_filter = nullptr;
    double *d_forceP = nullptr;
    int pme_tile = 16, pme_nt[3] = {0, 0, 0}, pme_ntile = 0, pme_cap = 0;
    int *d_pme_cnt = nullptr, *d_pme_bin = nullptr, *d_pme_ovf = nullptr;
    void *d_pme_head = nullptr, *d_pme_w = nullptr;
    double *d_twiddle64 = nullptr;
    float *d_twiddle32 = nullptr;
    bool filter_ok = false;
    double filter_h[9] = {0};
};

struct pinyb200_ctx {
    int device = 0;
    int precision = PINYB200_FP64;
    int P = 1;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    cudaStream_t pme_stream = nullptr;  // PME runs here, concurrently with the pair kernel
    bool pme_overlap = true;            // false: PME on the main stream after the pair kernel
    int pair_variant = 0;               // 0 molecule-pair kernel (when available), 1 site-list kernel
    int pair_blocks_per_sm = 16;        // grid cap of the pair kernels, blocks per SM
    bool pme_full_records = false;      // forward PME writes the full weight records (the adjoint reads them)
    int pair_carveout = 25;             // shared-memory share (%) the MIXED molecule-pair kernel asks for
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_pme[2] = {nullptr, nullptr};
    pinyb200::DeviceSystem sys;
    // host copies needed for energy bookkeeping
    std::vector<double> h_charge;
    std::vector<double> h_cutoff;  // per type pair (Bohr)
    double skin = 0;               // Verlet skin (Bohr)
    int nbond_typ = 0, nbend_typ = 0;
    double alp_ewd = 0, self_erf = 1, clong = 0;
    int iswit_vdw = 1;
    // Verlet list: full (parity) and active (force) CSR by i, j < i
    long list_cap = 0;
    long npairs = 0, nactive = 0;
    int *d_row = nullptr, *d_col = nullptr;        // full
    int *d_rowA = nullptr, *d_colA = nullptr;      // active
    int *d_count = nullptr;                        // [2*natm] scratch
    long long *d_tot = nullptr;                    // device totals [4]
    bool have_list = false;
    // molecule-pair list (sites grouped into molecules of <= 4 consecutive sites)
    bool use_mol = false;      // the system splits into such molecules
    int mol_stride = 0;        // sites per molecule when molecule m starts at site m * mol_stride, else 0
    // MIXED molecule-pair kernel with unrolled site pairs: usable when every
    // site pair of the molecule shares one cutoff and spline grid
    bool mix_ok = false;
    int mix_toff[16] = {0}, mix_eflag[16] = {0};
    float mix_q2[16] = {0};
    float4 *d_tabfe = nullptr;  // [2][nuniq][nsplin][2] vdW / Coulomb force and energy rows side by side
    float mix_rc2 = 0, mix_dri = 0, mix_rmd = 0, mix_tmax = 0;
    bool mol_ok = false;       // the current molecule list matches the site list
    int nmol = 0, mol_ns = 0;
    int *d_mstart = nullptr;   // [nmol+1]
    int *d_mcount = nullptr;   // [nmol]
    int *d_mrow = nullptr;     // [nmol+1]
    int *d_mj = nullptr;       // [nmp]
    unsigned *d_mmask = nullptr;   // active site pairs of each molecule pair
    unsigned *d_mmaskf = nullptr;  // all site pairs (PINY's list) of each molecule pair
    double *d_reach = nullptr;     // list build: reach of the molecule bound
    float4 *d_msf = nullptr;    // [nmol] wrapped fractional site-0 bead-1 positions (FP32)
    int4 *d_ent = nullptr;      // [ent_cap] molecule pairs found by the count pass (fill by scatter)
    long long ent_cap = 0;
    unsigned long long *d_nent = nullptr;  // [1] pairs the count pass found
    unsigned long long *d_reach_acc = nullptr;  // [4] reach maxima (bit patterns) and blocks done, kept zero
    long long *d_scan_part = nullptr;  // [scan_part_cap] tile sums of the device-wide scans
    long long scan_part_cap = 0;
    // link cells of the molecule-pair list build, planned at each host build
    int list_method = 0;        // PINYB200_LIST_LNK or PINYB200_LIST_NOLST
    int cell_n[3] = {0, 0, 0};  // cells along a, b, c (each >= 5); 0: every build sweeps
    int cell_cap = 0;           // cells the buffers below hold
    int *d_mcell = nullptr;     // [nmol] cell of each molecule
    int *d_ccnt = nullptr;      // [2][cell_cap] molecules per cell, scatter counters
    int *d_coff = nullptr;      // [cell_cap + 1] first molecule of each cell in d_cmol
    int *d_cmol = nullptr;      // [2][nmol] molecules in cell order: arrival, then sorted
    int *d_cellok = nullptr;    // [1] the cells serve the current build
    long long *d_ctot = nullptr;  // [1] scan total
    long long mlist_cap = 0, nmp = 0;
    int nchunk = 0;
    int *d_chunk = nullptr;    // [chunk_cap][3]
    long long chunk_cap = 0;
    int *d_nchunk = nullptr;   // device copy of the chunk count (the pair kernel reads it)
    // device list update (pinyb200_update_list_device)
    pinyb200::ListState *d_ls = nullptr;
    double *d_cs = nullptr;    // [npair_typ] cutskin^2 of the last device decision
    int *d_mchunk = nullptr;   // [nmol] chunks per molecule row, then [nmol + 1] offsets
    // work buffers
    double *d_posT = nullptr;     // [natm][3][P]
    double *d_forceT = nullptr;   // [natm][3][P]
    double *d_xmod = nullptr;     // [natm][3]
    double *d_x0 = nullptr;       // [natm][3] bead-1 positions at the last list build
    double *d_pos_aos = nullptr;  // [P][natm][3] staging for host calls
    double *d_force_aos = nullptr;
    double *d_acc = nullptr;      // [P][S_NSLOT]
    void *d_grid = nullptr;       // [P][Nc][Nb][Na] real charge / potential grid
    void *d_spec = nullptr;       // [P][Nc][Nb][Na/2+1] complex half spectrum
    void *d_filter = nullptr;     // [G] real: preg * bweight, 0 outside the sphere
    double *d_forceP = nullptr;   // [nchrg][3][P] PME forces, added to d_forceT after the join
    // charges binned by PME grid tile (pme_tile = 8 or 16 points per edge)
    int pme_tile = 16;
    int pme_nt[3] = {0, 0, 0};    // tiles per axis
    int pme_ntile = 0, pme_cap = 0;
    int *d_pme_cnt = nullptr;     // [P][ntile] entries per bin, then [1] overflow count
    int *d_pme_bin = nullptr;     // [P][ntile][cap] charge numbers (index into ichrg)
    int *d_pme_ovf = nullptr;     // [nchrg*P] overflowing (charge, bead) as k*P + b
    void *d_pme_head = nullptr;   // [nchrg*P] int4 stencil origin records
    void *d_pme_w = nullptr;      // [nchrg*P][6][NIP] B-spline weight records
    double *d_twiddle64 = nullptr;  // per axis twiddles
    float *d_twiddle32 = nullptr;
    int *d_err = nullptr;
    double filter_h[9] = {0};     // cell the filter was built for
    bool filter_ok = false;
    cudaEvent_t ev[8];
    float last_ms[5] = {0, 0, 0, 0, 0};
    // per-kernel timing (pinyb200_set_kernel_timing): an event after every
    // kernel of a serialised evaluation, named by the kernel it closes
    // cached CUDA graph of one evaluation (the single-box entry points)
    cudaGraphExec_t eg_exec = nullptr;
    std::vector<double> eg_key, eg_seen;
    bool no_graph = false;
    bool kt_on = false;
    int kt_n = 0;
    std::vector<cudaEvent_t> kt_ev;
    std::vector<const char *> kt_name;
    // bumped whenever launch shapes or device buffers may change (list
    // builds, tuning, PME tiles): captured graphs compare it before replay
    unsigned long long gen = 0;
    double *h_acc_pin = nullptr;  // pinned per-bead sums of the host-buffer call
    // RESPA split (pinyb200_set_respa): PINY's weights and switches
    bool respa_on = false;
    double r_wter = 1, r_wter_res = 1, r_wtra_res = 1, r_rheal = 1;
    int r_int_res_ter = 0, r_int_res_inter = 0, r_ires_bond = 0;
    int r_kres = 0;                   // reciprocal-space RESPA on one grid (nktot_res > 0)
    PmeSet pme_res;                   // PINY's separate RESPA PME mesh (pme_res_on), when on
    double *d_ecor_res_tab = nullptr; // [ecor_nsplin][4] cubic coefficients of ecor.cdv0_res
    double *d_cut_res = nullptr;      // [npair_typ] inner cutoffs (Bohr)
    double *d_bond_eq_res = nullptr;  // [nbond_typ] RESPA bond equilibria
    double *d_forceW = nullptr;       // [natm][3][P] weighted forces of one level
    double *d_forcet_aos = nullptr;   // [P][natm][3] staging of the virial forces
    int *d_rowR = nullptr, *d_colR = nullptr;  // RESPA pair list (CSR by i, j < i), capacity res_cap
    long long res_cap = 0;
    long long *d_rtot = nullptr;      // [2] RESPA list totals
    double *d_xm0 = nullptr;          // [natm][3] mode-1 positions at the last list build
    double *d_cs0 = nullptr;          // [npair_typ] cutskin^2 of the last list build
    double *d_cs_in = nullptr;        // [npair_typ] cutskin^2 passed to the current host list build
    pinyb200::Cell build_cell{};      // cell of the last host list build
    bool build_cell_ok = false;
    pinyb200::GradHost grad;      // tangent channels of pinyb200_grad_prepare
    std::string err;
};

namespace pinyb200 {

// launchers (defined in the .cu files)
// gate: device flag, 0 = skip (the device list update); st: nullptr = the
// context's stream
cudaError_t launch_build_list(pinyb200_ctx *c, const Cell &cell, const double *d_pos1,
                              const double *d_xm, const double *d_cutskin2, int pass, const int *gate = nullptr,
                              cudaStream_t st = nullptr);
cudaError_t launch_pair(pinyb200_ctx *c, const Cell &cell, bool energy);
cudaError_t launch_pair_respa(pinyb200_ctx *c, const Cell &cell, int mode, double *target);
cudaError_t launch_intra_respa(pinyb200_ctx *c, bool both, double *target);
cudaError_t launch_ecor_weighted(pinyb200_ctx *c, double w, double *target, int table = 0);
cudaError_t launch_pme_force_add_scaled(pinyb200_ctx *c, double w, double *target);
cudaError_t launch_mol_list(pinyb200_ctx *c, const Cell &cell, const double *d_pos1, const double *d_xm,
                            const double *d_cutskin2, int pass, const int *gate = nullptr,
                            cudaStream_t st = nullptr);
int mol_cells_plan(pinyb200_ctx *c, const Cell &cell, const double *d_pos1, const double *d_cutskin2);
// Exclusive prefix sums of K (1 or 2) arrays of n counts at count + k n into
// out_k[0..n] (out_k[n] the total) and tot[k]; uses c->d_scan_part.
int scan_tiles(int n);
cudaError_t launch_scan(pinyb200_ctx *c, const int *gate, int n, int K, const int *count, int *out0, int *out1,
                        long long *tot, cudaStream_t st);
cudaError_t launch_mol_pair(pinyb200_ctx *c, const Cell &cell, bool energy);
cudaError_t launch_mol_pair_mixed(pinyb200_ctx *c, const Cell &cell, bool energy);
cudaError_t launch_site_from_mol(pinyb200_ctx *c, int pass, const int *gate = nullptr, cudaStream_t st = nullptr);
cudaError_t launch_pme(pinyb200_ctx *c, const Cell &cell, bool energy);
cudaError_t launch_pme_force_add(pinyb200_ctx *c);

// evaluation steps (capi.cu): device work of one evaluation enqueued on
// c->stream without host synchronisation, and the host bookkeeping of its
// per-bead sums; cell of an hmat; error recording
int evaluate_enqueue(pinyb200_ctx *c, const Cell &cell, int flags, bool timing, double *h_acc,
                     double *respa_w = nullptr);
// RESPA pair list: the active pairs within cutoff_res + skin + spread at the
// last list build (PINY's jter_res), rebuilt with every list build
int respa_list_enqueue(pinyb200_ctx *c, const Cell &cell, const int *gate, cudaStream_t st);
int respa_list_reserve(pinyb200_ctx *c, const Cell &cell);
// one RESPA level on c->stream (see respa.cu); PINYB200_* level bits
int respa_level_enqueue(pinyb200_ctx *c, const Cell &cell, int level, int flags, double *h_acc);
cudaError_t launch_respa_scale_copy(pinyb200_ctx *c, double w, double *target);
// bead-1 and mode-1 positions and cutskin^2 of a list build, kept for the
// RESPA list (gated like the build on the device)
cudaError_t launch_keep_build_state(pinyb200_ctx *c, const int *gate, const double *d_pos1, const double *d_xm,
                                    const double *d_cs, cudaStream_t st);
int stage_positions(pinyb200_ctx *c, const double *d_pos, const double *d_xmod, const Cell &cell, int flags);
void evaluate_finish(pinyb200_ctx *c, const Cell &cell, int flags, const double *acc, pinyb200_energies *e);
int enqueue_device(pinyb200_ctx *c, const double *d_pos, const double *d_xmod, const Cell &cell, int flags,
                   double *d_force, bool timing, double *h_acc);
Cell cell_from_hmat(const double *hmat);
int pme_tiles_resize(pinyb200_ctx *c, int T);
void pme_swap(pinyb200_ctx *c, PmeSet &p);
int pme_res_setup(pinyb200_ctx *c, const int *ngrid, int n_interp, int nktot, const int *kastr, const int *kbstr,
                  const int *kcstr, const double *bweight);
void pme_res_free(pinyb200_ctx *c);
void table_coefs(const double *t, int nsplin, std::vector<double> &out);

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) once per kernel, device
// and size, so that repeated launches (and graph captures) do not repeat it.
inline cudaError_t smem_optin(const void *func, int bytes)
{
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, int> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    int &have = done[std::make_pair(func, dev)];
    if (have >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) have = bytes;
    return e;
}
// Timing event that stays a real event record when the stream is being
// captured into a graph (an external event node), so the phase times of a
// graph replay are measured as those of a plain run.
inline cudaError_t ev_rec(cudaEvent_t e, cudaStream_t s)
{
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    cudaError_t err = cudaStreamIsCapturing(s, &st);
    if (err != cudaSuccess) return err;
    return cudaEventRecordWithFlags(e, s, st == cudaStreamCaptureStatusActive ? cudaEventRecordExternal
                                                                              : cudaEventRecordDefault);
}

// Per-kernel timing mark: with kt_on, an event on c->stream closing the
// kernel `name` (the first mark, name nullptr, opens the evaluation).
inline cudaError_t kt_mark(pinyb200_ctx *c, const char *name)
{
    if (!c->kt_on) return cudaSuccess;
    if (c->kt_n >= (int)c->kt_ev.size()) {
        cudaEvent_t e;
        cudaError_t err = cudaEventCreate(&e);
        if (err != cudaSuccess) return err;
        c->kt_ev.push_back(e);
        c->kt_name.push_back(nullptr);
    }
    c->kt_name[c->kt_n] = name;
    return cudaEventRecord(c->kt_ev[c->kt_n++], c->stream);
}

// cudaFuncSetAttribute(PreferredSharedMemoryCarveout) once per kernel and
// device: a kernel that gathers from tables held in L1 asks for a small
// shared-memory share, leaving the rest of the unified cache to L1.
inline cudaError_t carveout_pref(const void *func, int percent)
{
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, int> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    int &have = done[std::make_pair(func, dev)];
    if (have == percent + 1) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributePreferredSharedMemoryCarveout, percent);
    if (e == cudaSuccess) have = percent + 1;
    return e;
}
int record_error(pinyb200_ctx *c, int code, const std::string &msg);
cudaError_t launch_intra(pinyb200_ctx *c, const Cell &cell, bool energy);
cudaError_t launch_ghost_pos(pinyb200_ctx *c);
cudaError_t launch_ghost_distrib(pinyb200_ctx *c, double *fT = nullptr);
cudaError_t launch_transpose_in(pinyb200_ctx *c, const double *d_pos_aos);
cudaError_t launch_transpose_out(pinyb200_ctx *c, double *d_force_aos, const double *fT = nullptr);
cudaError_t launch_list_count(pinyb200_ctx *c, const Cell &cell, const double *d_pos1, const double *d_xm,
                              const double *d_cutskin2, int *d_count, cudaStream_t st);
cudaError_t launch_list_check(pinyb200_ctx *c, const double *d_pos, unsigned long long *d_out, cudaStream_t st);
// device list update (update.cu)
int list_update_prepare(pinyb200_ctx *c);
int list_update_enqueue(pinyb200_ctx *c, const double *d_pos, const double *d_xm, const Cell &cell, cudaStream_t st);
int list_sync_counts(pinyb200_ctx *c);
int list_reset_flags(pinyb200_ctx *c);
cudaError_t launch_count_total(pinyb200_ctx *c, const int *d_count, unsigned long long *d_tot, cudaStream_t st);
size_t pme_plane_smem(int Na, int Nb, bool fp64);
size_t pme_slab_smem(int Na, int Nc, bool fp64);

}  // namespace pinyb200

namespace pinyb200 {
// Batched launches over many boxes: one persistent kernel per group of
// boxes that share a kernel's compile-time shape (boxtab.cuh).
int mix_pattern(const pinyb200_ctx *c);
cudaError_t launch_mol_extent(pinyb200_ctx *c);
cudaError_t launch_mol_extent_batch(const std::vector<pinyb200_ctx *> &box, int sm_count, cudaStream_t st);
cudaError_t launch_mol_pair_mixed_batch(const std::vector<pinyb200_ctx *> &box, const std::vector<Cell> &cells,
                                        bool energy, int sm_count, cudaStream_t st);
cudaError_t launch_pme_batch(const std::vector<pinyb200_ctx *> &box, const std::vector<Cell> &cells, bool energy,
                             int sm_count, cudaStream_t st);
cudaError_t launch_pme_force_add_batch(const std::vector<pinyb200_ctx *> &box, int sm_count, cudaStream_t st);
// zero byte ranges (pointer, bytes; 4-byte multiples) in one launch
cudaError_t launch_zero_batch(const std::vector<std::pair<void *, size_t>> &seg, int sm_count, cudaStream_t st);
// copies of n doubles src -> dst (device or pinned host memory); src null:
// dst = the bead centroid of posT [n][P]
struct CopySeg {
    const double *src;
    const double *posT;
    double *dst;
    long long n;
    int P;
};
cudaError_t launch_copy_batch(const std::vector<CopySeg> &seg, int sm_count, cudaStream_t st);
cudaError_t launch_transpose_in_batch(const std::vector<pinyb200_ctx *> &box, const std::vector<const double *> &d_pos,
                                      int sm_count, cudaStream_t st);
cudaError_t launch_transpose_out_batch(const std::vector<pinyb200_ctx *> &box, const std::vector<double *> &d_force,
                                       int sm_count, cudaStream_t st);
cudaError_t launch_ghost_batch(const std::vector<pinyb200_ctx *> &box, bool distrib, int sm_count, cudaStream_t st);
cudaError_t launch_intra_batch(const std::vector<pinyb200_ctx *> &box, bool energy, int sm_count, cudaStream_t st);
}  // namespace pinyb200
