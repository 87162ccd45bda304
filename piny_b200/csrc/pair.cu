// Real-space pair forces for all beads over the shared Verlet list.
//
// Restates force_npol (src/energy/inter/real_space/force_npol.c:28-329):
// per listed pair and bead the minimum-image separation (period / period_pimd
// with the mode-1 image shift, :829-871), the shave r < cutoff (:1291-1390),
// the spline index k = clamp((int)((r - rmin) dri + 0.5) + 3, 3, nsplin-2)
// with del = (r - r_k) dri (:685-819), and the 4-point cubic of the vdW and
// Ewald real-space tables (npol_vspl_fetch, :339-375):
//   F_ij = d_ij [S(cdv0) + q_i q_j S(cdv0_c)],  V = S(cv0) + q_i q_j S(cv0_c).
// The cubic's interval coefficients are formed once on the host with PINY's
// expressions, so each evaluation reads one 4-vector per table.
//
// B200 mapping: one warp per atom row i; lanes are (neighbour slot, bead)
// with the bead fastest, so the 32 beads of one neighbour j are one
// coalesced 256-byte load of the [atom][xyz][bead] position array.  The
// row's force on i stays in FP64 registers and is reduced with warp
// shuffles; the reaction on j is one coalesced FP64 red.add per component.
// MIXED: separations are formed in FP64 (positions and image shift), the
// rest of the pair arithmetic is FP32, every accumulation is FP64.
#include <cstddef>

#include "common.cuh"

namespace pinyb200 {

struct PairArgs {
    const int *row, *col;
    int natm, ntyp, nsplin, nuniq;
    const double *posT, *xmod;
    int use_xmod;
    const int *atm_typ;
    const double *charge;
    const int *inter_map;
    const double *cutoff, *rmin, *dr, *dri;
    const int *has_vdw;
    const void *tab;
    double *forceT;
    double *acc;
    int energy;
    const int *bad;  // device flags (overflow, mismatch) of the list update, or nullptr
    // RESPA split (force_npol.c:805-816, :1030-1060), over the RESPA pair
    // list and shaved at cut_res: 0 off; 1 inner level, force x swit w_res;
    // 2 the outer level's switched part, force x swit (w_res - w_full),
    // added to w_full times the plain forces (PINY's multiplier
    // swit w_res + (1 - swit) w_full).  swit = 1 - 3 br^2 + 2 br^3 with
    // br = clamp((r - cut_res + rheal) / rheal, 0, 1).
    int respa;
    const double *cut_res;
    double rheal, rheali, w_res, w_full;
};

template <typename R, int P, bool RSP>
__global__ void __launch_bounds__(256) pair_kernel(PairArgs a, Cell cell)
{
    if (a.bad && (a.bad[0] | a.bad[1])) {
        // the list update could not hold the new list: fail loudly
        if (blockIdx.x == 0 && threadIdx.x == 0) a.acc[S_VVDW] = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    typedef typename Vec4<R>::T V;
    constexpr int JPI = P >= 32 ? 1 : 32 / P;  // neighbours per warp step
    constexpr int BPL = P >= 32 ? P / 32 : 1;  // beads per lane
    const V *__restrict__ tab = (const V *)a.tab;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int jsub = P >= 32 ? 0 : lane / P;
    const int b0 = P >= 32 ? lane : lane % P;
    const int nsm2 = a.nsplin - 2;
    const double *__restrict__ posT = a.posT;

    double ev[BPL], ec[BPL], pv[BPL][6];
#pragma unroll
    for (int s = 0; s < BPL; s++) {
        ev[s] = ec[s] = 0.0;
#pragma unroll
        for (int c = 0; c < 6; c++) pv[s][c] = 0.0;
    }

    for (int i = warp; i < a.natm; i += nwarps) {
        const int beg = a.row[i], end = a.row[i + 1];
        if (beg == end) continue;
        const int ti = a.atm_typ[i];
        const double qi = a.charge[i];
        double xi[BPL][3], fi[BPL][3];
#pragma unroll
        for (int s = 0; s < BPL; s++)
#pragma unroll
            for (int d = 0; d < 3; d++) {
                xi[s][d] = posT[(3 * (size_t)i + d) * P + b0 + 32 * s];
                fi[s][d] = 0.0;
            }
        double xmi = 0, ymi = 0, zmi = 0;
        if (a.use_xmod) { xmi = a.xmod[3 * i]; ymi = a.xmod[3 * i + 1]; zmi = a.xmod[3 * i + 2]; }

        for (int jj = beg + jsub; jj < end; jj += JPI) {
            const int j = a.col[jj];
            const int pt = pair_type(ti, a.atm_typ[j], a.ntyp);
            const int u = a.inter_map[pt];
            const R rc = (R)(RSP ? a.cut_res[pt] : a.cutoff[pt]);
            const R rmin = (R)a.rmin[u], dr = (R)a.dr[u], dri = (R)a.dri[u];
            const int vdw = a.has_vdw[u];
            const R q2 = (R)(qi * a.charge[j]);
            double shx = 0, shy = 0, shz = 0;
            if (a.use_xmod) {
                // the image shift is the same for every bead (period_pimd)
                period_pimd_exact(shx, shy, shz, __dsub_rn(xmi, a.xmod[3 * j]), __dsub_rn(ymi, a.xmod[3 * j + 1]),
                                  __dsub_rn(zmi, a.xmod[3 * j + 2]), cell);
            }
            const V *tF = tab + ((size_t)T_CDV0C * a.nuniq + u) * a.nsplin;
            const V *tV = tab + ((size_t)T_CDV0 * a.nuniq + u) * a.nsplin;
            const V *eF = tab + ((size_t)T_CV0C * a.nuniq + u) * a.nsplin;
            const V *eV = tab + ((size_t)T_CV0 * a.nuniq + u) * a.nsplin;
#pragma unroll
            for (int s = 0; s < BPL; s++) {
                const int b = b0 + 32 * s;
                double dx = __dsub_rn(xi[s][0], posT[(3 * (size_t)j + 0) * P + b]);
                double dy = __dsub_rn(xi[s][1], posT[(3 * (size_t)j + 1) * P + b]);
                double dz = __dsub_rn(xi[s][2], posT[(3 * (size_t)j + 2) * P + b]);
                if (a.use_xmod) {
                    dx = __dadd_rn(dx, shx);
                    dy = __dadd_rn(dy, shy);
                    dz = __dadd_rn(dz, shz);
                } else {
                    period_exact(dx, dy, dz, cell);
                }
                const R rx = (R)dx, ry = (R)dy, rz = (R)dz;
                const R r = Idx<R>::dist(rx, ry, rz);
                if (!(r < rc)) continue;
                R del;
                const int k = Idx<R>::knot(r, rmin, dr, dri, nsm2, del);
                R dv = q2 * spline_eval<V, R>(ldg4(tF + (k - 1)), del);
                if (vdw) dv += spline_eval<V, R>(ldg4(tV + (k - 1)), del);
                R fx = rx * dv, fy = ry * dv, fz = rz * dv;
                if (RSP) {
                    R br = (r - rc + (R)a.rheal) * (R)a.rheali;
                    br = br > (R)0 ? br : (R)0;
                    br = br < (R)1 ? br : (R)1;
                    const R swit = br * br * (br * (R)2 - (R)3) + (R)1;
                    const R fm = a.respa == 1 ? swit * (R)a.w_res : swit * (R)(a.w_res - a.w_full);
                    fx *= fm;
                    fy *= fm;
                    fz *= fm;
                }
                fi[s][0] += (double)fx;
                fi[s][1] += (double)fy;
                fi[s][2] += (double)fz;
                atomicAdd(&a.forceT[(3 * (size_t)j + 0) * P + b], -(double)fx);
                atomicAdd(&a.forceT[(3 * (size_t)j + 1) * P + b], -(double)fy);
                atomicAdd(&a.forceT[(3 * (size_t)j + 2) * P + b], -(double)fz);
                if (a.energy) {
                    ec[s] += (double)(q2 * spline_eval<V, R>(ldg4(eF + (k - 1)), del));
                    if (vdw) ev[s] += (double)spline_eval<V, R>(ldg4(eV + (k - 1)), del);
                    pv[s][0] += (double)(rx * fx);
                    pv[s][1] += (double)(ry * fy);
                    pv[s][2] += (double)(rz * fz);
                    pv[s][3] += (double)(rx * fy);
                    pv[s][4] += (double)(rx * fz);
                    pv[s][5] += (double)(ry * fz);
                }
            }
        }
        // force on i: sum lanes that hold the same bead
#pragma unroll
        for (int s = 0; s < BPL; s++)
#pragma unroll
            for (int d = 0; d < 3; d++) {
                double v = fi[s][d];
                if (P < 32) v = warp_sum_strided(v, P);
                if (P >= 32 || lane < P) atomicAdd(&a.forceT[(3 * (size_t)i + d) * P + b0 + 32 * s], v);
            }
    }
    if (a.energy) {
#pragma unroll
        for (int s = 0; s < BPL; s++) {
            double v[8] = {ev[s], ec[s], pv[s][0], pv[s][1], pv[s][2], pv[s][3], pv[s][4], pv[s][5]};
            const int slot[8] = {S_VVDW, S_VCOUL, S_PXX, S_PYY, S_PZZ, S_PXY, S_PXZ, S_PYZ};
#pragma unroll
            for (int c = 0; c < 8; c++) {
                double t = v[c];
                if (P < 32) t = warp_sum_strided(t, P);
                if (P >= 32 || lane < P) atomicAdd(&a.acc[(size_t)(b0 + 32 * s) * S_NSLOT + slot[c]], t);
            }
        }
    }
}

template <typename R, int P, bool RSP>
static void launch_pair_t(pinyb200_ctx *c, const PairArgs &a, const Cell &cell)
{
    const int threads = 256;
    long long rows = c->sys.natm;
    long long blocks = (rows * 32 + threads - 1) / threads;
    long long maxb = (long long)c->sm_count * c->pair_blocks_per_sm;
    if (blocks > maxb) blocks = maxb;
    pair_kernel<R, P, RSP><<<(int)blocks, threads, 0, c->stream>>>(a, cell);
}

template <typename R, bool RSP>
static cudaError_t launch_pair_r(pinyb200_ctx *c, const PairArgs &a, const Cell &cell)
{
    switch (c->P) {
    case 1: launch_pair_t<R, 1, RSP>(c, a, cell); break;
    case 2: launch_pair_t<R, 2, RSP>(c, a, cell); break;
    case 4: launch_pair_t<R, 4, RSP>(c, a, cell); break;
    case 8: launch_pair_t<R, 8, RSP>(c, a, cell); break;
    case 16: launch_pair_t<R, 16, RSP>(c, a, cell); break;
    case 32: launch_pair_t<R, 32, RSP>(c, a, cell); break;
    case 64: launch_pair_t<R, 64, RSP>(c, a, cell); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

static PairArgs pair_args(pinyb200_ctx *c, bool energy)
{
    const DeviceSystem &s = c->sys;
    PairArgs a;
    a.row = c->d_rowA;
    a.col = c->d_colA;
    a.natm = s.natm;
    a.ntyp = s.ntyp;
    a.nsplin = s.nsplin;
    a.nuniq = s.nuniq;
    a.posT = c->d_posT;
    a.xmod = c->d_xmod;
    a.use_xmod = c->P > 1;
    a.atm_typ = s.atm_typ;
    a.charge = s.charge;
    a.inter_map = s.inter_map;
    a.cutoff = s.cutoff;
    a.rmin = s.rmin;
    a.dr = s.dr;
    a.dri = s.dri;
    a.has_vdw = s.has_vdw;
    a.forceT = c->d_forceT;
    a.acc = c->d_acc;
    a.energy = energy ? 1 : 0;
    a.bad = c->d_ls ? (const int *)((const char *)c->d_ls + offsetof(ListState, overflow)) : nullptr;
    a.tab = c->precision == PINYB200_FP64 ? (const void *)s.tab64 : (const void *)s.tab32;
    a.respa = 0;
    a.cut_res = nullptr;
    a.rheal = a.rheali = a.w_res = a.w_full = 1.0;
    return a;
}

cudaError_t launch_pair(pinyb200_ctx *c, const Cell &cell, bool energy)
{
    const PairArgs a = pair_args(c, energy);
    if (c->precision == PINYB200_FP64) return launch_pair_r<double, false>(c, a, cell);
    return launch_pair_r<float, false>(c, a, cell);
}

// One RESPA pass of the real-space pair forces over the RESPA pair list
// into target ([natm][3][P]); no energies.  mode as PairArgs::respa.
cudaError_t launch_pair_respa(pinyb200_ctx *c, const Cell &cell, int mode, double *target)
{
    PairArgs a = pair_args(c, false);
    a.row = c->d_rowR;
    a.col = c->d_colR;
    a.forceT = target;
    a.respa = mode;
    a.cut_res = c->d_cut_res;
    a.rheal = c->r_rheal;
    a.rheali = 1.0 / c->r_rheal;
    a.w_res = c->r_wter_res;
    a.w_full = c->r_wter;
    if (c->precision == PINYB200_FP64) return launch_pair_r<double, true>(c, a, cell);
    return launch_pair_r<float, true>(c, a, cell);
}

}  // namespace pinyb200
