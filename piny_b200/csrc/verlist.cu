// Verlet list build on the device.
//
// Restates PINY's list criterion (verlist_create.c:25-221 with
// vercreate_list_count_fill :373-503): the half list holds every pair i > j
// that is not excluded (set_exclude.c) and whose bead-1 minimum-image
// separation satisfies r^2 < cutskin^2 of its pair type, evaluated in FP64
// with PINY's operation order so that borderline pairs fall the same way.
// PINY enumerates candidates through link cells or a no-list sweep; the
// accepted set does not depend on the enumeration, so the device sweeps all
// j < i of a row with one warp (coalesced j loads, ballot compaction) and
// writes two CSR lists: the full one (parity with PINY) and the "active" one
// the force kernel walks (pairs with a charge product or a vdW table; the
// others contribute exactly zero in PINY too).
#include "common.cuh"

namespace pinyb200 {

template <int FILL>
__global__ void __launch_bounds__(256) list_kernel(const int *__restrict__ gate, int natm, int ntyp,
                                                   const double *__restrict__ pos1,
                                                   const double *__restrict__ xm, int use_xm, Cell cell,
                                                   const double *__restrict__ cutskin2,
                                                   const int *__restrict__ atm_typ,
                                                   const double *__restrict__ charge,
                                                   const int *__restrict__ inter_map,
                                                   const int *__restrict__ has_vdw,
                                                   const int *__restrict__ excl_off,
                                                   const int *__restrict__ excl_j, int *__restrict__ count,
                                                   const int *__restrict__ row, int *__restrict__ col,
                                                   const int *__restrict__ rowA, int *__restrict__ colA,
                                                   long long cap)
{
    if (gate && *gate == 0) return;  // device list update: no rebuild this step
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < natm; i += nwarps) {
        const double xi = pos1[3 * i], yi = pos1[3 * i + 1], zi = pos1[3 * i + 2];
        double xmi = 0, ymi = 0, zmi = 0;
        if (use_xm) { xmi = xm[3 * i]; ymi = xm[3 * i + 1]; zmi = xm[3 * i + 2]; }
        const int ti = atm_typ[i];
        const double qi = charge[i];
        const int e0 = excl_off[i], e1 = excl_off[i + 1];
        int nfull = 0, nact = 0;
        long long wfull = FILL ? row[i] : 0, wact = FILL ? rowA[i] : 0;
        for (int j0 = 0; j0 < i; j0 += 32) {
            const int j = j0 + lane;
            bool keep = false, act = false;
            if (j < i) {
                bool ex = false;
                for (int e = e0; e < e1; e++) ex |= (excl_j[e] == j);
                if (!ex) {
                    double dx = __dsub_rn(xi, pos1[3 * j]);
                    double dy = __dsub_rn(yi, pos1[3 * j + 1]);
                    double dz = __dsub_rn(zi, pos1[3 * j + 2]);
                    if (use_xm)
                        period_pimd_exact(dx, dy, dz, __dsub_rn(xmi, xm[3 * j]), __dsub_rn(ymi, xm[3 * j + 1]),
                                          __dsub_rn(zmi, xm[3 * j + 2]), cell);
                    else
                        period_exact(dx, dy, dz, cell);
                    double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                    const int pt = pair_type(ti, atm_typ[j], ntyp);
                    keep = r2 < cutskin2[pt];
                    act = keep && (has_vdw[inter_map[pt]] || (qi * charge[j] != 0.0));
                }
            }
            const unsigned bk = __ballot_sync(0xffffffffu, keep);
            const unsigned ba = __ballot_sync(0xffffffffu, act);
            if (FILL) {
                const unsigned below = (1u << lane) - 1u;
                if (keep) {
                    long long p = wfull + nfull + __popc(bk & below);
                    if (p < cap) col[p] = j;
                }
                if (act) {
                    long long p = wact + nact + __popc(ba & below);
                    if (p < cap) colA[p] = j;
                }
            }
            nfull += __popc(bk);
            nact += __popc(ba);
        }
        if (!FILL && lane == 0) {
            count[i] = nfull;
            count[natm + i] = nact;
        }
    }
}

cudaError_t launch_build_list(pinyb200_ctx *c, const Cell &cell, const double *d_pos1, const double *d_xm,
                              const double *d_cutskin2, int pass, const int *gate, cudaStream_t st)
{
    if (!st) st = c->stream;
    const DeviceSystem &s = c->sys;
    const int threads = 256;
    int blocks = (s.natm * 32 + threads - 1) / threads;
    const int maxb = c->sm_count * 8;
    if (blocks > maxb) blocks = maxb;
    if (pass == 0) {
        list_kernel<0><<<blocks, threads, 0, st>>>(gate, s.natm, s.ntyp, d_pos1, d_xm, d_xm != nullptr, cell,
                                                          d_cutskin2, s.atm_typ, s.charge, s.inter_map, s.has_vdw,
                                                          s.excl_off, s.excl_j, c->d_count, nullptr, nullptr,
                                                          nullptr, nullptr, 0);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        return launch_scan(c, gate, s.natm, 2, c->d_count, c->d_row, c->d_rowA, c->d_tot, st);
    } else {
        list_kernel<1><<<blocks, threads, 0, st>>>(gate, s.natm, s.ntyp, d_pos1, d_xm, d_xm != nullptr, cell,
                                                          d_cutskin2, s.atm_typ, s.charge, s.inter_map, s.has_vdw,
                                                          s.excl_off, s.excl_j, c->d_count, c->d_row, c->d_col,
                                                          c->d_rowA, c->d_colA, c->list_cap);
    }
    return cudaGetLastError();
}

}  // namespace pinyb200

namespace pinyb200 {

// Count pass alone, into a caller-supplied count array [2][natm] (full,
// active), on the given stream.  Every row's counts are written.
cudaError_t launch_list_count(pinyb200_ctx *c, const Cell &cell, const double *d_pos1, const double *d_xm,
                              const double *d_cutskin2, int *d_count, cudaStream_t st)
{
    const DeviceSystem &s = c->sys;
    const int threads = 256;
    int blocks = (s.natm * 32 + threads - 1) / threads;
    const int maxb = c->sm_count * 8;
    if (blocks > maxb) blocks = maxb;
    list_kernel<0><<<blocks, threads, 0, st>>>(nullptr, s.natm, s.ntyp, d_pos1, d_xm, d_xm != nullptr, cell, d_cutskin2,
                                               s.atm_typ, s.charge, s.inter_map, s.has_vdw, s.excl_off, s.excl_j,
                                               d_count, nullptr, nullptr, nullptr, nullptr, 0);
    return cudaGetLastError();
}

// Sums of the two count arrays added into tot[0] (full) and tot[1] (active);
// tot must hold zero before the launch.
__global__ void __launch_bounds__(256) count_total_kernel(int n, const int *__restrict__ count,
                                                          unsigned long long *__restrict__ tot)
{
    __shared__ unsigned long long part[2][8];
    unsigned long long s0 = 0, s1 = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        s0 += (unsigned)count[i];
        s1 += (unsigned)count[n + i];
    }
    for (int o = 16; o >= 1; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        part[0][w] = s0;
        part[1][w] = s1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t0 = 0, t1 = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) {
            t0 += part[0][k];
            t1 += part[1][k];
        }
        atomicAdd(&tot[0], t0);
        atomicAdd(&tot[1], t1);
    }
}

cudaError_t launch_count_total(pinyb200_ctx *c, const int *d_count, unsigned long long *d_tot, cudaStream_t st)
{
    const int n = c->sys.natm;
    int blocks = (n + 255) / 256;
    if (blocks > c->sm_count) blocks = c->sm_count;
    if (blocks < 1) blocks = 1;
    count_total_kernel<<<blocks, 256, 0, st>>>(n, d_count, d_tot);
    return cudaGetLastError();
}

}  // namespace pinyb200

namespace pinyb200 {

// Rebuild test of the Verlet list on the device (check_ver_list,
// nbr_list_control.c:182-247, and get_pimd_spread, pimd_estimators.c:
// 121-220): out[0] = max_i |r_i(bead 1) - r_i(at the last build)|^2,
// out[1] = max over beads b > 1 and atoms i of |r_i(b) - r_i(bead 1)|^2,
// both as the bit patterns of non-negative doubles (ordered like the
// values) and both zero on entry.  Squares are formed without FMA
// contraction, in PINY's order.  pos: [P][natm][3], x0: [natm][3].
__global__ void __launch_bounds__(256) list_check_kernel(int natm, int P, const double *__restrict__ pos,
                                                         const double *__restrict__ x0,
                                                         unsigned long long *__restrict__ out)
{
    double dmax = 0.0, smax = 0.0;
    const long long n = (long long)natm * P;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t / natm), i = (int)(t % natm);
        const double *p = pos + ((size_t)b * natm + i) * 3;
        const double *q = b == 0 ? x0 + (size_t)i * 3 : pos + (size_t)i * 3;
        const double dx = __dsub_rn(p[0], q[0]), dy = __dsub_rn(p[1], q[1]), dz = __dsub_rn(p[2], q[2]);
        const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
        if (b == 0) dmax = fmax(dmax, r2);
        else smax = fmax(smax, r2);
    }
    for (int o = 16; o >= 1; o >>= 1) {
        dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
        smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&out[0], (unsigned long long)__double_as_longlong(dmax));
        atomicMax(&out[1], (unsigned long long)__double_as_longlong(smax));
    }
}

cudaError_t launch_list_check(pinyb200_ctx *c, const double *d_pos, unsigned long long *d_out, cudaStream_t st)
{
    const long long n = (long long)c->sys.natm * c->P;
    long long blocks = (n + 255) / 256;
    if (blocks > (long long)c->sm_count * 4) blocks = (long long)c->sm_count * 4;
    if (blocks < 1) blocks = 1;
    list_check_kernel<<<(unsigned)blocks, 256, 0, st>>>(c->sys.natm, c->P, d_pos, c->d_x0, d_out);
    return cudaGetLastError();
}

}  // namespace pinyb200
