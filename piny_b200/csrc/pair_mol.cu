// Molecule-pair form of the real-space kernel.
//
// The site Verlet list of PINY (verlist_create.c) is regrouped by molecule:
// one entry per molecule pair (mi > mj) with a bit mask of the site pairs
// (si, sj) that PINY's list holds and that carry a force (a charge product
// or a vdW table).  The mask is computed with the same FP64 criterion as the
// site list (r^2 < cutskin^2 on the bead-1 minimum image, exclusions), so
// the molecule list and the site list contain exactly the same site pairs.
//
// Per site pair and bead the arithmetic is force_npol's (force_npol.c:
// 28-329, see pair.cu).  What the grouping buys on B200:
//   * one list index and one set of j positions per molecule pair;
//   * j-site reactions summed in registers over the molecule pair, one FP64
//     red.add per j site that received a force;
//   * rows cut into chunks of a few molecule pairs, so warps get even work;
//   * MIXED: the pair separation is d0 + e_i - e_j, with d0 the site-0
//     separation formed in FP64 and e the FP32 site offsets inside each
//     molecule; the per-site-pair image shift of period_pimd (period.c:121)
//     is evaluated from the mode-1 separations the same way.
//   * FP64: every site-pair separation and image shift in FP64 with PINY's
//     operation order, as in the site kernel.
#include <cstddef>

#include "common.cuh"

namespace pinyb200 {

// ---------------------------------------------------------------------------
// molecule-pair list build (count / fill), FP64 criterion of the site list.
//
// Each molecule pair (mi > mj) gets two masks of site pairs (si, sj) with
// r^2 < cutskin^2 on PINY's image: the full mask (PINY's list) and the
// active one (pairs that carry a force).  A molecule pair is kept when its
// full mask is not empty.  The site lists (full and active, rows i with
// ascending j < i) are expanded from the masks afterwards, so the FP64
// criterion is evaluated once per site pair.  Every pair inside a molecule
// is excluded (checked when the context is made), so no site pair is lost.
//
// A molecule pair is skipped without looking at its sites when a lower
// bound of the distance between any images of the two site-0 mode-1
// positions exceeds the reach R = max cutskin + 2 (e + d), e = largest
// distance of a site from its molecule's site 0 and d = largest distance of
// a bead-1 position from its mode-1 position (mode-1 positions: xm, or the
// bead-1 positions for one bead).  Any site pair of a pair so skipped is
// farther apart than max cutskin on every image.

// Lower bound of |dx + h n| over all lattice vectors h n: along each cell
// axis the wrapped fractional separation times the lattice-plane spacing.
__device__ __forceinline__ double image_lower_bound(double dx, double dy, double dz, const Cell &c)
{
    double lb = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double b0 = c.hi[d], b1 = c.hi[3 + d], b2 = c.hi[6 + d];
        const double sd = dx * b0 + dy * b1 + dz * b2;
        const double w = fabs(sd - rint(sd)) * rsqrt(b0 * b0 + b1 * b1 + b2 * b2);
        lb = fmax(lb, w);
    }
    return lb;
}

// The reach R (above) into *reach; one block.
__global__ void __launch_bounds__(1024) mol_reach_kernel(const int *__restrict__ gate, int nmol,
                                                          const int *__restrict__ mstart,
                                                          const double *__restrict__ pos1,
                                                          const double *__restrict__ xm, int use_xm,
                                                          const double *__restrict__ cs, int npt,
                                                          double *__restrict__ reach)
{
    if (gate && *gate == 0) return;
    __shared__ double red[3][32];
    double ext = 0.0, dev = 0.0, cmax = 0.0;
    for (int k = threadIdx.x; k < npt; k += blockDim.x) cmax = fmax(cmax, cs[k]);
    for (int m = threadIdx.x; m < nmol; m += blockDim.x) {
        const int i0 = mstart[m], i1 = mstart[m + 1];
        const double *x0 = (use_xm ? xm : pos1) + 3 * (size_t)i0;
        for (int i = i0; i < i1; i++) {
            const double *xi = (use_xm ? xm : pos1) + 3 * (size_t)i;
            const double ex = xi[0] - x0[0], ey = xi[1] - x0[1], ez = xi[2] - x0[2];
            ext = fmax(ext, sqrt(ex * ex + ey * ey + ez * ez));
            if (use_xm) {
                const double *p = pos1 + 3 * (size_t)i;
                const double qx = p[0] - xi[0], qy = p[1] - xi[1], qz = p[2] - xi[2];
                dev = fmax(dev, sqrt(qx * qx + qy * qy + qz * qz));
            }
        }
    }
    for (int o = 16; o >= 1; o >>= 1) {
        ext = fmax(ext, __shfl_xor_sync(0xffffffffu, ext, o));
        dev = fmax(dev, __shfl_xor_sync(0xffffffffu, dev, o));
        cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][w] = ext;
        red[1][w] = dev;
        red[2][w] = cmax;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); k++) {
            ext = fmax(ext, red[0][k]);
            dev = fmax(dev, red[1][k]);
            cmax = fmax(cmax, red[2][k]);
        }
        // rounding of the bound and of the criterion: a generous margin
        *reach = (sqrt(cmax) + 2.0 * (ext + dev)) * (1.0 + 1e-12) + 1e-9;
    }
}

template <int FILL, int NS>
__global__ void __launch_bounds__(256) mol_list_kernel(const int *__restrict__ gate, int nmol,
                                                       const int *__restrict__ mstart, int ntyp,
                                                       const double *__restrict__ pos1, const double *__restrict__ xm,
                                                       int use_xm, Cell cell, const double *__restrict__ cutskin2,
                                                       const int *__restrict__ atm_typ,
                                                       const double *__restrict__ charge,
                                                       const int *__restrict__ inter_map,
                                                       const int *__restrict__ has_vdw,
                                                       const double *__restrict__ reach, int *__restrict__ count,
                                                       const int *__restrict__ row, int *__restrict__ mj_out,
                                                       unsigned *__restrict__ mask_out, unsigned *__restrict__ maskf_out,
                                                       long long cap, unsigned long long *__restrict__ nsite)
{
    if (gate && *gate == 0) return;  // device list update: no rebuild this step
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const double R = *reach;
    const double *x0 = use_xm ? xm : pos1;  // site-0 mode-1 positions for the bound
    unsigned long long sites = 0;
    for (int mi = warp; mi < nmol; mi += nwarps) {
        const int i0 = mstart[mi], ni = mstart[mi + 1] - i0;
        const double bx = x0[3 * (size_t)i0], by = x0[3 * (size_t)i0 + 1], bz = x0[3 * (size_t)i0 + 2];
        int n = 0;
        const long long w0 = FILL ? row[mi] : 0;
        for (int m0 = 0; m0 < mi; m0 += 32) {
            const int mj = m0 + lane;
            unsigned mask = 0, maskf = 0;
            if (mj < mi) {
                const int j0 = mstart[mj], nj = mstart[mj + 1] - j0;
                const double lb = image_lower_bound(bx - x0[3 * (size_t)j0], by - x0[3 * (size_t)j0 + 1],
                                                    bz - x0[3 * (size_t)j0 + 2], cell);
                if (!(lb > R)) {
                    for (int si = 0; si < ni; si++) {
                        const int i = i0 + si;
                        const double xi = pos1[3 * i], yi = pos1[3 * i + 1], zi = pos1[3 * i + 2];
                        const int ti = atm_typ[i];
                        const double qi = charge[i];
                        for (int sj = 0; sj < nj; sj++) {
                            const int j = j0 + sj;
                            double dx = __dsub_rn(xi, pos1[3 * j]);
                            double dy = __dsub_rn(yi, pos1[3 * j + 1]);
                            double dz = __dsub_rn(zi, pos1[3 * j + 2]);
                            if (use_xm)
                                period_pimd_exact(dx, dy, dz, __dsub_rn(xm[3 * i], xm[3 * j]),
                                                  __dsub_rn(xm[3 * i + 1], xm[3 * j + 1]),
                                                  __dsub_rn(xm[3 * i + 2], xm[3 * j + 2]), cell);
                            else
                                period_exact(dx, dy, dz, cell);
                            const double r2 =
                                __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                            const int pt = pair_type(ti, atm_typ[j], ntyp);
                            if (r2 < cutskin2[pt]) {
                                const unsigned bit = 1u << (si * NS + sj);
                                maskf |= bit;
                                if (has_vdw[inter_map[pt]] || qi * charge[j] != 0.0) mask |= bit;
                            }
                        }
                    }
                }
            }
            const bool keep = maskf != 0;
            const unsigned bk = __ballot_sync(0xffffffffu, keep);
            if (FILL && keep) {
                const long long p = w0 + n + __popc(bk & ((1u << lane) - 1u));
                if (p < cap) {
                    mj_out[p] = mj;
                    mask_out[p] = mask;
                    maskf_out[p] = maskf;
                }
            }
            if (FILL) sites += __popc(mask);
            n += __popc(bk);
        }
        if (!FILL && lane == 0) count[mi] = n;
    }
    if (FILL) {
        for (int o = 16; o >= 1; o >>= 1) sites += __shfl_xor_sync(0xffffffffu, sites, o);
        if (lane == 0) atomicAdd(nsite, sites);
    }
}

// Site lists from the molecule masks.  Count: per site, the full and active
// pairs with lower-index sites; one warp per molecule row.
template <int NS>
__global__ void __launch_bounds__(256) site_count_kernel(const int *__restrict__ gate, int nmol, int natm,
                                                         const int *__restrict__ mstart, const int *__restrict__ mrow,
                                                         const unsigned *__restrict__ maskf,
                                                         const unsigned *__restrict__ mask, long long cap,
                                                         int *__restrict__ count)
{
    if (gate && *gate == 0) return;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    constexpr unsigned RM = (1u << NS) - 1u;
    for (int mi = warp; mi < nmol; mi += nwarps) {
        const int i0 = mstart[mi], ni = mstart[mi + 1] - i0;
        const int k1 = (int)(mrow[mi + 1] < cap ? mrow[mi + 1] : cap);
        int cf[NS], ca[NS];
#pragma unroll
        for (int si = 0; si < NS; si++) cf[si] = ca[si] = 0;
        for (int k = mrow[mi] + lane; k < k1; k += 32) {
            const unsigned f = maskf[k], a = mask[k];
#pragma unroll
            for (int si = 0; si < NS; si++) {
                cf[si] += __popc((f >> (si * NS)) & RM);
                ca[si] += __popc((a >> (si * NS)) & RM);
            }
        }
#pragma unroll
        for (int si = 0; si < NS; si++) {
            for (int o = 16; o >= 1; o >>= 1) {
                cf[si] += __shfl_xor_sync(0xffffffffu, cf[si], o);
                ca[si] += __shfl_xor_sync(0xffffffffu, ca[si], o);
            }
            if (lane == 0 && si < ni) {
                count[i0 + si] = cf[si];
                count[natm + i0 + si] = ca[si];
            }
        }
    }
}

// Fill: row i lists j = mstart[mj] + sj in molecule-row order (mj
// ascending), sj ascending within a molecule pair: ascending j.
template <int NS>
__global__ void __launch_bounds__(256) site_fill_kernel(const int *__restrict__ gate, int nmol,
                                                        const int *__restrict__ mstart, const int *__restrict__ mrow,
                                                        const int *__restrict__ mj, const unsigned *__restrict__ maskf,
                                                        const unsigned *__restrict__ mask, long long mcap,
                                                        const int *__restrict__ row, const int *__restrict__ rowA,
                                                        int *__restrict__ col, int *__restrict__ colA, long long cap)
{
    if (gate && *gate == 0) return;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    constexpr unsigned RM = (1u << NS) - 1u;
    for (int mi = warp; mi < nmol; mi += nwarps) {
        const int i0 = mstart[mi], ni = mstart[mi + 1] - i0;
        const int k1 = (int)(mrow[mi + 1] < mcap ? mrow[mi + 1] : mcap);
        for (int si = 0; si < ni; si++) {
            long long wf = row[i0 + si], wa = rowA[i0 + si];
            for (int k0 = mrow[mi]; k0 < k1; k0 += 32) {
                const int k = k0 + lane;
                unsigned f = 0, a = 0;
                int j0 = 0;
                if (k < k1) {
                    f = (maskf[k] >> (si * NS)) & RM;
                    a = (mask[k] >> (si * NS)) & RM;
                    j0 = mstart[mj[k]];
                }
                // exclusive prefix sums of the per-lane counts
                int nf = __popc(f), na = __popc(a), pf = nf, pa = na;
                for (int o = 1; o < 32; o <<= 1) {
                    const int tf = __shfl_up_sync(0xffffffffu, pf, o), ta = __shfl_up_sync(0xffffffffu, pa, o);
                    if (lane >= o) {
                        pf += tf;
                        pa += ta;
                    }
                }
                long long qf = wf + pf - nf, qa = wa + pa - na;
                for (unsigned m = f; m; m &= m - 1u) {
                    if (qf < cap) col[qf] = j0 + __ffs(m) - 1;
                    qf++;
                }
                for (unsigned m = a; m; m &= m - 1u) {
                    if (qa < cap) colA[qa] = j0 + __ffs(m) - 1;
                    qa++;
                }
                wf += __shfl_sync(0xffffffffu, pf, 31);
                wa += __shfl_sync(0xffffffffu, pa, 31);
            }
        }
    }
}

__global__ void __launch_bounds__(1024) mol_scan_kernel(const int *__restrict__ gate, int n,
                                                         const int *__restrict__ count, int *__restrict__ row,
                                                         long long *__restrict__ tot)
{
    if (gate && *gate == 0) return;
    __shared__ long long part[1024];
    const int t = threadIdx.x;
    const int chunk = (n + blockDim.x - 1) / blockDim.x;
    const int lo = min(n, t * chunk), hi = min(n, lo + chunk);
    long long s0 = 0;
    for (int i = lo; i < hi; i++) s0 += count[i];
    part[t] = s0;
    __syncthreads();
    for (int o = 1; o < blockDim.x; o <<= 1) {
        long long a0 = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += a0;
        __syncthreads();
    }
    long long b0 = part[t] - s0;
    for (int i = lo; i < hi; i++) {
        row[i] = (int)b0;
        b0 += count[i];
    }
    if (t == blockDim.x - 1) {
        row[n] = (int)part[t];
        *tot = part[t];
    }
}

// ---------------------------------------------------------------------------
// force kernel

struct MolArgs {
    const int *nchunk;  // device: chunks of the current list
    const int *chunk;   // [nchunk][3]: mi, begin, end
    const int *bad;     // device flags (overflow, mismatch) of the list update, or nullptr
    const int *mj;
    const unsigned *mask;
    const int *mstart;
    int ntyp, npt, nuniq, nsplin;
    const double *posT, *xmod;  // xmod: [natm][3] (bead positions when P == 1)
    int pimd;
    const int *atm_typ;
    const double *charge;
    const int *inter_map;
    const double *cutoff, *rmin, *dr, *dri;
    const int *has_vdw;
    const void *tab;
    double *forceT;
    double *acc;
    int energy;
};

// Site-pair constants of the (uniform) molecule for site si of molecule i
// and site sj of molecule j, sp = si * NS + sj:
//   MIXED  c = (rc^2, rmin, dri, q2)
//   FP64   c = (rc, rmin, dr, dri), q2 separately
//   o = (table row u * nsplin, vdW table present)
template <typename R>
struct PairConst {
    typename Vec4<R>::T c[16];
    R q2[16];
    int2 o[16];
};

// Exact PINY image shift -NINT(h^-1 dmode) of one site pair along the
// diagonal of an orthorhombic cell (period_pimd, period.c:163-176).
__device__ __forceinline__ double shift_exact(double dm, double hi) { return -nint_rn(__dmul_rn(dm, hi)); }

// Sites of a molecule sit within this distance (Bohr) of its site 0 in the
// mode-1 coordinates; a site pair can take a different image than the
// site-0 pair only when the site-0 separation is within twice this of half
// a box, and only then is its own shift evaluated.
#define PINYB200_MOL_EXTENT 5.0

// Resident blocks of 128 threads per SM the register allocation aims at.
#ifndef PINYB200_MOL_BLOCKS32
#define PINYB200_MOL_BLOCKS32 5
#endif
#ifndef PINYB200_MOL_BLOCKS64
#define PINYB200_MOL_BLOCKS64 3
#endif

// Spline knot of a MIXED site pair: t = (r - rmin) dri, k = nint(t) + 3
// clamped to the table, offset del = t - (k - 3).
__device__ __forceinline__ int knot32(float r, float rmin, float dri, int nsm2, float &del)
{
    const float t = (r - rmin) * dri;
    int k = (int)(t + 0.5f) + 3;
    k = k < nsm2 ? k : nsm2;
    k = k > 3 ? k : 3;
    del = t - (float)(k - 3);
    return k;
}

// One site pair of one bead: force -dV/dr * r_vec / r on i (returned in
// f), energies and virial accumulated.  r holds the separation i - j.
// The sum is force_npol's: q2 * Coulomb table + vdW table.
template <typename R, bool FAST, bool ENERGY>
__device__ __forceinline__ bool site_pair(const typename Vec4<R>::T *__restrict__ tab, size_t tstride, int nsm2,
                                          const PairConst<R> &pc, int sp, R rx, R ry, R rz, R &fx, R &fy, R &fz,
                                          R &evs, R &ecs, R *pvs)
{
    typedef typename Vec4<R>::T V;
    const V c = pc.c[sp];
    const int2 o = pc.o[sp];
    R del, q2;
    int kk;
    if constexpr (FAST) {
        // MIXED: cutoff on r^2, r from the reciprocal square root
        const R r2 = rx * rx + ry * ry + rz * rz;
        if (!(r2 < c.x)) return false;
        const R r = r2 * rsqrtf(r2);
        kk = knot32(r, c.y, c.z, nsm2, del);
        q2 = c.w;
    } else {
        const R r = Idx<R>::dist(rx, ry, rz);
        if (!(r < c.x)) return false;
        kk = Idx<R>::knot(r, c.y, c.z, c.w, nsm2, del);
        q2 = pc.q2[sp];
    }
    const size_t off = (size_t)o.x + (kk - 1);
    R dv = 0;
    if (q2 != (R)0) dv = q2 * spline_eval<V, R>(ldg4(tab + T_CDV0C * tstride + off), del);
    if (o.y) dv += spline_eval<V, R>(ldg4(tab + T_CDV0 * tstride + off), del);
    fx = rx * dv;
    fy = ry * dv;
    fz = rz * dv;
    if (ENERGY) {
        if (q2 != (R)0) ecs += q2 * spline_eval<V, R>(ldg4(tab + T_CV0C * tstride + off), del);
        if (o.y) evs += spline_eval<V, R>(ldg4(tab + T_CV0 * tstride + off), del);
        pvs[0] += rx * fx;
        pvs[1] += ry * fy;
        pvs[2] += rz * fz;
        pvs[3] += rx * fy;
        pvs[4] += rx * fz;
        pvs[5] += ry * fz;
    }
    return true;
}

// One molecule pair whose site-0 separation is within twice the molecular
// extent of half a box, so that its site pairs may take different images:
// every site pair gets its own period_pimd shift (period.c:163-176) and its
// separation in FP64; forces go straight to the force array.  Kept out of
// line: it is rare in large boxes and would otherwise burden the main
// loop with its registers.
template <typename R, int P, int NS, bool FAST, bool ENERGY>
__device__ __noinline__ void mol_pair_near(const double *__restrict__ posT, const double *__restrict__ xmod,
                                           double *__restrict__ forceT, const PairConst<R> *pc,
                                           const typename Vec4<R>::T *__restrict__ tab, size_t tstride, int nsm2,
                                           int i0, int j0, unsigned mask, int b, double hx, double hy, double hz,
                                           double hix, double hiy, double hiz, double *sacc)
{
    const double hd[3] = {hx, hy, hz}, hid[3] = {hix, hiy, hiz};
    R evs = 0, ecs = 0, pvs[6] = {0, 0, 0, 0, 0, 0};
    for (unsigned m = mask; m; m &= m - 1u) {
        const int sp = __ffs(m) - 1;
        const int si = sp / NS, sj = sp % NS;
        const int i = i0 + si, j = j0 + sj;
        double r[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const double sh = shift_exact(__dsub_rn(xmod[3 * (size_t)i + d], xmod[3 * (size_t)j + d]), hid[d]);
            r[d] = __dadd_rn(__dsub_rn(posT[(3 * (size_t)i + d) * P + b], posT[(3 * (size_t)j + d) * P + b]),
                             __dmul_rn(sh, hd[d]));
        }
        R fx, fy, fz;
        if (site_pair<R, FAST, ENERGY>(tab, tstride, nsm2, *pc, sp, (R)r[0], (R)r[1], (R)r[2], fx, fy, fz, evs, ecs,
                                       pvs)) {
            atomicAdd(&forceT[(3 * (size_t)i + 0) * P + b], (double)fx);
            atomicAdd(&forceT[(3 * (size_t)i + 1) * P + b], (double)fy);
            atomicAdd(&forceT[(3 * (size_t)i + 2) * P + b], (double)fz);
            atomicAdd(&forceT[(3 * (size_t)j + 0) * P + b], -(double)fx);
            atomicAdd(&forceT[(3 * (size_t)j + 1) * P + b], -(double)fy);
            atomicAdd(&forceT[(3 * (size_t)j + 2) * P + b], -(double)fz);
        }
    }
    if (ENERGY) {
        sacc[0] += (double)evs;
        sacc[128] += (double)ecs;
#pragma unroll
        for (int c = 0; c < 6; c++) sacc[128 * (2 + c)] += (double)pvs[c];
    }
}

template <typename R, int P, int NS, bool FAST, bool ENERGY>
__global__ void __launch_bounds__(128, sizeof(R) == 4 ? PINYB200_MOL_BLOCKS32 : PINYB200_MOL_BLOCKS64)
    mol_pair_kernel(MolArgs a, Cell cell)
{
    typedef typename Vec4<R>::T V;
    constexpr int G = P >= 32 ? 32 : P;  // lanes per molecule pair
    constexpr int JPI = 32 / G;          // molecule pairs per warp step
    __shared__ PairConst<R> pc;
    __shared__ double sacc[8][128];      // per-thread energy / virial sums
    if (threadIdx.x < NS * NS) {
        // every molecule has the sites of molecule 0 (checked on the host)
        const int si = threadIdx.x / NS, sj = threadIdx.x % NS;
        const int nm0 = a.mstart[1];
        const int ia = si < nm0 ? si : 0, ja = sj < nm0 ? sj : 0;
        const int p = pair_type(a.atm_typ[ia], a.atm_typ[ja], a.ntyp);
        const int u = a.inter_map[p];
        const double q2 = a.charge[ia] * a.charge[ja];
        V c;
        if (FAST) {
            c.x = (R)(a.cutoff[p] * a.cutoff[p]);
            c.y = (R)a.rmin[u];
            c.z = (R)a.dri[u];
            c.w = (R)q2;
        } else {
            c.x = (R)a.cutoff[p];
            c.y = (R)a.rmin[u];
            c.z = (R)a.dr[u];
            c.w = (R)a.dri[u];
        }
        pc.c[threadIdx.x] = c;
        pc.q2[threadIdx.x] = (R)q2;
        pc.o[threadIdx.x] = make_int2(u * a.nsplin, a.has_vdw[u]);
    }
    if (ENERGY)
        for (int c = 0; c < 8; c++) sacc[c][threadIdx.x] = 0.0;
    __syncthreads();
    if (a.bad && (a.bad[0] | a.bad[1])) {
        // the list update could not hold the new list: make the evaluation
        // fail loudly (non-finite energy) instead of using a stale list
        if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) a.acc[S_VVDW] = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    const V *__restrict__ tab = (const V *)a.tab;
    const size_t tstride = (size_t)a.nuniq * a.nsplin;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int sub = lane / G;
    const int b = (lane % G) + 32 * blockIdx.y;  // bead
    const int nsm2 = a.nsplin - 2;
    const double *__restrict__ posT = a.posT;

    const int nch = *a.nchunk;
    for (int ch = warp; ch < nch; ch += nwarps) {
        const int mi = a.chunk[3 * ch], beg = a.chunk[3 * ch + 1], end = a.chunk[3 * ch + 2];
        const int i0 = a.mstart[mi], ni = a.mstart[mi + 1] - i0;
        double xi[NS][3];  // FP64 positions (MIXED keeps site 0 only live)
        R ei[NS][3];       // MIXED: offsets from site 0
        R fi[NS][3];
#pragma unroll
        for (int s = 0; s < NS; s++) {
            const int i = i0 + (s < ni ? s : 0);
#pragma unroll
            for (int d = 0; d < 3; d++) {
                xi[s][d] = posT[(3 * (size_t)i + d) * P + b];
                fi[s][d] = (R)0;
            }
        }
#pragma unroll
        for (int s = 0; s < NS; s++)
#pragma unroll
            for (int d = 0; d < 3; d++) ei[s][d] = (R)(xi[s][d] - xi[0][d]);
        const double xm0x = a.xmod[3 * (size_t)i0], xm0y = a.xmod[3 * (size_t)i0 + 1],
                     xm0z = a.xmod[3 * (size_t)i0 + 2];
        R evs = 0, ecs = 0, pvs[6] = {0, 0, 0, 0, 0, 0};
        for (int k = beg + sub; k < end; k += JPI) {
            const int mj = __ldcg(a.mj + k);
            const unsigned mask = __ldcg(a.mask + k);
            const int j0 = a.mstart[mj];
            unsigned jm = 1u;
#pragma unroll
            for (int si = 0; si < NS; si++) jm |= (mask >> (si * NS)) & ((1u << NS) - 1u);
            double xj[NS][3];
#pragma unroll
            for (int s = 0; s < NS; s++) {
                const int j = j0 + (((jm >> s) & 1u) ? s : 0);
#pragma unroll
                for (int d = 0; d < 3; d++) xj[s][d] = __ldcg(posT + (3 * (size_t)j + d) * P + b);
            }
            // site-0 image (mode-1 separation, FP64) and whether the pair is
            // close enough to half a box for site pairs to differ from it
            double sh0[3];
            bool near = false;
            {
                const double dm[3] = {__dsub_rn(xm0x, __ldcg(a.xmod + 3 * (size_t)j0)),
                                      __dsub_rn(xm0y, __ldcg(a.xmod + 3 * (size_t)j0 + 1)),
                                      __dsub_rn(xm0z, __ldcg(a.xmod + 3 * (size_t)j0 + 2))};
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const double hid = cell.hi[4 * d];
                    const double t = __dmul_rn(dm[d], hid);
                    sh0[d] = -nint_rn(t);
                    near |= fabs(t + sh0[d]) > 0.5 - 2.0 * PINYB200_MOL_EXTENT * hid;
                }
            }
            if (near) {
                mol_pair_near<R, P, NS, FAST, ENERGY>(posT, a.xmod, a.forceT, &pc, tab, tstride, nsm2, i0, j0, mask, b,
                                                      cell.h[0], cell.h[4], cell.h[8], cell.hi[0], cell.hi[4],
                                                      cell.hi[8], &sacc[0][threadIdx.x]);
                continue;
            }
            R d0[3], ej[NS][3];
            if (FAST) {
#pragma unroll
                for (int d = 0; d < 3; d++) d0[d] = (R)(__dsub_rn(xi[0][d], xj[0][d]) + sh0[d] * cell.h[4 * d]);
#pragma unroll
                for (int s = 0; s < NS; s++)
#pragma unroll
                    for (int d = 0; d < 3; d++) ej[s][d] = (R)(xj[s][d] - xj[0][d]);
            }
            // j sites in a warp-uniform loop (for P >= 32 the mask is the
            // same in every lane); i sites unrolled so their offsets and
            // forces stay in fixed registers
#pragma unroll 1
            for (int sj = 0; sj < NS; sj++) {
                unsigned col = 0;
#pragma unroll
                for (int si = 0; si < NS; si++) col |= ((mask >> (si * NS + sj)) & 1u) << si;
                if (!col) continue;
                // j-site position: MIXED d0 - e_j, FP64 x_j
                R djx = 0, djy = 0, djz = 0;
                double xjx = 0, xjy = 0, xjz = 0;
#pragma unroll
                for (int s2 = 0; s2 < NS; s2++)
                    if (sj == s2) {
                        if (FAST) {
                            djx = d0[0] - ej[s2][0];
                            djy = d0[1] - ej[s2][1];
                            djz = d0[2] - ej[s2][2];
                        } else {
                            xjx = xj[s2][0];
                            xjy = xj[s2][1];
                            xjz = xj[s2][2];
                        }
                    }
                R fjx = 0, fjy = 0, fjz = 0;
#pragma unroll
                for (int si = 0; si < NS; si++) {
                    if (!((col >> si) & 1u)) continue;
                    // away from half a box every site pair takes the site-0 image
                    R rx, ry, rz;
                    if (FAST) {
                        rx = djx + ei[si][0];
                        ry = djy + ei[si][1];
                        rz = djz + ei[si][2];
                    } else {
                        rx = (R)__dadd_rn(__dsub_rn(xi[si][0], xjx), __dmul_rn(sh0[0], cell.h[0]));
                        ry = (R)__dadd_rn(__dsub_rn(xi[si][1], xjy), __dmul_rn(sh0[1], cell.h[4]));
                        rz = (R)__dadd_rn(__dsub_rn(xi[si][2], xjz), __dmul_rn(sh0[2], cell.h[8]));
                    }
                    R fx, fy, fz;
                    if (site_pair<R, FAST, ENERGY>(tab, tstride, nsm2, pc, si * NS + sj, rx, ry, rz, fx, fy, fz, evs,
                                                   ecs, pvs)) {
                        fi[si][0] += fx;
                        fi[si][1] += fy;
                        fi[si][2] += fz;
                        fjx -= fx;
                        fjy -= fy;
                        fjz -= fz;
                    }
                }
                if (fjx != (R)0 || fjy != (R)0 || fjz != (R)0) {
                    const int j = j0 + sj;
                    atomicAdd(&a.forceT[(3 * (size_t)j + 0) * P + b], (double)fjx);
                    atomicAdd(&a.forceT[(3 * (size_t)j + 1) * P + b], (double)fjy);
                    atomicAdd(&a.forceT[(3 * (size_t)j + 2) * P + b], (double)fjz);
                }
            }
        }
        // i-site forces: sum the lane groups that hold the same bead
#pragma unroll
        for (int s = 0; s < NS; s++) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                double v = (double)fi[s][d];
                if (G < 32) v = warp_sum_strided(v, G);
                if ((G == 32 || sub == 0) && s < ni && v != 0.0)
                    atomicAdd(&a.forceT[(3 * (size_t)(i0 + s) + d) * P + b], v);
            }
        }
        if (ENERGY) {
            sacc[0][threadIdx.x] += (double)evs;
            sacc[1][threadIdx.x] += (double)ecs;
#pragma unroll
            for (int c = 0; c < 6; c++) sacc[2 + c][threadIdx.x] += (double)pvs[c];
        }
    }
    if (ENERGY) {
        const int slot[8] = {S_VVDW, S_VCOUL, S_PXX, S_PYY, S_PZZ, S_PXY, S_PXZ, S_PYZ};
#pragma unroll
        for (int c = 0; c < 8; c++) {
            double t = sacc[c][threadIdx.x];
            if (G < 32) t = warp_sum_strided(t, G);
            if (G == 32 || sub == 0) atomicAdd(&a.acc[(size_t)b * S_NSLOT + slot[c]], t);
        }
    }
}

// ---------------------------------------------------------------------------
// MIXED kernel with unrolled site pairs.
//
// Same pairs, images, tables and accumulation scheme as mol_pair_kernel
// (lanes = beads, one molecule pair per lane group, i-site forces in
// registers over a chunk, one FP64 red.add per j site), with the per-pair
// work cut down for a molecular system whose pair types all share one
// cutoff and one spline grid (every PINY water input):
//   * the site-pair loops are unrolled and each site pair's table offset,
//     charge product and which tables it uses (q_i q_j cdv0_c / cv0_c, the
//     vdW cdv0 / cv0; force_npol.c:339-375) are kernel parameters (constant
//     bank): no shared-memory constant load and no address arithmetic on
//     the pair type is left per pair.  The rows stay PINY's per-table ones:
//     every charged pair reads the same Coulomb table, so the tables that
//     32 beads' knots scatter over stay few enough for L1;
//   * the knot nint((r - rmin) dri) (force_npol.c:345-352) is taken with the
//     1.5 * 2^23 rounding constant instead of float <-> int conversions, t
//     clamped to the table's intervals (what clamping the knot does for
//     every r inside the cutoff);
//   * molecules are uniform runs of sites: the j site index is mj * stride,
//     not a load.
// Pairs whose site-0 separation is within twice the molecular extent of half
// a box go through mol_pair_near (per-site-pair FP64 image), as in
// mol_pair_kernel.

// Table row load that asks L1 to keep the line (evict_last): the four
// tables a water system reads stay resident while positions stream past.
__device__ __forceinline__ float4 ldg_keep(const float4 *p)
{
    float4 v;
    asm("ld.global.nc.L1::evict_last.v4.f32 {%0, %1, %2, %3}, [%4];"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "l"(p));
    return v;
}

struct MixArgs {
    const int *nchunk, *chunk, *bad, *mj;
    const unsigned *mask;
    const int *mstart;
    int ntyp, nuniq, nsplin, stride;
    const double *posT, *xmod;
    const int *atm_typ;
    const double *charge;
    const int *inter_map;
    const double *cutoff, *rmin, *dri;
    const int *has_vdw;
    const float4 *tab;   // [4][nuniq][nsplin] interval coefficients (TabKind order)
    const float4 *tabfe; // [2][nuniq][nsplin][2]: vdW then Coulomb; force and energy rows interleaved
    double *forceT;
    double *acc;
    int toff[16];        // per site pair si * NS + sj: u * nsplin + 2, its rows at nint(t) = 0
    float q2[16];        // charge product of the site pair
    int eflag[16];       // tables the site pair uses: 1 vdW, 2 Coulomb
    int tstride;         // nuniq * nsplin, the distance between table kinds
    float rc2, dri_f, rmd, tmax;  // cutoff^2, 1/dr, rmin/dr, last interval
};

#ifndef PINYB200_MIX_BLOCKS
#define PINYB200_MIX_BLOCKS 6
#endif

// Site-pair table patterns known at compile time: bit si * NS + sj of CM
// (Coulomb table) and VM (vdW table).  kAnyPair takes them from
// MixArgs::eflag at run time.
constexpr unsigned kAnyPair = 0xffffffffu;
constexpr unsigned kTip4pCoul = 0xEEE0u, kTip4pVdw = 0x1u;  // O H H M: H, M charged; LJ on O-O
constexpr unsigned kSpcCoul = 0x1FFu, kSpcVdw = 0x1u;       // O H H: all charged; LJ on O-O

template <int P, int NS, bool ENERGY, unsigned CM = kAnyPair, unsigned VM = kAnyPair>
__global__ void __launch_bounds__(128, PINYB200_MIX_BLOCKS) mol_pair_mixed_kernel(MixArgs a, Cell cell)
{
    constexpr int G = P >= 32 ? 32 : P;  // lanes per molecule pair
    constexpr int JPI = 32 / G;          // molecule pairs per warp step
    __shared__ PairConst<float> pc;      // per-kind constants of the near path
    __shared__ double sacc[8][128];
    if (threadIdx.x < NS * NS) {
        const int si = threadIdx.x / NS, sj = threadIdx.x % NS;
        const int nm0 = a.mstart[1];
        const int ia = si < nm0 ? si : 0, ja = sj < nm0 ? sj : 0;
        const int p = pair_type(a.atm_typ[ia], a.atm_typ[ja], a.ntyp);
        const int u = a.inter_map[p];
        const double q2 = a.charge[ia] * a.charge[ja];
        float4 c;
        c.x = (float)(a.cutoff[p] * a.cutoff[p]);
        c.y = (float)a.rmin[u];
        c.z = (float)a.dri[u];
        c.w = (float)q2;
        pc.c[threadIdx.x] = c;
        pc.q2[threadIdx.x] = (float)q2;
        pc.o[threadIdx.x] = make_int2(u * a.nsplin, a.has_vdw[u]);
    }
    if (ENERGY)
        for (int c = 0; c < 8; c++) sacc[c][threadIdx.x] = 0.0;
    __syncthreads();
    if (a.bad && (a.bad[0] | a.bad[1])) {
        if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) a.acc[S_VVDW] = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    const float4 *__restrict__ tab = a.tab;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int sub = lane / G;
    const int b = (lane % G) + 32 * blockIdx.y;  // bead
    const double *__restrict__ posT = a.posT;
    const float rc2 = a.rc2, dri = a.dri_f, rmd = a.rmd, tmax = a.tmax;
    constexpr float kRound = 12582912.0f;  // 1.5 * 2^23: x + kRound - kRound = nearest integer of x

    const int nch = *a.nchunk;
    for (int ch = warp; ch < nch; ch += nwarps) {
        const int mi = a.chunk[3 * ch], beg = a.chunk[3 * ch + 1], end = a.chunk[3 * ch + 2];
        const int i0 = mi * a.stride, ni = a.stride;
        float ei[NS][3], fi[NS][3];
#pragma unroll
        for (int s = 0; s < NS; s++) {
            const int i = i0 + (s < ni ? s : 0);
#pragma unroll
            for (int d = 0; d < 3; d++) {
                ei[s][d] = (float)(posT[(3 * (size_t)i + d) * P + b] - posT[(3 * (size_t)i0 + d) * P + b]);
                fi[s][d] = 0.0f;
            }
        }
        float evs = 0.0f, ecs = 0.0f, pvs[6] = {0, 0, 0, 0, 0, 0};
        for (int k = beg + sub; k < end; k += JPI) {
            const int mj = __ldcg(a.mj + k);
            const unsigned mask = __ldcg(a.mask + k);
            const int j0 = mj * a.stride;
            // site-0 image from the mode-1 separation (FP64) and whether site
            // pairs may take other images
            double sh0[3];
            bool near = false;
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const double hid = cell.hi[4 * d];
                const double t = __dmul_rn(__dsub_rn(a.xmod[3 * (size_t)i0 + d], __ldcg(a.xmod + 3 * (size_t)j0 + d)), hid);
                sh0[d] = -nint_rn(t);
                near |= fabs(t + sh0[d]) > 0.5 - 2.0 * PINYB200_MOL_EXTENT * hid;
            }
            if (near) {
                mol_pair_near<float, P, NS, true, ENERGY>(posT, a.xmod, a.forceT, &pc, a.tab,
                                                           (size_t)a.nuniq * a.nsplin, a.nsplin - 2, i0, j0, mask, b,
                                                           cell.h[0], cell.h[4], cell.h[8], cell.hi[0], cell.hi[4],
                                                           cell.hi[8], &sacc[0][threadIdx.x]);
                continue;
            }
            unsigned jm = 1u;
#pragma unroll
            for (int si = 0; si < NS; si++) jm |= (mask >> (si * NS)) & ((1u << NS) - 1u);
            // dj[s] = x_i0 - x_j(s) + image, in FP32 from the FP64 site-0 separation
            float dj[NS][3];
            {
                // the i anchor is re-read (an L1 hit) rather than held over the chunk
                double xj0[3];
#pragma unroll
                for (int d = 0; d < 3; d++) xj0[d] = __ldcg(posT + (3 * (size_t)j0 + d) * P + b);
#pragma unroll
                for (int d = 0; d < 3; d++)
                    dj[0][d] = (float)(__dsub_rn(posT[(3 * (size_t)i0 + d) * P + b], xj0[d]) + sh0[d] * cell.h[4 * d]);
#pragma unroll
                for (int s = 1; s < NS; s++) {
                    const int j = j0 + (((jm >> s) & 1u) ? s : 0);
#pragma unroll
                    for (int d = 0; d < 3; d++)
                        dj[s][d] = dj[0][d] - (float)(__ldcg(posT + (3 * (size_t)j + d) * P + b) - xj0[d]);
                }
            }
#pragma unroll
            for (int sj = 0; sj < NS; sj++) {
                if (!((jm >> sj) & 1u)) continue;
                float fjx = 0.0f, fjy = 0.0f, fjz = 0.0f;
#pragma unroll
                for (int si = 0; si < NS; si++) {
                    const int sp = si * NS + sj;
                    const bool coul = CM == kAnyPair ? (a.eflag[sp] & 2) != 0 : ((CM >> sp) & 1u) != 0;
                    const bool vdw = VM == kAnyPair ? (a.eflag[sp] & 1) != 0 : ((VM >> sp) & 1u) != 0;
                    if (CM != kAnyPair && !coul && !vdw) continue;  // a pair the masks never hold
                    if (!((mask >> sp) & 1u)) continue;
                    const float rx = dj[sj][0] + ei[si][0];
                    const float ry = dj[sj][1] + ei[si][1];
                    const float rz = dj[sj][2] + ei[si][2];
                    const float r2 = rx * rx + ry * ry + rz * rz;
                    if (r2 < rc2) {
                        const float r = r2 * rsqrtf(r2);
                        const float t = fminf(fmaxf(fmaf(r, dri, -rmd), 0.0f), tmax);
                        const float tr = __fadd_rn(t, kRound);
                        const int kn = __float_as_int(tr) - __float_as_int(kRound);
                        const float del = t - __fsub_rn(tr, kRound);
                        // with energies: the force and energy rows of an interval
                        // sit side by side (one cache line for both loads)
                        const float4 *row = tab + (a.toff[sp] + kn);
                        const float4 *rfe = a.tabfe + 2 * (a.toff[sp] + kn);
                        float dv = 0.0f;
                        float4 ecf = make_float4(0.f, 0.f, 0.f, 0.f), evf = ecf;
                        if (coul) {
                            float4 cf;
                            if (ENERGY) {
                                cf = ldg_keep(rfe + 2 * a.tstride);
                                ecf = ldg_keep(rfe + 2 * a.tstride + 1);
                            } else {
                                cf = ldg_keep(row + T_CDV0C * a.tstride);
                            }
                            dv = a.q2[sp] * (cf.x + del * (cf.y + del * (cf.z + del * cf.w)));
                        }
                        if (vdw) {
                            float4 cf;
                            if (ENERGY) {
                                cf = ldg_keep(rfe);
                                evf = ldg_keep(rfe + 1);
                            } else {
                                cf = ldg_keep(row + T_CDV0 * a.tstride);
                            }
                            dv += cf.x + del * (cf.y + del * (cf.z + del * cf.w));
                        }
                        const float fx = rx * dv, fy = ry * dv, fz = rz * dv;
                        fi[si][0] += fx;
                        fi[si][1] += fy;
                        fi[si][2] += fz;
                        fjx -= fx;
                        fjy -= fy;
                        fjz -= fz;
                        if (ENERGY) {
                            if (vdw) evs += evf.x + del * (evf.y + del * (evf.z + del * evf.w));
                            if (coul) ecs += a.q2[sp] * (ecf.x + del * (ecf.y + del * (ecf.z + del * ecf.w)));
                        }
                    }
                }
                // virial: r = dj + e_i, so sum r (x) f = dj (x) sum_i f (= -fj here)
                // + e_i (x) f_i, the latter once per chunk below
                if (ENERGY) {
                    pvs[0] -= dj[sj][0] * fjx;
                    pvs[1] -= dj[sj][1] * fjy;
                    pvs[2] -= dj[sj][2] * fjz;
                    pvs[3] -= dj[sj][0] * fjy;
                    pvs[4] -= dj[sj][0] * fjz;
                    pvs[5] -= dj[sj][1] * fjz;
                }
                if (fjx != 0.0f || fjy != 0.0f || fjz != 0.0f) {
                    const int j = j0 + sj;
                    atomicAdd(&a.forceT[(3 * (size_t)j + 0) * P + b], (double)fjx);
                    atomicAdd(&a.forceT[(3 * (size_t)j + 1) * P + b], (double)fjy);
                    atomicAdd(&a.forceT[(3 * (size_t)j + 2) * P + b], (double)fjz);
                }
            }
        }
        if (ENERGY) {
            // the e_i (x) f_i part of the virial: e_i is fixed over the chunk
#pragma unroll
            for (int s = 0; s < NS; s++) {
                pvs[0] += ei[s][0] * fi[s][0];
                pvs[1] += ei[s][1] * fi[s][1];
                pvs[2] += ei[s][2] * fi[s][2];
                pvs[3] += ei[s][0] * fi[s][1];
                pvs[4] += ei[s][0] * fi[s][2];
                pvs[5] += ei[s][1] * fi[s][2];
            }
        }
#pragma unroll
        for (int s = 0; s < NS; s++) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                double v = (double)fi[s][d];
                if (G < 32) v = warp_sum_strided(v, G);
                if ((G == 32 || sub == 0) && s < ni && v != 0.0) atomicAdd(&a.forceT[(3 * (size_t)(i0 + s) + d) * P + b], v);
            }
        }
        if (ENERGY) {
            sacc[0][threadIdx.x] += (double)evs;
            sacc[1][threadIdx.x] += (double)ecs;
#pragma unroll
            for (int c = 0; c < 6; c++) sacc[2 + c][threadIdx.x] += (double)pvs[c];
        }
    }
    if (ENERGY) {
        const int slot[8] = {S_VVDW, S_VCOUL, S_PXX, S_PYY, S_PZZ, S_PXY, S_PXZ, S_PYZ};
#pragma unroll
        for (int c = 0; c < 8; c++) {
            double t = sacc[c][threadIdx.x];
            if (G < 32) t = warp_sum_strided(t, G);
            if (G == 32 || sub == 0) atomicAdd(&a.acc[(size_t)b * S_NSLOT + slot[c]], t);
        }
    }
}

// ---------------------------------------------------------------------------
// launchers

// pass 0: reach, counts, row offsets and the molecule-pair total (tot[2]);
// pass 1: the fill, adding the active site pairs into tot[3].
cudaError_t launch_mol_list(pinyb200_ctx *c, const Cell &cell, const double *d_pos1, const double *d_xm,
                            const double *d_cutskin2, int pass, const int *gate, cudaStream_t st)
{
    if (!st) st = c->stream;
    const DeviceSystem &s = c->sys;
    const int threads = 256;
    int blocks = (c->nmol * 32 + threads - 1) / threads;
    const int maxb = c->sm_count * 8;
    if (blocks > maxb) blocks = maxb;
    if (blocks < 1) blocks = 1;
    const int use_xm = d_xm != nullptr;
    if (pass == 0)
        mol_reach_kernel<<<1, 1024, 0, st>>>(gate, c->nmol, c->d_mstart, d_pos1, d_xm, use_xm, d_cutskin2,
                                             s.npair_typ, c->d_reach);
#define MOL_LIST(NSV)                                                                                             \
    if (pass == 0) {                                                                                              \
        mol_list_kernel<0, NSV><<<blocks, threads, 0, st>>>(                                                      \
            gate, c->nmol, c->d_mstart, s.ntyp, d_pos1, d_xm, use_xm, cell, d_cutskin2, s.atm_typ, s.charge,      \
            s.inter_map, s.has_vdw, c->d_reach, c->d_mcount, nullptr, nullptr, nullptr, nullptr, 0, nullptr);    \
        mol_scan_kernel<<<1, 1024, 0, st>>>(gate, c->nmol, c->d_mcount, c->d_mrow, c->d_tot + 2);                 \
    } else {                                                                                                      \
        mol_list_kernel<1, NSV><<<blocks, threads, 0, st>>>(                                                      \
            gate, c->nmol, c->d_mstart, s.ntyp, d_pos1, d_xm, use_xm, cell, d_cutskin2, s.atm_typ, s.charge,      \
            s.inter_map, s.has_vdw, c->d_reach, c->d_mcount, c->d_mrow, c->d_mj, c->d_mmask, c->d_mmaskf,         \
            c->mlist_cap, (unsigned long long *)(c->d_tot + 3));                                                  \
    }
    if (c->mol_ns == 3) { MOL_LIST(3) }
    else if (c->mol_ns == 4) { MOL_LIST(4) }
    else return cudaErrorInvalidValue;
#undef MOL_LIST
    return cudaGetLastError();
}

// Site lists from the molecule list.  pass 0: counts, row offsets, totals
// (tot[0], tot[1]); pass 1: the fill.
cudaError_t launch_site_from_mol(pinyb200_ctx *c, int pass, const int *gate, cudaStream_t st)
{
    if (!st) st = c->stream;
    const int threads = 256;
    int blocks = (c->nmol * 32 + threads - 1) / threads;
    const int maxb = c->sm_count * 8;
    if (blocks > maxb) blocks = maxb;
    if (blocks < 1) blocks = 1;
    const int natm = c->sys.natm;
#define SITE_LIST(NSV)                                                                                             \
    if (pass == 0) {                                                                                               \
        site_count_kernel<NSV><<<blocks, threads, 0, st>>>(gate, c->nmol, natm, c->d_mstart, c->d_mrow, c->d_mmaskf, \
                                                           c->d_mmask, c->mlist_cap, c->d_count);                 \
        scan_kernel<<<1, 1024, 0, st>>>(gate, natm, c->d_count, c->d_row, c->d_rowA, c->d_tot);                   \
    } else {                                                                                                       \
        site_fill_kernel<NSV><<<blocks, threads, 0, st>>>(gate, c->nmol, c->d_mstart, c->d_mrow, c->d_mj,          \
                                                          c->d_mmaskf, c->d_mmask, c->mlist_cap, c->d_row,        \
                                                          c->d_rowA, c->d_col, c->d_colA, c->list_cap);           \
    }
    if (c->mol_ns == 3) { SITE_LIST(3) }
    else if (c->mol_ns == 4) { SITE_LIST(4) }
    else return cudaErrorInvalidValue;
#undef SITE_LIST
    return cudaGetLastError();
}

template <typename R, int P, int NS>
static void launch_mol_t(pinyb200_ctx *c, const MolArgs &a, const Cell &cell, bool fast)
{
    const int threads = 128;
    long long blocks = ((long long)c->chunk_cap * 32 + threads - 1) / threads;
    const long long maxb = (long long)c->sm_count * c->pair_blocks_per_sm;
    if (blocks > maxb) blocks = maxb;
    if (blocks < 1) blocks = 1;
    dim3 grid((unsigned)blocks, P > 32 ? P / 32 : 1);
    if constexpr (sizeof(R) == 4) {
        if (fast) {
            if (a.energy) mol_pair_kernel<R, P, NS, true, true><<<grid, threads, 0, c->stream>>>(a, cell);
            else mol_pair_kernel<R, P, NS, true, false><<<grid, threads, 0, c->stream>>>(a, cell);
            return;
        }
    }
    if (a.energy) mol_pair_kernel<R, P, NS, false, true><<<grid, threads, 0, c->stream>>>(a, cell);
    else mol_pair_kernel<R, P, NS, false, false><<<grid, threads, 0, c->stream>>>(a, cell);
}

template <typename R, int NS>
static cudaError_t launch_mol_ns(pinyb200_ctx *c, const MolArgs &a, const Cell &cell, bool fast)
{
    switch (c->P) {
    case 1: launch_mol_t<R, 1, NS>(c, a, cell, fast); break;
    case 2: launch_mol_t<R, 2, NS>(c, a, cell, fast); break;
    case 4: launch_mol_t<R, 4, NS>(c, a, cell, fast); break;
    case 8: launch_mol_t<R, 8, NS>(c, a, cell, fast); break;
    case 16: launch_mol_t<R, 16, NS>(c, a, cell, fast); break;
    case 32: launch_mol_t<R, 32, NS>(c, a, cell, fast); break;
    case 64: launch_mol_t<R, 64, NS>(c, a, cell, fast); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_mol_pair(pinyb200_ctx *c, const Cell &cell, bool energy)
{
    const DeviceSystem &s = c->sys;
    MolArgs a;
    a.nchunk = c->d_nchunk;
    a.chunk = c->d_chunk;
    a.bad = c->d_ls ? (const int *)((const char *)c->d_ls + offsetof(ListState, overflow)) : nullptr;
    a.mj = c->d_mj;
    a.mask = c->d_mmask;
    a.mstart = c->d_mstart;
    a.ntyp = s.ntyp;
    a.npt = s.npair_typ;
    a.nuniq = s.nuniq;
    a.nsplin = s.nsplin;
    a.posT = c->d_posT;
    a.pimd = c->P > 1;
    a.xmod = c->P > 1 ? c->d_xmod : c->d_posT;  // P == 1: [natm][3][1] is [natm][3]
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
    if (c->precision == PINYB200_FP64) {
        a.tab = s.tab64;
        if (c->mol_ns == 3) return launch_mol_ns<double, 3>(c, a, cell, false);
        return launch_mol_ns<double, 4>(c, a, cell, false);
    }
    a.tab = s.tab32;
    if (c->mol_ns == 3) return launch_mol_ns<float, 3>(c, a, cell, true);
    return launch_mol_ns<float, 4>(c, a, cell, true);
}


template <int P, int NS, unsigned CM, unsigned VM>
static void launch_mix_pattern(pinyb200_ctx *c, const MixArgs &a, const Cell &cell, bool energy, dim3 grid)
{
    const int threads = 128;
    if (energy) {
        carveout_pref((const void *)mol_pair_mixed_kernel<P, NS, true, CM, VM>, c->pair_carveout);
        mol_pair_mixed_kernel<P, NS, true, CM, VM><<<grid, threads, 0, c->stream>>>(a, cell);
    } else {
        carveout_pref((const void *)mol_pair_mixed_kernel<P, NS, false, CM, VM>, c->pair_carveout);
        mol_pair_mixed_kernel<P, NS, false, CM, VM><<<grid, threads, 0, c->stream>>>(a, cell);
    }
}

template <int P, int NS>
static void launch_mix_t(pinyb200_ctx *c, const MixArgs &a, const Cell &cell, bool energy)
{
    const int threads = 128;
    long long blocks = ((long long)c->chunk_cap * 32 + threads - 1) / threads;
    const long long maxb = (long long)c->sm_count * c->pair_blocks_per_sm;
    if (blocks > maxb) blocks = maxb;
    if (blocks < 1) blocks = 1;
    dim3 grid((unsigned)blocks, P > 32 ? P / 32 : 1);
    // the site-pair table pattern of the molecule, from the per-pair flags
    unsigned cm = 0, vm = 0;
    for (int k = 0; k < NS * NS; k++) {
        if (c->mix_eflag[k] & 2) cm |= 1u << k;
        if (c->mix_eflag[k] & 1) vm |= 1u << k;
    }
    if (NS == 4 && cm == kTip4pCoul && vm == kTip4pVdw)
        launch_mix_pattern<P, NS, kTip4pCoul, kTip4pVdw>(c, a, cell, energy, grid);
    else if (NS == 3 && cm == kSpcCoul && vm == kSpcVdw)
        launch_mix_pattern<P, NS, kSpcCoul, kSpcVdw>(c, a, cell, energy, grid);
    else
        launch_mix_pattern<P, NS, kAnyPair, kAnyPair>(c, a, cell, energy, grid);
}

template <int NS>
static cudaError_t launch_mix_ns(pinyb200_ctx *c, const MixArgs &a, const Cell &cell, bool energy)
{
    switch (c->P) {
    case 1: launch_mix_t<1, NS>(c, a, cell, energy); break;
    case 2: launch_mix_t<2, NS>(c, a, cell, energy); break;
    case 4: launch_mix_t<4, NS>(c, a, cell, energy); break;
    case 8: launch_mix_t<8, NS>(c, a, cell, energy); break;
    case 16: launch_mix_t<16, NS>(c, a, cell, energy); break;
    case 32: launch_mix_t<32, NS>(c, a, cell, energy); break;
    case 64: launch_mix_t<64, NS>(c, a, cell, energy); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// The MIXED kernel with combined per-site-pair tables (pinyb200_ctx::mix_ok).
cudaError_t launch_mol_pair_mixed(pinyb200_ctx *c, const Cell &cell, bool energy)
{
    const DeviceSystem &s = c->sys;
    MixArgs a;
    a.nchunk = c->d_nchunk;
    a.chunk = c->d_chunk;
    a.bad = c->d_ls ? (const int *)((const char *)c->d_ls + offsetof(ListState, overflow)) : nullptr;
    a.mj = c->d_mj;
    a.mask = c->d_mmask;
    a.mstart = c->d_mstart;
    a.ntyp = s.ntyp;
    a.nuniq = s.nuniq;
    a.nsplin = s.nsplin;
    a.stride = c->mol_stride;
    a.posT = c->d_posT;
    a.xmod = c->P > 1 ? c->d_xmod : c->d_posT;
    a.atm_typ = s.atm_typ;
    a.charge = s.charge;
    a.inter_map = s.inter_map;
    a.cutoff = s.cutoff;
    a.rmin = s.rmin;
    a.dri = s.dri;
    a.has_vdw = s.has_vdw;
    a.tab = s.tab32;
    a.tabfe = c->d_tabfe;
    a.forceT = c->d_forceT;
    a.acc = c->d_acc;
    for (int k = 0; k < 16; k++) {
        a.toff[k] = c->mix_toff[k];
        a.q2[k] = c->mix_q2[k];
        a.eflag[k] = c->mix_eflag[k];
    }
    a.tstride = s.nuniq * s.nsplin;
    a.rc2 = c->mix_rc2;
    a.dri_f = c->mix_dri;
    a.rmd = c->mix_rmd;
    a.tmax = c->mix_tmax;
    if (c->mol_ns == 3) return launch_mix_ns<3>(c, a, cell, energy);
    return launch_mix_ns<4>(c, a, cell, energy);
}

}  // namespace pinyb200
