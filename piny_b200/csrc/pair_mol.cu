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
#include <algorithm>
#include <map>
#include <tuple>
#include <vector>
#include <cmath>
#include <cstddef>
#include <string>

#include "boxtab.cuh"
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
// bound of the distance between the images of the two site-0 bead-1
// positions exceeds the reach R = max cutskin + 2 e, e = largest distance of
// a bead-1 site from its molecule's site 0.  Every image shift period /
// period_pimd applies is a lattice vector and no image of a site pair is
// nearer than the nearest image less 2 e, so a pair so skipped has no site
// pair inside max cutskin.  The bound, from the wrapped fractional
// separation t along each cell axis times the lattice-plane spacing w: the
// exact minimum-image distance sqrt(sum (t w)^2) in an orthorhombic cell
// (where the axes separate), the largest t w otherwise.  It is evaluated in
// FP32 from fractional positions rounded to FP32, against R widened by more
// than that rounding can move it (bound_slack): a filter that only ever lets
// extra pairs through to the exact FP64 test.

// Plane spacings of the cell, whether it is orthorhombic, and the widened
// reach the FP32 bound is compared with (squared; set on the device).
struct CellPlanes {
    double w[3];
    int ortho;
};

// R plus the FP32 rounding allowance of the bound: fractional positions in
// [0, 1) rounded to FP32 (2^-25), their difference and wrap (2^-24 each),
// times w, with a factor 20 to spare; 1e-6 Bohr absolute.
__host__ __device__ inline double bound_slack(const CellPlanes &pl)
{
    return 4e-6 * fmax(pl.w[0], fmax(pl.w[1], pl.w[2])) + 1e-6;
}

// Squared bound from the fractional separations (FP32).
__device__ __forceinline__ float bound2_frac(float t0, float t1, float t2, const CellPlanes &pl)
{
    t0 = fabsf(t0 - rintf(t0)) * (float)pl.w[0];
    t1 = fabsf(t1 - rintf(t1)) * (float)pl.w[1];
    t2 = fabsf(t2 - rintf(t2)) * (float)pl.w[2];
    return pl.ortho ? t0 * t0 + t1 * t1 + t2 * t2 : fmaxf(t0 * t0, fmaxf(t1 * t1, t2 * t2));
}

// The reach R (above) into *reach.  Each block's maxima go into acc[0] and
// acc[2] by atomicMax on their bit patterns (non-negative doubles order as
// their bits; fmax has already dropped any NaN); the last block to finish
// turns them into R and clears acc[0..3] for the next launch.
__global__ void __launch_bounds__(256) mol_reach_kernel(const int *__restrict__ gate, int nmol,
                                                         const int *__restrict__ mstart,
                                                         const double *__restrict__ pos1,
                                                         const double *__restrict__ cs, int npt,
                                                         unsigned long long *__restrict__ acc,
                                                         double *__restrict__ reach)
{
    if (gate && *gate == 0) return;
    __shared__ double red[2][8];
    __shared__ int last;
    double ext = 0.0, cmax = 0.0;
    if (blockIdx.x == 0)
        for (int k = threadIdx.x; k < npt; k += blockDim.x) cmax = fmax(cmax, cs[k]);
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < nmol; m += gridDim.x * blockDim.x) {
        const int i0 = mstart[m], i1 = mstart[m + 1];
        const double *x0 = pos1 + 3 * (size_t)i0;
        for (int i = i0 + 1; i < i1; i++) {
            const double *xi = pos1 + 3 * (size_t)i;
            const double ex = xi[0] - x0[0], ey = xi[1] - x0[1], ez = xi[2] - x0[2];
            ext = fmax(ext, sqrt(ex * ex + ey * ey + ez * ez));
        }
    }
    for (int o = 16; o >= 1; o >>= 1) {
        ext = fmax(ext, __shfl_xor_sync(0xffffffffu, ext, o));
        cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][w] = ext;
        red[1][w] = cmax;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); k++) {
            ext = fmax(ext, red[0][k]);
            cmax = fmax(cmax, red[1][k]);
        }
        atomicMax(&acc[0], (unsigned long long)__double_as_longlong(ext));
        atomicMax(&acc[2], (unsigned long long)__double_as_longlong(cmax));
        __threadfence();
        last = atomicAdd(&acc[3], 1ull) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        const double e = __longlong_as_double((long long)atomicExch(&acc[0], 0ull));
        const double c2 = __longlong_as_double((long long)atomicExch(&acc[2], 0ull));
        atomicExch(&acc[3], 0ull);
        // rounding of the distances and of the criterion: a generous margin
        *reach = (sqrt(c2) + 2.0 * e) * (1.0 + 1e-12) + 1e-9;
    }
}

// Blocks of mol_reach_kernel.
static int reach_blocks(const pinyb200_ctx *c) { return std::max(1, std::min((c->nmol + 255) / 256, 2 * c->sm_count)); }

// Wrapped fractional site-0 bead-1 position of every molecule (FP32), and
// with cells, its cell and the cells' populations (ccnt, zeroed before).
__global__ void __launch_bounds__(256) mol_frac_kernel(const int *__restrict__ gate, int nmol,
                                                       const int *__restrict__ mstart, const double *__restrict__ pos1,
                                                       Cell cell, int na, int nb, int nc, float4 *__restrict__ msf,
                                                       int *__restrict__ mcell, int *__restrict__ ccnt)
{
    if (gate && *gate == 0) return;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmol) return;
    const double *x = pos1 + 3 * (size_t)mstart[m];
    const int n[3] = {na, nb, nc};
    float f[3];
    int k[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        double sd = x[0] * cell.hi[d] + x[1] * cell.hi[3 + d] + x[2] * cell.hi[6 + d];
        sd -= floor(sd);
        f[d] = (float)sd;
        int q = (int)(sd * n[d]);
        if (!(q >= 0 && q < n[d])) q = q >= n[d] ? n[d] - 1 : 0;  // sd == 1 after rounding, or not finite
        k[d] = q;
    }
    msf[m] = make_float4(f[0], f[1], f[2], 0.0f);
    if (mcell) {
        const int id = (k[2] * nb + k[1]) * na + k[0];
        mcell[m] = id;
        atomicAdd(&ccnt[id], 1);
    }
}

// PINY's list criterion for every site pair of one molecule pair (mi with
// sites i0.., mj with sites j0..): r^2 < cutskin^2 of the pair type on the
// bead-1 separation and PINY's image (period / period_pimd with the mode-1
// separation), in FP64 with PINY's operation order (verlist_create.c:
// 373-503).  maskf gets bit si * NS + sj for every site pair inside, mask
// for those that also carry a force (a vdW table or a charge product); the
// molecules are identical, so cutskin^2 and that flag come per (si, sj)
// from tcs2 / tact.
//
// The image.  In a cubic cell PINY's shift along an axis is -NINT of
// (separation * hi), the separation being the mode-1 one (period_pimd) or
// the bead-1 one (period).  Rounded subtraction and multiplication by
// hi > 0 are monotone, and so is NINT, so over all site pairs of the pair
// that NINT lies between its values at the two ends of the range of the
// separation, formed from the extreme site coordinates of the two
// molecules.  When those agree, every site pair has that NINT and it is
// applied once; otherwise each site pair evaluates its own.  The shifted
// separations are bit for bit PINY's either way.
template <int NS, bool XM>
__device__ __forceinline__ void mol_pair_masks(int i0, int ni, int j0, int nj, const double *__restrict__ pos1,
                                               const double *__restrict__ xm, const Cell &cell,
                                               const double *tcs2, const unsigned char *tact, unsigned &mask,
                                               unsigned &maskf)
{
    // mj's sites once into registers (each lane tests its own mj; mi is the
    // same across the warp, so its loads are broadcasts)
    double xj[NS][3], mj[NS][3];
#pragma unroll
    for (int sj = 0; sj < NS; sj++) {
        const int j = j0 + (sj < nj ? sj : 0);
#pragma unroll
        for (int d = 0; d < 3; d++) {
            xj[sj][d] = pos1[3 * j + d];
            if (XM) mj[sj][d] = xm[3 * j + d];
        }
    }
    // one image for the whole pair (cubic cell), when the range allows
    bool uni = cell.cubic;
    double nn[3] = {0.0, 0.0, 0.0};
    if (uni) {
        const double *ai = (XM ? xm : pos1) + 3 * (size_t)i0;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            double amin = ai[d], amax = ai[d];
            for (int si = 1; si < ni; si++) {
                amin = fmin(amin, ai[3 * si + d]);
                amax = fmax(amax, ai[3 * si + d]);
            }
            double bmin = XM ? mj[0][d] : xj[0][d], bmax = bmin;
#pragma unroll
            for (int sj = 1; sj < NS; sj++)
                if (sj < nj) {
                    const double b = XM ? mj[sj][d] : xj[sj][d];
                    bmin = fmin(bmin, b);
                    bmax = fmax(bmax, b);
                }
            const double hid = cell.hi[4 * d];
            const double lo = nint_rn(__dmul_rn(__dsub_rn(amin, bmax), hid));
            const double hi = nint_rn(__dmul_rn(__dsub_rn(amax, bmin), hid));
            uni = uni && lo == hi;
            nn[d] = lo;
        }
    }
    double sh[3];  // the pair's shift (period_pimd's -NINT * h)
#pragma unroll
    for (int d = 0; d < 3; d++) sh[d] = __dmul_rn(-nn[d], cell.h[4 * d]);
#pragma unroll 1
    for (int si = 0; si < ni; si++) {
        const int i = i0 + si;
        const double xi = pos1[3 * i], yi = pos1[3 * i + 1], zi = pos1[3 * i + 2];
        double mxi = 0.0, myi = 0.0, mzi = 0.0;
        if (XM && !uni) {
            mxi = xm[3 * i];
            myi = xm[3 * i + 1];
            mzi = xm[3 * i + 2];
        }
#pragma unroll
        for (int sj = 0; sj < NS; sj++) {
            if (sj >= nj) break;
            double dx = __dsub_rn(xi, xj[sj][0]);
            double dy = __dsub_rn(yi, xj[sj][1]);
            double dz = __dsub_rn(zi, xj[sj][2]);
            if (uni) {
                if (XM) {
                    dx = __dadd_rn(dx, sh[0]);
                    dy = __dadd_rn(dy, sh[1]);
                    dz = __dadd_rn(dz, sh[2]);
                } else {
                    dx = __dmul_rn(__dsub_rn(__dmul_rn(dx, cell.hi[0]), nn[0]), cell.h[0]);
                    dy = __dmul_rn(__dsub_rn(__dmul_rn(dy, cell.hi[4]), nn[1]), cell.h[4]);
                    dz = __dmul_rn(__dsub_rn(__dmul_rn(dz, cell.hi[8]), nn[2]), cell.h[8]);
                }
            } else if (XM) {
                period_pimd_exact(dx, dy, dz, __dsub_rn(mxi, mj[sj][0]), __dsub_rn(myi, mj[sj][1]),
                                  __dsub_rn(mzi, mj[sj][2]), cell);
            } else {
                period_exact(dx, dy, dz, cell);
            }
            const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
            const int k = si * NS + sj;
            if (r2 < tcs2[k]) {
                maskf |= 1u << k;
                if (tact[k]) mask |= 1u << k;
            }
        }
    }
}

// Arguments of the molecule-pair list kernels.  count: per molecule row
// (pass 0); row, mj, mask, maskf, cap, nsite: the fill (pass 1).  ent
// (ent_cap entries, nent counted): the pairs the count pass found, written
// as it goes when they fit, (mi, index in the row, mj, mask | maskf << 16),
// so that the fill is a scatter; a count pass that found more computes the
// fill again.
struct MolListArgs {
    const int *mstart;
    int stride;  // sites per molecule when molecule m starts at site m * stride, else 0
    int ntyp;
    const double *pos1, *xm;  // bead-1 positions; mode-1 positions or nullptr (one bead)
    const float4 *msf;        // wrapped fractional site-0 bead-1 positions
    const double *cutskin2;
    const int *atm_typ;
    const double *charge;
    const int *inter_map, *has_vdw;
    const double *reach;
    int *count;
    const int *row;
    int *mj;
    unsigned *mask, *maskf;
    long long cap;
    unsigned long long *nsite;
    int4 *ent;
    long long ent_cap;
    unsigned long long *nent;
};

// Per (si, sj) of the (identical) molecules: cutskin^2 of the pair type
// and whether the pair carries a force; NS * NS threads of the block.
template <int NS>
__device__ __forceinline__ void mol_site_tables(const MolListArgs &a, double *tcs2, unsigned char *tact)
{
    const int t = threadIdx.x;
    if (t < NS * NS) {
        const int n0 = a.mstart[1] - a.mstart[0];
        const int si = min(t / NS, n0 - 1), sj = min(t % NS, n0 - 1);
        const int pt = pair_type(a.atm_typ[si], a.atm_typ[sj], a.ntyp);
        tcs2[t] = a.cutskin2[pt];
        tact[t] = (a.has_vdw[a.inter_map[pt]] || a.charge[si] * a.charge[sj] != 0.0) ? 1 : 0;
    }
}

// Candidates of one row that passed the bound wait in a per-warp queue (a
// ring in shared memory) and are tested 32 at a time, one per lane, so the
// site-pair loop runs on full warps: on a dense row only a few candidates in
// a warp's 32 pass, and a lane-per-candidate test would keep the whole warp
// in the site-pair loop for each of them.  The queue keeps the candidates'
// order, so a row lists its pairs in the order they were enumerated.  The
// kernels bound four groups of 32 candidates per step (their loads in
// flight together) and call the test from one place, so that its code,
// which is most of the kernel, appears once.
#define PINYB200_QUEUE 256  // ring entries per warp (>= 31 left over + 4 x 32 appended)

struct MolQueue {
    int *q;    // PINYB200_QUEUE entries
    int head;  // first waiting entry
    int nq;    // entries waiting
};

// Append the lanes with pass set, in lane order.
__device__ __forceinline__ void mol_queue_append(MolQueue &Q, bool pass, int mj)
{
    const int lane = threadIdx.x & 31;
    const unsigned bp = __ballot_sync(0xffffffffu, pass);
    if (pass) Q.q[(Q.head + Q.nq + __popc(bp & ((1u << lane) - 1u))) & (PINYB200_QUEUE - 1)] = mj;
    Q.nq += __popc(bp);
}

// Test every full group of 32 waiting candidates, and with all, the rest.
template <int FILL, int NS, bool XM>
__device__ __forceinline__ void mol_queue_drain(MolQueue &Q, bool all, int mi, int i0, int ni, const MolListArgs &a,
                                                const Cell &cell, const double *tcs2, const unsigned char *tact,
                                                int &n, long long w0, unsigned long long &sites)
{
    const int lane = threadIdx.x & 31;
    __syncwarp();
    while (Q.nq >= 32 || (all && Q.nq > 0)) {
        const int k = min(Q.nq, 32);
        unsigned mask = 0, maskf = 0;
        int mj = 0;
        if (lane < k) {
            mj = Q.q[(Q.head + lane) & (PINYB200_QUEUE - 1)];
            const int j0 = a.stride ? mj * a.stride : a.mstart[mj];
            const int nj = a.stride ? a.stride : a.mstart[mj + 1] - j0;
            mol_pair_masks<NS, XM>(i0, ni, j0, nj, a.pos1, a.xm, cell, tcs2, tact, mask, maskf);
        }
        Q.head = (Q.head + k) & (PINYB200_QUEUE - 1);
        Q.nq -= k;
        const bool keep = maskf != 0;
        const unsigned bk = __ballot_sync(0xffffffffu, keep);
        const int below = __popc(bk & ((1u << lane) - 1u));
        if (FILL) {
            if (keep) {
                const long long p = w0 + n + below;
                if (p < a.cap) {
                    a.mj[p] = mj;
                    a.mask[p] = mask;
                    a.maskf[p] = maskf;
                }
            }
            sites += __popc(mask);
        } else if (bk) {
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(a.nent, (unsigned long long)__popc(bk));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (keep && base + __popc(bk) <= (unsigned long long)a.ent_cap)
                a.ent[base + below] = make_int4(mi, n + below, mj, (int)(mask | (maskf << 16)));
        }
        n += __popc(bk);
    }
    __syncwarp();
}

// The fill pass computes only when the count pass's pairs did not fit.
__device__ __forceinline__ bool fill_from_entries(const MolListArgs &a)
{
    return *a.nent <= (unsigned long long)a.ent_cap;
}

// The sweep: one warp per molecule row mi over every mj < mi, rows taken
// in pairs (r, nmol - 1 - r) so that every warp sweeps nmol - 1 candidates.
template <int FILL, int NS, bool XM>
__global__ void __launch_bounds__(256, 2) mol_list_kernel(const int *__restrict__ gate, int nmol, Cell cell,
                                                          CellPlanes pl, MolListArgs a,
                                                          const int *__restrict__ cells)
{
    if (gate && *gate == 0) return;  // device list update: no rebuild this step
    if (cells && *cells) return;     // the link-cell kernel builds this list
    if (FILL && fill_from_entries(a)) return;
    __shared__ int queue[8][PINYB200_QUEUE];
    __shared__ double tcs2[NS * NS];
    __shared__ unsigned char tact[NS * NS];
    mol_site_tables<NS>(a, tcs2, tact);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    MolQueue Q{queue[threadIdx.x >> 5], 0, 0};
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const double Rw = *a.reach + bound_slack(pl);
    const float R2 = (float)(Rw * Rw);
    unsigned long long sites = 0;
    for (int rr = warp; 2 * rr < nmol; rr += nwarps) {
        for (int h = 0; h < 2; h++) {
            const int mi = h ? nmol - 1 - rr : rr;
            if (h && mi == rr) break;
            const int i0 = a.mstart[mi], ni = a.mstart[mi + 1] - i0;
            const float4 si = a.msf[mi];
            int n = 0;
            const long long w0 = FILL ? a.row[mi] : 0;
            for (int m0 = 0;; m0 += 4 * 32) {
                const bool last = m0 >= mi;
                if (!last) {
                    // four candidates per lane in flight, then their bounds in order
                    float4 sj[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int mj = m0 + 32 * u + lane;
                        if (mj < mi) sj[u] = a.msf[mj];
                    }
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int mj = m0 + 32 * u + lane;
                        mol_queue_append(Q, mj < mi && !(bound2_frac(si.x - sj[u].x, si.y - sj[u].y,
                                                                     si.z - sj[u].z, pl) > R2), mj);
                    }
                }
                mol_queue_drain<FILL, NS, XM>(Q, last, mi, i0, ni, a, cell, tcs2, tact, n, w0, sites);
                if (last) break;
            }
            if (!FILL && lane == 0) a.count[mi] = n;
        }
    }
    if (FILL) {
        for (int o = 16; o >= 1; o >>= 1) sites += __shfl_xor_sync(0xffffffffu, sites, o);
        if (lane == 0) atomicAdd(a.nsite, sites);
    }
}

// The fill from the count pass's entries: every pair to its row position.
__global__ void __launch_bounds__(256) mol_scatter_kernel(const int *__restrict__ gate, MolListArgs a)
{
    if (gate && *gate == 0) return;
    if (!fill_from_entries(a)) return;  // the fill kernels compute
    const long long ne = (long long)*a.nent;
    unsigned long long sites = 0;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < ne;
         e += (long long)gridDim.x * blockDim.x) {
        const int4 v = a.ent[e];
        const long long p = (long long)a.row[v.x] + v.y;
        const unsigned mask = (unsigned)v.w & 0xffffu, maskf = (unsigned)v.w >> 16;
        if (p < a.cap) {
            a.mj[p] = v.z;
            a.mask[p] = mask;
            a.maskf[p] = maskf;
        }
        sites += __popc(mask);
    }
    for (int o = 16; o >= 1; o >>= 1) sites += __shfl_xor_sync(0xffffffffu, sites, o);
    if ((threadIdx.x & 31) == 0 && sites) atomicAdd(a.nsite, sites);
}

// ---------------------------------------------------------------------------
// Link cells for the molecule-pair list.
//
// PINY builds its Verlet list from a link-cell list by default (update_type
// lnk_list: make_lnk_lst.c:37, lnk_ver_gen_pad at verlist_control.c:1738).
// Here the molecules are binned by the wrapped fractional coordinates of
// their site-0 bead-1 position into n_a x n_b x n_c cells (each n >= 5)
// whose edges, measured between lattice planes, are at least half the reach
// R of the bound above.  A pair the bound keeps has, along each axis, a
// wrapped fractional separation of at most R / plane spacing <= 2 / n, so
// its cells are at most 2 apart on each axis: the 5 x 5 x 5 cells around a
// molecule's own hold every candidate.  One block per home cell stages the
// flattened candidate list of those 125 cells (molecule index and FP32
// fractional position) in shared memory, a batch at a time; warps take the
// home molecules, lanes the staged candidates mj < mi, and the pairs that
// pass the bound go through the warp queue to mol_pair_masks, the criterion
// of the sweep.  The list holds exactly the sweep's pairs, each row in the
// order of the neighbour cells and, within a cell, of molecule index (the
// members of each cell are sorted), so every build of the same positions
// gives the same list.  The grid is planned at each host build with room for
// R to grow by 15 %; a device rebuild whose R no longer fits the cells, or
// whose fullest cell holds more than PINYB200_CELL_HOME molecules, runs the
// sweep instead (cell_decide_kernel).

#define PINYB200_CELL_BATCH 4096  // candidate molecules staged at a time
#define PINYB200_CELL_HOME 256    // most molecules of a home cell the kernel keeps row counters for

// Molecules into their cells' ranges (in arrival order; fill: ncell
// counters, zeroed before).
__global__ void __launch_bounds__(256) cell_scatter_kernel(const int *__restrict__ gate, int nmol,
                                                           const int *__restrict__ mcell,
                                                           const int *__restrict__ coff, int *__restrict__ fill,
                                                           int *__restrict__ cmol)
{
    if (gate && *gate == 0) return;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmol) return;
    const int id = mcell[m];
    cmol[coff[id] + atomicAdd(&fill[id], 1)] = m;
}

// Each cell's members in index order (one warp per cell, rank by count of
// smaller indices); cells fuller than the kernel takes are left as they are.
__global__ void __launch_bounds__(256) cell_sort_kernel(const int *__restrict__ gate, int ncell,
                                                        const int *__restrict__ coff, const int *__restrict__ in,
                                                        int *__restrict__ out)
{
    if (gate && *gate == 0) return;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int c = warp; c < ncell; c += nwarps) {
        const int c0 = coff[c], len = coff[c + 1] - c0;
        if (len > PINYB200_CELL_HOME) continue;
        for (int k = lane; k < len; k += 32) {
            const int m = in[c0 + k];
            int r = 0;
            for (int u = 0; u < len; u++) r += in[c0 + u] < m;
            out[c0 + r] = m;
        }
    }
}

// Whether the cells serve this build: R within the cells' design (R at most
// twice the narrowest cell edge) and no cell fuller than the kernel takes.
__global__ void __launch_bounds__(1024) cell_decide_kernel(const int *__restrict__ gate, int ncell,
                                                           const int *__restrict__ coff,
                                                           const double *__restrict__ reach, double edge2,
                                                           int *__restrict__ ok)
{
    if (gate && *gate == 0) return;
    __shared__ int full;
    if (threadIdx.x == 0) full = 0;
    __syncthreads();
    int mx = 0;
    for (int c = threadIdx.x; c < ncell; c += blockDim.x) mx = max(mx, coff[c + 1] - coff[c]);
    atomicMax(&full, mx);
    __syncthreads();
    if (threadIdx.x == 0) *ok = (*reach * (1.0 + 1e-9) <= edge2 && full <= PINYB200_CELL_HOME) ? 1 : 0;
}

template <int FILL, int NS, bool XM>
__global__ void __launch_bounds__(256, 2) mol_list_cell_kernel(const int *__restrict__ gate,
                                                               const int *__restrict__ ok, int na, int nb, int nc,
                                                               const int *__restrict__ coff,
                                                               const int *__restrict__ cmol, CellPlanes pl,
                                                               Cell cell, MolListArgs a)
{
    if (gate && *gate == 0) return;
    if (!*ok) return;  // the sweep builds this list
    if (FILL && fill_from_entries(a)) return;
    extern __shared__ float4 cell_smem[];
    float4 *sx = cell_smem;  // [BATCH] fractional position, molecule index in .w
    __shared__ int nbase[125], nstart[126];  // each neighbour cell: start in cmol, start in the flattened list
    __shared__ int hcnt[PINYB200_CELL_HOME];
    __shared__ int queue[8][PINYB200_QUEUE];
    __shared__ double tcs2[NS * NS];
    __shared__ unsigned char tact[NS * NS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    MolQueue Q{queue[warp], 0, 0};
    const int home = blockIdx.x;
    const int ha = home % na, hb = (home / na) % nb, hc = home / (na * nb);
    const int h0 = coff[home], nhome = coff[home + 1] - h0;
    if (nhome == 0) return;
    mol_site_tables<NS>(a, tcs2, tact);
    if (threadIdx.x < 125) {
        const int k = threadIdx.x;
        const int da = k % 5 - 2, db = (k / 5) % 5 - 2, dc = k / 25 - 2;
        const int cid = ((hc + dc + nc) % nc * nb + (hb + db + nb) % nb) * na + (ha + da + na) % na;
        nbase[k] = coff[cid];
        nstart[k + 1] = coff[cid + 1] - coff[cid];
    }
    for (int k = threadIdx.x; k < PINYB200_CELL_HOME; k += blockDim.x) hcnt[k] = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        nstart[0] = 0;
        for (int k = 1; k <= 125; k++) nstart[k] += nstart[k - 1];
    }
    __syncthreads();
    const int total = nstart[125];
    const double Rw = *a.reach + bound_slack(pl);
    const float R2 = (float)(Rw * Rw);
    unsigned long long sites = 0;
    for (int b0 = 0; b0 < total; b0 += PINYB200_CELL_BATCH) {
        const int nst = min(PINYB200_CELL_BATCH, total - b0);
        __syncthreads();  // the previous batch is done with the staging buffer
        for (int e = threadIdx.x; e < nst; e += blockDim.x) {
            const int f = b0 + e;
            int lo = 0, hi = 125;  // the neighbour cell k with nstart[k] <= f < nstart[k + 1]
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (nstart[mid] <= f) lo = mid;
                else hi = mid;
            }
            const int mj = cmol[nbase[lo] + f - nstart[lo]];
            float4 v = a.msf[mj];
            v.w = __int_as_float(mj);
            sx[e] = v;
        }
        __syncthreads();
        for (int hk = warp; hk < nhome; hk += nwarp) {
            const int mi = cmol[h0 + hk];
            const int i0 = a.mstart[mi], ni = a.mstart[mi + 1] - i0;
            const float4 si = a.msf[mi];
            int n = hcnt[hk];
            const long long w0 = FILL ? a.row[mi] : 0;
            for (int q0 = 0;; q0 += 4 * 32) {
                const bool last = q0 >= nst;
                if (!last) {
                    float4 sj[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int e = q0 + 32 * u + lane;
                        sj[u] = e < nst ? sx[e] : make_float4(0.f, 0.f, 0.f, __int_as_float(0x7fffffff));
                    }
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int mj = __float_as_int(sj[u].w);  // past the batch: INT_MAX, never < mi
                        mol_queue_append(Q, mj < mi && !(bound2_frac(si.x - sj[u].x, si.y - sj[u].y,
                                                                     si.z - sj[u].z, pl) > R2), mj);
                    }
                }
                mol_queue_drain<FILL, NS, XM>(Q, last, mi, i0, ni, a, cell, tcs2, tact, n, w0, sites);
                if (last) break;
            }
            if (lane == 0) hcnt[hk] = n;
            __syncwarp();
        }
    }
    __syncthreads();
    if (!FILL)
        for (int hk = threadIdx.x; hk < nhome; hk += blockDim.x) a.count[cmol[h0 + hk]] = hcnt[hk];
    if (FILL) {
        for (int o = 16; o >= 1; o >>= 1) sites += __shfl_xor_sync(0xffffffffu, sites, o);
        if (lane == 0) atomicAdd(a.nsite, sites);
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
    const unsigned long long *ext;  // extent bound of the evaluation (mol_extent_kernel), or nullptr
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

// A site pair of a molecule pair can take a different image than the
// site-0 pair only when the site-0 separation (mode-1 coordinates) is
// within twice the molecular extent of half a box along some axis, and only
// then is its own shift evaluated.  The extent is measured on the device
// every evaluation (mol_extent_kernel: the largest |x_s - x_s0| over sites,
// molecules and axes); this fixed bound (Bohr) serves kernels given none.
#define PINYB200_MOL_EXTENT 5.0

// Twice the extent bound of this evaluation, with a margin for the
// rounding of the separations the image tests compare.
__device__ __forceinline__ double ext2_of(const unsigned long long *ext)
{
    if (!ext) return 2.0 * PINYB200_MOL_EXTENT;
    const double e = fmax(__longlong_as_double((long long)__ldcg(ext)), 0.0);
    return 2.0 * (e * (1.0 + 1e-6) + 1e-9);
}

// The extent of every molecule: max |x_s - x_s0| over its sites s and the
// three axes of the mode-1 positions xm [natm][3], as an atomic maximum of
// the bit pattern (non-negative doubles order as integers).
__device__ __forceinline__ void mol_extent_body(const int *__restrict__ mstart, int nmol, const double *__restrict__ xm,
                                                unsigned long long *out, const VBlk vb)
{
    double e = 0.0;
    for (int m = vb.x * (int)blockDim.x + (int)threadIdx.x; m < nmol; m += vb.gx * (int)blockDim.x) {
        const int s0 = mstart[m], s1 = mstart[m + 1];
        for (int s = s0 + 1; s < s1; s++)
            for (int d = 0; d < 3; d++) e = fmax(e, fabs(xm[3 * (size_t)s + d] - xm[3 * (size_t)s0 + d]));
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) e = fmax(e, __shfl_xor_sync(0xffffffffu, e, o));
    if ((threadIdx.x & 31) == 0 && e > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(e));
}

__global__ void __launch_bounds__(256) mol_extent_kernel(const int *__restrict__ mstart, int nmol,
                                                         const double *__restrict__ xm, unsigned long long *out)
{
    mol_extent_body(mstart, nmol, xm, out, hw_blk());
}

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

    const double ext2 = ext2_of(a.ext);  // image test margin of this evaluation
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
                    near |= fabs(t + sh0[d]) > 0.5 - ext2 * hid;
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

// The force and energy rows of one interval (32 bytes, 32-byte aligned) in
// one 256-bit load: one L1 request per lane instead of two.
__device__ __forceinline__ void ldg_keep_pair(const float4 *p, float4 &f, float4 &e)
{
    asm("ld.global.nc.L1::evict_last.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(f.x), "=f"(f.y), "=f"(f.z), "=f"(f.w), "=f"(e.x), "=f"(e.y), "=f"(e.z), "=f"(e.w)
        : "l"(p));
}

struct MixArgs {
    const int *nchunk, *chunk, *bad, *mj;
    const unsigned *mask;
    const int *mstart;
    const double *posT, *xmod;
    const unsigned long long *ext;  // extent bound of the evaluation (mol_extent_kernel), or nullptr
    const int *atm_typ;
    const double *charge;
    const int *inter_map;
    const double *cutoff, *rmin, *dri;
    const int *has_vdw;
    const float4 *tab;   // [4][nuniq][nsplin] interval coefficients (TabKind order)
    const float4 *tabfe; // [2][nuniq][nsplin][2]: vdW then Coulomb; force and energy rows interleaved
    double *forceT;
    double *acc;
};

// The water model's site-pair constants of the MIXED kernel: the same for
// every box of one model, so a multi-box launch takes them once, outside
// its per-box table.
struct MixSite {
    int ntyp, nuniq, nsplin, stride;
    int toff[16];        // per site pair si * NS + sj: u * nsplin + 2, its rows at nint(t) = 0
    float q2[16];        // charge product of the site pair
    int eflag[16];       // tables the site pair uses: 1 vdW, 2 Coulomb
    int tstride;         // nuniq * nsplin, the distance between table kinds
    float rc2, dri_f, rmd, tmax;  // cutoff^2, 1/dr, rmin/dr, last interval
};

// Resident blocks per SM of the MIXED molecule-pair kernel: 5 x 128
// threads leave it 96 registers and no spills (at 6, 85 registers spilled
// ~180 bytes per thread into L1, the cache its table gathers depend on).
#ifndef PINYB200_MIX_BLOCKS
#define PINYB200_MIX_BLOCKS 5
#endif

// Site-pair table patterns known at compile time: bit si * NS + sj of CM
// (Coulomb table) and VM (vdW table).  kAnyPair takes them from
// MixArgs::eflag at run time.
constexpr unsigned kAnyPair = 0xffffffffu;
constexpr unsigned kTip4pCoul = 0xEEE0u, kTip4pVdw = 0x1u;  // O H H M: H, M charged; LJ on O-O
constexpr unsigned kSpcCoul = 0x1FFu, kSpcVdw = 0x1u;       // O H H: all charged; LJ on O-O

template <int P, int NS, bool ENERGY, unsigned CM, unsigned VM>
__device__ __forceinline__ void mol_pair_mixed_body(const MixArgs &a, const MixSite &m, const Cell &cell,
                                                    const VBlk vb)
{
    constexpr int G = P >= 32 ? 32 : P;  // lanes per molecule pair
    constexpr int JPI = 32 / G;          // molecule pairs per warp step
    __shared__ PairConst<float> pc;      // per-kind constants of the near path
    __shared__ double sacc[8][128];
    if (threadIdx.x < NS * NS) {
        const int si = threadIdx.x / NS, sj = threadIdx.x % NS;
        const int nm0 = a.mstart[1];
        const int ia = si < nm0 ? si : 0, ja = sj < nm0 ? sj : 0;
        const int p = pair_type(a.atm_typ[ia], a.atm_typ[ja], m.ntyp);
        const int u = a.inter_map[p];
        const double q2 = a.charge[ia] * a.charge[ja];
        float4 c;
        c.x = (float)(a.cutoff[p] * a.cutoff[p]);
        c.y = (float)a.rmin[u];
        c.z = (float)a.dri[u];
        c.w = (float)q2;
        pc.c[threadIdx.x] = c;
        pc.q2[threadIdx.x] = (float)q2;
        pc.o[threadIdx.x] = make_int2(u * m.nsplin, a.has_vdw[u]);
    }
    if (ENERGY)
        for (int c = 0; c < 8; c++) sacc[c][threadIdx.x] = 0.0;
    __syncthreads();
    if (a.bad && (a.bad[0] | a.bad[1])) {
        if (vb.x == 0 && vb.y == 0 && threadIdx.x == 0) a.acc[S_VVDW] = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    const float4 *__restrict__ tab = a.tab;
    const int lane = threadIdx.x & 31;
    const int warp = (vb.x * (int)blockDim.x + (int)threadIdx.x) >> 5;
    const int nwarps = (vb.gx * (int)blockDim.x) >> 5;
    const int sub = lane / G;
    const int b = (lane % G) + 32 * vb.y;  // bead
    const double *__restrict__ posT = a.posT;
    const float rc2 = m.rc2, dri = m.dri_f, rmd = m.rmd, tmax = m.tmax;
    constexpr float kRound = 12582912.0f;  // 1.5 * 2^23: x + kRound - kRound = nearest integer of x

    const double ext2 = ext2_of(a.ext);  // image test margin of this evaluation
    const int nch = *a.nchunk;
    for (int ch = warp; ch < nch; ch += nwarps) {
        const int mi = a.chunk[3 * ch], beg = a.chunk[3 * ch + 1], end = a.chunk[3 * ch + 2];
        const int i0 = mi * m.stride, ni = m.stride;
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
            const int j0 = mj * m.stride;
            // site-0 image from the mode-1 separation (FP64) and whether site
            // pairs may take other images
            double sh0[3];
            bool near = false;
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const double hid = cell.hi[4 * d];
                const double t = __dmul_rn(__dsub_rn(a.xmod[3 * (size_t)i0 + d], __ldcg(a.xmod + 3 * (size_t)j0 + d)), hid);
                sh0[d] = -nint_rn(t);
                near |= fabs(t + sh0[d]) > 0.5 - ext2 * hid;
            }
            if (near) {
                mol_pair_near<float, P, NS, true, ENERGY>(posT, a.xmod, a.forceT, &pc, a.tab,
                                                           (size_t)m.nuniq * m.nsplin, m.nsplin - 2, i0, j0, mask, b,
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
                    const bool coul = CM == kAnyPair ? (m.eflag[sp] & 2) != 0 : ((CM >> sp) & 1u) != 0;
                    const bool vdw = VM == kAnyPair ? (m.eflag[sp] & 1) != 0 : ((VM >> sp) & 1u) != 0;
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
                        const float4 *row = tab + (m.toff[sp] + kn);
                        const float4 *rfe = a.tabfe + 2 * (m.toff[sp] + kn);
                        float dv = 0.0f;
                        float4 ecf = make_float4(0.f, 0.f, 0.f, 0.f), evf = ecf;
                        if (coul) {
                            float4 cf;
                            if (ENERGY) {
                                ldg_keep_pair(rfe + 2 * m.tstride, cf, ecf);
                            } else {
                                cf = ldg_keep(row + T_CDV0C * m.tstride);
                            }
                            dv = m.q2[sp] * (cf.x + del * (cf.y + del * (cf.z + del * cf.w)));
                        }
                        if (vdw) {
                            float4 cf;
                            if (ENERGY) {
                                ldg_keep_pair(rfe, cf, evf);
                            } else {
                                cf = ldg_keep(row + T_CDV0 * m.tstride);
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
                            if (coul) ecs += m.q2[sp] * (ecf.x + del * (ecf.y + del * (ecf.z + del * ecf.w)));
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


template <int P, int NS, bool ENERGY, unsigned CM = kAnyPair, unsigned VM = kAnyPair>
__global__ void __launch_bounds__(128, PINYB200_MIX_BLOCKS)
    mol_pair_mixed_kernel(const __grid_constant__ MixArgs a, const __grid_constant__ MixSite m,
                          const __grid_constant__ Cell cell)
{
    mol_pair_mixed_body<P, NS, ENERGY, CM, VM>(a, m, cell, hw_blk());
}

// Many boxes of one bead count and site pattern in one persistent launch.
struct MixBox {
    MixArgs a;
    Cell cell;
};

// Resident blocks per SM of the batched MIXED kernel: the argument table
// is indexed at run time, which costs registers (4 x 128 threads leave 128,
// no spills; at 5 it spills 100-200 bytes).
#ifndef PINYB200_MIX_BATCH_BLOCKS
#define PINYB200_MIX_BATCH_BLOCKS 4
#endif
template <int P, int NS, bool ENERGY, unsigned CM = kAnyPair, unsigned VM = kAnyPair>
__global__ void __launch_bounds__(128, PINYB200_MIX_BATCH_BLOCKS)
    mol_pair_mixed_batch_kernel(const __grid_constant__ BoxTab<MixBox> t, const __grid_constant__ MixSite m)
{
    PINYB200_BOX_LOOP(t, i, vb, (mol_pair_mixed_body<P, NS, ENERGY, CM, VM>(t.arg[i].a, m, t.arg[i].cell, vb)));
}

// ---------------------------------------------------------------------------
// launchers

static CellPlanes cell_planes(const Cell &cell)
{
    CellPlanes pl;
    for (int d = 0; d < 3; d++) {
        const double b0 = cell.hi[d], b1 = cell.hi[3 + d], b2 = cell.hi[6 + d];
        pl.w[d] = 1.0 / std::sqrt(b0 * b0 + b1 * b1 + b2 * b2);
    }
    pl.ortho = cell.h[1] == 0.0 && cell.h[2] == 0.0 && cell.h[3] == 0.0 && cell.h[5] == 0.0 && cell.h[6] == 0.0 &&
               cell.h[7] == 0.0;
    return pl;
}

// pass 0: reach, fractional positions (and cells), counts with the pairs
// into the entry buffer when they fit, row offsets and the molecule-pair
// total (tot[2]); pass 1: the fill (a scatter of the entries, or computed
// again when they did not fit), adding the active site pairs into tot[3].
cudaError_t launch_mol_list(pinyb200_ctx *c, const Cell &cell, const double *d_pos1, const double *d_xm,
                            const double *d_cutskin2, int pass, const int *gate, cudaStream_t st)
{
    if (!st) st = c->stream;
    const DeviceSystem &s = c->sys;
    const int threads = 256;
    int blocks = (((c->nmol + 1) / 2) * 32 + threads - 1) / threads;  // a warp per pair of rows
    const int maxb = c->sm_count * 8;
    if (blocks > maxb) blocks = maxb;
    if (blocks < 1) blocks = 1;
    const bool use_xm = d_xm != nullptr;
    MolListArgs a{};
    a.mstart = c->d_mstart;
    a.stride = c->mol_stride;
    a.ntyp = s.ntyp;
    a.pos1 = d_pos1;
    a.xm = d_xm;
    a.msf = c->d_msf;
    a.cutskin2 = d_cutskin2;
    a.atm_typ = s.atm_typ;
    a.charge = s.charge;
    a.inter_map = s.inter_map;
    a.has_vdw = s.has_vdw;
    a.reach = c->d_reach;
    a.count = c->d_mcount;
    a.ent = c->d_ent;
    a.ent_cap = c->d_ent ? c->ent_cap : 0;
    a.nent = c->d_nent;
    if (pass == 1) {
        a.row = c->d_mrow;
        a.mj = c->d_mj;
        a.mask = c->d_mmask;
        a.maskf = c->d_mmaskf;
        a.cap = c->mlist_cap;
        a.nsite = (unsigned long long *)(c->d_tot + 3);
    }
    const int ncell = c->cell_n[0] * c->cell_n[1] * c->cell_n[2];
    const bool cells = ncell > 0;
    const int *cellok = cells ? c->d_cellok : nullptr;
    const CellPlanes pl = cell_planes(cell);
    cudaError_t e;
    if (pass == 0) {
        const int mb = (c->nmol + 255) / 256;
        if ((e = cudaMemsetAsync(c->d_nent, 0, sizeof(unsigned long long), st)) != cudaSuccess) return e;
        if (cells && (e = cudaMemsetAsync(c->d_ccnt, 0, 2 * (size_t)c->cell_cap * sizeof(int), st)) != cudaSuccess)
            return e;
        mol_reach_kernel<<<reach_blocks(c), 256, 0, st>>>(gate, c->nmol, c->d_mstart, d_pos1, d_cutskin2,
                                                          s.npair_typ, c->d_reach_acc, c->d_reach);
        mol_frac_kernel<<<mb, 256, 0, st>>>(gate, c->nmol, c->d_mstart, d_pos1, cell, c->cell_n[0], c->cell_n[1],
                                            c->cell_n[2], c->d_msf, cells ? c->d_mcell : nullptr, c->d_ccnt);
        if (cells) {
            // cell membership (sorted), the cells' offsets, and whether they serve this build
            double edge2 = 1e300;
            for (int d = 0; d < 3; d++) edge2 = std::min(edge2, 2.0 * pl.w[d] / c->cell_n[d]);
            if ((e = launch_scan(c, gate, ncell, 1, c->d_ccnt, c->d_coff, nullptr, c->d_ctot, st)) != cudaSuccess)
                return e;
            cell_scatter_kernel<<<mb, 256, 0, st>>>(gate, c->nmol, c->d_mcell, c->d_coff, c->d_ccnt + c->cell_cap,
                                                    c->d_cmol);
            cell_sort_kernel<<<(ncell + 7) / 8, 256, 0, st>>>(gate, ncell, c->d_coff, c->d_cmol,
                                                              c->d_cmol + c->nmol);
            cell_decide_kernel<<<1, 1024, 0, st>>>(gate, ncell, c->d_coff, c->d_reach, edge2, c->d_cellok);
        }
    }
    const int cell_smem = PINYB200_CELL_BATCH * (int)sizeof(float4);
#define MOL_LIST(NSV, FILLV, XMV)                                                                                 \
    {                                                                                                             \
        if (cells) {                                                                                              \
            if ((e = smem_optin((const void *)mol_list_cell_kernel<FILLV, NSV, XMV>, cell_smem)) != cudaSuccess)  \
                return e;                                                                                         \
            mol_list_cell_kernel<FILLV, NSV, XMV><<<ncell, 256, cell_smem, st>>>(                                 \
                gate, cellok, c->cell_n[0], c->cell_n[1], c->cell_n[2], c->d_coff, c->d_cmol + c->nmol, pl, cell,  \
                a);                                                                                               \
        }                                                                                                         \
        mol_list_kernel<FILLV, NSV, XMV><<<blocks, threads, 0, st>>>(gate, c->nmol, cell, pl, a, cellok);       \
    }
#define MOL_LIST_XM(NSV, FILLV)                                                                                   \
    {                                                                                                             \
        if (use_xm) MOL_LIST(NSV, FILLV, true) else MOL_LIST(NSV, FILLV, false)                                   \
    }
    if (c->mol_ns == 3) {
        if (pass == 0) MOL_LIST_XM(3, 0) else MOL_LIST_XM(3, 1)
    } else if (c->mol_ns == 4) {
        if (pass == 0) MOL_LIST_XM(4, 0) else MOL_LIST_XM(4, 1)
    } else {
        return cudaErrorInvalidValue;
    }
#undef MOL_LIST_XM
#undef MOL_LIST
    if (pass == 1) mol_scatter_kernel<<<c->sm_count * 4, 256, 0, st>>>(gate, a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (pass == 0) return launch_scan(c, gate, c->nmol, 1, c->d_mcount, c->d_mrow, nullptr, c->d_tot + 2, st);
    return cudaSuccess;
}

// Plan the link cells for the positions of a host build (reach R measured
// on the device): n_d = floor(plane spacing / (1.15 R / 2)), at most 64,
// used when every n_d >= 5 and the 125 cells around a molecule are at most
// 40 % of the box (below that the sweep's simpler enumeration is as fast);
// otherwise every build sweeps.  Buffers grow as needed and are kept, so
// device rebuilds with the same plan allocate nothing.
int mol_cells_plan(pinyb200_ctx *c, const Cell &cell, const double *d_pos1, const double *d_cutskin2)
{
    cudaError_t e;
    mol_reach_kernel<<<reach_blocks(c), 256, 0, c->stream>>>(nullptr, c->nmol, c->d_mstart, d_pos1, d_cutskin2,
                                                             c->sys.npair_typ, c->d_reach_acc, c->d_reach);
    double R = 0.0;
    if ((e = cudaMemcpyAsync(&R, c->d_reach, sizeof(double), cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(c->stream)) != cudaSuccess)
        return record_error(c, PINYB200_ERR_CUDA, std::string("list cells: ") + cudaGetErrorString(e));
    int n[3];
    bool on = c->list_method == PINYB200_LIST_LNK && std::isfinite(R) && R > 0.0;
    for (int d = 0; d < 3 && on; d++) {
        const double b0 = cell.hi[d], b1 = cell.hi[3 + d], b2 = cell.hi[6 + d];
        const double w = 1.0 / std::sqrt(b0 * b0 + b1 * b1 + b2 * b2);
        const double k = std::floor(w / (1.15 * R / 2.0));
        n[d] = k > 64.0 ? 64 : (int)k;
        on = n[d] >= 5;
    }
    const long long ncell = on ? (long long)n[0] * n[1] * n[2] : 0;
    if (!on || ncell * 2 < 625) {  // 125 / ncell > 0.4
        c->cell_n[0] = c->cell_n[1] = c->cell_n[2] = 0;
        return PINYB200_OK;
    }
    auto alloc = [&](void **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
    };
    e = cudaSuccess;
    if (!c->d_mcell) {
        alloc((void **)&c->d_mcell, (size_t)c->nmol * sizeof(int));
        alloc((void **)&c->d_cmol, 2 * (size_t)c->nmol * sizeof(int));
        alloc((void **)&c->d_cellok, sizeof(int));
        alloc((void **)&c->d_ctot, sizeof(long long));
    }
    if (ncell > c->cell_cap) {
        if (c->d_ccnt) cudaFree(c->d_ccnt);
        if (c->d_coff) cudaFree(c->d_coff);
        c->d_ccnt = c->d_coff = nullptr;
        c->cell_cap = 0;
        alloc((void **)&c->d_ccnt, 2 * (size_t)ncell * sizeof(int));
        alloc((void **)&c->d_coff, ((size_t)ncell + 1) * sizeof(int));
        if (e == cudaSuccess) c->cell_cap = (int)ncell;
    }
    if (e != cudaSuccess) {
        c->cell_n[0] = c->cell_n[1] = c->cell_n[2] = 0;
        return record_error(c, PINYB200_ERR_CUDA, std::string("list cells: ") + cudaGetErrorString(e));
    }
    for (int d = 0; d < 3; d++) c->cell_n[d] = n[d];
    return PINYB200_OK;
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
    } else {                                                                                                       \
        site_fill_kernel<NSV><<<blocks, threads, 0, st>>>(gate, c->nmol, c->d_mstart, c->d_mrow, c->d_mj,          \
                                                          c->d_mmaskf, c->d_mmask, c->mlist_cap, c->d_row,        \
                                                          c->d_rowA, c->d_col, c->d_colA, c->list_cap);           \
    }
    if (c->mol_ns == 3) { SITE_LIST(3) }
    else if (c->mol_ns == 4) { SITE_LIST(4) }
    else return cudaErrorInvalidValue;
#undef SITE_LIST
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (pass == 0) return launch_scan(c, gate, natm, 2, c->d_count, c->d_row, c->d_rowA, c->d_tot, st);
    return cudaSuccess;
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
    a.ext = (const unsigned long long *)(c->d_acc + S_EXT);
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
static void launch_mix_pattern(pinyb200_ctx *c, const MixArgs &a, const MixSite &m, const Cell &cell, bool energy,
                               dim3 grid)
{
    const int threads = 128;
    if (energy) {
        carveout_pref((const void *)mol_pair_mixed_kernel<P, NS, true, CM, VM>, c->pair_carveout);
        mol_pair_mixed_kernel<P, NS, true, CM, VM><<<grid, threads, 0, c->stream>>>(a, m, cell);
    } else {
        carveout_pref((const void *)mol_pair_mixed_kernel<P, NS, false, CM, VM>, c->pair_carveout);
        mol_pair_mixed_kernel<P, NS, false, CM, VM><<<grid, threads, 0, c->stream>>>(a, m, cell);
    }
}

template <int P, int NS>
static void launch_mix_t(pinyb200_ctx *c, const MixArgs &a, const MixSite &m, const Cell &cell, bool energy)
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
        launch_mix_pattern<P, NS, kTip4pCoul, kTip4pVdw>(c, a, m, cell, energy, grid);
    else if (NS == 3 && cm == kSpcCoul && vm == kSpcVdw)
        launch_mix_pattern<P, NS, kSpcCoul, kSpcVdw>(c, a, m, cell, energy, grid);
    else
        launch_mix_pattern<P, NS, kAnyPair, kAnyPair>(c, a, m, cell, energy, grid);
}

template <int NS>
static cudaError_t launch_mix_ns(pinyb200_ctx *c, const MixArgs &a, const MixSite &m, const Cell &cell, bool energy)
{
    switch (c->P) {
    case 1: launch_mix_t<1, NS>(c, a, m, cell, energy); break;
    case 2: launch_mix_t<2, NS>(c, a, m, cell, energy); break;
    case 4: launch_mix_t<4, NS>(c, a, m, cell, energy); break;
    case 8: launch_mix_t<8, NS>(c, a, m, cell, energy); break;
    case 16: launch_mix_t<16, NS>(c, a, m, cell, energy); break;
    case 32: launch_mix_t<32, NS>(c, a, m, cell, energy); break;
    case 64: launch_mix_t<64, NS>(c, a, m, cell, energy); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// Arguments of the MIXED molecule-pair kernel for one context.
static MixArgs mix_args(pinyb200_ctx *c)
{
    const DeviceSystem &s = c->sys;
    MixArgs a;
    a.nchunk = c->d_nchunk;
    a.chunk = c->d_chunk;
    a.bad = c->d_ls ? (const int *)((const char *)c->d_ls + offsetof(ListState, overflow)) : nullptr;
    a.mj = c->d_mj;
    a.mask = c->d_mmask;
    a.mstart = c->d_mstart;
    a.posT = c->d_posT;
    a.xmod = c->P > 1 ? c->d_xmod : c->d_posT;
    a.ext = (const unsigned long long *)(c->d_acc + S_EXT);
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
    return a;
}

// Site-pair constants of the MIXED molecule-pair kernel for one context.
static MixSite mix_site(const pinyb200_ctx *c)
{
    const DeviceSystem &s = c->sys;
    MixSite m;
    memset(&m, 0, sizeof(m));
    m.ntyp = s.ntyp;
    m.nuniq = s.nuniq;
    m.nsplin = s.nsplin;
    m.stride = c->mol_stride;
    for (int k = 0; k < 16; k++) {
        m.toff[k] = c->mix_toff[k];
        m.q2[k] = c->mix_q2[k];
        m.eflag[k] = c->mix_eflag[k];
    }
    m.tstride = s.nuniq * s.nsplin;
    m.rc2 = c->mix_rc2;
    m.dri_f = c->mix_dri;
    m.rmd = c->mix_rmd;
    m.tmax = c->mix_tmax;
    return m;
}

// The MIXED kernel with combined per-site-pair tables (pinyb200_ctx::mix_ok).
cudaError_t launch_mol_pair_mixed(pinyb200_ctx *c, const Cell &cell, bool energy)
{
    const MixArgs a = mix_args(c);
    const MixSite m = mix_site(c);
    if (c->mol_ns == 3) return launch_mix_ns<3>(c, a, m, cell, energy);
    return launch_mix_ns<4>(c, a, m, cell, energy);
}

// The molecule extent bound of this evaluation into the context's per-bead
// sums (slot S_EXT of bead 0, cleared with them), from the mode-1 positions.
cudaError_t launch_mol_extent(pinyb200_ctx *c)
{
    if (!c->use_mol || c->nmol == 0) return cudaSuccess;
    const double *xm = c->P > 1 ? c->d_xmod : c->d_posT;
    const int blocks = std::max(1, std::min((c->nmol + 255) / 256, c->sm_count * 4));
    mol_extent_kernel<<<blocks, 256, 0, c->stream>>>(c->d_mstart, c->nmol, xm,
                                                      (unsigned long long *)(c->d_acc + S_EXT));
    return cudaGetLastError();
}

struct ExtBox {
    const int *mstart;
    int nmol;
    const double *xm;
    unsigned long long *out;
};

__global__ void __launch_bounds__(256) mol_extent_batch_kernel(const __grid_constant__ BoxTab<ExtBox> t)
{
    PINYB200_BOX_LOOP(t, i, vb, (mol_extent_body(t.arg[i].mstart, t.arg[i].nmol, t.arg[i].xm, t.arg[i].out, vb)));
}

cudaError_t launch_mol_extent_batch(const std::vector<pinyb200_ctx *> &box, int sm_count, cudaStream_t st)
{
    BoxTabBuilder<ExtBox> tb;
    for (pinyb200_ctx *c : box) {
        if (!c->use_mol || c->nmol == 0) continue;
        tb.add(ExtBox{c->d_mstart, c->nmol, c->P > 1 ? c->d_xmod : c->d_posT, (unsigned long long *)(c->d_acc + S_EXT)},
               (c->nmol + 255) / 256, 1, (double)c->nmol);
    }
    return launch_tables(tb, (const void *)mol_extent_batch_kernel, 256, 0, sm_count,
                         [&](const BoxTab<ExtBox> &t, int g) { mol_extent_batch_kernel<<<g, 256, 0, st>>>(t); });
}

// Site-pair table pattern of a context: 1 q-TIP4P/F-like (4 sites), 2
// q-SPC/Fw-like (3 sites), 0 another pattern.
int mix_pattern(const pinyb200_ctx *c)
{
    unsigned cm = 0, vm = 0;
    const int NS = c->mol_ns;
    for (int k = 0; k < NS * NS; k++) {
        if (c->mix_eflag[k] & 2) cm |= 1u << k;
        if (c->mix_eflag[k] & 1) vm |= 1u << k;
    }
    if (NS == 4 && cm == kTip4pCoul && vm == kTip4pVdw) return 1;
    if (NS == 3 && cm == kSpcCoul && vm == kSpcVdw) return 2;
    return 0;
}

template <int P, int NS, unsigned CM, unsigned VM>
static cudaError_t launch_mix_batch_t(const std::vector<pinyb200_ctx *> &box, const std::vector<Cell> &cells,
                                      bool energy, int sm_count, cudaStream_t st)
{
    BoxTabBuilder<MixBox> tb;
    const MixSite m = mix_site(box[0]);  // one model per group (launch_mol_pair_mixed_batch)
    // Blocks of each box's own grid-stride loop over its chunks: about 16
    // chunks' worth of 32-bead work per warp (a warp takes 32 / P molecule
    // pairs at a time below 32 beads), so that a block's set-up (site-pair
    // constants) and energy flush (FP64 atomics per bead and slot) are
    // spread over enough molecule pairs; more, down to 2 chunks per warp,
    // while the group has fewer than two blocks per resident CTA.
    const int G = P >= 32 ? 32 : P;
    std::vector<long long> vb(box.size());
    long long tot = 0;
    for (size_t i = 0; i < box.size(); i++) {
        vb[i] = std::max<long long>(1, (box[i]->chunk_cap * G + 4LL * 16 * 32 - 1) / (4LL * 16 * 32));
        tot += vb[i] * (P > 32 ? P / 32 : 1);
    }
    const long long want = 2LL * sm_count * PINYB200_MIX_BATCH_BLOCKS;
    const long long scale = tot < want ? (want + tot - 1) / tot : 1;
    for (size_t i = 0; i < box.size(); i++) {
        pinyb200_ctx *c = box[i];
        const long long v = std::min(vb[i] * scale, std::max<long long>(1, (c->chunk_cap + 7) / 8));
        tb.add(MixBox{mix_args(c), cells[i]}, (int)std::min<long long>(v, 1 << 20), P > 32 ? P / 32 : 1,
               (double)c->chunk_cap * P);
    }
    const void *fn = energy ? (const void *)mol_pair_mixed_batch_kernel<P, NS, true, CM, VM>
                            : (const void *)mol_pair_mixed_batch_kernel<P, NS, false, CM, VM>;
    cudaError_t err = carveout_pref(fn, box.empty() ? 25 : box[0]->pair_carveout);
    if (err != cudaSuccess) return err;
    return launch_tables(tb, fn, 128, 0, sm_count, [&](const BoxTab<MixBox> &t, int g) {
        if (energy) mol_pair_mixed_batch_kernel<P, NS, true, CM, VM><<<g, 128, 0, st>>>(t, m);
        else mol_pair_mixed_batch_kernel<P, NS, false, CM, VM><<<g, 128, 0, st>>>(t, m);
    });
}

template <int NS, unsigned CM, unsigned VM>
static cudaError_t launch_mix_batch_p(int P, const std::vector<pinyb200_ctx *> &box, const std::vector<Cell> &cells,
                                      bool energy, int sm_count, cudaStream_t st)
{
    switch (P) {
    case 1: return launch_mix_batch_t<1, NS, CM, VM>(box, cells, energy, sm_count, st);
    case 2: return launch_mix_batch_t<2, NS, CM, VM>(box, cells, energy, sm_count, st);
    case 4: return launch_mix_batch_t<4, NS, CM, VM>(box, cells, energy, sm_count, st);
    case 8: return launch_mix_batch_t<8, NS, CM, VM>(box, cells, energy, sm_count, st);
    case 16: return launch_mix_batch_t<16, NS, CM, VM>(box, cells, energy, sm_count, st);
    case 32: return launch_mix_batch_t<32, NS, CM, VM>(box, cells, energy, sm_count, st);
    case 64: return launch_mix_batch_t<64, NS, CM, VM>(box, cells, energy, sm_count, st);
    default: return cudaErrorInvalidValue;
    }
}

// MIXED molecule-pair forces of many boxes: one persistent launch per
// (bead count, site pattern) group.  Every box must have mix_pattern() != 0.
cudaError_t launch_mol_pair_mixed_batch(const std::vector<pinyb200_ctx *> &box, const std::vector<Cell> &cells,
                                        bool energy, int sm_count, cudaStream_t st)
{
    // groups of one bead count, site pattern and set of site-pair constants
    std::map<std::tuple<int, int, std::string>, std::pair<std::vector<pinyb200_ctx *>, std::vector<Cell>>> groups;
    for (size_t i = 0; i < box.size(); i++) {
        const MixSite ms = mix_site(box[i]);
        auto &g = groups[std::make_tuple(box[i]->P, mix_pattern(box[i]), std::string((const char *)&ms, sizeof(ms)))];
        g.first.push_back(box[i]);
        g.second.push_back(cells[i]);
    }
    for (auto &kv : groups) {
        const int P = std::get<0>(kv.first), pat = std::get<1>(kv.first);
        cudaError_t err;
        if (pat == 1)
            err = launch_mix_batch_p<4, kTip4pCoul, kTip4pVdw>(P, kv.second.first, kv.second.second, energy, sm_count,
                                                                st);
        else if (pat == 2)
            err = launch_mix_batch_p<3, kSpcCoul, kSpcVdw>(P, kv.second.first, kv.second.second, energy, sm_count, st);
        else
            err = cudaErrorInvalidValue;
        if (err != cudaSuccess) return err;
    }
    return cudaSuccess;
}

}  // namespace pinyb200
