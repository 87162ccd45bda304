// Smooth PME for all beads: charge spreading, batched 3D FFT, k-sphere
// convolution with energy and virial, force gather.
//
// Restates ewald3d_recip_pme_none (src/energy/inter/recip3d/ewald3d_pme.c:
// 95-600): scaled coordinates wrapped to (0,1] (:231-256), order-n cardinal
// B-splines by PINY's recursion and their derivatives from the order n-1
// splines (:301-338, :512-532), grid points ia - (j-2) wrapped (:274-300),
// the half-space spherical k list with preg = exp(-g^2/4a^2)/(g^2 V/4pi) and
// the B-spline weights (:366-425), and the gather F = -q sum grad(M) phi
// (:534-559).  PINY spreads into a complex grid with zero imaginary part and
// runs unnormalised complex FFTs (para_fft_gen3d_bck_to_g / _fwd_to_r).
// The device spreads into a real grid and keeps half of the spectrum
// (a <= Na/2): the charge grid is real, so the other half is its complex
// conjugate.  Filtering with the symmetric influence function equals PINY's
// half-list convolution plus Hermitian fill (pme_sngl_pack_coef,
// fft_package.c:458-503); half of the full-grid sum is PINY's energy.
//
// Kernels per evaluation (all beads in each launch):
//   bin         (charge, bead) -> grid tile of its stencil origin
//   spread      per (tile, bead): shared-memory copy of the tile, added to
//               the real grid once (FP32: 16-byte vector atomics)
//   plane_fwd   per (bead, c) plane: FFT along a then b in shared memory,
//               half spectrum out
//   conv_c      per (bead, b): FFT along c, filter + energy + virial,
//               inverse FFT along c
//   plane_inv   per (bead, c): inverse FFT along b, Hermitian completion,
//               inverse FFT along a, real potential out
//   gather      per (tile, bead): forces from a shared copy of the tile's
//               potential
#include <map>
#include <tuple>
#include <vector>

#include "boxtab.cuh"
#include "common.cuh"

namespace pinyb200 {

struct PmeArgs {
    int natm, P, nchrg;
    const int *ichrg;
    const double *charge;
    const double *posT;
    int Na, Nb, Nc, n;
    void *grid;  // real [P][Nc][Nb][Na]
    double *forceP;  // PME forces [nchrg][3][P]
    int4 *rhead;  // per (charge, bead) records, see RecGeom
    void *rw;
};

// B-spline weights of order NI at the fractional offset f (ewald3d_pme.c:
// 301-338).  m[j], j = 1..NI as in PINY (index 0 unused); dm[] are the
// derivative weights formed at order NI-1 (:512-532).
template <typename R, int NI, bool DERIV>
__device__ __forceinline__ void bspline(R f, R *m, R *dm)
{
    R u[NI + 1];
#pragma unroll
    for (int j = 1; j <= NI; j++) u[j] = f + (R)(j - 1);
    m[1] = (R)1 - fabs(u[1] - (R)1);
    m[2] = (R)1 - fabs(u[2] - (R)1);
#pragma unroll
    for (int j = 3; j <= NI; j++) m[j] = (R)0;
#pragma unroll
    for (int nn = 3; nn <= NI; nn++) {
        const R rn = (R)nn, rn1 = (R)1 / (R)(nn - 1);
#pragma unroll
        for (int j = nn; j >= 2; j--) m[j] = (u[j] * m[j] + (rn - u[j]) * m[j - 1]) * rn1;
        m[1] = u[1] * m[1] * rn1;
        if (DERIV && nn == NI - 1) {
            dm[1] = m[1];
#pragma unroll
            for (int j = 2; j <= NI; j++) dm[j] = m[j] - m[j - 1];
        }
    }
}

// Scaled coordinate of one charge along one axis, wrapped to (0,1] and
// multiplied by the grid size; returns floor and fraction (FP64, PINY order).
__device__ __forceinline__ void scaled(double s, int N, int &i0, double &frac)
{
    s = __dsub_rn(s, nint_rn(__dsub_rn(s, 0.5)));
    double xs = __dmul_rn(s, (double)N);
    i0 = (int)xs;
    frac = __dsub_rn(xs, (double)i0);
    // s == 1 exactly (a coordinate on a cell face) and non-finite positions
    // would index outside the grid; keep every access in bounds.
    if (i0 == N) i0 = 0;
    if (!(i0 >= 0 && i0 < N)) { i0 = 0; frac = 0.0; }
}

// First grid index per axis of one charge's stencil and the fractional
// offsets.  PINY's points ia-(j-2), j = 1..n, are the n consecutive indices
// ia-n+1 .. ia (wrapped), and point j carries weight m[j]; so grid index
// lo + t (t = 0..n-1) carries m[n - t].  The binning and both tile kernels
// call this same FP64 code, so they agree on every charge's tile.
__device__ __forceinline__ void stencil_origin(const PmeArgs &a, const Cell &cell, int at, int b, int ni, int &la,
                                               int &lb, int &lc, double &fa, double &fb, double &fc)
{
    const double x = a.posT[(3 * (size_t)at + 0) * a.P + b];
    const double y = a.posT[(3 * (size_t)at + 1) * a.P + b];
    const double z = a.posT[(3 * (size_t)at + 2) * a.P + b];
    const double sa = __dadd_rn(__dadd_rn(__dmul_rn(x, cell.hi[0]), __dmul_rn(y, cell.hi[3])), __dmul_rn(z, cell.hi[6]));
    const double sb = __dadd_rn(__dadd_rn(__dmul_rn(x, cell.hi[1]), __dmul_rn(y, cell.hi[4])), __dmul_rn(z, cell.hi[7]));
    const double sc = __dadd_rn(__dadd_rn(__dmul_rn(x, cell.hi[2]), __dmul_rn(y, cell.hi[5])), __dmul_rn(z, cell.hi[8]));
    int ia, ib, ic;
    scaled(sa, a.Na, ia, fa);
    scaled(sb, a.Nb, ib, fb);
    scaled(sc, a.Nc, ic, fc);
    la = ia - ni + 1;
    if (la < 0) la += a.Na;
    lb = ib - ni + 1;
    if (lb < 0) lb += a.Nb;
    lc = ic - ni + 1;
    if (lc < 0) lc += a.Nc;
}

// Charges binned by the grid tile that holds their stencil origin, per bead.
// Largest value of the order-n cardinal B-spline (PINY's m[] over the
// fractional offset, ewald3d_pme.c:301-338), sampled finely: a bound for the
// fixed-point spread.
static double bspline_peak(int n)
{
    double best = 0.0;
    for (int k = 0; k <= 1024; k++) {
        const double f = k / 1024.0;
        double m[16] = {0}, u[16];
        for (int j = 1; j <= n; j++) u[j] = f + (double)(j - 1);
        m[1] = 1.0 - std::fabs(u[1] - 1.0);
        m[2] = 1.0 - std::fabs(u[2] - 1.0);
        for (int nn = 3; nn <= n; nn++) {
            const double rn1 = 1.0 / (double)(nn - 1);
            for (int j = nn; j >= 2; j--) m[j] = (u[j] * m[j] + ((double)nn - u[j]) * m[j - 1]) * rn1;
            m[1] = u[1] * m[1] * rn1;
        }
        for (int j = 1; j <= n; j++) best = std::max(best, m[j]);
    }
    return best * (1.0 + 1e-6);
}

struct TileArgs {
    int T;  // tile edge (grid points)
    float qfix, qfix_inv;  // FP32 spread: fixed-point scale 2^S of the shared tile, and 2^-S
    int nta, ntb, ntc, ntile, cap;
    int *cnt;  // [P][ntile], then the overflow count
    int *bin;  // [P][ntile][cap] record numbers k*P + b
    int *ovf;  // [nchrg * P] record numbers that did not fit their bin
};

// Per (charge k, bead b) record, number idx = k*P + b, written by the bin
// kernel and read by spread and gather:
//   head[idx] = (atom, la, lb, lc)  stencil origin per axis
//   w[idx][j][t], j = 0..5 for M_a, M_b, M_c, dM_a, dM_b, dM_c, t = 0..NIP-1:
//                 weight of grid point lo + t (PINY's m[NI - t]), zero for t >= NI
template <int NI>
struct RecGeom {
    static constexpr int NIP = NI <= 4 ? 4 : (NI <= 8 ? 8 : 12);
    static constexpr int NW = 6 * NIP;
};

// Tile geometry: T^3 grid points own the charges whose stencil starts in
// them; the shared copy spans E = T + NI - 1 points per edge (the stencils
// reach NI - 1 beyond), rows padded to PA.
// With PA = 24 (E <= 24) the 4 b rows x 8 a points of a warp fall in 32
// distinct banks (row offsets 0, 24, 48, 72 = 0, 24, 16, 8 mod 32).
template <int NI, int TT>
struct TileGeom {
    static constexpr int T = TT;
    static constexpr int E = T + NI - 1;
    static constexpr int PA = E <= 24 ? 24 : ((E + 3) & ~3);
    static constexpr int NPT = E * E * PA;
};

// i mod N for 0 <= i < k N with small k.
__device__ __forceinline__ int wrapi(int i, int N)
{
    while (i >= N) i -= N;
    return i;
}

// Store n consecutive values of type R (n a multiple of 4) with vector stores.
__device__ __forceinline__ void store4(float *dst, const float *v, int n)
{
    for (int i = 0; i < n; i += 4) *(float4 *)(dst + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
}
__device__ __forceinline__ void store4(double *dst, const double *v, int n)
{
    for (int i = 0; i < n; i += 2) *(double2 *)(dst + i) = make_double2(v[i], v[i + 1]);
}
template <int N>
__device__ __forceinline__ void load4(float *v, const float *src)
{
#pragma unroll
    for (int i = 0; i < N; i += 4) {
        const float4 x = __ldg((const float4 *)(src + i));
        v[i] = x.x;
        v[i + 1] = x.y;
        v[i + 2] = x.z;
        v[i + 3] = x.w;
    }
}
template <int N>
__device__ __forceinline__ void load4(double *v, const double *src)
{
#pragma unroll
    for (int i = 0; i < N; i += 2) {
        const double2 x = __ldg((const double2 *)(src + i));
        v[i] = x.x;
        v[i + 1] = x.y;
    }
}

// Bin kernel: one thread per (charge, bead).  Stencil origin in FP64 with
// PINY's operation order, B-spline weights and derivatives in R, record
// written in (charge, bead) order, record number filed under its tile.
template <typename R, int NI>
__global__ void __launch_bounds__(256) pme_bin_kernel(PmeArgs a, Cell cell, TileArgs t)
{
    typedef RecGeom<NI> RG;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)a.nchrg * a.P) return;
    const int b = (int)(idx % a.P);
    const int k = (int)(idx / a.P);
    const int at = a.ichrg[k];
    int la, lb, lc;
    double fa, fb, fc;
    stencil_origin(a, cell, at, b, NI, la, lb, lc, fa, fb, fc);
    R m[NI + 1], d[NI + 1], w[RG::NIP];
    R *out = (R *)a.rw + (size_t)idx * RG::NW;
    const double fr[3] = {fa, fb, fc};
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
        bspline<R, NI, true>((R)fr[ax], m, d);
#pragma unroll
        for (int s = 0; s < RG::NIP; s++) w[s] = s < NI ? m[NI - s] : (R)0;
        store4(out + ax * RG::NIP, w, RG::NIP);
#pragma unroll
        for (int s = 0; s < RG::NIP; s++) w[s] = s < NI ? d[NI - s] : (R)0;
        store4(out + (3 + ax) * RG::NIP, w, RG::NIP);
    }
    a.rhead[idx] = make_int4(at, la, lb, lc);
    const int T = t.T;
    const int tile = ((lc / T) * t.ntb + lb / T) * t.nta + la / T;
    const int slot = atomicAdd(&t.cnt[b * t.ntile + tile], 1);
    if (slot < t.cap) t.bin[((size_t)b * t.ntile + tile) * t.cap + slot] = (int)idx;
    else t.ovf[atomicAdd(&t.cnt[a.P * t.ntile], 1)] = (int)idx;
}

// Weights of one record that a lane of an 8-lane group needs: its own a
// points (l8 and l8 + 8) and all b and c points; DERIV adds the derivatives.
template <typename R, int NI, bool DERIV>
struct LaneW {
    typedef RecGeom<NI> RG;
    R wa0, wa1, da0, da1;
    R mb[RG::NIP], mc[RG::NIP], db[DERIV ? RG::NIP : 1], dc[DERIV ? RG::NIP : 1];
    __device__ __forceinline__ void load(const R *rw, int idx, int l8)
    {
        const R *w = rw + (size_t)idx * RG::NW;
        wa0 = l8 < NI ? w[l8] : (R)0;
        wa1 = (NI > 8 && l8 + 8 < NI) ? w[l8 + 8] : (R)0;
        load4<RG::NIP>(mb, w + RG::NIP);
        load4<RG::NIP>(mc, w + 2 * RG::NIP);
        if (DERIV) {
            da0 = l8 < NI ? w[3 * RG::NIP + l8] : (R)0;
            da1 = (NI > 8 && l8 + 8 < NI) ? w[3 * RG::NIP + l8 + 8] : (R)0;
            load4<RG::NIP>(db, w + 4 * RG::NIP);
            load4<RG::NIP>(dc, w + 5 * RG::NIP);
        }
    }
};

// Spread one record straight into the global grid (overflow entries).
template <typename R, int NI>
__device__ __forceinline__ void spread_global(const PmeArgs &a, R *g, int la, int lb, int lc,
                                              const LaneW<R, NI, false> &lw, R q, int l8)
{
    const int ga0 = wrapi(la + l8, a.Na), ga1 = wrapi(la + l8 + 8, a.Na);
#pragma unroll
    for (int tc = 0; tc < NI; tc++) {
        const int gc = wrapi(lc + tc, a.Nc);
        const R qc = q * lw.mc[tc];
#pragma unroll
        for (int tb = 0; tb < NI; tb++) {
            const int gb = wrapi(lb + tb, a.Nb);
            const R w = lw.mb[tb] * qc;
            R *row = g + ((size_t)gc * a.Nb + gb) * a.Na;
            if (l8 < NI) atomicAdd(row + ga0, lw.wa0 * w);
            if (NI > 8 && l8 + 8 < NI) atomicAdd(row + ga1, lw.wa1 * w);
        }
    }
}

// Spread: one block per (tile, bead), one warp per record.  A warp adds its
// record's stencil to a shared copy of the tile with shared-memory atomics;
// its 32 lanes cover 8 a points x 4 b rows, so the 32 addresses of one
// atomic are distinct and, with rows padded to PA = 0 mod 8 floats,
// fall in distinct banks.  The copy is then added to the grid once, with
// 16-byte vector atomics where the rows allow.  Records whose origin lies
// outside the tile (none are expected) and overflow records go straight to
// the grid.
template <typename R, int NI, int TT>
size_t spread_smem()
{
    return (size_t)TileGeom<NI, TT>::NPT * sizeof(R);
}

template <typename R, int NI, int TT>
__global__ void __launch_bounds__(256) spread_tile_kernel(PmeArgs a, TileArgs t)
{
    typedef TileGeom<NI, TT> TG;
    typedef RecGeom<NI> RG;
    constexpr int NIP = RG::NIP;
    constexpr int NTB = (NI + 3) / 4;  // b rows per lane
    extern __shared__ unsigned char smem_raw[];
    R *tl = (R *)smem_raw;
    for (int i = threadIdx.x; i < TG::NPT; i += blockDim.x) tl[i] = (R)0;
    __syncthreads();
    const int tile = blockIdx.x, b = blockIdx.y;
    const int ta0 = (tile % t.nta) * TG::T, tb0 = ((tile / t.nta) % t.ntb) * TG::T, tc0 = (tile / (t.nta * t.ntb)) * TG::T;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int la8 = lane & 7, lb4 = lane >> 3;
    const int n = min(t.cnt[b * t.ntile + tile], t.cap);
    const int *list = t.bin + ((size_t)b * t.ntile + tile) * t.cap;
    const R *rw = (const R *)a.rw;
    R *g = (R *)a.grid + (size_t)b * a.Na * a.Nb * a.Nc;
    for (int e = warp; e < n; e += nwarp) {
        const int idx = list[e];
        const int4 h = a.rhead[idx];
        const int oa = h.y - ta0, ob = h.z - tb0, oc = h.w - tc0;
        const R q = (R)a.charge[h.x];
        const R *w = rw + (size_t)idx * RG::NW;
        if (oa >= 0 && oa < TG::T && ob >= 0 && ob < TG::T && oc >= 0 && oc < TG::T) {
            R mc[NIP];
            load4<NIP>(mc, w + 2 * NIP);
            R mbl[NTB];
#pragma unroll
            for (int i = 0; i < NTB; i++) mbl[i] = lb4 + 4 * i < NI ? w[NIP + lb4 + 4 * i] : (R)0;
            R *base = tl + (oc * TG::E + ob + lb4) * TG::PA + oa + la8;
#pragma unroll
            for (int sa = 0; sa < NI; sa += 8) {
                if (la8 + sa >= NI) break;
                const R qa = q * w[la8 + sa];
#pragma unroll
                for (int tc = 0; tc < NI; tc++) {
                    const R cq = qa * mc[tc];
#pragma unroll
                    for (int i = 0; i < NTB; i++)
                        if (lb4 + 4 * i < NI) atomicAdd(base + (tc * TG::E + 4 * i) * TG::PA + sa, cq * mbl[i]);
                }
            }
        } else if (lane < 8) {
            LaneW<R, NI, false> lw;
            lw.load(rw, idx, lane);
            spread_global<R, NI>(a, g, h.y, h.z, h.w, lw, q, lane);
        }
    }
    const int grp = threadIdx.x >> 3, l8 = threadIdx.x & 7, ngrp = blockDim.x >> 3;
    const int nov = t.cnt[a.P * t.ntile];
    const int gid = blockIdx.y * gridDim.x + blockIdx.x, nblk = gridDim.x * gridDim.y;
    for (int e = gid * ngrp + grp; e < nov; e += nblk * ngrp) {
        const int idx = t.ovf[e];
        const int4 h = a.rhead[idx];
        LaneW<R, NI, false> lw;
        lw.load(rw, idx, l8);
        R *g2 = (R *)a.grid + (size_t)(idx % a.P) * a.Na * a.Nb * a.Nc;
        spread_global<R, NI>(a, g2, h.y, h.z, h.w, lw, (R)a.charge[h.x], l8);
    }
    __syncthreads();
    // add the shared copy to the grid, a warp per row (or rows)
    constexpr int NROW = TG::E * TG::E;
    if (sizeof(R) == 4 && (a.Na & 3) == 0) {
        constexpr int NQ = TG::PA / 4;
        constexpr int RPI = 32 / NQ;  // rows per warp step
        for (int r0 = warp * RPI; r0 < NROW; r0 += nwarp * RPI) {
            const int row = r0 + lane / NQ, q4 = lane % NQ;
            if (lane >= RPI * NQ || row >= NROW) continue;
            const float4 v = ((const float4 *)tl)[row * NQ + q4];
            if (v.x == 0.f && v.y == 0.f && v.z == 0.f && v.w == 0.f) continue;
            const int cz = row / TG::E, by = row - cz * TG::E;
            const int gc = wrapi(tc0 + cz, a.Nc), gb = wrapi(tb0 + by, a.Nb), ga = wrapi(ta0 + 4 * q4, a.Na);
            atomicAdd((float4 *)((float *)g + ((size_t)gc * a.Nb + gb) * a.Na + ga), v);
        }
    } else {
        for (int row = warp; row < NROW; row += nwarp) {
            const int cz = row / TG::E, by = row - cz * TG::E;
            R *dst = g + ((size_t)wrapi(tc0 + cz, a.Nc) * a.Nb + wrapi(tb0 + by, a.Nb)) * a.Na;
            for (int ax = lane; ax < TG::E; ax += 32) {
                const R v = tl[row * TG::PA + ax];
                if (v != (R)0) atomicAdd(dst + wrapi(ta0 + ax, a.Na), v);
            }
        }
    }
}

// Gather sums of one record for lane l8: d/ds_a, d/ds_b, d/ds_c of
// sum M_a M_b M_c phi over the lane's a points; phi(tc, tb, ta) reads the
// potential at stencil point (tc, tb, ta).  The a weights factor out of the
// b and c sums, so a stencil point costs one load and two FMAs.
template <typename R, int NI, typename PHI>
__device__ __forceinline__ void gather_lane(PHI phi, const LaneW<R, NI, true> &lw, int l8, double &ea, double &eb,
                                            double &ec)
{
    ea = eb = ec = 0.0;
    if (l8 >= NI) return;
    R xa = 0, xb = 0, xc = 0;
#pragma unroll
    for (int j = 0; j < (NI > 8 ? 2 : 1); j++) {
        if (j == 1 && l8 + 8 >= NI) break;
        const int ta = l8 + 8 * j;
        R sa = 0, sb = 0, sc = 0;
#pragma unroll
        for (int tc = 0; tc < NI; tc++) {
            R um = 0, ud = 0;
#pragma unroll
            for (int tb = 0; tb < NI; tb++) {
                const R p = phi(tc, tb, ta);
                um += lw.mb[tb] * p;
                ud += lw.db[tb] * p;
            }
            sa += lw.mc[tc] * um;
            sb += lw.mc[tc] * ud;
            sc += lw.dc[tc] * um;
        }
        const R wa = j ? lw.wa1 : lw.wa0, da = j ? lw.da1 : lw.da0;
        xa += da * sa;
        xb += wa * sb;
        xc += wa * sc;
    }
    ea = (double)xa;
    eb = (double)xb;
    ec = (double)xc;
}

// Force of one record from its three sums (summed over the 8-lane group;
// lane 0 writes): F = -q h^-T (N_a e_a, N_b e_b, N_c e_c), stored (not
// added) at the record's slot idx = k * P + b of the PME force buffer
// [nchrg][3][P]; every record is written exactly once per evaluation.
__device__ __forceinline__ void gather_store(const PmeArgs &a, const Cell &cell, int at, int idx, double ea,
                                             double eb, double ec, int l8)
{
#pragma unroll
    for (int o = 4; o >= 1; o >>= 1) {
        ea += __shfl_xor_sync(0xffffffffu, ea, o);
        eb += __shfl_xor_sync(0xffffffffu, eb, o);
        ec += __shfl_xor_sync(0xffffffffu, ec, o);
    }
    if (l8 != 0) return;
    ea *= (double)a.Na;
    eb *= (double)a.Nb;
    ec *= (double)a.Nc;
    const double q = a.charge[at];
    const double gx = ea * cell.hi[0] + eb * cell.hi[1] + ec * cell.hi[2];
    const double gy = ea * cell.hi[3] + eb * cell.hi[4] + ec * cell.hi[5];
    const double gz = ea * cell.hi[6] + eb * cell.hi[7] + ec * cell.hi[8];
    const int k = idx / a.P, b = idx - k * a.P;
    double *f = a.forceP;
    f[(3 * (size_t)k + 0) * a.P + b] = -gx * q;
    f[(3 * (size_t)k + 1) * a.P + b] = -gy * q;
    f[(3 * (size_t)k + 2) * a.P + b] = -gz * q;
}

// Adds the PME forces [nchrg][3][P] to the site forces [natm][3][P].
__device__ __forceinline__ void pme_force_add_body(int nchrg, int P, const int *__restrict__ ichrg,
                                                   const double *__restrict__ fP, double *__restrict__ fT, const VBlk vb)
{
    const long long t = (long long)vb.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nchrg * 3 * P) return;
    const long long kd = t / P;
    const int b = (int)(t - kd * P);
    const int k = (int)(kd / 3), d = (int)(kd - 3LL * k);
    fT[(3 * (size_t)ichrg[k] + d) * P + b] += fP[t];
}

__global__ void __launch_bounds__(256) pme_force_add_kernel(int nchrg, int P, const int *__restrict__ ichrg,
                                                            const double *__restrict__ fP, double *__restrict__ fT)
{
    pme_force_add_body(nchrg, P, ichrg, fP, fT, hw_blk());
}

// RESPA outer level: PME forces x wght_ter into another buffer
// (ewald3d_pme.c: forces x wght_now before they are added).
__global__ void __launch_bounds__(256) pme_force_add_scaled_kernel(int nchrg, int P, const int *__restrict__ ichrg,
                                                                   const double *__restrict__ fP, double w,
                                                                   double *__restrict__ fT)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nchrg * 3 * P) return;
    const long long kd = t / P;
    const int b = (int)(t - kd * P);
    const int k = (int)(kd / 3), d = (int)(kd - 3LL * k);
    fT[(3 * (size_t)ichrg[k] + d) * P + b] += fP[t] * w;
}

// Gather: one block per (tile, bead); the tile's potential (with the
// stencil reach) is copied to shared memory once and the bin's records read
// it there.  Overflow records read the grid directly.  Every (charge, bead)
// is handled by exactly one 8-lane group, so the force update needs no
// atomics.
template <typename R, int NI, int TT>
__global__ void __launch_bounds__(256) gather_tile_kernel(PmeArgs a, Cell cell, TileArgs t)
{
    typedef TileGeom<NI, TT> TG;
    extern __shared__ unsigned char smem_raw[];
    R *tl = (R *)smem_raw;
    const int tile = blockIdx.x, b = blockIdx.y;
    const int ta0 = (tile % t.nta) * TG::T, tb0 = ((tile / t.nta) % t.ntb) * TG::T, tc0 = (tile / (t.nta * t.ntb)) * TG::T;
    const R *g = (const R *)a.grid + (size_t)b * a.Na * a.Nb * a.Nc;
    const int n = min(t.cnt[b * t.ntile + tile], t.cap);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    if (n > 0) {
        constexpr int NROW = TG::E * TG::E;
        if (sizeof(R) == 4 && (a.Na & 3) == 0) {
            // 16-byte chunks; the padding column takes whatever the grid holds there
            constexpr int NQ = TG::PA / 4;
            constexpr int RPI = 32 / NQ;
            for (int r0 = warp * RPI; r0 < NROW; r0 += nwarp * RPI) {
                const int row = r0 + lane / NQ, q4 = lane % NQ;
                if (lane >= RPI * NQ || row >= NROW) continue;
                const int cz = row / TG::E, by = row - cz * TG::E;
                const float *src = (const float *)g +
                                   ((size_t)wrapi(tc0 + cz, a.Nc) * a.Nb + wrapi(tb0 + by, a.Nb)) * a.Na +
                                   wrapi(ta0 + 4 * q4, a.Na);
                ((float4 *)tl)[row * NQ + q4] = __ldg((const float4 *)src);
            }
        } else {
            for (int row = warp; row < NROW; row += nwarp) {
                const int cz = row / TG::E, by = row - cz * TG::E;
                const R *src = g + ((size_t)wrapi(tc0 + cz, a.Nc) * a.Nb + wrapi(tb0 + by, a.Nb)) * a.Na;
                for (int ax = lane; ax < TG::PA; ax += 32)
                    tl[row * TG::PA + ax] = ax < TG::E ? src[wrapi(ta0 + ax, a.Na)] : (R)0;
            }
        }
    }
    __syncthreads();
    const int grp = threadIdx.x >> 3, l8 = threadIdx.x & 7, ngrp = blockDim.x >> 3;
    const int *list = t.bin + ((size_t)b * t.ntile + tile) * t.cap;
    const R *rw = (const R *)a.rw;
    // every lane of a warp takes part in the group reductions: loop to the
    // same trip count in all groups of the warp
    const int nr = (n + ngrp - 1) / ngrp;
    for (int r = 0; r < nr; r++) {
        const int e = r * ngrp + grp;
        const bool act = e < n;
        int at = 0, idx = 0;
        double ea = 0, eb = 0, ec = 0;
        if (act) {
            idx = list[e];
            const int4 h = a.rhead[idx];
            at = h.x;
            LaneW<R, NI, true> lw;
            lw.load(rw, idx, l8);
            const int oa = h.y - ta0, ob = h.z - tb0, oc = h.w - tc0;
            if (oa >= 0 && oa < TG::T && ob >= 0 && ob < TG::T && oc >= 0 && oc < TG::T) {
                const R *base = tl + (oc * TG::E + ob) * TG::PA + oa;
                gather_lane<R, NI>([&](int tc, int tb, int ta) { return base[(tc * TG::E + tb) * TG::PA + ta]; }, lw,
                                   l8, ea, eb, ec);
            } else {
                const int la = h.y, lb = h.z, lc = h.w;
                gather_lane<R, NI>(
                    [&](int tc, int tb, int ta) {
                        return g[((size_t)wrapi(lc + tc, a.Nc) * a.Nb + wrapi(lb + tb, a.Nb)) * a.Na +
                                 wrapi(la + ta, a.Na)];
                    },
                    lw, l8, ea, eb, ec);
            }
        }
        gather_store(a, cell, at, idx, ea, eb, ec, act ? l8 : 1);
    }
    const int nov = t.cnt[a.P * t.ntile];
    const int gid = blockIdx.y * gridDim.x + blockIdx.x, nblk = gridDim.x * gridDim.y;
    const int nr2 = (nov + nblk * ngrp - 1) / (nblk * ngrp);
    for (int r = 0; r < nr2; r++) {
        const int e = (r * nblk + gid) * ngrp + grp;
        const bool act = e < nov;
        int at = 0, b2 = 0, idx = 0;
        double ea = 0, eb = 0, ec = 0;
        if (act) {
            idx = t.ovf[e];
            const int4 h = a.rhead[idx];
            b2 = idx % a.P;
            at = h.x;
            LaneW<R, NI, true> lw;
            lw.load(rw, idx, l8);
            const R *g2 = (const R *)a.grid + (size_t)b2 * a.Na * a.Nb * a.Nc;
            const int la = h.y, lb = h.z, lc = h.w;
            gather_lane<R, NI>(
                [&](int tc, int tb, int ta) {
                    return g2[((size_t)wrapi(lc + tc, a.Nc) * a.Nb + wrapi(lb + tb, a.Nb)) * a.Na +
                              wrapi(la + ta, a.Na)];
                },
                lw, l8, ea, eb, ec);
        }
        gather_store(a, cell, at, idx, ea, eb, ec, act ? l8 : 1);
    }
}

// ---------------------------------------------------------------------------
// Compact forward path: bin, spread and gather without weight records.
//
// B-spline weights as polynomials of the fractional offset.  PINY's
// recursion (ewald3d_pme.c:301-338) makes the weight m[j] of order NI (at
// u = f + j - 1) a polynomial of degree NI - 1 in f on [0, 1), and the
// derivative weight dm[j] = m'[j] - m'[j - 1] formed from the order NI - 1
// splines (:512-532) one of degree NI - 2.  BsplinePoly runs that recursion
// on coefficient arrays at compile time; the kernels evaluate each lane's
// weights by Horner from a shared-memory copy.  The bin kernel writes, per
// (charge, bead), only the stencil origin and the three fractional offsets
// with the charge (32 bytes in FP32) instead of the 6 x NIP weights, and
// spread and gather read the next record while they work on the current one.
template <int NI>
struct BsplinePoly {
    double m[NI][NI];   // m[p][d]: coefficient of f^d of PINY's m[p + 1]
    double dm[NI][NI];  // dm[p][d]: of PINY's dm[p + 1]
    constexpr BsplinePoly() : m(), dm()
    {
        double cur[NI + 1][NI + 1] = {};
        cur[1][1] = 1.0;   // m[1] = 1 - |u_1 - 1| = f
        cur[2][0] = 1.0;   // m[2] = 1 - |u_2 - 1| = 1 - f
        cur[2][1] = -1.0;
        for (int nn = 3; nn <= NI; nn++) {
            const double rn1 = 1.0 / (double)(nn - 1);
            // m[j] = (u_j m[j] + (nn - u_j) m[j - 1]) / (nn - 1), u_j = f + j - 1
            for (int j = nn; j >= 2; j--) {
                double nw[NI + 1] = {};
                for (int d = 0; d < NI; d++) {
                    nw[d] += (double)(j - 1) * cur[j][d] + (double)(nn - j + 1) * cur[j - 1][d];
                    nw[d + 1] += cur[j][d] - cur[j - 1][d];
                }
                for (int d = 0; d <= NI; d++) cur[j][d] = nw[d] * rn1;
            }
            double nw1[NI + 1] = {};
            for (int d = 0; d < NI; d++) nw1[d + 1] = cur[1][d];
            for (int d = 0; d <= NI; d++) cur[1][d] = nw1[d] * rn1;
            if (nn == NI - 1)
                for (int j = 1; j <= NI; j++)
                    for (int d = 0; d < NI; d++) dm[j - 1][d] = cur[j][d] - (j >= 2 ? cur[j - 1][d] : 0.0);
        }
        for (int j = 1; j <= NI; j++)
            for (int d = 0; d < NI; d++) m[j - 1][d] = cur[j][d];
    }
};

template <int NI>
__constant__ BsplinePoly<NI> kBspline = BsplinePoly<NI>();

// Shared copy of the polynomials in R, rows padded to a multiple of 4.
template <typename R, int NI>
struct PolyTab {
    static constexpr int NP4 = (NI + 3) & ~3;
    R m[NI][NP4], dm[NI][NP4];
    __device__ __forceinline__ void fill(bool deriv)
    {
        for (int i = threadIdx.x; i < NI * NP4; i += blockDim.x) {
            const int p = i / NP4, d = i - p * NP4;
            m[p][d] = d < NI ? (R)kBspline<NI>.m[p][d] : (R)0;
            if (deriv) dm[p][d] = d < NI ? (R)kBspline<NI>.dm[p][d] : (R)0;
        }
    }
};

// Weight of stencil point t (grid index lo + t carries PINY's m[NI - t],
// piece NI - 1 - t) from its coefficient row, by Horner.
template <typename R, int NI>
__device__ __forceinline__ R poly_eval(const R (&row)[PolyTab<R, NI>::NP4], R f)
{
    constexpr int NP4 = PolyTab<R, NI>::NP4;
    R c[NP4];
    if constexpr (sizeof(R) == 4) {
#pragma unroll
        for (int i = 0; i < NP4; i += 4) {
            const float4 v = *(const float4 *)&row[i];
            c[i] = v.x;
            c[i + 1] = v.y;
            c[i + 2] = v.z;
            c[i + 3] = v.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < NP4; i += 2) {
            const double2 v = *(const double2 *)&row[i];
            c[i] = v.x;
            c[i + 1] = v.y;
        }
    }
    R w = c[NI - 1];
#pragma unroll
    for (int d = NI - 2; d >= 0; d--) w = w * f + c[d];
    return w;
}

template <typename R>
__device__ __forceinline__ typename Vec4<R>::T load_frac(const void *rw, int idx)
{
    if constexpr (sizeof(R) == 4) return __ldg((const float4 *)rw + idx);
    else return ldg4((const double4 *)rw + idx);
}

// Bin kernel of the compact path: one thread per (charge, bead), stencil
// origin in FP64 with PINY's operation order (as pme_bin_kernel), record
// (atom, la, lb, lc) + (fa, fb, fc, q), record number filed under its tile.
template <typename R, int NI>
__device__ __forceinline__ void pme_bin_compact_body(const PmeArgs &a, const Cell &cell, const TileArgs &t,
                                                     const VBlk vb)
{
    const long long idx = (long long)vb.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)a.nchrg * a.P) return;
    const int b = (int)(idx % a.P);
    const int k = (int)(idx / a.P);
    const int at = a.ichrg[k];
    int la, lb, lc;
    double fa, fb, fc;
    stencil_origin(a, cell, at, b, NI, la, lb, lc, fa, fb, fc);
    typename Vec4<R>::T fr;
    fr.x = (R)fa;
    fr.y = (R)fb;
    fr.z = (R)fc;
    fr.w = (R)a.charge[at];
    ((typename Vec4<R>::T *)a.rw)[idx] = fr;
    a.rhead[idx] = make_int4(at, la, lb, lc);
    const int T = t.T;
    const int tile = ((lc / T) * t.ntb + lb / T) * t.nta + la / T;
    const int slot = atomicAdd(&t.cnt[b * t.ntile + tile], 1);
    if (slot < t.cap) t.bin[((size_t)b * t.ntile + tile) * t.cap + slot] = (int)idx;
    else t.ovf[atomicAdd(&t.cnt[a.P * t.ntile], 1)] = (int)idx;
}

template <typename R, int NI>
__global__ void __launch_bounds__(256) pme_bin_compact_kernel(const __grid_constant__ PmeArgs a,
                                                              const __grid_constant__ Cell cell,
                                                              const __grid_constant__ TileArgs t)
{
    pme_bin_compact_body<R, NI>(a, cell, t, hw_blk());
}

// Weights one spread lane needs (lanes = 8 a points x 4 b rows): its a
// points la8 (+8), its b rows lb4 + 4 i, and all c points, the latter
// evaluated by lanes 0..NI-1 and shuffled.  Every lane of the warp calls it.
template <typename R, int NI>
struct SpreadW {
    static constexpr int NTB = (NI + 3) / 4, NSA = (NI + 7) / 8;
    R wa[NSA], mb[NTB], mc[NI];
    __device__ __forceinline__ void eval(const PolyTab<R, NI> &pt, const typename Vec4<R>::T &fr, int lane)
    {
        const int la8 = lane & 7, lb4 = lane >> 3;
#pragma unroll
        for (int s = 0; s < NSA; s++) wa[s] = la8 + 8 * s < NI ? poly_eval<R, NI>(pt.m[NI - 1 - (la8 + 8 * s)], fr.x) : (R)0;
#pragma unroll
        for (int i = 0; i < NTB; i++) mb[i] = lb4 + 4 * i < NI ? poly_eval<R, NI>(pt.m[NI - 1 - (lb4 + 4 * i)], fr.y) : (R)0;
        const R mcl = lane < NI ? poly_eval<R, NI>(pt.m[NI - 1 - lane], fr.z) : (R)0;
#pragma unroll
        for (int tc = 0; tc < NI; tc++) mc[tc] = __shfl_sync(0xffffffffu, mcl, tc);
    }
};

// One record spread straight into the grid g of its bead (origin outside
// the block's tile, or an overflow record); a warp, lanes as SpreadW.
template <typename R, int NI>
__device__ __forceinline__ void spread_warp_global(const PmeArgs &a, R *g, int la, int lb, int lc,
                                                   const SpreadW<R, NI> &w, R q, int lane)
{
    const int la8 = lane & 7, lb4 = lane >> 3;
#pragma unroll
    for (int s = 0; s < SpreadW<R, NI>::NSA; s++) {
        if (la8 + 8 * s >= NI) break;
        const int ga = wrapi(la + la8 + 8 * s, a.Na);
        const R qa = q * w.wa[s];
#pragma unroll
        for (int tc = 0; tc < NI; tc++) {
            const int gc = wrapi(lc + tc, a.Nc);
            const R cq = qa * w.mc[tc];
#pragma unroll
            for (int i = 0; i < SpreadW<R, NI>::NTB; i++)
                if (lb4 + 4 * i < NI) atomicAdd(g + ((size_t)gc * a.Nb + wrapi(lb + lb4 + 4 * i, a.Nb)) * a.Na + ga, cq * w.mb[i]);
        }
    }
}

// Spread of the compact path: as spread_tile_kernel (one block per (tile,
// bead), one warp per record into a shared copy of the tile, the copy added
// to the grid once), with the weights evaluated in the block and the next
// record read ahead.
template <typename R, int NI, int TT>
__device__ __forceinline__ void spread_tile_c_body(const PmeArgs &a, const TileArgs &t, const VBlk vb)
{
    typedef TileGeom<NI, TT> TG;
    typedef typename Vec4<R>::T R4;
    constexpr int NTB = SpreadW<R, NI>::NTB;
    extern __shared__ unsigned char smem_raw[];
    R *tl = (R *)smem_raw;
    __shared__ __align__(16) PolyTab<R, NI> pt;
    for (int i = threadIdx.x; i < TG::NPT; i += blockDim.x) tl[i] = (R)0;
    pt.fill(false);
    __syncthreads();
    const int tile = vb.x, b = vb.y;
    const int ta0 = (tile % t.nta) * TG::T, tb0 = ((tile / t.nta) % t.ntb) * TG::T, tc0 = (tile / (t.nta * t.ntb)) * TG::T;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int la8 = lane & 7, lb4 = lane >> 3;
    const int n = min(t.cnt[b * t.ntile + tile], t.cap);
    const int *list = t.bin + ((size_t)b * t.ntile + tile) * t.cap;
    R *g = (R *)a.grid + (size_t)b * a.Na * a.Nb * a.Nc;
    int4 hn = make_int4(0, 0, 0, 0);
    R4 fn = {};
    if (warp < n) {
        const int idx = list[warp];
        hn = a.rhead[idx];
        fn = load_frac<R>(a.rw, idx);
    }
    for (int e = warp; e < n; e += nwarp) {
        const int4 h = hn;
        const R4 fr = fn;
        if (e + nwarp < n) {
            const int idx = list[e + nwarp];
            hn = a.rhead[idx];
            fn = load_frac<R>(a.rw, idx);
        }
        SpreadW<R, NI> w;
        w.eval(pt, fr, lane);
        const R q = fr.w;
        const int oa = h.y - ta0, ob = h.z - tb0, oc = h.w - tc0;
        if (oa >= 0 && oa < TG::T && ob >= 0 && ob < TG::T && oc >= 0 && oc < TG::T) {
            const int off0 = (oc * TG::E + ob + lb4) * TG::PA + oa + la8;
#pragma unroll
            for (int s = 0; s < SpreadW<R, NI>::NSA; s++) {
                if (la8 + 8 * s >= NI) break;
                const R qa = q * w.wa[s];
#pragma unroll
                for (int tc = 0; tc < NI; tc++) {
                    const R cq = qa * w.mc[tc];
#pragma unroll
                    for (int i = 0; i < NTB; i++) {
                        if (lb4 + 4 * i >= NI) continue;
                        const int o = off0 + (tc * TG::E + 4 * i) * TG::PA + 8 * s;
                        if constexpr (sizeof(R) == 4) {
                            // fixed point: v 2^S + 1.5 2^23 is exact to the nearest
                            // integer for |v 2^S| < 2^22, whose bits less those of
                            // 1.5 2^23 are that integer; integer shared atomics run
                            // at twice the rate of FP32 ones
                            const float y = fmaf(cq * w.mb[i], t.qfix, 12582912.0f);
                            atomicAdd((int *)tl + o, __float_as_int(y) - 0x4B400000);
                        } else {
                            atomicAdd(tl + o, cq * w.mb[i]);
                        }
                    }
                }
            }
        } else {
            spread_warp_global<R, NI>(a, g, h.y, h.z, h.w, w, q, lane);
        }
    }
    // overflow records: one warp each, straight into the grid
    const int nov = t.cnt[a.P * t.ntile];
    const int gid = vb.y * vb.gx + vb.x, nblk = vb.gx * vb.gy;
    for (int e = gid * nwarp + warp; e < nov; e += nblk * nwarp) {
        const int idx = t.ovf[e];
        const int4 h = a.rhead[idx];
        const R4 fr = load_frac<R>(a.rw, idx);
        SpreadW<R, NI> w;
        w.eval(pt, fr, lane);
        R *g2 = (R *)a.grid + (size_t)(idx % a.P) * a.Na * a.Nb * a.Nc;
        spread_warp_global<R, NI>(a, g2, h.y, h.z, h.w, w, fr.w, lane);
    }
    __syncthreads();
    constexpr int NROW = TG::E * TG::E;
    if (sizeof(R) == 4 && (a.Na & 3) == 0) {
        constexpr int NQ = TG::PA / 4;
        constexpr int RPI = 32 / NQ;
        for (int r0 = warp * RPI; r0 < NROW; r0 += nwarp * RPI) {
            const int row = r0 + lane / NQ, q4 = lane % NQ;
            if (lane >= RPI * NQ || row >= NROW) continue;
            const int4 iv = ((const int4 *)tl)[row * NQ + q4];
            if ((iv.x | iv.y | iv.z | iv.w) == 0) continue;
            const float4 v = make_float4((float)iv.x * t.qfix_inv, (float)iv.y * t.qfix_inv,
                                         (float)iv.z * t.qfix_inv, (float)iv.w * t.qfix_inv);
            const int cz = row / TG::E, by = row - cz * TG::E;
            const int gc = wrapi(tc0 + cz, a.Nc), gb = wrapi(tb0 + by, a.Nb), ga = wrapi(ta0 + 4 * q4, a.Na);
            atomicAdd((float4 *)((float *)g + ((size_t)gc * a.Nb + gb) * a.Na + ga), v);
        }
    } else {
        for (int row = warp; row < NROW; row += nwarp) {
            const int cz = row / TG::E, by = row - cz * TG::E;
            R *dst = g + ((size_t)wrapi(tc0 + cz, a.Nc) * a.Nb + wrapi(tb0 + by, a.Nb)) * a.Na;
            for (int ax = lane; ax < TG::E; ax += 32) {
                R v;
                if constexpr (sizeof(R) == 4) v = (R)((float)((const int *)tl)[row * TG::PA + ax] * t.qfix_inv);
                else v = tl[row * TG::PA + ax];
                if (v != (R)0) atomicAdd(dst + wrapi(ta0 + ax, a.Na), v);
            }
        }
    }
}

template <typename R, int NI, int TT>
__global__ void __launch_bounds__(256) spread_tile_c_kernel(const __grid_constant__ PmeArgs a,
                                                            const __grid_constant__ TileArgs t)
{
    spread_tile_c_body<R, NI, TT>(a, t, hw_blk());
}

// Gather weights of one record for lane l8 of an 8-lane group: its a
// points (l8, l8 + 8) with derivatives, and all b and c points, evaluated by
// lane t % 8 of the group and shuffled.  Every lane of the warp calls it.
template <typename R, int NI>
__device__ __forceinline__ void gather_weights(const PolyTab<R, NI> &pt, const typename Vec4<R>::T &fr, int l8,
                                               LaneW<R, NI, true> &lw)
{
    const bool t0 = l8 < NI, t1 = NI > 8 && l8 + 8 < NI;
    const int p0 = NI - 1 - (t0 ? l8 : 0), p1 = NI - 1 - (t1 ? l8 + 8 : 0);
    lw.wa0 = t0 ? poly_eval<R, NI>(pt.m[p0], fr.x) : (R)0;
    lw.da0 = t0 ? poly_eval<R, NI>(pt.dm[p0], fr.x) : (R)0;
    lw.wa1 = t1 ? poly_eval<R, NI>(pt.m[p1], fr.x) : (R)0;
    lw.da1 = t1 ? poly_eval<R, NI>(pt.dm[p1], fr.x) : (R)0;
    R ob[2], odb[2], oc[2], odc[2];
    ob[0] = t0 ? poly_eval<R, NI>(pt.m[p0], fr.y) : (R)0;
    odb[0] = t0 ? poly_eval<R, NI>(pt.dm[p0], fr.y) : (R)0;
    oc[0] = t0 ? poly_eval<R, NI>(pt.m[p0], fr.z) : (R)0;
    odc[0] = t0 ? poly_eval<R, NI>(pt.dm[p0], fr.z) : (R)0;
    ob[1] = t1 ? poly_eval<R, NI>(pt.m[p1], fr.y) : (R)0;
    odb[1] = t1 ? poly_eval<R, NI>(pt.dm[p1], fr.y) : (R)0;
    oc[1] = t1 ? poly_eval<R, NI>(pt.m[p1], fr.z) : (R)0;
    odc[1] = t1 ? poly_eval<R, NI>(pt.dm[p1], fr.z) : (R)0;
#pragma unroll
    for (int s = 0; s < RecGeom<NI>::NIP; s++) {
        if (s >= NI) {
            lw.mb[s] = lw.mc[s] = lw.db[s] = lw.dc[s] = (R)0;
            continue;
        }
        const int h = s >= 8 ? 1 : 0;
        lw.mb[s] = __shfl_sync(0xffffffffu, ob[h], s & 7, 8);
        lw.db[s] = __shfl_sync(0xffffffffu, odb[h], s & 7, 8);
        lw.mc[s] = __shfl_sync(0xffffffffu, oc[h], s & 7, 8);
        lw.dc[s] = __shfl_sync(0xffffffffu, odc[h], s & 7, 8);
    }
}

// Gather of the compact path: as gather_tile_kernel (one block per (tile,
// bead), the tile's potential copied to shared memory once, 8 lanes per
// record), with the weights evaluated in the block and the next record
// read ahead.
template <typename R, int NI, int TT>
__device__ __forceinline__ void gather_tile_c_body(const PmeArgs &a, const Cell &cell, const TileArgs &t, const VBlk vb)
{
    typedef TileGeom<NI, TT> TG;
    typedef typename Vec4<R>::T R4;
    extern __shared__ unsigned char smem_raw[];
    R *tl = (R *)smem_raw;
    __shared__ __align__(16) PolyTab<R, NI> pt;
    pt.fill(true);
    const int tile = vb.x, b = vb.y;
    const int ta0 = (tile % t.nta) * TG::T, tb0 = ((tile / t.nta) % t.ntb) * TG::T, tc0 = (tile / (t.nta * t.ntb)) * TG::T;
    const R *g = (const R *)a.grid + (size_t)b * a.Na * a.Nb * a.Nc;
    const int n = min(t.cnt[b * t.ntile + tile], t.cap);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    if (n > 0) {
        constexpr int NROW = TG::E * TG::E;
        if (sizeof(R) == 4 && (a.Na & 3) == 0) {
            constexpr int NQ = TG::PA / 4;
            constexpr int RPI = 32 / NQ;
            for (int r0 = warp * RPI; r0 < NROW; r0 += nwarp * RPI) {
                const int row = r0 + lane / NQ, q4 = lane % NQ;
                if (lane >= RPI * NQ || row >= NROW) continue;
                const int cz = row / TG::E, by = row - cz * TG::E;
                const float *src = (const float *)g +
                                   ((size_t)wrapi(tc0 + cz, a.Nc) * a.Nb + wrapi(tb0 + by, a.Nb)) * a.Na +
                                   wrapi(ta0 + 4 * q4, a.Na);
                ((float4 *)tl)[row * NQ + q4] = __ldg((const float4 *)src);
            }
        } else {
            for (int row = warp; row < NROW; row += nwarp) {
                const int cz = row / TG::E, by = row - cz * TG::E;
                const R *src = g + ((size_t)wrapi(tc0 + cz, a.Nc) * a.Nb + wrapi(tb0 + by, a.Nb)) * a.Na;
                for (int ax = lane; ax < TG::PA; ax += 32)
                    tl[row * TG::PA + ax] = ax < TG::E ? src[wrapi(ta0 + ax, a.Na)] : (R)0;
            }
        }
    }
    __syncthreads();
    const int grp = threadIdx.x >> 3, l8 = threadIdx.x & 7, ngrp = blockDim.x >> 3;
    const int *list = t.bin + ((size_t)b * t.ntile + tile) * t.cap;
    const int nr = (n + ngrp - 1) / ngrp;  // same trip count in every group of a warp (shuffles)
    int4 hn = make_int4(0, 0, 0, 0);
    R4 fn = {};
    int in = 0;
    if (grp < n) {
        in = list[grp];
        hn = a.rhead[in];
        fn = load_frac<R>(a.rw, in);
    }
    for (int r = 0; r < nr; r++) {
        const int e = r * ngrp + grp;
        const bool act = e < n;
        const int idx = in;
        const int4 h = hn;
        const R4 fr = fn;
        if (e + ngrp < n) {
            in = list[e + ngrp];
            hn = a.rhead[in];
            fn = load_frac<R>(a.rw, in);
        }
        LaneW<R, NI, true> lw;
        gather_weights<R, NI>(pt, fr, l8, lw);
        double ea = 0, eb = 0, ec = 0;
        if (act) {
            const int oa = h.y - ta0, ob = h.z - tb0, oc = h.w - tc0;
            if (oa >= 0 && oa < TG::T && ob >= 0 && ob < TG::T && oc >= 0 && oc < TG::T) {
                const R *base = tl + (oc * TG::E + ob) * TG::PA + oa;
                gather_lane<R, NI>([&](int tc, int tb, int ta) { return base[(tc * TG::E + tb) * TG::PA + ta]; }, lw,
                                   l8, ea, eb, ec);
            } else {
                gather_lane<R, NI>(
                    [&](int tc, int tb, int ta) {
                        return g[((size_t)wrapi(h.w + tc, a.Nc) * a.Nb + wrapi(h.z + tb, a.Nb)) * a.Na +
                                 wrapi(h.y + ta, a.Na)];
                    },
                    lw, l8, ea, eb, ec);
            }
        }
        gather_store(a, cell, h.x, idx, ea, eb, ec, act ? l8 : 1);
    }
    const int nov = t.cnt[a.P * t.ntile];
    const int gid = vb.y * vb.gx + vb.x, nblk = vb.gx * vb.gy;
    const int nr2 = (nov + nblk * ngrp - 1) / (nblk * ngrp);
    for (int r = 0; r < nr2; r++) {
        const int e = (r * nblk + gid) * ngrp + grp;
        const bool act = e < nov;
        int idx = 0;
        int4 h = make_int4(0, 0, 0, 0);
        R4 fr = {};
        if (act) {
            idx = t.ovf[e];
            h = a.rhead[idx];
            fr = load_frac<R>(a.rw, idx);
        }
        LaneW<R, NI, true> lw;
        gather_weights<R, NI>(pt, fr, l8, lw);
        double ea = 0, eb = 0, ec = 0;
        if (act) {
            const R *g2 = (const R *)a.grid + (size_t)(idx % a.P) * a.Na * a.Nb * a.Nc;
            gather_lane<R, NI>(
                [&](int tc, int tb, int ta) {
                    return g2[((size_t)wrapi(h.w + tc, a.Nc) * a.Nb + wrapi(h.z + tb, a.Nb)) * a.Na +
                              wrapi(h.y + ta, a.Na)];
                },
                lw, l8, ea, eb, ec);
        }
        gather_store(a, cell, h.x, idx, ea, eb, ec, act ? l8 : 1);
    }
}

// Resident blocks per SM the FP32 gather (order <= 8) is compiled for: its
// shared tile of 16-point edges allows 4; at 4 the 64-register cap spills
// 60 bytes and the C3 evaluation is still 2.8 % faster than at 3 (80
// registers).  The others hold 2 (128 registers).
#ifndef PINYB200_GATHER_BLOCKS
#define PINYB200_GATHER_BLOCKS 4
#endif
template <typename R, int NI, int TT>
__global__ void __launch_bounds__(256, sizeof(R) == 4 && NI <= 8 ? PINYB200_GATHER_BLOCKS : 2)
    gather_tile_c_kernel(const __grid_constant__ PmeArgs a,
                                                            const __grid_constant__ Cell cell,
                                                            const __grid_constant__ TileArgs t)
{
    gather_tile_c_body<R, NI, TT>(a, cell, t, hw_blk());
}

// ---------------------------------------------------------------------------
// In-place FFTs of `nl` lines of length N held in shared memory: element n of
// line l at sm[l * ls + n * es].  Unnormalised, exp(sign 2 pi i n k / N);
// tw[2m], tw[2m+1] = cos, sin(2 pi m / N).  Power-of-two lengths up to 256
// use Stockham autosort passes of radix 8 and 4 (16 = 4x4, 32 = 8x4,
// 64 = 8x8, 128 = 8x4x4, 256 = 8x8x4): one butterfly per thread and pass,
// read into registers, barrier, written back in place.  Other lengths use a
// direct DFT done a block of lines at a time.  Every thread of the block
// must call these.

// R-point DFT in registers, exp(SIGN 2 pi i r k / R), R = 2, 4, 8.
template <typename R, int RAD, int SIGN>
__device__ __forceinline__ void dft_small(typename Cplx<R>::T *v)
{
    typedef typename Cplx<R>::T C2;
    if (RAD == 2) {
        const C2 a = v[0], b = v[1];
        v[0].x = a.x + b.x;
        v[0].y = a.y + b.y;
        v[1].x = a.x - b.x;
        v[1].y = a.y - b.y;
    } else if (RAD == 4) {
        const R s = (R)SIGN;
        const C2 t0 = {v[0].x + v[2].x, v[0].y + v[2].y}, t1 = {v[0].x - v[2].x, v[0].y - v[2].y};
        const C2 t2 = {v[1].x + v[3].x, v[1].y + v[3].y};
        // (v1 - v3) * (SIGN i)
        const C2 t3 = {-s * (v[1].y - v[3].y), s * (v[1].x - v[3].x)};
        v[0].x = t0.x + t2.x;
        v[0].y = t0.y + t2.y;
        v[2].x = t0.x - t2.x;
        v[2].y = t0.y - t2.y;
        v[1].x = t1.x + t3.x;
        v[1].y = t1.y + t3.y;
        v[3].x = t1.x - t3.x;
        v[3].y = t1.y - t3.y;
    } else {
        // radix 2 over two 4-point DFTs: X_k = E_k + w^k O_k, X_k+4 = E_k - w^k O_k
        C2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
        dft_small<R, 4, SIGN>(e);
        dft_small<R, 4, SIGN>(o);
        const R s = (R)SIGN, h = (R)0.70710678118654752440;  // cos(pi/4)
        C2 w[4];
        w[0] = o[0];
        w[1] = {h * (o[1].x - s * o[1].y), h * (o[1].y + s * o[1].x)};   // (1 + s i) / sqrt 2
        w[2] = {-s * o[2].y, s * o[2].x};                                  // s i
        w[3] = {h * (-o[3].x - s * o[3].y), h * (-o[3].y + s * o[3].x)};  // (-1 + s i) / sqrt 2
#pragma unroll
        for (int k = 0; k < 4; k++) {
            v[k].x = e[k].x + w[k].x;
            v[k].y = e[k].y + w[k].y;
            v[k + 4].x = e[k].x - w[k].x;
            v[k + 4].y = e[k].y - w[k].y;
        }
    }
}

__host__ __device__ constexpr int stockham_radix(int rem) { return rem == 16 ? 4 : (rem % 8 == 0 ? 8 : rem); }
__host__ __device__ constexpr int stockham_min_radix(int n, int ns)
{
    return ns >= n ? 8 : (stockham_radix(n / ns) < stockham_min_radix(n, ns * stockham_radix(n / ns))
                              ? stockham_radix(n / ns)
                              : stockham_min_radix(n, ns * stockham_radix(n / ns)));
}

// One Stockham pass (stride NS) over lines l0 .. l0+nlg-1, then the next.
// Consecutive threads take consecutive lines (G lines per round) and share
// the butterfly index j: a half-warp then touches 16 different lines at the
// same position, which fall in 16 different bank pairs both for lines along
// the fast axis (odd line stride) and across it (line stride 1), and reads
// one twiddle (a broadcast).
template <typename R, int N, int NS, int SIGN>
__device__ __forceinline__ void stockham_pass(typename Cplx<R>::T *sm, int l0, int nlg, int G, int ls, int es,
                                              const R *tw)
{
    typedef typename Cplx<R>::T C2;
    constexpr int RAD = stockham_radix(N / NS);
    constexpr int BPL = N / RAD;  // butterflies per line
    const int l = threadIdx.x % G, j = threadIdx.x / G;
    const bool act = l < nlg && j < BPL;
    C2 v[RAD];
    C2 *p = sm + (size_t)(l0 + (act ? l : 0)) * ls;
    if (act) {
#pragma unroll
        for (int r = 0; r < RAD; r++) v[r] = p[(j + r * BPL) * es];
        if (NS > 1) {
            const int k = j % NS;
#pragma unroll
            for (int r = 1; r < RAD; r++) {
                const int m = r * k * (N / (NS * RAD));
                const R wr = tw[2 * m], wi = (R)SIGN * tw[2 * m + 1];
                const R xr = v[r].x * wr - v[r].y * wi, xi = v[r].x * wi + v[r].y * wr;
                v[r].x = xr;
                v[r].y = xi;
            }
        }
        dft_small<R, RAD, SIGN>(v);
    }
    __syncthreads();
    if (act) {
        const int d = (j / NS) * NS * RAD + j % NS;
#pragma unroll
        for (int r = 0; r < RAD; r++) p[(d + r * NS) * es] = v[r];
    }
    __syncthreads();
    if constexpr (NS * RAD < N) stockham_pass<R, N, NS * RAD, SIGN>(sm, l0, nlg, G, ls, es, tw);
}

template <typename R, int N, int SIGN>
__device__ __forceinline__ void fft_pow2_inl(typename Cplx<R>::T *sm, int nl, int ls, int es, const R *tw)
{
    constexpr int BPLMAX = N / stockham_min_radix(N, 1);
    const int G = (int)blockDim.x / BPLMAX > 0 ? (int)blockDim.x / BPLMAX : 1;  // lines per round
    for (int l0 = 0; l0 < nl; l0 += G) stockham_pass<R, N, 1, SIGN>(sm, l0, min(G, nl - l0), G, ls, es, tw);
}

// Out-of-line copy for kernels whose lengths are known only at run time.
template <typename R, int N, int SIGN>
__device__ __noinline__ void fft_pow2(typename Cplx<R>::T *sm, int nl, int ls, int es, const R *tw)
{
    fft_pow2_inl<R, N, SIGN>(sm, nl, ls, es, tw);
}

template <typename R, int SIGN>
__device__ bool fft_pow2_dispatch(typename Cplx<R>::T *sm, int N, int nl, int ls, int es, const R *tw)
{
    switch (N) {
    case 2: fft_pow2<R, 2, SIGN>(sm, nl, ls, es, tw); return true;
    case 4: fft_pow2<R, 4, SIGN>(sm, nl, ls, es, tw); return true;
    case 8: fft_pow2<R, 8, SIGN>(sm, nl, ls, es, tw); return true;
    case 16: fft_pow2<R, 16, SIGN>(sm, nl, ls, es, tw); return true;
    case 32: fft_pow2<R, 32, SIGN>(sm, nl, ls, es, tw); return true;
    case 64: fft_pow2<R, 64, SIGN>(sm, nl, ls, es, tw); return true;
    case 128: fft_pow2<R, 128, SIGN>(sm, nl, ls, es, tw); return true;
    case 256: fft_pow2<R, 256, SIGN>(sm, nl, ls, es, tw); return true;
    default: return false;
    }
}

template <typename R>
__device__ void smem_fft(typename Cplx<R>::T *sm, int N, int nl, int ls, int es, const R *tw, int sign)
{
    typedef typename Cplx<R>::T C2;
    const int nt = blockDim.x;
    if (N == 1) return;
    if (sign > 0 ? fft_pow2_dispatch<R, 1>(sm, N, nl, ls, es, tw) : fft_pow2_dispatch<R, -1>(sm, N, nl, ls, es, tw))
        return;
    {
        const int per = nt / N;  // lines per pass
        for (int l0 = 0; l0 < nl; l0 += per) {
            const int l = l0 + threadIdx.x / N, k = threadIdx.x % N;
            R sr = 0, si = 0;
            const bool act = threadIdx.x < per * N && l < nl;
            if (act) {
                const C2 *p = sm + l * ls;
                for (int n = 0; n < N; n++) {
                    const int e = (int)(((long long)n * k) % N);
                    const R wr = tw[2 * e], wi = (R)sign * tw[2 * e + 1];
                    const C2 v = p[n * es];
                    sr += v.x * wr - v.y * wi;
                    si += v.x * wi + v.y * wr;
                }
            }
            __syncthreads();
            if (act) {
                sm[l * ls + k * es].x = sr;
                sm[l * ls + k * es].y = si;
            }
            __syncthreads();
        }
    }
}

// FFT of length NF known at compile time (NF > 0), else run-time N.
template <typename R, int NF>
__device__ __forceinline__ void line_fft(typename Cplx<R>::T *sm, int N, int nl, int ls, int es, const R *tw, int sign)
{
    if constexpr (NF > 0) {
        if (sign > 0) fft_pow2_inl<R, NF, 1>(sm, nl, ls, es, tw);
        else fft_pow2_inl<R, NF, -1>(sm, nl, ls, es, tw);
    } else {
        smem_fft<R>(sm, N, nl, ls, es, tw, sign);
    }
}

// Resident blocks per SM the FP32 plane and slab kernels of compile-time
// length are compiled for (their registers: 65536 / (256 x this)); the
// FP64 ones and the multi-box ones (whose run-time argument table costs
// registers) hold 2.
#ifndef PINYB200_FFT_BLOCKS
#define PINYB200_FFT_BLOCKS 4
#endif
#ifndef PINYB200_PLANE_BLOCKS
#define PINYB200_PLANE_BLOCKS PINYB200_FFT_BLOCKS  // the plane passes alone (their shared plane allows 6)
#endif
#define PINYB200_FFT_LB(R, NF) (NF > 0 ? (sizeof(R) == 4 ? PINYB200_FFT_BLOCKS : 2) : 1)
#define PINYB200_PLANE_LB(R, NF) (NF > 0 ? (sizeof(R) == 4 ? PINYB200_PLANE_BLOCKS : 2) : 1)

template <typename R>
__device__ __forceinline__ void load_twiddles(R *dst, const R *src, int N)
{
    for (int i = threadIdx.x; i < 2 * N; i += blockDim.x) dst[i] = src[i];
}

// Forward transform of one (bead, c) plane along a then b; half spectrum
// (a <= Na/2) out.  Shared: plane [Nb][Na+1] complex, twiddles.
template <typename R, int NF>
__device__ __forceinline__ void plane_fwd_body(const R *__restrict__ q, typename Cplx<R>::T *__restrict__ spec, int Na,
                                               int Nb, int Nc, const R *__restrict__ twa, const R *__restrict__ twb,
                                               const VBlk vb)
{
    if (NF > 0) Na = Nb = NF;  // cubic power-of-two grid known at compile time
    (void)Nc;
    typedef typename Cplx<R>::T C2;
    extern __shared__ unsigned char smem_raw[];
    C2 *pl = (C2 *)smem_raw;
    const int ls = Na + 1;
    R *ta = (R *)(pl + (size_t)Nb * ls);
    R *tb = ta + 2 * Na;
    const int Nh = Na / 2 + 1;
    const size_t plane = vb.x;  // bead * Nc + c
    load_twiddles(ta, twa, Na);
    load_twiddles(tb, twb, Nb);
    const R *src = q + plane * Na * Nb;
    for (int idx = threadIdx.x; idx < Na * Nb; idx += blockDim.x) {
        C2 v;
        v.x = src[idx];
        v.y = (R)0;
        pl[(idx / Na) * ls + idx % Na] = v;
    }
    __syncthreads();
    line_fft<R, NF>(pl, Na, Nb, ls, 1, ta, +1);   // along a, every row
    line_fft<R, NF>(pl, Nb, Nh, 1, ls, tb, +1);   // along b, columns a <= Na/2
    C2 *dst = spec + plane * (size_t)Nb * Nh;
    for (int idx = threadIdx.x; idx < Nb * Nh; idx += blockDim.x) dst[idx] = pl[(idx / Nh) * ls + idx % Nh];
}

template <typename R, int NF>
__global__ void __launch_bounds__(256, PINYB200_PLANE_LB(R, NF)) plane_fwd_kernel(const R *__restrict__ q, typename Cplx<R>::T *__restrict__ spec,
                                                        int Na, int Nb, int Nc, const R *__restrict__ twa,
                                                        const R *__restrict__ twb)
{
    plane_fwd_body<R, NF>(q, spec, Na, Nb, Nc, twa, twb, hw_blk());
}

// Inverse of plane_fwd: half spectrum in, along b, Hermitian completion of
// each row (U(Na-a) = conj U(a) once b and c are back in real space), along
// a, real part out.
template <typename R, int NF>
__device__ __forceinline__ void plane_inv_body(const typename Cplx<R>::T *__restrict__ spec, R *__restrict__ phi, int Na,
                                               int Nb, int Nc, const R *__restrict__ twa, const R *__restrict__ twb,
                                               const VBlk vb)
{
    if (NF > 0) Na = Nb = NF;  // cubic power-of-two grid known at compile time
    (void)Nc;
    typedef typename Cplx<R>::T C2;
    extern __shared__ unsigned char smem_raw[];
    C2 *pl = (C2 *)smem_raw;
    const int ls = Na + 1;
    R *ta = (R *)(pl + (size_t)Nb * ls);
    R *tb = ta + 2 * Na;
    const int Nh = Na / 2 + 1;
    const size_t plane = vb.x;
    load_twiddles(ta, twa, Na);
    load_twiddles(tb, twb, Nb);
    const C2 *src = spec + plane * (size_t)Nb * Nh;
    for (int idx = threadIdx.x; idx < Nb * Nh; idx += blockDim.x) pl[(idx / Nh) * ls + idx % Nh] = src[idx];
    __syncthreads();
    line_fft<R, NF>(pl, Nb, Nh, 1, ls, tb, -1);
    for (int idx = threadIdx.x; idx < Nb * Na; idx += blockDim.x) {
        const int b = idx / Na, a = idx % Na;
        if (a >= Nh) {
            C2 v = pl[b * ls + (Na - a)];
            v.y = -v.y;
            pl[b * ls + a] = v;
        }
    }
    __syncthreads();
    line_fft<R, NF>(pl, Na, Nb, ls, 1, ta, -1);
    R *dst = phi + plane * Na * Nb;
    for (int idx = threadIdx.x; idx < Na * Nb; idx += blockDim.x) dst[idx] = pl[(idx / Na) * ls + idx % Na].x;
}

template <typename R, int NF>
__global__ void __launch_bounds__(256, PINYB200_PLANE_LB(R, NF)) plane_inv_kernel(const typename Cplx<R>::T *__restrict__ spec, R *__restrict__ phi,
                                                        int Na, int Nb, int Nc, const R *__restrict__ twa,
                                                        const R *__restrict__ twb)
{
    plane_inv_body<R, NF>(spec, phi, Na, Nb, Nc, twa, twb, hw_blk());
}

// One (bead, b) slab of the half spectrum: FFT along c, energy and virial
// of the k-sphere terms (ewald3d_pme.c:366-425), multiplication by the
// influence function, inverse FFT along c.  Half-spectrum points with
// 0 < a < Na/2 stand for two full-grid points; E = 1/2 sum_full w |S|^2.
template <typename R, int NF>
__device__ __forceinline__ void conv_c_body(typename Cplx<R>::T *__restrict__ spec, const R *__restrict__ filt, int Na,
                                            int Nb, int Nc, const R *__restrict__ twc, const Cell &cell, double alp,
                                            double *__restrict__ acc, int energy, const VBlk vb)
{
    if (NF > 0) Na = Nb = Nc = NF;  // cubic power-of-two grid known at compile time
    typedef typename Cplx<R>::T C2;
    extern __shared__ unsigned char smem_raw[];
    C2 *sl = (C2 *)smem_raw;
    const int Nh = Na / 2 + 1;
    const int ls = Nh + 1;  // padded line stride: element c of column a at sl[c * ls + a]
    R *tc = (R *)(sl + (size_t)Nc * ls);
    __shared__ double red[7][8];
    const int bead = vb.x / Nb, b = vb.x % Nb;
    load_twiddles(tc, twc, Nc);
    C2 *base = spec + ((size_t)bead * Nc * Nb + b) * Nh;
    const size_t cstride = (size_t)Nb * Nh;
    for (int idx = threadIdx.x; idx < Nc * Nh; idx += blockDim.x) {
        const int c = idx / Nh, a = idx % Nh;
        sl[c * ls + a] = base[c * cstride + a];
    }
    __syncthreads();
    line_fft<R, NF>(sl, Nc, Nh, 1, ls, tc, +1);
    // per-point energy and virial terms in R (FP32 for MIXED), summed in FP64
    double e = 0, pxx = 0, pyy = 0, pzz = 0, pxy = 0, pxz = 0, pyz = 0;
    const R kb = (R)(b <= Nb / 2 ? b : b - Nb);
    const R tpi = (R)(2.0 * M_PI), falp2 = (R)(4.0 * alp * alp);
    R hi[9];
#pragma unroll
    for (int k = 0; k < 9; k++) hi[k] = (R)cell.hi[k];
    for (int idx = threadIdx.x; idx < Nc * Nh; idx += blockDim.x) {
        const int c = idx / Nh, a = idx % Nh;
        const R w = filt[((size_t)c * Nb + b) * Na + a];
        C2 s = sl[c * ls + a];
        if (w != (R)0 && energy) {
            const R ka = (R)a, kc = (R)(c <= Nc / 2 ? c : c - Nc);
            const R xk = tpi * (ka * hi[0] + kb * hi[1] + kc * hi[2]);
            const R yk = tpi * (ka * hi[3] + kb * hi[4] + kc * hi[5]);
            const R zk = tpi * (ka * hi[6] + kb * hi[7] + kc * hi[8]);
            const R g2 = xk * xk + yk * yk + zk * zk;
            const R mult = (a == 0 || 2 * a == Na) ? (R)0.5 : (R)1.0;
            const R sm = mult * (s.x * s.x + s.y * s.y) * w;
            const R prep = (R)-2.0 * ((g2 / falp2) + (R)1.0) / g2 * sm;
            e += (double)sm;
            pxx += (double)(prep * xk * xk);
            pyy += (double)(prep * yk * yk);
            pzz += (double)(prep * zk * zk);
            pxy += (double)(prep * xk * yk);
            pxz += (double)(prep * xk * zk);
            pyz += (double)(prep * yk * zk);
        }
        s.x *= w;
        s.y *= w;
        sl[c * ls + a] = s;
    }
    __syncthreads();
    line_fft<R, NF>(sl, Nc, Nh, 1, ls, tc, -1);
    for (int idx = threadIdx.x; idx < Nc * Nh; idx += blockDim.x) {
        const int c = idx / Nh, a = idx % Nh;
        base[c * cstride + a] = sl[c * ls + a];
    }
    if (!energy) return;
    double v[7] = {e, pxx, pyy, pzz, pxy, pxz, pyz};
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 7; k++) {
        double t = warp_sum(v[k]);
        if (lane == 0) red[k][wid] = t;
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        double t = 0;
        for (int w2 = 0; w2 < (int)(blockDim.x >> 5); w2++) t += red[threadIdx.x][w2];
        const int slot[7] = {S_VRECIP, S_PXX, S_PYY, S_PZZ, S_PXY, S_PXZ, S_PYZ};
        atomicAdd(&acc[(size_t)bead * S_NSLOT + slot[threadIdx.x]], t);
        if (threadIdx.x == 0) {
            // diagonal vnow term of the pressure tensor (ewald3d_pme.c:415-417)
            atomicAdd(&acc[(size_t)bead * S_NSLOT + S_PXX], t);
            atomicAdd(&acc[(size_t)bead * S_NSLOT + S_PYY], t);
            atomicAdd(&acc[(size_t)bead * S_NSLOT + S_PZZ], t);
        }
    }
}

template <typename R, int NF>
__global__ void __launch_bounds__(256, PINYB200_FFT_LB(R, NF)) conv_c_kernel(typename Cplx<R>::T *__restrict__ spec, const R *__restrict__ filt,
                                                     int Na, int Nb, int Nc, const R *__restrict__ twc,
                                                     const __grid_constant__ Cell cell, double alp,
                                                     double *__restrict__ acc, int energy)
{
    conv_c_body<R, NF>(spec, filt, Na, Nb, Nc, twc, cell, alp, acc, energy, hw_blk());
}

// ---------------------------------------------------------------------------
// Influence function on the full grid: preg * bweight for grid points whose
// k (or -k) is on PINY's list, zero elsewhere.
__global__ void filter_kernel(int Na, int Nb, int Nc, const int *__restrict__ kmask, const int *__restrict__ kvec,
                              const double *__restrict__ bw, Cell cell, double alp, double *__restrict__ f64,
                              float *__restrict__ f32)
{
    const size_t G = (size_t)Na * Nb * Nc;
    const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    const int idx = kmask[g];
    double w = 0.0;
    if (idx >= 0) {
        const double tpi = 2.0 * M_PI;
        const double aka = tpi * (double)kvec[3 * idx], akb = tpi * (double)kvec[3 * idx + 1],
                     akc = tpi * (double)kvec[3 * idx + 2];
        const double xk = (aka * cell.hi[0] + akb * cell.hi[1] + akc * cell.hi[2]);
        const double yk = (aka * cell.hi[3] + akb * cell.hi[4] + akc * cell.hi[5]);
        const double zk = (aka * cell.hi[6] + akb * cell.hi[7] + akc * cell.hi[8]);
        const double g2 = xk * xk + yk * yk + zk * zk;
        const double falp2 = 4.0 * alp * alp;
        const double pivol = cell.vol / (4.0 * M_PI);
        w = exp((-g2 / falp2)) / (g2 * pivol) * bw[idx];
    }
    f64[g] = w;
    f32[g] = (float)w;
}

// Shared memory of the plane and slab kernels.
size_t pme_plane_smem(int Na, int Nb, bool fp64)
{
    const size_t cs = fp64 ? 16 : 8, rs = fp64 ? 8 : 4;
    return cs * (size_t)Nb * (Na + 1) + rs * 2 * (size_t)(Na + Nb);
}
size_t pme_slab_smem(int Na, int Nc, bool fp64)
{
    const size_t cs = fp64 ? 16 : 8, rs = fp64 ? 8 : 4;
    return cs * (size_t)Nc * (Na / 2 + 2) + rs * 2 * (size_t)Nc;
}

// The three FFT kernels for grids of compile-time edge NF (0: run time).
template <typename R, int NF>
static cudaError_t launch_fft_t(pinyb200_ctx *c, const PmeArgs &a, const Cell &cell, typename Cplx<R>::T *spec,
                                const R *filt, const R *const *tw, size_t sp, size_t ss, bool energy)
{
    cudaError_t err = cudaSuccess;
    // opt in to more than 48 KB of dynamic shared memory where a plane needs it
    if (sp > 48 * 1024) {
        err = smem_optin((const void *)plane_fwd_kernel<R, NF>, (int)sp);
        if (err == cudaSuccess)
            err = smem_optin((const void *)plane_inv_kernel<R, NF>, (int)sp);
        if (err != cudaSuccess) return err;
    }
    if (ss > 48 * 1024) {
        err = smem_optin((const void *)conv_c_kernel<R, NF>, (int)ss);
        if (err != cudaSuccess) return err;
    }
    plane_fwd_kernel<R, NF><<<a.P * a.Nc, 256, sp, c->stream>>>((const R *)a.grid, spec, a.Na, a.Nb, a.Nc, tw[0],
                                                                tw[1]);
    if ((err = kt_mark(c, "pme_plane_fwd")) != cudaSuccess) return err;
    conv_c_kernel<R, NF><<<a.P * a.Nb, 256, ss, c->stream>>>(spec, filt, a.Na, a.Nb, a.Nc, tw[2], cell, c->alp_ewd,
                                                             c->d_acc, energy ? 1 : 0);
    if ((err = kt_mark(c, "pme_conv_c")) != cudaSuccess) return err;
    plane_inv_kernel<R, NF><<<a.P * a.Nc, 256, sp, c->stream>>>(spec, (R *)a.grid, a.Na, a.Nb, a.Nc, tw[0], tw[1]);
    if ((err = kt_mark(c, "pme_plane_inv")) != cudaSuccess) return err;
    return cudaGetLastError();
}

// Kernel arguments of a context's PME mesh.
static PmeArgs pme_args_of(pinyb200_ctx *c)
{
    const DeviceSystem &s = c->sys;
    PmeArgs a;
    a.natm = s.natm;
    a.P = c->P;
    a.nchrg = s.nchrg;
    a.ichrg = s.ichrg;
    a.charge = s.charge;
    a.posT = c->d_posT;
    a.Na = s.ngrid[0];
    a.Nb = s.ngrid[1];
    a.Nc = s.ngrid[2];
    a.n = s.n_interp;
    a.grid = c->d_grid;
    a.forceP = c->d_forceP;
    a.rhead = (int4 *)c->d_pme_head;
    a.rw = c->d_pme_w;
    return a;
}

// Tile binning arguments of a context's PME mesh for spline order NI and
// tile edge TT.
static TileArgs tile_args_of(pinyb200_ctx *c, int NI, int TT)
{
    TileArgs t;
    t.T = TT;
    // fixed-point scale of the FP32 spread tile: every contribution q M_a M_b
    // M_c (bounded by max |q| times the B-spline's peak cubed) below 2^22
    // after scaling, the range the rounding trick is exact in; at most 2^24
    // (a resolution of 6e-8 against contributions of up to ~0.15)
    {
        double qmax = 0.0;
        for (double q : c->h_charge) qmax = std::max(qmax, std::fabs(q));
        const double bmax = bspline_peak(NI);
        int S = 24;
        while (S > 8 && std::ldexp(qmax * bmax * bmax * bmax, S) >= 0.99 * std::ldexp(1.0, 22)) S--;
        t.qfix = (float)std::ldexp(1.0, S);
        t.qfix_inv = (float)std::ldexp(1.0, -S);
    }
    t.nta = c->pme_nt[0];
    t.ntb = c->pme_nt[1];
    t.ntc = c->pme_nt[2];
    t.ntile = c->pme_ntile;
    t.cap = c->pme_cap;
    t.cnt = c->d_pme_cnt;
    t.bin = c->d_pme_bin;
    t.ovf = c->d_pme_ovf;
    return t;
}

template <typename R, int NI, int TT>
static cudaError_t launch_pme_t(pinyb200_ctx *c, const Cell &cell, bool energy)
{
    typedef typename Cplx<R>::T C2;
    const PmeArgs a = pme_args_of(c);
    const size_t G = (size_t)a.Na * a.Nb * a.Nc;
    const bool f64 = sizeof(R) == 8;
    cudaError_t err = cudaMemsetAsync(c->d_grid, 0, sizeof(R) * G * c->P, c->stream);
    if (err != cudaSuccess) return err;
    if ((err = kt_mark(c, "pme_grid_clear (memset)")) != cudaSuccess) return err;
    const TileArgs t = tile_args_of(c, NI, TT);
    err = cudaMemsetAsync(t.cnt, 0, ((size_t)a.P * t.ntile + 1) * sizeof(int), c->stream);
    if (err != cudaSuccess) return err;
    const long long nt = (long long)a.nchrg * a.P;
    const int threads = 256;
    // the parameter adjoint reads the full weight records of the forward pass
    const bool full = c->pme_full_records;
    if (full) pme_bin_kernel<R, NI><<<(unsigned)((nt + threads - 1) / threads), threads, 0, c->stream>>>(a, cell, t);
    else pme_bin_compact_kernel<R, NI><<<(unsigned)((nt + threads - 1) / threads), threads, 0, c->stream>>>(a, cell, t);
    if ((err = kt_mark(c, "pme_bin")) != cudaSuccess) return err;
    const size_t st = (size_t)TileGeom<NI, TT>::NPT * sizeof(R), ss_spread = spread_smem<R, NI, TT>();
    if (ss_spread > 48 * 1024 - sizeof(PolyTab<R, NI>)) {
        err = smem_optin((const void *)spread_tile_kernel<R, NI, TT>, (int)ss_spread);
        if (err == cudaSuccess) err = smem_optin((const void *)spread_tile_c_kernel<R, NI, TT>, (int)ss_spread);
        if (err != cudaSuccess) return err;
    }
    if (st > 48 * 1024 - sizeof(PolyTab<R, NI>)) {
        err = smem_optin((const void *)gather_tile_kernel<R, NI, TT>, (int)st);
        if (err == cudaSuccess) err = smem_optin((const void *)gather_tile_c_kernel<R, NI, TT>, (int)st);
        if (err != cudaSuccess) return err;
    }
    const dim3 tgrid((unsigned)t.ntile, (unsigned)a.P);
    if (full) spread_tile_kernel<R, NI, TT><<<tgrid, 256, ss_spread, c->stream>>>(a, t);
    else spread_tile_c_kernel<R, NI, TT><<<tgrid, 256, ss_spread, c->stream>>>(a, t);
    if ((err = kt_mark(c, "pme_spread")) != cudaSuccess) return err;
    const R *twbase = (const R *)(f64 ? (const void *)c->d_twiddle64 : (const void *)c->d_twiddle32);
    const R *tw[3] = {twbase, twbase + 2 * 256, twbase + 4 * 256};
    const size_t sp = pme_plane_smem(a.Na, a.Nb, f64), ss = pme_slab_smem(a.Na, a.Nc, f64);
    C2 *spec = (C2 *)c->d_spec;
    const R *filt = f64 ? (const R *)c->d_filter : (const R *)((const double *)c->d_filter + G);
    const bool cube = a.Na == a.Nb && a.Na == a.Nc;
    switch (cube ? a.Na : 0) {
    case 16: err = launch_fft_t<R, 16>(c, a, cell, spec, filt, tw, sp, ss, energy); break;
    case 32: err = launch_fft_t<R, 32>(c, a, cell, spec, filt, tw, sp, ss, energy); break;
    case 64: err = launch_fft_t<R, 64>(c, a, cell, spec, filt, tw, sp, ss, energy); break;
    case 128: err = launch_fft_t<R, 128>(c, a, cell, spec, filt, tw, sp, ss, energy); break;
    default: err = launch_fft_t<R, 0>(c, a, cell, spec, filt, tw, sp, ss, energy); break;
    }
    if (err != cudaSuccess) return err;
    if (full) gather_tile_kernel<R, NI, TT><<<tgrid, 256, st, c->stream>>>(a, cell, t);
    else gather_tile_c_kernel<R, NI, TT><<<tgrid, 256, st, c->stream>>>(a, cell, t);
    if ((err = kt_mark(c, "pme_gather")) != cudaSuccess) return err;
    return cudaGetLastError();
}

template <typename R, int TT>
static cudaError_t launch_pme_rt(pinyb200_ctx *c, const Cell &cell, bool energy)
{
    switch (c->sys.n_interp) {
    case 4: return launch_pme_t<R, 4, TT>(c, cell, energy);
    case 5: return launch_pme_t<R, 5, TT>(c, cell, energy);
    case 6: return launch_pme_t<R, 6, TT>(c, cell, energy);
    case 7: return launch_pme_t<R, 7, TT>(c, cell, energy);
    case 8: return launch_pme_t<R, 8, TT>(c, cell, energy);
    case 10: return launch_pme_t<R, 10, TT>(c, cell, energy);
    default: return cudaErrorInvalidValue;
    }
}

template <typename R>
static cudaError_t launch_pme_r(pinyb200_ctx *c, const Cell &cell, bool energy)
{
    return c->pme_tile == 8 ? launch_pme_rt<R, 8>(c, cell, energy) : launch_pme_rt<R, 16>(c, cell, energy);
}

cudaError_t launch_pme_force_add(pinyb200_ctx *c)
{
    if (c->sys.nchrg == 0 || c->sys.nktot == 0) return cudaSuccess;
    const long long n = (long long)c->sys.nchrg * 3 * c->P;
    pme_force_add_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->sys.nchrg, c->P, c->sys.ichrg,
                                                                            c->d_forceP, c->d_forceT);
    return cudaGetLastError();
}

cudaError_t launch_pme_force_add_scaled(pinyb200_ctx *c, double w, double *target)
{
    if (c->sys.nchrg == 0 || c->sys.nktot == 0) return cudaSuccess;
    const long long n = (long long)c->sys.nchrg * 3 * c->P;
    pme_force_add_scaled_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->sys.nchrg, c->P,
                                                                                   c->sys.ichrg, c->d_forceP, w,
                                                                                   target);
    return cudaGetLastError();
}

cudaError_t launch_pme(pinyb200_ctx *c, const Cell &cell, bool energy)
{
    if (c->sys.nchrg == 0 || c->sys.nktot == 0) return cudaSuccess;
    const size_t G = (size_t)c->sys.ngrid[0] * c->sys.ngrid[1] * c->sys.ngrid[2];
    bool same = c->filter_ok;
    for (int i = 0; i < 9 && same; i++) same = c->filter_h[i] == cell.h[i];
    if (!same) {
        filter_kernel<<<(unsigned)((G + 255) / 256), 256, 0, c->stream>>>(
            c->sys.ngrid[0], c->sys.ngrid[1], c->sys.ngrid[2], c->sys.kmask, c->sys.kvec, c->sys.bweight, cell,
            c->alp_ewd, (double *)c->d_filter, (float *)((double *)c->d_filter + G));
        for (int i = 0; i < 9; i++) c->filter_h[i] = cell.h[i];
        c->filter_ok = true;
    }
    if (c->precision == PINYB200_FP64) return launch_pme_r<double>(c, cell, energy);
    return launch_pme_r<float>(c, cell, energy);
}

// ---------------------------------------------------------------------------
// Many boxes per launch (the batched evaluation): every forward PME kernel of
// the compact FP32 path over a table of boxes, one persistent launch per
// group of boxes that share the kernel's compile-time shape.

struct PmeBox {
    PmeArgs a;
    TileArgs t;
    Cell cell;
};

// Resident blocks per SM of the multi-box plane FFT passes and gather (their
// run-time argument tables cost registers over the one-box kernels'): 3 and
// 4 (80 and 64 registers, 16-36 bytes of spills) take the 64-box C4 step
// from 5.56 to 5.36 ms against 2 and 1.
#ifndef PINYB200_PLANE_BATCH_BLOCKS
#define PINYB200_PLANE_BATCH_BLOCKS 3
#endif
#ifndef PINYB200_GATHER_BATCH_BLOCKS
#define PINYB200_GATHER_BATCH_BLOCKS 4
#endif

struct FftBox {
    const void *q;      // real grid (forward input, inverse output)
    void *spec;         // half spectrum
    const void *filt;   // influence function (FP32)
    const void *tw[3];  // twiddles per axis
    int Na, Nb, Nc;
    Cell cell;
    double alp;
    double *acc;
    int energy;
};

struct AddBox {
    int nchrg, P;
    const int *ichrg;
    const double *fP;
    double *fT;
};

template <typename R, int NI>
__global__ void __launch_bounds__(256) pme_bin_batch_kernel(const __grid_constant__ BoxTab<PmeBox> t)
{
    PINYB200_BOX_LOOP(t, i, vb, (pme_bin_compact_body<R, NI>(t.arg[i].a, t.arg[i].cell, t.arg[i].t, vb)));
}

template <typename R, int NI, int TT>
__global__ void __launch_bounds__(256) spread_batch_kernel(const __grid_constant__ BoxTab<PmeBox> t)
{
    PINYB200_BOX_LOOP(t, i, vb, (spread_tile_c_body<R, NI, TT>(t.arg[i].a, t.arg[i].t, vb)));
}

template <typename R, int NI, int TT>
__global__ void __launch_bounds__(256, NI <= 8 ? PINYB200_GATHER_BATCH_BLOCKS : 1)
    gather_batch_kernel(const __grid_constant__ BoxTab<PmeBox> t)
{
    PINYB200_BOX_LOOP(t, i, vb, (gather_tile_c_body<R, NI, TT>(t.arg[i].a, t.arg[i].cell, t.arg[i].t, vb)));
}

template <typename R, int NF>
__global__ void __launch_bounds__(256, NF > 0 ? PINYB200_PLANE_BATCH_BLOCKS : 1)
    plane_fwd_batch_kernel(const __grid_constant__ BoxTab<FftBox> t)
{
    typedef typename Cplx<R>::T C2;
    PINYB200_BOX_LOOP(t, i, vb,
                      (plane_fwd_body<R, NF>((const R *)t.arg[i].q, (C2 *)t.arg[i].spec, t.arg[i].Na, t.arg[i].Nb,
                                             t.arg[i].Nc, (const R *)t.arg[i].tw[0], (const R *)t.arg[i].tw[1], vb)));
}

// (the multi-box slab pass: at 3, 80 registers spill 236 bytes and the C4
// step takes 5.50 against 5.37 ms)
#ifndef PINYB200_CONV_BATCH_BLOCKS
#define PINYB200_CONV_BATCH_BLOCKS 2
#endif
template <typename R, int NF>
__global__ void __launch_bounds__(256, NF > 0 ? PINYB200_CONV_BATCH_BLOCKS : 1)
    conv_c_batch_kernel(const __grid_constant__ BoxTab<FftBox> t)
{
    typedef typename Cplx<R>::T C2;
    PINYB200_BOX_LOOP(t, i, vb,
                      (conv_c_body<R, NF>((C2 *)t.arg[i].spec, (const R *)t.arg[i].filt, t.arg[i].Na, t.arg[i].Nb,
                                          t.arg[i].Nc, (const R *)t.arg[i].tw[2], t.arg[i].cell, t.arg[i].alp,
                                          t.arg[i].acc, t.arg[i].energy, vb)));
}

template <typename R, int NF>
__global__ void __launch_bounds__(256, NF > 0 ? PINYB200_PLANE_BATCH_BLOCKS : 1)
    plane_inv_batch_kernel(const __grid_constant__ BoxTab<FftBox> t)
{
    typedef typename Cplx<R>::T C2;
    PINYB200_BOX_LOOP(t, i, vb,
                      (plane_inv_body<R, NF>((const C2 *)t.arg[i].spec, (R *)t.arg[i].q, t.arg[i].Na, t.arg[i].Nb,
                                             t.arg[i].Nc, (const R *)t.arg[i].tw[0], (const R *)t.arg[i].tw[1], vb)));
}

__global__ void __launch_bounds__(256) pme_force_add_batch_kernel(const __grid_constant__ BoxTab<AddBox> t)
{
    PINYB200_BOX_LOOP(t, i, vb,
                      (pme_force_add_body(t.arg[i].nchrg, t.arg[i].P, t.arg[i].ichrg, t.arg[i].fP, t.arg[i].fT, vb)));
}

// stage 0 bin, 1 spread, 2 gather for the boxes of one (order, tile edge) group
template <int NI, int TT>
static cudaError_t pme_batch_tiles(const std::vector<PmeBox> &bx, const std::vector<int> &P, int sm_count,
                                   cudaStream_t st, int stage)
{
    typedef float R;
    BoxTabBuilder<PmeBox> tb;
    for (size_t i = 0; i < bx.size(); i++) {
        const double work = (double)bx[i].a.nchrg * P[i];
        if (stage == 0) tb.add(bx[i], (int)(((long long)bx[i].a.nchrg * P[i] + 255) / 256), 1, work);
        else tb.add(bx[i], bx[i].t.ntile, P[i], work);
    }
    if (stage == 0)
        return launch_tables(tb, (const void *)pme_bin_batch_kernel<R, NI>, 256, 0, sm_count,
                             [&](const BoxTab<PmeBox> &t, int g) { pme_bin_batch_kernel<R, NI><<<g, 256, 0, st>>>(t); });
    if (stage == 1) {
        const size_t ss = spread_smem<R, NI, TT>();
        return launch_tables(tb, (const void *)spread_batch_kernel<R, NI, TT>, 256, ss, sm_count,
                             [&](const BoxTab<PmeBox> &t, int g) { spread_batch_kernel<R, NI, TT><<<g, 256, ss, st>>>(t); });
    }
    const size_t sg = (size_t)TileGeom<NI, TT>::NPT * sizeof(R);
    return launch_tables(tb, (const void *)gather_batch_kernel<R, NI, TT>, 256, sg, sm_count,
                         [&](const BoxTab<PmeBox> &t, int g) { gather_batch_kernel<R, NI, TT><<<g, 256, sg, st>>>(t); });
}

template <int TT>
static cudaError_t pme_batch_tiles_n(int NI, const std::vector<PmeBox> &bx, const std::vector<int> &P, int sm_count,
                                     cudaStream_t st, int stage)
{
    switch (NI) {
    case 4: return pme_batch_tiles<4, TT>(bx, P, sm_count, st, stage);
    case 5: return pme_batch_tiles<5, TT>(bx, P, sm_count, st, stage);
    case 6: return pme_batch_tiles<6, TT>(bx, P, sm_count, st, stage);
    case 7: return pme_batch_tiles<7, TT>(bx, P, sm_count, st, stage);
    case 8: return pme_batch_tiles<8, TT>(bx, P, sm_count, st, stage);
    case 10: return pme_batch_tiles<10, TT>(bx, P, sm_count, st, stage);
    default: return cudaErrorInvalidValue;
    }
}

// stage 0 forward plane FFT, 1 c-axis FFT with the convolution, 2 inverse
// plane FFT for the boxes of one mesh
template <int NF>
static cudaError_t pme_batch_fft(const std::vector<FftBox> &bx, const std::vector<int> &P, int sm_count,
                                 cudaStream_t st, int stage)
{
    typedef float R;
    size_t sp = 0, ss = 0;
    BoxTabBuilder<FftBox> tb;
    for (size_t i = 0; i < bx.size(); i++) {
        sp = std::max(sp, pme_plane_smem(bx[i].Na, bx[i].Nb, false));
        ss = std::max(ss, pme_slab_smem(bx[i].Na, bx[i].Nc, false));
        const double work = (double)bx[i].Na * bx[i].Nb * bx[i].Nc * P[i];
        tb.add(bx[i], P[i] * (stage == 1 ? bx[i].Nb : bx[i].Nc), 1, work);
    }
    if (stage == 0)
        return launch_tables(tb, (const void *)plane_fwd_batch_kernel<R, NF>, 256, sp, sm_count,
                             [&](const BoxTab<FftBox> &t, int g) { plane_fwd_batch_kernel<R, NF><<<g, 256, sp, st>>>(t); });
    if (stage == 1)
        return launch_tables(tb, (const void *)conv_c_batch_kernel<R, NF>, 256, ss, sm_count,
                             [&](const BoxTab<FftBox> &t, int g) { conv_c_batch_kernel<R, NF><<<g, 256, ss, st>>>(t); });
    return launch_tables(tb, (const void *)plane_inv_batch_kernel<R, NF>, 256, sp, sm_count,
                         [&](const BoxTab<FftBox> &t, int g) { plane_inv_batch_kernel<R, NF><<<g, 256, sp, st>>>(t); });
}

static cudaError_t pme_batch_tiles_group(const std::pair<int, int> &key, const std::vector<PmeBox> &bx,
                                         const std::vector<int> &P, int sm_count, cudaStream_t st, int stage)
{
    return key.second == 8 ? pme_batch_tiles_n<8>(key.first, bx, P, sm_count, st, stage)
                           : pme_batch_tiles_n<16>(key.first, bx, P, sm_count, st, stage);
}

// Forward PME of many MIXED contexts on stream st, as launch_pme does for
// one: grids and bin counters cleared, charges binned, spread, transformed,
// convolved (energies and virials into each context's per-bead sums when
// `energy`), transformed back and gathered into each context's PME forces.
// The contexts' meshes use the compact records (pme_full_records off).
cudaError_t launch_pme_batch(const std::vector<pinyb200_ctx *> &box, const std::vector<Cell> &cells, bool energy,
                             int sm_count, cudaStream_t st)
{
    // groups: tiles by (order, tile edge), FFTs by mesh
    std::map<std::pair<int, int>, std::pair<std::vector<PmeBox>, std::vector<int>>> tiles;
    std::map<std::tuple<int, int, int>, std::pair<std::vector<FftBox>, std::vector<int>>> ffts;
    std::vector<std::pair<void *, size_t>> zero;
    for (size_t i = 0; i < box.size(); i++) {
        pinyb200_ctx *c = box[i];
        if (c->sys.nchrg == 0 || c->sys.nktot == 0) continue;
        if (c->precision != PINYB200_MIXED || c->pme_full_records) return cudaErrorInvalidValue;
        const Cell &cell = cells[i];
        const size_t G = (size_t)c->sys.ngrid[0] * c->sys.ngrid[1] * c->sys.ngrid[2];
        bool same = c->filter_ok;
        for (int k = 0; k < 9 && same; k++) same = c->filter_h[k] == cell.h[k];
        if (!same) {
            // the influence function of this cell (normally built by the plain run before capture)
            filter_kernel<<<(unsigned)((G + 255) / 256), 256, 0, st>>>(
                c->sys.ngrid[0], c->sys.ngrid[1], c->sys.ngrid[2], c->sys.kmask, c->sys.kvec, c->sys.bweight, cell,
                c->alp_ewd, (double *)c->d_filter, (float *)((double *)c->d_filter + G));
            for (int k = 0; k < 9; k++) c->filter_h[k] = cell.h[k];
            c->filter_ok = true;
        }
        PmeBox pb;
        pb.a = pme_args_of(c);
        pb.t = tile_args_of(c, c->sys.n_interp, c->pme_tile);
        pb.cell = cell;
        auto &tg = tiles[std::make_pair(c->sys.n_interp, c->pme_tile)];
        tg.first.push_back(pb);
        tg.second.push_back(c->P);
        FftBox fb;
        fb.q = c->d_grid;
        fb.spec = c->d_spec;
        fb.filt = (const void *)((const double *)c->d_filter + G);
        fb.tw[0] = c->d_twiddle32;
        fb.tw[1] = c->d_twiddle32 + 2 * 256;
        fb.tw[2] = c->d_twiddle32 + 4 * 256;
        fb.Na = c->sys.ngrid[0];
        fb.Nb = c->sys.ngrid[1];
        fb.Nc = c->sys.ngrid[2];
        fb.cell = cell;
        fb.alp = c->alp_ewd;
        fb.acc = c->d_acc;
        fb.energy = energy ? 1 : 0;
        auto &fg = ffts[std::make_tuple(fb.Na, fb.Nb, fb.Nc)];
        fg.first.push_back(fb);
        fg.second.push_back(c->P);
        zero.emplace_back(c->d_grid, sizeof(float) * G * c->P);
        zero.emplace_back(c->d_pme_cnt, ((size_t)c->P * c->pme_ntile + 1) * sizeof(int));
    }
    cudaError_t err = launch_zero_batch(zero, sm_count, st);
    for (int stage = 0; stage < 2 && err == cudaSuccess; stage++)
        for (auto &kv : tiles) {
            err = pme_batch_tiles_group(kv.first, kv.second.first, kv.second.second, sm_count, st, stage);
            if (err != cudaSuccess) break;
        }
    for (int stage = 0; stage < 3 && err == cudaSuccess; stage++)
        for (auto &kv : ffts) {
            const int Na = std::get<0>(kv.first), Nb = std::get<1>(kv.first), Nc = std::get<2>(kv.first);
            switch (Na == Nb && Na == Nc ? Na : 0) {
            case 16: err = pme_batch_fft<16>(kv.second.first, kv.second.second, sm_count, st, stage); break;
            case 32: err = pme_batch_fft<32>(kv.second.first, kv.second.second, sm_count, st, stage); break;
            case 64: err = pme_batch_fft<64>(kv.second.first, kv.second.second, sm_count, st, stage); break;
            case 128: err = pme_batch_fft<128>(kv.second.first, kv.second.second, sm_count, st, stage); break;
            default: err = pme_batch_fft<0>(kv.second.first, kv.second.second, sm_count, st, stage); break;
            }
            if (err != cudaSuccess) break;
        }
    for (auto &kv : tiles) {
        if (err != cudaSuccess) break;
        err = pme_batch_tiles_group(kv.first, kv.second.first, kv.second.second, sm_count, st, 2);
    }
    return err;
}

// PME forces of many contexts added to their site forces.
cudaError_t launch_pme_force_add_batch(const std::vector<pinyb200_ctx *> &box, int sm_count, cudaStream_t st)
{
    BoxTabBuilder<AddBox> tb;
    for (pinyb200_ctx *c : box) {
        if (c->sys.nchrg == 0 || c->sys.nktot == 0) continue;
        const long long n = (long long)c->sys.nchrg * 3 * c->P;
        tb.add(AddBox{c->sys.nchrg, c->P, c->sys.ichrg, c->d_forceP, c->d_forceT}, (int)((n + 255) / 256), 1,
               (double)n);
    }
    return launch_tables(tb, (const void *)pme_force_add_batch_kernel, 256, 0, sm_count,
                         [&](const BoxTab<AddBox> &t, int g) { pme_force_add_batch_kernel<<<g, 256, 0, st>>>(t); });
}

}  // namespace pinyb200

namespace pinyb200 {

// ---------------------------------------------------------------------------
// Adjoint of the reciprocal-space term (parameter gradients).
//
// With u the adjoint of the raw site forces, Q_u(g) = sum_s q_s u_s . grad
// M_s(g) is spread, convolved with the same influence function as the charge
// grid (chi = theta * Q_u), and gathered; with phi the forward potential:
//   charge tangent dq:   dE += sum_s dq_s phi_s
//                        dF += -sum_s dq_s (u_s . grad phi_s + chi_s)
//   ghost position w:    dF += -sum_s q_s (w_s . grad chi_s + u_s^T (grad grad phi)_s w_s)
// (symmetry of the influence function moves the convolution onto Q_u).

// Second-derivative weights of the order-NI B-spline at offset f, PINY's
// index j = 1..NI: d2[j] = m[j] - 2 m[j-1] + m[j-2] with m of order NI-2.
template <typename R, int NI>
__device__ __forceinline__ void bspline_d2(R f, R *d2)
{
    R u[NI + 1], m[NI + 1];
#pragma unroll
    for (int j = 1; j <= NI; j++) u[j] = f + (R)(j - 1);
    m[0] = (R)0;
    m[1] = (R)1 - fabs(u[1] - (R)1);
    m[2] = (R)1 - fabs(u[2] - (R)1);
#pragma unroll
    for (int j = 3; j <= NI; j++) m[j] = (R)0;
#pragma unroll
    for (int nn = 3; nn <= NI - 2; nn++) {
        const R rn = (R)nn, rn1 = (R)1 / (R)(nn - 1);
#pragma unroll
        for (int j = nn; j >= 2; j--) m[j] = (u[j] * m[j] + (rn - u[j]) * m[j - 1]) * rn1;
        m[1] = u[1] * m[1] * rn1;
    }
#pragma unroll
    for (int j = 1; j <= NI; j++) d2[j] = m[j] - (R)2 * (j >= 2 ? m[j - 1] : (R)0) + (j >= 3 ? m[j - 2] : (R)0);
}

// u (or w) in scaled-grid units: t_d = N_d sum_alpha hi[d + 3 alpha] v_alpha.
__device__ __forceinline__ void scaled_vec(const PmeArgs &a, const Cell &cell, double vx, double vy, double vz,
                                           double *t)
{
    const int N[3] = {a.Na, a.Nb, a.Nc};
#pragma unroll
    for (int d = 0; d < 3; d++) t[d] = N[d] * (cell.hi[d] * vx + cell.hi[d + 3] * vy + cell.hi[d + 6] * vz);
}

// Q_u: one warp per record, lanes 8 a points x 4 b rows, FP32/FP64 atomics.
template <typename R, int NI>
__global__ void __launch_bounds__(256) pme_dipole_spread_kernel(PmeArgs a, Cell cell, const double *__restrict__ uT,
                                                                R *__restrict__ grid2)
{
    typedef RecGeom<NI> RG;
    const int lane = threadIdx.x & 31;
    const int ta = lane & 7, tq = lane >> 3;
    const long long nrec = (long long)a.nchrg * a.P;
    const size_t G = (size_t)a.Na * a.Nb * a.Nc;
    for (long long idx = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; idx < nrec;
         idx += ((long long)gridDim.x * blockDim.x) >> 5) {
        const int b = (int)(idx % a.P);
        const int4 h = a.rhead[idx];
        const int at = h.x;
        const double ux = uT[(3 * (size_t)at + 0) * a.P + b], uy = uT[(3 * (size_t)at + 1) * a.P + b],
                     uz = uT[(3 * (size_t)at + 2) * a.P + b];
        if (ux == 0.0 && uy == 0.0 && uz == 0.0) continue;
        double ut[3];
        scaled_vec(a, cell, ux, uy, uz, ut);
        const R q = (R)a.charge[at];
        const R *w = (const R *)a.rw + (size_t)idx * RG::NW;
        R *g = grid2 + (size_t)b * G;
        for (int sa = 0; sa < NI; sa += 8) {
            const int t_a = ta + sa;
            if (t_a >= NI) break;
            const R ma = w[t_a], da = w[3 * RG::NIP + t_a];
            const int ga = wrapi(h.y + t_a, a.Na);
            for (int tb = tq; tb < NI; tb += 4) {
                const R mb = w[RG::NIP + tb], db = w[4 * RG::NIP + tb];
                const int gb = wrapi(h.z + tb, a.Nb);
                const R cab = q * ((R)ut[0] * da * mb + (R)ut[1] * ma * db), cc = q * (R)ut[2] * ma * mb;
                for (int tc = 0; tc < NI; tc++) {
                    const R val = cab * w[2 * RG::NIP + tc] + cc * w[5 * RG::NIP + tc];
                    atomicAdd(g + ((size_t)wrapi(h.w + tc, a.Nc) * a.Nb + gb) * a.Na + ga, val);
                }
            }
        }
    }
}

// Gathers phi, grad phi, chi, grad chi (and grad grad phi at sites with a
// ghost tangent) per record and contracts them with every channel.
template <typename R, int NI>
__global__ void __launch_bounds__(128) pme_adjoint_gather_kernel(PmeArgs a, Cell cell, GradArgs g,
                                                                 const R *__restrict__ phi, const R *__restrict__ chi)
{
    typedef RecGeom<NI> RG;
    __shared__ double sh[2 * PINYB200_MAX_TAN];
    double acc[2 * PINYB200_MAX_TAN];
    for (int k = 0; k < 2 * g.K; k++) acc[k] = 0.0;
    const long long nrec = (long long)a.nchrg * a.P;
    const size_t G = (size_t)a.Na * a.Nb * a.Nc;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < nrec;
         idx += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(idx % a.P);
        const int4 h = a.rhead[idx];
        const int at = h.x;
        R m[6][RG::NIP];
        const R *w = (const R *)a.rw + (size_t)idx * RG::NW;
#pragma unroll
        for (int j = 0; j < 6; j++) load4<RG::NIP>(m[j], w + j * RG::NIP);
        const R *pg = phi + (size_t)b * G, *cg = chi + (size_t)b * G;
        double P0 = 0, Pa = 0, Pb = 0, Pc = 0, X0 = 0, Xa = 0, Xb = 0, Xc = 0;
#pragma unroll 1
        for (int tc = 0; tc < NI; tc++) {
            const int gc = wrapi(h.w + tc, a.Nc);
            R p0 = 0, pa = 0, pb = 0, pc = 0, x0 = 0, xa = 0, xb = 0, xc = 0;
#pragma unroll
            for (int tb = 0; tb < NI; tb++) {
                const size_t row = ((size_t)gc * a.Nb + wrapi(h.z + tb, a.Nb)) * a.Na;
                R sp = 0, sdp = 0, sx = 0, sdx = 0;
#pragma unroll
                for (int t_a = 0; t_a < NI; t_a++) {
                    const int ga = wrapi(h.y + t_a, a.Na);
                    const R pv = pg[row + ga], xv = cg[row + ga];
                    sp += m[0][t_a] * pv;
                    sdp += m[3][t_a] * pv;
                    sx += m[0][t_a] * xv;
                    sdx += m[3][t_a] * xv;
                }
                p0 += m[1][tb] * sp;
                pa += m[1][tb] * sdp;
                pb += m[4][tb] * sp;
                x0 += m[1][tb] * sx;
                xa += m[1][tb] * sdx;
                xb += m[4][tb] * sx;
                (void)pc;
                (void)xc;
            }
            P0 += (double)(m[2][tc] * p0);
            Pa += (double)(m[2][tc] * pa);
            Pb += (double)(m[2][tc] * pb);
            Pc += (double)(m[5][tc] * p0);
            X0 += (double)(m[2][tc] * x0);
            Xa += (double)(m[2][tc] * xa);
            Xb += (double)(m[2][tc] * xb);
            Xc += (double)(m[5][tc] * x0);
        }
        const double ux = g.uT[(3 * (size_t)at + 0) * a.P + b], uy = g.uT[(3 * (size_t)at + 1) * a.P + b],
                     uz = g.uT[(3 * (size_t)at + 2) * a.P + b];
        double ut[3];
        scaled_vec(a, cell, ux, uy, uz, ut);
        const double udphi = ut[0] * Pa + ut[1] * Pb + ut[2] * Pc;
        const double q = a.charge[at];
        // the ghost-position tangents of this site, if any
        bool need_h = false;
        for (int k = 0; k < g.K; k++)
            if (g.ch[k].w) {
                const double *wv = g.ch[k].w;
                if (wv[(3 * (size_t)at) * a.P + b] != 0.0 || wv[(3 * (size_t)at + 1) * a.P + b] != 0.0 ||
                    wv[(3 * (size_t)at + 2) * a.P + b] != 0.0)
                    need_h = true;
            }
        double H[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        if (need_h) {
            int la, lb, lc;
            double fa, fb, fc;
            stencil_origin(a, cell, at, b, NI, la, lb, lc, fa, fb, fc);
            R d2[3][NI + 1];
            bspline_d2<R, NI>((R)fa, d2[0]);
            bspline_d2<R, NI>((R)fb, d2[1]);
            bspline_d2<R, NI>((R)fc, d2[2]);
            // grid order: point lo + t carries index NI - t
            double haa = 0, hbb = 0, hcc = 0, hab = 0, hac = 0, hbc = 0;
            for (int tc = 0; tc < NI; tc++) {
                const int gc = wrapi(h.w + tc, a.Nc);
                for (int tb = 0; tb < NI; tb++) {
                    const size_t row = ((size_t)gc * a.Nb + wrapi(h.z + tb, a.Nb)) * a.Na;
                    for (int t_a = 0; t_a < NI; t_a++) {
                        const double pv = (double)pg[row + wrapi(h.y + t_a, a.Na)];
                        const double ma = m[0][t_a], mb = m[1][tb], mc = m[2][tc];
                        const double da = m[3][t_a], db = m[4][tb], dc = m[5][tc];
                        haa += (double)d2[0][NI - t_a] * mb * mc * pv;
                        hbb += ma * (double)d2[1][NI - tb] * mc * pv;
                        hcc += ma * mb * (double)d2[2][NI - tc] * pv;
                        hab += da * db * mc * pv;
                        hac += da * mb * dc * pv;
                        hbc += ma * db * dc * pv;
                    }
                }
            }
            H[0][0] = haa;
            H[1][1] = hbb;
            H[2][2] = hcc;
            H[0][1] = H[1][0] = hab;
            H[0][2] = H[2][0] = hac;
            H[1][2] = H[2][1] = hbc;
        }
        for (int k = 0; k < g.K; k++) {
            const GradChan &ch = g.ch[k];
            if (ch.dq) {
                const double dq = ch.dq[at];
                if (dq != 0.0) {
                    acc[2 * k] += dq * P0 / (double)a.P;
                    acc[2 * k + 1] += -dq * (udphi + X0);
                }
            }
            if (ch.w && need_h) {
                const double wx = ch.w[(3 * (size_t)at) * a.P + b], wy = ch.w[(3 * (size_t)at + 1) * a.P + b],
                             wz = ch.w[(3 * (size_t)at + 2) * a.P + b];
                double wt[3];
                scaled_vec(a, cell, wx, wy, wz, wt);
                double uhw = 0;
                for (int d = 0; d < 3; d++)
                    for (int e = 0; e < 3; e++) uhw += ut[d] * H[d][e] * wt[e];
                acc[2 * k + 1] += -q * (wt[0] * Xa + wt[1] * Xb + wt[2] * Xc + uhw);
            }
        }
    }
    // block flush
    for (int i = threadIdx.x; i < 2 * g.K; i += blockDim.x) sh[i] = 0.0;
    __syncthreads();
    for (int i = 0; i < 2 * g.K; i++)
        if (acc[i] != 0.0) atomicAdd(&sh[i], acc[i]);
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * g.K; i += blockDim.x)
        if (sh[i] != 0.0) atomicAdd(&g.gacc[i], sh[i]);
}

template <typename R, int NI>
static cudaError_t launch_pme_adjoint_t(pinyb200_ctx *c, const Cell &cell, const GradArgs &g)
{
    typedef typename Cplx<R>::T C2;
    const DeviceSystem &s = c->sys;
    PmeArgs a;
    a.natm = s.natm;
    a.P = c->P;
    a.nchrg = s.nchrg;
    a.ichrg = s.ichrg;
    a.charge = s.charge;
    a.posT = c->d_posT;
    a.Na = s.ngrid[0];
    a.Nb = s.ngrid[1];
    a.Nc = s.ngrid[2];
    a.n = s.n_interp;
    a.grid = c->grad.d_grid2;
    a.forceP = c->d_forceP;
    a.rhead = (int4 *)c->d_pme_head;
    a.rw = c->d_pme_w;
    const size_t G = (size_t)a.Na * a.Nb * a.Nc;
    const bool f64 = sizeof(R) == 8;
    cudaError_t err = cudaMemsetAsync(c->grad.d_grid2, 0, sizeof(R) * G * c->P, c->stream);
    if (err != cudaSuccess) return err;
    const long long nrec = (long long)a.nchrg * a.P;
    long long blocks = (nrec * 32 + 255) / 256;
    if (blocks > (long long)c->sm_count * 16) blocks = (long long)c->sm_count * 16;
    pme_dipole_spread_kernel<R, NI><<<(unsigned)blocks, 256, 0, c->stream>>>(a, cell, g.uT, (R *)c->grad.d_grid2);
    const R *twbase = (const R *)(f64 ? (const void *)c->d_twiddle64 : (const void *)c->d_twiddle32);
    const R *tw[3] = {twbase, twbase + 2 * 256, twbase + 4 * 256};
    const size_t sp = pme_plane_smem(a.Na, a.Nb, f64), ss = pme_slab_smem(a.Na, a.Nc, f64);
    C2 *spec = (C2 *)c->d_spec;
    const R *filt = f64 ? (const R *)c->d_filter : (const R *)((const double *)c->d_filter + G);
    const bool cube = a.Na == a.Nb && a.Na == a.Nc;
    switch (cube ? a.Na : 0) {
    case 16: err = launch_fft_t<R, 16>(c, a, cell, spec, filt, tw, sp, ss, false); break;
    case 32: err = launch_fft_t<R, 32>(c, a, cell, spec, filt, tw, sp, ss, false); break;
    case 64: err = launch_fft_t<R, 64>(c, a, cell, spec, filt, tw, sp, ss, false); break;
    case 128: err = launch_fft_t<R, 128>(c, a, cell, spec, filt, tw, sp, ss, false); break;
    default: err = launch_fft_t<R, 0>(c, a, cell, spec, filt, tw, sp, ss, false); break;
    }
    if (err != cudaSuccess) return err;
    long long gb = (nrec + 127) / 128;
    if (gb > (long long)c->sm_count * 8) gb = (long long)c->sm_count * 8;
    pme_adjoint_gather_kernel<R, NI><<<(unsigned)(gb < 1 ? 1 : gb), 128, 0, c->stream>>>(
        a, cell, g, (const R *)c->d_grid, (const R *)c->grad.d_grid2);
    return cudaGetLastError();
}

template <typename R>
static cudaError_t launch_pme_adjoint_r(pinyb200_ctx *c, const Cell &cell, const GradArgs &g)
{
    switch (c->sys.n_interp) {
    case 4: return launch_pme_adjoint_t<R, 4>(c, cell, g);
    case 5: return launch_pme_adjoint_t<R, 5>(c, cell, g);
    case 6: return launch_pme_adjoint_t<R, 6>(c, cell, g);
    case 7: return launch_pme_adjoint_t<R, 7>(c, cell, g);
    case 8: return launch_pme_adjoint_t<R, 8>(c, cell, g);
    case 10: return launch_pme_adjoint_t<R, 10>(c, cell, g);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_pme_adjoint(pinyb200_ctx *c, const Cell &cell, const GradArgs &g)
{
    if (c->sys.nchrg == 0 || c->sys.nktot == 0 || !c->grad.d_grid2) return cudaSuccess;
    if (c->precision == PINYB200_FP64) return launch_pme_adjoint_r<double>(c, cell, g);
    return launch_pme_adjoint_r<float>(c, cell, g);
}

}  // namespace pinyb200
