// Smooth PME for all beads: charge spreading, batched 3D FFT, k-sphere
// convolution with energy and virial, force gather.
//
// Restates ewald3d_recip_pme_none (src/energy/inter/recip3d/ewald3d_pme.c:
// 95-600): scaled coordinates wrapped to (0,1] (:231-256), order-n cardinal
// B-splines by PINY's recursion and their derivatives from the order n-1
// splines (:301-338, :512-532), grid points ia - (j-2) wrapped (:274-300),
// the half-space spherical k list with preg = exp(-g^2/4a^2)/(g^2 V/4pi) and
// the B-spline weights (:366-425), and the gather F = -q sum grad(M) phi
// (:534-559).  PINY fills a complex grid and runs unnormalised complex FFTs
// (para_fft_gen3d_bck_to_g / _fwd_to_r); the device does the same per bead.
// Filtering with a symmetric kernel over the full grid equals PINY's
// half-list convolution plus Hermitian fill (pme_sngl_pack_coef,
// fft_package.c:458-503), and half the full-grid sum is PINY's energy.
#include "common.cuh"

namespace pinyb200 {

struct PmeArgs {
    int natm, P, nchrg;
    const int *ichrg;
    const double *charge;
    const double *posT;
    int Na, Nb, Nc, n;
    void *grid;
    double *forceT;
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

template <typename R, int NI>
__global__ void __launch_bounds__(256) spread_kernel(PmeArgs a, Cell cell)
{
    typedef typename Cplx<R>::T C2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)a.nchrg * a.P) return;
    const int b = (int)(t % a.P);
    const int ic = (int)(t / a.P);
    const int at = a.ichrg[ic];
    const double x = a.posT[(3 * (size_t)at + 0) * a.P + b];
    const double y = a.posT[(3 * (size_t)at + 1) * a.P + b];
    const double z = a.posT[(3 * (size_t)at + 2) * a.P + b];
    const double q = a.charge[at];
    const double sa = __dadd_rn(__dadd_rn(__dmul_rn(x, cell.hi[0]), __dmul_rn(y, cell.hi[3])), __dmul_rn(z, cell.hi[6]));
    const double sb = __dadd_rn(__dadd_rn(__dmul_rn(x, cell.hi[1]), __dmul_rn(y, cell.hi[4])), __dmul_rn(z, cell.hi[7]));
    const double sc = __dadd_rn(__dadd_rn(__dmul_rn(x, cell.hi[2]), __dmul_rn(y, cell.hi[5])), __dmul_rn(z, cell.hi[8]));
    int ia, ib, icc;
    double fa, fb, fc;
    scaled(sa, a.Na, ia, fa);
    scaled(sb, a.Nb, ib, fb);
    scaled(sc, a.Nc, icc, fc);
    R ma[NI + 1], mb[NI + 1], mc[NI + 1];
    bspline<R, NI, false>((R)fa, ma, nullptr);
    bspline<R, NI, false>((R)fb, mb, nullptr);
    bspline<R, NI, false>((R)fc, mc, nullptr);
    C2 *g = (C2 *)a.grid + (size_t)b * a.Na * a.Nb * a.Nc;
    int ga[NI + 1];
#pragma unroll
    for (int j = 1; j <= NI; j++) {
        int v = ia - (j - 2);
        ga[j] = (v > 0 ? v : a.Na + v) - 1;
    }
    for (int jc = 1; jc <= NI; jc++) {
        int vc = icc - (jc - 2);
        const int gc = (vc > 0 ? vc : a.Nc + vc) - 1;
        const R qc = (R)q * mc[jc];
        for (int jb = 1; jb <= NI; jb++) {
            int vb = ib - (jb - 2);
            const int gb = (vb > 0 ? vb : a.Nb + vb) - 1;
            const R qbc = mb[jb] * qc;
            C2 *rowp = g + ((size_t)gc * a.Nb + gb) * a.Na;
#pragma unroll
            for (int ja = 1; ja <= NI; ja++) atomicAdd(&rowp[ga[ja]].x, ma[ja] * qbc);
        }
    }
}

template <typename R, int NI>
__global__ void __launch_bounds__(256) gather_kernel(PmeArgs a, Cell cell)
{
    typedef typename Cplx<R>::T C2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)a.nchrg * a.P) return;
    const int b = (int)(t % a.P);
    const int ic = (int)(t / a.P);
    const int at = a.ichrg[ic];
    const double x = a.posT[(3 * (size_t)at + 0) * a.P + b];
    const double y = a.posT[(3 * (size_t)at + 1) * a.P + b];
    const double z = a.posT[(3 * (size_t)at + 2) * a.P + b];
    const double q = a.charge[at];
    const double sa = __dadd_rn(__dadd_rn(__dmul_rn(x, cell.hi[0]), __dmul_rn(y, cell.hi[3])), __dmul_rn(z, cell.hi[6]));
    const double sb = __dadd_rn(__dadd_rn(__dmul_rn(x, cell.hi[1]), __dmul_rn(y, cell.hi[4])), __dmul_rn(z, cell.hi[7]));
    const double sc = __dadd_rn(__dadd_rn(__dmul_rn(x, cell.hi[2]), __dmul_rn(y, cell.hi[5])), __dmul_rn(z, cell.hi[8]));
    int ia, ib, icc;
    double fa, fb, fc;
    scaled(sa, a.Na, ia, fa);
    scaled(sb, a.Nb, ib, fb);
    scaled(sc, a.Nc, icc, fc);
    R ma[NI + 1], mb[NI + 1], mc[NI + 1], da[NI + 1], db[NI + 1], dc[NI + 1];
    bspline<R, NI, true>((R)fa, ma, da);
    bspline<R, NI, true>((R)fb, mb, db);
    bspline<R, NI, true>((R)fc, mc, dc);
    const C2 *g = (const C2 *)a.grid + (size_t)b * a.Na * a.Nb * a.Nc;
    int ga[NI + 1];
#pragma unroll
    for (int j = 1; j <= NI; j++) {
        int v = ia - (j - 2);
        ga[j] = (v > 0 ? v : a.Na + v) - 1;
    }
    // separable sums: d/ds_a, d/ds_b, d/ds_c of sum M_a M_b M_c phi
    double ea = 0.0, eb = 0.0, ec = 0.0;
    for (int jc = 1; jc <= NI; jc++) {
        int vc = icc - (jc - 2);
        const int gc = (vc > 0 ? vc : a.Nc + vc) - 1;
        R sa_c = 0, sda_c = 0, sdb_c = 0;
        for (int jb = 1; jb <= NI; jb++) {
            int vb = ib - (jb - 2);
            const int gb = (vb > 0 ? vb : a.Nb + vb) - 1;
            const C2 *rowp = g + ((size_t)gc * a.Nb + gb) * a.Na;
            R s0 = 0, s1 = 0;
#pragma unroll
            for (int ja = 1; ja <= NI; ja++) {
                const R phi = rowp[ga[ja]].x;
                s0 += ma[ja] * phi;
                s1 += da[ja] * phi;
            }
            sa_c += mb[jb] * s0;      // for the c derivative
            sda_c += mb[jb] * s1;     // for the a derivative
            sdb_c += db[jb] * s0;     // for the b derivative
        }
        ea += (double)(mc[jc] * sda_c);
        eb += (double)(mc[jc] * sdb_c);
        ec += (double)(dc[jc] * sa_c);
    }
    ea *= (double)a.Na;
    eb *= (double)a.Nb;
    ec *= (double)a.Nc;
    const double gx = ea * cell.hi[0] + eb * cell.hi[1] + ec * cell.hi[2];
    const double gy = ea * cell.hi[3] + eb * cell.hi[4] + ec * cell.hi[5];
    const double gz = ea * cell.hi[6] + eb * cell.hi[7] + ec * cell.hi[8];
    double *f = a.forceT;
    f[(3 * (size_t)at + 0) * a.P + b] -= gx * q;
    f[(3 * (size_t)at + 1) * a.P + b] -= gy * q;
    f[(3 * (size_t)at + 2) * a.P + b] -= gz * q;
}

// ---------------------------------------------------------------------------
// Batched complex FFT along one axis of the [bead][c][b][a] grid.  A block
// stages TL lines of length N in shared memory with coalesced loads (lines
// are consecutive in a for the b and c axes), runs an in-place radix-2
// decimation-in-time transform (or a direct DFT when N is not a power of
// two), and writes the lines back.  Unnormalised, exp(sign 2 pi i nk/N).
template <typename R>
__global__ void __launch_bounds__(256) fft_axis_kernel(void *data, int axis, int Na, int Nb, int Nc, int P, int TL,
                                                       const R *__restrict__ tw, int sign)
{
    typedef typename Cplx<R>::T C2;
    extern __shared__ unsigned char smem_raw[];
    C2 *sm = (C2 *)smem_raw;
    C2 *g = (C2 *)data;
    const int N = axis == 0 ? Na : (axis == 1 ? Nb : Nc);
    const size_t G = (size_t)Na * Nb * Nc;
    size_t base;
    long long estride, lstride;
    const int tile = blockIdx.x;
    if (axis == 0) {
        base = (size_t)tile * TL * Na;
        estride = 1;
        lstride = Na;
    } else {
        const int nat = Na / TL;
        const int at = tile % nat;
        const int rest = tile / nat;
        const int outer = axis == 1 ? Nc : Nb;
        const int o = rest % outer;
        const int bead = rest / outer;
        if (axis == 1) base = (size_t)bead * G + (size_t)o * Na * Nb + (size_t)at * TL;
        else base = (size_t)bead * G + (size_t)o * Na + (size_t)at * TL;
        estride = axis == 1 ? Na : (long long)Na * Nb;
        lstride = 1;
    }
    const bool pow2 = (N & (N - 1)) == 0;
    int logn = 0;
    while ((1 << logn) < N) logn++;
    const int tot = TL * N;
    // load (bit-reversed for the radix-2 path)
    for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
        int l, nn;
        if (axis == 0) { l = idx / N; nn = idx % N; }
        else { nn = idx / TL; l = idx % TL; }
        C2 v = g[base + (size_t)l * lstride + (size_t)nn * estride];
        int dst = nn;
        if (pow2) dst = __brev(nn) >> (32 - logn);
        if (logn == 0) dst = 0;
        sm[l * N + dst] = v;
    }
    __syncthreads();
    if (pow2) {
        for (int half = 1; half < N; half <<= 1) {
            const int tstep = N / (2 * half);
            for (int idx = threadIdx.x; idx < TL * (N / 2); idx += blockDim.x) {
                const int l = idx / (N / 2);
                const int bf = idx % (N / 2);
                const int grp = bf / half, k = bf % half;
                const int i0 = grp * 2 * half + k, i1 = i0 + half;
                const R wr = tw[2 * (k * tstep)], wi = (R)sign * tw[2 * (k * tstep) + 1];
                C2 u = sm[l * N + i0], v = sm[l * N + i1];
                C2 vw;
                vw.x = v.x * wr - v.y * wi;
                vw.y = v.x * wi + v.y * wr;
                sm[l * N + i0].x = u.x + vw.x;
                sm[l * N + i0].y = u.y + vw.y;
                sm[l * N + i1].x = u.x - vw.x;
                sm[l * N + i1].y = u.y - vw.y;
            }
            __syncthreads();
        }
        for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
            int l, nn;
            if (axis == 0) { l = idx / N; nn = idx % N; }
            else { nn = idx / TL; l = idx % TL; }
            g[base + (size_t)l * lstride + (size_t)nn * estride] = sm[l * N + nn];
        }
    } else {
        for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
            int l, kk;
            if (axis == 0) { l = idx / N; kk = idx % N; }
            else { kk = idx / TL; l = idx % TL; }
            R sr = 0, si = 0;
            for (int nn = 0; nn < N; nn++) {
                const int e = (int)(((long long)nn * kk) % N);
                const R wr = tw[2 * e], wi = (R)sign * tw[2 * e + 1];
                const C2 v = sm[l * N + nn];
                sr += v.x * wr - v.y * wi;
                si += v.x * wi + v.y * wr;
            }
            C2 o;
            o.x = sr;
            o.y = si;
            g[base + (size_t)l * lstride + (size_t)kk * estride] = o;
        }
    }
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

// Energy, virial and convolution over one bead's transformed grid.  Energy
// per half-list entry is |S|^2 preg bw (ewald3d_pme.c:396); the full grid
// holds every entry twice, hence the 1/2.
template <typename R>
__global__ void __launch_bounds__(256) conv_kernel(void *data, const R *__restrict__ filt, int Na, int Nb, int Nc,
                                                   Cell cell, double alp, double *__restrict__ acc, int energy)
{
    typedef typename Cplx<R>::T C2;
    const size_t G = (size_t)Na * Nb * Nc;
    const int bead = blockIdx.y;
    const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0, pxx = 0, pyy = 0, pzz = 0, pxy = 0, pxz = 0, pyz = 0;
    if (g < G) {
        C2 *p = (C2 *)data + (size_t)bead * G + g;
        const R w = filt[g];
        C2 s = *p;
        if (w != (R)0 && energy) {
            const int a = (int)(g % Na);
            const int bb = (int)((g / Na) % Nb);
            const int c = (int)(g / ((size_t)Na * Nb));
            const double ka = a <= Na / 2 ? a : a - Na, kb = bb <= Nb / 2 ? bb : bb - Nb,
                         kc = c <= Nc / 2 ? c : c - Nc;
            const double tpi = 2.0 * M_PI;
            const double xk = tpi * (ka * cell.hi[0] + kb * cell.hi[1] + kc * cell.hi[2]);
            const double yk = tpi * (ka * cell.hi[3] + kb * cell.hi[4] + kc * cell.hi[5]);
            const double zk = tpi * (ka * cell.hi[6] + kb * cell.hi[7] + kc * cell.hi[8]);
            const double g2 = xk * xk + yk * yk + zk * zk;
            const double falp2 = 4.0 * alp * alp;
            const double sm = 0.5 * ((double)s.x * (double)s.x + (double)s.y * (double)s.y) * (double)w;
            e = sm;
            const double prep = -2.0 * ((g2 / falp2) + 1.0) / g2 * sm;
            pxx = prep * xk * xk;
            pyy = prep * yk * yk;
            pzz = prep * zk * zk;
            pxy = prep * xk * yk;
            pxz = prep * xk * zk;
            pyz = prep * yk * zk;
        }
        s.x *= w;
        s.y *= w;
        *p = s;
    }
    if (!energy) return;
    double v[7] = {e, pxx, pyy, pzz, pxy, pxz, pyz};
    __shared__ double red[7][8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 7; c++) {
        double t = warp_sum(v[c]);
        if (lane == 0) red[c][wid] = t;
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

// Lines per block: a power of two <= 16 that divides the line count of the
// tile decomposition and keeps the staged tile within 48 KB.
template <typename R>
static int pick_tl(long long divisor, int N)
{
    typedef typename Cplx<R>::T C2;
    int tl = 16;
    while (tl > 1 && ((divisor % tl) || (size_t)tl * N * sizeof(C2) > 48 * 1024)) tl >>= 1;
    return tl;
}

template <typename R, int NI>
static cudaError_t launch_pme_t(pinyb200_ctx *c, const Cell &cell, bool energy)
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
    a.forceT = c->d_forceT;
    typedef typename Cplx<R>::T C2;
    const size_t G = (size_t)a.Na * a.Nb * a.Nc;
    cudaError_t err = cudaMemsetAsync(c->d_grid, 0, sizeof(C2) * G * c->P, c->stream);
    if (err != cudaSuccess) return err;
    const long long nt = (long long)a.nchrg * a.P;
    const int threads = 256;
    spread_kernel<R, NI><<<(unsigned)((nt + threads - 1) / threads), threads, 0, c->stream>>>(a, cell);
    const R *tw[3];
    const R *twbase = (const R *)(sizeof(R) == 8 ? (const void *)c->d_twiddle64 : (const void *)c->d_twiddle32);
    const int maxN = 256;
    for (int ax = 0; ax < 3; ax++) tw[ax] = twbase + 2 * maxN * ax;
    const int dims[3] = {a.Na, a.Nb, a.Nc};
    const int TLs[3] = {pick_tl<R>((long long)a.Nb * a.Nc * a.P, a.Na), pick_tl<R>(a.Na, a.Nb),
                        pick_tl<R>(a.Na, a.Nc)};
    for (int pass = 0; pass < 2; pass++) {
        const int sign = pass == 0 ? +1 : -1;
        for (int ax = 0; ax < 3; ax++) {
            const int N = dims[ax];
            const int TL = TLs[ax];
            long long nlines = (long long)G * a.P / N;
            int tiles = (int)(nlines / TL);
            size_t sh = sizeof(C2) * TL * N;
            fft_axis_kernel<R><<<tiles, 256, sh, c->stream>>>(c->d_grid, ax, a.Na, a.Nb, a.Nc, a.P, TL, tw[ax], sign);
        }
        if (pass == 0) {
            dim3 grid((unsigned)((G + 255) / 256), (unsigned)a.P);
            const R *filt = (const R *)c->d_filter;
            if (sizeof(R) == 4) filt = (const R *)((const double *)c->d_filter + G);
            conv_kernel<R><<<grid, 256, 0, c->stream>>>(c->d_grid, filt, a.Na, a.Nb, a.Nc, cell, c->alp_ewd, c->d_acc,
                                                        energy ? 1 : 0);
        }
    }
    gather_kernel<R, NI><<<(unsigned)((nt + threads - 1) / threads), threads, 0, c->stream>>>(a, cell);
    return cudaGetLastError();
}

template <typename R>
static cudaError_t launch_pme_r(pinyb200_ctx *c, const Cell &cell, bool energy)
{
    switch (c->sys.n_interp) {
    case 4: return launch_pme_t<R, 4>(c, cell, energy);
    case 5: return launch_pme_t<R, 5>(c, cell, energy);
    case 6: return launch_pme_t<R, 6>(c, cell, energy);
    case 7: return launch_pme_t<R, 7>(c, cell, energy);
    case 8: return launch_pme_t<R, 8>(c, cell, energy);
    case 10: return launch_pme_t<R, 10>(c, cell, energy);
    default: return cudaErrorInvalidValue;
    }
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

}  // namespace pinyb200
