// Adjoint of the force path with respect to model parameters.
//
// For K parameters theta_k the caller supplies tangent channels: the
// derivative of the set-up data (charges, the vdW spline tables, ghost
// coefficients, bond and bend series) with respect to theta_k.  One call
// runs a fresh forward evaluation (raw site forces, PME potential, spline
// records) and then one adjoint pass that, for every channel, sums
//   dE_k = d(vintert + vintrat)/d theta_k            (PINY's bead averages)
//   dF_k = sum_{beads, atoms} Fbar . dF/d theta_k    (F: forces on atoms with
//          the ghost force distributed, Fbar: the caller's upstream gradient)
// Pair terms are recomputed from the list, not stored.  With the site
// adjoint u (u = Fbar on atoms, u_M = sum_c coef_c Fbar_c on ghosts):
//   parameter tangents:  dF_k += sum_s u_s . T_k F_raw,s
//   ghost-coefficient tangents move the ghosts by w_M = sum_c dcoef_c r_c:
//          dF_k += sum_s u_s . (-H w)_s + sum_M (sum_c dcoef_c Fbar_c) . F_raw,M
//          dE_k += -sum_M F_raw,M . w_M
// H is the Hessian of the energy (pairs, excluded-pair correction, PME).
#include "common.cuh"

namespace pinyb200 {

__device__ __forceinline__ void ld3(const double *T, int P, int i, int b, double &x, double &y, double &z)
{
    x = T[(3 * (size_t)i + 0) * P + b];
    y = T[(3 * (size_t)i + 1) * P + b];
    z = T[(3 * (size_t)i + 2) * P + b];
}

// Per-thread channel sums flushed through shared memory; every thread of the
// block must call it.
__device__ __forceinline__ void grad_flush(const GradArgs &g, const double *acc, double *sh)
{
    for (int i = threadIdx.x; i < 2 * g.K; i += blockDim.x) sh[i] = 0.0;
    __syncthreads();
    for (int i = 0; i < 2 * g.K; i++)
        if (acc[i] != 0.0) atomicAdd(&sh[i], acc[i]);
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * g.K; i += blockDim.x)
        if (sh[i] != 0.0) atomicAdd(&g.gacc[i], sh[i]);
}

// u from the upstream gradient of the distributed forces fbar [P][natm][3]
// (ghost rows are then overwritten by grad_u_ghost_kernel).
__global__ void grad_u_kernel(const double *__restrict__ fbar, double *__restrict__ uT, int natm, int P)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)natm * 3 * P) return;
    const int b = (int)(t % P);
    const long long id = t / P;  // 3 * i + d
    const int i = (int)(id / 3), d = (int)(id % 3);
    uT[t] = fbar[((size_t)b * natm + i) * 3 + d];
}

__global__ void grad_u_ghost_kernel(const double *__restrict__ fbar, double *__restrict__ uT, int natm, int P,
                                    int nghost, int ncomp, const int *__restrict__ gatom,
                                    const int *__restrict__ gcomp, const double *__restrict__ gcoef)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nghost * P) return;
    const int b = (int)(t % P), gh = (int)(t / P);
    const int gl = gatom[gh];
    for (int d = 0; d < 3; d++) {
        double s = 0.0;
        for (int c = 0; c < ncomp; c++) {
            const int at = gcomp[gh * ncomp + c];
            if (at >= 0) s += gcoef[gh * ncomp + c] * fbar[((size_t)b * natm + at) * 3 + d];
        }
        uT[(3 * (size_t)gl + d) * P + b] = s;
    }
}

// Ghost tangents: positions w, the energy term and the u-tangent term.
__global__ void __launch_bounds__(256) grad_ghost_kernel(GradArgs g, int natm, int P, int nghost, int ncomp,
                                                         const int *__restrict__ gatom, const int *__restrict__ gcomp,
                                                         const double *__restrict__ posT,
                                                         const double *__restrict__ forceT,
                                                         const double *__restrict__ fbar)
{
    __shared__ double sh[2 * PINYB200_MAX_TAN];
    double acc[2 * PINYB200_MAX_TAN];
    for (int k = 0; k < 2 * g.K; k++) acc[k] = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (long long)nghost * P;
         t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t % P), gh = (int)(t / P);
        const int gl = gatom[gh];
        double fx, fy, fz;
        ld3(forceT, P, gl, b, fx, fy, fz);
        for (int k = 0; k < g.K; k++) {
            const double *dc = g.ch[k].dcoef;
            if (!dc) continue;
            double w[3] = {0, 0, 0}, tu[3] = {0, 0, 0};
            for (int c = 0; c < ncomp; c++) {
                const int at = gcomp[gh * ncomp + c];
                if (at < 0) continue;
                const double cf = dc[gh * ncomp + c];
                double x, y, z;
                ld3(posT, P, at, b, x, y, z);
                w[0] += cf * x;
                w[1] += cf * y;
                w[2] += cf * z;
                if (fbar) {
                    tu[0] += cf * fbar[((size_t)b * natm + at) * 3 + 0];
                    tu[1] += cf * fbar[((size_t)b * natm + at) * 3 + 1];
                    tu[2] += cf * fbar[((size_t)b * natm + at) * 3 + 2];
                }
            }
            for (int d = 0; d < 3; d++) g.ch[k].w[(3 * (size_t)gl + d) * P + b] = w[d];
            acc[2 * k] += -(fx * w[0] + fy * w[1] + fz * w[2]) / (double)P;
            acc[2 * k + 1] += tu[0] * fx + tu[1] * fy + tu[2] * fz;
        }
    }
    grad_flush(g, acc, sh);
}

// Derivative d/ddel of the interval cubic.
template <typename V, typename R>
__device__ __forceinline__ R spline_deriv(const V &c, R del)
{
    return c.y + del * ((R)2 * c.z + (R)3 * del * c.w);
}

struct GradPairArgs {
    const int *row, *col;  // force-bearing list (CSR)
    int natm, P, ntyp, nsplin, nuniq, use_xmod;
    const double *posT, *xmod;
    const int *atm_typ;
    const double *charge;
    const int *inter_map;
    const double *cutoff, *rmin, *dr, *dri;
    const int *has_vdw;
    const void *tab;
};

// Pairs: one thread per (row i, bead), beads fastest.
template <typename R>
__global__ void __launch_bounds__(128) grad_pair_kernel(GradPairArgs a, GradArgs g, Cell cell)
{
    typedef typename Vec4<R>::T V;
    __shared__ double sh[2 * PINYB200_MAX_TAN];
    double acc[2 * PINYB200_MAX_TAN];
    for (int k = 0; k < 2 * g.K; k++) acc[k] = 0.0;
    const V *__restrict__ tab = (const V *)a.tab;
    const int P = a.P, nsm2 = a.nsplin - 2;
    const size_t tstride = (size_t)a.nuniq * a.nsplin;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (long long)a.natm * P;
         t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t % P), i = (int)(t / P);
        const int beg = a.row[i], end = a.row[i + 1];
        if (beg == end) continue;
        double xi, yi, zi, uix, uiy, uiz;
        ld3(a.posT, P, i, b, xi, yi, zi);
        ld3(g.uT, P, i, b, uix, uiy, uiz);
        const int ti = a.atm_typ[i];
        const double qi = a.charge[i];
        for (int jj = beg; jj < end; jj++) {
            const int j = a.col[jj];
            const int pt = pair_type(ti, a.atm_typ[j], a.ntyp);
            const int u = a.inter_map[pt];
            double xj, yj, zj;
            ld3(a.posT, P, j, b, xj, yj, zj);
            double dx = __dsub_rn(xi, xj), dy = __dsub_rn(yi, yj), dz = __dsub_rn(zi, zj);
            if (a.use_xmod) {
                double shx = 0, shy = 0, shz = 0;
                period_pimd_exact(shx, shy, shz, __dsub_rn(a.xmod[3 * i], a.xmod[3 * j]),
                                  __dsub_rn(a.xmod[3 * i + 1], a.xmod[3 * j + 1]),
                                  __dsub_rn(a.xmod[3 * i + 2], a.xmod[3 * j + 2]), cell);
                dx = __dadd_rn(dx, shx);
                dy = __dadd_rn(dy, shy);
                dz = __dadd_rn(dz, shz);
            } else {
                period_exact(dx, dy, dz, cell);
            }
            const R rx = (R)dx, ry = (R)dy, rz = (R)dz;
            const R r = Idx<R>::dist(rx, ry, rz);
            if (!(r < (R)a.cutoff[pt])) continue;
            R del;
            const int kk = Idx<R>::knot(r, (R)a.rmin[u], (R)a.dr[u], (R)a.dri[u], nsm2, del);
            const size_t off = (size_t)u * a.nsplin + (kk - 1);
            const R dri = (R)a.dri[u];
            const R qj = (R)a.charge[j];
            const R q2 = (R)qi * qj;
            const V cC = ldg4(tab + T_CDV0C * tstride + off), eC = ldg4(tab + T_CV0C * tstride + off);
            const bool vdw = a.has_vdw[u] != 0;
            const R sC = spline_eval<V, R>(cC, del), sEC = spline_eval<V, R>(eC, del);
            R dv = q2 * sC, dvp = q2 * spline_deriv<V, R>(cC, del) * dri;
            if (vdw) {
                const V cV = ldg4(tab + T_CDV0 * tstride + off);
                dv += spline_eval<V, R>(cV, del);
                dvp += spline_deriv<V, R>(cV, del) * dri;
            }
            double ujx, ujy, ujz;
            ld3(g.uT, P, j, b, ujx, ujy, ujz);
            const R ux = (R)(uix - ujx), uy = (R)(uiy - ujy), uz = (R)(uiz - ujz);
            const R ur = ux * rx + uy * ry + uz * rz;
            for (int k = 0; k < g.K; k++) {
                const GradChan &ch = g.ch[k];
                R eT = 0, fT = 0;
                if (ch.dq) {
                    const R tq = (R)(ch.dq[i] * a.charge[j] + qi * ch.dq[j]);
                    eT += tq * sEC;
                    fT += tq * sC;
                }
                if (ch.ttab) {
                    const V *tt = (const V *)ch.ttab;
                    eT += spline_eval<V, R>(ldg4(tt + off), del);
                    fT += spline_eval<V, R>(ldg4(tt + tstride + off), del);
                }
                double f = (double)(ur * fT);
                if (ch.w) {
                    double wix, wiy, wiz, wjx, wjy, wjz;
                    ld3(ch.w, P, i, b, wix, wiy, wiz);
                    ld3(ch.w, P, j, b, wjx, wjy, wjz);
                    const R wx = (R)(wix - wjx), wy = (R)(wiy - wjy), wz = (R)(wiz - wjz);
                    if (wx != (R)0 || wy != (R)0 || wz != (R)0) {
                        const R uw = ux * wx + uy * wy + uz * wz, rw = rx * wx + ry * wy + rz * wz;
                        // -(u . H w) of the pair: F_i = r dv(r)
                        f += (double)(uw * dv + ur * rw * dvp / r);
                    }
                }
                acc[2 * k] += (double)eT / (double)P;
                acc[2 * k + 1] += f;
            }
        }
    }
    grad_flush(g, acc, sh);
}

// Excluded charged pairs (ecor): V = q_i q_j S(cv0), F_i = r q_i q_j S(cdv0).
__global__ void __launch_bounds__(256) grad_ecor_kernel(GradArgs g, int P, int necor, const int *__restrict__ j1s,
                                                        const int *__restrict__ j2s, int nsplin, double rmin, double dr,
                                                        double dri, const double4 *__restrict__ tab,
                                                        const double *__restrict__ posT,
                                                        const double *__restrict__ charge)
{
    __shared__ double sh[2 * PINYB200_MAX_TAN];
    double acc[2 * PINYB200_MAX_TAN];
    for (int k = 0; k < 2 * g.K; k++) acc[k] = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (long long)necor * P;
         t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t % P), ie = (int)(t / P);
        const int j1 = j1s[ie], j2 = j2s[ie];
        double x1, y1, z1, x2, y2, z2;
        ld3(posT, P, j1, b, x1, y1, z1);
        ld3(posT, P, j2, b, x2, y2, z2);
        const double dx = x1 - x2, dy = y1 - y2, dz = z1 - z2;
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        int kk = (int)((r - rmin) * dri + 0.5) + 3;
        kk = kk < nsplin - 2 ? kk : nsplin - 2;
        kk = kk > 3 ? kk : 3;
        const double del = (r - ((double)(kk - 3) * dr + rmin)) * dri;
        const double4 cv = tab[kk - 1], cd = tab[nsplin + kk - 1];
        const double sv = spline_eval<double4, double>(cv, del), sd = spline_eval<double4, double>(cd, del);
        const double q12 = charge[j1] * charge[j2];
        const double dv = q12 * sd, dvp = q12 * spline_deriv<double4, double>(cd, del) * dri;
        double u1x, u1y, u1z, u2x, u2y, u2z;
        ld3(g.uT, P, j1, b, u1x, u1y, u1z);
        ld3(g.uT, P, j2, b, u2x, u2y, u2z);
        const double ux = u1x - u2x, uy = u1y - u2y, uz = u1z - u2z;
        const double ur = ux * dx + uy * dy + uz * dz;
        for (int k = 0; k < g.K; k++) {
            const GradChan &ch = g.ch[k];
            double f = 0.0;
            if (ch.dq) {
                const double tq = ch.dq[j1] * charge[j2] + charge[j1] * ch.dq[j2];
                acc[2 * k] += tq * sv / (double)P;
                f += ur * tq * sd;
            }
            if (ch.w) {
                double w1x, w1y, w1z, w2x, w2y, w2z;
                ld3(ch.w, P, j1, b, w1x, w1y, w1z);
                ld3(ch.w, P, j2, b, w2x, w2y, w2z);
                const double wx = w1x - w2x, wy = w1y - w2y, wz = w1z - w2z;
                const double uw = ux * wx + uy * wy + uz * wz, rw = dx * wx + dy * wy + dz * wz;
                f += uw * dv + ur * rw * dvp / r;
            }
            acc[2 * k + 1] += f;
        }
    }
    grad_flush(g, acc, sh);
}

// Bonds: V = sum c_n x^n, x = r - r0; tangents of the series and of r0.
__global__ void __launch_bounds__(256) grad_bond_kernel(GradArgs g, int P, int nbond, const int *__restrict__ bj,
                                                        const double *__restrict__ eq, const double *__restrict__ cc,
                                                        const double *__restrict__ posT)
{
    __shared__ double sh[2 * PINYB200_MAX_TAN];
    double acc[2 * PINYB200_MAX_TAN];
    for (int k = 0; k < 2 * g.K; k++) acc[k] = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (long long)nbond * P;
         t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t % P), ib = (int)(t / P);
        const int j1 = bj[3 * ib], j2 = bj[3 * ib + 1], ty = bj[3 * ib + 2];
        double x1, y1, z1, x2, y2, z2;
        ld3(posT, P, j1, b, x1, y1, z1);
        ld3(posT, P, j2, b, x2, y2, z2);
        const double dx = x1 - x2, dy = y1 - y2, dz = z1 - z2;
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const double x = r - eq[ty];
        const double *c = cc + 7 * ty;
        double d1 = 0, d2 = 0, xp = 1.0;  // dV/dx, d2V/dx2
        for (int n = 1; n <= 6; n++) {
            d1 += n * c[n] * xp;
            xp *= x;
        }
        xp = 1.0;
        for (int n = 2; n <= 6; n++) {
            d2 += n * (n - 1) * c[n] * xp;
            xp *= x;
        }
        double u1x, u1y, u1z, u2x, u2y, u2z;
        ld3(g.uT, P, j1, b, u1x, u1y, u1z);
        ld3(g.uT, P, j2, b, u2x, u2y, u2z);
        const double ur = ((u1x - u2x) * dx + (u1y - u2y) * dy + (u1z - u2z) * dz) / r;
        for (int k = 0; k < g.K; k++) {
            const GradChan &ch = g.ch[k];
            if (!ch.bond_dc && !ch.bond_deq) continue;
            double vt = 0, dvt = 0;
            if (ch.bond_dc) {
                const double *tc = ch.bond_dc + 7 * ty;
                double p = 1.0, pm1 = 0.0;  // x^n, x^(n-1)
                for (int n = 0; n <= 6; n++) {
                    vt += tc[n] * p;
                    if (n >= 1) dvt += n * tc[n] * pm1;
                    pm1 = p;
                    p *= x;
                }
            }
            if (ch.bond_deq) {
                const double de = ch.bond_deq[ty];
                vt -= de * d1;
                dvt -= de * d2;
            }
            // F_1 = -dV/dx r_vec / r
            acc[2 * k] += vt / (double)P;
            acc[2 * k + 1] += -dvt * ur;
        }
    }
    grad_flush(g, acc, sh);
}

// Bends: V and forces are linear in the series (c, s, dc, ds); the tangent
// series give the tangent energy and forces through the forward formulas.
__global__ void __launch_bounds__(256) grad_bend_kernel(GradArgs g, int P, int nbend, const int *__restrict__ bj,
                                                        const double *__restrict__ posT)
{
    __shared__ double sh[2 * PINYB200_MAX_TAN];
    double acc[2 * PINYB200_MAX_TAN];
    for (int k = 0; k < 2 * g.K; k++) acc[k] = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (long long)nbend * P;
         t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t % P), ib = (int)(t / P);
        const int a1 = bj[4 * ib], a2 = bj[4 * ib + 1], a3 = bj[4 * ib + 2], ty = bj[4 * ib + 3];
        double x1, y1, z1, x2, y2, z2, x3, y3, z3;
        ld3(posT, P, a1, b, x1, y1, z1);
        ld3(posT, P, a2, b, x2, y2, z2);
        ld3(posT, P, a3, b, x3, y3, z3);
        const double dx12 = x1 - x2, dy12 = y1 - y2, dz12 = z1 - z2;
        const double dx23 = x3 - x2, dy23 = y3 - y2, dz23 = z3 - z2;
        const double r122i = 1.0 / (dx12 * dx12 + dy12 * dy12 + dz12 * dz12);
        const double r12i = sqrt(r122i);
        const double r322i = 1.0 / (dx23 * dx23 + dy23 * dy23 + dz23 * dz23);
        const double r32i = sqrt(r322i);
        const double rpmag = r12i * r32i;
        double cost = (dx12 * dx23 + dy12 * dy23 + dz12 * dz23) * rpmag;
        cost = cost < 1.0 ? cost : 1.0;
        cost = cost > -1.0 ? cost : -1.0;
        double sint = sqrt(1.0 - cost * cost);
        sint = sint > 1.0e-8 ? sint : 1.0e-8;
        const double cos122 = cost * r122i, cos322 = cost * r322i;
        double u1[3], u2[3], u3[3];
        ld3(g.uT, P, a1, b, u1[0], u1[1], u1[2]);
        ld3(g.uT, P, a2, b, u2[0], u2[1], u2[2]);
        ld3(g.uT, P, a3, b, u3[0], u3[1], u3[2]);
        const double g1x = dx23 * rpmag - dx12 * cos122, g1y = dy23 * rpmag - dy12 * cos122,
                     g1z = dz23 * rpmag - dz12 * cos122;
        const double g3x = dx12 * rpmag - dx23 * cos322, g3y = dy12 * rpmag - dy23 * cos322,
                     g3z = dz12 * rpmag - dz23 * cos322;
        // sum_a u_a . F_a for F_1 = g1 pre, F_3 = g3 pre, F_2 = -(F_1 + F_3)
        const double ug = (u1[0] - u2[0]) * g1x + (u1[1] - u2[1]) * g1y + (u1[2] - u2[2]) * g1z +
                          (u3[0] - u2[0]) * g3x + (u3[1] - u2[1]) * g3y + (u3[2] - u2[2]) * g3z;
        for (int k = 0; k < g.K; k++) {
            const GradChan &ch = g.ch[k];
            if (!ch.bend_c) continue;
            const double *c = ch.bend_c + 7 * ty, *s = ch.bend_s + 7 * ty, *dc = ch.bend_dc + 7 * ty,
                         *ds = ch.bend_ds + 7 * ty;
            const double vc = ((((((c[6] * cost + c[5]) * cost + c[4]) * cost + c[3]) * cost + c[2]) * cost + c[1]) *
                                   cost +
                               c[0]);
            const double sisum = (((((s[6] * sint + s[5]) * sint + s[4]) * sint + s[3]) * sint + s[2]) * sint);
            const double vt = vc + (sisum * cost + s[1] * sint);
            const double dvc = (((((dc[6] * cost + dc[5]) * cost + dc[4]) * cost + dc[3]) * cost + dc[2]) * cost + dc[1]);
            double dvs = ((((ds[6] * sint + ds[5]) * sint + ds[4]) * sint + ds[3]) * sint + ds[2]);
            dvs = dvs * cost + ds[1];
            const double pre = -(dvc + sisum - dvs * cost / sint);
            acc[2 * k] += vt / (double)P;
            acc[2 * k + 1] += ug * pre;
        }
    }
    grad_flush(g, acc, sh);
}

// ---------------------------------------------------------------------------

static int nblk(long long n, int t, int sm)
{
    long long b = (n + t - 1) / t;
    if (b > (long long)sm * 8) b = (long long)sm * 8;
    return (int)(b < 1 ? 1 : b);
}

cudaError_t launch_grad_terms(pinyb200_ctx *c, const Cell &cell, const GradArgs &g, const double *d_fbar)
{
    const DeviceSystem &s = c->sys;
    const int P = c->P, sm = c->sm_count;
    cudaStream_t st = c->stream;
    const long long nsite = (long long)s.natm * 3 * P;
    if (d_fbar) {
        grad_u_kernel<<<(unsigned)((nsite + 255) / 256), 256, 0, st>>>(d_fbar, (double *)g.uT, s.natm, P);
        if (s.nghost)
            grad_u_ghost_kernel<<<(unsigned)(((long long)s.nghost * P + 255) / 256), 256, 0, st>>>(
                d_fbar, (double *)g.uT, s.natm, P, s.nghost, s.ghost_ncomp, s.ghost_atom, s.ghost_comp,
                s.ghost_coef);
    } else {
        cudaError_t e = cudaMemsetAsync((void *)g.uT, 0, nsite * sizeof(double), st);
        if (e != cudaSuccess) return e;
    }
    if (s.nghost)
        grad_ghost_kernel<<<nblk((long long)s.nghost * P, 256, sm), 256, 0, st>>>(
            g, s.natm, P, s.nghost, s.ghost_ncomp, s.ghost_atom, s.ghost_comp, c->d_posT, c->d_forceT, d_fbar);
    GradPairArgs a;
    a.row = c->d_rowA;
    a.col = c->d_colA;
    a.natm = s.natm;
    a.P = P;
    a.ntyp = s.ntyp;
    a.nsplin = s.nsplin;
    a.nuniq = s.nuniq;
    a.use_xmod = P > 1;
    a.posT = c->d_posT;
    a.xmod = P > 1 ? c->d_xmod : c->d_posT;
    a.atm_typ = s.atm_typ;
    a.charge = s.charge;
    a.inter_map = s.inter_map;
    a.cutoff = s.cutoff;
    a.rmin = s.rmin;
    a.dr = s.dr;
    a.dri = s.dri;
    a.has_vdw = s.has_vdw;
    if (c->precision == PINYB200_FP64) {
        a.tab = s.tab64;
        grad_pair_kernel<double><<<nblk((long long)s.natm * P, 128, sm), 128, 0, st>>>(a, g, cell);
    } else {
        a.tab = s.tab32;
        grad_pair_kernel<float><<<nblk((long long)s.natm * P, 128, sm), 128, 0, st>>>(a, g, cell);
    }
    if (s.necor)
        grad_ecor_kernel<<<nblk((long long)s.necor * P, 256, sm), 256, 0, st>>>(
            g, P, s.necor, s.ecor_j1, s.ecor_j2, s.ecor_nsplin, s.ecor_rmin, s.ecor_dr, s.ecor_dri, s.ecor_tab,
            c->d_posT, s.charge);
    if (s.nbond)
        grad_bond_kernel<<<nblk((long long)s.nbond * P, 256, sm), 256, 0, st>>>(g, P, s.nbond, s.bond_j, s.bond_eq,
                                                                               s.bond_c, c->d_posT);
    if (s.nbend)
        grad_bend_kernel<<<nblk((long long)s.nbend * P, 256, sm), 256, 0, st>>>(g, P, s.nbend, s.bend_j, c->d_posT);
    return cudaGetLastError();
}

}  // namespace pinyb200

// ---------------------------------------------------------------------------
// C ABI

using namespace pinyb200;

namespace {

template <typename T>
int grad_upload(pinyb200_ctx *c, const T *src, size_t n, const T **dst)
{
    *dst = nullptr;
    if (!src || n == 0) return PINYB200_OK;
    void *p = nullptr;
    if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess)
        return record_error(c, PINYB200_ERR_CUDA, "grad_prepare: device allocation failed");
    c->grad.dev.push_back(p);
    if (cudaMemcpy(p, src, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
        return record_error(c, PINYB200_ERR_CUDA, "grad_prepare: copy failed");
    *dst = (const T *)p;
    return PINYB200_OK;
}

void grad_release(pinyb200_ctx *c)
{
    for (void *p : c->grad.dev) cudaFree(p);
    c->grad.dev.clear();
    c->grad.K = 0;
    c->grad.d_u = nullptr;
    c->grad.d_gacc = nullptr;
    c->grad.d_grid2 = nullptr;
}

}  // namespace

extern "C" {

int pinyb200_grad_prepare(pinyb200_ctx *c, int ntan, const pinyb200_tangent *tan)
{
    if (!c || ntan < 0 || ntan > PINYB200_MAX_TAN || (ntan > 0 && !tan))
        return record_error(c, PINYB200_ERR_ARG, "grad_prepare: 0..16 tangents expected");
    if (cudaSetDevice(c->device) != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, "grad_prepare: device");
    cudaStreamSynchronize(c->stream);
    grad_release(c);
    GradHost &gh = c->grad;
    const DeviceSystem &s = c->sys;
    const int natm = s.natm, P = c->P;
    for (int k = 0; k < ntan; k++) {
        const pinyb200_tangent &t = tan[k];
        GradChan &ch = gh.ch[k];
        ch = GradChan();
        int rc = grad_upload(c, t.dcharge, t.dcharge ? (size_t)natm : 0, &ch.dq);
        if (rc) return rc;
        gh.dq_dot_q[k] = gh.dq_sum[k] = 0.0;
        if (t.dcharge)
            for (int i = 0; i < natm; i++) {
                gh.dq_dot_q[k] += c->h_charge[i] * t.dcharge[i];
                gh.dq_sum[k] += t.dcharge[i];
            }
        if (t.dcv0 || t.dcdv0) {
            // tangent tables as interval coefficients [2][nuniq][nsplin]
            const size_t per = (size_t)s.nsplin;
            std::vector<double> all((size_t)2 * 4 * s.nuniq * per, 0.0), tmp, zero(per, 0.0);
            const double *src[2] = {t.dcv0, t.dcdv0};
            for (int kind = 0; kind < 2; kind++)
                for (int u = 0; u < s.nuniq; u++) {
                    table_coefs(src[kind] ? src[kind] + (size_t)u * per : zero.data(), s.nsplin, tmp);
                    std::copy(tmp.begin(), tmp.end(), all.begin() + ((size_t)kind * s.nuniq + u) * per * 4);
                }
            if (c->precision == PINYB200_FP64) {
                const double *p = nullptr;
                rc = grad_upload(c, all.data(), all.size(), &p);
                ch.ttab = p;
            } else {
                std::vector<float> f32(all.begin(), all.end());
                const float *p = nullptr;
                rc = grad_upload(c, f32.data(), f32.size(), &p);
                ch.ttab = p;
            }
            if (rc) return rc;
        }
        if (t.dghost_coef && s.nghost > 0) {
            rc = grad_upload(c, t.dghost_coef, (size_t)s.nghost * s.ghost_ncomp, &ch.dcoef);
            if (rc) return rc;
            void *w = nullptr;
            if (cudaMalloc(&w, (size_t)natm * 3 * P * sizeof(double)) != cudaSuccess)
                return record_error(c, PINYB200_ERR_CUDA, "grad_prepare: device allocation failed");
            gh.dev.push_back(w);
            if (cudaMemset(w, 0, (size_t)natm * 3 * P * sizeof(double)) != cudaSuccess)
                return record_error(c, PINYB200_ERR_CUDA, "grad_prepare: memset failed");
            ch.w = (double *)w;
        }
        if (t.dbond_eq || t.dbond_c) {
            std::vector<double> z((size_t)7 * c->nbond_typ, 0.0), ze(c->nbond_typ, 0.0);
            rc = grad_upload(c, t.dbond_eq ? t.dbond_eq : ze.data(), ze.size(), &ch.bond_deq);
            if (!rc) rc = grad_upload(c, t.dbond_c ? t.dbond_c : z.data(), z.size(), &ch.bond_dc);
            if (rc) return rc;
        }
        if (t.dbend_c) {
            if (!t.dbend_s || !t.dbend_dc || !t.dbend_ds)
                return record_error(c, PINYB200_ERR_ARG, "grad_prepare: bend tangents need c, s, dc and ds");
            const size_t n = (size_t)7 * c->nbend_typ;
            rc = grad_upload(c, t.dbend_c, n, &ch.bend_c);
            if (!rc) rc = grad_upload(c, t.dbend_s, n, &ch.bend_s);
            if (!rc) rc = grad_upload(c, t.dbend_dc, n, &ch.bend_dc);
            if (!rc) rc = grad_upload(c, t.dbend_ds, n, &ch.bend_ds);
            if (rc) return rc;
        }
        gh.dclong[k] = t.dclong;
    }
    void *p = nullptr;
    if (cudaMalloc(&p, (size_t)natm * 3 * P * sizeof(double)) != cudaSuccess)
        return record_error(c, PINYB200_ERR_CUDA, "grad_prepare: device allocation failed");
    gh.dev.push_back(p);
    gh.d_u = (double *)p;
    if (cudaMalloc(&p, (size_t)2 * PINYB200_MAX_TAN * sizeof(double)) != cudaSuccess)
        return record_error(c, PINYB200_ERR_CUDA, "grad_prepare: device allocation failed");
    gh.dev.push_back(p);
    gh.d_gacc = (double *)p;
    if (s.nchrg > 0 && s.nktot > 0) {
        const size_t G = (size_t)s.ngrid[0] * s.ngrid[1] * s.ngrid[2];
        const size_t rsz = c->precision == PINYB200_FP64 ? sizeof(double) : sizeof(float);
        if (cudaMalloc(&p, G * P * rsz) != cudaSuccess)
            return record_error(c, PINYB200_ERR_CUDA, "grad_prepare: device allocation failed");
        gh.dev.push_back(p);
        gh.d_grid2 = p;
    }
    gh.K = ntan;
    return PINYB200_OK;
}

int pinyb200_grad(pinyb200_ctx *c, const double *d_pos, const double *d_xmod, const double *hmat,
                  const double *d_fbar, double *dE, double *dF, void *stream)
{
    if (!c || !d_pos || !hmat) return record_error(c, PINYB200_ERR_ARG, "grad: NULL argument");
    if (!c->have_list) return record_error(c, PINYB200_ERR_STATE, "grad: build the Verlet list first");
    if (!c->grad.d_gacc) return record_error(c, PINYB200_ERR_STATE, "grad: call pinyb200_grad_prepare first");
    if (cudaSetDevice(c->device) != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, "grad: device");
    cudaStream_t own = c->stream;
    if (stream) c->stream = (cudaStream_t)stream;
    struct Restore {
        pinyb200_ctx *c;
        cudaStream_t s;
        ~Restore() { c->stream = s; }
    } restore{c, own};
    const Cell cell = cell_from_hmat(hmat);
    const GradHost &gh = c->grad;
    const int K = gh.K;
    // forward: raw site forces (ghosts not distributed), potential grid, records
    c->pme_full_records = true;
    int rc = enqueue_device(c, d_pos, d_xmod, cell, 0, c->d_force_aos, false, nullptr);
    c->pme_full_records = false;
    if (rc) return rc;
    if (cudaMemsetAsync(gh.d_gacc, 0, (size_t)2 * PINYB200_MAX_TAN * sizeof(double), c->stream) != cudaSuccess)
        return record_error(c, PINYB200_ERR_CUDA, "grad: memset failed");
    GradArgs g;
    g.K = K;
    for (int k = 0; k < K; k++) g.ch[k] = gh.ch[k];
    g.uT = gh.d_u;
    g.gacc = gh.d_gacc;
    cudaError_t e = launch_grad_terms(c, cell, g, d_fbar);
    if (e == cudaSuccess) e = launch_pme_adjoint(c, cell, g);
    if (e != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, std::string("grad: ") + cudaGetErrorString(e));
    std::vector<double> h(2 * PINYB200_MAX_TAN, 0.0);
    e = cudaMemcpyAsync(h.data(), gh.d_gacc, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, std::string("grad: ") + cudaGetErrorString(e));
    // terms without forces: Ewald self and background (ewald3d_self_bgr.c:28-80), LJ tail
    double q1 = 0;
    for (double q : c->h_charge) q1 += q;
    const bool ewald = c->sys.nktot > 0 && c->sys.nchrg > 0;
    for (int k = 0; k < K; k++) {
        double de = h[2 * k];
        if (ewald) {
            de += -2.0 * gh.dq_dot_q[k] * c->alp_ewd * c->self_erf / sqrt(M_PI);
            de += -q1 * gh.dq_sum[k] * M_PI / (c->alp_ewd * c->alp_ewd * cell.vol);
        }
        de += gh.dclong[k] / cell.vol;
        if (dE) dE[k] = de;
        if (dF) dF[k] = h[2 * k + 1];
    }
    return PINYB200_OK;
}

}  // extern "C"
