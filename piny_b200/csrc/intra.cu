// Intramolecular terms, Ewald exclusion correction, ghost sites and the
// layout transposes, all in FP64 for every bead.
//
//   bonds   bond_both (src/energy/intra/bond_both.c:29-420): power series
//           V = sum c_n (r - r0)^n by Horner, F = -dV/dr d/r
//   bends   bend (src/energy/intra/bend.c:28-440): cos/sin series with the
//           sin clamp at 1e-8 and PINY's chain-rule forces
//   ecor    ecor (src/energy/intra/ecorr.c:28-274): q_i q_j S(cv0),
//           spline of -erf(alpha r)/r plus the finite-k correction
//   ghosts  get_ghost_pos / distrib_ghost_force
//           (src/energy/intra_con/ghost_control.c:28-129)
#include <algorithm>

#include <vector>

#include "boxtab.cuh"
#include "common.cuh"

namespace pinyb200 {

// Block-level reduction of per-thread energy/virial sums by bead: shared
// FP64 atomics (S_NSLOT slots per bead), then one global atomic per (bead,
// slot) per block.  Every thread of the block must call it.
template <int NV>
__device__ __forceinline__ void block_acc(double *acc, int P, int b, const int *slot, const double *v, double *sh)
{
    for (int i = threadIdx.x; i < P * NV; i += blockDim.x) sh[i] = 0.0;
    __syncthreads();
#pragma unroll
    for (int c = 0; c < NV; c++)
        if (v[c] != 0.0) atomicAdd(&sh[b * NV + c], v[c]);
    __syncthreads();
    for (int i = threadIdx.x; i < P * NV; i += blockDim.x)
        if (sh[i] != 0.0) atomicAdd(&acc[(size_t)(i / NV) * S_NSLOT + slot[i % NV]], sh[i]);
}

// out[c][r] = in[r][c] for an rows x cols matrix of doubles, through a
// 32 x 32 shared tile (padded against bank conflicts): both the global reads
// and the global writes are 256-byte rows.  Positions in: in = [P][natm*3]
// (PINY's bead-major order), out = [natm*3][P]; forces out the reverse.
__device__ __forceinline__ void transpose_tiled_body(const double *__restrict__ in, double *__restrict__ out, int rows,
                                                     long long cols, const VBlk vb)
{
    __shared__ double tile[32][33];
    const long long c0 = (long long)vb.x * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int r0 = vb.y * 32; r0 < rows; r0 += vb.gy * 32) {
#pragma unroll
        for (int k = 0; k < 32; k += 8) {
            const int r = r0 + ty + k;
            const long long c = c0 + tx;
            if (r < rows && c < cols) tile[ty + k][tx] = in[(size_t)r * cols + c];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 32; k += 8) {
            const long long c = c0 + ty + k;
            const int r = r0 + tx;
            if (r < rows && c < cols) out[(size_t)c * rows + r] = tile[tx][ty + k];
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) transpose_tiled_kernel(const double *__restrict__ in, double *__restrict__ out,
                                                              int rows, long long cols)
{
    transpose_tiled_body(in, out, rows, cols, hw_blk());
}

__device__ __forceinline__ void ghost_pos_body(double *__restrict__ posT, int P, int nghost, int ncomp,
                                 const int *__restrict__ gatom, const int *__restrict__ gcomp,
                                 const double *__restrict__ gcoef, const VBlk vb)
{
    const long long t = (long long)vb.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nghost * P) return;
    const int b = (int)(t % P);
    const int g = (int)(t / P);
    const int gl = gatom[g];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        double v = 0.0;
        for (int c = 0; c < ncomp; c++) {
            const int at = gcomp[g * ncomp + c];
            if (at < 0) continue;
            v = __dadd_rn(v, __dmul_rn(gcoef[g * ncomp + c], posT[(3 * (size_t)at + d) * P + b]));
        }
        posT[(3 * (size_t)gl + d) * P + b] = v;
    }
}

__global__ void ghost_pos_kernel(double *__restrict__ posT, int P, int nghost, int ncomp,
                                 const int *__restrict__ gatom, const int *__restrict__ gcomp,
                                 const double *__restrict__ gcoef)
{
    ghost_pos_body(posT, P, nghost, ncomp, gatom, gcomp, gcoef, hw_blk());
}

__device__ __forceinline__ void ghost_distrib_body(double *__restrict__ fT, int P, int nghost, int ncomp,
                                     const int *__restrict__ gatom, const int *__restrict__ gcomp,
                                     const double *__restrict__ gcoef, const VBlk vb)
{
    const long long t = (long long)vb.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nghost * P) return;
    const int b = (int)(t % P);
    const int g = (int)(t / P);
    const int gl = gatom[g];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double fg = fT[(3 * (size_t)gl + d) * P + b];
        for (int c = 0; c < ncomp; c++) {
            const int at = gcomp[g * ncomp + c];
            if (at < 0) continue;
            fT[(3 * (size_t)at + d) * P + b] += gcoef[g * ncomp + c] * fg;
        }
        fT[(3 * (size_t)gl + d) * P + b] = 0.0;
    }
}

__global__ void ghost_distrib_kernel(double *__restrict__ fT, int P, int nghost, int ncomp,
                                     const int *__restrict__ gatom, const int *__restrict__ gcomp,
                                     const double *__restrict__ gcoef)
{
    ghost_distrib_body(fT, P, nghost, ncomp, gatom, gcomp, gcoef, hw_blk());
}

struct IntraArgs {
    int natm, P;
    const double *posT;
    double *forceT;
    double *acc;
    const double *charge;
    int energy;
};

__device__ __forceinline__ void add_f(double *fT, int P, int at, int b, double fx, double fy, double fz)
{
    atomicAdd(&fT[(3 * (size_t)at + 0) * P + b], fx);
    atomicAdd(&fT[(3 * (size_t)at + 1) * P + b], fy);
    atomicAdd(&fT[(3 * (size_t)at + 2) * P + b], fz);
}

__device__ __forceinline__ void load_x(const double *posT, int P, int at, int b, double &x, double &y, double &z)
{
    x = posT[(3 * (size_t)at + 0) * P + b];
    y = posT[(3 * (size_t)at + 1) * P + b];
    z = posT[(3 * (size_t)at + 2) * P + b];
}

__device__ __forceinline__ void bond_body(const IntraArgs &a, int nbond, const int *__restrict__ bj,
                                                   const double *__restrict__ eq, const double *__restrict__ cc,
                                                   const double *__restrict__ dc, const VBlk vb)
{
    __shared__ double sh[64 * 7];
    const long long t0 = (long long)vb.x * blockDim.x + threadIdx.x;
    const long long stride = (long long)vb.gx * blockDim.x;  // a multiple of P
    const int b = (int)(t0 % a.P);
    double v = 0, p[6] = {0, 0, 0, 0, 0, 0};
    for (long long t = t0; t < (long long)nbond * a.P; t += stride) {
        const int ib = (int)(t / a.P);
        const int j1 = bj[3 * ib], j2 = bj[3 * ib + 1], ty = bj[3 * ib + 2];
        double x1, y1, z1, x2, y2, z2;
        load_x(a.posT, a.P, j1, b, x1, y1, z1);
        load_x(a.posT, a.P, j2, b, x2, y2, z2);
        const double dx = x1 - x2, dy = y1 - y2, dz = z1 - z2;
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const double rr0 = r - eq[ty];
        const double *c = cc + 7 * ty, *d = dc + 7 * ty;
        v += (((((c[6] * rr0 + c[5]) * rr0 + c[4]) * rr0 + c[3]) * rr0 + c[2]) * rr0 + c[1]) * rr0 + c[0];
        const double dv = ((((d[6] * rr0 + d[5]) * rr0 + d[4]) * rr0 + d[3]) * rr0 + d[2]) * rr0 + d[1];
        const double pre = -dv / r;
        const double fx = dx * pre, fy = dy * pre, fz = dz * pre;
        add_f(a.forceT, a.P, j1, b, fx, fy, fz);
        add_f(a.forceT, a.P, j2, b, -fx, -fy, -fz);
        p[0] += dx * fx; p[1] += dy * fy; p[2] += dz * fz; p[3] += dx * fy; p[4] += dx * fz; p[5] += dy * fz;
    }
    if (a.energy) {
        const int slot[7] = {S_VBOND, S_PXX, S_PYY, S_PZZ, S_PXY, S_PXZ, S_PYZ};
        const double vals[7] = {v, p[0], p[1], p[2], p[3], p[4], p[5]};
        block_acc<7>(a.acc, a.P, b, slot, vals, sh);
    }
}

__global__ void __launch_bounds__(256) bond_kernel(const __grid_constant__ IntraArgs a, int nbond, const int *__restrict__ bj,
                                                   const double *__restrict__ eq, const double *__restrict__ cc,
                                                   const double *__restrict__ dc)
{
    bond_body(a, nbond, bj, eq, cc, dc, hw_blk());
}

// One bend of one bead (bend.c:186-330): forces on the outer atoms f1, f3
// (the middle atom takes -(f1 + f3)), the bond vectors for the virial, and
// the energy.
struct BendTerm {
    double dx12, dy12, dz12, dx23, dy23, dz23;
    double fx1, fy1, fz1, fx3, fy3, fz3;
    double v;
};

__device__ __forceinline__ void bend_term(const double *posT, int P, int a1, int a2, int a3, int b,
                                          const double *c, const double *s, const double *dc, const double *ds,
                                          BendTerm &t)
{
    double x1, y1, z1, x2, y2, z2, x3, y3, z3;
    load_x(posT, P, a1, b, x1, y1, z1);
    load_x(posT, P, a2, b, x2, y2, z2);
    load_x(posT, P, a3, b, x3, y3, z3);
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
    const double vc = ((((((c[6] * cost + c[5]) * cost + c[4]) * cost + c[3]) * cost + c[2]) * cost + c[1]) * cost +
                       c[0]);
    const double sisum = (((((s[6] * sint + s[5]) * sint + s[4]) * sint + s[3]) * sint + s[2]) * sint);
    t.v = vc + (sisum * cost + s[1] * sint);
    const double dvc = (((((dc[6] * cost + dc[5]) * cost + dc[4]) * cost + dc[3]) * cost + dc[2]) * cost + dc[1]);
    double dvs = ((((ds[6] * sint + ds[5]) * sint + ds[4]) * sint + ds[3]) * sint + ds[2]);
    dvs = dvs * cost + ds[1];
    const double pre = -(dvc + sisum - dvs * cost / sint);
    t.fx1 = (dx23 * rpmag - dx12 * cos122) * pre;
    t.fy1 = (dy23 * rpmag - dy12 * cos122) * pre;
    t.fz1 = (dz23 * rpmag - dz12 * cos122) * pre;
    t.fx3 = (dx12 * rpmag - dx23 * cos322) * pre;
    t.fy3 = (dy12 * rpmag - dy23 * cos322) * pre;
    t.fz3 = (dz12 * rpmag - dz23 * cos322) * pre;
    t.dx12 = dx12; t.dy12 = dy12; t.dz12 = dz12;
    t.dx23 = dx23; t.dy23 = dy23; t.dz23 = dz23;
}

__device__ __forceinline__ void bend_body(const IntraArgs &a, int nbend, const int *__restrict__ bj,
                                                   const double *__restrict__ bc, const double *__restrict__ bs,
                                                   const double *__restrict__ bdc, const double *__restrict__ bds, const VBlk vb)
{
    __shared__ double sh[64 * 7];
    const long long t0 = (long long)vb.x * blockDim.x + threadIdx.x;
    const long long stride = (long long)vb.gx * blockDim.x;  // a multiple of P
    const int b = (int)(t0 % a.P);
    double v = 0, p[6] = {0, 0, 0, 0, 0, 0};
    for (long long t = t0; t < (long long)nbend * a.P; t += stride) {
        const int ib = (int)(t / a.P);
        const int a1 = bj[4 * ib], a2 = bj[4 * ib + 1], a3 = bj[4 * ib + 2], ty = bj[4 * ib + 3];
        BendTerm g;
        bend_term(a.posT, a.P, a1, a2, a3, b, bc + 7 * ty, bs + 7 * ty, bdc + 7 * ty, bds + 7 * ty, g);
        v += g.v;
        add_f(a.forceT, a.P, a1, b, g.fx1, g.fy1, g.fz1);
        add_f(a.forceT, a.P, a2, b, -(g.fx1 + g.fx3), -(g.fy1 + g.fy3), -(g.fz1 + g.fz3));
        add_f(a.forceT, a.P, a3, b, g.fx3, g.fy3, g.fz3);
        p[0] += g.dx12 * g.fx1 + g.dx23 * g.fx3;
        p[1] += g.dy12 * g.fy1 + g.dy23 * g.fy3;
        p[2] += g.dz12 * g.fz1 + g.dz23 * g.fz3;
        p[3] += g.dx12 * g.fy1 + g.dx23 * g.fy3;
        p[4] += g.dx12 * g.fz1 + g.dx23 * g.fz3;
        p[5] += g.dy12 * g.fz1 + g.dy23 * g.fz3;
    }
    if (a.energy) {
        const int slot[7] = {S_VBEND, S_PXX, S_PYY, S_PZZ, S_PXY, S_PXZ, S_PYZ};
        const double vals[7] = {v, p[0], p[1], p[2], p[3], p[4], p[5]};
        block_acc<7>(a.acc, a.P, b, slot, vals, sh);
    }
}

__global__ void __launch_bounds__(256) bend_kernel(const __grid_constant__ IntraArgs a, int nbend, const int *__restrict__ bj,
                                                   const double *__restrict__ bc, const double *__restrict__ bs,
                                                   const double *__restrict__ bdc, const double *__restrict__ bds)
{
    bend_body(a, nbend, bj, bc, bs, bdc, bds, hw_blk());
}

__device__ __forceinline__ void ecor_body(const IntraArgs &a, int necor, const int *__restrict__ j1s,
                                                   const int *__restrict__ j2s, int nsplin, double rmin, double dr,
                                                   double dri, const double4 *__restrict__ tab, const VBlk vb)
{
    __shared__ double sh[64 * 7];
    const long long t0 = (long long)vb.x * blockDim.x + threadIdx.x;
    const long long stride = (long long)vb.gx * blockDim.x;  // a multiple of P
    const int b = (int)(t0 % a.P);
    double v = 0, p[6] = {0, 0, 0, 0, 0, 0};
    for (long long t = t0; t < (long long)necor * a.P; t += stride) {
        const int ie = (int)(t / a.P);
        const int j1 = j1s[ie], j2 = j2s[ie];
        double x1, y1, z1, x2, y2, z2;
        load_x(a.posT, a.P, j1, b, x1, y1, z1);
        load_x(a.posT, a.P, j2, b, x2, y2, z2);
        const double dx = x1 - x2, dy = y1 - y2, dz = z1 - z2;
        const double r = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
        int k = __double2int_rz(__dadd_rn(__dmul_rn(__dsub_rn(r, rmin), dri), 0.5)) + 3;
        k = k < nsplin - 2 ? k : nsplin - 2;
        k = k > 3 ? k : 3;
        const double rsp = __dadd_rn(__dmul_rn((double)(k - 3), dr), rmin);
        const double del = __dmul_rn(__dsub_rn(r, rsp), dri);
        const double q12 = a.charge[j1] * a.charge[j2];
        v += spline_eval<double4, double>(tab[k - 1], del) * q12;
        const double dvt = spline_eval<double4, double>(tab[nsplin + k - 1], del) * q12;
        const double fx = dx * dvt, fy = dy * dvt, fz = dz * dvt;
        add_f(a.forceT, a.P, j1, b, fx, fy, fz);
        add_f(a.forceT, a.P, j2, b, -fx, -fy, -fz);
        p[0] += dx * fx; p[1] += dy * fy; p[2] += dz * fz; p[3] += dx * fy; p[4] += dx * fz; p[5] += dy * fz;
    }
    if (a.energy) {
        const int slot[7] = {S_VECOR, S_PXX, S_PYY, S_PZZ, S_PXY, S_PXZ, S_PYZ};
        const double vals[7] = {v, p[0], p[1], p[2], p[3], p[4], p[5]};
        block_acc<7>(a.acc, a.P, b, slot, vals, sh);
    }
}

__global__ void __launch_bounds__(256) ecor_kernel(const __grid_constant__ IntraArgs a, int necor, const int *__restrict__ j1s,
                                                   const int *__restrict__ j2s, int nsplin, double rmin, double dr,
                                                   double dri, const double4 *__restrict__ tab)
{
    ecor_body(a, necor, j1s, j2s, nsplin, rmin, dr, dri, tab, hw_blk());
}

// ---- RESPA: weighted intramolecular forces, no energies -------------------
// Bonds at an inter level (bond_both.c:270-420): the full series at eq and
// the RESPA series at eq_res, combined as w_res F_res + w_both (F - F_res).
// At an intra-only level (bond.c:113-118, :270-278): one series, at eq_res
// when use_res, times w_res.
__global__ void __launch_bounds__(256) bond_w_kernel(int P, const double *__restrict__ posT, double *__restrict__ fW,
                                                     int nbond, const int *__restrict__ bj,
                                                     const double *__restrict__ eq, const double *__restrict__ eq_res,
                                                     const double *__restrict__ dc, int both, int use_res,
                                                     double w_res, double w_both)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nbond * P) return;
    const int ib = (int)(t / P), b = (int)(t % P);
    const int j1 = bj[3 * ib], j2 = bj[3 * ib + 1], ty = bj[3 * ib + 2];
    double x1, y1, z1, x2, y2, z2;
    load_x(posT, P, j1, b, x1, y1, z1);
    load_x(posT, P, j2, b, x2, y2, z2);
    const double dx = x1 - x2, dy = y1 - y2, dz = z1 - z2;
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    const double *d = dc + 7 * ty;
    double fx, fy, fz;
    if (both) {
        const double rr0 = r - eq[ty], rr0r = r - eq_res[ty];
        const double dv = ((((d[6] * rr0 + d[5]) * rr0 + d[4]) * rr0 + d[3]) * rr0 + d[2]) * rr0 + d[1];
        const double dvr = ((((d[6] * rr0r + d[5]) * rr0r + d[4]) * rr0r + d[3]) * rr0r + d[2]) * rr0r + d[1];
        const double pre = -dv / r, prer = -dvr / r;
        const double f1x = dx * pre, f1y = dy * pre, f1z = dz * pre;
        const double f2x = dx * prer, f2y = dy * prer, f2z = dz * prer;
        fx = w_res * f2x + w_both * (f1x - f2x);
        fy = w_res * f2y + w_both * (f1y - f2y);
        fz = w_res * f2z + w_both * (f1z - f2z);
    } else {
        const double rr0 = r - (use_res ? eq_res[ty] : eq[ty]);
        const double dv = ((((d[6] * rr0 + d[5]) * rr0 + d[4]) * rr0 + d[3]) * rr0 + d[2]) * rr0 + d[1];
        const double pre = -dv / r;
        fx = dx * pre * w_res;
        fy = dy * pre * w_res;
        fz = dz * pre * w_res;
    }
    add_f(fW, P, j1, b, fx, fy, fz);
    add_f(fW, P, j2, b, -fx, -fy, -fz);
}

// Bends x w (bend.c:144, :380-393).
__global__ void __launch_bounds__(256) bend_w_kernel(int P, const double *__restrict__ posT, double *__restrict__ fW,
                                                     int nbend, const int *__restrict__ bj,
                                                     const double *__restrict__ bc, const double *__restrict__ bs,
                                                     const double *__restrict__ bdc, const double *__restrict__ bds,
                                                     double w)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nbend * P) return;
    const int ib = (int)(t / P), b = (int)(t % P);
    const int a1 = bj[4 * ib], a2 = bj[4 * ib + 1], a3 = bj[4 * ib + 2], ty = bj[4 * ib + 3];
    BendTerm g;
    bend_term(posT, P, a1, a2, a3, b, bc + 7 * ty, bs + 7 * ty, bdc + 7 * ty, bds + 7 * ty, g);
    const double fx2 = -(g.fx1 + g.fx3), fy2 = -(g.fy1 + g.fy3), fz2 = -(g.fz1 + g.fz3);
    add_f(fW, P, a1, b, g.fx1 * w, g.fy1 * w, g.fz1 * w);
    add_f(fW, P, a2, b, fx2 * w, fy2 * w, fz2 * w);
    add_f(fW, P, a3, b, g.fx3 * w, g.fy3 * w, g.fz3 * w);
}

// Ewald exclusion correction (ecorr.c): table 0, the force table x w
// (:100, :229-245); 1, the RESPA table x w (:103-106); 2, ecor_both's
// w F + (w_res - w) F_res with w_res = wght_ter_res (:349-351, :497-505).
__global__ void __launch_bounds__(256) ecor_w_kernel(int P, const double *__restrict__ posT, double *__restrict__ fW,
                                                     const double *__restrict__ charge, int necor,
                                                     const int *__restrict__ j1s, const int *__restrict__ j2s,
                                                     int nsplin, double rmin, double dr, double dri,
                                                     const double4 *__restrict__ tab,
                                                     const double4 *__restrict__ tab_res, int table, double w,
                                                     double w_res)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)necor * P) return;
    const int ie = (int)(t / P), b = (int)(t % P);
    const int j1 = j1s[ie], j2 = j2s[ie];
    double x1, y1, z1, x2, y2, z2;
    load_x(posT, P, j1, b, x1, y1, z1);
    load_x(posT, P, j2, b, x2, y2, z2);
    const double dx = x1 - x2, dy = y1 - y2, dz = z1 - z2;
    const double r = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    int k = __double2int_rz(__dadd_rn(__dmul_rn(__dsub_rn(r, rmin), dri), 0.5)) + 3;
    k = k < nsplin - 2 ? k : nsplin - 2;
    k = k > 3 ? k : 3;
    const double rsp = __dadd_rn(__dmul_rn((double)(k - 3), dr), rmin);
    const double del = __dmul_rn(__dsub_rn(r, rsp), dri);
    const double q12 = charge[j1] * charge[j2];
    double fx, fy, fz;
    if (table == 0 || table == 1) {
        const double dvt = spline_eval<double4, double>(table == 0 ? tab[nsplin + k - 1] : tab_res[k - 1], del) * q12;
        fx = dx * dvt * w;
        fy = dy * dvt * w;
        fz = dz * dvt * w;
    } else {
        const double dvt = spline_eval<double4, double>(tab[nsplin + k - 1], del) * q12;
        const double dvr = spline_eval<double4, double>(tab_res[k - 1], del) * q12;
        const double wd = w_res - w;
        fx = w * (dx * dvt) + wd * (dx * dvr);
        fy = w * (dy * dvt) + wd * (dy * dvr);
        fz = w * (dz * dvt) + wd * (dz * dvr);
    }
    add_f(fW, P, j1, b, fx, fy, fz);
    add_f(fW, P, j2, b, -fx, -fy, -fz);
}

static inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// grid-stride launch size for the intramolecular kernels
static inline unsigned nblk_gs(pinyb200_ctx *c, long long n)
{
    long long b = (n + 255) / 256, cap = (long long)c->sm_count * 4;
    return (unsigned)(b < cap ? (b > 0 ? b : 1) : cap);
}

cudaError_t launch_transpose_in(pinyb200_ctx *c, const double *d_aos)
{
    const long long M = (long long)c->sys.natm * 3;
    const dim3 grid((unsigned)((M + 31) / 32), (unsigned)((c->P + 31) / 32));
    transpose_tiled_kernel<<<grid, 256, 0, c->stream>>>(d_aos, c->d_posT, c->P, M);
    return cudaGetLastError();
}

cudaError_t launch_transpose_out(pinyb200_ctx *c, double *d_aos, const double *fT)
{
    const long long M = (long long)c->sys.natm * 3;
    const dim3 grid((unsigned)((c->P + 31) / 32), (unsigned)std::min<long long>((M + 31) / 32, 65535));
    transpose_tiled_kernel<<<grid, 256, 0, c->stream>>>(fT ? fT : c->d_forceT, d_aos, (int)M, c->P);
    return cudaGetLastError();
}

cudaError_t launch_ghost_pos(pinyb200_ctx *c)
{
    const DeviceSystem &s = c->sys;
    if (s.nghost == 0) return cudaSuccess;
    ghost_pos_kernel<<<nblk((long long)s.nghost * c->P, 256), 256, 0, c->stream>>>(
        c->d_posT, c->P, s.nghost, s.ghost_ncomp, s.ghost_atom, s.ghost_comp, s.ghost_coef);
    return cudaGetLastError();
}

cudaError_t launch_ghost_distrib(pinyb200_ctx *c, double *fT)
{
    const DeviceSystem &s = c->sys;
    if (s.nghost == 0) return cudaSuccess;
    ghost_distrib_kernel<<<nblk((long long)s.nghost * c->P, 256), 256, 0, c->stream>>>(
        fT ? fT : c->d_forceT, c->P, s.nghost, s.ghost_ncomp, s.ghost_atom, s.ghost_comp, s.ghost_coef);
    return cudaGetLastError();
}

cudaError_t launch_intra(pinyb200_ctx *c, const Cell &cell, bool energy)
{
    (void)cell;
    const DeviceSystem &s = c->sys;
    IntraArgs a;
    a.natm = s.natm;
    a.P = c->P;
    a.posT = c->d_posT;
    a.forceT = c->d_forceT;
    a.acc = c->d_acc;
    a.charge = s.charge;
    a.energy = energy ? 1 : 0;
    if (s.nbond)
        bond_kernel<<<nblk_gs(c, (long long)s.nbond * c->P), 256, 0, c->stream>>>(a, s.nbond, s.bond_j, s.bond_eq,
                                                                                  s.bond_c, s.bond_dc);
    if (s.nbend)
        bend_kernel<<<nblk_gs(c, (long long)s.nbend * c->P), 256, 0, c->stream>>>(a, s.nbend, s.bend_j, s.bend_c,
                                                                                  s.bend_s, s.bend_dc, s.bend_ds);
    if (s.necor)
        ecor_kernel<<<nblk_gs(c, (long long)s.necor * c->P), 256, 0, c->stream>>>(
            a, s.necor, s.ecor_j1, s.ecor_j2, s.ecor_nsplin, s.ecor_rmin, s.ecor_dr, s.ecor_dri, s.ecor_tab);
    return cudaGetLastError();
}

// Weighted bonds and bends of one RESPA level into target: bond_both's
// combination when both (inter levels), else bond() with PINY's ires_bond
// choice of equilibrium; bends x wght_tra_res.
cudaError_t launch_intra_respa(pinyb200_ctx *c, bool both, double *target)
{
    const DeviceSystem &s = c->sys;
    const double w_both = c->r_int_res_inter ? c->r_wter_res : c->r_wter;  // bond_both.c:156-161
    if (s.nbond)
        bond_w_kernel<<<nblk((long long)s.nbond * c->P, 256), 256, 0, c->stream>>>(
            c->P, c->d_posT, target, s.nbond, s.bond_j, s.bond_eq, c->d_bond_eq_res, s.bond_dc, both ? 1 : 0,
            c->r_ires_bond, c->r_wtra_res, w_both);
    if (s.nbend)
        bend_w_kernel<<<nblk((long long)s.nbend * c->P, 256), 256, 0, c->stream>>>(
            c->P, c->d_posT, target, s.nbend, s.bend_j, s.bend_c, s.bend_s, s.bend_dc, s.bend_ds, c->r_wtra_res);
    return cudaGetLastError();
}

cudaError_t launch_ecor_weighted(pinyb200_ctx *c, double w, double *target, int table)
{
    const DeviceSystem &s = c->sys;
    if (!s.necor) return cudaSuccess;
    ecor_w_kernel<<<nblk((long long)s.necor * c->P, 256), 256, 0, c->stream>>>(
        c->P, c->d_posT, target, s.charge, s.necor, s.ecor_j1, s.ecor_j2, s.ecor_nsplin, s.ecor_rmin, s.ecor_dr,
        s.ecor_dri, s.ecor_tab, (const double4 *)c->d_ecor_res_tab, table, w, c->r_wter_res);
    return cudaGetLastError();
}


// ---------------------------------------------------------------------------
// Many boxes per launch (the batched evaluation): staging, intramolecular
// terms and the finishing steps of every box in a few persistent launches.

struct ZeroBox {
    unsigned *p;
    long long n;  // 4-byte words
};

// 1024 words per block, 16-byte stores where the range allows
__device__ __forceinline__ void zero_body(unsigned *p, long long n, const VBlk vb)
{
    const long long w = ((long long)vb.x * blockDim.x + threadIdx.x) * 4;
    if (w >= n) return;
    if (w + 4 <= n && (((uintptr_t)(p + w)) & 15) == 0) {
        *(uint4 *)(p + w) = make_uint4(0u, 0u, 0u, 0u);
    } else {
        for (long long k = w; k < n && k < w + 4; k++) p[k] = 0u;
    }
}

__global__ void __launch_bounds__(256) zero_batch_kernel(const __grid_constant__ BoxTab<ZeroBox> t)
{
    PINYB200_BOX_LOOP(t, i, vb, (zero_body(t.arg[i].p, t.arg[i].n, vb)));
}

__global__ void __launch_bounds__(256) copy_batch_kernel(const __grid_constant__ BoxTab<CopySeg> t)
{
    PINYB200_BOX_LOOP(t, i, vb, {
        const CopySeg &c = t.arg[i];
        const long long k = (long long)vb.x * blockDim.x + threadIdx.x;
        if (k < c.n) {
            if (c.src) {
                c.dst[k] = c.src[k];
            } else {
                double v = 0.0;
                for (int b = 0; b < c.P; b++) v += c.posT[k * c.P + b];
                c.dst[k] = v / (double)c.P;
            }
        }
    });
}

struct TrBox {
    const double *in;
    double *out;
    int rows;
    long long cols;
};

__global__ void __launch_bounds__(256) transpose_batch_kernel(const __grid_constant__ BoxTab<TrBox> t)
{
    PINYB200_BOX_LOOP(t, i, vb, (transpose_tiled_body(t.arg[i].in, t.arg[i].out, t.arg[i].rows, t.arg[i].cols, vb)));
}

struct GhostBox {
    double *x;  // positions (placement) or forces (distribution)
    int P, nghost, ncomp;
    const int *gatom, *gcomp;
    const double *gcoef;
};

template <bool DISTRIB>
__global__ void __launch_bounds__(256) ghost_batch_kernel(const __grid_constant__ BoxTab<GhostBox> t)
{
    PINYB200_BOX_LOOP(t, i, vb, {
        const GhostBox &g = t.arg[i];
        if (DISTRIB) ghost_distrib_body(g.x, g.P, g.nghost, g.ncomp, g.gatom, g.gcomp, g.gcoef, vb);
        else ghost_pos_body(g.x, g.P, g.nghost, g.ncomp, g.gatom, g.gcomp, g.gcoef, vb);
    });
}

// One intramolecular term of one box: kind 0 bonds, 1 bends, 2 excluded-pair
// correction; the three kinds of every box share one launch (a typed work list).
struct IntraBox {
    IntraArgs a;
    int kind, n;
    const int *j1, *j2;
    const double *c0, *c1, *c2, *c3;
    int nsplin;
    double rmin, dr, dri;
    const double4 *tab;
};

__global__ void __launch_bounds__(256) intra_batch_kernel(const __grid_constant__ BoxTab<IntraBox> t)
{
    PINYB200_BOX_LOOP(t, i, vb, {
        const IntraBox &x = t.arg[i];
        if (x.kind == 0) bond_body(x.a, x.n, x.j1, x.c0, x.c1, x.c2, vb);
        else if (x.kind == 1) bend_body(x.a, x.n, x.j1, x.c0, x.c1, x.c2, x.c3, vb);
        else ecor_body(x.a, x.n, x.j1, x.j2, x.nsplin, x.rmin, x.dr, x.dri, x.tab, vb);
    });
}

cudaError_t launch_zero_batch(const std::vector<std::pair<void *, size_t>> &seg, int sm_count, cudaStream_t st)
{
    BoxTabBuilder<ZeroBox> tb;
    for (const auto &z : seg) {
        const long long n = (long long)(z.second / 4);
        tb.add(ZeroBox{(unsigned *)z.first, n}, (int)((n + 1023) / 1024), 1, (double)n);
    }
    return launch_tables(tb, (const void *)zero_batch_kernel, 256, 0, sm_count,
                         [&](const BoxTab<ZeroBox> &t, int g) { zero_batch_kernel<<<g, 256, 0, st>>>(t); });
}

cudaError_t launch_copy_batch(const std::vector<CopySeg> &seg, int sm_count, cudaStream_t st)
{
    BoxTabBuilder<CopySeg> tb;
    for (const CopySeg &c : seg) tb.add(c, (int)((c.n + 255) / 256), 1, (double)c.n * (c.src ? 1 : c.P));
    return launch_tables(tb, (const void *)copy_batch_kernel, 256, 0, sm_count,
                         [&](const BoxTab<CopySeg> &t, int g) { copy_batch_kernel<<<g, 256, 0, st>>>(t); });
}

// Positions of every box into its [atom][xyz][bead] layout (from d_pos[i],
// PINY's [bead][atom][xyz]).
cudaError_t launch_transpose_in_batch(const std::vector<pinyb200_ctx *> &box, const std::vector<const double *> &d_pos,
                                      int sm_count, cudaStream_t st)
{
    BoxTabBuilder<TrBox> tb;
    for (size_t i = 0; i < box.size(); i++) {
        pinyb200_ctx *c = box[i];
        const long long M = (long long)c->sys.natm * 3;
        tb.add(TrBox{d_pos[i], c->d_posT, c->P, M}, (int)((M + 31) / 32), (c->P + 31) / 32, (double)M * c->P);
    }
    return launch_tables(tb, (const void *)transpose_batch_kernel, 256, 0, sm_count,
                         [&](const BoxTab<TrBox> &t, int g) { transpose_batch_kernel<<<g, 256, 0, st>>>(t); });
}

// Site forces of every box out to d_force[i] in PINY's order.
cudaError_t launch_transpose_out_batch(const std::vector<pinyb200_ctx *> &box, const std::vector<double *> &d_force,
                                       int sm_count, cudaStream_t st)
{
    BoxTabBuilder<TrBox> tb;
    for (size_t i = 0; i < box.size(); i++) {
        pinyb200_ctx *c = box[i];
        const long long M = (long long)c->sys.natm * 3;
        tb.add(TrBox{c->d_forceT, d_force[i], (int)M, c->P}, (c->P + 31) / 32,
               (int)std::min<long long>((M + 31) / 32, 65535), (double)M * c->P);
    }
    return launch_tables(tb, (const void *)transpose_batch_kernel, 256, 0, sm_count,
                         [&](const BoxTab<TrBox> &t, int g) { transpose_batch_kernel<<<g, 256, 0, st>>>(t); });
}

cudaError_t launch_ghost_batch(const std::vector<pinyb200_ctx *> &box, bool distrib, int sm_count, cudaStream_t st)
{
    BoxTabBuilder<GhostBox> tb;
    for (pinyb200_ctx *c : box) {
        const DeviceSystem &s = c->sys;
        if (s.nghost == 0) continue;
        const long long n = (long long)s.nghost * c->P;
        tb.add(GhostBox{distrib ? c->d_forceT : c->d_posT, c->P, s.nghost, s.ghost_ncomp, s.ghost_atom, s.ghost_comp,
                        s.ghost_coef},
               (int)((n + 255) / 256), 1, (double)n);
    }
    if (distrib)
        return launch_tables(tb, (const void *)ghost_batch_kernel<true>, 256, 0, sm_count,
                             [&](const BoxTab<GhostBox> &t, int g) { ghost_batch_kernel<true><<<g, 256, 0, st>>>(t); });
    return launch_tables(tb, (const void *)ghost_batch_kernel<false>, 256, 0, sm_count,
                         [&](const BoxTab<GhostBox> &t, int g) { ghost_batch_kernel<false><<<g, 256, 0, st>>>(t); });
}

// Bonds, bends and excluded-pair corrections of every box in one launch.
cudaError_t launch_intra_batch(const std::vector<pinyb200_ctx *> &box, bool energy, int sm_count, cudaStream_t st)
{
    BoxTabBuilder<IntraBox> tb;
    for (pinyb200_ctx *c : box) {
        const DeviceSystem &s = c->sys;
        IntraBox x;
        memset(&x, 0, sizeof(x));
        x.a.natm = s.natm;
        x.a.P = c->P;
        x.a.posT = c->d_posT;
        x.a.forceT = c->d_forceT;
        x.a.acc = c->d_acc;
        x.a.charge = s.charge;
        x.a.energy = energy ? 1 : 0;
        if (s.nbond) {
            IntraBox b = x;
            b.kind = 0;
            b.n = s.nbond;
            b.j1 = s.bond_j;
            b.c0 = s.bond_eq;
            b.c1 = s.bond_c;
            b.c2 = s.bond_dc;
            tb.add(b, (int)nblk_gs(c, (long long)s.nbond * c->P), 1, (double)s.nbond * c->P);
        }
        if (s.nbend) {
            IntraBox b = x;
            b.kind = 1;
            b.n = s.nbend;
            b.j1 = s.bend_j;
            b.c0 = s.bend_c;
            b.c1 = s.bend_s;
            b.c2 = s.bend_dc;
            b.c3 = s.bend_ds;
            tb.add(b, (int)nblk_gs(c, (long long)s.nbend * c->P), 1, 2.0 * s.nbend * c->P);
        }
        if (s.necor) {
            IntraBox b = x;
            b.kind = 2;
            b.n = s.necor;
            b.j1 = s.ecor_j1;
            b.j2 = s.ecor_j2;
            b.nsplin = s.ecor_nsplin;
            b.rmin = s.ecor_rmin;
            b.dr = s.ecor_dr;
            b.dri = s.ecor_dri;
            b.tab = s.ecor_tab;
            tb.add(b, (int)nblk_gs(c, (long long)s.necor * c->P), 1, (double)s.necor * c->P);
        }
    }
    return launch_tables(tb, (const void *)intra_batch_kernel, 256, 0, sm_count,
                         [&](const BoxTab<IntraBox> &t, int g) { intra_batch_kernel<<<g, 256, 0, st>>>(t); });
}

}  // namespace pinyb200
