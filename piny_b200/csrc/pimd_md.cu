// Path-integral MD bookkeeping around the force call, on the device, FP64:
// PINY's NVT ring-polymer step (int_NVT_pimd), RESPA loops included.
//
// Per step with every RESPA count 1 (src/integrate/pimd/int_NVT_pimd.c:142-217):
//   chains, half kick            int_0_to_dt2_nvt_pimd (int_0_to_dt2_pimd.c:34-190)
//   positions -> modes, drift    control_pimd_trans_mode, x += v dt
//   springs on the modes         mode_energy_control (pimd_estimators.c:31-110)
//   mode 1 -> xmod, modes -> positions, ghost positions
//                                control_pimd_trans_pos (control_pimd_trans.c:146-250)
//   list test and rebuild        check_ver_list / verlist_control, on the device
//   force path, post-processing  energy_control_pimd.c:113-218: forces / P,
//                                centroid virial correction (pimd_pvten_forc_corr,
//                                pimd_estimators.c:223-305), forces -> modes,
//                                spring forces added
//   half kick, chains            int_dt2_to_dt_nvt_pimd (int_dt2_to_dt_pimd.c)
// The chain operator is apply_NHC_par (src/integrate/md/int_NVT.c:144-353):
// one thread per chain runs the RESPA x Yoshida-Suzuki loop; the kinetic
// energy of each chain is summed with FP64 atomics and the velocities are
// scaled afterwards.  With RESPA counts above 1 these are the inner steps of
// int_NVT_pimd's four nested loops (step_enqueue).  Layouts: bead arrays
// [P][natm][3]; chain state [beads of the set][len_nhc][num_nhc].
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace {

constexpr int kMaxLen = 8;   // links per chain
constexpr int kMaxYosh = 9;  // Yoshida-Suzuki stages

// accumulator slots (doubles)
enum Acc {
    A_KIN = 0,     // spring energy
    A_PVM = 1,     // spring tensor xx yy zz xy xz yz (6)
    A_VIR = 7,     // sum of d . f (virial estimator)
    A_PVC = 8,     // sum of d (x) f, 9 components row-major
    A_N = 17
};

struct NhcDev {
    int num = 0, len = 0, nres = 0, nyosh = 0, nb = 0;
    double w[kMaxYosh] = {0};
    int *inhc = nullptr;
    double *mass = nullptr, *gkt = nullptr;  // [len][num]
    double *x = nullptr, *v = nullptr;       // [nb][len][num]
    double *kin = nullptr, *sc = nullptr;    // [nb][num + 1]
    int *coord = nullptr;  // massive sets (one coordinate per chain): chain -> 3 i + d
};

struct ChainArgs {
    int num, len, nres, nyosh, nb;
    double w[kMaxYosh];
    const double *mass, *gkt;
    double *x, *v, *kin, *sc;
};

__global__ void nhc_kin_kernel(const double *__restrict__ v, int nb, int natm, const double *__restrict__ m,
                               size_t m_stride, const int *__restrict__ inhc, double *__restrict__ kin, int num)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n3 = (long long)natm * 3;
    if (t >= n3 * nb) return;
    const int b = (int)(t / n3);
    const int r = (int)(t - (long long)b * n3);
    const int i = r / 3, d = r - 3 * (r / 3);
    const double vv = v[t];
    const double e = __dmul_rn(__dmul_rn(m[(size_t)b * m_stride + i], vv), vv);
    atomicAdd(&kin[(size_t)b * (num + 1) + inhc[d * natm + i]], e);
}

// The chain operator of one chain (apply_NHC_par, int_NVT.c:144-353)
// on the chain's kinetic energy kin: updates the chain's x and v and returns
// the velocity scale.  LEN links known at compile time, so the chain stays
// in registers.
template <int LEN>
__device__ __forceinline__ double chain_run(const ChainArgs &a, int b, int k, double kin)
{
    const int num = a.num;
    constexpr int L = LEN - 1;
    double *x = a.x + (size_t)b * LEN * num + k;
    double *v = a.v + (size_t)b * LEN * num + k;
    double vn[LEN], f[LEN], ms[LEN], gk[LEN], xs[LEN];
#pragma unroll
    for (int c = 0; c <= L; c++) {
        vn[c] = v[(size_t)c * num];
        xs[c] = x[(size_t)c * num];
        ms[c] = a.mass[(size_t)c * num + k];
        gk[c] = a.gkt[(size_t)c * num + k];
    }
    double sc = 1.0;
    f[0] = (kin - gk[0]) / ms[0];
#pragma unroll
    for (int c = 0; c < L; c++) f[c + 1] = (ms[c] * vn[c] * vn[c] - gk[c + 1]) / ms[c + 1];
    for (int r = 0; r < a.nres; r++)
        for (int y = 0; y < a.nyosh; y++) {
            const double w2 = a.w[y] / 2.0, w4 = a.w[y] / 4.0, w8 = a.w[y] / 8.0;
            vn[L] += f[L] * w4;
            // the upward sweep needs exp(-w8 v[c+1]) of the same v[c+1] as
            // the downward one (nothing changes it in between): keep them
            double ex[LEN];
#pragma unroll
            for (int c = L - 1; c >= 0; c--) {
                const double aa = exp(-w8 * vn[c + 1]);
                ex[c] = aa;
                vn[c] = vn[c] * aa * aa + w4 * f[c] * aa;
            }
            const double aa = exp(-w2 * vn[0]);
            sc *= aa;
            kin *= aa * aa;
#pragma unroll
            for (int c = 0; c <= L; c++) xs[c] += vn[c] * w2;
            f[0] = (kin - gk[0]) / ms[0];
#pragma unroll
            for (int c = 0; c < L; c++) {
                const double ab = ex[c];
                vn[c] = vn[c] * ab * ab + w4 * f[c] * ab;
                f[c + 1] = (ms[c] * vn[c] * vn[c] - gk[c + 1]) / ms[c + 1];
            }
            vn[L] += f[L] * w4;
        }
#pragma unroll
    for (int c = 0; c <= L; c++) {
        x[(size_t)c * num] = xs[c];
        v[(size_t)c * num] = vn[c];
    }
    return sc;
}

// One thread per chain, kinetic energies summed beforehand (nhc_kin_kernel).
template <int LEN>
__global__ void __launch_bounds__(128, 6) nhc_chain_kernel(ChainArgs a)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)a.nb * a.num) return;
    const int b = (int)(t / a.num), k = (int)(t - (long long)b * a.num);
    const double sc = chain_run<LEN>(a, b, k, a.kin[(size_t)b * (a.num + 1) + k]);
    a.sc[(size_t)b * (a.num + 1) + k] = sc;
    if (k == 0) a.sc[(size_t)b * (a.num + 1) + a.num] = 1.0;  // null chain
}

// Massive sets (every chain thermostats one coordinate, as PINY's bead and
// option-6 class thermostats): kinetic energy, chain and velocity scaling in
// one thread per chain, with the operations of the three-kernel path (the
// kinetic energy m v v of the one coordinate, v x scale).
template <int LEN>
__global__ void __launch_bounds__(128, 6) nhc_massive_kernel(ChainArgs a, double *__restrict__ v0, int natm,
                                                             const double *__restrict__ m, size_t m_stride,
                                                             const int *__restrict__ coord)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)a.nb * a.num) return;
    const int b = (int)(t / a.num), k = (int)(t - (long long)b * a.num);
    const int r = coord[k];
    double *vp = v0 + (size_t)b * natm * 3 + r;
    const double vv = *vp;
    const double kin = __dmul_rn(__dmul_rn(m[(size_t)b * m_stride + r / 3], vv), vv);
    const double sc = chain_run<LEN>(a, b, k, kin);
    *vp = vv * sc;
}

__global__ void nhc_scale_kernel(double *__restrict__ v, int nb, int natm, const int *__restrict__ inhc,
                                 const double *__restrict__ sc, int num)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n3 = (long long)natm * 3;
    if (t >= n3 * nb) return;
    const int b = (int)(t / n3);
    const int r = (int)(t - (long long)b * n3);
    const int i = r / 3, d = r - 3 * (r / 3);
    v[t] *= sc[(size_t)b * (num + 1) + inhc[d * natm + i]];
}

// v += f dt2 / m_bead
__global__ void kick_kernel(double *__restrict__ v, const double *__restrict__ f, const double *__restrict__ bm,
                            long long n, double dt2)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const long long bi = t / 3;  // b * natm + i
    v[t] = __dadd_rn(v[t], __ddiv_rn(__dmul_rn(f[t], dt2), bm[bi]));
}

// x += v dt
__global__ void drift_kernel(double *__restrict__ x, const double *__restrict__ v, long long n, double dt)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    x[t] = __dadd_rn(x[t], __dmul_rn(v[t], dt));
}

__global__ void add_kernel(double *__restrict__ f, const double *__restrict__ g, long long n)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    f[t] = __dadd_rn(f[t], g[t]);
}

// Block sum of NV values per thread into acc[0..NV) with FP64 atomics.
template <int NV>
__device__ __forceinline__ void block_accumulate(double (&val)[NV], double *acc)
{
    __shared__ double red[NV][8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; q++) {
        double s = val[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) red[q][wid] = s;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[threadIdx.x][w];
        atomicAdd(acc + threadIdx.x, s);
    }
}

// Spring forces on the modes and their energy and tensor (mode_energy_control).
__global__ void __launch_bounds__(256) springs_kernel(const double *__restrict__ u, const double *__restrict__ prekf,
                                                      const double *__restrict__ veig, double wght, int natm, int P,
                                                      double *__restrict__ fm, double *__restrict__ acc)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double val[7] = {0, 0, 0, 0, 0, 0, 0};
    if (t < (long long)natm * P) {
        const int b = (int)(t / natm), i = (int)(t - (long long)b * natm);
        const double *p = u + 3 * t;
        const double fk = __dmul_rn(prekf[i], veig[b]);
        const double x = p[0], y = p[1], z = p[2];
        val[0] = __dmul_rn(fk, __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
        const double g = -2.0 * fk;
        const double gx = __dmul_rn(g, x), gy = __dmul_rn(g, y), gz = __dmul_rn(g, z);
        val[1] = __dmul_rn(x, gx);
        val[2] = __dmul_rn(y, gy);
        val[3] = __dmul_rn(z, gz);
        val[4] = __dmul_rn(x, gy);
        val[5] = __dmul_rn(x, gz);
        val[6] = __dmul_rn(y, gz);
        double *q = fm + 3 * t;
        q[0] = __dmul_rn(gx, wght);
        q[1] = __dmul_rn(gy, wght);
        q[2] = __dmul_rn(gz, wght);
    }
    block_accumulate<7>(val, acc + A_KIN);
}

// Bead forces / P and the centroid virial sums (d = x - xmod).
__global__ void __launch_bounds__(256) post_kernel(double *__restrict__ f, const double *__restrict__ x,
                                                   const double *__restrict__ xmod, int natm, int P, int correct,
                                                   double *__restrict__ acc)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double val[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (t < (long long)natm * P) {
        const int i = (int)(t % natm);
        double *g = f + 3 * t;
        const double dP = (double)P;
        const double g0 = __ddiv_rn(g[0], dP), g1 = __ddiv_rn(g[1], dP), g2 = __ddiv_rn(g[2], dP);
        g[0] = g0;
        g[1] = g1;
        g[2] = g2;
        if (correct) {
            const double *p = x + 3 * t;
            const double d0 = __dsub_rn(p[0], xmod[3 * i]), d1 = __dsub_rn(p[1], xmod[3 * i + 1]),
                         d2 = __dsub_rn(p[2], xmod[3 * i + 2]);
            val[0] = __dadd_rn(__dadd_rn(__dmul_rn(d0, g0), __dmul_rn(d1, g1)), __dmul_rn(d2, g2));
            val[1] = __dmul_rn(d0, g0);
            val[2] = __dmul_rn(d0, g1);
            val[3] = __dmul_rn(d0, g2);
            val[4] = __dmul_rn(d1, g0);
            val[5] = __dmul_rn(d1, g1);
            val[6] = __dmul_rn(d1, g2);
            val[7] = __dmul_rn(d2, g0);
            val[8] = __dmul_rn(d2, g1);
            val[9] = __dmul_rn(d2, g2);
        }
    }
    block_accumulate<10>(val, acc + A_VIR);
}

// Ghost positions from their components (get_ghost_pos) in the [P][natm][3]
// layout, with the force path's operation order.
__global__ void ghost_pos_aos_kernel(double *__restrict__ x, int natm, int P, int nghost, int ncomp,
                                     const int *__restrict__ gatom, const int *__restrict__ gcomp,
                                     const double *__restrict__ gcoef)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nghost * P) return;
    const int b = (int)(t / nghost), g = (int)(t - (long long)b * nghost);
    double *xb = x + (size_t)b * natm * 3;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        double v = 0.0;
        for (int c = 0; c < ncomp; c++) {
            const int at = gcomp[g * ncomp + c];
            if (at < 0) continue;
            v = __dadd_rn(v, __dmul_rn(gcoef[g * ncomp + c], xb[3 * (size_t)at + d]));
        }
        xb[3 * (size_t)gatom[g] + d] = v;
    }
}

inline unsigned blocks_for(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

struct pinyb200_pimd {
    int device = 0;
    int natm = 0, P = 1, kind = PINYB200_STAGING;
    double wght = 1.0, dt = 0.0, beta = 1.0;
    int nfree = 0;
    double *d_mass = nullptr, *d_bmass = nullptr, *d_prekf = nullptr, *d_veig = nullptr;
    double *d_fm = nullptr, *d_u = nullptr, *d_xmod = nullptr, *d_acc = nullptr;
    double *h_acc = nullptr;
    double *h_facc = nullptr;  // the force path's per-bead sums (pinned)
    NhcDev set[2];
    // the step as a CUDA graph, for the arguments it was captured with
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<double> key;     // pointers, cell, context and its generation
    std::vector<double> eager;   // key of the last eager step (the capture follows it)
    bool graph_mode = false;     // the last step ran as a graph (no per-phase timing)
    int nres[4] = {1, 1, 1, 1};  // RESPA counts: inter, torsion, intra, bead
    int ix_respa = 1;            // chains at the inner steps of loops of level <= ix_respa
    double *d_ft = nullptr;      // [P][natm][3] virial forces of the outer RESPA level
    bool timed = false;          // this call recorded the force path's phase events
    std::string err;
};

namespace {

int pimd_fail(pinyb200_pimd *pm, int code, const std::string &msg)
{
    if (pm) pm->err = msg;
    return pinyb200::record_error(nullptr, code, msg);
}

#define PCK(call)                                                                                     \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) return pimd_fail(pm, PINYB200_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

void free_set(NhcDev &s)
{
    cudaFree(s.inhc);
    cudaFree(s.mass);
    cudaFree(s.gkt);
    cudaFree(s.x);
    cudaFree(s.v);
    cudaFree(s.kin);
    cudaFree(s.sc);
    cudaFree(s.coord);
    s = NhcDev();
}

int upload_set(pinyb200_pimd *pm, NhcDev &s, const pinyb200_nhc_set &h, int nb)
{
    s.nb = nb;
    if (nb == 0 || h.num_nhc == 0) {
        s.num = 0;
        return PINYB200_OK;
    }
    if (h.num_nhc < 0 || h.len_nhc < 1 || h.len_nhc > kMaxLen || h.nres_nhc < 1 || h.nyosh_nhc < 1 ||
        h.nyosh_nhc > kMaxYosh || !h.wdti || !h.inhc || !h.mass_nhc || !h.gkt)
        return pimd_fail(pm, PINYB200_ERR_ARG, "pimd: chain set needs num>=0, len 1..8, nres>=1, nyosh 1..9 and its arrays");
    for (int k = 0; k < 3 * pm->natm; k++)
        if (h.inhc[k] < 0 || h.inhc[k] > h.num_nhc) return pimd_fail(pm, PINYB200_ERR_ARG, "pimd: chain index out of range");
    s.num = h.num_nhc;
    s.len = h.len_nhc;
    s.nres = h.nres_nhc;
    s.nyosh = h.nyosh_nhc;
    for (int y = 0; y < s.nyosh; y++) s.w[y] = h.wdti[y];
    const size_t tab = (size_t)s.len * s.num, st = tab * nb;
    PCK(cudaMalloc(&s.inhc, sizeof(int) * 3 * pm->natm));
    PCK(cudaMalloc(&s.mass, sizeof(double) * tab));
    PCK(cudaMalloc(&s.gkt, sizeof(double) * tab));
    PCK(cudaMalloc(&s.x, sizeof(double) * st));
    PCK(cudaMalloc(&s.v, sizeof(double) * st));
    PCK(cudaMalloc(&s.kin, sizeof(double) * (size_t)nb * (s.num + 1)));
    PCK(cudaMalloc(&s.sc, sizeof(double) * (size_t)nb * (s.num + 1)));
    PCK(cudaMemcpy(s.inhc, h.inhc, sizeof(int) * 3 * pm->natm, cudaMemcpyHostToDevice));
    PCK(cudaMemcpy(s.mass, h.mass_nhc, sizeof(double) * tab, cudaMemcpyHostToDevice));
    PCK(cudaMemcpy(s.gkt, h.gkt, sizeof(double) * tab, cudaMemcpyHostToDevice));
    PCK(cudaMemset(s.x, 0, sizeof(double) * st));
    PCK(cudaMemset(s.v, 0, sizeof(double) * st));
    // one coordinate per chain: the fused chain kernel applies
    std::vector<int> coord(s.num, -1);
    bool massive = true;
    for (int d = 0; d < 3 && massive; d++)
        for (int i = 0; i < pm->natm && massive; i++) {
            const int k = h.inhc[d * pm->natm + i];
            if (k == s.num) continue;  // the null chain
            if (coord[k] >= 0) massive = false;
            else coord[k] = 3 * i + d;
        }
    for (int k = 0; k < s.num && massive; k++) massive = coord[k] >= 0;
    if (massive) {
        PCK(cudaMalloc(&s.coord, sizeof(int) * (size_t)s.num));
        PCK(cudaMemcpy(s.coord, coord.data(), sizeof(int) * (size_t)s.num, cudaMemcpyHostToDevice));
    }
    return PINYB200_OK;
}

// apply_NHC_par on every bead of one set: bead0 is the set's first bead in
// the velocity array; m is the per-bead mass row (stride 0 for atom masses).
int apply_nhc(pinyb200_pimd *pm, NhcDev &s, double *d_v, int bead0, const double *m, size_t m_stride,
              cudaStream_t st)
{
    if (s.num == 0 || s.nb == 0) return PINYB200_OK;
    const long long n = (long long)pm->natm * 3 * s.nb;
    double *v = d_v + (size_t)bead0 * pm->natm * 3;
    if (!s.coord) {
        PCK(cudaMemsetAsync(s.kin, 0, sizeof(double) * (size_t)s.nb * (s.num + 1), st));
        nhc_kin_kernel<<<blocks_for(n, 256), 256, 0, st>>>(v, s.nb, pm->natm, m, m_stride, s.inhc, s.kin, s.num);
    }
    ChainArgs a;
    a.num = s.num;
    a.len = s.len;
    a.nres = s.nres;
    a.nyosh = s.nyosh;
    a.nb = s.nb;
    for (int y = 0; y < kMaxYosh; y++) a.w[y] = s.w[y];
    a.mass = s.mass;
    a.gkt = s.gkt;
    a.x = s.x;
    a.v = s.v;
    a.kin = s.kin;
    a.sc = s.sc;
    const unsigned nbk = blocks_for((long long)s.nb * s.num, 128);
    if (s.coord) {
        switch (s.len) {
        case 1: nhc_massive_kernel<1><<<nbk, 128, 0, st>>>(a, v, pm->natm, m, m_stride, s.coord); break;
        case 2: nhc_massive_kernel<2><<<nbk, 128, 0, st>>>(a, v, pm->natm, m, m_stride, s.coord); break;
        case 3: nhc_massive_kernel<3><<<nbk, 128, 0, st>>>(a, v, pm->natm, m, m_stride, s.coord); break;
        case 4: nhc_massive_kernel<4><<<nbk, 128, 0, st>>>(a, v, pm->natm, m, m_stride, s.coord); break;
        case 5: nhc_massive_kernel<5><<<nbk, 128, 0, st>>>(a, v, pm->natm, m, m_stride, s.coord); break;
        case 6: nhc_massive_kernel<6><<<nbk, 128, 0, st>>>(a, v, pm->natm, m, m_stride, s.coord); break;
        case 7: nhc_massive_kernel<7><<<nbk, 128, 0, st>>>(a, v, pm->natm, m, m_stride, s.coord); break;
        default: nhc_massive_kernel<8><<<nbk, 128, 0, st>>>(a, v, pm->natm, m, m_stride, s.coord); break;
        }
        PCK(cudaGetLastError());
        return PINYB200_OK;
    }
    switch (s.len) {
    case 1: nhc_chain_kernel<1><<<nbk, 128, 0, st>>>(a); break;
    case 2: nhc_chain_kernel<2><<<nbk, 128, 0, st>>>(a); break;
    case 3: nhc_chain_kernel<3><<<nbk, 128, 0, st>>>(a); break;
    case 4: nhc_chain_kernel<4><<<nbk, 128, 0, st>>>(a); break;
    case 5: nhc_chain_kernel<5><<<nbk, 128, 0, st>>>(a); break;
    case 6: nhc_chain_kernel<6><<<nbk, 128, 0, st>>>(a); break;
    case 7: nhc_chain_kernel<7><<<nbk, 128, 0, st>>>(a); break;
    default: nhc_chain_kernel<8><<<nbk, 128, 0, st>>>(a); break;
    }
    nhc_scale_kernel<<<blocks_for(n, 256), 256, 0, st>>>(v, s.nb, pm->natm, s.inhc, s.sc, s.num);
    PCK(cudaGetLastError());
    return PINYB200_OK;
}

int apply_all_nhc(pinyb200_pimd *pm, double *d_v, cudaStream_t st)
{
    int rc = apply_nhc(pm, pm->set[0], d_v, 0, pm->d_mass, 0, st);
    if (rc) return rc;
    return apply_nhc(pm, pm->set[1], d_v, 1, pm->d_bmass + pm->natm, (size_t)pm->natm, st);
}

int ghost_positions(pinyb200_pimd *pm, pinyb200_ctx *c, double *d_x, cudaStream_t st)
{
    const pinyb200::DeviceSystem &s = c->sys;
    if (s.nghost == 0) return PINYB200_OK;
    ghost_pos_aos_kernel<<<blocks_for((long long)s.nghost * pm->P, 256), 256, 0, st>>>(
        d_x, pm->natm, pm->P, s.nghost, s.ghost_ncomp, s.ghost_atom, s.ghost_comp, s.ghost_coef);
    PCK(cudaGetLastError());
    return PINYB200_OK;
}

// Force path and post-processing, enqueued on st (springs already in d_fm
// and acc): the force evaluation, forces / P with the centroid virial sums,
// forces to modes, springs added, and the sums copied to the host.  level 0
// is the plain evaluation; otherwise the RESPA level (PINYB200_* bits) of
// the force context's split, whose weighted forces are the step's forces
// and, at the outer level, whose virial forces feed the virial sums
// (pimd_pvten_forc_corr, pimd_estimators.c:262-301).  Nothing waits here;
// pimd_finish does, once per call.
int forces_enqueue(pinyb200_pimd *pm, pinyb200_ctx *c, double *d_x, const double *d_xmod, double *d_f,
                   const pinyb200::Cell &cell, cudaStream_t st, bool timing, int level = 0)
{
    cudaStream_t own = c->stream;
    c->stream = st;  // the evaluation runs on the caller's stream
    const long long nb = (long long)pm->natm * pm->P, n = nb * 3;
    int rc;
    if (level == 0) {
        rc = pinyb200::enqueue_device(c, d_x, pm->P > 1 ? d_xmod : nullptr, cell, PINYB200_DISTRIB_GHOSTS, d_f,
                                      timing, pm->h_facc);
        pm->timed = pm->timed || timing;
        c->stream = own;
        if (rc) return rc;
        post_kernel<<<blocks_for(nb, 256), 256, 0, st>>>(d_f, d_x, d_xmod, pm->natm, pm->P, pm->P > 1, pm->d_acc);
        PCK(cudaGetLastError());
    } else {
        const bool outer = level & PINYB200_FULL_INTER;
        rc = pinyb200::stage_positions(c, d_x, pm->P > 1 ? d_xmod : nullptr, cell, 0);
        if (!rc) rc = pinyb200::respa_level_enqueue(c, cell, level, PINYB200_DISTRIB_GHOSTS, outer ? pm->h_facc : nullptr);
        cudaError_t e = cudaSuccess;
        if (!rc) e = pinyb200::launch_transpose_out(c, d_f, c->d_forceW);
        if (!rc && e == cudaSuccess && outer) e = pinyb200::launch_transpose_out(c, pm->d_ft, c->d_forceT);
        c->stream = own;
        if (rc) return rc;
        PCK(e);
        // the virial estimator from the outer level's virial forces; the
        // weighted forces are only divided by P
        if (outer)
            post_kernel<<<blocks_for(nb, 256), 256, 0, st>>>(pm->d_ft, d_x, d_xmod, pm->natm, pm->P, pm->P > 1,
                                                             pm->d_acc);
        post_kernel<<<blocks_for(nb, 256), 256, 0, st>>>(d_f, d_x, d_xmod, pm->natm, pm->P, 0, pm->d_acc);
        PCK(cudaGetLastError());
    }
    if (pm->P > 1) {
        rc = pinyb200_pimd_transform(pm->natm, pm->P, pm->kind, PINYB200_FORCE_TO_MODES, d_f, st);
        if (rc) return rc;
    }
    add_kernel<<<blocks_for(n, 256), 256, 0, st>>>(d_f, pm->d_fm, n);
    PCK(cudaGetLastError());
    PCK(cudaMemcpyAsync(pm->h_acc, pm->d_acc, sizeof(double) * A_N, cudaMemcpyDeviceToHost, st));
    return PINYB200_OK;
}

// Wait for st, then the energies: the force path's bookkeeping
// (evaluate_finish) and the PIMD sums.
int pimd_finish(pinyb200_pimd *pm, pinyb200_ctx *c, const pinyb200::Cell &cell, pinyb200_pimd_energies *e,
                cudaStream_t st)
{
    PCK(cudaStreamSynchronize(st));
    if (!pm->graph_mode && pm->timed) {  // a replayed graph (or a RESPA step) records no phase events
        cudaEventElapsedTime(&c->last_ms[0], c->ev[0], c->ev[4]);
        cudaEventElapsedTime(&c->last_ms[1], c->ev[1], c->ev[2]);
        cudaEventElapsedTime(&c->last_ms[2], c->ev_pme[0], c->ev_pme[1]);
        cudaEventElapsedTime(&c->last_ms[3], c->ev[2], c->ev[3]);
    }
    pinyb200_energies fe;
    pinyb200::evaluate_finish(c, cell, PINYB200_DISTRIB_GHOSTS, pm->h_facc, &fe);
    if (!std::isfinite(fe.vintert + fe.vintrat))
        return pimd_fail(pm, PINYB200_ERR_NAN, "pimd: non-finite energy (positions, or a list that outgrew its room)");
    if (e) {
        const double *a = pm->h_acc;
        e->force = fe;
        e->kin_harm = a[A_KIN];
        const double P = (double)pm->P;
        const double akv = 3.0 * (double)pm->nfree / pm->beta;
        e->akvirx = pm->P > 1 ? 0.5 * (akv - a[A_VIR]) : 0.0;  // PINY corrects only with beads
        for (int k = 0; k < 9; k++) {
            const double base = fe.pvten[k] / P;
            e->pvten[k] = base - a[A_PVC + k];
            e->pvten_tot[k] = base - a[A_PVC + k];
        }
        const double *m = a + A_PVM;  // xx yy zz xy xz yz
        const double pm9[9] = {m[0], m[3], m[4], m[3], m[1], m[5], m[4], m[5], m[2]};
        std::memcpy(e->pvten_mode_tot, pm9, sizeof pm9);
    }
    return PINYB200_OK;
}

int springs(pinyb200_pimd *pm, const double *d_u, cudaStream_t st)
{
    const long long nb = (long long)pm->natm * pm->P;
    springs_kernel<<<blocks_for(nb, 256), 256, 0, st>>>(d_u, pm->d_prekf, pm->d_veig, pm->wght, pm->natm, pm->P,
                                                        pm->d_fm, pm->d_acc);
    PCK(cudaGetLastError());
    return PINYB200_OK;
}

void drop_graph(pinyb200_pimd *pm)
{
    if (pm->exec) cudaGraphExecDestroy(pm->exec);
    if (pm->graph) cudaGraphDestroy(pm->graph);
    pm->exec = nullptr;
    pm->graph = nullptr;
    pm->key.clear();
}

// Everything of one step up to the host read of its sums, enqueued on st
// with no waits (capturable): int_NVT_pimd's loops over the inter, torsion,
// intra and bead RESPA levels (int_NVT_pimd.c:142-223), one pass when every
// count is 1.
int step_enqueue(pinyb200_pimd *pm, pinyb200_ctx *c, double *d_x, double *d_v, double *d_f,
                 const pinyb200::Cell &cell, cudaStream_t st, bool timing)
{
    int rc;
    const long long n = (long long)pm->natm * pm->P * 3;
    const int nt = pm->nres[0], no = pm->nres[1], na = pm->nres[2], np = pm->nres[3];
    const bool respa = nt * no * na * np > 1;
    const double dti = pm->dt / (double)(nt * no * na * np), dti2 = dti / 2.0;
    for (int ir_ter = 1; ir_ter <= nt; ir_ter++)
        for (int ir_tor = 1; ir_tor <= no; ir_tor++)
            for (int ir_tra = 1; ir_tra <= na; ir_tra++)
                for (int ir_pimd = 1; ir_pimd <= np; ir_pimd++) {
                    // t -> t + dti/2: chains at the start of a loop of
                    // level <= ix_respa, half kick (int_0_to_dt2_pimd.c:~75-145)
                    int ix = 5;
                    if (ir_pimd == 1) {
                        ix = 4;
                        if (ir_tra == 1) {
                            ix = 3;
                            if (ir_tor == 1) ix = ir_ter == 1 ? 1 : 2;
                        }
                    }
                    if (pm->ix_respa >= ix && (rc = apply_all_nhc(pm, d_v, st))) return rc;
                    kick_kernel<<<blocks_for(n, 256), 256, 0, st>>>(d_v, d_f, pm->d_bmass, n, dti2);
                    PCK(cudaGetLastError());
                    // positions -> modes (first bead step), drift, springs
                    if (pm->P > 1 && ir_pimd == 1 &&
                        (rc = pinyb200_pimd_transform(pm->natm, pm->P, pm->kind, PINYB200_TO_MODES, d_x, st)))
                        return rc;
                    drift_kernel<<<blocks_for(n, 256), 256, 0, st>>>(d_x, d_v, n, dti);
                    PCK(cudaGetLastError());
                    PCK(cudaMemsetAsync(pm->d_acc, 0, sizeof(double) * A_N, st));
                    if ((rc = springs(pm, d_x, st))) return rc;
                    if (ir_pimd == np) {
                        // mode 1 -> xmod, modes -> positions, ghosts; the forces
                        PCK(cudaMemcpyAsync(pm->d_xmod, d_x, sizeof(double) * (size_t)pm->natm * 3,
                                            cudaMemcpyDeviceToDevice, st));
                        if (pm->P > 1 &&
                            (rc = pinyb200_pimd_transform(pm->natm, pm->P, pm->kind, PINYB200_TO_BEADS, d_x, st)))
                            return rc;
                        if ((rc = ghost_positions(pm, c, d_x, st))) return rc;
                        int level = 0;
                        if (respa) {  // int_NVT_pimd.c:175-189
                            const bool last_tra = ir_tra == na;
                            if (ir_ter == nt && ir_tor == no && last_tra) level |= PINYB200_FULL_INTER;
                            if (c->r_int_res_ter && ir_tor == no && last_tra) level |= PINYB200_RES_INTER;
                            if (last_tra) level |= PINYB200_FULL_INTRA;
                            level |= PINYB200_RES_INTRA;
                        }
                        // PINY's list test and, when due, the rebuild -- on the device,
                        // where the level asks for the intermolecular forces
                        if ((!respa || (level & (PINYB200_FULL_INTER | PINYB200_RES_INTER))) &&
                            (rc = pinyb200::list_update_enqueue(c, d_x, pm->P > 1 ? pm->d_xmod : nullptr, cell, st)))
                            return rc;
                        if ((rc = forces_enqueue(pm, c, d_x, pm->d_xmod, d_f, cell, st, timing && !respa, level)))
                            return rc;
                    } else {
                        // no force call: the spring forces alone (int_NVT_pimd.c:193-207)
                        PCK(cudaMemcpyAsync(d_f, pm->d_fm, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, st));
                    }
                    // t + dti/2 -> t + dti: half kick, chains at the end of a
                    // loop of level <= ix_respa (int_dt2_to_dt_pimd.c)
                    kick_kernel<<<blocks_for(n, 256), 256, 0, st>>>(d_v, d_f, pm->d_bmass, n, dti2);
                    PCK(cudaGetLastError());
                    ix = 5;
                    if (ir_pimd == np) {
                        ix = 4;
                        if (ir_tra == na) {
                            ix = 3;
                            if (ir_tor == no) ix = ir_ter == nt ? 1 : 2;
                        }
                    }
                    if (pm->ix_respa >= ix && (rc = apply_all_nhc(pm, d_v, st))) return rc;
                }
    return PINYB200_OK;
}

int check_ctx(pinyb200_pimd *pm, pinyb200_ctx *c)
{
    if (!pm || !c) return pimd_fail(pm, PINYB200_ERR_ARG, "pimd: null handle");
    if (c->sys.natm != pm->natm || c->P != pm->P)
        return pimd_fail(pm, PINYB200_ERR_ARG, "pimd: force context has other sites or beads");
    if (!c->have_list) return pimd_fail(pm, PINYB200_ERR_STATE, "pimd: build the force context's list first");
    if (pm->nres[0] * pm->nres[1] * pm->nres[2] * pm->nres[3] > 1 && !c->respa_on)
        return pimd_fail(pm, PINYB200_ERR_STATE, "pimd: RESPA counts > 1 need pinyb200_set_respa on the force context");
    if (cudaSetDevice(c->device) != cudaSuccess) return pimd_fail(pm, PINYB200_ERR_CUDA, "pimd: cannot select the device");
    return PINYB200_OK;
}

}  // namespace

extern "C" {

int pinyb200_pimd_create(const pinyb200_pimd_setup *s, pinyb200_pimd **out)
{
    pinyb200_pimd *pm = nullptr;
    if (!s || !out || s->natm < 1 || s->nbeads < 1 || !s->mass || !s->bead_mass || !s->prekf || !s->path_eig ||
        !(s->kind == PINYB200_STAGING || s->kind == PINYB200_NORMAL_MODES) || !(s->beta > 0.0))
        return pimd_fail(nullptr, PINYB200_ERR_ARG, "pimd_create: bad setup");
    if (s->nbeads > 64 || (s->nbeads & (s->nbeads - 1)))
        return pimd_fail(nullptr, PINYB200_ERR_UNSUPPORTED, "pimd_create: beads 1..64, powers of 2");
    *out = nullptr;
    pm = new pinyb200_pimd();
    cudaGetDevice(&pm->device);
    pm->natm = s->natm;
    pm->P = s->nbeads;
    pm->kind = s->kind;
    pm->wght = s->wght_pimd;
    pm->dt = s->dt;
    pm->beta = s->beta;
    pm->nfree = s->nfree_atoms;
    const int nres[4] = {s->nres_ter, s->nres_tor, s->nres_tra, s->nres_pimd};
    for (int k = 0; k < 4; k++) {
        if (nres[k] < 0 || nres[k] > 64) {
            delete pm;
            return pimd_fail(nullptr, PINYB200_ERR_ARG, "pimd_create: RESPA counts 0..64");
        }
        pm->nres[k] = nres[k] > 0 ? nres[k] : 1;
    }
    if (s->ix_respa < 0 || s->ix_respa > 5) {
        delete pm;
        return pimd_fail(nullptr, PINYB200_ERR_ARG, "pimd_create: ix_respa 1..5");
    }
    pm->ix_respa = s->ix_respa > 0 ? s->ix_respa : 1;
    const size_t na = (size_t)s->natm, nb = na * s->nbeads;
    auto cleanup = [&](int rc) {
        pinyb200_pimd_destroy(pm);
        return rc;
    };
#define CCK(call)                                                                                          \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return cleanup(pimd_fail(nullptr, PINYB200_ERR_CUDA, cudaGetErrorString(e_))); \
    } while (0)
    CCK(cudaMalloc(&pm->d_mass, sizeof(double) * na));
    CCK(cudaMalloc(&pm->d_bmass, sizeof(double) * nb));
    CCK(cudaMalloc(&pm->d_prekf, sizeof(double) * na));
    CCK(cudaMalloc(&pm->d_veig, sizeof(double) * s->nbeads));
    CCK(cudaMalloc(&pm->d_fm, sizeof(double) * nb * 3));
    CCK(cudaMalloc(&pm->d_u, sizeof(double) * nb * 3));
    CCK(cudaMalloc(&pm->d_xmod, sizeof(double) * na * 3));
    CCK(cudaMalloc(&pm->d_acc, sizeof(double) * A_N));
    if (pm->nres[0] * pm->nres[1] * pm->nres[2] * pm->nres[3] > 1) CCK(cudaMalloc(&pm->d_ft, sizeof(double) * nb * 3));
    CCK(cudaMallocHost(&pm->h_acc, sizeof(double) * A_N));
    CCK(cudaMallocHost(&pm->h_facc, sizeof(double) * (size_t)s->nbeads * pinyb200::S_NSLOT));
    CCK(cudaMemcpy(pm->d_mass, s->mass, sizeof(double) * na, cudaMemcpyHostToDevice));
    CCK(cudaMemcpy(pm->d_bmass, s->bead_mass, sizeof(double) * nb, cudaMemcpyHostToDevice));
    CCK(cudaMemcpy(pm->d_prekf, s->prekf, sizeof(double) * na, cudaMemcpyHostToDevice));
    CCK(cudaMemcpy(pm->d_veig, s->path_eig, sizeof(double) * s->nbeads, cudaMemcpyHostToDevice));
#undef CCK
    int rc = upload_set(pm, pm->set[0], s->class_nhc, 1);
    if (!rc) rc = upload_set(pm, pm->set[1], s->bead_nhc, s->nbeads - 1);
    if (rc) return cleanup(rc);
    *out = pm;
    return PINYB200_OK;
}

int pinyb200_pimd_destroy(pinyb200_pimd *pm)
{
    if (!pm) return PINYB200_OK;
    cudaFree(pm->d_mass);
    cudaFree(pm->d_bmass);
    cudaFree(pm->d_prekf);
    cudaFree(pm->d_veig);
    cudaFree(pm->d_fm);
    cudaFree(pm->d_u);
    cudaFree(pm->d_xmod);
    cudaFree(pm->d_acc);
    cudaFree(pm->d_ft);
    cudaFreeHost(pm->h_acc);
    cudaFreeHost(pm->h_facc);
    free_set(pm->set[0]);
    free_set(pm->set[1]);
    drop_graph(pm);
    if (pm->cap) cudaStreamDestroy(pm->cap);
    delete pm;
    return PINYB200_OK;
}

int pinyb200_pimd_set_nhc(pinyb200_pimd *pm, int set, const double *x_nhc, const double *v_nhc)
{
    if (!pm || set < 0 || set > 1 || !x_nhc || !v_nhc) return pimd_fail(pm, PINYB200_ERR_ARG, "pimd_set_nhc: bad arguments");
    NhcDev &s = pm->set[set];
    if (s.num == 0) return PINYB200_OK;
    const size_t n = (size_t)s.nb * s.len * s.num;
    PCK(cudaMemcpy(s.x, x_nhc, sizeof(double) * n, cudaMemcpyHostToDevice));
    PCK(cudaMemcpy(s.v, v_nhc, sizeof(double) * n, cudaMemcpyHostToDevice));
    return PINYB200_OK;
}

int pinyb200_pimd_get_nhc(pinyb200_pimd *pm, int set, double *x_nhc, double *v_nhc)
{
    if (!pm || set < 0 || set > 1 || !x_nhc || !v_nhc) return pimd_fail(pm, PINYB200_ERR_ARG, "pimd_get_nhc: bad arguments");
    NhcDev &s = pm->set[set];
    if (s.num == 0) return PINYB200_OK;
    const size_t n = (size_t)s.nb * s.len * s.num;
    PCK(cudaMemcpy(x_nhc, s.x, sizeof(double) * n, cudaMemcpyDeviceToHost));
    PCK(cudaMemcpy(v_nhc, s.v, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return PINYB200_OK;
}

int pinyb200_pimd_forces(pinyb200_pimd *pm, pinyb200_ctx *c, double *d_x, double *d_f, const double *hmat,
                         pinyb200_pimd_energies *e, void *stream)
{
    int rc = check_ctx(pm, c);
    if (rc) return rc;
    if (!d_x || !d_f || !hmat) return pimd_fail(pm, PINYB200_ERR_ARG, "pimd_forces: null pointer");
    pm->timed = false;
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;  // NULL: the force context's stream
    const size_t nbytes = sizeof(double) * (size_t)pm->natm * pm->P * 3;
    if ((rc = ghost_positions(pm, c, d_x, st))) return rc;
    PCK(cudaMemcpyAsync(pm->d_u, d_x, nbytes, cudaMemcpyDeviceToDevice, st));
    if (pm->P > 1 && (rc = pinyb200_pimd_transform(pm->natm, pm->P, pm->kind, PINYB200_TO_MODES, pm->d_u, st)))
        return rc;
    PCK(cudaMemsetAsync(pm->d_acc, 0, sizeof(double) * A_N, st));
    if ((rc = springs(pm, pm->d_u, st))) return rc;
    const pinyb200::Cell cell = pinyb200::cell_from_hmat(hmat);
    // with RESPA, the outer level (control_pimd.c:297-317): RES_INTER with
    // inter RESPA, RES_INTRA with intra RESPA (PINY's int_res_tra, set by
    // respa_steps_intra, set_sim_params.c:1626-1637).  Beside FULL_INTRA the
    // RES_INTRA bit changes only PINY's RESPA pressure guesses in pvten
    // (energy_control_inter_real.c:270-279), not the forces or pvten_tot.
    const int level = pm->nres[0] * pm->nres[1] * pm->nres[2] * pm->nres[3] > 1
                          ? PINYB200_FULL_INTER | PINYB200_FULL_INTRA | (pm->nres[2] > 1 ? PINYB200_RES_INTRA : 0) |
                                (c->r_int_res_ter ? PINYB200_RES_INTER : 0)
                          : 0;
    if ((rc = forces_enqueue(pm, c, d_x, pm->d_u, d_f, cell, st, level == 0, level))) return rc;
    pm->graph_mode = false;
    return pimd_finish(pm, c, cell, e, st);
}

int pinyb200_pimd_step(pinyb200_pimd *pm, pinyb200_ctx *c, double *d_x, double *d_v, double *d_f, const double *hmat,
                       pinyb200_pimd_energies *e, void *stream)
{
    int rc = check_ctx(pm, c);
    if (rc) return rc;
    if (!d_x || !d_v || !d_f || !hmat) return pimd_fail(pm, PINYB200_ERR_ARG, "pimd_step: null pointer");
    pm->timed = false;
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;  // NULL: the force context's stream
    const pinyb200::Cell cell = pinyb200::cell_from_hmat(hmat);
    // Steps with the same arguments replay one CUDA graph: the first such
    // step runs eagerly (it sets up everything the work needs), the second
    // is captured and launched, later ones are launched.
    std::vector<double> key = {(double)(uintptr_t)d_x, (double)(uintptr_t)d_v, (double)(uintptr_t)d_f,
                               (double)(uintptr_t)c, (double)c->gen};
    key.insert(key.end(), hmat, hmat + 9);
    if (pm->exec && key != pm->key) drop_graph(pm);
    if (!pm->exec && key != pm->eager) {
        if ((rc = step_enqueue(pm, c, d_x, d_v, d_f, cell, st, true))) return rc;
        pm->eager = key;
        pm->graph_mode = false;
        return pimd_finish(pm, c, cell, e, st);
    }
    if (!pm->exec) {
        if (!pm->cap) PCK(cudaStreamCreateWithFlags(&pm->cap, cudaStreamNonBlocking));
        PCK(cudaStreamBeginCapture(pm->cap, cudaStreamCaptureModeRelaxed));
        rc = step_enqueue(pm, c, d_x, d_v, d_f, cell, pm->cap, false);
        cudaGraph_t g = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(pm->cap, &g);
        if (rc || ee != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return rc ? rc : pimd_fail(pm, PINYB200_ERR_CUDA, std::string("pimd step capture: ") + cudaGetErrorString(ee));
        }
        pm->graph = g;
        PCK(cudaGraphInstantiate(&pm->exec, pm->graph, 0));
        pm->key = key;
    }
    PCK(cudaGraphLaunch(pm->exec, st));
    pm->graph_mode = true;
    return pimd_finish(pm, c, cell, e, st);
}

}  // extern "C"
