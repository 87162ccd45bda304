// Ring-polymer coordinate transforms of PINY's PIMD integrators, in FP64 on
// device arrays in the library's bead-major layout x[b][i][d] ([P][natm][3]),
// in place.  One thread per (atom, direction) walks the P beads; at fixed
// bead the 32 threads of a warp touch 32 consecutive doubles.
//
// Staging (pi_md_typ 1; src/energy/pimd/transform_stg.c), with
// rat1[ip] = (ip-1)/ip and rat2[ip] = 1/ip (transform_cnt.c:204-213):
//   modes:  u_1 = x_1;  u_ip = x_ip - (rat1 x_ip+1 + rat2 x_1), ip = 2..P-1;
//           u_P = x_P - (rat1 x_1 + rat2 x_1)             (convert_pimd_mode_stag)
//   back:   x_P = u_P + x_1;  x_ip = u_ip + (rat1 x_ip+1 + x_1 rat2), ip = P-1..2
//                                                         (convert_pimd_pos_stag)
//   forces: f_1 += f_2 + ... + f_P;  f_ip+1 += rat1[ip] f_ip, ip = 2..P-1
//                                                         (convert_pimd_force_stag)
// Normal modes (pi_md_typ 2; transform_cnt.c:240-491), bead ip at j = ip-1:
//   modes:  X_k = (1/P) sum_j x_j e^{+2 pi i j k / P}  (FFTPACK backward), packed
//           u_1 = Re X_0, u_2m = Re X_m, u_2m+1 = Im X_m (m = 1..P/2-1), u_P = Re X_P/2
//   back:   x_j = sum_k X_k e^{-2 pi i j k / P} with X_P-m = conj X_m
//   forces: F_k = sum_j f_j e^{+2 pi i j k / P}, packed as the modes with a
//           factor 2 on every mode but the first and the last
// Staging uses round-to-nearest multiply/add intrinsics, grouped as PINY
// groups them, so no multiply-add is contracted: results are bit-identical
// to PINY's.  The normal-mode DFTs are direct sums over beads (P <= 64) with
// the P twiddles e^{2 pi i m / P} in shared memory; they agree with PINY's
// FFT to rounding.
#include <climits>

#include "common.cuh"

namespace {

// A row's beads are loaded into registers first, so every load of the row
// is in flight at once; rat1[ip] = (ip-1)/ip and rat2[ip] = 1/ip are
// correctly rounded (as PINY's) into shared memory once per block.
template <int P, int WHAT>
__global__ void __launch_bounds__(128) staging_kernel(double *__restrict__ x, int natm)
{
    __shared__ double r1[P + 1], r2[P + 1];
    for (int ip = threadIdx.x; ip <= P; ip += blockDim.x) {
        r1[ip] = ip >= 2 ? __ddiv_rn((double)(ip - 1), (double)ip) : 0.0;
        r2[ip] = ip >= 2 ? __ddiv_rn(1.0, (double)ip) : 0.0;
    }
    __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;  // 3 * atom + direction
    if (t >= natm * 3) return;
    const size_t stride = (size_t)natm * 3;
    double v[P + 1];
#pragma unroll
    for (int ip = 1; ip <= P; ip++) v[ip] = x[(ip - 1) * stride + t];
    if (WHAT == PINYB200_TO_MODES) {
        // ascending: bead ip+1 is read before it is overwritten
#pragma unroll
        for (int ip = 2; ip <= P - 1; ip++)
            v[ip] = __dsub_rn(v[ip], __dadd_rn(__dmul_rn(r1[ip], v[ip + 1]), __dmul_rn(r2[ip], v[1])));
        v[P] = __dsub_rn(v[P], __dadd_rn(__dmul_rn(r1[P], v[1]), __dmul_rn(r2[P], v[1])));
    } else if (WHAT == PINYB200_TO_BEADS) {
        // descending: bead ip+1 is already a position when bead ip needs it
        v[P] = __dadd_rn(v[P], v[1]);
#pragma unroll
        for (int ip = P - 1; ip >= 2; ip--)
            v[ip] = __dadd_rn(v[ip], __dadd_rn(__dmul_rn(r1[ip], v[ip + 1]), __dmul_rn(v[1], r2[ip])));
    } else {
        // f_1 sums the original f_2..f_P in bead order, then f_ip+1 takes
        // rat1[ip] times the already updated f_ip
#pragma unroll
        for (int ip = 2; ip <= P; ip++) v[1] = __dadd_rn(v[1], v[ip]);
#pragma unroll
        for (int ip = 2; ip <= P - 1; ip++) v[ip + 1] = __dadd_rn(v[ip + 1], __dmul_rn(r1[ip], v[ip]));
    }
#pragma unroll
    for (int ip = 1; ip <= P; ip++) x[(ip - 1) * stride + t] = v[ip];
}

template <int P>
__global__ void __launch_bounds__(128) normal_mode_kernel(double *__restrict__ x, int natm, int what)
{
    __shared__ double2 tw[P];  // (cos, sin) of 2 pi m / P
    for (int m = threadIdx.x; m < P; m += blockDim.x) {
        double sn, cs;
        sincospi(__ddiv_rn(2.0 * (double)m, (double)P), &sn, &cs);
        tw[m] = make_double2(cs, sn);
    }
    __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= natm * 3) return;
    constexpr int NP2 = P / 2;
    const size_t stride = (size_t)natm * 3;
    double v[P];
#pragma unroll
    for (int j = 0; j < P; j++) v[j] = x[j * stride + t];
    // Every input of this row is in registers: outputs go straight back.
    if (what != PINYB200_TO_BEADS) {
        const double scale = what == PINYB200_TO_MODES ? __ddiv_rn(1.0, (double)P) : 1.0;
        const double pair = what == PINYB200_FORCE_TO_MODES ? 2.0 : 1.0;
        for (int k = 0; k <= NP2; k++) {
            double re = 0.0, im = 0.0;
#pragma unroll
            for (int j = 0; j < P; j++) {
                const double2 w = tw[(j * k) & (P - 1)];
                re = fma(v[j], w.x, re);
                im = fma(v[j], w.y, im);
            }
            if (what == PINYB200_TO_MODES) {
                re *= scale;
                im *= scale;
            }
            if (k == 0) x[t] = re;
            else if (k == NP2) x[(P - 1) * stride + t] = re;
            else {
                x[(2 * k - 1) * stride + t] = re * pair;  // mode 2k (1-based)
                x[(2 * k) * stride + t] = im * pair;      // mode 2k+1
            }
        }
    } else {
        for (int j = 0; j < P; j++) {
            double s = 0.0;
#pragma unroll
            for (int k = 1; k < NP2; k++) {
                // X_k e^{-i a} + conj(X_k) e^{+i a} = 2 (Re X_k cos a + Im X_k sin a)
                const double2 w = tw[(j * k) & (P - 1)];
                s = fma(v[2 * k - 1], w.x, s);
                s = fma(v[2 * k], w.y, s);
            }
            x[j * stride + t] = v[0] + ((j & 1) ? -v[P - 1] : v[P - 1]) + 2.0 * s;
        }
    }
}

}  // namespace

extern "C" {

int pinyb200_pimd_transform(int natm, int nbeads, int kind, int what, double *d_x, void *stream)
{
    if (natm < 1 || !d_x || !(kind == PINYB200_STAGING || kind == PINYB200_NORMAL_MODES) || what < 0 || what > 2)
        return pinyb200::record_error(nullptr, PINYB200_ERR_ARG, "pimd_transform: bad arguments");
    if (nbeads == 1) return PINYB200_OK;  // PINY skips pi_beads == 1
    if ((size_t)natm * 3 > (size_t)INT_MAX - 128)
        return pinyb200::record_error(nullptr, PINYB200_ERR_ARG, "pimd_transform: too many atoms");
    const int threads = 128, blocks = (natm * 3 + threads - 1) / threads;
    cudaStream_t st = (cudaStream_t)stream;
#define PIMD_CASE(PV)                                                                                   \
    case PV:                                                                                            \
        if (kind == PINYB200_NORMAL_MODES) normal_mode_kernel<PV><<<blocks, threads, 0, st>>>(d_x, natm, what); \
        else if (what == PINYB200_TO_MODES)                                                                \
            staging_kernel<PV, PINYB200_TO_MODES><<<blocks, threads, 0, st>>>(d_x, natm);                 \
        else if (what == PINYB200_TO_BEADS)                                                                \
            staging_kernel<PV, PINYB200_TO_BEADS><<<blocks, threads, 0, st>>>(d_x, natm);                 \
        else                                                                                               \
            staging_kernel<PV, PINYB200_FORCE_TO_MODES><<<blocks, threads, 0, st>>>(d_x, natm);           \
        break;
    switch (nbeads) {
        PIMD_CASE(2)
        PIMD_CASE(4)
        PIMD_CASE(8)
        PIMD_CASE(16)
        PIMD_CASE(32)
        PIMD_CASE(64)
    default: return pinyb200::record_error(nullptr, PINYB200_ERR_UNSUPPORTED, "pimd_transform: beads 1..64, powers of 2");
    }
#undef PIMD_CASE
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return pinyb200::record_error(nullptr, PINYB200_ERR_CUDA, cudaGetErrorString(e));
    return PINYB200_OK;
}

}  // extern "C"
