// Device helpers shared by the pinyb200 kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "internal.h"

namespace pinyb200 {

// NINT of PINY (round half away from zero, include/typ_defs/defines.h:96-97),
// written with round-to-nearest intrinsics so that no FMA contraction can
// change the operation the distance tests depend on.
__device__ __forceinline__ double nint_rn(double x)
{
    return (double)(x >= 0.0 ? __double2int_rz(__dadd_rn(x, 0.5)) : __double2int_rz(__dsub_rn(x, 0.5)));
}

// Pair type of two atom types in PINY's upper-triangle order
// (npol_posdata_fetch, src/energy/inter/real_space/force_npol.c:585-599).
__device__ __forceinline__ int pair_type(int ti, int tj, int ntyp)
{
    int i2 = ti + 1, i3 = tj + 1;
    int jj = i2 < i3 ? i2 : i3;
    int ii = i2 + i3 - jj;
    return ((jj - 1) * ((ntyp + 1) * 2 - jj)) / 2 + ii - jj;
}

// Minimum image of one separation (period(), period.c:27-114) with exact
// IEEE operation order.
__device__ __forceinline__ void period_exact(double &dx, double &dy, double &dz, const Cell &c)
{
    if (c.cubic) {
        double asx = __dmul_rn(dx, c.hi[0]), asy = __dmul_rn(dy, c.hi[4]), asz = __dmul_rn(dz, c.hi[8]);
        double sx = __dsub_rn(asx, nint_rn(asx)), sy = __dsub_rn(asy, nint_rn(asy)),
               sz = __dsub_rn(asz, nint_rn(asz));
        dx = __dmul_rn(sx, c.h[0]);
        dy = __dmul_rn(sy, c.h[4]);
        dz = __dmul_rn(sz, c.h[8]);
    } else {
        double asx = __dadd_rn(__dadd_rn(__dmul_rn(dx, c.hi[0]), __dmul_rn(dy, c.hi[3])), __dmul_rn(dz, c.hi[6]));
        double asy = __dadd_rn(__dadd_rn(__dmul_rn(dx, c.hi[1]), __dmul_rn(dy, c.hi[4])), __dmul_rn(dz, c.hi[7]));
        double asz = __dadd_rn(__dadd_rn(__dmul_rn(dx, c.hi[2]), __dmul_rn(dy, c.hi[5])), __dmul_rn(dz, c.hi[8]));
        double sx = __dsub_rn(asx, nint_rn(asx)), sy = __dsub_rn(asy, nint_rn(asy)),
               sz = __dsub_rn(asz, nint_rn(asz));
        dx = __dadd_rn(__dadd_rn(__dmul_rn(sx, c.h[0]), __dmul_rn(sy, c.h[3])), __dmul_rn(sz, c.h[6]));
        dy = __dadd_rn(__dadd_rn(__dmul_rn(sx, c.h[1]), __dmul_rn(sy, c.h[4])), __dmul_rn(sz, c.h[7]));
        dz = __dadd_rn(__dadd_rn(__dmul_rn(sx, c.h[2]), __dmul_rn(sy, c.h[5])), __dmul_rn(sz, c.h[8]));
    }
}

// PIMD minimum image: shift a bead separation by -NINT(h^-1 dmode) h where
// dmode is the mode-1 (centroid) separation (period_pimd, period.c:121-213).
__device__ __forceinline__ void period_pimd_exact(double &dx, double &dy, double &dz, double dxs, double dys,
                                                  double dzs, const Cell &c)
{
    if (c.cubic) {
        double sx = -nint_rn(__dmul_rn(dxs, c.hi[0]));
        double sy = -nint_rn(__dmul_rn(dys, c.hi[4]));
        double sz = -nint_rn(__dmul_rn(dzs, c.hi[8]));
        dx = __dadd_rn(dx, __dmul_rn(sx, c.h[0]));
        dy = __dadd_rn(dy, __dmul_rn(sy, c.h[4]));
        dz = __dadd_rn(dz, __dmul_rn(sz, c.h[8]));
    } else {
        double asx = __dadd_rn(__dadd_rn(__dmul_rn(dxs, c.hi[0]), __dmul_rn(dys, c.hi[3])), __dmul_rn(dzs, c.hi[6]));
        double asy = __dadd_rn(__dadd_rn(__dmul_rn(dxs, c.hi[1]), __dmul_rn(dys, c.hi[4])), __dmul_rn(dzs, c.hi[7]));
        double asz = __dadd_rn(__dadd_rn(__dmul_rn(dxs, c.hi[2]), __dmul_rn(dys, c.hi[5])), __dmul_rn(dzs, c.hi[8]));
        double sx = -nint_rn(asx), sy = -nint_rn(asy), sz = -nint_rn(asz);
        dx = __dadd_rn(dx, __dadd_rn(__dadd_rn(__dmul_rn(sx, c.h[0]), __dmul_rn(sy, c.h[3])), __dmul_rn(sz, c.h[6])));
        dy = __dadd_rn(dy, __dadd_rn(__dadd_rn(__dmul_rn(sx, c.h[1]), __dmul_rn(sy, c.h[4])), __dmul_rn(sz, c.h[7])));
        dz = __dadd_rn(dz, __dadd_rn(__dadd_rn(__dmul_rn(sx, c.h[2]), __dmul_rn(sy, c.h[5])), __dmul_rn(sz, c.h[8])));
    }
}

template <typename R> struct Vec4;
template <> struct Vec4<double> { typedef double4 T; };
template <> struct Vec4<float> { typedef float4 T; };
template <typename R> struct Cplx;
template <> struct Cplx<double> { typedef double2 T; };
template <> struct Cplx<float> { typedef float2 T; };

// Cubic of npol_vspl_fetch (force_npol.c:339-375) from precomputed
// interval coefficients (c0, c1, c2, c3) of knot k.
template <typename V, typename R>
__device__ __forceinline__ R spline_eval(const V &c, R del)
{
    return c.x + del * (c.y + del * (c.z + del * c.w));
}

// Read-only cached loads of a table 4-vector.
__device__ __forceinline__ float4 ldg4(const float4 *p) { return __ldg(p); }
__device__ __forceinline__ double4 ldg4(const double4 *p)
{
    const double2 a = __ldg((const double2 *)p), b = __ldg((const double2 *)p + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

template <typename R> struct Idx;

// Spline knot and offset.  FP64 keeps PINY's rounding exactly (no FMA), FP32
// uses plain arithmetic.
template <> struct Idx<double> {
    static __device__ __forceinline__ int knot(double r, double rmin, double dr, double dri, int nsm2, double &del)
    {
        int k = __double2int_rz(__dadd_rn(__dmul_rn(__dsub_rn(r, rmin), dri), 0.5)) + 3;
        k = k < nsm2 ? k : nsm2;
        k = k > 3 ? k : 3;
        double rsp = __dadd_rn(__dmul_rn((double)(k - 3), dr), rmin);
        del = __dmul_rn(__dsub_rn(r, rsp), dri);
        return k;
    }
    static __device__ __forceinline__ double dist(double dx, double dy, double dz)
    {
        return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    }
};
template <> struct Idx<float> {
    static __device__ __forceinline__ int knot(float r, float rmin, float dr, float dri, int nsm2, float &del)
    {
        int k = (int)((r - rmin) * dri + 0.5f) + 3;
        k = k < nsm2 ? k : nsm2;
        k = k > 3 ? k : 3;
        float rsp = (float)(k - 3) * dr + rmin;
        del = (r - rsp) * dri;
        return k;
    }
    static __device__ __forceinline__ float dist(float dx, float dy, float dz)
    {
        return sqrtf(dx * dx + dy * dy + dz * dz);
    }
};

// Warp sum of a double over the lanes that share (lane mod stride).
__device__ __forceinline__ double warp_sum_strided(double v, int stride)
{
    for (int o = 16; o >= stride; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace pinyb200
