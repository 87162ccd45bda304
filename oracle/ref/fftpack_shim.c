/*
 * Test infrastructure only: link shim that lets PINY's own C sources build
 * without a Fortran compiler.  Nothing here is part of the product.
 *
 * PINY's generic 3D FFT (src/mathlib/fft_package.c:1359-1423, fft_gen1d)
 * calls three FFTPACK routines from src/mathlib/fft_generic.f:
 *   DCFFTI_GENERIC(n, wsave)      -- set up for length n      (fft_generic.f:2)
 *   DCFFTF_GENERIC(n, c, wsave)   -- forward,  exp(-2 pi i jk/n) (fft_generic.f:86)
 *   DCFFTB_GENERIC(n, c, wsave)   -- backward, exp(+2 pi i jk/n) (fft_generic.f:513)
 * Both transforms are unnormalised, in place, on n interleaved complex values.
 * This file supplies the same contract with an independent mixed-radix
 * decimation-in-time FFT written from the DFT definition.  The layout of
 * wsave is private to this file: PINY sizes it at 4n+15 doubles
 * (fft_create_package.c) and never looks inside.  We keep the twiddle table
 * e^{-2 pi i k/n}, k<n, in wsave[2n..4n) and the factorisation in the
 * trailing 15 words; the first 2n words are not used (scratch is per call).
 *
 * DURAND (src/mathlib/blas_wrappers.f:39) is the Park-Miller minimal
 * standard generator, x <- 16807 x mod (2^31 - 1); PINY only uses it to
 * sample initial velocities, which never reach the force path, so an integer
 * restatement of the same recurrence is supplied.
 * The remaining Fortran symbols PINY references (LINPACK/EISPACK) are never
 * reached on the force path; they abort loudly if called.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAXFAC 13

static void factorize(int n, int *fac, int *nf)
{
    int m = n, k = 0;
    static const int pref[] = {4, 2, 3, 5};
    for (int t = 0; t < 4 && m > 1; t++) {
        while (m % pref[t] == 0 && k < MAXFAC) { fac[k++] = pref[t]; m /= pref[t]; }
    }
    for (int p = 7; m > 1 && k < MAXFAC; p += 2) {
        while (m % p == 0 && k < MAXFAC) { fac[k++] = p; m /= p; }
    }
    if (m != 1) { fprintf(stderr, "fftpack_shim: cannot factor %d\n", n); abort(); }
    *nf = k;
}

void dcffti_generic_(int *pn, double *wsave)
{
    int n = *pn;
    if (n <= 1) return;
    double *tw = wsave + 2 * n;
    for (int k = 0; k < n; k++) {
        double a = 2.0 * M_PI * (double)k / (double)n;
        tw[2 * k] = cos(a);
        tw[2 * k + 1] = -sin(a);
    }
    int fac[MAXFAC], nf = 0;
    factorize(n, fac, &nf);
    double *fw = wsave + 4 * n;
    fw[0] = (double)nf;
    for (int i = 0; i < nf; i++) fw[1 + i] = (double)fac[i];
}

/*
 * One Stockham stage: input x holds `m` interleaved sub-sequences of length
 * l*r laid out as (s, j) ... we use the classic recursive formulation
 * unrolled into stages: at stage with radix r, current transform length L
 * (= product of radices processed so far times r), the data are combined
 * r at a time with twiddles w_L^{s k}.
 */
static void fft_run(int n, double *c, const double *tw, const double *fw,
                    int sign)
{
    int nf = (int)fw[0];
    int fac[MAXFAC];
    for (int i = 0; i < nf; i++) fac[i] = (int)fw[1 + i];

    double *a = (double *)malloc(sizeof(double) * 2 * n);
    double *b = (double *)malloc(sizeof(double) * 2 * n);
    double *tmp = (double *)malloc(sizeof(double) * 2 * 64);
    if (!a || !b || !tmp) { fprintf(stderr, "fftpack_shim: oom\n"); abort(); }
    memcpy(a, c, sizeof(double) * 2 * n);

    /* Decimation in time, Stockham autosort.  At a stage, `l` is the length
     * of the already-transformed sub-transforms and `m = n/(l*r)` the number
     * of interleaved groups.  a[(j*l*r? ...)] -- we index explicitly. */
    int l = 1;
    for (int f = nf - 1; f >= 0; f--) {
        int r = fac[f];
        int m = n / (l * r);
        /* input a: for group q in [0,m), sub-sequence s in [0,r): transform
         * of length l stored at a[ ((s*m + q) * l + k) ], k<l.
         * output b: group q, transform of length l*r at b[(q*l*r + K)]. */
        double *t = (r <= 64) ? tmp : (double *)malloc(sizeof(double) * 2 * r);
        for (int q = 0; q < m; q++) {
            for (int k = 0; k < l; k++) {
                /* gather r inputs with twiddle w_{l r}^{s k} */
                for (int s = 0; s < r; s++) {
                    const double *x = a + 2 * ((size_t)(s * m + q) * l + k);
                    int e = (int)(((long)s * k * m) % n); /* w_{lr}^{sk} = w_n^{s k m} */
                    double wr = tw[2 * e], wi = sign * tw[2 * e + 1];
                    t[2 * s] = x[0] * wr - x[1] * wi;
                    t[2 * s + 1] = x[0] * wi + x[1] * wr;
                }
                /* length-r DFT of t, outputs at K = k + l*u */
                for (int u = 0; u < r; u++) {
                    double sr = 0.0, si = 0.0;
                    for (int s = 0; s < r; s++) {
                        int e = (int)(((long)s * u * l * m) % n); /* w_r^{su} */
                        double wr = tw[2 * e], wi = sign * tw[2 * e + 1];
                        sr += t[2 * s] * wr - t[2 * s + 1] * wi;
                        si += t[2 * s] * wi + t[2 * s + 1] * wr;
                    }
                    double *y = b + 2 * ((size_t)q * l * r + k + (size_t)l * u);
                    y[0] = sr;
                    y[1] = si;
                }
            }
        }
        if (t != tmp) free(t);
        double *sw = a; a = b; b = sw;
        l *= r;
    }
    memcpy(c, a, sizeof(double) * 2 * n);
    free(a); free(b); free(tmp);
}

void dcfftf_generic_(int *pn, double *c, double *wsave)
{
    int n = *pn;
    if (n <= 1) return;
    fft_run(n, c, wsave + 2 * n, wsave + 4 * n, +1);
}

void dcfftb_generic_(int *pn, double *c, double *wsave)
{
    int n = *pn;
    if (n <= 1) return;
    fft_run(n, c, wsave + 2 * n, wsave + 4 * n, -1);
}

void durand_(double *seed, int *n, double *x, int *ierr)
{
    const long long m = 2147483647LL;
    *ierr = 0;
    if (*n < 0 || *seed < 1.0 || *seed > 2147483646.0) { *ierr = 1; return; }
    long long s = (long long)(*seed);
    for (int j = 0; j < *n; j++) {
        s = (16807LL * s) % m;
        x[j] = (double)s / (double)m;
    }
    *seed = (double)s;
}

#define ABORT_STUB(name)                                                      \
    void name(void)                                                           \
    {                                                                         \
        fprintf(stderr, "fftpack_shim: %s is not available in this build\n", \
                #name);                                                       \
        abort();                                                              \
    }

ABORT_STUB(dgefa_)
ABORT_STUB(dgesl_)
ABORT_STUB(rs_)
ABORT_STUB(rsg_)
ABORT_STUB(gen_matmul_)
