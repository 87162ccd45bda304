// Device-wide exclusive prefix sums of per-row counts (the row offsets of the
// Verlet lists, their molecule and chunk forms, and the link cells): tiles of
// PINYB200_SCAN_TILE counts, one block each, in three launches -- the sum of
// every tile, the exclusive scan of those sums, the scan inside each tile
// with its tile's offset.  K arrays of n counts at count + k n are scanned
// side by side (blockIdx.y); out_k[n] and tot[k] receive array k's total.
#include "common.cuh"

namespace pinyb200 {

#define PINYB200_SCAN_TILE 4096  // counts per block (4 per thread)

namespace {

// Inclusive scan of v over the block (1024 threads); *total gets the sum.
__device__ __forceinline__ long long block_inclusive_scan(long long v, long long *warp_sums, long long *total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        const long long u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) warp_sums[w] = v;
    __syncthreads();
    if (w == 0) {
        long long s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const long long u = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += u;
        }
        warp_sums[lane] = s;  // inclusive over warps
    }
    __syncthreads();
    if (w > 0) v += warp_sums[w - 1];
    *total = warp_sums[(blockDim.x >> 5) - 1];
    return v;
}

}  // namespace

struct ScanOut {
    int *out[2];
};

__global__ void __launch_bounds__(1024) scan_tile_sum_kernel(const int *__restrict__ gate, int n,
                                                              const int *__restrict__ count, int ntile,
                                                              long long *__restrict__ part)
{
    if (gate && *gate == 0) return;
    __shared__ long long ws[32];
    const int k = blockIdx.y;
    const int *c = count + (size_t)k * n;
    const long long base = (long long)blockIdx.x * PINYB200_SCAN_TILE;
    long long s = 0;
    for (int i = threadIdx.x; i < PINYB200_SCAN_TILE; i += blockDim.x)
        if (base + i < n) s += c[base + i];
    long long total;
    block_inclusive_scan(s, ws, &total);
    if (threadIdx.x == 0) part[(size_t)k * ntile + blockIdx.x] = total;
}

// Exclusive scan of the tile sums in place (one block per array).
__global__ void __launch_bounds__(1024) scan_part_kernel(const int *__restrict__ gate, int n, int ntile,
                                                          long long *__restrict__ part, ScanOut o,
                                                          long long *__restrict__ tot)
{
    if (gate && *gate == 0) return;
    __shared__ long long ws[32];
    const int k = blockIdx.x;
    long long *p = part + (size_t)k * ntile;
    long long carry = 0;
    for (int b0 = 0; b0 < ntile; b0 += blockDim.x) {
        const int b = b0 + threadIdx.x;
        const long long v = b < ntile ? p[b] : 0;
        long long total;
        const long long inc = block_inclusive_scan(v, ws, &total);
        if (b < ntile) p[b] = carry + inc - v;
        carry += total;
        __syncthreads();  // ws is reused by the next chunk
    }
    if (threadIdx.x == 0) {
        o.out[k][n] = (int)carry;
        tot[k] = carry;
    }
}

// The scan inside each tile, offset by its tile's exclusive sum (part, or 0
// for a single tile, which also writes the totals).
__global__ void __launch_bounds__(1024) scan_tile_kernel(const int *__restrict__ gate, int n,
                                                          const int *__restrict__ count, int ntile,
                                                          const long long *__restrict__ part, ScanOut o,
                                                          long long *__restrict__ tot)
{
    if (gate && *gate == 0) return;
    __shared__ long long s[PINYB200_SCAN_TILE];
    __shared__ long long ws[32];
    const int k = blockIdx.y;
    const int *c = count + (size_t)k * n;
    int *out = o.out[k];
    const long long base = (long long)blockIdx.x * PINYB200_SCAN_TILE;
    for (int i = threadIdx.x; i < PINYB200_SCAN_TILE; i += blockDim.x) s[i] = base + i < n ? c[base + i] : 0;
    __syncthreads();
    constexpr int PER = PINYB200_SCAN_TILE / 1024;
    long long v[PER], sum = 0;
#pragma unroll
    for (int j = 0; j < PER; j++) {
        v[j] = s[PER * threadIdx.x + j];
        sum += v[j];
    }
    long long total;
    const long long inc = block_inclusive_scan(sum, ws, &total);
    long long run = (part ? part[(size_t)k * ntile + blockIdx.x] : 0) + inc - sum;
#pragma unroll
    for (int j = 0; j < PER; j++) {
        s[PER * threadIdx.x + j] = run;
        run += v[j];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < PINYB200_SCAN_TILE; i += blockDim.x)
        if (base + i < n) out[base + i] = (int)s[i];
    if (!part && threadIdx.x == 0) {
        out[n] = (int)total;
        tot[k] = total;
    }
}

int scan_tiles(int n) { return n > 0 ? (n + PINYB200_SCAN_TILE - 1) / PINYB200_SCAN_TILE : 1; }

cudaError_t launch_scan(pinyb200_ctx *c, const int *gate, int n, int K, const int *count, int *out0, int *out1,
                        long long *tot, cudaStream_t st)
{
    if (K < 1 || K > 2 || n < 0) return cudaErrorInvalidValue;
    const int ntile = scan_tiles(n);
    ScanOut o{{out0, out1}};
    if (ntile == 1) {
        scan_tile_kernel<<<dim3(1, K), 1024, 0, st>>>(gate, n, count, 1, nullptr, o, tot);
        return cudaGetLastError();
    }
    if ((long long)ntile * K > c->scan_part_cap) return cudaErrorInvalidValue;
    scan_tile_sum_kernel<<<dim3(ntile, K), 1024, 0, st>>>(gate, n, count, ntile, c->d_scan_part);
    scan_part_kernel<<<K, 1024, 0, st>>>(gate, n, ntile, c->d_scan_part, o, tot);
    scan_tile_kernel<<<dim3(ntile, K), 1024, 0, st>>>(gate, n, count, ntile, c->d_scan_part, o, tot);
    return cudaGetLastError();
}

}  // namespace pinyb200
