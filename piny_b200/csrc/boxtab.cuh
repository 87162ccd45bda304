// Many independent boxes per launch.
//
// A kernel body written against a VBlk (its block's place in the grid the
// single-box launch would have used) runs either as a plain kernel (VBlk
// from blockIdx/gridDim) or inside a batched kernel whose parameters carry
// a table of per-box arguments: the launch's blocks are the concatenation
// of every box's grid, and a fixed number of resident CTAs walks that
// (box, block) list in order -- a persistent loop, the heaviest boxes first.
// Bodies must reach their barriers uniformly across the block (as any
// kernel does); the loop adds one barrier between two blocks so that shared
// memory is not refilled while the previous block still reads it.
#pragma once

#include <algorithm>
#include <cstring>
#include <vector>

#include "internal.h"

namespace pinyb200 {

struct VBlk {
    int x, y;    // block index in the box's grid
    int gx, gy;  // the box's grid
};

__device__ __forceinline__ VBlk hw_blk() { return VBlk{(int)blockIdx.x, (int)blockIdx.y, (int)gridDim.x, (int)gridDim.y}; }

// Boxes per batched launch: the table rides in the kernel parameters
// (at most 32,764 bytes), so larger batches take several launches.
constexpr int kBoxTab = 32;

template <class A>
struct BoxTab {
    int n;                  // boxes in this launch
    int off[kBoxTab + 1];   // first block of box i in the launch; off[n] = blocks
    int gx[kBoxTab];        // x extent of box i's grid (y extent = blocks / gx)
    A arg[kBoxTab];
};

// Box of launch block w: the last i with off[i] <= w.
__device__ __forceinline__ int tab_box(const int *off, int n, int w)
{
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int m = (lo + hi) >> 1;
        if (off[m] <= w) lo = m;
        else hi = m;
    }
    return lo;
}

template <class A>
__device__ __forceinline__ VBlk tab_blk(const BoxTab<A> &t, int i, int w)
{
    const int l = w - t.off[i], gx = t.gx[i];
    return VBlk{l % gx, l / gx, gx, (t.off[i + 1] - t.off[i]) / gx};
}

// The persistent loop of a batched kernel over table t: binds box index i
// and VBlk vb for the body, then a block-wide barrier.
#define PINYB200_BOX_LOOP(t, i, vb, ...)                                         \
    for (int w_ = (int)blockIdx.x; w_ < (t).off[(t).n]; w_ += (int)gridDim.x) { \
        const int i = tab_box((t).off, (t).n, w_);                               \
        const VBlk vb = tab_blk((t), i, w_);                                     \
        __VA_ARGS__;                                                             \
        __syncthreads();                                                         \
    }

// Host side: collects (args, grid, work) entries and cuts them into tables
// of at most kBoxTab boxes, one persistent launch each.
template <class A>
struct BoxTabBuilder {
    struct Ent {
        A a;
        int gx, gy;
        double work;
    };
    std::vector<Ent> ent;
    void add(const A &a, int gx, int gy, double work)
    {
        if (gx > 0 && gy > 0) ent.push_back(Ent{a, gx, gy, work});
    }
    // tables, each box's blocks contiguous, heaviest boxes first
    std::vector<BoxTab<A>> tables() const
    {
        std::vector<Ent> e = ent;
        std::stable_sort(e.begin(), e.end(), [](const Ent &x, const Ent &y) { return x.work > y.work; });
        std::vector<BoxTab<A>> out;
        for (size_t k = 0; k < e.size(); k += kBoxTab) {
            BoxTab<A> t;
            memset(&t, 0, sizeof(t));
            t.n = (int)std::min<size_t>(kBoxTab, e.size() - k);
            t.off[0] = 0;
            for (int i = 0; i < t.n; i++) {
                const Ent &x = e[k + i];
                t.arg[i] = x.a;
                t.gx[i] = x.gx;
                t.off[i + 1] = t.off[i] + x.gx * x.gy;
            }
            out.push_back(t);
        }
        return out;
    }
};

// Waves of resident CTAs a batched launch holds (0: one CTA per block of
// the launch, which lets the block scheduler interleave launches of
// parallel graph branches).
#ifndef PINYB200_BATCH_WAVES
#define PINYB200_BATCH_WAVES 1
#endif

// CTAs of a persistent launch: the blocks of the launch, at most the SMs
// times the blocks of this kernel one SM holds (times the waves).
inline int persistent_grid(const void *func, int threads, size_t smem, int sm_count, int blocks)
{
    if (PINYB200_BATCH_WAVES <= 0) return std::max(1, blocks);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, threads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const long long cap = (long long)per_sm * sm_count * PINYB200_BATCH_WAVES;
    return (int)std::max<long long>(1, std::min<long long>(blocks, cap));
}

// One persistent launch per table of builder tb; `launch(table, grid)`
// issues the kernel.  Dynamic shared memory is opted in first (static plus
// dynamic may pass 48 KB below 48 KB of dynamic).
template <class A, class L>
inline cudaError_t launch_tables(const BoxTabBuilder<A> &tb, const void *fn, int threads, size_t smem, int sm_count,
                                 L &&launch)
{
    if (tb.ent.empty()) return cudaSuccess;
    if (smem > 0) {
        cudaError_t e = smem_optin(fn, (int)smem);
        if (e != cudaSuccess) return e;
    }
    for (const BoxTab<A> &t : tb.tables()) {
        launch(t, persistent_grid(fn, threads, smem, sm_count, t.off[t.n]));
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace pinyb200
