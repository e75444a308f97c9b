// swe_group.cuh -- group launches: the RK4 stages of several contexts (cube sizes
// and member counts of their own, one precision, the linear operator on Ch in SBP
// 4-2) as one grid per kernel.  The flat block index runs over the contexts' tile
// grids one after another; each block looks its context up in the table passed by
// value (a __grid_constant__ parameter, read through the constant cache) and runs the
// same tile body as a plain launch of that context, so a context advanced in a group
// gets the bits it gets alone with the same kernel configuration.
#pragma once

#include "swe_launch.cuh"
#include "swe_tiled.cuh"

namespace chswe {

// The context of flat block b (the last whose first block is <= b).
template <class T>
__device__ __forceinline__ int group_entry(const GroupTable<T> &g, unsigned b, bool edge)
{
    int k = 0;
#pragma unroll 1
    for (int q = 1; q < g.n; q++)
        if (b >= (edge ? g.e[q].edge0 : g.e[q].tile0)) k = q;
    return k;
}

template <class T>
__device__ __forceinline__ Blk group_blk(const GroupEntry<T> &e, unsigned b)
{
    const unsigned per = e.gx * e.gy;
    return Blk{b % e.gx, (b % per) / e.gx, b / per, e.gx, e.gy};
}

// The stage input of RK4 stage s (1..4) and the buffer stage s writes (the order of
// the context's own steps: v -> yb -> ya -> yb -> v).
template <class T>
__device__ __forceinline__ const T *group_stage_in(const GroupEntry<T> &e, int s)
{
    return s == 1 ? e.v : (s == 3 ? e.ya : e.yb);
}

template <class T, int TM, int OCC, bool RUNS>
__global__ void __launch_bounds__(STAGE_THREADS, OCC) k_co2contra_group(const __grid_constant__ GroupTable<T> g, int s)
{
    const GroupEntry<T> &e = g.e[group_entry(g, blockIdx.x, false)];
    co2contra_tile<T, TM, OCC, RUNS, 42>(group_blk(e, blockIdx.x - e.tile0), group_stage_in(e, s), e.w, e.es, e.d,
                                         e.m, e.dtm);
}

template <class T>
__global__ void __launch_bounds__(EDGE_THREADS) k_edge_group(const __grid_constant__ GroupTable<T> g)
{
    const GroupEntry<T> &e = g.e[group_entry(g, blockIdx.x, true)];
    const unsigned b = blockIdx.x - e.edge0, rest = b / e.nch;
    edge_chunk<T, 42>(b % e.nch, e.nch, rest % (NPAN * 4), rest / (NPAN * 4), e.es, e.es, e.e, e.d, e.m, e.dtm);
}

template <class T, int TM, int OCC, int MODE, bool RUNS>
__global__ void __launch_bounds__(STAGE_THREADS, OCC) k_stage_group(const __grid_constant__ GroupTable<T> g)
{
    const GroupEntry<T> &e = g.e[group_entry(g, blockIdx.x, false)];
    T *y1 = MODE == 1 ? e.yb : (MODE == 2 ? e.ya : (MODE == 3 ? e.yb : nullptr));
    const StageArgs a{MODE, 0.0, e.Hm, e.dtm, nullptr, nullptr, nullptr, nullptr};
    stage_tile<T, TM, OCC, MODE, false, RUNS, 42>(group_blk(e, blockIdx.x - e.tile0), group_stage_in(e, MODE), e.w,
                                                  e.e, e.v, y1, e.acc, e.cmp, e.d, e.m, a);
}

}  // namespace chswe
