// group_tu.cuh -- definitions of GroupTU (swe_launch.cuh): the group launches of one
// precision.  Included by the group_*.cu translation units only.
#pragma once

#include "swe_group.cuh"

namespace chswe {

template <class T, int TM, int OCC, int RUNS>
static cudaError_t group_optin_cfg()
{
    const int sc = (int)Co2Layout<T, TM>::bytes(), ss = (int)StageLayout<T, TM>::bytes();
    cudaError_t e = cudaFuncSetAttribute(k_co2contra_group<T, TM, OCC, RUNS>, cudaFuncAttributeMaxDynamicSharedMemorySize, sc);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage_group<T, TM, OCC, 1, RUNS>, cudaFuncAttributeMaxDynamicSharedMemorySize, ss);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage_group<T, TM, OCC, 2, RUNS>, cudaFuncAttributeMaxDynamicSharedMemorySize, ss);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage_group<T, TM, OCC, 3, RUNS>, cudaFuncAttributeMaxDynamicSharedMemorySize, ss);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage_group<T, TM, OCC, 4, RUNS>, cudaFuncAttributeMaxDynamicSharedMemorySize, ss);
    if (e == cudaSuccess) e = set_carveout(k_co2contra_group<T, TM, OCC, RUNS>);
    if (e == cudaSuccess) e = set_carveout(k_stage_group<T, TM, OCC, 1, RUNS>);
    if (e == cudaSuccess) e = set_carveout(k_stage_group<T, TM, OCC, 2, RUNS>);
    if (e == cudaSuccess) e = set_carveout(k_stage_group<T, TM, OCC, 3, RUNS>);
    if (e == cudaSuccess) e = set_carveout(k_stage_group<T, TM, OCC, 4, RUNS>);
    return e;
}

template <class T>
cudaError_t GroupTU<T>::optin()
{
    cudaError_t e = cudaSuccess;
#define CHSWE_GOPTIN(TM, OCC, RUNS) \
    if (e == cudaSuccess) e = group_optin_cfg<T, TM, OCC, RUNS>();
    CHSWE_GROUP_CFGS(CHSWE_GOPTIN)
#undef CHSWE_GOPTIN
    if (e == cudaSuccess) e = set_carveout(k_edge_group<T>);
    return e;
}

template <class T, int TM, int OCC, int RUNS>
static void group_step(const GroupTable<T> &g, unsigned tiles, unsigned edges, cudaStream_t st)
{
    const size_t sc = Co2Layout<T, TM>::bytes(), ss = StageLayout<T, TM>::bytes();
    const dim3 gt(tiles), ge(edges);
    launch_k(k_co2contra_group<T, TM, OCC, RUNS>, gt, stage_block(), sc, st, g, 1);
    launch_k(k_edge_group<T>, ge, dim3(EDGE_THREADS), 0, st, g);
    launch_k(k_stage_group<T, TM, OCC, 1, RUNS>, gt, stage_block(), ss, st, g);
    launch_k(k_co2contra_group<T, TM, OCC, RUNS>, gt, stage_block(), sc, st, g, 2);
    launch_k(k_edge_group<T>, ge, dim3(EDGE_THREADS), 0, st, g);
    launch_k(k_stage_group<T, TM, OCC, 2, RUNS>, gt, stage_block(), ss, st, g);
    launch_k(k_co2contra_group<T, TM, OCC, RUNS>, gt, stage_block(), sc, st, g, 3);
    launch_k(k_edge_group<T>, ge, dim3(EDGE_THREADS), 0, st, g);
    launch_k(k_stage_group<T, TM, OCC, 3, RUNS>, gt, stage_block(), ss, st, g);
    launch_k(k_co2contra_group<T, TM, OCC, RUNS>, gt, stage_block(), sc, st, g, 4);
    launch_k(k_edge_group<T>, ge, dim3(EDGE_THREADS), 0, st, g);
    launch_k(k_stage_group<T, TM, OCC, 4, RUNS>, gt, stage_block(), ss, st, g);
}

template <class T>
bool GroupTU<T>::rk4_step(int tm, int occ, int runs, const GroupTable<T> &g, unsigned tiles, unsigned edges,
                          cudaStream_t st)
{
#define CHSWE_GSTEP(TM, OCC, RUNS)                          \
    if (tm == TM && occ == OCC && runs == RUNS) {           \
        group_step<T, TM, OCC, RUNS>(g, tiles, edges, st);  \
        return true;                                        \
    }
    CHSWE_GROUP_CFGS(CHSWE_GSTEP)
#undef CHSWE_GSTEP
    return false;
}

template <class T>
cudaError_t GroupTU<T>::upload_tables(const Link *links, const int *cube_edges)
{
    cudaError_t e = cudaMemcpyToSymbol(c_link, links, sizeof(Link) * NPAN * 4);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_cube_edge, cube_edges, sizeof(int) * 12 * 2);
    return e;
}

}  // namespace chswe
