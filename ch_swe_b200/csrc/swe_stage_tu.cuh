// swe_stage_tu.cuh -- definitions of StageTU (swe_launch.cuh): the launches of the
// stage and contravariant kernels of one precision and tile size, for every built
// variant.  Included by the stage_*.cu translation units only.
#pragma once

#include "swe_launch.cuh"
#include "swe_tiled.cuh"

namespace chswe {

// The tiled kernels use more than 48 KB of dynamic shared memory: opt in once per
// device and element type (the attribute belongs to the device's context).
template <class T, int TM, int OCC, bool ADV, bool RUNS, int ORD>
static cudaError_t stage_smem_optin_modes()
{
    const int sb = (int)StageLayout<T, TM>::bytes();
    cudaError_t e = cudaFuncSetAttribute(k_stage<T, TM, OCC, 0, ADV, RUNS, ORD>, cudaFuncAttributeMaxDynamicSharedMemorySize, sb);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage<T, TM, OCC, 1, ADV, RUNS, ORD>, cudaFuncAttributeMaxDynamicSharedMemorySize, sb);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage<T, TM, OCC, 2, ADV, RUNS, ORD>, cudaFuncAttributeMaxDynamicSharedMemorySize, sb);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage<T, TM, OCC, 3, ADV, RUNS, ORD>, cudaFuncAttributeMaxDynamicSharedMemorySize, sb);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage<T, TM, OCC, 4, ADV, RUNS, ORD>, cudaFuncAttributeMaxDynamicSharedMemorySize, sb);
    if (e == cudaSuccess) e = set_carveout(k_stage<T, TM, OCC, 0, ADV, RUNS, ORD>);
    if (e == cudaSuccess) e = set_carveout(k_stage<T, TM, OCC, 1, ADV, RUNS, ORD>);
    if (e == cudaSuccess) e = set_carveout(k_stage<T, TM, OCC, 2, ADV, RUNS, ORD>);
    if (e == cudaSuccess) e = set_carveout(k_stage<T, TM, OCC, 3, ADV, RUNS, ORD>);
    if (e == cudaSuccess) e = set_carveout(k_stage<T, TM, OCC, 4, ADV, RUNS, ORD>);
    return e;
}

template <class T, int TM, int OCC, bool ADV, bool RUNS, int ORD>
static void launch_stage_modes(int members, const T *y, const T *w, const T *e, T *v0, T *y1, T *acc, T *cmp,
                               const Dims &d, const MetricView<T> &m, const StageArgs &a, cudaStream_t st)
{
    const dim3 g = stage_grid(d.N, members, TM);
    const size_t sb = StageLayout<T, TM>::bytes();
    switch (a.mode) {
    case 0: launch_k(k_stage<T, TM, OCC, 0, ADV, RUNS, ORD>, g, stage_block(), sb, st, y, w, e, v0, y1, acc, cmp, d, m, a); break;
    case 1: launch_k(k_stage<T, TM, OCC, 1, ADV, RUNS, ORD>, g, stage_block(), sb, st, y, w, e, v0, y1, acc, cmp, d, m, a); break;
    case 2: launch_k(k_stage<T, TM, OCC, 2, ADV, RUNS, ORD>, g, stage_block(), sb, st, y, w, e, v0, y1, acc, cmp, d, m, a); break;
    case 3: launch_k(k_stage<T, TM, OCC, 3, ADV, RUNS, ORD>, g, stage_block(), sb, st, y, w, e, v0, y1, acc, cmp, d, m, a); break;
    default: launch_k(k_stage<T, TM, OCC, 4, ADV, RUNS, ORD>, g, stage_block(), sb, st, y, w, e, v0, y1, acc, cmp, d, m, a); break;
    }
}

template <class T, int TMX>
cudaError_t StageTU<T, TMX>::optin()
{
    cudaError_t e = cudaSuccess;
#define CHSWE_OPTIN(TM, OCC, RUNS, ADV, ORD)                                                                       \
    if constexpr (TM == TMX) {                                                                                     \
        if (e == cudaSuccess && !ADV)                                                                              \
            e = cudaFuncSetAttribute(k_co2contra<T, TM, OCC, RUNS, ORD>,                                           \
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Co2Layout<T, TM>::bytes()); \
        if (e == cudaSuccess && !ADV) e = set_carveout(k_co2contra<T, TM, OCC, RUNS, ORD>);                       \
        if (e == cudaSuccess) e = stage_smem_optin_modes<T, TM, OCC, ADV, RUNS, ORD>();                           \
    }
#define CHSWE_OPTIN_42(TM, OCC, RUNS) CHSWE_OPTIN(TM, OCC, RUNS, false, 42)
#define CHSWE_OPTIN_21(TM, OCC, RUNS) CHSWE_OPTIN(TM, OCC, RUNS, false, 21)
#define CHSWE_OPTIN_63(TM, OCC, RUNS) CHSWE_OPTIN(TM, OCC, RUNS, false, 63)
#define CHSWE_OPTIN_ADV(TM, OCC, RUNS) CHSWE_OPTIN(TM, OCC, RUNS, true, 42)
#define CHSWE_OPTIN_ADV21(TM, OCC, RUNS) CHSWE_OPTIN(TM, OCC, RUNS, true, 21)
#define CHSWE_OPTIN_ADV63(TM, OCC, RUNS) CHSWE_OPTIN(TM, OCC, RUNS, true, 63)
    CHSWE_LINEAR_CFGS(CHSWE_OPTIN_42)
    CHSWE_LINEAR21_CFGS(CHSWE_OPTIN_21)
    CHSWE_LINEAR63_CFGS(CHSWE_OPTIN_63)
    CHSWE_ADV_CFGS(CHSWE_OPTIN_ADV)
    CHSWE_ADV21_CFGS(CHSWE_OPTIN_ADV21)
    CHSWE_ADV63_CFGS(CHSWE_OPTIN_ADV63)
#undef CHSWE_OPTIN
#undef CHSWE_OPTIN_42
#undef CHSWE_OPTIN_21
#undef CHSWE_OPTIN_63
#undef CHSWE_OPTIN_ADV
#undef CHSWE_OPTIN_ADV21
#undef CHSWE_OPTIN_ADV63
    return e;
}

// ord: SBP order (42, 21 or 63).  Configurations are validated when set.
template <class T, int TMX>
bool StageTU<T, TMX>::co2contra(int occ, int runs, int ord, int members, const T *y, T *w, T *es, const Dims &d,
                                const MetricView<T> &m, cudaStream_t st, const double *dtm)
{
    const dim3 g = stage_grid(d.N, members, TMX);
#define CHSWE_CO2(TM, OCC, RUNS, ORD)                                                                             \
    if constexpr (TM == TMX) {                                                                                    \
        if (occ == OCC && runs == RUNS && ord == ORD) {                                                           \
            launch_k(k_co2contra<T, TM, OCC, RUNS, ORD>, g, stage_block(), Co2Layout<T, TM>::bytes(), st, y, w,  \
                     es, d, m, dtm);                                                                              \
            return true;                                                                                          \
        }                                                                                                         \
    }
#define CHSWE_CO2_42(TM, OCC, RUNS) CHSWE_CO2(TM, OCC, RUNS, 42)
#define CHSWE_CO2_21(TM, OCC, RUNS) CHSWE_CO2(TM, OCC, RUNS, 21)
#define CHSWE_CO2_63(TM, OCC, RUNS) CHSWE_CO2(TM, OCC, RUNS, 63)
    CHSWE_LINEAR_CFGS(CHSWE_CO2_42)
    CHSWE_LINEAR21_CFGS(CHSWE_CO2_21)
    CHSWE_LINEAR63_CFGS(CHSWE_CO2_63)
#undef CHSWE_CO2
#undef CHSWE_CO2_42
#undef CHSWE_CO2_21
#undef CHSWE_CO2_63
    return false;
}

// The advective variant exists for the first blocks-per-SM value of each tile only
// (the caller passes that value).
template <class T, int TMX>
bool StageTU<T, TMX>::stage(int occ, int runs, int ord, int members, const T *y, const T *w, const T *e, T *v0,
                            T *y1, T *acc, T *cmp, const Dims &d, const MetricView<T> &m, const StageArgs &a,
                            cudaStream_t st)
{
    const bool adv = a.A != nullptr;
#define CHSWE_STG(TM, OCC, RUNS, ADV, ORD)                                                                      \
    if constexpr (TM == TMX) {                                                                                  \
        if (occ == OCC && runs == RUNS && adv == ADV && ord == ORD) {                                           \
            launch_stage_modes<T, TM, OCC, ADV, RUNS, ORD>(members, y, w, e, v0, y1, acc, cmp, d, m, a, st);    \
            return true;                                                                                        \
        }                                                                                                       \
    }
#define CHSWE_STG_42(TM, OCC, RUNS) CHSWE_STG(TM, OCC, RUNS, false, 42)
#define CHSWE_STG_21(TM, OCC, RUNS) CHSWE_STG(TM, OCC, RUNS, false, 21)
#define CHSWE_STG_63(TM, OCC, RUNS) CHSWE_STG(TM, OCC, RUNS, false, 63)
#define CHSWE_STG_ADV(TM, OCC, RUNS) CHSWE_STG(TM, OCC, RUNS, true, 42)
#define CHSWE_STG_ADV21(TM, OCC, RUNS) CHSWE_STG(TM, OCC, RUNS, true, 21)
#define CHSWE_STG_ADV63(TM, OCC, RUNS) CHSWE_STG(TM, OCC, RUNS, true, 63)
    CHSWE_LINEAR_CFGS(CHSWE_STG_42)
    CHSWE_LINEAR21_CFGS(CHSWE_STG_21)
    CHSWE_LINEAR63_CFGS(CHSWE_STG_63)
    CHSWE_ADV_CFGS(CHSWE_STG_ADV)
    CHSWE_ADV21_CFGS(CHSWE_STG_ADV21)
    CHSWE_ADV63_CFGS(CHSWE_STG_ADV63)
#undef CHSWE_STG
#undef CHSWE_STG_42
#undef CHSWE_STG_21
#undef CHSWE_STG_63
#undef CHSWE_STG_ADV
#undef CHSWE_STG_ADV21
#undef CHSWE_STG_ADV63
    return false;
}

template <class T, int TMX>
cudaError_t StageTU<T, TMX>::upload_tables(const Link *links, const int *cube_edges)
{
    cudaError_t e = cudaMemcpyToSymbol(c_link, links, sizeof(Link) * NPAN * 4);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_cube_edge, cube_edges, sizeof(int) * 12 * 2);
    return e;
}

}  // namespace chswe
