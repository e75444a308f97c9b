// fused_tu.cuh -- definitions of FusedTU (swe_launch.cuh): the launches of the fused
// stage and edge-strip kernels of one precision.  Included by the fused_*.cu
// translation units only.
#pragma once

#include "swe_launch.cuh"

namespace chswe {

template <class T, int TH, int OCC>
static cudaError_t fused_optin_modes()
{
    const int sb = (int)FusedLayout<T, TH>::bytes();
    cudaError_t e = cudaFuncSetAttribute(k_fstage<T, TH, OCC, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, sb);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fstage<T, TH, OCC, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sb);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fstage<T, TH, OCC, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sb);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fstage<T, TH, OCC, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, sb);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fstage<T, TH, OCC, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, sb);
    for (int k = 0; k < 5 && e == cudaSuccess; k++) {
        void (*f[5])(CUtensorMap, CUtensorMap, const T *, const T *, T *, T *, T *, T *, Dims, FusedMetric<T>,
                     StageArgs, int *) = {k_fstage<T, TH, OCC, 0>, k_fstage<T, TH, OCC, 1>, k_fstage<T, TH, OCC, 2>,
                                           k_fstage<T, TH, OCC, 3>, k_fstage<T, TH, OCC, 4>};
        e = set_carveout(f[k]);
    }
    return e;
}

template <class T, int TH, int OCC>
static void fused_launch_modes(const dim3 &g, const CUtensorMap &tmY, const CUtensorMap &tmM, const T *y, const T *e,
                               T *v0, T *y1, T *acc, T *cmp, const Dims &d, const FusedMetric<T> &fm,
                               const StageArgs &a, int *err, cudaStream_t st)
{
    const size_t sb = FusedLayout<T, TH>::bytes();
    const dim3 b(FUSED_THREADS);
    switch (a.mode) {
    case 0: launch_k(k_fstage<T, TH, OCC, 0>, g, b, sb, st, tmY, tmM, y, e, v0, y1, acc, cmp, d, fm, a, err); break;
    case 1: launch_k(k_fstage<T, TH, OCC, 1>, g, b, sb, st, tmY, tmM, y, e, v0, y1, acc, cmp, d, fm, a, err); break;
    case 2: launch_k(k_fstage<T, TH, OCC, 2>, g, b, sb, st, tmY, tmM, y, e, v0, y1, acc, cmp, d, fm, a, err); break;
    case 3: launch_k(k_fstage<T, TH, OCC, 3>, g, b, sb, st, tmY, tmM, y, e, v0, y1, acc, cmp, d, fm, a, err); break;
    default: launch_k(k_fstage<T, TH, OCC, 4>, g, b, sb, st, tmY, tmM, y, e, v0, y1, acc, cmp, d, fm, a, err); break;
    }
}

template <class T>
cudaError_t FusedTU<T>::optin()
{
    cudaError_t e = cudaSuccess;
#define CHSWE_FOPTIN(TH, OCC) \
    if (e == cudaSuccess) e = fused_optin_modes<T, TH, OCC>();
    if constexpr (sizeof(T) == 4) {
        CHSWE_FUSED_CFGS_F(CHSWE_FOPTIN)
    } else {
        CHSWE_FUSED_CFGS_D(CHSWE_FOPTIN)
    }
#undef CHSWE_FOPTIN
    if (e == cudaSuccess) e = set_carveout(k_strip<T>);
    return e;
}

template <class T>
bool FusedTU<T>::stage(int th, int occ, int members, const CUtensorMap &tmY, const CUtensorMap &tmM, const T *y,
                       const T *e, T *v0, T *y1, T *acc, T *cmp, const Dims &d, const FusedMetric<T> &fm,
                       const StageArgs &a, int *err, cudaStream_t st)
{
    dim3 g;
    if (!fused_grid(d.N, members, th, g)) return false;
#define CHSWE_FSTG(TH, OCC)                                                                          \
    if (th == TH && occ == OCC) {                                                                    \
        fused_launch_modes<T, TH, OCC>(g, tmY, tmM, y, e, v0, y1, acc, cmp, d, fm, a, err, st);     \
        return true;                                                                                 \
    }
    if constexpr (sizeof(T) == 4) {
        CHSWE_FUSED_CFGS_F(CHSWE_FSTG)
    } else {
        CHSWE_FUSED_CFGS_D(CHSWE_FSTG)
    }
#undef CHSWE_FSTG
    return false;
}

template <class T>
void FusedTU<T>::strip(int members, const T *y, T *es, const Dims &d, const FusedMetric<T> &fm, const double *dtm,
                       cudaStream_t st)
{
    const dim3 g((d.N + 1 + STRIP_CHUNK - 1) / STRIP_CHUNK, NPAN * 4, members);
    launch_k(k_strip<T>, g, dim3(STRIP_THREADS), 0, st, y, es, d, fm, dtm);
}

template <class T>
cudaError_t FusedTU<T>::upload_tables(const Link *links)
{
    cudaError_t e = cudaMemcpyToSymbol(c_link, links, sizeof(Link) * NPAN * 4);
    double w[XROW_LEN];
    T wt[XROW_LEN];
    xrow42_table(w);
    for (int m = 0; m < XROW_LEN; m++) wt[m] = T(w[m]);
    if (e == cudaSuccess) {
        if constexpr (sizeof(T) == 4) e = cudaMemcpyToSymbol(g_xrow_f, wt, sizeof(wt));
        else e = cudaMemcpyToSymbol(g_xrow_d, wt, sizeof(wt));
    }
    return e;
}

}  // namespace chswe
