// swe_launch.cuh -- host-side launch helpers shared by the C ABI (swe_api.cu) and the
// stage translation units (stage_*.cu): the kernel configurations, programmatic
// dependent launch, the tile grid, and StageTU, the entry points of the stage and
// contravariant kernels of one precision and tile size.  Each StageTU is compiled
// in a translation unit of its own: small device modules, built in parallel, whose
// generated code does not depend on how the compiler partitions one large module.
#pragma once

#include <cuda_runtime.h>

#include <cstdlib>

#include "swe_common.cuh"
#include "swe_kernels.cuh"

namespace chswe {

// Kernel configurations the stage kernels are built for: (maximal tile edge,
// resident blocks per SM the register allocation is capped for, stencil runs of
// several outputs per thread or one).  The advective operator's stage kernel is
// built for the first blocks-per-SM value of each tile only.
#define CHSWE_LINEAR_CFGS(X)                                                                                  \
    X(17, 3, 0) X(17, 4, 0) X(25, 2, 0) X(25, 3, 0) X(25, 4, 0) X(33, 2, 0) X(33, 3, 0) X(17, 3, 1) X(17, 4, 1) \
        X(25, 2, 1) X(25, 3, 1) X(25, 4, 1) X(33, 2, 1) X(33, 3, 1)
#define CHSWE_ADV_CFGS(X) X(17, 3, 0) X(25, 2, 0) X(33, 2, 0) X(17, 3, 1) X(25, 2, 1) X(33, 2, 1)
// SBP 2-1 stage kernels (linear operator): the first blocks-per-SM value of each
// tile, one output per element.
#define CHSWE_LINEAR21_CFGS(X) X(17, 3, 0) X(25, 2, 0) X(33, 2, 0)
// SBP 6-3 stage kernels: the same configurations
#define CHSWE_LINEAR63_CFGS(X) X(17, 3, 0) X(25, 2, 0) X(33, 2, 0)
// the advective operator in SBP 2-1 and 6-3: the same configurations
#define CHSWE_ADV21_CFGS(X) X(17, 3, 0) X(25, 2, 0) X(33, 2, 0)
#define CHSWE_ADV63_CFGS(X) X(17, 3, 0) X(25, 2, 0) X(33, 2, 0)

static inline dim3 stage_block() { return dim3(STAGE_THREADS, 1, 1); }

// The stage kernels are launched with programmatic stream serialization: each may
// start (and load its metric) while its predecessor finishes, and waits for the
// predecessor's results with griddepcontrol.wait.  CHSWE_PDL=0 in the environment
// launches them plainly.
static inline bool pdl_enabled()
{
    static const bool on = [] {
        const char *e = std::getenv("CHSWE_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}

template <typename... KArgs, typename... Args>
static inline void launch_k(void (*kern)(KArgs...), dim3 g, dim3 b, size_t smem, cudaStream_t st, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = g;
    cfg.blockDim = b;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kern, ((KArgs)args)...);
}
// Balanced tiles: ceil(N / (TM - 1)) tiles per direction, widths at most TM.
static inline dim3 stage_grid(int N, int members, int tm)
{
    const int nb = (N + tm - 2) / (tm - 1);
    return dim3(nb, nb, NPAN * members);
}


// The stage (k_stage) and contravariant (k_co2contra) kernels of precision T and
// maximal tile TM: every built (blocks per SM, runs, SBP order, operator) variant.
template <class T, int TM>
struct StageTU {
    // opt in to the dynamic shared memory of every variant (current device)
    static cudaError_t optin();
    static void co2contra(int occ, int runs, int ord, int members, const T *y, T *w, T *es, const Dims &d,
                          const MetricView<T> &m, cudaStream_t st, const double *dtm);
    static void stage(int occ, int runs, int ord, int members, const T *y, const T *w, const T *e, T *v0, T *y1,
                      T *acc, T *cmp, const Dims &d, const MetricView<T> &m, const StageArgs &a, cudaStream_t st);
    // this translation unit's copies of the panel links and cube edges (constant memory)
    static cudaError_t upload_tables(const Link *links, const int *cube_edges);
};

}  // namespace chswe
