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
#include "swe_fused.cuh"
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

// Whether (tile, blocks per SM, runs) is one of the SBP 4-2 linear configurations.
constexpr bool linear42_built(int tm, int occ, int runs)
{
    bool found = false;
#define CHSWE_IS_CFG(TM, OCC, RUNS) found = found || (tm == TM && occ == OCC && runs == RUNS);
    CHSWE_LINEAR_CFGS(CHSWE_IS_CFG)
#undef CHSWE_IS_CFG
    return found;
}

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

// CHSWE_CARVEOUT=1 asks for the largest shared-memory carveout on every kernel of the
// stage chain, so that an SM does not switch its L1 / shared-memory split between the
// small-memory edge kernels and the stage kernels that overlap them.
static inline bool carveout_max()
{
    static const bool on = [] {
        const char *e = std::getenv("CHSWE_CARVEOUT");
        return e && e[0] == '1';
    }();
    return on;
}
template <class K>
static inline cudaError_t set_carveout(K kern)
{
    return carveout_max() ? cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                                 (int)cudaSharedmemCarveoutMaxShared)
                          : cudaSuccess;
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
    // false: (occ, runs, ord, operator) is not a built configuration; nothing was launched
    static bool co2contra(int occ, int runs, int ord, int members, const T *y, T *w, T *es, const Dims &d,
                          const MetricView<T> &m, cudaStream_t st, const double *dtm);
    static bool stage(int occ, int runs, int ord, int members, const T *y, const T *w, const T *e, T *v0, T *y1,
                      T *acc, T *cmp, const Dims &d, const MetricView<T> &m, const StageArgs &a, cudaStream_t st);
    // this translation unit's copies of the panel links and cube edges (constant memory)
    static cudaError_t upload_tables(const Link *links, const int *cube_edges);
};

// The fused stage (swe_fused.cuh) of precision T: configurations (maximal tile
// height, resident blocks per SM the register allocation is capped for).  Every
// configuration takes tiles of at most FUSED_TW columns.
#define CHSWE_FUSED_CFGS_F(X) X(17, 4) X(25, 3) X(33, 2)
#define CHSWE_FUSED_CFGS_D(X) X(17, 2) X(25, 1)

template <class T>
struct FusedTU {
    static cudaError_t optin();
    // false: (th, occ) is not a built configuration, or the cube's tiles are too small
    static bool stage(int th, int occ, int members, const CUtensorMap &tmY, const CUtensorMap &tmM, const T *y,
                      const T *e, T *v0, T *y1, T *acc, T *cmp, const Dims &d, const FusedMetric<T> &fm,
                      const StageArgs &a, int *err, cudaStream_t st);
    static void strip(int members, const T *y, T *es, const Dims &d, const FusedMetric<T> &fm, const double *dtm,
                      cudaStream_t st);
    static cudaError_t upload_tables(const Link *links);
};

// One context of a group: its dimensions, metric, the state it advances and its
// scratch (the buffers of its own RK4 steps), and where its blocks sit in the grids.
template <class T>
struct GroupEntry {
    Dims d;
    MetricView<T> m;
    T *v;                  // the state (RK4 v0)
    T *ya, *yb;            // stage inputs / outputs
    T *acc, *cmp;          // RK4 accumulator; FP32 compensation (null in FP64)
    T *w, *es, *e;         // contravariant components, edge strips, synchronised edge values
    const double *Hm;      // per-member mean depth
    const double *dtm;     // per-member time step (0 freezes a member)
    unsigned gx, gy;       // stage tiles per panel direction
    unsigned nch;          // edge chunks per panel side
    unsigned tile0, edge0; // first flat block of this context in the tile and edge grids
};

constexpr int GROUP_MAX = 8;

template <class T>
struct GroupTable {
    int n;
    GroupEntry<T> e[GROUP_MAX];
};

// Group launches (swe_group.cuh) of precision T: the configurations (tile, blocks
// per SM, runs) they are built for, and one RK4 step of every context in the table
// as twelve launches (contravariant components, edge sync and stage, per stage).
#define CHSWE_GROUP_CFGS(X) X(17, 4, 0) X(25, 3, 0) X(33, 2, 0)

template <class T>
struct GroupTU {
    static cudaError_t optin();
    // false: (tm, occ, runs) is not a built group configuration; nothing was launched
    static bool rk4_step(int tm, int occ, int runs, const GroupTable<T> &g, unsigned tiles, unsigned edges,
                         cudaStream_t st);
    // this translation unit's copies of the panel links and cube edges (constant memory)
    static cudaError_t upload_tables(const Link *links, const int *cube_edges);
};

// Tiles of the fused stage: ceil((N+1) / FUSED_TW) columns and ceil((N+1) / th) rows
// of balanced tiles; the passes' ranges assume tiles of at least 13 x 9 points
// whenever a panel holds more than one.
static inline bool fused_grid(int N, int members, int th, dim3 &g)
{
    const int n = N + 1, gx = (n + FUSED_TW - 1) / FUSED_TW, gy = (n + th - 1) / th;
    if ((gx > 1 && n / gx < 13) || (gy > 1 && n / gy < 9)) return false;
    g = dim3(gx, gy, NPAN * members);
    return true;
}

}  // namespace chswe
