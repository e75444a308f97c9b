// swe_api.cu -- C ABI (include/chswe.h) of the B200 shallow-water step: context
// and state-vector management, host-side FP64 geometry, kernel launches and
// CUDA-graph capture of the RK4 loop.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "chswe.h"
#include "swe_common.cuh"
#include "swe_advective.cuh"
#include "swe_ah.cuh"
#include "swe_cgrid.cuh"
#include "swe_diff.cuh"
#include "swe_kernels.cuh"
#include "swe_launch.cuh"

namespace chswe {

// ---------------------------------------------------------------------------
// cube geometry (host)
// ---------------------------------------------------------------------------

// Panel frames of the reference's cube (cubed_sphere_topology_mod.f90:29-55):
// panel corner R*N + (i-1) EX + (j-1) EY on the integer lattice [0,N]^3, inward normal NRM.
static const int EX[NPAN][3] = {{-1, 0, 0}, {0, 0, -1}, {1, 0, 0}, {0, 0, 1}, {1, 0, 0}, {1, 0, 0}};
static const int EY[NPAN][3] = {{0, 1, 0}, {0, 1, 0}, {0, 1, 0}, {0, 1, 0}, {0, 0, 1}, {0, 0, -1}};
static const int NRM[NPAN][3] = {{0, 0, 1}, {-1, 0, 0}, {0, 0, -1}, {1, 0, 0}, {0, 1, 0}, {0, -1, 0}};
static const int ORG[NPAN][3] = {{1, 0, 0}, {1, 0, 1}, {0, 0, 1}, {0, 0, 0}, {0, 0, 0}, {0, 1, 1}};

static void lattice_point(int p, int i, int j, int n, int out[3])
{
    for (int d = 0; d < 3; d++) out[d] = n * ORG[p][d] + (i - 1) * EX[p][d] + (j - 1) * EY[p][d];
}

static void side_ij(int n, int s, int a, int &i, int &j)
{
    switch (s) {
    case SIDE_L: i = 1; j = a; break;
    case SIDE_R: i = n + 1; j = a; break;
    case SIDE_B: i = a; j = 1; break;
    default: i = a; j = n + 1; break;
    }
}

// Edge connectivity from the lattice: two vertices of side s of panel p are
// located on the sides of the other panels; their order gives the direction.
// The covariant component continuing across the edge keeps its sign when the
// coordinate that increases outward from p increases inward on the neighbour.
static void compute_links(Link L[NPAN][4])
{
    const int n = 4;
    for (int p = 0; p < NPAN; p++)
        for (int s = 0; s < 4; s++) {
            int i1, j1, i2, j2, P1[3], P2[3];
            side_ij(n, s, 2, i1, j1);
            side_ij(n, s, 3, i2, j2);
            lattice_point(p, i1, j1, n, P1);
            lattice_point(p, i2, j2, n, P2);
            L[p][s] = Link{-1, -1, 0, 0, 0};
            for (int q = 0; q < NPAN; q++) {
                if (q == p) continue;
                for (int s2 = 0; s2 < 4; s2++) {
                    int a1 = -1, a2 = -1;
                    for (int a = 1; a <= n + 1; a++) {
                        int ii, jj, X[3];
                        side_ij(n, s2, a, ii, jj);
                        lattice_point(q, ii, jj, n, X);
                        if (X[0] == P1[0] && X[1] == P1[1] && X[2] == P1[2]) a1 = a;
                        if (X[0] == P2[0] && X[1] == P2[1] && X[2] == P2[2]) a2 = a;
                    }
                    if (a1 > 0 && a2 > 0) {
                        int rev = a2 < a1;
                        int out_p = (s == SIDE_R || s == SIDE_T) ? 1 : -1;
                        int in_q = (s2 == SIDE_L || s2 == SIDE_B) ? 1 : -1;
                        L[p][s] = Link{q, s2, rev, out_p * in_q, rev ? -1 : 1};
                    }
                }
            }
        }
}

// Host FP64 metric of the equiangular panel (metric_2d_ecs_mod.f90:338-411):
// X = tan(alpha), Y = tan(beta), sigma = sqrt(1 + X^2 + Y^2).
struct HostMetric {
    int nx, ny;
    std::vector<double> J, Q1, Q2, Q3;   // [j][i], panel independent
};

static HostMetric host_metric(int N, double shift_i, double shift_j)
{
    const double pi = 3.141592653589793238462643383279502884;
    HostMetric m;
    m.nx = shift_i == 0.0 ? N + 1 : N;
    m.ny = shift_j == 0.0 ? N + 1 : N;
    const double a0 = -0.25 * pi, a1 = 0.25 * pi;
    const double hx = (a1 - a0) / ((double)m.nx - 1 + 2.0 * shift_i);
    const double hy = (a1 - a0) / ((double)m.ny - 1 + 2.0 * shift_j);
    m.J.resize((size_t)m.nx * m.ny); m.Q1 = m.J; m.Q2 = m.J; m.Q3 = m.J;
    for (int j = 1; j <= m.ny; j++) {
        double tb = std::tan(a0 + (j - 1 + shift_j) * hy);
        for (int i = 1; i <= m.nx; i++) {
            double ta = std::tan(a0 + (i - 1 + shift_i) * hx);
            double sg = std::sqrt(1.0 + ta * ta + tb * tb), s2 = sg * sg;
            size_t k = (size_t)(j - 1) * m.nx + (i - 1);
            m.Q1[k] = s2 / (1.0 + ta * ta);
            m.Q2[k] = s2 * ta * tb / ((1 + ta * ta) * (1 + tb * tb));
            m.Q3[k] = s2 / (1.0 + tb * tb);
            m.J[k] = (1.0 + ta * ta) * (1.0 + tb * tb) / (sg * sg * sg);
        }
    }
    return m;
}

// Unit position vector of an xy vertex on panel p (ecs_proto2realface, identity rotation).
static void vertex_r(int N, int p, int i, int j, double r[3])
{
    const double pi = 3.141592653589793238462643383279502884;
    const double hx = (0.25 * pi - (-0.25 * pi)) / (double)N;
    double ta = std::tan(-0.25 * pi + (i - 1) * hx), tb = std::tan(-0.25 * pi + (j - 1) * hx);
    double sg = std::sqrt(1.0 + ta * ta + tb * tb);
    double rp[3] = {ta / sg, tb / sg, 1.0 / sg};
    for (int d = 0; d < 3; d++) r[d] = EX[p][d] * rp[0] + EY[p][d] * rp[1] - NRM[p][d] * rp[2];
}

// Proto-face tangent vectors (metric_2d_ecs_mod.f90:136-199) for the vector-sync weights.
static void a1p(double al, double be, double a[3])
{
    double ta = std::tan(al), tb = std::tan(be);
    double s = std::pow(1.0 + std::pow(ta, 2.0) + std::pow(tb, 2.0), 1.5);
    a[0] = (1.0 + std::pow(ta, 2.0)) * (1.0 + std::pow(tb, 2.0)) / s;
    a[1] = -ta * tb * (1.0 + std::pow(ta, 2.0)) / s;
    a[2] = -ta * (1.0 + std::pow(ta, 2.0)) / s;
}
static void a2p(double al, double be, double a[3])
{
    double ta = std::tan(al), tb = std::tan(be);
    double s = std::pow(1.0 + std::pow(ta, 2.0) + std::pow(tb, 2.0), 1.5);
    a[0] = -ta * tb * (1.0 + std::pow(tb, 2.0)) / s;
    a[1] = (1.0 + std::pow(ta, 2.0)) * (1.0 + std::pow(tb, 2.0)) / s;
    a[2] = -tb * (1.0 + std::pow(tb, 2.0)) / s;
}
static void b1p(double al, double be, double b[3])
{
    double ta = std::tan(al), tb = std::tan(be), sg = std::sqrt(1.0 + ta * ta + tb * tb);
    b[0] = (1.0 + tb * tb - (ta * tb) * (ta * tb) / (1.0 + ta * ta)) / sg;
    b[1] = 0.0;
    b[2] = -ta * (1.0 + tb * tb / (1 + ta * ta)) / sg;
}
static void b2p(double al, double be, double b[3])
{
    double ta = std::tan(al), tb = std::tan(be), sg = std::sqrt(1.0 + ta * ta + tb * tb);
    b[0] = 0.0;
    b[1] = ((1 + ta * ta) - (ta * tb) * (ta * tb) / (1 + tb * tb)) / sg;
    b[2] = -tb * (ta * ta / (1 + tb * tb) + 1.0) / sg;
}

// Covariant ECS vector-sync weights (ecs_Ah_vec_sync_factory_mod.f90:97-158).
static void sync_weights(int N, std::vector<double> &qb, std::vector<double> &qt, std::vector<double> &ql,
                         std::vector<double> &qr)
{
    const double pi = 3.141592653589793238462643383279502884, q = 0.25 * pi;
    const double hx = (0.25 * pi - (-0.25 * pi)) / (double)N;
    qb.resize(N + 1); qt.resize(N + 1); ql.resize(N + 1); qr.resize(N + 1);
    for (int i = 1; i <= N + 1; i++) {
        double al = -0.25 * pi + (i - 1) * hx, a[3], v[3];
        a2p(al, -q, a); b1p(al, q, v);
        qb[i - 1] = a[0] * v[0] + a[1] * (-v[2]) + a[2] * v[1];
        a2p(al, q, a); b1p(al, -q, v);
        qt[i - 1] = a[0] * v[0] + a[1] * v[2] + a[2] * (-v[1]);
        double be = al;
        a1p(-q, be, a); b2p(q, be, v);
        ql[i - 1] = a[0] * (-v[2]) + a[1] * v[1] + a[2] * v[0];
        a1p(q, be, a); b2p(-q, be, v);
        qr[i - 1] = a[0] * v[2] + a[1] * v[1] + a[2] * (-v[0]);
    }
}

}  // namespace chswe

using namespace chswe;

// ---------------------------------------------------------------------------
// context and state vectors
// ---------------------------------------------------------------------------

template <class T>
struct DevMetric {
    T *base = nullptr;   // one allocation for everything below
    MetricView<T> v{};
};

// Metric of the Ah operator on the device.
template <class T>
struct DevAh {
    T *base = nullptr;
    AhView<T> v{};
};

// Static tables of the advective operator on the device.
template <class T>
struct DevAdv {
    T *base = nullptr;
    int *ibase = nullptr;
    AdvView<T> v{};
};

struct swe_ctx {
    swe_cfg cfg{};
    Dims dims{};
    int device = 0;
    cudaStream_t own_stream = nullptr, stream = nullptr;
    // advective operator: a second stream and events for the stage's independent
    // kernels (h averaging, wind halo, wind at the vertices), forked off the stream
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_havg = nullptr, ev_co2 = nullptr, ev_side = nullptr;
    bool branches = true;            // fork the advective stage (when the side stream exists); autotuned
    std::string err;
    long long launches = 0;
    size_t elem = 8;                 // bytes per element
    size_t box_elems = 0;            // elements of one state vector (all members)
    // device metric (the context uses the one matching its precision)
    DevMetric<double> m64;
    DevMetric<float> m32;
    double *Hm = nullptr;            // per-member H (device)
    std::vector<double> Hhost;
    // scratch (stage buffers and contravariant intermediates)
    void *ya = nullptr, *yb = nullptr, *acc = nullptr, *w = nullptr;
    void *edge = nullptr;            // synchronised panel-boundary values of the current stage
    void *es = nullptr;              // edge strips of the current stage (k_co2contra -> k_edge)
    // FP64 quadrature weights (J hx hy Ax Ay) on xy, y, x and o (cell-centre) meshes, [N+1][P]
    double *qw = nullptr;
    // FP64 tables of the curl and enstrophy on the o mesh (built on first use): J a
    // (one box), the Coriolis parameter f (one box per panel); then 6 N^2 curl values
    double *otab = nullptr;
    // lat-lon regrid of h (swe_regrid_latlon), built on first use for a grid size:
    // ints = per point (panel, x index, y index), then the ECS halo line indices;
    // reals = per point (wx[4], wy[4]), the ECS halo weights, the extended field, the output
    int ll_nlat = 0, ll_nlon = 0;
    int *ll_i = nullptr;
    double *ll_d = nullptr;
    // lat-lon regrid of the curl (cell centres, ECS_O halo), built on first use for a grid size
    int llo_nlat = 0, llo_nlon = 0;
    int *llo_i = nullptr;
    double *llo_d = nullptr;
    double *red = nullptr;           // reduction partials
    unsigned char *pinned = nullptr; // pinned host staging for uploads/downloads (whole batch)
    // captured RK4 step
    cudaGraphExec_t graph = nullptr;   // one RK4 step
    cudaGraphExec_t graphk = nullptr;  // GRAPH_STEPS RK4 steps
    const void *graph_v0 = nullptr;
    double graph_dt = 0.0;
    int graph_kernels = 0, graphk_kernels = 0;
    int tile = 33;                   // maximal tile edge of the stage kernels (17, 25 or 33)
    int occ = 2;                     // resident blocks per SM of the stage kernels' register cap
    int runs = 0;                    // 1: stencil runs of several outputs per thread
    int ord = 42;                    // SBP order of the Ch operators (42 or 21)
    // fused stage (swe_fused.cuh) of the linear Ch 4-2 operator: selected instead of the
    // three split kernels when `fused`; (fth, focc) is its configuration.  The split
    // configuration above stays valid for the diagnostics that launch k_co2contra.
    bool fused = false;
    int fth = 25, focc = 3;
    void *fmet = nullptr;            // FM_BOXES metric boxes of the fused stage (built on first use)
    CUtensorMap tm_metric;           // TMA map of fmet
    int *derr = nullptr;             // device error word: a bounded wait in a kernel gave up
    bool launch_miss = false;        // a stage or contravariant launch found no built configuration
    bool graph_members = false;      // the cached graph uses the per-member time steps
    double *dtm = nullptr;           // per-member time steps (device), swe_rk4_steps_members
    // advective operator (cfg.operator_kind == SWE_OP_ADVECTIVE)
    bool adv = false;
    DevAdv<double> a64;
    DevAdv<float> a32;
    void *fl = nullptr, *adt = nullptr;   // mass flux, advective tendencies (state boxes)
    void *fs = nullptr;              // mass-flux edge strips
    void *vh = nullptr;              // covariant wind at the virtual points beyond the panel edges
    void *hb = nullptr;              // panel-boundary h before the in-place averaging
    void *hs = nullptr;              // orography h_surf (one field box of panels), swe_set_orography
    double *ones = nullptr;          // per-member depth factor 1 (dh = -div F)
    double *negones = nullptr;       // per-member factor -1: the linear stage's dh is then div (outputs)
    // Ah staggering (cfg.staggering == SWE_STAG_AH): h, u, v on the vertices
    bool ah = false;
    DevAh<double> ah64;
    DevAh<float> ah32;
    double *qa = nullptr;            // SBP_Ah quadrature weights J hx hy Ax Ay at the vertices (one box)
    void *dif = nullptr;             // diffusion scratch: 5 sets of [member][4 fields][panel][box] (first use)
    int dif_order = 0;               // the diffusion step after every RK4 step (0: none; swe_set_diffusion)
    double dif_uv = 0.0, dif_h = 0.0;
    void *dif_b = nullptr;           // contravariant basis b1, b2 of the vertices, [panel][6][box] (first use)
    // C staggering (cfg.staggering == SWE_STAG_C): h on the cell centres, u on the x
    // points, v on the y points; the C-grid gradient, divergence and co2contra
    bool cstag = false;
    void *cmet = nullptr;            // CMetric boxes (swe_cgrid.cuh)
};

struct swe_stvec {
    swe_ctx *ctx = nullptr;
    void *d = nullptr;       // state
    float *cmp = nullptr;    // Kahan compensation of the FP32 RK4 state update
};

static void drop_graph(swe_ctx *c);

static int fail(swe_ctx *c, int code, const char *fmt, ...)
{
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        c->err = buf;
    }
    return code;
}

#define CU(ctx, call)                                                                                   \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) return fail((ctx), SWE_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// A stage or contravariant launch that found no built configuration (nothing was
// launched), or a CUDA launch error.
#define CU_LAUNCHED(ctx)                                                                                        \
    do {                                                                                                        \
        if ((ctx)->launch_miss) {                                                                               \
            (ctx)->launch_miss = false;                                                                         \
            return fail((ctx), SWE_EINVAL,                                                                      \
                        "no built stage-kernel configuration matches the context's (tile, blocks per SM, runs, " \
                        "SBP order, operator); nothing was launched");                                          \
        }                                                                                                       \
        CU(ctx, cudaGetLastError());                                                                            \
    } while (0)

static bool g_tables_ready[64] = {false};

// Maximal tile sizes the stage kernels are built for; ceil(N / (TM - 1)) balanced
// tiles per direction always fit, whatever N.
static bool valid_tile(int tm) { return tm == 17 || tm == 25 || tm == 33; }
struct KernelCfg {
    int tile, occ, runs;
};
#define CHSWE_CFG_ENTRY(TM, OCC, RUNS) {TM, OCC, RUNS},
static const KernelCfg k_cfgs[] = {CHSWE_LINEAR_CFGS(CHSWE_CFG_ENTRY)};
static const KernelCfg k_cfgs21[] = {CHSWE_LINEAR21_CFGS(CHSWE_CFG_ENTRY)};
static const KernelCfg k_cfgs63[] = {CHSWE_LINEAR63_CFGS(CHSWE_CFG_ENTRY)};
#undef CHSWE_CFG_ENTRY
static const int N_CFGS = sizeof(k_cfgs) / sizeof(k_cfgs[0]);
static const int N_CFGS21 = sizeof(k_cfgs21) / sizeof(k_cfgs21[0]);
static const int N_CFGS63 = sizeof(k_cfgs63) / sizeof(k_cfgs63[0]);
static int default_occ(int tm) { return tm == 17 ? 3 : 2; }
// the configurations built for SBP order ord
static const KernelCfg *cfgs_of(int ord, int *count)
{
    *count = ord == 21 ? N_CFGS21 : (ord == 63 ? N_CFGS63 : N_CFGS);
    return ord == 21 ? k_cfgs21 : (ord == 63 ? k_cfgs63 : k_cfgs);
}
static bool valid_cfg(int ord, int tm, int occ, int runs)
{
    int nc = 0;
    const KernelCfg *cs = cfgs_of(ord, &nc);
    for (int k = 0; k < nc; k++)
        if (cs[k].tile == tm && cs[k].occ == occ && cs[k].runs == runs) return true;
    return false;
}
// edge-strip lines per panel side for SBP order ord
static int ord_strip_lines(int ord) { return ord == 63 ? strip_lines<63>() : strip_lines<42>(); }
// Default before autotuning: tiles of about 24 points for the smaller cubes.
static int default_tile(int N) { return N <= 96 ? 25 : 33; }

static void cube_edges(int out[12][2]);

// The panel links and cube edges into the constant memory of this unit and of every
// stage translation unit (each holds its own copy), on the current device.
static cudaError_t upload_link_tables()
{
    Link L[NPAN][4];
    compute_links(L);
    int ce[12][2];
    cube_edges(ce);
    const Link *l = &L[0][0];
    const int *q = &ce[0][0];
    cudaError_t e = cudaMemcpyToSymbol(c_link, L, sizeof(L));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_cube_edge, ce, sizeof(ce));
    if (e == cudaSuccess) e = StageTU<float, 17>::upload_tables(l, q);
    if (e == cudaSuccess) e = StageTU<float, 25>::upload_tables(l, q);
    if (e == cudaSuccess) e = StageTU<float, 33>::upload_tables(l, q);
    if (e == cudaSuccess) e = StageTU<double, 17>::upload_tables(l, q);
    if (e == cudaSuccess) e = StageTU<double, 25>::upload_tables(l, q);
    if (e == cudaSuccess) e = StageTU<double, 33>::upload_tables(l, q);
    if (e == cudaSuccess) e = FusedTU<float>::upload_tables(l);
    if (e == cudaSuccess) e = FusedTU<double>::upload_tables(l);
    if (e == cudaSuccess) e = GroupTU<float>::upload_tables(l, q);
    if (e == cudaSuccess) e = GroupTU<double>::upload_tables(l, q);
    return e;
}

static int upload_tables(swe_ctx *c)
{
    if (c->device >= 0 && c->device < 64 && g_tables_ready[c->device]) return SWE_OK;
    CU(c, upload_link_tables());
    if (c->device >= 0 && c->device < 64) g_tables_ready[c->device] = true;
    return SWE_OK;
}

// Build the metric arrays in FP64 on the host and store them in precision T.
template <class T>
static int build_metric(swe_ctx *c, DevMetric<T> &dm)
{
    const int N = c->cfg.N, P = c->dims.P;
    const size_t box = (size_t)c->dims.ps;
    // 8 panel-independent boxes + fJ2 (6 boxes) + 4 edge vectors of N+1 + the edge tables
    // (ej: 4 sides x up to 7 lines, ef: 24, ea: 4, each of N+1)
    const size_t n_el = 8 * box + 6 * box + 4 * (size_t)(N + 1) + 56 * (size_t)(N + 1);
    std::vector<T> h(n_el, T(0));
    HostMetric my = host_metric(N, 0.5, 0.0), mx = host_metric(N, 0.0, 0.5), mxy = host_metric(N, 0.0, 0.0);
    const double a = c->cfg.radius;
    T *Q11y = h.data(), *iJy = Q11y + box, *Jy = iJy + box, *Q22x = Jy + box, *iJx = Q22x + box, *Jx = iJx + box,
      *JQ12 = Jx + box, *iJa = JQ12 + box, *fJ2 = iJa + box, *qb = fJ2 + 6 * box, *qt = qb + (N + 1),
      *ql = qt + (N + 1), *qr = ql + (N + 1);
    for (int j = 1; j <= N + 1; j++)
        for (int i = 1; i <= N; i++) {
            size_t k = (size_t)(j - 1) * my.nx + (i - 1), o = (size_t)box_off(P, i, j);
            Q11y[o] = T(my.Q1[k]); iJy[o] = T(1.0 / my.J[k]); Jy[o] = T(my.J[k]);
        }
    for (int j = 1; j <= N; j++)
        for (int i = 1; i <= N + 1; i++) {
            size_t k = (size_t)(j - 1) * mx.nx + (i - 1), o = (size_t)box_off(P, i, j);
            Q22x[o] = T(mx.Q3[k]); iJx[o] = T(1.0 / mx.J[k]); Jx[o] = T(mx.J[k]);
        }
    for (int j = 1; j <= N + 1; j++)
        for (int i = 1; i <= N + 1; i++) {
            size_t k = (size_t)(j - 1) * mxy.nx + (i - 1), o = (size_t)box_off(P, i, j);
            JQ12[o] = T(mxy.J[k] * mxy.Q2[k]);
            iJa[o] = T(1.0 / (mxy.J[k] * a));
            for (int p = 0; p < NPAN; p++) {
                double f;
                if (c->cfg.coriolis_constant) {
                    f = c->cfg.omega;
                } else {
                    double r[3];
                    vertex_r(N, p, i, j, r);
                    const double *ax = c->cfg.rotation_axis;
                    double pr = (ax[0] * r[0] + ax[1] * r[1] + ax[2] * r[2]) /
                                std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                    f = 2 * c->cfg.omega * pr;
                }
                fJ2[p * box + o] = T(f * mxy.J[k] * mxy.J[k]);
            }
        }
    std::vector<double> vb, vt, vl, vr;
    sync_weights(N, vb, vt, vl, vr);
    for (int i = 0; i <= N; i++) { qb[i] = T(vb[i]); qt[i] = T(vt[i]); ql[i] = T(vl[i]); qr[i] = T(vr[i]); }

    T *d = nullptr;
    if (cudaMalloc(&d, n_el * sizeof(T)) != cudaSuccess) return fail(c, SWE_ENOMEM, "metric allocation failed");
    dm.base = d;
    CU(c, cudaMemcpy(d, h.data(), n_el * sizeof(T), cudaMemcpyHostToDevice));
    MetricView<T> &v = dm.v;
    v.Q11y = d; v.iJy = d + box; v.Jy = d + 2 * box; v.Q22x = d + 3 * box; v.iJx = d + 4 * box; v.Jx = d + 5 * box;
    v.JQ12 = d + 6 * box; v.iJa = d + 7 * box; v.fJ2 = d + 8 * box;
    v.qb = d + 14 * box; v.qt = v.qb + (N + 1); v.ql = v.qt + (N + 1); v.qr = v.ql + (N + 1);
    T *ej = d + 14 * box + 4 * (N + 1), *ef = ej + 28 * (N + 1), *ea = ef + 24 * (N + 1);
    v.ej = ej; v.ef = ef; v.ea = ea;
    const double pi = 3.141592653589793238462643383279502884;
    const double hx = (0.25 * pi - (-0.25 * pi)) / (double)N;
    v.inv_hxa = T(1.0 / (hx * a));
    v.inv_hx = T(1.0 / hx);
    v.grav = T(c->cfg.grav);
    k_edge_tables<T><<<(N + 1 + 127) / 128, 128, 0, c->stream>>>(v, c->dims, ej, ef, ea, ord_strip_lines(c->ord));
    CU(c, cudaGetLastError());
    CU(c, cudaStreamSynchronize(c->stream));
    return SWE_OK;
}

// ---------------------------------------------------------------------------
// fused stage: metric boxes and TMA tensor maps
// ---------------------------------------------------------------------------
// cuTensorMapEncodeTiled from the driver, through the runtime (no -lcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
        return (PFN_cuTensorMapEncodeTiled_v12000)p;
    }();
    return fn;
}

// A 2-D map over `nrows` rows of P elements at base, with tiles of bw x bh elements.
static bool encode_rows(CUtensorMap *m, const void *base, size_t elem, int P, int64_t nrows, int bw, int bh)
{
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)P, (cuuint64_t)nrows};
    const cuuint64_t strides[1] = {(cuuint64_t)P * elem};
    const cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)bh};
    const cuuint32_t es[2] = {1, 1};
    return enc(m, elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(base),
               dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// TMA tile of the fused stage for maximal tile height th: box width by precision, th + 8 rows.
static int fused_box_w(const swe_ctx *c) { return c->elem == 8 ? FusedLayout<double, 17>::SW : FusedLayout<float, 17>::SW; }

// The fused stage's metric, FP64 on the host and stored in the context's precision:
// JQ12 = J Qi12 (xy), JQ11 = J Qi11 and 1/J (y mesh), JQ22 = J Qi22 and 1/J (x mesh),
// 1/(J a) (xy) and f J^2 of every panel, one panel box each (FM_* order).
template <class T>
static int build_fused_metric(swe_ctx *c, const MetricView<T> &mv)
{
    const int N = c->cfg.N, P = c->dims.P;
    const size_t box = (size_t)c->dims.ps;
    std::vector<T> h((size_t)FM_BOXES * box, T(0));
    HostMetric my = host_metric(N, 0.5, 0.0), mx = host_metric(N, 0.0, 0.5), mxy = host_metric(N, 0.0, 0.0);
    const double a = c->cfg.radius;
    T *JQ12 = h.data() + FM_JQ12 * box, *JQ11 = h.data() + FM_JQ11Y * box, *iJy = h.data() + FM_IJY * box,
      *JQ22 = h.data() + FM_JQ22X * box, *iJx = h.data() + FM_IJX * box, *iJa = h.data() + FM_IJA * box;
    for (int j = 1; j <= N + 1; j++)
        for (int i = 1; i <= N; i++) {
            size_t k = (size_t)(j - 1) * my.nx + (i - 1), o = (size_t)box_off(P, i, j);
            JQ11[o] = T(my.J[k] * my.Q1[k]);
            iJy[o] = T(1.0 / my.J[k]);
        }
    for (int j = 1; j <= N; j++)
        for (int i = 1; i <= N + 1; i++) {
            size_t k = (size_t)(j - 1) * mx.nx + (i - 1), o = (size_t)box_off(P, i, j);
            JQ22[o] = T(mx.J[k] * mx.Q3[k]);
            iJx[o] = T(1.0 / mx.J[k]);
        }
    for (int j = 1; j <= N + 1; j++)
        for (int i = 1; i <= N + 1; i++) {
            size_t k = (size_t)(j - 1) * mxy.nx + (i - 1), o = (size_t)box_off(P, i, j);
            JQ12[o] = T(mxy.J[k] * mxy.Q2[k]);
            iJa[o] = T(1.0 / (mxy.J[k] * a));
        }
    T *d = nullptr;
    if (cudaMalloc(&d, h.size() * sizeof(T)) != cudaSuccess) return fail(c, SWE_ENOMEM, "fused metric allocation failed");
    c->fmet = d;
    CU(c, cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    // f J^2 per panel: the same values the split kernels use
    CU(c, cudaMemcpy(d + FM_FJ2 * box, mv.fJ2, NPAN * box * sizeof(T), cudaMemcpyDeviceToDevice));
    if (!encode_rows(&c->tm_metric, d, sizeof(T), P, (int64_t)FM_BOXES * (N + 1 + 2 * MG), fused_box_w(c), c->fth + 8))
        return fail(c, SWE_ECUDA, "TMA tensor map of the fused metric");
    return SWE_OK;
}

// The fused stage serves the linear operator on the Ch grid in SBP 4-2.
static bool fused_supported(const swe_ctx *c) { return !c->adv && !c->ah && c->ord == 42; }

static bool fused_cfg_built(const swe_ctx *c, int th, int occ)
{
#define CHSWE_FCHK(TH, OCC) if (th == TH && occ == OCC) return true;
    if (c->elem == 4) {
        CHSWE_FUSED_CFGS_F(CHSWE_FCHK)
    } else {
        CHSWE_FUSED_CFGS_D(CHSWE_FCHK)
    }
#undef CHSWE_FCHK
    return false;
}

// Select the fused stage with configuration (th, occ): builds its metric on first use
// and re-encodes the metric map for the tile height.
static int select_fused(swe_ctx *c, int th, int occ)
{
    dim3 g;
    if (!fused_supported(c) || !fused_cfg_built(c, th, occ) || !fused_grid(c->cfg.N, c->cfg.n_members, th, g))
        return fail(c, SWE_EINVAL, "fused stage configuration (%d, %d) is not available for this context", th, occ);
    const bool retile = c->fth != th;
    c->fth = th;
    c->focc = occ;
    c->fused = true;
    if (!c->fmet) {
        int rc = c->elem == 8 ? build_fused_metric<double>(c, c->m64.v) : build_fused_metric<float>(c, c->m32.v);
        if (rc) { c->fused = false; return rc; }
    } else if (retile &&
               !encode_rows(&c->tm_metric, c->fmet, c->elem, c->dims.P,
                            (int64_t)FM_BOXES * (c->cfg.N + 1 + 2 * MG), fused_box_w(c), th + 8)) {
        c->fused = false;
        return fail(c, SWE_ECUDA, "TMA tensor map of the fused metric");
    }
    return SWE_OK;
}

// The C staggering's metric (FP64 on the host, stored in T), one panel box each:
// 1/(J a) and J Qi12 on the cell centres, Qi11, 1/J, J on the x points, Qi22, 1/J, J on
// the y points (metric_2d_ecs_mod.f90:338-411 on the o, x and y meshes).
template <class T>
static int build_c_metric(swe_ctx *c)
{
    const int N = c->cfg.N, P = c->dims.P;
    const size_t box = (size_t)c->dims.ps;
    std::vector<T> h(8 * box, T(0));
    HostMetric mo = host_metric(N, 0.5, 0.5), mx = host_metric(N, 0.0, 0.5), my = host_metric(N, 0.5, 0.0);
    const double a = c->cfg.radius;
    T *iJao = h.data(), *JQ12o = iJao + box, *Q11x = JQ12o + box, *iJx = Q11x + box, *Jx = iJx + box,
      *Q22y = Jx + box, *iJy = Q22y + box, *Jy = iJy + box;
    for (int j = 1; j <= N; j++)
        for (int i = 1; i <= N; i++) {
            const size_t k = (size_t)(j - 1) * mo.nx + (i - 1), o = (size_t)box_off(P, i, j);
            iJao[o] = T(1.0 / (mo.J[k] * a));
            JQ12o[o] = T(mo.J[k] * mo.Q2[k]);
        }
    for (int j = 1; j <= N; j++)
        for (int i = 1; i <= N + 1; i++) {
            const size_t k = (size_t)(j - 1) * mx.nx + (i - 1), o = (size_t)box_off(P, i, j);
            Q11x[o] = T(mx.Q1[k]); iJx[o] = T(1.0 / mx.J[k]); Jx[o] = T(mx.J[k]);
        }
    for (int j = 1; j <= N + 1; j++)
        for (int i = 1; i <= N; i++) {
            const size_t k = (size_t)(j - 1) * my.nx + (i - 1), o = (size_t)box_off(P, i, j);
            Q22y[o] = T(my.Q3[k]); iJy[o] = T(1.0 / my.J[k]); Jy[o] = T(my.J[k]);
        }
    T *d = nullptr;
    if (cudaMalloc(&d, h.size() * sizeof(T)) != cudaSuccess) return fail(c, SWE_ENOMEM, "C metric allocation failed");
    c->cmet = d;
    CU(c, cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return SWE_OK;
}

template <class T>
static CMetric<T> c_view(const swe_ctx *c)
{
    const size_t box = (size_t)c->dims.ps;
    const T *d = (const T *)c->cmet;
    const double pi = 3.141592653589793238462643383279502884;
    const double hx = (0.25 * pi - (-0.25 * pi)) / (double)c->cfg.N;
    return CMetric<T>{d, d + box, d + 2 * box, d + 3 * box, d + 4 * box, d + 5 * box, d + 6 * box, d + 7 * box,
                      T(1.0 / (hx * c->cfg.radius)), T(1.0 / hx)};
}

// The Ah operator's metric at the vertices (FP64 on the host, stored in T): J, the
// inverse metric Qi11, Qi12, Qi22, f J per panel (coriolis_colocated's f from
// calc_coriolis_parameter, coriolis_factory_mod.f90:239-280), and the SBP_Ah
// quadrature weights J hx hy Ax Ay with the node norm in both directions
// (quadrature_factory_mod.f90:31-66; Q42_A, sbp_operators_collection_mod.f90:35).
template <class T>
static int build_ah_metric(swe_ctx *c, DevAh<T> &da)
{
    const int N = c->cfg.N, P = c->dims.P, n = N + 1;
    const size_t box = (size_t)c->dims.ps;
    std::vector<T> h(10 * box, T(0));
    std::vector<double> q(box, 0.0);
    const HostMetric mxy = host_metric(N, 0.0, 0.0);
    // Q21_A, Q42_A, Q63_A (sbp_operators_collection_mod.f90:22,35,38-40)
    const double Q21A[2] = {0.5, 1.0}, Q42A[4] = {17.0 / 48.0, 59.0 / 48.0, 43.0 / 48.0, 49.0 / 48.0};
    const double *QA = c->ord == 21 ? Q21A : (c->ord == 63 ? SBP63_NN_A : Q42A);
    const int ne = c->ord == 21 ? 2 : (c->ord == 63 ? 6 : 4);
    auto A = [&](int i) { return i <= ne ? QA[i - 1] : (i >= n - ne + 1 ? QA[n - i] : 1.0); };
    const double pi = 3.141592653589793238462643383279502884, hx = 0.5 * pi / N;
    for (int j = 1; j <= n; j++)
        for (int i = 1; i <= n; i++) {
            const size_t k = (size_t)(j - 1) * n + (i - 1), o = (size_t)box_off(P, i, j);
            h[o] = T(mxy.J[k]);
            h[box + o] = T(mxy.Q1[k]);
            h[2 * box + o] = T(mxy.Q2[k]);
            h[3 * box + o] = T(mxy.Q3[k]);
            q[o] = mxy.J[k] * hx * hx * A(i) * A(j);
            for (int p = 0; p < NPAN; p++) {
                double f = c->cfg.omega;
                if (!c->cfg.coriolis_constant) {
                    double r[3];
                    vertex_r(N, p, i, j, r);
                    const double *ax = c->cfg.rotation_axis;
                    f = 2 * c->cfg.omega * (ax[0] * r[0] + ax[1] * r[1] + ax[2] * r[2]) /
                        std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                }
                h[(4 + p) * box + o] = T(f * mxy.J[k]);
            }
        }
    T *d = nullptr;
    if (cudaMalloc(&d, h.size() * sizeof(T)) != cudaSuccess) return fail(c, SWE_ENOMEM, "Ah metric allocation failed");
    da.base = d;
    CU(c, cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    da.v.J = d; da.v.Q1 = d + box; da.v.Q2 = d + 2 * box; da.v.Q3 = d + 3 * box; da.v.fJ = d + 4 * box;
    if (cudaMalloc(&c->qa, box * sizeof(double)) != cudaSuccess) return fail(c, SWE_ENOMEM, "Ah quadrature allocation failed");
    CU(c, cudaMemcpy(c->qa, q.data(), box * sizeof(double), cudaMemcpyHostToDevice));
    return SWE_OK;
}

// ---------------------------------------------------------------------------
// advective operator: static tables, FP64 on the host (same expressions as the
// reference's setup code), stored in the context's precision
// ---------------------------------------------------------------------------
static void p2r(int p, const double rp[3], double r[3])
{
    for (int d = 0; d < 3; d++) r[d] = EX[p][d] * rp[0] + EY[p][d] * rp[1] - NRM[p][d] * rp[2];
}

struct MeshGeom {
    int nx, ny;
    double shi, shj, hx, hy;
};
static MeshGeom mesh_geom(int N, double shi, double shj)
{
    const double pi = 3.141592653589793238462643383279502884;
    MeshGeom g;
    g.nx = shi == 0.0 ? N + 1 : N;
    g.ny = shj == 0.0 ? N + 1 : N;
    g.shi = shi;
    g.shj = shj;
    const double a0 = -0.25 * pi, a1 = 0.25 * pi;
    g.hx = (a1 - a0) / ((double)g.nx - 1 + 2.0 * shi);
    g.hy = (a1 - a0) / ((double)g.ny - 1 + 2.0 * shj);
    return g;
}
static void mesh_ab(const MeshGeom &g, int i, int j, double &alpha, double &beta)
{
    const double pi = 3.141592653589793238462643383279502884;
    alpha = -0.25 * pi + (i - 1 + g.shi) * g.hx;
    beta = -0.25 * pi + (j - 1 + g.shj) * g.hy;
}

// Position and covariant basis of a mesh point at any index (set_curvilinear_mesh,
// metric_2d_ecs_mod.f90:338-411).
static void mesh_point(const MeshGeom &g, int p, int i, int j, double r[3], double a1[3], double a2[3])
{
    double alpha, beta;
    mesh_ab(g, i, j, alpha, beta);
    const double ta = std::tan(alpha), tb = std::tan(beta);
    const double sigm = std::sqrt(1.0 + ta * ta + tb * tb);
    const double rp[3] = {ta / sigm, tb / sigm, 1.0 / sigm};
    p2r(p, rp, r);
    double q[3];
    a1p(alpha, beta, q);
    p2r(p, q, a1);
    a2p(alpha, beta, q);
    p2r(p, q, a2);
}

// transform_cartesian_to_native_ecs (metric_2d_ecs_mod.f90:310-335)
static void cart_to_native(const double r[3], int &panel, double &alpha, double &beta)
{
    int p = 0;
    double best = 0.0;
    for (int q = 0; q < NPAN; q++) {
        const double d = -(r[0] * NRM[q][0] + r[1] * NRM[q][1] + r[2] * NRM[q][2]);
        if (d > best) { p = q; best = d; }
    }
    panel = p;
    alpha = std::atan((EX[p][0] * r[0] + EX[p][1] * r[1] + EX[p][2] * r[2]) / best);
    beta = std::atan((EY[p][0] * r[0] + EY[p][1] * r[1] + EY[p][2] * r[2]) / best);
}

// bicubic_interp_t%calc_w (bicubic_interp_mod.f90:27-84)
static void bicubic_w(const MeshGeom &g, double alpha, double beta, int &ix, int &iy, double wx[4], double wy[4])
{
    const double pi = 3.141592653589793238462643383279502884;
    double dx = (alpha - (-0.25 * pi)) / g.hx + 1 - g.shi;
    double dy = (beta - (-0.25 * pi)) / g.hy + 1 - g.shj;
    ix = std::min(std::max(2, (int)dx), g.nx - 2);
    iy = std::min(std::max(2, (int)dy), g.ny - 2);
    dx = dx - ix;
    dy = dy - iy;
    double p1 = dx + 1.0, p2 = dx, p3 = dx - 1.0, p4 = dx - 2.0;
    wx[0] = -p2 * p3 * p4 / 6.0; wx[1] = p1 * p3 * p4 / 2.0; wx[2] = -p1 * p2 * p4 / 2.0; wx[3] = p1 * p2 * p3 / 6.0;
    p1 = dy + 1.0; p2 = dy; p3 = dy - 1.0; p4 = dy - 2.0;
    wy[0] = -p2 * p3 * p4 / 6.0; wy[1] = p1 * p3 * p4 / 2.0; wy[2] = -p1 * p2 * p4 / 2.0; wy[3] = p1 * p2 * p3 / 6.0;
}

// init_halo_xy_interp (ecs_halo_factory_mod.f90:236-270): target index i at halo row j
static void halo_xy_weights(int n, double dxa, int i, int j, double w[4], int &ind)
{
    const double pi = 3.141592653589793238462643383279502884;
    const double zb = 0.25 * pi + j * dxa;
    double za = -0.25 * pi + (i - 1.0) * dxa;
    double zx = std::tan(za);
    const double zz = std::tan(zb);
    zx = zx / zz;
    za = std::atan(zx);
    int k = (int)std::floor((za + 0.25 * pi) / dxa) + 1;
    k = std::min(std::max(2, k), n - 2);
    const double zxi = (za + 0.25 * pi) / dxa - (k - 1.0);
    w[0] = -(zxi * (zxi - 1.0) * (zxi - 2.0) / 6.0);
    w[1] = (zxi + 1.0) * (zxi - 1.0) * (zxi - 2.0) / 2.0;
    w[2] = -((zxi + 1.0) * zxi * (zxi - 2.0) / 2.0);
    w[3] = (zxi + 1.0) * zxi * (zxi - 1.0) / 6.0;
    ind = k;
}

// calculate_ecs_S (metric_2d_ecs_mod.f90:270-291)
static void christoffel_S(double alpha, double beta, double S[3][2])
{
    const double x = std::tan(alpha), y = std::tan(beta);
    const double x2 = x * x, y2 = y * y;
    const double sigma = 1.0 + x2 + y2;
    const double s3 = sigma * sigma * sigma;
    S[0][0] = 2.0 * x * y2 * ((1.0 + x2) * (1.0 + x2)) * (1.0 + y2) / s3;
    S[1][0] = -0.5 * y * (1.0 + y2) * (1.0 + x2) * (-(x2 * x2) + 3.0 * x2 * y2 + y2 + 1.0) / s3;
    S[2][0] = x * (1.0 + x2) * ((1.0 + y2) * (1.0 + y2)) * (-x2 + y2 - 1.0) / s3;
    S[0][1] = y * (1.0 + y2) * ((1.0 + x2) * (1.0 + x2)) * (-y2 + x2 - 1.0) / s3;
    S[1][1] = -0.5 * x * (1.0 + x2) * (1.0 + y2) * (-(y2 * y2) + 3.0 * y2 * x2 + x2 + 1.0) / s3;
    S[2][1] = 2.0 * y * x2 * ((1.0 + y2) * (1.0 + y2)) * (1.0 + x2) / s3;
}

// One virtual point of the covariant vector halo (ecs_halo_vec_Ch_factory_mod.f90:21-270):
// source panel, bicubic stencils on its y (u) and x (v) meshes, projections a.b1, a.b2.
static void vec_halo_entry(int N, const MeshGeom &gm, int t, int i, int j, bool comp_u, int &src, int ix[4], double w[18])
{
    double r[3], a1[3], a2[3], al, be, bp[3], b1[3], b2[3];
    mesh_point(gm, t, i, j, r, a1, a2);
    const double *a = comp_u ? a1 : a2;
    cart_to_native(r, src, al, be);
    bicubic_w(mesh_geom(N, 0.5, 0.0), al, be, ix[0], ix[1], w, w + 4);
    bicubic_w(mesh_geom(N, 0.0, 0.5), al, be, ix[2], ix[3], w + 8, w + 12);
    b1p(al, be, bp);
    p2r(src, bp, b1);
    b2p(al, be, bp);
    p2r(src, bp, b2);
    w[16] = a[0] * b1[0] + a[1] * b1[1] + a[2] * b1[2];
    w[17] = a[0] * b2[0] + a[1] * b2[1] + a[2] * b2[2];
}

template <class T>
static int build_adv_tables(swe_ctx *c, DevAdv<T> &da)
{
    const int N = c->cfg.N, n = N + 1, P = c->dims.P, hp = vh_points(N);
    const size_t box = (size_t)c->dims.ps;
    // layout: xyw [2][n][4] | hw [6][hp][18] | S [6 boxes]
    const size_t o_hw = 8 * (size_t)n, o_S = o_hw + (size_t)NPAN * hp * 18, n_el = o_S + 6 * box;
    // ints: xyind [2][n] | hsrc [6][hp] | hidx [6][hp][4]
    const size_t i_src = 2 * (size_t)n, i_idx = i_src + (size_t)NPAN * hp, n_int = i_idx + (size_t)NPAN * hp * 4;
    std::vector<T> h(n_el, T(0));
    std::vector<int> hi(n_int, 0);
    const MeshGeom gxy = mesh_geom(N, 0.0, 0.0), gy = mesh_geom(N, 0.5, 0.0), gx = mesh_geom(N, 0.0, 0.5);
    for (int d = 1; d <= 2; d++)
        for (int a = 1; a <= n; a++) {
            double w[4];
            int ind;
            halo_xy_weights(n, gxy.hx, a, d, w, ind);
            for (int k = 0; k < 4; k++) h[((size_t)(d - 1) * n + (a - 1)) * 4 + k] = T(w[k]);
            hi[(size_t)(d - 1) * n + (a - 1)] = ind;
        }
    for (int t = 0; t < NPAN; t++) {
        auto put = [&](int k, const MeshGeom &g, int i, int j, bool cu) {
            int src, ix[4];
            double w[18];
            vec_halo_entry(N, g, t, i, j, cu, src, ix, w);
            const size_t q = (size_t)t * hp + k;
            hi[i_src + q] = src;
            for (int e = 0; e < 4; e++) hi[i_idx + 4 * q + e] = ix[e];
            for (int e = 0; e < 18; e++) h[o_hw + 18 * q + e] = T(w[e]);
        };
        for (int d = 1; d <= 3; d++) {
            for (int i = 1; i <= N; i++) {
                put(vh_u_s(N) + (d - 1) * N + (i - 1), gy, i, 1 - d, true);
                put(vh_u_n(N) + (d - 1) * N + (i - 1), gy, i, N + 1 + d, true);
            }
            for (int j = 1; j <= N + 1; j++) {
                put(vh_u_w(N) + (d - 1) * (N + 1) + (j - 1), gy, 1 - d, j, true);
                put(vh_u_e(N) + (d - 1) * (N + 1) + (j - 1), gy, N + d, j, true);
            }
            for (int j = 1; j <= N; j++) {
                put(vh_v_w(N) + (d - 1) * N + (j - 1), gx, 1 - d, j, false);
                put(vh_v_e(N) + (d - 1) * N + (j - 1), gx, N + 1 + d, j, false);
            }
            for (int i = 1; i <= N + 1; i++) {
                put(vh_v_s(N) + (d - 1) * (N + 1) + (i - 1), gx, i, 1 - d, false);
                put(vh_v_n(N) + (d - 1) * (N + 1) + (i - 1), gx, i, N + d, false);
            }
        }
    }
    for (int j = 1; j <= N + 1; j++)
        for (int i = 1; i <= N; i++) {
            double al, be, S[3][2];
            mesh_ab(gy, i, j, al, be);
            christoffel_S(al, be, S);
            for (int k = 0; k < 3; k++) h[o_S + k * box + box_off(P, i, j)] = T(S[k][0]);
        }
    for (int j = 1; j <= N; j++)
        for (int i = 1; i <= N + 1; i++) {
            double al, be, S[3][2];
            mesh_ab(gx, i, j, al, be);
            christoffel_S(al, be, S);
            for (int k = 0; k < 3; k++) h[o_S + (3 + k) * box + box_off(P, i, j)] = T(S[k][1]);
        }
    if (cudaMalloc(&da.base, n_el * sizeof(T)) != cudaSuccess || cudaMalloc(&da.ibase, n_int * sizeof(int)) != cudaSuccess)
        return fail(c, SWE_ENOMEM, "advective tables allocation failed");
    CU(c, cudaMemcpy(da.base, h.data(), n_el * sizeof(T), cudaMemcpyHostToDevice));
    CU(c, cudaMemcpy(da.ibase, hi.data(), n_int * sizeof(int), cudaMemcpyHostToDevice));
    AdvView<T> &v = da.v;
    v.xyw = da.base;
    v.hw = da.base + o_hw;
    v.S = da.base + o_S;
    v.xyind = da.ibase;
    v.hsrc = da.ibase + i_src;
    v.hidx = da.ibase + i_idx;
    v.inv_neg_radius = T(-1.0 / c->cfg.radius);
    v.hp = hp;
    return SWE_OK;
}

// Cube edges as (panel, side) with (panel*4 + side) below the neighbour's.
static void cube_edges(int out[12][2])
{
    Link L[NPAN][4];
    compute_links(L);
    int k = 0;
    for (int p = 0; p < NPAN; p++)
        for (int s = 0; s < 4; s++)
            if (p * 4 + s < L[p][s].nb * 4 + L[p][s].nside && k < 12) { out[k][0] = p; out[k][1] = s; k++; }
}

// SBP quadrature weights J hx hy Ax Ay (quadrature_factory_mod.f90:89-188) for xy, y, x
// and o (cell centres, the Ch q mesh of the enstrophy) meshes.
static int build_quadrature(swe_ctx *c)
{
    const int N = c->cfg.N, P = c->dims.P;
    const size_t box = (size_t)c->dims.ps;
    std::vector<double> h(4 * box, 0.0);
    // edge weights of the SBP norms: D42_A_interfaces / D42_A_centers, or D21_*
    // (sbp_operators_collection_mod.f90:169-170,196-197)
    const double AI42[5] = {7.0 / 18.0, 9.0 / 8.0, 1.0, 71.0 / 72.0, 1.0};
    const double AC42[4] = {13.0 / 12.0, 7.0 / 8.0, 25.0 / 24.0, 1.0};
    const double AI21[2] = {0.5, 1.0}, AC21[2] = {1.0, 1.0};
    // D63_A_interfaces / D63_A_centers: the 6-3 norms (sbp_operators_collection_mod.f90:199-200)
    const bool o21 = c->ord == 21, o63 = c->ord == 63;
    auto coeff = [&](int i, int n, bool iface) {
        const double *e = iface ? (o21 ? AI21 : (o63 ? SBP63_H_I : AI42)) : (o21 ? AC21 : (o63 ? SBP63_H_C : AC42));
        int ne = o21 ? 2 : (o63 ? (iface ? 5 : 6) : (iface ? 5 : 4));
        double A = 1.0;
        if (i <= ne) A = e[i - 1];
        if (i >= n - ne + 1) A = e[n - i];
        return A;
    };
    const double pi = 3.141592653589793238462643383279502884;
    const double hx = (0.25 * pi - (-0.25 * pi)) / (double)N;
    HostMetric ms[4] = {host_metric(N, 0.0, 0.0), host_metric(N, 0.5, 0.0), host_metric(N, 0.0, 0.5),
                        host_metric(N, 0.5, 0.5)};
    for (int q = 0; q < 4; q++) {
        const HostMetric &m = ms[q];
        for (int j = 1; j <= m.ny; j++)
            for (int i = 1; i <= m.nx; i++) {
                double Ax = coeff(i, m.nx, m.nx == N + 1), Ay = coeff(j, m.ny, m.ny == N + 1);
                h[q * box + (size_t)box_off(P, i, j)] = m.J[(size_t)(j - 1) * m.nx + (i - 1)] * hx * hx * Ax * Ay;
            }
    }
    if (cudaMalloc(&c->qw, h.size() * sizeof(double)) != cudaSuccess)
        return fail(c, SWE_ENOMEM, "quadrature allocation failed");
    CU(c, cudaMemcpy(c->qw, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    if (cudaMalloc(&c->red, 4096 * sizeof(double)) != cudaSuccess)
        return fail(c, SWE_ENOMEM, "reduction buffer allocation failed");
    return SWE_OK;
}

extern "C" int swe_cfg_default(swe_cfg *cfg)
{
    if (!cfg) return SWE_EINVAL;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->N = 32;
    cfg->precision = SWE_FP64;
    cfg->n_members = 1;
    cfg->operator_kind = SWE_OP_LINEAR;
    cfg->radius = 0.6371229e7;
    cfg->grav = 9.80616;
    cfg->omega = 2.0 * 3.141592653589793238462643383279502884 / (23 * 60 * 60 + 56 * 60 + 4);
    cfg->rotation_axis[0] = 0.0; cfg->rotation_axis[1] = 0.0; cfg->rotation_axis[2] = 1.0;
    cfg->coriolis_constant = 0;
    cfg->h_mean = 1000.0;
    cfg->sbp_order = 42;
    cfg->staggering = SWE_STAG_CH;
    return SWE_OK;
}

// The advective stage forks its independent kernels onto a second stream;
// CHSWE_ADV_BRANCHES=0 in the environment keeps the whole stage on one stream.
static bool adv_branches_enabled()
{
    static const bool on = [] {
        const char *e = std::getenv("CHSWE_ADV_BRANCHES");
        return !(e && e[0] == '0');
    }();
    return on;
}

static void free_ctx(swe_ctx *c)
{
    if (c->graph) cudaGraphExecDestroy(c->graph);
    if (c->graphk) cudaGraphExecDestroy(c->graphk);
    cudaFree(c->m64.base); cudaFree(c->m32.base); cudaFree(c->Hm); cudaFree(c->dtm);
    cudaFree(c->ya); cudaFree(c->yb); cudaFree(c->acc); cudaFree(c->w); cudaFree(c->edge); cudaFree(c->es);
    cudaFree(c->qw); cudaFree(c->red); cudaFree(c->otab); cudaFree(c->ll_i); cudaFree(c->ll_d); cudaFree(c->llo_i); cudaFree(c->llo_d);
    cudaFree(c->a64.base); cudaFree(c->a64.ibase); cudaFree(c->a32.base); cudaFree(c->a32.ibase);
    cudaFree(c->fl); cudaFree(c->adt); cudaFree(c->fs); cudaFree(c->vh); cudaFree(c->ones); cudaFree(c->hb);
    cudaFree(c->ah64.base); cudaFree(c->ah32.base); cudaFree(c->qa); cudaFree(c->negones);
    cudaFree(c->dif); cudaFree(c->dif_b);
    cudaFree(c->fmet); cudaFree(c->derr); cudaFree(c->hs); cudaFree(c->cmet);
    if (c->pinned) cudaFreeHost(c->pinned);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    if (c->side) cudaStreamDestroy(c->side);
    for (cudaEvent_t e : {c->ev_fork, c->ev_havg, c->ev_co2, c->ev_side})
        if (e) cudaEventDestroy(e);
}

static int alloc_box(swe_ctx *c, void **p)
{
    size_t bytes = c->box_elems * c->elem;
    if (cudaMalloc(p, bytes) != cudaSuccess) return fail(c, SWE_ENOMEM, "device allocation of %zu bytes failed", bytes);
    CU(c, cudaMemset(*p, 0, bytes));
    return SWE_OK;
}

template <class T>
static cudaError_t stage_smem_optin();

extern "C" int swe_ctx_create(const swe_cfg *cfg, swe_ctx **out)
{
    if (!cfg || !out) return SWE_EINVAL;
    *out = nullptr;
    if (cfg->N < 8 || cfg->n_members < 1 || (cfg->precision != SWE_FP64 && cfg->precision != SWE_FP32) ||
        (cfg->operator_kind != SWE_OP_LINEAR && cfg->operator_kind != SWE_OP_ADVECTIVE) || !(cfg->radius > 0.0))
        return SWE_EINVAL;
    // SBP order: 4-2 (0 selects it too), 2-1 or 6-3 (N >= 16)
    const int ord = cfg->sbp_order == 0 ? 42 : cfg->sbp_order;
    if ((ord != 42 && ord != 21 && ord != 63) || (ord == 63 && cfg->N < 16)) return SWE_EINVAL;
    // Ah staggering: the linear operator with the SBP node operators
    if ((cfg->staggering != SWE_STAG_CH && cfg->staggering != SWE_STAG_AH && cfg->staggering != SWE_STAG_C) ||
        (cfg->staggering != SWE_STAG_CH && cfg->operator_kind != SWE_OP_LINEAR) ||
        (cfg->staggering == SWE_STAG_C && ord != 42))
        return SWE_EINVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return SWE_ENODEV;
    swe_ctx *c = new swe_ctx();
    c->cfg = *cfg;
    c->cfg.sbp_order = ord;
    c->ord = ord;
    cudaGetDevice(&c->device);
    const int N = cfg->N;
    c->dims.N = N;
    c->dims.P = (N + 1 + 2 * MG + 7) / 8 * 8;
    c->dims.ps = (int64_t)(N + 1 + 2 * MG) * c->dims.P;
    c->dims.fs = NPAN * c->dims.ps;
    c->dims.ms = 3 * c->dims.fs;
    c->elem = cfg->precision == SWE_FP64 ? 8 : 4;
    c->tile = default_tile(N);
    c->occ = default_occ(c->tile);
    c->runs = 0;
    c->box_elems = (size_t)c->dims.ms * cfg->n_members;
    int rc = SWE_OK;
    auto bail = [&](int code) { free_ctx(c); delete c; return code; };
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) return bail(SWE_ECUDA);
    c->stream = c->own_stream;
    if ((rc = upload_tables(c)) != SWE_OK) return bail(rc);
    if ((cfg->precision == SWE_FP64 ? stage_smem_optin<double>() : stage_smem_optin<float>()) != cudaSuccess)
        return bail(SWE_ECUDA);
    if (cfg->precision == SWE_FP64) rc = build_metric<double>(c, c->m64);
    else rc = build_metric<float>(c, c->m32);
    if (rc != SWE_OK) return bail(rc);
    if ((rc = build_quadrature(c)) != SWE_OK) return bail(rc);
    if (cfg->staggering == SWE_STAG_AH) {
        c->ah = true;
        rc = cfg->precision == SWE_FP64 ? build_ah_metric<double>(c, c->ah64) : build_ah_metric<float>(c, c->ah32);
        if (rc != SWE_OK) return bail(rc);
    }
    if (cfg->staggering == SWE_STAG_C) {
        c->cstag = true;
        rc = cfg->precision == SWE_FP64 ? build_c_metric<double>(c) : build_c_metric<float>(c);
        if (rc != SWE_OK) return bail(rc);
    }
    c->Hhost.assign(cfg->n_members, cfg->h_mean);
    if (cudaMalloc(&c->Hm, sizeof(double) * cfg->n_members) != cudaSuccess) return bail(SWE_ENOMEM);
    if (cudaMalloc(&c->dtm, sizeof(double) * cfg->n_members) != cudaSuccess) return bail(SWE_ENOMEM);
    if (cudaMalloc(&c->derr, sizeof(int)) != cudaSuccess) return bail(SWE_ENOMEM);
    if (cudaMemset(c->derr, 0, sizeof(int)) != cudaSuccess) return bail(SWE_ECUDA);
    if (cudaMemcpy(c->Hm, c->Hhost.data(), sizeof(double) * cfg->n_members, cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(SWE_ECUDA);
    if ((rc = alloc_box(c, &c->ya)) || (rc = alloc_box(c, &c->yb)) || (rc = alloc_box(c, &c->acc)) ||
        (rc = alloc_box(c, &c->w)))
        return bail(rc);
    {
        const size_t eb = (size_t)cfg->n_members * NPAN * 4 * (N + 1) * 3 * c->elem;
        if (cudaMalloc(&c->edge, eb) != cudaSuccess) return bail(SWE_ENOMEM);
        if (cudaMemset(c->edge, 0, eb) != cudaSuccess) return bail(SWE_ECUDA);
        const size_t sb = (size_t)strip_member(N, cfg->n_members, ord_strip_lines(ord)) * c->elem;
        if (cudaMalloc(&c->es, sb) != cudaSuccess) return bail(SWE_ENOMEM);
        if (cudaMemset(c->es, 0, sb) != cudaSuccess) return bail(SWE_ECUDA);
        if (cfg->operator_kind == SWE_OP_ADVECTIVE) {
            c->adv = true;
            if ((rc = alloc_box(c, &c->fl)) || (rc = alloc_box(c, &c->adt))) return bail(rc);
            if (cudaMalloc(&c->fs, sb) != cudaSuccess) return bail(SWE_ENOMEM);
            if (cudaMemset(c->fs, 0, sb) != cudaSuccess) return bail(SWE_ECUDA);
            const size_t vb = (size_t)cfg->n_members * NPAN * vh_points(N) * c->elem;
            if (cudaMalloc(&c->vh, vb) != cudaSuccess) return bail(SWE_ENOMEM);
            if (cudaMemset(c->vh, 0, vb) != cudaSuccess) return bail(SWE_ECUDA);
            const size_t hbb = (size_t)cfg->n_members * NPAN * 4 * (N + 1) * c->elem;
            if (cudaMalloc(&c->hb, hbb) != cudaSuccess) return bail(SWE_ENOMEM);
            if (cudaMemset(c->hb, 0, hbb) != cudaSuccess) return bail(SWE_ECUDA);
            std::vector<double> one(cfg->n_members, 1.0);
            if (cudaMalloc(&c->ones, sizeof(double) * cfg->n_members) != cudaSuccess) return bail(SWE_ENOMEM);
            if (cudaMemcpy(c->ones, one.data(), sizeof(double) * cfg->n_members, cudaMemcpyHostToDevice) != cudaSuccess)
                return bail(SWE_ECUDA);
            rc = cfg->precision == SWE_FP64 ? build_adv_tables<double>(c, c->a64) : build_adv_tables<float>(c, c->a32);
            if (rc != SWE_OK) return bail(rc);
            if (adv_branches_enabled()) {
                if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess) return bail(SWE_ECUDA);
                for (cudaEvent_t *e : {&c->ev_fork, &c->ev_havg, &c->ev_co2, &c->ev_side})
                    if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) return bail(SWE_ECUDA);
            }
        }
    }
    if (cudaHostAlloc((void **)&c->pinned, c->box_elems * c->elem, cudaHostAllocDefault) != cudaSuccess)
        return bail(SWE_ENOMEM);
    std::memset(c->pinned, 0, c->box_elems * c->elem);
    *out = c;
    return SWE_OK;
}

extern "C" int swe_ctx_destroy(swe_ctx *c)
{
    if (!c) return SWE_EINVAL;
    cudaStreamSynchronize(c->stream);
    free_ctx(c);
    delete c;
    return SWE_OK;
}

extern "C" const char *swe_last_error(const swe_ctx *c) { return c ? c->err.c_str() : "null context"; }

extern "C" int swe_set_stream(swe_ctx *c, void *s)
{
    if (!c) return SWE_EINVAL;
    c->stream = s ? (cudaStream_t)s : c->own_stream;
    if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
    if (c->graphk) { cudaGraphExecDestroy(c->graphk); c->graphk = nullptr; }
    return SWE_OK;
}

extern "C" int swe_synchronize(swe_ctx *c)
{
    if (!c) return SWE_EINVAL;
    CU(c, cudaStreamSynchronize(c->stream));
    // a kernel whose bounded wait for its tile loads ran out leaves a flag behind
    int flag = 0;
    CU(c, cudaMemcpy(&flag, c->derr, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        CU(c, cudaMemset(c->derr, 0, sizeof(int)));
        return fail(c, SWE_ECUDA, "a stage kernel gave up waiting for its tile loads; its outputs are incomplete");
    }
    return SWE_OK;
}

extern "C" long long swe_launch_count(const swe_ctx *c) { return c ? c->launches : -1; }

extern "C" int swe_set_member_h_mean(swe_ctx *c, int member, double H)
{
    if (!c || member < 0 || member >= c->cfg.n_members) return SWE_EINVAL;
    c->Hhost[member] = H;
    CU(c, cudaMemcpyAsync(c->Hm + member, &c->Hhost[member], sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CU(c, cudaStreamSynchronize(c->stream));
    return SWE_OK;
}

// Orography of the advective operator: h_surf packed like h ((N+1) x (N+1) per panel),
// shared by every member; NULL removes it.  The gradient's input becomes h + h_surf
// (operator_adv_swm_mod.f90:37-38,78).
extern "C" int swe_set_orography(swe_ctx *c, const double *h_surf)
{
    if (!c) return SWE_EINVAL;
    if (!c->adv) return fail(c, SWE_EINVAL, "swe_set_orography: orography belongs to the advective operator");
    if (!h_surf) {
        if (c->hs) CU(c, cudaStreamSynchronize(c->stream));
        cudaFree(c->hs);
        c->hs = nullptr;
        drop_graph(c);
        return SWE_OK;
    }
    const int N = c->cfg.N, n = N + 1, P = c->dims.P;
    const size_t box = (size_t)c->dims.ps, fbox = NPAN * box;
    std::vector<unsigned char> host(fbox * c->elem, 0);
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= n; j++)
            for (int i = 1; i <= n; i++) {
                const double v = h_surf[((size_t)t * n + j - 1) * n + i - 1];
                const size_t o = t * box + (size_t)box_off(P, i, j);
                if (c->elem == 8) ((double *)host.data())[o] = v;
                else ((float *)host.data())[o] = (float)v;
            }
    const bool fresh = !c->hs;
    if (fresh && cudaMalloc(&c->hs, host.size()) != cudaSuccess) {
        c->hs = nullptr;
        return fail(c, SWE_ENOMEM, "orography allocation failed");
    }
    CU(c, cudaMemcpyAsync(c->hs, host.data(), host.size(), cudaMemcpyHostToDevice, c->stream));
    CU(c, cudaStreamSynchronize(c->stream));
    if (fresh) drop_graph(c);   // captured steps hold the orography pointer
    return SWE_OK;
}

extern "C" int swe_stvec_create(swe_ctx *c, swe_stvec **out)
{
    if (!c || !out) return SWE_EINVAL;
    swe_stvec *v = new swe_stvec();
    v->ctx = c;
    int rc = alloc_box(c, &v->d);
    if (rc) { delete v; return rc; }
    *out = v;
    return SWE_OK;
}

extern "C" int swe_stvec_destroy(swe_stvec *v)
{
    if (!v) return SWE_EINVAL;
    cudaStreamSynchronize(v->ctx->stream);
    swe_ctx *c = v->ctx;
    if (c->graph_v0 == v->d) {
        // the cached graphs hold this vector's pointers: a later vector at the same
        // address must capture its own
        if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
        if (c->graphk) { cudaGraphExecDestroy(c->graphk); c->graphk = nullptr; }
        c->graph_v0 = nullptr;
    }
    cudaFree(v->d);
    cudaFree(v->cmp);
    delete v;
    return SWE_OK;
}

// Packed host member (Fortran per-panel layout) <-> padded device box.
// Points per panel of u (nx by ny) and v (ny by nx): the y and x meshes on Ch, the
// vertices on Ah.
// Packed extents (nx along i, ny along j) of field f (0 h, 1 u, 2 v) per panel: on Ch h on
// the vertices, u on the y points, v on the x points; on Ah all on the vertices; on C h on
// the cell centres, u on the x points, v on the y points.
static void field_extent(const swe_ctx *c, int f, int &nx, int &ny)
{
    const int N = c->cfg.N, n = N + 1;
    if (c->ah) { nx = ny = n; return; }
    if (c->cstag) {
        nx = f == 0 ? N : (f == 1 ? n : N);
        ny = f == 0 ? N : (f == 1 ? N : n);
        return;
    }
    nx = f == 0 ? n : (f == 1 ? N : n);
    ny = f == 0 ? n : (f == 1 ? n : N);
}

// Host copies between the packed arrays and the pinned staging box, one task per
// (member, panel): on several threads when the copy is large (the e2e path's host
// share), serially for small cubes.
template <class F>
static void panel_tasks(int count, int N, const F &task)
{
    const int ntask = count * NPAN;
    const unsigned hw = std::thread::hardware_concurrency();
    const int nthreads = (int)std::min<long long>(std::min<long long>(hw ? hw : 1, 16), ntask);
    if ((long long)ntask * (N + 1) * (N + 1) < (1LL << 15) || nthreads <= 1) {
        for (int k = 0; k < ntask; k++) task(k / NPAN, k % NPAN);
        return;
    }
    std::vector<std::thread> pool;
    for (int w = 0; w < nthreads; w++)
        pool.emplace_back([&, w] {
            for (int k = w; k < ntask; k += nthreads) task(k / NPAN, k % NPAN);
        });
    for (auto &th : pool) th.join();
}

template <class T>
static void pack_panel(const swe_ctx *c, const double *h, const double *u, const double *v, T *box, int t)
{
    const int P = c->dims.P;
    const size_t ps = c->dims.ps, fs = c->dims.fs;
    const double *src[3] = {h, u, v};
    for (int f = 0; f < 3; f++) {
        int nx, ny;
        field_extent(c, f, nx, ny);
        const double *p = src[f] + (size_t)t * nx * ny;
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) box[f * fs + t * ps + box_off(P, i + 1, j + 1)] = T(*p++);
    }
}

template <class T>
static void unpack_panel(const swe_ctx *c, const T *box, double *h, double *u, double *v, int t)
{
    const int P = c->dims.P;
    const size_t ps = c->dims.ps, fs = c->dims.fs;
    double *dst[3] = {h, u, v};
    for (int f = 0; f < 3; f++) {
        int nx, ny;
        field_extent(c, f, nx, ny);
        double *p = dst[f] + (size_t)t * nx * ny;
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) *p++ = double(box[f * fs + t * ps + box_off(P, i + 1, j + 1)]);
    }
}

static size_t member_sizes(const swe_ctx *c, size_t *nh, size_t *nu)
{
    int hx, hy, ux, uy;
    field_extent(c, 0, hx, hy);
    field_extent(c, 1, ux, uy);
    *nh = (size_t)NPAN * hx * hy;
    *nu = (size_t)NPAN * ux * uy;
    return *nh + 2 * *nu;
}

static int upload_range(swe_stvec *vec, int m0, int count, const double *h, const double *u, const double *v)
{
    swe_ctx *c = vec->ctx;
    size_t nh, nu;
    member_sizes(c, &nh, &nu);
    const size_t mbytes = (size_t)c->dims.ms * c->elem;
    CU(c, cudaStreamSynchronize(c->stream));   // the staging buffer may still feed an earlier copy
    unsigned char *buf = c->pinned;
    panel_tasks(count, c->cfg.N, [&](int k, int t) {
        if (c->elem == 8)
            pack_panel<double>(c, h + k * nh, u + k * nu, v + k * nu, (double *)(buf + k * mbytes), t);
        else
            pack_panel<float>(c, h + k * nh, u + k * nu, v + k * nu, (float *)(buf + k * mbytes), t);
    });
    CU(c, cudaMemcpyAsync((char *)vec->d + m0 * mbytes, buf, mbytes * count, cudaMemcpyHostToDevice, c->stream));
    if (vec->cmp) CU(c, cudaMemsetAsync((char *)vec->cmp + m0 * (size_t)c->dims.ms * 4, 0, (size_t)c->dims.ms * 4 * count, c->stream));
    CU(c, cudaStreamSynchronize(c->stream));
    return SWE_OK;
}

static int download_range(const swe_stvec *vec, int m0, int count, double *h, double *u, double *v)
{
    swe_ctx *c = vec->ctx;
    size_t nh, nu;
    member_sizes(c, &nh, &nu);
    const size_t mbytes = (size_t)c->dims.ms * c->elem;
    unsigned char *buf = c->pinned;
    CU(c, cudaMemcpyAsync(buf, (char *)vec->d + m0 * mbytes, mbytes * count, cudaMemcpyDeviceToHost, c->stream));
    CU(c, cudaStreamSynchronize(c->stream));
    panel_tasks(count, c->cfg.N, [&](int k, int t) {
        if (c->elem == 8)
            unpack_panel<double>(c, (const double *)(buf + k * mbytes), h + k * nh, u + k * nu, v + k * nu, t);
        else
            unpack_panel<float>(c, (const float *)(buf + k * mbytes), h + k * nh, u + k * nu, v + k * nu, t);
    });
    return SWE_OK;
}

extern "C" int swe_stvec_upload(swe_stvec *vec, int member, const double *h, const double *u, const double *v)
{
    if (!vec || !h || !u || !v || member < 0 || member >= vec->ctx->cfg.n_members) return SWE_EINVAL;
    return upload_range(vec, member, 1, h, u, v);
}
extern "C" int swe_stvec_download(const swe_stvec *vec, int member, double *h, double *u, double *v)
{
    if (!vec || !h || !u || !v || member < 0 || member >= vec->ctx->cfg.n_members) return SWE_EINVAL;
    return download_range(vec, member, 1, h, u, v);
}
extern "C" int swe_stvec_upload_all(swe_stvec *vec, const double *h, const double *u, const double *v)
{
    if (!vec || !h || !u || !v) return SWE_EINVAL;
    return upload_range(vec, 0, vec->ctx->cfg.n_members, h, u, v);
}
extern "C" int swe_stvec_download_all(const swe_stvec *vec, double *h, double *u, double *v)
{
    if (!vec || !h || !u || !v) return SWE_EINVAL;
    return download_range(vec, 0, vec->ctx->cfg.n_members, h, u, v);
}

extern "C" int swe_stvec_device_view(const swe_stvec *vec, void **ptr, size_t *bytes, int *precision, int *pitch)
{
    if (!vec) return SWE_EINVAL;
    if (ptr) *ptr = vec->d;
    if (bytes) *bytes = vec->ctx->box_elems * vec->ctx->elem;
    if (precision) *precision = vec->ctx->cfg.precision;
    if (pitch) *pitch = vec->ctx->dims.P;
    return SWE_OK;
}

static int launch_axpby(swe_ctx *c, void *y, const void *v1, const void *v2, double s1, double s2, int acc)
{
    const int64_t n = (int64_t)c->box_elems;
    int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
    if (c->elem == 8)
        k_axpby<double><<<blocks, 256, 0, c->stream>>>((double *)y, (const double *)v1, (const double *)v2, s1, s2, acc, n);
    else
        k_axpby<float><<<blocks, 256, 0, c->stream>>>((float *)y, (const float *)v1, (const float *)v2, s1, s2, acc, n);
    c->launches++;
    CU(c, cudaGetLastError());
    return SWE_OK;
}

extern "C" int swe_stvec_assign(swe_stvec *y, double s1, const swe_stvec *v1, double s2, const swe_stvec *v2)
{
    if (!y || !v1 || y->ctx != v1->ctx || (v2 && v2->ctx != y->ctx)) return SWE_EINVAL;
    return launch_axpby(y->ctx, y->d, v1->d, v2 ? v2->d : nullptr, s1, s2, 0);
}
extern "C" int swe_stvec_update(swe_stvec *y, double s1, const swe_stvec *v1, double s2, const swe_stvec *v2)
{
    if (!y || !v1 || y->ctx != v1->ctx || (v2 && v2->ctx != y->ctx)) return SWE_EINVAL;
    return launch_axpby(y->ctx, y->d, v1->d, v2 ? v2->d : nullptr, s1, s2, 1);
}

// ---------------------------------------------------------------------------
// operator application and RK4
// ---------------------------------------------------------------------------
// Dispatch to the stage translation units (stage_*.cu) by tile size.  The tiled
// kernels use more than 48 KB of dynamic shared memory: opt in once per device and
// element type (the attribute belongs to the device's context).
template <class T>
static cudaError_t stage_smem_optin()
{
    static bool done[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 64 && done[dev]) return cudaSuccess;
    e = StageTU<T, 17>::optin();
    if (e == cudaSuccess) e = StageTU<T, 25>::optin();
    if (e == cudaSuccess) e = StageTU<T, 33>::optin();
    if (e == cudaSuccess) e = FusedTU<T>::optin();
    if (e == cudaSuccess) e = GroupTU<T>::optin();
    if (e == cudaSuccess) e = set_carveout(k_edge<T, 42>);
    if (e == cudaSuccess) e = set_carveout(k_edge<T, 21>);
    if (e == cudaSuccess) e = set_carveout(k_edge<T, 63>);
    if (e == cudaSuccess && dev < 64) done[dev] = true;
    return e;
}

// ord: SBP order (42, 21 or 63).  Configurations are validated when set.
// false: no built configuration matched and nothing was launched.
template <class T>
static bool launch_co2contra(int tm, int occ, int runs, int ord, int members, const T *y, T *w, T *es, const Dims &d,
                             const MetricView<T> &m, cudaStream_t st, const double *dtm = nullptr)
{
    switch (tm) {
    case 17: return StageTU<T, 17>::co2contra(occ, runs, ord, members, y, w, es, d, m, st, dtm);
    case 25: return StageTU<T, 25>::co2contra(occ, runs, ord, members, y, w, es, d, m, st, dtm);
    default: return StageTU<T, 33>::co2contra(occ, runs, ord, members, y, w, es, d, m, st, dtm);
    }
}

// The advective variant exists for the first blocks-per-SM value of each tile only.
template <class T>
static bool launch_stage(int tm, int occ, int runs, int ord, int members, const T *y, const T *w, const T *e, T *v0,
                         T *y1, T *acc, T *cmp, const Dims &d, const MetricView<T> &m, const StageArgs &a,
                         cudaStream_t st)
{
    if (a.A) occ = default_occ(tm);
    switch (tm) {
    case 17: return StageTU<T, 17>::stage(occ, runs, ord, members, y, w, e, v0, y1, acc, cmp, d, m, a, st);
    case 25: return StageTU<T, 25>::stage(occ, runs, ord, members, y, w, e, v0, y1, acc, cmp, d, m, a, st);
    default: return StageTU<T, 33>::stage(occ, runs, ord, members, y, w, e, v0, y1, acc, cmp, d, m, a, st);
    }
}


static dim3 edge_grid(int N, int members) { return dim3((N + 1 + EDGE_CHUNK - 1) / EDGE_CHUNK, NPAN * 4, members); }
static dim3 edge_grid(const swe_ctx *c) { return edge_grid(c->cfg.N, c->cfg.n_members); }

template <class T> static const AdvView<T> &adv_view(const swe_ctx *c);
template <class T> static const AhView<T> &ah_view(const swe_ctx *c);
template <> const AhView<double> &ah_view<double>(const swe_ctx *c) { return c->ah64.v; }
template <> const AhView<float> &ah_view<float>(const swe_ctx *c) { return c->ah32.v; }
template <> const AdvView<double> &adv_view<double>(const swe_ctx *c) { return c->a64.v; }
template <> const AdvView<float> &adv_view<float>(const swe_ctx *c) { return c->a32.v; }

// The two launches of an Ah stage: the raw panel-boundary values, then every vertex.
template <class T, int ORD>
static void launch_ah(swe_ctx *c, const void *yin, void *v0, void *y1, void *acc, float *cmp, int mode,
                      const StageArgs &a, const AhView<T> &av, const MetricView<T> &mv, const double *dtm)
{
    const int n = c->cfg.N + 1, M = c->cfg.n_members;
    launch_k(k_ah_edge<T, ORD>, dim3((n + 127) / 128, NPAN * 4, M), dim3(128), 0, c->stream, (const T *)yin,
             (T *)c->edge, c->dims, av, mv, dtm);
    // balanced tiles of at most AH_TX x AH_TY vertices
    const dim3 pb(32, 8), pg((n + AH_TX - 1) / AH_TX, (n + AH_TY - 1) / AH_TY, NPAN * M);
    const T g = T(c->cfg.grav);
    const T *Y = (const T *)yin, *E = (const T *)c->edge;
    T *V = (T *)v0, *Y1 = (T *)y1, *A = (T *)acc, *C = (T *)cmp;
    switch (mode) {
    case 0: launch_k(k_ah_stage<T, 0, ORD>, pg, pb, 0, c->stream, Y, E, V, Y1, A, C, c->dims, av, mv, a, g); break;
    case 1: launch_k(k_ah_stage<T, 1, ORD>, pg, pb, 0, c->stream, Y, E, V, Y1, A, C, c->dims, av, mv, a, g); break;
    case 2: launch_k(k_ah_stage<T, 2, ORD>, pg, pb, 0, c->stream, Y, E, V, Y1, A, C, c->dims, av, mv, a, g); break;
    case 3: launch_k(k_ah_stage<T, 3, ORD>, pg, pb, 0, c->stream, Y, E, V, Y1, A, C, c->dims, av, mv, a, g); break;
    default: launch_k(k_ah_stage<T, 4, ORD>, pg, pb, 0, c->stream, Y, E, V, Y1, A, C, c->dims, av, mv, a, g); break;
    }
}

// One fused RK stage: edge strips, edge sync, tiles.
template <class T>
static bool enqueue_fused(swe_ctx *c, const void *yin, void *v0, void *y1, void *acc, float *cmp, int mode, double dt,
                          const double *dtm, const MetricView<T> &mv)
{
    const int M = c->cfg.n_members, N = c->cfg.N;
    const FusedMetric<T> fm{(const T *)c->fmet, mv.inv_hxa, mv.inv_hx, mv.grav};
    CUtensorMap tmY;
    if (!encode_rows(&tmY, yin, sizeof(T), c->dims.P, (int64_t)M * 3 * NPAN * (N + 1 + 2 * MG), fused_box_w(c),
                     c->fth + 8))
        return false;
    FusedTU<T>::strip(M, (const T *)yin, (T *)c->es, c->dims, fm, dtm, c->stream);
    launch_k(k_edge<T, 42>, edge_grid(c), dim3(EDGE_THREADS), 0, c->stream, (const T *)c->es, (const T *)c->es,
             (T *)c->edge, c->dims, mv, dtm);
    StageArgs a{mode, dt, c->Hm, dtm, nullptr, nullptr, nullptr};
    if (!FusedTU<T>::stage(c->fth, c->focc, M, tmY, c->tm_metric, (const T *)yin, (const T *)c->edge, (T *)v0,
                           (T *)y1, (T *)acc, (T *)cmp, c->dims, fm, a, c->derr, c->stream))
        return false;
    c->launches += 3;
    return true;
}

// The advective tendencies (k_advt): tiles of 32 x 16 xy points from C128 on, 32 x 8
// below (where taller tiles would leave fewer blocks than SMs).
template <class T>
static void launch_adv(swe_ctx *c, const void *yin, const AdvView<T> &av, const MetricView<T> &mv, const double *dtm,
                       cudaStream_t st)
{
    const int n = c->cfg.N + 1, M = c->cfg.n_members;
    const dim3 b(ADV_TX, ADV_THREADS / ADV_TX);
    if (c->cfg.N >= 128)
        launch_k(k_advt<T, 16>, dim3((n + ADV_TX - 1) / ADV_TX, (n + 15) / 16, NPAN * M), b, 0, st, (const T *)yin,
                 (const T *)c->w, (const T *)c->vh, (T *)c->adt, c->dims, av, mv, dtm);
    else
        launch_k(k_advt<T, 8>, dim3((n + ADV_TX - 1) / ADV_TX, (n + 7) / 8, NPAN * M), b, 0, st, (const T *)yin,
                 (const T *)c->w, (const T *)c->vh, (T *)c->adt, c->dims, av, mv, dtm);
}

template <class T>
static void enqueue_stage(swe_ctx *c, const void *yin, void *v0, void *y1, void *acc, float *cmp, int mode, double dt,
                          const double *dtm,
                          const MetricView<T> &mv)
{
    const int M = c->cfg.n_members;
    if (c->ah) {
        // Ah staggering: the raw panel-boundary values, then every vertex
        const AhView<T> &av = ah_view<T>(c);
        StageArgs a{mode, dt, c->Hm, dtm, nullptr, nullptr, nullptr};
        if (c->ord == 21) launch_ah<T, 21>(c, yin, v0, y1, acc, cmp, mode, a, av, mv, dtm);
        else if (c->ord == 63) launch_ah<T, 63>(c, yin, v0, y1, acc, cmp, mode, a, av, mv, dtm);
        else launch_ah<T, 42>(c, yin, v0, y1, acc, cmp, mode, a, av, mv, dtm);
        c->launches += 2;
        return;
    }
    if (!c->adv) {
        if (c->fused) {
            if (enqueue_fused<T>(c, yin, v0, y1, acc, cmp, mode, dt, dtm, mv)) return;
            // a tensor map that cannot be encoded: the split kernels take over
            c->fused = false;
            c->err = "fused stage unavailable (TMA tensor map); using the split stage kernels";
        }
        if (!launch_co2contra<T>(c->tile, c->occ, c->runs, c->ord, M, (const T *)yin, (T *)c->w, (T *)c->es, c->dims, mv,
                            c->stream, dtm)) c->launch_miss = true;
        launch_k(c->ord == 21 ? k_edge<T, 21> : (c->ord == 63 ? k_edge<T, 63> : k_edge<T, 42>), edge_grid(c), dim3(EDGE_THREADS), 0, c->stream, (const T *)c->es, (const T *)c->es,
                 (T *)c->edge, c->dims, mv, dtm);
        StageArgs a{mode, dt, c->Hm, dtm, nullptr, nullptr, nullptr};
        if (!launch_stage<T>(c->tile, c->occ, c->runs, c->ord, M, (const T *)yin, (const T *)c->w, (const T *)c->edge, (T *)v0, (T *)y1, (T *)acc,
                        (T *)cmp, c->dims, mv, a, c->stream)) c->launch_miss = true;
        c->launches += 3;
        return;
    }
    // advective operator (operator_adv_swm_mod.f90:81-96); the averaging of the
    // duplicated h vertices acts on the stage input in place, as in the reference
    const AdvView<T> &av = adv_view<T>(c);
    const int N = c->cfg.N, n = N + 1;
    const dim3 pb(32, 8), pg((n + 31) / 32, (n + 7) / 8, NPAN * M);
    const dim3 hg(1 + (12 * (N - 1) + HAVG_THREADS - 1) / HAVG_THREADS, M);
    const long long nvh = (long long)NPAN * av.hp * M;
    const dim3 vg((unsigned)((nvh + 255) / 256));
    const bool fork = c->side && c->branches;
    if (fork) {
        // The averaging of h and the wind halo depend on the stage input only, the
        // wind at the vertices and the advective tendencies (which read neither h
        // nor the mass flux) on k_co2contra: they run on the side stream beside
        // k_co2contra, k_flux and k_edge, and join before the stage kernel.
        cudaEventRecord(c->ev_fork, c->stream);
        cudaStreamWaitEvent(c->side, c->ev_fork, 0);
        launch_k(k_havg<T>, hg, dim3(HAVG_THREADS), 0, c->side, (T *)yin, (T *)c->hb, c->dims, dtm);
        cudaEventRecord(c->ev_havg, c->side);
        launch_k(k_vhalo<T>, vg, dim3(256), 0, c->side, (const T *)yin, (T *)c->vh, c->dims, av, M, dtm);
        if (!launch_co2contra<T>(c->tile, c->occ, c->runs, c->ord, M, (const T *)yin, (T *)c->w, (T *)c->es, c->dims, mv,
                            c->stream, dtm)) c->launch_miss = true;
        cudaEventRecord(c->ev_co2, c->stream);
        cudaStreamWaitEvent(c->side, c->ev_co2, 0);
        launch_adv<T>(c, yin, av, mv, dtm, c->side);
        cudaEventRecord(c->ev_side, c->side);
        cudaStreamWaitEvent(c->stream, c->ev_havg, 0);
    } else {
        if (!launch_co2contra<T>(c->tile, c->occ, c->runs, c->ord, M, (const T *)yin, (T *)c->w, (T *)c->es, c->dims, mv,
                            c->stream, dtm)) c->launch_miss = true;
        launch_k(k_havg<T>, hg, dim3(HAVG_THREADS), 0, c->stream, (T *)yin, (T *)c->hb, c->dims, dtm);
    }
    launch_k(k_flux<T>, pg, pb, 0, c->stream, (const T *)yin, (const T *)c->w, (T *)c->fl, (T *)c->fs, c->dims, av, dtm,
             ord_strip_lines(c->ord));
    launch_k(c->ord == 21 ? k_edge<T, 21> : (c->ord == 63 ? k_edge<T, 63> : k_edge<T, 42>), edge_grid(c), dim3(EDGE_THREADS), 0, c->stream, (const T *)c->es, (const T *)c->fs,
             (T *)c->edge, c->dims, mv, dtm);
    if (fork) {
        cudaStreamWaitEvent(c->stream, c->ev_side, 0);
    } else {
        launch_k(k_vhalo<T>, vg, dim3(256), 0, c->stream, (const T *)yin, (T *)c->vh, c->dims, av, M, dtm);
        launch_adv<T>(c, yin, av, mv, dtm, c->stream);
    }
    StageArgs a{mode, dt, c->ones, dtm, c->fl, c->adt, c->hb, c->hs};
    if (!launch_stage<T>(c->tile, c->occ, c->runs, c->ord, M, (const T *)yin, (const T *)c->w, (const T *)c->edge, (T *)v0, (T *)y1, (T *)acc,
                    (T *)cmp, c->dims, mv, a, c->stream)) c->launch_miss = true;
    c->launches += 7;
}

static void enqueue_apply(swe_ctx *c, void *out, const void *in)
{
    if (c->elem == 8) enqueue_stage<double>(c, in, nullptr, out, nullptr, nullptr, 0, 0.0, nullptr, c->m64.v);
    else enqueue_stage<float>(c, in, nullptr, out, nullptr, nullptr, 0, 0.0, nullptr, c->m32.v);
}

// C-grid kernels: one thread per point of the (N+1) x (N+1) box, 32 x 8 blocks.
static dim3 c_grid_dims(const swe_ctx *c) { const int n = c->cfg.N + 1; return dim3((n + 31) / 32, (n + 7) / 8, NPAN * c->cfg.n_members); }

// The linear operator and what builds on it do not exist on the C staggering (the
// reference's linear operator aborts in its C-grid Coriolis operator).
#define CHSWE_NOT_ON_C(ctx, what)                                                                              \
    do {                                                                                                       \
        if ((ctx)->cstag)                                                                                      \
            return fail((ctx), SWE_EINVAL,                                                                     \
                        "%s: the linear operator on the C staggering calls coriolis_Cgrid_t%%calc_coriolis, " \
                        "which aborts in the reference; C contexts offer swe_c_grad, swe_c_div and "          \
                        "swe_operator_contravariant",                                                          \
                        what);                                                                                 \
    } while (0)

extern "C" int swe_operator_apply(swe_ctx *c, swe_stvec *vout, const swe_stvec *vin)
{
    if (!c || !vout || !vin || vout->ctx != c || vin->ctx != c || vout == vin) return SWE_EINVAL;
    CHSWE_NOT_ON_C(c, "swe_operator_apply");
    enqueue_apply(c, vout->d, vin->d);
    CU_LAUNCHED(c);
    return SWE_OK;
}

// vout.u, vout.v = contravariant components of (vin.u, vin.v); vout.h is left as is.
extern "C" int swe_operator_contravariant(swe_ctx *c, swe_stvec *vout, const swe_stvec *vin)
{
    if (!c || !vout || !vin || vout->ctx != c || vin->ctx != c || vout == vin) return SWE_EINVAL;
    if (c->ah) return fail(c, SWE_EINVAL, "swe_operator_contravariant: built for the Ch and C staggerings");
    if (c->cstag) {
        // co2contra_c_sbp42_new
        if (c->elem == 8) launch_k(k_c_co2contra<double>, c_grid_dims(c), dim3(32, 8), 0, c->stream, (const double *)vin->d, (double *)vout->d, c->dims, c_view<double>(c));
        else launch_k(k_c_co2contra<float>, c_grid_dims(c), dim3(32, 8), 0, c->stream, (const float *)vin->d, (float *)vout->d, c->dims, c_view<float>(c));
        c->launches++;
        CU_LAUNCHED(c);
        return SWE_OK;
    }
    const int M = c->cfg.n_members;
    bool ok;
    if (c->elem == 8) {
        ok = launch_co2contra<double>(c->tile, c->occ, c->runs, c->ord, M, (const double *)vin->d, (double *)vout->d,
                                      (double *)c->es, c->dims, c->m64.v, c->stream);
    } else {
        ok = launch_co2contra<float>(c->tile, c->occ, c->runs, c->ord, M, (const float *)vin->d, (float *)vout->d,
                                     (float *)c->es, c->dims, c->m32.v, c->stream);
    }
    if (!ok) return fail(c, SWE_EINVAL, "swe_operator_contravariant: no built contravariant kernel for the configuration");
    c->launches++;
    CU_LAUNCHED(c);
    return SWE_OK;
}


extern "C" int swe_c_grad(swe_ctx *c, swe_stvec *vout, const swe_stvec *vin)
{
    if (!c || !vout || !vin || vout->ctx != c || vin->ctx != c || vout == vin) return SWE_EINVAL;
    if (!c->cstag) return fail(c, SWE_EINVAL, "swe_c_grad: the context has no C staggering");
    if (c->elem == 8) launch_k(k_c_grad<double>, c_grid_dims(c), dim3(32, 8), 0, c->stream, (const double *)vin->d, (double *)vout->d, c->dims, c_view<double>(c));
    else launch_k(k_c_grad<float>, c_grid_dims(c), dim3(32, 8), 0, c->stream, (const float *)vin->d, (float *)vout->d, c->dims, c_view<float>(c));
    c->launches++;
    CU_LAUNCHED(c);
    return SWE_OK;
}

extern "C" int swe_c_div(swe_ctx *c, swe_stvec *vout, const swe_stvec *vin)
{
    if (!c || !vout || !vin || vout->ctx != c || vin->ctx != c || vout == vin) return SWE_EINVAL;
    if (!c->cstag) return fail(c, SWE_EINVAL, "swe_c_div: the context has no C staggering");
    if (c->elem == 8) launch_k(k_c_div<double>, c_grid_dims(c), dim3(32, 8), 0, c->stream, (const double *)vin->d, (double *)vout->d, c->dims, c_view<double>(c));
    else launch_k(k_c_div<float>, c_grid_dims(c), dim3(32, 8), 0, c->stream, (const float *)vin->d, (float *)vout->d, c->dims, c_view<float>(c));
    c->launches++;
    CU_LAUNCHED(c);
    return SWE_OK;
}

template <class T>
static int enqueue_diffusion(swe_ctx *c, T *y, T *out, double dt, const double *dtm, int lap_order, double uv_coeff,
                             double h_coeff);

// One RK4 step (four stages: stage s reads its input and writes the next one, double
// buffered), then the diffusion step when one is set (shallow_water_mod.f90:112-118).
static void enqueue_rk4(swe_ctx *c, swe_stvec *v0, double dt, const double *dtm = nullptr)
{
    void *V = v0->d, *A = c->acc;
    if (c->elem == 8) {
        const MetricView<double> &m = c->m64.v;
        enqueue_stage<double>(c, V, V, c->yb, A, nullptr, 1, dt, dtm, m);
        enqueue_stage<double>(c, c->yb, V, c->ya, A, nullptr, 2, dt, dtm, m);
        enqueue_stage<double>(c, c->ya, V, c->yb, A, nullptr, 3, dt, dtm, m);
        enqueue_stage<double>(c, c->yb, V, nullptr, A, nullptr, 4, dt, dtm, m);
    } else {
        const MetricView<float> &m = c->m32.v;
        enqueue_stage<float>(c, V, V, c->yb, A, v0->cmp, 1, dt, dtm, m);
        enqueue_stage<float>(c, c->yb, V, c->ya, A, v0->cmp, 2, dt, dtm, m);
        enqueue_stage<float>(c, c->ya, V, c->yb, A, v0->cmp, 3, dt, dtm, m);
        enqueue_stage<float>(c, c->yb, V, nullptr, A, v0->cmp, 4, dt, dtm, m);
    }
    // the scratch and tables exist (swe_set_diffusion set them up outside any capture)
    if (c->dif_order && c->elem == 8) enqueue_diffusion<double>(c, (double *)V, nullptr, dt, dtm, c->dif_order, c->dif_uv, c->dif_h);
    else if (c->dif_order) enqueue_diffusion<float>(c, (float *)V, nullptr, dt, dtm, c->dif_order, c->dif_uv, c->dif_h);
}

static int ensure_cmp(swe_stvec *v)
{
    swe_ctx *c = v->ctx;
    if (c->elem == 4 && !v->cmp) {
        size_t bytes = c->box_elems * 4;
        if (cudaMalloc(&v->cmp, bytes) != cudaSuccess) return fail(c, SWE_ENOMEM, "compensation allocation failed");
        CU(c, cudaMemsetAsync(v->cmp, 0, bytes, c->stream));
    }
    return SWE_OK;
}

extern "C" int swe_rk4_step(swe_ctx *c, swe_stvec *v0, double dt)
{
    if (!c || !v0 || v0->ctx != c) return SWE_EINVAL;
    CHSWE_NOT_ON_C(c, "swe_rk4_step");
    int rc = ensure_cmp(v0);
    if (rc) return rc;
    enqueue_rk4(c, v0, dt);
    CU_LAUNCHED(c);
    return SWE_OK;
}

// RK4 steps per replay of the long graph: enough to hide the gaps between graph
// launches, small enough that a remainder costs little.
constexpr int GRAPH_STEPS = 8;

static int capture_steps(swe_ctx *c, swe_stvec *v0, double dt, bool members, int steps, cudaGraphExec_t *out,
                         int *kernels)
{
    cudaGraph_t g;
    long long before = c->launches;
    CU(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    for (int s = 0; s < steps; s++) enqueue_rk4(c, v0, dt, members ? c->dtm : nullptr);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (e != cudaSuccess) return fail(c, SWE_ECUDA, "graph capture: %s", cudaGetErrorString(e));
    *kernels = (int)(c->launches - before);
    c->launches = before;
    if (c->launch_miss) {
        cudaGraphDestroy(g);
        c->launch_miss = false;
        return fail(c, SWE_EINVAL, "no built stage-kernel configuration matches the context's; nothing was captured");
    }
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(c, SWE_ECUDA, "graph instantiate: %s", cudaGetErrorString(e));
    return SWE_OK;
}

// nsteps replays of captured RK4 steps (GRAPH_STEPS per replay, then single steps);
// members == true uses the per-member time steps in c->dtm (captured by pointer,
// so new values need no new capture).
static int run_steps(swe_ctx *c, swe_stvec *v0, double dt, bool members, int nsteps)
{
    int rc = ensure_cmp(v0);
    if (rc) return rc;
    if (nsteps == 0) return SWE_OK;
    if (c->graph_v0 != v0->d || c->graph_members != members || (!members && c->graph_dt != dt)) {
        if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
        if (c->graphk) { cudaGraphExecDestroy(c->graphk); c->graphk = nullptr; }
        c->graph_v0 = v0->d;
        c->graph_dt = dt;
        c->graph_members = members;
    }
    const int full = nsteps / GRAPH_STEPS, rest = nsteps % GRAPH_STEPS;
    if (full > 0 && !c->graphk && (rc = capture_steps(c, v0, dt, members, GRAPH_STEPS, &c->graphk, &c->graphk_kernels)))
        return rc;
    if (rest > 0 && !c->graph && (rc = capture_steps(c, v0, dt, members, 1, &c->graph, &c->graph_kernels))) return rc;
    for (int s = 0; s < full; s++) {
        CU(c, cudaGraphLaunch(c->graphk, c->stream));
        c->launches += c->graphk_kernels;
    }
    for (int s = 0; s < rest; s++) {
        CU(c, cudaGraphLaunch(c->graph, c->stream));
        c->launches += c->graph_kernels;
    }
    return SWE_OK;
}

extern "C" int swe_rk4_steps(swe_ctx *c, swe_stvec *v0, double dt, int nsteps)
{
    if (!c || !v0 || v0->ctx != c || nsteps < 0) return SWE_EINVAL;
    CHSWE_NOT_ON_C(c, "swe_rk4_steps");
    return run_steps(c, v0, dt, false, nsteps);
}

extern "C" int swe_rk4_steps_members(swe_ctx *c, swe_stvec *v0, const double *dt, int nsteps)
{
    if (!c || !v0 || v0->ctx != c || !dt || nsteps < 0) return SWE_EINVAL;
    CHSWE_NOT_ON_C(c, "swe_rk4_steps_members");
    const int M = c->cfg.n_members;
    for (int k = 0; k < M; k++)
        if (!(dt[k] >= 0.0) || !std::isfinite(dt[k]))
            return fail(c, SWE_EINVAL, "member %d: time step %g (need finite, >= 0)", k, dt[k]);
    if (nsteps == 0) return SWE_OK;
    CU(c, cudaMemcpyAsync(c->dtm, dt, sizeof(double) * M, cudaMemcpyHostToDevice, c->stream));
    return run_steps(c, v0, 0.0, true, nsteps);
}

// ---------------------------------------------------------------------------
// Groups: the RK4 steps of several contexts as one grid per kernel
// ---------------------------------------------------------------------------

struct swe_group {
    std::vector<swe_ctx *> ctx;
    size_t elem = 8;
    int tile = 25, occ = 3, runs = 0;
    cudaStream_t stream = nullptr;     // the first context's stream
    cudaEvent_t ev = nullptr;          // joins the contexts' streams and the group's
    std::vector<const void *> graph_v; // the states the captured graphs advance
    cudaGraphExec_t graph = nullptr, graphk = nullptr;   // one RK4 step, GRAPH_STEPS steps
    long long launches = 0;
    std::string err;
};

static int gfail(swe_group *g, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g->err = buf;
    return code;
}

static bool group_cfg_built(int tm, int occ, int runs)
{
    bool found = false;
#define CHSWE_IS_GCFG(TM, OCC, RUNS) found = found || (tm == TM && occ == OCC && runs == RUNS);
    CHSWE_GROUP_CFGS(CHSWE_IS_GCFG)
#undef CHSWE_IS_GCFG
    return found;
}

static void group_drop_graphs(swe_group *g)
{
    if (g->graph) { cudaGraphExecDestroy(g->graph); g->graph = nullptr; }
    if (g->graphk) { cudaGraphExecDestroy(g->graphk); g->graphk = nullptr; }
    g->graph_v.clear();
}

extern "C" int swe_group_create(swe_ctx *const *ctxs, int n, swe_group **out)
{
    if (!out) return SWE_EINVAL;
    *out = nullptr;
    if (!ctxs || n < 1 || n > GROUP_MAX || !ctxs[0]) return SWE_EINVAL;
    swe_ctx *c0 = ctxs[0];
    for (int k = 0; k < n; k++) {
        swe_ctx *c = ctxs[k];
        if (!c) return fail(c0, SWE_EINVAL, "group: context %d is null", k);
        for (int q = 0; q < k; q++)
            if (ctxs[q] == c) return fail(c0, SWE_EINVAL, "group: context %d appears twice", k);
        if (c->device != c0->device || c->elem != c0->elem)
            return fail(c0, SWE_EINVAL, "group: context %d has another device or precision than context 0", k);
        if (c->adv || c->ah || c->cstag || c->ord != 42)
            return fail(c0, SWE_EINVAL, "group: context %d is not the linear operator on Ch in SBP 4-2", k);
        if (c->fused || c->tile != c0->tile || c->occ != c0->occ || c->runs != c0->runs)
            return fail(c0, SWE_EINVAL, "group: context %d has another kernel configuration than context 0 "
                        "(the contexts share one split configuration)", k);
    }
    if (c0->fused || !group_cfg_built(c0->tile, c0->occ, c0->runs))
        return fail(c0, SWE_EINVAL, "group: kernel configuration (%d, %d, %d) has no group launch; built: "
                    "(17, 4, 0), (25, 3, 0), (33, 2, 0)", c0->tile, c0->occ, c0->runs);
    swe_group *g = new swe_group;
    g->ctx.assign(ctxs, ctxs + n);
    g->elem = c0->elem;
    g->tile = c0->tile;
    g->occ = c0->occ;
    g->runs = c0->runs;
    g->stream = c0->stream;
    if (cudaSetDevice(c0->device) != cudaSuccess || cudaEventCreateWithFlags(&g->ev, cudaEventDisableTiming) != cudaSuccess) {
        delete g;
        return fail(c0, SWE_ECUDA, "group: event creation failed");
    }
    *out = g;
    return SWE_OK;
}

extern "C" int swe_group_destroy(swe_group *g)
{
    if (!g) return SWE_OK;
    cudaSetDevice(g->ctx[0]->device);
    cudaStreamSynchronize(g->stream);
    group_drop_graphs(g);
    if (g->ev) cudaEventDestroy(g->ev);
    delete g;
    return SWE_OK;
}

extern "C" const char *swe_group_last_error(const swe_group *g) { return g ? g->err.c_str() : "null group"; }

extern "C" long long swe_group_launch_count(const swe_group *g) { return g ? g->launches : -1; }

template <class T>
static const MetricView<T> &metric_view(const swe_ctx *c);
template <> const MetricView<double> &metric_view<double>(const swe_ctx *c) { return c->m64.v; }
template <> const MetricView<float> &metric_view<float>(const swe_ctx *c) { return c->m32.v; }

// The table of one group step: every context's state and scratch, its tiles from
// flat block tile0 on and its edge chunks from edge0 on.
template <class T>
static void group_table(const swe_group *g, swe_stvec *const *st, GroupTable<T> &tab, unsigned &tiles,
                        unsigned &edges)
{
    tab = GroupTable<T>{};
    tab.n = (int)g->ctx.size();
    tiles = edges = 0;
    for (int k = 0; k < tab.n; k++) {
        const swe_ctx *c = g->ctx[k];
        GroupEntry<T> &e = tab.e[k];
        e.d = c->dims;
        e.m = metric_view<T>(c);
        e.v = (T *)st[k]->d;
        e.ya = (T *)c->ya;
        e.yb = (T *)c->yb;
        e.acc = (T *)c->acc;
        e.cmp = sizeof(T) == 4 ? (T *)st[k]->cmp : nullptr;
        e.w = (T *)c->w;
        e.es = (T *)c->es;
        e.e = (T *)c->edge;
        e.Hm = c->Hm;
        e.dtm = c->dtm;
        const dim3 sg = stage_grid(c->cfg.N, c->cfg.n_members, g->tile), eg = edge_grid(c);
        e.gx = sg.x;
        e.gy = sg.y;
        e.nch = eg.x;
        e.tile0 = tiles;
        e.edge0 = edges;
        tiles += sg.x * sg.y * sg.z;
        edges += eg.x * eg.y * eg.z;
    }
}

template <class T>
static bool group_enqueue_step(swe_group *g, swe_stvec *const *st)
{
    GroupTable<T> tab;
    unsigned tiles, edges;
    group_table<T>(g, st, tab, tiles, edges);
    if (!GroupTU<T>::rk4_step(g->tile, g->occ, g->runs, tab, tiles, edges, g->stream)) return false;
    g->launches += 12;
    return true;
}

static int group_capture(swe_group *g, swe_stvec *const *st, int steps, cudaGraphExec_t *out)
{
    cudaGraph_t gr;
    const long long before = g->launches;
    if (cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return gfail(g, SWE_ECUDA, "group: graph capture failed to begin");
    bool ok = true;
    for (int s = 0; s < steps && ok; s++)
        ok = g->elem == 8 ? group_enqueue_step<double>(g, st) : group_enqueue_step<float>(g, st);
    cudaError_t e = cudaStreamEndCapture(g->stream, &gr);
    g->launches = before;
    if (e != cudaSuccess) return gfail(g, SWE_ECUDA, "group: graph capture: %s", cudaGetErrorString(e));
    if (!ok) {
        cudaGraphDestroy(gr);
        return gfail(g, SWE_EINVAL, "group: no group launch for the kernel configuration");
    }
    e = cudaGraphInstantiate(out, gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) return gfail(g, SWE_ECUDA, "group: graph instantiate: %s", cudaGetErrorString(e));
    return SWE_OK;
}

extern "C" int swe_group_rk4_steps_members(swe_group *g, swe_stvec *const *states, const double *const *dt,
                                           int nsteps)
{
    if (!g || !states || !dt || nsteps < 0) return SWE_EINVAL;
    const int n = (int)g->ctx.size();
    for (int k = 0; k < n; k++) {
        swe_ctx *c = g->ctx[k];
        if (!states[k] || states[k]->ctx != c) return gfail(g, SWE_EINVAL, "group: state %d is not of context %d", k, k);
        if (!dt[k]) return gfail(g, SWE_EINVAL, "group: no time steps for context %d", k);
        for (int m = 0; m < c->cfg.n_members; m++)
            if (!(dt[k][m] >= 0.0) || !std::isfinite(dt[k][m]))
                return gfail(g, SWE_EINVAL, "group: context %d member %d: time step %g (need finite, >= 0)", k, m,
                             dt[k][m]);
        if (c->fused || c->tile != g->tile || c->occ != g->occ || c->runs != g->runs)
            return gfail(g, SWE_EINVAL, "group: context %d changed its kernel configuration", k);
    }
    if (nsteps == 0) return SWE_OK;
    if (cudaSetDevice(g->ctx[0]->device) != cudaSuccess) return gfail(g, SWE_ECUDA, "group: cudaSetDevice failed");
    for (int k = 0; k < n; k++) {
        int rc = ensure_cmp(states[k]);
        if (rc) return gfail(g, rc, "group: context %d: %s", k, g->ctx[k]->err.c_str());
    }
    // the group's stream waits for the work queued on every context's own stream
    for (int k = 1; k < n; k++)
        if (g->ctx[k]->stream != g->stream) {
            if (cudaEventRecord(g->ev, g->ctx[k]->stream) != cudaSuccess ||
                cudaStreamWaitEvent(g->stream, g->ev, 0) != cudaSuccess)
                return gfail(g, SWE_ECUDA, "group: stream join failed");
        }
    for (int k = 0; k < n; k++) {
        swe_ctx *c = g->ctx[k];
        if (cudaMemcpyAsync(c->dtm, dt[k], sizeof(double) * c->cfg.n_members, cudaMemcpyHostToDevice, g->stream) !=
            cudaSuccess)
            return gfail(g, SWE_ECUDA, "group: time step upload failed");
    }
    std::vector<const void *> v(n);
    for (int k = 0; k < n; k++) v[k] = states[k]->d;
    if (v != g->graph_v) {
        group_drop_graphs(g);
        g->graph_v = v;
    }
    const int full = nsteps / GRAPH_STEPS, rest = nsteps % GRAPH_STEPS;
    int rc;
    if (full > 0 && !g->graphk && (rc = group_capture(g, states, GRAPH_STEPS, &g->graphk))) return rc;
    if (rest > 0 && !g->graph && (rc = group_capture(g, states, 1, &g->graph))) return rc;
    for (int s = 0; s < full; s++) {
        if (cudaGraphLaunch(g->graphk, g->stream) != cudaSuccess) return gfail(g, SWE_ECUDA, "group: graph launch failed");
        g->launches += 12 * GRAPH_STEPS;
    }
    for (int s = 0; s < rest; s++) {
        if (cudaGraphLaunch(g->graph, g->stream) != cudaSuccess) return gfail(g, SWE_ECUDA, "group: graph launch failed");
        g->launches += 12;
    }
    // every context's own stream waits for the group's steps
    if (cudaEventRecord(g->ev, g->stream) != cudaSuccess) return gfail(g, SWE_ECUDA, "group: event record failed");
    for (int k = 1; k < n; k++)
        if (g->ctx[k]->stream != g->stream && cudaStreamWaitEvent(g->ctx[k]->stream, g->ev, 0) != cudaSuccess)
            return gfail(g, SWE_ECUDA, "group: stream join failed");
    return SWE_OK;
}

extern "C" int swe_group_synchronize(swe_group *g)
{
    if (!g) return SWE_EINVAL;
    if (cudaSetDevice(g->ctx[0]->device) != cudaSuccess || cudaStreamSynchronize(g->stream) != cudaSuccess)
        return gfail(g, SWE_ECUDA, "group: %s", cudaGetErrorString(cudaGetLastError()));
    return SWE_OK;
}

// ---------------------------------------------------------------------------
// FP64 integrals
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_quad(const T *__restrict__ y, const T *__restrict__ w, const double *__restrict__ qw, Dims d,
                       double *partial)
{
    // blockIdx.x: slice of the rows, blockIdx.y: term (0 mass, 1 <h,h>, 2 <u,ut>, 3 <v,vt>)
    const int term = blockIdx.y;
    const int n = d.N + 1, N = d.N;
    const int64_t npts = (int64_t)NPAN * n * n;
    double acc = 0.0;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < npts; k += (int64_t)gridDim.x * blockDim.x) {
        const int t = (int)(k / ((int64_t)n * n)), r = (int)(k % ((int64_t)n * n));
        const int j = r / n + 1, i = r % n + 1;
        const int64_t o = box_off(d.P, i, j);
        if (term <= 1) {
            double h = (double)y[0 * d.fs + t * d.ps + o];
            acc += (term == 0 ? h : h * h) * qw[o];
        } else if (term == 2) {
            if (i > N) continue;
            acc += (double)y[1 * d.fs + t * d.ps + o] * (double)w[1 * d.fs + t * d.ps + o] * qw[d.ps + o];
        } else {
            if (j > N) continue;
            acc += (double)y[2 * d.fs + t * d.ps + o] * (double)w[2 * d.fs + t * d.ps + o] * qw[2 * d.ps + o];
        }
    }
    __shared__ double sh[256];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = sh[0];
}

// ---------------------------------------------------------------------------
// horizontal diffusion on the Ah staggering (swe_diff.cuh)
// ---------------------------------------------------------------------------
template <class T>
static int dif_setup(swe_ctx *c)
{
    const int N = c->cfg.N, n = N + 1, P = c->dims.P;
    const size_t box = (size_t)c->dims.ps, M = (size_t)c->cfg.n_members;
    if (!c->dif_b) {
        // b1, b2 of the equiangular vertices on each panel (metric_2d_ecs_mod.f90:377-395),
        // then the 4-2 closure blocks of every boundary line
        const size_t nb = (size_t)NPAN * 6 * box, n42 = (size_t)2 * n * 2 * 48, n63 = (size_t)2 * n * 2 * 108;
        std::vector<T> h(nb + n42 + n63 + (size_t)2 * (3 + 5 + 7) * box, T(0));
        const double pi = 3.141592653589793238462643383279502884, hx = 0.5 * pi / N;
        for (int p = 0; p < NPAN; p++)
            for (int j = 1; j <= n; j++)
                for (int i = 1; i <= n; i++) {
                    const double al = -0.25 * pi + (i - 1) * hx, be = -0.25 * pi + (j - 1) * hx;
                    double bp[3], b1[3], b2[3];
                    b1p(al, be, bp);
                    p2r(p, bp, b1);
                    b2p(al, be, bp);
                    p2r(p, bp, b2);
                    const size_t o = (size_t)box_off(P, i, j);
                    for (int k = 0; k < 3; k++) {
                        h[((size_t)p * 6 + k) * box + o] = T(b1[k]);
                        h[((size_t)p * 6 + 3 + k) * box + o] = T(b2[k]);
                    }
                }
        const HostMetric mxy = host_metric(N, 0.0, 0.0);
        auto bq = [&](int dir, int line, int k) {   // Qi11 J at (k, line) or Qi22 J at (line, k)
            const size_t q = dir == 0 ? (size_t)(line - 1) * n + (k - 1) : (size_t)(k - 1) * n + (line - 1);
            return (dir == 0 ? mxy.Q1[q] : mxy.Q3[q]) * mxy.J[q];
        };
        // m_rc = sum_k w_rck b_k of each boundary line, rows R x columns C of a dense table
        auto blocks = [&](const double *W, int R, int C, size_t off) {
            for (int dir = 0; dir < 2; dir++)
                for (int line = 1; line <= n; line++)
                    for (int side = 0; side < 2; side++)
                        for (int r = 0; r < R; r++)
                            for (int cc = 0; cc < C; cc++) {
                                double m = 0.0;
                                for (int k = 1; k <= C; k++)
                                    m = m + W[((size_t)r * C + cc) * C + (k - 1)] * bq(dir, line, side ? n + 1 - k : k);
                                h[off + (size_t)dif_block_index(n, dir, line, side, R * C) + r * C + cc] = T(m);
                            }
        };
        if (N >= 11) {
            double D[6][8][8];
            lap42_dense(D);
            blocks(&D[0][0][0], 6, 8, nb);
        }
        if (N >= 17) {
            std::vector<double> E(9 * 12 * 12, 0.0);
            for (const Lap63Term &q : LAP63_M) E[((size_t)(q.r - 1) * 12 + (q.c - 1)) * 12 + (q.k - 1)] = q.w;
            blocks(E.data(), 9, 12, nb + n42);
        }
        // interior stencil weights of every vertex, the expressions of the reference's
        // interior sweeps (laplace_Ah_sbp21_narrow_mod.f90:131-143,
        // laplace_Ah_sbp42_narrow_mod.f90:263-282, laplace_Ah_sbp63_narrow_mod.f90:860-880)
        const size_t ow = nb + n42 + n63;
        for (int dir = 0; dir < 2; dir++)
            for (int j = 1; j <= n; j++)
                for (int i = 1; i <= n; i++) {
                    const int k = dir == 0 ? i : j, line = dir == 0 ? j : i;
                    auto bb = [&](int q) { return bq(dir, line, q); };
                    const size_t o = (size_t)box_off(P, i, j);
                    auto put = [&](int ord, int q, double w) {
                        const size_t base = ow + (ord == 21 ? 0 : (ord == 42 ? 2 * 3 * box : 2 * 8 * box));
                        h[base + ((size_t)dir * narrow_width(ord) + q) * box + o] = T(w);
                    };
                    if (k > 1 && k < n) {
                        const double bm = bb(k - 1), bc = bb(k), bp = bb(k + 1);
                        put(21, 0, (bm + bc) / 2);
                        put(21, 1, -(bm + 2 * bc + bp) / 2);
                        put(21, 2, (bp + bc) / 2);
                    }
                    if (k >= 7 && k <= n - 6) {
                        const double bmm = bb(k - 2), bm = bb(k - 1), bc = bb(k), bp = bb(k + 1), bpp = bb(k + 2);
                        put(42, 0, 1.0 / 6.0 * bm - 1.0 / 8.0 * bmm - 1.0 / 8.0 * bc);
                        put(42, 1, 1.0 / 6.0 * bmm + 1.0 / 6.0 * bp + 1.0 / 2.0 * bm + 1.0 / 2.0 * bc);
                        put(42, 2, -1.0 / 24.0 * bmm - 5.0 / 6.0 * bm - 5.0 / 6.0 * bp - 1.0 / 24.0 * bpp - 3.0 / 4.0 * bc);
                        put(42, 3, 1.0 / 6.0 * bm + 1.0 / 6.0 * bpp + 1.0 / 2.0 * bc + 1.0 / 2.0 * bp);
                        put(42, 4, 1.0 / 6.0 * bp - 1.0 / 8.0 * bc - 1.0 / 8.0 * bpp);
                    }
                    if (k >= 10 && k <= n - 9) {
                        const double bmmm = bb(k - 3), bmm = bb(k - 2), bm = bb(k - 1), bc = bb(k), bp = bb(k + 1),
                                     bpp = bb(k + 2), bppp = bb(k + 3);
                        const double a33 = 11.0 / 360, a32 = -1.0 / 40, a31 = -1.0 / 40, a30 = 11.0 / 360;
                        const double a23 = -1.0 / 20, a22 = -7.0 / 40, a21 = 3.0 / 10, a20 = -7.0 / 40, a2p = -1.0 / 20;
                        const double a13 = 1.0 / 40, a12 = 3.0 / 10, a11 = 17.0 / 40, a10 = 17.0 / 40, a1p = 3.0 / 10,
                                     a1q = 1.0 / 40;
                        const double c3 = -1.0 / 180, c2 = -1.0 / 8, c1 = -19.0 / 20, c0 = -101.0 / 180;
                        put(63, 0, a33 * bmmm + a32 * bmm + a31 * bm + a30 * bc);
                        put(63, 1, a23 * bmmm + a22 * bmm + a21 * bm + a20 * bc + a2p * bp);
                        put(63, 2, a13 * bmmm + a12 * bmm + a11 * bm + a10 * bc + a1p * bp + a1q * bpp);
                        put(63, 3, c3 * bmmm + c2 * bmm + c1 * bm + c0 * bc + c1 * bp + c2 * bpp + c3 * bppp);
                        put(63, 4, a13 * bppp + a12 * bpp + a11 * bp + a10 * bc + a1p * bm + a1q * bmm);
                        put(63, 5, a23 * bppp + a22 * bpp + a21 * bp + a20 * bc + a2p * bm);
                        put(63, 6, a33 * bppp + a32 * bpp + a31 * bp + a30 * bc);
                    }
                }
        if (cudaMalloc(&c->dif_b, h.size() * sizeof(T)) != cudaSuccess)
            return fail(c, SWE_ENOMEM, "diffusion basis allocation failed");
        CU(c, cudaMemcpy(c->dif_b, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    }
    if (!c->dif && cudaMalloc(&c->dif, 5 * M * DIF_FIELDS * NPAN * box * sizeof(T)) != cudaSuccess)
        return fail(c, SWE_ENOMEM, "diffusion scratch allocation failed");
    return SWE_OK;
}

// The diffusion coefficient of hordiff_scalar_t (diff_order 2, diff_coeff = coeff a hx,
// hordiff_factory_mod.f90:193-227, hordiff_scalar_mod.f90:46): -(coeff a hx)^4.
static double dif_coeff(const swe_ctx *c, double coeff)
{
    const double hx = 0.5 * 3.141592653589793238462643383279502884 / c->cfg.N;
    const double dc = coeff * c->cfg.radius * hx;
    return -1.0 * ((dc * dc) * (dc * dc));
}

// y: the state (read; updated in place unless out), out: the tendency (apply).
template <class T>
static int enqueue_diffusion(swe_ctx *c, T *y, T *out, double dt, const double *dtm, int lap_order, double uv_coeff,
                             double h_coeff)
{
    int rc = dif_setup<T>(c);
    if (rc) return rc;
    const int N = c->cfg.N, n = N + 1, M = c->cfg.n_members;
    const Dims d = c->dims;
    const size_t set = (size_t)M * DIF_FIELDS * NPAN * d.ps;
    T *X = (T *)c->dif, *D1X = X + set, *D1Y = X + 2 * set, *R = X + 3 * set, *A = X + 4 * set;
    const AhView<T> &av = ah_view<T>(c);
    const MetricView<T> &mv = metric_view<T>(c);
    const double hxa = 0.5 * 3.141592653589793238462643383279502884 / N * c->cfg.radius;
    const T *mb42 = (const T *)c->dif_b + (size_t)NPAN * 6 * d.ps, *mb63 = mb42 + (size_t)2 * n * 2 * 48;
    const T *w21 = mb63 + (size_t)2 * n * 2 * 108, *w42 = w21 + (size_t)2 * 3 * d.ps, *w63 = w42 + (size_t)2 * 5 * d.ps;
    const DifView<T> dv{(const T *)c->dif_b, mb42, mb63, w21, w42, w63, hxa * hxa};
    const dim3 pb(32, 8), pm((n + 31) / 32, (n + 7) / 8, NPAN * M), pf((n + 31) / 32, (n + 7) / 8, NPAN * M * DIF_FIELDS);
    const dim3 sg((4 * N + 255) / 256, 1, NPAN * M * DIF_FIELDS);
    launch_k(k_dif_prep<T>, pm, pb, 0, c->stream, (const T *)y, X, d, dv);
    // L(X) -> A, then L(A) -> X
    T *src = X, *dst = A;
    for (int pass = 0; pass < 2; pass++) {
        launch_k(lap_order == 63 ? k_dif_d1<T, 63> : (lap_order == 42 ? k_dif_d1<T, 42> : k_dif_d1<T, 21>), pf, pb, 0,
                 c->stream, (const T *)src, D1X, D1Y, d, av);
        launch_k(lap_order == 63 ? k_dif_lap<T, 63> : (lap_order == 42 ? k_dif_lap<T, 42> : k_dif_lap<T, 21>), pf, pb, 0,
                 c->stream, (const T *)src, (const T *)D1X, (const T *)D1Y, R, dst, d, av, dv);
        launch_k(k_dif_sync<T>, sg, dim3(256), 0, c->stream, (const T *)R, dst, d);
        std::swap(src, dst);
    }
    launch_k(k_dif_vraw<T>, pm, pb, 0, c->stream, (const T *)X, D1X, D1Y, d, dv, T(dif_coeff(c, uv_coeff)));
    if (out)
        launch_k(k_dif_update<T, true>, pm, pb, 0, c->stream, y, out, (const T *)X, (const T *)D1X, (const T *)D1Y, d, mv,
                 T(dif_coeff(c, h_coeff)), T(0), (const double *)nullptr);
    else
        launch_k(k_dif_update<T, false>, pm, pb, 0, c->stream, y, (T *)nullptr, (const T *)X, (const T *)D1X,
                 (const T *)D1Y, d, mv, T(dif_coeff(c, h_coeff)), T(dt), dtm);
    c->launches += 9;
    return SWE_OK;
}

static int diffusion_check(swe_ctx *c, int lap_order, const char *what)
{
    if (!c->ah)
        return fail(c, SWE_EINVAL,
                    "%s: the reference's narrow-Laplacian diffusion (hordiff_*_Ah_sbp_*_narrow) acts on the Ah "
                    "staggering; this context is not Ah",
                    what);
    if (lap_order != 21 && lap_order != 42 && lap_order != 63)
        return fail(c, SWE_EINVAL, "%s: no _sbp_%d_narrow diffusion (the orders are 21, 42 and 63)", what, lap_order);
    if (lap_order == 42 && c->cfg.N < 11)
        return fail(c, SWE_EINVAL, "%s: the _sbp_42_narrow closure blocks of six rows overlap below N = 11", what);
    if (lap_order == 63 && c->cfg.N < 17)
        return fail(c, SWE_EINVAL, "%s: the _sbp_63_narrow closure blocks of nine rows overlap below N = 17", what);
    return SWE_OK;
}

extern "C" int swe_diffusion_apply(swe_ctx *c, swe_stvec *vout, const swe_stvec *vin, int lap_order, double uv_coeff,
                                   double h_coeff)
{
    if (!c || !vout || !vin || vout->ctx != c || vin->ctx != c || vout == vin) return SWE_EINVAL;
    int rc = diffusion_check(c, lap_order, "swe_diffusion_apply");
    if (rc) return rc;
    rc = c->elem == 8
             ? enqueue_diffusion<double>(c, (double *)vin->d, (double *)vout->d, 0.0, nullptr, lap_order, uv_coeff, h_coeff)
             : enqueue_diffusion<float>(c, (float *)vin->d, (float *)vout->d, 0.0, nullptr, lap_order, uv_coeff, h_coeff);
    if (rc) return rc;
    CU_LAUNCHED(c);
    return SWE_OK;
}

extern "C" int swe_diffusion_step(swe_ctx *c, swe_stvec *v, double dt, int lap_order, double uv_coeff, double h_coeff)
{
    if (!c || !v || v->ctx != c) return SWE_EINVAL;
    int rc = diffusion_check(c, lap_order, "swe_diffusion_step");
    if (rc) return rc;
    rc = c->elem == 8 ? enqueue_diffusion<double>(c, (double *)v->d, nullptr, dt, nullptr, lap_order, uv_coeff, h_coeff)
                      : enqueue_diffusion<float>(c, (float *)v->d, nullptr, dt, nullptr, lap_order, uv_coeff, h_coeff);
    if (rc) return rc;
    CU_LAUNCHED(c);
    return SWE_OK;
}

// The diffusion step after every RK4 step of swe_rk4_step(s) and swe_rk4_steps_members
// (with each member's time step; frozen members stay put), captured with the RK4 stages.
extern "C" int swe_set_diffusion(swe_ctx *c, int lap_order, double uv_coeff, double h_coeff)
{
    if (!c) return SWE_EINVAL;
    if (lap_order != 0) {
        int rc = diffusion_check(c, lap_order, "swe_set_diffusion");
        if (rc) return rc;
        rc = c->elem == 8 ? dif_setup<double>(c) : dif_setup<float>(c);
        if (rc) return rc;
    }
    if (c->dif_order != lap_order || c->dif_uv != uv_coeff || c->dif_h != h_coeff) drop_graph(c);
    c->dif_order = lap_order;
    c->dif_uv = uv_coeff;
    c->dif_h = h_coeff;
    return SWE_OK;
}

extern "C" int swe_integrals(swe_ctx *c, const swe_stvec *vec, int member, double *mass, double *energy)
{
    if (!c || !vec || vec->ctx != c || member < 0 || member >= c->cfg.n_members) return SWE_EINVAL;
    CHSWE_NOT_ON_C(c, "swe_integrals");
    if (c->ah) {
        const int nb = 256;
        const size_t mo = (size_t)member * c->dims.ms;
        const dim3 g(nb, 3), b(256);
        if (c->elem == 8) k_quad_ah<double><<<g, b, 0, c->stream>>>((const double *)vec->d + mo, c->qa, c->ah64.v, c->dims, c->red);
        else k_quad_ah<float><<<g, b, 0, c->stream>>>((const float *)vec->d + mo, c->qa, c->ah32.v, c->dims, c->red);
        c->launches += 1;
        CU_LAUNCHED(c);
        std::vector<double> part(nb * 3);
        CU(c, cudaMemcpyAsync(part.data(), c->red, part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CU(c, cudaStreamSynchronize(c->stream));
        double sum[3] = {0, 0, 0};
        for (int q = 0; q < 3; q++)
            for (int k = 0; k < nb; k++) sum[q] += part[q * nb + k];
        if (mass) *mass = sum[0];
        if (energy) *energy = 0.5 * c->Hhost[member] * sum[2] + 0.5 * c->cfg.grav * sum[1];
        return SWE_OK;
    }
    const int nb = 256;
    dim3 g(nb, 4), b(256);
    // contravariant components of this member into the scratch, then the four sums
    Dims d1 = c->dims;
    const size_t mo = (size_t)member * c->dims.ms;
    if (c->elem == 8) {
        if (!launch_co2contra<double>(c->tile, c->occ, c->runs, c->ord, 1, (const double *)vec->d + mo, (double *)c->w, (double *)c->es, d1, c->m64.v,
                                 c->stream)) c->launch_miss = true;
        k_quad<double><<<g, b, 0, c->stream>>>((const double *)vec->d + mo, (const double *)c->w, c->qw, d1, c->red);
    } else {
        if (!launch_co2contra<float>(c->tile, c->occ, c->runs, c->ord, 1, (const float *)vec->d + mo, (float *)c->w, (float *)c->es, d1, c->m32.v,
                                c->stream)) c->launch_miss = true;
        k_quad<float><<<g, b, 0, c->stream>>>((const float *)vec->d + mo, (const float *)c->w, c->qw, d1, c->red);
    }
    c->launches += 2;
    CU_LAUNCHED(c);
    std::vector<double> part(nb * 4);
    CU(c, cudaMemcpyAsync(part.data(), c->red, part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CU(c, cudaStreamSynchronize(c->stream));
    double s[4] = {0, 0, 0, 0};
    for (int q = 0; q < 4; q++)
        for (int k = 0; k < nb; k++) s[q] += part[q * nb + k];
    if (mass) *mass = s[0];
    if (energy) *energy = 0.5 * c->Hhost[member] * (s[2] + s[3]) + 0.5 * c->cfg.grav * s[1];
    return SWE_OK;
}

// Extrema for the diagnostics (swm_output_diag_mod.f90:110-154, :160-171).  Per
// block: term 0 max h, 1 min h (xy mesh), 2 max |(cx ut) u| (y mesh),
// 3 max |(cy vt) v| (x mesh); w holds (ut, vt).  FP64 arithmetic.
template <class T>
__global__ void k_extrema(const T *__restrict__ y, const T *__restrict__ w, Dims d, double cx, double cy,
                          double *partial)
{
    const int term = blockIdx.y;
    const int n = d.N + 1, N = d.N;
    const int64_t npts = (int64_t)NPAN * n * n;
    double acc = term == 1 ? INFINITY : (term == 0 ? -INFINITY : 0.0);
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < npts; k += (int64_t)gridDim.x * blockDim.x) {
        const int t = (int)(k / ((int64_t)n * n)), r = (int)(k % ((int64_t)n * n));
        const int j = r / n + 1, i = r % n + 1;
        const int64_t o = box_off(d.P, i, j) + t * d.ps;
        if (term <= 1) {
            const double h = (double)y[o];
            acc = term == 0 ? fmax(acc, h) : fmin(acc, h);
        } else if (term == 2) {
            if (i > N) continue;
            acc = fmax(acc, fabs(cx * (double)w[d.fs + o] * (double)y[d.fs + o]));
        } else {
            if (j > N) continue;
            acc = fmax(acc, fabs(cy * (double)w[2 * d.fs + o] * (double)y[2 * d.fs + o]));
        }
    }
    __shared__ double sh[256];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            sh[threadIdx.x] = term == 1 ? fmin(sh[threadIdx.x], sh[threadIdx.x + s]) : fmax(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = sh[0];
}

extern "C" int swe_diag(swe_ctx *c, const swe_stvec *vec, int member, double dt, double *out)
{
    if (!c || !vec || vec->ctx != c || !out || member < 0 || member >= c->cfg.n_members) return SWE_EINVAL;
    CHSWE_NOT_ON_C(c, "swe_diag");
    if (c->ah) return fail(c, SWE_EINVAL, "%s: built for the Ch staggering", "swe_diag");
    const int nb = 256;
    dim3 g(nb, 4), b(256);
    Dims d1 = c->dims;
    const size_t mo = (size_t)member * c->dims.ms;
    const double pi = 3.141592653589793238462643383279502884;
    const double dx = c->cfg.radius * (0.5 * pi / c->cfg.N);   // dx = dy on the xy mesh
    const double cxy = 1.0 / (dx * dx);
    if (c->elem == 8) {
        if (!launch_co2contra<double>(c->tile, c->occ, c->runs, c->ord, 1, (const double *)vec->d + mo, (double *)c->w,
                                 (double *)c->es, d1, c->m64.v, c->stream)) c->launch_miss = true;
        k_extrema<double><<<g, b, 0, c->stream>>>((const double *)vec->d + mo, (const double *)c->w, d1, cxy, cxy, c->red);
    } else {
        if (!launch_co2contra<float>(c->tile, c->occ, c->runs, c->ord, 1, (const float *)vec->d + mo, (float *)c->w,
                                (float *)c->es, d1, c->m32.v, c->stream)) c->launch_miss = true;
        k_extrema<float><<<g, b, 0, c->stream>>>((const float *)vec->d + mo, (const float *)c->w, d1, cxy, cxy, c->red);
    }
    c->launches += 2;
    CU_LAUNCHED(c);
    std::vector<double> part(nb * 4);
    CU(c, cudaMemcpyAsync(part.data(), c->red, part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CU(c, cudaStreamSynchronize(c->stream));
    double hmax = -INFINITY, hmin = INFINITY, umax = 0.0, vmax = 0.0;
    for (int k = 0; k < nb; k++) {
        hmax = std::max(hmax, part[k]);
        hmin = std::min(hmin, part[nb + k]);
        umax = std::max(umax, part[2 * nb + k]);
        vmax = std::max(vmax, part[3 * nb + k]);
    }
    out[0] = hmin;
    out[1] = hmax;
    // the reference scales with its constant Earth_grav; this uses the context's g
    out[2] = std::sqrt((c->cfg.grav / (dx * dx)) * hmax) * dt;
    out[3] = std::sqrt(umax) * dt;
    out[4] = std::sqrt(vmax) * dt;
    return SWE_OK;
}

// ---------------------------------------------------------------------------
// Curl, energies and potential enstrophy (swm_output_diag_t%calc_energies)
// ---------------------------------------------------------------------------
// The neighbour's copy of the tangential covariant component on side s of panel t,
// at along-edge centre c (1..N): u on its B and T sides, v on L and R, with the
// orientation sign.  It is the halo value (index 0 / N+2) that the Ch vector
// exchange (exchange_halo_Ch_mod.f90) gives the curl SAT.
template <class T>
__device__ __forceinline__ double tan_halo(const T *Y, const Dims &d, int t, int s, int c)
{
    const Link L = c_link[t][s];
    const int N = d.N, cp = L.rev ? N + 1 - c : c;
    double x;
    switch (L.nside) {
    case SIDE_L: x = (double)gview(Y, d, 2, L.nb)(1, cp); break;
    case SIDE_R: x = (double)gview(Y, d, 2, L.nb)(N + 1, cp); break;
    case SIDE_B: x = (double)gview(Y, d, 1, L.nb)(cp, 1); break;
    default: x = (double)gview(Y, d, 1, L.nb)(cp, N + 1); break;
    }
    return L.st * x;
}

// curl_sbp_sat_t%calc_curl_tile for curl_ch_sbp_sat_{21,42,63} (curl_sbp_sat_mod.f90:48-74):
// at cell centre (i, j) of panel t, the i2c differences of the covariant u along y
// and v along x with their SAT terms, (Dx / hx - Dy / hy) / (J a).  FP64.
template <class T, int ORD>
__device__ double curl_at(const T *Y, const Dims &d, int t, int i, int j, double hx, double Ja)
{
    using SB = SbpOrder<ORD>;
    const int N = d.N;
    const GV<T> U = gview(Y, d, 1, t), V = gview(Y, d, 2, t);
    double dy = SB::template di2c<double>(j, N, [&](int k) { return (double)U(i, k); });
    double dx = SB::template di2c<double>(i, N, [&](int k) { return (double)V(k, j); });
    if (j <= SB::NSAT) dy += SB::satw(j) * ((double)U(i, 1) - tan_halo(Y, d, t, SIDE_B, i));
    if (j >= N + 1 - SB::NSAT) dy += SB::satw(N + 1 - j) * (tan_halo(Y, d, t, SIDE_T, i) - (double)U(i, N + 1));
    if (i <= SB::NSAT) dx += SB::satw(i) * ((double)V(1, j) - tan_halo(Y, d, t, SIDE_L, j));
    if (i >= N + 1 - SB::NSAT) dx += SB::satw(N + 1 - i) * (tan_halo(Y, d, t, SIDE_R, j) - (double)V(N + 1, j));
    return (dx / hx - dy / hx) / Ja;
}

// The curl of one member on the cell centres, packed [panel][j][i] in FP64.
template <class T, int ORD>
__global__ void k_curl(const T *__restrict__ y, const double *__restrict__ otab, Dims d, double hx,
                       double *__restrict__ out)
{
    const int N = d.N;
    const int64_t npts = (int64_t)NPAN * N * N;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < npts; k += (int64_t)gridDim.x * blockDim.x) {
        const int t = (int)(k / ((int64_t)N * N)), r = (int)(k % ((int64_t)N * N));
        const int j = r / N + 1, i = r % N + 1;
        out[k] = curl_at<T, ORD>(y, d, t, i, j, hx, otab[box_off(d.P, i, j)]);
    }
}

// The four sums of calc_energies (swm_output_diag_mod.f90:186-234), per block:
// term 0 <h h>_xy, 1 <hu ut u / 2>_y, 2 <hv vt v / 2>_x with hu, hv = I_i2c(h),
// 3 <(curl + f)^2 / (2 hq)>_o with hq = (I_i2c,y(hu) + I_i2c,x(hv)) / 2.
// w holds (ut, vt) in its fields 1 and 2.  FP64 arithmetic.
template <class T, int ORD>
__global__ void k_energies(const T *__restrict__ y, const T *__restrict__ w, const double *__restrict__ qw,
                           const double *__restrict__ otab, Dims d, double hx, double *partial)
{
    using SB = SbpOrder<ORD>;
    const int term = blockIdx.y;
    const int n = d.N + 1, N = d.N;
    const int64_t npts = (int64_t)NPAN * n * n;
    double acc = 0.0;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < npts; k += (int64_t)gridDim.x * blockDim.x) {
        const int t = (int)(k / ((int64_t)n * n)), r = (int)(k % ((int64_t)n * n));
        const int j = r / n + 1, i = r % n + 1;
        const int64_t o = box_off(d.P, i, j);
        const GV<T> H = gview(y, d, 0, t);
        if (term == 0) {
            const double h = (double)H(i, j);
            acc += h * h * qw[o];
        } else if (term == 1) {
            if (i > N) continue;
            const double hu = SB::template ii2c<double>(i, N, [&](int q) { return (double)H(q, j); });
            acc += 0.5 * (hu * (double)w[1 * d.fs + t * d.ps + o]) * (double)y[1 * d.fs + t * d.ps + o] * qw[d.ps + o];
        } else if (term == 2) {
            if (j > N) continue;
            const double hv = SB::template ii2c<double>(j, N, [&](int q) { return (double)H(i, q); });
            acc += 0.5 * (hv * (double)w[2 * d.fs + t * d.ps + o]) * (double)y[2 * d.fs + t * d.ps + o] *
                   qw[2 * d.ps + o];
        } else {
            if (i > N || j > N) continue;
            const double hqu = SB::template ii2c<double>(j, N, [&](int q) {
                return SB::template ii2c<double>(i, N, [&](int p) { return (double)H(p, q); });
            });
            const double hqv = SB::template ii2c<double>(i, N, [&](int q) {
                return SB::template ii2c<double>(j, N, [&](int p) { return (double)H(q, p); });
            });
            const double hq = 0.5 * hqu + 0.5 * hqv;
            const double c = curl_at<T, ORD>(y, d, t, i, j, hx, otab[o]) + otab[(1 + t) * d.ps + o];
            acc += 0.5 * c * c / hq * qw[3 * d.ps + o];
        }
    }
    __shared__ double sh[256];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = sh[0];
}

// J a and the Coriolis parameter (calc_coriolis_parameter, coriolis_factory_mod.f90:239-280)
// on the cell centres, and room for one member's curl: built on first use.
static int ensure_otab(swe_ctx *c)
{
    if (c->otab) return SWE_OK;
    const int N = c->cfg.N, P = c->dims.P;
    const size_t box = (size_t)c->dims.ps;
    std::vector<double> h(7 * box, 0.0);
    const HostMetric m = host_metric(N, 0.5, 0.5);
    const MeshGeom g = mesh_geom(N, 0.5, 0.5);
    for (int j = 1; j <= N; j++)
        for (int i = 1; i <= N; i++) {
            const size_t k = (size_t)(j - 1) * m.nx + (i - 1), o = (size_t)box_off(P, i, j);
            h[o] = m.J[k] * c->cfg.radius;
            for (int p = 0; p < NPAN; p++) {
                double f = c->cfg.omega;
                if (!c->cfg.coriolis_constant) {
                    double r[3], a1[3], a2[3];
                    mesh_point(g, p, i, j, r, a1, a2);
                    const double *ax = c->cfg.rotation_axis;
                    f = 2 * c->cfg.omega * (ax[0] * r[0] + ax[1] * r[1] + ax[2] * r[2]) /
                        std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                }
                h[(1 + p) * box + o] = f;
            }
        }
    const size_t ncurl = (size_t)NPAN * N * N;
    if (cudaMalloc(&c->otab, (h.size() + ncurl) * sizeof(double)) != cudaSuccess) {
        c->otab = nullptr;
        return fail(c, SWE_ENOMEM, "diagnostic table allocation failed");
    }
    CU(c, cudaMemcpy(c->otab, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    return SWE_OK;
}

template <class T>
static void launch_curl(swe_ctx *c, const T *y, const Dims &d, double hx, double *out)
{
    const int64_t npts = (int64_t)NPAN * d.N * d.N;
    const dim3 g((unsigned)std::min<int64_t>((npts + 255) / 256, 4096)), b(256);
    if (c->ord == 21) k_curl<T, 21><<<g, b, 0, c->stream>>>(y, c->otab, d, hx, out);
    else if (c->ord == 63) k_curl<T, 63><<<g, b, 0, c->stream>>>(y, c->otab, d, hx, out);
    else k_curl<T, 42><<<g, b, 0, c->stream>>>(y, c->otab, d, hx, out);
}

template <class T>
static void launch_energies(swe_ctx *c, const T *y, const Dims &d, double hx, int nb)
{
    const dim3 g(nb, 4), b(256);
    const T *w = (const T *)c->w;
    if (c->ord == 21) k_energies<T, 21><<<g, b, 0, c->stream>>>(y, w, c->qw, c->otab, d, hx, c->red);
    else if (c->ord == 63) k_energies<T, 63><<<g, b, 0, c->stream>>>(y, w, c->qw, c->otab, d, hx, c->red);
    else k_energies<T, 42><<<g, b, 0, c->stream>>>(y, w, c->qw, c->otab, d, hx, c->red);
}

extern "C" int swe_curl(swe_ctx *c, const swe_stvec *vec, int member, double *out)
{
    if (!c || !vec || vec->ctx != c || !out || member < 0 || member >= c->cfg.n_members) return SWE_EINVAL;
    CHSWE_NOT_ON_C(c, "swe_curl");
    if (c->ah) return fail(c, SWE_EINVAL, "%s: built for the Ch staggering", "swe_curl");
    int rc = ensure_otab(c);
    if (rc != SWE_OK) return rc;
    const size_t mo = (size_t)member * c->dims.ms, box = (size_t)c->dims.ps;
    const size_t ncurl = (size_t)NPAN * c->cfg.N * c->cfg.N;
    const double hx = 0.5 * 3.141592653589793238462643383279502884 / c->cfg.N;
    double *dcurl = c->otab + 7 * box;
    if (c->elem == 8) launch_curl<double>(c, (const double *)vec->d + mo, c->dims, hx, dcurl);
    else launch_curl<float>(c, (const float *)vec->d + mo, c->dims, hx, dcurl);
    c->launches += 1;
    CU_LAUNCHED(c);
    CU(c, cudaMemcpyAsync(out, dcurl, ncurl * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CU(c, cudaStreamSynchronize(c->stream));
    return SWE_OK;
}

extern "C" int swe_energies(swe_ctx *c, const swe_stvec *vec, int member, double *out)
{
    if (!c || !vec || vec->ctx != c || !out || member < 0 || member >= c->cfg.n_members) return SWE_EINVAL;
    CHSWE_NOT_ON_C(c, "swe_energies");
    if (c->ah) return fail(c, SWE_EINVAL, "%s: built for the Ch staggering", "swe_energies");
    int rc = ensure_otab(c);
    if (rc != SWE_OK) return rc;
    const int nb = 256;
    const size_t mo = (size_t)member * c->dims.ms;
    const double hx = 0.5 * 3.141592653589793238462643383279502884 / c->cfg.N;
    Dims d1 = c->dims;
    if (c->elem == 8) {
        if (!launch_co2contra<double>(c->tile, c->occ, c->runs, c->ord, 1, (const double *)vec->d + mo, (double *)c->w,
                                 (double *)c->es, d1, c->m64.v, c->stream)) c->launch_miss = true;
        launch_energies<double>(c, (const double *)vec->d + mo, d1, hx, nb);
    } else {
        if (!launch_co2contra<float>(c->tile, c->occ, c->runs, c->ord, 1, (const float *)vec->d + mo, (float *)c->w,
                                (float *)c->es, d1, c->m32.v, c->stream)) c->launch_miss = true;
        launch_energies<float>(c, (const float *)vec->d + mo, d1, hx, nb);
    }
    c->launches += 2;
    CU_LAUNCHED(c);
    std::vector<double> part(nb * 4);
    CU(c, cudaMemcpyAsync(part.data(), c->red, part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CU(c, cudaStreamSynchronize(c->stream));
    double sum[4] = {0, 0, 0, 0};
    for (int q = 0; q < 4; q++)
        for (int k = 0; k < nb; k++) sum[q] += part[q * nb + k];
    // the reference scales the potential energy with its constant Earth_grav; this uses the context's g
    const double pe = 0.5 * c->cfg.grav * sum[0], ke = sum[1] + sum[2];
    out[0] = ke + pe;
    out[1] = ke;
    out[2] = pe;
    out[3] = sum[3];
    return SWE_OK;
}

// ---------------------------------------------------------------------------
// Lat-lon regrid of h (latlon_outputer_t with the cubic latlon_regrid_t)
// ---------------------------------------------------------------------------
// Width of the ECS_xy halo the cubic stencil reads (init_halo_for_interp,
// regrid_factory_mod.f90:273-276), and the pitch of the extended panel.
constexpr int LL_HW = 2;
__host__ __device__ __forceinline__ int ll_pitch(int N) { return N + 1 + 2 * LL_HW; }

// h of the neighbour across side s of panel t, `depth` nodes inside the neighbour,
// at along index a (1..N+1) of this side: the xy 'full' exchange's halo value at
// index -depth (L, B) or N+2+depth (R, T).
template <class T>
__device__ __forceinline__ double xy_nb(const T *Y, const Dims &d, int t, int s, int depth, int a)
{
    const Link L = c_link[t][s];
    const int ap = L.rev ? d.N + 2 - a : a;
    int k, l;
    side_vertex(d.N, L.nside, ap, depth, k, l);
    return (double)gview(Y, d, 0, L.nb)(k, l);
}

// ext_ecs_tile_halo (ecs_halo_xy_mod.f90:109-235) at one point (i, j) of the extended
// panel (indices 1-LL_HW .. N+1+LL_HW): the averaged duplicated vertices, the corner
// diagonals and the rows / columns of virtual points interpolated along the
// neighbours' grid lines (cubic Lagrange, weights wt / lines kt per depth and along
// index).  raw: the panel's own value at (i, j) when inside; X(s, depth, a): the
// exchange's halo value across side s at that depth and along index a.
template <class RAW, class XF>
__device__ __forceinline__ double ecs_ext_point(int i, int j, int n, const int *kt, const double *wt, const RAW &raw,
                                                const XF &X)
{
    // corner diagonals at offset m (1..LL_HW) from the four corner vertices
    auto DBL = [&](int m) { return 0.5 * (X(SIDE_L, m, 1) + X(SIDE_B, m, 1)); };
    auto DBR = [&](int m) { return 0.5 * (X(SIDE_R, m, 1) + X(SIDE_B, m, n)); };
    auto DTR = [&](int m) { return 0.5 * (X(SIDE_R, m, n) + X(SIDE_T, m, n)); };
    auto DTL = [&](int m) { return 0.5 * (X(SIDE_T, m, 1) + X(SIDE_L, m, n)); };
    // the neighbour's grid line at depth m along side s, its ends replaced by the diagonals
    auto line = [&](int s, int m, int b) {
        if (b == 1) return s == SIDE_R ? DBR(m) : (s == SIDE_T ? DTL(m) : DBL(m));
        if (b == n) return s == SIDE_L ? DTL(m) : (s == SIDE_B ? DBR(m) : DTR(m));
        return X(s, m, b);
    };
    auto virt = [&](int s, int m, int a) {
        const int row = (m - 1) * (n + 2) + a;   // a in 2-m .. n+m-1, i.e. 0 .. n+1
        const int k = kt[row];
        const double *w = wt + 4 * row;
        return w[0] * line(s, m, k - 1) + w[1] * line(s, m, k) + w[2] * line(s, m, k + 1) + w[3] * line(s, m, k + 2);
    };
    if (i >= 1 && i <= n && j >= 1 && j <= n) {
        const double r = raw();
        const bool il = i == 1, ir = i == n, jb = j == 1, jt = j == n;
        if (il && jb) return (r + X(SIDE_B, 0, 1) + X(SIDE_L, 0, 1)) / 3.0;
        if (ir && jb) return (r + X(SIDE_B, 0, n) + X(SIDE_R, 0, 1)) / 3.0;
        if (ir && jt) return (r + X(SIDE_T, 0, n) + X(SIDE_R, 0, n)) / 3.0;
        if (il && jt) return (r + X(SIDE_L, 0, n) + X(SIDE_T, 0, 1)) / 3.0;
        if (jb) return 0.5 * (r + X(SIDE_B, 0, i));
        if (jt) return 0.5 * (r + X(SIDE_T, 0, i));
        if (il) return 0.5 * (r + X(SIDE_L, 0, j));
        if (ir) return 0.5 * (r + X(SIDE_R, 0, j));
        return r;
    }
    if (j < 1 && i >= 2 - (1 - j) && i <= n + (1 - j) - 1) return virt(SIDE_B, 1 - j, i);
    if (j > n && i >= 2 - (j - n) && i <= n + (j - n) - 1) return virt(SIDE_T, j - n, i);
    if (i < 1 && j >= 2 - (1 - i) && j <= n + (1 - i) - 1) return virt(SIDE_L, 1 - i, j);
    if (i > n && j >= 2 - (i - n) && j <= n + (i - n) - 1) return virt(SIDE_R, i - n, j);
    if (i < 1) return j < 1 ? DBL(1 - i) : DTL(1 - i);
    return j < 1 ? DBR(i - n) : DTR(i - n);
}

// get_ecs_halo (ecs_halo_xy_mod.f90:66-107) of h on every panel: the xy exchange's
// values (xy_nb) and ext_ecs_tile_halo at every point.  FP64 into ext[panel][j][i].
template <class T>
__global__ void k_ecs_xy_ext(const T *__restrict__ y, Dims d, const int *__restrict__ kt,
                             const double *__restrict__ wt, double *__restrict__ ext)
{
    const int N = d.N, n = N + 1, E = ll_pitch(N);
    const int64_t npts = (int64_t)NPAN * E * E;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < npts; q += (int64_t)gridDim.x * blockDim.x) {
        const int t = (int)(q / ((int64_t)E * E)), r = (int)(q % ((int64_t)E * E));
        const int j = r / E + 1 - LL_HW, i = r % E + 1 - LL_HW;
        ext[q] = ecs_ext_point(
            i, j, n, kt, wt, [&]() { return (double)gview(y, d, 0, t)(i, j); },
            [&](int s, int depth, int a) { return xy_nb(y, d, t, s, depth, a); });
    }
}

// The covariant wind at vertex (k, l) of panel p, interpolated from the Ch points
// (interp2d_uv2pvec_Ch_sbp42: the c2i interpolation of u along x, of v along y).
template <class T>
__device__ __forceinline__ void uv_at_vertex(const T *y, const Dims &d, int p, int k, int l, double &u, double &v)
{
    const int n = d.N + 1;
    const GV<T> U = gview(y, d, 1, p), V = gview(y, d, 2, p);
    u = ic2i<double>(k, n, [&](int c) { return (double)U(c, l); });
    v = ic2i<double>(l, n, [&](int c) { return (double)V(k, c); });
}

// The covariant ecs_xy_vec halo of the wind (ecs_halo_vec_xy_mod.f90:30-98) on every
// panel: at each halo point the neighbour's vertex wind as the vector exchange hands
// it over (halo_vec), turned into this panel's components by the transform matrix
// of the edge, depth and along index (tm: [edge B, T, L, R][depth 0..LL_HW][a 1..n][4]);
// then ext_ecs_tile_halo of each component.  FP64 into extu, extv.
template <class T>
__global__ void k_ecs_vec_ext(const T *__restrict__ y, Dims d, const int *__restrict__ kt,
                              const double *__restrict__ wt, const double *__restrict__ tm, double *__restrict__ extu,
                              double *__restrict__ extv)
{
    const int N = d.N, n = N + 1, E = ll_pitch(N);
    const int64_t npts = (int64_t)NPAN * E * E;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < npts; q += (int64_t)gridDim.x * blockDim.x) {
        const int t = (int)(q / ((int64_t)E * E)), r = (int)(q % ((int64_t)E * E));
        const int j = r / E + 1 - LL_HW, i = r % E + 1 - LL_HW;
        double uo = 0.0, vo = 0.0;
        if (i >= 1 && i <= n && j >= 1 && j <= n) uv_at_vertex(y, d, t, i, j, uo, vo);
        for (int comp = 0; comp < 2; comp++) {
            auto X = [&](int s, int depth, int a) {
                const Link L = c_link[t][s];
                int k, l;
                side_vertex(N, L.nside, L.rev ? n + 1 - a : a, depth, k, l);
                double un, vn, uh, vh;
                uv_at_vertex(y, d, L.nb, k, l, un, vn);
                halo_vec<double>(t, s, un, vn, uh, vh);
                const int e = s == SIDE_B ? 0 : (s == SIDE_T ? 1 : (s == SIDE_L ? 2 : 3));
                const double *M = tm + ((e * (LL_HW + 1) + depth) * n + (a - 1)) * 4;
                return comp == 0 ? M[0] * uh + M[1] * vh : M[2] * uh + M[3] * vh;
            };
            const double v = ecs_ext_point(i, j, n, kt, wt, [&]() { return comp == 0 ? uo : vo; }, X);
            (comp == 0 ? extu : extv)[q] = v;
        }
    }
}

// interp_t%interpolate (latlon_regrid_mod.f90:338-365): the 4 x 4 cubic stencil of
// every lat-lon point on the extended panel, FP64.
// ext: the extended panels, pitch E, point (i, j) at [panel][j + 1][i + 1] from i, j = -1 on
// (the xy panels start at 1 - LL_HW = -1 too).
__global__ void k_latlon(const double *__restrict__ ext, const int *__restrict__ idx, const double *__restrict__ w,
                         int E, int64_t npts, double *__restrict__ out)
{
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < npts; q += (int64_t)gridDim.x * blockDim.x) {
        const int t = idx[3 * q], xi = idx[3 * q + 1], yi = idx[3 * q + 2];
        const double *wx = w + 8 * q, *wy = wx + 4;
        const double *e = ext + ((int64_t)t * E + (yi + LL_HW - 1)) * E + (xi + LL_HW - 1);
        double acc = 0.0;
        for (int b = -1; b <= 2; b++)
            for (int a = -1; a <= 2; a++) acc = acc + wx[a + 1] * wy[b + 1] * e[b * E + a];
        out[q] = acc;
    }
}

// do_latlon_vector_regrid (latlon_regrid_mod.f90:132-212): the stencils of both
// components and their rotation to the eastward / northward components
// (q: [iv.b1, iv.b2, jv.b1, jv.b2] per point).
__global__ void k_latlon_vec(const double *__restrict__ extu, const double *__restrict__ extv,
                             const int *__restrict__ idx, const double *__restrict__ w, const double *__restrict__ qr,
                             int N, int64_t npts, double *__restrict__ uo, double *__restrict__ vo)
{
    const int E = ll_pitch(N);
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < npts; q += (int64_t)gridDim.x * blockDim.x) {
        const int t = idx[3 * q], xi = idx[3 * q + 1], yi = idx[3 * q + 2];
        const double *wx = w + 8 * q, *wy = wx + 4;
        const int64_t base = ((int64_t)t * E + (yi + LL_HW - 1)) * E + (xi + LL_HW - 1);
        double au = 0.0, av = 0.0;
        for (int b = -1; b <= 2; b++)
            for (int a = -1; a <= 2; a++) {
                au = au + wx[a + 1] * wy[b + 1] * extu[base + b * E + a];
                av = av + wx[a + 1] * wy[b + 1] * extv[base + b * E + a];
            }
        const double *Q = qr + 4 * q;
        uo[q] = Q[0] * au + Q[1] * av;
        vo[q] = Q[2] * au + Q[3] * av;
    }
}

// Point location and cubic weights (distribute_latlon_points_to_cubsphere,
// regrid_factory_mod.f90:165-262; init_interpolation, latlon_regrid_mod.f90:286-336;
// latlon_grid_generator_t%init / get_cartesian_coords) and the ECS_xy halo weights
// (init_halo_xy_interp, ecs_halo_factory_mod.f90:236-270), built on the host in FP64.
// Layout of the lat-lon regrid's device tables (ll_i ints, ll_d doubles).
struct LatlonLayout {
    size_t np, nrow, ntm, next;
    // ints: idx (3 per point), kt (nrow)
    size_t i_kt() const { return 3 * np; }
    size_t ints() const { return 3 * np + nrow; }
    // doubles: w (8 per point), qrot (4 per point), wt (4 per row), tm, ext u/h, ext v, out u/h, out v
    size_t d_q() const { return 8 * np; }
    size_t d_wt() const { return 12 * np; }
    size_t d_tm() const { return d_wt() + 4 * nrow; }
    size_t d_ext() const { return d_tm() + ntm; }
    size_t d_out() const { return d_ext() + 2 * next; }
    size_t doubles() const { return d_out() + 2 * np; }
};
static LatlonLayout latlon_layout(int N, int nlat, int nlon)
{
    const int n = N + 1, E = ll_pitch(N);
    LatlonLayout L;
    L.np = (size_t)nlat * nlon;
    L.nrow = (size_t)LL_HW * (n + 2);
    L.ntm = (size_t)4 * (LL_HW + 1) * n * 4;
    L.next = (size_t)NPAN * E * E;
    return L;
}

// init_transform_matrix for covariant components (ecs_halo_vec_xy_factory_mod.f90:103-186):
// at halo row j (1: the neighbour's copy of the edge row) and along index i of edge e
// (1 bottom, 2 top, 3 left, 4 right), the matrix taking the neighbour's covariant
// components, as the vector exchange hands them over, to this panel's.
static void xy_vec_tm(int e, int i, int j, double hx, double TM[4])
{
    static const int rot[4][3][3] = {{{1, 0, 0}, {0, 0, -1}, {0, 1, 0}},
                                     {{1, 0, 0}, {0, 0, 1}, {0, -1, 0}},
                                     {{0, 0, -1}, {0, 1, 0}, {1, 0, 0}},
                                     {{0, 0, 1}, {0, 1, 0}, {-1, 0, 0}}};
    static const int ab_shift[4] = {0, 0, 1, 1}, b_sign[4] = {1, -1, 1, -1};
    const double pi = 3.141592653589793238462643383279502884;
    const int q = e - 1;
    const double alpha = -0.25 * pi + (i - 1.0) * hx;
    const double beta = b_sign[q] * (0.25 * pi - (j - 1.0) * hx);
    const double as = (1 - ab_shift[q]) * alpha + ab_shift[q] * beta;
    const double bs = ab_shift[q] * alpha + (1 - ab_shift[q]) * beta;
    auto rotate = [&](const double v[3], double out[3]) {
        for (int d = 0; d < 3; d++) out[d] = rot[q][d][0] * v[0] + rot[q][d][1] * v[1] + rot[q][d][2] * v[2];
    };
    double v[3], a1s[3], a2s[3], r[3], b1t[3], b2t[3];
    b1p(as, bs, v);
    rotate(v, a1s);
    b2p(as, bs, v);
    rotate(v, a2s);
    const double ta = std::tan(as), tb = std::tan(bs);
    v[0] = ta / std::sqrt(1.0 + std::pow(ta, 2.0) + std::pow(tb, 2.0));
    v[1] = tb / std::sqrt(1.0 + std::pow(ta, 2.0) + std::pow(tb, 2.0));
    v[2] = 1.0 / std::sqrt(1.0 + std::pow(ta, 2.0) + std::pow(tb, 2.0));
    rotate(v, r);
    const double at = std::atan(r[0] / r[2]), bt = std::atan(r[1] / r[2]);
    a1p(at, bt, b1t);
    a2p(at, bt, b2t);
    TM[0] = a1s[0] * b1t[0] + a1s[1] * b1t[1] + a1s[2] * b1t[2];
    TM[1] = a2s[0] * b1t[0] + a2s[1] * b1t[1] + a2s[2] * b1t[2];
    TM[2] = a1s[0] * b2t[0] + a1s[1] * b2t[1] + a1s[2] * b2t[2];
    TM[3] = a2s[0] * b2t[0] + a2s[1] * b2t[1] + a2s[2] * b2t[2];
}

// Point location and cubic weights (distribute_latlon_points_to_cubsphere,
// regrid_factory_mod.f90:165-262; init_interpolation, latlon_regrid_mod.f90:286-336;
// latlon_grid_generator_t%init / get_cartesian_coords / get_basis_vectors), the
// rotation to lat-lon components (init_transform_to_latlon_vec_tile,
// regrid_factory_mod.f90:324-370), the ECS_xy halo weights (init_halo_xy_interp,
// ecs_halo_factory_mod.f90:236-270) and the vector halo's transform matrices, built
// on the host in FP64.
static int ensure_latlon(swe_ctx *c, int nlat, int nlon)
{
    if (c->ll_i && c->ll_nlat == nlat && c->ll_nlon == nlon) return SWE_OK;
    cudaFree(c->ll_i); cudaFree(c->ll_d);
    c->ll_i = nullptr; c->ll_d = nullptr; c->ll_nlat = c->ll_nlon = 0;
    const int N = c->cfg.N, n = N + 1;
    const LatlonLayout Lo = latlon_layout(N, nlat, nlon);
    std::vector<int> hi(Lo.ints(), 0);
    std::vector<double> hd(Lo.d_ext(), 0.0);
    const double pi = 3.141592653589793238462643383279502884;
    const double hx = 0.5 * pi / N, a0 = -0.25 * pi;
    for (int j = 1; j <= nlat; j++) {
        const double phi = -0.5 * pi + (j - 1) * pi / (nlat - 1.0);
        for (int i = 1; i <= nlon; i++) {
            const double lam = (i - 1) * 2.0 * pi / nlon;
            const double r[3] = {std::cos(phi) * std::cos(lam), std::cos(phi) * std::sin(lam), std::sin(phi)};
            int t;
            double alpha, beta;
            cart_to_native(r, t, alpha, beta);
            double zdx = (alpha - a0) / hx + 1 - 0.0, zdy = (beta - a0) / hx + 1 - 0.0;
            const int xi = (int)zdx, yi = (int)zdy;
            zdx = zdx - xi;
            zdy = zdy - yi;
            const size_t q = (size_t)(j - 1) * nlon + (i - 1);
            hi[3 * q] = t; hi[3 * q + 1] = xi; hi[3 * q + 2] = yi;
            double *wx = &hd[8 * q], *wy = wx + 4;
            wx[0] = -zdx * (zdx - 1.0) * (zdx - 2.0) / 6.0;
            wx[1] = (zdx + 1.0) * (zdx - 1.0) * (zdx - 2.0) / 2.0;
            wx[2] = -(zdx + 1.0) * zdx * (zdx - 2.0) / 2.0;
            wx[3] = (zdx + 1.0) * zdx * (zdx - 1.0) / 6.0;
            wy[0] = -zdy * (zdy - 1.0) * (zdy - 2.0) / 6.0;
            wy[1] = (zdy + 1.0) * (zdy - 1.0) * (zdy - 2.0) / 2.0;
            wy[2] = -(zdy + 1.0) * zdy * (zdy - 2.0) / 2.0;
            wy[3] = (zdy + 1.0) * zdy * (zdy - 1.0) / 6.0;
            // the stencil (indices xi-1 .. xi+2) stays inside the extended panel
            if (t < 0 || t >= NPAN || xi < 0 || xi > n || yi < 0 || yi > n)
                return fail(c, SWE_EINVAL, "lat-lon point (%d, %d) outside the cube panels", i, j);
            // q = [iv.b1, iv.b2; jv.b1, jv.b2] with the panel's contravariant basis b1, b2
            const double iv[3] = {-std::sin(lam), std::cos(lam), 0.0};
            const double jv[3] = {-std::sin(phi) * std::cos(lam), -std::sin(phi) * std::sin(lam), std::cos(phi)};
            double p1[3], p2[3], b1[3], b2[3];
            b1p(alpha, beta, p1);
            b2p(alpha, beta, p2);
            p2r(t, p1, b1);
            p2r(t, p2, b2);
            double *Q = &hd[Lo.d_q() + 4 * q];
            Q[0] = iv[0] * b1[0] + iv[1] * b1[1] + iv[2] * b1[2];
            Q[1] = iv[0] * b2[0] + iv[1] * b2[1] + iv[2] * b2[2];
            Q[2] = jv[0] * b1[0] + jv[1] * b1[1] + jv[2] * b1[2];
            Q[3] = jv[0] * b2[0] + jv[1] * b2[1] + jv[2] * b2[2];
        }
    }
    for (int m = 1; m <= LL_HW; m++)
        for (int a = 2 - m; a <= n + m - 1; a++) {
            const size_t row = (size_t)(m - 1) * (n + 2) + a;
            halo_xy_weights(n, hx, a, m, &hd[Lo.d_wt() + 4 * row], hi[Lo.i_kt() + row]);
        }
    for (int e = 0; e < 4; e++)
        for (int dep = 0; dep <= LL_HW; dep++)
            for (int a = 1; a <= n; a++)
                xy_vec_tm(e + 1, a, dep + 1, hx, &hd[Lo.d_tm() + ((size_t)(e * (LL_HW + 1) + dep) * n + (a - 1)) * 4]);
    if (cudaMalloc(&c->ll_i, hi.size() * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c->ll_d, Lo.doubles() * sizeof(double)) != cudaSuccess) {
        cudaFree(c->ll_i); c->ll_i = nullptr; c->ll_d = nullptr;
        return fail(c, SWE_ENOMEM, "lat-lon regrid allocation failed");
    }
    CU(c, cudaMemcpy(c->ll_i, hi.data(), hi.size() * sizeof(int), cudaMemcpyHostToDevice));
    CU(c, cudaMemcpy(c->ll_d, hd.data(), hd.size() * sizeof(double), cudaMemcpyHostToDevice));
    c->ll_nlat = nlat;
    c->ll_nlon = nlon;
    return SWE_OK;
}

// ---------------------------------------------------------------------------
// Lat-lon regrid of the curl (output_curl's curl.dat): the curl on the cell centres,
// its ECS_O halo of width 2, the cubic stencils on the cell-centre mesh
// ---------------------------------------------------------------------------
// Extended cell-centre panels: cells -1 .. N+2 in each direction.
__host__ __device__ __forceinline__ int llo_pitch(int N) { return N + 4; }

// init_halo_interp (ecs_halo_factory_mod.f90:190-230): for the cell-centre line i of virtual
// row j beyond a panel edge, the source face's cell left of the projected point and the
// cubic Lagrange weights on its cells ind-1 .. ind+2 (host, FP64).
static void halo_o_weights(double dxa, int i, int j, double w[4], int &ind)
{
    const double pi = 3.141592653589793238462643383279502884;
    const double zb = 0.25 * pi + (j - 0.5) * dxa;
    double za = -0.25 * pi + (i - 0.5) * dxa;
    double zx = std::tan(za);
    const double zz = std::tan(zb);
    zx = zx / zz;
    za = std::atan(zx);
    ind = (int)std::floor((za + 0.25 * pi - 0.5 * dxa) / dxa) + 1;
    const double zxi = (za + 0.25 * pi) / dxa - (ind - 0.5);
    w[0] = -(zxi * (zxi - 1.0) * (zxi - 2.0) / 6.0);
    w[1] = (zxi + 1.0) * (zxi - 1.0) * (zxi - 2.0) / 2.0;
    w[2] = -((zxi + 1.0) * zxi * (zxi - 2.0) / 2.0);
    w[3] = (zxi + 1.0) * zxi * (zxi - 1.0) / 6.0;
}

// ext_ecs_tile_halo (ecs_halo_mod.f90:109-175) of a cell-centre field f[panel][j][i] (FP64,
// N x N per panel) at every point of the extended panels: the cells; the virtual rows of
// each side interpolated along the neighbour's grid line from its cells at the same
// depth (ecs_ext_halo_1e, the first row without its end points); and the six special
// points of each cube corner (ecs_halo_1corner, :230-300), from the cells and the
// neighbours' cells as the o-point exchange hands them over.  Weights wt / lines kt per
// row m = 1, 2 and line index i = -1 .. N+2 (the corners use those of i = -1 .. 2,
// mirrored at the corners with a reversed i direction).
__global__ void k_ecs_o_ext(const double *__restrict__ f, int N, const int *__restrict__ kt,
                            const double *__restrict__ wt, double *__restrict__ ext)
{
    const int E = llo_pitch(N), ni = N + 4;
    const int64_t total = (int64_t)NPAN * E * E;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int t = (int)(q / (E * E)), r = (int)(q % (E * E));
        const int i = r % E - 1, j = r / E - 1;
        auto cell = [&](int p, int k, int l) { return f[((int64_t)p * N + (l - 1)) * N + (k - 1)]; };
        // the exchange's value across side s at depth m, along index b (1..N) of this side
        auto X = [&](int s, int m, int b) {
            int p, k, l;
            c_halo_cell(N, t, s, b, m, p, k, l);
            return cell(p, k, l);
        };
        // the exchanged field: a cell of this panel or of a neighbour
        auto pf = [&](int x, int y) {
            if (y < 1) return X(SIDE_B, 1 - y, x);
            if (y > N) return X(SIDE_T, y - N, x);
            if (x < 1) return X(SIDE_L, 1 - x, y);
            if (x > N) return X(SIDE_R, x - N, y);
            return cell(t, x, y);
        };
        auto W = [&](int k, int a, int m) { return wt[4 * ((m - 1) * ni + a + 1) + k + 1]; };
        double v;
        if (i >= 1 && i <= N && j >= 1 && j <= N) {
            v = cell(t, i, j);
        } else {
            // a virtual row: side, depth m, along index a
            int s = -1, m = 0, a = 0;
            if (j < 1) { s = SIDE_B; m = 1 - j; a = i; }
            else if (j > N) { s = SIDE_T; m = j - N; a = i; }
            if (s >= 0 && !(a >= (m == 1 ? 2 : 1) && a <= (m == 1 ? N - 1 : N))) s = -1;
            if (s < 0) {
                if (i < 1) { s = SIDE_L; m = 1 - i; a = j; }
                else if (i > N) { s = SIDE_R; m = i - N; a = j; }
                if (s >= 0 && !(a >= (m == 1 ? 2 : 1) && a <= (m == 1 ? N - 1 : N))) s = -1;
            }
            if (s >= 0) {
                const int K = kt[(m - 1) * ni + a + 1];
                v = W(-1, a, m) * X(s, m, K - 1) + W(0, a, m) * X(s, m, K) + W(1, a, m) * X(s, m, K + 1) +
                    W(2, a, m) * X(s, m, K + 2);
            } else {
                // a special point of the corner (ist, jst) with directions (idir, jdir)
                const int idir = i <= 1 ? 1 : -1, jdir = j <= 1 ? 1 : -1;
                const int ist = idir > 0 ? 0 : N + 1, jst = jdir > 0 ? 0 : N + 1;
                const int li = (i - ist) * idir, lj = (j - jst) * jdir;
                auto FC = [&](int x, int y) { return pf(ist + idir * x, jst + jdir * y); };
                auto PW = [&](int k, int a2, int m2) { return idir > 0 ? W(k, a2, m2) : W(1 - k, N + 1 - a2, m2); };
                const double z0 = PW(0, 1, 1), z1 = PW(1, 1, 1), z2 = PW(2, 1, 1);
                const double zw = PW(-1, 1, 1), zw2 = zw * zw, zw3 = zw2 * zw;
                if (li == 0 && lj == 1) {
                    const double zx = z0 * FC(0, 1) + z1 * FC(0, 2) + z2 * FC(0, 3);
                    const double zy = z0 * FC(1, 0) + z1 * FC(1, -1) + z2 * FC(1, -2);
                    const double zz = z0 * FC(1, 1) + z1 * FC(2, 1) + z2 * FC(3, 1);
                    v = (zx + zw * zy + zw2 * zz) / (1 - zw3);
                } else if (li == 1 && lj == 0) {
                    const double zx = z0 * FC(1, 0) + z1 * FC(2, 0) + z2 * FC(3, 0);
                    const double zy = z0 * FC(0, 1) + z1 * FC(-1, 1) + z2 * FC(-2, 1);
                    const double zz = z0 * FC(1, 1) + z1 * FC(1, 2) + z2 * FC(1, 3);
                    v = (zx + zw * zy + zw2 * zz) / (1 - zw3);
                } else if (li == 0 && lj == 0) {
                    double zx = z0 * FC(0, 1) + z1 * FC(0, 2) + z2 * FC(0, 3);
                    double zy = z0 * FC(1, 0) + z1 * FC(1, -1) + z2 * FC(1, -2);
                    double zz = z0 * FC(1, 1) + z1 * FC(2, 1) + z2 * FC(3, 1);
                    const double zfy1 = (zy + zw * zz + zw2 * zx) / (1 - zw3);
                    zx = z0 * FC(1, 0) + z1 * FC(2, 0) + z2 * FC(3, 0);
                    zy = z0 * FC(0, 1) + z1 * FC(-1, 1) + z2 * FC(-2, 1);
                    zz = z0 * FC(1, 1) + z1 * FC(1, 2) + z2 * FC(1, 3);
                    const double zfy2 = (zy + zw * zz + zw2 * zx) / (1 - zw3);
                    const double zff1 = PW(-1, 1, 2) * FC(2, 0) + PW(0, 1, 2) * FC(2, -1) + PW(1, 1, 2) * FC(2, -2) +
                                        PW(2, 1, 2) * FC(2, -3);
                    const double zff2 = PW(-1, 1, 2) * FC(0, 2) + PW(0, 1, 2) * FC(-1, 2) + PW(1, 1, 2) * FC(-2, 2) +
                                        PW(2, 1, 2) * FC(-3, 2);
                    v = 0.5 * (PW(-1, 0, 1) * zff1 + PW(0, 0, 1) * zfy1 + PW(1, 0, 1) * FC(0, 1) + PW(2, 0, 1) * FC(0, 2) +
                               PW(-1, 0, 1) * zff2 + PW(0, 0, 1) * zfy2 + PW(1, 0, 1) * FC(1, 0) + PW(2, 0, 1) * FC(2, 0));
                } else {
                    const double zff1 = PW(-1, 2, 1) * FC(1, 0) + PW(0, 2, 1) * FC(1, -1) + PW(1, 2, 1) * FC(1, -2) +
                                        PW(2, 2, 1) * FC(1, -3);
                    const double zff2 = PW(-1, 2, 1) * FC(0, 1) + PW(0, 2, 1) * FC(-1, 1) + PW(1, 2, 1) * FC(-2, 1) +
                                        PW(2, 2, 1) * FC(-3, 1);
                    if (li == -1 && lj == 0) {
                        v = PW(-1, 0, 2) * zff1 + PW(0, 0, 2) * FC(-1, 1) + PW(1, 0, 2) * FC(-1, 2) + PW(2, 0, 2) * FC(-1, 3);
                    } else if (li == 0 && lj == -1) {
                        v = PW(-1, 0, 2) * zff2 + PW(0, 0, 2) * FC(1, -1) + PW(1, 0, 2) * FC(2, -1) + PW(2, 0, 2) * FC(3, -1);
                    } else {
                        const double zff11 = PW(-1, 2, 2) * FC(2, -1) + PW(0, 2, 2) * FC(2, -2) + PW(1, 2, 2) * FC(2, -3) +
                                             PW(2, 2, 2) * FC(2, -4);
                        const double zff22 = PW(-1, 2, 2) * FC(-1, 2) + PW(0, 2, 2) * FC(-2, 2) + PW(1, 2, 2) * FC(-3, 2) +
                                             PW(2, 2, 2) * FC(-4, 2);
                        v = 0.5 * (PW(-1, -1, 2) * zff11 + PW(0, -1, 2) * zff1 + PW(1, -1, 2) * FC(-1, 1) +
                                   PW(2, -1, 2) * FC(-1, 2) + PW(-1, -1, 2) * zff22 + PW(0, -1, 2) * zff2 +
                                   PW(1, -1, 2) * FC(1, -1) + PW(2, -1, 2) * FC(2, -1));
                    }
                }
            }
        }
        ext[q] = v;
    }
}

// Layout of the curl regrid's tables: ints idx (3 per point), kt (2 (N+4)); doubles w (8
// per point), wt (4 per kt entry), the extended panels, the output.
struct LatlonOLayout {
    size_t np, nk, next;
    size_t i_kt() const { return 3 * np; }
    size_t ints() const { return 3 * np + nk; }
    size_t d_wt() const { return 8 * np; }
    size_t d_ext() const { return d_wt() + 4 * nk; }
    size_t d_out() const { return d_ext() + next; }
    size_t doubles() const { return d_out() + np; }
};
static LatlonOLayout latlon_o_layout(int N, int nlat, int nlon)
{
    LatlonOLayout L;
    L.np = (size_t)nlat * nlon;
    L.nk = (size_t)2 * llo_pitch(N);
    L.next = (size_t)NPAN * llo_pitch(N) * llo_pitch(N);
    return L;
}

// Point location and cubic weights on the cell-centre mesh (shift 1/2:
// init_interpolation, latlon_regrid_mod.f90:286-336, on mesh_o) and the ECS_O halo
// weights, built on the host in FP64.
static int ensure_latlon_o(swe_ctx *c, int nlat, int nlon)
{
    if (c->llo_i && c->llo_nlat == nlat && c->llo_nlon == nlon) return SWE_OK;
    cudaFree(c->llo_i); cudaFree(c->llo_d);
    c->llo_i = nullptr; c->llo_d = nullptr; c->llo_nlat = c->llo_nlon = 0;
    const int N = c->cfg.N;
    const LatlonOLayout Lo = latlon_o_layout(N, nlat, nlon);
    std::vector<int> hi(Lo.ints(), 0);
    std::vector<double> hd(Lo.d_ext(), 0.0);
    const double pi = 3.141592653589793238462643383279502884;
    const double hx = 0.5 * pi / N, a0 = -0.25 * pi;
    for (int j = 1; j <= nlat; j++) {
        const double phi = -0.5 * pi + (j - 1) * pi / (nlat - 1.0);
        for (int i = 1; i <= nlon; i++) {
            const double lam = (i - 1) * 2.0 * pi / nlon;
            const double r[3] = {std::cos(phi) * std::cos(lam), std::cos(phi) * std::sin(lam), std::sin(phi)};
            int t;
            double alpha, beta;
            cart_to_native(r, t, alpha, beta);
            double zdx = (alpha - a0) / hx + 1 - 0.5, zdy = (beta - a0) / hx + 1 - 0.5;
            const int xi = (int)zdx, yi = (int)zdy;
            zdx = zdx - xi;
            zdy = zdy - yi;
            // the stencil (cells xi-1 .. xi+2) stays inside the extended panel
            if (t < 0 || t >= NPAN || xi < 0 || xi > N || yi < 0 || yi > N)
                return fail(c, SWE_EINVAL, "lat-lon point (%d, %d) outside the cube panels", i, j);
            const size_t q = (size_t)(j - 1) * nlon + (i - 1);
            hi[3 * q] = t; hi[3 * q + 1] = xi; hi[3 * q + 2] = yi;
            double *wx = &hd[8 * q], *wy = wx + 4;
            wx[0] = -zdx * (zdx - 1.0) * (zdx - 2.0) / 6.0;
            wx[1] = (zdx + 1.0) * (zdx - 1.0) * (zdx - 2.0) / 2.0;
            wx[2] = -(zdx + 1.0) * zdx * (zdx - 2.0) / 2.0;
            wx[3] = (zdx + 1.0) * zdx * (zdx - 1.0) / 6.0;
            wy[0] = -zdy * (zdy - 1.0) * (zdy - 2.0) / 6.0;
            wy[1] = (zdy + 1.0) * (zdy - 1.0) * (zdy - 2.0) / 2.0;
            wy[2] = -(zdy + 1.0) * zdy * (zdy - 2.0) / 2.0;
            wy[3] = (zdy + 1.0) * zdy * (zdy - 1.0) / 6.0;
        }
    }
    const int ni = llo_pitch(N);
    for (int m = 1; m <= 2; m++)
        for (int a = -1; a <= N + 2; a++) {
            const size_t row = (size_t)(m - 1) * ni + a + 1;
            halo_o_weights(hx, a, m, &hd[Lo.d_wt() + 4 * row], hi[Lo.i_kt() + row]);
            // the rows' stencils read the neighbour's cells 1 .. N
            const int K = hi[Lo.i_kt() + row];
            if (a >= (m == 1 ? 2 : 1) && a <= (m == 1 ? N - 1 : N) && (K - 1 < 1 || K + 2 > N))
                return fail(c, SWE_EINVAL, "ECS_O halo: line %d of row %d reads outside the neighbour", a, m);
        }
    if (cudaMalloc(&c->llo_i, hi.size() * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c->llo_d, Lo.doubles() * sizeof(double)) != cudaSuccess) {
        cudaFree(c->llo_i); c->llo_i = nullptr; c->llo_d = nullptr;
        return fail(c, SWE_ENOMEM, "lat-lon curl regrid allocation failed");
    }
    CU(c, cudaMemcpy(c->llo_i, hi.data(), hi.size() * sizeof(int), cudaMemcpyHostToDevice));
    CU(c, cudaMemcpy(c->llo_d, hd.data(), hd.size() * sizeof(double), cudaMemcpyHostToDevice));
    c->llo_nlat = nlat;
    c->llo_nlon = nlon;
    return SWE_OK;
}

// The divergence of the wind of every member (div_ch_sbp_sat_<order>_proj of the
// contravariant components, the operator the diagnostics' div_operator_name names)
// into field 0 of the scratch box ya: the linear operator's stage kernel in mode 0
// with the depth factor -1, so that its dh = -(-1) div.
template <class T>
static int enqueue_div(swe_ctx *c, const void *yin, const MetricView<T> &mv)
{
    const int M = c->cfg.n_members;
    if (!c->negones) {
        std::vector<double> neg(M, -1.0);
        if (cudaMalloc(&c->negones, sizeof(double) * M) != cudaSuccess) {
            c->negones = nullptr;
            return fail(c, SWE_ENOMEM, "divergence factor allocation failed");
        }
        CU(c, cudaMemcpy(c->negones, neg.data(), sizeof(double) * M, cudaMemcpyHostToDevice));
    }
    if (!launch_co2contra<T>(c->tile, c->occ, c->runs, c->ord, M, (const T *)yin, (T *)c->w, (T *)c->es, c->dims, mv,
                        c->stream, nullptr)) c->launch_miss = true;
    launch_k(c->ord == 21 ? k_edge<T, 21> : (c->ord == 63 ? k_edge<T, 63> : k_edge<T, 42>), edge_grid(c),
             dim3(EDGE_THREADS), 0, c->stream, (const T *)c->es, (const T *)c->es, (T *)c->edge, c->dims, mv,
             (const double *)nullptr);
    StageArgs a{0, 0.0, c->negones, nullptr, nullptr, nullptr, nullptr};
    if (!launch_stage<T>(c->tile, c->occ, c->runs, c->ord, M, (const T *)yin, (const T *)c->w, (const T *)c->edge, nullptr,
                    (T *)c->ya, nullptr, nullptr, c->dims, mv, a, c->stream)) c->launch_miss = true;
    c->launches += 3;
    CU_LAUNCHED(c);
    return SWE_OK;
}

extern "C" int swe_regrid_latlon(swe_ctx *c, const swe_stvec *vec, int member, int field, int nlat, int nlon,
                                 double *out)
{
    if (!c || !vec || vec->ctx != c || !out || member < 0 || member >= c->cfg.n_members) return SWE_EINVAL;
    CHSWE_NOT_ON_C(c, "swe_regrid_latlon");
    if (field < 0 || field > 2)
        return fail(c, SWE_EINVAL, "lat-lon regrid: field 0 (h), 1 (the divergence of the wind) or 2 (its curl)");
    if (field >= 1 && c->ah) return fail(c, SWE_EINVAL, "lat-lon regrid of the divergence or the curl: built for Ch");
    if (nlat < 2 || nlon < 1 || (int64_t)nlat * nlon > (1 << 28))
        return fail(c, SWE_EINVAL, "lat-lon regrid: bad grid %d x %d", nlat, nlon);
    if (field == 2) {
        // output_curl: the curl on the cell centres, its ECS_O halo, the cubic stencils
        int rc = ensure_otab(c);
        if (rc == SWE_OK) rc = ensure_latlon_o(c, nlat, nlon);
        if (rc != SWE_OK) return rc;
        const int N = c->cfg.N;
        const LatlonOLayout Lo = latlon_o_layout(N, nlat, nlon);
        const int64_t np = (int64_t)Lo.np;
        const size_t mo = (size_t)member * c->dims.ms;
        const double hx = 0.5 * 3.141592653589793238462643383279502884 / N;
        double *dcurl = c->otab + 7 * (size_t)c->dims.ps;
        double *ext = c->llo_d + Lo.d_ext(), *dout = c->llo_d + Lo.d_out();
        if (c->elem == 8) launch_curl<double>(c, (const double *)vec->d + mo, c->dims, hx, dcurl);
        else launch_curl<float>(c, (const float *)vec->d + mo, c->dims, hx, dcurl);
        const dim3 b(256), g1((unsigned)std::min<int64_t>(((int64_t)Lo.next + 255) / 256, 8192)),
            g2((unsigned)std::min<int64_t>((np + 255) / 256, 8192));
        k_ecs_o_ext<<<g1, b, 0, c->stream>>>(dcurl, N, c->llo_i + Lo.i_kt(), c->llo_d + Lo.d_wt(), ext);
        k_latlon<<<g2, b, 0, c->stream>>>(ext, c->llo_i, c->llo_d, llo_pitch(N), np, dout);
        c->launches += 3;
        CU_LAUNCHED(c);
        CU(c, cudaMemcpyAsync(out, dout, (size_t)np * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CU(c, cudaStreamSynchronize(c->stream));
        return SWE_OK;
    }
    int rc = ensure_latlon(c, nlat, nlon);
    if (rc != SWE_OK) return rc;
    const int N = c->cfg.N;
    const LatlonLayout Lo = latlon_layout(N, nlat, nlon);
    const int64_t np = (int64_t)Lo.np;
    const int *kt = c->ll_i + Lo.i_kt();
    const double *wt = c->ll_d + Lo.d_wt();
    double *ext = c->ll_d + Lo.d_ext(), *dout = c->ll_d + Lo.d_out();
    const size_t mo = (size_t)member * c->dims.ms;
    const dim3 b(256), g1((unsigned)std::min<int64_t>(((int64_t)Lo.next + 255) / 256, 8192)),
        g2((unsigned)std::min<int64_t>((np + 255) / 256, 8192));
    const void *src = vec->d;
    if (field == 1) {
        rc = c->elem == 8 ? enqueue_div<double>(c, vec->d, c->m64.v) : enqueue_div<float>(c, vec->d, c->m32.v);
        if (rc != SWE_OK) return rc;
        src = c->ya;
    }
    if (c->elem == 8) k_ecs_xy_ext<double><<<g1, b, 0, c->stream>>>((const double *)src + mo, c->dims, kt, wt, ext);
    else k_ecs_xy_ext<float><<<g1, b, 0, c->stream>>>((const float *)src + mo, c->dims, kt, wt, ext);
    k_latlon<<<g2, b, 0, c->stream>>>(ext, c->ll_i, c->ll_d, ll_pitch(N), np, dout);
    c->launches += 2;
    CU_LAUNCHED(c);
    CU(c, cudaMemcpyAsync(out, dout, (size_t)np * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CU(c, cudaStreamSynchronize(c->stream));
    return SWE_OK;
}

extern "C" int swe_regrid_latlon_wind(swe_ctx *c, const swe_stvec *vec, int member, int nlat, int nlon, double *u_out,
                                      double *v_out)
{
    if (!c || !vec || vec->ctx != c || !u_out || !v_out || member < 0 || member >= c->cfg.n_members)
        return SWE_EINVAL;
    CHSWE_NOT_ON_C(c, "swe_regrid_latlon_wind");
    if (c->ah) return fail(c, SWE_EINVAL, "swe_regrid_latlon_wind: built for the Ch staggering");
    if (nlat < 2 || nlon < 1 || (int64_t)nlat * nlon > (1 << 28))
        return fail(c, SWE_EINVAL, "lat-lon regrid: bad grid %d x %d", nlat, nlon);
    int rc = ensure_latlon(c, nlat, nlon);
    if (rc != SWE_OK) return rc;
    const int N = c->cfg.N;
    const LatlonLayout Lo = latlon_layout(N, nlat, nlon);
    const int64_t np = (int64_t)Lo.np;
    const int *kt = c->ll_i + Lo.i_kt();
    const double *wt = c->ll_d + Lo.d_wt(), *tm = c->ll_d + Lo.d_tm(), *qr = c->ll_d + Lo.d_q();
    double *extu = c->ll_d + Lo.d_ext(), *extv = extu + Lo.next;
    double *uo = c->ll_d + Lo.d_out(), *vo = uo + np;
    const size_t mo = (size_t)member * c->dims.ms;
    const dim3 b(256), g1((unsigned)std::min<int64_t>(((int64_t)Lo.next + 255) / 256, 8192)),
        g2((unsigned)std::min<int64_t>((np + 255) / 256, 8192));
    if (c->elem == 8)
        k_ecs_vec_ext<double><<<g1, b, 0, c->stream>>>((const double *)vec->d + mo, c->dims, kt, wt, tm, extu, extv);
    else k_ecs_vec_ext<float><<<g1, b, 0, c->stream>>>((const float *)vec->d + mo, c->dims, kt, wt, tm, extu, extv);
    k_latlon_vec<<<g2, b, 0, c->stream>>>(extu, extv, c->ll_i, c->ll_d, qr, N, np, uo, vo);
    c->launches += 2;
    CU_LAUNCHED(c);
    CU(c, cudaMemcpyAsync(u_out, uo, (size_t)np * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CU(c, cudaMemcpyAsync(v_out, vo, (size_t)np * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CU(c, cudaStreamSynchronize(c->stream));
    return SWE_OK;
}

extern "C" int swe_edge_links(int *out)
{
    if (!out) return SWE_EINVAL;
    Link L[NPAN][4];
    compute_links(L);
    for (int p = 0; p < NPAN; p++)
        for (int s = 0; s < 4; s++) {
            int *o = out + (p * 4 + s) * 5;
            o[0] = L[p][s].nb; o[1] = L[p][s].nside; o[2] = L[p][s].rev; o[3] = L[p][s].sn; o[4] = L[p][s].st;
        }
    return SWE_OK;
}

// Diagnostic: run `nreps` RK4 steps launch by launch with CUDA events around every
// kernel on the context's stream; returns the mean duration (ms) of the
// contravariant kernel, the edge kernel and the fused stage kernel.
template <class T>
static void timed_stage(swe_ctx *c, const MetricView<T> &mv, const void *yin, void *v0, void *y1, float *cmp, int mode,
                        double dt, cudaEvent_t e0, cudaEvent_t e1, cudaEvent_t e2, cudaEvent_t e3)
{
    const int M = c->cfg.n_members;
    if (c->fused) {
        // fused stage: the edge-strip kernel, the edge sync, the tiles
        const FusedMetric<T> fm{(const T *)c->fmet, mv.inv_hxa, mv.inv_hx, mv.grav};
        CUtensorMap tmY;
        if (encode_rows(&tmY, yin, sizeof(T), c->dims.P, (int64_t)M * 3 * NPAN * (c->cfg.N + 1 + 2 * MG),
                        fused_box_w(c), c->fth + 8)) {
            cudaEventRecord(e0, c->stream);
            FusedTU<T>::strip(M, (const T *)yin, (T *)c->es, c->dims, fm, nullptr, c->stream);
            cudaEventRecord(e1, c->stream);
            launch_k(k_edge<T, 42>, edge_grid(c), dim3(EDGE_THREADS), 0, c->stream, (const T *)c->es,
                     (const T *)c->es, (T *)c->edge, c->dims, mv, (const double *)nullptr);
            cudaEventRecord(e2, c->stream);
            StageArgs a{mode, dt, c->Hm, nullptr, nullptr, nullptr, nullptr};
            FusedTU<T>::stage(c->fth, c->focc, M, tmY, c->tm_metric, (const T *)yin, (const T *)c->edge, (T *)v0,
                              (T *)y1, (T *)c->acc, (T *)cmp, c->dims, fm, a, c->derr, c->stream);
            cudaEventRecord(e3, c->stream);
            c->launches += 3;
            return;
        }
    }
    cudaEventRecord(e0, c->stream);
    if (!launch_co2contra<T>(c->tile, c->occ, c->runs, c->ord, M, (const T *)yin, (T *)c->w, (T *)c->es, c->dims, mv, c->stream)) c->launch_miss = true;
    cudaEventRecord(e1, c->stream);
    launch_k(c->ord == 21 ? k_edge<T, 21> : (c->ord == 63 ? k_edge<T, 63> : k_edge<T, 42>), edge_grid(c), dim3(EDGE_THREADS), 0, c->stream, (const T *)c->es, (const T *)c->es,
             (T *)c->edge, c->dims, mv, (const double *)nullptr);
    cudaEventRecord(e2, c->stream);
    StageArgs a{mode, dt, c->Hm, nullptr, nullptr, nullptr, nullptr};
    if (!launch_stage<T>(c->tile, c->occ, c->runs, c->ord, M, (const T *)yin, (const T *)c->w, (const T *)c->edge, (T *)v0, (T *)y1, (T *)c->acc,
                    (T *)cmp,
                    c->dims, mv, a, c->stream)) c->launch_miss = true;
    cudaEventRecord(e3, c->stream);
    c->launches += 3;
}

extern "C" int swe_kernel_times(swe_ctx *c, swe_stvec *v0, double dt, int nreps, double *ms_co2contra, double *ms_edge,
                                double *ms_stage)
{
    if (!c || !v0 || v0->ctx != c || nreps < 1) return SWE_EINVAL;
    CHSWE_NOT_ON_C(c, "swe_kernel_times");
    if (c->adv || c->ah) return fail(c, SWE_EINVAL, "swe_kernel_times times the Ch linear operator's three kernels");
    int rc = ensure_cmp(v0);
    if (rc) return rc;
    const int nst = 4 * nreps;
    std::vector<cudaEvent_t> ev(4 * nst);
    for (auto &e : ev) CU(c, cudaEventCreate(&e));
    void *bufs_in[4] = {v0->d, c->yb, c->ya, c->yb};
    void *bufs_out[4] = {c->yb, c->ya, c->yb, nullptr};
    for (int r = 0; r < nreps; r++)
        for (int s = 0; s < 4; s++) {
            cudaEvent_t *e = &ev[4 * (4 * r + s)];
            if (c->elem == 8)
                timed_stage<double>(c, c->m64.v, bufs_in[s], v0->d, bufs_out[s], nullptr, s + 1, dt, e[0], e[1], e[2], e[3]);
            else
                timed_stage<float>(c, c->m32.v, bufs_in[s], v0->d, bufs_out[s], v0->cmp, s + 1, dt, e[0], e[1], e[2], e[3]);
        }
    CU_LAUNCHED(c);
    CU(c, cudaStreamSynchronize(c->stream));
    double t_co = 0.0, t_ed = 0.0, t_st = 0.0;
    for (int q = 0; q < nst; q++) {
        float a = 0.f, b = 0.f, d = 0.f;
        cudaEventElapsedTime(&a, ev[4 * q], ev[4 * q + 1]);
        cudaEventElapsedTime(&b, ev[4 * q + 1], ev[4 * q + 2]);
        cudaEventElapsedTime(&d, ev[4 * q + 2], ev[4 * q + 3]);
        t_co += a; t_ed += b; t_st += d;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    if (ms_co2contra) *ms_co2contra = t_co / nst;
    if (ms_edge) *ms_edge = t_ed / nst;
    if (ms_stage) *ms_stage = t_st / nst;
    return SWE_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free operator apply.
//
// For host programs that cannot allocate device memory themselves (a Fortran
// model whose GPU memory is owned by another runtime or a fixed pool, or code
// running where cudaMalloc is not permitted): everything the linear operator
// needs besides the caller's input and output lives in one static device array
// of this library, sized for cubes up to SWE_NOALLOC_MAX_N.
// ---------------------------------------------------------------------------
namespace {
constexpr int NA_MAXN = SWE_NOALLOC_MAX_N;
constexpr int NA_TILE = 33, NA_OCC = 2;   // stage-kernel configuration of the allocation-free apply
constexpr int NA_ROWS = NA_MAXN + 1 + 2 * MG;
constexpr int NA_P = (NA_ROWS + 7) / 8 * 8;
constexpr size_t NA_BOX = (size_t)NA_ROWS * NA_P;
constexpr size_t NA_METRIC = 14 * NA_BOX + 48 * (size_t)(NA_MAXN + 1);
constexpr size_t NA_W = 3 * (size_t)NPAN * NA_BOX;
constexpr size_t NA_EDGE = (size_t)NPAN * 4 * (NA_MAXN + 1) * 3;
constexpr size_t NA_STRIPS = (size_t)NPAN * 4 * STRIP_LINES * (NA_MAXN + 1);
constexpr size_t NA_TOTAL = NA_METRIC + NA_W + NA_EDGE + NA_STRIPS + 8;

struct Frames {
    int ex[NPAN][3], ey[NPAN][3], nn[NPAN][3];
};

struct NoallocDevice {
    bool ready = false;
    double *base = nullptr;      // device address of g_noalloc_scratch on this device
    bool metric_ok = false;
    swe_cfg cached{};            // configuration the stored metric was computed for
};
NoallocDevice g_noalloc[64];
}  // namespace

// Metric, Coriolis weights, vector-sync weights and edge tables: [0, NA_METRIC);
// contravariant scratch W: [NA_METRIC, +NA_W); edge buffer: next NA_EDGE; edge
// strips: next NA_STRIPS; the mean depth H: last slot.
static __device__ __align__(256) double g_noalloc_scratch[NA_TOTAL];

// FP64 metric of an N-cube into the scratch layout used by build_metric (same
// formulas, evaluated on the device).
__global__ void k_noalloc_metric(double *M, int N, int P, int64_t box, double a, double omega, double ax, double ay,
                                 double az, int cc, Frames fr)
{
    const int n = N + 1;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const double pi = 3.141592653589793238462643383279502884;
    const double hx = (0.25 * pi - (-0.25 * pi)) / (double)N;
    double *Q11y = M, *iJy = M + box, *Jy = M + 2 * box, *Q22x = M + 3 * box, *iJx = M + 4 * box, *Jx = M + 5 * box,
           *JQ12 = M + 6 * box, *iJa = M + 7 * box, *fJ2 = M + 8 * box, *qv = M + 14 * box;
    if (i <= n && j <= n) {
        const int64_t o = box_off(P, i, j);
        const double ta_n = tan(-0.25 * pi + (i - 1) * hx), tb_n = tan(-0.25 * pi + (j - 1) * hx);
        const double ta_c = tan(-0.25 * pi + (i - 1 + 0.5) * hx), tb_c = tan(-0.25 * pi + (j - 1 + 0.5) * hx);
        if (i <= N) {   // y mesh: centre in i, node in j
            const double sg = sqrt(1.0 + ta_c * ta_c + tb_n * tb_n), s2 = sg * sg;
            const double J = (1.0 + ta_c * ta_c) * (1.0 + tb_n * tb_n) / (sg * sg * sg);
            Q11y[o] = s2 / (1.0 + ta_c * ta_c); Jy[o] = J; iJy[o] = 1.0 / J;
        }
        if (j <= N) {   // x mesh: node in i, centre in j
            const double sg = sqrt(1.0 + ta_n * ta_n + tb_c * tb_c), s2 = sg * sg;
            const double J = (1.0 + ta_n * ta_n) * (1.0 + tb_c * tb_c) / (sg * sg * sg);
            Q22x[o] = s2 / (1.0 + tb_c * tb_c); Jx[o] = J; iJx[o] = 1.0 / J;
        }
        const double sg = sqrt(1.0 + ta_n * ta_n + tb_n * tb_n), s2 = sg * sg;
        const double J = (1.0 + ta_n * ta_n) * (1.0 + tb_n * tb_n) / (sg * sg * sg);
        JQ12[o] = J * (s2 * ta_n * tb_n / ((1 + ta_n * ta_n) * (1 + tb_n * tb_n)));
        iJa[o] = 1.0 / (J * a);
        const double rp[3] = {ta_n / sg, tb_n / sg, 1.0 / sg};
        for (int p = 0; p < NPAN; p++) {
            double f;
            if (cc) {
                f = omega;
            } else {
                double r[3];
                for (int dd = 0; dd < 3; dd++) r[dd] = fr.ex[p][dd] * rp[0] + fr.ey[p][dd] * rp[1] - fr.nn[p][dd] * rp[2];
                const double pr = (ax * r[0] + ay * r[1] + az * r[2]) / sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                f = 2 * omega * pr;
            }
            fJ2[p * box + o] = f * J * J;
        }
    }
    if (j == 1 && i <= n) {   // covariant vector-sync weights along the sides
        const double q = 0.25 * pi, al = -0.25 * pi + (i - 1) * hx;
        auto tb = [](double al_, double be_, double &ta, double &tbv) { ta = tan(al_); tbv = tan(be_); };
        double ta, tbv;
        // qb: a2(al, -q) . b1(al, q) rotated
        {
            tb(al, -q, ta, tbv);
            double s = pow(1.0 + pow(ta, 2.0) + pow(tbv, 2.0), 1.5);
            double a2[3] = {-ta * tbv * (1.0 + pow(tbv, 2.0)) / s, (1.0 + pow(ta, 2.0)) * (1.0 + pow(tbv, 2.0)) / s,
                            -tbv * (1.0 + pow(tbv, 2.0)) / s};
            tb(al, q, ta, tbv);
            double sg2 = sqrt(1.0 + ta * ta + tbv * tbv);
            double b1[3] = {(1.0 + tbv * tbv - (ta * tbv) * (ta * tbv) / (1.0 + ta * ta)) / sg2, 0.0,
                            -ta * (1.0 + tbv * tbv / (1 + ta * ta)) / sg2};
            qv[i - 1] = a2[0] * b1[0] + a2[1] * (-b1[2]) + a2[2] * b1[1];
        }
        // qt: a2(al, q) . b1(al, -q)
        {
            tb(al, q, ta, tbv);
            double s = pow(1.0 + pow(ta, 2.0) + pow(tbv, 2.0), 1.5);
            double a2[3] = {-ta * tbv * (1.0 + pow(tbv, 2.0)) / s, (1.0 + pow(ta, 2.0)) * (1.0 + pow(tbv, 2.0)) / s,
                            -tbv * (1.0 + pow(tbv, 2.0)) / s};
            tb(al, -q, ta, tbv);
            double sg2 = sqrt(1.0 + ta * ta + tbv * tbv);
            double b1[3] = {(1.0 + tbv * tbv - (ta * tbv) * (ta * tbv) / (1.0 + ta * ta)) / sg2, 0.0,
                            -ta * (1.0 + tbv * tbv / (1 + ta * ta)) / sg2};
            qv[n + i - 1] = a2[0] * b1[0] + a2[1] * b1[2] + a2[2] * (-b1[1]);
        }
        const double be = al;
        // ql: a1(-q, be) . b2(q, be)
        {
            tb(-q, be, ta, tbv);
            double s = pow(1.0 + pow(ta, 2.0) + pow(tbv, 2.0), 1.5);
            double a1[3] = {(1.0 + pow(ta, 2.0)) * (1.0 + pow(tbv, 2.0)) / s, -ta * tbv * (1.0 + pow(ta, 2.0)) / s,
                            -ta * (1.0 + pow(ta, 2.0)) / s};
            tb(q, be, ta, tbv);
            double sg2 = sqrt(1.0 + ta * ta + tbv * tbv);
            double b2[3] = {0.0, ((1 + ta * ta) - (ta * tbv) * (ta * tbv) / (1 + tbv * tbv)) / sg2,
                            -tbv * (ta * ta / (1 + tbv * tbv) + 1.0) / sg2};
            qv[2 * n + i - 1] = a1[0] * (-b2[2]) + a1[1] * b2[1] + a1[2] * b2[0];
        }
        // qr: a1(q, be) . b2(-q, be)
        {
            tb(q, be, ta, tbv);
            double s = pow(1.0 + pow(ta, 2.0) + pow(tbv, 2.0), 1.5);
            double a1[3] = {(1.0 + pow(ta, 2.0)) * (1.0 + pow(tbv, 2.0)) / s, -ta * tbv * (1.0 + pow(ta, 2.0)) / s,
                            -ta * (1.0 + pow(ta, 2.0)) / s};
            tb(-q, be, ta, tbv);
            double sg2 = sqrt(1.0 + ta * ta + tbv * tbv);
            double b2[3] = {0.0, ((1 + ta * ta) - (ta * tbv) * (ta * tbv) / (1 + tbv * tbv)) / sg2,
                            -tbv * (ta * ta / (1 + tbv * tbv) + 1.0) / sg2};
            qv[3 * n + i - 1] = a1[0] * b2[2] + a1[1] * b2[1] + a1[2] * (-b2[0]);
        }
    }
}

__global__ void k_noalloc_set(double *p, double v) { *p = v; }

static bool same_geometry(const swe_cfg &a, const swe_cfg &b)
{
    return a.N == b.N && a.radius == b.radius && a.grav == b.grav && a.omega == b.omega &&
           a.rotation_axis[0] == b.rotation_axis[0] && a.rotation_axis[1] == b.rotation_axis[1] &&
           a.rotation_axis[2] == b.rotation_axis[2] && a.coriolis_constant == b.coriolis_constant;
}

extern "C" int swe_operator_apply_noalloc(const swe_cfg *cfg, const double *vin, double *vout, void *cuda_stream)
{
    if (!cfg || !vin || !vout || vin == vout) return SWE_EINVAL;
    if (cfg->N > NA_MAXN) {
        fprintf(stderr, "swe_operator_apply_noalloc: N = %d exceeds the static scratch limit SWE_NOALLOC_MAX_N = %d\n",
                cfg->N, NA_MAXN);
        return SWE_ETOOBIG;
    }
    if (cfg->N < 8 || cfg->precision != SWE_FP64 || cfg->n_members != 1 ||
        cfg->operator_kind != SWE_OP_LINEAR || !(cfg->radius > 0.0) || (cfg->sbp_order != 0 && cfg->sbp_order != 42) ||
        cfg->staggering != SWE_STAG_CH)
        return SWE_EINVAL;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return SWE_ENODEV;
    NoallocDevice &nd = g_noalloc[dev];
    cudaStream_t st = (cudaStream_t)cuda_stream;
    if (!nd.ready) {
        // once per device, with the device current: the array's device address and the edge tables
        if (cudaGetSymbolAddress((void **)&nd.base, g_noalloc_scratch) != cudaSuccess) return SWE_ECUDA;
        if (upload_link_tables() != cudaSuccess) return SWE_ECUDA;
        if (stage_smem_optin<double>() != cudaSuccess) return SWE_ECUDA;
        if (dev < 64) g_tables_ready[dev] = true;
        nd.ready = true;
    }
    const int N = cfg->N, n = N + 1;
    Dims dm;
    dm.N = N;
    dm.P = (N + 1 + 2 * MG + 7) / 8 * 8;
    dm.ps = (int64_t)(N + 1 + 2 * MG) * dm.P;
    dm.fs = NPAN * dm.ps;
    dm.ms = 3 * dm.fs;
    double *M = nd.base, *W = nd.base + NA_METRIC, *E = W + NA_W, *ES = E + NA_EDGE, *Hp = ES + NA_STRIPS;
    const int64_t box = dm.ps;
    MetricView<double> mv;
    mv.Q11y = M; mv.iJy = M + box; mv.Jy = M + 2 * box; mv.Q22x = M + 3 * box; mv.iJx = M + 4 * box;
    mv.Jx = M + 5 * box; mv.JQ12 = M + 6 * box; mv.iJa = M + 7 * box; mv.fJ2 = M + 8 * box;
    mv.qb = M + 14 * box; mv.qt = mv.qb + n; mv.ql = mv.qt + n; mv.qr = mv.ql + n;
    double *ej = M + 14 * box + 4 * n, *ef = ej + 16 * n, *ea = ef + 24 * n;
    mv.ej = ej; mv.ef = ef; mv.ea = ea;
    const double pi = 3.141592653589793238462643383279502884;
    const double hx = (0.25 * pi - (-0.25 * pi)) / (double)N;
    mv.inv_hxa = 1.0 / (hx * cfg->radius);
    mv.inv_hx = 1.0 / hx;
    mv.grav = cfg->grav;
    if (!nd.metric_ok || !same_geometry(nd.cached, *cfg)) {
        if (cudaMemsetAsync(M, 0, NA_METRIC * sizeof(double), st) != cudaSuccess) return SWE_ECUDA;
        Frames fr;
        for (int p = 0; p < NPAN; p++)
            for (int dd = 0; dd < 3; dd++) { fr.ex[p][dd] = EX[p][dd]; fr.ey[p][dd] = EY[p][dd]; fr.nn[p][dd] = NRM[p][dd]; }
        dim3 g((n + 15) / 16, (n + 15) / 16), b(16, 16);
        k_noalloc_metric<<<g, b, 0, st>>>(M, N, dm.P, box, cfg->radius, cfg->omega, cfg->rotation_axis[0],
                                          cfg->rotation_axis[1], cfg->rotation_axis[2], cfg->coriolis_constant, fr);
        k_edge_tables<double><<<(n + 127) / 128, 128, 0, st>>>(mv, dm, ej, ef, ea, STRIP_LINES);
        if (cudaGetLastError() != cudaSuccess) return SWE_ECUDA;
        nd.cached = *cfg;
        nd.metric_ok = true;
    }
    // the contravariant scratch is read with its zero margins, and the edge strips of an
    // earlier call of another size hold that size's layout: clear what this size uses
    if (cudaMemsetAsync(W, 0, (size_t)dm.ms * sizeof(double), st) != cudaSuccess) return SWE_ECUDA;
    if (cudaMemsetAsync(ES, 0, (size_t)strip_member(N, 1) * sizeof(double), st) != cudaSuccess) return SWE_ECUDA;
    k_noalloc_set<<<1, 1, 0, st>>>(Hp, cfg->h_mean);
    static_assert(linear42_built(NA_TILE, NA_OCC, 0), "the allocation-free apply uses a built configuration");
    if (!launch_co2contra<double>(NA_TILE, NA_OCC, 0, 42, 1, vin, W, ES, dm, mv, st)) return SWE_ECUDA;
    launch_k(k_edge<double, 42>, edge_grid(N, 1), dim3(EDGE_THREADS), 0, st, (const double *)ES, (const double *)ES, E, dm,
             mv, (const double *)nullptr);
    StageArgs a{0, 0.0, Hp, nullptr, nullptr, nullptr, nullptr};
    if (!launch_stage<double>(NA_TILE, NA_OCC, 0, 42, 1, vin, W, E, nullptr, vout, nullptr, nullptr, dm, mv, a, st))
        return SWE_ECUDA;
    if (cudaGetLastError() != cudaSuccess) return SWE_ECUDA;
    return SWE_OK;
}

// ---------------------------------------------------------------------------
// tile size and its autotuner
// ---------------------------------------------------------------------------
static void drop_graph(swe_ctx *c)
{
    if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
    if (c->graphk) { cudaGraphExecDestroy(c->graphk); c->graphk = nullptr; }
}

static void set_cfg(swe_ctx *c, int tile, int occ, int runs)
{
    if (c->tile != tile || c->occ != occ || c->runs != runs) drop_graph(c);
    c->tile = tile;
    c->occ = occ;
    c->runs = runs;
}

// runs 0 / 1: the split stage kernels (tile, blocks per SM, stencil runs); runs 2: the
// fused stage with tiles of at most `tile` rows (17, 25 or 33) and FUSED_TW columns.
static int apply_cfg(swe_ctx *c, int tile, int occ, int runs)
{
    if (runs == 2) {
        const bool changed = !c->fused || c->fth != tile || c->focc != occ;
        int rc = select_fused(c, tile, occ);
        if (rc) return rc;
        if (changed) drop_graph(c);
        return SWE_OK;
    }
    if (c->fused) drop_graph(c);
    c->fused = false;
    set_cfg(c, tile, occ, runs);
    return SWE_OK;
}

extern "C" int swe_set_tile(swe_ctx *c, int tile)
{
    if (!c || !valid_tile(tile)) return SWE_EINVAL;
    return apply_cfg(c, tile, default_occ(tile), 0);
}

extern "C" int swe_get_tile(const swe_ctx *c, int *tile)
{
    if (!c || !tile) return SWE_EINVAL;
    *tile = c->fused ? c->fth : c->tile;
    return SWE_OK;
}

extern "C" int swe_set_kernel_config(swe_ctx *c, int tile, int blocks_per_sm, int runs)
{
    if (!c) return SWE_EINVAL;
    if (runs == 2) return apply_cfg(c, tile, blocks_per_sm, runs);
    if (!valid_cfg(c->ord, tile, blocks_per_sm, runs)) return SWE_EINVAL;
    return apply_cfg(c, tile, blocks_per_sm, runs);
}

extern "C" int swe_get_kernel_config(const swe_ctx *c, int *tile, int *blocks_per_sm, int *runs)
{
    if (!c || !tile || !blocks_per_sm || !runs) return SWE_EINVAL;
    if (c->fused) {
        *tile = c->fth;
        *blocks_per_sm = c->focc;
        *runs = 2;
        return SWE_OK;
    }
    *tile = c->tile;
    *blocks_per_sm = c->occ;
    *runs = c->runs;
    return SWE_OK;
}

namespace {
struct TuneKey {
    int device, N, precision, members, op, ord;
    bool operator==(const TuneKey &o) const
    {
        return device == o.device && N == o.N && precision == o.precision && members == o.members && op == o.op &&
               ord == o.ord;
    }
};
struct TuneEntry {
    TuneKey key;
    int tile, occ, runs;
    double ms[3];
    bool branches;
};
std::vector<TuneEntry> g_tuned;   // process-wide results of swe_autotune
}  // namespace

// Time RK4 steps of a zero state for every built kernel configuration (tile edge
// and blocks per SM; the advective operator's stage kernel exists for one
// configuration per tile) and keep the fastest.  The state lives in a scratch
// vector of this context; the caller's states are not touched.  ms_per_step gets
// the best time of each tile edge.  Results are cached per (device, N, precision,
// members, operator).
extern "C" int swe_autotune(swe_ctx *c, int nreps, int *best_tile, double *ms_per_step)
{
    if (!c || nreps < 1) return SWE_EINVAL;
    if (c->ah || c->cstag) {   // the Ah and C kernels have no tile configuration
        if (best_tile) *best_tile = c->tile;
        if (ms_per_step) for (int k = 0; k < 3; k++) ms_per_step[k] = 0.0;
        return SWE_OK;
    }
    const TuneKey key{c->device, c->cfg.N, c->cfg.precision, c->cfg.n_members, c->cfg.operator_kind, c->ord};
    for (const TuneEntry &e : g_tuned)
        if (e.key == key) {
            if (int rc = apply_cfg(c, e.tile, e.occ, e.runs)) return rc;
            if (c->branches != e.branches) drop_graph(c);
            c->branches = e.branches;
            if (best_tile) *best_tile = e.tile;
            if (ms_per_step) for (int k = 0; k < 3; k++) ms_per_step[k] = e.ms[k];
            return SWE_OK;
        }
    swe_stvec *v = nullptr;
    int rc = swe_stvec_create(c, &v);
    if (rc) return rc;
    const int keep_tile = c->fused ? c->fth : c->tile, keep_occ = c->fused ? c->focc : c->occ,
              keep_runs = c->fused ? 2 : c->runs;
    double ms[3] = {1e300, 1e300, 1e300};
    int best_t = keep_tile, best_o = keep_occ, best_r = keep_runs;
    double best_ms = 1e300;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    rc = SWE_OK;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) rc = fail(c, SWE_ECUDA, "autotune events");
    const double dt = 1.0;
    // steps that capture both graphs nreps steps replay (GRAPH_STEPS-step and 1-step)
    const int warm = (nreps >= GRAPH_STEPS ? GRAPH_STEPS : 0) + (nreps % GRAPH_STEPS ? 1 : 0);
    int ncfg = 0;
    const KernelCfg *cfgs = cfgs_of(c->ord, &ncfg);
    std::vector<KernelCfg> all(cfgs, cfgs + ncfg);
    if (fused_supported(c)) {
        // the fused stage's configurations of this precision
#define CHSWE_FADD(TH, OCC) all.push_back(KernelCfg{TH, OCC, 2});
        if (c->elem == 4) {
            CHSWE_FUSED_CFGS_F(CHSWE_FADD)
        } else {
            CHSWE_FUSED_CFGS_D(CHSWE_FADD)
        }
#undef CHSWE_FADD
    }
    for (size_t k = 0; k < all.size() && rc == SWE_OK; k++) {
        const KernelCfg kc = all[k];
        if (c->adv && kc.occ != default_occ(kc.tile)) continue;
        if (apply_cfg(c, kc.tile, kc.occ, kc.runs) != SWE_OK) continue;   // a fused tile the cube cannot take
        // untimed: capture and instantiate the graphs the timed steps replay
        if ((rc = swe_rk4_steps(c, v, dt, warm)) != SWE_OK) break;
        if (cudaEventRecord(e0, c->stream) != cudaSuccess) { rc = fail(c, SWE_ECUDA, "autotune record"); break; }
        if ((rc = swe_rk4_steps(c, v, dt, nreps)) != SWE_OK) break;
        float t = 0.f;
        if (cudaEventRecord(e1, c->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) {
            rc = fail(c, SWE_ECUDA, "autotune timing");
            break;
        }
        const double m = t / nreps;
        const int ti = kc.tile == 17 ? 0 : (kc.tile == 25 ? 1 : 2);
        ms[ti] = std::min(ms[ti], m);
        if (m < best_ms) { best_ms = m; best_t = kc.tile; best_o = kc.occ; best_r = kc.runs; }
    }
    // advective operator: the best configuration with the stage forked onto the side
    // stream and on one stream (forking pays for small cubes, not always for C384)
    bool best_b = c->branches;
    if (rc == SWE_OK && c->side) {
        apply_cfg(c, best_t, best_o, best_r);
        double tb[2] = {1e300, 1e300};
        for (int b = 0; b < 2 && rc == SWE_OK; b++) {
            drop_graph(c);
            c->branches = b == 1;
            if ((rc = swe_rk4_steps(c, v, dt, warm)) != SWE_OK) break;
            float t = 0.f;
            if (cudaEventRecord(e0, c->stream) != cudaSuccess || swe_rk4_steps(c, v, dt, nreps) != SWE_OK ||
                cudaEventRecord(e1, c->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) {
                rc = fail(c, SWE_ECUDA, "autotune timing");
                break;
            }
            tb[b] = t / nreps;
        }
        best_b = tb[1] <= tb[0];
        c->branches = best_b;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    swe_stvec_destroy(v);
    drop_graph(c);
    if (rc != SWE_OK) { apply_cfg(c, keep_tile, keep_occ, keep_runs); return rc; }
    if ((rc = apply_cfg(c, best_t, best_o, best_r)) != SWE_OK) return rc;
    TuneEntry te{key, best_t, best_o, best_r, {ms[0], ms[1], ms[2]}, best_b};
    g_tuned.push_back(te);
    if (best_tile) *best_tile = best_t;
    if (ms_per_step) for (int k = 0; k < 3; k++) ms_per_step[k] = ms[k];
    return SWE_OK;
}
