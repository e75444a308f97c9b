// swe_diff.cuh -- horizontal diffusion on the Ah staggering, the operator the reference
// applies after each step of the dynamics (shallow_water_mod.f90:95-100,117-118;
// operator_swm_diff_mod.f90:27-49) in its _sbp_21_narrow, _sbp_42_narrow and
// _sbp_63_narrow forms (hordiff_factory_mod.f90:33-44,61-68):
//   h:     hordiff_scalar_Ah_sbp_<ord>_narrow   tend = -(c a hx)^4 L(L(h))
//   u, v:  hordiff_vec_xyz_Ah_sbp_<ord>_narrow  the covariant wind to Cartesian components
//          with the contravariant basis, the same scalar diffusion of each component,
//          back with the same basis (as cart2cube_vec does for covariant components,
//          vec_math_mod.f90:196-219), then the covariant ECS Ah vector sync
//          (hordiff_colocated_mod.f90:42-58)
// L is laplace_Ah_sbp<ord>_narrow (laplace_Ah_sbp21_narrow_mod.f90:25-239,
// laplace_Ah_sbp42_narrow_mod.f90:27-761, laplace_Ah_sbp63_narrow_mod.f90:498-1715):
// narrow second differences with the variable
// coefficients Qi11 J, Qi22 J, the mixed terms D1(Qi12 J D1 f), boundary penalties,
// / (hx a)^2 / J, and the Ah scalar sync.
//
// The four scalar fields of a member (h and the three Cartesian wind components) are
// diffused together: scratch sets hold [member][field 0..3][panel][box], and every
// Laplacian is three launches over all of them (first differences; the Laplacian's raw
// values, kept for the sync on the panel edges and final inside; the sync).  A step is
// nine launches: k_dif_prep, two Laplacians, k_dif_vraw (the Cartesian tendencies
// projected back), k_dif_update (the vector sync and the Euler update or the tendency).
#pragma once

#include "lap63.h"
#include "swe_ah.cuh"

namespace chswe {

constexpr int DIF_FIELDS = 4;   // h, and the wind's x, y, z components

// Closure rows 1..6 of the narrow SBP 4-2 second difference with a variable coefficient
// (laplace_Ah_sbp42_narrow_mod.f90:121-262): entry m_rc (r <= c) of the symmetric boundary
// block as sum_k w b_k over the coefficients b_k = Qi J at node k; row r of the difference
// is -(1 / h_r) sum_c m_rc f_c with the node norm h_r, mirrored at the far end (:284-423).
struct Lap42Term {
    int r, c, k;
    double w;
};
static constexpr Lap42Term LAP42_M[] = {
    {1, 1, 1, 12.0 / 17.0}, {1, 1, 2, 59.0 / 192.0}, {1, 1, 3, 27010400129.0 / 345067064608.0},
    {1, 1, 4, 69462376031.0 / 2070402387648.0}, {1, 2, 1, -59.0 / 68.0}, {1, 2, 3, -6025413881.0 / 21126554976.0},
    {1, 2, 4, -537416663.0 / 7042184992.0}, {1, 3, 1, 2.0 / 17.0}, {1, 3, 2, -59.0 / 192.0},
    {1, 3, 3, 2083938599.0 / 8024815456.0}, {1, 3, 4, 213318005.0 / 16049630912.0}, {1, 4, 1, 3.0 / 68.0},
    {1, 4, 3, -1244724001.0 / 21126554976.0}, {1, 4, 4, 752806667.0 / 21126554976.0},
    {1, 5, 3, 49579087.0 / 10149031312.0}, {1, 5, 4, -49579087.0 / 10149031312.0}, {1, 6, 3, 1.0 / 784.0},
    {1, 6, 4, -1.0 / 784.0}, {2, 2, 1, 3481.0 / 3264.0}, {2, 2, 3, 9258282831623875.0 / 7669235228057664.0},
    {2, 2, 4, 236024329996203.0 / 1278205871342944.0}, {2, 3, 1, -59.0 / 408.0},
    {2, 3, 3, -29294615794607.0 / 29725717938208.0}, {2, 3, 4, -2944673881023.0 / 29725717938208.0},
    {2, 4, 1, -59.0 / 1088.0}, {2, 4, 3, 260297319232891.0 / 2556411742685888.0},
    {2, 4, 4, -60834186813841.0 / 1278205871342944.0}, {2, 5, 3, -1328188692663.0 / 37594290333616.0},
    {2, 5, 4, 1328188692663.0 / 37594290333616.0}, {2, 6, 3, -8673.0 / 2904112.0}, {2, 6, 4, 8673.0 / 2904112.0},
    {3, 3, 1, 1.0 / 51.0}, {3, 3, 2, 59.0 / 192.0}, {3, 3, 3, 378288882302546512209.0 / 270764341349677687456.0},
    {3, 3, 4, 13777050223300597.0 / 26218083221499456.0}, {3, 3, 5, 564461.0 / 13384296.0}, {3, 4, 1, 1.0 / 136.0},
    {3, 4, 3, -4836340090442187227.0 / 5525802884687299744.0}, {3, 4, 4, -17220493277981.0 / 89177153814624.0},
    {3, 4, 5, -125059.0 / 743572.0}, {3, 5, 3, 1613976761032884305.0 / 7963657098519931984.0},
    {3, 5, 4, -10532412077335.0 / 42840005263888.0}, {3, 5, 5, 564461.0 / 4461432.0},
    {3, 6, 3, 33235054191.0 / 26452850508784.0}, {3, 6, 4, -960119.0 / 1280713392.0}, {3, 6, 5, -3391.0 / 6692148.0},
    {4, 4, 1, 3.0 / 1088.0}, {4, 4, 3, 507284006600757858213.0 / 475219048083107777984.0},
    {4, 4, 4, 1950062198436997.0 / 3834617614028832.0}, {4, 4, 5, 1869103.0 / 2230716.0}, {4, 4, 6, 1.0 / 24.0},
    {4, 5, 3, -4959271814984644613.0 / 20965546238960637264.0}, {4, 5, 4, -15998714909649.0 / 37594290333616.0},
    {4, 5, 5, -375177.0 / 743572.0}, {4, 5, 6, -1.0 / 6.0}, {4, 6, 3, 752806667.0 / 539854092016.0},
    {4, 6, 4, 1063649.0 / 8712336.0}, {4, 6, 5, -368395.0 / 2230716.0}, {4, 6, 6, 1.0 / 8.0},
    {5, 5, 3, 8386761355510099813.0 / 128413970713633903242.0}, {5, 5, 4, 2224717261773437.0 / 2763180339520776.0},
    {5, 5, 5, 280535.0 / 371786.0}, {5, 5, 6, 5.0 / 6.0}, {5, 5, 7, 1.0 / 24.0},
    {5, 6, 3, -13091810925.0 / 13226425254392.0}, {5, 6, 4, -35039615.0 / 213452232.0},
    {5, 6, 5, -1118749.0 / 2230716.0}, {5, 6, 6, -1.0 / 2.0}, {5, 6, 7, -1.0 / 6.0}, {5, 7, 5, 1.0 / 8.0},
    {5, 7, 6, -1.0 / 6.0}, {5, 7, 7, 1.0 / 8.0}, {6, 6, 3, 660204843.0 / 13226425254392.0},
    {6, 6, 4, 3290636.0 / 80044587.0}, {6, 6, 5, 5580181.0 / 6692148.0}, {6, 6, 6, 3.0 / 4.0}, {6, 6, 7, 5.0 / 6.0},
    {6, 6, 8, 1.0 / 24.0}, {6, 7, 5, -1.0 / 6.0}, {6, 7, 6, -1.0 / 2.0}, {6, 7, 7, -1.0 / 2.0},
    {6, 7, 8, -1.0 / 6.0}, {6, 8, 6, 1.0 / 8.0}, {6, 8, 7, -1.0 / 6.0}, {6, 8, 8, 1.0 / 8.0}
};
// The block densely, [r-1][c-1][k-1] with both triangles.
static inline void lap42_dense(double D[6][8][8])
{
    for (int r = 0; r < 6; r++)
        for (int c = 0; c < 8; c++)
            for (int k = 0; k < 8; k++) D[r][c][k] = 0.0;
    for (const Lap42Term &q : LAP42_M) {
        D[q.r - 1][q.c - 1][q.k - 1] = q.w;
        if (q.c <= 6) D[q.c - 1][q.r - 1][q.k - 1] = q.w;
    }
}
__host__ __device__ constexpr double lap42_h(int r)
{
    return r == 1 ? 17.0 / 48 : (r == 2 ? 59.0 / 48 : (r == 3 ? 43.0 / 48 : (r == 4 ? 49.0 / 48 : 1.0)));
}

// Closure block shape of the narrow second difference of an order: rows x columns.
template <int ORD> struct NarrowBlock;
template <> struct NarrowBlock<42> { static constexpr int R = 6, C = 8; };
template <> struct NarrowBlock<63> { static constexpr int R = 9, C = 12; };

// Row k of the narrow second difference of order ORD on a line of n nodes with the
// coefficients b(1..n) (the d2f_x / d2f_y sweeps of calc_laplace_tile); M: the line's
// closure blocks (near end, then far end) for the 4-2 order.
template <class T, int ORD, class B, class F>
__device__ __forceinline__ T narrow_d2(int k, int n, const B &b, const F &f, const T *M, const T *Wi, int64_t ws)
{
    // inside the closure rows: the interior stencil with the vertex's tabulated weights
    // Wi[q * ws], q over the offsets -h .. h, summed in the reference's order
    if constexpr (ORD == 21) {
        if (k > 1 && k < n) return (__ldg(Wi + 2 * ws) * f(k + 1) + __ldg(Wi + ws) * f(k) + __ldg(Wi) * f(k - 1));
    } else if constexpr (ORD == 42) {
        if (k >= 7 && k <= n - 6)
            return (__ldg(Wi) * f(k - 2) + __ldg(Wi + ws) * f(k - 1) + __ldg(Wi + 2 * ws) * f(k) +
                    __ldg(Wi + 3 * ws) * f(k + 1) + __ldg(Wi + 4 * ws) * f(k + 2));
    } else {
        if (k >= 10 && k <= n - 9)
            return (__ldg(Wi) * f(k - 3) + __ldg(Wi + ws) * f(k - 2) + __ldg(Wi + 2 * ws) * f(k - 1) +
                    __ldg(Wi + 3 * ws) * f(k) + __ldg(Wi + 4 * ws) * f(k + 1) + __ldg(Wi + 5 * ws) * f(k + 2) +
                    __ldg(Wi + 6 * ws) * f(k + 3));
    }
    if constexpr (ORD == 21) {
        if (k == 1) {
            const T bc = b(1), bp = b(2);
            return (-(bc + bp) * f(1) + (bc + bp) * f(2));
        }
        const T bc = b(n), bm = b(n - 1);   // k == n
        return (bc + bm) * f(n - 1) + (-(bc + bm)) * f(n);
    } else if constexpr (ORD == 63) {
        constexpr int R = NarrowBlock<63>::R, C = NarrowBlock<63>::C;
        const bool lo = k <= R;
        const int r = lo ? k : n + 1 - k;
        const T *m = M + (lo ? 0 : R * C) + (r - 1) * C;
        T acc = T(0);
#pragma unroll
        for (int c = 0; c < C; c++) acc = acc + __ldg(m + c) * f(lo ? c + 1 : n - c);
        return T(1) * acc;
    } else {
        const bool lo = k <= 6;
        const int r = lo ? k : n + 1 - k;
        const T *m = M + (lo ? 0 : NarrowBlock<42>::R * NarrowBlock<42>::C) + (r - 1) * NarrowBlock<42>::C;
        T acc = T(0);
#pragma unroll
        for (int c = 0; c < 8; c++) acc = acc + __ldg(m + c) * f(lo ? c + 1 : n - c);
        return T(-1.0 / lap42_h(r)) * acc;
    }
}

// One scalar field of the scratch sets: field q of member mem.
__device__ __forceinline__ int64_t dif_base(const Dims &d, int mem, int q)
{
    return ((int64_t)mem * DIF_FIELDS + q) * NPAN * d.ps;
}

// The contravariant basis b1, b2 (Cartesian, unit sphere) of every vertex: [panel][6][box];
// for the 4-2 and 6-3 orders the closure blocks m_rc = sum_k w b_k of every boundary line,
// built on the host in FP64: [direction x, y][line 1..n][near, far end][row][column]
// (line j of the x direction has b_k = Qi11 J at (k, j) from the near end, at (n+1-k, j)
// from the far end; the y direction Qi22 J along column i).
// The interior stencil weights of every vertex (the metric is the same on every panel):
// [direction x, y][offset -h .. h][box] for each order (3, 5, 7 offsets), host-built in FP64.
template <class T>
struct DifView {
    const T *b;
    const T *m42, *m63;
    const T *w21, *w42, *w63;
    double h2;   // (hx a)^2
};
__host__ __device__ constexpr int narrow_width(int ord) { return ord == 21 ? 3 : (ord == 42 ? 5 : 7); }
__host__ __device__ __forceinline__ int64_t dif_block_index(int n, int dir, int line, int side, int rc)
{
    return ((((int64_t)dir * n + (line - 1)) * 2 + side) * rc);
}

// (h, b1 u + b2 v) of the state -> the four scalar fields of each member.
template <class T>
__global__ void __launch_bounds__(256) k_dif_prep(const T *__restrict__ Y, T *__restrict__ X, Dims d, DifView<T> v)
{
    const int n = d.N + 1;
    const int mem = blockIdx.z / NPAN, t = blockIdx.z % NPAN;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    pdl_trigger();
    pdl_wait();
    if (i > n || j > n) return;
    const int64_t o = box_off(d.P, i, j), po = mem * d.ms + t * d.ps + o;
    const T h = Y[po], u = Y[po + d.fs], w = Y[po + 2 * d.fs];
    const T *b = v.b + (int64_t)t * 6 * d.ps + o;
    X[dif_base(d, mem, 0) + t * d.ps + o] = h;
#pragma unroll
    for (int k = 0; k < 3; k++)
        X[dif_base(d, mem, 1 + k) + t * d.ps + o] = b[k * d.ps] * u + b[(3 + k) * d.ps] * w;
}

// calc_tile_d1x_d1y: d1x = D1x(f) J Qi12, d1y = D1y(f) J Qi12 (sbp_diff_<ORD> node
// differences).  Grid z: panel + NPAN * (field + 4 member).
template <class T, int ORD>
__global__ void __launch_bounds__(256) k_dif_d1(const T *__restrict__ F, T *__restrict__ D1X, T *__restrict__ D1Y, Dims d,
                                                AhView<T> a)
{
    const int n = d.N + 1;
    const int t = blockIdx.z % NPAN;
    const int64_t base = (int64_t)(blockIdx.z / NPAN) * NPAN * d.ps + t * d.ps;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    pdl_trigger();
    pdl_wait();
    if (i > n || j > n) return;
    const GV<T> f{F + base, d.P};
    const int64_t o = box_off(d.P, i, j);
    const T J = __ldg(a.J + o), Q2 = __ldg(a.Q2 + o);
    D1X[base + o] = dn2n<T, ORD>(i, n, [&](int k) { return f(k, j); }) * J * Q2;
    D1Y[base + o] = dn2n<T, ORD>(j, n, [&](int l) { return f(i, l); }) * J * Q2;
}

// calc_laplace_tile and divide_by_J_self: the panel-local Laplacian of every vertex; the
// panel-boundary vertices' values go to R (for the sync), the others to OUT.
template <class T, int ORD>
__global__ void __launch_bounds__(256) k_dif_lap(const T *__restrict__ F, const T *__restrict__ D1X,
                                                 const T *__restrict__ D1Y, T *__restrict__ R, T *__restrict__ OUT, Dims d,
                                                 AhView<T> a, DifView<T> v)
{
    const int n = d.N + 1;
    const int t = blockIdx.z % NPAN;
    const int64_t base = (int64_t)(blockIdx.z / NPAN) * NPAN * d.ps + t * d.ps;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    pdl_trigger();
    pdl_wait();
    if (i > n || j > n) return;
    const GV<T> f{F + base, d.P}, dx1{D1X + base, d.P}, dy1{D1Y + base, d.P};
    const GV<T> J{a.J, d.P}, Q1{a.Q1, d.P}, Q3{a.Q3, d.P};
    // one end's closure block
    constexpr int RC = ORD == 63 ? NarrowBlock<63>::R * NarrowBlock<63>::C : NarrowBlock<42>::R * NarrowBlock<42>::C;
    const T *mb = ORD == 63 ? v.m63 : v.m42;
    const T *wi = (ORD == 21 ? v.w21 : (ORD == 42 ? v.w42 : v.w63)) + box_off(d.P, i, j);
    const int64_t wd = (int64_t)narrow_width(ORD) * d.ps;   // the y weights follow the x weights
    T d2x = narrow_d2<T, ORD>(i, n, [&](int k) { return Q1(k, j) * J(k, j); }, [&](int k) { return f(k, j); },
                              mb + dif_block_index(n, 0, j, 0, RC), wi, d.ps);
    const T d2y = narrow_d2<T, ORD>(j, n, [&](int l) { return Q3(i, l) * J(i, l); }, [&](int l) { return f(i, l); },
                                    mb + dif_block_index(n, 1, i, 0, RC), wi + wd, d.ps);
    // the boundary penalties 1/h_1 (-+2 d1f), all on d2f_x and in the reference's order
    const T pen = ORD == 21 ? T(2) : (ORD == 42 ? T(48.0 / 17) : T(43200.0 / 13649));
    if (i == 1) d2x = d2x - T(0.5) * (pen * (T(-2) * dy1(1, j)));
    if (i == n) d2x = d2x - T(0.5) * (pen * (T(2) * dy1(n, j)));
    if (j == 1) d2x = d2x - T(0.5) * (pen * (T(-2) * dx1(i, 1)));
    if (j == n) d2x = d2x - T(0.5) * (pen * (T(2) * dx1(i, n)));
    const T dyx = dn2n<T, ORD>(j, n, [&](int l) { return dx1(i, l); });
    const T dxy = dn2n<T, ORD>(i, n, [&](int k) { return dy1(k, j); });
    T r = d2x + d2y;
    r = r + dxy + dyx;
    r = r / T(v.h2);
    r = r / J(i, j);
    const int64_t o = box_off(d.P, i, j);
    if (i == 1 || i == n || j == 1 || j == n) R[base + o] = r;
    else OUT[base + o] = r;
}

// The Ah scalar sync of the panel-boundary vertices (halo_Ah_scalar_sync_mod.f90:43-98):
// the mean of the copies, in the reference's order.  Thread e of 4N takes boundary vertex
// e of its panel (bottom i = 1..N, right j = 1..N, top i = 2..N+1, left j = 2..N+1).
template <class T>
__global__ void __launch_bounds__(256) k_dif_sync(const T *__restrict__ R, T *__restrict__ OUT, Dims d)
{
    const int N = d.N, n = N + 1;
    const int t = blockIdx.z % NPAN;
    const int64_t fb = (int64_t)(blockIdx.z / NPAN) * NPAN * d.ps;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    pdl_trigger();
    pdl_wait();
    if (e >= 4 * N) return;
    const int s = e / N, a = e % N;
    int i, j;
    switch (s) {
    case 0: i = 1 + a; j = 1; break;
    case 1: i = n; j = 1 + a; break;
    case 2: i = 2 + a; j = n; break;
    default: i = 1; j = 2 + a; break;
    }
    auto val = [&](int p, int k, int l) { return R[fb + p * d.ps + box_off(d.P, k, l)]; };
    auto copy = [&](int side) {
        const Link L = c_link[t][side];
        int kk, ll;
        side_vertex(N, L.nside, nb_along(L, n, along(side, i, j)), 0, kk, ll);
        return val(L.nb, kk, ll);
    };
    const T own = val(t, i, j);
    const bool il = i == 1, ir = i == n, jb = j == 1, jt = j == n;
    T r;
    if ((il || ir) && (jb || jt)) r = (own + copy(il ? SIDE_L : SIDE_R) + copy(jb ? SIDE_B : SIDE_T)) / T(3);
    else if (il) r = T(0.5) * (copy(SIDE_L) + own);
    else if (ir) r = T(0.5) * (own + copy(SIDE_R));
    else if (jb) r = T(0.5) * (own + copy(SIDE_B));
    else r = T(0.5) * (own + copy(SIDE_T));
    OUT[fb + t * d.ps + box_off(d.P, i, j)] = r;
}

// The wind's Cartesian tendencies c_uv L(L(.)) projected on b1, b2 (before the vector sync).
template <class T>
__global__ void __launch_bounds__(256) k_dif_vraw(const T *__restrict__ B, T *__restrict__ UR, T *__restrict__ VR, Dims d,
                                                  DifView<T> v, T kuv)
{
    const int n = d.N + 1;
    const int mem = blockIdx.z / NPAN, t = blockIdx.z % NPAN;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    pdl_trigger();
    pdl_wait();
    if (i > n || j > n) return;
    const int64_t o = box_off(d.P, i, j), to = t * d.ps + o;
    const T tx = kuv * B[dif_base(d, mem, 1) + to], ty = kuv * B[dif_base(d, mem, 2) + to],
            tz = kuv * B[dif_base(d, mem, 3) + to];
    const T *b = v.b + (int64_t)t * 6 * d.ps + o;
    const int64_t mo = (int64_t)mem * NPAN * d.ps + to;
    UR[mo] = tx * b[0] + ty * b[d.ps] + tz * b[2 * d.ps];
    VR[mo] = tx * b[3 * d.ps] + ty * b[4 * d.ps] + tz * b[5 * d.ps];
}

// The covariant ECS Ah vector sync of (u, v) tendencies (syncronize_grad_on_edges with
// (U, V) = (v, u), ecs_Ah_vec_sync_mod.f90:34-125), h's tendency c_h L(L(h)), then
// APPLY: the tendency into OUT; otherwise the Euler update Y += dt tend (explicit_Eul1),
// dt per member from dtm when given.
template <class T, bool APPLY>
__global__ void __launch_bounds__(256) k_dif_update(T *Y, T *__restrict__ OUT, const T *__restrict__ B,
                                                    const T *__restrict__ UR, const T *__restrict__ VR, Dims d,
                                                    MetricView<T> m, T kh, T dt, const double *__restrict__ dtm)
{
    const int N = d.N, n = N + 1;
    const int mem = blockIdx.z / NPAN, t = blockIdx.z % NPAN;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    pdl_trigger();
    pdl_wait();
    if (i > n || j > n) return;
    const int64_t o = box_off(d.P, i, j), mb = (int64_t)mem * NPAN * d.ps;
    const T th = kh * B[dif_base(d, mem, 0) + t * d.ps + o];
    T gx = UR[mb + t * d.ps + o], gy = VR[mb + t * d.ps + o];
    const bool il = i == 1, ir = i == n, jb = j == 1, jt = j == n;
    const bool cx = il || ir, cy = jb || jt;
    if (cx || cy) {
        auto nb = [&](int s, int a, T &un, T &vn) {
            const Link L = c_link[t][s];
            int kk, ll;
            side_vertex(N, L.nside, nb_along(L, n, a), 0, kk, ll);
            const int64_t q = mb + L.nb * d.ps + box_off(d.P, kk, ll);
            halo_vec(t, s, UR[q], VR[q], un, vn);
        };
        T uhx = 0, vhx = 0, uhy = 0, vhy = 0, qx = 0, qy = 0;
        if (cx) {
            nb(il ? SIDE_L : SIDE_R, j, uhx, vhx);
            qx = (il ? m.ql : m.qr)[j - 1];
        }
        if (cy) {
            nb(jb ? SIDE_B : SIDE_T, i, uhy, vhy);
            qy = (jb ? m.qb : m.qt)[i - 1];
        }
        if (cx && cy) {
            const T sx = (gx + uhx + uhy + qx * vhx) / T(3);
            gy = (gy + vhx + vhy + qy * uhy) / T(3);
            gx = sx;
        } else if (cx) {
            gx = T(0.5) * (gx + uhx + qx * vhx);
            gy = T(0.5) * (gy + vhx);
        } else {
            gx = T(0.5) * (gx + uhy);
            gy = T(0.5) * (gy + vhy + qy * uhy);
        }
    }
    const int64_t po = mem * d.ms + t * d.ps + o;
    if constexpr (APPLY) {
        OUT[po] = th;
        OUT[po + d.fs] = gx;
        OUT[po + 2 * d.fs] = gy;
    } else {
        if (dtm) dt = T(dtm[mem]);
        Y[po] = Y[po] + dt * th;
        Y[po + d.fs] = Y[po + d.fs] + dt * gx;
        Y[po + 2 * d.fs] = Y[po + 2 * d.fs] + dt * gy;
    }
}

}  // namespace chswe
