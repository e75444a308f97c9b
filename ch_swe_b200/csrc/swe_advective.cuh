// swe_advective.cuh -- device kernels of the advective (nonlinear) shallow-water
// operator, covariant Ch branch (operator_adv_swm_mod.f90:62-96):
//   dh = -div(F),  F = up4 mass flux of h with (ut, vt)      (massflux_ch_mod.f90:61-121)
//   du = A_u - g grad_x h + Cor_u,  dv = A_v - g grad_y h + Cor_v
//   A  = -(v . grad) u (up4) + Christoffel terms, synchronised on the duplicated
//        panel-edge points                                     (vector_advection_Ch_mod.f90:33-115)
// Per RK stage, after k_co2contra (ut, vt and their edge strips):
//   k_havg   average h over the duplicated panel-edge vertices (in place, as the
//            reference's ECS_xy halo does to the operator's input)
//   k_flux   the up4 mass flux on u and v points, with the virtual h points beyond
//            the panel edges interpolated along the neighbour's grid lines; also the
//            flux edge strips for the divergence sync
//   k_edge   (swe_kernels.cuh) Coriolis from the ut/vt strips, divergence from the flux strips
//   k_vhalo  covariant u, v at the virtual points beyond the panel edges (bicubic
//            from the neighbour face, projected on this face's basis)
//   k_advt   up4 advection and Christoffel terms of u and v, with ut, vt interpolated
//            to the xy points and back inside its shared-memory tiles
//   k_stage  (swe_tiled.cuh) divergence of the flux, gradient, Coriolis, A and the RK update
#pragma once

#include "swe_kernels.cuh"

namespace chswe {

// Cube edges (panel, side) with (panel*4 + side) below its neighbour's, filled by the host.
static __constant__ int c_cube_edge[12][2];

// Static tables of the advective operator (host-computed in FP64, stored in T).
template <class T>
struct AdvView {
    const T *xyw;      // ECS_xy line weights [depth 0..1][a 0..N][4]
    const int *xyind;  // ECS_xy stencil base   [depth 0..1][a 0..N]
    const int *hsrc;   // vector halo: per panel, per point: source panel
    const int *hidx;   //   4 ints per point: ixu, iyu, ixv, iyv
    const T *hw;       //   18 per point: wxu[4], wyu[4], wxv[4], wyv[4], a.b1, a.b2
    const T *S;        // Christoffel S on the y mesh (3 boxes: S11, S12, S22 of u) then x mesh (3 boxes, v)
    T inv_neg_radius;  // -1/a, the scale of the covariant Christoffel terms
    int hp;            // vector halo points per panel: 24 N + 12
};

// vector halo sections (per panel, depths 1..3)
__host__ __device__ __forceinline__ int vh_u_s(int N) { return 0; }
__host__ __device__ __forceinline__ int vh_u_n(int N) { return 3 * N; }
__host__ __device__ __forceinline__ int vh_u_w(int N) { return 6 * N; }
__host__ __device__ __forceinline__ int vh_u_e(int N) { return 6 * N + 3 * (N + 1); }
__host__ __device__ __forceinline__ int vh_v_w(int N) { return 6 * N + 6 * (N + 1); }
__host__ __device__ __forceinline__ int vh_v_e(int N) { return 9 * N + 6 * (N + 1); }
__host__ __device__ __forceinline__ int vh_v_s(int N) { return 12 * N + 6 * (N + 1); }
__host__ __device__ __forceinline__ int vh_v_n(int N) { return 12 * N + 9 * (N + 1); }
__host__ __device__ __forceinline__ int vh_points(int N) { return 24 * N + 12; }

// The neighbour's copy (panel nb, vertex (kk, ll)) of panel-boundary xy vertex (k, l) of panel t across side s.
__device__ __forceinline__ void nb_copy(int N, int t, int s, int k, int l, int &nb, int &kk, int &ll)
{
    const Link L = c_link[t][s];
    nb = L.nb;
    side_vertex(N, L.nside, nb_along(L, N + 1, along(s, k, l)), 0, kk, ll);
}

// Panel-boundary values of h before the averaging: [member][panel][side][a = 1..N+1],
// the layout of the edge buffer with one value per vertex.
__device__ __forceinline__ int64_t hb_index(int N, int mem, int t, int s, int a)
{
    return (((int64_t)mem * NPAN + t) * 4 + s) * (N + 1) + (a - 1);
}

// ---------------------------------------------------------------------------
// k_havg: the averaging of duplicated vertices that the ECS_xy halo procedure
// performs on its field (ecs_halo_xy_mod.f90:109-175): corners become the mean of
// their three copies (in each panel's own order), other edge vertices the mean of
// their two copies.  The values before the averaging go to HB: the reference's
// gradient reads its copy h_total taken before (operator_adv_swm_mod.f90:77).
// Grid (1 + edge blocks, members): block 0 of a member takes the 24 corners (all
// corner reads precede its corner writes), the others one vertex pair each per
// thread (edge pairs never touch a corner).
// ---------------------------------------------------------------------------
constexpr int HAVG_THREADS = 256;

template <class T>
__global__ void __launch_bounds__(HAVG_THREADS) k_havg(T *__restrict__ Y, T *__restrict__ HB, Dims d,
                                                       const double *__restrict__ dtm)
{
    const int mem = blockIdx.y;
    if (member_frozen(dtm, mem)) return;
    pdl_trigger();
    pdl_wait();
    const int N = d.N, n = N + 1;
    T *h = Y + mem * d.ms;   // field 0
    auto at = [&](int t, int i, int j) -> T & { return h[t * d.ps + (j - 1 + MG) * d.P + (i - 1 + MG)]; };
    __shared__ T cval[NPAN * 4];
    const int q = threadIdx.x;
    if (blockIdx.x > 0) {
        const int e = (blockIdx.x - 1) * HAVG_THREADS + q;
        if (e >= 12 * (N - 1)) return;
        const int ce = e / (N - 1), a = 2 + e % (N - 1);
        const int t = c_cube_edge[ce][0], s = c_cube_edge[ce][1];
        int k, l, nb, kk, ll;
        side_vertex(N, s, a, 0, k, l);
        nb_copy(N, t, s, k, l, nb, kk, ll);
        const T x = at(t, k, l), y = at(nb, kk, ll);
        const T avg = T(0.5) * (x + y);
        HB[hb_index(N, mem, t, s, a)] = x;
        HB[hb_index(N, mem, nb, c_link[t][s].nside, nb_along(c_link[t][s], n, a))] = y;
        at(t, k, l) = avg;
        at(nb, kk, ll) = avg;
        return;
    }
    if (q < NPAN * 4) {
        const int t = q >> 2, c = q & 3;
        const int k0 = (c == 0 || c == 3) ? 1 : n, l0 = (c < 2) ? 1 : n;
        // reference order: (1,1): own, bottom, left; (n,1): own, bottom, right;
        //                  (n,n): own, top, right;    (1,n): own, left, top
        const int s1 = (c < 2) ? SIDE_B : (c == 2 ? SIDE_T : SIDE_L);
        const int s2 = (c == 0) ? SIDE_L : (c == 3 ? SIDE_T : SIDE_R);
        int p1, k1, l1, p2, k2, l2;
        nb_copy(N, t, s1, k0, l0, p1, k1, l1);
        nb_copy(N, t, s2, k0, l0, p2, k2, l2);
        const T own = at(t, k0, l0);
        cval[q] = (own + at(p1, k1, l1) + at(p2, k2, l2)) / T(3);
        // the corner is vertex 1 or n of side s1 (B/T) and of side s2 (L/R) of panel t
        const int sa = (c < 2) ? SIDE_B : SIDE_T, sb = (c == 0 || c == 3) ? SIDE_L : SIDE_R;
        HB[hb_index(N, mem, t, sa, k0)] = own;
        HB[hb_index(N, mem, t, sb, l0)] = own;
    }
    __syncthreads();
    if (q < NPAN * 4) {
        const int t = q >> 2, c = q & 3;
        at(t, (c == 0 || c == 3) ? 1 : n, (c < 2) ? 1 : n) = cval[q];
    }
}

// ---------------------------------------------------------------------------
// k_flux: up4 mass flux (massflux_ch_mod.f90:80-121)
// ---------------------------------------------------------------------------
// h at xy index (i, j) of panel t, where at most one index lies up to two points
// beyond the panel: the virtual point is interpolated along the neighbour's grid
// line at that depth (ecs_halo_xy_mod.f90:177-235); the line's end points are the
// averaged edge vertices k_havg left in the field.
template <class T>
__device__ __forceinline__ T h_ext(const T *h, const Dims &d, const AdvView<T> &av, int t, int i, int j)
{
    const int N = d.N, n = N + 1;
    int s, dep, a;
    if (i < 1) { s = SIDE_L; dep = 1 - i; a = j; }
    else if (i > n) { s = SIDE_R; dep = i - n; a = j; }
    else if (j < 1) { s = SIDE_B; dep = 1 - j; a = i; }
    else if (j > n) { s = SIDE_T; dep = j - n; a = i; }
    else return __ldg(h + t * d.ps + (j - 1 + MG) * d.P + (i - 1 + MG));
    const Link L = c_link[t][s];
    const int base = (dep - 1) * n + (a - 1);
    const int ind = __ldg(av.xyind + base);
    const T *w = av.xyw + 4 * base;
    const T *hn = h + L.nb * d.ps;
    T r = T(0);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        int kk, ll;
        side_vertex(N, L.nside, nb_along(L, n, ind - 1 + k), dep, kk, ll);
        const T v = __ldg(hn + (ll - 1 + MG) * d.P + (kk - 1 + MG));
        r = k == 0 ? __ldg(w) * v : r + __ldg(w + k) * v;
    }
    return r;
}

// up4 flux of f across a u (x) or v (y) point with velocity c: f(m2..p3) at offsets -2..3
template <class T>
__device__ __forceinline__ T up4_flux(T c, T fm2, T fm1, T f0, T fp1, T fp2, T fp3)
{
    const T zl = T(0.5) + copysign(T(0.5), c), zr = T(1) - zl;
    return c * (zl * (T(5) * fp1 + T(15) * f0 - T(5) * fm1 + fm2) + zr * (T(5) * f0 + T(15) * fp1 - T(5) * fp2 + fp3)) /
           T(16);
}

// Writes F (field 1: flux on the y mesh, field 2: on the x mesh) and the flux edge
// strips (the same layout k_co2contra writes for ut, vt: nl lines per side, the
// normal flux at depths 1..nl-1 and the tangential one on the edge line).
template <class T>
__global__ void __launch_bounds__(256) k_flux(const T *__restrict__ Y, const T *__restrict__ W, T *__restrict__ F,
                                              T *__restrict__ FS, Dims d, AdvView<T> av, const double *__restrict__ dtm,
                                              int nl)
{
    const int N = d.N, n = N + 1;
    const int mem = blockIdx.z / NPAN, t = blockIdx.z % NPAN;
    if (member_frozen(dtm, mem)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    pdl_trigger();
    pdl_wait();
    if (i > n || j > n) return;
    const T *h = Y + mem * d.ms;
    const int64_t o = box_off(d.P, i, j);
    const int64_t po = mem * d.ms + t * d.ps;
    T *fs = FS + strip_member(N, mem, nl) + (int64_t)t * 4 * nl * n - 1;
    const T *hr = h + t * d.ps + (j - 1 + MG) * d.P + (i - 1 + MG);   // h(i, j); the box has 4-point margins
    if (i <= N) {
        const T c = __ldg(W + po + d.fs + o);
        // the six points i-2 .. i+3 lie in the panel for 3 <= i <= N-2
        const T fx = (i >= 3 && i <= N - 2)
                         ? up4_flux(c, __ldg(hr - 2), __ldg(hr - 1), __ldg(hr), __ldg(hr + 1), __ldg(hr + 2), __ldg(hr + 3))
                         : up4_flux(c, h_ext(h, d, av, t, i - 2, j), h_ext(h, d, av, t, i - 1, j), h_ext(h, d, av, t, i, j),
                                    h_ext(h, d, av, t, i + 1, j), h_ext(h, d, av, t, i + 2, j), h_ext(h, d, av, t, i + 3, j));
        F[po + d.fs + o] = fx;
        if (i <= nl - 1) fs[(SIDE_L * nl + i - 1) * n + j] = fx;
        if (i >= N + 2 - nl) fs[(SIDE_R * nl + N - i) * n + j] = fx;
        if (j == 1) fs[(SIDE_B * nl + nl - 1) * n + i] = fx;
        if (j == n) fs[(SIDE_T * nl + nl - 1) * n + i] = fx;
    }
    if (j <= N) {
        const T c = __ldg(W + po + 2 * d.fs + o);
        const int P = d.P;
        const T fy = (j >= 3 && j <= N - 2)
                         ? up4_flux(c, __ldg(hr - 2 * P), __ldg(hr - P), __ldg(hr), __ldg(hr + P), __ldg(hr + 2 * P),
                                    __ldg(hr + 3 * P))
                         : up4_flux(c, h_ext(h, d, av, t, i, j - 2), h_ext(h, d, av, t, i, j - 1), h_ext(h, d, av, t, i, j),
                                    h_ext(h, d, av, t, i, j + 1), h_ext(h, d, av, t, i, j + 2), h_ext(h, d, av, t, i, j + 3));
        F[po + 2 * d.fs + o] = fy;
        if (j <= nl - 1) fs[(SIDE_B * nl + j - 1) * n + i] = fy;
        if (j >= N + 2 - nl) fs[(SIDE_T * nl + N - j) * n + i] = fy;
        if (i == 1) fs[(SIDE_L * nl + nl - 1) * n + j] = fy;
        if (i == n) fs[(SIDE_R * nl + nl - 1) * n + j] = fy;
    }
}

// ---------------------------------------------------------------------------
// k_vhalo: covariant wind at the virtual points beyond the panel edges
// (ecs_halo_vec_Ch_mod.f90:29-60): bicubic interpolation of the source face's u (y
// mesh) and v (x mesh), projected on this face's basis vector.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) k_vhalo(const T *__restrict__ Y, T *__restrict__ VH, Dims d, AdvView<T> av,
                                               int n_members, const double *__restrict__ dtm)
{
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int per = NPAN * av.hp;
    pdl_trigger();
    pdl_wait();
    if (g >= (int64_t)per * n_members) return;
    const int mem = (int)(g / per), k = (int)(g % per);
    if (member_frozen(dtm, mem)) return;
    const int p = __ldg(av.hsrc + k);
    const int *ix = av.hidx + 4 * k;
    const T *w = av.hw + 18 * k;
    const T *y = Y + mem * d.ms + p * d.ps;
    const GV<T> U{y + d.fs, d.P}, V{y + 2 * d.fs, d.P};
    auto bicubic = [&](const GV<T> &f, int bx, int by, const T *wx, const T *wy) {
        T r = T(0);
#pragma unroll
        for (int j1 = 0; j1 < 4; j1++) {
            T s = T(0);
#pragma unroll
            for (int i1 = 0; i1 < 4; i1++) s = s + __ldg(wx + i1) * f(bx - 1 + i1, by - 1 + j1);
            r = r + __ldg(wy + j1) * s;
        }
        return r;
    };
    const T vu = bicubic(U, __ldg(ix), __ldg(ix + 1), w, w + 4);
    const T vv = bicubic(V, __ldg(ix + 2), __ldg(ix + 3), w + 8, w + 12);
    VH[(int64_t)mem * per + k] = __ldg(w + 16) * vu + __ldg(w + 17) * vv;
}

// u (y mesh) / v (x mesh) of panel t at an index at most three points beyond the panel
template <class T>
__device__ __forceinline__ T u_ext(const T *y, const T *vh, const Dims &d, int hp, int t, int i, int j)
{
    const int N = d.N;
    const T *v = vh + t * hp;
    if (j < 1) return v[vh_u_s(N) + (-j) * N + (i - 1)];
    if (j > N + 1) return v[vh_u_n(N) + (j - N - 2) * N + (i - 1)];
    if (i < 1) return v[vh_u_w(N) + (-i) * (N + 1) + (j - 1)];
    if (i > N) return v[vh_u_e(N) + (i - N - 1) * (N + 1) + (j - 1)];
    return __ldg(y + t * d.ps + d.fs + (j - 1 + MG) * d.P + (i - 1 + MG));
}
template <class T>
__device__ __forceinline__ T v_ext(const T *y, const T *vh, const Dims &d, int hp, int t, int i, int j)
{
    const int N = d.N;
    const T *v = vh + t * hp;
    if (i < 1) return v[vh_v_w(N) + (-i) * N + (j - 1)];
    if (i > N + 1) return v[vh_v_e(N) + (i - N - 2) * N + (j - 1)];
    if (j < 1) return v[vh_v_s(N) + (-j) * (N + 1) + (i - 1)];
    if (j > N) return v[vh_v_n(N) + (j - N - 1) * (N + 1) + (i - 1)];
    return __ldg(y + t * d.ps + 2 * d.fs + (j - 1 + MG) * d.P + (i - 1 + MG));
}

// up4 derivative along one direction (v_nabla_mod.f90:127-141), values at offsets -3..3;
// the reference's division by 12 is a product with 1/12 here (within rounding)
template <class T>
__device__ __forceinline__ T up4_diff(T c, const T f[7])
{
    const T zl = T(0.5) + copysign(T(0.5), c), zr = T(1) - zl;
    return (zl * (T(3) * f[4] + T(10) * f[3] - T(18) * f[2] + T(6) * f[1] - f[0]) -
            zr * (T(3) * f[2] + T(10) * f[3] - T(18) * f[4] + T(6) * f[5] - f[6])) *
           T(1.0 / 12.0);
}

// ---------------------------------------------------------------------------
// k_advt: A_u, A_v = up4 advection + Christoffel terms (before the edge sync), tiled.
// A block takes ADV_TX x TY xy points of one
// panel and stages in shared memory
//   us, vs  the covariant u (y mesh) and v (x mesh) over the tile and the 3-point reach
//           of the up4 stencils, the points beyond the panel from the vector halo;
//   vhs     vh = I_c2i,y(vt) on the xy points of the tile's rows and of the columns the
//           i2c rows of its u points read;
//   uhs     uh = I_c2i,x(ut) likewise for the v points
// (interp2d_uv2pvec_Ch_sbp42), then evaluates each point from shared memory: v at u
// points = I_i2c,x(vh), u at v points = I_i2c,y(uh) (interp2d_pvec2uv_Ch_sbp42).  Tiles
// whose windows and interpolation stencils lie inside the panel fill them with direct
// loads and the interior interpolation rows; the others through the vector halo and the
// closure rows.  The interpolations take the operands of the point-wise formulas in the
// same order.
// ---------------------------------------------------------------------------
constexpr int ADV_TX = 32, ADV_THREADS = 256, ADV_WW = ADV_TX + 6;

template <class T, int TY>
__global__ void __launch_bounds__(ADV_THREADS) k_advt(const T *__restrict__ Y, const T *__restrict__ W,
                                                      const T *__restrict__ VH, T *__restrict__ A, Dims d,
                                                      AdvView<T> av, MetricView<T> m, const double *__restrict__ dtm)
{
    constexpr int WH = TY + 6, WW = ADV_WW, TX = ADV_TX;
    __shared__ T us[WH * WW], vs[WH * WW];   // cell (c, r) = index (i0 - 2 + c, j0 - 2 + r)
    __shared__ T vhs[TY * WW];               // rows j0+1 .. j0+TY, columns i0-2 .. i0+TX+3
    __shared__ T uhs[WH * TX];               // rows j0-2 .. j0+TY+3, columns i0+1 .. i0+TX
    const int N = d.N, n = N + 1;
    const int mem = blockIdx.z / NPAN, t = blockIdx.z % NPAN;
    if (member_frozen(dtm, mem)) return;
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
    const int tx = threadIdx.x, tid = threadIdx.y * 32 + threadIdx.x;
    pdl_trigger();
    pdl_wait();
    const T *y = Y + mem * d.ms;
    const T *vh = VH + (int64_t)mem * NPAN * av.hp;
    const int64_t po = mem * d.ms + t * d.ps;
    const int P = d.P;
    const GV<T> UT{W + po + d.fs, P}, VT{W + po + 2 * d.fs, P};
    // the tile's u points: i in (i0, iu], j in (j0, ju]; v points: i in (i0, iv], j in (j0, jv]
    const int iu = min(i0 + TX, N), ju = min(j0 + TY, n);
    const int iv = min(i0 + TX, n), jv = min(j0 + TY, N);
    if (i0 >= 4 && j0 >= 4 && i0 + TX + 4 <= N && j0 + TY + 4 <= N) {
        // windows, interpolation stencils and i2c rows all inside the panel
        const T *ub = y + t * d.ps + d.fs + (int64_t)(j0 - 3 + MG) * P + (i0 - 3 + MG);   // u(i0-2, j0-2)
        const T *vb = ub + d.fs;
#pragma unroll
        for (int q = 0; q < (WH + 7) / 8; q++) {
            const int r = threadIdx.y + 8 * q;
            if (r < WH) {
                const int64_t ro = (int64_t)r * P;
                us[r * WW + tx] = __ldg(ub + ro + tx);
                vs[r * WW + tx] = __ldg(vb + ro + tx);
                if (tx < WW - 32) {
                    us[r * WW + tx + 32] = __ldg(ub + ro + tx + 32);
                    vs[r * WW + tx + 32] = __ldg(vb + ro + tx + 32);
                }
            }
        }
        const T *vt0 = VT.p + (int64_t)(j0 + MG) * P + (i0 - 3 + MG);   // vt(i0-2, j0+1)
#pragma unroll 2
        for (int e = tid; e < TY * WW; e += ADV_THREADS) {
            const int r = e / WW, c = e % WW;
            const T *q = vt0 + (int64_t)r * P + c;   // vt(i0-2+c, j0+1+r)
            vhs[e] = (T(9) * (__ldg(q) + __ldg(q - P)) - (__ldg(q + P) + __ldg(q - 2 * P))) * T(0.0625);
        }
        const T *ut0 = UT.p + (int64_t)(j0 - 3 + MG) * P + (i0 + MG);   // ut(i0+1, j0-2)
#pragma unroll 2
        for (int e = tid; e < WH * TX; e += ADV_THREADS) {
            const int r = e / TX, c = e % TX;
            const T *q = ut0 + (int64_t)r * P + c;   // ut(i0+1+c, j0-2+r)
            uhs[e] = (T(9) * (__ldg(q) + __ldg(q - 1)) - (__ldg(q + 1) + __ldg(q - 2))) * T(0.0625);
        }
    } else {
#pragma unroll 1
        for (int e = tid; e < WH * WW; e += ADV_THREADS) {
            const int r = e / WW, c = e % WW;
            const int ii = i0 - 2 + c, jj = j0 - 2 + r;
            // u: the x reach of the rows (j0, ju], the y reach of the columns (i0, iu]
            if ((jj > j0 && jj <= ju && ii <= iu + 3) || (ii > i0 && ii <= iu && jj <= ju + 3))
                us[e] = u_ext(y, vh, d, av.hp, t, ii, jj);
            if ((jj > j0 && jj <= jv && ii <= iv + 3) || (ii > i0 && ii <= iv && jj <= jv + 3))
                vs[e] = v_ext(y, vh, d, av.hp, t, ii, jj);
        }
        // vh on the xy points (c, j): j in (j0, ju], c in [lo, hi] (the i2c rows of the
        // centres (i0, iu] read these: interior i-1 .. i+2, closures 1..5 and N-3 .. N+1)
        if (i0 < N) {
            const int lo = max(1, min(i0, N - 3)), hi = min(n, i0 + TX + 3);
#pragma unroll 1
            for (int e = tid; e < TY * WW; e += ADV_THREADS) {
                const int r = e / WW, c = e % WW;
                const int ii = i0 - 2 + c, jj = j0 + 1 + r;
                if (ii >= lo && ii <= hi && jj <= ju) vhs[e] = ic2i<T>(jj, n, [&](int q) { return VT(ii, q); });
            }
        }
        if (j0 < N) {
            const int lo = max(1, min(j0, N - 3)), hi = min(n, j0 + TY + 3);
#pragma unroll 1
            for (int e = tid; e < WH * TX; e += ADV_THREADS) {
                const int r = e / TX, c = e % TX;
                const int ii = i0 + 1 + c, jj = j0 - 2 + r;
                if (jj >= lo && jj <= hi && ii <= iv) uhs[e] = ic2i<T>(ii, n, [&](int q) { return UT(q, jj); });
            }
        }
    }
    __syncthreads();
    const int i = i0 + 1 + tx;
    const int64_t box = d.ps;
#pragma unroll 1
    for (int r = threadIdx.y; r < TY; r += ADV_THREADS / TX) {
        const int j = j0 + 1 + r;
        const int64_t o = box_off(P, i, j);
        if (i <= iu && j <= ju) {
            // u point: ut and v_at_u = I_i2c,x(vh)
            const T a = __ldg(W + po + d.fs + o);
            const T *vr = vhs + r * WW - (i0 - 2);
            const T b = ii2c<T>(i, N, [&](int q) { return vr[q]; });
            const T *w = us + (r + 3) * WW + (tx + 3);   // u(i, j)
            T fx[7], fy[7];
#pragma unroll
            for (int k = 0; k < 7; k++) {
                fx[k] = w[k - 3];
                fy[k] = w[(k - 3) * WW];
            }
            const T dx = up4_diff(a, fx), dy = up4_diff(b, fy);
            T tend = -(a * dx + b * dy) * m.inv_hxa;
            const T g11 = __ldg(av.S + o), g21 = __ldg(av.S + box + o), g22 = __ldg(av.S + 2 * box + o);
            tend = tend - (a * a * g11 + T(2) * a * b * g21 + b * b * g22) * av.inv_neg_radius;
            A[po + d.fs + o] = tend;
        }
        if (i <= iv && j <= jv) {
            // v point: u_at_v = I_i2c,y(uh) and vt
            const T b = __ldg(W + po + 2 * d.fs + o);
            const T *uc = uhs + tx - (j0 - 2) * TX;
            const T a = ii2c<T>(j, N, [&](int q) { return uc[q * TX]; });
            const T *w = vs + (r + 3) * WW + (tx + 3);   // v(i, j)
            T fx[7], fy[7];
#pragma unroll
            for (int k = 0; k < 7; k++) {
                fx[k] = w[k - 3];
                fy[k] = w[(k - 3) * WW];
            }
            const T dx = up4_diff(a, fx), dy = up4_diff(b, fy);
            T tend = -(a * dx + b * dy) * m.inv_hxa;
            const T *S = av.S + 3 * box;
            const T g11 = __ldg(S + o), g21 = __ldg(S + box + o), g22 = __ldg(S + 2 * box + o);
            tend = tend - (a * a * g11 + T(2) * a * b * g21 + b * b * g22) * av.inv_neg_radius;
            A[po + 2 * d.fs + o] = tend;
        }
    }
}

// A at a duplicated panel-edge point after the reference's 'cross' exchange and
// sync_ch_cov (vector_advection_Ch_mod.f90:56-115): the mean of this panel's value
// and the neighbour's tangential component (with its orientation sign).
// comp 1: u point (i, j) with j = 1 or N+1; comp 2: v point with i = 1 or N+1.
template <class T>
__device__ __forceinline__ T adv_edge_sync(const T *A, const Dims &d, int mem, int t, int comp, int i, int j, T own)
{
    const int N = d.N, n = N + 1;
    const int s = comp == 1 ? (j == 1 ? SIDE_B : SIDE_T) : (i == 1 ? SIDE_L : SIDE_R);
    const Link L = c_link[t][s];
    const int c = comp == 1 ? i : j;                 // centre index along the edge
    const int cp = L.rev ? N + 1 - c : c;
    const T *a = A + mem * d.ms + L.nb * d.ps;
    T nbv;
    if (L.nside >= SIDE_B) nbv = __ldg(a + d.fs + box_off(d.P, cp, L.nside == SIDE_B ? 1 : n));
    else nbv = __ldg(a + 2 * d.fs + box_off(d.P, L.nside == SIDE_L ? 1 : n, cp));
    return T(0.5) * (own + T(L.st) * nbv);
}

}  // namespace chswe
