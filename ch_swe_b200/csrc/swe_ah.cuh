// swe_ah.cuh -- the linear shallow-water operator on the Ah staggering: h, u and v
// all on the cell vertices (the xy mesh), the operator set of the reference's Ah
// configuration (gen_config_linear.sh:9-36):
//   grad_ah_sbp_proj_42     node-to-node SBP 4-2 differences (sbp_diff_42_mod.f90:30-156;
//                           2-1 and 6-3 for the _21 / _63 names)
//                           and the covariant ECS Ah vector sync of the panel-edge
//                           vertices (grad_sbp_proj_mod.f90:26-72, ecs_Ah_vec_sync_mod.f90:34-125)
//   co2contra_colocated     ut = Qi11 u + Qi12 v, vt = Qi12 u + Qi22 v at each vertex
//                           (co2contra_colocated_mod.f90:17-47)
//   coriolis_colocated      cor_u = f vt J, cor_v = -f ut J (coriolis_colocated_mod.f90:17-45)
//   div_ah_sbp_proj_42      the same differences of J ut, J vt over J a and the Ah scalar
//                           sync (div_sbp_proj_mod.f90:25-76, halo_Ah_scalar_sync_mod.f90:43-98)
// then du = -g grad_x h + cor_u, dv = -g grad_y h + cor_v, dh = -H div
// (operator_swm_lin_mod.f90:66-108) and the RK4 stage update.
// Per RK stage two launches: k_ah_edge (the raw gradient and divergence of every
// panel-boundary vertex, for its neighbours' syncs) and k_ah_stage (every vertex:
// raw values, the syncs on the panel edges, the tendency and the RK update).
#pragma once

#include "swe_kernels.cuh"

namespace chswe {

// Metric of the Ah operator at the vertices (host FP64, stored in T).
template <class T>
struct AhView {
    const T *J;            // J (one panel-independent box)
    const T *Q1, *Q2, *Q3; // the inverse metric Qi11, Qi12, Qi22 (boxes)
    const T *fJ;           // f J, one box per panel
};

namespace sbp {
// sbp_diff_42_mod.f90:10-23: the reference's decimal coefficients of the node-to-node
// SBP 4-2 first derivative's closure rows
constexpr double N11 = -1.4117647058823528, N12 = 1.7352941176470589, N13 = -0.2352941176470588,
                 N14 = -0.08823529411764705, N21 = -0.5, N23 = 0.5, N31 = 0.09302325581395347,
                 N32 = -0.686046511627907, N34 = 0.686046511627907, N35 = -0.09302325581395347,
                 N41 = 0.030612244897959186, N43 = -0.6020408163265307, N45 = 0.653061224489796,
                 N46 = -0.0816326530612245;
}  // namespace sbp

// SBP first derivative at node k of n nodes (inputs f(1..n), no halo) of order ORD:
// 2-1 (sbp_diff_21_mod.f90:8-40), 4-2 (sbp_diff_42_mod.f90:30-156), 6-3 (the table
// D_SBP63_NN_Q of sbp_diff_63_mod.f90:9-140).
template <class T, class F>
__device__ __forceinline__ T dn2n21(int k, int n, const F &f)
{
    if (k >= 2 && k <= n - 1) return (-f(k - 1) + f(k + 1)) / T(2);
    if (k == 1) return T(-1) * f(1) + T(1) * f(2);
    return -T(-1) * f(n) - T(1) * f(n - 1);
}
template <class T, class F>
__device__ __forceinline__ T dn2n63(int k, int n, const F &f)
{
    if (k >= 7 && k <= n - 6)
        return (-f(k - 3) + T(9) * f(k - 2) + T(-45) * f(k - 1) + T(45) * f(k + 1) + T(-9) * f(k + 2) + f(k + 3)) / T(60);
    const bool lo = k <= 6;
    const int r = lo ? k : n + 1 - k;
    T a = T(0);
#pragma unroll
    for (int q = 0; q < 9; q++) {
        const double c = D_SBP63_NN_Q[r - 1][q];
        if (c == 0.0) continue;
        a = lo ? a + T(c) * f(q + 1) : a - T(c) * f(n - q);
    }
    return a;
}
template <class T, class F>
__device__ __forceinline__ T dn2n42(int k, int n, const F &f)
{
    using namespace sbp;
    if (k >= 5 && k <= n - 4) return (f(k - 2) + T(-8) * f(k - 1) + T(8) * f(k + 1) + -f(k + 2)) / T(12);
    if (k == 1) return T(N11) * f(1) + T(N12) * f(2) + T(N13) * f(3) + T(N14) * f(4);
    if (k == 2) return T(N21) * f(1) + T(N23) * f(3);
    if (k == 3) return T(N31) * f(1) + T(N32) * f(2) + T(N34) * f(4) + T(N35) * f(5);
    if (k == 4) return T(N41) * f(1) + T(N43) * f(3) + T(N45) * f(5) + T(N46) * f(6);
    if (k == n - 3) return -T(N41) * f(n) - T(N43) * f(n - 2) - T(N45) * f(n - 4) - T(N46) * f(n - 5);
    if (k == n - 2) return -T(N31) * f(n) - T(N32) * f(n - 1) - T(N34) * f(n - 3) - T(N35) * f(n - 4);
    if (k == n - 1) return -T(N21) * f(n) - T(N23) * f(n - 2);
    return -T(N11) * f(n) - T(N12) * f(n - 1) - T(N13) * f(n - 2) - T(N14) * f(n - 3);
}

template <class T, int ORD, class F>
__device__ __forceinline__ T dn2n(int k, int n, const F &f)
{
    if constexpr (ORD == 21) return dn2n21<T>(k, n, f);
    else if constexpr (ORD == 63) return dn2n63<T>(k, n, f);
    else return dn2n42<T>(k, n, f);
}

// Raw (before the panel-edge syncs) gradient (gx, gy) and divergence of the
// contravariant wind at vertex (i, j) of panel t; y is the member's state.
template <class T, int ORD>
__device__ __forceinline__ void ah_raw(const T *y, const Dims &d, const AhView<T> &a, const MetricView<T> &m, int t,
                                       int i, int j, T &gx, T &gy, T &dv)
{
    const int n = d.N + 1;
    const GV<T> H = gview(y, d, 0, t), U = gview(y, d, 1, t), V = gview(y, d, 2, t);
    const GV<T> J = mview(a.J, d), Q1 = mview(a.Q1, d), Q2 = mview(a.Q2, d), Q3 = mview(a.Q3, d);
    gx = dn2n<T, ORD>(i, n, [&](int k) { return H(k, j); }) * m.inv_hxa;
    gy = dn2n<T, ORD>(j, n, [&](int k) { return H(i, k); }) * m.inv_hxa;
    const T dx = dn2n<T, ORD>(i, n, [&](int k) { return J(k, j) * (Q1(k, j) * U(k, j) + Q2(k, j) * V(k, j)); });
    const T dy = dn2n<T, ORD>(j, n, [&](int k) { return J(i, k) * (Q2(i, k) * U(i, k) + Q3(i, k) * V(i, k)); });
    dv = (dx * m.inv_hx + dy * m.inv_hx) * mview(m.iJa, d)(i, j);
}

// k_ah_edge: the raw (gx, gy, div) of every panel-boundary vertex into the edge
// buffer (edge_index: member, panel, side, along index).  Grid (along chunks,
// panel * 4 + side, member).
template <class T, int ORD>
__global__ void __launch_bounds__(128) k_ah_edge(const T *__restrict__ Y, T *__restrict__ E, Dims d, AhView<T> a,
                                                 MetricView<T> m, const double *__restrict__ dtm)
{
    const int N = d.N, n = N + 1;
    const int t = blockIdx.y >> 2, s = blockIdx.y & 3, mem = blockIdx.z;
    if (member_frozen(dtm, mem)) return;
    const int b = blockIdx.x * blockDim.x + threadIdx.x + 1;
    pdl_trigger();
    pdl_wait();
    if (b > n) return;
    int i, j;
    side_vertex(N, s, b, 0, i, j);
    T gx, gy, dv;
    ah_raw<T, ORD>(Y + mem * d.ms, d, a, m, t, i, j, gx, gy, dv);
    T *e = E + edge_index(N, mem, t, s, b);
    e[0] = gx;
    e[1] = gy;
    e[2] = dv;
}

// Tiles of k_ah_stage: AH_TX x AH_TY vertices per block of 32 x 8 threads (two rows
// per thread); the windows reach AH_R(ORD) vertices beyond the tile on each side, the
// farthest input of an SBP row of that order (2-1: 1; 4-2: 3, the closure rows 1
// and 4; 6-3: 8, the closure row 1 reaches f(9)).
constexpr int AH_TX = 32, AH_TY = 16;
template <int ORD>
__host__ __device__ constexpr int ah_reach() { return ORD == 21 ? 1 : (ORD == 63 ? 8 : 3); }

// k_ah_stage: every vertex of every panel and member, one tile per block.  The block
// stages h and the fluxes J (Qi11 u + Qi12 v), J (Qi12 u + Qi22 v) of its window in
// shared memory (each window vertex loaded and multiplied once), then each thread
// takes the x and y differences of its vertices from there: the raw values; on the
// panel edges the syncs with the neighbours' raw values from k_ah_edge (the
// neighbour's vector is handed over as the 'cross' exchange does, halo_vec); the
// tendency and the RK update of k_stage (modes 0..4; FP32 mode 4 Kahan-compensated).
template <class T, int MODE, int ORD>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 3) k_ah_stage(const T *__restrict__ Yin, const T *__restrict__ E, T *V0, T *Y1,
                                                  T *ACC, T *CMP, Dims d, AhView<T> a, MetricView<T> m, StageArgs sa,
                                                  T grav)
{
    constexpr int R = ah_reach<ORD>(), W = AH_TX + 2 * R, H = AH_TY + 2 * R;
    constexpr int NW = (H * W + 255) / 256;            // window points per thread
    constexpr int NB = sizeof(T) == 8 ? 2 : 4;         // of them loaded per batch
    constexpr int RR = AH_TY / 8;                      // tile rows per thread
    __shared__ T sH[H * W], sF[H * W], sG[H * W];
    const int N = d.N, n = N + 1;
    const int mem = blockIdx.z / NPAN, t = blockIdx.z % NPAN;
    if (member_frozen(sa.dtm, mem)) return;
    // balanced tiles of at most AH_TX x AH_TY vertices (no slivers at the panel's far side)
    const int i0 = 1 + (blockIdx.x * n) / gridDim.x, i1 = 1 + ((blockIdx.x + 1) * n) / gridDim.x;
    const int j0 = 1 + (blockIdx.y * n) / gridDim.y, j1 = 1 + ((blockIdx.y + 1) * n) / gridDim.y;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const T *y = Yin + mem * d.ms;
    const T *yh = y + t * d.ps, *yu = yh + d.fs, *yv = yh + 2 * d.fs;
    const int64_t po = mem * d.ms + t * d.ps;
    const int64_t fs = d.fs;
    pdl_trigger();
    pdl_wait();
    // the RK operands of this thread's vertices, in flight during the window phase
    constexpr bool LV = MODE >= 1, LA = MODE >= 2, LC = (sizeof(T) == 4) && MODE == 4;
    T pv[3][RR], pa[3][RR], pc[3][RR];
#pragma unroll
    for (int rr = 0; rr < RR; rr++) {
        const int i = i0 + threadIdx.x, j = j0 + threadIdx.y + 8 * rr;
        const bool ok = i < i1 && j < j1;
        const int64_t o = po + box_off(d.P, i, j);
#pragma unroll
        for (int f = 0; f < 3; f++) {
            pv[f][rr] = LV && ok ? V0[o + f * fs] : T(0);
            pa[f][rr] = LA && ok ? ACC[o + f * fs] : T(0);
            pc[f][rr] = LC && ok ? CMP[o + f * fs] : T(0);
        }
    }
    // the window: the tile's rows over the x reach and its columns over the y reach (the
    // corners are never read); vertices outside the panel hold zeros (no stencil reads
    // them).  Each batch issues all of its loads before its first multiply.
#pragma unroll
    for (int b0 = 0; b0 < NW; b0 += NB) {
        T rh[NB], ru[NB], rv[NB], rj[NB], r1[NB], r2[NB], r3[NB];
#pragma unroll
        for (int k = 0; k < NB; k++) {
            const int q = tid + (b0 + k) * 256;
            const int wi = q % W, wj = q / W;
            const int i = i0 - R + wi, j = j0 - R + wj;
            const bool band = (wj >= R && wj < R + AH_TY) || (wi >= R && wi < R + AH_TX);
            const bool ok = b0 + k < NW && q < H * W && band && i >= 1 && i <= n && j >= 1 && j <= n;
            const int64_t o = ok ? box_off(d.P, i, j) : 0;
            rh[k] = ok ? __ldcg(yh + o) : T(0);
            ru[k] = ok ? __ldcg(yu + o) : T(0);
            rv[k] = ok ? __ldcg(yv + o) : T(0);
            rj[k] = ok ? __ldg(a.J + o) : T(0);
            r1[k] = ok ? __ldg(a.Q1 + o) : T(0);
            r2[k] = ok ? __ldg(a.Q2 + o) : T(0);
            r3[k] = ok ? __ldg(a.Q3 + o) : T(0);
        }
#pragma unroll
        for (int k = 0; k < NB; k++) {
            const int q = tid + (b0 + k) * 256;
            if (b0 + k < NW && q < H * W) {
                sH[q] = rh[k];
                sF[q] = rj[k] * (r1[k] * ru[k] + r2[k] * rv[k]);
                sG[q] = rj[k] * (r2[k] * ru[k] + r3[k] * rv[k]);
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int rr = 0; rr < RR; rr++) {
        const int i = i0 + threadIdx.x, j = j0 + threadIdx.y + 8 * rr;
        if (i >= i1 || j >= j1) continue;
        const int ro = (j - j0 + R) * W - i0 + R, co = i - i0 + R - j0 * W + R * W;
        // row j of the window at column k, column i at row l
        T gx = dn2n<T, ORD>(i, n, [&](int k) { return sH[ro + k]; }) * m.inv_hxa;
        T gy = dn2n<T, ORD>(j, n, [&](int l) { return sH[co + l * W]; }) * m.inv_hxa;
        const T dx = dn2n<T, ORD>(i, n, [&](int k) { return sF[ro + k]; });
        const T dy = dn2n<T, ORD>(j, n, [&](int l) { return sG[co + l * W]; });
        T dv = (dx * m.inv_hx + dy * m.inv_hx) * __ldg(m.iJa + box_off(d.P, i, j));
    const bool il = i == 1, ir = i == n, jb = j == 1, jt = j == n;
    const bool cx = il || ir, cy = jb || jt;
    if (cx || cy) {
        T uhx = 0, vhx = 0, dvx = 0, uhy = 0, vhy = 0, dvy = 0, qx = 0, qy = 0;
        if (cx) {
            const int s = il ? SIDE_L : SIDE_R;
            const Link L = c_link[t][s];
            const T *e = E + edge_index(N, mem, L.nb, L.nside, nb_along(L, n, j));
            halo_vec(t, s, e[0], e[1], uhx, vhx);
            dvx = e[2];
            qx = (il ? m.ql : m.qr)[j - 1];
        }
        if (cy) {
            const int s = jb ? SIDE_B : SIDE_T;
            const Link L = c_link[t][s];
            const T *e = E + edge_index(N, mem, L.nb, L.nside, nb_along(L, n, i));
            halo_vec(t, s, e[0], e[1], uhy, vhy);
            dvy = e[2];
            qy = (jb ? m.qb : m.qt)[i - 1];
        }
        // syncronize_grad_on_edges(gy, gx) and sync_Ah_scalar_tile
        if (cx && cy) {
            const T sx = (gx + uhx + uhy + qx * vhx) / T(3);
            gy = (gy + vhx + vhy + qy * uhy) / T(3);
            gx = sx;
            dv = (dv + dvx + dvy) / T(3);
        } else if (cx) {
            gx = T(0.5) * (gx + uhx + qx * vhx);
            gy = T(0.5) * (gy + vhx);
            dv = T(0.5) * (dv + dvx);
        } else {
            gx = T(0.5) * (gx + uhy);
            gy = T(0.5) * (gy + vhy + qy * uhy);
            dv = T(0.5) * (dv + dvy);
        }
    }
    const int64_t o = box_off(d.P, i, j);
    const T u = __ldcg(yu + o), v = __ldcg(yv + o);
    const T ut = a.Q1[o] * u + a.Q2[o] * v, vt = a.Q2[o] * u + a.Q3[o] * v;
    const T fJ = a.fJ[t * d.ps + o];
    const T k3[3] = {-T(sa.Hm[mem]) * dv, -grav * gx + fJ * vt, -grav * gy - fJ * ut};
    const T dt = T(sa.dtm ? sa.dtm[mem] : sa.dt);
#pragma unroll
    for (int f = 0; f < 3; f++) {
        const int64_t of = po + o + f * fs;
        if constexpr (MODE == 0) {
            Y1[of] = k3[f];
        } else if constexpr (MODE <= 3) {
            const T ca = (MODE == 3) ? dt : T(0.5) * dt;
            const T cb = (MODE == 1) ? dt / T(6) : dt / T(3);
            Y1[of] = pv[f][rr] + ca * k3[f];
            ACC[of] = (MODE == 1) ? cb * k3[f] : pa[f][rr] + cb * k3[f];
        } else if constexpr (sizeof(T) == 4) {
            float sv = pv[f][rr], cv = pc[f][rr];
            kahan_add(sv, cv, pa[f][rr] + (dt / T(6)) * k3[f]);
            V0[of] = sv;
            CMP[of] = cv;
        } else {
            V0[of] = pv[f][rr] + (pa[f][rr] + (dt / T(6)) * k3[f]);
        }
    }
    }
}

// FP64 sums of the Ah integrals per block: term 0 <h, 1>, 1 <h, h>, 2 <u, ut> + <v, vt>
// with the SBP_Ah quadrature weights qa (J hx hy Ax Ay at the vertices).
template <class T>
__global__ void k_quad_ah(const T *__restrict__ y, const double *__restrict__ qa, AhView<T> a, Dims d,
                          double *partial)
{
    const int term = blockIdx.y;
    const int n = d.N + 1;
    const int64_t npts = (int64_t)NPAN * n * n;
    double acc = 0.0;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < npts; k += (int64_t)gridDim.x * blockDim.x) {
        const int t = (int)(k / ((int64_t)n * n)), r = (int)(k % ((int64_t)n * n));
        const int j = r / n + 1, i = r % n + 1;
        const int64_t o = box_off(d.P, i, j);
        const double h = (double)y[t * d.ps + o];
        if (term == 0) acc += h * qa[o];
        else if (term == 1) acc += h * h * qa[o];
        else {
            const double u = (double)y[d.fs + t * d.ps + o], v = (double)y[2 * d.fs + t * d.ps + o];
            const double ut = (double)a.Q1[o] * u + (double)a.Q2[o] * v, vt = (double)a.Q2[o] * u + (double)a.Q3[o] * v;
            acc += (u * ut + v * vt) * qa[o];
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

}  // namespace chswe
