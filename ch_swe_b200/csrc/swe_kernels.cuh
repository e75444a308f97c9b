// swe_kernels.cuh -- device building blocks of the linear shallow-water RK4 step
// on the Ch-staggered equiangular cubed sphere (SBP 4-2): global-memory panel
// views, the cube-edge halo reads that replace the reference's MPI exchanges,
// the edge synchronisations, and the elementwise kernels.  The per-stage
// kernels are in swe_tiled.cuh:
//   k_co2contra : (u, v) of the stage input -> contravariant (ut, vt)
//                 (co2contra_Ch_mod.f90:27-94)
//   k_stage     : gradient + SAT, Coriolis with the ECS vector edge sync,
//                 divergence + SAT with the Ah scalar edge sync, the linear
//                 tendency (operator_swm_lin_mod.f90:66-108) and the RK4 update
//                 (rk4_mod.f90:28-40) fused in one pass.
//   k_edge      : the synchronised Coriolis vector and divergence of every
//                 panel-boundary vertex, once per stage, into the edge buffer.
// Neighbouring panels live in the same allocation: threads read across a cube
// edge through the `Link` table instead of waiting for an exchange.
#pragma once

#include "swe_common.cuh"
#include "swe_sbp.cuh"

namespace chswe {

// Edge connectivity, filled once per device by the host.
static __constant__ Link c_link[NPAN][4];

// Read-only view of one field of one panel: v(i, j) with the reference's 1-based indices.
template <class T>
struct GV {
    const T *p;
    int P;
    __device__ __forceinline__ T operator()(int i, int j) const { return __ldg(p + (j - 1 + MG) * P + (i - 1 + MG)); }
};

template <class T>
__device__ __forceinline__ GV<T> gview(const T *member_base, const Dims &d, int field, int panel)
{
    return GV<T>{member_base + field * d.fs + panel * d.ps, d.P};
}
template <class T>
__device__ __forceinline__ GV<T> mview(const T *p, const Dims &d)
{
    return GV<T>{p, d.P};
}

// A member whose per-member time step is 0 is frozen: every block of it exits at once.
__device__ __forceinline__ bool member_frozen(const double *dtm, int mem) { return dtm && dtm[mem] == 0.0; }

// Vertex of side s at along-edge index a (1..N+1), `depth` nodes inward.
__device__ __forceinline__ void side_vertex(int N, int s, int a, int depth, int &i, int &j)
{
    switch (s) {
    case SIDE_L: i = 1 + depth; j = a; break;
    case SIDE_R: i = N + 1 - depth; j = a; break;
    case SIDE_B: i = a; j = 1 + depth; break;
    default: i = a; j = N + 1 - depth; break;
    }
}

// h at the neighbour's copy of the shared vertex (xy halo index 0 / N+2).
template <class T>
__device__ __forceinline__ T h_halo(const T *Y, const Dims &d, int t, int s, int a)
{
    const Link L = c_link[t][s];
    int ap = L.rev ? d.N + 2 - a : a;
    int k, l;
    side_vertex(d.N, L.nside, ap, 0, k, l);
    return gview(Y, d, 0, L.nb)(k, l);
}

// Edge buffer: for every member, panel, side and along-edge vertex a = 1..N+1
// the synchronised (up, vp, div) of that panel-boundary vertex.
__device__ __forceinline__ int64_t edge_index(int N, int mem, int t, int s, int a)
{
    return ((((int64_t)mem * NPAN + t) * 4 + s) * (N + 1) + (a - 1)) * 3;
}

// Edge strips: for every member, panel and side, the contravariant components the
// edge sync reads, contiguous along the side (written by k_co2contra):
//   line 0..2: the normal component at depth 1..3 (centres), at along-edge node b = 1..N+1
//   line 3   : the tangential component on the edge line, at along-edge centre c = 1..N
// Normal/tangential: ut/vt on the L and R sides, vt/ut on B and T.  Depth counts
// from the side (L: i = d, R: i = N+1-d, B: j = d, T: j = N+1-d).
// The lines per side are NDEP + 1 of the SBP order (4 for 4-2 and 2-1, 7 for 6-3).
constexpr int STRIP_LINES = 4;
template <int ORD> __host__ __device__ constexpr int strip_lines() { return SbpOrder<ORD>::NDEP + 1; }

__host__ __device__ __forceinline__ int64_t strip_member(int N, int mem, int nl = STRIP_LINES)
{
    return (int64_t)mem * NPAN * 4 * nl * (N + 1);
}

template <class T>
struct Strips {
    const T *es;   // member base
    int n;         // N + 1
    int nl;        // lines per side: normal depths 1..nl-1, then the tangential line
    // 1-based line of panel p, side s
    __device__ __forceinline__ const T *line(int p, int s, int k) const { return es + ((p * 4 + s) * nl + k) * n - 1; }
};

// Position of xy vertex (k, l) along side s (1..N+1).
__device__ __forceinline__ int along(int s, int k, int l) { return s <= SIDE_R ? l : k; }

// The neighbour's along-edge index of along index b on side s of panel p.
__device__ __forceinline__ int nb_along(const Link &L, int n, int b) { return L.rev ? n + 1 - b : b; }

// J * normal contravariant component of the neighbour across side s of panel p,
// at depth dd and along index b of this side, with the orientation sign: the halo
// the Ch vector exchange (exchange_halo_Ch_mod.f90) delivers for the divergence SAT.
template <class T>
__device__ __forceinline__ T sat_halo(const Strips<T> &S, const MetricView<T> &m, int p, int s, int b, int dd)
{
    const Link L = c_link[p][s];
    const int n = S.n, bp = nb_along(L, n, b);
    return T(L.sn) * (m.ej[(L.nside * S.nl + dd - 1) * n + bp - 1] * S.line(L.nb, L.nside, dd - 1)[bp]);
}

// One raw quantity at along index b of side s of panel p, before any edge sync:
//   q = 0: up = fJ2 I_c2i,y(vt)      q = 1: vp = -fJ2 I_c2i,x(ut)
//          (coriolis_Ch_mod.f90:97-120)
//   q = 2: c2i x-difference of J ut  q = 3: c2i y-difference of J vt
//          with the SAT terms of sbp_diff_c2i_42_mod.f90:195-251 (sbp_diff_c2i_21_mod.f90:100-146
//          for ORD 21) on the panel edge
//          (div_sbp_sat_mod.f90:54-80 before the 1/(hx J) scaling).
// Across the side the stencils are the first closure rows; along it the full
// SBP stencils, with the second SAT at the cube corners.
template <class T, int ORD = 42>
__device__ __forceinline__ T edge_raw(const Strips<T> &S, const MetricView<T> &m, int p, int s, int b, int q)
{
    using SB = SbpOrder<ORD>;
    const int n = S.n, N = n - 1, nl = S.nl;
    const bool lr = s <= SIDE_R, lo = (s == SIDE_L || s == SIDE_B);
    const T *tg = S.line(p, s, nl - 1);
    const T *jn = m.ej + s * nl * n - 1, *jt = m.ej + (s * nl + nl - 1) * n - 1;
    const bool across = lr ? (q == 1 || q == 2) : (q == 0 || q == 3);
    if (q <= 1) {
        const T f = m.ef[(p * 4 + s) * n + b - 1];
        T v;
        if (across) {
            // first c2i interpolation row on the normal lines at depths 1..NDEP
            v = T(SB::ic1(1)) * S.line(p, s, 0)[b];
#pragma unroll
            for (int dd = 2; dd <= SB::NDEP; dd++) v += T(SB::ic1(dd)) * S.line(p, s, dd - 1)[b];
        } else {
            v = SB::template ic2i<T>(b, n, [&](int c) { return tg[c]; });
        }
        return q == 0 ? f * v : -f * v;
    }
    if (across) {
        // J * normal component at depths 1..NDEP; first c2i difference row and the SAT
        T jd[SB::NDEP];
#pragma unroll
        for (int dd = 1; dd <= SB::NDEP; dd++) jd[dd - 1] = jn[(dd - 1) * n + b] * S.line(p, s, dd - 1)[b];
        T dd = T(SB::dc1(1)) * jd[0];
#pragma unroll
        for (int k = 2; k <= SB::NDEP; k++) dd += T(SB::dc1(k)) * jd[k - 1];
        if (!lo) dd = -dd;
        T ssum = T(SB::r1(1)) * (jd[0] - sat_halo(S, m, p, s, b, 1));
#pragma unroll
        for (int k = 2; k <= SB::NR; k++) ssum += T(SB::r1(k)) * (jd[k - 1] - sat_halo(S, m, p, s, b, k));
        const T sat = T(SB::SATC) * ssum;
        return lo ? dd + sat : dd - sat;
    }
    auto jtv = [&](int c) { return jt[c] * tg[c]; };
    T dd = SB::template dc2i<T>(b, n, jtv);
    if (b == 1 || b == n) {
        // cube corner: the SAT across the other side through this vertex
        const int s2 = lr ? (b == 1 ? SIDE_B : SIDE_T) : (b == 1 ? SIDE_L : SIDE_R);
        const int b2 = lo ? 1 : n;
        T ssum = T(SB::r1(1)) * (jtv(b == 1 ? 1 : N) - sat_halo(S, m, p, s2, b2, 1));
#pragma unroll
        for (int k = 2; k <= SB::NR; k++) ssum += T(SB::r1(k)) * (jtv(b == 1 ? k : N + 1 - k) - sat_halo(S, m, p, s2, b2, k));
        const T sat = T(SB::SATC) * ssum;
        dd = b == 1 ? dd + sat : dd - sat;
    }
    return dd;
}

// The neighbour's raw vertex vector (upn, vpn) in this panel's frame, as the
// reference's 'cross' vector exchange delivers it across side s.
template <class T>
__device__ __forceinline__ void halo_vec(int t, int s, T upn, T vpn, T &uh, T &vh)
{
    const Link L = c_link[t][s];
    const bool nlr = L.nside <= SIDE_R;
    const T nrm = nlr ? upn : vpn, tan = nlr ? vpn : upn;
    if (s <= SIDE_R) { uh = T(L.sn) * nrm; vh = T(L.st) * tan; }
    else { vh = T(L.sn) * nrm; uh = T(L.st) * tan; }
}

// Metric on the panel edges, contiguous along each side, for the edge sync:
//   ej[(s*nl + k)*(N+1) + b-1]: J at the normal component's depth k+1 (k < nl-1, node b)
//                               and at the tangential component on the edge line (k = nl-1, centre b)
//   (nl: the strip lines per side of the SBP order)
//   ef[(p*4 + s)*(N+1) + b-1]: fJ2 of panel p at boundary vertex b of side s
//   ea[s*(N+1) + b-1]        : 1/(J a) at boundary vertex b of side s
template <class T>
__global__ void k_edge_tables(MetricView<T> m, Dims d, T *ej, T *ef, T *ea, int nl)
{
    const int N = d.N, n = N + 1;
    const int b = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (b > n) return;
    const GV<T> Jy = mview(m.Jy, d), Jx = mview(m.Jx, d), iJa = mview(m.iJa, d);
    for (int s = 0; s < 4; s++) {
        for (int k = 1; k <= nl - 1; k++) {
            T v;
            switch (s) {
            case SIDE_L: v = Jy(k, b); break;
            case SIDE_R: v = Jy(n - k, b); break;
            case SIDE_B: v = Jx(b, k); break;
            default: v = Jx(b, n - k); break;
            }
            ej[(s * nl + k - 1) * n + b - 1] = v;
        }
        T v = 0;
        if (b <= N) {
            switch (s) {
            case SIDE_L: v = Jx(1, b); break;
            case SIDE_R: v = Jx(n, b); break;
            case SIDE_B: v = Jy(b, 1); break;
            default: v = Jy(b, n); break;
            }
        }
        ej[(s * nl + nl - 1) * n + b - 1] = v;
        int k, l;
        side_vertex(N, s, b, 0, k, l);
        ea[s * n + b - 1] = iJa(k, l);
        for (int p = 0; p < NPAN; p++) ef[(p * 4 + s) * n + b - 1] = mview(m.fJ2 + p * d.ps, d)(k, l);
    }
}

constexpr int EDGE_CHUNK = 32;    // along-edge vertices per block (balanced split, at most 32)
constexpr int EDGE_THREADS = 288; // 8 warps of raw stencils + 1 warp for the third panel at corners

// The panel-boundary vertices' synchronised Coriolis vector (ECS Ah covariant
// vector sync, ecs_Ah_vec_sync_mod.f90:62-125 with (U, V) = (vp, up)) and
// divergence (Ah scalar sync, halo_Ah_scalar_sync_mod.f90:43-98): the work the
// reference does with its 'cross' and 'full' exchanges before the edge loops.
// Block = (chunk of vertices along one side of one panel of one member); every
// read is from the edge strips and edge tables, contiguous along the side.
// Phase 1: every raw quantity the chunk needs is one thread's stencil: warp w < 8
// takes quantity w % 4 for copy w / 4 (own vertex / neighbour across this side),
// warp 8 the copy of the third panel at the two cube corners.  Phase 2 combines
// the copies from shared memory.  Copies are stored by direction (x-neighbour
// across L/R, y-neighbour across B/T).
// Chunk ch of nch along side s of panel t (ts = 4 t + s) of member mem.
template <class T, int ORD>
__device__ __forceinline__ void edge_chunk(unsigned ch, unsigned nch, unsigned ts, unsigned mem, const T *__restrict__ ES,
                                           const T *__restrict__ ESd, T *__restrict__ E, const Dims &d,
                                           const MetricView<T> &m, const double *__restrict__ dtm)
{
    __shared__ T raw[3][4][EDGE_CHUNK];   // [own, x-neighbour, y-neighbour][quantity][vertex]
    const int N = d.N, n = N + 1;
    const int t = ts >> 2, s = ts & 3;
    const int a0 = 1 + (ch * n) / nch, a1 = 1 + ((ch + 1) * n) / nch;
    if (member_frozen(dtm, mem)) return;
    // Coriolis parts (q 0, 1) from the ut/vt strips, divergence parts (q 2, 3) from
    // the strips of the field whose divergence is taken (ut/vt, or the mass flux)
    constexpr int NL = strip_lines<ORD>();
    const Strips<T> Sc{ES + strip_member(N, mem, NL), n, NL}, Sd{ESd + strip_member(N, mem, NL), n, NL};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool xs = s <= SIDE_R;
    pdl_trigger();
    // phase-1 task of this thread: raw quantity rq of the copy of panel rp, side rs,
    // along index rb (one call site keeps the kernel's code small: every block runs
    // once per SM on a cold instruction cache)
    int rp = -1, rs = 0, rb = 0, rq = 0, dst = 0;
    if (warp < 8) {
        const int a = a0 + lane;
        rq = warp & 3;
        if (a < a1) {
            if (warp < 4) {
                rp = t; rs = s; rb = a;
                dst = rq * EDGE_CHUNK + lane;
            } else {
                const Link L = c_link[t][s];
                rp = L.nb; rs = L.nside; rb = nb_along(L, n, a);
                dst = ((xs ? 1 : 2) * 4 + rq) * EDGE_CHUNK + lane;
            }
        }
    } else if (lane < 8) {
        // the other neighbour of the corner vertices a = 1 and a = N+1
        const int a = lane < 4 ? 1 : n;
        rq = lane & 3;
        if (a >= a0 && a < a1) {
            int k, l;
            side_vertex(N, s, a, 0, k, l);
            const int s2 = xs ? (l == 1 ? SIDE_B : SIDE_T) : (k == 1 ? SIDE_L : SIDE_R);
            const Link L2 = c_link[t][s2];
            rp = L2.nb; rs = L2.nside; rb = nb_along(L2, n, along(s2, k, l));
            dst = ((xs ? 2 : 1) * 4 + rq) * EDGE_CHUNK + (a - a0);
        }
    }
    // phase-2 metric of this thread's vertex, before the predecessor grid completes
    const int v = threadIdx.x, av = a0 + v;
    int kv = 1, lv = 1;
    if (av < a1) side_vertex(N, s, av, 0, kv, lv);
    const bool il = (kv == 1), ir = (kv == n), ib = (lv == 1), it = (lv == n);
    const bool cx = il || ir, cy = ib || it;
    T ea0 = 0, eax = 0, eay = 0, qx = 0, qy = 0;
    if (av < a1) {
        ea0 = m.ea[s * n + av - 1];
        if (cx) {
            const Link L = c_link[t][il ? SIDE_L : SIDE_R];
            eax = m.ea[L.nside * n + nb_along(L, n, lv) - 1];
            qx = __ldg((il ? m.ql : m.qr) + lv - 1);
        }
        if (cy) {
            const Link L = c_link[t][ib ? SIDE_B : SIDE_T];
            eay = m.ea[L.nside * n + nb_along(L, n, kv) - 1];
            qy = __ldg((ib ? m.qb : m.qt) + kv - 1);
        }
    }
    pdl_wait();
    if (rp >= 0) (&raw[0][0][0])[dst] = edge_raw<T, ORD>(rq < 2 ? Sc : Sd, m, rp, rs, rb, rq);
    __syncthreads();
    if (av >= a1) return;
    const T V = raw[0][0][v], U = raw[0][1][v];
    const T f = (raw[0][2][v] * m.inv_hx + raw[0][3][v] * m.inv_hx) * ea0;
    T uhx = 0, vhx = 0, fx = 0, uhy = 0, vhy = 0, fy = 0;
    if (cx) {
        halo_vec(t, il ? SIDE_L : SIDE_R, raw[1][0][v], raw[1][1][v], uhx, vhx);
        fx = (raw[1][2][v] * m.inv_hx + raw[1][3][v] * m.inv_hx) * eax;
    }
    if (cy) {
        halo_vec(t, ib ? SIDE_B : SIDE_T, raw[2][0][v], raw[2][1][v], uhy, vhy);
        fy = (raw[2][2][v] * m.inv_hx + raw[2][3][v] * m.inv_hx) * eay;
    }
    T sup, svp, sdiv;
    if (cx && cy) {
        sup = (V + uhx + uhy + qx * vhx) / T(3);
        svp = (U + vhx + vhy + qy * uhy) / T(3);
        sdiv = (f + fx + fy) / T(3);
    } else if (cx) {
        sup = T(0.5) * (V + uhx + qx * vhx);
        svp = T(0.5) * (U + vhx);
        sdiv = T(0.5) * (f + fx);
    } else {
        sup = T(0.5) * (V + uhy);
        svp = T(0.5) * (U + vhy + qy * uhy);
        sdiv = T(0.5) * (f + fy);
    }
    T *e = E + edge_index(N, mem, t, s, av);
    e[0] = sup;
    e[1] = svp;
    e[2] = sdiv;
}

template <class T, int ORD>
__global__ void __launch_bounds__(EDGE_THREADS) k_edge(const T *__restrict__ ES, const T *__restrict__ ESd,
                                                        T *__restrict__ E, Dims d, MetricView<T> m,
                                                        const double *__restrict__ dtm)
{
    edge_chunk<T, ORD>(blockIdx.x, gridDim.x, blockIdx.y, blockIdx.z, ES, ESd, E, d, m, dtm);
}

// Synchronised (up, vp, div) of panel-boundary vertex (k, l) from the edge buffer.
template <class T>
__device__ __forceinline__ const T *edge_entry(const T *E, int N, int mem, int t, int k, int l)
{
    const int n = N + 1;
    if (k == 1) return E + edge_index(N, mem, t, SIDE_L, l);
    if (k == n) return E + edge_index(N, mem, t, SIDE_R, l);
    if (l == 1) return E + edge_index(N, mem, t, SIDE_B, k);
    return E + edge_index(N, mem, t, SIDE_T, k);
}

// threads of a stage / contravariant tile block
constexpr int STAGE_THREADS = 256;

// RK4 stage parameters.
struct StageArgs {
    int mode;          // 0: write the tendency A(y) to out; 1..4: RK4 stage
    double dt;
    const double *Hm;  // per-member mean depth
    const double *dtm; // per-member time step (null: dt for all); 0 freezes a member
    // advective operator only (null for the linear one): the mass flux (fields 1, 2
    // of a state box) whose divergence gives dh, and the advective wind tendencies
    const void *F;
    const void *A;
    const void *HB;    // panel-boundary h before the in-place averaging (the gradient's input)
    const void *HS;    // advective operator: orography h_surf (one field box of panels), or null;
                       // the gradient's input is h + h_surf (operator_adv_swm_mod.f90:78)
};

// Kahan-compensated state update for FP32 (s += inc with compensation c).
__device__ __forceinline__ void kahan_add(float &s, float &c, float inc)
{
    float yk = inc - c;
    float tk = s + yk;
    c = (tk - s) - yk;
    s = tk;
}

// y = s1*v1 + s2*v2 (v2 may be null) or y += s1*v1 + s2*v2 over the whole box.
template <class T>
__global__ void k_axpby(T *y, const T *v1, const T *v2, double s1, double s2, int accumulate, int64_t n)
{
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; k < n; k += stride) {
        T r = T(s1) * v1[k];
        if (v2) r = r + T(s2) * v2[k];
        y[k] = accumulate ? y[k] + r : r;
    }
}

}  // namespace chswe
