// swe_fused.cuh -- the fused stage of the linear operator on the Ch grid (SBP 4-2):
// one kernel per RK stage that computes the contravariant components itself
// (co2contra_Ch_mod.f90:27-94), the gradient with its SAT, the Coriolis term with
// the ECS vector edge sync, the divergence with its SAT and scalar edge sync
// (operator_swm_lin_mod.f90:66-108) and the RK4 update (rk4_mod.f90:28-40).
//
// Per RK stage three launches, chained by programmatic dependent launch:
//   k_strip   : the contravariant components on the edge strips (normal component
//               at depths 1..3 and tangential component on the edge line of every
//               panel side), straight from the stage input;
//   k_edge    : the synchronised Coriolis vector and divergence of every
//               panel-boundary vertex from the strips (swe_kernels.cuh);
//   k_fstage  : every point of a tile.
// k_strip waits for the previous stage and then lets the other two launch, so
// k_fstage's tiles load and compute while the edge sync runs; only tiles that
// touch a panel edge wait for it, just before they need its values.
//
// Tiles are at most FUSED_TW = 26 columns by TH rows.  The block loads its
// windows (h, u, v of the stage input and seven metric arrays, each the tile plus
// four points on every side) with TMA 2-D tile loads into shared memory.  Every
// pass maps one lane to one column and the eight warps to rows, so a warp reads
// and writes consecutive shared-memory words for both x and y stencils (no bank
// conflicts at any pitch), y-stencil closures are warp-uniform, and the widest
// pass (tile + 6 columns) fits 32 lanes.
//
// Window slot layout: element (r, q) of every slot holds point
// (i0 - 4 - sx + q, j0 - 4 + r), where sx aligns the TMA tile's first column to
// 16 bytes.  Ranges of the passes (x; y is symmetric), for tile [i0, i1):
//   vq  = JQ12 I_c2i,y(v)          nodes   [i0-3, i1+3)
//   uq  = JQ12 I_c2i,x(u)          nodes   [i0-1, i1+2)
//   Jut = JQ11 u + I_i2c,x(vq)     centres [i0-2, i1+1)     (JQ11 = J Qi11)
//   Jvt = JQ22 v + I_i2c,y(uq)     nodes   [i0-1, i1+2)     (JQ22 = J Qi22)
//   up  = fJ2 I_c2i,y(vt)          nodes   [i0-1, i1+2)     (vt = Jvt / J)
//   vp  = -fJ2 I_c2i,x(ut)         nodes   [i0, i1)         (ut = Jut / J)
//   div = (D_c2i,x Jut + D_c2i,y Jvt) / (hx J a)  on the tile
// all clipped to the panel.  These are the interior stencil reaches; the SBP
// closure rows read within [1, 5] (or the mirror) of a panel edge, which the
// clipped ranges of a tile on that edge contain, and tiles away from the edges are
// at least 9 points from them (tiles are at least 13 x 9 points when a panel has
// more than one).
#pragma once

#include "swe_kernels.cuh"
#include "swe_tma.cuh"

namespace chswe {

constexpr int FUSED_THREADS = 256;
constexpr int FUSED_TW = 26;

// Boxes of the fused metric allocation, in order (one panel box each; fJ2 has six).
enum { FM_JQ12 = 0, FM_JQ11Y = 1, FM_IJY = 2, FM_JQ22X = 3, FM_IJX = 4, FM_IJA = 5, FM_FJ2 = 6, FM_BOXES = 12 };

template <class T>
struct FusedMetric {
    const T *base;   // FM_BOXES panel boxes of the metric (the strip kernel's plain loads)
    T inv_hxa;       // 1 / (hx a)
    T inv_hx;        // 1 / hx
    T grav;
};

template <class T, int TH>
struct FusedLayout {
    static constexpr int ALIGN = 16 / (int)sizeof(T);      // TMA x alignment, elements
    static constexpr int SW = sizeof(T) == 4 ? 40 : 36;     // TMA box width = slot pitch
    static constexpr int SR = TH + 8;                       // TMA box height = slot rows
    static constexpr int BOX_BYTES = SW * SR * (int)sizeof(T);
    static constexpr int SLOT_BYTES = (BOX_BYTES + 127) / 128 * 128;
    static constexpr int SLOT = SLOT_BYTES / (int)sizeof(T);
    static constexpr int NSLOT = 13;
    static constexpr int NLOAD = 10;                        // tiles loaded per block
    static constexpr int HALO = NSLOT * SLOT;               // the gradient SAT halos: 4 x 64
    static constexpr int BAR_OFF = NSLOT * SLOT_BYTES + 4 * 64 * (int)sizeof(T);
    static constexpr size_t bytes() { return (size_t)BAR_OFF + 16; }
    static constexpr int MR = (TH + 7) / 8;                 // tile rows per warp
    static constexpr int MW = (TH + 13) / 8;                // window rows per warp (up to TH + 6)
    static_assert(TH + 3 <= 40, "the boundary fill covers ranges of at most 40 points");
    static_assert(SW * (int)sizeof(T) % 16 == 0, "TMA box rows are whole 16-byte units");
    static_assert(SW - (ALIGN - 1) >= FUSED_TW + 8, "the box covers the widest window after alignment");
};

// Product of two shared-memory lines: f(c) = p[c s] q[c s].
template <class T>
struct Line2 {
    const T *p, *q;
    int s;
    __device__ __forceinline__ T operator()(int c) const { return p[c * s] * q[c * s]; }
};

// Closure rows out of line: one copy of each in the kernel's code, shared by every
// pass (the passes run once per block on a cold instruction cache, so code size
// costs more than the calls).
template <class T> __device__ __noinline__ T ic2i_cl2(int k, int nx, Line2<T> f) { return ic2i<T>(k, nx, f); }

// The SBP 4-2 operators at one output: interior rows inline, closure rows out of line.
template <class T>
__device__ __forceinline__ T f_ic2i(int k, int nx, const Line<T> &f)
{
    if (k >= 5 && k <= nx - 4) return (T(9) * (f(k) + f(k - 1)) - (f(k + 1) + f(k - 2))) * T(0.0625);
    return ic2i_cl<T>(k, nx, f);
}
template <class T>
__device__ __forceinline__ T f_ic2i(int k, int nx, const Line2<T> &f)
{
    if (k >= 5 && k <= nx - 4) return (T(9) * (f(k) + f(k - 1)) - (f(k + 1) + f(k - 2))) * T(0.0625);
    return ic2i_cl2<T>(k, nx, f);
}
template <class T>
__device__ __forceinline__ T f_ii2c(int k, int n, const Line<T> &f)
{
    if (k >= 4 && k <= n - 3) return (T(9) * (f(k + 1) + f(k)) - (f(k + 2) + f(k - 1))) * T(0.0625);
    return ii2c_cl<T>(k, n, f);
}
template <class T>
__device__ __forceinline__ T f_dc2i(int k, int nx, const Line<T> &f)
{
    if (k >= 5 && k <= nx - 4) return (T(27) * (f(k) - f(k - 1)) - (f(k + 1) - f(k - 2))) * T(1.0 / 24.0);
    return dc2i_cl<T>(k, nx, f);
}
template <class T>
__device__ __forceinline__ T f_di2c(int k, int n, const Line<T> &f)
{
    if (k >= 4 && k <= n - 3) return (T(27) * (f(k + 1) - f(k)) - (f(k + 2) - f(k - 1))) * T(1.0 / 24.0);
    return di2c_cl<T>(k, n, f);
}

// Branch-free x stencils: a lane owns one column k for a whole pass, so it looks up its
// SBP 4-2 row once -- interior or closure -- as five weights on the inputs base .. base+4,
// and every row of the pass is the same five-tap multiply-add on every lane (no divergent
// closure branches in the tiles on a panel's left and right edges).  The weights are
// those of swe_sbp.cuh (the interior rows and the closure rows with their mirrors).
template <class T>
struct XRow {
    int base;   // first input index
    T w[5];
    // p points at input `base` of the row
    __device__ __forceinline__ T dot(const T *p) const
    {
        T a = w[0] * p[0];
#pragma unroll
        for (int m = 1; m < 5; m++) a += w[m] * p[m];
        return a;
    }
    // the same on the product of two rows
    __device__ __forceinline__ T dot2(const T *p, const T *q) const
    {
        T a = w[0] * (p[0] * q[0]);
#pragma unroll
        for (int m = 1; m < 5; m++) a += w[m] * (p[m] * q[m]);
        return a;
    }
};

// The weight rows of the four x operators: [op][row][5], op 0 I_c2i (nodes k = 1..nx from
// centres 1..nx-1), 1 D_c2i, 2 I_i2c (centres k = 1..n from nodes 1..n+1), 3 D_i2c; rows
// 0-3 the closures at k = 1..4 (inputs 1..5), rows 4-7 their mirrors at k = nm - row + 4
// (inputs nm-4..nm for c2i, n-2..n+2 for i2c), row 8 the interior.  Filled on the host
// (xrow42_table) and copied to the table of each precision when a context is created.
constexpr int XROW_OPS = 4, XROW_ROWS = 9, XROW_LEN = XROW_OPS * XROW_ROWS * 5;
static __device__ float g_xrow_f[XROW_LEN];
static __device__ double g_xrow_d[XROW_LEN];

static inline void xrow42_table(double *out)
{
    using namespace sbp;
    for (int m = 0; m < XROW_LEN; m++) out[m] = 0.0;
    for (int op = 0; op < XROW_OPS; op++) {
        const bool D = op == 1 || op == 3, c2i = op <= 1;
        double q[4][5] = {};
        if (c2i) {
            const double c[4][5] = {{D ? DC11 : IC11, D ? DC12 : IC12, D ? DC13 : IC13, 0, 0},
                                    {D ? DC21 : IC21, D ? DC22 : IC22, D ? 0.0 : IC23, 0, 0},
                                    {D ? DC31 : IC31, D ? DC32 : IC32, D ? DC33 : IC33, D ? DC34 : IC34, 0},
                                    {D ? DC41 : IC41, D ? DC42 : IC42, D ? DC43 : IC43, D ? DC44 : IC44, D ? DC45 : IC45}};
            for (int r = 0; r < 4; r++)
                for (int m = 0; m < 5; m++) q[r][m] = c[r][m];
        } else {
            // the 4-2 i2c difference's third row skips its second input and reaches the fifth
            const double c[3][5] = {{D ? DI11 : II11, D ? DI12 : II12, D ? DI13 : II13, D ? DI14 : II14, 0},
                                    {D ? DI21 : II21, D ? DI22 : II22, D ? DI23 : II23, D ? DI24 : II24, 0},
                                    {D ? DI31 : II31, D ? 0.0 : II32, D ? DI33 : II33, D ? DI34 : II34, D ? DI35 : II35}};
            for (int r = 0; r < 3; r++)
                for (int m = 0; m < 5; m++) q[r][m] = c[r][m];
        }
        double *o = out + op * XROW_ROWS * 5;
        const int nrow = c2i ? 4 : 3;
        for (int r = 0; r < nrow; r++)
            for (int m = 0; m < 5; m++) {
                o[r * 5 + m] = q[r][m];
                // mirrored row: the input at distance m from the far end carries q[r][m]
                // (negated for the difference)
                o[(4 + r) * 5 + 4 - m] = D ? -q[r][m] : q[r][m];
            }
        const double in[4] = {D ? 1.0 / 24.0 : -0.0625, D ? -27.0 / 24.0 : 0.5625, D ? 27.0 / 24.0 : 0.5625,
                              D ? -1.0 / 24.0 : -0.0625};
        for (int m = 0; m < 4; m++) o[8 * 5 + m] = in[m];
    }
}

template <class T>
__device__ __forceinline__ const T *xrow_table()
{
    if constexpr (sizeof(T) == 4) return g_xrow_f;
    else return g_xrow_d;
}

// The weight row of operator op at output k of nm (nx for c2i, n for i2c), k in 1..nm.
template <class T>
__device__ __forceinline__ XRow<T> xrow42(int op, int k, int nm)
{
    const bool c2i = op <= 1;
    k = max(1, min(k, nm));
    int row, base;
    if (k <= (c2i ? 4 : 3)) {
        row = k - 1;
        base = 1;
    } else if (k > (c2i ? nm - 4 : nm - 3)) {
        row = 4 + nm - k;
        base = c2i ? nm - 5 : nm - 3;
    } else {
        row = 8;
        base = c2i ? k - 2 : k - 1;
    }
    const T *w = xrow_table<T>() + (op * XROW_ROWS + row) * 5;
    XRow<T> r;
    r.base = base;
#pragma unroll
    for (int m = 0; m < 5; m++) r.w[m] = __ldg(w + m);
    return r;
}

// h at the neighbour's copy of the shared vertex, read through L2 (the previous
// stage wrote it).
template <class T>
__device__ __forceinline__ T h_halo_cg(const T *Y, const Dims &d, int t, int s, int a)
{
    const Link L = c_link[t][s];
    const int ap = L.rev ? d.N + 2 - a : a;
    int k, l;
    side_vertex(d.N, L.nside, ap, 0, k, l);
    return ld_cg(Y + d.fs * 0 + L.nb * d.ps + box_off32(d.P, k, l));
}

__device__ __forceinline__ void ftile_range(int n, int &i0, int &i1, int &j0, int &j1)
{
    i0 = 1 + (blockIdx.x * n) / gridDim.x;
    i1 = 1 + ((blockIdx.x + 1) * n) / gridDim.x;
    j0 = 1 + (blockIdx.y * n) / gridDim.y;
    j1 = 1 + ((blockIdx.y + 1) * n) / gridDim.y;
}

// Time a block waits for its tile loads before it gives up and flags an error.
constexpr unsigned long long FUSED_WAIT_NS = 1000000000ull;

//   MODE 0: out = A(y);   1: Y1 = V0 + dt/2 k, ACC = dt/6 k;   2: Y1 = V0 + dt/2 k, ACC += dt/3 k;
//   3: Y1 = V0 + dt k, ACC += dt/3 k;   4: V0 += ACC + dt/6 k (FP32: Kahan with compensation CMP)
// tmY: the stage input as rows of P elements ([member][field][panel][row]); tmM: the
// fused metric ([box][row]); both with TMA boxes of SW x (TH + 8).
template <class T, int TH, int OCC, int MODE>
__global__ void __launch_bounds__(FUSED_THREADS, OCC)
    k_fstage(const __grid_constant__ CUtensorMap tmY, const __grid_constant__ CUtensorMap tmM, const T *__restrict__ Yin,
             const T *__restrict__ E, T *V0, T *Y1, T *ACC, T *CMP, Dims d, FusedMetric<T> fm, StageArgs a, int *err)
{
    constexpr int ORD = 42;
    using SB = SbpOrder<ORD>;
    using L = FusedLayout<T, TH>;
    constexpr int SW = L::SW;
    extern __shared__ __align__(128) unsigned char fsm_raw[];
    T *slot = reinterpret_cast<T *>(fsm_raw);
    T *const sH = slot, *const sU = slot + L::SLOT, *const sV = slot + 2 * L::SLOT, *const sJQ12 = slot + 3 * L::SLOT,
             *const sJQ11 = slot + 4 * L::SLOT, *const siJy = slot + 5 * L::SLOT, *const sJQ22 = slot + 6 * L::SLOT,
             *const siJx = slot + 7 * L::SLOT, *const sF = slot + 8 * L::SLOT, *const siJa = slot + 9 * L::SLOT,
             *const sVQ = slot + 10 * L::SLOT, *const sUQ = slot + 11 * L::SLOT, *const sJVT = slot + 12 * L::SLOT;
    // slots reused once their first contents are dead
    T *const sJUT = sJQ12, *const sUP = sVQ, *const sVP = sUQ, *const sDIV = sU;
    T *const hl = slot + L::HALO, *const hr = hl + 64, *const hb = hr + 64, *const ht = hb + 64;
    uint64_t *const bar = reinterpret_cast<uint64_t *>(fsm_raw + L::BAR_OFF);

    const int N = d.N, n = N + 1, P = d.P;
    int i0, i1, j0, j1;
    ftile_range(n, i0, i1, j0, j1);
    const int tw = i1 - i0, th = j1 - j0;
    const int t = blockIdx.z % NPAN, mem = blockIdx.z / NPAN;
    if (member_frozen(a.dtm, mem)) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int rows = N + 1 + 2 * MG;
    const int cc0 = i0 - 1;                          // box column of point i0 - 4
    const int sx = cc0 & (L::ALIGN - 1), ax = cc0 - sx;
    // slot offset of point (i, j)
    auto SI = [&](int i, int j) { return (j - j0 + 4) * SW + (i - i0 + 4 + sx); };

    pdl_trigger();
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_barrier_init();
        mbar_arrive_expect_tx(bar, (uint32_t)(L::NLOAD * L::BOX_BYTES));
        const int yr = (mem * 3 * NPAN + t) * rows + (j0 - 1), fr = NPAN * rows, mr = j0 - 1;
        tma_load_2d(sH, &tmY, bar, ax, yr);
        tma_load_2d(sU, &tmY, bar, ax, yr + fr);
        tma_load_2d(sV, &tmY, bar, ax, yr + 2 * fr);
        tma_load_2d(sJQ12, &tmM, bar, ax, FM_JQ12 * rows + mr);
        tma_load_2d(sJQ11, &tmM, bar, ax, FM_JQ11Y * rows + mr);
        tma_load_2d(siJy, &tmM, bar, ax, FM_IJY * rows + mr);
        tma_load_2d(sJQ22, &tmM, bar, ax, FM_JQ22X * rows + mr);
        tma_load_2d(siJx, &tmM, bar, ax, FM_IJX * rows + mr);
        tma_load_2d(sF, &tmM, bar, ax, (FM_FJ2 + t) * rows + mr);
        tma_load_2d(siJa, &tmM, bar, ax, FM_IJA * rows + mr);
    }
    // the neighbours' copies of the panel-edge vertices for the gradient SAT
    const bool sat_l = i0 <= SB::NSAT, sat_r = i1 - 1 >= N + 1 - SB::NSAT, sat_b = j0 <= SB::NSAT,
               sat_t = j1 - 1 >= N + 1 - SB::NSAT;
    {
        const T *ym = Yin + (int64_t)mem * d.ms;
        if (warp == 1)
            for (int q = lane; q < th; q += 32) {
                hl[q] = sat_l ? h_halo_cg(ym, d, t, SIDE_L, j0 + q) : T(0);
                hr[q] = sat_r ? h_halo_cg(ym, d, t, SIDE_R, j0 + q) : T(0);
            }
        if (warp == 2)
            for (int q = lane; q < tw; q += 32) {
                hb[q] = sat_b ? h_halo_cg(ym, d, t, SIDE_B, i0 + q) : T(0);
                ht[q] = sat_t ? h_halo_cg(ym, d, t, SIDE_T, i0 + q) : T(0);
            }
    }
    // The five-tap x rows read one input past the interior stencils with weight zero:
    // the slots computed over part of their area start at zero, so that such a tap
    // reads a finite value (the other slots hold loaded or earlier computed data)
    for (int q = threadIdx.x; q < L::SLOT; q += FUSED_THREADS) sVQ[q] = sUQ[q] = sJVT[q] = T(0);
    __syncthreads();
    if (!__syncthreads_and(mbar_wait(bar, 0, FUSED_WAIT_NS))) {
        // the tile loads did not arrive: record it and leave (after one more bounded
        // wait, so that no copy is still writing this block's shared memory)
        if (threadIdx.x == 0) {
            atomicExch(err, 1);
            mbar_wait(bar, 0, FUSED_WAIT_NS);
        }
        return;
    }

    // Every pass below hands each lane one column and each warp a contiguous block of
    // rows.  y stencils slide a four-value window down the column (one shared-memory
    // load per output); x stencils read four neighbours of the row.  Interior rows use
    // the inline interior formula, closure rows the out-of-line closure functions (the
    // row test is warp-uniform; the column test is per lane and fixed for the pass).
    auto rows_of = [&](int la, int lb, int &r0, int &r1) {
        const int R = (lb - la + 7) >> 3;
        r0 = la + warp * R;
        r1 = min(r0 + R, lb);
    };
    // interior rows of the 4-2 interpolations / differences on four taps v0..v3
    auto interp4 = [](T v0, T v1, T v2, T v3) { return (T(9) * (v2 + v1) - (v3 + v0)) * T(0.0625); };
    auto diff4 = [](T v0, T v1, T v2, T v3) { return (T(27) * (v2 - v1) - (v3 - v0)) * T(1.0 / 24.0); };

    // ---- P1: vq = JQ12 I_c2i,y(v) on nodes [i0-3, i1+3) x [j0-1, j1+2);
    //          uq = JQ12 I_c2i,x(u) on nodes [i0-1, i1+2) x [j0-3, j1+3)
    {
        const int ka = max(i0 - 3, 1), kb = min(i1 + 3, n + 1);
        int r0, r1;
        rows_of(max(j0 - 1, 1), min(j1 + 2, n + 1), r0, r1);
        const int k = ka + lane;
        if (k < kb && r0 < r1) {
            const T *col = sV + SI(k, 0), *jq = sJQ12 + SI(k, 0);
            T *out = sVQ + SI(k, 0);
            T f0 = col[(r0 - 2) * SW], f1 = col[(r0 - 1) * SW], f2 = col[r0 * SW];
#pragma unroll 1
            for (int l = r0; l < r1; l++) {
                const T f3 = col[(l + 1) * SW];
                const T v = (l >= 5 && l <= n - 4) ? interp4(f0, f1, f2, f3) : ic2i_cl<T>(l, n, Line<T>{col, SW});
                out[l * SW] = jq[l * SW] * v;
                f0 = f1; f1 = f2; f2 = f3;
            }
        }
    }
    {
        const int ka = max(i0 - 1, 1), kb = min(i1 + 2, n + 1);
        int r0, r1;
        rows_of(max(j0 - 3, 1), min(j1 + 3, n + 1), r0, r1);
        const int k = ka + lane;
        if (k < kb) {
            const XRow<T> xr = xrow42<T>(0, k, n);
            const T *row = sU + SI(xr.base, r0), *jq = sJQ12 + SI(k, r0);
            T *out = sUQ + SI(k, r0);
#pragma unroll 1
            for (int l = r0; l < r1; l++, row += SW, jq += SW, out += SW) *out = *jq * xr.dot(row);
        }
    }
    __syncthreads();

    // ---- P2: J ut = JQ11 u + I_i2c,x(vq) on u points [i0-2, i1+1) x [j0-1, j1+2);
    //          J vt = JQ22 v + I_i2c,y(uq) on v points [i0-1, i1+2) x [j0-2, j1+1)
    {
        const int ia = max(i0 - 2, 1), ib = min(i1 + 1, N + 1);
        int r0, r1;
        rows_of(max(j0 - 1, 1), min(j1 + 2, n + 1), r0, r1);
        const int i = ia + lane;
        if (i < ib) {
            const XRow<T> xr = xrow42<T>(2, i, N);
            const int o0 = SI(i, r0);
            const T *vq = sVQ + SI(xr.base, r0), *u = sU + o0, *jq = sJQ11 + o0;
            T *out = sJUT + o0;
#pragma unroll 1
            for (int j = r0; j < r1; j++, vq += SW, u += SW, jq += SW, out += SW) *out = *jq * *u + xr.dot(vq);
        }
    }
    {
        const int ia = max(i0 - 1, 1), ib = min(i1 + 2, n + 1);
        int r0, r1;
        rows_of(max(j0 - 2, 1), min(j1 + 1, N + 1), r0, r1);
        const int i = ia + lane;
        if (i < ib && r0 < r1) {
            const T *col = sUQ + SI(i, 0), *v = sV + SI(i, 0), *jq = sJQ22 + SI(i, 0);
            T *out = sJVT + SI(i, 0);
            T g0 = col[(r0 - 1) * SW], g1 = col[r0 * SW], g2 = col[(r0 + 1) * SW];
#pragma unroll 1
            for (int j = r0; j < r1; j++) {
                const T g3 = col[(j + 2) * SW];
                const T I = (j >= 4 && j <= N - 3) ? interp4(g0, g1, g2, g3) : ii2c_cl<T>(j, N, Line<T>{col, SW});
                out[j * SW] = jq[j * SW] * v[j * SW] + I;
                g0 = g1; g1 = g2; g2 = g3;
            }
        }
    }
    __syncthreads();

    // ---- RK4 operands of this thread's points (tile column i0 + lane, the warp's block
    // of tile rows), in flight during P3
    constexpr bool LV = MODE >= 1, LA = MODE >= 2, LC = (sizeof(T) == 4) && MODE == 4;
    const int64_t po = (int64_t)mem * d.ms + (int64_t)t * d.ps;
    const int64_t fs = d.fs;
    const int ip = i0 + lane;
    int q0, q1;
    rows_of(j0, j1, q0, q1);
    T pv[3][L::MR], pa[3][L::MR], pc[3][L::MR];
#pragma unroll
    for (int m = 0; m < L::MR; m++) {
        const int j = q0 + m;
        const bool ok = lane < tw && j < q1;
        const bool has[3] = {ok, ok && ip <= N, ok && j <= N};
        const int o = box_off32(P, ip, j);
#pragma unroll
        for (int f = 0; f < 3; f++) {
            pv[f][m] = LV && has[f] ? V0[po + o + f * fs] : T(0);
            pa[f][m] = LA && has[f] ? ACC[po + o + f * fs] : T(0);
            pc[f][m] = LC && has[f] ? CMP[po + o + f * fs] : T(0);
        }
    }

    // ---- P3: the Coriolis vertex vectors and the divergence away from the panel
    // boundary (its vertices take the synchronised values below)
    {
        // up = fJ2 I_c2i,y(vt) on [i0-1, i1+2) x [j0, j1), vt = J vt / J
        const int ka = max(i0 - 1, 1), kb = min(i1 + 2, n + 1);
        int r0, r1;
        rows_of(j0, j1, r0, r1);
        const int k = ka + lane;
        if (k < kb && k != 1 && k != n && r0 < r1) {
            const T *cj = sJVT + SI(k, 0), *ci = siJx + SI(k, 0), *fj = sF + SI(k, 0);
            T *out = sUP + SI(k, 0);
            T f0 = cj[(r0 - 2) * SW] * ci[(r0 - 2) * SW], f1 = cj[(r0 - 1) * SW] * ci[(r0 - 1) * SW],
              f2 = cj[r0 * SW] * ci[r0 * SW];
#pragma unroll 1
            for (int l = r0; l < r1; l++) {
                const T f3 = cj[(l + 1) * SW] * ci[(l + 1) * SW];
                if (l != 1 && l != n) {
                    const T v = (l >= 5 && l <= n - 4) ? interp4(f0, f1, f2, f3)
                                                       : ic2i_cl2<T>(l, n, Line2<T>{cj, ci, SW});
                    out[l * SW] = fj[l * SW] * v;
                }
                f0 = f1; f1 = f2; f2 = f3;
            }
        }
    }
    {
        // vp = -fJ2 I_c2i,x(ut) on [i0, i1) x [j0-1, j1+2), ut = J ut / J
        int r0, r1;
        rows_of(max(j0 - 1, 1), min(j1 + 2, n + 1), r0, r1);
        const int k = i0 + lane;
        if (lane < tw && k != 1 && k != n) {
            const XRow<T> xr = xrow42<T>(0, k, n);
            const int o0 = SI(k, r0), ob = SI(xr.base, r0);
            const T *rj = sJUT + ob, *ri = siJy + ob, *fj = sF + o0;
            T *out = sVP + o0;
#pragma unroll 1
            for (int l = r0; l < r1; l++, rj += SW, ri += SW, fj += SW, out += SW) {
                if (l == 1 || l == n) continue;
                *out = -*fj * xr.dot2(rj, ri);
            }
        }
    }
    {
        // div = (D_c2i,x(J ut) / hx + D_c2i,y(J vt) / hx) / (J a) on the tile
        int r0, r1;
        rows_of(j0, j1, r0, r1);
        const int k = i0 + lane;
        if (lane < tw && k != 1 && k != n && r0 < r1) {
            const XRow<T> xr = xrow42<T>(1, k, n);
            const T *cj = sJVT + SI(k, 0), *ia = siJa + SI(k, 0);
            const T *rj = sJUT + SI(xr.base, r0);
            T *out = sDIV + SI(k, 0);
            T f0 = cj[(r0 - 2) * SW], f1 = cj[(r0 - 1) * SW], f2 = cj[r0 * SW];
#pragma unroll 1
            for (int l = r0; l < r1; l++, rj += SW) {
                const T f3 = cj[(l + 1) * SW];
                if (l != 1 && l != n) {
                    const T dx = xr.dot(rj);
                    const T dy = (l >= 5 && l <= n - 4) ? diff4(f0, f1, f2, f3) : dc2i_cl<T>(l, n, Line<T>{cj, SW});
                    out[l * SW] = (dx * fm.inv_hx + dy * fm.inv_hx) * ia[l * SW];
                }
                f0 = f1; f1 = f2; f2 = f3;
            }
        }
    }
    // ---- P4: tiles on a panel edge wait for the edge sync and take the synchronised
    // (up, vp, div) of the panel-boundary vertices
    if (i0 == 1 || i1 == n + 1 || j0 == 1 || j1 == n + 1) {
        pdl_wait();
        // up: columns [i0-1, i1+2) x rows [j0, j1); vp: [i0, i1) x [j0-1, j1+2); div: the tile.
        // Task q: array q / 160, boundary line (q / 40) % 4 (columns 1, n, rows 1, n), offset q % 40
        // along it (every range is at most TH + 3 <= 36 long).
        const int ua = max(i0 - 1, 1), ub = min(i1 + 2, n + 1), va = max(j0 - 1, 1), vb = min(j1 + 2, n + 1);
        for (int q = threadIdx.x; q < 3 * 4 * 40; q += FUSED_THREADS) {
            const int which = q / 160, c = (q / 40) % 4, e = q % 40;
            const int ka = which == 0 ? ua : i0, kb = which == 0 ? ub : i1;
            const int la = which == 1 ? va : j0, lb = which == 1 ? vb : j1;
            int k, l;
            if (c < 2) {
                k = c == 0 ? 1 : n;
                l = la + e;
                if (k < ka || k >= kb || l >= lb) continue;
            } else {
                l = c == 2 ? 1 : n;
                k = ka + e;
                if (l < la || l >= lb || k >= kb) continue;
            }
            T *dst = which == 0 ? sUP : (which == 1 ? sVP : sDIV);
            dst[SI(k, l)] = ld_cg(edge_entry(E, N, mem, t, k, l) + which);
        }
    }
    __syncthreads();

    // ---- P5: the tendencies of the tile's points and the RK4 update
    const T H = T(a.Hm[mem]);
    const T dt = T(a.dtm ? a.dtm[mem] : a.dt);
    T *v0 = V0 + po, *y1 = Y1 + po, *acc = ACC + po;
    T *cmp = CMP ? CMP + po : nullptr;
    if (lane < tw && q0 < q1) {
        const int i = ip;
        const bool iu = i <= N;
        // x rows of the u points: the nodes->centres difference of h and interpolation of up
        const XRow<T> xd = xrow42<T>(3, iu ? i : N, N), xi = xrow42<T>(2, iu ? i : N, N);
        const T *hc = sH + SI(i, 0), *pc_ = sVP + SI(i, 0);
        // y windows of h (rows j-1 .. j+2) and vp
        T h0 = hc[(q0 - 1) * SW], h1 = hc[q0 * SW], h2 = hc[(q0 + 1) * SW];
        T p0 = pc_[(q0 - 1) * SW], p1 = pc_[q0 * SW], p2 = pc_[(q0 + 1) * SW];
#pragma unroll
        for (int m = 0; m < L::MR; m++) {
            const int j = q0 + m;
            if (j >= q1) break;
            const T h3 = hc[(j + 2) * SW], p3 = pc_[(j + 2) * SW];
            const int so = SI(i, j);
            T k3[3];
            k3[0] = -H * sDIV[so];
            k3[1] = T(0);
            k3[2] = T(0);
            if (iu) {
                const T *hr_ = sH + so;
                T gx = xd.dot(sH + SI(xd.base, j));
                const T cu = xi.dot(sUP + SI(xi.base, j));
                if (i <= SB::NSAT) gx += T(SB::satw(i)) * (hr_[1 - i] - hl[j - j0]);
                if (i >= N + 1 - SB::NSAT) gx += T(SB::satw(N + 1 - i)) * (hr[j - j0] - hr_[n - i]);
                k3[1] = -fm.grav * (gx * fm.inv_hxa) + cu * siJy[so];
            }
            if (j <= N) {
                const bool jin = j >= 4 && j <= N - 3;
                T gy = jin ? diff4(h0, h1, h2, h3) : di2c_cl<T>(j, N, Line<T>{hc, SW});
                const T cv = jin ? interp4(p0, p1, p2, p3) : ii2c_cl<T>(j, N, Line<T>{pc_, SW});
                if (j <= SB::NSAT) gy += T(SB::satw(j)) * (hc[SW] - hb[lane]);
                if (j >= N + 1 - SB::NSAT) gy += T(SB::satw(N + 1 - j)) * (ht[lane] - hc[n * SW]);
                gy = gy * fm.inv_hxa;
                k3[2] = -fm.grav * gy + cv * siJx[so];
            }
            h0 = h1; h1 = h2; h2 = h3;
            p0 = p1; p1 = p2; p2 = p3;
            const int o = box_off32(P, i, j);
            const bool has[3] = {true, iu, j <= N};
#pragma unroll
            for (int f = 0; f < 3; f++) {
                if (!has[f]) continue;
                const int64_t of = o + f * fs;
                if constexpr (MODE == 0) {
                    y1[of] = k3[f];
                } else if constexpr (MODE <= 3) {
                    const T ca = (MODE == 3) ? dt : T(0.5) * dt;
                    const T cb = (MODE == 1) ? dt / T(6) : dt / T(3);
                    y1[of] = pv[f][m] + ca * k3[f];
                    acc[of] = (MODE == 1) ? cb * k3[f] : pa[f][m] + cb * k3[f];
                } else if constexpr (sizeof(T) == 4) {
                    float sv = pv[f][m], cv_ = pc[f][m];
                    kahan_add(sv, cv_, pa[f][m] + (dt / T(6)) * k3[f]);
                    v0[of] = sv;
                    cmp[of] = cv_;
                } else {
                    v0[of] = pv[f][m] + (pa[f][m] + (dt / T(6)) * k3[f]);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// The edge strips straight from the stage input.
// ---------------------------------------------------------------------------
// Side coordinates of side s: across index x (1 at the edge), along index y.
//   node (x, y)  -> (i, j): L (x, y), R (n+1-x, y), B (y, x), T (y, n+1-x)
//   NF, the covariant component normal to the side (u on L/R, v on B/T), at
//       across centre x, along node y:  L u(x, y), R u(n-x, y), B v(y, x), T v(y, n-x)
//   TF, the tangential component (v on L/R, u on B/T), at across node x, along centre c
// With tq(x, y) = JQ12 I_c2i,along(TF(x, .))(y) and nq(y) = JQ12 I_c2i,across(NF(., y))(1)
// (the first closure row), the strip lines are
//   normal(dd, y)  = (JQn NF + I_i2c,across(tq(., y))(dd)) / Jn,   dd = 1..3
//   tangential(c)  = (JQt TF(1, c) + I_i2c,along(nq)(c)) / Jt
// the values k_fstage computes for the same points.  The across stencils at the far
// sides R and T are the mirrored closure rows (the interpolations are symmetric
// under the reversal of their inputs).
constexpr int STRIP_CHUNK = 64;     // along-edge nodes per block
constexpr int STRIP_THREADS = 128;
constexpr int STRIP_BL = STRIP_CHUNK + 8;   // band length along the side

template <class T>
__global__ void __launch_bounds__(STRIP_THREADS) k_strip(const T *__restrict__ Y, T *__restrict__ ES, Dims d,
                                                         FusedMetric<T> fm, const double *__restrict__ dtm)
{
    using SB = SbpOrder<42>;
    constexpr int XN = 5, ND = SB::NDEP, NL = ND + 1;
    constexpr int NT = NL * STRIP_CHUNK / STRIP_THREADS;                      // output tasks per thread
    constexpr int NB1 = (XN * STRIP_BL + STRIP_THREADS - 1) / STRIP_THREADS;  // band loads per thread
    constexpr int NB2 = (ND * STRIP_BL + STRIP_THREADS - 1) / STRIP_THREADS;
    __shared__ T tf[XN][STRIP_BL];    // TF at across nodes 1..XN, along centres y0 ..
    __shared__ T nf[ND][STRIP_BL];    // NF at across centres 1..ND, along nodes y0 ..
    __shared__ T jq[XN][STRIP_BL];    // JQ12 at across nodes 1..XN, along nodes y0 ..
    __shared__ T tq[XN][STRIP_CHUNK]; // tq at across nodes 1..XN, along nodes b0 ..
    __shared__ T nq[STRIP_BL];        // nq along nodes y0 ..
    const int N = d.N, n = N + 1, P = d.P;
    const int s = blockIdx.y & 3, t = blockIdx.y >> 2, mem = blockIdx.z;
    const int b0 = 1 + blockIdx.x * STRIP_CHUNK, b1 = min(b0 + STRIP_CHUNK, n + 1);
    const int y0 = b0 - 4;   // band origin along the side
    const bool lr = s <= SIDE_R, far = (s == SIDE_R || s == SIDE_T);
    const int64_t box = d.ps;
    const T *mJQ12 = fm.base + FM_JQ12 * box, *mJQn = fm.base + (lr ? FM_JQ11Y : FM_JQ22X) * box,
            *miJn = fm.base + (lr ? FM_IJY : FM_IJX) * box, *mJQt = fm.base + (lr ? FM_JQ22X : FM_JQ11Y) * box,
            *miJt = fm.base + (lr ? FM_IJX : FM_IJY) * box;
    // panel offsets of side coordinates: node (x, y) (also the TF point at across node
    // x, along centre y) and across-centre (x, y)
    auto node_off = [&](int x, int y) {
        const int xx = far ? n + 1 - x : x;
        return lr ? box_off32(P, xx, y) : box_off32(P, y, xx);
    };
    auto cen_off = [&](int x, int y) {
        const int xx = far ? n - x : x;
        return lr ? box_off32(P, xx, y) : box_off32(P, y, xx);
    };
    // ---- static data first (before the previous stage completes): the JQ12 band and
    // the metric of this thread's outputs (task q: line q / CHUNK, along b0 + q % CHUNK)
    T rj[NB1], mq[NT], mi[NT];
#pragma unroll
    for (int r = 0; r < NB1; r++) {
        const int q = threadIdx.x + r * STRIP_THREADS, x = 1 + q / STRIP_BL, y = y0 + q % STRIP_BL;
        rj[r] = (q < XN * STRIP_BL && y >= 1 && y <= n) ? __ldg(mJQ12 + node_off(x, y)) : T(0);
    }
#pragma unroll
    for (int r = 0; r < NT; r++) {
        const int q = threadIdx.x + r * STRIP_THREADS, line = q / STRIP_CHUNK, y = b0 + q % STRIP_CHUNK;
        mq[r] = mi[r] = T(0);
        if (y < b1 && line < ND) {
            const int o = cen_off(line + 1, y);
            mq[r] = __ldg(mJQn + o);
            mi[r] = __ldg(miJn + o);
        } else if (y < b1 && y <= N) {
            const int o = node_off(1, y);
            mq[r] = __ldg(mJQt + o);
            mi[r] = __ldg(miJt + o);
        }
    }
    pdl_wait();
    pdl_trigger();
    if (member_frozen(dtm, mem)) return;
    const T *yp = Y + (int64_t)mem * d.ms + (int64_t)t * d.ps;
    const T *gNF = yp + (lr ? 1 : 2) * d.fs, *gTF = yp + (lr ? 2 : 1) * d.fs;
    // ---- the band of the stage input, every load issued before the first store
    T rt[NB1], rn[NB2];
#pragma unroll
    for (int r = 0; r < NB1; r++) {
        const int q = threadIdx.x + r * STRIP_THREADS, x = 1 + q / STRIP_BL, y = y0 + q % STRIP_BL;
        rt[r] = (q < XN * STRIP_BL && y >= 1 && y <= N) ? ld_cg(gTF + node_off(x, y)) : T(0);
    }
#pragma unroll
    for (int r = 0; r < NB2; r++) {
        const int q = threadIdx.x + r * STRIP_THREADS, x = 1 + q / STRIP_BL, y = y0 + q % STRIP_BL;
        rn[r] = (q < ND * STRIP_BL && y >= 1 && y <= n) ? ld_cg(gNF + cen_off(x, y)) : T(0);
    }
#pragma unroll
    for (int r = 0; r < NB1; r++) {
        const int q = threadIdx.x + r * STRIP_THREADS;
        if (q < XN * STRIP_BL) {
            (&tf[0][0])[q] = rt[r];
            (&jq[0][0])[q] = rj[r];
        }
    }
#pragma unroll
    for (int r = 0; r < NB2; r++) {
        const int q = threadIdx.x + r * STRIP_THREADS;
        if (q < ND * STRIP_BL) (&nf[0][0])[q] = rn[r];
    }
    __syncthreads();
    // ---- tq on the chunk, nq on the band
    for (int q = threadIdx.x; q < XN * STRIP_CHUNK; q += STRIP_THREADS) {
        const int x = 1 + q / STRIP_CHUNK, y = b0 + q % STRIP_CHUNK;
        if (y >= b1) continue;
        const Line<T> line{&tf[x - 1][0] - y0, 1};
        tq[x - 1][y - b0] = jq[x - 1][y - y0] * f_ic2i<T>(y, n, line);
    }
    for (int q = threadIdx.x; q < STRIP_BL; q += STRIP_THREADS) {
        const int y = y0 + q;
        T v = T(0);
        if (y >= 1 && y <= n) {
            v = T(SB::ic1(1)) * nf[0][q];
#pragma unroll
            for (int dd = 2; dd <= ND; dd++) v += T(SB::ic1(dd)) * nf[dd - 1][q];
            v = jq[0][q] * v;
        }
        nq[q] = v;
    }
    __syncthreads();
    // ---- the strip lines: es[(s NL + line) n + b], b 1-based
    T *es = ES + strip_member(N, mem, NL) + (int64_t)t * 4 * NL * n - 1;
#pragma unroll
    for (int r = 0; r < NT; r++) {
        const int q = threadIdx.x + r * STRIP_THREADS, line = q / STRIP_CHUNK, y = b0 + q % STRIP_CHUNK;
        if (y >= b1) continue;
        T val;
        if (line < ND) {
            const Line<T> across{&tq[0][y - b0] - STRIP_CHUNK, STRIP_CHUNK};   // across(x) = tq[x-1][y-b0]
            val = (mq[r] * nf[line][y - y0] + f_ii2c<T>(line + 1, N, across)) * mi[r];
        } else {
            if (y > N) continue;
            const Line<T> along{&nq[0] - y0, 1};
            val = (mq[r] * tf[0][y - y0] + f_ii2c<T>(y, N, along)) * mi[r];
        }
        es[(s * NL + line) * n + y] = val;
    }
}

}  // namespace chswe
