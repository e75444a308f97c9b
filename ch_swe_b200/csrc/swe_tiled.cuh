// swe_tiled.cuh -- the per-stage stencil kernels, shared-memory tiled.
//
// A block of 256 threads owns a tile [i0, i1) x [j0, j1) of the (N+1) x (N+1)
// box of one panel of one member.  Tiles are balanced: gridDim.x tiles split the
// N+1 columns into widths floor/ceil((N+1)/gridDim.x) <= TM, likewise rows, so
// N+1 = (TM-1)k+1 gives no one-column slivers.  TM (odd) is a template
// parameter; the host picks it per cube size (autotuned).  The block copies the windows it
// needs (tile plus stencil footprint) from the zero-margined panel boxes into
// shared memory without bounds checks and evaluates the SBP stencils there.
//
// Every stencil pass is laid out so that its closure branch is warp-uniform:
// y-direction stencils run in row-major passes (consecutive lanes = consecutive
// columns of one row), x-direction stencils in column-major passes (consecutive
// lanes = consecutive rows of one column).  Shared-memory windows have odd
// pitches, so column-major passes are free of bank conflicts.  Panel-boundary
// vertices take their synchronised values from the edge buffer written by k_edge.
//
// Footprints: a nodes->centres stencil for outputs [a, b) reads inputs
// [a-2, b+3); a centres->nodes stencil reads [a-3, b+2) (closure rows included).
#pragma once

#include "swe_kernels.cuh"
#include "swe_advective.cuh"

#include <cuda_pipeline.h>

namespace chswe {

// Tiles of at most TM x TM points, ceil(N / (TM - 1)) of them per direction.
template <int TM>
struct Tile {
    static_assert(TM % 2 == 1, "odd shared-memory pitches need an odd maximal tile");
    static constexpr int XN = TM - 1;   // nominal width
    static constexpr int PW = TM + 6;   // odd pitch of (tile + 5)-wide windows
    static constexpr int PT = TM;       // odd pitch of tile-wide windows
    static constexpr int RW = TM + 5;   // rows of (tile + 5)-high windows
    // trip bounds of the flattened passes: (tile+5)^2 windows, (tile+5) x tile strips, tile^2
    static constexpr int IT_WIN = ((TM + 5) * (TM + 5) + STAGE_THREADS - 1) / STAGE_THREADS;
    static constexpr int IT_STRIP = ((TM + 5) * TM + STAGE_THREADS - 1) / STAGE_THREADS;
    static constexpr int IT_TILE = (TM * TM + STAGE_THREADS - 1) / STAGE_THREADS;
    // run-blocked kernel variant: runs of RBW (passes over tile + 5 cross lines) or RBT
    // (tile cross lines) outputs along the stencil direction, the longest runs that
    // keep every pass within one item per thread
    static constexpr int RBW = TM == 17 ? 2 : (TM == 25 ? 4 : 6);
    static constexpr int RBT = TM == 17 ? 2 : (TM == 25 ? 3 : 5);
};

// RUNS = false gives runs of one output: the flat element-per-thread passes.
#define CHSWE_TILE_CONSTANTS(TM, RUNS)                                                                     \
    constexpr int PW = Tile<TM>::PW, PT = Tile<TM>::PT, RW = Tile<TM>::RW, IT_WIN = Tile<TM>::IT_WIN,      \
                  IT_STRIP = Tile<TM>::IT_STRIP, RBW = (RUNS) ? Tile<TM>::RBW : 1,                          \
                  RBT = (RUNS) ? Tile<TM>::RBT : 1,                                                         \
                  IT_RW = ((TM + 5) * ((TM + RBW - 1) / RBW) + STAGE_THREADS - 1) / STAGE_THREADS,          \
                  IT_RT = (TM * ((TM + RBT - 1) / RBT) + STAGE_THREADS - 1) / STAGE_THREADS;                \
    (void)RW

// The block a tile kernel works on: tile (x, y) of gx x gy tiles per panel, z = member *
// 6 + panel.  A plain launch takes it from its grid; a group launch (one grid over the
// states of several contexts) decodes it from its flat block index.
struct Blk {
    unsigned x, y, z, gx, gy;
};
__device__ __forceinline__ Blk grid_blk() { return Blk{blockIdx.x, blockIdx.y, blockIdx.z, gridDim.x, gridDim.y}; }

__device__ __forceinline__ void tile_range(const Blk &b, int n, int &i0, int &i1, int &j0, int &j1)
{
    i0 = 1 + (b.x * n) / b.gx;
    i1 = 1 + ((b.x + 1) * n) / b.gx;
    j0 = 1 + (b.y * n) / b.gy;
    j1 = 1 + ((b.y + 1) * n) / b.gy;
}

// q -> (a, b) with q = a * w + b, 0 <= b < w (q < 2^16, w <= 64): exact with a float reciprocal.
__device__ __forceinline__ void split(int q, int w, float inv_w, int &a, int &b)
{
    a = __float2int_rz(((float)q + 0.5f) * inv_w);
    b = q - a * w;
}

// Shared-memory window of pitch NP with origin (x0, y0) (1-based indices).
template <class T, int NP>
struct SWin {
    T *a;
    int x0, y0;
    __device__ __forceinline__ T &at(int i, int j) const { return a[(j - y0) * NP + (i - x0)]; }
    __device__ __forceinline__ Line<T> row(int j) const { return Line<T>{a + (j - y0) * NP - x0, 1}; }
    __device__ __forceinline__ Line<T> col(int i) const { return Line<T>{a + (i - x0) - y0 * NP, NP}; }
};

// The four operators at one output: the interior rows inline, the closure rows
// through the general functions of swe_sbp.cuh (SbpOrder<ORD>).
template <class T, int ORD = 42> __device__ __forceinline__ T ic2i_u(int k, int nx, const Line<T> &f)
{
    using S = SbpOrder<ORD>;
    return (k >= S::C2I_LO && k <= nx - S::C2I_HI) ? S::template ic2i_in<T>(k, f) : S::template ic2i<T>(k, nx, f);
}
template <class T, int ORD = 42> __device__ __forceinline__ T ii2c_u(int k, int n, const Line<T> &f)
{
    using S = SbpOrder<ORD>;
    return (k >= S::I2C_LO && k <= n - S::I2C_HI) ? S::template ii2c_in<T>(k, f) : S::template ii2c<T>(k, n, f);
}
template <class T, int ORD = 42> __device__ __forceinline__ T dc2i_u(int k, int nx, const Line<T> &f)
{
    using S = SbpOrder<ORD>;
    return (k >= S::C2I_LO && k <= nx - S::C2I_HI) ? S::template dc2i_in<T>(k, f) : S::template dc2i<T>(k, nx, f);
}
template <class T, int ORD = 42> __device__ __forceinline__ T di2c_u(int k, int n, const Line<T> &f)
{
    using S = SbpOrder<ORD>;
    return (k >= S::I2C_LO && k <= n - S::I2C_HI) ? S::template di2c_in<T>(k, f) : S::template di2c<T>(k, n, f);
}

// Stencil runs.  A pass gives every thread whole runs of RB consecutive outputs
// along the stencil direction at one cross index; lanes take consecutive cross
// indices, so shared-memory accesses are conflict-free (odd pitches) and the closure
// tests are warp-uniform.  A run clear of the SBP closures loads its RB + 3 inputs
// once and evaluates the interior rows on registers; other runs (closures, or
// shorter than RB at the end of a tile) go output by output.  RB = 1 is the flat
// one-output-per-element form.
// v[m] = f(k0 + O + m): O = -2 for the centres->nodes rows (taps k-2..k+1), O = -1
// for the nodes->centres rows (taps k-1..k+2); the interior formulas then coincide.
template <class T, int RB, int O>
__device__ __forceinline__ void run_load(const Line<T> &f, int k0, T (&v)[RB + 3])
{
#pragma unroll
    for (int m = 0; m < RB + 3; m++) v[m] = f(k0 + O + m);
}
template <class T, int RB, int ORD>
__device__ __forceinline__ T run_interp(const T (&v)[RB + 3], int m)
{
    return SbpOrder<ORD>::template interp4<T>(v[m], v[m + 1], v[m + 2], v[m + 3]);
}
template <class T, int RB, int ORD>
__device__ __forceinline__ T run_diff(const T (&v)[RB + 3], int m)
{
    return SbpOrder<ORD>::template diff4<T>(v[m], v[m + 1], v[m + 2], v[m + 3]);
}

// Every global load of a pass is issued into registers before the first
// shared-memory store or stencil of that pass (fixed-trip unrolled loops), so a
// block pays one memory round trip per batch instead of one per loop iteration.

// ---------------------------------------------------------------------------
// contravariant components (co2contra_Ch_mod.f90:27-94)
//   ut = Qi11 u + J^-1 I_i2c,x( J Qi12 I_c2i,y(v) ),  vt = Qi22 v + J^-1 I_i2c,y( J Qi12 I_c2i,x(u) )
// ---------------------------------------------------------------------------
template <class T, int TM>
struct Co2Layout {
    static constexpr int PW = Tile<TM>::PW, PT = Tile<TM>::PT, RW = Tile<TM>::RW;
    static constexpr int V = 0, U = V + PW * RW, VQ = U + PW * RW, UQ = VQ + PW * TM, UX = UQ + PT * RW,
                         TOTAL = UX + PT * TM;
    static constexpr size_t bytes() { return sizeof(T) * TOTAL; }
};

// OCC: resident blocks per SM the register allocation is capped for; RUNS: stencil
// runs of several outputs per thread (both autotuned).
template <class T, int TM, int OCC, bool RUNS, int ORD>
__device__ __forceinline__ void co2contra_tile(const Blk &bk, const T *__restrict__ Y, T *__restrict__ W,
                                               T *__restrict__ ES, const Dims &d, const MetricView<T> &m,
                                               const double *__restrict__ dtm)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    using L = Co2Layout<T, TM>;
    CHSWE_TILE_CONSTANTS(TM, RUNS);
    using SB = SbpOrder<ORD>;
    T *sm = reinterpret_cast<T *>(smraw);
    const int N = d.N, n = N + 1, P = d.P;
    int i0, i1, j0, j1;
    tile_range(bk, n, i0, i1, j0, j1);
    const int tw = i1 - i0, th = j1 - j0, w5 = tw + 5, h5 = th + 5;
    const float iw5 = 1.0f / (float)w5, ih5 = 1.0f / (float)h5, iw = 1.0f / (float)tw, ih = 1.0f / (float)th;
    const int t = bk.z % NPAN, mem = bk.z / NPAN;
    if (member_frozen(dtm, mem)) return;
    const T *y = Y + mem * d.ms + t * d.ps;
    T *w = W + mem * d.ms + t * d.ps;
    constexpr int NDEP = SB::NDEP, NL = NDEP + 1;   // normal depths and lines per side of the strips
    T *es = ES + strip_member(N, mem, NL) + (int64_t)t * 4 * NL * n - 1;   // + (s*NL + line)*n + index
    const SWin<T, PW> sv{sm + L::V, i0 - 2, j0 - 3}, su{sm + L::U, i0 - 3, j0 - 2}, svq{sm + L::VQ, i0 - 2, j0};
    const SWin<T, PT> suq{sm + L::UQ, i0, j0 - 2}, sux{sm + L::UX, i0, j0};

    // runs along the tile width / height: window passes (RBW), tile passes (RBT)
    const int nww = (tw + RBW - 1) / RBW, nhw = (th + RBW - 1) / RBW, nwt = (tw + RBT - 1) / RBT,
              nht = (th + RBT - 1) / RBT;

    // ---- before the predecessor grid completes: J Qi12 at both xy intermediates (metric only)
    pdl_trigger();
    T jq1[IT_RW][RBW], jq2[IT_STRIP];
#pragma unroll
    for (int it = 0; it < IT_RW; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, x;
        split(q, w5, iw5, r, x);
        const int l0 = j0 + r * RBW;
#pragma unroll
        for (int mm = 0; mm < RBW; mm++)
            jq1[it][mm] = q < w5 * nhw && l0 + mm < j1 ? __ldg(m.JQ12 + box_off(P, sv.x0 + x, l0 + mm)) : T(0);
    }
#pragma unroll
    for (int it = 0; it < IT_STRIP; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, c;
        split(q, tw, iw, r, c);
        jq2[it] = q < tw * h5 ? __ldg(m.JQ12 + box_off(P, i0 + c, suq.y0 + r)) : T(0);
    }
    pdl_wait();
    // ---- batch 1: v and u windows
    {
        const T *gv = y + 2 * d.fs + box_off(P, sv.x0, sv.y0), *gu = y + d.fs + box_off(P, su.x0, su.y0);
        T rv[IT_WIN], ru[IT_WIN];
#pragma unroll
        for (int it = 0; it < IT_WIN; it++) {
            const int q = threadIdx.x + it * STAGE_THREADS;
            int r, c;
            split(q, w5, iw5, r, c);
            const bool ok = q < w5 * h5;
            rv[it] = ok ? __ldg(gv + r * P + c) : T(0);
            ru[it] = ok ? __ldg(gu + r * P + c) : T(0);
        }
#pragma unroll
        for (int it = 0; it < IT_WIN; it++) {
            const int q = threadIdx.x + it * STAGE_THREADS;
            int r, c;
            split(q, w5, iw5, r, c);
            if (q < w5 * h5) {
                sv.a[r * PW + c] = rv[it];
                su.a[r * PW + c] = ru[it];
            }
        }
    }
    // ---- batch 2 (in flight during the passes): the output metric, by output run
    T q11[IT_RT][RBT], ijy[IT_RT][RBT], q22[IT_RT][RBT], ijx[IT_RT][RBT];
#pragma unroll
    for (int it = 0; it < IT_RT; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, x;
        split(q, tw, iw, r, x);
        const int i = i0 + x, jr = j0 + r * RBT;
#pragma unroll
        for (int mm = 0; mm < RBT; mm++) {
            const int j = jr + mm;
            const int64_t o = box_off(P, i, j);
            const bool ok = q < tw * nht && j < j1;
            q11[it][mm] = ok && i <= N ? __ldg(m.Q11y + o) : T(0);
            ijy[it][mm] = ok && i <= N ? __ldg(m.iJy + o) : T(0);
            q22[it][mm] = ok && j <= N ? __ldg(m.Q22x + o) : T(0);
            ijx[it][mm] = ok && j <= N ? __ldg(m.iJx + o) : T(0);
        }
    }
    __syncthreads();
    // J Qi12 I_c2i,y(v) at xy nodes: columns of the window, runs along the tile rows
#pragma unroll
    for (int it = 0; it < IT_RW; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, x;
        split(q, w5, iw5, r, x);
        if (q >= w5 * nhw) continue;
        const int k = sv.x0 + x, l0 = j0 + r * RBW, cnt = min(RBW, j1 - l0);
        const Line<T> col = sv.col(k);
        T *o = &svq.at(k, l0);
        if (SB::RUN_OK && cnt == RBW && l0 >= SB::C2I_LO && l0 + RBW - 1 <= n - SB::C2I_HI) {
            T v[RBW + 3];
            run_load<T, RBW, -2>(col, l0, v);
#pragma unroll
            for (int mm = 0; mm < RBW; mm++) o[mm * PW] = run_interp<T, RBW, ORD>(v, mm) * jq1[it][mm];
        } else {
#pragma unroll
            for (int mm = 0; mm < RBW; mm++)
                if (mm < cnt) o[mm * PW] = ic2i_u<T, ORD>(l0 + mm, n, col) * jq1[it][mm];
        }
    }
    // I_c2i,x(u) at xy nodes: rows of the window, runs along the tile columns; the
    // J Qi12 factor follows
#pragma unroll
    for (int it = 0; it < IT_RW; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, x;
        split(q, h5, ih5, r, x);
        if (q >= h5 * nww) continue;
        const int l = suq.y0 + x, k0 = i0 + r * RBW, cnt = min(RBW, i1 - k0);
        const Line<T> row = su.row(l);
        T *o = &suq.at(k0, l);
        if (SB::RUN_OK && cnt == RBW && k0 >= SB::C2I_LO && k0 + RBW - 1 <= n - SB::C2I_HI) {
            T v[RBW + 3];
            run_load<T, RBW, -2>(row, k0, v);
#pragma unroll
            for (int mm = 0; mm < RBW; mm++) o[mm] = run_interp<T, RBW, ORD>(v, mm);
        } else {
#pragma unroll
            for (int mm = 0; mm < RBW; mm++)
                if (mm < cnt) o[mm] = ic2i_u<T, ORD>(k0 + mm, n, row);
        }
    }
    __syncthreads();
    // I_i2c,x of the first: tile rows, runs along the tile columns (u points, i <= N)
    const int iu1 = min(i1, n);
#pragma unroll
    for (int it = 0; it < IT_RT; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, x;
        split(q, th, ih, r, x);
        if (q >= th * nwt) continue;
        const int j = j0 + x, k0 = i0 + r * RBT, cnt = min(RBT, iu1 - k0);
        const Line<T> row = svq.row(j);
        T *o = &sux.at(k0, j);
        if (SB::RUN_OK && cnt == RBT && k0 >= SB::I2C_LO && k0 + RBT - 1 <= N - SB::I2C_HI) {
            T v[RBT + 3];
            run_load<T, RBT, -1>(row, k0, v);
#pragma unroll
            for (int mm = 0; mm < RBT; mm++) o[mm] = run_interp<T, RBT, ORD>(v, mm);
        } else {
#pragma unroll
            for (int mm = 0; mm < RBT; mm++)
                if (mm < cnt) o[mm] = ii2c_u<T, ORD>(k0 + mm, N, row);
        }
    }
    // J Qi12 factor of the second: row-major, in place
#pragma unroll
    for (int it = 0; it < IT_STRIP; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, c;
        split(q, tw, iw, r, c);
        if (q < tw * h5) suq.at(i0 + c, suq.y0 + r) *= jq2[it];
    }
    __syncthreads();
    // outputs: tile columns, runs along the tile rows (I_i2c,y of the second); lanes
    // store consecutive columns of a row (coalesced)
#pragma unroll
    for (int it = 0; it < IT_RT; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, x;
        split(q, tw, iw, r, x);
        if (q >= tw * nht) continue;
        const int i = i0 + x, jr = j0 + r * RBT, cnt = min(RBT, j1 - jr);
        const Line<T> col = suq.col(i);
        T vi[RBT];
        if (SB::RUN_OK && cnt == RBT && jr >= SB::I2C_LO && jr + RBT - 1 <= N - SB::I2C_HI) {
            T v[RBT + 3];
            run_load<T, RBT, -1>(col, jr, v);
#pragma unroll
            for (int mm = 0; mm < RBT; mm++) vi[mm] = run_interp<T, RBT, ORD>(v, mm);
        } else {
#pragma unroll
            for (int mm = 0; mm < RBT; mm++) vi[mm] = (mm < cnt && jr + mm <= N) ? ii2c_u<T, ORD>(jr + mm, N, col) : T(0);
        }
#pragma unroll
        for (int mm = 0; mm < RBT; mm++) {
            if (mm >= cnt) continue;
            const int j = jr + mm;
            const int64_t o = box_off(P, i, j);
            // the edge strips (k_edge reads them contiguous along each side)
            if (i <= N) {
                const T ut = q11[it][mm] * su.at(i, j) + sux.at(i, j) * ijy[it][mm];
                w[d.fs + o] = ut;
                if (i <= NDEP) es[(SIDE_L * NL + i - 1) * n + j] = ut;
                if (i >= N + 1 - NDEP) es[(SIDE_R * NL + N - i) * n + j] = ut;
                if (j == 1) es[(SIDE_B * NL + NL - 1) * n + i] = ut;
                if (j == n) es[(SIDE_T * NL + NL - 1) * n + i] = ut;
            }
            if (j <= N) {
                const T vt = q22[it][mm] * sv.at(i, j) + vi[mm] * ijx[it][mm];
                w[2 * d.fs + o] = vt;
                if (j <= NDEP) es[(SIDE_B * NL + j - 1) * n + i] = vt;
                if (j >= N + 1 - NDEP) es[(SIDE_T * NL + N - j) * n + i] = vt;
                if (i == 1) es[(SIDE_L * NL + NL - 1) * n + j] = vt;
                if (i == n) es[(SIDE_R * NL + NL - 1) * n + j] = vt;
            }
        }
    }
}

template <class T, int TM, int OCC, bool RUNS, int ORD>
__global__ void __launch_bounds__(STAGE_THREADS, OCC) k_co2contra(const T *__restrict__ Y, T *__restrict__ W,
                                                                 T *__restrict__ ES, Dims d, MetricView<T> m,
                                                                 const double *__restrict__ dtm)
{
    co2contra_tile<T, TM, OCC, RUNS, ORD>(grid_blk(), Y, W, ES, d, m, dtm);
}

// ---------------------------------------------------------------------------
// fused stage: tendency of the linear operator + RK4 update
// ---------------------------------------------------------------------------
template <class T, int TM>
struct StageLayout {
    static constexpr int PW = Tile<TM>::PW, PT = Tile<TM>::PT, RW = Tile<TM>::RW;
    static constexpr int H = 0, UT = H + PW * RW, VT = UT + PW * RW, JU = VT + PW * RW, JV = JU + PW * TM,
                         UP = JV + PT * RW, VP = UP + PW * TM, DX = VP + PT * RW, KX = DX + PT * TM,
                         HL = KX + PT * TM, HR = HL + TM, HB = HR + TM, HT = HB + TM, TOTAL = HT + TM;
    static constexpr size_t bytes() { return sizeof(T) * TOTAL; }
};

__device__ __forceinline__ bool on_boundary(int k, int l, int n) { return k == 1 || k == n || l == 1 || l == n; }

//   mode 0: out = A(y)
//   mode 1: Y1 = V0 + dt/2 k,  ACC = dt/6 k
//   mode 2: Y1 = V0 + dt/2 k,  ACC += dt/3 k
//   mode 3: Y1 = V0 + dt   k,  ACC += dt/3 k
//   mode 4: V0 += ACC + dt/6 k          (FP32: Kahan with compensation CMP)
// ADV: the advective operator (divergence of the mass flux a.F, tendencies a.A,
// gradient of the pre-averaging boundary h a.HB); false: the linear operator.
template <class T, int TM, int OCC, int MODE, bool ADV, bool RUNS, int ORD>
__device__ __forceinline__ void stage_tile(const Blk &bk, const T *__restrict__ Yin, const T *__restrict__ Wc,
                                           const T *__restrict__ E, T *V0, T *Y1, T *ACC, T *CMP, const Dims &d,
                                           const MetricView<T> &m, const StageArgs &a)
{
    using namespace sbp;
    extern __shared__ __align__(16) unsigned char smraw[];
    using L = StageLayout<T, TM>;
    CHSWE_TILE_CONSTANTS(TM, RUNS);
    using SB = SbpOrder<ORD>;
    T *sm = reinterpret_cast<T *>(smraw);
    const int N = d.N, n = N + 1, P = d.P;
    int i0, i1, j0, j1;
    tile_range(bk, n, i0, i1, j0, j1);
    const int tw = i1 - i0, th = j1 - j0;
    const int t = bk.z % NPAN, mem = bk.z / NPAN;
    if (member_frozen(a.dtm, mem)) return;
    const int64_t mo = mem * d.ms;
    const T *y = Yin + mo;                 // member base (the h halos read the other panels)
    const T *w = Wc + mo;
    const T *yp = y + t * d.ps, *wp = w + t * d.ps;
    const SWin<T, PW> sh{sm + L::H, i0 - 2, j0 - 2}, sut{sm + L::UT, i0 - 3, j0 - 2}, svt{sm + L::VT, i0 - 2, j0 - 3},
        sju{sm + L::JU, i0 - 3, j0}, sup{sm + L::UP, i0 - 2, j0};
    const SWin<T, PT> sjv{sm + L::JV, i0, j0 - 3}, svp{sm + L::VP, i0, j0 - 2}, sdx{sm + L::DX, i0, j0},
        skx{sm + L::KX, i0, j0};
    T *hl = sm + L::HL, *hr = sm + L::HR, *hb = sm + L::HB, *ht = sm + L::HT;
    const int w5 = tw + 5, h5 = th + 5;
    const float iw5 = 1.0f / (float)w5, ih5 = 1.0f / (float)h5, iw = 1.0f / (float)tw, ih = 1.0f / (float)th;
    const T *fJ2 = m.fJ2 + t * d.ps;
    const bool sat_l = i0 <= SB::NSAT, sat_r = i1 - 1 >= N + 1 - SB::NSAT, sat_b = j0 <= SB::NSAT,
               sat_t = j1 - 1 >= N + 1 - SB::NSAT;
    // runs along the tile width / height: window passes (RBW), tile passes (RBT)
    const int nww = (tw + RBW - 1) / RBW, nhw = (th + RBW - 1) / RBW, nwt = (tw + RBT - 1) / RBT,
              nht = (th + RBT - 1) / RBT;

    pdl_trigger();
    pdl_wait();
    // The windows (h, ut, vt, J on the u and v meshes; for the advective operator also
    // the mass flux, into the up and vp windows until the first pass phase reads it)
    // go straight into shared memory by asynchronous copies: one memory round trip and
    // no register staging.  The J ut and J vt products (J Fu, J Fv) and the advective
    // operator's substitutions in the h window follow in the first pass phase.
    const int64_t oh = box_off(P, sh.x0, sh.y0), ou = box_off(P, sut.x0, sut.y0), ov = box_off(P, svt.x0, svt.y0);
    {
        const T *gh = yp + oh, *gu = wp + d.fs + ou, *gv = wp + 2 * d.fs + ov, *gjy = m.Jy + ou, *gjx = m.Jx + ov;
        // the fields whose divergence is taken: ut, vt, or the advective operator's mass flux
        const T *gfu = ADV ? (const T *)a.F + mo + t * d.ps + d.fs + ou : nullptr;
        const T *gfv = ADV ? (const T *)a.F + mo + t * d.ps + 2 * d.fs + ov : nullptr;
#pragma unroll
        for (int it = 0; it < IT_WIN; it++) {
            const int q = threadIdx.x + it * STAGE_THREADS;
            int r, c;
            split(q, w5, iw5, r, c);
            if (q < w5 * h5) {
                const int go = r * P + c;
                __pipeline_memcpy_async(sh.a + r * PW + c, gh + go, sizeof(T));
                __pipeline_memcpy_async(sut.a + r * PW + c, gu + go, sizeof(T));
                __pipeline_memcpy_async(svt.a + r * PW + c, gv + go, sizeof(T));
                if (r >= 2 && r < th + 2) {
                    __pipeline_memcpy_async(sju.a + (r - 2) * PW + c, gjy + go, sizeof(T));
                    if constexpr (ADV) __pipeline_memcpy_async(sup.a + (r - 2) * PW + c, gfu + go, sizeof(T));
                }
                if (c >= 2 && c < tw + 2) {
                    __pipeline_memcpy_async(sjv.a + r * PT + (c - 2), gjx + go, sizeof(T));
                    if constexpr (ADV) __pipeline_memcpy_async(svp.a + r * PT + (c - 2), gfv + go, sizeof(T));
                }
            }
        }
        __pipeline_commit();
    }
    // ---- batch 1b: vt window with J vt, the h halos across the panel edges, and
    // fJ2 (or the synchronised edge value) for the up / vp passes
    T f1[IT_RW][RBW], f2[IT_STRIP];
    {
        T hx0 = 0, hx1 = 0, hy0 = 0, hy1 = 0;
        const int q = threadIdx.x;
        const T *hpre = ADV ? (const T *)a.HB : nullptr;
        auto halo = [&](int s, int along) {
            if (!ADV) return h_halo(y, d, t, s, along);
            const Link L = c_link[t][s];
            const int ap = nb_along(L, n, along);
            T hv = __ldg(hpre + hb_index(N, mem, L.nb, L.nside, ap));
            if (a.HS) {
                // the neighbour's h_surf at its copy of the vertex
                int k, l;
                side_vertex(N, L.nside, ap, 0, k, l);
                hv += __ldg((const T *)a.HS + L.nb * d.ps + box_off(P, k, l));
            }
            return hv;
        };
        if (q < th) {
            if (sat_l) hx0 = halo(SIDE_L, j0 + q);
            if (sat_r) hx1 = halo(SIDE_R, j0 + q);
        }
        if (q < tw) {
            if (sat_b) hy0 = halo(SIDE_B, i0 + q);
            if (sat_t) hy1 = halo(SIDE_T, i0 + q);
        }
#pragma unroll
        for (int it = 0; it < IT_RW; it++) {
            const int qq = threadIdx.x + it * STAGE_THREADS;
            int r, x;
            split(qq, w5, iw5, r, x);
            const int k = sup.x0 + x, l0 = j0 + r * RBW;
#pragma unroll
            for (int mm = 0; mm < RBW; mm++) {
                const int l = l0 + mm;
                if (qq >= w5 * nhw || l >= j1) f1[it][mm] = T(0);
                else if (on_boundary(k, l, n)) f1[it][mm] = (k >= 1 && k <= n) ? edge_entry(E, N, mem, t, k, l)[0] : T(0);
                else f1[it][mm] = __ldg(fJ2 + box_off(P, k, l));
            }
        }
#pragma unroll
        for (int it = 0; it < IT_STRIP; it++) {
            const int qq = threadIdx.x + it * STAGE_THREADS;
            int r, c;
            split(qq, tw, iw, r, c);
            const int k = i0 + c, l = svp.y0 + r;
            if (qq >= tw * h5) f2[it] = T(0);
            else if (l >= 1 && l <= n && on_boundary(k, l, n)) f2[it] = edge_entry(E, N, mem, t, k, l)[1];
            else f2[it] = __ldg(fJ2 + box_off(P, k, l));
        }
        if (q < th) { hl[q] = hx0; hr[q] = hx1; }
        if (q < tw) { hb[q] = hy0; ht[q] = hy1; }
    }

    // ---- batch 2 (in flight during the passes): the final pass's metric, or the
    // synchronised divergence on the panel boundary, by output run
    // (the advective operator: also its tendencies of the thread's points)
    T mja[IT_RT][RBT], mjy[IT_RT][RBT], mjx[IT_RT][RBT], mau[IT_RT][RBT], mav[IT_RT][RBT];
    const T *Aa = (const T *)a.A;
    // advective tendencies of this panel (u, v fields)
    const T *Au = ADV ? Aa + mo + t * d.ps + d.fs : nullptr, *Av = ADV ? Aa + mo + t * d.ps + 2 * d.fs : nullptr;
#pragma unroll
    for (int it = 0; it < IT_RT; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, x;
        split(q, tw, iw, r, x);
        const int i = i0 + x, jr = j0 + r * RBT;
#pragma unroll
        for (int mm = 0; mm < RBT; mm++) {
            const int j = jr + mm;
            const int64_t o = box_off(P, i, j);
            const bool ok = q < tw * nht && j < j1, hu = ok && i <= N, hv = ok && j <= N;
            mja[it][mm] = !ok ? T(0) : on_boundary(i, j, n) ? edge_entry(E, N, mem, t, i, j)[2] : __ldg(m.iJa + o);
            mjy[it][mm] = hu ? __ldg(m.iJy + o) : T(0);
            mjx[it][mm] = hv ? __ldg(m.iJx + o) : T(0);
            if constexpr (ADV) {
                mau[it][mm] = hu ? __ldg(Au + o) : T(0);
                mav[it][mm] = hv ? __ldg(Av + o) : T(0);
            }
        }
    }
    __pipeline_wait_prior(0);
    __syncthreads();
    {
        // J ut on the rows, J vt on the columns of the windows (read from the second phase
        // on); the advective operator: J times its mass flux, and in the h window the
        // values before the averaging of the duplicated boundary vertices (which the
        // gradient reads; only windows that reach a panel-boundary vertex) plus the
        // orography h_surf (the gradient's input is h + h_surf; zero margins)
        const T *hpre = ADV ? (const T *)a.HB : nullptr;
        const bool etile = i0 <= 3 || i1 + 2 >= n || j0 <= 3 || j1 + 2 >= n;
#pragma unroll
        for (int it = 0; it < IT_WIN; it++) {
            const int q = threadIdx.x + it * STAGE_THREADS;
            int r, c;
            split(q, w5, iw5, r, c);
            if (q < w5 * h5) {
                if (r >= 2 && r < th + 2) sju.a[(r - 2) * PW + c] *= (ADV ? sup.a[(r - 2) * PW + c] : sut.a[r * PW + c]);
                if (c >= 2 && c < tw + 2) sjv.a[r * PT + (c - 2)] *= (ADV ? svp.a[r * PT + (c - 2)] : svt.a[r * PW + c]);
                if constexpr (ADV) {
                    const int hi = sh.x0 + c, hj = sh.y0 + r;
                    if (etile && hi >= 1 && hi <= n && hj >= 1 && hj <= n && (hi == 1 || hi == n || hj == 1 || hj == n))
                        sh.a[r * PW + c] = __ldg(hpre + (hi == 1 || hi == n ? hb_index(N, mem, t, hi == 1 ? SIDE_L : SIDE_R, hj)
                                                                      : hb_index(N, mem, t, hj == 1 ? SIDE_B : SIDE_T, hi)));
                    if (a.HS) sh.a[r * PW + c] += __ldg((const T *)a.HS + t * d.ps + oh + r * P + c);
                }
            }
        }
        // the mass flux in the up and vp windows is read above: the passes below overwrite them
        if constexpr (ADV) __syncthreads();
    }

    // ---- P1: up = fJ2 I_c2i,y(vt): columns of the up window, runs along the tile rows
#pragma unroll
    for (int it = 0; it < IT_RW; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, x;
        split(q, w5, iw5, r, x);
        if (q >= w5 * nhw) continue;
        const int k = sup.x0 + x, l0 = j0 + r * RBW, cnt = min(RBW, j1 - l0);
        const Line<T> col = svt.col(k);
        T *o = &sup.at(k, l0);
        if (k == 1 || k == n) {
            // panel-boundary column: the synchronised values
#pragma unroll
            for (int mm = 0; mm < RBW; mm++)
                if (mm < cnt) o[mm * PW] = f1[it][mm];
        } else if (SB::RUN_OK && cnt == RBW && l0 >= SB::C2I_LO && l0 + RBW - 1 <= n - SB::C2I_HI) {
            T v[RBW + 3];
            run_load<T, RBW, -2>(col, l0, v);
#pragma unroll
            for (int mm = 0; mm < RBW; mm++) o[mm * PW] = f1[it][mm] * run_interp<T, RBW, ORD>(v, mm);
        } else {
#pragma unroll
            for (int mm = 0; mm < RBW; mm++) {
                const int l = l0 + mm;
                if (mm < cnt) o[mm * PW] = on_boundary(k, l, n) ? f1[it][mm] : f1[it][mm] * ic2i_u<T, ORD>(l, n, col);
            }
        }
    }
    // ---- P2: I_c2i,x(ut): rows of the vp window, runs along the tile columns
#pragma unroll
    for (int it = 0; it < IT_RW; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, x;
        split(q, h5, ih5, r, x);
        if (q >= h5 * nww) continue;
        const int l = svp.y0 + x, k0 = i0 + r * RBW, cnt = min(RBW, i1 - k0);
        const Line<T> row = sut.row(l);
        T *o = &svp.at(k0, l);
        if (SB::RUN_OK && cnt == RBW && k0 >= SB::C2I_LO && k0 + RBW - 1 <= n - SB::C2I_HI) {
            T v[RBW + 3];
            run_load<T, RBW, -2>(row, k0, v);
#pragma unroll
            for (int mm = 0; mm < RBW; mm++) o[mm] = run_interp<T, RBW, ORD>(v, mm);
        } else {
#pragma unroll
            for (int mm = 0; mm < RBW; mm++)
                if (mm < cnt) o[mm] = ic2i_u<T, ORD>(k0 + mm, n, row);
        }
    }
    __syncthreads();
    // ---- P3 (second phase: J ut is complete): x part of the divergence, c2i difference of
    // J ut; tile rows, runs along columns
#pragma unroll
    for (int it = 0; it < IT_RT; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, x;
        split(q, th, ih, r, x);
        if (q >= th * nwt) continue;
        const int j = j0 + x, k0 = i0 + r * RBT, cnt = min(RBT, i1 - k0);
        const Line<T> row = sju.row(j);
        T *o = &sdx.at(k0, j);
        if (SB::RUN_OK && cnt == RBT && k0 >= SB::C2I_LO && k0 + RBT - 1 <= n - SB::C2I_HI) {
            T v[RBT + 3];
            run_load<T, RBT, -2>(row, k0, v);
#pragma unroll
            for (int mm = 0; mm < RBT; mm++) o[mm] = run_diff<T, RBT, ORD>(v, mm);
        } else {
#pragma unroll
            for (int mm = 0; mm < RBT; mm++)
                if (mm < cnt) o[mm] = dc2i_u<T, ORD>(k0 + mm, n, row);
        }
    }
    // ---- P4: -g grad_x h (with SAT) and I_i2c,x(up) on the u points: tile rows, runs
    // along the columns; the second goes to the dead ut window and is scaled by 1/J
    // in the final pass
    const SWin<T, PT> scx{sm + L::UT, i0, j0};
    const int iu1 = min(i1, n);
#pragma unroll
    for (int it = 0; it < IT_RT; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, x;
        split(q, th, ih, r, x);
        if (q >= th * nwt) continue;
        const int j = j0 + x, k0 = i0 + r * RBT, cnt = min(RBT, iu1 - k0);
        const Line<T> hrow = sh.row(j), prow = sup.row(j);
        T *og = &skx.at(k0, j), *oc = &scx.at(k0, j);
        if (SB::RUN_OK && cnt == RBT && k0 >= SB::U_LO && k0 + RBT - 1 <= N - SB::U_HI) {
            T v[RBT + 3];
            run_load<T, RBT, -1>(hrow, k0, v);
#pragma unroll
            for (int mm = 0; mm < RBT; mm++) og[mm] = -m.grav * (run_diff<T, RBT, ORD>(v, mm) * m.inv_hxa);
            run_load<T, RBT, -1>(prow, k0, v);
#pragma unroll
            for (int mm = 0; mm < RBT; mm++) oc[mm] = run_interp<T, RBT, ORD>(v, mm);
        } else {
#pragma unroll
            for (int mm = 0; mm < RBT; mm++) {
                if (mm >= cnt) continue;
                const int i = k0 + mm;
                T gx = di2c_u<T, ORD>(i, N, hrow);
                if (i <= SB::NSAT) gx += T(SB::satw(i)) * (hrow(1) - hl[x]);
                if (i >= N + 1 - SB::NSAT) gx += T(SB::satw(N + 1 - i)) * (hr[x] - hrow(n));
                og[mm] = -m.grav * (gx * m.inv_hxa);
                oc[mm] = ii2c_u<T, ORD>(i, N, prow);
            }
        }
    }
    // ---- P4b (row-major): vp = -fJ2 I_c2i,x(ut), synchronised values on the panel boundary
#pragma unroll
    for (int it = 0; it < IT_STRIP; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, c;
        split(q, tw, iw, r, c);
        const int k = i0 + c, l = svp.y0 + r;
        if (q < tw * h5) {
            T &s = svp.at(k, l);
            s = (l >= 1 && l <= n && on_boundary(k, l, n)) ? f2[it] : -f2[it] * s;
        }
    }
    __syncthreads();

    // ---- P5: divergence and the tendencies of the thread's points (tile columns, runs
    // along the rows; lanes take consecutive columns, so the global accesses of the
    // RK4 update below are coalesced row by row)
    const T H = T(a.Hm[mem]);
    T kh[IT_RT][RBT], ku[IT_RT][RBT], kv[IT_RT][RBT];
#pragma unroll
    for (int it = 0; it < IT_RT; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, x;
        split(q, tw, iw, r, x);
        const int i = i0 + x, jr = j0 + r * RBT, cnt = q < tw * nht ? min(RBT, j1 - jr) : 0;
#pragma unroll
        for (int mm = 0; mm < RBT; mm++) kh[it][mm] = ku[it][mm] = kv[it][mm] = T(0);
        if (cnt <= 0) continue;
        const Line<T> dcol = sjv.col(i), hcol = sh.col(i), pcol = svp.col(i);
        if (SB::RUN_OK && cnt == RBT && jr >= SB::V_LO && jr + RBT - 1 <= N - SB::V_HI) {
            // rows clear of the closures, the SAT terms and the panel-boundary rows
            const bool bcol = (i == 1 || i == n), hasu = i <= N;
            T v[RBT + 3];
            run_load<T, RBT, -2>(dcol, jr, v);
#pragma unroll
            for (int mm = 0; mm < RBT; mm++) {
                const T dvg = bcol ? mja[it][mm]
                                   : (sdx.at(i, jr + mm) * m.inv_hx + run_diff<T, RBT, ORD>(v, mm) * m.inv_hx) * mja[it][mm];
                kh[it][mm] = -H * dvg;
            }
            if (hasu) {
#pragma unroll
                for (int mm = 0; mm < RBT; mm++) {
                    const int j = jr + mm;
                    if constexpr (ADV) {
                        const T au = mau[it][mm];
                        ku[it][mm] = (au + skx.at(i, j)) + scx.at(i, j) * mjy[it][mm];
                    } else {
                        ku[it][mm] = skx.at(i, j) + scx.at(i, j) * mjy[it][mm];
                    }
                }
            }
            run_load<T, RBT, -1>(hcol, jr, v);
            T gy[RBT];
#pragma unroll
            for (int mm = 0; mm < RBT; mm++) gy[mm] = run_diff<T, RBT, ORD>(v, mm) * m.inv_hxa;
            run_load<T, RBT, -1>(pcol, jr, v);
#pragma unroll
            for (int mm = 0; mm < RBT; mm++) {
                if constexpr (ADV) {
                    const int j = jr + mm;
                    T av = mav[it][mm];
                    if (i == 1 || i == n) av = adv_edge_sync(Aa, d, mem, t, 2, i, j, av);
                    kv[it][mm] = (av + -m.grav * gy[mm]) + run_interp<T, RBT, ORD>(v, mm) * mjx[it][mm];
                } else {
                    kv[it][mm] = -m.grav * gy[mm] + run_interp<T, RBT, ORD>(v, mm) * mjx[it][mm];
                }
            }
            continue;
        }
#pragma unroll
        for (int mm = 0; mm < RBT; mm++) {
            if (mm >= cnt) continue;
            const int j = jr + mm;
            T dvg;
            if (on_boundary(i, j, n)) {
                dvg = mja[it][mm];
            } else {
                const T dy = dc2i_u<T, ORD>(j, n, dcol);
                dvg = (sdx.at(i, j) * m.inv_hx + dy * m.inv_hx) * mja[it][mm];
            }
            kh[it][mm] = -H * dvg;
            if (i <= N) {
                if constexpr (ADV) {
                    // advective operator: (A + (-g) grad_x h) + Coriolis, A synchronised on the duplicated edge rows
                    T au = mau[it][mm];
                    if (j == 1 || j == n) au = adv_edge_sync(Aa, d, mem, t, 1, i, j, au);
                    ku[it][mm] = (au + skx.at(i, j)) + scx.at(i, j) * mjy[it][mm];
                } else {
                    ku[it][mm] = skx.at(i, j) + scx.at(i, j) * mjy[it][mm];
                }
            }
            if (j <= N) {
                T gy = di2c_u<T, ORD>(j, N, hcol);
                if (j <= SB::NSAT) gy += T(SB::satw(j)) * (hcol(1) - hb[x]);
                if (j >= N + 1 - SB::NSAT) gy += T(SB::satw(N + 1 - j)) * (ht[x] - hcol(n));
                gy = gy * m.inv_hxa;
                if constexpr (ADV) {
                    T av = mav[it][mm];
                    if (i == 1 || i == n) av = adv_edge_sync(Aa, d, mem, t, 2, i, j, av);
                    kv[it][mm] = (av + -m.grav * gy) + ii2c_u<T, ORD>(j, N, pcol) * mjx[it][mm];
                } else {
                    kv[it][mm] = -m.grav * gy + ii2c_u<T, ORD>(j, N, pcol) * mjx[it][mm];
                }
            }
        }
    }

    // ---- RK4 update, all operand loads of the thread in one batch
    T *v0 = V0 + mo + t * d.ps, *y1 = Y1 + mo + t * d.ps, *acc = ACC + mo + t * d.ps;
    T *cmp = CMP ? CMP + mo + t * d.ps : nullptr;
    const int64_t fs = d.fs;
    const T dt = T(a.dtm ? a.dtm[mem] : a.dt);
    constexpr bool LV = MODE >= 1, LA = MODE >= 2, LC = (sizeof(T) == 4) && MODE == 4;
    T pv[3][IT_RT][RBT], pa[3][IT_RT][RBT], pc[3][IT_RT][RBT];
#pragma unroll
    for (int it = 0; it < IT_RT; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, x;
        split(q, tw, iw, r, x);
        const int i = i0 + x, jr = j0 + r * RBT, cnt = q < tw * nht ? min(RBT, j1 - jr) : 0;
#pragma unroll
        for (int mm = 0; mm < RBT; mm++) {
            const int j = jr + mm;
            const int64_t o = box_off(P, i, j);
            const bool ok = mm < cnt;
            const bool has[3] = {ok, ok && i <= N, ok && j <= N};
#pragma unroll
            for (int f = 0; f < 3; f++) {
                pv[f][it][mm] = LV && has[f] ? v0[o + f * fs] : T(0);
                pa[f][it][mm] = LA && has[f] ? acc[o + f * fs] : T(0);
                pc[f][it][mm] = LC && has[f] ? cmp[o + f * fs] : T(0);
            }
        }
    }
#pragma unroll
    for (int it = 0; it < IT_RT; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, x;
        split(q, tw, iw, r, x);
        const int i = i0 + x, jr = j0 + r * RBT, cnt = q < tw * nht ? min(RBT, j1 - jr) : 0;
#pragma unroll
        for (int mm = 0; mm < RBT; mm++) {
            const int j = jr + mm;
            const int64_t o = box_off(P, i, j);
            const bool ok = mm < cnt;
            const bool has[3] = {ok, ok && i <= N, ok && j <= N};
            const T k3[3] = {kh[it][mm], ku[it][mm], kv[it][mm]};
#pragma unroll
            for (int f = 0; f < 3; f++) {
                if (!has[f]) continue;
                const int64_t of = o + f * fs;
                if constexpr (MODE == 0) {
                    y1[of] = k3[f];
                } else if constexpr (MODE <= 3) {
                    const T ca = (MODE == 3) ? dt : T(0.5) * dt;
                    const T cb = (MODE == 1) ? dt / T(6) : dt / T(3);
                    y1[of] = pv[f][it][mm] + ca * k3[f];
                    acc[of] = (MODE == 1) ? cb * k3[f] : pa[f][it][mm] + cb * k3[f];
                } else if constexpr (sizeof(T) == 4) {
                    float sv = pv[f][it][mm], cv = pc[f][it][mm];
                    kahan_add(sv, cv, pa[f][it][mm] + (dt / T(6)) * k3[f]);
                    v0[of] = sv;
                    cmp[of] = cv;
                } else {
                    v0[of] = pv[f][it][mm] + (pa[f][it][mm] + (dt / T(6)) * k3[f]);
                }
            }
        }
    }
}

template <class T, int TM, int OCC, int MODE, bool ADV, bool RUNS, int ORD>
__global__ void __launch_bounds__(STAGE_THREADS, OCC) k_stage(const T *__restrict__ Yin, const T *__restrict__ Wc,
                                                          const T *__restrict__ E, T *V0, T *Y1, T *ACC, T *CMP,
                                                          Dims d, MetricView<T> m, StageArgs a)
{
    stage_tile<T, TM, OCC, MODE, ADV, RUNS, ORD>(grid_blk(), Yin, Wc, E, V0, Y1, ACC, CMP, d, m, a);
}

}  // namespace chswe
