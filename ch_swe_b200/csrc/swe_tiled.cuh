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

namespace chswe {

constexpr int STAGE_THREADS = 256;

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
};

#define CHSWE_TILE_CONSTANTS(TM)                                                                           \
    constexpr int PW = Tile<TM>::PW, PT = Tile<TM>::PT, RW = Tile<TM>::RW, IT_WIN = Tile<TM>::IT_WIN,      \
                  IT_STRIP = Tile<TM>::IT_STRIP, IT_TILE = Tile<TM>::IT_TILE;                               \
    (void)RW

__device__ __forceinline__ void tile_range(int n, int &i0, int &i1, int &j0, int &j1)
{
    i0 = 1 + (blockIdx.x * n) / gridDim.x;
    i1 = 1 + ((blockIdx.x + 1) * n) / gridDim.x;
    j0 = 1 + (blockIdx.y * n) / gridDim.y;
    j1 = 1 + ((blockIdx.y + 1) * n) / gridDim.y;
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

// Interior rows of the four operators (the closure rows go through the general
// functions of swe_sbp.cuh).
template <class T> __device__ __forceinline__ T ic2i_in(int k, const Line<T> &f)
{
    return (T(9) * (f(k) + f(k - 1)) - (f(k + 1) + f(k - 2))) * T(0.0625);
}
template <class T> __device__ __forceinline__ T ii2c_in(int k, const Line<T> &f)
{
    return (T(9) * (f(k + 1) + f(k)) - (f(k + 2) + f(k - 1))) * T(0.0625);
}
template <class T> __device__ __forceinline__ T dc2i_in(int k, const Line<T> &f)
{
    return (T(27) * (f(k) - f(k - 1)) - (f(k + 1) - f(k - 2))) * T(1.0 / 24.0);
}
template <class T> __device__ __forceinline__ T di2c_in(int k, const Line<T> &f)
{
    return (T(27) * (f(k + 1) - f(k)) - (f(k + 2) - f(k - 1))) * T(1.0 / 24.0);
}
template <class T> __device__ __forceinline__ T ic2i_u(int k, int nx, const Line<T> &f)
{
    return (k >= 5 && k <= nx - 4) ? ic2i_in<T>(k, f) : ic2i<T>(k, nx, f);
}
template <class T> __device__ __forceinline__ T ii2c_u(int k, int n, const Line<T> &f)
{
    return (k >= 4 && k <= n - 3) ? ii2c_in<T>(k, f) : ii2c<T>(k, n, f);
}
template <class T> __device__ __forceinline__ T dc2i_u(int k, int nx, const Line<T> &f)
{
    return (k >= 5 && k <= nx - 4) ? dc2i_in<T>(k, f) : dc2i<T>(k, nx, f);
}
template <class T> __device__ __forceinline__ T di2c_u(int k, int n, const Line<T> &f)
{
    return (k >= 4 && k <= n - 3) ? di2c_in<T>(k, f) : di2c<T>(k, n, f);
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

// OCC: resident blocks per SM the register allocation is capped for (autotuned).
template <class T, int TM, int OCC>
__global__ void __launch_bounds__(STAGE_THREADS, OCC) k_co2contra(const T *__restrict__ Y, T *__restrict__ W,
                                                                 T *__restrict__ ES, Dims d, MetricView<T> m,
                                                                 const double *__restrict__ dtm)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    using L = Co2Layout<T, TM>;
    CHSWE_TILE_CONSTANTS(TM);
    T *sm = reinterpret_cast<T *>(smraw);
    const int N = d.N, n = N + 1, P = d.P;
    int i0, i1, j0, j1;
    tile_range(n, i0, i1, j0, j1);
    const int tw = i1 - i0, th = j1 - j0, w5 = tw + 5, h5 = th + 5;
    const float iw5 = 1.0f / (float)w5, ih5 = 1.0f / (float)h5, iw = 1.0f / (float)tw, ih = 1.0f / (float)th;
    const int t = blockIdx.z % NPAN, mem = blockIdx.z / NPAN;
    if (member_frozen(dtm, mem)) return;
    const T *y = Y + mem * d.ms + t * d.ps;
    T *w = W + mem * d.ms + t * d.ps;
    T *es = ES + strip_member(N, mem) + (int64_t)t * 4 * STRIP_LINES * n - 1;   // + (s*4 + line)*n + index
    const SWin<T, PW> sv{sm + L::V, i0 - 2, j0 - 3}, su{sm + L::U, i0 - 3, j0 - 2}, svq{sm + L::VQ, i0 - 2, j0};
    const SWin<T, PT> suq{sm + L::UQ, i0, j0 - 2}, sux{sm + L::UX, i0, j0};

    // ---- before the predecessor grid completes: J Qi12 at both xy intermediates (metric only)
    pdl_trigger();
    T jq1[IT_STRIP], jq2[IT_STRIP];
#pragma unroll
    for (int it = 0; it < IT_STRIP; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, c;
        split(q, w5, iw5, r, c);
        jq1[it] = q < w5 * th ? __ldg(m.JQ12 + box_off(P, sv.x0 + c, j0 + r)) : T(0);
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
    // ---- batch 2 (in flight during the passes): the output metric
    T q11[IT_TILE], ijy[IT_TILE], q22[IT_TILE], ijx[IT_TILE];
#pragma unroll
    for (int it = 0; it < IT_TILE; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, c;
        split(q, tw, iw, r, c);
        const int i = i0 + c, j = j0 + r;
        const int64_t o = box_off(P, i, j);
        const bool ok = q < tw * th;
        q11[it] = ok && i <= N ? __ldg(m.Q11y + o) : T(0);
        ijy[it] = ok && i <= N ? __ldg(m.iJy + o) : T(0);
        q22[it] = ok && j <= N ? __ldg(m.Q22x + o) : T(0);
        ijx[it] = ok && j <= N ? __ldg(m.iJx + o) : T(0);
    }
    __syncthreads();
    // J Qi12 I_c2i,y(v) at xy nodes: row-major (y stencil, warp-uniform closure)
#pragma unroll
    for (int it = 0; it < IT_STRIP; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, c;
        split(q, w5, iw5, r, c);
        const int k = sv.x0 + c, l = j0 + r;
        if (q < w5 * th) svq.at(k, l) = ic2i_u<T>(l, n, sv.col(k)) * jq1[it];
    }
    // I_c2i,x(u) at xy nodes: column-major (x stencil); the J Qi12 factor follows
#pragma unroll
    for (int it = 0; it < IT_STRIP; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int c, r;
        split(q, h5, ih5, c, r);
        const int k = i0 + c, l = suq.y0 + r;
        if (q < tw * h5) suq.at(k, l) = ic2i_u<T>(k, n, su.row(l));
    }
    __syncthreads();
    // I_i2c,x of the first: column-major
#pragma unroll
    for (int it = 0; it < IT_TILE; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int c, r;
        split(q, th, ih, c, r);
        const int i = i0 + c, j = j0 + r;
        if (q < tw * th && i <= N) sux.at(i, j) = ii2c_u<T>(i, N, svq.row(j));
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
    // outputs: row-major, I_i2c,y of the second (warp-uniform closure), coalesced stores
#pragma unroll
    for (int it = 0; it < IT_TILE; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, c;
        split(q, tw, iw, r, c);
        const int i = i0 + c, j = j0 + r;
        const int64_t o = box_off(P, i, j);
        if (q < tw * th) {
            // the edge strips (k_edge reads them contiguous along each side)
            if (i <= N) {
                const T ut = q11[it] * su.at(i, j) + sux.at(i, j) * ijy[it];
                w[d.fs + o] = ut;
                if (i <= 3) es[(SIDE_L * 4 + i - 1) * n + j] = ut;
                if (i >= N - 2) es[(SIDE_R * 4 + N - i) * n + j] = ut;
                if (j == 1) es[(SIDE_B * 4 + 3) * n + i] = ut;
                if (j == n) es[(SIDE_T * 4 + 3) * n + i] = ut;
            }
            if (j <= N) {
                const T vt = q22[it] * sv.at(i, j) + ii2c_u<T>(j, N, suq.col(i)) * ijx[it];
                w[2 * d.fs + o] = vt;
                if (j <= 3) es[(SIDE_B * 4 + j - 1) * n + i] = vt;
                if (j >= N - 2) es[(SIDE_T * 4 + N - j) * n + i] = vt;
                if (i == 1) es[(SIDE_L * 4 + 3) * n + j] = vt;
                if (i == n) es[(SIDE_R * 4 + 3) * n + j] = vt;
            }
        }
    }
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
template <class T, int TM, int OCC, int MODE, bool ADV>
__global__ void __launch_bounds__(STAGE_THREADS, OCC) k_stage(const T *__restrict__ Yin, const T *__restrict__ Wc,
                                                          const T *__restrict__ E, T *V0, T *Y1, T *ACC, T *CMP,
                                                          Dims d, MetricView<T> m, StageArgs a)
{
    using namespace sbp;
    extern __shared__ __align__(16) unsigned char smraw[];
    using L = StageLayout<T, TM>;
    CHSWE_TILE_CONSTANTS(TM);
    T *sm = reinterpret_cast<T *>(smraw);
    const int N = d.N, n = N + 1, P = d.P;
    int i0, i1, j0, j1;
    tile_range(n, i0, i1, j0, j1);
    const int tw = i1 - i0, th = j1 - j0;
    const int t = blockIdx.z % NPAN, mem = blockIdx.z / NPAN;
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
    const bool sat_l = i0 <= 3, sat_r = i1 - 1 >= N - 2, sat_b = j0 <= 3, sat_t = j1 - 1 >= N - 2;

    pdl_trigger();
    pdl_wait();
    // ---- batch 1a: h and ut windows with J ut
    {
        const int64_t oh = box_off(P, sh.x0, sh.y0), ou = box_off(P, sut.x0, sut.y0);
        const T *gh = yp + oh, *gu = wp + d.fs + ou, *gjy = m.Jy + ou;
        // the field whose divergence is taken: ut, or the mass flux of the advective operator
        const T *gf = ADV ? (const T *)a.F + mo + t * d.ps + d.fs + ou : nullptr;
        T rh[IT_WIN], ru[IT_WIN], rjy[IT_WIN], rfu[IT_WIN];
        const T *hpre = ADV ? (const T *)a.HB : nullptr;
        // only windows that reach a panel-boundary vertex read the pre-averaging values
        const bool etile = i0 <= 3 || i1 + 2 >= n || j0 <= 3 || j1 + 2 >= n;
#pragma unroll
        for (int it = 0; it < IT_WIN; it++) {
            const int q = threadIdx.x + it * STAGE_THREADS;
            int r, c;
            split(q, w5, iw5, r, c);
            const bool ok = q < w5 * h5;
            const int go = r * P + c;
            const bool jr = ok && r >= 2 && r < th + 2;
            rh[it] = ok ? __ldg(gh + go) : T(0);
            if (ADV && etile && ok) {
                // advective operator: the gradient reads h as it was before the averaging
                const int hi = sh.x0 + c, hj = sh.y0 + r;
                if (hi >= 1 && hi <= n && hj >= 1 && hj <= n && (hi == 1 || hi == n || hj == 1 || hj == n))
                    rh[it] = __ldg(hpre + (hi == 1 || hi == n ? hb_index(N, mem, t, hi == 1 ? SIDE_L : SIDE_R, hj)
                                                           : hb_index(N, mem, t, hj == 1 ? SIDE_B : SIDE_T, hi)));
            }
            ru[it] = ok ? __ldg(gu + go) : T(0);
            rjy[it] = jr ? __ldg(gjy + go) : T(0);
            rfu[it] = ADV && jr ? __ldg(gf + go) : ru[it];
        }
#pragma unroll
        for (int it = 0; it < IT_WIN; it++) {
            const int q = threadIdx.x + it * STAGE_THREADS;
            int r, c;
            split(q, w5, iw5, r, c);
            if (q < w5 * h5) {
                sh.a[r * PW + c] = rh[it];
                sut.a[r * PW + c] = ru[it];
                if (r >= 2 && r < th + 2) sju.a[(r - 2) * PW + c] = rjy[it] * rfu[it];
            }
        }
    }
    // ---- batch 1b: vt window with J vt, the h halos across the panel edges, and
    // fJ2 (or the synchronised edge value) for the up / vp passes
    T f1[IT_STRIP], f2[IT_STRIP];
    {
        const int64_t ov = box_off(P, svt.x0, svt.y0);
        const T *gv = wp + 2 * d.fs + ov, *gjx = m.Jx + ov;
        const T *gf = ADV ? (const T *)a.F + mo + t * d.ps + 2 * d.fs + ov : nullptr;
        T rv[IT_WIN], rjx[IT_WIN], rfv[IT_WIN];
#pragma unroll
        for (int it = 0; it < IT_WIN; it++) {
            const int q = threadIdx.x + it * STAGE_THREADS;
            int r, c;
            split(q, w5, iw5, r, c);
            const bool ok = q < w5 * h5;
            const int go = r * P + c;
            const bool jc = ok && c >= 2 && c < tw + 2;
            rv[it] = ok ? __ldg(gv + go) : T(0);
            rjx[it] = jc ? __ldg(gjx + go) : T(0);
            rfv[it] = ADV && jc ? __ldg(gf + go) : rv[it];
        }
        T hx0 = 0, hx1 = 0, hy0 = 0, hy1 = 0;
        const int q = threadIdx.x;
        const T *hpre = ADV ? (const T *)a.HB : nullptr;
        auto halo = [&](int s, int along) {
            if (!ADV) return h_halo(y, d, t, s, along);
            const Link L = c_link[t][s];
            return __ldg(hpre + hb_index(N, mem, L.nb, L.nside, nb_along(L, n, along)));
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
        for (int it = 0; it < IT_STRIP; it++) {
            const int qq = threadIdx.x + it * STAGE_THREADS;
            int r, c;
            split(qq, w5, iw5, r, c);
            int k = sup.x0 + c, l = j0 + r;
            if (qq >= w5 * th) f1[it] = T(0);
            else if (on_boundary(k, l, n)) f1[it] = (k >= 1 && k <= n) ? edge_entry(E, N, mem, t, k, l)[0] : T(0);
            else f1[it] = __ldg(fJ2 + box_off(P, k, l));
            split(qq, tw, iw, r, c);
            k = i0 + c;
            l = svp.y0 + r;
            if (qq >= tw * h5) f2[it] = T(0);
            else if (l >= 1 && l <= n && on_boundary(k, l, n)) f2[it] = edge_entry(E, N, mem, t, k, l)[1];
            else f2[it] = __ldg(fJ2 + box_off(P, k, l));
        }
#pragma unroll
        for (int it = 0; it < IT_WIN; it++) {
            const int qq = threadIdx.x + it * STAGE_THREADS;
            int r, c;
            split(qq, w5, iw5, r, c);
            if (qq < w5 * h5) {
                svt.a[r * PW + c] = rv[it];
                if (c >= 2 && c < tw + 2) sjv.a[r * PT + (c - 2)] = rjx[it] * rfv[it];
            }
        }
        if (q < th) { hl[q] = hx0; hr[q] = hx1; }
        if (q < tw) { hb[q] = hy0; ht[q] = hy1; }
    }

    // ---- batch 2 (in flight during the passes): the final pass's metric, or the
    // synchronised divergence on the panel boundary
    T mja[IT_TILE], mjy[IT_TILE], mjx[IT_TILE];
#pragma unroll
    for (int it = 0; it < IT_TILE; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, c;
        split(q, tw, iw, r, c);
        const int i = i0 + c, j = j0 + r;
        const int64_t o = box_off(P, i, j);
        const bool ok = q < tw * th, hu = ok && i <= N, hv = ok && j <= N;
        mja[it] = !ok ? T(0) : on_boundary(i, j, n) ? edge_entry(E, N, mem, t, i, j)[2] : __ldg(m.iJa + o);
        mjy[it] = hu ? __ldg(m.iJy + o) : T(0);
        mjx[it] = hv ? __ldg(m.iJx + o) : T(0);
    }
    __syncthreads();

    // ---- P1 (row-major): up = fJ2 I_c2i,y(vt) on the tile rows, tile columns +- footprint
#pragma unroll
    for (int it = 0; it < IT_STRIP; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, c;
        split(q, w5, iw5, r, c);
        const int k = sup.x0 + c, l = j0 + r;
        if (q < w5 * th) sup.at(k, l) = on_boundary(k, l, n) ? f1[it] : f1[it] * ic2i_u<T>(l, n, svt.col(k));
    }
    // ---- P2 (column-major): I_c2i,x(ut) on the tile columns, tile rows +- footprint
#pragma unroll
    for (int it = 0; it < IT_STRIP; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int c, r;
        split(q, h5, ih5, c, r);
        const int k = i0 + c, l = svp.y0 + r;
        if (q < tw * h5) svp.at(k, l) = ic2i_u<T>(k, n, sut.row(l));
    }
    // ---- P3 (column-major): x part of the divergence, c2i difference of J ut
#pragma unroll
    for (int it = 0; it < IT_TILE; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int c, r;
        split(q, th, ih, c, r);
        if (q < tw * th) sdx.at(i0 + c, j0 + r) = dc2i_u<T>(i0 + c, n, sju.row(j0 + r));
    }
    __syncthreads();
    // ---- P4 (column-major): -g grad_x h (with SAT) and I_i2c,x(up); the second goes to the
    // dead ut window and is scaled by 1/J in the final row-major pass
    const SWin<T, PT> scx{sm + L::UT, i0, j0};
#pragma unroll
    for (int it = 0; it < IT_TILE; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int c, r;
        split(q, th, ih, c, r);
        const int i = i0 + c, j = j0 + r;
        if (q < tw * th && i <= N) {
            const Line<T> hrow = sh.row(j);
            T gx = di2c_u<T>(i, N, hrow);
            if (i <= 3) {
                const T sat = i == 1 ? T(SATI1) : (i == 2 ? T(SATI2) : T(SATI3));
                gx += sat * (hrow(1) - hl[r]);
            }
            if (i >= N - 2) {
                const T sat = i == N ? T(SATI1) : (i == N - 1 ? T(SATI2) : T(SATI3));
                gx += sat * (hr[r] - hrow(n));
            }
            skx.at(i, j) = -m.grav * (gx * m.inv_hxa);
            scx.at(i, j) = ii2c_u<T>(i, N, sup.row(j));
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

    // ---- P5 (row-major): divergence and v tendency of the thread's points, then the
    // RK4 update with all its operand loads in one batch (coalesced)
    const T H = T(a.Hm[mem]);
    T kh[IT_TILE], ku[IT_TILE], kv[IT_TILE];
#pragma unroll
    for (int it = 0; it < IT_TILE; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, c;
        split(q, tw, iw, r, c);
        const int i = i0 + c, j = j0 + r;
        kh[it] = ku[it] = kv[it] = T(0);
        if (q >= tw * th) continue;
        T dvg;
        if (on_boundary(i, j, n)) {
            dvg = mja[it];
        } else {
            const T dy = dc2i_u<T>(j, n, sjv.col(i));
            dvg = (sdx.at(i, j) * m.inv_hx + dy * m.inv_hx) * mja[it];
        }
        kh[it] = -H * dvg;
        const T *Aa = (const T *)a.A;
        if (i <= N) {
            if constexpr (ADV) {
                // advective operator: (A + (-g) grad_x h) + Coriolis, A synchronised on the duplicated edge rows
                T au = __ldg(Aa + mo + t * d.ps + d.fs + box_off(P, i, j));
                if (j == 1 || j == n) au = adv_edge_sync(Aa, d, mem, t, 1, i, j, au);
                ku[it] = (au + skx.at(i, j)) + scx.at(i, j) * mjy[it];
            } else {
                ku[it] = skx.at(i, j) + scx.at(i, j) * mjy[it];
            }
        }
        if (j <= N) {
            const Line<T> hcol = sh.col(i);
            T gy = di2c_u<T>(j, N, hcol);
            if (j <= 3) {
                const T sat = j == 1 ? T(SATI1) : (j == 2 ? T(SATI2) : T(SATI3));
                gy += sat * (hcol(1) - hb[c]);
            }
            if (j >= N - 2) {
                const T sat = j == N ? T(SATI1) : (j == N - 1 ? T(SATI2) : T(SATI3));
                gy += sat * (ht[c] - hcol(n));
            }
            gy = gy * m.inv_hxa;
            if constexpr (ADV) {
                T av = __ldg(Aa + mo + t * d.ps + 2 * d.fs + box_off(P, i, j));
                if (i == 1 || i == n) av = adv_edge_sync(Aa, d, mem, t, 2, i, j, av);
                kv[it] = (av + -m.grav * gy) + ii2c_u<T>(j, N, svp.col(i)) * mjx[it];
            } else {
                kv[it] = -m.grav * gy + ii2c_u<T>(j, N, svp.col(i)) * mjx[it];
            }
        }
    }

    T *v0 = V0 + mo + t * d.ps, *y1 = Y1 + mo + t * d.ps, *acc = ACC + mo + t * d.ps;
    T *cmp = CMP ? CMP + mo + t * d.ps : nullptr;
    const int64_t fs = d.fs;
    const T dt = T(a.dtm ? a.dtm[mem] : a.dt);
    constexpr bool LV = MODE >= 1, LA = MODE >= 2, LC = (sizeof(T) == 4) && MODE == 4;
    T pv[3][IT_TILE], pa[3][IT_TILE], pc[3][IT_TILE];
#pragma unroll
    for (int it = 0; it < IT_TILE; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, c;
        split(q, tw, iw, r, c);
        const int i = i0 + c, j = j0 + r;
        const int64_t o = box_off(P, i, j);
        const bool ok = q < tw * th;
        const bool has[3] = {ok, ok && i <= N, ok && j <= N};
#pragma unroll
        for (int f = 0; f < 3; f++) {
            pv[f][it] = LV && has[f] ? v0[o + f * fs] : T(0);
            pa[f][it] = LA && has[f] ? acc[o + f * fs] : T(0);
            pc[f][it] = LC && has[f] ? cmp[o + f * fs] : T(0);
        }
    }
#pragma unroll
    for (int it = 0; it < IT_TILE; it++) {
        const int q = threadIdx.x + it * STAGE_THREADS;
        int r, c;
        split(q, tw, iw, r, c);
        const int i = i0 + c, j = j0 + r;
        const int64_t o = box_off(P, i, j);
        const bool ok = q < tw * th;
        const bool has[3] = {ok, ok && i <= N, ok && j <= N};
        const T k3[3] = {kh[it], ku[it], kv[it]};
#pragma unroll
        for (int f = 0; f < 3; f++) {
            if (!has[f]) continue;
            const int64_t of = o + f * fs;
            if constexpr (MODE == 0) {
                y1[of] = k3[f];
            } else if constexpr (MODE <= 3) {
                const T ca = (MODE == 3) ? dt : T(0.5) * dt;
                const T cb = (MODE == 1) ? dt / T(6) : dt / T(3);
                y1[of] = pv[f][it] + ca * k3[f];
                acc[of] = (MODE == 1) ? cb * k3[f] : pa[f][it] + cb * k3[f];
            } else if constexpr (sizeof(T) == 4) {
                float sv = pv[f][it], cv = pc[f][it];
                kahan_add(sv, cv, pa[f][it] + (dt / T(6)) * k3[f]);
                v0[of] = sv;
                cmp[of] = cv;
            } else {
                v0[of] = pv[f][it] + (pa[f][it] + (dt / T(6)) * k3[f]);
            }
        }
    }
}

}  // namespace chswe
