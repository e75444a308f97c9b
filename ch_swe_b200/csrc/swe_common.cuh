// swe_common.cuh -- device-side layout, SBP stencil tables and cube-edge halo
// reads shared by the shallow-water kernels.
//
// Layout in HBM (one allocation per state vector):
//   [member][field h=0,u=1,v=2][panel 0..5][row j=1..N+1][pitch P >= N+1]
// Every field uses the (N+1) x P box of the xy mesh: u (y mesh, i = 1..N,
// j = 1..N+1) leaves column N+1 unused, v (x mesh, i = 1..N+1, j = 1..N)
// leaves row N+1 unused.  Indices below are the reference's 1-based (i, j).
#pragma once

#include <cstdint>

namespace chswe {

constexpr int NPAN = 6;

// Sides of a panel: 0 left (i = 1), 1 right (i = N+1), 2 bottom (j = 1), 3 top (j = N+1).
enum { SIDE_L = 0, SIDE_R = 1, SIDE_B = 2, SIDE_T = 3 };

// Zero margin around every panel box: point (i, j), 1 <= i, j <= N+1, lives at
// row j - 1 + MG, column i - 1 + MG of an (N+1+2MG)-row box, so stencil windows
// reaching up to MG points beyond the panel read zeros without bounds checks.
constexpr int MG = 4;

__host__ __device__ __forceinline__ int64_t box_off(int P, int i, int j)
{
    return (int64_t)(j - 1 + MG) * P + (i - 1 + MG);
}
// The same offset in 32 bits, for device code indexing within one member's
// state (three fields of six panel boxes stay far below 2^31 elements).
__device__ __forceinline__ int box_off32(int P, int i, int j) { return (j - 1 + MG) * P + (i - 1 + MG); }

struct Dims {
    int N;         // cells per panel edge
    int P;         // row pitch in elements (>= N+1+2MG, multiple of 8)
    int64_t ps;    // panel stride   = (N+1+2MG) * P
    int64_t fs;    // field stride   = 6 * ps
    int64_t ms;    // member stride  = 3 * fs
};

// Edge connectivity: neighbour panel, its side, reversed along-edge order,
// sign of the normal and tangential covariant components across the edge.
struct Link {
    int nb, nside, rev, sn, st;
};

template <class T>
struct MetricView {
    const T *Q11y, *iJy, *Jy;     // y mesh (u points): Qi11, 1/J, J
    const T *Q22x, *iJx, *Jx;     // x mesh (v points): Qi22, 1/J, J
    const T *JQ12;                // xy mesh: J * Qi12
    const T *iJa;                 // xy mesh: 1 / (J * a)
    const T *fJ2;                 // xy mesh, per panel: f * J * J
    const T *qb, *qt, *ql, *qr;   // covariant vector-sync weights along the four sides
    const T *ej, *ef, *ea;        // edge tables of k_edge_tables: J on the edge strips, fJ2 and 1/(J a) on the edges
    T inv_hxa;                    // 1 / (hx * a)
    T inv_hx;                     // 1 / hx   (hx == hy)
    T grav;
};

// Programmatic dependent launch (sm_90+): a kernel launched with programmatic
// stream serialization may start while its predecessor in the stream still runs;
// pdl_wait() returns once the predecessor grid has completed and its writes are
// visible, pdl_trigger() lets this grid's successor launch.  Both are no-ops for
// a kernel launched without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

}  // namespace chswe
