/*
 * swe_oracle.c -- CPU FP64 oracle for the explicit shallow-water time step of
 * ch_swe on the "Ch"-staggered equiangular cubed sphere with SBP 4-2 operators.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against; it is never linked into, loaded by or called from the
 * product library.  Only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * reference arm of bench.py may load it.
 *
 * It is a sweep-by-sweep restatement of the reference (file:line below are
 * relative to the ch_swe source tree), including the MPI halo-exchange
 * semantics (tile intersections, pack order, sign flips and u<->v swaps),
 * executed here as in-process copies between the six panels:
 *
 *   topology ............ src/topology/cubed_sphere_topology_mod.f90:29-239
 *   partition extents ... src/parallel/partition_mod.f90:33-133
 *   exchanges ........... src/parallel/exchange_factory_mod.f90:197-333,369-723
 *   pack / unpack ....... src/parallel/buffer_mod.f90:24-476
 *   metric .............. src/metric/metric_2d_ecs_mod.f90:126-411
 *   meshes .............. src/mesh/mesh_factory_mod.f90:15-80,
 *                         src/domain/domain_factory_mod.f90:197-335
 *   SBP stencils ........ src/differential_operators/sbp_operators/
 *                         sbp_diff_i2c_42_mod.f90, sbp_diff_c2i_42_mod.f90,
 *                         sbp_interp_i2c_42_mod.f90, sbp_interp_c2i_42_mod.f90
 *   gradient ............ .../horizontal/gradient/grad_sbp_sat_mod.f90:24-76
 *   co2contra ........... .../horizontal/co2contra/co2contra_Ch_mod.f90:27-94
 *   Coriolis ............ .../horizontal/coriolis/coriolis_Ch_mod.f90:42-120,
 *                         coriolis_factory_mod.f90:154-280
 *   divergence .......... .../horizontal/divergence/div_sbp_sat_mod.f90:29-80
 *   Ah scalar sync ...... src/halo/halo_Ah_scalar_sync_mod.f90:21-98
 *   ECS Ah vector sync .. src/equiang_cs/ecs_Ah_vec_sync_mod.f90:34-125,
 *                         ecs_Ah_vec_sync_factory_mod.f90:97-158
 *   linear operator ..... src/models/shallow_water/operator/operator_swm_lin_mod.f90:66-108
 *   advective operator .. src/models/shallow_water/operator/operator_adv_swm_mod.f90:62-126
 *                         (covariant branch: co2contra_ch_sbp42, massflux_ch_up4,
 *                         div_ch_sbp_sat_42_proj, grad_ch_sbp_sat_42, coriolis_Ch_sbp42,
 *                         vector_advection_Ch_up4_cov)
 *   up4 mass flux ....... .../horizontal/massflux/massflux_ch_mod.f90:61-121
 *   ECS_xy scalar halo .. src/equiang_cs/ecs_halo_factory_mod.f90:70-114,190-270,
 *                         ecs_halo_xy_mod.f90:66-235
 *   vector advection .... .../horizontal/vec_advection/vector_advection_Ch_mod.f90:33-115,
 *                         vector_advection_factory_mod.f90:154-200,
 *                         .../v_dot_nabla/v_nabla_mod.f90:105-146,
 *                         .../Christofel/hor_Christofel_shallow_mod.f90:92-164,
 *                         hor_Christofel_factory_mod.f90:100-134,
 *                         src/metric/metric_2d_ecs_mod.f90:270-335
 *   ECS Ch vector halo .. src/equiang_cs/ecs_halo_vec_Ch_mod.f90:29-150,
 *                         ecs_halo_vec_Ch_factory_mod.f90:21-270,
 *                         src/particles/interpolations/bicubic_interp_mod.f90:27-115
 *   RK4 ................. src/time_schemes/rk4_mod.f90:20-42
 *   stvec algebra ....... src/grid_field_mod.f90:442-534
 *   quadrature .......... src/quadrature/sbp_quadrature_mod.f90:22-62,
 *                         quadrature_factory_mod.f90:89-188
 *   initial conditions .. src/test_fields/test_fields_mod.f90:491-514,586-615,857-894
 *
 * Parity status: no Fortran compiler exists in this environment and the
 * reference ships no golden vectors for this path, so the restatement is
 * pinned by algebraic known-answer properties (see tests/test_oracle.py):
 * exact SAT cancellation, polynomial exactness, discrete SBP adjointness,
 * mass conservation, Coriolis energy neutrality, the linear TS2 steady state.
 *
 * Expression order follows the Fortran statements (left-to-right evaluation,
 * no FMA contraction: build with -ffp-contract=off).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "sbp63.h"
#include "lap63.h"

#define NPAN 6

/* ------------------------------------------------------------------ */
/* cube topology: panel frames (cubed_sphere_topology_mod.f90:29-55)   */
/* ------------------------------------------------------------------ */
static const int T_EX[NPAN][3] = {{-1, 0, 0}, {0, 0, -1}, {1, 0, 0}, {0, 0, 1}, {1, 0, 0}, {1, 0, 0}};
static const int T_EY[NPAN][3] = {{0, 1, 0}, {0, 1, 0}, {0, 1, 0}, {0, 1, 0}, {0, 0, 1}, {0, 0, -1}};
static const int T_N[NPAN][3] = {{0, 0, 1}, {-1, 0, 0}, {0, 0, -1}, {1, 0, 0}, {0, 1, 0}, {0, -1, 0}};
static const int T_R[NPAN][3] = {{1, 0, 0}, {1, 0, 1}, {0, 0, 1}, {0, 0, 0}, {0, 0, 0}, {0, 1, 1}};

static int idot(const int a[3], const int b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* transform_index (cubed_sphere_topology_mod.f90:80-148); panels 0-based */
static void transform_index(int ps, int is_, int js_, int pt, int nx, int ny, int *it, int *jt)
{
    int exl[3] = {0, 0, 0}, eyl[3] = {0, 0, 0}, rl[3] = {0, 0, 0}, sh[2] = {0, 0}, d;
    if (ps == pt) {
        *it = is_;
        *jt = js_;
        return;
    }
    int is_right = idot(T_EX[pt], T_N[ps]) == -1;
    int is_left = idot(T_EX[pt], T_N[ps]) == 1;
    int is_bottom = idot(T_EY[pt], T_N[ps]) == 1;
    int is_top = idot(T_EY[pt], T_N[ps]) == -1;
    int is_opp = idot(T_N[pt], T_N[ps]) == -1;
    if (is_right) {
        for (d = 0; d < 3; d++) { exl[d] = T_N[pt][d]; eyl[d] = T_EY[pt][d]; rl[d] = T_R[pt][d] + T_EX[pt][d]; }
        sh[0] = nx;
    } else if (is_left) {
        for (d = 0; d < 3; d++) { exl[d] = -T_N[pt][d]; eyl[d] = T_EY[pt][d]; }
        for (d = 0; d < 3; d++) rl[d] = T_R[pt][d] - exl[d];
        sh[0] = -nx;
    } else if (is_bottom) {
        for (d = 0; d < 3; d++) { exl[d] = T_EX[pt][d]; eyl[d] = -T_N[pt][d]; rl[d] = T_R[pt][d] + T_N[pt][d]; }
        sh[1] = -ny;
    } else if (is_top) {
        for (d = 0; d < 3; d++) { exl[d] = T_EX[pt][d]; eyl[d] = T_N[pt][d]; rl[d] = T_R[pt][d] + T_EY[pt][d]; }
        sh[1] = ny;
    } else if (is_opp) {
        for (d = 0; d < 3; d++) { exl[d] = -T_EX[pt][d]; eyl[d] = T_EY[pt][d]; rl[d] = T_R[pt][d] + T_EX[pt][d] + T_N[pt][d]; }
        sh[0] = 2 * nx;
    }
    int rdiff[3];
    for (d = 0; d < 3; d++) rdiff[d] = T_R[ps][d] - rl[d];
    int ex_ex = idot(T_EX[ps], exl), ex_ey = idot(T_EY[ps], exl), ex_r = idot(rdiff, exl);
    int ey_ex = idot(T_EX[ps], eyl), ey_ey = idot(T_EY[ps], eyl), ey_r = idot(rdiff, eyl);
    *it = (is_ - 1) * ex_ex + (js_ - 1) * ex_ey + (nx - 1) * ex_r + 1 + sh[0];
    *jt = (is_ - 1) * ey_ex + (js_ - 1) * ey_ey + (ny - 1) * ey_r + 1 + sh[1];
}

/* find_basis_orientation (cubed_sphere_topology_mod.f90:180-239) */
static void basis_orientation(int ps, int pt, int *i_step, int *j_step, char *fdim)
{
    int exl[3] = {0, 0, 0}, eyl[3] = {0, 0, 0}, d;
    if (ps == pt) { *fdim = 'i'; *i_step = 1; *j_step = 1; return; }
    int is_right = idot(T_EX[pt], T_N[ps]) == -1;
    int is_left = idot(T_EX[pt], T_N[ps]) == 1;
    int is_bottom = idot(T_EY[pt], T_N[ps]) == 1;
    int is_top = idot(T_EY[pt], T_N[ps]) == -1;
    int is_opp = idot(T_N[pt], T_N[ps]) == -1;
    for (d = 0; d < 3; d++) {
        if (is_right) { exl[d] = T_N[pt][d]; eyl[d] = T_EY[pt][d]; }
        else if (is_left) { exl[d] = -T_N[pt][d]; eyl[d] = T_EY[pt][d]; }
        else if (is_bottom) { exl[d] = T_EX[pt][d]; eyl[d] = -T_N[pt][d]; }
        else if (is_top) { exl[d] = T_EX[pt][d]; eyl[d] = T_N[pt][d]; }
        else if (is_opp) { exl[d] = -T_EX[pt][d]; eyl[d] = T_EY[pt][d]; }
    }
    int ex_ex = idot(T_EX[ps], exl), ex_ey = idot(T_EY[ps], exl);
    int ey_ex = idot(T_EX[ps], eyl), ey_ey = idot(T_EY[ps], eyl);
    if (ex_ex != 0) { *fdim = 'i'; *i_step = ex_ex; *j_step = ey_ey; }
    else { *fdim = 'j'; *i_step = ex_ey; *j_step = ey_ex; }
}

typedef struct { int is, ie, js, je; } box_t;

static int box_npts(box_t b) { return (b.ie - b.is + 1) * (b.je - b.js + 1); }

/* transform_tile_coords (cubed_sphere_topology_mod.f90:149-178) */
static box_t transform_box(int ps, box_t src, int pt, int nx, int ny)
{
    int i0, j0, i1, j1;
    transform_index(ps, src.is, src.js, pt, nx, ny, &i0, &j0);
    transform_index(ps, src.ie, src.je, pt, nx, ny, &i1, &j1);
    box_t r;
    r.is = i0 < i1 ? i0 : i1; r.ie = i0 < i1 ? i1 : i0;
    r.js = j0 < j1 ? j0 : j1; r.je = j0 < j1 ? j1 : j0;
    return r;
}

static int imax(int a, int b) { return a > b ? a : b; }
static int imin(int a, int b) { return a < b ? a : b; }

/* find_tiles_halo_intersection (exchange_factory_mod.f90:673-723); cross = 'cross' halo type */
static int halo_intersection(box_t t1, int hwx, int hwy, box_t t2, int cross, box_t *out)
{
    box_t o;
    if (!cross) {
        o.is = imax(t1.is - hwx, t2.is); o.ie = imin(t1.ie + hwx, t2.ie);
        o.js = imax(t1.js - hwy, t2.js); o.je = imin(t1.je + hwy, t2.je);
        if (o.is <= o.ie && o.js <= o.je) { *out = o; return 1; }
        return 0;
    }
    o.is = imax(t1.is - hwx, t2.is); o.ie = imin(t1.ie + hwx, t2.ie);
    o.js = imax(t1.js, t2.js); o.je = imin(t1.je, t2.je);
    if (o.is <= o.ie && o.js <= o.je) { *out = o; return 1; }
    o.is = imax(t1.is, t2.is); o.ie = imin(t1.ie, t2.ie);
    o.js = imax(t1.js - hwy, t2.js); o.je = imin(t1.je + hwy, t2.je);
    if (o.is <= o.ie && o.js <= o.je) { *out = o; return 1; }
    return 0;
}

/* ------------------------------------------------------------------ */
/* fields: six panels, interior 1..nx x 1..ny, halo hw                  */
/* ------------------------------------------------------------------ */
typedef struct {
    int nx, ny, hw, ld;
    size_t psz;
    double *p;
} fld_t;

#define FA(f, t, i, j) ((f)->p[(size_t)(t) * (f)->psz + (size_t)((j) + (f)->hw - 1) * (f)->ld + (size_t)((i) + (f)->hw - 1)])

static void fld_init(fld_t *f, int nx, int ny, int hw)
{
    f->nx = nx; f->ny = ny; f->hw = hw; f->ld = nx + 2 * hw;
    f->psz = (size_t)f->ld * (size_t)(ny + 2 * hw);
    f->p = (double *)malloc(sizeof(double) * f->psz * NPAN);
    /* NaN-poisoned halos and interior (as -init=snan): any read of a value
       that no exchange or sweep wrote propagates NaN to the result */
    for (size_t k = 0; k < f->psz * NPAN; k++) f->p[k] = NAN;
}
static void fld_free(fld_t *f) { free(f->p); f->p = NULL; }

/* copy interior from / to the packed host layout (i fastest, then j, then panel) */
static void fld_from_packed(fld_t *f, const double *src)
{
    size_t k = 0;
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= f->ny; j++)
            for (int i = 1; i <= f->nx; i++) FA(f, t, i, j) = src[k++];
}
static void fld_to_packed(const fld_t *f, double *dst)
{
    size_t k = 0;
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= f->ny; j++)
            for (int i = 1; i <= f->nx; i++) dst[k++] = FA(f, t, i, j);
}

/* ------------------------------------------------------------------ */
/* halo exchanges as in-process messages                               */
/* ------------------------------------------------------------------ */
enum { PK_SCALAR = 0, PK_VEC = 1, PK_U_VEC = 2, PK_V_VEC = 3 };

typedef struct {
    int src, dst;      /* panels, 0-based */
    box_t sbox, rbox;  /* send box (src coords), recv box (dst coords) */
    char fdim;
    int istep, jstep;
    int src_from_u;    /* Ch exchanges: 1 if the packed field is the y-mesh one */
} msg_t;

typedef struct {
    int n;
    msg_t m[NPAN * NPAN];
    int pack;          /* PK_* */
    int dst_is_u;      /* Ch exchanges: receiving field (1: y-mesh "u", 0: x-mesh "v") */
} exch_t;

typedef struct {
    int valid;
    box_t b;
    char fdim;
    int is, js;
    int from_u;
} half_t;

static void exch_pair(exch_t *e, half_t send[NPAN][NPAN], half_t recv[NPAN][NPAN])
{
    e->n = 0;
    for (int s = 0; s < NPAN; s++)
        for (int r = 0; r < NPAN; r++) {
            if (s == r) continue;
            if (!send[s][r].valid && !recv[r][s].valid) continue;
            if (send[s][r].valid != recv[r][s].valid ||
                box_npts(send[s][r].b) != box_npts(recv[r][s].b)) {
                fprintf(stderr, "oracle: unmatched halo message %d->%d\n", s, r);
                abort();
            }
            msg_t *m = &e->m[e->n++];
            m->src = s; m->dst = r;
            m->sbox = send[s][r].b; m->rbox = recv[r][s].b;
            m->fdim = send[s][r].fdim; m->istep = send[s][r].is; m->jstep = send[s][r].js;
            m->src_from_u = send[s][r].from_u;
        }
}

/* create_xy_xyz_points_halo_exchange (exchange_factory_mod.f90:197-317) */
static void build_xy_exchange(exch_t *e, int N, int hw, int cross, int pack)
{
    static half_t send[NPAN][NPAN], recv[NPAN][NPAN];
    memset(send, 0, sizeof(send)); memset(recv, 0, sizeof(recv));
    box_t tile = {1, N + 1, 1, N + 1};
    for (int loc = 0; loc < NPAN; loc++)
        for (int rem = 0; rem < NPAN; rem++) {
            if (rem == loc) continue;
            box_t temp = transform_box(rem, tile, loc, N + 1, N + 1);
            box_t b;
            if (halo_intersection(tile, hw, hw, temp, cross, &b)) { recv[loc][rem].valid = 1; recv[loc][rem].b = b; }
            half_t *h = &send[loc][rem];
            basis_orientation(rem, loc, &h->is, &h->js, &h->fdim);
            if (halo_intersection(temp, hw, hw, tile, cross, &b)) { h->valid = 1; h->b = b; }
        }
    exch_pair(e, send, recv);
    e->pack = pack;
}

/* create_symm_halo_vec_exchange_U_points / _V_points (exchange_factory_mod.f90:369-672).
   fill_x: 1 builds exch_u (receives into the x-mesh field), 0 builds exch_v (y-mesh). */
static void build_ch_exchange(exch_t *e, int N, int hw, int cross, int fill_x)
{
    static half_t send[NPAN][NPAN], recv[NPAN][NPAN];
    memset(send, 0, sizeof(send)); memset(recv, 0, sizeof(recv));
    box_t tx = {1, N + 1, 1, N};   /* tiles_x: Nx = N+1, Ny = N */
    box_t ty = {1, N, 1, N + 1};   /* tiles_y: Nx = N,   Ny = N+1 */
    for (int loc = 0; loc < NPAN; loc++)
        for (int rem = 0; rem < NPAN; rem++) {
            if (rem == loc) continue;
            int hwx = hw, hwy = hw;
            char fd; int is, js;
            basis_orientation(rem, loc, &is, &js, &fd);
            box_t b, temp, ltile;
            if (fill_x) {
                ltile = tx;
                box_t rtile = (fd == 'i') ? tx : ty;
                temp = transform_box(rem, rtile, loc, N + 1, N);
                hwx = hw + 1;
                if (halo_intersection(ltile, hwx, hwy, temp, cross, &b)) { recv[loc][rem].valid = 1; recv[loc][rem].b = b; }
                hwx = hw; hwy = hw;
                half_t *h = &send[loc][rem];
                h->fdim = fd; h->is = is; h->js = js;
                if (fd == 'i') {
                    hwx = hw + 1;
                    h->from_u = 0;
                    if (halo_intersection(temp, hwx, hwy, tx, cross, &b)) { h->valid = 1; h->b = b; }
                } else {
                    box_t temp2 = transform_box(rem, tx, loc, N, N + 1);
                    hwy = hw + 1;
                    h->from_u = 1;
                    if (halo_intersection(temp2, hwx, hwy, ty, cross, &b)) { h->valid = 1; h->b = b; }
                }
            } else {
                ltile = ty;
                box_t rtile = (fd == 'i') ? ty : tx;
                temp = transform_box(rem, rtile, loc, N, N + 1);
                hwy = hw + 1;
                if (halo_intersection(ltile, hwx, hwy, temp, cross, &b)) { recv[loc][rem].valid = 1; recv[loc][rem].b = b; }
                hwx = hw; hwy = hw;
                half_t *h = &send[loc][rem];
                h->fdim = fd; h->is = is; h->js = js;
                if (fd == 'i') {
                    hwy = hw + 1;
                    h->from_u = 1;
                    if (halo_intersection(temp, hwx, hwy, ty, cross, &b)) { h->valid = 1; h->b = b; }
                } else {
                    box_t temp2 = transform_box(rem, ty, loc, N + 1, N);
                    hwx = hw + 1;
                    h->from_u = 0;
                    if (halo_intersection(temp2, hwx, hwy, tx, cross, &b)) { h->valid = 1; h->b = b; }
                }
            }
        }
    exch_pair(e, send, recv);
    e->pack = fill_x ? PK_V_VEC : PK_U_VEC;
    e->dst_is_u = fill_x ? 0 : 1;
}

/* create_o_points_halo_exchange -> create_o_z_points_halo_exchange (exchange_factory_mod.f90:13-27,45-150):
   the scalar exchange of the xy points on the cell-centre (o) tiles, N x N per panel. */
static void build_o_exchange(exch_t *e, int N, int hw, int cross)
{
    static half_t send[NPAN][NPAN], recv[NPAN][NPAN];
    memset(send, 0, sizeof(send)); memset(recv, 0, sizeof(recv));
    box_t tile = {1, N, 1, N};
    for (int loc = 0; loc < NPAN; loc++)
        for (int rem = 0; rem < NPAN; rem++) {
            if (rem == loc) continue;
            box_t temp = transform_box(rem, tile, loc, N, N);
            box_t b;
            if (halo_intersection(tile, hw, hw, temp, cross, &b)) { recv[loc][rem].valid = 1; recv[loc][rem].b = b; }
            half_t *h = &send[loc][rem];
            basis_orientation(rem, loc, &h->is, &h->js, &h->fdim);
            if (halo_intersection(temp, hw, hw, tile, cross, &b)) { h->valid = 1; h->b = b; }
        }
    exch_pair(e, send, recv);
    e->pack = PK_SCALAR;
}

/* create_symmetric_halo_vec_exchange_C (exchange_factory_mod.f90:335-350) with the C
   exchange's packing (exchange_halo_C_mod.f90: do_u packs pack_to_buf_u_vec into exch_u,
   do_v packs pack_to_buf_v_vec into exch_v): the tiles are those of the Ch exchange,
   but on C the x-mesh field is u (the alpha component) and the y-mesh field v.
   exch_do(e, u on x, v on y); fill_x 1: exch_u (fills u), 0: exch_v (fills v). */
static void build_c_exchange(exch_t *e, int N, int hw, int fill_x)
{
    build_ch_exchange(e, N, hw, 0, fill_x);
    e->pack = fill_x ? PK_U_VEC : PK_V_VEC;
    e->dst_is_u = fill_x;
}

/* pack traversal: returns the source points in the order of
   pack_to_buf* (buffer_mod.f90:44-476) */
static int pack_order(const msg_t *m, int *ii, int *jj)
{
    box_t b = m->sbox;
    int n = 0;
    if (m->fdim == 'i') {
        for (int jc = 0; jc <= b.je - b.js; jc++) {
            int j = m->jstep > 0 ? b.js + jc : b.je - jc;
            for (int ic = 0; ic <= b.ie - b.is; ic++) {
                int i = m->istep > 0 ? b.is + ic : b.ie - ic;
                ii[n] = i; jj[n] = j; n++;
            }
        }
    } else {
        for (int ic = 0; ic <= b.ie - b.is; ic++) {
            int i = m->istep > 0 ? b.is + ic : b.ie - ic;
            for (int jc = 0; jc <= b.je - b.js; jc++) {
                int j = m->jstep > 0 ? b.js + jc : b.je - jc;
                ii[n] = i; jj[n] = j; n++;
            }
        }
    }
    return n;
}

/* exchange_2D_halo_t%do / do_vec and exchange_2D_halo_Ch_t%do_u / do_v.
   For PK_SCALAR only f1 is used.  For PK_VEC (f1, f2) = (u, v) on the same mesh.
   For Ch exchanges f1 is the y-mesh field (Ch "u") and f2 the x-mesh field; for the C
   exchanges (build_c_exchange) f1 is the x-mesh field (C "u") and f2 the y-mesh field. */
static void exch_do(const exch_t *e, fld_t *f1, fld_t *f2)
{
    for (int k = 0; k < e->n; k++) {
        const msg_t *m = &e->m[k];
        int np = box_npts(m->sbox);
        int *ii = (int *)malloc(sizeof(int) * np), *jj = (int *)malloc(sizeof(int) * np);
        double *b1 = (double *)malloc(sizeof(double) * np), *b2 = (double *)malloc(sizeof(double) * np);
        pack_order(m, ii, jj);
        for (int q = 0; q < np; q++) {
            int i = ii[q], j = jj[q], s = m->src;
            switch (e->pack) {
            case PK_SCALAR: b1[q] = FA(f1, s, i, j); break;
            case PK_VEC:
                if (m->fdim == 'i') { b1[q] = m->istep * FA(f1, s, i, j); b2[q] = m->jstep * FA(f2, s, i, j); }
                else { b1[q] = m->jstep * FA(f2, s, i, j); b2[q] = m->istep * FA(f1, s, i, j); }
                break;
            case PK_U_VEC: /* pack_to_buf_u_vec: 'i' sends u (sign istep), 'j' sends v (sign jstep) */
                if (m->fdim == 'i') b1[q] = m->istep * FA(f1, s, i, j);
                else b1[q] = m->jstep * FA(f2, s, i, j);
                break;
            case PK_V_VEC: /* pack_to_buf_v_vec: 'i' sends v (sign jstep), 'j' sends u (sign istep) */
                if (m->fdim == 'i') b1[q] = m->jstep * FA(f2, s, i, j);
                else b1[q] = m->istep * FA(f1, s, i, j);
                break;
            }
        }
        /* negation by a +-1 integer step: value*(+1) and value*(-1) are exact */
        int q = 0;
        box_t r = m->rbox;
        for (int j = r.js; j <= r.je; j++)
            for (int i = r.is; i <= r.ie; i++, q++) {
                int t = m->dst;
                switch (e->pack) {
                case PK_SCALAR: FA(f1, t, i, j) = b1[q]; break;
                case PK_VEC: FA(f1, t, i, j) = b1[q]; FA(f2, t, i, j) = b2[q]; break;
                case PK_U_VEC: FA(f1, t, i, j) = b1[q]; break;
                case PK_V_VEC: FA(f2, t, i, j) = b1[q]; break;
                }
            }
        free(ii); free(jj); free(b1); free(b2);
    }
}

/* ------------------------------------------------------------------ */
/* metric on the meshes (metric_2d_ecs_mod.f90:338-411)                */
/* ------------------------------------------------------------------ */
typedef struct {
    int nx, ny;
    double shift_i, shift_j, hx, hy;
    double *J, *Q1, *Q2, *Q3, *rx, *ry, *rz; /* [t][j][i] interior, 1-based mapped to 0 */
    double *a1, *a2;                         /* [t][j][i][3] */
    double *b1, *b2;                         /* contravariant basis, [t][j][i][3] */
    double *Ax, *Ay;                         /* SBP norm weights */
} mesh_t;

#define MI(m, t, i, j) ((size_t)(t) * (size_t)(m)->nx * (size_t)(m)->ny + (size_t)((j) - 1) * (m)->nx + (size_t)((i) - 1))

static const double PI_ = 3.141592653589793238462643383279502884;

static void proto2real(int t, const double rp[3], double out[3])
{
    for (int d = 0; d < 3; d++)
        out[d] = T_EX[t][d] * rp[0] + T_EY[t][d] * rp[1] - T_N[t][d] * rp[2];
}

static void a1_proto(double alpha, double beta, double a[3])
{
    double ta = tan(alpha), tb = tan(beta);
    double s = pow(1.0 + pow(ta, 2.0) + pow(tb, 2.0), 1.5);
    a[0] = (1.0 + pow(ta, 2.0)) * (1.0 + pow(tb, 2.0)) / s;
    a[1] = -ta * tb * (1.0 + pow(ta, 2.0)) / s;
    a[2] = -ta * (1.0 + pow(ta, 2.0)) / s;
}
static void a2_proto(double alpha, double beta, double a[3])
{
    double ta = tan(alpha), tb = tan(beta);
    double s = pow(1.0 + pow(ta, 2.0) + pow(tb, 2.0), 1.5);
    a[0] = -ta * tb * (1.0 + pow(tb, 2.0)) / s;
    a[1] = (1.0 + pow(ta, 2.0)) * (1.0 + pow(tb, 2.0)) / s;
    a[2] = -tb * (1.0 + pow(tb, 2.0)) / s;
}
static void b1_proto(double alpha, double beta, double b[3])
{
    double ta = tan(alpha), tb = tan(beta);
    double sg = sqrt(1.0 + ta * ta + tb * tb);
    b[0] = (1.0 + tb * tb - (ta * tb) * (ta * tb) / (1.0 + ta * ta)) / sg;
    b[1] = 0.0;
    b[2] = -ta * (1.0 + tb * tb / (1 + ta * ta)) / sg;
}
static void b2_proto(double alpha, double beta, double b[3])
{
    double ta = tan(alpha), tb = tan(beta);
    double sg = sqrt(1.0 + ta * ta + tb * tb);
    b[0] = 0.0;
    b[1] = ((1 + ta * ta) - (ta * tb) * (ta * tb) / (1 + tb * tb)) / sg;
    b[2] = -tb * (ta * ta / (1 + tb * tb) + 1.0) / sg;
}

/* create_mass_coefficients (quadrature_factory_mod.f90:169-188) */
static void mass_coeffs(double *A, int n, const double *edge, int nedge)
{
    for (int i = 1; i <= n; i++) A[i - 1] = 1.0;
    for (int i = 1; i <= imin(nedge, n); i++) A[i - 1] = edge[i - 1];
    for (int i = imax(n - nedge + 1, 1); i <= n; i++) A[i - 1] = edge[n - i];
}

static const double A42_I[5] = {7.0 / 18.0, 9.0 / 8.0, 1.0, 71.0 / 72.0, 1.0};
static const double A42_C[4] = {13.0 / 12.0, 7.0 / 8.0, 25.0 / 24.0, 1.0};
/* D21_A_interfaces, D21_A_centers (sbp_operators_collection_mod.f90:169-170) */
static const double A21_I[2] = {0.5, 1.0};
static const double A21_C[2] = {1.0, 1.0};

/* quadrature edge weights of the mesh's two directions for SBP order ord */
static void mesh_mass(mesh_t *m, int ord)
{
    /* D63_A_interfaces / D63_A_centers (sbp_operators_collection_mod.f90:199-200) */
    const double *ei = ord == 21 ? A21_I : (ord == 63 ? SBP63_H_I : A42_I);
    const double *ec = ord == 21 ? A21_C : (ord == 63 ? SBP63_H_C : A42_C);
    const int ni = ord == 21 ? 2 : 5, nc = ord == 21 ? 2 : (ord == 63 ? 6 : 4);
    mass_coeffs(m->Ax, m->nx, m->shift_i == 0.0 ? ei : ec, m->shift_i == 0.0 ? ni : nc);
    mass_coeffs(m->Ay, m->ny, m->shift_j == 0.0 ? ei : ec, m->shift_j == 0.0 ? ni : nc);
}

static void mesh_build(mesh_t *m, int N, double shift_i, double shift_j)
{
    m->nx = (shift_i == 0.0) ? N + 1 : N;
    m->ny = (shift_j == 0.0) ? N + 1 : N;
    m->shift_i = shift_i; m->shift_j = shift_j;
    double alpha0 = -0.25 * PI_, alpha1 = 0.25 * PI_;
    m->hx = (alpha1 - alpha0) / ((double)m->nx - 1 + 2.0 * shift_i);
    m->hy = (alpha1 - alpha0) / ((double)m->ny - 1 + 2.0 * shift_j);
    size_t n = (size_t)NPAN * m->nx * m->ny;
    m->J = malloc(sizeof(double) * n); m->Q1 = malloc(sizeof(double) * n);
    m->Q2 = malloc(sizeof(double) * n); m->Q3 = malloc(sizeof(double) * n);
    m->rx = malloc(sizeof(double) * n); m->ry = malloc(sizeof(double) * n); m->rz = malloc(sizeof(double) * n);
    m->a1 = malloc(sizeof(double) * n * 3); m->a2 = malloc(sizeof(double) * n * 3);
    m->b1 = malloc(sizeof(double) * n * 3); m->b2 = malloc(sizeof(double) * n * 3);
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= m->ny; j++) {
            double beta = alpha0 + (j - 1 + shift_j) * m->hy;
            double tb = tan(beta);
            for (int i = 1; i <= m->nx; i++) {
                double alpha = alpha0 + (i - 1 + shift_i) * m->hx;
                double ta = tan(alpha);
                double sigm = sqrt(1.0 + ta * ta + tb * tb);
                double rp[3] = {ta / sigm, tb / sigm, 1.0 / sigm}, r[3];
                proto2real(t, rp, r);
                size_t k = MI(m, t, i, j);
                m->rx[k] = r[0]; m->ry[k] = r[1]; m->rz[k] = r[2];
                double s15 = pow(1.0 + pow(ta, 2.0) + pow(tb, 2.0), 1.5);
                double a1p[3] = {(1.0 + pow(ta, 2.0)) * (1.0 + pow(tb, 2.0)) / s15,
                                 -ta * tb * (1.0 + pow(ta, 2.0)) / s15, -ta * (1.0 + pow(ta, 2.0)) / s15};
                double a2p[3] = {-ta * tb * (1.0 + pow(tb, 2.0)) / s15,
                                 (1.0 + pow(ta, 2.0)) * (1.0 + pow(tb, 2.0)) / s15, -tb * (1.0 + pow(tb, 2.0)) / s15};
                proto2real(t, a1p, &m->a1[3 * k]);
                proto2real(t, a2p, &m->a2[3 * k]);
                double bp[3];
                b1_proto(alpha, beta, bp);
                proto2real(t, bp, &m->b1[3 * k]);
                b2_proto(alpha, beta, bp);
                proto2real(t, bp, &m->b2[3 * k]);
                double s2 = sigm * sigm;
                m->Q1[k] = s2 / (1.0 + ta * ta);
                m->Q2[k] = s2 * ta * tb / ((1 + ta * ta) * (1 + tb * tb));
                m->Q3[k] = s2 / (1.0 + tb * tb);
                m->J[k] = (1.0 + ta * ta) * (1.0 + tb * tb) / (sigm * sigm * sigm);
            }
        }
    m->Ax = malloc(sizeof(double) * m->nx);
    m->Ay = malloc(sizeof(double) * m->ny);
    mesh_mass(m, 42);
}

static void mesh_free(mesh_t *m)
{
    free(m->J); free(m->Q1); free(m->Q2); free(m->Q3); free(m->rx); free(m->ry); free(m->rz);
    free(m->a1); free(m->a2); free(m->b1); free(m->b2); free(m->Ax); free(m->Ay);
}

/* ------------------------------------------------------------------ */
/* SBP 4-2 coefficients (sbp_*_42_mod.f90)                             */
/* ------------------------------------------------------------------ */
/* i2c difference */
static const double DI_h11 = 13.0 / 12.0, DI_h22 = 7.0 / 8.0, DI_h33 = 25.0 / 24.0;
static const double R11 = 15.0 / 8.0, R12 = -5.0 / 4.0, R13 = 3.0 / 8.0;
static const double DI_q11 = -79.0 / 78.0, DI_q12 = 27.0 / 26.0, DI_q13 = -1.0 / 26.0, DI_q14 = 1.0 / 78.0,
                    DI_q21 = 2.0 / 21.0, DI_q22 = -9.0 / 7.0, DI_q23 = 9.0 / 7.0, DI_q24 = -2.0 / 21.0,
                    DI_q31 = 1.0 / 75.0, DI_q33 = -27.0 / 25.0, DI_q34 = 83.0 / 75.0, DI_q35 = -1.0 / 25.0;
/* c2i difference */
static const double DC_h11 = 7.0 / 18.0;
static const double DC_q11 = -2.0, DC_q12 = 3.0, DC_q13 = -1.0, DC_q21 = -1.0, DC_q22 = 1.0,
                    DC_q31 = 1.0 / 24.0, DC_q32 = -9.0 / 8.0, DC_q33 = 9.0 / 8.0, DC_q34 = -1.0 / 24.0,
                    DC_q41 = -1.0 / 71.0, DC_q42 = 6.0 / 71.0, DC_q43 = -83.0 / 71.0, DC_q44 = 81.0 / 71.0,
                    DC_q45 = -3.0 / 71.0;
/* SBP 2-1 (sbp_diff_i2c_21_mod.f90:12-15, sbp_diff_c2i_21_mod.f90:12-15): norms of the
   i2c difference (h11 = h22 = 1) and of the c2i difference (h11 = 1/2), boundary
   projection R11, R12 */
static const double S21_DI_h11 = 1.0, S21_DI_h22 = 1.0, S21_DC_h11 = 0.5;
static const double S21_R11 = 3.0 / 2.0, S21_R12 = -1.0 / 2.0;
/* SBP 6-3: coefficient tables (sbp63.h) and closure-row widths of the i2c and c2i
   operators (sbp_diff_i2c_63_mod.f90:84-134, sbp_diff_c2i_63_mod.f90:82-124) */
static const int S63_WI[6] = {5, 5, 6, 7, 8, 9};
static const int S63_WC[5] = {6, 6, 6, 6, 7};
/* interpolation free parameters */
static const double C13 = 0.1264926207034815, C14 = -0.029892648949074313;
static double II_q[15], IC_q[15];
static int coeffs_ready = 0;
static void init_coeffs(void)
{
    if (coeffs_ready) return;
    double c13 = C13, c14 = C14;
    /* i2c interpolation: q11 q12 q13 q14 q21 q22 q23 q24 q31 q32 q33 q34 q35 */
    II_q[0] = 1.0 / 2.0 + c13 + 2.0 * c14;
    II_q[1] = 1.0 / 2.0 - 2.0 * c13 - 3.0 * c14;
    II_q[2] = c13;
    II_q[3] = c14;
    II_q[4] = -8.0 / 63.0 - 52.0 / 21.0 * c13 - 104.0 / 21.0 * c14;
    II_q[5] = 29.0 / 42.0 + 104.0 / 21.0 * c13 + 52.0 / 7.0 * c14;
    II_q[6] = -52.0 / 21.0 * c13 + 1.0 / 2.0;
    II_q[7] = -52.0 / 21.0 * c14 - 4.0 / 63.0;
    II_q[8] = 26.0 / 25.0 * c13 + 52.0 / 25.0 * c14 - 1.0 / 25.0;
    II_q[9] = -1.0 / 50.0 - 52.0 / 25.0 * c13 - 78.0 / 25.0 * c14;
    II_q[10] = 3.0 / 5.0 + 26.0 / 25.0 * c13;
    II_q[11] = 13.0 / 25.0 + 26.0 / 25.0 * c14;
    II_q[12] = -3.0 / 50.0;
    /* c2i interpolation: q11 q12 q13 q21 q22 q23 q31 q32 q33 q34 q41 q42 q43 q44 q45 */
    IC_q[0] = 39.0 / 28.0 + 39.0 / 14.0 * c13 + 39.0 / 7.0 * c14;
    IC_q[1] = -2.0 / 7.0 - 39.0 / 7.0 * c13 - 78.0 / 7.0 * c14;
    IC_q[2] = 39.0 / 14.0 * c13 + 39.0 / 7.0 * c14 - 3.0 / 28.0;
    IC_q[3] = 13.0 / 27.0 - 52.0 / 27.0 * c13 - 26.0 / 9.0 * c14;
    IC_q[4] = 29.0 / 54.0 + 104.0 / 27.0 * c13 + 52.0 / 9.0 * c14;
    IC_q[5] = -1.0 / 54.0 - 52.0 / 27.0 * c13 - 26.0 / 9.0 * c14;
    IC_q[6] = 13.0 / 12.0 * c13;
    IC_q[7] = -13.0 / 6.0 * c13 + 7.0 / 16.0;
    IC_q[8] = 5.0 / 8.0 + 13.0 / 12.0 * c13;
    IC_q[9] = -1.0 / 16.0;
    IC_q[10] = 78.0 / 71.0 * c14;
    IC_q[11] = -156.0 / 71.0 * c14 - 4.0 / 71.0;
    IC_q[12] = 39.0 / 71.0 + 78.0 / 71.0 * c14;
    IC_q[13] = 81.0 / 142.0;
    IC_q[14] = -9.0 / 142.0;
    coeffs_ready = 1;
}

/* Line accessor: along-direction index k, cross index l.  dir 0 = x (i = k, j = l),
   dir 1 = y (i = l, j = k). */
#define L(f, t, dir, k, l) ((dir) == 0 ? FA(f, t, k, l) : FA(f, t, l, k))

/* sbp_diff_i2c_42_t%apply_tile + add_SAT_correction along dir; out has n = nodes-1 rows.
   ord 21: sbp_diff_i2c_21_t (sbp_diff_i2c_21_mod.f90:25-146). */
static void diff_i2c(fld_t *out, const fld_t *in, int t, int dir, int n, int ls, int le, int ord)
{
#define O(k) (*((dir) == 0 ? &FA(out, t, k, l) : &FA(out, t, l, k)))
#define I(k) L(in, t, dir, k, l)
    if (ord == 63) {
        /* sbp_diff_i2c_63_mod.f90:84-134 (rows), :335-395 (SAT on rows 1..4) */
        const double *C = SBP63_DI_C;
        for (int l = ls; l <= le; l++) {
            for (int r = 1; r <= 6; r++) {
                double a = 0.0, b = 0.0;
                for (int j = 0; j < S63_WI[r - 1]; j++) {
                    a += SBP63_DI_Q[r - 1][j] * I(j + 1);
                    b -= SBP63_DI_Q[r - 1][j] * I(n + 1 - j);
                }
                O(r) = a;
                O(n + 1 - r) = b;
            }
            for (int k = 7; k <= n - 6; k++)
                O(k) = C[0] * (I(k + 1) - I(k)) + C[1] * (I(k + 2) - I(k - 1)) + C[2] * (I(k + 3) - I(k - 2));
        }
        for (int l = ls; l <= le; l++)
            for (int r = 1; r <= 4; r++) {
                O(r) = O(r) + 0.5 * SBP63_R[r - 1] / SBP63_H_C[r - 1] * (I(1) - I(0));
                O(n + 1 - r) = O(n + 1 - r) + 0.5 * SBP63_R[r - 1] / SBP63_H_C[r - 1] * (I(n + 2) - I(n + 1));
            }
        return;
    }
    if (ord == 21) {
        for (int l = ls; l <= le; l++)
            for (int k = 1; k <= n; k++) O(k) = I(k + 1) - I(k);
        for (int l = ls; l <= le; l++) {
            O(1) = O(1) + 0.5 * S21_R11 / S21_DI_h11 * (I(1) - I(0));
            O(2) = O(2) + 0.5 * S21_R12 / S21_DI_h22 * (I(1) - I(0));
            O(n) = O(n) + 0.5 * S21_R11 / S21_DI_h11 * (I(n + 2) - I(n + 1));
            O(n - 1) = O(n - 1) + 0.5 * S21_R12 / S21_DI_h22 * (I(n + 2) - I(n + 1));
        }
        return;
    }
    for (int l = ls; l <= le; l++) {
        O(1) = DI_q11 * I(1) + DI_q12 * I(2) + DI_q13 * I(3) + DI_q14 * I(4);
        O(2) = DI_q21 * I(1) + DI_q22 * I(2) + DI_q23 * I(3) + DI_q24 * I(4);
        O(3) = DI_q31 * I(1) + DI_q33 * I(3) + DI_q34 * I(4) + DI_q35 * I(5);
        for (int k = 4; k <= n - 3; k++) O(k) = (27.0 * (I(k + 1) - I(k)) - (I(k + 2) - I(k - 1))) / 24.0;
        O(n - 2) = -DI_q31 * I(n + 1) - DI_q33 * I(n - 1) - DI_q34 * I(n - 2) - DI_q35 * I(n - 3);
        O(n - 1) = -DI_q21 * I(n + 1) - DI_q22 * I(n) - DI_q23 * I(n - 1) - DI_q24 * I(n - 2);
        O(n) = -DI_q11 * I(n + 1) - DI_q12 * I(n) - DI_q13 * I(n - 1) - DI_q14 * I(n - 2);
    }
    /* SAT (sbp_diff_i2c_42_mod.f90:162-274), applied after all rows */
    for (int l = ls; l <= le; l++) {
        O(1) = O(1) + 0.5 * R11 / DI_h11 * (I(1) - I(0));
        O(2) = O(2) + 0.5 * R12 / DI_h22 * (I(1) - I(0));
        O(3) = O(3) + 0.5 * R13 / DI_h33 * (I(1) - I(0));
        O(n) = O(n) + 0.5 * R11 / DI_h11 * (I(n + 2) - I(n + 1));
        O(n - 1) = O(n - 1) + 0.5 * R12 / DI_h22 * (I(n + 2) - I(n + 1));
        O(n - 2) = O(n - 2) + 0.5 * R13 / DI_h33 * (I(n + 2) - I(n + 1));
    }
}

/* sbp_diff_c2i_42_t%apply_tile + add_SAT_correction; out has nx = centres+1 rows.
   ord 21: sbp_diff_c2i_21_t (sbp_diff_c2i_21_mod.f90:24-146). */
static void diff_c2i(fld_t *out, const fld_t *in, int t, int dir, int nx, int ls, int le, int ord)
{
    if (ord == 63) {
        /* sbp_diff_c2i_63_mod.f90:82-124 (rows), :267-327 (SAT) */
        const double *C = SBP63_DC_C;
        for (int l = ls; l <= le; l++) {
            for (int r = 1; r <= 5; r++) {
                double a = 0.0, b = 0.0;
                for (int j = 0; j < S63_WC[r - 1]; j++) {
                    a += SBP63_DC_Q[r - 1][j] * I(j + 1);
                    b -= SBP63_DC_Q[r - 1][j] * I(nx - 1 - j);
                }
                O(r) = a;
                O(nx + 1 - r) = b;
            }
            for (int k = 6; k <= nx - 5; k++)
                O(k) = C[0] * (I(k) - I(k - 1)) + C[1] * (I(k + 1) - I(k - 2)) + C[2] * (I(k + 2) - I(k - 3));
        }
        for (int l = ls; l <= le; l++) {
            double s1 = 0.0, s2 = 0.0;
            for (int k = 1; k <= 4; k++) {
                s1 += SBP63_R[k - 1] * (I(k) - I(1 - k));
                s2 += SBP63_R[k - 1] * (I(nx - 1 + k) - I(nx - k));
            }
            O(1) = O(1) + 0.5 / SBP63_H_I[0] * s1;
            O(nx) = O(nx) + 0.5 / SBP63_H_I[0] * s2;
        }
        return;
    }
    if (ord == 21) {
        for (int l = ls; l <= le; l++) {
            O(1) = I(2) - I(1);
            for (int k = 2; k <= nx - 1; k++) O(k) = I(k) - I(k - 1);
            O(nx) = I(nx - 1) - I(nx - 2);
        }
        for (int l = ls; l <= le; l++) {
            O(1) = O(1) + 0.5 / S21_DC_h11 * (S21_R11 * (I(1) - I(0)) + S21_R12 * (I(2) - I(-1)));
            O(nx) = O(nx) - 0.5 / S21_DC_h11 * (S21_R11 * (I(nx - 1) - I(nx)) + S21_R12 * (I(nx - 2) - I(nx + 1)));
        }
        return;
    }
    for (int l = ls; l <= le; l++) {
        O(1) = DC_q11 * I(1) + DC_q12 * I(2) + DC_q13 * I(3);
        O(2) = DC_q21 * I(1) + DC_q22 * I(2);
        O(3) = DC_q31 * I(1) + DC_q32 * I(2) + DC_q33 * I(3) + DC_q34 * I(4);
        O(4) = DC_q41 * I(1) + DC_q42 * I(2) + DC_q43 * I(3) + DC_q44 * I(4) + DC_q45 * I(5);
        for (int k = 5; k <= nx - 4; k++) O(k) = (27.0 * (I(k) - I(k - 1)) - (I(k + 1) - I(k - 2))) / 24.0;
        O(nx - 3) = -DC_q41 * I(nx - 1) - DC_q42 * I(nx - 2) - DC_q43 * I(nx - 3) - DC_q44 * I(nx - 4) - DC_q45 * I(nx - 5);
        O(nx - 2) = -DC_q31 * I(nx - 1) - DC_q32 * I(nx - 2) - DC_q33 * I(nx - 3) - DC_q34 * I(nx - 4);
        O(nx - 1) = -DC_q21 * I(nx - 1) - DC_q22 * I(nx - 2);
        O(nx) = -DC_q11 * I(nx - 1) - DC_q12 * I(nx - 2) - DC_q13 * I(nx - 3);
    }
    for (int l = ls; l <= le; l++) {
        O(1) = O(1) + 0.5 / DC_h11 * (R11 * (I(1) - I(0)) + R12 * (I(2) - I(-1)) + R13 * (I(3) - I(-2)));
        O(nx) = O(nx) - 0.5 / DC_h11 * (R11 * (I(nx - 1) - I(nx)) + R12 * (I(nx - 2) - I(nx + 1)) + R13 * (I(nx - 3) - I(nx + 2)));
    }
}

/* sbp_interp_i2c_42_t%apply_tile; out has n centres.
   ord 21: sbp_interp_i2c_21_t (sbp_interp_i2c_21_mod.f90:17-56). */
static void interp_i2c(fld_t *out, const fld_t *in, int t, int dir, int n, int ls, int le, int ord)
{
    if (ord == 63) {
        /* sbp_interp_i2c_63_mod.f90:82-130 */
        const double *C = SBP63_II_C;
        for (int l = ls; l <= le; l++) {
            for (int r = 1; r <= 6; r++) {
                double a = 0.0, b = 0.0;
                for (int j = 0; j < S63_WI[r - 1]; j++) {
                    a += SBP63_II_Q[r - 1][j] * I(j + 1);
                    b += SBP63_II_Q[r - 1][j] * I(n + 1 - j);
                }
                O(r) = a;
                O(n + 1 - r) = b;
            }
            for (int k = 7; k <= n - 6; k++)
                O(k) = C[0] * (I(k + 1) + I(k)) + C[1] * (I(k + 2) + I(k - 1)) + C[2] * (I(k + 3) + I(k - 2));
        }
        return;
    }
    if (ord == 21) {
        for (int l = ls; l <= le; l++)
            for (int k = 1; k <= n; k++) O(k) = 0.5 * (I(k + 1) + I(k));
        return;
    }
    const double *q = II_q;
    for (int l = ls; l <= le; l++) {
        O(1) = q[0] * I(1) + q[1] * I(2) + q[2] * I(3) + q[3] * I(4);
        O(2) = q[4] * I(1) + q[5] * I(2) + q[6] * I(3) + q[7] * I(4);
        O(3) = q[8] * I(1) + q[9] * I(2) + q[10] * I(3) + q[11] * I(4) + q[12] * I(5);
        for (int k = 4; k <= n - 3; k++) O(k) = (9.0 * (I(k + 1) + I(k)) - (I(k + 2) + I(k - 1))) / 16.0;
        O(n - 2) = q[8] * I(n + 1) + q[9] * I(n) + q[10] * I(n - 1) + q[11] * I(n - 2) + q[12] * I(n - 3);
        O(n - 1) = q[4] * I(n + 1) + q[5] * I(n) + q[6] * I(n - 1) + q[7] * I(n - 2);
        O(n) = q[0] * I(n + 1) + q[1] * I(n) + q[2] * I(n - 1) + q[3] * I(n - 2);
    }
}

/* sbp_interp_c2i_42_t%apply_tile; out has nx = centres+1 nodes.
   ord 21: sbp_interp_c2i_21_t (sbp_interp_c2i_21_mod.f90:17-84). */
static void interp_c2i(fld_t *out, const fld_t *in, int t, int dir, int nx, int ls, int le, int ord)
{
    if (ord == 63) {
        /* sbp_interp_c2i_63_mod.f90:70-112 */
        const double *C = SBP63_IC_C;
        for (int l = ls; l <= le; l++) {
            for (int r = 1; r <= 5; r++) {
                double a = 0.0, b = 0.0;
                for (int j = 0; j < S63_WC[r - 1]; j++) {
                    a += SBP63_IC_Q[r - 1][j] * I(j + 1);
                    b += SBP63_IC_Q[r - 1][j] * I(nx - 1 - j);
                }
                O(r) = a;
                O(nx + 1 - r) = b;
            }
            for (int k = 6; k <= nx - 5; k++)
                O(k) = C[0] * (I(k) + I(k - 1)) + C[1] * (I(k + 1) + I(k - 2)) + C[2] * (I(k + 2) + I(k - 3));
        }
        return;
    }
    if (ord == 21) {
        for (int l = ls; l <= le; l++) {
            O(1) = I(1);
            for (int k = 2; k <= nx - 1; k++) O(k) = 0.5 * (I(k) + I(k - 1));
            O(nx) = I(nx - 1);
        }
        return;
    }
    const double *q = IC_q;
    for (int l = ls; l <= le; l++) {
        O(1) = q[0] * I(1) + q[1] * I(2) + q[2] * I(3);
        O(2) = q[3] * I(1) + q[4] * I(2) + q[5] * I(3);
        O(3) = q[6] * I(1) + q[7] * I(2) + q[8] * I(3) + q[9] * I(4);
        O(4) = q[10] * I(1) + q[11] * I(2) + q[12] * I(3) + q[13] * I(4) + q[14] * I(5);
        for (int k = 5; k <= nx - 4; k++) O(k) = (9.0 * (I(k) + I(k - 1)) - (I(k + 1) + I(k - 2))) / 16.0;
        O(nx - 3) = q[10] * I(nx - 1) + q[11] * I(nx - 2) + q[12] * I(nx - 3) + q[13] * I(nx - 4) + q[14] * I(nx - 5);
        O(nx - 2) = q[6] * I(nx - 1) + q[7] * I(nx - 2) + q[8] * I(nx - 3) + q[9] * I(nx - 4);
        O(nx - 1) = q[3] * I(nx - 1) + q[4] * I(nx - 2) + q[5] * I(nx - 3);
        O(nx) = q[0] * I(nx - 1) + q[1] * I(nx - 2) + q[2] * I(nx - 3);
    }
#undef O
#undef I
}

/* ------------------------------------------------------------------ */
/* context                                                              */
/* ------------------------------------------------------------------ */
typedef struct orc_ctx {
    int N;
    int ord;                     /* SBP order of the Ch operators: 42 (default) or 21 */
    double a, g, omega, H, axis[3];
    int coriolis_const;
    mesh_t mxy, mx, my;          /* xy (h), x (v), y (u) */
    double *fJ2;                 /* on xy, [t][j][i] */
    double *qb, *qt, *ql, *qr;   /* covariant ECS Ah sync weights, length N+1 */
    exch_t ex_xy3_full_s, ex_xy3_full_v, ex_xy1_full_s, ex_xy1_cross_v;
    exch_t ex_ch3_u, ex_ch3_v;   /* Ch: fills x-mesh field / y-mesh field */
    exch_t ex_ch4_u, ex_ch4_v;   /* width 4: the SBP 6-3 divergence SAT reads four halo depths */
    /* work fields */
    fld_t h, u, v, du, dv, dh;
    fld_t gx, gy, ut, vt, uq, vq, up, vp, Ju, Jv, Dx, Dy, div;
    fld_t k[4][3], y[3];
    /* advective operator */
    int nonlinear;
    exch_t ex_xy5_full_s, ex_ch1c_u, ex_ch1c_v;
    fld_t htot, hu, hv, cu, cv, uh, vh, vau, uav, uhal, vhal;
    double *hsurf;               /* orography h_surf on xy, [t][j][i]; NULL: none */
    /* C staggering (h on o, u on x, v on y): operators of the C-grid configurations, built
       on first use */
    int cgrid;
    exch_t ex_o3, ex_c3_u, ex_c3_v;
    fld_t c_h, c_u, c_v, c_gx, c_gy, c_ut, c_vt, c_uh, c_vh, c_Ju, c_Jv, c_Dx, c_Dy, c_div;
    /* energies and enstrophy of swm_output_diag_t: mesh o (cell centres, the Ch q mesh) */
    mesh_t mo;
    double *fo;                  /* Coriolis parameter on o, [t][j][i] */
    /* lat-lon regrid of an o field (the curl output): the o-point exchange of width 5 and
       the field with its ECS_O halo, built on first use */
    int llo;
    exch_t ex_o5;
    fld_t o_ll;
    fld_t oDx, oDy, curl, hqu, hqv, ehu, ehv;
    /* Ah staggering (h, u, v all on xy): state, work fields and RK4 stages */
    int ah;
    double *fxy;                 /* Coriolis parameter on xy, [t][j][i] */
    fld_t ah_u, ah_v, ah_du, ah_dv, ah_gx, ah_gy, ah_ut, ah_vt, ah_Ju, ah_Jv, ah_y[3], ah_k[4][3];
    /* diffusion on the Ah staggering (allocated on first use) */
    fld_t df_d1x, df_d1y, df_d2x, df_d2y, df_dxy, df_dyx, df_x[3], df_t[3];
} orc_ctx;

/* calc_coriolis_parameter (coriolis_factory_mod.f90:239-280) at point k of mesh m */
static double coriolis_f(const orc_ctx *c, const mesh_t *m, size_t k)
{
    if (c->coriolis_const) return c->omega;
    double nv[3] = {m->rx[k], m->ry[k], m->rz[k]};
    double pr = (c->axis[0] * nv[0] + c->axis[1] * nv[1] + c->axis[2] * nv[2]) /
                sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
    return 2 * c->omega * pr;
}

static void coriolis_parameter(orc_ctx *c)
{
    mesh_t *m = &c->mxy;
    size_t n = (size_t)NPAN * m->nx * m->ny;
    c->fJ2 = malloc(sizeof(double) * n);
    for (size_t k = 0; k < n; k++) {
        /* multiply_by_J_self applied twice (coriolis_factory_mod.f90:188-193) */
        c->fJ2[k] = coriolis_f(c, m, k) * m->J[k] * m->J[k];
    }
    const mesh_t *o = &c->mo;
    const size_t no = (size_t)NPAN * o->nx * o->ny;
    c->fo = malloc(sizeof(double) * no);
    for (size_t k = 0; k < no; k++) c->fo[k] = coriolis_f(c, o, k);
    c->fxy = malloc(sizeof(double) * n);
    for (size_t k = 0; k < n; k++) c->fxy[k] = coriolis_f(c, m, k);
}

static void sync_weights(orc_ctx *c)
{
    int n = c->N + 1;
    double hx = c->mxy.hx, q = 0.25 * PI_;
    c->qb = malloc(sizeof(double) * n); c->qt = malloc(sizeof(double) * n);
    c->ql = malloc(sizeof(double) * n); c->qr = malloc(sizeof(double) * n);
    for (int i = 1; i <= n; i++) {
        double al = -0.25 * PI_ + (i - 1) * hx, a[3], v[3], b[3];
        a2_proto(al, -q, a); b1_proto(al, q, v);
        b[0] = v[0]; b[1] = -v[2]; b[2] = v[1];
        c->qb[i - 1] = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
        a2_proto(al, q, a); b1_proto(al, -q, v);
        b[0] = v[0]; b[1] = v[2]; b[2] = -v[1];
        c->qt[i - 1] = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    }
    for (int j = 1; j <= n; j++) {
        double be = -0.25 * PI_ + (j - 1) * hx, a[3], v[3], b[3];
        a1_proto(-q, be, a); b2_proto(q, be, v);
        b[0] = -v[2]; b[1] = v[1]; b[2] = v[0];
        c->ql[j - 1] = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
        a1_proto(q, be, a); b2_proto(-q, be, v);
        b[0] = v[2]; b[1] = v[1]; b[2] = -v[0];
        c->qr[j - 1] = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    }
}

orc_ctx *orc_create(int N, double radius, double grav, double omega, double h_mean,
                    const double *axis, int coriolis_const)
{
    if (N < 8) return NULL;
    init_coeffs();
    orc_ctx *c = calloc(1, sizeof(orc_ctx));
    c->N = N; c->a = radius; c->g = grav; c->omega = omega; c->H = h_mean;
    c->axis[0] = axis ? axis[0] : 0.0; c->axis[1] = axis ? axis[1] : 0.0; c->axis[2] = axis ? axis[2] : 1.0;
    c->coriolis_const = coriolis_const;
    c->ord = 42;
    mesh_build(&c->mxy, N, 0.0, 0.0);
    mesh_build(&c->mx, N, 0.0, 0.5);
    mesh_build(&c->my, N, 0.5, 0.0);
    mesh_build(&c->mo, N, 0.5, 0.5);
    coriolis_parameter(c);
    sync_weights(c);
    build_xy_exchange(&c->ex_xy3_full_s, N, 3, 0, PK_SCALAR);
    build_xy_exchange(&c->ex_xy3_full_v, N, 3, 0, PK_VEC);
    build_xy_exchange(&c->ex_xy1_full_s, N, 1, 0, PK_SCALAR);
    build_xy_exchange(&c->ex_xy1_cross_v, N, 1, 1, PK_VEC);
    build_ch_exchange(&c->ex_ch3_u, N, 3, 0, 1);
    build_ch_exchange(&c->ex_ch3_v, N, 3, 0, 0);
    build_ch_exchange(&c->ex_ch4_u, N, 4, 0, 1);
    build_ch_exchange(&c->ex_ch4_v, N, 4, 0, 0);
    build_xy_exchange(&c->ex_xy5_full_s, N, 5, 0, PK_SCALAR);
    build_ch_exchange(&c->ex_ch1c_u, N, 1, 1, 1);
    build_ch_exchange(&c->ex_ch1c_v, N, 1, 1, 0);
    int hw = 5;
    fld_t *xy[] = {&c->h, &c->dh, &c->uq, &c->vq, &c->up, &c->vp, &c->Dx, &c->Dy, &c->div, &c->htot, &c->uh, &c->vh};
    fld_t *yy[] = {&c->u, &c->du, &c->gx, &c->ut, &c->Ju, &c->hu, &c->cu, &c->vau, &c->uhal};
    fld_t *xx[] = {&c->v, &c->dv, &c->gy, &c->vt, &c->Jv, &c->hv, &c->cv, &c->uav, &c->vhal};
    for (unsigned q = 0; q < sizeof(xy) / sizeof(xy[0]); q++) fld_init(xy[q], N + 1, N + 1, hw);
    for (unsigned q = 0; q < sizeof(yy) / sizeof(yy[0]); q++) fld_init(yy[q], N, N + 1, hw);
    for (unsigned q = 0; q < sizeof(xx) / sizeof(xx[0]); q++) fld_init(xx[q], N + 1, N, hw);
    for (int s = 0; s < 4; s++) {
        fld_init(&c->k[s][0], N + 1, N + 1, hw);
        fld_init(&c->k[s][1], N, N + 1, hw);
        fld_init(&c->k[s][2], N + 1, N, hw);
    }
    fld_init(&c->y[0], N + 1, N + 1, hw);
    fld_init(&c->y[1], N, N + 1, hw);
    fld_init(&c->y[2], N + 1, N, hw);
    fld_t *oo[] = {&c->oDx, &c->oDy, &c->curl, &c->hqu, &c->hqv};
    for (unsigned q = 0; q < sizeof(oo) / sizeof(oo[0]); q++) fld_init(oo[q], N, N, hw);
    fld_init(&c->ehu, N, N + 1, hw);
    fld_init(&c->ehv, N + 1, N, hw);
    fld_t *ah[] = {&c->ah_u, &c->ah_v, &c->ah_du, &c->ah_dv, &c->ah_gx, &c->ah_gy, &c->ah_ut, &c->ah_vt,
                   &c->ah_Ju, &c->ah_Jv, &c->ah_y[0], &c->ah_y[1], &c->ah_y[2]};
    for (unsigned q = 0; q < sizeof(ah) / sizeof(ah[0]); q++) fld_init(ah[q], N + 1, N + 1, hw);
    for (int s = 0; s < 4; s++)
        for (int f = 0; f < 3; f++) fld_init(&c->ah_k[s][f], N + 1, N + 1, hw);
    return c;
}

static void c_free(orc_ctx *c);

void orc_destroy(orc_ctx *c)
{
    if (!c) return;
    mesh_free(&c->mxy); mesh_free(&c->mx); mesh_free(&c->my); mesh_free(&c->mo);
    free(c->fJ2); free(c->fo); free(c->fxy); free(c->qb); free(c->qt); free(c->ql); free(c->qr);
    free(c->hsurf);
    c_free(c);
    if (c->llo) fld_free(&c->o_ll);
    fld_t *all[] = {&c->h, &c->u, &c->v, &c->du, &c->dv, &c->dh, &c->gx, &c->gy, &c->ut, &c->vt,
                    &c->uq, &c->vq, &c->up, &c->vp, &c->Ju, &c->Jv, &c->Dx, &c->Dy, &c->div,
                    &c->y[0], &c->y[1], &c->y[2], &c->htot, &c->hu, &c->hv, &c->cu, &c->cv, &c->uh,
                    &c->vh, &c->vau, &c->uav, &c->uhal, &c->vhal, &c->oDx, &c->oDy, &c->curl,
                    &c->hqu, &c->hqv, &c->ehu, &c->ehv, &c->ah_u, &c->ah_v, &c->ah_du, &c->ah_dv,
                    &c->ah_gx, &c->ah_gy, &c->ah_ut, &c->ah_vt, &c->ah_Ju, &c->ah_Jv,
                    &c->ah_y[0], &c->ah_y[1], &c->ah_y[2]};
    for (unsigned q = 0; q < sizeof(all) / sizeof(all[0]); q++) fld_free(all[q]);
    for (int s = 0; s < 4; s++) for (int f = 0; f < 3; f++) { fld_free(&c->k[s][f]); fld_free(&c->ah_k[s][f]); }
    fld_t *df[] = {&c->df_d1x, &c->df_d1y, &c->df_d2x, &c->df_d2y, &c->df_dxy, &c->df_dyx,
                   &c->df_x[0], &c->df_x[1], &c->df_x[2], &c->df_t[0], &c->df_t[1], &c->df_t[2]};
    for (unsigned q = 0; q < sizeof(df) / sizeof(df[0]); q++) fld_free(df[q]);
    free(c);
}

/* ------------------------------------------------------------------ */
/* operators                                                            */
/* ------------------------------------------------------------------ */

/* grad_sbp_sat_t%calc_grad (grad_sbp_sat_mod.f90:24-76): gx on y-mesh, gy on x-mesh */
static void op_grad(orc_ctx *c, fld_t *gx, fld_t *gy, fld_t *h)
{
    int N = c->N;
    exch_do(&c->ex_xy3_full_s, h, NULL);
    for (int t = 0; t < NPAN; t++) {
        diff_i2c(gx, h, t, 0, N, 1, N + 1, c->ord);
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N; i++) FA(gx, t, i, j) = FA(gx, t, i, j) / (c->my.hx * c->a);
        diff_i2c(gy, h, t, 1, N, 1, N + 1, c->ord);
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N + 1; i++) FA(gy, t, i, j) = FA(gy, t, i, j) / (c->mx.hy * c->a);
    }
}

/* co2contra_ch_sbp_t%transform (co2contra_Ch_mod.f90:27-94) */
static void op_co2contra(orc_ctx *c, fld_t *ut, fld_t *vt, fld_t *u, fld_t *v)
{
    int N = c->N;
    /* interp_uv2p_C_sbp (interpolator_uv2p_mod.f90:22-49) */
    exch_do(&c->ex_ch3_u, u, v);
    exch_do(&c->ex_ch3_v, u, v);
    for (int t = 0; t < NPAN; t++) {
        interp_c2i(&c->uq, u, t, 0, N + 1, 1, N + 1, c->ord);
        interp_c2i(&c->vq, v, t, 1, N + 1, 1, N + 1, c->ord);
    }
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N + 1; i++) {
                size_t k = MI(&c->mxy, t, i, j);
                double uu = FA(&c->uq, t, i, j) * c->mxy.J[k] * c->mxy.Q2[k];
                double vv = FA(&c->vq, t, i, j) * c->mxy.J[k] * c->mxy.Q2[k];
                FA(&c->uq, t, i, j) = vv;
                FA(&c->vq, t, i, j) = uu;
            }
    /* interp_pvec2uv_Ch (interpolator_p2uv_mod.f90:71-99) */
    exch_do(&c->ex_xy3_full_v, &c->uq, &c->vq);
    for (int t = 0; t < NPAN; t++) {
        interp_i2c(ut, &c->uq, t, 0, N, 1, N + 1, c->ord);
        interp_i2c(vt, &c->vq, t, 1, N, 1, N + 1, c->ord);
    }
    for (int t = 0; t < NPAN; t++) {
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N; i++) {
                size_t k = MI(&c->my, t, i, j);
                FA(ut, t, i, j) = c->my.Q1[k] * FA(u, t, i, j) + FA(ut, t, i, j) / c->my.J[k];
            }
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N + 1; i++) {
                size_t k = MI(&c->mx, t, i, j);
                FA(vt, t, i, j) = c->mx.Q3[k] * FA(v, t, i, j) + FA(vt, t, i, j) / c->mx.J[k];
            }
    }
}

/* syncronize_grad_on_edges (ecs_Ah_vec_sync_mod.f90:62-125) with (U, V) as passed */
static void sync_grad_on_edges(orc_ctx *c, fld_t *U, fld_t *V, int t)
{
    int n = c->N + 1, is = 1, ie = n, js = 1, je = n;
    const double *qb = c->qb, *qt = c->qt, *ql = c->ql, *qr = c->qr;
#define Q_(a, i) (a)[(i) - 1]
    FA(U, t, 1, 1) = (FA(U, t, 1, 1) + FA(U, t, 0, 1) + FA(U, t, 1, 0) + Q_(qb, 1) * FA(V, t, 1, 0)) / 3.0;
    FA(V, t, 1, 1) = (FA(V, t, 1, 1) + FA(V, t, 0, 1) + FA(V, t, 1, 0) + Q_(ql, 1) * FA(U, t, 0, 1)) / 3.0;
    FA(U, t, ie, 1) = (FA(U, t, ie, 1) + FA(U, t, ie + 1, 1) + FA(U, t, ie, 0) + Q_(qb, ie) * FA(V, t, ie, 0)) / 3.0;
    FA(V, t, ie, 1) = (FA(V, t, ie, 1) + FA(V, t, ie + 1, 1) + FA(V, t, ie, 0) + Q_(qr, 1) * FA(U, t, ie + 1, 1)) / 3.0;
    FA(U, t, 1, je) = (FA(U, t, 1, je) + FA(U, t, 0, je) + FA(U, t, 1, je + 1) + Q_(qt, 1) * FA(V, t, 1, je + 1)) / 3.0;
    FA(V, t, 1, je) = (FA(V, t, 1, je) + FA(V, t, 0, je) + FA(V, t, 1, je + 1) + Q_(ql, je) * FA(U, t, 0, je)) / 3.0;
    FA(U, t, ie, je) = (FA(U, t, ie, je) + FA(U, t, ie + 1, je) + FA(U, t, ie, je + 1) + Q_(qt, ie) * FA(V, t, ie, je + 1)) / 3.0;
    FA(V, t, ie, je) = (FA(V, t, ie, je) + FA(V, t, ie + 1, je) + FA(V, t, ie, je + 1) + Q_(qr, je) * FA(U, t, ie + 1, je)) / 3.0;
    for (int j = imax(js, 2); j <= imin(je, n - 1); j++) {
        FA(U, t, 1, j) = 0.5 * (FA(U, t, 0, j) + FA(U, t, 1, j));
        FA(V, t, 1, j) = 0.5 * (FA(V, t, 1, j) + FA(V, t, 0, j) + Q_(ql, j) * FA(U, t, 0, j));
    }
    for (int j = imax(js, 2); j <= imin(je, n - 1); j++) {
        FA(U, t, ie, j) = 0.5 * (FA(U, t, ie, j) + FA(U, t, ie + 1, j));
        FA(V, t, ie, j) = 0.5 * (FA(V, t, ie, j) + FA(V, t, ie + 1, j) + Q_(qr, j) * FA(U, t, ie + 1, j));
    }
    for (int i = imax(is, 2); i <= imin(ie, n - 1); i++) {
        FA(V, t, i, 1) = 0.5 * (FA(V, t, i, 0) + FA(V, t, i, 1));
        FA(U, t, i, 1) = 0.5 * (FA(U, t, i, 0) + FA(U, t, i, 1) + Q_(qb, i) * FA(V, t, i, 0));
    }
    for (int i = imax(is, 2); i <= imin(ie, n - 1); i++) {
        FA(V, t, i, je) = 0.5 * (FA(V, t, i, je) + FA(V, t, i, je + 1));
        FA(U, t, i, je) = 0.5 * (FA(U, t, i, je) + FA(U, t, i, je + 1) + Q_(qt, i) * FA(V, t, i, je + 1));
    }
#undef Q_
}

/* coriolis_Ch_t%calc_coriolis (coriolis_Ch_mod.f90:42-69,97-120) */
static void op_coriolis(orc_ctx *c, fld_t *cu, fld_t *cv, fld_t *ut, fld_t *vt)
{
    int N = c->N;
    exch_do(&c->ex_ch3_u, ut, vt);
    exch_do(&c->ex_ch3_v, ut, vt);
    for (int t = 0; t < NPAN; t++) {
        interp_c2i(&c->up, ut, t, 0, N + 1, 1, N + 1, c->ord);
        interp_c2i(&c->vp, vt, t, 1, N + 1, 1, N + 1, c->ord);
    }
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N + 1; i++) {
                double f = c->fJ2[MI(&c->mxy, t, i, j)];
                double tu = f * FA(&c->vp, t, i, j);
                double tv = -f * FA(&c->up, t, i, j);
                FA(&c->up, t, i, j) = tu;
                FA(&c->vp, t, i, j) = tv;
            }
    /* ecs_Ah_vec_sync_covariant: exchange (up, vp) then sync with (U, V) = (vp, up) */
    exch_do(&c->ex_xy1_cross_v, &c->up, &c->vp);
    for (int t = 0; t < NPAN; t++) sync_grad_on_edges(c, &c->vp, &c->up, t);
    exch_do(&c->ex_xy3_full_v, &c->up, &c->vp);
    for (int t = 0; t < NPAN; t++) {
        interp_i2c(cu, &c->up, t, 0, N, 1, N + 1, c->ord);
        interp_i2c(cv, &c->vp, t, 1, N, 1, N + 1, c->ord);
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N; i++) FA(cu, t, i, j) = FA(cu, t, i, j) / c->my.J[MI(&c->my, t, i, j)];
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N + 1; i++) FA(cv, t, i, j) = FA(cv, t, i, j) / c->mx.J[MI(&c->mx, t, i, j)];
    }
}

/* sync_Ah_scalar_tile (halo_Ah_scalar_sync_mod.f90:43-98) */
static void sync_ah_scalar(orc_ctx *c, fld_t *f, int t)
{
    int n = c->N + 1, ie = n, je = n;
    FA(f, t, 1, 1) = (FA(f, t, 1, 1) + FA(f, t, 0, 1) + FA(f, t, 1, 0)) / 3.0;
    for (int j = 2; j <= n - 1; j++) FA(f, t, 1, j) = 0.5 * (FA(f, t, 0, j) + FA(f, t, 1, j));
    FA(f, t, 1, je) = (FA(f, t, 1, je) + FA(f, t, 0, je) + FA(f, t, 1, je + 1)) / 3.0;
    FA(f, t, ie, 1) = (FA(f, t, ie, 1) + FA(f, t, ie + 1, 1) + FA(f, t, ie, 0)) / 3.0;
    for (int j = 2; j <= n - 1; j++) FA(f, t, ie, j) = 0.5 * (FA(f, t, ie, j) + FA(f, t, ie + 1, j));
    FA(f, t, ie, je) = (FA(f, t, ie, je) + FA(f, t, ie + 1, je) + FA(f, t, ie, je + 1)) / 3.0;
    for (int i = 2; i <= n - 1; i++) FA(f, t, i, 1) = 0.5 * (FA(f, t, i, 1) + FA(f, t, i, 0));
    for (int i = 2; i <= n - 1; i++) FA(f, t, i, je) = 0.5 * (FA(f, t, i, je) + FA(f, t, i, je + 1));
}

/* div_sbp_SAT_t%calc_div with Ah projection (div_sbp_sat_mod.f90:29-80) */
static void op_div(orc_ctx *c, fld_t *div, fld_t *ut, fld_t *vt)
{
    int N = c->N;
    for (int t = 0; t < NPAN; t++) {
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N; i++) FA(&c->Ju, t, i, j) = FA(ut, t, i, j) * c->my.J[MI(&c->my, t, i, j)];
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N + 1; i++) FA(&c->Jv, t, i, j) = FA(vt, t, i, j) * c->mx.J[MI(&c->mx, t, i, j)];
    }
    exch_do(c->ord == 63 ? &c->ex_ch4_u : &c->ex_ch3_u, &c->Ju, &c->Jv);
    exch_do(c->ord == 63 ? &c->ex_ch4_v : &c->ex_ch3_v, &c->Ju, &c->Jv);
    for (int t = 0; t < NPAN; t++) {
        diff_c2i(&c->Dx, &c->Ju, t, 0, N + 1, 1, N + 1, c->ord);
        diff_c2i(&c->Dy, &c->Jv, t, 1, N + 1, 1, N + 1, c->ord);
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N + 1; i++)
                FA(div, t, i, j) = (FA(&c->Dx, t, i, j) / c->mxy.hx + FA(&c->Dy, t, i, j) / c->mxy.hy) /
                                   (c->mxy.J[MI(&c->mxy, t, i, j)] * c->a);
    }
    exch_do(&c->ex_xy1_full_s, div, NULL);
    for (int t = 0; t < NPAN; t++) sync_ah_scalar(c, div, t);
}

/* operator_swm_lin_t%apply (operator_swm_lin_mod.f90:66-108) */
static void op_apply_lin(orc_ctx *c, fld_t *dh, fld_t *du, fld_t *dv, fld_t *h, fld_t *u, fld_t *v)
{
    int N = c->N;
    op_grad(c, &c->gx, &c->gy, h);
    for (int t = 0; t < NPAN; t++) {
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N; i++) FA(du, t, i, j) = -c->g * FA(&c->gx, t, i, j);
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N + 1; i++) FA(dv, t, i, j) = -c->g * FA(&c->gy, t, i, j);
    }
    op_co2contra(c, &c->ut, &c->vt, u, v);
    op_coriolis(c, &c->gx, &c->gy, &c->ut, &c->vt);
    for (int t = 0; t < NPAN; t++) {
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N; i++) FA(du, t, i, j) = FA(du, t, i, j) + 1.0 * FA(&c->gx, t, i, j);
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N + 1; i++) FA(dv, t, i, j) = FA(dv, t, i, j) + 1.0 * FA(&c->gy, t, i, j);
    }
    op_div(c, &c->div, &c->ut, &c->vt);
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N + 1; i++) FA(dh, t, i, j) = -c->H * FA(&c->div, t, i, j);
}


/* ================================================================== */
/* advective operator, covariant Ch branch                              */
/* ================================================================== */

/* Point of a mesh at any (also halo) index: position on the sphere and the
   covariant basis a1 / a2 (set_curvilinear_mesh, metric_2d_ecs_mod.f90:338-411);
   same expressions as mesh_build. */
static void mesh_point(const mesh_t *m, int t, int i, int j, double r[3], double a1[3], double a2[3])
{
    double alpha = -0.25 * PI_ + (i - 1 + m->shift_i) * m->hx, beta = -0.25 * PI_ + (j - 1 + m->shift_j) * m->hy;
    double ta = tan(alpha), tb = tan(beta);
    double sigm = sqrt(1.0 + ta * ta + tb * tb);
    double rp[3] = {ta / sigm, tb / sigm, 1.0 / sigm};
    proto2real(t, rp, r);
    double s15 = pow(1.0 + pow(ta, 2.0) + pow(tb, 2.0), 1.5);
    double a1p[3] = {(1.0 + pow(ta, 2.0)) * (1.0 + pow(tb, 2.0)) / s15, -ta * tb * (1.0 + pow(ta, 2.0)) / s15,
                     -ta * (1.0 + pow(ta, 2.0)) / s15};
    double a2p[3] = {-ta * tb * (1.0 + pow(tb, 2.0)) / s15, (1.0 + pow(ta, 2.0)) * (1.0 + pow(tb, 2.0)) / s15,
                     -tb * (1.0 + pow(tb, 2.0)) / s15};
    proto2real(t, a1p, a1);
    proto2real(t, a2p, a2);
}

/* transform_cartesian_to_native_ecs (metric_2d_ecs_mod.f90:310-335): the panel with
   the largest projection of r on its outer normal, and (alpha, beta) there. */
static void cart_to_native(const double r[3], int *panel, double *alpha, double *beta)
{
    int p = 0;
    double best = 0.0;
    for (int q = 0; q < NPAN; q++) {
        double d = -(r[0] * T_N[q][0] + r[1] * T_N[q][1] + r[2] * T_N[q][2]);
        if (d > best) { p = q; best = d; }
    }
    *panel = p;
    *alpha = atan((T_EX[p][0] * r[0] + T_EX[p][1] * r[1] + T_EX[p][2] * r[2]) / best);
    *beta = atan((T_EY[p][0] * r[0] + T_EY[p][1] * r[1] + T_EY[p][2] * r[2]) / best);
}

/* ---- ECS_xy scalar halo (massflux_factory_mod.f90:59-64: width 3) ---- */

/* init_halo_xy_interp (ecs_halo_factory_mod.f90:236-270): cubic Lagrange weights
   along the source face's grid line for target index i at halo row j. */
static void halo_xy_weights(int n, double dxa, int i, int j, double w[4], int *ind)
{
    double zb = 0.25 * PI_ + j * dxa;
    double za = -0.25 * PI_ + (i - 1.0) * dxa;
    double zx = tan(za);
    double zz = tan(zb);
    zx = zx / zz;
    za = atan(zx);
    int k = (int)floor((za + 0.25 * PI_) / dxa) + 1;
    k = imin(imax(2, k), n - 2);
    double zxi = (za + 0.25 * PI_) / dxa - (k - 1.0);
    w[0] = -(zxi * (zxi - 1.0) * (zxi - 2.0) / 6.0);
    w[1] = (zxi + 1.0) * (zxi - 1.0) * (zxi - 2.0) / 2.0;
    w[2] = -((zxi + 1.0) * zxi * (zxi - 2.0) / 2.0);
    w[3] = (zxi + 1.0) * zxi * (zxi - 1.0) / 6.0;
    *ind = k;
}

/* ecs_ext_halo_1e: interpolate one line (values zf[b] at b = 1..n) */
static double halo_xy_line(int n, double dxa, int i, int j, const double *zf)
{
    double w[4];
    int ii;
    halo_xy_weights(n, dxa, i, j, w, &ii);
    return w[0] * zf[ii - 1] + w[1] * zf[ii] + w[2] * zf[ii + 1] + w[3] * zf[ii + 2];
}

/* get_ecs_halo + ext_ecs_tile_halo (ecs_halo_xy_mod.f90:66-235) on the whole panel
   (one tile per panel): the exchange, then corner diagonals and the averaging of
   the duplicated vertices, then rows / columns of interpolated virtual points.
   Modifies the interior edge and corner values of f, as the reference does. */
static void ecs_xy_interp(orc_ctx *c, fld_t *f, int hw);
static void ecs_xy_halo(orc_ctx *c, fld_t *f, int hw)
{
    exch_do(&c->ex_xy5_full_s, f, NULL);
    ecs_xy_interp(c, f, hw);
}

/* ecs_tile_halo_xy_t%interp (ecs_halo_xy_mod.f90:109-235): the part after the exchange */
static void ecs_xy_interp(orc_ctx *c, fld_t *f, int hw)
{
    int n = c->N + 1;
    double dxa = c->mxy.hx;
    double *zb = malloc(sizeof(double) * (n + 2 * hw + 8));
    double *zl = zb + hw + 2;   /* zl[b], b = 1 - hw - 2 .. n + hw + 4 */
    for (int t = 0; t < NPAN; t++) {
        /* corners */
        FA(f, t, 1, 1) = (FA(f, t, 1, 1) + FA(f, t, 1, 0) + FA(f, t, 0, 1)) / 3.0;
        for (int j = 1; j <= hw; j++) {
            FA(f, t, 1 - j, 1 - j) = 0.5 * (FA(f, t, -j, 1) + FA(f, t, 1, -j));
            FA(f, t, -j, 1) = FA(f, t, 1 - j, 1 - j);
            FA(f, t, 1, -j) = FA(f, t, 1 - j, 1 - j);
        }
        FA(f, t, n, 1) = (FA(f, t, n, 1) + FA(f, t, n, 0) + FA(f, t, n + 1, 1)) / 3.0;
        for (int j = 1; j <= hw; j++) {
            FA(f, t, n + j, 1 - j) = 0.5 * (FA(f, t, n + j + 1, 1) + FA(f, t, n, -j));
            FA(f, t, n + j + 1, 1) = FA(f, t, n + j, 1 - j);
            FA(f, t, n, -j) = FA(f, t, n + j, 1 - j);
        }
        FA(f, t, n, n) = (FA(f, t, n, n) + FA(f, t, n, n + 1) + FA(f, t, n + 1, n)) / 3.0;
        for (int j = 1; j <= hw; j++) {
            FA(f, t, n + j, n + j) = 0.5 * (FA(f, t, n + j + 1, n) + FA(f, t, n, n + j + 1));
            FA(f, t, n + j + 1, n) = FA(f, t, n + j, n + j);
            FA(f, t, n, n + j + 1) = FA(f, t, n + j, n + j);
        }
        FA(f, t, 1, n) = (FA(f, t, 1, n) + FA(f, t, 0, n) + FA(f, t, 1, n + 1)) / 3.0;
        for (int j = 1; j <= hw; j++) {
            FA(f, t, 1 - j, n + j) = 0.5 * (FA(f, t, 1, n + j + 1) + FA(f, t, -j, n));
            FA(f, t, 1, n + j + 1) = FA(f, t, 1 - j, n + j);
            FA(f, t, -j, n) = FA(f, t, 1 - j, n + j);
        }
        /* edge 1 (j = 1) */
        for (int i = 2; i <= n - 1; i++) FA(f, t, i, 1) = 0.5 * (FA(f, t, i, 1) + FA(f, t, i, 0));
        for (int j = 1; j <= hw; j++) {
            for (int b = 1; b <= n; b++) zl[b] = FA(f, t, b, -j);
            for (int i = 2 - j; i <= n + j - 1; i++) FA(f, t, i, 1 - j) = halo_xy_line(n, dxa, i, j, zl);
        }
        /* edge 2 (j = n) */
        for (int i = 2; i <= n - 1; i++) FA(f, t, i, n) = 0.5 * (FA(f, t, i, n) + FA(f, t, i, n + 1));
        for (int j = 1; j <= hw; j++) {
            for (int b = 1; b <= n; b++) zl[b] = FA(f, t, b, n + j + 1);
            for (int i = 2 - j; i <= n + j - 1; i++) FA(f, t, i, n + j) = halo_xy_line(n, dxa, i, j, zl);
        }
        /* edge 3 (i = 1) */
        for (int j = 2; j <= n - 1; j++) FA(f, t, 1, j) = 0.5 * (FA(f, t, 1, j) + FA(f, t, 0, j));
        for (int i = 1; i <= hw; i++) {
            for (int b = 1; b <= n; b++) zl[b] = FA(f, t, -i, b);
            for (int j = 2 - i; j <= n + i - 1; j++) FA(f, t, 1 - i, j) = halo_xy_line(n, dxa, j, i, zl);
        }
        /* edge 4 (i = n) */
        for (int j = 2; j <= n - 1; j++) FA(f, t, n, j) = 0.5 * (FA(f, t, n, j) + FA(f, t, n + 1, j));
        for (int i = 1; i <= hw; i++) {
            for (int b = 1; b <= n; b++) zl[b] = FA(f, t, n + i + 1, b);
            for (int j = 2 - i; j <= n + i - 1; j++) FA(f, t, n + i, j) = halo_xy_line(n, dxa, j, i, zl);
        }
    }
    free(zb);
}

/* calc_ch_up4_massflux (massflux_ch_mod.f90:61-121): fx on the y mesh, fy on the x mesh */
static void op_massflux_up4(orc_ctx *c, fld_t *fx, fld_t *fy, fld_t *f, fld_t *u, fld_t *v)
{
    int N = c->N;
    ecs_xy_halo(c, f, 3);
    for (int t = 0; t < NPAN; t++) {
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N; i++) {
                double uu = FA(u, t, i, j);
                double zl = 0.5 + copysign(0.5, uu), zr = 1.0 - zl;
                FA(fx, t, i, j) = uu * (zl * (5.0 * FA(f, t, i + 1, j) + 15.0 * FA(f, t, i, j) - 5.0 * FA(f, t, i - 1, j) +
                                              FA(f, t, i - 2, j)) +
                                        zr * (5.0 * FA(f, t, i, j) + 15.0 * FA(f, t, i + 1, j) - 5.0 * FA(f, t, i + 2, j) +
                                              FA(f, t, i + 3, j))) /
                                  16.0;
            }
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N + 1; i++) {
                double vv = FA(v, t, i, j);
                double zl = 0.5 + copysign(0.5, vv), zr = 1.0 - zl;
                FA(fy, t, i, j) = vv * (zl * (5.0 * FA(f, t, i, j + 1) + 15.0 * FA(f, t, i, j) - 5.0 * FA(f, t, i, j - 1) +
                                              FA(f, t, i, j - 2)) +
                                        zr * (5.0 * FA(f, t, i, j) + 15.0 * FA(f, t, i, j + 1) - 5.0 * FA(f, t, i, j + 2) +
                                              FA(f, t, i, j + 3))) /
                                  16.0;
            }
    }
}

/* ---- ECS Ch covariant vector halo (ecs_halo_vec_Ch, width 3) ---- */

/* calc_w of bicubic_interp_t (bicubic_interp_mod.f90:27-84) on a mesh of the source face */
static void bicubic_w(const mesh_t *m, double alpha, double beta, int *ix, int *iy, double wx[4], double wy[4])
{
    double dx = (alpha - (-0.25 * PI_)) / m->hx + 1 - m->shift_i;
    double dy = (beta - (-0.25 * PI_)) / m->hy + 1 - m->shift_j;
    *ix = imin(imax(2, (int)dx), m->nx - 2);
    *iy = imin(imax(2, (int)dy), m->ny - 2);
    dx = dx - *ix;
    dy = dy - *iy;
    double p1 = dx + 1.0, p2 = dx, p3 = dx - 1.0, p4 = dx - 2.0;
    wx[0] = -p2 * p3 * p4 / 6.0; wx[1] = p1 * p3 * p4 / 2.0; wx[2] = -p1 * p2 * p4 / 2.0; wx[3] = p1 * p2 * p3 / 6.0;
    p1 = dy + 1.0; p2 = dy; p3 = dy - 1.0; p4 = dy - 2.0;
    wy[0] = -p2 * p3 * p4 / 6.0; wy[1] = p1 * p3 * p4 / 2.0; wy[2] = -p1 * p2 * p4 / 2.0; wy[3] = p1 * p2 * p3 / 6.0;
}

/* interp_2d_levs (bicubic_interp_mod.f90:86-113) */
static double bicubic_v(const fld_t *f, int t, int ix, int iy, const double wx[4], const double wy[4])
{
    double r = 0.0;
    for (int j1 = -1; j1 <= 2; j1++) {
        double p = 0.0;
        for (int i1 = -1; i1 <= 2; i1++) p = p + wx[i1 + 1] * FA(f, t, ix + i1, iy + j1);
        r = r + wy[j1 + 1] * p;
    }
    return r;
}

/* The covariant component along the target basis vector a of the wind at halo
   point r, interpolated from the source face's u (y mesh) and v (x mesh) and
   projected with a.b1, a.b2 (ecs_halo_vec_Ch_factory_mod.f90:238-266). */
static double vec_halo_value(orc_ctx *c, const fld_t *u, const fld_t *v, const double r[3], const double a[3])
{
    int p, ixu, iyu, ixv, iyv;
    double al, be, wxu[4], wyu[4], wxv[4], wyv[4], bp[3], b1[3], b2[3];
    cart_to_native(r, &p, &al, &be);
    bicubic_w(&c->my, al, be, &ixu, &iyu, wxu, wyu);
    bicubic_w(&c->mx, al, be, &ixv, &iyv, wxv, wyv);
    b1_proto(al, be, bp); proto2real(p, bp, b1);
    b2_proto(al, be, bp); proto2real(p, bp, b2);
    double wu = a[0] * b1[0] + a[1] * b1[1] + a[2] * b1[2];
    double wv = a[0] * b2[0] + a[1] * b2[1] + a[2] * b2[2];
    double vu = bicubic_v(u, p, ixu, iyu, wxu, wyu), vv = bicubic_v(v, p, ixv, iyv, wxv, wyv);
    return wu * vu + wv * vv;
}

/* get_halo_vector (ecs_halo_vec_Ch_mod.f90:29-150): every side-strip halo point of
   u (y mesh) and v (x mesh) up to depth hw, from the interior of the source faces */
static void ecs_vec_halo(orc_ctx *c, fld_t *u, fld_t *v, int hw)
{
    int N = c->N;
    exch_do(&c->ex_ch3_u, u, v);
    exch_do(&c->ex_ch3_v, u, v);
    /* all values first (the reference interpolates every particle, then assembles) */
    size_t cnt = (size_t)NPAN * hw * (2 * N + 2 * (N + 1)) * 2;
    double *val = malloc(sizeof(double) * cnt);
    double r[3], a1[3], a2[3];
    for (int pass = 0; pass < 2; pass++) {
        size_t q = 0;   /* both passes walk the points in the same order */
        for (int t = 0; t < NPAN; t++)
            for (int d = 1; d <= hw; d++) {
                /* u: rows beyond south / north, columns beyond west / east */
                for (int i = 1; i <= N; i++) {
                    int jj[2] = {1 - d, N + 1 + d};
                    for (int s = 0; s < 2; s++, q++) {
                        if (pass == 0) { mesh_point(&c->my, t, i, jj[s], r, a1, a2); val[q] = vec_halo_value(c, u, v, r, a1); }
                        else FA(u, t, i, jj[s]) = val[q];
                    }
                }
                for (int j = 1; j <= N + 1; j++) {
                    int ii[2] = {1 - d, N + d};
                    for (int s = 0; s < 2; s++, q++) {
                        if (pass == 0) { mesh_point(&c->my, t, ii[s], j, r, a1, a2); val[q] = vec_halo_value(c, u, v, r, a1); }
                        else FA(u, t, ii[s], j) = val[q];
                    }
                }
                /* v: columns beyond west / east, rows beyond south / north */
                for (int j = 1; j <= N; j++) {
                    int ii[2] = {1 - d, N + 1 + d};
                    for (int s = 0; s < 2; s++, q++) {
                        if (pass == 0) { mesh_point(&c->mx, t, ii[s], j, r, a1, a2); val[q] = vec_halo_value(c, u, v, r, a2); }
                        else FA(v, t, ii[s], j) = val[q];
                    }
                }
                for (int i = 1; i <= N + 1; i++) {
                    int jj[2] = {1 - d, N + d};
                    for (int s = 0; s < 2; s++, q++) {
                        if (pass == 0) { mesh_point(&c->mx, t, i, jj[s], r, a1, a2); val[q] = vec_halo_value(c, u, v, r, a2); }
                        else FA(v, t, i, jj[s]) = val[q];
                    }
                }
            }
    }
    free(val);
}

/* calc_v_nabla_up4_tile (v_nabla_mod.f90:105-146) on nx x ny points of one panel */
static void v_nabla_up4(fld_t *tend, const fld_t *f, const fld_t *ut, const fld_t *vt, int t, int nx, int ny, double hx,
                        double scale)
{
    for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
            double a = FA(ut, t, i, j), b = FA(vt, t, i, j);
            double zl = 0.5 + copysign(0.5, a), zr = 1.0 - zl;
            double dx = (zl * (3.0 * FA(f, t, i + 1, j) + 10.0 * FA(f, t, i, j) - 18.0 * FA(f, t, i - 1, j) +
                               6.0 * FA(f, t, i - 2, j) - FA(f, t, i - 3, j)) -
                         zr * (3.0 * FA(f, t, i - 1, j) + 10.0 * FA(f, t, i, j) - 18.0 * FA(f, t, i + 1, j) +
                               6.0 * FA(f, t, i + 2, j) - FA(f, t, i + 3, j))) /
                        12.0;
            zl = 0.5 + copysign(0.5, b);
            zr = 1.0 - zl;
            double dy = (zl * (3.0 * FA(f, t, i, j + 1) + 10.0 * FA(f, t, i, j) - 18.0 * FA(f, t, i, j - 1) +
                               6.0 * FA(f, t, i, j - 2) - FA(f, t, i, j - 3)) -
                         zr * (3.0 * FA(f, t, i, j - 1) + 10.0 * FA(f, t, i, j) - 18.0 * FA(f, t, i, j + 1) +
                               6.0 * FA(f, t, i, j + 2) - FA(f, t, i, j + 3))) /
                        12.0;
            FA(tend, t, i, j) = -(a * dx + b * dy) / (hx * scale);
        }
}

/* calculate_ecs_S (metric_2d_ecs_mod.f90:270-291): Christoffel symbols of the first kind */
static void christoffel_S(double alpha, double beta, double S[3][2])
{
    double x = tan(alpha), y = tan(beta);
    double x2 = x * x, y2 = y * y;
    double sigma = 1.0 + x2 + y2;
    double s3 = sigma * sigma * sigma;
    S[0][0] = 2.0 * x * y2 * ((1.0 + x2) * (1.0 + x2)) * (1.0 + y2) / s3;
    S[1][0] = -0.5 * y * (1.0 + y2) * (1.0 + x2) * (-(x2 * x2) + 3.0 * x2 * y2 + y2 + 1.0) / s3;
    S[2][0] = x * (1.0 + x2) * ((1.0 + y2) * (1.0 + y2)) * (-x2 + y2 - 1.0) / s3;
    S[0][1] = y * (1.0 + y2) * ((1.0 + x2) * (1.0 + x2)) * (-y2 + x2 - 1.0) / s3;
    S[1][1] = -0.5 * x * (1.0 + x2) * (1.0 + y2) * (-(y2 * y2) + 3.0 * y2 * x2 + x2 + 1.0) / s3;
    S[2][1] = 2.0 * y * x2 * ((1.0 + y2) * (1.0 + y2)) * (1.0 + x2) / s3;
}

/* add_cov_wind_advection (hor_Christofel_shallow_mod.f90:92-122,149-164), comp 0 = u, 1 = v */
static void christoffel_add(fld_t *tend, const fld_t *ut, const fld_t *vt, const mesh_t *m, int t, int comp, double a)
{
    double scale = -a;
    for (int j = 1; j <= m->ny; j++)
        for (int i = 1; i <= m->nx; i++) {
            double alpha = -0.25 * PI_ + (i - 1 + m->shift_i) * m->hx, beta = -0.25 * PI_ + (j - 1 + m->shift_j) * m->hy;
            double S[3][2];
            christoffel_S(alpha, beta, S);
            double g11 = S[0][comp], g21 = S[1][comp], g22 = S[2][comp];
            double uu = FA(ut, t, i, j), vv = FA(vt, t, i, j);
            FA(tend, t, i, j) = FA(tend, t, i, j) - (uu * uu * g11 + 2.0 * uu * vv * g21 + vv * vv * g22) / scale;
        }
}

/* calc_vec_advection (vector_advection_Ch_mod.f90:33-62) */
static void op_vec_adv(orc_ctx *c, fld_t *utd, fld_t *vtd, fld_t *u, fld_t *v, fld_t *ut, fld_t *vt)
{
    int N = c->N;
    /* interp2d_uv2pvec_Ch_sbp42: uh = I_c2i,x(ut), vh = I_c2i,y(vt) on xy */
    exch_do(&c->ex_ch3_u, ut, vt);
    exch_do(&c->ex_ch3_v, ut, vt);
    for (int t = 0; t < NPAN; t++) {
        /* the vector advection's interpolators are the _sbp42 ones whatever the operator's
           order (vector_advection_factory_mod.f90:65) */
        interp_c2i(&c->uh, ut, t, 0, N + 1, 1, N + 1, 42);
        interp_c2i(&c->vh, vt, t, 1, N + 1, 1, N + 1, 42);
    }
    /* interp2d_pvec2uv_Ch_sbp42 on (vh, uh): v_at_u = I_i2c,x(vh), u_at_v = I_i2c,y(uh)
       (its xy exchange fills halos that the SBP interpolation does not read) */
    for (int t = 0; t < NPAN; t++) {
        interp_i2c(&c->vau, &c->vh, t, 0, N, 1, N + 1, 42);
        interp_i2c(&c->uav, &c->uh, t, 1, N, 1, N + 1, 42);
    }
    /* u_halo = u, v_halo = v, then the ECS Ch vector halo of width 3 */
    for (int t = 0; t < NPAN; t++) {
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N; i++) FA(&c->uhal, t, i, j) = FA(u, t, i, j);
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N + 1; i++) FA(&c->vhal, t, i, j) = FA(v, t, i, j);
    }
    ecs_vec_halo(c, &c->uhal, &c->vhal, 3);
    for (int t = 0; t < NPAN; t++) {
        v_nabla_up4(utd, &c->uhal, ut, &c->vau, t, N, N + 1, c->my.hx, c->a);
        v_nabla_up4(vtd, &c->vhal, &c->uav, vt, t, N + 1, N, c->mx.hx, c->a);
        christoffel_add(utd, ut, &c->vau, &c->my, t, 0, c->a);
        christoffel_add(vtd, &c->uav, vt, &c->mx, t, 1, c->a);
    }
    /* CH_uv_exchange ('cross', width 1) and sync_ch_cov (vector_advection_Ch_mod.f90:73-115) */
    exch_do(&c->ex_ch1c_u, utd, vtd);
    exch_do(&c->ex_ch1c_v, utd, vtd);
    for (int t = 0; t < NPAN; t++) {
        for (int j = 1; j <= N; j++) FA(vtd, t, 1, j) = 0.5 * (FA(vtd, t, 1, j) + FA(vtd, t, 0, j));
        for (int j = 1; j <= N; j++) FA(vtd, t, N + 1, j) = 0.5 * (FA(vtd, t, N + 2, j) + FA(vtd, t, N + 1, j));
        for (int i = 1; i <= N; i++) FA(utd, t, i, 1) = 0.5 * (FA(utd, t, i, 1) + FA(utd, t, i, 0));
        for (int i = 1; i <= N; i++) FA(utd, t, i, N + 1) = 0.5 * (FA(utd, t, i, N + 2) + FA(utd, t, i, N + 1));
    }
}

/* operator_adv_swm_t%apply, covariant branch (operator_adv_swm_mod.f90:62-96); no orography */
static void op_apply_nl(orc_ctx *c, fld_t *dh, fld_t *du, fld_t *dv, fld_t *h, fld_t *u, fld_t *v)
{
    int N = c->N;
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N + 1; i++)
                FA(&c->htot, t, i, j) = 1.0 * FA(h, t, i, j) +
                                        1.0 * (c->hsurf ? c->hsurf[((size_t)t * (N + 1) + j - 1) * (N + 1) + i - 1] : 0.0);
    op_co2contra(c, &c->ut, &c->vt, u, v);
    op_massflux_up4(c, &c->hu, &c->hv, h, &c->ut, &c->vt);
    op_div(c, &c->div, &c->hu, &c->hv);
    op_grad(c, &c->gx, &c->gy, &c->htot);
    op_coriolis(c, &c->cu, &c->cv, &c->ut, &c->vt);
    op_vec_adv(c, du, dv, u, v, &c->ut, &c->vt);
    for (int t = 0; t < NPAN; t++) {
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N; i++)
                FA(du, t, i, j) = FA(du, t, i, j) + (-c->g) * FA(&c->gx, t, i, j) + 1.0 * FA(&c->cu, t, i, j);
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N + 1; i++)
                FA(dv, t, i, j) = FA(dv, t, i, j) + (-c->g) * FA(&c->gy, t, i, j) + 1.0 * FA(&c->cv, t, i, j);
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N + 1; i++) FA(dh, t, i, j) = -1.0 * FA(&c->div, t, i, j);
    }
}

/* ================================================================== */
/* C staggering: h on the cell centres (o), u on the x mesh, v on the y mesh          */
/* (domain_factory_mod.f90:281-295)                                                   */
/* ================================================================== */
static void c_init(orc_ctx *c)
{
    if (c->cgrid) return;
    const int N = c->N, hw = 5;
    build_o_exchange(&c->ex_o3, N, 3, 0);
    build_c_exchange(&c->ex_c3_u, N, 3, 1);
    build_c_exchange(&c->ex_c3_v, N, 3, 0);
    fld_t *oo[] = {&c->c_h, &c->c_uh, &c->c_vh, &c->c_Dx, &c->c_Dy, &c->c_div};
    fld_t *xx[] = {&c->c_u, &c->c_gx, &c->c_ut, &c->c_Ju};
    fld_t *yy[] = {&c->c_v, &c->c_gy, &c->c_vt, &c->c_Jv};
    for (unsigned q = 0; q < sizeof(oo) / sizeof(oo[0]); q++) fld_init(oo[q], N, N, hw);
    for (unsigned q = 0; q < sizeof(xx) / sizeof(xx[0]); q++) fld_init(xx[q], N + 1, N, hw);
    for (unsigned q = 0; q < sizeof(yy) / sizeof(yy[0]); q++) fld_init(yy[q], N, N + 1, hw);
    c->cgrid = 1;
}

static void c_free(orc_ctx *c)
{
    if (!c->cgrid) return;
    fld_t *all[] = {&c->c_h, &c->c_u, &c->c_v, &c->c_gx, &c->c_gy, &c->c_ut, &c->c_vt, &c->c_uh, &c->c_vh,
                    &c->c_Ju, &c->c_Jv, &c->c_Dx, &c->c_Dy, &c->c_div};
    for (unsigned q = 0; q < sizeof(all) / sizeof(all[0]); q++) fld_free(all[q]);
    c->cgrid = 0;
}

/* grad_c_sbp_sat_<order>: grad_sbp_sat_t with the centres->nodes difference and its SAT on
   the o-point halo of width 3 (grad_factory_mod.f90:115-150, grad_sbp_sat_mod.f90:24-76):
   gx on the x mesh, gy on the y mesh, each divided by h a. */
static void op_grad_c(orc_ctx *c, fld_t *gx, fld_t *gy, fld_t *h)
{
    const int N = c->N;
    exch_do(&c->ex_o3, h, NULL);
    for (int t = 0; t < NPAN; t++) {
        diff_c2i(gx, h, t, 0, N + 1, 1, N, c->ord);
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N + 1; i++) FA(gx, t, i, j) = FA(gx, t, i, j) / (c->mx.hx * c->a);
        diff_c2i(gy, h, t, 1, N + 1, 1, N, c->ord);
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N; i++) FA(gy, t, i, j) = FA(gy, t, i, j) / (c->my.hy * c->a);
    }
}

/* div_c_sbp_sat_<order>: div_sbp_SAT_t with the nodes->centres difference, its SAT on the
   C vector halo and no projection (div_factory_mod.f90:112-156, div_sbp_sat_mod.f90:29-80). */
static void op_div_c(orc_ctx *c, fld_t *div, fld_t *ut, fld_t *vt)
{
    const int N = c->N;
    for (int t = 0; t < NPAN; t++) {
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N + 1; i++) FA(&c->c_Ju, t, i, j) = FA(ut, t, i, j) * c->mx.J[MI(&c->mx, t, i, j)];
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N; i++) FA(&c->c_Jv, t, i, j) = FA(vt, t, i, j) * c->my.J[MI(&c->my, t, i, j)];
    }
    exch_do(&c->ex_c3_u, &c->c_Ju, &c->c_Jv);
    exch_do(&c->ex_c3_v, &c->c_Ju, &c->c_Jv);
    for (int t = 0; t < NPAN; t++) {
        diff_i2c(&c->c_Dx, &c->c_Ju, t, 0, N, 1, N, c->ord);
        diff_i2c(&c->c_Dy, &c->c_Jv, t, 1, N, 1, N, c->ord);
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N; i++)
                FA(div, t, i, j) = (FA(&c->c_Dx, t, i, j) / c->mo.hx + FA(&c->c_Dy, t, i, j) / c->mo.hy) /
                                   (c->mo.J[MI(&c->mo, t, i, j)] * c->a);
    }
}

/* co2contra_c_sbp<order>_new (co2contra_Cgrid_mod.f90, transform_co2contra_c_sbp_new): u, v to
   the cell centres (interp2d_uv2pvec_C: nodes->centres interpolation along x / y,
   interpolator_uv2p_mod.f90:22-49), there times J Qi12 and swapped, back to the faces
   (interp2d_pvec2uv_C: centres->nodes interpolation, interpolator_p2uv_mod.f90:54-99),
   then ut = Qi11 u + (.)/J, vt = Qi22 v + (.)/J.  The exchanges before the two
   interpolations fill halos the SBP closure rows never read. */
static void op_co2contra_c(orc_ctx *c, fld_t *ut, fld_t *vt, fld_t *u, fld_t *v)
{
    const int N = c->N;
    for (int t = 0; t < NPAN; t++) {
        interp_i2c(&c->c_uh, u, t, 0, N, 1, N, c->ord);
        interp_i2c(&c->c_vh, v, t, 1, N, 1, N, c->ord);
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N; i++) {
                const size_t k = MI(&c->mo, t, i, j);
                const double uu = FA(&c->c_uh, t, i, j) * c->mo.J[k] * c->mo.Q2[k];
                const double vv = FA(&c->c_vh, t, i, j) * c->mo.J[k] * c->mo.Q2[k];
                FA(&c->c_uh, t, i, j) = vv;
                FA(&c->c_vh, t, i, j) = uu;
            }
        interp_c2i(ut, &c->c_uh, t, 0, N + 1, 1, N, c->ord);
        interp_c2i(vt, &c->c_vh, t, 1, N + 1, 1, N, c->ord);
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N + 1; i++) {
                const size_t k = MI(&c->mx, t, i, j);
                FA(ut, t, i, j) = c->mx.Q1[k] * FA(u, t, i, j) + FA(ut, t, i, j) / c->mx.J[k];
            }
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N; i++) {
                const size_t k = MI(&c->my, t, i, j);
                FA(vt, t, i, j) = c->my.Q3[k] * FA(v, t, i, j) + FA(vt, t, i, j) / c->my.J[k];
            }
    }
}

static void op_apply(orc_ctx *c, fld_t *dh, fld_t *du, fld_t *dv, fld_t *h, fld_t *u, fld_t *v)
{
    if (c->nonlinear) op_apply_nl(c, dh, du, dv, h, u, v);
    else op_apply_lin(c, dh, du, dv, h, u, v);
}

/* ---- Ah staggering: the linear operator of gen_config_linear.sh:9-36 (div_ah_sbp_proj_*,
   grad_ah_sbp_proj_*, coriolis_colocated, co2contra_colocated), h, u, v on the xy mesh ---- */

/* node-to-node SBP first derivative along dir of a line of n nodes (no halo, one-sided
   closures): sbp_diff_21_mod.f90:8-40, sbp_diff_42_mod.f90:30-156 (the reference's decimal
   coefficients), sbp_diff_63_mod.f90:9-140 (SBP63_NN_Q) */
static const double N42_Q[4][6] = {{-1.4117647058823528, 1.7352941176470589, -0.2352941176470588, -0.08823529411764705, 0, 0},
                                   {-0.5, 0, 0.5, 0, 0, 0},
                                   {0.09302325581395347, -0.686046511627907, 0, 0.686046511627907, -0.09302325581395347, 0},
                                   {0.030612244897959186, 0, -0.6020408163265307, 0, 0.653061224489796, -0.0816326530612245}};
static void diff_n2n(fld_t *out, const fld_t *in, int t, int dir, int n, int ls, int le, int ord)
{
#define O(k) (*((dir) == 0 ? &FA(out, t, k, l) : &FA(out, t, l, k)))
#define I(k) L(in, t, dir, k, l)
    if (ord == 21) {
        /* sbp_diff_21_mod.f90: q11 = -1, q12 = 1; interior (-f(i-1) + f(i+1)) / 2 */
        for (int l = ls; l <= le; l++) {
            O(1) = -1.0 * I(1) + 1.0 * I(2);
            for (int k = 2; k <= n - 1; k++) O(k) = (-I(k - 1) + I(k + 1)) / 2.0;
            O(n) = -(-1.0) * I(n) - 1.0 * I(n - 1);
        }
        return;
    }
    if (ord == 63) {
        for (int l = ls; l <= le; l++) {
            for (int r = 1; r <= 6; r++) {
                double a = 0.0, b = 0.0;
                for (int q = 0; q < 9; q++) {
                    if (SBP63_NN_Q[r - 1][q] == 0.0) continue;
                    a = a + SBP63_NN_Q[r - 1][q] * I(q + 1);
                    b = b - SBP63_NN_Q[r - 1][q] * I(n + 1 - (q + 1));
                }
                O(r) = a;
                O(n + 1 - r) = b;
            }
            for (int k = 7; k <= n - 6; k++)
                O(k) = (-I(k - 3) + 9 * I(k - 2) + -45 * I(k - 1) + 45 * I(k + 1) + -9 * I(k + 2) + I(k + 3)) / 60.0;
        }
        return;
    }
    for (int l = ls; l <= le; l++) {
        for (int r = 1; r <= 4; r++) {
            double a = 0.0, b = 0.0;
            for (int q = 0; q < 6; q++) {
                if (N42_Q[r - 1][q] == 0.0) continue;
                a = a + N42_Q[r - 1][q] * I(q + 1);
                b = b - N42_Q[r - 1][q] * I(n + 1 - (q + 1));
            }
            O(r) = a;
            O(n + 1 - r) = b;
        }
        for (int k = 5; k <= n - 4; k++) O(k) = (I(k - 2) + -8 * I(k - 1) + 8 * I(k + 1) + -I(k + 2)) / 12.0;
    }
#undef O
#undef I
}

/* grad_sbp_proj_t%calc_grad (grad_sbp_proj_mod.f90:26-72) with the covariant
   ecs_Ah_vec_sync (ecs_Ah_vec_sync_mod.f90:34-60: syncronize_grad_on_edges(gy, gx)) */
static void op_grad_ah(orc_ctx *c, fld_t *gx, fld_t *gy, fld_t *h)
{
    int N = c->N, n = N + 1;
    const mesh_t *m = &c->mxy;
    for (int t = 0; t < NPAN; t++) {
        diff_n2n(gx, h, t, 0, n, 1, n, c->ord);
        diff_n2n(gy, h, t, 1, n, 1, n, c->ord);
        for (int j = 1; j <= n; j++)
            for (int i = 1; i <= n; i++) {
                FA(gx, t, i, j) = FA(gx, t, i, j) / (m->hx * c->a);
                FA(gy, t, i, j) = FA(gy, t, i, j) / (m->hy * c->a);
            }
    }
    exch_do(&c->ex_xy1_cross_v, gx, gy);
    for (int t = 0; t < NPAN; t++) sync_grad_on_edges(c, gy, gx, t);
}

/* div_sbp_proj_t%calc_div (div_sbp_proj_mod.f90:25-76) with the Ah scalar sync */
static void op_div_ah(orc_ctx *c, fld_t *div, fld_t *ut, fld_t *vt)
{
    int N = c->N, n = N + 1;
    const mesh_t *m = &c->mxy;
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= n; j++)
            for (int i = 1; i <= n; i++) {
                const double J = m->J[MI(m, t, i, j)];
                FA(&c->ah_Ju, t, i, j) = FA(ut, t, i, j) * J;
                FA(&c->ah_Jv, t, i, j) = FA(vt, t, i, j) * J;
            }
    for (int t = 0; t < NPAN; t++) {
        diff_n2n(&c->Dx, &c->ah_Ju, t, 0, n, 1, n, c->ord);
        diff_n2n(&c->Dy, &c->ah_Jv, t, 1, n, 1, n, c->ord);
        for (int j = 1; j <= n; j++)
            for (int i = 1; i <= n; i++)
                FA(div, t, i, j) = (FA(&c->Dx, t, i, j) / m->hx + FA(&c->Dy, t, i, j) / m->hy) /
                                   (m->J[MI(m, t, i, j)] * c->a);
    }
    exch_do(&c->ex_xy1_full_s, div, NULL);
    for (int t = 0; t < NPAN; t++) sync_ah_scalar(c, div, t);
}

/* operator_swm_lin_t%apply (operator_swm_lin_mod.f90:66-108) with the Ah operators:
   co2contra_colocated (co2contra_colocated_mod.f90:17-47: ut = Qi11 u + Qi12 v,
   vt = Qi12 u + Qi22 v) and coriolis_colocated (coriolis_colocated_mod.f90:17-45:
   cor_u = f vt J, cor_v = -f ut J) */
static void op_apply_ah(orc_ctx *c, fld_t *dh, fld_t *du, fld_t *dv, fld_t *h, fld_t *u, fld_t *v)
{
    int n = c->N + 1;
    const mesh_t *m = &c->mxy;
    op_grad_ah(c, &c->ah_gx, &c->ah_gy, h);
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= n; j++)
            for (int i = 1; i <= n; i++) {
                const size_t k = MI(m, t, i, j);
                FA(du, t, i, j) = -c->g * FA(&c->ah_gx, t, i, j);
                FA(dv, t, i, j) = -c->g * FA(&c->ah_gy, t, i, j);
                FA(&c->ah_ut, t, i, j) = m->Q1[k] * FA(u, t, i, j) + m->Q2[k] * FA(v, t, i, j);
                FA(&c->ah_vt, t, i, j) = m->Q2[k] * FA(u, t, i, j) + m->Q3[k] * FA(v, t, i, j);
            }
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= n; j++)
            for (int i = 1; i <= n; i++) {
                const size_t k = MI(m, t, i, j);
                const double cu = c->fxy[k] * FA(&c->ah_vt, t, i, j) * m->J[k];
                const double cv = -c->fxy[k] * FA(&c->ah_ut, t, i, j) * m->J[k];
                FA(du, t, i, j) = FA(du, t, i, j) + 1.0 * cu;
                FA(dv, t, i, j) = FA(dv, t, i, j) + 1.0 * cv;
            }
    op_div_ah(c, &c->div, &c->ah_ut, &c->ah_vt);
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= n; j++)
            for (int i = 1; i <= n; i++) FA(dh, t, i, j) = -c->H * FA(&c->div, t, i, j);
}

/* ---- diffusion on the Ah staggering: operator_swm_diff_t%apply (operator_swm_diff_mod.f90:27-49)
   with hordiff_vec_xyz_Ah_sbp_21_narrow for (u, v) and hordiff_scalar_Ah_sbp_21_narrow for h
   (hordiff_factory_mod.f90:33-34,61-62), stepped by explicit_Eul1 (explicit_Eul1_mod.f90:20-28)
   after each step of the dynamics (shallow_water_mod.f90:95-100,117-118) ---- */

static void diff_alloc(orc_ctx *c)
{
    if (c->df_d1x.p) return;
    const int n = c->N + 1, hw = 2;
    fld_t *df[] = {&c->df_d1x, &c->df_d1y, &c->df_d2x, &c->df_d2y, &c->df_dxy, &c->df_dyx,
                   &c->df_x[0], &c->df_x[1], &c->df_x[2], &c->df_t[0], &c->df_t[1], &c->df_t[2]};
    for (unsigned q = 0; q < sizeof(df) / sizeof(df[0]); q++) fld_init(df[q], n, n, hw);
}

/* Closure rows 1..6 of the narrow SBP 4-2 second difference with a variable coefficient
   (laplace_Ah_sbp42_narrow_mod.f90:121-262): entry m_rc (r <= c) of the symmetric boundary
   block as sum_k w b_k over the coefficients b_k = Qi J at node k; row r of the difference is
   -(1 / h_r) sum_c m_rc f_c with the node norm h_r (the same block mirrored at the far end,
   :284-423) */
static const struct { int r, c, k; double w; } LAP42_M[] = {
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
static const double LAP42_H[6] = {17.0 / 48, 59.0 / 48, 43.0 / 48, 49.0 / 48, 1, 1};

/* the narrow second difference of a line of n nodes (b, f, out 1-based): the d2f_x / d2f_y
   sweeps of calc_laplace_tile (laplace_Ah_sbp21_narrow_mod.f90:116-191 for 2-1,
   laplace_Ah_sbp42_narrow_mod.f90:121-699 for 4-2, laplace_Ah_sbp63_narrow_mod.f90:589-1664
   for 6-3) */
static void narrow_d2_line(int ord, int n, const double *b, const double *f, double *out)
{
    if (ord == 21) {
        double bc = b[1], bp = b[2];
        out[1] = (-(bc + bp) * f[1] + (bc + bp) * f[2]);
        for (int i = 2; i <= n - 1; i++) {
            const double bm = b[i - 1], bcc = b[i], bpp = b[i + 1];
            const double cm = (bm + bcc) / 2, cc = -(bm + 2 * bcc + bpp) / 2, cp = (bpp + bcc) / 2;
            out[i] = (cp * f[i + 1] + cc * f[i] + cm * f[i - 1]);
        }
        bc = b[n];
        const double bm = b[n - 1];
        out[n] = (bc + bm) * f[n - 1] + (-(bc + bm)) * f[n];
        return;
    }
    if (ord == 63) {
        static double E[9][12][12];
        static int ready63 = 0;
        if (!ready63) {
            for (unsigned q = 0; q < sizeof(LAP63_M) / sizeof(LAP63_M[0]); q++)
                E[LAP63_M[q].r - 1][LAP63_M[q].c - 1][LAP63_M[q].k - 1] = LAP63_M[q].w;
            ready63 = 1;
        }
        for (int side = 0; side < 2; side++)
            for (int r = 1; r <= 9; r++) {
                double acc = 0.0;
                for (int cc = 1; cc <= 12; cc++) {
                    double m = 0.0;
                    for (int k = 1; k <= 12; k++) m = m + E[r - 1][cc - 1][k - 1] * b[side ? n + 1 - k : k];
                    acc = acc + m * f[side ? n + 1 - cc : cc];
                }
                out[side ? n + 1 - r : r] = 1.0 * acc;
            }
        /* the interior rows (laplace_Ah_sbp63_narrow_mod.f90:860-880) */
        const double a33 = 11.0 / 360, a32 = -1.0 / 40, a31 = -1.0 / 40, a30 = 11.0 / 360;
        const double a23 = -1.0 / 20, a22 = -7.0 / 40, a21 = 3.0 / 10, a20 = -7.0 / 40, a2p = -1.0 / 20;
        const double a13 = 1.0 / 40, a12 = 3.0 / 10, a11 = 17.0 / 40, a10 = 17.0 / 40, a1p = 3.0 / 10, a1q = 1.0 / 40;
        const double c3 = -1.0 / 180, c2 = -1.0 / 8, c1 = -19.0 / 20, c0 = -101.0 / 180;
        for (int i = 10; i <= n - 9; i++) {
            const double bmmm = b[i - 3], bmm = b[i - 2], bm = b[i - 1], bc = b[i], bp = b[i + 1], bpp = b[i + 2],
                         bppp = b[i + 3];
            const double cmmm = a33 * bmmm + a32 * bmm + a31 * bm + a30 * bc;
            const double cmm = a23 * bmmm + a22 * bmm + a21 * bm + a20 * bc + a2p * bp;
            const double cm = a13 * bmmm + a12 * bmm + a11 * bm + a10 * bc + a1p * bp + a1q * bpp;
            const double ccc = c3 * bmmm + c2 * bmm + c1 * bm + c0 * bc + c1 * bp + c2 * bpp + c3 * bppp;
            const double cp = a13 * bppp + a12 * bpp + a11 * bp + a10 * bc + a1p * bm + a1q * bmm;
            const double cpp = a23 * bppp + a22 * bpp + a21 * bp + a20 * bc + a2p * bm;
            const double cppp = a33 * bppp + a32 * bpp + a31 * bp + a30 * bc;
            out[i] = (cmmm * f[i - 3] + cmm * f[i - 2] + cm * f[i - 1] + ccc * f[i] + cp * f[i + 1] + cpp * f[i + 2] +
                      cppp * f[i + 3]);
        }
        return;
    }
    static double D[6][8][8];
    static int ready = 0;
    if (!ready) {
        for (unsigned q = 0; q < sizeof(LAP42_M) / sizeof(LAP42_M[0]); q++) {
            const int r = LAP42_M[q].r, c = LAP42_M[q].c, k = LAP42_M[q].k;
            D[r - 1][c - 1][k - 1] = LAP42_M[q].w;
            if (c <= 6) D[c - 1][r - 1][k - 1] = LAP42_M[q].w;
        }
        ready = 1;
    }
    for (int side = 0; side < 2; side++)
        for (int r = 1; r <= 6; r++) {
            double acc = 0.0;
            for (int cc = 1; cc <= 8; cc++) {
                double m = 0.0;
                for (int k = 1; k <= 8; k++) m = m + D[r - 1][cc - 1][k - 1] * b[side ? n + 1 - k : k];
                acc = acc + m * f[side ? n + 1 - cc : cc];
            }
            out[side ? n + 1 - r : r] = -1.0 / LAP42_H[r - 1] * acc;
        }
    for (int i = 7; i <= n - 6; i++) {
        const double bmm = b[i - 2], bm = b[i - 1], bc = b[i], bp = b[i + 1], bpp = b[i + 2];
        const double cmm = 1.0 / 6.0 * bm - 1.0 / 8.0 * bmm - 1.0 / 8.0 * bc;
        const double cm = 1.0 / 6.0 * bmm + 1.0 / 6.0 * bp + 1.0 / 2.0 * bm + 1.0 / 2.0 * bc;
        const double cc = -1.0 / 24.0 * bmm - 5.0 / 6.0 * bm - 5.0 / 6.0 * bp - 1.0 / 24.0 * bpp - 3.0 / 4.0 * bc;
        const double cp = 1.0 / 6.0 * bm + 1.0 / 6.0 * bpp + 1.0 / 2.0 * bc + 1.0 / 2.0 * bp;
        const double cpp = 1.0 / 6.0 * bp - 1.0 / 8.0 * bc - 1.0 / 8.0 * bpp;
        out[i] = (cmm * f[i - 2] + cm * f[i - 1] + cc * f[i] + cp * f[i + 1] + cpp * f[i + 2]);
    }
}

/* laplace_Ah_sbp<ord>_narrow_t%calc_laplace (laplace_Ah_sbp21_narrow_mod.f90:25-56 and
   laplace_Ah_sbp42_narrow_mod.f90:27-63) with calc_tile_d1x_d1y and calc_laplace_tile:
   the narrow second differences with the variable coefficients Qi11 J and Qi22 J, the mixed
   terms D1(Qi12 J D1 f), the boundary penalties 1/h_1 (-+2 d1f) (all four added to d2f_x, as
   the reference does), the division by (hx a)^2 and by J, then the Ah scalar sync.  out may
   be f.  The halo exchanges of f, d1f_x and d1f_y ahead of the tile sweeps feed no stencil
   (every difference is one-sided at the panel edges) and are left out. */
static void lap_ah(orc_ctx *c, fld_t *out, fld_t *f, int ord)
{
    const int n = c->N + 1;
    const mesh_t *m = &c->mxy;
    fld_t *d1x = &c->df_d1x, *d1y = &c->df_d1y, *d2x = &c->df_d2x, *d2y = &c->df_d2y;
    fld_t *dxy = &c->df_dxy, *dyx = &c->df_dyx;
    const double pen = ord == 21 ? 2.0 : (ord == 42 ? 48.0 / 17 : 43200.0 / 13649);   /* 1 / h_1 of the node norm */
    double *bl = malloc(sizeof(double) * (n + 1)), *fl = malloc(sizeof(double) * (n + 1)),
           *ol = malloc(sizeof(double) * (n + 1));
    for (int t = 0; t < NPAN; t++) {
        diff_n2n(d1x, f, t, 0, n, 1, n, ord);
        diff_n2n(d1y, f, t, 1, n, 1, n, ord);
        for (int j = 1; j <= n; j++)
            for (int i = 1; i <= n; i++) {
                const size_t k = MI(m, t, i, j);
                FA(d1x, t, i, j) = FA(d1x, t, i, j) * m->J[k] * m->Q2[k];
                FA(d1y, t, i, j) = FA(d1y, t, i, j) * m->J[k] * m->Q2[k];
            }
    }
    const double h2 = (m->hx * c->a) * (m->hx * c->a);
    for (int t = 0; t < NPAN; t++) {
        for (int j = 1; j <= n; j++) {
            for (int i = 1; i <= n; i++) {
                const size_t k = MI(m, t, i, j);
                bl[i] = m->Q1[k] * m->J[k];
                fl[i] = FA(f, t, i, j);
            }
            narrow_d2_line(ord, n, bl, fl, ol);
            for (int i = 1; i <= n; i++) FA(d2x, t, i, j) = ol[i];
        }
        for (int i = 1; i <= n; i++) {
            for (int j = 1; j <= n; j++) {
                const size_t k = MI(m, t, i, j);
                bl[j] = m->Q3[k] * m->J[k];
                fl[j] = FA(f, t, i, j);
            }
            narrow_d2_line(ord, n, bl, fl, ol);
            for (int j = 1; j <= n; j++) FA(d2y, t, i, j) = ol[j];
        }
        for (int j = 1; j <= n; j++) {
            const double penalty = pen * (-2.0 * FA(d1y, t, 1, j));
            FA(d2x, t, 1, j) = FA(d2x, t, 1, j) - 0.5 * penalty;
        }
        for (int j = 1; j <= n; j++) {
            const double penalty = pen * (2 * FA(d1y, t, n, j));
            FA(d2x, t, n, j) = FA(d2x, t, n, j) - 0.5 * penalty;
        }
        for (int i = 1; i <= n; i++) {
            const double penalty = pen * (-2 * FA(d1x, t, i, 1));
            FA(d2x, t, i, 1) = FA(d2x, t, i, 1) - 0.5 * penalty;
        }
        for (int i = 1; i <= n; i++) {
            const double penalty = pen * (2 * FA(d1x, t, i, n));
            FA(d2x, t, i, n) = FA(d2x, t, i, n) - 0.5 * penalty;
        }
        diff_n2n(dyx, d1x, t, 1, n, 1, n, ord);
        diff_n2n(dxy, d1y, t, 0, n, 1, n, ord);
        for (int j = 1; j <= n; j++)
            for (int i = 1; i <= n; i++) {
                double v = 1.0 * FA(d2x, t, i, j) + 1.0 * FA(d2y, t, i, j);
                v = v + 1.0 * FA(dxy, t, i, j) + 1.0 * FA(dyx, t, i, j);
                FA(out, t, i, j) = v / h2;
            }
        for (int j = 1; j <= n; j++)
            for (int i = 1; i <= n; i++) FA(out, t, i, j) = FA(out, t, i, j) / m->J[MI(m, t, i, j)];
    }
    free(bl); free(fl); free(ol);
    exch_do(&c->ex_xy1_full_s, out, NULL);
    for (int t = 0; t < NPAN; t++) sync_ah_scalar(c, out, t);
}

/* hordiff_scalar_t%calc_diff (hordiff_scalar_mod.f90:30-50), diff_order 2 with
   diff_coeff = coeff a hx (hordiff_factory_mod.f90:276-298): tend = -(coeff a hx)^4 L(L(f)).
   f_work receives the iterate (it may be f). */
static void hordiff_ah(orc_ctx *c, fld_t *tend, fld_t *f, fld_t *work, double coeff, int ord)
{
    const int n = c->N + 1;
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= n; j++)
            for (int i = 1; i <= n; i++) FA(work, t, i, j) = 1.0 * FA(f, t, i, j);
    lap_ah(c, work, work, ord);
    lap_ah(c, work, work, ord);
    const double dc = coeff * c->a * c->mxy.hx;
    const double k = -1.0 * ((dc * dc) * (dc * dc));
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= n; j++)
            for (int i = 1; i <= n; i++) FA(tend, t, i, j) = k * FA(work, t, i, j);
}

/* operator_swm_diff_t%apply: (du, dv) by hordiff_colocated_xyz_t%calc_diff_vec_xyz
   (hordiff_colocated_mod.f90:42-58: covariant components to Cartesian with the contravariant
   basis, the scalar diffusion of each Cartesian component, back with the same basis as
   cart2cube_vec does for covariant components, vec_math_mod.f90:196-219, then the covariant
   ECS Ah vector sync), dh by the scalar diffusion */
static void op_diff_ah(orc_ctx *c, fld_t *dh, fld_t *du, fld_t *dv, fld_t *h, fld_t *u, fld_t *v, double uv_coeff,
                       double h_coeff, int ord)
{
    const int n = c->N + 1;
    const mesh_t *m = &c->mxy;
    diff_alloc(c);
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= n; j++)
            for (int i = 1; i <= n; i++) {
                const size_t k = MI(m, t, i, j);
                for (int d = 0; d < 3; d++)
                    FA(&c->df_x[d], t, i, j) = m->b1[3 * k + d] * FA(u, t, i, j) + m->b2[3 * k + d] * FA(v, t, i, j);
            }
    for (int d = 0; d < 3; d++) hordiff_ah(c, &c->df_t[d], &c->df_x[d], &c->df_x[d], uv_coeff, ord);
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= n; j++)
            for (int i = 1; i <= n; i++) {
                const size_t k = MI(m, t, i, j);
                const double tx = FA(&c->df_t[0], t, i, j), ty = FA(&c->df_t[1], t, i, j), tz = FA(&c->df_t[2], t, i, j);
                FA(du, t, i, j) = tx * m->b1[3 * k] + ty * m->b1[3 * k + 1] + tz * m->b1[3 * k + 2];
                FA(dv, t, i, j) = tx * m->b2[3 * k] + ty * m->b2[3 * k + 1] + tz * m->b2[3 * k + 2];
            }
    exch_do(&c->ex_xy1_cross_v, du, dv);
    for (int t = 0; t < NPAN; t++) sync_grad_on_edges(c, dv, du, t);
    hordiff_ah(c, dh, h, &c->df_x[0], h_coeff, ord);
}

/* stvec assign/update over interior points (grid_field_mod.f90:442-534) */
static void st_assign2(fld_t *y[3], double s1, fld_t *a[3], double s2, fld_t *b[3])
{
    for (int f = 0; f < 3; f++)
        for (int t = 0; t < NPAN; t++)
            for (int j = 1; j <= y[f]->ny; j++)
                for (int i = 1; i <= y[f]->nx; i++)
                    FA(y[f], t, i, j) = s1 * FA(a[f], t, i, j) + s2 * FA(b[f], t, i, j);
}
static void st_update2(fld_t *y[3], double s1, fld_t *a[3], double s2, fld_t *b[3])
{
    for (int f = 0; f < 3; f++)
        for (int t = 0; t < NPAN; t++)
            for (int j = 1; j <= y[f]->ny; j++)
                for (int i = 1; i <= y[f]->nx; i++)
                    FA(y[f], t, i, j) = FA(y[f], t, i, j) + s1 * FA(a[f], t, i, j) + s2 * FA(b[f], t, i, j);
}

/* rk4_t%step (rk4_mod.f90:20-42) for the Ah state */
static void rk4_step_ah(orc_ctx *c, double dt)
{
    fld_t *v0[3] = {&c->h, &c->ah_u, &c->ah_v};
    fld_t *y[3] = {&c->ah_y[0], &c->ah_y[1], &c->ah_y[2]};
    fld_t *k[4][3];
    for (int s = 0; s < 4; s++)
        for (int f = 0; f < 3; f++) k[s][f] = &c->ah_k[s][f];
    op_apply_ah(c, k[0][0], k[0][1], k[0][2], v0[0], v0[1], v0[2]);
    st_assign2(y, 1.0, v0, 0.5 * dt, k[0]);
    op_apply_ah(c, k[1][0], k[1][1], k[1][2], y[0], y[1], y[2]);
    st_assign2(y, 1.0, v0, 0.5 * dt, k[1]);
    op_apply_ah(c, k[2][0], k[2][1], k[2][2], y[0], y[1], y[2]);
    st_assign2(y, 1.0, v0, dt, k[2]);
    op_apply_ah(c, k[3][0], k[3][1], k[3][2], y[0], y[1], y[2]);
    st_update2(v0, dt / 6.0, k[0], dt / 3.0, k[1]);
    st_update2(v0, dt / 3.0, k[2], dt / 6.0, k[3]);
}

/* rk4_t%step (rk4_mod.f90:20-42) */
static void rk4_step(orc_ctx *c, double dt)
{
    fld_t *v0[3] = {&c->h, &c->u, &c->v};
    fld_t *y[3] = {&c->y[0], &c->y[1], &c->y[2]};
    fld_t *k1[3] = {&c->k[0][0], &c->k[0][1], &c->k[0][2]};
    fld_t *k2[3] = {&c->k[1][0], &c->k[1][1], &c->k[1][2]};
    fld_t *k3[3] = {&c->k[2][0], &c->k[2][1], &c->k[2][2]};
    fld_t *k4[3] = {&c->k[3][0], &c->k[3][1], &c->k[3][2]};
    op_apply(c, k1[0], k1[1], k1[2], v0[0], v0[1], v0[2]);
    st_assign2(y, 1.0, v0, 0.5 * dt, k1);
    op_apply(c, k2[0], k2[1], k2[2], y[0], y[1], y[2]);
    st_assign2(y, 1.0, v0, 0.5 * dt, k2);
    op_apply(c, k3[0], k3[1], k3[2], y[0], y[1], y[2]);
    st_assign2(y, 1.0, v0, dt, k3);
    op_apply(c, k4[0], k4[1], k4[2], y[0], y[1], y[2]);
    st_update2(v0, dt / 6.0, k1, dt / 3.0, k2);
    st_update2(v0, dt / 3.0, k3, dt / 6.0, k4);
}

/* ------------------------------------------------------------------ */
/* quadrature (sbp_quadrature_mod.f90:22-62, abstract_quadrature_mod.f90:29-64) */
/* ------------------------------------------------------------------ */
static double q_dot(const mesh_t *m, const fld_t *f1, const fld_t *f2)
{
    double out = 0.0;
    for (int t = 0; t < NPAN; t++) {
        double tile = 0.0;
        for (int j = 1; j <= m->ny; j++)
            for (int i = 1; i <= m->nx; i++) {
                double w = (f2 ? FA(f1, t, i, j) * FA(f2, t, i, j) : FA(f1, t, i, j));
                tile = tile + w * m->J[MI(m, t, i, j)] * m->hx * m->hy * m->Ax[i - 1] * m->Ay[j - 1];
            }
        out = out + tile;
    }
    return out;
}

/* curl_sbp_sat_t%calc_curl for curl_ch_sbp_sat_{21,42,63} (curl_sbp_sat_mod.f90:27-76,
   curl_factory_mod.f90:89-97,113-117): the i2c difference of the covariant u in y
   and of v in x, each with its SAT correction against the neighbour's copy of the
   tangential component on the panel edge (the Ch vector exchange puts it at halo
   index 0 / N+2), on mesh o:
       curl = (Dx(v) / hx - Dy(u) / hy) / (J a)                                     */
static void op_curl(orc_ctx *c, fld_t *curl, fld_t *u, fld_t *v)
{
    int N = c->N;
    exch_do(&c->ex_ch3_u, u, v);
    exch_do(&c->ex_ch3_v, u, v);
    const mesh_t *m = &c->mo;
    for (int t = 0; t < NPAN; t++) {
        diff_i2c(&c->oDy, u, t, 1, N, 1, N, c->ord);
        diff_i2c(&c->oDx, v, t, 0, N, 1, N, c->ord);
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N; i++)
                FA(curl, t, i, j) = (FA(&c->oDx, t, i, j) / m->hx - FA(&c->oDy, t, i, j) / m->hy) /
                                    (m->J[MI(m, t, i, j)] * c->a);
    }
}

/* swm_output_diag_t%calc_energies for covariant (u, v) on Ch (swm_output_diag_mod.f90:186-234;
   operators of the Ch diagnostics configuration: co2contra_ch_sbp*, curl_ch_sbp_sat_*,
   interp2d_p2uv_Ch_sbp*, interp2d_uv2qvec_Ch_sbp*, SBP_C*_quadrature):
     KE = <hu ut u>_u / 2 + <hv vt v>_v / 2,  hu, hv = I_i2c(h) along x, y
     PE = g/2 <h h>_xy  (no orography)
     enstrophy = < (curl + f)^2 / (2 hq) >_o,  hq = (I_i2c,y(hu) + I_i2c,x(hv)) / 2
   out = {TE, KE, PE, enstrophy} */
static void op_energies(orc_ctx *c, double *out, fld_t *h, fld_t *u, fld_t *v)
{
    int N = c->N;
    op_co2contra(c, &c->ut, &c->vt, u, v);
    op_curl(c, &c->curl, u, v);
    for (int t = 0; t < NPAN; t++) {
        interp_i2c(&c->ehu, h, t, 0, N, 1, N + 1, c->ord);
        interp_i2c(&c->ehv, h, t, 1, N, 1, N + 1, c->ord);
    }
    for (int t = 0; t < NPAN; t++) {
        interp_i2c(&c->hqu, &c->ehu, t, 1, N, 1, N, c->ord);
        interp_i2c(&c->hqv, &c->ehv, t, 0, N, 1, N, c->ord);
    }
    const mesh_t *m = &c->mo;
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N; i++) {
                const double hq = 0.5 * FA(&c->hqu, t, i, j) + 0.5 * FA(&c->hqv, t, i, j);
                const double w = FA(&c->curl, t, i, j) + c->fo[MI(m, t, i, j)];
                FA(&c->hqu, t, i, j) = 0.5 * w * w / hq;
            }
    for (int t = 0; t < NPAN; t++) {
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N; i++)
                FA(&c->ehu, t, i, j) = 0.5 * (FA(&c->ehu, t, i, j) * FA(&c->ut, t, i, j)) * FA(u, t, i, j);
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N + 1; i++)
                FA(&c->ehv, t, i, j) = 0.5 * (FA(&c->ehv, t, i, j) * FA(&c->vt, t, i, j)) * FA(v, t, i, j);
    }
    const double ke = q_dot(&c->my, &c->ehu, NULL) + q_dot(&c->mx, &c->ehv, NULL);
    const double pe = 0.5 * c->g * q_dot(&c->mxy, h, h);
    out[0] = ke + pe;
    out[1] = ke;
    out[2] = pe;
    out[3] = q_dot(m, &c->hqu, NULL);
}

/* ------------------------------------------------------------------ */
/* exported API (ctypes)                                               */
/* ------------------------------------------------------------------ */
static void load_state(orc_ctx *c, const double *h, const double *u, const double *v)
{
    fld_from_packed(&c->h, h); fld_from_packed(&c->u, u); fld_from_packed(&c->v, v);
}
static void store_state(orc_ctx *c, double *h, double *u, double *v)
{
    fld_to_packed(&c->h, h); fld_to_packed(&c->u, u); fld_to_packed(&c->v, v);
}

int orc_N(const orc_ctx *c) { return c->N; }

/* operator kind: 0 linear_swm_operator, 1 advective_swm_operator (covariant Ch) */
void orc_set_operator(orc_ctx *c, int kind) { c->nonlinear = kind == 1; }

/* C-grid operators on packed fields: h (6, N, N) on the cell centres, u (6, N, N+1) on the
   x mesh, v (6, N+1, N) on the y mesh, each [t][j][i] with i fastest. */
void orc_c_grad(orc_ctx *c, const double *h, double *gx, double *gy)
{
    c_init(c);
    fld_from_packed(&c->c_h, h);
    op_grad_c(c, &c->c_gx, &c->c_gy, &c->c_h);
    fld_to_packed(&c->c_gx, gx);
    fld_to_packed(&c->c_gy, gy);
}
void orc_c_div(orc_ctx *c, const double *ut, const double *vt, double *div)
{
    c_init(c);
    fld_from_packed(&c->c_ut, ut);
    fld_from_packed(&c->c_vt, vt);
    op_div_c(c, &c->c_div, &c->c_ut, &c->c_vt);
    fld_to_packed(&c->c_div, div);
}
void orc_c_co2contra(orc_ctx *c, const double *u, const double *v, double *ut, double *vt)
{
    c_init(c);
    fld_from_packed(&c->c_u, u);
    fld_from_packed(&c->c_v, v);
    op_co2contra_c(c, &c->c_ut, &c->c_vt, &c->c_u, &c->c_v);
    fld_to_packed(&c->c_ut, ut);
    fld_to_packed(&c->c_vt, vt);
}
/* SBP_C42 quadrature weights on the C meshes: mesh 0 = o, 1 = x, 2 = y (packed like the fields). */
void orc_c_weights(orc_ctx *c, int mesh, double *w)
{
    const mesh_t *m = mesh == 0 ? &c->mo : (mesh == 1 ? &c->mx : &c->my);
    size_t k = 0;
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= m->ny; j++)
            for (int i = 1; i <= m->nx; i++) {
                const size_t q = MI(m, t, i, j);
                w[k++] = m->J[q] * m->hx * m->hy * m->Ax[i - 1] * m->Ay[j - 1];
            }
}
/* The C halos as the exchanges deliver them: kind 0 the o-point scalar exchange of width 3
   (f on o), kind 1 the C vector exchange of width 3 (f = u on x, f2 = v on y); the ring of
   width w around every panel is written like orc_halo_probe's. */
void orc_c_halo_probe(orc_ctx *c, int kind, const double *f, const double *f2, int w, double *out, double *out2);

/* Orography h_surf of the advective operator (operator_adv_swm_mod.f90:37-38,78:
   h_total = h + h_surf is the gradient's input), packed [t][j][i] on xy; NULL clears it. */
void orc_set_orography(orc_ctx *c, const double *hs)
{
    const size_t n = (size_t)NPAN * (c->N + 1) * (c->N + 1);
    if (!hs) { free(c->hsurf); c->hsurf = NULL; return; }
    if (!c->hsurf) c->hsurf = malloc(sizeof(double) * n);
    memcpy(c->hsurf, hs, sizeof(double) * n);
}

/* SBP order of the Ch operators (the _21 / _42 / _63 operator names of the reference's
   factories: grad_ch_sbp_sat_*, div_ch_sbp_sat_*_proj, co2contra_ch_sbp*,
   coriolis_Ch_sbp*, SBP_C*_quadrature); returns 0, or -1 for an unknown order. */
int orc_set_sbp_order(orc_ctx *c, int ord)
{
    if (ord != 21 && ord != 42 && ord != 63) return -1;
    if (ord == 63 && c->N < 16) return -1;
    c->ord = ord;
    mesh_mass(&c->mxy, ord);
    mesh_mass(&c->mx, ord);
    mesh_mass(&c->my, ord);
    mesh_mass(&c->mo, ord);
    return 0;
}

void orc_apply(orc_ctx *c, const double *h, const double *u, const double *v, double *dh, double *du, double *dv)
{
    load_state(c, h, u, v);
    op_apply(c, &c->dh, &c->du, &c->dv, &c->h, &c->u, &c->v);
    fld_to_packed(&c->dh, dh); fld_to_packed(&c->du, du); fld_to_packed(&c->dv, dv);
}

void orc_rk4(orc_ctx *c, double *h, double *u, double *v, double dt, int nsteps)
{
    load_state(c, h, u, v);
    for (int s = 0; s < nsteps; s++) rk4_step(c, dt);
    store_state(c, h, u, v);
}

/* individual operators for fine-grained parity: outputs in packed layout */
void orc_grad(orc_ctx *c, const double *h, double *gx, double *gy)
{
    fld_from_packed(&c->h, h);
    op_grad(c, &c->gx, &c->gy, &c->h);
    fld_to_packed(&c->gx, gx); fld_to_packed(&c->gy, gy);
}
void orc_co2contra(orc_ctx *c, const double *u, const double *v, double *ut, double *vt)
{
    fld_from_packed(&c->u, u); fld_from_packed(&c->v, v);
    op_co2contra(c, &c->ut, &c->vt, &c->u, &c->v);
    fld_to_packed(&c->ut, ut); fld_to_packed(&c->vt, vt);
}
void orc_coriolis(orc_ctx *c, const double *ut, const double *vt, double *cu, double *cv)
{
    fld_from_packed(&c->ut, ut); fld_from_packed(&c->vt, vt);
    op_coriolis(c, &c->gx, &c->gy, &c->ut, &c->vt);
    fld_to_packed(&c->gx, cu); fld_to_packed(&c->gy, cv);
}
void orc_div(orc_ctx *c, const double *ut, const double *vt, double *div)
{
    fld_from_packed(&c->ut, ut); fld_from_packed(&c->vt, vt);
    op_div(c, &c->div, &c->ut, &c->vt);
    fld_to_packed(&c->div, div);
}

/* mass = <h,1>_Hh and the linear energy
   E = H/2 (<u,ut>_Hu + <v,vt>_Hv) + g/2 <h,h>_Hh  with (ut, vt) = co2contra(u, v) */
void orc_integrals(orc_ctx *c, const double *h, const double *u, const double *v, double *mass, double *energy)
{
    load_state(c, h, u, v);
    op_co2contra(c, &c->ut, &c->vt, &c->u, &c->v);
    double m = q_dot(&c->mxy, &c->h, NULL);
    double eu = q_dot(&c->my, &c->u, &c->ut);
    double ev = q_dot(&c->mx, &c->v, &c->vt);
    double eh = q_dot(&c->mxy, &c->h, &c->h);
    if (mass) *mass = m;
    if (energy) *energy = 0.5 * c->H * (eu + ev) + 0.5 * c->g * eh;
}

/* swm_output_diag_t diagnostics (swm_output_diag_mod.f90:110-154 print_CFL_diag,
   :160-171 the extrema of print_integrals_diag): out = {h_min, h_max, CFL of the
   gravity waves, advective CFL in x, in y}.  The CFL numbers are
   sqrt(max (g / min(dx,dy)^2) h) dt and sqrt(maxabs (1/dx^2) ut u) dt (likewise y),
   with (ut, vt) = co2contra(u, v) and dx = a hx on the xy mesh. */
void orc_diag(orc_ctx *c, const double *h, const double *u, const double *v, double dt, double *out)
{
    load_state(c, h, u, v);
    op_co2contra(c, &c->ut, &c->vt, &c->u, &c->v);
    const int N = c->N;
    const double dx = c->a * c->mxy.hx, dy = c->a * c->mxy.hy, dm = dx < dy ? dx : dy;
    const double cg = c->g / (dm * dm), cx = 1.0 / (dx * dx), cy = 1.0 / (dy * dy);
    double hmin = INFINITY, hmax = -INFINITY, gmax = -INFINITY, umax = 0.0, vmax = 0.0;
    for (int t = 0; t < NPAN; t++) {
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N + 1; i++) {
                const double hv = FA(&c->h, t, i, j);
                hmin = hv < hmin ? hv : hmin;
                hmax = hv > hmax ? hv : hmax;
                const double gv = cg * hv;
                gmax = gv > gmax ? gv : gmax;
            }
        for (int j = 1; j <= N + 1; j++)
            for (int i = 1; i <= N; i++) {
                const double p = fabs(cx * FA(&c->ut, t, i, j) * FA(&c->u, t, i, j));
                umax = p > umax ? p : umax;
            }
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N + 1; i++) {
                const double p = fabs(cy * FA(&c->vt, t, i, j) * FA(&c->v, t, i, j));
                vmax = p > vmax ? p : vmax;
            }
    }
    out[0] = hmin;
    out[1] = hmax;
    out[2] = sqrt(gmax) * dt;
    out[3] = sqrt(umax) * dt;
    out[4] = sqrt(vmax) * dt;
}

/* latlon_regrid_t%do_regrid of an xy scalar with cubic interpolation (latlon_outputer_mod.f90:30-53,
   regrid_factory_mod.f90:25-70,165-262 distribute_latlon_points_to_cubsphere,
   latlon_regrid_mod.f90:286-365 init_interpolation / interpolate,
   latlon_grid_generator_mod.f90 init / get_cartesian_coords): the field gets an ECS_xy
   halo of width 2 (on a copy), every point of the nlat x nlon grid
   (phi_j = -pi/2 + (j-1) pi/(nlat-1), lam_i = (i-1) 2pi/nlon) is located on its panel,
   and the 4 x 4 cubic Lagrange stencil around it is summed.  out[j][i], i fastest. */
void orc_latlon_xy(orc_ctx *c, const double *f, int nlat, int nlon, double *out)
{
    fld_t *b = &c->htot;
    fld_from_packed(b, f);
    ecs_xy_halo(c, b, 2);
    const mesh_t *m = &c->mxy;
    const double alpha0 = -0.25 * PI_, beta0 = -0.25 * PI_;
    for (int j = 1; j <= nlat; j++) {
        const double phi = -0.5 * PI_ + (j - 1) * PI_ / (nlat - 1.0);
        for (int i = 1; i <= nlon; i++) {
            const double lam = (i - 1) * 2.0 * PI_ / nlon;
            const double r[3] = {cos(phi) * cos(lam), cos(phi) * sin(lam), sin(phi)};
            int t;
            double alpha, beta;
            cart_to_native(r, &t, &alpha, &beta);
            double zdx = (alpha - alpha0) / m->hx + 1 - m->shift_i;
            double zdy = (beta - beta0) / m->hy + 1 - m->shift_j;
            const int xi = (int)zdx, yi = (int)zdy;
            zdx = zdx - xi;
            zdy = zdy - yi;
            double wx[4], wy[4];
            wx[0] = -zdx * (zdx - 1.0) * (zdx - 2.0) / 6.0;
            wx[1] = (zdx + 1.0) * (zdx - 1.0) * (zdx - 2.0) / 2.0;
            wx[2] = -(zdx + 1.0) * zdx * (zdx - 2.0) / 2.0;
            wx[3] = (zdx + 1.0) * zdx * (zdx - 1.0) / 6.0;
            wy[0] = -zdy * (zdy - 1.0) * (zdy - 2.0) / 6.0;
            wy[1] = (zdy + 1.0) * (zdy - 1.0) * (zdy - 2.0) / 2.0;
            wy[2] = -(zdy + 1.0) * zdy * (zdy - 2.0) / 2.0;
            wy[3] = (zdy + 1.0) * zdy * (zdy - 1.0) / 6.0;
            double acc = 0.0;
            for (int q = -1; q <= 2; q++)
                for (int p = -1; p <= 2; p++) acc = acc + wx[p + 1] * wy[q + 1] * FA(b, t, xi + p, yi + q);
            out[(size_t)(j - 1) * nlon + (i - 1)] = acc;
        }
    }
}

/* ---- ECS_O scalar halo of width 2 and the lat-lon regrid of an o field ---- */

/* init_halo_interp (ecs_halo_factory_mod.f90:190-230): for the cell-centre line i of a
   virtual row j beyond the edge, the source face's cell left of the projected point
   (*ind) and the cubic Lagrange weights w[0..3] on its cells ind-1 .. ind+2. */
static void halo_o_weights(double dxa, int i, int j, double w[4], int *ind)
{
    const double zb = 0.25 * PI_ + (j - 0.5) * dxa;
    double za = -0.25 * PI_ + (i - 0.5) * dxa;
    double zx = tan(za);
    const double zz = tan(zb);
    zx = zx / zz;
    za = atan(zx);
    const int k = (int)floor((za + 0.25 * PI_ - 0.5 * dxa) / dxa) + 1;
    const double zxi = (za + 0.25 * PI_) / dxa - (k - 0.5);
    w[0] = -(zxi * (zxi - 1.0) * (zxi - 2.0) / 6.0);
    w[1] = (zxi + 1.0) * (zxi - 1.0) * (zxi - 2.0) / 2.0;
    w[2] = -((zxi + 1.0) * zxi * (zxi - 2.0) / 2.0);
    w[3] = (zxi + 1.0) * zxi * (zxi - 1.0) / 6.0;
    *ind = k;
}

static void llo_init(orc_ctx *c)
{
    if (c->llo) return;
    build_o_exchange(&c->ex_o5, c->N, 5, 0);
    fld_init(&c->o_ll, c->N, c->N, 5);
    c->llo = 1;
}

/* get_ecs_halo + ext_ecs_tile_halo (ecs_halo_mod.f90:74-175) of an o field on whole
   panels, halo width 2: the o-point exchange; the six special points of every cube corner
   from the exchanged values (ecs_halo_corners / ecs_halo_1corner, :179-300); the rows
   of virtual points interpolated along the neighbours' grid lines (ecs_halo_edges_x /
   _y, ecs_ext_halo_1e, :340-477; the first row leaves out its two end points); then the
   corner values put in place (ecs_halo_corners_put, :302-338). */
static void ecs_o_halo(orc_ctx *c, fld_t *f)
{
    const int n = c->N, hw = 2, ni = n + 4;
    const double dxa = c->mo.hx;
    exch_do(&c->ex_o5, f, NULL);
    /* the weights of the x edges, target i = -1 .. n+2, rows 1..hw (wx: both directions and
       the corners use them) */
    double *W = malloc(sizeof(double) * 4 * ni * hw);
    int *K = malloc(sizeof(int) * ni * hw);
#define WI(i, j) (((j) - 1) * ni + (i) + 1)
    for (int j = 1; j <= hw; j++)
        for (int i = -1; i <= n + 2; i++) halo_o_weights(dxa, i, j, &W[4 * WI(i, j)], &K[WI(i, j)]);
    double *zl = malloc(sizeof(double) * (n + 2)), *zh = malloc(sizeof(double) * (n + 2));
    static const int idirs[4] = {1, -1, -1, 1}, jdirs[4] = {1, 1, -1, -1};
    for (int t = 0; t < NPAN; t++) {
        double sp[4][6];
        for (int q = 0; q < 4; q++) {
            const int idir = idirs[q], jdir = jdirs[q];
            const int ist = idir > 0 ? 0 : n + 1, jst = jdir > 0 ? 0 : n + 1;
#define FC(i, j) FA(f, t, ist + idir * (i), jst + jdir * (j))
            /* corner weights: pw(k, i, j) = w(k, i, j), mirrored (k -> 1-k, i -> n+1-i) where idir = -1 */
#define PW(k, i, j) (idir > 0 ? W[4 * WI((i), (j)) + (k) + 1] : W[4 * WI(n + 1 - (i), (j)) + (1 - (k)) + 1])
            const double z0 = PW(0, 1, 1), z1 = PW(1, 1, 1), z2 = PW(2, 1, 1);
            const double zw = PW(-1, 1, 1), zw2 = zw * zw, zw3 = zw2 * zw;
            double zx = z0 * FC(0, 1) + z1 * FC(0, 2) + z2 * FC(0, 3);
            double zy = z0 * FC(1, 0) + z1 * FC(1, -1) + z2 * FC(1, -2);
            double zz = z0 * FC(1, 1) + z1 * FC(2, 1) + z2 * FC(3, 1);
            sp[q][0] = (zx + zw * zy + zw2 * zz) / (1 - zw3);
            const double zfy1 = (zy + zw * zz + zw2 * zx) / (1 - zw3);
            zx = z0 * FC(1, 0) + z1 * FC(2, 0) + z2 * FC(3, 0);
            zy = z0 * FC(0, 1) + z1 * FC(-1, 1) + z2 * FC(-2, 1);
            zz = z0 * FC(1, 1) + z1 * FC(1, 2) + z2 * FC(1, 3);
            sp[q][1] = (zx + zw * zy + zw2 * zz) / (1 - zw3);
            const double zfy2 = (zy + zw * zz + zw2 * zx) / (1 - zw3);
            double zff1 = PW(-1, 1, 2) * FC(2, 0) + PW(0, 1, 2) * FC(2, -1) + PW(1, 1, 2) * FC(2, -2) +
                          PW(2, 1, 2) * FC(2, -3);
            double zff2 = PW(-1, 1, 2) * FC(0, 2) + PW(0, 1, 2) * FC(-1, 2) + PW(1, 1, 2) * FC(-2, 2) +
                          PW(2, 1, 2) * FC(-3, 2);
            sp[q][2] = 0.5 * (PW(-1, 0, 1) * zff1 + PW(0, 0, 1) * zfy1 + PW(1, 0, 1) * FC(0, 1) + PW(2, 0, 1) * FC(0, 2) +
                              PW(-1, 0, 1) * zff2 + PW(0, 0, 1) * zfy2 + PW(1, 0, 1) * FC(1, 0) + PW(2, 0, 1) * FC(2, 0));
            zff1 = PW(-1, 2, 1) * FC(1, 0) + PW(0, 2, 1) * FC(1, -1) + PW(1, 2, 1) * FC(1, -2) + PW(2, 2, 1) * FC(1, -3);
            const double zff11 = PW(-1, 2, 2) * FC(2, -1) + PW(0, 2, 2) * FC(2, -2) + PW(1, 2, 2) * FC(2, -3) +
                                 PW(2, 2, 2) * FC(2, -4);
            zff2 = PW(-1, 2, 1) * FC(0, 1) + PW(0, 2, 1) * FC(-1, 1) + PW(1, 2, 1) * FC(-2, 1) + PW(2, 2, 1) * FC(-3, 1);
            const double zff22 = PW(-1, 2, 2) * FC(-1, 2) + PW(0, 2, 2) * FC(-2, 2) + PW(1, 2, 2) * FC(-3, 2) +
                                 PW(2, 2, 2) * FC(-4, 2);
            sp[q][3] = PW(-1, 0, 2) * zff1 + PW(0, 0, 2) * FC(-1, 1) + PW(1, 0, 2) * FC(-1, 2) + PW(2, 0, 2) * FC(-1, 3);
            sp[q][4] = PW(-1, 0, 2) * zff2 + PW(0, 0, 2) * FC(1, -1) + PW(1, 0, 2) * FC(2, -1) + PW(2, 0, 2) * FC(3, -1);
            sp[q][5] = 0.5 * (PW(-1, -1, 2) * zff11 + PW(0, -1, 2) * zff1 + PW(1, -1, 2) * FC(-1, 1) +
                              PW(2, -1, 2) * FC(-1, 2) + PW(-1, -1, 2) * zff22 + PW(0, -1, 2) * zff2 +
                              PW(1, -1, 2) * FC(1, -1) + PW(2, -1, 2) * FC(2, -1));
#undef PW
        }
        /* edges: virtual row m (1..hw) of each side from the exchanged row m of the neighbour */
        for (int side = 0; side < 4; side++)
            for (int m = 1; m <= hw; m++) {
                for (int b = 1; b <= n; b++)
                    zl[b] = side == 0 ? FA(f, t, b, 1 - m) : side == 1 ? FA(f, t, b, n + m)
                          : side == 2 ? FA(f, t, 1 - m, b) : FA(f, t, n + m, b);
                const int a0 = m == 1 ? 2 : 1, a1 = m == 1 ? n - 1 : n;
                for (int a = a0; a <= a1; a++) {
                    const double *w = &W[4 * WI(a, m)];
                    const int ii = K[WI(a, m)];
                    zh[a] = w[0] * zl[ii - 1] + w[1] * zl[ii] + w[2] * zl[ii + 1] + w[3] * zl[ii + 2];
                }
                for (int a = a0; a <= a1; a++) {
                    if (side == 0) FA(f, t, a, 1 - m) = zh[a];
                    else if (side == 1) FA(f, t, a, n + m) = zh[a];
                    else if (side == 2) FA(f, t, 1 - m, a) = zh[a];
                    else FA(f, t, n + m, a) = zh[a];
                }
            }
        /* the special points: corner-local (0,1), (1,0), (0,0), (-1,0), (0,-1), (-1,-1) */
        static const int pi_[6] = {0, 1, 0, -1, 0, -1}, pj_[6] = {1, 0, 0, 0, -1, -1};
        for (int q = 0; q < 4; q++) {
            const int idir = idirs[q], jdir = jdirs[q];
            const int ist = idir > 0 ? 0 : n + 1, jst = jdir > 0 ? 0 : n + 1;
            for (int p = 0; p < 6; p++) FC(pi_[p], pj_[p]) = sp[q][p];
        }
#undef FC
    }
#undef WI
    free(W); free(K); free(zl); free(zh);
}

/* latlon_regrid_t%do_regrid of an o field (the curl output of output_curl on Ch,
   swm_output_diag_mod.f90:78-90; swm_output_diag_factory_mod.f90:48-52 curl_points 'o';
   init_halo_for_interp 'o' cubic: the ECS_O halo of width 2, regrid_factory_mod.f90:285-287):
   the cubic stencils of latlon_regrid_mod.f90:286-365 on the cell-centre mesh
   (shift 1/2).  f: (6, N, N) packed; out[j][i], i fastest. */
void orc_latlon_o(orc_ctx *c, const double *f, int nlat, int nlon, double *out)
{
    llo_init(c);
    fld_t *b = &c->o_ll;
    for (size_t k = 0; k < b->psz * NPAN; k++) b->p[k] = NAN;
    fld_from_packed(b, f);
    ecs_o_halo(c, b);
    const mesh_t *m = &c->mo;
    const double alpha0 = -0.25 * PI_, beta0 = -0.25 * PI_;
    for (int j = 1; j <= nlat; j++) {
        const double phi = -0.5 * PI_ + (j - 1) * PI_ / (nlat - 1.0);
        for (int i = 1; i <= nlon; i++) {
            const double lam = (i - 1) * 2.0 * PI_ / nlon;
            const double r[3] = {cos(phi) * cos(lam), cos(phi) * sin(lam), sin(phi)};
            int t;
            double alpha, beta;
            cart_to_native(r, &t, &alpha, &beta);
            double zdx = (alpha - alpha0) / m->hx + 1 - m->shift_i;
            double zdy = (beta - beta0) / m->hy + 1 - m->shift_j;
            const int xi = (int)zdx, yi = (int)zdy;
            zdx = zdx - xi;
            zdy = zdy - yi;
            double wx[4], wy[4];
            wx[0] = -zdx * (zdx - 1.0) * (zdx - 2.0) / 6.0;
            wx[1] = (zdx + 1.0) * (zdx - 1.0) * (zdx - 2.0) / 2.0;
            wx[2] = -(zdx + 1.0) * zdx * (zdx - 2.0) / 2.0;
            wx[3] = (zdx + 1.0) * zdx * (zdx - 1.0) / 6.0;
            wy[0] = -zdy * (zdy - 1.0) * (zdy - 2.0) / 6.0;
            wy[1] = (zdy + 1.0) * (zdy - 1.0) * (zdy - 2.0) / 2.0;
            wy[2] = -(zdy + 1.0) * zdy * (zdy - 2.0) / 2.0;
            wy[3] = (zdy + 1.0) * zdy * (zdy - 1.0) / 6.0;
            double acc = 0.0;
            for (int q = -1; q <= 2; q++)
                for (int p = -1; p <= 2; p++) acc = acc + wx[p + 1] * wy[q + 1] * FA(b, t, xi + p, yi + q);
            out[(size_t)(j - 1) * nlon + (i - 1)] = acc;
        }
    }
}

/* Ah staggering: the linear operator's tendency and RK4 steps of a state with h, u, v
   all on the xy mesh (each packed [t][j][i], (N+1) x (N+1) per panel) */
void orc_ah_apply(orc_ctx *c, const double *h, const double *u, const double *v, double *dh, double *du, double *dv)
{
    fld_from_packed(&c->h, h); fld_from_packed(&c->ah_u, u); fld_from_packed(&c->ah_v, v);
    op_apply_ah(c, &c->dh, &c->ah_du, &c->ah_dv, &c->h, &c->ah_u, &c->ah_v);
    fld_to_packed(&c->dh, dh); fld_to_packed(&c->ah_du, du); fld_to_packed(&c->ah_dv, dv);
}
/* the narrow Laplacian orders built: 2-1, 4-2 where its two closure blocks of six rows do not
   overlap (N >= 11), 6-3 where its blocks of nine rows do not (N >= 17) */
static int diff_order_ok(const orc_ctx *c, int lap_order)
{
    return lap_order == 21 || (lap_order == 42 && c->N >= 11) || (lap_order == 63 && c->N >= 17);
}
/* the diffusion operator's tendency (lap_order 21 or 42: the _sbp_<order>_narrow operators) */
int orc_diff_apply(orc_ctx *c, const double *h, const double *u, const double *v, double *dh, double *du, double *dv,
                   int lap_order, double uv_coeff, double h_coeff)
{
    if (!diff_order_ok(c, lap_order)) return -1;
    fld_from_packed(&c->h, h); fld_from_packed(&c->ah_u, u); fld_from_packed(&c->ah_v, v);
    op_diff_ah(c, &c->dh, &c->ah_du, &c->ah_dv, &c->h, &c->ah_u, &c->ah_v, uv_coeff, h_coeff, lap_order);
    fld_to_packed(&c->dh, dh); fld_to_packed(&c->ah_du, du); fld_to_packed(&c->ah_dv, dv);
    return 0;
}
/* the narrow Laplacian alone (laplace_Ah_sbp<lap_order>_narrow), for tests of the operator */
int orc_lap_ah(orc_ctx *c, const double *f, double *out, int lap_order)
{
    if (!diff_order_ok(c, lap_order)) return -1;
    diff_alloc(c);
    fld_from_packed(&c->df_x[0], f);
    lap_ah(c, &c->df_t[0], &c->df_x[0], lap_order);
    fld_to_packed(&c->df_t[0], out);
    return 0;
}
/* nsteps explicit_Eul1 steps of the diffusion: v0 = v0 + dt tend (stvec update_s1v1) */
int orc_diff_step(orc_ctx *c, double *h, double *u, double *v, double dt, int lap_order, double uv_coeff,
                  double h_coeff, int nsteps)
{
    if (!diff_order_ok(c, lap_order)) return -1;
    const int n = c->N + 1;
    fld_from_packed(&c->h, h); fld_from_packed(&c->ah_u, u); fld_from_packed(&c->ah_v, v);
    fld_t *y[3] = {&c->h, &c->ah_u, &c->ah_v}, *k[3] = {&c->dh, &c->ah_du, &c->ah_dv};
    for (int s = 0; s < nsteps; s++) {
        op_diff_ah(c, k[0], k[1], k[2], y[0], y[1], y[2], uv_coeff, h_coeff, lap_order);
        for (int f = 0; f < 3; f++)
            for (int t = 0; t < NPAN; t++)
                for (int j = 1; j <= n; j++)
                    for (int i = 1; i <= n; i++) FA(y[f], t, i, j) = FA(y[f], t, i, j) + dt * FA(k[f], t, i, j);
    }
    fld_to_packed(&c->h, h); fld_to_packed(&c->ah_u, u); fld_to_packed(&c->ah_v, v);
    return 0;
}
void orc_ah_rk4(orc_ctx *c, double *h, double *u, double *v, double dt, int nsteps)
{
    fld_from_packed(&c->h, h); fld_from_packed(&c->ah_u, u); fld_from_packed(&c->ah_v, v);
    for (int s = 0; s < nsteps; s++) rk4_step_ah(c, dt);
    fld_to_packed(&c->h, h); fld_to_packed(&c->ah_u, u); fld_to_packed(&c->ah_v, v);
}
/* mass <h,1> and linear energy H/2 (<u,ut> + <v,vt>) + g/2 <h,h> in the SBP_Ah quadrature
   (quadrature_factory_mod.f90:31-66: the node norm in both directions) */
void orc_ah_integrals(orc_ctx *c, const double *h, const double *u, const double *v, double *mass, double *energy)
{
    fld_from_packed(&c->h, h); fld_from_packed(&c->ah_u, u); fld_from_packed(&c->ah_v, v);
    const int n = c->N + 1;
    const mesh_t *m = &c->mxy;
    const double A42[4] = {17.0 / 48.0, 59.0 / 48.0, 43.0 / 48.0, 49.0 / 48.0};
    const double A21[2] = {0.5, 1.0};   /* Q21_A (sbp_operators_collection_mod.f90:22) */
    double *A = malloc(sizeof(double) * n);
    if (c->ord == 21) mass_coeffs(A, n, A21, 2);
    else if (c->ord == 63) mass_coeffs(A, n, SBP63_NN_A, 6);
    else mass_coeffs(A, n, A42, 4);
    double sm = 0.0, se = 0.0, sh = 0.0;
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= n; j++)
            for (int i = 1; i <= n; i++) {
                const size_t k = MI(m, t, i, j);
                const double w = m->J[k] * m->hx * m->hy * A[i - 1] * A[j - 1];
                const double uu = FA(&c->ah_u, t, i, j), vv = FA(&c->ah_v, t, i, j), hh = FA(&c->h, t, i, j);
                const double ut = m->Q1[k] * uu + m->Q2[k] * vv, vt = m->Q2[k] * uu + m->Q3[k] * vv;
                sm += hh * w;
                sh += hh * hh * w;
                se += (uu * ut + vv * vt) * w;
            }
    free(A);
    if (mass) *mass = sm;
    if (energy) *energy = 0.5 * c->H * se + 0.5 * c->g * sh;
}

/* init_transform_matrix (ecs_halo_vec_xy_factory_mod.f90:103-186), covariant
   components: for halo row j (1 = the neighbour's copy of the edge row) at along
   index i of edge e (1 bottom, 2 top, 3 left, 4 right), the 2 x 2 matrix taking the
   neighbour's covariant components (as the exchange delivers them) to this panel's. */
static void xy_vec_tm(int e, int i, int j, double hx, double TM[4])
{
    static const int rot[4][3][3] = {{{1, 0, 0}, {0, 0, -1}, {0, 1, 0}},
                                     {{1, 0, 0}, {0, 0, 1}, {0, -1, 0}},
                                     {{0, 0, -1}, {0, 1, 0}, {1, 0, 0}},
                                     {{0, 0, 1}, {0, 1, 0}, {-1, 0, 0}}};
    static const int ab_shift[4] = {0, 0, 1, 1}, b_sign[4] = {1, -1, 1, -1};
    const int q = e - 1;
    const double alpha = -0.25 * PI_ + (i - 1.0) * hx;
    const double beta = b_sign[q] * (0.25 * PI_ - (j - 1.0) * hx);
    const double as = (1 - ab_shift[q]) * alpha + ab_shift[q] * beta;
    const double bs = ab_shift[q] * alpha + (1 - ab_shift[q]) * beta;
    double v[3], a1s[3], a2s[3], r[3], b1t[3], b2t[3];
    /* rot_matrix(m, d, e) in Fortran order: element (m, d) = rot[q][d][m] */
#define ROT(out, vin)                                                                                   \
    for (int d = 0; d < 3; d++)                                                                         \
        out[d] = rot[q][d][0] * vin[0] + rot[q][d][1] * vin[1] + rot[q][d][2] * vin[2];
    b1_proto(as, bs, v);
    ROT(a1s, v);
    b2_proto(as, bs, v);
    ROT(a2s, v);
    {
        const double ta = tan(as), tb = tan(bs);
        v[0] = ta / sqrt(1.0 + pow(ta, 2.0) + pow(tb, 2.0));
        v[1] = tb / sqrt(1.0 + pow(ta, 2.0) + pow(tb, 2.0));
        v[2] = 1.0 / sqrt(1.0 + pow(ta, 2.0) + pow(tb, 2.0));
    }
    ROT(r, v);
#undef ROT
    const double at = atan(r[0] / r[2]), bt = atan(r[1] / r[2]);
    a1_proto(at, bt, b1t);
    a2_proto(at, bt, b2t);
    TM[0] = a1s[0] * b1t[0] + a1s[1] * b1t[1] + a1s[2] * b1t[2];
    TM[1] = a2s[0] * b1t[0] + a2s[1] * b1t[1] + a2s[2] * b1t[2];
    TM[2] = a1s[0] * b2t[0] + a1s[1] * b2t[1] + a1s[2] * b2t[2];
    TM[3] = a2s[0] * b2t[0] + a2s[1] * b2t[1] + a2s[2] * b2t[2];
}

/* latlon_vec_outputer_t%write for covariant (u, v) on Ch (latlon_outputer_mod.f90:55-85,
   regrid_factory_mod.f90:72-163 create_latlon_vector_regrid, latlon_regrid_mod.f90:132-212
   do_latlon_vector_regrid): interp2d_uv2pvec_Ch_sbp* to the vertices, the covariant
   ecs_xy_vec halo of width 2 (exchange, transform matrices, ECS_xy interpolation of
   each component; ecs_halo_vec_xy_mod.f90:30-98), the cubic stencils, and the rotation
   to the lat-lon components (init_transform_to_latlon_vec_tile, regrid_factory_mod.f90:
   324-370: q = [iv.b1, iv.b2; jv.b1, jv.b2]).  uo, vo: [nlat][nlon]. */
void orc_latlon_vec(orc_ctx *c, const double *u, const double *v, int nlat, int nlon, double *uo, double *vo)
{
    const int N = c->N, n = N + 1, hw = 2;
    fld_from_packed(&c->u, u);
    fld_from_packed(&c->v, v);
    exch_do(&c->ex_ch3_u, &c->u, &c->v);
    exch_do(&c->ex_ch3_v, &c->u, &c->v);
    fld_t *bu = &c->uq, *bv = &c->vq;
    for (int t = 0; t < NPAN; t++) {
        /* the outputer's interpolator is interp2d_uv2pvec_Ch_sbp42 whatever the model's order */
        interp_c2i(bu, &c->u, t, 0, N + 1, 1, N + 1, 42);
        interp_c2i(bv, &c->v, t, 1, N + 1, 1, N + 1, 42);
    }
    exch_do(&c->ex_xy3_full_v, bu, bv);
    const double hx = c->mxy.hx;
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= hw + 1; j++)
            for (int i = 1; i <= n; i++) {
                double TM[4], zu, zv;
                xy_vec_tm(1, i, j, hx, TM);
                zu = FA(bu, t, i, 1 - j); zv = FA(bv, t, i, 1 - j);
                FA(bu, t, i, 1 - j) = TM[0] * zu + TM[1] * zv;
                FA(bv, t, i, 1 - j) = TM[2] * zu + TM[3] * zv;
                xy_vec_tm(2, i, j, hx, TM);
                zu = FA(bu, t, i, n + j); zv = FA(bv, t, i, n + j);
                FA(bu, t, i, n + j) = TM[0] * zu + TM[1] * zv;
                FA(bv, t, i, n + j) = TM[2] * zu + TM[3] * zv;
                xy_vec_tm(3, i, j, hx, TM);
                zu = FA(bu, t, 1 - j, i); zv = FA(bv, t, 1 - j, i);
                FA(bu, t, 1 - j, i) = TM[0] * zu + TM[1] * zv;
                FA(bv, t, 1 - j, i) = TM[2] * zu + TM[3] * zv;
                xy_vec_tm(4, i, j, hx, TM);
                zu = FA(bu, t, n + j, i); zv = FA(bv, t, n + j, i);
                FA(bu, t, n + j, i) = TM[0] * zu + TM[1] * zv;
                FA(bv, t, n + j, i) = TM[2] * zu + TM[3] * zv;
            }
    ecs_xy_interp(c, bu, hw);
    ecs_xy_interp(c, bv, hw);
    const mesh_t *m = &c->mxy;
    for (int j = 1; j <= nlat; j++) {
        const double phi = -0.5 * PI_ + (j - 1) * PI_ / (nlat - 1.0);
        for (int i = 1; i <= nlon; i++) {
            const double lam = (i - 1) * 2.0 * PI_ / nlon;
            const double r[3] = {cos(phi) * cos(lam), cos(phi) * sin(lam), sin(phi)};
            int t;
            double alpha, beta;
            cart_to_native(r, &t, &alpha, &beta);
            double zdx = (alpha + 0.25 * PI_) / m->hx + 1, zdy = (beta + 0.25 * PI_) / m->hy + 1;
            const int xi = (int)zdx, yi = (int)zdy;
            zdx = zdx - xi;
            zdy = zdy - yi;
            double wx[4], wy[4];
            wx[0] = -zdx * (zdx - 1.0) * (zdx - 2.0) / 6.0;
            wx[1] = (zdx + 1.0) * (zdx - 1.0) * (zdx - 2.0) / 2.0;
            wx[2] = -(zdx + 1.0) * zdx * (zdx - 2.0) / 2.0;
            wx[3] = (zdx + 1.0) * zdx * (zdx - 1.0) / 6.0;
            wy[0] = -zdy * (zdy - 1.0) * (zdy - 2.0) / 6.0;
            wy[1] = (zdy + 1.0) * (zdy - 1.0) * (zdy - 2.0) / 2.0;
            wy[2] = -(zdy + 1.0) * zdy * (zdy - 2.0) / 2.0;
            wy[3] = (zdy + 1.0) * zdy * (zdy - 1.0) / 6.0;
            double au = 0.0, av = 0.0;
            for (int qq = -1; qq <= 2; qq++)
                for (int p = -1; p <= 2; p++) {
                    au = au + wx[p + 1] * wy[qq + 1] * FA(bu, t, xi + p, yi + qq);
                    av = av + wx[p + 1] * wy[qq + 1] * FA(bv, t, xi + p, yi + qq);
                }
            /* latlon basis iv, jv and the contravariant basis b1, b2 of panel t at (alpha, beta) */
            const double iv[3] = {-sin(lam), cos(lam), 0.0};
            const double jv[3] = {-sin(phi) * cos(lam), -sin(phi) * sin(lam), cos(phi)};
            double p1[3], p2[3], b1[3], b2[3];
            b1_proto(alpha, beta, p1);
            b2_proto(alpha, beta, p2);
            proto2real(t, p1, b1);
            proto2real(t, p2, b2);
            const double q11 = iv[0] * b1[0] + iv[1] * b1[1] + iv[2] * b1[2];
            const double q12 = iv[0] * b2[0] + iv[1] * b2[1] + iv[2] * b2[2];
            const double q21 = jv[0] * b1[0] + jv[1] * b1[1] + jv[2] * b1[2];
            const double q22 = jv[0] * b2[0] + jv[1] * b2[1] + jv[2] * b2[2];
            const size_t k = (size_t)(j - 1) * nlon + (i - 1);
            uo[k] = q11 * au + q12 * av;
            vo[k] = q21 * au + q22 * av;
        }
    }
}

/* curl of the covariant (u, v) on mesh o (N x N per panel, packed [t][j][i]) */
void orc_curl(orc_ctx *c, const double *u, const double *v, double *out)
{
    fld_from_packed(&c->u, u); fld_from_packed(&c->v, v);
    op_curl(c, &c->curl, &c->u, &c->v);
    fld_to_packed(&c->curl, out);
}

/* out = {TE, KE, PE, enstrophy} of swm_output_diag_t%calc_energies */
void orc_energies(orc_ctx *c, const double *h, const double *u, const double *v, double *out)
{
    load_state(c, h, u, v);
    op_energies(c, out, &c->h, &c->u, &c->v);
}

/* SBP-weighted inner product on mesh 0 = xy (h), 1 = y (u), 2 = x (v) */
double orc_dot(orc_ctx *c, int mesh, const double *a, const double *b)
{
    fld_t *f1 = mesh == 0 ? &c->dh : (mesh == 1 ? &c->du : &c->dv);
    fld_t *f2 = mesh == 0 ? &c->div : (mesh == 1 ? &c->gx : &c->gy);
    const mesh_t *m = mesh == 0 ? &c->mxy : (mesh == 1 ? &c->my : &c->mx);
    fld_from_packed(f1, a);
    if (b) fld_from_packed(f2, b);
    return q_dot(m, f1, b ? f2 : NULL);
}

/* Gaussian hill h = amp*exp(-(r/d0)^2) on xy points, u = v = 0
   (test_fields_mod.f90:491-514, gaussian_hill_linear_test_mod.f90:30-68) */
void orc_init_gaussian(orc_ctx *c, double lam0, double phi0, double d0, double amp, double *h, double *u, double *v)
{
    double x0 = cos(phi0) * cos(lam0), y0 = cos(phi0) * sin(lam0), z0 = sin(phi0);
    mesh_t *m = &c->mxy;
    size_t k = 0;
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= m->ny; j++)
            for (int i = 1; i <= m->nx; i++, k++) {
                size_t q = MI(m, t, i, j);
                double d = m->rx[q] * x0 + m->ry[q] * y0 + m->rz[q] * z0;
                d = d > 1.0 ? 1.0 : (d < -1.0 ? -1.0 : d);
                double r = acos(d);
                h[k] = amp * exp(-pow(r / d0, 2));
            }
    size_t nu = (size_t)NPAN * c->my.nx * c->my.ny, nv = (size_t)NPAN * c->mx.nx * c->mx.ny;
    for (size_t q = 0; q < nu; q++) u[q] = 0.0;
    for (size_t q = 0; q < nv; q++) v[q] = 0.0;
}

/* Williamson test 2 (Williamson_test2_mod.f90:32-111, test_fields_mod.f90:586-615,857-894):
   solid rotation about 'axis' with speed u0, covariant components, and the balanced
   height; linear_mode drops the u0^2/2 metric term. */
void orc_init_ts2(orc_ctx *c, double u0, double h_mean, const double *axis_in, int linear_mode,
                  double *h, double *u, double *v)
{
    double am = sqrt(axis_in[0] * axis_in[0] + axis_in[1] * axis_in[1] + axis_in[2] * axis_in[2]);
    double ax = axis_in[0] / am, ay = axis_in[1] / am, az = axis_in[2] / am;
    double metric_term = linear_mode ? 0.0 : 1.0;
    mesh_t *m = &c->mxy;
    size_t k = 0;
    for (int t = 0; t < NPAN; t++)
        for (int j = 1; j <= m->ny; j++)
            for (int i = 1; i <= m->nx; i++, k++) {
                size_t q = MI(m, t, i, j);
                double x = m->rx[q], yy = m->ry[q], z = m->rz[q];
                double nr = sqrt(x * x + yy * yy + z * z);
                double phi = asin(x / nr * ax + yy / nr * ay + z / nr * az);
                h[k] = h_mean - (c->a * c->omega * u0 + metric_term * 0.5 * (u0 * u0)) / c->g * pow(sin(phi), 2);
            }
    for (int pass = 0; pass < 2; pass++) {
        mesh_t *mm = pass == 0 ? &c->my : &c->mx;
        double *dst = pass == 0 ? u : v;
        const double *bvec = pass == 0 ? mm->a1 : mm->a2;
        size_t kk = 0;
        for (int t = 0; t < NPAN; t++)
            for (int j = 1; j <= mm->ny; j++)
                for (int i = 1; i <= mm->nx; i++, kk++) {
                    size_t q = MI(mm, t, i, j);
                    double x = mm->rx[q], yy = mm->ry[q], z = mm->rz[q];
                    double nr = sqrt(x * x + yy * yy + z * z);
                    double xn = x / nr, yn = yy / nr, zn = z / nr;
                    double vx = u0 * (ay * zn - az * yn), vy = -u0 * (ax * zn - az * xn), vz = u0 * (ax * yn - ay * xn);
                    dst[kk] = vx * bvec[3 * q] + vy * bvec[3 * q + 1] + vz * bvec[3 * q + 2];
                }
    }
}

/* metric export for parity of the device precompute: mesh 0 = xy, 1 = y, 2 = x;
   what 0 = J, 1..3 = Qi, 4 = fJ^2 (xy only) */
void orc_metric(orc_ctx *c, int mesh, int what, double *out)
{
    const mesh_t *m = mesh == 0 ? &c->mxy : (mesh == 1 ? &c->my : (mesh == 2 ? &c->mx : &c->mo));
    size_t n = (size_t)NPAN * m->nx * m->ny;
    /* what: 0 J, 1-3 Q1-Q3, 4 f J^2 (xy) or f (o), 5-7 the unit position vector */
    const double *src = what == 0 ? m->J : what == 1 ? m->Q1 : what == 2 ? m->Q2 : what == 3 ? m->Q3
                      : what == 5 ? m->rx : what == 6 ? m->ry : what == 7 ? m->rz : (mesh == 3 ? c->fo : c->fJ2);
    memcpy(out, src, sizeof(double) * n);
}
void orc_sync_weights(orc_ctx *c, double *qb, double *qt, double *ql, double *qr)
{
    size_t n = (size_t)(c->N + 1) * sizeof(double);
    memcpy(qb, c->qb, n); memcpy(qt, c->qt, n); memcpy(ql, c->ql, n); memcpy(qr, c->qr, n);
}

/* Halo-map probe: exchange a packed field through one of the reference exchanges
   and return the halo ring of width w (NaN where no exchange wrote).
   kind 0: xy scalar hw=3 full; 1: xy vector hw=1 cross (f2 required);
   2: Ch vector hw=3 full (f = y-mesh field, f2 = x-mesh field).
   Output layout per field: [t][j = 1-w .. ny+w][i = 1-w .. nx+w]. */
static void ring_out(const fld_t *f, int w, double *out)
{
    size_t k = 0;
    for (int t = 0; t < NPAN; t++)
        for (int j = 1 - w; j <= f->ny + w; j++)
            for (int i = 1 - w; i <= f->nx + w; i++) out[k++] = FA(f, t, i, j);
}
void orc_halo_probe(orc_ctx *c, int kind, const double *f, const double *f2, int w, double *out, double *out2)
{
    if (kind == 0) {
        fld_t a; fld_init(&a, c->N + 1, c->N + 1, 5);
        fld_from_packed(&a, f);
        exch_do(&c->ex_xy3_full_s, &a, NULL);
        ring_out(&a, w, out); fld_free(&a);
    } else if (kind == 1) {
        fld_t a, b; fld_init(&a, c->N + 1, c->N + 1, 5); fld_init(&b, c->N + 1, c->N + 1, 5);
        fld_from_packed(&a, f); fld_from_packed(&b, f2);
        exch_do(&c->ex_xy1_cross_v, &a, &b);
        ring_out(&a, w, out); ring_out(&b, w, out2); fld_free(&a); fld_free(&b);
    } else {
        /* kind 2: Ch 'full' exchange of width 3; kind 4: Ch 'cross' exchange of width 1
           (the tendency exchange of vector_advection_Ch_mod.f90:56) */
        fld_t a, b; fld_init(&a, c->N, c->N + 1, 5); fld_init(&b, c->N + 1, c->N, 5);
        fld_from_packed(&a, f); fld_from_packed(&b, f2);
        exch_do(kind == 4 ? &c->ex_ch1c_u : &c->ex_ch3_u, &a, &b);
        exch_do(kind == 4 ? &c->ex_ch1c_v : &c->ex_ch3_v, &a, &b);
        ring_out(&a, w, out); ring_out(&b, w, out2); fld_free(&a); fld_free(&b);
    }
}

void orc_c_halo_probe(orc_ctx *c, int kind, const double *f, const double *f2, int w, double *out, double *out2)
{
    c_init(c);
    if (kind == 0) {
        fld_t a; fld_init(&a, c->N, c->N, 5);
        fld_from_packed(&a, f);
        exch_do(&c->ex_o3, &a, NULL);
        ring_out(&a, w, out); fld_free(&a);
    } else {
        fld_t a, b; fld_init(&a, c->N + 1, c->N, 5); fld_init(&b, c->N, c->N + 1, 5);
        fld_from_packed(&a, f); fld_from_packed(&b, f2);
        exch_do(&c->ex_c3_u, &a, &b);
        exch_do(&c->ex_c3_v, &a, &b);
        ring_out(&a, w, out); ring_out(&b, w, out2); fld_free(&a); fld_free(&b);
    }
}

/* One-dimensional SBP 4-2 operator on a single line, for pinning the
   coefficient tables: op 0 = i2c difference (in: n+1 nodes, out: n centres),
   1 = c2i difference (in: n centres, out: n+1 nodes, no SAT), 2 = i2c
   interpolation, 3 = c2i interpolation.  Halo inputs are taken as zero. */
void orc_sbp1d(int op, int n, const double *in, double *out);

/* The same probe for SBP order ord (21 or 42); the 2-1 stencils restate
   sbp_diff_i2c_21_mod.f90:33-41, sbp_diff_c2i_21_mod.f90:32-42,
   sbp_interp_i2c_21_mod.f90:25-31 and sbp_interp_c2i_21_mod.f90:25-35 (no SAT). */
void orc_sbp1d_ord(int ord, int op, int n, const double *in, double *out)
{
    if (ord == 63) {
        /* rows of the 6-3 operators on one line, zero halo, without SAT */
        const int nin = (op == 0 || op == 2) ? n + 1 : n;
        fld_t a, b;
        fld_init(&a, nin, 1, 5);
        fld_init(&b, (op == 0 || op == 2) ? n : n + 1, 1, 5);
        for (int t = 0; t < NPAN; t++)
            for (int i = -4; i <= nin + 5; i++) FA(&a, t, i, 1) = 0.0;
        for (int i = 1; i <= nin; i++) FA(&a, 0, i, 1) = in[i - 1];
        if (op == 0) {
            diff_i2c(&b, &a, 0, 0, n, 1, 1, 63);
            /* undo the SAT: the halo is zero, so row r carries 0.5 R_r/h_r f(1) */
            for (int r = 1; r <= 4; r++) {
                FA(&b, 0, r, 1) -= 0.5 * SBP63_R[r - 1] / SBP63_H_C[r - 1] * FA(&a, 0, 1, 1);
                FA(&b, 0, n + 1 - r, 1) -= 0.5 * SBP63_R[r - 1] / SBP63_H_C[r - 1] * (0.0 - FA(&a, 0, n + 1, 1));
            }
        } else if (op == 1) {
            diff_c2i(&b, &a, 0, 0, n + 1, 1, 1, 63);
            double s1 = 0.0, s2 = 0.0;
            for (int k = 1; k <= 4; k++) {
                s1 += SBP63_R[k - 1] * (FA(&a, 0, k, 1) - FA(&a, 0, 1 - k, 1));
                s2 += SBP63_R[k - 1] * (FA(&a, 0, n + k, 1) - FA(&a, 0, n + 1 - k, 1));
            }
            FA(&b, 0, 1, 1) -= 0.5 / SBP63_H_I[0] * s1;
            FA(&b, 0, n + 1, 1) -= 0.5 / SBP63_H_I[0] * s2;
        } else if (op == 2) {
            interp_i2c(&b, &a, 0, 0, n, 1, 1, 63);
        } else {
            interp_c2i(&b, &a, 0, 0, n + 1, 1, 1, 63);
        }
        const int nout = (op == 0 || op == 2) ? n : n + 1;
        for (int i = 1; i <= nout; i++) out[i - 1] = FA(&b, 0, i, 1);
        fld_free(&a);
        fld_free(&b);
        return;
    }
    if (ord != 21) { orc_sbp1d(op, n, in, out); return; }
#define X(k) in[(k) - 1]
    switch (op) {
    case 0: for (int k = 1; k <= n; k++) out[k - 1] = X(k + 1) - X(k); break;
    case 1:
        out[0] = X(2) - X(1);
        for (int k = 2; k <= n; k++) out[k - 1] = X(k) - X(k - 1);
        out[n] = X(n) - X(n - 1);
        break;
    case 2: for (int k = 1; k <= n; k++) out[k - 1] = 0.5 * (X(k + 1) + X(k)); break;
    default:
        out[0] = X(1);
        for (int k = 2; k <= n; k++) out[k - 1] = 0.5 * (X(k) + X(k - 1));
        out[n] = X(n);
        break;
    }
#undef X
}

void orc_sbp1d(int op, int n, const double *in, double *out)
{
    init_coeffs();
    int nin = (op == 0 || op == 2) ? n + 1 : n;
    fld_t a, b;
    fld_init(&a, nin, 1, 5);
    fld_init(&b, (op == 0 || op == 2) ? n : n + 1, 1, 5);
    for (int t = 0; t < NPAN; t++)
        for (int i = -4; i <= nin + 5; i++) FA(&a, t, i, 1) = 0.0;
    for (int i = 1; i <= nin; i++) FA(&a, 0, i, 1) = in[i - 1];
    switch (op) {
    case 0: {
        /* apply_tile only (no SAT) */
        int t = 0, dir = 0, l = 1;
        fld_t *o = &b;
        const fld_t *ii = &a;
#define O2(k) FA(o, t, k, l)
#define I2(k) FA(ii, t, k, l)
        O2(1) = DI_q11 * I2(1) + DI_q12 * I2(2) + DI_q13 * I2(3) + DI_q14 * I2(4);
        O2(2) = DI_q21 * I2(1) + DI_q22 * I2(2) + DI_q23 * I2(3) + DI_q24 * I2(4);
        O2(3) = DI_q31 * I2(1) + DI_q33 * I2(3) + DI_q34 * I2(4) + DI_q35 * I2(5);
        for (int k = 4; k <= n - 3; k++) O2(k) = (27.0 * (I2(k + 1) - I2(k)) - (I2(k + 2) - I2(k - 1))) / 24.0;
        O2(n - 2) = -DI_q31 * I2(n + 1) - DI_q33 * I2(n - 1) - DI_q34 * I2(n - 2) - DI_q35 * I2(n - 3);
        O2(n - 1) = -DI_q21 * I2(n + 1) - DI_q22 * I2(n) - DI_q23 * I2(n - 1) - DI_q24 * I2(n - 2);
        O2(n) = -DI_q11 * I2(n + 1) - DI_q12 * I2(n) - DI_q13 * I2(n - 1) - DI_q14 * I2(n - 2);
        (void)dir;
        break;
    }
    case 1: {
        int t = 0, l = 1, nx = n + 1;
        fld_t *o = &b;
        const fld_t *ii = &a;
        O2(1) = DC_q11 * I2(1) + DC_q12 * I2(2) + DC_q13 * I2(3);
        O2(2) = DC_q21 * I2(1) + DC_q22 * I2(2);
        O2(3) = DC_q31 * I2(1) + DC_q32 * I2(2) + DC_q33 * I2(3) + DC_q34 * I2(4);
        O2(4) = DC_q41 * I2(1) + DC_q42 * I2(2) + DC_q43 * I2(3) + DC_q44 * I2(4) + DC_q45 * I2(5);
        for (int k = 5; k <= nx - 4; k++) O2(k) = (27.0 * (I2(k) - I2(k - 1)) - (I2(k + 1) - I2(k - 2))) / 24.0;
        O2(nx - 3) = -DC_q41 * I2(nx - 1) - DC_q42 * I2(nx - 2) - DC_q43 * I2(nx - 3) - DC_q44 * I2(nx - 4) - DC_q45 * I2(nx - 5);
        O2(nx - 2) = -DC_q31 * I2(nx - 1) - DC_q32 * I2(nx - 2) - DC_q33 * I2(nx - 3) - DC_q34 * I2(nx - 4);
        O2(nx - 1) = -DC_q21 * I2(nx - 1) - DC_q22 * I2(nx - 2);
        O2(nx) = -DC_q11 * I2(nx - 1) - DC_q12 * I2(nx - 2) - DC_q13 * I2(nx - 3);
#undef O2
#undef I2
        break;
    }
    case 2: interp_i2c(&b, &a, 0, 0, n, 1, 1, 42); break;
    default: interp_c2i(&b, &a, 0, 0, n + 1, 1, 1, 42); break;
    }
    int nout = (op == 0 || op == 2) ? n : n + 1;
    for (int i = 1; i <= nout; i++) out[i - 1] = FA(&b, 0, i, 1);
    fld_free(&a);
    fld_free(&b);
}
