/*
 * chswe.h -- C ABI of the B200 shallow-water time step (ch_swe hot path).
 *
 * The entry points mirror the Fortran interfaces a GPU-backed subclass replaces
 * (paths relative to the ch_swe source tree):
 *
 *   swe_stvec_*        <- stvec_t / stvec_swm_t            src/stvec/stvec_mod.f90:10-30,
 *                                                            src/models/shallow_water/stvec/stvec_swm_mod.f90:10-42
 *   swe_stvec_create   <- create_stvec_swm                  src/models/shallow_water/stvec/stvec_swm_factory_mod.f90:15-36
 *   swe_stvec_assign   <- stvec_t%assign(s1, v1, s2, v2)    src/stvec/stvec_flexible_mod.f90:196-250
 *   swe_stvec_update   <- stvec_t%update(s1, v1, s2, v2)    src/stvec/stvec_flexible_mod.f90:252-306
 *   swe_ctx_create     <- create_domain + create_swm_operator("linear_swm_operator")
 *                                                            src/domain/domain_factory_mod.f90:55-147,
 *                                                            src/models/shallow_water/operator/operator_swm_factory_mod.f90:586-685
 *   swe_operator_apply <- operator_swm_lin_t%apply(vout, vin, domain)
 *                                                            src/models/shallow_water/operator/operator_swm_lin_mod.f90:66-108
 *   swe_rk4_step       <- rk4_t%step(v0, operator, domain, dt)   src/time_schemes/rk4_mod.f90:20-42
 *   swe_rk4_steps      <- nsteps x rk4_t%step (the driver loop  src/models/shallow_water/shallow_water_mod.f90:112-143)
 *   swe_integrals      <- quadrature_t%mass / %dot           src/quadrature/abstract_quadrature_mod.f90:29-64
 *
 * Conventions
 *  - Every function returns 0 on success and a negative SWE_E* code on failure;
 *    swe_last_error(ctx) gives the message.  The reference has no return codes:
 *    it calls parcomm_global%abort (src/parallel/parcomm_mod.f90:73-90); a
 *    Fortran shim maps a nonzero status to that call.
 *  - Host state arrays use the reference's per-panel Fortran layout p(i,j) with
 *    halos stripped, panels 1..6 outermost:
 *       h : (N+1) x (N+1) per panel  (xy mesh)
 *       u : N     x (N+1) per panel  (y mesh, i fastest: N values per row, N+1 rows)
 *       v : (N+1) x N     per panel  (x mesh, N+1 values per row, N rows)
 *    u, v are covariant wind components as in the reference ("covariant" v_components_type).
 *  - A context owns one CUDA stream (or the one given by swe_set_stream) and
 *    all device scratch; it is not thread-safe.  Calls are asynchronous on the
 *    stream except upload/download/integrals, which synchronise it.
 *  - A context holds n_members ensemble members of the same cube size; every
 *    operation acts on all members at once.
 */
#ifndef CHSWE_H
#define CHSWE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SWE_OK 0
#define SWE_EINVAL (-1)   /* bad argument or configuration */
#define SWE_ECUDA (-2)    /* CUDA runtime failure (message holds the CUDA error) */
#define SWE_ENOMEM (-3)   /* device allocation failed */
#define SWE_ENODEV (-4)   /* no usable CUDA device (the library has no CPU fallback) */
#define SWE_ETOOBIG (-5)  /* cube size above SWE_NOALLOC_MAX_N for swe_operator_apply_noalloc */

#define SWE_FP64 0
#define SWE_FP32 1

#define SWE_OP_LINEAR 0   /* operator_swm_lin_t, Ch staggering, SBP 4-2 */
#define SWE_OP_ADVECTIVE 1 /* operator_adv_swm_t, covariant Ch branch (massflux_ch_up4,
                              vector_advection_Ch_up4_cov; operator_adv_swm_mod.f90:62-96);
                              h is the full depth, h_mean is not used, no orography */

#define SWE_STAG_CH 0      /* horizontal_staggering 'Ch': h on vertices, u on y, v on x points */
#define SWE_STAG_AH 1      /* horizontal_staggering 'Ah': h, u, v on the vertices (linear operator) */
#define SWE_STAG_C 2       /* horizontal_staggering 'C': h on the cell centres, u on the x points, v on
                              the y points (domain_factory_mod.f90:281-295); the C-grid gradient,
                              divergence and co2contra only (swe_c_grad, swe_c_div,
                              swe_operator_contravariant): see swe_c_grad */

typedef struct swe_ctx swe_ctx;
typedef struct swe_stvec swe_stvec;

typedef struct swe_cfg {
    int N;                    /* cells per panel edge (>= 8) */
    int precision;            /* SWE_FP64 or SWE_FP32 (FP32 stencils, FP64 metric/reductions, Kahan state) */
    int n_members;            /* ensemble members held by the context (>= 1) */
    int operator_kind;        /* SWE_OP_LINEAR */
    double radius;            /* planet radius, metric%scale        (default 6371229 m) */
    double grav;              /* gravity                              (default 9.80616) */
    double omega;             /* rotation rate, metric%omega          (default 2 pi / 86164 s) */
    double rotation_axis[3];  /* metric%rotation_axis                 (default 0, 0, 1) */
    int coriolis_constant;    /* metric%coriolis_const: f = omega instead of 2 omega sin(lat) */
    double h_mean;            /* operator h_mean (H) for every member (default 1000 m) */
    int sbp_order;            /* SBP order of the Ch operators: 42 (default; 0 also selects it),
                                 21 or 63 (63 needs N >= 16), for both operators: the
                                 _sbp_sat_42 / _21 / _63 names of grad_factory_mod.f90,
                                 div_factory_mod.f90, co2contra_factory_mod.f90,
                                 coriolis_factory_mod.f90 and the SBP_C42/C21/C63 quadratures */
    int staggering;           /* SWE_STAG_CH (default) or SWE_STAG_AH: h, u, v all on the cell
                                 vertices, the linear operator with div_ah_sbp_proj_<order>,
                                 grad_ah_sbp_proj_<order>, coriolis_colocated, co2contra_colocated
                                 and SBP_Ah<order>_quadrature (gen_config_linear.sh:9-36), the
                                 order from sbp_order (42, 21 or 63).  Packed u and v are then
                                 (N+1) x (N+1) per panel like h.
                                 SWE_STAG_C: packed h is N x N per panel, u (N+1) x N (x points,
                                 N+1 values per row, N rows), v N x (N+1) (y points). */
} swe_cfg;

/* Fill *cfg with the defaults listed above. */
int swe_cfg_default(swe_cfg *cfg);

int swe_ctx_create(const swe_cfg *cfg, swe_ctx **ctx);
int swe_ctx_destroy(swe_ctx *ctx);
const char *swe_last_error(const swe_ctx *ctx);
/* Run the context's work on an existing CUDA stream (cudaStream_t); NULL restores the own stream. */
int swe_set_stream(swe_ctx *ctx, void *cuda_stream);
int swe_synchronize(swe_ctx *ctx);
/* Per-member mean depth H (ensembles with different h_mean). */
int swe_set_member_h_mean(swe_ctx *ctx, int member, double h_mean);
/* Orography of the advective operator (operator_adv_swm_t%h_surf, operator_adv_swm_mod.f90:37-38;
   filled by the test case's orography generator, operator_swm_factory_mod.f90:365-366):
   h_surf packed like h, (N+1) x (N+1) per panel, shared by all members; NULL removes it.
   The gradient then acts on h + h_surf (operator_adv_swm_mod.f90:78).  SWE_EINVAL on a
   linear-operator context (the linear operator has no orography in the reference). */
int swe_set_orography(swe_ctx *ctx, const double *h_surf);

int swe_stvec_create(swe_ctx *ctx, swe_stvec **vec);
int swe_stvec_destroy(swe_stvec *vec);
int swe_stvec_upload(swe_stvec *vec, int member, const double *h, const double *u, const double *v);
int swe_stvec_download(const swe_stvec *vec, int member, double *h, double *u, double *v);
/* Whole-batch transfers: arrays hold n_members consecutive member states. */
int swe_stvec_upload_all(swe_stvec *vec, const double *h, const double *u, const double *v);
int swe_stvec_download_all(const swe_stvec *vec, double *h, double *u, double *v);
/* y = s1*v1 + s2*v2 ; v2 may be NULL (then y = s1*v1). */
int swe_stvec_assign(swe_stvec *y, double s1, const swe_stvec *v1, double s2, const swe_stvec *v2);
/* y = y + s1*v1 + s2*v2 ; v2 may be NULL. */
int swe_stvec_update(swe_stvec *y, double s1, const swe_stvec *v1, double s2, const swe_stvec *v2);
/* Device storage of a state vector: element type (SWE_FP64/SWE_FP32), base pointer,
   bytes, and the row pitch of the layout [member][field h,u,v][panel][N+9 rows][pitch],
   point (i, j) (1-based) at row j+3, column i+3; the 4-point margins hold zeros. */
int swe_stvec_device_view(const swe_stvec *vec, void **ptr, size_t *bytes, int *precision, int *pitch);

/* vout = A(vin), A the linear shallow-water operator. */
int swe_operator_apply(swe_ctx *ctx, swe_stvec *vout, const swe_stvec *vin);
/* vout.u, vout.v = contravariant components (ut, vt) of vin's covariant wind; vout.h unchanged.
   Mirrors co2contra_operator_t%transform (co2contra_Ch_mod.f90:27-94). */
int swe_operator_contravariant(swe_ctx *ctx, swe_stvec *vout, const swe_stvec *vin);

/* C staggering (contexts created with SWE_STAG_C, SBP 4-2, FP32 or FP64):
   swe_c_grad: vout.u, vout.v = grad_c_sbp_sat_42 of vin.h (grad_operator_t%calc_grad,
     grad_factory_mod.f90:115-150 with sbp_diff_c2i_42; grad_sbp_sat_mod.f90:24-76): the
     centres->nodes difference with its SAT across the panel edges, divided by h a.
   swe_c_div: vout.h = div_c_sbp_sat_42 of the contravariant (vin.u, vin.v)
     (div_operator_t%calc_div, div_factory_mod.f90:112-156 with sbp_diff_i2c_42;
     div_sbp_sat_mod.f90:29-80, no projection).
   swe_operator_contravariant on a C context: co2contra_c_sbp42_new
     (co2contra_Cgrid_mod.f90, transform_co2contra_c_sbp_new).
   The reference's linear operator cannot run on the C staggering: it calls
   coriolis_op%calc_coriolis, and both C-grid Coriolis operators abort there
   (coriolis_Cgrid_mod.f90:28-37, coriolis_Cgrid_noncons_mod.f90:96-106).  So
   swe_operator_apply, the RK4 steps and the linear energy return SWE_EINVAL on a C
   context; these three operators are what the reference runs on C (its Helmholtz,
   Laplace and diffusion operators use them). */
int swe_c_grad(swe_ctx *ctx, swe_stvec *vout, const swe_stvec *vin);
int swe_c_div(swe_ctx *ctx, swe_stvec *vout, const swe_stvec *vin);
/* One classic RK4 step of size dt on v0 (in place). */
int swe_rk4_step(swe_ctx *ctx, swe_stvec *v0, double dt);
/* nsteps RK4 steps (captured into a CUDA graph after the first call with the same shape). */
int swe_rk4_steps(swe_ctx *ctx, swe_stvec *v0, double dt, int nsteps);
/* nsteps RK4 steps with a time step per member (dt[0..n_members-1]); a member with
   dt 0 is frozen: its state is left untouched and its blocks exit at once.  This is
   the step of continuous batching (one context = one pool of member slots).  No
   reference counterpart: the reference advances one state per timescheme%step
   (src/time_schemes/rk4_mod.f90:20-42). */
int swe_rk4_steps_members(swe_ctx *ctx, swe_stvec *v0, const double *dt, int nsteps);

/* Groups: the RK4 steps of up to 8 contexts -- cube sizes and member counts of their
   own, one device and precision, the linear operator on Ch in SBP 4-2, one split
   kernel configuration (17, 4, 0), (25, 3, 0) or (33, 2, 0) -- launched as one grid
   per kernel: twelve launches per RK4 step whatever the number of contexts, on the
   first context's stream, ordered after the work queued on every context's stream
   and before the work queued there later.  A context advanced in a group gets the
   bits it gets from swe_rk4_steps_members with the same configuration.  The group
   uses each context's scratch and per-member time-step buffer: a context takes no
   other calls while its group's steps may be in flight on another stream, and
   outlives its group.  No reference counterpart: the reference advances one state per
   timescheme%step (src/time_schemes/rk4_mod.f90:20-42). */
typedef struct swe_group swe_group;
int swe_group_create(swe_ctx *const *ctxs, int n, swe_group **out);
int swe_group_destroy(swe_group *g);
/* nsteps RK4 steps of states[k] (of context k) with the per-member time steps dt[k]
   (n_members values of context k; 0 freezes a member). */
int swe_group_rk4_steps_members(swe_group *g, swe_stvec *const *states, const double *const *dt, int nsteps);
int swe_group_synchronize(swe_group *g);
const char *swe_group_last_error(const swe_group *g);
long long swe_group_launch_count(const swe_group *g);
/* Horizontal diffusion of an Ah context (every member):
     swe_diffusion_apply <- operator_swm_diff_t%apply(vout, vin, domain)
                            src/models/shallow_water/operator/operator_swm_diff_mod.f90:27-49
     swe_diffusion_step  <- explicit_Eul1_t%step(v, operator_diff, domain, dt), the diffusion
                            step after each dynamics step (shallow_water_mod.f90:95-100,117-118;
                            src/time_schemes/explicit_Eul1_mod.f90:20-28): v += dt tendency
   with hordiff_vec_xyz_Ah_sbp_<lap_order>_narrow (coefficient uv_coeff) for u, v and
   hordiff_scalar_Ah_sbp_<lap_order>_narrow (h_coeff) for h
   (src/differential_operators/horizontal/hordiff/hordiff_factory_mod.f90:33-44,61-68):
   tendency -(coeff a hx)^4 L(L(f)) of h and of the wind's Cartesian components, L the
   narrow SBP Laplacian (src/differential_operators/horizontal/laplace/laplace_Ah_sbp{21,42,63}_narrow_mod.f90).
   lap_order 21, 42 (N >= 11) or 63 (N >= 17); other orders and non-Ah contexts return
   SWE_EINVAL.  vout != vin. */
int swe_diffusion_apply(swe_ctx *ctx, swe_stvec *vout, const swe_stvec *vin, int lap_order, double uv_coeff,
                        double h_coeff);
int swe_diffusion_step(swe_ctx *ctx, swe_stvec *v, double dt, int lap_order, double uv_coeff, double h_coeff);
/* The driver loop's diffusion inside the RK4 steps: after this call every RK4 step of
   swe_rk4_step / swe_rk4_steps / swe_rk4_steps_members is followed by swe_diffusion_step
   with the same dt (each member's own with swe_rk4_steps_members; frozen members stay),
   captured in the same CUDA graphs.  lap_order 0 turns it off. */
int swe_set_diffusion(swe_ctx *ctx, int lap_order, double uv_coeff, double h_coeff);
/* FP64 SBP-quadrature mass <h,1> and linear energy H/2(<u,ut>+<v,vt>) + g/2<h,h> of one member. */
int swe_integrals(swe_ctx *ctx, const swe_stvec *vec, int member, double *mass, double *energy);

/* Diagnostics of swm_output_diag_t for one member (print_CFL_diag and the extrema
   of print_integrals_diag, swm_output_diag_mod.f90:110-171): out[0..4] = h_min,
   h_max, the gravity-wave CFL sqrt(max (g / dx^2) h) dt and the advective CFL
   numbers sqrt(max |ut u| / dx^2) dt and sqrt(max |vt v| / dy^2) dt, with (ut, vt)
   the contravariant components and dx = dy = a (pi/2) / N.  Synchronous. */
int swe_diag(swe_ctx *ctx, const swe_stvec *vec, int member, double dt, double *out);

/* Energies and potential enstrophy of swm_output_diag_t%calc_energies for one member
   with covariant (u, v) (swm_output_diag_mod.f90:186-234, with the operators of the Ch
   diagnostics configuration: co2contra_ch_sbp*, curl_ch_sbp_sat_*, interp2d_p2uv_Ch_sbp*,
   interp2d_uv2qvec_Ch_sbp*, SBP_C*_quadrature; gen_config_linear.sh:53-63):
   out[0..3] = TE, KE, PE, enstrophy with
     KE = <hu ut u>_u / 2 + <hv vt v>_v / 2   (hu, hv: h interpolated to the u, v points)
     PE = g/2 <h h>_h                          (no orography)
     enstrophy = <(curl + f)^2 / (2 hq)>_q     (q: cell centres; hq: the mean of the two
                                               interpolations of hu, hv to the centres)
   in the context's SBP order, FP64 arithmetic.  Synchronous. */
int swe_energies(swe_ctx *ctx, const swe_stvec *vec, int member, double *out);

/* Curl of the covariant (u, v) of one member on the cell centres (curl_ch_sbp_sat_{21,42,63},
   curl_sbp_sat_mod.f90:27-76): out[6][N][N] in FP64, i fastest.  Synchronous. */
int swe_curl(swe_ctx *ctx, const swe_stvec *vec, int member, double *out);

/* Cubic lat-lon regrid of h (field 0, xy points) of one member, the values that
   latlon_outputer_t%write puts in a record (latlon_outputer_mod.f90:30-53,
   latlon_regrid_mod.f90:75-365, regrid_factory_mod.f90:25-70,165-276): h gets an
   ECS_xy halo of width 2, the points phi_j = -pi/2 + (j-1) pi / (nlat-1),
   lam_i = (i-1) 2 pi / nlon are located on their panels and the 4 x 4 cubic Lagrange
   stencil is summed.  out[nlat][nlon] in FP64, longitude fastest (the reference's
   outputer uses nlat = 2N+1, nlon = 4N).  field 1: the divergence of the wind instead
   (output_div's div.dat: div_ch_sbp_sat_<order>_proj of the contravariant wind,
   swm_output_diag_mod.f90:92-106; Ch only).  field 2: the curl of the covariant wind
   (output_curl's curl.dat, swm_output_diag_mod.f90:78-90; Ch only): curl_ch_sbp_sat_<order>
   on the cell centres, its ECS_O halo of width 2 (the o-point exchange, the rows of
   virtual cells interpolated along the neighbours' grid lines and the six special
   points of each cube corner: ecs_halo_mod.f90:74-477, ecs_halo_factory_mod.f90:26-68,
   190-230) and the cubic stencils on the cell-centre mesh (shift 1/2,
   regrid_factory_mod.f90:285-287).  Other fields give SWE_EINVAL.  Synchronous. */
int swe_regrid_latlon(swe_ctx *ctx, const swe_stvec *vec, int member, int field, int nlat, int nlon,
                      double *out);

/* Cubic lat-lon regrid of the covariant wind of one member (Ch), the values that
   latlon_vec_outputer_t%write puts in the u.dat / v.dat records
   (latlon_outputer_mod.f90:55-85, regrid_factory_mod.f90:72-163,
   latlon_regrid_mod.f90:132-212): u, v interpolated to the vertices
   (interp2d_uv2pvec_Ch_sbp42), the covariant ecs_xy_vec halo of width 2
   (ecs_halo_vec_xy_mod.f90:30-98), the cubic stencils and the rotation to the
   eastward / northward components.  u_out, v_out [nlat][nlon] in FP64, longitude
   fastest.  Synchronous. */
int swe_regrid_latlon_wind(swe_ctx *ctx, const swe_stvec *vec, int member, int nlat, int nlon, double *u_out,
                           double *v_out);

/* Number of kernel launches issued on the context's stream since creation. */
long long swe_launch_count(const swe_ctx *ctx);

/* Diagnostic: advance v0 by nreps RK4 steps launched kernel by kernel with CUDA
   events around each launch; returns the mean duration in ms of the
   contravariant-component kernel, the panel-edge kernel and the fused stage kernel. */
int swe_kernel_times(swe_ctx *ctx, swe_stvec *v0, double dt, int nreps, double *ms_co2contra, double *ms_edge,
                     double *ms_stage);

/* Tile size of the stage kernels: the maximal tile edge, 17, 25 or 33 points
   (ceil(N / (tile - 1)) balanced tiles per panel direction).  Contexts start at 25
   for N <= 96 and 33 above.  No reference counterpart: the reference's tiles are
   MPI partitions of the panels (src/parallel/partition_mod.f90:83-129). */
int swe_set_tile(swe_ctx *ctx, int tile);
int swe_get_tile(const swe_ctx *ctx, int *tile);
/* Kernel configuration: tile edge, the resident blocks per SM that the stage
   kernels' register allocation is capped for, and runs (1: each thread evaluates
   runs of several consecutive outputs along a stencil, 0: one output per element).
   Built (tile, blocks) pairs: (17, 3), (17, 4), (25, 2), (25, 3), (25, 4), (33, 2),
   (33, 3), each with runs 0 and 1; swe_set_tile picks (17, 3, 0), (25, 2, 0) or
   (33, 2, 0).  The advective operator's stage kernel always uses the tile's first
   blocks-per-SM value.  No reference counterpart. */
int swe_set_kernel_config(swe_ctx *ctx, int tile, int blocks_per_sm, int runs);
int swe_get_kernel_config(const swe_ctx *ctx, int *tile, int *blocks_per_sm, int *runs);
/* Autotuner: times nreps graph-replayed RK4 steps of a scratch state for each built
   kernel configuration, keeps the fastest on the context and returns its tile;
   ms_per_step (3 entries, may be NULL) receives the best time per step of tiles 17,
   25 and 33.  Results are cached for the process per (device, N, precision, members,
   operator).  The caller's states are not touched. */
int swe_autotune(swe_ctx *ctx, int nreps, int *best_tile, double *ms_per_step);

/* Largest cube size swe_operator_apply_noalloc accepts (its scratch is a static device
   array of about 1.5 MB that every GPU using the library holds until the process exits). */
#define SWE_NOALLOC_MAX_N 64

/* vout = A(vin) for callers that cannot allocate device memory -- a host model whose
   GPU memory belongs to another runtime or a fixed pool, or code that must not call
   cudaMalloc.  This entry point allocates nothing and needs no context: the caller
   passes device pointers to one FP64 state (input) and one FP64 state (output) in the
   layout swe_stvec_device_view describes (one member, pitch = (N + 9) rounded up to a
   multiple of 8, 4-point zero margins around every panel, margins of vin zero), and
   every intermediate lives in one static device array of this library.  It has no
   counterpart in the reference (there the operator owns allocatable work fields).
   Limits and behaviour:
   - cfg->N <= SWE_NOALLOC_MAX_N, else SWE_ETOOBIG (with a message on stderr);
     cfg->precision SWE_FP64, cfg->n_members 1, SWE_OP_LINEAR, SBP order 4-2.
   - The first call on a device, with that device current, looks up the array's
     device address and uploads the edge tables; make that first call before any
     stream capture.  A call with a new geometry (N, radius, gravity, rotation rate,
     rotation axis, Coriolis mode) rewrites the shared metric in the array, under any call still running on
     another stream: when the geometry changes, issue all calls on one stream or
     synchronise before the call with the new geometry.
   - Work runs asynchronously on cuda_stream (NULL: the legacy default stream).
   - All calls share the one array, which keeps the last call's contents; calls that
     overlap on the GPU (other streams, other host threads) race on it.  Not thread-safe. */
int swe_operator_apply_noalloc(const swe_cfg *cfg, const double *vin, double *vout, void *cuda_stream);

/* Panel-edge connectivity used by the device halo reads (host-only, no GPU needed):
   for panel p (0..5) and side s (0 left i=1, 1 right i=N+1, 2 bottom j=1, 3 top j=N+1)
   writes {neighbour panel, neighbour side, reversed along-edge order,
           normal-component sign, tangential-component sign} to out[(p*4+s)*5 + 0..4]. */
int swe_edge_links(int *out);

#ifdef __cplusplus
}
#endif

#endif
