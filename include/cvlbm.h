/*
 * cvlbm.h -- C ABI of libcvlbm.so, the sm_100a implementation of the
 * curved-boundary vectorial lattice Boltzmann (VLBM) time step.
 *
 * The reference (JingsenFeng/curved-boundary-vlbm, curved_lbm 1.0.0) exposes
 * this path only as two Python solver classes whose methods launch Warp
 * kernels; it has no plugin system and no C interface.  Every entry point
 * below replaces one of those methods; the citation in front of each names
 * the reference method (file:line inside the reference project) whose device
 * work it performs.  The Python drop-in package (curved_lbm.*) binds these
 * symbols with ctypes (curved_lbm/_native.py mirrors every struct below).
 *
 * Conventions
 *   - Every pointer inside a *_problem or *_fields struct is a device pointer
 *     (cudaMalloc / torch CUDA storage) unless stated otherwise.
 *   - All floating point is IEEE binary64; indices and flags are int32.
 *   - 2-D node arrays are dense [component][i][j] with j fastest
 *     (N = nx*ny nodes); 3-D node arrays are compacted active nodes
 *     [component][p] (N = n_active).
 *   - Functions return CVLBM_OK (0) or a negative error code; they never
 *     throw across the ABI.  cvlbm_last_error() returns a thread-local message.
 *   - `stream` is a cudaStream_t passed as void*; NULL is the legacy stream.
 *     All work is asynchronous on that stream.
 *   - Device-side failures (non-positive Jacobian) never trap: kernels set
 *     fields->invalid[0] to a nonzero value, as the reference's `invalid`
 *     flag does.
 */
#ifndef CVLBM_H
#define CVLBM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CVLBM_OK 0
#define CVLBM_ERR_INVALID_ARG (-1)
#define CVLBM_ERR_CUDA (-2)
#define CVLBM_ERR_UNSUPPORTED (-3)

/* Material ids (curved_lbm two_d/vector_nonlinear_elastic_warp.py:37-43,
 * three_d/vector_nonlinear_elastic_warp3d.py:34-40). */
#define CVLBM_MATERIAL_SVK 0
#define CVLBM_MATERIAL_NEO_HOOKE 1
#define CVLBM_MATERIAL_LOG_NEO_HOOKE 2
#define CVLBM_MATERIAL_MOONEY_RIVLIN 3
#define CVLBM_MATERIAL_YEOH 4
#define CVLBM_MATERIAL_GENT 5
#define CVLBM_MATERIAL_SUGIYAMA_SVK_2D 6 /* 2-D id 6 */
#define CVLBM_MATERIAL_SPH_NEO_HOOKE_3D 6 /* 3-D id 6 */

typedef struct cvlbm_material {
  int32_t model;
  int32_t reserved;
  double lam, mu, p0, p1, p2;
  double j_floor;
} cvlbm_material;

/* ------------------------------------------------------------------------ */
/* D2Q4x6                                                                    */
/* ------------------------------------------------------------------------ */

/* One cut link in processing order (see cvlbm2d_problem.link_rows): what the
 * link kernel reads first, in one 96-byte row. */
typedef struct cvlbm2d_link_row {
  int32_t ell;       /* link id (index of the per-link tables) */
  int32_t node;      /* i*ny + j */
  int32_t upstream;  /* node (i,j) - c_q when it is active, else -1 */
  int32_t q;         /* outgoing direction */
  int32_t bid;       /* boundary id, clamped to [0, 8) */
  int32_t lsq_valid;
  int32_t i, j;
  double eta, xb, yb, nx, ny;
  double reserved[3];
} cvlbm2d_link_row;

/* Static description of one 2-D problem: lattice, material, boundary tables
 * and cut-link geometry.  Mirrors the constructor state of
 * WarpCurvedBoundaryLBM2D (two_d/curved_boundary_warp.py:3621-3843). */
typedef struct cvlbm2d_problem {
  int32_t nx, ny;
  int32_t n_links;
  int32_t recon;         /* reconstruction id, two_d numbering (0 bfl, 2 lsq_bfl,
                            9 compat_bfl, 11 local_char2, 12 local_f, 13 local_f_bfl) */
  int32_t normal_solver; /* 0 finite-difference Newton, 1 acoustic Newton, 2 energy */
  int32_t source_mode;   /* 0 none, 1 constant, 2 damping */
  double dx, dy, dt, omega, c;
  double source[6];
  cvlbm_material mat;
  int32_t disp_interval;   /* local displacement sweep every N steps (0 = off) */
  int32_t disp_sweeps;     /* sweeps per due step, 1..8 */
  int32_t disp_bid;        /* anchor boundary id, <0: all Dirichlet ids */
  int32_t rep_interval;    /* local F repair every N steps (0 = off) */
  int32_t interior_only;   /* repair only nodes with four active neighbours */
  int32_t use_dynamic_traction;
  double relax, weight, blend;
  /* geometry, all device pointers */
  const int32_t *active;                      /* [nx*ny] 0/1 */
  const int32_t *link_i, *link_j, *link_q, *link_bid;
  const double *link_eta, *link_xb, *link_yb, *link_nx, *link_ny;
  const int32_t *lsq_i, *lsq_j;               /* [n_links*24] */
  const double *lsq_wb, *lsq_wt, *lsq_wx, *lsq_wy;
  const int32_t *lsq_valid;                   /* [n_links] */
  const int32_t *node_link_start;             /* [nx*ny+1] CSR of links per node */
  const int32_t *node_link_list;              /* [n_links], ascending within a node */
  const int32_t *bc_kind, *bc_mode;           /* [8] per boundary id */
  const double *bc_params;                    /* [8*8] */
  const double *traction_x, *traction_y;      /* [n_links] dynamic traction */
  /* fused step (optional; all four set enables it when disp_sweeps <= 1) */
  const int32_t *tiles;                       /* [n_tiles] ids of tile_i x 32 tiles with active nodes */
  int32_t n_tiles, tiles_j;                   /* tile count, tiles along j */
  const uint8_t *need_fields;                 /* [nx*ny] node read by some link stencil */
  const int32_t *link_partner;                /* [n_links] link at the same node in the
                                                 incoming direction, or -1 */
  const int32_t *lsq_node;                    /* [n_links*24] lsq_i*ny+lsq_j, -1 unused */
  const int32_t *link_order;                  /* [n_links] processing order (optional) */
  int32_t tile_variant;                       /* compiled fused-kernel variant, see
                                                 cvlbm2d_tile_variant() */
  int32_t tile_i;                             /* tile rows the tile list was built for */
  int32_t n_tiles_inner;                      /* the first n_tiles_inner entries of `tiles`
                                                 are inner tiles: no cut-link node within
                                                 the tile's 3-node halo and no link-stencil
                                                 node in the tile; the rest are boundary
                                                 tiles (0: not classified) */
  int32_t overlap;                            /* nonzero: the next step's inner tiles run on
                                                 a second stream while the link kernel runs */
  /* cut links in processing order (optional): one row per slot, and the
     LSQ stencil node ids and weights in slot order, so that the link kernel
     starts its stencil gathers after one level of loads */
  const cvlbm2d_link_row *link_rows;          /* [n_links] */
  const int32_t *lsq_node_slot;               /* [n_links*24] */
  const double *lsq_wb_slot, *lsq_wt_slot, *lsq_wx_slot, *lsq_wy_slot;
  /* collision options (two_d/curved_boundary_warp.py:3629-3631); either one
     selects the per-phase kernels */
  int32_t collision_model;                    /* 0 bgk, 1 mrt_ghost (:1846-2040) */
  double ghost_omega;                         /* relaxation of the D2Q4 ghost moment */
  double kinetic_filter;                      /* ghost filter strength in [0, 1]
                                                 (:3101-3124), applied after each step */
} cvlbm2d_problem;

/* Tile rows (i extent, tiles are 32 nodes wide in j) of fused-kernel variant
 * v, or 0 if v is not compiled.  Used by autotuners to enumerate variants. */
int cvlbm2d_tile_variant(int32_t v);

/* Mutable state.  f0 is the current population field; a run swaps f0 and f1
 * once per step and writes the swapped pointers back. */
typedef struct cvlbm2d_fields {
  double *f0, *f1, *fpost;  /* [24*N] */
  double *U;                /* [6*N]  v_x v_y F11 F12 F21 F22 */
  double *u, *u_next;       /* [2*N]  displacement, sweep scratch */
  double *u_star;           /* [2*N]  trapezoidal half-step displacement */
  double *P, *sigma;        /* [4*N]  first Piola and Cauchy stress */
  int32_t *invalid;         /* [1]    sticky flag, reset at the start of a run */
  double *clock;            /* [2]    device time (ping-pong); graph_mode != 0 */
  double *link_scratch;     /* [6*n_links] fused step: post-collision populations
                               leaving through each cut link */
} cvlbm2d_fields;

/* Advance `nsteps` time steps starting at host time `time0` and step index
 * `step0` (used for the displacement/repair interval test).  Replaces
 * WarpCurvedBoundaryLBM2D.step (two_d/curved_boundary_warp.py:4163-4258)
 * called nsteps times.  With graph_mode != 0 the kernels read the time from
 * fields->clock and advance it, so the launch sequence can be captured in a
 * CUDA graph and replayed; nsteps must then be even. */
int cvlbm2d_run(const cvlbm2d_problem *p, cvlbm2d_fields *f, double time0, int64_t step0,
                int32_t nsteps, int32_t graph_mode, void *stream);

/* Same step as cvlbm2d_run (graph_mode 0) without any allocation and without
 * a caller-owned link scratch: fields->link_scratch is ignored and the
 * per-link scratch is a fixed array inside the library, one per device, for
 * at most CVLBM2D_STATIC_SCRATCH_MAX_LINKS cut links (768 KiB).  Problems
 * with more cut links are rejected with CVLBM_ERR_INVALID_ARG.  The fields
 * must live on the current device.  The first call on a device looks up the
 * array's address (cudaGetSymbolAddress); make that call before any stream
 * capture begins.  Calls in flight at the same time on one device share the
 * array and race; serialise them.  For hosts that cannot allocate device
 * memory between steps.  No counterpart in the reference. */
#define CVLBM2D_STATIC_SCRATCH_MAX_LINKS 16384
int cvlbm2d_run_static_scratch(const cvlbm2d_problem *p, cvlbm2d_fields *f, double time0,
                               int64_t step0, int32_t nsteps, void *stream);

/* Kinetic ghost filter (problem->kinetic_filter) applied in place to
 * fields->f0, as initialize_from_numpy does after its in-place boundary pass
 * (two_d/curved_boundary_warp.py:3947-3952; kernel :3101-3124).  A run
 * applies it after every step by itself. */
int cvlbm2d_kinetic_filter(const cvlbm2d_problem *p, cvlbm2d_fields *f, void *stream);

/* Initial populations of initialize_from_numpy, computed on the device
 * instead of by the reference's host NumPy (two_d/curved_boundary_warp.py:
 * 3855-3900 calling two_d/vector_nonlinear_elastic_warp.py:595-847): order 1
 * feq(U) - (dt/8) B(U); order 2 the second-order start from centred
 * differences of U; order 3 the same from active neighbours only.  U: device
 * [6][nx*ny], full lattice; f0: device [24][nx*ny] out, zero at inactive
 * nodes; work: device scratch of cvlbm2d_init_work_bytes(nx, ny) bytes.
 * *status (device int32) is set to 1 where the reference's host code raises
 * FloatingPointError (J <= 0 or the Gent chain limit in some flux
 * evaluation; the host code then retries with a smaller difference step) or
 * where the kernels' Jacobian floor would change a value: f0 is then not
 * the reference's and the caller repeats the host computation. */
int cvlbm2d_init_populations(const cvlbm2d_problem *p, const double *U, int32_t order,
                             double *f0, void *work, int32_t *status, void *stream);
int64_t cvlbm2d_init_work_bytes(int32_t nx, int32_t ny);

/* Field reductions of summary() (two_d/curved_boundary_warp.py:4343-4415 and
 * the 3-D class's summary) over the active nodes, from the refreshed fields:
 * out (host, 6 doubles) = max |u|, max |v|, min J, max J, finite (1/0: every
 * value finite - u and U in 2-D, U in 3-D - and J > 0), node count.  dim 2:
 * U [6][n], u [2][n], active [n] (0/1; null = all); dim 3: U [12][n], u [3][n]
 * (sparse active order, active null).  Each node's |u|, |v| and J are formed
 * with the reference's NumPy expressions; NaN propagates like NumPy's
 * max/min.  work: device scratch of cvlbm_field_summary_work_bytes() bytes.
 * Synchronises `stream`. */
int cvlbm_field_summary(int32_t dim, int64_t n, const double *U, const double *u,
                        const int32_t *active, void *work, double *out, void *stream);
int64_t cvlbm_field_summary_work_bytes(void);

/* Cut-link reconstruction at time t, fpost -> f1, or in place on f0 through a
 * frozen copy in fpost.  Replaces apply_boundary_reconstruction
 * (two_d/curved_boundary_warp.py:4020-4035). */
int cvlbm2d_apply_boundary(const cvlbm2d_problem *p, cvlbm2d_fields *f, double t,
                           int32_t in_place, void *stream);

/* Recompute U, u, P, sigma from f0 and u_star and reset `invalid`.
 * Replaces refresh_current (two_d/curved_boundary_warp.py:4260-4291). */
int cvlbm2d_refresh(const cvlbm2d_problem *p, cvlbm2d_fields *f, void *stream);

/* ------------------------------------------------------------------------ */
/* Batched D2Q4x6: many independent problems advanced together               */
/* ------------------------------------------------------------------------ */

/* A batch of independent 2-D problems (different geometries, load cases and
 * lattice sizes) stepped together: per lattice step one persistent node
 * launch walks the (instance, tile) work list of every instance, one
 * persistent link launch walks all instances' cut links, and a tick advances
 * each instance's device clock and step index.  Instances retire
 * individually when their residual |u - u_prev|_2 / (check_every |u|_2) over
 * active nodes (the relative displacement change per step since the previous
 * check) falls below a tolerance, or when their state becomes invalid
 * (non-positive Jacobian).  The reference runs one solver per geometry
 * (two_d/curved_boundary_warp.py:4163-4258 per instance); batching, the
 * residual criterion and early retirement have no counterpart there. */
typedef struct cvlbm2d_batch cvlbm2d_batch;

/* problems[i]/fields[i] describe instance i exactly as for cvlbm2d_run, with
 * the fused-step tables (tiles, need_fields, link_partner, lsq_node,
 * link_scratch) built for `tile_variant`; step0[i]/time0[i] are its step
 * index and time.  The batch keeps the field pointers: fields->f0 and
 * fields->u_star hold the state when the instance has taken an even number of
 * batch steps, f1 and u_next when odd (cvlbm2d_batch_status reports steps).
 * grid_blocks = 0 sizes the persistent node grid to the SMs' resident
 * capacity.  Allocates the work lists and a previous-displacement buffer
 * (2 doubles per lattice node) on the device. */
int cvlbm2d_batch_create(int32_t n_inst, const cvlbm2d_problem *problems,
                         const cvlbm2d_fields *fields, const int64_t *step0,
                         const double *time0, int32_t tile_variant, int32_t grid_blocks,
                         cvlbm2d_batch **out);

/* Advance every active instance by up to nsteps lattice steps; after every
 * check_every-th step, retire instances with time >= t_min and residual < tol
 * (check_every = 0: no checks).  Asynchronous on `stream`. */
int cvlbm2d_batch_run(cvlbm2d_batch *b, int32_t nsteps, int32_t check_every, double tol,
                      double t_min, void *stream);

/* cvlbm2d_batch_run captured into a replayable CUDA graph. */
int cvlbm2d_batch_graph_create(cvlbm2d_batch *b, int32_t nsteps, int32_t check_every,
                               double tol, double t_min, struct cvlbm_graph **out);

/* Per-instance state (any pointer may be NULL): active flag, status (0
 * running, 1 converged, -1 invalid), step index, time, last residual (-1
 * before the second check).  Synchronises `stream`. */
int cvlbm2d_batch_status(cvlbm2d_batch *b, int32_t *active, int32_t *status, int64_t *steps,
                         double *time, double *residual, void *stream);

/* Persistent node grid size and number of (instance, tile) work items. */
int cvlbm2d_batch_launch_grid(const cvlbm2d_batch *b, int32_t *node_grid, int32_t *n_work);

void cvlbm2d_batch_destroy(cvlbm2d_batch *b);

/* First Piola stress and Cauchy stress of the current U buffer at active
 * nodes (inactive nodes untouched).  The reference stores P and sigma in its
 * collision and repair kernels (two_d/curved_boundary_warp.py:1795-1803,
 * 3603-3615); this library evaluates them on demand from the same U. */
int cvlbm2d_stress(const cvlbm2d_problem *p, cvlbm2d_fields *f, void *stream);

/* ------------------------------------------------------------------------ */
/* D3Q6x12 (compacted active nodes)                                          */
/* ------------------------------------------------------------------------ */

/* Mirrors the constructor state of WarpSparseCurvedBoundaryLBM3D
 * (three_d/curved_boundary_warp3d.py:3859-4071). */
typedef struct cvlbm3d_problem {
  int32_t n_active, n_links;
  int32_t nx, ny, nz;
  int32_t recon;         /* three_d numbering: 0 bfl, 1 halfway, 2 compat_bfl,
                            3 local_f, 4 local_f_bfl */
  int32_t normal_solver; /* 0 finite-difference Newton, 1 acoustic Newton, 2 energy */
  int32_t source_mode;
  int32_t has_char;      /* characteristic stencil present (local_f + Neumann) */
  int32_t has_tangent_lsq;
  int32_t disp_interval, disp_sweeps, disp_bid, rep_interval;
  double dx, dy, dz, dt, omega, c;
  double source[12];
  cvlbm_material mat;
  double relax, weight, blend;
  const int32_t *active_i, *active_j, *active_k; /* [n_active] */
  const int32_t *neighbor;                        /* [6*n_active], -1 = none */
  const int32_t *link_p, *link_up, *link_q, *link_bid;
  const double *link_eta, *link_xb, *link_yb, *link_zb, *link_nx, *link_ny, *link_nz;
  const int32_t *lsq_p;                           /* [n_links*32] */
  const double *lsq_wt1, *lsq_wt2;
  const int32_t *lsq_valid;
  const int32_t *char_idx;                        /* [64*n_links] */
  const double *char_w;                           /* [4*64*n_links] */
  const int32_t *node_link_start, *node_link_list;/* CSR of links per active node */
  const int32_t *bc_kind, *bc_mode;               /* [16] */
  const int32_t *bc_comp_kind;                    /* [3*16] */
  const double *bc_params;                        /* [16*16] */
  const int32_t *dyn_enabled;                     /* [n_links] */
  const double *dyn_traction;                     /* [3*n_links] */
  /* fused step (optional; need_slot, link_partner and fields->link_scratch,
     fields->U_need all set enable it when disp_sweeps <= 1) */
  const int32_t *need_slot;                       /* [n_active] row of U_need holding the
                                                     node's post-step U, or -1 */
  int32_t n_need;                                 /* rows of U_need */
  int32_t node_variant;                           /* fused collide kernel: 0 one thread per
                                                     node within 128 registers, 1 six warps
                                                     per 32 nodes (shared memory), 2 one
                                                     thread per node within 168 registers,
                                                     3 / 4 the wavefront form (wave_*
                                                     tables) within 128 / 168 registers;
                                                     results are identical */
  const int32_t *char_slot;                       /* [64*n_links] char_idx mapped to
                                                     U_need rows (-1 unused) */
  const int32_t *link_partner;                    /* [n_links] link at the same node in the
                                                     incoming direction, or -1 */
  const int32_t *link_order;                      /* [n_links] processing order of the
                                                     one-thread-per-link kernels (optional) */
  const int32_t *link_nodes;                      /* [n_link_nodes] ascending active ids of
                                                     the nodes that hold a cut link */
  int32_t n_link_nodes;
  int32_t overlap;                                /* nonzero (fused step, a sweep every
                                                     step): the next step's moments of the
                                                     nodes without a cut link run on a
                                                     second stream while the link kernels
                                                     run (measured slower on shell192: the
                                                     link kernels are throughput-bound) */
  /* wavefront form of the fused node work (node_variant 3): moments, sweep
     and collide of x-plane chunks in one persistent launch, taken in
     dependency order from a ticket counter (needs fields->wave_sync) */
  const int32_t *wave_items;                      /* [4*n_wave_items] stage (0 moments,
                                                     1 sweep, 2 collide), x-plane, first and
                                                     end active id; ticket order */
  int32_t n_wave_items;
  int32_t n_planes;                               /* x-planes (nx) */
  const int32_t *wave_plane_chunks;               /* [n_planes] items of one stage per plane */
  /* link-major copies of the characteristic tables (optional; both set
     select the 4-lanes-per-link gather, which reads a sample's slot and its
     four weights as one 4-byte and two 16-byte loads) */
  const int32_t *char_slot_lm;                    /* [n_links][64] = char_slot transposed */
  const double *char_w_lm;                        /* [n_links][64][4]: char_w[k][m][l] at
                                                     [l][m][k] */
} cvlbm3d_problem;

typedef struct cvlbm3d_fields {
  double *f0, *f1;          /* [72*N]; f0 is collided in place */
  double *U;                /* [12*N] */
  double *u, *u_next, *u_star; /* [3*N] */
  int32_t *link_kind, *link_comp_kind; /* [n_links], [3*n_links] */
  double *link_bv;          /* [3*n_links] */
  double *link_Fb, *link_Pb;/* [9*n_links] */
  double *char_state;       /* [4*12*n_links] value, d/dx, d/dy, d/dz */
  int32_t *invalid;
  double *clock;
  double *link_scratch;     /* [12*n_links] fused step: post-collision populations
                               leaving through each cut link */
  double *U_need;           /* [n_need*12] fused step: post-step U of the nodes cut
                               links read, one 96-byte row per node */
  int32_t *wave_sync;       /* [2 + 3*n_planes] node_variant 3: ticket, wait-timeout
                               flag and per-plane completion counters, zeroed by every
                               step (a timed-out wait also sets invalid) */
} cvlbm3d_fields;

/* Replaces WarpSparseCurvedBoundaryLBM3D.step
 * (three_d/curved_boundary_warp3d.py:4549-4589) called nsteps times. */
int cvlbm3d_run(const cvlbm3d_problem *p, cvlbm3d_fields *f, double time0, int64_t step0,
                int32_t nsteps, int32_t graph_mode, void *stream);

/* Replaces apply_boundary_reconstruction (three_d/curved_boundary_warp3d.py:4339-4399):
 * link preparation (gather, Newton, Piola), BFL rows and characteristic rows. */
int cvlbm3d_apply_boundary(const cvlbm3d_problem *p, cvlbm3d_fields *f, double t,
                           int32_t in_place, void *stream);

/* Replaces refresh_current (three_d/curved_boundary_warp3d.py:4401-4424). */
int cvlbm3d_refresh(const cvlbm3d_problem *p, cvlbm3d_fields *f, void *stream);

/* Replaces the _sparse_set_ustar launch of _initialize_from_active
 * (three_d/curved_boundary_warp3d.py:2096-2106, 4270-4277):
 * u_star = displacement - dt/2 * v. */
int cvlbm3d_set_ustar(const cvlbm3d_problem *p, cvlbm3d_fields *f, const double *displacement,
                      void *stream);

/* ------------------------------------------------------------------------ */
/* 3-D geometry preprocessing on the device                                  */
/* ------------------------------------------------------------------------ */

/* Geometry of the cut links whose characteristic stencil is built.  All
 * pointers are device pointers; active_id is the dense [nx][ny][nz] map from
 * lattice node to active id (-1: not active).  Cut points (link_xb/yb/zb)
 * are physical coordinates of a lattice with cell-centred nodes
 * ((i + 1/2) dx) and isotropic spacing dx. */
typedef struct {
  int32_t nx, ny, nz, n_links;
  double dx;
  const int32_t *active_id;
  const int32_t *link_i, *link_j, *link_k, *link_q;
  const double *link_eta, *link_xb, *link_yb, *link_zb, *link_nx, *link_ny, *link_nz;
  const uint8_t *link_mask; /* [n_links]: nonzero = build this link; NULL = all */
} cvlbm3d_stencil_input;

/* Fixed geometry weights of the D3Q6 local_f characteristic closure for every
 * selected cut link.  Replaces build_characteristic_weights
 * (three_d/characteristic_stencil3d.py:18-171).  Outputs (device, caller
 * owned): indices [64][n_links] int32 (48 gradient samples, then 16 probe
 * samples; -1 unused), weights [4][64][n_links] (row 0 probe weights, rows
 * 1-3 the x/y/z gradient weights), modes [n_links] (2 probe pair, 1 single
 * probe, -k k upstream nodes, 0 not built) and status [n_links] (0 ok, 1 no
 * full-rank quadratic fit within three cells, 2 inconsistent gradient
 * weights: the reference raises ValueError for both).  Asynchronous on
 * `stream`. */
int cvlbm3d_build_char_stencil(const cvlbm3d_stencil_input *in, int32_t *indices, double *weights,
                               int32_t *modes, int32_t *status, void *stream);

/* ------------------------------------------------------------------------ */
/* Kernel timing                                                             */
/* ------------------------------------------------------------------------ */

/* A ring of CUDA-event pairs.  A run given a timer brackets the dominant
 * kernel of every step (the bulk node kernel) with the next free pair, on
 * the launch stream; inside a captured graph the pairs become event nodes
 * and are re-recorded by every replay.  No counterpart in the reference,
 * which has no profiling hooks. */
typedef struct cvlbm_timer cvlbm_timer;
int cvlbm_timer_create(int32_t capacity, cvlbm_timer **out);
void cvlbm_timer_destroy(cvlbm_timer *t);
/* Forget recorded pairs (next run starts at pair 0). */
int cvlbm_timer_reset(cvlbm_timer *t);
/* Wait for the recorded pairs and return their summed duration and count. */
int cvlbm_timer_elapsed(cvlbm_timer *t, double *total_ms, int32_t *count);
/* Attach (or detach with NULL) the timer used by subsequent runs/captures
 * on this thread. */
int cvlbm_timer_attach(cvlbm_timer *t);
/* Attach (or with NULL detach) a timer to the cut-link kernel of the 2-D
 * step, the same way: one event pair per launch of the link kernel. */
int cvlbm_timer_attach_links(cvlbm_timer *t);

/* Number of kernel launches this library has issued (host-side counter;
 * launches replayed from a CUDA graph are counted once, at capture). */
int64_t cvlbm_launch_count(void);

/* ------------------------------------------------------------------------ */
/* CUDA graphs of whole step sequences                                       */
/* ------------------------------------------------------------------------ */

typedef struct cvlbm_graph cvlbm_graph;

/* Capture `nsteps` (even) steps of cvlbm2d_run / cvlbm3d_run in graph mode
 * into an executable CUDA graph.  The graph keeps the field pointers it was
 * captured with; it is valid for replays whose starting step index has the
 * same phase modulo the displacement and repair intervals. */
int cvlbm2d_graph_create(const cvlbm2d_problem *p, const cvlbm2d_fields *f, int64_t step0,
                         int32_t nsteps, cvlbm_graph **out);
int cvlbm3d_graph_create(const cvlbm3d_problem *p, const cvlbm3d_fields *f, int64_t step0,
                         int32_t nsteps, cvlbm_graph **out);
int cvlbm_graph_launch(cvlbm_graph *g, void *stream);
void cvlbm_graph_destroy(cvlbm_graph *g);

/* ------------------------------------------------------------------------ */
/* BF16 tensor-core GEMM of the warm-start surrogate                         */
/* ------------------------------------------------------------------------ */

/* C[M x N] (fp32, row-major, ldc) = A[M x K] . B[N x K]^T, plus the old C when
 * accumulate != 0.  A and B are bf16 (uint16 storage), K-major, 16-byte
 * aligned; M % 128 == 0, N % 64 == 0, K % 64 == 0, lda and ldb multiples of 8.
 * sm_100a tcgen05.mma with fp32 accumulation in tensor memory.  A device
 * workspace of cvlbm_gemm_bf16_workspace() bytes (may be NULL / smaller)
 * lets long-K, few-tile products split K over more CTAs (fp32 partials summed
 * in a fixed order).  `error` is a device int32 set to 1 if a CTA's MMAs did
 * not complete in time (bounded wait; that CTA's tile is then not written).
 * No counterpart in the reference, which has no learned components. */
int cvlbm_gemm_bf16(const void *A, const void *B, float *C, int32_t M, int32_t N, int32_t K,
                    int32_t lda, int32_t ldb, int32_t ldc, int32_t accumulate, int32_t *error,
                    void *workspace, int64_t workspace_bytes, void *stream);
int64_t cvlbm_gemm_bf16_workspace(int32_t M, int32_t N, int32_t K);

/* ------------------------------------------------------------------------ */
/* Warm-start surrogate (Fourier neural operator): CUDA-core kernels          */
/* ------------------------------------------------------------------------ */
/* Activations are channel-major per sample, x[b][c][g] (g = lattice node);
 * spectral coefficients a[b][c][k] (k = retained real Fourier mode); weights
 * W[o][i], R[k][i][o].  All fp32 except the bf16 operands of
 * cvlbm_gemm_bf16.  At most 32 channels.  No counterpart in the reference. */

/* z = W x + bias (+ s), y = gelu(z) if act (z may be NULL). */
int cvlbm_fno_pointwise_fwd(int32_t B, int32_t G, int32_t Cin, int32_t Cout, const float *x,
                            const float *W, const float *bias, const float *s, int32_t act,
                            float *z, float *y, void *stream);
/* dz = dy * gelu'(z) over n elements. */
int cvlbm_fno_gelu_bwd(int64_t n, const float *z, const float *dy, float *dz, void *stream);
/* dx (+)= W^T dz (dx may be NULL); dW = sum dz x^T, db = sum dz over samples and
 * nodes (deterministic order).  scratch: cvlbm_fno_pointwise_scratch() floats. */
int cvlbm_fno_pointwise_bwd(int32_t B, int32_t G, int32_t Cin, int32_t Cout, const float *dz,
                            const float *x, const float *W, float *dx, int32_t accumulate_dx,
                            float *dW, float *db, float *scratch, void *stream);
int64_t cvlbm_fno_pointwise_scratch(int32_t B, int32_t G, int32_t Cin, int32_t Cout);
/* bh[b][o][k] = sum_i a[b][i][k] R[k][i][o], stored as bf16. */
int cvlbm_fno_spec_mix_fwd(int32_t B, int32_t C, int32_t M, const float *a, const float *R,
                           void *bh_bf16, void *stream);
/* da = R dbh (bf16 out) and dR[k][i][o] = sum_b a[b][i][k] dbh[b][o][k]. */
int cvlbm_fno_spec_mix_bwd(int32_t B, int32_t C, int32_t M, const float *a, const float *dbh,
                           const float *R, void *da_bf16, float *dR, void *stream);
int cvlbm_fno_to_bf16(int64_t n, const float *src, void *dst, void *stream);
/* masked weighted MSE: part[p] (n_parts blocks) sum to the loss; dy its gradient. */
int cvlbm_fno_mse(int32_t B, int32_t C, int32_t G, const float *y, const float *t,
                  const float *mask, const float *w, float inv_count, float *dy, float *part,
                  int32_t n_parts, void *stream);
/* Adam step, bias correction folded into lr. */
int cvlbm_fno_adam(int64_t n, float *p, const float *g, float *m, float *v, float lr, float b1,
                   float b2, float eps, void *stream);

/* sizeof of the ABI structs as this library was compiled: which = 0
 * cvlbm2d_problem, 1 cvlbm2d_fields, 2 cvlbm3d_problem, 3 cvlbm3d_fields,
 * 4 cvlbm3d_stencil_input; -1 for anything else.  Bindings compare it with their own layout. */
int64_t cvlbm_struct_size(int32_t which);

/* Library version (major*10000 + minor*100 + patch) and last error text. */
int cvlbm_version(void);
const char *cvlbm_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* CVLBM_H */
