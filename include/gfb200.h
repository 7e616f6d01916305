/*
 * gfb200.h -- C ABI of the B200 (sm_100a) FLIP/PIC/APIC substep library.
 *
 * Every entry point replaces one stage of the reference's per-substep pipeline
 * FlipSolver3D._step_impl (src/gpufluid/solvers/solver3d.py:3475-3667); the
 * citation beside each declaration names the reference kernel(s) it stands in
 * for.  The Python host (gpufluid_b200.solver.FlipSolver3D) binds these with
 * ctypes; a C or C++ host can call them directly.
 *
 * Conventions
 *  - Plain pointers and sizes only.  Device buffers passed in gf_fields /
 *    gf_particles are owned by the caller; the library never frees them.
 *    The library allocates its own scratch (binning arrays, sorted particle
 *    records, pressure workspace) inside gf_create / gf_reserve_particles.
 *  - Layout is the reference's: C order [i][j][k] (k fastest);
 *    u (nx+1,ny,nz), v (nx,ny+1,nz), w (nx,ny,nz+1), cell arrays (nx,ny,nz);
 *    labels are uint8 (0 air, 1 fluid, 2 solid); particles are (n,3) float32
 *    AoS, the APIC matrix (n,3,3) float32 row-major.
 *  - Every call returns a gf_status; on failure gf_last_error() describes it.
 *    No C++ exception crosses the ABI.  All work is asynchronous on the bound
 *    stream except calls documented as synchronising.
 *  - A context is not thread-safe; use one context per host thread.
 */
#ifndef GFB200_H
#define GFB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gf_status {
  GF_OK = 0,
  GF_INVALID_ARG = 1,   /* bad size, null pointer, unknown mode */
  GF_CUDA_ERROR = 2,    /* a CUDA runtime call failed */
  GF_NOT_CONVERGED = 3, /* iterative solve stopped at its iteration cap */
  GF_NAN = 4,           /* non-finite value met in a reduction */
  GF_BREAKDOWN = 5,     /* CG denominator vanished */
  GF_TIMEOUT = 6,       /* a device-side wait exceeded its spin limit */
  GF_NO_DEVICE = 7      /* no CUDA device / not an sm_100 device */
} gf_status;

typedef enum gf_transfer { GF_FLIP = 0, GF_PIC = 1, GF_APIC = 2 } gf_transfer;

typedef enum gf_solver {
  GF_JACOBI = 0, /* k3_jacobi_pressure, solver3d.py:878-938 */
  GF_GSRB = 1,   /* k3_gauss_seidel_rb, solver3d.py:1204-1267 */
  GF_PCG = 2,    /* _pressure_pcg, solver3d.py:2917-3043 (FP32) */
  GF_PCG_REFINED = 3 /* FP32 PCG with FP64 residual replacement (no reference counterpart) */
} gf_solver;

typedef struct gf_grid_desc {
  int32_t nx, ny, nz;
  float dx;     /* cell size; FlipSolver3D.__init__ solver3d.py:2381 */
  float dom[3]; /* domain extent n*dx rounded to float32 (advection clamp, :1456-1460) */
} gf_grid_desc;

typedef struct gf_fields {
  float *u, *v, *w;    /* MAC face velocities */
  float *uw, *vw, *ww; /* P2G weight sums (scratch of the reference too) */
  float *us, *vs, *ws; /* saved pre-force velocities for the FLIP delta */
  float *p;            /* pressure (nx,ny,nz) */
  float *div;          /* Poisson right-hand side (nx,ny,nz) */
  uint8_t *label;      /* 0 air, 1 fluid, 2 solid (nx,ny,nz) */
  const float *solid_u, *solid_v, *solid_w; /* nullable: static solids (velocity 0) */
} gf_fields;

typedef struct gf_particles {
  int64_t n;
  float *pos;   /* (n,3) */
  float *vel;   /* (n,3) */
  float *C;     /* (n,3,3); may be NULL unless transfer == GF_APIC */
  int32_t *pid; /* (n) original id of the particle held in each storage slot */
} gf_particles;

typedef struct gf_step_params {
  float dt;
  float gravity;     /* signed acceleration on y */
  float rho;
  float flip_blend;  /* FLIP/PIC blend alpha (GF_FLIP, GF_PIC) */
  int32_t transfer;  /* gf_transfer */
  int32_t solver;    /* gf_solver */
  int32_t max_iters; /* pressure_iters */
  int32_t check_every; /* PCG convergence test cadence (reference: 10) */
  double tol;        /* PCG: relative residual target (reference: 1e-4) */
  int32_t rhs_sign;  /* PCG: -1 solves A p = -div (physical, Jacobi's sign);
                        +1 reproduces the reference PCG's r0 = +div */
  int32_t flags;     /* GF_FLAG_* */
} gf_step_params;

/* flags: run PCG in the global-memory kernel even when the active region fits
 * the shared-memory solver (both give the same iterates up to reduction order) */
#define GF_FLAG_GLOBAL_PCG 1
/* flags: record the SM clock (clock64, cycles) at every phase boundary of the
 * shared-memory PCG in block 0; read the stamps with gf_pcg_trace */
#define GF_FLAG_TRACE 2
/* flags bits 2-3: sweeps (1-3) of a tile-local red-black symmetric
 * Gauss-Seidel preconditioner for GF_PCG / GF_PCG_REFINED in the
 * shared-memory kernel; 0 keeps the reference's Jacobi preconditioner.  Same
 * operator and stop test; fewer iterations, one neighbour exchange more per
 * iteration.  The global-memory kernel (active regions too large for the
 * shared-memory solver) applies the same tile preconditioner. */
#define GF_FLAG_SGS_SHIFT 2
#define GF_FLAG_SGS_MASK 12
/* flags: add a coarse correction to the shared-memory PCG's preconditioner
 * (no counterpart in the reference): one constant per active 8^3 tile, the
 * rows of B ~ (P^T A P)^-1 computed (to 1e-3, stored as bfloat16) by two
 * kernels before every solve, M^-1 = M_tile^-1 + P B P^T.  Same operator,
 * stop test and answer; fewer iterations.  The global-memory kernel ignores
 * it. */
#define GF_FLAG_COARSE 16
/* flags, test only: the shared-memory PCG's first grid reduction waits for a
 * publication count that no block writes, with a spin limit of 4096 polls
 * instead of the normal one, so every block's wait runs out, the kernel
 * returns and the solve reports GF_TIMEOUT (gf_pressure_result,
 * gf_health_read).  It exercises the bounded-wait exit path without a fault;
 * the context stays usable.  No effect on the global-memory kernel. */
#define GF_FLAG_TEST_STALL 64
/* flags: the refined PCG (shared-memory or global-memory kernel) starts from
 * the pressure in fields.p (the previous substep's solution) instead of from
 * zero; the initial residual b - A p is formed in FP64 and the stop test
 * stays ||b - A x|| <= tol ||b||, so the answer's accuracy is the cold
 * start's.  No counterpart in the reference (its solves start from zero every
 * substep); other solvers ignore it. */
#define GF_FLAG_WARM_START 128

/* ---- context ------------------------------------------------------------ */
/* Allocates scratch for a grid and up to max_particles particles on the
 * current CUDA device (FlipSolver3D.__init__, solver3d.py:2358-2500). */
int gf_create(const gf_grid_desc *grid, int64_t max_particles, void **ctx_out);
int gf_destroy(void *ctx);
/* Grows particle scratch to hold n particles (seed_box re-binding, :2826-2910). */
int gf_reserve_particles(void *ctx, int64_t n);
/* Binds caller-owned device buffers (rebinding invalidates captured graphs). */
int gf_bind(void *ctx, const gf_fields *fields, const gf_particles *parts);
int gf_set_stream(void *ctx, void *cuda_stream);
const char *gf_last_error(void *ctx);
/* Number of kernels this context has launched so far. */
int64_t gf_launch_count(void *ctx);

/* ---- stages ------------------------------------------------------------- */
/* k3_clear_grid marker reset (solver3d.py:41-65) + the cell/label part of
 * k3_p2g (:92-101) + canonical binning: per-particle cell key, fluid labels,
 * per-cell counts, (cell, pid) ordering, sorted particle records. */
int gf_bin(void *ctx, int32_t transfer);
/* k3_p2g (:72-114) / k3_p2g_apic (:1475-1588): weighted face sums into
 * u,v,w and weights into uw,vw,ww (pre-normalisation, as the reference). */
int gf_p2g(void *ctx, int32_t transfer);
/* k3_normalize (:121-142) + k3_add_gravity (:149-156) + k3_enforce_solid_bc
 * (:758-799) + k3_compute_divergence (:846-871), fused. */
int gf_forces_div(void *ctx, float gravity, float dt, float rho);
/* Pressure solve into fields.p: Jacobi/GS-RB loops (:3594-3631) or PCG
 * (_pressure_pcg :2917-3043).  *iters_out (nullable, host) receives the
 * iteration count; writing it synchronises the stream. */
int gf_pressure(void *ctx, const gf_step_params *prm, int32_t *iters_out);
/* k3_subtract_pressure_grad (:1364-1407) + k3_enforce_solid_bc, fused. */
int gf_project(void *ctx, float dt, float rho);
/* k3_g2p_and_advect (:1414-1463) / k3_g2p_apic_advect (:1591-1732); writes
 * pos, vel, C, pid back into the caller's buffers in sorted storage order. */
int gf_g2p(void *ctx, int32_t transfer, float flip_blend, float dt);
/* The whole substep in _step_impl order (:3475-3667). */
int gf_step(void *ctx, const gf_step_params *prm);
/* The substep captured once as a CUDA graph and replayed: the reference's
 * graph cache (_cuda_graph_*, solver3d.py:3361-3418).  gf_graph_capture
 * synchronises the bound stream, records gf_step(prm) on it (on a private
 * stream when none is bound) without running it, and returns an instantiated
 * graph in *graph_out; every parameter and the bound buffers are baked in,
 * so rebinding or new parameters need a new capture.  gf_graph_replay
 * launches it on the bound stream (asynchronous); gf_graph_destroy frees it.
 * gf_step allocates nothing and never synchronises, which is what makes it
 * capturable; the stage-timing events are left out of a capture. */
int gf_graph_capture(void *ctx, const gf_step_params *prm, void **graph_out);
int gf_graph_replay(void *ctx, void *graph);
int gf_graph_destroy(void *graph);

/* ---- results and diagnostics ------------------------------------------- */
/* Last solve's iteration count, final relative residual (||r||/||r0||),
 * status; synchronises the stream. */
int gf_pressure_result(void *ctx, int32_t *iters, double *relres, int32_t *status);
/* Copies the last gf_bin's results to host arrays (any may be NULL):
 * key[n] per-particle tile-major cell key (8x8x8 tiles) in storage order,
 * count[ntiles*512] particles per key, order[n] storage slot of each sorted
 * position.  *nkeys (nullable) receives ntiles*512.  Synchronises. */
int gf_bin_read(void *ctx, int32_t *key, int32_t *count, int32_t *order, int64_t *nkeys);
/* Per-stage device times of the last gf_step when timing is on (ms, 8
 * entries: bin, p2g, forces_div, pressure, project, g2p, total, and the
 * pressure solver's own kernel(s) without set-up and scatter). */
int gf_enable_timing(void *ctx, int32_t on);
int gf_stage_times(void *ctx, float *ms8);

typedef struct gf_pressure_info {
  int32_t iters;        /* iterations of the last solve */
  int32_t replacements; /* FP64 residual replacements (GF_PCG_REFINED) */
  int32_t status;       /* gf_status of the solve */
  int32_t n_active_tiles;
  int64_t n_fluid;      /* fluid cells in the system */
  double relres;        /* ||r||/||r0|| (PCG), ||b-Ax||/||b|| in FP64 (refined), -1 otherwise */
  int32_t kernel;       /* PCG kernel that ran: 1 shared-memory resident, 2 global-memory */
  int32_t coarse;       /* 1: the solve applied the GF_FLAG_COARSE correction */
} gf_pressure_info;
/* Copies the trace buffer of the last traced PCG solve (up to cap int64
 * entries: block 0's SM-cycle stamps in the first half, *n of them, then per
 * block twelve values: busy cycles outside the all-reduce, tiles owned, fluid
 * cells owned, faces bordering another block's tile, and the cycles of eight
 * iteration phases as block thread 0 sees them -- own update, SGS sweeps,
 * halo publication with the neighbour flags and in-block rings, remote rings,
 * stencil and dot products, grid all-reduce, the coarse correction's gather
 * of the tiles' residual sums, its e = B g and addition to z) into host
 * memory; synchronises. */
int gf_pcg_trace(void *ctx, int64_t *host, int32_t cap, int32_t *n);
/* Statistics of the last pressure solve; synchronises. */
int gf_pressure_stats(void *ctx, gf_pressure_info *info);
/* Health of the pressure solves since the last reset, folded in on the device
 * by every gf_pressure / gf_step (and every replay of a captured gf_step), so
 * a host can check once per frame instead of synchronising per substep.  The
 * reference's PCG stops silently at its cap (_pressure_pcg, solver3d.py:
 * 2917-3043); its only failure check is the per-frame NaN probe of
 * has_diverged (:2642-2656).  On a batch every scene counts as one solve.
 * reset != 0 zeroes the record after reading it.  Synchronises. */
typedef struct gf_health {
  int32_t worst_status;  /* most severe gf_status since the reset: GF_OK < GF_NOT_CONVERGED <
                            GF_BREAKDOWN < GF_NAN < GF_TIMEOUT */
  int32_t solves;        /* pressure solves since the reset */
  int32_t not_converged; /* solves that stopped at their iteration cap */
  int32_t failed;        /* solves that ended in GF_BREAKDOWN, GF_NAN or GF_TIMEOUT */
  int32_t last_status;   /* most severe status of the last solve call */
  int32_t wait_timeouts; /* stage-kernel waits that ran out since the reset (the G2P
                            tile loads); the stage's results are then incomplete */
} gf_health;
int gf_health_read(void *ctx, int32_t reset, gf_health *out);
/* The bounds-checked build (libgfb200_checked.so, compiled with
 * -DGF_BOUNDS_CHECK; no counterpart in the reference, whose kernels index
 * unchecked, solver3d.py:100-101) checks the grid, tile, sort-slot and
 * neighbour indices its binning, transfer and pressure kernels compute before
 * they address global or shared memory, skips any access out of range and
 * counts it.  This reads the count since the last reset (all contexts of the
 * process) and the source line of the first violation; *checked = 1 in that
 * build, 0 in the regular one (where the count is always 0).  Synchronises. */
int gf_bounds_status(int32_t reset, int64_t *violations, int32_t *first_line,
                     int32_t *checked);
/* Active 8^3 pressure tiles of the last solve (k_mark_active_blocks,
 * solver3d.py:953-972): count and tile ids (device pointer). */
int gf_active_tiles(void *ctx, int32_t *n_active, const int32_t **tiles);
/* Device |v|^2 max for CFL substepping (k3_vmax_sq_reduce :2241-2252);
 * synchronises. */
int gf_vmax(void *ctx, float *vmax_out);
/* Outflow regions (k3_mark_alive_outflows + k3_scatter_alive,
 * solver3d.py:1943-1985, driven by _apply_outflows_gpu :2659-2730): copies the
 * n particles (device pos, vel, (n,3) float32) that lie inside none of the
 * nbox boxes (host array of nbox x {lo.x, lo.y, lo.z, hi.x, hi.y, hi.z};
 * inside means lo <= p <= hi on all axes) to pos_out / vel_out (device, room
 * for n, not overlapping the inputs), keeping their order, and writes the new
 * count to *n_out.  Runs on the bound stream and synchronises for the count;
 * allocates its scratch in the context on first use.  A box with hi < lo is
 * GF_INVALID_ARG. */
int gf_outflow_compact(void *ctx, const float *pos, const float *vel, int64_t n,
                       const float *boxes, int32_t nbox, float *pos_out, float *vel_out,
                       int64_t *n_out);
/* The same compaction with a per-particle keep flag (alive[i] != 0, device
 * int32[n]) in place of the boxes: k3_scatter_alive / k_scatter_alive_pv
 * (solver3d.py:1968-1985, reseed.py:226-243). */
int gf_compact_alive(void *ctx, const float *pos, const float *vel, int64_t n,
                     const int32_t *alive, float *pos_out, float *vel_out, int64_t *n_out);
/* Reseed culling on the bound particles (k_count_particles_per_cell +
 * k_mark_keep_by_rank, reseed.py:161-222): bins them (as gf_bin; labels are
 * recomputed from the current positions), then writes alive[id] = 1 for the
 * first max_per_cell particles by id of each non-solid cell and 0 otherwise
 * (the reference ranks by atomic arrival; ranking by id is one of its
 * orders), and counts[nx*ny*nz] (device int32, C order) = particles per
 * cell.  Single-grid contexts; the bound pid must hold ids 0..n-1. */
int gf_reseed_mark(void *ctx, int32_t max_per_cell, int32_t *alive, int32_t *counts);
/* The emission count of reseeding (reseed.py:345-352): the sum over cells of
 * max(min_per_cell - counts, 0) where the cell is fluid (label 1, or counts >
 * 0) and not solid (label 2).  label (uint8) and counts (int32) are device
 * arrays of nx*ny*nz cells in C order: the labels the last substep left and
 * the counts gf_reseed_mark wrote.  Synchronises for the count. */
int gf_reseed_deficit(void *ctx, const uint8_t *label, const int32_t *counts,
                      int32_t min_per_cell, int64_t *n_emit);
/* The emitted positions (reseed.py:362-367): for each deficit cell in C
 * order, its deficit copies of (cell + 0.5 + jitter[e]) * dx into
 * pos_out[e] (device (n_emit,3) float32); jitter is a device (n_emit,3)
 * float32 array (the reference draws it on the host).  Asynchronous. */
int gf_reseed_emit(void *ctx, const uint8_t *label, const int32_t *counts, int32_t min_per_cell,
                   const float *jitter, float *pos_out);

/* ---- surface mesh after the substeps ------------------------------------ */
/* A mesher replaces MeshExtractor (src/gpufluid/meshing/surface.py:199-461):
 * it owns two cell-centred density fields of nx*ny*nz floats (dens /
 * dens_tmp, surface.py:206-216) and the extraction scratch, and runs on its
 * own stream.  It is independent of a solver context: pass it the particle
 * positions (device (n,3) float32) of any solver. */
#define GF_MESH_TRILINEAR 0 /* k_density_scatter, surface.py:14-43 */
#define GF_MESH_CUBIC 1     /* k_cubic_scatter, surface.py:53-84 */
#define GF_MESH_SDF 2       /* k_sdf_field, surface.py:100-122 (surface at phi <= 0) */
typedef struct gf_mesh_params {
  int32_t method;             /* GF_MESH_TRILINEAR | GF_MESH_CUBIC | GF_MESH_SDF */
  int32_t smooth_passes;      /* k_box_blur_3d passes (gridmath.py:103-121) */
  int32_t wall_margin_cells;  /* k_mc_zero_walls margin (surface.py:179-193); 0 = off;
                                 ignored by GF_MESH_SDF, as in the reference */
  float cubic_radius_cells;   /* GF_MESH_CUBIC support radius in cells */
  float sdf_particle_radius_cells; /* GF_MESH_SDF particle radius in cells */
  float sdf_search_radius_cells;   /* GF_MESH_SDF search radius in cells */
} gf_mesh_params;
int gf_mesher_create(int32_t nx, int32_t ny, int32_t nz, float dx, void *cuda_stream,
                     void **mesher_out);
int gf_mesher_destroy(void *mesher);
const char *gf_mesher_last_error(void *mesher);
int gf_mesher_set_stream(void *mesher, void *cuda_stream);
/* The density field the last gf_mesher_density left (device, nx*ny*nz,
 * C order); valid until the next gf_mesher_density. */
float *gf_mesher_field(void *mesher);
/* Copy that field (nx*ny*nz floats) to `out` (host or device).  Synchronising. */
int gf_mesher_copy_field(void *mesher, float *out);
/* Kernel launches issued by this mesher so far. */
int64_t gf_mesher_launches(void *mesher);
/* Zero the field, splat the n particles, blur smooth_passes times, zero the
 * wall margin (surface.py:388-425, the "trilinear" and "cubic" branches).
 * Asynchronous. */
int gf_mesher_density(void *mesher, const float *pos, int64_t n, const gf_mesh_params *prm);
/* Iso-surface {density >= iso_level} of `field` (device nx*ny*nz floats;
 * NULL = the mesher's own field); replaces the marching cubes of
 * _mc_extract_gpu / _mc_extract_cpu (surface.py:286-351).  By default
 * marching cubes: vertices on the axis edges at the linear crossing, the
 * triangles of each cube from a case table in which ambiguous faces keep
 * their inside corners apart (so neighbouring cubes agree and the surface is
 * closed), at most 5 per cube, facing from >= iso to < iso.  Vertices are
 * grid index * dx.  Writes the vertex and triangle counts (0, 0 when no
 * surface crosses the grid: the reference's "no surface" result) and keeps
 * the mesh in the mesher.  Synchronises once for the counts. */
int gf_mesher_extract(void *mesher, const float *field, float iso_level, int64_t *n_verts,
                      int64_t *n_tris);
/* Surface method of gf_mesher_extract: GF_SURFACE_MARCHING_CUBES (default) or
 * GF_SURFACE_MARCHING_TETRAHEDRA (the six-tetrahedron Kuhn split of each
 * cube: no ambiguous cases, vertices also on face and body diagonals, up to
 * 12 triangles per cube; its axis-edge vertices are the marching-cubes ones). */
#define GF_SURFACE_MARCHING_CUBES 0
#define GF_SURFACE_MARCHING_TETRAHEDRA 1
int gf_mesher_set_surface(void *mesher, int32_t method);
/* The marching-cubes case table gf_mesher_extract uses (host memory, no
 * device needed): edges[12][2] corner pairs (corner bit 0 +x, bit 1 +y, bit 2
 * +z), ntri[256] triangles per case (bit c of the case: corner c inside),
 * tri[256][15] edge indices, three per triangle. */
int gf_marching_cubes_table(uint8_t *edges, uint8_t *ntri, uint8_t *tri);
/* Which side of the level is inside for the next gf_mesher_extract: 0 (the
 * default after a GF_MESH_TRILINEAR / GF_MESH_CUBIC field) encloses
 * values >= iso, 1 (set by a GF_MESH_SDF field) values <= iso. */
int gf_mesher_set_inside_below(void *mesher, int32_t below);
/* Copy the last extraction out: verts (n_verts,3) float32, tris (n_tris,3)
 * int32, host or device memory.  Synchronising. */
int gf_mesher_copy(void *mesher, float *verts, int32_t *tris);
/* Uniform-Laplacian mesh smoothing (smoothing.py:22-72): `passes` steps of
 * v += lam L v (GF_MESH_SMOOTH_LAPLACIAN) or pairs v += lam L v; v += mu L v
 * (GF_MESH_SMOOTH_TAUBIN), L = D^-1 A - I of the triangles' 1-rings, in
 * float64 and in the reference's order of operations, then rounded to float32
 * in place.  verts/tris: device arrays, or verts = NULL for the mesher's last
 * extraction (before gf_mesher_copy).  Asynchronous. */
#define GF_MESH_SMOOTH_LAPLACIAN 0
#define GF_MESH_SMOOTH_TAUBIN 1
int gf_mesher_smooth(void *mesher, float *verts, int64_t n_verts, const int32_t *tris,
                     int64_t n_tris, int32_t method, int32_t passes, double lam, double mu);

/* ---- adjoint (differentiation through substeps) ------------------------- */
/* No counterpart in the reference (planned only there).  PIC transfer
 * (flip_blend 0) or APIC, with the cell labels held fixed within each substep.
 * gf_step_record runs gf_step and copies into `record` (a caller-owned device
 * buffer of gf_record_bytes bytes) what the adjoint needs: the substep's
 * sorted inputs, their storage slots, the P2G weight sums and normalised
 * velocities, the final face velocities and the labels.  The outputs of a
 * recorded substep are in its sorted order; gf_step_adjoint maps the adjoint
 * of those outputs (xbar_out, vbar_out, (n,3)) to the adjoint of its inputs
 * in their storage order (xbar_in, vbar_in): G2P/advection adjoint (a scatter
 * onto the faces), pressure-gradient adjoint, a second solve with the same
 * SPD Laplacian (prm->solver, rhs sign +1), divergence/boundary/normalisation
 * adjoint, P2G adjoint (a gather).  It overwrites the context's div, p and
 * label buffers. */
int gf_record_bytes(void *ctx, int64_t *bytes);
int gf_step_record(void *ctx, const gf_step_params *prm, void *record);
int gf_step_adjoint(void *ctx, const gf_step_params *prm, const void *record,
                    const float *xbar_out, const float *vbar_out, float *xbar_in,
                    float *vbar_in);
/* The same for an APIC substep (k3_p2g_apic :1475-1588, k3_g2p_apic_advect
 * :1591-1732), which also carries the adjoint of the affine matrices:
 * Cbar_out / Cbar_in are (n,3,3) row-major like C, in the output's sorted
 * order / the input's storage order. */
int gf_step_adjoint_apic(void *ctx, const gf_step_params *prm, const void *record,
                         const float *xbar_out, const float *vbar_out, const float *Cbar_out,
                         float *xbar_in, float *vbar_in, float *Cbar_in);
/* Cell-centred trilinear density splat of unit-mass particles into rho
 * (nx,ny,nz) (k_density_scatter, meshing/surface.py:14-43) and its adjoint
 * with respect to the positions.  On a batch context, n is the bound
 * particle count (scene after scene) and rho the scenes' cell arrays
 * concatenated. */
int gf_density_splat(void *ctx, const float *pos, int64_t n, float *rho);
int gf_density_splat_adjoint(void *ctx, const float *pos, int64_t n, const float *rho_bar,
                             float *pos_bar);
/* Velocities sampled from a cell-centred 3-component field (3,nx,ny,nz) with
 * the same weights, and the adjoint with respect to the field (a scatter).
 * On a batch context the field holds each scene's (3,nx,ny,nz) block at
 * 3 * cell0 and n is the bound particle count. */
int gf_sample_cells(void *ctx, const float *grid3, const float *pos, int64_t n, float *vel);
int gf_sample_cells_adjoint(void *ctx, const float *pos, int64_t n, const float *vel_bar,
                            float *grid3_bar);

/* ---- batches of independent scenes -------------------------------------- */
/* No counterpart in the reference (which steps one FlipSolver3D at a time).
 * A batch context steps many scenes of uneven grid sizes together: gf_step
 * (and every stage call) runs ONE launch per stage kernel over all scenes,
 * each item finding its scene in a segment table; the pressure PCG is one
 * persistent kernel that keeps per-scene scalars and stops each scene at its
 * own tolerance.  Scenes are concatenated in table order in every array:
 * cells (label, p, div), u-, v- and w-shaped faces, particles (the caller
 * passes each scene's particle count).  gf_batch_plan returns that layout
 * (per scene, nullable) and the totals without touching a GPU; solid
 * velocities must be NULL (static solids).  The adjoint, density-splat and
 * control-sampling calls work on batches too (one launch per kernel). */
typedef struct gf_scene_layout {
  int64_t cell0;           /* first cell of the scene in cell arrays */
  int64_t fu0, fv0, fw0;   /* first u, v, w face in the face arrays */
  int64_t tile0, ntiles;   /* its 8^3 tiles (sort key = tile*512 + local cell) */
  int64_t fslot0;          /* first (nx+1)(ny+1)(nz+1) face slot */
} gf_scene_layout;
typedef struct gf_batch_totals {
  int64_t ncell, nu, nv, nw, ntiles, nslot;
} gf_batch_totals;
int gf_batch_plan(const gf_grid_desc *scenes, int32_t n, gf_scene_layout *rows,
                  gf_batch_totals *totals);
int gf_batch_create(const gf_grid_desc *scenes, int32_t n, int64_t max_particles,
                    void **ctx_out);
/* fields: concatenated arrays sized by gf_batch_totals; parts: all scenes'
 * particles, scene after scene; counts[n]: particles per scene. */
int gf_batch_bind(void *ctx, const gf_fields *fields, const gf_particles *parts,
                  const int64_t *counts);
/* Per-scene iterations, relative residual and status of the last pressure
 * solve (arrays of n, each nullable); synchronises. */
int gf_batch_pressure_stats(void *ctx, int32_t *iters, double *relres, int32_t *status);

/* ---- launch-shape autotuner --------------------------------------------- */
/* No counterpart in the reference.  gf_autotune times real substeps (the
 * particle state is restored afterwards) and keeps the fastest tile and launch
 * shapes: the cell blocks of P2G and of the tile-staged G2P (single grid),
 * the batches' G2P block size, the grid-stride face/cell kernels and the
 * global-memory PCG's residency; gf_get_tune / gf_set_tune read or impose
 * them.  Synchronises. */
typedef struct gf_tune_info {
  int32_t g2p_threads;        /* threads per block of the batches' G2P (32..512) */
  int32_t grid_threads;       /* threads per block of forces/divergence/project */
  int32_t grid_blocks_per_sm; /* cap of their grid-stride launches */
  int32_t pcg_blocks_per_sm;  /* global-memory PCG residency, 0 = occupancy maximum */
  float step_ms_before, step_ms_after;  /* gf_autotune: substep time before / after */
  int32_t p2g_tiles_k;        /* P2G blocks: 8^3 cells (1) or 8 x 8 x 16 (2) */
  int32_t g2p_tiles_k;        /* tile-staged G2P blocks: 8^3 cells (1) or 8 x 8 x 16 (2);
                                 0: one thread per particle, no staged boxes */
  int32_t p2g_map;            /* P2G lanes: runs of a block's particles (0), one cell each (1),
                                 one cell each summed in registers first (2), the same
                                 reading the particles from coalesced shared staging (3),
                                 or from warp-staged rounds of 8 (4) or 4 (5) particles
                                 per cell */
} gf_tune_info;
int gf_autotune(void *ctx, const gf_step_params *prm, gf_tune_info *out);
int gf_get_tune(void *ctx, gf_tune_info *out);
int gf_set_tune(void *ctx, const gf_tune_info *in);

/* ---- allocation-free variant ------------------------------------------- */
/* No counterpart in the reference.  For callers that may not allocate device
 * memory (a host that owns every device allocation through its own pool and
 * forbids libraries from calling cudaMalloc / cudaFree): a Jacobi pressure
 * solve with the
 * arithmetic of gf_pressure(GF_JACOBI) on the dense grid -- label (uint8),
 * div and p are (nx,ny,nz) device arrays owned by the caller; p receives the
 * result of `iters` sweeps started from zero.  Its only scratch is a static
 * device array of GF_NOALLOC_MAX_CELLS floats (8 MiB) that every GPU loading
 * the library holds until exit; larger grids return GF_INVALID_ARG.  It calls
 * no cudaMalloc/cudaFree.  Calls share that array: calls overlapping on the
 * GPU race, calls in order on one stream are safe.  The first call on a
 * device resolves the array's device address (cudaGetSymbolAddress) and
 * should come before any stream capture (on a capturing stream it returns
 * GF_INVALID_ARG).  label, div, p and the stream belong to the current device.
 * Errors pending from earlier work are cleared on entry, so the status is
 * this call's own.  Asynchronous on cuda_stream. */
#define GF_NOALLOC_MAX_CELLS 2097152
int gf_jacobi_noalloc(int32_t nx, int32_t ny, int32_t nz, const uint8_t *label,
                      const float *div, float *p, int32_t iters, void *cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* GFB200_H */
