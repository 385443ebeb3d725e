/*
 * ssenss_b200 -- B200 (sm_100a) implementation of the SSENSS per-timestep
 * solve path behind a plain C ABI.
 *
 * The host (the SSENSS C driver: src/main.c, src/navier_stokes.c,
 * src/stokes.c, src/time.c) keeps its own call surface; a thin binding maps
 * each of the reference functions named below onto one of these entry
 * points.  All compute runs as hand-written CUDA kernels on one GPU; there is
 * no CPU fallback: every entry point fails with SSG_ERR_CUDA when no device
 * is usable.
 *
 * Conventions
 *  - A field is an element-local L-vector u[e][k][j][i], i fastest, nel * n^3
 *    doubles, n = GLL points per direction (N+1), exactly the contiguous
 *    block new_4d_array allocates (src/utils.c:64-81).  Vector fields are
 *    three such blocks, x then y then z.
 *  - Every field argument may be a host pointer or a device pointer (CUDA
 *    global memory); the library tells them apart with
 *    cudaPointerGetAttributes.  Host arguments are copied through pinned
 *    staging on the context's stream.
 *  - Every entry point returns an ssg_status; SSG_OK is 0.  Nothing exits
 *    the process (the reference's fatal_error, src/utils.c:162-174, does).
 *  - A context is re-entrant with respect to other contexts; calls on one
 *    context must not overlap.  All work of a context is ordered on its
 *    CUDA stream; calls return after that work has completed unless stated.
 *  - var follows src/poisson.h:33: SSG_PRESSURE selects the Laplacian
 *    (Poisson, nullspace removed, no Dirichlet mask), the velocities select
 *    the Helmholtz operator with lambda = (11/6) / (dt * visc)
 *    (src/helmholtz.c:37-38) and the Dirichlet mask.
 */
#ifndef SSENSS_B200_H
#define SSENSS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
	SSG_OK = 0,
	SSG_ERR_ARG = 1,        /* invalid argument or unsupported order */
	SSG_ERR_CUDA = 2,       /* CUDA runtime failure / no device */
	SSG_ERR_NOMEM = 3,      /* device allocation failed */
	SSG_ERR_BUDGET = 4,     /* request exceeds the HBM budget */
	SSG_MAXITER = 5,        /* iteration cap reached before eps */
	SSG_NONFINITE = 6,      /* NaN/Inf residual or breakdown */
	SSG_ERR_MESH = 7,       /* inconsistent connectivity */
	SSG_ERR_STATE = 8,      /* call out of order (no mesh yet, ...) */
	SSG_ERR_TIMEOUT = 9,    /* deadline or bounded device wait expired */
	SSG_ERR_CANCELLED = 10  /* request cancelled */
} ssg_status;

enum {
	SSG_PRESSURE = 0,
	SSG_X_VELOCITY = 1,
	SSG_Y_VELOCITY = 2,
	SSG_Z_VELOCITY = 3
};

/* arithmetic of the preconditioner (the outer Krylov loop, its residual and
 * inner products, DSS accumulation and the coarse solve stay FP64) */
enum {
	SSG_PRECISION_FP64 = 0,
	SSG_PRECISION_MIXED = 1  /* FP32 smoothers, transfers and local
	                            operator inside the p-multigrid V-cycle */
};

typedef struct ssg_context ssg_context;

/* Outcome of one solve.  history, when non-NULL, receives sqrt((r.r)_w)
 * after each outer iteration (the reference's residual check,
 * src/solver.c:72-73 and 151-152), at most history_cap values. */
typedef struct {
	int iterations;          /* outer iterations run */
	double residual;         /* final sqrt((r.r)_w) */
	double initial_residual; /* sqrt((r.r)_w) before the first iteration */
	double solve_ms;         /* device time of the solve (CUDA events) */
	double *history;
	int history_cap;
	int history_len;
} ssg_solve_info;

/* ---- context ---------------------------------------------------------- */

/* Create a context on CUDA device `device` with its own stream.  Replaces
 * the process-wide state main.c builds (src/main.c:36-90). */
ssg_status ssg_create(int device, ssg_context **out);
/* Same, ordering all work on the caller's stream (a cudaStream_t). */
ssg_status ssg_create_on_stream(int device, void *cuda_stream,
		ssg_context **out);
void ssg_destroy(ssg_context *ctx);
const char *ssg_status_string(ssg_status s);
/* Detail of the last failure on this context (never NULL). */
const char *ssg_last_error(const ssg_context *ctx);
/* The context's cudaStream_t. */
void *ssg_stream(const ssg_context *ctx);

/* struct parameters fields used by the solve path (src/structs.h:56-79). */
ssg_status ssg_set_parameters(ssg_context *ctx, double dt, double visc,
		double dens);
ssg_status ssg_set_precision(ssg_context *ctx, int precision);
/* Use CUDA graphs for the Krylov iterations (default on). */
ssg_status ssg_set_graphs(ssg_context *ctx, int enable);

/* ---- discretisation set-up ------------------------------------------- */

/* Set-up options of the next ssg_setup_mesh (no reference counterpart):
 * skip the dealiasing grid (convection unavailable) and/or the particle
 * geometry, for contexts that only solve -- e.g. the serving loop's.
 * SSG_SETUP_OPPOSITE_PAIRING pairs each face, edge and corner with the
 * geometrically opposite one of its neighbour (west with east, ...) instead
 * of the reference's first match (src/init.c:68-130, 298-320), which with
 * one or two elements along a periodic direction pairs west with west and
 * so solves a different, wrong system.  On meshes with three or more
 * elements in every direction both pairings are the same; the serving loop
 * uses the opposite pairing for every request. */
#define SSG_SETUP_NO_DEALIAS 1u
#define SSG_SETUP_NO_PARTICLES 2u
#define SSG_SETUP_OPPOSITE_PAIRING 4u
ssg_status ssg_set_setup_options(ssg_context *ctx, unsigned flags);
/* Spectral vanishing viscosity of the Helmholtz operator for the next
 * ssg_setup_mesh (params->svvn, params->svva; src/main.c:54-55): every
 * level's SVV derivative matrix is built with cut-off mode svvn and
 * amplitude svva as compute_svv_derivative_matrix does (src/deriv.c:81-112,
 * src/precon.c:130-132).  svvn < 0 takes the reference's default 2n/3; the
 * default amplitude is 0 (the reference's). */
ssg_status ssg_set_svv(ssg_context *ctx, int svvn, double svva);
/* Device memory (bytes) the context holds now. */
ssg_status ssg_memory_info(const ssg_context *ctx, size_t *device_bytes);

/* Build the whole discretisation from grid records, as read_grid +
 * connect_elements + initialise_preconditioners do (src/dataio.c:197-227,
 * src/init.c:38-50, src/precon.c:196-205): GLL bases of all p-multigrid
 * levels (src/precon.c:58-83), geometric factors, the dealiasing grid
 * (m = 3n/2, src/main.c:53), Jacobi diagonals, DSS pairing.
 *   vertices: nel x {x[8], y[8], z[8]} (trilinear n=2 element, x fastest)
 *   neigh:    nel x {face[6], edge[12], corner[8]} neighbour element ids,
 *             negative = wall code (-1 = no-slip / Dirichlet). */
ssg_status ssg_setup_mesh(ssg_context *ctx, int n, int nel,
		const double *vertices, const int *neigh);

/* Drop-in set-up from the host's own discretisation (what the reference
 * already holds in sel[i]->precon after initialise_preconditioners).
 * Call ssg_setup_connectivity, then ssg_setup_level for every level
 * 0..nlevels-1 (orders as new_preconditioner gives, src/precon.c:62-69),
 * then ssg_setup_finish.
 *   deriv, svv_deriv: n*n, the stored basis->deriv_matrix / svv_deriv_matrix
 *                     (d[j][i] = D_ij, src/basis.c:160-177)
 *   weights:          n GLL weights
 *   geom:             6 x nel x n^3: G11, G12, G13, G22, G23, G33
 *                     (geom_mat, src/geometry.c:130-135)
 *   jac_det:          nel x n^3
 *   interp:           level >= 1: the fine-duplicate basis interp_matrix,
 *                     n_coarse x n_fine doubles (src/precon.c:130-137);
 *                     NULL at level 0. */
ssg_status ssg_setup_connectivity(ssg_context *ctx, int nel,
		const int *neigh);
ssg_status ssg_setup_level(ssg_context *ctx, int level, int n,
		const double *deriv, const double *svv_deriv,
		const double *weights, const double *geom,
		const double *jac_det, const double *interp);
ssg_status ssg_setup_finish(ssg_context *ctx);

/* Dealiasing grid for convection_operator: conv_basis order m and its
 * factors (tinv_jac 9 x nel x m^3 row-major [a][b] after the transpose of
 * src/geometry.c:112, jac_det nel x m^3, weights m, deriv m*m stored as
 * d[j][i], interp = conv_basis->interp_matrix n x m). Drop-in path only;
 * ssg_setup_mesh builds it itself. */
ssg_status ssg_setup_dealias(ssg_context *ctx, int m, const double *deriv,
		const double *weights, const double *tinv_jac,
		const double *jac_det, const double *interp);

/* Level-0 data the particle walk reads (src/particles.c:493-539): the GLL
 * points (n; sel->basis->points, which the reference computes by an
 * eigenvalue solve, so they may differ in the last bit from this library's
 * own; NULL keeps the library's), jac (9 x nel x n^3, J[a][b] = dx_a/dr_b)
 * and tinv_jac (9 x nel x n^3) as the reference stores them.  Passing the
 * reference's arrays makes the walk bitwise the reference's. ssg_setup_mesh
 * builds its own; this call replaces them (before or after setup). */
ssg_status ssg_setup_particle_geometry(ssg_context *ctx, const double *points,
		const double *jac, const double *tinv_jac);

ssg_status ssg_mesh_info(const ssg_context *ctx, int *n, int *nel,
		int *nlevels, int *orders /* >= 8 entries or NULL */);
/* Read back level data: which 0..5 = G * rho * J (the factors the
 * operator streams), 6 = rho * J, 7 = Poisson diagonal inverse,
 * 8 = Helmholtz diagonal inverse, 9 = 1/multiplicity, 10 = Dirichlet mask,
 * 11 = inverse assembled mass (level 0), 12..14 = GLL grid x, y, z. */
ssg_status ssg_level_data(ssg_context *ctx, int level, int which,
		double *dst);

/* ---- operators ---------------------------------------------------------- */

/* ap = DSS(mask(A_e p)) -- global_opeval (src/solver.c:191-198) with
 * discrete_laplace_operator (var = SSG_PRESSURE, src/poisson.c:34-56) or
 * discrete_helmholtz_operator (src/helmholtz.c:33-49). */
ssg_status ssg_global_opeval(ssg_context *ctx, int var, const double *p,
		double *ap);
/* Element-local operator only, no mask or DSS (parity tests). */
ssg_status ssg_local_opeval(ssg_context *ctx, int var, const double *p,
		double *ap);
/* In-place DSS -- direct_stiffness_summation (src/global.c:241-257);
 * integer pairing and addition order as the reference's, so the result
 * is bitwise equal. */
ssg_status ssg_direct_stiffness_summation(ssg_context *ctx, double *u);
/* sum (x * w) * y, w = 1/multiplicity -- global_dot_product
 * (src/global.c:270-282). */
ssg_status ssg_global_dot_product(ssg_context *ctx, const double *x,
		const double *y, double *out);
/* Weighted inner product sum (x * w) * y over n doubles, the quantity
 * ssg_global_dot_product computes, from three caller-owned device arrays
 * (w = 1/multiplicity, as ssg_level_data selector 9 returns it).  The result
 * is written to the device double *result; the work is enqueued on
 * cuda_stream (a cudaStream_t, NULL = the default stream) without waiting.
 * Allocates no device memory, for applications that cannot let a library
 * call cudaMalloc (a process that hands all device memory to its own pool
 * under a fixed budget, or a loop that must not take cudaMalloc's implicit
 * synchronisation).  Its block partial sums live in one fixed 512 KiB array
 * per GPU shared by every call: n above 134,217,728 is rejected with
 * SSG_ERR_ARG, host pointers and pointers to another GPU's memory likewise
 * (every array must live on the current device, or be managed memory), and
 * calls that overlap on the GPU race on the array.  The first call on a
 * device looks the array's address up; make that call before any stream
 * capture on the device.  The address is kept for the life of the process;
 * calls after a cudaDeviceReset are not supported.
 * No counterpart in the reference. */
ssg_status ssg_weighted_dot_noalloc(const double *x, const double *y,
		const double *w, size_t n, double *result, void *cuda_stream);
/* u *= inverse assembled mass -- global_inverse_mass_matrix_operator
 * (src/poisson.c:77-87). */
ssg_status ssg_inverse_mass(ssg_context *ctx, double *u);

/* ---- solves ------------------------------------------------------------- */

/* solve_poisson_cg (src/solver.c:159-173): flexible CG with the
 * p-multigrid preconditioner to sqrt((r.r)_w) <= eps, at most max_iter
 * (the reference uses 5000).  u holds the initial guess and receives the
 * solution.  Returns SSG_MAXITER when the cap is hit (u still written). */
ssg_status ssg_solve_poisson_cg(ssg_context *ctx, const double *f, double *u,
		double eps, int max_iter, ssg_solve_info *info);
/* solve_helmholtz_cg (src/solver.c:175-189): CG with the Jacobi
 * preconditioner on the Helmholtz operator. */
ssg_status ssg_solve_helmholtz_cg(ssg_context *ctx, int var, const double *f,
		double *u, double eps, int max_iter, ssg_solve_info *info);
/* Helmholtz solves of several independent meshes in shared launches (no
 * reference counterpart: the reference solves one mesh per process).  The
 * context's mesh is the concatenation of nseg meshes: segment s is the
 * elements seg_first[s] .. seg_first[s+1]-1 (seg_first[0] = 0,
 * seg_first[nseg] = nel; no element may neighbour another segment's,
 * checked).  Segment s is solved as solve_helmholtz_cg would
 * (src/solver.c:33-81, 175-189) with Helmholtz constant lambda[s] (the
 * context's dt and viscosity are not used) and absolute stop eps[s], with
 * its own CG scalars, stop test and iteration count; every iteration's
 * element operator and DSS are one launch over all segments.  f, u: the
 * concatenated fields (u: initial guess in, solution out), host or device.
 * info[s] receives the segment's iterations and residuals (no history).
 * Each segment's sums are grouped differently from a solo solve's, so its
 * iterates agree with ssg_solve_helmholtz_cg on the same mesh to rounding.
 * Returns SSG_MAXITER when a segment hits max_iter. */
ssg_status ssg_solve_helmholtz_segments(ssg_context *ctx, int var, int nseg,
		const int *seg_first, const double *lambda, const double *f,
		double *u, const double *eps, int max_iter, ssg_solve_info *info);
/* conjugate_gradient with jacobi_preconditioner on either operator
 * (src/solver.c:33-81). */
ssg_status ssg_conjugate_gradient(ssg_context *ctx, int var, const double *f,
		double *u, double eps, int max_iter, ssg_solve_info *info);
/* z = r .* diag^-1 of the level-0 operator of var (Poisson for
 * SSG_PRESSURE, else the Helmholtz operator at the context's lambda):
 * jacobi_preconditioner (src/precon.c:311-315, diagonal_preconditioner with
 * omega 1, alpha 0).  z is output only. */
ssg_status ssg_jacobi_preconditioner(ssg_context *ctx, int var, const double *r,
		double *z);
/* One application z = M^-1 r of multigrid_preconditioner
 * (src/precon.c:227-236). */
ssg_status ssg_multigrid_preconditioner(ssg_context *ctx, const double *r,
		double *z, double eps);

/* ---- convection ----------------------------------------------------------- */

/* Dealiased skew-symmetric convection of the whole mesh --
 * convection_operator for every element (src/convection.c:31-69).
 * u (advecting), v (advected), udv: 3 x nel x n^3.  At n = 8 both forms
 * the time step calls run on the FP64 tensor cores: a field advected by
 * another (the RK4 stages, src/time.c:114-116) and, when u and v are the
 * same pointer, the velocity advecting itself (the history term,
 * src/navier_stokes.c:79-83: three fields interpolated instead of six);
 * the two agree to rounding. */
ssg_status ssg_convection_operator(ssg_context *ctx, const double *u,
		const double *v, double *udv);
/* convection_operator for the elements first .. first+count-1 only: the
 * reference's own per-element call (src/convection.c:31-35, one element per
 * call from src/time.c:115-117 and src/navier_stokes.c:82) is count = 1.
 * u, v, udv: 3 x count x n^3 (component-major over the range). */
ssg_status ssg_convection_elements(ssg_context *ctx, int first, int count,
		const double *u, const double *v, double *udv);

/* The velocity history the convection sub-steps interpolate in time
 * (add_interpolated_velocity, src/time.c:132-152): sel->u, sel->old->u,
 * sel->old->old->u (each 3 x nel x n^3, host or device, copied) at the
 * solver time t (params->t) with step dt (params->dt). */
ssg_status ssg_set_velocity_history(ssg_context *ctx, const double *u,
		const double *u_old, const double *u_oldold, double t, double dt);
/* integrate_convection_rk4 (src/time.c:84-130) on the device: u
 * (3 x nel x n^3, host or device, in/out) += beta * the history
 * interpolated at t0, then RK4 sub-steps of dt from t0 to t, each stage a
 * dealiased convection of the stage field by the interpolated velocity,
 * DSS and the inverse mass.  Needs the dealiasing grid and
 * ssg_set_velocity_history. */
ssg_status ssg_integrate_convection_rk4(ssg_context *ctx, double *u, double t0,
		double t, double dt, double beta);

/* ---- the whole time step on the device (src/navier_stokes.c) --------------- */

/* The per-element state integrate_navier_stokes (src/navier_stokes.c:
 * 224-235) reads and writes, gathered over the mesh: level 0 = the current
 * time (sel->u, sel->conv, sel->rot, sel->p), 1 = sel->old->..., 2 =
 * sel->old->old->...  u, conv, rot and f hold three components of
 * nel x n^3 each (component-major); p one.  Host or device pointers. */
typedef struct ssg_flow_fields {
	double *u[3];     /* velocity */
	double *conv[3];  /* convection history (the velocity's self-convection) */
	double *rot[3];   /* double-curl history (curl curl u times the mass) */
	double *p[3];     /* pressure */
	double *f;        /* body force (sel->f); may be null: zero */
} ssg_flow_fields;

/* Copy the state in (every level of u, conv, rot and p is needed) at
 * solver time t (params->t).  The fields then stay on the device; the
 * parameters of ssg_set_parameters are the step's dt, visc and dens.
 * Needs the dealiasing grid and the level-0 Jacobian
 * (ssg_setup_particle_geometry, or ssg_setup_mesh with particles). */
ssg_status ssg_flow_set(ssg_context *ctx, const ssg_flow_fields *in, double t);
/* Copy the resident state out into the non-null pointers of out; *t (if
 * not null) = the solver time. */
ssg_status ssg_flow_get(ssg_context *ctx, ssg_flow_fields *out, double *t);
/* One step of integrate_navier_stokes on the resident state: the convection
 * history and sub-steps, the pressure right-hand side, extrapolation and
 * solve, the velocity right-hand sides, extrapolation and solves; the time
 * advances by dt.  f (3 x nel x n^3, may be null: the resident body force
 * stays) is the step's source term (set_source_term at t + dt).  On a mesh
 * with walls, bc_u and bc_dudt (3 x nel x n^3 each) hold the boundary
 * functions sel->bc_func[c] and sel->bc_dfunc[c] at t + dt on every wall
 * node (other entries are not read); without walls they may be null.
 * info (may be null): 4 records, the pressure solve and the three velocity
 * solves in order.  Returns SSG_MAXITER (after finishing the step) when a
 * solve reached the reference's cap of 5000 iterations. */
ssg_status ssg_navier_stokes_step(ssg_context *ctx, const double *f,
		const double *bc_u, const double *bc_dudt, ssg_solve_info *info);

/* The Stokes operators of the step, element by element without a DSS, on
 * the same fields as the step (its scratch: not while a step runs):
 *   SSG_STOKES_DOUBLE_CURL: out (3 fields) = double_curl_operator(in)
 *     (src/stokes.c:94-105: the mass times curl curl of in, 3 fields);
 *   SSG_STOKES_PRESSURE_RHS: out (1 field) = -dens/dt times
 *     discrete_divergence_operator(in) (src/stokes.c:52-69) plus, on the
 *     wall faces, add_surface_integral of the three fields g
 *     (src/navier_stokes.c:132-141);
 *   SSG_STOKES_VELOCITY_RHS: out (3 fields) = the mass times in / (dt visc)
 *     minus (discrete_gradient_operator(g) plus, on the faces without a
 *     wall, add_surface_integral of g, one field) / (visc dens)
 *     (src/navier_stokes.c:180-196). */
enum {
	SSG_STOKES_DOUBLE_CURL = 0,
	SSG_STOKES_PRESSURE_RHS = 1,
	SSG_STOKES_VELOCITY_RHS = 2
};
ssg_status ssg_stokes_operator(ssg_context *ctx, int which, const double *in,
		const double *g, double *out);

/* ---- launch-shape autotuner (no reference counterpart) ---------------------- */

/* Time every candidate launch shape of the operator (elements per block),
 * the DSS (blocks per SM) and the vector kernels (blocks per SM) on this
 * context's mesh and levels, reps launches per trial (<= 0: 10), and keep
 * the fastest for every later launch in the process (keyed by order n).
 * Results are unchanged: every shape computes the same sums in the same
 * order. */
ssg_status ssg_autotune(ssg_context *ctx, int reps);
/* Device time of the level-0 element operator (var: Poisson or Helmholtz,
 * FP64) in microseconds per apply, on a deterministic pseudo-random field:
 * reps launches back to back on the context's stream between two CUDA
 * events, best of three trials. */
ssg_status ssg_time_operator(ssg_context *ctx, int var, int reps,
		double *us_per_apply);
/* Device time of the three kernels of one smoother CG iteration at a
 * multigrid level, FP64, in microseconds per launch, each timed alone as
 * in ssg_time_operator (no reference counterpart: a measurement aid):
 * us[0] the element operator, us[1] the DSS with the p.(Ap) partial sums,
 * us[2] the CG update (x, r, z and four partial sums). */
ssg_status ssg_time_smoother(ssg_context *ctx, int level, int reps, double *us);
/* Launch shapes in use for order n (tuned or default); elements per block
 * 0 = the FP64 tensor-core operator (n = 8: one warp per element), -1 = the
 * line-form operator (each thread contracts whole element lines), 1, 2, 4,
 * ... = the plane-form operator with that many elements per block. */
ssg_status ssg_tuning(int n, int *ax_elements_per_block,
		int *dss_blocks_per_sm, int *vector_blocks_per_sm);

/* ---- serving loop (no reference counterpart) ------------------------------- */

/* Independent solve requests of different meshes and orders, admitted in
 * arrival order by an HBM budget and run concurrently (continuous batching:
 * up to max_active at once, each on its own stream, new ones starting as
 * slots and memory free up).  Meshes, factors and Krylov workspaces stay
 * resident between requests of the same mesh_key. */
typedef struct ssg_server ssg_server;

typedef struct {
	int nel;                  /* mesh: elements, vertices (nel x 3 x 8), */
	const double *vertices;   /* neighbour table (nel x 26), copied at */
	const int *neigh;         /* submission */
	unsigned long long mesh_key;  /* caller's identity of the mesh; 0 = none */
	int n;                    /* GLL points per direction (N + 1), 2..12 */
	double lambda;            /* Helmholtz coefficient; 0 = Poisson */
	double eps;               /* stopping tolerance on sqrt((r.r)_w) */
	int relative;             /* 1: eps relative to sqrt((f.f)_w) */
	int precision;            /* SSG_PRECISION_FP64 / _MIXED (Poisson V-cycle) */
	int max_iter;             /* <= 0: 5000 */
	double deadline_ms;       /* <= 0: none; counted from submission */
} ssg_request;

typedef struct {
	unsigned long long submitted, completed, failed, cancelled, rejected;
	double p50_ms, p99_ms, mean_ms, max_ms;  /* submission -> result */
	double queue_p50_ms, queue_p99_ms;       /* submission -> start */
	double solves_per_s;      /* completed / (last result - first submission) */
	size_t hbm_in_use, hbm_peak, hbm_budget;
	unsigned long long mesh_hits, mesh_misses, evictions;
	int max_active_seen, resident_contexts;
	/* shared-launch batches run, and the requests they held */
	unsigned long long batches, batched_requests;
} ssg_server_stats;

/* GLL points and quadrature weights of n points on [-1, 1] (gll_basis,
 * src/basis.c:31-177); host only. */
ssg_status ssg_gll(int n, double *points, double *weights);
/* Admission estimate of a request's resident context (bytes); host only. */
size_t ssg_request_bytes(int n, int nel, int precision);
ssg_status ssg_server_create(int device, size_t hbm_budget, int max_active,
		ssg_server **out);
/* Shared launches across requests (off by default, max_batch 1): a small
 * Helmholtz request (at most max_points points, absolute eps) at the head of
 * the queue runs together with the small Helmholtz requests of the same
 * order queued directly behind it, up to max_batch in all, as one
 * ssg_solve_helmholtz_segments on their concatenated meshes -- one operator
 * and one DSS launch per iteration for all of them, each with its own
 * lambda, CG scalars and stop.  The requests' resident contexts provide the
 * data (copied device to device into one concatenated level); a request
 * whose mesh has no idle resident context yet runs alone.  Results agree
 * with the solo solve to rounding (not bitwise).  Each worker keeps a batch
 * arena of up to max_batch * max_points points (about 170 bytes a point),
 * outside the HBM budget. */
ssg_status ssg_server_set_batching(ssg_server *srv, int max_batch,
		size_t max_points);
/* rhs (host, nel x n^3, an assembled weak right-hand side) is copied at
 * submission; the solution is written to `solution` (host) before the
 * request completes.  Initial guess zero. */
ssg_status ssg_server_submit(ssg_server *srv, const ssg_request *req,
		const double *rhs, double *solution, unsigned long long *id);
/* Block until request id is done (timeout_ms < 0: no limit; else
 * SSG_ERR_TIMEOUT when it is not done in time).  *result is the request's
 * own status: SSG_OK, SSG_MAXITER, SSG_ERR_BUDGET (larger than the whole
 * budget), SSG_ERR_CANCELLED, SSG_ERR_TIMEOUT (deadline), ... */
ssg_status ssg_server_wait(ssg_server *srv, unsigned long long id,
		double timeout_ms, ssg_status *result, ssg_solve_info *info);
ssg_status ssg_server_cancel(ssg_server *srv, unsigned long long id);
/* Block until the queue is empty and nothing runs. */
ssg_status ssg_server_drain(ssg_server *srv, double timeout_ms);
ssg_status ssg_server_get_stats(ssg_server *srv, ssg_server_stats *out);
/* Cancels queued requests, waits for running ones, frees every context. */
void ssg_server_destroy(ssg_server *srv);

/* ---- instrumentation -------------------------------------------------------- */

/* Number of this library's kernel launches in the process so far (all
 * contexts). */
unsigned long long ssg_kernel_launch_count(void);

/* ---- particles -------------------------------------------------------------- */

/* Reference-domain velocity snapshots the particles see (sel->ur and its two
 * older levels, src/structs.h:96,116): ur is 3 levels (t-2dt, t-dt, t) x 3
 * components x nel x n^3. */
ssg_status ssg_set_particle_velocity(ssg_context *ctx, const double *ur);
/* integrate_particle_equations at one rank (src/particles.c:182-218):
 * advance every particle to time t, walking across element faces.
 *   state: np x {x, y, z, u, v, w, t, tau} (reference coordinates and
 *          reference-domain velocity, particle time, response time)
 *   ints:  np x {el, old_el, status}; on return status 0 = done,
 *          5 = needs a reseed (the reference draws a random position).
 * dt is the flow time step (struct parameters dt). */
ssg_status ssg_integrate_particle_equations(ssg_context *ctx, size_t np,
		double *state, int *ints, double t, double dt, int *passes);

#ifdef __cplusplus
}
#endif

#endif
