/*
 * Harness around the unmodified SSENSS sources (test infrastructure, built
 * into oracle/_ref/libssenss_ref.so).  It sets the solver up the way
 * src/main.c:36-90 does, but from an in-memory mesh, and exposes flat-array
 * entry points for Python (ctypes) to call: operator apply, DSS, weighted dot,
 * the Poisson/Helmholtz solves with their residual histories, one p-multigrid
 * application, dealiased convection, particle advance and the Navier-Stokes
 * step.  The reference is not re-entrant (src/precon.c:273-281), so all state
 * lives in file-scope variables and one mesh is set up at a time.
 *
 * Residual histories: the build renames global_dot_product in src/global.c to
 * ssgref_dot_impl and every caller's reference to ssgref_dot_hook; likewise
 * multigrid_preconditioner (src/precon.c) becomes ssgref_mg_impl behind
 * ssgref_mg_hook.  The hook records sqrt(x.x) for calls with x == y made
 * outside the preconditioner, which in conjugate_gradient and
 * flexible_conjugate_gradient (src/solver.c:72-73,151-152) is exactly the
 * residual check; the nullspace norm (x == y == ones, src/solver.c:207) is
 * filtered out.
 *
 * Built a second time with SSGREF_GPU_SHIM defined, into
 * oracle/_ref/libssenss_ref_gpu.so: the same reference sources with the
 * solve path taken by the library's C-ABI binding
 * (ssenss_b200/shim/ssenss_gpu_shim.c), attached right after
 * initialise_preconditioners as a host would attach it.  Histories then come
 * from the binding's record of each solve.
 *
 * Navier-Stokes steps: src/navier_stokes.c is compiled with its calls to
 * solve_poisson_cg / solve_helmholtz_cg renamed to ssgref_step_poisson /
 * ssgref_step_helmholtz, which log every solve of a step (kind, variable,
 * residual history) and then call the real solve.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "structs.h"
#include "utils.h"
#include "linalg.h"
#include "tripalg.h"
#include "basis.h"
#include "geometry.h"
#include "interpolation.h"
#include "deriv.h"
#include "init.h"
#include "final.h"
#include "poisson.h"
#include "helmholtz.h"
#include "global.h"
#include "solver.h"
#include "precon.h"
#include "convection.h"
#include "navier_stokes.h"
#include "particles.h"
#include "stokes.h"
#include "time.h"
#include "test.h"
#include "synth_dataio.h"
#ifdef SSGREF_GPU_SHIM
#include "ssenss_gpu_shim.h"
#endif

double ssgref_dot_impl(struct element **sel, double ****x, double ****y);
void ssgref_mg_impl(struct element **sel, double ****x, double ****px,
		int var, double eps, void (*opeval) ());

static struct parameters *H_params;
static struct communicator *H_comm;
static struct basis *H_gll;
static struct basis *H_conv;
static struct geometry **H_geom;
static struct geometry **H_cgeom;
static struct element **H_sel;
static int H_nel;
static int H_n;

static int H_recording;
static int H_precon_depth;
static double *H_hist;
static int H_hist_cap;
static int H_hist_len;

static int all_ones(double ****x, size_t len)
{
	const double *p = ***x;
	return p[0] == 1.0 && p[len / 2] == 1.0 && p[len - 1] == 1.0;
}

double ssgref_dot_hook(struct element **sel, double ****x, double ****y)
{
	const double v = ssgref_dot_impl(sel, x, y);
	const size_t len = (size_t) (*sel)->basis->ntot * (size_t) (*sel)->nel;
	if (H_recording && H_precon_depth == 0 && x == y && !all_ones(x, len)) {
		if (H_hist_len < H_hist_cap)
			H_hist[H_hist_len] = sqrt(v);
		++H_hist_len;
	}
	return v;
}

void ssgref_mg_hook(struct element **sel, double ****x, double ****px,
		int var, double eps, void (*opeval) ())
{
	++H_precon_depth;
	ssgref_mg_impl(sel, x, px, var, eps, opeval);
	--H_precon_depth;
}

static size_t npts(void)
{
	return (size_t) H_nel * (size_t) H_n * H_n * H_n;
}

/* Copy a flat L-vector into a fresh 4-D array (src/utils.c:64-81 layout). */
static double ****from_flat(const double *src)
{
	double ****a = new_4d_array(H_n, H_n, H_n, H_nel);
	memcpy(***a, src, npts() * sizeof(double));
	return a;
}

void ssgref_teardown(void)
{
	if (!H_sel)
		return;
#ifdef SSGREF_GPU_SHIM
	ssenss_gpu_detach();
#endif
	free_basis(H_gll);
	free_basis(H_conv);
	disconnect_elements(H_sel);
	free_elements(H_sel);
	free_communicator(H_comm);
	free_geometries(H_geom);
	free_geometries(H_cgeom);
	free_parameters(H_params);
	H_sel = NULL;
}

/* SVV parameters of the next set-up (src/main.c:54-55 fixes 2n/3 and 0) */
static int H_svvn = -1;
static double H_svva = 0.0;

void ssgref_set_svv(int svvn, double svva)
{
	H_svvn = svvn;
	H_svva = svva;
}

/* Set the solver up as src/main.c:36-90 does (minus files and particles). */
int ssgref_setup(int n, int nel, const double *vertices, const int *neigh,
		double dt, double visc, double dens)
{
	ssgref_teardown();
	ssgref_mesh.nel = nel;
	ssgref_mesh.vertices = vertices;
	ssgref_mesh.neigh = neigh;
	ssgref_mesh.init_velocity = NULL;

	H_comm = new_communicator(0, 1, MPI_COMM_WORLD, MPI_INFO_NULL);
	H_params = new_parameters(0, 1);
	H_params->n = n;
	H_params->dt = dt;
	H_params->visc = visc;
	H_params->dens = dens;
	H_params->nconv = (3 * n) / 2;
	H_params->svvn = H_svvn >= 0 ? H_svvn : 2 * n / 3;
	H_params->svva = H_svva;
	get_grid_size(H_params, H_comm, "");

	H_gll = new_gll_basis(n);
	H_conv = new_gll_basis(H_params->nconv);
	create_interpolation_matrices(H_gll, H_conv);
	compute_svv_derivative_matrix(H_gll, H_params->svvn, H_params->svva);

	H_geom = new_geometries(H_gll, H_params->nel, H_params->neltot);
	H_cgeom = new_geometries(H_conv, H_params->nel, H_params->neltot);
	read_grid(H_geom, H_comm, H_gll, "");
	read_grid(H_cgeom, H_comm, H_conv, "");

	H_sel = new_elements(H_geom, H_cgeom, H_gll, H_conv, H_params, H_comm);
	connect_elements(H_sel);
	initialise_preconditioners(H_sel);
#ifdef SSGREF_GPU_SHIM
	ssenss_gpu_attach(H_sel, 0);
#endif
	H_nel = nel;
	H_n = n;
	return (*H_sel)->precon->nlevels;
}

void ssgref_set_time(double t, double dt, double visc)
{
	H_params->t = t;
	H_params->dt = dt;
	H_params->visc = visc;
}

/* ---- discretisation data, exported for the oracle and for parity ---- */

int ssgref_level_order(int level)
{
	return (*H_sel)->precon->nmg[level];
}

int ssgref_conv_order(void)
{
	return H_params->nconv;
}

/* GLL points, weights and the stored derivative matrices d[j][i] = D_ij
 * of level `level` (src/basis.c:160-177, src/deriv.c:81-104). */
void ssgref_level_basis(int level, double *points, double *weights,
		double *deriv, double *svv_deriv)
{
	struct basis *b = (*H_sel)->precon->basis[2 * level];
	const int m = b->n;
	memcpy(points, b->points, m * sizeof(double));
	memcpy(weights, b->weights, m * sizeof(double));
	memcpy(deriv, *b->deriv_matrix, (size_t) m * m * sizeof(double));
	memcpy(svv_deriv, *b->svv_deriv_matrix, (size_t) m * m * sizeof(double));
}

/* Interpolation matrix between levels level-1 (fine) and level (coarse):
 * interp[p][i] = l_p^coarse(xi_i^fine), stored on the fine duplicate basis
 * (src/precon.c:130-137, src/interpolation.c:115-134). */
void ssgref_level_interp(int level, double *interp)
{
	struct basis *b = (*H_sel)->precon->basis[2 * level - 1];
	const int nf = b->n;
	const int nc = (*H_sel)->precon->nmg[level];
	memcpy(interp, *b->interp_matrix, (size_t) nf * nc * sizeof(double));
}

static void put_field(double *dst, double ***(*get)(struct element *, int),
		int level, int which)
{
	(void) level;
	const int m = (*H_sel)->basis->n;
	const size_t nt = (size_t) m * m * m;
	for (int e = 0; e < H_nel; ++e)
		memcpy(dst + e * nt, **get(H_sel[e], which), nt * sizeof(double));
}

static double ***geom_component(struct element *s, int which)
{
	struct geometry *g = s->geom;
	switch (which) {
	case 0: return g->geom_mat->x.x;
	case 1: return g->geom_mat->x.y;
	case 2: return g->geom_mat->x.z;
	case 3: return g->geom_mat->y.y;
	case 4: return g->geom_mat->y.z;
	case 5: return g->geom_mat->z.z;
	case 6: return g->jac_det;
	case 7: return g->grid->x;
	case 8: return g->grid->y;
	case 9: return g->grid->z;
	default:
		if (which >= 10 && which < 19)
			return *g->jac->ind[(which - 10) / 3][(which - 10) % 3];
		if (which >= 19 && which < 28)
			return *g->tinv_jac->ind[(which - 19) / 3][(which - 19) % 3];
		return (double ***) NULL;
	}
}

static void switch_level(int level)
{
	for (int e = 0; e < H_nel; ++e) {
		H_sel[e]->precon->level = level;
		H_sel[e]->basis = H_sel[e]->precon->basis[2 * level];
		H_sel[e]->geom = H_sel[e]->precon->geom[level];
	}
}

/* Geometric factors of a level: comp 0..5 = G11,G12,G13,G22,G23,G33,
 * 6 = det J, 7..9 = x,y,z of the GLL grid, 10..18 = jac[a][b] = dx_a/dr_b,
 * 19..27 = tinv_jac[a][b] (level 0: the factors the particle walk reads,
 * src/particles.c:517-539). */
void ssgref_level_geometry(int level, int comp, double *dst)
{
	switch_level(level);
	put_field(dst, geom_component, level, comp);
	switch_level(0);
}

/* Overwrite a level-0 factor the particle walk reads (comp 10..27 as
 * above), so that a particle test can run the reference on factors it
 * also hands to another implementation bit for bit. */
void ssgref_set_level0_factor(int comp, const double *src)
{
	if (comp < 10 || comp >= 28)
		return;
	const int m = (*H_sel)->basis->n;
	const size_t nt = (size_t) m * m * m;
	for (int e = 0; e < H_nel; ++e)
		memcpy(**geom_component(H_sel[e], comp), src + e * nt,
				nt * sizeof(double));
}

/* Per-level preconditioner arrays, contiguous over elements:
 * which 0 = Poisson diagonal inverse, 1 = Helmholtz diagonal inverse,
 * 2 = stiffness-summation scale 1/multiplicity, 3 = Dirichlet mask,
 * 4 = inverse assembled mass (level 0 only). */
void ssgref_level_precon(int level, int which, double *dst)
{
	struct preconditioner *pc = (*H_sel)->precon;
	const int m = pc->nmg[level];
	const size_t len = (size_t) H_nel * m * m * m;
	const double *src = NULL;
	switch (which) {
	case 0: src = **pc->poisson_diag[level]; break;
	case 1: src = **pc->helmholtz_diag[level]; break;
	case 2: src = **pc->stiffsum_scale[level]; break;
	case 3: src = **pc->dirichlet_mask[level]; break;
	case 4: src = **pc->inverse_mass; break;
	}
	memcpy(dst, src, len * sizeof(double));
}

/* Conversion-grid (dealiasing) factors: comp 0..8 = tinv_jac row-major
 * [a][b] after the final transpose (src/geometry.c:102-113), 9 = det J. */
void ssgref_conv_geometry(int comp, double *dst)
{
	const int m = H_params->nconv;
	const size_t nt = (size_t) m * m * m;
	for (int e = 0; e < H_nel; ++e) {
		struct geometry *g = H_sel[e]->conv_geom;
		double ***src = comp < 9 ? *g->tinv_jac->ind[comp / 3][comp % 3]
				: g->jac_det;
		memcpy(dst + e * nt, **src, nt * sizeof(double));
	}
}

void ssgref_conv_basis(double *points, double *weights, double *interp)
{
	const int m = H_conv->n;
	memcpy(points, H_conv->points, m * sizeof(double));
	memcpy(weights, H_conv->weights, m * sizeof(double));
	memcpy(interp, *H_conv->interp_matrix, (size_t) m * H_n * sizeof(double));
}

/* ---- operators ---- */

void ssgref_global_opeval(int var, const double *p, double *ap)
{
	double ****P = from_flat(p);
	double ****AP = new_4d_array(H_n, H_n, H_n, H_nel);
	void (*op)() = var == PRESSURE ? (void (*)()) discrete_laplace_operator
			: (void (*)()) discrete_helmholtz_operator;
	global_opeval(H_sel, P, AP, var, op);
	memcpy(ap, ***AP, npts() * sizeof(double));
	free_4d_array(P);
	free_4d_array(AP);
}

/* Element-local operator only (no mask, no DSS). */
void ssgref_local_opeval(int var, const double *p, double *ap)
{
	double ****P = from_flat(p);
	double ****AP = new_4d_array(H_n, H_n, H_n, H_nel);
	for (int e = 0; e < H_nel; ++e) {
		if (var == PRESSURE)
			discrete_laplace_operator(H_sel[e], P[e], AP[e]);
		else
			discrete_helmholtz_operator(H_sel[e], P[e], AP[e]);
	}
	memcpy(ap, ***AP, npts() * sizeof(double));
	free_4d_array(P);
	free_4d_array(AP);
}

void ssgref_dss(double *u)
{
	double ****U = from_flat(u);
	direct_stiffness_summation(H_sel, U);
	memcpy(u, ***U, npts() * sizeof(double));
	free_4d_array(U);
}

/* DSS at a coarser level (order of that level, nel * m^3 values). */
void ssgref_dss_level(int level, double *u)
{
	const int m = (*H_sel)->precon->nmg[level];
	switch_level(level);
	double ****U = new_4d_array(m, m, m, H_nel);
	memcpy(***U, u, (size_t) H_nel * m * m * m * sizeof(double));
	direct_stiffness_summation(H_sel, U);
	memcpy(u, ***U, (size_t) H_nel * m * m * m * sizeof(double));
	free_4d_array(U);
	switch_level(0);
}

double ssgref_dot(const double *x, const double *y)
{
	double ****X = from_flat(x);
	double ****Y = from_flat(y);
	double v = ssgref_dot_impl(H_sel, X, Y);
	free_4d_array(X);
	free_4d_array(Y);
	return v;
}

/* ---- solves (src/solver.c:159-189) ---- */

static void begin_record(double *hist, int cap)
{
	H_hist = hist;
	H_hist_cap = cap;
	H_hist_len = 0;
	H_recording = 1;
}

static int end_record(void)
{
	H_recording = 0;
#ifdef SSGREF_GPU_SHIM
	/* the binding's record of the solve just run */
	const struct ssenss_gpu_solve *g = ssenss_gpu_last_solve();
	H_hist_len = g->history_len;
	memcpy(H_hist, g->history, (size_t) (H_hist_len < H_hist_cap
			? H_hist_len : H_hist_cap) * sizeof(double));
#endif
	return H_hist_len;
}

/* ---- per-solve log of Navier-Stokes steps ---- */

struct step_solve {
	int kind;      /* 0 Poisson, 1 Helmholtz */
	int var;
	int len;
	double *hist;
};
static struct step_solve *H_steplog;
static int H_steplog_len, H_steplog_cap;

static void step_record(int kind, int var, const double *hist, int len)
{
	if (H_steplog_len == H_steplog_cap) {
		H_steplog_cap = H_steplog_cap ? 2 * H_steplog_cap : 64;
		H_steplog = realloc(H_steplog, H_steplog_cap * sizeof(*H_steplog));
	}
	struct step_solve *r = &H_steplog[H_steplog_len++];
	r->kind = kind;
	r->var = var;
	r->len = len;
	r->hist = malloc((len ? len : 1) * sizeof(double));
	memcpy(r->hist, hist, (size_t) len * sizeof(double));
}

void ssgref_step_log_clear(void)
{
	for (int i = 0; i < H_steplog_len; ++i)
		free(H_steplog[i].hist);
	H_steplog_len = 0;
}

int ssgref_step_log_count(void)
{
	return H_steplog_len;
}

/* Solve i of the log: kind, var and up to cap history values; returns the
 * history length. */
int ssgref_step_log_entry(int i, int *kind, int *var, double *hist, int cap)
{
	if (i < 0 || i >= H_steplog_len)
		return -1;
	const struct step_solve *r = &H_steplog[i];
	*kind = r->kind;
	*var = r->var;
	memcpy(hist, r->hist, (size_t) (r->len < cap ? r->len : cap)
			* sizeof(double));
	return r->len;
}

static double H_step_hist[5001];

void ssgref_step_poisson(struct element **sel, double ****f, int var,
		double eps)
{
	begin_record(H_step_hist, 5001);
	solve_poisson_cg(sel, f, var, eps);
	const int len = end_record();
	step_record(0, var, H_step_hist, len < 5001 ? len : 5001);
}

void ssgref_step_helmholtz(struct element **sel, double ****f, int var,
		double eps)
{
	begin_record(H_step_hist, 5001);
	solve_helmholtz_cg(sel, f, var, eps);
	const int len = end_record();
	step_record(1, var, H_step_hist, len < 5001 ? len : 5001);
}

/* Poisson: var = PRESSURE, initial guess in u (overwritten by the result). */
int ssgref_solve_poisson(const double *f, double *u, double eps,
		double *hist, int cap)
{
	double ****F = from_flat(f);
	for (int e = 0; e < H_nel; ++e)
		memcpy(**H_sel[e]->p, u + e * (size_t) H_n * H_n * H_n,
				(size_t) H_n * H_n * H_n * sizeof(double));
	begin_record(hist, cap);
	solve_poisson_cg(H_sel, F, PRESSURE, eps);
	const int it = end_record();
	for (int e = 0; e < H_nel; ++e)
		memcpy(u + e * (size_t) H_n * H_n * H_n, **H_sel[e]->p,
				(size_t) H_n * H_n * H_n * sizeof(double));
	free_4d_array(F);
	return it;
}

/* Helmholtz: var = X/Y/Z_VELOCITY (mask applies on walls). */
int ssgref_solve_helmholtz(int var, const double *f, double *u, double eps,
		double *hist, int cap)
{
	double ****F = from_flat(f);
	const size_t nt = (size_t) H_n * H_n * H_n;
	for (int e = 0; e < H_nel; ++e)
		memcpy(**variable_array(H_sel[e], var), u + e * nt,
				nt * sizeof(double));
	begin_record(hist, cap);
	solve_helmholtz_cg(H_sel, F, var, eps);
	const int it = end_record();
	for (int e = 0; e < H_nel; ++e)
		memcpy(u + e * nt, **variable_array(H_sel[e], var),
				nt * sizeof(double));
	free_4d_array(F);
	return it;
}

/* Raw Krylov calls with an iteration cap (returns the final residual). */
double ssgref_fcg_mg(const double *f, double *u, double eps, int max_iter)
{
	double ****F = from_flat(f);
	double ****U = from_flat(u);
#ifdef SSGREF_GPU_SHIM
	void (*mg)() = (void (*)()) multigrid_preconditioner;
#else
	void (*mg)() = (void (*)()) ssgref_mg_hook;
#endif
	double err = flexible_conjugate_gradient(H_sel, F, U, PRESSURE,
			discrete_laplace_operator, mg, eps, max_iter);
	memcpy(u, ***U, npts() * sizeof(double));
	free_4d_array(F);
	free_4d_array(U);
	return err;
}

double ssgref_cg_jacobi(int var, const double *f, double *u, double eps,
		int max_iter)
{
	double ****F = from_flat(f);
	double ****U = from_flat(u);
	void (*op)() = var == PRESSURE ? (void (*)()) discrete_laplace_operator
			: (void (*)()) discrete_helmholtz_operator;
	double err = conjugate_gradient(H_sel, F, U, var, op,
			jacobi_preconditioner, eps, max_iter);
	memcpy(u, ***U, npts() * sizeof(double));
	free_4d_array(F);
	free_4d_array(U);
	return err;
}

/* One application of the p-multigrid preconditioner z = M^-1 r
 * (src/precon.c:227-236). */
void ssgref_mg_precon(const double *r, double *z, double eps)
{
	double ****R = from_flat(r);
	double ****Z = new_4d_array(H_n, H_n, H_n, H_nel);
	ssgref_mg_hook(H_sel, R, Z, PRESSURE, eps,
			(void (*)()) discrete_laplace_operator);
	memcpy(z, ***Z, npts() * sizeof(double));
	free_4d_array(R);
	free_4d_array(Z);
}

/* ---- dealiased convection (src/convection.c:31-69) ---- */

static void trivec_in(struct trivec *t, const double *src, int e)
{
	const size_t nt = (size_t) H_n * H_n * H_n;
	for (int c = 0; c < 3; ++c)
		memcpy(***t->ind[c], src + ((size_t) c * H_nel + e) * nt,
				nt * sizeof(double));
}

static void trivec_out(struct trivec *t, double *dst, int e)
{
	const size_t nt = (size_t) H_n * H_n * H_n;
	for (int c = 0; c < 3; ++c)
		memcpy(dst + ((size_t) c * H_nel + e) * nt, ***t->ind[c],
				nt * sizeof(double));
}

/* u, v, out: 3 x nel x n^3 (component-major). */
void ssgref_convection(const double *u, const double *v, double *out)
{
	struct trivec *tu = new_trivec(H_n);
	struct trivec *tv = new_trivec(H_n);
	struct trivec *to = new_trivec(H_n);
	for (int e = 0; e < H_nel; ++e) {
		trivec_in(tu, u, e);
		trivec_in(tv, v, e);
		convection_operator(H_sel[e], tu, tv, to);
		trivec_out(to, out, e);
	}
	free_trivec(tu);
	free_trivec(tv);
	free_trivec(to);
}

/* integrate_convection_rk4 (src/time.c:84-130) on u (3 x nel x n^3,
 * in/out) with the velocity history set by ssgref_set_field and the time
 * by ssgref_set_time; in the build linked with the binding the call is the
 * binding's (the library's device sub-steps). */
void ssgref_integrate_convection_rk4(double *u, double t0, double t, double dt,
		double beta)
{
	struct trivec **tu = new_ptr_array(H_nel, H_n,
			(void *(*) ()) new_trivec);
	for (int e = 0; e < H_nel; ++e)
		trivec_in(tu[e], u, e);
	integrate_convection_rk4(H_sel, tu, t0, t, dt, beta);
	for (int e = 0; e < H_nel; ++e)
		trivec_out(tu[e], u, e);
	free_ptr_array(tu, H_nel, free_trivec);
}

/* The Stokes operators of a time step on flat fields, element by element
 * with the reference's functions (no DSS):
 * which 0: out (3 fields) = double_curl_operator(in) (src/stokes.c:94-105);
 * which 1: out (1 field) = discrete_divergence_operator(in) scaled by
 *   -dens/dt, plus add_surface_integral of g (3 fields) on the wall faces,
 *   the steps of compute_pressure_rhs (src/navier_stokes.c:132-141);
 * which 2: out (3 fields) = the steps of compute_velocity_rhs
 *   (src/navier_stokes.c:180-196) on in = u~ and g = p (1 field). */
void ssgref_stokes_operator(int which, const double *in, const double *g,
		double *out)
{
	static const int deriv[3] = { X_DERIV, Y_DERIV, Z_DERIV };
	const size_t nt = (size_t) H_n * H_n * H_n;
	struct trivec *ti = new_trivec(H_n);
	struct trivec *tg = new_trivec(H_n);
	struct trivec *to = new_trivec(H_n);
	double ***p = new_3d_array(H_n, H_n, H_n);
	for (int e = 0; e < H_nel; ++e) {
		struct element *s = H_sel[e];
		trivec_in(ti, in, e);
		if (which == 0) {
			double_curl_operator(s, ti, to);
			trivec_out(to, out, e);
		} else if (which == 1) {
			trivec_in(tg, g, e);
			discrete_divergence_operator(s, ti, p);
			scale_array(**p, s->ntot, -s->params->dens / s->params->dt);
			for (int j = 0; j < 3; ++j)
				add_surface_integral(s, *tg->ind[j], p, deriv[j],
						~s->bc);
			memcpy(out + e * nt, **p, nt * sizeof(double));
		} else {
			memcpy(**p, g + e * nt, nt * sizeof(double));
			scale_trivec(ti, s->ntot, 1.0 / (s->params->dt
					* s->params->visc));
			discrete_gradient_operator(s, p, tg);
			for (int j = 0; j < 3; ++j) {
				test_function_inner_product(s, *ti->ind[j],
						*to->ind[j]);
				add_surface_integral(s, p, *tg->ind[j], deriv[j],
						s->bc);
				add_array(***tg->ind[j], ***to->ind[j], s->ntot,
						-1.0 / (s->params->visc
						* s->params->dens));
			}
			trivec_out(to, out, e);
		}
	}
	free_3d_array(p);
	free_trivec(ti);
	free_trivec(tg);
	free_trivec(to);
}

/* ---- Navier-Stokes step on the Taylor-Green vortex ---- */

static double tgv_u(double x, double y, double z, double t)
{
	(void) t;
	return sin(x) * cos(y) * cos(z);
}

static double tgv_v(double x, double y, double z, double t)
{
	(void) t;
	return -cos(x) * sin(y) * cos(z);
}

static double tgv_w(double x, double y, double z, double t)
{
	(void) x;
	(void) y;
	(void) z;
	(void) t;
	return 0.0;
}

static double tgv_p(double x, double y, double z)
{
	return (cos(2.0 * x) + cos(2.0 * y)) * (cos(2.0 * z) + 2.0) / 16.0;
}

/* Initial condition as src/poisson.c:245-273 sets it from functions, pressure
 * in all three history levels, then the reference-domain velocity
 * (src/main.c:84). */
void ssgref_init_tgv(void)
{
	initialise_from_function(H_sel, tgv_u, tgv_v, tgv_w);
	const size_t nt = (size_t) H_n * H_n * H_n;
	for (int e = 0; e < H_nel; ++e) {
		struct element *s = H_sel[e];
		const double *x = **s->geom->grid->x;
		const double *y = **s->geom->grid->y;
		const double *z = **s->geom->grid->z;
		for (size_t q = 0; q < nt; ++q) {
			const double p = tgv_p(x[q], y[q], z[q]);
			(**s->p)[q] = p;
			(**s->old->p)[q] = p;
			(**s->old->old->p)[q] = p;
		}
	}
	compute_reference_domain_velocity(H_sel);
}

/* The analytic Ethier-Steinman case of the reference's --run-test
 * (src/main.c:82-84): velocity and the time-dependent Dirichlet values of
 * every wall from initialise_test (src/test.c:202-214), pressure left at
 * zero as the reference leaves it without an initial file, then the
 * reference-domain velocity. */
void ssgref_init_ethier_steinman(void)
{
	initialise_test(H_sel);
	compute_reference_domain_velocity(H_sel);
}

/* One step of src/main.c:101-111 without particles and logging. */
void ssgref_ns_step(void)
{
	set_source_term(H_sel, X_SOURCE, one_func, H_params->gx);
	set_source_term(H_sel, Y_SOURCE, one_func, H_params->gy);
	set_source_term(H_sel, Z_SOURCE, one_func, H_params->gz);
	integrate_navier_stokes(H_sel);
#ifdef SSGREF_GPU_SHIM
	/* a step the binding ran on the device: its four solves */
	const struct ssenss_gpu_solve *g;
	const int k = ssenss_gpu_step_solves(&g);
	for (int i = 0; i < k; ++i)
		step_record(g[i].kind, g[i].var, g[i].history,
				g[i].history_len < 5001 ? g[i].history_len : 5001);
#endif
}

#ifdef SSGREF_GPU_SHIM
/* integrate_navier_stokes on the device (1) or the reference's own step
 * with its solves bound to the library (0) */
void ssgref_gpu_device_step(int on)
{
	ssenss_gpu_device_step(on);
}
#endif

double ssgref_time(void)
{
	return H_params->t;
}

/* The field `which` of history level hist_level of element s:
 * 0..2 = u,v,w; 3 = p; 4..6 = reference-domain velocity ur; 7..9 = the
 * convection history conv; 10..12 = the double-curl history rot. */
static double ***state_field(struct element *s, int which, int hist_level)
{
	struct trivec *u = s->u, *ur = s->ur, *cv = s->conv, *rt = s->rot;
	double ***p = s->p;
	if (hist_level >= 1) {
		u = s->old->u; ur = s->old->ur; p = s->old->p;
		cv = s->old->conv; rt = s->old->rot;
	}
	if (hist_level >= 2) {
		u = s->old->old->u; ur = s->old->old->ur;
		p = s->old->old->p;
		cv = s->old->old->conv; rt = s->old->old->rot;
	}
	if (which < 3)
		return *u->ind[which];
	if (which == 3)
		return p;
	if (which < 7)
		return *ur->ind[which - 4];
	if (which < 10)
		return *cv->ind[which - 7];
	return *rt->ind[which - 10];
}

void ssgref_get_field(int which, int hist_level, double *dst)
{
	const size_t nt = (size_t) H_n * H_n * H_n;
	for (int e = 0; e < H_nel; ++e)
		memcpy(dst + e * nt, **state_field(H_sel[e], which, hist_level),
				nt * sizeof(double));
}

void ssgref_set_field(int which, int hist_level, const double *src)
{
	const size_t nt = (size_t) H_n * H_n * H_n;
	for (int e = 0; e < H_nel; ++e)
		memcpy(**state_field(H_sel[e], which, hist_level), src + e * nt,
				nt * sizeof(double));
}

/* ---- particles (src/particles.c:182-218) ---- */

/* Flat particle record exchanged with the caller:
 * x,y,z,u,v,w,t,tau as doubles and el, old_el, status as ints. */
int ssgref_particles_advance(size_t np, double *state /* np x 8 */,
		int *ints /* np x 3 */)
{
	struct plist pl;
	pl.n = np;
	pl.ntot = np;
	pl.nbuff = np + 1;
	pl.ntypes = 1;
	pl.tau = NULL;
	pl.nproc = 1;
	pl.mpi_comm = MPI_COMM_WORLD;
	pl.list = ec_malloc(sizeof(*pl.list) * pl.nbuff);
	for (size_t i = 0; i < np; ++i) {
		struct particle *q = &pl.list[i];
		const double *s = state + 8 * i;
		q->id = i;
		q->type = 0;
		q->x = s[0]; q->y = s[1]; q->z = s[2];
		q->u = s[3]; q->v = s[4]; q->w = s[5];
		q->t = s[6]; q->tau = s[7];
		q->el = ints[3 * i];
		q->old_el = ints[3 * i + 1];
		q->proc = 0;
		q->old_proc = 0;
		q->status = 0; /* P_NORMAL */
	}
	pl.list[np].status = 4; /* P_BUFFER */
	integrate_particle_equations(&pl, H_sel);
	/* particles are re-sorted by status (stable qsort is not guaranteed),
	 * so the id carries each particle back to its slot */
	for (size_t i = 0; i < np; ++i) {
		const struct particle *q = &pl.list[i];
		double *s = state + 8 * q->id;
		s[0] = q->x; s[1] = q->y; s[2] = q->z;
		s[3] = q->u; s[4] = q->v; s[5] = q->w;
		s[6] = q->t; s[7] = q->tau;
		ints[3 * q->id] = q->el;
		ints[3 * q->id + 1] = q->old_el;
		ints[3 * q->id + 2] = q->status;
	}
	free(pl.list);
	return 0;
}
