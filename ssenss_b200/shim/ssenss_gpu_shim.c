/*
 * ssenss_gpu_shim.c -- binds the SSENSS C host to libssenss_b200.
 *
 * This file is what a maintainer adds to the reference's sources.  It
 * defines the reference's own solve-path functions with their own names and
 * signatures and runs each of them on the GPU through the C ABI of
 * include/ssenss_b200.h:
 *
 *   solve_poisson_cg, solve_helmholtz_cg, conjugate_gradient,
 *   flexible_conjugate_gradient, global_opeval      (src/solver.h:24-34)
 *   direct_stiffness_summation, global_dot_product   (src/global.h:25-27)
 *   global_inverse_mass_matrix_operator              (src/poisson.h)
 *   jacobi_preconditioner, multigrid_preconditioner  (src/precon.h:47-50)
 *   convection_operator                              (src/convection.h:22-23)
 *   integrate_convection_rk4                         (src/time.h)
 *   integrate_navier_stokes                          (src/navier_stokes.h)
 *   integrate_particle_equations                     (src/particles.h:71)
 *
 * The reference's definitions of those names are renamed at build time
 * (-D<name>=host_<name> on the files that define them, and on solver.c and
 * precon.c, whose own CPU Krylov and multigrid code then keeps calling the
 * reference's versions).  Set-up stays the reference's: read_grid,
 * connect_elements and initialise_preconditioners run as before, and
 * ssenss_gpu_attach() then hands their results -- neighbour ids, stored
 * bases, derivative and interpolation matrices, geometric factors of every
 * multigrid level, the dealiasing grid and the particle walk's factors -- to
 * the library, so the GPU works on exactly the reference's numbers.
 *
 * Fields stay where the host keeps them (host memory, new_4d_array blocks);
 * each call copies its operands to the device and its result back.  Per
 * element state reached through variable_array() is gathered into one
 * contiguous buffer first, as the reference's own solve_*_cg do.
 *
 * Errors: the reference has no status codes; this file reports every
 * library failure through the reference's fatal_error (src/utils.c:162-174).
 * An iteration cap reached is silent, as in the reference, and recorded in
 * ssenss_gpu_last_solve().  One rank only; one context per process.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "structs.h"
#include "utils.h"
#include "basis.h"
#include "geometry.h"
#include "tripalg.h"
#include "precon.h"
#include "poisson.h"
#include "helmholtz.h"
#include "solver.h"
#include "global.h"
#include "convection.h"
#include "particles.h"
#include "time.h"
#include "navier_stokes.h"

#include "ssenss_b200.h"
#include "ssenss_gpu_shim.h"

#define SHIM_MAX_ITER 5000          /* the reference's cap, src/solver.c:168,184 */
#define SHIM_HISTORY_CAP (SHIM_MAX_ITER + 1)

static ssg_context *G;
static int G_n, G_nel, G_device;
static size_t G_nt;                 /* n^3 */
static double *G_u;                 /* nel n^3: gathered solution / guess */
static double *G_conv;              /* 9 n^3: one element's convection operands */
static double *G_rk;                /* 12 x npts: velocity history and the field of
                                     * integrate_convection_rk4 */
static double *G_flow;              /* 39 x npts: the state of integrate_navier_stokes */
static double G_hist[SHIM_HISTORY_CAP];
static struct ssenss_gpu_solve G_last;

static void fail(const char *what, ssg_status s)
{
	char msg[160];
	snprintf(msg, sizeof(msg), "ssenss_b200 %s: %s (%s)", what,
			ssg_status_string(s), G ? ssg_last_error(G) : "no context");
	fatal_error(msg);
}

static void check(ssg_status s, const char *what)
{
	if (s != SSG_OK)
		fail(what, s);
}

static void need(const char *what)
{
	if (!G) {
		char msg[96];
		snprintf(msg, sizeof(msg), "%s before ssenss_gpu_attach", what);
		fatal_error(msg);
	}
}

/* The calls this file replaces act on the finest level only: the library
 * holds the coarser levels itself. */
static void need_level0(struct element **sel, const char *what)
{
	need(what);
	if ((*sel)->basis->n != G_n || (*sel)->precon->level != 0
			|| (*sel)->nel != G_nel) {
		char msg[96];
		snprintf(msg, sizeof(msg), "%s on a level other than the finest",
				what);
		fatal_error(msg);
	}
}

static double *alloc_doubles(size_t count)
{
	double *p = malloc(count * sizeof(double));
	if (!p)
		fatal_error("ssenss_b200 shim: host allocation");
	return p;
}

/* ---- set-up ----------------------------------------------------------- */

static void gather_field(double *dst, struct element **sel, int level,
		double ***(*get)(struct geometry *, int), int which, size_t nt)
{
	for (int e = 0; e < (*sel)->nel; ++e) {
		struct geometry *g = level < 0 ? sel[e]->conv_geom
				: sel[e]->precon->geom[level];
		memcpy(dst + (size_t) e * nt, **get(g, which),
				nt * sizeof(double));
	}
}

/* geom_mat G11 G12 G13 G22 G23 G33 (src/geometry.c:130-135), det J,
 * jac[a][b], tinv_jac[a][b] */
static double ***geom_field(struct geometry *g, int which)
{
	switch (which) {
	case 0: return g->geom_mat->x.x;
	case 1: return g->geom_mat->x.y;
	case 2: return g->geom_mat->x.z;
	case 3: return g->geom_mat->y.y;
	case 4: return g->geom_mat->y.z;
	case 5: return g->geom_mat->z.z;
	case 6: return g->jac_det;
	default:
		if (which >= 10 && which < 19)
			return *g->jac->ind[(which - 10) / 3][(which - 10) % 3];
		return *g->tinv_jac->ind[(which - 19) / 3][(which - 19) % 3];
	}
}

int ssenss_gpu_attach(struct element **sel, int device)
{
	if (G)
		ssenss_gpu_detach();
	const struct parameters *prm = (*sel)->params;
	const struct preconditioner *pc = (*sel)->precon;
	const int nel = (*sel)->nel;
	if (prm->nproc != 1 || nel != prm->neltot)
		fatal_error("ssenss_b200 binds a single rank");

	/* neighbour ids: faces, edges, corners; negative = wall code */
	int *neigh = malloc(sizeof(int) * 26 * (size_t) nel);
	if (!neigh)
		fatal_error("ssenss_b200 shim: host allocation");
	for (int e = 0; e < nel; ++e) {
		const struct geometry *g = sel[e]->geom;
		int *nb = neigh + 26 * (size_t) e;
		for (int f = 0; f < 6; ++f)
			nb[f] = g->neigh_el[f];
		for (int q = 0; q < 12; ++q)
			nb[6 + q] = g->neigh_edge_el[q];
		for (int c = 0; c < 8; ++c)
			nb[18 + c] = g->neigh_corn_el[c];
	}

	check(ssg_create(device, &G), "create");
	G_device = device;
	check(ssg_set_parameters(G, prm->dt, prm->visc, prm->dens), "parameters");
	check(ssg_setup_connectivity(G, nel, neigh), "connectivity");
	free(neigh);

	for (int l = 0; l < pc->nlevels; ++l) {
		const int m = pc->nmg[l];
		const size_t mt = (size_t) m * m * m, mp = mt * nel;
		const struct basis *b = pc->basis[2 * l];
		double *geom = alloc_doubles(7 * mp);
		for (int a = 0; a < 7; ++a)
			gather_field(geom + a * mp, sel, l, geom_field, a, mt);
		const double *interp = l ? *pc->basis[2 * l - 1]->interp_matrix
				: NULL;
		check(ssg_setup_level(G, l, m, *b->deriv_matrix,
				*b->svv_deriv_matrix, b->weights, geom,
				geom + 6 * mp, interp), "level");
		free(geom);
	}
	check(ssg_setup_finish(G), "finish");

	/* dealiasing grid of convection_operator (src/convection.c:37-69) */
	const struct basis *cb = (*sel)->conv_basis;
	const int m = cb->n;
	const size_t mt = (size_t) m * m * m, mp = mt * nel;
	double *conv = alloc_doubles(10 * mp);
	for (int a = 0; a < 9; ++a)
		gather_field(conv + a * mp, sel, -1, geom_field, 19 + a, mt);
	gather_field(conv + 9 * mp, sel, -1, geom_field, 6, mt);
	check(ssg_setup_dealias(G, m, *cb->deriv_matrix, cb->weights, conv,
			conv + 9 * mp, *cb->interp_matrix), "dealias");
	free(conv);

	/* the particle walk's level-0 points and factors (src/particles.c:
	 * 493-539) */
	G_n = (*sel)->basis->n;
	G_nel = nel;
	G_nt = (size_t) G_n * G_n * G_n;
	const size_t np = G_nt * nel;
	double *pf = alloc_doubles(18 * np);
	for (int a = 0; a < 18; ++a)
		gather_field(pf + a * np, sel, 0, geom_field, 10 + a, G_nt);
	check(ssg_setup_particle_geometry(G, (*sel)->basis->points, pf,
			pf + 9 * np), "particle geometry");
	free(pf);

	G_u = alloc_doubles(9 * np > 9 * G_nt ? 9 * np : 9 * G_nt);
	G_conv = alloc_doubles(9 * G_nt);
	G_rk = alloc_doubles(12 * np);
	memset(&G_last, 0, sizeof(G_last));
	G_last.history = G_hist;
	return 0;
}

void ssenss_gpu_detach(void)
{
	if (G)
		ssg_destroy(G);
	G = NULL;
	free(G_u);
	free(G_conv);
	free(G_rk);
	free(G_flow);
	G_u = G_conv = G_rk = G_flow = NULL;
}

const struct ssenss_gpu_solve *ssenss_gpu_last_solve(void)
{
	return &G_last;
}

/* ---- solves (src/solver.c:33-189) ------------------------------------- */

static void gather_variable(struct element **sel, int var)
{
	for (int e = 0; e < G_nel; ++e)
		memcpy(G_u + (size_t) e * G_nt, **variable_array(sel[e], var),
				G_nt * sizeof(double));
}

static void scatter_variable(struct element **sel, int var)
{
	for (int e = 0; e < G_nel; ++e)
		memcpy(**variable_array(sel[e], var), G_u + (size_t) e * G_nt,
				G_nt * sizeof(double));
}

static void record(int kind, int var, double eps, ssg_status s,
		const ssg_solve_info *info)
{
	G_last.kind = kind;
	G_last.var = var;
	G_last.status = s;
	G_last.eps = eps;
	G_last.iterations = info->iterations;
	G_last.residual = info->residual;
	G_last.solve_ms = info->solve_ms;
	G_last.history_len = info->history_len < SHIM_HISTORY_CAP
			? info->history_len : SHIM_HISTORY_CAP;
	G_last.history = G_hist;
}

static ssg_solve_info new_info(void)
{
	ssg_solve_info info;
	memset(&info, 0, sizeof(info));
	info.history = G_hist;
	info.history_cap = SHIM_HISTORY_CAP;
	return info;
}

/* the Helmholtz coefficient lambda = (11/6) / (dt visc) follows the host's
 * current parameters (src/helmholtz.c:37-38) */
static void sync_parameters(struct element **sel)
{
	const struct parameters *prm = (*sel)->params;
	check(ssg_set_parameters(G, prm->dt, prm->visc, prm->dens),
			"parameters");
}

static ssg_status solve_status(ssg_status s, const char *what)
{
	if (s != SSG_OK && s != SSG_MAXITER)
		fail(what, s);
	return s;
}

void solve_poisson_cg(struct element **sel, double ****f, int var, double eps)
{
	need_level0(sel, "solve_poisson_cg");
	if (var != PRESSURE)
		fatal_error("ssenss_b200: solve_poisson_cg solves for the pressure");
	gather_variable(sel, var);
	ssg_solve_info info = new_info();
	ssg_status s = solve_status(ssg_solve_poisson_cg(G, ***f, G_u, eps,
			SHIM_MAX_ITER, &info), "solve_poisson_cg");
	record(0, var, eps, s, &info);
	scatter_variable(sel, var);
}

void solve_helmholtz_cg(struct element **sel, double ****f, int var,
		double eps)
{
	need_level0(sel, "solve_helmholtz_cg");
	if (var == PRESSURE)
		fatal_error("ssenss_b200: solve_helmholtz_cg solves for a velocity");
	sync_parameters(sel);
	gather_variable(sel, var);
	ssg_solve_info info = new_info();
	ssg_status s = solve_status(ssg_solve_helmholtz_cg(G, var, ***f, G_u,
			eps, SHIM_MAX_ITER, &info), "solve_helmholtz_cg");
	record(1, var, eps, s, &info);
	scatter_variable(sel, var);
}

/* The operator a call names must be the one var implies: the Laplacian for
 * the pressure, the Helmholtz operator for a velocity (the only pairings
 * the reference makes, src/solver.c:159-189). */
static void check_operator(int var, void (*opeval) (), const char *what)
{
	const int laplace = opeval == (void (*)()) discrete_laplace_operator;
	const int helmholtz = opeval == (void (*)()) discrete_helmholtz_operator;
	if ((var == PRESSURE && !laplace) || (var != PRESSURE && !helmholtz)) {
		char msg[96];
		snprintf(msg, sizeof(msg), "%s: operator does not match var", what);
		fatal_error(msg);
	}
}

double conjugate_gradient(struct element **sel, double ****f, double ****u,
		int var, void (*opeval) (), void (*precon) (), double eps,
		int max_iter)
{
	need_level0(sel, "conjugate_gradient");
	check_operator(var, opeval, "conjugate_gradient");
	if (precon != (void (*)()) jacobi_preconditioner)
		fatal_error("ssenss_b200: conjugate_gradient runs with the Jacobi preconditioner");
	sync_parameters(sel);
	ssg_solve_info info = new_info();
	ssg_status s = solve_status(ssg_conjugate_gradient(G, var, ***f, ***u,
			eps, max_iter, &info), "conjugate_gradient");
	record(2, var, eps, s, &info);
	return info.residual;
}

double flexible_conjugate_gradient(struct element **sel, double ****f,
		double ****u, int var, void (*opeval) (), void (*precon) (),
		double eps, int max_iter)
{
	need_level0(sel, "flexible_conjugate_gradient");
	check_operator(var, opeval, "flexible_conjugate_gradient");
	if (var != PRESSURE
			|| precon != (void (*)()) multigrid_preconditioner)
		fatal_error("ssenss_b200: flexible_conjugate_gradient runs the pressure with p-multigrid");
	ssg_solve_info info = new_info();
	ssg_status s = solve_status(ssg_solve_poisson_cg(G, ***f, ***u, eps,
			max_iter, &info), "flexible_conjugate_gradient");
	record(0, var, eps, s, &info);
	return info.residual;
}

void global_opeval(struct element **sel, double ****p, double ****ap, int var,
		void (*opeval) ())
{
	need_level0(sel, "global_opeval");
	check_operator(var, opeval, "global_opeval");
	if (var != PRESSURE)
		sync_parameters(sel);
	check(ssg_global_opeval(G, var, ***p, ***ap), "global_opeval");
}

/* ---- DSS, inner product, mass (src/global.c:241-282, src/poisson.c) --- */

void direct_stiffness_summation(struct element **sel, double ****u)
{
	need_level0(sel, "direct_stiffness_summation");
	check(ssg_direct_stiffness_summation(G, ***u),
			"direct_stiffness_summation");
}

double global_dot_product(struct element **sel, double ****x, double ****y)
{
	double r = 0.0;
	need_level0(sel, "global_dot_product");
	check(ssg_global_dot_product(G, ***x, ***y, &r), "global_dot_product");
	return r;
}

void global_inverse_mass_matrix_operator(struct element **sel, double ****u,
		double ****mu)
{
	need_level0(sel, "global_inverse_mass_matrix_operator");
	if (mu != u)
		memcpy(***mu, ***u, G_nt * G_nel * sizeof(double));
	check(ssg_inverse_mass(G, ***mu), "global_inverse_mass_matrix_operator");
}

/* ---- preconditioners (src/precon.c:227-236, 311-315) ------------------- */

void jacobi_preconditioner(struct element **sel, double ****x, double ****px,
		int var, double eps, void (*opeval) ())
{
	(void) eps;
	(void) opeval;
	need_level0(sel, "jacobi_preconditioner");
	if (var != PRESSURE)
		sync_parameters(sel);
	check(ssg_jacobi_preconditioner(G, var, ***x, ***px),
			"jacobi_preconditioner");
}

void multigrid_preconditioner(struct element **sel, double ****x,
		double ****px, int var, double eps, void (*opeval) ())
{
	(void) opeval;
	need_level0(sel, "multigrid_preconditioner");
	if (var != PRESSURE)
		fatal_error("ssenss_b200: multigrid_preconditioner serves the pressure");
	check(ssg_multigrid_preconditioner(G, ***x, ***px, eps),
			"multigrid_preconditioner");
}

/* ---- convection (src/convection.c:31-35) ------------------------------ */

/* One element per call, as the reference's callers make them
 * (src/time.c:115-117); a host that can gather its fields should call
 * ssg_convection_operator once for the whole mesh instead. */
void convection_operator(struct element *sel, struct trivec *u,
		struct trivec *v, struct trivec *udv)
{
	need("convection_operator");
	const int e = sel->geom->id;
	if (sel->basis->n != G_n || e < 0 || e >= G_nel)
		fatal_error("ssenss_b200: convection_operator on an unknown element");
	/* the velocity advecting itself (u == v, the step's history term,
	 * src/navier_stokes.c:79-83): one staged field, which the library runs
	 * on its self-convection kernel */
	const double *gv = u == v ? G_conv : G_conv + 3 * G_nt;
	for (int c = 0; c < 3; ++c) {
		memcpy(G_conv + c * G_nt, ***u->ind[c], G_nt * sizeof(double));
		if (u != v)
			memcpy(G_conv + (3 + c) * G_nt, ***v->ind[c],
					G_nt * sizeof(double));
	}
	check(ssg_convection_elements(G, e, 1, G_conv, gv, G_conv + 6 * G_nt),
			"convection_operator");
	for (int c = 0; c < 3; ++c)
		memcpy(***udv->ind[c], G_conv + (6 + c) * G_nt,
				G_nt * sizeof(double));
}

/* ---- convection sub-steps (src/time.c:84-130) --------------------------- */

/* trivec fields of every element into / out of one contiguous buffer,
 * component-major, elements by their global id */
static void gather_trivec(double *dst, struct element **sel, struct trivec **v,
		struct trivec *(*pick)(struct element *))
{
	const size_t np = G_nt * G_nel;
	for (int i = 0; i < G_nel; ++i) {
		const int e = sel[i]->geom->id;
		struct trivec *t = v ? v[i] : pick(sel[i]);
		for (int c = 0; c < 3; ++c)
			memcpy(dst + c * np + e * G_nt, ***t->ind[c],
					G_nt * sizeof(double));
	}
}

static struct trivec *vel_now(struct element *s) { return s->u; }
static struct trivec *vel_old(struct element *s) { return s->old->u; }
static struct trivec *vel_oldold(struct element *s) { return s->old->old->u; }

/* The whole mesh's convection sub-steps in one library call: the velocity
 * history and u go to the device once, the 8 stages of the two RK4
 * sub-steps run there, u comes back. */
void integrate_convection_rk4(struct element **sel, struct trivec **u,
		double t0, double t, double dt, double beta)
{
	need("integrate_convection_rk4");
	if ((*sel)->nel != G_nel || (*sel)->basis->n != G_n)
		fatal_error("ssenss_b200: integrate_convection_rk4 on another mesh");
	const size_t np = G_nt * G_nel;
	double *h = G_rk, *f = G_rk + 9 * np;
	gather_trivec(h, sel, NULL, vel_now);
	gather_trivec(h + 3 * np, sel, NULL, vel_old);
	gather_trivec(h + 6 * np, sel, NULL, vel_oldold);
	check(ssg_set_velocity_history(G, h, h + 3 * np, h + 6 * np,
			(*sel)->params->t, (*sel)->params->dt),
			"integrate_convection_rk4 (history)");
	gather_trivec(f, sel, u, NULL);
	check(ssg_integrate_convection_rk4(G, f, t0, t, dt, beta),
			"integrate_convection_rk4");
	for (int i = 0; i < G_nel; ++i) {
		const int e = sel[i]->geom->id;
		for (int c = 0; c < 3; ++c)
			memcpy(***u[i]->ind[c], f + c * np + e * G_nt,
					G_nt * sizeof(double));
	}
}

/* ---- the whole time step (src/navier_stokes.c:224-235) ------------------ */

static int G_device_step = 1;
static struct ssenss_gpu_solve G_step[4];
static double G_step_hist[4][SHIM_HISTORY_CAP];
static int G_step_len;

void ssenss_gpu_device_step(int on)
{
	G_device_step = on;
}

int ssenss_gpu_step_solves(const struct ssenss_gpu_solve **solves)
{
	*solves = G_step;
	return G_step_len;
}

/* the state of history level l (0 = now, 1 = old, 2 = old->old) */
struct level_state {
	struct trivec *u, *conv, *rot;
	double ***p;
};

static struct level_state level_state(struct element *s, int l)
{
	struct level_state r = { s->u, s->conv, s->rot, s->p };
	struct old_element *o = s->old;
	for (int k = 0; k < l; ++k) {
		r.u = o->u;
		r.conv = o->conv;
		r.rot = o->rot;
		r.p = o->p;
		o = o->old;
	}
	return r;
}

/* one trivec per element into / out of dst, component-major */
static void move_trivec(double *buf, struct trivec *t, int e, int out)
{
	const size_t np = G_nt * G_nel;
	for (int c = 0; c < 3; ++c) {
		double *d = buf + c * np + (size_t) e * G_nt;
		if (out)
			memcpy(***t->ind[c], d, G_nt * sizeof(double));
		else
			memcpy(d, ***t->ind[c], G_nt * sizeof(double));
	}
}

/* staging layout: per level u, conv, rot (3 fields each), p (1 field);
 * then f, the wall values of u and of du/dt (3 fields each) */
static void flow_fields(ssg_flow_fields *ff)
{
	const size_t np = G_nt * G_nel;
	for (int l = 0; l < 3; ++l) {
		double *b = G_flow + (size_t) l * 10 * np;
		ff->u[l] = b;
		ff->conv[l] = b + 3 * np;
		ff->rot[l] = b + 6 * np;
		ff->p[l] = b + 9 * np;
	}
	ff->f = G_flow + 30 * np;
}

static void move_state(struct element **sel, int out)
{
	ssg_flow_fields ff;
	flow_fields(&ff);
	for (int i = 0; i < G_nel; ++i) {
		const int e = sel[i]->geom->id;
		for (int l = 0; l < 3; ++l) {
			struct level_state st = level_state(sel[i], l);
			move_trivec(ff.u[l], st.u, e, out);
			move_trivec(ff.conv[l], st.conv, e, out);
			move_trivec(ff.rot[l], st.rot, e, out);
			double *d = ff.p[l] + (size_t) e * G_nt;
			if (out)
				memcpy(**st.p, d, G_nt * sizeof(double));
			else
				memcpy(d, **st.p, G_nt * sizeof(double));
		}
		if (!out)
			move_trivec(ff.f, sel[i]->f, e, 0);
	}
}

/* bc_func and bc_dfunc of every element at t + dt on its wall nodes, as
 * set_dirichlet_boundaries evaluates them (src/poisson.c:101-143) */
static void wall_values(struct element **sel, double *bu, double *bd)
{
	const size_t np = G_nt * G_nel;
	const int n = G_n, m = n - 1;
	memset(bu, 0, 3 * np * sizeof(double));
	memset(bd, 0, 3 * np * sizeof(double));
	for (int i = 0; i < G_nel; ++i) {
		const struct element *s = sel[i];
		const int bc = s->bc, e = s->geom->id;
		if (!bc)
			continue;
		const double t = s->params->t + s->params->dt;
		const double *x = **s->geom->grid->x;
		const double *y = **s->geom->grid->y;
		const double *z = **s->geom->grid->z;
		for (size_t q = 0; q < G_nt; ++q) {
			const int a = q % n, b = (q / n) % n, k = q / (n * n);
			const int wall = ((bc & DIRICHLET_W) && a == 0)
					|| ((bc & DIRICHLET_E) && a == m)
					|| ((bc & DIRICHLET_S) && b == 0)
					|| ((bc & DIRICHLET_N) && b == m)
					|| ((bc & DIRICHLET_B) && k == 0)
					|| ((bc & DIRICHLET_T) && k == m);
			if (!wall)
				continue;
			for (int c = 0; c < 3; ++c) {
				const size_t g = c * np + (size_t) e * G_nt + q;
				bu[g] = s->bc_func[c](x[q], y[q], z[q], t);
				bd[g] = s->bc_dfunc[c](x[q], y[q], z[q], t);
			}
		}
	}
}

/* The whole step on the device: the state goes to the library, one
 * ssg_navier_stokes_step runs the convection history and sub-steps, the
 * pressure and velocity right-hand sides, extrapolations and the four
 * solves there, and the state comes back.  With the device step switched
 * off (ssenss_gpu_device_step(0)) the reference's own integrate_navier_
 * stokes runs, its solves and convection calls through this binding. */
void integrate_navier_stokes(struct element **sel)
{
	G_step_len = 0;
	if (!G_device_step) {
		host_integrate_navier_stokes(sel);
		return;
	}
	need_level0(sel, "integrate_navier_stokes");
	sync_parameters(sel);
	const size_t np = G_nt * G_nel;
	if (!G_flow)
		G_flow = alloc_doubles(39 * np);
	move_state(sel, 0);
	ssg_flow_fields ff;
	flow_fields(&ff);
	check(ssg_flow_set(G, &ff, (*sel)->params->t), "integrate_navier_stokes (state)");
	double *bu = G_flow + 33 * np, *bd = G_flow + 36 * np;
	wall_values(sel, bu, bd);
	ssg_solve_info info[4];
	for (int k = 0; k < 4; ++k) {
		info[k] = new_info();
		info[k].history = G_step_hist[k];
	}
	ssg_status st = solve_status(ssg_navier_stokes_step(G, ff.f, bu, bd, info),
			"integrate_navier_stokes");
	ff.f = NULL;
	check(ssg_flow_get(G, &ff, NULL), "integrate_navier_stokes (state)");
	move_state(sel, 1);
	for (int k = 0; k < 4; ++k) {
		struct ssenss_gpu_solve *r = &G_step[k];
		r->kind = k ? 1 : 0;
		r->var = k ? X_VELOCITY + k - 1 : PRESSURE;
		r->status = st;
		r->iterations = info[k].iterations;
		r->eps = 0.0;
		r->residual = info[k].residual;
		r->solve_ms = info[k].solve_ms;
		r->history_len = info[k].history_len;
		r->history = G_step_hist[k];
	}
	G_step_len = 4;
	(*sel)->params->t += (*sel)->params->dt;
}

/* ---- particles (src/particles.c:182-218) ------------------------------ */

void integrate_particle_equations(struct plist *p, struct element **sel)
{
	need_level0(sel, "integrate_particle_equations");
	const size_t np = p->n, nf = G_nt * G_nel;
	/* the reference-domain velocity at t - 2dt, t - dt, t */
	for (int e = 0; e < G_nel; ++e) {
		struct trivec *lev[3] = { sel[e]->old->old->ur, sel[e]->old->ur,
				sel[e]->ur };
		for (int l = 0; l < 3; ++l)
			for (int c = 0; c < 3; ++c)
				memcpy(G_u + (size_t) (3 * l + c) * nf
						+ (size_t) e * G_nt,
						***lev[l]->ind[c],
						G_nt * sizeof(double));
	}
	check(ssg_set_particle_velocity(G, G_u), "particle velocity");

	double *state = alloc_doubles(8 * (np ? np : 1));
	int *ints = malloc(sizeof(int) * 3 * (np ? np : 1));
	if (!ints)
		fatal_error("ssenss_b200 shim: host allocation");
	for (size_t i = 0; i < np; ++i) {
		const struct particle *q = &p->list[i];
		double *s = state + 8 * i;
		s[0] = q->x; s[1] = q->y; s[2] = q->z;
		s[3] = q->u; s[4] = q->v; s[5] = q->w;
		s[6] = q->t; s[7] = q->tau;
		ints[3 * i] = q->el;
		ints[3 * i + 1] = q->old_el;
		ints[3 * i + 2] = 0;
	}
	int passes = 0;
	const double t = (*sel)->params->t;
	check(ssg_integrate_particle_equations(G, np, state, ints, t,
			(*sel)->params->dt, &passes), "integrate_particle_equations");
	for (size_t i = 0; i < np; ++i) {
		struct particle *q = &p->list[i];
		const double *s = state + 8 * i;
		q->x = s[0]; q->y = s[1]; q->z = s[2];
		q->u = s[3]; q->v = s[4]; q->w = s[5];
		q->t = s[6]; q->tau = s[7];
		q->el = ints[3 * i];
		q->old_el = ints[3 * i + 1];
		q->status = 0;          /* P_NORMAL */
		if (ints[3 * i + 2] == 5) {
			/* the walk did not settle within the reference's pass
			 * limit: draw a new position, as the reference does
			 * (src/particles.c:192-198) */
			initialise_particle_position(q, sel[q->el]);
			q->t = t;
			printf("Particle %d reinitialised\n", (int) q->id);
		}
	}
	free(state);
	free(ints);
}
