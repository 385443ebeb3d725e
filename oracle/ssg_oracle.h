/*
 * CPU restatement of the SSENSS per-timestep solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA path is checked
 * against; the product never links, loads or calls it.  Each function cites
 * the reference file:line it restates.  The restatement is pinned against the
 * reference compiled in place (oracle/_ref) by tests/test_oracle_vs_ref.py and
 * against the committed fixtures in tests/golden/.
 *
 * Layout: every field is an element-local L-vector u[e][k][j][i], i fastest,
 * nel * n^3 doubles (src/utils.c:64-81); n = points per direction (N+1).
 */
#ifndef SSG_ORACLE_H
#define SSG_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct og_ctx og_ctx;

/* ---- 1-D GLL data (src/basis.c) ---- */
void og_gll(int n, double *x, double *w);
/* D[i*n + m] = dl_m/dx (x_i) */
void og_deriv(int n, const double *x, double *D);
/* spectral-vanishing-viscosity variant (src/deriv.c:81-112), same layout */
void og_svv_deriv(int n, const double *x, const double *w, int msvv,
		double c, double *S);
/* J[i*nfrom + p] = l_p^{from}(xto_i) (src/interpolation.c:115-123) */
void og_interp(int nto, const double *xto, int nfrom, const double *xfrom,
		double *J);

/* ---- setup (src/main.c:53-79, src/precon.c:121-183,336-413) ---- */
/* SVV cut-off mode and amplitude of the contexts created next (svvn < 0:
 * 2n/3; the reference's defaults are 2n/3 and 0, src/main.c:54-55) */
void og_set_svv(int svvn, double svva);
og_ctx *og_create(int n, int nel, const double *vertices, const int *neigh,
		double dt, double visc, double dens);
void og_destroy(og_ctx *c);
void og_set_params(og_ctx *c, double t, double dt, double visc);
int og_nlevels(const og_ctx *c);
int og_level_n(const og_ctx *c, int level);
int og_conv_n(const og_ctx *c);
/* comp 0..5 = G11,G12,G13,G22,G23,G33, 6 = det J, 7..9 = grid x,y,z,
 * 10..18 = J[a][b] = dx_a/dr_b, 19..27 = tinv[a][b] = dr_b/dx_a */
void og_level_geometry(const og_ctx *c, int level, int comp, double *dst);
/* which 0 = Poisson diag inverse, 1 = Helmholtz diag inverse,
 * 2 = 1/multiplicity, 3 = Dirichlet mask, 4 = inverse assembled mass */
void og_level_precon(const og_ctx *c, int level, int which, double *dst);
/* DSS pairing of `level`'s connectivity: for every element 26 pairs
 * (neighbour element, matched face/edge/corner index), -1 where none
 * (src/init.c:68-130). */
void og_dss_pairs(const og_ctx *c, int *pairs);
/* conv-grid factors: comp 0..8 = tinv[a][b], 9 = det J */
void og_conv_geometry(const og_ctx *c, int comp, double *dst);

/* ---- operators (src/poisson.c, src/helmholtz.c, src/global.c) ---- */
void og_local_opeval(og_ctx *c, int level, int var, const double *p,
		double *ap);
void og_global_opeval(og_ctx *c, int level, int var, const double *p,
		double *ap);
void og_dss(og_ctx *c, int level, double *u);
double og_dot(og_ctx *c, int level, const double *x, const double *y);
/* conditioning probe: later og_dot results are scaled by (1 + rel * xi),
 * xi uniform in [-1, 1) from a generator seeded with seed; rel = 0 off */
void og_set_dot_perturbation(og_ctx *c, double rel, unsigned long long seed);

/* ---- solvers (src/solver.c, src/precon.c) ---- */
int og_solve_poisson(og_ctx *c, const double *f, double *u, double eps,
		int max_iter, double *hist, int cap);
int og_solve_helmholtz(og_ctx *c, int var, const double *f, double *u,
		double eps, int max_iter, double *hist, int cap);
void og_mg_precon(og_ctx *c, const double *r, double *z, double eps);

/* ---- dealiased convection (src/convection.c:31-140) ---- */
/* u, v, out: 3 x nel x n^3 (component-major) */
void og_convection(og_ctx *c, const double *u, const double *v, double *out);

/* ---- Lagrangian particles (src/particles.c:182-546) ---- */
/* ur: 3 history levels (t-2dt, t-dt, t) x 3 components x nel x n^3.
 * state: np x {x,y,z,u,v,w,t,tau}; ints: np x {el, old_el, status}.
 * Returns the number of walk passes. */
/* particle walk on the caller's GLL points and level-0 jac / tinv
 * (9 x nel x n^3 each), e.g. the reference's own */
void og_set_particle_basis(og_ctx *c, const double *points, const double *jac,
		const double *tinv);
int og_particles_advance(og_ctx *c, size_t np, double *state, int *ints,
		const double *ur);
double og_point_interp(int n, const double *x, const double *f, double xp,
		double yp, double zp);

#ifdef __cplusplus
}
#endif

#endif
