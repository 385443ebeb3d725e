/*
 * CPU restatement of the SSENSS per-timestep solve path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU baseline load it.  Written from
 * the reference's algorithm, not from its code: each routine names the
 * reference file:line whose arithmetic it follows.  Floating-point sums use
 * the reference's per-point operation order where that order is visible in
 * plain C (pointwise products, the DSS addition order, the particle
 * integrator); where the reference delegates to BLAS (DGEMM/DDOT) the sum
 * runs in natural index order, so those results agree with the reference to
 * rounding, not bitwise.  Compiled with -ffp-contract=off.
 */
#define _DEFAULT_SOURCE
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "ssg_oracle.h"

enum { VAR_PRESSURE = 0 };
enum { ST_NORMAL = 0, ST_COLLISION = 1, ST_OUTSIDE = 2, ST_RESEED = 5 };

#define MAXLEV 8
#define MAXN 18

typedef struct {
	int n;
	double x[MAXN], w[MAXN];
	double D[MAXN * MAXN];    /* D[i*n+m] = l_m'(x_i) */
	double S[MAXN * MAXN];    /* SVV variant, same layout */
} basis1d;

typedef struct {
	int n;
	size_t nt;                /* n^3 */
	basis1d b;
	double *grid[3];
	double *jac[9];           /* J[a][b] = dx_a/dr_b */
	double *tinv[9];          /* tinv[a][b] = dr_b/dx_a */
	double *det;
	double *g[6];             /* G11 G12 G13 G22 G23 G33 */
	double *diag_p, *diag_h, *scale, *mask;
	double jf[MAXN * MAXN];   /* from the finer level: jf[i*nc+p] = l_p^c(x_i^f) */
} level_t;

struct og_ctx {
	int nel;
	int nlev;
	int n;
	int *neigh;               /* nel x 26 */
	int *pairs;               /* nel x 26 x 2 */
	int *bc;                  /* Dirichlet bits per element */
	double dt, visc, dens, t;
	level_t lev[MAXLEV];
	level_t conv;
	double jconv[MAXN * MAXN];  /* jconv[i*n+p] = l_p^n(x_i^m) */
	double *inv_mass;
	/* particle walk: GLL points and level-0 jac / tinv it reads; NULL =
	 * the oracle's own (og_set_particle_basis overrides them) */
	double *ppts, *pjac, *ptinv;
	/* conditioning probe (og_set_dot_perturbation): 0 = off */
	double dot_pert;
	unsigned long long dot_seed;
};

static double *dalloc(size_t n)
{
	return (double *) calloc(n ? n : 1, sizeof(double));
}

/* ------------------------------------------------------------------ */
/* 1-D GLL basis (src/basis.c:31-177)                                 */
/* ------------------------------------------------------------------ */

/* P_N(x) and P_{N-1}(x) by the three-term recurrence. */
static void legendre2(int N, double x, double *pn, double *pnm1)
{
	double p0 = 1.0, p1 = x;
	if (N == 0) {
		*pn = 1.0;
		*pnm1 = 0.0;
		return;
	}
	for (int k = 1; k < N; ++k) {
		const double p2 = ((2.0 * k + 1.0) * x * p1 - k * p0) / (k + 1.0);
		p0 = p1;
		p1 = p2;
	}
	*pn = p1;
	*pnm1 = p0;
}

static double legendre(int N, double x)
{
	double a, b;
	legendre2(N, x, &a, &b);
	return a;
}

/* GLL nodes: x_0 = -1, x_N = 1 and the interior roots of P_N', by Newton on
 * (1-x^2) P_N'(x), whose derivative is -N(N+1) P_N(x) (src/basis.c:123-148),
 * from Chebyshev-Gauss-Lobatto starting guesses; weights
 * 2 / (N(N+1) P_N(x_i)^2) (src/basis.c:150-158). */
void og_gll(int n, double *x, double *w)
{
	const int N = n - 1;
	x[0] = -1.0;
	x[N] = 1.0;
	for (int i = 1; i < N; ++i) {
		double xi = -cos(M_PI * i / N);
		for (int it = 0; it < 100; ++it) {
			double pn, pm;
			legendre2(N, xi, &pn, &pm);
			const double dpn = N * (xi * pn - pm) / (xi * xi - 1.0);
			const double step = (1.0 - xi * xi) * dpn /
					(N * (N + 1.0) * pn);
			xi += step;
			if (fabs(step) < 1e-16)
				break;
		}
		x[i] = xi;
	}
	for (int i = 0; i < n; ++i) {
		const double pn = legendre(N, x[i]);
		w[i] = 2.0 / (N * (N + 1.0) * pn * pn);
	}
}

/* D_im = P_N(x_i) / (P_N(x_m) (x_i - x_m)), corners -+N(N+1)/4
 * (src/basis.c:160-177). */
void og_deriv(int n, const double *x, double *D)
{
	const int N = n - 1;
	for (int i = 0; i < n; ++i)
		for (int m = 0; m < n; ++m)
			D[i * n + m] = i == m ? 0.0 : legendre(N, x[i]) /
					(legendre(N, x[m]) * (x[i] - x[m]));
	D[0] = -(double) n * (double) (n - 1) / 4.0;
	D[n * n - 1] = -D[0];
}

/* S = V diag(sqrt(1 + c Q_r)) F D with the discrete Legendre transform
 * F(r,k) = (r+1/2) w_k P_r(x_k), V(i,r) = P_r(x_i) and the SVV kernel
 * Q_r = exp(-((N-r)/(msvv-r))^2) for r > msvv, else 0
 * (src/deriv.c:81-112, src/basis.c:190-209). */
void og_svv_deriv(int n, const double *x, const double *w, int msvv,
		double c, double *S)
{
	const int N = n - 1;
	double D[MAXN * MAXN], FD[MAXN * MAXN];
	og_deriv(n, x, D);
	for (int r = 0; r < n; ++r) {
		const double q = r <= msvv ? 0.0 :
				exp(-pow((double) (N - r) / (double) (msvv - r), 2));
		const double sig = sqrt(1.0 + c * q);
		for (int col = 0; col < n; ++col) {
			double s = 0.0;
			for (int k = 0; k < n; ++k)
				s += (r + 0.5) * w[k] * legendre(r, x[k]) *
						D[k * n + col];
			FD[r * n + col] = s * sig;
		}
	}
	for (int i = 0; i < n; ++i)
		for (int col = 0; col < n; ++col) {
			double s = 0.0;
			for (int r = 0; r < n; ++r)
				s += legendre(r, x[i]) * FD[r * n + col];
			S[i * n + col] = s;
		}
}

/* Lagrange cardinal function l_p of the `nfrom` nodes at xt, as the running
 * product of src/interpolation.c:31-39. */
static double lagrange(double xt, const double *xf, int p, int nfrom)
{
	double l = 1.0;
	for (int q = 0; q < p; ++q)
		l *= (xt - xf[q]) / (xf[p] - xf[q]);
	for (int q = p + 1; q < nfrom; ++q)
		l *= (xt - xf[q]) / (xf[p] - xf[q]);
	return l;
}

void og_interp(int nto, const double *xto, int nfrom, const double *xfrom,
		double *J)
{
	for (int i = 0; i < nto; ++i)
		for (int p = 0; p < nfrom; ++p)
			J[i * nfrom + p] = lagrange(xto[i], xfrom, p, nfrom);
}

static void make_basis(basis1d *b, int n, int msvv, double csvv)
{
	b->n = n;
	og_gll(n, b->x, b->w);
	og_deriv(n, b->x, b->D);
	og_svv_deriv(n, b->x, b->w, msvv, csvv, b->S);
}

/* ------------------------------------------------------------------ */
/* tensor-product contractions (src/deriv.c:29-66,                     */
/* src/interpolation.c:136-176)                                        */
/* ------------------------------------------------------------------ */

/* out = (Az x Ay x Ax) in, A*[o*ni + q], stages in x, y, z order like
 * interpolate_to_grid. in: ni^3, out: no^3. */
static void tensor3(int ni, int no, const double *A, const double *in,
		double *out)
{
	double *t1 = dalloc((size_t) no * ni * ni);
	double *t2 = dalloc((size_t) no * no * ni);
	for (int k = 0; k < ni; ++k)
		for (int j = 0; j < ni; ++j)
			for (int i = 0; i < no; ++i) {
				double s = 0.0;
				for (int q = 0; q < ni; ++q)
					s += A[i * ni + q] * in[(k * ni + j) * ni + q];
				t1[(k * ni + j) * no + i] = s;
			}
	for (int k = 0; k < ni; ++k)
		for (int j = 0; j < no; ++j)
			for (int i = 0; i < no; ++i) {
				double s = 0.0;
				for (int q = 0; q < ni; ++q)
					s += A[j * ni + q] * t1[(k * ni + q) * no + i];
				t2[(k * no + j) * no + i] = s;
			}
	for (int k = 0; k < no; ++k)
		for (int j = 0; j < no; ++j)
			for (int i = 0; i < no; ++i) {
				double s = 0.0;
				for (int q = 0; q < ni; ++q)
					s += A[k * ni + q] * t2[(q * no + j) * no + i];
				out[(k * no + j) * no + i] = s;
			}
	free(t1);
	free(t2);
}

/* out = (A^T x A^T x A^T) in where A[i*no + p] maps no -> ni, i.e. the
 * weak-form restriction integrate_to_grid (src/interpolation.c:157-176).
 * in: ni^3, out: no^3. */
static void tensor3_t(int ni, int no, const double *A, const double *in,
		double *out)
{
	double *At = dalloc((size_t) no * ni);
	for (int i = 0; i < ni; ++i)
		for (int p = 0; p < no; ++p)
			At[p * ni + i] = A[i * no + p];
	tensor3(ni, no, At, in, out);
	free(At);
}

/* derivative along r, s or t of a block, D[i*n+m] */
static void dx_r(int n, const double *D, const double *u, double *du)
{
	for (int kj = 0; kj < n * n; ++kj)
		for (int i = 0; i < n; ++i) {
			double s = 0.0;
			for (int m = 0; m < n; ++m)
				s += D[i * n + m] * u[kj * n + m];
			du[kj * n + i] = s;
		}
}

static void dx_s(int n, const double *D, const double *u, double *du)
{
	for (int k = 0; k < n; ++k)
		for (int j = 0; j < n; ++j)
			for (int i = 0; i < n; ++i) {
				double s = 0.0;
				for (int m = 0; m < n; ++m)
					s += D[j * n + m] * u[(k * n + m) * n + i];
				du[(k * n + j) * n + i] = s;
			}
}

static void dx_t(int n, const double *D, const double *u, double *du)
{
	for (int k = 0; k < n; ++k)
		for (int ji = 0; ji < n * n; ++ji) {
			double s = 0.0;
			for (int m = 0; m < n; ++m)
				s += D[k * n + m] * u[m * n * n + ji];
			du[k * n * n + ji] = s;
		}
}

/* transposed derivatives: du_i = sum_m D[m*n+i] u_m (src/deriv.c:54-66) */
static void dxt_r(int n, const double *D, const double *u, double *du)
{
	for (int kj = 0; kj < n * n; ++kj)
		for (int i = 0; i < n; ++i) {
			double s = 0.0;
			for (int m = 0; m < n; ++m)
				s += D[m * n + i] * u[kj * n + m];
			du[kj * n + i] = s;
		}
}

static void dxt_s(int n, const double *D, const double *u, double *du)
{
	for (int k = 0; k < n; ++k)
		for (int j = 0; j < n; ++j)
			for (int i = 0; i < n; ++i) {
				double s = 0.0;
				for (int m = 0; m < n; ++m)
					s += D[m * n + j] * u[(k * n + m) * n + i];
				du[(k * n + j) * n + i] = s;
			}
}

static void dxt_t(int n, const double *D, const double *u, double *du)
{
	for (int k = 0; k < n; ++k)
		for (int ji = 0; ji < n * n; ++ji) {
			double s = 0.0;
			for (int m = 0; m < n; ++m)
				s += D[m * n + k] * u[m * n * n + ji];
			du[k * n * n + ji] = s;
		}
}

/* ------------------------------------------------------------------ */
/* geometry (src/geometry.c:102-135, src/tripalg.c:165-234)           */
/* ------------------------------------------------------------------ */

static void alloc_level(level_t *L, int n, int nel)
{
	L->n = n;
	L->nt = (size_t) n * n * n;
	const size_t len = L->nt * nel;
	for (int a = 0; a < 3; ++a)
		L->grid[a] = dalloc(len);
	for (int a = 0; a < 9; ++a) {
		L->jac[a] = dalloc(len);
		L->tinv[a] = dalloc(len);
	}
	for (int a = 0; a < 6; ++a)
		L->g[a] = dalloc(len);
	L->det = dalloc(len);
	L->diag_p = dalloc(len);
	L->diag_h = dalloc(len);
	L->scale = dalloc(len);
	L->mask = dalloc(len);
}

static void free_level(level_t *L)
{
	for (int a = 0; a < 3; ++a)
		free(L->grid[a]);
	for (int a = 0; a < 9; ++a) {
		free(L->jac[a]);
		free(L->tinv[a]);
	}
	for (int a = 0; a < 6; ++a)
		free(L->g[a]);
	free(L->det);
	free(L->diag_p);
	free(L->diag_h);
	free(L->scale);
	free(L->mask);
}

/* Jacobian by differentiating the grid, its determinant by cofactor
 * expansion along the first row, the inverse by cofactors / det
 * (src/tripalg.c:165-222, same per-point operation order), the metric
 * G_ab = sum_j Ji[a][j] Ji[b][j] (src/geometry.c:130-135) and the stored
 * transposed inverse (src/geometry.c:112). */
static void compute_factors(level_t *L, int nel)
{
	const int n = L->n;
	const size_t nt = L->nt;
	for (int e = 0; e < nel; ++e) {
		const size_t o = e * nt;
		for (int a = 0; a < 3; ++a) {
			dx_r(n, L->b.D, L->grid[a] + o, L->jac[3 * a + 0] + o);
			dx_s(n, L->b.D, L->grid[a] + o, L->jac[3 * a + 1] + o);
			dx_t(n, L->b.D, L->grid[a] + o, L->jac[3 * a + 2] + o);
		}
	}
	static const int k0[3] = { 1, 0, 0 }, k1[3] = { 2, 2, 1 },
			k2[3] = { 2, 0, 1 }, k3[3] = { 1, 2, 0 };
	static const double sg[3] = { 1.0, -1.0, 1.0 };
	const size_t len = nt * nel;
	for (size_t q = 0; q < len; ++q) {
		double a[3][3], ai[3][3];
		for (int r = 0; r < 3; ++r)
			for (int c = 0; c < 3; ++c)
				a[r][c] = L->jac[3 * r + c][q];
		double det = 0.0;
		for (int i = 0; i < 3; ++i) {
			const int j = (2 - i) / 2;
			const int k = 3 - i - j;
			double t = a[1][j] * a[2][k];
			t = -(a[1][k] * a[2][j]) + t;
			det = i == 0 ? a[0][i] * t : sg[i] * a[0][i] * t + det;
		}
		L->det[q] = det;
		for (int i = 0; i < 3; ++i)
			for (int j = 0; j < 3; ++j) {
				double t = a[k0[j]][k3[i]] * a[k1[j]][k2[i]];
				t = -(a[k0[j]][k2[i]] * a[k1[j]][k3[i]]) + t;
				ai[i][j] = sg[j] * t / det;
			}
		double g[3][3];
		for (int i = 0; i < 3; ++i)
			for (int l = 0; l < 3; ++l) {
				double s = ai[l][0] * ai[i][0];
				s = ai[l][1] * ai[i][1] + s;
				s = ai[l][2] * ai[i][2] + s;
				g[i][l] = s;
			}
		L->g[0][q] = g[0][0];
		L->g[1][q] = g[1][0];
		L->g[2][q] = g[2][0];
		L->g[3][q] = g[1][1];
		L->g[4][q] = g[2][1];
		L->g[5][q] = g[2][2];
		for (int r = 0; r < 3; ++r)
			for (int c = 0; c < 3; ++c)
				L->tinv[3 * r + c][q] = ai[c][r];
	}
}

/* GLL grid of every element from its 8 trilinear vertices, the n=2 grid
 * record interpolated like copy_grid_from_struct (src/dataio.c:407-452). */
static void grid_from_vertices(level_t *L, int nel, const double *vert)
{
	double xv[2] = { -1.0, 1.0 };
	double J[MAXN * 2];
	og_interp(L->n, L->b.x, 2, xv, J);
	for (int e = 0; e < nel; ++e)
		for (int a = 0; a < 3; ++a)
			tensor3(2, L->n, J, vert + 24 * (size_t) e + 8 * a,
					L->grid[a] + e * L->nt);
}

/* ------------------------------------------------------------------ */
/* DSS pairing and summation (src/init.c:68-130, src/global.c:38-257) */
/* ------------------------------------------------------------------ */

static int face_node(int n, int f, int p)
{
	const int a = p / n, b = p % n, m = n - 1;
	switch (f) {
	case 0: return (a * n + b) * n;
	case 1: return (a * n + b) * n + m;
	case 2: return (a * n + 0) * n + b;
	case 3: return (a * n + m) * n + b;
	case 4: return (0 * n + a) * n + b;
	default: return (m * n + a) * n + b;
	}
}

static int edge_node(int n, int q, int p)
{
	const int m = n - 1;
	switch (q) {
	case 0: return (p * n + 0) * n + 0;
	case 1: return (p * n + 0) * n + m;
	case 2: return (p * n + m) * n + 0;
	case 3: return (p * n + m) * n + m;
	case 4: return (0 * n + p) * n + 0;
	case 5: return (0 * n + p) * n + m;
	case 6: return (m * n + p) * n + 0;
	case 7: return (m * n + p) * n + m;
	case 8: return (0 * n + 0) * n + p;
	case 9: return (0 * n + m) * n + p;
	case 10: return (m * n + 0) * n + p;
	default: return (m * n + m) * n + p;
	}
}

static int corner_node(int n, int c)
{
	const int m = n - 1;
	return ((c / 4) * m * n + ((c / 2) % 2) * m) * n + (c % 2) * m;
}

/* For every face/edge/corner with a neighbour on this rank, the neighbour's
 * matching face/edge/corner is the FIRST of its list that names this element
 * (surfind/edgeind/cornerind first-match, src/init.c:68-130,298-320). */
static void build_pairs(og_ctx *c)
{
	static const int base[3] = { 0, 6, 18 }, cnt[3] = { 6, 12, 8 };
	for (int e = 0; e < c->nel; ++e)
		for (int kind = 0; kind < 3; ++kind)
			for (int j = 0; j < cnt[kind]; ++j) {
				const int slot = base[kind] + j;
				const int nb = c->neigh[26 * e + slot];
				int *pr = c->pairs + 2 * (26 * e + slot);
				pr[0] = -1;
				pr[1] = -1;
				if (nb < 0)
					continue;
				for (int s = 0; s < cnt[kind]; ++s)
					if (c->neigh[26 * nb + base[kind] + s] == e) {
						pr[0] = nb;
						pr[1] = s;
						break;
					}
			}
}

static void dss_level(const og_ctx *c, int level, double *u)
{
	const int n = c->lev[level].n;
	const size_t nt = c->lev[level].nt;
	double *pre = dalloc(nt * c->nel);
	memcpy(pre, u, nt * c->nel * sizeof(double));
	for (int e = 0; e < c->nel; ++e) {
		double *ue = u + e * nt;
		const int *pr = c->pairs + 52 * e;
		for (int f = 0; f < 6; ++f, pr += 2)
			if (pr[0] >= 0)
				for (int p = 0; p < n * n; ++p)
					ue[face_node(n, f, p)] += pre[pr[0] * nt +
							face_node(n, pr[1], p)];
		for (int q = 0; q < 12; ++q, pr += 2)
			if (pr[0] >= 0)
				for (int p = 0; p < n; ++p)
					ue[edge_node(n, q, p)] += pre[pr[0] * nt +
							edge_node(n, pr[1], p)];
		for (int k = 0; k < 8; ++k, pr += 2)
			if (pr[0] >= 0)
				ue[corner_node(n, k)] += pre[pr[0] * nt +
						corner_node(n, pr[1])];
	}
	free(pre);
}

void og_dss(og_ctx *c, int level, double *u)
{
	dss_level(c, level, u);
}

/* sum (x*w)*y, w = 1/multiplicity (src/global.c:270-282) */
double og_dot(og_ctx *c, int level, const double *x, const double *y)
{
	const level_t *L = &c->lev[level];
	const size_t len = L->nt * c->nel;
	double s = 0.0;
	for (size_t q = 0; q < len; ++q)
		s += (x[q] * L->scale[q]) * y[q];
	if (c->dot_pert != 0.0) {
		/* 64-bit LCG (Knuth's MMIX constants); xi uniform in [-1, 1) */
		c->dot_seed = c->dot_seed * 6364136223846793005ULL +
			1442695040888963407ULL;
		const double xi = (double) (c->dot_seed >> 11) *
			(2.0 / 9007199254740992.0) - 1.0;
		s *= 1.0 + c->dot_pert * xi;
	}
	return s;
}

/* Conditioning probe, not part of the reference's algorithm: every later
 * og_dot result is scaled by (1 + rel * xi), xi drawn per call from a
 * seeded generator.  With rel at the size of one rounding (2e-16) the
 * spread of the perturbed solves is how far the solution is determined by
 * the arithmetic at all: any other correct summation order (the
 * reference's BLAS ddot, a parallel reduction) lands inside it. */
void og_set_dot_perturbation(og_ctx *c, double rel, unsigned long long seed)
{
	c->dot_pert = rel;
	c->dot_seed = seed;
}

/* ------------------------------------------------------------------ */
/* local operators (src/poisson.c:34-66, src/helmholtz.c:33-77)       */
/* ------------------------------------------------------------------ */

static double helm_lambda(const og_ctx *c)
{
	return (11.0 / 6.0) / (c->dt * c->visc);
}

/* Laplacian A_e u = D^T (rho J (G . D u)) per element.  The Helmholtz
 * operator swaps only the stored deriv_matrix for the SVV matrix, so its
 * r-derivative and its s/t transposed derivatives use S while the other three
 * use D (src/helmholtz.c:41-44 with src/deriv.c:29-66), then adds
 * lambda * (u rho) J. */
static void local_op(const og_ctx *c, int level, int var, const double *p,
		double *ap)
{
	const level_t *L = &c->lev[level];
	const int n = L->n;
	const size_t nt = L->nt;
	const int helm = var != VAR_PRESSURE;
	const double *Dx = helm ? L->b.S : L->b.D;
	const double *Dyz = L->b.D;
	const double lam = helm_lambda(c);
	double *ur = dalloc(nt), *us = dalloc(nt), *ut = dalloc(nt);
	double *w0 = dalloc(nt), *w1 = dalloc(nt), *w2 = dalloc(nt);
	double *t0 = dalloc(nt);
	for (int e = 0; e < c->nel; ++e) {
		const size_t o = e * nt;
		const double *u = p + o;
		dx_r(n, Dx, u, ur);
		dx_s(n, Dyz, u, us);
		dx_t(n, Dyz, u, ut);
		for (size_t q = 0; q < nt; ++q) {
			const int i = q % n, j = (q / n) % n, k = q / (n * n);
			const double rho = (L->b.w[i] * L->b.w[j]) * L->b.w[k];
			const double J = L->det[o + q];
			const double g00 = L->g[0][o + q], g01 = L->g[1][o + q],
					g02 = L->g[2][o + q], g11 = L->g[3][o + q],
					g12 = L->g[4][o + q], g22 = L->g[5][o + q];
			double a = g00 * ur[q];
			a = g01 * us[q] + a;
			a = g02 * ut[q] + a;
			double b = g01 * ur[q];
			b = g11 * us[q] + b;
			b = g12 * ut[q] + b;
			double d = g02 * ur[q];
			d = g12 * us[q] + d;
			d = g22 * ut[q] + d;
			w0[q] = (a * rho) * J;
			w1[q] = (b * rho) * J;
			w2[q] = (d * rho) * J;
		}
		double *out = ap + o;
		dxt_r(n, Dyz, w0, out);
		dxt_s(n, Dx, w1, t0);
		for (size_t q = 0; q < nt; ++q)
			out[q] += t0[q];
		dxt_t(n, Dx, w2, t0);
		for (size_t q = 0; q < nt; ++q)
			out[q] += t0[q];
		if (helm)
			for (size_t q = 0; q < nt; ++q) {
				const int i = q % n, j = (q / n) % n, k = q / (n * n);
				const double rho = (L->b.w[i] * L->b.w[j]) * L->b.w[k];
				out[q] += lam * ((u[q] * rho) * L->det[o + q]);
			}
	}
	free(ur); free(us); free(ut); free(w0); free(w1); free(w2); free(t0);
}

void og_local_opeval(og_ctx *c, int level, int var, const double *p,
		double *ap)
{
	local_op(c, level, var, p, ap);
}

static void mask_apply(const og_ctx *c, int level, int var, double *u)
{
	if (var == VAR_PRESSURE)
		return;
	const level_t *L = &c->lev[level];
	const size_t len = L->nt * c->nel;
	for (size_t q = 0; q < len; ++q)
		u[q] = u[q] * L->mask[q];
}

/* per-element operator, Dirichlet mask, DSS (src/solver.c:191-198) */
void og_global_opeval(og_ctx *c, int level, int var, const double *p,
		double *ap)
{
	local_op(c, level, var, p, ap);
	mask_apply(c, level, var, ap);
	dss_level(c, level, ap);
}

/* ------------------------------------------------------------------ */
/* preconditioner data (src/precon.c:336-413, src/helmholtz.c:51-77)  */
/* ------------------------------------------------------------------ */

static void set_diagonal(og_ctx *c, int level, double lam, double *dst)
{
	level_t *L = &c->lev[level];
	const int n = L->n;
	const size_t nt = L->nt;
	const double *D = L->b.D, *w = L->b.w;
	for (int e = 0; e < c->nel; ++e) {
		const size_t o = e * nt;
		for (int k = 0; k < n; ++k)
			for (int j = 0; j < n; ++j)
				for (int i = 0; i < n; ++i) {
					double t = 0.0;
					for (int p = 0; p < n; ++p) {
						const double di = D[p * n + i];
						const double dj = D[p * n + j];
						const double dk = D[p * n + k];
						t += ((w[p] * w[j]) * w[k]) * (di * di) *
								L->g[0][o + (k * n + j) * n + p];
						t += ((w[i] * w[p]) * w[k]) * (dj * dj) *
								L->g[3][o + (k * n + p) * n + i];
						t += ((w[i] * w[j]) * w[p]) * (dk * dk) *
								L->g[5][o + (p * n + j) * n + i];
					}
					const double rho = (w[i] * w[j]) * w[k];
					t += lam * rho * L->det[o + (k * n + j) * n + i];
					dst[o + (k * n + j) * n + i] = t;
				}
	}
	dss_level(c, level, dst);
	for (size_t q = 0; q < nt * c->nel; ++q)
		dst[q] = 1.0 / dst[q];
}

static void init_precon(og_ctx *c)
{
	static const int dbit[6] = { 1, 2, 4, 8, 16, 32 };
	for (int l = 0; l < c->nlev; ++l) {
		level_t *L = &c->lev[l];
		const size_t len = L->nt * c->nel;
		set_diagonal(c, l, 0.0, L->diag_p);
		set_diagonal(c, l, (11.0 / 6.0) * 1.0 / (c->dt * c->visc),
				L->diag_h);
		for (size_t q = 0; q < len; ++q)
			L->scale[q] = 1.0;
		dss_level(c, l, L->scale);
		for (size_t q = 0; q < len; ++q)
			L->scale[q] = 1.0 / L->scale[q];
		for (size_t q = 0; q < len; ++q)
			L->mask[q] = 1.0;
		for (int e = 0; e < c->nel; ++e)
			for (int f = 0; f < 6; ++f)
				if (c->bc[e] & dbit[f])
					for (int p = 0; p < L->n * L->n; ++p)
						L->mask[e * L->nt +
								face_node(L->n, f, p)] = 0.0;
	}
	level_t *L = &c->lev[0];
	const size_t len = L->nt * c->nel;
	c->inv_mass = dalloc(len);
	for (int e = 0; e < c->nel; ++e)
		for (size_t q = 0; q < L->nt; ++q) {
			const int n = L->n;
			const int i = q % n, j = (q / n) % n, k = q / (n * n);
			const double rho = (L->b.w[i] * L->b.w[j]) * L->b.w[k];
			c->inv_mass[e * L->nt + q] = rho * L->det[e * L->nt + q];
		}
	dss_level(c, 0, c->inv_mass);
	for (size_t q = 0; q < len; ++q)
		c->inv_mass[q] = 1.0 / c->inv_mass[q];
}

/* ------------------------------------------------------------------ */
/* setup (src/main.c:53-79, src/precon.c:58-183)                      */
/* ------------------------------------------------------------------ */

/* SVV cut-off mode and amplitude of the contexts created next
 * (params->svvn, params->svva; src/main.c:54-55): svvn < 0 is 2n/3 */
static int og_next_svvn = -1;
static double og_next_svva = 0.0;

void og_set_svv(int svvn, double svva)
{
	og_next_svvn = svvn;
	og_next_svva = svva;
}

og_ctx *og_create(int n, int nel, const double *vertices, const int *neigh,
		double dt, double visc, double dens)
{
	if (n < 2 || n > MAXN || (3 * n) / 2 > MAXN)
		return NULL;
	og_ctx *c = (og_ctx *) calloc(1, sizeof(*c));
	c->nel = nel;
	c->n = n;
	c->dt = dt;
	c->visc = visc;
	c->dens = dens;
	c->neigh = (int *) malloc(sizeof(int) * 26 * (size_t) nel);
	memcpy(c->neigh, neigh, sizeof(int) * 26 * (size_t) nel);
	c->pairs = (int *) malloc(sizeof(int) * 52 * (size_t) nel);
	c->bc = (int *) calloc(nel, sizeof(int));
	for (int e = 0; e < nel; ++e)
		for (int f = 0; f < 6; ++f)
			if (neigh[26 * e + f] == -1)
				c->bc[e] |= 1 << f;
	build_pairs(c);

	/* level orders nmg[i] = max(2, (n-1)/2^i + 1) until 2 (precon.c:62-69) */
	int nlev = 0;
	for (int i = 0; i < MAXLEV; ++i) {
		int m = (n - 1) / (1 << i) + 1;
		if (m < 2)
			m = 2;
		c->lev[i].n = m;
		nlev = i + 1;
		if (m == 2)
			break;
	}
	c->nlev = nlev;
	/* one cut-off mode and amplitude for every level (src/precon.c:130-132) */
	const int msvv = og_next_svvn >= 0 ? og_next_svvn : 2 * n / 3;
	for (int l = 0; l < nlev; ++l) {
		level_t *L = &c->lev[l];
		alloc_level(L, L->n, nel);
		make_basis(&L->b, L->n, msvv, og_next_svva);
	}
	grid_from_vertices(&c->lev[0], nel, vertices);
	compute_factors(&c->lev[0], nel);
	for (int l = 1; l < nlev; ++l) {
		level_t *F = &c->lev[l - 1], *L = &c->lev[l];
		og_interp(F->n, F->b.x, L->n, L->b.x, L->jf);
		/* coarse grid = fine grid evaluated at the coarse nodes
		 * (src/precon.c:151-160) */
		double Jc[MAXN * MAXN];
		og_interp(L->n, L->b.x, F->n, F->b.x, Jc);
		for (int e = 0; e < nel; ++e)
			for (int a = 0; a < 3; ++a)
				tensor3(F->n, L->n, Jc, F->grid[a] + e * F->nt,
						L->grid[a] + e * L->nt);
		compute_factors(L, nel);
	}
	/* dealiasing grid m = 3n/2, built from the vertices (src/main.c:53,71) */
	const int m = (3 * n) / 2;
	alloc_level(&c->conv, m, nel);
	make_basis(&c->conv.b, m, 2 * m / 3, 0.0);
	grid_from_vertices(&c->conv, nel, vertices);
	compute_factors(&c->conv, nel);
	og_interp(m, c->conv.b.x, n, c->lev[0].b.x, c->jconv);
	init_precon(c);
	return c;
}

void og_destroy(og_ctx *c)
{
	if (!c)
		return;
	for (int l = 0; l < c->nlev; ++l)
		free_level(&c->lev[l]);
	free_level(&c->conv);
	free(c->neigh);
	free(c->pairs);
	free(c->bc);
	free(c->inv_mass);
	free(c->ppts);
	free(c->pjac);
	free(c->ptinv);
	free(c);
}

/* The reference's GLL points come from an eigenvalue solve, so they can
 * differ from og_gll's in the last bit; a bitwise particle walk has to read
 * the caller's points and factors (jac, tinv: 9 x nel x n^3 each). */
void og_set_particle_basis(og_ctx *c, const double *points, const double *jac,
		const double *tinv)
{
	const size_t np = c->lev[0].nt * c->nel;
	free(c->ppts);
	free(c->pjac);
	free(c->ptinv);
	c->ppts = dalloc(c->n);
	c->pjac = dalloc(9 * np);
	c->ptinv = dalloc(9 * np);
	memcpy(c->ppts, points, c->n * sizeof(double));
	memcpy(c->pjac, jac, 9 * np * sizeof(double));
	memcpy(c->ptinv, tinv, 9 * np * sizeof(double));
}

void og_set_params(og_ctx *c, double t, double dt, double visc)
{
	c->t = t;
	c->dt = dt;
	c->visc = visc;
	for (int l = 0; l < c->nlev; ++l)
		set_diagonal(c, l, (11.0 / 6.0) * 1.0 / (dt * visc),
				c->lev[l].diag_h);
}

int og_nlevels(const og_ctx *c)
{
	return c->nlev;
}

int og_level_n(const og_ctx *c, int level)
{
	return c->lev[level].n;
}

int og_conv_n(const og_ctx *c)
{
	return c->conv.n;
}

static const double *level_comp(const level_t *L, int comp)
{
	if (comp < 6)
		return L->g[comp];
	if (comp == 6)
		return L->det;
	if (comp < 10)
		return L->grid[comp - 7];
	if (comp < 19)
		return L->jac[comp - 10];
	return L->tinv[comp - 19];
}

void og_level_geometry(const og_ctx *c, int level, int comp, double *dst)
{
	const level_t *L = &c->lev[level];
	memcpy(dst, level_comp(L, comp), L->nt * c->nel * sizeof(double));
}

void og_level_precon(const og_ctx *c, int level, int which, double *dst)
{
	const level_t *L = &c->lev[level];
	const double *src = which == 0 ? L->diag_p : which == 1 ? L->diag_h :
			which == 2 ? L->scale : which == 3 ? L->mask : c->inv_mass;
	memcpy(dst, src, L->nt * c->nel * sizeof(double));
}

void og_dss_pairs(const og_ctx *c, int *pairs)
{
	memcpy(pairs, c->pairs, sizeof(int) * 52 * (size_t) c->nel);
}

void og_conv_geometry(const og_ctx *c, int comp, double *dst)
{
	const double *src = comp < 9 ? c->conv.tinv[comp] : c->conv.det;
	memcpy(dst, src, c->conv.nt * c->nel * sizeof(double));
}

/* ------------------------------------------------------------------ */
/* Krylov solvers (src/solver.c:33-213, src/precon.c:227-324)         */
/* ------------------------------------------------------------------ */

static void subtract_nullspace(og_ctx *c, int level, int var, double *u)
{
	if (var != VAR_PRESSURE)
		return;
	const level_t *L = &c->lev[level];
	const size_t len = L->nt * c->nel;
	double nunique = 0.0, comp = 0.0;
	for (size_t q = 0; q < len; ++q)
		nunique += L->scale[q];
	for (size_t q = 0; q < len; ++q)
		comp += (u[q] * L->scale[q]);
	const double a = -comp / nunique;
	for (size_t q = 0; q < len; ++q)
		u[q] += a;
}

static void jacobi(const og_ctx *c, int level, int var, const double *r,
		double *z)
{
	const level_t *L = &c->lev[level];
	const double *d = var == VAR_PRESSURE ? L->diag_p : L->diag_h;
	const size_t len = L->nt * c->nel;
	for (size_t q = 0; q < len; ++q)
		z[q] = r[q] * d[q];
}

/* record sqrt((r.r)_w) of each iteration */
typedef struct {
	double *hist;
	int cap;
	int len;
} history;

static void record(history *h, double v)
{
	if (!h)
		return;
	if (h->len < h->cap)
		h->hist[h->len] = v;
	++h->len;
}

static void mg_precon(og_ctx *c, int var, const double *r, double *z,
		double eps);

/* Preconditioned CG, do-while with the absolute stop
 * sqrt((r.r)_w) <= eps or max_iter iterations (src/solver.c:33-81). */
static double cg(og_ctx *c, int level, int var, double *f, double *u,
		double eps, int max_iter, history *h)
{
	const size_t len = c->lev[level].nt * c->nel;
	double *r = dalloc(len), *z = dalloc(len), *p = dalloc(len),
			*ap = dalloc(len);
	mask_apply(c, level, var, f);
	og_global_opeval(c, level, var, u, r);
	for (size_t q = 0; q < len; ++q)
		r[q] = f[q] + -r[q];
	subtract_nullspace(c, level, var, r);
	jacobi(c, level, var, r, z);
	subtract_nullspace(c, level, var, z);
	memcpy(p, z, len * sizeof(double));
	double rdz = og_dot(c, level, r, z);
	int j = 0;
	double err;
	do {
		og_global_opeval(c, level, var, p, ap);
		const double alpha = rdz / og_dot(c, level, p, ap);
		for (size_t q = 0; q < len; ++q)
			u[q] += alpha * p[q];
		for (size_t q = 0; q < len; ++q)
			r[q] += -alpha * ap[q];
		jacobi(c, level, var, r, z);
		subtract_nullspace(c, level, var, z);
		const double rdz_old = rdz;
		rdz = og_dot(c, level, r, z);
		const double beta = rdz / rdz_old;
		for (size_t q = 0; q < len; ++q)
			p[q] = beta * p[q] + z[q];
		mask_apply(c, level, var, p);
		err = sqrt(og_dot(c, level, r, r));
		record(h, err);
	} while (err > eps && ++j < max_iter);
	free(r); free(z); free(p); free(ap);
	return err;
}

/* x <- (Jf^T)^3 x then DSS-average at the coarse level
 * (src/precon.c:283-291, src/global.c:259-268) */
static void restrict_to(og_ctx *c, int level, const double *fine,
		double *coarse)
{
	const level_t *F = &c->lev[level - 1], *L = &c->lev[level];
	for (int e = 0; e < c->nel; ++e)
		tensor3_t(F->n, L->n, L->jf, fine + e * F->nt,
				coarse + e * L->nt);
	dss_level(c, level, coarse);
	for (size_t q = 0; q < L->nt * c->nel; ++q)
		coarse[q] = coarse[q] * L->scale[q];
}

/* fine <- (Jf)^3 coarse (src/precon.c:293-300) */
static void prolong_from(og_ctx *c, int level, const double *coarse,
		double *fine)
{
	const level_t *F = &c->lev[level], *L = &c->lev[level + 1];
	for (int e = 0; e < c->nel; ++e)
		tensor3(L->n, F->n, L->jf, coarse + e * L->nt,
				fine + e * F->nt);
}

/* V-cycle with CG-Jacobi post-smoothing (15 iterations) and a CG-Jacobi
 * coarse solve (500 iterations), both stopping at eps
 * (src/precon.c:238-271). */
static double mg_recurse(og_ctx *c, int level, int var, double *f, double *x,
		double eps)
{
	if (level == c->nlev - 1)
		return cg(c, level, var, f, x, eps, 500, NULL);
	const level_t *F = &c->lev[level], *L = &c->lev[level + 1];
	const size_t nf = F->nt * c->nel, nc = L->nt * c->nel;
	double *r = dalloc(nf), *fn = dalloc(nc), *e = dalloc(nc);
	if (level == 0) {
		og_global_opeval(c, level, var, x, r);
		for (size_t q = 0; q < nf; ++q)
			r[q] = f[q] + -r[q];
	} else {
		memcpy(r, f, nf * sizeof(double));
	}
	restrict_to(c, level + 1, r, fn);
	mg_recurse(c, level + 1, var, fn, e, eps);
	prolong_from(c, level, e, r);
	for (size_t q = 0; q < nf; ++q)
		x[q] += r[q];
	const double err = cg(c, level, var, f, x, eps, 15, NULL);
	free(r); free(fn); free(e);
	return err;
}

/* z = Jacobi(r), then one V-cycle (src/precon.c:227-236) */
static void mg_precon(og_ctx *c, int var, const double *r, double *z,
		double eps)
{
	const size_t len = c->lev[0].nt * c->nel;
	double *f = dalloc(len);
	memcpy(f, r, len * sizeof(double));
	jacobi(c, 0, var, f, z);
	mg_recurse(c, 0, var, f, z, eps);
	free(f);
}

void og_mg_precon(og_ctx *c, const double *r, double *z, double eps)
{
	mg_precon(c, VAR_PRESSURE, r, z, eps);
}

/* Flexible CG with the truncation window m = min(j, max(1, j mod 11)) and
 * the shifted direction history (src/solver.c:83-157).  The history is a
 * ring here; the reference shifts copies, which is the same arithmetic. */
static double fcg_mg(og_ctx *c, const double *f_in, double *u, double eps,
		int max_iter, history *h)
{
	const int var = VAR_PRESSURE, mmax = 10;
	const size_t len = c->lev[0].nt * c->nel;
	double *f = dalloc(len), *r = dalloc(len), *z = dalloc(len);
	double *P[11], *AP[10];
	double pap[10] = { 0 }, beta[10];
	for (int i = 0; i <= mmax; ++i)
		P[i] = dalloc(len);
	for (int i = 0; i < mmax; ++i)
		AP[i] = dalloc(len);
	memcpy(f, f_in, len * sizeof(double));
	og_global_opeval(c, 0, var, u, r);
	for (size_t q = 0; q < len; ++q)
		r[q] = f[q] + -r[q];
	subtract_nullspace(c, 0, var, r);
	int j = 0;
	double err;
	do {
		int m = j < 1 ? 0 : (j % (mmax + 1) > 1 ? j % (mmax + 1) : 1);
		if (m > j)
			m = j;
		mg_precon(c, var, r, z, eps);
		subtract_nullspace(c, 0, var, z);
		for (int k = 0; k < m; ++k)
			beta[k] = og_dot(c, 0, z, AP[k]) / pap[k];
		/* p[k+1] <- p[k] for k = m-1..0 */
		double *tail = P[m];
		for (int k = m; k > 0; --k)
			P[k] = P[k - 1];
		P[0] = tail;
		memcpy(P[0], z, len * sizeof(double));
		for (int k = 1; k < m + 1; ++k)
			for (size_t q = 0; q < len; ++q)
				P[0][q] += -beta[k - 1] * P[k][q];
		mask_apply(c, 0, var, P[0]);
		int m2 = (j + 1) % (mmax + 1) > 1 ? (j + 1) % (mmax + 1) : 1;
		if (m2 > j + 1)
			m2 = j + 1;
		double *atail = AP[m2 - 1];
		for (int k = m2 - 1; k > 0; --k) {
			AP[k] = AP[k - 1];
			pap[k] = pap[k - 1];
		}
		AP[0] = atail;
		og_global_opeval(c, 0, var, P[0], AP[0]);
		pap[0] = og_dot(c, 0, P[0], AP[0]);
		const double alpha = og_dot(c, 0, P[0], r) / pap[0];
		for (size_t q = 0; q < len; ++q)
			u[q] += alpha * P[0][q];
		for (size_t q = 0; q < len; ++q)
			r[q] += -alpha * AP[0][q];
		err = sqrt(og_dot(c, 0, r, r));
		record(h, err);
	} while (err > eps && ++j < max_iter);
	for (int i = 0; i <= mmax; ++i)
		free(P[i]);
	for (int i = 0; i < mmax; ++i)
		free(AP[i]);
	free(f); free(r); free(z);
	return err;
}

int og_solve_poisson(og_ctx *c, const double *f, double *u, double eps,
		int max_iter, double *hist, int cap)
{
	history h = { hist, cap, 0 };
	fcg_mg(c, f, u, eps, max_iter, &h);
	return h.len;
}

int og_solve_helmholtz(og_ctx *c, int var, const double *f, double *u,
		double eps, int max_iter, double *hist, int cap)
{
	history h = { hist, cap, 0 };
	const size_t len = c->lev[0].nt * c->nel;
	double *fc = dalloc(len);
	memcpy(fc, f, len * sizeof(double));
	cg(c, 0, var, fc, u, eps, max_iter, &h);
	free(fc);
	return h.len;
}

/* ------------------------------------------------------------------ */
/* dealiased skew-symmetric convection (src/convection.c:37-140)      */
/* ------------------------------------------------------------------ */

void og_convection(og_ctx *c, const double *u, const double *v, double *out)
{
	const level_t *L0 = &c->lev[0], *M = &c->conv;
	const int n = L0->n, m = M->n;
	const size_t nt = L0->nt, mt = M->nt, nel = c->nel;
	double *ui[3], *vi[3], *dv[9], *cv[3], *cs[3], *tmp = dalloc(mt),
			*uv = dalloc(mt), *ts[3];
	for (int a = 0; a < 3; ++a) {
		ui[a] = dalloc(mt);
		vi[a] = dalloc(mt);
		cv[a] = dalloc(mt);
		cs[a] = dalloc(mt);
		ts[a] = dalloc(mt);
	}
	for (int a = 0; a < 9; ++a)
		dv[a] = dalloc(mt);
	double *res = dalloc(nt);
	for (size_t e = 0; e < nel; ++e) {
		const size_t om = e * mt;
		for (int a = 0; a < 3; ++a) {
			tensor3(n, m, c->jconv, u + (a * nel + e) * nt, ui[a]);
			tensor3(n, m, c->jconv, v + (a * nel + e) * nt, vi[a]);
		}
		/* convective form: dv[c][b] = d v_c / d r_b, then
		 * (u . grad) v_c with grad = tinv (src/convection.c:71-93) */
		for (int a = 0; a < 3; ++a) {
			dx_r(m, M->b.D, vi[a], dv[3 * a + 0]);
			dx_s(m, M->b.D, vi[a], dv[3 * a + 1]);
			dx_t(m, M->b.D, vi[a], dv[3 * a + 2]);
		}
		for (size_t q = 0; q < mt; ++q) {
			const int i = q % m, j = (q / m) % m, k = q / (m * m);
			const double rho = (M->b.w[i] * M->b.w[j]) * M->b.w[k];
			const double J = M->det[om + q];
			double t[3][3];
			for (int a = 0; a < 3; ++a)
				for (int b = 0; b < 3; ++b)
					t[a][b] = M->tinv[3 * a + b][om + q];
			for (int cc = 0; cc < 3; ++cc) {
				double d[3];
				for (int a = 0; a < 3; ++a) {
					double s = t[a][0] * dv[3 * cc + 0][q];
					s = t[a][1] * dv[3 * cc + 1][q] + s;
					s = t[a][2] * dv[3 * cc + 2][q] + s;
					d[a] = s;
				}
				double s = ui[0][q] * d[0];
				s = ui[1][q] * d[1] + s;
				s = ui[2][q] * d[2] + s;
				cv[cc][q] = (s * rho) * J;
			}
		}
		/* conservative form: sum_a sum_b tinv[a][b] d_b(u_b v_i)
		 * (src/convection.c:95-127) */
		for (int cc = 0; cc < 3; ++cc) {
			for (size_t q = 0; q < mt; ++q)
				uv[q] = ui[0][q] * vi[cc][q];
			dx_r(m, M->b.D, uv, ts[0]);
			for (size_t q = 0; q < mt; ++q)
				uv[q] = ui[1][q] * vi[cc][q];
			dx_s(m, M->b.D, uv, ts[1]);
			for (size_t q = 0; q < mt; ++q)
				uv[q] = ui[2][q] * vi[cc][q];
			dx_t(m, M->b.D, uv, ts[2]);
			for (size_t q = 0; q < mt; ++q) {
				const int i = q % m, j = (q / m) % m, k = q / (m * m);
				const double rho = (M->b.w[i] * M->b.w[j]) * M->b.w[k];
				double d[3];
				for (int a = 0; a < 3; ++a) {
					double s = M->tinv[3 * a + 0][om + q] * ts[0][q];
					s = M->tinv[3 * a + 1][om + q] * ts[1][q] + s;
					s = M->tinv[3 * a + 2][om + q] * ts[2][q] + s;
					d[a] = s;
				}
				double s = d[0];
				s += d[1];
				s += d[2];
				cs[cc][q] = (s * rho) * M->det[om + q];
			}
		}
		/* skew-symmetric average, weak projection back to n
		 * (src/convection.c:129-140,58-60) */
		for (int cc = 0; cc < 3; ++cc) {
			for (size_t q = 0; q < mt; ++q)
				tmp[q] = 0.5 * cv[cc][q] + 0.5 * cs[cc][q];
			tensor3_t(m, n, c->jconv, tmp, res);
			memcpy(out + (cc * nel + e) * nt, res, nt * sizeof(double));
		}
	}
	for (int a = 0; a < 3; ++a) {
		free(ui[a]); free(vi[a]); free(cv[a]); free(cs[a]); free(ts[a]);
	}
	for (int a = 0; a < 9; ++a)
		free(dv[a]);
	free(tmp); free(uv); free(res);
}

/* ------------------------------------------------------------------ */
/* Lagrangian particles (src/particles.c:182-546,                     */
/* src/interpolation.c:31-104)                                        */
/* ------------------------------------------------------------------ */

/* first node of the 5-point stencil (src/interpolation.c:106-112) */
static int first_point(const double *x, double xp, int n)
{
	for (int i = 0; i < n - 4; ++i)
		if (x[i] > xp)
			return i - 2 > 0 ? i - 2 : 0;
	return n - 5;
}

/* point value of a field block; 5-point tensor Lagrange stencil for n > 5,
 * full tensor Lagrange otherwise (src/interpolation.c:41-104) */
double og_point_interp(int n, const double *x, const double *f, double xp,
		double yp, double zp)
{
	if (n <= 5) {
		double lx[MAXN], ly[MAXN], lz[MAXN];
		for (int i = 0; i < n; ++i) {
			lx[i] = lagrange(xp, x, i, n);
			ly[i] = lagrange(yp, x, i, n);
			lz[i] = lagrange(zp, x, i, n);
		}
		double s = 0.0;
		for (int k = 0; k < n; ++k) {
			double sj = 0.0;
			for (int j = 0; j < n; ++j) {
				double si = 0.0;
				for (int i = 0; i < n; ++i)
					si += f[(k * n + j) * n + i] * lx[i];
				sj += si * ly[j];
			}
			s += sj * lz[k];
		}
		return s;
	}
	const int i1 = first_point(x, xp, n), j1 = first_point(x, yp, n),
			k1 = first_point(x, zp, n);
	double lx[5], ly[5], lz[5];
	for (int i = 0; i < 5; ++i) {
		lx[i] = lagrange(xp, x + i1, i, 5);
		ly[i] = lagrange(yp, x + j1, i, 5);
		lz[i] = lagrange(zp, x + k1, i, 5);
	}
	double s = 0.0;
	for (int k = 0; k < 5; ++k)
		for (int j = 0; j < 5; ++j)
			for (int i = 0; i < 5; ++i)
				s += f[((k1 + k) * n + j1 + j) * n + i1 + i] *
						lx[i] * ly[j] * lz[k];
	return s;
}

typedef struct {
	og_ctx *c;
	const double *ur;     /* [lev][comp][e][n^3] */
	const double *x;      /* GLL points */
} pctx;

static const double *pfactor(const pctx *P, int tinv, int a, int e)
{
	const og_ctx *c = P->c;
	const level_t *L = &c->lev[0];
	const double *stored = tinv ? c->ptinv : c->pjac;
	if (stored)
		return stored + ((size_t) a * c->nel + e) * L->nt;
	return (tinv ? L->tinv[a] : L->jac[a]) + e * L->nt;
}

static const double *ur_block(const pctx *P, int lev, int comp, int e)
{
	const level_t *L = &P->c->lev[0];
	return P->ur + (((size_t) lev * 3 + comp) * P->c->nel + e) * L->nt;
}

/* quadratic Lagrange in time over t0-2dt, t0-dt, t0 with levels whose
 * weight is below 1e-6 skipped (src/particles.c:493-515) */
static double fluid_velocity(const pctx *P, int e, const double *y, double t,
		int comp)
{
	const og_ctx *c = P->c;
	const level_t *L = &c->lev[0];
	const double eps = 1.0e-6;
	const double d0 = t - c->t + 2.0 * c->dt, d1 = t - c->t + c->dt,
			d2 = t - c->t;
	const double dt2 = pow(c->dt, 2);
	const double a = 0.5 * d1 * d2 / dt2;
	const double b = -d0 * d2 / dt2;
	const double cc = 0.5 * d0 * d1 / dt2;
	double u0 = 0.0, u1 = 0.0, u2 = 0.0;
	if (fabs(a) > eps)
		u0 = og_point_interp(L->n, P->x, ur_block(P, 0, comp, e),
				y[0], y[1], y[2]);
	if (fabs(b) > eps)
		u1 = og_point_interp(L->n, P->x, ur_block(P, 1, comp, e),
				y[0], y[1], y[2]);
	if (fabs(cc) > eps)
		u2 = og_point_interp(L->n, P->x, ur_block(P, 2, comp, e),
				y[0], y[1], y[2]);
	return a * u0 + b * u1 + cc * u2;
}

static void particle_rhs(const pctx *P, int e, double tau, const double *y,
		double t, double *f)
{
	const double a = 1.0 / tau;
	for (int i = 0; i < 3; ++i) {
		f[i] = y[i + 3];
		f[i + 3] = a * (fluid_velocity(P, e, y, t, i) - y[i + 3]);
	}
}

static int crossed(const double *y)
{
	for (int i = 0; i < 3; ++i)
		if (fabs(y[i]) > 1.0)
			return 1;
	return 0;
}

/* classic RK4 in reference coordinates; stages that leave [-1,1]^3 abort
 * unless forced (src/particles.c:238-269).  The reference's stage 0 reads
 * f[0] before writing it, multiplied by a[0] = 0; it is zero here. */
static void rk4(const pctx *P, double *s, int *st, double dt, int force)
{
	const double aa[4] = { 0.0, 0.5, 0.5, 1.0 };
	const int e = st[0];
	double y[6], y0[6], f[4][6];
	memcpy(y0, s, sizeof(y0));
	memset(f, 0, sizeof(f));
	for (int j = 0; j < 4; ++j) {
		const double t = s[6] + aa[j] * dt;
		const int jm = j - 1 > 0 ? j - 1 : 0;
		for (int i = 0; i < 6; ++i)
			y[i] = y0[i] + aa[j] * dt * f[jm][i];
		if (j > 0 && crossed(y) && !force) {
			st[2] = ST_OUTSIDE;
			return;
		}
		particle_rhs(P, e, s[7], y, t, f[j]);
	}
	for (int i = 0; i < 6; ++i)
		y[i] = y0[i] + dt * (f[0][i] / 6.0 + f[1][i] / 3.0 +
				f[2][i] / 3.0 + f[3][i] / 6.0);
	if (crossed(y)) {
		st[2] = ST_OUTSIDE;
		return;
	}
	memcpy(s, y, sizeof(y));
	s[6] = P->c->t;
}

static double step_to_boundary(const double *y, const double *f)
{
	double d[3];
	for (int i = 0; i < 3; ++i)
		d[i] = (copysign(1.0, f[i]) - y[i]) / f[i];
	const double m01 = d[0] < d[1] ? d[0] : d[1];
	return m01 < d[2] ? m01 : d[2];
}

/* RK4-weighted straight step to the element face (src/particles.c:271-316);
 * the reference's random reseed is replaced by the status ST_RESEED. */
static void to_boundary(const pctx *P, double *s, int *st, double dt)
{
	const double aa[4] = { 0.0, 0.5, 0.5, 1.0 };
	const int e = st[0];
	double y[6], y0[6], f[5][6];
	double dtau = 0.0;
	memcpy(y0, s, sizeof(y0));
	memset(f, 0, sizeof(f));
	for (int j = 0; j < 4; ++j) {
		const double t = s[6] + aa[j] * dtau;
		const int jm = j - 1 > 0 ? j - 1 : 0;
		for (int i = 0; i < 6; ++i)
			y[i] = y0[i] + aa[j] * dtau * f[jm][i];
		particle_rhs(P, e, s[7], y, t, f[j]);
		dtau = step_to_boundary(y0, f[j]);
	}
	for (int i = 0; i < 6; ++i)
		f[4][i] = (f[0][i] / 6.0 + f[1][i] / 3.0 + f[2][i] / 3.0 +
				f[3][i] / 6.0);
	dtau = step_to_boundary(y0, f[4]);
	if (dtau < dt) {
		s[6] += dtau;
		for (int i = 0; i < 6; ++i)
			s[i] += dtau * f[4][i];
	} else {
		st[2] = ST_NORMAL;
		rk4(P, s, st, dt, 1);
		if (st[2] != ST_NORMAL)
			st[2] = ST_RESEED;
	}
}

static int closest_face(const double *s)
{
	double hmin = 2.0;
	int k = 0;
	for (int i = 0; i < 6; ++i) {
		const double h = fabs(s[i / 2] - (i % 2 ? 1.0 : -1.0));
		if (h < hmin) {
			hmin = h;
			k = i;
		}
	}
	return k;
}

/* interpolate a 3x3 geometric factor component block at the particle */
static double factor_at(const pctx *P, int tinv, int a, int e, const double *s)
{
	return og_point_interp(P->c->lev[0].n, P->x, pfactor(P, tinv, a, e), s[0],
			s[1], s[2]);
}

/* Cross into the neighbour through the closest face, converting the
 * velocity to physical components by the interpolated Jacobian (component
 * by component, each using the already converted ones, as
 * src/particles.c:333-349 and 517-527 do); a wall reverses the normal
 * velocity. */
static void new_element(const pctx *P, double *s, int *st)
{
	const og_ctx *c = P->c;
	const int e = st[0];
	const int j = closest_face(s);
	const int nb = c->neigh[26 * e + j];
	if (nb >= 0) {
		st[0] = nb;
		for (int comp = 0; comp < 3; ++comp) {
			double dx[3];
			for (int i = 0; i < 3; ++i)
				dx[i] = factor_at(P, 0, 3 * comp + i, e, s);
			s[3 + comp] = s[3] * dx[0] + s[4] * dx[1] + s[5] * dx[2];
		}
	} else {
		st[2] = ST_COLLISION;
		s[3 + j / 2] *= -1.0;
	}
}

/* Entry face = the LAST face of the new element whose neighbour is the old
 * element; its coordinate becomes -+1; velocity back to reference
 * components via the interpolated transposed inverse (src/particles.c:
 * 351-378, 529-539). */
static void new_location(const pctx *P, double *s, int *st)
{
	const og_ctx *c = P->c;
	const int e = st[0];
	double y0[6], x[2];
	memcpy(y0, s, sizeof(y0));
	int k = closest_face(s);
	int j = 0;
	for (int i = 0; i < 3; ++i)
		if (i != k / 2)
			x[j++] = y0[i];
	for (int i = 0; i < 6; ++i)
		if (c->neigh[26 * e + i] == st[1])
			k = i;
	s[k / 2] = k % 2 ? 1.0 : -1.0;
	j = 0;
	for (int i = 0; i < 3; ++i) {
		if (i != k / 2)
			s[i] = x[j++];
		double dx[3];
		for (int a = 0; a < 3; ++a)
			dx[a] = factor_at(P, 1, 3 * a + i, e, s);
		s[3 + i] = s[3] * dx[0] + s[4] * dx[1] + s[5] * dx[2];
	}
	st[1] = st[0];
}

/* src/particles.c:182-218 at one rank; reseeds are reported, not drawn */
int og_particles_advance(og_ctx *c, size_t np, double *state, int *ints,
		const double *ur)
{
	pctx P = { c, ur, c->ppts ? c->ppts : c->lev[0].b.x };
	for (size_t i = 0; i < np; ++i)
		ints[3 * i + 2] = ST_OUTSIDE;
	int pass = 0, unfinished;
	do {
		for (size_t i = 0; i < np; ++i) {
			double *s = state + 8 * i;
			int *st = ints + 3 * i;
			if (st[2] == ST_NORMAL || st[2] == ST_RESEED)
				continue;
			st[2] = ST_NORMAL;
			if (pass > 10) {
				st[2] = ST_RESEED;
				continue;
			}
			rk4(&P, s, st, c->t - s[6], 0);
			if (st[2] == ST_OUTSIDE)
				to_boundary(&P, s, st, 2.0 * c->dt);
			if (st[2] == ST_OUTSIDE)
				new_element(&P, s, st);
		}
		for (size_t i = 0; i < np; ++i)
			if (ints[3 * i + 2] == ST_OUTSIDE)
				new_location(&P, state + 8 * i, ints + 3 * i);
		++pass;
		unfinished = 0;
		for (size_t i = 0; i < np; ++i)
			if (ints[3 * i + 2] != ST_NORMAL &&
					ints[3 * i + 2] != ST_RESEED)
				unfinished = 1;
	} while (unfinished);
	return pass;
}
