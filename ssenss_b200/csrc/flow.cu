// The whole time step on the device: integrate_navier_stokes
// (src/navier_stokes.c:224-235) over fields that stay in HBM between steps.
//
// One step, in the reference's order:
//   lagrangian_convection_integration (src/navier_stokes.c:71-92): the
//     convection history shifts and takes the velocity's self-convection;
//     the intermediate velocity u~ starts at zero and takes the three
//     convection sub-step integrations (timestep.cu) and dt f;
//   solve_pressure_poisson (src/navier_stokes.c:148-159): the double-curl
//     history shifts and takes curl curl u (stokes.cu); the pressure
//     gradient estimate (estimate_pressure_gradient, src/stokes.c:107-130)
//     goes through the DSS and the inverse mass; the right-hand side
//     (compute_pressure_rhs, src/navier_stokes.c:115-146) through the DSS;
//     the pressure is extrapolated (estimate_pressure, src/navier_stokes.c:
//     101-113) and solved for (FCG + p-multigrid);
//   solve_velocity_helmholtz (src/navier_stokes.c:203-222): the three
//     right-hand sides (compute_velocity_rhs, src/navier_stokes.c:177-201)
//     through the DSS, the velocity extrapolated with its wall values
//     (estimate_velocity, src/navier_stokes.c:161-175) and solved for
//     (Jacobi CG), one component at a time;
// then the time advances by dt.  Each solve's tolerance is the reference's
// residual_tolerance (src/navier_stokes.c:94-99) of its right-hand side.
//
// The history shifts (time_shift, src/time.c:30-42) rotate buffers instead
// of copying them; the velocity and pressure keep their current level in one
// buffer (the solves' CUDA graphs are captured per solution vector).  Wall values come from the caller, evaluated at t + dt
// at every node: the reference evaluates its boundary functions on the host
// (set_dirichlet_boundaries, src/poisson.c:101-143), and so does a caller.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <utility>
#include <vector>

#include "ssg_internal.h"
#include "ssg_kernels.h"

namespace ssg {
namespace dev {

#define SSG_FLOW_LOOP(q, n)                                                     \
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < (n);      \
       q += (size_t)gridDim.x * blockDim.x)

// node q of an element of order n lies on one of the faces in `walls`
// (bit f for face f of W E S N B T)
__device__ __forceinline__ bool on_wall(int walls, int n, int q) {
  if (!walls) return false;
  const int i = q % n, j = (q / n) % n, k = q / (n * n), m = n - 1;
  return ((walls & 1) && i == 0) || ((walls & 2) && i == m) || ((walls & 4) && j == 0) ||
         ((walls & 8) && j == m) || ((walls & 16) && k == 0) || ((walls & 32) && k == m);
}

struct DpdArgs {
  const double* f;      // body force (3 x npts)
  const double* dbc;    // wall values of du/dt (3 x npts) or null
  const int* bc;
  const double *rho, *det;
  const double *cv0, *cv1, *cv2;   // convection history, newest first
  const double *r0, *r1, *r2;      // double-curl history, newest first
  double c1, c2, c3;    // extrapolation weights of the convection terms
  double v1, v2, v3;    // ... and of the viscous terms
  double dens;
  double* out;          // 3 x npts
  size_t npts;
  int n, nt;
};

// estimate_pressure_gradient (src/stokes.c:107-130) after its double curl:
// dens (mass(f - du_wall/dt) + c1 cv0 + c2 cv1 + c3 cv2 + v1 r0 + v2 r1 + v3 r2),
// each sum an axpy
__global__ void k_pressure_gradient_estimate(DpdArgs A) {
  SSG_FLOW_LOOP(g, A.npts) {
    const int e = (int)(g / A.nt), q = (int)(g % A.nt);
    const bool wall = A.dbc && on_wall(A.bc[e], A.n, q);
    const double w = A.rho[q];
    const double dj = A.det[g];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t x = c * A.npts + g;
      double v = A.f[x];
      if (wall) v = fma(-1.0, A.dbc[x], v);
      v = __dmul_rn(__dmul_rn(v, w), dj);
      v = fma(A.c1, A.cv0[x], v);
      v = fma(A.c2, A.cv1[x], v);
      v = fma(A.c3, A.cv2[x], v);
      v = fma(A.v1, A.r0[x], v);
      v = fma(A.v2, A.r1[x], v);
      v = fma(A.v3, A.r2[x], v);
      A.out[x] = __dmul_rn(v, A.dens);
    }
  }
}

// cur <- a1 cur + a2 old + a3 oldold (three axpys onto zero,
// single_stiffly_stable, src/time.c:51-75), then the wall values where
// given (set_dirichlet_boundaries), and oldold <- the previous cur: with the
// old and oldold slots swapped afterwards this is the time shift, while the
// current level stays in one buffer (the solves' graphs are keyed on it)
__global__ void k_extrapolate(size_t npts, int ncomp, double* cur, const double* old,
                              double* oldold, double a1, double a2, double a3,
                              const double* wallv, const int* bc, int n, int nt) {
  SSG_FLOW_LOOP(g, npts) {
    const bool wall = wallv && on_wall(bc[g / nt], n, (int)(g % nt));
    for (int c = 0; c < ncomp; ++c) {
      const size_t x = c * npts + g;
      const double u0 = cur[x];
      double v = fma(a1, u0, 0.0);
      v = fma(a2, old[x], v);
      v = fma(a3, oldold[x], v);
      oldold[x] = u0;
      cur[x] = wall ? wallv[x] : v;
    }
  }
}

// y += a x
__global__ void k_flow_axpy(size_t n, double* __restrict__ y, const double* __restrict__ x,
                            double a) {
  SSG_FLOW_LOOP(q, n) y[q] = fma(a, x[q], y[q]);
}

}  // namespace dev

namespace {

constexpr int kMaxIter = 5000;          // the reference's cap (src/solver.c:168,184)
constexpr double kAbsTol = 1.0e-10;     // ABSTOL, RELTOL (src/navier_stokes.c:33-34)
constexpr double kRelTol = 1.0e-10;

// Surface weights of add_surface_integral (src/poisson.c:145-194) per
// element, derivative d and face f of W E S N B T: (w_inner w_outer) times
// component d of the face's area-weighted normal (compute_surface_normal,
// src/geometry.c:138-186), the cross product of the two Jacobian columns
// along the face, signed outwards.  Face nodes in the reference's [outer]
// [inner] order: W/E (z, y), S/N (z, x), B/T (y, x).
void surface_weights(const HostLevel& L, int nel, std::vector<double>& sw) {
  const int n = L.n, m = n - 1;
  const size_t nt = L.nt, nn = (size_t)n * n;
  sw.assign((size_t)nel * 18 * nn, 0.0);
  // in-plane Jacobian columns (p, q) and orientation of each face
  const int P[6] = {1, 1, 0, 0, 0, 0}, Q[6] = {2, 2, 2, 2, 1, 1};
  const double S[6] = {-1.0, 1.0, 1.0, -1.0, -1.0, 1.0};
  parallel_elements(nel, [&](int e0, int e1) {
    for (int e = e0; e < e1; ++e)
      for (int f = 0; f < 6; ++f)
        for (int o = 0; o < n; ++o)
          for (int in = 0; in < n; ++in) {
            int x, y, z;
            if (f < 2) {
              x = f == 0 ? 0 : m;
              y = in;
              z = o;
            } else if (f < 4) {
              x = in;
              y = f == 2 ? 0 : m;
              z = o;
            } else {
              x = in;
              y = o;
              z = f == 4 ? 0 : m;
            }
            const size_t g = e * nt + ((size_t)z * n + y) * n + x;
            auto J = [&](int a, int b) { return L.jac[3 * a + b][g]; };
            const int p = P[f], q = Q[f];
            const double X = J(1, p) * J(2, q) - J(2, p) * J(1, q);
            const double Y = J(0, p) * J(2, q) - J(2, p) * J(0, q);
            const double Z = J(0, p) * J(1, q) - J(1, p) * J(0, q);
            const double nrm[3] = {S[f] * X, -S[f] * Y, S[f] * Z};
            const double ww = L.w[in] * L.w[o];
            for (int d = 0; d < 3; ++d)
              sw[((size_t)(e * 3 + d) * 6 + f) * nn + o * n + in] = ww * nrm[d];
          }
  });
}

ssg_status flow_alloc(ssg_context* c) {
  if (c->flow_buf) return SSG_OK;
  const HostLevel& L = c->host.lev[0];
  const size_t np = c->lev[0].npts;
  if (L.jac[0].size() != np)
    return fail(c, SSG_ERR_STATE,
                "the time step needs the level-0 Jacobian (ssg_setup_particle_geometry)");
  // velocity, convection and double-curl histories (3 levels x 3 fields),
  // pressure history, body force, u~, two scratch triples, wall values
  const size_t nvec = 9 + 9 + 9 + 3 + 3 + 3 + 3 + 3 + (c->has_walls ? 6 : 0);
  std::vector<double> sw;
  surface_weights(L, c->nel, sw);
  void* p = nullptr;
  if (cudaMalloc(&p, nvec * np * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return fail(c, SSG_ERR_NOMEM, "time-step fields");
  }
  double* b = static_cast<double*>(p);
  c->flow_buf = b;
  for (int l = 0; l < 3; ++l) {
    c->fu[l] = b + (0 + 3 * l) * np;
    c->fconv[l] = b + (9 + 3 * l) * np;
    c->frot[l] = b + (18 + 3 * l) * np;
    c->fp[l] = b + (27 + l) * np;
  }
  c->ff = b + 30 * np;
  c->fut = b + 33 * np;
  c->fa = b + 36 * np;
  c->fb = b + 39 * np;
  c->fbc = c->has_walls ? b + 42 * np : nullptr;
  c->dev_bytes += nvec * np * sizeof(double);
  SSG_CUDA(c, cudaMalloc((void**)&c->flow_sw, sw.size() * sizeof(double)));
  SSG_CUDA(c, cudaMemcpy(c->flow_sw, sw.data(), sw.size() * sizeof(double),
                         cudaMemcpyHostToDevice));
  SSG_CUDA(c, cudaMalloc((void**)&c->flow_bc, c->nel * sizeof(int)));
  SSG_CUDA(c, cudaMemcpy(c->flow_bc, c->host.bc.data(), c->nel * sizeof(int),
                         cudaMemcpyHostToDevice));
  c->dev_bytes += sw.size() * sizeof(double) + c->nel * sizeof(int);
  return SSG_OK;
}

ssg_status copy_fields(ssg_context* c, double* dst, const double* src, size_t count) {
  SSG_CUDA(c, cudaMemcpyAsync(dst, src, count * sizeof(double), cudaMemcpyDefault, c->stream));
  return SSG_OK;
}

// the reference's residual_tolerance of a right-hand side
ssg_status tolerance(ssg_context* c, const double* rhs, double* eps) {
  double d = 0.0;
  SSG_TRY(ssg_global_dot_product(c, rhs, rhs, &d));
  const double x = std::sqrt(d) * kRelTol;
  const double lo = kAbsTol < x ? kAbsTol : x;
  *eps = 1.0e-10 > lo ? 1.0e-10 : lo;
  return SSG_OK;
}

void rotate(double* a[3]) {
  double* t = a[2];
  a[2] = a[1];
  a[1] = a[0];
  a[0] = t;
}

ssg_status stokes(ssg_context* c, int which, const double* in, const double* g, double* out,
                  double x, double y) {
  const DevLevel& L = c->lev[0];
  SSG_CUDA(c, run_stokes(c->stream, which, c->n, c->nel, c->p_tinv, L.rho, L.det, L.D,
                         c->flow_bc, c->flow_sw, L.npts, in, g, out, x, y));
  return SSG_OK;
}

ssg_status need_flow(ssg_context* c) {
  if (!c) return SSG_ERR_ARG;
  if (!c->ready) return fail(c, SSG_ERR_STATE, "no mesh set up on this context");
  if (!c->conv_w) return fail(c, SSG_ERR_STATE, "no dealiasing grid set up");
  if (!c->p_tinv) return fail(c, SSG_ERR_STATE, "no level-0 Jacobian set up");
  SSG_CUDA(c, cudaSetDevice(c->device));
  return SSG_OK;
}

}  // namespace
}  // namespace ssg

using namespace ssg;

extern "C" {

ssg_status ssg_flow_set(ssg_context* c, const ssg_flow_fields* in, double t) {
  SSG_TRY(need_flow(c));
  if (!in || !std::isfinite(t)) return fail(c, SSG_ERR_ARG, "null fields or bad time");
  for (int l = 0; l < 3; ++l)
    if (!in->u[l] || !in->conv[l] || !in->rot[l] || !in->p[l])
      return fail(c, SSG_ERR_ARG, "every history level of u, conv, rot and p is needed");
  SSG_TRY(flow_alloc(c));
  const size_t np = c->lev[0].npts;
  for (int l = 0; l < 3; ++l) {
    SSG_TRY(copy_fields(c, c->fu[l], in->u[l], 3 * np));
    SSG_TRY(copy_fields(c, c->fconv[l], in->conv[l], 3 * np));
    SSG_TRY(copy_fields(c, c->frot[l], in->rot[l], 3 * np));
    SSG_TRY(copy_fields(c, c->fp[l], in->p[l], np));
  }
  if (in->f)
    SSG_TRY(copy_fields(c, c->ff, in->f, 3 * np));
  else
    SSG_CUDA(c, cudaMemsetAsync(c->ff, 0, 3 * np * sizeof(double), c->stream));
  SSG_CUDA(c, cudaStreamSynchronize(c->stream));
  c->flow_t = t;
  c->flow_ready = true;
  return SSG_OK;
}

ssg_status ssg_flow_get(ssg_context* c, ssg_flow_fields* out, double* t) {
  SSG_TRY(need_flow(c));
  if (!out) return fail(c, SSG_ERR_ARG, "null fields");
  if (!c->flow_ready) return fail(c, SSG_ERR_STATE, "ssg_flow_set first");
  const size_t np = c->lev[0].npts;
  for (int l = 0; l < 3; ++l) {
    if (out->u[l]) SSG_TRY(copy_fields(c, out->u[l], c->fu[l], 3 * np));
    if (out->conv[l]) SSG_TRY(copy_fields(c, out->conv[l], c->fconv[l], 3 * np));
    if (out->rot[l]) SSG_TRY(copy_fields(c, out->rot[l], c->frot[l], 3 * np));
    if (out->p[l]) SSG_TRY(copy_fields(c, out->p[l], c->fp[l], np));
  }
  if (out->f) SSG_TRY(copy_fields(c, out->f, c->ff, 3 * np));
  SSG_CUDA(c, cudaStreamSynchronize(c->stream));
  if (t) *t = c->flow_t;
  return SSG_OK;
}

ssg_status ssg_stokes_operator(ssg_context* c, int which, const double* in, const double* g,
                               double* out) {
  SSG_TRY(need_flow(c));
  if (which < SSG_STOKES_DOUBLE_CURL || which > SSG_STOKES_VELOCITY_RHS)
    return fail(c, SSG_ERR_ARG, "bad Stokes operator");
  if (!in || !out || (which != SSG_STOKES_DOUBLE_CURL && !g))
    return fail(c, SSG_ERR_ARG, "null field");
  SSG_TRY(flow_alloc(c));
  const size_t np = c->lev[0].npts;
  const size_t nin = 3 * np, ng = which == SSG_STOKES_PRESSURE_RHS ? 3 * np : np;
  const size_t nout = which == SSG_STOKES_PRESSURE_RHS ? np : 3 * np;
  // operands into the step's scratch (u~, the two triples)
  SSG_TRY(copy_fields(c, c->fut, in, nin));
  if (which != SSG_STOKES_DOUBLE_CURL) SSG_TRY(copy_fields(c, c->fb, g, ng));
  const double x = which == SSG_STOKES_PRESSURE_RHS ? -c->dens / c->dt : 1.0 / (c->dt * c->visc);
  const double y = -1.0 / (c->visc * c->dens);
  SSG_TRY(stokes(c, which, c->fut, c->fb, c->fa, x, y));
  SSG_TRY(copy_fields(c, out, c->fa, nout));
  SSG_CUDA(c, cudaStreamSynchronize(c->stream));
  return SSG_OK;
}

ssg_status ssg_navier_stokes_step(ssg_context* c, const double* f, const double* bc_u,
                                  const double* bc_dudt, ssg_solve_info* info) {
  SSG_TRY(need_flow(c));
  if (!c->flow_ready) return fail(c, SSG_ERR_STATE, "ssg_flow_set first");
  if (c->has_walls && (!bc_u || !bc_dudt))
    return fail(c, SSG_ERR_ARG, "a mesh with walls needs their values (bc_u, bc_dudt)");
  const DevLevel& L = c->lev[0];
  const size_t np = L.npts;
  const int nb = vec_blocks(np);
  const double dt = c->dt, t = c->flow_t;
  cudaStream_t s = c->stream;
  if (f) SSG_TRY(copy_fields(c, c->ff, f, 3 * np));
  const double* wall_u = nullptr;
  const double* wall_dudt = nullptr;
  if (c->has_walls) {
    SSG_TRY(copy_fields(c, c->fbc, bc_u, 3 * np));
    SSG_TRY(copy_fields(c, c->fbc + 3 * np, bc_dudt, 3 * np));
    wall_u = c->fbc;
    wall_dudt = c->fbc + 3 * np;
  }

  // lagrangian_convection_integration
  rotate(c->fconv);
  SSG_CUDA(c, run_convection(s, c->nel, 0, c->nel, c->n, c->m, c->fu[0], c->fu[0], c->fconv[0],
                             c->conv_w, c->host.conv.D.data(), c->host.jconv.data(), c->conv_D,
                             c->conv_J, c->conv_scratch));
  SSG_CUDA(c, cudaMemsetAsync(c->fut, 0, 3 * np * sizeof(double), s));
  const double tt[4] = {t - 2.0 * dt, t - dt, t, t + dt};
  const double beta[3] = {1.0 / 3.0, -3.0 / 2.0, 3.0};
  for (int r = 0; r < 3; ++r)
    SSG_TRY(convection_rk4(c, c->fut, tt[r], tt[r + 1], dt / 2.0, beta[r], c->fu[2], c->fu[1],
                           c->fu[0], t, dt));
  count_launch();
  dev::k_flow_axpy<<<vec_blocks(3 * np), 256, 0, s>>>(3 * np, c->fut, c->ff, dt);
  SSG_CUDA(c, cudaGetLastError());

  // compute_pressure_rhs
  rotate(c->frot);
  SSG_TRY(stokes(c, SSG_STOKES_DOUBLE_CURL, c->fu[0], nullptr, c->frot[0], 0.0, 0.0));
  {
    dev::DpdArgs A;
    A.f = c->ff;
    A.dbc = wall_dudt;
    A.bc = c->flow_bc;
    A.rho = L.rho;
    A.det = L.det;
    A.cv0 = c->fconv[0];
    A.cv1 = c->fconv[1];
    A.cv2 = c->fconv[2];
    A.r0 = c->frot[0];
    A.r1 = c->frot[1];
    A.r2 = c->frot[2];
    // stiffly_stable EXPLICIT3 (src/time.c:66-70) with c = SUBTRACT_NEW and
    // with c = -visc
    const double cc = -1.0, cv = -c->visc;
    A.c1 = 3.0 * cc;
    A.c2 = -3.0 * cc;
    A.c3 = 1.0 * cc;
    A.v1 = 3.0 * cv;
    A.v2 = -3.0 * cv;
    A.v3 = 1.0 * cv;
    A.dens = c->dens;
    A.out = c->fa;
    A.npts = np;
    A.n = L.n;
    A.nt = (int)L.nt;
    count_launch();
    dev::k_pressure_gradient_estimate<<<nb, 256, 0, s>>>(A);
    SSG_CUDA(c, cudaGetLastError());
  }
  SSG_CUDA(c, run_dss3(s, true, L.n, c->nel, c->fa, c->fb, np, c->d_nbreg, L.dss_ec, c->inv_mass));
  SSG_TRY(stokes(c, SSG_STOKES_PRESSURE_RHS, c->fut, c->fb, c->fa, -c->dens / dt, 0.0));
  SSG_CUDA(c, run_dss(s, DSS_PLAIN, false, L.n, c->nel, c->fa, c->fb, c->d_nbreg, L.dss_ec,
                      nullptr, nullptr, nullptr, nullptr));
  double eps_p = 0.0;
  SSG_TRY(tolerance(c, c->fb, &eps_p));

  // estimate_pressure, then the pressure solve
  count_launch();
  dev::k_extrapolate<<<nb, 256, 0, s>>>(np, 1, c->fp[0], c->fp[1], c->fp[2], 3.0, -3.0, 1.0,
                                        nullptr, c->flow_bc, L.n, (int)L.nt);
  SSG_CUDA(c, cudaGetLastError());
  std::swap(c->fp[1], c->fp[2]);
  ssg_status worst = SSG_OK;
  ssg_status st = ssg_solve_poisson_cg(c, c->fb, c->fp[0], eps_p, kMaxIter,
                                       info ? &info[0] : nullptr);
  if (st == SSG_MAXITER)
    worst = st;
  else if (st != SSG_OK)
    return st;

  // compute_velocity_rhs
  SSG_TRY(stokes(c, SSG_STOKES_VELOCITY_RHS, c->fut, c->fp[0], c->fa, 1.0 / (dt * c->visc),
                 -1.0 / (c->visc * c->dens)));
  SSG_CUDA(c, run_dss3(s, false, L.n, c->nel, c->fa, c->fb, np, c->d_nbreg, L.dss_ec, nullptr));
  double eps_u[3];
  for (int d = 0; d < 3; ++d) SSG_TRY(tolerance(c, c->fb + d * np, &eps_u[d]));

  // estimate_velocity, then the three Helmholtz solves
  count_launch();
  dev::k_extrapolate<<<nb, 256, 0, s>>>(np, 3, c->fu[0], c->fu[1], c->fu[2], 3.0, -3.0, 1.0,
                                        wall_u, c->flow_bc, L.n, (int)L.nt);
  SSG_CUDA(c, cudaGetLastError());
  std::swap(c->fu[1], c->fu[2]);
  for (int d = 0; d < 3; ++d) {
    st = ssg_solve_helmholtz_cg(c, SSG_X_VELOCITY + d, c->fb + d * np, c->fu[0] + d * np,
                                eps_u[d], kMaxIter, info ? &info[1 + d] : nullptr);
    if (st == SSG_MAXITER)
      worst = st;
    else if (st != SSG_OK)
      return st;
  }
  c->flow_t = t + dt;
  return worst;
}

}  // extern "C"
