// The convection sub-steps of the time step on the device:
// integrate_convection_rk4 (src/time.c:84-130) with add_interpolated_velocity
// (src/time.c:132-152) and trivec_inverse_mass_matrix (src/time.c:154-167).
// The reference's lagrangian_convection_integration (src/navier_stokes.c:
// 71-92) calls it three times a step; each call runs two RK4 sub-steps of
// four stages, and each stage evaluates the dealiased convection of a stage
// field advected by the velocity interpolated in time from the last three
// steps -- 24 of the 25 convection evaluations of a step.  Here a stage is
// three launches: one pass that forms the stage field and the interpolated
// velocity, the convection over all elements, and one DSS of the three
// components whose epilogue multiplies by the inverse mass; a sub-step ends with
// one pass of the four stage updates.  The velocity history and the stage
// fields stay on the device.
//
// The vector updates keep the reference's operation order, each axpy
// y += alpha x as one fused multiply-add (the BLAS daxpy form), also where
// one pass applies several in sequence; the
// interpolation weights are computed on the host exactly as the reference
// computes them.  The convection and the DSS agree with the reference's to
// their own tolerances (1e-13 and bitwise), so the result agrees to
// rounding.
#include <cuda_runtime.h>

#include <cmath>
#include <utility>

#include "ssg_internal.h"
#include "ssg_kernels.h"

namespace ssg {
namespace dev {

#define SSG_TS_LOOP(q, n)                                                       \
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < (n);      \
       q += (size_t)gridDim.x * blockDim.x)

// out = (init ? out : 0) + wa uoo + wb uo + wc u, each term only where its
// flag is set, in that order (add_interpolated_velocity)
__global__ void k_interp_velocity(size_t n, double* __restrict__ out, bool init,
                                  const double* __restrict__ uoo, const double* __restrict__ uo,
                                  const double* __restrict__ u, double wa, double wb, double wc,
                                  bool fa, bool fb, bool fc) {
  SSG_TS_LOOP(q, n) {
    double v = init ? out[q] : 0.0;
    if (fa) v = fma(wa, uoo[q], v);
    if (fb) v = fma(wb, uo[q], v);
    if (fc) v = fma(wc, u[q], v);
    out[q] = v;
  }
}

// one stage's inputs: the stage field y = u (+ alpha f) and the velocity
// interpolated in time, ut = wa uoo + wb uo + wc u (each term only where its
// flag is set, in that order)
__global__ void k_stage_inputs(size_t n, double* __restrict__ y, const double* __restrict__ u,
                               const double* __restrict__ f, double alpha, bool add,
                               double* __restrict__ ut, const double* __restrict__ uoo,
                               const double* __restrict__ uo, const double* __restrict__ uc,
                               double wa, double wb, double wc, bool fa, bool fb, bool fc) {
  SSG_TS_LOOP(q, n) {
    y[q] = add ? fma(alpha, f[q], u[q]) : u[q];
    double v = 0.0;
    if (fa) v = fma(wa, uoo[q], v);
    if (fb) v = fma(wb, uo[q], v);
    if (fc) v = fma(wc, uc[q], v);
    ut[q] = v;
  }
}

// u += c0 f0; u += c1 f1; u += c2 f2; u += c3 f3 (four axpys in that order,
// each rounded as its own fused multiply-add)
__global__ void k_axpy4(size_t n, double* __restrict__ u, const double* __restrict__ f0,
                        const double* __restrict__ f1, const double* __restrict__ f2,
                        const double* __restrict__ f3, double c0, double c1, double c2,
                        double c3) {
  SSG_TS_LOOP(q, n) {
    double v = u[q];
    v = fma(c0, f0[q], v);
    v = fma(c1, f1[q], v);
    v = fma(c2, f2[q], v);
    u[q] = fma(c3, f3[q], v);
  }
}

}  // namespace dev
}  // namespace ssg

using namespace ssg;

namespace {

// weights of the quadratic interpolation in time of the velocity history
// at time t (src/time.c:135-141), with the history's own time and step
struct InterpWeights {
  double a, b, c;
  bool fa, fb, fc;
};

InterpWeights interp_weights(double t0, double dt0, double t, double alpha) {
  const double d[3] = {t - t0 + 2.0 * dt0, t - t0 + dt0, t - t0};
  const double a = 0.5 * d[1] * d[2] / std::pow(dt0, 2);
  const double b = -d[0] * d[2] / std::pow(dt0, 2);
  const double cc = 0.5 * d[0] * d[1] / std::pow(dt0, 2);
  const double eps = 1.0e-6;
  InterpWeights w;
  w.a = a * alpha;
  w.b = b * alpha;
  w.c = cc * alpha;
  w.fa = std::fabs(a) > eps;
  w.fb = std::fabs(b) > eps;
  w.fc = std::fabs(cc) > eps;
  return w;
}

}  // namespace

namespace ssg {

ssg_status ensure_rk_scratch(ssg_context* c) {
  if (c->rk_scratch) return SSG_OK;
  // the stage field y, the interpolated velocity, f_0 .. f_3 and the field
  // of the C entry point, 3 x npts each
  void* p = nullptr;
  if (cudaMalloc(&p, 7 * 3 * c->lev[0].npts * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return fail(c, SSG_ERR_NOMEM, "convection sub-step scratch");
  }
  c->rk_scratch = static_cast<double*>(p);
  return SSG_OK;
}

ssg_status convection_rk4(ssg_context* c, double* du, double t0, double t, double dt,
                          double beta, const double* uoo, const double* uo, const double* uc,
                          double th, double dth) {
  const DevLevel& L = c->lev[0];
  const size_t npc = L.npts, np = 3 * npc;
  cudaStream_t s = c->stream;
  SSG_TRY(ensure_rk_scratch(c));
  // f[i] holds the stage's raw convection, then the buffer y held is swapped
  // in: the DSS with the inverse mass product reads f[i] and writes y, and
  // the stage field's buffer is free again once the convection has run
  double* y = c->rk_scratch;
  double* ut = y + np;
  double* f[4] = {ut + np, ut + 2 * np, ut + 3 * np, ut + 4 * np};
  const int nb = vec_blocks(np);
  const double a[4] = {0.0, 0.5, 0.5, 1.0};
  const double b[4] = {1.0, 2.0, 2.0, 1.0};
  {
    const InterpWeights w = interp_weights(th, dth, t0, beta);
    count_launch();
    dev::k_interp_velocity<<<nb, 256, 0, s>>>(np, du, true, uoo, uo, uc, w.a, w.b, w.c, w.fa,
                                               w.fb, w.fc);
    SSG_CUDA(c, cudaGetLastError());
  }
  int k = 0;
  while (t0 + (double)k++ * dt < t - 0.5 * dt) {
    for (int i = 0; i < 4; ++i) {
      const InterpWeights w = interp_weights(th, dth, t0 + ((double)(k - 1) + a[i]) * dt, 1.0);
      count_launch();
      dev::k_stage_inputs<<<nb, 256, 0, s>>>(np, y, du, i > 0 ? f[i - 1] : du, -dt * a[i],
                                             i > 0, ut, uoo, uo, uc, w.a, w.b, w.c, w.fa, w.fb,
                                             w.fc);
      SSG_CUDA(c, cudaGetLastError());
      SSG_CUDA(c, run_convection(s, c->nel, 0, c->nel, c->n, c->m, ut, y, f[i], c->conv_w,
                                 c->host.conv.D.data(), c->host.jconv.data(), c->conv_D,
                                 c->conv_J, c->conv_scratch));
      // trivec_inverse_mass_matrix: per component the DSS, then the product
      // with 1 / DSS(mass), the three components in one pass
      SSG_CUDA(c, run_dss3(s, true, L.n, c->nel, f[i], y, npc, c->d_nbreg, L.dss_ec, c->inv_mass));
      std::swap(f[i], y);
    }
    count_launch();
    dev::k_axpy4<<<nb, 256, 0, s>>>(np, du, f[0], f[1], f[2], f[3], -dt * b[0] / 6.0,
                                    -dt * b[1] / 6.0, -dt * b[2] / 6.0, -dt * b[3] / 6.0);
    SSG_CUDA(c, cudaGetLastError());
  }
  return SSG_OK;
}

}  // namespace ssg

extern "C" {

ssg_status ssg_set_velocity_history(ssg_context* c, const double* u, const double* u_old,
                                    const double* u_oldold, double t, double dt) {
  if (!c) return SSG_ERR_ARG;
  if (!c->ready) return fail(c, SSG_ERR_STATE, "no mesh set up on this context");
  if (!u || !u_old || !u_oldold) return fail(c, SSG_ERR_ARG, "null velocity level");
  if (!(dt > 0.0) || !std::isfinite(t)) return fail(c, SSG_ERR_ARG, "dt must be > 0");
  SSG_CUDA(c, cudaSetDevice(c->device));
  const size_t np = 3 * c->lev[0].npts;
  if (!c->vhist) {
    void* p = nullptr;
    if (cudaMalloc(&p, 3 * np * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      return fail(c, SSG_ERR_NOMEM, "velocity history");
    }
    c->vhist = static_cast<double*>(p);
  }
  // levels in the order the interpolation weights them: oldest first
  const double* lv[3] = {u_oldold, u_old, u};
  for (int l = 0; l < 3; ++l)
    SSG_CUDA(c, cudaMemcpyAsync(c->vhist + l * np, lv[l], np * sizeof(double),
                                cudaMemcpyDefault, c->stream));
  SSG_CUDA(c, cudaStreamSynchronize(c->stream));
  c->vhist_t = t;
  c->vhist_dt = dt;
  return SSG_OK;
}

ssg_status ssg_integrate_convection_rk4(ssg_context* c, double* u, double t0, double t,
                                        double dt, double beta) {
  if (!c) return SSG_ERR_ARG;
  if (!c->ready) return fail(c, SSG_ERR_STATE, "no mesh set up on this context");
  if (!c->conv_w) return fail(c, SSG_ERR_STATE, "no dealiasing grid set up");
  if (!c->vhist) return fail(c, SSG_ERR_STATE, "ssg_set_velocity_history first");
  if (!u) return fail(c, SSG_ERR_ARG, "null field");
  if (!(dt > 0.0) || !std::isfinite(t0) || !std::isfinite(t) || !std::isfinite(beta))
    return fail(c, SSG_ERR_ARG, "bad time arguments");
  SSG_CUDA(c, cudaSetDevice(c->device));
  SSG_TRY(ensure_rk_scratch(c));
  const size_t np = 3 * c->lev[0].npts;
  double* du = c->rk_scratch + 6 * np;
  SSG_CUDA(c, cudaMemcpyAsync(du, u, np * sizeof(double), cudaMemcpyDefault, c->stream));
  const double* h = c->vhist;
  SSG_TRY(convection_rk4(c, du, t0, t, dt, beta, h, h + np, h + 2 * np, c->vhist_t,
                         c->vhist_dt));
  SSG_CUDA(c, cudaMemcpyAsync(u, du, np * sizeof(double), cudaMemcpyDefault, c->stream));
  SSG_CUDA(c, cudaStreamSynchronize(c->stream));
  return SSG_OK;
}

}  // extern "C"
