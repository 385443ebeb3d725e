// The convection sub-steps of the time step on the device:
// integrate_convection_rk4 (src/time.c:84-130) with add_interpolated_velocity
// (src/time.c:132-152) and trivec_inverse_mass_matrix (src/time.c:154-167).
// The reference's lagrangian_convection_integration (src/navier_stokes.c:
// 71-92) calls it three times a step; each call runs two RK4 sub-steps of
// four stages, and each stage evaluates the dealiased convection of a stage
// field advected by the velocity interpolated in time from the last three
// steps -- 24 of the 25 convection evaluations of a step.  Here a stage is
// one convection launch over all elements, one DSS and one inverse-mass
// product per component, and a few vector kernels; the velocity history and
// the stage fields stay on the device.
//
// The vector updates keep the reference's operation order, each axpy
// y += alpha x as one fused multiply-add (the BLAS daxpy form); the
// interpolation weights are computed on the host exactly as the reference
// computes them.  The convection and the DSS agree with the reference's to
// their own tolerances (1e-13 and bitwise), so the result agrees to
// rounding.
#include <cuda_runtime.h>

#include <cmath>

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

// y = u (+ alpha f): the stage field
__global__ void k_stage_field(size_t n, double* __restrict__ y, const double* __restrict__ u,
                              const double* __restrict__ f, double alpha, bool add) {
  SSG_TS_LOOP(q, n) y[q] = add ? fma(alpha, f[q], u[q]) : u[q];
}

// u += alpha f
__global__ void k_axpy(size_t n, double* __restrict__ u, const double* __restrict__ f,
                       double alpha) {
  SSG_TS_LOOP(q, n) u[q] = fma(alpha, f[q], u[q]);
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

InterpWeights interp_weights(const ssg_context* c, double t, double alpha) {
  const double t0 = c->vhist_t, dt0 = c->vhist_dt;
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
  const DevLevel& L = c->lev[0];
  const size_t npc = L.npts, np = 3 * npc;
  cudaStream_t s = c->stream;
  if (!c->rk_scratch) {
    // staged u, the stage field y, the interpolated velocity, f_0 .. f_3
    void* p = nullptr;
    if (cudaMalloc(&p, 7 * np * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      return fail(c, SSG_ERR_NOMEM, "convection sub-step scratch");
    }
    c->rk_scratch = static_cast<double*>(p);
  }
  double* du = c->rk_scratch;
  double* y = du + np;
  double* ut = y + np;
  double* f[4] = {ut + np, ut + 2 * np, ut + 3 * np, ut + 4 * np};
  const double* uoo = c->vhist;
  const double* uo = c->vhist + np;
  const double* uc = c->vhist + 2 * np;
  const int nb = vec_blocks(np);
  SSG_CUDA(c, cudaMemcpyAsync(du, u, np * sizeof(double), cudaMemcpyDefault, s));

  auto interp = [&](double* out, bool init, double tt, double alpha) -> ssg_status {
    const InterpWeights w = interp_weights(c, tt, alpha);
    count_launch();
    dev::k_interp_velocity<<<nb, 256, 0, s>>>(np, out, init, uoo, uo, uc, w.a, w.b, w.c, w.fa,
                                               w.fb, w.fc);
    SSG_CUDA(c, cudaGetLastError());
    return SSG_OK;
  };
  const double a[4] = {0.0, 0.5, 0.5, 1.0};
  const double b[4] = {1.0, 2.0, 2.0, 1.0};

  SSG_TRY(interp(du, true, t0, beta));
  int k = 0;
  while (t0 + (double)k++ * dt < t - 0.5 * dt) {
    for (int i = 0; i < 4; ++i) {
      count_launch();
      dev::k_stage_field<<<nb, 256, 0, s>>>(np, y, du, i > 0 ? f[i - 1] : du, -dt * a[i], i > 0);
      SSG_CUDA(c, cudaGetLastError());
      SSG_TRY(interp(ut, false, t0 + ((double)(k - 1) + a[i]) * dt, 1.0));
      SSG_CUDA(c, run_convection(s, c->nel, 0, c->nel, c->n, c->m, ut, y, f[i], c->conv_w,
                                 c->host.conv.D.data(), c->host.jconv.data(), c->conv_D,
                                 c->conv_J, c->conv_scratch));
      // trivec_inverse_mass_matrix: per component DSS, then 1 / DSS(mass)
      for (int comp = 0; comp < 3; ++comp) {
        double* fc = f[i] + comp * npc;
        SSG_CUDA(c, run_dss(s, DSS_PLAIN, false, L.n, c->nel, fc, y + comp * npc, c->d_pairs,
                            L.dss_ec, nullptr, nullptr, nullptr, nullptr));
        SSG_CUDA(c, cudaMemcpyAsync(fc, y + comp * npc, npc * sizeof(double),
                                    cudaMemcpyDeviceToDevice, s));
        SSG_CUDA(c, run_mul(s, false, npc, fc, c->inv_mass));
      }
    }
    for (int i = 0; i < 4; ++i) {
      count_launch();
      dev::k_axpy<<<nb, 256, 0, s>>>(np, du, f[i], -dt * b[i] / 6.0);
      SSG_CUDA(c, cudaGetLastError());
    }
  }
  SSG_CUDA(c, cudaMemcpyAsync(u, du, np * sizeof(double), cudaMemcpyDefault, s));
  SSG_CUDA(c, cudaStreamSynchronize(s));
  return SSG_OK;
}

}  // extern "C"
