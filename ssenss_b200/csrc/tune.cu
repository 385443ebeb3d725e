// Launch-shape autotuner.
//
// The element kernels have one free shape parameter per order n and the
// vector kernels one overall:
//   * the operator of every order but 8: the line-form kernel k_axl, or the
//     plane-form k_ax with 1, 2, 4, ... elements per block up to the
//     256-thread / 96 KB limit of ax_epb_max(n); order 8 runs the FP64
//     tensor-core operator k_ax8_dmma, which has no shape parameter;
//   * the cap of the DSS grid (one node per thread below it): 4 .. 64
//     blocks per SM;
//   * the cap of the vector kernels' grid (one point per thread below it):
//     2 .. 64 blocks per SM, timed on the CG update.
// ssg_autotune times every candidate on the context's own mesh and levels
// (CUDA events on the context stream, best of three runs of ten launches)
// and keeps the fastest in the process-wide tables the launchers read.  The
// tables are keyed by order only, so one tuning serves every mesh of that
// order on the device.  Captured CUDA graphs hold the old shapes and are
// dropped.  Nothing here changes results: each candidate computes the same
// sums in the same order.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "ssg_internal.h"
#include "ssg_kernels.h"

namespace ssg {
namespace {

// best-of-3 time of `reps` launches of f (ms)
template <typename F>
ssg_status time_launches(ssg_context* c, int reps, F&& f, float* best) {
  *best = 1e30f;
  for (int trial = 0; trial < 3; ++trial) {
    SSG_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    for (int r = 0; r < reps; ++r) SSG_CUDA(c, f());
    SSG_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    SSG_CUDA(c, cudaEventSynchronize(c->ev1));
    float ms = 0.f;
    SSG_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    *best = std::min(*best, ms);
  }
  return SSG_OK;
}

}  // namespace

// scratch vectors of the tuning runs: three level-sized FP64 buffers
static ssg_status tune_level(ssg_context* c, int level, double* a, double* b, double* y,
                             int reps) {
  const DevLevel& L = c->lev[level];
  const int n = L.n;
  // operator: elements per block (order 8 has the tensor-core kernel only)
  if (n != 8) {
    int best_epb = 0;
    float best = 1e30f;
    for (int epb = kAxLine; epb <= ax_epb_max(n); epb = epb == kAxLine ? 1 : 2 * epb) {
      g_tune_ax_epb[n] = epb;
      SSG_CUDA(c, run_ax(c->stream, n, c->nel, epb, false, false, a, b, L.gf, L.npts, nullptr,
                         L.D, L.D, 0.0, nullptr));
      float t = 0.f;
      SSG_TRY(time_launches(c, reps, [&] {
        return run_ax(c->stream, n, c->nel, epb, false, false, a, b, L.gf, L.npts, nullptr,
                      L.D, L.D, 0.0, nullptr);
      }, &t));
      if (t < best) {
        best = t;
        best_epb = epb;
      }
    }
    g_tune_ax_epb[n] = best_epb;
  }
  // DSS: blocks per SM of the persistent grid
  {
    int best_bps = 0;
    float best = 1e30f;
    for (int bps = 4; bps <= 64; bps *= 2) {
      g_tune_dss_bps[n] = bps;
      float t = 0.f;
      SSG_TRY(time_launches(c, reps, [&] {
        return run_dss(c->stream, DSS_DOT, false, n, c->nel, a, b, c->d_nbreg, L.dss_ec,
                       nullptr, y, nullptr, c->d_part, nullptr, nullptr);
      }, &t));
      if (t < best) {
        best = t;
        best_bps = bps;
      }
    }
    g_tune_dss_bps[n] = best_bps;
  }
  return SSG_OK;
}

}  // namespace ssg

using namespace ssg;

extern "C" {

ssg_status ssg_autotune(ssg_context* c, int reps) {
  if (!c) return SSG_ERR_ARG;
  if (!c->ready) return fail(c, SSG_ERR_STATE, "no mesh set up on this context");
  if (reps <= 0) reps = 10;
  SSG_CUDA(c, cudaSetDevice(c->device));
  const size_t np0 = c->lev[0].npts;
  std::vector<double*> buf(6, nullptr);
  for (auto& p : buf) {
    if (cudaMalloc(&p, np0 * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      for (auto& q : buf)
        if (q) cudaFree(q);
      return fail(c, SSG_ERR_NOMEM, "autotune scratch");
    }
    cudaMemsetAsync(p, 0, np0 * sizeof(double), c->stream);
  }
  ssg_status st = SSG_OK;
  bool seen[SSG_MAXN + 1] = {false};
  for (int l = 0; l < c->nlev && st == SSG_OK; ++l) {
    const int n = c->lev[l].n;
    if (seen[n]) continue;
    seen[n] = true;
    st = tune_level(c, l, buf[0], buf[1], buf[2], reps);
  }
  // vector kernels: the grid cap, timed on the heaviest of them, the CG
  // update (x += alpha p, r -= alpha ap, z = dinv r, four partial sums)
  if (st == SSG_OK) {
    int best_bps = 0;
    float best = 1e30f;
    for (int bps : {2, 3, 4, 6, 8, 16, 32, 64}) {
      if (st != SSG_OK) break;
      g_tune_vec_bps = bps;
      const int nb = vec_blocks(np0);
      float t = 0.f;
      st = time_launches(c, reps, [&] {
        return run_cg_update(c->stream, false, np0, c->d_sums, buf[0], buf[1], buf[2], buf[3],
                             buf[4], c->lev[0].mult, buf[5], c->d_part, nb, nullptr, nullptr);
      }, &t);
      if (t < best) {
        best = t;
        best_bps = bps;
      }
    }
    g_tune_vec_bps = best_bps;
  }
  cudaStreamSynchronize(c->stream);
  for (auto& p : buf) cudaFree(p);
  invalidate_graphs(c);
  return st;
}

// Deterministic non-zero test field in [-1, 1) (splitmix64 of the index),
// so timed kernels read and write real numbers rather than zeros.
static ssg_status fill_field(ssg_context* c, double* dst, size_t n) {
  std::vector<double> h(n);
  for (size_t i = 0; i < n; ++i) {
    unsigned long long z = (unsigned long long)i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    h[i] = (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
  }
  SSG_CUDA(c, cudaMemcpyAsync(dst, h.data(), n * sizeof(double), cudaMemcpyHostToDevice,
                              c->stream));
  SSG_CUDA(c, cudaStreamSynchronize(c->stream));
  return SSG_OK;
}

ssg_status ssg_time_operator(ssg_context* c, int var, int reps, double* us_per_apply) {
  if (!c || !us_per_apply || reps <= 0) return SSG_ERR_ARG;
  if (!c->ready) return fail(c, SSG_ERR_STATE, "no mesh set up on this context");
  SSG_CUDA(c, cudaSetDevice(c->device));
  SSG_TRY(ensure_workspace(c));
  if (var != SSG_PRESSURE) SSG_TRY(helmholtz_diag_update(c));
  const DevLevel& L = c->lev[0];
  const bool helm = var != SSG_PRESSURE;
  const double lam = (11.0 / 6.0) / (c->dt * c->visc);
  double* in = workspace_scratch(c);
  double* out = c->d_stage[0];
  SSG_TRY(fill_field(c, in, L.npts));
  auto launch = [&] {
    return run_ax(c->stream, L.n, c->nel, 0, helm, false, in, out, L.gf, L.npts, L.bj, L.D,
                  L.S, lam, nullptr);
  };
  SSG_CUDA(c, launch());
  float best = 0.f;
  SSG_TRY(time_launches(c, reps, launch, &best));
  *us_per_apply = 1e3 * (double)best / reps;
  return SSG_OK;
}

ssg_status ssg_time_smoother(ssg_context* c, int level, int reps, double* us) {
  if (!c || !us || reps <= 0) return SSG_ERR_ARG;
  if (!c->ready) return fail(c, SSG_ERR_STATE, "no mesh set up on this context");
  if (level < 0 || level >= c->nlev) return fail(c, SSG_ERR_ARG, "level out of range");
  SSG_CUDA(c, cudaSetDevice(c->device));
  const DevLevel& L = c->lev[level];
  const size_t np = L.npts;
  std::vector<double*> buf(6, nullptr);
  for (auto& p : buf) {
    if (cudaMalloc(&p, np * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      for (auto& q : buf)
        if (q) cudaFree(q);
      return fail(c, SSG_ERR_NOMEM, "timing scratch");
    }
  }
  for (auto& p : buf) {
    const ssg_status fs = fill_field(c, p, np);
    if (fs != SSG_OK) {
      for (auto& q : buf) cudaFree(q);
      return fs;
    }
  }
  const int nb = vec_blocks(np);
  auto op = [&] {
    return run_ax(c->stream, L.n, c->nel, 0, false, false, buf[0], buf[1], L.gf, np, nullptr,
                  L.D, L.D, 0.0, nullptr);
  };
  auto dss = [&] {
    return run_dss(c->stream, DSS_DOT, false, L.n, c->nel, buf[1], buf[2], c->d_nbreg,
                   L.dss_ec, nullptr, buf[0], nullptr, c->d_part, nullptr, nullptr);
  };
  auto upd = [&] {
    return run_cg_update(c->stream, false, np, c->d_sums, buf[3], buf[0], buf[4], buf[2],
                         L.dinv_p, L.mult, buf[5], c->d_part, nb, nullptr, nullptr);
  };
  ssg_status st = SSG_OK;
  float t = 0.f;
  if (st == SSG_OK) st = time_launches(c, reps, op, &t);
  us[0] = 1e3 * (double)t / reps;
  if (st == SSG_OK) st = time_launches(c, reps, dss, &t);
  us[1] = 1e3 * (double)t / reps;
  if (st == SSG_OK) st = time_launches(c, reps, upd, &t);
  us[2] = 1e3 * (double)t / reps;
  cudaStreamSynchronize(c->stream);
  for (auto& p : buf) cudaFree(p);
  return st;
}

ssg_status ssg_tuning(int n, int* ax_elements_per_block, int* dss_blocks_per_sm,
                      int* vector_blocks_per_sm) {
  if (n < 2 || n > SSG_MAXN) return SSG_ERR_ARG;
  // 0: the FP64 tensor-core operator (one warp per element)
  const bool dmma = n == 8;
  if (ax_elements_per_block) *ax_elements_per_block = dmma ? 0 : ax_epb(n);
  if (dss_blocks_per_sm) *dss_blocks_per_sm = g_tune_dss_bps[n].load() > 0 ? g_tune_dss_bps[n].load() : 8;
  if (vector_blocks_per_sm) *vector_blocks_per_sm = g_tune_vec_bps.load() > 0 ? g_tune_vec_bps.load() : kVecBpsDefault;
  return SSG_OK;
}

}  // extern "C"
