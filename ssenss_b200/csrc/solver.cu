// Krylov solvers and the p-multigrid V-cycle on the device.
//
//   cg_solve   conjugate_gradient with jacobi_preconditioner
//              (src/solver.c:33-81, src/precon.c:311-324)
//   mg_apply   multigrid_preconditioner / multigrid_recurse
//              (src/precon.c:227-300)
//   fcg_solve  flexible_conjugate_gradient with the window
//              m = min(j, max(1, j mod 11)) (src/solver.c:83-157)
//
// All vectors and scalars stay on the device; the scalar algebra (alpha,
// beta, nullspace constant, residual norm, stop flag) runs in the
// reduction kernel, so the host only reads the stop flag.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "ssg_internal.h"
#include "ssg_kernels.h"

namespace ssg {

struct LevelWork {
  void *f = nullptr, *x = nullptr, *rr = nullptr, *r = nullptr, *z = nullptr;
  void *p = nullptr, *ap = nullptr, *aploc = nullptr, *tc = nullptr;
};

struct Workspace {
  LevelWork w64[SSG_MAXLEV];
  LevelWork w32[SSG_MAXLEV];
  bool have32 = false;
  double *r = nullptr, *z = nullptr, *aploc = nullptr;
  double* P[11] = {};
  double* AP[10] = {};
  double* hist = nullptr;
  int hist_cap = 0;
  double* scratch = nullptr;   // level-0 vector for set-up work (Helmholtz diagonal)
  std::vector<void*> blocks;
  // the V-cycle r -> z as one CUDA graph (its launch sequence is static:
  // smoother iterations past convergence exit on a device flag)
  cudaGraphExec_t vcycle = nullptr;
  double vcycle_eps = -1.0;
  int vcycle_precision = -1;
  unsigned long long vcycle_kernels = 0;
  bool vcycle_failed = false;
  double warm_eps = -1.0;   // eps / precision of the last direct V-cycle
  int warm_precision = -1;
  // FCG iterations as graphs: one per window state (the slot rotation of
  // the direction history is periodic: state 0 for the first iteration,
  // then 44 states that repeat), each an IF node that runs the iteration
  // only while the solve has not stopped, so iterations are enqueued ahead
  // without a host synchronisation
  static constexpr int kFcgStates = 45;
  cudaGraphExec_t fcg[kFcgStates] = {};
  unsigned long long fcg_kernels[kFcgStates] = {};
  double fcg_eps = -1.0;
  int fcg_precision = -1, fcg_max_iter = -1, fcg_hcap = -1;
  const double* fcg_u = nullptr;   // the solution vector the graphs update
  bool fcg_failed = false;
  int fcg_warm = 0;          // solves run directly with this configuration
  // the Jacobi CG loop (iterations after the first) as one WHILE graph per
  // operand set, a few kept (the three velocity components of a time step
  // each have their own), the least recently used replaced
  static constexpr int kLoops = 4;
  cudaGraphExec_t cgloop[kLoops] = {};
  unsigned long long cgloop_kernels[kLoops] = {};
  unsigned long long cgloop_used[kLoops] = {};
  unsigned long long cgloop_clock = 0;
  struct LoopKey {
    const void* f = nullptr;
    const void* x = nullptr;
    const double* hist = nullptr;
    double eps = -1.0, lam = 0.0;
    int max_iter = -1, hist_cap = 0, var = -1, level = -1, frame = -1;
    bool fp32 = false;
    bool operator==(const LoopKey& o) const {
      return f == o.f && x == o.x && hist == o.hist && eps == o.eps && lam == o.lam &&
             max_iter == o.max_iter && hist_cap == o.hist_cap && var == o.var &&
             level == o.level && frame == o.frame && fp32 == o.fp32;
    }
  } cgloop_key[kLoops];
  bool cgloop_failed = false;
};

static void drop_iteration_graphs(Workspace* w) {
  for (auto& g : w->fcg)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  w->fcg_failed = false;
  w->fcg_warm = 0;
  w->fcg_eps = -1.0;
  w->fcg_u = nullptr;
  for (int i = 0; i < Workspace::kLoops; ++i) {
    if (w->cgloop[i]) cudaGraphExecDestroy(w->cgloop[i]);
    w->cgloop[i] = nullptr;
    w->cgloop_key[i] = Workspace::LoopKey();
    w->cgloop_used[i] = 0;
  }
  w->cgloop_failed = false;
}

void free_workspace(Workspace* w) {
  if (!w) return;
  drop_iteration_graphs(w);
  if (w->vcycle) cudaGraphExecDestroy(w->vcycle);
  for (void* p : w->blocks) cudaFree(p);
  delete w;
}

void invalidate_graphs(ssg_context* c) {
  if (!c->ws) return;
  if (c->ws->vcycle) cudaGraphExecDestroy(c->ws->vcycle);
  c->ws->vcycle = nullptr;
  c->ws->vcycle_failed = false;
  drop_iteration_graphs(c->ws);
}

// Guard of a conditional graph node: its body runs while the solve's stop
// flag is clear (device side, no host round trip).
__global__ void k_set_running(cudaGraphConditionalHandle h, const double* __restrict__ done) {
  cudaGraphSetConditional(h, *done == 0.0 ? 1u : 0u);
}

// A graph whose conditional node (IF or WHILE) holds the work `enqueue`
// puts on the stream, guarded by k_set_running on the stop flag `done`; for
// WHILE the body ends with the same guard.  Returns false when the driver
// refuses any step (the caller then launches directly).
template <typename F>
static bool build_conditional_graph(ssg_context* c, bool loop, const double* done, F&& enqueue,
                                    cudaGraphExec_t* exec, unsigned long long* kernels) {
  cudaStream_t s = c->stream;
  cudaGraph_t g = nullptr;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) return false;
  bool ok = false;
  do {
    cudaGraphConditionalHandle h;
    if (cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault) != cudaSuccess)
      break;
    // the guard kernel, then the conditional node after it
    cudaGraphNode_t guard = nullptr;
    {
      cudaKernelNodeParams kp = {};
      void* args[] = {&h, &done};
      kp.func = (void*)k_set_running;
      kp.gridDim = dim3(1);
      kp.blockDim = dim3(1);
      kp.kernelParams = args;
      if (cudaGraphAddKernelNode(&guard, g, nullptr, 0, &kp) != cudaSuccess) break;
    }
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = loop ? cudaGraphCondTypeWhile : cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t cn = nullptr;
    if (cudaGraphAddNode(&cn, g, &guard, 1, &cp) != cudaSuccess) break;
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    const unsigned long long before = t_launches;
    if (cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      break;
    const ssg_status st = enqueue();
    if (loop && st == SSG_OK) k_set_running<<<1, 1, 0, s>>>(h, done);
    cudaGraph_t out = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(s, &out);
    const unsigned long long captured = t_launches - before;
    g_launches -= captured;   // recorded, not launched
    t_launches = before;
    if (st != SSG_OK || ce != cudaSuccess) break;
    if (cudaGraphInstantiate(exec, g, 0) != cudaSuccess) break;
    *kernels = captured;
    ok = true;
  } while (false);
  if (!ok) {
    cudaGetLastError();
    c->err.clear();
  }
  cudaGraphDestroy(g);
  return ok;
}

static ssg_status wsalloc(ssg_context* c, Workspace* w, void** p, size_t bytes) {
  SSG_CUDA(c, cudaMalloc(p, bytes));
  w->blocks.push_back(*p);
  c->dev_bytes += bytes;
  return SSG_OK;
}

static ssg_status alloc_level_work(ssg_context* c, Workspace* w, LevelWork& L, size_t np,
                                   size_t bytes) {
  void** v[] = {&L.f, &L.x, &L.rr, &L.r, &L.z, &L.p, &L.ap, &L.aploc, &L.tc};
  for (void** p : v) SSG_TRY(wsalloc(c, w, p, np * bytes));
  return SSG_OK;
}

ssg_status ensure_workspace(ssg_context* c) {
  if (!c->ws) {
    Workspace* w = new Workspace();
    c->ws = w;
    for (int l = 0; l < c->nlev; ++l)
      SSG_TRY(alloc_level_work(c, w, w->w64[l], c->lev[l].npts, sizeof(double)));
    const size_t np = c->lev[0].npts * sizeof(double);
    SSG_TRY(wsalloc(c, w, (void**)&w->r, np));
    SSG_TRY(wsalloc(c, w, (void**)&w->z, np));
    SSG_TRY(wsalloc(c, w, (void**)&w->aploc, np));
    for (auto& p : w->P) SSG_TRY(wsalloc(c, w, (void**)&p, np));
    for (auto& p : w->AP) SSG_TRY(wsalloc(c, w, (void**)&p, np));
    w->hist_cap = 8192;
    SSG_TRY(wsalloc(c, w, (void**)&w->hist, w->hist_cap * sizeof(double)));
    SSG_TRY(wsalloc(c, w, (void**)&w->scratch, np));
  }
  if (c->precision == SSG_PRECISION_MIXED && !c->ws->have32) {
    for (int l = 0; l < c->nlev; ++l)
      SSG_TRY(alloc_level_work(c, c->ws, c->ws->w32[l], c->lev[l].npts, sizeof(float)));
    c->ws->have32 = true;
    invalidate_graphs(c);
  }
  return SSG_OK;
}

double* workspace_scratch(ssg_context* c) { return c->ws ? c->ws->scratch : nullptr; }

static inline double lambda_of(const ssg_context* c) {
  return (11.0 / 6.0) / (c->dt * c->visc);
}

// out = A_e in (global: then mask and DSS), at one level
ssg_status op_apply(ssg_context* c, int level, int var, bool fp32, const void* in,
                    void* out, bool global) {
  SSG_TRY(ensure_workspace(c));
  const DevLevel& L = c->lev[level];
  const bool helm = var != SSG_PRESSURE;
  if (helm && (fp32 || level != 0))
    return fail(c, SSG_ERR_ARG, "the Helmholtz operator is FP64 at level 0 only");
  void* loc = global ? (fp32 ? c->ws->w32[level].aploc : c->ws->w64[level].aploc) : out;
  SSG_CUDA(c, run_ax(c->stream, L.n, c->nel, 0, helm, fp32, in, loc,
                     fp32 ? (const void*)L.gf32 : (const void*)L.gf, L.npts, L.bj, L.D, L.S,
                     lambda_of(c), nullptr));
  if (global)
    SSG_CUDA(c, run_dss(c->stream, DSS_PLAIN, fp32, L.n, c->nel, loc, out, c->d_nbreg, L.dss_ec,
                        helm ? L.mask : nullptr, nullptr, nullptr, nullptr));
  return SSG_OK;
}

// cancellation flag and deadline of the running solve, checked where the
// host already synchronises with the stream (a kernel in flight is never
// interrupted)
static ssg_status check_interrupt(ssg_context* c) {
  if (c->cancel && *c->cancel) return fail(c, SSG_ERR_CANCELLED, "solve cancelled");
  if (c->deadline > 0.0) {
    const double now =
        std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
            .count();
    if (now > c->deadline) return fail(c, SSG_ERR_TIMEOUT, "solve deadline expired");
  }
  return SSG_OK;
}

static ssg_status read_flag(ssg_context* c, const double* dptr, double* v) {
  SSG_CUDA(c, cudaMemcpyAsync(c->h_pin, dptr, sizeof(double), cudaMemcpyDeviceToHost,
                              c->stream));
  SSG_CUDA(c, cudaStreamSynchronize(c->stream));
  *v = c->h_pin[0];
  return SSG_OK;
}

ssg_status cg_solve(ssg_context* c, int level, int var, bool fp32, void* f, void* x,
                    double eps, int max_iter, int frame, double* hist, int hist_cap,
                    bool sync_each) {
  const DevLevel& L = c->lev[level];
  LevelWork& W = fp32 ? c->ws->w32[level] : c->ws->w64[level];
  const size_t np = L.npts;
  const int nb = vec_blocks(np);
  const int nbd = dss_grid(L.n, c->nel);
  const bool helm = var != SSG_PRESSURE;
  const bool pres = !helm;
  if (helm && (fp32 || level != 0))
    return fail(c, SSG_ERR_ARG, "the Helmholtz operator is FP64 at level 0 only");
  const double* mask = helm && c->has_walls ? L.mask : nullptr;
  double* fr = c->d_sc + frame * F_SIZE;
  const void* dinv = helm ? (const void*)L.dinv_h
                          : (fp32 ? (const void*)L.dinv_p32 : (const void*)L.dinv_p);
  const void* gf = fp32 ? (const void*)L.gf32 : (const void*)L.gf;
  const double lam = lambda_of(c);
  cudaStream_t s = c->stream;
  ScalarOp op;
  op.sums = c->d_sums;
  op.counter = c->d_counter;
  op.frame = fr;
  op.pressure = pres;
  op.nunique = L.nunique;
  op.eps = eps;
  op.max_iter = max_iter;
  op.hist = hist;
  op.hist_cap = hist_cap;

  // mask f; r = f - A x; subtract_nullspace(r)
  if (mask) SSG_CUDA(c, run_mul(s, fp32, np, f, mask));
  SSG_CUDA(c, run_ax(s, L.n, c->nel, 0, helm, fp32, x, W.aploc, gf, np, L.bj, L.D, L.S, lam,
                     nullptr));
  op.code = OP_NULL_C;
  SSG_CUDA(c, run_dss(s, DSS_RESID, fp32, L.n, c->nel, W.aploc, W.r, c->d_nbreg, L.dss_ec, mask, f,
                      nullptr, c->d_part, nullptr, &op));
  if (pres) SSG_CUDA(c, run_add_const(s, fp32, np, W.r, fr + F_C, 1));
  // z = M^-1 r and its nullspace constant
  op.code = OP_CG_INIT_C;
  SSG_CUDA(c, run_jacobi(s, fp32, np, W.r, dinv, L.mult, W.z, c->d_part, nb, &op));

  PUpdateArgs pu;
  pu.z = W.z;
  pu.beta = fr + F_BETA;
  pu.c = pres ? fr + F_C : nullptr;
  pu.mask = mask;
  // Once the stop flag is set every kernel of a later iteration returns at
  // once, so iterations are enqueued ahead without waiting for the flag:
  // all of them for a smoother (sync_each false), chunks of 8 otherwise.
  const double* stop = fr + F_DONE;
  pu.stop = stop;
  // Mixed precision (FP32 storage): (p w).DSS(mask A p) = p . (mask A p)
  // for a continuous, masked p, so the operator kernel reduces it, alpha is
  // known before the DSS, and the DSS gather feeds the update directly (two
  // kernels per iteration, ap never stored).  FP64 keeps the reference's
  // arithmetic: alpha from the weighted dot of the assembled ap
  // (src/solver.c:62-65), then the update -- the rounding of the fused form
  // moves a well-converged solution by a few 1e-11.
  const bool fused = fp32;
  ScalarOp dop = op;
  if (fused) {
    pu.dot = &dop;
    pu.part = c->d_part;
  }
  DssCg cg;
  cg.x = x;
  cg.p = W.p;
  cg.r = W.r;
  cg.dinv = dinv;
  cg.z = W.z;
  cg.alpha = fr + F_ALPHA;
  // A solve (sync_each) whose first iteration has run: the remaining ones
  // as one WHILE graph node -- its body is one iteration, repeated on the
  // device while the stop flag is clear, so the solve synchronises with the
  // host once.  Captured per (operands, eps, cap, lambda, history) and
  // replayed; a refused capture falls back to chunks of 8 launched
  // iterations with a host check between chunks.
  Workspace* wsp = c->ws;
  Workspace::LoopKey key;
  key.f = f;
  key.x = x;
  key.hist = hist;
  key.eps = eps;
  key.lam = helm ? lam : 0.0;
  key.max_iter = max_iter;
  key.hist_cap = hist_cap;
  key.var = var;
  key.level = level;
  key.frame = frame;
  key.fp32 = fp32;
  const bool loop_graph = sync_each && c->graphs && !wsp->cgloop_failed && max_iter > 1;
  for (int it = 0; it < max_iter; ++it) {
    if (loop_graph && it == 1) {
      // the cached graph of these operands, else the slot to capture into
      // (an empty one, or the least recently used)
      int slot = -1;
      for (int i = 0; i < Workspace::kLoops && slot < 0; ++i)
        if (wsp->cgloop[i] && wsp->cgloop_key[i] == key) slot = i;
      if (slot < 0) {
        slot = 0;
        for (int i = 1; i < Workspace::kLoops; ++i)
          if (wsp->cgloop_used[i] < wsp->cgloop_used[slot]) slot = i;
        if (wsp->cgloop[slot]) cudaGraphExecDestroy(wsp->cgloop[slot]);
        wsp->cgloop[slot] = nullptr;
        wsp->cgloop_used[slot] = 0;
        pu.first = 0;
        dop.code = OP_CG_ALPHA;
        const bool ok = build_conditional_graph(
            c, true, stop,
            [&]() -> ssg_status {
              SSG_CUDA(c, run_ax(s, L.n, c->nel, 0, helm, fp32, W.p, W.aploc, gf, np, L.bj, L.D,
                                 L.S, lam, &pu));
              if (fused) {
                op.code = OP_CG_BETA;
                SSG_CUDA(c, run_dss(s, DSS_CGUPD, fp32, L.n, c->nel, W.aploc, nullptr, c->d_nbreg,
                                    L.dss_ec, mask, nullptr, nullptr, c->d_part, stop, &op, &cg));
              } else {
                op.code = OP_CG_ALPHA;
                SSG_CUDA(c, run_dss(s, DSS_DOT, fp32, L.n, c->nel, W.aploc, W.ap, c->d_nbreg,
                                    L.dss_ec, mask, W.p, nullptr, c->d_part, stop, &op));
                op.code = OP_CG_BETA;
                SSG_CUDA(c, run_cg_update(s, fp32, np, fr + F_ALPHA, x, W.p, W.r, W.ap, dinv,
                                          L.mult, W.z, c->d_part, nb, stop, &op));
              }
              return SSG_OK;
            },
            &wsp->cgloop[slot], &wsp->cgloop_kernels[slot]);
        if (ok) {
          wsp->cgloop_key[slot] = key;
        } else {
          wsp->cgloop_failed = true;
        }
      }
      if (wsp->cgloop[slot]) {
        wsp->cgloop_used[slot] = ++wsp->cgloop_clock;
        SSG_CUDA(c, cudaGraphLaunch(wsp->cgloop[slot], s));
        double iters;
        SSG_TRY(read_flag(c, fr + F_ITER, &iters));
        SSG_TRY(check_interrupt(c));
        // guard + one body (and its guard) per iteration that ran
        const unsigned long long k = 1 + (unsigned long long)std::max(0.0, iters - 1.0) *
                                             (wsp->cgloop_kernels[slot] + 1);
        g_launches += k;
        t_launches += k;
        break;
      }
    }
    // p = beta p + (z - c) (first: p = z - c), masked; aploc = A p
    // (fused: pap = p . aploc and alpha = rdz / pap; first: pap only)
    pu.first = it == 0;
    dop.code = it == 0 ? OP_STORE_PAP : OP_CG_ALPHA;
    SSG_CUDA(c, run_ax(s, L.n, c->nel, 0, helm, fp32, W.p, W.aploc, gf, np, L.bj, L.D, L.S,
                       lam, &pu));
    if (it == 0) {
      // rdz = (r w).p, |r|_w (src/solver.c:58-61) (fused: and alpha)
      PtrList ys;
      ys.p[0] = W.p;
      ys.p[1] = W.r;
      op.code = fused ? OP_CG_INIT_RDZ_ALPHA : OP_CG_INIT_RDZ;
      SSG_CUDA(c, run_dots(s, fp32, np, W.r, ys, 2, L.mult, c->d_part, nb, &op));
    }
    if (fused) {
      // ap = DSS(mask aploc); x += alpha p; r -= alpha ap; z = M^-1 r; beta; err
      op.code = OP_CG_BETA;
      SSG_CUDA(c, run_dss(s, DSS_CGUPD, fp32, L.n, c->nel, W.aploc, nullptr, c->d_nbreg,
                          L.dss_ec, mask, nullptr, nullptr, c->d_part, stop, &op, &cg));
    } else {
      // ap = DSS(mask aploc); alpha = rdz / (p w).ap
      op.code = OP_CG_ALPHA;
      SSG_CUDA(c, run_dss(s, DSS_DOT, fp32, L.n, c->nel, W.aploc, W.ap, c->d_nbreg, L.dss_ec,
                          mask, W.p, nullptr, c->d_part, stop, &op));
      // x += alpha p; r -= alpha ap; z = M^-1 r; beta; err
      op.code = OP_CG_BETA;
      SSG_CUDA(c, run_cg_update(s, fp32, np, fr + F_ALPHA, x, W.p, W.r, W.ap, dinv, L.mult,
                                W.z, c->d_part, nb, stop, &op));
    }
    if (sync_each && (it % 8 == 7)) {
      double done;
      SSG_TRY(read_flag(c, fr + F_DONE, &done));
      SSG_TRY(check_interrupt(c));
      if (done != 0.0) break;
    }
  }
  if (!sync_each) return SSG_OK;   // smoother: outcome stays on the device
  double err, iters;
  SSG_TRY(read_flag(c, fr + F_ERR, &err));
  SSG_TRY(read_flag(c, fr + F_ITER, &iters));
  if (!std::isfinite(err)) return fail(c, SSG_NONFINITE, "non-finite CG residual");
  if (!(err <= eps) && iters >= max_iter) return SSG_MAXITER;
  return SSG_OK;
}

// coarsest level (n = 2): CG-Jacobi, 500 iterations, in one cooperative launch
static ssg_status coarse_solve(ssg_context* c, int L, double* f, double* x, double eps,
                               int max_iter, double rel = 0.0) {
  const DevLevel& C = c->lev[L];
  LevelWork& W = c->ws->w64[L];
  if (C.n != 2) {
    return cg_solve(c, L, SSG_PRESSURE, false, f, x, eps, max_iter, FR_LEVEL0 + L, nullptr,
                    0, false);
  }
  SSG_CUDA(c, run_coarse_cg(c->stream, c->device, c->nel, f, x, (double*)W.r, (double*)W.z,
                            (double*)W.p, (double*)W.aploc, (double*)W.ap, C.gf, C.D,
                            C.dinv_p, C.mult, c->d_pairs, C.nunique, eps, rel, max_iter,
                            c->d_part,
                            c->part_cap, c->d_sc + (FR_LEVEL0 + L) * F_SIZE));
  return SSG_OK;
}

// V-cycle from level L (multigrid_recurse, src/precon.c:238-271)
static ssg_status mg_recurse(ssg_context* c, int L, void* f, void* x, double eps,
                             bool fp32) {
  const int last = c->nlev - 1;
  cudaStream_t s = c->stream;
  if (L == last) {
    // coarsest level: CG-Jacobi to eps, 500 iterations, always FP64
    if (fp32) {
      LevelWork& W64 = c->ws->w64[L];
      const size_t np = c->lev[L].npts;
      SSG_CUDA(c, run_convert(s, np, f, true, W64.f, false));
      SSG_CUDA(c, cudaMemsetAsync(W64.x, 0, np * sizeof(double), s));
      SSG_TRY(coarse_solve(c, L, (double*)W64.f, (double*)W64.x, eps, 500));
      SSG_CUDA(c, run_convert(s, np, W64.x, false, x, true));
      return SSG_OK;
    }
    return coarse_solve(c, L, (double*)f, (double*)x, eps, 500);
  }
  const DevLevel& F = c->lev[L];
  const DevLevel& C = c->lev[L + 1];
  LevelWork& W = fp32 ? c->ws->w32[L] : c->ws->w64[L];
  LevelWork& Wc = fp32 ? c->ws->w32[L + 1] : c->ws->w64[L + 1];
  const void* rin = f;
  if (L == 0) {
    // r = f - A x (compute_residual, src/precon.c:302-309)
    SSG_CUDA(c, run_ax(s, F.n, c->nel, 0, false, fp32, x, W.aploc,
                       fp32 ? (const void*)F.gf32 : (const void*)F.gf, F.npts, nullptr, F.D,
                       F.D, 0.0, nullptr));
    SSG_CUDA(c, run_dss(s, DSS_RESID, fp32, F.n, c->nel, W.aploc, W.rr, c->d_nbreg, F.dss_ec, nullptr,
                        f, nullptr, c->d_part));
    rin = W.rr;
  }
  // restriction: (J^T)^3 then DSS-average at the coarse level
  SSG_CUDA(c, run_tensor3(s, fp32, false, c->nel, F.n, C.n,
                          C.Ar, rin, Wc.tc));
  SSG_CUDA(c, run_dss(s, DSS_AVG, fp32, C.n, c->nel, Wc.tc, Wc.f, c->d_nbreg, C.dss_ec, nullptr,
                      nullptr, nullptr, nullptr));
  SSG_CUDA(c, cudaMemsetAsync(Wc.x, 0, C.npts * (fp32 ? sizeof(float) : sizeof(double)), s));
  SSG_TRY(mg_recurse(c, L + 1, Wc.f, Wc.x, eps, fp32));
  // prolongation J^3 and x += e
  SSG_CUDA(c, run_tensor3(s, fp32, true, c->nel, C.n, F.n,
                          C.Ap, Wc.x, x));
  // post-smoothing: CG-Jacobi, 15 iterations, stop at eps.  An n = 4 level
  // (262,144 points at 4096 elements) is too small to keep the device busy
  // with one launch per kernel, so in FP64 its whole CG runs in one
  // cooperative launch (0.3 ms less per C2 solve).  The FP32-storage
  // V-cycle keeps the fused two-kernel iteration: with FP32 storage the
  // cooperative form (the unfused arithmetic, ap stored before the update)
  // took the outer FCG 16 iterations instead of 11 on the C2 solve.

  if (F.n == 4 && !fp32) {
    LevelCgRun R;
    R.nel = c->nel;
    R.f = f;
    R.x = x;
    R.r = W.r;
    R.z = W.z;
    R.p = W.p;
    R.aploc = W.aploc;
    R.ap = W.ap;
    R.gf = fp32 ? (const void*)F.gf32 : (const void*)F.gf;
    R.D = F.D;
    R.dinv = fp32 ? (const void*)F.dinv_p32 : (const void*)F.dinv_p;
    R.mult = F.mult;
    R.pairs = c->d_pairs;
    R.nunique = F.nunique;
    R.eps = eps;
    R.max_iter = 15;
    R.part = c->d_part;
    R.part_cap = c->part_cap;
    SSG_CUDA(c, run_level_cg(s, c->device, F.n, fp32, R));
    return SSG_OK;
  }
  return cg_solve(c, L, SSG_PRESSURE, fp32, f, x, eps, 15, FR_LEVEL0 + L, nullptr, 0, false);
}

// z = M^-1 r: Jacobi then one V-cycle (multigrid_preconditioner,
// src/precon.c:227-236)
ssg_status mg_apply(ssg_context* c, const double* r, double* z, double eps) {
  SSG_TRY(ensure_workspace(c));
  const bool fp32 = c->precision == SSG_PRECISION_MIXED;
  const DevLevel& L = c->lev[0];
  const size_t np = L.npts;
  const int nb = vec_blocks(np);
  cudaStream_t s = c->stream;
  void* f0 = (void*)r;
  void* x0 = z;
  if (fp32) {
    f0 = c->ws->w32[0].f;
    x0 = c->ws->w32[0].x;
    SSG_CUDA(c, run_convert(s, np, r, false, f0, true));
  }
  SSG_CUDA(c, run_jacobi(s, fp32, np, f0, fp32 ? (const void*)L.dinv_p32 : (const void*)L.dinv_p,
                         L.mult, x0, c->d_part,
                         nb));
  if (c->nlev > 1) SSG_TRY(mg_recurse(c, 0, f0, x0, eps, fp32));
  if (fp32) SSG_CUDA(c, run_convert(s, np, x0, true, z, false));
  return SSG_OK;
}

// z = M^-1 r for the FCG workspace vectors (r = ws->r, z = ws->z): replays
// the captured V-cycle graph, capturing it on first use for this eps and
// precision.  A capture the driver refuses falls back to direct launches.
static ssg_status vcycle_ws(ssg_context* c, double eps) {
  Workspace* w = c->ws;
  if (!c->graphs || w->vcycle_failed) return mg_apply(c, w->r, w->z, eps);
  cudaStream_t s = c->stream;
  if (w->vcycle && (w->vcycle_eps != eps || w->vcycle_precision != c->precision))
    invalidate_graphs(c);
  if (!w->vcycle && (w->warm_eps != eps || w->warm_precision != c->precision)) {
    // first V-cycle of this configuration runs directly: one-time kernel
    // attribute settings happen outside any capture
    w->warm_eps = eps;
    w->warm_precision = c->precision;
    return mg_apply(c, w->r, w->z, eps);
  }
  if (!w->vcycle) {
    const unsigned long long before = t_launches;
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      w->vcycle_failed = true;
      return mg_apply(c, w->r, w->z, eps);
    }
    const ssg_status st = mg_apply(c, w->r, w->z, eps);
    const cudaError_t ce = cudaStreamEndCapture(s, &g);
    const unsigned long long captured = t_launches - before;
    g_launches -= captured;   // recorded, not launched
    t_launches = before;
    cudaGraphExec_t ex = nullptr;
    if (st != SSG_OK || ce != cudaSuccess || !g ||
        cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) {
      cudaGetLastError();
      if (g) cudaGraphDestroy(g);
      w->vcycle_failed = true;
      c->err.clear();
      return mg_apply(c, w->r, w->z, eps);
    }
    cudaGraphDestroy(g);
    w->vcycle = ex;
    w->vcycle_eps = eps;
    w->vcycle_precision = c->precision;
    w->vcycle_kernels = captured;
  }
  SSG_CUDA(c, cudaGraphLaunch(w->vcycle, s));
  g_launches += w->vcycle_kernels;
  t_launches += w->vcycle_kernels;
  return SSG_OK;
}

ssg_status fcg_solve(ssg_context* c, const double* f, double* u, double eps, int max_iter,
                     ssg_solve_info* info) {
  SSG_TRY(ensure_workspace(c));
  Workspace* w = c->ws;
  const DevLevel& L = c->lev[0];
  const size_t np = L.npts;
  const int nb = vec_blocks(np);
  const int nbd = dss_grid(L.n, c->nel);
  cudaStream_t s = c->stream;
  double* fr = c->d_sc + FR_FCG * F_SIZE;
  const int hcap = info && info->history && info->history_cap > 0
                       ? std::min(std::min(info->history_cap, max_iter), w->hist_cap)
                       : 0;
  ScalarOp op;
  op.sums = c->d_sums;
  op.counter = c->d_counter;
  op.frame = fr;
  op.pressure = 1;
  op.nunique = L.nunique;
  op.eps = eps;
  op.max_iter = max_iter;
  op.hist = hcap ? w->hist : nullptr;
  op.hist_cap = hcap;

  // r = f - A u; subtract_nullspace(r)
  SSG_CUDA(c, run_ax(s, L.n, c->nel, 0, false, false, u, w->aploc, L.gf, np, nullptr, L.D,
                     L.D, 0.0, nullptr));
  op.code = OP_NULL_C;
  SSG_CUDA(c, run_dss(s, DSS_RESID, false, L.n, c->nel, w->aploc, w->r, c->d_nbreg, L.dss_ec, nullptr,
                      f, nullptr, c->d_part, nullptr, &op));
  SSG_CUDA(c, run_add_const(s, false, np, w->r, fr + F_C, 1));
  PtrList ys;
  ys.p[0] = w->r;
  op.code = OP_ERR0;
  SSG_CUDA(c, run_dots(s, false, np, w->r, ys, 1, L.mult, c->d_part, nb, &op));

  int pslot[11], aslot[10];
  for (int k = 0; k < 11; ++k) pslot[k] = k;
  for (int k = 0; k < 10; ++k) aslot[k] = k;
  const int mmax = 10;
  // Iteration j: the window m = min(j, max(1, j mod 11)) and the rotation of
  // the direction slots; enqueue = false only advances the slots (the
  // iteration's launches are already in a graph).  vcycle_graph: the
  // V-cycle from its own graph (direct launches inside an iteration graph).
  auto iteration = [&](int j, bool enqueue, bool vcycle_graph) -> ssg_status {
    int m = std::max(1, j % (mmax + 1));
    m = std::min(m, j);
    if (enqueue) {
      if (vcycle_graph)
        SSG_TRY(vcycle_ws(c, eps));
      else
        SSG_TRY(mg_apply(c, w->r, w->z, eps));
      // subtract_nullspace(z)
      op.code = OP_NULL_C;
      SSG_CUDA(c, run_wsum(s, false, np, w->z, L.mult, c->d_part, nb, &op));
      SSG_CUDA(c, run_add_const(s, false, np, w->z, fr + F_C, 1));
      // beta_k = (z w).ap_k / pap_k
      if (m > 0) {
        PtrList yb;
        for (int k = 0; k < m; ++k) {
          yb.p[k] = w->AP[aslot[k]];
          op.pap_idx[k] = aslot[k];
        }
        op.m = m;
        op.code = OP_FCG_BETA;
        SSG_CUDA(c, run_dots(s, false, np, w->z, yb, m, L.mult, c->d_part, nb, &op));
      }
    }
    // shift the directions and form p0 = z - sum beta_k p_k
    const int tail = pslot[m];
    for (int k = m; k > 0; --k) pslot[k] = pslot[k - 1];
    pslot[0] = tail;
    double* p0 = w->P[pslot[0]];
    if (enqueue) {
      SSG_CUDA(c, cudaMemcpyAsync(p0, w->z, np * sizeof(double), cudaMemcpyDeviceToDevice, s));
      if (m > 0) {
        PtrList yp;
        for (int k = 0; k < m; ++k) yp.p[k] = w->P[pslot[k + 1]];
        SSG_CUDA(c, run_combine(s, np, p0, yp, fr + F_FBETA, m, -1.0));
      }
    }
    // shift the ap history
    int m2 = std::max(1, (j + 1) % (mmax + 1));
    m2 = std::min(m2, j + 1);
    const int atail = aslot[m2 - 1];
    for (int k = m2 - 1; k > 0; --k) aslot[k] = aslot[k - 1];
    aslot[0] = atail;
    if (!enqueue) return SSG_OK;
    double* ap0 = w->AP[aslot[0]];
    // ap0 = A p0; pap0 and alpha = (p0 w).r / pap0
    SSG_CUDA(c, run_ax(s, L.n, c->nel, 0, false, false, p0, w->aploc, L.gf, np, nullptr, L.D,
                       L.D, 0.0, nullptr));
    op.pap_idx[0] = aslot[0];
    op.code = OP_FCG_ALPHA;
    SSG_CUDA(c, run_dss(s, DSS_DOT2, false, L.n, c->nel, w->aploc, ap0, c->d_nbreg, L.dss_ec, nullptr,
                        p0, w->r, c->d_part, nullptr, &op));
    // u += alpha p0; r -= alpha ap0; err
    op.code = OP_FCG_ERR;
    SSG_CUDA(c, run_fcg_update(s, np, fr + F_ALPHA, u, p0, w->r, ap0, L.mult, c->d_part, nb,
                               &op));
    return SSG_OK;
  };

  // Graph mode: once a configuration (eps, precision, iteration cap,
  // history) has run directly, every iteration is one graph launch -- the
  // graph of its window state, captured on first use -- and iterations are
  // enqueued ahead in chunks of 16, 32, 64, ... with one host
  // synchronisation per chunk (a C2 solve of 11 iterations: one).
  // Iterations past the stop skip their work on the device.  Results are
  // those of the direct launches (the same kernels in the same order).
  const bool same_cfg = w->fcg_eps == eps && w->fcg_precision == c->precision &&
                        w->fcg_max_iter == max_iter && w->fcg_hcap == hcap && w->fcg_u == u;
  if (!same_cfg) {
    drop_iteration_graphs(w);
    w->fcg_eps = eps;
    w->fcg_precision = c->precision;
    w->fcg_max_iter = max_iter;
    w->fcg_hcap = hcap;
    w->fcg_u = u;
  }
  const bool graph_mode = c->graphs && !w->fcg_failed && w->fcg_warm > 0 && !w->vcycle_failed;
  bool graph_mode_used = false;
  int graph_iters = 0;   // iteration graphs enqueued (each runs its guard)
  if (!graph_mode) {
    for (int j = 0; j < max_iter; ++j) {
      SSG_TRY(iteration(j, true, true));
      double done;
      SSG_TRY(read_flag(c, fr + F_DONE, &done));
      if (done != 0.0) break;
      SSG_TRY(check_interrupt(c));
    }
    ++w->fcg_warm;
  } else {
    graph_mode_used = true;
    int j = 0, chunk = 16;
    while (j < max_iter) {
      const int end = std::min(max_iter, j + chunk);
      for (; j < end; ++j) {
        const int key = j == 0 ? 0 : 1 + (j - 1) % (Workspace::kFcgStates - 1);
        if (!w->fcg[key]) {
          int ps[11], as[10];
          std::memcpy(ps, pslot, sizeof(ps));
          std::memcpy(as, aslot, sizeof(as));
          const bool ok = build_conditional_graph(
              c, false, fr + F_DONE, [&] { return iteration(j, true, false); }, &w->fcg[key],
              &w->fcg_kernels[key]);
          std::memcpy(pslot, ps, sizeof(ps));
          std::memcpy(aslot, as, sizeof(as));
          if (!ok) {
            // finish this solve with direct launches
            w->fcg_failed = true;
            w->fcg[key] = nullptr;
            for (; j < max_iter; ++j) {
              SSG_TRY(iteration(j, true, true));
              double done;
              SSG_TRY(read_flag(c, fr + F_DONE, &done));
              if (done != 0.0) break;
              SSG_TRY(check_interrupt(c));
            }
            break;
          }
        }
        SSG_TRY(iteration(j, false, false));
        SSG_CUDA(c, cudaGraphLaunch(w->fcg[key], s));
        ++graph_iters;
      }
      if (w->fcg_failed) break;
      double done;
      SSG_TRY(read_flag(c, fr + F_DONE, &done));
      if (done != 0.0) break;
      SSG_TRY(check_interrupt(c));
      chunk *= 2;
    }
  }
  double h[F_SIZE];
  SSG_CUDA(c, cudaMemcpyAsync(c->h_pin, fr, F_SIZE * sizeof(double), cudaMemcpyDeviceToHost,
                              s));
  SSG_CUDA(c, cudaStreamSynchronize(s));
  std::memcpy(h, c->h_pin, sizeof(h));
  if (graph_mode_used) {
    // launch count: every enqueued graph's guard, the bodies of the
    // iterations that ran
    unsigned long long k = (unsigned long long)graph_iters;
    const int ran = (int)h[F_ITER];
    for (int j = 0; j < ran && j < graph_iters; ++j)
      k += w->fcg_kernels[j == 0 ? 0 : 1 + (j - 1) % (Workspace::kFcgStates - 1)];
    g_launches += k;
    t_launches += k;
  }
  if (info) {
    info->iterations = (int)h[F_ITER];
    info->residual = h[F_ERR];
    info->initial_residual = h[F_ERR0];
    info->history_len = std::min((int)h[F_ITER], hcap);
    if (hcap)
      SSG_CUDA(c, cudaMemcpy(info->history, w->hist, info->history_len * sizeof(double),
                             cudaMemcpyDeviceToHost));
  }
  if (!std::isfinite(h[F_ERR])) return fail(c, SSG_NONFINITE, "non-finite FCG residual");
  if (!(h[F_ERR] <= eps)) return SSG_MAXITER;
  return SSG_OK;
}

}  // namespace ssg
