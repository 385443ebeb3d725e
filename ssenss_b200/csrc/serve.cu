// Serving loop: independent Helmholtz / Poisson solve requests of different
// meshes and orders, continuously admitted and overlapped on one GPU.
//
// No reference counterpart: the reference solves one mesh per process.
// Every request runs the same device path as a direct call
// (ssg_solve_poisson_cg: FCG + p-multigrid, nullspace removed; or
// ssg_solve_helmholtz_cg: Jacobi CG), so its result does not depend on what
// else is in flight.
//
//   * Residency: a context (mesh, factors at every level, Krylov workspace)
//     stays on the device after its request, keyed by the caller's mesh key
//     and precision, and serves the next request on that mesh without set-up.
//   * Admission: strict arrival order.  The head request starts when a slot
//     is free and its context fits the HBM budget -- an idle resident
//     context of the same key, or a new one whose estimated bytes
//     (ssg_request_bytes) fit after evicting idle contexts least recently
//     used first.  A request larger than the whole budget is rejected.
//   * Continuous batching: up to max_active requests run at once, each on
//     its own CUDA stream and host thread; a request that arrives while
//     others are on the GPU starts as soon as a slot and memory free up, and
//     its kernels interleave with theirs on the device.
//   * Shared launches (ssg_server_set_batching): when the head of the queue
//     is a small Helmholtz request and the requests right behind it are
//     small Helmholtz requests of the same order whose meshes have idle
//     resident contexts, up to max_batch of them run as one segmented solve
//     (seg_solve, batch.cu): their resident level-0 data is copied device to
//     device into one concatenated level (a per-worker arena, reused), and
//     every operator and DSS launch of an iteration serves all of them, each
//     with its own lambda, CG scalars and stop.  Off by default: a batched
//     result agrees with the request's solo result to rounding, not bitwise.
//   * Cancellation and deadlines: queued requests end at once; running ones
//     at their next host synchronisation point (once per outer iteration).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "ssg_internal.h"
#include "ssg_kernels.h"

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct Request {
  unsigned long long id = 0;
  ssg_request d{};
  std::vector<double> vert;
  std::vector<int> neigh;
  std::vector<double> rhs;
  double* out = nullptr;
  bool walls = false;          // a wall code in the neighbour table
  size_t bytes_est = 0;
  double t_submit = 0, t_start = 0, t_done = 0, deadline = 0;
  bool done = false;
  volatile int cancel = 0;
  ssg_status result = SSG_OK;
  ssg_solve_info info{};
};

struct Resident {
  unsigned long long key = 0;
  int precision = 0;
  ssg_context* ctx = nullptr;
  size_t bytes = 0;
  bool busy = false;
  double last_used = 0;
};

}  // namespace

struct ssg_server {
  int device = 0;
  size_t budget = 0;
  int max_active = 1;
  int max_batch = 1;                 // > 1: shared-launch Helmholtz batches
  size_t batch_points = 0;           // largest request (points) that batches
  std::mutex mu;
  std::condition_variable cv;        // queue / budget / completion changes
  std::deque<Request*> queue;
  std::unordered_map<unsigned long long, std::unique_ptr<Request>> reqs;
  std::list<Resident> resident;
  size_t in_use = 0, peak = 0;
  int active = 0, max_active_seen = 0;
  unsigned long long next_id = 1;
  bool stop = false;
  std::vector<std::thread> workers;
  // statistics
  std::vector<double> lat_ms, queue_ms;
  unsigned long long submitted = 0, completed = 0, failed = 0, cancelled = 0, rejected = 0;
  unsigned long long hits = 0, misses = 0, evictions = 0;
  unsigned long long batches = 0, batched = 0;
  double t_first = 0, t_last = 0;
};

namespace {

size_t estimate_bytes(int n, int nel, int precision) {
  int orders[SSG_MAXLEV];
  const int nlev = ssg::level_orders(n, orders);
  const size_t np0 = (size_t)n * n * n * nel;
  size_t b = 0;
  for (int l = 0; l < nlev; ++l) {
    const int m = orders[l];
    const size_t np = (size_t)m * m * m * nel;
    const int I = m > 2 ? m - 2 : 0;
    // gf 48, bj, kdiag, dinv_p, dinv_h 32, mult 1, gf32 24, dinv_p32 4
    b += np * 109;
    b += (size_t)nel * (12 * I * 4 + 64) * sizeof(int);   // DSS edge/corner records
    b += np * sizeof(int);                                 // DSS gather words
    b += np * 9 * sizeof(double);                          // level work vectors
    if (precision == SSG_PRECISION_MIXED) b += np * 9 * sizeof(float);
  }
  b += (size_t)nel * (52 + 26 + 26) * sizeof(int);   // pairing, neighbour tables
  b += np0 * (8 + 8 + 8);                  // inverse mass, det J, workspace scratch
  b += np0 * 4 * 8;                        // staging (one field per slot)
  b += np0 * 24 * 8;                       // FCG: r, z, A p local, 11 + 10 directions
  const size_t vb = std::min((np0 + 255) / 256, (size_t)148 * 64);
  b += (std::max(16 * vb, (size_t)4 * 148 * 64) + 64) * 8;   // reduction partials
  b += 8192 * 8 + (1 << 20);               // history, small buffers
  return b;
}

void finish_request(ssg_server* S, Request* r, ssg_status st) {
  r->result = st;
  r->t_done = now_s();
  r->done = true;
  if (st == SSG_OK || st == SSG_MAXITER) {
    ++S->completed;
    S->lat_ms.push_back(1e3 * (r->t_done - r->t_submit));
    S->queue_ms.push_back(1e3 * ((r->t_start > 0 ? r->t_start : r->t_done) - r->t_submit));
    S->t_last = std::max(S->t_last, r->t_done);
  } else if (st == SSG_ERR_CANCELLED) {
    ++S->cancelled;
  } else if (st == SSG_ERR_BUDGET) {
    ++S->rejected;
  } else {
    ++S->failed;
  }
}

bool batchable(const ssg_server* S, const Request* r) {
  return S->max_batch > 1 && r->d.lambda > 0.0 && !r->d.relative && !r->cancel && !r->walls &&
         (size_t)r->d.nel * r->d.n * r->d.n * r->d.n <= S->batch_points;
}

// evict idle contexts, least recently used first, until `need` fits; false
// when it cannot fit yet (lock held)
bool make_room(ssg_server* S, size_t need, std::vector<ssg_context*>& evict) {
  while (S->in_use + need > S->budget) {
    auto lru = S->resident.end();
    for (auto it = S->resident.begin(); it != S->resident.end(); ++it)
      if (!it->busy && (lru == S->resident.end() || it->last_used < lru->last_used)) lru = it;
    if (lru == S->resident.end()) break;
    S->in_use -= lru->bytes;
    evict.push_back(lru->ctx);
    S->resident.erase(lru);
    ++S->evictions;
  }
  return S->in_use + need <= S->budget;
}

// Decide for the head of the queue (lock held).  Returns the request to run
// and the resident slot it uses (new ones already reserved), or nullptr.
// A shared-launch batch: *batch receives its requests (the head first) and
// *batch_slots the resident context each reads (marked busy); *slot stays
// null.
Request* admit(ssg_server* S, Resident** slot, std::vector<ssg_context*>& evict,
               std::vector<Request*>* batch, std::vector<Resident*>* batch_slots) {
  while (!S->queue.empty()) {
    Request* r = S->queue.front();
    if (r->cancel) {
      S->queue.pop_front();
      finish_request(S, r, SSG_ERR_CANCELLED);
      S->cv.notify_all();
      continue;
    }
    if (r->deadline > 0 && now_s() > r->deadline) {
      S->queue.pop_front();
      finish_request(S, r, SSG_ERR_TIMEOUT);
      S->cv.notify_all();
      continue;
    }
    if (S->active >= S->max_active) return nullptr;
    // small Helmholtz requests of one order queued back to back, each with
    // an idle resident context of its mesh (or sharing one with an earlier
    // member: the level data is only read): one shared-launch batch
    // (arrival order kept: only the run at the head)
    if (batchable(S, r)) {
      std::vector<Request*> b;
      std::vector<Resident*> sl;
      for (size_t i = 0; i < S->queue.size() && (int)b.size() < S->max_batch; ++i) {
        Request* q = S->queue[i];
        if (!batchable(S, q) || q->d.n != r->d.n || q->d.mesh_key == 0) break;
        Resident* x = nullptr;
        for (size_t k = 0; k < b.size() && !x; ++k)
          if (b[k]->d.mesh_key == q->d.mesh_key) x = sl[k];
        if (!x)
          for (auto& y : S->resident)
            if (!y.busy && y.ctx && y.key == q->d.mesh_key) {
              x = &y;
              break;
            }
        if (!x) break;
        x->busy = true;
        b.push_back(q);
        sl.push_back(x);
      }
      if (b.size() >= 2) {
        for (size_t k = 0; k < b.size(); ++k) S->queue.pop_front();
        S->hits += b.size();
        ++S->batches;
        S->batched += b.size();
        *batch = std::move(b);
        *batch_slots = std::move(sl);
        return r;
      }
      for (Resident* x : sl) x->busy = false;
    }
    // an idle resident context of this mesh and precision
    if (r->d.mesh_key != 0)
      for (auto& x : S->resident)
        if (!x.busy && x.key == r->d.mesh_key && x.precision == r->d.precision) {
          x.busy = true;
          *slot = &x;
          ++S->hits;
          S->queue.pop_front();
          return r;
        }
    const size_t need = r->bytes_est;
    if (need > S->budget) {
      S->queue.pop_front();
      finish_request(S, r, SSG_ERR_BUDGET);
      S->cv.notify_all();
      continue;
    }
    // evict idle contexts, least recently used first, until it fits
    if (!make_room(S, need, evict)) return nullptr;   // wait for a completion
    S->in_use += need;
    S->peak = std::max(S->peak, S->in_use);
    Resident res;
    res.key = r->d.mesh_key;
    res.precision = r->d.precision;
    res.bytes = need;
    res.busy = true;
    S->resident.push_back(res);
    *slot = &S->resident.back();
    ++S->misses;
    S->queue.pop_front();
    return r;
  }
  return nullptr;
}

ssg_status run_request(ssg_server* S, Request* r, Resident* slot) {
  ssg_context* c = slot->ctx;
  if (!c) {
    SSG_TRY(ssg_create(S->device, &c));
    slot->ctx = c;
    ssg_set_setup_options(c, SSG_SETUP_NO_DEALIAS | SSG_SETUP_NO_PARTICLES |
                                 SSG_SETUP_OPPOSITE_PAIRING);
    ssg_status st = ssg_setup_mesh(c, r->d.n, r->d.nel, r->vert.data(), r->neigh.data());
    if (st != SSG_OK) {
      // a context whose set-up failed never serves: the worker then drops
      // the slot, so later requests with this mesh key set up afresh
      ssg_destroy(c);
      slot->ctx = nullptr;
      return st;
    }
  }
  c->cancel = &r->cancel;
  c->deadline = r->deadline;
  const bool helm = r->d.lambda > 0.0;
  // lambda = (11/6) / (dt visc): dt = 11 / (6 lambda), visc = 1
  SSG_TRY(ssg_set_parameters(c, helm ? 11.0 / (6.0 * r->d.lambda) : 1.0, 1.0, 1.0));
  SSG_TRY(ssg_set_precision(c, helm ? SSG_PRECISION_FP64 : r->d.precision));
  double eps = r->d.eps;
  if (r->d.relative) {
    double ff = 0.0;
    SSG_TRY(ssg_global_dot_product(c, r->rhs.data(), r->rhs.data(), &ff));
    eps = r->d.eps * std::sqrt(ff);
  }
  const int max_iter = r->d.max_iter > 0 ? r->d.max_iter : 5000;
  std::memset(r->out, 0, sizeof(double) * (size_t)r->d.nel * r->d.n * r->d.n * r->d.n);
  r->info = ssg_solve_info{};
  ssg_status st = helm ? ssg_solve_helmholtz_cg(c, SSG_X_VELOCITY, r->rhs.data(), r->out, eps,
                                                max_iter, &r->info)
                       : ssg_solve_poisson_cg(c, r->rhs.data(), r->out, eps, max_iter,
                                              &r->info);
  c->cancel = nullptr;
  c->deadline = 0.0;
  return st;
}

// Per-worker device arena of shared-launch batches: the concatenated
// level-0 data and the segmented solve's scratch, grown to the largest batch
// and reused; its own context gives the stream and error reporting.
struct BatchArena {
  ssg_context* c = nullptr;
  ssg::SegScratch W;
  double *gf = nullptr, *bj = nullptr, *kdiag = nullptr, *det = nullptr;
  uint8_t* mult = nullptr;
  int* dss = nullptr;
  size_t cap_points = 0, cap_dss = 0;
  void release() {
    ssg::seg_scratch_free(W);
    void* ps[] = {gf, bj, kdiag, det, mult, dss};
    for (void* p : ps)
      if (p) cudaFree(p);
    gf = bj = kdiag = det = nullptr;
    mult = nullptr;
    dss = nullptr;
    cap_points = cap_dss = 0;
    if (c) ssg_destroy(c);
    c = nullptr;
  }
};

template <typename T>
ssg_status arena_alloc(ssg_context* c, T** p, size_t count) {
  if (*p) cudaFree(*p);
  *p = nullptr;
  void* q = nullptr;
  if (cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    return ssg::fail(c, SSG_ERR_NOMEM, "batch arena");
  }
  *p = static_cast<T*>(q);
  return SSG_OK;
}

// The batch's level-0 data concatenated in the arena (device to device from
// the resident contexts, DSS map indices shifted), then one segmented solve.
ssg_status run_batch(ssg_server* S, BatchArena& A, std::vector<Request*>& b,
                     std::vector<Resident*>& sl) {
  if (!A.c) SSG_TRY(ssg_create(S->device, &A.c));
  ssg_context* c = A.c;
  const int n = b[0]->d.n;
  const size_t nt = (size_t)n * n * n;
  std::vector<int> first{0};
  std::vector<double> f, lam, eps;
  for (Request* r : b) {
    first.push_back(first.back() + r->d.nel);
    f.insert(f.end(), r->rhs.begin(), r->rhs.end());
    lam.push_back(r->d.lambda);
    eps.push_back(r->d.eps);
  }
  const int nel = first.back();
  const size_t np = (size_t)nel * nt;
  const size_t ndss = ssg::dss_map_records_offset(np) + ssg::dss_record_ints(n) * nel;
  // grown at most to the largest batch the settings allow (a cudaFree on
  // growth synchronises the device), so sized for that the first time
  const size_t full = std::min<size_t>((size_t)S->max_batch * S->batch_points, (size_t)1 << 24);
  if (np > A.cap_points) {
    const size_t cap = std::max(np, full);
    A.cap_points = 0;
    SSG_TRY(arena_alloc(c, &A.gf, 6 * cap));
    SSG_TRY(arena_alloc(c, &A.bj, cap));
    SSG_TRY(arena_alloc(c, &A.kdiag, cap));
    SSG_TRY(arena_alloc(c, &A.det, cap));
    SSG_TRY(arena_alloc(c, &A.mult, cap));
    A.cap_points = cap;
  }
  if (ndss > A.cap_dss) {
    // records per point are largest at the smallest order (n = 2: 64 ints
    // per 8 points)
    const size_t cap = std::max(ndss, ssg::dss_map_records_offset(full) + 8 * full);
    A.cap_dss = 0;
    SSG_TRY(arena_alloc(c, &A.dss, cap));
    A.cap_dss = cap;
  }
  cudaStream_t s = c->stream;
  for (size_t k = 0; k < b.size(); ++k) {
    const ssg::DevLevel& D = sl[k]->ctx->lev[0];
    const size_t P = (size_t)first[k] * nt, m = D.npts;
    for (int a = 0; a < 6; ++a)
      SSG_CUDA(c, cudaMemcpyAsync(A.gf + a * np + P, D.gf + a * m, m * sizeof(double),
                                  cudaMemcpyDeviceToDevice, s));
    SSG_CUDA(c, cudaMemcpyAsync(A.bj + P, D.bj, m * sizeof(double), cudaMemcpyDeviceToDevice, s));
    SSG_CUDA(c, cudaMemcpyAsync(A.kdiag + P, D.kdiag, m * sizeof(double),
                                cudaMemcpyDeviceToDevice, s));
    SSG_CUDA(c, cudaMemcpyAsync(A.det + P, D.det, m * sizeof(double), cudaMemcpyDeviceToDevice,
                                s));
    SSG_CUDA(c, cudaMemcpyAsync(A.mult + P, D.mult, m, cudaMemcpyDeviceToDevice, s));
    SSG_CUDA(c, ssg::run_dss_map_shift(s, D.dss_ec, n, b[k]->d.nel, A.dss, P, np, first[k]));
  }
  const ssg::DevLevel& D0 = sl[0]->ctx->lev[0];
  ssg::SegLevel L;
  L.n = n;
  L.nel = nel;
  L.nt = nt;
  L.npts = np;
  L.gf = A.gf;
  L.bj = A.bj;
  L.kdiag = A.kdiag;
  L.rho = D0.rho;
  L.det = A.det;
  L.mask = nullptr;     // batched meshes have no walls
  L.D = D0.D;
  L.S = D0.S;
  L.mult = A.mult;
  L.dss = A.dss;
  std::vector<double> u(np, 0.0);
  std::vector<ssg_solve_info> info(b.size());
  int max_iter = 0;
  for (Request* r : b) max_iter = std::max(max_iter, r->d.max_iter > 0 ? r->d.max_iter : 5000);
  c->cancel = &b[0]->cancel;
  const ssg_status st = ssg::seg_solve(c, L, A.W, (int)b.size(), first.data(), lam.data(),
                                       f.data(), u.data(), eps.data(), max_iter, info.data());
  c->cancel = nullptr;
  if (st != SSG_OK && st != SSG_MAXITER) return st;
  for (size_t k = 0; k < b.size(); ++k) {
    Request* r = b[k];
    std::memcpy(r->out, u.data() + (size_t)first[k] * nt, sizeof(double) * r->d.nel * nt);
    r->info = info[k];
  }
  return SSG_OK;
}

void worker(ssg_server* S) {
  cudaSetDevice(S->device);
  BatchArena arena;
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    Resident* slot = nullptr;
    std::vector<ssg_context*> evict;
    std::vector<Request*> batch;
    std::vector<Resident*> batch_slots;
    Request* r = nullptr;
    S->cv.wait(lk, [&] {
      if (S->stop && S->queue.empty()) return true;
      r = admit(S, &slot, evict, &batch, &batch_slots);
      return r != nullptr || !evict.empty();
    });
    if (!r && evict.empty() && S->stop && S->queue.empty()) {
      lk.unlock();
      arena.release();
      return;
    }
    if (!r) {
      lk.unlock();
      for (ssg_context* c : evict) ssg_destroy(c);
      lk.lock();
      S->cv.notify_all();
      continue;
    }
    ++S->active;
    S->max_active_seen = std::max(S->max_active_seen, S->active);
    r->t_start = now_s();
    if (!batch.empty()) {
      for (Request* q : batch) q->t_start = r->t_start;
      lk.unlock();
      for (ssg_context* c : evict) ssg_destroy(c);
      const ssg_status bst = run_batch(S, arena, batch, batch_slots);
      lk.lock();
      --S->active;
      const double now = now_s();
      for (Resident* x : batch_slots) {
        x->busy = false;
        x->last_used = now;
      }
      for (Request* q : batch) {
        // each request's own outcome: its segment's stop
        ssg_status qs = bst;
        if (bst == SSG_OK && !(q->info.residual <= q->d.eps)) qs = SSG_MAXITER;
        finish_request(S, q, qs);
      }
      S->cv.notify_all();
      continue;
    }
    lk.unlock();
    for (ssg_context* c : evict) ssg_destroy(c);
    const ssg_status st = run_request(S, r, slot);
    size_t actual = 0;
    if (slot->ctx) ssg_memory_info(slot->ctx, &actual);
    lk.lock();
    --S->active;
    if (slot->ctx && st != SSG_ERR_CUDA && st != SSG_ERR_NOMEM) {
      // account the context's real footprint from now on
      if (actual > 0) {
        S->in_use = S->in_use - slot->bytes + actual;
        slot->bytes = actual;
        S->peak = std::max(S->peak, S->in_use);
      }
      slot->busy = false;
      slot->last_used = now_s();
    } else {
      // a failed set-up or device error: drop the context
      ssg_context* dead = slot->ctx;
      S->in_use -= slot->bytes;
      for (auto it = S->resident.begin(); it != S->resident.end(); ++it)
        if (&*it == slot) {
          S->resident.erase(it);
          break;
        }
      lk.unlock();
      if (dead) ssg_destroy(dead);
      lk.lock();
    }
    finish_request(S, r, st);
    S->cv.notify_all();
  }
}

double percentile(std::vector<double> v, double p) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  // nearest rank
  size_t k = (size_t)std::ceil(p / 100.0 * (double)v.size());
  k = std::max<size_t>(1, std::min(k, v.size()));
  return v[k - 1];
}

}  // namespace

extern "C" {

size_t ssg_request_bytes(int n, int nel, int precision) {
  if (n < 2 || n > 12 || nel <= 0) return 0;
  return estimate_bytes(n, nel, precision);
}

ssg_status ssg_server_create(int device, size_t hbm_budget, int max_active, ssg_server** out) {
  if (!out || max_active < 1 || max_active > 256 || hbm_budget == 0) return SSG_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return SSG_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) return SSG_ERR_ARG;
  ssg_server* S = new ssg_server();
  S->device = device;
  S->budget = hbm_budget;
  S->max_active = max_active;
  for (int i = 0; i < max_active; ++i) S->workers.emplace_back(worker, S);
  *out = S;
  return SSG_OK;
}

ssg_status ssg_server_set_batching(ssg_server* S, int max_batch, size_t max_points) {
  if (!S || max_batch < 1 || max_batch > 1024) return SSG_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  S->max_batch = max_batch;
  S->batch_points = max_points;
  S->cv.notify_all();
  return SSG_OK;
}

ssg_status ssg_server_submit(ssg_server* S, const ssg_request* d, const double* rhs,
                             double* solution, unsigned long long* id) {
  if (!S || !d || !rhs || !solution || !id) return SSG_ERR_ARG;
  if (d->n < 2 || d->n > 12 || d->nel <= 0 || !d->vertices || !d->neigh || !(d->eps > 0.0) ||
      d->lambda < 0.0 ||
      (d->precision != SSG_PRECISION_FP64 && d->precision != SSG_PRECISION_MIXED))
    return SSG_ERR_ARG;
  auto r = std::make_unique<Request>();
  r->d = *d;
  const size_t np = (size_t)d->nel * d->n * d->n * d->n;
  r->vert.assign(d->vertices, d->vertices + 24 * (size_t)d->nel);
  r->neigh.assign(d->neigh, d->neigh + 26 * (size_t)d->nel);
  for (int v : r->neigh) r->walls = r->walls || v < 0;
  r->d.vertices = nullptr;
  r->d.neigh = nullptr;
  r->rhs.assign(rhs, rhs + np);
  r->out = solution;
  r->bytes_est = estimate_bytes(d->n, d->nel, d->precision);
  r->t_submit = now_s();
  r->deadline = d->deadline_ms > 0 ? r->t_submit + 1e-3 * d->deadline_ms : 0.0;
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->stop) return SSG_ERR_STATE;
  r->id = S->next_id++;
  *id = r->id;
  if (S->submitted == 0) S->t_first = r->t_submit;
  ++S->submitted;
  S->queue.push_back(r.get());
  S->reqs.emplace(r->id, std::move(r));
  S->cv.notify_all();
  return SSG_OK;
}

ssg_status ssg_server_wait(ssg_server* S, unsigned long long id, double timeout_ms,
                           ssg_status* result, ssg_solve_info* info) {
  if (!S) return SSG_ERR_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return SSG_ERR_ARG;
  Request* r = it->second.get();
  auto pred = [&] { return r->done; };
  if (timeout_ms < 0)
    S->cv.wait(lk, pred);
  else if (!S->cv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), pred))
    return SSG_ERR_TIMEOUT;
  if (result) *result = r->result;
  if (info) {
    info->iterations = r->info.iterations;
    info->residual = r->info.residual;
    info->initial_residual = r->info.initial_residual;
    info->solve_ms = 1e3 * (r->t_done - r->t_submit);
    info->history_len = 0;
  }
  return SSG_OK;
}

ssg_status ssg_server_cancel(ssg_server* S, unsigned long long id) {
  if (!S) return SSG_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return SSG_ERR_ARG;
  it->second->cancel = 1;
  S->cv.notify_all();
  return SSG_OK;
}

ssg_status ssg_server_drain(ssg_server* S, double timeout_ms) {
  if (!S) return SSG_ERR_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  auto pred = [&] { return S->queue.empty() && S->active == 0; };
  if (timeout_ms < 0)
    S->cv.wait(lk, pred);
  else if (!S->cv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), pred))
    return SSG_ERR_TIMEOUT;
  return SSG_OK;
}

ssg_status ssg_server_get_stats(ssg_server* S, ssg_server_stats* o) {
  if (!S || !o) return SSG_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  std::memset(o, 0, sizeof(*o));
  o->submitted = S->submitted;
  o->completed = S->completed;
  o->failed = S->failed;
  o->cancelled = S->cancelled;
  o->rejected = S->rejected;
  o->p50_ms = percentile(S->lat_ms, 50.0);
  o->p99_ms = percentile(S->lat_ms, 99.0);
  o->max_ms = percentile(S->lat_ms, 100.0);
  double sum = 0.0;
  for (double v : S->lat_ms) sum += v;
  o->mean_ms = S->lat_ms.empty() ? 0.0 : sum / (double)S->lat_ms.size();
  o->queue_p50_ms = percentile(S->queue_ms, 50.0);
  o->queue_p99_ms = percentile(S->queue_ms, 99.0);
  const double span = S->t_last - S->t_first;
  o->solves_per_s = span > 0 ? (double)S->completed / span : 0.0;
  o->hbm_in_use = S->in_use;
  o->hbm_peak = S->peak;
  o->hbm_budget = S->budget;
  o->mesh_hits = S->hits;
  o->mesh_misses = S->misses;
  o->evictions = S->evictions;
  o->max_active_seen = S->max_active_seen;
  o->resident_contexts = (int)S->resident.size();
  o->batches = S->batches;
  o->batched_requests = S->batched;
  return SSG_OK;
}

void ssg_server_destroy(ssg_server* S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    for (Request* r : S->queue) r->cancel = 1;
    S->stop = true;
    S->cv.notify_all();
  }
  for (auto& t : S->workers) t.join();
  cudaSetDevice(S->device);
  for (auto& x : S->resident)
    if (x.ctx) ssg_destroy(x.ctx);
  delete S;
}

}  // extern "C"
