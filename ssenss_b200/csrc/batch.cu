// Jacobi-CG Helmholtz solves of several independent meshes in shared
// launches (no reference counterpart: the reference solves one mesh per
// process).  The context's mesh is the concatenation of nseg meshes whose
// elements never neighbour across a segment; each segment runs the
// reference's conjugate_gradient with jacobi_preconditioner
// (src/solver.c:33-81, src/precon.c:361-371) with its own lambda, its own
// scalars (rdz, alpha, beta), its own stop test and iteration count, while
// the element operator and the DSS of an iteration are one launch over all
// segments' elements.
//
// Per iteration: operator (lambda folded into a per-segment scaled mass
// array, lambda = 1 in the kernel), DSS, then four segmented kernels over
// fixed chunks of points that never straddle two segments:
//   pap      chunk partials of (p w).ap
//   update   alpha = rdz / (sum of the segment's pap partials, chunk order);
//            x += alpha p, r -= alpha ap, z = dinv r; partials (r w).z, (r w).r
//   finish   per segment: rdz' = sum, beta = rdz'/rdz, err = sqrt(sum),
//            iteration count, stop (err <= eps or the cap); active count
//   p        p = (beta p + z) .* mask for segments still iterating
// The sums are taken in a fixed chunk order, so a batch is deterministic; a
// segment's sums are grouped differently from a solo solve's, so its
// iterates agree with a solo solve to rounding, not bitwise.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "kernels.cuh"
#include "ssg_internal.h"
#include "ssg_kernels.h"

namespace ssg {
namespace dev {

constexpr int kSegThreads = 256;
constexpr int kSegPer = 8;                          // points per thread
constexpr int kSegChunk = kSegThreads * kSegPer;    // points per chunk (one block)

// per-segment scalars
enum { SG_RDZ = 0, SG_BETA, SG_ERR, SG_ITER, SG_DONE, SG_EPS, SG_R0, SG_SIZE = 8 };

struct SegArgs {
  const int* chunk_seg;       // chunk -> segment
  const size_t* chunk_lo;     // first point of the chunk
  const int* chunk_n;         // points in the chunk
  const int* seg_chunk0;      // first chunk of each segment (nseg + 1)
  double* part;               // [chunk][4] partial sums
  double* sc;                 // [segment][SG_SIZE]
  int* active;                // segments still iterating (one int)
  int nseg;
  int max_iter;
};

// block sum of one value per thread in a fixed tree order
__device__ double seg_block_sum(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int off = kSegThreads / 2; off > 0; off >>= 1) {
    if (threadIdx.x < off) sh[threadIdx.x] += sh[threadIdx.x + off];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

// r = f - ap; z = dinv r; p = z; partials (r w).z, (r w).r
__global__ void __launch_bounds__(kSegThreads) k_seg_init(SegArgs a, const double* __restrict__ f,
                                                          const double* __restrict__ ap,
                                                          const double* __restrict__ dinv,
                                                          const uint8_t* __restrict__ mult,
                                                          double* __restrict__ r,
                                                          double* __restrict__ z,
                                                          double* __restrict__ p) {
  __shared__ double sh[kSegThreads];
  const int ch = blockIdx.x;
  const size_t lo = a.chunk_lo[ch];
  const int cnt = a.chunk_n[ch];
  double s0 = 0.0, s1 = 0.0;
  for (int k = 0; k < kSegPer; ++k) {
    const int o = k * kSegThreads + threadIdx.x;
    if (o < cnt) {
      const size_t q = lo + o;
      const double rq = f[q] + -ap[q];
      const double zq = rq * dinv[q];
      r[q] = rq;
      z[q] = zq;
      p[q] = zq;
      const double rw = rq * inv_count(mult[q]);
      s0 += rw * zq;
      s1 += rw * rq;
    }
  }
  s0 = seg_block_sum(s0, sh);
  s1 = seg_block_sum(s1, sh);
  if (threadIdx.x == 0) {
    a.part[4 * ch] = s0;
    a.part[4 * ch + 1] = s1;
  }
}

// per segment, after k_seg_init: rdz, iteration 0, not done
__global__ void k_seg_init_finish(SegArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.nseg) return;
  double rdz = 0.0, rr = 0.0;
  for (int ch = a.seg_chunk0[s]; ch < a.seg_chunk0[s + 1]; ++ch) {
    rdz += a.part[4 * ch];
    rr += a.part[4 * ch + 1];
  }
  double* sc = a.sc + SG_SIZE * s;
  sc[SG_RDZ] = rdz;
  sc[SG_R0] = sqrt(rr);
  sc[SG_ITER] = 0.0;
  sc[SG_DONE] = a.max_iter > 0 ? 0.0 : 1.0;
  if (s == 0) *a.active = a.max_iter > 0 ? a.nseg : 0;
}

__global__ void __launch_bounds__(kSegThreads) k_seg_pap(SegArgs a, const double* __restrict__ p,
                                                         const double* __restrict__ ap,
                                                         const uint8_t* __restrict__ mult) {
  __shared__ double sh[kSegThreads];
  const int ch = blockIdx.x;
  if (a.sc[SG_SIZE * a.chunk_seg[ch] + SG_DONE] != 0.0) return;   // uniform over the block
  const size_t lo = a.chunk_lo[ch];
  const int cnt = a.chunk_n[ch];
  double s0 = 0.0;
  for (int k = 0; k < kSegPer; ++k) {
    const int o = k * kSegThreads + threadIdx.x;
    if (o < cnt) {
      const size_t q = lo + o;
      s0 += (p[q] * inv_count(mult[q])) * ap[q];
    }
  }
  s0 = seg_block_sum(s0, sh);
  if (threadIdx.x == 0) a.part[4 * ch + 2] = s0;
}

__global__ void __launch_bounds__(kSegThreads) k_seg_update(
    SegArgs a, double* __restrict__ x, const double* __restrict__ p, double* __restrict__ r,
    const double* __restrict__ ap, const double* __restrict__ dinv,
    const uint8_t* __restrict__ mult, double* __restrict__ z) {
  __shared__ double sh[kSegThreads];
  const int ch = blockIdx.x;
  const int s = a.chunk_seg[ch];
  const double* sc = a.sc + SG_SIZE * s;
  if (sc[SG_DONE] != 0.0) return;
  // alpha = rdz / (p w).ap of the whole segment, its chunks in order
  double pap = 0.0;
  for (int c2 = a.seg_chunk0[s]; c2 < a.seg_chunk0[s + 1]; ++c2) pap += a.part[4 * c2 + 2];
  const double alpha = sc[SG_RDZ] / pap;
  const size_t lo = a.chunk_lo[ch];
  const int cnt = a.chunk_n[ch];
  double s0 = 0.0, s1 = 0.0;
  for (int k = 0; k < kSegPer; ++k) {
    const int o = k * kSegThreads + threadIdx.x;
    if (o < cnt) {
      const size_t q = lo + o;
      x[q] = x[q] + alpha * p[q];
      const double rq = r[q] + -alpha * ap[q];
      r[q] = rq;
      const double zq = rq * dinv[q];
      z[q] = zq;
      const double rw = rq * inv_count(mult[q]);
      s0 += rw * zq;
      s1 += rw * rq;
    }
  }
  s0 = seg_block_sum(s0, sh);
  s1 = seg_block_sum(s1, sh);
  if (threadIdx.x == 0) {
    a.part[4 * ch] = s0;
    a.part[4 * ch + 1] = s1;
  }
}

// one thread per segment: beta, err, iteration count, stop; then the
// number of segments still iterating (one block of up to 1024 threads
// loops over the segments)
__global__ void __launch_bounds__(1024) k_seg_finish(SegArgs a) {
  __shared__ int nact;
  if (threadIdx.x == 0) nact = 0;
  __syncthreads();
  int mine = 0;
  for (int s = threadIdx.x; s < a.nseg; s += blockDim.x) {
    double* sc = a.sc + SG_SIZE * s;
    if (sc[SG_DONE] != 0.0) continue;
    double rdz = 0.0, rr = 0.0;
    for (int ch = a.seg_chunk0[s]; ch < a.seg_chunk0[s + 1]; ++ch) {
      rdz += a.part[4 * ch];
      rr += a.part[4 * ch + 1];
    }
    sc[SG_BETA] = rdz / sc[SG_RDZ];
    sc[SG_RDZ] = rdz;
    const double err = sqrt(rr);
    sc[SG_ERR] = err;
    sc[SG_ITER] += 1.0;
    // continue while err > eps and the count is below the cap
    // (src/solver.c:78-79); a non-finite err stops the segment
    const bool more = err > sc[SG_EPS] && sc[SG_ITER] < (double)a.max_iter;
    if (!more) sc[SG_DONE] = 1.0;
    mine += more ? 1 : 0;
  }
  atomicAdd(&nact, mine);
  __syncthreads();
  if (threadIdx.x == 0) *a.active = nact;
}

__global__ void __launch_bounds__(kSegThreads) k_seg_p(SegArgs a, double* __restrict__ p,
                                                       const double* __restrict__ z,
                                                       const double* __restrict__ mask) {
  const int ch = blockIdx.x;
  const double* sc = a.sc + SG_SIZE * a.chunk_seg[ch];
  if (sc[SG_DONE] != 0.0) return;
  const double beta = sc[SG_BETA];
  const size_t lo = a.chunk_lo[ch];
  const int cnt = a.chunk_n[ch];
  for (int k = 0; k < kSegPer; ++k) {
    const int o = k * kSegThreads + threadIdx.x;
    if (o < cnt) {
      const size_t q = lo + o;
      double v = beta * p[q] + z[q];
      if (mask) v = v * mask[q];
      p[q] = v;
    }
  }
}

// one context's DSS map (dss_map_table layout: gather words, then per
// element records) into a concatenation's map at point offset P and element
// offset E: every point index (>= 0) moves by P, record codes and -1 stay
__global__ void k_dss_map_shift(const int* __restrict__ src, size_t npts, size_t head,
                                size_t rec_ints, int* __restrict__ dst, size_t P,
                                size_t head_dst, size_t rec_dst) {
  const size_t n = npts + rec_ints;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    if (i < npts) {
      const int w = src[i];
      dst[P + i] = w >= 0 ? w + (int)P : w;
    } else {
      const size_t k = i - npts;
      const int v = src[head + k];
      dst[head_dst + rec_dst + k] = v >= 0 ? v + (int)P : v;
    }
  }
}

// bj_s = lambda_s bj over one segment's points
__global__ void k_seg_scale(size_t lo, size_t n, double lam, const double* __restrict__ bj,
                            double* __restrict__ out) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x)
    out[lo + q] = lam * bj[lo + q];
}

}  // namespace dev
}  // namespace ssg

namespace ssg {

namespace {

template <typename T>
ssg_status seg_alloc(ssg_context* c, T** p, size_t count) {
  void* q = nullptr;
  if (cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    return fail(c, SSG_ERR_NOMEM, "segmented solve scratch");
  }
  *p = static_cast<T*>(q);
  return SSG_OK;
}

template <typename T>
void seg_release(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

// capacity for nch chunks, nseg segments and np points (grown, never shrunk;
// a grown group is reallocated whole, contents not kept)
ssg_status seg_reserve(ssg_context* c, SegScratch& W, size_t nch, size_t nseg, size_t np) {
  if (nch > W.cap_chunks) {
    seg_release(W.chunk_seg);
    seg_release(W.chunk_n);
    seg_release(W.chunk_lo);
    seg_release(W.part);
    W.cap_chunks = 0;
    SSG_TRY(seg_alloc(c, &W.chunk_seg, nch));
    SSG_TRY(seg_alloc(c, &W.chunk_n, nch));
    SSG_TRY(seg_alloc(c, &W.chunk_lo, nch));
    SSG_TRY(seg_alloc(c, &W.part, 4 * nch));
    W.cap_chunks = nch;
  }
  if (nseg > W.cap_segs) {
    seg_release(W.seg_chunk0);
    seg_release(W.sc);
    W.cap_segs = 0;
    SSG_TRY(seg_alloc(c, &W.seg_chunk0, nseg + 1));
    SSG_TRY(seg_alloc(c, &W.sc, (size_t)dev::SG_SIZE * nseg));
    W.cap_segs = nseg;
  }
  if (!W.active) SSG_TRY(seg_alloc(c, &W.active, 1));
  if (np > W.cap_points) {
    double** vecs[] = {&W.bj_s, &W.dinv_s, &W.x, &W.r, &W.z, &W.p, &W.ap, &W.aploc, &W.f};
    for (double** v : vecs) seg_release(*v);
    W.cap_points = 0;
    for (double** v : vecs) SSG_TRY(seg_alloc(c, v, np));
    W.cap_points = np;
  }
  return SSG_OK;
}

}  // namespace

void seg_scratch_free(SegScratch& W) {
  seg_release(W.chunk_seg);
  seg_release(W.chunk_n);
  seg_release(W.chunk_lo);
  seg_release(W.part);
  seg_release(W.seg_chunk0);
  seg_release(W.sc);
  seg_release(W.active);
  double** vecs[] = {&W.bj_s, &W.dinv_s, &W.x, &W.r, &W.z, &W.p, &W.ap, &W.aploc, &W.f};
  for (double** v : vecs) seg_release(*v);
  W = SegScratch();
}

ssg_status seg_solve(ssg_context* c, const SegLevel& L, SegScratch& W, int nseg,
                     const int* seg_first, const double* lambda, const double* f, double* u,
                     const double* eps, int max_iter, ssg_solve_info* info) {
  const size_t np = L.npts, nt = L.nt;
  cudaStream_t s = c->stream;
  // chunk tables: fixed chunks of points inside each segment
  std::vector<int> chunk_seg, chunk_n, seg_chunk0(nseg + 1);
  std::vector<size_t> chunk_lo;
  for (int sg = 0; sg < nseg; ++sg) {
    seg_chunk0[sg] = (int)chunk_seg.size();
    const size_t lo = (size_t)seg_first[sg] * nt, hi = (size_t)seg_first[sg + 1] * nt;
    for (size_t q = lo; q < hi; q += dev::kSegChunk) {
      chunk_seg.push_back(sg);
      chunk_lo.push_back(q);
      chunk_n.push_back((int)std::min<size_t>(dev::kSegChunk, hi - q));
    }
  }
  seg_chunk0[nseg] = (int)chunk_seg.size();
  const int nch = (int)chunk_seg.size();
  SSG_TRY(seg_reserve(c, W, nch, nseg, np));

  SSG_CUDA(c, cudaMemcpyAsync(W.chunk_seg, chunk_seg.data(), nch * sizeof(int),
                              cudaMemcpyHostToDevice, s));
  SSG_CUDA(c, cudaMemcpyAsync(W.chunk_n, chunk_n.data(), nch * sizeof(int),
                              cudaMemcpyHostToDevice, s));
  SSG_CUDA(c, cudaMemcpyAsync(W.chunk_lo, chunk_lo.data(), nch * sizeof(size_t),
                              cudaMemcpyHostToDevice, s));
  SSG_CUDA(c, cudaMemcpyAsync(W.seg_chunk0, seg_chunk0.data(), (nseg + 1) * sizeof(int),
                              cudaMemcpyHostToDevice, s));
  std::vector<double> sc((size_t)dev::SG_SIZE * nseg, 0.0);
  for (int sg = 0; sg < nseg; ++sg) sc[(size_t)dev::SG_SIZE * sg + dev::SG_EPS] = eps[sg];
  SSG_CUDA(c, cudaMemcpyAsync(W.sc, sc.data(), sc.size() * sizeof(double),
                              cudaMemcpyHostToDevice, s));
  SSG_CUDA(c, cudaMemcpyAsync(W.f, f, np * sizeof(double), cudaMemcpyDefault, s));
  SSG_CUDA(c, cudaMemcpyAsync(W.x, u, np * sizeof(double), cudaMemcpyDefault, s));
  dev::SegArgs a;
  a.chunk_seg = W.chunk_seg;
  a.chunk_lo = W.chunk_lo;
  a.chunk_n = W.chunk_n;
  a.seg_chunk0 = W.seg_chunk0;
  a.part = W.part;
  a.sc = W.sc;
  a.active = W.active;
  a.nseg = nseg;
  a.max_iter = max_iter;

  // per segment: lambda_s bj for the operator (lambda 1 in the kernel) and
  // the Jacobi inverse 1 / DSS(kdiag + (lambda_s rho) J) (src/helmholtz.c:
  // 51-68, src/precon.c:336-359)
  for (int sg = 0; sg < nseg; ++sg) {
    const size_t lo = (size_t)seg_first[sg] * nt;
    const size_t n = (size_t)(seg_first[sg + 1] - seg_first[sg]) * nt;
    count_launch();
    dev::k_seg_scale<<<vec_blocks(n), 256, 0, s>>>(lo, n, lambda[sg], L.bj, W.bj_s);
    SSG_CUDA(c, cudaGetLastError());
    SSG_CUDA(c, run_helm_diag(s, n, nt, L.kdiag + lo, L.rho, L.det + lo, lambda[sg],
                              W.aploc + lo));
  }
  SSG_CUDA(c, run_dss(s, DSS_PLAIN, false, L.n, L.nel, W.aploc, W.dinv_s, nullptr, L.dss,
                      nullptr, nullptr, nullptr, nullptr));
  SSG_CUDA(c, run_recip(s, np, W.dinv_s));

  // mask f; r = f - DSS(mask A x); z = dinv r; p = z; rdz
  if (L.mask) SSG_CUDA(c, run_mul(s, false, np, W.f, L.mask));
  auto op = [&](const double* in) -> ssg_status {
    SSG_CUDA(c, run_ax(s, L.n, L.nel, 0, true, false, in, W.aploc, L.gf, np, W.bj_s, L.D, L.S,
                       1.0, nullptr));
    SSG_CUDA(c, run_dss(s, DSS_PLAIN, false, L.n, L.nel, W.aploc, W.ap, nullptr, L.dss, L.mask,
                        nullptr, nullptr, nullptr));
    return SSG_OK;
  };
  SSG_TRY(op(W.x));
  count_launch();
  dev::k_seg_init<<<nch, dev::kSegThreads, 0, s>>>(a, W.f, W.ap, W.dinv_s, L.mult, W.r, W.z,
                                                   W.p);
  SSG_CUDA(c, cudaGetLastError());
  count_launch();
  dev::k_seg_init_finish<<<(nseg + 255) / 256, 256, 0, s>>>(a);
  SSG_CUDA(c, cudaGetLastError());

  // iterations, enqueued in chunks of 8 with a host check of the active
  // count between chunks
  for (int it = 0; it < max_iter; ++it) {
    SSG_TRY(op(W.p));
    count_launch();
    dev::k_seg_pap<<<nch, dev::kSegThreads, 0, s>>>(a, W.p, W.ap, L.mult);
    count_launch();
    dev::k_seg_update<<<nch, dev::kSegThreads, 0, s>>>(a, W.x, W.p, W.r, W.ap, W.dinv_s, L.mult,
                                                       W.z);
    count_launch();
    dev::k_seg_finish<<<1, 1024, 0, s>>>(a);
    count_launch();
    dev::k_seg_p<<<nch, dev::kSegThreads, 0, s>>>(a, W.p, W.z, L.mask);
    SSG_CUDA(c, cudaGetLastError());
    if (it % 8 == 7 || it == max_iter - 1) {
      SSG_CUDA(c, cudaMemcpyAsync(c->h_pin, W.active, sizeof(int), cudaMemcpyDeviceToHost, s));
      SSG_CUDA(c, cudaStreamSynchronize(s));
      int act = 0;
      std::memcpy(&act, c->h_pin, sizeof(int));
      if (c->cancel && *c->cancel) return fail(c, SSG_ERR_CANCELLED, "solve cancelled");
      if (act == 0) break;
    }
  }
  SSG_CUDA(c, cudaMemcpyAsync(u, W.x, np * sizeof(double), cudaMemcpyDefault, s));
  SSG_CUDA(c, cudaMemcpyAsync(sc.data(), W.sc, sc.size() * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
  SSG_CUDA(c, cudaStreamSynchronize(s));
  ssg_status st = SSG_OK;
  for (int sg = 0; sg < nseg; ++sg) {
    const double* q = sc.data() + (size_t)dev::SG_SIZE * sg;
    info[sg].iterations = (int)q[dev::SG_ITER];
    info[sg].residual = q[dev::SG_ERR];
    info[sg].initial_residual = q[dev::SG_R0];
    info[sg].solve_ms = 0.0;
    info[sg].history_len = 0;
    if (!std::isfinite(q[dev::SG_ERR]))
      st = SSG_NONFINITE;
    else if (!(q[dev::SG_ERR] <= eps[sg]) && st == SSG_OK)
      st = SSG_MAXITER;
  }
  return st;
}

size_t dss_record_ints(int n) {
  const int I = n > 2 ? n - 2 : 0;
  return (size_t)12 * I * 4 + 8 * 8;
}

cudaError_t run_dss_map_shift(cudaStream_t s, const int* src, int n, int nel, int* dst,
                              size_t P, size_t npts_dst, int E) {
  const size_t nt = (size_t)n * n * n, npts = nt * nel;
  const size_t rec = dss_record_ints(n);
  const size_t total = npts + rec * nel;
  count_launch();
  dev::k_dss_map_shift<<<vec_blocks(total), 256, 0, s>>>(
      src, npts, dss_map_records_offset(npts), rec * nel, dst, P,
      dss_map_records_offset(npts_dst), rec * (size_t)E);
  return cudaGetLastError();
}

}  // namespace ssg

using namespace ssg;

extern "C" ssg_status ssg_solve_helmholtz_segments(ssg_context* c, int var, int nseg,
                                                   const int* seg_first, const double* lambda,
                                                   const double* f, double* u,
                                                   const double* eps, int max_iter,
                                                   ssg_solve_info* info) {
  if (!c) return SSG_ERR_ARG;
  if (!c->ready) return fail(c, SSG_ERR_STATE, "no mesh set up on this context");
  if (var < SSG_X_VELOCITY || var > SSG_Z_VELOCITY)
    return fail(c, SSG_ERR_ARG, "Helmholtz var must be a velocity component");
  if (nseg < 1 || !seg_first || !lambda || !f || !u || !eps || !info || max_iter < 1)
    return fail(c, SSG_ERR_ARG, "bad segmented solve arguments");
  if (seg_first[0] != 0 || seg_first[nseg] != c->nel)
    return fail(c, SSG_ERR_ARG, "segments must cover the elements 0 .. nel - 1");
  for (int s = 0; s < nseg; ++s) {
    if (seg_first[s + 1] <= seg_first[s])
      return fail(c, SSG_ERR_ARG, "every segment needs at least one element");
    if (!(lambda[s] > 0.0) || !std::isfinite(lambda[s]) || !(eps[s] > 0.0))
      return fail(c, SSG_ERR_ARG, "segment lambda and eps must be > 0");
    // no element of a segment may neighbour another segment's element
    for (int e = seg_first[s]; e < seg_first[s + 1]; ++e)
      for (int k = 0; k < 26; ++k) {
        const int nb = c->host.neigh[26 * (size_t)e + k];
        if (nb >= 0 && (nb < seg_first[s] || nb >= seg_first[s + 1]))
          return fail(c, SSG_ERR_ARG, "an element neighbours another segment");
      }
  }
  SSG_CUDA(c, cudaSetDevice(c->device));
  const DevLevel& D = c->lev[0];
  SegLevel L;
  L.n = D.n;
  L.nel = c->nel;
  L.nt = D.nt;
  L.npts = D.npts;
  L.gf = D.gf;
  L.bj = D.bj;
  L.kdiag = D.kdiag;
  L.rho = D.rho;
  L.det = D.det;
  L.mask = c->has_walls ? D.mask : nullptr;
  L.D = D.D;
  L.S = D.S;
  L.mult = D.mult;
  L.dss = D.dss_ec;
  if (!c->seg) c->seg = new SegScratch();
  return seg_solve(c, L, *c->seg, nseg, seg_first, lambda, f, u, eps, max_iter, info);
}
