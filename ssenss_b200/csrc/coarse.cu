// Coarsest p-multigrid level (n = 2): the whole Jacobi-preconditioned CG
// solve in one persistent cooperative kernel.
//
// The reference solves the coarsest level with conjugate_gradient +
// jacobi_preconditioner to the absolute eps, at most 500 iterations
// (src/precon.c:242-244, src/solver.c:33-81).  The level is tiny (8 points
// per element), so one kernel launch per CG iteration would be pure launch
// latency; here every iteration runs inside one launch, with grid-wide
// barriers between the element operator, the DSS and the vector update.
// Each block reduces the same block partials in the same order, so every
// block takes the same alpha, beta and stop decision, and the result does
// not depend on timing.  The loop is bounded by max_iter.
#include <atomic>
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cmath>

#include "kernels.cuh"
#include "ssg_internal.h"
#include "ssg_kernels.h"

namespace cg = cooperative_groups;

namespace ssg {
namespace dev {

struct CoarseArgs {
  int nel = 0;
  size_t npts = 0;
  const double* f = nullptr;
  double* x = nullptr;
  double *r = nullptr, *z = nullptr, *p = nullptr, *aploc = nullptr, *ap = nullptr;
  const double* gf = nullptr;     // 6 x npts
  const double* D = nullptr;      // 2 x 2, D[i*2+m]
  const double* dinv = nullptr;
  const uint8_t* mult = nullptr;
  const int2* pairs = nullptr;
  double nunique = 1.0;
  double eps = 0.0;
  double rel = 0.0;   // also stop once err <= rel * err0 (0: eps only)
  int max_iter = 0;
  double* partA = nullptr;        // >= 4 * gridDim.x
  double* partB = nullptr;        // >= 3 * gridDim.x
  double* frame = nullptr;
};

// A_e u at one point g of an n = 2 element (the contraction order of k_ax:
// r-, s-, t-derivatives as two-term sums, the metric products
// w_a = sum_b G_ab u_b, then (D^T w0 + D^T w1) + D^T w2).  The element's 8
// points are held by 8 consecutive lanes (lane & 7 = point index in the
// element) and the neighbours' values come by shuffles, so the operator
// runs with one point per thread.  All 32 lanes of the warp call it (lanes
// past the end pass valid = false).
__device__ __forceinline__ double point_op2(const CoarseArgs& a, const double* sD, double uown,
                                            size_t g, bool valid) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, grp = lane & ~7, q = lane & 7;
  const int i = q & 1, j = (q >> 1) & 1, k = q >> 2;
  double ur = 0, us = 0, ut = 0;
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    const double vr = __shfl_sync(full, uown, grp | ((k * 2 + j) * 2 + m));
    const double vs = __shfl_sync(full, uown, grp | ((k * 2 + m) * 2 + i));
    const double vt = __shfl_sync(full, uown, grp | ((m * 2 + j) * 2 + i));
    ur += sD[i * 2 + m] * vr;
    us += sD[j * 2 + m] * vs;
    ut += sD[k * 2 + m] * vt;
  }
  double g0 = 0, g1 = 0, g2 = 0, g3 = 0, g4 = 0, g5 = 0;
  if (valid) {
    g0 = a.gf[g];
    g1 = a.gf[a.npts + g];
    g2 = a.gf[2 * a.npts + g];
    g3 = a.gf[3 * a.npts + g];
    g4 = a.gf[4 * a.npts + g];
    g5 = a.gf[5 * a.npts + g];
  }
  const double w0 = g0 * ur + g1 * us + g2 * ut;
  const double w1 = g1 * ur + g3 * us + g4 * ut;
  const double w2 = g2 * ur + g4 * us + g5 * ut;
  double acc = 0, acs = 0, act = 0;
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    const double v0 = __shfl_sync(full, w0, grp | ((k * 2 + j) * 2 + m));
    const double v1 = __shfl_sync(full, w1, grp | ((k * 2 + m) * 2 + i));
    const double v2 = __shfl_sync(full, w2, grp | ((m * 2 + j) * 2 + i));
    acc += sD[m * 2 + i] * v0;
    acs += sD[m * 2 + j] * v1;
    act += sD[m * 2 + k] * v2;
  }
  return (acc + acs) + act;
}

// sum over all blocks of NQ partial arrays, identical in every block
template <int NQ>
__device__ __forceinline__ void grid_sums(const double* part, int G, double (&s)[NQ],
                                          double* sred, double* sbc) {
  double v[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    v[q] = 0.0;
    for (int b = threadIdx.x; b < G; b += blockDim.x) v[q] += part[q * G + b];
  }
  block_reduce<NQ>(v, sred);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < NQ; ++q) sbc[q] = v[q];
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NQ; ++q) s[q] = sbc[q];
  __syncthreads();
}

template <int NQ>
__device__ __forceinline__ void block_partials(double (&v)[NQ], double* part, double* sred) {
  block_reduce<NQ>(v, sred);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < NQ; ++q) part[q * gridDim.x + blockIdx.x] = v[q];
}

__global__ void __launch_bounds__(256) k_coarse_cg(CoarseArgs a) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double sred[4 * 32];
  __shared__ double sbc[4];
  __shared__ double sD[4];
  if (threadIdx.x < 4) sD[threadIdx.x] = a.D[threadIdx.x];
  __syncthreads();
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t nthr = (size_t)gridDim.x * blockDim.x;
  const int G = gridDim.x;

  // one point per thread, an element's 8 points in 8 consecutive lanes; the
  // loop runs warp-uniformly (point_op2 shuffles across the warp)
  const size_t wbase = tid - (threadIdx.x & 31);

  // r = f - DSS(A x); nullspace of r (src/solver.c:49-53)
  for (size_t b = wbase; b < a.npts; b += nthr) {
    const size_t g = b + (threadIdx.x & 31);
    const bool valid = g < a.npts;
    const double o = point_op2(a, sD, valid ? a.x[g] : 0.0, g, valid);
    if (valid) a.aploc[g] = o;
  }
  grid.sync();
  {
    double v[1] = {0.0};
    for (size_t q = tid; q < a.npts; q += nthr) {
      int cnt;
      const double acc = dss_gather<2, double>(a.aploc, nullptr, a.pairs + (q >> 3) * 26, q,
                                               (int)(q & 7), cnt);
      const double rq = a.f[q] + -acc;
      a.r[q] = rq;
      v[0] += rq * inv_count(1u + (unsigned)cnt);
    }
    block_partials<1>(v, a.partA, sred);
  }
  grid.sync();
  double s[4];
  {
    double t[1];
    grid_sums<1>(a.partA, G, t, sred, sbc);
    const double c = t[0] / a.nunique;
    double v[1] = {0.0};
    for (size_t q = tid; q < a.npts; q += nthr) {
      const double rq = a.r[q] + -c;
      a.r[q] = rq;
      const double zq = rq * a.dinv[q];
      a.z[q] = zq;
      v[0] += zq * inv_count(a.mult[q]);
    }
    block_partials<1>(v, a.partB, sred);
  }
  grid.sync();
  double cz, rdz = 0.0, beta = 0.0, err = 0.0, err0 = 0.0;
  {
    double t[1];
    grid_sums<1>(a.partB, G, t, sred, sbc);
    cz = t[0] / a.nunique;
  }
  int it = 0;
  for (; it < a.max_iter; ++it) {
    const bool first = it == 0;
    // p = beta p + (z - c) (first: p = z - c); aploc = A_e p
    for (size_t b = wbase; b < a.npts; b += nthr) {
      const size_t g = b + (threadIdx.x & 31);
      const bool valid = g < a.npts;
      double pv = 0.0;
      if (valid) {
        const double zc = a.z[g] - cz;
        pv = first ? zc : beta * a.p[g] + zc;
        a.p[g] = pv;
      }
      const double o = point_op2(a, sD, pv, g, valid);
      if (valid) a.aploc[g] = o;
    }
    grid.sync();
    // ap = DSS(aploc); (p w).ap; first: (r w).p and (r w).r
    {
      double v[3] = {0.0, 0.0, 0.0};
      for (size_t q = tid; q < a.npts; q += nthr) {
        int cnt;
        const double acc = dss_gather<2, double>(a.aploc, nullptr, a.pairs + (q >> 3) * 26, q,
                                                 (int)(q & 7), cnt);
        a.ap[q] = acc;
        const double w = inv_count(1u + (unsigned)cnt);
        const double pw = a.p[q] * w;
        v[0] += pw * acc;
        if (first) {
          const double rw = a.r[q] * w;
          v[1] += rw * a.p[q];
          v[2] += rw * a.r[q];
        }
      }
      block_partials<3>(v, a.partB, sred);
    }
    grid.sync();
    // alpha; x += alpha p; r -= alpha ap; z = M^-1 r
    {
      double t[3];
      grid_sums<3>(a.partB, G, t, sred, sbc);
      if (first) {
        rdz = t[1];
        err0 = sqrt(t[2]);
      }
      const double alpha = rdz / t[0];
      double v[4] = {0.0, 0.0, 0.0, 0.0};
      for (size_t q = tid; q < a.npts; q += nthr) {
        a.x[q] = a.x[q] + alpha * a.p[q];
        const double rq = a.r[q] + -alpha * a.ap[q];
        a.r[q] = rq;
        const double zq = rq * a.dinv[q];
        a.z[q] = zq;
        const double w = inv_count(a.mult[q]);
        const double rw = rq * w;
        v[0] += rw * zq;
        v[1] += rw * rq;
        v[2] += w * zq;
        v[3] += rw;
      }
      block_partials<4>(v, a.partA, sred);
    }
    grid.sync();
    grid_sums<4>(a.partA, G, s, sred, sbc);
    cz = s[2] / a.nunique;
    const double rdz_new = s[0] - cz * s[3];
    beta = rdz_new / rdz;
    rdz = rdz_new;
    err = sqrt(s[1]);
    if (!(err > a.eps) || !(err > a.rel * err0) || it + 1 >= a.max_iter) {
      ++it;
      break;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.frame[F_ITER] = (double)it;
    a.frame[F_ERR] = err;
    a.frame[F_ERR0] = err0;
    a.frame[F_DONE] = 1.0;
  }
}

// ---------------------------------------------------------------------------
// The post-smoother CG of a small multigrid level (conjugate_gradient with
// jacobi_preconditioner on the Poisson operator, src/solver.c:33-81: what
// cg_solve launches as three kernels per iteration) in one cooperative
// launch.  Same per-point arithmetic as those kernels (the element operator
// is the shared ax_element, the DSS the reference-ordered dss_gather, the
// vector updates k_add_const / k_jacobi / k_dots / k_cg_update written out);
// the reductions are block partials summed identically by every block, so
// every block takes the same alpha, beta and stop decision.  Three grid
// barriers per iteration; the loop is bounded by max_iter.
// ---------------------------------------------------------------------------
template <typename T>
struct LevelCgArgs {
  int nel = 0;
  size_t npts = 0;
  const T* f = nullptr;
  T* x = nullptr;
  T *r = nullptr, *z = nullptr, *p = nullptr, *aploc = nullptr, *ap = nullptr;
  const T* gf = nullptr;          // 6 x npts
  const double* D = nullptr;
  const T* dinv = nullptr;
  const uint8_t* mult = nullptr;
  const int2* pairs = nullptr;
  double nunique = 1.0;
  double eps = 0.0;
  int max_iter = 0;
  double* partA = nullptr;        // >= 4 * gridDim.x
  double* partB = nullptr;        // >= 3 * gridDim.x
};

template <int N>
constexpr size_t level_cg_smem() {
  return (size_t)(AxSmem<N>::MATS + (256 / (N * N)) * 3 * AxSmem<N>::BLK) * sizeof(double);
}

template <int N, typename T>
__global__ void __launch_bounds__(256) k_level_cg(LevelCgArgs<T> a) {
  using L = AxSmem<N>;
  static_assert(256 % (N * N) == 0, "whole element planes per block");
  constexpr int NT = N * N * N, EPB = 256 / (N * N);
  cg::grid_group grid = cg::this_grid();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sD = reinterpret_cast<double*>(smem_raw);
  __shared__ double sred[4 * 32];
  __shared__ double sbc[4];
  const int tb = threadIdx.x;
  const int i = tb % N, j = (tb / N) % N, slot = tb / (N * N);
  double* su = sD + L::MATS + slot * 3 * L::BLK;
  ax_load_mats<N, false>(sD, a.D, a.D, tb, 256);   // visible after the first barrier
  const size_t tid = (size_t)blockIdx.x * blockDim.x + tb;
  const size_t nthr = (size_t)gridDim.x * blockDim.x;
  const int G = gridDim.x;
  const int ngroups = (a.nel + EPB - 1) / EPB;
  // aploc = A_e in (fusep: in = p, formed from z first); block-uniform loop
  auto op_pass = [&](T* in, bool fusep, bool first, double beta, double cz) {
    for (int grp = blockIdx.x; grp < ngroups; grp += G) {
      const int e = grp * EPB + slot;
      if (fusep)
        ax_element<N, T, false, true>(e, e < a.nel, i, j, sD, su, su + L::BLK,
                                      su + 2 * L::BLK, in, a.aploc, a.gf, a.npts, nullptr,
                                      0.0, a.z, beta, cz, nullptr, first);
      else
        ax_element<N, T, false, false>(e, e < a.nel, i, j, sD, su, su + L::BLK,
                                       su + 2 * L::BLK, in, a.aploc, a.gf, a.npts, nullptr,
                                       0.0, nullptr, 0.0, 0.0, nullptr, false);
    }
  };

  // r = f - DSS(A x) with sum w r (DSS_RESID)
  op_pass(a.x, false, false, 0.0, 0.0);
  grid.sync();
  {
    double v[1] = {0.0};
    for (size_t q = tid; q < a.npts; q += nthr) {
      int cnt;
      const double acc = dss_gather<N, T>(a.aploc, nullptr, a.pairs + (q / NT) * 26, q,
                                          (int)(q % NT), cnt);
      const T rv = (T)((double)a.f[q] + -acc);
      a.r[q] = rv;
      v[0] += (double)rv * inv_count(1u + (unsigned)cnt);
    }
    block_partials<1>(v, a.partA, sred);
  }
  grid.sync();
  // r -= c (nullspace); z = M^-1 r with sum w z (k_add_const, k_jacobi)
  {
    double t[1];
    grid_sums<1>(a.partA, G, t, sred, sbc);
    const double nc = -(t[0] / a.nunique);
    double v[1] = {0.0};
    for (size_t q = tid; q < a.npts; q += nthr) {
      const T rq = (T)((double)a.r[q] + nc);
      a.r[q] = rq;
      const T zq = (T)((double)rq * (double)a.dinv[q]);
      a.z[q] = zq;
      v[0] += (double)zq * inv_count(a.mult[q]);
    }
    block_partials<1>(v, a.partB, sred);
  }
  grid.sync();
  double cz, rdz = 0.0, beta = 0.0;
  {
    double t[1];
    grid_sums<1>(a.partB, G, t, sred, sbc);
    cz = t[0] / a.nunique;
  }
  for (int it = 0; it < a.max_iter; ++it) {
    const bool first = it == 0;
    // p = beta p + (z - c) (first: z - c); aploc = A_e p
    op_pass(a.p, true, first, beta, cz);
    grid.sync();
    // ap = DSS(aploc), (p w).ap; first: (r w).p, (r w).r (k_dss DOT, k_dots)
    {
      double v[3] = {0.0, 0.0, 0.0};
      // four points per thread at a time: all their gathers are issued
      // before any store (a store could alias the next gather), then the
      // points are summed in the same order as one at a time
      constexpr int U = 4;
      for (size_t q0 = tid; q0 < a.npts; q0 += U * nthr) {
        double acc[U];
        int cnt[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const size_t q = q0 + u * nthr;
          acc[u] = 0.0;
          cnt[u] = 0;
          if (q < a.npts)
            acc[u] = dss_gather<N, T>(a.aploc, nullptr, a.pairs + (q / NT) * 26, q,
                                      (int)(q % NT), cnt[u]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const size_t q = q0 + u * nthr;
          if (q >= a.npts) break;
          const T av = (T)acc[u];
          a.ap[q] = av;
          const double pv = (double)a.p[q];
          v[0] += (pv * inv_count(1u + (unsigned)cnt[u])) * (double)av;
          if (first) {
            const double rw = (double)a.r[q] * inv_count(a.mult[q]);
            v[1] += rw * pv;
            v[2] += rw * (double)a.r[q];
          }
        }
      }
      block_partials<3>(v, a.partB, sred);
    }
    grid.sync();
    // alpha; x += alpha p; r -= alpha ap; z = M^-1 r (k_cg_update)
    {
      double t[3];
      grid_sums<3>(a.partB, G, t, sred, sbc);
      if (first) rdz = t[1];
      const double alpha = rdz / t[0];
      double v[4] = {0.0, 0.0, 0.0, 0.0};
      // four points per thread: every load before any store
      constexpr int U = 4;
      for (size_t q0 = tid; q0 < a.npts; q0 += U * nthr) {
        double xv[U], pv[U], rv[U], av[U], dv[U];
        unsigned mv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const size_t q = q0 + u * nthr;
          const size_t qq = q < a.npts ? q : q0;
          xv[u] = (double)a.x[qq];
          pv[u] = (double)a.p[qq];
          rv[u] = (double)a.r[qq];
          av[u] = (double)a.ap[qq];
          dv[u] = (double)a.dinv[qq];
          mv[u] = a.mult[qq];
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const size_t q = q0 + u * nthr;
          if (q >= a.npts) break;
          a.x[q] = (T)(xv[u] + alpha * pv[u]);
          const T rq = (T)(rv[u] + -alpha * av[u]);
          a.r[q] = rq;
          const T zq = (T)((double)rq * dv[u]);
          a.z[q] = zq;
          const double w = inv_count(mv[u]);
          const double rw = (double)rq * w;
          v[0] += rw * (double)zq;
          v[1] += rw * (double)rq;
          v[2] += w * (double)zq;
          v[3] += rw;
        }
      }
      block_partials<4>(v, a.partA, sred);
    }
    grid.sync();
    // nullspace constant, beta, residual, stop (OP_CG_BETA)
    double s4[4];
    grid_sums<4>(a.partA, G, s4, sred, sbc);
    cz = s4[2] / a.nunique;
    const double rdz_new = s4[0] - cz * s4[3];
    beta = rdz_new / rdz;
    rdz = rdz_new;
    const double err = sqrt(s4[1]);
    if (!(err > a.eps) || it + 1 >= a.max_iter) break;
  }
}

}  // namespace dev

// Blocks per device that a cooperative launch may use, filled on first use.
// Serving worker threads launch concurrently, so the entries are atomics; a
// race only repeats the same occupancy query and stores the same value.
static constexpr int kMaxDevices = 64;
static std::atomic<int> g_coarse_grid[kMaxDevices];
static std::atomic<int> g_level_grid[2][kMaxDevices];

static cudaError_t cooperative_cap(std::atomic<int>& slot, const void* kernel, size_t smem,
                                   int device, int* out) {
  int c = slot.load(std::memory_order_relaxed);
  if (c == 0) {
    int per_sm = 0, nsm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, smem);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    c = per_sm * nsm;
    if (c < 1) return cudaErrorCooperativeLaunchTooLarge;
    slot.store(c, std::memory_order_relaxed);
  }
  *out = c;
  return cudaSuccess;
}

cudaError_t run_coarse_cg(cudaStream_t s, int device, int nel, const double* f, double* x,
                          double* r, double* z, double* p, double* aploc, double* ap,
                          const double* gf, const double* D, const double* dinv,
                          const uint8_t* mult, const int* pairs, double nunique, double eps,
                          double rel, int max_iter, double* part, size_t part_cap,
                          double* frame) {
  dev::CoarseArgs a;
  a.nel = nel;
  a.npts = (size_t)nel * 8;
  a.f = f;
  a.x = x;
  a.r = r;
  a.z = z;
  a.p = p;
  a.aploc = aploc;
  a.ap = ap;
  a.gf = gf;
  a.D = D;
  a.dinv = dinv;
  a.mult = mult;
  a.pairs = reinterpret_cast<const int2*>(pairs);
  a.nunique = nunique;
  a.eps = eps;
  a.rel = rel;
  a.max_iter = max_iter;
  a.frame = frame;
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  int cap = 0;
  cudaError_t ce = cooperative_cap(g_coarse_grid[device], (const void*)dev::k_coarse_cg, 0,
                                   device, &cap);
  if (ce != cudaSuccess) return ce;
  int G = (int)((a.npts + 255) / 256);
  if (G > cap) G = cap;
  // blocks per SM beyond what the occupancy query guarantees are never used
  if ((size_t)7 * G > part_cap) G = (int)(part_cap / 7);
  if (G < 1) return cudaErrorInvalidValue;
  a.partA = part;
  a.partB = part + 4 * (size_t)G;
  void* args[] = {&a};
  count_launch();
  return cudaLaunchCooperativeKernel((const void*)dev::k_coarse_cg, dim3(G), dim3(256), args,
                                     0, s);
}

}  // namespace ssg

namespace ssg {

template <typename T>
static cudaError_t launch_level_cg4(cudaStream_t s, int device, const LevelCgRun& L) {
  constexpr int N = 4;
  dev::LevelCgArgs<T> a;
  a.nel = L.nel;
  a.npts = (size_t)L.nel * N * N * N;
  a.f = (const T*)L.f;
  a.x = (T*)L.x;
  a.r = (T*)L.r;
  a.z = (T*)L.z;
  a.p = (T*)L.p;
  a.aploc = (T*)L.aploc;
  a.ap = (T*)L.ap;
  a.gf = (const T*)L.gf;
  a.D = L.D;
  a.dinv = (const T*)L.dinv;
  a.mult = L.mult;
  a.pairs = reinterpret_cast<const int2*>(L.pairs);
  a.nunique = L.nunique;
  a.eps = L.eps;
  a.max_iter = L.max_iter;
  const size_t smem = dev::level_cg_smem<N>();
  // blocks the device runs at once (a cooperative launch must not exceed it)
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  int c = 0;
  cudaError_t ce = cooperative_cap(g_level_grid[sizeof(T) == 4][device],
                                   (const void*)dev::k_level_cg<N, T>, smem, device, &c);
  if (ce != cudaSuccess) return ce;
  const int groups = (L.nel + 15) / 16;
  int G = groups < c ? groups : c;
  if ((size_t)7 * G > L.part_cap) G = (int)(L.part_cap / 7);
  if (G < 1) return cudaErrorInvalidValue;
  a.partA = L.part;
  a.partB = L.part + 4 * (size_t)G;
  void* args[] = {&a};
  count_launch();
  return cudaLaunchCooperativeKernel((const void*)dev::k_level_cg<N, T>, dim3(G), dim3(256),
                                     args, smem, s);
}

cudaError_t run_level_cg(cudaStream_t s, int device, int n, bool fp32, const LevelCgRun& L) {
  if (n != 4) return cudaErrorInvalidValue;
  return fp32 ? launch_level_cg4<float>(s, device, L) : launch_level_cg4<double>(s, device, L);
}

}  // namespace ssg
