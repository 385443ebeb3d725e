// Device kernels of the solve path, shared by the dispatch units.
//
// Thread layout of the element kernels: blockDim = (n, n, epb); thread
// (i, j) of element slot z walks the k-planes of element blockIdx.x*epb + z
// (the "2-D thread blocking" of tensor-product operators).  Elements and
// the 1-D matrices live in dynamic shared memory.
#pragma once

#include <cuda/atomic>
#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

#include "ssg_kernels.h"

namespace ssg {
namespace dev {

// 1/m for a node multiplicity m >= 1, bitwise the IEEE quotient 1.0 / m:
// powers of two (every multiplicity of a conforming mesh: 1, 2, 4, 8) by
// their exponent alone, anything else by the division.
__device__ __forceinline__ double inv_count(unsigned m) {
  if ((m & (m - 1)) == 0u)
    return __longlong_as_double((long long)(1023 - (__ffs((int)m) - 1)) << 52);
  return 1.0 / (double)m;
}

// ---------------------------------------------------------------------------
// node numbering of faces / edges / corners (src/global.c:38-177)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int face_node(int n, int f, int a, int b) {
  const int m = n - 1;
  switch (f) {
    case 0: return (a * n + b) * n;          // w: [a][b][0]
    case 1: return (a * n + b) * n + m;      // e: [a][b][n-1]
    case 2: return (a * n) * n + b;          // s: [a][0][b]
    case 3: return (a * n + m) * n + b;      // n: [a][n-1][b]
    case 4: return a * n + b;                // b: [0][a][b]
    default: return (m * n + a) * n + b;     // t: [n-1][a][b]
  }
}

__device__ __forceinline__ int edge_node(int n, int q, int p) {
  const int m = n - 1;
  switch (q) {
    case 0: return (p * n) * n;
    case 1: return (p * n) * n + m;
    case 2: return (p * n + m) * n;
    case 3: return (p * n + m) * n + m;
    case 4: return p * n;
    case 5: return p * n + m;
    case 6: return (m * n + p) * n;
    case 7: return (m * n + p) * n + m;
    case 8: return p;
    case 9: return m * n + p;
    case 10: return (m * n) * n + p;
    default: return (m * n + m) * n + p;
  }
}

__device__ __forceinline__ int corner_node(int n, int c) {
  const int m = n - 1;
  return (((c >> 2) & 1) * m * n + ((c >> 1) & 1) * m) * n + (c & 1) * m;
}

// ---------------------------------------------------------------------------
// DSS of one local node (direct_stiffness_summation, src/global.c:241-257):
// the node's own value plus its neighbours' pre-sum copies, in the
// reference's order -- faces w, e, s, n, b, t, then edges sw..tn, then
// corners -- through the pairing pr (26 (element, matched index) pairs of
// this node's element).  FP64 accumulation; cnt = contributions added.
// ---------------------------------------------------------------------------
template <int N, typename T>
__device__ __forceinline__ double dss_gather(const T* __restrict__ in,
                                             const double* __restrict__ mask,
                                             const int2* pr, size_t gi, int loc, int& cnt) {
  constexpr int NT = N * N * N, M = N - 1;
  const int i = loc % N, j = (loc / N) % N, k = loc / (N * N);
  double acc = (double)in[gi];
  if (mask) acc = acc * mask[gi];
  cnt = 0;
  const bool ei = i == 0 || i == M, ej = j == 0 || j == M, ek = k == 0 || k == M;
  if (!(ei || ej || ek)) return acc;
  // source of every possible contribution, in the reference's order: the
  // x-face (w/e), y-face (s/n), z-face (b/t), the xy-, xz-, yz-edge, the
  // corner; -1 where the node has none.  All loads are issued before the
  // additions, which then run in that order.
  long long s0 = -1, s1 = -1, s2 = -1, s3 = -1, s4 = -1, s5 = -1, s6 = -1;
  if (ei) {
    const int2 p = pr[i == M];
    if (p.x >= 0) s0 = (long long)p.x * NT + face_node(N, p.y, k, j);
  }
  if (ej) {
    const int2 p = pr[2 + (j == M)];
    if (p.x >= 0) s1 = (long long)p.x * NT + face_node(N, p.y, k, i);
  }
  if (ek) {
    const int2 p = pr[4 + (k == M)];
    if (p.x >= 0) s2 = (long long)p.x * NT + face_node(N, p.y, j, i);
  }
  if (ei && ej) {
    const int2 p = pr[6 + ((i == M) | ((j == M) << 1))];
    if (p.x >= 0) s3 = (long long)p.x * NT + edge_node(N, p.y, k);
  }
  if (ek && ei) {
    const int2 p = pr[10 + ((i == M) | ((k == M) << 1))];
    if (p.x >= 0) s4 = (long long)p.x * NT + edge_node(N, p.y, j);
  }
  if (ek && ej) {
    const int2 p = pr[14 + ((j == M) | ((k == M) << 1))];
    if (p.x >= 0) s5 = (long long)p.x * NT + edge_node(N, p.y, i);
  }
  if (ei && ej && ek) {
    const int2 p = pr[18 + ((i == M) | ((j == M) << 1) | ((k == M) << 2))];
    if (p.x >= 0) s6 = (long long)p.x * NT + corner_node(N, p.y);
  }
#define SSG_LD(S) ((S) >= 0 ? (mask ? (double)in[(S)] * mask[(S)] : (double)in[(S)]) : 0.0)
  const double v0 = SSG_LD(s0), v1 = SSG_LD(s1), v2 = SSG_LD(s2), v3 = SSG_LD(s3),
               v4 = SSG_LD(s4), v5 = SSG_LD(s5), v6 = SSG_LD(s6);
#undef SSG_LD
  if (s0 >= 0) { acc += v0; ++cnt; }
  if (s1 >= 0) { acc += v1; ++cnt; }
  if (s2 >= 0) { acc += v2; ++cnt; }
  if (s3 >= 0) { acc += v3; ++cnt; }
  if (s4 >= 0) { acc += v4; ++cnt; }
  if (s5 >= 0) { acc += v5; ++cnt; }
  if (s6 >= 0) { acc += v6; ++cnt; }
  return acc;
}

// Node visited by task t of an element, tasks ordered by node class so a
// warp's nodes share one branch path: face interiors (6 (N-2)^2), edge
// interiors (12 (N-2)), corners (8), interior nodes ((N-2)^3).
template <int N>
__device__ __forceinline__ int class_ordered_node(int t) {
  if constexpr (N <= 2) {
    return t;   // every node is a corner
  } else {
    constexpr int I = N - 2, F = 6 * I * I, E = 12 * I;
    if (t < F) {
      const int f = t / (I * I), r = t % (I * I);
      return face_node(N, f, 1 + r / I, 1 + r % I);
    }
    t -= F;
    if (t < E) return edge_node(N, t / I, 1 + t % I);
    t -= E;
    if (t < 8) return corner_node(N, t);
    t -= 8;
    const int a = t / (I * I), b = (t / I) % I, c = t % I;
    return ((1 + a) * N + 1 + b) * N + 1 + c;
  }
}

// CG direction update fused into the operator (device copy of PUpdateArgs)
struct PUpdate {
  const void* z = nullptr;        // T*
  const double* beta = nullptr;
  const double* c = nullptr;      // nullspace constant (pressure) or null
  const double* mask = nullptr;
  const double* stop = nullptr;   // solver's stop flag: skip when set
  int first = 0;
  double* part = nullptr;         // set: also reduce p . (A p) (unweighted)
};

// ---------------------------------------------------------------------------
// block reduction of NQ doubles over a 1-D block whose size is a multiple of
// 32; fixed shuffle pattern, so the result is deterministic.  Valid in
// thread 0.  sred: NQ * 32 doubles of shared memory.
// ---------------------------------------------------------------------------
template <int NQ>
__device__ __forceinline__ void block_reduce(double (&v)[NQ], double* sred) {
  const int tid = threadIdx.x;
  const int lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double x = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sred[q * 32 + wid] = x;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double x = lane < nw ? sred[q * 32 + lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      v[q] = x;
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
__device__ inline void apply_scalar_op(const ScalarOp& op, const double* __restrict__ sums) {
  double* f = op.frame;
  switch (op.code) {
    case OP_NONE:
      break;
    case OP_CG_INIT_C:   // c = (w.z)/nunique (pressure); a new solve starts
      f[F_C] = op.pressure ? sums[0] / op.nunique : 0.0;
      f[F_ITER] = 0.0;
      f[F_DONE] = 0.0;
      break;
    case OP_CG_INIT_RDZ:  // rdz = (r w).p, |r|_w ; reset counters
      f[F_RDZ] = sums[0];
      f[F_ERR0] = sqrt(sums[1]);
      f[F_ITER] = 0.0;
      f[F_DONE] = 0.0;
      f[F_ERR] = sqrt(sums[1]);
      break;
    case OP_CG_ALPHA:     // alpha = rdz / (p w).ap
      f[F_PAP] = sums[0];
      f[F_ALPHA] = f[F_RDZ] / sums[0];
      break;
    case OP_CG_BETA: {    // sums: (r w).z, (r w).r, w.z, w.r
      const double c = op.pressure ? sums[2] / op.nunique : 0.0;
      const double rdz = sums[0] - c * sums[3];
      f[F_C] = c;
      f[F_BETA] = rdz / f[F_RDZ];
      f[F_RDZ] = rdz;
      const double err = sqrt(sums[1]);
      f[F_ERR] = err;
      f[F_ITER] += 1.0;
      const bool go = (err > op.eps) && (f[F_ITER] < (double)op.max_iter);
      f[F_DONE] = go ? 0.0 : 1.0;
      if (op.hist && (int)f[F_ITER] <= op.hist_cap) op.hist[(int)f[F_ITER] - 1] = err;
      break;
    }
    case OP_NULL_C:       // c = (w.x)/nunique into frame slot
      f[F_C] = sums[0] / op.nunique;
      break;
    case OP_FCG_BETA:     // beta_k = sums[k] / pap[k]
      for (int k = 0; k < op.m; ++k) f[F_FBETA + k] = sums[k] / f[F_FPAP + op.pap_idx[k]];
      break;
    case OP_FCG_ALPHA:    // pap0 and alpha = (p0 w).r / pap0
      f[F_FPAP + op.pap_idx[0]] = sums[0];
      f[F_ALPHA] = sums[1] / sums[0];
      break;
    case OP_FCG_ERR: {
      const double err = sqrt(sums[0]);
      f[F_ERR] = err;
      f[F_ITER] += 1.0;
      const bool go = (err > op.eps) && (f[F_ITER] < (double)op.max_iter);
      f[F_DONE] = go ? 0.0 : 1.0;
      if (op.hist && (int)f[F_ITER] <= op.hist_cap) op.hist[(int)f[F_ITER] - 1] = err;
      break;
    }
    case OP_ERR0:
      f[F_ERR0] = sqrt(sums[0]);
      f[F_ITER] = 0.0;
      f[F_DONE] = 0.0;
      f[F_ERR] = sqrt(sums[0]);
      break;
    case OP_STORE_PAP:
      f[F_PAP] = sums[0];
      break;
    case OP_CG_INIT_RDZ_ALPHA:
      f[F_RDZ] = sums[0];
      f[F_ERR0] = sqrt(sums[1]);
      f[F_ITER] = 0.0;
      f[F_DONE] = 0.0;
      f[F_ERR] = sqrt(sums[1]);
      f[F_ALPHA] = sums[0] / f[F_PAP];
      break;
  }
}

// ---------------------------------------------------------------------------
// end of a reducing kernel: thread 0 holds the block's NQ partial sums.  They
// are stored at part[q * gridDim.x + block]; when op.counter is set, the
// last block to arrive sums all partials in index order (so the result does
// not depend on which block is last), stores them in op.sums, applies the
// solver scalar algebra and re-arms the counter.
// ---------------------------------------------------------------------------
template <int NQ>
__device__ __forceinline__ void finish(const double (&v)[NQ], double* __restrict__ part,
                                       const ScalarOp& op, double* sred) {
  __shared__ int s_last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) part[q * gridDim.x + blockIdx.x] = v[q];
    s_last = 0;
    if (op.counter) {
      // release: this block's partials are visible before its arrival
      // counts; acquire: the last block sees every partial
      cuda::atomic_ref<unsigned, cuda::thread_scope_device> arrived(*op.counter);
      const unsigned prev = arrived.fetch_add(1u, cuda::memory_order_acq_rel);
      s_last = prev == gridDim.x - 1;
    }
  }
  __syncthreads();
  if (!s_last) return;
  double s[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    s[q] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
      s[q] += __ldcg(part + (size_t)q * gridDim.x + b);
  }
  block_reduce<NQ>(s, sred);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) op.sums[q] = s[q];
    apply_scalar_op(op, op.sums);
    *op.counter = 0u;
  }
}


// One value per thread of a block of any shape (flat index tid < nthr <=
// 256): block sum in a fixed order, then finish<1>'s last-block protocol.
__device__ __forceinline__ void finish_flat(double v, int tid, int nthr,
                                            double* __restrict__ part, const ScalarOp& op,
                                            double* sflat) {
  __shared__ int s_last;
  auto block_sum = [&](double x) -> double {
    sflat[tid] = x;
    __syncthreads();
    double t = 0.0;
    if (tid < 32) {
      for (int q = tid; q < nthr; q += 32) t += sflat[q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    }
    __syncthreads();
    return t;   // valid in tid 0
  };
  const double b = block_sum(v);
  if (tid == 0) {
    part[blockIdx.x] = b;
    s_last = 0;
    if (op.counter) {
      cuda::atomic_ref<unsigned, cuda::thread_scope_device> arrived(*op.counter);
      const unsigned prev = arrived.fetch_add(1u, cuda::memory_order_acq_rel);
      s_last = prev == gridDim.x - 1;
    }
  }
  __syncthreads();
  if (!s_last) return;
  double x = 0.0;
  for (int q = tid; q < (int)gridDim.x; q += nthr) x += __ldcg(part + q);
  const double total = block_sum(x);
  if (tid == 0) {
    op.sums[0] = total;
    apply_scalar_op(op, op.sums);
    *op.counter = 0u;
  }
}


// Ask L2 for a contiguous chunk ahead of its use (a hint: no destination,
// no completion to wait for).  Address and size 16-byte multiples.
// D = A B + C on the FP64 tensor cores, one m8n8k4 tile (lane = 4g + t):
// a = A[g][t], b = B[t][g], {c0, c1} = C[g][2t], C[g][2t + 1]
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b, double c0,
                                     double c1) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%4,%5};\n"
               : "=d"(d0), "=d"(d1)
               : "d"(a), "d"(b), "d"(c0), "d"(c1));
}

__device__ __forceinline__ void bulk_prefetch_l2(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
}

// ---------------------------------------------------------------------------
// element operator building blocks (k_ax in kernels.cu, the small-level
// cooperative CG in coarse.cu)
// ---------------------------------------------------------------------------
// padded row stride of the shared 1-D matrices: even (16-byte aligned rows
// for double2 loads) and chosen so the rows fall on distinct bank groups
template <int N>
struct AxLayout {
  static constexpr int P = (N % 2 == 0) ? N + 2 : N + 1;   // matrix rows
  static constexpr int Q = N + (N & 1);                    // field rows
};

// sum_m a[m] b[m] over m = 0..N-1 in order, both rows 16-byte aligned
template <int N>
__device__ __forceinline__ double row_dot(const double* a, const double* b) {
  double s = 0.0;
#pragma unroll
  for (int m = 0; m + 1 < N; m += 2) {
    const double2 x = *reinterpret_cast<const double2*>(a + m);
    const double2 y = *reinterpret_cast<const double2*>(b + m);
    s += x.x * y.x;
    s += x.y * y.y;
  }
  if (N & 1) s += a[N - 1] * b[N - 1];
  return s;
}

// sum_m a[m] b[m * stride] over m in order; a a 16-byte aligned row
template <int N>
__device__ __forceinline__ double row_col_dot(const double* a, const double* b, int stride) {
  double s = 0.0;
#pragma unroll
  for (int m = 0; m + 1 < N; m += 2) {
    const double2 x = *reinterpret_cast<const double2*>(a + m);
    s += x.x * b[m * stride];
    s += x.y * b[(m + 1) * stride];
  }
  if (N & 1) s += a[N - 1] * b[(N - 1) * stride];
  return s;
}

// sum_m a[m] r[m] over m in order; a a 16-byte aligned row, r registers
template <int N>
__device__ __forceinline__ double row_reg_dot(const double* a, const double (&r)[N]) {
  double s = 0.0;
#pragma unroll
  for (int m = 0; m + 1 < N; m += 2) {
    const double2 x = *reinterpret_cast<const double2*>(a + m);
    s += x.x * r[m];
    s += x.y * r[m + 1];
  }
  if (N & 1) s += a[N - 1] * r[N - 1];
  return s;
}

// Shared memory: D, D^T, S, S^T rows (padded), then per element the u plane
// stack and the r/s fluxes.  Every per-thread access to a 1-D matrix is a
// row, read as double2.
template <int N>
struct AxSmem {
  static constexpr int P = AxLayout<N>::P, Q = AxLayout<N>::Q;
  static constexpr int PLANE = N * Q, BLK = N * PLANE;
  static constexpr int MATS = 4 * N * P;   // doubles of D, D^T, S, S^T
};

// D, D^T, S (Helmholtz) or D, S^T into the block's shared rows
template <int N, bool HELM>
__device__ __forceinline__ void ax_load_mats(double* sD, const double* __restrict__ Dg,
                                             const double* __restrict__ Sg, int tid,
                                             int nthr) {
  constexpr int P = AxSmem<N>::P;
  double* sDT = sD + N * P;
  double* sS = sDT + N * P;
  double* sST = sS + N * P;
  for (int q = tid; q < N * N; q += nthr) {
    const int r = q / N, c = q % N;
    const double d = Dg[q], sv = HELM ? Sg[q] : Dg[q];
    sD[r * P + c] = d;
    sDT[c * P + r] = d;
    sS[r * P + c] = sv;
    sST[c * P + r] = sv;
  }
}

// One element's operator, thread (i, j) of its N x N plane owning the
// k-column (k in registers); FUSEP first forms the direction
// p = (first ? z - c : beta p + (z - c)) .* mask, stored back into u.  Both
// block barriers are inside, so every thread of the block calls it (active
// false for a padding slot).  Returns this thread's share of p . (A p)
// (FUSEP).  sD: the four matrices (ax_load_mats); su, sw0, sw1: this
// slot's planes.
template <int N, typename T, bool HELM, bool FUSEP>
__device__ __forceinline__ double ax_element(int e, bool active, int i, int j, const double* sD,
                                             double* su, double* sw0, double* sw1,
                                             T* __restrict__ u, T* __restrict__ au,
                                             const T* __restrict__ gf, size_t npts,
                                             const double* __restrict__ bj, double lambda,
                                             const T* __restrict__ z, double beta, double c,
                                             const double* __restrict__ mask, bool first) {
  constexpr int NN = N * N, P = AxSmem<N>::P, Q = AxSmem<N>::Q, PLANE = AxSmem<N>::PLANE;
  const double* sDT = sD + N * P;
  const double* sS = sDT + N * P;
  const double* sST = sS + N * P;
  const size_t off = (size_t)(active ? e : 0) * (NN * N) + j * N + i;
  double ru[N], rw2[N];
  if (FUSEP) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      double v = 0.0;
      if (active) {
        const size_t o = off + (size_t)k * NN;
        const double zc = (double)z[o] - c;
        v = first ? zc : beta * (double)u[o] + zc;
        if (mask) v = v * mask[o];
        const T vt = (T)v;
        u[o] = vt;
        v = (double)vt;
      }
      ru[k] = v;
      su[k * PLANE + j * Q + i] = v;
    }
  } else {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      ru[k] = active ? (double)u[off + (size_t)k * NN] : 0.0;
      su[k * PLANE + j * Q + i] = ru[k];
    }
  }
  __syncthreads();
  // r-derivative with S for Helmholtz (the swapped deriv_matrix), D otherwise
  const double* Dx = HELM ? sS : sD;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    const double ur = row_dot<N>(Dx + i * P, su + k * PLANE + j * Q);
    const double us = row_col_dot<N>(sD + j * P, su + k * PLANE + i, Q);
    const double ut = row_reg_dot<N>(sD + k * P, ru);
    const size_t o = off + (size_t)k * NN;
    double g0 = 0, g1 = 0, g2 = 0, g3 = 0, g4 = 0, g5 = 0;
    if (active) {
      g0 = (double)__ldg(gf + o);
      g1 = (double)__ldg(gf + npts + o);
      g2 = (double)__ldg(gf + 2 * npts + o);
      g3 = (double)__ldg(gf + 3 * npts + o);
      g4 = (double)__ldg(gf + 4 * npts + o);
      g5 = (double)__ldg(gf + 5 * npts + o);
    }
    sw0[k * PLANE + j * Q + i] = g0 * ur + g1 * us + g2 * ut;
    sw1[k * PLANE + j * Q + i] = g1 * ur + g3 * us + g4 * ut;
    rw2[k] = g2 * ur + g4 * us + g5 * ut;
  }
  __syncthreads();
  // transposed derivatives: r with D^T, s and t with S^T (= D^T for Poisson)
  double pap = 0.0;   // p . (A p) over this thread's points (FUSEP)
#pragma unroll
  for (int k = 0; k < N; ++k) {
    const double acc = row_dot<N>(sDT + i * P, sw0 + k * PLANE + j * Q);
    const double acs = row_col_dot<N>(sST + j * P, sw1 + k * PLANE + i, Q);
    const double act = row_reg_dot<N>(sST + k * P, rw2);
    double out = (acc + acs) + act;
    if (HELM && active) out += lambda * (__ldg(bj + off + (size_t)k * NN) * ru[k]);
    if (active) au[off + (size_t)k * NN] = (T)out;
    if (FUSEP && active) pap += ru[k] * (double)(T)out;
  }
  return pap;
}

// ---------------------------------------------------------------------------
// line-form element operator (k_axl in kernels.cu, the fused cooperative
// smoother in coarse.cu): each thread contracts one whole line of an
// element (N points along i, j or k) held in registers, so a matrix row is
// read once per line instead of a shared row and a shared field value per
// multiply-add.  Per element: the field is staged in shared memory; lines
// along i and j give the r- and s-derivatives; the lines along k take the
// t-derivative in registers, apply the six metric terms at their points and
// form the t-transposed contribution S^T w2 in registers; lines along i and
// j then turn w0 and w1 into D^T w0 and S^T w1 (D for Poisson) in place, and
// the k-lines write the output (acc + acs) + act, the order of ax_element:
// three staged fields and four block barriers per element group.  The matrices sit in shared memory and every lane of a warp
// reads the same entry (a broadcast), two entries per paired load.  EPB
// elements per group fill about 256 threads.  The arithmetic runs in the
// storage type T: FP64 for the solves, FP32 in the mixed-precision V-cycle
// (the fused direction update and the p . (A p) sum stay FP64).
// ---------------------------------------------------------------------------
template <int N>
struct AxLine {
  static constexpr int EPB = (256 / (N * N)) > 0 ? 256 / (N * N) : 1;
  static constexpr int TASKS = EPB * N * N;
  static constexpr int THREADS = (TASKS + 31) / 32 * 32;
  static constexpr int RM = N + (N & 1);                 // matrix rows (pair-aligned)
  static constexpr int RS = N + ((2 - N % 4) + 4) % 4;   // field rows: 2 mod 4 values
  static constexpr int FS = N * N * RS;                  // one staged field
  static constexpr int MATS = 4 * N * RM;
  static constexpr int SMEM = MATS + EPB * 3 * FS;       // values of type T
};

// sum_l A[o][l] x[l] (A rows of RM values, pair-aligned), in l order; every
// lane of the warp reads the same A entries
template <int N, int RM, typename C>
__device__ __forceinline__ C line_row(const C* A, int o, const C (&x)[N]) {
  using V2 = typename std::conditional<sizeof(C) == 8, double2, float2>::type;
  C acc = 0;
#pragma unroll
  for (int l = 0; l + 1 < N; l += 2) {
    const V2 a = *reinterpret_cast<const V2*>(A + o * RM + l);
    acc += a.x * x[l];
    acc += a.y * x[l + 1];
  }
  if (N & 1) acc += A[o * RM + N - 1] * x[N - 1];
  return acc;
}

// dst[o * stride] (=, or += when ADD) sum_l A[o][l] x[l] for o < N; the
// output loop is not unrolled, so a line's matrix rows are read one row at
// a time and the registers hold the line only
template <int N, int RM, bool ADD, typename C>
__device__ __forceinline__ void line_apply(const C* A, const C (&x)[N], C* dst, int stride) {
#pragma unroll 2
  for (int o = 0; o < N; ++o) {
    const C v = line_row<N, RM, C>(A, o, x);
    if (ADD)
      dst[o * stride] += v;
    else
      dst[o * stride] = v;
  }
}

// D, D^T, S (Helmholtz) or D, S^T = D^T into the first MATS values of the
// block's shared memory; visible after the next barrier
template <int N, typename T, bool HELM>
__device__ __forceinline__ void axl_load_mats(T* sD, const double* __restrict__ Dg,
                                              const double* __restrict__ Sg) {
  constexpr int RM = AxLine<N>::RM;
  T* sDT = sD + N * RM;
  T* sS = sDT + N * RM;
  T* sST = sS + N * RM;
  for (int q = threadIdx.x; q < N * N; q += blockDim.x) {
    const int r = q / N, c = q % N;
    const T d = (T)Dg[q], sv = HELM ? (T)Sg[q] : d;
    sD[r * RM + c] = d;
    sDT[c * RM + r] = d;
    sS[r * RM + c] = sv;
    sST[c * RM + r] = sv;
  }
}

// A_e u for the ne <= EPB elements e0 .. e0 + ne - 1, all threads of a block
// of AxLine<N>::THREADS (barriers inside); sD: the matrices (axl_load_mats)
// followed by the group's field space.  FUSEP: the input is the direction
// p = (first ? z - c : beta u + (z - c)) .* mask, written back to u.
// rdot, mult (optional): also sum (rdot w) p over the staged points, w =
// 1 / mult, into *rdz.  Returns this thread's share of p . (A p) (FUSEP).
template <int N, typename T, bool HELM, bool FUSEP>
__device__ __forceinline__ double axl_group(int e0, int ne, T* __restrict__ u,
                                            T* __restrict__ au, const T* __restrict__ gf,
                                            size_t npts, const double* __restrict__ bj,
                                            double lambda, const T* __restrict__ z,
                                            double beta, double c,
                                            const double* __restrict__ mask, bool first,
                                            T* sD, const T* __restrict__ rdot,
                                            const uint8_t* __restrict__ mult, double* rdz) {
  using L = AxLine<N>;
  using C = T;
  constexpr int NN = N * N, NT = N * N * N, RM = L::RM, RS = L::RS, FS = L::FS;
  const C* sDT = sD + N * RM;
  const C* sS = sDT + N * RM;
  const C* sST = sS + N * RM;
  C* fld = sD + L::MATS;   // per slot: U, F1, F2 (FS values each)
  const int tid = threadIdx.x;
  const size_t base = (size_t)e0 * NT;
  const int npb = ne > 0 ? ne * NT : 0;   // points of this group
  // the group's six metric chunks into L2 now: they are read only after
  // the three derivative passes (a hint, no buffer; 16-byte aligned chunks
  // of a multiple of 16 bytes only)
  if (tid < 6 && npb > 0) {
    const T* chunk = gf + (size_t)tid * npts + base;
    const unsigned bytes = (unsigned)(npb * sizeof(T));
    if (((reinterpret_cast<uintptr_t>(chunk) | bytes) & 15u) == 0)
      bulk_prefetch_l2(chunk, bytes);
  }
  __syncthreads();   // the previous group's last pass has read the fields
  // P0: stage the field (forming p first when fused), coalesced
  for (int q = tid; q < npb; q += blockDim.x) {
    const size_t o = base + q;
    C v;
    if (FUSEP) {
      const double zc = (double)z[o] - c;
      double pv = first ? zc : beta * (double)u[o] + zc;
      if (mask) pv = pv * mask[o];
      const T vt = (T)pv;
      u[o] = vt;
      v = (C)vt;
      if (rdot) *rdz += ((double)rdot[o] * inv_count(mult[o])) * (double)vt;
    } else {
      v = (C)u[o];
    }
    const int sl = q / NT, p = q % NT;
    fld[sl * 3 * FS + (p / NN) * N * RS + ((p / N) % N) * RS + p % N] = v;
  }
  __syncthreads();
  const bool task = tid < ne * NN;
  const int sl = tid / NN, a0 = (tid % NN) % N, a1 = (tid % NN) / N;
  C* U = fld + sl * 3 * FS;
  C* F1 = U + FS;
  C* F2 = F1 + FS;
  // P1, P2: derivatives along i (r, with S for Helmholtz) and j (s)
  if (task) {
    C x[N];
    {   // lines (j = a0, k = a1) along i
      const C* src = U + a1 * N * RS + a0 * RS;
#pragma unroll
      for (int l = 0; l < N; ++l) x[l] = src[l];
      line_apply<N, RM, false, C>(HELM ? sS : sD, x, F1 + a1 * N * RS + a0 * RS, 1);
    }
    {   // lines (i = a0, k = a1) along j
      const C* src = U + a1 * N * RS + a0;
#pragma unroll
      for (int l = 0; l < N; ++l) x[l] = src[l * RS];
      line_apply<N, RM, false, C>(sD, x, F2 + a1 * N * RS + a0, RS);
    }
  }
  __syncthreads();
  // P3: lines (i = a0, j = a1) along k: the t-derivative in registers, the
  // metric product at each point of the line (w0, w1 in place of ur, us;
  // w2 in registers), then the t-transposed contribution act = S^T w2 of
  // the line, kept in registers for the output pass
  C act[N];
  const size_t eo = base + (size_t)sl * NT + a1 * N + a0;
  if (task) {
    C x[N], w2[N];
    const C* src = U + a1 * RS + a0;
#pragma unroll
    for (int l = 0; l < N; ++l) x[l] = src[l * N * RS];
#pragma unroll 2
    for (int k = 0; k < N; ++k) {
      const C ut = line_row<N, RM, C>(sD, k, x);
      const int q = k * N * RS + a1 * RS + a0;
      const size_t o = eo + (size_t)k * NN;
      const C ur = F1[q], us = F2[q];
      const C g0 = __ldg(gf + o), g1 = __ldg(gf + npts + o), g2 = __ldg(gf + 2 * npts + o),
              g3 = __ldg(gf + 3 * npts + o), g4 = __ldg(gf + 4 * npts + o),
              g5 = __ldg(gf + 5 * npts + o);
      F1[q] = g0 * ur + g1 * us + g2 * ut;
      F2[q] = g1 * ur + g3 * us + g4 * ut;
      w2[k] = g2 * ur + g4 * us + g5 * ut;
    }
#pragma unroll
    for (int k = 0; k < N; ++k) act[k] = line_row<N, RM, C>(sST, k, w2);
  }
  __syncthreads();
  // P4: the r-transposed D^T w0 along i and the s-transposed S^T w1 along
  // j, each written over its own input line (a thread reads the whole line
  // before it writes it)
  if (task) {
    C x[N];
    {   // lines (j = a0, k = a1) along i
      C* line = F1 + a1 * N * RS + a0 * RS;
#pragma unroll
      for (int l = 0; l < N; ++l) x[l] = line[l];
      line_apply<N, RM, false, C>(sDT, x, line, 1);
    }
    {   // lines (i = a0, k = a1) along j
      C* line = F2 + a1 * N * RS + a0;
#pragma unroll
      for (int l = 0; l < N; ++l) x[l] = line[l * RS];
      line_apply<N, RM, false, C>(sST, x, line, RS);
    }
  }
  __syncthreads();
  // P5: the output (acc + acs) + act at each point of the k-line (rows of
  // points across lanes: coalesced stores)
  double pap = 0.0;
  if (task) {
    const int q0 = a1 * RS + a0;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const size_t o = eo + (size_t)k * NN;
      C out = (F1[k * N * RS + q0] + F2[k * N * RS + q0]) + act[k];
      C pv = 0;
      if (HELM || FUSEP) pv = u[o];
      if (HELM) out += (C)lambda * ((C)__ldg(bj + o) * pv);
      au[o] = (T)out;
      if (FUSEP) pap += (double)pv * (double)out;
    }
  }
  return pap;
}

}  // namespace dev
}  // namespace ssg
