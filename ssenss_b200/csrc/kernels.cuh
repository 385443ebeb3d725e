// Device kernels of the solve path, shared by the dispatch units.
//
// Thread layout of the element kernels: blockDim = (n, n, epb); thread
// (i, j) of element slot z walks the k-planes of element blockIdx.x*epb + z
// (the "2-D thread blocking" of tensor-product operators).  Elements and
// the 1-D matrices live in dynamic shared memory.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace ssg {
namespace dev {

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
  auto add = [&](int2 p, int node) {
    if (p.x >= 0) {
      const size_t s = (size_t)p.x * NT + node;
      double v = (double)in[s];
      if (mask) v = v * mask[s];
      acc += v;
      ++cnt;
    }
  };
  if (i == 0) add(pr[0], face_node(N, pr[0].y, k, j));
  if (i == M) add(pr[1], face_node(N, pr[1].y, k, j));
  if (j == 0) add(pr[2], face_node(N, pr[2].y, k, i));
  if (j == M) add(pr[3], face_node(N, pr[3].y, k, i));
  if (k == 0) add(pr[4], face_node(N, pr[4].y, j, i));
  if (k == M) add(pr[5], face_node(N, pr[5].y, j, i));
  if (ei && ej) {
    const int q = 6 + ((i == M) | ((j == M) << 1));
    add(pr[q], edge_node(N, pr[q].y, k));
  }
  if (ek && ei) {
    const int q = 10 + ((i == M) | ((k == M) << 1));
    add(pr[q], edge_node(N, pr[q].y, j));
  }
  if (ek && ej) {
    const int q = 14 + ((j == M) | ((k == M) << 1));
    add(pr[q], edge_node(N, pr[q].y, i));
  }
  if (ei && ej && ek) {
    const int q = 18 + ((i == M) | ((j == M) << 1) | ((k == M) << 2));
    add(pr[q], corner_node(N, pr[q].y));
  }
  return acc;
}

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

}  // namespace dev
}  // namespace ssg
