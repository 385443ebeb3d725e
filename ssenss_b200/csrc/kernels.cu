// Element operators, direct stiffness summation, transfers and fused vector
// kernels of the SSENSS solve path, for sm_100a.
//
// Precision: fields and factors are stored as T (double, or float inside the
// mixed-precision V-cycle); every kernel computes in FP64 and rounds only on
// store.  (Derivatives of smooth fields taken in FP32 arithmetic lose digits
// in proportion to the operator's condition number; FP32 storage of the
// metric factors is a relative perturbation of the quadratic form and does
// not.)
//
// Local operator (discrete_laplace_operator / discrete_helmholtz_operator,
// src/poisson.c:34-56, src/helmholtz.c:33-49):
//   A_e u = D^T (rho J G . D u)  [+ lambda rho J u]
// streamed once per point: u, the six G_ab * rho * J factors, (rho J), out.
// Each element block and the 1-D derivative matrices sit in shared memory;
// thread (i, j) keeps its k-column of u and of the t-flux in registers.
//
// DSS (direct_stiffness_summation, src/global.c:241-257): each local node
// adds its neighbours' pre-sum copies in the reference's order (faces w, e,
// s, n, b, t; edges sw..tn; corners 0..7) from the pairing built on the host
// (src/init.c:68-130), accumulating in FP64: for FP64 data the result is
// bitwise equal to the reference's.
#include <cuda/atomic>
#include <atomic>
#include <cuda_runtime.h>

#include <initializer_list>
#include <type_traits>

#include <cstdint>
#include <cstdio>

#include "kernels.cuh"
#include "ssg_internal.h"
#include "ssg_kernels.h"

namespace ssg {
namespace dev {

// ---------------------------------------------------------------------------
// local operator of every order but 8, optionally preceded by the CG
// direction update p = ((beta p + (z - c)) .* mask) (first: (z - c) .* mask)
// (src/solver.c:59-60,75-77 with subtract_nullspace folded in): one element
// per (N, N) thread plane, epb planes per block; the element body is
// ax_element (kernels.cuh), shared with the cooperative level smoother
// ---------------------------------------------------------------------------

template <int N, typename T, bool HELM, bool FUSEP>
__global__ void __launch_bounds__(256, (N >= 10 ? 1 : 2)) k_ax(int nel, T* __restrict__ u,
                                               T* __restrict__ au,
                                               const T* __restrict__ gf, size_t npts,
                                               const double* __restrict__ bj,
                                               const double* __restrict__ Dg,
                                               const double* __restrict__ Sg,
                                               double lambda, PUpdate pu, ScalarOp dop) {
  using L = AxSmem<N>;
  if (FUSEP && pu.stop && *pu.stop != 0.0) return;   // uniform over the block
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sD = reinterpret_cast<double*>(smem_raw);
  double* su = sD + L::MATS + threadIdx.z * 3 * L::BLK;
  const int i = threadIdx.x, j = threadIdx.y;
  const int tid = i + N * (j + N * threadIdx.z);
  const int nthr = N * N * blockDim.z;
  ax_load_mats<N, HELM>(sD, Dg, Sg, tid, nthr);   // visible after the first barrier
  const int e = blockIdx.x * blockDim.z + threadIdx.z;
  const T* z = FUSEP ? reinterpret_cast<const T*>(pu.z) : nullptr;
  const double beta = (FUSEP && !pu.first) ? *pu.beta : 0.0;
  const double c = (FUSEP && pu.c) ? *pu.c : 0.0;
  const double pap = ax_element<N, T, HELM, FUSEP>(e, e < nel, i, j, sD, su, su + L::BLK,
                                                   su + 2 * L::BLK, u, au, gf, npts, bj,
                                                   lambda, z, beta, c, pu.mask, pu.first != 0);
  if (FUSEP && pu.part) {
    __shared__ double sflat[256];
    finish_flat(pap, tid, nthr, pu.part, dop, sflat);
  }
}

// ---------------------------------------------------------------------------
// local operator of every order but 8, line form: each thread contracts one
// whole line of an element (N points along i, j or k) held in registers, so
// a matrix row is read once per line instead of a shared row and a shared
// field value per multiply-add.  Per element: the field is staged in shared
// memory; three passes (lines along i, j, k) give the r-, s- and
// t-derivatives; a point-wise pass applies the six metric terms; three
// transposed passes sum D^T w0 + S^T w1 + S^T w2 (D for Poisson) in the
// order (acc + acs) + act of ax_element.  The matrices sit in shared memory
// and every lane of a warp reads the same entry (a broadcast), two entries
// per 16-byte load.  EPB elements per block fill about 256 threads.  Same
// interface as k_ax (optional direction update and p . (A p)).
// ---------------------------------------------------------------------------
template <int N, typename T, bool HELM, bool FUSEP>
__global__ void __launch_bounds__(AxLine<N>::THREADS)
    k_axl(int nel, T* __restrict__ u, T* __restrict__ au, const T* __restrict__ gf,
          size_t npts, const double* __restrict__ bj, const double* __restrict__ Dg,
          const double* __restrict__ Sg, double lambda, PUpdate pu, ScalarOp dop) {
  using L = AxLine<N>;
  if (FUSEP && pu.stop && *pu.stop != 0.0) return;   // uniform over the block
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sD = reinterpret_cast<T*>(smem_raw);
  axl_load_mats<N, T, HELM>(sD, Dg, Sg);
  const int e0 = blockIdx.x * L::EPB;
  const T* z = FUSEP ? reinterpret_cast<const T*>(pu.z) : nullptr;
  const double beta = (FUSEP && !pu.first) ? *pu.beta : 0.0;
  const double c = (FUSEP && pu.c) ? *pu.c : 0.0;
  double rdz = 0.0;
  const double pap = axl_group<N, T, HELM, FUSEP>(
      e0, min(L::EPB, nel - e0), u, au, gf, npts, bj, lambda, z, beta, c, pu.mask,
      pu.first != 0, sD, nullptr, nullptr, &rdz);
  if (FUSEP && pu.part) {
    __shared__ double sflat[AxLine<N>::THREADS];
    finish_flat(pap, threadIdx.x, blockDim.x, pu.part, dop, sflat);
  }
}

// ---------------------------------------------------------------------------
// DSS gather with fused epilogues
//   DSS_PLAIN: out = DSS(mask .* in)
//   DSS_DOT:   store; partial sum (y w) out                       [1]
//   DSS_DOT2:  store; partial sums (y w) out, (y w) y2            [2]
//   DSS_RESID: out = y - DSS; partial sum w out                   [1]
//   DSS_AVG:   out = DSS * w (direct_stiffness_averaging)
//   DSS_SCALE: out = DSS * y (the DSS, then the inverse mass product)
// w = 1 / multiplicity = 1 / (1 + number of contributions).
// ---------------------------------------------------------------------------
template <int N, typename T, int MODE>
// (64 registers, four blocks per SM, except the modes with the longest
// epilogues)
__global__ void __launch_bounds__(256, (MODE == DSS_CGUPD || MODE == DSS_DOT2) ? 3 : 4)
    k_dss(int nel, const T* __restrict__ in,
                                             T* __restrict__ out,
                                             const int* __restrict__ map,
                                             const double* __restrict__ mask,
                                             const T* __restrict__ y,
                                             const T* __restrict__ y2,
                                             double* __restrict__ part,
                                             const double* __restrict__ stop, ScalarOp op,
                                             DssCg cg) {
  constexpr int NT = N * N * N;
  constexpr int I = N > 2 ? N - 2 : 0, ECI = 12 * I;
  if (stop && *stop != 0.0) return;   // uniform over the block
  // the level's DSS map (dss_map_table): one gather word per local point,
  // then the edge/corner source records
  const size_t ntask = (size_t)nel * NT;
  const int* __restrict__ gword = map;
  const int4* __restrict__ ec =
      reinterpret_cast<const int4*>(map + dss_map_records_offset(ntask));
  __shared__ double sred[2 * 32];
  __shared__ double sred4[MODE == DSS_CGUPD ? 4 * 32 : 1];
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  const double alpha = MODE == DSS_CGUPD ? *cg.alpha : 0.0;
  T* const cx = reinterpret_cast<T*>(cg.x);
  const T* const cp = reinterpret_cast<const T*>(cg.p);
  T* const cr = reinterpret_cast<T*>(cg.r);
  const T* const cd = reinterpret_cast<const T*>(cg.dinv);
  T* const cz = reinterpret_cast<T*>(cg.z);
  // one node task per thread, grid-stride over all elements' tasks; no
  // block-wide staging, so no barrier inside the loop
  const size_t S = (size_t)gridDim.x * blockDim.x;
  // two node tasks in flight per thread (q and q + S): every source of both
  // is resolved and loaded before any sum, branch-free, so their load
  // chains (gather word -> neighbour value, or -> record -> values) overlap
  constexpr int U = 2;
  for (size_t q0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q0 < ntask; q0 += U * S) {
    size_t gi[U];
    bool ok[U];
    int src[U][7];
    double own[U], v[U][7];
    // epilogue operands, loaded with the gather (independent of it)
    double ex[U], ep[U], er[U], ed[U], ey[U], ey2[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const size_t q = q0 + u * S;
      ok[u] = q < ntask;
      const size_t qq = ok[u] ? q : 0;
      // nodes in natural order: a warp's own loads and stores are coalesced
      const int e = (int)(qq / NT);
      gi[u] = qq;
      const int gw = __ldg(gword + qq);
      // face interior: the gather word is the neighbour's copy; edges and
      // corners: the ordered lists of the set-up records (-1 = none)
      int4 a = make_int4(-1, -1, -1, -1), b = make_int4(-1, -1, -1, -1);
      if (gw <= -2) {
        const int code = -gw - 2;
        const int4* rec = ec + (size_t)e * (ECI + 16) + (code >> 1);
        a = __ldg(rec);
        if (code & 1) b = __ldg(rec + 1);
      }
      src[u][0] = gw >= 0 ? gw : a.x;
      src[u][1] = a.y;
      src[u][2] = a.z;
      src[u][3] = a.w;
      src[u][4] = b.x;
      src[u][5] = b.y;
      src[u][6] = b.z;
      own[u] = (double)in[qq];
      if (mask) own[u] = own[u] * mask[qq];
      if (MODE == DSS_CGUPD) {
        ex[u] = (double)cx[qq];
        ep[u] = (double)cp[qq];
        er[u] = (double)cr[qq];
        ed[u] = (double)cd[qq];
      }
      if (MODE == DSS_RESID || MODE == DSS_DOT || MODE == DSS_DOT2 || MODE == DSS_SCALE)
        ey[u] = (double)y[qq];
      if (MODE == DSS_DOT2) ey2[u] = (double)y2[qq];
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll 7
      for (int m = 0; m < 7; ++m) {
        v[u][m] = 0.0;
        if (src[u][m] >= 0) {
          v[u][m] = (double)in[src[u][m]];
          if (mask) v[u][m] = v[u][m] * mask[src[u][m]];
        }
      }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (ok[u]) {
      // the reference's order: own value, then the sources in slot order
      double acc = own[u];
      int cnt = 0;
#pragma unroll 7
      for (int m = 0; m < 7; ++m)
        if (src[u][m] >= 0) {
          acc += v[u][m];
          ++cnt;
        }
      const size_t g = gi[u];
      const double w = inv_count(1u + (unsigned)cnt);
      if (MODE == DSS_CGUPD) {
        // ap = acc: x += alpha p; r -= alpha ap; z = dinv r  (src/solver.c:66-71)
        cx[g] = (T)(ex[u] + alpha * ep[u]);
        const T rq = (T)(er[u] + -alpha * acc);
        cr[g] = rq;
        const T zq = (T)((double)rq * ed[u]);
        cz[g] = zq;
        const double rw = (double)rq * w;
        s0 += rw * (double)zq;
        s1 += rw * (double)rq;
        s2 += w * (double)zq;
        s3 += rw;
      } else if (MODE == DSS_RESID) {
        const T rv = (T)(ey[u] + -acc);
        out[g] = rv;
        s0 += (double)rv * w;
      } else if (MODE == DSS_AVG) {
        out[g] = (T)(acc * w);
      } else if (MODE == DSS_SCALE) {
        out[g] = (T)(acc * ey[u]);
      } else {
        const T av = (T)acc;
        out[g] = av;
        if (MODE == DSS_DOT || MODE == DSS_DOT2) {
          const double yw = ey[u] * w;
          s0 += yw * (double)av;
          if (MODE == DSS_DOT2) s1 += yw * ey2[u];
        }
      }
      }
    }
  }
  if (MODE == DSS_DOT || MODE == DSS_RESID) {
    double v[1] = {s0};
    block_reduce<1>(v, sred);
    finish<1>(v, part, op, sred);
  } else if (MODE == DSS_DOT2) {
    double v[2] = {s0, s1};
    block_reduce<2>(v, sred);
    finish<2>(v, part, op, sred);
  } else if (MODE == DSS_CGUPD) {
    double v[4] = {s0, s1, s2, s3};
    block_reduce<4>(v, sred4);
    finish<4>(v, part, op, sred4);
  }
}

// DSS of three fields `stride` apart that share one gather map (the
// components of a vector field): out_c = DSS(in_c), with SCALE times y (the
// inverse mass); each node's sources are decoded once for the three, and
// each sum is the reference's order as in k_dss
template <int N, bool SCALE>
__global__ void __launch_bounds__(256) k_dss3(int nel, const double* __restrict__ in,
                                              double* __restrict__ out, size_t stride,
                                              const int* __restrict__ map,
                                              const double* __restrict__ y) {
  constexpr int NT = N * N * N;
  constexpr int I = N > 2 ? N - 2 : 0, ECI = 12 * I;
  const size_t ntask = (size_t)nel * NT;
  const int4* __restrict__ ec =
      reinterpret_cast<const int4*>(map + dss_map_records_offset(ntask));
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < ntask;
       q += (size_t)gridDim.x * blockDim.x) {
    const int e = (int)(q / NT);
    const int gw = __ldg(map + q);
    int4 a = make_int4(-1, -1, -1, -1), b = make_int4(-1, -1, -1, -1);
    if (gw <= -2) {
      const int code = -gw - 2;
      const int4* rec = ec + (size_t)e * (ECI + 16) + (code >> 1);
      a = __ldg(rec);
      if (code & 1) b = __ldg(rec + 1);
    }
    const int src[7] = {gw >= 0 ? gw : a.x, a.y, a.z, a.w, b.x, b.y, b.z};
    double own[3], v[3][7];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      own[c] = in[c * stride + q];
#pragma unroll
      for (int m = 0; m < 7; ++m) v[c][m] = src[m] >= 0 ? in[c * stride + src[m]] : 0.0;
    }
    const double w = SCALE ? y[q] : 1.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double acc = own[c];
#pragma unroll
      for (int m = 0; m < 7; ++m)
        if (src[m] >= 0) acc += v[c][m];
      out[c * stride + q] = SCALE ? acc * w : acc;
    }
  }
}

// ---------------------------------------------------------------------------
// DSS over runs of P consecutive nodes of an element x-line, for meshes
// whose every face, edge and corner is paired with the opposite one of its
// neighbour (checked on the host when the mesh is set up: every mesh with
// three or more elements along each periodic direction, walls or not, and
// the opposite pairing of small boxes).  There a neighbour's copy of node
// (i, j, k) is the same node with the shared coordinates flipped
// (0 <-> N-1), so the sources of every node follow from the element's 26
// neighbour ids (nb26, -1 for none) without a per-node map:
//   node i of line (j, k) adds, in the reference's order
//   (src/global.c:241-257: faces w e s n b t, edges sw..tn, corners 0..7,
//   pre-sum values):
//     x-face  i = 0: w's (N-1, j, k)      i = N-1: e's (0, j, k)
//     y-face  (j = 0: s, j = N-1: n)      the neighbour's node, j flipped
//     z-face  (k = 0: b, k = N-1: t)      the neighbour's node, k flipped
//     xy-edge i and j extreme             sw / se / nw / ne, i and j flipped
//     xz-edge i and k extreme             bw / be / tw / te, i and k flipped
//     yz-edge j and k extreme             bs / bn / ts / tn, j and k flipped
//     corner  i, j and k extreme          the opposite corner
// Same sums in the same order as k_dss, so the gathered values are bitwise
// the same.  Each thread takes a run of P consecutive nodes of a line (half
// or whole lines, DssRun), loaded and stored as 16- or 8-byte vectors where
// the run allows; consecutive threads take consecutive runs, so a warp's
// loads of its own nodes, of a face or edge neighbour's nodes and its
// stores are contiguous, and only the line ends gather single values.  The
// grid is one full wave of resident blocks walking the runs grid-stride.
// ---------------------------------------------------------------------------
template <int N, typename T>
struct DssRun {
  // nodes per thread, measured on the B200 at the periodic 16^3 box: FP64
  // half lines from N = 6 (n = 8: 14.4 us per DSS + dot against 22.6 us
  // for pairs and 16.4 us for whole lines; n = 12: 39.0 against 41.0 for
  // whole lines), whole lines below and at odd orders (no vector split);
  // FP32 whole lines (the mixed V-cycle's gather + update at n = 8: 19.5
  // against 20.4 ms per solve with half lines)
  static constexpr int P = sizeof(T) == 8 ? ((N % 2 == 0 && N >= 6) ? N / 2 : N) : N;
  static constexpr int R = N / P;   // runs per line
};

template <int P, typename T>
__device__ __forceinline__ void ld_run(const T* __restrict__ p, double (&v)[P]) {
  if constexpr (sizeof(T) == 8 && P % 2 == 0) {
#pragma unroll
    for (int q = 0; q < P; q += 2) {
      const double2 t = *reinterpret_cast<const double2*>(p + q);
      v[q] = t.x;
      v[q + 1] = t.y;
    }
  } else if constexpr (sizeof(T) == 4 && P % 4 == 0) {
#pragma unroll
    for (int q = 0; q < P; q += 4) {
      const float4 t = *reinterpret_cast<const float4*>(p + q);
      v[q] = t.x;
      v[q + 1] = t.y;
      v[q + 2] = t.z;
      v[q + 3] = t.w;
    }
  } else if constexpr (sizeof(T) == 4 && P % 2 == 0) {
#pragma unroll
    for (int q = 0; q < P; q += 2) {
      const float2 t = *reinterpret_cast<const float2*>(p + q);
      v[q] = t.x;
      v[q + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int q = 0; q < P; ++q) v[q] = (double)p[q];
  }
}

template <int P, typename T>
__device__ __forceinline__ void st_run(T* __restrict__ p, const T (&v)[P]) {
  if constexpr (sizeof(T) == 8 && P % 2 == 0) {
#pragma unroll
    for (int q = 0; q < P; q += 2)
      *reinterpret_cast<double2*>(p + q) = make_double2(v[q], v[q + 1]);
  } else if constexpr (sizeof(T) == 4 && P % 4 == 0) {
#pragma unroll
    for (int q = 0; q < P; q += 4)
      *reinterpret_cast<float4*>(p + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
  } else if constexpr (sizeof(T) == 4 && P % 2 == 0) {
#pragma unroll
    for (int q = 0; q < P; q += 2)
      *reinterpret_cast<float2*>(p + q) = make_float2(v[q], v[q + 1]);
  } else {
#pragma unroll
    for (int q = 0; q < P; ++q) p[q] = v[q];
  }
}

// The gathered run starting at global node g = run * P: own values plus
// every contribution in the reference's order, and each node's contribution
// count.  MASK: every value (own and neighbours') times the Dirichlet mask at
// its own position.
template <int N, int P, typename T, bool MASK>
__device__ __forceinline__ void gather_run(const T* __restrict__ in,
                                           const double* __restrict__ mask,
                                           const int* __restrict__ nb26, size_t run,
                                           double (&acc)[P], int (&cnt)[P]) {
  constexpr int R = N / P;
  constexpr int M = N - 1, NN = N * N;
  constexpr size_t NT = (size_t)NN * N;
  const size_t line = run / R;
  const int i0 = (int)(run - line * R) * P;
  const size_t e = line / NN;
  const int jk = (int)(line - e * NN);
  const int j = jk % N, k = jk / N;
  const int lo = jk * N + i0;                // local index of the run's first node
  const bool lo_end = i0 == 0, hi_end = i0 + P - 1 == M;
  const bool jhi = j == M, khi = k == M;
  const bool yf = j == 0 || jhi, zf = k == 0 || khi, yz = yf && zf;
  const int dy = jhi ? -M * N : M * N;       // flip j
  const int dz = khi ? -M * NN : M * NN;     // flip k
  const int* __restrict__ nbe = nb26 + e * 26;
  // neighbour element ids of the run's slots (an element's 26 ids are read
  // by all its runs: L1 hits)
  const int nw = lo_end ? __ldg(nbe + 0) : -1;
  const int ne = hi_end ? __ldg(nbe + 1) : -1;
  const int ny = yf ? __ldg(nbe + 2 + jhi) : -1;
  const int nz = zf ? __ldg(nbe + 4 + khi) : -1;
  const int nxy0 = (yf && lo_end) ? __ldg(nbe + 6 + 2 * jhi) : -1;
  const int nxy1 = (yf && hi_end) ? __ldg(nbe + 7 + 2 * jhi) : -1;
  const int nxz0 = (zf && lo_end) ? __ldg(nbe + 10 + 2 * khi) : -1;
  const int nxz1 = (zf && hi_end) ? __ldg(nbe + 11 + 2 * khi) : -1;
  const int nyz = yz ? __ldg(nbe + 14 + jhi + 2 * khi) : -1;
  const int nc0 = (yz && lo_end) ? __ldg(nbe + 18 + 2 * jhi + 4 * khi) : -1;
  const int nc1 = (yz && hi_end) ? __ldg(nbe + 19 + 2 * jhi + 4 * khi) : -1;
  auto val = [&](size_t g) -> double {
    double v = (double)in[g];
    if (MASK) v = v * mask[g];
    return v;
  };
  auto runv = [&](size_t g, double (&v)[P]) {
    ld_run<P, T>(in + g, v);
    if (MASK) {
      double m[P];
      ld_run<P, double>(mask + g, m);
#pragma unroll
      for (int q = 0; q < P; ++q) v[q] = v[q] * m[q];
    }
  };
  double own[P], vy[P], vz[P], vyz[P];
#pragma unroll
  for (int q = 0; q < P; ++q) vy[q] = vz[q] = vyz[q] = 0.0;
  runv(e * NT + lo, own);
  if (ny >= 0) runv((size_t)ny * NT + (lo + dy), vy);
  if (nz >= 0) runv((size_t)nz * NT + (lo + dz), vz);
  if (nyz >= 0) runv((size_t)nyz * NT + (lo + dy + dz), vyz);
  // line ends: node i = 0 reads its sources at i = N-1 (lo + M), node
  // i = N-1 at i = 0 (lo - M)
  const double vw = nw >= 0 ? val((size_t)nw * NT + (lo + M)) : 0.0;
  const double ve = ne >= 0 ? val((size_t)ne * NT + (lo + P - 1 - M)) : 0.0;
  const double vxy0 = nxy0 >= 0 ? val((size_t)nxy0 * NT + (lo + dy + M)) : 0.0;
  const double vxy1 = nxy1 >= 0 ? val((size_t)nxy1 * NT + (lo + P - 1 + dy - M)) : 0.0;
  const double vxz0 = nxz0 >= 0 ? val((size_t)nxz0 * NT + (lo + dz + M)) : 0.0;
  const double vxz1 = nxz1 >= 0 ? val((size_t)nxz1 * NT + (lo + P - 1 + dz - M)) : 0.0;
  const double vc0 = nc0 >= 0 ? val((size_t)nc0 * NT + (lo + dy + dz + M)) : 0.0;
  const double vc1 = nc1 >= 0 ? val((size_t)nc1 * NT + (lo + P - 1 + dy + dz - M)) : 0.0;
#pragma unroll
  for (int q = 0; q < P; ++q) {
    // q == 0 with lo_end is node i = 0, q == P-1 with hi_end node i = N-1
    const bool first = q == 0, last = q == P - 1;
    double a = own[q];
    int c = 0;
    if (first && nw >= 0) { a += vw; ++c; }
    if (last && ne >= 0) { a += ve; ++c; }
    if (ny >= 0) { a += vy[q]; ++c; }
    if (nz >= 0) { a += vz[q]; ++c; }
    if (first && nxy0 >= 0) { a += vxy0; ++c; }
    if (last && nxy1 >= 0) { a += vxy1; ++c; }
    if (first && nxz0 >= 0) { a += vxz0; ++c; }
    if (last && nxz1 >= 0) { a += vxz1; ++c; }
    if (nyz >= 0) { a += vyz[q]; ++c; }
    if (first && nc0 >= 0) { a += vc0; ++c; }
    if (last && nc1 >= 0) { a += vc1; ++c; }
    acc[q] = a;
    cnt[q] = c;
  }
}

template <int N, int P, typename T, int MODE, bool MASK>
__global__ void __launch_bounds__(256) k_dss_runs(int nel, const T* __restrict__ in,
                                                  T* __restrict__ out,
                                                  const int* __restrict__ nb26,
                                                  const double* __restrict__ mask,
                                                  const T* __restrict__ y,
                                                  const T* __restrict__ y2,
                                                  double* __restrict__ part,
                                                  const double* __restrict__ stop, ScalarOp op,
                                                  DssCg cg) {
  if (stop && *stop != 0.0) return;   // uniform over the block
  __shared__ double sred[2 * 32];
  __shared__ double sred4[MODE == DSS_CGUPD ? 4 * 32 : 1];
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  const double alpha = MODE == DSS_CGUPD ? *cg.alpha : 0.0;
  const size_t nruns = (size_t)nel * N * N * (N / P);
  for (size_t run = blockIdx.x * (size_t)blockDim.x + threadIdx.x; run < nruns;
       run += (size_t)gridDim.x * blockDim.x) {
    double acc[P];
    int cnt[P];
    gather_run<N, P, T, MASK>(in, mask, nb26, run, acc, cnt);
    const size_t g = run * P;
    if (MODE == DSS_CGUPD) {
      // ap = acc: x += alpha p; r -= alpha ap; z = dinv r  (src/solver.c:66-71)
      double ex[P], ep[P], er[P], ed[P];
      ld_run<P, T>(reinterpret_cast<const T*>(cg.x) + g, ex);
      ld_run<P, T>(reinterpret_cast<const T*>(cg.p) + g, ep);
      ld_run<P, T>(reinterpret_cast<const T*>(cg.r) + g, er);
      ld_run<P, T>(reinterpret_cast<const T*>(cg.dinv) + g, ed);
      T xo[P], ro[P], zo[P];
#pragma unroll
      for (int q = 0; q < P; ++q) {
        const double w = inv_count(1u + (unsigned)cnt[q]);
        xo[q] = (T)(ex[q] + alpha * ep[q]);
        ro[q] = (T)(er[q] + -alpha * acc[q]);
        zo[q] = (T)((double)ro[q] * ed[q]);
        const double rw = (double)ro[q] * w;
        s0 += rw * (double)zo[q];
        s1 += rw * (double)ro[q];
        s2 += w * (double)zo[q];
        s3 += rw;
      }
      st_run<P, T>(reinterpret_cast<T*>(cg.x) + g, xo);
      st_run<P, T>(reinterpret_cast<T*>(cg.r) + g, ro);
      st_run<P, T>(reinterpret_cast<T*>(cg.z) + g, zo);
    } else {
      double ey[P], ey2[P];
      if (MODE == DSS_RESID || MODE == DSS_DOT || MODE == DSS_DOT2 || MODE == DSS_SCALE)
        ld_run<P, T>(y + g, ey);
      if (MODE == DSS_DOT2) ld_run<P, T>(y2 + g, ey2);
      T o[P];
#pragma unroll
      for (int q = 0; q < P; ++q) {
        const double w = inv_count(1u + (unsigned)cnt[q]);
        if (MODE == DSS_RESID) {
          o[q] = (T)(ey[q] + -acc[q]);
          s0 += (double)o[q] * w;
        } else if (MODE == DSS_AVG) {
          o[q] = (T)(acc[q] * w);
        } else if (MODE == DSS_SCALE) {
          o[q] = (T)(acc[q] * ey[q]);
        } else {
          o[q] = (T)acc[q];
          if (MODE == DSS_DOT || MODE == DSS_DOT2) {
            const double yw = ey[q] * w;
            s0 += yw * (double)o[q];
            if (MODE == DSS_DOT2) s1 += yw * ey2[q];
          }
        }
      }
      st_run<P, T>(out + g, o);
    }
  }
  if (MODE == DSS_DOT || MODE == DSS_RESID) {
    double v[1] = {s0};
    block_reduce<1>(v, sred);
    finish<1>(v, part, op, sred);
  } else if (MODE == DSS_DOT2) {
    double v[2] = {s0, s1};
    block_reduce<2>(v, sred);
    finish<2>(v, part, op, sred);
  } else if (MODE == DSS_CGUPD) {
    double v[4] = {s0, s1, s2, s3};
    block_reduce<4>(v, sred4);
    finish<4>(v, part, op, sred4);
  }
}

// k_dss3 over line runs (the opposite pairing, as k_dss_runs): the three
// components' gathers of a run in flight together
template <int N, int P, bool SCALE>
__global__ void __launch_bounds__(256) k_dss3_runs(int nel, const double* __restrict__ in,
                                                   double* __restrict__ out, size_t stride,
                                                   const int* __restrict__ nb26,
                                                   const double* __restrict__ y) {
  const size_t nruns = (size_t)nel * N * N * (N / P);
  for (size_t run = blockIdx.x * (size_t)blockDim.x + threadIdx.x; run < nruns;
       run += (size_t)gridDim.x * blockDim.x) {
    const size_t g = run * P;
    double w[P];
    if (SCALE) ld_run<P, double>(y + g, w);
    double acc[3][P];
    int cnt[3][P];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      gather_run<N, P, double, false>(in + c * stride, nullptr, nb26, run, acc[c], cnt[c]);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double o[P];
#pragma unroll
      for (int q = 0; q < P; ++q) o[q] = SCALE ? acc[c][q] * w[q] : acc[c][q];
      st_run<P, double>(out + c * stride + g, o);
    }
  }
}

// ---------------------------------------------------------------------------
// tensor-product transfer between orders, stages in x, y, z order
// (interpolate_to_grid / integrate_to_grid, src/interpolation.c:136-176):
// out (no^3) [+]= (A x A x A) in (ni^3), A[o*ni + q] in FP64
// ---------------------------------------------------------------------------
// epb elements per block (their stages side by side in shared memory); NI,
// NO > 0: the orders at compile time (contractions unrolled), 0: runtime
template <typename T, bool ADD, int NI, int NO>
__global__ void __launch_bounds__(256) k_tensor3(int nel, int ni_rt, int no_rt, int epb,
                                                 const double* __restrict__ A,
                                                 const T* __restrict__ in,
                                                 T* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ni = NI > 0 ? NI : ni_rt, no = NO > 0 ? NO : no_rt;
  const int nti = ni * ni * ni, nto = no * no * no, n1 = no * ni * ni, n2 = no * no * ni;
  double* sA = reinterpret_cast<double*>(smem_raw);
  double* sin = sA + no * ni;            // epb x nti
  double* t1 = sin + epb * nti;          // epb x n1
  double* t2 = t1 + epb * n1;            // epb x n2
  const int e0 = blockIdx.x * epb;
  const int ne = nel - e0 < epb ? nel - e0 : epb;
  for (int q = threadIdx.x; q < no * ni; q += blockDim.x) sA[q] = A[q];
  for (int q = threadIdx.x; q < ne * nti; q += blockDim.x)
    sin[q] = (double)in[(size_t)e0 * nti + q];
  __syncthreads();
  for (int qq = threadIdx.x; qq < ne * n1; qq += blockDim.x) {
    const int el = qq / n1, q = qq - el * n1;
    const int o = q % no, kj = q / no;
    const double* x = sin + el * nti + kj * ni;
    double s = 0;
#pragma unroll
    for (int r = 0; r < (NI > 0 ? NI : ni); ++r) s += sA[o * ni + r] * x[r];
    t1[qq] = s;
  }
  __syncthreads();
  for (int qq = threadIdx.x; qq < ne * n2; qq += blockDim.x) {
    const int el = qq / n2, q = qq - el * n2;
    const int o1 = q % no, o2 = (q / no) % no, k = q / (no * no);
    const double* x = t1 + el * n1;
    double s = 0;
#pragma unroll
    for (int r = 0; r < (NI > 0 ? NI : ni); ++r) s += sA[o2 * ni + r] * x[(k * ni + r) * no + o1];
    t2[qq] = s;
  }
  __syncthreads();
  for (int qq = threadIdx.x; qq < ne * nto; qq += blockDim.x) {
    const int el = qq / nto, q = qq - el * nto;
    const int o12 = q % (no * no), o3 = q / (no * no);
    const double* x = t2 + el * n2;
    double s = 0;
#pragma unroll
    for (int r = 0; r < (NI > 0 ? NI : ni); ++r) s += sA[o3 * ni + r] * x[r * no * no + o12];
    const size_t g = (size_t)e0 * nto + qq;
    if (ADD)
      out[g] = (T)((double)out[g] + s);
    else
      out[g] = (T)s;
  }
}

// ---------------------------------------------------------------------------
// fused vector kernels (grid-stride, 256 threads, one partial per block)
// ---------------------------------------------------------------------------
#define SSG_GRID_LOOP(q, n)                                                    \
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < (n);     \
       q += (size_t)gridDim.x * blockDim.x)

// Helmholtz diagonal before DSS: kdiag + (lambda rho) J, the reference's
// association (src/helmholtz.c:66)
__global__ void __launch_bounds__(256) k_helm_diag(size_t npts, size_t nt,
                                                   const double* __restrict__ kd,
                                                   const double* __restrict__ rho,
                                                   const double* __restrict__ det, double lam,
                                                   double* __restrict__ out) {
  SSG_GRID_LOOP(q, npts) out[q] = kd[q] + (lam * rho[q % nt]) * det[q];
}

__global__ void __launch_bounds__(256) k_recip(size_t npts, double* __restrict__ x) {
  SSG_GRID_LOOP(q, npts) x[q] = 1.0 / x[q];
}

// CG step after ap is known (src/solver.c:66-71):
//   x += alpha p; r -= alpha ap; z = dinv .* r
// partials: (r w).z, (r w).r, w.z, w.r
// Grid-stride loops with four points in flight per thread: the loads of
// points q, q + S, q + 2S, q + 3S (S = grid stride; those past the end
// predicated off) are issued before any of them is used.  Each thread's
// partial sums follow that fixed visiting order (deterministic).
#define SSG_U4_LOOP(q, n, LOAD, USE)                                            \
  {                                                                            \
    const size_t S_ = (size_t)gridDim.x * blockDim.x;                          \
    for (size_t q0_ = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q0_ < (n); \
         q0_ += 4 * S_) {                                                      \
      _Pragma("unroll") for (int u_ = 0; u_ < 4; ++u_) {                       \
        const size_t q = q0_ + u_ * S_;                                        \
        if (q < (n)) { LOAD(u_, q) }                                           \
      }                                                                        \
      _Pragma("unroll") for (int u_ = 0; u_ < 4; ++u_) {                       \
        const size_t q = q0_ + u_ * S_;                                        \
        if (q < (n)) { USE(u_, q) }                                            \
      }                                                                        \
    }                                                                          \
  }

template <typename T>
__global__ void __launch_bounds__(256, 3) k_cg_update(size_t npts,
                                                   const double* __restrict__ alpha_p,
                                                   T* __restrict__ x, const T* __restrict__ p,
                                                   T* __restrict__ r, const T* __restrict__ ap,
                                                   const T* __restrict__ dinv,
                                                   const uint8_t* __restrict__ mult,
                                                   T* __restrict__ z,
                                                   double* __restrict__ part,
                                                   const double* __restrict__ stop,
                                                   ScalarOp op) {
  if (stop && *stop != 0.0) return;
  __shared__ double sred[4 * 32];
  const double alpha = *alpha_p;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  T xv[4], pv[4], rv[4], av[4], dv[4];
  unsigned mv[4];
#define SSG_LD(u, i) xv[u] = x[i]; pv[u] = p[i]; rv[u] = r[i]; av[u] = ap[i]; \
  dv[u] = dinv[i]; mv[u] = mult[i];
#define SSG_USE(u, i)                                                         \
  {                                                                           \
    x[i] = (T)((double)xv[u] + alpha * (double)pv[u]);                        \
    const T rq = (T)((double)rv[u] + -alpha * (double)av[u]);                 \
    r[i] = rq;                                                                \
    const T zq = (T)((double)rq * (double)dv[u]);                             \
    z[i] = zq;                                                                \
    const double w = inv_count(mv[u]);                                        \
    const double rw = (double)rq * w;                                         \
    v[0] += rw * (double)zq;                                                  \
    v[1] += rw * (double)rq;                                                  \
    v[2] += w * (double)zq;                                                   \
    v[3] += rw;                                                               \
  }
  SSG_U4_LOOP(q, npts, SSG_LD, SSG_USE)
#undef SSG_LD
#undef SSG_USE
  block_reduce<4>(v, sred);
  finish<4>(v, part, op, sred);
}

// z = dinv .* r; partial w.z (Jacobi preconditioner, src/precon.c:311-324)
template <typename T>
__global__ void __launch_bounds__(256) k_jacobi(size_t npts, const T* __restrict__ r,
                                                const T* __restrict__ dinv,
                                                const uint8_t* __restrict__ mult,
                                                T* __restrict__ z, double* __restrict__ part,
                                                ScalarOp op) {
  __shared__ double sred[32];
  double v[1] = {0.0};
  T rv[4], dv[4];
  unsigned mv[4];
#define SSG_LD(u, i) rv[u] = r[i]; dv[u] = dinv[i]; mv[u] = mult[i];
#define SSG_USE(u, i)                                   \
  {                                                     \
    const T zq = (T)((double)rv[u] * (double)dv[u]);    \
    z[i] = zq;                                          \
    v[0] += (double)zq * inv_count(mv[u]);              \
  }
  SSG_U4_LOOP(q, npts, SSG_LD, SSG_USE)
#undef SSG_LD
#undef SSG_USE
  block_reduce<1>(v, sred);
  finish<1>(v, part, op, sred);
}

// partial sums of (x w) y_k, k < K (up to 10 vectors)
template <typename T, int K>
__global__ void __launch_bounds__(256) k_dots(size_t npts, const T* __restrict__ x, PtrList ys,
                                              const uint8_t* __restrict__ mult,
                                              double* __restrict__ part, ScalarOp op) {
  __shared__ double sred[K * 32];
  double v[K];
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = 0.0;
  SSG_GRID_LOOP(q, npts) {
    const double xw = (double)x[q] * inv_count(mult[q]);
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] += xw * (double)((const T*)ys.p[k])[q];
  }
  block_reduce<K>(v, sred);
  finish<K>(v, part, op, sred);
}

// partial sums of w x (the nullspace component, src/solver.c:200-213)
template <typename T>
__global__ void __launch_bounds__(256) k_wsum(size_t npts, const T* __restrict__ x,
                                              const uint8_t* __restrict__ mult,
                                              double* __restrict__ part, ScalarOp op) {
  __shared__ double sred[32];
  double v[1] = {0.0};
  T xv[4];
  unsigned mv[4];
#define SSG_LD(u, i) xv[u] = x[i]; mv[u] = mult[i];
#define SSG_USE(u, i) v[0] += (double)xv[u] * inv_count(mv[u]);
  SSG_U4_LOOP(q, npts, SSG_LD, SSG_USE)
#undef SSG_LD
#undef SSG_USE
  block_reduce<1>(v, sred);
  finish<1>(v, part, op, sred);
}

// x = x + sum_k (sign coef_k) y_k   (FCG direction, FP64)
__global__ void __launch_bounds__(256) k_combine(size_t npts, double* __restrict__ x, PtrList ys,
                                                 const double* __restrict__ coef, int K,
                                                 double sign) {
  SSG_GRID_LOOP(q, npts) {
    double v = x[q];
    for (int k = 0; k < K; ++k) v = v + (sign * coef[k]) * ((const double*)ys.p[k])[q];
    x[q] = v;
  }
}

// u += alpha p; r -= alpha ap; partial (r w).r   (src/solver.c:148-152)
__global__ void __launch_bounds__(256) k_fcg_update(size_t npts, const double* __restrict__ alpha_p,
                                                    double* __restrict__ u,
                                                    const double* __restrict__ p,
                                                    double* __restrict__ r,
                                                    const double* __restrict__ ap,
                                                    const uint8_t* __restrict__ mult,
                                                    double* __restrict__ part, ScalarOp op) {
  __shared__ double sred[32];
  const double alpha = *alpha_p;
  double v[1] = {0.0};
  double uv[4], pv[4], rv[4], av[4];
  unsigned mv[4];
#define SSG_LD(k, i) uv[k] = u[i]; pv[k] = p[i]; rv[k] = r[i]; av[k] = ap[i]; mv[k] = mult[i];
#define SSG_USE(k, i)                                  \
  {                                                    \
    u[i] = uv[k] + alpha * pv[k];                      \
    const double rq = rv[k] + -alpha * av[k];          \
    r[i] = rq;                                         \
    v[0] += (rq * inv_count(mv[k])) * rq;              \
  }
  SSG_U4_LOOP(q, npts, SSG_LD, SSG_USE)
#undef SSG_LD
#undef SSG_USE
  block_reduce<1>(v, sred);
  finish<1>(v, part, op, sred);
}

template <typename T>
__global__ void __launch_bounds__(256) k_add_const(size_t npts, T* __restrict__ x,
                                                   const double* __restrict__ a_p, int neg) {
  const double a = neg ? -*a_p : *a_p;
  SSG_GRID_LOOP(q, npts) x[q] = (T)((double)x[q] + a);
}

template <typename TI, typename TO>
__global__ void __launch_bounds__(256) k_convert(size_t npts, const TI* __restrict__ in,
                                                 TO* __restrict__ out) {
  SSG_GRID_LOOP(q, npts) out[q] = (TO)in[q];
}

template <typename T>
__global__ void __launch_bounds__(256) k_mul(size_t npts, T* __restrict__ x,
                                             const double* __restrict__ y) {
  SSG_GRID_LOOP(q, npts) x[q] = (T)((double)x[q] * y[q]);
}

// one-block reduction of partials written without a counter
__global__ void __launch_bounds__(256) k_reduce(const double* __restrict__ part, int nblk,
                                                int nq, double* __restrict__ sums,
                                                ScalarOp op) {
  if (op.stop && *op.stop != 0.0) return;
  __shared__ double sred[32];
  for (int q = 0; q < nq; ++q) {
    double v[1] = {0.0};
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) v[0] += part[(size_t)q * nblk + b];
    block_reduce<1>(v, sred);
    if (threadIdx.x == 0) sums[q] = v[0];
  }
  if (threadIdx.x == 0) apply_scalar_op(op, sums);
}

}  // namespace dev

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
using namespace dev;

static ScalarOp op_or_none(const ScalarOp* op) { return op ? *op : ScalarOp(); }

std::atomic<unsigned long long> g_launches{0};   // every launch of this library bumps it
thread_local unsigned long long t_launches = 0;
#define SSG_COUNT() count_launch()

// Launch shapes chosen by the autotuner (tune.cu); 0 = the default rule.
// Process-wide: they depend on the order and the device, not on the mesh.
std::atomic<int> g_tune_ax_epb[SSG_MAXN + 1] = {};
std::atomic<int> g_tune_dss_bps[SSG_MAXN + 1] = {};
std::atomic<int> g_tune_vec_bps{0};

int ax_epb_max(int n) {
  // elements per block: up to 256 threads, <= 96 KB of FP64 shared memory
  const int q = n + (n & 1);
  int epb = 1;
  while (epb * 2 * n * n <= 256 && (size_t)(epb * 2) * 3 * n * n * q * 8 <= 96 * 1024) epb *= 2;
  return epb;
}

// grid of the vector kernels: one point per thread up to the cap of bps
// blocks per SM (latency is hidden by resident warps); beyond it the
// kernels loop grid-stride with four points in flight per thread
int vec_blocks(size_t npts) {
  size_t b = (npts + 255) / 256;
  const size_t cap = (size_t)148 * (g_tune_vec_bps.load() > 0 ? g_tune_vec_bps.load() : kVecBpsDefault);
  return (int)(b < cap ? (b ? b : 1) : cap);
}

int ax_epb(int n) {
  if (n >= 0 && n <= SSG_MAXN && g_tune_ax_epb[n].load() != 0) return g_tune_ax_epb[n].load();
  return kAxLine;
}

template <int N, typename T, bool HELM, bool FUSEP>
static cudaError_t launch_ax_t(cudaStream_t s, int nel, int epb, T* u, T* au, const T* gf,
                               size_t npts, const double* bj, const double* D,
                               const double* S, double lambda, const PUpdate& pu,
                               const ScalarOp& dop) {
  const size_t smem = (4 * N * AxLayout<N>::P + (size_t)epb * 3 * N * N * AxLayout<N>::Q) *
                      sizeof(double);
  static SmemAttr attr;
  {
    cudaError_t e = attr.ensure((const void*)k_ax<N, T, HELM, FUSEP>, 200 * 1024);
    if (e != cudaSuccess) return e;
  }
  dim3 blk(N, N, epb);
  dim3 grd((nel + epb - 1) / epb);
  { SSG_COUNT(); k_ax<N, T, HELM, FUSEP><<<grd, blk, smem, s>>>(nel, u, au, gf, npts, bj, D, S, lambda, pu, dop); }
  return cudaGetLastError();
}

template <int N, typename T, bool HELM, bool FUSEP>
static cudaError_t launch_axl_t(cudaStream_t s, int nel, T* u, T* au, const T* gf,
                                size_t npts, const double* bj, const double* D,
                                const double* S, double lambda, const PUpdate& pu,
                                const ScalarOp& dop) {
  using L = AxLine<N>;
  constexpr size_t smem = (size_t)L::SMEM * sizeof(T);
  static SmemAttr attr;
  {
    cudaError_t e = attr.ensure((const void*)k_axl<N, T, HELM, FUSEP>, smem);
    if (e != cudaSuccess) return e;
  }
  const int grd = (nel + L::EPB - 1) / L::EPB;
  { SSG_COUNT(); k_axl<N, T, HELM, FUSEP><<<grd, L::THREADS, smem, s>>>(nel, u, au, gf, npts, bj, D, S, lambda, pu, dop); }
  return cudaGetLastError();
}

template <typename T, bool HELM, bool FUSEP>
static cudaError_t ax_dispatch(int n, cudaStream_t s, int nel, int epb, T* u, T* au,
                               const T* gf, size_t npts, const double* bj, const double* D,
                               const double* S, double lambda, const PUpdate& pu,
                               const ScalarOp& dop) {
  switch (n) {
#define SSG_AXN(NV)                                                                   \
  case NV:                                                                            \
    if (epb == kAxLine)                                                               \
      return launch_axl_t<NV, T, HELM, FUSEP>(s, nel, u, au, gf, npts, bj, D, S,      \
                                              lambda, pu, dop);                       \
    return launch_ax_t<NV, T, HELM, FUSEP>(s, nel, epb, u, au, gf, npts, bj, D, S,    \
                                           lambda, pu, dop);
    SSG_AXN(2) SSG_AXN(3) SSG_AXN(4) SSG_AXN(5) SSG_AXN(6) SSG_AXN(7)
    SSG_AXN(8) SSG_AXN(9) SSG_AXN(10) SSG_AXN(11) SSG_AXN(12)
#undef SSG_AXN
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t run_ax(cudaStream_t s, int n, int nel, int epb, bool helm, bool fp32,
                   const void* in, void* out, const void* gf, size_t npts,
                   const double* bj, const double* D, const double* S, double lambda,
                   const PUpdateArgs* pua) {
  PUpdate pu;
  const bool fuse = pua != nullptr;
  ScalarOp dop;
  if (fuse) {
    pu.z = pua->z;
    pu.beta = pua->beta;
    pu.c = pua->c;
    pu.mask = pua->mask;
    pu.stop = pua->stop;
    pu.first = pua->first;
    if (pua->dot) {
      pu.part = pua->part;
      dop = *pua->dot;
    }
  }
  // n = 8 in FP64: the FP64 tensor-core kernel (the level's FP64 metric
  // factors are stored in its fragment order); in FP32 (the mixed V-cycle,
  // whose FP32 factors are stored in natural order) the line-form kernel
  // computing in FP32
  const bool dmma = n == 8 && !fp32;
  if (dmma)
    return run_ax8_dmma(s, nel, helm, fp32, (void*)in, out, gf, npts, bj, D, S, lambda,
                        fuse ? &pu : nullptr, &dop);
  if (epb == 0) epb = ax_epb(n);
  if (fp32) {
    if (helm) return cudaErrorInvalidValue;
    if (fuse)
      return ax_dispatch<float, false, true>(n, s, nel, epb, (float*)in, (float*)out,
                                             (const float*)gf, npts, nullptr, D, D, 0.0, pu, dop);
    return ax_dispatch<float, false, false>(n, s, nel, epb, (float*)in, (float*)out,
                                            (const float*)gf, npts, nullptr, D, D, 0.0, pu, dop);
  }
  if (helm) {
    if (fuse)
      return ax_dispatch<double, true, true>(n, s, nel, epb, (double*)in, (double*)out,
                                             (const double*)gf, npts, bj, D, S, lambda, pu, dop);
    return ax_dispatch<double, true, false>(n, s, nel, epb, (double*)in, (double*)out,
                                            (const double*)gf, npts, bj, D, S, lambda, pu, dop);
  }
  if (fuse)
    return ax_dispatch<double, false, true>(n, s, nel, epb, (double*)in, (double*)out,
                                            (const double*)gf, npts, nullptr, D, D, 0.0, pu, dop);
  return ax_dispatch<double, false, false>(n, s, nel, epb, (double*)in, (double*)out,
                                           (const double*)gf, npts, nullptr, D, D, 0.0, pu, dop);
}

// one 256-thread block per 256 node tasks, capped at bps blocks per SM
// (the kernel walks the rest grid-stride)
int dss_grid(int n, int nel) {
  const size_t tasks = (size_t)nel * n * n * n;
  const size_t g = (tasks + 255) / 256;
  const int bps = (n >= 0 && n <= SSG_MAXN && g_tune_dss_bps[n].load() > 0) ? g_tune_dss_bps[n].load() : 8;
  const size_t cap = (size_t)148 * bps;
  return (int)(g < cap ? (g ? g : 1) : cap);
}

// one full wave: the kernel's resident blocks per SM (queried once per
// kernel) on every SM, each thread walking its runs grid-stride
template <typename K>
static int full_wave(K kern, std::atomic<int>& occ, size_t runs) {
  int v = occ.load(std::memory_order_relaxed);
  if (v <= 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kern, 256, 0) != cudaSuccess || v < 1)
      v = 1;
    occ.store(v, std::memory_order_relaxed);
  }
  const size_t need = (runs + 255) / 256, cap = (size_t)148 * v;
  return (int)(need < cap ? (need ? need : 1) : cap);
}

template <int N, typename T, int MODE, bool MASK>
static void launch_runs(cudaStream_t s, int nel, const T* in, T* out, const int* nb26,
                        const double* mask, const T* y, const T* y2, double* part,
                        const double* stop, const ScalarOp& op, const DssCg& cg) {
  constexpr int P = DssRun<N, T>::P;
  static std::atomic<int> occ{0};
  auto kern = &k_dss_runs<N, P, T, MODE, MASK>;
  const int grd = full_wave(kern, occ, (size_t)nel * N * N * (N / P));
  kern<<<grd, 256, 0, s>>>(nel, in, out, nb26, mask, y, y2, part, stop, op, cg);
}

template <int N, typename T, int MODE>
static void launch_dss(cudaStream_t s, int nel, const T* in, T* out, const int* nb26,
                       const int* ec_tab, const double* mask, const T* y, const T* y2,
                       double* part, const double* stop, const ScalarOp& op, const DssCg& cg) {
  SSG_COUNT();
  if (nb26) {
    if (mask)
      launch_runs<N, T, MODE, true>(s, nel, in, out, nb26, mask, y, y2, part, stop, op, cg);
    else
      launch_runs<N, T, MODE, false>(s, nel, in, out, nb26, nullptr, y, y2, part, stop, op, cg);
  } else {
    k_dss<N, T, MODE><<<dss_grid(N, nel), 256, 0, s>>>(nel, in, out, ec_tab, mask, y, y2, part,
                                                      stop, op, cg);
  }
}

template <int N, typename T>
static cudaError_t run_dss_n(cudaStream_t s, int mode, int nel, const T* in, T* out,
                             const int* nb26, const int* ec_tab, const double* mask, const T* y,
                             const T* y2, double* part, const double* stop,
                             const ScalarOp& op, const DssCg& cg) {
  switch (mode) {
#define SSG_DSSM(MV) \
  case MV: launch_dss<N, T, MV>(s, nel, in, out, nb26, ec_tab, mask, y, y2, part, stop, op, cg); break;
    SSG_DSSM(DSS_PLAIN) SSG_DSSM(DSS_DOT) SSG_DSSM(DSS_DOT2) SSG_DSSM(DSS_RESID)
    SSG_DSSM(DSS_AVG) SSG_DSSM(DSS_CGUPD)
#undef SSG_DSSM
    case DSS_SCALE:
      if constexpr (sizeof(T) == sizeof(double)) {
        launch_dss<N, T, DSS_SCALE>(s, nel, in, out, nb26, ec_tab, mask, y, y2, part, stop, op,
                                    cg);
      } else {
        return cudaErrorInvalidValue;
      }
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <typename T>
static cudaError_t run_dss_t(cudaStream_t s, int mode, int n, int nel, const T* in, T* out,
                             const int* nb26, const int* ec_tab, const double* mask,
                             const T* y, const T* y2, double* part, const double* stop,
                             const ScalarOp& op, const DssCg& cg) {
  switch (n) {
#define SSG_DSSN(NV) \
  case NV: return run_dss_n<NV, T>(s, mode, nel, in, out, nb26, ec_tab, mask, y, y2, part, stop, op, cg);
    SSG_DSSN(2) SSG_DSSN(3) SSG_DSSN(4) SSG_DSSN(5) SSG_DSSN(6) SSG_DSSN(7)
    SSG_DSSN(8) SSG_DSSN(9) SSG_DSSN(10) SSG_DSSN(11) SSG_DSSN(12)
#undef SSG_DSSN
    default: return cudaErrorInvalidValue;
  }
}

// the line-run kernels load and store runs of a line as 8- or 16-byte
// vectors when n is even: every array must then start on a 16-byte boundary
// (the library's own vectors always do; a caller's pointer may not)
static bool lines_aligned(int n, std::initializer_list<const void*> ptrs) {
  if (n % 2) return true;
  for (const void* p : ptrs)
    if (reinterpret_cast<uintptr_t>(p) % 16u) return false;
  return true;
}

cudaError_t run_dss(cudaStream_t s, int mode, bool fp32, int n, int nel, const void* in,
                    void* out, const int* nb26, const int* ec_tab, const double* mask,
                    const void* y, const void* y2, double* part, const double* stop,
                    const ScalarOp* op, const DssCg* cg) {
  const ScalarOp o = op_or_none(op);
  const DssCg g = cg ? *cg : DssCg();
  if ((!ec_tab && !nb26) || (mode == DSS_CGUPD && !cg)) return cudaErrorInvalidValue;
  if (nb26 && !lines_aligned(n, {in, out, mask, y, y2, g.x, g.p, g.r, g.dinv, g.z})) {
    if (!ec_tab) return cudaErrorMisalignedAddress;
    nb26 = nullptr;
  }
  if (fp32)
    return run_dss_t<float>(s, mode, n, nel, (const float*)in, (float*)out, nb26, ec_tab,
                            mask, (const float*)y, (const float*)y2, part, stop, o, g);
  return run_dss_t<double>(s, mode, n, nel, (const double*)in, (double*)out, nb26, ec_tab,
                           mask, (const double*)y, (const double*)y2, part, stop, o, g);
}

template <int N>
static cudaError_t run_dss3_n(cudaStream_t s, bool scale, int nel, const double* in,
                              double* out, size_t stride, const int* nb26, const int* ec_tab,
                              const double* y) {
  SSG_COUNT();
  if (nb26) {
    constexpr int P = DssRun<N, double>::P;
    static std::atomic<int> occ_s{0}, occ_p{0};
    const size_t runs = (size_t)nel * N * N * (N / P);
    if (scale) {
      auto kern = &k_dss3_runs<N, P, true>;
      kern<<<full_wave(kern, occ_s, runs), 256, 0, s>>>(nel, in, out, stride, nb26, y);
    } else {
      auto kern = &k_dss3_runs<N, P, false>;
      kern<<<full_wave(kern, occ_p, runs), 256, 0, s>>>(nel, in, out, stride, nb26, y);
    }
    return cudaGetLastError();
  }
  const int grd = dss_grid(N, nel);
  if (scale)
    k_dss3<N, true><<<grd, 256, 0, s>>>(nel, in, out, stride, ec_tab, y);
  else
    k_dss3<N, false><<<grd, 256, 0, s>>>(nel, in, out, stride, ec_tab, y);
  return cudaGetLastError();
}

cudaError_t run_dss3(cudaStream_t s, bool scale, int n, int nel, const double* in, double* out,
                     size_t stride, const int* nb26, const int* ec_tab, const double* y) {
  if ((!ec_tab && !nb26) || (scale && !y)) return cudaErrorInvalidValue;
  if (nb26 &&
      (!lines_aligned(n, {in, out, y}) || (n % 2 == 0 && (stride * sizeof(double)) % 16u))) {
    if (!ec_tab) return cudaErrorMisalignedAddress;
    nb26 = nullptr;
  }
  switch (n) {
#define SSG_DSS3N(NV) \
  case NV: return run_dss3_n<NV>(s, scale, nel, in, out, stride, nb26, ec_tab, y);
    SSG_DSS3N(2) SSG_DSS3N(3) SSG_DSS3N(4) SSG_DSS3N(5) SSG_DSS3N(6) SSG_DSS3N(7)
    SSG_DSS3N(8) SSG_DSS3N(9) SSG_DSS3N(10) SSG_DSS3N(11) SSG_DSS3N(12)
#undef SSG_DSS3N
    default: return cudaErrorInvalidValue;
  }
}

template <typename T, bool ADD>
static cudaError_t launch_tensor3(cudaStream_t s, int nel, int ni, int no, const double* A,
                                  const T* in, T* out) {
  // elements per block: their stages within 40 KB of shared memory, <= 8
  const size_t per = (size_t)ni * ni * ni + (size_t)no * ni * ni + (size_t)no * no * ni;
  int epb = (int)((40 * 1024 / sizeof(double) - (size_t)no * ni) / per);
  epb = epb < 1 ? 1 : (epb > 8 ? 8 : epb);
  const size_t smem = ((size_t)no * ni + epb * per) * sizeof(double);
  const int grid = (nel + epb - 1) / epb;
  if (grid < 1) return cudaSuccess;
  auto kern = &dev::k_tensor3<T, ADD, 0, 0>;
  // the transfers between consecutive multigrid orders (n, (n - 1)/2 + 1)
#define SSG_T3(A_, B_)                                                         \
  if (ni == A_ && no == B_) kern = &dev::k_tensor3<T, ADD, A_, B_>;            \
  if (ni == B_ && no == A_) kern = &dev::k_tensor3<T, ADD, B_, A_>;
  SSG_T3(12, 6) SSG_T3(11, 6) SSG_T3(10, 5) SSG_T3(9, 5) SSG_T3(8, 4)
  SSG_T3(7, 4) SSG_T3(6, 3) SSG_T3(5, 3) SSG_T3(4, 2) SSG_T3(3, 2)
#undef SSG_T3
  SSG_COUNT();
  kern<<<grid, 256, smem, s>>>(nel, ni, no, epb, A, in, out);
  return cudaGetLastError();
}

cudaError_t run_tensor3(cudaStream_t s, bool fp32, bool add, int nel, int ni, int no,
                        const double* A, const void* in, void* out) {
  if (fp32)
    return add ? launch_tensor3<float, true>(s, nel, ni, no, A, (const float*)in, (float*)out)
               : launch_tensor3<float, false>(s, nel, ni, no, A, (const float*)in,
                                              (float*)out);
  return add ? launch_tensor3<double, true>(s, nel, ni, no, A, (const double*)in, (double*)out)
             : launch_tensor3<double, false>(s, nel, ni, no, A, (const double*)in,
                                             (double*)out);
}

cudaError_t run_helm_diag(cudaStream_t s, size_t npts, size_t nt, const double* kd,
                          const double* rho, const double* det, double lam, double* out) {
  SSG_COUNT();
  k_helm_diag<<<vec_blocks(npts), 256, 0, s>>>(npts, nt, kd, rho, det, lam, out);
  return cudaGetLastError();
}

cudaError_t run_recip(cudaStream_t s, size_t npts, double* x) {
  SSG_COUNT();
  k_recip<<<vec_blocks(npts), 256, 0, s>>>(npts, x);
  return cudaGetLastError();
}

cudaError_t run_cg_update(cudaStream_t s, bool fp32, size_t npts, const double* alpha,
                          void* x, const void* p, void* r, const void* ap, const void* dinv,
                          const uint8_t* mult, void* z, double* part, int nblk,
                          const double* stop, const ScalarOp* op) {
  const ScalarOp o = op_or_none(op);
  if (fp32)
    { SSG_COUNT(); k_cg_update<float><<<nblk, 256, 0, s>>>(npts, alpha, (float*)x, (const float*)p, (float*)r,
                                            (const float*)ap, (const float*)dinv, mult,
                                            (float*)z, part, stop, o); }
  else
    { SSG_COUNT(); k_cg_update<double><<<nblk, 256, 0, s>>>(npts, alpha, (double*)x, (const double*)p,
                                             (double*)r, (const double*)ap,
                                             (const double*)dinv, mult, (double*)z, part, stop, o); }
  return cudaGetLastError();
}

cudaError_t run_jacobi(cudaStream_t s, bool fp32, size_t npts, const void* r, const void* dinv,
                       const uint8_t* mult, void* z, double* part, int nblk,
                       const ScalarOp* op) {
  const ScalarOp o = op_or_none(op);
  if (fp32)
    { SSG_COUNT(); k_jacobi<float><<<nblk, 256, 0, s>>>(npts, (const float*)r, (const float*)dinv, mult,
                                         (float*)z, part, o); }
  else
    { SSG_COUNT(); k_jacobi<double><<<nblk, 256, 0, s>>>(npts, (const double*)r, (const double*)dinv, mult,
                                          (double*)z, part, o); }
  return cudaGetLastError();
}

template <typename T>
static cudaError_t run_dots_t(cudaStream_t s, size_t npts, const T* x, const PtrList& ys, int K,
                              const uint8_t* mult, double* part, int nblk, const ScalarOp& o) {
  switch (K) {
#define SSG_DOTK(KV)                                                   \
  case KV:                                                             \
    SSG_COUNT();                                                       \
    k_dots<T, KV><<<nblk, 256, 0, s>>>(npts, x, ys, mult, part, o);    \
    break;
    SSG_DOTK(1) SSG_DOTK(2) SSG_DOTK(3) SSG_DOTK(4) SSG_DOTK(5)
    SSG_DOTK(6) SSG_DOTK(7) SSG_DOTK(8) SSG_DOTK(9) SSG_DOTK(10)
#undef SSG_DOTK
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t run_dots(cudaStream_t s, bool fp32, size_t npts, const void* x, const PtrList& ys,
                     int K, const uint8_t* mult, double* part, int nblk, const ScalarOp* op) {
  const ScalarOp o = op_or_none(op);
  if (fp32) return run_dots_t<float>(s, npts, (const float*)x, ys, K, mult, part, nblk, o);
  return run_dots_t<double>(s, npts, (const double*)x, ys, K, mult, part, nblk, o);
}

cudaError_t run_wsum(cudaStream_t s, bool fp32, size_t npts, const void* x,
                     const uint8_t* mult, double* part, int nblk, const ScalarOp* op) {
  const ScalarOp o = op_or_none(op);
  if (fp32)
    { SSG_COUNT(); k_wsum<float><<<nblk, 256, 0, s>>>(npts, (const float*)x, mult, part, o); }
  else
    { SSG_COUNT(); k_wsum<double><<<nblk, 256, 0, s>>>(npts, (const double*)x, mult, part, o); }
  return cudaGetLastError();
}

cudaError_t run_combine(cudaStream_t s, size_t npts, double* x, const PtrList& ys,
                        const double* coef, int K, double sign) {
  { SSG_COUNT(); k_combine<<<vec_blocks(npts), 256, 0, s>>>(npts, x, ys, coef, K, sign); }
  return cudaGetLastError();
}

cudaError_t run_fcg_update(cudaStream_t s, size_t npts, const double* alpha, double* u,
                           const double* p, double* r, const double* ap, const uint8_t* mult,
                           double* part, int nblk, const ScalarOp* op) {
  const ScalarOp o = op_or_none(op);
  { SSG_COUNT(); k_fcg_update<<<nblk, 256, 0, s>>>(npts, alpha, u, p, r, ap, mult, part, o); }
  return cudaGetLastError();
}

cudaError_t run_add_const(cudaStream_t s, bool fp32, size_t npts, void* x, const double* a,
                          int neg) {
  if (fp32)
    { SSG_COUNT(); k_add_const<float><<<vec_blocks(npts), 256, 0, s>>>(npts, (float*)x, a, neg); }
  else
    { SSG_COUNT(); k_add_const<double><<<vec_blocks(npts), 256, 0, s>>>(npts, (double*)x, a, neg); }
  return cudaGetLastError();
}

cudaError_t run_convert(cudaStream_t s, size_t npts, const void* in, bool in32, void* out,
                        bool out32) {
  const int nb = vec_blocks(npts);
  if (in32 && !out32)
    { SSG_COUNT(); k_convert<float, double><<<nb, 256, 0, s>>>(npts, (const float*)in, (double*)out); }
  else if (!in32 && out32)
    { SSG_COUNT(); k_convert<double, float><<<nb, 256, 0, s>>>(npts, (const double*)in, (float*)out); }
  else if (in32)
    { SSG_COUNT(); k_convert<float, float><<<nb, 256, 0, s>>>(npts, (const float*)in, (float*)out); }
  else
    { SSG_COUNT(); k_convert<double, double><<<nb, 256, 0, s>>>(npts, (const double*)in, (double*)out); }
  return cudaGetLastError();
}

cudaError_t run_mul(cudaStream_t s, bool fp32, size_t npts, void* x, const double* y) {
  if (fp32)
    { SSG_COUNT(); k_mul<float><<<vec_blocks(npts), 256, 0, s>>>(npts, (float*)x, y); }
  else
    { SSG_COUNT(); k_mul<double><<<vec_blocks(npts), 256, 0, s>>>(npts, (double*)x, y); }
  return cudaGetLastError();
}

cudaError_t run_reduce(cudaStream_t s, const double* part, int nblk, int nq, double* sums,
                       const ScalarOp& op) {
  { SSG_COUNT(); k_reduce<<<1, 256, 0, s>>>(part, nblk, nq, sums, op); }
  return cudaGetLastError();
}

}  // namespace ssg

extern "C" unsigned long long ssg_kernel_launch_count(void) { return ssg::g_launches.load(); }
