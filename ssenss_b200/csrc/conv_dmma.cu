// Dealiased skew-symmetric convection at n = 8, m = 12 on the FP64 tensor
// cores, both forms the time step calls: the velocity advecting itself (the
// per-element history term, convection_operator(sel, u, u, conv),
// src/navier_stokes.c:79-83: one call per step) and a field advected by
// another (the RK4 stages of the convection sub-steps,
// convection_operator(sel, utmp, y, f), src/time.c:114-116: 24 calls per
// step).
//
// Same arithmetic as k_convection (convection.cu): interpolate the fields
// to the m-point grid (src/interpolation.c:136-155), per reference
// direction b add A_b d_b v_c + B_b d_b(u_b v_c) with
// A_b = sum_a u_a W[a][b], B_b = sum_a W[a][b] (src/convection.c:71-140
// regrouped), project back with (J^T)^3 (src/interpolation.c:157-176).
// Every contraction is a small GEMM
//     Out[row][o] = sum_l F(row, l) M[o][l]
// over the rows of an element's lines (64 to 144 of them), with M one of J
// (12 x 8), D (12 x 12) or J^T (8 x 12); each warp takes 8-row tiles and
// runs them as mma.sync.m8n8k4.f64, with the lane's B fragments of the
// stage's matrix in registers (read per stage from a lane-ordered table in
// shared memory that each block fills once).
//
//   self (u == v):  three fields interpolated instead of six; one pass per
//                   direction forms all three components' derivatives from
//                   the same loads and reads the weights W once.
//   general:        u and v interpolated (six fields), then the same
//                   passes over all three advected components.
//
// Fragment layouts (lane = 4g + t): A (8x4) a = A[g][t]; B (4x8) b = B[t][g];
// C (8x8) c0 = C[g][2t], c1 = C[g][2t+1].  Output columns o >= 12 of the
// second column tile have zero B and are dropped.
//
// One element per block at a time.  Shared memory: m-grid fields [k][j][i]
// with rows of 12 and planes of 148 doubles (= 4 mod 16), which makes every
// A-fragment load conflict-free except the j-direction tiles that straddle
// two planes.
//   self:     U (3 fields), SK (3)        88.5 KB, 12 warps, two blocks per SM
//   general:  U (3), V (3), SK (3)       131.2 KB, 24 warps, one block per SM
// The interpolation and projection stages use the regions not live at the
// time.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"
#include "ssg_internal.h"
#include "ssg_kernels.h"

namespace ssg {
namespace dev {

namespace cdm {
constexpr int N = 8, M = 12;
constexpr int NT = N * N * N, MT = M * M * M;
// self-convection: twelve warps, two blocks per SM; the general form:
// twenty-four warps, one block per SM (its three advected fields take the
// shared memory of two)
constexpr int WARPS = 12, THREADS = 32 * WARPS, THREADS_UV = 2 * THREADS;
// U / V / SK fields: [k][j][i]
constexpr int RU = M, PU = M * M + 4, FU = M * PU;
// T1 (interpolation x out): [k < 8][j < 8][o < 12]
constexpr int PT1 = N * M + 4, FT1 = N * PT1;
// T2 (interpolation y out): [k < 8][o2][o1]
constexpr int PT2 = PU, FT2 = N * PT2;
// P1 (projection i out): [k < 12][j < 12][p < 8]
constexpr int RP1 = N, PP1 = M * N, FP1 = M * PP1;
// P2 (projection j out): [k < 12][p2 < 8][p1 < 8]
constexpr int PP2 = N * N + 8, FP2 = M * PP2;
// lane-ordered B fragments: J (2 column tiles x 2 k-steps), D (2 x 3),
// J^T (3 k-steps), each [.][lane]
constexpr int FJ = 0, FD = FJ + 4 * 32, FPJ = FD + 6 * 32, FRAGS = FPJ + 3 * 32;
constexpr size_t SMEM_SELF = (6 * (size_t)FU + FRAGS) * sizeof(double);
constexpr size_t SMEM_GEN = (9 * (size_t)FU + FRAGS) * sizeof(double);
// scratch of three fields' stages in three field regions (self: T1, P1 in
// U; T2, P2 in SK; general: T1 in the field being made, T2 in V or SK, P1
// in U, P2 in V)
static_assert(3 * FT1 <= 3 * FU && 3 * FT2 <= 3 * FU && 3 * FP1 <= 3 * FU &&
                  3 * FP2 <= 3 * FU,
              "three fields' stage scratch fits");
static_assert(FU % 2 == 0 && PU % 2 == 0 && FT1 % 2 == 0 && FP1 % 2 == 0,
              "16-byte stores land on 16-byte boundaries");
}  // namespace cdm

struct ConvDmmaMats {
  double D[cdm::M * cdm::M];   // D[o * M + l]
  double J[cdm::M * cdm::N];   // J[o * N + p]
};

namespace cdm {

// B fragments b = Mx[8 ct + g][4 s + t] (zero past the matrix) into the
// block's table: a warp's fragment is then one conflict-free shared load
// instead of a constant load whose 32 lanes want 32 different addresses
__device__ __forceinline__ void load_fragments(const ConvDmmaMats& mt, double* FR) {
  for (int q = threadIdx.x; q < FRAGS; q += blockDim.x) {
    const int l = q & 31, gg = l >> 2, tt = l & 3, f = q >> 5;
    double v;
    if (f < 4) {                       // J: f = 2 ct + s
      const int o = 8 * (f >> 1) + gg;
      v = o < M ? mt.J[o * N + 4 * (f & 1) + tt] : 0.0;
    } else if (f < 10) {               // D: f - 4 = 3 ct + s
      const int o = 8 * ((f - 4) / 3) + gg;
      v = o < M ? mt.D[o * M + 4 * ((f - 4) % 3) + tt] : 0.0;
    } else {                           // J^T: f - 10 = s
      v = mt.J[(4 * (f - 10) + tt) * N + gg];
    }
    FR[q] = v;
  }
}

// interpolation x of nf fields (field f at src + f * fstride, n^3 in
// global): T1[f][k][j][o] = sum_p u[k][j][p] J[o][p]; nf x 8 tiles
__device__ __forceinline__ void interp_x(int nf, const double* __restrict__ src0, size_t fstride,
                                         double* T1, const double* FR) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const int nw = blockDim.x >> 5;
  double bJ[2][2];
#pragma unroll
  for (int ct = 0; ct < 2; ++ct)
#pragma unroll
    for (int s = 0; s < 2; ++s) bJ[ct][s] = FR[FJ + (2 * ct + s) * 32 + lane];
  for (int job = warp; job < nf * N; job += nw) {
    const int f = job / N, k = job % N;
    const double* src = src0 + f * fstride + k * N * N + g * N;
    double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const double a = src[4 * s + t];
#pragma unroll
      for (int ct = 0; ct < 2; ++ct) dmma(acc[ct][0], acc[ct][1], a, bJ[ct][s], acc[ct][0], acc[ct][1]);
    }
    double* dst = T1 + f * FT1 + k * PT1 + g * M + 2 * t;
    *reinterpret_cast<double2*>(dst) = make_double2(acc[0][0], acc[0][1]);
    if (t < 2) *reinterpret_cast<double2*>(dst + 8) = make_double2(acc[1][0], acc[1][1]);
  }
}

// interpolation y: T2[f][k][o2][o1] = sum_p T1[k][p][o1] J[o2][p];
// rows (k, o1), nf x 12 tiles
__device__ __forceinline__ void interp_y(int nf, const double* T1, double* T2, const double* FR) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const int nw = blockDim.x >> 5;
  double bJ[2][2];
#pragma unroll
  for (int ct = 0; ct < 2; ++ct)
#pragma unroll
    for (int s = 0; s < 2; ++s) bJ[ct][s] = FR[FJ + (2 * ct + s) * 32 + lane];
  for (int job = warp; job < nf * 12; job += nw) {
    const int f = job / 12, r = 8 * (job % 12) + g;
    const int k = r / M, o1 = r % M;
    const double* src = T1 + f * FT1 + k * PT1 + o1;
    double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const double a = src[(4 * s + t) * M];
#pragma unroll
      for (int ct = 0; ct < 2; ++ct) dmma(acc[ct][0], acc[ct][1], a, bJ[ct][s], acc[ct][0], acc[ct][1]);
    }
    double* dst = T2 + f * FT2 + k * PT2 + o1;
#pragma unroll
    for (int ct = 0; ct < 2; ++ct)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int o2 = 8 * ct + 2 * t + h;
        if (o2 < M) dst[o2 * M] = acc[ct][h];
      }
  }
}

// interpolation z: F[f][o3][o2][o1] = sum_p T2[p][o2][o1] J[o3][p] (fields
// FU apart); rows (o2, o1), nf x 18 tiles
__device__ __forceinline__ void interp_z(int nf, const double* T2, double* F, const double* FR) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const int nw = blockDim.x >> 5;
  double bJ[2][2];
#pragma unroll
  for (int ct = 0; ct < 2; ++ct)
#pragma unroll
    for (int s = 0; s < 2; ++s) bJ[ct][s] = FR[FJ + (2 * ct + s) * 32 + lane];
  for (int job = warp; job < nf * 18; job += nw) {
    const int f = job / 18, r = 8 * (job % 18) + g;
    const double* src = T2 + f * FT2 + r;
    double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const double a = src[(4 * s + t) * PT2];
#pragma unroll
      for (int ct = 0; ct < 2; ++ct) dmma(acc[ct][0], acc[ct][1], a, bJ[ct][s], acc[ct][0], acc[ct][1]);
    }
    // rows of 12 are contiguous within a plane: (o3, o2, o1) -> o3 PU + r
    double* dst = F + f * FU + r;
#pragma unroll
    for (int ct = 0; ct < 2; ++ct)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int o3 = 8 * ct + 2 * t + h;
        if (o3 < M) dst[o3 * PU] = acc[ct][h];
      }
  }
}

// nf fields interpolated from global (field f at src + f * fstride) into F
// (fields FU apart), stages in T1 and T2 (barriers included)
__device__ __forceinline__ void interpolate(int nf, const double* __restrict__ src,
                                            size_t fstride, double* T1, double* T2, double* F,
                                            const double* FR) {
  interp_x(nf, src, fstride, T1, FR);
  __syncthreads();
  interp_y(nf, T1, T2, FR);
  __syncthreads();
  interp_z(nf, T2, F, FR);
  __syncthreads();
}

// weak projection of nc fields of SK (FU apart) to out (field c at
// out + c * fstride, n^3 in global), stages in P1 and P2 (barriers between
// the stages; none after the last, which writes global memory only)
__device__ __forceinline__ void project(int nc, const double* SK, double* P1, double* P2,
                                        double* __restrict__ out, size_t fstride,
                                        const double* FR) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const int nw = blockDim.x >> 5;
  double bP[3];   // J^T[g][4 s + t]
#pragma unroll
  for (int s = 0; s < 3; ++s) bP[s] = FR[FPJ + s * 32 + lane];
  // i: P1[c][k][j][p] = sum_o SK[k][j][o] J[o][p]; nc x 18 tiles
  for (int job = warp; job < nc * 18; job += nw) {
    const int c = job / 18, r = 8 * (job % 18) + g;
    const double* src = SK + c * FU + (r / M) * PU + (r % M) * RU;
    double acc0 = 0.0, acc1 = 0.0;
#pragma unroll
    for (int s = 0; s < 3; ++s) dmma(acc0, acc1, src[4 * s + t], bP[s], acc0, acc1);
    *reinterpret_cast<double2*>(P1 + c * FP1 + (r / M) * PP1 + (r % M) * RP1 + 2 * t) =
        make_double2(acc0, acc1);
  }
  __syncthreads();
  // j: P2[c][k][p2][p1] = sum_o P1[k][o][p1] J[o][p2]; rows (k, p1), nc x 12
  for (int job = warp; job < nc * 12; job += nw) {
    const int c = job / 12, k = job % 12;
    const double* src = P1 + c * FP1 + k * PP1 + g;
    double acc0 = 0.0, acc1 = 0.0;
#pragma unroll
    for (int s = 0; s < 3; ++s) dmma(acc0, acc1, src[(4 * s + t) * RP1], bP[s], acc0, acc1);
    double* dst = P2 + c * FP2 + k * PP2 + g;
    dst[(2 * t) * N] = acc0;
    dst[(2 * t + 1) * N] = acc1;
  }
  __syncthreads();
  // k: out[c][p3][p2][p1] = sum_o P2[o][p2][p1] J[o][p3]; rows (p2, p1), nc x 8
  for (int job = warp; job < nc * N; job += nw) {
    const int c = job / N, p2 = job % N;
    const double* src = P2 + c * FP2 + p2 * N + g;
    double acc0 = 0.0, acc1 = 0.0;
#pragma unroll
    for (int s = 0; s < 3; ++s) dmma(acc0, acc1, src[(4 * s + t) * PP2], bP[s], acc0, acc1);
    double* dst = out + c * fstride + p2 * N + g;
    dst[(2 * t) * N * N] = acc0;
    dst[(2 * t + 1) * N * N] = acc1;
  }
}

// The three direction passes (barriers included): for each direction b and
// each advected component c < NC,
//   SK_c (=, +=) A_b d_b v_c + B_b d_b(u_b v_c)
// with U the advecting field's three components and V the advected
// components (V == U for self-convection, NC = 3; one component, NC = 1,
// for the general form).  A job is one row tile and one column tile
// (o < 8 or 8 <= o < 12).
template <int NC>
__device__ __forceinline__ void direction_passes(const double* U, const double* V, double* SK,
                                                 const double* __restrict__ Wb, size_t wstride,
                                                 const double* FR) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const int nw = blockDim.x >> 5;
#pragma unroll 1
  for (int b = 0; b < 3; ++b) {
    for (int job = warp; job < 36; job += nw) {
      const int r = 8 * (job >> 1) + g, ct = job & 1;
      double bD[3];
#pragma unroll
      for (int s = 0; s < 3; ++s) bD[s] = FR[FD + (3 * ct + s) * 32 + lane];
      // shared base and step of this lane's line; unpadded point index base
      int sb, ss, gb, gs;
      if (b == 0) {
        sb = (r / M) * PU + (r % M) * RU; ss = 1;
        gb = r * M; gs = 1;
      } else if (b == 1) {
        sb = (r / M) * PU + (r % M); ss = RU;
        gb = (r / M) * M * M + (r % M); gs = M;
      } else {
        sb = r; ss = PU;
        gb = r; gs = M * M;
      }
      // the lane's output points o0 = 8 ct + 2 t and o0 + 1 (both below 12
      // or neither): A_b and B_b there first, so that the weights' loads
      // overlap the tensor-core work.  Along i (b = 0) the two points are
      // adjacent: one 16-byte access each.
      const int o0 = 8 * ct + 2 * t;
      const bool out = o0 < M;
      double fa[2] = {0.0, 0.0}, fb[2] = {0.0, 0.0};
      if (out) {
        const double* wp = Wb + 3 * b * wstride + gb + o0 * gs;
        double w[3][2], ua[3][2];
        if (b == 0) {
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            const double2 wv = __ldg(reinterpret_cast<const double2*>(wp + a * wstride));
            const double2 uv = *reinterpret_cast<const double2*>(U + a * FU + sb + o0);
            w[a][0] = wv.x; w[a][1] = wv.y;
            ua[a][0] = uv.x; ua[a][1] = uv.y;
          }
        } else {
#pragma unroll
          for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              w[a][h] = __ldg(wp + a * wstride + h * gs);
              ua[a][h] = U[a * FU + sb + (o0 + h) * ss];
            }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          double A = w[0][h] * ua[0][h];
          A = fma(w[1][h], ua[1][h], A);
          A = fma(w[2][h], ua[2][h], A);
          fa[h] = A;
          fb[h] = (w[0][h] + w[1][h]) + w[2][h];
        }
      }
      double dv[NC][2], dp[NC][2];
#pragma unroll
      for (int c = 0; c < NC; ++c) dv[c][0] = dv[c][1] = dp[c][0] = dp[c][1] = 0.0;
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const int q = sb + (4 * s + t) * ss;
        const double ab = U[b * FU + q];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const double av = V[c * FU + q];
          dmma(dv[c][0], dv[c][1], av, bD[s], dv[c][0], dv[c][1]);
          dmma(dp[c][0], dp[c][1], ab * av, bD[s], dp[c][0], dp[c][1]);
        }
      }
      if (out) {
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          double s0 = fa[0] * dv[c][0];
          s0 = fma(fb[0], dp[c][0], s0);
          double s1 = fa[1] * dv[c][1];
          s1 = fma(fb[1], dp[c][1], s1);
          if (b == 0) {
            *reinterpret_cast<double2*>(SK + c * FU + sb + o0) = make_double2(s0, s1);
          } else {
            double* p = SK + c * FU + sb + o0 * ss;
            p[0] += s0;
            p[ss] += s1;
          }
        }
      }
    }
    __syncthreads();
  }
}

// the next element's fields and weights into L2 while this one computes:
// lanes of warp 0 issue one bulk prefetch each (the three components of f0,
// and of f1 when given, NT values each, `fstride` apart; the nine weight
// arrays of MT values `wstride` apart); skipped for any address not on a
// 16-byte boundary (a prefetch is only a hint)
__device__ __forceinline__ void prefetch_element(int en, int nel, int e0, const double* f0,
                                                 const double* f1, size_t fstride,
                                                 const double* W, size_t wstride) {
  if (threadIdx.x >= 32 || en >= nel) return;
  const int lane = threadIdx.x;
  const double* p = nullptr;
  unsigned bytes = 0;
  const int nf = f1 ? 6 : 3;
  if (lane < nf) {
    p = (lane < 3 ? f0 : f1) + (size_t)en * NT + (size_t)(lane % 3) * fstride;
    bytes = NT * sizeof(double);
  } else if (lane < nf + 9) {
    p = W + (size_t)(e0 + en) * MT + (size_t)(lane - nf) * wstride;
    bytes = MT * sizeof(double);
  }
  if (p && (reinterpret_cast<uintptr_t>(p) & 15u) == 0) bulk_prefetch_l2(p, bytes);
}

}  // namespace cdm

// u advecting itself: U (3 fields), SK (3 fields)
__global__ void __launch_bounds__(cdm::THREADS, 2)
    k_convection_dmma(int nel, int e0, int nel_fac, const double* __restrict__ u,
                      double* __restrict__ udv, const double* __restrict__ W,
                      const __grid_constant__ ConvDmmaMats mt) {
  using namespace cdm;
  extern __shared__ __align__(16) double smem[];
  double* const U = smem;
  double* const SK = smem + 3 * FU;
  double* const FR = smem + 6 * FU;
  load_fragments(mt, FR);
  __syncthreads();
  const size_t nptsn = (size_t)nel * NT, wstride = (size_t)nel_fac * MT;
  for (int e = blockIdx.x; e < nel; e += gridDim.x) {
    const double* Wb = W + (size_t)(e0 + e) * MT;
    prefetch_element(e + gridDim.x, nel, e0, u, nullptr, nptsn, W, wstride);
    // T1 in U, T2 in SK
    interpolate(3, u + (size_t)e * NT, nptsn, U, SK, U, FR);
    direction_passes<3>(U, U, SK, Wb, wstride, FR);
    // P1 in U, P2 in SK; the next element's interpolation x writes U only
    // (P1 was last read before a barrier) and its stage y writes SK after
    // the barrier that follows
    project(3, SK, U, SK, udv + (size_t)e * NT, nptsn, FR);
  }
}

// v advected by u: U (3 fields), V (3), SK (3)
__global__ void __launch_bounds__(cdm::THREADS_UV, 1)
    k_convection_dmma_uv(int nel, int e0, int nel_fac, const double* __restrict__ u,
                         const double* __restrict__ v, double* __restrict__ udv,
                         const double* __restrict__ W, const __grid_constant__ ConvDmmaMats mt) {
  using namespace cdm;
  extern __shared__ __align__(16) double smem[];
  double* const U = smem;
  double* const V = smem + 3 * FU;
  double* const SK = V + 3 * FU;
  double* const FR = SK + 3 * FU;
  load_fragments(mt, FR);
  __syncthreads();
  const size_t nptsn = (size_t)nel * NT, wstride = (size_t)nel_fac * MT;
  for (int e = blockIdx.x; e < nel; e += gridDim.x) {
    const double* Wb = W + (size_t)(e0 + e) * MT;
    prefetch_element(e + gridDim.x, nel, e0, u, v, nptsn, W, wstride);
    // u: T1 in U, T2 in V; v: T1 in V, T2 in SK
    interpolate(3, u + (size_t)e * NT, nptsn, U, V, U, FR);
    interpolate(3, v + (size_t)e * NT, nptsn, V, SK, V, FR);
    direction_passes<3>(U, V, SK, Wb, wstride, FR);
    // P1 in U, P2 in V; the next element's interpolation x writes U only
    // (P1 was last read before a barrier) and its stage y writes V after
    // the barrier that follows
    project(3, SK, U, V, udv + (size_t)e * NT, nptsn, FR);
  }
}

}  // namespace dev

bool convection_dmma_applies(int n, int m) { return n == dev::cdm::N && m == dev::cdm::M; }

cudaError_t run_convection_dmma(cudaStream_t s, int nel, int e0, int nel_fac, const double* u,
                                const double* v, double* udv, const double* W,
                                const double* Dh, const double* Jh) {
  using namespace dev::cdm;
  if (nel <= 0) return cudaSuccess;
  dev::ConvDmmaMats mt;
  for (int q = 0; q < M * M; ++q) mt.D[q] = Dh[q];
  for (int q = 0; q < M * N; ++q) mt.J[q] = Jh[q];
  int dev = 0, sms = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return err;
  static SmemAttr attr_self, attr_uv;
  const bool self = u == v;
  err = self ? attr_self.ensure((const void*)dev::k_convection_dmma, SMEM_SELF)
             : attr_uv.ensure((const void*)dev::k_convection_dmma_uv, SMEM_GEN);
  if (err != cudaSuccess) return err;
  err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (err != cudaSuccess) return err;
  count_launch();
  if (self) {
    const int grid = nel < 2 * sms ? nel : 2 * sms;
    dev::k_convection_dmma<<<grid, THREADS, SMEM_SELF, s>>>(nel, e0, nel_fac, u, udv, W, mt);
  } else {
    const int grid = nel < sms ? nel : sms;
    dev::k_convection_dmma_uv<<<grid, THREADS_UV, SMEM_GEN, s>>>(nel, e0, nel_fac, u, v, udv,
                                                                 W, mt);
  }
  return cudaGetLastError();
}

}  // namespace ssg
