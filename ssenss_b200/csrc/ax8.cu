// Element operator for n = 8 (N = 7) on the FP64 tensor cores.
//
// Same operator as k_ax (discrete_laplace_operator, src/poisson.c:34-56, or
// discrete_helmholtz_operator, src/helmholtz.c:33-49): A_e u = D^T(G rho J D u)
// per element, with the SVV matrix S in place of D for the Helmholtz
// r-derivative and the transposed s/t-derivatives.  One warp per element;
// the 8 x 8 contractions of the r- and s-directions are
// mma.sync.m8n8k4.f64 (tcgen05 has no FP64 kind; DMMA is the FP64 tensor
// path of sm_100a), the t-direction is plain FP64 FMAs in registers.
//
// Fragment layouts of m8n8k4 (lane = 4g + t, g < 8, t < 4):
//   A (8x4, row):  a = A[g][t]          B (4x8, col):  b = B[t][g]
//   C (8x8):       c0 = C[g][2t], c1 = C[g][2t+1]
// Every lane owns the 16 points (i = g, j = 2t + s, k = 0..7), s = 0, 1.
//   forward r:  C_k[i][j] = sum_l D[i][l] u[k][j][l]   A = D,  B = u (L1 loads)
//   forward s:  C_k[i][j] = sum_l u[k][l][i] D[j][l]   A = u (L1 loads), B = D^T
//   forward t:  sum_l D[k][l] u[l][j][i]                registers
//   backward r: C_k[i][j] = sum_l D[l][i] w0[k][j][l]  A = D^T, B = w0 (shuffles)
//   backward s: C_k[i][j] = sum_l w1[k][l][i] D[l][j]  A = w1 (shuffles), B = D
//   backward t: sum_l D[l][k] w2[l][j][i]               registers
// so the three derivatives of a point and the three transposed
// contributions to it all land in the lane that owns it: the metric product
// and the final sum need no exchange.  The metric factors of this order are
// stored in that ownership ("fragment order", ax8_fragment_index) so each
// lane reads its two points of a plane with one 2-wide load.  Shared memory
// holds D, S and, per
// warp, the per-plane results the t-direction needs at the end (each lane
// touches only its own slots).
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "kernels.cuh"
#include "ssg_internal.h"
#include "ssg_kernels.h"

namespace ssg {
namespace dev {

template <typename T, bool HELM, bool FUSEP>
__global__ void __launch_bounds__(128, 4) k_ax8_dmma(int nel, T* __restrict__ u,
                                                     T* __restrict__ au,
                                                     const T* __restrict__ gf,
                                                     size_t npts, const double* __restrict__ bj,
                                                     const double* __restrict__ Dg,
                                                     const double* __restrict__ Sg,
                                                     double lambda, PUpdate pu, ScalarOp dop) {
  constexpr int N = 8, NN = 64, NT = 512, WPB = 4;
  using V2 = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
  if (FUSEP && pu.stop && *pu.stop != 0.0) return;   // uniform over the grid
  __shared__ double sD[NN], sS[NN];
  // per warp: the transposed r/s contributions and the t-flux of every
  // plane, [k][s][lane]
  __shared__ double sAcc[WPB][N][2][32], sW2[WPB][N][2][32];
  for (int q = threadIdx.x; q < NN; q += blockDim.x) {
    sD[q] = Dg[q];
    sS[q] = HELM ? Sg[q] : Dg[q];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  // derivative fragments: D[g][4c+t] (A of forward r, B of forward s) and
  // D[4c+t][g] (A of backward r, B of backward s); S where Helmholtz has it
  double fA[2], fB[2], bA[2], bB[2];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    fA[c] = (HELM ? sS : sD)[g * N + 4 * c + t];   // forward r: S (Helmholtz)
    fB[c] = sD[g * N + 4 * c + t];                 // forward s: D^T chunk
    bA[c] = sD[(4 * c + t) * N + g];               // backward r: D^T
    bB[c] = (HELM ? sS : sD)[(4 * c + t) * N + g]; // backward s: S (Helmholtz)
  }
  const double* Xt = HELM ? sS : sD;               // backward t matrix
  const double beta = FUSEP ? (pu.first ? 0.0 : *pu.beta) : 0.0;
  const double cc = (FUSEP && pu.c) ? *pu.c : 0.0;
  const T* z = FUSEP ? reinterpret_cast<const T*>(pu.z) : nullptr;
  const double* mask = FUSEP ? pu.mask : nullptr;
  double (*acc)[2][32] = sAcc[wid];
  double (*w2)[2][32] = sW2[wid];
  const int warps = WPB * gridDim.x;
  double pap = 0.0;   // p . (A p) over this lane's points (FUSEP with a dot)
  for (int e = blockIdx.x * WPB + wid; e < nel; e += warps) {
    const size_t base = (size_t)e * NT;
    // value of the input field at local node q of this element (FUSEP: the
    // updated direction p = beta p + (z - c), masked)
    // (stored as T: the value the kernel writes back for FUSEP)
    auto val = [&](int q) -> double {
      const size_t o = base + q;
      if (!FUSEP) return (double)u[o];
      const double zc = (double)z[o] - cc;
      double v = pu.first ? zc : beta * (double)u[o] + zc;
      if (mask) v = v * mask[o];
      return (double)(T)v;
    };
    double uo[N][2];
#pragma unroll
    for (int k = 0; k < N; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) uo[k][s] = val(k * NN + (2 * t + s) * N + g);
    // the warp's next element: its field (and, fused, z) into L2 now (the
    // caller's arrays only when 16-byte aligned, as the bulk copy requires;
    // elements are 16-byte multiples)
    if (e + warps < nel && lane < (FUSEP ? 2 : 1)) {
      const T* f = lane == 0 ? (const T*)u : z;
      if ((reinterpret_cast<uintptr_t>(f) & 15u) == 0)
        bulk_prefetch_l2(f + (size_t)(e + warps) * NT, NT * sizeof(T));
    }
#pragma unroll 1
    for (int k = 0; k < N; ++k) {
      // the next plane's six metric factors (this element's k + 1, or the
      // next element's plane 0) into L2 while this plane computes: one
      // contiguous 64-value chunk per factor in fragment order
      {
        const int kn = k + 1 < N ? k + 1 : 0;
        const int en = k + 1 < N ? e : e + warps;
        if (lane < 6 && en < nel)
          bulk_prefetch_l2(gf + lane * npts + (size_t)en * NT + kn * NN, NN * sizeof(T));
      }
      // forward r: B = u[k][j = g][l = 4c + t]; forward s: A = u[k][l = 4c + t][i = g]
      const double b0 = val(k * NN + g * N + t), b1 = val(k * NN + g * N + 4 + t);
      const double a0 = val(k * NN + t * N + g), a1 = val(k * NN + (4 + t) * N + g);
      // metric factors in fragment order: this lane's two points of plane k
      // are adjacent (ax8_fragment_index), one 2-wide load per factor
      double gg[2][6];
      {
        const size_t o = base + k * NN + 2 * lane;
#pragma unroll
        for (int a = 0; a < 6; ++a) {
          const V2 v = __ldg(reinterpret_cast<const V2*>(gf + a * npts + o));
          gg[0][a] = (double)v.x;
          gg[1][a] = (double)v.y;
        }
      }
      double ur0 = 0.0, ur1 = 0.0, us0 = 0.0, us1 = 0.0;
      dmma(ur0, ur1, fA[0], b0, ur0, ur1);
      dmma(ur0, ur1, fA[1], b1, ur0, ur1);
      dmma(us0, us1, a0, fB[0], us0, us1);
      dmma(us0, us1, a1, fB[1], us0, us1);
      const double urv[2] = {ur0, ur1}, usv[2] = {us0, us1};
      double w0[2], w1[2];
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        // forward t in registers: sum_l D[k][l] u[l][j][i]
        double ut = 0.0;
#pragma unroll
        for (int l = 0; l < N; ++l) ut += sD[k * N + l] * uo[l][s];
        w0[s] = gg[s][0] * urv[s] + gg[s][1] * usv[s] + gg[s][2] * ut;
        w1[s] = gg[s][1] * urv[s] + gg[s][3] * usv[s] + gg[s][4] * ut;
        w2[k][s][lane] = gg[s][2] * urv[s] + gg[s][4] * usv[s] + gg[s][5] * ut;
      }
      // backward r: B[t][g] = w0[k][j = g][i = 4c + t], held by lane
      // 4 (4c + t) + g/2 as its value s = g & 1
      double or0 = 0.0, or1 = 0.0, os0 = 0.0, os1 = 0.0;
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int src = 4 * (4 * c + t) + (g >> 1);
        const double v0 = __shfl_sync(0xffffffffu, w0[0], src);
        const double v1 = __shfl_sync(0xffffffffu, w0[1], src);
        dmma(or0, or1, bA[c], (g & 1) ? v1 : v0, or0, or1);
      }
      // backward s: A[g][t] = w1[k][j = 4c + t][i = g], held by lane
      // 4 g + 2c + t/2 as its value s = t & 1
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int src = 4 * g + 2 * c + (t >> 1);
        const double v0 = __shfl_sync(0xffffffffu, w1[0], src);
        const double v1 = __shfl_sync(0xffffffffu, w1[1], src);
        dmma(os0, os1, (t & 1) ? v1 : v0, bB[c], os0, os1);
      }
      acc[k][0][lane] = or0 + os0;
      acc[k][1][lane] = or1 + os1;
    }
    // backward t (each lane reads only its own column of w2), the sum, the
    // Helmholtz mass term
    double w2r[N][2];
#pragma unroll
    for (int l = 0; l < N; ++l)
#pragma unroll
      for (int s = 0; s < 2; ++s) w2r[l][s] = w2[l][s][lane];
#pragma unroll
    for (int k = 0; k < N; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        double ot = 0.0;
#pragma unroll
        for (int l = 0; l < N; ++l) ot += Xt[l * N + k] * w2r[l][s];
        const size_t o = base + k * NN + (2 * t + s) * N + g;
        double out = acc[k][s][lane] + ot;
        if (HELM) out += lambda * (__ldg(bj + o) * uo[k][s]);
        au[o] = (T)out;
        if (FUSEP) pap += uo[k][s] * (double)(T)out;
      }
    if (FUSEP) {
      // every lane has read this element's old direction: store the new one
      __syncwarp();
#pragma unroll
      for (int k = 0; k < N; ++k)
#pragma unroll
        for (int s = 0; s < 2; ++s) u[base + k * NN + (2 * t + s) * N + g] = (T)uo[k][s];
    }
  }
  if (FUSEP && pu.part) {
    __shared__ double sred[32];
    double v[1] = {pap};
    block_reduce<1>(v, sred);
    finish<1>(v, pu.part, dop, sred);
  }
}

}  // namespace dev

// blocks of 4 warps (one element each), grid capped at 8 blocks per SM and
// walking the elements (FP64 fields: T = double)
template <typename T>
static cudaError_t launch_ax8(cudaStream_t s, int nel, bool helm, T* u, T* au, const T* gf,
                              size_t npts, const double* bj, const double* D, const double* S,
                              double lambda, const dev::PUpdate* pu, const ScalarOp& dop) {
  const int wpb = 4;
  int grid = (nel + wpb - 1) / wpb;
  if (grid > 148 * 8) grid = 148 * 8;
  if (grid < 1) return cudaSuccess;
  const dev::PUpdate p = pu ? *pu : dev::PUpdate();
  count_launch();
  if (helm) {
    if (pu)
      dev::k_ax8_dmma<T, true, true><<<grid, 32 * wpb, 0, s>>>(nel, u, au, gf, npts, bj, D, S,
                                                             lambda, p, dop);
    else
      dev::k_ax8_dmma<T, true, false><<<grid, 32 * wpb, 0, s>>>(nel, u, au, gf, npts, bj, D, S,
                                                              lambda, p, dop);
  } else {
    if (pu)
      dev::k_ax8_dmma<T, false, true><<<grid, 32 * wpb, 0, s>>>(nel, u, au, gf, npts, bj, D,
                                                              D, 0.0, p, dop);
    else
      dev::k_ax8_dmma<T, false, false><<<grid, 32 * wpb, 0, s>>>(nel, u, au, gf, npts, bj, D,
                                                               D, 0.0, p, dop);
  }
  return cudaGetLastError();
}

cudaError_t run_ax8_dmma(cudaStream_t s, int nel, bool helm, bool fp32, void* u, void* au,
                         const void* gf, size_t npts, const double* bj, const double* D,
                         const double* S, double lambda, const dev::PUpdate* pu,
                         const ScalarOp* dop) {
  const ScalarOp o = dop ? *dop : ScalarOp();
  // FP32 storage (the mixed V-cycle) runs the line-form operator in FP32
  // arithmetic; this kernel is the FP64 operator of order 8
  if (fp32) return cudaErrorInvalidValue;
  return launch_ax8<double>(s, nel, helm, (double*)u, (double*)au, (const double*)gf, npts, bj,
                            D, S, lambda, pu, o);
}

}  // namespace ssg
