// Dealiased skew-symmetric convection (convection_operator ->
// antialiased_convection_operator, src/convection.c:31-140), one element per
// block, all in FP64:
//   1. interpolate the advecting u and advected v (3 components each) from
//      the n-point to the m = 3n/2-point GLL grid (interpolate_to_grid,
//      src/interpolation.c:136-155);
//   2. per dealiasing point, the convective form (u . grad) v_c with grad
//      through the conv-grid tinv (src/convection.c:71-93) and the
//      conservative form sum_a sum_b tinv[a][b] d_b(u_b v_c)
//      (src/convection.c:95-127), both weighted by rho J, averaged with
//      weights 1/2 (src/convection.c:129-140);
//   3. project back with (J^T)^3 (integrate_to_grid, src/interpolation.c:
//      157-176).
//
// Step 2 is regrouped per reference direction b (the same sums):
//   skew = sum_b ( A_b d_b v_c + B_b d_b(u_b v_c) ),
//   A_b = sum_a u_a W[a][b],  B_b = sum_a W[a][b],  W[a][b] = rho J tinv[a][b] / 2,
// with W stored at set-up.  So each direction b is one pass over the
// m-point lines along b: a thread holds one line of v_c and of u_b v_c in
// registers, takes both derivatives along it and adds its points' A_b and
// B_b terms -- the contributions of the three directions meet in shared
// memory.  Every contraction (interpolation, derivative, projection) works
// on whole lines held in registers, and the small matrices (D, J, J^T) live
// in the kernel's parameter space: with the loops unrolled, each matrix
// entry is a constant-bank operand of the FMA, so the shared-memory pipe
// carries only the line loads (one per line point instead of two per FMA).
//
// Orders with m^3 fields beyond shared memory (n = 12) and dealiasing orders
// other than 3n/2 run a runtime-order kernel of the same arithmetic that
// keeps the matrices in shared memory and its fields in a global scratch
// region when needed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "kernels.cuh"
#include "ssg_internal.h"
#include "ssg_kernels.h"

namespace ssg {
namespace dev {

// ----------------------------------------------------------------------------
// compile-time-order kernel
// ----------------------------------------------------------------------------

// row stride of an m-wide shared array: 2 mod 4 doubles, so that the
// 16-byte loads of lines along i by lanes walking j hit distinct banks
__host__ __device__ constexpr int conv_row(int w) { return w + ((2 - w % 4) + 4) % 4; }

template <int N, int M>
struct ConvMats {
  double D[M * M];   // D[o * M + l] = l_l'(x_o), m-point grid
  double J[M * N];   // J[o * N + p] = l_p^n(x_o^m)
  double JT[N * M];  // JT[p * M + o] = J[o * N + p]
};

template <int N, int M>
struct ConvLayout {
  static constexpr int RM = conv_row(M);      // row stride, m-wide rows
  static constexpr int RN = conv_row(N);      // row stride, n-wide rows
  static constexpr int FM = M * M * RM;       // an m^3 field
  static constexpr int T1 = N * N * RM;       // interpolation stage x: [k][j][o]
  static constexpr int T2 = N * M * RM;       // stage y: [k][o2][o1]
  static constexpr int P1 = M * M * RN;       // projection stage i: [k][j][p]
  static constexpr int P2 = M * N * RN;       // stage j: [k][p2][p1]
  // UI (3 FM), VC (FM), SK (FM), T1, T2; P1 reuses VC, P2 reuses T2
  static constexpr int TOTAL = 5 * FM + T1 + T2;
  static_assert(P1 <= FM && P2 <= T2, "projection scratch aliases");
};

template <int N, int M>
constexpr size_t conv_smem_bytes() {
  return (size_t)ConvLayout<N, M>::TOTAL * sizeof(double);
}

// y[o] = sum_{l < NI} A[o * NI + l] x[l], summed in l order
template <int NI, int NO>
__device__ __forceinline__ void line_contract(const double* A, const double (&x)[NI],
                                              double (&y)[NO]) {
#pragma unroll
  for (int o = 0; o < NO; ++o) y[o] = A[o * NI] * x[0];
#pragma unroll
  for (int l = 1; l < NI; ++l)
#pragma unroll
    for (int o = 0; o < NO; ++o) y[o] = fma(A[o * NI + l], x[l], y[o]);
}

template <int L>
__device__ __forceinline__ void load_line(const double* p, int stride, double (&x)[L]) {
#pragma unroll
  for (int l = 0; l < L; ++l) x[l] = p[l * stride];
}

// contiguous line (stride 1) at a 16-byte aligned address
template <int L>
__device__ __forceinline__ void load_line_v(const double* p, double (&x)[L]) {
  if constexpr (L % 2 == 0) {
#pragma unroll
    for (int l = 0; l < L; l += 2) {
      const double2 v = *reinterpret_cast<const double2*>(p + l);
      x[l] = v.x;
      x[l + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int l = 0; l < L; ++l) x[l] = p[l];
  }
}

template <int L>
__device__ __forceinline__ void store_line(double* p, int stride, const double (&x)[L]) {
#pragma unroll
  for (int l = 0; l < L; ++l) p[l * stride] = x[l];
}

// n^3 field (global, [k][j][i]) -> m^3 field (shared, rows RM, planes M RM)
template <int N, int M>
__device__ __forceinline__ void interpolate_field(const ConvMats<N, M>& mt,
                                                  const double* __restrict__ src,
                                                  double* t1, double* t2, double* dst) {
  using Lay = ConvLayout<N, M>;
  constexpr int RM = Lay::RM;
  // x: lines (j, k) of n points -> m points, T1[k][j][o]
  for (int t = threadIdx.x; t < N * N; t += blockDim.x) {
    double x[N], y[M];
    if constexpr (N % 2 == 0)
      load_line_v<N>(src + t * N, x);
    else
      load_line<N>(src + t * N, 1, x);
    line_contract<N, M>(mt.J, x, y);
    store_line<M>(t1 + t * RM, 1, y);
  }
  __syncthreads();
  // y: lines (o1, k) along j -> T2[k][o2][o1]
  for (int t = threadIdx.x; t < M * N; t += blockDim.x) {
    const int o1 = t % M, k = t / M;
    double x[N], y[M];
    load_line<N>(t1 + k * N * RM + o1, RM, x);
    line_contract<N, M>(mt.J, x, y);
    store_line<M>(t2 + k * M * RM + o1, RM, y);
  }
  __syncthreads();
  // z: lines (o1, o2) along k -> dst[o3][o2][o1]
  for (int t = threadIdx.x; t < M * M; t += blockDim.x) {
    const int o1 = t % M, o2 = t / M;
    double x[N], y[M];
    load_line<N>(t2 + o2 * RM + o1, M * RM, x);
    line_contract<N, M>(mt.J, x, y);
    store_line<M>(dst + o2 * RM + o1, M * RM, y);
  }
  __syncthreads();
}

// one direction b of the skew-symmetric form for advected component vc:
// lines along b; SK (=/+=) A_b d_b vc + B_b d_b(u_b vc) at every point
template <int N, int M, int B>
__device__ __forceinline__ void convection_pass(const ConvMats<N, M>& mt,
                                                const double* __restrict__ W,
                                                size_t wstride, const double* ui,
                                                const double* vc, double* sk) {
  using Lay = ConvLayout<N, M>;
  constexpr int RM = Lay::RM, FM = Lay::FM;
  // line step in shared memory / in the unpadded global point index
  constexpr int SS = B == 0 ? 1 : (B == 1 ? RM : M * RM);
  constexpr int SG = B == 0 ? 1 : (B == 1 ? M : M * M);
  for (int t = threadIdx.x; t < M * M; t += blockDim.x) {
    const int a0 = t % M, a1 = t / M;   // the two coordinates across the line
    int base_s, base_g;
    if constexpr (B == 0) {            // (j, k)
      base_s = a0 * RM + a1 * M * RM;
      base_g = a0 * M + a1 * M * M;
    } else if constexpr (B == 1) {     // (i, k)
      base_s = a0 + a1 * M * RM;
      base_g = a0 + a1 * M * M;
    } else {                           // (i, j)
      base_s = a0 + a1 * RM;
      base_g = a0 + a1 * M;
    }
    double v[M], p[M];
    if constexpr (B == 0) {
      load_line_v<M>(vc + base_s, v);
      load_line_v<M>(ui + base_s, p);
    } else {
      load_line<M>(vc + base_s, SS, v);
      load_line<M>(ui + B * FM + base_s, SS, p);
    }
    double dv[M];
    line_contract<M, M>(mt.D, v, dv);
#pragma unroll
    for (int o = 0; o < M; ++o) p[o] = p[o] * v[o];
    double dp[M];
    line_contract<M, M>(mt.D, p, dp);
#pragma unroll
    for (int o = 0; o < M; ++o) {
      const int q = base_s + o * SS;
      const size_t g = base_g + o * SG;
      const double w0 = __ldg(W + g), w1 = __ldg(W + wstride + g),
                   w2 = __ldg(W + 2 * wstride + g);
      double A = w0 * ui[q];
      A = fma(w1, ui[FM + q], A);
      A = fma(w2, ui[2 * FM + q], A);
      const double Bb = (w0 + w1) + w2;
      double s = A * dv[o];
      s = fma(Bb, dp[o], s);
      if constexpr (B == 0)
        sk[q] = s;
      else
        sk[q] += s;
    }
  }
  __syncthreads();
}

// m^3 shared field -> n^3 global field through (J^T)^3
template <int N, int M>
__device__ __forceinline__ void project_field(const ConvMats<N, M>& mt, const double* sk,
                                              double* p1, double* p2,
                                              double* __restrict__ dst) {
  using Lay = ConvLayout<N, M>;
  constexpr int RM = Lay::RM, RN = Lay::RN;
  // i: lines (j, k) of m points -> n points, P1[k][j][p]
  for (int t = threadIdx.x; t < M * M; t += blockDim.x) {
    const int j = t % M, k = t / M;
    double x[M], y[N];
    load_line_v<M>(sk + j * RM + k * M * RM, x);
    line_contract<M, N>(mt.JT, x, y);
    store_line<N>(p1 + (k * M + j) * RN, 1, y);
  }
  __syncthreads();
  // j: lines (p1, k) -> P2[k][p2][p1]
  for (int t = threadIdx.x; t < N * M; t += blockDim.x) {
    const int q1 = t % N, k = t / N;
    double x[M], y[N];
    load_line<M>(p1 + k * M * RN + q1, RN, x);
    line_contract<M, N>(mt.JT, x, y);
    store_line<N>(p2 + k * N * RN + q1, RN, y);
  }
  __syncthreads();
  // k: lines (p1, p2) -> dst[p3][p2][p1]
  for (int t = threadIdx.x; t < N * N; t += blockDim.x) {
    const int q1 = t % N, q2 = t / N;
    double x[M], y[N];
    load_line<M>(p2 + q2 * RN + q1, N * RN, x);
    line_contract<M, N>(mt.JT, x, y);
    store_line<N>(dst + q2 * N + q1, N * N, y);
  }
  __syncthreads();
}

constexpr int kConvThreads = 160;

// Fields u, v, udv hold `nel` elements (component stride nel n^3); the
// dealiasing factors W hold all `nel_fac` elements of the mesh, and field
// element e reads the factors of mesh element e0 + e.  W: 9 arrays in the
// order (b, a), W[(3b + a)][e][q] = rho J tinv[a][b] / 2.
template <int N, int M>
__global__ void __launch_bounds__(kConvThreads, 2)
    k_convection(int nel, int e0, int nel_fac, const double* __restrict__ u,
                 const double* __restrict__ v, double* __restrict__ udv,
                 const double* __restrict__ W, const __grid_constant__ ConvMats<N, M> mt) {
  using Lay = ConvLayout<N, M>;
  extern __shared__ __align__(16) double smem[];
  double* ui = smem;                 // 3 x FM
  double* vc = ui + 3 * Lay::FM;     // FM; projection stage 1 reuses it
  double* sk = vc + Lay::FM;         // FM
  double* t1 = sk + Lay::FM;
  double* t2 = t1 + Lay::T1;         // projection stage 2 reuses it
  constexpr int NT = N * N * N, MT = M * M * M;
  const size_t nptsn = (size_t)nel * NT, wstride = (size_t)nel_fac * MT;
  for (int e = blockIdx.x; e < nel; e += gridDim.x) {
    const double* Wb = W + (size_t)(e0 + e) * MT;
#pragma unroll 1
    for (int f = 0; f < 3; ++f)
      interpolate_field<N, M>(mt, u + f * nptsn + (size_t)e * NT, t1, t2, ui + f * Lay::FM);
#pragma unroll 1
    for (int c = 0; c < 3; ++c) {
      interpolate_field<N, M>(mt, v + c * nptsn + (size_t)e * NT, t1, t2, vc);
      convection_pass<N, M, 0>(mt, Wb, wstride, ui, vc, sk);
      convection_pass<N, M, 1>(mt, Wb + 3 * wstride, wstride, ui, vc, sk);
      convection_pass<N, M, 2>(mt, Wb + 6 * wstride, wstride, ui, vc, sk);
      project_field<N, M>(mt, sk, vc, t2, udv + c * nptsn + (size_t)e * NT);
    }
  }
}

// ----------------------------------------------------------------------------
// runtime-order kernel (any n, m; fields in a global scratch region when they
// exceed shared memory)
// ----------------------------------------------------------------------------

// out (no^3) = (A x A x A) in (ni^3), stages x, y, z; A[o*ni + q]
// (transpose = true: A[q*no + o], the weak projection).  Block-cooperative.
__device__ void block_tensor3(int ni, int no, const double* A, bool transpose,
                              const double* in, double* t1, double* t2, double* out) {
  auto a = [&](int o, int q) { return transpose ? A[q * no + o] : A[o * ni + q]; };
  for (int q = threadIdx.x; q < ni * ni * no; q += blockDim.x) {
    const int o = q % no, kj = q / no;
    double s = 0;
    for (int r = 0; r < ni; ++r) s += a(o, r) * in[kj * ni + r];
    t1[q] = s;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < ni * no * no; q += blockDim.x) {
    const int o1 = q % no, o2 = (q / no) % no, k = q / (no * no);
    double s = 0;
    for (int r = 0; r < ni; ++r) s += a(o2, r) * t1[(k * ni + r) * no + o1];
    t2[q] = s;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < no * no * no; q += blockDim.x) {
    const int o12 = q % (no * no), o3 = q / (no * no);
    double s = 0;
    for (int r = 0; r < ni; ++r) s += a(o3, r) * t2[r * no * no + o12];
    out[q] = s;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(512, 1) k_convection_rt(
    int nel, int e0, int nel_fac, int n, int m, const double* __restrict__ u,
    const double* __restrict__ v, double* __restrict__ udv, const double* __restrict__ W,
    const double* __restrict__ Dm, const double* __restrict__ J, double* __restrict__ gscr) {
  extern __shared__ __align__(16) double srt[];
  const int nt = n * n * n, mt = m * m * m;
  const int tmax = n * m * m > n * n * m ? n * m * m : n * n * m;
  double* sD = srt;                  // D[i*m + l]
  double* sJ = sD + m * m;           // J[i*n + p]
  double* t1 = sJ + m * n;
  double* t2 = t1 + tmax;
  double* stage = t2 + tmax;         // nt
  double* ui = gscr ? gscr + (size_t)blockIdx.x * 5 * mt : stage + nt;   // 3 x mt
  double* vc = ui + 3 * mt;
  double* sk = vc + mt;
  const size_t nptsn = (size_t)nel * nt, wstride = (size_t)nel_fac * mt;
  for (int q = threadIdx.x; q < m * m; q += blockDim.x) sD[q] = Dm[q];
  for (int q = threadIdx.x; q < m * n; q += blockDim.x) sJ[q] = J[q];
  for (size_t e = blockIdx.x; e < (size_t)nel; e += gridDim.x) {
    for (int f = 0; f < 3; ++f) {
      __syncthreads();
      for (int q = threadIdx.x; q < nt; q += blockDim.x) stage[q] = u[f * nptsn + e * nt + q];
      __syncthreads();
      block_tensor3(n, m, sJ, false, stage, t1, t2, ui + f * mt);
    }
    for (int c = 0; c < 3; ++c) {
      __syncthreads();
      for (int q = threadIdx.x; q < nt; q += blockDim.x) stage[q] = v[c * nptsn + e * nt + q];
      __syncthreads();
      block_tensor3(n, m, sJ, false, stage, t1, t2, vc);
      for (int q = threadIdx.x; q < mt; q += blockDim.x) {
        const int i = q % m, j = (q / m) % m, k = q / (m * m);
        const size_t g = (e + e0) * mt + q;
        const int base[3] = {(k * m + j) * m, k * m * m + i, j * m + i};
        const int step[3] = {1, m, m * m};
        const int at[3] = {i, j, k};
        double s = 0.0;
        for (int b = 0; b < 3; ++b) {
          double dv = 0.0, dp = 0.0;
          for (int l = 0; l < m; ++l) {
            const double d = sD[at[b] * m + l];
            const double vl = vc[base[b] + l * step[b]];
            dv = fma(d, vl, dv);
            dp = fma(d, ui[b * mt + base[b] + l * step[b]] * vl, dp);
          }
          const double w0 = W[(3 * b) * wstride + g], w1 = W[(3 * b + 1) * wstride + g],
                       w2 = W[(3 * b + 2) * wstride + g];
          double A = w0 * ui[q];
          A = fma(w1, ui[mt + q], A);
          A = fma(w2, ui[2 * mt + q], A);
          const double Bb = (w0 + w1) + w2;
          s = b == 0 ? A * dv : fma(A, dv, s);
          s = fma(Bb, dp, s);
        }
        sk[q] = s;
      }
      __syncthreads();
      block_tensor3(m, n, sJ, true, sk, t1, t2, stage);
      for (int q = threadIdx.x; q < nt; q += blockDim.x) udv[c * nptsn + e * nt + q] = stage[q];
    }
    __syncthreads();
  }
}

}  // namespace dev

static size_t convection_rt_smem(int n, int m, bool fields) {
  const size_t nt = (size_t)n * n * n, mt = (size_t)m * m * m;
  const size_t tmax = std::max((size_t)n * m * m, (size_t)n * n * m);
  return (m * m + m * n + 2 * tmax + nt + (fields ? 5 * mt : 0)) * sizeof(double);
}

static constexpr size_t kConvSmemMax = 227 * 1024;

template <int N>
static constexpr bool conv_fast_order() {
  return dev::conv_smem_bytes<N, (3 * N) / 2>() <= kConvSmemMax;
}

static bool conv_fast(int n, int m) {
  if (m != (3 * n) / 2) return false;
  switch (n) {
#define SSG_CONVF(NV) \
  case NV:            \
    return conv_fast_order<NV>();
    SSG_CONVF(2) SSG_CONVF(3) SSG_CONVF(4) SSG_CONVF(5) SSG_CONVF(6) SSG_CONVF(7)
    SSG_CONVF(8) SSG_CONVF(9) SSG_CONVF(10) SSG_CONVF(11)
#undef SSG_CONVF
    default:
      return false;
  }
}

size_t convection_scratch_doubles(int n, int m) {
  if (conv_fast(n, m) || convection_rt_smem(n, m, true) <= kConvSmemMax) return 0;
  return (size_t)kConvScratchBlocks * 5 * m * m * m;
}

template <int N>
static cudaError_t launch_fast(cudaStream_t s, int nel, int e0, int nel_fac, const double* u,
                               const double* v, double* udv, const double* W,
                               const double* Dh, const double* Jh, int grid) {
  constexpr int M = (3 * N) / 2;
  if constexpr (!conv_fast_order<N>()) {
    return cudaErrorInvalidValue;
  } else {
    dev::ConvMats<N, M> mt;
    for (int q = 0; q < M * M; ++q) mt.D[q] = Dh[q];
    for (int o = 0; o < M; ++o)
      for (int p = 0; p < N; ++p) {
        mt.J[o * N + p] = Jh[o * N + p];
        mt.JT[p * M + o] = Jh[o * N + p];
      }
    constexpr size_t smem = dev::conv_smem_bytes<N, M>();
    static SmemAttr attr;
    cudaError_t e = attr.ensure((const void*)dev::k_convection<N, M>, smem);
    if (e != cudaSuccess) return e;
    count_launch();
    dev::k_convection<N, M><<<grid, dev::kConvThreads, smem, s>>>(nel, e0, nel_fac, u, v, udv,
                                                                 W, mt);
    return cudaGetLastError();
  }
}

cudaError_t run_convection(cudaStream_t s, int nel, int e0, int nel_fac, int n, int m,
                           const double* u, const double* v, double* udv, const double* W,
                           const double* Dh, const double* Jh, const double* Dd,
                           const double* Jd, double* scratch) {
  if (nel <= 0) return cudaSuccess;
  if (convection_dmma_applies(n, m))
    return run_convection_dmma(s, nel, e0, nel_fac, u, v, udv, W, Dh, Jh);
  // the compile-time-order kernel reads element lines with 16-byte loads:
  // fields at addresses that are not 16-byte aligned take the runtime-order
  // kernel
  const bool aligned =
      ((reinterpret_cast<uintptr_t>(u) | reinterpret_cast<uintptr_t>(v)) & 15u) == 0;
  if (aligned && conv_fast(n, m)) {
    switch (n) {
#define SSG_CONVL(NV) \
  case NV:            \
    return launch_fast<NV>(s, nel, e0, nel_fac, u, v, udv, W, Dh, Jh, nel);
      SSG_CONVL(2) SSG_CONVL(3) SSG_CONVL(4) SSG_CONVL(5) SSG_CONVL(6) SSG_CONVL(7)
      SSG_CONVL(8) SSG_CONVL(9) SSG_CONVL(10) SSG_CONVL(11)
#undef SSG_CONVL
      default:
        break;
    }
  }
  const bool in_smem = convection_rt_smem(n, m, true) <= kConvSmemMax;
  if (!in_smem && !scratch) return cudaErrorInvalidValue;
  const size_t smem = convection_rt_smem(n, m, in_smem);
  if (smem > kConvSmemMax) return cudaErrorInvalidValue;
  static SmemAttr attr;
  {
    cudaError_t e = attr.ensure((const void*)dev::k_convection_rt, kConvSmemMax);
    if (e != cudaSuccess) return e;
  }
  const int grid = in_smem ? nel : std::min(nel, kConvScratchBlocks);
  count_launch();
  dev::k_convection_rt<<<grid, 512, smem, s>>>(nel, e0, nel_fac, n, m, u, v, udv, W, Dd, Jd,
                                               in_smem ? nullptr : scratch);
  return cudaGetLastError();
}

}  // namespace ssg
