// Stokes operators of the time step, one element per block:
//   * the double curl curl(curl u) times the mass (double_curl_operator and
//     discrete_curl_operator, src/stokes.c:71-105), the viscous term of the
//     pressure gradient estimate;
//   * the pressure equation's right-hand side before its DSS: the weak
//     divergence of the intermediate velocity (discrete_divergence_operator,
//     src/stokes.c:52-69) scaled by -dens / dt, plus the surface integrals
//     of the estimated pressure gradient over the wall faces
//     (compute_pressure_rhs, src/navier_stokes.c:115-146, with
//     add_surface_integral, src/poisson.c:145-194);
//   * the velocity equations' right-hand sides before their DSS: the mass
//     times the intermediate velocity over dt visc, minus the weak pressure
//     gradient (discrete_gradient_operator, src/stokes.c:30-50) with its
//     surface integrals over the faces without a wall, over visc dens
//     (compute_velocity_rhs, src/navier_stokes.c:177-201).
//
// Each follows the reference's operation order per point: derivatives in
// the reference coordinates from the GLL derivative matrix, then the
// combination with the transposed inverse Jacobian in the reference's term
// order, the mass product as (u rho) det, and the surface terms face by face
// (W E S N B T) and derivative by derivative.  Products and sums outside the
// derivative contractions are rounded one by one (no contraction into fused
// multiply-adds, as the reference's scalar loops), the BLAS axpy and the
// derivative sums as fused multiply-adds.
#include <cuda_runtime.h>

#include "ssg_internal.h"
#include "ssg_kernels.h"

namespace ssg {
namespace dev {

struct StokesGeom {
  const double* tinv = nullptr;   // 9 x npts: tinv[3a + b] = dr_b / dx_a
  const double* rho = nullptr;    // n^3 GLL weight products
  const double* det = nullptr;    // npts: det J
  const double* D = nullptr;      // n x n: D[i n + m] = l_m'(x_i)
  const int* bc = nullptr;        // wall faces per element: bit f for face f of W E S N B T
  const double* sw = nullptr;     // nel x 3 x 6 x n^2: (w_inner w_outer) n_d on each face
  size_t npts = 0;
};

// d f / d(r, s, t) at node (i, j, k) of an element staged in shared memory
template <int N>
__device__ __forceinline__ void ref_grad(const double* __restrict__ f,
                                         const double* __restrict__ sD, int i, int j, int k,
                                         double& dr, double& ds, double& dt) {
  double a = 0.0, b = 0.0, c = 0.0;
#pragma unroll
  for (int m = 0; m < N; ++m) {
    a = fma(sD[i * N + m], f[(k * N + j) * N + m], a);
    b = fma(sD[j * N + m], f[(k * N + m) * N + i], b);
    c = fma(sD[k * N + m], f[(m * N + j) * N + i], c);
  }
  dr = a;
  ds = b;
  dt = c;
}

// (D_r^T x + D_s^T y) + D_t^T z at node (i, j, k) (transpose_divergence,
// src/deriv.c:54-66: three products summed in that order)
template <int N>
__device__ __forceinline__ double ref_tdiv(const double* __restrict__ x,
                                           const double* __restrict__ y,
                                           const double* __restrict__ z,
                                           const double* __restrict__ sD, int i, int j, int k) {
  double a = 0.0, b = 0.0, c = 0.0;
#pragma unroll
  for (int m = 0; m < N; ++m) {
    a = fma(sD[m * N + i], x[(k * N + j) * N + m], a);
    b = fma(sD[m * N + j], y[(k * N + m) * N + i], b);
    c = fma(sD[m * N + k], z[(m * N + j) * N + i], c);
  }
  return __dadd_rn(__dadd_rn(a, b), c);
}

// curl at a point from J[a][b] = du_a / dr_b and T[a][b] = dr_b / dx_a
// (discrete_curl_operator, src/stokes.c:71-92): component j sums, over i,
// s_j J[k][i] T[l][i] and then -s_j J[l][i] T[k][i], with (k, l) = (2, 1),
// (2, 0), (1, 0) and s_j = +1, -1, +1
__device__ __forceinline__ void curl_point(const double J[3][3], const double T[3][3],
                                           double w[3]) {
  const int K[3] = {2, 2, 1}, L[3] = {1, 0, 0};
  const double S[3] = {1.0, -1.0, 1.0};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double t1 = __dmul_rn(S[c] * J[K[c]][i], T[L[c]][i]);
      acc = i == 0 ? t1 : __dadd_rn(t1, acc);
      acc = __dadd_rn(__dmul_rn(-S[c] * J[L[c]][i], T[K[c]][i]), acc);
    }
    w[c] = acc;
  }
}

__device__ __forceinline__ void load_tinv(const StokesGeom& G, size_t g, double T[3][3]) {
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) T[a][b] = __ldg(G.tinv + (size_t)(3 * a + b) * G.npts + g);
}

// the mass product (test_function_inner_product, src/poisson.c:58-66)
__device__ __forceinline__ double mass(const StokesGeom& G, double v, int q, size_t g) {
  return __dmul_rn(__dmul_rn(v, __ldg(G.rho + q)), __ldg(G.det + g));
}

// v plus the surface terms of derivative d over the faces in `faces` that
// node (i, j, k) lies on, in the face order W E S N B T
// (add_surface_integral, src/poisson.c:145-194)
template <int N>
__device__ __forceinline__ double add_surface(const StokesGeom& G, int e, int faces, int d,
                                              int i, int j, int k, double v, double gv) {
  constexpr int M = N - 1, NN = N * N;
  const double* s = G.sw + ((size_t)e * 3 + d) * 6 * NN;
  if ((faces & 1) && i == 0) v = __dadd_rn(v, __dmul_rn(s[0 * NN + k * N + j], gv));
  if ((faces & 2) && i == M) v = __dadd_rn(v, __dmul_rn(s[1 * NN + k * N + j], gv));
  if ((faces & 4) && j == 0) v = __dadd_rn(v, __dmul_rn(s[2 * NN + k * N + i], gv));
  if ((faces & 8) && j == M) v = __dadd_rn(v, __dmul_rn(s[3 * NN + k * N + i], gv));
  if ((faces & 16) && k == 0) v = __dadd_rn(v, __dmul_rn(s[4 * NN + j * N + i], gv));
  if ((faces & 32) && k == M) v = __dadd_rn(v, __dmul_rn(s[5 * NN + j * N + i], gv));
  return v;
}

template <int N>
__global__ void __launch_bounds__(256) k_double_curl(const double* __restrict__ u,
                                                     double* __restrict__ rot, StokesGeom G) {
  constexpr int NT = N * N * N;
  extern __shared__ double sm[];
  double* sD = sm;
  double* sU = sD + N * N;
  double* sW = sU + 3 * NT;
  const int e = blockIdx.x;
  const size_t o = (size_t)e * NT;
  for (int q = threadIdx.x; q < N * N; q += blockDim.x) sD[q] = G.D[q];
  for (int q = threadIdx.x; q < NT; q += blockDim.x)
#pragma unroll
    for (int c = 0; c < 3; ++c) sU[c * NT + q] = u[c * G.npts + o + q];
  __syncthreads();
  for (int q = threadIdx.x; q < NT; q += blockDim.x) {
    const int i = q % N, j = (q / N) % N, k = q / (N * N);
    double J[3][3], T[3][3], w[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) ref_grad<N>(sU + a * NT, sD, i, j, k, J[a][0], J[a][1], J[a][2]);
    load_tinv(G, o + q, T);
    curl_point(J, T, w);
#pragma unroll
    for (int c = 0; c < 3; ++c) sW[c * NT + q] = w[c];
  }
  __syncthreads();
  for (int q = threadIdx.x; q < NT; q += blockDim.x) {
    const int i = q % N, j = (q / N) % N, k = q / (N * N);
    double J[3][3], T[3][3], w[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) ref_grad<N>(sW + a * NT, sD, i, j, k, J[a][0], J[a][1], J[a][2]);
    load_tinv(G, o + q, T);
    curl_point(J, T, w);
#pragma unroll
    for (int c = 0; c < 3; ++c) rot[c * G.npts + o + q] = mass(G, w[c], q, o + q);
  }
}

// rhs = mass(div ut) * scale, plus the surface terms of g over the wall faces
template <int N>
__global__ void __launch_bounds__(256) k_pressure_rhs(const double* __restrict__ ut,
                                                      const double* __restrict__ g,
                                                      double* __restrict__ rhs, double scale,
                                                      StokesGeom G) {
  constexpr int NT = N * N * N;
  extern __shared__ double sm[];
  double* sD = sm;
  double* sU = sD + N * N;
  const int e = blockIdx.x;
  const size_t o = (size_t)e * NT;
  for (int q = threadIdx.x; q < N * N; q += blockDim.x) sD[q] = G.D[q];
  for (int q = threadIdx.x; q < NT; q += blockDim.x)
#pragma unroll
    for (int c = 0; c < 3; ++c) sU[c * NT + q] = ut[c * G.npts + o + q];
  __syncthreads();
  const int walls = G.bc[e];
  for (int q = threadIdx.x; q < NT; q += blockDim.x) {
    const int i = q % N, j = (q / N) % N, k = q / (N * N);
    double J[3][3], T[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a) ref_grad<N>(sU + a * NT, sD, i, j, k, J[a][0], J[a][1], J[a][2]);
    load_tinv(G, o + q, T);
    // sum over i, then j, of du_i/dr_j dr_j/dx_i (src/stokes.c:61-65)
    double div = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const double t = __dmul_rn(J[a][b], T[a][b]);
        div = (a == 0 && b == 0) ? t : __dadd_rn(t, div);
      }
    double v = __dmul_rn(mass(G, div, q, o + q), scale);
    if (walls)
#pragma unroll
      for (int d = 0; d < 3; ++d)
        v = add_surface<N>(G, e, walls, d, i, j, k, v, g[d * G.npts + o + q]);
    rhs[o + q] = v;
  }
}

// rhs_d = mass(ut_d s) + a (-grad_d p + surface terms of p over the faces
// without a wall), d = 0, 1, 2
template <int N>
__global__ void __launch_bounds__(256) k_velocity_rhs(const double* __restrict__ ut,
                                                      const double* __restrict__ p,
                                                      double* __restrict__ rhs, double s,
                                                      double a, StokesGeom G) {
  constexpr int NT = N * N * N;
  extern __shared__ double sm[];
  double* sD = sm;
  double* sP = sD + N * N;   // mass(p)
  double* sT = sP + NT;      // tinv[d][i] mass(p), i = 0, 1, 2
  const int e = blockIdx.x;
  const size_t o = (size_t)e * NT;
  for (int q = threadIdx.x; q < N * N; q += blockDim.x) sD[q] = G.D[q];
  for (int q = threadIdx.x; q < NT; q += blockDim.x) sP[q] = mass(G, p[o + q], q, o + q);
  const int open = ~G.bc[e] & 63;
  for (int d = 0; d < 3; ++d) {
    __syncthreads();   // sP ready; the previous derivative's reads of sT done
    for (int q = threadIdx.x; q < NT; q += blockDim.x)
#pragma unroll
      for (int i = 0; i < 3; ++i)
        sT[i * NT + q] = __dmul_rn(__ldg(G.tinv + (size_t)(3 * d + i) * G.npts + o + q), sP[q]);
    __syncthreads();
    for (int q = threadIdx.x; q < NT; q += blockDim.x) {
      const int i = q % N, j = (q / N) % N, k = q / (N * N);
      double gr = -ref_tdiv<N>(sT, sT + NT, sT + 2 * NT, sD, i, j, k);
      gr = add_surface<N>(G, e, open, d, i, j, k, gr, p[o + q]);
      const double r = mass(G, __dmul_rn(ut[d * G.npts + o + q], s), q, o + q);
      rhs[d * G.npts + o + q] = fma(a, gr, r);
    }
  }
}

}  // namespace dev

namespace {

template <int N>
size_t stokes_smem(int which) {
  constexpr size_t NT = (size_t)N * N * N;
  const size_t fields = which == 0 ? 6 * NT : (which == 1 ? 3 * NT : 4 * NT);
  return (N * N + fields) * sizeof(double);
}

template <int N>
cudaError_t launch_stokes(cudaStream_t s, int which, int nel, const dev::StokesGeom& G,
                          const double* in, const double* g, double* out, double x, double y) {
  static SmemAttr attr[3];
  const size_t smem = stokes_smem<N>(which);
  const int threads = N * N * N >= 256 ? 256 : ((N * N * N + 31) / 32) * 32;
  cudaError_t e;
  count_launch();
  switch (which) {
    case 0:
      if ((e = attr[0].ensure((const void*)&dev::k_double_curl<N>, smem)) != cudaSuccess)
        return e;
      dev::k_double_curl<N><<<nel, threads, smem, s>>>(in, out, G);
      break;
    case 1:
      if ((e = attr[1].ensure((const void*)&dev::k_pressure_rhs<N>, smem)) != cudaSuccess)
        return e;
      dev::k_pressure_rhs<N><<<nel, threads, smem, s>>>(in, g, out, x, G);
      break;
    default:
      if ((e = attr[2].ensure((const void*)&dev::k_velocity_rhs<N>, smem)) != cudaSuccess)
        return e;
      dev::k_velocity_rhs<N><<<nel, threads, smem, s>>>(in, g, out, x, y, G);
      break;
  }
  return cudaGetLastError();
}

}  // namespace

// which: 0 = double curl of in (3 fields) into out (3 fields); 1 = pressure
// right-hand side of in = ut (3 fields) and g (3 fields) into out (1 field),
// x = scale; 2 = velocity right-hand sides of in = ut (3 fields) and g = p
// (1 field) into out (3 fields), x = s, y = a
cudaError_t run_stokes(cudaStream_t s, int which, int n, int nel, const double* tinv,
                       const double* rho, const double* det, const double* D, const int* bc,
                       const double* sw, size_t npts, const double* in, const double* g,
                       double* out, double x, double y) {
  if (nel <= 0) return cudaSuccess;
  dev::StokesGeom G;
  G.tinv = tinv;
  G.rho = rho;
  G.det = det;
  G.D = D;
  G.bc = bc;
  G.sw = sw;
  G.npts = npts;
  switch (n) {
#define SSG_STOKESN(NV) \
  case NV: return launch_stokes<NV>(s, which, nel, G, in, g, out, x, y);
    SSG_STOKESN(2) SSG_STOKESN(3) SSG_STOKESN(4) SSG_STOKESN(5) SSG_STOKESN(6)
    SSG_STOKESN(7) SSG_STOKESN(8) SSG_STOKESN(9) SSG_STOKESN(10) SSG_STOKESN(11)
    SSG_STOKESN(12)
#undef SSG_STOKESN
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace ssg
