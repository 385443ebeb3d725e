// Dealiased skew-symmetric convection (convection_operator ->
// antialiased_convection_operator, src/convection.c:31-140), one element per
// block, all in FP64:
//   1. interpolate the advecting u and advected v (3 components each) from
//      the n-point to the m = 3n/2-point GLL grid (interpolate_to_grid,
//      src/interpolation.c:136-155);
//   2. per dealiasing point, convective form (u . grad) v_c with grad from the
//      conv-grid tinv (src/convection.c:71-93) and conservative form
//      sum_a sum_b tinv[a][b] d_b(u_b v_c) (src/convection.c:95-127), both
//      weighted by rho J, averaged with weights 1/2 (src/convection.c:129-140);
//   3. project back with (J^T)^3 (integrate_to_grid, src/interpolation.c:
//      157-176).
// The derivatives of the products u_b v_c are taken on the fly from the
// interpolated fields; per element the three advecting components, one
// advected component and its result are stored (the advected components
// are taken one at a time): in shared memory while they fit, else in a
// global scratch region of 5 m^3 doubles per block.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "kernels.cuh"
#include "ssg_internal.h"
#include "ssg_kernels.h"

namespace ssg {
namespace dev {

// out (no^3) = (A x A x A) in (ni^3), stages x, y, z; A[o*ni + q]
// (transpose = true: A[q*no + o], the weak projection).  Block-cooperative.
// NI, NO > 0: compile-time orders (loops unrolled); 0: the runtime ni, no.
template <int NI, int NO>
__device__ void block_tensor3(int ni_rt, int no_rt, const double* A, bool transpose,
                              const double* in, double* t1, double* t2, double* out,
                              double* gout) {
  const int ni = NI > 0 ? NI : ni_rt, no = NO > 0 ? NO : no_rt;
  auto a = [&](int o, int q) { return transpose ? A[q * no + o] : A[o * ni + q]; };
  for (int q = threadIdx.x; q < ni * ni * no; q += blockDim.x) {
    const int o = q % no, kj = q / no;
    double s = 0;
#pragma unroll
    for (int r = 0; r < (NI > 0 ? NI : ni); ++r) s += a(o, r) * in[kj * ni + r];
    t1[q] = s;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < ni * no * no; q += blockDim.x) {
    const int o1 = q % no, o2 = (q / no) % no, k = q / (no * no);
    double s = 0;
#pragma unroll
    for (int r = 0; r < (NI > 0 ? NI : ni); ++r) s += a(o2, r) * t1[(k * ni + r) * no + o1];
    t2[q] = s;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < no * no * no; q += blockDim.x) {
    const int o12 = q % (no * no), o3 = q / (no * no);
    double s = 0;
#pragma unroll
    for (int r = 0; r < (NI > 0 ? NI : ni); ++r) s += a(o3, r) * t2[r * no * no + o12];
    if (gout)
      gout[q] = s;
    else
      out[q] = s;
  }
  __syncthreads();
}

// row stride of the shared derivative matrix: odd in doubles, so the rows
// that neighbouring threads read start on different banks
__host__ __device__ constexpr int conv_dstride(int m) { return m | 1; }

// NC, MC > 0: the orders n, m at compile time (every contraction unrolled);
// 0: the runtime n, m (any dealiasing order a caller sets up)
template <int NC, int MC>
__global__ void __launch_bounds__(512, 2) k_convection(int nel, int n_rt, int m_rt,
                                                   const double* __restrict__ u,
                                                   const double* __restrict__ v,
                                                   double* __restrict__ udv,
                                                   const double* __restrict__ tinv,
                                                   const double* __restrict__ bj,
                                                   const double* __restrict__ Dm,
                                                   const double* __restrict__ J,
                                                   double* __restrict__ gscr) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = NC > 0 ? NC : n_rt, m = MC > 0 ? MC : m_rt;
  const int ds_ = conv_dstride(m);
  const int nt = n * n * n, mt = m * m * m;
  const int tmax = n * m * m > n * n * m ? n * m * m : n * n * m;
  double* sD = reinterpret_cast<double*>(smem_raw);   // D[i][l] at i * ds_ + l
  double* sJ = sD + m * ds_;                  // J[i*n + p] = l_p^n(x_i^m)
  double* t1 = sJ + m * n;
  double* t2 = t1 + tmax;
  double* stage = t2 + tmax;                  // nt
  double* ui = gscr ? gscr + (size_t)blockIdx.x * 5 * mt : stage + nt;   // 3 x mt
  double* vc = ui + 3 * mt;                   // advected component c
  double* sk = vc + mt;                       // its skew-symmetric term
  const size_t nptsn = (size_t)nel * nt, nptsm = (size_t)nel * mt;
  for (int q = threadIdx.x; q < m * m; q += blockDim.x) sD[(q / m) * ds_ + q % m] = Dm[q];
  for (int q = threadIdx.x; q < m * n; q += blockDim.x) sJ[q] = J[q];
  for (size_t e = blockIdx.x; e < (size_t)nel; e += gridDim.x) {
    // 1. the advecting field on the dealiasing grid
    for (int f = 0; f < 3; ++f) {
      const double* src = u + (size_t)f * nptsn + e * nt;
      __syncthreads();
      for (int q = threadIdx.x; q < nt; q += blockDim.x) stage[q] = src[q];
      __syncthreads();
      block_tensor3<NC, MC>(n, m, sJ, false, stage, t1, t2, ui + f * mt, nullptr);
    }
    // 2. one advected component at a time (half the shared memory of
    // holding all three: two blocks per SM): interpolate, convective and
    // conservative forms at every dealiasing point, weak projection back
    for (int c = 0; c < 3; ++c) {
      const double* src = v + (size_t)c * nptsn + e * nt;
      __syncthreads();
      for (int q = threadIdx.x; q < nt; q += blockDim.x) stage[q] = src[q];
      __syncthreads();
      block_tensor3<NC, MC>(n, m, sJ, false, stage, t1, t2, vc, nullptr);
      for (int q = threadIdx.x; q < mt; q += blockDim.x) {
        const int i = q % m, j = (q / m) % m, k = q / (m * m);
        const size_t g = e * mt + q;
        double t[3][3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int b = 0; b < 3; ++b) t[a][b] = __ldg(tinv + (size_t)(3 * a + b) * nptsm + g);
        const double w = __ldg(bj + g);
        const double* Di = sD + i * ds_;
        const double* Dj = sD + j * ds_;
        const double* Dk = sD + k * ds_;
        const int rbase = (k * m + j) * m, sbase = k * m * m + i, tbase = j * m + i;
        // convective: d v_c / d r_b; conservative: d_r(u_x v_c), d_s(u_y v_c),
        // d_t(u_z v_c) -- one pass over l, each matrix entry and each v_c
        // value loaded once for both (every sum still runs over l in order)
        double dr = 0, ds = 0, dt = 0, er = 0, es = 0, et = 0;
#pragma unroll
        for (int l = 0; l < (MC > 0 ? MC : m); ++l) {
          const double di = Di[l], dj = Dj[l], dk = Dk[l];
          const double vr = vc[rbase + l], vs = vc[sbase + l * m], vt = vc[tbase + l * m * m];
          dr += di * vr;
          ds += dj * vs;
          dt += dk * vt;
          er += di * (ui[rbase + l] * vr);
          es += dj * (ui[mt + sbase + l * m] * vs);
          et += dk * (ui[2 * mt + tbase + l * m * m] * vt);
        }
        // convective form: grad through tinv, dotted with u
        double d[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          double s = t[a][0] * dr;
          s = t[a][1] * ds + s;
          s = t[a][2] * dt + s;
          d[a] = s;
        }
        double cv = ui[q] * d[0];
        cv = ui[mt + q] * d[1] + cv;
        cv = ui[2 * mt + q] * d[2] + cv;
        cv = cv * w;
        // conservative form through tinv
        double cs = 0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          double s = t[a][0] * er;
          s = t[a][1] * es + s;
          s = t[a][2] * et + s;
          cs += s;
        }
        cs = cs * w;
        sk[q] = 0.5 * cv + 0.5 * cs;
      }
      __syncthreads();
      block_tensor3<MC, NC>(m, n, sJ, true, sk, t1, t2, nullptr,
                            udv + (size_t)c * nptsn + e * nt);
    }
    __syncthreads();
  }
}

}  // namespace dev

static size_t convection_smem(int n, int m, bool fields) {
  const size_t nt = (size_t)n * n * n, mt = (size_t)m * m * m;
  const size_t tmax = std::max((size_t)n * m * m, (size_t)n * n * m);
  return (m * dev::conv_dstride(m) + m * n + 2 * tmax + nt + (fields ? 5 * mt : 0)) *
         sizeof(double);
}

// one instantiation per order the library builds itself (m = 3n/2), the
// runtime-order kernel for any other dealiasing order
using ConvKernel = void (*)(int, int, int, const double*, const double*, double*,
                            const double*, const double*, const double*, const double*,
                            double*);
static ConvKernel conv_kernel(int n, int m) {
  if (m == (3 * n) / 2) switch (n) {
#define SSG_CONVN(NV) \
  case NV:            \
    return dev::k_convection<NV, (3 * NV) / 2>;
      SSG_CONVN(2) SSG_CONVN(3) SSG_CONVN(4) SSG_CONVN(5) SSG_CONVN(6) SSG_CONVN(7)
      SSG_CONVN(8) SSG_CONVN(9) SSG_CONVN(10) SSG_CONVN(11) SSG_CONVN(12)
#undef SSG_CONVN
      default: break;
    }
  return dev::k_convection<0, 0>;
}

static constexpr size_t kConvSmemMax = 220 * 1024;

size_t convection_scratch_doubles(int n, int m) {
  if (convection_smem(n, m, true) <= kConvSmemMax) return 0;
  return (size_t)kConvScratchBlocks * 5 * m * m * m;
}

cudaError_t run_convection(cudaStream_t s, int nel, int n, int m, const double* u,
                           const double* v, double* udv, const double* tinv,
                           const double* bj, const double* Dm, const double* J,
                           double* scratch) {
  const bool in_smem = convection_smem(n, m, true) <= kConvSmemMax;
  if (!in_smem && !scratch) return cudaErrorInvalidValue;
  const size_t smem = convection_smem(n, m, in_smem);
  if (smem > kConvSmemMax) return cudaErrorInvalidValue;
  const ConvKernel kern = conv_kernel(n, m);
  // the dynamic shared-memory limit, once per kernel variant
  static std::vector<ConvKernel> attr;
  if (std::find(attr.begin(), attr.end(), kern) == attr.end()) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kConvSmemMax);
    if (e != cudaSuccess) return e;
    attr.push_back(kern);
  }
  if (nel <= 0) return cudaSuccess;
  const int grid = in_smem ? nel : std::min(nel, kConvScratchBlocks);
  count_launch();
  kern<<<grid, 512, smem, s>>>(nel, n, m, u, v, udv, tinv, bj, Dm, J,
                               in_smem ? nullptr : scratch);
  return cudaGetLastError();
}

}  // namespace ssg
