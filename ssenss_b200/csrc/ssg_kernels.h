// Launch interface of the device kernels (kernels.cu) used by the solver.
#pragma once

#include <cuda_runtime.h>
#include <atomic>
#include <cstddef>
#include <cstdint>

namespace ssg {

enum OpCode {
  OP_NONE = 0,
  OP_CG_INIT_C,     // c = (w.z)/nunique (pressure) else 0
  OP_CG_INIT_RDZ,   // rdz = (r w).p, reset iteration counters
  OP_CG_ALPHA,      // alpha = rdz / (p w).ap
  OP_CG_BETA,       // nullspace constant, beta, err, done flag
  OP_NULL_C,        // c = (w.x)/nunique
  OP_FCG_BETA,      // beta_k = (z w).ap_k / pap_k
  OP_FCG_ALPHA,     // pap_0, alpha = (p0 w).r / pap_0
  OP_FCG_ERR,       // err, iteration count, done flag
  OP_ERR0,          // initial residual norm
  OP_STORE_PAP,     // pap = sum (first CG iteration: rdz comes next)
  OP_CG_INIT_RDZ_ALPHA   // OP_CG_INIT_RDZ, then alpha = rdz / pap
};

// slots of one solver frame (doubles)
enum {
  F_RDZ = 0, F_ALPHA = 1, F_BETA = 2, F_C = 3, F_ERR = 4, F_ITER = 5,
  F_DONE = 6, F_PAP = 7, F_ERR0 = 8,
  F_FBETA = 16,     // 10 slots
  F_FPAP = 32,      // 10 slots
  F_SIZE = 48
};

struct ScalarOp {
  int code = OP_NONE;
  int pressure = 0;
  double nunique = 1.0;
  double eps = 0.0;
  int max_iter = 0;
  double* frame = nullptr;
  double* hist = nullptr;   // device history buffer (optional)
  int hist_cap = 0;
  int m = 0;
  int pap_idx[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  const double* stop = nullptr;   // skip when *stop != 0 (finished solve)
  double* sums = nullptr;         // raw reduced sums (16 doubles)
  unsigned* counter = nullptr;    // last-block counter; null: partials only
};

// up to 10 vectors passed by value to a kernel (capturable: no upload)
struct PtrList {
  const void* p[10] = {nullptr, nullptr, nullptr, nullptr, nullptr,
                       nullptr, nullptr, nullptr, nullptr, nullptr};
};

// DSS epilogue modes (kernels.cu); DSS_CGUPD: the gathered ap feeds the CG
// update x += alpha p, r -= alpha ap, z = dinv r with its four partial sums;
// DSS_SCALE: out = DSS * y pointwise (FP64 only: the inverse mass product)
enum { DSS_PLAIN = 0, DSS_DOT = 1, DSS_RESID = 2, DSS_AVG = 3, DSS_DOT2 = 4, DSS_CGUPD = 5,
       DSS_SCALE = 6 };

// vectors of the DSS_CGUPD epilogue (storage type of the level)
struct DssCg {
  void* x = nullptr;
  const void* p = nullptr;
  void* r = nullptr;
  const void* dinv = nullptr;
  void* z = nullptr;
  const double* alpha = nullptr;
};

// CG direction update fused into the operator: p = (beta p + (z - c)) .* mask
struct PUpdateArgs {
  const void* z = nullptr;
  const double* beta = nullptr;
  const double* c = nullptr;
  const double* mask = nullptr;
  const double* stop = nullptr;
  int first = 0;
  // set: the operator also reduces p . (A p) (unweighted; for a continuous p
  // this is the weighted (p w).DSS(A p)) and applies *dot to the sum
  const ScalarOp* dot = nullptr;
  double* part = nullptr;
};

// kernel launches of this library: process-wide, and per host thread (the
// per-thread count tells a stream capture how many launches it recorded)
extern std::atomic<unsigned long long> g_launches;
extern thread_local unsigned long long t_launches;
inline void count_launch() {
  ++g_launches;
  ++t_launches;
}

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) for a kernel, once per
// device (the attribute belongs to the device's context) and again only when
// a larger size is asked; safe from several host threads (a race at worst
// sets the same attribute twice).  One object per kernel, as a static.
struct SmemAttr {
  std::atomic<int> bytes[64] = {};
  cudaError_t ensure(const void* func, size_t need) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (bytes[dev].load(std::memory_order_acquire) >= (int)need) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need);
    if (e == cudaSuccess) {
      int cur = bytes[dev].load(std::memory_order_relaxed);
      while (cur < (int)need &&
             !bytes[dev].compare_exchange_weak(cur, (int)need, std::memory_order_release))
        ;
    }
    return e;
  }
};

int vec_blocks(size_t npts);
// elements-per-block value of the operator launch that selects the line-form
// kernel (k_axl, a fixed number of elements per block) for orders other
// than 8; 1, 2, 4, ... select the plane-form kernel k_ax with that many
// elements per block; 0 asks for the order's default (ax_epb)
constexpr int kAxLine = -1;
int ax_epb(int n);
int ax_epb_max(int n);
int dss_grid(int n, int nel);
// autotuned launch shapes (0 = default rule), indexed by order n; atomics:
// the tuner may run while other host threads launch
extern std::atomic<int> g_tune_ax_epb[];
extern std::atomic<int> g_tune_dss_bps[];
extern std::atomic<int> g_tune_vec_bps;
// untuned vector-kernel blocks per SM: the CG update's residency (3 x 256
// threads at <= 85 registers), so its grid is one full wave
constexpr int kVecBpsDefault = 3;
namespace dev { struct PUpdate; }
cudaError_t run_ax8_dmma(cudaStream_t s, int nel, bool helm, bool fp32, void* u, void* au,
                         const void* gf, size_t npts, const double* bj, const double* D,
                         const double* S, double lambda, const dev::PUpdate* pu,
                         const ScalarOp* dop);

cudaError_t run_ax(cudaStream_t s, int n, int nel, int epb, bool helm, bool fp32,
                   const void* in, void* out, const void* gf, size_t npts,
                   const double* bj, const double* D, const double* S, double lambda,
                   const PUpdateArgs* pua);
// ints before the edge/corner records of a DSS map: one gather word per
// local point, rounded up to 16 bytes
inline __host__ __device__ constexpr size_t dss_map_records_offset(size_t npts) {
  return (npts + 3) / 4 * 4;
}
// ec_tab: the DSS map of order n (dss_map_table); nb26: the mesh's 26
// neighbour ids per element when every face, edge and corner is paired with
// the opposite one of its neighbour (the line-run kernel, no per-node
// map read), else null (the gather-word kernel on ec_tab).  Both give the
// same sums in the same order.
cudaError_t run_dss(cudaStream_t s, int mode, bool fp32, int n, int nel, const void* in,
                    void* out, const int* nb26, const int* ec_tab, const double* mask,
                    const void* y, const void* y2, double* part, const double* stop = nullptr,
                    const ScalarOp* op = nullptr, const DssCg* cg = nullptr);
// DSS of three FP64 fields `stride` apart (a vector field's components) in
// one launch, out-of-place; scale: then times y pointwise (the inverse mass)
cudaError_t run_dss3(cudaStream_t s, bool scale, int n, int nel, const double* in, double* out,
                     size_t stride, const int* nb26, const int* ec_tab, const double* y);
cudaError_t run_tensor3(cudaStream_t s, bool fp32, bool add, int nel, int ni, int no,
                        const double* A, const void* in, void* out);
cudaError_t run_cg_update(cudaStream_t s, bool fp32, size_t npts, const double* alpha,
                          void* x, const void* p, void* r, const void* ap, const void* dinv,
                          const uint8_t* mult, void* z, double* part, int nblk,
                          const double* stop = nullptr, const ScalarOp* op = nullptr);
cudaError_t run_jacobi(cudaStream_t s, bool fp32, size_t npts, const void* r, const void* dinv,
                       const uint8_t* mult, void* z, double* part, int nblk,
                       const ScalarOp* op = nullptr);
cudaError_t run_dots(cudaStream_t s, bool fp32, size_t npts, const void* x, const PtrList& ys,
                     int K, const uint8_t* mult, double* part, int nblk,
                     const ScalarOp* op = nullptr);
cudaError_t run_wsum(cudaStream_t s, bool fp32, size_t npts, const void* x,
                     const uint8_t* mult, double* part, int nblk,
                     const ScalarOp* op = nullptr);
cudaError_t run_combine(cudaStream_t s, size_t npts, double* x, const PtrList& ys,
                        const double* coef, int K, double sign);
cudaError_t run_fcg_update(cudaStream_t s, size_t npts, const double* alpha, double* u,
                           const double* p, double* r, const double* ap, const uint8_t* mult,
                           double* part, int nblk, const ScalarOp* op = nullptr);
cudaError_t run_add_const(cudaStream_t s, bool fp32, size_t npts, void* x, const double* a,
                          int neg);
cudaError_t run_convert(cudaStream_t s, size_t npts, const void* in, bool in32, void* out,
                        bool out32);
cudaError_t run_mul(cudaStream_t s, bool fp32, size_t npts, void* x, const double* y);
// Helmholtz diagonal: out = kd + (lam rho[q mod nt]) det; then x = 1 / x
cudaError_t run_helm_diag(cudaStream_t s, size_t npts, size_t nt, const double* kd,
                          const double* rho, const double* det, double lam, double* out);
cudaError_t run_recip(cudaStream_t s, size_t npts, double* x);
cudaError_t run_reduce(cudaStream_t s, const double* part, int nblk, int nq, double* sums,
                       const ScalarOp& op);
// post-smoother CG-Jacobi of a small level (n = 4) in one cooperative
// launch (coarse.cu): same arithmetic per point as cg_solve's kernels
struct LevelCgRun {
  int nel = 0;
  const void* f = nullptr;
  void *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *aploc = nullptr,
       *ap = nullptr;
  const void* gf = nullptr;
  const double* D = nullptr;
  const void* dinv = nullptr;
  const uint8_t* mult = nullptr;
  const int* pairs = nullptr;
  double nunique = 1.0, eps = 0.0;
  int max_iter = 0;
  double* part = nullptr;
  size_t part_cap = 0;
};
cudaError_t run_level_cg(cudaStream_t s, int device, int n, bool fp32, const LevelCgRun& L);
// whole CG-Jacobi solve of an n = 2 level in one cooperative launch
// (coarse.cu); it stops at sqrt((r.r)_w) <= eps, or <= rel times the first
// residual when rel > 0
cudaError_t run_coarse_cg(cudaStream_t s, int device, int nel, const double* f, double* x,
                          double* r, double* z, double* p, double* aploc, double* ap,
                          const double* gf, const double* D, const double* dinv,
                          const uint8_t* mult, const int* pairs, double nunique, double eps, double rel,
                          int max_iter, double* part, size_t part_cap, double* frame);
// dealiased skew-symmetric convection of 3-component fields (convection.cu)
// of the nel elements e0 .. e0+nel-1 of a mesh of nel_fac elements (fields
// hold the nel elements, the factors tinv and bj all nel_fac); for m^3
// fields beyond shared memory, scratch holds convection_scratch_doubles(n, m)
// doubles (0: none needed)
constexpr int kConvScratchBlocks = 296;
size_t convection_scratch_doubles(int n, int m);
// W: 9 x nel_fac x m^3 in the order (b, a), W[3b + a] = rho J tinv[a][b] / 2;
// Dh, Jh: host copies of the m-point derivative matrix D[i*m + l] and the
// interpolation matrix J[i*n + p] (carried in the kernel's parameters);
// Dd, Jd: the same on the device (runtime-order kernel)
cudaError_t run_convection(cudaStream_t s, int nel, int e0, int nel_fac, int n, int m,
                           const double* u, const double* v, double* udv, const double* W,
                           const double* Dh, const double* Jh, const double* Dd,
                           const double* Jd, double* scratch);
// Convection at n = 8, m = 12 on the FP64 tensor cores (conv_dmma.cu): the
// self-convection kernel when u == v, else the general one; run_convection
// takes them at that order
bool convection_dmma_applies(int n, int m);
cudaError_t run_convection_dmma(cudaStream_t s, int nel, int e0, int nel_fac, const double* u,
                                const double* v, double* udv, const double* W,
                                const double* Dh, const double* Jh);
// Stokes operators of the time step, one element per block (stokes.cu):
// which 0 = the double curl of in (3 fields) into out (3 fields); 1 = the
// pressure right-hand side of in = u~ (3 fields) and g (3 fields, surface
// terms on the wall faces) into out (1 field), x = -dens / dt; 2 = the
// velocity right-hand sides of in = u~ and g = p (1 field, surface terms on
// the other faces) into out (3 fields), x = 1 / (dt visc), y = -1 / (visc
// dens).  tinv: 9 x npts; rho: n^3; det: npts; D: n x n; bc: wall face bits
// per element; sw: surface weights (nel x 3 x 6 x n^2)
cudaError_t run_stokes(cudaStream_t s, int which, int n, int nel, const double* tinv,
                       const double* rho, const double* det, const double* D, const int* bc,
                       const double* sw, size_t npts, const double* in, const double* g,
                       double* out, double x, double y);
// Lagrangian particle advance to time t (particles.cu); passes: device int
// that receives the largest per-particle pass count (atomicMax, caller zeroes).
// order (np ints) and bucket (2 (nel + 1) ints): scratch of the element-order
// sort the particles are processed in; order == nullptr keeps array order.
cudaError_t run_particles(cudaStream_t s, int n, int nel, size_t npts, const double* x,
                          const double* ur, const double* jac, const double* tinv,
                          const int* neigh, double t, double dt, size_t np, double* state,
                          int* ints, int* passes, int* order, int* bucket);

}  // namespace ssg
