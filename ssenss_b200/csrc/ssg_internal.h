// Internal declarations of libssenss_b200 (not installed).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "ssenss_b200.h"

#define SSG_MAXLEV 8
#define SSG_MAXN 18

namespace ssg {

// ---------------------------------------------------------------------------
// host-side discretisation (setup.cpp)
// ---------------------------------------------------------------------------
struct HostLevel {
  int n = 0;
  size_t nt = 0;                        // n^3
  std::vector<double> x, w;             // GLL points, weights
  std::vector<double> D, S;             // D[i*n+m] = l_m'(x_i); S = SVV variant
  std::vector<double> jf;               // from the finer level: jf[i*n+p] = l_p(x_i^fine)
  std::vector<double> g[6];             // G11 G12 G13 G22 G23 G33 (unscaled)
  std::vector<double> det;              // det J
  std::vector<double> grid[3];
  std::vector<double> jac[9];           // J[a][b] = dx_a/dr_b (level 0, conv)
  std::vector<double> tinv[9];          // tinv[a][b] = dr_b/dx_a
};

struct HostMesh {
  int n = 0, nel = 0, nlev = 0;
  std::vector<int> neigh;               // nel x 26
  std::vector<int> pairs;               // nel x 26 x 2: (element, matched index)
  std::vector<int> bc;                  // Dirichlet face bits per element
  HostLevel lev[SSG_MAXLEV];
  HostLevel conv;                       // dealiasing grid (m = 3n/2)
  std::vector<double> jconv;            // jconv[i*n+p] = l_p^n(x_i^m)
  bool has_conv = false;
  bool has_particle_geom = false;
  std::vector<double> ppoints;          // GLL points of the particle walk (empty: lev[0].x)
};

// Run f(e0, e1) over element ranges on up to 32 host threads.  Every
// element is computed by one thread with the same arithmetic as a serial
// loop, so the results do not depend on the thread count.
template <class F>
inline void parallel_elements(int nel, F&& f) {
  unsigned hw = std::thread::hardware_concurrency();
  int nth = (int)std::min<unsigned>(hw ? hw : 1, 32u);
  nth = std::max(1, std::min(nth, nel / 8));
  if (nth <= 1) {
    f(0, nel);
    return;
  }
  std::vector<std::thread> th;
  const int chunk = (nel + nth - 1) / nth;
  for (int t = 0; t < nth; ++t) {
    const int e0 = t * chunk, e1 = std::min(nel, e0 + chunk);
    if (e0 >= e1) break;
    th.emplace_back([&f, e0, e1] { f(e0, e1); });
  }
  for (auto& x : th) x.join();
}

// Position of natural node q = (k n + j) n + i of an n = 8 element in the
// tensor-core operator's fragment order: plane k, lane 4i + j/2, slot j%2
// (the lane that owns the point, ax8.cu), so a lane's two points of a plane
// are adjacent.
inline int ax8_fragment_index(int q) {
  const int k = q >> 6, j = (q >> 3) & 7, i = q & 7;
  return k * 64 + (4 * i + (j >> 1)) * 2 + (j & 1);
}

int level_orders(int n, int* orders);
void gll_basis(int n, double* x, double* w);
void deriv_matrix(int n, const double* x, double* D);
void svv_deriv_matrix(int n, const double* x, const double* w, int msvv, double c,
                      double* S);
void interp_matrix(int nto, const double* xto, int nfrom, const double* xfrom, double* J);
ssg_status build_mesh(HostMesh& m, int n, int nel, const double* vertices,
                      const int* neigh, std::string& err, unsigned opts = 0,
                      int svvn = -1, double svva = 0.0);
ssg_status build_pairs(HostMesh& m, std::string& err, bool opposite = false);
void stiffness_diagonal(const HostLevel& L, int nel, double* out);
void host_dss(const HostMesh& m, int n, double* u);
// DSS map of one level (one int array):
//   [0, npts)         one gather word per local point, natural order: the
//                     index (element * n^3 + node) of the face neighbour's
//                     copy of a face-interior node; -(2 + (r << 1 | c)) for
//                     an edge (c = 0) or corner (c = 1) node whose source
//                     record starts r int4 into its element's records; -1
//                     for an interior node or a face without a neighbour
//   then, from dss_map_records_offset(npts), per element the ordered source
//   lists of the edge nodes (12 (n-2) records of 4 ints: 3 sources + pad)
//   and corner nodes (8 records of 8 ints: 7 sources + pad); a source is
//   element * n^3 + node, -1 where the node has none.
void dss_map_table(const HostMesh& m, int n, std::vector<int>& tab);

// ---------------------------------------------------------------------------
// device-side level
// ---------------------------------------------------------------------------
struct DevLevel {
  int n = 0;
  size_t nt = 0, npts = 0;
  double* gf = nullptr;        // 6 x npts: G_ab * rho * J
  double* bj = nullptr;        // rho * J
  double* kdiag = nullptr;     // element-local stiffness diagonal
  double* dinv_p = nullptr;    // Poisson Jacobi inverse
  double* dinv_h = nullptr;    // Helmholtz Jacobi inverse (for lambda_h)
  double* det = nullptr;       // det J (level 0: the Helmholtz diagonal's lambda term)
  double* rho = nullptr;       // GLL weight products rho_ijk (n^3, level 0)
  uint8_t* mult = nullptr;     // multiplicity (1 + DSS contributions)
  int* dss_ec = nullptr;       // DSS map of this order (dss_map_table)
  double* mask = nullptr;      // Dirichlet mask (null without walls)
  double* D = nullptr;         // n*n
  double* S = nullptr;         // n*n
  double* Ar = nullptr;        // restriction into this level: n x n_finer
  double* Ap = nullptr;        // prolongation from this level: n_finer x n
  float* gf32 = nullptr;       // FP32 copies for the mixed-precision V-cycle
  float* dinv_p32 = nullptr;
  double nunique = 0.0;        // sum of 1/multiplicity
  double lambda_h = -1.0;      // lambda the Helmholtz diagonal holds
};

struct Workspace;

void free_workspace(Workspace* w);

// The level-0 data a segmented Helmholtz solve reads (batch.cu): a context's
// own level, or the serving loop's assembly of several contexts' levels.
struct SegLevel {
  int n = 0, nel = 0;
  size_t nt = 0, npts = 0;
  const double *gf = nullptr, *bj = nullptr, *kdiag = nullptr, *rho = nullptr, *det = nullptr;
  const double *mask = nullptr, *D = nullptr, *S = nullptr;
  const uint8_t* mult = nullptr;
  const int* dss = nullptr;    // DSS map (dss_map_table layout)
};

// Device scratch of segmented solves, grown on demand and reused.
struct SegScratch {
  int *chunk_seg = nullptr, *chunk_n = nullptr, *seg_chunk0 = nullptr, *active = nullptr;
  size_t* chunk_lo = nullptr;
  double *part = nullptr, *sc = nullptr;
  double *bj_s = nullptr, *dinv_s = nullptr, *x = nullptr, *r = nullptr, *z = nullptr;
  double *p = nullptr, *ap = nullptr, *aploc = nullptr, *f = nullptr;
  size_t cap_chunks = 0, cap_segs = 0, cap_points = 0;
};
void seg_scratch_free(SegScratch& W);

}  // namespace ssg

struct ssg_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;
  double dt = 1.0, visc = 1.0, dens = 1.0;
  int precision = SSG_PRECISION_FP64;
  bool graphs = true;
  bool ready = false;
  unsigned setup_opts = 0;      // SSG_SETUP_* flags of the next ssg_setup_mesh
  int svvn = -1;                // SVV cut-off mode of the next set-up (< 0: 2n/3)
  double svva = 0.0;            // SVV amplitude of the next set-up
  size_t dev_bytes = 0;         // device memory this context holds
  const volatile int* cancel = nullptr;   // nonzero: stop the running solve
  double deadline = 0.0;        // steady-clock seconds; 0 = none
  int n = 0, nel = 0, nlev = 0;
  int orders[SSG_MAXLEV] = {0};
  ssg::HostMesh host;
  int* d_pairs = nullptr;       // nel x 26 x int2
  // nel x 26 neighbour ids when every pairing is the opposite face, edge
  // or corner (the line-run DSS), else null (the gather-word DSS)
  int* d_nbreg = nullptr;
  bool has_walls = false;
  ssg::DevLevel lev[SSG_MAXLEV];
  double* inv_mass = nullptr;   // level 0
  // dealiasing grid
  int m = 0;
  double* conv_w = nullptr;     // 9 x nel x m^3: W[3b + a] = rho J tinv[a][b] / 2
  double* conv_D = nullptr;     // m*m
  double* conv_J = nullptr;     // m*n, jconv[i*n+p]
  double* conv_scratch = nullptr;  // interpolated fields when m^3 exceeds shared memory
  // particles
  double* p_jac = nullptr;      // 9 x npts (level 0)
  double* p_tinv = nullptr;     // 9 x npts
  double* p_ur = nullptr;       // 3 x 3 x npts
  double* p_x = nullptr;        // GLL points of level 0
  int* d_neigh = nullptr;       // nel x 26 face/edge/corner neighbours
  int* d_passes = nullptr;      // particle pass count
  bool has_ur = false;          // particle velocity snapshots set
  double* p_state = nullptr;    // staging of host particle arrays
  int* p_ints = nullptr;
  size_t p_cap = 0;
  int* p_order = nullptr;       // element-order sort of the particles:
  int* p_bucket = nullptr;      //   permutation (p_order_cap) and 2 (nel + 1) counters
  size_t p_order_cap = 0;
  // reductions / scalars
  double* d_part = nullptr;     // block partial sums
  size_t part_cap = 0;
  double* d_sums = nullptr;     // 16 raw sums
  unsigned* d_counter = nullptr;  // last-block counter of the fused reductions
  double* d_sc = nullptr;       // solver frames
  double* h_pin = nullptr;      // pinned host scalars
  // staging for host arguments
  double* d_stage[4] = {nullptr, nullptr, nullptr, nullptr};
  size_t stage_cap = 0;
  ssg::Workspace* ws = nullptr;
  ssg::SegScratch* seg = nullptr;   // segmented Helmholtz solves (batch.cu)
  // convection sub-steps (timestep.cu): velocity history (oldest first,
  // 3 levels x 3 components x npts) with its time and step, and scratch
  double* vhist = nullptr;
  double vhist_t = 0.0, vhist_dt = 0.0;
  double* rk_scratch = nullptr;
  // resident time step (flow.cu): one allocation holding the velocity,
  // convection and double-curl histories (3 fields each), the pressure
  // history, the body force, u~, two scratch triples and the wall values;
  // history slots newest first, rotated by the time shifts
  double* flow_buf = nullptr;
  double* fu[3] = {nullptr, nullptr, nullptr};
  double* fconv[3] = {nullptr, nullptr, nullptr};
  double* frot[3] = {nullptr, nullptr, nullptr};
  double* fp[3] = {nullptr, nullptr, nullptr};
  double* ff = nullptr;
  double* fut = nullptr;
  double* fa = nullptr;
  double* fb = nullptr;
  double* fbc = nullptr;        // walls: u (3 fields), then du/dt (3 fields)
  double* flow_sw = nullptr;    // surface weights (nel x 3 x 6 x n^2)
  int* flow_bc = nullptr;       // wall face bits per element
  double flow_t = 0.0;
  bool flow_ready = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace ssg {

ssg_status fail(ssg_context* c, ssg_status s, const std::string& msg);
ssg_status cuda_fail(ssg_context* c, cudaError_t e, const char* what);
#define SSG_CUDA(c, call)                                           \
  do {                                                              \
    cudaError_t _e = (call);                                        \
    if (_e != cudaSuccess) return ::ssg::cuda_fail((c), _e, #call); \
  } while (0)
#define SSG_TRY(call)                    \
  do {                                   \
    ssg_status _s = (call);              \
    if (_s != SSG_OK) return _s;         \
  } while (0)

bool is_device_ptr(const void* p);

enum Frame { FR_LEVEL0 = 0, FR_HELM = 8, FR_FCG = 9, FR_MISC = 10, FR_COUNT = 12 };

// batch.cu: segments seg_first[s] .. seg_first[s+1]-1 of L, each its own
// Jacobi-CG Helmholtz solve (lambda[s], eps[s]) sharing every operator and
// DSS launch; f, u host or device; on c's stream
ssg_status seg_solve(ssg_context* c, const SegLevel& L, SegScratch& W, int nseg,
                     const int* seg_first, const double* lambda, const double* f, double* u,
                     const double* eps, int max_iter, ssg_solve_info* info);

// ints per element of the edge/corner records of a DSS map of order n, and
// the copy of one context's map into a concatenation's (points shifted by P,
// records placed at element offset E; npts_dst: the concatenation's points)
size_t dss_record_ints(int n);
cudaError_t run_dss_map_shift(cudaStream_t s, const int* src, int n, int nel, int* dst,
                              size_t P, size_t npts_dst, int E);

// solver.cu
ssg_status ensure_workspace(ssg_context* c);
double* workspace_scratch(ssg_context* c);   // one level-0 FP64 vector
ssg_status op_apply(ssg_context* c, int level, int var, bool fp32, const void* in,
                    void* out, bool global);
ssg_status cg_solve(ssg_context* c, int level, int var, bool fp32, void* f, void* x,
                    double eps, int max_iter, int frame, double* hist, int hist_cap,
                    bool sync_each);
ssg_status mg_apply(ssg_context* c, const double* r, double* z, double eps);
ssg_status fcg_solve(ssg_context* c, const double* f, double* u, double eps, int max_iter,
                     ssg_solve_info* info);
ssg_status helmholtz_diag_update(ssg_context* c);
// timestep.cu: the convection sub-steps of integrate_convection_rk4 on
// device fields (du, 3 fields, in/out; the velocity history oldest first,
// at time th with step dth), and the scratch they use
ssg_status ensure_rk_scratch(ssg_context* c);
ssg_status convection_rk4(ssg_context* c, double* du, double t0, double t, double dt,
                          double beta, const double* uoo, const double* uo, const double* uc,
                          double th, double dth);
// drop captured CUDA graphs (launch shapes or buffers changed)
void invalidate_graphs(ssg_context* c);

}  // namespace ssg
