// Host-side discretisation set-up: what read_grid, connect_elements and
// initialise_preconditioners compute before the first solve
// (src/dataio.c:197-227,407-452, src/init.c:38-130, src/precon.c:58-183,
// 336-413).  Runs once per mesh; the results are uploaded to the device.
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "ssg_internal.h"
#include "ssg_kernels.h"

namespace ssg {


int level_orders(int n, int* orders) {
  // nmg[i] = max(2, (n-1)/2^i + 1), stopping at 2 (src/precon.c:62-69)
  int nl = 0;
  for (int i = 0; i < SSG_MAXLEV; ++i) {
    int m = (n - 1) / (1 << i) + 1;
    if (m < 2) m = 2;
    orders[i] = m;
    nl = i + 1;
    if (m == 2) break;
  }
  return nl;
}

static void legendre_pair(int N, double x, double* pn, double* pnm1) {
  double p0 = 1.0, p1 = x;
  if (N == 0) {
    *pn = 1.0;
    *pnm1 = 0.0;
    return;
  }
  for (int k = 1; k < N; ++k) {
    const double p2 = ((2.0 * k + 1.0) * x * p1 - k * p0) / (k + 1.0);
    p0 = p1;
    p1 = p2;
  }
  *pn = p1;
  *pnm1 = p0;
}

static double legendre(int N, double x) {
  double a, b;
  legendre_pair(N, x, &a, &b);
  return a;
}

// GLL nodes and weights (src/basis.c:123-158): interior nodes are the roots of
// P_N', found by Newton on (1 - x^2) P_N'(x) from Chebyshev-Gauss-Lobatto
// guesses; w_i = 2 / (N (N+1) P_N(x_i)^2).
void gll_basis(int n, double* x, double* w) {
  const int N = n - 1;
  x[0] = -1.0;
  x[N] = 1.0;
  for (int i = 1; i < N; ++i) {
    double xi = -std::cos(M_PI * i / N);
    for (int it = 0; it < 100; ++it) {
      double pn, pm;
      legendre_pair(N, xi, &pn, &pm);
      const double dpn = N * (xi * pn - pm) / (xi * xi - 1.0);
      const double step = (1.0 - xi * xi) * dpn / (N * (N + 1.0) * pn);
      xi += step;
      if (std::fabs(step) < 1e-16) break;
    }
    x[i] = xi;
  }
  for (int i = 0; i < n; ++i) {
    const double pn = legendre(N, x[i]);
    w[i] = 2.0 / (N * (N + 1.0) * pn * pn);
  }
}

// D[i*n+m] = l_m'(x_i) (src/basis.c:160-177)
void deriv_matrix(int n, const double* x, double* D) {
  const int N = n - 1;
  for (int i = 0; i < n; ++i)
    for (int m = 0; m < n; ++m)
      D[i * n + m] = i == m ? 0.0 : legendre(N, x[i]) / (legendre(N, x[m]) * (x[i] - x[m]));
  D[0] = -(double)n * (double)(n - 1) / 4.0;
  D[n * n - 1] = -D[0];
}

// spectral vanishing viscosity derivative (src/deriv.c:81-112): modal
// filter sqrt(1 + c Q_r) between the discrete Legendre transform and its
// inverse; equals D to rounding when c = 0.
void svv_deriv_matrix(int n, const double* x, const double* w, int msvv, double c,
                      double* S) {
  const int N = n - 1;
  std::vector<double> D(n * n), FD(n * n);
  deriv_matrix(n, x, D.data());
  for (int r = 0; r < n; ++r) {
    const double q =
        r <= msvv ? 0.0 : std::exp(-std::pow((double)(N - r) / (double)(msvv - r), 2));
    const double sig = std::sqrt(1.0 + c * q);
    for (int col = 0; col < n; ++col) {
      double s = 0.0;
      for (int k = 0; k < n; ++k) s += (r + 0.5) * w[k] * legendre(r, x[k]) * D[k * n + col];
      FD[r * n + col] = s * sig;
    }
  }
  for (int i = 0; i < n; ++i)
    for (int col = 0; col < n; ++col) {
      double s = 0.0;
      for (int r = 0; r < n; ++r) s += legendre(r, x[i]) * FD[r * n + col];
      S[i * n + col] = s;
    }
}

static double lagrange(double xt, const double* xf, int p, int nf) {
  double l = 1.0;
  for (int q = 0; q < p; ++q) l *= (xt - xf[q]) / (xf[p] - xf[q]);
  for (int q = p + 1; q < nf; ++q) l *= (xt - xf[q]) / (xf[p] - xf[q]);
  return l;
}

// J[i*nfrom+p] = l_p(xto_i) (src/interpolation.c:115-123)
void interp_matrix(int nto, const double* xto, int nfrom, const double* xfrom, double* J) {
  for (int i = 0; i < nto; ++i)
    for (int p = 0; p < nfrom; ++p) J[i * nfrom + p] = lagrange(xto[i], xfrom, p, nfrom);
}

// out (no^3) = (A x A x A) in (ni^3), stages x, y, z; A[o*ni + q]
static void tensor3(int ni, int no, const double* A, const double* in, double* out) {
  std::vector<double> t1((size_t)no * ni * ni), t2((size_t)no * no * ni);
  for (int kj = 0; kj < ni * ni; ++kj)
    for (int o = 0; o < no; ++o) {
      double s = 0.0;
      for (int q = 0; q < ni; ++q) s += A[o * ni + q] * in[kj * ni + q];
      t1[kj * no + o] = s;
    }
  for (int k = 0; k < ni; ++k)
    for (int o2 = 0; o2 < no; ++o2)
      for (int o1 = 0; o1 < no; ++o1) {
        double s = 0.0;
        for (int q = 0; q < ni; ++q) s += A[o2 * ni + q] * t1[(k * ni + q) * no + o1];
        t2[(k * no + o2) * no + o1] = s;
      }
  for (int o3 = 0; o3 < no; ++o3)
    for (int o12 = 0; o12 < no * no; ++o12) {
      double s = 0.0;
      for (int q = 0; q < ni; ++q) s += A[o3 * ni + q] * t2[q * no * no + o12];
      out[o3 * no * no + o12] = s;
    }
}

static void alloc_level(HostLevel& L, int n, int nel, bool full) {
  L.n = n;
  L.nt = (size_t)n * n * n;
  const size_t len = L.nt * nel;
  std::vector<std::vector<double>*> arrays;
  for (auto& a : L.g) arrays.push_back(&a);
  arrays.push_back(&L.det);
  for (auto& a : L.grid) arrays.push_back(&a);
  if (full) {
    for (auto& a : L.jac) arrays.push_back(&a);
    for (auto& a : L.tinv) arrays.push_back(&a);
  }
  // zero-filled in parallel (one host thread per array)
  std::vector<std::thread> th;
  for (auto* a : arrays) th.emplace_back([a, len] { a->assign(len, 0.0); });
  for (auto& t : th) t.join();
}

// Jacobian from the grid, determinant by first-row cofactors, inverse by
// cofactors / det with the per-point operation order of src/tripalg.c:165-222,
// metric G_ab = sum_j Ji[a][j] Ji[b][j] (src/geometry.c:130-135) and the
// stored transposed inverse (src/geometry.c:112).
static void compute_factors(HostLevel& L, int nel, bool keep_jac) {
  const int n = L.n;
  const size_t nt = L.nt;
  static const int k0[3] = {1, 0, 0}, k1[3] = {2, 2, 1}, k2[3] = {2, 0, 1}, k3[3] = {1, 2, 0};
  static const double sg[3] = {1.0, -1.0, 1.0};
  // one element at a time per thread: its Jacobian in a local buffer, then
  // the per-point algebra
  parallel_elements(nel, [&](int e0, int e1) {
  std::vector<double> jbuf(9 * nt);
  double* jac[9];
  for (int a = 0; a < 9; ++a) jac[a] = jbuf.data() + a * nt;
  for (int e = e0; e < e1; ++e) {
    const size_t o = e * nt;
    for (int a = 0; a < 3; ++a) {
      const double* g = L.grid[a].data() + o;
      for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
          for (int i = 0; i < n; ++i) {
            double sr = 0.0, ss = 0.0, st = 0.0;
            for (int m = 0; m < n; ++m) {
              sr += L.D[i * n + m] * g[(k * n + j) * n + m];
              ss += L.D[j * n + m] * g[(k * n + m) * n + i];
              st += L.D[k * n + m] * g[(m * n + j) * n + i];
            }
            const size_t q = (k * n + j) * n + i;
            jac[3 * a + 0][q] = sr;
            jac[3 * a + 1][q] = ss;
            jac[3 * a + 2][q] = st;
          }
    }
  for (size_t ql = 0; ql < nt; ++ql) {
    const size_t q = o + ql;
    double a[3][3], ai[3][3];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) a[r][c] = jac[3 * r + c][ql];
    double det = 0.0;
    for (int i = 0; i < 3; ++i) {
      const int j = (2 - i) / 2, k = 3 - i - j;
      double t = a[1][j] * a[2][k];
      t = -(a[1][k] * a[2][j]) + t;
      det = i == 0 ? a[0][i] * t : sg[i] * a[0][i] * t + det;
    }
    L.det[q] = det;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        double t = a[k0[j]][k3[i]] * a[k1[j]][k2[i]];
        t = -(a[k0[j]][k2[i]] * a[k1[j]][k3[i]]) + t;
        ai[i][j] = sg[j] * t / det;
      }
    double g[3][3];
    for (int i = 0; i < 3; ++i)
      for (int l = 0; l < 3; ++l) {
        double s = ai[l][0] * ai[i][0];
        s = ai[l][1] * ai[i][1] + s;
        s = ai[l][2] * ai[i][2] + s;
        g[i][l] = s;
      }
    L.g[0][q] = g[0][0];
    L.g[1][q] = g[1][0];
    L.g[2][q] = g[2][0];
    L.g[3][q] = g[1][1];
    L.g[4][q] = g[2][1];
    L.g[5][q] = g[2][2];
    if (keep_jac)
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
          L.jac[3 * r + c][q] = a[r][c];
          L.tinv[3 * r + c][q] = ai[c][r];
        }
  }
  }
  });
}

static void make_basis(HostLevel& L, int n, int msvv, double csvv) {
  L.x.resize(n);
  L.w.resize(n);
  L.D.resize(n * n);
  L.S.resize(n * n);
  gll_basis(n, L.x.data(), L.w.data());
  deriv_matrix(n, L.x.data(), L.D.data());
  svv_deriv_matrix(n, L.x.data(), L.w.data(), msvv, csvv, L.S.data());
}

static void grid_from_vertices(HostLevel& L, int nel, const double* vert) {
  const double xv[2] = {-1.0, 1.0};
  std::vector<double> J(L.n * 2);
  interp_matrix(L.n, L.x.data(), 2, xv, J.data());
  parallel_elements(nel, [&](int e0, int e1) {
    for (int e = e0; e < e1; ++e)
      for (int a = 0; a < 3; ++a)
        tensor3(2, L.n, J.data(), vert + 24 * (size_t)e + 8 * a, L.grid[a].data() + e * L.nt);
  });
}

// Pairing of faces, edges and corners: the neighbour's matching entry is the
// FIRST of its list naming this element (src/init.c:68-130 with
// surfind/edgeind/cornerind, src/init.c:298-320).  With one or two elements
// along a periodic direction that search pairs a face with the neighbour's
// face on the same side (west with west), a defect of the reference the
// drop-in path keeps.  opposite = true pairs every face, edge and corner
// with the geometrically opposite one of the neighbour instead (west with
// east; edge and corner sides all flipped), which is the correct pairing of
// an aligned mesh and the same as the first match wherever every
// direction has three or more elements.
ssg_status build_pairs(HostMesh& m, std::string& err, bool opposite) {
  static const int base[3] = {0, 6, 18}, cnt[3] = {6, 12, 8};
  m.pairs.assign((size_t)m.nel * 52, -1);
  m.bc.assign(m.nel, 0);
  for (int e = 0; e < m.nel; ++e) {
    for (int f = 0; f < 6; ++f)
      if (m.neigh[26 * (size_t)e + f] == -1) m.bc[e] |= 1 << f;
    for (int kind = 0; kind < 3; ++kind)
      for (int j = 0; j < cnt[kind]; ++j) {
        const int slot = base[kind] + j;
        const int nb = m.neigh[26 * (size_t)e + slot];
        if (nb < 0) continue;
        if (nb >= m.nel) {
          err = "neighbour id out of range";
          return SSG_ERR_MESH;
        }
        int found = -1;
        if (opposite) {
          // faces w,e | s,n | b,t: flip the side; edges: both sides of the
          // group (sw,se,nw,ne | bw,be,tw,te | bs,bn,ts,tn); corners: all three
          const int opp = kind == 0 ? (j ^ 1) : (kind == 1 ? (j ^ 3) : (j ^ 7));
          if (m.neigh[26 * (size_t)nb + base[kind] + opp] == e) found = opp;
        } else {
          for (int s = 0; s < cnt[kind]; ++s)
            if (m.neigh[26 * (size_t)nb + base[kind] + s] == e) {
              found = s;
              break;
            }
        }
        if (found < 0) {
          err = "element " + std::to_string(e) + " slot " + std::to_string(slot) +
                ": neighbour " + std::to_string(nb) + " does not name it back";
          return SSG_ERR_MESH;
        }
        m.pairs[2 * (26 * (size_t)e + slot)] = nb;
        m.pairs[2 * (26 * (size_t)e + slot) + 1] = found;
      }
  }
  return SSG_OK;
}

static int face_node(int n, int f, int a, int b) {
  const int m = n - 1;
  switch (f) {
    case 0: return (a * n + b) * n;
    case 1: return (a * n + b) * n + m;
    case 2: return (a * n) * n + b;
    case 3: return (a * n + m) * n + b;
    case 4: return a * n + b;
    default: return (m * n + a) * n + b;
  }
}

static int edge_node(int n, int q, int p) {
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

static int corner_node(int n, int c) {
  const int m = n - 1;
  return (((c >> 2) & 1) * m * n + ((c >> 1) & 1) * m) * n + (c & 1) * m;
}

// DSS on the host (set-up only: diagonals, multiplicities), same order as
// direct_stiffness_summation (src/global.c:241-257).
void host_dss(const HostMesh& m, int n, double* u) {
  const size_t nt = (size_t)n * n * n;
  std::vector<double> pre(u, u + nt * m.nel);
  parallel_elements(m.nel, [&](int e0, int e1) {
  for (int e = e0; e < e1; ++e) {
    double* ue = u + e * nt;
    const int* pr = m.pairs.data() + 52 * (size_t)e;
    for (int f = 0; f < 6; ++f, pr += 2)
      if (pr[0] >= 0)
        for (int p = 0; p < n * n; ++p)
          ue[face_node(n, f, p / n, p % n)] +=
              pre[pr[0] * nt + face_node(n, pr[1], p / n, p % n)];
    for (int q = 0; q < 12; ++q, pr += 2)
      if (pr[0] >= 0)
        for (int p = 0; p < n; ++p)
          ue[edge_node(n, q, p)] += pre[pr[0] * nt + edge_node(n, pr[1], p)];
    for (int c = 0; c < 8; ++c, pr += 2)
      if (pr[0] >= 0) ue[corner_node(n, c)] += pre[pr[0] * nt + corner_node(n, pr[1])];
  }
  });
}

// Ordered DSS sources of one local node (element e, node loc): its
// neighbours' copies in the reference's order -- the x-, y- and z-face
// (w/e, s/n, b/t), the xy-, xz- and yz-edge, the corner -- as
// element * n^3 + node, -1 for none.  Same pairing and order as host_dss.
static void node_sources(const HostMesh& m, int n, int e, int loc, int (&src)[7]) {
  const long long nt = (long long)n * n * n;
  const int M = n - 1;
  const int i = loc % n, j = (loc / n) % n, k = loc / (n * n);
  const int* pr = m.pairs.data() + 52 * (size_t)e;
  for (auto& v : src) v = -1;
  const bool ei = i == 0 || i == M, ej = j == 0 || j == M, ek = k == 0 || k == M;
  auto put = [&](int a, int sl, int node) {
    if (pr[2 * sl] >= 0) src[a] = (int)(pr[2 * sl] * nt + node);
  };
  if (ei) { const int sl = i == M; put(0, sl, face_node(n, pr[2 * sl + 1], k, j)); }
  if (ej) { const int sl = 2 + (j == M); put(1, sl, face_node(n, pr[2 * sl + 1], k, i)); }
  if (ek) { const int sl = 4 + (k == M); put(2, sl, face_node(n, pr[2 * sl + 1], j, i)); }
  if (ei && ej) {
    const int sl = 6 + ((i == M) | ((j == M) << 1));
    put(3, sl, edge_node(n, pr[2 * sl + 1], k));
  }
  if (ek && ei) {
    const int sl = 10 + ((i == M) | ((k == M) << 1));
    put(4, sl, edge_node(n, pr[2 * sl + 1], j));
  }
  if (ek && ej) {
    const int sl = 14 + ((j == M) | ((k == M) << 1));
    put(5, sl, edge_node(n, pr[2 * sl + 1], i));
  }
  if (ei && ej && ek) {
    const int sl = 18 + ((i == M) | ((j == M) << 1) | ((k == M) << 2));
    put(6, sl, corner_node(n, pr[2 * sl + 1]));
  }
}

void dss_map_table(const HostMesh& m, int n, std::vector<int>& tab) {
  const int I = n > 2 ? n - 2 : 0;
  const int nt = n * n * n;
  const size_t npts = (size_t)nt * m.nel;
  const size_t head = dss_map_records_offset(npts);
  const size_t per = (size_t)12 * I * 4 + 8 * 8;
  tab.assign(head + per * m.nel, -1);
  // per order: the record code of every edge/corner node, -1 elsewhere
  std::vector<int> rec(nt, -1);
  for (int q = 0; q < 12; ++q)
    for (int p = 1; p <= I; ++p) rec[edge_node(n, q, p)] = (q * I + p - 1) << 1;
  for (int c = 0; c < 8; ++c) rec[corner_node(n, c)] = ((12 * I + 2 * c) << 1) | 1;
  parallel_elements(m.nel, [&](int e0, int e1) {
  for (int e = e0; e < e1; ++e) {
    // gather words, natural order: the face neighbour's copy, or the
    // edge/corner record, or -1 (interior node, or a face without one)
    int* g = tab.data() + (size_t)e * nt;
    int src[7];
    for (int t = 0; t < nt; ++t) {
      const int i = t % n, j = (t / n) % n, k = t / (n * n);
      const int nb = (i == 0 || i == n - 1) + (j == 0 || j == n - 1) + (k == 0 || k == n - 1);
      if (nb == 1) {
        node_sources(m, n, e, t, src);
        g[t] = src[0] >= 0 ? src[0] : (src[1] >= 0 ? src[1] : src[2]);
      } else if (nb >= 2) {
        g[t] = -(2 + rec[t]);
      }
    }
    // edge / corner records
    int* t = tab.data() + head + per * e;
    for (int q = 0; q < 12; ++q)
      for (int p = 1; p <= I; ++p, t += 4) {
        node_sources(m, n, e, edge_node(n, q, p), src);
        int w = 0;
        for (int a = 0; a < 7; ++a)
          if (src[a] >= 0) t[w++] = src[a];
      }
    for (int c = 0; c < 8; ++c, t += 8) {
      node_sources(m, n, e, corner_node(n, c), src);
      int w = 0;
      for (int a = 0; a < 7; ++a)
        if (src[a] >= 0) t[w++] = src[a];
    }
  }
  });
}

// Element-local Jacobi diagonal of the Laplacian in the reference's form
// (helmholtz_diagonal with lambda = 0, src/helmholtz.c:51-68): the metric
// terms G11, G22, G33 without the Jacobian determinant.  The Helmholtz
// diagonal is this plus lambda * rho * J, accumulated last.
void stiffness_diagonal(const HostLevel& L, int nel, double* out) {
  const int n = L.n;
  const double *D = L.D.data(), *w = L.w.data();
  parallel_elements(nel, [&](int e0, int e1) {
  for (int e = e0; e < e1; ++e) {
    const size_t o = e * L.nt;
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          double t = 0.0;
          for (int p = 0; p < n; ++p) {
            const double di = D[p * n + i], dj = D[p * n + j], dk = D[p * n + k];
            t += ((w[p] * w[j]) * w[k]) * (di * di) * L.g[0][o + (k * n + j) * n + p];
            t += ((w[i] * w[p]) * w[k]) * (dj * dj) * L.g[3][o + (k * n + p) * n + i];
            t += ((w[i] * w[j]) * w[p]) * (dk * dk) * L.g[5][o + (p * n + j) * n + i];
          }
          out[o + (k * n + j) * n + i] = t;
        }
  }
  });
}

ssg_status build_mesh(HostMesh& m, int n, int nel, const double* vert, const int* neigh,
                      std::string& err, unsigned opts, int svvn, double svva) {
  if (n < 2 || n > 12 || (3 * n) / 2 > SSG_MAXN) {
    err = "order n must be in [2, 12]";
    return SSG_ERR_ARG;
  }
  if (nel <= 0) {
    err = "nel must be positive";
    return SSG_ERR_ARG;
  }
  m.n = n;
  m.nel = nel;
  m.neigh.assign(neigh, neigh + 26 * (size_t)nel);
  ssg_status st = build_pairs(m, err, (opts & SSG_SETUP_OPPOSITE_PAIRING) != 0);
  if (st != SSG_OK) return st;
  int orders[SSG_MAXLEV];
  m.nlev = level_orders(n, orders);
  // one cut-off mode and amplitude for every level (src/precon.c:130-132)
  const int msvv = svvn >= 0 ? svvn : 2 * n / 3;
  for (int l = 0; l < m.nlev; ++l) {
    alloc_level(m.lev[l], orders[l], nel, l == 0 && !(opts & SSG_SETUP_NO_PARTICLES));
    make_basis(m.lev[l], orders[l], msvv, svva);
  }
  const bool particles = !(opts & SSG_SETUP_NO_PARTICLES);
  grid_from_vertices(m.lev[0], nel, vert);
  compute_factors(m.lev[0], nel, particles);
  m.has_particle_geom = particles;
  for (int l = 1; l < m.nlev; ++l) {
    HostLevel &F = m.lev[l - 1], &L = m.lev[l];
    L.jf.resize((size_t)F.n * L.n);
    interp_matrix(F.n, F.x.data(), L.n, L.x.data(), L.jf.data());
    // coarse grid = fine grid evaluated at the coarse nodes (src/precon.c:151-160)
    std::vector<double> Jc((size_t)L.n * F.n);
    interp_matrix(L.n, L.x.data(), F.n, F.x.data(), Jc.data());
    parallel_elements(nel, [&](int e0, int e1) {
      for (int e = e0; e < e1; ++e)
        for (int a = 0; a < 3; ++a)
          tensor3(F.n, L.n, Jc.data(), F.grid[a].data() + e * F.nt,
                  L.grid[a].data() + e * L.nt);
    });
    compute_factors(L, nel, false);
  }
  if (opts & SSG_SETUP_NO_DEALIAS) return SSG_OK;
  // dealiasing grid, m = 3n/2, from the vertices (src/main.c:53,71)
  const int mc = (3 * n) / 2;
  alloc_level(m.conv, mc, nel, true);
  make_basis(m.conv, mc, 2 * mc / 3, 0.0);
  grid_from_vertices(m.conv, nel, vert);
  compute_factors(m.conv, nel, true);
  m.jconv.resize((size_t)mc * n);
  interp_matrix(mc, m.conv.x.data(), n, m.lev[0].x.data(), m.jconv.data());
  m.has_conv = true;
  return SSG_OK;
}

}  // namespace ssg
