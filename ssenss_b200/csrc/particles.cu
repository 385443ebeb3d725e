// Lagrangian inertial particles (integrate_particle_equations at one rank,
// src/particles.c:182-546, with the point interpolation of
// src/interpolation.c:31-104).  One thread per particle.
//
// Element ids and reference coordinates must be bitwise those of the
// reference, so this file is compiled with --fmad=false and every expression
// keeps the reference's operation order: Lagrange weights as running
// products, the 5 x 5 x 5 stencil sum ((f lx) ly) lz in k, j, i order, the
// RK4 stage sums, the face walk.  pow(dt, 2) is dt * dt and pow(-1, k+1) is
// -+1, both exact.  The reference runs the passes of all particles
// together; particles do not interact at one rank, so a per-particle loop
// over the same passes gives the same result.  Where the reference would
// reseed a particle at a random position (more than 10 passes, or a forced
// step that still leaves the element) the status becomes 5 and the particle
// is left for the host to reseed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "ssg_internal.h"
#include "ssg_kernels.h"

namespace ssg {
namespace dev {

enum { P_NORMAL = 0, P_COLLISION = 1, P_OUTSIDE = 2, P_RESEED = 5 };

struct PartCtx {
  int n = 0;
  int nel = 0;
  size_t npts = 0;
  const double* x = nullptr;      // GLL points (n)
  const double* ur = nullptr;     // 3 levels x 3 comps x npts, oldest level first
  const double* jac = nullptr;    // 9 x npts, J[a][b] = dx_a/dr_b
  const double* tinv = nullptr;   // 9 x npts, tinv[a][b] = dr_b/dx_a
  const int* neigh = nullptr;     // nel x 26
  double t = 0.0;                 // flow time the particles advance to
  double dt = 0.0;                // flow time step
};

__device__ double lagrange(double xt, const double* xf, int p, int nf) {
  double l = 1.0;
  for (int q = 0; q < p; ++q) l *= (xt - xf[q]) / (xf[p] - xf[q]);
  for (int q = p + 1; q < nf; ++q) l *= (xt - xf[q]) / (xf[p] - xf[q]);
  return l;
}

// first node of the 5-point stencil (src/interpolation.c:106-112)
__device__ int first_point(const double* x, double xp, int n) {
  for (int i = 0; i < n - 4; ++i)
    if (x[i] > xp) return i - 2 > 0 ? i - 2 : 0;
  return n - 5;
}

// Lagrange weights of one point (src/interpolation.c:31-104): the full
// n-point stencil for n <= 5, else the 5-point stencil from first_point in
// each direction.  They depend on the position only, so one set serves
// every field interpolated at that point (the reference recomputes them per
// field; the values are the same).
struct Stencil {
  int i1, j1, k1;
  double lx[5], ly[5], lz[5];
};

__device__ __forceinline__ void stencil_at(int n, const double* x, double xp, double yp,
                                           double zp, Stencil& w) {
  if (n <= 5) {
    w.i1 = w.j1 = w.k1 = 0;
    for (int i = 0; i < n; ++i) {
      w.lx[i] = lagrange(xp, x, i, n);
      w.ly[i] = lagrange(yp, x, i, n);
      w.lz[i] = lagrange(zp, x, i, n);
    }
    return;
  }
  w.i1 = first_point(x, xp, n);
  w.j1 = first_point(x, yp, n);
  w.k1 = first_point(x, zp, n);
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    w.lx[i] = lagrange(xp, x + w.i1, i, 5);
    w.ly[i] = lagrange(yp, x + w.j1, i, 5);
    w.lz[i] = lagrange(zp, x + w.k1, i, 5);
  }
}

// point value of one element block f (n^3) with the weights w, in the
// reference's summation order for each stencil form
__device__ __forceinline__ double interp_at(int n, const Stencil& w, const double* f) {
  if (n <= 5) {
    double s = 0.0;
    for (int k = 0; k < n; ++k) {
      double sj = 0.0;
      for (int j = 0; j < n; ++j) {
        double si = 0.0;
        for (int i = 0; i < n; ++i) si += f[(k * n + j) * n + i] * w.lx[i];
        sj += si * w.ly[j];
      }
      s += sj * w.lz[k];
    }
    return s;
  }
  double s = 0.0;
#pragma unroll 1
  for (int k = 0; k < 5; ++k)
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const double* row = f + ((w.k1 + k) * n + w.j1 + j) * n + w.i1;
#pragma unroll
      for (int i = 0; i < 5; ++i) s += row[i] * w.lx[i] * w.ly[j] * w.lz[k];
    }
  return s;
}

__device__ const double* ur_block(const PartCtx& P, int lev, int comp, int e) {
  return P.ur + ((size_t)(lev * 3 + comp)) * P.npts + (size_t)e * P.n * P.n * P.n;
}

// quadratic Lagrange in time over t0-2dt, t0-dt, t0 (src/particles.c:493-515),
// the three components at one point
__device__ void fluid_velocity3(const PartCtx& P, int e, const double* y, double t,
                                double* uf) {
  const double eps = 1.0e-6;
  const double d0 = t - P.t + 2.0 * P.dt, d1 = t - P.t + P.dt, d2 = t - P.t;
  const double dt2 = P.dt * P.dt;
  const double a = 0.5 * d1 * d2 / dt2;
  const double b = -d0 * d2 / dt2;
  const double c = 0.5 * d0 * d1 / dt2;
  Stencil w;
  stencil_at(P.n, P.x, y[0], y[1], y[2], w);
  for (int comp = 0; comp < 3; ++comp) {
    double u0 = 0.0, u1 = 0.0, u2 = 0.0;
    if (fabs(a) > eps) u0 = interp_at(P.n, w, ur_block(P, 0, comp, e));
    if (fabs(b) > eps) u1 = interp_at(P.n, w, ur_block(P, 1, comp, e));
    if (fabs(c) > eps) u2 = interp_at(P.n, w, ur_block(P, 2, comp, e));
    uf[comp] = a * u0 + b * u1 + c * u2;
  }
}

__device__ void particle_rhs(const PartCtx& P, int e, double tau, const double* y, double t,
                             double* f) {
  const double a = 1.0 / tau;
  double uf[3];
  fluid_velocity3(P, e, y, t, uf);
  for (int i = 0; i < 3; ++i) {
    f[i] = y[i + 3];
    f[i + 3] = a * (uf[i] - y[i + 3]);
  }
}

__device__ bool crossed(const double* y) {
  for (int i = 0; i < 3; ++i)
    if (fabs(y[i]) > 1.0) return true;
  return false;
}

// classic RK4 (src/particles.c:238-269); s = {x,y,z,u,v,w,t,tau}
__device__ void rk4(const PartCtx& P, double* s, int* st, double dt, bool force) {
  const double aa[4] = {0.0, 0.5, 0.5, 1.0};
  const int e = st[0];
  double y[6], y0[6], f[4][6];
  for (int i = 0; i < 6; ++i) y0[i] = s[i];
  for (int j = 0; j < 4; ++j)
    for (int i = 0; i < 6; ++i) f[j][i] = 0.0;
  for (int j = 0; j < 4; ++j) {
    const double t = s[6] + aa[j] * dt;
    const int jm = j - 1 > 0 ? j - 1 : 0;
    for (int i = 0; i < 6; ++i) y[i] = y0[i] + aa[j] * dt * f[jm][i];
    if (j > 0 && crossed(y) && !force) {
      st[2] = P_OUTSIDE;
      return;
    }
    particle_rhs(P, e, s[7], y, t, f[j]);
  }
  for (int i = 0; i < 6; ++i)
    y[i] = y0[i] + dt * (f[0][i] / 6.0 + f[1][i] / 3.0 + f[2][i] / 3.0 + f[3][i] / 6.0);
  if (crossed(y)) {
    st[2] = P_OUTSIDE;
    return;
  }
  for (int i = 0; i < 6; ++i) s[i] = y[i];
  s[6] = P.t;
}

__device__ double step_to_boundary(const double* y, const double* f) {
  double d[3];
  for (int i = 0; i < 3; ++i) d[i] = (copysign(1.0, f[i]) - y[i]) / f[i];
  const double m01 = d[0] < d[1] ? d[0] : d[1];
  return m01 < d[2] ? m01 : d[2];
}

// RK4-weighted straight step to the element face (src/particles.c:271-316)
__device__ void to_boundary(const PartCtx& P, double* s, int* st, double dt) {
  const double aa[4] = {0.0, 0.5, 0.5, 1.0};
  const int e = st[0];
  double y[6], y0[6], f[5][6];
  double dtau = 0.0;
  for (int i = 0; i < 6; ++i) y0[i] = s[i];
  for (int j = 0; j < 5; ++j)
    for (int i = 0; i < 6; ++i) f[j][i] = 0.0;
  for (int j = 0; j < 4; ++j) {
    const double t = s[6] + aa[j] * dtau;
    const int jm = j - 1 > 0 ? j - 1 : 0;
    for (int i = 0; i < 6; ++i) y[i] = y0[i] + aa[j] * dtau * f[jm][i];
    particle_rhs(P, e, s[7], y, t, f[j]);
    dtau = step_to_boundary(y0, f[j]);
  }
  for (int i = 0; i < 6; ++i)
    f[4][i] = (f[0][i] / 6.0 + f[1][i] / 3.0 + f[2][i] / 3.0 + f[3][i] / 6.0);
  dtau = step_to_boundary(y0, f[4]);
  if (dtau < dt) {
    s[6] += dtau;
    for (int i = 0; i < 6; ++i) s[i] += dtau * f[4][i];
  } else {
    st[2] = P_NORMAL;
    rk4(P, s, st, dt, true);
    if (st[2] != P_NORMAL) st[2] = P_RESEED;
  }
}

__device__ int closest_face(const double* s) {
  double hmin = 2.0;
  int k = 0;
  for (int i = 0; i < 6; ++i) {
    const double h = fabs(s[i / 2] - (i % 2 ? 1.0 : -1.0));
    if (h < hmin) {
      hmin = h;
      k = i;
    }
  }
  return k;
}

__device__ double factor_at(const PartCtx& P, const Stencil& w, const double* fac, int a,
                           int e) {
  return interp_at(P.n, w, fac + (size_t)a * P.npts + (size_t)e * P.n * P.n * P.n);
}

// cross into the neighbour through the closest face; physical velocity by
// the interpolated Jacobian, component by component (src/particles.c:
// 333-349, 517-527); a wall reverses the normal velocity
__device__ void new_element(const PartCtx& P, double* s, int* st) {
  const int e = st[0];
  const int j = closest_face(s);
  const int nb = P.neigh[26 * (size_t)e + j];
  if (nb >= 0) {
    st[0] = nb;
    // the position does not change in this loop: one set of weights
    Stencil w;
    stencil_at(P.n, P.x, s[0], s[1], s[2], w);
    for (int comp = 0; comp < 3; ++comp) {
      double dx[3];
      for (int i = 0; i < 3; ++i) dx[i] = factor_at(P, w, P.jac, 3 * comp + i, e);
      s[3 + comp] = s[3] * dx[0] + s[4] * dx[1] + s[5] * dx[2];
    }
  } else {
    st[2] = P_COLLISION;
    s[3 + j / 2] *= -1.0;
  }
}

// entry face = the last face of the new element whose neighbour is the old
// element; velocity back to reference components (src/particles.c:351-378,
// 529-539)
__device__ void new_location(const PartCtx& P, double* s, int* st) {
  const int e = st[0];
  double y0[6], x[2];
  for (int i = 0; i < 6; ++i) y0[i] = s[i];
  int k = closest_face(s);
  int j = 0;
  for (int i = 0; i < 3; ++i)
    if (i != k / 2) x[j++] = y0[i];
  for (int i = 0; i < 6; ++i)
    if (P.neigh[26 * (size_t)e + i] == st[1]) k = i;
  s[k / 2] = k % 2 ? 1.0 : -1.0;
  j = 0;
  for (int i = 0; i < 3; ++i) {
    if (i != k / 2) s[i] = x[j++];
    // the position changes from one i to the next: weights per i
    Stencil w;
    stencil_at(P.n, P.x, s[0], s[1], s[2], w);
    double dx[3];
    for (int a = 0; a < 3; ++a) dx[a] = factor_at(P, w, P.tinv, 3 * a + i, e);
    s[3 + i] = s[3] * dx[0] + s[4] * dx[1] + s[5] * dx[2];
  }
  st[1] = st[0];
}

// Particles are taken in element order (a counting sort of their element
// ids each call) so that the threads of a warp interpolate in the same
// element's fields and share their cache lines; each particle's own
// arithmetic is unchanged, so the order does not change any result.
__global__ void k_part_count(size_t np, const int* __restrict__ ints, int nel,
                             int* __restrict__ count) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += (size_t)gridDim.x * blockDim.x) {
    const int e = ints[3 * i];
    atomicAdd(count + (e >= 0 && e < nel ? e : nel), 1);
  }
}

// exclusive prefix sum of count[0 .. nb) into start[0 .. nb), one block
__global__ void __launch_bounds__(1024) k_part_scan(int nb, const int* __restrict__ count,
                                                    int* __restrict__ start) {
  __shared__ int part[1024];
  const int chunk = (nb + 1023) / 1024;
  const int lo = threadIdx.x * chunk, hi = min(nb, lo + chunk);
  int sum = 0;
  for (int q = lo; q < hi; ++q) sum += count[q];
  part[threadIdx.x] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {   // inclusive scan of the chunk sums
    const int v = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = part[threadIdx.x] - sum;
  for (int q = lo; q < hi; ++q) {
    start[q] = run;
    run += count[q];
  }
}

__global__ void k_part_scatter(size_t np, const int* __restrict__ ints, int nel,
                               int* __restrict__ cursor, int* __restrict__ order) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += (size_t)gridDim.x * blockDim.x) {
    const int e = ints[3 * i];
    order[atomicAdd(cursor + (e >= 0 && e < nel ? e : nel), 1)] = (int)i;
  }
}

__global__ void __launch_bounds__(128) k_particles(PartCtx P, size_t np, double* __restrict__ state,
                                                   int* __restrict__ ints, int* __restrict__ passes,
                                                   const int* __restrict__ order) {
  const size_t ti = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ti >= np) return;
  const size_t pi = order ? (size_t)order[ti] : ti;
  double s[8];
  int st[3];
  for (int a = 0; a < 8; ++a) s[a] = state[8 * pi + a];
  for (int a = 0; a < 3; ++a) st[a] = ints[3 * pi + a];
  if (st[0] < 0 || st[0] >= P.nel) {   // invalid element: leave untouched
    ints[3 * pi + 2] = P_RESEED;
    return;
  }
  st[2] = P_OUTSIDE;
  int pass = 0;
  // at most 12 passes: after 10 the reference reseeds (src/particles.c:192)
  while (st[2] != P_NORMAL && st[2] != P_RESEED) {
    st[2] = P_NORMAL;
    if (pass > 10) {
      st[2] = P_RESEED;
    } else {
      rk4(P, s, st, P.t - s[6], false);
      if (st[2] == P_OUTSIDE) to_boundary(P, s, st, 2.0 * P.dt);
      if (st[2] == P_OUTSIDE) new_element(P, s, st);
      if (st[2] == P_OUTSIDE) new_location(P, s, st);
    }
    ++pass;
  }
  for (int a = 0; a < 8; ++a) state[8 * pi + a] = s[a];
  for (int a = 0; a < 3; ++a) ints[3 * pi + a] = st[a];
  atomicMax(passes, pass);
}

}  // namespace dev

cudaError_t run_particles(cudaStream_t s, int n, int nel, size_t npts, const double* x,
                          const double* ur, const double* jac, const double* tinv,
                          const int* neigh, double t, double dt, size_t np, double* state,
                          int* ints, int* passes, int* order, int* bucket) {
  dev::PartCtx P;
  P.n = n;
  P.nel = nel;
  P.npts = npts;
  P.x = x;
  P.ur = ur;
  P.jac = jac;
  P.tinv = tinv;
  P.neigh = neigh;
  P.t = t;
  P.dt = dt;
  if (np == 0) return cudaSuccess;
  if (np > (size_t)INT32_MAX) return cudaErrorInvalidValue;
  if (order) {
    // bucket: counts then start offsets, nel + 1 each (the last bucket holds
    // particles with an invalid element id)
    int* count = bucket;
    int* cursor = bucket + nel + 1;
    cudaError_t err = cudaMemsetAsync(count, 0, (nel + 1) * sizeof(int), s);
    if (err != cudaSuccess) return err;
    const unsigned g = (unsigned)std::min<size_t>((np + 255) / 256, 4096);
    count_launch();
    dev::k_part_count<<<g, 256, 0, s>>>(np, ints, nel, count);
    count_launch();
    dev::k_part_scan<<<1, 1024, 0, s>>>(nel + 1, count, cursor);
    count_launch();
    dev::k_part_scatter<<<g, 256, 0, s>>>(np, ints, nel, cursor, order);
  }
  const unsigned blocks = (unsigned)((np + 127) / 128);
  count_launch();
  dev::k_particles<<<blocks, 128, 0, s>>>(P, np, state, ints, passes, order);
  return cudaGetLastError();
}

}  // namespace ssg
