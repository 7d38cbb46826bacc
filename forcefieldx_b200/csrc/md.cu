// md.cu -- molecular dynamics on the device: velocity Verlet with SETTLE rigid waters.
//
// VelocityVerlet.preForce / postForce (algorithms/.../integrators/VelocityVerlet.java:73-120)
// around the library's own energy + gradient, with SettleConstraint
// (P/constraint/SettleConstraint.java:169-441) for rigid three-site molecules, so a
// trajectory never leaves the GPU between steps.  Units are the reference's: A, ps, amu,
// kcal/mol; a = -418.4 * gradient / mass (Constants.KCAL_TO_GRAM_ANG2_PER_PS2).
//
// SETTLE positions follow the analytical construction of Miyamoto and Kollman
// (J. Comput. Chem. 13, 952-962, 1992): the unconstrained new positions are expressed in
// a frame built from the old molecular plane and the new centre-atom position about the
// new centre of mass; the canonical triangle is rotated by phi and psi (out of plane) and
// by theta (in plane, from conservation of angular momentum), then mapped back.  The
// velocity step removes the relative velocity along the three sides with the impulses
// that solve the 3 x 3 linear system of RATTLE's velocity conditions (solved here by
// Cramer's rule).
#include <cmath>
#include <cstring>
#include <vector>

#include "ffx_internal.cuh"

namespace ffx {

constexpr double kKcalToAmuA2Ps2 = 418.4;

namespace {
struct V3 {
  double x, y, z;
};
__device__ __forceinline__ V3 v3(double x, double y, double z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator*(double s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ V3 unit(V3 a) { return (1.0 / sqrt(dot(a, a))) * a; }
__device__ __forceinline__ V3 load3(const double *p, int i) { return v3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
__device__ __forceinline__ void store3(double *p, int i, V3 a) {
  p[3 * i] = a.x;
  p[3 * i + 1] = a.y;
  p[3 * i + 2] = a.z;
}
}  // namespace

// v += a dt/2; x += v dt (the half kick and the drift of preForce); keeps the prior x.
__global__ void k_md_pre(int n, double dt, const double *__restrict__ mass, double *x, double *v,
                         const double *__restrict__ a, double *xprior) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= 3 * n) return;
  const double m = mass[j / 3];
  xprior[j] = x[j];
  if (m > 0.0) {
    const double vv = v[j] + a[j] * (0.5 * dt);
    v[j] = vv;
    x[j] = x[j] + vv * dt;
  }
}

// SETTLE on positions: one thread per rigid molecule (centre atom A, partners B and C;
// d1 = |AB| = |AC|, d2 = |BC|; the partners have equal masses).
__global__ void k_settle_positions(int nw, const int *__restrict__ idx, double d1, double d2,
                                   const double *__restrict__ mass, const double *__restrict__ x0, double *x) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nw) return;
  const int ia = idx[3 * w], ib = idx[3 * w + 1], ic = idx[3 * w + 2];
  const double mA = mass[ia], mB = mass[ib], mC = mass[ic];
  const double M = mA + mB + mC;
  // Old geometry relative to A, and the unconstrained new positions.
  const V3 A0 = load3(x0, ia), B0 = load3(x0, ib) - A0, C0 = load3(x0, ic) - A0;
  const V3 A1n = load3(x, ia), B1n = load3(x, ib), C1n = load3(x, ic);
  // New positions relative to the old A, and the new centre of mass.
  const V3 a1r = A1n - A0, b1r = B1n - A0, c1r = C1n - A0;
  const V3 com = (1.0 / M) * (mA * a1r + mB * b1r + mC * c1r);
  const V3 a1 = a1r - com, b1 = b1r - com, c1 = c1r - com;
  // Frame: Z normal to the old plane, X normal to Z and the new A, Y completes it.
  const V3 ez = unit(cross(B0, C0));
  const V3 ex = unit(cross(a1, ez));
  const V3 ey = unit(cross(ez, ex));
  // Old triangle in the frame (in plane), new positions in the frame.
  const double bx0 = dot(B0, ex), by0 = dot(B0, ey), cx0 = dot(C0, ex), cy0 = dot(C0, ey);
  const double za1 = dot(a1, ez);
  const double bx1 = dot(b1, ex), by1 = dot(b1, ey), bz1 = dot(b1, ez);
  const double cx1 = dot(c1, ex), cy1 = dot(c1, ey), cz1 = dot(c1, ez);
  // Canonical triangle about the centre of mass: A at (0, ra), B, C at (-+rc, -rb).
  const double rc = 0.5 * d2;
  const double h = sqrt(d1 * d1 - rc * rc);
  const double ra = h * (mB + mC) / M;
  const double rb = h - ra;
  // Out-of-plane rotations (phi about X, psi about Y') that reproduce the new heights.
  const double sphi = za1 / ra;
  const double cphi = sqrt(1.0 - sphi * sphi);
  const double spsi = (bz1 - cz1) / (2.0 * rc * cphi);
  const double cpsi = sqrt(1.0 - spsi * spsi);
  const double ya2 = ra * cphi;
  const double xb2 = -rc * cpsi, xc2 = rc * cpsi;
  const double yb2 = -rb * cphi - rc * spsi * sphi;
  const double yc2 = -rb * cphi + rc * spsi * sphi;
  // In-plane rotation theta from conservation of angular momentum about Z.
  const double al = xb2 * (bx0 - cx0) + by0 * yb2 + cy0 * yc2;
  const double be = xb2 * (cy0 - by0) + bx0 * yb2 + cx0 * yc2;
  const double ga = bx0 * by1 - bx1 * by0 + cx0 * cy1 - cx1 * cy0;
  const double ab2 = al * al + be * be;
  const double sth = (al * ga - be * sqrt(ab2 - ga * ga)) / ab2;
  const double cth = sqrt(1.0 - sth * sth);
  const V3 a3 = (-ya2 * sth) * ex + (ya2 * cth) * ey + za1 * ez;
  const V3 b3 = (xb2 * cth - yb2 * sth) * ex + (xb2 * sth + yb2 * cth) * ey + bz1 * ez;
  const V3 c3 = (xc2 * cth - yc2 * sth) * ex + (xc2 * sth + yc2 * cth) * ey + cz1 * ez;
  store3(x, ia, A0 + com + a3);
  store3(x, ib, A0 + com + b3);
  store3(x, ic, A0 + com + c3);
}

// v = (x - x_prior) / dt after the constrained drift (VelocityVerlet.preForce).
__global__ void k_md_velocity_from_step(int n, double dt, const double *__restrict__ mass,
                                        const double *__restrict__ x, const double *__restrict__ xprior, double *v) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= 3 * n) return;
  if (mass[j / 3] > 0.0) v[j] = (x[j] - xprior[j]) / dt;
}

// a = -418.4 g / m; v += a dt/2 (postForce).
__global__ void k_md_post(int n, double dt, const double *__restrict__ mass, const double *__restrict__ g, double *v,
                          double *a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= 3 * n) return;
  const double m = mass[j / 3];
  if (m > 0.0) {
    const double aj = -kKcalToAmuA2Ps2 * g[j] / m;
    a[j] = aj;
    v[j] = v[j] + aj * (0.5 * dt);
  }
}

// a = -418.4 g / m only (the accelerations of the starting configuration).
__global__ void k_md_accel(int n, const double *__restrict__ mass, const double *__restrict__ g, double *a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= 3 * n) return;
  const double m = mass[j / 3];
  a[j] = (m > 0.0) ? -kKcalToAmuA2Ps2 * g[j] / m : 0.0;
}

// SETTLE on velocities: impulses t along the unit sides e_AB, e_BC, e_CA such that the
// relative velocity along every side vanishes:
//   v_AB - (1/mA + 1/mB) t_AB + (e_BC.e_AB / mB) t_BC + (e_CA.e_AB / mA) t_CA = 0, etc.
__global__ void k_settle_velocities(int nw, const int *__restrict__ idx, const double *__restrict__ mass,
                                    const double *__restrict__ x, double *v) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nw) return;
  const int ia = idx[3 * w], ib = idx[3 * w + 1], ic = idx[3 * w + 2];
  const double iA = 1.0 / mass[ia], iB = 1.0 / mass[ib], iC = 1.0 / mass[ic];
  const V3 A = load3(x, ia), B = load3(x, ib), C = load3(x, ic);
  const V3 eAB = unit(B - A), eBC = unit(C - B), eCA = unit(A - C);
  const V3 vA = load3(v, ia), vB = load3(v, ib), vC = load3(v, ic);
  const double r0 = dot(vB - vA, eAB), r1 = dot(vC - vB, eBC), r2 = dot(vA - vC, eCA);
  const double cAB_BC = dot(eAB, eBC), cBC_CA = dot(eBC, eCA), cCA_AB = dot(eCA, eAB);
  // K t = r with K symmetric.
  const double k00 = iA + iB, k11 = iB + iC, k22 = iC + iA;
  const double k01 = -cAB_BC * iB, k12 = -cBC_CA * iC, k02 = -cCA_AB * iA;
  const double det = k00 * (k11 * k22 - k12 * k12) - k01 * (k01 * k22 - k12 * k02) + k02 * (k01 * k12 - k11 * k02);
  const double t0 = (r0 * (k11 * k22 - k12 * k12) - k01 * (r1 * k22 - k12 * r2) + k02 * (r1 * k12 - k11 * r2)) / det;
  const double t1 = (k00 * (r1 * k22 - k12 * r2) - r0 * (k01 * k22 - k12 * k02) + k02 * (k01 * r2 - r1 * k02)) / det;
  const double t2 = (k00 * (k11 * r2 - r1 * k12) - k01 * (k01 * r2 - r1 * k02) + r0 * (k01 * k12 - k11 * k02)) / det;
  store3(v, ia, vA + iA * (t0 * eAB - t2 * eCA));
  store3(v, ib, vB + iB * (t1 * eBC - t0 * eAB));
  store3(v, ic, vC + iC * (t2 * eCA - t1 * eBC));
}

// Kinetic energy 1/2 sum m v^2 / 418.4 (kcal/mol) in a fixed order by one block.
__global__ void __launch_bounds__(256) k_md_kinetic(int n, const double *__restrict__ mass,
                                                    const double *__restrict__ v, double *out) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) {
    const double vx = v[3 * i], vy = v[3 * i + 1], vz = v[3 * i + 2];
    s += mass[i] * (vx * vx + vy * vy + vz * vz);
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < 256; k++) t += sh[k];
    *out = 0.5 * t / kKcalToAmuA2Ps2;
  }
}

// ---------------------------------------------------------------------------
int md_setup(Handle &h, const ffxg_md *md) {
  const size_t N = h.n;
  if (!md || !md->mass) { h.err = "md: masses required"; return FFXG_ERR_BAD_ARG; }
  if (md->n_settle < 0 || (md->n_settle > 0 && !md->settle)) { h.err = "md: bad SETTLE list"; return FFXG_ERR_BAD_ARG; }
  if (md->n_settle > 0 && !(md->settle_d1 > 0.0 && md->settle_d2 > 0.0 && md->settle_d2 < 2.0 * md->settle_d1)) {
    h.err = "md: SETTLE distances must satisfy 0 < d2 < 2 d1";
    return FFXG_ERR_BAD_ARG;
  }
  std::vector<int> seen(N, 0);
  for (int w = 0; w < md->n_settle; w++)
    for (int q = 0; q < 3; q++) {
      const int a = md->settle[3 * w + q];
      if (a < 0 || a >= (int)N || seen[a]++) { h.err = "md: SETTLE atom out of range or repeated"; return FFXG_ERR_BAD_ARG; }
    }
  for (size_t i = 0; i < N; i++)
    if (!(md->mass[i] >= 0.0)) { h.err = "md: masses must be non-negative"; return FFXG_ERR_BAD_ARG; }
  if (!h.d_mass) {
    if (cudaMalloc(&h.d_mass, N * sizeof(double)) != cudaSuccess || cudaMalloc(&h.d_mdx, 3 * N * sizeof(double)) ||
        cudaMalloc(&h.d_mdv, 3 * N * sizeof(double)) || cudaMalloc(&h.d_mda, 3 * N * sizeof(double)) ||
        cudaMalloc(&h.d_mdxp, 3 * N * sizeof(double)) || cudaMalloc(&h.d_mdg, 3 * N * sizeof(double)) ||
        cudaMalloc(&h.d_mdke, sizeof(double))) {
      h.err = "md: device allocation failed";
      return FFXG_ERR_CUDA;
    }
  }
  if (h.d_settle) { cudaFree(h.d_settle); h.d_settle = nullptr; }
  h.n_settle = md->n_settle;
  if (h.n_settle > 0) {
    if (cudaMalloc(&h.d_settle, 3 * (size_t)h.n_settle * sizeof(int)) != cudaSuccess) {
      h.err = "md: device allocation failed";
      return FFXG_ERR_CUDA;
    }
    cudaMemcpy(h.d_settle, md->settle, 3 * (size_t)h.n_settle * sizeof(int), cudaMemcpyHostToDevice);
  }
  cudaMemcpy(h.d_mass, md->mass, N * sizeof(double), cudaMemcpyHostToDevice);
  h.settle_d1 = md->settle_d1;
  h.settle_d2 = md->settle_d2;
  h.md_ready = true;
  return cudaGetLastError() == cudaSuccess ? FFXG_OK : FFXG_ERR_CUDA;
}

int md_run(Handle &h, double dt, int steps, double *xyz, double *vel, double *epot, double *ekin,
           int (*force)(Handle &, const double *, double *, double *)) {
  if (!h.md_ready) { h.err = "md: call ffxg_md_setup first"; return FFXG_ERR_BAD_ARG; }
  if (!(dt > 0.0) || steps < 0 || !xyz || !vel) { h.err = "md: bad arguments"; return FFXG_ERR_BAD_ARG; }
  const int n = h.n;
  const size_t N3 = 3 * (size_t)n;
  const int nb = nblocks(3 * (int64_t)n, 256), nw = nblocks(h.n_settle, 128);
  cudaMemcpyAsync(h.d_mdx, xyz, N3 * sizeof(double), cudaMemcpyHostToDevice, h.stream);
  cudaMemcpyAsync(h.d_mdv, vel, N3 * sizeof(double), cudaMemcpyHostToDevice, h.stream);
  double terms[FFXG_N_TERMS];
  // FFXG_ERR_RANGE (the mixed form's fixed-point sums out of their exact range) leaves
  // complete forces: the run goes on and reports it at the end.
  bool range = false;
  auto fatal = [&](int st) {
    if (st == FFXG_ERR_RANGE) { range = true; return false; }
    return st != FFXG_OK;
  };
  // Accelerations of the starting configuration.
  int st = force(h, h.d_mdx, h.d_mdg, terms);
  if (fatal(st)) return st;
  k_md_accel<<<nb, 256, 0, h.stream>>>(n, h.d_mass, h.d_mdg, h.d_mda);
  for (int s = 0; s < steps; s++) {
    k_md_pre<<<nb, 256, 0, h.stream>>>(n, dt, h.d_mass, h.d_mdx, h.d_mdv, h.d_mda, h.d_mdxp);
    if (h.n_settle > 0) {
      k_settle_positions<<<nw, 128, 0, h.stream>>>(h.n_settle, h.d_settle, h.settle_d1, h.settle_d2, h.d_mass,
                                                   h.d_mdxp, h.d_mdx);
      k_md_velocity_from_step<<<nb, 256, 0, h.stream>>>(n, dt, h.d_mass, h.d_mdx, h.d_mdxp, h.d_mdv);
    }
    st = force(h, h.d_mdx, h.d_mdg, terms);
    if (fatal(st)) return st;
    k_md_post<<<nb, 256, 0, h.stream>>>(n, dt, h.d_mass, h.d_mdg, h.d_mdv, h.d_mda);
    if (h.n_settle > 0)
      k_settle_velocities<<<nw, 128, 0, h.stream>>>(h.n_settle, h.d_settle, h.d_mass, h.d_mdx, h.d_mdv);
    if (ekin) {
      k_md_kinetic<<<1, 256, 0, h.stream>>>(n, h.d_mass, h.d_mdv, h.d_mdke);
      cudaMemcpyAsync(&h.h_scalars[12], h.d_mdke, sizeof(double), cudaMemcpyDeviceToHost, h.stream);
      if (cudaStreamSynchronize(h.stream) != cudaSuccess) return FFXG_ERR_CUDA;
      ekin[s] = h.h_scalars[12];
    }
    if (epot) epot[s] = terms[FFXG_TERM_TOTAL];
  }
  cudaMemcpyAsync(h.h_xyz_pin, h.d_mdx, N3 * sizeof(double), cudaMemcpyDeviceToHost, h.stream);
  cudaMemcpyAsync(h.h_grad_pin, h.d_mdv, N3 * sizeof(double), cudaMemcpyDeviceToHost, h.stream);
  if (cudaStreamSynchronize(h.stream) != cudaSuccess) return FFXG_ERR_CUDA;
  std::memcpy(xyz, h.h_xyz_pin, N3 * sizeof(double));
  std::memcpy(vel, h.h_grad_pin, N3 * sizeof(double));
  return range ? FFXG_ERR_RANGE : FFXG_OK;
}

}  // namespace ffx
