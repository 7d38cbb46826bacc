// pme.cu -- multipole rotation and the particle-mesh Ewald reciprocal space.
//
//  k_rotate           InitializationRegion.RotateMultipolesLoop (pme/InitializationRegion.java:375-480)
//                     with MultipoleType.getRotationMatrix / rotateMultipole (MultipoleType.java:385-536, 1031-1062)
//  k_bsplines         ReciprocalSpace.BSplineLoop (ReciprocalSpace.java:1338-1412), UniformBSpline (:98-183),
//                     toFractionalMultipole (:1212-1236)
//  k_spread_*         SpatialPermanentLoop / SpatialInducedLoop (ReciprocalSpace.java:1445-1505, 1573-1628)
//  k_fft_axis         Complex3DParallel.convolution (N/fft/Complex3DParallel.java:445, 775-795, 972-1010):
//                     X and Y passes, a fused Z pass (FFT, influence function, inverse FFT), inverse Y, X.
//  k_phi              PermanentPhiLoop / InducedPhiLoop (ReciprocalSpace.java:2295-2454, 2506-2775)
//
// The mesh is one interleaved complex double grid [nz][ny][nx], 16 B per point, kept
// L2-resident between passes.  Spreading uses FP64 atomics into the mesh.
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>

#include <cooperative_groups.h>

#include "ffx_internal.cuh"

namespace cg = cooperative_groups;

namespace ffx {

enum { t000 = 0, t100, t010, t001, t200, t020, t002, t110, t101, t011,
       t300, t030, t003, t210, t201, t120, t021, t102, t012, t111 };


// ---------------------------------------------------------------------------
__device__ __forceinline__ void d_norm(double *v) {
  const double l = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  v[0] /= l; v[1] /= l; v[2] /= l;
}

__device__ __forceinline__ void k_rotate(VGrid vg, int n, const double *__restrict__ x, const double *__restrict__ y,
                         const double *__restrict__ z, const int *__restrict__ frame, const int *__restrict__ axis,
                         const double *__restrict__ lmp, double *gm, double *rot) {
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double R[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  const int fr = frame[i];
  if (fr != FFXG_FRAME_NONE) {
    const double o[3] = {x[i], y[i], z[i]};
    double zA[3], xA[3], yA[3];
    const int az = axis[i], ax = axis[n + i], ay = axis[2 * n + i];
    zA[0] = x[az] - o[0]; zA[1] = y[az] - o[1]; zA[2] = z[az] - o[2];
    if (ax >= 0) { xA[0] = x[ax] - o[0]; xA[1] = y[ax] - o[1]; xA[2] = z[ax] - o[2]; }
    if (ay >= 0) { yA[0] = x[ay] - o[0]; yA[1] = y[ay] - o[1]; yA[2] = z[ay] - o[2]; }
    if (fr == FFXG_FRAME_BISECTOR) {
      d_norm(zA); d_norm(xA);
      for (int d = 0; d < 3; d++) zA[d] = xA[d] + zA[d];
      d_norm(zA);
      R[0][2] = zA[0]; R[1][2] = zA[1]; R[2][2] = zA[2];
      const double dt = xA[0] * zA[0] + xA[1] * zA[1] + xA[2] * zA[2];
      for (int d = 0; d < 3; d++) xA[d] = xA[d] - zA[d] * dt;
      d_norm(xA);
    } else if (fr == FFXG_FRAME_ZTHENBISECTOR) {
      d_norm(zA);
      R[0][2] = zA[0]; R[1][2] = zA[1]; R[2][2] = zA[2];
      d_norm(xA); d_norm(yA);
      for (int d = 0; d < 3; d++) xA[d] = xA[d] + yA[d];
      d_norm(xA);
      const double dt = xA[0] * zA[0] + xA[1] * zA[1] + xA[2] * zA[2];
      for (int d = 0; d < 3; d++) xA[d] = xA[d] - zA[d] * dt;
      d_norm(xA);
    } else if (fr == FFXG_FRAME_ZONLY) {
      d_norm(zA);
      R[0][2] = zA[0]; R[1][2] = zA[1]; R[2][2] = zA[2];
      xA[0] = 1.0; xA[1] = 0.0; xA[2] = 0.0;
      double dt = R[0][2];
      if (fabs(dt) > 0.866) { xA[0] = 0.0; xA[1] = 1.0; dt = R[1][2]; }
      for (int d = 0; d < 3; d++) xA[d] = xA[d] - zA[d] * dt;
      d_norm(xA);
    } else if (fr == FFXG_FRAME_THREEFOLD) {
      d_norm(zA); d_norm(xA); d_norm(yA);
      double s[3];
      for (int d = 0; d < 3; d++) s[d] = (zA[d] + xA[d]) + yA[d];
      d_norm(s);
      R[0][2] = s[0]; R[1][2] = s[1]; R[2][2] = s[2];
      const double dt = zA[0] * s[0] + zA[1] * s[1] + zA[2] * s[2];
      for (int d = 0; d < 3; d++) xA[d] = zA[d] - s[d] * dt;
      d_norm(xA);
    } else {  // ZTHENX
      d_norm(zA);
      R[0][2] = zA[0]; R[1][2] = zA[1]; R[2][2] = zA[2];
      const double dt = xA[0] * zA[0] + xA[1] * zA[1] + xA[2] * zA[2];
      for (int d = 0; d < 3; d++) xA[d] = xA[d] - zA[d] * dt;
      d_norm(xA);
    }
    R[0][0] = xA[0]; R[1][0] = xA[1]; R[2][0] = xA[2];
    R[0][1] = R[2][0] * R[1][2] - R[1][0] * R[2][2];
    R[1][1] = R[0][0] * R[2][2] - R[2][0] * R[0][2];
    R[2][1] = R[1][0] * R[0][2] - R[0][0] * R[1][2];
  }
  const double d[3] = {lmp[t100 * n + i], lmp[t010 * n + i], lmp[t001 * n + i]};
  double Q[3][3];
  Q[0][0] = lmp[t200 * n + i]; Q[1][1] = lmp[t020 * n + i]; Q[2][2] = lmp[t002 * n + i];
  Q[0][1] = Q[1][0] = lmp[t110 * n + i];
  Q[0][2] = Q[2][0] = lmp[t101 * n + i];
  Q[1][2] = Q[2][1] = lmp[t011 * n + i];
  double rd[3], rq[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    rd[a] = R[a][0] * d[0] + R[a][1] * d[1] + R[a][2] * d[2];
#pragma unroll
    for (int b = a; b < 3; b++) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 3; k++) s += R[a][k] * (R[b][0] * Q[k][0] + R[b][1] * Q[k][1] + R[b][2] * Q[k][2]);
      rq[a][b] = s;
    }
  }
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) rot[(3 * a + b) * n + i] = R[a][b];   // kept for the parameter gradients
  gm[t000 * n + i] = lmp[i];
  gm[t100 * n + i] = rd[0]; gm[t010 * n + i] = rd[1]; gm[t001 * n + i] = rd[2];
  gm[t200 * n + i] = rq[0][0]; gm[t020 * n + i] = rq[1][1]; gm[t002 * n + i] = rq[2][2];
  gm[t110 * n + i] = rq[0][1]; gm[t101 * n + i] = rq[0][2]; gm[t011 * n + i] = rq[1][2];
}

// ---------------------------------------------------------------------------
// Order-5 B-spline values and three derivatives (UniformBSpline.bSplineDerivatives),
// in the mesh precision S.
template <typename S>
__device__ __forceinline__ void bspline5(S x, S *out /* [5][4] */) {
  S w[5][6];
#pragma unroll
  for (int a = 0; a < 5; a++)
#pragma unroll
    for (int b = 0; b < 6; b++) w[a][b] = S(0);
  w[1][0] = S(1) - x;
  w[1][1] = x;
  w[2][0] = S(0.5) * (S(1) - x) * w[1][0];
  w[2][1] = S(0.5) * ((x + S(1)) * w[1][0] + (S(2) - x) * w[1][1]);
  w[2][2] = S(0.5) * x * w[1][1];
#pragma unroll
  for (int k = 3; k < 5; k++) {
    const S div = S(1) / (S)k;
    const S k1mw = (S)k + (S(1) - x);
    w[k][k] = div * x * w[k - 1][k - 1];
#pragma unroll
    for (int i = 1; i < k; i++) w[k][k - i] = div * ((x + (S)i) * w[k - 1][k - 1 - i] + (k1mw - (S)i) * w[k - 1][k - i]);
    w[k][0] = div * (S(1) - x) * w[k - 1][0];
  }
  // bSplineDiff(work[o2], o1); (work[o3], o2), (o3, o1); (o4, o3), (o4, o2), (o4, o1) with order 5.
  auto diff = [](S *c, int order) {
    const int o1 = order - 1;
    c[order] = c[o1];
    for (int i = o1; i > 0; i--) c[i] = c[i - 1] - c[i];
    c[0] = -c[0];
  };
  diff(w[3], 4);
  diff(w[2], 3); diff(w[2], 4);
  diff(w[1], 2); diff(w[1], 3); diff(w[1], 4);
#pragma unroll
  for (int k = 0; k < 5; k++)
#pragma unroll
    for (int j = 0; j < 4; j++) out[k * 4 + j] = w[4 - j][k];
}

template <typename S>
__device__ __forceinline__ void k_bsplines(VGrid vg, int n, const double *__restrict__ x, const double *__restrict__ y,
                           const double *__restrict__ z, const double *__restrict__ gm, int nfx, int nfy, int nfz,
                           S *spl, int *igrid, double *fm, const PmeConst &pc) {
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double xi = x[i], yi = y[i], zi = z[i];
  const int nf[3] = {nfx, nfy, nfz};
  double w[3];
  w[0] = xi * pc.recip[0][0] + yi * pc.recip[1][0] + zi * pc.recip[2][0];
  w[1] = xi * pc.recip[0][1] + yi * pc.recip[1][1] + zi * pc.recip[2][1];
  w[2] = xi * pc.recip[0][2] + yi * pc.recip[1][2] + zi * pc.recip[2][2];
  for (int d = 0; d < 3; d++) {
    const double u = w[d] - floor(w[d] + 0.5) + 0.5;
    const double fr = nf[d] * u;
    const int ifr = (int)fr;
    igrid[d * n + i] = ifr - kOrder;
    bspline5<S>((S)(fr - ifr), spl + ((size_t)i * 3 + d) * kOrder * 4);
  }
  double g[10];
#pragma unroll
  for (int j = 0; j < 10; j++) g[j] = gm[j * n + i];
  fm[i] = g[0];
#pragma unroll
  for (int j = 1; j < 4; j++) {
    double f = 0.0;
#pragma unroll
    for (int k = 1; k < 4; k++) f = fma(pc.tmm[j][k], g[k], f);
    fm[j * n + i] = f;
  }
#pragma unroll
  for (int j = 4; j < 10; j++) {
    double f = 0.0;
#pragma unroll
    for (int k = 4; k < 7; k++) f = fma(pc.tmm[j][k], g[k], f);
#pragma unroll
    for (int k = 7; k < 10; k++) f = fma(pc.tmm[j][k] * 2.0, g[k], f);
    fm[j * n + i] = f * (1.0 / 3.0);
  }
}

__device__ __forceinline__ int jmod(int a, int m) {
  int r = a % m;
  return r < 0 ? r + m : r;
}

// Mesh accumulation with FP64 atomics.  FP64 form: into the complex double mesh that the
// FFT transforms in place.  Mixed form: into two planes of doubles (real parts, then
// imaginary parts, ng points each), so that a warp's row of five support points touches
// two 32-byte sectors instead of three; each FP32 contribution is first rounded to a
// multiple of 2^-32, so sums of such values are exact in FP64 (below 2^21 in magnitude)
// and the accumulated mesh has the same bits whatever order the atoms arrive in.  The
// first FFT pass reads the planes and continues in FP32.
__device__ __forceinline__ double mesh_quantize(float v) {
  return rint((double)v * 4294967296.0) * 2.3283064365386962890625e-10;
}
// A mixed-form contribution of kQuantLimit or more raises FLAG_QUANT_RANGE (the first FFT
// pass checks the accumulated values as it reads them).
__device__ __forceinline__ void mesh_add(double2 *grid, size_t, size_t idx, double re, int *) {
  atomicAdd(&grid[idx].x, re);
}
__device__ __forceinline__ void mesh_add(double2 *grid, size_t, size_t idx, float re, int *flags) {
  if (quant_out(re)) atomicOr(flags, FLAG_QUANT_RANGE);
  atomicAdd(reinterpret_cast<double *>(grid) + idx, mesh_quantize(re));
}
__device__ __forceinline__ void mesh_add(double2 *grid, size_t, size_t idx, double re, double im, int *) {
  atomicAdd(&grid[idx].x, re);
  atomicAdd(&grid[idx].y, im);
}
__device__ __forceinline__ void mesh_add(double2 *grid, size_t ng, size_t idx, float re, float im, int *flags) {
  if (quant_out(re) || quant_out(im)) atomicOr(flags, FLAG_QUANT_RANGE);
  double *plane = reinterpret_cast<double *>(grid);
  atomicAdd(plane + idx, mesh_quantize(re));
  atomicAdd(plane + ng + idx, mesh_quantize(im));
}

// Wrap a support index (within one period of the mesh) into [0, m).
__device__ __forceinline__ int wrap1(int v, int m) { return v < 0 ? v + m : (v >= m ? v - m : v); }

// One warp per atom.  Lane l < 25 owns the (x, y) point (l % 5, l / 5) of the atom's
// support and walks the five z layers, so the per-point work is the B-spline product and
// the atomic add (no integer division in the loop).
template <typename S>
__device__ __forceinline__ void k_spread_permanent(VGrid vg, int n, const double *__restrict__ fm, const S *__restrict__ spl,
                                   const int *__restrict__ igrid, int nfx, int nfy, int nfz, double2 *grid,
                                   int *flags) {
  const int warp = (vg.bid * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n || lane >= 25) return;
  const int i = warp;
  const size_t ng = (size_t)nfx * nfy * nfz;
  const S *s = spl + (size_t)i * 3 * kOrder * 4;
  const S *sx = s, *sy = s + kOrder * 4, *sz = s + 2 * kOrder * 4;
  const int a1 = lane % 5, a2 = lane / 5;
  const int ii = wrap1(igrid[i] + 1 + a1, nfx), jj = wrap1(igrid[n + i] + 1 + a2, nfy);
  const int k0 = igrid[2 * n + i] + 1;
  S f[10];
#pragma unroll
  for (int j = 0; j < 10; j++) f[j] = (S)fm[j * n + i];
  const S x0 = sx[a1 * 4], x1 = sx[a1 * 4 + 1], x2 = sx[a1 * 4 + 2];
  const S u0 = sy[a2 * 4], u1 = sy[a2 * 4 + 1], u2 = sy[a2 * 4 + 2];
  const size_t row = (size_t)jj * nfx + ii;
#pragma unroll
  for (int a3 = 0; a3 < 5; a3++) {
    const S v0 = sz[a3 * 4], v1 = sz[a3 * 4 + 1], v2 = sz[a3 * 4 + 2];
    const S c0dz1qzz2 = f[t000] * v0 + f[t001] * v1 + f[t002] * v2;
    const S dy0qyz1 = f[t010] * v0 + f[t011] * v1;
    const S dx0qxz1 = f[t100] * v0 + f[t101] * v1;
    const S term0 = fma(c0dz1qzz2, u0, fma(dy0qyz1, u1, f[t020] * v0 * u2));
    const S term1 = fma(dx0qxz1, u0, f[t110] * v0 * u1);
    const S term2 = f[t200] * v0 * u0;
    const S val = fma(x0, term0, fma(x1, term1, x2 * term2));
    const int kk = wrap1(k0 + a3, nfz);
    mesh_add(grid, ng, (size_t)kk * nfy * nfx + row, val, flags);
  }
}

template <typename S>
__device__ __forceinline__ void k_spread_induced(
    VGrid vg, int const &n, const double *__restrict__ const &ud, const double *__restrict__ const &up,
    const S *__restrict__ const &spl, const int *__restrict__ const &igrid, int const &nfx, int const &nfy,
    int const &nfz, double2 * const &grid, const PmeConst &pc, int * const &flags) {
  const int warp = (vg.bid * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n || lane >= 25) return;
  const int i = warp;
  const size_t ng = (size_t)nfx * nfy * nfz;
  const S *s = spl + (size_t)i * 3 * kOrder * 4;
  const S *sx = s, *sy = s + kOrder * 4, *sz = s + 2 * kOrder * 4;
  const int a1 = lane % 5, a2 = lane / 5;
  const int ii = wrap1(igrid[i] + 1 + a1, nfx), jj = wrap1(igrid[n + i] + 1 + a2, nfy);
  const int k0 = igrid[2 * n + i] + 1;
  S u[3], q[3];
  const double c[3] = {ud[i], ud[n + i], ud[2 * n + i]};
  const double cp[3] = {up[i], up[n + i], up[2 * n + i]};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    u[a] = (S)(pc.afrac[a][0] * c[0] + pc.afrac[a][1] * c[1] + pc.afrac[a][2] * c[2]);
    q[a] = (S)(pc.afrac[a][0] * cp[0] + pc.afrac[a][1] * cp[1] + pc.afrac[a][2] * cp[2]);
  }
  const S x0 = sx[a1 * 4], x1 = sx[a1 * 4 + 1];
  const S u0 = sy[a2 * 4], u1 = sy[a2 * 4 + 1];
  // Per (x, y) point the z-layer value is  v0 * A + v1 * B  for each set.
  const S Ad = x0 * u[1] * u1 + x1 * u[0] * u0, Bd = x0 * u[2] * u0;
  const S Ap = x0 * q[1] * u1 + x1 * q[0] * u0, Bp = x0 * q[2] * u0;
  const size_t row = (size_t)jj * nfx + ii;
#pragma unroll
  for (int a3 = 0; a3 < 5; a3++) {
    const S v0 = sz[a3 * 4], v1 = sz[a3 * 4 + 1];
    const S re = fma(v0, Ad, v1 * Bd);
    const S im = fma(v0, Ap, v1 * Bp);
    const int kk = wrap1(k0 + a3, nfz);
    mesh_add(grid, ng, (size_t)kk * nfy * nfx + row, re, im, flags);
  }
}

// ---------------------------------------------------------------------------
// Batched line FFT in shared memory: a CTA transforms `L` lines of length `len`.
// Stockham self-sorting mixed-radix passes (radices 4, 2, 3, 5, 7), ping-pong
// between two shared buffers.  `tw` holds exp(-2*pi*i*j/len), j < len.

template <typename V2>
__device__ __forceinline__ V2 cmul(V2 a, V2 b) {
  V2 r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}

// Radix-R Stockham butterfly for one (line, j) pair.  R is a compile-time constant so
// the R values stay in registers; the small DFTs of R = 2, 3, 4 use their closed
// forms, R = 5 and 7 use the twiddle table.
// The twiddle table tw is in global memory (GTW: read through the read-only path) or in
// shared memory (the fixed-length kernels).
template <typename V2, bool GTW>
__device__ __forceinline__ V2 tw_at(const V2 *tw, int i) {
  if constexpr (GTW) return __ldg(tw + i);
  else return tw[i];
}

template <int R, typename S, bool GTW = false>
__device__ __forceinline__ void fft_butterfly(const typename Vec2<S>::type *in, typename Vec2<S>::type *out, int j,
                                              int l, int L, int nb, int Ns, int len, int sg,
                                              const typename Vec2<S>::type *__restrict__ tw) {
  using V2 = typename Vec2<S>::type;
  V2 v[R];
  const int k = j % Ns;
  const int tstep = len / (Ns * R);
#pragma unroll
  for (int r = 0; r < R; r++) {
    V2 a = in[(j + r * nb) * L + l];
    if (r > 0 && k > 0) {
      V2 w = tw_at<V2, GTW>(tw, r * k * tstep);
      if (sg > 0) w.y = -w.y;
      a = cmul(a, w);
    }
    v[r] = a;
  }
  const int idxD = (j / Ns) * Ns * R + k;
  V2 y[R];
  if (R == 2) {
    y[0] = mk2<S>(v[0].x + v[1].x, v[0].y + v[1].y);
    y[1] = mk2<S>(v[0].x - v[1].x, v[0].y - v[1].y);
  } else if (R == 4) {
    // W4 = exp(sg * i * pi / 2) = sg * i.
    const V2 s02 = mk2<S>(v[0].x + v[2].x, v[0].y + v[2].y);
    const V2 d02 = mk2<S>(v[0].x - v[2].x, v[0].y - v[2].y);
    const V2 s13 = mk2<S>(v[1].x + v[3].x, v[1].y + v[3].y);
    const V2 d13 = mk2<S>(v[1].x - v[3].x, v[1].y - v[3].y);
    // i * d13 = (-d13.y, d13.x)
    const V2 id13 = mk2<S>((S)(-sg) * d13.y, (S)sg * d13.x);
    y[0] = mk2<S>(s02.x + s13.x, s02.y + s13.y);
    y[1] = mk2<S>(d02.x + id13.x, d02.y + id13.y);
    y[2] = mk2<S>(s02.x - s13.x, s02.y - s13.y);
    y[3] = mk2<S>(d02.x - id13.x, d02.y - id13.y);
  } else if (R == 3) {
    const S c = S(-0.5), s = (S)sg * S(0.86602540378443864676);  // cos(2 pi / 3), sg * sin(2 pi / 3)
    const V2 t = mk2<S>(v[1].x + v[2].x, v[1].y + v[2].y);
    const V2 d = mk2<S>(v[1].x - v[2].x, v[1].y - v[2].y);
    y[0] = mk2<S>(v[0].x + t.x, v[0].y + t.y);
    const V2 m = mk2<S>(v[0].x + c * t.x, v[0].y + c * t.y);
    y[1] = mk2<S>(m.x - s * d.y, m.y + s * d.x);
    y[2] = mk2<S>(m.x + s * d.y, m.y - s * d.x);
  } else {
    const int wstep = len / R;
#pragma unroll
    for (int q = 0; q < R; q++) {
      V2 acc = v[0];
#pragma unroll
      for (int r = 1; r < R; r++) {
        V2 w = tw_at<V2, GTW>(tw, ((r * q) % R) * wstep);
        if (sg > 0) w.y = -w.y;
        const V2 m = cmul(v[r], w);
        acc.x += m.x; acc.y += m.y;
      }
      y[q] = acc;
    }
  }
#pragma unroll
  for (int q = 0; q < R; q++) out[(idxD + q * Ns) * L + l] = y[q];
}

// Radix-R pass for any R known only at run time (prime factors above 7, as the general
// pass of Complex.java:173-330 handles them): each output q of the length-R DFT is summed
// from the R twiddled inputs read from shared memory, O(R^2) per butterfly.
template <typename S, bool GTW = false>
__device__ __forceinline__ void fft_butterfly_any(int R, const typename Vec2<S>::type *in,
                                                  typename Vec2<S>::type *out, int j, int l, int L, int nb, int Ns,
                                                  int len, int sg, const typename Vec2<S>::type *__restrict__ tw) {
  using V2 = typename Vec2<S>::type;
  const int k = j % Ns;
  const int tstep = len / (Ns * R);
  const int wstep = len / R;
  const int idxD = (j / Ns) * Ns * R + k;
  for (int q = 0; q < R; q++) {
    V2 acc = in[j * L + l];
    for (int r = 1; r < R; r++) {
      V2 a = in[(j + r * nb) * L + l];
      if (k > 0) {
        V2 w = tw_at<V2, GTW>(tw, r * k * tstep);
        if (sg > 0) w.y = -w.y;
        a = cmul(a, w);
      }
      V2 w = tw_at<V2, GTW>(tw, ((r * q) % R) * wstep);
      if (sg > 0) w.y = -w.y;
      a = cmul(a, w);
      acc.x += a.x;
      acc.y += a.y;
    }
    out[(idxD + q * Ns) * L + l] = acc;
  }
}

// FROMD (mixed form, first pass only): the input is the double accumulation mesh `src`
// (real plane, then imaginary plane at src + src_ng), converted to FP32 on load and
// cleared behind the read, so that the next spread starts from zero without a memset.
template <bool FUSE_G, typename S, bool FROMD>
__device__ __forceinline__ void k_fft_axis(VGrid vg, typename Vec2<S>::type *grid, const FftAxis &ax, int sign,
                                                  const typename Vec2<S>::type *__restrict__ tw,
                                                  const S *__restrict__ G, int gnx, int gny,
                                                  double *src, size_t src_ng, int *flags) {
  using V2 = typename Vec2<S>::type;
  // Shared layout is element-major, line-minor: buf[j * L + l].  Consecutive threads
  // take consecutive lines, so butterflies are bank-conflict free and the Y and Z
  // passes (adjacent lines adjacent in memory) load and store coalesced.
  extern __shared__ __align__(16) unsigned char sm_raw[];
  V2 *sm = reinterpret_cast<V2 *>(sm_raw);
  const int len = ax.len, L = ax.L;
  V2 *buf0 = sm, *buf1 = sm + (size_t)len * L;
  const int gi = vg.bid % ax.groups_inner, go = vg.bid / ax.groups_inner;
  const size_t base = (size_t)gi * ax.group_step_inner + (size_t)go * ax.group_step_outer;
  const bool contiguous = (ax.stride == 1);
  for (int t = threadIdx.x; t < len * L; t += blockDim.x) {
    const int l = contiguous ? t / len : t % L, j = contiguous ? t % len : t / L;
    const size_t g = base + (size_t)l * ax.line_step + (size_t)j * ax.stride;
    if (FROMD) {
      const double2 q = make_double2(src[g], src[src_ng + g]);
      if (quant_out(q.x) || quant_out(q.y)) atomicOr(flags, FLAG_QUANT_RANGE);
      src[g] = 0.0;
      src[src_ng + g] = 0.0;
      buf0[j * L + l] = mk2<S>((S)q.x, (S)q.y);
    } else {
      buf0[j * L + l] = grid[g];
    }
  }
  __syncthreads();
  V2 *in = buf0, *out = buf1;
  const int npass = FUSE_G ? 2 : 1;
  for (int pass = 0; pass < npass; pass++) {
    const int sg = (pass == 0) ? sign : -sign;
    int Ns = 1;
    for (int st = 0; st < ax.nradix; st++) {
      const int R = ax.radix[st];
      const int nb = len / R;
      for (int t = threadIdx.x; t < nb * L; t += blockDim.x) {
        const int l = t % L, j = t / L;
        switch (R) {
          case 4: fft_butterfly<4, S, true>(in, out, j, l, L, nb, Ns, len, sg, tw); break;
          case 2: fft_butterfly<2, S, true>(in, out, j, l, L, nb, Ns, len, sg, tw); break;
          case 3: fft_butterfly<3, S, true>(in, out, j, l, L, nb, Ns, len, sg, tw); break;
          case 5: fft_butterfly<5, S, true>(in, out, j, l, L, nb, Ns, len, sg, tw); break;
          case 7: fft_butterfly<7, S, true>(in, out, j, l, L, nb, Ns, len, sg, tw); break;
          default: fft_butterfly_any<S, true>(R, in, out, j, l, L, nb, Ns, len, sg, tw); break;
        }
      }
      __syncthreads();
      V2 *tmp = in; in = out; out = tmp;
      Ns *= R;
    }
    if (FUSE_G && pass == 0) {
      // Influence function: lines run along z at fixed (x, y) = base + l (line_step 1).
      for (int t = threadIdx.x; t < len * L; t += blockDim.x) {
        const int l = t % L, j = t / L;
        const S g = __ldg(G + (size_t)j * gnx * gny + base + (size_t)l * ax.line_step);
        in[j * L + l].x *= g;
        in[j * L + l].y *= g;
      }
      __syncthreads();
    }
  }
  for (int t = threadIdx.x; t < len * L; t += blockDim.x) {
    const int l = contiguous ? t / len : t % L, j = contiguous ? t % len : t / L;
    grid[base + (size_t)l * ax.line_step + (size_t)j * ax.stride] = in[j * L + l];
  }
}

// Fixed-length line FFT (length LEN known at compile time, L lines per CTA, 256
// threads).  The same Stockham passes as k_fft_axis, but every index division is by a
// constant and the twiddle table sits in shared memory: at 64^3 the runtime-length
// kernel spends most of its issue slots on integer division.
__host__ __device__ constexpr int plan_radix(int len, int st) {
  int m = len;
  const int f[5] = {4, 2, 3, 5, 7};
  for (int q = 0; q < 5; q++)
    while (m % f[q] == 0) {
      if (st == 0) return f[q];
      st--;
      m /= f[q];
    }
  return 0;
}

// LS: the element stride of the shared layout (L, or L + 1 to spread a line's elements
// over the banks when lines are loaded along their elements).
template <int LEN, int ST, int NS, int L, typename S, int LS = L>
__device__ __forceinline__ void fixed_stages(typename Vec2<S>::type *&in, typename Vec2<S>::type *&out,
                                             const typename Vec2<S>::type *tw, int sg) {
  constexpr int R = plan_radix(LEN, ST);
  if constexpr (R != 0) {
    constexpr int NB = LEN / R;
    for (int t = threadIdx.x; t < NB * L; t += 256) {
      const int l = t % L, j = t / L;
      fft_butterfly<R, S>(in, out, j, l, LS, NB, NS, LEN, sg, tw);
    }
    __syncthreads();
    typename Vec2<S>::type *tmp = in;
    in = out;
    out = tmp;
    fixed_stages<LEN, ST + 1, NS * R, L, S, LS>(in, out, tw, sg);
  }
}

// Two-dimensional FFT of the 64 x 64 (x, y) planes of an FP32 mesh by a cluster of four
// CTAs per z plane.  Forward: CTA c transforms rows y in [16c, 16c + 16) along x, the
// cluster synchronises, and CTA c gathers columns x in [16c, 16c + 16) of every row from
// the four CTAs' shared memory and transforms them along y.  Inverse: the same with the
// axes swapped (y first, then x).  Two mesh passes become one launch, and the exchange
// between them stays on chip.  FROMD (forward only): the input is the planar double
// accumulation mesh (real plane, imaginary plane at + src_ng), which is cleared behind
// the read so that the next spread starts from zero.
template <bool INVERSE, bool FROMD>
__global__ void __cluster_dims__(4, 1, 1) __launch_bounds__(256)
    k_fft_plane64(float2 *grid, int sign, const float2 *__restrict__ twg, double *src, size_t src_ng, int *flags) {
  constexpr int LEN = 64, L = 16, LS = L + 1, NP = LEN * L, NB = LEN * LS, PER = NP / 256;
  __shared__ float2 buf[3][NB];
  __shared__ float2 tw[LEN];
  cg::cluster_group cluster = cg::this_cluster();
  const int c = (int)cluster.block_rank();
  const size_t plane = (size_t)(blockIdx.x >> 2) * LEN * LEN;
  for (int t = threadIdx.x; t < LEN; t += 256) tw[t] = twg[t];
  // Phase A lines: rows [16c, 16c + 16) along x (forward) or columns (inverse), stored
  // element-major, line-minor with stride LS: a[j * LS + l].  All loads of a thread are
  // issued before any store.
  {
    float2 v[PER];
    size_t g[PER];
    int at[PER];
#pragma unroll
    for (int u = 0; u < PER; u++) {
      const int t = threadIdx.x + 256 * u;
      int j, l;
      if (!INVERSE) {   // row l = t / 64, element x = t % 64 (coalesced rows)
        l = t / LEN; j = t % LEN;
        g[u] = plane + (size_t)(16 * c + l) * LEN + j;
      } else {          // column x = 16c + t % 16, element y = t / 16
        l = t % L; j = t / L;
        g[u] = plane + (size_t)j * LEN + 16 * c + l;
      }
      at[u] = j * LS + l;
      if (FROMD) {
        const double re = src[g[u]], im = src[src_ng + g[u]];
        if (quant_out(re) || quant_out(im)) atomicOr(flags, FLAG_QUANT_RANGE);
        v[u] = make_float2((float)re, (float)im);
      } else {
        v[u] = grid[g[u]];
      }
    }
#pragma unroll
    for (int u = 0; u < PER; u++) {
      if (FROMD) {
        src[g[u]] = 0.0;
        src[src_ng + g[u]] = 0.0;
      }
      buf[0][at[u]] = v[u];
    }
  }
  __syncthreads();
  float2 *in = buf[0], *out = buf[1];
  fixed_stages<LEN, 0, 1, L, float, LS>(in, out, tw, sign);
  // The first phase's result sits at the same offset in every CTA of the cluster.
  const int res = (int)((in - &buf[0][0]) / NB);
  const int spare = (res == 0) ? 1 : 0;
  cluster.sync();
  // Phase B lines: the other axis, gathered from the four CTAs into buf[2].  Forward:
  // element y = j of column x = 16c + l lives in CTA y / 16 as its row y % 16, element x.
  // Inverse: element x = j of row y = 16c + l lives in CTA x / 16 as its column x % 16,
  // element y.  Both sit at [(16c + l) * LS + j % 16] of the owner.
  {
    float2 v[PER];
#pragma unroll
    for (int u = 0; u < PER; u++) {
      const int t = threadIdx.x + 256 * u;
      const int l = t % L, j = t / L;
      const float2 *peer = cluster.map_shared_rank(&buf[res][0], j >> 4);
      v[u] = peer[(16 * c + l) * LS + (j & 15)];
    }
#pragma unroll
    for (int u = 0; u < PER; u++) {
      const int t = threadIdx.x + 256 * u;
      buf[2][(t / L) * LS + t % L] = v[u];
    }
  }
  cluster.sync();   // every peer has read this CTA's phase-A result
  in = buf[2];
  out = buf[spare];
  fixed_stages<LEN, 0, 1, L, float, LS>(in, out, tw, sign);
  for (int t = threadIdx.x; t < NP; t += 256) {
    size_t g;
    int j, l;
    if (!INVERSE) {   // column x = 16c + t % 16, element y = t / 16
      l = t % L; j = t / L;
      g = plane + (size_t)j * LEN + 16 * c + l;
    } else {          // row y = 16c + t / 64, element x = t % 64
      l = t / LEN; j = t % LEN;
      g = plane + (size_t)(16 * c + l) * LEN + j;
    }
    grid[g] = in[j * LS + l];
  }
}

template <int LEN, int L, bool FUSE_G, typename S, bool FROMD>
__device__ __forceinline__ void k_fft_fixed(VGrid vg, typename Vec2<S>::type *grid, const FftAxis &ax, int sign,
                                                   const typename Vec2<S>::type *__restrict__ twg,
                                                   const S *__restrict__ G, int gnx, int gny,
                                                   double *src, size_t src_ng, int *flags) {
  using V2 = typename Vec2<S>::type;
  __shared__ V2 buf[2][LEN * L];
  __shared__ V2 tw[LEN];
  for (int t = threadIdx.x; t < LEN; t += 256) tw[t] = twg[t];
  const int gi = vg.bid % ax.groups_inner, go = vg.bid / ax.groups_inner;
  const size_t base = (size_t)gi * ax.group_step_inner + (size_t)go * ax.group_step_outer;
  const bool contiguous = (ax.stride == 1);
  for (int t = threadIdx.x; t < LEN * L; t += 256) {
    const int l = contiguous ? t / LEN : t % L, j = contiguous ? t % LEN : t / L;
    const size_t g = base + (size_t)l * ax.line_step + (size_t)j * ax.stride;
    if (FROMD) {
      const double2 q = make_double2(src[g], src[src_ng + g]);
      if (quant_out(q.x) || quant_out(q.y)) atomicOr(flags, FLAG_QUANT_RANGE);
      src[g] = 0.0;
      src[src_ng + g] = 0.0;
      buf[0][j * L + l] = mk2<S>((S)q.x, (S)q.y);
    } else {
      buf[0][j * L + l] = grid[g];
    }
  }
  __syncthreads();
  V2 *in = buf[0], *out = buf[1];
  fixed_stages<LEN, 0, 1, L, S>(in, out, tw, sign);
  if (FUSE_G) {
    for (int t = threadIdx.x; t < LEN * L; t += 256) {
      const int l = t % L, j = t / L;
      const S gv = G[(size_t)j * gnx * gny + base + (size_t)l * ax.line_step];
      in[j * L + l].x *= gv;
      in[j * L + l].y *= gv;
    }
    __syncthreads();
    fixed_stages<LEN, 0, 1, L, S>(in, out, tw, -sign);
  }
  for (int t = threadIdx.x; t < LEN * L; t += 256) {
    const int l = contiguous ? t / LEN : t % L, j = contiguous ? t % LEN : t / L;
    grid[base + (size_t)l * ax.line_step + (size_t)j * ax.stride] = in[j * L + l];
  }
}

// ---------------------------------------------------------------------------
// Sum over the 32 lanes of v[0 .. 32): after a halving butterfly (16 + 8 + 4 + 2 + 1
// shuffles instead of five per value) lane l holds the total of entry l.  Fixed order.
template <typename S>
__device__ __forceinline__ S lane_totals32(S (&v)[32]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    const bool upper = (lane & s) != 0;
#pragma unroll
    for (int k = 0; k < s; k++) {
      const S send = upper ? v[k] : v[k + s];
      const S keep = upper ? v[k + s] : v[k];
      v[k] = keep + __shfl_xor_sync(0xffffffffu, send, s);
    }
  }
  return v[0];
}

// Potential and its derivatives at each atom from the mesh (real or imaginary part), one
// warp per atom: lane l < 25 owns the (x, y) support column (l % 5, l / 5) and walks the
// five z layers, then the lanes' partial sums are totalled with lane_totals32 (lane t
// holds term t).  The reference's order of terms (ReciprocalSpace.java:2506-2775).
template <int NT, typename S>
__device__ __forceinline__ S phi_terms_warp(int i, int n, const S *__restrict__ spl, const int *__restrict__ igrid,
                                            const typename Vec2<S>::type *__restrict__ grid, int nfx, int nfy,
                                            int nfz, bool imag) {
  const int lane = threadIdx.x & 31;
  S v[32];
#pragma unroll
  for (int t = 0; t < 32; t++) v[t] = S(0);
  if (lane < 25) {
    const S *sp = spl + (size_t)i * 3 * kOrder * 4;
    const S *sx = sp + (lane % 5) * 4, *sy = sp + kOrder * 4 + (lane / 5) * 4, *sz = sp + 2 * kOrder * 4;
    const int ii = wrap1(igrid[i] + 1 + lane % 5, nfx), jj = wrap1(igrid[n + i] + 1 + lane / 5, nfy);
    const int k0 = igrid[2 * n + i] + 1;
    const S x0 = sx[0], x1 = sx[1], x2 = sx[2], x3 = sx[3];
    const S y0 = sy[0], y1 = sy[1], y2 = sy[2], y3 = sy[3];
    const S a00 = x0 * y0, a10 = x1 * y0, a01 = x0 * y1, a20 = x2 * y0, a02 = x0 * y2, a11 = x1 * y1;
    const S a30 = x3 * y0, a03 = x0 * y3, a21 = x2 * y1, a12 = x1 * y2;
    const auto *col = grid + (size_t)jj * nfx + ii;
#pragma unroll
    for (int a3 = 0; a3 < kOrder; a3++) {
      const auto gv = col[(size_t)wrap1(k0 + a3, nfz) * nfy * nfx];
      const S q = imag ? gv.y : gv.x;
      const S q0 = q * sz[a3 * 4], q1 = q * sz[a3 * 4 + 1];
      v[t000] = fma(a00, q0, v[t000]); v[t100] = fma(a10, q0, v[t100]);
      v[t010] = fma(a01, q0, v[t010]); v[t001] = fma(a00, q1, v[t001]);
      if (NT > 4) {
        const S q2 = q * sz[a3 * 4 + 2], q3 = q * sz[a3 * 4 + 3];
        v[t200] = fma(a20, q0, v[t200]); v[t020] = fma(a02, q0, v[t020]);
        v[t002] = fma(a00, q2, v[t002]); v[t110] = fma(a11, q0, v[t110]);
        v[t101] = fma(a10, q1, v[t101]); v[t011] = fma(a01, q1, v[t011]);
        v[t300] = fma(a30, q0, v[t300]); v[t030] = fma(a03, q0, v[t030]);
        v[t003] = fma(a00, q3, v[t003]); v[t210] = fma(a21, q0, v[t210]);
        v[t201] = fma(a20, q1, v[t201]); v[t120] = fma(a12, q0, v[t120]);
        v[t021] = fma(a02, q1, v[t021]); v[t102] = fma(a10, q2, v[t102]);
        v[t012] = fma(a01, q2, v[t012]); v[t111] = fma(a11, q1, v[t111]);
      }
    }
  }
  return lane_totals32<S>(v);
}

// fphi (fractional terms, lane t < NT writes term t) and cphi (Cartesian: lane j < 10
// transforms the terms it gathers from the lanes that hold them).
template <int NT, typename S>
__device__ __forceinline__ void store_phi_warp(int i, int n, S term, double *fphi, double *cphi, const PmeConst &pc) {
  const int lane = threadIdx.x & 31;
  const double tv = (double)term;
  if (fphi && lane < NT) fphi[(size_t)lane * n + i] = tv;
  double g[10];
#pragma unroll
  for (int k = 0; k < 10; k++) g[k] = __shfl_sync(0xffffffffu, tv, k);
  double c = 0.0;
  if (lane == 0) {
    c = pc.tfm[0][0] * g[0];
  } else if (lane < 4) {
#pragma unroll
    for (int k = 1; k < 4; k++) c = fma(pc.tfm[lane][k], g[k], c);
  } else if (lane < 10 && NT > 4) {
#pragma unroll
    for (int k = 4; k < 10; k++) c = fma(pc.tfm[lane][k], g[k], c);
  }
  if (lane < (NT > 4 ? 10 : 4)) cphi[(size_t)lane * n + i] = c;
}

template <int NT, typename S>
__device__ __forceinline__ void k_phi(VGrid vg, int n, const S *__restrict__ spl, const int *__restrict__ igrid,
                                             const typename Vec2<S>::type *__restrict__ grid, int nfx, int nfy,
                                             int nfz, double *fphiR, double *cphiR, double *fphiI, double *cphiI,
                                             const PmeConst &pc) {
  const int i = (vg.bid * blockDim.x + threadIdx.x) >> 5;
  if (i >= n) return;
  store_phi_warp<NT, S>(i, n, phi_terms_warp<NT, S>(i, n, spl, igrid, grid, nfx, nfy, nfz, false), fphiR, cphiR, pc);
  if (cphiI)
    store_phi_warp<NT, S>(i, n, phi_terms_warp<NT, S>(i, n, spl, igrid, grid, nfx, nfy, nfz, true), fphiI, cphiI,
                          pc);
}

// ---------------------------------------------------------------------------
// Host set-up: transform matrices (ReciprocalSpace.java:1123-1210), twiddles and the
// generalized influence function with zeta-corrected B-spline moduli (:435-492, :1045-1121).
static void bspline_coeffs_host(double x, int order, double *c) {
  double w[16] = {0};
  w[0] = 1.0 - x;
  w[1] = x;
  for (int k = 2; k < order; k++) {
    double t[16] = {0};
    const double div = 1.0 / (double)k;
    const double k1mw = k + (1.0 - x);
    t[k] = div * x * w[k - 1];
    for (int i = 1; i < k; i++) t[k - i] = div * ((x + (double)i) * w[k - 1 - i] + (k1mw - (double)i) * w[k - i]);
    t[0] = div * (1.0 - x) * w[0];
    std::memcpy(w, t, sizeof(w));
  }
  for (int k = 0; k < order; k++) c[k] = w[k];
}

static std::vector<double> bsmod_host(int nfft, int order, const std::vector<double> &bsarray) {
  const double PI = 3.14159265358979323846;
  std::vector<double> bsmod(nfft);
  double factor = 2.0 * PI / nfft;
  for (int i = 0; i < nfft; i++) {
    double s1 = 0.0, s2 = 0.0;
    for (int j = 0; j < nfft; j++) {
      const double arg = factor * (double)(i * j);
      s1 = s1 + bsarray[j] * std::cos(arg);
      s2 = s2 + bsarray[j] * std::sin(arg);
    }
    bsmod[i] = s1 * s1 + s2 * s2;
  }
  const double eps = 1.0e-7;
  if (bsmod[0] < eps) bsmod[0] = 0.5 * bsmod[1];
  for (int i = 1; i < nfft - 1; i++)
    if (bsmod[i] < eps) bsmod[i] = 0.5 * (bsmod[i - 1] + bsmod[i + 1]);
  if (bsmod[nfft - 1] < eps) bsmod[nfft - 1] = 0.5 * bsmod[nfft - 2];
  for (int i = 0; i < nfft; i++) {
    int k = i;
    if (i > nfft / 2) k = k - nfft;
    double zeta = 1.0;
    if (k != 0) {
      double sum1 = 1.0, sum2 = 1.0;
      const double fct = PI * k / nfft;
      for (int j = 0; j < 50; j++) {
        const double arg = fct / (fct + PI * (j + 1));
        sum1 = sum1 + std::pow(arg, order);
        sum2 = sum2 + std::pow(arg, 2 * order);
      }
      for (int j = 0; j < 50; j++) {
        const double arg = fct / (fct - PI * (j + 1));
        sum1 = sum1 + std::pow(arg, order);
        sum2 = sum2 + std::pow(arg, 2 * order);
      }
      zeta = sum2 / sum1;
    }
    bsmod[i] = bsmod[i] * zeta * zeta;
  }
  return bsmod;
}

static FftAxis make_axis(int axis, const int nf[3]) {
  FftAxis a{};
  const int nx = nf[0], ny = nf[1];
  a.len = nf[axis];
  int m = a.len;
  a.nradix = 0;
  for (int f : {4, 2, 3, 5, 7}) {
    while (m % f == 0) { a.radix[a.nradix++] = f; m /= f; }
  }
  for (int f = 11; m > 1 && a.nradix < 12; f += 2) {   // remaining primes: the general pass
    while (m % f == 0 && a.nradix < 12) { a.radix[a.nradix++] = f; m /= f; }
  }
  // Lines of a CTA: consecutive along the fastest index that is not the transform axis;
  // up to 1,024 elements for short lines (a whole plane of a small mesh per CTA, so that
  // the 256 threads have work in every stage), else 16 lines.  Length 64 keeps 16: the
  // fixed-length kernel takes exactly that shape.
  const int inner = (axis == 0) ? ny : nx;
  int L = 1;
  const int cap = (a.len == 64) ? 16 : std::max(1, std::max(std::min(16, 4096 / a.len), std::min(64, 1024 / a.len)));
  for (int d = 1; d <= cap; d++)
    if (inner % d == 0) L = d;
  a.L = L;
  if (axis == 0) {          // lines (y, z); elements contiguous
    a.stride = 1; a.line_step = nx;
    a.groups_inner = ny / L; a.group_step_inner = L * nx; a.group_step_outer = nx * ny;
  } else if (axis == 1) {   // lines (x, z); elements stride nx
    a.stride = nx; a.line_step = 1;
    a.groups_inner = nx / L; a.group_step_inner = L; a.group_step_outer = nx * ny;
  } else {                  // lines (x, y); elements stride nx*ny
    a.stride = nx * ny; a.line_step = 1;
    a.groups_inner = nx / L; a.group_step_inner = L; a.group_step_outer = nx;
  }
  return a;
}


// The dynamic shared-memory limit of the generic FFT kernels is an attribute of each kernel
// on a device, shared by every handle in the process.  It only ever grows: a handle raises
// it to the largest line batch of its three axes, so a handle created later (with smaller
// axes, or its largest axis in another position) never lowers a limit on which an earlier
// handle's launches rely.
static std::mutex g_fft_smem_mu;
static std::map<int, int> g_fft_smem;   // device -> current attribute value (bytes)

// The generic FFT pass as launched by fft_convolution, with its argument types fixed so
// that the instances whose shared-memory limit raise_fft_smem sets are the ones launched.
template <bool FUSE, typename S, bool FROMD>
struct FftAxisPass {
  using V = typename Vec2<S>::type;
  static void launch(Handle &h, int blocks, size_t smem, V *grid, FftAxis a, int sign, const V *tw, const S *infl,
                     int nfx, int nfy, double *plane, size_t ng) {
    launch_on<k_fft_axis<FUSE, S, FROMD>, 256, 0>(h.rec, blocks, 256, smem, h.stream, grid, a, sign, tw, infl, nfx,
                                                  nfy, plane, ng, h.d_flags);
  }
  static cudaError_t raise(int need) {
    const cudaError_t e1 = cudaFuncSetAttribute(
        one_fn<k_fft_axis<FUSE, S, FROMD>, 256, 0, V *, FftAxis, int, const V *, const S *, int, int, double *, size_t,
               int *>(),
        cudaFuncAttributeMaxDynamicSharedMemorySize, need);
    const cudaError_t e2 = cudaFuncSetAttribute(
        many_fn<k_fft_axis<FUSE, S, FROMD>, 256, 0, V *, FftAxis, int, const V *, const S *, int, int, double *, size_t,
                int *>(),
        cudaFuncAttributeMaxDynamicSharedMemorySize, need);
    return e1 != cudaSuccess ? e1 : e2;
  }
};

static cudaError_t raise_fft_smem(int device, int need) {
  std::lock_guard<std::mutex> lock(g_fft_smem_mu);
  int &cur = g_fft_smem[device];
  if (need <= cur) return cudaSuccess;
  const cudaError_t e[5] = {FftAxisPass<false, double, false>::raise(need), FftAxisPass<true, double, false>::raise(need),
                            FftAxisPass<false, float, false>::raise(need), FftAxisPass<false, float, true>::raise(need),
                            FftAxisPass<true, float, false>::raise(need)};
  for (cudaError_t q : e)
    if (q != cudaSuccess) return q;
  cur = need;
  return cudaSuccess;
}

// Dynamic shared memory of one generic FFT pass over axis a (both sizes of the mesh type
// fit in the FP64 figure).
static size_t fft_axis_smem(const FftAxis &a) { return 2 * (size_t)a.len * a.L * sizeof(double2); }

int setup_pme(Handle &h) {
  const int nfx = h.prm.pme_grid[0], nfy = h.prm.pme_grid[1], nfz = h.prm.pme_grid[2];
  h.nfft[0] = nfx; h.nfft[1] = nfy; h.nfft[2] = nfz;
  const int nf[3] = {nfx, nfy, nfz};
  // Crystal.A: lower triangular (zero off the diagonal for an orthorhombic cell).
  const double A[3][3] = {{h.box.A00, 0, 0}, {h.box.A10, h.box.A11, 0}, {h.box.A20, h.box.A21, h.box.A22}};
  static const int qi1[6] = {0, 1, 2, 0, 0, 1};
  static const int qi2[6] = {0, 1, 2, 1, 2, 2};
  double a[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) a[j][i] = nf[j] * A[i][j];
  std::memset(h.pc.tmm, 0, sizeof(h.pc.tmm));
  h.pc.tmm[0][0] = 1.0;
  for (int i = 1; i < 4; i++)
    for (int j = 0; j < 3; j++) h.pc.tmm[i][1 + j] = a[i - 1][j];
  for (int i1 = 0; i1 < 3; i1++)
    for (int i2 = 0; i2 < 6; i2++) h.pc.tmm[i1 + 4][i2 + 4] = a[qi1[i1]][qi1[i2]] * a[qi1[i1]][qi2[i2]];
  for (int i1 = 3; i1 < 6; i1++) {
    const int k = qi1[i1], l = qi2[i1];
    for (int i2 = 0; i2 < 6; i2++) {
      const int ii = qi1[i2], jj = qi2[i2];
      h.pc.tmm[i1 + 4][i2 + 4] = a[k][ii] * a[l][jj] + a[k][jj] * a[l][ii];
    }
  }
  double af[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) af[i][j] = nf[j] * A[i][j];
  std::memset(h.pc.tfm, 0, sizeof(h.pc.tfm));
  h.pc.tfm[0][0] = 1.0;
  for (int i = 1; i < 4; i++)
    for (int j = 0; j < 3; j++) h.pc.tfm[i][1 + j] = af[i - 1][j];
  for (int i1 = 0; i1 < 3; i1++) {
    const int k = qi1[i1];
    for (int i2 = 0; i2 < 3; i2++) h.pc.tfm[i1 + 4][i2 + 4] = af[k][qi1[i2]] * af[k][qi1[i2]];
    for (int i2 = 3; i2 < 6; i2++) h.pc.tfm[i1 + 4][i2 + 4] = 2.0 * af[k][qi1[i2]] * af[k][qi2[i2]];
  }
  for (int i1 = 3; i1 < 6; i1++) {
    const int k = qi1[i1], nn = qi2[i1];
    for (int i2 = 0; i2 < 3; i2++) h.pc.tfm[i1 + 4][i2 + 4] = af[k][qi1[i2]] * af[nn][qi1[i2]];
    for (int i2 = 3; i2 < 6; i2++) {
      const int ii = qi1[i2], jj = qi2[i2];
      h.pc.tfm[i1 + 4][i2 + 4] = af[k][ii] * af[nn][jj] + af[nn][ii] * af[k][jj];
    }
  }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) h.pc.afrac[i][j] = nf[i] * A[j][i];
  std::memcpy(h.pc.recip, A, sizeof(A));

  // Influence function.
  const int order = h.prm.pme_order;
  const int maxfft = std::max(std::max(std::max(nfx, nfy), nfz), order + 1);
  std::vector<double> bsarray(maxfft, 0.0);
  double c[16];
  bspline_coeffs_host(0.0, order, c);
  for (int i = 0; i < order; i++) bsarray[1 + i] = c[i];
  const std::vector<double> bx = bsmod_host(nfx, order, bsarray), by = bsmod_host(nfy, order, bsarray),
                            bz = bsmod_host(nfz, order, bsarray);
  const double PI = 3.14159265358979323846;
  const double aewald = h.prm.ewald_alpha;
  const double piTerm = (PI / aewald) * (PI / aewald);
  const double volTerm = PI * h.box.volume;
  std::vector<double> G((size_t)nfx * nfy * nfz, 0.0);
  const int nX2 = (nfx + 1) / 2, nY2 = (nfy + 1) / 2, nZ2 = (nfz + 1) / 2;
  for (int kz = 0; kz < nfz; kz++)
    for (int ky = 0; ky < nfy; ky++)
      for (int kx = 0; kx < nfx; kx++) {
        if (kx == 0 && ky == 0 && kz == 0) continue;
        int hh = kx, k = ky, l = kz;
        if (kx >= nX2) hh -= nfx;
        if (ky >= nY2) k -= nfy;
        if (kz >= nZ2) l -= nfz;
        const double sX = A[0][0] * hh + A[0][1] * k + A[0][2] * l;
        const double sY = A[1][0] * hh + A[1][1] * k + A[1][2] * l;
        const double sZ = A[2][0] * hh + A[2][1] * k + A[2][2] * l;
        const double s2 = sX * sX + sY * sY + sZ * sZ;
        const double term = -piTerm * s2;
        double e = 0.0;
        if (term > -50.0) e = std::exp(term) / (s2 * volTerm * bx[kx] * by[ky] * bz[kz]);
        G[((size_t)kz * nfy + ky) * nfx + kx] = e;
      }
  cudaMemcpy(h.d_influence, G.data(), G.size() * sizeof(double), cudaMemcpyHostToDevice);
  const int maxn = std::max(nfx, std::max(nfy, nfz));
  std::vector<double2> tw(3 * (size_t)maxn);
  for (int d = 0; d < 3; d++)
    for (int j = 0; j < nf[d]; j++) {
      const double ang = 2.0 * PI * (double)j / (double)nf[d];
      tw[(size_t)d * maxn + j] = make_double2(std::cos(ang), -std::sin(ang));
    }
  cudaMemcpy(h.d_twiddle, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice);
  if (h.mixed) {
    // The influence function and twiddles are computed in FP64 and rounded once.
    std::vector<float> Gf(G.size());
    for (size_t q = 0; q < G.size(); q++) Gf[q] = (float)G[q];
    std::vector<float2> twf(tw.size());
    for (size_t q = 0; q < tw.size(); q++) twf[q] = make_float2((float)tw[q].x, (float)tw[q].y);
    cudaMemcpy(h.d_influencef, Gf.data(), Gf.size() * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(h.d_twiddlef, twf.data(), twf.size() * sizeof(float2), cudaMemcpyHostToDevice);
  }
  for (int d = 0; d < 3; d++) h.axes[d] = make_axis(d, nf);
  size_t smem = 48 * 1024;
  for (int d = 0; d < 3; d++) smem = std::max(smem, fft_axis_smem(h.axes[d]));
  if (smem > 227 * 1024) {
    h.err = "PME grid dimension too long for the shared-memory FFT";
    return FFXG_ERR_BAD_ARG;
  }
  const cudaError_t e = raise_fft_smem(h.device, (int)smem);
  if (e != cudaSuccess) {
    h.err = std::string("FFT shared-memory attribute: ") + cudaGetErrorString(e);
    return FFXG_ERR_CUDA;
  }
  return FFXG_OK;
}

// ---------------------------------------------------------------------------
void launch_rotate(Handle &h) {
  launch_on<k_rotate, 0, 0>(h.rec, nblocks(h.n, 128), 128, 0, h.stream, h.n, (const double *)h.d_x,
                            (const double *)h.d_y, (const double *)h.d_z, (const int *)h.d_frame,
                            (const int *)h.d_axis, (const double *)h.d_lmp, h.d_gm, h.d_rot);
  FFX_LAUNCHED(h);
}

void launch_bsplines(Handle &h) {
  if (h.mixed)
    launch_on<k_bsplines<float>, 0, 0>(h.rec, nblocks(h.n, 128), 128, 0, h.stream, h.n, (const double *)h.d_x,
                                       (const double *)h.d_y, (const double *)h.d_z, (const double *)h.d_gm,
                                       h.nfft[0], h.nfft[1], h.nfft[2], reinterpret_cast<float *>(h.d_spl),
                                       h.d_igrid, h.d_fm, h.pc);
  else
    launch_on<k_bsplines<double>, 0, 0>(h.rec, nblocks(h.n, 128), 128, 0, h.stream, h.n, (const double *)h.d_x,
                                        (const double *)h.d_y, (const double *)h.d_z, (const double *)h.d_gm,
                                        h.nfft[0], h.nfft[1], h.nfft[2], h.d_spl, h.d_igrid, h.d_fm, h.pc);
  FFX_LAUNCHED(h);
}

static size_t grid_points(const Handle &h) { return (size_t)h.nfft[0] * h.nfft[1] * h.nfft[2]; }

// The FP64 mesh cleared before a spread.
__device__ __forceinline__ void k_clear_mesh(VGrid vg, size_t m, double2 *grid) {
  for (size_t j = (size_t)vg.bid * blockDim.x + threadIdx.x; j < m; j += (size_t)vg.nblk * blockDim.x)
    grid[j] = make_double2(0.0, 0.0);
}
static void clear_mesh(Handle &h) {
  const size_t m = grid_points(h);
  launch_on<k_clear_mesh, 0, 0>(h.rec, (int)std::min<size_t>(nblocks((int64_t)m, 256), 4 * (size_t)h.num_sms), 256, 0,
                                h.stream, m, h.d_grid);
  FFX_LAUNCHED(h);
}

// Both forms accumulate into the double mesh d_grid; the FP64 form clears it first, the
// mixed form keeps it clear between uses (its first FFT pass zeroes what it reads) and
// continues in the FP32 mesh d_gridf.
void launch_spread_permanent(Handle &h) {
  if (h.vacuum) return;   // no reciprocal space: the mesh and potentials stay zero
  const int nb = nblocks((int64_t)h.n * 32, 256);
  if (!h.mixed) clear_mesh(h);
  if (h.mixed)
    launch_on<k_spread_permanent<float>, 0, 0>(h.rec, nb, 256, 0, h.stream, h.n, (const double *)h.d_fm,
                                               reinterpret_cast<const float *>(h.d_spl), (const int *)h.d_igrid,
                                               h.nfft[0], h.nfft[1], h.nfft[2], h.d_grid, h.d_flags);
  else
    launch_on<k_spread_permanent<double>, 0, 0>(h.rec, nb, 256, 0, h.stream, h.n, (const double *)h.d_fm,
                                                (const double *)h.d_spl, (const int *)h.d_igrid, h.nfft[0],
                                                h.nfft[1], h.nfft[2], h.d_grid, h.d_flags);
  FFX_LAUNCHED(h);
}

void launch_spread_induced(Handle &h, const double *ud, const double *up) {
  if (h.vacuum) return;   // no reciprocal space: the mesh and potentials stay zero
  const int nb = nblocks((int64_t)h.n * 32, 256);
  if (!h.mixed) clear_mesh(h);
  if (h.mixed)
    launch_on<k_spread_induced<float>, 0, 0>(h.rec, nb, 256, 0, h.stream, h.n, ud, up,
                                             reinterpret_cast<const float *>(h.d_spl), (const int *)h.d_igrid,
                                             h.nfft[0], h.nfft[1], h.nfft[2], h.d_grid, h.pc, h.d_flags);
  else
    launch_on<k_spread_induced<double>, 0, 0>(h.rec, nb, 256, 0, h.stream, h.n, ud, up, (const double *)h.d_spl,
                                              (const int *)h.d_igrid, h.nfft[0], h.nfft[1], h.nfft[2], h.d_grid,
                                              h.pc, h.d_flags);
  FFX_LAUNCHED(h);
}

template <typename S>
static void fft_convolution(Handle &h, typename Vec2<S>::type *grid, const typename Vec2<S>::type *twiddle,
                            const S *influence) {
  using V = typename Vec2<S>::type;
  const int nfx = h.nfft[0], nfy = h.nfft[1], nfz = h.nfft[2];
  const int maxn = std::max(nfx, std::max(nfy, nfz));
  // The mixed form's accumulation mesh: real plane, then imaginary plane.
  double *plane = h.d_grid_planes();
  const size_t ng = (size_t)nfx * nfy * nfz;
  auto run = [&](int d, int sign, bool fuse, bool fromd) {
    const FftAxis &a = h.axes[d];
    const int outer = (d == 0) ? nfz : ((d == 1) ? nfz : nfy);
    const int blocks = a.groups_inner * outer;
    const size_t smem = 2 * (size_t)a.len * a.L * sizeof(V);
    const V *tw = twiddle + (size_t)d * maxn;
    const S *none = nullptr;
    if (a.len == 64 && a.L == 16) {
      if (fuse)
        launch_on<k_fft_fixed<64, 16, true, S, false>, 256, 0>(h.rec, blocks, 256, 0, h.stream, grid, a, sign, tw,
                                                               influence, nfx, nfy, (double *)nullptr, (size_t)0,
                                                               h.d_flags);
      else if (fromd)
        launch_on<k_fft_fixed<64, 16, false, S, true>, 256, 0>(h.rec, blocks, 256, 0, h.stream, grid, a, sign, tw,
                                                               none, nfx, nfy, plane, ng, h.d_flags);
      else
        launch_on<k_fft_fixed<64, 16, false, S, false>, 256, 0>(h.rec, blocks, 256, 0, h.stream, grid, a, sign, tw,
                                                                none, nfx, nfy, (double *)nullptr, (size_t)0,
                                                                h.d_flags);
      FFX_LAUNCHED(h);
      return;
    }
    if (fuse)
      FftAxisPass<true, S, false>::launch(h, blocks, smem, grid, a, sign, tw, influence, nfx, nfy, nullptr, 0);
    else if (fromd)
      FftAxisPass<false, S, true>::launch(h, blocks, smem, grid, a, sign, tw, none, nfx, nfy, plane, ng);
    else
      FftAxisPass<false, S, false>::launch(h, blocks, smem, grid, a, sign, tw, none, nfx, nfy, nullptr, 0);
    FFX_LAUNCHED(h);
  };
  const bool fromd = (sizeof(S) == 4);   // mixed: the first pass reads the double mesh
  if (sizeof(S) == 4 && nfx == 64 && nfy == 64 && h.axes[2].len == 64 && h.axes[2].L == 16 && !h.rec) {
    // Mixed form on 64 x 64 planes: xy, z (with the influence function), yx.  (A recorded
    // batch takes the per-axis passes instead: a cluster launch cannot span systems.)
    float2 *gf = reinterpret_cast<float2 *>(grid);
    const float2 *tw = reinterpret_cast<const float2 *>(twiddle);
    k_fft_plane64<false, true><<<nfz * 4, 256, 0, h.stream>>>(gf, -1, tw, h.d_grid_planes(), ng, h.d_flags);
    FFX_LAUNCHED(h);
    run(2, -1, true, false);
    k_fft_plane64<true, false><<<nfz * 4, 256, 0, h.stream>>>(gf, +1, tw, nullptr, 0, h.d_flags);
    FFX_LAUNCHED(h);
    return;
  }
  run(0, -1, false, fromd);
  run(1, -1, false, false);
  run(2, -1, true, false);
  run(1, +1, false, false);
  run(0, +1, false, false);
}

void launch_fft_convolution(Handle &h) {
  if (h.vacuum) return;   // no reciprocal space: the mesh and potentials stay zero
  if (h.mixed)
    fft_convolution<float>(h, h.d_gridf, h.d_twiddlef, h.d_influencef);
  else
    fft_convolution<double>(h, h.d_grid, h.d_twiddle, h.d_influence);
}

template <typename S>
static void phi(Handle &h, int which) {
  const S *spl = reinterpret_cast<const S *>(h.d_spl);
  const auto *grid = reinterpret_cast<const typename Vec2<S>::type *>(h.mixed ? (void *)h.d_gridf : (void *)h.d_grid);
  const int nb = nblocks((int64_t)h.n * 32, 256);
  if (which == 0)
    launch_on<k_phi<20, S>, 256, 0, sizeof(S) == 4 ? 6 : 3>(h.rec, nb, 256, 0, h.stream, h.n, spl, (const int *)h.d_igrid, grid, h.nfft[0],
                                    h.nfft[1], h.nfft[2], h.d_fphi, h.d_cphi, (double *)nullptr, (double *)nullptr,
                                    h.pc);
  else
    launch_on<k_phi<20, S>, 256, 0, sizeof(S) == 4 ? 6 : 3>(h.rec, nb, 256, 0, h.stream, h.n, spl, (const int *)h.d_igrid, grid, h.nfft[0],
                                    h.nfft[1], h.nfft[2], h.d_fphiI, h.d_cphiI, h.d_fphiP, h.d_cphiP, h.pc);
  FFX_LAUNCHED(h);
}

void launch_phi_permanent(Handle &h) {
  if (h.vacuum) return;   // no reciprocal space: the mesh and potentials stay zero
  if (h.mixed) phi<float>(h, 0); else phi<double>(h, 0);
}

void launch_phi_induced(Handle &h) {
  if (h.vacuum) return;   // no reciprocal space: the mesh and potentials stay zero
  if (h.mixed) phi<float>(h, 1); else phi<double>(h, 1);
}


// ===========================================================================
// Allocation-free permanent reciprocal-space potential (ffxg_pme_recip_permanent_noalloc).
//
// For callers that may not allocate device memory: a host process whose device
// memory is owned by another allocator (a framework's caching pool that has
// reserved the GPU, a JVM or plugin host that forbids new device allocations after
// start-up), or latency-critical callers that must not pay cudaMalloc's implicit
// synchronisation.  Inputs and outputs are the caller's device buffers; every
// intermediate (mesh, influence function, twiddles, B-spline moduli, partial
// sums) lives in the one file-scope array below, sized for at most
// kNaMaxAtoms atoms and a kNaMaxDim^3 mesh.  The array exists once per device
// that loads the library and is held until the process exits.
namespace {
constexpr int kNaMaxAtoms = 32768;
constexpr int kNaMaxDim = 64;
constexpr int kNaMaxPoints = kNaMaxDim * kNaMaxDim * kNaMaxDim;
constexpr int kNaThreads = 128;
constexpr int kNaPartials = kNaMaxAtoms / kNaThreads;   // one partial energy per phi block
constexpr int kNaMaxDevices = 64;

struct NoAllocScratch {
  double2 grid[kNaMaxPoints];        // complex mesh
  double influence[kNaMaxPoints];    // generalized influence function
  double2 twiddle[3 * kNaMaxDim];    // exp(-2 pi i j / n) per axis
  double bsmod[3 * kNaMaxDim];       // zeta-corrected B-spline moduli per axis
  double partial[kNaPartials];       // per-block energy sums
};
}  // namespace

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Device address of the array, looked up once per device.  In host code the name
// g_noalloc_scratch is only a host-side stand-in, never a device address.
static std::atomic<NoAllocScratch *> g_noalloc_ptr[kNaMaxDevices];

__device__ void na_bspline_coeffs(double x, double *c) {  // UniformBSpline.bSpline, order 5
  double w[6] = {1.0 - x, x, 0, 0, 0, 0};
  for (int k = 2; k < kOrder; k++) {
    double t[6] = {0, 0, 0, 0, 0, 0};
    const double div = 1.0 / (double)k;
    const double k1mw = k + (1.0 - x);
    t[k] = div * x * w[k - 1];
    for (int i = 1; i < k; i++) t[k - i] = div * ((x + (double)i) * w[k - 1 - i] + (k1mw - (double)i) * w[k - i]);
    t[0] = div * (1.0 - x) * w[0];
    for (int i = 0; i < 6; i++) w[i] = t[i];
  }
  for (int i = 0; i < kOrder; i++) c[i] = w[i];
}

// One block per axis: twiddles, raw moduli, the reference's sequential fix-ups of
// tiny moduli, then the zeta correction (ReciprocalSpace.discreteFTMod, :435-492).
__global__ void k_na_tables(int nx, int ny, int nz, NoAllocScratch *s) {
  const int d = blockIdx.x;
  const int nf = d == 0 ? nx : (d == 1 ? ny : nz);
  const int t = threadIdx.x;
  const double PI = 3.14159265358979323846;
  double *bsmod = s->bsmod + d * kNaMaxDim;
  if (t < nf) {
    double sn, cs;
    sincospi(2.0 * (double)t / (double)nf, &sn, &cs);
    s->twiddle[d * kNaMaxDim + t] = make_double2(cs, -sn);
    double c[kOrder];
    na_bspline_coeffs(0.0, c);
    const double factor = 2.0 * PI / nf;
    double s1 = 0.0, s2 = 0.0;
    for (int j = 0; j < nf; j++) {
      const double bj = (j >= 1 && j <= kOrder) ? c[j - 1] : 0.0;
      const double arg = factor * (double)(t * j);
      s1 = s1 + bj * cos(arg);
      s2 = s2 + bj * sin(arg);
    }
    bsmod[t] = s1 * s1 + s2 * s2;
  }
  __syncthreads();
  if (t == 0) {
    const double eps = 1.0e-7;
    if (bsmod[0] < eps) bsmod[0] = 0.5 * bsmod[1];
    for (int i = 1; i < nf - 1; i++)
      if (bsmod[i] < eps) bsmod[i] = 0.5 * (bsmod[i - 1] + bsmod[i + 1]);
    if (bsmod[nf - 1] < eps) bsmod[nf - 1] = 0.5 * bsmod[nf - 2];
  }
  __syncthreads();
  if (t < nf) {
    int k = t;
    if (t > nf / 2) k = k - nf;
    double zeta = 1.0;
    if (k != 0) {
      double sum1 = 1.0, sum2 = 1.0;
      const double fct = PI * k / nf;
      for (int j = 0; j < 50; j++) {
        const double arg = fct / (fct + PI * (j + 1));
        sum1 = sum1 + pow(arg, (double)kOrder);
        sum2 = sum2 + pow(arg, (double)(2 * kOrder));
      }
      for (int j = 0; j < 50; j++) {
        const double arg = fct / (fct - PI * (j + 1));
        sum1 = sum1 + pow(arg, (double)kOrder);
        sum2 = sum2 + pow(arg, (double)(2 * kOrder));
      }
      zeta = sum2 / sum1;
    }
    bsmod[t] = bsmod[t] * zeta * zeta;
  }
}

// Influence function (ReciprocalSpace.generalizedInfluenceFunction, :1045-1121) and a
// cleared mesh: every call starts from zero regardless of what the last call left.
__global__ void k_na_influence(int nx, int ny, int nz, double ax, double ay, double az, double aewald,
                               double volume, NoAllocScratch *s) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nx * ny * nz) return;
  s->grid[m] = make_double2(0.0, 0.0);
  const int kx = m % nx, ky = (m / nx) % ny, kz = m / (nx * ny);
  if (m == 0) { s->influence[0] = 0.0; return; }
  const double PI = 3.14159265358979323846;
  int h = kx, k = ky, l = kz;
  if (kx >= (nx + 1) / 2) h -= nx;
  if (ky >= (ny + 1) / 2) k -= ny;
  if (kz >= (nz + 1) / 2) l -= nz;
  const double sX = ax * h, sY = ay * k, sZ = az * l;
  const double s2 = sX * sX + sY * sY + sZ * sZ;
  const double term = -(PI / aewald) * (PI / aewald) * s2;
  double e = 0.0;
  if (term > -50.0)
    e = exp(term) / (s2 * (PI * volume) * s->bsmod[kx] * s->bsmod[kNaMaxDim + ky] * s->bsmod[2 * kNaMaxDim + kz]);
  s->influence[m] = e;
}

// Grid origin and order-5 splines of one coordinate (BSplineLoop, :1338-1412).
__device__ __forceinline__ int na_spline(double w, int nf, double *out) {
  const double u = w - floor(w + 0.5) + 0.5;
  const double fr = nf * u;
  const int ifr = (int)fr;
  bspline5<double>(fr - ifr, out);
  return ifr - kOrder;
}

// Warp per atom: lanes 0-2 build the three spline sets and lanes 0-9 the fractional
// multipole in shared memory, then all lanes spread the 125 mesh points.
__global__ void k_na_spread(int n, const double *__restrict__ xyz, const double *__restrict__ mpole, int nx, int ny,
                            int nz, PmeConst pc, NoAllocScratch *s) {
  __shared__ double sp[kNaThreads / 32][3][kOrder * 4];
  __shared__ double sfm[kNaThreads / 32][10];
  __shared__ int sg[kNaThreads / 32][3];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * (kNaThreads / 32) + wib;
  if (i >= n) return;
  const int nf[3] = {nx, ny, nz};
  if (lane < 3) {
    const double w = xyz[3 * i] * pc.recip[0][lane] + xyz[3 * i + 1] * pc.recip[1][lane] +
                     xyz[3 * i + 2] * pc.recip[2][lane];
    sg[wib][lane] = na_spline(w, nf[lane], sp[wib][lane]);
  }
  if (lane < 10) {
    const double *g = mpole + 10 * (size_t)i;
    double f = 0.0;
    if (lane == 0) {
      f = g[0];
    } else if (lane < 4) {
      for (int k = 1; k < 4; k++) f = fma(pc.tmm[lane][k], g[k], f);
    } else {
      for (int k = 4; k < 7; k++) f = fma(pc.tmm[lane][k], g[k], f);
      for (int k = 7; k < 10; k++) f = fma(pc.tmm[lane][k] * 2.0, g[k], f);
      f = f * (1.0 / 3.0);
    }
    sfm[wib][lane] = f;
  }
  __syncwarp();
  const double *sx = sp[wib][0], *sy = sp[wib][1], *sz = sp[wib][2];
  const double *f = sfm[wib];
  for (int p = lane; p < 125; p += 32) {
    const int a1 = p % 5, a2 = (p / 5) % 5, a3 = p / 25;
    const double v0 = sz[a3 * 4], v1 = sz[a3 * 4 + 1], v2 = sz[a3 * 4 + 2];
    const double u0 = sy[a2 * 4], u1 = sy[a2 * 4 + 1], u2 = sy[a2 * 4 + 2];
    const double c0dz1qzz2 = f[t000] * v0 + f[t001] * v1 + f[t002] * v2;
    const double dy0qyz1 = f[t010] * v0 + f[t011] * v1;
    const double dx0qxz1 = f[t100] * v0 + f[t101] * v1;
    const double term0 = fma(c0dz1qzz2, u0, fma(dy0qyz1, u1, f[t020] * v0 * u2));
    const double term1 = fma(dx0qxz1, u0, f[t110] * v0 * u1);
    const double term2 = f[t200] * v0 * u0;
    const double val = fma(sx[a1 * 4], term0, fma(sx[a1 * 4 + 1], term1, sx[a1 * 4 + 2] * term2));
    const int ii = jmod(sg[wib][0] + 1 + a1, nx), jj = jmod(sg[wib][1] + 1 + a2, ny), kk = jmod(sg[wib][2] + 1 + a3, nz);
    atomicAdd(&s->grid[((size_t)kk * ny + jj) * nx + ii].x, val);
  }
}

// Thread per atom: Cartesian potential and derivatives (10 terms, [n][10]) and the
// per-block sum of M . Phi (PermanentReciprocalEnergyLoop, :430-446).
__global__ void k_na_phi(int n, const double *__restrict__ xyz, const double *__restrict__ mpole, int nx, int ny,
                         int nz, PmeConst pc, double *phi_out, NoAllocScratch *s) {
  __shared__ double red[kNaThreads / 32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0;
  if (i < n) {
    const int nf[3] = {nx, ny, nz};
    double spl[3][kOrder * 4];
    int g0[3];
    for (int d = 0; d < 3; d++) {
      const double w = xyz[3 * i] * pc.recip[0][d] + xyz[3 * i + 1] * pc.recip[1][d] + xyz[3 * i + 2] * pc.recip[2][d];
      g0[d] = na_spline(w, nf[d], spl[d]);
    }
    double tuv[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int a3 = 0; a3 < kOrder; a3++) {
      const int kk = jmod(g0[2] + 1 + a3, nz);
      double tu00 = 0, tu10 = 0, tu01 = 0, tu20 = 0, tu11 = 0, tu02 = 0;
      for (int a2 = 0; a2 < kOrder; a2++) {
        const int jj = jmod(g0[1] + 1 + a2, ny);
        double t0 = 0, t1 = 0, t2 = 0;
        for (int a1 = 0; a1 < kOrder; a1++) {
          const int ii = jmod(g0[0] + 1 + a1, nx);
          const double tq = s->grid[((size_t)kk * ny + jj) * nx + ii].x;
          t0 = fma(tq, spl[0][a1 * 4], t0);
          t1 = fma(tq, spl[0][a1 * 4 + 1], t1);
          t2 = fma(tq, spl[0][a1 * 4 + 2], t2);
        }
        const double u0 = spl[1][a2 * 4], u1 = spl[1][a2 * 4 + 1], u2 = spl[1][a2 * 4 + 2];
        tu00 = fma(t0, u0, tu00); tu10 = fma(t1, u0, tu10); tu01 = fma(t0, u1, tu01);
        tu20 = fma(t2, u0, tu20); tu11 = fma(t1, u1, tu11); tu02 = fma(t0, u2, tu02);
      }
      const double v0 = spl[2][a3 * 4], v1 = spl[2][a3 * 4 + 1], v2 = spl[2][a3 * 4 + 2];
      tuv[t000] = fma(tu00, v0, tuv[t000]); tuv[t100] = fma(tu10, v0, tuv[t100]);
      tuv[t010] = fma(tu01, v0, tuv[t010]); tuv[t001] = fma(tu00, v1, tuv[t001]);
      tuv[t200] = fma(tu20, v0, tuv[t200]); tuv[t020] = fma(tu02, v0, tuv[t020]);
      tuv[t002] = fma(tu00, v2, tuv[t002]); tuv[t110] = fma(tu11, v0, tuv[t110]);
      tuv[t101] = fma(tu10, v1, tuv[t101]); tuv[t011] = fma(tu01, v1, tuv[t011]);
    }
    double c[10];
    c[0] = pc.tfm[0][0] * tuv[0];
    for (int j = 1; j < 4; j++) {
      double v = 0.0;
      for (int k = 1; k < 4; k++) v = fma(pc.tfm[j][k], tuv[k], v);
      c[j] = v;
    }
    for (int j = 4; j < 10; j++) {
      double v = 0.0;
      for (int k = 4; k < 10; k++) v = fma(pc.tfm[j][k], tuv[k], v);
      c[j] = v;
    }
    const double *mp = mpole + 10 * (size_t)i;
    if (phi_out)
      for (int j = 0; j < 10; j++) phi_out[10 * (size_t)i + j] = c[j];
    e = mp[t000] * c[t000] + mp[t100] * c[t100] + mp[t010] * c[t010] + mp[t001] * c[t001] +
        (1.0 / 3.0) * (mp[t200] * c[t200] + mp[t020] * c[t020] + mp[t002] * c[t002] +
                       2.0 * (mp[t110] * c[t110] + mp[t101] * c[t101] + mp[t011] * c[t011]));
  }
  e = warp_sum(e);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    for (int w = 0; w < kNaThreads / 32; w++) b += red[w];
    s->partial[blockIdx.x] = b;
  }
}

__global__ void k_na_energy(int nb, double electric, const NoAllocScratch *s, double *energy) {
  if (threadIdx.x == 0) {
    double sum = 0.0;
    for (int b = 0; b < nb; b++) sum += s->partial[b];
    *energy = 0.5 * electric * sum;
  }
}

static bool na_dim_ok(int n) { return n >= kOrder; }   // any length: the general radix pass

extern "C" int ffxg_pme_recip_permanent_noalloc(const double *d_xyz, const double *d_mpole, int32_t n_atoms,
                                                const double box[3], const int32_t pme_grid[3], double ewald_alpha,
                                                double electric, double *d_phi, double *d_energy, void *stream) {
  if (!d_xyz || !d_mpole || !d_energy || !box || !pme_grid || n_atoms <= 0 || !(ewald_alpha > 0.0))
    return FFXG_ERR_BAD_ARG;
  for (int d = 0; d < 3; d++) {
    if (!(box[d] > 0.0)) return FFXG_ERR_BAD_ARG;
    if (pme_grid[d] > kNaMaxDim) return FFXG_ERR_CAPACITY;
    if (!na_dim_ok(pme_grid[d])) return FFXG_ERR_BAD_ARG;
  }
  if (n_atoms > kNaMaxAtoms) return FFXG_ERR_CAPACITY;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNaMaxDevices) return FFXG_ERR_CUDA;
  NoAllocScratch *s = g_noalloc_ptr[dev].load();
  if (!s) {
    // First call on this device (device current): resolve the array's device address.
    if (cudaGetSymbolAddress((void **)&s, g_noalloc_scratch) != cudaSuccess || !s) return FFXG_ERR_CUDA;
    g_noalloc_ptr[dev].store(s);
  }
  cudaStream_t st = (cudaStream_t)stream;
  // Transforms of this box and mesh, on the host stack.
  const int nf[3] = {pme_grid[0], pme_grid[1], pme_grid[2]};
  const double A[3][3] = {{1.0 / box[0], 0, 0}, {0, 1.0 / box[1], 0}, {0, 0, 1.0 / box[2]}};
  static const int qi1[6] = {0, 1, 2, 0, 0, 1};
  static const int qi2[6] = {0, 1, 2, 1, 2, 2};
  PmeConst pc{};
  double a[3][3], af[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) { a[j][i] = nf[j] * A[i][j]; af[i][j] = nf[j] * A[i][j]; }
  pc.tmm[0][0] = 1.0;
  for (int i = 1; i < 4; i++)
    for (int j = 0; j < 3; j++) pc.tmm[i][1 + j] = a[i - 1][j];
  for (int i1 = 0; i1 < 3; i1++)
    for (int i2 = 0; i2 < 6; i2++) pc.tmm[i1 + 4][i2 + 4] = a[qi1[i1]][qi1[i2]] * a[qi1[i1]][qi2[i2]];
  for (int i1 = 3; i1 < 6; i1++)
    for (int i2 = 0; i2 < 6; i2++) {
      const int k = qi1[i1], l = qi2[i1], ii = qi1[i2], jj = qi2[i2];
      pc.tmm[i1 + 4][i2 + 4] = a[k][ii] * a[l][jj] + a[k][jj] * a[l][ii];
    }
  pc.tfm[0][0] = 1.0;
  for (int i = 1; i < 4; i++)
    for (int j = 0; j < 3; j++) pc.tfm[i][1 + j] = af[i - 1][j];
  for (int i1 = 0; i1 < 3; i1++) {
    const int k = qi1[i1];
    for (int i2 = 0; i2 < 3; i2++) pc.tfm[i1 + 4][i2 + 4] = af[k][qi1[i2]] * af[k][qi1[i2]];
    for (int i2 = 3; i2 < 6; i2++) pc.tfm[i1 + 4][i2 + 4] = 2.0 * af[k][qi1[i2]] * af[k][qi2[i2]];
  }
  for (int i1 = 3; i1 < 6; i1++) {
    const int k = qi1[i1], nn = qi2[i1];
    for (int i2 = 0; i2 < 3; i2++) pc.tfm[i1 + 4][i2 + 4] = af[k][qi1[i2]] * af[nn][qi1[i2]];
    for (int i2 = 3; i2 < 6; i2++) {
      const int ii = qi1[i2], jj = qi2[i2];
      pc.tfm[i1 + 4][i2 + 4] = af[k][ii] * af[nn][jj] + af[nn][ii] * af[k][jj];
    }
  }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) pc.recip[i][j] = A[i][j];
  const int npts = nf[0] * nf[1] * nf[2];
  // Each launch reports its own error (cudaLaunchKernelEx returns it), so an error the
  // caller left pending is neither taken for this call's nor cleared by it.
  auto launch = [&](auto kernel, int blocks, int threads, size_t smem, auto... args) {
    cudaLaunchConfig_t c{};
    c.gridDim = dim3(blocks);
    c.blockDim = dim3(threads);
    c.dynamicSmemBytes = smem;
    c.stream = st;
    return cudaLaunchKernelEx(&c, kernel, args...);
  };
  if (launch(k_na_tables, 3, kNaMaxDim, 0, nf[0], nf[1], nf[2], s) != cudaSuccess) return FFXG_ERR_CUDA;
  if (launch(k_na_influence, nblocks(npts, 256), 256, 0, nf[0], nf[1], nf[2], A[0][0], A[1][1], A[2][2], ewald_alpha,
             box[0] * box[1] * box[2], s) != cudaSuccess)
    return FFXG_ERR_CUDA;
  if (launch(k_na_spread, nblocks(n_atoms, kNaThreads / 32), kNaThreads, 0, (int)n_atoms, d_xyz, d_mpole, nf[0], nf[1],
             nf[2], pc, s) != cudaSuccess)
    return FFXG_ERR_CUDA;
  double2 *grid = s->grid;
  const double *no_influence = nullptr;
  double *no_plane = nullptr;
  int *no_flags = nullptr;   // only the mixed form's first pass reads it
  for (int pass = 0; pass < 5; pass++) {
    const int d = (pass < 2) ? pass : (pass == 2 ? 2 : 4 - pass);
    const int sign = (pass < 3) ? -1 : +1;
    const FftAxis ax = make_axis(d, nf);
    const int outer = (d == 2) ? nf[1] : nf[2];
    const size_t smem = fft_axis_smem(ax);   // <= 32 KB at kNaMaxDim: no attribute needed
    using OneFft = void (*)(double2 *, FftAxis, int, const double2 *, const double *, int, int, double *, size_t,
                            int *);
    const OneFft f =
        (pass == 2) ? (OneFft)one_fn<k_fft_axis<true, double, false>, 256, 0, double2 *, FftAxis, int, const double2 *,
                                     const double *, int, int, double *, size_t, int *>()
                    : (OneFft)one_fn<k_fft_axis<false, double, false>, 256, 0, double2 *, FftAxis, int,
                                     const double2 *, const double *, int, int, double *, size_t, int *>();
    const cudaError_t e = launch(f, ax.groups_inner * outer, 256, smem, grid, ax, sign,
                                 (const double2 *)(s->twiddle + d * kNaMaxDim),
                                 pass == 2 ? (const double *)s->influence : no_influence, nf[0], nf[1], no_plane,
                                 (size_t)0, no_flags);
    if (e != cudaSuccess) return FFXG_ERR_CUDA;
  }
  const int nb = nblocks(n_atoms, kNaThreads);
  if (launch(k_na_phi, nb, kNaThreads, 0, (int)n_atoms, d_xyz, d_mpole, nf[0], nf[1], nf[2], pc, d_phi, s) !=
      cudaSuccess)
    return FFXG_ERR_CUDA;
  if (launch(k_na_energy, 1, 32, 0, nb, electric, (const NoAllocScratch *)s, d_energy) != cudaSuccess)
    return FFXG_ERR_CUDA;
  return FFXG_OK;
}

}  // namespace ffx
