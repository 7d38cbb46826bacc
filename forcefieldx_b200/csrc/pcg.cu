// pcg.cu -- preconditioned conjugate-gradient induced-dipole solver.
//
// PCGSolver.scfByPCG (pme/PCGSolver.java:487-602) with InitResidualRegion (:609-663),
// InitConjugateRegion (:670-770), UpdateResidualRegion (:773-985) and
// UpdateConjugateRegion (:991-1180, Fletcher-Reeves).  The D and CR systems advance
// together with separate scalars.
//
// The real-space part of every dipole field reuses the pairs that k_realspace_field
// cached for this evaluation (displacement r_ik and coefficients A_ik, B_ik): the field
// at i of a dipole set u is sum_k -A_ik u_k + B_ik (u_k . r_ik) r_ik, so each field costs
// one streamed pass over the Ewald (or preconditioner) row plus one gathered source
// record per pair, with no minimum image, erfc, exp or sqrt.
//
// The field operator T is linear, so with p = z + beta p_old an iteration only needs
// T z: T p = T z + beta T p_old, with T p_old kept from the previous iteration.  T z is
// available as soon as the preconditioner has produced z, and its real-space part
// (k_pair_field) runs on a second stream beside the spread and FFT convolution of z,
// which leave most SMs idle.  One iteration: k_pcg_precond (z, r . z partials), {spread
// z, FFT} || k_pair_field (and beta), k_pcg_combine (mesh field of z, self term, T p, p,
// A p and its dot products), k_pcg_update (r, u, norms; its last block applies the
// reference's stopping rules on the device).  Vectors are FP64 [3][n]; every dot product is a
// fixed-order sum of per-block partials (by one block of the pair field, every block of
// k_pcg_update, or k_pcg_update's last block).
#include <algorithm>
#include <cmath>

#include "ffx_internal.cuh"

namespace ffx {

constexpr int kFieldThreads = 128;               // blocks of the pair-field kernels
constexpr int kVecThreads = 256;
constexpr int kVecBlocks = 148 * 2;
// Lane groups of the pair-field kernels: G lanes per atom (a warp takes 32 / G atoms), a
// grid that gives every group one atom.  The short preconditioner rows (~40 pairs at
// 4.5 A) take 4 lanes with four gathers in flight each, the Ewald rows (~140 pairs at
// 7 A) 16 lanes with two (measured best of 4/8 and 8/16/32).  Grids follow the system
// size, so the kernels of many small systems can share the device (batches).
constexpr int kPrecondGroup = 4;
constexpr int kEwaldGroup = 16;
static int group_blocks(int n, int G) { return std::max(1, (n + kFieldThreads / G - 1) / (kFieldThreads / G)); }
// The vector kernels stride over atoms with a fixed grid for large systems.
static int vec_blocks(int n) { return std::min(kVecBlocks, std::max(1, (n + kVecThreads - 1) / kVecThreads)); }
// The combine takes one atom per warp; its partial rows are one per block.
// The combine takes kCombineGroup lanes per atom (32 / kCombineGroup atoms per warp);
// its partial rows are one per block.
constexpr int kCombineGroup = 8;
static int combine_blocks(int n) { return nblocks((int64_t)n * kCombineGroup, 256); }
// Totals of the PCG scalars in Handle::d_scalars.
enum { T_PAP = 0, T_PAPP, T_RZ, T_RZP, T_RZN, T_RZNP, T_BETA, T_BETAP };
// Counters (each returns to 0 after use) in Handle::d_counter.
enum { K_UPDATE = 0, K_FIELD, K_PRECOND };

// Fixed-order total of column c over nb rows by one warp (lane l sums l, l+32, ...; four
// rows' loads in flight at a time).
__device__ __forceinline__ double warp_total(const double *__restrict__ part, int nb, int c) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int b0 = lane; b0 < nb; b0 += 128) {
    double v[4];
#pragma unroll
    for (int u = 0; u < 4; u++) v[u] = (b0 + 32 * u < nb) ? part[(b0 + 32 * u) * 8 + c] : 0.0;
#pragma unroll
    for (int u = 0; u < 4; u++) s += v[u];
  }
  return warp_sum(s);
}

// Block sum of NV per-thread values into part[vg.bid][0 .. NV); the last block to
// finish sums all rows in block order into tot[t0 .. t0 + NV) and re-arms the counter.
// Returns true in the last block (all threads).
template <int NV>
__device__ __forceinline__ bool block_partials(VGrid vg, const double *v, double *part, unsigned *counter, double *tot,
                                               int t0) {
  __shared__ double sh[NV][32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; q++) {
    const double s = warp_sum(v[q]);
    if (lane == 0) sh[q][wid] = s;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int w = 0; w < nw; w++) s += sh[threadIdx.x][w];
    part[vg.bid * 8 + threadIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == vg.nblk - 1);
  __syncthreads();
  if (last && threadIdx.x < 32) {
    __threadfence();
#pragma unroll
    for (int q = 0; q < NV; q++) {
      const double t = warp_total(part, vg.nblk, q);
      if (threadIdx.x == 0) tot[t0 + q] = t;
    }
    if (threadIdx.x == 0) *counter = 0u;
  }
  return last;
}

// Block sum of NV values already reduced to lane 0 of each warp, stored as
// part[vg.bid][0 .. NV) (no atomics; beta_block or k_pcg_update finishes the sum).
template <int NV>
__device__ __forceinline__ void block_store_lane0(VGrid vg, const double *v, double *part) {
  __shared__ double sh[NV][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NV; q++) sh[q][wid] = v[q];
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int w = 0; w < nw; w++) s += sh[threadIdx.x][w];
    part[vg.bid * 8 + threadIdx.x] = s;
  }
}

// beta = r.z_new / r.z_old for both systems (a zero r.z_old counts as 1) from the
// preconditioner's partial rows, by one whole block: thread t sums rows t, t + blockDim,
// ... (eight rows' loads in flight), then a fixed warp tree and the warps in order.  The
// new r.z totals go to tot[T_RZN], tot[T_RZNP].
__device__ void beta_block(const double *__restrict__ part, int nrows, double *tot) {
  __shared__ double sh[2][32];
  double s0 = 0.0, s1 = 0.0;
  constexpr int U = 8;
  for (int b0 = threadIdx.x; b0 < nrows; b0 += U * blockDim.x) {
    double v[U][2];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int b = b0 + u * blockDim.x;
      v[u][0] = (b < nrows) ? part[b * 8] : 0.0;
      v[u][1] = (b < nrows) ? part[b * 8 + 1] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; u++) { s0 += v[u][0]; s1 += v[u][1]; }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  if (lane == 0) { sh[0][wid] = s0; sh[1][wid] = s1; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t0 = 0.0, t1 = 0.0;
    for (int w = 0; w < nw; w++) { t0 += sh[0][w]; t1 += sh[1][w]; }
    tot[T_RZN] = t0;
    tot[T_RZNP] = t1;
    double old = tot[T_RZ], oldP = tot[T_RZP];
    if (old == 0.0) old = 1.0;
    if (oldP == 0.0) oldP = 1.0;
    tot[T_BETA] = t0 / old;
    tot[T_BETAP] = t1 / oldP;
  }
}

// Contribution of one neighbour: -A u_k + B (u_k . r) r for both sets.
template <typename T>
__device__ __forceinline__ void field_term(T xr, T yr, T zr, T A, T B, const T *s, T *acc) {
  const T ukr = B * (s[0] * xr + s[1] * yr + s[2] * zr);
  const T pkr = B * (s[3] * xr + s[4] * yr + s[5] * zr);
  acc[0] += -A * s[0] + ukr * xr; acc[1] += -A * s[1] + ukr * yr; acc[2] += -A * s[2] + ukr * zr;
  acc[3] += -A * s[3] + pkr * xr; acc[4] += -A * s[4] + pkr * yr; acc[5] += -A * s[5] + pkr * zr;
}

// Lane partials of the dipole field at atom i from the cached pair row, taken by the G
// lanes (sub = 0 .. G-1) of one aligned lane group: the displacement and A, B of each pair
// stream in coalesced; only the neighbour's source record is gathered.  T is double
// (plain form) or float (mixed form).  Each lane handles NU entries (a, a + G, ...)
// together so that all their loads are in flight at once; the summation order stays a,
// a + G, a + 2G, ...  i < 0 marks an idle group (no atom left), which still takes part in
// the group's shuffles.
template <typename T, int NU, int G>
__device__ __forceinline__ void pair_field(int i, int sub, const int *__restrict__ lst, const int *__restrict__ lst_cnt,
                                           int cap, const PairRec<T> *__restrict__ pr, const T *__restrict__ pb,
                                           const T *__restrict__ rec, T *acc) {
  const int cnt = (i < 0) ? 0 : min(lst_cnt[i], cap);
  const size_t e0 = (size_t)(i < 0 ? 0 : i) * cap;
  for (int a = sub; a < cnt; a += G * NU) {
    int ix[NU], kk[NU];
    T xx[NU], yy[NU], zz[NU], AA[NU], BB[NU], ss[NU][6];
#pragma unroll
    for (int u = 0; u < NU; u++) {
      ix[u] = (a + G * u < cnt) ? a + G * u : a;
      load_pair_b(pb, lst, e0 + ix[u], kk[u], BB[u]);
    }
#pragma unroll
    for (int u = 0; u < NU; u++) {
      load_pair(pr, e0 + ix[u], xx[u], yy[u], zz[u], AA[u]);
      get_rec(rec, kk[u], ss[u]);
    }
#pragma unroll
    for (int u = 0; u < NU; u++)
      if (a + G * u < cnt) field_term(xx[u], yy[u], zz[u], AA[u], BB[u], ss[u], acc);
  }
}

// Sum over the G lanes of an aligned lane group (every lane of the warp takes part).
template <int G>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Fractional-to-Cartesian transform of the potential gradient (rows and columns 1-3 of
// ReciprocalSpace.transformFieldMatrix).
struct FieldXform {
  double m[3][3];
};

// Lane partials of the fractional potential gradient of the (Re, Im) mesh at atom i:
// lane l < 25 owns the (x, y) support point (l % 5, l / 5) and walks the five z layers
// (InducedPhiLoop, ReciprocalSpace.java:2506-2775, first derivatives only).  The caller
// sums the lanes and applies the fractional-to-Cartesian transform.
template <typename T>
__device__ __forceinline__ void mesh_field(int i, int n, const int *__restrict__ igrid, const T *__restrict__ spl,
                                           const typename Vec2<T>::type *__restrict__ mesh, int nfx, int nfy, int nfz,
                                           T *acc) {
  const int lane = threadIdx.x & 31;
  if (lane >= 25) return;
  const T *sp = spl + (size_t)i * 3 * kOrder * 4;
  const T *sx = sp, *sy = sp + kOrder * 4, *sz = sp + 2 * kOrder * 4;
  const int a1 = lane % 5, a2 = lane / 5;
  int ii = igrid[i] + 1 + a1, jj = igrid[n + i] + 1 + a2;
  ii += (ii < 0) ? nfx : ((ii >= nfx) ? -nfx : 0);
  jj += (jj < 0) ? nfy : ((jj >= nfy) ? -nfy : 0);
  const int k0 = igrid[2 * n + i] + 1;
  const T x0 = sx[a1 * 4], x1 = sx[a1 * 4 + 1];
  const T y0 = sy[a2 * 4], y1 = sy[a2 * 4 + 1];
  const T w10 = x1 * y0, w01 = x0 * y1, w00 = x0 * y0;
  const auto *col = mesh + (size_t)jj * nfx + ii;
  T g[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int a3 = 0; a3 < 5; a3++) {
    int kk = k0 + a3;
    kk += (kk < 0) ? nfz : ((kk >= nfz) ? -nfz : 0);
    const auto m = col[(size_t)kk * nfy * nfx];
    const T z0 = sz[a3 * 4], z1 = sz[a3 * 4 + 1];
    const T wx = w10 * z0, wy = w01 * z0, wz = w00 * z1;
    g[0] = fma(m.x, wx, g[0]); g[1] = fma(m.x, wy, g[1]); g[2] = fma(m.x, wz, g[2]);
    g[3] = fma(m.y, wx, g[3]); g[4] = fma(m.y, wy, g[4]); g[5] = fma(m.y, wz, g[5]);
  }
#pragma unroll
  for (int q = 0; q < 6; q++) acc[q] += g[q];
}

// The same for a group of G lanes per atom (sub = 0 .. G-1): lane sub takes the (x, y)
// support points sub, sub + G, ... of the 25, each with its five z layers, so that every
// lane has several gathers in flight.  i < 0: an idle group (no loads, zero partials).
template <typename T, int G>
__device__ __forceinline__ void mesh_field_group(int i, int sub, int n, const int *__restrict__ igrid,
                                                 const T *__restrict__ spl,
                                                 const typename Vec2<T>::type *__restrict__ mesh, int nfx, int nfy,
                                                 int nfz, T *acc) {
  if (i < 0) return;
  const T *sp = spl + (size_t)i * 3 * kOrder * 4;
  const T *sx = sp, *sy = sp + kOrder * 4, *sz = sp + 2 * kOrder * 4;
  const int i0 = igrid[i] + 1, j0 = igrid[n + i] + 1, k0 = igrid[2 * n + i] + 1;
  T g[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int t = 0; t < (25 + G - 1) / G; t++) {
    const int pt = sub + G * t;
    if (pt < 25) {
      const int a1 = pt % 5, a2 = pt / 5;
      int ii = i0 + a1, jj = j0 + a2;
      ii += (ii < 0) ? nfx : ((ii >= nfx) ? -nfx : 0);
      jj += (jj < 0) ? nfy : ((jj >= nfy) ? -nfy : 0);
      const T x0 = sx[a1 * 4], x1 = sx[a1 * 4 + 1];
      const T y0 = sy[a2 * 4], y1 = sy[a2 * 4 + 1];
      const T w10 = x1 * y0, w01 = x0 * y1, w00 = x0 * y0;
      const auto *col = mesh + (size_t)jj * nfx + ii;
#pragma unroll
      for (int a3 = 0; a3 < 5; a3++) {
        int kk = k0 + a3;
        kk += (kk < 0) ? nfz : ((kk >= nfz) ? -nfz : 0);
        const auto m = col[(size_t)kk * nfy * nfx];
        const T z0 = sz[a3 * 4], z1 = sz[a3 * 4 + 1];
        const T wx = w10 * z0, wy = w01 * z0, wz = w00 * z1;
        g[0] = fma(m.x, wx, g[0]); g[1] = fma(m.x, wy, g[1]); g[2] = fma(m.x, wz, g[2]);
        g[3] = fma(m.y, wx, g[3]); g[4] = fma(m.y, wy, g[4]); g[5] = fma(m.y, wz, g[5]);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 6; q++) acc[q] += g[q];
}

// Real-space pair field of the source records `rec` (u, then z) at every atom, into
// out[6][n] (D xyz, CR xyz).  A group of G lanes takes one atom; the groups of a warp take
// consecutive atoms and stride over the system together.
template <typename T, int G, int NU>
__device__ __forceinline__ void k_pair_field(VGrid vg, int n, const int *__restrict__ ewl,
                                                              const int *__restrict__ ewl_cnt, int capE,
                                                              const PairRec<T> *__restrict__ coefE,
                                                              const T *__restrict__ coefEB,
                                                              const T *__restrict__ rec, double *out,
                                                              const double *__restrict__ beta_part, int beta_rows,
                                                              double *tot) {
  // Block 0 first forms beta from the preconditioner's partial rows (the combine, after
  // the join, reads it): no separate totals launch on the solver's chain.
  if (beta_part && vg.bid == 0) beta_block(beta_part, beta_rows, tot);
  constexpr int GPW = 32 / G;
  const int lane = threadIdx.x & 31, sub = lane & (G - 1), gi = lane / G;
  const int astride = vg.nblk * (blockDim.x >> 5) * GPW;
  for (int i0 = (vg.bid * (blockDim.x >> 5) + (threadIdx.x >> 5)) * GPW; i0 < n; i0 += astride) {
    const int i = i0 + gi;
    const bool live = i < n;
    T a6[6] = {0, 0, 0, 0, 0, 0};
    pair_field<T, NU, G>(live ? i : -1, sub, ewl, ewl_cnt, capE, coefE, coefEB, rec, a6);
    double f[6];
#pragma unroll
    for (int q = 0; q < 6; q++) f[q] = group_sum<G>((double)a6[q]);
    if (live && sub == 0) {
#pragma unroll
      for (int q = 0; q < 6; q++) out[(size_t)q * n + i] = f[q];
    }
  }
}

// E(v) = pair field (tpair) + reciprocal field from the mesh + self field aewald3 v,
// for the source v = (vD, vP), then
// MODE 1: initial residual r = (u_dir - u) / alpha + E(u) with u == u_dir
//         (InitResidualRegion) and the preconditioner source record alpha r.
// MODE 2: v = z.  T p = E(z) + beta T p_old and p = z + beta p_old (first: T p = E(z),
//         p = z); vec = p / alpha - T p; p . vec and r . z finished into d_scalars
//         (UpdateApLoop).
// kCombineGroup lanes per atom: the group interpolates the mesh, then its lane q < 6
// finishes component q (D x, y, z, CR x, y, z).
template <int MODE, typename T>
__device__ __forceinline__ void k_pcg_combine(
    VGrid vg, int const &n, const int *__restrict__ const &igrid, const T *__restrict__ const &spl,
    const typename Vec2<T>::type *__restrict__ const &mesh, int const &nfx, int const &nfy, int const &nfz,
    const FieldXform &xf, const double *__restrict__ const &tpair, const double *__restrict__ const &vD,
    const double *__restrict__ const &vP, double const &aewald3, const double *__restrict__ const &polar,
    const double *__restrict__ const &udirD, const double *__restrict__ const &udirP, double * const &p,
    double * const &pP, double * const &tp, int const &first, const double *__restrict__ const &r,
    const double *__restrict__ const &rP, double * const &outD, double * const &outP, T * const &recP,
    double * const &part, unsigned * const &counter, double * const &tot) {
  constexpr int G = kCombineGroup;
  const int lane = threadIdx.x & 31, sub = lane & (G - 1), g0 = lane & ~(G - 1);
  const int i = (vg.bid * blockDim.x + threadIdx.x) / G;
  const bool live = i < n;
  double acc[4] = {0, 0, 0, 0};
  T a6[6] = {0, 0, 0, 0, 0, 0};
  mesh_field_group<T, G>(live ? i : -1, sub, n, igrid, spl, mesh, nfx, nfy, nfz, a6);
  T g[6];
#pragma unroll
  for (int q = 0; q < 6; q++) {
    T v = a6[q];
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    g[q] = v;
  }
  double rec_v = 0.0;
  if (live && sub < 6) {
    // Lane sub takes Cartesian field component sub: -(xf . gradient) of its set.
    const int d = sub % 3, set = sub / 3;
    const double *row = xf.m[d];
    const double mine = -(row[0] * (double)(set ? g[3] : g[0]) + row[1] * (double)(set ? g[4] : g[1]) +
                          row[2] * (double)(set ? g[5] : g[2]));
    const size_t j = (size_t)d * n + i, jt = (size_t)sub * n + i;
    const double *v = set ? vP : vD;
    const double vj = v[j];
    const double e = mine + tpair[jt] + aewald3 * vj;
    const double a = polar[i];
    const bool ok = a > 0.0;
    const double ip = ok ? 1.0 / a : 0.0;
    if (MODE == 1) {
      const double *ud = set ? udirP : udirD;
      const double rv = ok ? (ud[j] - vj) * ip + e : 0.0;
      (set ? outP : outD)[j] = rv;
      rec_v = a * rv;
    } else {
      const double b = first ? 0.0 : tot[set ? T_BETAP : T_BETA];
      double *pp = set ? pP : p;
      double t = e, pv = vj;
      if (!first) {
        t += b * tp[jt];
        pv += b * pp[j];
      }
      tp[jt] = t;
      pp[j] = pv;
      const double vv = ok ? pv * ip - t : 0.0;
      (set ? outP : outD)[j] = vv;
      const double pav = pv * vv, rzv = (set ? rP : r)[j] * vj;
      acc[0] = set ? 0.0 : pav;
      acc[1] = set ? pav : 0.0;
      acc[2] = set ? 0.0 : rzv;
      acc[3] = set ? rzv : 0.0;
    }
  }
  if (MODE == 1) {
    double w[6];
#pragma unroll
    for (int q = 0; q < 6; q++) w[q] = __shfl_sync(0xffffffffu, rec_v, g0 + q);
    if (live && sub == 0) put_rec(recP, i, w[0], w[1], w[2], w[3], w[4], w[5]);
  }
  if (MODE == 2) {
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
    block_store_lane0<4>(vg, acc, part);
  }
}

// z = alpha (E_precond(alpha r) + s r) (InitConjugateRegion / UpdatePreconditionerLoop)
// and z's source record for the next field.  INIT also sets p = z; otherwise r . z_new
// is finished into d_scalars and the last block forms beta = r.z_new / r.z_old
// (UpdateConjugateLoop, Fletcher-Reeves; a zero r.z_old counts as 1).
template <bool INIT, typename T, int G>
__device__ __forceinline__ void k_pcg_precond(
    VGrid vg, int const &n, const int *__restrict__ const &prl, const int *__restrict__ const &prl_cnt,
    int const &capP, const PairRec<T> *__restrict__ const &coefP, const T *__restrict__ const &coefPB,
    const T *__restrict__ const &recP, const double *__restrict__ const &polar,
    const double *__restrict__ const &r, const double *__restrict__ const &rP, double const &s,
    double * const &zz, double * const &zP, double * const &p, double * const &pP, T * const &recF,
    double * const &part, unsigned * const &counter, double * const &tot) {
  constexpr int GPW = 32 / G;
  constexpr int QPL = (6 + G - 1) / G;   // components finished per lane: q = sub, sub + G, ...
  const int lane = threadIdx.x & 31, sub = lane & (G - 1), gi = lane / G, g0 = lane & ~(G - 1);
  const int astride = vg.nblk * (blockDim.x >> 5) * GPW;
  double acc[2] = {0, 0};
  for (int i0 = (vg.bid * (blockDim.x >> 5) + (threadIdx.x >> 5)) * GPW; i0 < n; i0 += astride) {
    const int i = i0 + gi;
    const bool live = i < n;
    T a6[6] = {0, 0, 0, 0, 0, 0};
    pair_field<T, 4, G>(live ? i : -1, sub, prl, prl_cnt, capP, coefP, coefPB, recP, a6);
    double f[6];
#pragma unroll
    for (int q = 0; q < 6; q++) f[q] = group_sum<G>((double)a6[q]);
    double zq[QPL];
#pragma unroll
    for (int u = 0; u < QPL; u++) {
      const int q = sub + u * G;
      double mine = f[0];
#pragma unroll
      for (int c = 1; c < 6; c++)
        if (q == c) mine = f[c];
      zq[u] = 0.0;
      if (live && q < 6) {
        const int d = q % 3, set = q / 3;
        const size_t j = (size_t)d * n + i;
        const double rj = (set ? rP : r)[j];
        const double zv = polar[i] * (mine + s * rj);
        zq[u] = zv;
        (set ? zP : zz)[j] = zv;
        if (INIT) (set ? pP : p)[j] = zv;
        if (set) acc[1] += rj * zv;
        else acc[0] += rj * zv;
      }
    }
    double w[6];
#pragma unroll
    for (int q = 0; q < 6; q++) w[q] = __shfl_sync(0xffffffffu, zq[q / G], g0 + q % G);
    if (live && sub == 0) put_rec(recF, i, w[0], w[1], w[2], w[3], w[4], w[5]);
  }
  if (!INIT) {
#pragma unroll
    for (int q = 0; q < 2; q++) acc[q] = group_sum<32>(acc[q]);
    block_store_lane0<2>(vg, acc, part);
  }
}

// PCGSolver.scfByPCG stopping rules (pme/PCGSolver.java:541-570) applied on the device:
// eps = 4.80321 sqrt(max(|r_D|^2, |r_CR|^2) / n); stop with an error when eps grew (or
// is not finite) or the iteration limit is reached, stop converged when eps < polar-eps.
// A list overflow seen earlier in the evaluation also stops the loop (the host repeats
// the evaluation with larger lists).
__device__ __forceinline__ void k_pcg_reset(VGrid vg, PcgState *st) {
  st->eps = 100.0;
  st->iter = 0;
  st->status = FFXG_OK;
  st->cont = 1;
}

// alpha = r.z / p.Ap; r -= alpha vec; u += alpha p; the preconditioner source record
// alpha_pol r; |r|^2 partials.  The last block finishes both norms, applies the stopping
// rules to PcgState, re-arms the counter and, inside a captured graph, sets the
// condition of the PCG while node.
template <typename T>
__device__ __forceinline__ void k_pcg_update(VGrid vg, 
    int n, const double *__restrict__ vec, const double *__restrict__ vecP, const double *__restrict__ p,
    const double *__restrict__ pP, double *r, double *rP, double *uD, double *uP, double *tot,
    double *partE, unsigned *counter, PcgState *st, int max_iter, double polar_eps, const int *flags,
    cudaGraphConditionalHandle cond, int use_cond, const double *__restrict__ polar, T *recP, int n_eps,
    const double *__restrict__ partC, int rowsC) {
  // p.Ap and r.z of both systems: every block sums the combine's partial rows itself, in
  // one fixed order (so every block holds the same values), instead of a separate totals
  // launch on the critical path; block 0 keeps them for the next beta.
  __shared__ double tsum[4][kVecThreads / 32];
  __shared__ double tv[4];
  {
    // Rows b, b + blockDim, ... per thread, eight rows' loads in flight at a time.
    double s4[4] = {0.0, 0.0, 0.0, 0.0};
    constexpr int U = 8;
    for (int b0 = threadIdx.x; b0 < rowsC; b0 += U * blockDim.x) {
      double v[U][4];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int b = b0 + u * blockDim.x;
#pragma unroll
        for (int q = 0; q < 4; q++) v[u][q] = (b < rowsC) ? partC[b * 8 + q] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < U; u++)
#pragma unroll
        for (int q = 0; q < 4; q++) s4[q] += v[u][q];
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const double w = warp_sum(s4[q]);
      if (lane == 0) tsum[q][wid] = w;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += tsum[threadIdx.x][w];
      tv[threadIdx.x] = t;
      if (vg.bid == 0) tot[T_PAP + threadIdx.x] = t;
    }
    __syncthreads();
  }
  const double pap = tv[0], papP = tv[1], rz = tv[2], rzP = tv[3];
  const double alpha0 = (pap != 0.0) ? rz / pap : rz;
  const double alpha1 = (papP != 0.0) ? rzP / papP : rzP;
  double v[2] = {0.0, 0.0};
  const int stride = vg.nblk * blockDim.x;
  for (int i = vg.bid * blockDim.x + threadIdx.x; i < n; i += stride) {
    // Every load first (one memory round trip), then the arithmetic, then the stores.
    double r0[3], r1[3], v0[3], v1[3], p0[3], p1[3], u0[3], u1[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const size_t j = (size_t)d * n + i;
      r0[d] = r[j]; r1[d] = rP[j]; v0[d] = vec[j]; v1[d] = vecP[j];
      p0[d] = p[j]; p1[d] = pP[j]; u0[d] = uD[j]; u1[d] = uP[j];
    }
    const double a = polar[i];
    double nr[6];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const double rr = r0[d] - alpha0 * v0[d];
      const double rp = r1[d] - alpha1 * v1[d];
      v[0] += rr * rr;
      v[1] += rp * rp;
      nr[d] = rr;
      nr[3 + d] = rp;
      u0[d] += alpha0 * p0[d];
      u1[d] += alpha1 * p1[d];
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const size_t j = (size_t)d * n + i;
      r[j] = nr[d]; rP[j] = nr[3 + d]; uD[j] = u0[d]; uP[j] = u1[d];
    }
    put_rec(recP, i, a * nr[0], a * nr[1], a * nr[2], a * nr[3], a * nr[4], a * nr[5]);
  }
  __shared__ double norms[2];
  if (block_partials<2>(vg, v, partE, counter, norms, 0) && threadIdx.x == 0) {
    const double e0 = norms[0], e1 = norms[1];
    const double m = (e0 < e1) ? e1 : e0;
    const double eps = kElecAngToDebye * sqrt(m / (double)n_eps);
    const double previous = st->eps;
    const int iter = st->iter + 1;
    int status = FFXG_OK, cont = 1;
    if (!(eps <= previous)) {
      status = isfinite(eps) ? FFXG_ERR_SCF_DIVERGED : FFXG_ERR_NONFINITE;
      cont = 0;
    } else if (iter >= max_iter) {
      status = FFXG_ERR_SCF_MAXITER;
      cont = 0;
    } else if (eps < polar_eps) {
      cont = 0;
    }
    if (*flags & (FLAG_NBR_OVERFLOW | FLAG_EWALD_OVERFLOW | FLAG_PRECOND_OVERFLOW | FLAG_NONFINITE)) cont = 0;
    st->eps = eps;
    st->iter = iter;
    st->status = status;
    st->cont = cont;
    if (use_cond) cudaGraphSetConditional(cond, (unsigned)cont);
  }
}

// ---------------------------------------------------------------------------
// Always-stable predictor-corrector initial guess (SCFPredictorParameters.aspcPredictor,
// pme/SCFPredictorParameters.java:80-123; saveMutualInducedDipoles, :269-303).  The ring
// ring[6][6][n] holds u - u_dir (D xyz, CR xyz) of the last six converged solves; state[0]
// is the slot of the most recent one and state[1] how many are stored.  With six stored,
// the solve starts from u = u_dir + sum_k c_k ring[(state[0] + k) % 6].
__device__ __forceinline__ void k_aspc_predict(VGrid vg, int n, const double *__restrict__ ring, const int *__restrict__ state,
                               const double *__restrict__ udD, const double *__restrict__ udP, double *uD, double *uP,
                               void *recF, int mixed) {
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n || state[1] < 6) return;
  const double c[6] = {22.0 / 7.0, -55.0 / 14.0, 55.0 / 21.0, -22.0 / 21.0, 5.0 / 21.0, -1.0 / 42.0};
  double u[6];
  for (int q = 0; q < 6; q++) u[q] = (q < 3) ? udD[q * n + i] : udP[(q - 3) * n + i];
  int slot = state[0];
  for (int k = 0; k < 6; k++) {
    for (int q = 0; q < 6; q++) u[q] += c[k] * ring[((size_t)slot * 6 + q) * n + i];
    slot = (slot + 1 == 6) ? 0 : slot + 1;
  }
  for (int d = 0; d < 3; d++) {
    uD[d * n + i] = u[d];
    uP[d * n + i] = u[3 + d];
  }
  if (mixed) put_rec(reinterpret_cast<float *>(recF), i, u[0], u[1], u[2], u[3], u[4], u[5]);
  else put_rec(reinterpret_cast<double *>(recF), i, u[0], u[1], u[2], u[3], u[4], u[5]);
}

// Store u - u_dir of a converged solve in the slot before state[0] (k_aspc_commit then
// advances the state); nothing is stored after a failed solve or a list overflow.
__device__ __forceinline__ void k_aspc_save(VGrid vg, int n, double *ring, const int *__restrict__ state, const double *__restrict__ uD,
                            const double *__restrict__ uP, const double *__restrict__ udD,
                            const double *__restrict__ udP, const PcgState *__restrict__ st, const int *flags) {
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n || st->status != FFXG_OK) return;
  if (*flags & (FLAG_NBR_OVERFLOW | FLAG_EWALD_OVERFLOW | FLAG_PRECOND_OVERFLOW | FLAG_NONFINITE)) return;
  const int slot = (state[0] + 5) % 6;
  for (int d = 0; d < 3; d++) {
    ring[((size_t)slot * 6 + d) * n + i] = uD[d * n + i] - udD[d * n + i];
    ring[((size_t)slot * 6 + 3 + d) * n + i] = uP[d * n + i] - udP[d * n + i];
  }
}

__device__ __forceinline__ void k_aspc_commit(VGrid vg, int *state, const PcgState *__restrict__ st, const int *flags) {
  if (st->status != FFXG_OK) return;
  if (*flags & (FLAG_NBR_OVERFLOW | FLAG_EWALD_OVERFLOW | FLAG_PRECOND_OVERFLOW | FLAG_NONFINITE)) return;
  state[0] = (state[0] + 5) % 6;
  if (state[1] < 6) state[1] += 1;
}

static void aspc_predict(Handle &h) {
  if (h.scf_predictor != FFXG_PREDICTOR_ASPC) return;
  launch_on<k_aspc_predict, 0, 0>(h.rec, nblocks(h.n, 256), 256, 0, h.stream, h.n, (const double *)h.d_aspc,
                                   (const int *)h.d_aspc_state, (const double *)h.d_udirD,
                                   (const double *)h.d_udirP, h.d_uD, h.d_uP, (void *)h.d_recF, h.mixed ? 1 : 0);
  FFX_LAUNCHED(h);
}

static void aspc_save(Handle &h) {
  if (h.scf_predictor != FFXG_PREDICTOR_ASPC) return;
  launch_on<k_aspc_save, 0, 0>(h.rec, nblocks(h.n, 256), 256, 0, h.stream, h.n, h.d_aspc,
                                (const int *)h.d_aspc_state, (const double *)h.d_uD, (const double *)h.d_uP,
                                (const double *)h.d_udirD, (const double *)h.d_udirP, (const PcgState *)h.d_pcg,
                                (const int *)h.d_flags);
  launch_on<k_aspc_commit, 0, 0>(h.rec, 1, 1, 0, h.stream, h.d_aspc_state, (const PcgState *)h.d_pcg,
                                  (const int *)h.d_flags);
  h.launches += 2;
}

static double aewald3_of(const Handle &h) {
  const double a = ewald_alpha_of(h);
  return 4.0 / 3.0 * pow(a, 3.0) / 1.7724538509055160273;
}

// Partial-sum regions of d_part2 (combine, preconditioner, update): one row of 8 per
// block of the largest grid that writes them.
int pcg_partial_rows(int n) {
  return std::max(std::max(kVecBlocks, combine_blocks(n)), group_blocks(n, kPrecondGroup));
}
static double *part_region(const Handle &h, int k) { return h.d_part2 + (size_t)k * h.part_rows * 8; }

// Gathers in flight per lane (NU): three for one FP32 system (ind_field 280 -> 264 us per
// evaluation of the 24k box against two; four and one measured no better), two in the
// FP64 form and in a batch, whose instance is held to 48 registers.
template <typename T>
static void pair_field_launch(Handle &h, cudaStream_t st, bool beta) {
  auto go = [&](auto body) {
    launch_on<decltype(body)::value, kFieldThreads, 0, sizeof(T) == 4 ? 10 : 0>(
        h.rec, group_blocks(h.n, kEwaldGroup), kFieldThreads, 0, st, h.n, (const int *)h.d_ewl,
        (const int *)h.d_ewl_cnt, h.cap_ewl, reinterpret_cast<const PairRec<T> *>(h.d_coefE),
        reinterpret_cast<const T *>(h.d_coefEB), reinterpret_cast<const T *>(h.d_recF), h.d_tpair,
        (const double *)(beta ? part_region(h, 1) : nullptr), group_blocks(h.n, kPrecondGroup), h.d_scalars);
  };
  bool done = false;
  if constexpr (sizeof(T) == 4) {
    if (!h.rec) {
      go(BodyOf<k_pair_field<T, kEwaldGroup, 3>>{});
      done = true;
    }
  }
  if (!done) go(BodyOf<k_pair_field<T, kEwaldGroup, 2>>{});
  FFX_LAUNCHED(h);
}

template <int MODE, typename T>
static void combine(Handle &h, const double *vD, const double *vP, bool first, double *outD, double *outP) {
  using V2 = typename Vec2<T>::type;
  FieldXform xf;
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) xf.m[a][b] = h.pc.tfm[1 + a][1 + b];
  const V2 *mesh = reinterpret_cast<const V2 *>(h.mixed ? (const void *)h.d_gridf : (const void *)h.d_grid);
  launch_on<k_pcg_combine<MODE, T>, 256, 0, 3>(
      h.rec, combine_blocks(h.n), 256, 0, h.stream, h.n, (const int *)h.d_igrid, reinterpret_cast<const T *>(h.d_spl),
      mesh, h.nfft[0], h.nfft[1], h.nfft[2], xf, (const double *)h.d_tpair, vD, vP, aewald3_of(h),
      (const double *)h.d_polar, (const double *)h.d_udirD, (const double *)h.d_udirP, h.d_p, h.d_pP, h.d_tp,
      first ? 1 : 0, (const double *)h.d_r, (const double *)h.d_rP, outD, outP, reinterpret_cast<T *>(h.d_recP),
      part_region(h, 0), h.d_counter + K_FIELD, h.d_scalars);
  FFX_LAUNCHED(h);
}

// The full field of (vD, vP), whose source record is in d_recF: the pair field on the
// auxiliary stream, concurrently with spread + FFT on the main stream, then the combine.
template <int MODE>
static void field_of(Handle &h, const double *vD, const double *vP, bool first, double *outD, double *outP) {
  // Stage timing (direct launches, ffxg_set_timing) keeps the pair field on the main
  // stream, so that its events time the kernel alone rather than its overlap.
  // A recording batch orders its stages itself: no fork.
  cudaStream_t ax = (h.timing || h.rec) ? h.stream : ((h.stream == h.side) ? h.aux_side : h.aux);
  if (!h.rec) {
    cudaEventRecord(h.ev_fork, h.stream);
    cudaStreamWaitEvent(ax, h.ev_fork, 0);
  }
  int tk = timer_begin_on(h, FFXG_STAGE_IND_FIELD, ax);
  // After a non-initial preconditioner step the pair field also forms beta.
  const bool beta = (MODE == 2) && !first;
  if (h.mixed) pair_field_launch<float>(h, ax, beta); else pair_field_launch<double>(h, ax, beta);
  timer_end_on(h, tk, ax);
  if (!h.rec) cudaEventRecord(h.ev_join, ax);
  tk = timer_begin(h, FFXG_STAGE_IND_RECIP);
  launch_spread_induced(h, vD, vP);
  launch_fft_convolution(h);
  timer_end(h, tk);
  if (!h.rec) cudaStreamWaitEvent(h.stream, h.ev_join, 0);
  tk = timer_begin(h, FFXG_STAGE_PCG_VECTOR);
  if (h.mixed) combine<MODE, float>(h, vD, vP, first, outD, outP);
  else combine<MODE, double>(h, vD, vP, first, outD, outP);
  timer_end(h, tk);
}

template <bool INIT, typename T>
static void precond(Handle &h) {
  launch_on<k_pcg_precond<INIT, T, kPrecondGroup>, kFieldThreads, 7, sizeof(T) == 4 ? 5 : 0>(
      h.rec, group_blocks(h.n, kPrecondGroup), kFieldThreads, 0, h.stream, h.n, (const int *)h.d_prl,
      (const int *)h.d_prl_cnt, h.cap_prl, reinterpret_cast<const PairRec<T> *>(h.d_coefP),
      reinterpret_cast<const T *>(h.d_coefPB), reinterpret_cast<const T *>(h.d_recP), (const double *)h.d_polar,
      (const double *)h.d_r, (const double *)h.d_rP, h.prm.precond_scale, h.d_zpre, h.d_zpreP, h.d_p, h.d_pP,
      reinterpret_cast<T *>(h.d_recF), part_region(h, 1), h.d_counter + K_PRECOND, h.d_scalars);
  FFX_LAUNCHED(h);
}

template <bool INIT>
static void launch_precond(Handle &h) {
  if (h.mixed) precond<INIT, float>(h); else precond<INIT, double>(h);
}

template <typename T>
static void update(Handle &h, cudaGraphConditionalHandle cond, int use_cond) {
  launch_on<k_pcg_update<T>, kVecThreads, 0, 3>(
      h.rec, vec_blocks(h.n), kVecThreads, 0, h.stream, h.n, (const double *)h.d_vec, (const double *)h.d_vecP,
      (const double *)h.d_p, (const double *)h.d_pP, h.d_r, h.d_rP, h.d_uD, h.d_uP, h.d_scalars, part_region(h, 2),
      h.d_counter + K_UPDATE, h.d_pcg, h.prm.max_scf_iter, h.prm.polar_eps, (const int *)h.d_flags, cond, use_cond,
      (const double *)h.d_polar, reinterpret_cast<T *>(h.d_recP), h.eps_atoms > 0 ? h.eps_atoms : h.n,
      (const double *)part_region(h, 0), combine_blocks(h.n));
  FFX_LAUNCHED(h);
}

// One PCG step up to the stopping test: T p from T z, A p with its dot products, update.
static void pcg_step(Handle &h, bool first, cudaGraphConditionalHandle cond, int use_cond) {
  field_of<2>(h, h.d_zpre, h.d_zpreP, first, h.d_vec, h.d_vecP);
  const int tk = timer_begin(h, FFXG_STAGE_PCG_VECTOR);
  if (h.mixed) update<float>(h, cond, use_cond); else update<double>(h, cond, use_cond);
  timer_end(h, tk);
}

static void pcg_precond(Handle &h) {
  const int tk = timer_begin(h, FFXG_STAGE_PRECOND);
  launch_precond<false>(h);
  timer_end(h, tk);
}

// The solve.  Directly (capture false): the host reads the device's stopping decision
// after every update (24 bytes).  Under stream capture (capture true): the first step is
// recorded in line and the rest as a conditional WHILE node whose body (preconditioner,
// step) the update kernel re-arms on the device, so the loop runs with no host round
// trip.  Either way the loop ends by max_scf_iter at the latest.
int run_pcg(Handle &h, bool capture) {
  launch_on<k_pcg_reset, 0, 0>(h.rec, 1, 1, 0, h.stream, h.d_pcg);
  FFX_LAUNCHED(h);
  aspc_predict(h);
  // Field of the direct dipoles (u == u_dir at entry) gives the initial residual.
  field_of<1>(h, h.d_uD, h.d_uP, true, h.d_r, h.d_rP);
  int tk = timer_begin(h, FFXG_STAGE_PRECOND);
  launch_precond<true>(h);
  timer_end(h, tk);
  if (h.rec) {
    // A batch records the solve: the first step in line, then the loop body, which the
    // batch runs as one conditional WHILE node for all its systems (k_many skips the
    // systems whose solve has stopped).
    pcg_step(h, true, 0, 0);
    h.rec->phase = 1;
    const int64_t before = h.launches;
    pcg_precond(h);
    pcg_step(h, false, 0, 0);
    h.graph_body_launches = h.launches - before;
    h.rec->phase = 2;
    aspc_save(h);
    return FFXG_OK;
  }
  if (!capture) {
    bool first = true;
    while (true) {
      pcg_step(h, first, 0, 0);
      first = false;
      cudaMemcpyAsync(h.h_pcg, h.d_pcg, sizeof(PcgState), cudaMemcpyDeviceToHost, h.stream);
      if (cudaStreamSynchronize(h.stream) != cudaSuccess) return FFXG_ERR_CUDA;
      if (!h.h_pcg->cont) break;
      pcg_precond(h);
    }
    aspc_save(h);
    h.scf_iter = h.h_pcg->iter;
    return h.h_pcg->status;
  }
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t ndeps = 0;
  if (cudaStreamGetCaptureInfo(h.stream, &cs, nullptr, &g, &deps, &ndeps) != cudaSuccess ||
      cs != cudaStreamCaptureStatusActive)
    return FFXG_ERR_CUDA;
  cudaGraphConditionalHandle cond;
  if (cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault) != cudaSuccess) return FFXG_ERR_CUDA;
  pcg_step(h, true, cond, 1);
  if (cudaStreamGetCaptureInfo(h.stream, &cs, nullptr, &g, &deps, &ndeps) != cudaSuccess) return FFXG_ERR_CUDA;
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  if (cudaGraphAddNode(&node, g, deps, ndeps, &cp) != cudaSuccess) return FFXG_ERR_CUDA;
  if (cudaStreamUpdateCaptureDependencies(h.stream, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess)
    return FFXG_ERR_CUDA;
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  if (cudaStreamBeginCaptureToGraph(h.side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess)
    return FFXG_ERR_CUDA;
  cudaStream_t main = h.stream;
  h.stream = h.side;
  const int64_t before = h.launches;
  pcg_precond(h);
  pcg_step(h, false, cond, 1);
  h.graph_body_launches = h.launches - before;
  h.stream = main;
  if (cudaStreamEndCapture(h.side, &body) != cudaSuccess) return FFXG_ERR_CUDA;
  aspc_save(h);   // after the while node
  return FFXG_OK;
}

}  // namespace ffx
