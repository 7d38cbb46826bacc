// pcg.cu -- preconditioned conjugate-gradient induced-dipole solver.
//
// PCGSolver.scfByPCG (pme/PCGSolver.java:487-602) with InitResidualRegion (:609-663),
// InitConjugateRegion (:670-770), UpdateResidualRegion (:773-985) and
// UpdateConjugateRegion (:991-1180, Fletcher-Reeves).  The D and CR systems advance
// together with separate scalars.
//
// The real-space part of every dipole field reuses the pairs that k_realspace_field
// cached for this evaluation (displacement r_ik and coefficients A_ik, B_ik): the field
// at i of a dipole set u is sum_k -A_ik u_k + B_ik (u_k . r_ik) r_ik.  So each field
// costs one streamed pass over the Ewald (or preconditioner) row plus one gathered
// source record per pair, with no minimum image, erfc, exp or sqrt.  The field kernels fold in the PCG vector work
// (A p = p / alpha - T p with its dot products, or z = alpha (E_precond + s r) with
// r . z).  Vectors are FP64 [3][n]; every dot product is a fixed-order sum over the
// blocks of a fixed-size grid, so runs are bitwise reproducible.  The residual norms
// are finished by the last block and read back once per iteration (16 bytes) to apply
// the reference's stopping rules.
#include <cmath>

#include "ffx_internal.cuh"

namespace ffx {

constexpr int kFieldThreads = 128;               // 4 warps, one atom per warp per step
constexpr int kFieldBlocks = 148 * 8;            // fixed grid: deterministic partials
constexpr int kVecThreads = 256;
constexpr int kVecBlocks = 148 * 2;
// Columns of the partial-sum table d_part2[block][8].
enum { C_PAP = 0, C_PAPP, C_RZ, C_RZP, C_RZN, C_RZNP, C_EPS, C_EPSP };

// Fixed-order total of column c over nb blocks by one warp (lane l sums l, l+32, ...).
__device__ __forceinline__ double warp_total(const double *__restrict__ part, int nb, int c) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int b = lane; b < nb; b += 32) s += part[b * 8 + c];
  return warp_sum(s);
}

// Block sum of up to 4 per-warp values, written to part[blockIdx.x][c0 .. c0+nv).
template <int NV>
__device__ __forceinline__ void block_store(const double *v, double *part, int c0) {
  __shared__ double sh[NV][32];
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
    part[blockIdx.x * 8 + c0 + threadIdx.x] = s;
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

// Dipole field at atom i from the cached pair row (warp cooperative): the displacement
// and A, B of each pair stream in coalesced; only the neighbour's source record is
// gathered.  T is double (plain form) or float (mixed form, FP64 reduction).  Each lane
// handles entries a and a + 32 together so that both entries' loads are in flight; the
// summation order stays a, a + 32, a + 64, ...
template <typename T>
__device__ __forceinline__ void coef_field(int i, const int *__restrict__ lst, const int *__restrict__ lst_cnt,
                                           int cap, const PairRec<T> *__restrict__ pr, const T *__restrict__ pb,
                                           const T *__restrict__ rec, double *f) {
  const int lane = threadIdx.x & 31;
  T acc[6] = {0, 0, 0, 0, 0, 0};
  const int cnt = min(lst_cnt[i], cap);
  const size_t e0 = (size_t)i * cap;
  const int *row = lst + e0;
  for (int a = lane; a < cnt; a += 64) {
    const bool two = a + 32 < cnt;
    const int a1 = two ? a + 32 : a;
    const int k0 = row[a], k1 = row[a1];
    T x0, y0, z0, A0, x1, y1, z1, A1;
    load_pair(pr, e0 + a, x0, y0, z0, A0);
    load_pair(pr, e0 + a1, x1, y1, z1, A1);
    const T B0 = pb[e0 + a], B1 = pb[e0 + a1];
    T s0[6], s1[6];
    get_rec(rec, k0, s0);
    get_rec(rec, k1, s1);
    field_term(x0, y0, z0, A0, B0, s0, acc);
    if (two) field_term(x1, y1, z1, A1, B1, s1, acc);
  }
#pragma unroll
  for (int q = 0; q < 6; q++) f[q] = warp_sum((double)acc[q]);
}

// MODE 1: initial residual r = (u_dir - u) / alpha + E(u) with u == u_dir (InitResidualRegion);
//         also writes the preconditioner source record alpha r.
// MODE 2: vec = p / alpha - E(p) and partials of p . vec and r . z (UpdateApLoop).
template <int MODE, typename T>
__global__ void __launch_bounds__(kFieldThreads) k_pcg_field(
    int n, const int *__restrict__ ewl, const int *__restrict__ ewl_cnt, int capE,
    const PairRec<T> *__restrict__ coefE, const T *__restrict__ coefEB, const T *__restrict__ rec, const double *__restrict__ ud,
    const double *__restrict__ up, const double *__restrict__ cphiD, const double *__restrict__ cphiP,
    double aewald3, const double *__restrict__ polar, const double *__restrict__ udirD,
    const double *__restrict__ udirP, const double *__restrict__ r, const double *__restrict__ rP,
    const double *__restrict__ zz, const double *__restrict__ zP, double *outD, double *outP, T *recP,
    double *part) {
  const int lane = threadIdx.x & 31;
  const int wstride = gridDim.x * (blockDim.x >> 5);
  double acc[4] = {0, 0, 0, 0};
  for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += wstride) {
    double f[6];
    coef_field(i, ewl, ewl_cnt, capE, coefE, coefEB, rec, f);
    if (lane == 0) {
      for (int d = 0; d < 3; d++) {
        f[d] += aewald3 * ud[d * n + i] - cphiD[(1 + d) * n + i];
        f[3 + d] += aewald3 * up[d * n + i] - cphiP[(1 + d) * n + i];
      }
      const double a = polar[i];
      const bool ok = a > 0.0;
      const double ip = ok ? 1.0 / a : 0.0;
      double nr[6];
      for (int d = 0; d < 3; d++) {
        const size_t j = (size_t)d * n + i;
        if (MODE == 1) {
          const double rv = ok ? (udirD[j] - ud[j]) * ip + f[d] : 0.0;
          const double rp = ok ? (udirP[j] - up[j]) * ip + f[3 + d] : 0.0;
          outD[j] = rv;
          outP[j] = rp;
          nr[d] = a * rv;
          nr[3 + d] = a * rp;
        } else {
          const double vv = ok ? ud[j] * ip - f[d] : 0.0;
          const double vp = ok ? up[j] * ip - f[3 + d] : 0.0;
          outD[j] = vv;
          outP[j] = vp;
          acc[0] += ud[j] * vv;
          acc[1] += up[j] * vp;
          acc[2] += r[j] * zz[j];
          acc[3] += rP[j] * zP[j];
        }
      }
      if (MODE == 1) put_rec(recP, i, nr[0], nr[1], nr[2], nr[3], nr[4], nr[5]);
    }
  }
  if (MODE == 2) block_store<4>(acc, part, C_PAP);
}

// z = alpha (E_precond(alpha r) + s r) (InitConjugateRegion / UpdatePreconditionerLoop);
// INIT also sets p = z (and its source record), otherwise the partials of r . z_new are
// stored.  The source record holds alpha r.
template <bool INIT, typename T>
__global__ void __launch_bounds__(kFieldThreads) k_pcg_precond(
    int n, const int *__restrict__ prl, const int *__restrict__ prl_cnt, int capP,
    const PairRec<T> *__restrict__ coefP, const T *__restrict__ coefPB, const T *__restrict__ recP, const double *__restrict__ polar,
    const double *__restrict__ r, const double *__restrict__ rP, double s, double *zz, double *zP, double *p,
    double *pP, T *recF, double *part) {
  const int lane = threadIdx.x & 31;
  const int wstride = gridDim.x * (blockDim.x >> 5);
  double acc[2] = {0, 0};
  for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += wstride) {
    double f[6];
    coef_field(i, prl, prl_cnt, capP, coefP, coefPB, recP, f);
    if (lane == 0) {
      const double a = polar[i];
      double nz[6];
      for (int d = 0; d < 3; d++) {
        const size_t j = (size_t)d * n + i;
        const double vz = a * (f[d] + s * r[j]);
        const double vp = a * (f[3 + d] + s * rP[j]);
        zz[j] = vz;
        zP[j] = vp;
        if (INIT) {
          p[j] = vz;
          pP[j] = vp;
        }
        nz[d] = vz;
        nz[3 + d] = vp;
        acc[0] += r[j] * vz;
        acc[1] += rP[j] * vp;
      }
      if (INIT) put_rec(recF, i, nz[0], nz[1], nz[2], nz[3], nz[4], nz[5]);
    }
  }
  if (!INIT) block_store<2>(acc, part, C_RZN);
}

// PCGSolver.scfByPCG stopping rules (pme/PCGSolver.java:541-570) applied on the device:
// eps = 4.80321 sqrt(max(|r_D|^2, |r_CR|^2) / n); stop with an error when eps grew (or
// is not finite) or the iteration limit is reached, stop converged when eps < polar-eps.
// A list overflow seen earlier in the evaluation also stops the loop (the host repeats
// the evaluation with larger lists).
__global__ void k_pcg_reset(PcgState *st) {
  st->eps = 100.0;
  st->iter = 0;
  st->status = FFXG_OK;
  st->cont = 1;
}

// alpha = r.z / p.Ap; r -= alpha vec; u += alpha p; |r|^2 partials; the last block
// finishes both norms, applies the stopping rules to PcgState, re-arms the counter and,
// inside a captured graph, sets the condition of the PCG while node.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_pcg_update(int n, int nbf, const double *__restrict__ vec,
                                                            const double *__restrict__ vecP,
                                                            const double *__restrict__ p,
                                                            const double *__restrict__ pP, double *r, double *rP,
                                                            double *uD, double *uP, const double *__restrict__ partF,
                                                            double *partE, unsigned *counter, PcgState *st,
                                                            int max_iter, double polar_eps, const int *flags,
                                                            cudaGraphConditionalHandle cond, int use_cond,
                                                            const double *__restrict__ polar, T *recP) {
  __shared__ double alpha[2];
  __shared__ bool last;
  if (threadIdx.x < 32) {
    const double pap = warp_total(partF, nbf, C_PAP), papP = warp_total(partF, nbf, C_PAPP);
    const double rz = warp_total(partF, nbf, C_RZ), rzP = warp_total(partF, nbf, C_RZP);
    if (threadIdx.x == 0) {
      alpha[0] = (pap != 0.0) ? rz / pap : rz;
      alpha[1] = (papP != 0.0) ? rzP / papP : rzP;
    }
  }
  __syncthreads();
  double v[2] = {0.0, 0.0};
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    double nr[6];
    for (int d = 0; d < 3; d++) {
      const size_t j = (size_t)d * n + i;
      const double rr = r[j] - alpha[0] * vec[j];
      const double rp = rP[j] - alpha[1] * vecP[j];
      r[j] = rr; rP[j] = rp;
      uD[j] += alpha[0] * p[j];
      uP[j] += alpha[1] * pP[j];
      v[0] += rr * rr;
      v[1] += rp * rp;
      nr[d] = rr;
      nr[3 + d] = rp;
    }
    const double a = polar[i];
    put_rec(recP, i, a * nr[0], a * nr[1], a * nr[2], a * nr[3], a * nr[4], a * nr[5]);
  }
  block_store<2>(v, partE, C_EPS);
  __threadfence();
  if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (last && threadIdx.x < 32) {
    __threadfence();
    const double e0 = warp_total(partE, gridDim.x, C_EPS), e1 = warp_total(partE, gridDim.x, C_EPSP);
    if (threadIdx.x == 0) {
      const double m = (e0 < e1) ? e1 : e0;
      const double eps = kElecAngToDebye * sqrt(m / (double)n);
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
      *counter = 0u;
      if (use_cond) cudaGraphSetConditional(cond, (unsigned)cont);
    }
  }
}

// beta = r.z_new / r.z_old; p = z + beta p (UpdateConjugateLoop, Fletcher-Reeves); also
// writes p's source record.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_pcg_p(int n, int nbf, const double *__restrict__ part,
                                                       const double *__restrict__ zz, const double *__restrict__ zP,
                                                       double *p, double *pP, T *recF) {
  __shared__ double beta[2];
  if (threadIdx.x < 32) {
    double old = warp_total(part, nbf, C_RZ), oldP = warp_total(part, nbf, C_RZP);
    const double nw = warp_total(part, nbf, C_RZN), nwP = warp_total(part, nbf, C_RZNP);
    if (threadIdx.x == 0) {
      if (old == 0.0) old = 1.0;
      if (oldP == 0.0) oldP = 1.0;
      beta[0] = nw / old;
      beta[1] = nwP / oldP;
    }
  }
  __syncthreads();
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    double np[6];
    for (int d = 0; d < 3; d++) {
      const size_t j = (size_t)d * n + i;
      const double a = zz[j] + beta[0] * p[j];
      const double b = zP[j] + beta[1] * pP[j];
      p[j] = a;
      pP[j] = b;
      np[d] = a;
      np[3 + d] = b;
    }
    put_rec(recF, i, np[0], np[1], np[2], np[3], np[4], np[5]);
  }
}

// ---------------------------------------------------------------------------
static double aewald3_of(const Handle &h) {
  const double a = h.prm.ewald_alpha;
  return 4.0 / 3.0 * pow(a, 3.0) / 1.7724538509055160273;
}

template <int MODE, typename T>
static void field(Handle &h, const double *ud, const double *up, double *outD, double *outP) {
  k_pcg_field<MODE, T><<<kFieldBlocks, kFieldThreads, 0, h.stream>>>(
      h.n, h.d_ewl, h.d_ewl_cnt, h.cap_ewl, reinterpret_cast<const PairRec<T> *>(h.d_coefE),
      reinterpret_cast<const T *>(h.d_coefEB), reinterpret_cast<const T *>(h.d_recF), ud, up, h.d_cphiI, h.d_cphiP,
      aewald3_of(h), h.d_polar, h.d_udirD, h.d_udirP, h.d_r, h.d_rP, h.d_zpre, h.d_zpreP, outD, outP,
      reinterpret_cast<T *>(h.d_recP), h.d_part2);
  FFX_LAUNCHED(h);
}

template <int MODE>
static void launch_field(Handle &h, const double *ud, const double *up, double *outD, double *outP) {
  if (h.mixed) field<MODE, float>(h, ud, up, outD, outP); else field<MODE, double>(h, ud, up, outD, outP);
}

template <bool INIT, typename T>
static void precond(Handle &h) {
  k_pcg_precond<INIT, T><<<kFieldBlocks, kFieldThreads, 0, h.stream>>>(
      h.n, h.d_prl, h.d_prl_cnt, h.cap_prl, reinterpret_cast<const PairRec<T> *>(h.d_coefP),
      reinterpret_cast<const T *>(h.d_coefPB), reinterpret_cast<const T *>(h.d_recP), h.d_polar, h.d_r, h.d_rP,
      h.prm.precond_scale, h.d_zpre, h.d_zpreP, h.d_p, h.d_pP, reinterpret_cast<T *>(h.d_recF), h.d_part2);
  FFX_LAUNCHED(h);
}

template <bool INIT>
static void launch_precond(Handle &h) {
  if (h.mixed) precond<INIT, float>(h); else precond<INIT, double>(h);
}

template <typename T>
static void update(Handle &h, cudaGraphConditionalHandle cond, int use_cond) {
  k_pcg_update<T><<<kVecBlocks, kVecThreads, 0, h.stream>>>(
      h.n, kFieldBlocks, h.d_vec, h.d_vecP, h.d_p, h.d_pP, h.d_r, h.d_rP, h.d_uD, h.d_uP, h.d_part2,
      h.d_part2 + 8 * 2048, h.d_counter, h.d_pcg, h.prm.max_scf_iter, h.prm.polar_eps, h.d_flags, cond, use_cond,
      h.d_polar, reinterpret_cast<T *>(h.d_recP));
  FFX_LAUNCHED(h);
}

template <typename T>
static void new_direction(Handle &h) {
  k_pcg_p<T><<<kVecBlocks, kVecThreads, 0, h.stream>>>(h.n, kFieldBlocks, h.d_part2, h.d_zpre, h.d_zpreP, h.d_p,
                                                       h.d_pP, reinterpret_cast<T *>(h.d_recF));
  FFX_LAUNCHED(h);
}

// One PCG step up to the stopping test: recip field of p, A p with its dot products, update.
static void pcg_step(Handle &h, cudaGraphConditionalHandle cond, int use_cond) {
  int tk = timer_begin(h, FFXG_STAGE_IND_RECIP);
  launch_induced_recip(h, h.d_p, h.d_pP);
  timer_end(h, tk);
  tk = timer_begin(h, FFXG_STAGE_IND_FIELD);
  launch_field<2>(h, h.d_p, h.d_pP, h.d_vec, h.d_vecP);
  timer_end(h, tk);
  tk = timer_begin(h, FFXG_STAGE_PCG_VECTOR);
  if (h.mixed) update<float>(h, cond, use_cond); else update<double>(h, cond, use_cond);
  timer_end(h, tk);
}

// New search direction: z = M r (with r . z partials), then p = z + beta p.
static void pcg_direction(Handle &h) {
  int tk = timer_begin(h, FFXG_STAGE_PRECOND);
  launch_precond<false>(h);
  timer_end(h, tk);
  tk = timer_begin(h, FFXG_STAGE_PCG_VECTOR);
  if (h.mixed) new_direction<float>(h); else new_direction<double>(h);
  timer_end(h, tk);
}

// The solve.  Directly (capture false): the host reads the device's stopping decision
// after every update (24 bytes).  Under stream capture (capture true): the first step is
// recorded in line and the rest as a conditional WHILE node whose body (direction, step)
// the update kernel re-arms on the device, so the loop runs with no host round trip.
// Either way the loop ends by max_scf_iter at the latest.
int run_pcg(Handle &h, bool capture) {
  k_pcg_reset<<<1, 1, 0, h.stream>>>(h.d_pcg);
  FFX_LAUNCHED(h);
  // Field of the direct dipoles (u == u_dir at entry) gives the initial residual.
  int tk = timer_begin(h, FFXG_STAGE_IND_RECIP);
  launch_induced_recip(h, h.d_uD, h.d_uP);
  timer_end(h, tk);
  tk = timer_begin(h, FFXG_STAGE_IND_FIELD);
  launch_field<1>(h, h.d_uD, h.d_uP, h.d_r, h.d_rP);
  timer_end(h, tk);
  tk = timer_begin(h, FFXG_STAGE_PRECOND);
  launch_precond<true>(h);
  timer_end(h, tk);
  if (!capture) {
    while (true) {
      pcg_step(h, 0, 0);
      cudaMemcpyAsync(h.h_pcg, h.d_pcg, sizeof(PcgState), cudaMemcpyDeviceToHost, h.stream);
      if (cudaStreamSynchronize(h.stream) != cudaSuccess) return FFXG_ERR_CUDA;
      if (!h.h_pcg->cont) break;
      pcg_direction(h);
    }
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
  pcg_step(h, cond, 1);
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
  pcg_direction(h);
  pcg_step(h, cond, 1);
  h.graph_body_launches = h.launches - before;
  h.stream = main;
  if (cudaStreamEndCapture(h.side, &body) != cudaSuccess) return FFXG_ERR_CUDA;
  return FFXG_OK;
}

}  // namespace ffx
