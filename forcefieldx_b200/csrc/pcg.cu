// pcg.cu -- preconditioned conjugate-gradient induced-dipole solver.
//
// PCGSolver.scfByPCG (pme/PCGSolver.java:487-602) with InitResidualRegion (:609-663),
// InitConjugateRegion (:670-770), UpdateResidualRegion (:773-985) and
// UpdateConjugateRegion (:991-1180, Fletcher-Reeves).  The D and CR systems advance
// together with separate scalars.  Vectors are FP64 [3][n]; every dot product is a
// fixed-order two-level sum (per-block partials, then a fixed-order total), so runs
// are bitwise reproducible.  The host reads back one 16-byte pair of residual norms
// per iteration to apply the reference's stopping rules.
#include <cmath>

#include "ffx_internal.cuh"

namespace ffx {

constexpr int kPcgThreads = 256;
enum { P_PAP = 0, P_PAPP, P_RZ, P_RZP, P_EPS, P_EPSP, P_RZN, P_RZNP, P_NCOL };

__device__ __forceinline__ void block_sums(double *vals, int nv, double *part) {
  __shared__ double sh[P_NCOL][kPcgThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int v = 0; v < nv; v++) {
    const double s = warp_sum(vals[v]);
    if (lane == 0) sh[v][wid] = s;
  }
  __syncthreads();
  if (threadIdx.x < nv) {
    double s = 0.0;
    for (int w = 0; w < kPcgThreads / 32; w++) s += sh[threadIdx.x][w];
    part[threadIdx.x] = s;
  }
}

// Fixed-order total of column c over nb blocks; computed by every block identically.
__device__ __forceinline__ double total(const double *__restrict__ part, int nb, int c) {
  double s = 0.0;
  for (int b = 0; b < nb; b++) s += part[b * P_NCOL + c];
  return s;
}

__global__ void k_pcg_residual_init(int n, const double *__restrict__ polar, const double *__restrict__ udD,
                                    const double *__restrict__ udP, const double *__restrict__ uD,
                                    const double *__restrict__ uP, const double *__restrict__ fD,
                                    const double *__restrict__ fP, double *r, double *rP) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double a = polar[i];
  const bool ok = a > 0.0;
  const double ip = ok ? 1.0 / a : 0.0;
  for (int d = 0; d < 3; d++) {
    const size_t j = (size_t)d * n + i;
    r[j] = ok ? (udD[j] - uD[j]) * ip + fD[j] : 0.0;
    rP[j] = ok ? (udP[j] - uP[j]) * ip + fP[j] : 0.0;
  }
}

// z = alpha (E_precond + s r); optionally p = z (first iteration) and partial r.z_new.
template <bool INIT>
__global__ void __launch_bounds__(kPcgThreads) k_pcg_z(int n, const double *__restrict__ polar,
                                                       const double *__restrict__ preD,
                                                       const double *__restrict__ preP, const double *__restrict__ r,
                                                       const double *__restrict__ rP, double s, double *z, double *zP,
                                                       double *p, double *pP, double *part) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (i < n) {
    const double a = polar[i];
    for (int d = 0; d < 3; d++) {
      const size_t j = (size_t)d * n + i;
      const double zz = a * (preD[j] + s * r[j]);
      const double zp = a * (preP[j] + s * rP[j]);
      z[j] = zz; zP[j] = zp;
      if (INIT) { p[j] = zz; pP[j] = zp; }
      v[0] += r[j] * zz;
      v[1] += rP[j] * zp;
    }
  }
  if (!INIT) block_sums(v, 2, part + blockIdx.x * P_NCOL + P_RZN);
}

// vec = p / alpha - T p; partials of p.Ap and r.z (UpdateApLoop).
__global__ void __launch_bounds__(kPcgThreads) k_pcg_ap(int n, const double *__restrict__ polar,
                                                        const double *__restrict__ p, const double *__restrict__ pP,
                                                        const double *__restrict__ fD, const double *__restrict__ fP,
                                                        const double *__restrict__ r, const double *__restrict__ rP,
                                                        const double *__restrict__ z, const double *__restrict__ zP,
                                                        double *vec, double *vecP, double *part) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[4] = {0, 0, 0, 0};
  if (i < n) {
    const double a = polar[i];
    const bool ok = a > 0.0;
    const double ip = ok ? 1.0 / a : 0.0;
    for (int d = 0; d < 3; d++) {
      const size_t j = (size_t)d * n + i;
      const double vv = ok ? p[j] * ip - fD[j] : 0.0;
      const double vp = ok ? pP[j] * ip - fP[j] : 0.0;
      vec[j] = vv; vecP[j] = vp;
      v[0] += p[j] * vv;
      v[1] += pP[j] * vp;
      v[2] += r[j] * z[j];
      v[3] += rP[j] * zP[j];
    }
  }
  block_sums(v, 4, part + blockIdx.x * P_NCOL + P_PAP);
}

// r -= alpha vec; u += alpha p; partial |r|^2 (UpdateResidualAndInducedLoop).
__global__ void __launch_bounds__(kPcgThreads) k_pcg_update(int n, int nb, const double *__restrict__ vec,
                                                            const double *__restrict__ vecP,
                                                            const double *__restrict__ p,
                                                            const double *__restrict__ pP, double *r, double *rP,
                                                            double *uD, double *uP, double *part) {
  __shared__ double alpha[2];
  if (threadIdx.x == 0) {
    const double pap = total(part, nb, P_PAP), papP = total(part, nb, P_PAPP);
    const double rz = total(part, nb, P_RZ), rzP = total(part, nb, P_RZP);
    alpha[0] = (pap != 0.0) ? rz / pap : rz;
    alpha[1] = (papP != 0.0) ? rzP / papP : rzP;
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (i < n) {
    for (int d = 0; d < 3; d++) {
      const size_t j = (size_t)d * n + i;
      const double rr = r[j] - alpha[0] * vec[j];
      const double rp = rP[j] - alpha[1] * vecP[j];
      r[j] = rr; rP[j] = rp;
      uD[j] += alpha[0] * p[j];
      uP[j] += alpha[1] * pP[j];
      v[0] += rr * rr;
      v[1] += rp * rp;
    }
  }
  __syncthreads();
  block_sums(v, 2, part + blockIdx.x * P_NCOL + P_EPS);
}

__global__ void k_pcg_eps(int nb, const double *__restrict__ part, double *out) {
  if (threadIdx.x == 0) {
    out[0] = total(part, nb, P_EPS);
    out[1] = total(part, nb, P_EPSP);
  }
}

// beta = r.z_new / r.z_old; p = z + beta p (UpdateConjugateLoop).
__global__ void __launch_bounds__(kPcgThreads) k_pcg_p(int n, int nb, const double *__restrict__ part,
                                                       const double *__restrict__ z, const double *__restrict__ zP,
                                                       double *p, double *pP) {
  __shared__ double beta[2];
  if (threadIdx.x == 0) {
    double old = total(part, nb, P_RZ), oldP = total(part, nb, P_RZP);
    if (old == 0.0) old = 1.0;
    if (oldP == 0.0) oldP = 1.0;
    beta[0] = total(part, nb, P_RZN) / old;
    beta[1] = total(part, nb, P_RZNP) / oldP;
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int d = 0; d < 3; d++) {
    const size_t j = (size_t)d * n + i;
    p[j] = z[j] + beta[0] * p[j];
    pP[j] = zP[j] + beta[1] * pP[j];
  }
}

// Reciprocal (spread, FFT, potential) and real-space parts of one induced field, timed separately.
static void induced_field_timed(Handle &h, const double *ud, const double *up, double *outD, double *outP) {
  int tk = timer_begin(h, FFXG_STAGE_IND_RECIP);
  launch_induced_recip(h, ud, up);
  timer_end(h, tk);
  tk = timer_begin(h, FFXG_STAGE_IND_FIELD);
  launch_induced_real(h, ud, up, outD, outP);
  timer_end(h, tk);
}

int run_pcg(Handle &h) {
  const int n = h.n;
  const int nb = nblocks(n, kPcgThreads);
  double *part = h.d_partials;
  double *fD = h.d_fieldD, *fP = h.d_fieldP;  // reused as T p scratch
  double *preD = h.d_vec + 0, *preP = h.d_vecP;  // preconditioner field scratch shares vec storage
  // Field of the direct dipoles: u == udir at entry.
  induced_field_timed(h, h.d_uD, h.d_uP, fD, fP);
  int tk = timer_begin(h, FFXG_STAGE_PCG_VECTOR);
  k_pcg_residual_init<<<nblocks(n, 256), 256, 0, h.stream>>>(n, h.d_polar, h.d_udirD, h.d_udirP, h.d_uD, h.d_uP, fD,
                                                              fP, h.d_r, h.d_rP);
  timer_end(h, tk);
  tk = timer_begin(h, FFXG_STAGE_PRECOND);
  launch_precond_field(h, h.d_r, h.d_rP, preD, preP);
  timer_end(h, tk);
  tk = timer_begin(h, FFXG_STAGE_PCG_VECTOR);
  k_pcg_z<true><<<nb, kPcgThreads, 0, h.stream>>>(n, h.d_polar, preD, preP, h.d_r, h.d_rP, h.prm.precond_scale,
                                                  h.d_zpre, h.d_zpreP, h.d_p, h.d_pP, part);
  timer_end(h, tk);
  h.launches += 2;
  int iter = 0;
  double eps = 100.0;
  int status = FFXG_OK;
  while (true) {
    induced_field_timed(h, h.d_p, h.d_pP, fD, fP);
    tk = timer_begin(h, FFXG_STAGE_PCG_VECTOR);
    k_pcg_ap<<<nb, kPcgThreads, 0, h.stream>>>(n, h.d_polar, h.d_p, h.d_pP, fD, fP, h.d_r, h.d_rP, h.d_zpre, h.d_zpreP,
                                               h.d_vec, h.d_vecP, part);
    k_pcg_update<<<nb, kPcgThreads, 0, h.stream>>>(n, nb, h.d_vec, h.d_vecP, h.d_p, h.d_pP, h.d_r, h.d_rP, h.d_uD,
                                                   h.d_uP, part);
    k_pcg_eps<<<1, 32, 0, h.stream>>>(nb, part, h.d_scalars);
    timer_end(h, tk);
    h.launches += 3;
    cudaMemcpyAsync(h.h_scalars, h.d_scalars, 2 * sizeof(double), cudaMemcpyDeviceToHost, h.stream);
    if (cudaStreamSynchronize(h.stream) != cudaSuccess) return FFXG_ERR_CUDA;
    const double previous = eps;
    eps = kElecAngToDebye * std::sqrt(std::max(h.h_scalars[0], h.h_scalars[1]) / (double)n);
    iter++;
    if (!(eps <= previous)) { status = std::isfinite(eps) ? FFXG_ERR_SCF_DIVERGED : FFXG_ERR_NONFINITE; break; }
    if (iter >= h.prm.max_scf_iter) { status = FFXG_ERR_SCF_MAXITER; break; }
    if (eps < h.prm.polar_eps) break;
    tk = timer_begin(h, FFXG_STAGE_PRECOND);
    launch_precond_field(h, h.d_r, h.d_rP, preD, preP);
    timer_end(h, tk);
    tk = timer_begin(h, FFXG_STAGE_PCG_VECTOR);
    k_pcg_z<false><<<nb, kPcgThreads, 0, h.stream>>>(n, h.d_polar, preD, preP, h.d_r, h.d_rP, h.prm.precond_scale,
                                                     h.d_zpre, h.d_zpreP, nullptr, nullptr, part);
    k_pcg_p<<<nb, kPcgThreads, 0, h.stream>>>(n, nb, part, h.d_zpre, h.d_zpreP, h.d_p, h.d_pP);
    timer_end(h, tk);
    h.launches += 2;
  }
  h.scf_iter = iter;
  return status;
}

}  // namespace ffx
