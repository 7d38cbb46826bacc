// real.cu -- real-space Ewald pair kernels (warp per atom, gather over the full list).
//
//  k_permanent_field   PermanentRealSpaceFieldLoop (pme/PermanentFieldRegion.java:595-815)
//  k_direct            DirectLoop (pme/DirectRegion.java:170-243)
//  k_induced_field     InducedDipoleFieldRegion (pme/InducedDipoleFieldRegion.java:308-470) plus the
//                      self and reciprocal terms of InducedDipoleFieldReduceRegion (:159-207)
//  k_precond_field     InducedPreconditionerFieldLoop (pme/PCGSolver.java:1254-1400), Ewald off
//  k_real_energy       RealSpaceEnergyLoop.permanentPair / polarizationPair
//                      (pme/RealSpaceEnergyRegion.java:1190-1476, 1700-2177)
//
// Each list stores a pair in both directions, so a warp accumulates only its own
// atom's field, force and torque: no atomics, deterministic sums, and the
// reference's k-side terms (ttm3) are never evaluated.  Pair energies are taken
// with weight 1/2 per direction.  Mask scale factors come from the per-atom
// exclusion list; the masks are symmetric, so the i-side lookup reproduces the
// reference's applyMask(i) (PermanentFieldRegion.java:231-258,
// RealSpaceEnergyRegion.java:307-342).
#include "ffx_internal.cuh"

namespace ffx {

enum { t000 = 0, t100, t010, t001, t200, t020, t002, t110, t101, t011 };


struct EwaldCoef {
  double aewald, an0, an1, an2, an3, an4, an5, aewald3, electric;
};

__device__ __forceinline__ unsigned excl_code(int i, int k, const int *__restrict__ ptr, const int *__restrict__ ek,
                                              const unsigned *__restrict__ code, const int *__restrict__ lo,
                                              const int *__restrict__ hi) {
  if (k < lo[i] || k > hi[i]) return 0u;
  const int e1 = ptr[i + 1];
  for (int e = ptr[i]; e < e1; e++)
    if (ek[e] == k) return code[e];
  return 0u;
}

struct Excl {
  const int *ptr, *k, *lo, *hi;
  const unsigned *code;
};

// ---------------------------------------------------------------------------
__global__ void k_permanent_field(int n, const double *__restrict__ x, const double *__restrict__ y,
                                  const double *__restrict__ z, Box bx, const double *__restrict__ gm,
                                  const double *__restrict__ ipdamp, const double *__restrict__ thole,
                                  const int *__restrict__ ewl, const int *__restrict__ ewl_cnt, int capE, Excl ex,
                                  EwaldCoef ec, ScaleTables c_scales, double *fieldD, double *fieldP) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int i = warp;
  const double xi = x[i], yi = y[i], zi = z[i];
  const double pdi = ipdamp[i], pti = thole[i];
  double fx = 0, fy = 0, fz = 0, px = 0, py = 0, pz = 0;
  const int cnt = min(ewl_cnt[i], capE);
  const int *row = ewl + (size_t)i * capE;
  for (int a = lane; a < cnt; a += 32) {
    const int k = row[a];
    double xr = __dsub_rn(x[k], xi), yr = __dsub_rn(y[k], yi), zr = __dsub_rn(z[k], zi);
    const double r2 = image_exact(xr, yr, zr, bx);
    const double ck = gm[t000 * n + k], dkx = gm[t100 * n + k], dky = gm[t010 * n + k], dkz = gm[t001 * n + k];
    const double qkxx = gm[t200 * n + k] * (1.0 / 3.0), qkyy = gm[t020 * n + k] * (1.0 / 3.0);
    const double qkzz = gm[t002 * n + k] * (1.0 / 3.0), qkxy = gm[t110 * n + k] * (1.0 / 3.0);
    const double qkxz = gm[t101 * n + k] * (1.0 / 3.0), qkyz = gm[t011 * n + k] * (1.0 / 3.0);
    const double r = sqrt(r2);
    const double ralpha = ec.aewald * r;
    const double exp2a = exp(-ralpha * ralpha);
    const double rr1 = 1.0 / r, rr2 = rr1 * rr1;
    const double bn0 = erfc(ralpha) * rr1;
    const double bn1 = (bn0 + ec.an0 * exp2a) * rr2;
    const double bn2 = (3.0 * bn1 + ec.an1 * exp2a) * rr2;
    const double bn3 = (5.0 * bn2 + ec.an2 * exp2a) * rr2;
    double scale3 = 1.0, scale5 = 1.0, scale7 = 1.0;
    double damp = pdi * ipdamp[k];
    const double pgamma = fmin(pti, thole[k]);
    const double rdamp = r * damp;
    damp = -pgamma * rdamp * rdamp * rdamp;
    if (damp > -50.0) {
      const double expdamp = exp(damp);
      scale3 = 1.0 - expdamp;
      scale5 = 1.0 - expdamp * (1.0 - damp);
      scale7 = 1.0 - expdamp * (1.0 - damp + 0.6 * damp * damp);
    }
    const unsigned code = excl_code(i, k, ex.ptr, ex.k, ex.code, ex.lo, ex.hi);
    const double scale = c_scales.d[(code >> 6) & 1u];
    const double scalep = c_scales.p[(code >> 3) & 7u];
    const double dsc3 = scale3 * scale, dsc5 = scale5 * scale, dsc7 = scale7 * scale;
    const double psc3 = scale3 * scalep, psc5 = scale5 * scalep, psc7 = scale7 * scalep;
    const double rr3 = rr1 * rr2, rr5 = 3.0 * rr3 * rr2, rr7 = 5.0 * rr5 * rr2;
    const double drr3 = (1.0 - dsc3) * rr3, drr5 = (1.0 - dsc5) * rr5, drr7 = (1.0 - dsc7) * rr7;
    const double prr3 = (1.0 - psc3) * rr3, prr5 = (1.0 - psc5) * rr5, prr7 = (1.0 - psc7) * rr7;
    const double dkr = dkx * xr + dky * yr + dkz * zr;
    const double qkx = 2.0 * (qkxx * xr + qkxy * yr + qkxz * zr);
    const double qky = 2.0 * (qkxy * xr + qkyy * yr + qkyz * zr);
    const double qkz = 2.0 * (qkxz * xr + qkyz * yr + qkzz * zr);
    const double qkr = (qkx * xr + qky * yr + qkz * zr) * 0.5;
    const double bn123k = bn1 * ck - bn2 * dkr + bn3 * qkr;
    const double fimx = -xr * bn123k - bn1 * dkx + bn2 * qkx;
    const double fimy = -yr * bn123k - bn1 * dky + bn2 * qky;
    const double fimz = -zr * bn123k - bn1 * dkz + bn2 * qkz;
    const double drr357k = drr3 * ck - drr5 * dkr + drr7 * qkr;
    const double fidx = -xr * drr357k - drr3 * dkx + drr5 * qkx;
    const double fidy = -yr * drr357k - drr3 * dky + drr5 * qky;
    const double fidz = -zr * drr357k - drr3 * dkz + drr5 * qkz;
    fx += fimx - fidx; fy += fimy - fidy; fz += fimz - fidz;
    const double prr357k = prr3 * ck - prr5 * dkr + prr7 * qkr;
    const double fipx = -xr * prr357k - prr3 * dkx + prr5 * qkx;
    const double fipy = -yr * prr357k - prr3 * dky + prr5 * qky;
    const double fipz = -zr * prr357k - prr3 * dkz + prr5 * qkz;
    px += fimx - fipx; py += fimy - fipy; pz += fimz - fipz;
  }
  fx = warp_sum(fx); fy = warp_sum(fy); fz = warp_sum(fz);
  px = warp_sum(px); py = warp_sum(py); pz = warp_sum(pz);
  if (lane == 0) {
    fieldD[i] = fx; fieldD[n + i] = fy; fieldD[2 * n + i] = fz;
    fieldP[i] = px; fieldP[n + i] = py; fieldP[2 * n + i] = pz;
  }
}

// Real-space lists, permanent field, cached pair coefficients and direct dipoles in one
// pass (PermanentRealSpaceFieldLoop, pme/PermanentFieldRegion.java:595-815, which also
// derives the Ewald and preconditioner lists; DirectLoop, pme/DirectRegion.java:170-243).
// Phase 1 compacts the buffered row into the Ewald row (r2 <= off2) and the
// preconditioner row (r < pcut).  Phase 2 walks the Ewald row: it accumulates the D and
// CR permanent fields and stores, per entry, the two symmetric coefficients of the
// unmasked Thole-damped dipole field, A = bn1 - (1 - s3) rr3 and B = bn2 - (1 - s5) rr5,
// so the field of any dipole set is -A u_k + B (u_k . r) r; entries inside the
// preconditioner cutoff also store the Ewald-free pair (pme/PCGSolver.java:1300-1331).
__global__ void __launch_bounds__(128) k_realspace_field(
    int n, const double *__restrict__ x, const double *__restrict__ y, const double *__restrict__ z, Box bx,
    const double *__restrict__ gm, const double *__restrict__ ipdamp, const double *__restrict__ thole,
    const int *__restrict__ nbr, const int *__restrict__ nbr_cnt, int cap, double off2, double pcut, int *ewl,
    int *ewl_cnt, int capE, int *prl, int *prl_cnt, int capP, double2 *coefE, double2 *coefP, Excl ex, EwaldCoef ec,
    ScaleTables c_scales, const double *__restrict__ cphi, const double *__restrict__ polar, int direct,
    double *fieldD, double *fieldP, double *uD, double *uP, double *udD, double *udP, int *flags) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int i = warp;
  const unsigned lt = (1u << lane) - 1u;
  const double xi = x[i], yi = y[i], zi = z[i];
  // ---- phase 1: sub-lists
  {
    const int cnt = min(nbr_cnt[i], cap);
    const int *row = nbr + (size_t)i * cap;
    int ce = 0, cp = 0;
    for (int base = 0; base < cnt; base += 32) {
      const int a = base + lane;
      bool ew = false, pr = false;
      int k = -1;
      if (a < cnt) {
        k = row[a];
        double dx = __dsub_rn(x[k], xi), dy = __dsub_rn(y[k], yi), dz = __dsub_rn(z[k], zi);
        const double r2 = image_exact(dx, dy, dz, bx);
        ew = r2 <= off2;
        pr = ew && (sqrt(r2) < pcut);
      }
      const unsigned me = __ballot_sync(0xffffffffu, ew);
      const unsigned mp = __ballot_sync(0xffffffffu, pr);
      if (ew) {
        const int pos = ce + __popc(me & lt);
        if (pos < capE) ewl[(size_t)i * capE + pos] = k;
      }
      if (pr) {
        const int pos = cp + __popc(mp & lt);
        if (pos < capP) prl[(size_t)i * capP + pos] = k;
      }
      ce += __popc(me);
      cp += __popc(mp);
    }
    if (lane == 0) {
      ewl_cnt[i] = ce;
      prl_cnt[i] = cp;
      if (ce > capE) atomicOr(flags, FLAG_EWALD_OVERFLOW);
      if (cp > capP) atomicOr(flags, FLAG_PRECOND_OVERFLOW);
    }
  }
  __syncwarp();
  // ---- phase 2: permanent field and coefficients
  const double pdi = ipdamp[i], pti = thole[i];
  double fx = 0, fy = 0, fz = 0, px = 0, py = 0, pz = 0;
  const int cnt = min(ewl_cnt[i], capE);
  const int *row = ewl + (size_t)i * capE;
  int cp = 0;
  for (int base = 0; base < cnt; base += 32) {
    const int a = base + lane;
    const bool act = a < cnt;
    bool pr = false;
    double2 cpre = make_double2(0.0, 0.0);
    if (act) {
      const int k = row[a];
      double xr = __dsub_rn(x[k], xi), yr = __dsub_rn(y[k], yi), zr = __dsub_rn(z[k], zi);
      const double r2 = image_exact(xr, yr, zr, bx);
      const double ck = gm[t000 * n + k], dkx = gm[t100 * n + k], dky = gm[t010 * n + k], dkz = gm[t001 * n + k];
      const double qkxx = gm[t200 * n + k] * (1.0 / 3.0), qkyy = gm[t020 * n + k] * (1.0 / 3.0);
      const double qkzz = gm[t002 * n + k] * (1.0 / 3.0), qkxy = gm[t110 * n + k] * (1.0 / 3.0);
      const double qkxz = gm[t101 * n + k] * (1.0 / 3.0), qkyz = gm[t011 * n + k] * (1.0 / 3.0);
      const double r = sqrt(r2);
      const double ralpha = ec.aewald * r;
      const double exp2a = exp(-ralpha * ralpha);
      const double rr1 = 1.0 / r, rr2 = rr1 * rr1;
      const double bn0 = erfc(ralpha) * rr1;
      const double bn1 = (bn0 + ec.an0 * exp2a) * rr2;
      const double bn2 = (3.0 * bn1 + ec.an1 * exp2a) * rr2;
      const double bn3 = (5.0 * bn2 + ec.an2 * exp2a) * rr2;
      double scale3 = 1.0, scale5 = 1.0, scale7 = 1.0;
      double damp = pdi * ipdamp[k];
      const double pgamma = fmin(pti, thole[k]);
      const double rdamp = r * damp;
      damp = -pgamma * rdamp * rdamp * rdamp;
      if (damp > -50.0) {
        const double expdamp = exp(damp);
        scale3 = 1.0 - expdamp;
        scale5 = 1.0 - expdamp * (1.0 - damp);
        scale7 = 1.0 - expdamp * (1.0 - damp + 0.6 * damp * damp);
      }
      const unsigned code = excl_code(i, k, ex.ptr, ex.k, ex.code, ex.lo, ex.hi);
      const double scale = c_scales.d[(code >> 6) & 1u];
      const double scalep = c_scales.p[(code >> 3) & 7u];
      const double dsc3 = scale3 * scale, dsc5 = scale5 * scale, dsc7 = scale7 * scale;
      const double psc3 = scale3 * scalep, psc5 = scale5 * scalep, psc7 = scale7 * scalep;
      const double rr3 = rr1 * rr2, rr5 = 3.0 * rr3 * rr2, rr7 = 5.0 * rr5 * rr2;
      const double drr3 = (1.0 - dsc3) * rr3, drr5 = (1.0 - dsc5) * rr5, drr7 = (1.0 - dsc7) * rr7;
      const double prr3 = (1.0 - psc3) * rr3, prr5 = (1.0 - psc5) * rr5, prr7 = (1.0 - psc7) * rr7;
      const double dkr = dkx * xr + dky * yr + dkz * zr;
      const double qkx = 2.0 * (qkxx * xr + qkxy * yr + qkxz * zr);
      const double qky = 2.0 * (qkxy * xr + qkyy * yr + qkyz * zr);
      const double qkz = 2.0 * (qkxz * xr + qkyz * yr + qkzz * zr);
      const double qkr = (qkx * xr + qky * yr + qkz * zr) * 0.5;
      const double bn123k = bn1 * ck - bn2 * dkr + bn3 * qkr;
      const double fimx = -xr * bn123k - bn1 * dkx + bn2 * qkx;
      const double fimy = -yr * bn123k - bn1 * dky + bn2 * qky;
      const double fimz = -zr * bn123k - bn1 * dkz + bn2 * qkz;
      const double drr357k = drr3 * ck - drr5 * dkr + drr7 * qkr;
      const double fidx = -xr * drr357k - drr3 * dkx + drr5 * qkx;
      const double fidy = -yr * drr357k - drr3 * dky + drr5 * qky;
      const double fidz = -zr * drr357k - drr3 * dkz + drr5 * qkz;
      fx += fimx - fidx; fy += fimy - fidy; fz += fimz - fidz;
      const double prr357k = prr3 * ck - prr5 * dkr + prr7 * qkr;
      const double fipx = -xr * prr357k - prr3 * dkx + prr5 * qkx;
      const double fipy = -yr * prr357k - prr3 * dky + prr5 * qky;
      const double fipz = -zr * prr357k - prr3 * dkz + prr5 * qkz;
      px += fimx - fipx; py += fimy - fipy; pz += fimz - fipz;
      // Induced-field coefficients (no masks), InducedDipoleFieldRegion.java:383-404.
      const double urr3 = (1.0 - scale3) * rr3, urr5 = (1.0 - scale5) * rr5;
      if (a < capE) coefE[(size_t)i * capE + a] = make_double2(bn1 - urr3, bn2 - urr5);
      pr = r < pcut;
      if (pr) {
        const double b1 = rr1 * rr2, b2 = 3.0 * b1 * rr2;   // Ewald off: bn0 = 1/r
        cpre = make_double2(b1 - urr3, b2 - urr5);
      }
    }
    const unsigned mp = __ballot_sync(0xffffffffu, pr);
    if (pr) {
      const int pos = cp + __popc(mp & lt);
      if (pos < capP) coefP[(size_t)i * capP + pos] = cpre;
    }
    cp += __popc(mp);
  }
  fx = warp_sum(fx); fy = warp_sum(fy); fz = warp_sum(fz);
  px = warp_sum(px); py = warp_sum(py); pz = warp_sum(pz);
  if (lane == 0) {
    if (direct) {
      const double a = polar[i];
      const double f0 = ec.aewald3 * gm[t100 * n + i] - cphi[1 * n + i];
      const double f1 = ec.aewald3 * gm[t010 * n + i] - cphi[2 * n + i];
      const double f2 = ec.aewald3 * gm[t001 * n + i] - cphi[3 * n + i];
      fx += f0; fy += f1; fz += f2;
      px += f0; py += f1; pz += f2;
      uD[i] = a * fx; uD[n + i] = a * fy; uD[2 * n + i] = a * fz;
      uP[i] = a * px; uP[n + i] = a * py; uP[2 * n + i] = a * pz;
      udD[i] = a * fx; udD[n + i] = a * fy; udD[2 * n + i] = a * fz;
      udP[i] = a * px; udP[n + i] = a * py; udP[2 * n + i] = a * pz;
    }
    fieldD[i] = fx; fieldD[n + i] = fy; fieldD[2 * n + i] = fz;
    fieldP[i] = px; fieldP[n + i] = py; fieldP[2 * n + i] = pz;
  }
}

// field += aewald3 * d_i - phi_recip (DirectLoop); u = alpha * field.
__global__ void k_direct(int n, const double *__restrict__ gm, const double *__restrict__ cphi,
                         const double *__restrict__ polar, double aewald3, double *fieldD, double *fieldP, double *uD,
                         double *uP, double *udD, double *udP) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double a = polar[i];
  for (int d = 0; d < 3; d++) {
    const double f = aewald3 * gm[(1 + d) * n + i] - cphi[(1 + d) * n + i];
    const double fd = fieldD[d * n + i] + f, fp = fieldP[d * n + i] + f;
    fieldD[d * n + i] = fd;
    fieldP[d * n + i] = fp;
    uD[d * n + i] = a * fd; udD[d * n + i] = a * fd;
    uP[d * n + i] = a * fp; udP[d * n + i] = a * fp;
  }
}

// Real-space field of two dipole sets over a list; with self/recip terms when cphi != null.
template <bool EWALD>
__global__ void k_dipole_field(int n, const double *__restrict__ x, const double *__restrict__ y,
                               const double *__restrict__ z, Box bx, const double *__restrict__ ipdamp,
                               const double *__restrict__ thole, const int *__restrict__ lst,
                               const int *__restrict__ lst_cnt, int cap, EwaldCoef ec,
                               const double *__restrict__ ud, const double *__restrict__ up,
                               const double *__restrict__ scale_by,  // polarizability multiplier or null
                               const double *__restrict__ cphiD, const double *__restrict__ cphiP, double *outD,
                               double *outP) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int i = warp;
  const double xi = x[i], yi = y[i], zi = z[i];
  const double pdi = ipdamp[i], pti = thole[i];
  double fx = 0, fy = 0, fz = 0, px = 0, py = 0, pz = 0;
  const int cnt = min(lst_cnt[i], cap);
  const int *row = lst + (size_t)i * cap;
  for (int a = lane; a < cnt; a += 32) {
    const int k = row[a];
    double xr = __dsub_rn(x[k], xi), yr = __dsub_rn(y[k], yi), zr = __dsub_rn(z[k], zi);
    const double r2 = image_exact(xr, yr, zr, bx);
    const double r = sqrt(r2);
    const double rr1 = 1.0 / r, rr2 = rr1 * rr1;
    double bn1, bn2;
    if (EWALD) {
      const double ralpha = ec.aewald * r;
      const double exp2a = exp(-ralpha * ralpha);
      const double bn0 = erfc(ralpha) * rr1;
      bn1 = (bn0 + ec.an0 * exp2a) * rr2;
      bn2 = (3.0 * bn1 + ec.an1 * exp2a) * rr2;
    } else {
      bn1 = rr1 * rr2;
      bn2 = 3.0 * bn1 * rr2;
    }
    double scale3 = 1.0, scale5 = 1.0;
    double damp = pdi * ipdamp[k];
    const double pgamma = fmin(pti, thole[k]);
    const double rdamp = r * damp;
    damp = -pgamma * rdamp * rdamp * rdamp;
    if (damp > -50.0) {
      const double expdamp = exp(damp);
      scale3 = 1.0 - expdamp;
      scale5 = 1.0 - expdamp * (1.0 - damp);
    }
    double rr3 = rr1 * rr2;
    double rr5 = 3.0 * rr3 * rr2;
    rr3 *= (1.0 - scale3);
    rr5 *= (1.0 - scale5);
    const double sk = scale_by ? scale_by[k] : 1.0;
    const double ukx = sk * ud[k], uky = sk * ud[n + k], ukz = sk * ud[2 * n + k];
    const double ukr = ukx * xr + uky * yr + ukz * zr;
    const double bn2ukr = bn2 * ukr, rr5ukr = rr5 * ukr;
    fx += (-bn1 * ukx + bn2ukr * xr) - (-rr3 * ukx + rr5ukr * xr);
    fy += (-bn1 * uky + bn2ukr * yr) - (-rr3 * uky + rr5ukr * yr);
    fz += (-bn1 * ukz + bn2ukr * zr) - (-rr3 * ukz + rr5ukr * zr);
    const double pkx = sk * up[k], pky = sk * up[n + k], pkz = sk * up[2 * n + k];
    const double pkr = pkx * xr + pky * yr + pkz * zr;
    const double bn2pkr = bn2 * pkr, rr5pkr = rr5 * pkr;
    px += (-bn1 * pkx + bn2pkr * xr) - (-rr3 * pkx + rr5pkr * xr);
    py += (-bn1 * pky + bn2pkr * yr) - (-rr3 * pky + rr5pkr * yr);
    pz += (-bn1 * pkz + bn2pkr * zr) - (-rr3 * pkz + rr5pkr * zr);
  }
  fx = warp_sum(fx); fy = warp_sum(fy); fz = warp_sum(fz);
  px = warp_sum(px); py = warp_sum(py); pz = warp_sum(pz);
  if (lane == 0) {
    if (cphiD) {
      fx += ec.aewald3 * ud[i] - cphiD[1 * n + i];
      fy += ec.aewald3 * ud[n + i] - cphiD[2 * n + i];
      fz += ec.aewald3 * ud[2 * n + i] - cphiD[3 * n + i];
      px += ec.aewald3 * up[i] - cphiP[1 * n + i];
      py += ec.aewald3 * up[n + i] - cphiP[2 * n + i];
      pz += ec.aewald3 * up[2 * n + i] - cphiP[3 * n + i];
    }
    outD[i] = fx; outD[n + i] = fy; outD[2 * n + i] = fz;
    outP[i] = px; outP[n + i] = py; outP[2 * n + i] = pz;
  }
}

// ---------------------------------------------------------------------------
// Permanent and polarization real-space energy, i-side force and torque.
__global__ void __launch_bounds__(128) k_real_energy(
    int n, const double *__restrict__ x, const double *__restrict__ y, const double *__restrict__ z, Box bx,
    const double *__restrict__ gm, const double *__restrict__ uD, const double *__restrict__ uP,
    const double *__restrict__ ipdamp, const double *__restrict__ thole, const int *__restrict__ ewl,
    const int *__restrict__ ewl_cnt, int capE, Excl ex, EwaldCoef ec, ScaleTables c_scales, int polarization, int gradient,
    double *eatom_perm, double *eatom_pol, long long *catom, double *grad, double *torque) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int i = warp;
  const double xi = x[i], yi = y[i], zi = z[i];
  const double ci = gm[t000 * n + i], dix = gm[t100 * n + i], diy = gm[t010 * n + i], diz = gm[t001 * n + i];
  const double qixx = gm[t200 * n + i] * (1.0 / 3.0), qiyy = gm[t020 * n + i] * (1.0 / 3.0);
  const double qizz = gm[t002 * n + i] * (1.0 / 3.0), qixy = gm[t110 * n + i] * (1.0 / 3.0);
  const double qixz = gm[t101 * n + i] * (1.0 / 3.0), qiyz = gm[t011 * n + i] * (1.0 / 3.0);
  const double uix = uD[i], uiy = uD[n + i], uiz = uD[2 * n + i];
  const double pix = uP[i], piy = uP[n + i], piz = uP[2 * n + i];
  const double pdi = ipdamp[i], pti = thole[i];
  const bool doPol = polarization != FFXG_POLAR_NONE;
  double eP = 0, eI = 0;
  long long cnt_pairs = 0;
  double gx = 0, gy = 0, gz = 0, tx = 0, ty = 0, tz = 0;
  const int cnt = min(ewl_cnt[i], capE);
  const int *row = ewl + (size_t)i * capE;
  for (int a = lane; a < cnt; a += 32) {
    const int k = row[a];
    double xr = __dsub_rn(x[k], xi), yr = __dsub_rn(y[k], yi), zr = __dsub_rn(z[k], zi);
    const double r2 = image_exact(xr, yr, zr, bx);
    const double ck = gm[t000 * n + k], dkx = gm[t100 * n + k], dky = gm[t010 * n + k], dkz = gm[t001 * n + k];
    const double qkxx = gm[t200 * n + k] * (1.0 / 3.0), qkyy = gm[t020 * n + k] * (1.0 / 3.0);
    const double qkzz = gm[t002 * n + k] * (1.0 / 3.0), qkxy = gm[t110 * n + k] * (1.0 / 3.0);
    const double qkxz = gm[t101 * n + k] * (1.0 / 3.0), qkyz = gm[t011 * n + k] * (1.0 / 3.0);
    const double ukx = uD[k], uky = uD[n + k], ukz = uD[2 * n + k];
    const double pkx = uP[k], pky = uP[n + k], pkz = uP[2 * n + k];
    const unsigned code = excl_code(i, k, ex.ptr, ex.k, ex.code, ex.lo, ex.hi);
    const double scale = c_scales.m[code & 7u];
    const double scalep = c_scales.p[(code >> 3) & 7u];
    const double scaled = c_scales.d[(code >> 6) & 1u];
    const double r = sqrt(r2);
    const double ralpha = ec.aewald * r;
    const double exp2a = exp(-ralpha * ralpha);
    const double rr1 = 1.0 / r, rr2 = rr1 * rr1;
    const double bn0 = erfc(ralpha) * rr1;
    const double bn1 = (bn0 + ec.an0 * exp2a) * rr2;
    const double bn2 = (3.0 * bn1 + ec.an1 * exp2a) * rr2;
    const double bn3 = (5.0 * bn2 + ec.an2 * exp2a) * rr2;
    const double bn4 = (7.0 * bn3 + ec.an3 * exp2a) * rr2;
    const double bn5 = (9.0 * bn4 + ec.an4 * exp2a) * rr2;
    const double rr3 = rr1 * rr2, rr5 = 3.0 * rr3 * rr2, rr7 = 5.0 * rr5 * rr2;
    const double rr9 = 7.0 * rr7 * rr2, rr11 = 9.0 * rr9 * rr2;
    double scale3 = 1.0, scale5 = 1.0, scale7 = 1.0;
    double ddsc3x = 0, ddsc3y = 0, ddsc3z = 0, ddsc5x = 0, ddsc5y = 0, ddsc5z = 0, ddsc7x = 0, ddsc7y = 0, ddsc7z = 0;
    double damp = pdi * ipdamp[k];
    const double tho = fmin(pti, thole[k]);
    const double rdamp = r * damp;
    damp = -tho * rdamp * rdamp * rdamp;
    if (damp > -50.0) {
      const double expdamp = exp(damp);
      scale3 = 1.0 - expdamp;
      scale5 = 1.0 - expdamp * (1.0 - damp);
      scale7 = 1.0 - expdamp * (1.0 - damp + 0.6 * damp * damp);
      const double temp3 = -3.0 * damp * expdamp * rr2;
      const double temp5 = -damp;
      const double temp7 = -0.2 - 0.6 * damp;
      ddsc3x = temp3 * xr; ddsc3y = temp3 * yr; ddsc3z = temp3 * zr;
      ddsc5x = temp5 * ddsc3x; ddsc5y = temp5 * ddsc3y; ddsc5z = temp5 * ddsc3z;
      ddsc7x = temp7 * ddsc5x; ddsc7y = temp7 * ddsc5y; ddsc7z = temp7 * ddsc5z;
    }
    // ---- permanentPair
    {
      const double dixdkx = diy * dkz - diz * dky, dixdky = diz * dkx - dix * dkz, dixdkz = dix * dky - diy * dkx;
      const double dixrx = diy * zr - diz * yr, dixry = diz * xr - dix * zr, dixrz = dix * yr - diy * xr;
      const double dkxrx = dky * zr - dkz * yr, dkxry = dkz * xr - dkx * zr, dkxrz = dkx * yr - dky * xr;
      const double qirx = qixx * xr + qixy * yr + qixz * zr;
      const double qiry = qixy * xr + qiyy * yr + qiyz * zr;
      const double qirz = qixz * xr + qiyz * yr + qizz * zr;
      const double qkrx = qkxx * xr + qkxy * yr + qkxz * zr;
      const double qkry = qkxy * xr + qkyy * yr + qkyz * zr;
      const double qkrz = qkxz * xr + qkyz * yr + qkzz * zr;
      const double qiqkrx = qixx * qkrx + qixy * qkry + qixz * qkrz;
      const double qiqkry = qixy * qkrx + qiyy * qkry + qiyz * qkrz;
      const double qiqkrz = qixz * qkrx + qiyz * qkry + qizz * qkrz;
      const double qkqirx = qkxx * qirx + qkxy * qiry + qkxz * qirz;
      const double qkqiry = qkxy * qirx + qkyy * qiry + qkyz * qirz;
      const double qkqirz = qkxz * qirx + qkyz * qiry + qkzz * qirz;
      const double qixqkx = qixy * qkxz + qiyy * qkyz + qiyz * qkzz - qixz * qkxy - qiyz * qkyy - qizz * qkyz;
      const double qixqky = qixz * qkxx + qiyz * qkxy + qizz * qkxz - qixx * qkxz - qixy * qkyz - qixz * qkzz;
      const double qixqkz = qixx * qkxy + qixy * qkyy + qixz * qkyz - qixy * qkxx - qiyy * qkxy - qiyz * qkxz;
      const double rxqirx = yr * qirz - zr * qiry, rxqiry = zr * qirx - xr * qirz, rxqirz = xr * qiry - yr * qirx;
      const double rxqkrx = yr * qkrz - zr * qkry, rxqkry = zr * qkrx - xr * qkrz, rxqkrz = xr * qkry - yr * qkrx;
      const double rxqikrx = yr * qiqkrz - zr * qiqkry, rxqikry = zr * qiqkrx - xr * qiqkrz, rxqikrz = xr * qiqkry - yr * qiqkrx;
      const double rxqkirx = yr * qkqirz - zr * qkqiry, rxqkiry = zr * qkqirx - xr * qkqirz, rxqkirz = xr * qkqiry - yr * qkqirx;
      const double qkrxqirx = qkry * qirz - qkrz * qiry, qkrxqiry = qkrz * qirx - qkrx * qirz, qkrxqirz = qkrx * qiry - qkry * qirx;
      const double qidkx = qixx * dkx + qixy * dky + qixz * dkz;
      const double qidky = qixy * dkx + qiyy * dky + qiyz * dkz;
      const double qidkz = qixz * dkx + qiyz * dky + qizz * dkz;
      const double qkdix = qkxx * dix + qkxy * diy + qkxz * diz;
      const double qkdiy = qkxy * dix + qkyy * diy + qkyz * diz;
      const double qkdiz = qkxz * dix + qkyz * diy + qkzz * diz;
      const double dixqkrx = diy * qkrz - diz * qkry, dixqkry = diz * qkrx - dix * qkrz, dixqkrz = dix * qkry - diy * qkrx;
      const double dkxqirx = dky * qirz - dkz * qiry, dkxqiry = dkz * qirx - dkx * qirz, dkxqirz = dkx * qiry - dky * qirx;
      const double rxqidkx = yr * qidkz - zr * qidky, rxqidky = zr * qidkx - xr * qidkz, rxqidkz = xr * qidky - yr * qidkx;
      const double rxqkdix = yr * qkdiz - zr * qkdiy, rxqkdiy = zr * qkdix - xr * qkdiz, rxqkdiz = xr * qkdiy - yr * qkdix;
      const double sc2 = dix * dkx + diy * dky + diz * dkz;
      const double sc3 = dix * xr + diy * yr + diz * zr;
      const double sc4 = dkx * xr + dky * yr + dkz * zr;
      const double sc5 = qirx * xr + qiry * yr + qirz * zr;
      const double sc6 = qkrx * xr + qkry * yr + qkrz * zr;
      const double sc7 = qirx * dkx + qiry * dky + qirz * dkz;
      const double sc8 = qkrx * dix + qkry * diy + qkrz * diz;
      const double sc9 = qirx * qkrx + qiry * qkry + qirz * qkrz;
      const double sc10 = 2.0 * (qixy * qkxy + qixz * qkxz + qiyz * qkyz) + qixx * qkxx + qiyy * qkyy + qizz * qkzz;
      const double gl0 = ci * ck, gl1 = ck * sc3 - ci * sc4, gl2 = ci * sc6 + ck * sc5 - sc3 * sc4;
      const double gl3 = sc3 * sc6 - sc4 * sc5, gl4 = sc5 * sc6, gl5 = -4.0 * sc9, gl6 = sc2;
      const double gl7 = 2.0 * (sc7 - sc8), gl8 = 2.0 * sc10;
      const double scale1 = 1.0 - scale;
      const double ereal = gl0 * bn0 + (gl1 + gl6) * bn1 + (gl2 + gl7 + gl8) * bn2 + (gl3 + gl5) * bn3 + gl4 * bn4;
      const double efix = scale1 * (gl0 * rr1 + (gl1 + gl6) * rr3 + (gl2 + gl7 + gl8) * rr5 + (gl3 + gl5) * rr7 + gl4 * rr9);
      const double e = ereal - efix;
      if (e != 0.0) { eP += 0.5 * e; if (k > i) cnt_pairs++; }
      if (gradient) {
        const double gf1 = bn1 * gl0 + bn2 * (gl1 + gl6) + bn3 * (gl2 + gl7 + gl8) + bn4 * (gl3 + gl5) + bn5 * gl4;
        const double gf2 = -ck * bn1 + sc4 * bn2 - sc6 * bn3;
        const double gf3 = ci * bn1 + sc3 * bn2 + sc5 * bn3;
        const double gf4 = 2.0 * bn2;
        const double gf5 = 2.0 * (-ck * bn2 + sc4 * bn3 - sc6 * bn4);
        const double gf6 = 2.0 * (-ci * bn2 - sc3 * bn3 - sc5 * bn4);
        const double gf7 = 4.0 * bn3;
        double ftm2x = gf1 * xr + gf2 * dix + gf3 * dkx + gf4 * (qkdix - qidkx) + gf5 * qirx + gf6 * qkrx + gf7 * (qiqkrx + qkqirx);
        double ftm2y = gf1 * yr + gf2 * diy + gf3 * dky + gf4 * (qkdiy - qidky) + gf5 * qiry + gf6 * qkry + gf7 * (qiqkry + qkqiry);
        double ftm2z = gf1 * zr + gf2 * diz + gf3 * dkz + gf4 * (qkdiz - qidkz) + gf5 * qirz + gf6 * qkrz + gf7 * (qiqkrz + qkqirz);
        double ttm2x = -bn1 * dixdkx + gf2 * dixrx + gf4 * (dixqkrx + dkxqirx + rxqidkx - 2.0 * qixqkx) - gf5 * rxqirx - gf7 * (rxqikrx + qkrxqirx);
        double ttm2y = -bn1 * dixdky + gf2 * dixry + gf4 * (dixqkry + dkxqiry + rxqidky - 2.0 * qixqky) - gf5 * rxqiry - gf7 * (rxqikry + qkrxqiry);
        double ttm2z = -bn1 * dixdkz + gf2 * dixrz + gf4 * (dixqkrz + dkxqirz + rxqidkz - 2.0 * qixqkz) - gf5 * rxqirz - gf7 * (rxqikrz + qkrxqirz);
        double ttm3x = bn1 * dixdkx + gf3 * dkxrx - gf4 * (dixqkrx + dkxqirx + rxqkdix - 2.0 * qixqkx) - gf6 * rxqkrx - gf7 * (rxqkirx - qkrxqirx);
        double ttm3y = bn1 * dixdky + gf3 * dkxry - gf4 * (dixqkry + dkxqiry + rxqkdiy - 2.0 * qixqky) - gf6 * rxqkry - gf7 * (rxqkiry - qkrxqiry);
        double ttm3z = bn1 * dixdkz + gf3 * dkxrz - gf4 * (dixqkrz + dkxqirz + rxqkdiz - 2.0 * qixqkz) - gf6 * rxqkrz - gf7 * (rxqkirz - qkrxqirz);
        if (scale1 != 0.0) {
          const double gfr1 = rr3 * gl0 + rr5 * (gl1 + gl6) + rr7 * (gl2 + gl7 + gl8) + rr9 * (gl3 + gl5) + rr11 * gl4;
          const double gfr2 = -ck * rr3 + sc4 * rr5 - sc6 * rr7;
          const double gfr3 = ci * rr3 + sc3 * rr5 + sc5 * rr7;
          const double gfr4 = 2.0 * rr5;
          const double gfr5 = 2.0 * (-ck * rr5 + sc4 * rr7 - sc6 * rr9);
          const double gfr6 = 2.0 * (-ci * rr5 - sc3 * rr7 - sc5 * rr9);
          const double gfr7 = 4.0 * rr7;
          const double ftm2rx = gfr1 * xr + gfr2 * dix + gfr3 * dkx + gfr4 * (qkdix - qidkx) + gfr5 * qirx + gfr6 * qkrx + gfr7 * (qiqkrx + qkqirx);
          const double ftm2ry = gfr1 * yr + gfr2 * diy + gfr3 * dky + gfr4 * (qkdiy - qidky) + gfr5 * qiry + gfr6 * qkry + gfr7 * (qiqkry + qkqiry);
          const double ftm2rz = gfr1 * zr + gfr2 * diz + gfr3 * dkz + gfr4 * (qkdiz - qidkz) + gfr5 * qirz + gfr6 * qkrz + gfr7 * (qiqkrz + qkqirz);
          const double ttm2rx = -rr3 * dixdkx + gfr2 * dixrx + gfr4 * (dixqkrx + dkxqirx + rxqidkx - 2.0 * qixqkx) - gfr5 * rxqirx - gfr7 * (rxqikrx + qkrxqirx);
          const double ttm2ry = -rr3 * dixdky + gfr2 * dixry + gfr4 * (dixqkry + dkxqiry + rxqidky - 2.0 * qixqky) - gfr5 * rxqiry - gfr7 * (rxqikry + qkrxqiry);
          const double ttm2rz = -rr3 * dixdkz + gfr2 * dixrz + gfr4 * (dixqkrz + dkxqirz + rxqidkz - 2.0 * qixqkz) - gfr5 * rxqirz - gfr7 * (rxqikrz + qkrxqirz);
          const double ttm3rx = rr3 * dixdkx + gfr3 * dkxrx - gfr4 * (dixqkrx + dkxqirx + rxqkdix - 2.0 * qixqkx) - gfr6 * rxqkrx - gfr7 * (rxqkirx - qkrxqirx);
          const double ttm3ry = rr3 * dixdky + gfr3 * dkxry - gfr4 * (dixqkry + dkxqiry + rxqkdiy - 2.0 * qixqky) - gfr6 * rxqkry - gfr7 * (rxqkiry - qkrxqiry);
          const double ttm3rz = rr3 * dixdkz + gfr3 * dkxrz - gfr4 * (dixqkrz + dkxqirz + rxqkdiz - 2.0 * qixqkz) - gfr6 * rxqkrz - gfr7 * (rxqkirz - qkrxqirz);
          ftm2x -= scale1 * ftm2rx; ftm2y -= scale1 * ftm2ry; ftm2z -= scale1 * ftm2rz;
          ttm2x -= scale1 * ttm2rx; ttm2y -= scale1 * ttm2ry; ttm2z -= scale1 * ttm2rz;
          ttm3x -= scale1 * ttm3rx; ttm3y -= scale1 * ttm3ry; ttm3z -= scale1 * ttm3rz;
        }
        const double pre = ec.electric;
        gx += pre * ftm2x; gy += pre * ftm2y; gz += pre * ftm2z;
        tx += pre * ttm2x; ty += pre * ttm2y; tz += pre * ttm2z;
      }
    }
    if (!doPol) continue;
    // ---- polarizationPair
    {
      const double dsc3 = 1.0 - scale3 * scaled, dsc5 = 1.0 - scale5 * scaled, dsc7 = 1.0 - scale7 * scaled;
      const double psc3 = 1.0 - scale3 * scalep, psc5 = 1.0 - scale5 * scalep, psc7 = 1.0 - scale7 * scalep;
      const double usc3 = 1.0 - scale3, usc5 = 1.0 - scale5;
      const double dixukx = diy * ukz - diz * uky, dixuky = diz * ukx - dix * ukz, dixukz = dix * uky - diy * ukx;
      const double dkxuix = dky * uiz - dkz * uiy, dkxuiy = dkz * uix - dkx * uiz, dkxuiz = dkx * uiy - dky * uix;
      const double dixukpx = diy * pkz - diz * pky, dixukpy = diz * pkx - dix * pkz, dixukpz = dix * pky - diy * pkx;
      const double dkxuipx = dky * piz - dkz * piy, dkxuipy = dkz * pix - dkx * piz, dkxuipz = dkx * piy - dky * pix;
      const double dixrx = diy * zr - diz * yr, dixry = diz * xr - dix * zr, dixrz = dix * yr - diy * xr;
      const double dkxrx = dky * zr - dkz * yr, dkxry = dkz * xr - dkx * zr, dkxrz = dkx * yr - dky * xr;
      const double qirx = qixx * xr + qixy * yr + qixz * zr;
      const double qiry = qixy * xr + qiyy * yr + qiyz * zr;
      const double qirz = qixz * xr + qiyz * yr + qizz * zr;
      const double qkrx = qkxx * xr + qkxy * yr + qkxz * zr;
      const double qkry = qkxy * xr + qkyy * yr + qkyz * zr;
      const double qkrz = qkxz * xr + qkyz * yr + qkzz * zr;
      const double rxqirx = yr * qirz - zr * qiry, rxqiry = zr * qirx - xr * qirz, rxqirz = xr * qiry - yr * qirx;
      const double rxqkrx = yr * qkrz - zr * qkry, rxqkry = zr * qkrx - xr * qkrz, rxqkrz = xr * qkry - yr * qkrx;
      const double qiukx = qixx * ukx + qixy * uky + qixz * ukz;
      const double qiuky = qixy * ukx + qiyy * uky + qiyz * ukz;
      const double qiukz = qixz * ukx + qiyz * uky + qizz * ukz;
      const double qkuix = qkxx * uix + qkxy * uiy + qkxz * uiz;
      const double qkuiy = qkxy * uix + qkyy * uiy + qkyz * uiz;
      const double qkuiz = qkxz * uix + qkyz * uiy + qkzz * uiz;
      const double qiukpx = qixx * pkx + qixy * pky + qixz * pkz;
      const double qiukpy = qixy * pkx + qiyy * pky + qiyz * pkz;
      const double qiukpz = qixz * pkx + qiyz * pky + qizz * pkz;
      const double qkuipx = qkxx * pix + qkxy * piy + qkxz * piz;
      const double qkuipy = qkxy * pix + qkyy * piy + qkyz * piz;
      const double qkuipz = qkxz * pix + qkyz * piy + qkzz * piz;
      const double uixqkrx = uiy * qkrz - uiz * qkry, uixqkry = uiz * qkrx - uix * qkrz, uixqkrz = uix * qkry - uiy * qkrx;
      const double ukxqirx = uky * qirz - ukz * qiry, ukxqiry = ukz * qirx - ukx * qirz, ukxqirz = ukx * qiry - uky * qirx;
      const double uixqkrpx = piy * qkrz - piz * qkry, uixqkrpy = piz * qkrx - pix * qkrz, uixqkrpz = pix * qkry - piy * qkrx;
      const double ukxqirpx = pky * qirz - pkz * qiry, ukxqirpy = pkz * qirx - pkx * qirz, ukxqirpz = pkx * qiry - pky * qirx;
      const double rxqiukx = yr * qiukz - zr * qiuky, rxqiuky = zr * qiukx - xr * qiukz, rxqiukz = xr * qiuky - yr * qiukx;
      const double rxqkuix = yr * qkuiz - zr * qkuiy, rxqkuiy = zr * qkuix - xr * qkuiz, rxqkuiz = xr * qkuiy - yr * qkuix;
      const double rxqiukpx = yr * qiukpz - zr * qiukpy, rxqiukpy = zr * qiukpx - xr * qiukpz, rxqiukpz = xr * qiukpy - yr * qiukpx;
      const double rxqkuipx = yr * qkuipz - zr * qkuipy, rxqkuipy = zr * qkuipx - xr * qkuipz, rxqkuipz = xr * qkuipy - yr * qkuipx;
      const double sc3 = dix * xr + diy * yr + diz * zr;
      const double sc4 = dkx * xr + dky * yr + dkz * zr;
      const double sc5 = qirx * xr + qiry * yr + qirz * zr;
      const double sc6 = qkrx * xr + qkry * yr + qkrz * zr;
      const double sci1 = uix * dkx + uiy * dky + uiz * dkz + dix * ukx + diy * uky + diz * ukz;
      const double sci3 = uix * xr + uiy * yr + uiz * zr;
      const double sci4 = ukx * xr + uky * yr + ukz * zr;
      const double sci7 = qirx * ukx + qiry * uky + qirz * ukz;
      const double sci8 = qkrx * uix + qkry * uiy + qkrz * uiz;
      const double scip1 = pix * dkx + piy * dky + piz * dkz + dix * pkx + diy * pky + diz * pkz;
      const double scip2 = uix * pkx + uiy * pky + uiz * pkz + pix * ukx + piy * uky + piz * ukz;
      const double scip3 = pix * xr + piy * yr + piz * zr;
      const double scip4 = pkx * xr + pky * yr + pkz * zr;
      const double scip7 = qirx * pkx + qiry * pky + qirz * pkz;
      const double scip8 = qkrx * pix + qkry * piy + qkrz * piz;
      const double gli1 = ck * sci3 - ci * sci4, gli2 = -sc3 * sci4 - sci3 * sc4, gli3 = sci3 * sc6 - sci4 * sc5;
      const double gli6 = sci1, gli7 = 2.0 * (sci7 - sci8);
      const double glip1 = ck * scip3 - ci * scip4, glip2 = -sc3 * scip4 - scip3 * sc4, glip3 = scip3 * sc6 - scip4 * sc5;
      const double glip6 = scip1, glip7 = 2.0 * (scip7 - scip8);
      const double ereal = (gli1 + gli6) * bn1 + (gli2 + gli7) * bn2 + gli3 * bn3;
      const double efix = (gli1 + gli6) * rr3 * psc3 + (gli2 + gli7) * rr5 * psc5 + gli3 * rr7 * psc7;
      eI += 0.25 * (ereal - efix);
      if (!gradient) continue;
      const bool dorli = (psc3 != 0.0 || dsc3 != 0.0 || usc3 != 0.0);
      const double gfi1 = 0.5 * bn2 * (gli1 + glip1 + gli6 + glip6) + 0.5 * bn2 * scip2 +
                          0.5 * bn3 * (gli2 + glip2 + gli7 + glip7) - 0.5 * bn3 * (sci3 * scip4 + scip3 * sci4) +
                          0.5 * bn4 * (gli3 + glip3);
      const double gfi2 = -ck * bn1 + sc4 * bn2 - sc6 * bn3;
      const double gfi3 = ci * bn1 + sc3 * bn2 + sc5 * bn3;
      const double gfi4 = 2.0 * bn2;
      const double gfi5 = bn3 * (sci4 + scip4);
      const double gfi6 = -bn3 * (sci3 + scip3);
      double ftm2ix = gfi1 * xr + 0.5 * (gfi2 * (uix + pix) + bn2 * (sci4 * pix + scip4 * uix) + gfi3 * (ukx + pkx) +
                                         bn2 * (sci3 * pkx + scip3 * ukx) + (sci4 + scip4) * bn2 * dix +
                                         (sci3 + scip3) * bn2 * dkx + gfi4 * (qkuix + qkuipx - qiukx - qiukpx)) +
                      gfi5 * qirx + gfi6 * qkrx;
      double ftm2iy = gfi1 * yr + 0.5 * (gfi2 * (uiy + piy) + bn2 * (sci4 * piy + scip4 * uiy) + gfi3 * (uky + pky) +
                                         bn2 * (sci3 * pky + scip3 * uky) + (sci4 + scip4) * bn2 * diy +
                                         (sci3 + scip3) * bn2 * dky + gfi4 * (qkuiy + qkuipy - qiuky - qiukpy)) +
                      gfi5 * qiry + gfi6 * qkry;
      double ftm2iz = gfi1 * zr + 0.5 * (gfi2 * (uiz + piz) + bn2 * (sci4 * piz + scip4 * uiz) + gfi3 * (ukz + pkz) +
                                         bn2 * (sci3 * pkz + scip3 * ukz) + (sci4 + scip4) * bn2 * diz +
                                         (sci3 + scip3) * bn2 * dkz + gfi4 * (qkuiz + qkuipz - qiukz - qiukpz)) +
                      gfi5 * qirz + gfi6 * qkrz;
      const double gti2 = 0.5 * bn2 * (sci4 + scip4), gti3 = 0.5 * bn2 * (sci3 + scip3);
      const double gti4 = gfi4, gti5 = gfi5, gti6 = gfi6;
      double ttm2ix = -0.5 * bn1 * (dixukx + dixukpx) + gti2 * dixrx - gti5 * rxqirx + 0.5 * gti4 * (ukxqirx + rxqiukx + ukxqirpx + rxqiukpx);
      double ttm2iy = -0.5 * bn1 * (dixuky + dixukpy) + gti2 * dixry - gti5 * rxqiry + 0.5 * gti4 * (ukxqiry + rxqiuky + ukxqirpy + rxqiukpy);
      double ttm2iz = -0.5 * bn1 * (dixukz + dixukpz) + gti2 * dixrz - gti5 * rxqirz + 0.5 * gti4 * (ukxqirz + rxqiukz + ukxqirpz + rxqiukpz);
      double ttm3ix = -0.5 * bn1 * (dkxuix + dkxuipx) + gti3 * dkxrx - gti6 * rxqkrx - 0.5 * gti4 * (uixqkrx + rxqkuix + uixqkrpx + rxqkuipx);
      double ttm3iy = -0.5 * bn1 * (dkxuiy + dkxuipy) + gti3 * dkxry - gti6 * rxqkry - 0.5 * gti4 * (uixqkry + rxqkuiy + uixqkrpy + rxqkuipy);
      double ttm3iz = -0.5 * bn1 * (dkxuiz + dkxuipz) + gti3 * dkxrz - gti6 * rxqkrz - 0.5 * gti4 * (uixqkrz + rxqkuiz + uixqkrpz + rxqkuipz);
      double ftm2rix = 0, ftm2riy = 0, ftm2riz = 0, ttm2rix = 0, ttm2riy = 0, ttm2riz = 0, ttm3rix = 0, ttm3riy = 0, ttm3riz = 0;
      if (dorli) {
        const double gfri1 = 0.5 * rr5 * ((gli1 + gli6) * psc3 + (glip1 + glip6) * dsc3 + scip2 * usc3) +
                             0.5 * rr7 * ((gli7 + gli2) * psc5 + (glip7 + glip2) * dsc5 - (sci3 * scip4 + scip3 * sci4) * usc5) +
                             0.5 * rr9 * (gli3 * psc7 + glip3 * dsc7);
        const double gfri4 = 2.0 * rr5;
        const double gfri5 = rr7 * (sci4 * psc7 + scip4 * dsc7);
        const double gfri6 = -rr7 * (sci3 * psc7 + scip3 * dsc7);
        ftm2rix = gfri1 * xr + 0.5 * (-rr3 * ck * (uix * psc3 + pix * dsc3) + rr5 * sc4 * (uix * psc5 + pix * dsc5) - rr7 * sc6 * (uix * psc7 + pix * dsc7)) +
                  (rr3 * ci * (ukx * psc3 + pkx * dsc3) + rr5 * sc3 * (ukx * psc5 + pkx * dsc5) + rr7 * sc5 * (ukx * psc7 + pkx * dsc7)) * 0.5 +
                  rr5 * usc5 * (sci4 * pix + scip4 * uix + sci3 * pkx + scip3 * ukx) * 0.5 +
                  0.5 * (sci4 * psc5 + scip4 * dsc5) * rr5 * dix + 0.5 * (sci3 * psc5 + scip3 * dsc5) * rr5 * dkx +
                  0.5 * gfri4 * ((qkuix - qiukx) * psc5 + (qkuipx - qiukpx) * dsc5) + gfri5 * qirx + gfri6 * qkrx;
        ftm2riy = gfri1 * yr + 0.5 * (-rr3 * ck * (uiy * psc3 + piy * dsc3) + rr5 * sc4 * (uiy * psc5 + piy * dsc5) - rr7 * sc6 * (uiy * psc7 + piy * dsc7)) +
                  (rr3 * ci * (uky * psc3 + pky * dsc3) + rr5 * sc3 * (uky * psc5 + pky * dsc5) + rr7 * sc5 * (uky * psc7 + pky * dsc7)) * 0.5 +
                  rr5 * usc5 * (sci4 * piy + scip4 * uiy + sci3 * pky + scip3 * uky) * 0.5 +
                  0.5 * (sci4 * psc5 + scip4 * dsc5) * rr5 * diy + 0.5 * (sci3 * psc5 + scip3 * dsc5) * rr5 * dky +
                  0.5 * gfri4 * ((qkuiy - qiuky) * psc5 + (qkuipy - qiukpy) * dsc5) + gfri5 * qiry + gfri6 * qkry;
        ftm2riz = gfri1 * zr + 0.5 * (-rr3 * ck * (uiz * psc3 + piz * dsc3) + rr5 * sc4 * (uiz * psc5 + piz * dsc5) - rr7 * sc6 * (uiz * psc7 + piz * dsc7)) +
                  (rr3 * ci * (ukz * psc3 + pkz * dsc3) + rr5 * sc3 * (ukz * psc5 + pkz * dsc5) + rr7 * sc5 * (ukz * psc7 + pkz * dsc7)) * 0.5 +
                  rr5 * usc5 * (sci4 * piz + scip4 * uiz + sci3 * pkz + scip3 * ukz) * 0.5 +
                  0.5 * (sci4 * psc5 + scip4 * dsc5) * rr5 * diz + 0.5 * (sci3 * psc5 + scip3 * dsc5) * rr5 * dkz +
                  0.5 * gfri4 * ((qkuiz - qiukz) * psc5 + (qkuipz - qiukpz) * dsc5) + gfri5 * qirz + gfri6 * qkrz;
        const double gtri2 = 0.5 * rr5 * (sci4 * psc5 + scip4 * dsc5);
        const double gtri3 = 0.5 * rr5 * (sci3 * psc5 + scip3 * dsc5);
        const double gtri4 = gfri4, gtri5 = gfri5, gtri6 = gfri6;
        ttm2rix = -rr3 * (dixukx * psc3 + dixukpx * dsc3) * 0.5 + gtri2 * dixrx - gtri5 * rxqirx + gtri4 * ((ukxqirx + rxqiukx) * psc5 + (ukxqirpx + rxqiukpx) * dsc5) * 0.5;
        ttm2riy = -rr3 * (dixuky * psc3 + dixukpy * dsc3) * 0.5 + gtri2 * dixry - gtri5 * rxqiry + gtri4 * ((ukxqiry + rxqiuky) * psc5 + (ukxqirpy + rxqiukpy) * dsc5) * 0.5;
        ttm2riz = -rr3 * (dixukz * psc3 + dixukpz * dsc3) * 0.5 + gtri2 * dixrz - gtri5 * rxqirz + gtri4 * ((ukxqirz + rxqiukz) * psc5 + (ukxqirpz + rxqiukpz) * dsc5) * 0.5;
        ttm3rix = -rr3 * (dkxuix * psc3 + dkxuipx * dsc3) * 0.5 + gtri3 * dkxrx - gtri6 * rxqkrx - gtri4 * ((uixqkrx + rxqkuix) * psc5 + (uixqkrpx + rxqkuipx) * dsc5) * 0.5;
        ttm3riy = -rr3 * (dkxuiy * psc3 + dkxuipy * dsc3) * 0.5 + gtri3 * dkxry - gtri6 * rxqkry - gtri4 * ((uixqkry + rxqkuiy) * psc5 + (uixqkrpy + rxqkuipy) * dsc5) * 0.5;
        ttm3riz = -rr3 * (dkxuiz * psc3 + dkxuipz * dsc3) * 0.5 + gtri3 * dkxrz - gtri6 * rxqkrz - gtri4 * ((uixqkrz + rxqkuiz) * psc5 + (uixqkrpz + rxqkuipz) * dsc5) * 0.5;
      }
      double temp3 = 0.5 * rr3 * ((gli1 + gli6) * scalep + (glip1 + glip6) * scaled);
      double temp5 = 0.5 * rr5 * ((gli2 + gli7) * scalep + (glip2 + glip7) * scaled);
      const double temp7 = 0.5 * rr7 * (gli3 * scalep + glip3 * scaled);
      const double fridmpx = temp3 * ddsc3x + temp5 * ddsc5x + temp7 * ddsc7x;
      const double fridmpy = temp3 * ddsc3y + temp5 * ddsc5y + temp7 * ddsc7y;
      const double fridmpz = temp3 * ddsc3z + temp5 * ddsc5z + temp7 * ddsc7z;
      temp3 = 0.5 * rr3 * scip2;
      temp5 = -0.5 * rr5 * (sci3 * scip4 + scip3 * sci4);
      const double findmpx = temp3 * ddsc3x + temp5 * ddsc5x;
      const double findmpy = temp3 * ddsc3y + temp5 * ddsc5y;
      const double findmpz = temp3 * ddsc3z + temp5 * ddsc5z;
      ftm2ix = ftm2ix - fridmpx - findmpx;
      ftm2iy = ftm2iy - fridmpy - findmpy;
      ftm2iz = ftm2iz - fridmpz - findmpz;
      if (polarization == FFXG_POLAR_DIRECT) {
        const double gfd = 0.5 * (bn2 * scip2 - bn3 * (scip3 * sci4 + sci3 * scip4));
        const double gfdr = 0.5 * (rr5 * scip2 * usc3 - rr7 * (scip3 * sci4 + sci3 * scip4) * usc5);
        ftm2ix = ftm2ix - gfd * xr - 0.5 * bn2 * (sci4 * pix + scip4 * uix + sci3 * pkx + scip3 * ukx);
        ftm2iy = ftm2iy - gfd * yr - 0.5 * bn2 * (sci4 * piy + scip4 * uiy + sci3 * pky + scip3 * uky);
        ftm2iz = ftm2iz - gfd * zr - 0.5 * bn2 * (sci4 * piz + scip4 * uiz + sci3 * pkz + scip3 * ukz);
        const double fdirx = gfdr * xr + 0.5 * usc5 * rr5 * (sci4 * pix + scip4 * uix + sci3 * pkx + scip3 * ukx);
        const double fdiry = gfdr * yr + 0.5 * usc5 * rr5 * (sci4 * piy + scip4 * uiy + sci3 * pky + scip3 * uky);
        const double fdirz = gfdr * zr + 0.5 * usc5 * rr5 * (sci4 * piz + scip4 * uiz + sci3 * pkz + scip3 * ukz);
        ftm2ix = ftm2ix + fdirx + findmpx;
        ftm2iy = ftm2iy + fdiry + findmpy;
        ftm2iz = ftm2iz + fdirz + findmpz;
      }
      ftm2ix -= ftm2rix; ftm2iy -= ftm2riy; ftm2iz -= ftm2riz;
      ttm2ix -= ttm2rix; ttm2iy -= ttm2riy; ttm2iz -= ttm2riz;
      ttm3ix -= ttm3rix; ttm3iy -= ttm3riy; ttm3iz -= ttm3riz;
      const double sc = ec.electric;
      gx += sc * ftm2ix; gy += sc * ftm2iy; gz += sc * ftm2iz;
      tx += sc * ttm2ix; ty += sc * ttm2iy; tz += sc * ttm2iz;
    }

  }
  eP = warp_sum(eP); eI = warp_sum(eI);
  gx = warp_sum(gx); gy = warp_sum(gy); gz = warp_sum(gz);
  tx = warp_sum(tx); ty = warp_sum(ty); tz = warp_sum(tz);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cnt_pairs += __shfl_xor_sync(0xffffffffu, cnt_pairs, o);
  if (lane == 0) {
    eatom_perm[i] = eP * ec.electric;
    eatom_pol[i] = eI * ec.electric;
    catom[i] = cnt_pairs;
    if (gradient) {
      grad[i] = gx; grad[n + i] = gy; grad[2 * n + i] = gz;
      torque[i] = tx; torque[n + i] = ty; torque[2 * n + i] = tz;
    }
  }
}

// ---------------------------------------------------------------------------
static EwaldCoef ewald_coef(const Handle &h, double aewald) {
  EwaldCoef c{};
  const double SQRT_PI = 1.7724538509055160273;
  c.aewald = aewald;
  c.electric = h.prm.electric;
  c.aewald3 = 4.0 / 3.0 * pow(aewald, 3.0) / SQRT_PI;
  if (aewald > 0.0) {
    const double alsq2 = 2.0 * aewald * aewald;
    const double piEwald = 1.0 / (SQRT_PI * aewald);
    c.an0 = alsq2 * piEwald; c.an1 = alsq2 * c.an0; c.an2 = alsq2 * c.an1;
    c.an3 = alsq2 * c.an2; c.an4 = alsq2 * c.an3; c.an5 = alsq2 * c.an4;
  }
  return c;
}

static Excl excl(const Handle &h) {
  Excl e;
  e.ptr = h.d_excl_ptr; e.k = h.d_excl_k; e.lo = h.d_excl_lo; e.hi = h.d_excl_hi; e.code = h.d_excl_code;
  return e;
}


void launch_realspace_field(Handle &h) {
  const double off2 = h.prm.ewald_cutoff * h.prm.ewald_cutoff;
  k_realspace_field<<<nblocks((int64_t)h.n * 32, 128), 128, 0, h.stream>>>(
      h.n, h.d_x, h.d_y, h.d_z, h.box, h.d_gm, h.d_ipdamp, h.d_thole, h.d_nbr, h.d_nbr_cnt, h.cap_nbr, off2,
      h.prm.precond_cutoff, h.d_ewl, h.d_ewl_cnt, h.cap_ewl, h.d_prl, h.d_prl_cnt, h.cap_prl, h.d_coefE, h.d_coefP,
      excl(h), ewald_coef(h, h.prm.ewald_alpha), h.scales, h.d_cphi, h.d_polar,
      h.prm.polarization != FFXG_POLAR_NONE ? 1 : 0, h.d_fieldD, h.d_fieldP, h.d_uD, h.d_uP, h.d_udirD, h.d_udirP,
      h.d_flags);
  FFX_LAUNCHED(h);
}

EwaldCoef ewald_coef_public(const Handle &h) { return ewald_coef(h, h.prm.ewald_alpha); }

void launch_permanent_field(Handle &h) {
  k_permanent_field<<<nblocks((int64_t)h.n * 32, 128), 128, 0, h.stream>>>(
      h.n, h.d_x, h.d_y, h.d_z, h.box, h.d_gm, h.d_ipdamp, h.d_thole, h.d_ewl, h.d_ewl_cnt, h.cap_ewl, excl(h),
      ewald_coef(h, h.prm.ewald_alpha), h.scales, h.d_fieldD, h.d_fieldP);
  FFX_LAUNCHED(h);
}

void launch_direct(Handle &h) {
  const EwaldCoef ec = ewald_coef(h, h.prm.ewald_alpha);
  k_direct<<<nblocks(h.n, 256), 256, 0, h.stream>>>(h.n, h.d_gm, h.d_cphi, h.d_polar, ec.aewald3, h.d_fieldD,
                                                     h.d_fieldP, h.d_uD, h.d_uP, h.d_udirD, h.d_udirP);
  FFX_LAUNCHED(h);
}

void launch_induced_recip(Handle &h, const double *ud, const double *up) {
  // Spread both sets (Re = D, Im = CR), convolve, interpolate the field terms.
  launch_spread_induced(h, ud, up);
  launch_fft_convolution(h);
  launch_phi_induced(h, false);
}

void launch_induced_real(Handle &h, const double *ud, const double *up, double *outD, double *outP) {
  k_dipole_field<true><<<nblocks((int64_t)h.n * 32, 128), 128, 0, h.stream>>>(
      h.n, h.d_x, h.d_y, h.d_z, h.box, h.d_ipdamp, h.d_thole, h.d_ewl, h.d_ewl_cnt, h.cap_ewl,
      ewald_coef(h, h.prm.ewald_alpha), ud, up, nullptr, h.d_cphiI, h.d_cphiP, outD, outP);
  FFX_LAUNCHED(h);
}

void launch_precond_field(Handle &h, const double *rD, const double *rP, double *outD, double *outP) {
  k_dipole_field<false><<<nblocks((int64_t)h.n * 32, 128), 128, 0, h.stream>>>(
      h.n, h.d_x, h.d_y, h.d_z, h.box, h.d_ipdamp, h.d_thole, h.d_prl, h.d_prl_cnt, h.cap_prl, ewald_coef(h, 0.0),
      rD, rP, h.d_polar, nullptr, nullptr, outD, outP);
  FFX_LAUNCHED(h);
}

void launch_real_energy(Handle &h, bool grad) {
  k_real_energy<<<nblocks((int64_t)h.n * 32, 128), 128, 0, h.stream>>>(
      h.n, h.d_x, h.d_y, h.d_z, h.box, h.d_gm, h.d_uD, h.d_uP, h.d_ipdamp, h.d_thole, h.d_ewl, h.d_ewl_cnt,
      h.cap_ewl, excl(h), ewald_coef(h, h.prm.ewald_alpha), h.scales, h.prm.polarization, grad ? 1 : 0,
      h.d_eatom + 1 * (size_t)h.n, h.d_eatom + 2 * (size_t)h.n, h.d_catom + (size_t)h.n, h.d_grad, h.d_torque);
  FFX_LAUNCHED(h);
}

}  // namespace ffx
