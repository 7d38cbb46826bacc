// real.cu -- real-space Ewald pair kernels (warp per atom, gather over the full list).
//
//  k_permanent_field   PermanentRealSpaceFieldLoop (pme/PermanentFieldRegion.java:595-815)
//  k_direct_dipoles    DirectLoop (pme/DirectRegion.java:170-243)
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
#include <cmath>

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


// Real-space lists, permanent real-space field and cached pair coefficients in one pass (PermanentRealSpaceFieldLoop, pme/PermanentFieldRegion.java:595-815, which also
// derives the Ewald and preconditioner lists; DirectLoop, pme/DirectRegion.java:170-243).
// Phase 1 compacts the buffered row into the Ewald row (r2 <= off2) and the
// preconditioner row (r < pcut).  Phase 2 walks the Ewald row: it accumulates the D and
// CR permanent fields and stores, per entry, the two symmetric coefficients of the
// unmasked Thole-damped dipole field, A = bn1 - (1 - s3) rr3 and B = bn2 - (1 - s5) rr5,
// so the field of any dipole set is -A u_k + B (u_k . r) r; entries inside the
// preconditioner cutoff also store the Ewald-free pair (pme/PCGSolver.java:1300-1331).
template <typename R>
__device__ __forceinline__ void k_realspace_field(
    VGrid vg, int const &n, const double *__restrict__ const &x, const double *__restrict__ const &y,
    const double *__restrict__ const &z, const Box &bx, const double *__restrict__ const &gm,
    const double *__restrict__ const &ipdamp, const double *__restrict__ const &thole,
    const int *__restrict__ const &nbr, const int *__restrict__ const &nbr_cnt, int const &cap,
    const int *__restrict__ const &nbr_sh, double const &off2, double const &pcut2, int * const &ewl,
    int * const &ewl_cnt, int const &capE, int * const &ewl_sh, int * const &prl, int * const &prl_cnt,
    int const &capP, PairRec<R> * const &coefE, R * const &coefEB, PairRec<R> * const &coefP, R * const &coefPB,
    const Excl &ex, const EwaldCoef &ec, const ScaleTables &c_scales, double * const &fieldD,
    double * const &fieldP, int * const &flags, const double2 *__restrict__ const &pos,
    const R *__restrict__ const &rec, const int *__restrict__ const &nbl, const int *__restrict__ const &nbl_cnt,
    int const &capN) {
  using V2 = typename Vec2<R>::type;
  const int warp = (vg.bid * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int i = warp;
  const unsigned lt = (1u << lane) - 1u;
  const double xi = x[i], yi = y[i], zi = z[i];
  // ---- phase 1: sub-lists, from the near row when the near list is valid (every Ewald
  // pair of this evaluation is in it), else from the buffered row
  {
    const bool nearrow = nbl && !(*flags & FLAG_NEAR_INVALID);
    const int cnt = nearrow ? min(nbl_cnt[i], capN) : min(nbr_cnt[i], cap);
    const int *row = nearrow ? nbl + (size_t)i * capN : nbr + (size_t)i * cap;
    int ce = 0, cp = 0;
    for (int base = 0; base < cnt; base += 32) {
      const int a = base + lane;
      bool ew = false, pr = false;
      int k = -1;
      if (a < cnt) {
        k = row[a];
        double xk, yk, zk;
        load_pos(pos, k, xk, yk, zk);
        double dx = __dsub_rn(xk, xi), dy = __dsub_rn(yk, yi), dz = __dsub_rn(zk, zi);
        const double r2 = pair_image(dx, dy, dz, bx, nbr_sh, (size_t)i * cap + a, 1.0);
        ew = r2 <= off2;
        pr = ew && (r2 <= pcut2);   // sqrt(r2) < pcut, exactly (pcut2 from below_sqrt)
      }
      const unsigned me = __ballot_sync(0xffffffffu, ew);
      const unsigned mp = __ballot_sync(0xffffffffu, pr);
      if (ew) {
        const int pos = ce + __popc(me & lt);
        if (pos < capE) {
          ewl[(size_t)i * capE + pos] = k;
          if (nbr_sh) ewl_sh[(size_t)i * capE + pos] = nbr_sh[(size_t)i * cap + a];
        }
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
  const R pdi = ipdamp[i], pti = thole[i];
  const R aewald = ec.aewald, an0 = ec.an0, an1 = ec.an1, an2 = ec.an2;
  R fx = 0, fy = 0, fz = 0, px = 0, py = 0, pz = 0;
  const int cnt = min(ewl_cnt[i], capE);
  const int *row = ewl + (size_t)i * capE;
  int cp = 0;
  for (int base = 0; base < cnt; base += 32) {
    const int a = base + lane;
    const bool act = a < cnt;
    bool pr = false;
    R pA = R(0), pB = R(0), px_ = R(0), py_ = R(0), pz_ = R(0);
    int pk = 0;
    if (act) {
      const int k = row[a];
      const size_t ent = (size_t)i * capE + a;
      double xk, yk, zk;
      load_pos(pos, k, xk, yk, zk);
      R mk[12];
      load_rec<0, 12>(rec, k, mk);
      double xd = __dsub_rn(xk, xi), yd = __dsub_rn(yk, yi), zd = __dsub_rn(zk, zi);
      const double r2d = pair_image(xd, yd, zd, bx, ewl_sh, ent, 1.0);
      const R xr = (R)xd, yr = (R)yd, zr = (R)zd, r2 = (R)r2d;
      const R ck = mk[t000], dkx = mk[t100], dky = mk[t010], dkz = mk[t001];
      const R qkxx = mk[t200], qkyy = mk[t020], qkzz = mk[t002], qkxy = mk[t110], qkxz = mk[t101], qkyz = mk[t011];
      const R r = m_sqrt(r2);
      const R ralpha = aewald * r;
      const R exp2a = m_exp(-ralpha * ralpha);
      const R rr1 = R(1.0) / r, rr2 = rr1 * rr1;
      const R bn0 = m_erfc(ralpha) * rr1;
      const R bn1 = (bn0 + an0 * exp2a) * rr2;
      const R bn2 = (R(3.0) * bn1 + an1 * exp2a) * rr2;
      const R bn3 = (R(5.0) * bn2 + an2 * exp2a) * rr2;
      R scale3 = R(1.0), scale5 = R(1.0), scale7 = R(1.0);
      R damp = pdi * mk[10];
      const R pgamma = m_min(pti, mk[11]);
      const R rdamp = r * damp;
      damp = -pgamma * rdamp * rdamp * rdamp;
      if (damp > -R(50.0)) {
        const R expdamp = m_exp(damp);
        scale3 = R(1.0) - expdamp;
        scale5 = R(1.0) - expdamp * (R(1.0) - damp);
        scale7 = R(1.0) - expdamp * (R(1.0) - damp + R(0.6) * damp * damp);
      }
      const unsigned code = pair_primary(ewl_sh, ent) ? excl_code(i, k, ex.ptr, ex.k, ex.code, ex.lo, ex.hi) : 0u;
      const R scale = c_scales.d[(code >> 6) & 1u];
      const R scalep = c_scales.p[(code >> 3) & 7u];
      const R dsc3 = scale3 * scale, dsc5 = scale5 * scale, dsc7 = scale7 * scale;
      const R psc3 = scale3 * scalep, psc5 = scale5 * scalep, psc7 = scale7 * scalep;
      const R rr3 = rr1 * rr2, rr5 = R(3.0) * rr3 * rr2, rr7 = R(5.0) * rr5 * rr2;
      const R drr3 = (R(1.0) - dsc3) * rr3, drr5 = (R(1.0) - dsc5) * rr5, drr7 = (R(1.0) - dsc7) * rr7;
      const R prr3 = (R(1.0) - psc3) * rr3, prr5 = (R(1.0) - psc5) * rr5, prr7 = (R(1.0) - psc7) * rr7;
      const R dkr = dkx * xr + dky * yr + dkz * zr;
      const R qkx = R(2.0) * (qkxx * xr + qkxy * yr + qkxz * zr);
      const R qky = R(2.0) * (qkxy * xr + qkyy * yr + qkyz * zr);
      const R qkz = R(2.0) * (qkxz * xr + qkyz * yr + qkzz * zr);
      const R qkr = (qkx * xr + qky * yr + qkz * zr) * R(0.5);
      const R bn123k = bn1 * ck - bn2 * dkr + bn3 * qkr;
      const R fimx = -xr * bn123k - bn1 * dkx + bn2 * qkx;
      const R fimy = -yr * bn123k - bn1 * dky + bn2 * qky;
      const R fimz = -zr * bn123k - bn1 * dkz + bn2 * qkz;
      const R drr357k = drr3 * ck - drr5 * dkr + drr7 * qkr;
      const R fidx = -xr * drr357k - drr3 * dkx + drr5 * qkx;
      const R fidy = -yr * drr357k - drr3 * dky + drr5 * qky;
      const R fidz = -zr * drr357k - drr3 * dkz + drr5 * qkz;
      fx += fimx - fidx; fy += fimy - fidy; fz += fimz - fidz;
      const R prr357k = prr3 * ck - prr5 * dkr + prr7 * qkr;
      const R fipx = -xr * prr357k - prr3 * dkx + prr5 * qkx;
      const R fipy = -yr * prr357k - prr3 * dky + prr5 * qky;
      const R fipz = -zr * prr357k - prr3 * dkz + prr5 * qkz;
      px += fimx - fipx; py += fimy - fipy; pz += fimz - fipz;
      // Induced-field coefficients (no masks), InducedDipoleFieldRegion.java:383-404.
      const R urr3 = (R(1.0) - scale3) * rr3, urr5 = (R(1.0) - scale5) * rr5;
      if (a < capE) {
        store_pair(coefE, (size_t)i * capE + a, xr, yr, zr, bn1 - urr3);
        store_pair_b(coefEB, (size_t)i * capE + a, k, bn2 - urr5);
      }
      pr = r2d <= pcut2;   // the same test, in FP64, that selected the preconditioner row
      if (pr) {
        const R b1 = rr1 * rr2, b2 = R(3.0) * b1 * rr2;   // Ewald off: bn0 = 1/r
        pA = b1 - urr3;
        pB = b2 - urr5;
        pk = k;
        px_ = xr; py_ = yr; pz_ = zr;
      }
    }
    const unsigned mp = __ballot_sync(0xffffffffu, pr);
    if (pr) {
      const int pos = cp + __popc(mp & lt);
      if (pos < capP) {
        store_pair(coefP, (size_t)i * capP + pos, px_, py_, pz_, pA);
        store_pair_b(coefPB, (size_t)i * capP + pos, pk, pB);
      }
    }
    cp += __popc(mp);
  }
  double Fx = warp_sum((double)fx), Fy = warp_sum((double)fy), Fz = warp_sum((double)fz);
  double Px = warp_sum((double)px), Py = warp_sum((double)py), Pz = warp_sum((double)pz);
  if (lane == 0) {
    fieldD[i] = Fx; fieldD[n + i] = Fy; fieldD[2 * n + i] = Fz;
    fieldP[i] = Px; fieldP[n + i] = Py; fieldP[2 * n + i] = Pz;
  }
}


// Direct dipoles of both sets, u = alpha (E_real + E_self + E_recip), from the real-space
// fields, the Ewald self field of the dipole and the reciprocal potential gradient
// (DirectLoop, pme/DirectRegion.java:170-243), and their source record for the first PCG
// field; the field rows are completed in place.  Separate from k_realspace_field so that
// the permanent reciprocal chain can run beside it.
template <typename R>
__device__ __forceinline__ void k_direct_dipoles(VGrid vg, int n, const double *__restrict__ gm, const double *__restrict__ cphi,
                                 const double *__restrict__ polar, double aewald3, double *fieldD, double *fieldP,
                                 double *uD, double *uP, double *udD, double *udP, R *recF) {
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double a = polar[i];
  double d[3], q[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const size_t j = (size_t)c * n + i;
    const double f = aewald3 * gm[(size_t)(1 + c) * n + i] - cphi[(size_t)(1 + c) * n + i];
    const double fd = fieldD[j] + f, fp = fieldP[j] + f;
    fieldD[j] = fd;
    fieldP[j] = fp;
    d[c] = a * fd;
    q[c] = a * fp;
    uD[j] = d[c]; udD[j] = d[c];
    uP[j] = q[c]; udP[j] = q[c];
  }
  put_rec(recF, i, d[0], d[1], d[2], q[0], q[1], q[2]);
}

// ---------------------------------------------------------------------------
// Permanent and polarization real-space energy, i-side force and torque.
// LAM: the electrostatic lambda variant (RealSpaceEnergyRegion.java:873-883, 1190-1690,
// 2153-2176): pairs with a soft atom take r^2 + beta and the scale permScale in the
// permanent part, the polarization part is scaled by polScale, and dU/dL, d2U/dL2, the
// lambda gradient and torque are gathered (written to edl/ed2l/lgrad/ltorque).
// Adds (vx, vy, vz) to row-major [3][n] v at atom k.  FP64 form: FP64 atomics.  FP32 form:
// each value is rounded to a multiple of 2^-32 first, so the sums are exact in FP64 (below
// 2^21 in magnitude) and independent of the order of the atomics.
// A contribution of kQuantLimit or more raises FLAG_QUANT_RANGE (the accumulated values are
// checked where the gradient is assembled).
template <typename R>
__device__ __forceinline__ void real_acc(double *v, int k, double vx, double vy, double vz, int n, int *flags) {
  if constexpr (sizeof(R) == 4) {
    if (quant_out(vx) || quant_out(vy) || quant_out(vz)) atomicOr(flags, FLAG_QUANT_RANGE);
    vx = rint(vx * 4294967296.0) * 2.3283064365386962890625e-10;
    vy = rint(vy * 4294967296.0) * 2.3283064365386962890625e-10;
    vz = rint(vz * 4294967296.0) * 2.3283064365386962890625e-10;
  }
  atomicAdd(v + k, vx); atomicAdd(v + n + k, vy); atomicAdd(v + 2 * (size_t)n + k, vz);
}

#ifndef FFX_REAL_ENERGY_MIN_BLOCKS
#define FFX_REAL_ENERGY_MIN_BLOCKS 4   // FP32 form: resident 128-thread blocks per SM
#endif
template <typename R, bool LAM, bool DIRECT>
__device__ __forceinline__ void k_real_energy(VGrid vg, 
    int n, const double *__restrict__ x, const double *__restrict__ y, const double *__restrict__ z, const Box &bx,
    const double *__restrict__ gm, const double *__restrict__ uD, const double *__restrict__ uP,
    const double *__restrict__ ipdamp, const double *__restrict__ thole, const int *__restrict__ ewl,
    const int *__restrict__ ewl_cnt, int capE, const int *__restrict__ ewl_sh, const Excl &ex, const EwaldCoef &ec, const ScaleTables &c_scales, int polarization, int gradient,
    double *eatom_perm, double *eatom_pol, long long *catom, double *grad, double *torque,
    const int *__restrict__ soft, const ElecStep &st, double *edl, double *ed2l, double *lgrad, double *ltorque,
    const double2 *__restrict__ pos, const R *__restrict__ rec, int *flags) {
  constexpr bool HALF = !LAM && !DIRECT;   // the softcore and direct forms walk the full rows
  __shared__ int qbuf[HALF ? 4 : 1][64];
  const int warp = (vg.bid * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  // Warps stride over the atoms: the single-system launch keeps its grid to the blocks
  // that are resident at once.
  for (int i = warp; i < n; i += (vg.nblk * (int)blockDim.x) >> 5) {
    const double xi = x[i], yi = y[i], zi = z[i];
    const R ci = gm[t000 * n + i], dix = gm[t100 * n + i], diy = gm[t010 * n + i], diz = gm[t001 * n + i];
    const R qixx = gm[t200 * n + i] * (R(1.0) / R(3.0)), qiyy = gm[t020 * n + i] * (R(1.0) / R(3.0));
    const R qizz = gm[t002 * n + i] * (R(1.0) / R(3.0)), qixy = gm[t110 * n + i] * (R(1.0) / R(3.0));
    const R qixz = gm[t101 * n + i] * (R(1.0) / R(3.0)), qiyz = gm[t011 * n + i] * (R(1.0) / R(3.0));
    const R uix = uD[i], uiy = uD[n + i], uiz = uD[2 * n + i];
    const R pix = uP[i], piy = uP[n + i], piz = uP[2 * n + i];
    const R pdi = ipdamp[i], pti = thole[i];
    const R aewald = ec.aewald, an0 = ec.an0, an1 = ec.an1, an2 = ec.an2, an3 = ec.an3, an4 = ec.an4;
    const R an5 = ec.an5;
    const R electric = ec.electric;
    const bool doPol = polarization != FFXG_POLAR_NONE && (!LAM || st.doPol);
    const bool doPerm = !LAM || st.doPermReal;
    const bool gr = gradient || LAM;
    double eP = 0, eI = 0;
    long long cnt_pairs = 0;
    R gx = 0, gy = 0, gz = 0, tx = 0, ty = 0, tz = 0;
    double dl = 0, d2l = 0;
    R lgx = 0, lgy = 0, lgz = 0, ltx = 0, lty = 0, ltz = 0;
    const int soft_i = LAM ? soft[i] : 0;
    const int cnt = min(ewl_cnt[i], capE);
    const int *row = ewl + (size_t)i * capE;
    // One pair of the Ewald row (entry a).  The full form (HALF false) takes every entry and
    // keeps only atom i's share; the half form takes each pair once (pair_counted) and adds
    // atom k's force and torque (RealSpaceEnergyRegion.java:1457-1460, 2157-2160) with
    // atomics into grad and torque, zeroed by k_pack_induced.
    auto pair = [&](int a) {
      const int k = row[a];
      const size_t ent = (size_t)i * capE + a;
      double xk, yk, zk;
      load_pos(pos, k, xk, yk, zk);
      R mk[12], uk[8];
      load_rec<0, 12>(rec, k, mk);
      load_rec<kRecInduced, 8>(rec, k, uk);
      double xd = __dsub_rn(xk, xi), yd = __dsub_rn(yk, yi), zd = __dsub_rn(zk, zi);
      const double r2d = pair_image(xd, yd, zd, bx, ewl_sh, ent, 1.0);
      const R xr = (R)xd, yr = (R)yd, zr = (R)zd, r2 = (R)r2d;
      const R ck = mk[t000], dkx = mk[t100], dky = mk[t010], dkz = mk[t001];
      const R qkxx = mk[t200], qkyy = mk[t020], qkzz = mk[t002], qkxy = mk[t110], qkxz = mk[t101], qkyz = mk[t011];
      const R ukx = uk[0], uky = uk[1], ukz = uk[2];
      const R pkx = uk[3], pky = uk[4], pkz = uk[5];
      const unsigned code = pair_primary(ewl_sh, ent) ? excl_code(i, k, ex.ptr, ex.k, ex.code, ex.lo, ex.hi) : 0u;
      const R scale = c_scales.m[code & 7u];
      const R scalep = c_scales.p[(code >> 3) & 7u];
      const R scaled = c_scales.d[(code >> 6) & 1u];
      bool spair = false;
      R l2 = R(1.0);
      double r2s = r2d;
      if (LAM) {
        spair = soft_i || soft[k];
        if (spair && st.doPermReal) { r2s = r2d + st.beta; l2 = (R)st.permScale; }
      }
      const R r = m_sqrt(LAM ? (R)r2s : r2);
      const R ralpha = aewald * r;
      const R exp2a = m_exp(-ralpha * ralpha);
      const R rr1 = R(1.0) / r, rr2 = rr1 * rr1;
      const R bn0 = m_erfc(ralpha) * rr1;
      const R bn1 = (bn0 + an0 * exp2a) * rr2;
      const R bn2 = (R(3.0) * bn1 + an1 * exp2a) * rr2;
      const R bn3 = (R(5.0) * bn2 + an2 * exp2a) * rr2;
      const R bn4 = (R(7.0) * bn3 + an3 * exp2a) * rr2;
      const R bn5 = (R(9.0) * bn4 + an4 * exp2a) * rr2;
      const R rr3 = rr1 * rr2, rr5 = R(3.0) * rr3 * rr2, rr7 = R(5.0) * rr5 * rr2;
      const R rr9 = R(7.0) * rr7 * rr2, rr11 = R(9.0) * rr9 * rr2;
      R scale3 = R(1.0), scale5 = R(1.0), scale7 = R(1.0);
      R ddsc3x = 0, ddsc3y = 0, ddsc3z = 0, ddsc5x = 0, ddsc5y = 0, ddsc5z = 0, ddsc7x = 0, ddsc7y = 0, ddsc7z = 0;
      (void)an5;
      R damp = pdi * mk[10];
      const R tho = m_min(pti, mk[11]);
      const R rdamp = r * damp;
      damp = -tho * rdamp * rdamp * rdamp;
      if (damp > -R(50.0)) {
        const R expdamp = m_exp(damp);
        scale3 = R(1.0) - expdamp;
        scale5 = R(1.0) - expdamp * (R(1.0) - damp);
        scale7 = R(1.0) - expdamp * (R(1.0) - damp + R(0.6) * damp * damp);
        const R temp3 = -R(3.0) * damp * expdamp * rr2;
        const R temp5 = -damp;
        const R temp7 = -R(0.2) - R(0.6) * damp;
        ddsc3x = temp3 * xr; ddsc3y = temp3 * yr; ddsc3z = temp3 * zr;
        ddsc5x = temp5 * ddsc3x; ddsc5y = temp5 * ddsc3y; ddsc5z = temp5 * ddsc3z;
        ddsc7x = temp7 * ddsc5x; ddsc7y = temp7 * ddsc5y; ddsc7z = temp7 * ddsc5z;
      }
      // ---- permanentPair
      if (doPerm) {
        const R dixdkx = diy * dkz - diz * dky, dixdky = diz * dkx - dix * dkz, dixdkz = dix * dky - diy * dkx;
        const R dixrx = diy * zr - diz * yr, dixry = diz * xr - dix * zr, dixrz = dix * yr - diy * xr;
        const R dkxrx = dky * zr - dkz * yr, dkxry = dkz * xr - dkx * zr, dkxrz = dkx * yr - dky * xr;
        const R qirx = qixx * xr + qixy * yr + qixz * zr;
        const R qiry = qixy * xr + qiyy * yr + qiyz * zr;
        const R qirz = qixz * xr + qiyz * yr + qizz * zr;
        const R qkrx = qkxx * xr + qkxy * yr + qkxz * zr;
        const R qkry = qkxy * xr + qkyy * yr + qkyz * zr;
        const R qkrz = qkxz * xr + qkyz * yr + qkzz * zr;
        const R qiqkrx = qixx * qkrx + qixy * qkry + qixz * qkrz;
        const R qiqkry = qixy * qkrx + qiyy * qkry + qiyz * qkrz;
        const R qiqkrz = qixz * qkrx + qiyz * qkry + qizz * qkrz;
        const R qkqirx = qkxx * qirx + qkxy * qiry + qkxz * qirz;
        const R qkqiry = qkxy * qirx + qkyy * qiry + qkyz * qirz;
        const R qkqirz = qkxz * qirx + qkyz * qiry + qkzz * qirz;
        const R qixqkx = qixy * qkxz + qiyy * qkyz + qiyz * qkzz - qixz * qkxy - qiyz * qkyy - qizz * qkyz;
        const R qixqky = qixz * qkxx + qiyz * qkxy + qizz * qkxz - qixx * qkxz - qixy * qkyz - qixz * qkzz;
        const R qixqkz = qixx * qkxy + qixy * qkyy + qixz * qkyz - qixy * qkxx - qiyy * qkxy - qiyz * qkxz;
        const R rxqirx = yr * qirz - zr * qiry, rxqiry = zr * qirx - xr * qirz, rxqirz = xr * qiry - yr * qirx;
        const R rxqkrx = yr * qkrz - zr * qkry, rxqkry = zr * qkrx - xr * qkrz, rxqkrz = xr * qkry - yr * qkrx;
        const R rxqikrx = yr * qiqkrz - zr * qiqkry, rxqikry = zr * qiqkrx - xr * qiqkrz, rxqikrz = xr * qiqkry - yr * qiqkrx;
        const R rxqkirx = yr * qkqirz - zr * qkqiry, rxqkiry = zr * qkqirx - xr * qkqirz, rxqkirz = xr * qkqiry - yr * qkqirx;
        const R qkrxqirx = qkry * qirz - qkrz * qiry, qkrxqiry = qkrz * qirx - qkrx * qirz, qkrxqirz = qkrx * qiry - qkry * qirx;
        const R qidkx = qixx * dkx + qixy * dky + qixz * dkz;
        const R qidky = qixy * dkx + qiyy * dky + qiyz * dkz;
        const R qidkz = qixz * dkx + qiyz * dky + qizz * dkz;
        const R qkdix = qkxx * dix + qkxy * diy + qkxz * diz;
        const R qkdiy = qkxy * dix + qkyy * diy + qkyz * diz;
        const R qkdiz = qkxz * dix + qkyz * diy + qkzz * diz;
        const R dixqkrx = diy * qkrz - diz * qkry, dixqkry = diz * qkrx - dix * qkrz, dixqkrz = dix * qkry - diy * qkrx;
        const R dkxqirx = dky * qirz - dkz * qiry, dkxqiry = dkz * qirx - dkx * qirz, dkxqirz = dkx * qiry - dky * qirx;
        const R rxqidkx = yr * qidkz - zr * qidky, rxqidky = zr * qidkx - xr * qidkz, rxqidkz = xr * qidky - yr * qidkx;
        const R rxqkdix = yr * qkdiz - zr * qkdiy, rxqkdiy = zr * qkdix - xr * qkdiz, rxqkdiz = xr * qkdiy - yr * qkdix;
        const R sc2 = dix * dkx + diy * dky + diz * dkz;
        const R sc3 = dix * xr + diy * yr + diz * zr;
        const R sc4 = dkx * xr + dky * yr + dkz * zr;
        const R sc5 = qirx * xr + qiry * yr + qirz * zr;
        const R sc6 = qkrx * xr + qkry * yr + qkrz * zr;
        const R sc7 = qirx * dkx + qiry * dky + qirz * dkz;
        const R sc8 = qkrx * dix + qkry * diy + qkrz * diz;
        const R sc9 = qirx * qkrx + qiry * qkry + qirz * qkrz;
        const R sc10 = R(2.0) * (qixy * qkxy + qixz * qkxz + qiyz * qkyz) + qixx * qkxx + qiyy * qkyy + qizz * qkzz;
        const R gl0 = ci * ck, gl1 = ck * sc3 - ci * sc4, gl2 = ci * sc6 + ck * sc5 - sc3 * sc4;
        const R gl3 = sc3 * sc6 - sc4 * sc5, gl4 = sc5 * sc6, gl5 = -R(4.0) * sc9, gl6 = sc2;
        const R gl7 = R(2.0) * (sc7 - sc8), gl8 = R(2.0) * sc10;
        // The masked part (scale1 = 1 - scale of the Ewald-free tensor) enters every energy,
        // force and torque expression linearly in the radial factors, so the combined factors
        // b_k = bn_k - scale1 rr_(2k+1) give ereal - efix and the corrected forces and torques
        // in one contraction (the reference evaluates the masked correction as a second pass).
        const R scale1 = R(1.0) - scale;
        const R b0 = bn0 - scale1 * rr1, b1 = bn1 - scale1 * rr3, b2 = bn2 - scale1 * rr5;
        const R b3 = bn3 - scale1 * rr7, b4 = bn4 - scale1 * rr9, b5 = bn5 - scale1 * rr11;
        const R e = gl0 * b0 + (gl1 + gl6) * b1 + (gl2 + gl7 + gl8) * b2 + (gl3 + gl5) * b3 + gl4 * b4;
        if (e != R(0.0)) { eP += (HALF ? R(1.0) : R(0.5)) * (LAM ? l2 * e : e); if (pair_counted(i, k, ewl_sh, ent)) cnt_pairs++; }
        if (gr) {
          const R gf1 = b1 * gl0 + b2 * (gl1 + gl6) + b3 * (gl2 + gl7 + gl8) + b4 * (gl3 + gl5) + b5 * gl4;
          const R gf2 = -ck * b1 + sc4 * b2 - sc6 * b3;
          const R gf3 = ci * b1 + sc3 * b2 + sc5 * b3;
          const R gf4 = R(2.0) * b2;
          const R gf5 = R(2.0) * (-ck * b2 + sc4 * b3 - sc6 * b4);
          const R gf6 = R(2.0) * (-ci * b2 - sc3 * b3 - sc5 * b4);
          const R gf7 = R(4.0) * b3;
          const R ftm2x = gf1 * xr + gf2 * dix + gf3 * dkx + gf4 * (qkdix - qidkx) + gf5 * qirx + gf6 * qkrx + gf7 * (qiqkrx + qkqirx);
          const R ftm2y = gf1 * yr + gf2 * diy + gf3 * dky + gf4 * (qkdiy - qidky) + gf5 * qiry + gf6 * qkry + gf7 * (qiqkry + qkqiry);
          const R ftm2z = gf1 * zr + gf2 * diz + gf3 * dkz + gf4 * (qkdiz - qidkz) + gf5 * qirz + gf6 * qkrz + gf7 * (qiqkrz + qkqirz);
          const R ttm2x = -b1 * dixdkx + gf2 * dixrx + gf4 * (dixqkrx + dkxqirx + rxqidkx - R(2.0) * qixqkx) - gf5 * rxqirx - gf7 * (rxqikrx + qkrxqirx);
          const R ttm2y = -b1 * dixdky + gf2 * dixry + gf4 * (dixqkry + dkxqiry + rxqidky - R(2.0) * qixqky) - gf5 * rxqiry - gf7 * (rxqikry + qkrxqiry);
          const R ttm2z = -b1 * dixdkz + gf2 * dixrz + gf4 * (dixqkrz + dkxqirz + rxqidkz - R(2.0) * qixqkz) - gf5 * rxqirz - gf7 * (rxqikrz + qkrxqirz);
          const R ttm3x = b1 * dixdkx + gf3 * dkxrx - gf4 * (dixqkrx + dkxqirx + rxqkdix - R(2.0) * qixqkx) - gf6 * rxqkrx - gf7 * (rxqkirx - qkrxqirx);
          const R ttm3y = b1 * dixdky + gf3 * dkxry - gf4 * (dixqkry + dkxqiry + rxqkdiy - R(2.0) * qixqky) - gf6 * rxqkry - gf7 * (rxqkiry - qkrxqiry);
          const R ttm3z = b1 * dixdkz + gf3 * dkxrz - gf4 * (dixqkrz + dkxqirz + rxqkdiz - R(2.0) * qixqkz) - gf6 * rxqkrz - gf7 * (rxqkirz - qkrxqirz);
          const R pre = LAM ? electric * l2 : electric;
          gx += pre * ftm2x; gy += pre * ftm2y; gz += pre * ftm2z;
          tx += pre * ttm2x; ty += pre * ttm2y; tz += pre * ttm2z;
          if constexpr (HALF) {
            real_acc<R>(grad, k, -pre * ftm2x, -pre * ftm2y, -pre * ftm2z, n, flags);
            real_acc<R>(torque, k, pre * ttm3x, pre * ttm3y, pre * ttm3z, n, flags);
          }
          if (LAM && spair) {   // d[dlPow * ereal]/dX (:1465-1475)
            const R pf = electric * (R)(st.dEdLSign * st.dlPowPerm);
            lgx += pf * ftm2x; lgy += pf * ftm2y; lgz += pf * ftm2z;
            ltx += pf * ttm2x; lty += pf * ttm2y; ltz += pf * ttm2z;
          }
        }
        if (LAM && spair) {
          // dU/dL, d2U/dL2 through the scale and the softcore shift; dU/dL/dX of the second
          // term, every radial order one higher (:1477-1690).  Half weight per direction.
          const R bn6 = (R(11.0) * bn5 + an5 * exp2a) * rr2;
          const R rr13 = R(11.0) * rr11 * rr2;
          const R b6 = bn6 - scale1 * rr13;
          // ereal - efix = e and the radial derivatives of both through the combined factors
          // (one radial order higher per derivative).
          const R dEdL1 = gl0 * b1 + (gl1 + gl6) * b2 + (gl2 + gl7 + gl8) * b3 + (gl3 + gl5) * b4 + gl4 * b5;
          const R dEdL2 = gl0 * b2 + (gl1 + gl6) * b3 + (gl2 + gl7 + gl8) * b4 + (gl3 + gl5) * b5 + gl4 * b6;
          const double sg = st.dEdLSign, dP = st.dlPowPerm, d2P = st.d2lPowPerm, dA = st.dlAlpha, d2A = st.d2lAlpha;
          const double L2 = (double)l2;
          dl += 0.5 * (sg * dP * (double)e + L2 * dA * (double)dEdL1);
          d2l += 0.5 * (sg * (d2P * (double)e + 2.0 * dP * dA * (double)dEdL1) + L2 * d2A * (double)dEdL1 +
                        L2 * dA * dA * (double)dEdL2);
          const R gf1 = b2 * gl0 + b3 * (gl1 + gl6) + b4 * (gl2 + gl7 + gl8) + b5 * (gl3 + gl5) + b6 * gl4;
          const R gf2 = -ck * b2 + sc4 * b3 - sc6 * b4;
          const R gf3 = ci * b2 + sc3 * b3 + sc5 * b4;
          const R gf4 = R(2.0) * b3;
          const R gf5 = R(2.0) * (-ck * b3 + sc4 * b4 - sc6 * b5);
          const R gf6 = R(2.0) * (-ci * b3 - sc3 * b4 - sc5 * b5);
          const R gf7 = R(4.0) * b4;
          const R fx = gf1 * xr + gf2 * dix + gf3 * dkx + gf4 * (qkdix - qidkx) + gf5 * qirx + gf6 * qkrx + gf7 * (qiqkrx + qkqirx);
          const R fy = gf1 * yr + gf2 * diy + gf3 * dky + gf4 * (qkdiy - qidky) + gf5 * qiry + gf6 * qkry + gf7 * (qiqkry + qkqiry);
          const R fz = gf1 * zr + gf2 * diz + gf3 * dkz + gf4 * (qkdiz - qidkz) + gf5 * qirz + gf6 * qkrz + gf7 * (qiqkrz + qkqirz);
          const R qx = -b2 * dixdkx + gf2 * dixrx + gf4 * (dixqkrx + dkxqirx + rxqidkx - R(2.0) * qixqkx) - gf5 * rxqirx - gf7 * (rxqikrx + qkrxqirx);
          const R qy = -b2 * dixdky + gf2 * dixry + gf4 * (dixqkry + dkxqiry + rxqidky - R(2.0) * qixqky) - gf5 * rxqiry - gf7 * (rxqikry + qkrxqiry);
          const R qz = -b2 * dixdkz + gf2 * dixrz + gf4 * (dixqkrz + dkxqirz + rxqidkz - R(2.0) * qixqkz) - gf5 * rxqirz - gf7 * (rxqikrz + qkrxqirz);
          const R pf = electric * l2 * (R)st.dlAlpha;
          lgx += pf * fx; lgy += pf * fy; lgz += pf * fz;
          ltx += pf * qx; lty += pf * qy; ltz += pf * qz;
        }
      }
      if (!doPol) return;
      // ---- polarizationPair
      {
        const R dsc3 = R(1.0) - scale3 * scaled, dsc5 = R(1.0) - scale5 * scaled, dsc7 = R(1.0) - scale7 * scaled;
        const R psc3 = R(1.0) - scale3 * scalep, psc5 = R(1.0) - scale5 * scalep, psc7 = R(1.0) - scale7 * scalep;
        const R usc3 = R(1.0) - scale3, usc5 = R(1.0) - scale5;
        const R dixukx = diy * ukz - diz * uky, dixuky = diz * ukx - dix * ukz, dixukz = dix * uky - diy * ukx;
        const R dkxuix = dky * uiz - dkz * uiy, dkxuiy = dkz * uix - dkx * uiz, dkxuiz = dkx * uiy - dky * uix;
        const R dixukpx = diy * pkz - diz * pky, dixukpy = diz * pkx - dix * pkz, dixukpz = dix * pky - diy * pkx;
        const R dkxuipx = dky * piz - dkz * piy, dkxuipy = dkz * pix - dkx * piz, dkxuipz = dkx * piy - dky * pix;
        const R dixrx = diy * zr - diz * yr, dixry = diz * xr - dix * zr, dixrz = dix * yr - diy * xr;
        const R dkxrx = dky * zr - dkz * yr, dkxry = dkz * xr - dkx * zr, dkxrz = dkx * yr - dky * xr;
        const R qirx = qixx * xr + qixy * yr + qixz * zr;
        const R qiry = qixy * xr + qiyy * yr + qiyz * zr;
        const R qirz = qixz * xr + qiyz * yr + qizz * zr;
        const R qkrx = qkxx * xr + qkxy * yr + qkxz * zr;
        const R qkry = qkxy * xr + qkyy * yr + qkyz * zr;
        const R qkrz = qkxz * xr + qkyz * yr + qkzz * zr;
        const R rxqirx = yr * qirz - zr * qiry, rxqiry = zr * qirx - xr * qirz, rxqirz = xr * qiry - yr * qirx;
        const R rxqkrx = yr * qkrz - zr * qkry, rxqkry = zr * qkrx - xr * qkrz, rxqkrz = xr * qkry - yr * qkrx;
        const R qiukx = qixx * ukx + qixy * uky + qixz * ukz;
        const R qiuky = qixy * ukx + qiyy * uky + qiyz * ukz;
        const R qiukz = qixz * ukx + qiyz * uky + qizz * ukz;
        const R qkuix = qkxx * uix + qkxy * uiy + qkxz * uiz;
        const R qkuiy = qkxy * uix + qkyy * uiy + qkyz * uiz;
        const R qkuiz = qkxz * uix + qkyz * uiy + qkzz * uiz;
        const R qiukpx = qixx * pkx + qixy * pky + qixz * pkz;
        const R qiukpy = qixy * pkx + qiyy * pky + qiyz * pkz;
        const R qiukpz = qixz * pkx + qiyz * pky + qizz * pkz;
        const R qkuipx = qkxx * pix + qkxy * piy + qkxz * piz;
        const R qkuipy = qkxy * pix + qkyy * piy + qkyz * piz;
        const R qkuipz = qkxz * pix + qkyz * piy + qkzz * piz;
        const R uixqkrx = uiy * qkrz - uiz * qkry, uixqkry = uiz * qkrx - uix * qkrz, uixqkrz = uix * qkry - uiy * qkrx;
        const R ukxqirx = uky * qirz - ukz * qiry, ukxqiry = ukz * qirx - ukx * qirz, ukxqirz = ukx * qiry - uky * qirx;
        const R uixqkrpx = piy * qkrz - piz * qkry, uixqkrpy = piz * qkrx - pix * qkrz, uixqkrpz = pix * qkry - piy * qkrx;
        const R ukxqirpx = pky * qirz - pkz * qiry, ukxqirpy = pkz * qirx - pkx * qirz, ukxqirpz = pkx * qiry - pky * qirx;
        const R rxqiukx = yr * qiukz - zr * qiuky, rxqiuky = zr * qiukx - xr * qiukz, rxqiukz = xr * qiuky - yr * qiukx;
        const R rxqkuix = yr * qkuiz - zr * qkuiy, rxqkuiy = zr * qkuix - xr * qkuiz, rxqkuiz = xr * qkuiy - yr * qkuix;
        const R rxqiukpx = yr * qiukpz - zr * qiukpy, rxqiukpy = zr * qiukpx - xr * qiukpz, rxqiukpz = xr * qiukpy - yr * qiukpx;
        const R rxqkuipx = yr * qkuipz - zr * qkuipy, rxqkuipy = zr * qkuipx - xr * qkuipz, rxqkuipz = xr * qkuipy - yr * qkuipx;
        const R sc3 = dix * xr + diy * yr + diz * zr;
        const R sc4 = dkx * xr + dky * yr + dkz * zr;
        const R sc5 = qirx * xr + qiry * yr + qirz * zr;
        const R sc6 = qkrx * xr + qkry * yr + qkrz * zr;
        const R sci1 = uix * dkx + uiy * dky + uiz * dkz + dix * ukx + diy * uky + diz * ukz;
        const R sci3 = uix * xr + uiy * yr + uiz * zr;
        const R sci4 = ukx * xr + uky * yr + ukz * zr;
        const R sci7 = qirx * ukx + qiry * uky + qirz * ukz;
        const R sci8 = qkrx * uix + qkry * uiy + qkrz * uiz;
        const R scip1 = pix * dkx + piy * dky + piz * dkz + dix * pkx + diy * pky + diz * pkz;
        const R scip2 = uix * pkx + uiy * pky + uiz * pkz + pix * ukx + piy * uky + piz * ukz;
        const R scip3 = pix * xr + piy * yr + piz * zr;
        const R scip4 = pkx * xr + pky * yr + pkz * zr;
        const R scip7 = qirx * pkx + qiry * pky + qirz * pkz;
        const R scip8 = qkrx * pix + qkry * piy + qkrz * piz;
        const R gli1 = ck * sci3 - ci * sci4, gli2 = -sc3 * sci4 - sci3 * sc4, gli3 = sci3 * sc6 - sci4 * sc5;
        const R gli6 = sci1, gli7 = R(2.0) * (sci7 - sci8);
        const R glip1 = ck * scip3 - ci * scip4, glip2 = -sc3 * scip4 - scip3 * sc4, glip3 = scip3 * sc6 - scip4 * sc5;
        const R glip6 = scip1, glip7 = R(2.0) * (scip7 - scip8);
        // As for the permanent pair, the Thole-damped masked parts (p-, d- and u-scaled rr
        // terms) are linear in the radial factors: P, D and U below are bn_k minus the rr
        // term of each scale family, Pa..Dc the same one radial order higher, and every
        // energy, force and torque takes one contraction with them.
        const R P1 = bn1 - rr3 * psc3, P2 = bn2 - rr5 * psc5, P3 = bn3 - rr7 * psc7;
        const R epol = R(0.25) * ((gli1 + gli6) * P1 + (gli2 + gli7) * P2 + gli3 * P3);
        eI += HALF ? R(2.0) * epol : (LAM ? (R)st.polScale * epol : epol);
        if (LAM) {
          dl += st.dEdLSign * st.dlPowPol * (double)epol;
          d2l += st.dEdLSign * st.d2lPowPol * (double)epol;
        }
        if (!gr) return;
        const R D1 = bn1 - rr3 * dsc3, D2 = bn2 - rr5 * dsc5, D3 = bn3 - rr7 * dsc7;
        const R U2 = bn2 - rr5 * usc5;
        const R Pa = bn2 - rr5 * psc3, Da = bn2 - rr5 * dsc3, Ua = bn2 - rr5 * usc3;
        const R Pb = bn3 - rr7 * psc5, Db = bn3 - rr7 * dsc5, Ub = bn3 - rr7 * usc5;
        const R Pc = bn4 - rr9 * psc7, Dc = bn4 - rr9 * dsc7;
        const R sci34 = sci3 * scip4 + scip3 * sci4;
        const R gfi1 = R(0.5) * ((gli1 + gli6) * Pa + (glip1 + glip6) * Da + scip2 * Ua + (gli2 + gli7) * Pb +
                                 (glip2 + glip7) * Db - sci34 * Ub + gli3 * Pc + glip3 * Dc);
        const R fu = -ck * P1 + sc4 * P2 - sc6 * P3, fp = -ck * D1 + sc4 * D2 - sc6 * D3;
        const R ku = ci * P1 + sc3 * P2 + sc5 * P3, kp = ci * D1 + sc3 * D2 + sc5 * D3;
        const R di2 = sci4 * P2 + scip4 * D2, dk2 = sci3 * P2 + scip3 * D2;
        const R qi3 = sci4 * P3 + scip4 * D3, qk3 = sci3 * P3 + scip3 * D3;
        R ftm2ix = gfi1 * xr + R(0.5) * (uix * fu + pix * fp + ukx * ku + pkx * kp) +
                   R(0.5) * U2 * (sci4 * pix + scip4 * uix + sci3 * pkx + scip3 * ukx) + R(0.5) * (dix * di2 + dkx * dk2) +
                   (qkuix - qiukx) * P2 + (qkuipx - qiukpx) * D2 + qirx * qi3 - qkrx * qk3;
        R ftm2iy = gfi1 * yr + R(0.5) * (uiy * fu + piy * fp + uky * ku + pky * kp) +
                   R(0.5) * U2 * (sci4 * piy + scip4 * uiy + sci3 * pky + scip3 * uky) + R(0.5) * (diy * di2 + dky * dk2) +
                   (qkuiy - qiuky) * P2 + (qkuipy - qiukpy) * D2 + qiry * qi3 - qkry * qk3;
        R ftm2iz = gfi1 * zr + R(0.5) * (uiz * fu + piz * fp + ukz * ku + pkz * kp) +
                   R(0.5) * U2 * (sci4 * piz + scip4 * uiz + sci3 * pkz + scip3 * ukz) + R(0.5) * (diz * di2 + dkz * dk2) +
                   (qkuiz - qiukz) * P2 + (qkuipz - qiukpz) * D2 + qirz * qi3 - qkrz * qk3;
        const R ttm2ix = -R(0.5) * (dixukx * P1 + dixukpx * D1) + R(0.5) * dixrx * di2 - rxqirx * qi3 +
                         (ukxqirx + rxqiukx) * P2 + (ukxqirpx + rxqiukpx) * D2;
        const R ttm2iy = -R(0.5) * (dixuky * P1 + dixukpy * D1) + R(0.5) * dixry * di2 - rxqiry * qi3 +
                         (ukxqiry + rxqiuky) * P2 + (ukxqirpy + rxqiukpy) * D2;
        const R ttm2iz = -R(0.5) * (dixukz * P1 + dixukpz * D1) + R(0.5) * dixrz * di2 - rxqirz * qi3 +
                         (ukxqirz + rxqiukz) * P2 + (ukxqirpz + rxqiukpz) * D2;
        const R ttm3ix = -R(0.5) * (dkxuix * P1 + dkxuipx * D1) + R(0.5) * dkxrx * dk2 + rxqkrx * qk3 -
                         (uixqkrx + rxqkuix) * P2 - (uixqkrpx + rxqkuipx) * D2;
        const R ttm3iy = -R(0.5) * (dkxuiy * P1 + dkxuipy * D1) + R(0.5) * dkxry * dk2 + rxqkry * qk3 -
                         (uixqkry + rxqkuiy) * P2 - (uixqkrpy + rxqkuipy) * D2;
        const R ttm3iz = -R(0.5) * (dkxuiz * P1 + dkxuipz * D1) + R(0.5) * dkxrz * dk2 + rxqkrz * qk3 -
                         (uixqkrz + rxqkuiz) * P2 - (uixqkrpz + rxqkuipz) * D2;
        R temp3 = R(0.5) * rr3 * ((gli1 + gli6) * scalep + (glip1 + glip6) * scaled);
        R temp5 = R(0.5) * rr5 * ((gli2 + gli7) * scalep + (glip2 + glip7) * scaled);
        const R temp7 = R(0.5) * rr7 * (gli3 * scalep + glip3 * scaled);
        const R fridmpx = temp3 * ddsc3x + temp5 * ddsc5x + temp7 * ddsc7x;
        const R fridmpy = temp3 * ddsc3y + temp5 * ddsc5y + temp7 * ddsc7y;
        const R fridmpz = temp3 * ddsc3z + temp5 * ddsc5z + temp7 * ddsc7z;
        temp3 = R(0.5) * rr3 * scip2;
        temp5 = -R(0.5) * rr5 * (sci3 * scip4 + scip3 * sci4);
        const R findmpx = temp3 * ddsc3x + temp5 * ddsc5x;
        const R findmpy = temp3 * ddsc3y + temp5 * ddsc5y;
        const R findmpz = temp3 * ddsc3z + temp5 * ddsc5z;
        ftm2ix = ftm2ix - fridmpx - findmpx;
        ftm2iy = ftm2iy - fridmpy - findmpy;
        ftm2iz = ftm2iz - fridmpz - findmpz;
        if (DIRECT) {   // the direct-polarization terms (compiled out of the mutual form)
          const R gfd = R(0.5) * (scip2 * Ua - sci34 * Ub);
          ftm2ix = ftm2ix - gfd * xr - R(0.5) * U2 * (sci4 * pix + scip4 * uix + sci3 * pkx + scip3 * ukx) + findmpx;
          ftm2iy = ftm2iy - gfd * yr - R(0.5) * U2 * (sci4 * piy + scip4 * uiy + sci3 * pky + scip3 * uky) + findmpy;
          ftm2iz = ftm2iz - gfd * zr - R(0.5) * U2 * (sci4 * piz + scip4 * uiz + sci3 * pkz + scip3 * ukz) + findmpz;
        }
        const R sc = LAM ? electric * (R)st.polScale : electric;
        gx += sc * ftm2ix; gy += sc * ftm2iy; gz += sc * ftm2iz;
        tx += sc * ttm2ix; ty += sc * ttm2iy; tz += sc * ttm2iz;
        if constexpr (HALF) {
          real_acc<R>(grad, k, -sc * ftm2ix, -sc * ftm2iy, -sc * ftm2iz, n, flags);
          real_acc<R>(torque, k, sc * ttm3ix, sc * ttm3iy, sc * ttm3iz, n, flags);
        }
        if (LAM) {   // RealSpaceEnergyRegion.java:2163-2174
          const R sl = electric * (R)(st.dEdLSign * st.dlPowPol);
          lgx += sl * ftm2ix; lgy += sl * ftm2iy; lgz += sl * ftm2iz;
          ltx += sl * ttm2ix; lty += sl * ttm2iy; ltz += sl * ttm2iz;
        }
      }

    };
    if constexpr (HALF) {
      // Counted entries are queued in shared memory and evaluated 32 at a time, so the
      // pair arithmetic runs on full warps although half of each row is skipped.
      // One call site of the pair body: fill to 32 or the end of the row, evaluate, shift.
      int *q = qbuf[threadIdx.x >> 5];
      int qn = 0, base = 0;   // warp-uniform; qn < 64 after every fill
      while (true) {
        while (qn < 32 && base < cnt) {
          const int a = base + lane;
          const bool take = a < cnt && pair_counted(i, row[a], ewl_sh, (size_t)i * capE + a);
          const unsigned bal = __ballot_sync(0xffffffffu, take);
          if (take) q[qn + __popc(bal & ((1u << lane) - 1u))] = a;
          qn += __popc(bal);
          base += 32;
        }
        __syncwarp();
        if (qn == 0) break;
        if (lane < qn) pair(q[lane]);
        __syncwarp();
        const int rest = qn > 32 ? qn - 32 : 0;
        if (lane < rest) q[lane] = q[lane + 32];
        __syncwarp();
        qn = rest;
      }
    } else {
      for (int a = lane; a < cnt; a += 32) pair(a);
    }
    eP = warp_sum(eP); eI = warp_sum(eI);
    const double Gx = warp_sum((double)gx), Gy = warp_sum((double)gy), Gz = warp_sum((double)gz);
    const double Tx = warp_sum((double)tx), Ty = warp_sum((double)ty), Tz = warp_sum((double)tz);
  #pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt_pairs += __shfl_xor_sync(0xffffffffu, cnt_pairs, o);
    double L[8];
    if (LAM) {
      L[0] = warp_sum(dl); L[1] = warp_sum(d2l);
      L[2] = warp_sum((double)lgx); L[3] = warp_sum((double)lgy); L[4] = warp_sum((double)lgz);
      L[5] = warp_sum((double)ltx); L[6] = warp_sum((double)lty); L[7] = warp_sum((double)ltz);
    }
    if (lane == 0) {
      eatom_perm[i] = eP * ec.electric;
      eatom_pol[i] = eI * ec.electric;
      catom[i] = cnt_pairs;
      if (gr) {
        if constexpr (HALF) {
          real_acc<R>(grad, i, Gx, Gy, Gz, n, flags);
          real_acc<R>(torque, i, Tx, Ty, Tz, n, flags);
        } else {
          grad[i] = Gx; grad[n + i] = Gy; grad[2 * n + i] = Gz;
          torque[i] = Tx; torque[n + i] = Ty; torque[2 * n + i] = Tz;
        }
      }
      if (LAM) {
        edl[i] = L[0] * ec.electric;
        ed2l[i] = L[1] * ec.electric;
        lgrad[i] = L[2]; lgrad[n + i] = L[3]; lgrad[2 * n + i] = L[4];
        ltorque[i] = L[5]; ltorque[n + i] = L[6]; ltorque[2 * n + i] = L[7];
      }
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


// Gather records (kRecStride layout): multipole part from the global-frame multipoles and
// the Thole parameters, induced part from u_D and u_P.  The quadrupole is divided by 3 in
// the pair kernels' own expression.
template <typename R>
__device__ __forceinline__ void k_pack_mpole(VGrid vg, int n, const double *__restrict__ gm, const double *__restrict__ ipdamp,
                             const double *__restrict__ thole, R *rec) {
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n) return;
  R v[16];
#pragma unroll
  for (int j = 0; j < 4; j++) v[j] = (R)gm[(size_t)j * n + i];
#pragma unroll
  for (int j = 4; j < 10; j++) v[j] = (R)(gm[(size_t)j * n + i] * (R(1.0) / R(3.0)));
  v[10] = (R)ipdamp[i];
  v[11] = (R)thole[i];
  v[12] = v[13] = v[14] = v[15] = R(0);
  R *o = rec + (size_t)i * kRecStride;
#pragma unroll
  for (int j = 0; j < 16; j++) o[j] = v[j];
}

template <typename R>
__device__ __forceinline__ void k_pack_induced(VGrid vg, int n, const double *__restrict__ uD, const double *__restrict__ uP, R *rec,
                               double *grad, double *torque) {
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (grad) {   // the half-row real-space energy adds into these
    grad[i] = grad[n + i] = grad[2 * (size_t)n + i] = 0.0;
    torque[i] = torque[n + i] = torque[2 * (size_t)n + i] = 0.0;
  }
  R *o = rec + (size_t)i * kRecStride + kRecInduced;
  o[0] = (R)uD[i]; o[1] = (R)uD[n + i]; o[2] = (R)uD[2 * (size_t)n + i];
  o[3] = (R)uP[i]; o[4] = (R)uP[n + i]; o[5] = (R)uP[2 * (size_t)n + i];
  o[6] = o[7] = R(0);
}

// The largest double t with sqrt(t) < c.  sqrt is correctly rounded, hence monotone, so
// the preconditioner-cutoff test sqrt(r2) < c is exactly r2 <= t.
static double below_sqrt(double c) {
  if (!(c > 0.0)) return -1.0;
  double t = c * c;
  while (std::sqrt(t) >= c) t = std::nextafter(t, 0.0);
  while (std::sqrt(std::nextafter(t, INFINITY)) < c) t = std::nextafter(t, INFINITY);
  return t;
}

template <typename R>
static void realspace_field(Handle &h) {
  using V2 = typename Vec2<R>::type;
  const double off2 = h.vacuum ? INFINITY : h.prm.ewald_cutoff * h.prm.ewald_cutoff;
  launch_on<k_pack_mpole<R>, 0, 0>(h.rec, nblocks(h.n, 256), 256, 0, h.stream, h.n, (const double *)h.d_gm,
                                   (const double *)h.d_ipdamp, (const double *)h.d_thole,
                                   reinterpret_cast<R *>(h.d_erec));
  FFX_LAUNCHED(h);
  launch_on<k_realspace_field<R>, 128, sizeof(R) == 4 ? 8 : 1>(
      h.rec, nblocks((int64_t)h.n * 32, 128), 128, 0, h.stream, h.n, (const double *)h.d_x, (const double *)h.d_y,
      (const double *)h.d_z, h.box, (const double *)h.d_gm, (const double *)h.d_ipdamp, (const double *)h.d_thole,
      (const int *)h.d_nbr, (const int *)h.d_nbr_cnt, h.cap_nbr, (const int *)h.d_nbr_sh, off2,
      below_sqrt(h.prm.precond_cutoff), h.d_ewl, h.d_ewl_cnt, h.cap_ewl, h.d_ewl_sh, h.d_prl, h.d_prl_cnt, h.cap_prl,
      reinterpret_cast<PairRec<R> *>(h.d_coefE), reinterpret_cast<R *>(h.d_coefEB),
      reinterpret_cast<PairRec<R> *>(h.d_coefP), reinterpret_cast<R *>(h.d_coefPB), excl(h),
      ewald_coef(h, ewald_alpha_of(h)), h.scales, h.d_fieldD, h.d_fieldP, h.d_flags, (const double2 *)h.d_pos,
      reinterpret_cast<const R *>(h.d_erec), (const int *)(h.near_list ? h.d_nbl : nullptr), (const int *)h.d_nbl_cnt,
      h.cap_nbl);
  FFX_LAUNCHED(h);
}

template <typename R>
static void direct_dipoles(Handle &h) {
  launch_on<k_direct_dipoles<R>, 0, 0>(h.rec, nblocks(h.n, 256), 256, 0, h.stream, h.n, (const double *)h.d_gm,
                                       (const double *)h.d_cphi, (const double *)h.d_polar,
                                       ewald_coef(h, ewald_alpha_of(h)).aewald3, h.d_fieldD, h.d_fieldP, h.d_uD,
                                       h.d_uP, h.d_udirD, h.d_udirP, reinterpret_cast<R *>(h.d_recF));
  FFX_LAUNCHED(h);
}

void launch_direct_dipoles(Handle &h) {
  if (h.prm.polarization == FFXG_POLAR_NONE) return;
  if (h.mixed) direct_dipoles<float>(h); else direct_dipoles<double>(h);
}

void launch_realspace_field(Handle &h) {
  if (h.mixed)
    realspace_field<float>(h);
  else
    realspace_field<double>(h);
}



template <typename R>
static void real_energy(Handle &h, bool grad) {
  const bool direct = h.prm.polarization == FFXG_POLAR_DIRECT;
  const bool half = !h.step.lam && !direct;   // k_real_energy's HALF form
  launch_on<k_pack_induced<R>, 0, 0>(h.rec, nblocks(h.n, 256), 256, 0, h.stream, h.n, (const double *)h.d_uD,
                                     (const double *)h.d_uP, reinterpret_cast<R *>(h.d_erec),
                                     half && grad ? h.d_grad : (double *)nullptr, h.d_torque);
  FFX_LAUNCHED(h);
  // One system: the resident blocks only (FP32 form FFX_REAL_ENERGY_MIN_BLOCKS per SM;
  // FP64 form two, its 255 registers a thread), the warps striding over the atoms: no
  // tail of late blocks (FP32 700 -> 707, FP64 463 -> 469 evals/s).  A batch keeps one
  // warp per atom, each system's blocks a range of the batch grid.
  const int full = nblocks((int64_t)h.n * 32, 128);
  const int grid = h.rec ? full : std::min(full, (sizeof(R) == 4 ? FFX_REAL_ENERGY_MIN_BLOCKS : 2) * h.num_sms);
  auto go = [&](auto body) {
    launch_on<decltype(body)::value, 128, sizeof(R) == 4 ? FFX_REAL_ENERGY_MIN_BLOCKS : 1>(
        h.rec, grid, 128, 0, h.stream, h.n, (const double *)h.d_x, (const double *)h.d_y,
        (const double *)h.d_z, h.box, (const double *)h.d_gm, (const double *)h.d_uD, (const double *)h.d_uP,
        (const double *)h.d_ipdamp, (const double *)h.d_thole, (const int *)h.d_ewl, (const int *)h.d_ewl_cnt,
        h.cap_ewl, (const int *)h.d_ewl_sh, excl(h), ewald_coef(h, ewald_alpha_of(h)), h.scales, h.prm.polarization,
        grad ? 1 : 0, h.d_eatom + 1 * (size_t)h.n, h.d_eatom + 2 * (size_t)h.n, h.d_catom + (size_t)h.n, h.d_grad,
        h.d_torque, (const int *)h.d_soft, h.step, h.d_eatom + 9 * (size_t)h.n, h.d_eatom + 10 * (size_t)h.n, h.d_lg,
        h.d_lt, (const double2 *)h.d_pos, reinterpret_cast<const R *>(h.d_erec), h.d_flags);
  };
  if (h.step.lam) {
    if (direct) go(BodyOf<k_real_energy<R, true, true>>{});
    else go(BodyOf<k_real_energy<R, true, false>>{});
  } else {
    if (direct) go(BodyOf<k_real_energy<R, false, true>>{});
    else go(BodyOf<k_real_energy<R, false, false>>{});
  }
  FFX_LAUNCHED(h);
}

// ---------------------------------------------------------------------------
// Parameter gradients of the last evaluation: dE/dM of each atom's local-frame multipole
// (stored components) and dE/dalpha of its polarizability (Thole damping fixed).
// dE_perm/dM_i is the potential of all other multipoles at i (bilinear energy); with
// E_pol = -1/2 electric E_d^T A^-1 E_p and A symmetric, the CR dipoles u_P = A^-1 E_p are
// the adjoint solution: dE_pol/dM = -1/2 electric (F_d^T u_P + F_p^T u_D), and
// dE_pol/dalpha_i = -1/2 electric alpha_i^-2 u_D,i . u_P,i.  FP64 in both forms.

// d e_pair/d M_t for the source multipole (ck, dk, qk = Q/3) at r = x_s - x_t and radial
// coefficients b[0..4]: the derivative of permanentPair's gl sums
// (RealSpaceEnergyRegion.java:1190-1290).  Accumulated into acc with weight wgt.
__device__ __forceinline__ void quad_acc(const double G[3][3], double wgt, double *acc) {
  acc[4] += wgt * G[0][0] / 3.0; acc[5] += wgt * G[1][1] / 3.0; acc[6] += wgt * G[2][2] / 3.0;
  acc[7] += wgt * (G[0][1] + G[1][0]) / 3.0;
  acc[8] += wgt * (G[0][2] + G[2][0]) / 3.0;
  acc[9] += wgt * (G[1][2] + G[2][1]) / 3.0;
}

__device__ __forceinline__ void pair_pot_acc(double ck, const double *dk, const double qk[3][3], const double *r,
                                             const double *b, double wgt, double *acc) {
  double qkr[3];
  for (int a = 0; a < 3; a++) qkr[a] = qk[a][0] * r[0] + qk[a][1] * r[1] + qk[a][2] * r[2];
  const double sc4 = dk[0] * r[0] + dk[1] * r[1] + dk[2] * r[2];
  const double sc6 = qkr[0] * r[0] + qkr[1] * r[1] + qkr[2] * r[2];
  acc[0] += wgt * (ck * b[0] - sc4 * b[1] + sc6 * b[2]);
  const double cd = ck * b[1] - sc4 * b[2] + sc6 * b[3];
  for (int a = 0; a < 3; a++) acc[1 + a] += wgt * (cd * r[a] + b[1] * dk[a] - 2.0 * b[2] * qkr[a]);
  double G[3][3];
  for (int a = 0; a < 3; a++)
    for (int c = 0; c < 3; c++)
      G[a][c] = (ck * r[a] * r[c] + 2.0 * dk[a] * r[c] + 2.0 * qk[a][c]) * b[2] +
                (-sc4 * r[a] * r[c] - 4.0 * qkr[a] * r[c]) * b[3] + sc6 * r[a] * r[c] * b[4];
  quad_acc(G, wgt, acc);
}

// d (u . E(M_t))/d M_t for a dipole u at r = x_u - x_t, field coefficients b1..b3
// (PermanentFieldRegion.java:703-760).
__device__ __forceinline__ void dip_pot_acc(const double *u, const double *r, double b1, double b2, double b3,
                                            double wgt, double *acc) {
  const double ur = u[0] * r[0] + u[1] * r[1] + u[2] * r[2];
  acc[0] += wgt * ur * b1;
  for (int a = 0; a < 3; a++) acc[1 + a] += wgt * (ur * b2 * r[a] - b1 * u[a]);
  double G[3][3];
  for (int a = 0; a < 3; a++)
    for (int c = 0; c < 3; c++) G[a][c] = ur * b3 * r[a] * r[c] - 2.0 * b2 * u[a] * r[c];
  quad_acc(G, wgt, acc);
}

// One warp per atom over its Ewald row: the real-space parts of dE/dM_i (global frame)
// into phi[10][n].
__global__ void __launch_bounds__(128) k_param_real(
    int n, const double *__restrict__ x, const double *__restrict__ y, const double *__restrict__ z, Box bx,
    const double *__restrict__ gm, const double *__restrict__ uD, const double *__restrict__ uP,
    const double *__restrict__ ipdamp, const double *__restrict__ thole, const int *__restrict__ ewl,
    const int *__restrict__ ewl_cnt, int capE, const int *__restrict__ ewl_sh, Excl ex, EwaldCoef ec,
    const __grid_constant__ ScaleTables c_scales, int pol, double *phi) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int i = warp;
  const double xi = x[i], yi = y[i], zi = z[i];
  const double pdi = ipdamp[i], pti = thole[i];
  const double electric = ec.electric;
  double acc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  const int cnt = min(ewl_cnt[i], capE);
  const int *row = ewl + (size_t)i * capE;
  for (int a = lane; a < cnt; a += 32) {
    const int k = row[a];
    const size_t ent = (size_t)i * capE + a;
    double xr = __dsub_rn(x[k], xi), yr = __dsub_rn(y[k], yi), zr = __dsub_rn(z[k], zi);
    const double r2 = pair_image(xr, yr, zr, bx, ewl_sh, ent, 1.0);
    const unsigned code = pair_primary(ewl_sh, ent) ? excl_code(i, k, ex.ptr, ex.k, ex.code, ex.lo, ex.hi) : 0u;
    const double sm = c_scales.m[code & 7u], sp = c_scales.p[(code >> 3) & 7u], sd = c_scales.d[(code >> 6) & 1u];
    const double r = sqrt(r2);
    const double ralpha = ec.aewald * r, exp2a = exp(-ralpha * ralpha);
    const double rr1 = 1.0 / r, rr2 = rr1 * rr1;
    const double bn0 = erfc(ralpha) * rr1;
    const double bn1 = (bn0 + ec.an0 * exp2a) * rr2, bn2 = (3.0 * bn1 + ec.an1 * exp2a) * rr2;
    const double bn3 = (5.0 * bn2 + ec.an2 * exp2a) * rr2, bn4 = (7.0 * bn3 + ec.an3 * exp2a) * rr2;
    const double rr3 = rr1 * rr2, rr5 = 3.0 * rr3 * rr2, rr7 = 5.0 * rr5 * rr2, rr9 = 7.0 * rr7 * rr2;
    const double rv[3] = {xr, yr, zr};
    const double ck = gm[t000 * n + k];
    const double dk[3] = {gm[t100 * n + k], gm[t010 * n + k], gm[t001 * n + k]};
    double qk[3][3];
    qk[0][0] = gm[t200 * n + k] / 3.0; qk[1][1] = gm[t020 * n + k] / 3.0; qk[2][2] = gm[t002 * n + k] / 3.0;
    qk[0][1] = qk[1][0] = gm[t110 * n + k] / 3.0;
    qk[0][2] = qk[2][0] = gm[t101 * n + k] / 3.0;
    qk[1][2] = qk[2][1] = gm[t011 * n + k] / 3.0;
    const double bE[5] = {bn0, bn1, bn2, bn3, bn4}, bR[5] = {rr1, rr3, rr5, rr7, rr9};
    pair_pot_acc(ck, dk, qk, rv, bE, electric, acc);
    pair_pot_acc(ck, dk, qk, rv, bR, -electric * (1.0 - sm), acc);
    if (!pol) continue;
    double scale3 = 1.0, scale5 = 1.0, scale7 = 1.0;
    double damp = pdi * ipdamp[k];
    const double tho = fmin(pti, thole[k]);
    const double rdamp = r * damp;
    damp = -tho * rdamp * rdamp * rdamp;
    if (damp > -50.0) {
      const double expdamp = exp(damp);
      scale3 = 1.0 - expdamp;
      scale5 = 1.0 - expdamp * (1.0 - damp);
      scale7 = 1.0 - expdamp * (1.0 - damp + 0.6 * damp * damp);
    }
    const double up[3] = {uP[k], uP[n + k], uP[2 * n + k]}, ud[3] = {uD[k], uD[n + k], uD[2 * n + k]};
    const double hw = -0.5 * electric;
    dip_pot_acc(up, rv, bn1 - (1.0 - scale3 * sd) * rr3, bn2 - (1.0 - scale5 * sd) * rr5,
                bn3 - (1.0 - scale7 * sd) * rr7, hw, acc);
    dip_pot_acc(ud, rv, bn1 - (1.0 - scale3 * sp) * rr3, bn2 - (1.0 - scale5 * sp) * rr5,
                bn3 - (1.0 - scale7 * sp) * rr7, hw, acc);
  }
#pragma unroll
  for (int t = 0; t < 10; t++) acc[t] = warp_sum(acc[t]);
  if (lane == 0)
    for (int t = 0; t < 10; t++) phi[(size_t)t * n + i] = acc[t];
}

struct ParamConst {
  double electric, aewald1, aewald2, aewald3, dcorr;
  int pol;
};

// Reciprocal, self and charge-correction parts, then the local frame (d = R d_l,
// Q = R Q_l R^T) and dE/dalpha; out[n][10], outA[n].
__global__ void k_param_finish(int n, const double *__restrict__ phi, const double *__restrict__ gm,
                               const double *__restrict__ cphi, const double *__restrict__ cphiI,
                               const double *__restrict__ cphiP, const double *__restrict__ uD,
                               const double *__restrict__ uP, const double *__restrict__ polar,
                               const double *__restrict__ rot, ParamConst pc, double *out, double *outA) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double w[10] = {1.0, 1.0, 1.0, 1.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0};
  double f[10], m[10];
  for (int t = 0; t < 10; t++) {
    m[t] = gm[(size_t)t * n + i];
    f[t] = phi[(size_t)t * n + i] + pc.electric * w[t] * cphi[(size_t)t * n + i];
  }
  f[0] += 2.0 * pc.aewald1 * m[0] + pc.dcorr;
  for (int a = 1; a < 4; a++) f[a] += pc.aewald1 * pc.aewald2 * 2.0 * m[a] / 3.0;
  for (int a = 4; a < 7; a++) f[a] += pc.aewald1 * pc.aewald2 * 2.0 * pc.aewald2 * 2.0 * m[a] / 45.0;
  for (int a = 7; a < 10; a++) f[a] += pc.aewald1 * pc.aewald2 * 2.0 * pc.aewald2 * 4.0 * m[a] / 45.0;
  double dA = 0.0;
  if (pc.pol) {
    const double h = -0.5 * pc.electric;
    for (int t = 0; t < 10; t++) f[t] -= h * w[t] * (cphiP[(size_t)t * n + i] + cphiI[(size_t)t * n + i]);
    double ud = 0.0;
    for (int a = 0; a < 3; a++) {
      const double pa = uP[(size_t)a * n + i], da = uD[(size_t)a * n + i];
      f[1 + a] += h * pc.aewald3 * (pa + da);
      ud += da * pa;
    }
    const double al = polar[i];
    if (al > 0.0) dA = h * ud / (al * al);
  }
  double R[3][3];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) R[a][b] = rot[(size_t)(3 * a + b) * n + i];
  double *o = out + 10 * (size_t)i;
  o[0] = f[0];
  for (int b = 0; b < 3; b++) o[1 + b] = R[0][b] * f[1] + R[1][b] * f[2] + R[2][b] * f[3];
  double G[3][3];
  G[0][0] = f[4]; G[1][1] = f[5]; G[2][2] = f[6];
  G[0][1] = G[1][0] = 0.5 * f[7]; G[0][2] = G[2][0] = 0.5 * f[8]; G[1][2] = G[2][1] = 0.5 * f[9];
  double L[3][3];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) {
      double v = 0.0;
      for (int c = 0; c < 3; c++)
        for (int d = 0; d < 3; d++) v += R[c][a] * G[c][d] * R[d][b];
      L[a][b] = v;
    }
  o[4] = L[0][0]; o[5] = L[1][1]; o[6] = L[2][2];
  o[7] = 2.0 * L[0][1]; o[8] = 2.0 * L[0][2]; o[9] = 2.0 * L[1][2];
  outA[i] = dA;
}

// dE/dM [n][10] (device) and dE/dalpha [n] (device) of the last evaluation's state.
int param_gradients(Handle &h, double *d_dM, double *d_dA) {
  const size_t N = h.n;
  double *scratch = nullptr;
  if (cudaMallocAsync(&scratch, 10 * N * sizeof(double), h.stream) != cudaSuccess) return FFXG_ERR_CUDA;
  const bool pol = h.prm.polarization != FFXG_POLAR_NONE;
  k_param_real<<<nblocks((int64_t)h.n * 32, 128), 128, 0, h.stream>>>(
      h.n, h.d_x, h.d_y, h.d_z, h.box, h.d_gm, h.d_uD, h.d_uP, h.d_ipdamp, h.d_thole, h.d_ewl, h.d_ewl_cnt,
      h.cap_ewl, h.d_ewl_sh, excl(h), ewald_coef(h, ewald_alpha_of(h)), h.scales, pol ? 1 : 0, scratch);
  ParamConst pc{};
  const double SQRT_PI = 1.7724538509055160273, PI = 3.14159265358979323846;
  const double a = ewald_alpha_of(h);
  pc.electric = h.prm.electric;
  pc.aewald1 = -pc.electric * a / SQRT_PI;
  pc.aewald2 = 2.0 * a * a;
  pc.aewald3 = 4.0 / 3.0 * a * a * a / SQRT_PI;
  double q = 0.0;
  for (size_t i = 0; i < N; i++) q += h.sys.multipole[10 * i];
  pc.dcorr = (q != 0.0 && a > 0.0) ? -pc.electric * PI * q / (h.box.volume * a * a) : 0.0;
  pc.pol = pol ? 1 : 0;
  k_param_finish<<<nblocks(h.n, 128), 128, 0, h.stream>>>(h.n, scratch, h.d_gm, h.d_cphi, h.d_cphiI, h.d_cphiP,
                                                          h.d_uD, h.d_uP, h.d_polar, h.d_rot, pc, d_dM, d_dA);
  cudaFreeAsync(scratch, h.stream);
  h.launches += 2;
  return cudaGetLastError() == cudaSuccess ? FFXG_OK : FFXG_ERR_CUDA;
}

void launch_real_energy(Handle &h, bool grad) {
  if (h.mixed)
    real_energy<float>(h, grad);
  else
    real_energy<double>(h, grad);
}

}  // namespace ffx
