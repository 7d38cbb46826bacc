// vdw.cu -- buffered 14-7 van der Waals on the hydrogen-reduced coordinates.
//
// VanDerWaalsLoop (VanDerWaals.java:1602-1850) with the Halgren constants
// (VanDerWaalsForm.java:313-334; delta 0.07, gamma 0.12), the multiplicative taper
// from vdw-taper * cutoff to the cutoff (MultiplicativeSwitch.java:84-124, 234-236) and
// the 1-2/1-3/1-4 masks (VanDerWaals.applyMask, :412-428).  A warp owns an atom i and
// scans its buffered row in both directions (a partner's reduced position and type from
// one 32-byte record); entries inside the cutoff go to a per-warp queue in shared memory
// and are evaluated 32 at a time.  The force on i's reduced site accumulates in
// registers; k_vdw_distribute then splits every reduced-site force between the hydrogen
// and its heavy atom (VanDerWaals.java:1786-1797) as a gather.
#include <algorithm>

#include "ffx_internal.cuh"

namespace ffx {


struct VdwForm {
  double off2, cut2, t1n, gamma1, delta, gamma;
  double c0, c1, c2, c3, c4, c5;
  double cut, iwidth;   // taper start and 1 / (cutoff - taper start)
};

__device__ __forceinline__ unsigned vexcl_code(int i, int k, const int *__restrict__ ptr, const int *__restrict__ ek,
                                               const unsigned *__restrict__ code, const int *__restrict__ lo,
                                               const int *__restrict__ hi) {
  if (k < lo[i] || k > hi[i]) return 0u;
  const int e1 = ptr[i + 1];
  for (int e = ptr[i]; e < e1; e++)
    if (ek[e] == k) return code[e];
  return 0u;
}

// ALCH: the softcore variant (launched only while soft atoms are set).
template <typename R, bool ALCH>
__device__ __forceinline__ void k_vdw(
    VGrid vg, int const &n, const double *__restrict__ const &rx, const double *__restrict__ const &ry,
    const double *__restrict__ const &rz, const Box &bx, const int *__restrict__ const &vtype, int const &ntypes,
    const double *__restrict__ const &vrad, const double *__restrict__ const &veps,
    const int *__restrict__ const &nbr, const int *__restrict__ const &nbr_cnt, int const &cap,
    const int *__restrict__ const &nbr_sh, const int *__restrict__ const &eptr,
    const int *__restrict__ const &ek, const unsigned *__restrict__ const &ecode,
    const int *__restrict__ const &elo, const int *__restrict__ const &ehi, const VdwForm &vf,
    const ScaleTables &c_vscales, int const &gradient, double * const &eatom, long long * const &catom,
    double * const &gred, const int *__restrict__ const &soft, const int *__restrict__ const &mol,
    const AlchConst &al, double * const &edl, double * const &ed2l, double * const &lgred,
    const double2 *__restrict__ const &rpos) {
  struct Queue { R x[64], y[64], z[64], r[64], m[64]; int k[64], t[64], f[64]; };
  __shared__ Queue qbuf[8];
  const int warp = (vg.bid * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nwarps = (vg.nblk * blockDim.x) >> 5;
  for (int i = warp; i < n; i += nwarps) {
    const double xi = rx[i], yi = ry[i], zi = rz[i];
    const int ti = vtype[i];
    const R delta = vf.delta, gamma = vf.gamma, gamma1 = vf.gamma1, t1n = vf.t1n;
    const R c0 = vf.c0, c1 = vf.c1, c2 = vf.c2, c3 = vf.c3, c4 = vf.c4, c5 = vf.c5;
    const R cut = vf.cut, iwidth = vf.iwidth;
    double e = 0.0, dl = 0.0, d2l = 0.0;
    R gx = 0, gy = 0, gz = 0, lx = 0, ly = 0, lz = 0;
    long long cnt = 0;
    const int soft_i = ALCH ? soft[i] : 0;
    const int mol_i = ALCH ? mol[i] : 0;
    const int m = min(nbr_cnt[i], cap);
    const int *row = nbr + (size_t)i * cap;
    // Entries inside the cutoff (with a non-zero mask) are queued in shared memory and
    // evaluated 32 at a time, so the pair arithmetic runs on full warps instead of on the
    // ~55% of lanes whose entry lies inside 9 A of an 11 A row.
    R *qx = qbuf[wib].x, *qy = qbuf[wib].y, *qz = qbuf[wib].z, *qr = qbuf[wib].r, *qm = qbuf[wib].m;
    int *qk = qbuf[wib].k, *qt = qbuf[wib].t, *qf = qbuf[wib].f;
    auto pair_math = [&](int k, int tk, int qflags, R dx, R dy, R dz, R r2, R mask) {
      const bool tap = (qflags & 1) != 0, counted = (qflags & 2) != 0;
      const R irv = vrad[ti * ntypes + tk];
        const R r = m_sqrt(r2);
        // Softcore pair (VanDerWaals.java:1728-1761): exactly one atom soft, or both soft under
        // the intermolecular / intramolecular softcore options.
        bool spair = false;
        if (ALCH) {
          const int sk = soft[k];
          spair = (soft_i != sk);
          if (soft_i && sk) {
            const bool same = (mol_i == mol[k]);
            if (al.inter && !same) spair = true;
            else if (al.intra && same) spair = true;
          }
        }
        // The energy and gradient arithmetic with its roundings fixed (xmul / xadd / xfma),
        // so that a system's vdW term is the same bits alone and in a batch.
        const R alpha = spair ? (R)al.sc1 : R(0);
        const R lambda5 = spair ? (R)al.sc2 : R(1);
        const R ev = xmul(mask, veps[ti * ntypes + tk]);
        const R eps_lambda = xmul(ev, lambda5);
        const R rho = xmul(r, irv);
        const R rho2 = xmul(rho, rho);
        const R rhoDisp1 = xmul(xmul(rho2, rho2), rho2);
        const R rhoDisp = xmul(rhoDisp1, rho);
        const R rd = xadd(rho, delta), rd2 = xmul(rd, rd);
        const R rhoDelta1 = xmul(xmul(rd2, rd2), rd2);
        const R rhoDelta = xmul(rhoDelta1, rd);
        const R t1d = R(1.0) / xadd(alpha, rhoDelta);
        const R t2d = R(1.0) / xadd(xadd(alpha, rhoDisp), gamma);
        const R t1 = xmul(t1n, t1d);
        const R t2a = xmul(gamma1, t2d);
        const R t2 = xadd(t2a, R(-2.0));
        const R eik = xmul(xmul(eps_lambda, t1), t2);
        R taper = R(1.0), dtaper = R(0.0);
        if (tap) {
          if (sizeof(R) == 8) {
            // The polynomial summed left to right, as the reference sums its terms.
            const R r3 = xmul(r2, r), r4 = xmul(r2, r2), r5 = xmul(r2, r3);
            taper = xadd(xfma(c1, r, xfma(c2, r2, xfma(c3, r3, xfma(c4, r4, xmul(c5, r5))))), c0);
            dtaper = xadd(xfma(R(2.0) * c2, r, xfma(R(3.0) * c3, r2, xfma(R(4.0) * c4, r3, xmul(R(5.0) * c5, r4)))),
                          c1);
          } else {
            // The same quintic in t = (r - cut) / (off - cut): 1 - 10 t^3 + 15 t^4 - 6 t^5.
            // The power form above cancels ~1e6-sized terms and is unusable in FP32.
            const R t = xmul(xadd(r, -cut), iwidth), t2 = xmul(t, t);
            taper = xfma(xmul(t2, t), xfma(t, xfma(R(-6), t, R(15)), R(-10)), R(1));
            dtaper = xmul(xmul(t2, xfma(t, xfma(R(-30), t, R(60)), R(-30))), iwidth);
          }
        }
        e += xmul(xmul(R(0.5), eik), taper);
        if (counted) cnt++;
        if (gradient || (ALCH && spair)) {
          const R dt1d_dr = xmul(xmul(R(7.0), rhoDelta1), irv);
          const R dt2d_dr = xmul(xmul(R(7.0), rhoDisp1), irv);
          const R dt1_dr = xmul(xmul(t1, dt1d_dr), t1d);
          const R dt2_dr = xmul(xmul(t2a, dt2d_dr), t2d);
          const R dedr = -xmul(eps_lambda, xfma(dt1_dr, t2, xmul(t1, dt2_dr)));
          const R ir = R(1.0) / r;
          if (gradient) {
            const R dsw = xfma(eik, dtaper, xmul(dedr, taper));
            gx = xfma(xmul(dsw, dx), ir, gx);
            gy = xfma(xmul(dsw, dy), ir, gy);
            gz = xfma(xmul(dsw, dz), ir, gz);
          }
          if (ALCH && spair) {
            // dU/dL, d2U/dL2 and dU/dX dL of the softcore pair (VanDerWaals.java:1842-1880); each
            // direction of the full list carries half of the pair's lambda derivatives.
            const R dsc1 = (R)al.dsc1dL, d2sc1 = (R)al.d2sc1dL2, sc2 = (R)al.sc2, dsc2 = (R)al.dsc2dL;
            const R d2sc2 = (R)al.d2sc2dL2;
            const R dt1 = -t1 * t1d * dsc1;
            const R dt2 = -t2a * t2d * dsc1;
            const R dedl = ev * (dsc2 * t1 * t2 + sc2 * dt1 * t2 + sc2 * t1 * dt2);
            dl += 0.5 * (double)(dedl * taper);
            const R t1d2 = -dsc1 * t1d * t1d;
            const R t2d2 = -dsc1 * t2d * t2d;
            const R d2t1 = -dt1 * t1d * dsc1 - t1 * t1d * d2sc1 - t1 * t1d2 * dsc1;
            const R d2t2 = -dt2 * t2d * dsc1 - t2a * t2d * d2sc1 - t2a * t2d2 * dsc1;
            const R df1 = d2sc2 * t1 * t2 + dsc2 * dt1 * t2 + dsc2 * t1 * dt2;
            const R df2 = dsc2 * dt1 * t2 + sc2 * d2t1 * t2 + sc2 * dt1 * dt2;
            const R df3 = dsc2 * t1 * dt2 + sc2 * dt1 * dt2 + sc2 * t1 * d2t2;
            d2l += 0.5 * (double)(ev * (df1 + df2 + df3) * taper);
            if (gradient) {
              const R t11 = -dsc2 * t2 * dt1_dr;
              const R t21 = -dsc2 * t1 * dt2_dr;
              const R t13 = R(2.0) * sc2 * t2 * dt1_dr * dsc1 * t1d;
              const R t23 = R(2.0) * sc2 * t1 * dt2_dr * dsc1 * t2d;
              const R t12 = -sc2 * dt2 * dt1_dr;
              const R t22 = -sc2 * dt1 * dt2_dr;
              const R dedldr = ev * (t11 + t12 + t13 + t21 + t22 + t23);
              const R lsw = dedl * dtaper + dedldr * taper;
              lx += lsw * dx * ir; ly += lsw * dy * ir; lz += lsw * dz * ir;
            }
          }
        }
    };
    int qn = 0;
    for (int base = 0; base < m; base += 32) {
      const int a = base + lane;
      bool pass = false;
      int k = 0, tk = 0, qflags = 0;
      R dx = 0, dy = 0, dz = 0, r2 = 0, mask = 0;
      if (a < m) {
        k = row[a];
        const size_t ent = (size_t)i * cap + a;
        double pk[4];
        ldg_32b(reinterpret_cast<const double *>(rpos + 2 * (size_t)k), pk);
        double dxd = __dsub_rn(xi, pk[0]), dyd = __dsub_rn(yi, pk[1]), dzd = __dsub_rn(zi, pk[2]);
        const double r2d = pair_image(dxd, dyd, dzd, bx, nbr_sh, ent, -1.0);
        tk = (int)__double_as_longlong(pk[3]);
        const R irv = vrad[ti * ntypes + tk];
        if (r2d <= vf.off2 && irv > R(0.0)) {
          const unsigned code = pair_primary(nbr_sh, ent) ? vexcl_code(i, k, eptr, ek, ecode, elo, ehi) : 0u;
          mask = c_vscales.v[(code >> 7) & 3u];
          pass = mask > R(0.0);
          dx = (R)dxd; dy = (R)dyd; dz = (R)dzd; r2 = (R)r2d;
          qflags = (r2d > vf.cut2 ? 1 : 0) | (pair_counted(i, k, nbr_sh, ent) ? 2 : 0);
        }
      }
      const unsigned bal = __ballot_sync(0xffffffffu, pass);
      if (pass) {
        const int q = qn + __popc(bal & ((1u << lane) - 1u));
        qk[q] = k; qt[q] = tk; qf[q] = qflags; qx[q] = dx; qy[q] = dy; qz[q] = dz; qr[q] = r2; qm[q] = mask;
      }
      qn += __popc(bal);
      __syncwarp();
      if (qn >= 32) {
        pair_math(qk[lane], qt[lane], qf[lane], qx[lane], qy[lane], qz[lane], qr[lane], qm[lane]);
        __syncwarp();
        if (lane < qn - 32) {
          const int q = lane + 32;
          qk[lane] = qk[q]; qt[lane] = qt[q]; qf[lane] = qf[q]; qx[lane] = qx[q]; qy[lane] = qy[q];
          qz[lane] = qz[q]; qr[lane] = qr[q]; qm[lane] = qm[q];
        }
        __syncwarp();
        qn -= 32;
      }
    }
    if (lane < qn) pair_math(qk[lane], qt[lane], qf[lane], qx[lane], qy[lane], qz[lane], qr[lane], qm[lane]);
    e = warp_sum(e);
    const double Gx = warp_sum((double)gx), Gy = warp_sum((double)gy), Gz = warp_sum((double)gz);
  #pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (ALCH) {
      dl = warp_sum(dl);
      d2l = warp_sum(d2l);
    }
    double Lx = 0.0, Ly = 0.0, Lz = 0.0;
    if (ALCH && gradient) {
      Lx = warp_sum((double)lx); Ly = warp_sum((double)ly); Lz = warp_sum((double)lz);
    }
    if (lane == 0) {
      eatom[i] = e;
      catom[i] = cnt;
      edl[i] = dl;
      ed2l[i] = d2l;
      if (gradient) { gred[i] = Gx; gred[n + i] = Gy; gred[2 * n + i] = Gz; }
      if (ALCH && gradient) { lgred[i] = Lx; lgred[n + i] = Ly; lgred[2 * n + i] = Lz; }
    }
  }
}

// g[j] = red_j * G[j] (reduced hydrogen) or G[j] (heavy / unreduced) + sum over the
// hydrogens c reduced toward j of (1 - red_c) * G[c].
__device__ __forceinline__ void k_vdw_distribute(VGrid vg, int n, const double *__restrict__ gred, const int *__restrict__ redp,
                                 const double *__restrict__ redf, const int *__restrict__ cptr,
                                 const int *__restrict__ child, double *gvdw) {
  const int j = vg.bid * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const double w = (redp[j] != j) ? redf[j] : 1.0 - redf[j];
  double s0 = w * gred[j], s1 = w * gred[n + j], s2 = w * gred[2 * n + j];
  for (int e = cptr[j]; e < cptr[j + 1]; e++) {
    const int c = child[e];
    const double wc = 1.0 - redf[c];
    s0 += wc * gred[c]; s1 += wc * gred[n + c]; s2 += wc * gred[2 * n + c];
  }
  gvdw[j] = s0; gvdw[n + j] = s1; gvdw[2 * n + j] = s2;
}


// One vdW launch.  The batch instance is held to four resident blocks of 256 threads in
// the FP32 form (64 registers, as the single-system instance uses).
template <typename R, bool ALCH>
static void vdw_launch(Handle &h, bool grad, cudaStream_t st, const VdwForm &vf, int blocks) {
  launch_on<k_vdw<R, ALCH>, 256, 0, sizeof(R) == 4 ? 4 : 0>(
      h.rec, blocks, 256, 0, st, h.n, (const double *)h.d_rx, (const double *)h.d_ry, (const double *)h.d_rz, h.box,
      (const int *)h.d_vtype, h.ntypes, (const double *)h.d_vrad, (const double *)h.d_veps, (const int *)h.d_nbr,
      (const int *)h.d_nbr_cnt, h.cap_nbr, (const int *)h.d_nbr_sh, (const int *)h.d_excl_ptr,
      (const int *)h.d_excl_k, (const unsigned *)h.d_excl_code, (const int *)h.d_excl_lo, (const int *)h.d_excl_hi,
      vf, h.scales, grad ? 1 : 0, h.d_eatom, h.d_catom, h.d_gred, (const int *)h.d_soft, (const int *)h.d_mol, h.alch,
      h.d_eatom + 7 * (size_t)h.n, h.d_eatom + 8 * (size_t)h.n, h.d_lgred, (const double2 *)h.d_rpos);
}

void launch_vdw(Handle &h, bool grad, cudaStream_t st) {
  if (h.vacuum) return;   // a vacuum sub-system carries electrostatics only
  VdwForm vf{};
  const double off = h.prm.vdw_cutoff, cut = h.prm.vdw_taper * h.prm.vdw_cutoff;
  vf.off2 = off * off;
  vf.cut2 = cut * cut;
  vf.delta = 0.07;
  vf.gamma = 0.12;
  vf.t1n = pow(1.0 + vf.delta, 7.0);
  vf.gamma1 = 1.0 + vf.gamma;
  const double a = cut, b = off, a2 = a * a, b2 = b * b, den = pow(b - a, 5.0);
  vf.c0 = b * b2 * (b2 - 5.0 * a * b + 10.0 * a2) / den;
  vf.c1 = -30.0 * a2 * b2 / den;
  vf.c2 = 30.0 * b * a * (b + a) / den;
  vf.c3 = -10.0 * (a2 + 4.0 * a * b + b2) / den;
  vf.c4 = 15.0 * (a + b) / den;
  vf.c5 = -6.0 / den;
  vf.cut = cut;
  vf.iwidth = 1.0 / (off - cut);
  // In a captured evaluation vdW is a low-priority branch beside the permanent field and
  // the solver: one block of eight warps per SM, warps striding over atoms.  Its blocks
  // stay resident until the term is done, so a wider branch holds the registers the
  // other kernels need: at four blocks per SM (the whole register file) the permanent
  // field and reciprocal chain waited ~140 us for it on the 24k box; at one block per SM
  // it runs in the solver's idle issue slots (657-668 -> 696 evals/s; 128-thread blocks
  // or two per SM measured slower).
  const int full = nblocks((int64_t)h.n * 32, 256);
  const int blocks = h.capturing ? std::min(full, h.num_sms) : full;
  if (h.alch.active) {
    if (h.mixed) vdw_launch<float, true>(h, grad, st, vf, blocks);
    else vdw_launch<double, true>(h, grad, st, vf, blocks);
  } else {
    if (h.mixed) vdw_launch<float, false>(h, grad, st, vf, blocks);
    else vdw_launch<double, false>(h, grad, st, vf, blocks);
  }
  FFX_LAUNCHED(h);
  if (grad) {
    // Rows 3-5 of d_gred hold the distributed per-atom vdW gradient.
    launch_on<k_vdw_distribute, 0, 0>(h.rec, nblocks(h.n, 256), 256, 0, st, h.n, (const double *)h.d_gred,
                                      (const int *)h.d_redp, (const double *)h.d_redf, (const int *)h.d_red_ptr,
                                      (const int *)h.d_red_child, h.d_gred + 3 * (size_t)h.n);
    FFX_LAUNCHED(h);
    if (h.alch.active) {   // dU/dX dL rows 3-5 of d_lgred, distributed the same way
      launch_on<k_vdw_distribute, 0, 0>(h.rec, nblocks(h.n, 256), 256, 0, st, h.n, (const double *)h.d_lgred,
                                      (const int *)h.d_redp, (const double *)h.d_redf, (const int *)h.d_red_ptr,
                                      (const int *)h.d_red_child, h.d_lgred + 3 * (size_t)h.n);
      FFX_LAUNCHED(h);
    }
  }
}

}  // namespace ffx
