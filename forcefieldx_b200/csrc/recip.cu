// recip.cu -- reciprocal-space energy/gradient, torque to gradient, assembly, reductions.
//
//  k_recip_energy   PermanentReciprocalEnergyLoop and InducedDipoleReciprocalEnergyLoop
//                   (pme/ReciprocalEnergyRegion.java:381-543, 545-740)
//  k_torque_gather  Torque.torque (pme/Torque.java:111-316) applied by ReduceRegion.TorqueLoop
//                   (pme/ReduceRegion.java:184-248), written as a gather: atom j collects the
//                   frame-atom forces of every atom whose frame it defines.
//  k_assemble       ForceFieldEnergy.fillGradient (ForceFieldEnergy.java:2848): vdW + PME.
//  k_sum_*          deterministic two-level sums of the per-atom energies and counts.
#include <algorithm>

#include "ffx_internal.cuh"

namespace ffx {

enum { t000 = 0, t100, t010, t001, t200, t020, t002, t110, t101, t011,
       t300, t030, t003, t210, t201, t120, t021, t102, t012, t111 };


struct RecipCoef {
  double electric, aewald1, aewald2, aw3, aw4;
  int nf[3];
  int polarization;
};

__device__ __forceinline__ void k_recip_energy(VGrid vg, int n, const double *__restrict__ gm, const double *__restrict__ fm,
                               const double *__restrict__ cphi, const double *__restrict__ fphi,
                               const double *__restrict__ uD, const double *__restrict__ uP,
                               const double *__restrict__ cphiI, const double *__restrict__ cphiP,
                               const double *__restrict__ fphiI, const double *__restrict__ fphiP, const RecipCoef &rc,
                               const PmeConst &pc, int gradient, double *eatom, double *grad, double *torque, const ElecStep &st,
                               double *lgrad, double *ltorque) {
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double mp[10], f[10];
#pragma unroll
  for (int j = 0; j < 10; j++) { mp[j] = gm[j * n + i]; f[j] = fm[j * n + i]; }
  double ph[10];
#pragma unroll
  for (int j = 0; j < 10; j++) ph[j] = cphi[j * n + i];
  const double cii = mp[t000] * mp[t000];
  const double dii = mp[t100] * mp[t100] + mp[t010] * mp[t010] + mp[t001] * mp[t001];
  const double qii = mp[t200] * mp[t200] + mp[t020] * mp[t020] + mp[t002] * mp[t002] +
                     2.0 * (mp[t110] * mp[t110] + mp[t101] * mp[t101] + mp[t011] * mp[t011]);
  const double eSelf = rc.aewald1 * (cii + rc.aewald2 * (dii / 3.0 + 2.0 * rc.aewald2 * qii / 45.0));
  const double e = mp[t000] * ph[t000] + mp[t100] * ph[t100] + mp[t010] * ph[t010] + mp[t001] * ph[t001] +
                   (1.0 / 3.0) * (mp[t200] * ph[t200] + mp[t020] * ph[t020] + mp[t002] * ph[t002] +
                                  2.0 * (mp[t110] * ph[t110] + mp[t101] * ph[t101] + mp[t011] * ph[t011]));
  // Lambda scheme (ReciprocalEnergyRegion.java:230-255, 385-530, 545-740): permanent parts x
  // permScale, induced parts x polScale; dU/dL takes dEdLSign * dlPow * the unscaled parts.
  const double sP = st.permScale, sI = st.polScale;
  const double eRecip = 0.5 * rc.electric * e;
  eatom[3 * (size_t)n + i] = sP * eSelf;
  eatom[4 * (size_t)n + i] = sP * eRecip;
  double gx = 0, gy = 0, gz = 0, tqx = 0, tqy = 0, tqz = 0;
  if (gradient) {
    double fp[20];
#pragma unroll
    for (int t = 0; t < 20; t++) fp[t] = fphi[t * n + i];
    double ax = f[t000] * fp[t100] + f[t100] * fp[t200] + f[t010] * fp[t110] + f[t001] * fp[t101] +
                f[t200] * fp[t300] + f[t020] * fp[t120] + f[t002] * fp[t102] + f[t110] * fp[t210] +
                f[t101] * fp[t201] + f[t011] * fp[t111];
    double ay = f[t000] * fp[t010] + f[t100] * fp[t110] + f[t010] * fp[t020] + f[t001] * fp[t011] +
                f[t200] * fp[t210] + f[t020] * fp[t030] + f[t002] * fp[t012] + f[t110] * fp[t120] +
                f[t101] * fp[t111] + f[t011] * fp[t021];
    double az = f[t000] * fp[t001] + f[t100] * fp[t101] + f[t010] * fp[t011] + f[t001] * fp[t002] +
                f[t200] * fp[t201] + f[t020] * fp[t021] + f[t002] * fp[t003] + f[t110] * fp[t111] +
                f[t101] * fp[t102] + f[t011] * fp[t012];
    ax *= rc.nf[0]; ay *= rc.nf[1]; az *= rc.nf[2];
    gx = rc.electric * (pc.recip[0][0] * ax + pc.recip[0][1] * ay + pc.recip[0][2] * az);
    gy = rc.electric * (pc.recip[1][0] * ax + pc.recip[1][1] * ay + pc.recip[1][2] * az);
    gz = rc.electric * (pc.recip[2][0] * ax + pc.recip[2][1] * ay + pc.recip[2][2] * az);
    double tx = -mp[t010] * ph[t001] + mp[t001] * ph[t010];
    double ty = -mp[t001] * ph[t100] + mp[t100] * ph[t001];
    double tz = -mp[t100] * ph[t010] + mp[t010] * ph[t100];
    tx -= (2.0 / 3.0) * (mp[t110] * ph[t101] + mp[t020] * ph[t011] + mp[t011] * ph[t002] - mp[t101] * ph[t110] -
                         mp[t011] * ph[t020] - mp[t002] * ph[t011]);
    ty -= (2.0 / 3.0) * (mp[t101] * ph[t200] + mp[t011] * ph[t110] + mp[t002] * ph[t101] - mp[t200] * ph[t101] -
                         mp[t110] * ph[t011] - mp[t101] * ph[t002]);
    tz -= (2.0 / 3.0) * (mp[t200] * ph[t110] + mp[t110] * ph[t020] + mp[t101] * ph[t011] - mp[t110] * ph[t200] -
                         mp[t020] * ph[t110] - mp[t011] * ph[t101]);
    tqx = rc.electric * tx; tqy = rc.electric * ty; tqz = rc.electric * tz;
  }
  const double gPx = gx, gPy = gy, gPz = gz, tPx = tqx, tPy = tqy, tPz = tqz;
  gx = gy = gz = tqx = tqy = tqz = 0.0;
  double eSelfI = 0.0, eRecipI = 0.0;
  if (rc.polarization != FFXG_POLAR_NONE) {
    const double u0 = uD[i], u1 = uD[n + i], u2 = uD[2 * n + i];
    const double p0 = uP[i], p1 = uP[n + i], p2 = uP[2 * n + i];
    eSelfI = rc.aw3 * (u0 * mp[t100] + u1 * mp[t010] + u2 * mp[t001]);
    double fi[3], fiCR[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      fi[a] = pc.afrac[a][0] * u0 + pc.afrac[a][1] * u1 + pc.afrac[a][2] * u2;
      fiCR[a] = pc.afrac[a][0] * p0 + pc.afrac[a][1] * p1 + pc.afrac[a][2] * p2;
    }
    const double fP100 = fphi[t100 * n + i], fP010 = fphi[t010 * n + i], fP001 = fphi[t001 * n + i];
    eRecipI = 0.5 * rc.electric * (fi[0] * fP100 + fi[1] * fP010 + fi[2] * fP001);
    if (gradient) {
      const double uix = 0.5 * (u0 + p0), uiy = 0.5 * (u1 + p1), uiz = 0.5 * (u2 + p2);
      tqx += rc.aw4 * (mp[t010] * uiz - mp[t001] * uiy);
      tqy += rc.aw4 * (mp[t001] * uix - mp[t100] * uiz);
      tqz += rc.aw4 * (mp[t100] * uiy - mp[t010] * uix);
      double fP[20], fI[20], fC[20], sPhi[10], sfPhi[20];
#pragma unroll
      for (int t = 0; t < 20; t++) {
        fP[t] = fphi[t * n + i];
        fI[t] = fphiI[t * n + i];
        fC[t] = fphiP[t * n + i];
        sfPhi[t] = fI[t] + fC[t];
      }
#pragma unroll
      for (int t = 0; t < 10; t++) sPhi[t] = 0.5 * (cphiI[t * n + i] + cphiP[t * n + i]);
      const double indx = fi[0], indy = fi[1], indz = fi[2];
      const double inpx = fiCR[0], inpy = fiCR[1], inpz = fiCR[2];
      const double insx = indx + inpx, insy = indy + inpy, insz = indz + inpz;
      double ax = insx * fP[t200] + insy * fP[t110] + insz * fP[t101];
      double ay = insx * fP[t110] + insy * fP[t020] + insz * fP[t011];
      double az = insx * fP[t101] + insy * fP[t011] + insz * fP[t002];
      if (rc.polarization == FFXG_POLAR_MUTUAL) {
        ax += indx * fC[t200] + inpx * fI[t200] + indy * fC[t110] + inpy * fI[t110] + indz * fC[t101] + inpz * fI[t101];
        ay += indx * fC[t110] + inpx * fI[t110] + indy * fC[t020] + inpy * fI[t020] + indz * fC[t011] + inpz * fI[t011];
        az += indx * fC[t101] + inpx * fI[t101] + indy * fC[t011] + inpy * fI[t011] + indz * fC[t002] + inpz * fI[t002];
      }
      ax += f[t000] * sfPhi[t100] + f[t100] * sfPhi[t200] + f[t010] * sfPhi[t110] + f[t001] * sfPhi[t101] +
            f[t200] * sfPhi[t300] + f[t020] * sfPhi[t120] + f[t002] * sfPhi[t102] + f[t110] * sfPhi[t210] +
            f[t101] * sfPhi[t201] + f[t011] * sfPhi[t111];
      ay += f[t000] * sfPhi[t010] + f[t100] * sfPhi[t110] + f[t010] * sfPhi[t020] + f[t001] * sfPhi[t011] +
            f[t200] * sfPhi[t210] + f[t020] * sfPhi[t030] + f[t002] * sfPhi[t012] + f[t110] * sfPhi[t120] +
            f[t101] * sfPhi[t111] + f[t011] * sfPhi[t021];
      az += f[t000] * sfPhi[t001] + f[t100] * sfPhi[t101] + f[t010] * sfPhi[t011] + f[t001] * sfPhi[t002] +
            f[t200] * sfPhi[t201] + f[t020] * sfPhi[t021] + f[t002] * sfPhi[t003] + f[t110] * sfPhi[t111] +
            f[t101] * sfPhi[t102] + f[t011] * sfPhi[t012];
      ax *= rc.nf[0]; ay *= rc.nf[1]; az *= rc.nf[2];
      const double h = 0.5 * rc.electric;
      gx += h * (pc.recip[0][0] * ax + pc.recip[0][1] * ay + pc.recip[0][2] * az);
      gy += h * (pc.recip[1][0] * ax + pc.recip[1][1] * ay + pc.recip[1][2] * az);
      gz += h * (pc.recip[2][0] * ax + pc.recip[2][1] * ay + pc.recip[2][2] * az);
      double tx = -mp[t010] * sPhi[t001] + mp[t001] * sPhi[t010];
      double ty = -mp[t001] * sPhi[t100] + mp[t100] * sPhi[t001];
      double tz = -mp[t100] * sPhi[t010] + mp[t010] * sPhi[t100];
      tx -= (2.0 / 3.0) * (mp[t110] * sPhi[t101] + mp[t020] * sPhi[t011] + mp[t011] * sPhi[t002] -
                           mp[t101] * sPhi[t110] - mp[t011] * sPhi[t020] - mp[t002] * sPhi[t011]);
      ty -= (2.0 / 3.0) * (mp[t101] * sPhi[t200] + mp[t011] * sPhi[t110] + mp[t002] * sPhi[t101] -
                           mp[t200] * sPhi[t101] - mp[t110] * sPhi[t011] - mp[t101] * sPhi[t002]);
      tz -= (2.0 / 3.0) * (mp[t200] * sPhi[t110] + mp[t110] * sPhi[t020] + mp[t101] * sPhi[t011] -
                           mp[t110] * sPhi[t200] - mp[t020] * sPhi[t110] - mp[t011] * sPhi[t101]);
      tqx += rc.electric * tx; tqy += rc.electric * ty; tqz += rc.electric * tz;
    }
  }
  eatom[5 * (size_t)n + i] = sI * eSelfI;
  eatom[6 * (size_t)n + i] = sI * eRecipI;
  if (gradient) {
    grad[i] += sP * gPx + sI * gx; grad[n + i] += sP * gPy + sI * gy; grad[2 * n + i] += sP * gPz + sI * gz;
    torque[i] += sP * tPx + sI * tqx; torque[n + i] += sP * tPy + sI * tqy; torque[2 * n + i] += sP * tPz + sI * tqz;
  }
  if (st.lam) {   // adds to the rows and arrays k_real_energy<R, true> wrote
    const double lP = st.dEdLSign * st.dlPowPerm, l2P = st.dEdLSign * st.d2lPowPerm;
    const double lI = st.dEdLSign * st.dlPowPol, l2I = st.dEdLSign * st.d2lPowPol;
    eatom[9 * (size_t)n + i] += lP * (eSelf + eRecip) + lI * (eSelfI + eRecipI);
    eatom[10 * (size_t)n + i] += l2P * (eSelf + eRecip) + l2I * (eSelfI + eRecipI);
    lgrad[i] += lP * gPx + lI * gx; lgrad[n + i] += lP * gPy + lI * gy; lgrad[2 * n + i] += lP * gPz + lI * gz;
    ltorque[i] += lP * tPx + lI * tqx; ltorque[n + i] += lP * tPy + lI * tqy;
    ltorque[2 * n + i] += lP * tPz + lI * tqz;
  }
}

// ---------------------------------------------------------------------------
__device__ __forceinline__ void cross3(const double *a, const double *b, double *c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
__device__ __forceinline__ double len3(const double *v) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
__device__ __forceinline__ void nrm3(double *v) {
  const double l = len3(v);
  v[0] /= l; v[1] /= l; v[2] /= l;
}

// Cartesian force on frame slot `slot` (0 = z, 1 = x, 2 = y, 3 = the atom) from atom i's torque.
__device__ __forceinline__ void torque_slot(int i, int slot, int n, const double *__restrict__ x, const double *__restrict__ y,
                            const double *__restrict__ z, const int *__restrict__ frame, const int *__restrict__ axis,
                            const double *trq, double *out) {
  out[0] = out[1] = out[2] = 0.0;
  const int fr = frame[i];
  if (fr == FFXG_FRAME_NONE) return;
  const int iz = axis[i], ix = axis[n + i], iy = axis[2 * n + i];
  const double o[3] = {x[i], y[i], z[i]};
  double vZ[3] = {x[iz] - o[0], y[iz] - o[1], z[iz] - o[2]};
  const double rZ = len3(vZ);
  double vX[3], vY[3];
  if (fr != FFXG_FRAME_ZONLY) {
    vX[0] = x[ix] - o[0]; vX[1] = y[ix] - o[1]; vX[2] = z[ix] - o[2];
  } else {
    vX[0] = 1.0; vX[1] = 0.0; vX[2] = 0.0;
    if (fabs(vZ[0] / rZ) > 0.866) { vX[0] = 0.0; vX[1] = 1.0; }
  }
  const double rX = len3(vX);
  if (fr == FFXG_FRAME_ZTHENBISECTOR || fr == FFXG_FRAME_THREEFOLD) {
    vY[0] = x[iy] - o[0]; vY[1] = y[iy] - o[1]; vY[2] = z[iy] - o[2];
  } else {
    cross3(vZ, vX, vY);
  }
  const double rY = len3(vY);
  for (int d = 0; d < 3; d++) { vZ[d] *= 1.0 / rZ; vX[d] *= 1.0 / rX; vY[d] *= 1.0 / rY; }
  double xXZ[3], xYZ[3], xYX[3];
  cross3(vX, vZ, xXZ); cross3(vY, vZ, xYZ); cross3(vY, vX, xYX);
  nrm3(xXZ); nrm3(xYZ); nrm3(xYX);
  const double cosZX = dot3(vZ, vX);
  const double sinZX = sqrt(1.0 - cosZX * cosZX);
  const double dPhidZ = -(trq[0] * vZ[0] + trq[1] * vZ[1] + trq[2] * vZ[2]);
  const double dPhidX = -(trq[0] * vX[0] + trq[1] * vX[1] + trq[2] * vX[2]);
  const double dPhidY = -(trq[0] * vY[0] + trq[1] * vY[1] + trq[2] * vY[2]);
  double g[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  if (fr == FFXG_FRAME_ZONLY) {
    for (int j = 0; j < 3; j++) {
      const double dZ = xXZ[j] * dPhidX / (rZ * sinZX) + xYZ[j] * dPhidY / rZ;
      g[0][j] = dZ; g[3][j] = -dZ;
    }
  } else if (fr == FFXG_FRAME_ZTHENX) {
    for (int j = 0; j < 3; j++) {
      const double dZ = xXZ[j] * dPhidX / (rZ * sinZX) + xYZ[j] * dPhidY / rZ;
      const double dX = -xXZ[j] * dPhidZ / (rX * sinZX);
      g[0][j] = dZ; g[1][j] = dX; g[3][j] = -(dZ + dX);
    }
  } else if (fr == FFXG_FRAME_BISECTOR) {
    for (int j = 0; j < 3; j++) {
      const double dZ = xXZ[j] * dPhidX / (rZ * sinZX) + 0.5 * xYZ[j] * dPhidY / rZ;
      const double dX = -xXZ[j] * dPhidZ / (rX * sinZX) + 0.5 * xYX[j] * dPhidY / rX;
      g[0][j] = dZ; g[1][j] = dX; g[3][j] = -(dZ + dX);
    }
  } else if (fr == FFXG_FRAME_ZTHENBISECTOR) {
    double sumXY[3] = {vX[0] + vY[0], vX[1] + vY[1], vX[2] + vY[2]};
    double xZXY[3], xXYZ[3], xxZXYZ[3], t1[3], t2[3];
    cross3(vZ, sumXY, xZXY);
    nrm3(sumXY); nrm3(xZXY);
    cross3(sumXY, vZ, xXYZ);
    cross3(xZXY, vZ, xxZXYZ);
    nrm3(xXYZ); nrm3(xxZXYZ);
    const double cosZXY = dot3(vZ, sumXY), sinZXY = sqrt(1.0 - cosZXY * cosZXY);
    const double cosXZXY = dot3(vX, xZXY), sinXZXY = sqrt(1.0 - cosXZXY * cosXZXY);
    const double cosYZXY = dot3(vY, xZXY), sinYZXY = sqrt(1.0 - cosYZXY * cosYZXY);
    for (int d = 0; d < 3; d++) { t1[d] = vX[d] + xZXY[d] * -cosXZXY; t2[d] = vY[d] + xZXY[d] * -cosYZXY; }
    nrm3(t1); nrm3(t2);
    const double ut1cos = dot3(vZ, t1), ut1sin = sqrt(1.0 - ut1cos * ut1cos);
    const double ut2cos = dot3(vZ, t2), ut2sin = sqrt(1.0 - ut2cos * ut2cos);
    const double dPhidR = -(trq[0] * sumXY[0] + trq[1] * sumXY[1] + trq[2] * sumXY[2]);
    const double dPhidZXY = -(trq[0] * xZXY[0] + trq[1] * xZXY[1] + trq[2] * xZXY[2]);
    for (int j = 0; j < 3; j++) {
      const double dZ = xXYZ[j] * dPhidR / (rZ * sinZXY) + xxZXYZ[j] * dPhidZXY / rZ;
      const double dX = (sinXZXY * xZXY[j] - cosXZXY * t1[j]) * dPhidZ / (rX * (ut1sin + ut2sin));
      const double dY = (sinYZXY * xZXY[j] - cosYZXY * t2[j]) * dPhidZ / (rY * (ut1sin + ut2sin));
      g[0][j] = dZ; g[1][j] = dX; g[2][j] = dY; g[3][j] = -(dZ + dX + dY);
    }
  } else if (fr == FFXG_FRAME_THREEFOLD) {
    double s[3] = {(vZ[0] + vX[0]) + vY[0], (vZ[1] + vX[1]) + vY[1], (vZ[2] + vX[2]) + vY[2]};
    const double rZXY = len3(s);
    for (int d = 0; d < 3; d++) s[d] *= 1.0 / rZXY;
    const double cosYSum = dot3(vY, s), cosZSum = dot3(vZ, s), cosXSum = dot3(vX, s);
    const double *va[3] = {vZ, vX, vY};
    const double ra[3] = {rZ, rX, rY};
    const double cs[3] = {cosZSum, cosXSum, cosYSum};
#pragma unroll
    for (int q = 0; q < 3; q++) {
      // q = 0: r = x + y about z; q = 1: r = z + y about x; q = 2: r = z + x about y
      const double *a1 = (q == 0) ? vX : vZ;
      const double *a2 = (q == 2) ? vX : vY;
      double rr[3] = {a1[0] + a2[0], a1[1] + a2[1], a1[2] + a2[2]}, del[3], eps[3];
      nrm3(rr);
      const double cosR = dot3(rr, va[q]), sinR = sqrt(1.0 - cosR * cosR);
      const double dPhidR = -trq[0] * rr[0] - trq[1] * rr[1] - trq[2] * rr[2];
      cross3(rr, va[q], del);
      nrm3(del);
      const double dPhidDel = -trq[0] * del[0] - trq[1] * del[1] - trq[2] * del[2];
      cross3(del, va[q], eps);
      const int slotq = (q == 0) ? 0 : ((q == 1) ? 1 : 2);
      for (int j = 0; j < 3; j++) {
        const double d = del[j] * dPhidR / (ra[q] * sinR) + eps[j] * dPhidDel * cs[q] / (ra[q] * rZXY);
        g[slotq][j] = d;
        g[3][j] -= d;
      }
    }
  }
  // Select the slot with compares so that g stays in registers (a runtime index would put
  // it in local memory).
#pragma unroll
  for (int j = 0; j < 3; j++) out[j] = (slot == 0) ? g[0][j] : (slot == 1) ? g[1][j] : (slot == 2) ? g[2][j] : g[3][j];
}

__device__ __forceinline__ void k_torque_gather(VGrid vg, int n, const double *__restrict__ x, const double *__restrict__ y,
                                const double *__restrict__ z, const int *__restrict__ frame,
                                const int *__restrict__ axis, const double *__restrict__ torque,
                                const int *__restrict__ tq_ptr, const int *__restrict__ tq_ent, double *gtq,
                                int *flags, int quant) {
  const int j = vg.bid * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double s0 = 0, s1 = 0, s2 = 0;
  for (int e = tq_ptr[j]; e < tq_ptr[j + 1]; e++) {
    const int ent = tq_ent[e];
    const int i = ent >> 2, slot = ent & 3;
    const double trq[3] = {torque[i], torque[n + i], torque[2 * n + i]};
    // The mixed form's accumulated torques (fixed-point sums) must stay in their exact range.
    if (quant && slot == 3 && (quant_out(trq[0]) || quant_out(trq[1]) || quant_out(trq[2])))
      atomicOr(flags, FLAG_QUANT_RANGE);
    double g[3];
    torque_slot(i, slot, n, x, y, z, frame, axis, trq, g);
    s0 += g[0]; s1 += g[1]; s2 += g[2];
  }
  if (!isfinite(s0) || !isfinite(s1) || !isfinite(s2)) atomicOr(flags, FLAG_NONFINITE);
  gtq[j] = s0; gtq[n + j] = s1; gtq[2 * n + j] = s2;
}

__device__ __forceinline__ void k_assemble(VGrid vg, int n, const double *__restrict__ grad, const double *__restrict__ gtq,
                           const double *__restrict__ gvdw, double *out, int *flags, int quant) {
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int d = 0; d < 3; d++) {
    const double ge = grad[d * n + i];
    if (quant && quant_out(ge)) atomicOr(flags, FLAG_QUANT_RANGE);   // mixed form: fixed-point sums
    const double v = ge + gtq[d * n + i] + gvdw[d * n + i];
    if (!isfinite(v)) atomicOr(flags, FLAG_NONFINITE);
    out[3 * i + d] = v;
  }
}

// Two-level deterministic sums: blocks reduce contiguous chunks in a fixed order.
constexpr int kSumBlocks = 148;
constexpr int kNE = kEnergyRows, kNC = 2;   // energy rows (kEnergyRows), count rows

__device__ __forceinline__ void k_sum_partial(VGrid vg, int n, const double *__restrict__ eatom, const long long *__restrict__ catom,
                              double *pe, long long *pc) {
  __shared__ double se[kNE][256];
  __shared__ long long sc[kNC][256];
  const int chunk = (n + vg.nblk - 1) / vg.nblk;
  const int s = vg.bid * chunk, e = min(n, s + chunk);
  double acc[kNE] = {0};
  long long cc[kNC] = {0};
  for (int i = s + threadIdx.x; i < e; i += blockDim.x) {
    for (int t = 0; t < kNE; t++) acc[t] += eatom[(size_t)t * n + i];
    for (int t = 0; t < kNC; t++) cc[t] += catom[(size_t)t * n + i];
  }
  for (int t = 0; t < kNE; t++) se[t][threadIdx.x] = acc[t];
  for (int t = 0; t < kNC; t++) sc[t][threadIdx.x] = cc[t];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      for (int t = 0; t < kNE; t++) se[t][threadIdx.x] += se[t][threadIdx.x + w];
      for (int t = 0; t < kNC; t++) sc[t][threadIdx.x] += sc[t][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int t = 0; t < kNE; t++) pe[vg.bid * kNE + t] = se[t][0];
    for (int t = 0; t < kNC; t++) pc[vg.bid * kNC + t] = sc[t][0];
  }
}

// Row t of the totals by warp t: lane l sums blocks l, l + 32, ..., then a fixed shuffle
// tree (the same order on every call).
__device__ __forceinline__ void k_sum_final(VGrid vg, int nb, const double *__restrict__ pe, const long long *__restrict__ pc, double *out,
                            long long *cout) {
  const int lane = threadIdx.x & 31, row = threadIdx.x >> 5;
  if (row < kNE) {
    double s = 0.0;
    for (int b = lane; b < nb; b += 32) s += pe[b * kNE + row];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[row] = s;
  } else if (row < kNE + kNC) {
    const int t = row - kNE;
    long long s = 0;
    for (int b = lane; b < nb; b += 32) s += pc[b * kNC + t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) cout[t] = s;
  }
}

// ---------------------------------------------------------------------------

void launch_recip_energy(Handle &h, bool grad) {
  const double SQRT_PI = 1.7724538509055160273;
  RecipCoef rc{};
  const double a = h.prm.ewald_alpha;
  rc.electric = h.prm.electric;
  rc.aewald1 = -rc.electric * a / SQRT_PI;
  rc.aewald2 = 2.0 * a * a;
  rc.aw3 = -2.0 / 3.0 * rc.electric * a * a * a / SQRT_PI;
  rc.aw4 = -2.0 * rc.aw3;
  rc.nf[0] = h.nfft[0]; rc.nf[1] = h.nfft[1]; rc.nf[2] = h.nfft[2];
  rc.polarization = h.step.doPol ? h.prm.polarization : FFXG_POLAR_NONE;
  if (h.vacuum) return;   // no reciprocal space and no Ewald self terms (alpha 0)
  launch_on<k_recip_energy, 0, 0>(h.rec, nblocks(h.n, 128), 128, 0, h.stream, h.n, (const double *)h.d_gm,
                                   (const double *)h.d_fm, (const double *)h.d_cphi, (const double *)h.d_fphi,
                                   (const double *)h.d_uD, (const double *)h.d_uP, (const double *)h.d_cphiI,
                                   (const double *)h.d_cphiP, (const double *)h.d_fphiI, (const double *)h.d_fphiP, rc,
                                   h.pc, (grad || h.step.lam) ? 1 : 0, h.d_eatom, h.d_grad, h.d_torque, h.step, h.d_lg,
                                   h.d_lt);
  FFX_LAUNCHED(h);
}

void launch_torque(Handle &h) { launch_torque_of(h, h.d_torque, h.d_vec); }

// Torque -> Cartesian gradient of `torque` into out[3][n] (written, not added).
void launch_torque_of(Handle &h, const double *torque, double *out) {
  launch_on<k_torque_gather, 0, 0>(h.rec, nblocks(h.n, 128), 128, 0, h.stream, h.n, (const double *)h.d_x,
                                    (const double *)h.d_y, (const double *)h.d_z, (const int *)h.d_frame,
                                    (const int *)h.d_axis, torque, (const int *)h.d_tq_ptr, (const int *)h.d_tq_ent,
                                    out, h.d_flags, h.mixed && torque == h.d_torque ? 1 : 0);
  FFX_LAUNCHED(h);
}

void launch_assemble(Handle &h, double *d_grad_xyz) {
  launch_on<k_assemble, 0, 0>(h.rec, nblocks(h.n, 256), 256, 0, h.stream, h.n, (const double *)h.d_grad,
                              (const double *)h.d_vec, (const double *)(h.d_gred + 3 * (size_t)h.n), d_grad_xyz,
                              h.d_flags, h.mixed ? 1 : 0);
  FFX_LAUNCHED(h);
}

// ---------------------------------------------------------------------------
// Electrostatic lambda: the steps' results summed in d_acc, rows [0,3) gradient, [3,6)
// torque, [6,14) energy rows 1-6, 9, 10, [14,17) lambda gradient, [17,20) lambda torque.
__device__ __constant__ int kAccRows[8] = {1, 2, 3, 4, 5, 6, 9, 10};

__device__ __forceinline__ void k_elec_accumulate(VGrid vg, int n, int first, const double *__restrict__ grad, const double *__restrict__ torque,
                                  const double *__restrict__ eatom, const double *__restrict__ lg,
                                  const double *__restrict__ lt, double *acc) {
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v[20];
  for (int d = 0; d < 3; d++) {
    v[d] = grad[d * n + i];
    v[3 + d] = torque[d * n + i];
    v[14 + d] = lg[d * n + i];
    v[17 + d] = lt[d * n + i];
  }
  for (int r = 0; r < 8; r++) v[6 + r] = eatom[(size_t)kAccRows[r] * n + i];
  for (int r = 0; r < 20; r++) acc[(size_t)r * n + i] = first ? v[r] : acc[(size_t)r * n + i] + v[r];
}

__device__ __forceinline__ void k_elec_restore(VGrid vg, int n, const double *__restrict__ acc, double *grad, double *torque, double *eatom,
                               double *lg, double *lt) {
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int d = 0; d < 3; d++) {
    grad[d * n + i] = acc[(size_t)d * n + i];
    torque[d * n + i] = acc[(size_t)(3 + d) * n + i];
    lg[d * n + i] = acc[(size_t)(14 + d) * n + i];
    lt[d * n + i] = acc[(size_t)(17 + d) * n + i];
  }
  for (int r = 0; r < 8; r++) eatom[(size_t)kAccRows[r] * n + i] = acc[(size_t)(6 + r) * n + i];
}

// out[3][n] += lg + the torque-derived part of the lambda gradient.
__device__ __forceinline__ void k_lambda_grad_add(VGrid vg, int n, const double *__restrict__ lg, const double *__restrict__ lgtq, double *out) {
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int d = 0; d < 3; d++) out[d * n + i] += lg[d * n + i] + lgtq[d * n + i];
}

// Zero the global and fractional multipoles of the soft atoms (the condensed step without
// them: an atom with no multipoles and no polarizability takes no part).
__device__ __forceinline__ void k_zero_soft_multipoles(VGrid vg, int n, const int *__restrict__ soft, double *gm, double *fm) {
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n || !soft[i]) return;
  for (int t = 0; t < 10; t++) { gm[(size_t)t * n + i] = 0.0; fm[(size_t)t * n + i] = 0.0; }
}

void launch_elec_accumulate(Handle &h, bool first) {
  launch_on<k_elec_accumulate, 0, 0>(h.rec, nblocks(h.n, 256), 256, 0, h.stream, h.n, first ? 1 : 0,
                                     (const double *)h.d_grad, (const double *)h.d_torque, (const double *)h.d_eatom,
                                     (const double *)h.d_lg, (const double *)h.d_lt, h.d_acc);
  FFX_LAUNCHED(h);
}

void launch_elec_restore(Handle &h) {
  launch_on<k_elec_restore, 0, 0>(h.rec, nblocks(h.n, 256), 256, 0, h.stream, h.n, (const double *)h.d_acc, h.d_grad,
                                  h.d_torque, h.d_eatom, h.d_lg, h.d_lt);
  FFX_LAUNCHED(h);
}

void launch_lambda_grad_add(Handle &h, double *out) {
  // The torque-derived part goes through d_vec's scratch rows, like launch_torque.
  launch_torque_of(h, h.d_lt, h.d_vec);
  launch_on<k_lambda_grad_add, 0, 0>(h.rec, nblocks(h.n, 256), 256, 0, h.stream, h.n, (const double *)h.d_lg,
                                     (const double *)h.d_vec, out);
  FFX_LAUNCHED(h);
}

void launch_zero_soft_multipoles(Handle &h) {
  launch_on<k_zero_soft_multipoles, 0, 0>(h.rec, nblocks(h.n, 256), 256, 0, h.stream, h.n, (const int *)h.d_soft,
                                          h.d_gm, h.d_fm);
  FFX_LAUNCHED(h);
}

void launch_reduce_results(Handle &h) {
  double *pe = h.d_partials;
  long long *pc = reinterpret_cast<long long *>(h.d_partials + kSumBlocks * kNE);
  const int nb = std::min(kSumBlocks, std::max(1, (h.n + 255) / 256));   // fewer blocks for small systems
  launch_on<k_sum_partial, 0, 0>(h.rec, nb, 256, 0, h.stream, h.n, (const double *)h.d_eatom,
                                 (const long long *)h.d_catom, pe, pc);
  launch_on<k_sum_final, 0, 0>(h.rec, 1, 32 * (kNE + kNC), 0, h.stream, nb, (const double *)pe,
                               (const long long *)pc, h.d_result, h.d_cresult);
  h.launches += 2;
}

}  // namespace ffx
