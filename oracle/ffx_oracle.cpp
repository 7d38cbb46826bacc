// ffx_oracle.cpp -- CPU FP64 restatement of Force Field X's AMOEBA energy/gradient path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the oracle the CUDA library is checked
// against and the CPU baseline it is timed beside.  Only tests/, the smoke check
// in __graft_entry__.py and bench.py's CPU-baseline leg may load it; the product
// (forcefieldx_b200/) never calls it.
//
// Every routine restates the reference Java loop it cites (paths relative to
// modules/ in the Force Field X tree):
//   potential/src/main/java/ffx/potential/...   (P/ below)
//   numerics/src/main/java/ffx/numerics/...     (N/ below)
//   crystal/src/main/java/ffx/crystal/...       (C/ below)
// It is compiled with -ffp-contract=off so that, like Java, a*b+c is never fused
// unless the reference writes Math.fma explicitly (ReciprocalSpace spreading and
// potential interpolation), where std::fma is used.
//
// Scope: P1 orthorhombic cells that hold the buffered cutoff sphere without
// replicates (nSymm = 1), mutual / direct / no polarization, PCG SCF.

#include "../include/ffxcuda.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kElecAngToDebye = 4.80321;    // Constants.ELEC_ANG_TO_DEBYE (utilities/.../Constants.java:196)
constexpr double kSqrtPi = 1.7724538509055160273;
constexpr double kPi = 3.14159265358979323846;

enum { t000 = 0, t100, t010, t001, t200, t020, t002, t110, t101, t011,
       t300, t030, t003, t210, t201, t120, t021, t102, t012, t111 };

// ---------------------------------------------------------------------------
// C/Crystal.java:1069-1083 minimum image by the fractional round trip.
struct Cell {
  double a, b, c, volume;
  double A00, A10, A20, A11, A21, A22;        // A = (A^-1)^-1, columns = reciprocal vectors
  double Ai00, Ai10, Ai20, Ai11, Ai21, Ai22;  // A^-1 rows = lattice vectors
  double A[3][3];
  bool ortho = true;                          // all angles 90: A and A^-1 diagonal
  double width[3];                            // perpendicular widths 1 / |a*_d|
};

inline double jsignum(double v) { return v > 0.0 ? 1.0 : (v < 0.0 ? -1.0 : v); }

inline double image(double &x, double &y, double &z, const Cell &c) {
  double xf = x * c.A00 + y * c.A10 + z * c.A20;
  double yf = y * c.A11 + z * c.A21;
  double zf = z * c.A22;
  xf = std::floor(std::fabs(xf) + 0.5) * jsignum(-xf) + xf;
  yf = std::floor(std::fabs(yf) + 0.5) * jsignum(-yf) + yf;
  zf = std::floor(std::fabs(zf) + 0.5) * jsignum(-zf) + zf;
  x = xf * c.Ai00 + yf * c.Ai10 + zf * c.Ai20;
  y = yf * c.Ai11 + zf * c.Ai21;
  z = zf * c.Ai22;
  return x * x + y * y + z * z;
}

// Crystal.updateCrystal (C/Crystal.java:1428-1548): the lattice vectors a = (a, 0, 0),
// b = (b cos g, b sin g, 0), c = (c cos b, c beta_term, c gamma_term) as the rows of A^-1,
// A its inverse (lower triangular, so inverted in closed form here) and the volume, by the
// orthorhombic, monoclinic (only beta differs from 90) and general branches.  Angles of 0
// read as 90.
Cell make_cell(const double box[3], const double angles[3]) {
  Cell c{};
  c.a = box[0]; c.b = box[1]; c.c = box[2];
  double ang[3];
  for (int d = 0; d < 3; d++) ang[d] = (angles && angles[d] > 0.0) ? angles[d] : 90.0;
  std::memset(c.A, 0, sizeof(c.A));
  if (ang[0] == 90.0 && ang[1] == 90.0 && ang[2] == 90.0) {
    c.volume = c.a * c.b * c.c;  // Crystal.java (orthorhombic branch)
    c.Ai00 = c.a; c.Ai10 = 0.0; c.Ai20 = 0.0; c.Ai11 = c.b; c.Ai21 = 0.0; c.Ai22 = c.c;
    // LU inverse of a diagonal matrix is the elementwise reciprocal.
    c.A00 = 1.0 / c.a; c.A10 = 0.0; c.A20 = 0.0; c.A11 = 1.0 / c.b; c.A21 = 0.0; c.A22 = 1.0 / c.c;
    c.A[0][0] = c.A00; c.A[1][1] = c.A11; c.A[2][2] = c.A22;
    c.ortho = true;
    c.width[0] = c.a; c.width[1] = c.b; c.width[2] = c.c;
    return c;
  }
  const double deg = 0.017453292519943295;   // Math.toRadians
  double cos_alpha, sin_beta, cos_beta, sin_gamma, cos_gamma, beta_term, gamma_term;
  if (ang[0] == 90.0 && ang[2] == 90.0) {    // monoclinic
    cos_alpha = 0.0;
    sin_beta = std::sin(ang[1] * deg);
    cos_beta = std::cos(ang[1] * deg);
    sin_gamma = 1.0;
    cos_gamma = 0.0;
    beta_term = 0.0;
    gamma_term = sin_beta;
    c.volume = sin_beta * c.a * c.b * c.c;
  } else {                                   // triclinic, hexagonal, trigonal
    cos_alpha = std::cos(ang[0] * deg);
    sin_beta = std::sin(ang[1] * deg);
    cos_beta = std::cos(ang[1] * deg);
    sin_gamma = std::sin(ang[2] * deg);
    cos_gamma = std::cos(ang[2] * deg);
    beta_term = (cos_alpha - cos_beta * cos_gamma) / sin_gamma;
    gamma_term = std::sqrt(sin_beta * sin_beta - beta_term * beta_term);
    c.volume = sin_gamma * gamma_term * c.a * c.b * c.c;
  }
  c.Ai00 = c.a;
  c.Ai10 = c.b * cos_gamma; c.Ai11 = c.b * sin_gamma;
  c.Ai20 = c.c * cos_beta; c.Ai21 = c.c * beta_term; c.Ai22 = c.c * gamma_term;
  c.A00 = 1.0 / c.Ai00;
  c.A11 = 1.0 / c.Ai11;
  c.A22 = 1.0 / c.Ai22;
  c.A10 = -c.Ai10 / (c.Ai00 * c.Ai11);
  c.A21 = -c.Ai21 / (c.Ai11 * c.Ai22);
  c.A20 = (c.Ai10 * c.Ai21 - c.Ai11 * c.Ai20) / (c.Ai00 * c.Ai11 * c.Ai22);
  c.A[0][0] = c.A00; c.A[1][0] = c.A10; c.A[1][1] = c.A11;
  c.A[2][0] = c.A20; c.A[2][1] = c.A21; c.A[2][2] = c.A22;
  c.ortho = false;
  c.width[0] = 1.0 / std::sqrt(c.A00 * c.A00 + c.A10 * c.A10 + c.A20 * c.A20);
  c.width[1] = 1.0 / std::sqrt(c.A11 * c.A11 + c.A21 * c.A21);
  c.width[2] = 1.0 / std::fabs(c.A22);
  return c;
}

// Fractional coordinates x A (Crystal.toFractionalCoordinates order).
inline void to_frac(double x, double y, double z, const Cell &c, double &fx, double &fy, double &fz) {
  if (c.ortho) { fx = x * c.A00; fy = y * c.A11; fz = z * c.A22; return; }
  fx = x * c.A00 + y * c.A10 + z * c.A20;
  fy = y * c.A11 + z * c.A21;
  fz = z * c.A22;
}

// The lattice translation n A^-1 added to a displacement (multi-image lists).
inline void add_shift(double &dx, double &dy, double &dz, int nx, int ny, int nz, double sign, const Cell &c) {
  if (c.ortho) {
    dx += sign * ((double)nx * c.a);
    dy += sign * ((double)ny * c.b);
    dz += sign * ((double)nz * c.c);
    return;
  }
  dx += sign * ((double)nx * c.Ai00 + (double)ny * c.Ai10 + (double)nz * c.Ai20);
  dy += sign * ((double)ny * c.Ai11 + (double)nz * c.Ai21);
  dz += sign * ((double)nz * c.Ai22);
}

// ---------------------------------------------------------------------------
// N/spline/UniformBSpline.java:74-183 (B-spline values and derivatives).
void bspline_recursion(double x, int order, const double *c, double *nc) {
  const double div = 1.0 / (double)order;
  const double k1mw = order + (1.0 - x);
  const int km1 = order - 1;
  nc[order] = div * x * c[km1];
  for (int i = 1; i < order; i++) {
    const int kmi = order - i;
    const int km1i = km1 - i;
    const double x1 = x + (double)i;
    const double k1mwi = k1mw - (double)i;
    nc[kmi] = div * (x1 * c[km1i] + k1mwi * c[kmi]);
  }
  nc[0] = div * (1.0 - x) * c[0];
}

void bspline_diff(double *c, int order) {
  const int order1 = order - 1;
  c[order] = c[order1];
  for (int i = order1; i > 0; i--) c[i] = c[i - 1] - c[i];
  c[0] = -c[0];
}

void bspline_coeffs(double x, int order, double *coeff) {  // UniformBSpline.bSpline
  double w[16] = {0};
  w[0] = 1.0 - x;
  w[1] = x;
  for (int k = 2; k < order; k++) {
    double t[16] = {0};
    bspline_recursion(x, k, w, t);
    std::memcpy(w, t, sizeof(w));
  }
  for (int k = 0; k < order; k++) coeff[k] = w[k];
}

// Order `order`, derivatives 0..min(3, order-1); out[k*4 + j] = d^j/dx^j of node k.
void bspline_derivs(double x, int order, double *out) {
  double work[8][8];
  std::memset(work, 0, sizeof(work));
  work[1][0] = 1.0 - x;
  work[1][1] = x;
  work[2][0] = 0.5 * (1.0 - x) * work[1][0];
  work[2][1] = 0.5 * ((x + 1.0) * work[1][0] + (2.0 - x) * work[1][1]);
  work[2][2] = 0.5 * x * work[1][1];
  for (int k = 3; k < order; k++) bspline_recursion(x, k, work[k - 1], work[k]);
  const int deriv = std::min(3, order - 1);
  const int o1 = order - 1, o2 = order - 2, o3 = order - 3, o4 = order - 4;
  if (deriv > 0) bspline_diff(work[o2], o1);
  if (deriv > 1) { bspline_diff(work[o3], o2); bspline_diff(work[o3], o1); }
  if (deriv > 2) { bspline_diff(work[o4], o3); bspline_diff(work[o4], o2); bspline_diff(work[o4], o1); }
  for (int k = 0; k < order; k++)
    for (int j = 0; j < 4; j++) out[k * 4 + j] = (j <= deriv) ? work[o1 - j][k] : 0.0;
}

// ---------------------------------------------------------------------------
// Mixed-radix complex FFT (the oracle's own; N/fft/Complex.java computes the same
// transform with its own radix passes).  sign = -1 forward, +1 unnormalised inverse.
struct FFT1D {
  int n = 0;
  std::vector<int> factors;
  std::vector<std::complex<double>> wf, wb;  // exp(-+2*pi*i*j/n), j < n
  explicit FFT1D(int n_ = 0) : n(n_) {
    int m = n;
    for (int f : {4, 2, 3, 5, 7}) {
      while (m % f == 0) { factors.push_back(f); m /= f; }
    }
    for (int f = 11; m > 1; f += 2) {
      while (m % f == 0) { factors.push_back(f); m /= f; }
    }
    wf.resize(n); wb.resize(n);
    for (int j = 0; j < n; j++) {
      const double ang = 2.0 * kPi * (double)j / (double)n;
      wf[j] = std::complex<double>(std::cos(ang), -std::sin(ang));
      wb[j] = std::complex<double>(std::cos(ang), std::sin(ang));
    }
  }
  // Recursive decimation in time on a strided view; w is the length-n twiddle table.
  void rec(const std::complex<double> *in, std::complex<double> *out, int len, int stride,
           size_t fi, const std::complex<double> *w, std::vector<std::complex<double>> &tmp,
           std::vector<std::complex<double>> &acc) const {
    if (len == 1) { out[0] = in[0]; return; }
    const int p = factors[fi];
    const int m = len / p;
    for (int q = 0; q < p; q++) rec(in + (size_t)q * stride, out + (size_t)q * m, m, stride * p, fi + 1, w, tmp, acc);
    const int step = n / len;   // W_len^e = W_n^(e*step)
    const int pstep = n / p;    // W_p^e   = W_n^(e*pstep)
    for (int k = 0; k < m; k++) {
      for (int q = 0; q < p; q++) tmp[q] = out[(size_t)q * m + k] * w[((size_t)q * k * step) % n];
      for (int s = 0; s < p; s++) {
        std::complex<double> a = 0.0;
        for (int q = 0; q < p; q++) a += tmp[q] * w[(size_t)((q * s) % p) * pstep];
        acc[s] = a;
      }
      for (int s = 0; s < p; s++) out[(size_t)s * m + k] = acc[s];
    }
  }
  void transform(std::complex<double> *data, int sign) const {
    std::vector<std::complex<double>> in(data, data + n), out(n), tmp(n), acc(n);
    rec(in.data(), out.data(), n, 1, 0, sign < 0 ? wf.data() : wb.data(), tmp, acc);
    std::copy(out.begin(), out.end(), data);
  }
};

// 3D transform in place on grid[(k*ny + j)*nx + i].
void fft3d(std::vector<std::complex<double>> &g, int nx, int ny, int nz, int sign) {
  FFT1D fx(nx), fy(ny), fz(nz);
#pragma omp parallel
  {
    std::vector<std::complex<double>> line(std::max(nx, std::max(ny, nz)));
#pragma omp for
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++) fx.transform(&g[((size_t)k * ny + j) * nx], sign);
#pragma omp for
    for (int k = 0; k < nz; k++)
      for (int i = 0; i < nx; i++) {
        for (int j = 0; j < ny; j++) line[j] = g[((size_t)k * ny + j) * nx + i];
        fy.transform(line.data(), sign);
        for (int j = 0; j < ny; j++) g[((size_t)k * ny + j) * nx + i] = line[j];
      }
#pragma omp for
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        for (int k = 0; k < nz; k++) line[k] = g[((size_t)k * ny + j) * nx + i];
        fz.transform(line.data(), sign);
        for (int k = 0; k < nz; k++) g[((size_t)k * ny + j) * nx + i] = line[k];
      }
  }
}

// ---------------------------------------------------------------------------
// Alchemical state of the vdW term (VanDerWaals.setLambda, :599-647; initSoftCore,
// :1150-1180).  Set through oracle_set_alchemy, read by Oracle::vdw.
struct Alchemy {
  bool on = false;
  std::vector<int> soft, mol;
  double sc1 = 0, dsc1dL = 0, d2sc1dL2 = 0, sc2 = 1, dsc2dL = 0, d2sc2dL2 = 0;
  bool inter = false, intra = false;
  double dEdL = 0, d2EdL2 = 0;
  std::vector<double> lgrad;   // [n][3] dU/dX dL
  // Electrostatics (elec-lambdaterm, OST mode): keys of AlchemicalParameters
  // (pme/AlchemicalParameters.java:60-190) and their values at lambda (update, :306-380).
  bool elec = false;
  double permAlpha = 2.0, permExp = 3.0, permStart = 0.4, permEnd = 1.0;
  double polStart = 0.75, polEnd = 1.0, polExp = 3.0;
  bool vaporElec = true, noLigandSCF = true;
  double lambda = 1.0;
  double lAlpha = 0, dlAlpha = 0, d2lAlpha = 0;
  double lPowPerm = 1, dlPowPerm = 0, d2lPowPerm = 0;
  double lPowPol = 1, dlPowPol = 0, d2lPowPol = 0;

  void update_elec(double l) {
    lambda = l;
    lPowPerm = 1.0; dlPowPerm = 0.0; d2lPowPerm = 0.0;
    lAlpha = 0.0; dlAlpha = 0.0; d2lAlpha = 0.0;
    if (l < permStart) {
      lPowPerm = 0.0;
    } else if (l <= permEnd) {
      const double scale = 1.0 / (permEnd - permStart);
      const double pl = scale * (l - permStart);
      lAlpha = permAlpha * (1.0 - pl) * (1.0 - pl);
      dlAlpha = permAlpha * (1.0 - pl);
      d2lAlpha = -permAlpha;
      lPowPerm = std::pow(pl, permExp);
      dlPowPerm = permExp * std::pow(pl, permExp - 1.0);
      d2lPowPerm = 0.0;
      if (permExp >= 2.0) d2lPowPerm = permExp * (permExp - 1.0) * std::pow(pl, permExp - 2.0);
      dlAlpha *= scale;
      d2lAlpha *= scale * scale;
      dlPowPerm *= scale;
      d2lPowPerm *= scale * scale;
    }
    lPowPol = 1.0; dlPowPol = 0.0; d2lPowPol = 0.0;
    if (l < polStart) {
      lPowPol = 0.0;
    } else if (l <= polEnd) {
      const double scale = 1.0 / (polEnd - polStart);
      const double pl = scale * (l - polStart);
      if (polExp > 0.0) {
        lPowPol = std::pow(pl, polExp);
        if (polExp >= 1.0) {
          dlPowPol = polExp * std::pow(pl, polExp - 1.0);
          if (polExp >= 2.0) d2lPowPol = polExp * (polExp - 1.0) * std::pow(pl, polExp - 2.0);
        }
      }
      dlPowPol *= scale;
      d2lPowPol *= scale * scale;
    }
  }
};
Alchemy g_alch;

// Multi-image lists forced on for boxes where the minimum image would also do (a
// consistency hook for tests; oracle_set_images).
int g_force_images = 0;

// Packed lattice shift of a multi-image list entry: n = (nx, ny, nz) in 10-bit fields
// offset by 512, bit 30 set on the minimum-image entry of the pair (the only one the
// bonded masks touch).
inline int pack_shift(int nx, int ny, int nz, bool primary) {
  return (nx + 512) | ((ny + 512) << 10) | ((nz + 512) << 20) | (primary ? (1 << 30) : 0);
}

struct Oracle {
  // ---- inputs
  int n = 0;
  Cell cell;
  ffxg_params p{};
  std::vector<double> x, y, z;           // coordinates
  std::vector<double> lmp;               // [n][10] local multipoles
  std::vector<int> frame, axis;          // [n], [n][3]
  std::vector<double> polar, thole, ipdamp;
  std::vector<int> vtype, redi;
  std::vector<double> redv;
  int ntypes = 0;
  std::vector<double> vrad, veps;
  std::vector<std::vector<int>> m12, m13, m14, m15, ip11;
  int nthreads = 1;

  // ---- derived
  double aewald = 0, off2 = 0, an0 = 0, an1 = 0, an2 = 0, an3 = 0, an4 = 0, an5 = 0, aewald3 = 0;
  std::vector<std::vector<int>> nlist;   // half list (i < k) at cutoff + buffer
  std::vector<std::vector<int>> ewald;   // realSpaceLists
  std::vector<std::vector<int>> precond; // preconditionerLists
  // Multi-image mode: the box is at most twice an interaction cutoff, so a pair may
  // interact through several lattice images (the reference's ReplicatesCrystal,
  // C/ReplicatesCrystal.java:172-202, whose replicate supercell sums the same images).
  // Each list entry then carries a packed shift (pack_shift) in the parallel lists below.
  bool multi_image = false;
  std::vector<std::vector<int>> nsh, esh, psh;

  // ---- one electrostatics evaluation of the lambda scheme (ParticleMeshEwald
  // condensedEnergy / condensedNoLigandSCF / ligandElec, PME:1609-1796): which atoms take
  // part (use), the scales of the permanent and polarization parts, and the lambda
  // derivative accumulators (dU/dL, d2U/dL2, dU/dX dL with its torque).
  std::vector<char> use;                 // empty: every atom
  std::vector<double> pol_eff;           // polarizability, 0 for atoms not in use (PCG)
  bool lam = false;                      // lambdaTerm
  bool vapor = false;                    // LambdaMode.VAPOR
  bool recip_on = true;                  // reciprocal space (off with Ewald alpha 0)
  bool doPermReal = true, doPol = true;
  double permScale = 1.0, polScale = 1.0, dEdLSign = 1.0;
  double stepAlpha = 0.0, stepDlAlpha = 0.0, stepD2lAlpha = 0.0;
  double eDL = 0.0, eD2L = 0.0;
  std::vector<double> lgE, ltE;          // [n][3]
  bool used(int i) const { return use.empty() || use[i]; }
  // VAPOR pairs skipped by the inter/intramolecular softcore options
  // (PermanentFieldRegion.java:665-670, RealSpaceEnergyRegion.java:865-870).
  bool vapor_skip(int i, int k) const {
    if (!vapor) return false;
    const bool same = g_alch.mol.empty() ? (i == k) : (g_alch.mol[i] == g_alch.mol[k]);
    return (g_alch.inter && !same) || (g_alch.intra && same);
  }

  // Displacement of list entry e of atom i, given x_k - x_i on entry: the minimum image
  // (Crystal.image) or, in multi-image mode, x_k + n L - x_i.  sign = -1 for the vdW
  // convention x_i - x_k.  Returns r^2 in Crystal.image's operation order.
  double disp(double &dx, double &dy, double &dz, const std::vector<std::vector<int>> &sh, int i, size_t e,
              double sign = 1.0) const {
    if (!multi_image) return image(dx, dy, dz, cell);
    const int c = sh[i][e];
    add_shift(dx, dy, dz, (c & 1023) - 512, ((c >> 10) & 1023) - 512, ((c >> 20) & 1023) - 512, sign, cell);
    return dx * dx + dy * dy + dz * dz;
  }
  // Whether entry e of atom i is the pair's minimum image (masks apply only there).
  bool primary(const std::vector<std::vector<int>> &sh, int i, size_t e) const {
    return !multi_image || ((sh[i][e] >> 30) & 1);
  }
  std::vector<double> gm;                // [n][10] global multipoles
  std::vector<double> fm;                // [n][10] fractional multipoles
  int nfx = 0, nfy = 0, nfz = 0, order = 5;
  std::vector<double> splx, sply, splz;  // [n][order][4]
  std::vector<int> igrid;                // [n][3]
  std::vector<double> influence;         // [nfx*nfy*nfz]
  double tmm[10][10], tfm[10][10], afrac[3][3];
  std::vector<double> cphi, fphi;        // permanent [n][20]
  std::vector<double> cphiI, cphiP, fphiI, fphiP;  // induced [n][20]
  std::vector<double> fieldD, fieldP;    // [n][3]
  std::vector<double> uD, uP, udir, udirP;  // [n][3]
  std::vector<double> grad, torque;      // [n][3]
  int scf_iter = 0, scf_total = 0;
  int status = FFXG_OK;

  void setup(const ffxg_system *s, const ffxg_params *prm, const double *xyz) {
    n = s->n_atoms;
    p = *prm;
    cell = make_cell(p.box, p.angles);
    x.resize(n); y.resize(n); z.resize(n);
    for (int i = 0; i < n; i++) { x[i] = xyz[3 * i]; y[i] = xyz[3 * i + 1]; z[i] = xyz[3 * i + 2]; }
    lmp.assign(s->multipole, s->multipole + 10 * (size_t)n);
    frame.assign(s->frame, s->frame + n);
    axis.assign(s->axis, s->axis + 3 * (size_t)n);
    polar.assign(s->polarizability, s->polarizability + n);
    thole.assign(s->thole, s->thole + n);
    ipdamp.resize(n);
    for (int i = 0; i < n; i++) {  // ParticleMeshEwald.java:1401-1406
      double pd = s->pdamp[i];
      ipdamp[i] = (pd > 0.0) ? 1.0 / pd : INFINITY;
    }
    vtype.assign(s->vdw_type, s->vdw_type + n);
    redi.assign(s->red_parent, s->red_parent + n);
    redv.assign(s->red_factor, s->red_factor + n);
    ntypes = s->n_vdw_types;
    vrad.assign(s->vdw_inv_rmin, s->vdw_inv_rmin + (size_t)ntypes * ntypes);
    veps.assign(s->vdw_eps, s->vdw_eps + (size_t)ntypes * ntypes);
    auto csr = [&](const int32_t *ptr, const int32_t *idx, std::vector<std::vector<int>> &out) {
      out.assign(n, {});
      for (int i = 0; i < n; i++) out[i].assign(idx + ptr[i], idx + ptr[i + 1]);
    };
    csr(s->mask12_ptr, s->mask12_idx, m12);
    csr(s->mask13_ptr, s->mask13_idx, m13);
    csr(s->mask14_ptr, s->mask14_idx, m14);
    csr(s->mask15_ptr, s->mask15_idx, m15);
    csr(s->ip11_ptr, s->ip11_idx, ip11);
    // pme/EwaldParameters.java:100-125
    aewald = p.ewald_alpha;
    off2 = p.ewald_cutoff * p.ewald_cutoff;
    const double alsq2 = 2.0 * aewald * aewald;
    const double piEwald = (aewald > 0.0) ? 1.0 / (kSqrtPi * aewald) : INFINITY;
    aewald3 = 4.0 / 3.0 * std::pow(aewald, 3.0) / kSqrtPi;
    if (aewald > 0.0) {
      an0 = alsq2 * piEwald; an1 = alsq2 * an0; an2 = alsq2 * an1;
      an3 = alsq2 * an2; an4 = alsq2 * an3; an5 = alsq2 * an4;
    }
    nfx = p.pme_grid[0]; nfy = p.pme_grid[1]; nfz = p.pme_grid[2];
    order = p.pme_order;
    const double maxcut = std::max(std::max(p.vdw_cutoff, p.ewald_cutoff), p.precond_cutoff);
    multi_image = g_force_images != 0;
    for (int d = 0; d < 3; d++)
      if (cell.width[d] <= 2.0 * maxcut) multi_image = true;
    setup_recip();
  }

  // ---------------------------------------------------------------------------
  // NeighborList.java:905-1115 on the hydrogen-reduced coordinates of
  // VanDerWaals.ExpandLoop (VanDerWaals.java:1505-1541).  The search is a
  // complete cell search; the pair set is defined by d2 <= (cutoff + buffer)^2.
  void reduced_coords(std::vector<double> &rx, std::vector<double> &ry, std::vector<double> &rz) const {
    rx.resize(n); ry.resize(n); rz.resize(n);
    for (int i = 0; i < n; i++) {
      const int r = redi[i];
      const double a = redv[i];
      if (r != i || a != 0.0) {
        rx[i] = a * (x[i] - x[r]) + x[r];
        ry[i] = a * (y[i] - y[r]) + y[r];
        rz[i] = a * (z[i] - z[r]) + z[r];
      } else {
        rx[i] = x[i]; ry[i] = y[i]; rz[i] = z[i];
      }
    }
  }

  // Multi-image list: every image k + n L (k >= i; n > 0 in (z, y, x) lexicographic order
  // for k == i) within the buffered cutoff.  n runs over n0 + m, n0 the minimum-image
  // shift of the raw difference and |m_d| <= floor(rlist / w_d + 1/2) (w_d the
  // perpendicular width), which covers every image inside rlist.  Brute force over atom
  // pairs: boxes this small hold few atoms.
  //
  // The primary image of a pair (the one the bonded masks apply to) is the reference's
  // iSymm = 0 pair: the minimum image in its replicate supercell of l x m x n unit cells,
  // the smallest counts whose interfacial radii (half the perpendicular widths) reach the
  // buffered cutoff (ReplicatesCrystal.replicatesCrystalFactory, C/ReplicatesCrystal.java:
  // 172-202).  For the covalent partners of a whole molecule that is the molecule's own
  // geometry even when the unit cell is narrower than the molecule.
  void build_list_images(const std::vector<double> &rx, const std::vector<double> &ry,
                         const std::vector<double> &rz, double rlist) {
    const double rl2 = rlist * rlist;
    const int R[3] = {(int)std::floor(rlist / cell.width[0] + 0.5), (int)std::floor(rlist / cell.width[1] + 0.5),
                      (int)std::floor(rlist / cell.width[2] + 0.5)};
    int rep[3];
    double sbox[3];
    for (int d = 0; d < 3; d++) {
      rep[d] = 1;
      while (cell.width[d] / 2.0 * rep[d] < rlist) rep[d]++;
    }
    sbox[0] = cell.a * rep[0]; sbox[1] = cell.b * rep[1]; sbox[2] = cell.c * rep[2];
    const Cell super = make_cell(sbox, p.angles);
    nlist.assign(n, {});
    nsh.assign(n, {});
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < n; i++) {
      for (int k = i; k < n; k++) {
        const double dx = rx[k] - rx[i], dy = ry[k] - ry[i], dz = rz[k] - rz[i];
        double fx, fy, fz;
        to_frac(dx, dy, dz, cell, fx, fy, fz);
        const int n0x = (int)(std::floor(std::fabs(fx) + 0.5) * jsignum(-fx));
        const int n0y = (int)(std::floor(std::fabs(fy) + 0.5) * jsignum(-fy));
        const int n0z = (int)(std::floor(std::fabs(fz) + 0.5) * jsignum(-fz));
        double sx, sy, sz;
        to_frac(dx, dy, dz, super, sx, sy, sz);
        const int px = rep[0] * (int)(std::floor(std::fabs(sx) + 0.5) * jsignum(-sx));
        const int py = rep[1] * (int)(std::floor(std::fabs(sy) + 0.5) * jsignum(-sy));
        const int pz = rep[2] * (int)(std::floor(std::fabs(sz) + 0.5) * jsignum(-sz));
        for (int mz = -R[2]; mz <= R[2]; mz++)
          for (int my = -R[1]; my <= R[1]; my++)
            for (int mx = -R[0]; mx <= R[0]; mx++) {
              const int nx = n0x + mx, ny = n0y + my, nz = n0z + mz;
              if (k == i && !(nz > 0 || (nz == 0 && (ny > 0 || (ny == 0 && nx > 0))))) continue;
              double ex = dx, ey = dy, ez = dz;
              add_shift(ex, ey, ez, nx, ny, nz, 1.0, cell);
              const double d2 = ex * ex + ey * ey + ez * ez;
              if (d2 <= rl2) {
                nlist[i].push_back(k);
                nsh[i].push_back(pack_shift(nx, ny, nz, nx == px && ny == py && nz == pz));
              }
            }
      }
    }
  }

  void build_list() {
    std::vector<double> rx, ry, rz;
    reduced_coords(rx, ry, rz);
    const double rlist = std::max(p.vdw_cutoff, p.ewald_cutoff) + p.list_buffer;
    const double rl2 = rlist * rlist;
    if (multi_image) {
      build_list_images(rx, ry, rz, rlist);
      return;
    }
    // Cells at least rlist/2 wide; search +-2 cells (nEdge = 2, NeighborList.java:1296-1345).
    const int nca = std::max(1, (int)std::floor(cell.width[0] / (rlist * 0.5)));
    const int ncb = std::max(1, (int)std::floor(cell.width[1] / (rlist * 0.5)));
    const int ncc = std::max(1, (int)std::floor(cell.width[2] / (rlist * 0.5)));
    std::vector<std::vector<int>> cells((size_t)nca * ncb * ncc);
    auto cidx = [&](int i, int &ca, int &cb, int &cc) {
      double fx, fy, fz;
      to_frac(rx[i], ry[i], rz[i], cell, fx, fy, fz);
      fx -= std::floor(fx); fy -= std::floor(fy); fz -= std::floor(fz);
      ca = std::min(nca - 1, (int)(fx * nca));
      cb = std::min(ncb - 1, (int)(fy * ncb));
      cc = std::min(ncc - 1, (int)(fz * ncc));
    };
    std::vector<int> ca(n), cb(n), cc(n);
    for (int i = 0; i < n; i++) {
      cidx(i, ca[i], cb[i], cc[i]);
      cells[((size_t)cc[i] * ncb + cb[i]) * nca + ca[i]].push_back(i);
    }
    // Offsets -2..2 when a dimension has at least 5 cells, otherwise every cell of
    // that dimension once (a +-2 search would revisit or miss cells).
    auto offsets = [](int nc) {
      std::vector<int> o;
      if (nc >= 5) { for (int d = -2; d <= 2; d++) o.push_back(d); }
      else { for (int d = 0; d < nc; d++) o.push_back(d); }
      return o;
    };
    const std::vector<int> oa = offsets(nca), ob = offsets(ncb), oc = offsets(ncc);
    nlist.assign(n, {});
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; i++) {
      std::vector<int> &li = nlist[i];
      for (int dc : oc)
        for (int db : ob)
          for (int da : oa) {
            const int a2 = ((ca[i] + da) % nca + nca) % nca;
            const int b2 = ((cb[i] + db) % ncb + ncb) % ncb;
            const int c2 = ((cc[i] + dc) % ncc + ncc) % ncc;
            for (int k : cells[((size_t)c2 * ncb + b2) * nca + a2]) {
              if (k <= i) continue;
              double dx = rx[i] - rx[k], dy = ry[i] - ry[k], dz = rz[i] - rz[k];
              const double d2 = image(dx, dy, dz, cell);
              if (d2 <= rl2) li.push_back(k);
            }
          }
      std::sort(li.begin(), li.end());
    }
  }

  // ---------------------------------------------------------------------------
  // Buffered 14-7 van der Waals, VanDerWaals.java:1602-1850; VanDerWaalsForm.java:313-334;
  // MultiplicativeSwitch.java:84-124, 234-236.
  double vdw(bool gradient, int64_t &count) {
    std::vector<double> rx, ry, rz;
    reduced_coords(rx, ry, rz);
    const double off = p.vdw_cutoff, cut = p.vdw_taper * p.vdw_cutoff;
    const double off2v = off * off, cut2 = cut * cut;
    const double delta = 0.07, gamma = 0.12;  // VDWType DEFAULT_DELTA / DEFAULT_GAMMA
    const double t1n = std::pow(1.0 + delta, 7.0), gamma1 = 1.0 + gamma;
    const double a = cut, b = off, a2 = a * a, b2 = b * b, den = std::pow(b - a, 5.0);
    const double c0 = b * b2 * (b2 - 5.0 * a * b + 10.0 * a2) / den;
    const double c1 = -30.0 * a2 * b2 / den;
    const double c2 = 30.0 * b * a * (b + a) / den;
    const double c3 = -10.0 * (a2 + 4.0 * a * b + b2) / den;
    const double c4 = 15.0 * (a + b) / den;
    const double c5 = -6.0 / den;
    double energy = 0.0, dEdL = 0.0, d2EdL2 = 0.0;
    int64_t cnt = 0;
    const Alchemy &al = g_alch;
    std::vector<std::vector<double>> tg(nthreads, std::vector<double>(3 * (size_t)n, 0.0));
    std::vector<std::vector<double>> tl(al.on ? nthreads : 0, std::vector<double>(3 * (size_t)n, 0.0));
#pragma omp parallel reduction(+ : energy, cnt, dEdL, d2EdL2)
    {
      int tid = 0;
#ifdef _OPENMP
      tid = omp_get_thread_num();
#endif
      std::vector<double> &g = tg[tid];
      std::vector<double> mask(n, 1.0);
#pragma omp for schedule(dynamic, 64)
      for (int i = 0; i < n; i++) {
        for (int k : m12[i]) mask[k] = p.v12;
        for (int k : m13[i]) mask[k] = p.v13;
        for (int k : m14[i]) mask[k] = p.v14;
        const double xi = rx[i], yi = ry[i], zi = rz[i];
        const double rv = redv[i], rdv = 1.0 - rv;
        const int ri = redi[i];
        const int ti = vtype[i];
        for (size_t e = 0; e < nlist[i].size(); e++) {
          const int k = nlist[i][e];
          double dx = xi - rx[k], dy = yi - ry[k], dz = zi - rz[k];
          const double r2 = disp(dx, dy, dz, nsh, i, e, -1.0);
          const int tk = vtype[k];
          const double irv = vrad[(size_t)ti * ntypes + tk];
          const double mk = primary(nsh, i, e) ? mask[k] : 1.0;
          if (!(r2 <= off2v && mk > 0.0 && irv > 0.0)) continue;
          const double r = std::sqrt(r2);
          // Softcore pair (VanDerWaals.java:1728-1761): exactly one atom soft, or both
          // soft under the intermolecular / intramolecular softcore options.
          bool soft = false;
          if (al.on) {
            const int si = al.soft[i], sk = al.soft[k];
            soft = (si != sk);
            if (si && sk) {
              const bool same = al.mol[i] == al.mol[k];
              if (al.inter && !same) soft = true;
              else if (al.intra && same) soft = true;
            }
          }
          const double alpha = soft ? al.sc1 : 0.0;
          const double lambda5 = soft ? al.sc2 : 1.0;
          const double ev = mk * veps[(size_t)ti * ntypes + tk];
          const double eps_lambda = ev * lambda5;
          const double rho = r * irv;
          const double rho2 = rho * rho;
          const double rhoDisp1 = rho2 * rho2 * rho2;
          const double rhoDisp = rhoDisp1 * rho;
          const double rd = rho + delta, rd2 = rd * rd;
          const double rhoDelta1 = rd2 * rd2 * rd2;
          const double rhoDelta = rhoDelta1 * rd;
          const double t1d = 1.0 / (alpha + rhoDelta);
          const double t2d = 1.0 / (alpha + rhoDisp + gamma);
          const double t1 = t1n * t1d;
          const double t2a = gamma1 * t2d;
          const double t2 = t2a - 2.0;
          const double eik = eps_lambda * t1 * t2;
          double taper = 1.0, dtaper = 0.0;
          if (r2 > cut2) {
            const double r3 = r2 * r, r4 = r2 * r2, r5 = r2 * r3;
            taper = c5 * r5 + c4 * r4 + c3 * r3 + c2 * r2 + c1 * r + c0;
            dtaper = 5.0 * c5 * r4 + 4.0 * c4 * r3 + 3.0 * c3 * r2 + 2.0 * c2 * r + c1;
          }
          energy += eik * taper;
          cnt++;
          if (!gradient && !soft) continue;
          const double dt1d_dr = 7.0 * rhoDelta1 * irv;
          const double dt2d_dr = 7.0 * rhoDisp1 * irv;
          const double dt1_dr = t1 * dt1d_dr * t1d;
          const double dt2_dr = t2a * dt2d_dr * t2d;
          const double dedr = -eps_lambda * (dt1_dr * t2 + t1 * dt2_dr);
          const double ir = 1.0 / r;
          if (soft) {
            // dU/dL, d2U/dL2 and dU/dX dL of the softcore pair (VanDerWaals.java:1842-1880).
            const double dt1 = -t1 * t1d * al.dsc1dL;
            const double dt2 = -t2a * t2d * al.dsc1dL;
            const double f1 = al.dsc2dL * t1 * t2;
            const double f2 = al.sc2 * dt1 * t2;
            const double f3 = al.sc2 * t1 * dt2;
            const double dedl = ev * (f1 + f2 + f3);
            dEdL += dedl * taper;
            const double t1d2 = -al.dsc1dL * t1d * t1d;
            const double t2d2 = -al.dsc1dL * t2d * t2d;
            const double d2t1 = -dt1 * t1d * al.dsc1dL - t1 * t1d * al.d2sc1dL2 - t1 * t1d2 * al.dsc1dL;
            const double d2t2 = -dt2 * t2d * al.dsc1dL - t2a * t2d * al.d2sc1dL2 - t2a * t2d2 * al.dsc1dL;
            const double df1 = al.d2sc2dL2 * t1 * t2 + al.dsc2dL * dt1 * t2 + al.dsc2dL * t1 * dt2;
            const double df2 = al.dsc2dL * dt1 * t2 + al.sc2 * d2t1 * t2 + al.sc2 * dt1 * dt2;
            const double df3 = al.dsc2dL * t1 * dt2 + al.sc2 * dt1 * dt2 + al.sc2 * t1 * d2t2;
            d2EdL2 += ev * (df1 + df2 + df3) * taper;
            if (gradient) {
              const double t11 = -al.dsc2dL * t2 * dt1_dr;
              const double t21 = -al.dsc2dL * t1 * dt2_dr;
              const double t13 = 2.0 * al.sc2 * t2 * dt1_dr * al.dsc1dL * t1d;
              const double t23 = 2.0 * al.sc2 * t1 * dt2_dr * al.dsc1dL * t2d;
              const double t12 = -al.sc2 * dt2 * dt1_dr;
              const double t22 = -al.sc2 * dt1 * dt2_dr;
              const double dedldr = ev * (t11 + t12 + t13 + t21 + t22 + t23);
              const double lsw = dedl * dtaper + dedldr * taper;
              const double lx = lsw * dx * ir, ly = lsw * dy * ir, lz = lsw * dz * ir;
              std::vector<double> &lg = tl[tid];
              lg[3 * i] += lx * rv; lg[3 * i + 1] += ly * rv; lg[3 * i + 2] += lz * rv;
              lg[3 * ri] += lx * rdv; lg[3 * ri + 1] += ly * rdv; lg[3 * ri + 2] += lz * rdv;
              const int rk = redi[k];
              const double red = redv[k], redk = 1.0 - red;
              lg[3 * k] -= red * lx; lg[3 * k + 1] -= red * ly; lg[3 * k + 2] -= red * lz;
              lg[3 * rk] -= redk * lx; lg[3 * rk + 1] -= redk * ly; lg[3 * rk + 2] -= redk * lz;
            }
          }
          if (!gradient) continue;
          const double dswitch = eik * dtaper + dedr * taper;
          const double dedx = dswitch * dx * ir, dedy = dswitch * dy * ir, dedz = dswitch * dz * ir;
          g[3 * i] += dedx * rv; g[3 * i + 1] += dedy * rv; g[3 * i + 2] += dedz * rv;
          g[3 * ri] += dedx * rdv; g[3 * ri + 1] += dedy * rdv; g[3 * ri + 2] += dedz * rdv;
          const int rk = redi[k];
          const double red = redv[k], redk = 1.0 - red;
          g[3 * k] -= red * dedx; g[3 * k + 1] -= red * dedy; g[3 * k + 2] -= red * dedz;
          g[3 * rk] -= redk * dedx; g[3 * rk + 1] -= redk * dedy; g[3 * rk + 2] -= redk * dedz;
        }
        for (int k : m12[i]) mask[k] = 1.0;
        for (int k : m13[i]) mask[k] = 1.0;
        for (int k : m14[i]) mask[k] = 1.0;
      }
    }
    if (gradient)
      for (int t = 0; t < nthreads; t++)
        for (size_t j = 0; j < 3 * (size_t)n; j++) grad[j] += tg[t][j];
    if (al.on) {
      g_alch.dEdL = dEdL;
      g_alch.d2EdL2 = d2EdL2;
      g_alch.lgrad.assign(3 * (size_t)n, 0.0);
      if (gradient)
        for (int t = 0; t < nthreads; t++)
          for (size_t j = 0; j < 3 * (size_t)n; j++) g_alch.lgrad[j] += tl[t][j];
    }
    count = cnt;
    return energy;
  }

  // ---------------------------------------------------------------------------
  // Multipole rotation, pme/InitializationRegion.java:375-480 and
  // P/parameters/MultipoleType.java:385-536 (getRotationMatrix), :1031-1062 (rotateMultipole).
  static void norm3(double *v) {
    const double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] /= l; v[1] /= l; v[2] /= l;
  }
  static double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

  void rotation_matrix(int i, double R[3][3]) const {
    const double o[3] = {x[i], y[i], z[i]};
    double zA[3], xA[3], yA[3];
    double fc[3][3];
    for (int s = 0; s < 3; s++) {
      const int a = axis[3 * i + s];
      if (a >= 0) { fc[s][0] = x[a]; fc[s][1] = y[a]; fc[s][2] = z[a]; }
    }
    R[0][0] = 1; R[0][1] = 0; R[0][2] = 0;
    R[1][0] = 0; R[1][1] = 1; R[1][2] = 0;
    R[2][0] = 0; R[2][1] = 0; R[2][2] = 1;
    switch (frame[i]) {
      case FFXG_FRAME_NONE: return;
      case FFXG_FRAME_BISECTOR: {
        for (int d = 0; d < 3; d++) { zA[d] = fc[0][d] - o[d]; xA[d] = fc[1][d] - o[d]; }
        norm3(zA); norm3(xA);
        for (int d = 0; d < 3; d++) zA[d] = xA[d] + zA[d];
        norm3(zA);
        R[0][2] = zA[0]; R[1][2] = zA[1]; R[2][2] = zA[2];
        const double dt = dot3(xA, zA);
        for (int d = 0; d < 3; d++) zA[d] = zA[d] * dt;
        for (int d = 0; d < 3; d++) xA[d] = xA[d] - zA[d];
        norm3(xA);
        break;
      }
      case FFXG_FRAME_ZTHENBISECTOR: {
        for (int d = 0; d < 3; d++) { zA[d] = fc[0][d] - o[d]; }
        norm3(zA);
        R[0][2] = zA[0]; R[1][2] = zA[1]; R[2][2] = zA[2];
        for (int d = 0; d < 3; d++) { xA[d] = fc[1][d] - o[d]; yA[d] = fc[2][d] - o[d]; }
        norm3(xA); norm3(yA);
        for (int d = 0; d < 3; d++) xA[d] = xA[d] + yA[d];
        norm3(xA);
        const double dt = dot3(xA, zA);
        for (int d = 0; d < 3; d++) zA[d] = zA[d] * dt;
        for (int d = 0; d < 3; d++) xA[d] = xA[d] - zA[d];
        norm3(xA);
        break;
      }
      case FFXG_FRAME_ZONLY: {
        for (int d = 0; d < 3; d++) zA[d] = fc[0][d] - o[d];
        norm3(zA);
        R[0][2] = zA[0]; R[1][2] = zA[1]; R[2][2] = zA[2];
        xA[0] = 1.0; xA[1] = 0.0; xA[2] = 0.0;
        double dt = R[0][2];
        if (std::fabs(dt) > 0.866) { xA[0] = 0.0; xA[1] = 1.0; dt = R[1][2]; }
        for (int d = 0; d < 3; d++) zA[d] = zA[d] * dt;
        for (int d = 0; d < 3; d++) xA[d] = xA[d] - zA[d];
        norm3(xA);
        break;
      }
      case FFXG_FRAME_THREEFOLD: {
        for (int d = 0; d < 3; d++) { zA[d] = fc[0][d] - o[d]; xA[d] = fc[1][d] - o[d]; yA[d] = fc[2][d] - o[d]; }
        norm3(zA); norm3(xA); norm3(yA);
        double sum[3];
        for (int d = 0; d < 3; d++) sum[d] = zA[d] + xA[d];
        for (int d = 0; d < 3; d++) sum[d] = sum[d] + yA[d];
        norm3(sum);
        R[0][2] = sum[0]; R[1][2] = sum[1]; R[2][2] = sum[2];
        const double dt = dot3(zA, sum);
        for (int d = 0; d < 3; d++) sum[d] = sum[d] * dt;
        for (int d = 0; d < 3; d++) xA[d] = zA[d] - sum[d];
        norm3(xA);
        break;
      }
      case FFXG_FRAME_ZTHENX:
      default: {
        for (int d = 0; d < 3; d++) { zA[d] = fc[0][d] - o[d]; xA[d] = fc[1][d] - o[d]; }
        norm3(zA);
        R[0][2] = zA[0]; R[1][2] = zA[1]; R[2][2] = zA[2];
        const double dt = dot3(xA, zA);
        for (int d = 0; d < 3; d++) zA[d] = zA[d] * dt;
        for (int d = 0; d < 3; d++) xA[d] = xA[d] - zA[d];
        norm3(xA);
        break;
      }
    }
    R[0][0] = xA[0]; R[1][0] = xA[1]; R[2][0] = xA[2];
    R[0][1] = R[2][0] * R[1][2] - R[1][0] * R[2][2];
    R[1][1] = R[0][0] * R[2][2] - R[2][0] * R[0][2];
    R[2][1] = R[1][0] * R[0][2] - R[0][0] * R[1][2];
  }

  void rotate_multipoles() {
    gm.assign(10 * (size_t)n, 0.0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
      double R[3][3];
      rotation_matrix(i, R);
      const double *in = &lmp[10 * (size_t)i];
      const double d[3] = {in[t100], in[t010], in[t001]};
      double Q[3][3];
      Q[0][0] = in[t200]; Q[1][1] = in[t020]; Q[2][2] = in[t002];
      Q[0][1] = Q[1][0] = in[t110];
      Q[0][2] = Q[2][0] = in[t101];
      Q[1][2] = Q[2][1] = in[t011];
      double rd[3] = {0, 0, 0}, rq[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int a = 0; a < 3; a++) {
        for (int b = 0; b < 3; b++) {
          rd[a] += R[a][b] * d[b];
          if (b < a) {
            rq[a][b] = rq[b][a];
          } else {
            for (int k = 0; k < 3; k++)
              rq[a][b] += R[a][k] * (R[b][0] * Q[k][0] + R[b][1] * Q[k][1] + R[b][2] * Q[k][2]);
          }
        }
      }
      double *out = &gm[10 * (size_t)i];
      out[t000] = in[0];
      out[t100] = rd[0]; out[t010] = rd[1]; out[t001] = rd[2];
      out[t200] = rq[0][0]; out[t020] = rq[1][1]; out[t002] = rq[2][2];
      out[t110] = rq[0][1]; out[t101] = rq[0][2]; out[t011] = rq[1][2];
    }
  }

  // ---------------------------------------------------------------------------
  // Reciprocal space set-up: ReciprocalSpace.java:1123-1210 (transform matrices),
  // :435-492 (discreteFTMod), :1045-1121 (generalizedInfluenceFunction).
  void setup_recip() {
    static const int qi1[6] = {0, 1, 2, 0, 0, 1};
    static const int qi2[6] = {0, 1, 2, 1, 2, 2};
    const int nf[3] = {nfx, nfy, nfz};
    double a[3][3];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) a[j][i] = nf[j] * cell.A[i][j];
    std::memset(tmm, 0, sizeof(tmm));
    tmm[0][0] = 1.0;
    for (int i = 1; i < 4; i++)
      for (int j = 0; j < 3; j++) tmm[i][1 + j] = a[i - 1][j];
    for (int i1 = 0; i1 < 3; i1++) {
      const int k = qi1[i1];
      for (int i2 = 0; i2 < 6; i2++) tmm[i1 + 4][i2 + 4] = a[k][qi1[i2]] * a[k][qi2[i2]];
    }
    for (int i1 = 3; i1 < 6; i1++) {
      const int k = qi1[i1], l = qi2[i1];
      for (int i2 = 0; i2 < 6; i2++) {
        const int ii = qi1[i2], jj = qi2[i2];
        tmm[i1 + 4][i2 + 4] = a[k][ii] * a[l][jj] + a[k][jj] * a[l][ii];
      }
    }
    double af[3][3];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) af[i][j] = nf[j] * cell.A[i][j];
    std::memset(tfm, 0, sizeof(tfm));
    tfm[0][0] = 1.0;
    for (int i = 1; i < 4; i++)
      for (int j = 0; j < 3; j++) tfm[i][1 + j] = af[i - 1][j];
    for (int i1 = 0; i1 < 3; i1++) {
      const int k = qi1[i1];
      for (int i2 = 0; i2 < 3; i2++) { const int ii = qi1[i2]; tfm[i1 + 4][i2 + 4] = af[k][ii] * af[k][ii]; }
      for (int i2 = 3; i2 < 6; i2++) {
        const int ii = qi1[i2], jj = qi2[i2];
        tfm[i1 + 4][i2 + 4] = 2.0 * af[k][ii] * af[k][jj];
      }
    }
    for (int i1 = 3; i1 < 6; i1++) {
      const int k = qi1[i1], nn = qi2[i1];
      for (int i2 = 0; i2 < 3; i2++) { const int ii = qi1[i2]; tfm[i1 + 4][i2 + 4] = af[k][ii] * af[nn][ii]; }
      for (int i2 = 3; i2 < 6; i2++) {
        const int ii = qi1[i2], jj = qi2[i2];
        tfm[i1 + 4][i2 + 4] = af[k][ii] * af[nn][jj] + af[nn][ii] * af[k][jj];
      }
    }
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) afrac[i][j] = nf[i] * cell.A[j][i];
    // Influence function.
    const int maxfft = std::max(std::max(std::max(nfx, nfy), nfz), order + 1);
    std::vector<double> bsarray(maxfft, 0.0);
    double c[16];
    bspline_coeffs(0.0, order, c);
    for (int i = 0; i < order; i++) bsarray[1 + i] = c[i];
    auto ftmod = [&](int nfft) {
      std::vector<double> bsmod(nfft);
      const double factor = 2.0 * kPi / nfft;
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
      const int jcut = 50, order2 = 2 * order;
      for (int i = 0; i < nfft; i++) {
        int k = i;
        if (i > nfft / 2) k = k - nfft;
        double zeta;
        if (k == 0) {
          zeta = 1.0;
        } else {
          double sum1 = 1.0, sum2 = 1.0;
          const double fct = kPi * k / nfft;
          for (int j = 0; j < jcut; j++) {
            const double arg = fct / (fct + kPi * (j + 1));
            sum1 = sum1 + std::pow(arg, order);
            sum2 = sum2 + std::pow(arg, order2);
          }
          for (int j = 0; j < jcut; j++) {
            const double arg = fct / (fct - kPi * (j + 1));
            sum1 = sum1 + std::pow(arg, order);
            sum2 = sum2 + std::pow(arg, order2);
          }
          zeta = sum2 / sum1;
        }
        bsmod[i] = bsmod[i] * zeta * zeta;
      }
      return bsmod;
    };
    const std::vector<double> bx = ftmod(nfx), by = ftmod(nfy), bz = ftmod(nfz);
    influence.assign((size_t)nfx * nfy * nfz, 0.0);
    const double piTerm = (kPi / aewald) * (kPi / aewald);
    const double volTerm = kPi * cell.volume;
    const int nX2 = (nfx + 1) / 2, nY2 = (nfy + 1) / 2, nZ2 = (nfz + 1) / 2;
    for (int kz = 0; kz < nfz; kz++)
      for (int ky = 0; ky < nfy; ky++)
        for (int kx = 0; kx < nfx; kx++) {
          if (kx == 0 && ky == 0 && kz == 0) continue;
          int h = kx, k = ky, l = kz;
          if (kx >= nX2) h -= nfx;
          if (ky >= nY2) k -= nfy;
          if (kz >= nZ2) l -= nfz;
          const double sX = cell.A[0][0] * h + cell.A[0][1] * k + cell.A[0][2] * l;
          const double sY = cell.A[1][0] * h + cell.A[1][1] * k + cell.A[1][2] * l;
          const double sZ = cell.A[2][0] * h + cell.A[2][1] * k + cell.A[2][2] * l;
          const double s2 = sX * sX + sY * sY + sZ * sZ;
          const double term = -piTerm * s2;
          double expterm = 0.0;
          if (term > -50.0) {
            const double denom = s2 * volTerm * bx[kx] * by[ky] * bz[kz];
            expterm = std::exp(term) / denom;
          }
          influence[((size_t)kz * nfy + ky) * nfx + kx] = expterm;
        }
  }

  // ReciprocalSpace.BSplineLoop (ReciprocalSpace.java:1338-1412).
  void compute_bsplines() {
    splx.assign((size_t)n * order * 4, 0.0);
    sply.assign((size_t)n * order * 4, 0.0);
    splz.assign((size_t)n * order * 4, 0.0);
    igrid.assign(3 * (size_t)n, 0);
    const double r00 = cell.A[0][0], r01 = cell.A[0][1], r02 = cell.A[0][2];
    const double r10 = cell.A[1][0], r11 = cell.A[1][1], r12 = cell.A[1][2];
    const double r20 = cell.A[2][0], r21 = cell.A[2][1], r22 = cell.A[2][2];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
      const double xi = x[i], yi = y[i], zi = z[i];
      const double wx = xi * r00 + yi * r10 + zi * r20;
      const double ux = wx - std::floor(wx + 0.5) + 0.5;
      const double frx = nfx * ux;
      const int ifrx = (int)frx;
      igrid[3 * i] = ifrx - order;
      bspline_derivs(frx - ifrx, order, &splx[(size_t)i * order * 4]);
      const double wy = xi * r01 + yi * r11 + zi * r21;
      const double uy = wy - std::floor(wy + 0.5) + 0.5;
      const double fry = nfy * uy;
      const int ifry = (int)fry;
      igrid[3 * i + 1] = ifry - order;
      bspline_derivs(fry - ifry, order, &sply[(size_t)i * order * 4]);
      const double wz = xi * r02 + yi * r12 + zi * r22;
      const double uz = wz - std::floor(wz + 0.5) + 0.5;
      const double frz = nfz * uz;
      const int ifrz = (int)frz;
      igrid[3 * i + 2] = ifrz - order;
      bspline_derivs(frz - ifrz, order, &splz[(size_t)i * order * 4]);
    }
  }

  static int jmod(int a, int m) { int r = a % m; return r < 0 ? r + m : r; }

  // Fractional multipoles (ReciprocalSpace.toFractionalMultipole, :1212-1236) and the
  // SpatialPermanentLoop.gridMultipoleDensity spreading (:1445-1505).
  void spread_permanent(std::vector<std::complex<double>> &grid) {
    fm.assign(10 * (size_t)n, 0.0);
    for (int i = 0; i < n; i++) {
      const double *g = &gm[10 * (size_t)i];
      double *f = &fm[10 * (size_t)i];
      f[0] = g[0];
      for (int j = 1; j < 4; j++) {
        f[j] = 0.0;
        for (int k = 1; k < 4; k++) f[j] = std::fma(tmm[j][k], g[k], f[j]);
      }
      for (int j = 4; j < 10; j++) {
        f[j] = 0.0;
        for (int k = 4; k < 7; k++) f[j] = std::fma(tmm[j][k], g[k], f[j]);
        for (int k = 7; k < 10; k++) f[j] = std::fma(tmm[j][k] * 2.0, g[k], f[j]);
        f[j] = f[j] * (1.0 / 3.0);
      }
    }
    grid.assign((size_t)nfx * nfy * nfz, 0.0);
    for (int i = 0; i < n; i++) {
      if (!used(i)) continue;   // atoms not in use are not spread (ReciprocalSpace.java:2821, 2884)
      const double *f = &fm[10 * (size_t)i];
      const double *sx = &splx[(size_t)i * order * 4], *sy = &sply[(size_t)i * order * 4],
                   *sz = &splz[(size_t)i * order * 4];
      const int i0g = igrid[3 * i], j0g = igrid[3 * i + 1];
      int k0 = igrid[3 * i + 2];
      for (int a3 = 0; a3 < order; a3++) {
        const double v0 = sz[a3 * 4], v1 = sz[a3 * 4 + 1], v2 = sz[a3 * 4 + 2];
        const double c0 = f[t000] * v0, dx0 = f[t100] * v0, dy0 = f[t010] * v0, dz1 = f[t001] * v1;
        const double qxx0 = f[t200] * v0, qyy0 = f[t020] * v0, qzz2 = f[t002] * v2;
        const double qxy0 = f[t110] * v0, qxz1 = f[t101] * v1, qyz1 = f[t011] * v1;
        const double c0dz1qzz2 = c0 + dz1 + qzz2;
        const double dy0qyz1 = dy0 + qyz1;
        const double dx0qxz1 = dx0 + qxz1;
        const int kk = jmod(++k0, nfz);
        int j0 = j0g;
        for (int a2 = 0; a2 < order; a2++) {
          const double u0 = sy[a2 * 4], u1 = sy[a2 * 4 + 1], u2 = sy[a2 * 4 + 2];
          const double term0 = std::fma(c0dz1qzz2, u0, std::fma(dy0qyz1, u1, qyy0 * u2));
          const double term1 = std::fma(dx0qxz1, u0, qxy0 * u1);
          const double term2 = qxx0 * u0;
          const int jj = jmod(++j0, nfy);
          int ii0 = i0g;
          for (int a1 = 0; a1 < order; a1++) {
            const int ii = jmod(++ii0, nfx);
            std::complex<double> &cur = grid[((size_t)kk * nfy + jj) * nfx + ii];
            double upd = std::fma(sx[a1 * 4], term0, cur.real());
            upd = std::fma(sx[a1 * 4 + 1], term1, upd);
            upd = std::fma(sx[a1 * 4 + 2], term2, upd);
            cur = std::complex<double>(upd, cur.imag());
          }
        }
      }
    }
  }

  // Complex3DParallel.convolution: forward FFT, multiply by the influence function,
  // unnormalised inverse FFT (N/fft/Complex3DParallel.java:445, 775-795, 972-1010).
  void convolve(std::vector<std::complex<double>> &grid) {
    fft3d(grid, nfx, nfy, nfz, -1);
    for (size_t i = 0; i < grid.size(); i++) grid[i] *= influence[i];
    fft3d(grid, nfx, nfy, nfz, +1);
  }

  // PermanentPhiLoop / InducedPhiLoop (ReciprocalSpace.java:2295-2454, 2506-2775):
  // 20 fractional potential terms of the real (part = 0) or imaginary (part = 1) grid.
  void interpolate(const std::vector<std::complex<double>> &grid, int part, std::vector<double> &frac,
                   std::vector<double> &cart) {
    frac.assign(20 * (size_t)n, 0.0);
    cart.assign(20 * (size_t)n, 0.0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
      const double *sx = &splx[(size_t)i * order * 4], *sy = &sply[(size_t)i * order * 4],
                   *sz = &splz[(size_t)i * order * 4];
      const int i0g = igrid[3 * i], j0g = igrid[3 * i + 1];
      int k0 = igrid[3 * i + 2];
      double tuv[20] = {0};
      for (int a3 = 0; a3 < order; a3++) {
        const int kk = jmod(++k0, nfz);
        int j0 = j0g;
        double tu00 = 0, tu10 = 0, tu01 = 0, tu20 = 0, tu11 = 0, tu02 = 0, tu30 = 0, tu21 = 0, tu12 = 0, tu03 = 0;
        for (int a2 = 0; a2 < order; a2++) {
          const int jj = jmod(++j0, nfy);
          int ii0 = i0g;
          double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
          for (int a1 = 0; a1 < order; a1++) {
            const int ii = jmod(++ii0, nfx);
            const std::complex<double> &g = grid[((size_t)kk * nfy + jj) * nfx + ii];
            const double tq = part == 0 ? g.real() : g.imag();
            t0 = std::fma(tq, sx[a1 * 4], t0);
            t1 = std::fma(tq, sx[a1 * 4 + 1], t1);
            t2 = std::fma(tq, sx[a1 * 4 + 2], t2);
            t3 = std::fma(tq, sx[a1 * 4 + 3], t3);
          }
          const double u0 = sy[a2 * 4], u1 = sy[a2 * 4 + 1], u2 = sy[a2 * 4 + 2], u3 = sy[a2 * 4 + 3];
          tu00 = std::fma(t0, u0, tu00); tu10 = std::fma(t1, u0, tu10);
          tu01 = std::fma(t0, u1, tu01); tu20 = std::fma(t2, u0, tu20);
          tu11 = std::fma(t1, u1, tu11); tu02 = std::fma(t0, u2, tu02);
          tu30 = std::fma(t3, u0, tu30); tu21 = std::fma(t2, u1, tu21);
          tu12 = std::fma(t1, u2, tu12); tu03 = std::fma(t0, u3, tu03);
        }
        const double v0 = sz[a3 * 4], v1 = sz[a3 * 4 + 1], v2 = sz[a3 * 4 + 2], v3 = sz[a3 * 4 + 3];
        tuv[t000] = std::fma(tu00, v0, tuv[t000]); tuv[t100] = std::fma(tu10, v0, tuv[t100]);
        tuv[t010] = std::fma(tu01, v0, tuv[t010]); tuv[t001] = std::fma(tu00, v1, tuv[t001]);
        tuv[t200] = std::fma(tu20, v0, tuv[t200]); tuv[t020] = std::fma(tu02, v0, tuv[t020]);
        tuv[t002] = std::fma(tu00, v2, tuv[t002]); tuv[t110] = std::fma(tu11, v0, tuv[t110]);
        tuv[t101] = std::fma(tu10, v1, tuv[t101]); tuv[t011] = std::fma(tu01, v1, tuv[t011]);
        tuv[t300] = std::fma(tu30, v0, tuv[t300]); tuv[t030] = std::fma(tu03, v0, tuv[t030]);
        tuv[t003] = std::fma(tu00, v3, tuv[t003]); tuv[t210] = std::fma(tu21, v0, tuv[t210]);
        tuv[t201] = std::fma(tu20, v1, tuv[t201]); tuv[t120] = std::fma(tu12, v0, tuv[t120]);
        tuv[t021] = std::fma(tu02, v1, tuv[t021]); tuv[t102] = std::fma(tu10, v2, tuv[t102]);
        tuv[t012] = std::fma(tu01, v2, tuv[t012]); tuv[t111] = std::fma(tu11, v1, tuv[t111]);
      }
      double *fo = &frac[20 * (size_t)i];
      for (int t = 0; t < 20; t++) fo[t] = tuv[t];
      double *co = &cart[20 * (size_t)i];
      co[0] = tfm[0][0] * fo[0];
      for (int j = 1; j < 4; j++) {
        co[j] = 0.0;
        for (int k = 1; k < 4; k++) co[j] = std::fma(tfm[j][k], fo[k], co[j]);
      }
      for (int j = 4; j < 10; j++) {
        co[j] = 0.0;
        for (int k = 4; k < 10; k++) co[j] = std::fma(tfm[j][k], fo[k], co[j]);
      }
    }
  }

  // SpatialInducedLoop.gridDensity (ReciprocalSpace.java:1573-1628): Re = D, Im = CR.
  void spread_induced(const std::vector<double> &d, const std::vector<double> &pcr,
                      std::vector<std::complex<double>> &grid) {
    grid.assign((size_t)nfx * nfy * nfz, 0.0);
    for (int i = 0; i < n; i++) {
      if (!used(i)) continue;   // atoms not in use are not spread (ReciprocalSpace.java:2821, 2884)
      double u[3], q[3];
      for (int a = 0; a < 3; a++) {
        u[a] = afrac[a][0] * d[3 * i] + afrac[a][1] * d[3 * i + 1] + afrac[a][2] * d[3 * i + 2];
        q[a] = afrac[a][0] * pcr[3 * i] + afrac[a][1] * pcr[3 * i + 1] + afrac[a][2] * pcr[3 * i + 2];
      }
      const double *sx = &splx[(size_t)i * order * 4], *sy = &sply[(size_t)i * order * 4],
                   *sz = &splz[(size_t)i * order * 4];
      const int i0g = igrid[3 * i], j0g = igrid[3 * i + 1];
      int k0 = igrid[3 * i + 2];
      for (int a3 = 0; a3 < order; a3++) {
        const double v0 = sz[a3 * 4], v1 = sz[a3 * 4 + 1];
        const double dx0 = u[0] * v0, dy0 = u[1] * v0, dz1 = u[2] * v1;
        const double px0 = q[0] * v0, py0 = q[1] * v0, pz1 = q[2] * v1;
        const int kk = jmod(++k0, nfz);
        int j0 = j0g;
        for (int a2 = 0; a2 < order; a2++) {
          const double u0 = sy[a2 * 4], u1 = sy[a2 * 4 + 1];
          const double term0 = std::fma(dz1, u0, dy0 * u1);
          const double term1 = dx0 * u0;
          const double termp0 = std::fma(pz1, u0, py0 * u1);
          const double termp1 = px0 * u0;
          const int jj = jmod(++j0, nfy);
          int ii0 = i0g;
          for (int a1 = 0; a1 < order; a1++) {
            const int ii = jmod(++ii0, nfx);
            std::complex<double> &cur = grid[((size_t)kk * nfy + jj) * nfx + ii];
            const double re = std::fma(sx[a1 * 4], term0, std::fma(sx[a1 * 4 + 1], term1, cur.real()));
            const double im = std::fma(sx[a1 * 4], termp0, std::fma(sx[a1 * 4 + 1], termp1, cur.imag()));
            cur = std::complex<double>(re, im);
          }
        }
      }
    }
  }

  // ---------------------------------------------------------------------------
  // Masks.  pme/PermanentFieldRegion.java:231-258 (field), RealSpaceEnergyRegion.java:307-342 (energy).
  struct Masks {
    std::vector<double> energy, field, group;
  };

  // ---------------------------------------------------------------------------
  // PermanentRealSpaceFieldLoop (pme/PermanentFieldRegion.java:595-815); builds the
  // Ewald and preconditioner lists from the neighbour list.
  void permanent_field() {
    fieldD.assign(3 * (size_t)n, 0.0);
    fieldP.assign(3 * (size_t)n, 0.0);
    ewald.assign(n, {});
    precond.assign(n, {});
    esh.assign(multi_image ? n : 0, {});
    psh.assign(multi_image ? n : 0, {});
    std::vector<std::vector<double>> tD(nthreads, std::vector<double>(3 * (size_t)n, 0.0));
    std::vector<std::vector<double>> tP(nthreads, std::vector<double>(3 * (size_t)n, 0.0));
#pragma omp parallel
    {
      int tid = 0;
#ifdef _OPENMP
      tid = omp_get_thread_num();
#endif
      std::vector<double> &fd = tD[tid], &fp = tP[tid];
      std::vector<double> emask(n, 1.0), imask(n, 1.0);
#pragma omp for schedule(dynamic, 64)
      for (int i = 0; i < n; i++) {
        if (!used(i)) continue;
        double fix = 0, fiy = 0, fiz = 0, fixCR = 0, fiyCR = 0, fizCR = 0;
        const double pdi = ipdamp[i], pti = thole[i];
        const double xi = x[i], yi = y[i], zi = z[i];
        const double *mi = &gm[10 * (size_t)i];
        const double ci = mi[t000], dix = mi[t100], diy = mi[t010], diz = mi[t001];
        const double qixx = mi[t200] / 3.0, qiyy = mi[t020] / 3.0, qizz = mi[t002] / 3.0;
        const double qixy = mi[t110] / 3.0, qixz = mi[t101] / 3.0, qiyz = mi[t011] / 3.0;
        for (int k : m12[i]) emask[k] = p.p12;
        for (int k : m13[i]) emask[k] = p.p13;
        for (int k : m14[i]) {
          emask[k] = p.p14;
          for (int g : ip11[i]) if (g == k) { emask[k] = p.intra14 * p.p14; break; }
        }
        for (int g : ip11[i]) imask[g] = p.d11;
        for (size_t e = 0; e < nlist[i].size(); e++) {
          const int k = nlist[i][e];
          if (!used(k) || vapor_skip(i, k)) continue;
          double xr = x[k] - xi, yr = y[k] - yi, zr = z[k] - zi;
          const double r2 = disp(xr, yr, zr, nsh, i, e);
          if (!(r2 <= off2)) continue;
          ewald[i].push_back(k);
          if (multi_image) esh[i].push_back(nsh[i][e]);
          const bool prim = primary(nsh, i, e);
          const double pdk = ipdamp[k], ptk = thole[k];
          const double *mk = &gm[10 * (size_t)k];
          const double ck = mk[t000], dkx = mk[t100], dky = mk[t010], dkz = mk[t001];
          const double qkxx = mk[t200] / 3.0, qkyy = mk[t020] / 3.0, qkzz = mk[t002] / 3.0;
          const double qkxy = mk[t110] / 3.0, qkxz = mk[t101] / 3.0, qkyz = mk[t011] / 3.0;
          const double r = std::sqrt(r2);
          if (r < p.precond_cutoff) {
            precond[i].push_back(k);
            if (multi_image) psh[i].push_back(nsh[i][e]);
          }
          const double ralpha = aewald * r;
          const double exp2a = std::exp(-ralpha * ralpha);
          const double rr1 = 1.0 / r, rr2 = rr1 * rr1;
          const double bn0 = std::erfc(ralpha) * rr1;
          const double bn1 = (bn0 + an0 * exp2a) * rr2;
          const double bn2 = (3.0 * bn1 + an1 * exp2a) * rr2;
          const double bn3 = (5.0 * bn2 + an2 * exp2a) * rr2;
          double scale3 = 1.0, scale5 = 1.0, scale7 = 1.0;
          double damp = pdi * pdk;
          const double pgamma = std::min(pti, ptk);
          const double rdamp = r * damp;
          damp = -pgamma * rdamp * rdamp * rdamp;
          if (damp > -50.0) {
            const double expdamp = std::exp(damp);
            scale3 = 1.0 - expdamp;
            scale5 = 1.0 - expdamp * (1.0 - damp);
            scale7 = 1.0 - expdamp * (1.0 - damp + 0.6 * damp * damp);
          }
          const double scale = prim ? imask[k] : 1.0, scalep = prim ? emask[k] : 1.0;
          const double dsc3 = scale3 * scale, dsc5 = scale5 * scale, dsc7 = scale7 * scale;
          const double psc3 = scale3 * scalep, psc5 = scale5 * scalep, psc7 = scale7 * scalep;
          const double rr3 = rr1 * rr2, rr5 = 3.0 * rr3 * rr2, rr7 = 5.0 * rr5 * rr2;
          const double drr3 = (1.0 - dsc3) * rr3, drr5 = (1.0 - dsc5) * rr5, drr7 = (1.0 - dsc7) * rr7;
          const double prr3 = (1.0 - psc3) * rr3, prr5 = (1.0 - psc5) * rr5, prr7 = (1.0 - psc7) * rr7;
          const double dir = dix * xr + diy * yr + diz * zr;
          const double qix = 2.0 * (qixx * xr + qixy * yr + qixz * zr);
          const double qiy = 2.0 * (qixy * xr + qiyy * yr + qiyz * zr);
          const double qiz = 2.0 * (qixz * xr + qiyz * yr + qizz * zr);
          const double qir = (qix * xr + qiy * yr + qiz * zr) * 0.5;
          const double bn123i = bn1 * ci + bn2 * dir + bn3 * qir;
          const double fkmx = xr * bn123i - bn1 * dix - bn2 * qix;
          const double fkmy = yr * bn123i - bn1 * diy - bn2 * qiy;
          const double fkmz = zr * bn123i - bn1 * diz - bn2 * qiz;
          const double ddr357i = drr3 * ci + drr5 * dir + drr7 * qir;
          const double fkdx = xr * ddr357i - drr3 * dix - drr5 * qix;
          const double fkdy = yr * ddr357i - drr3 * diy - drr5 * qiy;
          const double fkdz = zr * ddr357i - drr3 * diz - drr5 * qiz;
          fd[3 * k] += fkmx - fkdx; fd[3 * k + 1] += fkmy - fkdy; fd[3 * k + 2] += fkmz - fkdz;
          const double prr357i = prr3 * ci + prr5 * dir + prr7 * qir;
          const double fkpx = xr * prr357i - prr3 * dix - prr5 * qix;
          const double fkpy = yr * prr357i - prr3 * diy - prr5 * qiy;
          const double fkpz = zr * prr357i - prr3 * diz - prr5 * qiz;
          fp[3 * k] += fkmx - fkpx; fp[3 * k + 1] += fkmy - fkpy; fp[3 * k + 2] += fkmz - fkpz;
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
          fix += fimx - fidx; fiy += fimy - fidy; fiz += fimz - fidz;
          const double prr357k = prr3 * ck - prr5 * dkr + prr7 * qkr;
          const double fipx = -xr * prr357k - prr3 * dkx + prr5 * qkx;
          const double fipy = -yr * prr357k - prr3 * dky + prr5 * qky;
          const double fipz = -zr * prr357k - prr3 * dkz + prr5 * qkz;
          fixCR += fimx - fipx; fiyCR += fimy - fipy; fizCR += fimz - fipz;
        }
        fd[3 * i] += fix; fd[3 * i + 1] += fiy; fd[3 * i + 2] += fiz;
        fp[3 * i] += fixCR; fp[3 * i + 1] += fiyCR; fp[3 * i + 2] += fizCR;
        for (int k : m12[i]) emask[k] = 1.0;
        for (int k : m13[i]) emask[k] = 1.0;
        for (int k : m14[i]) emask[k] = 1.0;
        for (int g : ip11[i]) imask[g] = 1.0;
      }
    }
    for (int t = 0; t < nthreads; t++)
      for (size_t j = 0; j < 3 * (size_t)n; j++) { fieldD[j] += tD[t][j]; fieldP[j] += tP[t][j]; }
  }

  // InducedDipoleFieldRegion real space (pme/InducedDipoleFieldRegion.java:308-470) on the
  // Ewald list with the given Ewald coefficient (0 plus the short list gives the
  // preconditioner field, PCGSolver.java:1254-1400).
  void dipole_field(const std::vector<double> &ud, const std::vector<double> &up,
                    const std::vector<std::vector<int>> &lists, const std::vector<std::vector<int>> &shifts,
                    double alpha,
                    std::vector<double> &outD, std::vector<double> &outP) {
    outD.assign(3 * (size_t)n, 0.0);
    outP.assign(3 * (size_t)n, 0.0);
    double a0 = 0.0, a1 = 0.0;
    if (alpha > 0.0) {
      const double alsq2 = 2.0 * alpha * alpha;
      a0 = alsq2 / (kSqrtPi * alpha);
      a1 = alsq2 * a0;
    }
    std::vector<std::vector<double>> tD(nthreads, std::vector<double>(3 * (size_t)n, 0.0));
    std::vector<std::vector<double>> tP(nthreads, std::vector<double>(3 * (size_t)n, 0.0));
#pragma omp parallel
    {
      int tid = 0;
#ifdef _OPENMP
      tid = omp_get_thread_num();
#endif
      std::vector<double> &fd = tD[tid], &fp = tP[tid];
#pragma omp for schedule(dynamic, 64)
      for (int i = 0; i < n; i++) {
        if (!used(i)) continue;
        double fx = 0, fy = 0, fz = 0, px = 0, py = 0, pz = 0;
        const double xi = x[i], yi = y[i], zi = z[i];
        const double pdi = ipdamp[i], pti = thole[i];
        const double uix = ud[3 * i], uiy = ud[3 * i + 1], uiz = ud[3 * i + 2];
        const double pix = up[3 * i], piy = up[3 * i + 1], piz = up[3 * i + 2];
        for (size_t e = 0; e < lists[i].size(); e++) {
          const int k = lists[i][e];
          if (!used(k) || vapor_skip(i, k)) continue;
          double xr = x[k] - xi, yr = y[k] - yi, zr = z[k] - zi;
          const double r2 = disp(xr, yr, zr, shifts, i, e);
          const double r = std::sqrt(r2);
          const double rr1 = 1.0 / r, rr2 = rr1 * rr1;
          const double ralpha = alpha * r;
          const double exp2a = std::exp(-ralpha * ralpha);
          const double bn0 = std::erfc(ralpha) * rr1;
          const double bn1 = (bn0 + a0 * exp2a) * rr2;
          const double bn2 = (3.0 * bn1 + a1 * exp2a) * rr2;
          double scale3 = 1.0, scale5 = 1.0;
          double damp = pdi * ipdamp[k];
          const double pgamma = std::min(pti, thole[k]);
          const double rdamp = r * damp;
          damp = -pgamma * rdamp * rdamp * rdamp;
          if (damp > -50.0) {
            const double expdamp = std::exp(damp);
            scale3 = 1.0 - expdamp;
            scale5 = 1.0 - expdamp * (1.0 - damp);
          }
          double rr3 = rr1 * rr2;
          double rr5 = 3.0 * rr3 * rr2;
          rr3 *= (1.0 - scale3);
          rr5 *= (1.0 - scale5);
          const double ukx = ud[3 * k], uky = ud[3 * k + 1], ukz = ud[3 * k + 2];
          const double ukr = ukx * xr + uky * yr + ukz * zr;
          const double bn2ukr = bn2 * ukr, rr5ukr = rr5 * ukr;
          fx += (-bn1 * ukx + bn2ukr * xr) - (-rr3 * ukx + rr5ukr * xr);
          fy += (-bn1 * uky + bn2ukr * yr) - (-rr3 * uky + rr5ukr * yr);
          fz += (-bn1 * ukz + bn2ukr * zr) - (-rr3 * ukz + rr5ukr * zr);
          const double pkx = up[3 * k], pky = up[3 * k + 1], pkz = up[3 * k + 2];
          const double pkr = pkx * xr + pky * yr + pkz * zr;
          const double bn2pkr = bn2 * pkr, rr5pkr = rr5 * pkr;
          px += (-bn1 * pkx + bn2pkr * xr) - (-rr3 * pkx + rr5pkr * xr);
          py += (-bn1 * pky + bn2pkr * yr) - (-rr3 * pky + rr5pkr * yr);
          pz += (-bn1 * pkz + bn2pkr * zr) - (-rr3 * pkz + rr5pkr * zr);
          const double uir = uix * xr + uiy * yr + uiz * zr;
          const double bn2uir = bn2 * uir, rr5uir = rr5 * uir;
          fd[3 * k] += (-bn1 * uix + bn2uir * xr) - (-rr3 * uix + rr5uir * xr);
          fd[3 * k + 1] += (-bn1 * uiy + bn2uir * yr) - (-rr3 * uiy + rr5uir * yr);
          fd[3 * k + 2] += (-bn1 * uiz + bn2uir * zr) - (-rr3 * uiz + rr5uir * zr);
          const double pir = pix * xr + piy * yr + piz * zr;
          const double bn2pir = bn2 * pir, rr5pir = rr5 * pir;
          fp[3 * k] += (-bn1 * pix + bn2pir * xr) - (-rr3 * pix + rr5pir * xr);
          fp[3 * k + 1] += (-bn1 * piy + bn2pir * yr) - (-rr3 * piy + rr5pir * yr);
          fp[3 * k + 2] += (-bn1 * piz + bn2pir * zr) - (-rr3 * piz + rr5pir * zr);
        }
        fd[3 * i] += fx; fd[3 * i + 1] += fy; fd[3 * i + 2] += fz;
        fp[3 * i] += px; fp[3 * i + 1] += py; fp[3 * i + 2] += pz;
      }
    }
    for (int t = 0; t < nthreads; t++)
      for (size_t j = 0; j < 3 * (size_t)n; j++) { outD[j] += tD[t][j]; outP[j] += tP[t][j]; }
  }

  // ParticleMeshEwald.computeInduceDipoleField (ParticleMeshEwald.java:763-803) with
  // InducedDipoleFieldReduceRegion (pme/InducedDipoleFieldReduceRegion.java:159-207).
  void induced_field(const std::vector<double> &ud, const std::vector<double> &up,
                     std::vector<double> &outD, std::vector<double> &outP) {
    if (recip_on) {
      std::vector<std::complex<double>> grid;
      spread_induced(ud, up, grid);
      convolve(grid);
      interpolate(grid, 0, fphiI, cphiI);
      interpolate(grid, 1, fphiP, cphiP);
    } else {
      cphiI.assign(20 * (size_t)n, 0.0); cphiP.assign(20 * (size_t)n, 0.0);
      fphiI.assign(20 * (size_t)n, 0.0); fphiP.assign(20 * (size_t)n, 0.0);
    }
    dipole_field(ud, up, ewald, esh, aewald, outD, outP);
    for (int i = 0; i < n; i++)
      for (int a = 0; a < 3; a++) {
        outD[3 * i + a] += aewald3 * ud[3 * i + a] - cphiI[20 * (size_t)i + 1 + a];
        outP[3 * i + a] += aewald3 * up[3 * i + a] - cphiP[20 * (size_t)i + 1 + a];
      }
  }

  // PCGSolver.scfByPCG (pme/PCGSolver.java:487-602) with its regions (:609-1180).
  int pcg() {
    const size_t m = 3 * (size_t)n;
    std::vector<double> r(m), rCR(m), z(m), zCR(m), pv(m), pCR(m), vec(m), vecCR(m);
    std::vector<double> fD, fP, preD, preP;
    // Field of the direct dipoles.
    induced_field(uD, uP, fD, fP);
    for (int i = 0; i < n; i++) {
      const bool ok = pol_eff[i] > 0.0;
      const double ip = ok ? 1.0 / pol_eff[i] : 0.0;
      for (int a = 0; a < 3; a++) {
        const size_t j = 3 * (size_t)i + a;
        r[j] = ok ? (udir[j] - uD[j]) * ip + fD[j] : 0.0;
        rCR[j] = ok ? (udirP[j] - uP[j]) * ip + fP[j] : 0.0;
      }
    }
    auto precondition = [&]() {
      std::vector<double> ur(m), pr(m);
      for (int i = 0; i < n; i++)
        for (int a = 0; a < 3; a++) {
          ur[3 * i + a] = pol_eff[i] * r[3 * i + a];
          pr[3 * i + a] = pol_eff[i] * rCR[3 * i + a];
        }
      dipole_field(ur, pr, precond, psh, 0.0, preD, preP);
    };
    precondition();
    for (int i = 0; i < n; i++)
      for (int a = 0; a < 3; a++) {
        const size_t j = 3 * (size_t)i + a;
        z[j] = pol_eff[i] * (preD[j] + p.precond_scale * r[j]);
        zCR[j] = pol_eff[i] * (preP[j] + p.precond_scale * rCR[j]);
        pv[j] = z[j]; pCR[j] = zCR[j];
      }
    int iter = 0;
    double eps = 100.0;
    while (true) {
      std::vector<double> Ap, ApCR;
      induced_field(pv, pCR, Ap, ApCR);
      double pAp = 0, pApCR = 0, rz = 0, rzCR = 0;
      for (int i = 0; i < n; i++) {
        const bool ok = pol_eff[i] > 0.0;
        const double ip = ok ? 1.0 / pol_eff[i] : 0.0;
        for (int a = 0; a < 3; a++) {
          const size_t j = 3 * (size_t)i + a;
          vec[j] = ok ? pv[j] * ip - Ap[j] : 0.0;
          vecCR[j] = ok ? pCR[j] * ip - ApCR[j] : 0.0;
          pAp += pv[j] * vec[j];
          pApCR += pCR[j] * vecCR[j];
          rz += r[j] * z[j];
          rzCR += rCR[j] * zCR[j];
        }
      }
      const double alpha = (pAp != 0.0) ? rz / pAp : rz;
      const double alphaCR = (pApCR != 0.0) ? rzCR / pApCR : rzCR;
      double e1 = 0.0, e2 = 0.0;
      for (size_t j = 0; j < m; j++) {
        r[j] -= alpha * vec[j];
        rCR[j] -= alphaCR * vecCR[j];
        uD[j] += alpha * pv[j];
        uP[j] += alphaCR * pCR[j];
        e1 += r[j] * r[j];
        e2 += rCR[j] * rCR[j];
      }
      const double previous = eps;
      eps = kElecAngToDebye * std::sqrt(std::max(e1, e2) / (double)n);
      iter++;
      if (eps > previous) { scf_iter = iter; return FFXG_ERR_SCF_DIVERGED; }
      if (iter >= p.max_scf_iter) { scf_iter = iter; return FFXG_ERR_SCF_MAXITER; }
      if (eps < p.polar_eps) break;
      precondition();
      double rzNew = 0, rzNewCR = 0;
      for (int i = 0; i < n; i++)
        for (int a = 0; a < 3; a++) {
          const size_t j = 3 * (size_t)i + a;
          z[j] = pol_eff[i] * (preD[j] + p.precond_scale * r[j]);
          zCR[j] = pol_eff[i] * (preP[j] + p.precond_scale * rCR[j]);
          rzNew += r[j] * z[j];
          rzNewCR += rCR[j] * zCR[j];
        }
      const double beta = rzNew / (rz == 0.0 ? 1.0 : rz);
      const double betaCR = rzNewCR / (rzCR == 0.0 ? 1.0 : rzCR);
      for (size_t j = 0; j < m; j++) {
        pv[j] = z[j] + beta * pv[j];
        pCR[j] = zCR[j] + betaCR * pCR[j];
      }
    }
    scf_iter = iter;
    return FFXG_OK;
  }

  // ---------------------------------------------------------------------------
  // Reciprocal-space energy, gradient and torque, pme/ReciprocalEnergyRegion.java:381-740.
  void recip_energy(bool gradient, double &eSelf, double &eRecip, double &eCorr, double &eSelfI,
                    double &eRecipI) {
    const double electric = p.electric;
    const double aewald1 = -electric * aewald / kSqrtPi;
    const double aewald2 = 2.0 * aewald * aewald;
    const double aw3 = -2.0 / 3.0 * electric * aewald * aewald * aewald / kSqrtPi;
    const double aw4 = -2.0 * aw3;
    eSelf = eRecip = eSelfI = eRecipI = 0.0;
    const bool gr = gradient || lam;      // lambda derivatives need the forces (PME:940)
    // Scales of the lambda scheme (ReciprocalEnergyRegion.java:230-255, 385-530, 545-740):
    // permanent parts x permScale, induced parts x polScale; dU/dL picks up
    // dEdLSign * dlPow * (the unscaled contribution).
    const double lP = lam ? dEdLSign * g_alch.dlPowPerm : 0.0, l2P = lam ? dEdLSign * g_alch.d2lPowPerm : 0.0;
    const double lI = lam ? dEdLSign * g_alch.dlPowPol : 0.0, l2I = lam ? dEdLSign * g_alch.d2lPowPol : 0.0;
    double qtot = 0.0;
    for (int i = 0; i < n; i++) {
      if (!used(i)) continue;
      const double *in = &gm[10 * (size_t)i];
      qtot += in[t000];
      const double cii = in[t000] * in[t000];
      const double dii = in[t100] * in[t100] + in[t010] * in[t010] + in[t001] * in[t001];
      const double qii = in[t200] * in[t200] + in[t020] * in[t020] + in[t002] * in[t002] +
                         2.0 * (in[t110] * in[t110] + in[t101] * in[t101] + in[t011] * in[t011]);
      eSelf += aewald1 * (cii + aewald2 * (dii / 3.0 + 2.0 * aewald2 * qii / 45.0));
    }
    eDL += lP * eSelf;
    eD2L += l2P * eSelf;
    eSelf *= permScale;
    const int nf[3] = {nfx, nfy, nfz};
    double dUdL = 0.0, d2UdL2 = 0.0;
    for (int i = 0; i < n; i++) {
      if (!used(i)) continue;
      const double *ph = &cphi[20 * (size_t)i];
      const double *mp = &gm[10 * (size_t)i];
      const double *f = &fm[10 * (size_t)i];
      const double e = mp[t000] * ph[t000] + mp[t100] * ph[t100] + mp[t010] * ph[t010] + mp[t001] * ph[t001] +
                       (1.0 / 3.0) * (mp[t200] * ph[t200] + mp[t020] * ph[t020] + mp[t002] * ph[t002] +
                                      2.0 * (mp[t110] * ph[t110] + mp[t101] * ph[t101] + mp[t011] * ph[t011]));
      eRecip += e;
      dUdL += lP * e;
      d2UdL2 += l2P * e;
      if (!gr) continue;
      const double *fp = &fphi[20 * (size_t)i];
      double gx = f[t000] * fp[t100] + f[t100] * fp[t200] + f[t010] * fp[t110] + f[t001] * fp[t101] +
                  f[t200] * fp[t300] + f[t020] * fp[t120] + f[t002] * fp[t102] + f[t110] * fp[t210] +
                  f[t101] * fp[t201] + f[t011] * fp[t111];
      double gy = f[t000] * fp[t010] + f[t100] * fp[t110] + f[t010] * fp[t020] + f[t001] * fp[t011] +
                  f[t200] * fp[t210] + f[t020] * fp[t030] + f[t002] * fp[t012] + f[t110] * fp[t120] +
                  f[t101] * fp[t111] + f[t011] * fp[t021];
      double gz = f[t000] * fp[t001] + f[t100] * fp[t101] + f[t010] * fp[t011] + f[t001] * fp[t002] +
                  f[t200] * fp[t201] + f[t020] * fp[t021] + f[t002] * fp[t003] + f[t110] * fp[t111] +
                  f[t101] * fp[t102] + f[t011] * fp[t012];
      gx *= nf[0]; gy *= nf[1]; gz *= nf[2];
      const double dfx = cell.A[0][0] * gx + cell.A[0][1] * gy + cell.A[0][2] * gz;
      const double dfy = cell.A[1][0] * gx + cell.A[1][1] * gy + cell.A[1][2] * gz;
      const double dfz = cell.A[2][0] * gx + cell.A[2][1] * gy + cell.A[2][2] * gz;
      double tqx = -mp[t010] * ph[t001] + mp[t001] * ph[t010];
      double tqy = -mp[t001] * ph[t100] + mp[t100] * ph[t001];
      double tqz = -mp[t100] * ph[t010] + mp[t010] * ph[t100];
      tqx -= (2.0 / 3.0) * (mp[t110] * ph[t101] + mp[t020] * ph[t011] + mp[t011] * ph[t002] -
                            mp[t101] * ph[t110] - mp[t011] * ph[t020] - mp[t002] * ph[t011]);
      tqy -= (2.0 / 3.0) * (mp[t101] * ph[t200] + mp[t011] * ph[t110] + mp[t002] * ph[t101] -
                            mp[t200] * ph[t101] - mp[t110] * ph[t011] - mp[t101] * ph[t002]);
      tqz -= (2.0 / 3.0) * (mp[t200] * ph[t110] + mp[t110] * ph[t020] + mp[t101] * ph[t011] -
                            mp[t110] * ph[t200] - mp[t020] * ph[t110] - mp[t011] * ph[t101]);
      const double fs = permScale * electric;
      grad[3 * i] += fs * dfx; grad[3 * i + 1] += fs * dfy; grad[3 * i + 2] += fs * dfz;
      torque[3 * i] += fs * tqx; torque[3 * i + 1] += fs * tqy; torque[3 * i + 2] += fs * tqz;
      if (lam) {
        const double fl = lP * electric;
        lgE[3 * i] += fl * dfx; lgE[3 * i + 1] += fl * dfy; lgE[3 * i + 2] += fl * dfz;
        ltE[3 * i] += fl * tqx; ltE[3 * i + 1] += fl * tqy; ltE[3 * i + 2] += fl * tqz;
      }
    }
    eDL += 0.5 * dUdL * electric;
    eD2L += 0.5 * d2UdL2 * electric;
    eRecip *= permScale * 0.5 * electric;
    eCorr = 0.0;
    if (qtot != 0.0) {
      eCorr = -0.5 * electric * kPi * (qtot * qtot) / (cell.volume * aewald * aewald);
      eDL += lP * eCorr;
      eD2L += l2P * eCorr;
      eCorr *= permScale;
    }
    if (p.polarization == FFXG_POLAR_NONE || !doPol) return;
    for (int i = 0; i < n; i++) {
      if (!used(i)) continue;
      const double *mp = &gm[10 * (size_t)i];
      const double dii = uD[3 * i] * mp[t100] + uD[3 * i + 1] * mp[t010] + uD[3 * i + 2] * mp[t001];
      eSelfI += aw3 * dii;
    }
    eDL += lI * eSelfI;
    eD2L += l2I * eSelfI;
    eSelfI *= polScale;
    if (gr) {
      for (int i = 0; i < n; i++) {
        if (!used(i)) continue;
        const double *mp = &gm[10 * (size_t)i];
        const double dix = mp[t100], diy = mp[t010], diz = mp[t001];
        const double uix = 0.5 * (uD[3 * i] + uP[3 * i]);
        const double uiy = 0.5 * (uD[3 * i + 1] + uP[3 * i + 1]);
        const double uiz = 0.5 * (uD[3 * i + 2] + uP[3 * i + 2]);
        const double tx = aw4 * (diy * uiz - diz * uiy), ty = aw4 * (diz * uix - dix * uiz),
                     tz = aw4 * (dix * uiy - diy * uix);
        torque[3 * i] += polScale * tx; torque[3 * i + 1] += polScale * ty; torque[3 * i + 2] += polScale * tz;
        if (lam) { ltE[3 * i] += lI * tx; ltE[3 * i + 1] += lI * ty; ltE[3 * i + 2] += lI * tz; }
      }
    }
    for (int i = 0; i < n; i++) {
      if (!used(i)) continue;
      const double *fP = &fphi[20 * (size_t)i];
      double fi[3], fiCR[3];
      for (int a = 0; a < 3; a++) {
        fi[a] = afrac[a][0] * uD[3 * i] + afrac[a][1] * uD[3 * i + 1] + afrac[a][2] * uD[3 * i + 2];
        fiCR[a] = afrac[a][0] * uP[3 * i] + afrac[a][1] * uP[3 * i + 1] + afrac[a][2] * uP[3 * i + 2];
      }
      const double indx = fi[0], indy = fi[1], indz = fi[2];
      eRecipI += indx * fP[t100] + indy * fP[t010] + indz * fP[t001];
      if (!gr) continue;
      const double *iPhi = &cphiI[20 * (size_t)i], *iCRPhi = &cphiP[20 * (size_t)i];
      const double *fiPhi = &fphiI[20 * (size_t)i], *fiCRPhi = &fphiP[20 * (size_t)i];
      const double *mp = &gm[10 * (size_t)i];
      const double *f = &fm[10 * (size_t)i];
      const double inpx = fiCR[0], inpy = fiCR[1], inpz = fiCR[2];
      const double insx = indx + inpx, insy = indy + inpy, insz = indz + inpz;
      double sPhi[20], sfPhi[20];
      for (int t = 0; t < 20; t++) { sPhi[t] = 0.5 * (iPhi[t] + iCRPhi[t]); sfPhi[t] = fiPhi[t] + fiCRPhi[t]; }
      double gx = insx * fP[t200] + insy * fP[t110] + insz * fP[t101];
      double gy = insx * fP[t110] + insy * fP[t020] + insz * fP[t011];
      double gz = insx * fP[t101] + insy * fP[t011] + insz * fP[t002];
      if (p.polarization == FFXG_POLAR_MUTUAL) {
        gx += indx * fiCRPhi[t200] + inpx * fiPhi[t200] + indy * fiCRPhi[t110] + inpy * fiPhi[t110] +
              indz * fiCRPhi[t101] + inpz * fiPhi[t101];
        gy += indx * fiCRPhi[t110] + inpx * fiPhi[t110] + indy * fiCRPhi[t020] + inpy * fiPhi[t020] +
              indz * fiCRPhi[t011] + inpz * fiPhi[t011];
        gz += indx * fiCRPhi[t101] + inpx * fiPhi[t101] + indy * fiCRPhi[t011] + inpy * fiPhi[t011] +
              indz * fiCRPhi[t002] + inpz * fiPhi[t002];
      }
      gx += f[t000] * sfPhi[t100] + f[t100] * sfPhi[t200] + f[t010] * sfPhi[t110] + f[t001] * sfPhi[t101] +
            f[t200] * sfPhi[t300] + f[t020] * sfPhi[t120] + f[t002] * sfPhi[t102] + f[t110] * sfPhi[t210] +
            f[t101] * sfPhi[t201] + f[t011] * sfPhi[t111];
      gy += f[t000] * sfPhi[t010] + f[t100] * sfPhi[t110] + f[t010] * sfPhi[t020] + f[t001] * sfPhi[t011] +
            f[t200] * sfPhi[t210] + f[t020] * sfPhi[t030] + f[t002] * sfPhi[t012] + f[t110] * sfPhi[t120] +
            f[t101] * sfPhi[t111] + f[t011] * sfPhi[t021];
      gz += f[t000] * sfPhi[t001] + f[t100] * sfPhi[t101] + f[t010] * sfPhi[t011] + f[t001] * sfPhi[t002] +
            f[t200] * sfPhi[t201] + f[t020] * sfPhi[t021] + f[t002] * sfPhi[t003] + f[t110] * sfPhi[t111] +
            f[t101] * sfPhi[t102] + f[t011] * sfPhi[t012];
      gx *= nf[0]; gy *= nf[1]; gz *= nf[2];
      double dfx = cell.A[0][0] * gx + cell.A[0][1] * gy + cell.A[0][2] * gz;
      double dfy = cell.A[1][0] * gx + cell.A[1][1] * gy + cell.A[1][2] * gz;
      double dfz = cell.A[2][0] * gx + cell.A[2][1] * gy + cell.A[2][2] * gz;
      dfx *= 0.5 * electric; dfy *= 0.5 * electric; dfz *= 0.5 * electric;
      double tqx = -mp[t010] * sPhi[t001] + mp[t001] * sPhi[t010];
      double tqy = -mp[t001] * sPhi[t100] + mp[t100] * sPhi[t001];
      double tqz = -mp[t100] * sPhi[t010] + mp[t010] * sPhi[t100];
      tqx -= (2.0 / 3.0) * (mp[t110] * sPhi[t101] + mp[t020] * sPhi[t011] + mp[t011] * sPhi[t002] -
                            mp[t101] * sPhi[t110] - mp[t011] * sPhi[t020] - mp[t002] * sPhi[t011]);
      tqy -= (2.0 / 3.0) * (mp[t101] * sPhi[t200] + mp[t011] * sPhi[t110] + mp[t002] * sPhi[t101] -
                            mp[t200] * sPhi[t101] - mp[t110] * sPhi[t011] - mp[t101] * sPhi[t002]);
      tqz -= (2.0 / 3.0) * (mp[t200] * sPhi[t110] + mp[t110] * sPhi[t020] + mp[t101] * sPhi[t011] -
                            mp[t110] * sPhi[t200] - mp[t020] * sPhi[t110] - mp[t011] * sPhi[t101]);
      grad[3 * i] += polScale * dfx; grad[3 * i + 1] += polScale * dfy; grad[3 * i + 2] += polScale * dfz;
      const double ft = polScale * electric;
      torque[3 * i] += ft * tqx; torque[3 * i + 1] += ft * tqy; torque[3 * i + 2] += ft * tqz;
      if (lam) {
        lgE[3 * i] += lI * dfx; lgE[3 * i + 1] += lI * dfy; lgE[3 * i + 2] += lI * dfz;
        const double fl = lI * electric;
        ltE[3 * i] += fl * tqx; ltE[3 * i + 1] += fl * tqy; ltE[3 * i + 2] += fl * tqz;
      }
    }
    eRecipI *= 0.5 * electric;
    eDL += lI * eRecipI;
    eD2L += l2I * eRecipI;
    eRecipI *= polScale;
  }

  // ---------------------------------------------------------------------------
  // Real-space permanent and polarization energy, force and torque:
  // pme/RealSpaceEnergyRegion.java:822-1183 (chunk), :1190-1476 (permanentPair),
  // :1700-2177 (polarizationPair).  Returns energies in kcal/mol.
  void real_energy(bool gradient, double &ePerm, double &ePol, int64_t &count) {
    const double electric = p.electric;
    double eP = 0.0, eI = 0.0, eDLt = 0.0, eD2Lt = 0.0;
    int64_t cnt = 0;
    const bool polOn = p.polarization != FFXG_POLAR_NONE && doPol;
    const bool gr = gradient || lam;
    std::vector<std::vector<double>> tg(nthreads, std::vector<double>(3 * (size_t)n, 0.0));
    std::vector<std::vector<double>> tt(nthreads, std::vector<double>(3 * (size_t)n, 0.0));
    std::vector<std::vector<double>> tlg(lam ? nthreads : 0, std::vector<double>(3 * (size_t)n, 0.0));
    std::vector<std::vector<double>> tlt(lam ? nthreads : 0, std::vector<double>(3 * (size_t)n, 0.0));
#pragma omp parallel reduction(+ : eP, eI, cnt, eDLt, eD2Lt)
    {
      int tid = 0;
#ifdef _OPENMP
      tid = omp_get_thread_num();
#endif
      std::vector<double> &g = tg[tid], &tq = tt[tid];
      std::vector<double> *lgp = lam ? &tlg[tid] : nullptr, *ltp = lam ? &tlt[tid] : nullptr;
      std::vector<double> mmask(n, 1.0), pmask(n, 1.0), dmask(n, 1.0);
#pragma omp for schedule(dynamic, 64)
      for (int i = 0; i < n; i++) {
        if (!used(i)) continue;
        for (int k : m12[i]) { pmask[k] = p.p12; mmask[k] = p.m12; }
        for (int k : m13[i]) { pmask[k] = p.p13; mmask[k] = p.m13; }
        for (int k : m14[i]) {
          pmask[k] = p.p14; mmask[k] = p.m14;
          for (int gg : ip11[i]) if (gg == k) { pmask[k] = p.intra14 * p.p14; break; }
        }
        for (int k : m15[i]) mmask[k] = p.m15;
        for (int gg : ip11[i]) dmask[gg] = p.d11;
        const double xi = x[i], yi = y[i], zi = z[i];
        const double *mi = &gm[10 * (size_t)i];
        const double ci = mi[t000], dix = mi[t100], diy = mi[t010], diz = mi[t001];
        const double qixx = mi[t200] / 3.0, qiyy = mi[t020] / 3.0, qizz = mi[t002] / 3.0;
        const double qixy = mi[t110] / 3.0, qixz = mi[t101] / 3.0, qiyz = mi[t011] / 3.0;
        const double uix = uD[3 * i], uiy = uD[3 * i + 1], uiz = uD[3 * i + 2];
        const double pix = uP[3 * i], piy = uP[3 * i + 1], piz = uP[3 * i + 2];
        const double pdi = ipdamp[i], pti = thole[i];
        for (size_t e = 0; e < ewald[i].size(); e++) {
          const int k = ewald[i][e];
          if (!used(k) || vapor_skip(i, k)) continue;
          double xr = x[k] - xi, yr = y[k] - yi, zr = z[k] - zi;
          const double r2 = disp(xr, yr, zr, esh, i, e);
          const bool prim = primary(esh, i, e);
          // Softcore pairs (RealSpaceEnergyRegion.java:873-883): a soft atom in the pair and
          // permanent real space on: r^2 + lAlpha and the permanent scale l2.
          const bool soft = lam && (g_alch.soft[i] || g_alch.soft[k]);
          double beta = 0.0, l2 = 1.0;
          if (soft && doPermReal) { beta = stepAlpha; l2 = permScale; }
          const double *mk = &gm[10 * (size_t)k];
          const double ck = mk[t000], dkx = mk[t100], dky = mk[t010], dkz = mk[t001];
          const double qkxx = mk[t200] / 3.0, qkyy = mk[t020] / 3.0, qkzz = mk[t002] / 3.0;
          const double qkxy = mk[t110] / 3.0, qkxz = mk[t101] / 3.0, qkyz = mk[t011] / 3.0;
          const double ukx = uD[3 * k], uky = uD[3 * k + 1], ukz = uD[3 * k + 2];
          const double pkx = uP[3 * k], pky = uP[3 * k + 1], pkz = uP[3 * k + 2];
          const double scale = prim ? mmask[k] : 1.0, scalep = prim ? pmask[k] : 1.0;
          const double scaled = prim ? dmask[k] : 1.0;
          const double r = std::sqrt(r2 + beta);
          const double ralpha = aewald * r;
          const double exp2a = std::exp(-ralpha * ralpha);
          const double rr1 = 1.0 / r, rr2 = rr1 * rr1;
          const double bn0 = std::erfc(ralpha) * rr1;
          const double bn1 = (bn0 + an0 * exp2a) * rr2;
          const double bn2 = (3.0 * bn1 + an1 * exp2a) * rr2;
          const double bn3 = (5.0 * bn2 + an2 * exp2a) * rr2;
          const double bn4 = (7.0 * bn3 + an3 * exp2a) * rr2;
          const double bn5 = (9.0 * bn4 + an4 * exp2a) * rr2;
          const double bn6 = (11.0 * bn5 + an5 * exp2a) * rr2;
          const double rr3 = rr1 * rr2, rr5 = 3.0 * rr3 * rr2, rr7 = 5.0 * rr5 * rr2;
          const double rr9 = 7.0 * rr7 * rr2, rr11 = 9.0 * rr9 * rr2, rr13 = 11.0 * rr11 * rr2;
          double scale3 = 1.0, scale5 = 1.0, scale7 = 1.0;
          double ddsc3x = 0, ddsc3y = 0, ddsc3z = 0, ddsc5x = 0, ddsc5y = 0, ddsc5z = 0, ddsc7x = 0, ddsc7y = 0, ddsc7z = 0;
          double damp = pdi * ipdamp[k];
          const double tho = std::min(pti, thole[k]);
          const double rdamp = r * damp;
          damp = -tho * rdamp * rdamp * rdamp;
          if (damp > -50.0) {
            const double expdamp = std::exp(damp);
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
          if (doPermReal) {
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
            if (e != 0.0) { eP += l2 * e; cnt++; }
            if (gr) {
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
              const double pre = electric * l2;
              g[3 * i] += pre * ftm2x; g[3 * i + 1] += pre * ftm2y; g[3 * i + 2] += pre * ftm2z;
              tq[3 * i] += pre * ttm2x; tq[3 * i + 1] += pre * ttm2y; tq[3 * i + 2] += pre * ttm2z;
              g[3 * k] -= pre * ftm2x; g[3 * k + 1] -= pre * ftm2y; g[3 * k + 2] -= pre * ftm2z;
              tq[3 * k] += pre * ttm3x; tq[3 * k + 1] += pre * ttm3y; tq[3 * k + 2] += pre * ttm3z;
              if (soft) {   // dU/dL/dX of the first term, d[dlPow * ereal]/dX (:1465-1475)
                const double pf = electric * dEdLSign * g_alch.dlPowPerm;
                std::vector<double> &lg = *lgp, &lt = *ltp;
                lg[3 * i] += pf * ftm2x; lg[3 * i + 1] += pf * ftm2y; lg[3 * i + 2] += pf * ftm2z;
                lt[3 * i] += pf * ttm2x; lt[3 * i + 1] += pf * ttm2y; lt[3 * i + 2] += pf * ttm2z;
                lg[3 * k] -= pf * ftm2x; lg[3 * k + 1] -= pf * ftm2y; lg[3 * k + 2] -= pf * ftm2z;
                lt[3 * k] += pf * ttm3x; lt[3 * k + 1] += pf * ttm3y; lt[3 * k + 2] += pf * ttm3z;
              }
            }
            if (soft) {
              // dU/dL and d2U/dL2 of the pair through the scale and the softcore shift, and
              // dU/dL/dX of the second term with every radial order one higher (:1477-1690).
              const double dRealdL = gl0 * bn1 + (gl1 + gl6) * bn2 + (gl2 + gl7 + gl8) * bn3 + (gl3 + gl5) * bn4 + gl4 * bn5;
              const double d2RealdL2 = gl0 * bn2 + (gl1 + gl6) * bn3 + (gl2 + gl7 + gl8) * bn4 + (gl3 + gl5) * bn5 + gl4 * bn6;
              const double dlP = g_alch.dlPowPerm, d2lP = g_alch.d2lPowPerm;
              eDLt += dEdLSign * dlP * ereal + l2 * stepDlAlpha * dRealdL;
              eD2Lt += dEdLSign * (d2lP * ereal + dlP * stepDlAlpha * dRealdL + dlP * stepDlAlpha * dRealdL) +
                       l2 * stepD2lAlpha * dRealdL + l2 * stepDlAlpha * stepDlAlpha * d2RealdL2;
              double dFixdL = gl0 * rr3 + (gl1 + gl6) * rr5 + (gl2 + gl7 + gl8) * rr7 + (gl3 + gl5) * rr9 + gl4 * rr11;
              double d2FixdL2 = gl0 * rr5 + (gl1 + gl6) * rr7 + (gl2 + gl7 + gl8) * rr9 + (gl3 + gl5) * rr11 + gl4 * rr13;
              dFixdL *= scale1;
              d2FixdL2 *= scale1;
              eDLt -= dEdLSign * dlP * efix + l2 * stepDlAlpha * dFixdL;
              eD2Lt -= dEdLSign * (d2lP * efix + dlP * stepDlAlpha * dFixdL + dlP * stepDlAlpha * dFixdL) +
                       l2 * stepD2lAlpha * dFixdL + l2 * stepDlAlpha * stepDlAlpha * d2FixdL2;
              const double gf1 = bn2 * gl0 + bn3 * (gl1 + gl6) + bn4 * (gl2 + gl7 + gl8) + bn5 * (gl3 + gl5) + bn6 * gl4;
              const double gf2 = -ck * bn2 + sc4 * bn3 - sc6 * bn4;
              const double gf3 = ci * bn2 + sc3 * bn3 + sc5 * bn4;
              const double gf4 = 2.0 * bn3;
              const double gf5 = 2.0 * (-ck * bn3 + sc4 * bn4 - sc6 * bn5);
              const double gf6 = 2.0 * (-ci * bn3 - sc3 * bn4 - sc5 * bn5);
              const double gf7 = 4.0 * bn4;
              double ftm2x = gf1 * xr + gf2 * dix + gf3 * dkx + gf4 * (qkdix - qidkx) + gf5 * qirx + gf6 * qkrx + gf7 * (qiqkrx + qkqirx);
              double ftm2y = gf1 * yr + gf2 * diy + gf3 * dky + gf4 * (qkdiy - qidky) + gf5 * qiry + gf6 * qkry + gf7 * (qiqkry + qkqiry);
              double ftm2z = gf1 * zr + gf2 * diz + gf3 * dkz + gf4 * (qkdiz - qidkz) + gf5 * qirz + gf6 * qkrz + gf7 * (qiqkrz + qkqirz);
              double ttm2x = -bn2 * dixdkx + gf2 * dixrx + gf4 * (dixqkrx + dkxqirx + rxqidkx - 2.0 * qixqkx) - gf5 * rxqirx - gf7 * (rxqikrx + qkrxqirx);
              double ttm2y = -bn2 * dixdky + gf2 * dixry + gf4 * (dixqkry + dkxqiry + rxqidky - 2.0 * qixqky) - gf5 * rxqiry - gf7 * (rxqikry + qkrxqiry);
              double ttm2z = -bn2 * dixdkz + gf2 * dixrz + gf4 * (dixqkrz + dkxqirz + rxqidkz - 2.0 * qixqkz) - gf5 * rxqirz - gf7 * (rxqikrz + qkrxqirz);
              double ttm3x = bn2 * dixdkx + gf3 * dkxrx - gf4 * (dixqkrx + dkxqirx + rxqkdix - 2.0 * qixqkx) - gf6 * rxqkrx - gf7 * (rxqkirx - qkrxqirx);
              double ttm3y = bn2 * dixdky + gf3 * dkxry - gf4 * (dixqkry + dkxqiry + rxqkdiy - 2.0 * qixqky) - gf6 * rxqkry - gf7 * (rxqkiry - qkrxqiry);
              double ttm3z = bn2 * dixdkz + gf3 * dkxrz - gf4 * (dixqkrz + dkxqirz + rxqkdiz - 2.0 * qixqkz) - gf6 * rxqkrz - gf7 * (rxqkirz - qkrxqirz);
              if (scale1 != 0.0) {
                const double gfr1 = rr5 * gl0 + rr7 * (gl1 + gl6) + rr9 * (gl2 + gl7 + gl8) + rr11 * (gl3 + gl5) + rr13 * gl4;
                const double gfr2 = -ck * rr5 + sc4 * rr7 - sc6 * rr9;
                const double gfr3 = ci * rr5 + sc3 * rr7 + sc5 * rr9;
                const double gfr4 = 2.0 * rr7;
                const double gfr5 = 2.0 * (-ck * rr7 + sc4 * rr9 - sc6 * rr11);
                const double gfr6 = 2.0 * (-ci * rr7 - sc3 * rr9 - sc5 * rr11);
                const double gfr7 = 4.0 * rr9;
                ftm2x -= scale1 * (gfr1 * xr + gfr2 * dix + gfr3 * dkx + gfr4 * (qkdix - qidkx) + gfr5 * qirx + gfr6 * qkrx + gfr7 * (qiqkrx + qkqirx));
                ftm2y -= scale1 * (gfr1 * yr + gfr2 * diy + gfr3 * dky + gfr4 * (qkdiy - qidky) + gfr5 * qiry + gfr6 * qkry + gfr7 * (qiqkry + qkqiry));
                ftm2z -= scale1 * (gfr1 * zr + gfr2 * diz + gfr3 * dkz + gfr4 * (qkdiz - qidkz) + gfr5 * qirz + gfr6 * qkrz + gfr7 * (qiqkrz + qkqirz));
                ttm2x -= scale1 * (-rr5 * dixdkx + gfr2 * dixrx + gfr4 * (dixqkrx + dkxqirx + rxqidkx - 2.0 * qixqkx) - gfr5 * rxqirx - gfr7 * (rxqikrx + qkrxqirx));
                ttm2y -= scale1 * (-rr5 * dixdky + gfr2 * dixry + gfr4 * (dixqkry + dkxqiry + rxqidky - 2.0 * qixqky) - gfr5 * rxqiry - gfr7 * (rxqikry + qkrxqiry));
                ttm2z -= scale1 * (-rr5 * dixdkz + gfr2 * dixrz + gfr4 * (dixqkrz + dkxqirz + rxqidkz - 2.0 * qixqkz) - gfr5 * rxqirz - gfr7 * (rxqikrz + qkrxqirz));
                ttm3x -= scale1 * (rr5 * dixdkx + gfr3 * dkxrx - gfr4 * (dixqkrx + dkxqirx + rxqkdix - 2.0 * qixqkx) - gfr6 * rxqkrx - gfr7 * (rxqkirx - qkrxqirx));
                ttm3y -= scale1 * (rr5 * dixdky + gfr3 * dkxry - gfr4 * (dixqkry + dkxqiry + rxqkdiy - 2.0 * qixqky) - gfr6 * rxqkry - gfr7 * (rxqkiry - qkrxqiry));
                ttm3z -= scale1 * (rr5 * dixdkz + gfr3 * dkxrz - gfr4 * (dixqkrz + dkxqirz + rxqkdiz - 2.0 * qixqkz) - gfr6 * rxqkrz - gfr7 * (rxqkirz - qkrxqirz));
              }
              const double pf = electric * l2 * stepDlAlpha;
              std::vector<double> &lg = *lgp, &lt = *ltp;
              lg[3 * i] += pf * ftm2x; lg[3 * i + 1] += pf * ftm2y; lg[3 * i + 2] += pf * ftm2z;
              lt[3 * i] += pf * ttm2x; lt[3 * i + 1] += pf * ttm2y; lt[3 * i + 2] += pf * ttm2z;
              lg[3 * k] -= pf * ftm2x; lg[3 * k + 1] -= pf * ftm2y; lg[3 * k + 2] -= pf * ftm2z;
              lt[3 * k] += pf * ttm3x; lt[3 * k + 1] += pf * ttm3y; lt[3 * k + 2] += pf * ttm3z;
            }
          }
          if (!polOn) continue;
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
            const double epol = 0.5 * (ereal - efix);
            eI += polScale * epol;
            if (lam) {
              eDLt += dEdLSign * g_alch.dlPowPol * epol;
              eD2Lt += dEdLSign * g_alch.d2lPowPol * epol;
            }
            if (!gr) continue;
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
            if (p.polarization == FFXG_POLAR_DIRECT) {
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
            const double sc = electric * polScale;
            g[3 * i] += sc * ftm2ix; g[3 * i + 1] += sc * ftm2iy; g[3 * i + 2] += sc * ftm2iz;
            tq[3 * i] += sc * ttm2ix; tq[3 * i + 1] += sc * ttm2iy; tq[3 * i + 2] += sc * ttm2iz;
            g[3 * k] -= sc * ftm2ix; g[3 * k + 1] -= sc * ftm2iy; g[3 * k + 2] -= sc * ftm2iz;
            tq[3 * k] += sc * ttm3ix; tq[3 * k + 1] += sc * ttm3iy; tq[3 * k + 2] += sc * ttm3iz;
            if (lam) {   // RealSpaceEnergyRegion.java:2163-2174
              const double sl = electric * dEdLSign * g_alch.dlPowPol;
              std::vector<double> &lg = *lgp, &lt = *ltp;
              lg[3 * i] += sl * ftm2ix; lg[3 * i + 1] += sl * ftm2iy; lg[3 * i + 2] += sl * ftm2iz;
              lt[3 * i] += sl * ttm2ix; lt[3 * i + 1] += sl * ttm2iy; lt[3 * i + 2] += sl * ttm2iz;
              lg[3 * k] -= sl * ftm2ix; lg[3 * k + 1] -= sl * ftm2iy; lg[3 * k + 2] -= sl * ftm2iz;
              lt[3 * k] += sl * ttm3ix; lt[3 * k + 1] += sl * ttm3iy; lt[3 * k + 2] += sl * ttm3iz;
            }
          }
        }
        for (int k : m12[i]) { pmask[k] = 1.0; mmask[k] = 1.0; }
        for (int k : m13[i]) { pmask[k] = 1.0; mmask[k] = 1.0; }
        for (int k : m14[i]) { pmask[k] = 1.0; mmask[k] = 1.0; }
        for (int k : m15[i]) mmask[k] = 1.0;
        for (int gg : ip11[i]) dmask[gg] = 1.0;
      }
    }
    if (gr)
      for (int t = 0; t < nthreads; t++)
        for (size_t j = 0; j < 3 * (size_t)n; j++) { grad[j] += tg[t][j]; torque[j] += tt[t][j]; }
    if (lam) {
      for (int t = 0; t < nthreads; t++)
        for (size_t j = 0; j < 3 * (size_t)n; j++) { lgE[j] += tlg[t][j]; ltE[j] += tlt[t][j]; }
      eDL += eDLt * electric;
      eD2L += eD2Lt * electric;
    }
    ePerm = eP * electric;
    ePol = eI * electric;
    count = cnt;
  }

  // ---------------------------------------------------------------------------
  // Torque to Cartesian gradient, pme/Torque.java:111-316.
  static void cross(const double *a, const double *b, double *c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
  }
  static double len3(const double *v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

  void torque_one(int i, const double *trq, int idx[4], double g[4][3]) const {
    for (int a = 0; a < 4; a++) { idx[a] = -1; g[a][0] = g[a][1] = g[a][2] = 0.0; }
    const int fr = frame[i];
    if (fr == FFXG_FRAME_NONE) return;
    const int iz = axis[3 * i], ix = axis[3 * i + 1], iy = axis[3 * i + 2];
    idx[0] = iz; idx[1] = ix; idx[2] = iy; idx[3] = i;
    const double o[3] = {x[i], y[i], z[i]};
    double vZ[3] = {x[iz] - o[0], y[iz] - o[1], z[iz] - o[2]};
    const double rZ = len3(vZ);
    double vX[3], vY[3];
    if (fr != FFXG_FRAME_ZONLY) {
      vX[0] = x[ix] - o[0]; vX[1] = y[ix] - o[1]; vX[2] = z[ix] - o[2];
    } else {
      vX[0] = 1.0; vX[1] = 0.0; vX[2] = 0.0;
      const double dt = vZ[0] / rZ;
      if (std::fabs(dt) > 0.866) { vX[0] = 0.0; vX[1] = 1.0; }
    }
    const double rX = len3(vX);
    if (fr == FFXG_FRAME_ZTHENBISECTOR || fr == FFXG_FRAME_THREEFOLD) {
      vY[0] = x[iy] - o[0]; vY[1] = y[iy] - o[1]; vY[2] = z[iy] - o[2];
    } else {
      cross(vZ, vX, vY);
    }
    const double rY = len3(vY);
    for (int d = 0; d < 3; d++) { vZ[d] *= 1.0 / rZ; vX[d] *= 1.0 / rX; vY[d] *= 1.0 / rY; }
    double xXZ[3], xYZ[3], xYX[3];
    cross(vX, vZ, xXZ); cross(vY, vZ, xYZ); cross(vY, vX, xYX);
    norm3(xXZ); norm3(xYZ); norm3(xYX);
    const double cosZX = dot3(vZ, vX);
    const double sinZX = std::sqrt(1.0 - cosZX * cosZX);
    const double dPhidZ = -(trq[0] * vZ[0] + trq[1] * vZ[1] + trq[2] * vZ[2]);
    const double dPhidX = -(trq[0] * vX[0] + trq[1] * vX[1] + trq[2] * vX[2]);
    const double dPhidY = -(trq[0] * vY[0] + trq[1] * vY[1] + trq[2] * vY[2]);
    switch (fr) {
      case FFXG_FRAME_ZONLY:
        for (int j = 0; j < 3; j++) {
          const double dZ = xXZ[j] * dPhidX / (rZ * sinZX) + xYZ[j] * dPhidY / rZ;
          g[0][j] = dZ; g[3][j] = -dZ;
        }
        break;
      case FFXG_FRAME_ZTHENX:
        for (int j = 0; j < 3; j++) {
          const double dZ = xXZ[j] * dPhidX / (rZ * sinZX) + xYZ[j] * dPhidY / rZ;
          const double dX = -xXZ[j] * dPhidZ / (rX * sinZX);
          g[0][j] = dZ; g[1][j] = dX; g[3][j] = -(dZ + dX);
        }
        break;
      case FFXG_FRAME_BISECTOR:
        for (int j = 0; j < 3; j++) {
          const double dZ = xXZ[j] * dPhidX / (rZ * sinZX) + 0.5 * xYZ[j] * dPhidY / rZ;
          const double dX = -xXZ[j] * dPhidZ / (rX * sinZX) + 0.5 * xYX[j] * dPhidY / rX;
          g[0][j] = dZ; g[1][j] = dX; g[3][j] = -(dZ + dX);
        }
        break;
      case FFXG_FRAME_ZTHENBISECTOR: {
        double sumXY[3] = {vX[0] + vY[0], vX[1] + vY[1], vX[2] + vY[2]};
        double xZXY[3], xXYZ[3], xxZXYZ[3], xxZXYX[3], xxZXYY[3], t1[3], t2[3];
        cross(vZ, sumXY, xZXY);
        norm3(sumXY); norm3(xZXY);
        cross(sumXY, vZ, xXYZ);
        cross(xZXY, vZ, xxZXYZ);
        cross(xZXY, vX, xxZXYX);
        cross(xZXY, vY, xxZXYY);
        norm3(xXYZ); norm3(xxZXYZ); norm3(xxZXYX); norm3(xxZXYY);
        const double cosZXY = dot3(vZ, sumXY), sinZXY = std::sqrt(1.0 - cosZXY * cosZXY);
        const double cosXZXY = dot3(vX, xZXY), sinXZXY = std::sqrt(1.0 - cosXZXY * cosXZXY);
        const double cosYZXY = dot3(vY, xZXY), sinYZXY = std::sqrt(1.0 - cosYZXY * cosYZXY);
        for (int d = 0; d < 3; d++) { t1[d] = vX[d] + xZXY[d] * -cosXZXY; t2[d] = vY[d] + xZXY[d] * -cosYZXY; }
        norm3(t1); norm3(t2);
        const double ut1cos = dot3(vZ, t1), ut1sin = std::sqrt(1.0 - ut1cos * ut1cos);
        const double ut2cos = dot3(vZ, t2), ut2sin = std::sqrt(1.0 - ut2cos * ut2cos);
        const double dPhidR = -(trq[0] * sumXY[0] + trq[1] * sumXY[1] + trq[2] * sumXY[2]);
        const double dPhidZXY = -(trq[0] * xZXY[0] + trq[1] * xZXY[1] + trq[2] * xZXY[2]);
        for (int j = 0; j < 3; j++) {
          const double dZ = xXYZ[j] * dPhidR / (rZ * sinZXY) + xxZXYZ[j] * dPhidZXY / rZ;
          const double dX = (sinXZXY * xZXY[j] - cosXZXY * t1[j]) * dPhidZ / (rX * (ut1sin + ut2sin));
          const double dY = (sinYZXY * xZXY[j] - cosYZXY * t2[j]) * dPhidZ / (rY * (ut1sin + ut2sin));
          g[0][j] = dZ; g[1][j] = dX; g[2][j] = dY; g[3][j] = -(dZ + dX + dY);
        }
        break;
      }
      case FFXG_FRAME_THREEFOLD: {
        double sumZXY[3] = {vZ[0] + vX[0], vZ[1] + vX[1], vZ[2] + vX[2]};
        for (int d = 0; d < 3; d++) sumZXY[d] = vY[d] + sumZXY[d];
        const double rZXY = len3(sumZXY);
        for (int d = 0; d < 3; d++) sumZXY[d] *= 1.0 / rZXY;
        const double cosYSum = dot3(vY, sumZXY), cosZSum = dot3(vZ, sumZXY), cosXSum = dot3(vX, sumZXY);
        double rr[3], del[3], eps[3];
        for (int d = 0; d < 3; d++) rr[d] = vX[d] + vY[d];
        norm3(rr);
        double cosR = dot3(rr, vZ), sinR = std::sqrt(1.0 - cosR * cosR);
        double dPhidR = -trq[0] * rr[0] - trq[1] * rr[1] - trq[2] * rr[2];
        cross(rr, vZ, del); norm3(del);
        double dPhidDel = -trq[0] * del[0] - trq[1] * del[1] - trq[2] * del[2];
        cross(del, vZ, eps);
        for (int j = 0; j < 3; j++) {
          const double dZ = del[j] * dPhidR / (rZ * sinR) + eps[j] * dPhidDel * cosZSum / (rZ * rZXY);
          g[0][j] = dZ; g[3][j] = -dZ;
        }
        for (int d = 0; d < 3; d++) rr[d] = vZ[d] + vY[d];
        norm3(rr);
        cosR = dot3(rr, vX); sinR = std::sqrt(1.0 - cosR * cosR);
        dPhidR = -trq[0] * rr[0] - trq[1] * rr[1] - trq[2] * rr[2];
        cross(rr, vX, del); norm3(del);
        dPhidDel = -trq[0] * del[0] - trq[1] * del[1] - trq[2] * del[2];
        cross(del, vX, eps);
        for (int j = 0; j < 3; j++) {
          const double dX = del[j] * dPhidR / (rX * sinR) + eps[j] * dPhidDel * cosXSum / (rX * rZXY);
          g[1][j] = dX; g[3][j] -= dX;
        }
        for (int d = 0; d < 3; d++) rr[d] = vZ[d] + vX[d];
        norm3(rr);
        cosR = dot3(rr, vY); sinR = std::sqrt(1.0 - cosR * cosR);
        dPhidR = -trq[0] * rr[0] - trq[1] * rr[1] - trq[2] * rr[2];
        cross(rr, vY, del); norm3(del);
        dPhidDel = -trq[0] * del[0] - trq[1] * del[1] - trq[2] * del[2];
        cross(del, vY, eps);
        for (int j = 0; j < 3; j++) {
          const double dY = del[j] * dPhidR / (rY * sinR) + eps[j] * dPhidDel * cosYSum / (rY * rZXY);
          g[2][j] = dY; g[3][j] -= dY;
        }
        break;
      }
      default: break;
    }
  }

  void torque_to_gradient() { torque_to_gradient(torque, grad); }

  void torque_to_gradient(const std::vector<double> &tq, std::vector<double> &gr) {
    for (int i = 0; i < n; i++) {
      int idx[4];
      double g[4][3];
      torque_one(i, &tq[3 * (size_t)i], idx, g);
      for (int a = 0; a < 4; a++)
        if (idx[a] >= 0)
          for (int d = 0; d < 3; d++) gr[3 * (size_t)idx[a] + d] += g[a][d];
    }
  }

  // ---------------------------------------------------------------------------
  // Parameter gradients (after energy()): dE/dM for each atom's local-frame multipole
  // (stored components q, d, Q as in lmp) and dE/dalpha for its polarizability (with the
  // Thole damping held fixed).  The permanent energy is bilinear in the multipoles, so
  // dE_perm/dM_i is the potential of all other multipoles at i (real space with its
  // masks, reciprocal, self, charge correction).  The polarization energy is
  // E_pol = -1/2 electric E_d^T A^-1 E_p with A = alpha^-1 - T symmetric, u_D = A^-1 E_d and
  // u_P = A^-1 E_p, so dE_pol/dM = -1/2 electric (F_d^T u_P + F_p^T u_D): the CR dipoles
  // are the adjoint solution and no further solve is needed; and
  // dE_pol/dalpha_i = -1/2 electric alpha_i^-2 u_D,i . u_P,i.

  // d e_pair / d M_t (stored components) of the permanent pair energy for the target
  // multipole t and source Ms at r = x_s - x_t with radial coefficients b[0..4]
  // (the derivative of RealSpaceEnergyRegion.permanentPair's gl sums, :1190-1290).
  static void pair_pot(const double *Ms, const double r[3], const double b[5], double out[10]) {
    const double ck = Ms[t000], dk[3] = {Ms[t100], Ms[t010], Ms[t001]};
    double qk[3][3];
    qk[0][0] = Ms[t200] / 3.0; qk[1][1] = Ms[t020] / 3.0; qk[2][2] = Ms[t002] / 3.0;
    qk[0][1] = qk[1][0] = Ms[t110] / 3.0; qk[0][2] = qk[2][0] = Ms[t101] / 3.0; qk[1][2] = qk[2][1] = Ms[t011] / 3.0;
    double qkr[3];
    for (int a = 0; a < 3; a++) qkr[a] = qk[a][0] * r[0] + qk[a][1] * r[1] + qk[a][2] * r[2];
    const double sc4 = dk[0] * r[0] + dk[1] * r[1] + dk[2] * r[2];
    const double sc6 = qkr[0] * r[0] + qkr[1] * r[1] + qkr[2] * r[2];
    out[t000] = ck * b[0] - sc4 * b[1] + sc6 * b[2];
    const double cd = ck * b[1] - sc4 * b[2] + sc6 * b[3];
    for (int a = 0; a < 3; a++) out[1 + a] = cd * r[a] + b[1] * dk[a] - 2.0 * b[2] * qkr[a];
    double G[3][3];
    for (int a = 0; a < 3; a++)
      for (int c = 0; c < 3; c++)
        G[a][c] = (ck * r[a] * r[c] + 2.0 * dk[a] * r[c] + 2.0 * qk[a][c]) * b[2] +
                  (-sc4 * r[a] * r[c] - 4.0 * qkr[a] * r[c]) * b[3] + sc6 * r[a] * r[c] * b[4];
    quad_out(G, out);
  }

  // d (u . E(M_t))/d M_t for a dipole u at r = x_u - x_t from the target multipole, with the
  // radial coefficients b1..b3 of the field (PermanentFieldRegion.java:703-760: Ewald bn
  // less the masked, Thole-damped corrections).
  static void dip_pot(const double u[3], const double r[3], double b1, double b2, double b3, double out[10]) {
    const double ur = u[0] * r[0] + u[1] * r[1] + u[2] * r[2];
    out[t000] = ur * b1;
    for (int a = 0; a < 3; a++) out[1 + a] = ur * b2 * r[a] - b1 * u[a];
    double G[3][3];
    for (int a = 0; a < 3; a++)
      for (int c = 0; c < 3; c++) G[a][c] = ur * b3 * r[a] * r[c] - 2.0 * b2 * u[a] * r[c];
    quad_out(G, out);
  }

  // Derivatives w.r.t. q_ab = Q_ab / 3 (full matrix G) as derivatives w.r.t. the stored
  // quadrupole components (diagonal once, each off-diagonal pair once).
  static void quad_out(const double G[3][3], double *out) {
    out[t200] = G[0][0] / 3.0; out[t020] = G[1][1] / 3.0; out[t002] = G[2][2] / 3.0;
    out[t110] = (G[0][1] + G[1][0]) / 3.0;
    out[t101] = (G[0][2] + G[2][0]) / 3.0;
    out[t011] = (G[1][2] + G[2][1]) / 3.0;
  }

  void param_gradients(std::vector<double> &dM, std::vector<double> &dA) {
    const double electric = p.electric;
    std::vector<double> phi(10 * (size_t)n, 0.0);   // dE/dM, global frame
    const bool pol = p.polarization != FFXG_POLAR_NONE;
    // Real space, over the Ewald lists (each pair once, both sides).
    for (int i = 0; i < n; i++) {
      std::vector<double> mm(n, 1.0), dd(n, 1.0), pp(n, 1.0);
      for (int k : m12[i]) { mm[k] = p.m12; pp[k] = p.p12; }
      for (int k : m13[i]) { mm[k] = p.m13; pp[k] = p.p13; }
      for (int k : m14[i]) {
        mm[k] = p.m14; pp[k] = p.p14;
        for (int g : ip11[i]) if (g == k) { pp[k] = p.intra14 * p.p14; break; }
      }
      for (int k : m15[i]) mm[k] = p.m15;
      for (int g : ip11[i]) dd[g] = p.d11;
      for (size_t e = 0; e < ewald[i].size(); e++) {
        const int k = ewald[i][e];
        double xr = x[k] - x[i], yr = y[k] - y[i], zr = z[k] - z[i];
        const double r2 = disp(xr, yr, zr, esh, i, e);
        const bool prim = primary(esh, i, e);
        const double r = std::sqrt(r2);
        const double ralpha = aewald * r, exp2a = std::exp(-ralpha * ralpha);
        const double rr1 = 1.0 / r, rr2 = rr1 * rr1;
        const double bn0 = std::erfc(ralpha) * rr1;
        const double bn1 = (bn0 + an0 * exp2a) * rr2, bn2 = (3.0 * bn1 + an1 * exp2a) * rr2;
        const double bn3 = (5.0 * bn2 + an2 * exp2a) * rr2, bn4 = (7.0 * bn3 + an3 * exp2a) * rr2;
        const double rr3 = rr1 * rr2, rr5 = 3.0 * rr3 * rr2, rr7 = 5.0 * rr5 * rr2, rr9 = 7.0 * rr7 * rr2;
        const double rik[3] = {xr, yr, zr}, rki[3] = {-xr, -yr, -zr};
        const double scale1 = 1.0 - (prim ? mm[k] : 1.0);
        const double bE[5] = {bn0, bn1, bn2, bn3, bn4}, bR[5] = {rr1, rr3, rr5, rr7, rr9};
        double a[10], c[10];
        // permanent: target i (source k at r_ik), target k (source i at r_ki)
        pair_pot(&gm[10 * (size_t)k], rik, bE, a);
        pair_pot(&gm[10 * (size_t)k], rik, bR, c);
        for (int t = 0; t < 10; t++) phi[10 * (size_t)i + t] += electric * (a[t] - scale1 * c[t]);
        pair_pot(&gm[10 * (size_t)i], rki, bE, a);
        pair_pot(&gm[10 * (size_t)i], rki, bR, c);
        for (int t = 0; t < 10; t++) phi[10 * (size_t)k + t] += electric * (a[t] - scale1 * c[t]);
        if (!pol) continue;
        double scale3 = 1.0, scale5 = 1.0, scale7 = 1.0;
        double damp = ipdamp[i] * ipdamp[k];
        const double tho = std::min(thole[i], thole[k]);
        const double rdamp = r * damp;
        damp = -tho * rdamp * rdamp * rdamp;
        if (damp > -50.0) {
          const double expdamp = std::exp(damp);
          scale3 = 1.0 - expdamp;
          scale5 = 1.0 - expdamp * (1.0 - damp);
          scale7 = 1.0 - expdamp * (1.0 - damp + 0.6 * damp * damp);
        }
        const double sd = prim ? dd[k] : 1.0, sp = prim ? pp[k] : 1.0;
        const double db1 = bn1 - (1.0 - scale3 * sd) * rr3, db2 = bn2 - (1.0 - scale5 * sd) * rr5,
                     db3 = bn3 - (1.0 - scale7 * sd) * rr7;
        const double pb1 = bn1 - (1.0 - scale3 * sp) * rr3, pb2 = bn2 - (1.0 - scale5 * sp) * rr5,
                     pb3 = bn3 - (1.0 - scale7 * sp) * rr7;
        const double h = -0.5 * electric;
        // target i: dipoles at k; target k: dipoles at i.
        dip_pot(&uP[3 * (size_t)k], rik, db1, db2, db3, a);
        dip_pot(&uD[3 * (size_t)k], rik, pb1, pb2, pb3, c);
        for (int t = 0; t < 10; t++) phi[10 * (size_t)i + t] += h * (a[t] + c[t]);
        dip_pot(&uP[3 * (size_t)i], rki, db1, db2, db3, a);
        dip_pot(&uD[3 * (size_t)i], rki, pb1, pb2, pb3, c);
        for (int t = 0; t < 10; t++) phi[10 * (size_t)k + t] += h * (a[t] + c[t]);
      }
    }
    // Reciprocal space, self terms, charge correction.
    const double w[10] = {1.0, 1.0, 1.0, 1.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0};
    const double aewald1 = -electric * aewald / kSqrtPi, aewald2 = 2.0 * aewald * aewald;
    double qtot = 0.0;
    for (int i = 0; i < n; i++) qtot += gm[10 * (size_t)i];
    const double dcorr = (qtot != 0.0) ? -electric * kPi * qtot / (cell.volume * aewald * aewald) : 0.0;
    for (int i = 0; i < n; i++) {
      double *f = &phi[10 * (size_t)i];
      const double *m = &gm[10 * (size_t)i];
      for (int t = 0; t < 10; t++) f[t] += electric * w[t] * cphi[20 * (size_t)i + t];
      f[t000] += 2.0 * aewald1 * m[t000] + dcorr;
      for (int a = 1; a < 4; a++) f[a] += aewald1 * aewald2 * 2.0 * m[a] / 3.0;
      for (int a = 4; a < 7; a++) f[a] += aewald1 * aewald2 * 2.0 * aewald2 * 2.0 * m[a] / 45.0;
      for (int a = 7; a < 10; a++) f[a] += aewald1 * aewald2 * 2.0 * aewald2 * 4.0 * m[a] / 45.0;
      if (pol) {
        const double h = -0.5 * electric;
        for (int t = 0; t < 10; t++)
          f[t] += h * -w[t] * (cphiP[20 * (size_t)i + t] + cphiI[20 * (size_t)i + t]);
        for (int a = 0; a < 3; a++) f[1 + a] += h * aewald3 * (uP[3 * (size_t)i + a] + uD[3 * (size_t)i + a]);
      }
    }
    // Global -> local frame: d = R d_l, Q = R Q_l R^T (rotate_multipoles).
    dM.assign(10 * (size_t)n, 0.0);
    dA.assign(n, 0.0);
    for (int i = 0; i < n; i++) {
      double R[3][3];
      rotation_matrix(i, R);
      const double *f = &phi[10 * (size_t)i];
      double *o = &dM[10 * (size_t)i];
      o[t000] = f[t000];
      for (int b = 0; b < 3; b++) o[1 + b] = R[0][b] * f[1] + R[1][b] * f[2] + R[2][b] * f[3];
      double G[3][3];
      G[0][0] = f[t200]; G[1][1] = f[t020]; G[2][2] = f[t002];
      G[0][1] = G[1][0] = 0.5 * f[t110]; G[0][2] = G[2][0] = 0.5 * f[t101]; G[1][2] = G[2][1] = 0.5 * f[t011];
      double L[3][3];
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
          double v = 0.0;
          for (int c = 0; c < 3; c++)
            for (int d = 0; d < 3; d++) v += R[c][a] * G[c][d] * R[d][b];
          L[a][b] = v;
        }
      o[t200] = L[0][0]; o[t020] = L[1][1]; o[t002] = L[2][2];
      o[t110] = 2.0 * L[0][1]; o[t101] = 2.0 * L[0][2]; o[t011] = 2.0 * L[1][2];
      if (pol && polar[i] > 0.0) {
        const double ud = uD[3 * (size_t)i] * uP[3 * (size_t)i] + uD[3 * (size_t)i + 1] * uP[3 * (size_t)i + 1] +
                          uD[3 * (size_t)i + 2] * uP[3 * (size_t)i + 2];
        dA[i] = -0.5 * electric * ud / (polar[i] * polar[i]);
      }
    }
  }

  // Per-term electrostatic energies of one evaluation.
  struct ElecTerms {
    double eSelf = 0, eRecip = 0, eCorr = 0, eSelfI = 0, eRecipI = 0, eReal = 0, eRealI = 0;
    int64_t nreal = 0;
    void add(const ElecTerms &o) {
      eSelf += o.eSelf; eRecip += o.eRecip; eCorr += o.eCorr; eSelfI += o.eSelfI; eRecipI += o.eRecipI;
      eReal += o.eReal; eRealI += o.eRealI;
    }
  };

  // ParticleMeshEwald.computeEnergy (ParticleMeshEwald.java:1871-2183) for the current
  // step state: permanent field, SCF, reciprocal and real-space energy and gradient.
  int electrostatics_step(bool gradient, ElecTerms &t) {
    if (recip_on) {
      std::vector<std::complex<double>> grid;
      spread_permanent(grid);
      convolve(grid);
      interpolate(grid, 0, fphi, cphi);
    } else {
      cphi.assign(20 * (size_t)n, 0.0);
      fphi.assign(20 * (size_t)n, 0.0);
    }
    permanent_field();
    uD.assign(3 * (size_t)n, 0.0); uP.assign(3 * (size_t)n, 0.0);
    udir.assign(3 * (size_t)n, 0.0); udirP.assign(3 * (size_t)n, 0.0);
    int st = FFXG_OK;
    if (p.polarization != FFXG_POLAR_NONE && doPol) {
      // DirectRegion (pme/DirectRegion.java:170-243).
      for (int i = 0; i < n; i++)
        for (int a = 0; a < 3; a++) {
          const size_t j = 3 * (size_t)i + a;
          const double f = aewald3 * gm[10 * (size_t)i + 1 + a] - cphi[20 * (size_t)i + 1 + a];
          fieldD[j] += f; fieldP[j] += f;
          uD[j] = polar[i] * fieldD[j]; udir[j] = uD[j];
          uP[j] = polar[i] * fieldP[j]; udirP[j] = uP[j];
        }
      int it = 0;
      if (p.polarization == FFXG_POLAR_MUTUAL) {
        st = pcg();
        it = scf_iter;
      }
      scf_total += it;
      if (st != FFXG_OK) return st;
      std::vector<double> fD, fP;
      induced_field(uD, uP, fD, fP);  // final field (PCGSolver.java:601)
    }
    if (recip_on) recip_energy(gradient, t.eSelf, t.eRecip, t.eCorr, t.eSelfI, t.eRecipI);
    real_energy(gradient, t.eReal, t.eRealI, t.nreal);
    return st;
  }

  // The three evaluations of elec-lambdaterm in OST mode (ParticleMeshEwald.energy,
  // PME:897-935): condensedEnergy (:1609-1640), condensedNoLigandSCF (:1650-1700) and
  // ligandElec (:1704-1796).  The vacuum step solves by PCG (the reference: SOR).
  int lambda_electrostatics(bool gradient, ElecTerms &sum, int64_t &nreal) {
    const Alchemy &al = g_alch;
    const double l = al.lambda;
    lgE.assign(3 * (size_t)n, 0.0);
    ltE.assign(3 * (size_t)n, 0.0);
    eDL = eD2L = 0.0;
    lam = true;
    // 1. Everything, softcore permanent real space, scaled reciprocal and polarization.
    use.clear();
    pol_eff = polar;
    vapor = false; recip_on = true; doPermReal = true;
    permScale = al.lPowPerm; dEdLSign = 1.0;
    stepAlpha = al.lAlpha; stepDlAlpha = al.dlAlpha; stepD2lAlpha = al.d2lAlpha;
    if (l < al.polStart) { doPol = false; polScale = 0.0; }
    else if (l <= al.polEnd) { doPol = true; polScale = al.lPowPol; }
    else { doPol = true; polScale = 1.0; }
    ElecTerms t1;
    int st = electrostatics_step(gradient, t1);
    if (st != FFXG_OK) return st;
    sum.add(t1);
    nreal = t1.nreal;
    // 2. Without the soft atoms: reciprocal permanent and polarization, complements.
    use.assign(n, 1);
    bool any = false;
    for (int i = 0; i < n; i++) { use[i] = !al.soft[i]; any = any || use[i]; }
    for (int i = 0; i < n; i++) pol_eff[i] = use[i] ? polar[i] : 0.0;
    doPermReal = false;
    permScale = 1.0 - al.lPowPerm; dEdLSign = -1.0;
    if (l <= al.polEnd && al.noLigandSCF) { doPol = true; polScale = 1.0 - al.lPowPol; }
    else { doPol = false; polScale = 0.0; }
    if (any) {
      ElecTerms t2;
      st = electrostatics_step(gradient, t2);
      if (st != FFXG_OK) return st;
      sum.add(t2);
    }
    // 3. The soft atoms alone in vacuum: no Ewald screening, no cutoff, no images.
    if (al.vaporElec) {
      for (int i = 0; i < n; i++) { use[i] = al.soft[i] != 0; pol_eff[i] = use[i] ? polar[i] : 0.0; }
      vapor = true; doPermReal = true;
      permScale = 1.0 - al.lPowPerm; dEdLSign = -1.0;
      stepAlpha = stepDlAlpha = stepD2lAlpha = 0.0;
      if (l <= al.polEnd) { doPol = true; polScale = 1.0 - al.lPowPol; }
      else { doPol = false; polScale = 0.0; }
      const double sv[9] = {aewald, an0, an1, an2, an3, an4, an5, aewald3, off2};
      const bool mi = multi_image;
      std::vector<std::vector<int>> nl = nlist, ns = nsh;
      aewald = an0 = an1 = an2 = an3 = an4 = an5 = aewald3 = 0.0;
      off2 = INFINITY;
      recip_on = false;
      multi_image = true;
      nlist.assign(n, {});
      nsh.assign(n, {});
      for (int i = 0; i < n; i++)
        if (use[i])
          for (int k = i + 1; k < n; k++)
            if (use[k]) { nlist[i].push_back(k); nsh[i].push_back(pack_shift(0, 0, 0, true)); }
      ElecTerms t3;
      st = electrostatics_step(gradient, t3);
      aewald = sv[0]; an0 = sv[1]; an1 = sv[2]; an2 = sv[3]; an3 = sv[4]; an4 = sv[5]; an5 = sv[6];
      aewald3 = sv[7]; off2 = sv[8];
      multi_image = mi;
      nlist.swap(nl);
      nsh.swap(ns);
      recip_on = true;
      if (st != FFXG_OK) return st;
      sum.add(t3);
    }
    lam = false; vapor = false; use.clear(); pol_eff = polar;
    doPermReal = true; doPol = true; permScale = polScale = dEdLSign = 1.0;
    stepAlpha = stepDlAlpha = stepD2lAlpha = 0.0;
    return FFXG_OK;
  }

  // ---------------------------------------------------------------------------
  // ForceFieldEnergy.energy (ForceFieldEnergy.java:1638-1800) restricted to vdW + PME,
  // with ParticleMeshEwald.energy / computeEnergy (ParticleMeshEwald.java:837-954, 1871-2183).
  int energy(bool gradient, double *terms, double *g_out, int64_t *counts) {
    grad.assign(3 * (size_t)n, 0.0);
    torque.assign(3 * (size_t)n, 0.0);
    build_list();
    int64_t nv = 0;
    const double evdw = vdw(gradient, nv);
    rotate_multipoles();
    compute_bsplines();
    scf_iter = 0;
    scf_total = 0;
    int st = FFXG_OK;
    ElecTerms et;
    int64_t nreal = 0;
    if (g_alch.on && g_alch.elec) {
      st = lambda_electrostatics(gradient, et, nreal);
      if (st != FFXG_OK) return st;
      torque_to_gradient(ltE, lgE);
      g_alch.dEdL += eDL;
      g_alch.d2EdL2 += eD2L;
      if (g_alch.lgrad.size() == lgE.size())
        for (size_t j = 0; j < lgE.size(); j++) g_alch.lgrad[j] += lgE[j];
    } else {
      use.clear();
      pol_eff = polar;
      st = electrostatics_step(gradient, et);
      if (st != FFXG_OK) return st;
      nreal = et.nreal;
    }
    scf_iter = scf_total;
    const double eSelf = et.eSelf, eRecip = et.eRecip, eCorr = et.eCorr, eSelfI = et.eSelfI,
                 eRecipI = et.eRecipI, eReal = et.eReal, eRealI = et.eRealI;
    if (gradient) torque_to_gradient();
    if (terms) {
      terms[FFXG_TERM_VDW] = evdw;
      terms[FFXG_TERM_PERM_REAL] = eReal;
      terms[FFXG_TERM_PERM_SELF] = eSelf;
      terms[FFXG_TERM_PERM_RECIP] = eRecip + eCorr;
      terms[FFXG_TERM_POL_REAL] = eRealI;
      terms[FFXG_TERM_POL_SELF] = eSelfI;
      terms[FFXG_TERM_POL_RECIP] = eRecipI;
      terms[FFXG_TERM_PERMANENT] = eSelf + eRecip + eReal + eCorr;
      terms[FFXG_TERM_POLARIZATION] = eSelfI + eRecipI + eRealI;
      terms[FFXG_TERM_TOTAL] = evdw + terms[FFXG_TERM_PERMANENT] + terms[FFXG_TERM_POLARIZATION];
    }
    if (counts) {
      int64_t np = 0;
      for (int i = 0; i < n; i++) np += (int64_t)nlist[i].size();
      counts[FFXG_COUNT_VDW] = nv;
      counts[FFXG_COUNT_PERMANENT] = nreal + n;
      counts[FFXG_COUNT_SCF_ITER] = scf_iter;
      counts[FFXG_COUNT_LIST_BUILDS] = 1;
      counts[FFXG_COUNT_LIST_PAIRS] = np;
    }
    if (gradient && g_out) std::memcpy(g_out, grad.data(), 3 * (size_t)n * sizeof(double));
    return st;
  }
};

}  // namespace

extern "C" {

// Energy / gradient of the system at xyz; optional outputs may be NULL.
int oracle_energy(const ffxg_system *sys, const ffxg_params *prm, const double *xyz, int want_grad,
                  int nthreads, double *terms, double *grad, int64_t *counts, double *induced,
                  double *induced_cr, double *global_mpole) {
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  omp_set_num_threads(nthreads);
#else
  nthreads = 1;
#endif
  Oracle o;
  o.nthreads = nthreads;
  o.setup(sys, prm, xyz ? xyz : sys->xyz);
  const int st = o.energy(want_grad != 0, terms, grad, counts);
  if (induced && !o.uD.empty()) std::memcpy(induced, o.uD.data(), 3 * (size_t)o.n * sizeof(double));
  if (induced_cr && !o.uP.empty()) std::memcpy(induced_cr, o.uP.data(), 3 * (size_t)o.n * sizeof(double));
  if (global_mpole && !o.gm.empty()) std::memcpy(global_mpole, o.gm.data(), 10 * (size_t)o.n * sizeof(double));
  return st;
}

// Unordered pairs (i < k) of the buffered neighbour list; pairs may be NULL to count.
int64_t oracle_neighbor_pairs(const ffxg_system *sys, const ffxg_params *prm, const double *xyz,
                              int32_t *pairs) {
  Oracle o;
  o.nthreads = 1;
#ifdef _OPENMP
  o.nthreads = omp_get_max_threads();
#endif
  o.setup(sys, prm, xyz ? xyz : sys->xyz);
  o.build_list();
  int64_t c = 0;
  for (int i = 0; i < o.n; i++)
    for (int k : o.nlist[i]) {
      if (pairs) { pairs[2 * c] = i; pairs[2 * c + 1] = k; }
      c++;
    }
  return c;
}

// Image pairs of the buffered list, one line per pair image: (i, k, nx, ny, nz) with the
// lattice shift n of x_k + n L - x_i (minimum image: n from Crystal.image's rounding),
// i < k, or i == k with n > 0.  out may be NULL to count.
int64_t oracle_neighbor_images(const ffxg_system *sys, const ffxg_params *prm, const double *xyz,
                               int32_t *out) {
  Oracle o;
  o.nthreads = 1;
#ifdef _OPENMP
  o.nthreads = omp_get_max_threads();
#endif
  o.setup(sys, prm, xyz ? xyz : sys->xyz);
  o.build_list();
  int64_t c = 0;
  for (int i = 0; i < o.n; i++)
    for (size_t e = 0; e < o.nlist[i].size(); e++) {
      if (out) {
        const int k = o.nlist[i][e];
        int nx = 0, ny = 0, nz = 0;
        if (o.multi_image) {
          const int code = o.nsh[i][e];
          nx = (code & 1023) - 512; ny = ((code >> 10) & 1023) - 512; nz = ((code >> 20) & 1023) - 512;
        }
        int32_t *q = out + 5 * c;
        q[0] = i; q[1] = k; q[2] = nx; q[3] = ny; q[4] = nz;
      }
      c++;
    }
  return c;
}

// Energy, then the parameter gradients: dEdM[n][10] w.r.t. each atom's local multipole
// (stored components) and dEdA[n] w.r.t. its polarizability (Thole damping fixed).
int oracle_param_grad(const ffxg_system *sys, const ffxg_params *prm, const double *xyz, double *dEdM,
                      double *dEdA) {
  Oracle o;
  o.nthreads = 1;
#ifdef _OPENMP
  o.nthreads = omp_get_max_threads();
#endif
  o.setup(sys, prm, xyz ? xyz : sys->xyz);
  const int st = o.energy(false, nullptr, nullptr, nullptr);
  if (st != FFXG_OK) return st;
  std::vector<double> dM, dA;
  o.param_gradients(dM, dA);
  std::memcpy(dEdM, dM.data(), dM.size() * sizeof(double));
  std::memcpy(dEdA, dA.data(), dA.size() * sizeof(double));
  return FFXG_OK;
}

// Force (1) or release (0) multi-image lists for boxes where the minimum image suffices.
void oracle_set_images(int force_all) { g_force_images = force_all; }

// Soft atoms and softcore keys for the next oracle_energy calls (NULL clears), at lambda.
void oracle_set_alchemy(const ffxg_alchemy *a, int n, double lambda) {
  g_alch = Alchemy();
  if (!a) return;
  g_alch.on = true;
  g_alch.soft.assign(a->soft, a->soft + n);
  g_alch.mol.resize(n);
  for (int i = 0; i < n; i++) g_alch.mol[i] = a->molecule ? a->molecule[i] : i;
  g_alch.inter = a->intermolecular_softcore != 0;
  g_alch.intra = a->intramolecular_softcore != 0;
  // VanDerWaals.setLambda (VanDerWaals.java:599-628).
  double l = lambda;
  if (l > a->vdw_lambda_end) l = 1.0; else l = l / a->vdw_lambda_end;
  const double al = a->vdw_lambda_alpha, ex = a->vdw_lambda_exponent;
  g_alch.sc1 = al * (1.0 - l) * (1.0 - l);
  g_alch.dsc1dL = -2.0 * al * (1.0 - l);
  g_alch.d2sc1dL2 = 2.0 * al;
  g_alch.sc2 = std::pow(l, ex);
  g_alch.dsc2dL = ex * std::pow(l, ex - 1.0);
  g_alch.d2sc2dL2 = (ex >= 2.0) ? ex * (ex - 1.0) * std::pow(l, ex - 2.0) : 0.0;
  g_alch.elec = a->elec != 0;
  if (g_alch.elec) {
    g_alch.permAlpha = a->permanent_lambda_alpha;
    g_alch.permExp = a->permanent_lambda_exponent;
    g_alch.permStart = a->permanent_lambda_start;
    g_alch.permEnd = a->permanent_lambda_end;
    g_alch.polStart = a->polarization_lambda_start;
    g_alch.polEnd = a->polarization_lambda_end;
    g_alch.polExp = a->polarization_lambda_exponent;
    g_alch.vaporElec = a->ligand_vapor_elec != 0;
    g_alch.noLigandSCF = a->no_ligand_condensed_scf != 0;
    g_alch.update_elec(lambda);
  }
}

// dU/dL, d2U/dL2 and dU/dX dL [n][3] of the last oracle_energy call.
void oracle_get_dEdL(double *dEdL, double *d2EdL2, double *dEdXdL) {
  if (dEdL) *dEdL = g_alch.dEdL;
  if (d2EdL2) *d2EdL2 = g_alch.d2EdL2;
  if (dEdXdL && !g_alch.lgrad.empty()) std::memcpy(dEdXdL, g_alch.lgrad.data(), g_alch.lgrad.size() * sizeof(double));
}

// Known-answer hooks for the numerics unit tests.
double oracle_erfc(double x) { return std::erfc(x); }

void oracle_bspline(double x, int order, double *out /* [order][4] */) { bspline_derivs(x, order, out); }

// In-place 3D complex transform of data[(k*ny + j)*nx + i] (interleaved re, im).
void oracle_fft3d(double *data, int nx, int ny, int nz, int sign) {
  std::vector<std::complex<double>> g((size_t)nx * ny * nz);
  for (size_t i = 0; i < g.size(); i++) g[i] = std::complex<double>(data[2 * i], data[2 * i + 1]);
  fft3d(g, nx, ny, nz, sign);
  for (size_t i = 0; i < g.size(); i++) { data[2 * i] = g[i].real(); data[2 * i + 1] = g[i].imag(); }
}

}  // extern "C"
