// ffx_internal.cuh -- shared definitions of the B200 AMOEBA energy/gradient library.
//
// Data layout in HBM (all per-atom arrays are structure-of-arrays, index = atom):
//   x,y,z            coordinates (double)
//   rx,ry,rz         hydrogen-reduced vdW coordinates (double)
//   gm[10][n]        global-frame multipoles
//   fm[10][n]        fractional multipoles (PME)
//   uD,uP[3][n]      induced dipoles (direct-field / chain-rule systems)
//   nbr[n][cap]      buffered Verlet list (both directions), nbr_cnt[n]
//   ewl[n][capE]     real-space (Ewald) list, ewl_cnt[n]
//   prl[n][capP]     preconditioner list, prl_cnt[n]
//   grid[nz][ny][nx] interleaved complex PME mesh (double2)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/ffxcuda.h"
#include "launch.cuh"

namespace ffx {

constexpr int kWarp = 32;
constexpr int kOrder = 5;            // PME B-spline order supported by the kernels
constexpr double kElecAngToDebye = 4.80321;

// Status bits written by kernels into Handle::d_flags.
enum : int {
  FLAG_NBR_OVERFLOW = 1,
  FLAG_EWALD_OVERFLOW = 2,
  FLAG_PRECOND_OVERFLOW = 4,
  FLAG_NONFINITE = 8,
  FLAG_REBUILD = 16,
  FLAG_IMAGE_RANGE = 32,   // a multi-image shift beyond the 10-bit packing (|n| > 511)
  FLAG_NEAR_INVALID = 64,  // a hydrogen's reduction offset exceeds the near list's margin
  FLAG_QUANT_RANGE = 128,  // mixed form: a fixed-point (2^-32) value reached kQuantLimit
};

// The mixed form accumulates forces, torques and the PME mesh as FP64 sums of values
// rounded to multiples of 2^-32: such sums are exact, hence independent of the order of
// the atomics, while every partial sum stays below 2^21 in magnitude.  A contribution or
// an accumulated value of kQuantLimit = 2^20 or more raises FLAG_QUANT_RANGE, and the
// evaluation returns FFXG_ERR_RANGE: its results are complete and FP64-accurate, but no
// longer guaranteed to repeat bit for bit.
constexpr double kQuantLimit = 1048576.0;
__device__ __forceinline__ bool quant_out(double v) { return fabs(v) >= kQuantLimit; }

// The near list: at every rebuild of the buffered list the cell builder also keeps the
// pairs within ewald-cutoff + buffer + 2 kNearDelta on the reduced coordinates, where
// kNearDelta bounds |x - x_reduced| of every atom.  Any pair within the Ewald cutoff at
// a later evaluation (real coordinates) is in it, so the Ewald sub-list scans that row
// instead of the full one; an atom whose reduction offset exceeds kNearDelta makes that
// evaluation scan the full row (FLAG_NEAR_INVALID).
constexpr double kNearDelta = 0.25;

// Exclusion codes: bits 0-2 mpole class, 3-5 polar class, 6 same polarization group,
// 7-8 vdW class.
struct ScaleTables {
  double m[5];   // 1, m12, m13, m14, m15
  double p[5];   // 1, p12, p13, p14, intra14*p14
  double d[2];   // 1, d11
  double v[4];   // 1, v12, v13, v14
};

// Cell / Crystal description for the device: the rows of A^-1 are the lattice vectors
// (a, 0, 0), (b cos g, b sin g, 0), (c cos b, c beta_term, c gamma_term) and A their inverse
// (Crystal.updateCrystal, C/Crystal.java:1428-1548).  tric == 0 (every angle 90) keeps the
// diagonal arithmetic of the orthorhombic cell; otherwise Crystal.image's general
// fractional round trip is kept term by term.
struct Box {
  double a, b, c;
  double A00, A11, A22;    // 1/a, 1/b, 1/c when orthorhombic
  double Ai00, Ai11, Ai22; // a, b, c when orthorhombic
  double volume;
  double A10, A20, A21;    // off-diagonal terms of A (lower triangular)
  double Ai10, Ai20, Ai21; // off-diagonal terms of A^-1 (lower triangular)
  int tric;
};

// Minimum image exactly as Crystal.image (Crystal.java:1069-1083): no FMA
// contraction, Java signum semantics, same operation order.
__device__ __forceinline__ double jsignum(double v) { return v > 0.0 ? 1.0 : (v < 0.0 ? -1.0 : v); }

// Fractional coordinates x A in Crystal.image's operation order.
__device__ __forceinline__ void to_frac(double x, double y, double z, const Box &bx, double &xf, double &yf,
                                        double &zf) {
  if (!bx.tric) {
    xf = __dmul_rn(x, bx.A00);
    yf = __dmul_rn(y, bx.A11);
    zf = __dmul_rn(z, bx.A22);
    return;
  }
  xf = __dadd_rn(__dadd_rn(__dmul_rn(x, bx.A00), __dmul_rn(y, bx.A10)), __dmul_rn(z, bx.A20));
  yf = __dadd_rn(__dmul_rn(y, bx.A11), __dmul_rn(z, bx.A21));
  zf = __dmul_rn(z, bx.A22);
}

__device__ __forceinline__ double image_exact(double &x, double &y, double &z, const Box &bx) {
  double xf, yf, zf;
  to_frac(x, y, z, bx, xf, yf, zf);
  xf = __dadd_rn(__dmul_rn(floor(__dadd_rn(fabs(xf), 0.5)), jsignum(-xf)), xf);
  yf = __dadd_rn(__dmul_rn(floor(__dadd_rn(fabs(yf), 0.5)), jsignum(-yf)), yf);
  zf = __dadd_rn(__dmul_rn(floor(__dadd_rn(fabs(zf), 0.5)), jsignum(-zf)), zf);
  if (!bx.tric) {
    x = __dmul_rn(xf, bx.Ai00);
    y = __dmul_rn(yf, bx.Ai11);
    z = __dmul_rn(zf, bx.Ai22);
  } else {
    x = __dadd_rn(__dadd_rn(__dmul_rn(xf, bx.Ai00), __dmul_rn(yf, bx.Ai10)), __dmul_rn(zf, bx.Ai20));
    y = __dadd_rn(__dmul_rn(yf, bx.Ai11), __dmul_rn(zf, bx.Ai21));
    z = __dmul_rn(zf, bx.Ai22);
  }
  return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

// The lattice translation sign * (n A^-1) added to a displacement, in the oracle's order.
__device__ __forceinline__ void add_shift(double &x, double &y, double &z, int nx, int ny, int nz, double sign,
                                          const Box &bx) {
  if (!bx.tric) {
    x = __dadd_rn(x, sign * __dmul_rn((double)nx, bx.Ai00));
    y = __dadd_rn(y, sign * __dmul_rn((double)ny, bx.Ai11));
    z = __dadd_rn(z, sign * __dmul_rn((double)nz, bx.Ai22));
    return;
  }
  const double sx = __dadd_rn(__dadd_rn(__dmul_rn((double)nx, bx.Ai00), __dmul_rn((double)ny, bx.Ai10)),
                              __dmul_rn((double)nz, bx.Ai20));
  const double sy = __dadd_rn(__dmul_rn((double)ny, bx.Ai11), __dmul_rn((double)nz, bx.Ai21));
  const double sz = __dmul_rn((double)nz, bx.Ai22);
  x = __dadd_rn(x, sign * sx);
  y = __dadd_rn(y, sign * sy);
  z = __dadd_rn(z, sign * sz);
}

// Multi-image lists (boxes at most twice an interaction cutoff; the reference's
// ReplicatesCrystal case, C/ReplicatesCrystal.java:172-202): each list entry carries the
// lattice shift n of its image x_k + n L in a parallel int array, packed as three 10-bit
// fields offset by 512 with bit 30 set on the pair's minimum-image entry (the only one the
// bonded masks touch).  sh == nullptr selects the minimum image.
__device__ __host__ __forceinline__ int pack_shift(int nx, int ny, int nz, bool primary) {
  return (nx + 512) | ((ny + 512) << 10) | ((nz + 512) << 20) | (primary ? (1 << 30) : 0);
}

// r = (x_k - x_i) + sign * n L for entry e (sign = -1 for the vdW convention x_i - x_k),
// else Crystal.image; r^2 in Crystal.image's operation order, without contraction.
__device__ __forceinline__ double pair_image(double &x, double &y, double &z, const Box &bx,
                                             const int *__restrict__ sh, size_t e, double sign) {
  if (sh == nullptr) return image_exact(x, y, z, bx);
  const int c = sh[e];
  add_shift(x, y, z, (c & 1023) - 512, ((c >> 10) & 1023) - 512, ((c >> 20) & 1023) - 512, sign, bx);
  return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

// Whether entry e is its pair's minimum image (always, outside multi-image mode).
__device__ __forceinline__ bool pair_primary(const int *__restrict__ sh, size_t e) {
  return sh == nullptr || ((sh[e] >> 30) & 1);
}

// Whether entry e (atom i, partner k) is the one that counts an image pair once: k > i, or
// k == i with n > 0 in (z, y, x) lexicographic order.
__device__ __forceinline__ bool pair_counted(int i, int k, const int *__restrict__ sh, size_t e) {
  if (k != i) return k > i;
  if (sh == nullptr) return false;
  const int c = sh[e];
  const int nx = (c & 1023) - 512, ny = ((c >> 10) & 1023) - 512, nz = ((c >> 20) & 1023) - 512;
  return nz > 0 || (nz == 0 && (ny > 0 || (ny == 0 && nx > 0)));
}

// Arithmetic of the two precision forms.  Pair kernels are templates on the pair-math
// type R: double for the plain FP64 form, float for the mixed form (displacements,
// list tests, reductions and accumulators stay FP64 in both).
template <typename R> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };
template <typename R> __device__ __forceinline__ typename Vec2<R>::type mk2(R a, R b);
template <> __device__ __forceinline__ double2 mk2<double>(double a, double b) { return make_double2(a, b); }
template <> __device__ __forceinline__ float2 mk2<float>(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double m_sqrt(double v) { return sqrt(v); }
__device__ __forceinline__ float m_sqrt(float v) { return sqrtf(v); }
__device__ __forceinline__ double m_exp(double v) { return exp(v); }
__device__ __forceinline__ float m_exp(float v) { return expf(v); }
__device__ __forceinline__ double m_erfc(double v) { return erfc(v); }
__device__ __forceinline__ float m_erfc(float v) { return erfcf(v); }
__device__ __forceinline__ double m_min(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ float m_min(float a, float b) { return fminf(a, b); }
// Products, sums and fused multiply-adds whose rounding is fixed in the source: the
// compiler neither fuses nor splits them, so every instance of a kernel body (one system
// or a batch, launch.cuh) rounds alike.
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float xfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double xfma(double a, double b, double c) { return __fma_rn(a, b, c); }

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// One 32-byte read-only global load: a single 256-bit access on sm_100 (one pass through
// the L1 for a gathered record instead of two or three).  p must be 32-byte aligned and
// point to global memory.
__device__ __forceinline__ void ldg_32b(const float *p, float *v) {
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
      : "l"(__cvta_generic_to_global(p)));
}
__device__ __forceinline__ void ldg_32b(const double *p, double *v) {
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
      : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
      : "l"(__cvta_generic_to_global(p)));
}

// Packed per-atom source records for the field gathers: T[8] per atom = (D xyz, CR xyz,
// pad), T = double (plain form) or float (mixed form), so a neighbour costs one 64- or
// 32-byte record instead of six scattered loads.  Positions are packed as double2
// pairs (x, y), (z, 0).
template <typename T>
__device__ __forceinline__ void put_rec(T *rec, int i, double d0, double d1, double d2, double p0, double p1,
                                        double p2) {
  T *q = rec + 8 * (size_t)i;
  if constexpr (sizeof(T) == 8) {
    reinterpret_cast<double2 *>(q)[0] = make_double2(d0, d1);
    reinterpret_cast<double2 *>(q)[1] = make_double2(d2, p0);
    reinterpret_cast<double2 *>(q)[2] = make_double2(p1, p2);
  } else {
    reinterpret_cast<float4 *>(q)[0] = make_float4((float)d0, (float)d1, (float)d2, (float)p0);
    reinterpret_cast<float2 *>(q)[2] = make_float2((float)p1, (float)p2);
  }
}

template <typename T>
__device__ __forceinline__ void get_rec(const T *__restrict__ rec, int k, T *v) {
  const T *q = rec + 8 * (size_t)k;
  if constexpr (sizeof(T) == 8) {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(q)), b = __ldg(reinterpret_cast<const double2 *>(q) + 1),
                  c = __ldg(reinterpret_cast<const double2 *>(q) + 2);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y; v[4] = c.x; v[5] = c.y;
  } else {
    float a[8];
    ldg_32b(q, a);
#pragma unroll
    for (int c = 0; c < 6; c++) v[c] = a[c];
  }
}

// Per-atom gather records of the real-space energy and field kernels, kRecStride values
// of the pair type per atom: 0-9 the global-frame multipole (quadrupole divided by 3),
// 10 the Thole damping factor, 11 the Thole parameter, 12-15 zero, 16-18 u_D, 19-21 u_P,
// 22-23 zero.  A pair reads its partner's row as a few aligned 16-byte loads from 2-3
// (FP32) or 4-6 (FP64) sectors instead of one sector per structure-of-arrays column.
constexpr int kRecStride = 24;
constexpr int kRecInduced = 16;

// M entries of atom k's record from entry OFF (both multiples of four values or two).
template <int OFF, int M>
__device__ __forceinline__ void load_rec(const float *__restrict__ rec, int k, float *v) {
  static_assert(OFF % 8 == 0 && M % 4 == 0, "float records load as 32 bytes, then 16");
  const float *q = rec + (size_t)k * kRecStride + OFF;
#pragma unroll
  for (int j = 0; j < M / 8; j++) ldg_32b(q + 8 * j, v + 8 * j);
  if constexpr (M % 8 == 4) {
    const float4 t = __ldg(reinterpret_cast<const float4 *>(q + M - 4));
    v[M - 4] = t.x; v[M - 3] = t.y; v[M - 2] = t.z; v[M - 1] = t.w;
  }
}
template <int OFF, int M>
__device__ __forceinline__ void load_rec(const double *__restrict__ rec, int k, double *v) {
  static_assert(OFF % 2 == 0 && M % 2 == 0, "double records load as double2");
  const double2 *q = reinterpret_cast<const double2 *>(rec + (size_t)k * kRecStride + OFF);
#pragma unroll
  for (int j = 0; j < M / 2; j++) {
    const double2 t = __ldg(q + j);
    v[2 * j] = t.x; v[2 * j + 1] = t.y;
  }
}

// Position of atom k from the packed (x, y), (z, 0) pairs: one 32-byte sector.
__device__ __forceinline__ void load_pos(const double2 *__restrict__ pos, int k, double &x, double &y, double &z) {
  double t[4];
  ldg_32b(reinterpret_cast<const double *>(pos + 2 * (size_t)k), t);
  x = t[0]; y = t[1]; z = t[2];
}

// One cached pair of the dipole-field lists: the minimum-image displacement r = x_k - x_i
// and the coefficients A (scalar part) and B (dyadic part) of the field -A u + B (u.r) r.
// Plain form: FP64, 40 bytes; mixed form: FP32, 20 bytes.  Stored as a 32- or 16-byte
// record (x, y, z, A) plus B in a parallel array of 8-byte slots (store_pair_b), both read
// as coalesced streams.
template <typename T> struct PairRec;
template <> struct alignas(32) PairRec<double> { double2 xy, za; };
template <> struct alignas(16) PairRec<float> { float4 v; };

__device__ __forceinline__ void store_pair(PairRec<double> *p, size_t e, double x, double y, double z, double a) {
  p[e].xy = make_double2(x, y);
  p[e].za = make_double2(z, a);
}
__device__ __forceinline__ void store_pair(PairRec<float> *p, size_t e, float x, float y, float z, float a) {
  p[e].v = make_float4(x, y, z, a);
}
__device__ __forceinline__ void load_pair(const PairRec<double> *__restrict__ p, size_t e, double &x, double &y,
                                          double &z, double &a) {
  const double2 u = __ldg(&p[e].xy), v = __ldg(&p[e].za);
  x = u.x; y = u.y; z = v.x; a = v.y;
}
__device__ __forceinline__ void load_pair(const PairRec<float> *__restrict__ p, size_t e, float &x, float &y,
                                          float &z, float &a) {
  const float4 u = __ldg(&p[e].v);
  x = u.x; y = u.y; z = u.z; a = u.w;
}

// The dyadic coefficient B of cached pair e and its partner k.  Plain form: B in its own
// FP64 array, k from the list row.  Mixed form: (k, B) packed in the same 8-byte slot, so
// one load brings both (the list row is still written for the other pair kernels).
__device__ __forceinline__ void store_pair_b(double *pb, size_t e, int, double b) { pb[e] = b; }
__device__ __forceinline__ void store_pair_b(float *pb, size_t e, int k, float b) {
  reinterpret_cast<int2 *>(pb)[e] = make_int2(k, __float_as_int(b));
}
__device__ __forceinline__ void load_pair_b(const double *__restrict__ pb, const int *__restrict__ lst, size_t e,
                                            int &k, double &b) {
  k = __ldg(lst + e);
  b = __ldg(pb + e);
}
__device__ __forceinline__ void load_pair_b(const float *__restrict__ pb, const int *__restrict__, size_t e, int &k,
                                            float &b) {
  const int2 t = __ldg(reinterpret_cast<const int2 *>(pb) + e);
  k = t.x;
  b = __int_as_float(t.y);
}

// PME transforms of one handle (passed to kernels by value).
struct PmeConst {
  double tmm[10][10];   // ReciprocalSpace.transformMultipoleMatrix
  double tfm[10][10];   // ReciprocalSpace.transformFieldMatrix
  double afrac[3][3];   // Cartesian -> fractional dipole (ReciprocalSpace.a)
  double recip[3][3];   // crystal.A
};

// One axis of the batched line FFT (see pme.cu).
struct FftAxis {
  int len;            // transform length
  int stride;         // element stride within a line (complex units)
  int L;              // lines per CTA
  int line_step;      // memory step between adjacent lines of a CTA group
  int groups_inner;   // CTA groups along the inner index
  int group_step_inner, group_step_outer;
  int nradix;
  int radix[12];
};

// Device-side state of the PCG solve (read by the host after the loop).
struct PcgState {
  double eps;     // last convergence measure, Debye
  int iter;       // completed iterations
  int status;     // FFXG_OK or the SCF error status
  int cont;       // 1 while the loop should continue
  int pad;
};

// vdW softcore constants of the current lambda (VanDerWaals.setLambda).
struct AlchConst {
  double sc1, dsc1dL, d2sc1dL2, sc2, dsc2dL, d2sc2dL2;
  int active, inter, intra;
};

// One electrostatics evaluation of the lambda scheme (ParticleMeshEwald condensedEnergy /
// condensedNoLigandSCF / ligandElec, PME:1609-1796): which parts run, their scales, the
// softcore shift of pairs with a soft atom and the lambda derivatives to accumulate.
// The default is the plain evaluation.
struct ElecStep {
  int lam;                 // accumulate dU/dL, d2U/dL2, dU/dX dL
  int doPermReal;          // permanent real space
  int doPol;               // polarization
  double permScale;        // reciprocal/self permanent scale; real-space scale of soft pairs
  double polScale;
  double dEdLSign;
  double beta, dlAlpha, d2lAlpha;               // softcore shift and its lambda derivatives
  double dlPowPerm, d2lPowPerm, dlPowPol, d2lPowPol;
};
inline ElecStep plain_step() { return ElecStep{0, 1, 1, 1.0, 1.0, 1.0, 0, 0, 0, 0, 0, 0, 0}; }

// Electrostatic lambda keys and their values at lambda (AlchemicalParameters,
// pme/AlchemicalParameters.java:60-190, update :306-380).
struct ElecAlchemy {
  bool on = false;
  double permAlpha = 2.0, permExp = 3.0, permStart = 0.4, permEnd = 1.0;
  double polStart = 0.75, polEnd = 1.0, polExp = 3.0;
  bool vaporElec = true, noLigandSCF = true;
  double lAlpha = 0, dlAlpha = 0, d2lAlpha = 0;
  double lPowPerm = 1, dlPowPerm = 0, d2lPowPerm = 0;
  double lPowPol = 1, dlPowPol = 0, d2lPowPol = 0;
};

// Host copy of the system inputs (kept to build sub-systems, e.g. the vacuum ligand).
struct SystemCopy {
  int n = 0, n_vdw_types = 0;
  std::vector<double> xyz, multipole, polarizability, thole, pdamp, red_factor, vdw_inv_rmin, vdw_eps;
  std::vector<int> frame, axis, vdw_type, red_parent;
  std::vector<std::vector<int>> m12, m13, m14, m15, ip11;
};

struct Handle {
  // ---- configuration
  int n = 0;
  ffxg_params prm{};
  bool mixed = false;            // FFXG_PRECISION_MIXED: FP32 pair math, B-splines, mesh and FFT
  Box box{};
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  int64_t launches = 0;
  Recorder *rec = nullptr;            // set while a batch records this system's launches
  unsigned char *d_stage = nullptr;   // while recording: this system's slot of the batch's result staging

  // ---- static per-atom parameters (device)
  double *d_lmp = nullptr;        // [10][n] local multipoles
  int *d_frame = nullptr;         // [n]
  int *d_axis = nullptr;          // [3][n]
  double *d_polar = nullptr, *d_thole = nullptr, *d_ipdamp = nullptr;
  int *d_vtype = nullptr, *d_redp = nullptr;
  double *d_redf = nullptr;
  int ntypes = 0;
  double *d_vrad = nullptr, *d_veps = nullptr;   // [t][t]
  int *d_excl_ptr = nullptr, *d_excl_k = nullptr;  // exclusions CSR (sorted by k)
  unsigned *d_excl_code = nullptr;
  int *d_excl_lo = nullptr, *d_excl_hi = nullptr;  // min/max partner per atom
  int *d_tq_ptr = nullptr, *d_tq_ent = nullptr;    // torque gather CSR: entry = i*4 + slot
  int *d_red_ptr = nullptr, *d_red_child = nullptr;  // reduction children CSR
  ScaleTables scales{};

  // ---- coordinates and list state
  double *d_x = nullptr, *d_y = nullptr, *d_z = nullptr;
  double *d_rx = nullptr, *d_ry = nullptr, *d_rz = nullptr;
  double *d_refx = nullptr, *d_refy = nullptr, *d_refz = nullptr;  // list reference coords
  bool list_valid = false;
  int ncell[3] = {0, 0, 0};
  int cell_cap = 0;                           // cells the cell-list arrays hold
  int *d_cell_cnt = nullptr, *d_cell_start = nullptr, *d_cell_atoms = nullptr, *d_atom_cell = nullptr;
  int cap_nbr = 0, cap_ewl = 0, cap_prl = 0;
  int *d_nbr = nullptr, *d_nbr_cnt = nullptr;
  bool near_list = false;                     // minimum-image cell lists with a near list
  int cap_nbl = 0;
  int *d_nbl = nullptr, *d_nbl_cnt = nullptr;
  int *d_ewl = nullptr, *d_ewl_cnt = nullptr;
  int *d_prl = nullptr, *d_prl_cnt = nullptr;
  // Multi-image lists: on when an edge is at most twice an interaction cutoff (or forced
  // with ffxg_set_image_mode); then every buffered and Ewald entry has a packed shift.
  int64_t graph_gen = 0;                             // bumped whenever captured graphs go stale
  bool images = false;
  int image_mode = 0;                                // FFXG_IMAGES_AUTO / FFXG_IMAGES_ALL
  int img_range[3] = {0, 0, 0};                      // |n - n0| bound per axis of the builder
  int img_rep[3] = {1, 1, 1};                        // replicate supercell whose minimum image is primary
  Box img_super{};                                   // that supercell
  double width[3] = {0, 0, 0};                       // perpendicular widths of the cell
  int *d_nbr_sh = nullptr, *d_ewl_sh = nullptr;
  // Cached dipole-field pairs of the Ewald and preconditioner rows (PairRec + B), sized
  // for the FP64 records; the mixed form uses the leading half.
  PairRec<double> *d_coefE = nullptr, *d_coefP = nullptr;
  double *d_coefEB = nullptr, *d_coefPB = nullptr;
  double *d_part2 = nullptr;                        // PCG partial sums of the fixed-grid kernels
  unsigned *d_counter = nullptr;                    // last-block counter (returns to 0 after each use)

  // ---- electrostatics work arrays
  double *d_gm = nullptr;                     // [10][n]
  double *d_rot = nullptr;                    // [9][n] local-to-global rotation (row-major)
  double *d_fm = nullptr;                     // [10][n]
  double *d_spl = nullptr;                    // [n][3][order][4]
  int *d_igrid = nullptr;                     // [3][n]
  double *d_cphi = nullptr, *d_fphi = nullptr;    // [20][n] permanent
  double *d_cphiI = nullptr, *d_fphiI = nullptr;  // [20][n] induced D
  double *d_cphiP = nullptr, *d_fphiP = nullptr;  // [20][n] induced CR
  double *d_fieldD = nullptr, *d_fieldP = nullptr;  // [3][n]
  double *d_uD = nullptr, *d_uP = nullptr, *d_udirD = nullptr, *d_udirP = nullptr;
  // PCG vectors [3][n]
  double *d_r = nullptr, *d_rP = nullptr, *d_zpre = nullptr, *d_zpreP = nullptr, *d_p = nullptr, *d_pP = nullptr;
  double *d_vec = nullptr, *d_vecP = nullptr;
  // Packed gather records: positions (x, y), (z, 0) per atom, and the field source
  // dipoles of the PCG fields, [n][8] of double (plain) or float (mixed): d_recF holds
  // the dipoles whose field is taken (u, then p), d_recP holds alpha r.
  double2 *d_pos = nullptr;
  void *d_recF = nullptr, *d_recP = nullptr;
  void *d_erec = nullptr;                     // [n][kRecStride] real-space gather records
  double2 *d_rpos = nullptr;                  // [n] (rx, ry), (rz, vdW type bits): vdW gather record
  double *d_tpair = nullptr;                  // [6][n] pair field of the current source
  double *d_tp = nullptr;                     // [6][n] field of the PCG direction p
  cudaStream_t aux = nullptr;                 // runs the pair field beside spread + FFT
  cudaStream_t aux_side = nullptr;            // the same inside the PCG while-node body capture
                                              // (a stream forked into a capture stays in it)
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  double *d_partials = nullptr;               // block partial sums [nblk][8]
  int part_rows = 0;                          // rows of each PCG partial-sum region of d_part2
  double *d_scalars = nullptr;                // PCG scalars on device
  double *h_scalars = nullptr;                // pinned mirror
  // PME
  int nfft[3] = {0, 0, 0};
  double2 *d_grid = nullptr;
  double *d_influence = nullptr;
  double2 *d_twiddle = nullptr;               // per-axis twiddle tables (3 x max n)
  // Mixed form: d_spl holds float data; spreading accumulates (exactly) in the double
  // mesh d_grid and the FFT and interpolation run on the FP32 mesh d_gridf.
  float2 *d_gridf = nullptr;
  float *d_influencef = nullptr;
  float2 *d_twiddlef = nullptr;
  // The mixed form's accumulation mesh as two planes of doubles (real, imaginary).
  double *d_grid_planes() const { return reinterpret_cast<double *>(d_grid); }
  PmeConst pc{};
  FftAxis axes[3]{};

  // ---- outputs
  double *d_grad = nullptr, *d_torque = nullptr;  // [3][n]
  double *d_gred = nullptr;                        // [3][n] vdW reduced-site force
  double *d_eatom = nullptr;                       // [kEnergyRows][n] per-atom energy terms
  long long *d_catom = nullptr;                    // [2][n] per-atom counts
  double *d_result = nullptr;                      // reduced terms
  long long *d_cresult = nullptr;
  int *d_flags = nullptr;
  int *h_flags = nullptr;
  double *d_xyz_in = nullptr, *d_grad_out = nullptr;  // interleaved staging [n][3]
  double *h_xyz_pin = nullptr, *h_grad_pin = nullptr;

  int scf_iter = 0;
  // Alchemical state (vdW softcore): soft flags, molecule ids, keys, lambda and the
  // lambda derivatives of the last evaluation.
  AlchConst alch{0, 0, 0, 1, 0, 0, 0, 0, 0};
  double alch_alpha = 0.25, alch_exponent = 3.0, alch_end = 1.0, lambda = 1.0;
  int *d_soft = nullptr, *d_mol = nullptr;
  double *d_lgred = nullptr;                       // [6][n]: reduced-site and distributed dU/dX dL
  double dEdL = 0.0, d2EdL2 = 0.0;
  bool lgrad_valid = false;
  // Electrostatic lambda (elec-lambdaterm): keys, the current step, the lambda gradient and
  // torque of the electrostatics, per-step accumulators, the polarizabilities with the soft
  // atoms removed, the charge corrections of the whole and soft-free systems, and the
  // vacuum sub-system of the soft atoms (lig[j] = its atom j in this system).
  ElecAlchemy elec;
  ElecStep step = plain_step();
  double *d_lg = nullptr, *d_lt = nullptr;          // [3][n] each
  double *d_acc = nullptr;                          // [3+3+8+3+3][n] step accumulators
  double *d_polar_all = nullptr, *d_polar_env = nullptr;
  double e_corr_env = 0.0;
  Handle *vac = nullptr;
  std::vector<int> lig;
  std::vector<int> soft_host, mol_host;             // the last ffxg_set_alchemy's atoms
  int *d_lig = nullptr;
  bool vacuum = false;                              // this handle is a vacuum sub-system
  int eps_atoms = 0;                                // atom count of the PCG residual norm (0: n);
                                                    // a sub-system uses its parent's (PCGSolver.java:546)
  SystemCopy sys;
  // Molecular dynamics state (md.cu): masses, SETTLE molecules and the trajectory arrays
  // (interleaved [n][3]): positions, velocities, accelerations, prior positions, gradient.
  bool md_ready = false;
  double *d_mass = nullptr, *d_mdx = nullptr, *d_mdv = nullptr, *d_mda = nullptr, *d_mdxp = nullptr;
  double *d_mdg = nullptr, *d_mdke = nullptr;
  int *d_settle = nullptr;
  int n_settle = 0;
  double settle_d1 = 0.0, settle_d2 = 0.0;
  PcgState *d_pcg = nullptr, *h_pcg = nullptr;
  int scf_predictor = FFXG_PREDICTOR_NONE;
  double *d_aspc = nullptr;                         // [6][6][n] ASPC ring of u - u_dir
  int *d_aspc_state = nullptr;                      // most recent slot, slots stored
  // Graph execution: the whole evaluation captured once per gradient mode and replayed.
  bool use_graphs = true;
  bool want_grad = true;                            // gradient requested by the current call
  bool grad_to_pin = false, grad_pinned = false;    // host-gradient call: D2H queued before the sync
  cudaStream_t side = nullptr;                      // captures the PCG while-node body
  // Captured evaluations run the vdW term (independent of electrostatics) on its own
  // low-priority stream beside the permanent field and the PCG, joined before the gradient.
  bool capturing = false;
  bool batch_branch = false;                        // captured as one branch of a batch graph
  int num_sms = 148;
  cudaStream_t vdw_stream = nullptr;
  cudaEvent_t ev_vdw_fork = nullptr, ev_vdw_join = nullptr;
  // ... and the reciprocal-space chains (permanent: beside the real-space field; final
  // induced: beside the real-space energy) on a second high-priority stream.
  cudaStream_t recip_stream = nullptr;
  cudaEvent_t ev_recip_fork = nullptr, ev_recip_join = nullptr;
  bool recip_forked = false;
  // Per call kind: energy only, gradient on the device, gradient to the host (the graph
  // then ends with the gradient's device-to-host copy beside the energy sums).
  cudaGraphExec_t graph_exec[3] = {nullptr, nullptr, nullptr};
  int64_t graph_launches[3] = {0, 0, 0};            // kernels outside the PCG body
  int64_t graph_body_launches = 0;
  double e_charge_correction = 0.0;
  // Stage timers (PMETimings counterpart).
  bool timing = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<int> ev_stage;       // stage of each begin/end pair recorded this call
  int ev_used = 0;
  double stage_ms[16] = {0};
  int64_t stage_calls[16] = {0};
  int64_t list_builds = 0;
  int64_t growths = 0;             // list capacity regrowths during the current call
};

// Ewald coefficient of the evaluation: 0 for a vacuum sub-system (no screening).
inline double ewald_alpha_of(const Handle &h) { return h.vacuum ? 0.0 : h.prm.ewald_alpha; }

// Rows of Handle::d_eatom: vdW, permanent real, polarization real, permanent self,
// permanent reciprocal, polarization self, polarization reciprocal, vdW dU/dL, vdW d2U/dL2,
// electrostatic dU/dL, electrostatic d2U/dL2.
constexpr int kEnergyRows = 11;

// ---- kernels / launchers (defined in the .cu files)
void launch_set_coordinates(Handle &h, const double *d_xyz);
void launch_neighbor_list(Handle &h, bool force);
void launch_vdw(Handle &h, bool grad, cudaStream_t st);
void launch_rotate(Handle &h);
void launch_bsplines(Handle &h);
// Copies m doubles into dst (the pinned staging buffer) and tests them for Inf/NaN in the
// same pass (exponent bits all ones); false if any is not finite.
bool copy_finite(double *dst, const double *src, size_t m);
bool copy_finite_parallel(double *dst, const double *src, size_t m);
void copy_parallel(double *dst, const double *src, size_t m);
void launch_spread_permanent(Handle &h);
void launch_spread_induced(Handle &h, const double *ud, const double *up);
void launch_fft_convolution(Handle &h);
void launch_phi_permanent(Handle &h);
void launch_phi_induced(Handle &h);
void launch_realspace_field(Handle &h);
void launch_direct_dipoles(Handle &h);
int run_pcg(Handle &h, bool capture);
// Evaluation entry points shared by the single-system ABI and batches (handle.cu).
int evaluate(Handle &h, const double *d_xyz, double *d_grad_xyz, bool grad, double *terms, int64_t *counts);
int eval_capture_body(Handle &h, const double *d_xyz, double *d_grad);
int eval_after_graph(Handle &h, double *terms, int64_t *counts);
Handle &handle_of(ffxg_handle *hh);
int pcg_partial_rows(int n);
int md_setup(Handle &h, const ffxg_md *md);
int md_run(Handle &h, double dt, int steps, double *xyz, double *vel, double *epot, double *ekin,
           int (*force)(Handle &, const double *, double *, double *));
void launch_recip_energy(Handle &h, bool grad);
void launch_real_energy(Handle &h, bool grad);
void launch_torque(Handle &h);
void launch_torque_of(Handle &h, const double *torque, double *out);
void launch_elec_accumulate(Handle &h, bool first);
void launch_elec_restore(Handle &h);
void launch_lambda_grad_add(Handle &h, double *out);
void launch_zero_soft_multipoles(Handle &h);
void launch_assemble(Handle &h, double *d_grad_xyz);
void launch_reduce_results(Handle &h);
int param_gradients(Handle &h, double *dEdM, double *dEdA);
int setup_pme(Handle &h);   // FFXG_OK or a status (h.err set)

inline int nblocks(int64_t n, int t) { return (int)((n + t - 1) / t); }

// Bracket a stage with events when timing is on; returns a token for timer_end.
inline int timer_begin(Handle &h, int stage) {
  if (!h.timing) return -1;
  if (h.ev_used + 2 > (int)h.ev_pool.size()) {
    for (int k = 0; k < 64; k++) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      h.ev_pool.push_back(e);
    }
  }
  const int tok = h.ev_used;
  h.ev_used += 2;
  h.ev_stage.push_back(stage);
  cudaEventRecord(h.ev_pool[tok], h.stream);
  return tok;
}
inline void timer_end(Handle &h, int tok) {
  if (tok >= 0) cudaEventRecord(h.ev_pool[tok + 1], h.stream);
}
// The same on another stream of the handle.
inline int timer_begin_on(Handle &h, int stage, cudaStream_t st) {
  cudaStream_t keep = h.stream;
  h.stream = st;
  const int tok = timer_begin(h, stage);
  h.stream = keep;
  return tok;
}
inline void timer_end_on(Handle &h, int tok, cudaStream_t st) {
  if (tok >= 0) cudaEventRecord(h.ev_pool[tok + 1], st);
}
// Accumulate the recorded pairs (stream must be synchronised).
inline void timer_collect(Handle &h) {
  for (size_t q = 0; q < h.ev_stage.size(); q++) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h.ev_pool[2 * q], h.ev_pool[2 * q + 1]);
    h.stage_ms[h.ev_stage[q]] += ms;
    h.stage_calls[h.ev_stage[q]] += 1;
  }
  h.ev_stage.clear();
  h.ev_used = 0;
}

#define FFX_LAUNCHED(h) ((h).launches++)

}  // namespace ffx
