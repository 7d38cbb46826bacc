// handle.cu -- the C ABI (include/ffxcuda.h) and the per-evaluation pipeline.
//
// One evaluation follows ForceFieldEnergy.energy (ForceFieldEnergy.java:1638-1800) for the
// vdW and PME terms and ParticleMeshEwald.computeEnergy (ParticleMeshEwald.java:1871-2183):
//   coordinates -> reduced coordinates + motion check -> (re)build lists when needed
//   -> vdW -> rotate multipoles -> B-splines -> permanent spread/FFT/phi -> permanent field
//   -> direct dipoles -> PCG -> induced phi -> reciprocal and real-space energy/gradient
//   -> torque to gradient -> deterministic sums.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "ffx_internal.cuh"

struct ffxg_handle {
  ffx::Handle h;
};

using namespace ffx;

static std::string g_create_error;

// Gathers and scatters between a system and its vacuum sub-system (lig[j] = atom j's index).
__global__ void k_gather_xyz(int m, const int *__restrict__ idx, const double *__restrict__ src, double *dst) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const int i = idx[j];
  for (int d = 0; d < 3; d++) dst[3 * j + d] = src[3 * i + d];
}

__global__ void k_scatter_add_xyz(int m, const int *__restrict__ idx, const double *__restrict__ src, double *dst) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const int i = idx[j];
  for (int d = 0; d < 3; d++) dst[3 * i + d] += src[3 * j + d];
}

__global__ void k_scatter_add_soa(int m, int n, const int *__restrict__ idx, const double *__restrict__ src,
                                  double *dst) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const int i = idx[j];
  for (int d = 0; d < 3; d++) dst[(size_t)d * n + i] += src[(size_t)d * m + j];
}


#define CK(call)                                                                    \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      h.err = std::string(#call) + ": " + cudaGetErrorString(e_);                   \
      return FFXG_ERR_CUDA;                                                         \
    }                                                                               \
  } while (0)

template <typename T>
static cudaError_t dalloc(T **p, size_t count) {
  return cudaMalloc((void **)p, std::max<size_t>(count, 1) * sizeof(T));
}

// Any mesh length of at least the B-spline order: radices 2, 3, 4, 5, 7 have their own
// butterflies and larger prime factors the general pass (Complex.java:173-330, 371-383).
// A length has at most 12 factors (4096 = 4^6 needs 6).
static bool fft_supported(int n) {
  if (n < kOrder || n > 4096) return false;
  int m = n, count = 0;
  for (int f : {4, 2, 3, 5, 7})
    while (m % f == 0) { m /= f; count++; }
  for (int f = 11; m > 1; f += 2)
    while (m % f == 0) { m /= f; count++; }
  return count <= 12;
}

__device__ __forceinline__ void k_set_flags(VGrid, int *flags, int v) { *flags = v; }

// m doubles cleared.
__device__ __forceinline__ void k_zero(VGrid vg, size_t m, double *p) {
  for (size_t j = (size_t)vg.bid * blockDim.x + threadIdx.x; j < m; j += (size_t)vg.nblk * blockDim.x) p[j] = 0.0;
}

// words 4-byte words copied (a result into a batch's staging buffer).
__device__ __forceinline__ void k_copy_words(VGrid, const unsigned *src, unsigned *dst, int words) {
  for (int j = threadIdx.x; j < words; j += blockDim.x) dst[j] = src[j];
}

static void zero_doubles(Handle &h, double *p, size_t m) {
  launch_on<k_zero, 0, 0>(h.rec, (int)std::min<size_t>(nblocks((int64_t)m, 256), 2 * (size_t)h.num_sms), 256, 0,
                          h.stream, m, p);
  FFX_LAUNCHED(h);
}

// A result read back to the host: queued on the handle's stream, or, while a batch records
// the evaluation, copied on the device into the system's slot of the batch's staging
// buffer (the batch reads every slot back with one copy and hands each system its bytes).
static void copy_result(Handle &h, void *host, const void *dev, size_t bytes) {
  if (h.rec) {
    const size_t off = h.rec->stage_bytes;
    launch_on<k_copy_words, 0, 0>(h.rec, 1, 32, 0, h.stream, (const unsigned *)dev,
                                  (unsigned *)(h.d_stage + off), (int)(bytes / 4));
    h.rec->copies.push_back(Recorder::Copy{dev, off, host, bytes});
    h.rec->stage_bytes += (bytes + 15) & ~(size_t)15;
    return;
  }
  cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, h.stream);
}

static void drop_graphs(Handle &h) {
  for (cudaGraphExec_t &g : h.graph_exec)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  h.graph_gen++;   // batches holding this handle's evaluation recapture
}

static int alloc_lists(Handle &h) {
  drop_graphs(h);   // the captured kernels hold the old list pointers
  if (h.d_nbr) cudaFree(h.d_nbr);
  if (h.d_nbl) cudaFree(h.d_nbl);
  h.d_nbl = nullptr;
  if (h.d_ewl) cudaFree(h.d_ewl);
  if (h.d_prl) cudaFree(h.d_prl);
  if (h.d_coefE) cudaFree(h.d_coefE);
  if (h.d_coefP) cudaFree(h.d_coefP);
  if (h.d_coefEB) cudaFree(h.d_coefEB);
  if (h.d_coefPB) cudaFree(h.d_coefPB);
  if (h.d_nbr_sh) cudaFree(h.d_nbr_sh);
  if (h.d_ewl_sh) cudaFree(h.d_ewl_sh);
  h.d_nbr_sh = h.d_ewl_sh = nullptr;
  h.d_nbr = h.d_ewl = h.d_prl = nullptr;
  h.d_coefE = h.d_coefP = nullptr;
  h.d_coefEB = h.d_coefPB = nullptr;
  CK(dalloc(&h.d_nbr, (size_t)h.n * h.cap_nbr));
  if (h.near_list) CK(dalloc(&h.d_nbl, (size_t)h.n * h.cap_nbl));
  CK(dalloc(&h.d_ewl, (size_t)h.n * h.cap_ewl));
  CK(dalloc(&h.d_prl, (size_t)h.n * h.cap_prl));
  CK(dalloc(&h.d_coefE, (size_t)h.n * h.cap_ewl));
  CK(dalloc(&h.d_coefP, (size_t)h.n * h.cap_prl));
  CK(dalloc(&h.d_coefEB, (size_t)h.n * h.cap_ewl));
  CK(dalloc(&h.d_coefPB, (size_t)h.n * h.cap_prl));
  if (h.images) {
    CK(dalloc(&h.d_nbr_sh, (size_t)h.n * h.cap_nbr));
    CK(dalloc(&h.d_ewl_sh, (size_t)h.n * h.cap_ewl));
  }
  h.list_valid = false;
  return FFXG_OK;
}

static int round32(double v) { return ((int)std::ceil(v) + 31) / 32 * 32; }

// Crystal.updateCrystal (C/Crystal.java:1428-1548): lattice vectors as the rows of A^-1,
// A their inverse (lower triangular: closed form), the volume and the perpendicular widths
// 1 / |a*_d|, by the orthorhombic, monoclinic (only beta differs from 90) and general
// branches.  Angles of 0 read as 90.
static Box make_box(const double box[3], const double angles[3], double width[3]) {
  Box b{};
  b.a = box[0]; b.b = box[1]; b.c = box[2];
  double ang[3];
  for (int d = 0; d < 3; d++) ang[d] = (angles[d] > 0.0) ? angles[d] : 90.0;
  if (ang[0] == 90.0 && ang[1] == 90.0 && ang[2] == 90.0) {
    b.A00 = 1.0 / b.a; b.A11 = 1.0 / b.b; b.A22 = 1.0 / b.c;
    b.Ai00 = b.a; b.Ai11 = b.b; b.Ai22 = b.c;
    b.volume = b.a * b.b * b.c;
    b.tric = 0;
    width[0] = b.a; width[1] = b.b; width[2] = b.c;
    return b;
  }
  const double deg = 0.017453292519943295;   // Math.toRadians
  double cos_alpha, sin_beta, cos_beta, sin_gamma, cos_gamma, beta_term, gamma_term;
  if (ang[0] == 90.0 && ang[2] == 90.0) {
    cos_alpha = 0.0; sin_beta = std::sin(ang[1] * deg); cos_beta = std::cos(ang[1] * deg);
    sin_gamma = 1.0; cos_gamma = 0.0; beta_term = 0.0; gamma_term = sin_beta;
    b.volume = sin_beta * b.a * b.b * b.c;
  } else {
    cos_alpha = std::cos(ang[0] * deg); sin_beta = std::sin(ang[1] * deg); cos_beta = std::cos(ang[1] * deg);
    sin_gamma = std::sin(ang[2] * deg); cos_gamma = std::cos(ang[2] * deg);
    beta_term = (cos_alpha - cos_beta * cos_gamma) / sin_gamma;
    gamma_term = std::sqrt(sin_beta * sin_beta - beta_term * beta_term);
    b.volume = sin_gamma * gamma_term * b.a * b.b * b.c;
  }
  b.Ai00 = b.a;
  b.Ai10 = b.b * cos_gamma; b.Ai11 = b.b * sin_gamma;
  b.Ai20 = b.c * cos_beta; b.Ai21 = b.c * beta_term; b.Ai22 = b.c * gamma_term;
  b.A00 = 1.0 / b.Ai00; b.A11 = 1.0 / b.Ai11; b.A22 = 1.0 / b.Ai22;
  b.A10 = -b.Ai10 / (b.Ai00 * b.Ai11);
  b.A21 = -b.Ai21 / (b.Ai11 * b.Ai22);
  b.A20 = (b.Ai10 * b.Ai21 - b.Ai11 * b.Ai20) / (b.Ai00 * b.Ai11 * b.Ai22);
  b.tric = 1;
  width[0] = 1.0 / std::sqrt(b.A00 * b.A00 + b.A10 * b.A10 + b.A20 * b.A20);
  width[1] = 1.0 / std::sqrt(b.A11 * b.A11 + b.A21 * b.A21);
  width[2] = 1.0 / std::fabs(b.A22);
  return b;
}

static bool angles_ok(const double angles[3]) {
  for (int d = 0; d < 3; d++) {
    const double v = angles[d] > 0.0 ? angles[d] : 90.0;
    if (!(v > 0.0 && v < 180.0)) return false;
  }
  return true;
}

static void set_cell(Handle &h, const double box[3], const double angles[3]) {
  for (int d = 0; d < 3; d++) {
    h.prm.box[d] = box[d];
    h.prm.angles[d] = angles[d];
  }
  h.box = make_box(box, angles, h.width);
}

// Cells of the list builder: fractional slabs at least half the buffered cutoff wide.
static void set_cell_grid(Handle &h) {
  const double rlist = std::max(h.prm.vdw_cutoff, h.prm.ewald_cutoff) + h.prm.list_buffer;
  for (int d = 0; d < 3; d++) h.ncell[d] = std::max(1, (int)std::floor(h.width[d] / (rlist * 0.5)));
}

// Charge correction of a charged cell, -1/2 electric pi q^2 / (V alpha^2)
// (ReciprocalEnergyRegion.java:229-255), for total charge q.
static double charge_correction(const Handle &h, double q) {
  const double PI = 3.14159265358979323846;
  return (q != 0.0) ? -0.5 * h.prm.electric * PI * (q * q) / (h.box.volume * h.prm.ewald_alpha * h.prm.ewald_alpha)
                    : 0.0;
}

// The PME mesh of h.prm.pme_grid, its influence function and twiddles (any earlier mesh
// is released first).
static int alloc_mesh(Handle &h) {
  for (void *q : {(void *)h.d_grid, (void *)h.d_influence, (void *)h.d_twiddle, (void *)h.d_gridf,
                  (void *)h.d_influencef, (void *)h.d_twiddlef})
    if (q) cudaFree(q);
  h.d_grid = nullptr; h.d_influence = nullptr; h.d_twiddle = nullptr;
  h.d_gridf = nullptr; h.d_influencef = nullptr; h.d_twiddlef = nullptr;
  const int nfx = h.prm.pme_grid[0], nfy = h.prm.pme_grid[1], nfz = h.prm.pme_grid[2];
  const size_t ng = (size_t)nfx * nfy * nfz;
  CK(dalloc(&h.d_grid, ng)); CK(dalloc(&h.d_influence, ng));
  CK(cudaMemset(h.d_grid, 0, ng * sizeof(double2)));   // the mixed form keeps it clear between uses
  CK(dalloc(&h.d_twiddle, 3 * (size_t)std::max(nfx, std::max(nfy, nfz))));
  if (h.mixed) {
    CK(dalloc(&h.d_gridf, ng));
    CK(dalloc(&h.d_influencef, ng));
    CK(dalloc(&h.d_twiddlef, 3 * (size_t)std::max(nfx, std::max(nfy, nfz))));
  }
  return FFXG_OK;
}

static double near_radius(const Handle &h) {
  return h.prm.ewald_cutoff + h.prm.list_buffer + 2.0 * kNearDelta;
}

// Multi-image mode and the shift range of its list builder: |n_d - n0_d| <=
// floor(rlist / w_d + 1/2), n0 the minimum-image shift and w_d the perpendicular width,
// covers every image within rlist.  The primary image of a pair (the one the bonded masks
// apply to) is the minimum image in the replicate supercell of the reference
// (ReplicatesCrystal.replicatesCrystalFactory, C/ReplicatesCrystal.java:172-202: the
// smallest counts whose interfacial radii, half the widths, reach rlist).
static void configure_images(Handle &h) {
  const ffxg_params *p = &h.prm;
  const double rcut = std::max(std::max(p->vdw_cutoff, p->ewald_cutoff), p->precond_cutoff);
  const double rlist = std::max(p->vdw_cutoff, p->ewald_cutoff) + p->list_buffer;
  h.images = h.image_mode == FFXG_IMAGES_ALL;
  double sbox[3], sw[3];
  for (int d = 0; d < 3; d++) {
    if (h.width[d] <= 2.0 * rcut) h.images = true;
    h.img_range[d] = (int)std::floor(rlist / h.width[d] + 0.5);
    h.img_rep[d] = 1;
    while (h.width[d] / 2.0 * h.img_rep[d] < rlist) h.img_rep[d]++;
    sbox[d] = p->box[d] * h.img_rep[d];
  }
  h.img_super = make_box(sbox, p->angles, sw);
  h.near_list = !h.images && !h.vacuum && near_radius(h) < rlist;
}

// Host copy of the inputs (sub-systems are built from it).
static void copy_system(const ffxg_system *s, SystemCopy &c) {
  const int n = s->n_atoms;
  c.n = n;
  c.n_vdw_types = s->n_vdw_types;
  c.xyz.assign(s->xyz, s->xyz + 3 * (size_t)n);
  c.multipole.assign(s->multipole, s->multipole + 10 * (size_t)n);
  c.frame.assign(s->frame, s->frame + n);
  c.axis.assign(s->axis, s->axis + 3 * (size_t)n);
  c.polarizability.assign(s->polarizability, s->polarizability + n);
  c.thole.assign(s->thole, s->thole + n);
  c.pdamp.assign(s->pdamp, s->pdamp + n);
  c.vdw_type.assign(s->vdw_type, s->vdw_type + n);
  c.red_parent.assign(s->red_parent, s->red_parent + n);
  c.red_factor.assign(s->red_factor, s->red_factor + n);
  const size_t t2 = (size_t)s->n_vdw_types * s->n_vdw_types;
  c.vdw_inv_rmin.assign(s->vdw_inv_rmin, s->vdw_inv_rmin + t2);
  c.vdw_eps.assign(s->vdw_eps, s->vdw_eps + t2);
  auto csr = [&](const int32_t *ptr, const int32_t *idx, std::vector<std::vector<int>> &out) {
    out.assign(n, {});
    if (!ptr) return;
    for (int i = 0; i < n; i++) out[i].assign(idx + ptr[i], idx + ptr[i + 1]);
  };
  csr(s->mask12_ptr, s->mask12_idx, c.m12);
  csr(s->mask13_ptr, s->mask13_idx, c.m13);
  csr(s->mask14_ptr, s->mask14_idx, c.m14);
  csr(s->mask15_ptr, s->mask15_idx, c.m15);
  csr(s->ip11_ptr, s->ip11_idx, c.ip11);
}

static int create_impl(const ffxg_system *s, const ffxg_params *p, Handle &h) {
  const int n = s->n_atoms;
  h.n = n;
  h.prm = *p;
  if (n <= 0) { h.err = "n_atoms must be positive"; return FFXG_ERR_BAD_ARG; }
  if (!s->xyz || !s->multipole || !s->frame || !s->axis || !s->polarizability || !s->thole || !s->pdamp ||
      !s->vdw_type || !s->red_parent || !s->red_factor || !s->vdw_inv_rmin || !s->vdw_eps) {
    h.err = "null per-atom array"; return FFXG_ERR_BAD_ARG;
  }
  copy_system(s, h.sys);
  if (p->pme_order != kOrder) { h.err = "only pme-order 5 is supported"; return FFXG_ERR_BAD_ARG; }
  if (!angles_ok(p->angles)) { h.err = "cell angles must lie in (0, 180) degrees"; return FFXG_ERR_BAD_ARG; }
  for (int d = 0; d < 3; d++) {
    if (!(p->box[d] > 0.0)) { h.err = "box edges must be positive"; return FFXG_ERR_BAD_ARG; }
    if (!fft_supported(p->pme_grid[d])) {
      h.err = "PME grid dimensions must lie in [5, 4096]";
      return FFXG_ERR_BAD_ARG;
    }
  }
  set_cell(h, p->box, p->angles);
  if (!(h.box.volume > 0.0)) { h.err = "the cell angles give no volume"; return FFXG_ERR_BAD_ARG; }
  // ReplicatesCrystal (C/ReplicatesCrystal.java:172-202) switches to a supercell of
  // replicate cells when an edge is shorter than twice the buffered list cutoff.  While
  // every interaction cutoff stays below half of each edge, each pair has exactly one
  // image within any cutoff, so the minimum image on the unit cell (with the buffered
  // list, whose extra images lie beyond every cutoff) gives the same energy.  A cutoff of
  // half an edge or more takes multi-image lists: every lattice image inside the cutoffs,
  // the sum the replicate supercell forms.
  h.image_mode = FFXG_IMAGES_AUTO;
  configure_images(h);
  const double rlist = std::max(p->vdw_cutoff, p->ewald_cutoff) + p->list_buffer;
  if (p->ewald_alpha <= 0.0) { h.err = "ewald-alpha must be positive"; return FFXG_ERR_BAD_ARG; }
  if (p->precision != FFXG_PRECISION_FP64 && p->precision != FFXG_PRECISION_MIXED) {
    h.err = "unknown precision"; return FFXG_ERR_BAD_ARG;
  }
  h.mixed = (p->precision == FFXG_PRECISION_MIXED);
  if (p->polarization < FFXG_POLAR_NONE || p->polarization > FFXG_POLAR_MUTUAL) {
    h.err = "unknown polarization"; return FFXG_ERR_BAD_ARG;
  }
  // Device.
  int dev = 0;
  CK(cudaGetDevice(&dev));
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, dev));
  if (prop.major < 10) { h.err = "requires an sm_100 (Blackwell) device"; return FFXG_ERR_CUDA; }
  h.device = dev;
  // The PCG's mesh chain (spread, FFT, combine) is its critical path; the real-space pair
  // field beside it runs on lower-priority streams so that it fills the SMs the chain
  // leaves idle instead of taking them from it.
  int prio_low = 0, prio_high = 0;
  CK(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
  CK(cudaStreamCreateWithPriority(&h.stream, cudaStreamNonBlocking, prio_high));
  CK(cudaStreamCreateWithPriority(&h.side, cudaStreamNonBlocking, prio_high));
  CK(cudaStreamCreateWithPriority(&h.aux, cudaStreamNonBlocking, prio_low));
  CK(cudaStreamCreateWithPriority(&h.aux_side, cudaStreamNonBlocking, prio_low));
  CK(cudaStreamCreateWithPriority(&h.vdw_stream, cudaStreamNonBlocking, prio_low));
  h.num_sms = prop.multiProcessorCount;
  CK(cudaEventCreateWithFlags(&h.ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&h.ev_join, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&h.ev_vdw_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&h.ev_vdw_join, cudaEventDisableTiming));
  CK(cudaStreamCreateWithPriority(&h.recip_stream, cudaStreamNonBlocking, prio_high));
  CK(cudaEventCreateWithFlags(&h.ev_recip_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&h.ev_recip_join, cudaEventDisableTiming));


  // ---- validate topology indices
  for (int i = 0; i < n; i++) {
    const int fr = s->frame[i];
    if (fr < FFXG_FRAME_NONE || fr > FFXG_FRAME_THREEFOLD) { h.err = "bad frame type"; return FFXG_ERR_BAD_ARG; }
    const int need = (fr == FFXG_FRAME_NONE) ? 0 : (fr == FFXG_FRAME_ZONLY) ? 1
                     : (fr == FFXG_FRAME_ZTHENBISECTOR || fr == FFXG_FRAME_THREEFOLD) ? 3 : 2;
    for (int a = 0; a < need; a++) {
      const int ax = s->axis[3 * i + a];
      if (ax < 0 || ax >= n || ax == i) { h.err = "bad frame-defining atom index"; return FFXG_ERR_BAD_ARG; }
    }
    if (s->red_parent[i] < 0 || s->red_parent[i] >= n) { h.err = "bad reduction parent"; return FFXG_ERR_BAD_ARG; }
    if (s->vdw_type[i] < 0 || s->vdw_type[i] >= s->n_vdw_types) { h.err = "bad vdW type"; return FFXG_ERR_BAD_ARG; }
  }

  // ---- exclusion codes: bits 0-2 mpole class, 3-5 polar class, 6 group, 7-8 vdW class
  std::vector<std::map<int, unsigned>> ex(n);
  auto each = [&](const int32_t *ptr, const int32_t *idx, auto fn) {
    for (int i = 0; i < n; i++)
      for (int e = ptr[i]; e < ptr[i + 1]; e++) fn(i, idx[e]);
  };
  auto setbits = [&](int i, int k, unsigned mask, unsigned val) {
    if (k < 0 || k >= n || k == i) return;
    unsigned &c = ex[i][k];
    c = (c & ~mask) | val;
  };
  each(s->mask12_ptr, s->mask12_idx, [&](int i, int k) { setbits(i, k, 7u | (7u << 3) | (3u << 7), 1u | (1u << 3) | (1u << 7)); });
  each(s->mask13_ptr, s->mask13_idx, [&](int i, int k) { setbits(i, k, 7u | (7u << 3) | (3u << 7), 2u | (2u << 3) | (2u << 7)); });
  each(s->mask14_ptr, s->mask14_idx, [&](int i, int k) { setbits(i, k, 7u | (7u << 3) | (3u << 7), 3u | (3u << 3) | (3u << 7)); });
  each(s->mask15_ptr, s->mask15_idx, [&](int i, int k) { setbits(i, k, 7u, 4u); });
  each(s->ip11_ptr, s->ip11_idx, [&](int i, int k) { setbits(i, k, 1u << 6, 1u << 6); });
  // A 1-4 partner inside the same polarization group takes polar-14-intra (PermanentFieldRegion.java:241-248).
  for (int i = 0; i < n; i++)
    for (auto &kv : ex[i])
      if (((kv.second >> 3) & 7u) == 3u && (kv.second & (1u << 6))) kv.second = (kv.second & ~(7u << 3)) | (4u << 3);
  std::vector<int> eptr(n + 1, 0), ek, elo(n, 0x7fffffff), ehi(n, -1);
  std::vector<unsigned> ecode;
  for (int i = 0; i < n; i++) {
    for (auto &kv : ex[i]) {
      ek.push_back(kv.first);
      ecode.push_back(kv.second);
      elo[i] = std::min(elo[i], kv.first);
      ehi[i] = std::max(ehi[i], kv.first);
    }
    eptr[i + 1] = (int)ek.size();
  }
  h.scales.m[0] = 1.0; h.scales.m[1] = p->m12; h.scales.m[2] = p->m13; h.scales.m[3] = p->m14; h.scales.m[4] = p->m15;
  h.scales.p[0] = 1.0; h.scales.p[1] = p->p12; h.scales.p[2] = p->p13; h.scales.p[3] = p->p14;
  h.scales.p[4] = p->intra14 * p->p14;
  h.scales.d[0] = 1.0; h.scales.d[1] = p->d11;
  h.scales.v[0] = 1.0; h.scales.v[1] = p->v12; h.scales.v[2] = p->v13; h.scales.v[3] = p->v14;

  // ---- torque gather CSR: atom j <- (i, slot) for each frame atom of i and i itself
  std::vector<std::vector<int>> tq(n);
  std::vector<std::vector<int>> kids(n);
  for (int i = 0; i < n; i++) {
    const int fr = s->frame[i];
    if (fr != FFXG_FRAME_NONE) {
      tq[s->axis[3 * i]].push_back(i * 4 + 0);
      if (fr != FFXG_FRAME_ZONLY) tq[s->axis[3 * i + 1]].push_back(i * 4 + 1);
      if (fr == FFXG_FRAME_ZTHENBISECTOR || fr == FFXG_FRAME_THREEFOLD) tq[s->axis[3 * i + 2]].push_back(i * 4 + 2);
      tq[i].push_back(i * 4 + 3);
    }
    if (s->red_parent[i] != i) kids[s->red_parent[i]].push_back(i);
  }
  std::vector<int> tqp(n + 1, 0), tqe, rp(n + 1, 0), rc;
  for (int j = 0; j < n; j++) {
    std::sort(tq[j].begin(), tq[j].end());
    tqe.insert(tqe.end(), tq[j].begin(), tq[j].end());
    tqp[j + 1] = (int)tqe.size();
    rc.insert(rc.end(), kids[j].begin(), kids[j].end());
    rp[j + 1] = (int)rc.size();
  }

  // ---- capacities from the density
  const double rho = n / h.box.volume;
  const double PI = 3.14159265358979323846;
  auto sphere = [&](double r) { return 4.0 / 3.0 * PI * r * r * r * rho; };
  h.cap_nbr = round32(1.3 * sphere(rlist) + 64);
  h.cap_nbl = round32(1.3 * sphere(std::min(near_radius(h), rlist)) + 64);
  h.cap_ewl = round32(1.3 * sphere(p->ewald_cutoff) + 32);
  h.cap_prl = round32(1.3 * sphere(p->precond_cutoff) + 32);
  set_cell_grid(h);
  const int ncells = h.ncell[0] * h.ncell[1] * h.ncell[2];
  h.cell_cap = ncells;

  // ---- allocations
  const size_t N = n;
  CK(dalloc(&h.d_lmp, 10 * N)); CK(dalloc(&h.d_frame, N)); CK(dalloc(&h.d_axis, 3 * N));
  CK(dalloc(&h.d_polar, N)); CK(dalloc(&h.d_thole, N)); CK(dalloc(&h.d_ipdamp, N));
  CK(dalloc(&h.d_vtype, N)); CK(dalloc(&h.d_redp, N)); CK(dalloc(&h.d_redf, N));
  h.ntypes = s->n_vdw_types;
  CK(dalloc(&h.d_vrad, (size_t)h.ntypes * h.ntypes)); CK(dalloc(&h.d_veps, (size_t)h.ntypes * h.ntypes));
  CK(dalloc(&h.d_excl_ptr, N + 1)); CK(dalloc(&h.d_excl_k, ek.size())); CK(dalloc(&h.d_excl_code, ecode.size()));
  CK(dalloc(&h.d_excl_lo, N)); CK(dalloc(&h.d_excl_hi, N));
  CK(dalloc(&h.d_tq_ptr, N + 1)); CK(dalloc(&h.d_tq_ent, tqe.size()));
  CK(dalloc(&h.d_red_ptr, N + 1)); CK(dalloc(&h.d_red_child, rc.size()));
  CK(dalloc(&h.d_x, N)); CK(dalloc(&h.d_y, N)); CK(dalloc(&h.d_z, N));
  CK(dalloc(&h.d_rx, N)); CK(dalloc(&h.d_ry, N)); CK(dalloc(&h.d_rz, N));
  CK(dalloc(&h.d_refx, N)); CK(dalloc(&h.d_refy, N)); CK(dalloc(&h.d_refz, N));
  CK(dalloc(&h.d_cell_cnt, 2 * (size_t)ncells)); CK(dalloc(&h.d_cell_start, (size_t)ncells + 1));
  CK(dalloc(&h.d_cell_atoms, N)); CK(dalloc(&h.d_atom_cell, N));
  CK(dalloc(&h.d_nbr_cnt, N)); CK(dalloc(&h.d_ewl_cnt, N)); CK(dalloc(&h.d_prl_cnt, N));
  CK(dalloc(&h.d_nbl_cnt, N));
  if (int st = alloc_lists(h)) return st;
  CK(dalloc(&h.d_gm, 10 * N)); CK(dalloc(&h.d_fm, 10 * N)); CK(dalloc(&h.d_rot, 9 * N));
  CK(dalloc(&h.d_spl, N * 3 * kOrder * 4)); CK(dalloc(&h.d_igrid, 3 * N));
  CK(dalloc(&h.d_cphi, 20 * N)); CK(dalloc(&h.d_fphi, 20 * N));
  CK(dalloc(&h.d_cphiI, 20 * N)); CK(dalloc(&h.d_fphiI, 20 * N));
  CK(dalloc(&h.d_cphiP, 20 * N)); CK(dalloc(&h.d_fphiP, 20 * N));
  CK(dalloc(&h.d_fieldD, 3 * N)); CK(dalloc(&h.d_fieldP, 3 * N));
  CK(dalloc(&h.d_uD, 3 * N)); CK(dalloc(&h.d_uP, 3 * N)); CK(dalloc(&h.d_udirD, 3 * N)); CK(dalloc(&h.d_udirP, 3 * N));
  CK(dalloc(&h.d_r, 3 * N)); CK(dalloc(&h.d_rP, 3 * N)); CK(dalloc(&h.d_zpre, 3 * N)); CK(dalloc(&h.d_zpreP, 3 * N));
  CK(dalloc(&h.d_p, 3 * N)); CK(dalloc(&h.d_pP, 3 * N));
  CK(dalloc(&h.d_pos, 2 * N)); CK(dalloc(&h.d_rpos, 2 * N));
  CK(cudaMalloc(&h.d_erec, (size_t)kRecStride * N * sizeof(double)));
  CK(cudaMemset(h.d_erec, 0, (size_t)kRecStride * N * sizeof(double)));
  CK(dalloc(&h.d_tpair, 6 * N)); CK(dalloc(&h.d_tp, 6 * N));
  CK(cudaMalloc(&h.d_recF, 8 * N * sizeof(double)));
  CK(cudaMalloc(&h.d_recP, 8 * N * sizeof(double))); CK(dalloc(&h.d_vec, 3 * N)); CK(dalloc(&h.d_vecP, 3 * N));
  const size_t nparts = std::max<size_t>((size_t)nblocks(n, 256) * 8, 148 * 16) + 64;
  CK(dalloc(&h.d_partials, nparts));
  h.part_rows = pcg_partial_rows(n);
  CK(dalloc(&h.d_part2, 3 * (size_t)h.part_rows * 8));
  CK(dalloc(&h.d_counter, 4));
  CK(cudaMemset(h.d_counter, 0, 4 * sizeof(unsigned)));
  CK(dalloc(&h.d_scalars, 16));
  CK(cudaMallocHost((void **)&h.h_scalars, 16 * sizeof(double)));
  CK(cudaMalloc((void **)&h.d_pcg, sizeof(PcgState)));
  CK(cudaMallocHost((void **)&h.h_pcg, sizeof(PcgState)));
  if (int st = alloc_mesh(h)) return st;
  CK(dalloc(&h.d_grad, 3 * N)); CK(dalloc(&h.d_torque, 3 * N)); CK(dalloc(&h.d_gred, 6 * N));
  CK(dalloc(&h.d_eatom, (size_t)kEnergyRows * N)); CK(dalloc(&h.d_catom, 2 * N));
  CK(cudaMemset(h.d_eatom, 0, (size_t)kEnergyRows * N * sizeof(double)));
  CK(dalloc(&h.d_result, 16)); CK(dalloc(&h.d_cresult, 8));
  CK(dalloc(&h.d_flags, 1));
  CK(cudaMallocHost((void **)&h.h_flags, 64));
  CK(dalloc(&h.d_xyz_in, 3 * N)); CK(dalloc(&h.d_grad_out, 3 * N));
  CK(cudaMallocHost((void **)&h.h_xyz_pin, 3 * N * sizeof(double)));
  CK(cudaMallocHost((void **)&h.h_grad_pin, 3 * N * sizeof(double)));

  // ---- uploads (SoA)
  std::vector<double> lmp(10 * N);
  std::vector<int> axis(3 * N);
  std::vector<double> ipd(N);
  for (int i = 0; i < n; i++) {
    for (int t = 0; t < 10; t++) lmp[t * N + i] = s->multipole[10 * (size_t)i + t];
    for (int a = 0; a < 3; a++) axis[a * N + i] = s->axis[3 * (size_t)i + a];
    ipd[i] = (s->pdamp[i] > 0.0) ? 1.0 / s->pdamp[i] : INFINITY;  // ParticleMeshEwald.java:1401-1406
  }
  CK(cudaMemcpy(h.d_lmp, lmp.data(), 10 * N * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_frame, s->frame, N * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_axis, axis.data(), 3 * N * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_polar, s->polarizability, N * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_thole, s->thole, N * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_ipdamp, ipd.data(), N * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_vtype, s->vdw_type, N * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_redp, s->red_parent, N * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_redf, s->red_factor, N * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_vrad, s->vdw_inv_rmin, (size_t)h.ntypes * h.ntypes * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_veps, s->vdw_eps, (size_t)h.ntypes * h.ntypes * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_excl_ptr, eptr.data(), (N + 1) * sizeof(int), cudaMemcpyHostToDevice));
  if (!ek.empty()) {
    CK(cudaMemcpy(h.d_excl_k, ek.data(), ek.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h.d_excl_code, ecode.data(), ecode.size() * sizeof(unsigned), cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(h.d_excl_lo, elo.data(), N * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_excl_hi, ehi.data(), N * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_tq_ptr, tqp.data(), (N + 1) * sizeof(int), cudaMemcpyHostToDevice));
  if (!tqe.empty()) CK(cudaMemcpy(h.d_tq_ent, tqe.data(), tqe.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_red_ptr, rp.data(), (N + 1) * sizeof(int), cudaMemcpyHostToDevice));
  if (!rc.empty()) CK(cudaMemcpy(h.d_red_child, rc.data(), rc.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemset(h.d_refx, 0, N * sizeof(double)));
  CK(cudaMemset(h.d_refy, 0, N * sizeof(double)));
  CK(cudaMemset(h.d_refz, 0, N * sizeof(double)));
  CK(cudaMemset(h.d_grad, 0, 3 * N * sizeof(double)));
  CK(cudaMemset(h.d_torque, 0, 3 * N * sizeof(double)));
  CK(cudaMemset(h.d_gred, 0, 6 * N * sizeof(double)));
  CK(cudaMemset(h.d_eatom, 0, 10 * N * sizeof(double)));
  CK(cudaMemset(h.d_catom, 0, 2 * N * sizeof(long long)));
  CK(cudaMemset(h.d_uD, 0, 3 * N * sizeof(double)));
  CK(cudaMemset(h.d_uP, 0, 3 * N * sizeof(double)));
  // Charge correction for a charged cell (ReciprocalEnergyRegion.java:229-255).
  {
    double q = 0.0;
    for (int i = 0; i < n; i++) q += s->multipole[10 * (size_t)i];
    h.e_charge_correction = charge_correction(h, q);
  }
  if (const int st = setup_pme(h)) return st;
  CK(cudaGetLastError());
  // Coordinates.
  std::memcpy(h.h_xyz_pin, s->xyz, 3 * N * sizeof(double));
  CK(cudaMemcpy(h.d_xyz_in, h.h_xyz_pin, 3 * N * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaDeviceSynchronize());
  return FFXG_OK;
}

static void free_all(Handle &h);

static void drop_vacuum(Handle &h) {
  if (h.vac) {
    free_all(*h.vac);
    delete h.vac;
    h.vac = nullptr;
  }
}

static void free_all(Handle &h) {
  drop_vacuum(h);
  if (h.d_polar_all) h.d_polar = h.d_polar_all;   // the step-2 swap never outlives a call
  void *ptrs[] = {h.d_lmp, h.d_frame, h.d_axis, h.d_polar, h.d_thole, h.d_ipdamp, h.d_vtype, h.d_redp, h.d_redf,
                  h.d_vrad, h.d_veps, h.d_excl_ptr, h.d_excl_k, h.d_excl_code, h.d_excl_lo, h.d_excl_hi, h.d_tq_ptr,
                  h.d_tq_ent, h.d_red_ptr, h.d_red_child, h.d_x, h.d_y, h.d_z, h.d_rx, h.d_ry, h.d_rz, h.d_refx,
                  h.d_refy, h.d_refz, h.d_cell_cnt, h.d_cell_start, h.d_cell_atoms, h.d_atom_cell, h.d_nbr,
                  h.d_nbr_cnt, h.d_nbl, h.d_nbl_cnt, h.d_ewl, h.d_ewl_cnt, h.d_prl, h.d_prl_cnt, h.d_gm, h.d_fm, h.d_spl, h.d_igrid,
                  h.d_cphi, h.d_fphi, h.d_cphiI, h.d_fphiI, h.d_cphiP, h.d_fphiP, h.d_fieldD, h.d_fieldP, h.d_uD,
                  h.d_uP, h.d_udirD, h.d_udirP, h.d_r, h.d_rP, h.d_zpre, h.d_zpreP, h.d_p, h.d_pP, h.d_vec, h.d_vecP,
                  h.d_partials, h.d_scalars, h.d_grid, h.d_influence, h.d_twiddle, h.d_gridf, h.d_influencef, h.d_twiddlef, h.d_grad, h.d_torque, h.d_gred,
                  h.d_eatom, h.d_catom, h.d_result, h.d_cresult, h.d_flags, h.d_xyz_in, h.d_grad_out,
                  h.d_coefE, h.d_coefP, h.d_coefEB, h.d_coefPB, h.d_part2, h.d_counter, h.d_pos, h.d_rpos, h.d_erec, h.d_recF, h.d_recP, h.d_tpair, h.d_tp, h.d_soft, h.d_mol, h.d_lgred, h.d_mass, h.d_mdx, h.d_mdv, h.d_mda, h.d_mdxp, h.d_mdg, h.d_mdke, h.d_settle, h.d_aspc, h.d_aspc_state, h.d_nbr_sh, h.d_ewl_sh, h.d_lg, h.d_lt, h.d_acc, h.d_polar_env, h.d_lig, h.d_rot};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  if (h.h_scalars) cudaFreeHost(h.h_scalars);
  if (h.h_flags) cudaFreeHost(h.h_flags);
  if (h.h_xyz_pin) cudaFreeHost(h.h_xyz_pin);
  if (h.h_grad_pin) cudaFreeHost(h.h_grad_pin);
  for (cudaEvent_t e : h.ev_pool) cudaEventDestroy(e);
  drop_graphs(h);
  if (h.d_pcg) cudaFree(h.d_pcg);
  if (h.h_pcg) cudaFreeHost(h.h_pcg);
  if (h.side) cudaStreamDestroy(h.side);
  if (h.aux) cudaStreamDestroy(h.aux);
  if (h.aux_side) cudaStreamDestroy(h.aux_side);
  if (h.vdw_stream) cudaStreamDestroy(h.vdw_stream);
  if (h.ev_fork) cudaEventDestroy(h.ev_fork);
  if (h.ev_join) cudaEventDestroy(h.ev_join);
  if (h.ev_vdw_fork) cudaEventDestroy(h.ev_vdw_fork);
  if (h.ev_vdw_join) cudaEventDestroy(h.ev_vdw_join);
  if (h.recip_stream) cudaStreamDestroy(h.recip_stream);
  if (h.ev_recip_fork) cudaEventDestroy(h.ev_recip_fork);
  if (h.ev_recip_join) cudaEventDestroy(h.ev_recip_join);
  if (h.stream) cudaStreamDestroy(h.stream);
}

namespace ffx {
bool copy_finite(double *dst, const double *src, size_t m) {
  uint64_t bad = 0;
  for (size_t j = 0; j < m; j++) {
    uint64_t u;
    std::memcpy(&u, src + j, sizeof(u));
    std::memcpy(dst + j, &u, sizeof(u));
    bad |= (uint64_t)((u & 0x7ff0000000000000ull) == 0x7ff0000000000000ull);
  }
  return bad == 0;
}

// Large host copies (a batch's coordinates in, its gradients out: tens of MB) split over
// up to eight host threads, one per 2^18 values (2 MB).
static int copy_threads(size_t m) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  return (int)std::min<size_t>(std::min<size_t>(8, hw), std::max<size_t>(1, m >> 18));
}
bool copy_finite_parallel(double *dst, const double *src, size_t m) {
  const int T = copy_threads(m);
  if (T == 1) return copy_finite(dst, src, m);
  const size_t chunk = (m + T - 1) / T;
  std::vector<char> ok(T, 1);
  std::vector<std::thread> th;
  for (int t = 1; t < T; t++) {
    const size_t a = std::min(m, t * chunk), b = std::min(m, a + chunk);
    th.emplace_back([=, &ok]() { ok[t] = copy_finite(dst + a, src + a, b - a); });
  }
  ok[0] = copy_finite(dst, src, std::min(m, chunk));
  for (std::thread &x : th) x.join();
  for (char c : ok)
    if (!c) return false;
  return true;
}
void copy_parallel(double *dst, const double *src, size_t m) {
  const int T = copy_threads(m);
  const size_t chunk = (m + T - 1) / T;
  std::vector<std::thread> th;
  for (int t = 1; t < T; t++) {
    const size_t a = std::min(m, t * chunk), b = std::min(m, a + chunk);
    th.emplace_back([=]() { std::memcpy(dst + a, src + a, (b - a) * sizeof(double)); });
  }
  std::memcpy(dst, src, std::min(m, chunk) * sizeof(double));
  for (std::thread &x : th) x.join();
}
}  // namespace ffx

// Captured evaluations of systems with a reciprocal space run the reciprocal chains as
// graph branches; inside a batch graph, whose systems are branches already, they stay in
// line (the extra branches made a 512-system batch 25% slower).
static bool branch_recip(const Handle &h) { return h.capturing && !h.vacuum && !h.batch_branch; }

// ---------------------------------------------------------------------------
// Evaluation.  emit_front (coordinates .. permanent field) and emit_back (energies,
// torques, gradient, reductions) are shared by the direct path and the captured graph.
static void emit_front(Handle &h, const double *d_xyz) {
  int tk = timer_begin(h, FFXG_STAGE_LISTS);
  launch_on<k_set_flags, 0, 0>(h.rec, 1, 1, 0, h.stream, h.d_flags, h.list_valid ? 0 : FLAG_REBUILD);
  FFX_LAUNCHED(h);
  launch_set_coordinates(h, d_xyz);
  launch_neighbor_list(h, false);
  timer_end(h, tk);
  if (h.capturing && !h.vacuum && !h.batch_branch) {
    // A branch of the graph: vdW depends on the list alone, and only the gradient
    // assembly and the sums read it (emit_back joins it there).  Inside a batch graph the
    // systems are the branches, and vdW stays in line (measured 16% more systems/s).
    cudaEventRecord(h.ev_vdw_fork, h.stream);
    cudaStreamWaitEvent(h.vdw_stream, h.ev_vdw_fork, 0);
    launch_vdw(h, h.want_grad, h.vdw_stream);
    cudaEventRecord(h.ev_vdw_join, h.vdw_stream);
  } else {
    tk = timer_begin(h, FFXG_STAGE_VDW);
    launch_vdw(h, h.want_grad, h.stream);
    timer_end(h, tk);
  }
  tk = timer_begin(h, FFXG_STAGE_MULTIPOLES);
  launch_rotate(h);
  if (!branch_recip(h)) launch_bsplines(h);
  timer_end(h, tk);
  if (branch_recip(h)) {
    // The permanent reciprocal chain needs only the global multipoles: a graph branch on
    // the second high-priority stream beside the real-space field, joined before the
    // direct dipoles.
    cudaEventRecord(h.ev_recip_fork, h.stream);
    cudaStreamWaitEvent(h.recip_stream, h.ev_recip_fork, 0);
    cudaStream_t main = h.stream;
    h.stream = h.recip_stream;
    launch_bsplines(h);
    launch_spread_permanent(h);
    launch_fft_convolution(h);
    launch_phi_permanent(h);
    cudaEventRecord(h.ev_recip_join, h.recip_stream);
    h.stream = main;
  } else {
    tk = timer_begin(h, FFXG_STAGE_PERM_RECIP);
    launch_spread_permanent(h);
    launch_fft_convolution(h);
    launch_phi_permanent(h);
    timer_end(h, tk);
  }
  tk = timer_begin(h, FFXG_STAGE_PERM_FIELD);
  launch_realspace_field(h);   // sub-lists, permanent real-space field, pair coefficients
  if (branch_recip(h)) cudaStreamWaitEvent(h.stream, h.ev_recip_join, 0);
  launch_direct_dipoles(h);
  timer_end(h, tk);
}

// The reciprocal potential of the converged dipoles.  In a captured evaluation it is a
// branch beside the real-space energy (which needs only the dipoles), joined in emit_back
// before the reciprocal energy.
static void emit_final_induced(Handle &h) {
  if (branch_recip(h)) {
    cudaEventRecord(h.ev_recip_fork, h.stream);
    cudaStreamWaitEvent(h.recip_stream, h.ev_recip_fork, 0);
    cudaStream_t main = h.stream;
    h.stream = h.recip_stream;
    launch_spread_induced(h, h.d_uD, h.d_uP);
    launch_fft_convolution(h);
    launch_phi_induced(h);
    cudaEventRecord(h.ev_recip_join, h.recip_stream);
    h.stream = main;
    h.recip_forked = true;
    return;
  }
  const int tk = timer_begin(h, FFXG_STAGE_IND_RECIP);
  launch_spread_induced(h, h.d_uD, h.d_uP);
  launch_fft_convolution(h);
  launch_phi_induced(h);
  timer_end(h, tk);
}

static void emit_no_polarization(Handle &h) {
  zero_doubles(h, h.d_uD, 3 * (size_t)h.n);
  zero_doubles(h, h.d_uP, 3 * (size_t)h.n);
}

static void emit_back(Handle &h, double *d_grad_xyz) {
  int tk = timer_begin(h, FFXG_STAGE_REAL_ENERGY);
  launch_real_energy(h, h.want_grad);
  timer_end(h, tk);
  if (h.recip_forked) {
    cudaStreamWaitEvent(h.stream, h.ev_recip_join, 0);
    h.recip_forked = false;
  }
  tk = timer_begin(h, FFXG_STAGE_RECIP_ENERGY);
  launch_recip_energy(h, h.want_grad);
  timer_end(h, tk);
  if (h.capturing && !h.vacuum && !h.batch_branch) cudaStreamWaitEvent(h.stream, h.ev_vdw_join, 0);
  tk = timer_begin(h, FFXG_STAGE_GRADIENT);
  // In a captured evaluation the energy sums, which read only the per-atom energy and
  // count rows (complete here), are a branch beside the torque gather and the gradient
  // assembly.
  const bool fork_sums = h.capturing && !h.vacuum && !h.batch_branch && !h.step.lam;
  if (fork_sums) {
    cudaEventRecord(h.ev_fork, h.stream);
    cudaStreamWaitEvent(h.aux, h.ev_fork, 0);
    cudaStream_t main = h.stream;
    h.stream = h.aux;
    launch_reduce_results(h);
    h.stream = main;
    cudaEventRecord(h.ev_join, h.aux);
  }
  if (h.want_grad) {
    launch_torque(h);
    launch_assemble(h, d_grad_xyz);
    if (h.capturing && h.grad_to_pin && !h.vacuum) {
      // Host-gradient graphs: the copy to the pinned buffer runs beside the energy sums.
      cudaEventRecord(h.ev_recip_fork, h.stream);
      cudaStreamWaitEvent(h.recip_stream, h.ev_recip_fork, 0);
      cudaMemcpyAsync(h.h_grad_pin, d_grad_xyz, 3 * (size_t)h.n * sizeof(double), cudaMemcpyDeviceToHost,
                      h.recip_stream);
      cudaEventRecord(h.ev_recip_join, h.recip_stream);
      h.recip_forked = true;
    }
  }
  if (h.step.lam) {   // electrostatic lambda gradient into the dU/dX dL rows (after the vdW part)
    if (h.vacuum) zero_doubles(h, h.d_lgred + 3 * (size_t)h.n, 3 * (size_t)h.n);
    launch_lambda_grad_add(h, h.d_lgred + 3 * (size_t)h.n);
  }
  if (fork_sums) cudaStreamWaitEvent(h.stream, h.ev_join, 0);
  else launch_reduce_results(h);
  timer_end(h, tk);
  copy_result(h, h.h_scalars, h.d_result, kEnergyRows * sizeof(double));
  copy_result(h, h.h_flags + 2, h.d_cresult, 2 * sizeof(long long));
  copy_result(h, h.h_flags, h.d_flags, sizeof(int));
  if (h.recip_forked) {
    cudaStreamWaitEvent(h.stream, h.ev_recip_join, 0);
    h.recip_forked = false;
  }
}

static const char *scf_message(int st) {
  return (st == FFXG_ERR_SCF_DIVERGED) ? "SCF convergence failure (residual grew)"
         : (st == FFXG_ERR_SCF_MAXITER) ? "maximum SCF iterations reached"
                                        : "non-finite SCF residual";
}

// Terms and counts from the pinned copies written by emit_back.
static int finish(Handle &h, bool rebuilt, double *terms, int64_t *counts) {
  double res[kEnergyRows];
  long long cres[2];
  std::memcpy(res, h.h_scalars, kEnergyRows * sizeof(double));
  h.dEdL = res[7] + res[9];
  h.d2EdL2 = res[8] + res[10];
  h.lgrad_valid = (h.alch.active && h.want_grad) || h.step.lam;
  std::memcpy(cres, h.h_flags + 2, 2 * sizeof(long long));
  double eCorr = h.vacuum ? 0.0 : h.e_charge_correction;
  if (h.step.lam && !h.vacuum) {
    // Charge corrections of the whole system (step 1, x lPowPerm) and of the system without
    // the soft atoms (step 2, x (1 - lPowPerm)); ReciprocalEnergyRegion.java:230-255.
    const ElecAlchemy &el = h.elec;
    const double ca = h.e_charge_correction, ce = h.e_corr_env;
    eCorr = el.lPowPerm * ca + (1.0 - el.lPowPerm) * ce;
    h.dEdL += el.dlPowPerm * ca - el.dlPowPerm * ce;
    h.d2EdL2 += el.d2lPowPerm * ca - el.d2lPowPerm * ce;
  }
  if (terms) {
    terms[FFXG_TERM_VDW] = res[0];
    terms[FFXG_TERM_PERM_REAL] = res[1];
    terms[FFXG_TERM_POL_REAL] = res[2];
    terms[FFXG_TERM_PERM_SELF] = res[3];
    terms[FFXG_TERM_PERM_RECIP] = res[4] + eCorr;
    terms[FFXG_TERM_POL_SELF] = res[5];
    terms[FFXG_TERM_POL_RECIP] = res[6];
    terms[FFXG_TERM_PERMANENT] = res[1] + res[3] + res[4] + eCorr;
    terms[FFXG_TERM_POLARIZATION] = res[2] + res[5] + res[6];
    terms[FFXG_TERM_TOTAL] = res[0] + terms[FFXG_TERM_PERMANENT] + terms[FFXG_TERM_POLARIZATION];
  }
  if (counts) {
    counts[FFXG_COUNT_VDW] = cres[0];
    counts[FFXG_COUNT_PERMANENT] = cres[1] + h.n;
    counts[FFXG_COUNT_SCF_ITER] = h.scf_iter;
    counts[FFXG_COUNT_LIST_BUILDS] = rebuilt ? 1 : 0;
    counts[FFXG_COUNT_LIST_PAIRS] = -1;
    counts[FFXG_COUNT_LIST_GROWTHS] = h.growths;
  }
  if (h.h_flags[0] & FLAG_NONFINITE) { h.err = "non-finite energy, torque or gradient"; return FFXG_ERR_NONFINITE; }
  for (int t = 0; t < 7; t++)
    if (!std::isfinite(res[t])) { h.err = "non-finite energy"; return FFXG_ERR_NONFINITE; }
  if (h.h_flags[0] & FLAG_QUANT_RANGE) {
    h.err = "a fixed-point force, torque or mesh sum reached 2^20: results are valid but not bitwise reproducible";
    return FFXG_ERR_RANGE;
  }
  return FFXG_OK;
}

static int grow_lists(Handle &h, int f) {
  h.growths++;
  if (f & FLAG_NBR_OVERFLOW) {   // the buffered row or the near row
    h.cap_nbr = round32(h.cap_nbr * 1.5);
    h.cap_nbl = round32(h.cap_nbl * 1.5);
  }
  if (f & FLAG_EWALD_OVERFLOW) h.cap_ewl = round32(h.cap_ewl * 1.5);
  if (f & FLAG_PRECOND_OVERFLOW) h.cap_prl = round32(h.cap_prl * 1.5);
  return alloc_lists(h);
}

static constexpr int kOverflow = FLAG_NBR_OVERFLOW | FLAG_EWALD_OVERFLOW | FLAG_PRECOND_OVERFLOW;

static int graph_key(const Handle &h) { return h.want_grad ? (h.grad_to_pin ? 2 : 1) : 0; }

// ffxg_energy with a host gradient: the device-to-host copy into the pinned buffer is
// queued before the evaluation's own synchronisation, so the call waits once.
static void copy_grad_to_pinned(Handle &h, const double *d_grad) {
  if (!h.grad_to_pin || !h.want_grad) return;
  cudaMemcpyAsync(h.h_grad_pin, d_grad, 3 * (size_t)h.n * sizeof(double), cudaMemcpyDeviceToHost, h.stream);
  h.grad_pinned = true;
}

// Direct execution: one host check of the list and coordinate flags before the solver,
// the solver's stopping test read back per iteration.  Grows list capacities and repeats
// on overflow.
static int evaluate_direct(Handle &h, const double *d_xyz, double *d_grad_xyz, double *terms, int64_t *counts) {
  for (int attempt = 0; attempt < 4; attempt++) {
    h.ev_stage.clear();
    h.ev_used = 0;
    emit_front(h, d_xyz);
    // List overflow invalidates everything downstream and non-finite coordinates
    // make the evaluation meaningless: check both before the solver.
    cudaMemcpyAsync(h.h_flags, h.d_flags, sizeof(int), cudaMemcpyDeviceToHost, h.stream);
    if (cudaStreamSynchronize(h.stream) != cudaSuccess) {
      h.err = std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError());
      return FFXG_ERR_CUDA;
    }
    const int f = h.h_flags[0];
    if (f & FLAG_NONFINITE) { h.err = "non-finite coordinates"; return FFXG_ERR_NONFINITE; }
    if (f & FLAG_IMAGE_RANGE) { h.err = "atoms more than 500 box edges apart"; return FFXG_ERR_BAD_ARG; }
    if (f & kOverflow) {
      if (int a = grow_lists(h, f)) return a;
      continue;
    }
    const bool rebuilt = (f & FLAG_REBUILD) != 0;
    if (rebuilt) h.list_builds++;
    h.list_valid = true;
    int st = FFXG_OK;
    h.scf_iter = 0;
    if (h.prm.polarization != FFXG_POLAR_NONE && h.step.doPol) {
      if (h.prm.polarization == FFXG_POLAR_MUTUAL) st = run_pcg(h, false);
      if (st == FFXG_OK) emit_final_induced(h);
    } else {
      emit_no_polarization(h);
    }
    if (st != FFXG_OK) { h.err = scf_message(st); return st; }
    emit_back(h, d_grad_xyz);
    copy_grad_to_pinned(h, d_grad_xyz);
    if (cudaStreamSynchronize(h.stream) != cudaSuccess) {
      h.err = std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError());
      return FFXG_ERR_CUDA;
    }
    if (h.timing) timer_collect(h);
    return finish(h, rebuilt, terms, counts);
  }
  h.err = "neighbour capacity could not be satisfied";
  return FFXG_ERR_CAPACITY;
}

namespace ffx {

// The whole evaluation issued onto h.stream, which is capturing (alone, or as one branch
// of a batch capture): inputs from d_xyz, gradient into d_grad, and the pinned copies of
// scalars, flags and solver state that eval_after_graph reads.
int eval_capture_body(Handle &h, const double *d_xyz, double *d_grad) {
  const int key = graph_key(h);
  const int64_t before = h.launches;
  h.capturing = true;
  emit_front(h, d_xyz);
  int st = FFXG_OK;
  if (h.prm.polarization != FFXG_POLAR_NONE) {
    if (h.prm.polarization == FFXG_POLAR_MUTUAL) st = run_pcg(h, true);
    emit_final_induced(h);
  } else {
    emit_no_polarization(h);
  }
  emit_back(h, d_grad);
  h.capturing = false;
  copy_result(h, h.h_pcg, h.d_pcg, sizeof(PcgState));
  h.graph_launches[key] = h.launches - before - h.graph_body_launches;
  return st;
}

}  // namespace ffx

// Capture the whole evaluation (internal coordinate and gradient buffers) as one graph.
static int capture_graph(Handle &h) {
  const int key = graph_key(h);
  if (cudaStreamBeginCapture(h.stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return FFXG_ERR_CUDA;
  const int st = eval_capture_body(h, h.d_xyz_in, h.d_grad_out);
  cudaGraph_t graph = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(h.stream, &graph);
  if (st != FFXG_OK || ec != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return FFXG_ERR_CUDA;
  }
  const cudaError_t ei = cudaGraphInstantiate(&h.graph_exec[key], graph, cudaGraphInstantiateFlagUseNodePriority);
  cudaGraphDestroy(graph);
  if (ei != cudaSuccess) {
    h.graph_exec[key] = nullptr;
    cudaGetLastError();
    return FFXG_ERR_CUDA;
  }
  return FFXG_OK;
}

// Graph execution: one launch, one synchronisation.  Returns -1 when the evaluation must
// be repeated directly (list overflow, or the graph could not be built).
static int evaluate_graph(Handle &h, const double *d_xyz, double *d_grad_xyz, double *terms, int64_t *counts) {
  const int key = graph_key(h);
  if (!h.graph_exec[key] && capture_graph(h) != FFXG_OK) {
    h.use_graphs = false;   // fall back to direct launches for this handle
    return -1;
  }
  if (d_xyz != h.d_xyz_in)
    cudaMemcpyAsync(h.d_xyz_in, d_xyz, 3 * (size_t)h.n * sizeof(double), cudaMemcpyDeviceToDevice, h.stream);
  if (cudaGraphLaunch(h.graph_exec[key], h.stream) != cudaSuccess) {
    h.err = std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError());
    return FFXG_ERR_CUDA;
  }
  if (h.want_grad && d_grad_xyz != h.d_grad_out)
    cudaMemcpyAsync(d_grad_xyz, h.d_grad_out, 3 * (size_t)h.n * sizeof(double), cudaMemcpyDeviceToDevice, h.stream);
  if (key == 2) h.grad_pinned = true;   // the graph ends with the copy
  else copy_grad_to_pinned(h, d_grad_xyz);
  if (cudaStreamSynchronize(h.stream) != cudaSuccess) {
    h.err = std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError());
    return FFXG_ERR_CUDA;
  }
  return eval_after_graph(h, terms, counts);
}

namespace ffx {

// Results of a finished graph replay (the handle's own or a batch's) from the pinned copies.
// Returns -1 when a list overflowed: capacities grew, the handle's graphs are gone, and the
// evaluation must be repeated directly.
int eval_after_graph(Handle &h, double *terms, int64_t *counts) {
  const int key = graph_key(h);
  const int f = h.h_flags[0];
  if (f & kOverflow) {
    if (int a = grow_lists(h, f)) return a;   // also drops the graphs
    return -1;
  }
  if (f & FLAG_IMAGE_RANGE) { h.err = "atoms more than 500 box edges apart"; return FFXG_ERR_BAD_ARG; }
  if (f & FLAG_NONFINITE) {
    // k_reduce_coordinates raises the flag for non-finite input coordinates.
    h.err = "non-finite coordinates or energy";
    return FFXG_ERR_NONFINITE;
  }
  const bool rebuilt = (f & FLAG_REBUILD) != 0;
  if (rebuilt) h.list_builds++;
  h.scf_iter = 0;
  h.launches = h.graph_launches[key];
  if (h.prm.polarization == FFXG_POLAR_MUTUAL) {
    h.scf_iter = h.h_pcg->iter;
    h.launches += h.graph_body_launches * (int64_t)std::max(0, h.scf_iter - 1);
    if (h.h_pcg->status != FFXG_OK) { h.err = scf_message(h.h_pcg->status); return h.h_pcg->status; }
  }
  return finish(h, rebuilt, terms, counts);
}

}  // namespace ffx

// One evaluation on device-resident coordinates.  The graph path is used once the
// neighbour list exists (its first build and any regrowth run directly) and when stage
// timing is off.
// Electrostatic lambda (elec-lambdaterm, OST; ParticleMeshEwald.energy, PME:897-935) as
// direct launches: (1) every atom, softcore permanent real space, reciprocal and
// polarization scaled (condensedEnergy, :1609-1640); (2) without the soft atoms -- their
// multipoles and polarizabilities zeroed, which removes them exactly as use[] does --
// reciprocal permanent and polarization by the complements (condensedNoLigandSCF,
// :1650-1700); (3) the soft atoms alone in vacuum by the sub-system (ligandElec,
// :1704-1796).  The steps' results are summed before the torques become forces.
static int evaluate_elec(Handle &h, const double *d_xyz, double *d_grad_xyz, double *terms, int64_t *counts) {
  const ElecAlchemy &el = h.elec;
  const double L = h.lambda;
  const bool mutual = h.prm.polarization == FFXG_POLAR_MUTUAL;
  const bool anyPol = h.prm.polarization != FFXG_POLAR_NONE;
  h.want_grad = true;
  for (int attempt = 0; attempt < 4; attempt++) {
    h.ev_stage.clear();
    h.ev_used = 0;
    h.step = plain_step();
    h.step.lam = 1;
    h.step.permScale = el.lPowPerm;
    h.step.dEdLSign = 1.0;
    h.step.beta = el.lAlpha; h.step.dlAlpha = el.dlAlpha; h.step.d2lAlpha = el.d2lAlpha;
    h.step.dlPowPerm = el.dlPowPerm; h.step.d2lPowPerm = el.d2lPowPerm;
    h.step.dlPowPol = el.dlPowPol; h.step.d2lPowPol = el.d2lPowPol;
    if (L < el.polStart) { h.step.doPol = 0; h.step.polScale = 0.0; }
    else if (L <= el.polEnd) { h.step.doPol = 1; h.step.polScale = el.lPowPol; }
    else { h.step.doPol = 1; h.step.polScale = 1.0; }
    emit_front(h, d_xyz);
    cudaMemcpyAsync(h.h_flags, h.d_flags, sizeof(int), cudaMemcpyDeviceToHost, h.stream);
    if (cudaStreamSynchronize(h.stream) != cudaSuccess) {
      h.err = std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError());
      h.step = plain_step();
      return FFXG_ERR_CUDA;
    }
    const int f = h.h_flags[0];
    if (f & FLAG_NONFINITE) { h.err = "non-finite coordinates"; h.step = plain_step(); return FFXG_ERR_NONFINITE; }
    if (f & FLAG_IMAGE_RANGE) { h.err = "atoms more than 500 box edges apart"; h.step = plain_step(); return FFXG_ERR_BAD_ARG; }
    if (f & kOverflow) {
      if (int a = grow_lists(h, f)) { h.step = plain_step(); return a; }
      continue;
    }
    const bool rebuilt = (f & FLAG_REBUILD) != 0;
    if (rebuilt) h.list_builds++;
    h.list_valid = true;
    int st = FFXG_OK, iters = 0;
    // 1.
    if (anyPol && h.step.doPol) {
      if (mutual) st = run_pcg(h, false);
      iters += h.scf_iter;
      if (st == FFXG_OK) emit_final_induced(h);
    } else {
      emit_no_polarization(h);
    }
    if (st != FFXG_OK) { h.err = scf_message(st); h.step = plain_step(); return st; }
    launch_real_energy(h, true);
    launch_recip_energy(h, true);
    launch_elec_accumulate(h, true);
    // 2.
    bool any_env = false;
    for (int i = 0; i < h.n && !any_env; i++) any_env = !std::binary_search(h.lig.begin(), h.lig.end(), i);
    if (any_env) {
      h.step.doPermReal = 0;
      h.step.permScale = 1.0 - el.lPowPerm;
      h.step.dEdLSign = -1.0;
      h.step.beta = h.step.dlAlpha = h.step.d2lAlpha = 0.0;
      if (L <= el.polEnd && el.noLigandSCF) { h.step.doPol = 1; h.step.polScale = 1.0 - el.lPowPol; }
      else { h.step.doPol = 0; h.step.polScale = 0.0; }
      launch_zero_soft_multipoles(h);
      h.d_polar = h.d_polar_env;
      launch_spread_permanent(h);
      launch_fft_convolution(h);
      launch_phi_permanent(h);
      launch_realspace_field(h);
      launch_direct_dipoles(h);
      h.scf_iter = 0;
      if (anyPol && h.step.doPol) {
        if (mutual) st = run_pcg(h, false);
        iters += h.scf_iter;
        if (st == FFXG_OK) emit_final_induced(h);
      } else {
        emit_no_polarization(h);
      }
      if (st == FFXG_OK) {
        launch_real_energy(h, true);
        launch_recip_energy(h, true);
        launch_elec_accumulate(h, false);
      }
      h.d_polar = h.d_polar_all;
      if (st != FFXG_OK) { h.err = scf_message(st); h.step = plain_step(); return st; }
    }
    launch_elec_restore(h);
    // Torques to forces, vdW, the lambda gradient, sums (the reductions of emit_back).
    launch_torque(h);
    launch_assemble(h, d_grad_xyz);
    launch_lambda_grad_add(h, h.d_lgred + 3 * (size_t)h.n);
    launch_reduce_results(h);
    cudaMemcpyAsync(h.h_scalars, h.d_result, kEnergyRows * sizeof(double), cudaMemcpyDeviceToHost, h.stream);
    cudaMemcpyAsync(h.h_flags + 2, h.d_cresult, 2 * sizeof(long long), cudaMemcpyDeviceToHost, h.stream);
    cudaMemcpyAsync(h.h_flags, h.d_flags, sizeof(int), cudaMemcpyDeviceToHost, h.stream);
    if (cudaStreamSynchronize(h.stream) != cudaSuccess) {
      h.err = std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError());
      h.step = plain_step();
      return FFXG_ERR_CUDA;
    }
    h.scf_iter = iters;
    st = finish(h, rebuilt, terms, counts);
    if (st != FFXG_OK) { h.step = plain_step(); return st; }
    // 3.
    if (el.vaporElec && h.vac) {
      Handle &v = *h.vac;
      const int m = v.n;
      v.lambda = h.lambda;
      v.step = plain_step();
      v.step.lam = 1;
      v.step.permScale = 1.0 - el.lPowPerm;
      v.step.dEdLSign = -1.0;
      v.step.dlPowPerm = el.dlPowPerm; v.step.d2lPowPerm = el.d2lPowPerm;
      v.step.dlPowPol = el.dlPowPol; v.step.d2lPowPol = el.d2lPowPol;
      if (L <= el.polEnd) { v.step.doPol = 1; v.step.polScale = 1.0 - el.lPowPol; }
      else { v.step.doPol = 0; v.step.polScale = 0.0; }
      k_gather_xyz<<<nblocks(m, 128), 128, 0, h.stream>>>(m, h.d_lig, d_xyz, v.d_xyz_in);
      FFX_LAUNCHED(h);
      if (cudaStreamSynchronize(h.stream) != cudaSuccess) {
        h.err = std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError());
        h.step = plain_step();
        return FFXG_ERR_CUDA;
      }
      double vt[FFXG_N_TERMS];
      int64_t vc[FFXG_N_COUNTS];
      v.want_grad = true;
      st = evaluate_direct(v, v.d_xyz_in, v.d_grad_out, vt, vc);
      if (st != FFXG_OK) { h.err = "vacuum step: " + v.err; h.step = plain_step(); return st; }
      k_scatter_add_xyz<<<nblocks(m, 128), 128, 0, h.stream>>>(m, h.d_lig, v.d_grad_out, d_grad_xyz);
      k_scatter_add_soa<<<nblocks(m, 128), 128, 0, h.stream>>>(m, h.n, h.d_lig, v.d_lgred + 3 * (size_t)m,
                                                                h.d_lgred + 3 * (size_t)h.n);
      h.launches += 2;
      if (cudaStreamSynchronize(h.stream) != cudaSuccess) {
        h.err = std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError());
        h.step = plain_step();
        return FFXG_ERR_CUDA;
      }
      h.dEdL += v.dEdL;
      h.d2EdL2 += v.d2EdL2;
      h.scf_iter += v.scf_iter;
      if (terms) {
        terms[FFXG_TERM_PERM_REAL] += vt[FFXG_TERM_PERM_REAL];
        terms[FFXG_TERM_POL_REAL] += vt[FFXG_TERM_POL_REAL];
        terms[FFXG_TERM_PERMANENT] += vt[FFXG_TERM_PERMANENT];
        terms[FFXG_TERM_POLARIZATION] += vt[FFXG_TERM_POLARIZATION];
        terms[FFXG_TERM_TOTAL] += vt[FFXG_TERM_PERMANENT] + vt[FFXG_TERM_POLARIZATION];
      }
      if (counts) counts[FFXG_COUNT_SCF_ITER] = h.scf_iter;
    }
    h.lgrad_valid = true;
    h.step = plain_step();
    return FFXG_OK;
  }
  h.step = plain_step();
  h.err = "neighbour capacity could not be satisfied";
  return FFXG_ERR_CAPACITY;
}

static int evaluate_any(Handle &h, const double *d_xyz, double *d_grad_xyz, bool grad, double *terms,
                        int64_t *counts) {
  if (h.elec.on && h.alch.active && !h.vacuum) {
    h.launches = 0;
    return evaluate_elec(h, d_xyz, d_grad_xyz, terms, counts);
  }
  h.launches = 0;
  h.want_grad = grad;
  if (h.use_graphs && h.list_valid && !h.timing) {
    const int st = evaluate_graph(h, d_xyz, d_grad_xyz, terms, counts);
    if (st != -1) return st;
    h.launches = 0;
  }
  return evaluate_direct(h, d_xyz, d_grad_xyz, terms, counts);
}

namespace ffx {
// A launch that the runtime refuses (a bad configuration, too much shared memory) leaves
// no trace in the stream, only in the thread's last-error state: an evaluation that began
// with that state clear and ends with an error reports it instead of a partial result.
// An error the caller left pending is neither cleared nor taken for this call's.
int evaluate(Handle &h, const double *d_xyz, double *d_grad_xyz, bool grad, double *terms, int64_t *counts) {
  const bool clear = cudaPeekAtLastError() == cudaSuccess;
  const int st = evaluate_any(h, d_xyz, d_grad_xyz, grad, terms, counts);
  if (clear && cudaPeekAtLastError() != cudaSuccess) {
    h.err = std::string("CUDA launch error: ") + cudaGetErrorString(cudaGetLastError());
    return FFXG_ERR_CUDA;
  }
  return st;
}

Handle &handle_of(ffxg_handle *hh) { return hh->h; }
}  // namespace ffx

extern "C" {

int ffxg_create(const ffxg_system *sys, const ffxg_params *params, ffxg_handle **out) {
  if (!sys || !params || !out) { g_create_error = "null argument"; return FFXG_ERR_BAD_ARG; }
  *out = nullptr;
  ffxg_handle *hh = new ffxg_handle();
  const int st = create_impl(sys, params, hh->h);
  if (st != FFXG_OK) {
    g_create_error = hh->h.err;
    free_all(hh->h);
    delete hh;
    return st;
  }
  *out = hh;
  return FFXG_OK;
}

void ffxg_destroy(ffxg_handle *hh) {
  if (!hh) return;
  free_all(hh->h);
  delete hh;
}

const char *ffxg_last_error(const ffxg_handle *hh) { return hh ? hh->h.err.c_str() : g_create_error.c_str(); }

int ffxg_set_coordinates(ffxg_handle *hh, const double *xyz) {
  if (!hh || !xyz) return FFXG_ERR_BAD_ARG;
  Handle &h = hh->h;
  if (!copy_finite(h.h_xyz_pin, xyz, 3 * (size_t)h.n)) { h.err = "non-finite coordinates"; return FFXG_ERR_NONFINITE; }
  CK(cudaMemcpyAsync(h.d_xyz_in, h.h_xyz_pin, 3 * (size_t)h.n * sizeof(double), cudaMemcpyHostToDevice, h.stream));
  return FFXG_OK;
}

static int setup_elec(Handle &h, const std::vector<int> &soft, const std::vector<int> &mol);

// Crystal change (ForceFieldEnergy.setCrystal, ForceFieldEnergy.java:2650-2666, which passes
// it to VanDerWaals, ParticleMeshEwald.setCrystal :1262-1283 and ReciprocalSpace.setCrystal
// :750-761 / initConvolution :909-1000).
int ffxg_set_box(ffxg_handle *hh, const double box[3], const double angles[3], const int32_t pme_grid[3]) {
  if (!hh || !box) return FFXG_ERR_BAD_ARG;
  Handle &h = hh->h;
  if (h.vacuum) { h.err = "a vacuum sub-system has no cell"; return FFXG_ERR_BAD_ARG; }
  const double right[3] = {90.0, 90.0, 90.0};
  if (!angles) angles = right;
  if (!angles_ok(angles)) { h.err = "cell angles must lie in (0, 180) degrees"; return FFXG_ERR_BAD_ARG; }
  for (int d = 0; d < 3; d++) {
    if (!(box[d] > 0.0) || !std::isfinite(box[d])) { h.err = "box edges must be positive"; return FFXG_ERR_BAD_ARG; }
    if (pme_grid && !fft_supported(pme_grid[d])) {
      h.err = "PME grid dimensions must lie in [5, 4096]";
      return FFXG_ERR_BAD_ARG;
    }
  }
  CK(cudaStreamSynchronize(h.stream));   // nothing in flight reads the old tables
  const bool images_before = h.images, near_before = h.near_list;
  const Box keep_box = h.box;
  double keep_prm[6], keep_w[3];
  for (int d = 0; d < 3; d++) { keep_prm[d] = h.prm.box[d]; keep_prm[3 + d] = h.prm.angles[d]; keep_w[d] = h.width[d]; }
  set_cell(h, box, angles);
  if (!(h.box.volume > 0.0)) {
    h.box = keep_box;
    for (int d = 0; d < 3; d++) { h.prm.box[d] = keep_prm[d]; h.prm.angles[d] = keep_prm[3 + d]; h.width[d] = keep_w[d]; }
    h.err = "the cell angles give no volume";
    return FFXG_ERR_BAD_ARG;
  }
  configure_images(h);
  set_cell_grid(h);
  const int ncells = h.ncell[0] * h.ncell[1] * h.ncell[2];
  if (ncells > h.cell_cap) {
    cudaFree(h.d_cell_cnt);
    cudaFree(h.d_cell_start);
    h.d_cell_cnt = h.d_cell_start = nullptr;
    CK(dalloc(&h.d_cell_cnt, 2 * (size_t)ncells));
    CK(dalloc(&h.d_cell_start, (size_t)ncells + 1));
    h.cell_cap = ncells;
  }
  if (pme_grid && (pme_grid[0] != h.prm.pme_grid[0] || pme_grid[1] != h.prm.pme_grid[1] ||
                   pme_grid[2] != h.prm.pme_grid[2])) {
    for (int d = 0; d < 3; d++) h.prm.pme_grid[d] = pme_grid[d];
    if (int st = alloc_mesh(h)) return st;
  }
  if (int st = setup_pme(h)) return st;
  double q = 0.0, qenv = 0.0;
  for (int i = 0; i < h.n; i++) {
    const double qi = h.sys.multipole[10 * (size_t)i];
    q += qi;
    if (!h.soft_host.empty() && !h.soft_host[i]) qenv += qi;
  }
  h.e_charge_correction = charge_correction(h, q);
  if (h.elec.on) h.e_corr_env = charge_correction(h, qenv);
  if (h.images != images_before || h.near_list != near_before) {
    if (int st = alloc_lists(h)) return st;   // also drops the graphs and invalidates the list
  } else {
    drop_graphs(h);          // captured launches hold the cell and the PME transforms by value
    h.list_valid = false;    // the next evaluation rebuilds the list
  }
  CK(cudaGetLastError());
  return FFXG_OK;
}

// New parameter values for the same atoms and topology (OpenMMEnergy.updateParameters,
// OpenMMEnergy.java:623-631, over ForceFieldEnergy's parameter arrays): local multipoles,
// polarizabilities, Thole and damping, hydrogen reduction factors and the vdW pair tables.
// Uploaded in place: no allocation and no new capture while the sizes stay the same.
int ffxg_update_parameters(ffxg_handle *hh, const ffxg_system *s) {
  if (!hh || !s) return FFXG_ERR_BAD_ARG;
  Handle &h = hh->h;
  const int n = h.n;
  if (s->n_atoms != n || s->n_vdw_types != h.ntypes) {
    h.err = "update_parameters: the atom and vdW type counts must not change";
    return FFXG_ERR_BAD_ARG;
  }
  if (!s->multipole || !s->polarizability || !s->thole || !s->pdamp || !s->red_factor || !s->vdw_inv_rmin ||
      !s->vdw_eps) {
    h.err = "update_parameters: null parameter array";
    return FFXG_ERR_BAD_ARG;
  }
  for (int i = 0; i < n; i++) {
    const double *m = s->multipole + 10 * (size_t)i;
    bool ok = std::isfinite(s->polarizability[i]) && s->polarizability[i] >= 0.0 && std::isfinite(s->thole[i]) &&
              std::isfinite(s->pdamp[i]) && std::isfinite(s->red_factor[i]);
    for (int t = 0; t < 10; t++) ok = ok && std::isfinite(m[t]);
    if (!ok) { h.err = "update_parameters: non-finite or negative parameter"; return FFXG_ERR_BAD_ARG; }
  }
  CK(cudaStreamSynchronize(h.stream));
  const size_t N = n;
  SystemCopy &c = h.sys;
  c.multipole.assign(s->multipole, s->multipole + 10 * N);
  c.polarizability.assign(s->polarizability, s->polarizability + N);
  c.thole.assign(s->thole, s->thole + N);
  c.pdamp.assign(s->pdamp, s->pdamp + N);
  c.red_factor.assign(s->red_factor, s->red_factor + N);
  const size_t t2 = (size_t)h.ntypes * h.ntypes;
  c.vdw_inv_rmin.assign(s->vdw_inv_rmin, s->vdw_inv_rmin + t2);
  c.vdw_eps.assign(s->vdw_eps, s->vdw_eps + t2);
  std::vector<double> lmp(10 * N), ipd(N);
  for (size_t i = 0; i < N; i++) {
    for (int t = 0; t < 10; t++) lmp[t * N + i] = s->multipole[10 * i + t];
    ipd[i] = (s->pdamp[i] > 0.0) ? 1.0 / s->pdamp[i] : INFINITY;   // ParticleMeshEwald.java:1401-1406
  }
  // With electrostatic lambda on, d_polar_all holds the full set and d_polar_env the set
  // without the soft atoms.
  double *d_pol = h.d_polar_all ? h.d_polar_all : h.d_polar;
  CK(cudaMemcpy(h.d_lmp, lmp.data(), 10 * N * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_pol, s->polarizability, N * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_thole, s->thole, N * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_ipdamp, ipd.data(), N * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_redf, s->red_factor, N * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_vrad, s->vdw_inv_rmin, t2 * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_veps, s->vdw_eps, t2 * sizeof(double), cudaMemcpyHostToDevice));
  double q = 0.0;
  for (size_t i = 0; i < N; i++) q += s->multipole[10 * i];
  h.e_charge_correction = charge_correction(h, q);
  if (h.elec.on && h.alch.active) {
    // The soft-free polarizabilities, the soft-free charge correction and the vacuum
    // sub-system follow the new values.
    if (int st = setup_elec(h, h.soft_host, h.mol_host)) return st;
  }
  return FFXG_OK;
}

int ffxg_energy(ffxg_handle *hh, int want_grad, double *terms, double *grad, int64_t *counts) {
  if (!hh) return FFXG_ERR_BAD_ARG;
  Handle &h = hh->h;
  h.grad_to_pin = want_grad && grad;
  h.grad_pinned = false;
  h.growths = 0;
  const int st = evaluate(h, h.d_xyz_in, h.d_grad_out, want_grad != 0, terms, counts);
  h.grad_to_pin = false;
  if (st != FFXG_OK && st != FFXG_ERR_RANGE) return st;   // RANGE: every output is complete
  if (want_grad && grad) {
    if (!h.grad_pinned) {   // paths that synchronise more than once copy afterwards
      CK(cudaMemcpyAsync(h.h_grad_pin, h.d_grad_out, 3 * (size_t)h.n * sizeof(double), cudaMemcpyDeviceToHost,
                         h.stream));
      CK(cudaStreamSynchronize(h.stream));
    }
    std::memcpy(grad, h.h_grad_pin, 3 * (size_t)h.n * sizeof(double));
  }
  return st;
}

int ffxg_energy_and_gradient(ffxg_handle *hh, const double *xyz, double *terms, double *grad, int64_t *counts) {
  if (const int st = ffxg_set_coordinates(hh, xyz)) return st;
  return ffxg_energy(hh, grad != nullptr, terms, grad, counts);
}

int ffxg_energy_device(ffxg_handle *hh, const double *d_xyz, double *d_grad, double *terms, int64_t *counts) {
  if (!hh || !d_xyz) return FFXG_ERR_BAD_ARG;
  Handle &h = hh->h;
  h.growths = 0;
  return evaluate(h, d_xyz, d_grad ? d_grad : h.d_grad_out, d_grad != nullptr, terms, counts);
}

int ffxg_get_induced_dipoles(ffxg_handle *hh, double *u, double *u_cr) {
  if (!hh) return FFXG_ERR_BAD_ARG;
  Handle &h = hh->h;
  const size_t N = h.n;
  std::vector<double> a(3 * N), b(3 * N);
  CK(cudaMemcpy(a.data(), h.d_uD, 3 * N * sizeof(double), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(b.data(), h.d_uP, 3 * N * sizeof(double), cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < N; i++)
    for (int d = 0; d < 3; d++) {
      if (u) u[3 * i + d] = a[d * N + i];
      if (u_cr) u_cr[3 * i + d] = b[d * N + i];
    }
  return FFXG_OK;
}

int ffxg_get_permanent_potential(ffxg_handle *hh, double *phi) {
  if (!hh || !phi) return FFXG_ERR_BAD_ARG;
  Handle &h = hh->h;
  if (!h.list_valid) { h.err = "no evaluation yet: call ffxg_energy first"; return FFXG_ERR_BAD_ARG; }
  const size_t N = h.n;
  std::vector<double> a(20 * N);
  CK(cudaMemcpy(a.data(), h.d_cphi, 20 * N * sizeof(double), cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < N; i++)
    for (int t = 0; t < 20; t++) phi[20 * i + t] = a[t * N + i];
  return FFXG_OK;
}

int ffxg_get_global_multipoles(ffxg_handle *hh, double *mpole) {
  if (!hh || !mpole) return FFXG_ERR_BAD_ARG;
  Handle &h = hh->h;
  const size_t N = h.n;
  std::vector<double> a(10 * N);
  CK(cudaMemcpy(a.data(), h.d_gm, 10 * N * sizeof(double), cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < N; i++)
    for (int t = 0; t < 10; t++) mpole[10 * i + t] = a[t * N + i];
  return FFXG_OK;
}

// Image pairs of the buffered list, each once: rows (i, k, nx, ny, nz) with k > i, or
// k == i and n > 0 in (z, y, x) lexicographic order; n = 0 outside multi-image mode.
static int list_images(Handle &h, int32_t *rows, int stride, int64_t *n_rows) {
  if (!h.list_valid) { h.err = "no neighbour list yet: call ffxg_energy first"; return FFXG_ERR_BAD_ARG; }
  const size_t N = h.n;
  std::vector<int> cnt(N), lst(N * h.cap_nbr), sh;
  CK(cudaMemcpy(cnt.data(), h.d_nbr_cnt, N * sizeof(int), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(lst.data(), h.d_nbr, N * h.cap_nbr * sizeof(int), cudaMemcpyDeviceToHost));
  if (h.images) {
    sh.resize(N * h.cap_nbr);
    CK(cudaMemcpy(sh.data(), h.d_nbr_sh, N * h.cap_nbr * sizeof(int), cudaMemcpyDeviceToHost));
  }
  int64_t c = 0;
  for (size_t i = 0; i < N; i++)
    for (int a = 0; a < std::min(cnt[i], h.cap_nbr); a++) {
      const size_t e = i * h.cap_nbr + a;
      const int k = lst[e];
      int n3[3] = {0, 0, 0};
      if (h.images) {
        n3[0] = (sh[e] & 1023) - 512; n3[1] = ((sh[e] >> 10) & 1023) - 512; n3[2] = ((sh[e] >> 20) & 1023) - 512;
      }
      const bool pos = n3[2] > 0 || (n3[2] == 0 && (n3[1] > 0 || (n3[1] == 0 && n3[0] > 0)));
      if (k > (int)i || (k == (int)i && pos)) {
        if (rows) {
          int32_t *q = rows + stride * c;
          q[0] = (int32_t)i; q[1] = k;
          if (stride == 5) { q[2] = n3[0]; q[3] = n3[1]; q[4] = n3[2]; }
        }
        c++;
      }
    }
  *n_rows = c;
  return FFXG_OK;
}

int ffxg_get_neighbor_pairs(ffxg_handle *hh, int32_t *pairs, int64_t *n_pairs) {
  if (!hh || !n_pairs) return FFXG_ERR_BAD_ARG;
  return list_images(hh->h, pairs, 2, n_pairs);
}

int ffxg_get_neighbor_images(ffxg_handle *hh, int32_t *rows, int64_t *n_rows) {
  if (!hh || !n_rows) return FFXG_ERR_BAD_ARG;
  return list_images(hh->h, rows, 5, n_rows);
}

int ffxg_param_grad(ffxg_handle *hh, double *dEdM, double *dEdalpha) {
  if (!hh || !dEdM || !dEdalpha) return FFXG_ERR_BAD_ARG;
  Handle &h = hh->h;
  if (!h.list_valid) { h.err = "no evaluation yet: call ffxg_energy first"; return FFXG_ERR_BAD_ARG; }
  if (h.elec.on && h.alch.active) { h.err = "parameter gradients are not defined under electrostatic lambda"; return FFXG_ERR_BAD_ARG; }
  const size_t N = h.n;
  double *d = nullptr;
  CK(cudaMalloc(&d, 11 * N * sizeof(double)));
  int st = param_gradients(h, d, d + 10 * N);
  if (st == FFXG_OK) {
    std::vector<double> a(11 * N);
    if (cudaMemcpyAsync(a.data(), d, 11 * N * sizeof(double), cudaMemcpyDeviceToHost, h.stream) != cudaSuccess ||
        cudaStreamSynchronize(h.stream) != cudaSuccess) {
      st = FFXG_ERR_CUDA;
    } else {
      std::memcpy(dEdM, a.data(), 10 * N * sizeof(double));
      std::memcpy(dEdalpha, a.data() + 10 * N, N * sizeof(double));
    }
  }
  cudaFree(d);
  if (st != FFXG_OK) h.err = std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError());
  return st;
}

int ffxg_set_image_mode(ffxg_handle *hh, int mode) {
  if (!hh) return FFXG_ERR_BAD_ARG;
  Handle &h = hh->h;
  if (mode != FFXG_IMAGES_AUTO && mode != FFXG_IMAGES_ALL) { h.err = "unknown image mode"; return FFXG_ERR_BAD_ARG; }
  h.image_mode = mode;
  configure_images(h);
  return alloc_lists(h);
}

// VanDerWaals.setLambda (VanDerWaals.java:599-628): softcore constants at lambda.
static void update_alchemy(Handle &h) {
  double l = h.lambda;
  if (l > h.alch_end) l = 1.0; else l = l / h.alch_end;
  const double a = h.alch_alpha, ex = h.alch_exponent;
  h.alch.sc1 = a * (1.0 - l) * (1.0 - l);
  h.alch.dsc1dL = -2.0 * a * (1.0 - l);
  h.alch.d2sc1dL2 = 2.0 * a;
  h.alch.sc2 = std::pow(l, ex);
  h.alch.dsc2dL = ex * std::pow(l, ex - 1.0);
  h.alch.d2sc2dL2 = (ex >= 2.0) ? ex * (ex - 1.0) * std::pow(l, ex - 2.0) : 0.0;
  // Electrostatics: AlchemicalParameters.update (pme/AlchemicalParameters.java:306-380).
  ElecAlchemy &el = h.elec;
  const double L = h.lambda;
  el.lPowPerm = 1.0; el.dlPowPerm = 0.0; el.d2lPowPerm = 0.0;
  el.lAlpha = 0.0; el.dlAlpha = 0.0; el.d2lAlpha = 0.0;
  if (L < el.permStart) {
    el.lPowPerm = 0.0;
  } else if (L <= el.permEnd) {
    const double sc = 1.0 / (el.permEnd - el.permStart);
    const double pl = sc * (L - el.permStart);
    el.lAlpha = el.permAlpha * (1.0 - pl) * (1.0 - pl);
    el.dlAlpha = el.permAlpha * (1.0 - pl) * sc;
    el.d2lAlpha = -el.permAlpha * sc * sc;
    el.lPowPerm = std::pow(pl, el.permExp);
    el.dlPowPerm = el.permExp * std::pow(pl, el.permExp - 1.0) * sc;
    el.d2lPowPerm = (el.permExp >= 2.0) ? el.permExp * (el.permExp - 1.0) * std::pow(pl, el.permExp - 2.0) * sc * sc : 0.0;
  }
  el.lPowPol = 1.0; el.dlPowPol = 0.0; el.d2lPowPol = 0.0;
  if (L < el.polStart) {
    el.lPowPol = 0.0;
  } else if (L <= el.polEnd) {
    const double sc = 1.0 / (el.polEnd - el.polStart);
    const double pl = sc * (L - el.polStart);
    if (el.polExp > 0.0) {
      el.lPowPol = std::pow(pl, el.polExp);
      if (el.polExp >= 1.0) {
        el.dlPowPol = el.polExp * std::pow(pl, el.polExp - 1.0);
        if (el.polExp >= 2.0) el.d2lPowPol = el.polExp * (el.polExp - 1.0) * std::pow(pl, el.polExp - 2.0);
      }
    }
    el.dlPowPol *= sc;
    el.d2lPowPol *= sc * sc;
  }
  drop_graphs(h);   // the captured vdW launch holds the constants
}

// ---------------------------------------------------------------------------
// Vacuum sub-system of the soft atoms (ligandElec, PME:1704-1796): their multipoles,
// polarizabilities, frames and masks, an all-pairs list without images, Ewald alpha 0
// and no reciprocal space.
static int build_vacuum(Handle &h, const std::vector<int> &soft, const std::vector<int> &mol) {
  drop_vacuum(h);
  const SystemCopy &c = h.sys;
  std::vector<int> map(h.n, -1);
  h.lig.clear();
  for (int i = 0; i < h.n; i++)
    if (soft[i]) { map[i] = (int)h.lig.size(); h.lig.push_back(i); }
  const int m = (int)h.lig.size();
  if (m == 0) return FFXG_OK;
  std::vector<double> xyz(3 * (size_t)m), mp(10 * (size_t)m), pol(m), th(m), pd(m), rf(m);
  std::vector<int> fr(m), ax(3 * (size_t)m, -1), vt(m), rp(m), vmol(m);
  for (int j = 0; j < m; j++) {
    const int i = h.lig[j];
    for (int d = 0; d < 3; d++) xyz[3 * j + d] = c.xyz[3 * (size_t)i + d];
    for (int t = 0; t < 10; t++) mp[10 * j + t] = c.multipole[10 * (size_t)i + t];
    pol[j] = c.polarizability[i]; th[j] = c.thole[i]; pd[j] = c.pdamp[i];
    fr[j] = c.frame[i];
    for (int a = 0; a < 3; a++) {
      const int k = c.axis[3 * (size_t)i + a];
      if (k >= 0 && map[k] < 0) { h.err = "a frame-defining atom of a soft atom is not soft"; return FFXG_ERR_BAD_ARG; }
      ax[3 * j + a] = k >= 0 ? map[k] : -1;
    }
    vt[j] = c.vdw_type[i];
    rp[j] = map[c.red_parent[i]] >= 0 ? map[c.red_parent[i]] : j;
    rf[j] = map[c.red_parent[i]] >= 0 ? c.red_factor[i] : 0.0;
    vmol[j] = mol[i];
  }
  auto sub_csr = [&](const std::vector<std::vector<int>> &L, std::vector<int> &ptr, std::vector<int> &idx) {
    ptr.assign(m + 1, 0);
    idx.clear();
    for (int j = 0; j < m; j++) {
      for (int k : L[h.lig[j]])
        if (map[k] >= 0) idx.push_back(map[k]);
      ptr[j + 1] = (int)idx.size();
    }
  };
  std::vector<int> p12, i12, p13, i13, p14, i14, p15, i15, p11, i11;
  sub_csr(c.m12, p12, i12); sub_csr(c.m13, p13, i13); sub_csr(c.m14, p14, i14); sub_csr(c.m15, p15, i15);
  sub_csr(c.ip11, p11, i11);
  ffxg_system sub{};
  sub.n_atoms = m; sub.xyz = xyz.data(); sub.multipole = mp.data(); sub.frame = fr.data(); sub.axis = ax.data();
  sub.polarizability = pol.data(); sub.thole = th.data(); sub.pdamp = pd.data(); sub.vdw_type = vt.data();
  sub.red_parent = rp.data(); sub.red_factor = rf.data(); sub.n_vdw_types = c.n_vdw_types;
  sub.vdw_inv_rmin = c.vdw_inv_rmin.data(); sub.vdw_eps = c.vdw_eps.data();
  sub.mask12_ptr = p12.data(); sub.mask12_idx = i12.data(); sub.mask13_ptr = p13.data(); sub.mask13_idx = i13.data();
  sub.mask14_ptr = p14.data(); sub.mask14_idx = i14.data(); sub.mask15_ptr = p15.data(); sub.mask15_idx = i15.data();
  sub.ip11_ptr = p11.data(); sub.ip11_idx = i11.data();
  ffxg_params prm = h.prm;
  prm.pme_grid[0] = prm.pme_grid[1] = prm.pme_grid[2] = 8;   // unused: no reciprocal space
  Handle *v = new Handle();
  int st = create_impl(&sub, &prm, *v);
  if (st != FFXG_OK) { h.err = "vacuum sub-system: " + v->err; free_all(*v); delete v; return st; }
  v->vacuum = true;
  v->near_list = false;
  v->use_graphs = false;
  v->eps_atoms = h.n;
  v->images = true;
  v->cap_nbr = v->cap_ewl = v->cap_prl = round32(m);
  Handle &vh = *v;
  auto fail = [&](int code) { h.err = "vacuum sub-system: " + vh.err; free_all(vh); delete v; return code; };
  if ((st = alloc_lists(vh)) != FFXG_OK) return fail(st);
  const size_t M = m;
  std::vector<int> ones(M, 1);
#define VK(call) do { if ((call) != cudaSuccess) { vh.err = #call; return fail(FFXG_ERR_CUDA); } } while (0)
  VK(dalloc(&vh.d_soft, M)); VK(dalloc(&vh.d_mol, M)); VK(dalloc(&vh.d_lgred, 6 * M));
  VK(dalloc(&vh.d_lg, 3 * M)); VK(dalloc(&vh.d_lt, 3 * M));
  VK(cudaMemcpy(vh.d_soft, ones.data(), M * sizeof(int), cudaMemcpyHostToDevice));
  VK(cudaMemcpy(vh.d_mol, vmol.data(), M * sizeof(int), cudaMemcpyHostToDevice));
  VK(cudaMemset(vh.d_lgred, 0, 6 * M * sizeof(double)));
  // No reciprocal space or vdW: the mesh, potentials, their energy rows and the vdW
  // gradient stay zero.
  const size_t ng = (size_t)vh.nfft[0] * vh.nfft[1] * vh.nfft[2];
  VK(cudaMemset(vh.d_grid, 0, ng * sizeof(double2)));
  if (vh.d_gridf) VK(cudaMemset(vh.d_gridf, 0, ng * sizeof(float2)));
  for (double *q : {vh.d_cphi, vh.d_fphi, vh.d_cphiI, vh.d_fphiI, vh.d_cphiP, vh.d_fphiP})
    VK(cudaMemset(q, 0, 20 * M * sizeof(double)));
  VK(cudaMemset(vh.d_eatom, 0, (size_t)kEnergyRows * M * sizeof(double)));
  VK(cudaMemset(vh.d_gred, 0, 6 * M * sizeof(double)));
#undef VK
  vh.alch = h.alch;
  vh.alch.active = 0;   // the vdW softcore stays with the full system
  CK(dalloc(&h.d_lig, M));
  CK(cudaMemcpy(h.d_lig, h.lig.data(), M * sizeof(int), cudaMemcpyHostToDevice));
  h.vac = v;
  return FFXG_OK;
}

// Electrostatic lambda state: lambda arrays, step accumulators, the polarizabilities
// without the soft atoms, the charge correction without them, the vacuum sub-system.
static int setup_elec(Handle &h, const std::vector<int> &soft, const std::vector<int> &mol) {
  const size_t N = h.n;
  if (!h.d_lg) {
    CK(dalloc(&h.d_lg, 3 * N)); CK(dalloc(&h.d_lt, 3 * N));
    CK(dalloc(&h.d_acc, 20 * N)); CK(dalloc(&h.d_polar_env, N));
    h.d_polar_all = h.d_polar;
  }
  std::vector<double> pe(N);
  double q = 0.0;
  for (size_t i = 0; i < N; i++) {
    pe[i] = soft[i] ? 0.0 : h.sys.polarizability[i];
    if (!soft[i]) q += h.sys.multipole[10 * i];
  }
  CK(cudaMemcpy(h.d_polar_env, pe.data(), N * sizeof(double), cudaMemcpyHostToDevice));
  // ReciprocalEnergyRegion.java:228-238 for the atoms in use.
  h.e_corr_env = charge_correction(h, q);
  return build_vacuum(h, soft, mol);
}

int ffxg_set_alchemy(ffxg_handle *hh, const ffxg_alchemy *a) {
  if (!hh) return FFXG_ERR_BAD_ARG;
  Handle &h = hh->h;
  if (!a) {
    h.alch.active = 0;
    h.elec.on = false;
    drop_vacuum(h);
    CK(cudaMemset(h.d_eatom + 9 * (size_t)h.n, 0, 2 * (size_t)h.n * sizeof(double)));
    update_alchemy(h);
    return FFXG_OK;
  }
  if (a->elec && (!(a->permanent_lambda_alpha >= 0.0) || !(a->permanent_lambda_exponent >= 0.0) ||
                  !(a->permanent_lambda_start >= 0.0 && a->permanent_lambda_start <= 1.0) ||
                  !(a->permanent_lambda_end >= a->permanent_lambda_start && a->permanent_lambda_end <= 1.0) ||
                  !(a->polarization_lambda_start >= 0.0 && a->polarization_lambda_start <= 1.0) ||
                  !(a->polarization_lambda_end >= a->polarization_lambda_start &&
                    a->polarization_lambda_end <= 1.0) ||
                  !(a->polarization_lambda_exponent >= 0.0))) {
    h.err = "alchemy: electrostatic lambda windows must lie in [0, 1] with start <= end; alpha, exponents >= 0";
    return FFXG_ERR_BAD_ARG;
  }
  if (!a->soft || !(a->vdw_lambda_alpha >= 0.0) || !(a->vdw_lambda_exponent >= 1.0) ||
      !(a->vdw_lambda_end > 0.0 && a->vdw_lambda_end <= 1.0)) {
    h.err = "alchemy: soft flags required, vdw-lambda-alpha >= 0, vdw-lambda-exponent >= 1, 0 < vdw-lambda-end <= 1";
    return FFXG_ERR_BAD_ARG;
  }
  const size_t N = h.n;
  if (!h.d_soft) {
    CK(dalloc(&h.d_soft, N));
    CK(dalloc(&h.d_mol, N));
    CK(dalloc(&h.d_lgred, 6 * N));
  }
  std::vector<int> soft(N), mol(N);
  for (size_t i = 0; i < N; i++) {
    soft[i] = a->soft[i] != 0;
    mol[i] = a->molecule ? a->molecule[i] : (int)i;
  }
  h.soft_host = soft;
  h.mol_host = mol;
  CK(cudaMemcpy(h.d_soft, soft.data(), N * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h.d_mol, mol.data(), N * sizeof(int), cudaMemcpyHostToDevice));
  h.alch_alpha = a->vdw_lambda_alpha;
  h.alch_exponent = a->vdw_lambda_exponent;
  h.alch_end = a->vdw_lambda_end;
  h.alch.inter = a->intermolecular_softcore != 0;
  h.alch.intra = a->intramolecular_softcore != 0;
  h.alch.active = 1;
  ElecAlchemy &el = h.elec;
  el.on = a->elec != 0;
  if (el.on) {
    el.permAlpha = a->permanent_lambda_alpha; el.permExp = a->permanent_lambda_exponent;
    el.permStart = a->permanent_lambda_start; el.permEnd = a->permanent_lambda_end;
    el.polStart = a->polarization_lambda_start; el.polEnd = a->polarization_lambda_end;
    el.polExp = a->polarization_lambda_exponent;
    el.vaporElec = a->ligand_vapor_elec != 0;
    el.noLigandSCF = a->no_ligand_condensed_scf != 0;
    if (int st = setup_elec(h, soft, mol)) { el.on = false; return st; }
  } else {
    drop_vacuum(h);
    CK(cudaMemset(h.d_eatom + 9 * (size_t)h.n, 0, 2 * (size_t)h.n * sizeof(double)));
  }
  update_alchemy(h);
  return FFXG_OK;
}

int ffxg_set_lambda(ffxg_handle *hh, double lambda) {
  if (!hh) return FFXG_ERR_BAD_ARG;
  Handle &h = hh->h;
  if (!(lambda >= 0.0 && lambda <= 1.0)) { h.err = "lambda must lie in [0, 1]"; return FFXG_ERR_BAD_ARG; }
  h.lambda = lambda;
  update_alchemy(h);
  return FFXG_OK;
}

int ffxg_get_dEdL(ffxg_handle *hh, double *dEdL, double *d2EdL2, double *dEdXdL) {
  if (!hh) return FFXG_ERR_BAD_ARG;
  Handle &h = hh->h;
  if (dEdL) *dEdL = h.alch.active ? h.dEdL : 0.0;
  if (d2EdL2) *d2EdL2 = h.alch.active ? h.d2EdL2 : 0.0;
  if (dEdXdL) {
    const size_t N = h.n;
    if (!h.lgrad_valid) {
      std::memset(dEdXdL, 0, 3 * N * sizeof(double));
      return FFXG_OK;
    }
    std::vector<double> a(3 * N);
    CK(cudaMemcpy(a.data(), h.d_lgred + 3 * N, 3 * N * sizeof(double), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < N; i++)
      for (int d = 0; d < 3; d++) dEdXdL[3 * i + d] = a[d * N + i];
  }
  return FFXG_OK;
}

int ffxg_set_scf_predictor(ffxg_handle *hh, int predictor) {
  if (!hh) return FFXG_ERR_BAD_ARG;
  Handle &h = hh->h;
  if (predictor != FFXG_PREDICTOR_NONE && predictor != FFXG_PREDICTOR_ASPC) {
    h.err = "unknown SCF predictor";
    return FFXG_ERR_BAD_ARG;
  }
  if (predictor == FFXG_PREDICTOR_ASPC && !h.d_aspc) {
    CK(dalloc(&h.d_aspc, 36 * (size_t)h.n));
    CK(dalloc(&h.d_aspc_state, 2));
  }
  if (h.d_aspc_state) CK(cudaMemset(h.d_aspc_state, 0, 2 * sizeof(int)));
  h.scf_predictor = predictor;
  drop_graphs(h);
  return FFXG_OK;
}

static int md_force(Handle &h, const double *d_xyz, double *d_grad, double *terms) {
  h.growths = 0;
  return evaluate(h, d_xyz, d_grad, true, terms, nullptr);
}

int ffxg_md_setup(ffxg_handle *hh, const ffxg_md *md) {
  if (!hh) return FFXG_ERR_BAD_ARG;
  return md_setup(hh->h, md);
}

int ffxg_md_run(ffxg_handle *hh, double dt, int32_t n_steps, double *xyz, double *vel, double *epot, double *ekin) {
  if (!hh) return FFXG_ERR_BAD_ARG;
  return md_run(hh->h, dt, n_steps, xyz, vel, epot, ekin, md_force);
}

void *ffxg_stream(ffxg_handle *hh) { return hh ? (void *)hh->h.stream : nullptr; }

int64_t ffxg_list_builds(const ffxg_handle *hh) { return hh ? hh->h.list_builds : -1; }

int64_t ffxg_last_launch_count(const ffxg_handle *hh) { return hh ? hh->h.launches : 0; }

int ffxg_set_graph_mode(ffxg_handle *hh, int on) {
  if (!hh) return FFXG_ERR_BAD_ARG;
  Handle &h = hh->h;
  h.use_graphs = on != 0;
  if (!h.use_graphs) drop_graphs(h);
  return FFXG_OK;
}

int ffxg_set_timing(ffxg_handle *hh, int on) {
  if (!hh) return FFXG_ERR_BAD_ARG;
  Handle &h = hh->h;
  h.timing = on != 0;
  for (int s = 0; s < 16; s++) { h.stage_ms[s] = 0.0; h.stage_calls[s] = 0; }
  h.ev_stage.clear();
  h.ev_used = 0;
  return FFXG_OK;
}

int ffxg_get_timings(ffxg_handle *hh, double *ms, int64_t *launches, int n) {
  if (!hh || n < 0) return FFXG_ERR_BAD_ARG;
  Handle &h = hh->h;
  for (int s = 0; s < n && s < FFXG_N_STAGES; s++) {
    if (ms) ms[s] = h.stage_ms[s];
    if (launches) launches[s] = h.stage_calls[s];
  }
  return FFXG_OK;
}

}  // extern "C"
