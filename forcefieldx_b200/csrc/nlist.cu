// nlist.cu -- coordinates, hydrogen reduction, cell list and Verlet lists.
//
// Replaces NeighborList.buildList/run (NeighborList.java:351-572): the buffered
// list at max(vdw, ewald) cutoff + buffer on the hydrogen-reduced coordinates of
// VanDerWaals.ExpandLoop (VanDerWaals.java:1505-1541), rebuilt only when an atom
// moved more than half the buffer (MotionLoop, NeighborList.java:777-799).  The
// pair test is Crystal.image's exact arithmetic (d2 <= (cutoff+buffer)^2), so the
// pair set is the reference's.  The list is stored in both directions so every
// pair kernel gathers into its own atom without atomics.
#include "ffx_internal.cuh"

namespace ffx {

struct CellOffsets {
  int n[3];
  int off[3][5];
};

// Interleaved [n][3] -> SoA, plus reduced coordinates r = a*(x - x_p) + x_p evaluated
// without contraction like Java (VanDerWaals.java:1521-1527).
__device__ __forceinline__ void k_set_coordinates(VGrid vg, int n, const double *__restrict__ xyz, const int *__restrict__ redp,
                                  const double *__restrict__ redf, double *x, double *y, double *z,
                                  double *rx, double *ry, double *rz, double2 *pos) {
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double a = xyz[3 * i], b = xyz[3 * i + 1], c = xyz[3 * i + 2];
  x[i] = a;
  y[i] = b;
  z[i] = c;
  pos[2 * i] = make_double2(a, b);
  pos[2 * i + 1] = make_double2(c, 0.0);
}

__device__ __forceinline__ void k_reduce_coordinates(VGrid vg, int n, const double *__restrict__ x, const double *__restrict__ y,
                                     const double *__restrict__ z, const int *__restrict__ redp,
                                     const double *__restrict__ redf, double *rx, double *ry, double *rz,
                                     const double *__restrict__ refx, const double *__restrict__ refy,
                                     const double *__restrict__ refz, double half_buffer2, int *flags,
                                     const int *__restrict__ vtype, double2 *rpos) {
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = redp[i];
  const double a = redf[i];
  const double xi = x[i], yi = y[i], zi = z[i];
  double vx = xi, vy = yi, vz = zi;
  if (p != i || a != 0.0) {
    const double px = x[p], py = y[p], pz = z[p];
    vx = __dadd_rn(__dmul_rn(a, __dsub_rn(xi, px)), px);
    vy = __dadd_rn(__dmul_rn(a, __dsub_rn(yi, py)), py);
    vz = __dadd_rn(__dmul_rn(a, __dsub_rn(zi, pz)), pz);
  }
  rx[i] = vx; ry[i] = vy; rz[i] = vz;
  rpos[2 * i] = make_double2(vx, vy);
  rpos[2 * i + 1] = make_double2(vz, __longlong_as_double((long long)vtype[i]));
  const double dx = vx - refx[i], dy = vy - refy[i], dz = vz - refz[i];
  const double d2 = dx * dx + dy * dy + dz * dz;
  if (!(d2 <= half_buffer2)) atomicOr(flags, FLAG_REBUILD);
  const double ox = xi - vx, oy = yi - vy, oz = zi - vz;
  if (!(ox * ox + oy * oy + oz * oz <= kNearDelta * kNearDelta)) atomicOr(flags, FLAG_NEAR_INVALID);
  if (!isfinite(vx) || !isfinite(vy) || !isfinite(vz)) atomicOr(flags, FLAG_NONFINITE);
}

// Cell index along one axis of a fractional coordinate f (wrapped into [0, 1)).
__device__ __forceinline__ int cell_of(double f, int nc) {
  f = f - floor(f);
  int c = (int)(f * nc);
  return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
}

__device__ __forceinline__ void k_cell_count(VGrid vg, int n, const double *__restrict__ rx, const double *__restrict__ ry,
                             const double *__restrict__ rz, const Box &bx, int ncx, int ncy, int ncz,
                             int *cell_cnt, int *atom_cell, const int *flags) {
  if (!(*flags & FLAG_REBUILD)) return;
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double fx, fy, fz;
  to_frac(rx[i], ry[i], rz[i], bx, fx, fy, fz);
  const int cx = cell_of(fx, ncx), cy = cell_of(fy, ncy), cz = cell_of(fz, ncz);
  const int c = (cz * ncy + cy) * ncx + cx;
  atom_cell[i] = c;
  atomicAdd(&cell_cnt[c], 1);
}

// Exclusive scan of the cell counts in one CTA (cells <= a few 1e5).
__device__ __forceinline__ void k_cell_scan(VGrid vg, int ncells, const int *__restrict__ cnt, int *start, const int *flags) {
  if (!(*flags & FLAG_REBUILD)) return;
  __shared__ int warp_tot[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < ncells; base += blockDim.x) {
    const int idx = base + threadIdx.x;
    const int v = idx < ncells ? cnt[idx] : 0;
    int incl = v;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      int w = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += t;
      }
      warp_tot[lane] = w;
    }
    __syncthreads();
    const int prev = (wid > 0) ? warp_tot[wid - 1] : 0;
    if (idx < ncells) start[idx] = carry + prev + incl - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += prev + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) start[ncells] = carry;
}

// Deterministic placement: an atom's slot is the number of lower-indexed atoms in
// its cell (cells hold tens of atoms; the scan over the cell is short).
__device__ __forceinline__ void k_cell_fill(VGrid vg, int n, const int *__restrict__ atom_cell, const int *__restrict__ start,
                            int *cell_atoms, int *cell_cursor, const int *flags) {
  if (!(*flags & FLAG_REBUILD)) return;
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = atom_cell[i];
  const int slot = atomicAdd(&cell_cursor[c], 1);
  cell_atoms[start[c] + slot] = i;
}

__device__ __forceinline__ void k_cell_sort(VGrid vg, int ncells, const int *__restrict__ start, int *cell_atoms, const int *flags) {
  if (!(*flags & FLAG_REBUILD)) return;
  const int c = vg.bid * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  const int s = start[c], e = start[c + 1];
  for (int a = s + 1; a < e; a++) {
    const int v = cell_atoms[a];
    int b = a - 1;
    while (b >= s && cell_atoms[b] > v) { cell_atoms[b + 1] = cell_atoms[b]; b--; }
    cell_atoms[b + 1] = v;
  }
}

// One warp per atom i: every atom k != i of the neighbouring cells with
// image d2 <= rl2 on reduced coordinates (NeighborList.atomCellPairs, :1026-1115).
__device__ __forceinline__ void k_verlet(VGrid vg, int n, const double *__restrict__ rx, const double *__restrict__ ry,
                         const double *__restrict__ rz, const Box &bx, const CellOffsets &co,
                         const int *__restrict__ atom_cell, const int *__restrict__ start,
                         const int *__restrict__ cell_atoms, double rl2, int cap, int *nbr, int *nbr_cnt,
                         int *flags, double rn2, int capN, int *nbl, int *nbl_cnt) {
  if (!(*flags & FLAG_REBUILD)) return;
  const int warp = (vg.bid * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int i = warp;
  const double xi = rx[i], yi = ry[i], zi = rz[i];
  const int c = atom_cell[i];
  const int ncx = co.n[0], ncy = co.n[1], ncz = co.n[2];
  const int cx = c % ncx, cy = (c / ncx) % ncy, cz = c / (ncx * ncy);
  int count = 0, countN = 0;
  int *row = nbr + (size_t)i * cap;
  int *rowN = nbl ? nbl + (size_t)i * capN : nullptr;
  for (int oz = 0; oz < 5; oz++) {
    const int dz = co.off[2][oz];
    if (dz == 0x7fff) break;
    const int z2 = ((cz + dz) % ncz + ncz) % ncz;
    for (int oy = 0; oy < 5; oy++) {
      const int dy = co.off[1][oy];
      if (dy == 0x7fff) break;
      const int y2 = ((cy + dy) % ncy + ncy) % ncy;
      for (int ox = 0; ox < 5; ox++) {
        const int dx = co.off[0][ox];
        if (dx == 0x7fff) break;
        const int x2 = ((cx + dx) % ncx + ncx) % ncx;
        const int cell = (z2 * ncy + y2) * ncx + x2;
        const int s = start[cell], e = start[cell + 1];
        for (int base = s; base < e; base += 32) {
          const int a = base + lane;
          bool pass = false, near = false;
          int k = -1;
          if (a < e) {
            k = cell_atoms[a];
            if (k != i) {
              double ddx = __dsub_rn(xi, rx[k]), ddy = __dsub_rn(yi, ry[k]), ddz = __dsub_rn(zi, rz[k]);
              const double d2 = image_exact(ddx, ddy, ddz, bx);
              pass = d2 <= rl2;
              near = d2 <= rn2;
            }
          }
          const unsigned lt = (1u << lane) - 1u;
          const unsigned m = __ballot_sync(0xffffffffu, pass);
          if (pass) {
            const int pos = count + __popc(m & lt);
            if (pos < cap) row[pos] = k;
          }
          count += __popc(m);
          if (rowN) {
            const unsigned mn = __ballot_sync(0xffffffffu, near);
            if (near) {
              const int pos = countN + __popc(mn & lt);
              if (pos < capN) rowN[pos] = k;
            }
            countN += __popc(mn);
          }
        }
      }
    }
  }
  if (lane == 0) {
    nbr_cnt[i] = count;
    if (count > cap) atomicOr(flags, FLAG_NBR_OVERFLOW);
    if (rowN) {
      nbl_cnt[i] = countN;
      if (countN > capN) atomicOr(flags, FLAG_NBR_OVERFLOW);
    }
  }
}

// Multi-image list: one warp per atom i, lanes over every atom k, and every shift
// n = n0 + m (n0 the minimum-image shift of the reduced-coordinate difference, |m_d| <=
// R_d) with |x_k + n L - x_i|^2 <= rl2, except k == i at n = 0.  Entries keep k and the
// packed shift; the order (k chunk, then m) is fixed, so lists are reproducible.
__device__ __forceinline__ void k_verlet_images(VGrid vg, int n, const double *__restrict__ rx, const double *__restrict__ ry,
                                const double *__restrict__ rz, const Box &bx, int R0, int R1, int R2, double rl2,
                                int cap, int *nbr, int *nbr_sh, int *nbr_cnt, int *flags, const Box &super, int P0,
                                int P1, int P2) {
  if (!(*flags & FLAG_REBUILD)) return;
  const int warp = (vg.bid * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int i = warp;
  const double xi = rx[i], yi = ry[i], zi = rz[i];
  int count = 0;
  int *row = nbr + (size_t)i * cap;
  int *rsh = nbr_sh + (size_t)i * cap;
  for (int base = 0; base < n; base += 32) {
    const int k = base + lane;
    const bool valid = k < n;
    double dx = 0.0, dy = 0.0, dz = 0.0;
    int n0x = 0, n0y = 0, n0z = 0, px = 0, py = 0, pz = 0;
    bool ok = valid;
    if (valid) {
      dx = __dsub_rn(rx[k], xi); dy = __dsub_rn(ry[k], yi); dz = __dsub_rn(rz[k], zi);
      double fx, fy, fz, sx, sy, sz;
      to_frac(dx, dy, dz, bx, fx, fy, fz);
      const double gx = floor(__dadd_rn(fabs(fx), 0.5)) * jsignum(-fx);
      const double gy = floor(__dadd_rn(fabs(fy), 0.5)) * jsignum(-fy);
      const double gz = floor(__dadd_rn(fabs(fz), 0.5)) * jsignum(-fz);
      // The primary image: the minimum image in the replicate supercell (P0 x P1 x P2 cells).
      to_frac(dx, dy, dz, super, sx, sy, sz);
      const double hx = floor(__dadd_rn(fabs(sx), 0.5)) * jsignum(-sx);
      const double hy = floor(__dadd_rn(fabs(sy), 0.5)) * jsignum(-sy);
      const double hz = floor(__dadd_rn(fabs(sz), 0.5)) * jsignum(-sz);
      if (fabs(gx) + R0 > 511.0 || fabs(gy) + R1 > 511.0 || fabs(gz) + R2 > 511.0) {
        atomicOr(flags, FLAG_IMAGE_RANGE);
        ok = false;
      } else {
        n0x = (int)gx; n0y = (int)gy; n0z = (int)gz;
        px = P0 * (int)hx; py = P1 * (int)hy; pz = P2 * (int)hz;
      }
    }
    for (int mz = -R2; mz <= R2; mz++)
      for (int my = -R1; my <= R1; my++)
        for (int mx = -R0; mx <= R0; mx++) {
          const int nx = n0x + mx, ny = n0y + my, nz = n0z + mz;
          bool pass = false;
          if (ok && !(k == i && nx == 0 && ny == 0 && nz == 0)) {
            double ex = dx, ey = dy, ez = dz;
            add_shift(ex, ey, ez, nx, ny, nz, 1.0, bx);
            const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)), __dmul_rn(ez, ez));
            pass = d2 <= rl2;
          }
          const unsigned m = __ballot_sync(0xffffffffu, pass);
          if (pass) {
            const int pos = count + __popc(m & ((1u << lane) - 1u));
            if (pos < cap) {
              row[pos] = k;
              rsh[pos] = pack_shift(nx, ny, nz, nx == px && ny == py && nz == pz);
            }
          }
          count += __popc(m);
        }
  }
  if (lane == 0) {
    nbr_cnt[i] = count;
    if (count > cap) atomicOr(flags, FLAG_NBR_OVERFLOW);
  }
}

// Vacuum sub-system: every pair (k != i), no images, the shift field zero and marked
// minimum image; pairs dropped by the vapor softcore options (intermolecular: different
// molecules; intramolecular: the same molecule; PermanentFieldRegion.java:665-670).
__device__ __forceinline__ void k_vacuum_pairs(VGrid vg, int n, const int *__restrict__ mol, int inter, int intra, int cap, int *nbr,
                               int *nbr_sh, int *nbr_cnt, int *flags) {
  if (!(*flags & FLAG_REBUILD)) return;
  const int warp = (vg.bid * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int i = warp;
  int count = 0;
  for (int base = 0; base < n; base += 32) {
    const int k = base + lane;
    bool pass = k < n && k != i;
    if (pass) {
      const bool same = mol[k] == mol[i];
      if ((inter && !same) || (intra && same)) pass = false;
    }
    const unsigned m = __ballot_sync(0xffffffffu, pass);
    if (pass) {
      const int pos = count + __popc(m & ((1u << lane) - 1u));
      if (pos < cap) {
        nbr[(size_t)i * cap + pos] = k;
        nbr_sh[(size_t)i * cap + pos] = pack_shift(0, 0, 0, true);
      }
    }
    count += __popc(m);
  }
  if (lane == 0) {
    nbr_cnt[i] = count;
    if (count > cap) atomicOr(flags, FLAG_NBR_OVERFLOW);
  }
}

__device__ __forceinline__ void k_list_done(VGrid vg, int n, double *refx, double *refy, double *refz, const double *__restrict__ rx,
                            const double *__restrict__ ry, const double *__restrict__ rz, const int *flags) {
  if (!(*flags & FLAG_REBUILD)) return;
  const int i = vg.bid * blockDim.x + threadIdx.x;
  if (i >= n) return;
  refx[i] = rx[i]; refy[i] = ry[i]; refz[i] = rz[i];
}

// Cell counts and cursors cleared before a rebuild.
__device__ __forceinline__ void k_cell_clear(VGrid vg, int m, int *cnt, const int *flags) {
  if (!(*flags & FLAG_REBUILD)) return;
  for (int j = vg.bid * blockDim.x + threadIdx.x; j < m; j += vg.nblk * blockDim.x) cnt[j] = 0;
}

// ---------------------------------------------------------------------------
void launch_set_coordinates(Handle &h, const double *d_xyz) {
  const int n = h.n;
  launch_on<k_set_coordinates, 0, 0>(h.rec, nblocks(n, 256), 256, 0, h.stream, n, d_xyz, (const int *)h.d_redp,
                                     (const double *)h.d_redf, h.d_x, h.d_y, h.d_z, h.d_rx, h.d_ry, h.d_rz, h.d_pos);
  FFX_LAUNCHED(h);
  const double hb = 0.5 * h.prm.list_buffer;
  launch_on<k_reduce_coordinates, 0, 0>(h.rec, nblocks(n, 256), 256, 0, h.stream, n, (const double *)h.d_x,
                                        (const double *)h.d_y, (const double *)h.d_z, (const int *)h.d_redp,
                                        (const double *)h.d_redf, h.d_rx, h.d_ry, h.d_rz, (const double *)h.d_refx,
                                        (const double *)h.d_refy, (const double *)h.d_refz, hb * hb, h.d_flags,
                                        (const int *)h.d_vtype, h.d_rpos);
  FFX_LAUNCHED(h);
}

static CellOffsets cell_offsets(const int nc[3]) {
  CellOffsets co;
  for (int d = 0; d < 3; d++) {
    co.n[d] = nc[d];
    for (int j = 0; j < 5; j++) co.off[d][j] = 0x7fff;
    if (nc[d] >= 5) {
      for (int j = 0; j < 5; j++) co.off[d][j] = j - 2;
    } else {
      for (int j = 0; j < nc[d]; j++) co.off[d][j] = j;
    }
  }
  return co;
}

void launch_neighbor_list(Handle &h, bool force) {
  const int n = h.n;
  if (force) {
    int f = FLAG_REBUILD;
    cudaMemcpyAsync(h.d_flags, &f, sizeof(int), cudaMemcpyHostToDevice, h.stream);
    cudaStreamSynchronize(h.stream);
  }
  const double rl = fmax(h.prm.vdw_cutoff, h.prm.ewald_cutoff) + h.prm.list_buffer;
  const double rn = h.prm.ewald_cutoff + h.prm.list_buffer + 2.0 * kNearDelta;
  const int warps = nblocks((int64_t)n * 32, 256);
  const double *rx = h.d_rx, *ry = h.d_ry, *rz = h.d_rz;
  const int *flags = h.d_flags;
  if (h.vacuum) {
    launch_on<k_vacuum_pairs, 0, 0>(h.rec, warps, 256, 0, h.stream, n, (const int *)h.d_mol, h.alch.inter,
                                    h.alch.intra, h.cap_nbr, h.d_nbr, h.d_nbr_sh, h.d_nbr_cnt, h.d_flags);
    launch_on<k_list_done, 0, 0>(h.rec, nblocks(n, 256), 256, 0, h.stream, n, h.d_refx, h.d_refy, h.d_refz, rx, ry,
                                 rz, flags);
    h.launches += 2;
    return;
  }
  if (h.images) {
    launch_on<k_verlet_images, 0, 0>(h.rec, warps, 256, 0, h.stream, n, rx, ry, rz, h.box, h.img_range[0],
                                     h.img_range[1], h.img_range[2], rl * rl, h.cap_nbr, h.d_nbr, h.d_nbr_sh,
                                     h.d_nbr_cnt, h.d_flags, h.img_super, h.img_rep[0], h.img_rep[1], h.img_rep[2]);
    launch_on<k_list_done, 0, 0>(h.rec, nblocks(n, 256), 256, 0, h.stream, n, h.d_refx, h.d_refy, h.d_refz, rx, ry,
                                 rz, flags);
    h.launches += 2;
    return;
  }
  const int ncells = h.ncell[0] * h.ncell[1] * h.ncell[2];
  launch_on<k_cell_clear, 0, 0>(h.rec, nblocks(2 * ncells, 256), 256, 0, h.stream, 2 * ncells, h.d_cell_cnt,
                                flags);   // counts and cursors
  launch_on<k_cell_count, 0, 0>(h.rec, nblocks(n, 256), 256, 0, h.stream, n, rx, ry, rz, h.box, h.ncell[0],
                                h.ncell[1], h.ncell[2], h.d_cell_cnt, h.d_atom_cell, flags);
  launch_on<k_cell_scan, 0, 0>(h.rec, 1, 1024, 0, h.stream, ncells, (const int *)h.d_cell_cnt, h.d_cell_start,
                               flags);
  launch_on<k_cell_fill, 0, 0>(h.rec, nblocks(n, 256), 256, 0, h.stream, n, (const int *)h.d_atom_cell,
                               (const int *)h.d_cell_start, h.d_cell_atoms, h.d_cell_cnt + ncells, flags);
  launch_on<k_cell_sort, 0, 0>(h.rec, nblocks(ncells, 128), 128, 0, h.stream, ncells, (const int *)h.d_cell_start,
                               h.d_cell_atoms, flags);
  launch_on<k_verlet, 0, 0>(h.rec, warps, 256, 0, h.stream, n, rx, ry, rz, h.box, cell_offsets(h.ncell),
                            (const int *)h.d_atom_cell, (const int *)h.d_cell_start, (const int *)h.d_cell_atoms,
                            rl * rl, h.cap_nbr, h.d_nbr, h.d_nbr_cnt, h.d_flags, rn * rn, h.cap_nbl,
                            h.near_list ? h.d_nbl : (int *)nullptr, h.d_nbl_cnt);
  launch_on<k_list_done, 0, 0>(h.rec, nblocks(n, 256), 256, 0, h.stream, n, h.d_refx, h.d_refy, h.d_refz, rx, ry, rz,
                               flags);
  h.launches += 7;
}

}  // namespace ffx
