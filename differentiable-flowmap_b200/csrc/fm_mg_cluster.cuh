// fm_mg_cluster.cuh -- the coarse end of the MG V-cycle in one cluster launch.
//
// Included by fm_mgpcg.cu (needs DevState, kMaxLevels, rn_* and div_nd).
//
// The V-cycle below some level `lc` (at most 32768 cells) is latency-bound:
// each RBGS half-sweep, restriction and prolongation of the reference
// (3D/mgpcg.py:157-205) touches a few thousand cells but costs a kernel launch.
// k_mg_coarse does all of it -- levels lc .. L-1, down sweeps, restrictions,
// bottom smoothing, prolongations, up sweeps -- in one launch of a thread-block
// cluster of NC <= 8 CTAs:
//
//  * level lc is split along axis 0 into NC slabs of P = n0/NC planes (P even,
//    so every coarse plane of level lc+1 belongs to one CTA).  Each CTA keeps
//    its slab of r and z in shared memory, z with one ghost plane on each side.
//    After updating a cell of its first/last plane a CTA also stores the value
//    into the neighbour CTA's ghost plane (DSMEM through map_shared_rank); a
//    cluster barrier (release/acquire) ends every half-sweep.  A red half-sweep
//    writes red ghost cells while the neighbour reads only black ones (and vice
//    versa), so pushes never race with reads.
//  * the restriction of level lc writes straight into CTA 0's shared copy of
//    level lc+1; CTA 0 then runs levels lc+1 .. L-1 (each <= 4096 cells) alone
//    with __syncthreads, the bottom smoothing on a named barrier sized to the
//    bottom level's warps.
//  * prolongation reads CTA 0's level lc+1 through DSMEM; every CTA prolongs its
//    ghost planes itself (same operands, same rounding as the owner), so no
//    exchange is needed before the up sweeps.
//
// Instruction economy (a half-sweep is issue- and latency-bound at these sizes):
//  * z is stored with a ring of zero cells around each level (the slab's ghost
//    planes double as the ring along axis 0), so neighbour loads need no
//    bounds tests.  A missing neighbour then adds +0.0: the sum starts at +0.0
//    and a round-to-nearest sum of +0.0 and anything is never -0.0, so adding
//    +0.0 changes no partial sum and the result equals the skipping sum.
//  * cells are handled in (red, black) pairs along the innermost axis, one pair
//    per thread and slot, so every lane of a warp updates a cell in every
//    half-sweep (no colour divergence).
//  * the division by the neighbour count is div_nd: in FP32 a reciprocal
//    multiply with an FMA correction, equal to the IEEE quotient.
//
// Every arithmetic step is the reference's, in its order, without FMA
// contraction, so the result equals the sequential CPU V-cycle bit for bit.
#pragma once

#include <cooperative_groups.h>

namespace fm {

constexpr int kCoarseThreads = 1024;
constexpr int kCoarsePPT = 2;  // cell pairs per thread
constexpr int kCoarseMaxNC = 8;

struct CoarseArgs {
  Shape lv[kMaxLevels];
  int roff[kMaxLevels];  // deep level l (> lc): compact r at element roff[l] of CTA 0's deep area
  int zoff[kMaxLevels];  //                     zero-ringed z at element zoff[l]
  int lc, L;             // first cluster level, number of levels
  int pre_post, bottom, bottom_mode;
  const void* r_top;     // level lc residual (global)
  void* z_top;           // level lc correction (global)
};

// Strides of a zero-ringed array: (n0+2) x (n1+2) x (n2+2) in 3D, (n0+2) x (n1+2) in 2D.
template <int D>
struct Ring {
  int si, sj;  // the innermost stride is 1
  __device__ __forceinline__ explicit Ring(const Shape& s) {
    sj = D == 3 ? s.s2 + 2 : 1;
    si = (s.s1 + 2) * sj;
  }
  __device__ __forceinline__ int at(int p, int j, int k) const {  // p: plane in the array, ring included
    return p * si + (j + 1) * sj + (D == 3 ? k + 1 : 0);
  }
};
template <int D>
__host__ __device__ __forceinline__ long ring_size(const Shape& s, int planes) {
  return (long)planes * (s.s1 + 2) * (D == 3 ? s.s2 + 2 : 1);
}

// n / d for 0 <= n < 2^22, d >= 1, without an integer division.
__device__ __forceinline__ int small_div(int n, int d) {
  int q = __float2int_rz(__fdividef((float)n, (float)d));
  int r = n - q * d;
  while (r < 0) { --q; r += d; }
  while (r >= d) { ++q; r -= d; }
  return q;
}

template <int D>
__device__ __forceinline__ int n_dom(const Shape& s, int i, int j, int k) {
  int nd = 2 * D - (i == 0) - (i == s.s0 - 1) - (j == 0) - (j == s.s1 - 1);
  if (D == 3) nd -= (k == 0) + (k == s.s2 - 1);
  return nd;
}

// One thread's cell pairs in a block of planes [i0, i0+np) of level s.  A pair
// is cells k0 and k0+1 along the innermost axis (k in 3D, j in 2D).
// info: bit 0 parity of the first cell, bits 1-3 / 4-6 neighbour counts of the
// first / second cell, bit 7 second cell exists, bit 8 first plane of the
// block, bit 9 last plane.  zo < 0: no pair.
struct PairSet {
  int zo[kCoarsePPT];  // ringed z offset of the first cell (plane index relative to the block, ring plane = 0)
  int ro[kCoarsePPT];  // compact r offset of the first cell
  int info[kCoarsePPT];
};

template <int D>
__device__ __forceinline__ void pairs_init(PairSet& ps, const Shape& s, int i0, int np, int tid, int nthr) {
  const Ring<D> rg(s);
  const int nin = D == 3 ? s.s2 : s.s1;  // innermost extent
  const int npr = (nin + 1) >> 1;        // pairs per row
  const int rows_per_plane = D == 3 ? s.s1 : 1;
  const int npairs = np * rows_per_plane * npr;
#pragma unroll
  for (int m = 0; m < kCoarsePPT; ++m) {
    const int t = tid + m * nthr;
    ps.zo[m] = -1;
    ps.ro[m] = 0;
    ps.info[m] = 0;
    if (t >= npairs) continue;
    const int row = small_div(t, npr), kk = t - row * npr;
    int p, j, k;
    if (D == 3) {
      p = small_div(row, s.s1);
      j = row - p * s.s1;
      k = 2 * kk;
    } else {
      p = row;
      j = 2 * kk;
      k = 0;
    }
    const int i = i0 + p;
    const bool second = (D == 3 ? k : j) + 1 < nin;
    ps.zo[m] = rg.at(p + 1, j, k);
    ps.ro[m] = (p * s.s1 + j) * s.s2 + k;
    const int nd0 = n_dom<D>(s, i, j, k);
    const int nd1 = second ? (D == 3 ? n_dom<D>(s, i, j, k + 1) : n_dom<D>(s, i, j + 1, k)) : 0;
    ps.info[m] = ((i + j + k) & 1) | (nd0 << 1) | (nd1 << 4) | ((int)second << 7) | ((p == 0) << 8) |
                 ((p == np - 1) << 9);
  }
}

// One RBGS half-sweep of colour c (3D/mgpcg.py:170-177) over a thread's pairs.
// push_lo / push_hi (or null): the neighbour CTAs' z arrays, receiving the new
// values of the block's first / last plane at offset o + lo_shift / o + hi_shift.
template <typename T, int D>
__device__ __forceinline__ void sweep_pairs(const PairSet& ps, T* z, const T* r, int si, int sj, int c,
                                            T* push_lo, int lo_shift, T* push_hi, int hi_shift) {
#pragma unroll
  for (int m = 0; m < kCoarsePPT; ++m) {
    const int info = ps.info[m];
    const int sel = (info ^ c) & 1;  // 0: the first cell has colour c
    if (ps.zo[m] < 0 || (sel && !(info & 128))) continue;
    const int o = ps.zo[m] + sel;
    T nb = 0;
    nb += z[o + si];
    nb += z[o - si];
    nb += z[o + sj];
    nb += z[o - sj];
    if (D == 3) {
      nb += z[o + 1];
      nb += z[o - 1];
    }
    const T v = div_nd(r[ps.ro[m] + sel] + nb, sel ? (info >> 4) & 7 : (info >> 1) & 7);
    z[o] = v;
    if (push_lo && (info & 256)) push_lo[o + lo_shift] = v;
    if (push_hi && (info & 512)) push_hi[o + hi_shift] = v;
  }
}

// Residual r - A z at a cell of a ringed array (restrict, 3D/mgpcg.py:157-163).
template <typename T, int D>
__device__ __forceinline__ T residual_ring(const T* z, int o, T rv, int si, int sj, int nd) {
  T nb = 0;
  nb += z[o + si];
  nb += z[o - si];
  nb += z[o + sj];
  nb += z[o - sj];
  if (D == 3) {
    nb += z[o + 1];
    nb += z[o - 1];
  }
  return rn_sub(rv, rn_sub(rn_mul((T)nd, z[o]), nb));
}

// Gather-restriction of coarse cell (I, J, K) from a block of fine planes
// starting at global plane i0 (ringed z: plane p of the block at ring plane p+1).
template <typename T, int D>
__device__ __forceinline__ T restrict_ring(const T* z, const T* r, const Shape& sf, int i0, int I, int J, int K) {
  const T scale = (T)1.0 / (T)(D - 1.0);
  const Ring<D> rg(sf);
  T acc = 0;
#pragma unroll
  for (int di = 0; di < 2; ++di)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj)
#pragma unroll
      for (int dk = 0; dk < (D == 3 ? 2 : 1); ++dk) {
        const int i = 2 * I + di, j = 2 * J + dj, k = D == 3 ? 2 * K + dk : 0;
        const T rv = r[((i - i0) * sf.s1 + j) * sf.s2 + k];
        const T res = residual_ring<T, D>(z, rg.at(i - i0 + 1, j, k), rv, rg.si, rg.sj, n_dom<D>(sf, i, j, k));
        acc = rn_add(acc, rn_mul(res, scale));
      }
  return acc;
}

// Smoothing pairs of one whole deep level by the first `nthr` threads of the
// CTA, each half-sweep ended by a barrier over those threads.
template <typename T, int D>
__device__ __forceinline__ void level_sweeps(const Shape& s, T* z, const T* r, int first, int pairs, int tid,
                                             int nthr, int bar_id) {
  if (pairs <= 0) return;
  PairSet ps;
  pairs_init<D>(ps, s, 0, s.s0, tid, nthr);
  const Ring<D> rg(s);
  for (int it = 0; it < pairs; ++it) {
    sweep_pairs<T, D>(ps, z, r, rg.si, rg.sj, first, nullptr, 0, nullptr, 0);
    asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthr) : "memory");
    sweep_pairs<T, D>(ps, z, r, rg.si, rg.sj, 1 - first, nullptr, 0, nullptr, 0);
    asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthr) : "memory");
  }
}

// Prolongation z_f += z_c (3D/mgpcg.py:165-168) over ring planes [p_lo, p_hi)
// of a ringed fine block whose ring plane 0 is global plane i0 - 1.
template <typename T, int D>
__device__ __forceinline__ void prolong_ring(T* zf, const Shape& sf, int i0, int p_lo, int p_hi, const T* zc,
                                             const Shape& sc, int tid, int nthr) {
  const Ring<D> rf(sf), rc(sc);
  const int rowlen = D == 3 ? sf.s2 : sf.s1;
  const int rows_per_plane = D == 3 ? sf.s1 : 1;
  const int n = (p_hi - p_lo) * rows_per_plane * rowlen;
  for (int q = tid; q < n; q += nthr) {
    const int row = small_div(q, rowlen), x = q - row * rowlen;
    int p, j, k;
    if (D == 3) {
      const int pp = small_div(row, sf.s1);
      p = p_lo + pp;
      j = row - pp * sf.s1;
      k = x;
    } else {
      p = p_lo + row;
      j = x;
      k = 0;
    }
    const int i = i0 - 1 + p;
    zf[rf.at(p, j, k)] += zc[rc.at((i >> 1) + 1, j >> 1, k >> 1)];
  }
}

template <typename T, int D>
__global__ void __launch_bounds__(kCoarseThreads, 1) k_mg_coarse(CoarseArgs a, const DevState* st) {
  pdl_begin();
  namespace cg = cooperative_groups;
  if (st->done) return;  // same value in every CTA of the cluster
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int NC = (int)cluster.num_blocks();
  const int tid = threadIdx.x, nthr = blockDim.x;
  extern __shared__ double smem_d[];
  T* sm = reinterpret_cast<T*>(smem_d);

  const Shape s = a.lv[a.lc];
  const int P = s.s0 / NC, i0 = rank * P;
  const Ring<D> rg(s);
  const int zsz = (int)ring_size<D>(s, P + 2), rsz = P * s.s1 * s.s2;
  T* z = sm;           // ring planes 0 .. P+1: ghost, own planes, ghost
  T* r = z + zsz;      // own planes, compact
  T* deep = r + rsz;   // levels lc+1 .. L-1 (used by CTA 0)
  T* push_lo = rank > 0 ? cluster.map_shared_rank(z, rank - 1) : nullptr;
  T* push_hi = rank < NC - 1 ? cluster.map_shared_rank(z, rank + 1) : nullptr;
  const int lo_shift = P * rg.si, hi_shift = -P * rg.si;

  const T* rt = reinterpret_cast<const T*>(a.r_top) + (long)i0 * s.s1 * s.s2;
  for (int q = tid; q < rsz; q += nthr) r[q] = rt[q];
  for (int q = tid; q < zsz; q += nthr) z[q] = 0;
  PairSet ps;
  pairs_init<D>(ps, s, i0, P, tid, nthr);
  cluster.sync();  // ghosts zeroed everywhere before the first push

  // pre-smoothing of level lc (z starts at zero)
  for (int it = 0; it < a.pre_post; ++it) {
    sweep_pairs<T, D>(ps, z, r, rg.si, rg.sj, 0, push_lo, lo_shift, push_hi, hi_shift);
    cluster.sync();
    sweep_pairs<T, D>(ps, z, r, rg.si, rg.sj, 1, push_lo, lo_shift, push_hi, hi_shift);
    cluster.sync();
  }
  // restriction into CTA 0's level lc+1
  const Shape s1 = a.lv[a.lc + 1];
  {
    T* r1 = cluster.map_shared_rank(deep + a.roff[a.lc + 1], 0);
    const int cplane = s1.s1 * s1.s2, ncell = (P / 2) * cplane;
    for (int q = tid; q < ncell; q += nthr) {
      const int pI = small_div(q, cplane), rem = q - pI * cplane;
      const int J = D == 3 ? small_div(rem, s1.s2) : rem, K = D == 3 ? rem - J * s1.s2 : 0;
      const int I = i0 / 2 + pI;
      r1[I * cplane + rem] = restrict_ring<T, D>(z, r, s, i0, I, J, K);
    }
  }
  cluster.sync();

  if (rank == 0) {
    auto rl = [&](int l) { return deep + a.roff[l]; };
    auto zl = [&](int l) { return deep + a.zoff[l]; };
    for (int l = a.lc + 1; l < a.L - 1; ++l) {
      const Shape sl = a.lv[l];
      const int zs = (int)ring_size<D>(sl, sl.s0 + 2);
      for (int q = tid; q < zs; q += nthr) zl(l)[q] = 0;
      __syncthreads();
      level_sweeps<T, D>(sl, zl(l), rl(l), 0, a.pre_post, tid, nthr, 0);
      const Shape sc = a.lv[l + 1];
      for (int q = tid; q < sc.size(); q += nthr) {
        int I, J, K;
        unflatten(sc, q, I, J, K);
        rl(l + 1)[q] = restrict_ring<T, D>(zl(l), rl(l), sl, 0, I, J, K);
      }
      __syncthreads();
    }
    // bottom smoothing (3D/mgpcg.py:197-199; mgpcg_solid.py:263-268)
    const int b = a.L - 1;
    const Shape sb = a.lv[b];
    {
      const int zs = (int)ring_size<D>(sb, sb.s0 + 2);
      for (int q = tid; q < zs; q += nthr) zl(b)[q] = 0;
    }
    __syncthreads();
    const int nin = D == 3 ? sb.s2 : sb.s1;
    const int npairs = sb.s0 * (D == 3 ? sb.s1 : 1) * ((nin + 1) >> 1);
    const int nb_thr = npairs < nthr ? ((npairs + 31) & ~31) : nthr;
    if (tid < nb_thr) {
      if (a.bottom_mode == 0) {
        level_sweeps<T, D>(sb, zl(b), rl(b), 0, a.bottom, tid, nb_thr, 1);
      } else {
        level_sweeps<T, D>(sb, zl(b), rl(b), 0, a.bottom / 2, tid, nb_thr, 1);
        level_sweeps<T, D>(sb, zl(b), rl(b), 1, a.bottom / 2, tid, nb_thr, 1);
      }
    }
    __syncthreads();
    for (int l = a.L - 2; l > a.lc; --l) {
      const Shape sl = a.lv[l];
      prolong_ring<T, D>(zl(l), sl, 0, 1, sl.s0 + 1, zl(l + 1), a.lv[l + 1], tid, nthr);
      __syncthreads();
      level_sweeps<T, D>(sl, zl(l), rl(l), 1, a.pre_post, tid, nthr, 0);
    }
  }
  cluster.sync();

  // prolongation into the slab, ghost planes inside the domain included
  {
    const T* z1 = cluster.map_shared_rank(deep + a.zoff[a.lc + 1], 0);
    const int p_lo = rank > 0 ? 0 : 1, p_hi = rank < NC - 1 ? P + 2 : P + 1;
    prolong_ring<T, D>(z, s, i0, p_lo, p_hi, z1, s1, tid, nthr);
  }
  cluster.sync();  // all reads of CTA 0 done, ghosts prolonged before any push
  for (int it = 0; it < a.pre_post; ++it) {
    sweep_pairs<T, D>(ps, z, r, rg.si, rg.sj, 1, push_lo, lo_shift, push_hi, hi_shift);
    cluster.sync();
    sweep_pairs<T, D>(ps, z, r, rg.si, rg.sj, 0, push_lo, lo_shift, push_hi, hi_shift);
    cluster.sync();
  }
  // write the own planes back (compact)
  T* zt = reinterpret_cast<T*>(a.z_top) + (long)i0 * s.s1 * s.s2;
  for (int q = tid; q < rsz; q += nthr) {
    int p, j, k;
    if (D == 3) {
      const int row = small_div(q, s.s2);
      k = q - row * s.s2;
      p = small_div(row, s.s1);
      j = row - p * s.s1;
    } else {
      p = small_div(q, s.s1);
      j = q - p * s.s1;
      k = 0;
    }
    zt[q] = z[rg.at(p + 1, j, k)];
  }
}

}  // namespace fm
