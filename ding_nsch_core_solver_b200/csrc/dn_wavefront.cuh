// dn_wavefront.cuh -- pipelined anti-diagonal wavefront for the 5-point ICC(0) / ILDLT(0) triangular solves
// (apply_preconditioner, ch_sparse_krylov.hpp:444-513) of the pressure operator.
//
// Factor storage.  For the 5-point pattern with nx, ny >= 4 the incomplete factors have no fill interaction
// (every L entry is a_rc / max(d_c, floor)), so only dinv = 1/max(d, floor) is stored and L is formed on the
// fly as a_rc * dinv_c.  Forward (ICC):  y_r = (r_r - sum_c a_rc w_c) dinv_r  with w_c = dinv_c y_c;
// backward (ICC): z_r = (y_r - dinv_r sum_{c>r} a_rc z_c) dinv_r.  ILDLT: y_r = r_r - sum a_rc w_c with
// w_c = Dinv_c y_c, z_r = Dinv_r (y_r - sum a_rc z_c).  The subtraction order per row follows the reference's
// CSR column order (wrap, W, wrap, S forward; N, wrap, E, wrap backward).
//
// Mapping.  Sweep warp k owns x-lines i = 32k + t (t = lane) for both sweeps and marches along j; lane t runs
// t steps behind lane t-1 (forward) or one step behind lane t+1 (backward), so the neighbour line's value of
// the previous step arrives by one warp shuffle.  Inputs are staged into shared memory by cp.async in
// 32-column chunks, two chunks ahead, into a 128-column ring (lane t reads column j at ring slot j & 127:
// row pitch 128 doubles keeps the skewed reads conflict-free).  Neighbouring warps hand over their edge
// line through shared memory (same CTA) or through global memory with release/acquire progress flags
// (different CTAs), published every 8 columns.  Every wait is bounded and reports kDevTimeout.
#pragma once

#include "dn_common.cuh"

namespace dn {

constexpr int kRing = 64;   // ring columns per staged array
constexpr int kChunk = 8;   // columns per cp.async chunk (= one hand-over group of steps)
constexpr int kHand = 8;    // columns per boundary publication
constexpr int kAhead = 3;   // chunks staged ahead of the one being consumed

struct Sweep5 {
  int nx, ny, n, px, py;
  int prec;     // kPrecICC (2) or kPrecLDLT (1)
  int varcoef;  // 0: constant off-diagonals cx/cy (split operator); 1: per-row slots aW, aS, aN, aE
  const double *aW, *aS, *aN, *aE;
  double cx, cy;  // -1/dx^2, -1/dy^2 for the constant operator
  const double *dinv;
  const double *r;  // forward input (the pending mean m_r is subtracted on the fly)
  double *y, *z;
  double *bnd_f, *bnd_b;      // [nsweep][ny] edge lines handed between CTAs
  double *wline0, *zlast;     // periodic-x wrap lines: w of line 0 (forward), z of line nx-1 (backward)
  unsigned int *prog_f, *prog_b;  // [nsweep] progress, monotonic across applications
  int nsweep, sw;             // sweep warps in total / per CTA
  int warp_smem;              // bytes between consecutive sweep warps' shared-memory regions
  int *status;
  double *prof;               // per sweep warp, 4 counters (ns): forward total, hand-over waits, staging waits, backward total
};

// per-warp shared-memory footprint (bytes) for `na` staged arrays and a ny-long hand-over line
__host__ __device__ inline size_t sweep_warp_smem(int na, int ny) {
  return (size_t)na * 32 * kRing * sizeof(double) + (size_t)((ny + 1) & ~1) * sizeof(double) + 64;
}

__device__ __forceinline__ unsigned int ld_acquire_cta(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.cta.shared.u32 %0, [%1];" : "=r"(v) : "r"((unsigned)__cvta_generic_to_shared(p)) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_cta(unsigned int *p, unsigned int v) {
  asm volatile("st.release.cta.shared.u32 [%0], %1;" ::"r"((unsigned)__cvta_generic_to_shared(p)), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned int *p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait2() { asm volatile("cp.async.wait_group 2;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_ahead() { asm volatile("cp.async.wait_group 3;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void st_global_if(double *p, double v, bool pred) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q st.global.f64 [%0], %1;\n\t}" ::"l"(p), "d"(v),
               "r"((int)pred));
}

// Bounded warp-uniform wait for a progress counter (shared or global) to reach `target`.
template <bool SHARED>
__device__ __forceinline__ unsigned int wait_progress(const unsigned int *cnt, unsigned int target, int *status) {
  const int lane = threadIdx.x & 31;
  long long spins = 0;
  unsigned int v = 0;
  while (true) {
    if (lane == 0) v = SHARED ? ld_acquire_cta(cnt) : ld_acquire_gpu(cnt);
    v = __shfl_sync(0xffffffffu, v, 0);
    if (v >= target) return v;
    ++spins;
    if ((spins & 1023) == 0 && (spins > kSpinLimit || *(volatile int *)status != kDevOk)) {
      if (lane == 0) atomicCAS(status, kDevOk, kDevTimeout);
      return 0;
    }
  }
}

// Stage columns [c0, c0+kChunk) of 32 lines starting at line i0 of array `src` into ring slot columns.
__device__ __forceinline__ void stage_chunk(double *ring, const double *src, int i0, int nlines, int ny, int c0,
                                           bool vec16) {
  const int lane = threadIdx.x & 31;
  if (c0 >= ny || c0 < 0) return;
  const int ncol = min(kChunk, ny - c0);
  if (vec16) {
    constexpr int per_line = kChunk / 2;  // 16-byte pieces per line
    for (int p = lane; p < 32 * per_line; p += 32) {
      const int line = p / per_line, pc = (p % per_line) * 2;
      if (line < nlines && pc < ncol)
        cp_async16(&ring[line * kRing + ((c0 + pc) & (kRing - 1))], &src[(size_t)(i0 + line) * ny + c0 + pc]);
    }
  } else {
    for (int p = lane; p < 32 * kChunk; p += 32) {
      const int line = p / kChunk, pc = p % kChunk;
      if (line < nlines && pc < ncol)
        cp_async8(&ring[line * kRing + ((c0 + pc) & (kRing - 1))], &src[(size_t)(i0 + line) * ny + c0 + pc]);
    }
  }
}

// Forward sweep of sweep warp k (warp slot `ws` inside its CTA).  Accumulates rz (= y^T y for ICC,
// y^T D^-1 y for ILDLT) and the sum of the projected residual into acc[1], acc[2].  Steps run in groups
// of kHand: the hand-over check precedes a group, the publication follows it; within a group every
// lane computes unconditionally (ring slots are always in range) and only stores / carries are
// predicated, so the per-step dependency chain is one shuffle and one FMA.
template <bool ICC, bool VAR>
__device__ __forceinline__ void fwd5_staged(const Sweep5 &P, char *smem_warp, unsigned int *cnt_cta, int k, int ws,
                                            unsigned int epoch, double m_r, double (&acc)[3]) {
  const int lane = threadIdx.x & 31;
  const int nx = P.nx, ny = P.ny, nsweep = P.nsweep, sw = P.sw;
  const int px = P.px, py = P.py;
  constexpr bool varcoef = VAR, icc = ICC;
  const double cx = P.cx, cy = P.cy;
  double *const yout = P.y;
  const double *const gr = P.r;
  const double *const gd = P.dinv;
  const double *const gW = P.aW;
  const double *const gS = P.aS;
  const double *const gN = P.aN;
  const double *const gE = P.aE;
  double *const bnd_f = P.bnd_f;
  double *const wline0 = P.wline0;
  unsigned int *const prog_f = P.prog_f;
  int *const status = P.status;
  double *const prof = P.prof;
  const int i0 = 32 * k;
  const int nlines = min(32, nx - i0);
  const int i = i0 + lane;
  const bool valid = lane < nlines;
  const int na = varcoef ? 4 : 2;
  double *ring_r = (double *)smem_warp;
  double *ring_d = ring_r + 32 * kRing;
  double *ring_w = ring_d + 32 * kRing;
  double *ring_s = ring_w + 32 * kRing;
  double *bline = ring_r + (size_t)na * 32 * kRing;
  const bool vec16 = (ny % 2) == 0;
  const bool prod_local = (k > 0) && (ws > 0);
  const bool cons_local = (k + 1 < nsweep) && (ws + 1 < sw);
  const bool last_warp = (k + 1 >= nsweep);
  const unsigned int base = epoch * (unsigned int)(ny + 1);
  const int total = ny + nlines - 1;
  const int nchunk = (total + kChunk - 1) / kChunk;
  double *next_bline = cons_local ? (double *)(smem_warp + P.warp_smem) + (size_t)na * 32 * kRing : nullptr;
  unsigned int *my_cnt = &cnt_cta[2 * ws];
  unsigned int *next_cnt = &cnt_cta[2 * (ws + 1)];
  const double aw_const = (valid && i > 0) ? cx : 0.0;  // W coefficient of the constant operator
  auto stage = [&](int c) {
    const int c0 = c * kChunk;
    stage_chunk(ring_r, gr, i0, nlines, ny, c0, vec16);
    stage_chunk(ring_d, gd, i0, nlines, ny, c0, vec16);
    if (varcoef) {
      stage_chunk(ring_w, gW, i0, nlines, ny, c0, vec16);
      stage_chunk(ring_s, gS, i0, nlines, ny, c0, vec16);
    }
    cp_async_commit();
  };
  const unsigned long long t_begin = global_ns();
  unsigned long long t_wait = 0;
  for (int c = 0; c < kAhead; ++c) stage(c);
  double w_prev = 0.0, w_first = 0.0, w_step = 0.0, bvals = 0.0;
  double rz = 0.0, rsum = 0.0;
  unsigned int avail = 0;
  const double *rowr = ring_r + lane * kRing;
  const double *rowd = ring_d + lane * kRing;
  const double *roww = ring_w + lane * kRing;
  const double *rows = ring_s + lane * kRing;
  double *ydst = yout + (size_t)i * ny;
  for (int q = 0; q < nchunk; ++q) {
    stage(q + kAhead);
    cp_async_wait_ahead();
    __syncwarp();
    {
      const int s0 = q * kChunk;
      // hand-over values of line i0-1 for columns [s0, s0+kHand), held by lanes 0..kHand-1
      if (k > 0 && s0 < ny) {
        const unsigned int need = base + (unsigned int)min(ny, s0 + kHand);
        if (avail + base < need) {
          const unsigned long long tw0 = global_ns();
          const unsigned int v = prod_local ? wait_progress<true>(my_cnt, need, status)
                                            : wait_progress<false>(&prog_f[k - 1], need, status);
          t_wait += global_ns() - tw0;
          if (v == 0) return;
          avail = v - base;
        }
        const int col = s0 + lane;
        if (lane < kHand && col < ny) bvals = prod_local ? bline[col] : __ldcg(&bnd_f[(size_t)(k - 1) * ny + col]);
      }
      // steady state: every lane of the group is inside [0, ny) -- no range checks, no wraps
      if (s0 >= 32 && s0 + kHand < ny && s0 + kHand <= total && !(px && i0 + 31 >= nx - 1 && i0 <= nx - 1)) {
        const bool hand = (lane == 31) && !last_warp;
#pragma unroll
        for (int ss = 0; ss < kHand; ++ss) {
          const int j = s0 + ss - lane;
          const int slot = j & (kRing - 1);
          const double rv = rowr[slot] - m_r;
          const double dv = rowd[slot];
          const double as = varcoef ? rows[slot] : cy;
          const double aw = varcoef ? ((i > 0) ? roww[slot] : 0.0) : aw_const;
          const double t1 = fma(-as, w_prev, rv);
          double w_up = __shfl_up_sync(0xffffffffu, w_step, 1);
          if (k > 0) {
            const double b = __shfl_sync(0xffffffffu, bvals, ss);
            if (lane == 0) w_up = b;
          }
          const double sum = fma(-aw, w_up, t1);
          const double yv = icc ? sum * dv : sum;
          const double wv = sum * (icc ? dv * dv : dv);
          st_global_if(&ydst[j], yv, valid);
          rz = fma(yv, icc ? yv : wv, rz);
          rsum += rv;
          if (cons_local) {
            if (hand) next_bline[j] = wv;
          } else {
            st_global_if(&bnd_f[(size_t)k * ny + j], wv, hand);
          }
          w_prev = valid ? wv : 0.0;
          w_step = valid ? wv : 0.0;
        }
        if (!valid) {
          rz = 0.0;
          rsum = 0.0;
        }
      } else {
#pragma unroll
      for (int ss = 0; ss < kHand; ++ss) {
        const int s = s0 + ss;
        const int j = s - lane;
        const bool act = valid && j >= 0 && j < ny && s < total;
        const int slot = j & (kRing - 1);
        const double rv = rowr[slot] - m_r;
        const double dv = rowd[slot];
        const double as = (j > 0) ? (varcoef ? rows[slot] : cy) : 0.0;
        const double aw = varcoef ? ((valid && i > 0) ? roww[slot] : 0.0) : aw_const;
        // own-line terms first (periodic-x wrap, periodic-y wrap, S), so that only one FMA follows the
        // shuffle that brings w of line i-1
        double t1 = rv;
        if (px && i == nx - 1 && act) t1 -= (varcoef ? gE[(size_t)i * ny + j] : cx) * __ldcg(&wline0[j]);
        if (py && j == ny - 1 && valid) t1 = fma(-(varcoef ? gN[(size_t)i * ny + j] : cy), w_first, t1);
        t1 = fma(-as, w_prev, t1);
        double w_up = __shfl_up_sync(0xffffffffu, w_step, 1);
        if (k > 0) {
          const double b = __shfl_sync(0xffffffffu, bvals, ss);
          if (lane == 0) w_up = b;
        }
        const double sum = fma(-aw, w_up, t1);
        const double yv = icc ? sum * dv : sum;
        const double wv = sum * (icc ? dv * dv : dv);
        if (act) {
          ydst[j] = yv;
          rz = fma(yv, icc ? yv : wv, rz);
          rsum += rv;
          if (px && i == 0) wline0[j] = wv;
          if (lane == 31 && !last_warp) {
            if (cons_local)
              next_bline[j] = wv;
            else
              bnd_f[(size_t)k * ny + j] = wv;
          }
          if (j == 0) w_first = wv;
          w_prev = wv;
          w_step = wv;
        }
      }
      }
      // publish columns finished by lane 31 (the hand-over line)
      const int done = min(ny, s0 + kHand - 31);
      if (!last_warp && done > 0) {
        __syncwarp();
        if (lane == 31) {
          if (cons_local)
            st_release_cta(next_cnt, base + (unsigned int)done);
          else
            st_release_gpu(&prog_f[k], base + (unsigned int)done);
        }
      }
    }
    __syncwarp();
  }
  cp_async_wait0();
  __syncwarp();
  acc[1] += rz;
  acc[2] += rsum;
  if (prof && lane == 0 && k < 16) {
    prof[4 * k + 0] = (double)(global_ns() - t_begin);
    prof[4 * k + 1] = (double)t_wait;
    prof[4 * k + 2] = 0.0;
  }
}

// Backward sweep of sweep warp k.  The lead lane is the last valid one (line i0+nlines-1); lane t runs
// (nlines-1-t) steps behind it.  Accumulates the sum of z into acc[0].
template <bool ICC, bool VAR>
__device__ __forceinline__ void bwd5_staged(const Sweep5 &P, char *smem_warp, unsigned int *cnt_cta, int k, int ws,
                                            unsigned int epoch, double (&acc)[3]) {
  const int lane = threadIdx.x & 31;
  const int nx = P.nx, ny = P.ny, nsweep = P.nsweep, sw = P.sw;
  const int px = P.px, py = P.py;
  constexpr bool varcoef = VAR, icc = ICC;
  const double cx = P.cx, cy = P.cy;
  double *const zout = P.z;
  const double *const gy = P.y;
  const double *const gd = P.dinv;
  const double *const gN = P.aN;
  const double *const gE = P.aE;
  const double *const gS = P.aS;
  const double *const gW = P.aW;
  double *const bnd_b = P.bnd_b;
  double *const zlast = P.zlast;
  unsigned int *const prog_b = P.prog_b;
  int *const status = P.status;
  double *const prof = P.prof;
  const int i0 = 32 * k;
  const int nlines = min(32, nx - i0);
  const int i = i0 + lane;
  const bool valid = lane < nlines;
  const int lead = nlines - 1;
  const int na = varcoef ? 4 : 2;
  double *ring_y = (double *)smem_warp;
  double *ring_d = ring_y + 32 * kRing;
  double *ring_n = ring_d + 32 * kRing;
  double *ring_e = ring_n + 32 * kRing;
  double *bline = ring_y + (size_t)na * 32 * kRing;
  const bool vec16 = (ny % 2) == 0;
  const bool prod_local = (k + 1 < nsweep) && (ws + 1 < sw);
  const bool cons_local = (k > 0) && (ws > 0);
  const unsigned int base = epoch * (unsigned int)(ny + 1);
  const int total = ny + nlines - 1;
  const int nchunk = (total + kChunk - 1) / kChunk;
  double *prev_bline = cons_local ? (double *)(smem_warp - P.warp_smem) + (size_t)na * 32 * kRing : nullptr;
  unsigned int *my_cnt = &cnt_cta[2 * ws + 1];
  unsigned int *prev_cnt = &cnt_cta[2 * (ws - 1) + 1];
  const double ae_const = (valid && i + 1 < nx) ? cx : 0.0;
  auto stage = [&](int c) {
    const int c0 = ny - kChunk * (c + 1);
    if (ny - kChunk * c <= 0) {
      cp_async_commit();
      return;
    }
    if (c0 >= 0) {
      stage_chunk(ring_y, gy, i0, nlines, ny, c0, vec16);
      stage_chunk(ring_d, gd, i0, nlines, ny, c0, vec16);
      if (varcoef) {
        stage_chunk(ring_n, gN, i0, nlines, ny, c0, vec16);
        stage_chunk(ring_e, gE, i0, nlines, ny, c0, vec16);
      }
    } else {
      const int hi = ny - kChunk * c;
      for (int p = lane; p < 32 * kChunk; p += 32) {
        const int line = p / kChunk, pc = p % kChunk;
        if (line < nlines && pc < hi) {
          const size_t gi = (size_t)(i0 + line) * ny + pc;
          const int sidx = line * kRing + (pc & (kRing - 1));
          cp_async8(&ring_y[sidx], &gy[gi]);
          cp_async8(&ring_d[sidx], &gd[gi]);
          if (varcoef) {
            cp_async8(&ring_n[sidx], &gN[gi]);
            cp_async8(&ring_e[sidx], &gE[gi]);
          }
        }
      }
    }
    cp_async_commit();
  };
  __syncwarp();  // y of these lines was written by this warp's forward sweep
  const unsigned long long t_begin = global_ns();
  for (int c = 0; c < kAhead; ++c) stage(c);
  double z_prev = 0.0, z_first = 0.0, z_step = 0.0, bvals = 0.0, zsum = 0.0;
  unsigned int avail = 0;
  const double *rowy = ring_y + lane * kRing;
  const double *rowd = ring_d + lane * kRing;
  const double *rown = ring_n + lane * kRing;
  const double *rowe = ring_e + lane * kRing;
  double *zdst = zout + (size_t)i * ny;
  for (int q = 0; q < nchunk; ++q) {
    stage(q + kAhead);
    cp_async_wait_ahead();
    __syncwarp();
    {
      const int s0 = q * kChunk;
      if (k + 1 < nsweep && s0 < ny) {
        const unsigned int need = base + (unsigned int)min(ny, s0 + kHand);
        if (avail + base < need) {
          const unsigned int v = prod_local ? wait_progress<true>(my_cnt, need, status)
                                            : wait_progress<false>(&prog_b[k + 1], need, status);
          if (v == 0) return;
          avail = v - base;
        }
        const int col = ny - 1 - (s0 + lane);
        if (lane < kHand && col >= 0)
          bvals = prod_local ? bline[col] : __ldcg(&bnd_b[(size_t)(k + 1) * ny + col]);
      }
      // steady state: every valid lane of the group is inside [0, ny) -- no range checks, no wraps
      if (s0 >= 32 && s0 + kHand < ny && s0 + kHand <= total && !(px && i0 == 0)) {
        const bool hand = (lane == 0) && (k > 0);
#pragma unroll
        for (int ss = 0; ss < kHand; ++ss) {
          const int j = ny - 1 - (s0 + ss - (lead - lane));
          const int slot = j & (kRing - 1);
          const double yv = rowy[slot];
          const double dv = rowd[slot];
          const double an = varcoef ? rown[slot] : cy;
          const double ae = varcoef ? ((i + 1 < nx) ? rowe[slot] : 0.0) : ae_const;
          const double t = an * z_prev;
          double z_dn = __shfl_down_sync(0xffffffffu, z_step, 1);
          if (k + 1 < nsweep) {
            const double b = __shfl_sync(0xffffffffu, bvals, ss);
            if (lane == lead) z_dn = b;
          }
          const double zv = icc ? fma(-(dv * dv), fma(ae, z_dn, t), yv * dv) : dv * (yv - fma(ae, z_dn, t));
          st_global_if(&zdst[j], zv, valid);
          zsum += valid ? zv : 0.0;
          if (cons_local) {
            if (hand) prev_bline[j] = zv;
          } else {
            st_global_if(&bnd_b[(size_t)k * ny + j], zv, hand);
          }
          z_prev = valid ? zv : 0.0;
          z_step = valid ? zv : 0.0;
        }
      } else {
#pragma unroll
      for (int ss = 0; ss < kHand; ++ss) {
        const int s = s0 + ss;
        const int j = ny - 1 - (s - (lead - lane));
        const bool act = valid && j >= 0 && j < ny && s < total;
        const int slot = j & (kRing - 1);
        const double yv = rowy[slot];
        const double dv = rowd[slot];
        const double an = (j + 1 < ny) ? (varcoef ? rown[slot] : cy) : 0.0;
        const double ae = varcoef ? ((valid && i + 1 < nx) ? rowe[slot] : 0.0) : ae_const;
        // upper neighbours in ascending column order: (i,j+1), (i,ny-1) [j==0], (i+1,j), (nx-1,j) [i==0]
        // own-line terms first; one FMA (plus the final scaling) follows the shuffle from line i+1
        double t = an * z_prev;
        if (py && j == 0 && valid) t = fma(varcoef ? gS[(size_t)i * ny] : cy, z_first, t);
        if (px && i == 0 && act) t = fma(varcoef ? gW[j] : cx, __ldcg(&zlast[j]), t);
        double z_dn = __shfl_down_sync(0xffffffffu, z_step, 1);
        if (k + 1 < nsweep) {
          const double b = __shfl_sync(0xffffffffu, bvals, ss);
          if (lane == lead) z_dn = b;
        }
        // ICC: z = (y - d t) d = y d - d^2 t ; ILDLT: z = D^-1 (y - t)
        const double zv = icc ? fma(-(dv * dv), fma(ae, z_dn, t), yv * dv) : dv * (yv - fma(ae, z_dn, t));
        if (act) {
          zdst[j] = zv;
          zsum += zv;
          if (px && i == nx - 1) zlast[j] = zv;
          if (lane == 0 && k > 0) {
            if (cons_local)
              prev_bline[j] = zv;
            else
              bnd_b[(size_t)k * ny + j] = zv;
          }
          if (j == ny - 1) z_first = zv;
          z_prev = zv;
          z_step = zv;
        }
      }
      }
      const int done = min(ny, s0 + kHand - lead);
      if (k > 0 && done > 0) {
        __syncwarp();
        if (lane == 0) {
          if (cons_local)
            st_release_cta(prev_cnt, base + (unsigned int)done);
          else
            st_release_gpu(&prog_b[k], base + (unsigned int)done);
        }
      }
    }
    __syncwarp();
  }
  cp_async_wait0();
  __syncwarp();
  acc[0] += zsum;
  if (prof && lane == 0 && k < 16) prof[4 * k + 3] = (double)(global_ns() - t_begin);
}

}  // namespace dn
