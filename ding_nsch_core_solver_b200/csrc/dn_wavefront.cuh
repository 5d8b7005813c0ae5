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
// Mapping.  Sweep warp k owns the kLines = 31 x-lines i = 31k .. 31k+30 and marches along j.  The 32nd lane
// is a ghost that replays the neighbouring warp's edge line (line 31k-1 in the forward sweep, 31k+31 in the
// backward sweep) from a shared-memory hand-over line through the same arithmetic with zero coefficients
// and unit dinv, so every lane receives its neighbour's value of the previous step by one plain warp
// shuffle and a step has no lane-dependent selects.  Lanes that own no line read a zero row and carry 0.
// Inputs are staged by cp.async in 16-column chunks, one chunk ahead, into per-lane ring rows of 64
// columns plus a 16-column mirror (row pitch 80 elements: skewed reads stay bank-conflict free), so that
// the 16 steps of a group read at fixed offsets from one base pointer.  Neighbouring warps hand over their
// edge line through a shared-memory line (same CTA) or a global line (different CTAs) without flags: the
// lines hold a NaN sentinel until the producer stores a value, and the consumer waits on the values
// themselves and writes the sentinel back after use.  Every wait is bounded and reports kDevTimeout.
#pragma once

#include "dn_common.cuh"

namespace dn {

constexpr int kRing = 64;                // ring columns per staged array
constexpr int kMirror = 16;              // mirrored columns so a group of kHand steps never wraps
constexpr int kPitch = kRing + kMirror;  // doubles per ring row
constexpr int kChunk = 16;               // columns per cp.async chunk (= one group of steps)
constexpr int kHand = 16;                // steps per group (hand-over columns checked together)
constexpr int kAhead = 1;                // chunks staged ahead of the one being consumed
constexpr int kLines = 31;               // grid lines per sweep warp (lane 31 / lane 0 is the ghost)
constexpr int kWrapPad = 32;             // elements of padding on each side of a periodic-x wrap line

// T is the storage and arithmetic type of the sweep (double, or float for the inner solves of the
// mixed-precision form); the sums handed back (r.z, sum z, sum r) are accumulated in double either way.
template <typename T>
struct Sweep5T {
  int nx, ny, n, px, py;
  int prec;     // kPrecICC (2) or kPrecLDLT (1)
  int varcoef;  // 0: constant off-diagonals cx/cy (split operator); 1: per-row slots aW, aS, aN, aE
  const T *aW, *aS, *aN, *aE;
  T cx, cy;  // -1/dx^2, -1/dy^2 for the constant operator
  const T *dinv;
  const T *r;  // forward input (the pending mean m_r is subtracted on the fly)
  T *y, *z;
  T *bnd_f, *bnd_b;           // [2][nsweep][ny] edge lines handed between CTAs (by application parity)
  T *wline0, *zlast;          // [2][ny] periodic-x wrap lines (by application parity): w of line 0 for
                              // line nx-1 (forward), z of line nx-1 for line 0 (backward)
  unsigned int *prog_f, *prog_b;  // unused by the staged path (kept for the launch arguments' layout)
  int nsweep, sw;             // sweep warps in total (ceil(nx / kLines)) / per CTA
  int warp_smem;              // bytes between consecutive sweep warps' shared-memory regions
  int *status;
  double *prof;               // per sweep warp, 4 counters (ns): forward total, hand-over waits, 0, backward total
};
using Sweep5 = Sweep5T<double>;

__host__ __device__ inline int staged_sweep_warps(int nx) { return (nx + kLines - 1) / kLines; }

// Elements of one periodic-x wrap line in shared memory (values or coefficients), padding included.
__host__ __device__ inline size_t wrap_line_stride(int ny) { return (size_t)((ny + 3) & ~3) + 2 * kWrapPad; }
// per-warp shared-memory footprint (bytes) for `na` staged arrays of `esize`-byte elements, two ny-long
// hand-over lines (forward, backward), the zero / unit rows read by lanes that own no line, and with
// periodic x the wrap values and coefficients
__host__ __device__ inline size_t sweep_warp_smem(int na, int ny, int esize = 8, bool px = false) {
  return (size_t)na * 32 * kPitch * esize + 2 * (size_t)((ny + 3) & ~3) * esize + 2 * (size_t)kPitch * esize + 64 +
         (px ? 2 * wrap_line_stride(ny) * esize : 0);
}
// Offset (elements) of a sweep warp's forward hand-over line in its region; the backward line follows it.
__host__ __device__ inline size_t sweep_hand_line(int na) { return (size_t)na * 32 * kPitch; }

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
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(gmem)
               : "memory");
}
template <typename T>
__device__ __forceinline__ void cp_async_elem(void *smem, const void *gmem) {
  if (sizeof(T) == 8)
    cp_async8(smem, gmem);
  else
    cp_async4(smem, gmem);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
static_assert(kAhead == 1, "cp_async_wait_ahead waits for all but the newest kAhead groups");
static_assert(kLines + kChunk * (kAhead + 1) <= kRing, "the ring holds the skew window plus the staged chunks");
__device__ __forceinline__ void cp_async_wait_ahead() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Cross-CTA hand-over.  The edge line goes through global memory without flags or fences: each launch
// fills the line buffers with a NaN sentinel, the producer stores its values, and the consumer polls the
// values themselves (relaxed GPU-scope loads) and writes the sentinel back after use.  Buffers alternate
// by application parity, so a reset lands two applications (and several grid barriers) before reuse.
constexpr unsigned long long kHandEmpty = 0x7ff4dead5eed0001ull;
constexpr unsigned int kHandEmpty32 = 0x7fa5eed1u;
__device__ __forceinline__ double ld_relaxed_gpu(const double *p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ float ld_relaxed_gpu(const float *p) {
  float v;
  asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ bool hand_empty(double v) {
  return (unsigned long long)__double_as_longlong(v) == kHandEmpty;
}
__device__ __forceinline__ bool hand_empty(float v) { return (unsigned int)__float_as_uint(v) == kHandEmpty32; }
template <typename T>
__device__ __forceinline__ T hand_empty_value();
template <>
__device__ __forceinline__ double hand_empty_value<double>() {
  return __longlong_as_double((long long)kHandEmpty);
}
template <>
__device__ __forceinline__ float hand_empty_value<float>() {
  return __uint_as_float(kHandEmpty32);
}

// Stores under a per-lane predicate without a branch: the warp stays converged for the shuffle that
// follows in the same step.
__device__ __forceinline__ void st_global_if(double *p, double v, bool pred) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q st.global.f64 [%0], %1;\n\t}" ::"l"(p), "d"(v),
               "r"((int)pred)
               : "memory");
}
__device__ __forceinline__ void st_generic_if(double *p, double v, bool pred) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q st.f64 [%0], %1;\n\t}" ::"l"(p), "d"(v),
               "r"((int)pred)
               : "memory");
}
__device__ __forceinline__ void st_global_if(float *p, float v, bool pred) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q st.global.f32 [%0], %1;\n\t}" ::"l"(p), "f"(v),
               "r"((int)pred)
               : "memory");
}
__device__ __forceinline__ void st_generic_if(float *p, float v, bool pred) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q st.f32 [%0], %1;\n\t}" ::"l"(p), "f"(v),
               "r"((int)pred)
               : "memory");
}

// Same-CTA hand-over without flags: the consumer's line starts as the sentinel, the producer stores its
// values into it, the consumer waits (bounded) until the group's columns are no longer the sentinel and
// writes the sentinel back after use.  `cols` gives lane t's column of the group (negative: none).
template <typename T>
__device__ __forceinline__ bool wait_local_line(T *line, int col, int *status, unsigned long long &t_wait) {
  bool miss = col >= 0 && hand_empty(*(volatile T *)&line[col]);
  if (__any_sync(0xffffffffu, miss)) {
    const unsigned long long tw0 = global_ns();
    long long spins = 0;
    while (__any_sync(0xffffffffu, miss)) {
      ++spins;
      if (spins > spin_limit(status) || ((spins & 1023) == 0 && *(volatile int *)status != kDevOk)) {
        if ((threadIdx.x & 31) == 0) atomicCAS(status, kDevOk, kDevTimeout);
        return false;
      }
      if (spins > 32) __nanosleep(64);
      if (miss) miss = hand_empty(*(volatile T *)&line[col]);
    }
    t_wait += global_ns() - tw0;
  }
  __syncwarp();
  return true;
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
    // a warp that waits long (a backward sweep waiting for the whole chain above it) sleeps between
    // polls, so that it takes no issue slots from a sweep warp sharing its scheduler
    if (spins > 32) __nanosleep(64);
    if (spins > spin_limit(status) || ((spins & 1023) == 0 && *(volatile int *)status != kDevOk)) {
      if (lane == 0) atomicCAS(status, kDevOk, kDevTimeout);
      return 0;
    }
  }
}

// Stage columns [c0, c1) of `nl` grid lines starting at line i0 into ring rows row0 .. row0+nl-1.  Column j
// goes to row offset off + (j & 63); the mirrored columns are written twice (forward: slots 0..15 again at
// 64..79, off = 0; backward: slots 48..63 again at 0..15, off = 16).  16-byte pieces when ny allows them.
template <bool FWD, typename T>
__device__ __forceinline__ void stage_cols(T *ring, const T *src, int i0, int row0, int nl, int ny, int c0,
                                           int c1, bool vec16) {
  const int lane = threadIdx.x & 31;
  c0 = max(c0, 0);
  c1 = min(c1, ny);
  if (c0 >= c1) return;
  constexpr int off = FWD ? 0 : kMirror;
  constexpr int E = 16 / (int)sizeof(T);  // elements per 16-byte piece
  if (vec16) {  // ny a multiple of E: c0 and c1 are too
    const int npair = (c1 - c0) / E;
    for (int p = lane; p < nl * npair; p += 32) {
      const int line = p / npair, j = c0 + E * (p - line * npair);
      const T *g = &src[(size_t)(i0 + line) * ny + j];
      T *row = ring + (size_t)(row0 + line) * kPitch;
      const int slot = j & (kRing - 1);
      cp_async16(&row[off + slot], g);
      if (FWD ? (slot < kMirror) : (slot >= kRing - kMirror)) cp_async16(&row[FWD ? kRing + slot : slot - (kRing - kMirror)], g);
    }
  } else {
    const int ncol = c1 - c0;
    for (int p = lane; p < nl * ncol; p += 32) {
      const int line = p / ncol, j = c0 + (p - line * ncol);
      const T *g = &src[(size_t)(i0 + line) * ny + j];
      T *row = ring + (size_t)(row0 + line) * kPitch;
      const int slot = j & (kRing - 1);
      cp_async_elem<T>(&row[off + slot], g);
      if (FWD ? (slot < kMirror) : (slot >= kRing - kMirror))
        cp_async_elem<T>(&row[FWD ? kRing + slot : slot - (kRing - kMirror)], g);
    }
  }
}

// Stage one whole chunk [c0, c0+kChunk) (ny a multiple of the 16-byte piece; for the backward ring also
// ny % kChunk == 0, so that the chunk sits at a chunk-aligned ring slot): lane t copies one 16-byte piece
// (2 doubles or 4 floats) per array of line t / PL + LI it, PL pieces per line, with no division and
// addresses from one per-lane offset.  The chunk at the mirrored slot is copied a second time (forward:
// slot 0 again at kRing, backward: slot kRing - kChunk again at 0).
template <bool FWD, int NA, typename T>
__device__ __forceinline__ void stage_full(T *r0, T *r1, T *r2, T *r3, const T *s0, const T *s1, const T *s2,
                                           const T *s3, int i0, int row0, int nl, int ny, int c0) {
  constexpr int E = 16 / (int)sizeof(T);  // elements per 16-byte piece
  constexpr int PL = kChunk / E;          // pieces per line of the chunk
  constexpr int LI = 32 / PL;             // lines per pass of the warp
  constexpr int IT = (kLines + LI - 1) / LI;
  const int lane = threadIdx.x & 31;
  const int l0 = lane / PL, cc = E * (lane % PL);
  const int slot = c0 & (kRing - 1);
  constexpr int off = FWD ? 0 : kMirror;
  const bool mirror = FWD ? (slot == 0) : (slot == kRing - kChunk);
  constexpr int mdelta = FWD ? kRing : -kRing;
  const size_t gofs = (size_t)(i0 + l0) * ny + c0 + cc;
  const int sofs = (row0 + l0) * kPitch + off + slot + cc;
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    if (l0 + LI * it < nl) {
      const size_t g = gofs + (size_t)(LI * it) * ny;
      const int sd = sofs + LI * it * kPitch;
      cp_async16(r0 + sd, s0 + g);
      cp_async16(r1 + sd, s1 + g);
      if (NA == 4) {
        cp_async16(r2 + sd, s2 + g);
        cp_async16(r3 + sd, s3 + g);
      }
      if (mirror) {
        cp_async16(r0 + sd + mdelta, s0 + g);
        cp_async16(r1 + sd + mdelta, s1 + g);
        if (NA == 4) {
          cp_async16(r2 + sd + mdelta, s2 + g);
          cp_async16(r3 + sd + mdelta, s3 + g);
        }
      }
    }
  }
}

// Wait (bounded) until this lane's value v of src[col] is no longer the sentinel; `mine` lanes only.
// Returns false, with status set to kDevTimeout, when the wait gives up.
template <typename T>
__device__ __forceinline__ bool poll_line(const T *src, int col, bool mine, T &v, int *status,
                                          unsigned long long &t_wait) {
  bool miss = mine && hand_empty(v);
  if (!__any_sync(0xffffffffu, miss)) return true;
  const unsigned long long tw0 = global_ns();
  long long spins = 0;
  while (__any_sync(0xffffffffu, miss)) {
    ++spins;
    if (spins > spin_limit(status) || ((spins & 1023) == 0 && *(volatile int *)status != kDevOk)) {
      if ((threadIdx.x & 31) == 0) atomicCAS(status, kDevOk, kDevTimeout);
      return false;
    }
    if (spins > 32) __nanosleep(64);
    if (miss) {
      v = ld_relaxed_gpu(src + col);
      miss = hand_empty(v);
    }
  }
  t_wait += global_ns() - tw0;
  return true;
}

// Forward sweep of sweep warp k (warp slot `ws` inside its CTA).  Lane 0 is the ghost of line 31k-1, lanes
// 1..nl own lines 31k .. 31k+nl-1; lane t runs t steps behind the ghost.  Accumulates rz (= y^T y for
// ICC, y^T D^-1 y for ILDLT) and the sum of the projected residual into acc[1], acc[2].  Steps run in
// groups of kHand: the hand-over check precedes a group, the publication follows it.
template <bool ICC, bool VAR, typename T = double, bool PX = false>
__device__ __forceinline__ void fwd5_staged(const Sweep5T<T> &P, char *smem_warp, unsigned int *cnt_cta, int k, int ws,
                                            unsigned int epoch, double m_r, double (&acc)[3]) {
  const int lane = threadIdx.x & 31;
  const int nx = P.nx, ny = P.ny, nsweep = P.nsweep, sw = P.sw;
  const int py = P.py;
  const T cx = P.cx, cy = P.cy;
  T *const yout = P.y;
  const T *const gr = P.r;
  const T *const gd = P.dinv;
  const T *const gW = P.aW;
  const T *const gS = P.aS;
  const T *const gN = P.aN;
  T *const bnd_f = P.bnd_f;
  int *const status = P.status;
  double *const prof = P.prof;
  const int i0 = kLines * k;
  const int nl = min(kLines, nx - i0);
  const bool real = lane >= 1 && lane <= nl;
  const bool has_prod = k > 0;
  const bool lin = (lane == 0) && has_prod;  // the ghost replays the hand-over line
  const int i = i0 + lane - 1;
  constexpr int na = VAR ? 4 : 2;
  T *ring_r = (T *)smem_warp;
  T *ring_d = ring_r + 32 * kPitch;
  T *ring_w = ring_d + 32 * kPitch;
  T *ring_s = ring_w + 32 * kPitch;
  T *bline = ring_r + sweep_hand_line(na);  // forward hand-over line (line i0-1), written by the producer
  T *zrow = bline + 2 * ((ny + 3) & ~3);
  T *ones = zrow + kPitch;
  // Periodic x (nsweep >= 2): row (nx-1, j) also subtracts aE(nx-1, j) w(0, j).  Line 0 (lane 1 of warp 0)
  // stores w into the global wrap line; the last warp's lanes 16..31 land it, one group ahead, into a
  // shared line (with the coefficients beside it), from which the lane of line nx-1 reads at fixed offsets.
  T *const xline = ones + kPitch + kWrapPad;
  T *const xcoef = xline + wrap_line_stride(ny);
  const bool wprod = PX && k == 0 && lane == 1;
  const bool wcons = PX && k == nsweep - 1;
  const int wl = nx - i0;  // lane of line nx-1 in the last warp
  const bool wlane = wcons && lane == wl;
  T *const wbuf = PX ? P.wline0 + (size_t)(epoch & 1u) * ny : nullptr;
  const bool vec16 = (ny % (16 / (int)sizeof(T))) == 0;  // 16-byte pieces
  const bool prod_local = has_prod && (ws > 0);
  const bool has_cons = (k + 1 < nsweep);
  const bool cons_local = has_cons && (ws + 1 < sw);
  const int total = ny + nl;
  const int nchunk = (total + kChunk - 1) / kChunk;
  const T empty = hand_empty_value<T>();
  // per-lane rows: real lanes their ring rows, the ghost unit dinv, everything else zeros
  const T *r_row = real ? ring_r + lane * kPitch : zrow;
  const T *d_row = real ? ring_d + lane * kPitch : (lin ? ones : zrow);
  const T *w_row = real ? ring_w + lane * kPitch : zrow;
  const T *s_row = real ? ring_s + lane * kPitch : zrow;
  const T m_lane = real ? (T)m_r : T(0);
  const T as_c = real ? cy : T(0);
  const T aw_c = (real && i > 0) ? cx : T(0);
  T *const ydst = yout + (size_t)(real ? i : 0) * ny;
  const bool hand = has_cons && lane == 31;  // a warp with a consumer has nl = 31
  T *const hdst = cons_local ? (T *)(smem_warp + P.warp_smem) + sweep_hand_line(na)
                                  : bnd_f + ((size_t)(epoch & 1u) * nsweep + k) * ny;
  auto stage = [&](int c) {
    const int c0 = c * kChunk;
    if (c0 < ny) {
      if (vec16 && c0 + kChunk <= ny) {
        stage_full<true, na, T>(ring_r, ring_d, ring_w, ring_s, gr, gd, gW, gS, i0, 1, nl, ny, c0);
      } else {
        stage_cols<true, T>(ring_r, gr, i0, 1, nl, ny, c0, c0 + kChunk, vec16);
        stage_cols<true, T>(ring_d, gd, i0, 1, nl, ny, c0, c0 + kChunk, vec16);
        if (VAR) {
          stage_cols<true, T>(ring_w, gW, i0, 1, nl, ny, c0, c0 + kChunk, vec16);
          stage_cols<true, T>(ring_s, gS, i0, 1, nl, ny, c0, c0 + kChunk, vec16);
        }
      }
    }
    cp_async_commit();
  };
  const unsigned long long t_begin = global_ns();
  unsigned long long t_wait = 0;
  for (int t = lane; t < kPitch; t += 32) {
    zrow[t] = T(0);
    ones[t] = T(1);
  }
  // A producer in another CTA hands its line over through global memory: the values of group c are loaded
  // kAhead groups early (issued at the start of a group, landed in the shared line at its end).
  const bool remote = has_prod && !prod_local;
  T *const hin = has_prod ? bnd_f + ((size_t)(epoch & 1u) * nsweep + (k - 1)) * ny : nullptr;
  auto hand_issue = [&](int c) -> T {
    const int col = c * kChunk + lane;
    return (lane < kHand && col < ny) ? ld_relaxed_gpu(hin + col) : T(0);
  };
  auto hand_land = [&](int c, T v) -> bool {
    const int col = c * kChunk + lane;
    const bool mine = lane < kHand && col < ny;
    bool miss = mine && hand_empty(v);
    if (__any_sync(0xffffffffu, miss)) {
      const unsigned long long tw0 = global_ns();
      long long spins = 0;
      while (__any_sync(0xffffffffu, miss)) {
        ++spins;
        if (spins > spin_limit(status) || ((spins & 1023) == 0 && *(volatile int *)status != kDevOk)) {
          if (lane == 0) atomicCAS(status, kDevOk, kDevTimeout);
          return false;
        }
        if (spins > 32) __nanosleep(64);
        if (miss) {
          v = ld_relaxed_gpu(hin + col);
          miss = hand_empty(v);
        }
      }
      t_wait += global_ns() - tw0;
    }
    if (mine) {
      bline[col] = v;
      hin[col] = hand_empty_value<T>();
    }
    __syncwarp();
    return true;
  };
  auto wrap_col = [&](int c) { return c * kChunk - wl + (lane - 16); };
  auto wrap_issue = [&](int c, T &cf) -> T {
    const int col = wrap_col(c);
    const bool mine = lane >= 16 && col >= 0 && col < ny;
    cf = (VAR && mine) ? P.aE[(size_t)(nx - 1) * ny + col] : T(0);
    return mine ? ld_relaxed_gpu(wbuf + col) : T(0);
  };
  auto wrap_land = [&](int c, T v, T cf) -> bool {
    const int col = wrap_col(c);
    const bool mine = lane >= 16 && col >= 0 && col < ny;
    if (!poll_line(wbuf, col, mine, v, status, t_wait)) return false;
    if (mine) {
      xline[col] = v;
      if (VAR) xcoef[col] = cf;
      wbuf[col] = hand_empty_value<T>();
    }
    __syncwarp();
    return true;
  };
  for (int c = 0; c < kAhead; ++c) {
    if (remote && !hand_land(c, hand_issue(c))) {
      cp_async_wait0();
      return;
    }
    if (wcons) {
      T cf;
      const T v = wrap_issue(c, cf);
      if (!wrap_land(c, v, cf)) {
        cp_async_wait0();
        return;
      }
    }
    stage(c);
  }
  T w_prev = T(0), w_first = T(0);
  double rz = 0.0, rsum = 0.0;  // r.z and sum r accumulate in double
  for (int q = 0; q < nchunk; ++q) {
    stage(q + kAhead);
    const T hv = remote ? hand_issue(q + kAhead) : T(0);
    T xcf = T(0);
    const T xv = wcons ? wrap_issue(q + kAhead, xcf) : T(0);
    cp_async_wait_ahead();
    __syncwarp();
    const int s0 = q * kChunk;
    const int hcol = (lane < kHand && s0 + lane < ny) ? s0 + lane : -1;  // this group's hand-over columns
    if (prod_local && s0 < ny && !wait_local_line(bline, hcol, status, t_wait)) {
      cp_async_wait0();
      return;
    }
    if (s0 >= 32 && s0 + kHand < ny) {
      // steady state: every lane's column lies in [1, ny-2]; fixed offsets from one base per array
      const int j0 = s0 - lane;
      const int slot = j0 & (kRing - 1);
      const T *rb = lin ? bline + j0 : r_row + slot;
      const T *db = d_row + slot;
      const T *wb = w_row + slot;
      const T *sb = s_row + slot;
      T *yp = ydst + j0;
      T *hp = hdst + j0;
      T rvv[kHand], dvv[kHand], asv[kHand], awv[kHand], xvv[PX ? kHand : 1], xcv[PX ? kHand : 1];
#pragma unroll
      for (int ss = 0; ss < kHand; ++ss) {
        rvv[ss] = rb[ss];
        dvv[ss] = db[ss];
        asv[ss] = VAR ? sb[ss] : as_c;
        awv[ss] = VAR ? wb[ss] : aw_c;
      }
      if constexpr (PX) {
        const T *xb = wlane ? xline + j0 : zrow + slot;
        const T *xc = wlane ? xcoef + j0 : zrow + slot;
        const T ae_w = wlane ? cx : T(0);
#pragma unroll
        for (int ss = 0; ss < kHand; ++ss) {
          xvv[ss] = xb[ss];
          xcv[ss] = VAR ? xc[ss] : ae_w;
        }
      }
#pragma unroll
      for (int ss = 0; ss < kHand; ++ss) {
        const T rv = rvv[ss] - m_lane;
        const T dv = dvv[ss];
        const T as = asv[ss];
        const T aw = awv[ss];
        T t0 = rv;
        if constexpr (PX) t0 = fma(-xcv[ss], xvv[ss], t0);  // wrap (0, j): the smallest column of row (nx-1, j)
        const T t1 = fma(-as, w_prev, t0);
        const T w_up = __shfl_up_sync(0xffffffffu, w_prev, 1);
        const T sum = fma(-aw, w_up, t1);
        const T yv = ICC ? sum * dv : sum;
        const T wv = sum * (ICC ? dv * dv : dv);
        st_global_if(yp + ss, yv, real);
        rz = fma((double)yv, (double)(ICC ? yv : wv), rz);
        rsum += rv;
        st_generic_if(hp + ss, wv, hand);
        if constexpr (PX) st_global_if(wbuf + j0 + ss, wv, wprod);
        w_prev = wv;
      }
    } else {
      // ramp-up / ramp-down group (some lane's column outside [0, ny), or the periodic-y wrap column):
      // the steady arithmetic, with the carried state, the stores and the sums gated by the column range
      const int j0 = s0 - lane;
      const int slot = j0 & (kRing - 1);
      const T *rb = lin ? bline + j0 : r_row + slot;
      const T *db = d_row + slot;
      const T *wb = w_row + slot;
      const T *sb = s_row + slot;
      T rvv[kHand], dvv[kHand], asv[kHand], awv[kHand];
#pragma unroll
      for (int ss = 0; ss < kHand; ++ss) {
        rvv[ss] = rb[ss];
        dvv[ss] = db[ss];
        asv[ss] = VAR ? sb[ss] : as_c;
        awv[ss] = VAR ? wb[ss] : aw_c;
      }
#pragma unroll
      for (int ss = 0; ss < kHand; ++ss) {
        const int j = j0 + ss;
        const bool act = j >= 0 && j < ny;
        const T rv = rvv[ss] - m_lane;
        const T dv = dvv[ss];
        // own-line terms first (periodic-y wrap, S), so that one FMA follows the shuffle from line i-1; a
        // lane's first active step has w_prev = 0, so the S term vanishes at j = 0
        T t1 = rv;
        if constexpr (PX) {
          if (wlane && act) t1 = fma(-(VAR ? xcoef[j] : cx), xline[j], t1);
        }
        if (py && j == ny - 1 && real) t1 = fma(-(VAR ? gN[(size_t)i * ny + j] : cy), w_first, t1);
        t1 = fma(-asv[ss], w_prev, t1);
        const T w_up = __shfl_up_sync(0xffffffffu, w_prev, 1);
        const T sum = fma(-awv[ss], w_up, t1);
        const T yv = ICC ? sum * dv : sum;
        const T wv = sum * (ICC ? dv * dv : dv);
        st_global_if(ydst + j, yv, act && real);
        rz = (act && real) ? fma((double)yv, (double)(ICC ? yv : wv), rz) : rz;
        rsum = (act && real) ? rsum + rv : rsum;
        st_generic_if(hdst + j, wv, act && hand);
        if constexpr (PX) st_global_if(wbuf + j, wv, act && wprod);
        w_first = (py && j == 0) ? wv : w_first;
        w_prev = act ? wv : w_prev;
      }
    }
    __syncwarp();
    if (prod_local && hcol >= 0) bline[hcol] = empty;  // consumed: back to the sentinel for the next application
    if (remote && !hand_land(q + kAhead, hv)) {
      cp_async_wait0();
      return;
    }
    if (wcons && !wrap_land(q + kAhead, xv, xcf)) {
      cp_async_wait0();
      return;
    }
  }
  cp_async_wait0();
  __syncwarp();
  if (!real) {
    rz = 0.0;
    rsum = 0.0;
  }
  acc[1] += rz;
  acc[2] += rsum;
  if (prof && lane == 0 && k < 16) {
    prof[4 * k + 0] = (double)(global_ns() - t_begin);
    prof[4 * k + 1] = (double)t_wait;
    prof[4 * k + 2] = 0.0;
  }
}

// Backward sweep of sweep warp k.  Lanes 0..nl-1 own lines 31k .. 31k+nl-1; lane 31 is the ghost of line
// 31k+31 when a next warp exists.  The lead lane (the ghost, or the last real lane of the last warp) runs
// first, lane t (lead-t) steps behind it.  Accumulates the sum of z into acc[0].
template <bool ICC, bool VAR, typename T = double, bool PX = false>
__device__ __forceinline__ void bwd5_staged(const Sweep5T<T> &P, char *smem_warp, unsigned int *cnt_cta, int k, int ws,
                                            unsigned int epoch, double (&acc)[3]) {
  const int lane = threadIdx.x & 31;
  const int nx = P.nx, ny = P.ny, nsweep = P.nsweep, sw = P.sw;
  const int py = P.py;
  const T cx = P.cx, cy = P.cy;
  T *const zout = P.z;
  const T *const gy = P.y;
  const T *const gd = P.dinv;
  const T *const gN = P.aN;
  const T *const gE = P.aE;
  const T *const gS = P.aS;
  T *const bnd_b = P.bnd_b;
  int *const status = P.status;
  double *const prof = P.prof;
  const int i0 = kLines * k;
  const int nl = min(kLines, nx - i0);
  const bool has_prod = (k + 1 < nsweep);
  const bool prod_local = has_prod && (ws + 1 < sw);
  const bool has_cons = k > 0;
  const bool cons_local = has_cons && (ws > 0);
  const int lead = has_prod ? 31 : nl - 1;
  const bool real = lane < nl;
  const bool lin = (lane == 31) && has_prod;
  const int skew = lead - lane;  // negative for the idle lanes above the lead of the last warp
  const int i = i0 + lane;
  constexpr int na = VAR ? 4 : 2;
  T *ring_y = (T *)smem_warp;
  T *ring_d = ring_y + 32 * kPitch;
  T *ring_n = ring_d + 32 * kPitch;
  T *ring_e = ring_n + 32 * kPitch;
  T *bline = ring_y + sweep_hand_line(na) + ((ny + 3) & ~3);  // backward hand-over line (line i0+31)
  T *zrow = ring_y + sweep_hand_line(na) + 2 * ((ny + 3) & ~3);
  T *ones = zrow + kPitch;
  // Periodic x (nsweep >= 2): row (0, j) also adds aW(0, j) z(nx-1, j) to its upper sum.  Line nx-1 (the
  // lead lane of the last warp) stores z into the global wrap line; warp 0's lanes 16..31 land it into the
  // shared wrap line (free again: warp 0 is not the forward's wrap consumer), read by lane 0 (line 0).
  T *const xline = ones + kPitch + kWrapPad;
  T *const xcoef = xline + wrap_line_stride(ny);
  const bool zprod = PX && k == nsweep - 1 && lane == nl - 1;
  const bool zcons = PX && k == 0;
  const bool zlane = zcons && lane == 0;
  T *const zbuf = PX ? P.zlast + (size_t)(epoch & 1u) * ny : nullptr;
  unsigned long long t_wrap = 0;
  const bool vec16 = (ny % (16 / (int)sizeof(T))) == 0;  // 16-byte pieces
  const int total = ny + lead;
  const int nchunk = (total + kChunk - 1) / kChunk;
  const T empty = hand_empty_value<T>();
  const T *y_row = real ? ring_y + lane * kPitch : zrow;
  const T *d_row = real ? ring_d + lane * kPitch : (lin ? ones : zrow);
  const T *n_row = real ? ring_n + lane * kPitch : zrow;
  const T *e_row = real ? ring_e + lane * kPitch : zrow;
  const T an_c = real ? cy : T(0);
  const T ae_c = (real && i + 1 < nx) ? cx : T(0);
  T *const zdst = zout + (size_t)(real ? i : 0) * ny;
  const bool hand = has_cons && lane == 0;
  T *const hdst = cons_local ? (T *)(smem_warp - P.warp_smem) + sweep_hand_line(na) + ((ny + 3) & ~3)
                                  : bnd_b + ((size_t)(epoch & 1u) * nsweep + k) * ny;
  auto stage = [&](int c) {
    const int c1 = ny - kChunk * c;
    if (c1 > 0) {
      if (vec16 && (ny % kChunk) == 0) {
        stage_full<false, na, T>(ring_y, ring_d, ring_n, ring_e, gy, gd, gN, gE, i0, 0, nl, ny, c1 - kChunk);
      } else {
        stage_cols<false, T>(ring_y, gy, i0, 0, nl, ny, c1 - kChunk, c1, vec16);
        stage_cols<false, T>(ring_d, gd, i0, 0, nl, ny, c1 - kChunk, c1, vec16);
        if (VAR) {
          stage_cols<false, T>(ring_n, gN, i0, 0, nl, ny, c1 - kChunk, c1, vec16);
          stage_cols<false, T>(ring_e, gE, i0, 0, nl, ny, c1 - kChunk, c1, vec16);
        }
      }
    }
    cp_async_commit();
  };
  __syncwarp();  // y of these lines was written by this warp's forward sweep
  const unsigned long long t_begin = global_ns();
  for (int t = lane; t < kPitch; t += 32) {
    zrow[t] = T(0);
    ones[t] = T(1);
  }
  // a producer in another CTA: values loaded kAhead groups early and polled, as in the forward sweep
  const bool remote = has_prod && !prod_local;
  T *const hin = has_prod ? bnd_b + ((size_t)(epoch & 1u) * nsweep + (k + 1)) * ny : nullptr;
  auto hand_issue = [&](int c) -> T {
    const int col = ny - 1 - (c * kChunk + lane);
    return (lane < kHand && col >= 0) ? ld_relaxed_gpu(hin + col) : T(0);
  };
  auto hand_land = [&](int c, T v) -> bool {
    const int col = ny - 1 - (c * kChunk + lane);
    const bool mine = lane < kHand && col >= 0;
    bool miss = mine && hand_empty(v);
    long long spins = 0;
    while (__any_sync(0xffffffffu, miss)) {
      ++spins;
      if (spins > spin_limit(status) || ((spins & 1023) == 0 && *(volatile int *)status != kDevOk)) {
        if (lane == 0) atomicCAS(status, kDevOk, kDevTimeout);
        return false;
      }
      if (spins > 32) __nanosleep(64);
      if (miss) {
        v = ld_relaxed_gpu(hin + col);
        miss = hand_empty(v);
      }
    }
    if (mine) {
      bline[col] = v;
      hin[col] = hand_empty_value<T>();
    }
    __syncwarp();
    return true;
  };
  // lane 0 (skew `lead`) reads columns ny-1-(c*kChunk-lead)-ss in group c
  auto wrap_col = [&](int c) { return ny - 1 - (c * kChunk - lead) - (lane - 16); };
  auto wrap_issue = [&](int c, T &cf) -> T {
    const int col = wrap_col(c);
    const bool mine = lane >= 16 && col >= 0 && col < ny;
    cf = (VAR && mine) ? P.aW[col] : T(0);
    return mine ? ld_relaxed_gpu(zbuf + col) : T(0);
  };
  auto wrap_land = [&](int c, T v, T cf) -> bool {
    const int col = wrap_col(c);
    const bool mine = lane >= 16 && col >= 0 && col < ny;
    if (!poll_line(zbuf, col, mine, v, status, t_wrap)) return false;
    if (mine) {
      xline[col] = v;
      if (VAR) xcoef[col] = cf;
      zbuf[col] = hand_empty_value<T>();
    }
    __syncwarp();
    return true;
  };
  for (int c = 0; c < kAhead; ++c) {
    if (remote && !hand_land(c, hand_issue(c))) {
      cp_async_wait0();
      return;
    }
    if (zcons) {
      T cf;
      const T v = wrap_issue(c, cf);
      if (!wrap_land(c, v, cf)) {
        cp_async_wait0();
        return;
      }
    }
    stage(c);
  }
  T z_prev = T(0), z_first = T(0);
  double zsum = 0.0;
  for (int q = 0; q < nchunk; ++q) {
    stage(q + kAhead);
    const T hv = remote ? hand_issue(q + kAhead) : T(0);
    T xcf = T(0);
    const T xv = zcons ? wrap_issue(q + kAhead, xcf) : T(0);
    cp_async_wait_ahead();
    __syncwarp();
    const int s0 = q * kChunk;
    // this group's hand-over columns (line i0+31, columns ny-1-s0 down to ny-kHand-s0)
    const int hcol = (lane < kHand && ny - 1 - (s0 + lane) >= 0) ? ny - 1 - (s0 + lane) : -1;
    unsigned long long t_unused = 0;
    if (prod_local && s0 < ny && !wait_local_line(bline, hcol, status, t_unused)) {
      cp_async_wait0();
      return;
    }
    if (s0 >= 32 && s0 + kHand < ny) {
      // steady state: every real lane's column lies in [1, ny-2]
      const int jt = ny - 1 - (s0 - skew);
      const int slot = jt & (kRing - 1);
      const T *yb = lin ? bline + jt : y_row + kMirror + slot;
      const T *db = d_row + kMirror + slot;
      const T *nb = n_row + kMirror + slot;
      const T *eb = e_row + kMirror + slot;
      T *zp = zdst + jt;
      T *hp = hdst + jt;
      T yvv[kHand], dvv[kHand], anv[kHand], aev[kHand], xvv[PX ? kHand : 1], xcv[PX ? kHand : 1];
#pragma unroll
      for (int ss = 0; ss < kHand; ++ss) {
        yvv[ss] = yb[-ss];
        dvv[ss] = db[-ss];
        anv[ss] = VAR ? nb[-ss] : an_c;
        aev[ss] = VAR ? eb[-ss] : ae_c;
      }
      if constexpr (PX) {
        const T *xb = zlane ? xline + jt : zrow + kMirror + slot;
        const T *xc = zlane ? xcoef + jt : zrow + kMirror + slot;
        const T aw_w = zlane ? cx : T(0);
#pragma unroll
        for (int ss = 0; ss < kHand; ++ss) {
          xvv[ss] = xb[-ss];
          xcv[ss] = VAR ? xc[-ss] : aw_w;
        }
      }
#pragma unroll
      for (int ss = 0; ss < kHand; ++ss) {
        const T yv = yvv[ss];
        const T dv = dvv[ss];
        const T an = anv[ss];
        const T ae = aev[ss];
        T t = an * z_prev;
        if constexpr (PX) t = fma(xcv[ss], xvv[ss], t);  // wrap (nx-1, j) of row (0, j)
        const T z_dn = __shfl_down_sync(0xffffffffu, z_prev, 1);
        const T zv = ICC ? fma(-(dv * dv), fma(ae, z_dn, t), yv * dv) : dv * (yv - fma(ae, z_dn, t));
        st_global_if(zp - ss, zv, real);
        zsum += zv;
        st_generic_if(hp - ss, zv, hand);
        if constexpr (PX) st_global_if(zbuf + jt - ss, zv, zprod);
        z_prev = zv;
      }
    } else {
      // ramp-up / ramp-down group: the steady arithmetic with the state, stores and sums gated by the
      // column range; a lane's first active step has z_prev = 0, so the N term vanishes at j = ny-1
      const int jt = ny - 1 - (s0 - skew);
      const int slot = jt & (kRing - 1);
      const T *yb = lin ? bline + jt : y_row + kMirror + slot;
      const T *db = d_row + kMirror + slot;
      const T *nb = n_row + kMirror + slot;
      const T *eb = e_row + kMirror + slot;
      T yvv[kHand], dvv[kHand], anv[kHand], aev[kHand];
#pragma unroll
      for (int ss = 0; ss < kHand; ++ss) {
        yvv[ss] = yb[-ss];
        dvv[ss] = db[-ss];
        anv[ss] = VAR ? nb[-ss] : an_c;
        aev[ss] = VAR ? eb[-ss] : ae_c;
      }
#pragma unroll
      for (int ss = 0; ss < kHand; ++ss) {
        const int j = jt - ss;
        const bool act = j >= 0 && j < ny;
        const T yv = yvv[ss];
        const T dv = dvv[ss];
        const T ae = aev[ss];
        // upper neighbours in ascending column order: (i,j+1), (i,ny-1) [j==0], (i+1,j); own-line terms
        // first, one FMA (plus the final scaling) follows the shuffle from line i+1
        T t = anv[ss] * z_prev;
        if (py && j == 0 && real) t = fma(VAR ? gS[(size_t)i * ny] : cy, z_first, t);
        if constexpr (PX) {
          if (zlane && act) t = fma(VAR ? xcoef[j] : cx, xline[j], t);
        }
        const T z_dn = __shfl_down_sync(0xffffffffu, z_prev, 1);
        // ICC: z = (y - d t) d = y d - d^2 t ; ILDLT: z = D^-1 (y - t)
        const T zv = ICC ? fma(-(dv * dv), fma(ae, z_dn, t), yv * dv) : dv * (yv - fma(ae, z_dn, t));
        st_global_if(zdst + j, zv, act && real);
        zsum = (act && real) ? zsum + zv : zsum;
        st_generic_if(hdst + j, zv, act && hand);
        if constexpr (PX) st_global_if(zbuf + j, zv, act && zprod);
        z_first = (py && j == ny - 1) ? zv : z_first;
        z_prev = act ? zv : z_prev;
      }
    }
    __syncwarp();
    if (prod_local && hcol >= 0) bline[hcol] = empty;  // consumed: back to the sentinel
    if (remote && !hand_land(q + kAhead, hv)) {
      cp_async_wait0();
      return;
    }
    if (zcons && !wrap_land(q + kAhead, xv, xcf)) {
      cp_async_wait0();
      return;
    }
  }
  cp_async_wait0();
  __syncwarp();
  if (!real) zsum = 0.0;
  acc[0] += zsum;
  if (prof && lane == 0 && k < 16) prof[4 * k + 3] = (double)(global_ns() - t_begin);
}

}  // namespace dn
