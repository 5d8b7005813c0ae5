// dn_krylov.cuh -- sparse operators, incomplete factorizations and the persistent PCG / BiCGSTAB kernels.
//
// Matrices are stored by stencil slot: a[s*n + r] is the coefficient of row r (= i*ny + j) at the slot's
// offset, with periodic wrap; 0 means "absent" (the reference drops |a| < 1e-18 entries,
// ch_sparse_krylov.hpp:116).  The 5-point slots are W,S,C,N,E; the 13-point slots are the offsets of
// L^2 in lexicographic (di, dj) order, so that for interior rows slot order equals the reference's CSR
// column order and slot s mirrors to slot S-1-s.
//
// The PCG kernel is persistent: one cooperative launch runs the whole solve (all iterations) with bounded
// grid barriers between phases.  The ICC(0)/ILDLT(0) triangular solves of the 5-point pressure operator
// run as a register/shuffle-pipelined anti-diagonal wavefront: lane t of a sweep warp owns x-line
// i = 32k + t and marches along j; the value of line i-1 arrives from lane t-1 by warp shuffle one step
// earlier, and across warps through the y array plus a monotonic progress flag.  This applies exactly the
// reference's incomplete factors (same preconditioner, same iteration counts up to round-off).
#pragma once

#include "dn_common.cuh"
#include "dn_wavefront.cuh"

namespace dn {

// ---------------------------------------------------------------------------------------------------
// Stencils
// ---------------------------------------------------------------------------------------------------
template <int S>
struct Stencil;
template <>
struct Stencil<5> {
  static constexpr int n = 5;
  static constexpr int center = 2;
  __host__ __device__ static constexpr int di(int s) { return s == 0 ? -1 : (s == 4 ? 1 : 0); }
  __host__ __device__ static constexpr int dj(int s) { return s == 1 ? -1 : (s == 3 ? 1 : 0); }
};
template <>
struct Stencil<13> {
  static constexpr int n = 13;
  static constexpr int center = 6;
  __host__ __device__ static constexpr int di(int s) {
    return s == 0 ? -2 : (s <= 3 ? -1 : (s <= 8 ? 0 : (s <= 11 ? 1 : 2)));
  }
  __host__ __device__ static constexpr int dj(int s) {
    return s == 0 ? 0 : (s <= 3 ? s - 2 : (s <= 8 ? s - 6 : (s <= 11 ? s - 10 : 0)));
  }
};

// Column of slot s in row (i, j), or -1 when the neighbour lies outside a non-periodic boundary.
template <int S>
__device__ __forceinline__ long long slot_col(int i, int j, int s, int nx, int ny, int px, int py) {
  int ii = i + Stencil<S>::di(s), jj = j + Stencil<S>::dj(s);
  if (ii < 0 || ii >= nx) {
    if (!px) return -1;
    ii = (ii + nx) % nx;
  }
  if (jj < 0 || jj >= ny) {
    if (!py) return -1;
    jj = (jj + ny) % ny;
  }
  return (long long)ii * ny + jj;
}

template <typename T>
struct SpOpT {
  const T *a;  // [S][n]
  int n, nx, ny, px, py;
};
using SpOp = SpOpT<double>;

template <int S, typename T>
__device__ __forceinline__ T spmv_row(const SpOpT<T> &A, const T *x, int i, int j) {
  const long long r = (long long)i * A.ny + j;
  T sum = T(0);
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const T a = A.a[(size_t)s * A.n + r];
    if (a != T(0)) {
      const long long c = slot_col<S>(i, j, s, A.nx, A.ny, A.px, A.py);
      sum += a * x[c];
    }
  }
  return sum;
}

// ---------------------------------------------------------------------------------------------------
// Incomplete factorizations (try_build_incomplete_ldlt / try_build_incomplete_cholesky,
// ch_sparse_krylov.hpp:252-419).  Level-scheduled, one CTA: rows of one level are independent.
//   5-point: level(i, j) = i + j (valid for every periodicity).
//   13-point: level(i, j) = 2i + j when y is not periodic; with periodic y the 13-point dependency graph
//   is a single chain (row (i,0) depends on (i-1,ny-1)), so rows are processed in order.
// ---------------------------------------------------------------------------------------------------
struct Factor {
  double *l;     // [S][n]: L at lower slots, 0 elsewhere
  double *d;     // [n]: d (ICC) or D (LDLT)
  double *dinv;  // [n]: 1 / max(d, floor)
  double floor;
};

template <int S>
__device__ __forceinline__ int num_levels(int nx, int ny, int py) {
  if (S == 5) return nx + ny - 1;
  return py ? nx * ny : 2 * (nx - 1) + ny;
}
template <int S>
__device__ __forceinline__ void level_range(int lev, int nx, int ny, int py, int &i0, int &i1) {
  if (S == 5) {
    i0 = max(0, lev - (ny - 1));
    i1 = min(nx - 1, lev);
  } else if (py) {
    i0 = i1 = -1;
  } else {
    i0 = max(0, (lev - (ny - 1) + 1) / 2);
    i1 = min(nx - 1, lev / 2);
  }
}
template <int S>
__device__ __forceinline__ void level_row(int lev, int i, int ny, int py, int &ri, int &rj) {
  if (S == 13 && py) {
    ri = lev / ny;
    rj = lev % ny;
  } else {
    ri = i;
    rj = (S == 5) ? lev - i : lev - 2 * i;
  }
}

// Sorted lower slots of row (i, j): fills slots[] (ascending column), returns the count.
template <int S>
__device__ __forceinline__ int lower_slots(const SpOp &A, int i, int j, int *slots, long long *cols) {
  const long long r = (long long)i * A.ny + j;
  int cnt = 0;
  for (int s = 0; s < S; ++s) {
    if (fabs(A.a[(size_t)s * A.n + r]) < 1.0e-18) continue;
    const long long c = slot_col<S>(i, j, s, A.nx, A.ny, A.px, A.py);
    if (c < 0 || c >= r) continue;
    int p = cnt++;
    while (p > 0 && cols[p - 1] > c) {
      cols[p] = cols[p - 1];
      slots[p] = slots[p - 1];
      --p;
    }
    cols[p] = c;
    slots[p] = s;
  }
  return cnt;
}

// L value of row c at column k (0 when k is not a lower entry of row c).
template <int S>
__device__ __forceinline__ double find_lower(const SpOp &A, const Factor &F, long long c, long long k) {
  const int ci = (int)(c / A.ny), cj = (int)(c % A.ny);
  for (int s = 0; s < S; ++s) {
    if (slot_col<S>(ci, cj, s, A.nx, A.ny, A.px, A.py) == k) {
      if (fabs(A.a[(size_t)s * A.n + c]) < 1.0e-18 || k >= c) return 0.0;
      return F.l[(size_t)s * A.n + c];
    }
  }
  return 0.0;
}

// kind: 1 = ILDLT, 2 = ICC.  status: set to kDevFactorFailed on a pivot below the floor.
template <int S>
__global__ void k_factor(SpOp A, Factor F, int kind, int *status) {
  __shared__ double shmax[32];
  __shared__ double sh_floor;
  // max |diag| (ch_sparse_krylov.hpp:258-263 / 343-348)
  double m = 0.0;
  for (long long r = threadIdx.x; r < A.n; r += blockDim.x) {
    m = fmax(m, fabs(A.a[(size_t)Stencil<S>::center * A.n + r]));
    for (int s = 0; s < S; ++s) F.l[(size_t)s * A.n + r] = 0.0;
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) shmax[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) mm = fmax(mm, shmax[w]);
    sh_floor = (kind == 2) ? sqrt(fmax(1.0, mm) * 1.0e-12) : fmax(1.0, mm) * 1.0e-12;
  }
  __syncthreads();
  const double floor = sh_floor;
  const double floor_sq = floor * floor;
  const int nlev = num_levels<S>(A.nx, A.ny, A.py);
  const bool seq = (S == 13 && A.py);
  for (int lev = 0; lev < nlev; ++lev) {
    int i0, i1;
    level_range<S>(lev, A.nx, A.ny, A.py, i0, i1);
    if (seq) {
      i0 = 0;
      i1 = 0;
    }
    for (int ii = i0 + (int)threadIdx.x; ii <= i1; ii += blockDim.x) {
      int i, j;
      level_row<S>(lev, ii, A.ny, A.py, i, j);
      const long long r = (long long)i * A.ny + j;
      int slots[S];
      long long cols[S];
      const int cnt = lower_slots<S>(A, i, j, slots, cols);
      for (int p = 0; p < cnt; ++p) {
        const long long c = cols[p];
        double sum = A.a[(size_t)slots[p] * A.n + r];
        for (int q = 0; q < p; ++q) {
          const long long k = cols[q];
          if (k >= c) break;
          const double l_ck = find_lower<S>(A, F, c, k);
          if (l_ck != 0.0) {
            if (kind == 2)
              sum -= F.l[(size_t)slots[q] * A.n + r] * l_ck;
            else
              sum -= F.l[(size_t)slots[q] * A.n + r] * F.d[k] * l_ck;
          }
        }
        const double denom = max_ref(F.d[c], floor);
        F.l[(size_t)slots[p] * A.n + r] = sum / denom;
      }
      double d = A.a[(size_t)Stencil<S>::center * A.n + r];
      for (int p = 0; p < cnt; ++p) {
        const double lv = F.l[(size_t)slots[p] * A.n + r];
        if (kind == 2)
          d -= lv * lv;
        else
          d -= lv * lv * F.d[cols[p]];
      }
      if (kind == 2) {
        if (!isfinite(d) || d <= floor_sq) {
          atomicExch(status, kDevFactorFailed);
          d = floor_sq * 4.0;
        }
        d = sqrt(d);
      } else if (!isfinite(d) || d <= floor) {
        atomicExch(status, kDevFactorFailed);
        d = floor * 2.0;
      }
      F.d[r] = d;
      F.dinv[r] = 1.0 / max_ref(d, floor);
    }
    __syncthreads();
  }
}

// Diagonal preconditioner (build_diagonal_preconditioner, ch_sparse_krylov.hpp:421-432).
template <int S>
__global__ void k_diag_inverse(SpOp A, double *dinv) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= A.n) return;
  dinv[r] = 1.0 / max_ref(fabs(A.a[(size_t)Stencil<S>::center * A.n + r]), 1.0e-30);
}

// ---------------------------------------------------------------------------------------------------
// 13-point factor rows in application order (built once per factorization, used when y is not periodic).
// Per row r and p < K: the lower entries L_rc (ascending c, the reference's CSR order) and the upper
// entries L_cr (ascending c, its lower_transpose order), padded with zeros.  K = 6 (the stencil's lower
// half; built only when no direction is periodic -- wrapped rows would couple to up to 10).  src codes where the
// neighbour's value sits during a level-scheduled sweep: (d << 16) | ci reads the shared ring of the level
// d steps back (forward) or ahead (backward) at line ci; -1 reads the vector in global memory at col.
// ---------------------------------------------------------------------------------------------------
constexpr int kLvlRing = 8;  // levels kept in the shared ring (neighbours are at most 4 levels away)
struct Rows13 {
  double *lval, *uval;  // [K][n]
  int *lcol, *ucol;     // [K][n]
  int *lsrc, *usrc;     // [K][n]
  int k;                // entries per row (6)
};

__device__ __forceinline__ int ring_code(int d, int ci) {
  return (d >= 1 && d < kLvlRing && ci < 65536) ? ((d << 16) | ci) : -1;
}

__global__ void k_rows13(SpOp A, Factor F, Rows13 R) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= A.n) return;
  const int n = A.n, ny = A.ny;
  const int i = (int)(r / ny), j = (int)(r % ny);
  const int lev = 2 * i + j;
  int slots[13];
  long long cols[13];
  const int cnt = lower_slots<13>(A, i, j, slots, cols);
  for (int p = 0; p < R.k; ++p) {
    if (p < cnt) {
      const long long c = cols[p];
      const int ci = (int)(c / ny), cj = (int)(c % ny);
      R.lval[(size_t)p * n + r] = F.l[(size_t)slots[p] * n + r];
      R.lcol[(size_t)p * n + r] = (int)c;
      R.lsrc[(size_t)p * n + r] = ring_code(lev - (2 * ci + cj), ci);
    } else {
      R.lval[(size_t)p * n + r] = 0.0;
      R.lcol[(size_t)p * n + r] = (int)r;
      R.lsrc[(size_t)p * n + r] = -1;
    }
  }
  // upper neighbours c of r with L_cr != 0, ascending c (as apply_levels orders them)
  int ucnt = 0;
  for (int s = 0; s < 13; ++s) {
    const long long c = slot_col<13>(i, j, s, A.nx, A.ny, A.px, A.py);
    if (c <= r) continue;
    const double lcr = F.l[(size_t)(12 - s) * n + c];
    if (lcr == 0.0) continue;
    int p = ucnt++;
    while (p > 0 && cols[p - 1] > c) {
      cols[p] = cols[p - 1];
      slots[p] = slots[p - 1];
      --p;
    }
    cols[p] = c;
    slots[p] = s;
  }
  for (int p = 0; p < R.k; ++p) {
    if (p < ucnt) {
      const long long c = cols[p];
      const int ci = (int)(c / ny), cj = (int)(c % ny);
      R.uval[(size_t)p * n + r] = F.l[(size_t)(12 - slots[p]) * n + c];
      R.ucol[(size_t)p * n + r] = (int)c;
      R.usrc[(size_t)p * n + r] = ring_code((2 * ci + cj) - lev, ci);
    } else {
      R.uval[(size_t)p * n + r] = 0.0;
      R.ucol[(size_t)p * n + r] = (int)r;
      R.usrc[(size_t)p * n + r] = -1;
    }
  }
}

// ---------------------------------------------------------------------------------------------------
// Persistent PCG (solve_preconditioned_cg, ch_sparse_krylov.hpp:515-660)
// ---------------------------------------------------------------------------------------------------
// T is the type of the operator, the factor and the Krylov vectors (double; float for the inner solves of
// the mixed-precision form).  Dot products, norms and the projection means are accumulated in double.
template <typename T>
struct PcgArgsT {
  SpOpT<T> A;
  const T *l;     // factor slots [S][n]
  const T *dinv;  // [n]
  int prec;       // PrecKind
  const T *b;
  T *x, *r, *z, *y, *p0, *p1, *ap;
  int project;  // mean projection of x, r, z, p (pressure null space, pressure.cpp:225-239)
  int max_it;
  double tol;      // relative stopping tolerance
  double tol_abs;  // absolute stopping tolerance (the reference uses tol for both; 0 disables it)
  // synchronisation
  unsigned int *bar_count;
  unsigned int *bar_gen;
  int *status;
  unsigned int *prog_f, *prog_b;  // per sweep warp progress, monotonic across applications
  double *partials;
  double *out;  // [0] iterations [1] abs residual [2] rel residual [3] iterate residual
  int nsweep;      // sweep warps (ceil(nx/32)) for the 5-point wavefront
  Rows13 rows13;   // ordered factor rows of the 13-point operator (SWEEP 1, y not periodic); lval null: unused
  Sweep5T<T> s5;   // staged wavefront (SWEEP 3)
  int warp_smem;   // shared-memory bytes per sweep warp (SWEEP 3)
  int seq_lines;   // 13-point with periodic y: 1 = line-staged sequential sweeps (seq13 dynamic smem)
  double *mon;     // per-iteration record [iteration][4]: abs residual, rel residual, iterate residual, alpha
  int mon_cap;     // iterations the record holds (0: no record)
};
using PcgArgs = PcgArgsT<double>;

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned int *p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Warp-uniform bounded wait until *flag >= target; returns the observed value (or 0 on timeout).
__device__ __forceinline__ unsigned int wait_flag(const unsigned int *flag, unsigned int target, int *status) {
  unsigned int v = 0;
  const int lane = threadIdx.x & 31;
  long long spins = 0;
  while (true) {
    if (lane == 0) v = ld_acquire(flag);
    v = __shfl_sync(0xffffffffu, v, 0);
    if (v >= target) return v;
    ++spins;
    if (spins > spin_limit(status) || ((spins & 1023) == 0 && *(volatile int *)status != kDevOk)) {
      if (lane == 0) atomicCAS(status, kDevOk, kDevTimeout);
      return 0;
    }
  }
}

constexpr int kPub = 16;  // columns between progress publications of a sweep warp

// Forward sweep of the 5-point factor for sweep warp k.  Reads r (minus the pending mean m_r; when
// projecting, writes the projected residual back), writes y.  ICC: y = (r - sum L y) / d.  LDLT: y = r - sum L y.
template <typename T>
__device__ void fwd5(const PcgArgsT<T> &P, int k, unsigned int epoch, double m_r) {
  const int lane = threadIdx.x & 31;
  const int nx = P.A.nx, ny = P.A.ny, n = P.A.n;
  const int i = 32 * k + lane;
  const bool valid = i < nx;
  const unsigned int base = epoch * (unsigned int)(ny + 1);
  const T *lW = P.l, *lS = P.l + n, *lN = P.l + 3 * (size_t)n, *lE = P.l + 4 * (size_t)n;
  T y_prev = T(0), y_first = T(0), y_step = T(0);
  unsigned int avail = 0;
  for (int s = 0; s < ny + 31; ++s) {
    const int j = s - lane;
    T y_up = __shfl_up_sync(0xffffffffu, y_step, 1);
    if (k > 0 && s < ny) {
      if ((unsigned int)s >= avail) {
        const unsigned int v = wait_flag(&P.prog_f[k - 1], base + (unsigned int)s + 1u, P.status);
        if (v == 0) return;
        avail = v - base;
      }
      if (lane == 0) y_up = __ldcg(&P.y[(size_t)(i - 1) * ny + s]);
    }
    if (valid && j >= 0 && j < ny) {
      const size_t idx = (size_t)i * ny + j;
      const T rv = __ldcg(&P.r[idx]) - (T)m_r;
      T sum = rv;
      if (P.A.px && i == nx - 1) sum -= __ldg(&lE[idx]) * __ldcg(&P.y[j]);
      if (i > 0) sum -= __ldg(&lW[idx]) * y_up;
      if (P.A.py && j == ny - 1) sum -= __ldg(&lN[idx]) * y_first;
      if (j > 0) sum -= __ldg(&lS[idx]) * y_prev;
      const T yv = (P.prec == kPrecICC) ? sum * __ldg(&P.dinv[idx]) : sum;
      P.y[idx] = yv;
      y_prev = yv;
      if (j == 0) y_first = yv;
      y_step = yv;
    }
    const int done = s - 30;  // columns finished by lane 31
    if (done > 0 && (done % kPub == 0 || done == ny)) {
      __syncwarp();
      if (lane == 31) {
        __threadfence();
        st_release(&P.prog_f[k], base + (unsigned int)done);
      }
    }
  }
}

// Backward sweep for sweep warp k (lines nx-1-32k-t, marching j downward).  Accumulates sum z,
// sum r.z and sum r into acc[0..2].  ICC: z = (y - sum L^T z) / d.  LDLT: z = y / D - sum L^T z.
template <typename T>
__device__ void bwd5(const PcgArgsT<T> &P, int k, unsigned int epoch, double m_r, double (&acc)[3]) {
  const int lane = threadIdx.x & 31;
  const int nx = P.A.nx, ny = P.A.ny, n = P.A.n;
  const int i = nx - 1 - (32 * k + lane);
  const bool valid = i >= 0;
  const unsigned int base = epoch * (unsigned int)(ny + 1);
  const T *lW = P.l, *lS = P.l + n, *lN = P.l + 3 * (size_t)n, *lE = P.l + 4 * (size_t)n;
  // the whole forward sweep must be finished (its last warp publishes ny columns last)
  if (k == 0) {
    if (wait_flag(&P.prog_f[P.nsweep - 1], base + (unsigned int)ny, P.status) == 0) return;
  }
  T z_prev = T(0), z_first = T(0), z_step = T(0);
  unsigned int avail = 0;
  for (int s = 0; s < ny + 31; ++s) {
    const int j = ny - 1 - (s - lane);
    T z_dn = __shfl_up_sync(0xffffffffu, z_step, 1);
    if (k > 0 && s < ny) {
      if ((unsigned int)s >= avail) {
        const unsigned int v = wait_flag(&P.prog_b[k - 1], base + (unsigned int)s + 1u, P.status);
        if (v == 0) return;
        avail = v - base;
      }
      if (lane == 0) z_dn = __ldcg(&P.z[(size_t)(i + 1) * ny + (ny - 1 - s)]);
    }
    if (valid && j >= 0 && j < ny) {
      const size_t idx = (size_t)i * ny + j;
      const T yv = __ldcg(&P.y[idx]);
      T sum = (P.prec == kPrecICC) ? yv : yv * __ldg(&P.dinv[idx]);
      if (j + 1 < ny) sum -= __ldg(&lS[idx + 1]) * z_prev;
      if (P.A.py && j == 0) sum -= __ldg(&lN[(size_t)i * ny + ny - 1]) * z_first;
      if (i + 1 < nx) sum -= __ldg(&lW[idx + ny]) * z_dn;
      if (P.A.px && i == 0) {
        const size_t e = (size_t)(nx - 1) * ny + j;
        sum -= __ldg(&lE[e]) * __ldcg(&P.z[e]);
      }
      const T zv = (P.prec == kPrecICC) ? sum * __ldg(&P.dinv[idx]) : sum;
      P.z[idx] = zv;
      z_prev = zv;
      if (j == ny - 1) z_first = zv;
      z_step = zv;
      const T rv = __ldcg(&P.r[idx]) - (T)m_r;
      acc[0] += zv;
      acc[1] += (double)rv * (double)zv;
      acc[2] += rv;
    }
    const int done = s - 30;
    if (done > 0 && (done % kPub == 0 || done == ny)) {
      __syncwarp();
      if (lane == 31) {
        __threadfence();
        st_release(&P.prog_b[k], base + (unsigned int)done);
      }
    }
  }
}

// Level-scheduled forward+backward application of a general slot factor by one CTA (13-point CH
// operator; also handles periodic y, where the 13-point graph is a chain).  Accumulates like bwd5.
template <int S>
__device__ void apply_levels(const PcgArgs &P, double m_r, double (&acc)[3]) {
  const SpOp &A = P.A;
  const int n = A.n;
  const bool seq = (S == 13 && A.py);
  const int nlev = num_levels<S>(A.nx, A.ny, A.py);
  // forward: y_r = r_r - sum_{lower} L y  (ICC divides by d)
  for (int lev = 0; lev < nlev; ++lev) {
    int i0, i1;
    level_range<S>(lev, A.nx, A.ny, A.py, i0, i1);
    if (seq) i0 = i1 = 0;
    for (int ii = i0 + (int)threadIdx.x; ii <= i1; ii += blockDim.x) {
      int i, j;
      level_row<S>(lev, ii, A.ny, A.py, i, j);
      const long long r = (long long)i * A.ny + j;
      int slots[S];
      long long cols[S];
      const int cnt = lower_slots<S>(A, i, j, slots, cols);
      double sum = P.r[r] - m_r;
      for (int p = 0; p < cnt; ++p) sum -= P.l[(size_t)slots[p] * n + r] * P.y[cols[p]];
      P.y[r] = (P.prec == kPrecICC) ? sum * P.dinv[r] : sum;
    }
    if (!seq) __syncthreads();
  }
  __syncthreads();
  // backward: z_r = y_r (/D) - sum_{c > r, L_cr != 0} L_cr z_c, ascending c (lower_transpose order)
  for (int lev = nlev - 1; lev >= 0; --lev) {
    int i0, i1;
    level_range<S>(lev, A.nx, A.ny, A.py, i0, i1);
    if (seq) i0 = i1 = 0;
    for (int ii = i0 + (int)threadIdx.x; ii <= i1; ii += blockDim.x) {
      int i, j;
      level_row<S>(lev, ii, A.ny, A.py, i, j);
      const long long r = (long long)i * A.ny + j;
      // upper neighbours c of r: slot s of r with col c > r; L_cr sits in row c at the mirrored slot
      int slots[S];
      long long cols[S];
      int cnt = 0;
      for (int s = 0; s < S; ++s) {
        const long long c = slot_col<S>(i, j, s, A.nx, A.ny, A.px, A.py);
        if (c <= r) continue;
        const double lcr = P.l[(size_t)(S - 1 - s) * n + c];
        if (lcr == 0.0) continue;
        int p = cnt++;
        while (p > 0 && cols[p - 1] > c) {
          cols[p] = cols[p - 1];
          slots[p] = slots[p - 1];
          --p;
        }
        cols[p] = c;
        slots[p] = s;
      }
      double sum = (P.prec == kPrecICC) ? P.y[r] : P.y[r] * P.dinv[r];
      for (int p = 0; p < cnt; ++p) sum -= P.l[(size_t)(S - 1 - slots[p]) * n + cols[p]] * P.z[cols[p]];
      const double zv = (P.prec == kPrecICC) ? sum * P.dinv[r] : sum;
      P.z[r] = zv;
      const double rv = P.r[r] - m_r;
      acc[0] += zv;
      acc[1] += rv * zv;
      acc[2] += rv;
    }
    if (!seq) __syncthreads();
  }
}

// Level-scheduled forward+backward application of the 13-point factor (y not periodic) by one CTA, from
// the ordered rows (K entries each): the values of the last kLvlRing levels stay in a shared ring (`ring`,
// kLvlRing x nx doubles), so a level reads its neighbours from shared memory; every row does the same six
// multiply-subtract steps, the padded ones subtract exact zeros.  Same arithmetic and order as apply_levels.
//
// Every stored neighbour of this path is at most 4 levels away at a line below 65536 (the ring is built
// only then), so it sits in the ring; the entries with src < 0 are the zero padding, whose column is the
// row itself, and they read the row's own vector entry as it stands before the row is written.
//
// The per-level chain is a memory round trip for the row's coefficients, then the ring reads, the six
// steps and a barrier.  Each thread therefore issues the loads of its first row of level l + 1 (which no
// thread writes before that level) before it computes level l, so the round trip overlaps level l's
// compute and barrier; further rows of a wide level are loaded as they come.
template <int K>
struct LevelRow {
  long long r;   // row index, or -1: the thread has no row at that level
  double v[K];   // lval / uval
  int src[K];    // lsrc / usrc
  double self;   // y[r] (forward) / z[r] (backward): the padding's value
  double a, b;   // forward: r[r], dinv[r];  backward: y[r], dinv[r]
};

template <int K, bool FWD>
__device__ __forceinline__ void load_level_row(const PcgArgs &P, int lev, int i, LevelRow<K> &q) {
  const int n = P.A.n, ny = P.A.ny;
  const Rows13 &R = P.rows13;
  const long long r = (long long)i * ny + (lev - 2 * i);
  q.r = r;
#pragma unroll
  for (int p = 0; p < K; ++p) {
    q.v[p] = FWD ? R.lval[(size_t)p * n + r] : R.uval[(size_t)p * n + r];
    q.src[p] = FWD ? R.lsrc[(size_t)p * n + r] : R.usrc[(size_t)p * n + r];
  }
  q.self = FWD ? P.y[r] : P.z[r];
  q.a = FWD ? P.r[r] : P.y[r];
  q.b = P.dinv[r];
}

template <int K, bool FWD>
__device__ __forceinline__ void level_row_of(const PcgArgs &P, int lev, int first, LevelRow<K> &q) {
  const int nx = P.A.nx, ny = P.A.ny;
  const int i0 = max(0, (lev - (ny - 1) + 1) / 2), i1 = min(nx - 1, lev / 2);
  const int i = i0 + first;
  if (i <= i1)
    load_level_row<K, FWD>(P, lev, i, q);
  else
    q.r = -1;
}

template <int K>
__device__ void apply_levels13_ring(const PcgArgs &P, double m_r, double (&acc)[3], double *ring) {
  const int nx = P.A.nx, ny = P.A.ny;
  const int nlev = 2 * (nx - 1) + ny;
  const bool icc = P.prec == kPrecICC;
  // forward: y = L^-1 (r - m_r), scaled by dinv for ICC
  auto fwd_row = [&](int lev, int i, const LevelRow<K> &q) {
    double yc[K];
#pragma unroll
    for (int p = 0; p < K; ++p) {
      const int src = q.src[p];
      const int off = src >= 0 ? ((lev - (src >> 16)) & (kLvlRing - 1)) * nx + (src & 0xffff) : 0;
      const double from_ring = ring[off];
      yc[p] = src >= 0 ? from_ring : q.self;
    }
    double sum = q.a - m_r;
#pragma unroll
    for (int p = 0; p < K; ++p) sum -= q.v[p] * yc[p];
    const double yv = icc ? sum * q.b : sum;
    P.y[q.r] = yv;
    ring[(lev & (kLvlRing - 1)) * nx + i] = yv;
  };
  LevelRow<K> nxt;
  level_row_of<K, true>(P, 0, threadIdx.x, nxt);
  for (int lev = 0; lev < nlev; ++lev) {
    const int i0 = max(0, (lev - (ny - 1) + 1) / 2), i1 = min(nx - 1, lev / 2);
    const LevelRow<K> cur = nxt;
    if (lev + 1 < nlev) level_row_of<K, true>(P, lev + 1, threadIdx.x, nxt);
    if (cur.r >= 0) fwd_row(lev, i0 + (int)threadIdx.x, cur);
    for (int i = i0 + (int)threadIdx.x + (int)blockDim.x; i <= i1; i += blockDim.x) {
      LevelRow<K> q;
      load_level_row<K, true>(P, lev, i, q);
      fwd_row(lev, i, q);
    }
    __syncthreads();
  }
  // backward: z = L^-T y (ICC: D^-1 scaling of the result; LDLT: of the input)
  auto bwd_row = [&](int lev, int i, const LevelRow<K> &q) {
    double zc[K];
#pragma unroll
    for (int p = 0; p < K; ++p) {
      const int src = q.src[p];
      const int off = src >= 0 ? ((lev + (src >> 16)) & (kLvlRing - 1)) * nx + (src & 0xffff) : 0;
      const double from_ring = ring[off];
      zc[p] = src >= 0 ? from_ring : q.self;
    }
    double sum = icc ? q.a : q.a * q.b;
#pragma unroll
    for (int p = 0; p < K; ++p) sum -= q.v[p] * zc[p];
    const double zv = icc ? sum * q.b : sum;
    P.z[q.r] = zv;
    ring[(lev & (kLvlRing - 1)) * nx + i] = zv;
    const double rv = P.r[q.r] - m_r;
    acc[0] += zv;
    acc[1] += rv * zv;
    acc[2] += rv;
  };
  level_row_of<K, false>(P, nlev - 1, threadIdx.x, nxt);
  for (int lev = nlev - 1; lev >= 0; --lev) {
    const int i0 = max(0, (lev - (ny - 1) + 1) / 2), i1 = min(nx - 1, lev / 2);
    const LevelRow<K> cur = nxt;
    if (lev > 0) level_row_of<K, false>(P, lev - 1, threadIdx.x, nxt);
    if (cur.r >= 0) bwd_row(lev, i0 + (int)threadIdx.x, cur);
    for (int i = i0 + (int)threadIdx.x + (int)blockDim.x; i <= i1; i += blockDim.x) {
      LevelRow<K> q;
      load_level_row<K, false>(P, lev, i, q);
      bwd_row(lev, i, q);
    }
    __syncthreads();
  }
}

// 13-point ILDLT/ICC sweeps with periodic y, where the dependency graph is one chain over all rows in
// natural order.  The chain is only carried along a line: a row's lower neighbours in earlier lines were
// finished with those lines, and in the reference's ascending column order they come before its same-line
// neighbours (its upper neighbours in later lines come after them).  So, per line, all threads of CTA 0
// first gather everything a row needs into shared memory -- its earlier-line sum (forward) or later-line
// products (backward), and the coefficients and offsets of its same-line neighbours -- and thread 0 then
// runs the line's recurrence from shared memory alone, interior rows (2 <= j < ny-2, same-line neighbours
// j-1, j-2 / j+1, j+2) with the previous values in registers.  Every row performs the same operations in the
// same order as apply_levels, so the results are identical.
constexpr int kSeqSame = 4;   // same-line neighbours of a row, at most (wrap rows)
constexpr int kSeqLater = 8;  // later-line upper neighbours of a row, at most (periodic x)
__host__ __device__ constexpr int seq13_smem_doubles_per_row() { return 5 + 2 * kSeqSame + kSeqLater; }

__device__ void apply_seq13(const PcgArgs &P, double m_r, double (&acc)[3], double *sm) {
  constexpr int S = 13;
  const SpOp &A = P.A;
  const int n = A.n, nx = A.nx, ny = A.ny;
  const bool icc = P.prec == kPrecICC;
  double *part = sm;                  // earlier-line sum (forward) / y or y D^-1 (backward)
  double *dv = sm + ny;               // dinv
  double *ln = sm + 2 * ny;           // the current line's y (forward) or z (backward)
  double *ns = sm + 3 * ny;           // number of same-line neighbours (then of later-line products)
  double *sc = sm + 4 * ny;           // [kSeqSame][ny] same-line coefficients, ascending column
  int *so = (int *)(sm + (4 + kSeqSame) * ny);  // [kSeqSame][ny] their columns j'
  double *q = sm + (4 + 2 * kSeqSame) * ny;     // [kSeqLater][ny] backward: later-line products, ascending column
  double *rr = sm + (4 + 2 * kSeqSame + kSeqLater) * ny;  // backward: r of the line
  // ---- forward: y_r = (r_r - m - sum_{lower, ascending} L y) (* dinv for ICC)
  for (int i = 0; i < nx; ++i) {
    const long long base = (long long)i * ny;
    for (int j = threadIdx.x; j < ny; j += blockDim.x) {
      const long long r = base + j;
      int slots[S];
      long long cols[S];
      const int cnt = lower_slots<S>(A, i, j, slots, cols);
      double sum = P.r[r] - m_r;
      int p = 0;
      for (; p < cnt && cols[p] < base; ++p) sum -= P.l[(size_t)slots[p] * n + r] * P.y[cols[p]];
      part[j] = sum;
      int k = 0;
      for (; p < cnt && k < kSeqSame; ++p, ++k) {
        sc[(size_t)k * ny + j] = P.l[(size_t)slots[p] * n + r];
        so[(size_t)k * ny + j] = (int)(cols[p] - base);
      }
      ns[j] = (double)k;
      dv[j] = P.dinv[r];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      auto general = [&](int j) -> double {
        double sum = part[j];
        const int k = (int)ns[j];
        for (int t = 0; t < k; ++t) sum -= sc[(size_t)t * ny + j] * ln[so[(size_t)t * ny + j]];
        const double yv = icc ? sum * dv[j] : sum;
        ln[j] = yv;
        P.y[base + j] = yv;
        return yv;
      };
      double ym2 = general(0);  // y(i, j-2)
      double ym1 = general(1);  // y(i, j-1)
#pragma unroll 4
      for (int j = 2; j < ny - 2; ++j) {
        // same-line neighbours (i, j-2), (i, j-1) in that order; an absent one has coefficient 0 here and
        // is skipped by apply_levels: subtracting 0 * y leaves the sum unchanged
        const int kk = (int)ns[j];
        const double l2 = kk == 2 ? sc[j] : ((kk == 1 && so[j] == j - 2) ? sc[j] : 0.0);
        const double l1 = kk == 2 ? sc[(size_t)ny + j] : ((kk == 1 && so[j] == j - 1) ? sc[j] : 0.0);
        double sum = part[j];
        sum -= l2 * ym2;
        sum -= l1 * ym1;
        const double yv = icc ? sum * dv[j] : sum;
        ln[j] = yv;
        P.y[base + j] = yv;
        ym2 = ym1;
        ym1 = yv;
      }
      general(ny - 2);
      general(ny - 1);
    }
    __syncthreads();
  }
  // ---- backward: z_r = y_r (/D) - sum_{c > r ascending} L_cr z_c (* dinv for ICC); rows in descending order
  for (int i = nx - 1; i >= 0; --i) {
    const long long base = (long long)i * ny;
    for (int j = threadIdx.x; j < ny; j += blockDim.x) {
      const long long r = base + j;
      int slots[S];
      long long cols[S];
      int cnt = 0;
      for (int s = 0; s < S; ++s) {
        const long long c = slot_col<S>(i, j, s, A.nx, A.ny, A.px, A.py);
        if (c <= r) continue;
        if (P.l[(size_t)(S - 1 - s) * n + c] == 0.0) continue;
        int p = cnt++;
        while (p > 0 && cols[p - 1] > c) {
          cols[p] = cols[p - 1];
          slots[p] = slots[p - 1];
          --p;
        }
        cols[p] = c;
        slots[p] = s;
      }
      int p = 0, k = 0;
      for (; p < cnt && cols[p] < base + ny && k < kSeqSame; ++p, ++k) {
        sc[(size_t)k * ny + j] = P.l[(size_t)(S - 1 - slots[p]) * n + cols[p]];
        so[(size_t)k * ny + j] = (int)(cols[p] - base);
      }
      int t = 0;
      for (; p < cnt && t < kSeqLater; ++p, ++t)
        q[(size_t)t * ny + j] = P.l[(size_t)(S - 1 - slots[p]) * n + cols[p]] * P.z[cols[p]];
      ns[j] = (double)(k + 16 * t);  // same-line count + 16 x later-line count
      part[j] = icc ? P.y[r] : P.y[r] * P.dinv[r];
      dv[j] = P.dinv[r];
      rr[j] = P.r[r];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double zp1 = 0.0, zp2 = 0.0;  // z(i, j+1), z(i, j+2)
      for (int j = ny - 1; j >= 0; --j) {
        const int code = (int)ns[j];
        const int k = code & 15, t = code >> 4;
        double sum = part[j];
        if (j >= 2 && j < ny - 2) {
          // same-line neighbours (i, j+1), (i, j+2) in that order (coefficient 0 when absent)
          const double e1 = (k >= 1 && so[j] == j + 1) ? sc[j] : 0.0;
          const double e2 = (k == 2) ? sc[(size_t)ny + j] : ((k == 1 && so[j] == j + 2) ? sc[j] : 0.0);
          sum -= e1 * zp1;
          sum -= e2 * zp2;
        } else {
          for (int u = 0; u < k; ++u) sum -= sc[(size_t)u * ny + j] * ln[so[(size_t)u * ny + j]];
        }
        for (int u = 0; u < t; ++u) sum -= q[(size_t)u * ny + j];
        const double zv = icc ? sum * dv[j] : sum;
        ln[j] = zv;
        const long long r = base + j;
        P.z[r] = zv;
        const double rv = rr[j] - m_r;
        acc[0] += zv;
        acc[1] += rv * zv;
        acc[2] += rv;
        zp2 = zp1;
        zp1 = zv;
      }
    }
    __syncthreads();
  }
}

// One persistent launch runs the whole PCG.  SWEEP: 0 = 5-point pipelined wavefront on global memory,
// 1 = level-scheduled slot factor (CTA 0), 2 = diagonal, 3 = 5-point wavefront staged through shared memory,
// 4 = the staged wavefront with the periodic-x wrap terms (nx >= 32).
// The residual r is kept unprojected in memory; the mean of the latest update (m_r) is subtracted on the
// fly by the preconditioner and folded in by the next update, which equals projecting r after every
// update (pressure.cpp:225-239 applied in ch_sparse_krylov.hpp:602-605).
constexpr int kRowsInFlight = 2;  // rows per thread whose loads the SpMV and update phases issue together

// P1 rows of one thread: p = z - m_z + beta p_old, Ap, and the sums (sum p, p.Ap, sum Ap).  kRowsInFlight rows
// at a time: their loads are issued before any of their stores, so the memory system has that many rows in
// flight per thread (the kernel runs one 256-thread CTA per SM); the sums still run over the thread's rows
// in increasing order.
template <int S, typename T>
__device__ __forceinline__ void pcg_spmv_rows(const PcgArgsT<T> &P, long long lo, long long hi, bool first, T m_z_t,
                                           T beta_t, const T *p_old, T *p_new, double (&v)[3]) {
  const SpOpT<T> &A = P.A;
  const int n = A.n, ny = A.ny;
  for (long long r0 = lo + threadIdx.x; r0 < hi; r0 += (long long)kRowsInFlight * blockDim.x) {
    T prv[kRowsInFlight], apvv[kRowsInFlight];
#pragma unroll
    for (int q = 0; q < kRowsInFlight; ++q) {
      const long long r = r0 + (long long)q * blockDim.x;
      prv[q] = T(0);
      apvv[q] = T(0);
      if (r < hi) {
        const int ri = (int)r, i = ri / ny, j = ri - i * ny;
        T apv = T(0);
#pragma unroll
        for (int s = 0; s < S; ++s) {
          const T a = A.a[(size_t)s * n + r];
          if (a != T(0)) {
            const long long c = slot_col<S>(i, j, s, A.nx, A.ny, A.px, A.py);
            const T pc = first ? (P.z[c] - m_z_t) : (P.z[c] - m_z_t) + beta_t * p_old[c];
            apv += a * pc;
          }
        }
        prv[q] = first ? (P.z[r] - m_z_t) : (P.z[r] - m_z_t) + beta_t * p_old[r];
        apvv[q] = apv;
      }
    }
#pragma unroll
    for (int q = 0; q < kRowsInFlight; ++q) {
      const long long r = r0 + (long long)q * blockDim.x;
      if (r < hi) {
        p_new[r] = prv[q];
        P.ap[r] = apvv[q];
        const double prd = prv[q], apd = apvv[q];
        v[0] += prd;
        v[1] += prd * apd;
        v[2] += apd;
      }
    }
  }
}

// P2 rows of one thread: p -= m_p, x += alpha p, r -= alpha Ap, and the sums for the norms; rows in flight
// as in pcg_spmv_rows.
template <typename T>
__device__ __forceinline__ void pcg_update_rows(const PcgArgsT<T> &P, long long lo, long long hi, T m_p_t, T alpha_t,
                                             T m_x_t, T m_r_t, T *p_new, double (&w)[5]) {
  for (long long r0 = lo + threadIdx.x; r0 < hi; r0 += (long long)kRowsInFlight * blockDim.x) {
    T ppv[kRowsInFlight], xvv[kRowsInFlight], rvv[kRowsInFlight], dv[kRowsInFlight];
#pragma unroll
    for (int q = 0; q < kRowsInFlight; ++q) {
      const long long r = r0 + (long long)q * blockDim.x;
      if (r < hi) {
        const T pp = p_new[r] - m_p_t;
        const T delta = alpha_t * pp;
        ppv[q] = pp;
        dv[q] = delta;
        xvv[q] = (P.x[r] - m_x_t) + delta;
        rvv[q] = (P.r[r] - m_r_t) - alpha_t * P.ap[r];
      }
    }
#pragma unroll
    for (int q = 0; q < kRowsInFlight; ++q) {
      const long long r = r0 + (long long)q * blockDim.x;
      if (r < hi) {
        p_new[r] = ppv[q];
        P.x[r] = xvv[q];
        P.r[r] = rvv[q];
        const double dd = dv[q], xd = xvv[q], rd = rvv[q];
        w[0] += dd * dd;
        w[1] += xd * xd;
        w[2] += xd;
        w[3] += rd;
        w[4] += rd * rd;
      }
    }
  }
}

template <int S, int SWEEP, typename T = double>
__global__ void __launch_bounds__(kBlock) k_pcg(PcgArgsT<T> P) {
  __shared__ double sh[8 * 32 + 8];
  extern __shared__ __align__(16) char dsm[];
  const GridBarrier bar{P.bar_count, P.bar_gen, P.status, gridDim.x};
  int parity = 0;
  const SpOpT<T> &A = P.A;
  const int n = A.n, ny = A.ny;
  const double dn_ = (double)n;
  const long long per = (n + gridDim.x - 1) / gridDim.x;
  const long long lo = (long long)blockIdx.x * per, hi = min((long long)n, lo + per);
  const int warp = threadIdx.x >> 5;
  const int nwarps_cta = blockDim.x >> 5;
  unsigned int *cnt_cta = (unsigned int *)dsm;
  if (SWEEP == 3 || SWEEP == 4) {
    if (threadIdx.x < 16) cnt_cta[threadIdx.x] = 0u;
    // cross-CTA hand-over lines start empty; the first grid reduction orders this before any sweep
    const size_t nb = 2 * (size_t)P.s5.nsweep * P.s5.ny;
    const T empty = hand_empty_value<T>();
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < nb; t += (size_t)gridDim.x * blockDim.x) {
      P.s5.bnd_f[t] = empty;
      P.s5.bnd_b[t] = empty;
    }
    if (SWEEP == 4)  // the periodic-x wrap lines, [2][ny] each
      for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < 2 * (size_t)P.s5.ny;
           t += (size_t)gridDim.x * blockDim.x) {
        P.s5.wline0[t] = empty;
        P.s5.zlast[t] = empty;
      }
    // so do the same-CTA hand-over lines (forward and backward) of this CTA's sweep warps
    const int na = P.s5.varcoef ? 4 : 2;
    const size_t lines = 2 * (size_t)((P.s5.ny + 3) & ~3);
    for (int w = 0; w < P.s5.sw; ++w) {
      T *line = (T *)(dsm + 64 + (size_t)w * P.warp_smem) + sweep_hand_line(na);
      for (size_t t = threadIdx.x; t < lines; t += blockDim.x) line[t] = empty;
    }
    __syncthreads();
  }

  // ---- r = b - A x0, initial residual (ch_sparse_krylov.hpp:531-558)
  double v3[3] = {0.0, 0.0, 0.0};
  for (long long r = lo + threadIdx.x; r < hi; r += blockDim.x) {
    const int i = (int)(r / ny), j = (int)(r % ny);
    const T rr = P.b[r] - spmv_row<S>(A, P.x, i, j);
    P.r[r] = rr;
    const double rd = rr, bd = P.b[r];
    v3[0] += rd;
    v3[1] += rd * rd;
    v3[2] += bd * bd;
  }
  if (!grid_sum<3>(v3, P.partials, parity, sh, bar)) return;
  double m_r = P.project ? v3[0] / dn_ : 0.0;
  double rn2 = P.project ? max_ref(v3[1] - v3[0] * v3[0] / dn_, 0.0) : v3[1];
  const double rhs_norm = sqrt(max_ref(v3[2], 0.0));
  double absr = sqrt(max_ref(rn2, 0.0));
  double relr = absr / max_ref(rhs_norm, 1.0e-30);
  int iterations = 0;
  double iter_res = 0.0;
  if (relr < P.tol || absr < P.tol_abs) {  // x stays x0 (the reference projects r only)
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      P.out[0] = 0;
      P.out[1] = absr;
      P.out[2] = relr;
      P.out[3] = 0.0;
    }
    return;
  }

  unsigned int epoch = 0;
  // acc[0] = sum z, acc[1] = r.z (= r^T M^-1 r), acc[2] = sum of the projected r
  auto precondition = [&](double m_r_now, double (&acc)[3]) -> bool {
    acc[0] = acc[1] = acc[2] = 0.0;
    ++epoch;
    if (SWEEP == 0) {
      for (int k = blockIdx.x + (int)gridDim.x * warp; k < P.nsweep; k += (int)gridDim.x * nwarps_cta)
        fwd5(P, k, epoch, m_r_now);
      for (int k = blockIdx.x + (int)gridDim.x * warp; k < P.nsweep; k += (int)gridDim.x * nwarps_cta)
        bwd5(P, k, epoch, m_r_now, acc);
    } else if (SWEEP == 3 || SWEEP == 4) {
      constexpr bool PX = SWEEP == 4;
      const int k = blockIdx.x * P.s5.sw + warp;
      if (warp < P.s5.sw && k < P.s5.nsweep) {
        char *mine = dsm + 64 + (size_t)warp * P.warp_smem;
        if (P.prec == kPrecICC) {
          if (P.s5.varcoef) {
            fwd5_staged<true, true, T, PX>(P.s5, mine, cnt_cta, k, warp, epoch, m_r_now, acc);
            bwd5_staged<true, true, T, PX>(P.s5, mine, cnt_cta, k, warp, epoch, acc);
          } else {
            fwd5_staged<true, false, T, PX>(P.s5, mine, cnt_cta, k, warp, epoch, m_r_now, acc);
            bwd5_staged<true, false, T, PX>(P.s5, mine, cnt_cta, k, warp, epoch, acc);
          }
        } else {
          if (P.s5.varcoef) {
            fwd5_staged<false, true, T, PX>(P.s5, mine, cnt_cta, k, warp, epoch, m_r_now, acc);
            bwd5_staged<false, true, T, PX>(P.s5, mine, cnt_cta, k, warp, epoch, acc);
          } else {
            fwd5_staged<false, false, T, PX>(P.s5, mine, cnt_cta, k, warp, epoch, m_r_now, acc);
            bwd5_staged<false, false, T, PX>(P.s5, mine, cnt_cta, k, warp, epoch, acc);
          }
        }
      }
    } else if (SWEEP == 1) {
      if constexpr (sizeof(T) == sizeof(double)) {
        if (blockIdx.x == 0) {
          if (S == 13 && P.rows13.lval != nullptr && P.rows13.k == 6)
            apply_levels13_ring<6>(P, m_r_now, acc, (double *)dsm);
          else if (S == 13 && P.seq_lines)
            apply_seq13(P, m_r_now, acc, (double *)dsm);
          else
            apply_levels<S>(P, m_r_now, acc);
        }
      }
    } else {
      const T m = (T)m_r_now;
      for (long long r = lo + threadIdx.x; r < hi; r += blockDim.x) {
        const T rv = P.r[r] - m;
        const T zv = P.dinv[r] * rv;
        P.z[r] = zv;
        acc[0] += zv;
        acc[1] += (double)rv * (double)zv;
        acc[2] += rv;
      }
    }
    return grid_sum<3>(acc, P.partials, parity, sh, bar);
  };

  double acc[3];
  unsigned long long t_p1 = 0, t_p2 = 0, t_pc = 0, t0 = global_ns();
  if (!precondition(m_r, acc)) return;
  t_pc += global_ns() - t0;
  double m_z = P.project ? acc[0] / dn_ : 0.0;
  double rz_old = P.project ? acc[1] - m_z * acc[2] : acc[1];
  if (!isfinite(rz_old) || rz_old <= 0.0) {
    if (threadIdx.x == 0) atomicCAS(P.status, kDevOk, kDevPcgBreakdownRz0);
    return;
  }
  double beta = 0.0;
  double m_x = 0.0;
  T *p_old = P.p0, *p_new = P.p1;
  bool first = true;
  const int limit = P.max_it > 1 ? P.max_it : 1;
  for (int it = 0; it < limit; ++it) {
    // ---- P1: p = z - m_z + beta p_old ; Ap = A p  (p at neighbours formed on the fly)
    t0 = global_ns();
    const T m_z_t = (T)m_z, beta_t = (T)beta;
    double v[3] = {0.0, 0.0, 0.0};
    pcg_spmv_rows<S, T>(P, lo, hi, first, m_z_t, beta_t, p_old, p_new, v);
    if (!grid_sum<3>(v, P.partials, parity, sh, bar)) return;
    const double m_p = P.project ? v[0] / dn_ : 0.0;
    const double pap = P.project ? v[1] - m_p * v[2] : v[1];
    if (!isfinite(pap) || fabs(pap) < 1.0e-30) {
      if (threadIdx.x == 0) atomicCAS(P.status, kDevOk, kDevPcgBreakdownPap);
      return;
    }
    const double alpha = rz_old / pap;
    const unsigned long long t1 = global_ns();
    t_p1 += t1 - t0;
    // ---- P2: x += alpha p ; r -= alpha Ap ; norms (ch_sparse_krylov.hpp:592-610)
    const T m_p_t = (T)m_p, alpha_t = (T)alpha, m_x_t = (T)m_x, m_r_t = (T)m_r;
    double w[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    pcg_update_rows<T>(P, lo, hi, m_p_t, alpha_t, m_x_t, m_r_t, p_new, w);
    if (!grid_sum<5>(w, P.partials, parity, sh, bar)) return;
    const unsigned long long t2 = global_ns();
    t_p2 += t2 - t1;
    m_x = P.project ? w[2] / dn_ : 0.0;
    m_r = P.project ? w[3] / dn_ : 0.0;
    rn2 = P.project ? max_ref(w[4] - w[3] * w[3] / dn_, 0.0) : w[4];
    iterations = it + 1;
    iter_res = sqrt(w[0] / max_ref(w[1], 1.0e-30));
    absr = sqrt(max_ref(rn2, 0.0));
    relr = absr / max_ref(rhs_norm, 1.0e-30);
    if (P.mon && it < P.mon_cap && blockIdx.x == 0 && threadIdx.x == 0) {  // the CG monitor's record
      P.mon[4 * it + 0] = absr;
      P.mon[4 * it + 1] = relr;
      P.mon[4 * it + 2] = iter_res;
      P.mon[4 * it + 3] = alpha;
    }
    if (relr < P.tol || absr < P.tol_abs) break;
    // ---- z = M^{-1} r, project z, r.z (ch_sparse_krylov.hpp:626-635)
    if (!precondition(m_r, acc)) return;
    t_pc += global_ns() - t2;
    m_z = P.project ? acc[0] / dn_ : 0.0;
    const double rz_new = P.project ? acc[1] - m_z * acc[2] : acc[1];
    if (!isfinite(rz_new) || rz_new <= 0.0) {
      if (threadIdx.x == 0) atomicCAS(P.status, kDevOk, kDevPcgBreakdownRz);
      return;
    }
    beta = rz_new / rz_old;
    rz_old = rz_new;
    T *t = p_old;
    p_old = p_new;
    p_new = t;
    first = false;
  }
  // pending projection of x
  if (P.project && m_x != 0.0) {
    const T m_x_t = (T)m_x;
    for (long long r = lo + threadIdx.x; r < hi; r += blockDim.x) P.x[r] = P.x[r] - m_x_t;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    P.out[0] = (double)iterations;
    P.out[1] = absr;
    P.out[2] = relr;
    P.out[3] = iter_res;
    P.out[4] = (double)t_p1 * 1e-6;
    P.out[5] = (double)t_p2 * 1e-6;
    P.out[6] = (double)t_pc * 1e-6;
  }
}

// Equation residual of the CH solve, phase_field.cpp:484-502: partial sums of (b - A x)^2 and b^2.
template <int S>
__global__ void k_residual_partials(SpOp A, const double *b, const double *x, double *partials) {
  __shared__ double sh[8 * 32];
  double v[2] = {0.0, 0.0};
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < A.n; r += (long long)gridDim.x * blockDim.x) {
    const int i = (int)((unsigned)r / (unsigned)A.ny), j = (int)((unsigned)r - (unsigned)i * (unsigned)A.ny);
    const double d = b[r] - spmv_row<S>(A, x, i, j);
    v[0] += d * d;
    v[1] += b[r] * b[r];
  }
  block_sum<2>(v, sh);
  if (threadIdx.x == 0) {
    partials[blockIdx.x * 2] = v[0];
    partials[blockIdx.x * 2 + 1] = v[1];
  }
}

// One application z = M^-1 r of the 5-point ICC/ILDLT preconditioner (apply_preconditioner,
// ch_sparse_krylov.hpp:444-513) on its own, for solvers that need the direction but not the CG recurrence
// (the conjugate-directions backend): the same sweeps as k_pcg<5, SWEEP> (the staged wavefront, with the
// periodic-x wrap for SWEEP 4, or the global-memory wavefront for SWEEP 0) on P.r / P.s5.r, m_r = 0.
// P.out[0..2] receive sum z, r.z and sum r.
template <int SWEEP>
__global__ void __launch_bounds__(kBlock) k_prec_apply(PcgArgs P) {
  __shared__ double sh[8 * 32 + 8];
  extern __shared__ __align__(16) char dsm[];
  const GridBarrier bar{P.bar_count, P.bar_gen, P.status, gridDim.x};
  int parity = 0;
  const int warp = threadIdx.x >> 5;
  const int nwarps_cta = blockDim.x >> 5;
  unsigned int *cnt_cta = (unsigned int *)dsm;
  if (SWEEP == 3 || SWEEP == 4) {
    if (threadIdx.x < 16) cnt_cta[threadIdx.x] = 0u;
    const size_t nb = 2 * (size_t)P.s5.nsweep * P.s5.ny;
    const double empty = hand_empty_value<double>();
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < nb; t += (size_t)gridDim.x * blockDim.x) {
      P.s5.bnd_f[t] = empty;
      P.s5.bnd_b[t] = empty;
    }
    if (SWEEP == 4)
      for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < 2 * (size_t)P.s5.ny;
           t += (size_t)gridDim.x * blockDim.x) {
        P.s5.wline0[t] = empty;
        P.s5.zlast[t] = empty;
      }
    const int na = P.s5.varcoef ? 4 : 2;
    const size_t lines = 2 * (size_t)((P.s5.ny + 3) & ~3);
    for (int w = 0; w < P.s5.sw; ++w) {
      double *line = (double *)(dsm + 64 + (size_t)w * P.warp_smem) + sweep_hand_line(na);
      for (size_t t = threadIdx.x; t < lines; t += blockDim.x) line[t] = empty;
    }
    __syncthreads();
  }
  double acc[3] = {0.0, 0.0, 0.0};
  if (!grid_sum<3>(acc, P.partials, parity, sh, bar)) return;  // orders the set-up before any sweep
  acc[0] = acc[1] = acc[2] = 0.0;
  const unsigned int epoch = 1;
  if (SWEEP == 0) {
    for (int k = blockIdx.x + (int)gridDim.x * warp; k < P.nsweep; k += (int)gridDim.x * nwarps_cta)
      fwd5(P, k, epoch, 0.0);
    for (int k = blockIdx.x + (int)gridDim.x * warp; k < P.nsweep; k += (int)gridDim.x * nwarps_cta)
      bwd5(P, k, epoch, 0.0, acc);
  } else {
    constexpr bool PX = SWEEP == 4;
    const int k = blockIdx.x * P.s5.sw + warp;
    if (warp < P.s5.sw && k < P.s5.nsweep) {
      char *mine = dsm + 64 + (size_t)warp * P.warp_smem;
      if (P.prec == kPrecICC) {
        if (P.s5.varcoef) {
          fwd5_staged<true, true, double, PX>(P.s5, mine, cnt_cta, k, warp, epoch, 0.0, acc);
          bwd5_staged<true, true, double, PX>(P.s5, mine, cnt_cta, k, warp, epoch, acc);
        } else {
          fwd5_staged<true, false, double, PX>(P.s5, mine, cnt_cta, k, warp, epoch, 0.0, acc);
          bwd5_staged<true, false, double, PX>(P.s5, mine, cnt_cta, k, warp, epoch, acc);
        }
      } else {
        if (P.s5.varcoef) {
          fwd5_staged<false, true, double, PX>(P.s5, mine, cnt_cta, k, warp, epoch, 0.0, acc);
          bwd5_staged<false, true, double, PX>(P.s5, mine, cnt_cta, k, warp, epoch, acc);
        } else {
          fwd5_staged<false, false, double, PX>(P.s5, mine, cnt_cta, k, warp, epoch, 0.0, acc);
          bwd5_staged<false, false, double, PX>(P.s5, mine, cnt_cta, k, warp, epoch, acc);
        }
      }
    }
  }
  if (!grid_sum<3>(acc, P.partials, parity, sh, bar)) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    P.out[0] = acc[0];
    P.out[1] = acc[1];
    P.out[2] = acc[2];
  }
}

}  // namespace dn
