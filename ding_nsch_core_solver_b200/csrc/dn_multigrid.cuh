// dn_multigrid.cuh -- the FP32 inner solver of the mixed-precision pressure correction: conjugate gradients
// preconditioned by one geometric multigrid V-cycle.
//
// The mixed form wraps FP32 inner solves of A e = r in an FP64 defect-correction loop that stops on the
// reference's own rule (relative or absolute FP64 residual below pressure_tolerance, the test of
// solve_pressure_correction_*, pressure.cpp:302-365).  The inner preconditioner does not have to be the
// reference's IC(0): the outer loop decides the answer.  ICC/ILDLT triangular solves are one long
// dependency chain across the grid (nx + ny anti-diagonals per sweep), while a V-cycle is a handful of
// fully parallel passes per level, and its iteration count does not grow with the grid.
//
// Hierarchy.  Level 0 is the assembled 5-point operator (k_p_assemble's W,S,C,N,E slots) rounded to FP32.
// Level l+1 halves both extents while both are even, >= 4, and the level has more than kMgCoarseMax cells.
// Its operator is the cell-centred rediscretisation: a coarse face weight is the mean of the two fine face
// weights it covers; the diagonal is the sum of the coarse off-diagonal weights plus half the summed
// boundary excess (diagonal minus off-diagonal sum, non-zero only on Dirichlet sides) of the four children.
// On the coarsest level (<= kMgCoarseMax cells) the operator is inverted exactly in FP64 (Gauss-Jordan on
// the SPD matrix; the pure-Neumann / periodic null space is removed by the rank-one shift A + mean(diag) /
// n * 1 1^T, which leaves the solution of a mean-free right-hand side unchanged) and applied in FP32.
//
// Transfer operators: bilinear cell-centred prolongation P (weights 3/4, 1/4 per direction; across a wall
// the ghost parent mirrors the boundary cell with sign +1 for a Neumann side and -1 for a Dirichlet side;
// periodic directions wrap) and restriction R = P^T.  Smoother: red-black Gauss-Seidel, nu sweeps red-then-
// black before the coarse correction and nu sweeps black-then-red after it, so that the V-cycle is a
// symmetric positive definite operator and the outer iteration is plain CG.  Vectors, operators and the
// SpMV accumulate in FP32; the CG dot products and norms accumulate in FP64.
#pragma once

#include <cooperative_groups.h>

#include "dn_common.cuh"
#include "dn_krylov.cuh"

namespace dn {

constexpr int kMgCoarseMax = 128;  // cells of the directly inverted coarsest level (128^2 doubles of shared memory)
constexpr int kMgMaxLevels = 24;
constexpr int kMgParts = 1024;     // CTAs of the CG vector kernels at most (per-CTA partial sums)
constexpr int kMgSweeps = 2;       // red-black sweeps before and after each coarse correction
constexpr int kMgBottomCells = 8192;  // levels this small run inside the one-CTA bottom kernel

// one level of the hierarchy: operator slots [5][n] (W,S,C,N,E), iterate, right-hand side, residual
struct MgLevel {
  const float *a;
  float *x, *b, *r;
  int nx, ny;
};
// wall folding signs of the bilinear transfer (left, right, bottom, top) and the periodicity
struct MgFold {
  float s[4];
  int px, py;
};

__device__ __forceinline__ float mg_row_sum(const MgLevel &L, const float *x, int i, int j, long long r, long long n,
                                            int px, int py) {
  // sum of the off-diagonal terms a_s * x_nb, FP32 accumulation in slot order
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    if (k == 2) continue;
    const float a = L.a[(size_t)k * n + r];
    if (a != 0.0f) {
      const long long c = slot_col<5>(i, j, k, L.nx, L.ny, px, py);
      if (c >= 0) s += a * x[c];
    }
  }
  return s;
}

// Red-black Gauss-Seidel half sweep at cell t of the colour's cells ((i + j) & 1 == color); ny is even on every
// smoothed level, so each row holds ny/2 cells of each colour.  first: the iterate is zero on entry, so the
// colour's cells take b / diag and the other colour's cells are set to zero.
__device__ __forceinline__ void mg_smooth_at(const MgLevel &L, int color, int first, int px, int py, unsigned t) {
  const int half = L.ny >> 1;
  const int i = (int)(t / (unsigned)half);
  const int j = 2 * (int)(t - (unsigned)i * (unsigned)half) + ((i + color) & 1);
  const long long n = (long long)L.nx * L.ny;
  const long long r = (long long)i * L.ny + j;
  float s = L.b[r];
  if (!first) s -= mg_row_sum(L, L.x, i, j, r, n, px, py);
  L.x[r] = s / L.a[2 * n + r];
  if (first) L.x[(long long)i * L.ny + (j ^ 1)] = 0.0f;
}

// r = b - A x at cell t
__device__ __forceinline__ void mg_residual_at(const MgLevel &L, int px, int py, unsigned t) {
  const unsigned n = (unsigned)L.nx * (unsigned)L.ny;
  const int i = (int)(t / (unsigned)L.ny), j = (int)(t - (unsigned)i * (unsigned)L.ny);
  L.r[t] = L.b[t] - (L.a[2 * (size_t)n + t] * L.x[t] + mg_row_sum(L, L.x, i, j, t, n, px, py));
}

// 1D bilinear weight of coarse index I in the interpolation of fine index i (fine extent 2 * nc)
__device__ __forceinline__ float mg_w1(int i, int I, int nc, int per, float s_lo, float s_hi) {
  const int par = i >> 1;
  int nb = (i & 1) ? par + 1 : par - 1;
  float w = (par == I) ? 0.75f : 0.0f;
  if (nb >= 0 && nb < nc) {
    if (nb == I) w += 0.25f;
  } else if (per) {
    nb = nb < 0 ? nb + nc : nb - nc;
    if (nb == I) w += 0.25f;
  } else if (par == I) {
    w += 0.25f * (nb < 0 ? s_lo : s_hi);
  }
  return w;
}

// coarse b = P^T (fine r) at coarse cell t: the 4 x 4 fine cells whose interpolation it enters
__device__ __forceinline__ void mg_restrict_at(const MgLevel &F, const MgLevel &C, const MgFold &fold, unsigned t) {
  const int I = (int)(t / (unsigned)C.ny), J = (int)(t - (unsigned)I * (unsigned)C.ny);
  float sum = 0.0f;
#pragma unroll
  for (int di = -1; di <= 2; ++di) {
    int i = 2 * I + di;
    if (i < 0 || i >= F.nx) {
      if (!fold.px) continue;
      i = i < 0 ? i + F.nx : i - F.nx;
    }
    const float wx = mg_w1(i, I, C.nx, fold.px, fold.s[0], fold.s[1]);
    if (wx == 0.0f) continue;
    float row = 0.0f;
#pragma unroll
    for (int dj = -1; dj <= 2; ++dj) {
      int j = 2 * J + dj;
      if (j < 0 || j >= F.ny) {
        if (!fold.py) continue;
        j = j < 0 ? j + F.ny : j - F.ny;
      }
      const float wy = mg_w1(j, J, C.ny, fold.py, fold.s[2], fold.s[3]);
      if (wy != 0.0f) row += wy * F.r[(long long)i * F.ny + j];
    }
    sum += wx * row;
  }
  C.b[t] = sum;
}

// fine x += P (coarse x) at fine cell t: its parent and the parents' neighbours toward it
__device__ __forceinline__ void mg_prolong_at(const MgLevel &C, const MgLevel &F, const MgFold &fold, unsigned t) {
  const int i = (int)(t / (unsigned)F.ny), j = (int)(t - (unsigned)i * (unsigned)F.ny);
  int I[2], J[2];
  float wx[2], wy[2];
  I[0] = i >> 1;
  I[1] = (i & 1) ? I[0] + 1 : I[0] - 1;
  wx[0] = 0.75f;
  wx[1] = 0.25f;
  if (I[1] < 0 || I[1] >= C.nx) {
    if (fold.px) {
      I[1] = I[1] < 0 ? I[1] + C.nx : I[1] - C.nx;
    } else {
      wx[0] += 0.25f * (I[1] < 0 ? fold.s[0] : fold.s[1]);
      wx[1] = 0.0f;
      I[1] = I[0];
    }
  }
  J[0] = j >> 1;
  J[1] = (j & 1) ? J[0] + 1 : J[0] - 1;
  wy[0] = 0.75f;
  wy[1] = 0.25f;
  if (J[1] < 0 || J[1] >= C.ny) {
    if (fold.py) {
      J[1] = J[1] < 0 ? J[1] + C.ny : J[1] - C.ny;
    } else {
      wy[0] += 0.25f * (J[1] < 0 ? fold.s[2] : fold.s[3]);
      wy[1] = 0.0f;
      J[1] = J[0];
    }
  }
  float v = 0.0f;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) v += wx[a] * wy[b] * C.x[(long long)I[a] * C.ny + J[b]];
  F.x[t] += v;
}

// one launch per phase on the levels above kMgBottomCells cells
__global__ void k_mg_smooth(MgLevel L, int color, int first, int px, int py) {
  pdl_entry();
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < (unsigned)L.nx * (unsigned)(L.ny >> 1)) mg_smooth_at(L, color, first, px, py, t);
}
__global__ void k_mg_residual(MgLevel L, int px, int py) {
  pdl_entry();
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < (unsigned)L.nx * (unsigned)L.ny) mg_residual_at(L, px, py, t);
}
__global__ void k_mg_restrict(MgLevel F, MgLevel C, MgFold fold) {
  pdl_entry();
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < (unsigned)C.nx * (unsigned)C.ny) mg_restrict_at(F, C, fold, t);
}
__global__ void k_mg_prolong(MgLevel C, MgLevel F, MgFold fold) {
  pdl_entry();
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < (unsigned)F.nx * (unsigned)F.ny) mg_prolong_at(C, F, fold, t);
}

// The bottom of the V-cycle in one CTA: levels first .. last-1 (each at most kMgBottomCells cells) smoothed,
// restricted, the coarsest (last) solved with its inverse, then prolonged and smoothed back up to `first`.
// Phases are separated by __syncthreads instead of kernel boundaries; every cell sees the same operations
// in the same order as with the per-phase kernels, so the result is the same.
struct MgChain {
  MgLevel lv[kMgMaxLevels];
  int first, last;
  MgFold fold;
  const float *inv;
};
__global__ void __launch_bounds__(1024) k_mg_bottom(MgChain Ch) {
  pdl_entry();
  const unsigned tid = threadIdx.x, nt = blockDim.x;
  const int px = Ch.fold.px, py = Ch.fold.py;
  for (int l = Ch.first; l < Ch.last; ++l) {
    const MgLevel &F = Ch.lv[l], &C = Ch.lv[l + 1];
    const unsigned nf = (unsigned)F.nx * (unsigned)F.ny, nh = nf >> 1, nc = (unsigned)C.nx * (unsigned)C.ny;
    for (int k = 0; k < kMgSweeps; ++k) {
      for (unsigned t = tid; t < nh; t += nt) mg_smooth_at(F, 0, k == 0, px, py, t);
      __syncthreads();
      for (unsigned t = tid; t < nh; t += nt) mg_smooth_at(F, 1, 0, px, py, t);
      __syncthreads();
    }
    for (unsigned t = tid; t < nf; t += nt) mg_residual_at(F, px, py, t);
    __syncthreads();
    for (unsigned t = tid; t < nc; t += nt) mg_restrict_at(F, C, Ch.fold, t);
    __syncthreads();
  }
  {
    const MgLevel &L = Ch.lv[Ch.last];
    const int n = L.nx * L.ny;
    for (int i = (int)tid; i < n; i += (int)nt) {  // inv is symmetric: thread i reads column i (coalesced)
      float s = 0.0f;
      for (int k = 0; k < n; ++k) s += Ch.inv[(size_t)k * n + i] * L.b[k];
      L.x[i] = s;
    }
    __syncthreads();
  }
  for (int l = Ch.last - 1; l >= Ch.first; --l) {
    const MgLevel &F = Ch.lv[l], &C = Ch.lv[l + 1];
    const unsigned nf = (unsigned)F.nx * (unsigned)F.ny, nh = nf >> 1;
    for (unsigned t = tid; t < nf; t += nt) mg_prolong_at(C, F, Ch.fold, t);
    __syncthreads();
    for (int k = 0; k < kMgSweeps; ++k) {
      for (unsigned t = tid; t < nh; t += nt) mg_smooth_at(F, 1, 0, px, py, t);
      __syncthreads();
      for (unsigned t = tid; t < nh; t += nt) mg_smooth_at(F, 0, 0, px, py, t);
      __syncthreads();
    }
  }
}

// Coarse operator of level l+1 from the FP64 slots of level l (see the file header), in FP64 with an FP32 copy.
// mass: a uniform diagonal term of level l's operator (the shift of a shifted Laplacian K + m I), kept apart
// from the boundary excess: under R = P^T it aggregates over the four children (4 m on level l+1), while the
// boundary excess, like the face weights, is rediscretised (half the children's sum).
__global__ void k_mg_coarsen(const double *af, int nxf, int nyf, double mass, double *ac, float *acf, int nxc,
                             int nyc) {
  const unsigned nc = (unsigned)nxc * (unsigned)nyc;
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nc) return;
  const int I = (int)(t / (unsigned)nyc), J = (int)(t - (unsigned)I * (unsigned)nyc);
  const long long nf = (long long)nxf * nyf;
  auto at = [&](int s, int i, int j) { return af[(size_t)s * nf + (long long)i * nyf + j]; };
  double exc = 0.0;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b) {
      const int i = 2 * I + a, j = 2 * J + b;
      const double d = at(2, i, j);
      double e = d + at(0, i, j) + at(1, i, j) + at(3, i, j) + at(4, i, j) - mass;
      if (fabs(e) <= 1.0e-12 * fabs(d)) e = 0.0;  // interior and Neumann rows: round-off of an exact zero
      exc += e;
    }
  const double w = 0.5 * (at(0, 2 * I, 2 * J) + at(0, 2 * I, 2 * J + 1));
  const double s = 0.5 * (at(1, 2 * I, 2 * J) + at(1, 2 * I + 1, 2 * J));
  const double nn = 0.5 * (at(3, 2 * I, 2 * J + 1) + at(3, 2 * I + 1, 2 * J + 1));
  const double e = 0.5 * (at(4, 2 * I + 1, 2 * J) + at(4, 2 * I + 1, 2 * J + 1));
  const double c = -(w + s + nn + e) + 0.5 * exc + 4.0 * mass;
  const double v[5] = {w, s, c, nn, e};
  for (int k = 0; k < 5; ++k) {
    ac[(size_t)k * nc + t] = v[k];
    acf[(size_t)k * nc + t] = (float)v[k];
  }
}

// Level 0 of the CH preconditioner's hierarchy: K + m I with K = -L, L the 5-point Laplacian with reflecting
// rows at walls (build_laplacian_matrix, ch_sparse_krylov.hpp:135-177: a row counts only the neighbours that
// exist), in the W,S,C,N,E slots.
__global__ void k_shifted_laplacian(Grid G, double m, double *a, float *af) {
  const long long n = (long long)G.nx * G.ny;
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int i = (int)(r / G.ny), j = (int)(r % G.ny);
  const double cx = 1.0 / (G.dx * G.dx), cy = 1.0 / (G.dy * G.dy);
  const double w = (G.px || i > 0) ? cx : 0.0, e = (G.px || i < G.nx - 1) ? cx : 0.0;
  const double s = (G.py || j > 0) ? cy : 0.0, nn = (G.py || j < G.ny - 1) ? cy : 0.0;
  const double v[5] = {-w, -s, w + e + s + nn + m, -nn, -e};
  for (int k = 0; k < 5; ++k) {
    a[(size_t)k * n + r] = v[k];
    af[(size_t)k * n + r] = (float)v[k];
  }
}

// Inverse of the coarsest operator (n <= kMgCoarseMax cells), dense, by Gauss-Jordan elimination without
// pivoting (the matrix is SPD, shifted by mean(diag) / n on every entry when singular), in FP64 shared
// memory; the FP32 result is stored column-major (= row-major, it is symmetric).  *flag = 1 when a pivot is
// not positive and finite, and the caller then does not use the hierarchy.
__global__ void k_mg_coarse_inverse(const double *a, int nx, int ny, int px, int py, int singular, float *inv,
                                    int *flag) {
  extern __shared__ double M[];
  __shared__ double f[kMgCoarseMax];
  __shared__ double shift, piv;
  const int n = nx * ny, tid = threadIdx.x, nt = blockDim.x;
  for (int k = tid; k < n * n; k += nt) M[k] = 0.0;
  __syncthreads();
  if (tid == 0) {
    double dsum = 0.0;
    for (int r = 0; r < n; ++r) dsum += a[2 * (size_t)n + r];
    shift = singular ? dsum / ((double)n * (double)n) : 0.0;
    *flag = 0;
  }
  __syncthreads();
  for (int r = tid; r < n; r += nt) {
    const int i = r / ny, j = r % ny;
    for (int s = 0; s < 5; ++s) {
      const double v = a[(size_t)s * n + r];
      if (v == 0.0) continue;
      const long long c = slot_col<5>(i, j, s, nx, ny, px, py);
      if (c >= 0) M[r * n + (int)c] += v;  // a row owns its entries: no other thread writes row r
    }
    for (int c = 0; c < n; ++c) M[r * n + c] += shift;
  }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    if (tid == 0) {
      piv = M[k * n + k];
      if (!(piv > 0.0) || !isfinite(piv)) *flag = 1;
    }
    __syncthreads();
    const double p = piv;
    if (!(p > 0.0) || !isfinite(p)) return;  // uniform across the block
    for (int j = tid; j < n; j += nt) M[k * n + j] = (j == k) ? 1.0 / p : M[k * n + j] / p;
    for (int i = tid; i < n; i += nt) f[i] = (i == k) ? 0.0 : M[i * n + k];
    __syncthreads();
    for (int e = tid; e < n * n; e += nt) {
      const int i = e / n, j = e - (e / n) * n;
      if (i == k) continue;
      M[e] = ((j == k) ? 0.0 : M[e]) - f[i] * M[k * n + j];
    }
    __syncthreads();
  }
  for (int e = tid; e < n * n; e += nt) inv[e] = (float)M[e];
}

// ---------------------------------------------------------------------------------------------------
// CG on the FP32 operator of level 0.  Scalars and the loop control live on the device (slots below): the
// iterations run inside a CUDA graph's conditional while node whose condition k_mgcg_ctrl sets, so the host
// reads nothing until the whole solve has ended.
// ---------------------------------------------------------------------------------------------------
enum MgScal {
  kMgRz = 0, kMgPq = 1, kMgRr = 2, kMgAlpha = 3, kMgBeta = 4, kMgMeanZ = 5, kMgBad = 6,
  kMgIt = 7,   // iterations of this inner solve
  kMgCap = 8,  // its iteration limit
  kMgScalCount = 16
};

// The record of one defect-correction solve (FP64 outer loop around FP32 inner solves), kDcSize doubles on
// the device: what the host reads once the solve's graph has run, and the outer loop's own state.
enum DcSlot {
  kDcTotal = 0,    // inner iterations, all cycles
  kDcCycles = 1,   // outer cycles
  kDcAbs = 2,      // FP64 residual |b - A x| (projected when singular) of the last check
  kDcRel = 3,      // the same relative to |b|
  kDcPrev = 4,     // the residual of the previous cycle (a cycle that does not reduce it ends the multigrid)
  kDcUseMg = 5,    // the next inner solve is the multigrid CG (else the IC/ILDLT persistent PCG)
  kDcIres = 6,     // CH: the last correction's size relative to the iterate
  kDcMean = 7,     // mean of the residual removed before the inner solve (singular systems)
  kDcErr = 8,      // device status of a failed inner solve or factor (0: none)
  kDcIcZero = 9,   // the IC inner solve returned without an iteration
  kDcIcReady = 10, // the FP32 IC/ILDLT factor has been made in this solve
  kDcStarted = 11, // the first check has run
  kDcUsedMg0 = 12, // the solve started with the multigrid inner solver
  kDcIcCycles = 13,// cycles run by the IC inner solver
  kDcMgIts = 14,   // iterations run by the multigrid inner solver
  kDcSize = 16
};

struct MgVec {
  SpOpT<float> A;
  float *x, *r, *z, *p, *q;
  double *part;  // [gridDim.x][3] per-CTA partial sums
  double *scal;
};

// q = A p (the 5-point pressure or the 13-point CH operator), partial sums of p.q
template <int S>
__global__ void k_mgp_apply(MgVec V) {
  pdl_entry();
  __shared__ double sh[32];
  double v[1] = {0.0};
  const unsigned n = (unsigned)V.A.n, ny = (unsigned)V.A.ny;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int i = (int)(t / ny), j = (int)(t - (unsigned)i * ny);
    const float s = spmv_row<S>(V.A, V.p, i, j);
    V.q[t] = s;
    v[0] += (double)V.p[t] * (double)s;
  }
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) V.part[3 * blockIdx.x] = v[0];
}
// x += alpha p, r -= alpha q, partial sums of r.r
__global__ void k_mgp_update(MgVec V) {
  pdl_entry();
  __shared__ double sh[32];
  double v[1] = {0.0};
  const float alpha = (float)V.scal[kMgAlpha];
  const unsigned n = (unsigned)V.A.n;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    V.x[t] += alpha * V.p[t];
    const float r = V.r[t] - alpha * V.q[t];
    V.r[t] = r;
    v[0] += (double)r * (double)r;
  }
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) V.part[3 * blockIdx.x] = v[0];
}
// partial sums of r.z, z and r (the projected r.z of a singular system needs the last two)
__global__ void k_mgp_rz(MgVec V) {
  pdl_entry();
  __shared__ double sh[3 * 32];
  double v[3] = {0.0, 0.0, 0.0};
  const unsigned n = (unsigned)V.A.n;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const double z = V.z[t], r = V.r[t];
    v[0] += r * z;
    v[1] += z;
    v[2] += r;
  }
  block_sum<3>(v, sh);
  if (threadIdx.x == 0) {
    V.part[3 * blockIdx.x] = v[0];
    V.part[3 * blockIdx.x + 1] = v[1];
    V.part[3 * blockIdx.x + 2] = v[2];
  }
}
// p = (z - mean z) + beta p (first: p = z - mean z; first < 0: the first iteration of the solve)
__global__ void k_mgp_direction(MgVec V, int first) {
  pdl_entry();
  const float beta = (float)V.scal[kMgBeta], mz = (float)V.scal[kMgMeanZ];
  if (first < 0) first = V.scal[kMgIt] == 0.0 ? 1 : 0;
  const unsigned n = (unsigned)V.A.n;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    V.p[t] = first ? V.z[t] - mz : (V.z[t] - mz) + beta * V.p[t];
}
// The scalar step after each reduction, by one warp in a fixed order.
//   mode 0 (after k_mgp_apply):  pq, alpha = rz / pq
//   mode 1 (after k_mgp_update): rr
//   mode 2 (after k_mgp_rz):     mean z, rz' (projected when singular), beta = rz' / rz (0 when first), rz = rz'
// A non-positive or non-finite pq or rz' sets kMgBad (k_mgcg_ctrl then ends the inner solve).  first < 0:
// the first iteration of the solve.
__global__ void k_mgp_scalars(const double *part, int nparts, double *scal, int mode, int first, int project,
                              double n) {
  pdl_entry();
  const int lane = threadIdx.x;
  if (first < 0) first = scal[kMgIt] == 0.0 ? 1 : 0;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int p = lane; p < nparts; p += 32) {
    s0 += part[3 * p];
    if (mode == 2) {
      s1 += part[3 * p + 1];
      s2 += part[3 * p + 2];
    }
  }
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  s2 = warp_sum(s2);
  if (lane != 0) return;
  if (mode == 0) {
    scal[kMgPq] = s0;
    if (!(s0 > 0.0) || !isfinite(s0)) scal[kMgBad] = 1.0;
    scal[kMgAlpha] = scal[kMgRz] / s0;
  } else if (mode == 1) {
    scal[kMgRr] = s0;
  } else {
    const double mz = project ? s1 / n : 0.0;
    const double rz = project ? s0 - mz * s2 : s0;
    if (!(rz > 0.0) || !isfinite(rz)) scal[kMgBad] = 1.0;
    scal[kMgMeanZ] = mz;
    scal[kMgBeta] = first ? 0.0 : rz / scal[kMgRz];
    scal[kMgRz] = rz;
  }
}

// Start of an inner solve: its scalars cleared and its iteration limit, the outer loop's budget left
// (max(1, max_it - inner iterations so far)).  Sets the while node's condition.
__global__ void k_mgcg_init(double *scal, const double *rec, int max_it, cudaGraphConditionalHandle loop) {
  pdl_entry();
  if (threadIdx.x != 0) return;
  for (int k = 0; k < kMgScalCount; ++k) scal[k] = 0.0;
  scal[kMgCap] = (double)max(1, max_it - (int)rec[kDcTotal]);
  cudaGraphSetConditional(loop, 1u);
}

// End of one inner iteration (after the r.r reduction): counts it, and continues while no breakdown was
// flagged, |r| / |b| >= tol (|b| = the outer residual the inner right-hand side was made from; a NaN ends
// it) and the iteration limit is not reached.
__global__ void k_mgcg_ctrl(double *scal, double *rec, double tol, cudaGraphConditionalHandle loop) {
  pdl_entry();
  if (threadIdx.x != 0) return;
  const double it = scal[kMgIt] + 1.0;
  scal[kMgIt] = it;
  rec[kDcTotal] += 1.0;
  rec[kDcMgIts] += 1.0;
  bool more = it < scal[kMgCap];
  if (scal[kMgBad] != 0.0) {
    more = false;
  } else {
    const double rr = scal[kMgRr], b = rec[kDcAbs];  // std::max semantics: a NaN stays a NaN
    const double rel = sqrt(rr < 0.0 ? 0.0 : rr) / (b < 1.0e-300 ? 1.0e-300 : b);
    if (!(rel >= tol)) more = false;
  }
  cudaGraphSetConditional(loop, more ? 1u : 0u);
}

// ---------------------------------------------------------------------------------------------------
// The inner CG as one thread-block cluster (level-0 grids up to mg_cluster_cells cells).  Small grids leave a
// full-device launch per phase latency-bound: a V-cycle is about 11 launches per level, each a few
// microseconds for a few thousand cells.  Here 1-8 CTAs of 1024 threads, which the hardware schedules
// together, run every iteration of the solve: V-cycles, r.z, direction, A p, p.q and the update as phases
// separated by cluster barriers (barrier.cluster with release / acquire, which orders the global memory the
// phases exchange), dot products reduced through distributed shared memory in rank order, so every CTA holds
// the same scalars and takes the same stopping decision.  One launch per inner solve; nothing waits on
// another launch or spins.  The cell arithmetic is the per-phase kernels' (mg_*_at), phase for phase.
// ---------------------------------------------------------------------------------------------------
constexpr int kMgClusterThreads = 1024;
constexpr int kMgClusterMax = 8;              // CTAs per cluster at most (the portable cluster size)
constexpr long long kMgClusterCells = 0;  // default: off (set from measurements)
constexpr int kMgClusterSmemMax = 160 * 1024;  // dynamic shared memory of the bottom levels at most

struct MgClusterArgs {
  const MgChain *ch;     // levels 0 .. last of the preconditioner's hierarchy, in device memory (lv[0].b / .x
                         // are replaced per V-cycle)
  SpOpT<float> A;        // the CG operator on level 0 (the 5-point pressure or the 13-point CH operator)
  float *x, *r, *z, *p, *q, *tmp;
  const float *b;        // the inner right-hand side (x is zero on entry)
  int vcycles, project, max_it;
  int bottom;            // the first level of at most kMgBottomCells cells: it and the coarser ones run on CTA 0
                         // in shared memory (3 floats per cell of those levels, dynamic)
  double tol;            // relative to |b| = R[kDcAbs]
  double *R;             // the defect-correction record: iterations added to kDcTotal and kDcMgIts
};

__device__ __forceinline__ void mgc_sync() { cooperative_groups::this_cluster().sync(); }

// K sums over the cluster: the CTA's sums, then every CTA adds the CTAs' sums in rank order (warp 0 reads
// them from distributed shared memory), so all threads of all CTAs hold the same bits.  `slot` alternates
// by `par` so that a CTA writing the next reduction never overwrites sums another CTA is still reading.
template <int K>
__device__ __forceinline__ void mgc_sum(double (&v)[K], double *sh, double (*slot)[4], double *bc, int &par) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  block_sum<K>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) slot[par][k] = v[k];
  }
  cl.sync();
  if (threadIdx.x == 0) {
    const unsigned cs = cl.num_blocks();
#pragma unroll
    for (int k = 0; k < K; ++k) bc[k] = 0.0;
    for (unsigned j = 0; j < cs; ++j) {
      const double *o = cl.map_shared_rank(&slot[par][0], j);
#pragma unroll
      for (int k = 0; k < K; ++k) bc[k] += o[k];
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = bc[k];
  __syncthreads();
  par ^= 1;
}

// The off-diagonal sum of mg_row_sum for up to kMgBatch cells at once: every load of the batch is issued
// before any sum is formed (the neighbours' x values do not wait for the coefficients), then each cell's sum
// is taken in slot order over its non-zero coefficients, as mg_row_sum takes it.
constexpr int kMgBatch = 4;
__device__ __forceinline__ void mg_row_sums(const MgLevel &L, const float *x, const int (&ci)[kMgBatch],
                                            const int (&cj)[kMgBatch], const bool (&on)[kMgBatch], long long n,
                                            int px, int py, float (&out)[kMgBatch]) {
  constexpr int ks[4] = {0, 1, 3, 4};
  float av[kMgBatch][4], xv[kMgBatch][4];
#pragma unroll
  for (int u = 0; u < kMgBatch; ++u) {
    const long long r = (long long)ci[u] * L.ny + cj[u];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      av[u][q] = 0.0f;
      xv[u][q] = 0.0f;
      if (on[u]) {
        const long long c = slot_col<5>(ci[u], cj[u], ks[q], L.nx, L.ny, px, py);
        av[u][q] = __ldg(&L.a[(size_t)ks[q] * n + r]);
        if (c >= 0) xv[u][q] = x[c];
        else av[u][q] = 0.0f;  // mg_row_sum skips a missing neighbour
      }
    }
  }
#pragma unroll
  for (int u = 0; u < kMgBatch; ++u) {
    float s = 0.0f;
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (av[u][q] != 0.0f) s += av[u][q] * xv[u][q];
    out[u] = s;
  }
}

// mg_smooth_at for the cells t0, t0 + st, ... (kMgBatch of them, those below lim): one colour, so no cell of
// the batch reads another's x, and all loads go before the stores.  The arithmetic is mg_smooth_at's.
__device__ __forceinline__ void mg_smooth_batch(const MgLevel &L, int color, int first, int px, int py, unsigned t0,
                                                unsigned st, unsigned lim) {
  const int half = L.ny >> 1;
  const long long n = (long long)L.nx * L.ny;
  int ci[kMgBatch], cj[kMgBatch];
  bool on[kMgBatch];
  float bv[kMgBatch], dv[kMgBatch], rs[kMgBatch];
#pragma unroll
  for (int u = 0; u < kMgBatch; ++u) {
    const unsigned t = t0 + (unsigned)u * st;
    on[u] = t < lim;
    const unsigned tt = on[u] ? t : 0u;
    ci[u] = (int)(tt / (unsigned)half);
    cj[u] = 2 * (int)(tt - (unsigned)ci[u] * (unsigned)half) + ((ci[u] + color) & 1);
    const long long r = (long long)ci[u] * L.ny + cj[u];
    bv[u] = on[u] ? L.b[r] : 0.0f;
    dv[u] = on[u] ? __ldg(&L.a[2 * n + r]) : 1.0f;
  }
  if (!first) mg_row_sums(L, L.x, ci, cj, on, n, px, py, rs);
#pragma unroll
  for (int u = 0; u < kMgBatch; ++u) {
    if (!on[u]) continue;
    const long long r = (long long)ci[u] * L.ny + cj[u];
    float s = bv[u];
    if (!first) s -= rs[u];
    L.x[r] = s / dv[u];
    if (first) L.x[(long long)ci[u] * L.ny + (cj[u] ^ 1)] = 0.0f;
  }
}

// mg_residual_at for a batch of cells, loads before stores (r is written, x only read)
__device__ __forceinline__ void mg_residual_batch(const MgLevel &L, int px, int py, unsigned t0, unsigned st,
                                                  unsigned lim) {
  const long long n = (long long)L.nx * L.ny;
  int ci[kMgBatch], cj[kMgBatch];
  bool on[kMgBatch];
  float bv[kMgBatch], dv[kMgBatch], xc[kMgBatch], rs[kMgBatch];
#pragma unroll
  for (int u = 0; u < kMgBatch; ++u) {
    const unsigned t = t0 + (unsigned)u * st;
    on[u] = t < lim;
    const unsigned tt = on[u] ? t : 0u;
    ci[u] = (int)(tt / (unsigned)L.ny);
    cj[u] = (int)(tt - (unsigned)ci[u] * (unsigned)L.ny);
    bv[u] = on[u] ? L.b[tt] : 0.0f;
    dv[u] = on[u] ? __ldg(&L.a[2 * n + tt]) : 0.0f;
    xc[u] = on[u] ? L.x[tt] : 0.0f;
  }
  mg_row_sums(L, L.x, ci, cj, on, n, px, py, rs);
#pragma unroll
  for (int u = 0; u < kMgBatch; ++u)
    if (on[u]) L.r[t0 + (unsigned)u * st] = bv[u] - (dv[u] * xc[u] + rs[u]);
}

// Levels `first` .. last of C in one CTA with __syncthreads between phases (k_mg_bottom's order of phases);
// lv: the levels with their x, b, r (in shared memory for the cluster form).
__device__ void mg_bottom_cta(const MgChain &C, const MgLevel *lv, int first) {
  const unsigned tid = threadIdx.x, nt = blockDim.x;
  const int px = C.fold.px, py = C.fold.py, last = C.last;
  for (int l = first; l < last; ++l) {
    const MgLevel &F = lv[l], &Cl = lv[l + 1];
    const unsigned nf = (unsigned)F.nx * (unsigned)F.ny, nh = nf >> 1, nc = (unsigned)Cl.nx * (unsigned)Cl.ny;
    for (int k = 0; k < kMgSweeps; ++k) {
      for (unsigned t = tid; t < nh; t += kMgBatch * nt) mg_smooth_batch(F, 0, k == 0, px, py, t, nt, nh);
      __syncthreads();
      for (unsigned t = tid; t < nh; t += kMgBatch * nt) mg_smooth_batch(F, 1, 0, px, py, t, nt, nh);
      __syncthreads();
    }
    for (unsigned t = tid; t < nf; t += kMgBatch * nt) mg_residual_batch(F, px, py, t, nt, nf);
    __syncthreads();
    for (unsigned t = tid; t < nc; t += nt) mg_restrict_at(F, Cl, C.fold, t);
    __syncthreads();
  }
  {
    const MgLevel &L = lv[last];
    const int n = L.nx * L.ny;
    for (int i = (int)tid; i < n; i += (int)nt) {  // inv is symmetric: thread i reads column i
      float s = 0.0f;
      for (int k = 0; k < n; ++k) s += __ldg(&C.inv[(size_t)k * n + i]) * L.b[k];
      L.x[i] = s;
    }
    __syncthreads();
  }
  for (int l = last - 1; l >= first; --l) {
    const MgLevel &F = lv[l], &Cl = lv[l + 1];
    const unsigned nf = (unsigned)F.nx * (unsigned)F.ny, nh = nf >> 1;
    for (unsigned t = tid; t < nf; t += nt) mg_prolong_at(Cl, F, C.fold, t);
    __syncthreads();
    for (int k = 0; k < kMgSweeps; ++k) {
      for (unsigned t = tid; t < nh; t += kMgBatch * nt) mg_smooth_batch(F, 1, 0, px, py, t, nt, nh);
      __syncthreads();
      for (unsigned t = tid; t < nh; t += kMgBatch * nt) mg_smooth_batch(F, 0, 0, px, py, t, nt, nh);
      __syncthreads();
    }
  }
}

// One V-cycle x0 = B b0 over every level of `C`.  The levels above `bf` (the first of at most kMgBottomCells
// cells) run on the whole cluster, its threads striding over each phase's cells in batches, with a cluster
// barrier between phases.  The levels from bf down run on CTA 0 alone with their x, b, r in shared memory
// (`smem`, 3 x their cells floats), entered with level bf's b and left with its x through global memory.
__device__ void mgc_vcycle(const MgChain &C, int bf, float *smem, MgLevel *s_lv, float *b0, float *x0, unsigned gt,
                           unsigned GT) {
  const int px = C.fold.px, py = C.fold.py, last = C.last;
  auto level = [&](int l) {
    MgLevel L = C.lv[l];
    if (l == 0) {
      L.b = b0;
      L.x = x0;
    }
    return L;
  };
  for (int l = 0; l < bf; ++l) {
    const MgLevel F = level(l), Cl = level(l + 1);
    const unsigned nf = (unsigned)F.nx * (unsigned)F.ny, nh = nf >> 1, nc = (unsigned)Cl.nx * (unsigned)Cl.ny;
    for (int k = 0; k < kMgSweeps; ++k) {
      for (unsigned t = gt; t < nh; t += kMgBatch * GT) mg_smooth_batch(F, 0, k == 0, px, py, t, GT, nh);
      mgc_sync();
      for (unsigned t = gt; t < nh; t += kMgBatch * GT) mg_smooth_batch(F, 1, 0, px, py, t, GT, nh);
      mgc_sync();
    }
    for (unsigned t = gt; t < nf; t += kMgBatch * GT) mg_residual_batch(F, px, py, t, GT, nf);
    mgc_sync();
    for (unsigned t = gt; t < nc; t += GT) mg_restrict_at(F, Cl, C.fold, t);
    mgc_sync();
  }
  if (cooperative_groups::this_cluster().block_rank() == 0) {
    if (threadIdx.x == 0) {  // the bottom levels' table, their vectors in shared memory
      float *q = smem;
      for (int l = bf; l <= last; ++l) {
        MgLevel L = C.lv[l];
        const unsigned nl = (unsigned)L.nx * (unsigned)L.ny;
        L.x = q;
        L.b = q + nl;
        L.r = q + 2 * nl;
        q += 3 * nl;
        s_lv[l] = L;
      }
    }
    __syncthreads();
    const MgLevel E = level(bf);  // the entry level's global b and x
    const unsigned ne = (unsigned)E.nx * (unsigned)E.ny;
    float *eb = s_lv[bf].b;
    for (unsigned t = threadIdx.x; t < ne; t += blockDim.x) eb[t] = E.b[t];
    __syncthreads();
    mg_bottom_cta(C, s_lv, bf);
    const float *ex = s_lv[bf].x;
    for (unsigned t = threadIdx.x; t < ne; t += blockDim.x) E.x[t] = ex[t];
  }
  mgc_sync();
  for (int l = bf - 1; l >= 0; --l) {
    const MgLevel F = level(l), Cl = level(l + 1);
    const unsigned nf = (unsigned)F.nx * (unsigned)F.ny, nh = nf >> 1;
    for (unsigned t = gt; t < nf; t += GT) mg_prolong_at(Cl, F, C.fold, t);
    mgc_sync();
    for (int k = 0; k < kMgSweeps; ++k) {
      for (unsigned t = gt; t < nh; t += kMgBatch * GT) mg_smooth_batch(F, 1, 0, px, py, t, GT, nh);
      mgc_sync();
      for (unsigned t = gt; t < nh; t += kMgBatch * GT) mg_smooth_batch(F, 0, 0, px, py, t, GT, nh);
      mgc_sync();
    }
  }
}

// The whole inner solve: r = b; per iteration z = M r (vcycles V-cycles, through tmp when two), r.z (the
// mean of z removed when the system is singular), p = (z - mean z) + beta p, q = A p, alpha = r.z / p.q,
// x += alpha p, r -= alpha q; it ends as k_mgcg_ctrl ends the per-phase form: a non-positive or non-finite
// r.z or p.q, |r| < tol |b|, or the iteration budget left in R (at least one iteration).
template <int S>
__global__ void __launch_bounds__(kMgClusterThreads, 1) k_mgcg_cluster(const MgClusterArgs P) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const unsigned gt = cl.block_rank() * blockDim.x + threadIdx.x, GT = cl.num_blocks() * blockDim.x;
  __shared__ double sh[3 * 32];
  __shared__ double slot[2][4];
  __shared__ double bc[4];
  __shared__ MgLevel s_lv[kMgMaxLevels];
  extern __shared__ float mgc_smem[];
  int par = 0;
  const unsigned n = (unsigned)P.A.n, ny = (unsigned)P.A.ny;
  const double bnorm = P.R[kDcAbs];
  const int cap = max(1, P.max_it - (int)P.R[kDcTotal]);
  for (unsigned t = gt; t < n; t += GT) P.r[t] = P.b[t];
  mgc_sync();
  double rz_old = 0.0;
  int it = 0;
  for (;;) {
    if (P.vcycles == 2) {
      mgc_vcycle(*P.ch, P.bottom, mgc_smem, s_lv, P.r, P.tmp, gt, GT);
      mgc_vcycle(*P.ch, P.bottom, mgc_smem, s_lv, P.tmp, P.z, gt, GT);
    } else {
      mgc_vcycle(*P.ch, P.bottom, mgc_smem, s_lv, P.r, P.z, gt, GT);
    }
    double v3[3] = {0.0, 0.0, 0.0};
    for (unsigned t = gt; t < n; t += GT) {
      const double z = P.z[t], r = P.r[t];
      v3[0] += r * z;
      v3[1] += z;
      v3[2] += r;
    }
    mgc_sum<3>(v3, sh, slot, bc, par);
    const double mz = P.project ? v3[1] / (double)n : 0.0;
    const double rz = P.project ? v3[0] - mz * v3[2] : v3[0];
    bool bad = !(rz > 0.0) || !isfinite(rz);
    const float beta = it == 0 ? 0.0f : (float)(rz / rz_old), fmz = (float)mz;
    rz_old = rz;
    for (unsigned t = gt; t < n; t += GT) P.p[t] = it == 0 ? P.z[t] - fmz : (P.z[t] - fmz) + beta * P.p[t];
    mgc_sync();
    double v1[1] = {0.0};
    for (unsigned t = gt; t < n; t += GT) {
      const int i = (int)(t / ny), j = (int)(t - (unsigned)i * ny);
      const float s = spmv_row<S>(P.A, P.p, i, j);
      P.q[t] = s;
      v1[0] += (double)P.p[t] * (double)s;
    }
    mgc_sum<1>(v1, sh, slot, bc, par);
    if (!(v1[0] > 0.0) || !isfinite(v1[0])) bad = true;
    const float alpha = (float)(rz / v1[0]);
    double v2[1] = {0.0};
    for (unsigned t = gt; t < n; t += GT) {
      P.x[t] += alpha * P.p[t];
      const float r = P.r[t] - alpha * P.q[t];
      P.r[t] = r;
      v2[0] += (double)r * (double)r;
    }
    mgc_sum<1>(v2, sh, slot, bc, par);
    ++it;
    // std::max semantics, as k_mgcg_ctrl: a NaN ends the solve
    const double rr = v2[0], rel = sqrt(rr < 0.0 ? 0.0 : rr) / (bnorm < 1.0e-300 ? 1.0e-300 : bnorm);
    if (bad || !(rel >= P.tol) || it >= cap) break;
  }
  if (gt == 0) {
    P.R[kDcTotal] += (double)it;
    P.R[kDcMgIts] += (double)it;
  }
  mgc_sync();  // no CTA leaves while another may still read its shared memory
}

}  // namespace dn
