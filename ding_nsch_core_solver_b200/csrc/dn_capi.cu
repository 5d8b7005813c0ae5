// dn_capi.cu -- host side of libdn_cuda: handle, device state, the time-step driver and the C-ABI.
//
// The driver replays Solver::advance_one_timestep (src/core/coupled/solver.cpp:224-283) as a sequence of
// kernels on one stream; the three linear solves run as persistent cooperative kernels (dn_krylov.cuh,
// dn_momentum.cuh).  There is no CPU fallback: every numeric step runs on the GPU, and a missing or
// failing device reports an error status.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cctype>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <functional>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "dn_adjoint.cuh"
#include "dn_common.cuh"
#include "dn_fields.cuh"
#include "dn_krylov.cuh"
#include "dn_momentum.cuh"
#include "dn_momentum_adjoint.cuh"
#include "dn_multigrid.cuh"

using namespace dn;

namespace {

constexpr double kSqrt2 = 1.4142135623730950488;
constexpr int kHostScal = 8192;  // pinned host scratch (doubles): scalars and reduction partials
constexpr int kCapDepth = 4;     // conditional graph nodes nested at most this deep
constexpr int kDiagParts = 128;  // CTAs of the diagnostics reduction
// Sweep warps per CTA: one per SM sub-partition (scheduler).  A fifth warp shares a scheduler with the
// first and slows both; fewer warps per CTA put more hand-overs across CTAs (measured 81.9 ms per pressure
// solve with 4, 87.8 with 5, 92.6 with 1 on the 192 x 384 bench workload).
constexpr int kSweepWarpsPerCta = 4;
// dynamic shared memory the CH PCG kernel may use (the ring of the level sweep, the periodic-y line buffers)
constexpr size_t kSeqSmemMax = 96 * 1024;
// rows per CTA of the persistent PCG's SpMV / update phases: they are latency-bound, so more CTAs shorten them
constexpr long long kPcgRowsPerCta = 512;

// ---------------------------------------------------------------------------------------------------
// Pressure system (build_pressure_linear_system, pressure.cpp:123-196) into 5 slots W,S,C,N,E + rhs
// ---------------------------------------------------------------------------------------------------
__device__ double split_divergence(const Fv &pe, const Fv &rm, const Grid &G, int i, int j, double rho_ref) {
  // liu_split_explicit_divergence, operators.cpp:424-444
  const bool eo = G.px || i < G.nx - 1, wo = G.px || i > 0, no = G.py || j < G.ny - 1, so = G.py || j > 0;
  const double fe = eo ? (1.0 - rho_ref / xface(rm, G, i + 1, j)) * gfx(pe, G, i + 1, j) : 0.0;
  const double fw = wo ? (1.0 - rho_ref / xface(rm, G, i, j)) * gfx(pe, G, i, j) : 0.0;
  const double fn = no ? (1.0 - rho_ref / yface(rm, G, i, j + 1)) * gfy(pe, G, i, j + 1) : 0.0;
  const double fs = so ? (1.0 - rho_ref / yface(rm, G, i, j)) * gfy(pe, G, i, j) : 0.0;
  return (fe - fw) / G.dx + (fn - fs) / G.dy;
}

__global__ void k_p_assemble(Grid G, BCSet bc, Fv rm, Fv us, Fv vs, Fv pe, int split, double rho_ref, double dt,
                             double *a, double *rhs) {
  const long long n = (long long)G.nx * G.ny;
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int i = (int)(r / G.ny), j = (int)(r % G.ny);
  const double dx = G.dx, dy = G.dy;
  const bool he = G.px || i < G.nx - 1, hw = G.px || i > 0, hn = G.py || j < G.ny - 1, hs = G.py || j > 0;
  const double ce = split ? 1.0 / (dx * dx) : 1.0 / (xface(rm, G, i + 1, j) * dx * dx);
  const double cw = split ? 1.0 / (dx * dx) : 1.0 / (xface(rm, G, i, j) * dx * dx);
  const double cn = split ? 1.0 / (dy * dy) : 1.0 / (yface(rm, G, i, j + 1) * dy * dy);
  const double cs = split ? 1.0 / (dy * dy) : 1.0 / (yface(rm, G, i, j) * dy * dy);
  double diag = 0.0;
  double rv = split ? -(split_divergence(pe, rm, G, i, j, rho_ref) + rho_ref * div_cell(us, vs, G, i, j) / dt)
                    : -div_cell(us, vs, G, i, j) / dt;
  auto boundary = [&](int side, double coeff, double spacing) {
    const BCSide &b = bc.p[side];
    if (b.type == DN_BC_DIRICHLET) {
      diag += 2.0 * coeff;
      rv += 2.0 * coeff * b.value;
    } else {
      rv += coeff * b.value * spacing;
    }
  };
  double aE = 0.0, aW = 0.0, aN = 0.0, aS = 0.0;
  if (he) {
    diag += ce;
    aE = 0.0 + -ce;
  } else {
    boundary(DN_RIGHT, ce, dx);
  }
  if (hw) {
    diag += cw;
    aW = 0.0 + -cw;
  } else {
    boundary(DN_LEFT, cw, dx);
  }
  if (hn) {
    diag += cn;
    aN = 0.0 + -cn;
  } else {
    boundary(DN_TOP, cn, dy);
  }
  if (hs) {
    diag += cs;
    aS = 0.0 + -cs;
  } else {
    boundary(DN_BOTTOM, cs, dy);
  }
  auto keep = [](double v) { return fabs(v) < 1.0e-18 ? 0.0 : v; };
  a[0 * n + r] = keep(aW);
  a[1 * n + r] = keep(aS);
  a[2 * n + r] = 0.0 + diag;
  a[3 * n + r] = keep(aN);
  a[4 * n + r] = keep(aE);
  rhs[r] = rv;
}

// ---------------------------------------------------------------------------------------------------
// Mixed-precision pressure solve: FP64 defect correction around FP32 inner PCG solves
// ---------------------------------------------------------------------------------------------------
__global__ void k_to_float(const double *src, float *dst, long long n) {
  pdl_entry();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dst[t] = (float)src[t];
}
// r = b - A x in FP64, with per-CTA sums of r, r^2 and b^2 (the outer residual and its stopping norms)
template <int S>
__global__ void k_outer_residual(SpOp A, const double *b, const double *x, double *r, double *partials) {
  pdl_entry();
  __shared__ double sh[3 * 32];
  double v[3] = {0.0, 0.0, 0.0};
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < A.n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / A.ny), j = (int)(t % A.ny);
    const double rr = b[t] - spmv_row<S>(A, x, i, j);
    r[t] = rr;
    v[0] += rr;
    v[1] += rr * rr;
    v[2] += b[t] * b[t];
  }
  block_sum<3>(v, sh);
  if (threadIdx.x == 0) {
    partials[3 * blockIdx.x + 0] = v[0];
    partials[3 * blockIdx.x + 1] = v[1];
    partials[3 * blockIdx.x + 2] = v[2];
  }
}
// the three sums of k_outer_residual, added in a fixed order by one warp
__global__ void k_finish3(const double *partials, int nparts, double *out) {
  pdl_entry();
  const int lane = threadIdx.x;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int p = lane; p < nparts; p += 32) {
    s0 += partials[3 * p];
    s1 += partials[3 * p + 1];
    s2 += partials[3 * p + 2];
  }
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  s2 = warp_sum(s2);
  if (lane == 0) {
    out[0] = s0;
    out[1] = s1;
    out[2] = s2;
  }
}
__global__ void k_add_correction(double *x, const float *e, long long n) {
  pdl_entry();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) x[t] += (double)e[t];
}
// x += e with per-CTA sums of e^2 and of the updated x^2 (the iterate residual |dx| / |x| of the CH report)
__global__ void k_add_correction_norms(double *x, const float *e, long long n, double *partials) {
  pdl_entry();
  __shared__ double sh[3 * 32];
  double v[3] = {0.0, 0.0, 0.0};
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const double d = (double)e[t], xn = x[t] + d;
    x[t] = xn;
    v[0] += d * d;
    v[1] += xn * xn;
  }
  block_sum<3>(v, sh);
  if (threadIdx.x == 0) {
    partials[3 * blockIdx.x + 0] = v[0];
    partials[3 * blockIdx.x + 1] = v[1];
    partials[3 * blockIdx.x + 2] = 0.0;
  }
}

// ---- the defect-correction loop's decisions on the device (the record layout is DcSlot)
constexpr int kDcMaxCycles = 40;  // outer cycles of one mixed-precision solve at most
constexpr int kRecPressure = 0;   // offsets of the records in h->rec
constexpr int kRecCh = 16;
constexpr int kRecCount = 64;

struct DcParams {
  double tol;          // the reference's stopping tolerance, on the relative or the absolute FP64 residual
  double n;            // cells (the projected norms of a singular system)
  int max_it;          // inner iterations of the whole solve at most
  int max_cycles;      // outer cycles at most
  int project;         // singular pressure system: the residual is projected (its mean removed)
  int ch;              // CH rules: multigrid inner solves only, a cycle that does not reduce the residual ends
  const int *mg_flag;  // the coarsest level's inverse status of the inner hierarchy (0: usable); null: none
};

// max with std::max's semantics (a NaN first argument is kept, so a non-finite residual never reads as
// converged)
__device__ __forceinline__ double smax(double a, double b) { return a < b ? b : a; }

// right-hand side of an inner solve: the FP64 residual less its mean (R[kDcMean]) rounded to FP32; the
// correction starts at 0
__global__ void k_inner_rhs_dev(const double *r, const double *R, float *rf, float *ef, long long n) {
  pdl_entry();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const double mean = R[kDcMean];
  if (t < n) {
    rf[t] = (float)(r[t] - mean);
    ef[t] = 0.0f;
  }
}

// The check after each FP64 residual (sums = r, r^2, b^2 from k_outer_residual / k_finish3): the stopping
// rule of the reference (rel < tol or abs < tol), the cycle and iteration budgets, and the stall rule (a
// multigrid cycle that did not reduce the residual hands the pressure solve to the IC inner solver; any
// other stalled cycle ends the solve).  Sets the outer while node's condition.
__global__ void k_dc_decide(const double *sums, double *R, DcParams P, cudaGraphConditionalHandle loop) {
  pdl_entry();
  if (threadIdx.x != 0) return;
  if (R[kDcStarted] == 0.0) {
    R[kDcStarted] = 1.0;
    R[kDcPrev] = INFINITY;
    R[kDcUseMg] = (P.mg_flag != nullptr && *P.mg_flag == 0) ? 1.0 : 0.0;
    R[kDcUsedMg0] = R[kDcUseMg];
  }
  bool more = true;
  if (R[kDcErr] != 0.0 || R[kDcIcZero] != 0.0) {
    more = false;  // a failed inner solve, or an IC inner solve that could not move (x unchanged)
  } else {
    const double s0 = sums[0], s1 = sums[1], s2 = sums[2];
    const double mean = P.project ? s0 / P.n : 0.0;
    const double rn2 = P.project ? smax(s1 - s0 * s0 / P.n, 0.0) : (P.ch ? smax(s1, 0.0) : s1);
    const double absr = sqrt(rn2);
    const double relr = absr / smax(sqrt(smax(s2, 0.0)), 1.0e-30);
    R[kDcAbs] = absr;
    R[kDcRel] = relr;
    R[kDcMean] = mean;
    if (relr < P.tol || absr < P.tol) {
      more = false;
    } else if (R[kDcCycles] >= (double)P.max_cycles || R[kDcTotal] >= (double)P.max_it) {
      more = false;
    } else if (!(absr < R[kDcPrev])) {
      if (P.ch || R[kDcUseMg] == 0.0) more = false;
      else R[kDcUseMg] = 0.0;
    }
    if (more) R[kDcPrev] = absr;
  }
  cudaGraphSetConditional(loop, more ? 1u : 0u);
}

// the inner solver of this cycle: multigrid CG (has_mg: the graph holds that branch) or the IC persistent PCG
__global__ void k_dc_branch(const double *R, int has_mg, cudaGraphConditionalHandle mg,
                            cudaGraphConditionalHandle ic) {
  pdl_entry();
  if (threadIdx.x != 0) return;
  const bool use_mg = R[kDcUseMg] != 0.0;
  if (has_mg) cudaGraphSetConditional(mg, use_mg ? 1u : 0u);
  cudaGraphSetConditional(ic, use_mg ? 0u : 1u);
}

// end of a cycle: counted; with the CH's norms (|e|^2, |x|^2 after the update) the iterate residual
__global__ void k_dc_cycle_end(const double *norms, double *R) {
  pdl_entry();
  if (threadIdx.x != 0) return;
  R[kDcCycles] += 1.0;
  if (norms) R[kDcIres] = sqrt(smax(norms[0], 0.0) / smax(norms[1], 1.0e-30));
}

// the IC inner solver's factor is made once per solve: `make` on its first use, `go` once it exists
__global__ void k_ic_need(const double *R, cudaGraphConditionalHandle make, cudaGraphConditionalHandle go) {
  if (threadIdx.x != 0) return;
  const bool ready = R[kDcIcReady] != 0.0;
  cudaGraphSetConditional(make, ready ? 0u : 1u);
  cudaGraphSetConditional(go, ready ? 1u : 0u);
}
// after the factor: a failed one is recorded (and the inner solve skipped), else it is ready
__global__ void k_ic_gate(const int *status, double *R, cudaGraphConditionalHandle go) {
  if (threadIdx.x != 0) return;
  const bool failed = *status == kDevFactorFailed;
  if (failed) R[kDcErr] = (double)kDevFactorFailed;
  else R[kDcIcReady] = 1.0;
  cudaGraphSetConditional(go, failed ? 0u : 1u);
}
// after the IC inner solve (its out[0] = iterations, status): iterations counted, a failure recorded
__global__ void k_ic_done(const double *out, const int *status, double *R) {
  pdl_entry();
  if (threadIdx.x != 0) return;
  if (*status != kDevOk) {
    R[kDcErr] = (double)*status;
    return;
  }
  R[kDcTotal] += out[0];
  R[kDcIcCycles] += 1.0;
  if (out[0] == 0.0) R[kDcIcZero] = 1.0;
}

// ---------------------------------------------------------------------------------------------------
// CH operator A = alpha0 I - beta1 L + beta2 L^2 (build_laplacian_matrix / multiply /
// build_cahn_hilliard_operator, ch_sparse_krylov.hpp:135-233) with std::map accumulation semantics.
// ---------------------------------------------------------------------------------------------------
struct SmallMap {
  long long col[16];
  double val[16];
  int cnt;
  __device__ void clear() { cnt = 0; }
  __device__ void add(long long c, double v) {
    for (int k = 0; k < cnt; ++k)
      if (col[k] == c) {
        val[k] += v;
        return;
      }
    col[cnt] = c;
    val[cnt] = 0.0 + v;
    ++cnt;
  }
  __device__ void sort() {
    for (int a = 1; a < cnt; ++a) {
      long long c = col[a];
      double v = val[a];
      int b = a - 1;
      while (b >= 0 && col[b] > c) {
        col[b + 1] = col[b];
        val[b + 1] = val[b];
        --b;
      }
      col[b + 1] = c;
      val[b + 1] = v;
    }
  }
  __device__ void drop_tiny() {  // finalize_row_maps, ch_sparse_krylov.hpp:116
    int w = 0;
    for (int k = 0; k < cnt; ++k)
      if (!(fabs(val[k]) < 1.0e-18)) {
        col[w] = col[k];
        val[w] = val[k];
        ++w;
      }
    cnt = w;
  }
};

__device__ void laplacian_row(int i, int j, const Grid &G, SmallMap &m) {
  const int nx = G.nx, ny = G.ny;
  const double inv_dx2 = 1.0 / (G.dx * G.dx), inv_dy2 = 1.0 / (G.dy * G.dy);
  const long long row = (long long)i * ny + j;
  double diag = 0.0;
  m.clear();
  if (G.px || i > 0) {
    const int iw = (G.px && i == 0) ? nx - 1 : i - 1;
    m.add((long long)iw * ny + j, inv_dx2);
    diag -= inv_dx2;
  }
  if (G.px || i < nx - 1) {
    const int ie = (G.px && i == nx - 1) ? 0 : i + 1;
    m.add((long long)ie * ny + j, inv_dx2);
    diag -= inv_dx2;
  }
  if (G.py || j > 0) {
    const int js = (G.py && j == 0) ? ny - 1 : j - 1;
    m.add((long long)i * ny + js, inv_dy2);
    diag -= inv_dy2;
  }
  if (G.py || j < ny - 1) {
    const int jn = (G.py && j == ny - 1) ? 0 : j + 1;
    m.add((long long)i * ny + jn, inv_dy2);
    diag -= inv_dy2;
  }
  m.add(row, diag);
  m.sort();
  m.drop_tiny();
}

__global__ void k_ch_matrix(Grid G, double alpha0, double beta1, double beta2, double *a13, int *status) {
  const long long n = (long long)G.nx * G.ny;
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int i = (int)(r / G.ny), j = (int)(r % G.ny);
  SmallMap L, Lm, L2, A;
  laplacian_row(i, j, G, L);
  L2.clear();
  for (int p = 0; p < L.cnt; ++p) {
    const long long mid = L.col[p];
    laplacian_row((int)(mid / G.ny), (int)(mid % G.ny), G, Lm);
    for (int q = 0; q < Lm.cnt; ++q) L2.add(Lm.col[q], L.val[p] * Lm.val[q]);
  }
  L2.sort();
  L2.drop_tiny();
  A.clear();
  A.add(r, alpha0);
  for (int p = 0; p < L.cnt; ++p) A.add(L.col[p], -beta1 * L.val[p]);
  for (int p = 0; p < L2.cnt; ++p) A.add(L2.col[p], beta2 * L2.val[p]);
  A.drop_tiny();
  for (int s = 0; s < 13; ++s) a13[(size_t)s * n + r] = 0.0;
  for (int p = 0; p < A.cnt; ++p) {
    int slot = -1;
    for (int s = 0; s < 13; ++s)
      if (slot_col<13>(i, j, s, G.nx, G.ny, G.px, G.py) == A.col[p]) {
        slot = s;
        break;
      }
    if (slot < 0) {
      atomicExch(status, 1);  // column outside the 13-point stencil (grid too small)
      continue;
    }
    a13[(size_t)slot * n + r] = A.val[p];
  }
}

// ---------------------------------------------------------------------------------------------------
// Initial conditions (initialize_phase / initialize_velocity, solver.cpp:115-221)
// ---------------------------------------------------------------------------------------------------
struct InitParams {
  int mode, phase_initializer, velocity_profile, invert_phase, couette;
  double cn, lx, ly, cx, cy, radius, amplitude, wavenumber, slot_w, slot_d, advect_u, advect_v;
  double rcx, rcy, omega, ub, ut;
};

__device__ double sd_box(double x, double y, double cx, double cy, double hx, double hy) {
  const double qx = fabs(x - cx) - hx, qy = fabs(y - cy) - hy;
  const double ox = fmax(qx, 0.0), oy = fmax(qy, 0.0);
  return hypot(ox, oy) + fmin(fmax(qx, qy), 0.0);
}

__global__ void k_init_phase(Fv c, Grid G, InitParams P) {
  DN_FOR_INTERIOR(c);
  const double x = ((double)i + 0.5) * G.dx, y = ((double)j + 0.5) * G.dy;
  double value = 1.0;
  if (P.phase_initializer == 1) {
    const double shw = 0.5 * P.slot_w, st = P.cy + P.radius, sb = st - P.slot_d;
    const double scy = 0.5 * (st + sb), shh = 0.5 * (st - sb);
    const double sm = fmax(2.0 * kSqrt2 * P.cn, 1.0e-12);
    const double dsd = hypot(x - P.cx, y - P.cy) - P.radius;
    const double shape = fmax(dsd, -sd_box(x, y, P.cx, scy, shw, shh));
    value = 0.5 - 0.5 * tanh(shape / sm);
    c.at(i, j) = P.invert_phase ? (1.0 - value) : value;
    return;
  }
  if (P.mode == DN_MODE_SINGLE_PHASE) {
    c.at(i, j) = P.invert_phase ? 0.0 : 1.0;
    return;
  }
  if (P.mode != DN_MODE_ADVECTION_ONLY) {
    if (P.radius > 0.0) {
      const double rx = x - P.cx, ry = y - P.cy;
      const double r = sqrt(rx * rx + ry * ry);
      value = 0.5 - 0.5 * tanh((r - P.radius) / (2.0 * kSqrt2 * P.cn));
    } else {
      const double y0 = P.cy + P.amplitude * cos(2.0 * M_PI * P.wavenumber * x / fmax(P.lx, 1.0e-12));
      value = 0.5 - 0.5 * tanh((y - y0) / (2.0 * kSqrt2 * P.cn));
    }
  }
  c.at(i, j) = P.invert_phase ? (1.0 - value) : value;
}

__global__ void k_init_u(Fv u, Grid G, InitParams P, int full) {
  const long long nxg = u.nx + 2 * u.g, nyg = u.ny + 2 * u.g;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nxg * nyg) return;
  const int i = (int)(t / nyg) - u.g, j = (int)(t % nyg) - u.g;
  if (P.velocity_profile == 1) {
    const double y = ((double)j + 0.5) * G.dy;
    u.at(i, j) = -P.omega * (y - P.rcy);
    return;
  }
  if (i < 0 || i >= u.nx || j < 0 || j >= u.ny || !full) return;
  if (P.couette) {
    const double y = ((double)j + 0.5) * G.dy;
    u.at(i, j) = P.ub + (P.ut - P.ub) * y / fmax(P.ly, 1.0e-30);
  } else {
    u.at(i, j) = P.advect_u;
  }
}
__global__ void k_init_v(Fv v, Grid G, InitParams P) {
  const long long nxg = v.nx + 2 * v.g, nyg = v.ny + 2 * v.g;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nxg * nyg) return;
  const int i = (int)(t / nyg) - v.g, j = (int)(t % nyg) - v.g;
  if (P.velocity_profile == 1) {
    const double x = ((double)i + 0.5) * G.dx;
    v.at(i, j) = P.omega * (x - P.rcx);
    return;
  }
  if (i < 0 || i >= v.nx || j < 0 || j >= v.ny) return;
  v.at(i, j) = P.advect_v;
}

}  // namespace

// ---------------------------------------------------------------------------------------------------
// Handle
// ---------------------------------------------------------------------------------------------------
// A multigrid hierarchy on the device (dn_multigrid.cuh): lv[0] is the finest level, whose arrays may belong to
// the caller; levels >= 1 own theirs.  Empty when the grid does not coarsen to <= kMgCoarseMax cells.
struct MgHier {
  struct Lv {
    int nx = 0, ny = 0;
    const double *a64 = nullptr;  // FP64 operator slots (the source of the coarse operators)
    double *a64_own = nullptr;
    const float *a = nullptr;
    float *x = nullptr, *b = nullptr, *r = nullptr;
  };
  std::vector<Lv> lv;
  float *inv = nullptr;  // the coarsest level's inverse
  int *flag = nullptr;
  MgChain *dchain = nullptr;  // the levels as one device record (the cluster inner solve reads it)
  MgFold fold{};
  double mass = 0.0;  // uniform diagonal term of level 0 (CH: the shift s)
  int singular = 0;   // pure-Neumann / periodic pressure: shift the coarsest matrix's null space away
  int levels() const { return (int)lv.size(); }
};

// Kernel launches recorded per region of a solve graph, so that a replay can count the launches it ran:
// once, per outer cycle, per multigrid inner iteration, per IC inner solve.
struct DcNodes {
  long long fixed = 0, cycle = 0, iter = 0, ic = 0;
  long long make = 0;  // the IC inner solver's factor branch, run once in a solve that uses it
};

struct dn_handle {
  dn_config cfg;
  int device = 0;
  int num_sms = 148;
  int cta_cap = 148;  // CTAs one persistent launch may take: num_sms / device_share
  int bicg_occ = 1;   // co-resident CTAs per SM of k_bicgstab alone
  cudaStream_t stream = nullptr;
  Grid G;
  BCSet bc;
  bool has_dirichlet = false;
  Fv f[DN_F_COUNT];
  // ghosted work fields
  Fv mob, lap, bih, mu_t, afx, afy, arhs, dfx, dfy, ddiv, E_new, cmid, mm, pe, urhs, vrhs, hu, hv, sm_c, sm_u, sm_v;
  // compact Krylov vectors
  long long n = 0;
  double *b = nullptr, *x = nullptr, *r = nullptr, *z = nullptr, *y = nullptr, *p0 = nullptr, *p1 = nullptr,
         *ap = nullptr;
  // pressure operator + factor
  double *a5 = nullptr, *l5 = nullptr, *d5 = nullptr, *dinv5 = nullptr;
  bool p_factor_valid = false;
  int p_factor_kind = 0;
  // CH operator + factor
  double *a13 = nullptr, *l13 = nullptr, *d13 = nullptr, *dinv13 = nullptr;
  Rows13 rows13{};       // ordered factor rows for the ring-based level sweeps (y not periodic)
  bool rows13_ok = false;
  double ch_alpha0 = -1.0;
  int ch_prec = kPrecLDLT;  // kPrecLDLT or kPrecDiag
  // momentum
  long long nm = 0;
  MomLayout ml;
  double *mcoef = nullptr;
  int *mtgt = nullptr;
  double *mtcoef = nullptr;  // M^T for the momentum adjoint (allocated on its first call)
  int *mttgt = nullptr;
  double *mb = nullptr, *mx = nullptr, *mr = nullptr, *mrhat = nullptr, *mp0 = nullptr, *mp1 = nullptr, *mv0 = nullptr,
         *mv1 = nullptr, *mphat = nullptr, *ms = nullptr, *mshat = nullptr, *mt = nullptr, *mupd = nullptr,
         *mdinv = nullptr;
  // synchronisation + scratch
  unsigned int *bar_count = nullptr, *bar_gen = nullptr, *prog = nullptr;
  int *status = nullptr;
  double *partials = nullptr;
  double *scal = nullptr;       // device scalars
  double *prof = nullptr;       // device profiling counters of the last pressure solve (64 doubles)
  double *host_scal = nullptr;  // pinned
  int max_coop_blocks = 0;
  int nsweep = 0;   // 32-line sweep warps of the global-memory wavefront (periodic x)
  int nsweep5 = 0;  // 31-line sweep warps of the staged wavefront
  // staged wavefront: hand-over lines, periodic-x wrap lines and launch shape
  double *bnd_f = nullptr, *bnd_b = nullptr, *wline0 = nullptr, *zlast = nullptr;
  double *dcdm_dirs = nullptr, *dcdm_adirs = nullptr;  // split_dcdm_icpcg direction history, [keep][n] each
  double *mon = nullptr;  // pressure-solve monitor record [mon_cap][4] (dn_set_pressure_monitor), device
  int mon_cap = 0, mon_count = 0;
  std::vector<double> mon_host;  // the same record for the host-driven solvers
  int dcdm_keep = 0;
  int sw5 = 0;                 // sweep warps per CTA, 0 = staged path unavailable
  int sw5_budget = 0;          // the most sweep warps per CTA the shared memory allows
  long long rows_per_cta = 512;  // rows per CTA of the PCG kernels' SpMV / update phases
  int sw5_blocks_max = 0;      // co-resident CTAs of k_pcg<5,3> (k_pcg<5,4> with periodic x) at sw5 warps
  int sw5_blocks_by_sw[kSweepWarpsPerCta + 1] = {};  // the same for each sweep-warp count up to sw5_budget
  size_t sw5_warp_smem[2] = {0, 0};  // per sweep warp, [constant operator, variable operator]
  int smem_optin = 0;
  double initial_mass = 0.0;
  long long launches = 0;
  std::string err;
  std::vector<void *> allocations;
  cudaEvent_t ev[5] = {};
  cudaEvent_t kev[2] = {};
  double phase_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // ch, momentum, pressure, correction, pressure PCG kernel,
                                                 // CH PCG kernel, BiCGSTAB kernel, pressure PCG iterations
  // mixed-precision form: FP32 operator, factor and inner Krylov vectors; FP32 staged launch shape
  float *fa5 = nullptr, *fl5 = nullptr, *fdinv5 = nullptr;
  float *fb = nullptr, *fx = nullptr, *fr = nullptr, *fz = nullptr, *fy = nullptr, *fp0 = nullptr, *fp1 = nullptr,
        *fap = nullptr;
  int sw5f = 0, sw5f_blocks_max = 0;
  size_t sw5f_warp_smem[2] = {0, 0};
  // mixed form, multigrid-preconditioned inner CG (dn_multigrid.cuh): the pressure hierarchy (level 0 = the
  // FP32 pressure operator fa5, with the inner CG's r / z and fy as its right-hand side / iterate / residual)
  // and the CH preconditioner's hierarchy (level 0 = the shifted Laplacian K + s I, own buffers).
  MgHier mgp, mgc;
  double *mg_scal = nullptr, *mg_part = nullptr;  // CG scalars and per-CTA partial sums (one solve at a time)
  // one V-cycle of a hierarchy for one (right-hand side, result) pair, captured once as a CUDA graph
  struct MgGraph {
    const MgHier *H;
    const float *b0;
    const float *x0;
    cudaGraphExec_t exec;
    long long nodes;
  };
  std::vector<MgGraph> mg_graphs;
  // graph capture: side streams for conditional node bodies, nested up to kCapDepth deep; `capturing` while
  // the handle's work is being recorded into a graph (no read-backs then: results go to `rec`)
  cudaStream_t cap_streams[kCapDepth] = {};
  int cap_depth = 0;
  bool capturing = false;
  double *rec = nullptr;  // device records of the recorded solves and steps (kRecCount doubles)
  long long graph_epoch = 0;  // bumped when a launch shape changes: recorded graphs are made again
  // the eager mixed solves, each captured once with its loops on the device: [0] pressure, [1] CH
  struct SolveGraph {
    cudaGraphExec_t exec = nullptr;
    long long epoch = -1;
    DcNodes nodes;
  };
  SolveGraph dc_graph[2];
  bool ch_mg_ok = false;  // the (K + s I) hierarchy built for ch_mg_alpha0 is usable
  long long mg_cluster_cells = kMgClusterCells;  // level-0 grids this small: each inner CG is one cluster launch
  // captured steps (dn_set_step_graph): the step recorded once into a graph and replayed
  bool graph_steps = false;  // replay captured steps where the step allows it
  bool steady = false;       // an eager step with step >= 1 has made every operator, factor and hierarchy
  cudaGraphExec_t step_exec = nullptr;
  long long step_epoch = -1;
  dn_report step_rep{};      // the report fields fixed at capture (preconditioner kinds)
  long long step_nodes = 0;  // kernel launches of one replay outside the mixed solves' loops
  DcNodes step_dcn[2];       // the mixed solves' loops: [0] pressure, [1] CH
  long long step_retry = 0;  // kernel launches of the CH solve's retry branch (run after a breakdown only)
  cudaEvent_t cap_ev = nullptr;  // joins this handle's branch of a batch capture
  long long uid = 0;             // unique among the process's handles (a batch graph names its handles by it)
  // the batch graph this handle leads (dn_step_batch with it first): every handle's step in one graph
  struct BatchGraph {
    std::vector<long long> uids, epochs;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr;
  } batch;
  // mixed CH solve: FP32 13-point operator and CG vectors; the alpha0 its operator and hierarchy were built for
  float *fa13 = nullptr, *cx32 = nullptr, *cr32 = nullptr, *cz32 = nullptr, *cp32 = nullptr, *cq32 = nullptr,
        *ct32 = nullptr, *cb32 = nullptr;
  double ch_mg_alpha0 = -1.0;
  bool ch_mg = false;  // the CH solve runs the mixed form (FP64 defect correction around the FP32 inner CG)
  bool mgp_split_ready = false;  // the split operator's FP32 copy and hierarchy exist
  bool mixed_used_mg = false;  // the last mixed pressure solve started with the multigrid inner solver
  int refinement_cycles = 0;  // outer cycles of the last mixed-precision pressure solve
  dn_diag last_diag{};        // diagnostics at the end of the last dn_step (compute_diagnostics, solver.cpp:276)
  int step = 0;  // step index of the step in progress (split extrapolation, operators.cpp:416)
  double pcg_split_ms[3] = {0, 0, 0};  // pressure PCG, in-kernel: [P1 SpMV+barrier, P2 update+barrier, sweeps]
};

namespace {

bool solve_ch(const dn_config &c) {
  return c.mode != DN_MODE_ADVECTION_ONLY && !(c.mode == DN_MODE_SINGLE_PHASE || c.freeze_ch);
}
bool compute_mu(const dn_config &c) { return c.mode != DN_MODE_ADVECTION_ONLY && c.mode != DN_MODE_SINGLE_PHASE; }
bool use_split(const dn_config &c) {
  return c.pressure_scheme == DN_P_SPLIT_ICPCG || c.pressure_scheme == DN_P_SPLIT_ILDLT_PCG ||
         c.pressure_scheme == DN_P_SPLIT_DCDM_ICPCG;
}
double rho_ref_of(const dn_config &c) { return std::min(1.0, c.density_ratio); }

dn_status fail(dn_handle *h, dn_status s, const std::string &msg) {
  if (h) h->err = msg;
  return s;
}

#define DN_CUDA(h, call)                                                                        \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) return fail(h, DN_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define DN_TRY(expr)              \
  do {                            \
    dn_status s_ = (expr);        \
    if (s_ != DN_OK) return s_;   \
  } while (0)

template <typename T>
dn_status dalloc(dn_handle *h, T **p, size_t count) {
  void *q = nullptr;
  DN_CUDA(h, cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
  DN_CUDA(h, cudaMemsetAsync(q, 0, std::max<size_t>(count, 1) * sizeof(T), h->stream));
  h->allocations.push_back(q);
  *p = static_cast<T *>(q);
  return DN_OK;
}

dn_status falloc(dn_handle *h, Fv &f, int nx, int ny, double init) {
  f.nx = nx;
  f.ny = ny;
  f.g = h->cfg.ghost;
  DN_TRY(dalloc(h, &f.d, f.size()));
  if (init != 0.0) {
    const long long n = (long long)f.size();
    k_fill<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(f.d, init, n);
    h->launches++;
  }
  return DN_OK;
}

inline unsigned blocks_for(long long n, int bs = 256) { return (unsigned)((n + bs - 1) / bs); }

dn_status check_launch(dn_handle *h, const char *what) {
  h->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(h, DN_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return DN_OK;
}

// A launch with programmatic stream serialization: the kernel (which opens with pdl_entry) may be launched
// while its predecessor in the stream is still finishing, and waits for it on the device.
template <typename... KArgs, typename... Args>
dn_status launch_pdl(dn_handle *h, const char *name, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                     Args &&...args) {
  cudaLaunchConfig_t lc{};
  lc.gridDim = grid;
  lc.blockDim = block;
  lc.dynamicSmemBytes = smem;
  lc.stream = h->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&lc, kernel, std::forward<Args>(args)...);
  if (e != cudaSuccess) return fail(h, DN_ERR_CUDA, std::string(name) + ": " + cudaGetErrorString(e));
  return check_launch(h, name);
}

bool is_uish(int id) { return id == DN_F_U || id == DN_F_U_PREV || id == DN_F_U_STAR || id == DN_F_SFX_U || id == DN_F_HU_PREV; }
bool is_vish(int id) { return id == DN_F_V || id == DN_F_V_PREV || id == DN_F_V_STAR || id == DN_F_SFY_V || id == DN_F_HV_PREV; }

// ---- boundary conditions
dn_status bc(dn_handle *h, const Fv &f, int kind) {
  const BCSet &B = h->bc;
  BCSide L{}, R{}, Bt{}, T{};
  if (kind == kBCPressure) {
    L = B.p[0]; R = B.p[1]; Bt = B.p[2]; T = B.p[3];
  } else if (kind == kBCU) {
    L = B.u[0]; R = B.u[1]; Bt = B.u[2]; T = B.u[3];
    k_bc_faces_u<<<blocks_for(f.ny), 256, 0, h->stream>>>(f, h->G, L, R);
    DN_TRY(check_launch(h, "k_bc_faces_u"));
  } else if (kind == kBCV) {
    L = B.v[0]; R = B.v[1]; Bt = B.v[2]; T = B.v[3];
    k_bc_faces_v<<<blocks_for(f.nx), 256, 0, h->stream>>>(f, h->G, Bt, T);
    DN_TRY(check_launch(h, "k_bc_faces_v"));
  }
  const long long nghost = 2LL * f.g * f.ny + 2LL * f.g * (f.nx + 2 * f.g);
  k_bc_ghosts<<<blocks_for(nghost), 256, 0, h->stream>>>(f, h->G, kind, L, R, Bt, T);
  return check_launch(h, "k_bc_ghosts");
}

dn_status copy_field(dn_handle *h, const Fv &dst, const Fv &src) {
  DN_CUDA(h, cudaMemcpyAsync(dst.d, src.d, src.size() * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  return DN_OK;
}

dn_status fill_field(dn_handle *h, const Fv &f, double v) {
  k_fill<<<blocks_for((long long)f.size()), 256, 0, h->stream>>>(f.d, v, (long long)f.size());
  return check_launch(h, "k_fill");
}

// mean of a field's interior into h->scal[slot] (device)
dn_status field_mean(dn_handle *h, const Fv &f, int slot) {
  const int nb = 128;
  k_field_sum<<<nb, 256, 0, h->stream>>>(f, 1.0, h->partials);
  DN_TRY(check_launch(h, "k_field_sum"));
  k_finish_mean<<<1, 32, 0, h->stream>>>(h->partials, nb, (double)f.nx * f.ny, h->scal + slot);
  return check_launch(h, "k_finish_mean");
}
dn_status subtract_mean(dn_handle *h, const Fv &f) {
  DN_TRY(field_mean(h, f, 0));
  k_add_scalar_interior<<<blocks_for((long long)f.nx * f.ny), 256, 0, h->stream>>>(f, h->scal);
  return check_launch(h, "k_add_scalar_interior");
}

dn_status read_scalars(dn_handle *h, int count, double *out) {
  DN_CUDA(h, cudaMemcpyAsync(h->host_scal, h->scal + 8, count * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  std::memcpy(out, h->host_scal, count * sizeof(double));
  return DN_OK;
}

dn_status read_status(dn_handle *h, int *status) {
  DN_CUDA(h, cudaMemcpyAsync(h->host_scal + 32, h->status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  std::memcpy(status, h->host_scal + 32, sizeof(int));
  return DN_OK;
}

dn_status reset_sync(dn_handle *h) {
  DN_CUDA(h, cudaMemsetAsync(h->bar_count, 0, sizeof(unsigned int), h->stream));
  DN_CUDA(h, cudaMemsetAsync(h->status, 0, sizeof(int), h->stream));
  DN_CUDA(h, cudaMemsetAsync(h->prog, 0, 2 * (size_t)kMaxBlocks * 8 * sizeof(unsigned int), h->stream));
  return DN_OK;
}

dn_status dev_status_to_dn(dn_handle *h, int st) {
  switch (st) {
  case kDevOk: return DN_OK;
  case kDevTimeout: return fail(h, DN_ERR_TIMEOUT, "device wait timed out (grid barrier or wavefront flag)");
  case kDevPcgBreakdownRz0: return fail(h, DN_ERR_PCG_BREAKDOWN, "pcg preconditioner breakdown: non-positive r^T M^{-1} r");
  case kDevPcgBreakdownPap: return fail(h, DN_ERR_PCG_BREAKDOWN, "pcg breakdown: p^T A p is invalid");
  case kDevPcgBreakdownRz: return fail(h, DN_ERR_PCG_BREAKDOWN, "pcg preconditioner breakdown: non-positive new r^T M^{-1} r");
  case kDevBicgRho: return fail(h, DN_ERR_BICGSTAB_BREAKDOWN, "bicgstab breakdown: invalid rho");
  case kDevBicgRhatV: return fail(h, DN_ERR_BICGSTAB_BREAKDOWN, "bicgstab breakdown: invalid r_hat^T A M^{-1} p");
  case kDevBicgTT: return fail(h, DN_ERR_BICGSTAB_BREAKDOWN, "bicgstab breakdown: invalid t^T t");
  case kDevBicgOmega: return fail(h, DN_ERR_BICGSTAB_BREAKDOWN, "bicgstab breakdown: invalid omega");
  case kDevJacobiDiverged: return fail(h, DN_ERR_NONFINITE, "Jacobi pressure solve diverged");
  default: return fail(h, DN_ERR_CUDA, "unknown device status");
  }
}

// ---- persistent PCG launch
// The arguments and launch shape of the persistent PCG kernel k_pcg<S, SWEEP> (and of k_prec_apply, which
// runs its sweeps alone).
template <int S, int SWEEP>
dn_status pcg_launch_args(dn_handle *h, const double *a, const double *l, const double *dinv, int prec, int project,
                          int max_it, double tol, PcgArgs &P, size_t &dyn_smem_out, int &blocks_out) {
  P.A = SpOp{a, (int)h->n, h->G.nx, h->G.ny, h->G.px, h->G.py};
  P.l = l;
  P.dinv = dinv;
  P.prec = prec;
  P.b = h->b;
  P.x = h->x;
  P.r = h->r;
  P.z = h->z;
  P.y = h->y;
  P.p0 = h->p0;
  P.p1 = h->p1;
  P.ap = h->ap;
  P.project = project;
  P.max_it = max_it;
  P.tol = tol;
  P.tol_abs = tol;  // the reference stops on rel < tol || abs < tol
  P.bar_count = h->bar_count;
  P.bar_gen = h->bar_gen;
  P.status = h->status;
  P.prog_f = h->prog;
  P.prog_b = h->prog + kMaxBlocks * 8;
  P.partials = h->partials;
  P.out = h->scal + 8;
  P.nsweep = h->nsweep;
  P.warp_smem = 0;
  P.rows13 = Rows13{};
  size_t dyn_smem = 0;
  P.seq_lines = 0;
  P.mon = S == 5 ? h->mon : nullptr;
  P.mon_cap = S == 5 ? h->mon_cap : 0;
  if (S == 13 && SWEEP == 1 && h->rows13.lval != nullptr) {  // ring of kLvlRing levels x nx doubles
    P.rows13 = h->rows13;
    dyn_smem = (size_t)kLvlRing * h->G.nx * sizeof(double);
  } else if (S == 13 && SWEEP == 1 && h->G.py &&
             (size_t)seq13_smem_doubles_per_row() * h->G.ny * sizeof(double) <= kSeqSmemMax) {
    P.seq_lines = 1;  // periodic y: line-staged sequential sweeps
    dyn_smem = (size_t)seq13_smem_doubles_per_row() * h->G.ny * sizeof(double);
  }
  // about 512 rows per CTA: the SpMV / update phases are latency-bound, so more CTAs shorten them
  const long long rows_per_cta = h->rows_per_cta;
  int blocks = (int)std::min<long long>(h->cta_cap,
                                        std::max<long long>(h->nsweep, (h->n + rows_per_cta - 1) / rows_per_cta));
  blocks = std::max(blocks, (h->nsweep + kBlock / 32 - 1) / (kBlock / 32));  // the wavefront warps' CTAs
  blocks = std::max(1, std::min(blocks, h->max_coop_blocks));
  if (SWEEP == 3 || SWEEP == 4) {
    const dn_config &c = h->cfg;
    const bool var = !use_split(c);
    Sweep5 &W = P.s5;
    W.nx = h->G.nx;
    W.ny = h->G.ny;
    W.n = (int)h->n;
    W.px = h->G.px;
    W.py = h->G.py;
    W.prec = prec;
    W.varcoef = var ? 1 : 0;
    W.aW = a;
    W.aS = a + h->n;
    W.aN = a + 3 * h->n;
    W.aE = a + 4 * h->n;
    W.cx = -(1.0 / (h->G.dx * h->G.dx));
    W.cy = -(1.0 / (h->G.dy * h->G.dy));
    W.dinv = dinv;
    W.r = h->r;
    W.y = h->y;
    W.z = h->z;
    W.bnd_f = h->bnd_f;
    W.bnd_b = h->bnd_b;
    W.wline0 = h->wline0;
    W.zlast = h->zlast;
    W.prog_f = h->prog;
    W.prog_b = h->prog + kMaxBlocks * 8;
    W.nsweep = h->nsweep5;
    W.sw = h->sw5;
    W.status = h->status;
    P.warp_smem = (int)h->sw5_warp_smem[var ? 1 : 0];
    W.warp_smem = P.warp_smem;
    W.prof = h->prof;
    dyn_smem = 64 + (size_t)h->sw5 * P.warp_smem;
    const int sweep_ctas = (h->nsweep5 + h->sw5 - 1) / h->sw5;
    blocks = std::max(blocks, sweep_ctas);
    blocks = std::min(blocks, h->sw5_blocks_by_sw[h->sw5]);
    if (blocks < sweep_ctas) return fail(h, DN_ERR_UNSUPPORTED, "not enough co-resident CTAs for the wavefront");
  }
  if (SWEEP == 0 && (long long)blocks * (kBlock / 32) < h->nsweep)
    return fail(h, DN_ERR_UNSUPPORTED, "grid too wide for the co-resident wavefront warps");
  dyn_smem_out = dyn_smem;
  blocks_out = blocks;
  return DN_OK;
}

// results of a persistent solve (out[0..count) and its status word) into a record block: [0, count) and
// [count] = the status
__global__ void k_rec_copy(const double *out, int count, const int *status, double *dst) {
  if (threadIdx.x != 0) return;
  for (int k = 0; k < count; ++k) dst[k] = out[k];
  dst[count] = (double)*status;
}

// 1 into a record slot (a branch that ran)
__global__ void k_rec_flag(double *dst) {
  if (threadIdx.x == 0) *dst = 1.0;
}
// the condition of the CH solve's retry with the diagonal preconditioner: the PCG broke down
__global__ void k_cond_breakdown(const int *status, cudaGraphConditionalHandle hd) {
  if (threadIdx.x != 0) return;
  const int st = *status;
  cudaGraphSetConditional(hd, (st == kDevPcgBreakdownRz0 || st == kDevPcgBreakdownPap || st == kDevPcgBreakdownRz)
                                  ? 1u : 0u);
}
// sqrt(sum r^2 / sum b^2) of per-CTA pairs (k_residual_partials), added in a fixed order by one warp
__global__ void k_eq_residual(const double *partials, int nb, double *dst) {
  double rs = 0.0, bs = 0.0;
  for (int k = threadIdx.x; k < nb; k += 32) {
    rs += partials[2 * k];
    bs += partials[2 * k + 1];
  }
  rs = warp_sum(rs);
  bs = warp_sum(bs);
  if (threadIdx.x == 0) *dst = sqrt(rs / (bs < 1.0e-30 ? 1.0e-30 : bs));
}

// Slots of a step's record (h->rec + kRecStep): the persistent solves' out[0..4) and status, and the rest
// of what dn_step reports, so that a step recorded into a graph is read back once.
constexpr int kRecStep = 32;
enum StepSlot {
  kSChPcg = 0,     // CH PCG: iterations, abs, rel, iterate residual; [4] status
  kSChRetry = 5,   // the CH PCG broke down and was retried with the diagonal preconditioner
  kSChEq = 6,      // CH equation residual |b - A x| / |b|
  kSMom = 8,       // BiCGSTAB: iterations, residual, ...; [12] status
  kSP = 16,        // pressure PCG: iterations, abs, rel, iterate residual; [20] status
  kSPFactor = 21,  // the pressure factor's status (variable operator)
};

// rec: where a solve recorded into a graph (h->capturing) leaves its out[0..4) and status (k_rec_copy);
// nothing is read back then
template <int S, int SWEEP>
dn_status run_pcg(dn_handle *h, const double *a, const double *l, const double *dinv, int prec, int project, int max_it,
                  double tol, double out[4], double *rec = nullptr) {
  PcgArgs P{};
  size_t dyn_smem = 0;
  int blocks = 1;
  DN_TRY((pcg_launch_args<S, SWEEP>(h, a, l, dinv, prec, project, max_it, tol, P, dyn_smem, blocks)));
  DN_TRY(reset_sync(h));
  void *args[] = {&P};
  if (h->capturing) {
    if (!rec) return fail(h, DN_ERR_UNSUPPORTED, "a recorded PCG solve needs a record");
    DN_CUDA(h, cudaLaunchCooperativeKernel((const void *)k_pcg<S, SWEEP>, dim3(blocks), dim3(kBlock), args, dyn_smem,
                                           h->stream));
    h->launches++;
    k_rec_copy<<<1, 32, 0, h->stream>>>(h->scal + 8, 4, h->status, rec);
    out[0] = out[1] = out[2] = out[3] = 0.0;
    return check_launch(h, "k_rec_copy");
  }
  cudaEventRecord(h->kev[0], h->stream);
  DN_CUDA(h, cudaLaunchCooperativeKernel((const void *)k_pcg<S, SWEEP>, dim3(blocks), dim3(kBlock), args, dyn_smem,
                                         h->stream));
  cudaEventRecord(h->kev[1], h->stream);
  h->launches++;
  int st = 0;
  DN_TRY(read_status(h, &st));
  if (st != kDevOk) return dev_status_to_dn(h, st);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, h->kev[0], h->kev[1]);
  h->phase_ms[S == 5 ? 4 : 5] += ms;
  double tmp[7];
  DN_TRY(read_scalars(h, 7, tmp));
  for (int k = 0; k < 4; ++k) out[k] = tmp[k];
  if (S == 5) {
    h->pcg_split_ms[0] = tmp[4];
    h->pcg_split_ms[1] = tmp[5];
    h->pcg_split_ms[2] = tmp[6];
  }
  return DN_OK;
}

// One FP32 inner PCG solve (the persistent kernel instantiated for float) on the handle's FP32 buffers.
dn_status run_pcg32(dn_handle *h, int prec, int project, int max_it, double tol, double out[4]) {
  PcgArgsT<float> P{};
  P.mon = nullptr;
  P.mon_cap = 0;
  P.A = SpOpT<float>{h->fa5, (int)h->n, h->G.nx, h->G.ny, h->G.px, h->G.py};
  P.l = h->fl5;
  P.dinv = h->fdinv5;
  P.prec = prec;
  P.b = h->fb;
  P.x = h->fx;
  P.r = h->fr;
  P.z = h->fz;
  P.y = h->fy;
  P.p0 = h->fp0;
  P.p1 = h->fp1;
  P.ap = h->fap;
  P.project = project;
  P.max_it = std::max(1, max_it);
  P.tol = tol;
  P.tol_abs = 0.0;  // an inner solve stops on its relative residual only
  P.bar_count = h->bar_count;
  P.bar_gen = h->bar_gen;
  P.status = h->status;
  P.prog_f = h->prog;
  P.prog_b = h->prog + kMaxBlocks * 8;
  P.partials = h->partials;
  P.out = h->scal + 8;
  P.nsweep = h->nsweep;
  P.warp_smem = 0;
  size_t dyn_smem = 0;
  // about 512 rows per CTA: the SpMV / update phases are latency-bound, so more CTAs shorten them
  const long long rows_per_cta = h->rows_per_cta;
  int blocks = (int)std::min<long long>(h->cta_cap,
                                        std::max<long long>(h->nsweep, (h->n + rows_per_cta - 1) / rows_per_cta));
  blocks = std::max(blocks, (h->nsweep + kBlock / 32 - 1) / (kBlock / 32));  // the wavefront warps' CTAs
  blocks = std::max(1, std::min(blocks, h->max_coop_blocks));
  const bool staged = h->sw5f > 0;
  if (staged) {
    const bool var = !use_split(h->cfg);
    Sweep5T<float> &W = P.s5;
    W.nx = h->G.nx;
    W.ny = h->G.ny;
    W.n = (int)h->n;
    W.px = h->G.px;
    W.py = h->G.py;
    W.prec = prec;
    W.varcoef = var ? 1 : 0;
    W.aW = h->fa5;
    W.aS = h->fa5 + h->n;
    W.aN = h->fa5 + 3 * h->n;
    W.aE = h->fa5 + 4 * h->n;
    W.cx = (float)(-(1.0 / (h->G.dx * h->G.dx)));
    W.cy = (float)(-(1.0 / (h->G.dy * h->G.dy)));
    W.dinv = h->fdinv5;
    W.r = h->fr;
    W.y = h->fy;
    W.z = h->fz;
    W.bnd_f = reinterpret_cast<float *>(h->bnd_f);  // the FP64 hand-over buffers, reused
    W.bnd_b = reinterpret_cast<float *>(h->bnd_b);
    W.wline0 = reinterpret_cast<float *>(h->wline0);
    W.zlast = reinterpret_cast<float *>(h->zlast);
    W.prog_f = h->prog;
    W.prog_b = h->prog + kMaxBlocks * 8;
    W.nsweep = h->nsweep5;
    W.sw = h->sw5f;
    W.status = h->status;
    P.warp_smem = (int)h->sw5f_warp_smem[var ? 1 : 0];
    W.warp_smem = P.warp_smem;
    W.prof = h->prof;
    dyn_smem = 64 + (size_t)h->sw5f * P.warp_smem;
    const int sweep_ctas = (h->nsweep5 + h->sw5f - 1) / h->sw5f;
    blocks = std::max(blocks, sweep_ctas);
    blocks = std::min(blocks, h->sw5f_blocks_max);
    if (blocks < sweep_ctas) return fail(h, DN_ERR_UNSUPPORTED, "not enough co-resident CTAs for the wavefront");
  } else if ((long long)blocks * (kBlock / 32) < h->nsweep) {
    return fail(h, DN_ERR_UNSUPPORTED, "grid too wide for the co-resident wavefront warps");
  }
  DN_TRY(reset_sync(h));
  void *args[] = {&P};
  const void *kern = !staged ? (const void *)k_pcg<5, 0, float>
                     : h->G.px ? (const void *)k_pcg<5, 4, float>
                               : (const void *)k_pcg<5, 3, float>;
  if (h->capturing) {  // recorded into a graph: status and results stay on the device (h->status, h->scal + 8)
    DN_CUDA(h, cudaLaunchCooperativeKernel(kern, dim3(blocks), dim3(kBlock), args, dyn_smem, h->stream));
    h->launches++;
    out[0] = out[1] = out[2] = out[3] = 0.0;
    return DN_OK;
  }
  cudaEventRecord(h->kev[0], h->stream);
  DN_CUDA(h, cudaLaunchCooperativeKernel(kern, dim3(blocks), dim3(kBlock), args, dyn_smem, h->stream));
  cudaEventRecord(h->kev[1], h->stream);
  h->launches++;
  int st = 0;
  DN_TRY(read_status(h, &st));
  if (st != kDevOk) return dev_status_to_dn(h, st);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, h->kev[0], h->kev[1]);
  h->phase_ms[4] += ms;
  double tmp[7];
  DN_TRY(read_scalars(h, 7, tmp));
  for (int k = 0; k < 4; ++k) out[k] = tmp[k];
  h->pcg_split_ms[0] += tmp[4];
  h->pcg_split_ms[1] += tmp[5];
  h->pcg_split_ms[2] += tmp[6];
  return DN_OK;
}

// ---------------------------------------------------------------------------------------------------
// Multigrid-preconditioned FP32 inner CG of the mixed form (kernels and design: dn_multigrid.cuh)
// ---------------------------------------------------------------------------------------------------
MgLevel mg_level(const MgHier &H, int l) {
  const MgHier::Lv &m = H.lv[l];
  return MgLevel{m.a, m.x, m.b, m.r, m.nx, m.ny};
}

// H's levels (fixed once its level 0 is set) as one device record, for the cluster inner solve
dn_status mg_upload_chain(dn_handle *h, MgHier &H) {
  if (H.levels() == 0) return DN_OK;
  MgChain ch{};
  for (int l = 0; l < H.levels(); ++l) ch.lv[l] = mg_level(H, l);
  ch.first = 0;
  ch.last = H.levels() - 1;
  ch.fold = H.fold;
  ch.inv = H.inv;
  DN_TRY(dalloc(h, &H.dchain, 1));
  DN_CUDA(h, cudaMemcpyAsync(H.dchain, &ch, sizeof(ch), cudaMemcpyHostToDevice, h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));  // `ch` lives on this stack frame
  return DN_OK;
}

// Levels 1.. of a hierarchy whose level 0 is an nx x ny grid: halve both extents while they are even and >= 4
// and the level is larger than the direct coarse solve.  Leaves H empty when the grid never gets there.
dn_status mg_alloc(dn_handle *h, MgHier &H, int nx, int ny, const BCSide *sides) {
  std::vector<std::pair<int, int>> dims{{nx, ny}};
  int lx = nx, ly = ny;
  while ((long long)lx * ly > kMgCoarseMax && lx % 2 == 0 && ly % 2 == 0 && lx >= 4 && ly >= 4 &&
         (int)dims.size() < kMgMaxLevels) {
    lx /= 2;
    ly /= 2;
    dims.push_back({lx, ly});
  }
  H.lv.clear();
  if ((long long)lx * ly > kMgCoarseMax) return DN_OK;
  dn_status s = DN_OK;
  auto A = [&](dn_status st) {
    if (s == DN_OK) s = st;
  };
  H.lv.resize(dims.size());
  H.lv[0].nx = nx;
  H.lv[0].ny = ny;
  for (size_t l = 1; l < dims.size(); ++l) {
    MgHier::Lv &m = H.lv[l];
    m.nx = dims[l].first;
    m.ny = dims[l].second;
    const size_t nl = (size_t)m.nx * m.ny;
    double *a64 = nullptr;
    float *a = nullptr;
    A(dalloc(h, &a64, 5 * nl));
    A(dalloc(h, &a, 5 * nl));
    A(dalloc(h, &m.x, nl));
    A(dalloc(h, &m.b, nl));
    A(dalloc(h, &m.r, nl));
    m.a64 = m.a64_own = a64;
    m.a = a;
  }
  A(dalloc(h, &H.inv, (size_t)kMgCoarseMax * kMgCoarseMax));
  A(dalloc(h, &H.flag, 1));
  if (s != DN_OK) {
    H.lv.clear();
    return s;
  }
  for (int k = 0; k < 4; ++k) H.fold.s[k] = sides[k].type == DN_BC_DIRICHLET ? -1.0f : 1.0f;
  H.fold.px = h->G.px;
  H.fold.py = h->G.py;
  cudaFuncSetAttribute(k_mg_coarse_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(sizeof(double) * kMgCoarseMax * kMgCoarseMax));
  return DN_OK;
}

// Coarse operators of H's current level-0 operator and the inverse of the coarsest one; H.flag (device) is
// set when the coarsest matrix has a non-positive pivot.
dn_status mg_setup_launch(dn_handle *h, MgHier &H) {
  if (H.levels() > 0 && (!H.lv[0].a64 || !H.lv[0].a || !H.lv[0].r))
    return fail(h, DN_ERR_INVALID_ARGUMENT, "multigrid level 0 has no operator");
  double mass = H.mass;
  for (int l = 1; l < H.levels(); ++l) {
    const MgHier::Lv &f = H.lv[l - 1];
    MgHier::Lv &m = H.lv[l];
    k_mg_coarsen<<<blocks_for((long long)m.nx * m.ny), 256, 0, h->stream>>>(f.a64, f.nx, f.ny, mass, m.a64_own,
                                                                            const_cast<float *>(m.a), m.nx, m.ny);
    DN_TRY(check_launch(h, "k_mg_coarsen"));
    mass *= 4.0;
  }
  const MgHier::Lv &c = H.lv.back();
  const int nc = c.nx * c.ny;
  k_mg_coarse_inverse<<<1, 256, sizeof(double) * nc * nc, h->stream>>>(c.a64, c.nx, c.ny, h->G.px, h->G.py,
                                                                         H.singular, H.inv, H.flag);
  return check_launch(h, "k_mg_coarse_inverse");
}

// mg_setup_launch, then its flag read back: *usable = false when the coarsest matrix has a non-positive pivot
// (the caller then does not use the hierarchy).
dn_status mg_setup(dn_handle *h, MgHier &H, bool *usable) {
  *usable = false;
  DN_TRY(mg_setup_launch(h, H));
  int flag = 0;
  DN_CUDA(h, cudaMemcpyAsync(h->host_scal + 33, H.flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  std::memcpy(&flag, h->host_scal + 33, sizeof(int));
  *usable = flag == 0;
  return DN_OK;
}

// x0 = B b0: one V-cycle from level 0 with right-hand side b0 and result x0 (level 0's residual buffer is
// H.lv[0].r)
dn_status mg_vcycle_launch(dn_handle *h, MgHier &H, float *b0, float *x0) {
  const int L = H.levels(), px = h->G.px, py = h->G.py;
  H.lv[0].b = b0;
  H.lv[0].x = x0;
  // levels from `bottom` down run inside one CTA (k_mg_bottom); the ones above get a launch per phase
  int bottom = L - 1;
  while (bottom > 0 && (long long)H.lv[bottom - 1].nx * H.lv[bottom - 1].ny <= kMgBottomCells) --bottom;
  auto smooth = [&](const MgLevel &M, int color, int first) -> dn_status {
    return launch_pdl(h, "k_mg_smooth", k_mg_smooth, dim3(blocks_for((long long)M.nx * (M.ny / 2))), dim3(256), 0, M, color, first, px, py);
  };
  for (int l = 0; l < bottom; ++l) {
    const MgLevel F = mg_level(H, l), C = mg_level(H, l + 1);
    for (int k = 0; k < kMgSweeps; ++k) {
      DN_TRY(smooth(F, 0, k == 0));
      DN_TRY(smooth(F, 1, 0));
    }
    DN_TRY(launch_pdl(h, "k_mg_residual", k_mg_residual, dim3(blocks_for((long long)F.nx * F.ny)), dim3(256), 0, F, px, py));
    DN_TRY(launch_pdl(h, "k_mg_restrict", k_mg_restrict, dim3(blocks_for((long long)C.nx * C.ny)), dim3(256), 0, F, C, H.fold));
  }
  MgChain ch{};
  for (int l = 0; l < L; ++l) ch.lv[l] = mg_level(H, l);
  ch.first = bottom;
  ch.last = L - 1;
  ch.fold = H.fold;
  ch.inv = H.inv;
  DN_TRY(launch_pdl(h, "k_mg_bottom", k_mg_bottom, dim3(1), dim3(1024), 0, ch));
  for (int l = bottom - 1; l >= 0; --l) {
    const MgLevel F = mg_level(H, l), C = mg_level(H, l + 1);
    DN_TRY(launch_pdl(h, "k_mg_prolong", k_mg_prolong, dim3(blocks_for((long long)F.nx * F.ny)), dim3(256), 0, C, F, H.fold));
    for (int k = 0; k < kMgSweeps; ++k) {
      DN_TRY(smooth(F, 1, 0));
      DN_TRY(smooth(F, 0, 0));
    }
  }
  return DN_OK;
}

// The V-cycle's ~11 launches per level are replayed from a CUDA graph captured on first use for this
// (hierarchy, b0, x0): the kernels' arguments are the level buffers' pointers, which never change, and the
// operators are rewritten in place by mg_setup.
dn_status mg_vcycle(dn_handle *h, MgHier &H, float *b0, float *x0) {
  if (h->capturing) return mg_vcycle_launch(h, H, b0, x0);  // recorded into the enclosing graph
  for (const dn_handle::MgGraph &g : h->mg_graphs)
    if (g.H == &H && g.b0 == b0 && g.x0 == x0) {
      DN_CUDA(h, cudaGraphLaunch(g.exec, h->stream));
      h->launches += g.nodes;
      return DN_OK;
    }
  const long long before = h->launches;
  DN_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  const dn_status st = mg_vcycle_launch(h, H, b0, x0);
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(h->stream, &graph);
  const long long nodes = h->launches - before;
  h->launches = before;
  if (st != DN_OK || ce != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return st != DN_OK ? st : fail(h, DN_ERR_CUDA, std::string("V-cycle capture: ") + cudaGetErrorString(ce));
  }
  cudaGraphExec_t exec = nullptr;
  const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) return fail(h, DN_ERR_CUDA, std::string("V-cycle graph: ") + cudaGetErrorString(ie));
  h->mg_graphs.push_back(dn_handle::MgGraph{&H, b0, x0, exec, nodes});
  DN_CUDA(h, cudaGraphLaunch(exec, h->stream));
  h->launches += nodes;
  return DN_OK;
}

// ---------------------------------------------------------------------------------------------------
// CUDA graphs with device-side loop control.  A conditional node (while / if) is recorded into the stream
// capture in progress on h->stream: its handle is created on the graph being captured, the node follows
// the capture's current dependencies, and its body is captured into the node's body graph on a side
// stream (h->stream points there while `body` runs).  Kernels inside the graph set the conditions
// (cudaGraphSetConditional), so a whole solve -- its iterations and its stopping decisions -- runs without
// the host.
// ---------------------------------------------------------------------------------------------------
dn_status cap_info(dn_handle *h, cudaGraph_t *g, const cudaGraphNode_t **deps, size_t *nd) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  DN_CUDA(h, cudaStreamGetCaptureInfo(h->stream, &cs, nullptr, g, deps, nd));
  if (cs != cudaStreamCaptureStatusActive) return fail(h, DN_ERR_CUDA, "conditional node outside a stream capture");
  return DN_OK;
}

// a condition handle on the graph being captured; 0 at every launch of the graph until a kernel sets it
dn_status cond_create(dn_handle *h, cudaGraphConditionalHandle *hd) {
  cudaGraph_t g = nullptr;
  DN_TRY(cap_info(h, &g, nullptr, nullptr));
  DN_CUDA(h, cudaGraphConditionalHandleCreate(hd, g, 0, cudaGraphCondAssignDefault));
  return DN_OK;
}

template <class Body>
dn_status cond_node(dn_handle *h, cudaGraphConditionalHandle hd, cudaGraphConditionalNodeType type, Body &&body) {
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  DN_TRY(cap_info(h, &g, &deps, &nd));
  if (h->cap_depth >= kCapDepth) return fail(h, DN_ERR_UNSUPPORTED, "conditional graph nodes nested too deeply");
  cudaGraphNodeParams p{};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = hd;
  p.conditional.type = type;
  p.conditional.size = 1;
  cudaGraphNode_t node = nullptr;
  DN_CUDA(h, cudaGraphAddNode(&node, g, deps, nd, &p));
  cudaStream_t outer = h->stream, side = h->cap_streams[h->cap_depth];
  DN_CUDA(h, cudaStreamBeginCaptureToGraph(side, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal));
  h->stream = side;
  ++h->cap_depth;
  const dn_status st = body();
  --h->cap_depth;
  h->stream = outer;
  cudaGraph_t captured = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(side, &captured);
  DN_TRY(st);
  if (ce != cudaSuccess) return fail(h, DN_ERR_CUDA, std::string("conditional body capture: ") + cudaGetErrorString(ce));
  DN_CUDA(h, cudaStreamUpdateCaptureDependencies(outer, &node, 1, cudaStreamSetCaptureDependencies));
  return DN_OK;
}

// `record` captured into an executable graph (nothing runs); h->capturing is set meanwhile, so the step
// pieces record their results on the device instead of reading them back
template <class Record>
dn_status capture_exec(dn_handle *h, cudaGraphExec_t *exec, Record &&record) {
  *exec = nullptr;
  DN_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  h->capturing = true;
  const dn_status st = record();
  h->capturing = false;
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(h->stream, &g);
  if (st != DN_OK || ce != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return st != DN_OK ? st : fail(h, DN_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
  }
  const cudaError_t ie = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) {
    *exec = nullptr;
    return fail(h, DN_ERR_CUDA, std::string("graph instantiation: ") + cudaGetErrorString(ie));
  }
  return DN_OK;
}

// One FP32 inner solve A e = b by CG preconditioned with `vcycles` V-cycles of H applied in sequence (1 for
// the pressure operator; 2 for the CH operator, preconditioned by (K + s I)^-2), recorded into the capture:
// r = b, then a while node whose body is one iteration (precondition, r.z, direction, A p, p.q, update,
// r.r) ending in k_mgcg_ctrl, which stops at |r| < tol |b| (|b| = R[kDcAbs]), a breakdown or the inner
// iteration budget left in R.  Grids of at most mg_cluster_cells cells run the same solve as one
// thread-block cluster launch instead (k_mgcg_cluster).  V: the operator and the vectors (V.x is e, zero on
// entry); tmp: a level-0 buffer for the output of the first of two V-cycles.
template <int S>
dn_status rec_mgcg32(dn_handle *h, MgHier &H, MgVec V, const float *b, float *tmp, int vcycles, int project,
                     int max_it, double tol, double *R, DcNodes *nodes) {
  const long long n = V.A.n;
  // the bottom levels (the first of at most kMgBottomCells cells and the coarser ones) of the cluster form, in
  // shared memory: 3 floats per cell
  int bottom = H.levels() - 1;
  while (bottom > 0 && (long long)H.lv[bottom - 1].nx * H.lv[bottom - 1].ny <= kMgBottomCells) --bottom;
  size_t bottom_smem = 0;
  for (int l = bottom; l < H.levels(); ++l) bottom_smem += 3 * sizeof(float) * (size_t)H.lv[l].nx * H.lv[l].ny;
  if (n <= h->mg_cluster_cells && bottom_smem <= (size_t)kMgClusterSmemMax) {  // one cluster launch
    if (!H.dchain) return fail(h, DN_ERR_INVALID_ARGUMENT, "multigrid levels not uploaded");
    MgClusterArgs P{};
    P.bottom = bottom;
    P.ch = H.dchain;
    P.A = V.A;
    P.x = V.x;
    P.r = V.r;
    P.z = V.z;
    P.p = V.p;
    P.q = V.q;
    P.tmp = tmp;
    P.b = b;
    P.vcycles = vcycles;
    P.project = project;
    P.max_it = max_it;
    P.tol = tol;
    P.R = R;
    // about 4 cells per thread on level 0, at most the portable cluster size
    const unsigned cs = (unsigned)std::min<long long>(kMgClusterMax, std::max<long long>(1, (n + 4095) / 4096));
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(cs);
    lc.blockDim = dim3(kMgClusterThreads);
    lc.dynamicSmemBytes = bottom_smem;
    lc.stream = h->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    DN_CUDA(h, cudaLaunchKernelEx(&lc, k_mgcg_cluster<S>, P));
    return check_launch(h, "k_mgcg_cluster");
  }
  V.part = h->mg_part;
  V.scal = h->mg_scal;
  const int nb = (int)std::min<long long>({(long long)kMgParts, 4LL * h->num_sms, (long long)blocks_for(n)});
  const double dn_ = (double)n;
  auto finish = [&](int mode, int first) -> dn_status {
    return launch_pdl(h, "k_mgp_scalars", k_mgp_scalars, dim3(1), dim3(32), 0, h->mg_part, nb, h->mg_scal, mode, first, project, dn_);
  };
  DN_CUDA(h, cudaMemcpyAsync(V.r, b, n * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
  cudaGraphConditionalHandle loop = 0;
  DN_TRY(cond_create(h, &loop));
  DN_TRY(launch_pdl(h, "k_mgcg_init", k_mgcg_init, dim3(1), dim3(32), 0, h->mg_scal, R, max_it, loop));
  return cond_node(h, loop, cudaGraphCondTypeWhile, [&]() -> dn_status {
    const long long before = h->launches;
    if (vcycles == 2) {
      DN_TRY(mg_vcycle(h, H, V.r, tmp));
      DN_TRY(mg_vcycle(h, H, tmp, V.z));
    } else {
      DN_TRY(mg_vcycle(h, H, V.r, V.z));
    }
    DN_TRY(launch_pdl(h, "k_mgp_rz", k_mgp_rz, dim3(nb), dim3(256), 0, V));
    DN_TRY(finish(2, -1));
    DN_TRY(launch_pdl(h, "k_mgp_direction", k_mgp_direction, dim3(nb), dim3(256), 0, V, -1));
    DN_TRY(launch_pdl(h, "k_mgp_apply", k_mgp_apply<S>, dim3(nb), dim3(256), 0, V));
    DN_TRY(finish(0, 0));
    DN_TRY(launch_pdl(h, "k_mgp_update", k_mgp_update, dim3(nb), dim3(256), 0, V));
    DN_TRY(finish(1, 0));
    DN_TRY(launch_pdl(h, "k_mgcg_ctrl", k_mgcg_ctrl, dim3(1), dim3(32), 0, h->mg_scal, R, tol, loop));
    if (nodes) nodes->iter = h->launches - before;
    return DN_OK;
  });
}

dn_status pressure_factor(dn_handle *h, bool split, bool icc);

// The FP64 IC/ILDLT factor of the pressure operator (unless the constant split operator's is already
// valid) and its FP32 copies for the IC inner solver, recorded into the capture; a failed factor is
// recorded in R[kDcErr] and leaves the condition `gate` (the IC inner solve's branch) at 0.
dn_status rec_ic32_factor(dn_handle *h, bool split, int kind, double *R, cudaGraphConditionalHandle gate) {
  const long long n = h->n;
  if (!(split && h->p_factor_valid && h->p_factor_kind == kind)) {
    DN_CUDA(h, cudaMemsetAsync(h->status, 0, sizeof(int), h->stream));
    Factor F{h->l5, h->d5, h->dinv5, 0.0};
    k_factor<5><<<1, 1024, 0, h->stream>>>(SpOp{h->a5, (int)n, h->G.nx, h->G.ny, h->G.px, h->G.py}, F, kind,
                                            h->status);
    DN_TRY(check_launch(h, "k_factor<5>"));
  } else {
    DN_CUDA(h, cudaMemsetAsync(h->status, 0, sizeof(int), h->stream));
  }
  if (h->G.px) {  // the global-memory wavefront reads the L slots
    k_to_float<<<blocks_for(5 * n), 256, 0, h->stream>>>(h->l5, h->fl5, 5 * n);
    DN_TRY(check_launch(h, "k_to_float"));
  }
  k_to_float<<<blocks_for(n), 256, 0, h->stream>>>(h->dinv5, h->fdinv5, n);
  DN_TRY(check_launch(h, "k_to_float"));
  k_ic_gate<<<1, 32, 0, h->stream>>>(h->status, R, gate);
  return check_launch(h, "k_ic_gate");
}

// The coarse operators of a hierarchy and the coarsest level's inverse (kernels only: the inverse's
// usability flag stays on the device, where the solve's first check reads it).
dn_status mg_setup_launch(dn_handle *h, MgHier &H);

// Mixed-precision pressure solve, recorded into the capture: x = 0 on entry; repeat r = b - A x (FP64,
// projected when the system is singular), stop on the reference's rule (rel < tol or abs < tol on the FP64
// residual), else solve A e = r in FP32 to the relative tolerance mixed_inner_tolerance and add e to x in
// FP64.  The inner solver is CG with the multigrid V-cycle (when the grid has a usable hierarchy and
// mixed_preconditioner allows it) or the persistent PCG with the scheme's IC/ILDLT factor rounded to FP32;
// a multigrid cycle after which the FP64 residual does not decrease hands the rest of the solve to the IC
// inner solver.  The operator is the FP64 one rounded to FP32.  Every decision is k_dc_decide's, on the
// device; the result is the record R = h->rec + kRecPressure.
dn_status rec_mixed_pressure(dn_handle *h, bool split, int kind, DcNodes *nodes) {
  const dn_config &cfg = h->cfg;
  const long long n = h->n;
  const int project = h->has_dirichlet ? 0 : 1;
  double *R = h->rec + kRecPressure;
  const long long start = h->launches;
  if (!split) {  // the variable operator changes every step: its FP32 copy and hierarchy are made here
    DN_TRY(launch_pdl(h, "k_to_float", k_to_float, dim3(blocks_for(5 * n)), dim3(256), 0, h->a5, h->fa5, 5 * n));
    if (h->mgp.levels() > 0) DN_TRY(mg_setup_launch(h, h->mgp));
  }
  DcParams P{};
  P.tol = cfg.pressure_tolerance;
  P.n = (double)n;
  P.max_it = cfg.poisson_iterations;
  P.max_cycles = kDcMaxCycles;
  P.project = project;
  P.ch = 0;
  P.mg_flag = h->mgp.levels() > 0 ? h->mgp.flag : nullptr;
  const SpOp A{h->a5, (int)n, h->G.nx, h->G.ny, h->G.px, h->G.py};
  const int nb = 128;
  DN_CUDA(h, cudaMemsetAsync(R, 0, kDcSize * sizeof(double), h->stream));
  cudaGraphConditionalHandle loop = 0;
  DN_TRY(cond_create(h, &loop));
  auto check = [&]() -> dn_status {
    DN_TRY(launch_pdl(h, "k_outer_residual", k_outer_residual<5>, dim3(nb), dim3(256), 0, A, h->b, h->x, h->r, h->partials));
    DN_TRY(launch_pdl(h, "k_finish3", k_finish3, dim3(1), dim3(32), 0, h->partials, nb, h->scal + 8));
    return launch_pdl(h, "k_dc_decide", k_dc_decide, dim3(1), dim3(32), 0, h->scal + 8, R, P, loop);
  };
  DN_TRY(check());
  if (nodes) nodes->fixed = h->launches - start;
  return cond_node(h, loop, cudaGraphCondTypeWhile, [&]() -> dn_status {
    const long long c0 = h->launches;
    // every condition handle belongs to a node of the graph: the multigrid branch exists with a hierarchy
    const bool has_mg = h->mgp.levels() > 0;
    cudaGraphConditionalHandle use_mg = 0, use_ic = 0;
    if (has_mg) DN_TRY(cond_create(h, &use_mg));
    DN_TRY(cond_create(h, &use_ic));
    DN_TRY(launch_pdl(h, "k_dc_branch", k_dc_branch, dim3(1), dim3(32), 0, R, has_mg ? 1 : 0, use_mg, use_ic));
    DN_TRY(launch_pdl(h, "k_inner_rhs", k_inner_rhs_dev, dim3(blocks_for(n)), dim3(256), 0, h->r, R, h->fb, h->fx, n));
    if (has_mg) {
      DN_TRY(cond_node(h, use_mg, cudaGraphCondTypeIf, [&]() -> dn_status {
        MgVec V{};
        V.A = SpOpT<float>{h->fa5, (int)n, h->G.nx, h->G.ny, h->G.px, h->G.py};
        V.x = h->fx;
        V.r = h->fr;
        V.z = h->fz;
        V.p = h->fp0;
        V.q = h->fap;
        return rec_mgcg32<5>(h, h->mgp, V, h->fb, nullptr, 1, project, cfg.poisson_iterations,
                             cfg.mixed_inner_tolerance, R, nodes);
      }));
    }
    DN_TRY(cond_node(h, use_ic, cudaGraphCondTypeIf, [&]() -> dn_status {
      const long long i0 = h->launches;
      cudaGraphConditionalHandle make = 0, go = 0;
      DN_TRY(cond_create(h, &make));
      DN_TRY(cond_create(h, &go));
      k_ic_need<<<1, 32, 0, h->stream>>>(R, make, go);  // the factor once per solve
      DN_TRY(check_launch(h, "k_ic_need"));
      const long long m0 = h->launches;
      DN_TRY(cond_node(h, make, cudaGraphCondTypeIf, [&]() { return rec_ic32_factor(h, split, kind, R, go); }));
      if (nodes) nodes->make = h->launches - m0;
      DN_TRY(cond_node(h, go, cudaGraphCondTypeIf, [&]() -> dn_status {
        double unused[4];  // the results stay on the device (h->capturing)
        DN_TRY(run_pcg32(h, kind, project, cfg.poisson_iterations, cfg.mixed_inner_tolerance, unused));
        return launch_pdl(h, "k_ic_done", k_ic_done, dim3(1), dim3(32), 0, h->scal + 8, h->status, R);
      }));
      if (nodes) nodes->ic = h->launches - i0 - nodes->make;
      return DN_OK;
    }));
    DN_TRY(launch_pdl(h, "k_add_correction", k_add_correction, dim3(blocks_for(n)), dim3(256), 0, h->x, h->fx, n));
    DN_TRY(launch_pdl(h, "k_dc_cycle_end", k_dc_cycle_end, dim3(1), dim3(32), 0, nullptr, R));
    DN_TRY(check());
    if (nodes) nodes->cycle = h->launches - c0 - nodes->iter - nodes->ic - nodes->make;
    return DN_OK;
  });
}

// kernel launches a solve graph's loops ran, from its record: per outer cycle, per multigrid inner
// iteration, per IC inner solve, and the IC factor branch once
long long dc_launches(const DcNodes &d, const double *R) {
  return (long long)R[kDcCycles] * d.cycle + (long long)R[kDcMgIts] * d.iter + (long long)R[kDcIcCycles] * d.ic +
         (R[kDcIcCycles] > 0.0 ? d.make : 0);
}

// The eager form of a recorded solve: captured once per handle (and again after a launch-shape change),
// replayed, and its record read back with one synchronisation.
dn_status replay_solve(dn_handle *h, dn_handle::SolveGraph &g, const std::function<dn_status(DcNodes *)> &record,
                       double *R, double host[kDcSize], float *ms) {
  if (!g.exec || g.epoch != h->graph_epoch) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
    DcNodes nodes;
    const long long before = h->launches;
    DN_TRY(capture_exec(h, &g.exec, [&]() { return record(&nodes); }));
    h->launches = before;
    g.nodes = nodes;
    g.epoch = h->graph_epoch;
  }
  cudaEventRecord(h->kev[0], h->stream);
  DN_CUDA(h, cudaGraphLaunch(g.exec, h->stream));
  cudaEventRecord(h->kev[1], h->stream);
  DN_CUDA(h, cudaMemcpyAsync(h->host_scal + 96, R, kDcSize * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  std::memcpy(host, h->host_scal + 96, kDcSize * sizeof(double));
  *ms = 0.0f;
  cudaEventElapsedTime(ms, h->kev[0], h->kev[1]);
  h->launches += g.nodes.fixed + dc_launches(g.nodes, host);
  return DN_OK;
}

dn_status dc_error(dn_handle *h, const double R[kDcSize], int kind) {
  const int st = (int)R[kDcErr];
  if (st == 0) return DN_OK;
  if (st == kDevFactorFailed)
    return fail(h, kind == kPrecICC ? DN_ERR_ICC_FAILED : DN_ERR_ILDLT_FAILED,
                kind == kPrecICC ? "ICC preconditioner construction failed" : "ILDLT preconditioner construction failed");
  return dev_status_to_dn(h, st);
}

// Mixed-precision pressure solve (rec_mixed_pressure), eager or recorded into a step graph.  The split
// operator is the same every step: its FP32 copy and hierarchy are made once, here, and so is its IC/ILDLT
// factor where the IC inner solver runs from the start (no usable hierarchy).  out: [0] inner iterations in
// total, [1] abs and [2] rel FP64 residual, [3] 0.
dn_status mixed_pressure(dn_handle *h, bool split, int kind, double out[4]) {
  const long long n = h->n;
  if (split && !h->mgp_split_ready) {
    if (h->capturing) return fail(h, DN_ERR_UNSUPPORTED, "the split operator's hierarchy is made by an eager step");
    k_to_float<<<blocks_for(5 * n), 256, 0, h->stream>>>(h->a5, h->fa5, 5 * n);
    DN_TRY(check_launch(h, "k_to_float"));
    if (h->mgp.levels() > 0) {
      bool usable = false;
      DN_TRY(mg_setup(h, h->mgp, &usable));
      if (!usable) DN_TRY(pressure_factor(h, true, kind == kPrecICC));
    } else {
      DN_TRY(pressure_factor(h, true, kind == kPrecICC));  // the IC inner solver's factor, made once
    }
    h->mgp_split_ready = true;
  }
  h->phase_ms[4] = 0.0;
  h->pcg_split_ms[0] = h->pcg_split_ms[1] = h->pcg_split_ms[2] = 0.0;
  out[0] = out[1] = out[2] = out[3] = 0.0;
  if (h->capturing) return rec_mixed_pressure(h, split, kind, &h->step_dcn[0]);
  double R[kDcSize];
  float ms = 0.0f;
  DN_TRY(replay_solve(h, h->dc_graph[0], [&](DcNodes *nd) { return rec_mixed_pressure(h, split, kind, nd); },
                      h->rec + kRecPressure, R, &ms));
  h->phase_ms[4] = ms;
  DN_TRY(dc_error(h, R, kind));
  h->refinement_cycles = (int)R[kDcCycles];
  h->mixed_used_mg = R[kDcUsedMg0] != 0.0;
  out[0] = R[kDcTotal];
  out[1] = R[kDcAbs];
  out[2] = R[kDcRel];
  return DN_OK;
}

// Mixed-precision CH solve (precision = mixed, multigrid hierarchy present): the FP64 defect-correction loop
// of rec_mixed_pressure around FP32 inner CG solves of the 13-point operator A = alpha0 I + beta1 K + beta2 K^2
// (K = -L, build_cahn_hilliard_operator, ch_sparse_krylov.hpp:205-233), preconditioned by two V-cycles of
// K + s I with s = sqrt(alpha0 / beta2).  beta2 (K + s I)^2 has A's K^2 and constant terms, and on every
// eigenvector of K (eigenvalue k >= 0) the ratio (alpha0 + beta1 k + beta2 k^2) / (beta2 (k + s)^2) lies
// between 1/2 + beta1 / (4 beta2 s) (at k = s) and 1, so the preconditioned condition number stays below 2
// on every grid.  Stops on the reference's rule (relative or absolute FP64 residual below ch_tolerance,
// solve_preconditioned_cg, ch_sparse_krylov.hpp:545-560), or when a cycle does not reduce the residual; x
// starts at the state (h->x).  Recorded into the capture; the record is R = h->rec + kRecCh, with the last
// correction's size relative to the iterate (the analogue of the PCG's iterate residual) in R[kDcIres].
dn_status rec_mixed_ch(dn_handle *h, DcNodes *nodes) {
  const dn_config &cfg = h->cfg;
  const long long n = h->n;
  double *R = h->rec + kRecCh;
  const long long start = h->launches;
  DcParams P{};
  P.tol = cfg.ch_tolerance;
  P.n = (double)n;
  P.max_it = cfg.ch_inner_iterations;
  P.max_cycles = kDcMaxCycles;
  P.project = 0;
  P.ch = 1;
  P.mg_flag = h->mgc.flag;
  const SpOp A{h->a13, (int)n, h->G.nx, h->G.ny, h->G.px, h->G.py};
  const int nb = 128;
  DN_CUDA(h, cudaMemsetAsync(R, 0, kDcSize * sizeof(double), h->stream));
  cudaGraphConditionalHandle loop = 0;
  DN_TRY(cond_create(h, &loop));
  auto check = [&]() -> dn_status {
    DN_TRY(launch_pdl(h, "k_outer_residual", k_outer_residual<13>, dim3(nb), dim3(256), 0, A, h->b, h->x, h->r, h->partials));
    DN_TRY(launch_pdl(h, "k_finish3", k_finish3, dim3(1), dim3(32), 0, h->partials, nb, h->scal + 8));
    return launch_pdl(h, "k_dc_decide", k_dc_decide, dim3(1), dim3(32), 0, h->scal + 8, R, P, loop);
  };
  DN_TRY(check());
  if (nodes) nodes->fixed = h->launches - start;
  return cond_node(h, loop, cudaGraphCondTypeWhile, [&]() -> dn_status {
    const long long c0 = h->launches;
    DN_TRY(launch_pdl(h, "k_inner_rhs", k_inner_rhs_dev, dim3(blocks_for(n)), dim3(256), 0, h->r, R, h->cb32, h->cx32, n));
    MgVec V{};
    V.A = SpOpT<float>{h->fa13, (int)n, h->G.nx, h->G.ny, h->G.px, h->G.py};
    V.x = h->cx32;
    V.r = h->cr32;
    V.z = h->cz32;
    V.p = h->cp32;
    V.q = h->cq32;
    DN_TRY(rec_mgcg32<13>(h, h->mgc, V, h->cb32, h->ct32, 2, 0, cfg.ch_inner_iterations, cfg.mixed_inner_tolerance,
                          R, nodes));
    DN_TRY(launch_pdl(h, "k_add_correction_norms", k_add_correction_norms, dim3(nb), dim3(256), 0, h->x, h->cx32, n, h->partials));
    DN_TRY(launch_pdl(h, "k_finish3", k_finish3, dim3(1), dim3(32), 0, h->partials, nb, h->scal + 8));
    DN_TRY(launch_pdl(h, "k_dc_cycle_end", k_dc_cycle_end, dim3(1), dim3(32), 0, h->scal + 8, R));
    DN_TRY(check());
    if (nodes) nodes->cycle = h->launches - c0 - nodes->iter;
    return DN_OK;
  });
}

// The mixed CH solve (rec_mixed_ch), eager or recorded into a step graph.  The FP32 operator and the
// (K + s I) hierarchy are made when alpha0 changes (an eager step).  *used = false when the hierarchy is
// unusable (the caller then runs the FP64 ILDLT PCG).
dn_status mixed_ch(dn_handle *h, double alpha0, dn_report *rep, double *iter_res, bool *used) {
  const dn_config &cfg = h->cfg;
  const long long n = h->n;
  *used = false;
  if (h->ch_mg_alpha0 != alpha0) {
    if (h->capturing) return fail(h, DN_ERR_UNSUPPORTED, "the CH hierarchy is made by an eager step");
    const double a2 = cfg.cn > 0.0 ? (3.0 * kSqrt2 * cfg.cn / 4.0) : 0.0;
    const double beta2 = a2 / cfg.pe;
    if (!(beta2 > 0.0) || !(alpha0 > 0.0)) return DN_OK;
    const double shift = std::sqrt(alpha0 / beta2);
    k_to_float<<<blocks_for(13 * n), 256, 0, h->stream>>>(h->a13, h->fa13, 13 * n);
    DN_TRY(check_launch(h, "k_to_float"));
    MgHier::Lv &l0 = h->mgc.lv[0];
    k_shifted_laplacian<<<blocks_for(n), 256, 0, h->stream>>>(h->G, shift, l0.a64_own, const_cast<float *>(l0.a));
    DN_TRY(check_launch(h, "k_shifted_laplacian"));
    h->mgc.mass = shift;
    h->mgc.singular = 0;
    bool ok = false;
    DN_TRY(mg_setup(h, h->mgc, &ok));
    h->ch_mg_ok = ok;
    h->ch_mg_alpha0 = alpha0;
  }
  if (!h->ch_mg_ok) return DN_OK;
  *used = true;
  rep->ch_preconditioner = 3;
  if (h->capturing) return rec_mixed_ch(h, &h->step_dcn[1]);
  double R[kDcSize];
  float ms = 0.0f;
  DN_TRY(replay_solve(h, h->dc_graph[1], [&](DcNodes *nd) { return rec_mixed_ch(h, nd); }, h->rec + kRecCh, R, &ms));
  h->phase_ms[5] += ms;
  rep->ch_iterations = (int)R[kDcTotal];
  *iter_res = R[kDcIres];
  return DN_OK;
}

// Jacobi-BiCGSTAB on the momentum system (the handle's M, or another operator in the same row format --
// the adjoint's M^T -- with its own stopping rule: relative when use_rel, else the reference's absolute one).
dn_status run_bicgstab(dn_handle *h, double out[4], const double *coef = nullptr, const int *tgt = nullptr,
                       int use_rel = 0, double tol = -1.0, int max_it = -1, double *rec = nullptr) {
  BicgArgs P;
  P.n = h->nm;
  P.coef = coef ? coef : h->mcoef;
  P.tgt = tgt ? tgt : h->mtgt;
  P.b = h->mb;
  P.x = h->mx;
  P.r = h->mr;
  P.rhat = h->mrhat;
  P.p0 = h->mp0;
  P.p1 = h->mp1;
  P.v0 = h->mv0;
  P.v1 = h->mv1;
  P.phat = h->mphat;
  P.s = h->ms;
  P.shat = h->mshat;
  P.t = h->mt;
  P.upd = h->mupd;
  P.dinv = h->mdinv;
  P.max_it = max_it > 0 ? max_it : h->cfg.momentum_iterations;
  P.tol = tol > 0.0 ? tol : h->cfg.momentum_tolerance;
  P.use_rel = use_rel;  // the forward solve: 0, momentum.cpp:470-472's absolute tolerance
  P.bar_count = h->bar_count;
  P.bar_gen = h->bar_gen;
  P.status = h->status;
  P.partials = h->partials;
  P.out = h->scal + 8;
  k_mom_dinv<<<blocks_for(h->nm), 256, 0, h->stream>>>(P);
  DN_TRY(check_launch(h, "k_mom_dinv"));
  DN_TRY(reset_sync(h));
  // every co-resident CTA of this kernel (its gathers are latency-bound), at least 1024 unknowns per CTA
  int blocks = (int)std::min<long long>((long long)h->bicg_occ * h->cta_cap, std::max<long long>(1, h->nm / 1024));
  blocks = std::max(1, std::min(blocks, kMaxBlocks));
  void *args[] = {&P};
  if (h->capturing) {  // recorded into a graph: out and status into rec (k_rec_copy)
    if (!rec) return fail(h, DN_ERR_UNSUPPORTED, "a recorded BiCGSTAB solve needs a record");
    DN_CUDA(h, cudaLaunchCooperativeKernel((const void *)k_bicgstab, dim3(blocks), dim3(kBlock), args, 0, h->stream));
    h->launches++;
    k_rec_copy<<<1, 32, 0, h->stream>>>(h->scal + 8, 4, h->status, rec);
    out[0] = out[1] = out[2] = out[3] = 0.0;
    return check_launch(h, "k_rec_copy");
  }
  cudaEventRecord(h->kev[0], h->stream);
  DN_CUDA(h, cudaLaunchCooperativeKernel((const void *)k_bicgstab, dim3(blocks), dim3(kBlock), args, 0, h->stream));
  cudaEventRecord(h->kev[1], h->stream);
  h->launches++;
  int st = 0;
  DN_TRY(read_status(h, &st));
  if (st != kDevOk) return dev_status_to_dn(h, st);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, h->kev[0], h->kev[1]);
  h->phase_ms[6] += ms;
  return read_scalars(h, 4, out);
}


// ---------------------------------------------------------------------------------------------------
// Step pieces
// ---------------------------------------------------------------------------------------------------
#define LAUNCH_INTERIOR(kernel, F, ...)                                                           \
  do {                                                                                            \
    kernel<<<blocks_for((long long)(F).nx * (F).ny), 256, 0, h->stream>>>(__VA_ARGS__);           \
    DN_TRY(check_launch(h, #kernel));                                                             \
  } while (0)

dn_status materials(dn_handle *h, const Fv &c, const Fv &rho, const Fv &eta) {
  LAUNCH_INTERIOR(k_materials, c, c, rho, eta, h->cfg.density_ratio, h->cfg.viscosity_ratio);
  DN_TRY(bc(h, rho, kBCScalar));
  return bc(h, eta, kBCScalar);
}

dn_status midpoint(dn_handle *h) {
  Fv *f = h->f;
  LAUNCH_INTERIOR(k_midpoint, f[DN_F_RHO_MID], f[DN_F_RHO_PREV], f[DN_F_RHO], f[DN_F_ETA_PREV], f[DN_F_ETA],
                  f[DN_F_RHO_MID], f[DN_F_ETA_MID]);
  DN_TRY(bc(h, f[DN_F_RHO_MID], kBCScalar));
  return bc(h, f[DN_F_ETA_MID], kBCScalar);
}

dn_status chem(dn_handle *h, const Fv &c, const Fv &mu) {
  LAUNCH_INTERIOR(k_chem, mu, c, mu, h->G, h->cfg.cn);
  return bc(h, mu, kBCScalar);
}

dn_status refresh_mu(dn_handle *h) {
  if (compute_mu(h->cfg)) return chem(h, h->f[DN_F_C], h->f[DN_F_MU]);
  DN_TRY(fill_field(h, h->f[DN_F_MU], 0.0));
  return bc(h, h->f[DN_F_MU], kBCScalar);
}

dn_status clear_surface_force(dn_handle *h) {
  Fv *f = h->f;
  for (int id : {DN_F_SFX_CELL, DN_F_SFY_CELL, DN_F_SFX_U, DN_F_SFY_V}) DN_TRY(fill_field(h, f[id], 0.0));
  DN_TRY(bc(h, f[DN_F_SFX_CELL], kBCScalar));
  DN_TRY(bc(h, f[DN_F_SFY_CELL], kBCScalar));
  DN_TRY(bc(h, f[DN_F_SFX_U], kBCU));
  return bc(h, f[DN_F_SFY_V], kBCV);
}

dn_status smooth(dn_handle *h, const Fv &f, const Fv &scratch, int kind) {
  const double nw = h->cfg.surface_tension_smoothing_weight, cw = 1.0 - 4.0 * nw;
  for (int pass = 0; pass < h->cfg.surface_tension_smoothing_passes; ++pass) {
    DN_TRY(bc(h, f, kind));
    LAUNCH_INTERIOR(k_smooth, scratch, f, scratch, cw, nw);
    DN_TRY(bc(h, scratch, kind));
    DN_TRY(copy_field(h, f, scratch));
  }
  return DN_OK;
}

// update_surface_tension_force, phase_field.cpp:179-256
dn_status surface_force(dn_handle *h, const Fv &c_old, const Fv &c_new) {
  const dn_config &cfg = h->cfg;
  if (cfg.surface_tension_multiplier == 0.0 || !compute_mu(cfg)) return clear_surface_force(h);
  Fv *f = h->f;
  const double scale = cfg.surface_tension_multiplier / (cfg.re * cfg.ca);
  {  // c_mid, mu_mid and the four forces in one tiled pass (k_surface_force)
    constexpr int TI = 16, TJ = 32;
    const dim3 grid((unsigned)((h->G.ny + TJ - 1) / TJ), (unsigned)((h->G.nx + TI - 1) / TI));
    k_surface_force<TI, TJ><<<grid, 256, 0, h->stream>>>(c_old, c_new, f[DN_F_SFX_CELL], f[DN_F_SFY_CELL],
                                                         f[DN_F_SFX_U], f[DN_F_SFY_V], h->G, cfg.cn, scale);
    DN_TRY(check_launch(h, "k_surface_force"));
  }
  DN_TRY(bc(h, f[DN_F_SFX_CELL], kBCScalar));
  DN_TRY(bc(h, f[DN_F_SFY_CELL], kBCScalar));
  DN_TRY(bc(h, f[DN_F_SFX_U], kBCU));
  DN_TRY(bc(h, f[DN_F_SFY_V], kBCV));
  if (cfg.surface_tension_smoothing_passes <= 0 || cfg.surface_tension_smoothing_weight <= 0.0) return DN_OK;
  DN_TRY(smooth(h, f[DN_F_SFX_CELL], h->sm_c, kBCScalar));
  DN_TRY(smooth(h, f[DN_F_SFY_CELL], h->sm_c, kBCScalar));
  DN_TRY(smooth(h, f[DN_F_SFX_U], h->sm_u, kBCU));
  return smooth(h, f[DN_F_SFY_V], h->sm_v, kBCV);
}

// build_phase_explicit_operator, phase_field.cpp:354-396 -> h->E_new
dn_status phase_explicit(dn_handle *h, const Fv &c, const Fv &u, const Fv &v) {
  const dn_config &cfg = h->cfg;
  LAUNCH_INTERIOR(k_mob_lap, h->mob, c, h->mob, h->lap, h->G);
  DN_TRY(bc(h, h->mob, kBCScalar));
  DN_TRY(bc(h, h->lap, kBCScalar));
  LAUNCH_INTERIOR(k_lap, h->bih, h->lap, h->bih, h->G);
  DN_TRY(bc(h, h->bih, kBCScalar));
  DN_TRY(chem(h, c, h->mu_t));
  LAUNCH_INTERIOR(k_adv_flux_x, h->afx, c, u, h->afx);
  LAUNCH_INTERIOR(k_adv_flux_y, h->afy, c, v, h->afy);
  DN_TRY(bc(h, h->afx, kBCU));
  DN_TRY(bc(h, h->afy, kBCV));
  LAUNCH_INTERIOR(k_flux_div, h->arhs, h->afx, h->afy, h->arhs, h->G, 1);
  DN_TRY(bc(h, h->arhs, kBCScalar));
  LAUNCH_INTERIOR(k_diff_flux_x, h->dfx, h->mu_t, h->mob, h->dfx, h->G);
  LAUNCH_INTERIOR(k_diff_flux_y, h->dfy, h->mu_t, h->mob, h->dfy, h->G);
  DN_TRY(bc(h, h->dfx, kBCU));
  DN_TRY(bc(h, h->dfy, kBCV));
  LAUNCH_INTERIOR(k_flux_div, h->ddiv, h->dfx, h->dfy, h->ddiv, h->G, 0);
  DN_TRY(bc(h, h->ddiv, kBCScalar));
  const double a1 = cfg.cn > 0.0 ? (3.0 * kSqrt2 / (16.0 * cfg.cn)) : 0.0;
  const double a2 = cfg.cn > 0.0 ? (3.0 * kSqrt2 * cfg.cn / 4.0) : 0.0;
  LAUNCH_INTERIOR(k_explicit, h->E_new, h->ddiv, h->lap, h->bih, h->arhs, h->E_new, a1, a2, cfg.pe);
  return bc(h, h->E_new, kBCScalar);
}

// ensure_ch_linear_system, phase_field.cpp:130-142 (+ build_preconditioner, ch_sparse_krylov.hpp:434-442)
dn_status ensure_ch_system(dn_handle *h, double alpha0) {
  if (std::fabs(alpha0 - h->ch_alpha0) <= 1.0e-14 * std::max(1.0, std::fabs(alpha0))) return DN_OK;
  const dn_config &cfg = h->cfg;
  const double a1 = cfg.cn > 0.0 ? (3.0 * kSqrt2 / (16.0 * cfg.cn)) : 0.0;
  const double a2 = cfg.cn > 0.0 ? (3.0 * kSqrt2 * cfg.cn / 4.0) : 0.0;
  const double beta1 = a1 / cfg.pe, beta2 = a2 / cfg.pe;
  DN_CUDA(h, cudaMemsetAsync(h->status, 0, sizeof(int), h->stream));
  k_ch_matrix<<<blocks_for(h->n, 128), 128, 0, h->stream>>>(h->G, alpha0, beta1, beta2, h->a13, h->status);
  DN_TRY(check_launch(h, "k_ch_matrix"));
  int st = 0;
  DN_TRY(read_status(h, &st));
  if (st) return fail(h, DN_ERR_UNSUPPORTED, "grid too small for the 13-point CH stencil");
  Factor F{h->l13, h->d13, h->dinv13, 0.0};
  k_factor<13><<<1, 1024, 0, h->stream>>>(SpOp{h->a13, (int)h->n, h->G.nx, h->G.ny, h->G.px, h->G.py}, F, kPrecLDLT,
                                           h->status);
  DN_TRY(check_launch(h, "k_factor<13>"));
  DN_TRY(read_status(h, &st));
  if (st == kDevFactorFailed) {
    h->ch_prec = kPrecDiag;
    k_diag_inverse<13><<<blocks_for(h->n), 256, 0, h->stream>>>(SpOp{h->a13, (int)h->n, h->G.nx, h->G.ny, h->G.px, h->G.py},
                                                              h->dinv13);
    DN_TRY(check_launch(h, "k_diag_inverse"));
  } else {
    h->ch_prec = kPrecLDLT;
    if (h->rows13.lval != nullptr) {
      k_rows13<<<blocks_for(h->n), 256, 0, h->stream>>>(SpOp{h->a13, (int)h->n, h->G.nx, h->G.ny, h->G.px, h->G.py}, F,
                                                       h->rows13);
      DN_TRY(check_launch(h, "k_rows13"));
    }
  }
  h->ch_alpha0 = alpha0;
  return DN_OK;
}

// solve_phase_linear_system_eq25, phase_field.cpp:437-503; b = rhs, x = initial guess (compact).  On exit x
// holds the solution.
dn_status ch_linear_solve(dn_handle *h, double alpha0, dn_report *rep, double *iter_res, double *eq_res) {
  DN_TRY(ensure_ch_system(h, alpha0));
  double out[4];
  bool mixed_done = false;
  if (h->ch_mg && h->cfg.precision == DN_PRECISION_MIXED) DN_TRY(mixed_ch(h, alpha0, rep, iter_res, &mixed_done));
  rep->ch_preconditioner = mixed_done ? 3 : (h->ch_prec == kPrecLDLT) ? 1 : 0;
  if (!mixed_done && h->capturing) {
    // recorded: results in the step record; a breakdown retries with the diagonal preconditioner
    // (phase_field.cpp:468-473) in a conditional branch
    double *R = h->rec + kRecStep;
    if (h->ch_prec == kPrecLDLT) {
      DN_TRY((run_pcg<13, 1>(h, h->a13, h->l13, h->dinv13, kPrecLDLT, 0, h->cfg.ch_inner_iterations,
                             h->cfg.ch_tolerance, out, R + kSChPcg)));
      cudaGraphConditionalHandle retry = 0;
      DN_TRY(cond_create(h, &retry));
      k_cond_breakdown<<<1, 32, 0, h->stream>>>(h->status, retry);
      DN_TRY(check_launch(h, "k_cond_breakdown"));
      const long long r0 = h->launches;
      DN_TRY(cond_node(h, retry, cudaGraphCondTypeIf, [&]() -> dn_status {
        k_diag_inverse<13><<<blocks_for(h->n), 256, 0, h->stream>>>(
            SpOp{h->a13, (int)h->n, h->G.nx, h->G.ny, h->G.px, h->G.py}, h->dinv13);
        DN_TRY(check_launch(h, "k_diag_inverse"));
        DN_TRY((run_pcg<13, 2>(h, h->a13, h->l13, h->dinv13, kPrecDiag, 0, h->cfg.ch_inner_iterations,
                               h->cfg.ch_tolerance, out, R + kSChPcg)));
        k_rec_flag<<<1, 32, 0, h->stream>>>(R + kSChRetry);
        return check_launch(h, "k_rec_flag");
      }));
      h->step_retry = h->launches - r0;
    } else {
      DN_TRY((run_pcg<13, 2>(h, h->a13, h->l13, h->dinv13, kPrecDiag, 0, h->cfg.ch_inner_iterations,
                             h->cfg.ch_tolerance, out, R + kSChPcg)));
    }
  } else if (!mixed_done) {
    dn_status s;
    if (h->ch_prec == kPrecLDLT)
      s = run_pcg<13, 1>(h, h->a13, h->l13, h->dinv13, kPrecLDLT, 0, h->cfg.ch_inner_iterations, h->cfg.ch_tolerance,
                         out);
    else
      s = run_pcg<13, 2>(h, h->a13, h->l13, h->dinv13, kPrecDiag, 0, h->cfg.ch_inner_iterations, h->cfg.ch_tolerance,
                         out);
    if (s == DN_ERR_PCG_BREAKDOWN) {
      // phase_field.cpp:468-473: retry with the diagonal preconditioner from the current iterate
      h->ch_prec = kPrecDiag;
      k_diag_inverse<13><<<blocks_for(h->n), 256, 0, h->stream>>>(
          SpOp{h->a13, (int)h->n, h->G.nx, h->G.ny, h->G.px, h->G.py}, h->dinv13);
      DN_TRY(check_launch(h, "k_diag_inverse"));
      rep->ch_preconditioner = 2;
      s = run_pcg<13, 2>(h, h->a13, h->l13, h->dinv13, kPrecDiag, 0, h->cfg.ch_inner_iterations,
                         h->cfg.ch_tolerance, out);
    }
    DN_TRY(s);
    rep->ch_iterations = (int)out[0];
    *iter_res = out[3];
  }
  // equation residual ||b - A x|| / ||b||: enough CTAs to keep every SM's loads in flight
  const int nb = 1024;
  k_residual_partials<13><<<nb, 256, 0, h->stream>>>(SpOp{h->a13, (int)h->n, h->G.nx, h->G.ny, h->G.px, h->G.py}, h->b,
                                                      h->x, h->partials);
  DN_TRY(check_launch(h, "k_residual_partials"));
  double *eq = h->rec + kRecStep + kSChEq;
  k_eq_residual<<<1, 32, 0, h->stream>>>(h->partials, nb, eq);
  DN_TRY(check_launch(h, "k_eq_residual"));
  *eq_res = 0.0;
  if (h->capturing) return DN_OK;
  DN_CUDA(h, cudaMemcpyAsync(h->host_scal + 64, eq, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  *eq_res = h->host_scal[64];
  return DN_OK;
}

// solve_cahn_hilliard_semi_implicit, phase_field.cpp:667-708
dn_status ch_semi_implicit(dn_handle *h, int step, dn_report *rep) {
  Fv *f = h->f;
  const dn_config &cfg = h->cfg;
  const double dt = cfg.dt;
  const double alpha0 = (step == 0) ? (1.0 / dt) : (3.0 / (2.0 * dt));
  // the explicit operator E(c, u, v) and the BDF right-hand side in one tiled pass (k_ch_explicit_rhs)
  {
    constexpr int TI = 16, TJ = 32;
    const double a1 = cfg.cn > 0.0 ? (3.0 * kSqrt2 / (16.0 * cfg.cn)) : 0.0;
    const double a2 = cfg.cn > 0.0 ? (3.0 * kSqrt2 * cfg.cn / 4.0) : 0.0;
    const dim3 grid((unsigned)((h->G.ny + TJ - 1) / TJ), (unsigned)((h->G.nx + TI - 1) / TI));
    k_ch_explicit_rhs<TI, TJ><<<grid, 256, 0, h->stream>>>(
        f[DN_F_C], f[DN_F_U], f[DN_F_V], f[DN_F_C_PREV], f[DN_F_C_PREV2], f[DN_F_E_PREV], h->E_new, h->b, h->x, h->G,
        h->bc.u[DN_LEFT], h->bc.u[DN_RIGHT], h->bc.v[DN_BOTTOM], h->bc.v[DN_TOP], cfg.cn, a1, a2, cfg.pe, step, dt);
    DN_TRY(check_launch(h, "k_ch_explicit_rhs"));
    DN_TRY(bc(h, h->E_new, kBCScalar));
  }
  double iter_res = 0.0, eq_res = 0.0;
  DN_TRY(ch_linear_solve(h, alpha0, rep, &iter_res, &eq_res));
  LAUNCH_INTERIOR(k_scatter_compact, f[DN_F_C], h->x, f[DN_F_C]);
  DN_TRY(bc(h, f[DN_F_C], kBCScalar));
  DN_TRY(chem(h, f[DN_F_C], f[DN_F_MU]));
  rep->ch_equation_residual = eq_res;
  rep->ch_residual = iter_res;
  return copy_field(h, f[DN_F_E_PREV], h->E_new);
}

dn_status phase(dn_handle *h, int step, dn_report *rep) {
  Fv *f = h->f;
  if (solve_ch(h->cfg)) {
    DN_TRY(ch_semi_implicit(h, step, rep));
    DN_TRY(materials(h, f[DN_F_C], f[DN_F_RHO], f[DN_F_ETA]));
    DN_TRY(midpoint(h));
    DN_TRY(surface_force(h, f[DN_F_C_PREV], f[DN_F_C]));
    rep->coupling_iterations = 1;
    return DN_OK;
  }
  DN_TRY(materials(h, f[DN_F_C], f[DN_F_RHO], f[DN_F_ETA]));
  DN_TRY(midpoint(h));
  DN_TRY(refresh_mu(h));
  DN_TRY(surface_force(h, f[DN_F_C_PREV], f[DN_F_C]));
  rep->ch_iterations = 0;
  rep->ch_preconditioner = -1;
  rep->ch_equation_residual = 0.0;
  rep->ch_residual = 0.0;
  rep->coupling_iterations = 0;
  return DN_OK;
}

// compute_momentum_fluxes + solve_momentum_predictor, momentum.cpp:55-502
dn_status momentum(dn_handle *h, int step, dn_report *rep) {
  Fv *f = h->f;
  const dn_config &cfg = h->cfg;
  const double alpha = 0.5 * cfg.dt / cfg.re;
  // H (centred convection, with the face BC of the flux arrays) and the predictor rhs in one pass
  k_mom_conv_rhs<<<blocks_for(h->nm), 256, 0, h->stream>>>(
      f[DN_F_U], f[DN_F_V], f[DN_F_RHO_MID], f[DN_F_ETA_PREV], h->hu, h->hv, f[DN_F_HU_PREV], f[DN_F_HV_PREV],
      f[DN_F_SFX_U], f[DN_F_SFY_V], h->urhs, h->vrhs, h->G, h->bc.u[DN_LEFT], h->bc.u[DN_RIGHT], h->bc.v[DN_BOTTOM],
      h->bc.v[DN_TOP], step, cfg.dt, alpha, cfg.body_force_x, cfg.body_force_y);
  DN_TRY(check_launch(h, "k_mom_conv_rhs"));
  DN_TRY(bc(h, h->hu, kBCU));  // the ghosts of H (the faces it recomputes are the values already written)
  DN_TRY(bc(h, h->hv, kBCV));
  k_mom_assemble<<<blocks_for(h->nm, 128), 128, 0, h->stream>>>(h->ml, h->G, h->bc, f[DN_F_U], f[DN_F_V], f[DN_F_RHO_MID],
                                                           f[DN_F_ETA], h->urhs, h->vrhs, alpha, h->mcoef, h->mtgt, h->mb,
                                                           h->mx);
  DN_TRY(check_launch(h, "k_mom_assemble"));
  double out[4];
  DN_TRY(run_bicgstab(h, out, nullptr, nullptr, 0, -1.0, -1, h->rec + kRecStep + kSMom));
  rep->momentum_iterations = (int)out[0];
  rep->momentum_residual = out[1];
  DN_TRY(copy_field(h, f[DN_F_U_STAR], f[DN_F_U]));
  DN_TRY(copy_field(h, f[DN_F_V_STAR], f[DN_F_V]));
  k_mom_scatter<<<blocks_for(h->nm), 256, 0, h->stream>>>(h->ml, h->mx, f[DN_F_U_STAR], f[DN_F_V_STAR]);
  DN_TRY(check_launch(h, "k_mom_scatter"));
  DN_TRY(bc(h, f[DN_F_U_STAR], kBCU));
  DN_TRY(bc(h, f[DN_F_V_STAR], kBCV));
  DN_TRY(copy_field(h, f[DN_F_HU_PREV], h->hu));
  return copy_field(h, f[DN_F_HV_PREV], h->hv);
}

dn_status split_extrapolation(dn_handle *h, int step) {
  Fv *f = h->f;
  LAUNCH_INTERIOR(k_p_ext, h->pe, f[DN_F_P], f[DN_F_P_PREV], h->pe, step == 0 ? 1 : 0);
  return bc(h, h->pe, kBCPressure);
}

// solve_pressure_correction_{icpcg,ildlt_pcg,liu_split_icpcg,liu_split_ildlt_pcg}, pressure.cpp:302-365, 470-491
dn_status pressure_factor_solve(dn_handle *h, bool split, bool icc, dn_report *rep);
dn_status pressure_factor(dn_handle *h, bool split, bool icc);
dn_status dcdm_solve(dn_handle *h, dn_report *rep);

// x -= mean(x) for a compact vector of the n cells
dn_status compact_subtract_mean(dn_handle *h, double *x) {
  const int nb = 128;
  k_vec_sum<<<nb, 256, 0, h->stream>>>(x, h->n, h->partials);
  DN_TRY(check_launch(h, "k_vec_sum"));
  k_finish_mean<<<1, 32, 0, h->stream>>>(h->partials, nb, (double)h->n, h->scal);
  DN_TRY(check_launch(h, "k_finish_mean"));
  k_vec_sub_scalar<<<blocks_for(h->n), 256, 0, h->stream>>>(x, h->n, h->scal);
  return check_launch(h, "k_vec_sub_scalar");
}

__global__ void k_spmv5(SpOp A, const double *x, double *y) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= A.n) return;
  y[r] = spmv_row<5>(A, x, (int)(r / A.ny), (int)(r % A.ny));
}
__global__ void k_residual5(SpOp A, const double *b, const double *x, double *r) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A.n) return;
  r[t] = b[t] - spmv_row<5>(A, x, (int)(t / A.ny), (int)(t % A.ny));
}

// solve_pressure_correction_jacobi, pressure.cpp:250-300: the variable-coefficient system (as icpcg builds it,
// regularised) solved by Jacobi sweeps from x = 0 until max |b - A x| < tol or the iteration limit.  The
// sweeps and the residual checks are launched in batches; a device flag stops the batch at convergence, and
// the host reads the flag, the count and the residual after each batch.
dn_status pressure_jacobi(dn_handle *h, dn_report *rep) {
  Fv *f = h->f;
  const dn_config &cfg = h->cfg;
  DN_TRY(fill_field(h, f[DN_F_P_CORR], 0.0));
  DN_TRY(bc(h, f[DN_F_P_CORR], kBCPressure));
  k_p_assemble<<<blocks_for(h->n), 256, 0, h->stream>>>(h->G, h->bc, f[DN_F_RHO_MID], f[DN_F_U_STAR], f[DN_F_V_STAR],
                                                       h->pe, 0, 1.0, cfg.dt, h->a5, h->b);
  DN_TRY(check_launch(h, "k_p_assemble"));
  if (!h->has_dirichlet) DN_TRY(compact_subtract_mean(h, h->b));
  double *xb[2] = {h->x, h->y};
  DN_CUDA(h, cudaMemsetAsync(h->x, 0, h->n * sizeof(double), h->stream));
  DN_CUDA(h, cudaMemsetAsync(h->y, 0, h->n * sizeof(double), h->stream));
  DN_CUDA(h, cudaMemsetAsync(h->status, 0, sizeof(int), h->stream));
  unsigned int *done = h->prog, *iters = h->prog + 1;
  DN_CUDA(h, cudaMemsetAsync(h->prog, 0, 2 * sizeof(unsigned int), h->stream));
  double *resid = h->scal + 24;
  const int nb = (int)((h->n + 255) / 256);
  const int limit = std::max(0, cfg.poisson_iterations);
  int launched = 0;
  unsigned int host_flags[2] = {0u, 0u};
  while (launched < limit) {
    const int batch = std::min(256, limit - launched);
    for (int k = 0; k < batch; ++k) {
      const int it = launched + k;
      k_jacobi_sweep<<<nb, 256, 0, h->stream>>>(h->a5, (int)h->n, h->G.nx, h->G.ny, h->G.px, h->G.py, h->b,
                                                 xb[it & 1], xb[(it + 1) & 1], h->partials, done, h->status);
      k_jacobi_check<<<1, 32, 0, h->stream>>>(h->partials, nb, cfg.pressure_tolerance, done, iters, resid);
    }
    DN_TRY(check_launch(h, "k_jacobi_sweep"));
    launched += batch;
    DN_CUDA(h, cudaMemcpyAsync(h->host_scal + 40, h->prog, 2 * sizeof(unsigned int), cudaMemcpyDeviceToHost,
                               h->stream));
    DN_CUDA(h, cudaStreamSynchronize(h->stream));
    std::memcpy(host_flags, h->host_scal + 40, sizeof(host_flags));
    int st = 0;
    DN_TRY(read_status(h, &st));
    if (st != kDevOk) return dev_status_to_dn(h, st);
    if (host_flags[0]) break;
  }
  const int its = (int)host_flags[1];
  double res = 0.0;
  if (its > 0) {
    DN_CUDA(h, cudaMemcpyAsync(h->host_scal + 44, resid, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    DN_CUDA(h, cudaStreamSynchronize(h->stream));
    std::memcpy(&res, h->host_scal + 44, sizeof(double));
  }
  h->launches += 2LL * its + 1;
  rep->pressure_iterations = its;
  rep->pressure_residual = res;
  rep->refinement_cycles = 0;
  rep->mixed_inner_multigrid = 0;
  h->phase_ms[7] = its;
  LAUNCH_INTERIOR(k_scatter_compact, f[DN_F_P_CORR], xb[its & 1], f[DN_F_P_CORR]);
  if (!h->has_dirichlet) DN_TRY(subtract_mean(h, f[DN_F_P_CORR]));
  return bc(h, f[DN_F_P_CORR], kBCPressure);
}

// z = M^-1 in with the ICC (or LDLT) factor of the pressure system (k_prec_apply); z lands in h->z.
dn_status prec_apply(dn_handle *h, const double *in, int kind = kPrecICC) {
  PcgArgs P{};
  size_t dyn_smem = 0;
  int blocks = 1;
  const bool staged = h->sw5 > 0;
  const void *kern;
  if (staged && h->G.px) {
    DN_TRY((pcg_launch_args<5, 4>(h, h->a5, h->l5, h->dinv5, kind, 0, 1, 0.0, P, dyn_smem, blocks)));
    kern = (const void *)k_prec_apply<4>;
  } else if (staged) {
    DN_TRY((pcg_launch_args<5, 3>(h, h->a5, h->l5, h->dinv5, kind, 0, 1, 0.0, P, dyn_smem, blocks)));
    kern = (const void *)k_prec_apply<3>;
  } else {
    DN_TRY((pcg_launch_args<5, 0>(h, h->a5, h->l5, h->dinv5, kind, 0, 1, 0.0, P, dyn_smem, blocks)));
    kern = (const void *)k_prec_apply<0>;
  }
  P.r = const_cast<double *>(in);
  P.s5.r = in;
  DN_TRY(reset_sync(h));
  void *args[] = {&P};
  DN_CUDA(h, cudaLaunchCooperativeKernel(kern, dim3(blocks), dim3(kBlock), args, dyn_smem, h->stream));
  h->launches++;
  int st = 0;
  DN_TRY(read_status(h, &st));
  return st == kDevOk ? DN_OK : dev_status_to_dn(h, st);
}

// Host sums of k_dots4's partials in block order: out[0..3] the four products, out[4] the non-finite count.
dn_status dots4(dn_handle *h, const double *a0, const double *b0, const double *a1, const double *b1,
                const double *a2, const double *b2, const double *a3, const double *b3, const double *f0,
                const double *f1, double out[5]) {
  const int nb = 128;
  k_dots4<<<nb, 256, 0, h->stream>>>(a0, b0, a1, b1, a2, b2, a3, b3, f0, f1, h->n, h->partials);
  DN_TRY(check_launch(h, "k_dots4"));
  DN_CUDA(h, cudaMemcpyAsync(h->host_scal, h->partials, 5 * nb * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  for (int k = 0; k < 5; ++k) {
    double v = 0.0;
    for (int b = 0; b < nb; ++b) v += h->host_scal[k * nb + b];
    out[k] = v;
  }
  return DN_OK;
}

// solve_dcdm_conjugate_directions (ch_sparse_krylov.hpp:662-837) on the assembled split system b, from
// x = 0, directions from the ICC factor (or the identity), history in h->dcdm_dirs / dcdm_adirs.  Every
// vector operation and its order follow the reference; the scalars come back to the host, which decides the
// fallbacks as the reference does.
dn_status dcdm_solve(dn_handle *h, dn_report *rep) {
  const dn_config &cfg = h->cfg;
  const long long n = h->n;
  const int nb = blocks_for(n);
  const double floor_ = 1.0e-30, tol = cfg.pressure_tolerance;
  const bool project = !h->has_dirichlet;
  const SpOp A{h->a5, (int)n, h->G.nx, h->G.ny, h->G.px, h->G.py};
  double *x = h->x, *r = h->r, *rh = h->p0, *z = h->z, *d = h->p1, *ad = h->ap, *delta = h->y;
  auto proj = [&](double *v) -> dn_status { return project ? compact_subtract_mean(h, v) : DN_OK; };
  auto copy = [&](double *dst, const double *src) -> dn_status {
    DN_CUDA(h, cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    return DN_OK;
  };
  DN_CUDA(h, cudaMemsetAsync(x, 0, n * sizeof(double), h->stream));
  k_residual5<<<nb, 256, 0, h->stream>>>(A, h->b, x, r);
  DN_TRY(check_launch(h, "k_residual5"));
  DN_TRY(proj(r));
  DN_TRY(proj(x));
  double q[5];
  DN_TRY(dots4(h, h->b, h->b, r, r, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, q));
  const double rhs_norm = std::sqrt(std::max(q[0], 0.0));
  double absr = std::sqrt(std::max(q[1], 0.0));
  double relr = absr / std::max(rhs_norm, 1.0e-30);
  int its = 0;
  rep->pressure_residual = relr;
  if (relr < tol || absr < tol) {
    rep->pressure_iterations = 0;
    return DN_OK;
  }
  const int hist = cfg.dcdm_history_size, keep = h->dcdm_keep;
  h->mon_host.clear();
  std::vector<int> slot;      // slot[k]: storage row of the k-th oldest stored direction
  std::vector<double> den;    // d.Ad of each stored direction (the reference recomputes the same value)
  const int limit = std::max(1, cfg.poisson_iterations);
  for (int it = 0; it < limit; ++it) {
    if (cfg.dcdm_restart_interval > 0 && it > 0 && it % cfg.dcdm_restart_interval == 0) {
      slot.clear();
      den.clear();
    }
    DN_TRY(dots4(h, r, r, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, q));
    const double rnorm = std::sqrt(std::max(q[0], 0.0));
    if (rnorm < tol) break;
    k_div_scalar<<<nb, 256, 0, h->stream>>>(r, rh, n, std::max(rnorm, floor_));
    DN_TRY(check_launch(h, "k_div_scalar"));
    if (cfg.dcdm_direction_mode == 1) {
      DN_TRY(copy(z, rh));
    } else {
      DN_TRY(prec_apply(h, rh));
    }
    DN_TRY(dots4(h, z, z, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, z, nullptr, q));
    if (q[4] != 0.0 || std::sqrt(std::max(q[0], 0.0)) < floor_) DN_TRY(copy(z, r));
    DN_TRY(proj(z));
    DN_TRY(dots4(h, z, z, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, z, nullptr, q));
    if (q[4] != 0.0 || std::sqrt(std::max(q[0], 0.0)) < floor_) {
      DN_TRY(copy(z, r));
      DN_TRY(proj(z));
    }
    DN_TRY(copy(d, z));
    const int stored = (int)slot.size();
    const int begin = (hist > 0 && stored > hist) ? stored - hist : 0;
    for (int k = begin; k < stored; ++k) {
      if (!std::isfinite(den[(size_t)k]) || std::fabs(den[(size_t)k]) < floor_) continue;
      const double *dir = h->dcdm_dirs + (size_t)slot[(size_t)k] * n;
      const double *adir = h->dcdm_adirs + (size_t)slot[(size_t)k] * n;
      DN_TRY(dots4(h, d, adir, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, q));
      k_sub_scaled<<<nb, 256, 0, h->stream>>>(d, dir, n, q[0] / den[(size_t)k]);
      DN_TRY(check_launch(h, "k_sub_scaled"));
    }
    DN_TRY(proj(d));
    k_spmv5<<<nb, 256, 0, h->stream>>>(A, d, ad);
    DN_TRY(check_launch(h, "k_spmv5"));
    DN_TRY(dots4(h, r, d, d, ad, d, d, nullptr, nullptr, d, ad, q));
    double rd = q[0], dad = q[1];
    if (q[4] != 0.0 || std::sqrt(std::max(q[2], 0.0)) < floor_ || !std::isfinite(rd) || rd <= 0.0 ||
        !std::isfinite(dad) || std::fabs(dad) < floor_) {
      DN_TRY(copy(d, r));
      DN_TRY(proj(d));
      k_spmv5<<<nb, 256, 0, h->stream>>>(A, d, ad);
      DN_TRY(check_launch(h, "k_spmv5"));
      DN_TRY(dots4(h, r, d, d, ad, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, q));
      rd = q[0];
      dad = q[1];
      if (!std::isfinite(rd) || rd <= 0.0 || !std::isfinite(dad) || std::fabs(dad) < floor_)
        return fail(h, DN_ERR_PCG_BREAKDOWN, "dcdm breakdown: invalid fallback direction");
    }
    const double alpha = rd / dad;
    k_x_step<<<nb, 256, 0, h->stream>>>(x, d, delta, n, alpha);
    DN_TRY(check_launch(h, "k_x_step"));
    DN_TRY(dots4(h, delta, delta, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, q));
    const double update_sq = q[0];
    DN_TRY(proj(x));
    k_residual5<<<nb, 256, 0, h->stream>>>(A, h->b, x, r);
    DN_TRY(check_launch(h, "k_residual5"));
    DN_TRY(proj(r));
    DN_TRY(dots4(h, x, x, r, r, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, q));
    its = it + 1;
    absr = std::sqrt(std::max(q[1], 0.0));
    relr = absr / std::max(rhs_norm, 1.0e-30);
    if (it < h->mon_cap) {
      const double rec[4] = {absr, relr, std::sqrt(update_sq / std::max(q[0], 1.0e-30)), alpha};
      h->mon_host.insert(h->mon_host.end(), rec, rec + 4);
    }
    // push_back, dropping the oldest beyond `keep`
    int row;
    if ((int)slot.size() < keep) {
      row = (int)slot.size();
    } else {
      row = slot.front();
      slot.erase(slot.begin());
      den.erase(den.begin());
    }
    DN_TRY(copy(h->dcdm_dirs + (size_t)row * n, d));
    DN_TRY(copy(h->dcdm_adirs + (size_t)row * n, ad));
    slot.push_back(row);
    den.push_back(dad);
    if (relr < tol || absr < tol) break;
  }
  rep->pressure_iterations = its;
  rep->pressure_residual = relr;
  h->phase_ms[7] = its;
  h->mon_count = std::min(its, h->mon_cap);
  return DN_OK;
}

// ---- pressure analysis (Solver::run_pressure_analysis_from_snapshot, pressure_analysis.cpp:156-328) ----
// 1 where |2c - 1| < cutoff (the interface band), else 0, per compact row i*ny + j
__global__ void k_interface_mask(Fv c, double cutoff, double *mask) {
  const long long n = (long long)c.nx * c.ny;
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const double phi = 2.0 * c.at((int)(r / c.ny), (int)(r % c.ny)) - 1.0;
  mask[r] = fabs(phi) < cutoff ? 1.0 : 0.0;
}
// per block: max |r|, the sum of r^2 over the band, the sum of r^2 outside it
__global__ void k_resid_stats(const double *r, const double *mask, long long n, double *partials) {
  __shared__ double sm[3][256];
  double mx = 0.0, in = 0.0, out = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const double v = r[t];
    mx = fmax(mx, fabs(v));
    if (mask[t] > 0.5)
      in += v * v;
    else
      out += v * v;
  }
  sm[0][threadIdx.x] = mx;
  sm[1][threadIdx.x] = in;
  sm[2][threadIdx.x] = out;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      sm[0][threadIdx.x] = fmax(sm[0][threadIdx.x], sm[0][threadIdx.x + o]);
      sm[1][threadIdx.x] += sm[1][threadIdx.x + o];
      sm[2][threadIdx.x] += sm[2][threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) partials[(size_t)k * gridDim.x + blockIdx.x] = sm[k][0];
}
// z = in / max(|diag|, 1e-30): build_diagonal_preconditioner / apply_preconditioner (ch_sparse_krylov.hpp:421-432)
__global__ void k_diag_apply(const double *diag, const double *in, double *z, long long n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) z[t] = (1.0 / max_ref(fabs(diag[t]), 1.0e-30)) * in[t];
}
__global__ void k_p_update(double *p, const double *z, long long n, double beta) {  // p = z + beta p
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) p[t] = z[t] + beta * p[t];
}

// %.17g, as an ostream with setprecision(17) prints a double
std::string g17(double v) {
  char b[40];
  std::snprintf(b, sizeof b, "%.17g", v);
  return b;
}
// write_matrix_csv (pressure_analysis.cpp:46-61) of a compact vector (row i*ny + j): ny lines of nx values
bool write_field_csv(const std::filesystem::path &path, const std::vector<double> &v, int nx, int ny) {
  FILE *fp = std::fopen(path.string().c_str(), "w");
  if (!fp) return false;
  for (int j = 0; j < ny; ++j) {
    for (int i = 0; i < nx; ++i) std::fprintf(fp, i > 0 ? ",%.17g" : "%.17g", v[(size_t)i * ny + j]);
    std::fputc('\n', fp);
  }
  return std::fclose(fp) == 0;
}

// Sums (max for k == 0 when `max0`) of per-block partials written by a 128-block kernel, in block order.
dn_status host_partials(dn_handle *h, int k_count, int nb, bool max0, double *out) {
  DN_CUDA(h, cudaMemcpyAsync(h->host_scal, h->partials, (size_t)k_count * nb * sizeof(double),
                             cudaMemcpyDeviceToHost, h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  for (int k = 0; k < k_count; ++k) {
    double v = 0.0;
    for (int b = 0; b < nb; ++b) v = (max0 && k == 0) ? std::max(v, h->host_scal[k * nb + b]) : v + h->host_scal[k * nb + b];
    out[k] = v;
  }
  return DN_OK;
}

dn_status download(dn_handle *h, const double *dev, std::vector<double> &host, size_t count) {
  host.resize(count);
  DN_CUDA(h, cudaMemcpyAsync(host.data(), dev, count * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  return DN_OK;
}

dn_status pressure_analysis(dn_handle *h, int step, const std::string &source) {
  namespace fs = std::filesystem;
  Fv *f = h->f;
  const dn_config &cfg = h->cfg;
  const long long n = h->n;
  const int nb = blocks_for(n), nx = h->G.nx, ny = h->G.ny;
  const bool split = use_split(cfg);
  const bool ildlt = cfg.pressure_scheme == DN_P_ILDLT_PCG || cfg.pressure_scheme == DN_P_SPLIT_ILDLT_PCG;
  const bool project = !h->has_dirichlet;
  const double tol = cfg.pressure_tolerance;
  // the key iterations (analysis_key_iterations, pressure_analysis.cpp:108-124)
  std::set<int> keys;
  {
    const std::string list = cfg.analysis_spectrum_iterations;
    size_t at = 0;
    while (at <= list.size()) {
      const size_t comma = std::min(list.find(',', at), list.size());
      std::string tok;
      for (size_t q = at; q < comma; ++q)
        if (!std::isspace((unsigned char)list[q])) tok += list[q];
      at = comma + 1;
      std::string low = tok;
      for (char &ch : low) ch = (char)std::tolower((unsigned char)ch);
      if (tok.empty() || low == "final") continue;
      try {
        keys.insert(std::stoi(tok));
      } catch (const std::exception &) {
        return fail(h, DN_ERR_CONFIG, "invalid analysis_spectrum_iterations entry: " + tok);
      }
    }
  }
  // the system as the scheme assembles it, and its preconditioner (ICC / ILDLT, the diagonal when it fails)
  if (split) DN_TRY(split_extrapolation(h, step));
  k_p_assemble<<<blocks_for(n), 256, 0, h->stream>>>(h->G, h->bc, f[DN_F_RHO_MID], f[DN_F_U_STAR], f[DN_F_V_STAR],
                                                    h->pe, split ? 1 : 0, split ? rho_ref_of(cfg) : 1.0, cfg.dt,
                                                    h->a5, h->b);
  DN_TRY(check_launch(h, "k_p_assemble"));
  if (project) DN_TRY(compact_subtract_mean(h, h->b));
  const int kind = ildlt ? kPrecLDLT : kPrecICC;
  bool diag = false;
  {
    const dn_status fs_ = pressure_factor(h, split, !ildlt);
    if (fs_ == DN_ERR_ICC_FAILED || fs_ == DN_ERR_ILDLT_FAILED) {
      diag = true;
      h->err.clear();
    } else if (fs_ != DN_OK) {
      return fs_;
    }
  }
  const std::string solver_name = ildlt ? (split ? "SplitILDLTPCG" : "ILDLTPCG")
                                  : cfg.pressure_scheme == DN_P_SPLIT_DCDM_ICPCG ? "SplitDCDMICC"
                                  : split                                        ? "SplitICCPCG"
                                                                                 : "ICCPCG";
  const std::string prec_name = diag ? "Diagonal" : ildlt ? "ILDLT" : "ICC";
  const SpOp A{h->a5, (int)n, nx, ny, h->G.px, h->G.py};
  double *x = h->x, *r = h->r, *z = h->z, *p = h->p0, *ap = h->ap, *delta = h->y, *mask = h->p1;
  auto proj = [&](double *v) -> dn_status { return project ? compact_subtract_mean(h, v) : DN_OK; };
  auto precondition = [&]() -> dn_status {  // z = M^-1 r, projected
    if (diag) {
      k_diag_apply<<<nb, 256, 0, h->stream>>>(h->a5 + 2 * (size_t)n, r, z, n);
      DN_TRY(check_launch(h, "k_diag_apply"));
    } else {
      DN_TRY(prec_apply(h, r, kind));
    }
    return proj(z);
  };
  k_interface_mask<<<nb, 256, 0, h->stream>>>(f[DN_F_C], std::tanh(cfg.analysis_interface_band_multiplier /
                                                                    (2.0 * std::sqrt(2.0))), mask);
  DN_TRY(check_launch(h, "k_interface_mask"));

  // output paths (pressure_analysis.cpp:187-198)
  const int snap_step = step + 1;
  const double time = (double)snap_step * cfg.dt;
  char stem_c[256];
  std::snprintf(stem_c, sizeof stem_c, "%s_%s_step_%06d", cfg.name, source.c_str(), snap_step);
  const fs::path dir = fs::path(cfg.output_dir) / cfg.name / "pressure_analysis";
  const fs::path field_dir = dir / (std::string(stem_c) + "_fields");
  const fs::path iter_path = dir / (std::string(stem_c) + "_pcg.csv");
  try {
    fs::create_directories(field_dir);
  } catch (const std::exception &e) {
    return fail(h, DN_ERR_INVALID_ARGUMENT, std::string("cannot create pressure analysis directory: ") + e.what());
  }
  FILE *it_out = std::fopen(iter_path.string().c_str(), "w");
  if (!it_out) return fail(h, DN_ERR_INVALID_ARGUMENT, "cannot open pressure analysis iteration file: " + iter_path.string());
  std::fputs("case_name,case_group,source_mode,step,time,grid_size,density_ratio,sigma,viscosity_ratio,solver_name,"
             "preconditioner_name,max_iter,tolerance,initial_guess_type,iter,true_res_l2,rel_true_res_l2,"
             "true_res_linf,precond_res,alpha_k,beta_k,q_k,interface_res_l2,bulk_res_l2,interface_res_fraction,"
             "bulk_res_fraction\n", it_out);
  const double sigma = cfg.surface_tension_multiplier == 0.0
                           ? 0.0
                           : cfg.surface_tension_multiplier / std::max(cfg.re * cfg.ca, 1.0e-30);
  char grid_c[32];
  std::snprintf(grid_c, sizeof grid_c, "%dx%d", nx, ny);
  // the columns before `iter`, shared by every row and by the summary row
  const std::string lead = std::string(cfg.name) + "," + cfg.analysis_case_group + "," + source + "," +
                           std::to_string(snap_step) + "," + g17(time) + "," + grid_c + "," + g17(cfg.density_ratio) +
                           "," + g17(sigma) + "," + g17(cfg.viscosity_ratio) + "," + solver_name + "," + prec_name +
                           "," + std::to_string(cfg.poisson_iterations) + "," + g17(tol) + "," +
                           cfg.analysis_initial_guess;
  std::vector<double> hostv;
  double prev_abs = 0.0, final_abs = 0.0, final_rel = 0.0;
  int final_it = 0;
  dn_status st = DN_OK;
  // one CGMonitor call: the row of the iteration file and, at a key iteration, the residual field
  auto monitor = [&](int it, double alpha, double beta, double absr, double relr, double precr) -> dn_status {
    k_resid_stats<<<128, 256, 0, h->stream>>>(r, mask, n, h->partials);
    DN_TRY(check_launch(h, "k_resid_stats"));
    double q[3];
    DN_TRY(host_partials(h, 3, 128, true, q));
    const double il2 = std::sqrt(q[1]), bl2 = std::sqrt(q[2]);
    const double qk = (it == 0 || prev_abs <= 0.0) ? 1.0 : absr / prev_abs;
    std::fprintf(it_out, "%s,%d,%s,%s,%s,%s,%s,%s,%s,%s,%s,%s,%s\n", lead.c_str(), it, g17(absr).c_str(),
                 g17(relr).c_str(), g17(q[0]).c_str(), g17(precr).c_str(), g17(alpha).c_str(), g17(beta).c_str(),
                 g17(qk).c_str(), g17(il2).c_str(), g17(bl2).c_str(), g17(absr > 0.0 ? il2 / absr : 0.0).c_str(),
                 g17(absr > 0.0 ? bl2 / absr : 0.0).c_str());
    prev_abs = absr;
    final_it = it;
    final_abs = absr;
    final_rel = relr;
    if (keys.count(it)) {
      DN_TRY(download(h, r, hostv, (size_t)n));
      char name[64];
      std::snprintf(name, sizeof name, "residual_iter_%06d.csv", it);
      if (!write_field_csv(field_dir / name, hostv, nx, ny))
        return fail(h, DN_ERR_INVALID_ARGUMENT, "cannot open pressure analysis field file: " + (field_dir / name).string());
    }
    return DN_OK;
  };
  // solve_preconditioned_cg (ch_sparse_krylov.hpp:515-660) from x = 0 with the monitor above
  auto solve = [&]() -> dn_status {
    double q[5];
    DN_CUDA(h, cudaMemsetAsync(x, 0, n * sizeof(double), h->stream));
    k_residual5<<<nb, 256, 0, h->stream>>>(A, h->b, x, r);
    DN_TRY(check_launch(h, "k_residual5"));
    DN_TRY(proj(r));
    DN_TRY(dots4(h, h->b, h->b, r, r, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, q));
    const double rhs_norm = std::sqrt(std::max(q[0], 0.0));
    double absr = std::sqrt(std::max(q[1], 0.0));
    double relr = absr / std::max(rhs_norm, 1.0e-30);
    if (relr < tol || absr < tol) return monitor(0, 0.0, 0.0, absr, relr, 0.0);
    DN_TRY(precondition());
    DN_TRY(dots4(h, r, z, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, q));
    double rz_old = q[0];
    if (!std::isfinite(rz_old) || rz_old <= 0.0)
      return fail(h, DN_ERR_PCG_BREAKDOWN, "pcg preconditioner breakdown: non-positive r^T M^{-1} r");
    DN_TRY(monitor(0, 0.0, 0.0, absr, relr, std::sqrt(std::max(rz_old, 0.0))));
    DN_CUDA(h, cudaMemcpyAsync(p, z, n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    const int limit = std::max(1, cfg.poisson_iterations);
    for (int it = 0; it < limit; ++it) {
      k_spmv5<<<nb, 256, 0, h->stream>>>(A, p, ap);
      DN_TRY(check_launch(h, "k_spmv5"));
      DN_TRY(dots4(h, p, ap, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, q));
      const double pap = q[0];
      if (!std::isfinite(pap) || std::fabs(pap) < 1.0e-30)
        return fail(h, DN_ERR_PCG_BREAKDOWN, "pcg breakdown: p^T A p is invalid");
      const double alpha = rz_old / pap;
      k_x_step<<<nb, 256, 0, h->stream>>>(x, p, delta, n, alpha);
      DN_TRY(check_launch(h, "k_x_step"));
      k_sub_scaled<<<nb, 256, 0, h->stream>>>(r, ap, n, alpha);
      DN_TRY(check_launch(h, "k_sub_scaled"));
      DN_TRY(proj(x));
      DN_TRY(proj(r));
      DN_TRY(dots4(h, r, r, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, q));
      absr = std::sqrt(std::max(q[0], 0.0));
      relr = absr / std::max(rhs_norm, 1.0e-30);
      if (relr < tol || absr < tol) return monitor(it + 1, alpha, 0.0, absr, relr, 0.0);
      DN_TRY(precondition());
      DN_TRY(dots4(h, r, z, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, q));
      const double rz_new = q[0];
      if (!std::isfinite(rz_new) || rz_new <= 0.0)
        return fail(h, DN_ERR_PCG_BREAKDOWN, "pcg preconditioner breakdown: non-positive new r^T M^{-1} r");
      const double beta = rz_new / rz_old;
      DN_TRY(monitor(it + 1, alpha, beta, absr, relr, std::sqrt(std::max(rz_new, 0.0))));
      k_p_update<<<nb, 256, 0, h->stream>>>(p, z, n, beta);
      DN_TRY(check_launch(h, "k_p_update"));
      DN_TRY(proj(p));
      rz_old = rz_new;
    }
    return DN_OK;
  };
  // the fields written before the solve: rhs, interface mask, rho_mid, phi (pressure_analysis.cpp:213-227)
  std::vector<double> cells((size_t)n), full;
  auto write = [&](const char *name, const std::vector<double> &v) -> dn_status {
    if (!write_field_csv(field_dir / name, v, nx, ny))
      return fail(h, DN_ERR_INVALID_ARGUMENT, "cannot open pressure analysis field file: " + (field_dir / name).string());
    return DN_OK;
  };
  if (st == DN_OK) st = download(h, h->b, hostv, (size_t)n);
  if (st == DN_OK) st = write("rhs.csv", hostv);
  if (st == DN_OK) st = download(h, mask, hostv, (size_t)n);
  if (st == DN_OK) st = write("interface_mask.csv", hostv);
  if (st == DN_OK) st = download(h, f[DN_F_RHO_MID].d, full, f[DN_F_RHO_MID].size());
  if (st == DN_OK) {
    const Fv &rm = f[DN_F_RHO_MID];
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j) cells[(size_t)i * ny + j] = full[(size_t)(i + rm.g) * rm.pitch() + (j + rm.g)];
    st = write("rho_mid.csv", cells);
  }
  if (st == DN_OK) st = download(h, f[DN_F_C].d, full, f[DN_F_C].size());
  if (st == DN_OK) {
    const Fv &cf = f[DN_F_C];
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j)
        cells[(size_t)i * ny + j] = 2.0 * full[(size_t)(i + cf.g) * cf.pitch() + (j + cf.g)] - 1.0;
    st = write("phi.csv", cells);
  }
  if (st == DN_OK) st = solve();
  std::fclose(it_out);
  if (st != DN_OK) return st;
  // the final residual b - A x of the last monitored iterate, the pressure means and the summary row
  k_residual5<<<nb, 256, 0, h->stream>>>(A, h->b, x, r);
  DN_TRY(check_launch(h, "k_residual5"));
  DN_TRY(proj(r));
  DN_TRY(download(h, r, hostv, (size_t)n));
  DN_TRY(write("residual_final.csv", hostv));
  double sums[1];
  k_vec_sum<<<128, 256, 0, h->stream>>>(h->b, n, h->partials);
  DN_TRY(check_launch(h, "k_vec_sum"));
  DN_TRY(host_partials(h, 1, 128, false, sums));
  const double rhs_sum = sums[0];
  k_vec_sum<<<128, 256, 0, h->stream>>>(x, n, h->partials);
  DN_TRY(check_launch(h, "k_vec_sum"));
  DN_TRY(host_partials(h, 1, 128, false, sums));
  const double mean_before = sums[0] / (double)n;
  double mean_after = mean_before;
  if (project) {
    DN_TRY(proj(x));
    k_vec_sum<<<128, 256, 0, h->stream>>>(x, n, h->partials);
    DN_TRY(check_launch(h, "k_vec_sum"));
    DN_TRY(host_partials(h, 1, 128, false, sums));
    mean_after = sums[0] / (double)n;
  }
  const fs::path summary = dir / "summary.csv";
  const bool exists = fs::exists(summary);
  FILE *sp = std::fopen(summary.string().c_str(), "a");
  if (!sp) return fail(h, DN_ERR_INVALID_ARGUMENT, "cannot open pressure analysis summary file: " + summary.string());
  if (!exists)
    std::fputs("case_name,case_group,source_mode,step,time,grid_size,density_ratio,sigma,viscosity_ratio,solver_name,"
               "preconditioner_name,max_iter,tolerance,initial_guess_type,rhs_volume_mean,rhs_sum,"
               "pressure_mean_before_fix,pressure_mean_after_fix,nullspace_treatment,final_iter,final_true_res_l2,"
               "final_rel_true_res_l2\n", sp);
  std::fprintf(sp, "%s,%s,%s,%s,%s,%s,%d,%s,%s\n", lead.c_str(), g17(rhs_sum / (double)n).c_str(), g17(rhs_sum).c_str(),
               g17(mean_before).c_str(), g17(mean_after).c_str(), cfg.analysis_nullspace_treatment, final_it,
               g17(final_abs).c_str(), g17(final_rel).c_str());
  std::fclose(sp);
  return DN_OK;
}

// The CH advective term rhs = -div(u c) of `c` (its scalar BC ghosts refilled first) into h->arhs.
dn_status advective_rhs(dn_handle *h, const Fv &c) {
  Fv *f = h->f;
  DN_TRY(bc(h, c, kBCScalar));
  LAUNCH_INTERIOR(k_adv_flux_x, h->afx, c, f[DN_F_U], h->afx);
  LAUNCH_INTERIOR(k_adv_flux_y, h->afy, c, f[DN_F_V], h->afy);
  DN_TRY(bc(h, h->afx, kBCU));
  DN_TRY(bc(h, h->afy, kBCV));
  LAUNCH_INTERIOR(k_flux_div, h->arhs, h->afx, h->afy, h->arhs, h->G, 1);
  return DN_OK;
}

// mode = advection_only (solver.cpp:232-245 with solve_phase_advection_only, phase_field.cpp:398-435): c
// advanced by SSPRK3 with WENO5 fluxes in the current velocity, materials from the new c, mu = 0.
dn_status advection_step(dn_handle *h, dn_report *rep) {
  Fv *f = h->f;
  const double dt = h->cfg.dt;
  const Fv &c0 = h->cmid, &c1 = h->mm, &c2 = h->sm_c;
  DN_TRY(copy_field(h, c0, f[DN_F_C]));
  DN_TRY(advective_rhs(h, c0));
  LAUNCH_INTERIOR(k_ssprk3_stage, c1, c0, c0, h->arhs, c1, dt, 1);
  DN_TRY(advective_rhs(h, c1));
  LAUNCH_INTERIOR(k_ssprk3_stage, c2, c0, c1, h->arhs, c2, dt, 2);
  DN_TRY(advective_rhs(h, c2));
  LAUNCH_INTERIOR(k_ssprk3_stage, f[DN_F_C], c0, c2, h->arhs, f[DN_F_C], dt, 3);
  DN_TRY(bc(h, f[DN_F_C], kBCScalar));
  // ch_residual: ||c - c0|| / ||c|| over the interior (field_diff_l2)
  const int nb = 128;
  k_diff_l2_partials<<<nb, 256, 0, h->stream>>>(f[DN_F_C], c0, h->partials);
  DN_TRY(check_launch(h, "k_diff_l2_partials"));
  DN_CUDA(h, cudaMemcpyAsync(h->host_scal, h->partials, 2 * nb * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  DN_TRY(materials(h, f[DN_F_C], f[DN_F_RHO], f[DN_F_ETA]));
  DN_TRY(fill_field(h, f[DN_F_MU], 0.0));
  DN_TRY(bc(h, f[DN_F_MU], kBCScalar));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  double d2 = 0.0, n2 = 0.0;
  for (int b = 0; b < nb; ++b) {
    d2 += h->host_scal[b];
    n2 += h->host_scal[nb + b];
  }
  rep->ch_residual = std::sqrt(d2 / std::max(n2, 1.0e-30));
  rep->ch_iterations = 3;
  rep->momentum_iterations = 0;
  rep->pressure_iterations = 0;
  rep->coupling_iterations = 0;
  rep->boundary_speed_pre = 0.0;
  rep->boundary_speed_post = 0.0;
  rep->ch_equation_residual = 0.0;
  return DN_OK;
}

dn_status pressure(dn_handle *h, int step, dn_report *rep) {
  Fv *f = h->f;
  const dn_config &cfg = h->cfg;
  if (cfg.pressure_scheme == DN_P_JACOBI) return pressure_jacobi(h, rep);
  const bool split = use_split(cfg);
  const bool icc = cfg.pressure_scheme == DN_P_ICPCG || cfg.pressure_scheme == DN_P_SPLIT_ICPCG;
  DN_TRY(fill_field(h, f[DN_F_P_CORR], 0.0));
  DN_TRY(bc(h, f[DN_F_P_CORR], kBCPressure));
  const double rho_ref = split ? rho_ref_of(cfg) : 1.0;
  if (split) DN_TRY(split_extrapolation(h, step));
  k_p_assemble<<<blocks_for(h->n), 256, 0, h->stream>>>(h->G, h->bc, f[DN_F_RHO_MID], f[DN_F_U_STAR], f[DN_F_V_STAR],
                                                       h->pe, split ? 1 : 0, rho_ref, cfg.dt, h->a5, h->b);
  DN_TRY(check_launch(h, "k_p_assemble"));
  if (!h->has_dirichlet) DN_TRY(compact_subtract_mean(h, h->b));  // pressure.cpp:198-212
  if (cfg.pressure_scheme == DN_P_SPLIT_DCDM_ICPCG) {
    DN_TRY(pressure_factor(h, true, true));  // build_icc_preconditioner_strict
    DN_TRY(dcdm_solve(h, rep));
  } else {
    DN_TRY(pressure_factor_solve(h, split, icc, rep));
  }
  LAUNCH_INTERIOR(k_scatter_compact, f[DN_F_P_CORR], h->x, f[DN_F_P_CORR]);
  if (!h->has_dirichlet) DN_TRY(subtract_mean(h, f[DN_F_P_CORR]));
  return bc(h, f[DN_F_P_CORR], kBCPressure);
}

// x = A^-1 b for the assembled pressure operator a5 and right-hand side b, from x = 0: the factor (built
// once for the constant split operator, every call for the variable one), then the PCG of the configured
// precision and sweep form.
dn_status pressure_factor(dn_handle *h, bool split, bool icc) {
  const int kind = icc ? kPrecICC : kPrecLDLT;
  if (!(split && h->p_factor_valid && h->p_factor_kind == kind)) {
    DN_CUDA(h, cudaMemsetAsync(h->status, 0, sizeof(int), h->stream));
    Factor F{h->l5, h->d5, h->dinv5, 0.0};
    k_factor<5><<<1, 1024, 0, h->stream>>>(SpOp{h->a5, (int)h->n, h->G.nx, h->G.ny, h->G.px, h->G.py}, F, kind,
                                            h->status);
    DN_TRY(check_launch(h, "k_factor<5>"));
    if (h->capturing) {  // recorded: the status goes to the step record (a failed factor is reported after)
      k_rec_copy<<<1, 32, 0, h->stream>>>(nullptr, 0, h->status, h->rec + kRecStep + kSPFactor);
      return check_launch(h, "k_rec_copy");
    }
    int st = 0;
    DN_TRY(read_status(h, &st));
    if (st == kDevFactorFailed) {
      h->p_factor_valid = false;
      return fail(h, icc ? DN_ERR_ICC_FAILED : DN_ERR_ILDLT_FAILED,
                  icc ? "ICC preconditioner construction failed" : "ILDLT preconditioner construction failed");
    }
    h->p_factor_valid = split;
    h->p_factor_kind = kind;
  }
  return DN_OK;
}

dn_status pressure_factor_solve(dn_handle *h, bool split, bool icc, dn_report *rep) {
  const dn_config &cfg = h->cfg;
  const int kind = icc ? kPrecICC : kPrecLDLT;
  // the mixed form builds the factor only when its inner solves use it
  if (cfg.precision != DN_PRECISION_MIXED) DN_TRY(pressure_factor(h, split, icc));
  DN_CUDA(h, cudaMemsetAsync(h->x, 0, h->n * sizeof(double), h->stream));
  double out[4];
  rep->refinement_cycles = 0;
  rep->mixed_inner_multigrid = 0;
  if (cfg.precision == DN_PRECISION_MIXED) {
    DN_TRY(mixed_pressure(h, split, kind, out));
    rep->refinement_cycles = h->refinement_cycles;
    rep->mixed_inner_multigrid = h->mixed_used_mg ? 1 : 0;
  } else if (h->sw5 > 0 && h->G.px) {
    DN_TRY((run_pcg<5, 4>(h, h->a5, h->l5, h->dinv5, kind, h->has_dirichlet ? 0 : 1, cfg.poisson_iterations,
                          cfg.pressure_tolerance, out, h->rec + kRecStep + kSP)));
  } else if (h->sw5 > 0) {
    DN_TRY((run_pcg<5, 3>(h, h->a5, h->l5, h->dinv5, kind, h->has_dirichlet ? 0 : 1, cfg.poisson_iterations,
                          cfg.pressure_tolerance, out, h->rec + kRecStep + kSP)));
  } else {
    DN_TRY((run_pcg<5, 0>(h, h->a5, h->l5, h->dinv5, kind, h->has_dirichlet ? 0 : 1, cfg.poisson_iterations,
                          cfg.pressure_tolerance, out, h->rec + kRecStep + kSP)));
  }
  rep->pressure_iterations = (int)out[0];
  rep->pressure_residual = out[2];
  h->phase_ms[7] = out[0];
  h->mon_count = cfg.precision == DN_PRECISION_MIXED ? 0 : std::min((int)out[0], h->mon_cap);
  return DN_OK;
}

// apply_pressure_velocity_correction, operators.cpp:480-534
dn_status correct(dn_handle *h, int step, dn_report *rep) {
  Fv *f = h->f;
  const dn_config &cfg = h->cfg;
  k_boundary_speed<<<1, 256, 0, h->stream>>>(f[DN_F_U_STAR], f[DN_F_V_STAR], h->G, h->scal + 16);
  DN_TRY(check_launch(h, "k_boundary_speed"));
  const bool split = use_split(cfg);
  const double rho_ref = split ? rho_ref_of(cfg) : 1.0;
  if (split) DN_TRY(split_extrapolation(h, step));
  LAUNCH_INTERIOR(k_correct_u, f[DN_F_U], f[DN_F_U], f[DN_F_U_STAR], f[DN_F_RHO_MID], f[DN_F_P_CORR], h->pe, h->G,
                  split ? 1 : 0, rho_ref, cfg.dt);
  LAUNCH_INTERIOR(k_correct_v, f[DN_F_V], f[DN_F_V], f[DN_F_V_STAR], f[DN_F_RHO_MID], f[DN_F_P_CORR], h->pe, h->G,
                  split ? 1 : 0, rho_ref, cfg.dt);
  DN_TRY(bc(h, f[DN_F_U], kBCU));
  DN_TRY(bc(h, f[DN_F_V], kBCV));
  k_boundary_speed<<<1, 256, 0, h->stream>>>(f[DN_F_U], f[DN_F_V], h->G, h->scal + 17);
  DN_TRY(check_launch(h, "k_boundary_speed"));
  DN_TRY(copy_field(h, f[DN_F_P_PREV], f[DN_F_P]));
  LAUNCH_INTERIOR(k_copy_interior, f[DN_F_P], f[DN_F_P], f[DN_F_P_CORR]);
  if (!h->has_dirichlet) DN_TRY(subtract_mean(h, f[DN_F_P]));
  DN_TRY(bc(h, f[DN_F_P], kBCPressure));
  if (h->capturing) return DN_OK;  // the boundary speeds are read with the step record
  double bs[2];
  DN_CUDA(h, cudaMemcpyAsync(h->host_scal, h->scal + 16, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  std::memcpy(bs, h->host_scal, sizeof bs);
  rep->boundary_speed_pre = bs[0];
  rep->boundary_speed_post = bs[1];
  return DN_OK;
}

dn_status begin_step(dn_handle *h) {
  Fv *f = h->f;
  DN_TRY(copy_field(h, f[DN_F_C_PREV2], f[DN_F_C_PREV]));
  DN_TRY(copy_field(h, f[DN_F_C_PREV], f[DN_F_C]));
  DN_TRY(copy_field(h, f[DN_F_RHO_PREV], f[DN_F_RHO]));
  DN_TRY(copy_field(h, f[DN_F_ETA_PREV], f[DN_F_ETA]));
  DN_TRY(copy_field(h, f[DN_F_U_PREV], f[DN_F_U]));
  return copy_field(h, f[DN_F_V_PREV], f[DN_F_V]);
}

dn_status diag_launch(dn_handle *h) {
  Fv *f = h->f;
  k_diag_partials<<<kDiagParts, 256, 0, h->stream>>>(f[DN_F_C], f[DN_F_U], f[DN_F_V], f[DN_F_MU], f[DN_F_RHO],
                                                     f[DN_F_ETA], h->G, h->cfg.cn, h->partials);
  return check_launch(h, "k_diag_partials");
}

// compute_diagnostics (diagnostics.cpp:114-167) from k_diag_partials' per-CTA values (host copy `part`)
dn_status diag_finish(dn_handle *h, const double *part, dn_diag *d) {
  const int nb = kDiagParts;
  const int ops[kNDiag] = {0, 0, 1, 1, 1, 0, 2, 1, 2, 1, 0, 1, 1, 1};
  double a[kNDiag];
  for (int k = 0; k < kNDiag; ++k) {
    a[k] = ops[k] == 0 ? 0.0 : (ops[k] == 1 ? -INFINITY : INFINITY);
    for (int b = 0; b < nb; ++b) {
      const double v = part[b * kNDiag + k];
      a[k] = ops[k] == 0 ? a[k] + v : (ops[k] == 1 ? std::max(a[k], v) : std::min(a[k], v));
    }
  }
  const dn_config &c = h->cfg;
  std::memset(d, 0, sizeof(*d));
  d->mass = a[0];
  d->mass_drift = std::fabs(a[0] - h->initial_mass);
  d->divergence_l2 = std::sqrt(a[1] / (double)(c.nx * c.ny));
  d->max_divergence = std::max(0.0, a[2]);
  d->max_abs_mu = std::max(0.0, a[3]);
  d->max_velocity = std::max(0.0, a[4]);
  d->kinetic_energy = a[5];
  d->rho_min = a[6];
  d->rho_max = std::max(0.0, a[7]);
  d->eta_min = a[8];
  d->eta_max = std::max(0.0, a[9]);
  d->total_free_energy = a[10];
  // populate_timestep_limits, diagnostics.cpp:48-112
  const double h_ = std::min(h->G.dx, h->G.dy), tiny = 1.0e-30;
  const double mar = std::max(0.0, a[11]);
  d->dt_limit_advective = mar > tiny ? 0.5 / mar : INFINITY;
  d->dt_limit_capillary = INFINITY;
  d->dt_limit_ch_explicit = INFINITY;
  if (solve_ch(c)) {
    const double rs = std::max(d->rho_max, tiny);
    d->dt_limit_capillary = 0.5 * std::sqrt(std::max(c.re * c.ca * h_ * h_ * h_ / rs, 0.0));
    const double mob = std::max(0.0, a[12]), wpp = std::max(0.0, a[13]);
    if (mob > tiny) {
      const double coeff = 6.0 * kSqrt2 * mob * wpp / std::max(c.pe * c.cn, tiny);
      d->dt_limit_ch_explicit = coeff > tiny ? 0.25 * h_ * h_ / coeff : INFINITY;
    }
  }
  d->dt_limit_active = d->dt_limit_advective;
  if (d->dt_limit_capillary < d->dt_limit_active) d->dt_limit_active = d->dt_limit_capillary;
  if (d->dt_limit_ch_explicit < d->dt_limit_active) d->dt_limit_active = d->dt_limit_ch_explicit;
  d->dt_limit_ratio = (!std::isfinite(d->dt_limit_active) || d->dt_limit_active <= tiny) ? 0.0 : c.dt / d->dt_limit_active;
  if (!std::isfinite(d->mass_drift) || !std::isfinite(d->divergence_l2) || !std::isfinite(d->max_velocity) ||
      !std::isfinite(d->max_abs_mu))
    return fail(h, DN_ERR_NONFINITE, "non-finite diagnostic detected");
  return DN_OK;
}


// ---- captured steps
// A step with no host decision left -- the CH operator and its factor or hierarchy made for this alpha0, the
// split operator's factor or hierarchy made, no pressure analysis, monitor or DCDM / Jacobi scheme -- is
// recorded once into a CUDA graph: the solves' loops are conditional nodes, every result lands in h->rec
// (read back once per step), the phase boundaries are event nodes.  Every kernel that depends on the step
// index tests step == 0 only, so one recording serves every step >= 1.
constexpr int kHostRec = 4096;   // pinned host copies of a replayed step: the record and boundary speeds,
constexpr int kHostDiag = 4352;  // and the diagnostics partials

bool step_capturable(const dn_handle *h, int step) {
  const dn_config &c = h->cfg;
  if (!h->graph_steps || !h->steady || step < 1) return false;
  if (c.mode == DN_MODE_ADVECTION_ONLY || c.analysis_enabled || h->mon_cap > 0) return false;
  if (c.pressure_scheme == DN_P_JACOBI || c.pressure_scheme == DN_P_SPLIT_DCDM_ICPCG) return false;
  if (solve_ch(c)) {
    const double alpha0 = 3.0 / (2.0 * c.dt);
    if (!(std::fabs(alpha0 - h->ch_alpha0) <= 1.0e-14 * std::max(1.0, std::fabs(alpha0)))) return false;
    if (h->ch_mg && c.precision == DN_PRECISION_MIXED && h->ch_mg_alpha0 != alpha0) return false;
  }
  if (use_split(c)) {
    const int kind = c.pressure_scheme == DN_P_SPLIT_ICPCG ? kPrecICC : kPrecLDLT;
    if (c.precision == DN_PRECISION_MIXED ? !h->mgp_split_ready : !(h->p_factor_valid && h->p_factor_kind == kind))
      return false;
  }
  return true;
}

// dn_step's work with h->capturing set (nothing read back); rep receives the fields fixed at capture
dn_status record_step(dn_handle *h, int step, dn_report *rep) {
  std::memset(rep, 0, sizeof(*rep));
  rep->ch_preconditioner = -1;
  const long long before = h->launches;
  h->step_dcn[0] = h->step_dcn[1] = DcNodes{};
  h->step_retry = 0;
  h->step = step;
  DN_CUDA(h, cudaEventRecordWithFlags(h->ev[0], h->stream, cudaEventRecordExternal));
  DN_TRY(begin_step(h));
  DN_TRY(phase(h, step, rep));
  DN_CUDA(h, cudaEventRecordWithFlags(h->ev[1], h->stream, cudaEventRecordExternal));
  DN_TRY(momentum(h, step, rep));
  DN_CUDA(h, cudaEventRecordWithFlags(h->ev[2], h->stream, cudaEventRecordExternal));
  DN_TRY(pressure(h, step, rep));
  DN_CUDA(h, cudaEventRecordWithFlags(h->ev[3], h->stream, cudaEventRecordExternal));
  DN_TRY(correct(h, step, rep));
  DN_CUDA(h, cudaEventRecordWithFlags(h->ev[4], h->stream, cudaEventRecordExternal));
  DN_TRY(diag_launch(h));
  // launches of one replay outside the loops (each loop body was recorded once)
  long long bodies = 0;
  for (const DcNodes &d : h->step_dcn) bodies += d.cycle + d.iter + d.ic + d.make;
  bodies += h->step_retry;
  h->step_nodes = h->launches - before - bodies;
  h->launches = before;
  return DN_OK;
}

dn_status ensure_step_graph(dn_handle *h, int step) {
  if (h->step_exec && h->step_epoch == h->graph_epoch) return DN_OK;
  if (h->step_exec) cudaGraphExecDestroy(h->step_exec);
  h->step_exec = nullptr;
  DN_TRY(capture_exec(h, &h->step_exec, [&]() { return record_step(h, step, &h->step_rep); }));
  h->step_epoch = h->graph_epoch;
  return DN_OK;
}

// the copies a replayed step's results need, issued on `st` after the replay
dn_status step_readback(dn_handle *h, cudaStream_t st) {
  DN_CUDA(h, cudaMemcpyAsync(h->host_scal + kHostRec, h->rec, kRecCount * sizeof(double), cudaMemcpyDeviceToHost, st));
  DN_CUDA(h, cudaMemcpyAsync(h->host_scal + kHostRec + kRecCount, h->scal + 16, 2 * sizeof(double),
                             cudaMemcpyDeviceToHost, st));
  DN_CUDA(h, cudaMemcpyAsync(h->host_scal + kHostDiag, h->partials, (size_t)kDiagParts * kNDiag * sizeof(double),
                             cudaMemcpyDeviceToHost, st));
  return DN_OK;
}


// The report, statuses and diagnostics of a replayed step from its record (after step_readback and a
// synchronisation), as dn_step reports them.
dn_status step_complete(dn_handle *h, int step, dn_report *rep) {
  const dn_config &c = h->cfg;
  const double *R = h->host_scal + kHostRec;
  const double *S = R + kRecStep;
  *rep = h->step_rep;
  h->step = step;
  for (int k = 0; k < 4; ++k) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, h->ev[k], h->ev[k + 1]);
    h->phase_ms[k] = ms;
  }
  for (int k = 4; k < 8; ++k) h->phase_ms[k] = 0.0;
  long long launches = h->step_nodes;
  if (solve_ch(c)) {
    if (rep->ch_preconditioner == 3) {
      const double *C = R + kRecCh;
      rep->ch_iterations = (int)C[kDcTotal];
      rep->ch_residual = C[kDcIres];
      launches += dc_launches(h->step_dcn[1], C);
    } else {
      const int st = (int)S[kSChPcg + 4];
      if (st != kDevOk) return dev_status_to_dn(h, st);
      rep->ch_iterations = (int)S[kSChPcg];
      rep->ch_residual = S[kSChPcg + 3];
      if (S[kSChRetry] != 0.0) {  // phase_field.cpp:468-473: the diagonal preconditioner from now on
        launches += h->step_retry;
        rep->ch_preconditioner = 2;
        h->ch_prec = kPrecDiag;
        ++h->graph_epoch;
      }
    }
    rep->ch_equation_residual = S[kSChEq];
  }
  {
    const int st = (int)S[kSMom + 4];
    if (st != kDevOk) return dev_status_to_dn(h, st);
    rep->momentum_iterations = (int)S[kSMom];
    rep->momentum_residual = S[kSMom + 1];
  }
  const bool split = use_split(c);
  const bool icc = c.pressure_scheme == DN_P_ICPCG || c.pressure_scheme == DN_P_SPLIT_ICPCG;
  if (c.precision == DN_PRECISION_MIXED) {
    const double *P = R + kRecPressure;
    DN_TRY(dc_error(h, P, icc ? kPrecICC : kPrecLDLT));
    rep->pressure_iterations = (int)P[kDcTotal];
    rep->pressure_residual = P[kDcRel];
    rep->refinement_cycles = (int)P[kDcCycles];
    rep->mixed_inner_multigrid = P[kDcUsedMg0] != 0.0 ? 1 : 0;
    h->refinement_cycles = rep->refinement_cycles;
    h->mixed_used_mg = rep->mixed_inner_multigrid != 0;
    launches += dc_launches(h->step_dcn[0], P);
  } else {
    if (!split && (int)S[kSPFactor] == kDevFactorFailed)
      return fail(h, icc ? DN_ERR_ICC_FAILED : DN_ERR_ILDLT_FAILED,
                  icc ? "ICC preconditioner construction failed" : "ILDLT preconditioner construction failed");
    const int st = (int)S[kSP + 4];
    if (st != kDevOk) return dev_status_to_dn(h, st);
    rep->pressure_iterations = (int)S[kSP];
    rep->pressure_residual = S[kSP + 2];
  }
  h->phase_ms[7] = rep->pressure_iterations;
  rep->boundary_speed_pre = R[kRecCount];
  rep->boundary_speed_post = R[kRecCount + 1];
  h->launches += launches;
  return diag_finish(h, h->host_scal + kHostDiag, &h->last_diag);
}

// one step replayed from the handle's graph (recorded on first use)
dn_status graph_step(dn_handle *h, int step, dn_report *rep) {
  DN_TRY(ensure_step_graph(h, step));
  DN_CUDA(h, cudaGraphLaunch(h->step_exec, h->stream));
  DN_TRY(step_readback(h, h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  return step_complete(h, step, rep);
}

// One step of every handle as one launch: each handle's step recorded as a branch of one graph (the handle's
// stream joins the capture of the batch stream, records its step, and is joined back), captured once for
// this list of handles and replayed; the results of every handle are read back with one synchronisation.
dn_status batch_graph_step(dn_handle *const *hs, int count, const int *steps, dn_report *reports) {
  dn_handle *o = hs[0];
  dn_handle::BatchGraph &B = o->batch;
  bool fresh = B.exec != nullptr && (int)B.uids.size() == count;
  for (int a = 0; fresh && a < count; ++a)
    fresh = B.uids[(size_t)a] == hs[a]->uid && B.epochs[(size_t)a] == hs[a]->graph_epoch;
  if (!fresh) {
    if (B.exec) cudaGraphExecDestroy(B.exec);
    B.exec = nullptr;
    if (!B.stream) DN_CUDA(o, cudaStreamCreateWithFlags(&B.stream, cudaStreamNonBlocking));
    if (!B.fork) DN_CUDA(o, cudaEventCreateWithFlags(&B.fork, cudaEventDisableTiming));
    DN_CUDA(o, cudaStreamBeginCapture(B.stream, cudaStreamCaptureModeThreadLocal));
    dn_status st = DN_OK;
    if (cudaEventRecord(B.fork, B.stream) != cudaSuccess) st = fail(o, DN_ERR_CUDA, "batch capture fork");
    int joined = 0;
    for (int a = 0; a < count && st == DN_OK; ++a) {
      dn_handle *h = hs[a];
      if (cudaStreamWaitEvent(h->stream, B.fork, 0) != cudaSuccess) {
        st = fail(o, DN_ERR_CUDA, "batch capture join");
        break;
      }
      h->capturing = true;
      st = record_step(h, steps[a], &h->step_rep);
      h->capturing = false;
      if (cudaEventRecord(h->cap_ev, h->stream) != cudaSuccess || cudaStreamWaitEvent(B.stream, h->cap_ev, 0) != cudaSuccess)
        if (st == DN_OK) st = fail(o, DN_ERR_CUDA, "batch capture rejoin");
      ++joined;
      if (st != DN_OK && h != o) o->err = h->err;
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(B.stream, &g);
    if (st != DN_OK || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return st != DN_OK ? st : fail(o, DN_ERR_CUDA, std::string("batch capture: ") + cudaGetErrorString(ce));
    }
    const cudaError_t ie = cudaGraphInstantiate(&B.exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      B.exec = nullptr;
      return fail(o, DN_ERR_CUDA, std::string("batch graph: ") + cudaGetErrorString(ie));
    }
    (void)joined;
    B.uids.assign((size_t)count, 0);
    B.epochs.assign((size_t)count, 0);
    for (int a = 0; a < count; ++a) {
      B.uids[(size_t)a] = hs[a]->uid;
      B.epochs[(size_t)a] = hs[a]->graph_epoch;
    }
  }
  DN_CUDA(o, cudaGraphLaunch(B.exec, B.stream));
  for (int a = 0; a < count; ++a) DN_TRY(step_readback(hs[a], B.stream));
  DN_CUDA(o, cudaStreamSynchronize(B.stream));
  dn_status first = DN_OK;
  for (int a = 0; a < count; ++a) {
    dn_report local{};
    const dn_status st = step_complete(hs[a], steps[a], reports ? &reports[a] : &local);
    if (st != DN_OK && first == DN_OK) first = st;
  }
  return first;
}
}  // namespace

// ===================================================================================================
// C-ABI
// ===================================================================================================
extern "C" {

const char *dn_status_string(dn_status s) {
  switch (s) {
  case DN_OK: return "ok";
  case DN_ERR_INVALID_ARGUMENT: return "invalid argument";
  case DN_ERR_CONFIG: return "invalid configuration";
  case DN_ERR_CUDA: return "CUDA error";
  case DN_ERR_ICC_FAILED: return "ICC preconditioner construction failed";
  case DN_ERR_ILDLT_FAILED: return "ILDLT preconditioner construction failed";
  case DN_ERR_PCG_BREAKDOWN: return "pcg breakdown";
  case DN_ERR_BICGSTAB_BREAKDOWN: return "bicgstab breakdown";
  case DN_ERR_TIMEOUT: return "device wait timed out";
  case DN_ERR_NONFINITE: return "non-finite diagnostic detected";
  case DN_ERR_UNSUPPORTED: return "unsupported configuration";
  }
  return "unknown status";
}

const char *dn_last_error(const dn_handle *h) { return h ? h->err.c_str() : "null handle"; }

dn_status dn_create(const dn_config *cfg, int device, dn_handle **out) {
  if (!cfg || !out) return DN_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  dn_handle *h = new dn_handle();
  h->cfg = *cfg;
  const dn_config &c = h->cfg;
  auto bad = [&](dn_status s, const std::string &m) {
    h->err = m;
    *out = h;
    return s;
  };
  if (c.nx < 8 || c.ny < 8) return bad(DN_ERR_UNSUPPORTED, "the CUDA backend needs nx, ny >= 8");
  if (c.ghost < 3) return bad(DN_ERR_UNSUPPORTED, "ghost must be >= 3 (WENO5 stencil)");
  if ((long long)c.nx * c.ny > (1LL << 30)) return bad(DN_ERR_UNSUPPORTED, "grid too large");
  // validate_boundary_configuration, operators.cpp:11-34
  static const char *names[4] = {"left", "right", "bottom", "top"};
  for (int s = 0; s < 4; ++s) {
    const int periodic = (s < 2) ? c.periodic_x : c.periodic_y;
    if (!periodic) continue;
    if (c.p_bc[s].type != DN_BC_UNSET)
      return bad(DN_ERR_CONFIG, std::string("pressure_bc_") + names[s] + " cannot be set when the direction is periodic");
    if (c.u_bc[s].type != DN_BC_UNSET)
      return bad(DN_ERR_CONFIG, std::string("u_bc_") + names[s] + " cannot be set when the direction is periodic");
    if (c.v_bc[s].type != DN_BC_UNSET)
      return bad(DN_ERR_CONFIG, std::string("v_bc_") + names[s] + " cannot be set when the direction is periodic");
  }
  if (c.surface_tension_smoothing_passes < 0)
    return bad(DN_ERR_CONFIG, "surface_tension_smoothing_passes must be non-negative");
  if (c.surface_tension_smoothing_weight < 0.0 || c.surface_tension_smoothing_weight > 0.25)
    return bad(DN_ERR_CONFIG, "surface_tension_smoothing_weight must lie in [0, 0.25]");

  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return bad(DN_ERR_CUDA, "no CUDA device available");
  if (device < 0) cudaGetDevice(&device);
  h->device = device;
  if (cudaSetDevice(device) != cudaSuccess) return bad(DN_ERR_CUDA, "cudaSetDevice failed");
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  h->num_sms = prop.multiProcessorCount;
  h->cta_cap = std::max(1, h->num_sms / std::max(1, cfg->device_share));
  h->rows_per_cta = cfg->pcg_rows_per_cta > 0 ? cfg->pcg_rows_per_cta : kPcgRowsPerCta;
  h->mg_cluster_cells = cfg->mg_cluster_cells > 0 ? cfg->mg_cluster_cells : kMgClusterCells;
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return bad(DN_ERR_CUDA, "stream");
  for (cudaStream_t &cs : h->cap_streams)
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return bad(DN_ERR_CUDA, "stream");
  for (auto &e : h->ev) cudaEventCreate(&e);
  for (auto &e : h->kev) cudaEventCreate(&e);
  cudaEventCreateWithFlags(&h->cap_ev, cudaEventDisableTiming);
  {
    static std::atomic<long long> next_uid{0};
    h->uid = ++next_uid;
  }

  // grid and effective BCs (operators.cpp:36-112)
  h->G.nx = c.nx;
  h->G.ny = c.ny;
  h->G.g = c.ghost;
  h->G.px = c.periodic_x;
  h->G.py = c.periodic_y;
  h->G.dx = c.lx / std::max((double)c.nx, 1.0);
  h->G.dy = c.ly / std::max((double)c.ny, 1.0);
  for (int s = 0; s < 4; ++s) {
    h->bc.p[s] = c.p_bc[s].type != DN_BC_UNSET ? BCSide{c.p_bc[s].type, c.p_bc[s].value} : BCSide{DN_BC_NEUMANN, 0.0};
    h->bc.v[s] = c.v_bc[s].type != DN_BC_UNSET ? BCSide{c.v_bc[s].type, c.v_bc[s].value} : BCSide{DN_BC_DIRICHLET, 0.0};
    if (c.u_bc[s].type != DN_BC_UNSET) {
      h->bc.u[s] = BCSide{c.u_bc[s].type, c.u_bc[s].value};
    } else {
      double v = 0.0;
      if (s == DN_BOTTOM) v = c.bottom_wall_velocity_x;
      if (s == DN_TOP) v = c.top_wall_velocity_x;
      h->bc.u[s] = BCSide{DN_BC_DIRICHLET, v};
    }
  }
  h->has_dirichlet = (!c.periodic_x && (h->bc.p[0].type == DN_BC_DIRICHLET || h->bc.p[1].type == DN_BC_DIRICHLET)) ||
                     (!c.periodic_y && (h->bc.p[2].type == DN_BC_DIRICHLET || h->bc.p[3].type == DN_BC_DIRICHLET));

  dn_status s = DN_OK;
  auto A = [&](dn_status st) {
    if (s == DN_OK) s = st;
  };
  const int nx = c.nx, ny = c.ny;
  for (int k = 0; k < DN_F_COUNT; ++k) {
    const bool one = k == DN_F_RHO || k == DN_F_ETA || k == DN_F_RHO_PREV || k == DN_F_ETA_PREV ||
                     k == DN_F_RHO_MID || k == DN_F_ETA_MID;
    A(falloc(h, h->f[k], is_uish(k) ? nx + 1 : nx, is_vish(k) ? ny + 1 : ny, one ? 1.0 : 0.0));
  }
  for (Fv *w : {&h->mob, &h->lap, &h->bih, &h->mu_t, &h->arhs, &h->ddiv, &h->E_new, &h->cmid, &h->mm, &h->pe, &h->sm_c})
    A(falloc(h, *w, nx, ny, 0.0));
  for (Fv *w : {&h->afx, &h->dfx, &h->urhs, &h->hu, &h->sm_u}) A(falloc(h, *w, nx + 1, ny, 0.0));
  for (Fv *w : {&h->afy, &h->dfy, &h->vrhs, &h->hv, &h->sm_v}) A(falloc(h, *w, nx, ny + 1, 0.0));
  h->n = (long long)nx * ny;
  for (double **p : {&h->b, &h->x, &h->r, &h->z, &h->y, &h->p0, &h->p1, &h->ap, &h->d5, &h->dinv5, &h->d13, &h->dinv13})
    A(dalloc(h, p, h->n));
  A(dalloc(h, &h->a5, 5 * h->n));
  A(dalloc(h, &h->l5, 5 * h->n));
  A(dalloc(h, &h->a13, 13 * h->n));
  A(dalloc(h, &h->l13, 13 * h->n));
  // ordered factor rows for the ring-based CH sweeps: neither direction periodic and the ring fits in shared
  // memory (periodic x keeps the level sweep on global memory: a self-checked run of the wrapped rows found
  // no bad index, but the unchecked build faulted on them, so that combination stays off)
  if (!c.periodic_x && !c.periodic_y && (size_t)kLvlRing * nx * sizeof(double) <= 96 * 1024 && nx < 65536) {
    const int k = 6;
    h->rows13.k = k;
    A(dalloc(h, &h->rows13.lval, (size_t)k * h->n));
    A(dalloc(h, &h->rows13.uval, (size_t)k * h->n));
    A(dalloc(h, &h->rows13.lcol, (size_t)k * h->n));
    A(dalloc(h, &h->rows13.ucol, (size_t)k * h->n));
    A(dalloc(h, &h->rows13.lsrc, (size_t)k * h->n));
    A(dalloc(h, &h->rows13.usrc, (size_t)k * h->n));
  }
  // the CH PCG kernel's dynamic shared memory (the ring, or the periodic-y line buffers): allow the largest
  // amount any handle uses
  if ((h->rows13.lval != nullptr || c.periodic_y) && s == DN_OK)
    cudaFuncSetAttribute(k_pcg<13, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSeqSmemMax);
  h->ml = MomLayout{nx, ny, c.periodic_x, c.periodic_y, (long long)(nx + 1) * ny, (long long)nx * (ny + 1)};
  h->nm = h->ml.nu + h->ml.nv;
  if (h->nm >= (1LL << 31))
    return bad(DN_ERR_INVALID_ARGUMENT, "grid too large for the momentum system's 32-bit column indices");
  A(dalloc(h, &h->mcoef, 9 * h->nm));
  A(dalloc(h, &h->mtgt, 9 * h->nm));
  for (double **p : {&h->mb, &h->mx, &h->mr, &h->mrhat, &h->mp0, &h->mp1, &h->mv0, &h->mv1, &h->mphat, &h->ms, &h->mshat,
                     &h->mt, &h->mupd, &h->mdinv})
    A(dalloc(h, p, h->nm));
  A(dalloc(h, &h->bar_count, 1));
  A(dalloc(h, &h->bar_gen, 1));
  A(dalloc(h, &h->status, 4));  // [status, pad, poll limit of the device waits (long long)]
  A(dalloc(h, &h->prog, 2 * (size_t)kMaxBlocks * 8));
  A(dalloc(h, &h->partials, 2 * (size_t)kMaxBlocks * 8));
  A(dalloc(h, &h->scal, 64));
  A(dalloc(h, &h->rec, kRecCount));
  A(dalloc(h, &h->prof, 64));
  if (s == DN_OK && cudaMallocHost(&h->host_scal, kHostScal * sizeof(double)) != cudaSuccess) s = DN_ERR_CUDA;
  if (s != DN_OK) return bad(s, "device allocation failed: " + h->err);
  {
    const long long limit = c.device_wait_limit;  // 0: the device code's default
    if (cudaMemcpyAsync(h->status + 2, &limit, sizeof limit, cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
      return bad(DN_ERR_CUDA, "setting the device wait limit failed");
  }
  h->nsweep = (nx + 31) / 32;
  h->nsweep5 = staged_sweep_warps(nx);
  A(dalloc(h, &h->bnd_f, 2 * (size_t)std::max(h->nsweep, h->nsweep5) * ny));
  A(dalloc(h, &h->bnd_b, 2 * (size_t)std::max(h->nsweep, h->nsweep5) * ny));
  A(dalloc(h, &h->wline0, 2 * (size_t)ny));
  A(dalloc(h, &h->zlast, 2 * (size_t)ny));
  if (s != DN_OK) return bad(s, "device allocation failed: " + h->err);
  {
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    h->smem_optin = optin;
    auto round16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
    // periodic x takes the staged path with its wrap terms when line nx-1 lies in another warp than line 0
    const bool px = c.periodic_x != 0;
    const bool stageable = !px || h->nsweep5 >= 2;
    const void *k53 = px ? (const void *)k_pcg<5, 4> : (const void *)k_pcg<5, 3>;
    h->sw5_warp_smem[0] = round16(sweep_warp_smem(2, ny, 8, px));
    h->sw5_warp_smem[1] = round16(sweep_warp_smem(4, ny, 8, px));
    const size_t per = h->sw5_warp_smem[use_split(c) ? 0 : 1];
    const size_t budget = (size_t)optin > 64 + 2304 ? (size_t)optin - 64 - 2304 : 0;  // minus static smem
    int sw = stageable ? (int)std::min<size_t>(kSweepWarpsPerCta, budget / per) : 0;
    sw = std::min(sw, h->nsweep5);
    h->sw5_budget = stageable ? sw : 0;
    if (sw > 0 && c.sweep_warps_per_cta > 0) sw = std::min(sw, c.sweep_warps_per_cta);
    h->sw5 = stageable ? sw : 0;
    if (h->sw5 > 0) {
      const size_t dyn = 64 + (size_t)sw * per;
      // The limit is a property of the kernel on this device, shared by every handle: set it to the device
      // maximum, so that a later handle with a smaller grid never lowers it below an earlier handle's need.
      cudaFuncAttributes fa{};
      cudaFuncGetAttributes(&fa, k53);
      cudaFuncSetAttribute(k53, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           std::max((int)dyn, optin - (int)fa.sharedSizeBytes));
      for (int w = 1; w <= h->sw5_budget; ++w) {
        int occ5 = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ5, k53, kBlock, 64 + (size_t)w * per);
        h->sw5_blocks_by_sw[w] = std::min(kMaxBlocks, std::max(0, occ5) * h->num_sms);
      }
      h->sw5_blocks_max = h->sw5_blocks_by_sw[sw];
      if (h->sw5_blocks_max == 0) h->sw5 = 0;
    }
  }
  if (c.pressure_scheme == DN_P_SPLIT_DCDM_ICPCG) {  // the direction history
    h->dcdm_keep = std::max(c.dcdm_max_stored_directions, std::max(c.dcdm_history_size, 1));
    A(dalloc(h, &h->dcdm_dirs, (size_t)h->dcdm_keep * h->n));
    A(dalloc(h, &h->dcdm_adirs, (size_t)h->dcdm_keep * h->n));
    if (s != DN_OK) return bad(s, "device allocation failed: " + h->err);
  }
  // the cluster form of the multigrid inner CG keeps its bottom levels in shared memory
  for (const void *k : {(const void *)k_mgcg_cluster<5>, (const void *)k_mgcg_cluster<13>})
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMgClusterSmemMax);
  // the preconditioner-only kernel (DCDM directions, the pressure analysis) may use shared memory as k_pcg does
  for (const void *k : {(const void *)k_prec_apply<3>, (const void *)k_prec_apply<4>}) {
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, k);
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, h->smem_optin - (int)fa.sharedSizeBytes);
  }
  if (c.precision == DN_PRECISION_MIXED) {
    A(dalloc(h, &h->fa5, 5 * h->n));
    A(dalloc(h, &h->fl5, 5 * h->n));
    for (float **p : {&h->fdinv5, &h->fb, &h->fx, &h->fr, &h->fz, &h->fy, &h->fp0, &h->fp1, &h->fap})
      A(dalloc(h, p, h->n));
    if (s != DN_OK) return bad(s, "device allocation failed: " + h->err);
    if (c.mixed_preconditioner == DN_MIXED_PREC_MULTIGRID) {
      A(mg_alloc(h, h->mgp, h->G.nx, h->G.ny, h->bc.p));
      if (h->mgp.levels() > 0) {  // level 0 is the FP32 pressure operator, its CG's vectors and residual fy
        h->mgp.lv[0].a64 = h->a5;
        h->mgp.lv[0].a = h->fa5;
        h->mgp.lv[0].r = h->fy;
      }
      h->mgp.singular = h->has_dirichlet ? 0 : 1;
      A(dalloc(h, &h->mg_scal, 16));
      A(dalloc(h, &h->mg_part, 3 * (size_t)kMgParts));
      // the CH solve: FP32 13-point operator, CG vectors and the (K + s I) hierarchy, when the operator has
      // its biharmonic part (cn > 0) and the grid coarsens
      const BCSide reflect[4] = {{DN_BC_NEUMANN, 0.0}, {DN_BC_NEUMANN, 0.0}, {DN_BC_NEUMANN, 0.0},
                                 {DN_BC_NEUMANN, 0.0}};
      if (c.cn > 0.0 && solve_ch(c)) {
        A(mg_alloc(h, h->mgc, h->G.nx, h->G.ny, reflect));
        if (h->mgc.levels() > 0) {
          double *a64 = nullptr;
          float *a32 = nullptr;
          A(dalloc(h, &a64, 5 * h->n));
          A(dalloc(h, &a32, 5 * h->n));
          A(dalloc(h, &h->mgc.lv[0].r, h->n));
          h->mgc.lv[0].a64 = h->mgc.lv[0].a64_own = a64;
          h->mgc.lv[0].a = a32;
          A(dalloc(h, &h->fa13, 13 * h->n));
          for (float **q : {&h->cx32, &h->cr32, &h->cz32, &h->cp32, &h->cq32, &h->ct32, &h->cb32})
            A(dalloc(h, q, h->n));
          h->ch_mg = true;
        }
      }
      if (s != DN_OK) return bad(s, "device allocation failed: " + h->err);
      A(mg_upload_chain(h, h->mgp));
      A(mg_upload_chain(h, h->mgc));
      if (s != DN_OK) return bad(s, "device allocation failed: " + h->err);
    }
    const int optin = h->smem_optin;
    auto round16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
    const bool px = c.periodic_x != 0;
    const bool stageable = !px || h->nsweep5 >= 2;
    const void *k53f = px ? (const void *)k_pcg<5, 4, float> : (const void *)k_pcg<5, 3, float>;
    h->sw5f_warp_smem[0] = round16(sweep_warp_smem(2, ny, 4, px));
    h->sw5f_warp_smem[1] = round16(sweep_warp_smem(4, ny, 4, px));
    const size_t per = h->sw5f_warp_smem[use_split(c) ? 0 : 1];
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, k53f);
    const size_t budget = (size_t)optin > 64 + fa.sharedSizeBytes ? (size_t)optin - 64 - fa.sharedSizeBytes : 0;
    int sw = stageable ? (int)std::min<size_t>(kSweepWarpsPerCta, budget / per) : 0;
    sw = std::min(sw, h->nsweep5);
    if (sw > 0 && c.sweep_warps_per_cta > 0) sw = std::min(sw, c.sweep_warps_per_cta);
    h->sw5f = stageable ? sw : 0;
    if (h->sw5f > 0) {
      const size_t dyn = 64 + (size_t)sw * per;
      cudaFuncSetAttribute(k53f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           std::max((int)dyn, optin - (int)fa.sharedSizeBytes));
      int occf = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occf, k53f, kBlock, dyn);
      h->sw5f_blocks_max = std::min(kMaxBlocks, std::max(0, occf) * h->num_sms);
      if (h->sw5f_blocks_max == 0) h->sw5f = 0;
    }
  }
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pcg<5, 0>, kBlock, 0);
  int occ2 = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, k_pcg<13, 1>, kBlock, 0);
  int occ3 = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ3, k_bicgstab, kBlock, 0);
  h->bicg_occ = std::max(1, occ3);
  occ = std::min(occ, std::min(occ2, occ3));
  if (c.precision == DN_PRECISION_MIXED) {
    int occ4 = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ4, k_pcg<5, 0, float>, kBlock, 0);
    occ = std::min(occ, occ4);
  }
  h->max_coop_blocks = std::min(kMaxBlocks, std::max(1, occ) * h->num_sms);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return bad(DN_ERR_CUDA, "initial synchronisation failed");
  *out = h;
  return DN_OK;
}

dn_status dn_destroy(dn_handle *h) {
  if (!h) return DN_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (const dn_handle::MgGraph &g : h->mg_graphs) cudaGraphExecDestroy(g.exec);
  for (dn_handle::SolveGraph &g : h->dc_graph)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (h->step_exec) cudaGraphExecDestroy(h->step_exec);
  if (h->cap_ev) cudaEventDestroy(h->cap_ev);
  if (h->batch.exec) cudaGraphExecDestroy(h->batch.exec);
  if (h->batch.fork) cudaEventDestroy(h->batch.fork);
  if (h->batch.stream) cudaStreamDestroy(h->batch.stream);
  for (void *p : h->allocations) cudaFree(p);
  if (h->mon) cudaFree(h->mon);
  if (h->host_scal) cudaFreeHost(h->host_scal);
  for (auto &e : h->ev)
    if (e) cudaEventDestroy(e);
  for (auto &e : h->kev)
    if (e) cudaEventDestroy(e);
  for (cudaStream_t cs : h->cap_streams)
    if (cs) cudaStreamDestroy(cs);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return DN_OK;
}

dn_status dn_initialize(dn_handle *h) {
  if (!h || !h->stream) return DN_ERR_INVALID_ARGUMENT;
  const dn_config &c = h->cfg;
  Fv *f = h->f;
  InitParams P{};
  P.mode = c.mode;
  P.phase_initializer = c.phase_initializer;
  P.velocity_profile = c.velocity_profile;
  P.invert_phase = c.invert_phase;
  P.cn = c.cn;
  P.lx = c.lx;
  P.ly = c.ly;
  P.cx = c.interface_center_x;
  P.cy = c.interface_center_y;
  P.radius = c.interface_radius;
  P.amplitude = c.interface_amplitude;
  P.wavenumber = c.interface_wavenumber;
  P.slot_w = c.zalesak_slot_width;
  P.slot_d = c.zalesak_slot_depth;
  P.advect_u = c.advect_u;
  P.advect_v = c.advect_v;
  P.rcx = c.rotation_center_x;
  P.rcy = c.rotation_center_y;
  P.omega = c.angular_velocity;
  P.ub = h->bc.u[DN_BOTTOM].value;
  P.ut = h->bc.u[DN_TOP].value;
  P.couette = !c.periodic_y && h->bc.u[DN_BOTTOM].type == DN_BC_DIRICHLET && h->bc.u[DN_TOP].type == DN_BC_DIRICHLET &&
              (std::fabs(P.ut) > 0.0 || std::fabs(P.ub) > 0.0);
  LAUNCH_INTERIOR(k_init_phase, f[DN_F_C], f[DN_F_C], h->G, P);
  k_init_u<<<blocks_for((long long)f[DN_F_U].size()), 256, 0, h->stream>>>(f[DN_F_U], h->G, P, 1);
  DN_TRY(check_launch(h, "k_init_u"));
  k_init_v<<<blocks_for((long long)f[DN_F_V].size()), 256, 0, h->stream>>>(f[DN_F_V], h->G, P);
  DN_TRY(check_launch(h, "k_init_v"));
  if (c.velocity_profile != 1) {
    DN_TRY(bc(h, f[DN_F_U], kBCU));
    DN_TRY(bc(h, f[DN_F_V], kBCV));
  }
  DN_TRY(bc(h, f[DN_F_C], kBCScalar));
  DN_TRY(copy_field(h, f[DN_F_C_PREV], f[DN_F_C]));
  DN_TRY(copy_field(h, f[DN_F_C_PREV2], f[DN_F_C]));
  DN_TRY(copy_field(h, f[DN_F_U_PREV], f[DN_F_U]));
  DN_TRY(copy_field(h, f[DN_F_V_PREV], f[DN_F_V]));
  DN_TRY(materials(h, f[DN_F_C], f[DN_F_RHO], f[DN_F_ETA]));
  DN_TRY(copy_field(h, f[DN_F_RHO_PREV], f[DN_F_RHO]));
  DN_TRY(copy_field(h, f[DN_F_ETA_PREV], f[DN_F_ETA]));
  DN_TRY(copy_field(h, f[DN_F_RHO_MID], f[DN_F_RHO]));
  DN_TRY(copy_field(h, f[DN_F_ETA_MID], f[DN_F_ETA]));
  DN_TRY(refresh_mu(h));
  DN_TRY(clear_surface_force(h));
  double m = 0.0;
  DN_TRY(dn_compute_mass(h, DN_F_C, &m));
  h->initial_mass = m;
  DN_TRY(fill_field(h, f[DN_F_P], 0.0));
  DN_TRY(bc(h, f[DN_F_P], kBCPressure));
  DN_TRY(copy_field(h, f[DN_F_P_PREV], f[DN_F_P]));
  DN_TRY(fill_field(h, f[DN_F_E_PREV], 0.0));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  return DN_OK;
}

dn_status dn_set_field(dn_handle *h, int field, const double *host, size_t count) {
  if (!h || !host || field < 0 || field >= DN_F_COUNT) return DN_ERR_INVALID_ARGUMENT;
  if (count != h->f[field].size()) return fail(h, DN_ERR_INVALID_ARGUMENT, "field size mismatch");
  DN_CUDA(h, cudaMemcpyAsync(h->f[field].d, host, count * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  return DN_OK;
}

dn_status dn_get_field(dn_handle *h, int field, double *host, size_t count) {
  if (!h || !host || field < 0 || field >= DN_F_COUNT) return DN_ERR_INVALID_ARGUMENT;
  if (count != h->f[field].size()) return fail(h, DN_ERR_INVALID_ARGUMENT, "field size mismatch");
  DN_CUDA(h, cudaMemcpyAsync(host, h->f[field].d, count * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  return DN_OK;
}

dn_status dn_field_device_ptr(dn_handle *h, int field, double **dev_ptr, size_t *count) {
  if (!h || field < 0 || field >= DN_F_COUNT) return DN_ERR_INVALID_ARGUMENT;
  if (dev_ptr) *dev_ptr = h->f[field].d;
  if (count) *count = h->f[field].size();
  return DN_OK;
}

void dn_set_initial_mass(dn_handle *h, double mass) {
  if (h) h->initial_mass = mass;
}

dn_status dn_refresh_derived(dn_handle *h) {
  if (!h) return DN_ERR_INVALID_ARGUMENT;
  Fv *f = h->f;
  DN_TRY(bc(h, f[DN_F_C], kBCScalar));
  DN_TRY(bc(h, f[DN_F_C_PREV], kBCScalar));
  DN_TRY(bc(h, f[DN_F_C_PREV2], kBCScalar));
  DN_TRY(bc(h, f[DN_F_P], kBCPressure));
  DN_TRY(bc(h, f[DN_F_P_PREV], kBCPressure));
  DN_TRY(bc(h, f[DN_F_U], kBCU));
  DN_TRY(bc(h, f[DN_F_V], kBCV));
  DN_TRY(bc(h, f[DN_F_U_PREV], kBCU));
  DN_TRY(bc(h, f[DN_F_V_PREV], kBCV));
  DN_TRY(materials(h, f[DN_F_C], f[DN_F_RHO], f[DN_F_ETA]));
  DN_TRY(materials(h, f[DN_F_C_PREV], f[DN_F_RHO_PREV], f[DN_F_ETA_PREV]));
  DN_TRY(midpoint(h));
  DN_TRY(refresh_mu(h));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  return DN_OK;
}

// ---- restart snapshot v2 (Solver::write_restart_snapshot / load_restart_snapshot, io.cpp:271-437) ----
// Native-endian binary: the magic string, version 2, step, initial mass, mode string, grid and physics
// scalars, periodicity, the 12 configured boundary specs, then 12 Field2D arrays with their extents.
namespace {
constexpr char kRestartMagic[] = "ding_nsch_restart_v1";
const int kRestartFields[12] = {DN_F_C,      DN_F_C_PREV, DN_F_C_PREV2, DN_F_P,      DN_F_P_PREV,  DN_F_U,
                                DN_F_V,      DN_F_U_PREV, DN_F_V_PREV,  DN_F_E_PREV, DN_F_HU_PREV, DN_F_HV_PREV};

const char *mode_name(int m) {
  return m == DN_MODE_SINGLE_PHASE ? "single_phase" : (m == DN_MODE_ADVECTION_ONLY ? "advection_only" : "coupled");
}
bool restart_nearly_equal(double a, double b) {  // io.cpp:86-89
  const double scale = std::max({1.0, std::fabs(a), std::fabs(b)});
  return std::fabs(a - b) <= 1.0e-12 * scale;
}
const double *restart_scalars(const dn_config &c, double (&v)[13]) {
  const double t[13] = {c.dt, c.lx, c.ly, c.re, c.ca, c.pe, c.cn, c.density_ratio, c.viscosity_ratio,
                        c.body_force_x, c.body_force_y, c.top_wall_velocity_x, c.bottom_wall_velocity_x};
  std::copy(t, t + 13, v);
  return v;
}
const char *const kRestartScalarNames[13] = {"dt", "lx", "ly", "re", "ca", "pe", "cn", "density_ratio",
                                             "viscosity_ratio", "body_force_x", "body_force_y",
                                             "top_wall_velocity_x", "bottom_wall_velocity_x"};
}  // namespace

dn_status dn_write_restart(dn_handle *h, int step, const char *path) {
  if (!h || !path) return DN_ERR_INVALID_ARGUMENT;
  const dn_config &c = h->cfg;
  DN_CUDA(h, cudaStreamSynchronize(h->stream));  // the state of every launched step
  const std::string tmp = std::string(path) + ".tmp";
  std::FILE *fp = std::fopen(tmp.c_str(), "wb");
  if (!fp) return fail(h, DN_ERR_INVALID_ARGUMENT, "cannot open restart snapshot for writing");
  bool ok = true;
  auto wr = [&](const void *p, size_t n) { ok = ok && std::fwrite(p, 1, n, fp) == n; };
  auto ws = [&](const std::string &v) {
    const std::uint64_t n = v.size();
    wr(&n, sizeof n);
    wr(v.data(), v.size());
  };
  ws(kRestartMagic);
  const std::uint32_t version = 2;
  wr(&version, sizeof version);
  wr(&step, sizeof step);
  wr(&h->initial_mass, sizeof(double));
  ws(mode_name(c.mode));
  wr(&c.nx, sizeof(int));
  wr(&c.ny, sizeof(int));
  wr(&c.ghost, sizeof(int));
  double sc[13];
  wr(restart_scalars(c, sc), sizeof sc);
  const int px = c.periodic_x != 0, py = c.periodic_y != 0;
  wr(&px, sizeof px);
  wr(&py, sizeof py);
  for (const dn_bc *set : {c.p_bc, c.u_bc, c.v_bc})
    for (int sd = 0; sd < 4; ++sd) {
      wr(&set[sd].type, sizeof(int));
      wr(&set[sd].value, sizeof(double));
    }
  std::vector<double> buf;
  for (int id : kRestartFields) {
    const Fv &f = h->f[id];
    const std::uint64_t size = f.size();
    wr(&f.nx, sizeof(int));
    wr(&f.ny, sizeof(int));
    wr(&f.g, sizeof(int));
    wr(&size, sizeof size);
    buf.resize(size);
    if (cudaMemcpyAsync(buf.data(), f.d, size * sizeof(double), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
      ok = false;
    wr(buf.data(), size * sizeof(double));
  }
  ok = (std::fflush(fp) == 0) && ok;
  ok = (std::fclose(fp) == 0) && ok;
  if (!ok) {
    std::remove(tmp.c_str());
    return fail(h, DN_ERR_INVALID_ARGUMENT, "failed to write restart snapshot");
  }
  if (std::rename(tmp.c_str(), path) != 0) return fail(h, DN_ERR_INVALID_ARGUMENT, "failed to rename restart snapshot");
  return DN_OK;
}

dn_status dn_load_restart(dn_handle *h, const char *path, int *step) {
  if (!h || !path) return DN_ERR_INVALID_ARGUMENT;
  const dn_config &c = h->cfg;
  std::FILE *fp = std::fopen(path, "rb");
  if (!fp) return fail(h, DN_ERR_INVALID_ARGUMENT, std::string("cannot open restart snapshot: ") + path);
  std::vector<double> buf;
  auto body = [&]() -> dn_status {
    bool ok = true;
    auto rd = [&](void *p, size_t n) { ok = ok && std::fread(p, 1, n, fp) == n; };
    auto rs = [&](std::string &v) {
      std::uint64_t n = 0;
      rd(&n, sizeof n);
      if (!ok || n > 4096) {
        ok = false;
        return;
      }
      v.assign((size_t)n, '\0');
      rd(&v[0], (size_t)n);
    };
    auto incompatible = [&](const std::string &what) {
      return fail(h, DN_ERR_CONFIG, "restart snapshot incompatible with config: " + what);
    };
    std::string magic, mode;
    rs(magic);
    if (!ok) return fail(h, DN_ERR_CONFIG, "failed to read restart snapshot string");
    if (magic != kRestartMagic) return incompatible("unrecognized restart file");
    std::uint32_t version = 0;
    int rstep = 0;
    double mass = 0.0;
    rd(&version, sizeof version);
    if (!ok || (version != 1u && version != 2u)) return incompatible("unsupported restart file version");
    rd(&rstep, sizeof rstep);
    rd(&mass, sizeof mass);
    rs(mode);
    if (!ok) return fail(h, DN_ERR_CONFIG, "failed to read restart snapshot");
    if (mode != mode_name(c.mode)) return incompatible("mode");
    int iv[3];
    rd(iv, sizeof iv);
    if (!ok) return fail(h, DN_ERR_CONFIG, "failed to read restart snapshot");
    if (iv[0] != c.nx) return incompatible("nx");
    if (iv[1] != c.ny) return incompatible("ny");
    if (iv[2] != c.ghost) return incompatible("ghost");
    double sc[13], mine[13];
    rd(sc, sizeof sc);
    if (!ok) return fail(h, DN_ERR_CONFIG, "failed to read restart snapshot");
    restart_scalars(c, mine);
    for (int k = 0; k < 13; ++k)
      if (!restart_nearly_equal(sc[k], mine[k])) return incompatible(kRestartScalarNames[k]);
    int per[2];
    rd(per, sizeof per);
    if (!ok) return fail(h, DN_ERR_CONFIG, "failed to read restart snapshot");
    if (per[0] != (c.periodic_x != 0)) return incompatible("periodic_x");
    if (per[1] != (c.periodic_y != 0)) return incompatible("periodic_y");
    if (version >= 2u) {
      static const char *sides[4] = {"left", "right", "bottom", "top"};
      const char *kinds[3] = {"pressure", "u", "v"};
      const dn_bc *sets[3] = {c.p_bc, c.u_bc, c.v_bc};
      for (int k = 0; k < 3; ++k)
        for (int sd = 0; sd < 4; ++sd) {
          int type = 0;
          double value = 0.0;
          rd(&type, sizeof type);
          rd(&value, sizeof value);
          if (!ok) return fail(h, DN_ERR_CONFIG, "failed to read restart snapshot");
          const std::string name = std::string(kinds[k]) + "_bc_" + sides[sd];
          if (type != sets[k][sd].type) return incompatible(name + "_type");
          if (!restart_nearly_equal(value, sets[k][sd].value)) return incompatible(name + "_value");
        }
    }
    for (int id : kRestartFields) {
      const Fv &f = h->f[id];
      int ext[3];
      std::uint64_t size = 0;
      rd(ext, sizeof ext);
      rd(&size, sizeof size);
      if (!ok) return fail(h, DN_ERR_CONFIG, "failed to read restart snapshot field");
      if (ext[0] != f.nx || ext[1] != f.ny || ext[2] != f.g || size != f.size())
        return fail(h, DN_ERR_CONFIG, "restart snapshot field size mismatch");
      buf.resize(size);
      rd(buf.data(), size * sizeof(double));
      if (!ok) return fail(h, DN_ERR_CONFIG, "failed to read restart snapshot field");
      DN_CUDA(h, cudaMemcpyAsync(f.d, buf.data(), size * sizeof(double), cudaMemcpyHostToDevice, h->stream));
      DN_CUDA(h, cudaStreamSynchronize(h->stream));  // buf is reused by the next field
    }
    h->initial_mass = mass;
    if (step) *step = rstep;
    return DN_OK;
  };
  const dn_status st = body();
  std::fclose(fp);
  if (st != DN_OK) return st;
  // the restart's rebuild (io.cpp:412-436): BC ghosts, materials n and n-1, midpoint, mu; cleared work fields
  DN_TRY(dn_refresh_derived(h));
  for (int id : {DN_F_P_CORR, DN_F_U_STAR, DN_F_V_STAR, DN_F_SFX_CELL, DN_F_SFY_CELL, DN_F_SFX_U, DN_F_SFY_V})
    DN_TRY(fill_field(h, h->f[id], 0.0));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  return DN_OK;
}

dn_status dn_pressure_analysis(dn_handle *h, int step, const char *source_mode) {
  if (!h || !source_mode || step < 0) return DN_ERR_INVALID_ARGUMENT;
  return pressure_analysis(h, step, source_mode);
}

// Launch-shape autotuner of the pressure PCG: times one pressure solve of the handle's current state (its
// u*, v*, rho_mid, p, p_prev, as a step leaves them) for each candidate (rows per CTA of the SpMV / update
// phases x sweep warps per CTA of the staged wavefront) and keeps the fastest on the handle.
dn_status dn_autotune_pressure(dn_handle *h, int *rows_per_cta, int *sweep_warps_per_cta, double *best_ms) {
  if (!h) return DN_ERR_INVALID_ARGUMENT;
  if (h->cfg.pressure_scheme == DN_P_JACOBI || h->cfg.pressure_scheme == DN_P_SPLIT_DCDM_ICPCG)
    return fail(h, DN_ERR_UNSUPPORTED, "the launch-shape autotuner covers the PCG pressure schemes");
  const long long rows_c[] = {256, 512, 1024, 2048, 4096};
  // sweep-warp counts whose wavefront CTAs are co-resident; the FP64 staged path only (the mixed form's
  // FP32 wavefront keeps its own)
  std::vector<int> sws;
  if (h->sw5 > 0 && h->cfg.precision != DN_PRECISION_MIXED) {
    for (int w = 1; w <= h->sw5_budget; ++w)
      if ((h->nsweep5 + w - 1) / w <= h->sw5_blocks_by_sw[w]) sws.push_back(w);
  } else {
    sws.push_back(h->sw5);
  }
  const long long rows0 = h->rows_per_cta;
  const int sw0 = h->sw5;
  long long best_rows = rows0;
  int best_sw = sw0;
  double best = INFINITY;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  dn_status st = DN_OK;
  for (int pass = 0; pass < 2 && st == DN_OK; ++pass)  // the first pass also warms up each shape
    for (long long rows : rows_c)
      for (int sw : sws) {
        h->rows_per_cta = rows;
        h->sw5 = sw;
        ++h->graph_epoch;  // recorded solves hold launch shapes
        dn_report rep{};
        cudaEventRecord(e0, h->stream);
        st = pressure(h, h->step, &rep);
        cudaEventRecord(e1, h->stream);
        if (st != DN_OK) break;
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (pass == 1 && ms < best) {
          best = ms;
          best_rows = rows;
          best_sw = sw;
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  h->rows_per_cta = st == DN_OK ? best_rows : rows0;
  h->sw5 = st == DN_OK ? best_sw : sw0;
  ++h->graph_epoch;
  if (st != DN_OK) return st;
  if (rows_per_cta) *rows_per_cta = (int)best_rows;
  if (sweep_warps_per_cta) *sweep_warps_per_cta = best_sw;
  if (best_ms) *best_ms = best;
  return DN_OK;
}

// ---- CG monitor (the per-iteration record of the reference's CGMonitor, ch_sparse_krylov.hpp:515-660, as the
// pressure analysis hook reads it, pressure_analysis.cpp:156-328) ----
dn_status dn_set_pressure_monitor(dn_handle *h, int capacity) {
  if (!h || capacity < 0) return DN_ERR_INVALID_ARGUMENT;
  if (h->mon) {
    cudaFree(h->mon);
    h->mon = nullptr;
  }
  h->mon_cap = 0;
  h->mon_count = 0;
  if (capacity > 0) {
    DN_CUDA(h, cudaMalloc(&h->mon, (size_t)capacity * 4 * sizeof(double)));
    h->mon_cap = capacity;
  }
  return DN_OK;
}

dn_status dn_pressure_monitor(dn_handle *h, double *out, int capacity, int *count) {
  if (!h || (capacity > 0 && !out)) return DN_ERR_INVALID_ARGUMENT;
  const int m = std::min(capacity, h->mon_count);
  if (m > 0) {
    if (h->cfg.pressure_scheme == DN_P_SPLIT_DCDM_ICPCG) {
      std::memcpy(out, h->mon_host.data(), (size_t)m * 4 * sizeof(double));
    } else {
      DN_CUDA(h, cudaMemcpyAsync(out, h->mon, (size_t)m * 4 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
      DN_CUDA(h, cudaStreamSynchronize(h->stream));
    }
  }
  if (count) *count = h->mon_count;
  return DN_OK;
}

// ---- history.csv (Solver::write_history_csv_header / append_history_csv_entry, io.cpp:179-206) ----
namespace {
const char kHistoryHeader[] =
    "step,time,mass,mass_drift,divergence_l2,max_divergence,max_abs_mu,max_velocity,kinetic_energy,"
    "total_free_energy,ch_inner_residual,ch_equation_residual,coupling_residual,pressure_correction_residual,"
    "momentum_residual,boundary_speed_pre_correction,boundary_speed_post_correction,rho_min,rho_max,eta_min,"
    "eta_max,dt_limit_advective,dt_limit_capillary,dt_limit_ch_explicit,dt_limit_active,dt_limit_ratio,"
    "ch_iterations,coupling_iterations,pressure_iterations,momentum_iterations,"
    "ch_solver_name,momentum_solver_name,pressure_solver_name,dt_limit_source\n";

const char *pressure_solver_label(int scheme) {  // pressure.cpp:1031-1071
  switch (scheme) {
  case DN_P_SPLIT_ICPCG: return "SplitICCPCG";
  case DN_P_SPLIT_DCDM_ICPCG: return "SplitDCDMICC";
  case DN_P_SPLIT_ILDLT_PCG: return "SplitILDLTPCG";
  case DN_P_ICPCG: return "ICCPCG";
  case DN_P_ILDLT_PCG: return "ILDLTPCG";
  default: return "Jacobi";
  }
}
const char *ch_solver_label(const dn_config &c, int prec) {  // phase_field.cpp:20-28, 277, 464-470; solver.cpp:244
  if (c.mode == DN_MODE_ADVECTION_ONLY) return "PureAdvectionSSPRK3[WENO5]";
  switch (prec) {
  case 1: return "SparsePCG[ILDLT]";
  case 0: return "SparsePCG[Diagonal]";
  case 2: return "SparsePCG[DiagonalFallback]";
  default: return "NotUsed";
  }
}
}  // namespace

size_t dn_history_csv_header(char *buf, size_t len) {
  const size_t n = sizeof(kHistoryHeader) - 1;
  if (buf && len > 0) {
    const size_t m = std::min(n, len - 1);
    std::memcpy(buf, kHistoryHeader, m);
    buf[m] = '\0';
  }
  return n;
}

dn_status dn_history_csv_row(dn_handle *h, int step, double time, const dn_report *rep, char *buf, size_t len,
                             size_t *written) {
  if (!h || !rep || !buf || len == 0) return DN_ERR_INVALID_ARGUMENT;
  dn_diag d{};
  DN_TRY(dn_diagnostics(h, &d));
  const dn_config &c = h->cfg;
  const bool adv = c.mode == DN_MODE_ADVECTION_ONLY;
  // populate_timestep_limits, diagnostics.cpp:96-110
  const char *source = "advective";
  double active = d.dt_limit_advective;
  if (d.dt_limit_capillary < active) {
    active = d.dt_limit_capillary;
    source = "capillary";
  }
  if (d.dt_limit_ch_explicit < active) {
    active = d.dt_limit_ch_explicit;
    source = "ch_explicit";
  }
  if (!std::isfinite(active) || active <= 1.0e-30) source = "unbounded";
  const int n = std::snprintf(
      buf, len,
      "%d,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,"
      "%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%d,%d,%d,%d,%s,%s,%s,%s\n",
      step, time, d.mass, d.mass_drift, d.divergence_l2, d.max_divergence, d.max_abs_mu, d.max_velocity,
      d.kinetic_energy, d.total_free_energy, rep->ch_residual, adv ? 0.0 : rep->ch_equation_residual, 0.0,
      adv ? 0.0 : rep->pressure_residual, adv ? 0.0 : rep->momentum_residual, rep->boundary_speed_pre,
      rep->boundary_speed_post, d.rho_min, d.rho_max, d.eta_min, d.eta_max, d.dt_limit_advective,
      d.dt_limit_capillary, d.dt_limit_ch_explicit, d.dt_limit_active, d.dt_limit_ratio, rep->ch_iterations,
      rep->coupling_iterations, rep->pressure_iterations, rep->momentum_iterations,
      ch_solver_label(c, rep->ch_preconditioner),
      adv ? "NotUsed" : "ExplicitConvection+MonolithicImplicitViscosityBiCGSTAB[Diagonal]",
      adv ? "NotUsed" : pressure_solver_label(c.pressure_scheme), source);
  if (n < 0) return fail(h, DN_ERR_INVALID_ARGUMENT, "history row formatting failed");
  if (written) *written = (size_t)n;
  if ((size_t)n >= len) return fail(h, DN_ERR_INVALID_ARGUMENT, "history row buffer too small");
  return DN_OK;
}

dn_status dn_begin_step(dn_handle *h, int step) {
  if (!h) return DN_ERR_INVALID_ARGUMENT;
  h->step = step;
  return begin_step(h);
}

dn_status dn_phase(dn_handle *h, int step, dn_report *rep) {
  if (!h || !rep) return DN_ERR_INVALID_ARGUMENT;
  return phase(h, step, rep);
}

dn_status dn_momentum(dn_handle *h, int step, dn_report *rep) {
  if (!h || !rep) return DN_ERR_INVALID_ARGUMENT;
  return momentum(h, step, rep);
}

dn_status dn_pressure(dn_handle *h, dn_report *rep) {
  if (!h || !rep) return DN_ERR_INVALID_ARGUMENT;
  return pressure(h, h->step, rep);
}

dn_status dn_correct(dn_handle *h, dn_report *rep) {
  if (!h || !rep) return DN_ERR_INVALID_ARGUMENT;
  return correct(h, h->step, rep);
}

dn_status dn_step(dn_handle *h, int step, dn_report *rep) {
  if (!h) return DN_ERR_INVALID_ARGUMENT;
  dn_report local;
  if (!rep) rep = &local;
  if (step_capturable(h, step)) return graph_step(h, step, rep);
  std::memset(rep, 0, sizeof(*rep));
  rep->ch_preconditioner = -1;
  h->step = step;
  for (int k = 4; k < 8; ++k) h->phase_ms[k] = 0.0;
  cudaEventRecord(h->ev[0], h->stream);
  DN_TRY(begin_step(h));
  if (h->cfg.mode == DN_MODE_ADVECTION_ONLY) {
    DN_TRY(advection_step(h, rep));
    for (int k = 0; k < 4; ++k) h->phase_ms[k] = 0.0;
    return dn_diagnostics(h, &h->last_diag);  // solver.cpp:252 and the run loop's abort (solver.cpp:355-364)
  }
  DN_TRY(phase(h, step, rep));
  cudaEventRecord(h->ev[1], h->stream);
  DN_TRY(momentum(h, step, rep));
  cudaEventRecord(h->ev[2], h->stream);
  // the pressure analysis at its trigger step: frozen before the solve (solver.cpp:270), online after it
  // for the PCG schemes (pressure.cpp:1078-1087)
  const dn_config &c = h->cfg;
  const bool analyse = c.analysis_enabled && step + 1 == c.analysis_trigger_step;
  if (analyse && (c.analysis_mode == DN_ANALYSIS_FROZEN || c.analysis_mode == DN_ANALYSIS_BOTH))
    DN_TRY(pressure_analysis(h, step, "frozen"));
  DN_TRY(pressure(h, step, rep));
  if (analyse && (c.analysis_mode == DN_ANALYSIS_ONLINE || c.analysis_mode == DN_ANALYSIS_BOTH) &&
      c.pressure_scheme != DN_P_JACOBI)
    DN_TRY(pressure_analysis(h, step, "online"));
  cudaEventRecord(h->ev[3], h->stream);
  DN_TRY(correct(h, step, rep));
  cudaEventRecord(h->ev[4], h->stream);
  DN_CUDA(h, cudaEventSynchronize(h->ev[4]));
  for (int k = 0; k < 4; ++k) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, h->ev[k], h->ev[k + 1]);
    h->phase_ms[k] = ms;
  }
  // the step ends with compute_diagnostics (solver.cpp:276); the reference's run loop aborts on a
  // non-finite one (solver.cpp:355-364), which here is the step's status DN_ERR_NONFINITE
  const dn_status ds = dn_diagnostics(h, &h->last_diag);
  if (ds == DN_OK && step >= 1) h->steady = true;  // every operator, factor and hierarchy of a step >= 1 exists
  return ds;
}

dn_status dn_set_step_graph(dn_handle *h, int enable) {
  if (!h) return DN_ERR_INVALID_ARGUMENT;
  h->graph_steps = enable != 0;
  return DN_OK;
}

dn_status dn_last_diagnostics(dn_handle *h, dn_diag *d) {
  if (!h || !d) return DN_ERR_INVALID_ARGUMENT;
  *d = h->last_diag;
  return DN_OK;
}

// Batched ensemble: one step of each handle, the handles advanced concurrently.  Each handle's kernels run
// on its own stream from a host worker of its own, so the GPU overlaps the instances: a single instance's
// wavefront keeps only a few warps busy, many instances fill the device.  Every handle computes exactly
// what dn_step computes for it alone.
dn_status dn_step_batch(dn_handle *const *handles, int count, const int *steps, dn_report *reports) {
  if (!handles || count < 0) return DN_ERR_INVALID_ARGUMENT;
  for (int a = 0; a < count; ++a) {
    if (!handles[a]) return DN_ERR_INVALID_ARGUMENT;
    for (int b2 = 0; b2 < a; ++b2)
      if (handles[b2] == handles[a]) return DN_ERR_INVALID_ARGUMENT;  // one handle twice would race with itself
  }
  // every handle replays captured steps and the step allows it: the whole batch is one graph launch
  bool one_graph = count > 0 && steps != nullptr;
  for (int a = 0; one_graph && a < count; ++a)
    one_graph = step_capturable(handles[a], steps[a]) && handles[a]->device == handles[0]->device;
  if (one_graph) {
    if (cudaSetDevice(handles[0]->device) != cudaSuccess) return fail(handles[0], DN_ERR_CUDA, "cudaSetDevice failed");
    return batch_graph_step(handles, count, steps, reports);
  }
  std::vector<dn_status> st;
  try {
    st.assign((size_t)count, DN_OK);
  } catch (...) {
    return DN_ERR_INVALID_ARGUMENT;
  }
  std::atomic<int> next{0};
  auto worker = [&]() {
    for (int a = next.fetch_add(1); a < count; a = next.fetch_add(1)) {
      dn_handle *h = handles[a];
      if (cudaSetDevice(h->device) != cudaSuccess) {
        st[(size_t)a] = fail(h, DN_ERR_CUDA, "cudaSetDevice failed");
        continue;
      }
      st[(size_t)a] = dn_step(h, steps ? steps[a] : 0, reports ? &reports[a] : nullptr);
    }
  };
  const int nworkers = std::min(count, 64);
  std::vector<std::thread> pool;
  try {
    pool.reserve((size_t)std::max(0, nworkers - 1));
    for (int w = 1; w < nworkers; ++w) pool.emplace_back(worker);
  } catch (...) {
    // no more threads: the ones started and this thread share the remaining handles
  }
  if (nworkers > 0) worker();
  for (auto &t : pool) t.join();
  for (int a = 0; a < count; ++a)
    if (st[(size_t)a] != DN_OK) return st[(size_t)a];
  return DN_OK;
}

dn_status dn_ch_linear_solve(dn_handle *h, const double *rhs_field, double alpha0, double *c_state,
                             double *iterate_residual, double *equation_residual, int *iterations) {
  if (!h || !rhs_field || !c_state) return DN_ERR_INVALID_ARGUMENT;
  // stage rhs and c_state through the work fields (cell-field layout)
  const size_t cnt = h->E_new.size();
  DN_CUDA(h, cudaMemcpyAsync(h->E_new.d, rhs_field, cnt * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  DN_CUDA(h, cudaMemcpyAsync(h->cmid.d, c_state, cnt * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  LAUNCH_INTERIOR(k_gather_compact, h->E_new, h->E_new, h->b);
  LAUNCH_INTERIOR(k_gather_compact, h->cmid, h->cmid, h->x);
  dn_report rep{};
  double it = 0.0, eq = 0.0;
  DN_TRY(ch_linear_solve(h, alpha0, &rep, &it, &eq));
  LAUNCH_INTERIOR(k_scatter_compact, h->cmid, h->x, h->cmid);
  DN_TRY(bc(h, h->cmid, kBCScalar));
  DN_CUDA(h, cudaMemcpyAsync(c_state, h->cmid.d, cnt * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  if (iterate_residual) *iterate_residual = it;
  if (equation_residual) *equation_residual = eq;
  if (iterations) *iterations = rep.ch_iterations;
  return DN_OK;
}

dn_status dn_pressure_solve(dn_handle *h, int step, const double *u_star, const double *v_star, const double *rho_mid,
                            const double *p, const double *p_prev, double *p_corr, int *iterations,
                            double *relative_residual) {
  if (!h || !u_star || !v_star || !rho_mid || !p || !p_prev || !p_corr) return DN_ERR_INVALID_ARGUMENT;
  Fv *f = h->f;
  auto up = [&](int id, const double *src) -> dn_status {
    DN_CUDA(h, cudaMemcpyAsync(f[id].d, src, f[id].size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    return DN_OK;
  };
  DN_TRY(up(DN_F_U_STAR, u_star));
  DN_TRY(up(DN_F_V_STAR, v_star));
  DN_TRY(up(DN_F_RHO_MID, rho_mid));
  DN_TRY(up(DN_F_P, p));
  DN_TRY(up(DN_F_P_PREV, p_prev));
  dn_report rep{};
  DN_TRY(pressure(h, step, &rep));
  DN_CUDA(h, cudaMemcpyAsync(p_corr, f[DN_F_P_CORR].d, f[DN_F_P_CORR].size() * sizeof(double), cudaMemcpyDeviceToHost,
                             h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  if (iterations) *iterations = rep.pressure_iterations;
  if (relative_residual) *relative_residual = rep.pressure_residual;
  return DN_OK;
}

// The projection on caller device buffers: u*, v*, p, p_prev in, u, v, p_new, p_prev_new out (Field2D
// layouts of the handle's u, v and cell fields).  It runs the step's own pressure solve and correction on
// the handle's fields, with the handle's rho_mid.
dn_status dn_projection(dn_handle *h, int step, const double *u_star, const double *v_star, const double *p,
                        const double *p_prev, double *u, double *v, double *p_new, double *p_prev_new, int *iterations,
                        double *relative_residual) {
  if (!h || !u_star || !v_star || !p || !p_prev || !u || !v || !p_new || !p_prev_new) return DN_ERR_INVALID_ARGUMENT;
  Fv *f = h->f;
  auto d2d = [&](double *dst, const double *src, int id) -> dn_status {
    DN_CUDA(h, cudaMemcpyAsync(dst, src, f[id].size() * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    return DN_OK;
  };
  DN_TRY(d2d(f[DN_F_U_STAR].d, u_star, DN_F_U_STAR));
  DN_TRY(d2d(f[DN_F_V_STAR].d, v_star, DN_F_V_STAR));
  DN_TRY(d2d(f[DN_F_P].d, p, DN_F_P));
  DN_TRY(d2d(f[DN_F_P_PREV].d, p_prev, DN_F_P_PREV));
  dn_report rep{};
  DN_TRY(pressure(h, step, &rep));
  DN_TRY(correct(h, step, &rep));
  DN_TRY(d2d(u, f[DN_F_U].d, DN_F_U));
  DN_TRY(d2d(v, f[DN_F_V].d, DN_F_V));
  DN_TRY(d2d(p_new, f[DN_F_P].d, DN_F_P));
  DN_TRY(d2d(p_prev_new, f[DN_F_P_PREV].d, DN_F_P_PREV));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  if (iterations) *iterations = rep.pressure_iterations;
  if (relative_residual) *relative_residual = rep.pressure_residual;
  return DN_OK;
}

// Transpose of dn_projection's linear part (rho_mid fixed): cotangents of the interior values of u, v,
// p_new, p_prev_new in; cotangents of the interior values of u*, v*, p, p_prev out (ghosts zero).
// With arho: also the cotangent of rho_mid (k_proj_rho_adj), for which the forward's p, p_prev and p_new are
// needed (p_new is p_corr less its mean, which no rho_mid term sees).
dn_status projection_adjoint(dn_handle *h, int step, const double *gu, const double *gv, const double *gp,
                             const double *gpp, double *au, double *av, double *ap, double *app, const double *p,
                             const double *p_prev, const double *p_new, double *arho, int *iterations,
                             double *relative_residual) {
  const dn_config &cfg = h->cfg;
  if (cfg.pressure_scheme == DN_P_JACOBI)
    return fail(h, DN_ERR_UNSUPPORTED, "pressure_scheme jacobi is not implemented by the CUDA backend");
  Fv *f = h->f;
  const Fv &U = f[DN_F_U], &V = f[DN_F_V], &P = f[DN_F_P];
  const Fv GU{const_cast<double *>(gu), U.nx, U.ny, U.g}, GV{const_cast<double *>(gv), V.nx, V.ny, V.g};
  const Fv GP{const_cast<double *>(gp), P.nx, P.ny, P.g}, GPP{const_cast<double *>(gpp), P.nx, P.ny, P.g};
  const Fv AU{au, U.nx, U.ny, U.g}, AV{av, V.nx, V.ny, V.g}, AP{ap, P.nx, P.ny, P.g}, APP{app, P.nx, P.ny, P.g};
  DN_CUDA(h, cudaMemsetAsync(au, 0, U.size() * sizeof(double), h->stream));
  DN_CUDA(h, cudaMemsetAsync(av, 0, V.size() * sizeof(double), h->stream));
  DN_CUDA(h, cudaMemsetAsync(ap, 0, P.size() * sizeof(double), h->stream));
  DN_CUDA(h, cudaMemsetAsync(app, 0, P.size() * sizeof(double), h->stream));
  const bool split = use_split(cfg);
  const bool icc = cfg.pressure_scheme == DN_P_ICPCG || cfg.pressure_scheme == DN_P_SPLIT_ICPCG ||
                   cfg.pressure_scheme == DN_P_SPLIT_DCDM_ICPCG;
  const double rho_ref = split ? rho_ref_of(cfg) : 1.0;
  // face cotangents through the BCs; u* and v* take them unchanged (u = u* - ...)
  LAUNCH_INTERIOR(k_adj_fold_u, AU, GU, AU, h->G, h->bc);
  LAUNCH_INTERIOR(k_adj_fold_v, AV, GV, AV, h->G, h->bc);
  // the operator of the current rho_mid, assembled as the forward assembles it (its right-hand side is
  // replaced below)
  k_p_assemble<<<blocks_for(h->n), 256, 0, h->stream>>>(h->G, h->bc, f[DN_F_RHO_MID], f[DN_F_U_STAR], f[DN_F_V_STAR],
                                                       h->pe, split ? 1 : 0, rho_ref, cfg.dt, h->a5, h->b);
  DN_TRY(check_launch(h, "k_p_assemble"));
  k_adj_cells_pre<<<blocks_for(h->n), 256, 0, h->stream>>>(AU, AV, GP, f[DN_F_RHO_MID], h->G, split ? 1 : 0, rho_ref,
                                                           cfg.dt, h->b, APP);
  DN_TRY(check_launch(h, "k_adj_cells_pre"));
  // p_corr and the right-hand side are both mean-free without a Dirichlet side: project before and after
  if (!h->has_dirichlet) DN_TRY(compact_subtract_mean(h, h->b));
  dn_report rep{};
  DN_TRY(pressure_factor_solve(h, split, icc, &rep));
  if (!h->has_dirichlet) DN_TRY(compact_subtract_mean(h, h->x));
  const double kappa = (split ? rho_ref : 1.0) / cfg.dt;
  LAUNCH_INTERIOR(k_adj_div_u, AU, AU, h->x, h->G, kappa);
  LAUNCH_INTERIOR(k_adj_div_v, AV, AV, h->x, h->G, kappa);
  k_adj_cells_post<<<blocks_for(h->n), 256, 0, h->stream>>>(h->x, GPP, f[DN_F_RHO_MID], h->G, split ? 1 : 0, rho_ref,
                                                            step, AP, APP);
  DN_TRY(check_launch(h, "k_adj_cells_post"));
  if (arho) {
    const Fv AR{arho, P.nx, P.ny, P.g};
    DN_CUDA(h, cudaMemsetAsync(arho, 0, P.size() * sizeof(double), h->stream));
    const size_t pb = P.size() * sizeof(double);
    DN_CUDA(h, cudaMemcpyAsync(h->bih.d, p_new, pb, cudaMemcpyDeviceToDevice, h->stream));
    DN_TRY(bc(h, h->bih, kBCPressure));
    if (split) {
      DN_CUDA(h, cudaMemcpyAsync(f[DN_F_P].d, p, pb, cudaMemcpyDeviceToDevice, h->stream));
      DN_CUDA(h, cudaMemcpyAsync(f[DN_F_P_PREV].d, p_prev, pb, cudaMemcpyDeviceToDevice, h->stream));
      DN_TRY(bc(h, f[DN_F_P], kBCPressure));
      DN_TRY(bc(h, f[DN_F_P_PREV], kBCPressure));
      DN_TRY(split_extrapolation(h, step));
    }
    LAUNCH_INTERIOR(k_adj_fold_u, h->urhs, GU, h->urhs, h->G, h->bc);
    LAUNCH_INTERIOR(k_adj_fold_v, h->vrhs, GV, h->vrhs, h->G, h->bc);
    const long long nf = (long long)(h->G.nx + 1) * h->G.ny + (long long)h->G.nx * (h->G.ny + 1);
    k_proj_rho_adj<<<blocks_for(nf), 256, 0, h->stream>>>(h->urhs, h->vrhs, h->x, h->bih, h->pe, f[DN_F_RHO_MID], AR,
                                                          h->G, h->bc, split ? 1 : 0, rho_ref, cfg.dt);
    DN_TRY(check_launch(h, "k_proj_rho_adj"));
  }
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  if (iterations) *iterations = rep.pressure_iterations;
  if (relative_residual) *relative_residual = rep.pressure_residual;
  return DN_OK;
}

dn_status dn_projection_adjoint(dn_handle *h, int step, const double *gu, const double *gv, const double *gp,
                                const double *gpp, double *au, double *av, double *ap, double *app, int *iterations,
                                double *relative_residual) {
  if (!h || !gu || !gv || !gp || !gpp || !au || !av || !ap || !app) return DN_ERR_INVALID_ARGUMENT;
  return projection_adjoint(h, step, gu, gv, gp, gpp, au, av, ap, app, nullptr, nullptr, nullptr, nullptr,
                            iterations, relative_residual);
}

// dn_projection with rho_mid as an input (scalar BC applied), and its vector-Jacobian product including the
// cotangent of rho_mid.  DEVICE buffers.
dn_status dn_projection_rho(dn_handle *h, int step, const double *u_star, const double *v_star, const double *p,
                            const double *p_prev, const double *rho_mid, double *u, double *v, double *p_new,
                            double *p_prev_new, int *iterations, double *relative_residual) {
  if (!h || !rho_mid) return DN_ERR_INVALID_ARGUMENT;
  const Fv &R = h->f[DN_F_RHO_MID];
  DN_CUDA(h, cudaMemcpyAsync(R.d, rho_mid, R.size() * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  DN_TRY(bc(h, R, kBCScalar));
  return dn_projection(h, step, u_star, v_star, p, p_prev, u, v, p_new, p_prev_new, iterations, relative_residual);
}
dn_status dn_projection_rho_adjoint(dn_handle *h, int step, const double *rho_mid, const double *p,
                                    const double *p_prev, const double *p_new, const double *gu, const double *gv,
                                    const double *gp, const double *gpp, double *au, double *av, double *ap,
                                    double *app, double *arho, int *iterations, double *relative_residual) {
  if (!h || !rho_mid || !p || !p_prev || !p_new || !gu || !gv || !gp || !gpp || !au || !av || !ap || !app || !arho)
    return DN_ERR_INVALID_ARGUMENT;
  const Fv &R = h->f[DN_F_RHO_MID];
  DN_CUDA(h, cudaMemcpyAsync(R.d, rho_mid, R.size() * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  DN_TRY(bc(h, R, kBCScalar));
  return projection_adjoint(h, step, gu, gv, gp, gpp, au, av, ap, app, p, p_prev, p_new, arho, iterations,
                            relative_residual);
}

// The momentum predictor as a map (u, v, H_prev, f, rho_mid, eta, eta_prev) -> (u*, v*, H)
// (compute_momentum_fluxes + solve_momentum_predictor, momentum.cpp:55-85, 157-502).  DEVICE Field2D buffers.
dn_status dn_momentum_map(dn_handle *h, int step, const double *u, const double *v, const double *hu_prev,
                          const double *hv_prev, const double *fxu, const double *fyv, const double *rho_mid,
                          const double *eta, const double *eta_prev, double *u_star, double *v_star, double *hu,
                          double *hv, int *iterations, double *residual) {
  if (!h || !u || !v || !hu_prev || !hv_prev || !fxu || !fyv || !rho_mid || !eta || !eta_prev || !u_star ||
      !v_star || !hu || !hv)
    return DN_ERR_INVALID_ARGUMENT;
  Fv *f = h->f;
  auto d2d = [&](double *dst, const double *src, int id) -> dn_status {
    DN_CUDA(h, cudaMemcpyAsync(dst, src, f[id].size() * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    return DN_OK;
  };
  DN_TRY(d2d(f[DN_F_U].d, u, DN_F_U));
  DN_TRY(d2d(f[DN_F_V].d, v, DN_F_V));
  DN_TRY(bc(h, f[DN_F_U], kBCU));
  DN_TRY(bc(h, f[DN_F_V], kBCV));
  DN_TRY(d2d(f[DN_F_HU_PREV].d, hu_prev, DN_F_HU_PREV));
  DN_TRY(d2d(f[DN_F_HV_PREV].d, hv_prev, DN_F_HV_PREV));
  DN_TRY(d2d(f[DN_F_SFX_U].d, fxu, DN_F_SFX_U));
  DN_TRY(d2d(f[DN_F_SFY_V].d, fyv, DN_F_SFY_V));
  const int mats[3] = {DN_F_RHO_MID, DN_F_ETA, DN_F_ETA_PREV};
  const double *msrc[3] = {rho_mid, eta, eta_prev};
  for (int k = 0; k < 3; ++k) {
    DN_TRY(d2d(f[mats[k]].d, msrc[k], mats[k]));
    DN_TRY(bc(h, f[mats[k]], kBCScalar));
  }
  dn_report rep{};
  DN_TRY(momentum(h, step, &rep));
  DN_TRY(d2d(u_star, f[DN_F_U_STAR].d, DN_F_U_STAR));
  DN_TRY(d2d(v_star, f[DN_F_V_STAR].d, DN_F_V_STAR));
  DN_TRY(d2d(hu, f[DN_F_HU_PREV].d, DN_F_HU_PREV));  // momentum() leaves this step's H there
  DN_TRY(d2d(hv, f[DN_F_HV_PREV].d, DN_F_HV_PREV));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  if (iterations) *iterations = rep.momentum_iterations;
  if (residual) *residual = rep.momentum_residual;
  return DN_OK;
}

// Vector-Jacobian product of dn_momentum_map at its forward point (u, v, H_prev, materials, and the
// solution u*, v*) (dn_momentum_adjoint.cuh): cotangents of u*, v*, H in; cotangents of u, v, H_prev
// (ahu, ahv), f (afu, afv), rho_mid, eta and eta_prev out (ghosts zero).  The transposed solve runs to a
// relative residual of 1e-14 (at most 20 x momentum_iterations iterations).
dn_status dn_momentum_adjoint(dn_handle *h, int step, const double *u, const double *v, const double *hu_prev,
                              const double *hv_prev, const double *rho_mid, const double *eta, const double *eta_prev,
                              const double *u_star, const double *v_star, const double *gu_star,
                              const double *gv_star, const double *ghu, const double *ghv, double *au, double *av,
                              double *ahu, double *ahv, double *afu, double *afv, double *arho, double *aeta,
                              double *aeta_prev, int *iterations, double *residual) {
  if (!h || !u || !v || !hu_prev || !hv_prev || !rho_mid || !eta || !eta_prev || !u_star || !v_star || !gu_star ||
      !gv_star || !ghu || !ghv || !au || !av || !ahu || !ahv || !afu || !afv || !arho || !aeta || !aeta_prev)
    return DN_ERR_INVALID_ARGUMENT;
  const dn_config &cfg = h->cfg;
  Fv *f = h->f;
  const Fv &U = f[DN_F_U], &V = f[DN_F_V], &Cell = f[DN_F_RHO_MID];
  auto view = [](const double *p, const Fv &like) { return Fv{const_cast<double *>(p), like.nx, like.ny, like.g}; };
  const Fv GU = view(gu_star, U), GV = view(gv_star, V), GHU = view(ghu, U), GHV = view(ghv, V);
  const Fv AU = view(au, U), AV = view(av, V), AHU = view(ahu, U), AHV = view(ahv, V), AFU = view(afu, U),
           AFV = view(afv, V), AR = view(arho, Cell), AE = view(aeta, Cell), AEP = view(aeta_prev, Cell);
  for (const Fv *o : {&AU, &AV, &AHU, &AHV, &AFU, &AFV, &AR, &AE, &AEP})
    DN_CUDA(h, cudaMemsetAsync(o->d, 0, o->size() * sizeof(double), h->stream));
  auto load = [&](int id, const double *src, int kind) -> dn_status {
    DN_CUDA(h, cudaMemcpyAsync(f[id].d, src, f[id].size() * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    return kind >= 0 ? bc(h, f[id], kind) : DN_OK;
  };
  DN_TRY(load(DN_F_U, u, kBCU));
  DN_TRY(load(DN_F_V, v, kBCV));
  DN_TRY(load(DN_F_U_STAR, u_star, kBCU));
  DN_TRY(load(DN_F_V_STAR, v_star, kBCV));
  DN_TRY(load(DN_F_HU_PREV, hu_prev, -1));
  DN_TRY(load(DN_F_HV_PREV, hv_prev, -1));
  DN_TRY(load(DN_F_RHO_MID, rho_mid, kBCScalar));
  DN_TRY(load(DN_F_ETA, eta, kBCScalar));
  DN_TRY(load(DN_F_ETA_PREV, eta_prev, kBCScalar));
  if (!h->mtcoef) {
    dn_status s = dalloc(h, &h->mtcoef, 9 * h->nm);
    if (s == DN_OK) s = dalloc(h, &h->mttgt, 9 * h->nm);
    if (s != DN_OK) return fail(h, s, "device allocation failed: " + h->err);
  }
  const double alpha = 0.5 * cfg.dt / cfg.re;
  // M at these materials (its right-hand side is not used), then M^T
  k_mom_assemble<<<blocks_for(h->nm, 128), 128, 0, h->stream>>>(h->ml, h->G, h->bc, U, V, f[DN_F_RHO_MID], f[DN_F_ETA],
                                                           h->urhs, h->vrhs, alpha, h->mcoef, h->mtgt, h->mb, h->mx);
  DN_TRY(check_launch(h, "k_mom_assemble"));
  k_mom_transpose<<<blocks_for(h->nm), 256, 0, h->stream>>>(h->ml, h->mcoef, h->mtgt, h->mtcoef, h->mttgt);
  DN_TRY(check_launch(h, "k_mom_transpose"));
  // the cotangent of u*, v* through their face BCs, at the active faces
  LAUNCH_INTERIOR(k_adj_fold_u, h->urhs, GU, h->urhs, h->G, h->bc);
  LAUNCH_INTERIOR(k_adj_fold_v, h->vrhs, GV, h->vrhs, h->G, h->bc);
  k_mom_gather<<<blocks_for(h->nm), 256, 0, h->stream>>>(h->ml, h->urhs, h->vrhs, h->mb);
  DN_TRY(check_launch(h, "k_mom_gather"));
  DN_CUDA(h, cudaMemsetAsync(h->mx, 0, h->nm * sizeof(double), h->stream));
  double out[4];
  DN_TRY(run_bicgstab(h, out, h->mtcoef, h->mttgt, 1, 1.0e-14, 20 * std::max(1, cfg.momentum_iterations)));
  // lambda on the faces (h->hu, h->hv); H's cotangent through H's face BC (h->urhs, h->vrhs)
  DN_TRY(fill_field(h, h->hu, 0.0));
  DN_TRY(fill_field(h, h->hv, 0.0));
  k_mom_scatter<<<blocks_for(h->nm), 256, 0, h->stream>>>(h->ml, h->mx, h->hu, h->hv);
  DN_TRY(check_launch(h, "k_mom_scatter"));
  LAUNCH_INTERIOR(k_adj_fold_u, h->urhs, GHU, h->urhs, h->G, h->bc);
  LAUNCH_INTERIOR(k_adj_fold_v, h->vrhs, GHV, h->vrhs, h->G, h->bc);
  k_mom_rhs_adj<<<blocks_for(h->nm), 256, 0, h->stream>>>(h->ml, U, V, f[DN_F_RHO_MID], f[DN_F_ETA_PREV], h->hu, h->hv,
                                                          h->urhs, h->vrhs, AU, AV, AFU, AFV, AHU, AHV, h->G, step,
                                                          cfg.dt, alpha);
  DN_TRY(check_launch(h, "k_mom_rhs_adj"));
  k_mom_material_adj<<<blocks_for(h->nm), 256, 0, h->stream>>>(h->ml, f[DN_F_U_STAR], f[DN_F_V_STAR], U, V,
                                                               f[DN_F_HU_PREV], f[DN_F_HV_PREV], h->hu, h->hv, AR, AE,
                                                               AEP, h->G, step, cfg.dt, alpha, cfg.body_force_x,
                                                               cfg.body_force_y);
  DN_TRY(check_launch(h, "k_mom_material_adj"));
  // the input BCs: ghosts onto the values they copy, then the boundary faces
  auto ghosts = [&](const Fv &F, int kind, const BCSide *b) -> dn_status {
    const long long ng = 2LL * F.g * F.ny + 2LL * F.g * (F.nx + 2 * F.g);
    k_adj_ghosts<<<blocks_for(ng), 256, 0, h->stream>>>(F, h->G, kind, b[DN_LEFT], b[DN_RIGHT], b[DN_BOTTOM],
                                                        b[DN_TOP]);
    return check_launch(h, "k_adj_ghosts");
  };
  DN_TRY(ghosts(AU, kBCU, h->bc.u));
  DN_TRY(ghosts(AV, kBCV, h->bc.v));
  for (const Fv *m : {&AR, &AE, &AEP}) DN_TRY(ghosts(*m, kBCScalar, h->bc.p));
  LAUNCH_INTERIOR(k_adj_fold_u, h->urhs, AU, h->urhs, h->G, h->bc);
  LAUNCH_INTERIOR(k_adj_fold_v, h->vrhs, AV, h->vrhs, h->G, h->bc);
  LAUNCH_INTERIOR(k_copy_interior, AU, AU, h->urhs);
  LAUNCH_INTERIOR(k_copy_interior, AV, AV, h->vrhs);
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  if (iterations) *iterations = (int)out[0];
  if (residual) *residual = out[2];
  return DN_OK;
}

// The face surface forces as a map (c_old, c_new) -> (fxu, fyv) (update_surface_tension_force,
// phase_field.cpp:179-256, with the step's smoothing passes).  DEVICE Field2D buffers.
dn_status dn_surface_force_map(dn_handle *h, const double *c_old, const double *c_new, double *fxu, double *fyv) {
  if (!h || !c_old || !c_new || !fxu || !fyv) return DN_ERR_INVALID_ARGUMENT;
  Fv *f = h->f;
  const size_t cb = h->mob.size() * sizeof(double);
  DN_CUDA(h, cudaMemcpyAsync(h->mob.d, c_old, cb, cudaMemcpyDeviceToDevice, h->stream));
  DN_CUDA(h, cudaMemcpyAsync(h->lap.d, c_new, cb, cudaMemcpyDeviceToDevice, h->stream));
  DN_TRY(bc(h, h->mob, kBCScalar));
  DN_TRY(bc(h, h->lap, kBCScalar));
  DN_TRY(surface_force(h, h->mob, h->lap));
  DN_CUDA(h, cudaMemcpyAsync(fxu, f[DN_F_SFX_U].d, f[DN_F_SFX_U].size() * sizeof(double), cudaMemcpyDeviceToDevice,
                             h->stream));
  DN_CUDA(h, cudaMemcpyAsync(fyv, f[DN_F_SFY_V].d, f[DN_F_SFY_V].size() * sizeof(double), cudaMemcpyDeviceToDevice,
                             h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  return DN_OK;
}

// Vector-Jacobian product of dn_surface_force_map (dn_momentum_adjoint.cuh, k_sf_adj_faces, k_chem_adj):
// cotangents of the interior face forces in, of the interior values of c_old and c_new out (equal: the
// forces depend on c_mid = (c_old + c_new) / 2 only).  Not available with smoothing passes.
dn_status dn_surface_force_adjoint(dn_handle *h, const double *c_old, const double *c_new, const double *gfxu,
                                   const double *gfyv, double *ac_old, double *ac_new) {
  if (!h || !c_old || !c_new || !gfxu || !gfyv || !ac_old || !ac_new) return DN_ERR_INVALID_ARGUMENT;
  const dn_config &cfg = h->cfg;
  Fv *f = h->f;
  const Fv &Cc = f[DN_F_C];
  const Fv ACO{ac_old, Cc.nx, Cc.ny, Cc.g}, ACN{ac_new, Cc.nx, Cc.ny, Cc.g};
  DN_CUDA(h, cudaMemsetAsync(ac_old, 0, Cc.size() * sizeof(double), h->stream));
  DN_CUDA(h, cudaMemsetAsync(ac_new, 0, Cc.size() * sizeof(double), h->stream));
  if (cfg.surface_tension_multiplier == 0.0 || !compute_mu(cfg)) return DN_OK;
  if (cfg.surface_tension_smoothing_passes > 0 && cfg.surface_tension_smoothing_weight > 0.0)
    return fail(h, DN_ERR_UNSUPPORTED, "the surface-force adjoint does not cover smoothing passes");
  const Fv &FU = f[DN_F_SFX_U], &FV = f[DN_F_SFY_V];
  const Fv GFU{const_cast<double *>(gfxu), FU.nx, FU.ny, FU.g}, GFV{const_cast<double *>(gfyv), FV.nx, FV.ny, FV.g};
  // c_mid (scalar BC ghosts) and mu_mid, as the forward builds them
  const size_t cb = Cc.size() * sizeof(double);
  DN_CUDA(h, cudaMemcpyAsync(h->mob.d, c_old, cb, cudaMemcpyDeviceToDevice, h->stream));
  DN_CUDA(h, cudaMemcpyAsync(h->lap.d, c_new, cb, cudaMemcpyDeviceToDevice, h->stream));
  DN_TRY(bc(h, h->mob, kBCScalar));
  DN_TRY(bc(h, h->lap, kBCScalar));
  LAUNCH_INTERIOR(k_cmid, h->cmid, h->mob, h->lap, h->cmid);
  DN_TRY(bc(h, h->cmid, kBCScalar));
  LAUNCH_INTERIOR(k_chem, h->mm, h->cmid, h->mm, h->G, cfg.cn);
  // the forces' face BCs folded (into the face work arrays), then the transposed stencils
  LAUNCH_INTERIOR(k_adj_fold_u, h->urhs, GFU, h->urhs, h->G, h->bc);
  LAUNCH_INTERIOR(k_adj_fold_v, h->vrhs, GFV, h->vrhs, h->G, h->bc);
  DN_TRY(fill_field(h, h->bih, 0.0));   // c_mid cotangent
  DN_TRY(fill_field(h, h->ddiv, 0.0));  // mu_mid cotangent
  const double scale = cfg.surface_tension_multiplier / (cfg.re * cfg.ca);
  const long long nf = (long long)(h->G.nx + 1) * h->G.ny + (long long)h->G.nx * (h->G.ny + 1);
  k_sf_adj_faces<<<blocks_for(nf), 256, 0, h->stream>>>(h->urhs, h->vrhs, h->cmid, h->mm, h->bih, h->ddiv, h->G, scale);
  DN_TRY(check_launch(h, "k_sf_adj_faces"));
  LAUNCH_INTERIOR(k_chem_adj, h->cmid, h->cmid, h->ddiv, h->bih, h->G, cfg.cn);
  const Fv &B = h->bih;
  const long long ng = 2LL * B.g * B.ny + 2LL * B.g * (B.nx + 2 * B.g);
  k_adj_ghosts<<<blocks_for(ng), 256, 0, h->stream>>>(B, h->G, kBCScalar, h->bc.p[DN_LEFT], h->bc.p[DN_RIGHT],
                                                      h->bc.p[DN_BOTTOM], h->bc.p[DN_TOP]);
  DN_TRY(check_launch(h, "k_adj_ghosts"));
  LAUNCH_INTERIOR(k_half_interior, ACO, B, ACO);
  LAUNCH_INTERIOR(k_half_interior, ACN, B, ACN);
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  return DN_OK;
}

// The CH advective term on caller device buffers: c (cell), u, v (faces) in, rhs = -div(u c) (cell) out,
// computed as the phase step computes it (WENO5 faces, velocity face BCs on the fluxes).
dn_status dn_advection(dn_handle *h, const double *c, const double *u, const double *v, double *rhs) {
  if (!h || !c || !u || !v || !rhs) return DN_ERR_INVALID_ARGUMENT;
  Fv *f = h->f;
  const Fv &CF = f[DN_F_C], &UF = f[DN_F_U], &VF = f[DN_F_V];
  const Fv U{const_cast<double *>(u), UF.nx, UF.ny, UF.g}, V{const_cast<double *>(v), VF.nx, VF.ny, VF.g};
  const Fv R{rhs, CF.nx, CF.ny, CF.g};
  DN_CUDA(h, cudaMemcpyAsync(h->cmid.d, c, CF.size() * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  DN_TRY(bc(h, h->cmid, kBCScalar));
  LAUNCH_INTERIOR(k_adv_flux_x, h->afx, h->cmid, U, h->afx);
  LAUNCH_INTERIOR(k_adv_flux_y, h->afy, h->cmid, V, h->afy);
  DN_TRY(bc(h, h->afx, kBCU));
  DN_TRY(bc(h, h->afy, kBCV));
  LAUNCH_INTERIOR(k_flux_div, R, h->afx, h->afy, R, h->G, 1);
  DN_TRY(bc(h, R, kBCScalar));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  return DN_OK;
}

// Vector-Jacobian product of dn_advection at (c, u, v): cotangent g_rhs of the interior of rhs in;
// cotangents of the interior values of c, u, v out (ghosts set to 0).
dn_status dn_advection_adjoint(dn_handle *h, const double *c, const double *u, const double *v, const double *g_rhs,
                               double *c_bar, double *u_bar, double *v_bar) {
  if (!h || !c || !u || !v || !g_rhs || !c_bar || !u_bar || !v_bar) return DN_ERR_INVALID_ARGUMENT;
  Fv *f = h->f;
  const Fv &CF = f[DN_F_C], &UF = f[DN_F_U], &VF = f[DN_F_V];
  const Fv U{const_cast<double *>(u), UF.nx, UF.ny, UF.g}, V{const_cast<double *>(v), VF.nx, VF.ny, VF.g};
  const Fv RB{const_cast<double *>(g_rhs), CF.nx, CF.ny, CF.g};
  const Fv CB{c_bar, CF.nx, CF.ny, CF.g}, UB{u_bar, UF.nx, UF.ny, UF.g}, VB{v_bar, VF.nx, VF.ny, VF.g};
  DN_CUDA(h, cudaMemsetAsync(c_bar, 0, CF.size() * sizeof(double), h->stream));
  DN_CUDA(h, cudaMemsetAsync(u_bar, 0, UF.size() * sizeof(double), h->stream));
  DN_CUDA(h, cudaMemsetAsync(v_bar, 0, VF.size() * sizeof(double), h->stream));
  DN_CUDA(h, cudaMemcpyAsync(h->cmid.d, c, CF.size() * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  DN_TRY(bc(h, h->cmid, kBCScalar));
  LAUNCH_INTERIOR(k_adv_adj_u, UB, h->cmid, U, RB, UB, h->G, h->bc);
  LAUNCH_INTERIOR(k_adv_adj_v, VB, h->cmid, V, RB, VB, h->G, h->bc);
  LAUNCH_INTERIOR(k_adv_adj_c, CB, h->cmid, U, V, RB, CB, h->G, h->bc);
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  return DN_OK;
}

// The CH explicit operator E(c, u, v) on caller device buffers (cell c, faces u, v in; cell E out, ghosts
// filled), computed as the phase step computes it.
dn_status dn_explicit_operator(dn_handle *h, const double *c, const double *u, const double *v, double *E) {
  if (!h || !c || !u || !v || !E) return DN_ERR_INVALID_ARGUMENT;
  Fv *f = h->f;
  const Fv &CF = f[DN_F_C], &UF = f[DN_F_U], &VF = f[DN_F_V];
  const Fv U{const_cast<double *>(u), UF.nx, UF.ny, UF.g}, V{const_cast<double *>(v), VF.nx, VF.ny, VF.g};
  DN_CUDA(h, cudaMemcpyAsync(h->cmid.d, c, CF.size() * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  DN_TRY(bc(h, h->cmid, kBCScalar));
  DN_TRY(phase_explicit(h, h->cmid, U, V));
  DN_CUDA(h, cudaMemcpyAsync(E, h->E_new.d, CF.size() * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  return DN_OK;
}

// Vector-Jacobian product of dn_explicit_operator at (c, u, v): cotangent gE of the interior of E in;
// cotangents of the interior values of c, u, v out (ghosts 0).
dn_status dn_explicit_operator_adjoint(dn_handle *h, const double *c, const double *u, const double *v,
                                       const double *gE, double *c_bar, double *u_bar, double *v_bar) {
  if (!h || !c || !u || !v || !gE || !c_bar || !u_bar || !v_bar) return DN_ERR_INVALID_ARGUMENT;
  Fv *f = h->f;
  const dn_config &cfg = h->cfg;
  const Fv &CF = f[DN_F_C], &UF = f[DN_F_U], &VF = f[DN_F_V];
  const Fv U{const_cast<double *>(u), UF.nx, UF.ny, UF.g}, V{const_cast<double *>(v), VF.nx, VF.ny, VF.g};
  const Fv RB{const_cast<double *>(gE), CF.nx, CF.ny, CF.g};
  const Fv CB{c_bar, CF.nx, CF.ny, CF.g}, UB{u_bar, UF.nx, UF.ny, UF.g}, VB{v_bar, VF.nx, VF.ny, VF.g};
  DN_CUDA(h, cudaMemsetAsync(c_bar, 0, CF.size() * sizeof(double), h->stream));
  DN_CUDA(h, cudaMemsetAsync(u_bar, 0, UF.size() * sizeof(double), h->stream));
  DN_CUDA(h, cudaMemsetAsync(v_bar, 0, VF.size() * sizeof(double), h->stream));
  // forward intermediates: c with its ghosts, mobility, chemical potential
  DN_CUDA(h, cudaMemcpyAsync(h->cmid.d, c, CF.size() * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  DN_TRY(bc(h, h->cmid, kBCScalar));
  LAUNCH_INTERIOR(k_mob_lap, h->mob, h->cmid, h->mob, h->lap, h->G);
  DN_TRY(bc(h, h->mob, kBCScalar));
  DN_TRY(chem(h, h->cmid, h->mu_t));
  // the cotangent with its scalar-BC ghosts (for the transposed Laplacians)
  DN_CUDA(h, cudaMemcpyAsync(h->E_new.d, gE, CF.size() * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  DN_TRY(bc(h, h->E_new, kBCScalar));
  const double inv_pe = 1.0 / cfg.pe;
  // diffusive part: face cotangents, then mobility and chemical potential per cell
  LAUNCH_INTERIOR(k_eadj_face_x, h->afx, h->E_new, h->mob, h->mu_t, h->afx, h->dfx, h->G, h->bc, inv_pe);
  LAUNCH_INTERIOR(k_eadj_face_y, h->afy, h->E_new, h->mob, h->mu_t, h->afy, h->dfy, h->G, h->bc, inv_pe);
  LAUNCH_INTERIOR(k_eadj_cells, CB, h->cmid, h->afx, h->dfx, h->afy, h->dfy, h->ddiv, CB, h->G, cfg.cn);
  DN_TRY(bc(h, h->ddiv, kBCScalar));
  const double alpha = 6.0 * kSqrt2;
  LAUNCH_INTERIOR(k_add_scaled_lap, CB, h->ddiv, CB, h->G, -alpha * cfg.cn);
  // -(a1 L c - a2 L L c) / pe: L^T (-(a1/pe) g + (a2/pe) L^T g)
  const double a1 = cfg.cn > 0.0 ? (3.0 * kSqrt2 / (16.0 * cfg.cn)) : 0.0;
  const double a2 = cfg.cn > 0.0 ? (3.0 * kSqrt2 * cfg.cn / 4.0) : 0.0;
  LAUNCH_INTERIOR(k_lin_lap, h->arhs, h->E_new, h->arhs, h->G, -a1 * inv_pe, a2 * inv_pe);
  DN_TRY(bc(h, h->arhs, kBCScalar));
  LAUNCH_INTERIOR(k_add_scaled_lap, CB, h->arhs, CB, h->G, 1.0);
  // advective part
  LAUNCH_INTERIOR(k_adv_adj_u, UB, h->cmid, U, RB, UB, h->G, h->bc);
  LAUNCH_INTERIOR(k_adv_adj_v, VB, h->cmid, V, RB, VB, h->G, h->bc);
  LAUNCH_INTERIOR(k_adv_adj_c, CB, h->cmid, U, V, RB, CB, h->G, h->bc);
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  return DN_OK;
}

dn_status dn_compute_mass(dn_handle *h, int field, double *mass) {
  if (!h || !mass || field < 0 || field >= DN_F_COUNT) return DN_ERR_INVALID_ARGUMENT;
  const int nb = 128;
  const Fv &f = h->f[field];
  k_field_sum<<<nb, 256, 0, h->stream>>>(f, h->G.dx * h->G.dy, h->partials);
  DN_TRY(check_launch(h, "k_field_sum"));
  k_finish_mean<<<1, 32, 0, h->stream>>>(h->partials, nb, 1.0, h->scal + 8);
  DN_TRY(check_launch(h, "k_finish_mean"));
  return read_scalars(h, 1, mass);
}

dn_status dn_diagnostics(dn_handle *h, dn_diag *d) {
  if (!h || !d) return DN_ERR_INVALID_ARGUMENT;
  DN_TRY(diag_launch(h));
  DN_CUDA(h, cudaMemcpyAsync(h->host_scal, h->partials, (size_t)kDiagParts * kNDiag * sizeof(double),
                             cudaMemcpyDeviceToHost, h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  return diag_finish(h, h->host_scal, d);
}

dn_status dn_synchronize(dn_handle *h) {
  if (!h) return DN_ERR_INVALID_ARGUMENT;
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  return DN_OK;
}

void *dn_stream(dn_handle *h) { return h ? (void *)h->stream : nullptr; }

dn_status dn_last_phase_times(dn_handle *h, double *out) {
  if (!h || !out) return DN_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < 8; ++k) out[k] = h->phase_ms[k];
  for (int k = 0; k < 3; ++k) out[8 + k] = h->pcg_split_ms[k];
  return DN_OK;
}

long long dn_kernel_launches(const dn_handle *h) { return h ? h->launches : 0; }

dn_status dn_profile_counters(dn_handle *h, double *out, int count) {
  if (!h || !out || count < 0 || count > 64) return DN_ERR_INVALID_ARGUMENT;
  DN_CUDA(h, cudaMemcpyAsync(out, h->prof, (size_t)count * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  DN_CUDA(h, cudaStreamSynchronize(h->stream));
  return DN_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------------
// Allocation-free pressure solve: dn_pressure_solve_static.
//
// Some callers cannot allocate device memory when they need a pressure solve: a host framework whose
// caching pool has already reserved the GPU's memory, a real-time loop that may not stall on cudaMalloc
// (which synchronises the device), or a caller that holds nothing but raw device pointers and no handle
// lifetime.  This variant of the pressure PCG runs on the caller's device buffers and stream and keeps
// every intermediate (operator, factor, Krylov vectors, hand-over lines, reduction partials, barrier
// words) in one fixed file-scope device array, so it calls no allocator at all.  The array is part of the
// library's device image: every GPU that loads the library holds DN_STATIC_SCRATCH_BYTES of it until the
// process exits.  All calls share it, so calls that overlap in time on one device (two host threads, or
// two streams) race on it; the caller serialises them.
// ---------------------------------------------------------------------------------------------------
static __device__ __align__(256) double g_pressure_scratch[DN_STATIC_SCRATCH_BYTES / sizeof(double)];

namespace {

constexpr int kStaticMaxDevices = 64;

// Per device: the launch limits of the PCG kernels, resolved once with that device current.  The device
// address of g_pressure_scratch (the name is only a host-side stand-in) is not cached here: it is resolved
// by cudaGetSymbolAddress on every call, so that a context that was destroyed and re-created (for instance
// after cudaDeviceReset, which loads the module again) never sees a stale address.
struct StaticDevice {
  bool ready;
  char *base;
  int num_sms;
  int smem_optin;
  int max_coop_blocks;
  int pcg3_static_smem;  // static shared memory of k_pcg<5,3> / k_pcg<5,4> (the larger)
};
std::mutex g_static_mu;
StaticDevice g_static_dev[kStaticMaxDevices];

dn_status static_fail(char *err, size_t err_len, dn_status s, const char *fmt, ...) {
  if (err && err_len) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, err_len, fmt, ap);
    va_end(ap);
  }
  return s;
}

#define DN_SCUDA(call)                                                                                   \
  do {                                                                                                   \
    cudaError_t e_ = (call);                                                                             \
    if (e_ != cudaSuccess) return static_fail(err, err_len, DN_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

#define DN_SLAUNCH(what)                                                                                 \
  do {                                                                                                   \
    cudaError_t e_ = cudaGetLastError();                                                                 \
    if (e_ != cudaSuccess) return static_fail(err, err_len, DN_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e_)); \
  } while (0)

// Byte offsets of the sub-buffers inside the scratch array, each on a 256-byte boundary.
struct StaticLayout {
  size_t bar_count, bar_gen, status, prog, partials, scal, prof;
  size_t b, x, r, z, y, p0, p1, ap, a5, l5, d5, dinv5, pe, bnd_f, bnd_b, wline0, zlast;
  size_t total;
};

StaticLayout static_layout(int nx, int ny, int g) {
  StaticLayout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off += (bytes + 255) & ~(size_t)255;
    return at;
  };
  const size_t n = (size_t)nx * ny;
  const size_t nsweep = std::max((size_t)(nx + 31) / 32, (size_t)staged_sweep_warps(nx));
  L.bar_count = take(sizeof(unsigned int));
  L.bar_gen = take(sizeof(unsigned int));
  L.status = take(4 * sizeof(int));  // [status, pad, poll limit]: the limit stays 0 (the default)
  L.prog = take(2 * (size_t)kMaxBlocks * 8 * sizeof(unsigned int));
  L.partials = take(2 * (size_t)kMaxBlocks * 8 * sizeof(double));
  L.scal = take(64 * sizeof(double));
  L.prof = take(64 * sizeof(double));
  for (size_t *v : {&L.b, &L.x, &L.r, &L.z, &L.y, &L.p0, &L.p1, &L.ap}) *v = take(n * sizeof(double));
  L.a5 = take(5 * n * sizeof(double));
  L.l5 = take(5 * n * sizeof(double));
  L.d5 = take(n * sizeof(double));
  L.dinv5 = take(n * sizeof(double));
  L.pe = take((size_t)(nx + 2 * g) * (ny + 2 * g) * sizeof(double));
  L.bnd_f = take(2 * nsweep * ny * sizeof(double));
  L.bnd_b = take(2 * nsweep * ny * sizeof(double));
  L.wline0 = take(2 * (size_t)ny * sizeof(double));
  L.zlast = take(2 * (size_t)ny * sizeof(double));
  L.total = off;
  return L;
}

// Set-up of the current device: the array's device address (every call) and the launch limits (first
// call on the device).  Symbol lookups, occupancy queries and attribute calls allocate nothing.
dn_status static_setup(int device, StaticDevice *out, char *err, size_t err_len) {
  std::lock_guard<std::mutex> lock(g_static_mu);
  StaticDevice &d = g_static_dev[device];
  void *ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&ptr, g_pressure_scratch);
  if (e != cudaSuccess)
    return static_fail(err, err_len, DN_ERR_CUDA, "cudaGetSymbolAddress(g_pressure_scratch): %s",
                       cudaGetErrorString(e));
  if (!d.ready) {
    StaticDevice t{};
    DN_SCUDA(cudaDeviceGetAttribute(&t.num_sms, cudaDevAttrMultiProcessorCount, device));
    DN_SCUDA(cudaDeviceGetAttribute(&t.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    cudaFuncAttributes fa{};
    DN_SCUDA(cudaFuncGetAttributes(&fa, k_pcg<5, 3>));
    t.pcg3_static_smem = (int)fa.sharedSizeBytes;
    DN_SCUDA(cudaFuncGetAttributes(&fa, k_pcg<5, 4>));
    t.pcg3_static_smem = std::max(t.pcg3_static_smem, (int)fa.sharedSizeBytes);
    // the same co-residency bound as a handle's (all persistent kernels of the library)
    int occ = 0, occ2 = 0, occ3 = 0;
    DN_SCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pcg<5, 0>, kBlock, 0));
    DN_SCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, k_pcg<13, 1>, kBlock, 0));
    DN_SCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ3, k_bicgstab, kBlock, 0));
    occ = std::min(occ, std::min(occ2, occ3));
    t.max_coop_blocks = std::min(kMaxBlocks, std::max(1, occ) * t.num_sms);
    t.ready = true;
    d = t;
  }
  *out = d;
  out->base = static_cast<char *>(ptr);
  return DN_OK;
}

dn_status static_device_status(int st, char *err, size_t err_len) {
  switch (st) {
  case kDevOk: return DN_OK;
  case kDevTimeout:
    return static_fail(err, err_len, DN_ERR_TIMEOUT, "device wait timed out (grid barrier or wavefront flag)");
  case kDevPcgBreakdownRz0:
    return static_fail(err, err_len, DN_ERR_PCG_BREAKDOWN, "pcg preconditioner breakdown: non-positive r^T M^{-1} r");
  case kDevPcgBreakdownPap:
    return static_fail(err, err_len, DN_ERR_PCG_BREAKDOWN, "pcg breakdown: p^T A p is invalid");
  case kDevPcgBreakdownRz:
    return static_fail(err, err_len, DN_ERR_PCG_BREAKDOWN,
                       "pcg preconditioner breakdown: non-positive new r^T M^{-1} r");
  default: return static_fail(err, err_len, DN_ERR_CUDA, "unknown device status %d", st);
  }
}

dn_status static_read(void *host, const void *dev, size_t bytes, cudaStream_t st, char *err, size_t err_len) {
  DN_SCUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, st));
  DN_SCUDA(cudaStreamSynchronize(st));
  return DN_OK;
}

dn_status static_bc_pressure(const Fv &f, const Grid &G, const BCSet &B, cudaStream_t st, char *err,
                             size_t err_len) {
  const long long nghost = 2LL * f.g * f.ny + 2LL * f.g * (f.nx + 2 * f.g);
  k_bc_ghosts<<<blocks_for(nghost), 256, 0, st>>>(f, G, kBCPressure, B.p[0], B.p[1], B.p[2], B.p[3]);
  DN_SLAUNCH("k_bc_ghosts");
  return DN_OK;
}

}  // namespace

extern "C" {

dn_status dn_pressure_solve_static(const dn_config *cfg, int step, const double *u_star, const double *v_star,
                                   const double *rho_mid, const double *p, const double *p_prev, double *p_corr,
                                   void *stream, int *iterations, double *relative_residual, char *err,
                                   size_t err_len) {
  if (err && err_len) err[0] = '\0';
  if (!cfg || !u_star || !v_star || !rho_mid || !p || !p_prev || !p_corr)
    return static_fail(err, err_len, DN_ERR_INVALID_ARGUMENT, "null pointer argument");
  const dn_config &c = *cfg;
  if (c.nx < 8 || c.ny < 8) return static_fail(err, err_len, DN_ERR_UNSUPPORTED, "the CUDA backend needs nx, ny >= 8");
  if (c.ghost < 3) return static_fail(err, err_len, DN_ERR_UNSUPPORTED, "ghost must be >= 3 (WENO5 stencil)");
  if (c.pressure_scheme == DN_P_JACOBI)
    return static_fail(err, err_len, DN_ERR_UNSUPPORTED,
                       "pressure_scheme jacobi is not implemented by the CUDA backend");
  if (c.pressure_scheme == DN_P_SPLIT_DCDM_ICPCG)
    return static_fail(err, err_len, DN_ERR_UNSUPPORTED,
                       "pressure_scheme split_dcdm_icpcg keeps a direction history and needs a handle");
  if (c.pressure_scheme < DN_P_ICPCG || c.pressure_scheme > DN_P_SPLIT_ILDLT_PCG)
    return static_fail(err, err_len, DN_ERR_CONFIG, "unknown pressure_scheme %d", c.pressure_scheme);
  if (c.precision != DN_PRECISION_FP64)
    return static_fail(err, err_len, DN_ERR_UNSUPPORTED, "precision mixed is not available in this build");
  static const char *names[4] = {"left", "right", "bottom", "top"};
  for (int s = 0; s < 4; ++s) {  // validate_boundary_configuration, operators.cpp:11-34 (pressure and velocity)
    const int periodic = (s < 2) ? c.periodic_x : c.periodic_y;
    if (periodic && (c.p_bc[s].type != DN_BC_UNSET || c.u_bc[s].type != DN_BC_UNSET || c.v_bc[s].type != DN_BC_UNSET))
      return static_fail(err, err_len, DN_ERR_CONFIG, "boundary conditions on side %s cannot be set when the direction is periodic",
                         names[s]);
  }
  if ((long long)c.nx * c.ny > (1LL << 30)) return static_fail(err, err_len, DN_ERR_UNSUPPORTED, "grid too large");
  const StaticLayout L = static_layout(c.nx, c.ny, c.ghost);
  if (L.total > (size_t)DN_STATIC_SCRATCH_BYTES)
    return static_fail(err, err_len, DN_ERR_UNSUPPORTED,
                       "grid %d x %d needs %zu bytes of scratch; the static scratch array holds %zu bytes", c.nx,
                       c.ny, L.total, (size_t)DN_STATIC_SCRATCH_BYTES);

  int device = 0;
  DN_SCUDA(cudaGetDevice(&device));
  if (device < 0 || device >= kStaticMaxDevices)
    return static_fail(err, err_len, DN_ERR_UNSUPPORTED, "device ordinal %d beyond the set-up table", device);
  StaticDevice D{};
  {
    const dn_status s = static_setup(device, &D, err, err_len);
    if (s != DN_OK) return s;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (st != nullptr) {  // the scratch address and the launch limits belong to the current device
    int stream_device = -1;
    DN_SCUDA(cudaStreamGetDevice(st, &stream_device));
    if (stream_device != device)
      return static_fail(err, err_len, DN_ERR_INVALID_ARGUMENT,
                         "stream belongs to device %d, but device %d is current", stream_device, device);
  }

  // grid and effective pressure BCs (operators.cpp:36-112), as a handle derives them
  Grid G;
  G.nx = c.nx;
  G.ny = c.ny;
  G.g = c.ghost;
  G.px = c.periodic_x;
  G.py = c.periodic_y;
  G.dx = c.lx / std::max((double)c.nx, 1.0);
  G.dy = c.ly / std::max((double)c.ny, 1.0);
  BCSet B{};
  for (int s = 0; s < 4; ++s)
    B.p[s] = c.p_bc[s].type != DN_BC_UNSET ? BCSide{c.p_bc[s].type, c.p_bc[s].value} : BCSide{DN_BC_NEUMANN, 0.0};
  const bool has_dirichlet = (!c.periodic_x && (B.p[0].type == DN_BC_DIRICHLET || B.p[1].type == DN_BC_DIRICHLET)) ||
                             (!c.periodic_y && (B.p[2].type == DN_BC_DIRICHLET || B.p[3].type == DN_BC_DIRICHLET));
  const bool split = c.pressure_scheme == DN_P_SPLIT_ICPCG || c.pressure_scheme == DN_P_SPLIT_ILDLT_PCG;
  const bool icc = c.pressure_scheme == DN_P_ICPCG || c.pressure_scheme == DN_P_SPLIT_ICPCG;
  const int kind = icc ? kPrecICC : kPrecLDLT;
  const double rho_ref = split ? std::min(1.0, c.density_ratio) : 1.0;
  const int nx = c.nx, ny = c.ny, g = c.ghost;
  const long long n = (long long)nx * ny;
  const int nsweep = (nx + 31) / 32;
  const int nsweep5 = staged_sweep_warps(nx);

  // caller's fields (read only, except p_corr) and the scratch sub-buffers
  Fv f_us{const_cast<double *>(u_star), nx + 1, ny, g};
  Fv f_vs{const_cast<double *>(v_star), nx, ny + 1, g};
  Fv f_rm{const_cast<double *>(rho_mid), nx, ny, g};
  Fv f_p{const_cast<double *>(p), nx, ny, g};
  Fv f_pp{const_cast<double *>(p_prev), nx, ny, g};
  Fv f_pc{p_corr, nx, ny, g};
  char *base = D.base;
  auto dptr = [&](size_t off) { return reinterpret_cast<double *>(base + off); };
  auto uptr = [&](size_t off) { return reinterpret_cast<unsigned int *>(base + off); };
  Fv f_pe{dptr(L.pe), nx, ny, g};
  double *b = dptr(L.b), *x = dptr(L.x), *a5 = dptr(L.a5), *partials = dptr(L.partials), *scal = dptr(L.scal);
  int *status = reinterpret_cast<int *>(base + L.status);

  // Every call starts from a cleared array: barrier words, status, progress counters, the iterate x and
  // the hand-over lines all have to begin at zero, and clearing the whole used prefix costs a few us.
  DN_SCUDA(cudaMemsetAsync(base, 0, L.total, st));

  // solve_pressure_correction_{icpcg,ildlt_pcg,liu_split_icpcg,liu_split_ildlt_pcg}, pressure.cpp:302-365
  k_fill<<<blocks_for((long long)f_pc.size()), 256, 0, st>>>(f_pc.d, 0.0, (long long)f_pc.size());
  DN_SLAUNCH("k_fill");
  {
    const dn_status s = static_bc_pressure(f_pc, G, B, st, err, err_len);
    if (s != DN_OK) return s;
  }
  if (split) {  // extrapolated pressure p~ = 2p - p_prev (p at step 0), operators.cpp:416
    k_p_ext<<<blocks_for(n), 256, 0, st>>>(f_p, f_pp, f_pe, step == 0 ? 1 : 0);
    DN_SLAUNCH("k_p_ext");
    const dn_status s = static_bc_pressure(f_pe, G, B, st, err, err_len);
    if (s != DN_OK) return s;
  }
  k_p_assemble<<<blocks_for(n), 256, 0, st>>>(G, B, f_rm, f_us, f_vs, f_pe, split ? 1 : 0, rho_ref, c.dt, a5, b);
  DN_SLAUNCH("k_p_assemble");
  if (!has_dirichlet) {  // regularize_pressure_linear_system, pressure.cpp:198-212
    const int nb = 128;
    k_vec_sum<<<nb, 256, 0, st>>>(b, n, partials);
    DN_SLAUNCH("k_vec_sum");
    k_finish_mean<<<1, 32, 0, st>>>(partials, nb, (double)n, scal);
    DN_SLAUNCH("k_finish_mean");
    k_vec_sub_scalar<<<blocks_for(n), 256, 0, st>>>(b, n, scal);
    DN_SLAUNCH("k_vec_sub_scalar");
  }
  const SpOp A{a5, (int)n, nx, ny, G.px, G.py};
  k_factor<5><<<1, 1024, 0, st>>>(A, Factor{dptr(L.l5), dptr(L.d5), dptr(L.dinv5), 0.0}, kind, status);
  DN_SLAUNCH("k_factor<5>");
  int dev_st = 0;
  {
    const dn_status s = static_read(&dev_st, status, sizeof(int), st, err, err_len);
    if (s != DN_OK) return s;
  }
  if (dev_st == kDevFactorFailed)
    return static_fail(err, err_len, icc ? DN_ERR_ICC_FAILED : DN_ERR_ILDLT_FAILED,
                       icc ? "ICC preconditioner construction failed" : "ILDLT preconditioner construction failed");
  if (dev_st != kDevOk) return static_device_status(dev_st, err, err_len);

  // the persistent PCG kernel, launched with the default shape a handle would use for this grid and
  // configuration (device_share included); shapes a handle picked with dn_autotune_pressure are not known
  // here and are not reproduced (pass them as pcg_rows_per_cta / sweep_warps_per_cta)
  PcgArgs P{};
  P.A = A;
  P.l = dptr(L.l5);
  P.dinv = dptr(L.dinv5);
  P.prec = kind;
  P.b = b;
  P.x = x;
  P.r = dptr(L.r);
  P.z = dptr(L.z);
  P.y = dptr(L.y);
  P.p0 = dptr(L.p0);
  P.p1 = dptr(L.p1);
  P.ap = dptr(L.ap);
  P.project = has_dirichlet ? 0 : 1;
  P.max_it = c.poisson_iterations;
  P.tol = c.pressure_tolerance;
  P.tol_abs = c.pressure_tolerance;
  P.bar_count = uptr(L.bar_count);
  P.bar_gen = uptr(L.bar_gen);
  P.status = status;
  P.prog_f = uptr(L.prog);
  P.prog_b = uptr(L.prog) + kMaxBlocks * 8;
  P.partials = partials;
  P.out = scal + 8;
  P.nsweep = nsweep;
  P.warp_smem = 0;
  const long long rows_per_cta = c.pcg_rows_per_cta > 0 ? c.pcg_rows_per_cta : kPcgRowsPerCta;
  const int cta_cap = std::max(1, D.num_sms / std::max(1, c.device_share));
  int blocks = (int)std::min<long long>(cta_cap, std::max<long long>(nsweep, (n + rows_per_cta - 1) / rows_per_cta));
  blocks = std::max(blocks, (nsweep + kBlock / 32 - 1) / (kBlock / 32));  // the wavefront warps' CTAs
  blocks = std::max(1, std::min(blocks, D.max_coop_blocks));
  // staged wavefront: sweep warps per CTA from the shared-memory budget, as dn_create chooses them
  int sw = 0, sw_blocks_max = 0;
  size_t warp_smem = 0;
  const void *k53 = G.px ? (const void *)k_pcg<5, 4> : (const void *)k_pcg<5, 3>;
  if (!G.px || nsweep5 >= 2) {
    const size_t per = (sweep_warp_smem(split ? 2 : 4, ny, 8, G.px != 0) + 15) & ~(size_t)15;
    const size_t budget = (size_t)D.smem_optin > 64 + 2304 ? (size_t)D.smem_optin - 64 - 2304 : 0;
    sw = (int)std::min<size_t>(kSweepWarpsPerCta, budget / per);
    sw = std::min(sw, nsweep5);
    if (sw > 0 && c.sweep_warps_per_cta > 0) sw = std::min(sw, c.sweep_warps_per_cta);
    if (sw > 0) {
      const size_t dyn = 64 + (size_t)sw * per;
      if (dyn + (size_t)D.pcg3_static_smem > (size_t)D.smem_optin) {
        sw = 0;
      } else {
        // raise the kernel's dynamic shared-memory limit to the device maximum: never below what any
        // handle on this device launches it with
        DN_SCUDA(cudaFuncSetAttribute(k53, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      D.smem_optin - D.pcg3_static_smem));
        int occ5 = 0;
        DN_SCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ5, k53, kBlock, dyn));
        sw_blocks_max = std::min(kMaxBlocks, std::max(0, occ5) * D.num_sms);
        if (sw_blocks_max == 0) sw = 0;
        warp_smem = per;
      }
    }
  }
  void *args[] = {&P};
  if (sw > 0) {
    Sweep5 &W = P.s5;
    W.nx = nx;
    W.ny = ny;
    W.n = (int)n;
    W.px = G.px;
    W.py = G.py;
    W.prec = kind;
    W.varcoef = split ? 0 : 1;
    W.aW = a5;
    W.aS = a5 + n;
    W.aN = a5 + 3 * n;
    W.aE = a5 + 4 * n;
    W.cx = -(1.0 / (G.dx * G.dx));
    W.cy = -(1.0 / (G.dy * G.dy));
    W.dinv = P.dinv;
    W.r = P.r;
    W.y = P.y;
    W.z = P.z;
    W.bnd_f = dptr(L.bnd_f);
    W.bnd_b = dptr(L.bnd_b);
    W.wline0 = dptr(L.wline0);
    W.zlast = dptr(L.zlast);
    W.prog_f = P.prog_f;
    W.prog_b = P.prog_b;
    W.nsweep = nsweep5;
    W.sw = sw;
    W.status = status;
    P.warp_smem = (int)warp_smem;
    W.warp_smem = P.warp_smem;
    W.prof = dptr(L.prof);
    const int sweep_ctas = (nsweep5 + sw - 1) / sw;
    blocks = std::max(blocks, sweep_ctas);
    blocks = std::min(blocks, sw_blocks_max);
    if (blocks < sweep_ctas)
      return static_fail(err, err_len, DN_ERR_UNSUPPORTED, "not enough co-resident CTAs for the wavefront");
    DN_SCUDA(cudaLaunchCooperativeKernel(k53, dim3(blocks), dim3(kBlock), args, 64 + (size_t)sw * warp_smem, st));
  } else {
    if ((long long)blocks * (kBlock / 32) < nsweep)
      return static_fail(err, err_len, DN_ERR_UNSUPPORTED, "grid too wide for the co-resident wavefront warps");
    DN_SCUDA(cudaLaunchCooperativeKernel((const void *)k_pcg<5, 0>, dim3(blocks), dim3(kBlock), args, 0, st));
  }
  {
    const dn_status s = static_read(&dev_st, status, sizeof(int), st, err, err_len);
    if (s != DN_OK) return s;
  }
  if (dev_st != kDevOk) return static_device_status(dev_st, err, err_len);
  double out[4];
  {
    const dn_status s = static_read(out, scal + 8, sizeof(out), st, err, err_len);
    if (s != DN_OK) return s;
  }
  k_scatter_compact<<<blocks_for(n), 256, 0, st>>>(x, f_pc);
  DN_SLAUNCH("k_scatter_compact");
  if (!has_dirichlet) {  // remove the mean of the correction (pressure.cpp:317, 338, 361)
    const int nb = 128;
    k_field_sum<<<nb, 256, 0, st>>>(f_pc, 1.0, partials);
    DN_SLAUNCH("k_field_sum");
    k_finish_mean<<<1, 32, 0, st>>>(partials, nb, (double)n, scal);
    DN_SLAUNCH("k_finish_mean");
    k_add_scalar_interior<<<blocks_for(n), 256, 0, st>>>(f_pc, scal);
    DN_SLAUNCH("k_add_scalar_interior");
  }
  {
    const dn_status s = static_bc_pressure(f_pc, G, B, st, err, err_len);
    if (s != DN_OK) return s;
  }
  DN_SCUDA(cudaStreamSynchronize(st));
  if (iterations) *iterations = (int)out[0];
  if (relative_residual) *relative_residual = out[2];
  return DN_OK;
}

}  // extern "C"
