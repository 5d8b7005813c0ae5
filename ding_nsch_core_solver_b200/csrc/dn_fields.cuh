// dn_fields.cuh -- stencil / pointwise kernels of the CHNS step on ghosted Field2D-layout arrays.
//
// Each kernel restates one loop of the reference (file:line cited) with the reference's operand order;
// with --fmad=false these kernels reproduce the reference's doubles bit for bit.  One thread per cell;
// the whole step is HBM/L2 bound and these kernels are a few percent of it (the Krylov solves dominate).
#pragma once

#include "dn_common.cuh"

namespace dn {

// One thread per interior cell, j fastest.  Grids are capped at 2^30 cells (dn_create), so the index math
// stays in 32-bit unsigned arithmetic: a 64-bit division is a long software sequence on the GPU.
#define DN_FOR_INTERIOR(F)                                                          \
  const unsigned _n = (unsigned)(F).nx * (unsigned)(F).ny;                          \
  const unsigned _t = blockIdx.x * blockDim.x + threadIdx.x;                        \
  if (_t >= _n) return;                                                             \
  const int i = (int)(_t / (unsigned)(F).ny), j = (int)(_t - (unsigned)i * (unsigned)(F).ny);

// ------------------------------------------------------------------------------------------------------
// Boundary conditions (operators.cpp:130-289).  The reference fills x-ghost layers for interior j and then
// y-ghost layers for every i; here every ghost cell is computed from interior values in one pass, which
// gives the same value everywhere except the corner cells that are >= 2 cells outside in both directions
// (the reference copies a not-yet-refreshed x-ghost there).  No stencil of the step reads those corners.
// ------------------------------------------------------------------------------------------------------
enum BCKind { kBCScalar = 0, kBCPressure = 1, kBCU = 2, kBCV = 3 };

// u boundary faces, operators.cpp:189-200
__global__ void k_bc_faces_u(Fv f, Grid G, BCSide left, BCSide right) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= f.ny) return;
  if (G.px) {
    f.at(f.nx - 1, j) = f.at(0, j);
  } else {
    f.at(0, j) = (left.type == DN_BC_DIRICHLET) ? left.value : f.at(1, j) + left.value * G.dx;
    f.at(f.nx - 1, j) = (right.type == DN_BC_DIRICHLET) ? right.value : f.at(f.nx - 2, j) + right.value * G.dx;
  }
}
// v boundary faces, operators.cpp:245-256
__global__ void k_bc_faces_v(Fv f, Grid G, BCSide bottom, BCSide top) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= f.nx) return;
  if (G.py) {
    f.at(i, f.ny - 1) = f.at(i, 0);
  } else {
    f.at(i, 0) = (bottom.type == DN_BC_DIRICHLET) ? bottom.value : f.at(i, 1) + bottom.value * G.dy;
    f.at(i, f.ny - 1) = (top.type == DN_BC_DIRICHLET) ? top.value : f.at(i, f.ny - 2) + top.value * G.dy;
  }
}

// x-direction ghost value at (i, j), j interior, i outside [0, nx').
__device__ __forceinline__ double bc_xval(const Fv &f, const Grid &G, int kind, const BCSide &L, const BCSide &R,
                                          int i, int j) {
  const int nx = f.nx;
  if (i >= 0 && i < nx) return f.at(i, j);
  const bool left = i < 0;
  const int g = left ? -i : i - (nx - 1);
  if (G.px) {
    if (kind == kBCU) return left ? f.at(nx - g - 1, j) : f.at(g, j);
    return left ? f.at(nx - g, j) : f.at(g - 1, j);
  }
  if (kind == kBCScalar) return left ? f.at(0, j) : f.at(nx - 1, j);
  const BCSide &b = left ? L : R;
  if (kind == kBCU) {
    const double off = 2.0 * (double)g * b.value * G.dx;
    const double in = left ? f.at(g, j) : f.at(nx - 1 - g, j);
    return (b.type == DN_BC_DIRICHLET) ? 2.0 * b.value - in : in + off;
  }
  // pressure and v: cell-centred in x
  const double off = 2.0 * ((double)g - 0.5) * b.value * G.dx;
  const double in = left ? f.at(g - 1, j) : f.at(nx - g, j);
  return (b.type == DN_BC_DIRICHLET) ? 2.0 * b.value - in : in + off;
}

__global__ void k_bc_ghosts(Fv f, Grid G, int kind, BCSide L, BCSide R, BCSide B, BCSide T) {
  const int gw = f.g, nx = f.nx, ny = f.ny;
  const long long nxg = 2LL * gw * ny;               // x-ghost strips, interior j
  const long long nyg = 2LL * gw * (nx + 2 * gw);    // y-ghost strips, all i
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nxg) {
    const int j = (int)(t % ny);
    const int k = (int)(t / ny);  // 0..2g-1
    const int i = (k < gw) ? -(k + 1) : nx - 1 + (k - gw + 1);
    f.at(i, j) = bc_xval(f, G, kind, L, R, i, j);
    return;
  }
  t -= nxg;
  if (t >= nyg) return;
  const int i = (int)(t % (nx + 2 * gw)) - gw;
  const int k = (int)(t / (nx + 2 * gw));
  const bool bottom = k < gw;
  const int g = bottom ? k + 1 : k - gw + 1;
  const int j = bottom ? -g : ny - 1 + g;
  double val;
  if (G.py) {
    if (kind == kBCV)
      val = bottom ? bc_xval(f, G, kind, L, R, i, ny - g - 1) : bc_xval(f, G, kind, L, R, i, g);
    else
      val = bottom ? bc_xval(f, G, kind, L, R, i, ny - g) : bc_xval(f, G, kind, L, R, i, g - 1);
  } else if (kind == kBCScalar) {
    val = bottom ? bc_xval(f, G, kind, L, R, i, 0) : bc_xval(f, G, kind, L, R, i, ny - 1);
  } else {
    const BCSide &b = bottom ? B : T;
    if (kind == kBCV) {
      const double off = 2.0 * (double)g * b.value * G.dy;
      const double in = bottom ? bc_xval(f, G, kind, L, R, i, g) : bc_xval(f, G, kind, L, R, i, ny - 1 - g);
      val = (b.type == DN_BC_DIRICHLET) ? 2.0 * b.value - in : in + off;
    } else {
      const double off = 2.0 * ((double)g - 0.5) * b.value * G.dy;
      const double in = bottom ? bc_xval(f, G, kind, L, R, i, g - 1) : bc_xval(f, G, kind, L, R, i, ny - g);
      val = (b.type == DN_BC_DIRICHLET) ? 2.0 * b.value - in : in + off;
    }
  }
  f.at(i, j) = val;
}

// ------------------------------------------------------------------------------------------------------
// Face / corner interpolation (operators.cpp:328-398)
// ------------------------------------------------------------------------------------------------------
__device__ __forceinline__ double xface(const Fv &f, const Grid &G, int i, int j) {
  if (i <= 0) return G.px ? 0.5 * (f.at(G.nx - 1, j) + f.at(0, j)) : f.at(0, j);
  if (i >= G.nx) return G.px ? 0.5 * (f.at(G.nx - 1, j) + f.at(0, j)) : f.at(G.nx - 1, j);
  return 0.5 * (f.at(i - 1, j) + f.at(i, j));
}
__device__ __forceinline__ double yface(const Fv &f, const Grid &G, int i, int j) {
  if (j <= 0) return G.py ? 0.5 * (f.at(i, G.ny - 1) + f.at(i, 0)) : f.at(i, 0);
  if (j >= G.ny) return G.py ? 0.5 * (f.at(i, G.ny - 1) + f.at(i, 0)) : f.at(i, G.ny - 1);
  return 0.5 * (f.at(i, j - 1) + f.at(i, j));
}
__device__ __forceinline__ double corner(const Fv &f, int i, int j) {
  return 0.25 * (f.at(i, j) + f.at(i - 1, j) + f.at(i, j - 1) + f.at(i - 1, j - 1));
}
__device__ __forceinline__ double lapc(const Fv &f, const Grid &G, int i, int j) {
  return (f.at(i + 1, j) - 2.0 * f.at(i, j) + f.at(i - 1, j)) / (G.dx * G.dx) +
         (f.at(i, j + 1) - 2.0 * f.at(i, j) + f.at(i, j - 1)) / (G.dy * G.dy);
}
__device__ __forceinline__ double gfx(const Fv &f, const Grid &G, int i, int j) {
  return (f.at(i, j) - f.at(i - 1, j)) / G.dx;
}
__device__ __forceinline__ double gfy(const Fv &f, const Grid &G, int i, int j) {
  return (f.at(i, j) - f.at(i, j - 1)) / G.dy;
}
__device__ __forceinline__ double div_cell(const Fv &u, const Fv &v, const Grid &G, int i, int j) {
  return (u.at(i + 1, j) - u.at(i, j)) / G.dx + (v.at(i, j + 1) - v.at(i, j)) / G.dy;
}
__device__ __forceinline__ double sq(double v) { return v * v; }

// ------------------------------------------------------------------------------------------------------
// Pointwise / stencil kernels
// ------------------------------------------------------------------------------------------------------
__global__ void k_copy(double *dst, const double *src, long long n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dst[t] = src[t];
}
__global__ void k_fill(double *dst, double v, long long n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dst[t] = v;
}
__global__ void k_copy_interior(Fv dst, Fv src) {
  DN_FOR_INTERIOR(dst);
  dst.at(i, j) = src.at(i, j);
}
__global__ void k_add_scalar_interior(Fv f, const double *sub) {
  DN_FOR_INTERIOR(f);
  f.at(i, j) -= *sub;
}

// update_materials_from_phase, phase_field.cpp:57-66
__global__ void k_materials(Fv c, Fv rho, Fv eta, double dr, double vr) {
  DN_FOR_INTERIOR(c);
  const double cc = c.at(i, j);
  rho.at(i, j) = cc + (1.0 - cc) * dr;
  eta.at(i, j) = cc + (1.0 - cc) * vr;
}
// update_midpoint_materials, phase_field.cpp:70-79
__global__ void k_midpoint(Fv rp, Fv r, Fv ep, Fv e, Fv rm, Fv em) {
  DN_FOR_INTERIOR(rm);
  rm.at(i, j) = 0.5 * (rp.at(i, j) + r.at(i, j));
  em.at(i, j) = 0.5 * (ep.at(i, j) + e.at(i, j));
}
// update_chemical_potential, phase_field.cpp:97-109 (input already carries its scalar BC ghosts)
__global__ void k_chem(Fv c, Fv mu, Grid G, double cn) {
  DN_FOR_INTERIOR(mu);
  const double alpha = 6.0 * 1.4142135623730950488;  // 6*sqrt(2), correctly rounded like std::sqrt
  const double cc = c.at(i, j);
  const double dw = 0.5 * cc * (1.0 - cc) * (1.0 - 2.0 * cc);
  mu.at(i, j) = alpha * (dw / cn - cn * lapc(c, G, i, j));
}
// mobility and laplacian, phase_field.cpp:367-372
__global__ void k_mob_lap(Fv c, Fv mob, Fv lap, Grid G) {
  DN_FOR_INTERIOR(mob);
  const double cc = c.at(i, j);
  mob.at(i, j) = fmax(0.0, cc * (1.0 - cc));
  lap.at(i, j) = lapc(c, G, i, j);
}
__global__ void k_lap(Fv in, Fv out, Grid G) {
  DN_FOR_INTERIOR(out);
  out.at(i, j) = lapc(in, G, i, j);
}

// weno5_left, phase_field.cpp:144-157
__device__ __forceinline__ double weno5_left(double v1, double v2, double v3, double v4, double v5) {
  const double eps = 1.0e-6;
  const double q0 = (2.0 * v1 - 7.0 * v2 + 11.0 * v3) / 6.0;
  const double q1 = (-v2 + 5.0 * v3 + 2.0 * v4) / 6.0;
  const double q2 = (2.0 * v3 + 5.0 * v4 - v5) / 6.0;
  const double b0 = 13.0 / 12.0 * sq(v1 - 2.0 * v2 + v3) + 0.25 * sq(v1 - 4.0 * v2 + 3.0 * v3);
  const double b1 = 13.0 / 12.0 * sq(v2 - 2.0 * v3 + v4) + 0.25 * sq(v2 - v4);
  const double b2 = 13.0 / 12.0 * sq(v3 - 2.0 * v4 + v5) + 0.25 * sq(3.0 * v3 - 4.0 * v4 + v5);
  const double a0 = 0.1 / sq(eps + b0);
  const double a1 = 0.6 / sq(eps + b1);
  const double a2 = 0.3 / sq(eps + b2);
  const double sum = a0 + a1 + a2;
  return (a0 * q0 + a1 * q1 + a2 * q2) / sum;
}

// advective face fluxes with WENO5 face values, phase_field.cpp:163-177, 288-300
__global__ void k_adv_flux_x(Fv c, Fv ua, Fv fx) {
  DN_FOR_INTERIOR(fx);
  const double uu = ua.at(i, j);
  const double face = (uu >= 0.0) ? weno5_left(c.at(i - 3, j), c.at(i - 2, j), c.at(i - 1, j), c.at(i, j), c.at(i + 1, j))
                                  : weno5_left(c.at(i + 2, j), c.at(i + 1, j), c.at(i, j), c.at(i - 1, j), c.at(i - 2, j));
  fx.at(i, j) = uu * face;
}
__global__ void k_adv_flux_y(Fv c, Fv va, Fv fy) {
  DN_FOR_INTERIOR(fy);
  const double vv = va.at(i, j);
  const double face = (vv >= 0.0) ? weno5_left(c.at(i, j - 3), c.at(i, j - 2), c.at(i, j - 1), c.at(i, j), c.at(i, j + 1))
                                  : weno5_left(c.at(i, j + 2), c.at(i, j + 1), c.at(i, j), c.at(i, j - 1), c.at(i, j - 2));
  fy.at(i, j) = vv * face;
}
// diffusive face fluxes, phase_field.cpp:315-341
__global__ void k_diff_flux_x(Fv mu, Fv mob, Fv fx, Grid G) {
  DN_FOR_INTERIOR(fx);
  const double m = xface(mob, G, i, j);
  fx.at(i, j) = m * gfx(mu, G, i, j);
}
__global__ void k_diff_flux_y(Fv mu, Fv mob, Fv fy, Grid G) {
  DN_FOR_INTERIOR(fy);
  const double m = yface(mob, G, i, j);
  fy.at(i, j) = m * gfy(mu, G, i, j);
}
// adv_rhs (phase_field.cpp:304-309) and diffusion divergence (:345-350)
__global__ void k_flux_div(Fv fx, Fv fy, Fv out, Grid G, int negate) {
  DN_FOR_INTERIOR(out);
  if (negate)
    out.at(i, j) = -(fx.at(i + 1, j) - fx.at(i, j)) / G.dx - (fy.at(i, j + 1) - fy.at(i, j)) / G.dy;
  else
    out.at(i, j) = (fx.at(i + 1, j) - fx.at(i, j)) / G.dx + (fy.at(i, j + 1) - fy.at(i, j)) / G.dy;
}
// explicit operator, phase_field.cpp:386-394
__global__ void k_explicit(Fv ddiv, Fv lap, Fv bih, Fv arhs, Fv E, double a1, double a2, double pe) {
  DN_FOR_INTERIOR(E);
  E.at(i, j) = ddiv.at(i, j) / pe - (a1 * lap.at(i, j) - a2 * bih.at(i, j)) / pe + arhs.at(i, j);
}
// BDF1/BDF2 + AB2 right-hand side, phase_field.cpp:679-690; written straight into the compact Krylov rhs
__global__ void k_ch_rhs(Fv cp, Fv cp2, Fv E, Fv Ep, double *rhs, double *x0, Fv c, int step, double dt) {
  DN_FOR_INTERIOR(E);
  double v;
  if (step == 0)
    v = cp.at(i, j) / dt + E.at(i, j);
  else
    v = (4.0 * cp.at(i, j) - cp2.at(i, j)) / (2.0 * dt) + 2.0 * E.at(i, j) - Ep.at(i, j);
  const long long r = (long long)i * E.ny + j;
  rhs[r] = v;
  x0[r] = c.at(i, j);
}
// ------------------------------------------------------------------------------------------------------
// Fused CH explicit operator + BDF right-hand side (build_phase_explicit_operator, phase_field.cpp:354-396,
// with the rhs of solve_cahn_hilliard_semi_implicit, :679-690): one pass over a TI x TJ tile of cells.
// The tile of c with a 3-cell halo is staged in shared memory; the Laplacian and the chemical potential
// on the tile plus a 1-cell halo, then the advective (WENO5) and diffusive face fluxes of the tile, are
// computed there, and each cell writes E, the Krylov right-hand side and the initial iterate.  The result
// is bit-for-bit that of the separate kernels (k_mob_lap, k_lap, k_chem, k_adv_flux_*, k_diff_flux_*,
// k_flux_div, k_explicit, k_ch_rhs) with their boundary passes in between:
//  - a halo value of a scalar field (lap, mu) outside the domain is its ghost under the scalar BC: in a
//    wall direction the boundary cell's value (the position is clamped), in a periodic direction the value
//    at the ghost position computed from c's periodic ghosts, whose operands equal those at the wrapped
//    interior position;
//  - a boundary face flux on a wall side is replaced as the face BC of a u (v) array replaces it
//    (k_bc_faces_u/v: the Dirichlet value, or the next interior face's flux plus value * dx); in a periodic
//    direction face nx is computed and equals face 0, whose operands it repeats.
// Algorithmic bytes per cell: reads c, u, v, c_prev, c_prev2, E_prev; writes E, rhs, x0 (72 B).
// ------------------------------------------------------------------------------------------------------
template <int TI, int TJ>
__global__ void __launch_bounds__(256) k_ch_explicit_rhs(Fv c, Fv u, Fv v, Fv cp, Fv cp2, Fv Ep, Fv E,
                                                         double *rhs, double *x0, Grid G, BCSide uL, BCSide uR,
                                                         BCSide vB, BCSide vT, double cn, double a1, double a2,
                                                         double pe, int step, double dt) {
  constexpr int CI = TI + 6, CJ = TJ + 6;  // c with a 3-cell halo
  constexpr int HI = TI + 2, HJ = TJ + 2;  // lap and mu with a 1-cell halo
  __shared__ double cs[CI * CJ];
  __shared__ double laps[HI * HJ], mus[HI * HJ];
  __shared__ double fax[(TI + 1) * TJ], fdx[(TI + 1) * TJ];  // x faces i0 .. i0+TI
  __shared__ double fay[TI * (TJ + 1)], fdy[TI * (TJ + 1)];  // y faces j0 .. j0+TJ
  const int nx = G.nx, ny = G.ny;
  const int i0 = blockIdx.y * TI, j0 = blockIdx.x * TJ;
  const int tid = threadIdx.x, nt = blockDim.x;
  auto C = [&](int gi, int gj) -> double { return cs[(gi - i0 + 3) * CJ + (gj - j0 + 3)]; };
  // 1. c over the tile and its 3-cell halo (the ghost layers hold the BC values)
  for (int e = tid; e < CI * CJ; e += nt) {
    const int li = e / CJ, lj = e - (e / CJ) * CJ;
    const int gi = i0 - 3 + li, gj = j0 - 3 + lj;
    cs[e] = (gi >= -3 && gi < nx + 3 && gj >= -3 && gj < ny + 3) ? c.at(gi, gj) : 0.0;
  }
  __syncthreads();
  // 2. lap (lapc) and mu (k_chem) on the tile and its 1-cell halo, corners excluded
  const double alpha = 6.0 * 1.4142135623730950488;
  for (int e = tid; e < HI * HJ; e += nt) {
    const int li = e / HJ, lj = e - (e / HJ) * HJ;
    if ((li == 0 || li == HI - 1) && (lj == 0 || lj == HJ - 1)) continue;
    int gi = i0 - 1 + li, gj = j0 - 1 + lj;
    if (gi > nx || gj > ny) continue;  // beyond the last ghost row / column a tile covers
    if (!G.px) gi = min(max(gi, 0), nx - 1);
    if (!G.py) gj = min(max(gj, 0), ny - 1);
    const double lap = (C(gi + 1, gj) - 2.0 * C(gi, gj) + C(gi - 1, gj)) / (G.dx * G.dx) +
                       (C(gi, gj + 1) - 2.0 * C(gi, gj) + C(gi, gj - 1)) / (G.dy * G.dy);
    const double cc = C(gi, gj);
    const double dw = 0.5 * cc * (1.0 - cc) * (1.0 - 2.0 * cc);
    laps[e] = lap;
    mus[e] = alpha * (dw / cn - cn * lap);
  }
  __syncthreads();
  auto LAP = [&](int gi, int gj) -> double { return laps[(gi - i0 + 1) * HJ + (gj - j0 + 1)]; };
  auto MU = [&](int gi, int gj) -> double { return mus[(gi - i0 + 1) * HJ + (gj - j0 + 1)]; };
  auto mob = [](double cc) { return fmax(0.0, cc * (1.0 - cc)); };
  // 3. face fluxes (k_adv_flux_x/y, k_diff_flux_x/y)
  for (int e = tid; e < (TI + 1) * TJ; e += nt) {
    const int fi = e / TJ, fj = e - (e / TJ) * TJ;
    const int gi = i0 + fi, gj = j0 + fj;
    if (gi > nx || gj >= ny) continue;
    const double uu = u.at(gi, gj);
    const double face = (uu >= 0.0) ? weno5_left(C(gi - 3, gj), C(gi - 2, gj), C(gi - 1, gj), C(gi, gj), C(gi + 1, gj))
                                    : weno5_left(C(gi + 2, gj), C(gi + 1, gj), C(gi, gj), C(gi - 1, gj), C(gi - 2, gj));
    fax[e] = uu * face;
    // xface(mob): interior faces and, periodic, faces 0 and nx average the two adjacent cells (the halo of c
    // holds the periodic neighbour); wall boundary faces are replaced below
    const double m = 0.5 * (mob(C(gi - 1, gj)) + mob(C(gi, gj)));
    fdx[e] = m * ((MU(gi, gj) - MU(gi - 1, gj)) / G.dx);
  }
  for (int e = tid; e < TI * (TJ + 1); e += nt) {
    const int fi = e / (TJ + 1), fj = e - (e / (TJ + 1)) * (TJ + 1);
    const int gi = i0 + fi, gj = j0 + fj;
    if (gi >= nx || gj > ny) continue;
    const double vv = v.at(gi, gj);
    const double face = (vv >= 0.0) ? weno5_left(C(gi, gj - 3), C(gi, gj - 2), C(gi, gj - 1), C(gi, gj), C(gi, gj + 1))
                                    : weno5_left(C(gi, gj + 2), C(gi, gj + 1), C(gi, gj), C(gi, gj - 1), C(gi, gj - 2));
    fay[e] = vv * face;
    const double m = 0.5 * (mob(C(gi, gj - 1)) + mob(C(gi, gj)));
    fdy[e] = m * ((MU(gi, gj) - MU(gi, gj - 1)) / G.dy);
  }
  __syncthreads();
  // wall boundary faces (k_bc_faces_u / k_bc_faces_v on the flux arrays)
  if (!G.px) {
    for (int fj = tid; fj < TJ; fj += nt) {
      const int gj = j0 + fj;
      if (gj >= ny) continue;
      if (i0 == 0) {
        const int e = fj, e1 = TJ + fj;  // faces 0 and 1
        fax[e] = (uL.type == DN_BC_DIRICHLET) ? uL.value : fax[e1] + uL.value * G.dx;
        fdx[e] = (uL.type == DN_BC_DIRICHLET) ? uL.value : fdx[e1] + uL.value * G.dx;
      }
      if (nx >= i0 && nx <= i0 + TI) {
        const int e = (nx - i0) * TJ + fj, e1 = (nx - 1 - i0) * TJ + fj;  // faces nx and nx-1
        fax[e] = (uR.type == DN_BC_DIRICHLET) ? uR.value : fax[e1] + uR.value * G.dx;
        fdx[e] = (uR.type == DN_BC_DIRICHLET) ? uR.value : fdx[e1] + uR.value * G.dx;
      }
    }
  }
  if (!G.py) {
    for (int fi = tid; fi < TI; fi += nt) {
      const int gi = i0 + fi;
      if (gi >= nx) continue;
      if (j0 == 0) {
        const int e = fi * (TJ + 1), e1 = fi * (TJ + 1) + 1;  // faces 0 and 1
        fay[e] = (vB.type == DN_BC_DIRICHLET) ? vB.value : fay[e1] + vB.value * G.dy;
        fdy[e] = (vB.type == DN_BC_DIRICHLET) ? vB.value : fdy[e1] + vB.value * G.dy;
      }
      if (ny >= j0 && ny <= j0 + TJ) {
        const int e = fi * (TJ + 1) + (ny - j0), e1 = fi * (TJ + 1) + (ny - 1 - j0);  // faces ny and ny-1
        fay[e] = (vT.type == DN_BC_DIRICHLET) ? vT.value : fay[e1] + vT.value * G.dy;
        fdy[e] = (vT.type == DN_BC_DIRICHLET) ? vT.value : fdy[e1] + vT.value * G.dy;
      }
    }
  }
  __syncthreads();
  // 4. cells: divergences, the explicit operator and the BDF right-hand side
  for (int e = tid; e < TI * TJ; e += nt) {
    const int li = e / TJ, lj = e - (e / TJ) * TJ;
    const int gi = i0 + li, gj = j0 + lj;
    if (gi >= nx || gj >= ny) continue;
    const double axp = fax[(li + 1) * TJ + lj], axm = fax[li * TJ + lj];
    const double ayp = fay[li * (TJ + 1) + lj + 1], aym = fay[li * (TJ + 1) + lj];
    const double dxp = fdx[(li + 1) * TJ + lj], dxm = fdx[li * TJ + lj];
    const double dyp = fdy[li * (TJ + 1) + lj + 1], dym = fdy[li * (TJ + 1) + lj];
    const double arhs = -(axp - axm) / G.dx - (ayp - aym) / G.dy;
    const double ddiv = (dxp - dxm) / G.dx + (dyp - dym) / G.dy;
    const double bih = (LAP(gi + 1, gj) - 2.0 * LAP(gi, gj) + LAP(gi - 1, gj)) / (G.dx * G.dx) +
                       (LAP(gi, gj + 1) - 2.0 * LAP(gi, gj) + LAP(gi, gj - 1)) / (G.dy * G.dy);
    const double en = ddiv / pe - (a1 * LAP(gi, gj) - a2 * bih) / pe + arhs;
    E.at(gi, gj) = en;
    double val;
    if (step == 0)
      val = cp.at(gi, gj) / dt + en;
    else
      val = (4.0 * cp.at(gi, gj) - cp2.at(gi, gj)) / (2.0 * dt) + 2.0 * en - Ep.at(gi, gj);
    const long long r = (long long)gi * ny + gj;
    rhs[r] = val;
    x0[r] = C(gi, gj);
  }
}

__global__ void k_scatter_compact(const double *x, Fv f) {
  DN_FOR_INTERIOR(f);
  f.at(i, j) = x[(long long)i * f.ny + j];
}
__global__ void k_gather_compact(Fv f, double *x) {
  DN_FOR_INTERIOR(f);
  x[(long long)i * f.ny + j] = f.at(i, j);
}

// c_mid, phase_field.cpp:185-191
__global__ void k_cmid(Fv co, Fv cn_, Fv cm) {
  DN_FOR_INTERIOR(cm);
  cm.at(i, j) = 0.5 * (co.at(i, j) + cn_.at(i, j));
}
// face surface-tension forces, phase_field.cpp:206-226
__global__ void k_sf_u(Fv mm, Fv cm, Fv fxu, Grid G, double scale) {
  DN_FOR_INTERIOR(fxu);
  const int nx = G.nx;
  const double mf = (i <= 0) ? 0.5 * (mm.at(nx - 1, j) + mm.at(0, j))
                             : (i >= nx ? 0.5 * (mm.at(nx - 1, j) + mm.at(0, j)) : 0.5 * (mm.at(i - 1, j) + mm.at(i, j)));
  fxu.at(i, j) = scale * mf * gfx(cm, G, i, j);
}
__global__ void k_sf_v(Fv mm, Fv cm, Fv fyv, Grid G, double scale) {
  DN_FOR_INTERIOR(fyv);
  const int ny = G.ny;
  const double mf = (j <= 0) ? 0.5 * (mm.at(i, ny - 1) + mm.at(i, 0))
                             : (j >= ny ? 0.5 * (mm.at(i, ny - 1) + mm.at(i, 0)) : 0.5 * (mm.at(i, j - 1) + mm.at(i, j)));
  fyv.at(i, j) = scale * mf * gfy(cm, G, i, j);
}
// cell surface-tension forces, phase_field.cpp:197-202
__global__ void k_sf_cell(Fv mm, Fv cm, Fv fxc, Fv fyc, Grid G, double scale) {
  DN_FOR_INTERIOR(fxc);
  fxc.at(i, j) = scale * mm.at(i, j) * ((cm.at(i + 1, j) - cm.at(i - 1, j)) / (2.0 * G.dx));
  fyc.at(i, j) = scale * mm.at(i, j) * ((cm.at(i, j + 1) - cm.at(i, j - 1)) / (2.0 * G.dy));
}
// Fused surface force (update_surface_tension_force, phase_field.cpp:179-226): c_mid = (c_old + c_new) / 2
// and its chemical potential mu_mid on a TI x TJ tile with halos in shared memory, then the cell forces
// (k_sf_cell) and the face forces (k_sf_u / k_sf_v) of the tile.  Bit-for-bit the separate kernels with
// their boundary passes: c_mid at a ghost position is the half sum of the two ghost values, which is the
// scalar BC's ghost of c_mid (clamp or periodic copy); mu_mid at a halo position outside a wall side is the
// boundary cell's value (clamped), in a periodic direction the value computed at the ghost position.  The
// wall boundary faces written here are replaced by the caller's face BC pass, as before.
// Algorithmic bytes per cell: reads c_old, c_new; writes the two cell forces and the two face forces (48 B).
template <int TI, int TJ>
__global__ void __launch_bounds__(256) k_surface_force(Fv co, Fv cn_, Fv fxc, Fv fyc, Fv fxu, Fv fyv, Grid G,
                                                       double cn, double scale) {
  constexpr int MI = TI + 4, MJ = TJ + 4;  // c_mid with a 2-cell halo
  constexpr int HI = TI + 2, HJ = TJ + 2;  // mu_mid with a 1-cell halo
  __shared__ double cms[MI * MJ], mms[HI * HJ];
  const int nx = G.nx, ny = G.ny;
  const int i0 = blockIdx.y * TI, j0 = blockIdx.x * TJ;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < MI * MJ; e += nt) {
    const int li = e / MJ, lj = e - (e / MJ) * MJ;
    const int gi = i0 - 2 + li, gj = j0 - 2 + lj;
    cms[e] = (gi < nx + 3 && gj < ny + 3) ? 0.5 * (co.at(gi, gj) + cn_.at(gi, gj)) : 0.0;
  }
  __syncthreads();
  auto CM = [&](int gi, int gj) -> double { return cms[(gi - i0 + 2) * MJ + (gj - j0 + 2)]; };
  const double alpha = 6.0 * 1.4142135623730950488;
  for (int e = tid; e < HI * HJ; e += nt) {
    const int li = e / HJ, lj = e - (e / HJ) * HJ;
    if ((li == 0 || li == HI - 1) && (lj == 0 || lj == HJ - 1)) continue;
    int gi = i0 - 1 + li, gj = j0 - 1 + lj;
    if (gi > nx || gj > ny) continue;
    if (!G.px) gi = min(max(gi, 0), nx - 1);
    if (!G.py) gj = min(max(gj, 0), ny - 1);
    const double lap = (CM(gi + 1, gj) - 2.0 * CM(gi, gj) + CM(gi - 1, gj)) / (G.dx * G.dx) +
                       (CM(gi, gj + 1) - 2.0 * CM(gi, gj) + CM(gi, gj - 1)) / (G.dy * G.dy);
    const double cc = CM(gi, gj);
    const double dw = 0.5 * cc * (1.0 - cc) * (1.0 - 2.0 * cc);
    mms[e] = alpha * (dw / cn - cn * lap);
  }
  __syncthreads();
  auto MM = [&](int gi, int gj) -> double { return mms[(gi - i0 + 1) * HJ + (gj - j0 + 1)]; };
  for (int e = tid; e < TI * TJ; e += nt) {
    const int li = e / TJ, lj = e - (e / TJ) * TJ;
    const int gi = i0 + li, gj = j0 + lj;
    if (gi >= nx || gj >= ny) continue;
    fxc.at(gi, gj) = scale * MM(gi, gj) * ((CM(gi + 1, gj) - CM(gi - 1, gj)) / (2.0 * G.dx));
    fyc.at(gi, gj) = scale * MM(gi, gj) * ((CM(gi, gj + 1) - CM(gi, gj - 1)) / (2.0 * G.dy));
  }
  // faces i0 .. i0+TI-1 of this tile, and face nx in the last tile
  for (int e = tid; e < (TI + 1) * TJ; e += nt) {
    const int fi = e / TJ, fj = e - (e / TJ) * TJ;
    const int gi = i0 + fi, gj = j0 + fj;
    if (gj >= ny || gi > nx || (fi == TI && gi != nx)) continue;
    const double mf = 0.5 * (MM(gi - 1, gj) + MM(gi, gj));
    fxu.at(gi, gj) = scale * mf * ((CM(gi, gj) - CM(gi - 1, gj)) / G.dx);
  }
  for (int e = tid; e < TI * (TJ + 1); e += nt) {
    const int fi = e / (TJ + 1), fj = e - (e / (TJ + 1)) * (TJ + 1);
    const int gi = i0 + fi, gj = j0 + fj;
    if (gi >= nx || gj > ny || (fj == TJ && gj != ny)) continue;
    const double mf = 0.5 * (MM(gi, gj - 1) + MM(gi, gj));
    fyv.at(gi, gj) = scale * mf * ((CM(gi, gj) - CM(gi, gj - 1)) / G.dy);
  }
}
// smoothing pass, phase_field.cpp:234-249
__global__ void k_smooth(Fv f, Fv out, double cw, double nw) {
  DN_FOR_INTERIOR(out);
  out.at(i, j) = cw * f.at(i, j) + nw * (f.at(i - 1, j) + f.at(i + 1, j) + f.at(i, j - 1) + f.at(i, j + 1));
}

// centred momentum convection, momentum.cpp:55-85
__global__ void k_mom_flux_u(Fv u, Fv v, Fv hu, Grid G) {
  DN_FOR_INTERIOR(hu);
  const double uf = u.at(i, j);
  const double dudx = (u.at(i + 1, j) - u.at(i - 1, j)) / (2.0 * G.dx);
  const double dudy = (u.at(i, j + 1) - u.at(i, j - 1)) / (2.0 * G.dy);
  const double vf = 0.25 * (v.at(i - 1, j) + v.at(i, j) + v.at(i - 1, j + 1) + v.at(i, j + 1));
  hu.at(i, j) = uf * dudx + vf * dudy;
}
__global__ void k_mom_flux_v(Fv u, Fv v, Fv hv, Grid G) {
  DN_FOR_INTERIOR(hv);
  const double vf = v.at(i, j);
  const double dvdx = (v.at(i + 1, j) - v.at(i - 1, j)) / (2.0 * G.dx);
  const double dvdy = (v.at(i, j + 1) - v.at(i, j - 1)) / (2.0 * G.dy);
  const double uf = 0.25 * (u.at(i, j - 1) + u.at(i, j) + u.at(i + 1, j - 1) + u.at(i + 1, j));
  hv.at(i, j) = uf * dvdx + vf * dvdy;
}

// viscous stress divergence, momentum.cpp:91-155
__device__ __forceinline__ double visc_u(const Fv &u, const Fv &v, const Fv &eta, const Grid &G, int i, int j) {
  const double eta_e = xface(eta, G, i + 1, j), eta_w = xface(eta, G, i, j);
  const double dudx_e = (u.at(i + 1, j) - u.at(i, j)) / G.dx;
  const double dudx_w = (u.at(i, j) - u.at(i - 1, j)) / G.dx;
  const double normal = (2.0 * eta_e * dudx_e - 2.0 * eta_w * dudx_w) / G.dx;
  const double eta_n = corner(eta, i, j + 1), eta_s = corner(eta, i, j);
  const double dudy_n = (u.at(i, j + 1) - u.at(i, j)) / G.dy;
  const double dudy_s = (u.at(i, j) - u.at(i, j - 1)) / G.dy;
  const double shear_self = (eta_n * dudy_n - eta_s * dudy_s) / G.dy;
  const double self = normal + shear_self;
  const double dvdx_n = (v.at(i, j + 1) - v.at(i - 1, j + 1)) / G.dx;
  const double dvdx_s = (v.at(i, j) - v.at(i - 1, j)) / G.dx;
  const double cross = (eta_n * dvdx_n - eta_s * dvdx_s) / G.dy;
  return self + cross;
}
__device__ __forceinline__ double visc_v(const Fv &u, const Fv &v, const Fv &eta, const Grid &G, int i, int j) {
  const double eta_e = corner(eta, i + 1, j), eta_w = corner(eta, i, j);
  const double dvdx_e = (v.at(i + 1, j) - v.at(i, j)) / G.dx;
  const double dvdx_w = (v.at(i, j) - v.at(i - 1, j)) / G.dx;
  const double shear_self = (eta_e * dvdx_e - eta_w * dvdx_w) / G.dx;
  const double eta_n = yface(eta, G, i, j + 1), eta_s = yface(eta, G, i, j);
  const double dvdy_n = (v.at(i, j + 1) - v.at(i, j)) / G.dy;
  const double dvdy_s = (v.at(i, j) - v.at(i, j - 1)) / G.dy;
  const double normal = (2.0 * eta_n * dvdy_n - 2.0 * eta_s * dvdy_s) / G.dy;
  const double self = shear_self + normal;
  const double dudy_e = (u.at(i + 1, j) - u.at(i + 1, j - 1)) / G.dy;
  const double dudy_w = (u.at(i, j) - u.at(i, j - 1)) / G.dy;
  const double cross = (eta_e * dudy_e - eta_w * dudy_w) / G.dx;
  return self + cross;
}

// split extrapolation p~ = 2p^n - p^{n-1} (p^n at step 0), operators.cpp:413-422
__global__ void k_p_ext(Fv p, Fv pp, Fv pe, int first) {
  DN_FOR_INTERIOR(pe);
  pe.at(i, j) = first ? p.at(i, j) : (2.0 * p.at(i, j) - pp.at(i, j));
}

// velocity correction, operators.cpp:490-516
__global__ void k_correct_u(Fv u, Fv us, Fv rm, Fv pc, Fv pe, Grid G, int split, double rho_ref, double dt) {
  DN_FOR_INTERIOR(u);
  const double se = split ? (1.0 / xface(rm, G, i, j) - 1.0 / rho_ref) * gfx(pe, G, i, j) : 0.0;
  const double si = split ? gfx(pc, G, i, j) / rho_ref : gfx(pc, G, i, j) / xface(rm, G, i, j);
  u.at(i, j) = us.at(i, j) - dt * (si + se);
}
__global__ void k_correct_v(Fv v, Fv vs, Fv rm, Fv pc, Fv pe, Grid G, int split, double rho_ref, double dt) {
  DN_FOR_INTERIOR(v);
  const double se = split ? (1.0 / yface(rm, G, i, j) - 1.0 / rho_ref) * gfy(pe, G, i, j) : 0.0;
  const double si = split ? gfy(pc, G, i, j) / rho_ref : gfy(pc, G, i, j) / yface(rm, G, i, j);
  v.at(i, j) = vs.at(i, j) - dt * (si + se);
}

// ------------------------------------------------------------------------------------------------------
// Reductions used outside the Krylov kernels (two-stage, deterministic)
// ------------------------------------------------------------------------------------------------------
enum RedOp { kRedSum = 0, kRedMax = 1, kRedMin = 2 };

// Stage 1: per-block partials of up to 4 interior reductions of a cell field (value index selects the
// quantity).  Used for means and the diagnostics.
__device__ __forceinline__ double red_identity(int op) { return op == kRedSum ? 0.0 : (op == kRedMax ? -INFINITY : INFINITY); }
__device__ __forceinline__ double red_combine(int op, double a, double b) {
  return op == kRedSum ? a + b : (op == kRedMax ? fmax(a, b) : fmin(a, b));
}

__global__ void k_reduce_final(const double *partials, int nparts, int nvals, const int *ops, double *out) {
  // one warp per value
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (w >= nvals) return;
  const int op = ops[w];
  double s = red_identity(op);
  for (int b = lane; b < nparts; b += 32) s = red_combine(op, s, partials[(size_t)b * nvals + w]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s = red_combine(op, s, __shfl_xor_sync(0xffffffffu, s, o));
  if (lane == 0) out[w] = s;
}

// Interior sum of a field (for subtract_mean, operators.cpp:447-460, and compute_mass, diagnostics.cpp:24-32).
__global__ void k_field_sum(Fv f, double scale, double *partials) {
  __shared__ double sh[8 * 32];
  const long long n = (long long)f.nx * f.ny;
  double v[1] = {0.0};
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / f.ny), j = (int)(t % f.ny);
    v[0] += f.at(i, j) * scale;
  }
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}
// Jacobi pressure iteration (solve_pressure_correction_jacobi, pressure.cpp:250-300): one sweep
// xn = x + (b - A x) / |diag| over the 5-point system, each row's A x summed in ascending column order (the
// CSR order), and the block maxima of |b - A x|.  Skips when `done` is set, so batches of launches past
// convergence do nothing.
__global__ void k_jacobi_sweep(const double *a, int n, int nx, int ny, int px, int py, const double *rhs,
                               const double *x, double *xn, double *bmax, const unsigned int *done, int *status) {
  __shared__ double sh[32];
  if (*(volatile const unsigned int *)done) return;
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double res = 0.0;
  if (r < n) {
    const int i = (int)(r / ny), j = (int)(r % ny);
    // neighbours W, S, C, N, E with periodic wraps, sorted by column
    long long col[5];
    double val[5];
    int cnt = 0;
    const int di[5] = {-1, 0, 0, 0, 1}, dj[5] = {0, -1, 0, 1, 0};
    for (int s = 0; s < 5; ++s) {
      const double v = a[(size_t)s * n + r];
      if (v == 0.0) continue;
      int ii = i + di[s], jj = j + dj[s];
      if (ii < 0 || ii >= nx) ii = (ii + nx) % nx;  // a nonzero entry across the boundary is periodic
      if (jj < 0 || jj >= ny) jj = (jj + ny) % ny;
      const long long c = (long long)ii * ny + jj;
      int p = cnt++;
      while (p > 0 && col[p - 1] > c) {
        col[p] = col[p - 1];
        val[p] = val[p - 1];
        --p;
      }
      col[p] = c;
      val[p] = v;
    }
    double diag = 0.0, ax = 0.0;
    for (int p = 0; p < cnt; ++p) {
      ax += val[p] * x[col[p]];
      if (col[p] == r) diag = val[p];
    }
    const double rr = rhs[r] - ax;
    if (!isfinite(rr) || !isfinite(diag) || fabs(diag) < 1.0e-30) atomicCAS(status, kDevOk, kDevJacobiDiverged);
    xn[r] = x[r] + 1.0 * rr / fmax(fabs(diag), 1.0e-30);
    res = fabs(rr);
  }
  res = warp_max(res);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = res;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    v = warp_max(v);
    if (threadIdx.x == 0) bmax[blockIdx.x] = v;
  }
}
// After a sweep: the residual max |b - A x| (one warp), the iteration count, and done when it is below tol.
__global__ void k_jacobi_check(const double *bmax, int nb, double tol, unsigned int *done, unsigned int *iters,
                               double *residual) {
  if (*(volatile unsigned int *)done) return;
  double m = 0.0;
  for (int b = threadIdx.x; b < nb; b += 32) m = fmax(m, bmax[b]);
  m = warp_max(m);
  if (threadIdx.x == 0) {
    *residual = m;
    *iters += 1u;
    if (m < tol) *done = 1u;
  }
}
// SSPRK3 stage (solve_phase_advection_only, phase_field.cpp:398-435): stage 1 out = c0 + dt rs; stage 2
// out = 3/4 c0 + 1/4 (cs + dt rs); stage 3 out = 1/3 c0 + 2/3 (cs + dt rs).
__global__ void k_ssprk3_stage(Fv c0, Fv cs, Fv rs, Fv out, double dt, int stage) {
  DN_FOR_INTERIOR(out);
  if (stage == 1) {
    out.at(i, j) = c0.at(i, j) + dt * rs.at(i, j);
  } else {
    const double pred = cs.at(i, j) + dt * rs.at(i, j);
    out.at(i, j) = stage == 2 ? 0.75 * c0.at(i, j) + 0.25 * pred : (1.0 / 3.0) * c0.at(i, j) + (2.0 / 3.0) * pred;
  }
}
// Per-block partial sums of (a - b)^2 and a^2 over the interior (field_diff_l2 of the reference), [2][nb].
__global__ void k_diff_l2_partials(Fv a, Fv b, double *partials) {
  __shared__ double sh[8 * 32 * 2];
  const long long n = (long long)a.nx * a.ny;
  double v[2] = {0.0, 0.0};
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / a.ny), j = (int)(t % a.ny);
    const double d = a.at(i, j) - b.at(i, j);
    v[0] += d * d;
    v[1] += a.at(i, j) * a.at(i, j);
  }
  block_sum<2>(v, sh);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = v[0];
    partials[gridDim.x + blockIdx.x] = v[1];
  }
}
// Per-block partial sums of up to four products sum a_k b_k (a null a_k contributes 0) and the number of
// non-finite values in f0 and f1 (null: none), [5][gridDim.x]; the caller adds the blocks in order.
__global__ void k_dots4(const double *a0, const double *b0, const double *a1, const double *b1, const double *a2,
                        const double *b2, const double *a3, const double *b3, const double *f0, const double *f1,
                        long long n, double *partials) {
  __shared__ double sh[8 * 32 * 5];
  double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    if (a0) v[0] += a0[t] * b0[t];
    if (a1) v[1] += a1[t] * b1[t];
    if (a2) v[2] += a2[t] * b2[t];
    if (a3) v[3] += a3[t] * b3[t];
    if (f0 && !isfinite(f0[t])) v[4] += 1.0;
    if (f1 && !isfinite(f1[t])) v[4] += 1.0;
  }
  block_sum<5>(v, sh);
  if (threadIdx.x == 0)
    for (int k = 0; k < 5; ++k) partials[(size_t)k * gridDim.x + blockIdx.x] = v[k];
}
__global__ void k_div_scalar(const double *in, double *out, long long n, double d) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = in[t] / d;
}
__global__ void k_sub_scaled(double *y, const double *x, long long n, double a) {  // y -= a x
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) y[t] -= a * x[t];
}
__global__ void k_x_step(double *x, const double *d, double *delta, long long n, double alpha) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) {
    const double dl = alpha * d[t];
    x[t] += dl;
    delta[t] = dl;
  }
}
__global__ void k_vec_sum(const double *x, long long n, double *partials) {
  __shared__ double sh[8 * 32];
  double v[1] = {0.0};
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    v[0] += x[t];
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}
__global__ void k_finish_mean(const double *partials, int nparts, double count, double *out) {
  const int lane = threadIdx.x;
  double s = 0.0;
  for (int b = lane; b < nparts; b += 32) s += partials[b];
  s = warp_sum(s);
  if (lane == 0) out[0] = s / count;
}
__global__ void k_vec_sub_scalar(double *x, long long n, const double *sub) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) x[t] -= *sub;
}

// periodic_boundary_speed_stat, operators.cpp:463-478 (single CTA)
__global__ void k_boundary_speed(Fv u, Fv v, Grid G, double *out) {
  double m = 0.0;
  if (G.px)
    for (int j = threadIdx.x; j < u.ny; j += blockDim.x) m = fmax(m, fmax(fabs(u.at(0, j)), fabs(u.at(G.nx, j))));
  if (G.py)
    for (int i = threadIdx.x; i < v.nx; i += blockDim.x) m = fmax(m, fmax(fabs(v.at(i, 0)), fabs(v.at(i, G.ny))));
  __shared__ double sh[32];
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, sh[w]);
    *out = r;
  }
}

// Diagnostics, diagnostics.cpp:24-167: per-block partials of
//   0 mass  1 div_sq  2 div_max  3 mu_max  4 vel_max  5 ke  6 rho_min  7 rho_max  8 eta_min  9 eta_max
//   10 free energy  11 max advective rate  12 mobility max  13 |W''| max
constexpr int kNDiag = 14;
__global__ void k_diag_partials(Fv c, Fv u, Fv v, Fv mu, Fv rho, Fv eta, Grid G, double cn, double *partials) {
  double a[kNDiag];
  const int ops[kNDiag] = {0, 0, 1, 1, 1, 0, 2, 1, 2, 1, 0, 1, 1, 1};
#pragma unroll
  for (int k = 0; k < kNDiag; ++k) a[k] = red_identity(ops[k]);
  const long long n = (long long)G.nx * G.ny;
  const double alpha = 6.0 * 1.4142135623730950488;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / G.ny), j = (int)(t % G.ny);
    const double cc = c.at(i, j);
    a[0] += cc * G.dx * G.dy;
    const double dv = div_cell(u, v, G, i, j);
    const double uc = 0.5 * (u.at(i, j) + u.at(i + 1, j)), vc = 0.5 * (v.at(i, j) + v.at(i, j + 1));
    a[1] += dv * dv;
    a[2] = fmax(a[2], fabs(dv));
    a[3] = fmax(a[3], fabs(mu.at(i, j)));
    a[4] = fmax(a[4], sqrt(uc * uc + vc * vc));
    a[5] += 0.5 * rho.at(i, j) * (uc * uc + vc * vc) * G.dx * G.dy;
    a[6] = fmin(a[6], rho.at(i, j));
    a[7] = fmax(a[7], rho.at(i, j));
    a[8] = fmin(a[8], eta.at(i, j));
    a[9] = fmax(a[9], eta.at(i, j));
    const double bulk = 0.25 * cc * cc * sq(1.0 - cc) / cn;
    const double gx = (c.at(i + 1, j) - c.at(i - 1, j)) / (2.0 * G.dx);
    const double gy = (c.at(i, j + 1) - c.at(i, j - 1)) / (2.0 * G.dy);
    a[10] += alpha * (bulk + 0.5 * cn * (sq(gx) + sq(gy))) * G.dx * G.dy;
    a[11] = fmax(a[11], fabs(uc) / fmax(G.dx, 1.0e-30) + fabs(vc) / fmax(G.dy, 1.0e-30));
    a[12] = fmax(a[12], fmax(0.0, cc * (1.0 - cc)));
    a[13] = fmax(a[13], fabs(0.5 - 3.0 * cc + 3.0 * cc * cc));
  }
  __shared__ double sh[kNDiag][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kNDiag; ++k) {
    double s = a[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s = red_combine(ops[k], s, __shfl_xor_sync(0xffffffffu, s, o));
    if (lane == 0) sh[k][w] = s;
  }
  __syncthreads();
  if (threadIdx.x < kNDiag) {
    const int k = threadIdx.x;
    double s = red_identity(ops[k]);
    for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww) s = red_combine(ops[k], s, sh[k][ww]);
    partials[(size_t)blockIdx.x * kNDiag + k] = s;
  }
}

}  // namespace dn
