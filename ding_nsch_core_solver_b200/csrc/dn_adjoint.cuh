// dn_adjoint.cuh -- discrete adjoint (vector-Jacobian product) of the pressure projection.
//
// The projection is the last part of a time step: the pressure system of the predicted velocity
// (build_pressure_linear_system, pressure.cpp:123-212, with the split explicit term of
// liu_split_explicit_divergence, operators.cpp:424-444), its PCG solve, and the velocity correction
// (apply_pressure_velocity_correction, operators.cpp:480-534) followed by the face BCs (apply_u_bc /
// apply_v_bc, operators.cpp:183-289).  With rho_mid held fixed it is an affine map
//
//     (u*, v*, p, p_prev)  ->  (u, v, p_new, p_prev_new = p)
//
// of interior values (faces 0..nx x 0..ny-1 for u, cells for p).  These kernels apply its transpose to a
// cotangent (gu, gv, gp, gpp).  The pressure operator is symmetric, so the transposed solve is the same
// PCG on a different right-hand side.  The reference has no adjoint; every transposition below follows the
// forward kernels of this library term by term.
#pragma once

#include "dn_common.cuh"
#include "dn_fields.cuh"

namespace dn {

// Cotangent of the face BCs applied after the correction.  A boundary face is overwritten by its BC:
// Dirichlet sets a constant (its cotangent is dropped); Neumann copies the adjacent face plus a constant
// (the cotangent moves to that face); periodic copies face 0 onto face nx (the cotangent of face nx moves to
// face 0).  `out` receives the folded cotangent of the corrected, pre-BC face values.
__global__ void k_adj_fold_u(Fv gu, Fv out, Grid G, BCSet bc) {
  DN_FOR_INTERIOR(out);
  const int last = G.nx;
  double v = gu.at(i, j);
  if (G.px) {
    if (i == last) v = 0.0;
    else if (i == 0) v += gu.at(last, j);
  } else if (i == 0 || i == last) {
    v = 0.0;
  } else {
    if (i == 1 && bc.u[DN_LEFT].type != DN_BC_DIRICHLET) v += gu.at(0, j);
    if (i == last - 1 && bc.u[DN_RIGHT].type != DN_BC_DIRICHLET) v += gu.at(last, j);
  }
  out.at(i, j) = v;
}
__global__ void k_adj_fold_v(Fv gv, Fv out, Grid G, BCSet bc) {
  DN_FOR_INTERIOR(out);
  const int last = G.ny;
  double v = gv.at(i, j);
  if (G.py) {
    if (j == last) v = 0.0;
    else if (j == 0) v += gv.at(i, last);
  } else if (j == 0 || j == last) {
    v = 0.0;
  } else {
    if (j == 1 && bc.v[DN_BOTTOM].type != DN_BC_DIRICHLET) v += gv.at(i, 0);
    if (j == last - 1 && bc.v[DN_TOP].type != DN_BC_DIRICHLET) v += gv.at(i, last);
  }
  out.at(i, j) = v;
}

// Face weights of the correction u(f) -= dt * (alpha(f) dx(p_corr)(f) + beta(f) dx(p_ext)(f)):
// alpha = 1/rho_ref, beta = 1/rho_face - 1/rho_ref for the split scheme; alpha = 1/rho_face, beta = 0 else.
__device__ __forceinline__ double adj_alpha(bool x, const Fv &rm, const Grid &G, int i, int j, int split,
                                            double rho_ref) {
  return split ? 1.0 / rho_ref : 1.0 / (x ? xface(rm, G, i, j) : yface(rm, G, i, j));
}
__device__ __forceinline__ double adj_beta(bool x, const Fv &rm, const Grid &G, int i, int j, int split,
                                           double rho_ref) {
  return split ? 1.0 / (x ? xface(rm, G, i, j) : yface(rm, G, i, j)) - 1.0 / rho_ref : 0.0;
}

// Per cell: the cotangent of p_corr from the correction, plus gp (p_new = p_corr up to the mean), into the
// compact right-hand side `b` of the transposed solve; and the cotangent of the extrapolated pressure from
// the correction into `pe_bar` (split scheme).  fu, fv hold the folded face cotangents.  A face gradient
// reads the cell on each side; the only ghost cell that receives a cotangent is the periodic one west of
// face 0 (south of face 0), whose cotangent lands on cell nx-1 (ny-1): that is the east (north) face term
// of the last cell, taken at face 0.
__global__ void k_adj_cells_pre(Fv fu, Fv fv, Fv gp, Fv rm, Grid G, int split, double rho_ref, double dt,
                                double *b, Fv pe_bar) {
  const long long n = (long long)G.nx * G.ny;
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int i = (int)(r / G.ny), j = (int)(r % G.ny);
  const int fe = (G.px && i == G.nx - 1) ? 0 : i + 1;
  const int fn = (G.py && j == G.ny - 1) ? 0 : j + 1;
  const double cx = dt / G.dx, cy = dt / G.dy;
  const double pc = cx * (adj_alpha(true, rm, G, fe, j, split, rho_ref) * fu.at(fe, j) -
                          adj_alpha(true, rm, G, i, j, split, rho_ref) * fu.at(i, j)) +
                    cy * (adj_alpha(false, rm, G, i, fn, split, rho_ref) * fv.at(i, fn) -
                          adj_alpha(false, rm, G, i, j, split, rho_ref) * fv.at(i, j));
  b[r] = pc + gp.at(i, j);
  double pe = 0.0;
  if (split)
    pe = cx * (adj_beta(true, rm, G, fe, j, split, rho_ref) * fu.at(fe, j) -
               adj_beta(true, rm, G, i, j, split, rho_ref) * fu.at(i, j)) +
         cy * (adj_beta(false, rm, G, i, fn, split, rho_ref) * fv.at(i, fn) -
               adj_beta(false, rm, G, i, j, split, rho_ref) * fv.at(i, j));
  pe_bar.at(i, j) = pe;
}

// Transposed divergence: rhs(c) holds -kappa * div(u*, v*)(c), kappa = rho_ref/dt (split) or 1/dt, and
// div reads faces c and c+1 directly (face nx too when periodic), so u*(f) gets kappa/dx (rbar(f) -
// rbar(f-1)) with rbar = 0 outside the cells.  rbar is compact (row = i*ny + j).
__global__ void k_adj_div_u(Fv au, const double *rbar, Grid G, double kappa) {
  DN_FOR_INTERIOR(au);
  const double e = i < G.nx ? rbar[(long long)i * G.ny + j] : 0.0;
  const double w = i > 0 ? rbar[(long long)(i - 1) * G.ny + j] : 0.0;
  au.at(i, j) += kappa / G.dx * (e - w);
}
__global__ void k_adj_div_v(Fv av, const double *rbar, Grid G, double kappa) {
  DN_FOR_INTERIOR(av);
  const double nn = j < G.ny ? rbar[(long long)i * G.ny + j] : 0.0;
  const double s = j > 0 ? rbar[(long long)i * G.ny + j - 1] : 0.0;
  av.at(i, j) += kappa / G.dy * (nn - s);
}

// Cotangent of one split flux F(f) = w(f) (p_ext(f) - p_ext(f-1)) / h, w = 1 - rho_ref / rho_face, that
// enters rhs(f-1) as -F/h and rhs(f) as +F/h when the face is open (periodic, or not on the boundary).
__device__ __forceinline__ double adj_flux_x(const double *rbar, const Grid &G, int f, int j) {
  if (!(G.px || (f > 0 && f < G.nx))) return 0.0;
  const double e = f < G.nx ? rbar[(long long)f * G.ny + j] : 0.0;
  const double w = f > 0 ? rbar[(long long)(f - 1) * G.ny + j] : 0.0;
  return (e - w) / G.dx;
}
__device__ __forceinline__ double adj_flux_y(const double *rbar, const Grid &G, int i, int f) {
  if (!(G.py || (f > 0 && f < G.ny))) return 0.0;
  const double nn = f < G.ny ? rbar[(long long)i * G.ny + f] : 0.0;
  const double s = f > 0 ? rbar[(long long)i * G.ny + f - 1] : 0.0;
  return (nn - s) / G.dy;
}

// Per cell: the cotangent of the extrapolated pressure (correction part in pe_bar, plus the split
// explicit divergence), then p_ext = s p - [step > 0] p_prev with s = 1 on step 0 and 2 after
// (build_liu_split_pressure_extrapolation, operators.cpp:413-422), and p_prev_new = p.  Periodic ghost
// cells east of face nx / west of face 0 fold onto cells 0 / nx-1.  ap and app are written here; app held
// pe_bar on entry (the same cell, read before it is written).
__global__ void k_adj_cells_post(const double *rbar, Fv gpp, Fv rm, Grid G, int split, double rho_ref, int step,
                                 Fv ap, Fv app) {
  const long long n = (long long)G.nx * G.ny;
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int i = (int)(r / G.ny), j = (int)(r % G.ny);
  double pe = app.at(i, j);
  if (split) {
    auto wx = [&](int f) { return 1.0 - rho_ref / xface(rm, G, f, j); };
    auto wy = [&](int f) { return 1.0 - rho_ref / yface(rm, G, i, f); };
    pe += (wx(i) * adj_flux_x(rbar, G, i, j) - wx(i + 1) * adj_flux_x(rbar, G, i + 1, j)) / G.dx;
    pe += (wy(j) * adj_flux_y(rbar, G, i, j) - wy(j + 1) * adj_flux_y(rbar, G, i, j + 1)) / G.dy;
    if (G.px && i == 0) pe += wx(G.nx) * adj_flux_x(rbar, G, G.nx, j) / G.dx;   // ghost east of face nx
    if (G.px && i == G.nx - 1) pe -= wx(0) * adj_flux_x(rbar, G, 0, j) / G.dx;  // ghost west of face 0
    if (G.py && j == 0) pe += wy(G.ny) * adj_flux_y(rbar, G, i, G.ny) / G.dy;
    if (G.py && j == G.ny - 1) pe -= wy(0) * adj_flux_y(rbar, G, i, 0) / G.dy;
  }
  const double s = step == 0 ? 1.0 : 2.0;
  ap.at(i, j) = (split ? s * pe : 0.0) + gpp.at(i, j);
  app.at(i, j) = (split && step != 0) ? -pe : 0.0;
}

// ------------------------------------------------------------------------------------------------------
// Adjoint of the CH advective term rhs = -div(F), F_x(f) = u(f) W(c stencil of f), with W the WENO5 face
// value (weno5_left, phase_field.cpp:144-157, upwinded by the sign of the face velocity) of c extended by
// its scalar BC ghosts (apply_scalar_bc, operators.cpp:130-141), and the face BCs of the velocity applied to
// F (build_phase_advection_fluxes, phase_field.cpp:283-311).  Differentiated with the nonlinear weights
// included; the upwind switch is piecewise (the derivative in u is taken on the side of the sign of u).
// ------------------------------------------------------------------------------------------------------

// W and dW/dv_m for W = weno5_left(v1..v5): W = sum a_k q_k / S, a_k = d_k / (eps + b_k)^2, S = sum a_k, so
// dW = sum_k a_k dq_k / S + sum_k (q_k - W) da_k / S with da_k = -2 d_k / (eps + b_k)^3 db_k.
__device__ __forceinline__ double weno5_left_grad(const double (&v)[5], double (&dw)[5]) {
  const double eps = 1.0e-6;
  const double q[3] = {(2.0 * v[0] - 7.0 * v[1] + 11.0 * v[2]) / 6.0, (-v[1] + 5.0 * v[2] + 2.0 * v[3]) / 6.0,
                       (2.0 * v[2] + 5.0 * v[3] - v[4]) / 6.0};
  const double dq[3][5] = {{2.0 / 6.0, -7.0 / 6.0, 11.0 / 6.0, 0.0, 0.0},
                           {0.0, -1.0 / 6.0, 5.0 / 6.0, 2.0 / 6.0, 0.0},
                           {0.0, 0.0, 2.0 / 6.0, 5.0 / 6.0, -1.0 / 6.0}};
  // b_k = 13/12 s_k^2 + 1/4 t_k^2 with s_k, t_k linear in v
  const double ds[3][5] = {{1, -2, 1, 0, 0}, {0, 1, -2, 1, 0}, {0, 0, 1, -2, 1}};
  const double dt[3][5] = {{1, -4, 3, 0, 0}, {0, 1, 0, -1, 0}, {0, 0, 3, -4, 1}};
  const double dk[3] = {0.1, 0.6, 0.3};
  double a[3], da[3][5], S = 0.0, num = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double sk = 0.0, tk = 0.0;
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      sk += ds[k][m] * v[m];
      tk += dt[k][m] * v[m];
    }
    const double b = 13.0 / 12.0 * sk * sk + 0.25 * tk * tk;
    const double e = eps + b;
    a[k] = dk[k] / (e * e);
    const double c = -2.0 * dk[k] / (e * e * e);
#pragma unroll
    for (int m = 0; m < 5; ++m) da[k][m] = c * (13.0 / 6.0 * sk * ds[k][m] + 0.5 * tk * dt[k][m]);
    S += a[k];
    num += a[k] * q[k];
  }
  const double W = num / S;
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    double g = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) g += a[k] * dq[k][m] + (q[k] - W) * da[k][m];
    dw[m] = g / S;
  }
  return W;
}

// Extended cell index (-3 .. n+2) -> interior cell holding its value under the scalar BCs.
__device__ __forceinline__ int scalar_bc_source(int e, int n, int periodic) {
  if (e >= 0 && e < n) return e;
  if (periodic) return e < 0 ? e + n : e - n;
  return e < 0 ? 0 : n - 1;
}

// Cotangent of the flux at x-face f, after the velocity face BC written onto the fluxes (the same fold as
// k_adj_fold_u) and before it: F(f) enters rhs(f-1) as -F/dx and rhs(f) as +F/dx.
__device__ __forceinline__ double adv_flux_bar_x(const Fv &rb, const Grid &G, const BCSet &bc, int f, int j) {
  auto raw = [&](int q) {
    const double e = q < G.nx ? rb.at(q, j) : 0.0;
    const double w = q > 0 ? rb.at(q - 1, j) : 0.0;
    return (e - w) / G.dx;
  };
  const int last = G.nx;
  if (G.px) return f == last ? 0.0 : (f == 0 ? raw(0) + raw(last) : raw(f));
  if (f == 0 || f == last) return 0.0;
  double v = raw(f);
  if (f == 1 && bc.u[DN_LEFT].type != DN_BC_DIRICHLET) v += raw(0);
  if (f == last - 1 && bc.u[DN_RIGHT].type != DN_BC_DIRICHLET) v += raw(last);
  return v;
}
__device__ __forceinline__ double adv_flux_bar_y(const Fv &rb, const Grid &G, const BCSet &bc, int i, int f) {
  auto raw = [&](int q) {
    const double nn = q < G.ny ? rb.at(i, q) : 0.0;
    const double s = q > 0 ? rb.at(i, q - 1) : 0.0;
    return (nn - s) / G.dy;
  };
  const int last = G.ny;
  if (G.py) return f == last ? 0.0 : (f == 0 ? raw(0) + raw(last) : raw(f));
  if (f == 0 || f == last) return 0.0;
  double v = raw(f);
  if (f == 1 && bc.v[DN_BOTTOM].type != DN_BC_DIRICHLET) v += raw(0);
  if (f == last - 1 && bc.v[DN_TOP].type != DN_BC_DIRICHLET) v += raw(last);
  return v;
}

// Stencil of face f along one direction: the five values in weno5_left order and, per slot, the extended
// cell index it reads (u >= 0: cells f-3 .. f+1; u < 0: f+2 .. f-2).
__device__ __forceinline__ int adv_slot_cell(int f, int m, bool up) { return up ? f - 3 + m : f + 2 - m; }

// u_bar(f) = F_bar(f) W(f)
__global__ void k_adv_adj_u(Fv ce, Fv u, Fv rb, Fv ubar, Grid G, BCSet bc) {
  DN_FOR_INTERIOR(ubar);
  const bool up = u.at(i, j) >= 0.0;
  double v[5], dw[5];
#pragma unroll
  for (int m = 0; m < 5; ++m) v[m] = ce.at(adv_slot_cell(i, m, up), j);
  ubar.at(i, j) = adv_flux_bar_x(rb, G, bc, i, j) * weno5_left_grad(v, dw);
}
__global__ void k_adv_adj_v(Fv ce, Fv vv, Fv rb, Fv vbar, Grid G, BCSet bc) {
  DN_FOR_INTERIOR(vbar);
  const bool up = vv.at(i, j) >= 0.0;
  double v[5], dw[5];
#pragma unroll
  for (int m = 0; m < 5; ++m) v[m] = ce.at(i, adv_slot_cell(j, m, up));
  vbar.at(i, j) = adv_flux_bar_y(rb, G, bc, i, j) * weno5_left_grad(v, dw);
}

// Extended indices (-3 .. n+2) whose BC ghost value is interior cell i: i itself, the three ghosts beyond
// a non-periodic edge cell, or the periodic image.  Returns how many (at most 4).
__device__ __forceinline__ int scalar_bc_images(int i, int n, int periodic, int (&e)[4]) {
  int k = 0;
  e[k++] = i;
  if (periodic) {
    if (i >= n - 3) e[k++] = i - n;
    if (i <= 2) e[k++] = i + n;
  } else {
    if (i == 0)
      for (int g = 1; g <= 3; ++g) e[k++] = -g;
    else if (i == n - 1)
      for (int g = 0; g < 3; ++g) e[k++] = n + g;
  }
  return k;
}

// Sum over the faces along one direction whose stencil reads extended index e, of F_bar(f) u(f) dW/dv_m.
// X selects x (faces f along i at row j) or y (faces f along j at column i).
template <bool X>
__device__ __forceinline__ double adv_adj_gather(const Fv &ce, const Fv &vel, const Fv &rb, const Grid &G,
                                                 const BCSet &bc, int i, int j, int e) {
  const int nf = X ? G.nx : G.ny;
  double acc = 0.0;
  for (int f = max(e - 2, 0); f <= min(e + 3, nf); ++f) {
    const double w = X ? vel.at(f, j) : vel.at(i, f);
    const bool up = w >= 0.0;
    const int m = up ? e - f + 3 : f + 2 - e;
    if (m < 0 || m > 4) continue;
    const double fb = X ? adv_flux_bar_x(rb, G, bc, f, j) : adv_flux_bar_y(rb, G, bc, i, f);
    double v[5], dw[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) v[k] = X ? ce.at(adv_slot_cell(f, k, up), j) : ce.at(i, adv_slot_cell(f, k, up));
    weno5_left_grad(v, dw);
    acc += fb * w * dw[m];
  }
  return acc;
}

// c_bar(i, j): every face whose stencil reads cell (i, j), directly or through a BC ghost, in a fixed order.
__global__ void k_adv_adj_c(Fv ce, Fv u, Fv vv, Fv rb, Fv cbar, Grid G, BCSet bc) {
  DN_FOR_INTERIOR(cbar);
  double acc = 0.0;
  int e[4];
  const int kx = scalar_bc_images(i, G.nx, G.px, e);
  for (int k = 0; k < kx; ++k) acc += adv_adj_gather<true>(ce, u, rb, G, bc, i, j, e[k]);
  const int ky = scalar_bc_images(j, G.ny, G.py, e);
  for (int k = 0; k < ky; ++k) acc += adv_adj_gather<false>(ce, vv, rb, G, bc, i, j, e[k]);
  cbar.at(i, j) += acc;  // accumulates: the caller clears cbar first
}

// ------------------------------------------------------------------------------------------------------
// Adjoint of the CH explicit operator (build_phase_explicit_operator, phase_field.cpp:354-396)
//   E = div(M grad mu) / pe - (a1 L c - a2 L L c) / pe + adv(c, u, v),
//   M = max(0, c (1 - c)) on faces by xface, mu = 6 sqrt2 (W'(c) / cn - cn L c), W' = c (1 - c) (1 - 2c) / 2,
// with L the scalar-BC Laplacian (symmetric, so it is its own transpose) and the velocity face BCs written
// onto the diffusive fluxes.  The advective part is k_adv_adj_*.
// ------------------------------------------------------------------------------------------------------

// Cotangent of the diffusive flux at x-face f before its face BC: the flux enters ddiv(f-1) as +F/dx and
// ddiv(f) as -F/dx, scaled by 1/pe; the fold is that of the velocity face BC (k_adj_fold_u).
__device__ __forceinline__ double diff_flux_bar_x(const Fv &g, const Grid &G, const BCSet &bc, int f, int j,
                                                  double inv_pe) {
  auto raw = [&](int q) {
    const double w = q > 0 ? g.at(q - 1, j) : 0.0;
    const double e = q < G.nx ? g.at(q, j) : 0.0;
    return (w - e) * inv_pe / G.dx;
  };
  const int last = G.nx;
  if (G.px) return f == last ? 0.0 : (f == 0 ? raw(0) + raw(last) : raw(f));
  if (f == 0 || f == last) return 0.0;
  double v = raw(f);
  if (f == 1 && bc.u[DN_LEFT].type != DN_BC_DIRICHLET) v += raw(0);
  if (f == last - 1 && bc.u[DN_RIGHT].type != DN_BC_DIRICHLET) v += raw(last);
  return v;
}
__device__ __forceinline__ double diff_flux_bar_y(const Fv &g, const Grid &G, const BCSet &bc, int i, int f,
                                                  double inv_pe) {
  auto raw = [&](int q) {
    const double s = q > 0 ? g.at(i, q - 1) : 0.0;
    const double nn = q < G.ny ? g.at(i, q) : 0.0;
    return (s - nn) * inv_pe / G.dy;
  };
  const int last = G.ny;
  if (G.py) return f == last ? 0.0 : (f == 0 ? raw(0) + raw(last) : raw(f));
  if (f == 0 || f == last) return 0.0;
  double v = raw(f);
  if (f == 1 && bc.v[DN_BOTTOM].type != DN_BC_DIRICHLET) v += raw(0);
  if (f == last - 1 && bc.v[DN_TOP].type != DN_BC_DIRICHLET) v += raw(last);
  return v;
}

// Per x-face: with F = M_face * dmu/dx, the cotangents M_bar = F_bar dmu/dx (into mb) and
// G_bar = F_bar M_face (into gb).
__global__ void k_eadj_face_x(Fv g, Fv mob, Fv mu, Fv mb, Fv gb, Grid G, BCSet bc, double inv_pe) {
  DN_FOR_INTERIOR(mb);
  const double p = diff_flux_bar_x(g, G, bc, i, j, inv_pe);
  mb.at(i, j) = p * gfx(mu, G, i, j);
  gb.at(i, j) = p * xface(mob, G, i, j);
}
__global__ void k_eadj_face_y(Fv g, Fv mob, Fv mu, Fv mb, Fv gb, Grid G, BCSet bc, double inv_pe) {
  DN_FOR_INTERIOR(mb);
  const double p = diff_flux_bar_y(g, G, bc, i, j, inv_pe);
  mb.at(i, j) = p * gfy(mu, G, i, j);
  gb.at(i, j) = p * yface(mob, G, i, j);
}

// Per cell: the mobility cotangent (each face average puts half on either cell; the periodic face 0 pairs
// cells nx-1 and 0) and the chemical-potential cotangent mu_bar (into mub); c_bar (into cbar) gets the local
// parts mob_bar M'(c) + 6 sqrt2 W''(c) / cn mu_bar.
__global__ void k_eadj_cells(Fv c, Fv mbx, Fv gbx, Fv mby, Fv gby, Fv mub, Fv cbar, Grid G, double cn) {
  DN_FOR_INTERIOR(cbar);
  const int fe = (G.px && i == G.nx - 1) ? 0 : i + 1;
  const int fn = (G.py && j == G.ny - 1) ? 0 : j + 1;
  const double mobb = 0.5 * (mbx.at(i, j) + mbx.at(fe, j)) + 0.5 * (mby.at(i, j) + mby.at(i, fn));
  const double mu_b = (gbx.at(i, j) - gbx.at(fe, j)) / G.dx + (gby.at(i, j) - gby.at(i, fn)) / G.dy;
  const double cc = c.at(i, j);
  const double dmob = cc * (1.0 - cc) > 0.0 ? 1.0 - 2.0 * cc : 0.0;
  const double alpha = 6.0 * 1.4142135623730950488;
  const double ddw = 0.5 * (1.0 - 6.0 * cc + 6.0 * cc * cc);
  mub.at(i, j) = mu_b;
  cbar.at(i, j) = mobb * dmob + alpha * ddw / cn * mu_b;
}

// out += s * L in  (in carries its scalar-BC ghosts)
__global__ void k_add_scaled_lap(Fv in, Fv out, Grid G, double s) {
  DN_FOR_INTERIOR(out);
  out.at(i, j) += s * lapc(in, G, i, j);
}
// out = s0 in + s1 L in
__global__ void k_lin_lap(Fv in, Fv out, Grid G, double s0, double s1) {
  DN_FOR_INTERIOR(out);
  out.at(i, j) = s0 * in.at(i, j) + s1 * lapc(in, G, i, j);
}

}  // namespace dn
