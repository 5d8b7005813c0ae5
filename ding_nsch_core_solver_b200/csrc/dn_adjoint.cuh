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

}  // namespace dn
