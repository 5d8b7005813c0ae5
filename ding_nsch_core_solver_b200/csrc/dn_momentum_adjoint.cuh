// dn_momentum_adjoint.cuh -- discrete adjoint of the momentum predictor (solve_momentum_predictor,
// momentum.cpp:157-502) as a map of the velocity state, at fixed materials.
//
// The map: (u, v, H_prev, f) -> (u*, v*).  The inputs' BCs are applied (bc(u, kBCU), bc(v, kBCV)), the
// predictor right-hand side is formed (k_mom_conv_rhs: rho_face u + dt (-rho_face conv + rho_face g + f) +
// alpha visc(u, v; eta_prev), conv = H(u, v) on step 0 and 1.5 H - 0.5 H_prev after), the coupled system
// M(rho_mid, eta) x = rhs is solved, x is scattered to the active faces and the faces' BCs fill the rest.
// rho_mid, eta and eta_prev are constants of the map.  Its adjoint, for a cotangent (gu*, gv*):
//   1. fold the cotangent through the output face BCs (k_adj_fold_u / _v) and gather it at the active faces;
//   2. solve M^T lambda = g (M^T assembled from M's rows, solved by the same Jacobi-BiCGSTAB);
//   3. lambda is the cotangent of the right-hand side: f_bar = dt lambda, H_prev_bar = 0.5 dt rho_face lambda
//      (steps > 0), and (u, v)_bar collect rho_face lambda plus the transposed stencils of the centred
//      convection (linearised at the forward's u, v) and of the viscous divergence (k_mom_rhs_adj);
//   4. the input BCs are undone: each ghost's cotangent moves to the interior value its BC copies (sign -1
//      through a Dirichlet reflection, k_adj_ghosts), then the face BCs are folded (k_adj_fold_u / _v).
// Scatters use FP64 atomics (the summation order of a cotangent entry is not fixed, so gradients agree to
// round-off, not bit for bit).
#pragma once

#include "dn_adjoint.cuh"
#include "dn_momentum.cuh"

namespace dn {

// Canonical targets of unknown t (the 9 columns of its row before folding and dropping; -2 for a target
// outside the active set) and its face (i, j, is_u).
__device__ __forceinline__ void mom_row_targets(const MomLayout &L, long long t, long long (&tg)[9], int &i, int &j,
                                                bool &is_u) {
  is_u = t < L.nu;
  if (is_u) {
    i = (int)(t / L.ny);
    j = (int)(t % L.ny);
  } else {
    i = (int)((t - L.nu) / (L.ny + 1));
    j = (int)((t - L.nu) % (L.ny + 1));
  }
  auto uT = [&](int ii, int jj) -> long long { return L.u_active(ii, jj) ? L.uidx(ii, jj) : -2; };
  auto vT = [&](int ii, int jj) -> long long { return L.v_active(ii, jj) ? L.vidx(ii, jj) : -2; };
  if (is_u) {
    tg[0] = L.uidx(i, j);
    tg[1] = uT(L.cui(i + 1), j);
    tg[2] = uT(L.cui(i - 1), j);
    tg[3] = uT(i, L.cuj(j + 1));
    tg[4] = uT(i, L.cuj(j - 1));
    tg[5] = vT(L.cui(i), L.cuj(j + 1));
    tg[6] = vT(L.cui(i - 1), L.cuj(j + 1));
    tg[7] = vT(L.cui(i), L.cuj(j));
    tg[8] = vT(L.cui(i - 1), L.cuj(j));
  } else {
    tg[0] = L.vidx(i, j);
    tg[1] = vT(L.cui(i + 1), j);
    tg[2] = vT(L.cui(i - 1), j);
    tg[3] = vT(i, L.cuj(j + 1));
    tg[4] = vT(i, L.cuj(j - 1));
    tg[5] = uT(L.cui(i + 1), L.cuj(j));
    tg[6] = uT(L.cui(i + 1), L.cuj(j - 1));
    tg[7] = uT(L.cui(i), L.cuj(j));
    tg[8] = uT(L.cui(i), L.cuj(j - 1));
  }
}

// M^T in the same row format: row c of M^T holds, for each distinct canonical target r of row c, the sum of
// row r's stored coefficients whose column is c.  The coupled stencil is structurally symmetric (row r
// targets c exactly when row c targets r), so every entry of M lands in M^T.
__global__ void k_mom_transpose(MomLayout L, const double *coef, const int *tgt, double *tcoef, int *ttgt) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long N = L.n();
  if (c >= N) return;
  long long tg[9];
  int i, j;
  bool is_u;
  mom_row_targets(L, c, tg, i, j, is_u);
  const bool active = is_u ? L.u_active(i, j) : L.v_active(i, j);
  for (int k = 0; k < 9; ++k) {
    const long long r = tg[k];
    bool dup = false;
    for (int q = 0; q < k; ++q) dup = dup || (tg[q] == r);
    double val = 0.0;
    if (active && r >= 0 && !dup) {
      for (int q = 0; q < 9; ++q)
        if (tgt[(size_t)q * N + r] == (int)c) val += coef[(size_t)q * N + r];
    }
    const bool keep = k == 0 ? active : val != 0.0;
    tcoef[(size_t)k * N + c] = keep ? val : 0.0;
    ttgt[(size_t)k * N + c] = keep ? (int)r : -1;
  }
}

// the cotangent g of the solution vector at the active faces (from face fields), 0 elsewhere
__global__ void k_mom_gather(MomLayout L, Fv gu, Fv gv, double *g) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= L.n()) return;
  if (t < L.nu) {
    const int i = (int)(t / L.ny), j = (int)(t % L.ny);
    g[t] = L.u_active(i, j) ? gu.at(i, j) : 0.0;
  } else {
    const int i = (int)((t - L.nu) / (L.ny + 1)), j = (int)((t - L.nu) % (L.ny + 1));
    g[t] = L.v_active(i, j) ? gv.at(i, j) : 0.0;
  }
}

// Cotangents of the predictor right-hand side's inputs, one thread per face with lambda != 0 (the cotangent
// of that face's rhs): rho_face lambda onto the face's own velocity, the transposed centred convection
// (H = uf du/dx + vf du/dy for u faces, uf dv/dx + vf dv/dy for v faces; momentum.cpp:55-85) scaled by
// -dt rho_face (1 or 1.5), the transposed viscous divergence (visc_u / visc_v) scaled by alpha, and the
// direct f and H_prev cotangents.  au, av are ghosted and zero on entry.
__global__ void k_mom_rhs_adj(MomLayout L, Fv u, Fv v, Fv rm, Fv etap, Fv lu, Fv lv, Fv au, Fv av, Fv afu, Fv afv,
                              Fv ahu, Fv ahv, Grid G, int step, double dt, double alpha) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= L.n()) return;
  const double dx = G.dx, dy = G.dy;
  const double ch = (step == 0) ? 1.0 : 1.5;
  auto addu = [&](int i, int j, double val) { atomicAdd(&au.at(i, j), val); };
  auto addv = [&](int i, int j, double val) { atomicAdd(&av.at(i, j), val); };
  if (t < L.nu) {
    const int i = (int)(t / L.ny), j = (int)(t % L.ny);
    const double w = lu.at(i, j);
    if (w == 0.0) return;
    const double rf = xface(rm, G, i, j);
    afu.at(i, j) = dt * w;
    if (step != 0) ahu.at(i, j) = 0.5 * dt * rf * w;
    addu(i, j, rf * w);
    // convection: H = uf * dudx + vf * dudy
    const double c = -dt * rf * ch * w;
    const double uf = u.at(i, j);
    const double dudx = (u.at(i + 1, j) - u.at(i - 1, j)) / (2.0 * dx);
    const double dudy = (u.at(i, j + 1) - u.at(i, j - 1)) / (2.0 * dy);
    const double vf = 0.25 * (v.at(i - 1, j) + v.at(i, j) + v.at(i - 1, j + 1) + v.at(i, j + 1));
    addu(i, j, c * dudx);
    addu(i + 1, j, c * uf / (2.0 * dx));
    addu(i - 1, j, -c * uf / (2.0 * dx));
    addu(i, j + 1, c * vf / (2.0 * dy));
    addu(i, j - 1, -c * vf / (2.0 * dy));
    const double cv = 0.25 * c * dudy;
    addv(i - 1, j, cv);
    addv(i, j, cv);
    addv(i - 1, j + 1, cv);
    addv(i, j + 1, cv);
    // viscous divergence visc_u (linear in u, v at fixed eta_prev)
    const double a = alpha * w;
    const double eta_e = xface(etap, G, i + 1, j), eta_w = xface(etap, G, i, j);
    const double eta_n = corner(etap, i, j + 1), eta_s = corner(etap, i, j);
    const double ce = 2.0 * eta_e / (dx * dx), cw = 2.0 * eta_w / (dx * dx);
    const double cn = eta_n / (dy * dy), cs = eta_s / (dy * dy);
    const double xn = eta_n / (dx * dy), xs = eta_s / (dx * dy);
    addu(i + 1, j, a * ce);
    addu(i - 1, j, a * cw);
    addu(i, j, -a * (ce + cw + cn + cs));
    addu(i, j + 1, a * cn);
    addu(i, j - 1, a * cs);
    addv(i, j + 1, a * xn);
    addv(i - 1, j + 1, -a * xn);
    addv(i, j, -a * xs);
    addv(i - 1, j, a * xs);
  } else {
    const long long q = t - L.nu;
    const int i = (int)(q / (L.ny + 1)), j = (int)(q % (L.ny + 1));
    const double w = lv.at(i, j);
    if (w == 0.0) return;
    const double rf = yface(rm, G, i, j);
    afv.at(i, j) = dt * w;
    if (step != 0) ahv.at(i, j) = 0.5 * dt * rf * w;
    addv(i, j, rf * w);
    // convection: H = uf * dvdx + vf * dvdy
    const double c = -dt * rf * ch * w;
    const double vf = v.at(i, j);
    const double dvdx = (v.at(i + 1, j) - v.at(i - 1, j)) / (2.0 * dx);
    const double dvdy = (v.at(i, j + 1) - v.at(i, j - 1)) / (2.0 * dy);
    const double uf = 0.25 * (u.at(i, j - 1) + u.at(i, j) + u.at(i + 1, j - 1) + u.at(i + 1, j));
    addv(i, j, c * dvdy);
    addv(i + 1, j, c * uf / (2.0 * dx));
    addv(i - 1, j, -c * uf / (2.0 * dx));
    addv(i, j + 1, c * vf / (2.0 * dy));
    addv(i, j - 1, -c * vf / (2.0 * dy));
    const double cu = 0.25 * c * dvdx;
    addu(i, j - 1, cu);
    addu(i, j, cu);
    addu(i + 1, j - 1, cu);
    addu(i + 1, j, cu);
    // viscous divergence visc_v
    const double a = alpha * w;
    const double eta_e = corner(etap, i + 1, j), eta_w = corner(etap, i, j);
    const double eta_n = yface(etap, G, i, j + 1), eta_s = yface(etap, G, i, j);
    const double ce = eta_e / (dx * dx), cw = eta_w / (dx * dx);
    const double cn = 2.0 * eta_n / (dy * dy), cs = 2.0 * eta_s / (dy * dy);
    const double xe = eta_e / (dx * dy), xw = eta_w / (dx * dy);
    addv(i + 1, j, a * ce);
    addv(i - 1, j, a * cw);
    addv(i, j, -a * (ce + cw + cn + cs));
    addv(i, j + 1, a * cn);
    addv(i, j - 1, a * cs);
    addu(i + 1, j, a * xe);
    addu(i + 1, j - 1, -a * xe);
    addu(i, j, -a * xw);
    addu(i, j - 1, a * xw);
  }
}

// The interior value (si, sj) a ghost value at x-position i (outside [0, nx') or not) and interior row j
// copies under bc_xval, with the sign of the copy (-1 through a Dirichlet reflection); nx' = f.nx.
__device__ __forceinline__ double ghost_x_source(const Fv &f, const Grid &G, int kind, const BCSide &L,
                                                 const BCSide &R, int i, int &si) {
  const int nx = f.nx;
  if (i >= 0 && i < nx) {
    si = i;
    return 1.0;
  }
  const bool left = i < 0;
  const int g = left ? -i : i - (nx - 1);
  if (G.px) {
    si = (kind == kBCU) ? (left ? nx - g - 1 : g) : (left ? nx - g : g - 1);
    return 1.0;
  }
  if (kind == kBCScalar) {
    si = left ? 0 : nx - 1;
    return 1.0;
  }
  const BCSide &b = left ? L : R;
  si = (kind == kBCU) ? (left ? g : nx - 1 - g) : (left ? g - 1 : nx - g);
  return (b.type == DN_BC_DIRICHLET) ? -1.0 : 1.0;
}

// Adjoint of k_bc_ghosts: every ghost's cotangent moves (with the copy's sign) onto the interior value its BC
// reads, and the ghost's cotangent is cleared.  Ghost values are affine in one interior value each
// (k_bc_ghosts computes them from interior values only), so one pass with atomics suffices.
__global__ void k_adj_ghosts(Fv f, Grid G, int kind, BCSide L, BCSide R, BCSide B, BCSide T) {
  const int gw = f.g, nx = f.nx, ny = f.ny;
  const long long nxg = 2LL * gw * ny;
  const long long nyg = 2LL * gw * (nx + 2 * gw);
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, si, sj;
  double coef;
  if (t < nxg) {
    j = (int)(t % ny);
    const int k = (int)(t / ny);
    i = (k < gw) ? -(k + 1) : nx - 1 + (k - gw + 1);
    coef = ghost_x_source(f, G, kind, L, R, i, si);
    sj = j;
  } else {
    t -= nxg;
    if (t >= nyg) return;
    i = (int)(t % (nx + 2 * gw)) - gw;
    const int k = (int)(t / (nx + 2 * gw));
    const bool bottom = k < gw;
    const int g = bottom ? k + 1 : k - gw + 1;
    j = bottom ? -g : ny - 1 + g;
    double cy = 1.0;
    if (G.py) {
      sj = (kind == kBCV) ? (bottom ? ny - g - 1 : g) : (bottom ? ny - g : g - 1);
    } else if (kind == kBCScalar) {
      sj = bottom ? 0 : ny - 1;
    } else {
      const BCSide &b = bottom ? B : T;
      sj = (kind == kBCV) ? (bottom ? g : ny - 1 - g) : (bottom ? g - 1 : ny - g);
      cy = (b.type == DN_BC_DIRICHLET) ? -1.0 : 1.0;
    }
    coef = cy * ghost_x_source(f, G, kind, L, R, i, si);
  }
  const double gv = f.at(i, j);
  if (gv != 0.0) atomicAdd(&f.at(si, sj), coef * gv);
  f.at(i, j) = 0.0;
}

}  // namespace dn
