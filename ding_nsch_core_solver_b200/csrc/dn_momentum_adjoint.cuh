// dn_momentum_adjoint.cuh -- discrete adjoint of the momentum predictor (solve_momentum_predictor,
// momentum.cpp:157-502) as a map of the velocity state, at fixed materials.
//
// The map: (u, v, H_prev, f, rho_mid, eta, eta_prev) -> (u*, v*, H).  The inputs' BCs are applied (bc(u, kBCU), bc(v, kBCV)), the
// predictor right-hand side is formed (k_mom_conv_rhs: rho_face u + dt (-rho_face conv + rho_face g + f) +
// alpha visc(u, v; eta_prev), conv = H(u, v) on step 0 and 1.5 H - 0.5 H_prev after), the coupled system
// M(rho_mid, eta) x = rhs is solved, x is scattered to the active faces and the faces' BCs fill the rest.
// H = H(u, v) with its face BC is the next step's H_prev.  Its adjoint, for cotangents (gu*, gv*, gH):
//   1. fold the cotangent through the output face BCs (k_adj_fold_u / _v) and gather it at the active faces;
//   2. solve M^T lambda = g (M^T assembled from M's rows, solved by the same Jacobi-BiCGSTAB);
//   3. lambda is the cotangent of the right-hand side: f_bar = dt lambda, H_prev_bar = 0.5 dt rho_face lambda
//      (steps > 0), and (u, v)_bar collect rho_face lambda plus the transposed stencils of the centred
//      convection (linearised at the forward's u, v; with gH folded through H's face BC) and of the viscous
//      divergence (k_mom_rhs_adj); the materials' cotangents follow from -lambda^T dF/dm
//      (k_mom_material_adj);
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
// gh_u, gh_v: the (face-BC folded) cotangent of the map's H output, which enters the convection transposes
// with lambda's -dt rho_face (1 or 1.5).
__global__ void k_mom_rhs_adj(MomLayout L, Fv u, Fv v, Fv rm, Fv etap, Fv lu, Fv lv, Fv gh_u, Fv gh_v, Fv au, Fv av,
                              Fv afu, Fv afv, Fv ahu, Fv ahv, Grid G, int step, double dt, double alpha) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= L.n()) return;
  const double dx = G.dx, dy = G.dy;
  const double ch = (step == 0) ? 1.0 : 1.5;
  auto addu = [&](int i, int j, double val) { atomicAdd(&au.at(i, j), val); };
  auto addv = [&](int i, int j, double val) { atomicAdd(&av.at(i, j), val); };
  if (t < L.nu) {
    const int i = (int)(t / L.ny), j = (int)(t % L.ny);
    const double w = lu.at(i, j), gh = gh_u.at(i, j);
    if (w == 0.0 && gh == 0.0) return;
    const double rf = xface(rm, G, i, j);
    afu.at(i, j) = dt * w;
    if (step != 0) ahu.at(i, j) = 0.5 * dt * rf * w;
    addu(i, j, rf * w);
    // convection: H = uf * dudx + vf * dudy
    const double c = -dt * rf * ch * w + gh;
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
    const double w = lv.at(i, j), gh = gh_v.at(i, j);
    if (w == 0.0 && gh == 0.0) return;
    const double rf = yface(rm, G, i, j);
    afv.at(i, j) = dt * w;
    if (step != 0) ahv.at(i, j) = 0.5 * dt * rf * w;
    addv(i, j, rf * w);
    // convection: H = uf * dvdx + vf * dvdy
    const double c = -dt * rf * ch * w + gh;
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

// Cotangents of the materials, one thread per face with lambda != 0.  With the solution x (u*, v*; its BC
// ghosts filled), the row of the solved system is F = rf x - alpha visc(x; eta) - rhs(u, v; rf, eta_prev) = 0
// (M's Dirichlet / Neumann folds are the BC ghosts of x, their constants the rhs's folds), so for every
// material m:  dL/dm = -lambda^T dF/dm, that is
//   rf:       -lambda (x - u + dt conv - dt g)      onto rho_mid through xface / yface;
//   eta:      +alpha lambda dvisc(x; eta)/deta       onto the face / corner means of eta;
//   eta_prev: +alpha lambda dvisc(u; eta_prev)/deta  the same with the forward's u, v.
// The corner means read eta's ghosts; the caller moves those cotangents with k_adj_ghosts (scalar BC).
__device__ __forceinline__ void add_face_mean(const Fv &a, const Grid &G, bool xdir, int i, int j, double val) {
  // adjoint of xface(f, G, i, j) (xdir) / yface(f, G, i, j)
  const int n = xdir ? G.nx : G.ny, k = xdir ? i : j;
  const int per = xdir ? G.px : G.py;
  auto at = [&](int kk) -> double & { return xdir ? a.at(kk, j) : a.at(i, kk); };
  if (k <= 0 || k >= n) {
    if (per) {
      atomicAdd(&at(n - 1), 0.5 * val);
      atomicAdd(&at(0), 0.5 * val);
    } else {
      atomicAdd(&at(k <= 0 ? 0 : n - 1), val);
    }
  } else {
    atomicAdd(&at(k - 1), 0.5 * val);
    atomicAdd(&at(k), 0.5 * val);
  }
}
__device__ __forceinline__ void add_corner_mean(const Fv &a, int i, int j, double val) {
  // adjoint of corner(f, i, j)
  const double q = 0.25 * val;
  atomicAdd(&a.at(i, j), q);
  atomicAdd(&a.at(i - 1, j), q);
  atomicAdd(&a.at(i, j - 1), q);
  atomicAdd(&a.at(i - 1, j - 1), q);
}
// d visc_u(x) / d (eta_e, eta_w, eta_n, eta_s) scaled by s, onto eta (momentum.cpp:91-155 terms)
__device__ __forceinline__ void visc_u_eta_adj(const Fv &x, const Fv &y, const Fv &a, const Grid &G, int i, int j,
                                               double s) {
  const double dudx_e = (x.at(i + 1, j) - x.at(i, j)) / G.dx, dudx_w = (x.at(i, j) - x.at(i - 1, j)) / G.dx;
  const double dudy_n = (x.at(i, j + 1) - x.at(i, j)) / G.dy, dudy_s = (x.at(i, j) - x.at(i, j - 1)) / G.dy;
  const double dvdx_n = (y.at(i, j + 1) - y.at(i - 1, j + 1)) / G.dx, dvdx_s = (y.at(i, j) - y.at(i - 1, j)) / G.dx;
  add_face_mean(a, G, true, i + 1, j, s * 2.0 * dudx_e / G.dx);
  add_face_mean(a, G, true, i, j, -s * 2.0 * dudx_w / G.dx);
  add_corner_mean(a, i, j + 1, s * (dudy_n + dvdx_n) / G.dy);
  add_corner_mean(a, i, j, -s * (dudy_s + dvdx_s) / G.dy);
}
__device__ __forceinline__ void visc_v_eta_adj(const Fv &x, const Fv &y, const Fv &a, const Grid &G, int i, int j,
                                               double s) {
  // x: u, y: v
  const double dvdx_e = (y.at(i + 1, j) - y.at(i, j)) / G.dx, dvdx_w = (y.at(i, j) - y.at(i - 1, j)) / G.dx;
  const double dvdy_n = (y.at(i, j + 1) - y.at(i, j)) / G.dy, dvdy_s = (y.at(i, j) - y.at(i, j - 1)) / G.dy;
  const double dudy_e = (x.at(i + 1, j) - x.at(i + 1, j - 1)) / G.dy, dudy_w = (x.at(i, j) - x.at(i, j - 1)) / G.dy;
  add_corner_mean(a, i + 1, j, s * (dvdx_e + dudy_e) / G.dx);
  add_corner_mean(a, i, j, -s * (dvdx_w + dudy_w) / G.dx);
  add_face_mean(a, G, false, i, j + 1, s * 2.0 * dvdy_n / G.dy);
  add_face_mean(a, G, false, i, j, -s * 2.0 * dvdy_s / G.dy);
}
__global__ void k_mom_material_adj(MomLayout L, Fv us, Fv vs, Fv u, Fv v, Fv hup, Fv hvp, Fv lu, Fv lv, Fv arho,
                                   Fv aeta, Fv aetap, Grid G, int step, double dt, double alpha, double bfx,
                                   double bfy) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= L.n()) return;
  if (t < L.nu) {
    const int i = (int)(t / L.ny), j = (int)(t % L.ny);
    const double w = lu.at(i, j);
    if (w == 0.0) return;
    const double h = mom_flux_u_at(u, v, G, i, j);
    const double conv = (step == 0) ? h : 1.5 * h - 0.5 * hup.at(i, j);
    add_face_mean(arho, G, true, i, j, -w * (us.at(i, j) - u.at(i, j) + dt * conv - dt * bfx));
    visc_u_eta_adj(us, vs, aeta, G, i, j, alpha * w);
    visc_u_eta_adj(u, v, aetap, G, i, j, alpha * w);
  } else {
    const long long q = t - L.nu;
    const int i = (int)(q / (L.ny + 1)), j = (int)(q % (L.ny + 1));
    const double w = lv.at(i, j);
    if (w == 0.0) return;
    const double h = mom_flux_v_at(u, v, G, i, j);
    const double conv = (step == 0) ? h : 1.5 * h - 0.5 * hvp.at(i, j);
    add_face_mean(arho, G, false, i, j, -w * (vs.at(i, j) - v.at(i, j) + dt * conv - dt * bfy));
    visc_v_eta_adj(us, vs, aeta, G, i, j, alpha * w);
    visc_v_eta_adj(u, v, aetap, G, i, j, alpha * w);
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

// ---------------------------------------------------------------------------------------------------
// Adjoint of the face surface forces (update_surface_tension_force, phase_field.cpp:179-226, no smoothing):
// c_mid = (c_old + c_new) / 2 (scalar BC ghosts), mu_mid = chem(c_mid), f_u = scale mf (c_mid(i) - c_mid(i-1)) / dx
// with mf the face mean of mu_mid (0.5 (mu(nx-1) + mu(0)) on faces 0 and nx), f_v likewise; the forces'
// face BCs are folded by the caller.  Cotangents are accumulated with atomics into cmb (c_mid, ghosted) and
// mmb (mu_mid, interior).
// ---------------------------------------------------------------------------------------------------
__global__ void k_sf_adj_faces(Fv gfu, Fv gfv, Fv cm, Fv mm, Fv cmb, Fv mmb, Grid G, double scale) {
  const long long nu = (long long)(G.nx + 1) * G.ny, nv = (long long)G.nx * (G.ny + 1);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nu) {
    const int i = (int)(t / G.ny), j = (int)(t % G.ny);
    const double g = gfu.at(i, j);
    if (g == 0.0) return;
    const bool edge = i <= 0 || i >= G.nx;
    const int ia = edge ? G.nx - 1 : i - 1, ib = edge ? 0 : i;
    const double mf = 0.5 * (mm.at(ia, j) + mm.at(ib, j));
    const double gr = (cm.at(i, j) - cm.at(i - 1, j)) / G.dx;
    atomicAdd(&mmb.at(ia, j), 0.5 * scale * gr * g);
    atomicAdd(&mmb.at(ib, j), 0.5 * scale * gr * g);
    atomicAdd(&cmb.at(i, j), scale * mf * g / G.dx);
    atomicAdd(&cmb.at(i - 1, j), -scale * mf * g / G.dx);
  } else if (t < nu + nv) {
    const long long q = t - nu;
    const int i = (int)(q / (G.ny + 1)), j = (int)(q % (G.ny + 1));
    const double g = gfv.at(i, j);
    if (g == 0.0) return;
    const bool edge = j <= 0 || j >= G.ny;
    const int ja = edge ? G.ny - 1 : j - 1, jb = edge ? 0 : j;
    const double mf = 0.5 * (mm.at(i, ja) + mm.at(i, jb));
    const double gr = (cm.at(i, j) - cm.at(i, j - 1)) / G.dy;
    atomicAdd(&mmb.at(i, ja), 0.5 * scale * gr * g);
    atomicAdd(&mmb.at(i, jb), 0.5 * scale * gr * g);
    atomicAdd(&cmb.at(i, j), scale * mf * g / G.dy);
    atomicAdd(&cmb.at(i, j - 1), -scale * mf * g / G.dy);
  }
}
// chem (k_chem: mu = alpha (dw(c) / cn - cn lap c), dw = c (1 - c) (1 - 2 c) / 2) transposed at cell (i, j)
__global__ void k_chem_adj(Fv cm, Fv mmb, Fv cmb, Grid G, double cn) {
  DN_FOR_INTERIOR(cm);
  const double g = mmb.at(i, j);
  if (g == 0.0) return;
  const double alpha = 6.0 * 1.4142135623730950488;
  const double c = cm.at(i, j);
  const double dwp = 0.5 * (1.0 - 6.0 * c + 6.0 * c * c);
  const double a = alpha * g, l = -a * cn;
  const double cx = 1.0 / (G.dx * G.dx), cy = 1.0 / (G.dy * G.dy);
  atomicAdd(&cmb.at(i, j), a * dwp / cn - 2.0 * l * (cx + cy));
  atomicAdd(&cmb.at(i + 1, j), l * cx);
  atomicAdd(&cmb.at(i - 1, j), l * cx);
  atomicAdd(&cmb.at(i, j + 1), l * cy);
  atomicAdd(&cmb.at(i, j - 1), l * cy);
}
// ---------------------------------------------------------------------------------------------------
// rho_mid cotangent of the projection (build_pressure_linear_system, pressure.cpp:123-196; the split
// explicit divergence, operators.cpp:424-444; the correction, operators.cpp:490-516), one thread per face,
// given the folded face cotangents (fu, fv) of the corrected velocities, rbar = A^-T (cotangent of p_corr)
// (compact, projected), the forward's p_corr (pc) and extrapolated pressure (pe), both with pressure-BC
// ghosts.  Per face with density rf = xface / yface(rho_mid):
//   correction u -= dt (a dx(pc) + b dx(pe)), a = 1/rf (variable) or 1/rho_ref, b = 1/rf - 1/rho_ref (split)
//       -> rf_bar += f_bar dt / rf^2 dx(pc or pe);
//   split rhs  -= div(w dx(pe)), w = 1 - rho_ref / rf   -> rf_bar += F_bar dx(pe) rho_ref / rf^2;
//   variable operator coefficient c = 1 / (rf h^2): open face  c_bar = -(rbar_a - rbar_b)(pc_a - pc_b);
//       Dirichlet side c_bar = rbar_r (2 value - 2 pc_r); Neumann side c_bar = rbar_r value h
//       -> rf_bar += c_bar (-1 / (rf^2 h^2)).
// The face means are transposed onto rho_mid's cells (add_face_mean).  A periodic face shared by the last and
// the first cell is counted once for the operator (face 0) and once per side for the split flux.
// ---------------------------------------------------------------------------------------------------
__global__ void k_proj_rho_adj(Fv fu, Fv fv, const double *rbar, Fv pc, Fv pe, Fv rm, Fv arho, Grid G, BCSet bc,
                               int split, double rho_ref, double dt) {
  const long long nu = (long long)(G.nx + 1) * G.ny, nv = (long long)G.nx * (G.ny + 1);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nu + nv) return;
  const bool xd = t < nu;
  int i, j;
  if (xd) {
    i = (int)(t / G.ny);
    j = (int)(t % G.ny);
  } else {
    const long long q = t - nu;
    i = (int)(q / (G.ny + 1));
    j = (int)(q % (G.ny + 1));
  }
  const int n = xd ? G.nx : G.ny, k = xd ? i : j, per = xd ? G.px : G.py;
  const double h = xd ? G.dx : G.dy;
  const double rf = xd ? xface(rm, G, i, j) : yface(rm, G, i, j);
  const double dpc = xd ? gfx(pc, G, i, j) : gfy(pc, G, i, j);
  const double dpe = split ? (xd ? gfx(pe, G, i, j) : gfy(pe, G, i, j)) : 0.0;
  const double fb = xd ? fu.at(i, j) : fv.at(i, j);
  double bar = fb * dt / (rf * rf) * (split ? dpe : dpc);
  auto rb = [&](int kk) { return rbar[xd ? (long long)kk * G.ny + j : (long long)i * G.ny + kk]; };
  const bool open = per || (k > 0 && k < n);
  if (split) {
    if (open) {
      const double e = k < n ? rb(k) : 0.0, w = k > 0 ? rb(k - 1) : 0.0;
      bar += (e - w) / h * dpe * rho_ref / (rf * rf);
    }
  } else {
    double cbar = 0.0;
    if (open) {
      if (!(per && k == n)) {
        const int a = k > 0 ? k - 1 : n - 1, b = k < n ? k : 0;
        const double pa = xd ? pc.at(a, j) : pc.at(i, a), pb = xd ? pc.at(b, j) : pc.at(i, b);
        cbar = -(rb(a) - rb(b)) * (pa - pb);
      }
    } else {
      const int r = k <= 0 ? 0 : n - 1;
      const BCSide &side = bc.p[xd ? (k <= 0 ? DN_LEFT : DN_RIGHT) : (k <= 0 ? DN_BOTTOM : DN_TOP)];
      const double pr = xd ? pc.at(r, j) : pc.at(i, r);
      cbar = (side.type == DN_BC_DIRICHLET) ? rb(r) * (2.0 * side.value - 2.0 * pr) : rb(r) * side.value * h;
    }
    bar += cbar * (-1.0 / (rf * rf * h * h));
  }
  if (bar != 0.0) add_face_mean(arho, G, xd, i, j, bar);
}

// out = in / 2 at the interior cells
__global__ void k_half_interior(Fv in, Fv out) {
  DN_FOR_INTERIOR(out);
  out.at(i, j) = 0.5 * in.at(i, j);
}

}  // namespace dn
