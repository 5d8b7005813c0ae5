// dn_momentum.cuh -- momentum predictor (solve_momentum_predictor, momentum.cpp:157-502) on the GPU.
//
// The monolithic u-v system is kept matrix-free-by-row: each active unknown owns 9 coefficients over a
// fixed target set (self, 4 same-component neighbours, 4 cross-component neighbours) plus a folded
// right-hand side.  The assembly kernel replays the reference's add_*_entry calls in the same order,
// including the Dirichlet / Neumann folding of boundary neighbours (momentum.cpp:309-393), so every fold
// lands on one of the 9 targets.  Unknown vector: u part (nx+1)*ny (index i*ny+j), then v part
// nx*(ny+1) (index NU + i*(ny+1)+j); inactive entries stay 0 in every Krylov vector.
#pragma once

#include "dn_fields.cuh"

namespace dn {

struct MomLayout {
  int nx, ny, px, py;
  long long nu, nv;  // sizes of the u and v parts
  __device__ __forceinline__ long long n() const { return nu + nv; }
  __device__ __forceinline__ bool u_active(int i, int j) const {
    if (j < 0 || j >= ny) return false;
    if (px) return !(i < 0 || i >= nx);
    return !(i <= 0 || i >= nx);
  }
  __device__ __forceinline__ bool v_active(int i, int j) const {
    if (i < 0 || i >= nx) return false;
    if (py) return !(j < 0 || j >= ny);
    return !(j <= 0 || j >= ny);
  }
  __device__ __forceinline__ int cui(int i) const { return !px ? i : (i < 0 ? nx - 1 : (i >= nx ? 0 : i)); }
  __device__ __forceinline__ int cuj(int j) const { return !py ? j : (j < 0 ? ny - 1 : (j >= ny ? 0 : j)); }
  __device__ __forceinline__ long long uidx(int i, int j) const { return (long long)i * ny + j; }
  __device__ __forceinline__ long long vidx(int i, int j) const { return nu + (long long)i * (ny + 1) + j; }
};

struct MomRowBuilder {
  long long tgt[9];
  double c[9];
  double rhs;
  __device__ __forceinline__ void add(long long t, double v) {
    for (int k = 0; k < 9; ++k)
      if (tgt[k] == t) {
        c[k] += v;
        return;
      }
  }
};

// Assembles coefficients, targets, rhs and x0 for every unknown (inactive unknowns: all zero, target -1).
__global__ void k_mom_assemble(MomLayout L, Grid G, BCSet bc, Fv u, Fv v, Fv rm, Fv eta, Fv urhs, Fv vrhs,
                               double alpha, double *coef, int *tgt, double *rhs, double *x0) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long N = L.n();
  if (t >= N) return;
  MomRowBuilder R;
  const double dx = G.dx, dy = G.dy;
  const bool is_u = t < L.nu;
  int i, j;
  if (is_u) {
    i = (int)(t / L.ny);
    j = (int)(t % L.ny);
  } else {
    i = (int)((t - L.nu) / (L.ny + 1));
    j = (int)((t - L.nu) % (L.ny + 1));
  }
  const bool active = is_u ? L.u_active(i, j) : L.v_active(i, j);
  if (!active) {
    for (int k = 0; k < 9; ++k) {
      coef[(size_t)k * N + t] = 0.0;
      tgt[(size_t)k * N + t] = -1;
    }
    rhs[t] = 0.0;
    x0[t] = 0.0;
    return;
  }
  const BCSide &lu = bc.u[DN_LEFT], &ru = bc.u[DN_RIGHT], &bu = bc.u[DN_BOTTOM], &tu = bc.u[DN_TOP];
  const BCSide &lv = bc.v[DN_LEFT], &rv = bc.v[DN_RIGHT], &bv = bc.v[DN_BOTTOM], &tv = bc.v[DN_TOP];
  // target sets (canonical indices; inactive targets keep an index that never matches an unknown)
  auto uT = [&](int ii, int jj) -> long long { return L.u_active(ii, jj) ? L.uidx(ii, jj) : -2; };
  auto vT = [&](int ii, int jj) -> long long { return L.v_active(ii, jj) ? L.vidx(ii, jj) : -2; };
  if (is_u) {
    R.tgt[0] = L.uidx(i, j);
    R.tgt[1] = uT(L.cui(i + 1), j);
    R.tgt[2] = uT(L.cui(i - 1), j);
    R.tgt[3] = uT(i, L.cuj(j + 1));
    R.tgt[4] = uT(i, L.cuj(j - 1));
    R.tgt[5] = vT(L.cui(i), L.cuj(j + 1));
    R.tgt[6] = vT(L.cui(i - 1), L.cuj(j + 1));
    R.tgt[7] = vT(L.cui(i), L.cuj(j));
    R.tgt[8] = vT(L.cui(i - 1), L.cuj(j));
  } else {
    R.tgt[0] = L.vidx(i, j);
    R.tgt[1] = vT(L.cui(i + 1), j);
    R.tgt[2] = vT(L.cui(i - 1), j);
    R.tgt[3] = vT(i, L.cuj(j + 1));
    R.tgt[4] = vT(i, L.cuj(j - 1));
    R.tgt[5] = uT(L.cui(i + 1), L.cuj(j));
    R.tgt[6] = uT(L.cui(i + 1), L.cuj(j - 1));
    R.tgt[7] = uT(L.cui(i), L.cuj(j));
    R.tgt[8] = uT(L.cui(i), L.cuj(j - 1));
  }
  for (int k = 0; k < 9; ++k) R.c[k] = 0.0;

  // add_u_x_entry, momentum.cpp:309-329
  auto add_u_x = [&](int ui, int uj, double value) {
    if (L.u_active(ui, uj)) {
      R.add(L.uidx(ui, uj), value);
      return;
    }
    const bool is_left = ui <= 0;
    const BCSide &b = is_left ? lu : ru;
    if (b.type == DN_BC_DIRICHLET) {
      R.rhs -= value * b.value;
    } else {
      const int ii = is_left ? 1 : L.nx - 1;
      R.add(L.uidx(ii, uj), value);
      R.rhs -= value * b.value * dx;
    }
  };
  // add_u_y_entry, momentum.cpp:331-350
  auto add_u_y = [&](int ui, int uj, double value) {
    if (L.u_active(ui, uj)) {
      R.add(L.uidx(ui, uj), value);
      return;
    }
    const bool is_bottom = uj < 0;
    const BCSide &b = is_bottom ? bu : tu;
    const int jj = is_bottom ? 0 : L.ny - 1;
    if (b.type == DN_BC_DIRICHLET) {
      R.add(L.uidx(ui, jj), -value);
      R.rhs -= value * (2.0 * b.value);
    } else {
      R.add(L.uidx(ui, jj), value);
      R.rhs -= value * b.value * dy;
    }
  };
  // add_v_y_entry, momentum.cpp:352-372
  auto add_v_y = [&](int vi, int vj, double value) {
    if (L.v_active(vi, vj)) {
      R.add(L.vidx(vi, vj), value);
      return;
    }
    const bool is_bottom = vj <= 0;
    const BCSide &b = is_bottom ? bv : tv;
    if (b.type == DN_BC_DIRICHLET) {
      R.rhs -= value * b.value;
    } else {
      const int jj = is_bottom ? 1 : L.ny - 1;
      R.add(L.vidx(vi, jj), value);
      R.rhs -= value * b.value * dy;
    }
  };
  // add_v_x_entry, momentum.cpp:374-393
  auto add_v_x = [&](int vi, int vj, double value) {
    if (L.v_active(vi, vj)) {
      R.add(L.vidx(vi, vj), value);
      return;
    }
    const bool is_left = vi < 0;
    const BCSide &b = is_left ? lv : rv;
    const int ii = is_left ? 0 : L.nx - 1;
    if (b.type == DN_BC_DIRICHLET) {
      R.add(L.vidx(ii, vj), -value);
      R.rhs -= value * (2.0 * b.value);
    } else {
      R.add(L.vidx(ii, vj), value);
      R.rhs -= value * b.value * dx;
    }
  };

  if (is_u) {  // momentum.cpp:395-429
    R.rhs = urhs.at(i, j);
    x0[t] = u.at(i, j);
    const double rf = xface(rm, G, i, j);
    const double eta_e = xface(eta, G, i + 1, j), eta_w = xface(eta, G, i, j);
    const double eta_n = corner(eta, i, j + 1), eta_s = corner(eta, i, j);
    const double ce = 2.0 * eta_e / (dx * dx), cw = 2.0 * eta_w / (dx * dx);
    const double cn = eta_n / (dy * dy), cs = eta_s / (dy * dy);
    const double xn = eta_n / (dx * dy), xs = eta_s / (dx * dy);
    R.c[0] += rf + alpha * (ce + cw + cn + cs);
    add_u_x(L.cui(i + 1), j, -alpha * ce);
    add_u_x(L.cui(i - 1), j, -alpha * cw);
    add_u_y(i, L.cuj(j + 1), -alpha * cn);
    add_u_y(i, L.cuj(j - 1), -alpha * cs);
    add_v_y(L.cui(i), L.cuj(j + 1), -alpha * xn);
    add_v_y(L.cui(i - 1), L.cuj(j + 1), alpha * xn);
    add_v_y(L.cui(i), L.cuj(j), alpha * xs);
    add_v_y(L.cui(i - 1), L.cuj(j), -alpha * xs);
  } else {  // momentum.cpp:431-465
    R.rhs = vrhs.at(i, j);
    x0[t] = v.at(i, j);
    const double rf = yface(rm, G, i, j);
    const double eta_e = corner(eta, i + 1, j), eta_w = corner(eta, i, j);
    const double eta_n = yface(eta, G, i, j + 1), eta_s = yface(eta, G, i, j);
    const double ce = eta_e / (dx * dx), cw = eta_w / (dx * dx);
    const double cn = 2.0 * eta_n / (dy * dy), cs = 2.0 * eta_s / (dy * dy);
    const double xe = eta_e / (dx * dy), xw = eta_w / (dx * dy);
    R.c[0] += rf + alpha * (ce + cw + cn + cs);
    add_v_x(L.cui(i + 1), j, -alpha * ce);
    add_v_x(L.cui(i - 1), j, -alpha * cw);
    add_v_y(i, L.cuj(j + 1), -alpha * cn);
    add_v_y(i, L.cuj(j - 1), -alpha * cs);
    add_u_x(L.cui(i + 1), L.cuj(j), -alpha * xe);
    add_u_x(L.cui(i + 1), L.cuj(j - 1), alpha * xe);
    add_u_x(L.cui(i), L.cuj(j), alpha * xw);
    add_u_x(L.cui(i), L.cuj(j - 1), -alpha * xw);
  }
  for (int k = 0; k < 9; ++k) {
    // finalize_row_maps drops |a| < 1e-18 (ch_sparse_krylov.hpp:116)
    const bool keep = R.tgt[k] >= 0 && fabs(R.c[k]) >= 1.0e-18;
    coef[(size_t)k * N + t] = keep ? R.c[k] : 0.0;
    tgt[(size_t)k * N + t] = keep ? (int)R.tgt[k] : -1;  // nu + nv < 2^31 (checked at creation)
  }
  rhs[t] = R.rhs;
}

// Momentum RHS, momentum.cpp:167-187
__global__ void k_mom_rhs_u(Fv u, Fv v, Fv rm, Fv etap, Fv hu, Fv hup, Fv fxu, Fv out, Grid G, int step, double dt,
                            double alpha, double bfx) {
  DN_FOR_INTERIOR(out);
  const double rf = xface(rm, G, i, j);
  const double conv = (step == 0) ? hu.at(i, j) : 1.5 * hu.at(i, j) - 0.5 * hup.at(i, j);
  const double vo = visc_u(u, v, etap, G, i, j);
  out.at(i, j) = rf * u.at(i, j) + dt * (-rf * conv + rf * bfx + fxu.at(i, j)) + alpha * vo;
}
__global__ void k_mom_rhs_v(Fv u, Fv v, Fv rm, Fv etap, Fv hv, Fv hvp, Fv fyv, Fv out, Grid G, int step, double dt,
                            double alpha, double bfy) {
  DN_FOR_INTERIOR(out);
  const double rf = yface(rm, G, i, j);
  const double conv = (step == 0) ? hv.at(i, j) : 1.5 * hv.at(i, j) - 0.5 * hvp.at(i, j);
  const double vo = visc_v(u, v, etap, G, i, j);
  out.at(i, j) = rf * v.at(i, j) + dt * (-rf * conv + rf * bfy + fyv.at(i, j)) + alpha * vo;
}

// Fused momentum convection + right-hand side (compute_momentum_fluxes, momentum.cpp:55-85, with the rhs of
// solve_momentum_predictor, :167-187): one thread per u face (t < nu) or v face, writing H (hu / hv) and the
// rhs (urhs / vrhs) in one pass.  The face BC that the flux arrays get before the rhs reads them
// (k_bc_faces_u / k_bc_faces_v) is applied in the thread: a wall boundary face takes the Dirichlet value or
// the next interior face's H (recomputed here) plus value * spacing; on a periodic side face nx (ny) takes
// face 0's H, computed from the same operands.  Bit-for-bit k_mom_flux_u/v + the face BC + k_mom_rhs_u/v;
// the caller still runs the ghost pass of H.  Algorithmic bytes per face: reads u, v, rho_mid, eta_prev,
// H_prev and the face force; writes H and the rhs (64 B).
__device__ __forceinline__ double mom_flux_u_at(const Fv &u, const Fv &v, const Grid &G, int i, int j) {
  const double uf = u.at(i, j);
  const double dudx = (u.at(i + 1, j) - u.at(i - 1, j)) / (2.0 * G.dx);
  const double dudy = (u.at(i, j + 1) - u.at(i, j - 1)) / (2.0 * G.dy);
  const double vf = 0.25 * (v.at(i - 1, j) + v.at(i, j) + v.at(i - 1, j + 1) + v.at(i, j + 1));
  return uf * dudx + vf * dudy;
}
__device__ __forceinline__ double mom_flux_v_at(const Fv &u, const Fv &v, const Grid &G, int i, int j) {
  const double vf = v.at(i, j);
  const double dvdx = (v.at(i + 1, j) - v.at(i - 1, j)) / (2.0 * G.dx);
  const double dvdy = (v.at(i, j + 1) - v.at(i, j - 1)) / (2.0 * G.dy);
  const double uf = 0.25 * (u.at(i, j - 1) + u.at(i, j) + u.at(i + 1, j - 1) + u.at(i + 1, j));
  return uf * dvdx + vf * dvdy;
}
__global__ void k_mom_conv_rhs(Fv u, Fv v, Fv rm, Fv etap, Fv hu, Fv hv, Fv hup, Fv hvp, Fv fxu, Fv fyv, Fv urhs,
                               Fv vrhs, Grid G, BCSide uL, BCSide uR, BCSide vB, BCSide vT, int step, double dt,
                               double alpha, double bfx, double bfy) {
  const long long nu = (long long)(G.nx + 1) * G.ny, nv = (long long)G.nx * (G.ny + 1);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nu) {
    const int i = (int)(t / G.ny), j = (int)(t - (t / G.ny) * G.ny);
    double h;
    if (G.px) {
      h = mom_flux_u_at(u, v, G, i == G.nx ? 0 : i, j);
    } else if (i == 0) {
      h = (uL.type == DN_BC_DIRICHLET) ? uL.value : mom_flux_u_at(u, v, G, 1, j) + uL.value * G.dx;
    } else if (i == G.nx) {
      h = (uR.type == DN_BC_DIRICHLET) ? uR.value : mom_flux_u_at(u, v, G, G.nx - 1, j) + uR.value * G.dx;
    } else {
      h = mom_flux_u_at(u, v, G, i, j);
    }
    hu.at(i, j) = h;
    const double rf = xface(rm, G, i, j);
    const double conv = (step == 0) ? h : 1.5 * h - 0.5 * hup.at(i, j);
    const double vo = visc_u(u, v, etap, G, i, j);
    urhs.at(i, j) = rf * u.at(i, j) + dt * (-rf * conv + rf * bfx + fxu.at(i, j)) + alpha * vo;
  } else if (t < nu + nv) {
    const long long q = t - nu;
    const int i = (int)(q / (G.ny + 1)), j = (int)(q - (q / (G.ny + 1)) * (G.ny + 1));
    double h;
    if (G.py) {
      h = mom_flux_v_at(u, v, G, i, j == G.ny ? 0 : j);
    } else if (j == 0) {
      h = (vB.type == DN_BC_DIRICHLET) ? vB.value : mom_flux_v_at(u, v, G, i, 1) + vB.value * G.dy;
    } else if (j == G.ny) {
      h = (vT.type == DN_BC_DIRICHLET) ? vT.value : mom_flux_v_at(u, v, G, i, G.ny - 1) + vT.value * G.dy;
    } else {
      h = mom_flux_v_at(u, v, G, i, j);
    }
    hv.at(i, j) = h;
    const double rf = yface(rm, G, i, j);
    const double conv = (step == 0) ? h : 1.5 * h - 0.5 * hvp.at(i, j);
    const double vo = visc_v(u, v, etap, G, i, j);
    vrhs.at(i, j) = rf * v.at(i, j) + dt * (-rf * conv + rf * bfy + fyv.at(i, j)) + alpha * vo;
  }
}

// scatter of the solution into u*, v* (momentum.cpp:474-489); u*, v* were copied from u, v first
__global__ void k_mom_scatter(MomLayout L, const double *x, Fv us, Fv vs) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= L.n()) return;
  if (t < L.nu) {
    const int i = (int)(t / L.ny), j = (int)(t % L.ny);
    if (L.u_active(i, j)) us.at(i, j) = x[t];
  } else {
    const int i = (int)((t - L.nu) / (L.ny + 1)), j = (int)((t - L.nu) % (L.ny + 1));
    if (L.v_active(i, j)) vs.at(i, j) = x[t];
  }
}

// ---------------------------------------------------------------------------------------------------
// Persistent Jacobi-BiCGSTAB (solve_preconditioned_bicgstab, ch_sparse_krylov.hpp:839-963)
// ---------------------------------------------------------------------------------------------------
struct BicgArgs {
  long long n;
  const double *coef;   // [9][n]
  const int *tgt;       // [9][n], -1 = no entry
  const double *b;
  double *x, *r, *rhat, *p0, *p1, *v0, *v1, *phat, *s, *shat, *t, *upd, *dinv;
  int max_it;
  double tol;
  int use_rel;
  unsigned int *bar_count, *bar_gen;
  int *status;
  double *partials;
  double *out;  // [0] iterations [1] abs residual [2] rel residual [3] iterate residual
};

__device__ __forceinline__ double mom_row_apply(const BicgArgs &P, long long r, const double *x) {
  double sum = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const int c = P.tgt[(size_t)k * P.n + r];
    if (c >= 0) sum += P.coef[(size_t)k * P.n + r] * x[c];
  }
  return sum;
}

__global__ void k_mom_dinv(BicgArgs P) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= P.n) return;
  const int c0 = P.tgt[r];
  P.dinv[r] = (c0 >= 0) ? 1.0 / max_ref(fabs(P.coef[r]), 1.0e-30) : 0.0;
}

__global__ void __launch_bounds__(kBlock) k_bicgstab(BicgArgs P) {
  __shared__ double sh[8 * 32 + 8];
  const GridBarrier bar{P.bar_count, P.bar_gen, P.status, gridDim.x};
  int parity = 0;
  const long long n = P.n;
  const long long per = (n + gridDim.x - 1) / gridDim.x;
  const long long lo = (long long)blockIdx.x * per, hi = min(n, lo + per);
  auto finish = [&](int its, double absr, double relr, double itres) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      P.out[0] = its;
      P.out[1] = absr;
      P.out[2] = relr;
      P.out[3] = itres;
    }
  };
  // r = b - A x (ch_sparse_krylov.hpp:855-869)
  double v2[2] = {0.0, 0.0};
  for (long long q = lo + threadIdx.x; q < hi; q += blockDim.x) {
    const double rr = P.b[q] - mom_row_apply(P, q, P.x);
    P.r[q] = rr;
    P.rhat[q] = rr;
    P.p0[q] = 0.0;
    P.v0[q] = 0.0;
    P.upd[q] = 0.0;
    v2[0] += P.b[q] * P.b[q];
    v2[1] += rr * rr;
  }
  if (!grid_sum<2>(v2, P.partials, parity, sh, bar)) return;
  const double rhs_norm = sqrt(max_ref(v2[0], 0.0));
  double absr = sqrt(max_ref(v2[1], 0.0));
  double relr = absr / max_ref(rhs_norm, 1.0e-30);
  if ((P.use_rel && relr < P.tol) || absr < P.tol) {
    finish(0, absr, relr, 0.0);
    return;
  }
  double rho_old = 1.0, alpha = 1.0, omega = 1.0;
  double rho_new = v2[1];  // r_hat = r, so r_hat . r = r . r (same partial sums)
  double *p_old = P.p0, *p_new = P.p1, *v_old = P.v0, *v_new = P.v1;
  const int limit = P.max_it > 1 ? P.max_it : 1;
  for (int it = 0; it < limit; ++it) {
    if (!isfinite(rho_new) || fabs(rho_new) < 1.0e-30) {
      if (threadIdx.x == 0) atomicCAS(P.status, kDevOk, kDevBicgRho);
      return;
    }
    const double beta = (it == 0) ? 0.0 : (rho_new / rho_old) * (alpha / omega);
    // p = r + beta (p - omega v); phat = D^-1 p (stored, then gathered: one load per neighbour)
    for (long long q = lo + threadIdx.x; q < hi; q += blockDim.x) {
      const double pq = P.r[q] + beta * (p_old[q] - omega * v_old[q]);
      p_new[q] = pq;
      P.phat[q] = P.dinv[q] * pq;
    }
    if (!bar.sync()) return;
    // v = A phat
    double a1[1] = {0.0};
    for (long long q = lo + threadIdx.x; q < hi; q += blockDim.x) {
      double sum = 0.0;
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const int c = P.tgt[(size_t)k * n + q];
        if (c >= 0) sum += P.coef[(size_t)k * n + q] * P.phat[c];
      }
      v_new[q] = sum;
      a1[0] += P.rhat[q] * sum;
    }
    if (!grid_sum<1>(a1, P.partials, parity, sh, bar)) return;
    const double rhat_v = a1[0];
    if (!isfinite(rhat_v) || fabs(rhat_v) < 1.0e-30) {
      if (threadIdx.x == 0) atomicCAS(P.status, kDevOk, kDevBicgRhatV);
      return;
    }
    alpha = rho_new / rhat_v;
    double a2[1] = {0.0};
    for (long long q = lo + threadIdx.x; q < hi; q += blockDim.x) {
      const double sv = P.r[q] - alpha * v_new[q];
      P.s[q] = sv;
      P.shat[q] = P.dinv[q] * sv;  // gathered by t = A shat after the barrier of the reduction below
      P.upd[q] = alpha * P.phat[q];
      a2[0] += sv * sv;
    }
    if (!grid_sum<1>(a2, P.partials, parity, sh, bar)) return;
    const double s_norm = sqrt(max_ref(a2[0], 0.0));
    if ((P.use_rel && s_norm / max_ref(rhs_norm, 1.0e-30) < P.tol) || s_norm < P.tol) {
      double a3[2] = {0.0, 0.0};
      for (long long q = lo + threadIdx.x; q < hi; q += blockDim.x) {
        const double xv = P.x[q] + P.upd[q];
        P.x[q] = xv;
        a3[0] += P.upd[q] * P.upd[q];
        a3[1] += xv * xv;
      }
      if (!grid_sum<2>(a3, P.partials, parity, sh, bar)) return;
      finish(it + 1, s_norm, s_norm / max_ref(rhs_norm, 1.0e-30), sqrt(a3[0] / max_ref(a3[1], 1.0e-30)));
      return;
    }
    // shat = D^-1 s; t = A shat
    double a4[2] = {0.0, 0.0};
    for (long long q = lo + threadIdx.x; q < hi; q += blockDim.x) {
      double sum = 0.0;
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const int c = P.tgt[(size_t)k * n + q];
        if (c >= 0) sum += P.coef[(size_t)k * n + q] * P.shat[c];
      }
      P.t[q] = sum;
      a4[0] += sum * sum;
      a4[1] += sum * P.s[q];
    }
    if (!grid_sum<2>(a4, P.partials, parity, sh, bar)) return;
    const double tt = a4[0];
    if (!isfinite(tt) || fabs(tt) < 1.0e-30) {
      if (threadIdx.x == 0) atomicCAS(P.status, kDevOk, kDevBicgTT);
      return;
    }
    omega = a4[1] / tt;
    if (!isfinite(omega) || fabs(omega) < 1.0e-30) {
      if (threadIdx.x == 0) atomicCAS(P.status, kDevOk, kDevBicgOmega);
      return;
    }
    double a5[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long q = lo + threadIdx.x; q < hi; q += blockDim.x) {
      const double uu = P.upd[q] + omega * P.shat[q];
      P.upd[q] = uu;
      const double xv = P.x[q] + uu;
      P.x[q] = xv;
      const double rv = P.s[q] - omega * P.t[q];
      P.r[q] = rv;
      a5[0] += uu * uu;
      a5[1] += xv * xv;
      a5[2] += rv * rv;
      a5[3] += P.rhat[q] * rv;
    }
    if (!grid_sum<4>(a5, P.partials, parity, sh, bar)) return;
    absr = sqrt(max_ref(a5[2], 0.0));
    relr = absr / max_ref(rhs_norm, 1.0e-30);
    const double itres = sqrt(a5[0] / max_ref(a5[1], 1.0e-30));
    if ((P.use_rel && relr < P.tol) || absr < P.tol) {
      finish(it + 1, absr, relr, itres);
      return;
    }
    finish(it + 1, absr, relr, itres);
    rho_old = rho_new;
    rho_new = a5[3];
    double *tp = p_old;
    p_old = p_new;
    p_new = tp;
    tp = v_old;
    v_old = v_new;
    v_new = tp;
  }
}

}  // namespace dn
