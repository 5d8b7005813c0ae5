/*
 * dn_oracle.c -- CPU restatement of the reference CHNS time step (TEST INFRASTRUCTURE ONLY).
 *
 * Parity status: pinned.  This file is checked bit for bit against the reference compiled from its
 * own sources (oracle/_ref, built by oracle/Makefile) and against the reference's published golden
 * run (176Result/static_droplet_surface_tension_validation_128, reduced into tests/golden/).
 *
 * Every function restates one reference function, cited by file:line inside the reference project.
 * Expressions keep the reference's operand order on purpose: the oracle must reproduce the
 * reference's IEEE-754 double results exactly (compile with -O2 -ffp-contract=off, no -ffast-math).
 * The CUDA product never links or calls this code.
 */
#include "dn_oracle.h"

#include <math.h>
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define KSQRT2 1.4142135623730950488
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------------------------------ */
/* Field2D (field.hpp:9-36)                                                                    */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
  int nx, ny, g;
  double *d;
} fld;

#define AT(f, i, j) ((f)->d[(size_t)((i) + (f)->g) * (size_t)((f)->ny + 2 * (f)->g) + (size_t)((j) + (f)->g)])

static size_t fld_size(const fld *f) { return (size_t)(f->nx + 2 * f->g) * (size_t)(f->ny + 2 * f->g); }

static void fld_init(fld *f, int nx, int ny, int g, double v) {
  f->nx = nx;
  f->ny = ny;
  f->g = g;
  f->d = (double *)malloc(fld_size(f) * sizeof(double));
  for (size_t k = 0; k < fld_size(f); ++k) f->d[k] = v;
}
static void fld_free(fld *f) {
  free(f->d);
  f->d = NULL;
}
static void fld_fill(fld *f, double v) {
  for (size_t k = 0; k < fld_size(f); ++k) f->d[k] = v;
}
static void fld_copy(fld *dst, const fld *src) { memcpy(dst->d, src->d, fld_size(src) * sizeof(double)); }

/* ------------------------------------------------------------------------------------------ */
/* Sparse CSR (ch_sparse_krylov.hpp:12-18) and std::map-style row accumulation                */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
  int n;
  int *row_ptr, *col, *diag_pos;
  double *val;
  int nnz, cap;
} csr;

typedef struct {
  int cnt;
  int col[64];
  double val[64];
} rowacc; /* one std::map<int,double> row: operator[] inserts 0.0, then += */

static void ra_clear(rowacc *r) { r->cnt = 0; }
static void ra_add(rowacc *r, int col, double v) {
  for (int k = 0; k < r->cnt; ++k) {
    if (r->col[k] == col) {
      r->val[k] += v;
      return;
    }
  }
  r->col[r->cnt] = col;
  r->val[r->cnt] = 0.0 + v;
  r->cnt++;
}
static void ra_sort(rowacc *r) {
  for (int a = 1; a < r->cnt; ++a) {
    int c = r->col[a];
    double v = r->val[a];
    int b = a - 1;
    while (b >= 0 && r->col[b] > c) {
      r->col[b + 1] = r->col[b];
      r->val[b + 1] = r->val[b];
      --b;
    }
    r->col[b + 1] = c;
    r->val[b + 1] = v;
  }
}

static void csr_reset(csr *m, int n, int cap) {
  if (m->cap < cap) {
    free(m->col);
    free(m->val);
    m->col = (int *)malloc((size_t)cap * sizeof(int));
    m->val = (double *)malloc((size_t)cap * sizeof(double));
    m->cap = cap;
  }
  if (m->n != n || !m->row_ptr) {
    free(m->row_ptr);
    free(m->diag_pos);
    m->row_ptr = (int *)malloc((size_t)(n + 1) * sizeof(int));
    m->diag_pos = (int *)malloc((size_t)n * sizeof(int));
  }
  m->n = n;
  m->nnz = 0;
  m->row_ptr[0] = 0;
}
static void csr_free(csr *m) {
  free(m->row_ptr);
  free(m->col);
  free(m->diag_pos);
  free(m->val);
  memset(m, 0, sizeof(*m));
}

/* ------------------------------------------------------------------------------------------ */
/* Solver state (solver.hpp:64-130)                                                            */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
  int type; /* 0 diagonal, 1 ildlt, 2 icc */
  double *diagonal_inverse;
  double *lower; /* aligned with csr val */
  double *diag;
  int *lt_ptr, *lt_row; /* lower_transpose as CSR over rows */
  double *lt_val;
  double diagonal_floor;
  int n, cap;
} precond;

typedef double (*proj_fn)(void *ctx, double *v, int n);

struct orc_solver {
  orc_config cfg;
  double dx, dy;
  fld f[ORC_F_COUNT];
  double initial_mass;
  int current_step_index;
  orc_report rep;
  /* CH caches (solver.hpp:112-117) */
  int ch_ops_ready;
  csr ch_lap, ch_biharm, ch_sys;
  double ch_cached_alpha0;
  precond ch_pc;
  /* scratch */
  csr pm;      /* pressure / momentum matrix */
  precond ppc; /* pressure / momentum preconditioner */
  double *w[16];
  int wn;
  rowacc *rows; /* assembly rows */
  int nrows_cap;
  char err[256];
  jmp_buf *jb;
  double *mon;      /* CG monitor record of the last pressure solve, [iteration][4] */
  int mon_cap, mon_count, mon_active;
};

static void fail(orc_solver *s, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(s->err, sizeof(s->err), fmt, ap);
  va_end(ap);
  if (s->jb) longjmp(*s->jb, 1);
}

static double sq(double v) { return v * v; }
/* std::max / std::min (a NaN first argument passes through), as the reference calls them */
static double dmax(double a, double b) { return (a < b) ? b : a; }
static double dmin(double a, double b) { return (b < a) ? b : a; }

static rowacc *rows_get(orc_solver *s, int n) {
  if (s->nrows_cap < n) {
    free(s->rows);
    s->rows = (rowacc *)malloc((size_t)n * sizeof(rowacc));
    s->nrows_cap = n;
  }
  for (int r = 0; r < n; ++r) ra_clear(&s->rows[r]);
  return s->rows;
}

/* finalize_row_maps, ch_sparse_krylov.hpp:105-133 */
static void finalize_rows(orc_solver *s, rowacc *rows, int n, csr *m) {
  int cap = 0;
  for (int r = 0; r < n; ++r) cap += rows[r].cnt;
  csr_reset(m, n, cap > 0 ? cap : 1);
  for (int r = 0; r < n; ++r) {
    ra_sort(&rows[r]);
    m->diag_pos[r] = -1;
    for (int k = 0; k < rows[r].cnt; ++k) {
      if (fabs(rows[r].val[k]) < 1.0e-18) continue;
      m->col[m->nnz] = rows[r].col[k];
      m->val[m->nnz] = rows[r].val[k];
      if (rows[r].col[k] == r) m->diag_pos[r] = m->nnz;
      m->nnz++;
    }
    m->row_ptr[r + 1] = m->nnz;
  }
  for (int r = 0; r < n; ++r)
    if (m->diag_pos[r] < 0) fail(s, "sparse matrix assembly failed to produce a diagonal entry");
}

/* ------------------------------------------------------------------------------------------ */
/* Boundary conditions (operators.cpp:36-289)                                                  */
/* ------------------------------------------------------------------------------------------ */
static orc_bc eff_p_bc(const orc_solver *s, int side) {
  if (s->cfg.p_bc[side].type != ORC_BC_UNSET) return s->cfg.p_bc[side];
  orc_bc b = {ORC_BC_NEUMANN, 0.0};
  return b;
}
static orc_bc eff_u_bc(const orc_solver *s, int side) {
  if (s->cfg.u_bc[side].type != ORC_BC_UNSET) return s->cfg.u_bc[side];
  orc_bc b = {ORC_BC_DIRICHLET, 0.0};
  if (side == ORC_BOTTOM) b.value = s->cfg.bottom_wall_velocity_x;
  if (side == ORC_TOP) b.value = s->cfg.top_wall_velocity_x;
  return b;
}
static orc_bc eff_v_bc(const orc_solver *s, int side) {
  if (s->cfg.v_bc[side].type != ORC_BC_UNSET) return s->cfg.v_bc[side];
  orc_bc b = {ORC_BC_DIRICHLET, 0.0};
  return b;
}
static int pressure_has_dirichlet(const orc_solver *s) {
  if (!s->cfg.periodic_x) {
    if (eff_p_bc(s, ORC_LEFT).type == ORC_BC_DIRICHLET || eff_p_bc(s, ORC_RIGHT).type == ORC_BC_DIRICHLET) return 1;
  }
  if (!s->cfg.periodic_y) {
    if (eff_p_bc(s, ORC_BOTTOM).type == ORC_BC_DIRICHLET || eff_p_bc(s, ORC_TOP).type == ORC_BC_DIRICHLET) return 1;
  }
  return 0;
}

/* apply_scalar_bc, operators.cpp:130-141 */
static void bc_scalar(const orc_solver *s, fld *f) {
  const int px = s->cfg.periodic_x, py = s->cfg.periodic_y;
  for (int g = 1; g <= f->g; ++g) {
    for (int j = 0; j < f->ny; ++j) {
      AT(f, -g, j) = px ? AT(f, f->nx - g, j) : AT(f, 0, j);
      AT(f, f->nx - 1 + g, j) = px ? AT(f, g - 1, j) : AT(f, f->nx - 1, j);
    }
    for (int i = -f->g; i < f->nx + f->g; ++i) {
      AT(f, i, -g) = py ? AT(f, i, f->ny - g) : AT(f, i, 0);
      AT(f, i, f->ny - 1 + g) = py ? AT(f, i, g - 1) : AT(f, i, f->ny - 1);
    }
  }
}

/* apply_pressure_bc, operators.cpp:143-181 */
static void bc_pressure(const orc_solver *s, fld *f) {
  const orc_bc lb = eff_p_bc(s, ORC_LEFT), rb = eff_p_bc(s, ORC_RIGHT);
  const orc_bc bb = eff_p_bc(s, ORC_BOTTOM), tb = eff_p_bc(s, ORC_TOP);
  for (int g = 1; g <= f->g; ++g) {
    for (int j = 0; j < f->ny; ++j) {
      if (s->cfg.periodic_x) {
        AT(f, -g, j) = AT(f, f->nx - g, j);
        AT(f, f->nx - 1 + g, j) = AT(f, g - 1, j);
      } else {
        const double lo = 2.0 * ((double)g - 0.5) * lb.value * s->dx;
        const double ro = 2.0 * ((double)g - 0.5) * rb.value * s->dx;
        AT(f, -g, j) = (lb.type == ORC_BC_DIRICHLET) ? 2.0 * lb.value - AT(f, g - 1, j) : AT(f, g - 1, j) + lo;
        AT(f, f->nx - 1 + g, j) =
            (rb.type == ORC_BC_DIRICHLET) ? 2.0 * rb.value - AT(f, f->nx - g, j) : AT(f, f->nx - g, j) + ro;
      }
    }
    for (int i = -f->g; i < f->nx + f->g; ++i) {
      if (s->cfg.periodic_y) {
        AT(f, i, -g) = AT(f, i, f->ny - g);
        AT(f, i, f->ny - 1 + g) = AT(f, i, g - 1);
      } else {
        const double bo = 2.0 * ((double)g - 0.5) * bb.value * s->dy;
        const double to = 2.0 * ((double)g - 0.5) * tb.value * s->dy;
        AT(f, i, -g) = (bb.type == ORC_BC_DIRICHLET) ? 2.0 * bb.value - AT(f, i, g - 1) : AT(f, i, g - 1) + bo;
        AT(f, i, f->ny - 1 + g) =
            (tb.type == ORC_BC_DIRICHLET) ? 2.0 * tb.value - AT(f, i, f->ny - g) : AT(f, i, f->ny - g) + to;
      }
    }
  }
}

/* apply_u_bc, operators.cpp:183-233 */
static void bc_u(const orc_solver *s, fld *f) {
  const orc_bc lb = eff_u_bc(s, ORC_LEFT), rb = eff_u_bc(s, ORC_RIGHT);
  const orc_bc bb = eff_u_bc(s, ORC_BOTTOM), tb = eff_u_bc(s, ORC_TOP);
  if (s->cfg.periodic_x) {
    for (int j = 0; j < f->ny; ++j) AT(f, f->nx - 1, j) = AT(f, 0, j);
  } else {
    for (int j = 0; j < f->ny; ++j) {
      AT(f, 0, j) = (lb.type == ORC_BC_DIRICHLET) ? lb.value : AT(f, 1, j) + lb.value * s->dx;
      AT(f, f->nx - 1, j) = (rb.type == ORC_BC_DIRICHLET) ? rb.value : AT(f, f->nx - 2, j) + rb.value * s->dx;
    }
  }
  for (int g = 1; g <= f->g; ++g) {
    for (int j = 0; j < f->ny; ++j) {
      if (s->cfg.periodic_x) {
        AT(f, -g, j) = AT(f, f->nx - g - 1, j);
        AT(f, f->nx - 1 + g, j) = AT(f, g, j);
      } else {
        const double lo = 2.0 * (double)g * lb.value * s->dx;
        const double ro = 2.0 * (double)g * rb.value * s->dx;
        AT(f, -g, j) = (lb.type == ORC_BC_DIRICHLET) ? 2.0 * lb.value - AT(f, g, j) : AT(f, g, j) + lo;
        AT(f, f->nx - 1 + g, j) =
            (rb.type == ORC_BC_DIRICHLET) ? 2.0 * rb.value - AT(f, f->nx - 1 - g, j) : AT(f, f->nx - 1 - g, j) + ro;
      }
    }
    for (int i = -f->g; i < f->nx + f->g; ++i) {
      if (s->cfg.periodic_y) {
        AT(f, i, -g) = AT(f, i, f->ny - g);
        AT(f, i, f->ny - 1 + g) = AT(f, i, g - 1);
      } else {
        const double bo = 2.0 * ((double)g - 0.5) * bb.value * s->dy;
        const double to = 2.0 * ((double)g - 0.5) * tb.value * s->dy;
        AT(f, i, -g) = (bb.type == ORC_BC_DIRICHLET) ? 2.0 * bb.value - AT(f, i, g - 1) : AT(f, i, g - 1) + bo;
        AT(f, i, f->ny - 1 + g) =
            (tb.type == ORC_BC_DIRICHLET) ? 2.0 * tb.value - AT(f, i, f->ny - g) : AT(f, i, f->ny - g) + to;
      }
    }
  }
}

/* apply_v_bc, operators.cpp:239-289 */
static void bc_v(const orc_solver *s, fld *f) {
  const orc_bc lb = eff_v_bc(s, ORC_LEFT), rb = eff_v_bc(s, ORC_RIGHT);
  const orc_bc bb = eff_v_bc(s, ORC_BOTTOM), tb = eff_v_bc(s, ORC_TOP);
  if (s->cfg.periodic_y) {
    for (int i = 0; i < f->nx; ++i) AT(f, i, f->ny - 1) = AT(f, i, 0);
  } else {
    for (int i = 0; i < f->nx; ++i) {
      AT(f, i, 0) = (bb.type == ORC_BC_DIRICHLET) ? bb.value : AT(f, i, 1) + bb.value * s->dy;
      AT(f, i, f->ny - 1) = (tb.type == ORC_BC_DIRICHLET) ? tb.value : AT(f, i, f->ny - 2) + tb.value * s->dy;
    }
  }
  for (int g = 1; g <= f->g; ++g) {
    for (int j = 0; j < f->ny; ++j) {
      if (s->cfg.periodic_x) {
        AT(f, -g, j) = AT(f, f->nx - g, j);
        AT(f, f->nx - 1 + g, j) = AT(f, g - 1, j);
      } else {
        const double lo = 2.0 * ((double)g - 0.5) * lb.value * s->dx;
        const double ro = 2.0 * ((double)g - 0.5) * rb.value * s->dx;
        AT(f, -g, j) = (lb.type == ORC_BC_DIRICHLET) ? 2.0 * lb.value - AT(f, g - 1, j) : AT(f, g - 1, j) + lo;
        AT(f, f->nx - 1 + g, j) =
            (rb.type == ORC_BC_DIRICHLET) ? 2.0 * rb.value - AT(f, f->nx - g, j) : AT(f, f->nx - g, j) + ro;
      }
    }
    for (int i = -f->g; i < f->nx + f->g; ++i) {
      if (s->cfg.periodic_y) {
        AT(f, i, -g) = AT(f, i, f->ny - g - 1);
        AT(f, i, f->ny - 1 + g) = AT(f, i, g);
      } else {
        const double bo = 2.0 * (double)g * bb.value * s->dy;
        const double to = 2.0 * (double)g * tb.value * s->dy;
        AT(f, i, -g) = (bb.type == ORC_BC_DIRICHLET) ? 2.0 * bb.value - AT(f, i, g) : AT(f, i, g) + bo;
        AT(f, i, f->ny - 1 + g) =
            (tb.type == ORC_BC_DIRICHLET) ? 2.0 * tb.value - AT(f, i, f->ny - 1 - g) : AT(f, i, f->ny - 1 - g) + to;
      }
    }
  }
}

/* ------------------------------------------------------------------------------------------ */
/* Stencils and face interpolation (operators.cpp:299-398)                                     */
/* ------------------------------------------------------------------------------------------ */
static double lap_c(const orc_solver *s, const fld *f, int i, int j) {
  return (AT(f, i + 1, j) - 2.0 * AT(f, i, j) + AT(f, i - 1, j)) / (s->dx * s->dx) +
         (AT(f, i, j + 1) - 2.0 * AT(f, i, j) + AT(f, i, j - 1)) / (s->dy * s->dy);
}
static double gcx(const orc_solver *s, const fld *f, int i, int j) {
  return (AT(f, i + 1, j) - AT(f, i - 1, j)) / (2.0 * s->dx);
}
static double gcy(const orc_solver *s, const fld *f, int i, int j) {
  return (AT(f, i, j + 1) - AT(f, i, j - 1)) / (2.0 * s->dy);
}
static double gfx(const orc_solver *s, const fld *f, int i, int j) { return (AT(f, i, j) - AT(f, i - 1, j)) / s->dx; }
static double gfy(const orc_solver *s, const fld *f, int i, int j) { return (AT(f, i, j) - AT(f, i, j - 1)) / s->dy; }
static double ccu(const fld *u, int i, int j) { return 0.5 * (AT(u, i, j) + AT(u, i + 1, j)); }
static double ccv(const fld *v, int i, int j) { return 0.5 * (AT(v, i, j) + AT(v, i, j + 1)); }

/* rho_u_face / eta_u_face, operators.cpp:330-362 (same formula for any cell field) */
static double xface(const orc_solver *s, const fld *f, int i, int j) {
  const int nx = s->cfg.nx;
  if (i <= 0) return s->cfg.periodic_x ? 0.5 * (AT(f, nx - 1, j) + AT(f, 0, j)) : AT(f, 0, j);
  if (i >= nx) return s->cfg.periodic_x ? 0.5 * (AT(f, nx - 1, j) + AT(f, 0, j)) : AT(f, nx - 1, j);
  return 0.5 * (AT(f, i - 1, j) + AT(f, i, j));
}
/* rho_v_face / eta_v_face, operators.cpp:342-374 */
static double yface(const orc_solver *s, const fld *f, int i, int j) {
  const int ny = s->cfg.ny;
  if (j <= 0) return s->cfg.periodic_y ? 0.5 * (AT(f, i, ny - 1) + AT(f, i, 0)) : AT(f, i, 0);
  if (j >= ny) return s->cfg.periodic_y ? 0.5 * (AT(f, i, ny - 1) + AT(f, i, 0)) : AT(f, i, ny - 1);
  return 0.5 * (AT(f, i, j - 1) + AT(f, i, j));
}
/* rho_corner / eta_corner, operators.cpp:378-386 */
static double corner(const fld *f, int i, int j) {
  return 0.25 * (AT(f, i, j) + AT(f, i - 1, j) + AT(f, i, j - 1) + AT(f, i - 1, j - 1));
}
static double div_cell(const orc_solver *s, const fld *u, const fld *v, int i, int j) {
  return (AT(u, i + 1, j) - AT(u, i, j)) / s->dx + (AT(v, i, j + 1) - AT(v, i, j)) / s->dy;
}

/* subtract_mean, operators.cpp:447-460 */
static void subtract_mean(const orc_solver *s, fld *f) {
  double mean = 0.0;
  for (int i = 0; i < s->cfg.nx; ++i)
    for (int j = 0; j < s->cfg.ny; ++j) mean += AT(f, i, j);
  mean /= (double)(s->cfg.nx * s->cfg.ny);
  for (int i = 0; i < s->cfg.nx; ++i)
    for (int j = 0; j < s->cfg.ny; ++j) AT(f, i, j) -= mean;
}

static double field_diff_l2(const fld *a, const fld *b, int i0, int i1, int j0, int j1) {
  double diff_sq = 0.0, norm_sq = 0.0;
  for (int i = i0; i < i1; ++i)
    for (int j = j0; j < j1; ++j) {
      diff_sq += sq(AT(a, i, j) - AT(b, i, j));
      norm_sq += sq(AT(a, i, j));
    }
  return sqrt(diff_sq / dmax(norm_sq, 1.0e-30));
}

/* periodic_boundary_speed_stat, operators.cpp:463-478 */
static double boundary_speed(const orc_solver *s, const fld *u, const fld *v) {
  double m = 0.0;
  if (s->cfg.periodic_x)
    for (int j = 0; j < u->ny; ++j) {
      m = dmax(m, fabs(AT(u, 0, j)));
      m = dmax(m, fabs(AT(u, s->cfg.nx, j)));
    }
  if (s->cfg.periodic_y)
    for (int i = 0; i < v->nx; ++i) {
      m = dmax(m, fabs(AT(v, i, 0)));
      m = dmax(m, fabs(AT(v, i, s->cfg.ny)));
    }
  return m;
}

/* ------------------------------------------------------------------------------------------ */
/* Krylov kernels (ch_sparse_krylov.hpp)                                                       */
/* ------------------------------------------------------------------------------------------ */
static double dot(const double *a, const double *b, int n) {
  double v = 0.0;
  for (int k = 0; k < n; ++k) v += a[k] * b[k];
  return v;
}

/* apply_matrix, ch_sparse_krylov.hpp:235-250 */
static void spmv(const csr *m, const double *x, double *y) {
  for (int r = 0; r < m->n; ++r) {
    double sum = 0.0;
    for (int p = m->row_ptr[r]; p < m->row_ptr[r + 1]; ++p) sum += m->val[p] * x[m->col[p]];
    y[r] = sum;
  }
}

static void pc_alloc(precond *pc, int n, int nnz) {
  if (pc->cap < nnz || pc->n != n) {
    free(pc->lower);
    free(pc->lt_row);
    free(pc->lt_val);
    free(pc->diag);
    free(pc->diagonal_inverse);
    free(pc->lt_ptr);
    pc->lower = (double *)calloc((size_t)nnz, sizeof(double));
    pc->lt_row = (int *)calloc((size_t)nnz, sizeof(int));
    pc->lt_val = (double *)calloc((size_t)nnz, sizeof(double));
    pc->diag = (double *)calloc((size_t)n, sizeof(double));
    pc->diagonal_inverse = (double *)calloc((size_t)n, sizeof(double));
    pc->lt_ptr = (int *)calloc((size_t)n + 1, sizeof(int));
    pc->cap = nnz;
    pc->n = n;
  }
}
static void pc_free(precond *pc) {
  free(pc->lower);
  free(pc->lt_row);
  free(pc->lt_val);
  free(pc->diag);
  free(pc->diagonal_inverse);
  free(pc->lt_ptr);
  memset(pc, 0, sizeof(*pc));
}

/* build_diagonal_preconditioner, ch_sparse_krylov.hpp:421-432 */
static void build_diag_pc(const csr *m, precond *pc) {
  pc_alloc(pc, m->n, m->nnz);
  pc->type = 0;
  for (int r = 0; r < m->n; ++r) pc->diagonal_inverse[r] = 1.0 / dmax(fabs(m->val[m->diag_pos[r]]), 1.0e-30);
}

static double find_lower(const csr *m, const precond *pc, int row, int target) {
  for (int p = m->row_ptr[row]; p < m->row_ptr[row + 1]; ++p) {
    const int c = m->col[p];
    if (c >= row || c > target) break;
    if (c == target) return pc->lower[p];
  }
  return 0.0;
}

static void build_transpose(const csr *m, precond *pc) {
  for (int r = 0; r <= m->n; ++r) pc->lt_ptr[r] = 0;
  for (int r = 0; r < m->n; ++r)
    for (int p = m->row_ptr[r]; p < m->row_ptr[r + 1]; ++p) {
      const int c = m->col[p];
      if (c >= r) break;
      pc->lt_ptr[c + 1]++;
    }
  for (int r = 0; r < m->n; ++r) pc->lt_ptr[r + 1] += pc->lt_ptr[r];
  int *fillp = (int *)malloc((size_t)m->n * sizeof(int));
  for (int r = 0; r < m->n; ++r) fillp[r] = pc->lt_ptr[r];
  for (int r = 0; r < m->n; ++r)
    for (int p = m->row_ptr[r]; p < m->row_ptr[r + 1]; ++p) {
      const int c = m->col[p];
      if (c >= r) break;
      pc->lt_row[fillp[c]] = r;
      pc->lt_val[fillp[c]] = pc->lower[p];
      fillp[c]++;
    }
  free(fillp);
}

/* try_build_incomplete_ldlt, ch_sparse_krylov.hpp:252-335 */
static int try_ildlt(const csr *m, precond *pc) {
  pc_alloc(pc, m->n, m->nnz);
  pc->type = 1;
  for (int k = 0; k < m->nnz; ++k) pc->lower[k] = 0.0;
  for (int r = 0; r < m->n; ++r) pc->diag[r] = 0.0;
  double max_diag = 0.0;
  for (int r = 0; r < m->n; ++r) max_diag = dmax(max_diag, fabs(m->val[m->diag_pos[r]]));
  pc->diagonal_floor = dmax(1.0, max_diag) * 1.0e-12;
  for (int r = 0; r < m->n; ++r) {
    for (int p = m->row_ptr[r]; p < m->row_ptr[r + 1]; ++p) {
      const int c = m->col[p];
      if (c >= r) break;
      double sum = m->val[p];
      for (int q = m->row_ptr[r]; q < p; ++q) {
        const int k = m->col[q];
        if (k >= c) break;
        const double l_ck = find_lower(m, pc, c, k);
        if (l_ck != 0.0) sum -= pc->lower[q] * pc->diag[k] * l_ck;
      }
      const double denom = dmax(pc->diag[c], pc->diagonal_floor);
      pc->lower[p] = sum / denom;
    }
    double d = m->val[m->diag_pos[r]];
    for (int p = m->row_ptr[r]; p < m->row_ptr[r + 1]; ++p) {
      const int c = m->col[p];
      if (c >= r) break;
      d -= sq(pc->lower[p]) * pc->diag[c];
    }
    if (!isfinite(d) || d <= pc->diagonal_floor) return 0;
    pc->diag[r] = d;
  }
  build_transpose(m, pc);
  return 1;
}

/* try_build_incomplete_cholesky, ch_sparse_krylov.hpp:337-419 */
static int try_icc(const csr *m, precond *pc) {
  pc_alloc(pc, m->n, m->nnz);
  pc->type = 2;
  for (int k = 0; k < m->nnz; ++k) pc->lower[k] = 0.0;
  for (int r = 0; r < m->n; ++r) pc->diag[r] = 0.0;
  double max_diag = 0.0;
  for (int r = 0; r < m->n; ++r) max_diag = dmax(max_diag, fabs(m->val[m->diag_pos[r]]));
  pc->diagonal_floor = sqrt(dmax(1.0, max_diag) * 1.0e-12);
  const double floor_sq = sq(pc->diagonal_floor);
  for (int r = 0; r < m->n; ++r) {
    for (int p = m->row_ptr[r]; p < m->row_ptr[r + 1]; ++p) {
      const int c = m->col[p];
      if (c >= r) break;
      double sum = m->val[p];
      for (int q = m->row_ptr[r]; q < p; ++q) {
        const int k = m->col[q];
        if (k >= c) break;
        const double l_ck = find_lower(m, pc, c, k);
        if (l_ck != 0.0) sum -= pc->lower[q] * l_ck;
      }
      const double denom = dmax(pc->diag[c], pc->diagonal_floor);
      pc->lower[p] = sum / denom;
    }
    double d = m->val[m->diag_pos[r]];
    for (int p = m->row_ptr[r]; p < m->row_ptr[r + 1]; ++p) {
      const int c = m->col[p];
      if (c >= r) break;
      d -= sq(pc->lower[p]);
    }
    if (!isfinite(d) || d <= floor_sq) return 0;
    pc->diag[r] = sqrt(d);
  }
  build_transpose(m, pc);
  return 1;
}

/* apply_preconditioner, ch_sparse_krylov.hpp:444-513 */
static void apply_pc(const csr *m, const precond *pc, const double *r, double *z, double *y) {
  const int n = m->n;
  if (pc->type == 0) {
    for (int k = 0; k < n; ++k) z[k] = pc->diagonal_inverse[k] * r[k];
    return;
  }
  if (pc->type == 2) {
    for (int row = 0; row < n; ++row) {
      double sum = r[row];
      for (int p = m->row_ptr[row]; p < m->row_ptr[row + 1]; ++p) {
        const int c = m->col[p];
        if (c >= row) break;
        sum -= pc->lower[p] * y[c];
      }
      y[row] = sum / dmax(pc->diag[row], pc->diagonal_floor);
    }
    memcpy(z, y, (size_t)n * sizeof(double));
    for (int row = n - 1; row >= 0; --row) {
      double sum = z[row];
      for (int e = pc->lt_ptr[row]; e < pc->lt_ptr[row + 1]; ++e) sum -= pc->lt_val[e] * z[pc->lt_row[e]];
      z[row] = sum / dmax(pc->diag[row], pc->diagonal_floor);
    }
    return;
  }
  for (int row = 0; row < n; ++row) {
    double sum = r[row];
    for (int p = m->row_ptr[row]; p < m->row_ptr[row + 1]; ++p) {
      const int c = m->col[p];
      if (c >= row) break;
      sum -= pc->lower[p] * y[c];
    }
    y[row] = sum;
  }
  for (int row = 0; row < n; ++row) y[row] /= dmax(pc->diag[row], pc->diagonal_floor);
  memcpy(z, y, (size_t)n * sizeof(double));
  for (int row = n - 1; row >= 0; --row) {
    double sum = z[row];
    for (int e = pc->lt_ptr[row]; e < pc->lt_ptr[row + 1]; ++e) sum -= pc->lt_val[e] * z[pc->lt_row[e]];
    z[row] = sum;
  }
}

typedef struct {
  int iterations;
  double absolute_residual, relative_residual, iterate_residual;
} solve_rep;

/* CGMonitor data of one iteration (ch_sparse_krylov.hpp:515-660), kept while a pressure solve runs */
static void monitor_record(orc_solver *s, int it, const solve_rep *rep, double alpha) {
  if (!s->mon_active || it >= s->mon_cap) return;
  s->mon[4 * it + 0] = rep->absolute_residual;
  s->mon[4 * it + 1] = rep->relative_residual;
  s->mon[4 * it + 2] = rep->iterate_residual;
  s->mon[4 * it + 3] = alpha;
  s->mon_count = it + 1;
}

/* mean projection, pressure.cpp:225-239 (std::accumulate order) */
static void project_mean(double *v, int n) {
  if (n <= 0) return;
  double acc = 0.0;
  for (int k = 0; k < n; ++k) acc += v[k];
  const double mean = acc / dmax((double)n, 1.0);
  for (int k = 0; k < n; ++k) v[k] -= mean;
}

/* solve_preconditioned_cg, ch_sparse_krylov.hpp:515-660 */
static solve_rep pcg(orc_solver *s, const csr *m, const precond *pc, const double *rhs, int max_it, double tol,
                     double *x, int project) {
  const int n = m->n;
  double *ax = s->w[0], *r = s->w[1], *z = s->w[2], *p = s->w[3], *ap = s->w[4], *y = s->w[5];
  solve_rep rep = {0, 0.0, 0.0, 0.0};
  if (n <= 0) fail(s, "cannot solve an empty linear system");
  spmv(m, x, ax);
  for (int k = 0; k < n; ++k) r[k] = rhs[k] - ax[k];
  if (project) project_mean(r, n);
  const double rhs_norm = sqrt(dmax(dot(rhs, rhs, n), 0.0));
  rep.absolute_residual = sqrt(dmax(dot(r, r, n), 0.0));
  rep.relative_residual = rep.absolute_residual / dmax(rhs_norm, 1.0e-30);
  if (rep.relative_residual < tol || rep.absolute_residual < tol) return rep;
  apply_pc(m, pc, r, z, y);
  if (project) project_mean(z, n);
  double rz_old = dot(r, z, n);
  if (!isfinite(rz_old) || rz_old <= 0.0) fail(s, "pcg preconditioner breakdown: non-positive r^T M^{-1} r");
  memcpy(p, z, (size_t)n * sizeof(double));
  const int limit = max_it > 1 ? max_it : 1;
  for (int it = 0; it < limit; ++it) {
    spmv(m, p, ap);
    const double pap = dot(p, ap, n);
    if (!isfinite(pap) || fabs(pap) < 1.0e-30) fail(s, "pcg breakdown: p^T A p is invalid");
    const double alpha = rz_old / pap;
    double update_sq = 0.0, x_norm_sq = 0.0;
    for (int k = 0; k < n; ++k) {
      const double delta = alpha * p[k];
      x[k] += delta;
      r[k] -= alpha * ap[k];
      update_sq += delta * delta;
      x_norm_sq += x[k] * x[k];
    }
    if (project) {
      project_mean(x, n);
      project_mean(r, n);
    }
    rep.iterations = it + 1;
    rep.iterate_residual = sqrt(update_sq / dmax(x_norm_sq, 1.0e-30));
    rep.absolute_residual = sqrt(dmax(dot(r, r, n), 0.0));
    rep.relative_residual = rep.absolute_residual / dmax(rhs_norm, 1.0e-30);
    monitor_record(s, it, &rep, alpha);
    if (rep.relative_residual < tol || rep.absolute_residual < tol) break;
    apply_pc(m, pc, r, z, y);
    if (project) project_mean(z, n);
    const double rz_new = dot(r, z, n);
    if (!isfinite(rz_new) || rz_new <= 0.0) fail(s, "pcg preconditioner breakdown: non-positive new r^T M^{-1} r");
    const double beta = rz_new / rz_old;
    for (int k = 0; k < n; ++k) p[k] = z[k] + beta * p[k];
    if (project) project_mean(p, n);
    rz_old = rz_new;
  }
  return rep;
}

/* solve_preconditioned_bicgstab, ch_sparse_krylov.hpp:839-963 */
static solve_rep bicgstab(orc_solver *s, const csr *m, const precond *pc, const double *rhs, int max_it, double tol,
                          double *x, int use_rel) {
  const int n = m->n;
  double *ax = s->w[0], *r = s->w[1], *rhat = s->w[2], *p = s->w[3], *v = s->w[4], *phat = s->w[5];
  double *sv = s->w[6], *shat = s->w[7], *t = s->w[8], *upd = s->w[9], *y = s->w[10];
  solve_rep rep = {0, 0.0, 0.0, 0.0};
  if (n <= 0) fail(s, "cannot solve an empty linear system");
  spmv(m, x, ax);
  for (int k = 0; k < n; ++k) r[k] = rhs[k] - ax[k];
  const double rhs_norm = sqrt(dmax(dot(rhs, rhs, n), 0.0));
  rep.absolute_residual = sqrt(dmax(dot(r, r, n), 0.0));
  rep.relative_residual = rep.absolute_residual / dmax(rhs_norm, 1.0e-30);
  if ((use_rel && rep.relative_residual < tol) || rep.absolute_residual < tol) return rep;
  memcpy(rhat, r, (size_t)n * sizeof(double));
  for (int k = 0; k < n; ++k) {
    p[k] = 0.0;
    v[k] = 0.0;
    sv[k] = 0.0;
    t[k] = 0.0;
    upd[k] = 0.0;
  }
  double rho_old = 1.0, alpha = 1.0, omega = 1.0;
  const int limit = max_it > 1 ? max_it : 1;
  for (int it = 0; it < limit; ++it) {
    const double rho_new = dot(rhat, r, n);
    if (!isfinite(rho_new) || fabs(rho_new) < 1.0e-30) fail(s, "bicgstab breakdown: invalid rho");
    const double beta = (it == 0) ? 0.0 : (rho_new / rho_old) * (alpha / omega);
    for (int k = 0; k < n; ++k) p[k] = r[k] + beta * (p[k] - omega * v[k]);
    apply_pc(m, pc, p, phat, y);
    spmv(m, phat, v);
    const double rhat_v = dot(rhat, v, n);
    if (!isfinite(rhat_v) || fabs(rhat_v) < 1.0e-30) fail(s, "bicgstab breakdown: invalid r_hat^T A M^{-1} p");
    alpha = rho_new / rhat_v;
    for (int k = 0; k < n; ++k) {
      sv[k] = r[k] - alpha * v[k];
      upd[k] = alpha * phat[k];
    }
    const double s_norm = sqrt(dmax(dot(sv, sv, n), 0.0));
    if ((use_rel && s_norm / dmax(rhs_norm, 1.0e-30) < tol) || s_norm < tol) {
      double update_sq = 0.0, x_norm_sq = 0.0;
      for (int k = 0; k < n; ++k) {
        x[k] += upd[k];
        update_sq += upd[k] * upd[k];
        x_norm_sq += x[k] * x[k];
      }
      rep.iterations = it + 1;
      rep.iterate_residual = sqrt(update_sq / dmax(x_norm_sq, 1.0e-30));
      rep.absolute_residual = s_norm;
      rep.relative_residual = s_norm / dmax(rhs_norm, 1.0e-30);
      return rep;
    }
    apply_pc(m, pc, sv, shat, y);
    spmv(m, shat, t);
    const double tt = dot(t, t, n);
    if (!isfinite(tt) || fabs(tt) < 1.0e-30) fail(s, "bicgstab breakdown: invalid t^T t");
    omega = dot(t, sv, n) / tt;
    if (!isfinite(omega) || fabs(omega) < 1.0e-30) fail(s, "bicgstab breakdown: invalid omega");
    double update_sq = 0.0, x_norm_sq = 0.0;
    for (int k = 0; k < n; ++k) {
      upd[k] += omega * shat[k];
      x[k] += upd[k];
      r[k] = sv[k] - omega * t[k];
      update_sq += upd[k] * upd[k];
      x_norm_sq += x[k] * x[k];
    }
    rep.iterations = it + 1;
    rep.iterate_residual = sqrt(update_sq / dmax(x_norm_sq, 1.0e-30));
    rep.absolute_residual = sqrt(dmax(dot(r, r, n), 0.0));
    rep.relative_residual = rep.absolute_residual / dmax(rhs_norm, 1.0e-30);
    if ((use_rel && rep.relative_residual < tol) || rep.absolute_residual < tol) return rep;
    rho_old = rho_new;
  }
  return rep;
}

/* build_laplacian_matrix, ch_sparse_krylov.hpp:135-177 */
static void build_laplacian(orc_solver *s, csr *out) {
  const int nx = s->cfg.nx, ny = s->cfg.ny, n = nx * ny;
  const int px = s->cfg.periodic_x, py = s->cfg.periodic_y;
  const double inv_dx2 = 1.0 / (s->dx * s->dx), inv_dy2 = 1.0 / (s->dy * s->dy);
  rowacc *rows = rows_get(s, n);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      const int row = i * ny + j;
      double diag = 0.0;
      if (px || i > 0) {
        const int iw = px && i == 0 ? nx - 1 : i - 1;
        ra_add(&rows[row], iw * ny + j, inv_dx2);
        diag -= inv_dx2;
      }
      if (px || i < nx - 1) {
        const int ie = px && i == nx - 1 ? 0 : i + 1;
        ra_add(&rows[row], ie * ny + j, inv_dx2);
        diag -= inv_dx2;
      }
      if (py || j > 0) {
        const int js = py && j == 0 ? ny - 1 : j - 1;
        ra_add(&rows[row], i * ny + js, inv_dy2);
        diag -= inv_dy2;
      }
      if (py || j < ny - 1) {
        const int jn = py && j == ny - 1 ? 0 : j + 1;
        ra_add(&rows[row], i * ny + jn, inv_dy2);
        diag -= inv_dy2;
      }
      ra_add(&rows[row], row, diag);
    }
  finalize_rows(s, rows, n, out);
}

/* multiply, ch_sparse_krylov.hpp:179-203 */
static void csr_multiply(orc_solver *s, const csr *a, const csr *b, csr *out) {
  rowacc *rows = rows_get(s, a->n);
  for (int r = 0; r < a->n; ++r)
    for (int pa = a->row_ptr[r]; pa < a->row_ptr[r + 1]; ++pa) {
      const int mid = a->col[pa];
      const double va = a->val[pa];
      for (int pb = b->row_ptr[mid]; pb < b->row_ptr[mid + 1]; ++pb) ra_add(&rows[r], b->col[pb], va * b->val[pb]);
    }
  finalize_rows(s, rows, a->n, out);
}

/* build_cahn_hilliard_operator, ch_sparse_krylov.hpp:205-233 */
static void build_ch_operator(orc_solver *s, const csr *lap, const csr *bih, double alpha0, double beta1,
                              double beta2, csr *out) {
  rowacc *rows = rows_get(s, lap->n);
  for (int r = 0; r < lap->n; ++r) {
    ra_add(&rows[r], r, alpha0);
    for (int p = lap->row_ptr[r]; p < lap->row_ptr[r + 1]; ++p) ra_add(&rows[r], lap->col[p], -beta1 * lap->val[p]);
    for (int p = bih->row_ptr[r]; p < bih->row_ptr[r + 1]; ++p) ra_add(&rows[r], bih->col[p], beta2 * bih->val[p]);
  }
  finalize_rows(s, rows, lap->n, out);
}

/* ------------------------------------------------------------------------------------------ */
/* Materials, chemical potential, CH explicit operator (phase_field.cpp)                       */
/* ------------------------------------------------------------------------------------------ */
static int is_adv_only(const orc_solver *s) { return s->cfg.mode == ORC_MODE_ADVECTION_ONLY; }
static int is_single(const orc_solver *s) { return s->cfg.mode == ORC_MODE_SINGLE_PHASE; }
static int solve_ch(const orc_solver *s) { return !is_adv_only(s) && !(is_single(s) || s->cfg.freeze_ch); }
static int compute_mu_on(const orc_solver *s) { return !is_adv_only(s) && !is_single(s); }

/* update_materials_from_phase, phase_field.cpp:57-66 */
static void materials_from(orc_solver *s, const fld *c, fld *rho, fld *eta) {
  for (int i = 0; i < s->cfg.nx; ++i)
    for (int j = 0; j < s->cfg.ny; ++j) {
      AT(rho, i, j) = AT(c, i, j) + (1.0 - AT(c, i, j)) * s->cfg.density_ratio;
      AT(eta, i, j) = AT(c, i, j) + (1.0 - AT(c, i, j)) * s->cfg.viscosity_ratio;
    }
  bc_scalar(s, rho);
  bc_scalar(s, eta);
}
static void update_materials(orc_solver *s) { materials_from(s, &s->f[ORC_F_C], &s->f[ORC_F_RHO], &s->f[ORC_F_ETA]); }

/* update_midpoint_materials, phase_field.cpp:70-79 */
static void update_midpoint(orc_solver *s) {
  fld *rm = &s->f[ORC_F_RHO_MID], *em = &s->f[ORC_F_ETA_MID];
  for (int i = 0; i < s->cfg.nx; ++i)
    for (int j = 0; j < s->cfg.ny; ++j) {
      AT(rm, i, j) = 0.5 * (AT(&s->f[ORC_F_RHO_PREV], i, j) + AT(&s->f[ORC_F_RHO], i, j));
      AT(em, i, j) = 0.5 * (AT(&s->f[ORC_F_ETA_PREV], i, j) + AT(&s->f[ORC_F_ETA], i, j));
    }
  bc_scalar(s, rm);
  bc_scalar(s, em);
}

/* update_chemical_potential, phase_field.cpp:97-109 */
static void chem_potential(orc_solver *s, const fld *c_state, fld *mu) {
  fld work;
  fld_init(&work, c_state->nx, c_state->ny, c_state->g, 0.0);
  fld_copy(&work, c_state);
  bc_scalar(s, &work);
  const double alpha = 6.0 * sqrt(2.0);
  for (int i = 0; i < s->cfg.nx; ++i)
    for (int j = 0; j < s->cfg.ny; ++j) {
      const double c = AT(&work, i, j);
      const double dw = 0.5 * c * (1.0 - c) * (1.0 - 2.0 * c);
      AT(mu, i, j) = alpha * (dw / s->cfg.cn - s->cfg.cn * lap_c(s, &work, i, j));
    }
  bc_scalar(s, mu);
  fld_free(&work);
}

static void refresh_mu(orc_solver *s) {
  if (compute_mu_on(s)) {
    chem_potential(s, &s->f[ORC_F_C], &s->f[ORC_F_MU]);
    return;
  }
  fld_fill(&s->f[ORC_F_MU], 0.0);
  bc_scalar(s, &s->f[ORC_F_MU]);
}

static void clear_surface_force(orc_solver *s) {
  fld_fill(&s->f[ORC_F_SFX_CELL], 0.0);
  fld_fill(&s->f[ORC_F_SFY_CELL], 0.0);
  fld_fill(&s->f[ORC_F_SFX_U], 0.0);
  fld_fill(&s->f[ORC_F_SFY_V], 0.0);
  bc_scalar(s, &s->f[ORC_F_SFX_CELL]);
  bc_scalar(s, &s->f[ORC_F_SFY_CELL]);
  bc_u(s, &s->f[ORC_F_SFX_U]);
  bc_v(s, &s->f[ORC_F_SFY_V]);
}

/* weno5_left, phase_field.cpp:144-157 */
static double weno5_left(double v1, double v2, double v3, double v4, double v5) {
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
static double weno5_right(double v1, double v2, double v3, double v4, double v5) {
  return weno5_left(v5, v4, v3, v2, v1);
}

/* build_phase_advection_fluxes, phase_field.cpp:283-311 (WENO5 faces, :163-177) */
static void adv_fluxes(orc_solver *s, const fld *c_state, const fld *ua, const fld *va, fld *fx, fld *fy,
                       fld *rhs) {
  fld ce;
  fld_init(&ce, c_state->nx, c_state->ny, c_state->g, 0.0);
  fld_copy(&ce, c_state);
  bc_scalar(s, &ce);
  const int nx = s->cfg.nx, ny = s->cfg.ny;
  for (int i = 0; i < nx + 1; ++i)
    for (int j = 0; j < ny; ++j) {
      const double face = (AT(ua, i, j) >= 0.0) ? weno5_left(AT(&ce, i - 3, j), AT(&ce, i - 2, j), AT(&ce, i - 1, j),
                                                             AT(&ce, i, j), AT(&ce, i + 1, j))
                                                  : weno5_right(AT(&ce, i - 2, j), AT(&ce, i - 1, j), AT(&ce, i, j),
                                                                AT(&ce, i + 1, j), AT(&ce, i + 2, j));
      AT(fx, i, j) = AT(ua, i, j) * face;
    }
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny + 1; ++j) {
      const double face = (AT(va, i, j) >= 0.0) ? weno5_left(AT(&ce, i, j - 3), AT(&ce, i, j - 2), AT(&ce, i, j - 1),
                                                             AT(&ce, i, j), AT(&ce, i, j + 1))
                                                  : weno5_right(AT(&ce, i, j - 2), AT(&ce, i, j - 1), AT(&ce, i, j),
                                                                AT(&ce, i, j + 1), AT(&ce, i, j + 2));
      AT(fy, i, j) = AT(va, i, j) * face;
    }
  bc_u(s, fx);
  bc_v(s, fy);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      AT(rhs, i, j) = -(AT(fx, i + 1, j) - AT(fx, i, j)) / s->dx - (AT(fy, i, j + 1) - AT(fy, i, j)) / s->dy;
  bc_scalar(s, rhs);
  fld_free(&ce);
}

/* build_phase_diffusion_fluxes, phase_field.cpp:313-352 */
static void diff_fluxes(orc_solver *s, const fld *sc, const fld *mob, fld *fx, fld *fy, fld *div) {
  const int nx = s->cfg.nx, ny = s->cfg.ny;
  for (int i = 0; i < nx + 1; ++i)
    for (int j = 0; j < ny; ++j) {
      const double m = xface(s, mob, i, j);
      AT(fx, i, j) = m * gfx(s, sc, i, j);
    }
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny + 1; ++j) {
      const double m = yface(s, mob, i, j);
      AT(fy, i, j) = m * gfy(s, sc, i, j);
    }
  bc_u(s, fx);
  bc_v(s, fy);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      AT(div, i, j) = (AT(fx, i + 1, j) - AT(fx, i, j)) / s->dx + (AT(fy, i, j + 1) - AT(fy, i, j)) / s->dy;
  bc_scalar(s, div);
}

/* build_phase_explicit_operator, phase_field.cpp:354-396 */
static void phase_explicit(orc_solver *s, const fld *c, const fld *ua, const fld *va, fld *E) {
  const int nx = s->cfg.nx, ny = s->cfg.ny, g = s->cfg.ghost;
  fld mob, mu, afx, afy, arhs, dfx, dfy, ddiv, lap, bih;
  fld_init(&mob, nx, ny, g, 0.0);
  fld_init(&mu, nx, ny, g, 0.0);
  fld_init(&afx, nx + 1, ny, g, 0.0);
  fld_init(&afy, nx, ny + 1, g, 0.0);
  fld_init(&arhs, nx, ny, g, 0.0);
  fld_init(&dfx, nx + 1, ny, g, 0.0);
  fld_init(&dfy, nx, ny + 1, g, 0.0);
  fld_init(&ddiv, nx, ny, g, 0.0);
  fld_init(&lap, nx, ny, g, 0.0);
  fld_init(&bih, nx, ny, g, 0.0);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      AT(&mob, i, j) = dmax(0.0, AT(c, i, j) * (1.0 - AT(c, i, j)));
      AT(&lap, i, j) = lap_c(s, c, i, j);
    }
  bc_scalar(s, &mob);
  bc_scalar(s, &lap);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) AT(&bih, i, j) = lap_c(s, &lap, i, j);
  bc_scalar(s, &bih);
  chem_potential(s, c, &mu);
  adv_fluxes(s, c, ua, va, &afx, &afy, &arhs);
  diff_fluxes(s, &mu, &mob, &dfx, &dfy, &ddiv);
  const double a1 = (s->cfg.cn > 0.0) ? (3.0 * KSQRT2 / (16.0 * s->cfg.cn)) : 0.0;
  const double a2 = (s->cfg.cn > 0.0) ? (3.0 * KSQRT2 * s->cfg.cn / 4.0) : 0.0;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      AT(E, i, j) = AT(&ddiv, i, j) / s->cfg.pe - (a1 * AT(&lap, i, j) - a2 * AT(&bih, i, j)) / s->cfg.pe +
                    AT(&arhs, i, j);
  bc_scalar(s, E);
  fld_free(&mob);
  fld_free(&mu);
  fld_free(&afx);
  fld_free(&afy);
  fld_free(&arhs);
  fld_free(&dfx);
  fld_free(&dfy);
  fld_free(&ddiv);
  fld_free(&lap);
  fld_free(&bih);
}

/* ensure_ch_operator_matrices / ensure_ch_linear_system, phase_field.cpp:119-142 */
static void ensure_ch_system(orc_solver *s, double alpha0) {
  if (!s->ch_ops_ready) {
    build_laplacian(s, &s->ch_lap);
    csr_multiply(s, &s->ch_lap, &s->ch_lap, &s->ch_biharm);
    s->ch_ops_ready = 1;
  }
  if (fabs(alpha0 - s->ch_cached_alpha0) <= 1.0e-14 * dmax(1.0, fabs(alpha0))) return;
  const double a1 = (s->cfg.cn > 0.0) ? (3.0 * KSQRT2 / (16.0 * s->cfg.cn)) : 0.0;
  const double a2 = (s->cfg.cn > 0.0) ? (3.0 * KSQRT2 * s->cfg.cn / 4.0) : 0.0;
  const double beta1 = a1 / s->cfg.pe, beta2 = a2 / s->cfg.pe;
  build_ch_operator(s, &s->ch_lap, &s->ch_biharm, alpha0, beta1, beta2, &s->ch_sys);
  /* build_preconditioner, ch_sparse_krylov.hpp:434-442: ILDLT, else diagonal */
  if (!try_ildlt(&s->ch_sys, &s->ch_pc)) build_diag_pc(&s->ch_sys, &s->ch_pc);
  s->ch_cached_alpha0 = alpha0;
}

/* solve_phase_linear_system_eq25, phase_field.cpp:437-503 (sparse_pcg path) */
static void ch_linear_solve(orc_solver *s, const fld *rhs_field, double alpha0, fld *c_state, double *iter_res,
                            double *eq_res) {
  const int nx = s->cfg.nx, ny = s->cfg.ny, n = nx * ny;
  ensure_ch_system(s, alpha0);
  double *rhs = s->w[11], *x = s->w[12], *ax = s->w[13];
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      rhs[i * ny + j] = AT(rhs_field, i, j);
      x[i * ny + j] = AT(c_state, i, j);
    }
  *iter_res = 0.0;
  *eq_res = 0.0;
  s->rep.ch_preconditioner = s->ch_pc.type == 1 ? 1 : 0;
  solve_rep rep;
  jmp_buf local, *saved = s->jb;
  s->jb = &local;
  if (setjmp(local) == 0) {
    rep = pcg(s, &s->ch_sys, &s->ch_pc, rhs, s->cfg.ch_inner_iterations, s->cfg.ch_tolerance, x, 0);
    s->jb = saved;
  } else {
    s->jb = saved;
    build_diag_pc(&s->ch_sys, &s->ch_pc);
    s->rep.ch_preconditioner = 2;
    rep = pcg(s, &s->ch_sys, &s->ch_pc, rhs, s->cfg.ch_inner_iterations, s->cfg.ch_tolerance, x, 0);
  }
  s->rep.ch_iterations = rep.iterations;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) AT(c_state, i, j) = x[i * ny + j];
  bc_scalar(s, c_state);
  double rhs_norm_sq = 0.0;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      x[i * ny + j] = AT(c_state, i, j);
      rhs_norm_sq += sq(rhs[i * ny + j]);
    }
  spmv(&s->ch_sys, x, ax);
  double residual_sq = 0.0;
  for (int k = 0; k < n; ++k) residual_sq += sq(rhs[k] - ax[k]);
  *iter_res = rep.iterate_residual;
  *eq_res = sqrt(residual_sq / dmax(rhs_norm_sq, 1.0e-30));
}

/* compute_mass, diagnostics.cpp:24-32 */
static double mass_of(const orc_solver *s, const fld *f) {
  double sum = 0.0;
  for (int i = 0; i < s->cfg.nx; ++i)
    for (int j = 0; j < s->cfg.ny; ++j) sum += AT(f, i, j) * s->dx * s->dy;
  return sum;
}

/* update_surface_tension_force, phase_field.cpp:179-256 */
static void smooth(orc_solver *s, fld *f, void (*bc)(const orc_solver *, fld *)) {
  fld scratch;
  fld_init(&scratch, f->nx, f->ny, f->g, 0.0);
  const double nw = s->cfg.surface_tension_smoothing_weight;
  const double cw = 1.0 - 4.0 * nw;
  for (int pass = 0; pass < s->cfg.surface_tension_smoothing_passes; ++pass) {
    bc(s, f);
    for (int i = 0; i < f->nx; ++i)
      for (int j = 0; j < f->ny; ++j)
        AT(&scratch, i, j) =
            cw * AT(f, i, j) + nw * (AT(f, i - 1, j) + AT(f, i + 1, j) + AT(f, i, j - 1) + AT(f, i, j + 1));
    bc(s, &scratch);
    fld_copy(f, &scratch);
  }
  fld_free(&scratch);
}

static void surface_force(orc_solver *s, const fld *c_old, const fld *c_new) {
  if (s->cfg.surface_tension_multiplier == 0.0 || !compute_mu_on(s)) {
    clear_surface_force(s);
    return;
  }
  const int nx = s->cfg.nx, ny = s->cfg.ny;
  fld cm, mm;
  fld_init(&cm, c_new->nx, c_new->ny, c_new->g, 0.0);
  fld_copy(&cm, c_new);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) AT(&cm, i, j) = 0.5 * (AT(c_old, i, j) + AT(c_new, i, j));
  bc_scalar(s, &cm);
  fld_init(&mm, nx, ny, s->cfg.ghost, 0.0);
  chem_potential(s, &cm, &mm);
  const double scale = s->cfg.surface_tension_multiplier / (s->cfg.re * s->cfg.ca);
  fld *fxc = &s->f[ORC_F_SFX_CELL], *fyc = &s->f[ORC_F_SFY_CELL], *fxu = &s->f[ORC_F_SFX_U],
      *fyv = &s->f[ORC_F_SFY_V];
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      AT(fxc, i, j) = scale * AT(&mm, i, j) * gcx(s, &cm, i, j);
      AT(fyc, i, j) = scale * AT(&mm, i, j) * gcy(s, &cm, i, j);
    }
  bc_scalar(s, fxc);
  bc_scalar(s, fyc);
  for (int i = 0; i < nx + 1; ++i)
    for (int j = 0; j < ny; ++j) {
      const double mf = (i <= 0) ? 0.5 * (AT(&mm, nx - 1, j) + AT(&mm, 0, j))
                                 : (i >= nx ? 0.5 * (AT(&mm, nx - 1, j) + AT(&mm, 0, j))
                                            : 0.5 * (AT(&mm, i - 1, j) + AT(&mm, i, j)));
      AT(fxu, i, j) = scale * mf * gfx(s, &cm, i, j);
    }
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny + 1; ++j) {
      const double mf = (j <= 0) ? 0.5 * (AT(&mm, i, ny - 1) + AT(&mm, i, 0))
                                 : (j >= ny ? 0.5 * (AT(&mm, i, ny - 1) + AT(&mm, i, 0))
                                            : 0.5 * (AT(&mm, i, j - 1) + AT(&mm, i, j)));
      AT(fyv, i, j) = scale * mf * gfy(s, &cm, i, j);
    }
  bc_u(s, fxu);
  bc_v(s, fyv);
  fld_free(&cm);
  fld_free(&mm);
  if (s->cfg.surface_tension_smoothing_passes <= 0 || s->cfg.surface_tension_smoothing_weight <= 0.0) return;
  smooth(s, fxc, bc_scalar);
  smooth(s, fyc, bc_scalar);
  smooth(s, fxu, bc_u);
  smooth(s, fyv, bc_v);
}

/* solve_cahn_hilliard_semi_implicit, phase_field.cpp:667-708 */
static double ch_semi_implicit(orc_solver *s, const fld *ua, const fld *va, int step) {
  const int nx = s->cfg.nx, ny = s->cfg.ny, g = s->cfg.ghost;
  fld rhsf, En, cs;
  fld_init(&rhsf, nx, ny, g, 0.0);
  fld_init(&En, nx, ny, g, 0.0);
  fld_init(&cs, nx, ny, g, 0.0);
  fld_copy(&cs, &s->f[ORC_F_C]);
  phase_explicit(s, &s->f[ORC_F_C], ua, va, &En);
  const double dt = s->cfg.dt;
  const double alpha0 = (step == 0) ? (1.0 / dt) : (3.0 / (2.0 * dt));
  const fld *cp = &s->f[ORC_F_C_PREV], *cp2 = &s->f[ORC_F_C_PREV2], *Ep = &s->f[ORC_F_E_PREV];
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      if (step == 0)
        AT(&rhsf, i, j) = AT(cp, i, j) / dt + AT(&En, i, j);
      else
        AT(&rhsf, i, j) =
            (4.0 * AT(cp, i, j) - AT(cp2, i, j)) / (2.0 * dt) + 2.0 * AT(&En, i, j) - AT(Ep, i, j);
    }
  bc_scalar(s, &rhsf);
  double iter_res = 0.0, eq_res = 0.0;
  ch_linear_solve(s, &rhsf, alpha0, &cs, &iter_res, &eq_res);
  fld_copy(&s->f[ORC_F_C], &cs);
  bc_scalar(s, &s->f[ORC_F_C]);
  chem_potential(s, &s->f[ORC_F_C], &s->f[ORC_F_MU]);
  s->rep.ch_equation_residual = eq_res;
  fld_copy(&s->f[ORC_F_E_PREV], &En);
  fld_free(&rhsf);
  fld_free(&En);
  fld_free(&cs);
  return iter_res;
}

/* solve_phase_advection_only (SSPRK3 + WENO5), phase_field.cpp:398-435 */
static double advection_only(orc_solver *s) {
  const int nx = s->cfg.nx, ny = s->cfg.ny, g = s->cfg.ghost;
  const double dt = s->cfg.dt;
  fld fx, fy, rs, c0, c1, c2;
  fld_init(&fx, nx + 1, ny, g, 0.0);
  fld_init(&fy, nx, ny + 1, g, 0.0);
  fld_init(&rs, nx, ny, g, 0.0);
  fld_init(&c0, nx, ny, g, 0.0);
  fld_init(&c1, nx, ny, g, 0.0);
  fld_init(&c2, nx, ny, g, 0.0);
  fld *c = &s->f[ORC_F_C], *u = &s->f[ORC_F_U], *v = &s->f[ORC_F_V];
  fld_copy(&c0, c);
  fld_copy(&c1, c);
  fld_copy(&c2, c);
  adv_fluxes(s, &c0, u, v, &fx, &fy, &rs);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) AT(&c1, i, j) = AT(&c0, i, j) + dt * AT(&rs, i, j);
  bc_scalar(s, &c1);
  adv_fluxes(s, &c1, u, v, &fx, &fy, &rs);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      const double pred = AT(&c1, i, j) + dt * AT(&rs, i, j);
      AT(&c2, i, j) = 0.75 * AT(&c0, i, j) + 0.25 * pred;
    }
  bc_scalar(s, &c2);
  adv_fluxes(s, &c2, u, v, &fx, &fy, &rs);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      const double pred = AT(&c2, i, j) + dt * AT(&rs, i, j);
      AT(c, i, j) = (1.0 / 3.0) * AT(&c0, i, j) + (2.0 / 3.0) * pred;
    }
  bc_scalar(s, c);
  const double res = field_diff_l2(c, &c0, 0, nx, 0, ny);
  fld_free(&fx);
  fld_free(&fy);
  fld_free(&rs);
  fld_free(&c0);
  fld_free(&c1);
  fld_free(&c2);
  return res;
}

/* ------------------------------------------------------------------------------------------ */
/* Momentum predictor (momentum.cpp)                                                            */
/* ------------------------------------------------------------------------------------------ */
/* compute_momentum_fluxes, momentum.cpp:55-85 */
static void momentum_fluxes(orc_solver *s, fld *ua, fld *va) {
  const fld *u = &s->f[ORC_F_U], *v = &s->f[ORC_F_V];
  fld_fill(ua, 0.0);
  fld_fill(va, 0.0);
  for (int i = 0; i < u->nx; ++i)
    for (int j = 0; j < u->ny; ++j) {
      const double uf = AT(u, i, j);
      const double dudx = (AT(u, i + 1, j) - AT(u, i - 1, j)) / (2.0 * s->dx);
      const double dudy = (AT(u, i, j + 1) - AT(u, i, j - 1)) / (2.0 * s->dy);
      const double vf = 0.25 * (AT(v, i - 1, j) + AT(v, i, j) + AT(v, i - 1, j + 1) + AT(v, i, j + 1));
      AT(ua, i, j) = uf * dudx + vf * dudy;
    }
  for (int i = 0; i < v->nx; ++i)
    for (int j = 0; j < v->ny; ++j) {
      const double vf = AT(v, i, j);
      const double dvdx = (AT(v, i + 1, j) - AT(v, i - 1, j)) / (2.0 * s->dx);
      const double dvdy = (AT(v, i, j + 1) - AT(v, i, j - 1)) / (2.0 * s->dy);
      const double uf = 0.25 * (AT(u, i, j - 1) + AT(u, i, j) + AT(u, i + 1, j - 1) + AT(u, i + 1, j));
      AT(va, i, j) = uf * dvdx + vf * dvdy;
    }
  bc_u(s, ua);
  bc_v(s, va);
}

/* viscous stress divergence, momentum.cpp:91-155 */
static double visc_u(const orc_solver *s, const fld *u, const fld *v, const fld *eta, int i, int j) {
  const double eta_e = xface(s, eta, i + 1, j), eta_w = xface(s, eta, i, j);
  const double dudx_e = (AT(u, i + 1, j) - AT(u, i, j)) / s->dx;
  const double dudx_w = (AT(u, i, j) - AT(u, i - 1, j)) / s->dx;
  const double normal = (2.0 * eta_e * dudx_e - 2.0 * eta_w * dudx_w) / s->dx;
  const double eta_n = corner(eta, i, j + 1), eta_s = corner(eta, i, j);
  const double dudy_n = (AT(u, i, j + 1) - AT(u, i, j)) / s->dy;
  const double dudy_s = (AT(u, i, j) - AT(u, i, j - 1)) / s->dy;
  const double shear_self = (eta_n * dudy_n - eta_s * dudy_s) / s->dy;
  const double self = normal + shear_self;
  const double dvdx_n = (AT(v, i, j + 1) - AT(v, i - 1, j + 1)) / s->dx;
  const double dvdx_s = (AT(v, i, j) - AT(v, i - 1, j)) / s->dx;
  const double cross = (eta_n * dvdx_n - eta_s * dvdx_s) / s->dy;
  return self + cross;
}
static double visc_v(const orc_solver *s, const fld *u, const fld *v, const fld *eta, int i, int j) {
  const double eta_e = corner(eta, i + 1, j), eta_w = corner(eta, i, j);
  const double dvdx_e = (AT(v, i + 1, j) - AT(v, i, j)) / s->dx;
  const double dvdx_w = (AT(v, i, j) - AT(v, i - 1, j)) / s->dx;
  const double shear_self = (eta_e * dvdx_e - eta_w * dvdx_w) / s->dx;
  const double eta_n = yface(s, eta, i, j + 1), eta_s = yface(s, eta, i, j);
  const double dvdy_n = (AT(v, i, j + 1) - AT(v, i, j)) / s->dy;
  const double dvdy_s = (AT(v, i, j) - AT(v, i, j - 1)) / s->dy;
  const double normal = (2.0 * eta_n * dvdy_n - 2.0 * eta_s * dvdy_s) / s->dy;
  const double self = shear_self + normal;
  const double dudy_e = (AT(u, i + 1, j) - AT(u, i + 1, j - 1)) / s->dy;
  const double dudy_w = (AT(u, i, j) - AT(u, i, j - 1)) / s->dy;
  const double cross = (eta_e * dudy_e - eta_w * dudy_w) / s->dx;
  return self + cross;
}

typedef struct {
  orc_solver *s;
  int *u_row_of, *v_row_of;
  int u_unknowns;
  orc_bc lu, ru, bu, tu, lv, rv, bv, tv;
  rowacc *rows;
  double *rhs;
} mom_ctx;

static int u_active(const orc_solver *s, int i, int j) {
  if (j < 0 || j >= s->cfg.ny) return 0;
  if (s->cfg.periodic_x) {
    if (i < 0 || i >= s->cfg.nx) return 0;
  } else if (i <= 0 || i >= s->cfg.nx) {
    return 0;
  }
  return 1;
}
static int v_active(const orc_solver *s, int i, int j) {
  if (i < 0 || i >= s->cfg.nx) return 0;
  if (s->cfg.periodic_y) {
    if (j < 0 || j >= s->cfg.ny) return 0;
  } else if (j <= 0 || j >= s->cfg.ny) {
    return 0;
  }
  return 1;
}
static int can_ui(const orc_solver *s, int i) {
  if (!s->cfg.periodic_x) return i;
  if (i < 0) return s->cfg.nx - 1;
  if (i >= s->cfg.nx) return 0;
  return i;
}
static int can_uj(const orc_solver *s, int j) {
  if (!s->cfg.periodic_y) return j;
  if (j < 0) return s->cfg.ny - 1;
  if (j >= s->cfg.ny) return 0;
  return j;
}
#define can_vi can_ui
#define can_vj can_uj

static int u_row(mom_ctx *m, int i, int j) { return m->u_row_of[i * m->s->cfg.ny + j]; }
static int v_row(mom_ctx *m, int i, int j) { return m->u_unknowns + m->v_row_of[i * (m->s->cfg.ny + 1) + j]; }

/* add_u_x_entry / add_u_y_entry / add_v_y_entry / add_v_x_entry, momentum.cpp:309-393 */
static void add_u_x(mom_ctx *m, int row, int ui, int uj, double value) {
  orc_solver *s = m->s;
  if (u_active(s, ui, uj)) {
    ra_add(&m->rows[row], u_row(m, ui, uj), value);
    return;
  }
  if (!s->cfg.periodic_x && (ui <= 0 || ui >= s->cfg.nx)) {
    const int is_left = ui <= 0;
    const orc_bc bc = is_left ? m->lu : m->ru;
    if (bc.type == ORC_BC_DIRICHLET) {
      m->rhs[row] -= value * bc.value;
    } else {
      const int ii = is_left ? 1 : s->cfg.nx - 1;
      ra_add(&m->rows[row], u_row(m, ii, uj), value);
      m->rhs[row] -= value * bc.value * s->dx;
    }
    return;
  }
  fail(s, "unexpected inactive u x-neighbor in momentum predictor");
}
static void add_u_y(mom_ctx *m, int row, int ui, int uj, double value) {
  orc_solver *s = m->s;
  if (u_active(s, ui, uj)) {
    ra_add(&m->rows[row], u_row(m, ui, uj), value);
    return;
  }
  if (!s->cfg.periodic_y && (uj < 0 || uj >= s->cfg.ny)) {
    const int is_bottom = uj < 0;
    const orc_bc bc = is_bottom ? m->bu : m->tu;
    const int jj = is_bottom ? 0 : s->cfg.ny - 1;
    if (bc.type == ORC_BC_DIRICHLET) {
      ra_add(&m->rows[row], u_row(m, ui, jj), -value);
      m->rhs[row] -= value * (2.0 * bc.value);
    } else {
      ra_add(&m->rows[row], u_row(m, ui, jj), value);
      m->rhs[row] -= value * bc.value * s->dy;
    }
    return;
  }
  fail(s, "unexpected inactive u y-neighbor in momentum predictor");
}
static void add_v_y(mom_ctx *m, int row, int vi, int vj, double value) {
  orc_solver *s = m->s;
  if (v_active(s, vi, vj)) {
    ra_add(&m->rows[row], v_row(m, vi, vj), value);
    return;
  }
  if (!s->cfg.periodic_y && (vj <= 0 || vj >= s->cfg.ny)) {
    const int is_bottom = vj <= 0;
    const orc_bc bc = is_bottom ? m->bv : m->tv;
    if (bc.type == ORC_BC_DIRICHLET) {
      m->rhs[row] -= value * bc.value;
    } else {
      const int jj = is_bottom ? 1 : s->cfg.ny - 1;
      ra_add(&m->rows[row], v_row(m, vi, jj), value);
      m->rhs[row] -= value * bc.value * s->dy;
    }
    return;
  }
  fail(s, "unexpected inactive v y-neighbor in momentum predictor");
}
static void add_v_x(mom_ctx *m, int row, int vi, int vj, double value) {
  orc_solver *s = m->s;
  if (v_active(s, vi, vj)) {
    ra_add(&m->rows[row], v_row(m, vi, vj), value);
    return;
  }
  if (!s->cfg.periodic_x && (vi < 0 || vi >= s->cfg.nx)) {
    const int is_left = vi < 0;
    const orc_bc bc = is_left ? m->lv : m->rv;
    const int ii = is_left ? 0 : s->cfg.nx - 1;
    if (bc.type == ORC_BC_DIRICHLET) {
      ra_add(&m->rows[row], v_row(m, ii, vj), -value);
      m->rhs[row] -= value * (2.0 * bc.value);
    } else {
      ra_add(&m->rows[row], v_row(m, ii, vj), value);
      m->rhs[row] -= value * bc.value * s->dx;
    }
    return;
  }
  fail(s, "unexpected inactive v x-neighbor in momentum predictor");
}

/* solve_momentum_predictor, momentum.cpp:157-502 */
static double momentum_predictor(orc_solver *s, const fld *uadv, const fld *vadv, int step) {
  const int nx = s->cfg.nx, ny = s->cfg.ny, g = s->cfg.ghost;
  const double dt = s->cfg.dt;
  const double alpha = 0.5 * dt / s->cfg.re;
  const fld *u = &s->f[ORC_F_U], *v = &s->f[ORC_F_V];
  const fld *rm = &s->f[ORC_F_RHO_MID], *eta = &s->f[ORC_F_ETA], *etap = &s->f[ORC_F_ETA_PREV];
  fld urhs, vrhs;
  fld_init(&urhs, nx + 1, ny, g, 0.0);
  fld_init(&vrhs, nx, ny + 1, g, 0.0);
  for (int i = 0; i < nx + 1; ++i)
    for (int j = 0; j < ny; ++j) {
      const double rf = xface(s, rm, i, j);
      const double conv = (step == 0) ? AT(uadv, i, j) : 1.5 * AT(uadv, i, j) - 0.5 * AT(&s->f[ORC_F_HU_PREV], i, j);
      const double vo = visc_u(s, u, v, etap, i, j);
      AT(&urhs, i, j) = rf * AT(u, i, j) +
                        dt * (-rf * conv + rf * s->cfg.body_force_x + AT(&s->f[ORC_F_SFX_U], i, j)) + alpha * vo;
    }
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny + 1; ++j) {
      const double rf = yface(s, rm, i, j);
      const double conv = (step == 0) ? AT(vadv, i, j) : 1.5 * AT(vadv, i, j) - 0.5 * AT(&s->f[ORC_F_HV_PREV], i, j);
      const double vo = visc_v(s, u, v, etap, i, j);
      AT(&vrhs, i, j) = rf * AT(v, i, j) +
                        dt * (-rf * conv + rf * s->cfg.body_force_y + AT(&s->f[ORC_F_SFY_V], i, j)) + alpha * vo;
    }
  mom_ctx m;
  m.s = s;
  m.u_row_of = (int *)malloc((size_t)(nx + 1) * ny * sizeof(int));
  m.v_row_of = (int *)malloc((size_t)nx * (ny + 1) * sizeof(int));
  m.lu = eff_u_bc(s, ORC_LEFT);
  m.ru = eff_u_bc(s, ORC_RIGHT);
  m.bu = eff_u_bc(s, ORC_BOTTOM);
  m.tu = eff_u_bc(s, ORC_TOP);
  m.lv = eff_v_bc(s, ORC_LEFT);
  m.rv = eff_v_bc(s, ORC_RIGHT);
  m.bv = eff_v_bc(s, ORC_BOTTOM);
  m.tv = eff_v_bc(s, ORC_TOP);
  int un = 0, vn = 0;
  for (int i = 0; i < nx + 1; ++i)
    for (int j = 0; j < ny; ++j) m.u_row_of[i * ny + j] = u_active(s, i, j) ? un++ : -1;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny + 1; ++j) m.v_row_of[i * (ny + 1) + j] = v_active(s, i, j) ? vn++ : -1;
  m.u_unknowns = un;
  const int total = un + vn;
  m.rows = rows_get(s, total);
  m.rhs = s->w[14];
  double *x = s->w[15];
  for (int k = 0; k < total; ++k) {
    m.rhs[k] = 0.0;
    x[k] = 0.0;
  }
  const double dx = s->dx, dy = s->dy;
  for (int i = 0; i < nx + 1; ++i)
    for (int j = 0; j < ny; ++j) {
      if (!u_active(s, i, j)) continue;
      const int row = u_row(&m, i, j);
      m.rhs[row] = AT(&urhs, i, j);
      x[row] = AT(u, i, j);
      const double rf = xface(s, rm, i, j);
      const double eta_e = xface(s, eta, i + 1, j), eta_w = xface(s, eta, i, j);
      const double eta_n = corner(eta, i, j + 1), eta_s = corner(eta, i, j);
      const double ce = 2.0 * eta_e / (dx * dx), cw = 2.0 * eta_w / (dx * dx);
      const double cn = eta_n / (dy * dy), cs = eta_s / (dy * dy);
      const double xn = eta_n / (dx * dy), xs = eta_s / (dx * dy);
      ra_add(&m.rows[row], row, rf + alpha * (ce + cw + cn + cs));
      add_u_x(&m, row, can_ui(s, i + 1), j, -alpha * ce);
      add_u_x(&m, row, can_ui(s, i - 1), j, -alpha * cw);
      add_u_y(&m, row, i, can_uj(s, j + 1), -alpha * cn);
      add_u_y(&m, row, i, can_uj(s, j - 1), -alpha * cs);
      add_v_y(&m, row, can_vi(s, i), can_vj(s, j + 1), -alpha * xn);
      add_v_y(&m, row, can_vi(s, i - 1), can_vj(s, j + 1), alpha * xn);
      add_v_y(&m, row, can_vi(s, i), can_vj(s, j), alpha * xs);
      add_v_y(&m, row, can_vi(s, i - 1), can_vj(s, j), -alpha * xs);
    }
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny + 1; ++j) {
      if (!v_active(s, i, j)) continue;
      const int row = v_row(&m, i, j);
      m.rhs[row] = AT(&vrhs, i, j);
      x[row] = AT(v, i, j);
      const double rf = yface(s, rm, i, j);
      const double eta_e = corner(eta, i + 1, j), eta_w = corner(eta, i, j);
      const double eta_n = yface(s, eta, i, j + 1), eta_s = yface(s, eta, i, j);
      const double ce = eta_e / (dx * dx), cw = eta_w / (dx * dx);
      const double cn = 2.0 * eta_n / (dy * dy), cs = 2.0 * eta_s / (dy * dy);
      const double xe = eta_e / (dx * dy), xw = eta_w / (dx * dy);
      ra_add(&m.rows[row], row, rf + alpha * (ce + cw + cn + cs));
      add_v_x(&m, row, can_vi(s, i + 1), j, -alpha * ce);
      add_v_x(&m, row, can_vi(s, i - 1), j, -alpha * cw);
      add_v_y(&m, row, i, can_vj(s, j + 1), -alpha * cn);
      add_v_y(&m, row, i, can_vj(s, j - 1), -alpha * cs);
      add_u_x(&m, row, can_ui(s, i + 1), can_uj(s, j), -alpha * xe);
      add_u_x(&m, row, can_ui(s, i + 1), can_uj(s, j - 1), alpha * xe);
      add_u_x(&m, row, can_ui(s, i), can_uj(s, j), alpha * xw);
      add_u_x(&m, row, can_ui(s, i), can_uj(s, j - 1), -alpha * xw);
    }
  finalize_rows(s, m.rows, total, &s->pm);
  build_diag_pc(&s->pm, &s->ppc);
  const solve_rep rep =
      bicgstab(s, &s->pm, &s->ppc, m.rhs, s->cfg.momentum_iterations, s->cfg.momentum_tolerance, x, 0);
  fld *us = &s->f[ORC_F_U_STAR], *vs = &s->f[ORC_F_V_STAR];
  fld_copy(us, u);
  fld_copy(vs, v);
  for (int i = 0; i < nx + 1; ++i)
    for (int j = 0; j < ny; ++j)
      if (u_active(s, i, j)) AT(us, i, j) = x[u_row(&m, i, j)];
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny + 1; ++j)
      if (v_active(s, i, j)) AT(vs, i, j) = x[v_row(&m, i, j)];
  bc_u(s, us);
  bc_v(s, vs);
  fld_copy(&s->f[ORC_F_HU_PREV], uadv);
  fld_copy(&s->f[ORC_F_HV_PREV], vadv);
  s->rep.momentum_iterations = rep.iterations;
  free(m.u_row_of);
  free(m.v_row_of);
  fld_free(&urhs);
  fld_free(&vrhs);
  return rep.absolute_residual;
}

/* ------------------------------------------------------------------------------------------ */
/* Pressure correction (pressure.cpp, operators.cpp:400-534)                                    */
/* ------------------------------------------------------------------------------------------ */
static int use_split(const orc_solver *s) {
  return s->cfg.pressure_scheme == ORC_P_SPLIT_ICPCG || s->cfg.pressure_scheme == ORC_P_SPLIT_ILDLT_PCG ||
         s->cfg.pressure_scheme == ORC_P_SPLIT_DCDM_ICPCG;
}
static double split_rho_ref(const orc_solver *s) { return dmin(1.0, s->cfg.density_ratio); }

/* build_liu_split_pressure_extrapolation, operators.cpp:413-422 */
static void split_extrapolation(orc_solver *s, fld *pe) {
  const fld *p = &s->f[ORC_F_P], *pp = &s->f[ORC_F_P_PREV];
  for (int i = 0; i < s->cfg.nx; ++i)
    for (int j = 0; j < s->cfg.ny; ++j)
      AT(pe, i, j) = (s->current_step_index == 0) ? AT(p, i, j) : (2.0 * AT(p, i, j) - AT(pp, i, j));
  bc_pressure(s, pe);
}

/* liu_split_explicit_divergence, operators.cpp:424-444 */
static double split_divergence(const orc_solver *s, const fld *pe, int i, int j) {
  const double rho_ref = split_rho_ref(s);
  const fld *rm = &s->f[ORC_F_RHO_MID];
  const int eo = s->cfg.periodic_x || i < s->cfg.nx - 1, wo = s->cfg.periodic_x || i > 0;
  const int no = s->cfg.periodic_y || j < s->cfg.ny - 1, so = s->cfg.periodic_y || j > 0;
  const double fe = eo ? (1.0 - rho_ref / xface(s, rm, i + 1, j)) * gfx(s, pe, i + 1, j) : 0.0;
  const double fw = wo ? (1.0 - rho_ref / xface(s, rm, i, j)) * gfx(s, pe, i, j) : 0.0;
  const double fn = no ? (1.0 - rho_ref / yface(s, rm, i, j + 1)) * gfy(s, pe, i, j + 1) : 0.0;
  const double fs = so ? (1.0 - rho_ref / yface(s, rm, i, j)) * gfy(s, pe, i, j) : 0.0;
  return (fe - fw) / s->dx + (fn - fs) / s->dy;
}

/* build_pressure_linear_system + regularize_pressure_linear_system, pressure.cpp:123-212 */
static void pressure_system(orc_solver *s, int split, double rho_ref, const fld *pe, double *rhs) {
  const int nx = s->cfg.nx, ny = s->cfg.ny, n = nx * ny;
  const int px = s->cfg.periodic_x, py = s->cfg.periodic_y;
  const double dx = s->dx, dy = s->dy, dt = s->cfg.dt;
  const fld *rm = &s->f[ORC_F_RHO_MID], *us = &s->f[ORC_F_U_STAR], *vs = &s->f[ORC_F_V_STAR];
  rowacc *rows = rows_get(s, n);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      const int row = i * ny + j;
      const int he = px || i < nx - 1, hw = px || i > 0, hn = py || j < ny - 1, hs = py || j > 0;
      const double ce = split ? 1.0 / (dx * dx) : 1.0 / (xface(s, rm, i + 1, j) * dx * dx);
      const double cw = split ? 1.0 / (dx * dx) : 1.0 / (xface(s, rm, i, j) * dx * dx);
      const double cn = split ? 1.0 / (dy * dy) : 1.0 / (yface(s, rm, i, j + 1) * dy * dy);
      const double cs = split ? 1.0 / (dy * dy) : 1.0 / (yface(s, rm, i, j) * dy * dy);
      double diag = 0.0;
      double rv = split ? -(split_divergence(s, pe, i, j) + rho_ref * div_cell(s, us, vs, i, j) / dt)
                        : -div_cell(s, us, vs, i, j) / dt;
#define ADD_BOUNDARY(side, coeff, spacing)                                                                      \
  do {                                                                                                            \
    const orc_bc bc_ = eff_p_bc(s, side);                                                                         \
    if (bc_.type == ORC_BC_DIRICHLET) {                                                                           \
      diag += 2.0 * (coeff);                                                                                      \
      rv += 2.0 * (coeff)*bc_.value;                                                                              \
    } else {                                                                                                      \
      rv += (coeff)*bc_.value * (spacing);                                                                        \
    }                                                                                                             \
  } while (0)
      if (he) {
        diag += ce;
        const int ie = px && i == nx - 1 ? 0 : i + 1;
        ra_add(&rows[row], ie * ny + j, -ce);
      } else {
        ADD_BOUNDARY(ORC_RIGHT, ce, dx);
      }
      if (hw) {
        diag += cw;
        const int iw = px && i == 0 ? nx - 1 : i - 1;
        ra_add(&rows[row], iw * ny + j, -cw);
      } else {
        ADD_BOUNDARY(ORC_LEFT, cw, dx);
      }
      if (hn) {
        diag += cn;
        const int jn = py && j == ny - 1 ? 0 : j + 1;
        ra_add(&rows[row], i * ny + jn, -cn);
      } else {
        ADD_BOUNDARY(ORC_TOP, cn, dy);
      }
      if (hs) {
        diag += cs;
        const int js = py && j == 0 ? ny - 1 : j - 1;
        ra_add(&rows[row], i * ny + js, -cs);
      } else {
        ADD_BOUNDARY(ORC_BOTTOM, cs, dy);
      }
#undef ADD_BOUNDARY
      ra_add(&rows[row], row, diag);
      rhs[row] = rv;
    }
  if (!pressure_has_dirichlet(s)) {
    double acc = 0.0;
    for (int k = 0; k < n; ++k) acc += rhs[k];
    const double mean = acc / dmax((double)n, 1.0);
    for (int k = 0; k < n; ++k) rhs[k] -= mean;
  }
  finalize_rows(s, rows, n, &s->pm);
}

static void scatter_pressure(orc_solver *s, const double *x) {
  fld *pc = &s->f[ORC_F_P_CORR];
  for (int i = 0; i < s->cfg.nx; ++i)
    for (int j = 0; j < s->cfg.ny; ++j) AT(pc, i, j) = x[i * s->cfg.ny + j];
}

/* solve_pressure_correction_{icpcg,ildlt_pcg,liu_split_icpcg,liu_split_ildlt_pcg}, pressure.cpp:302-365, 470-491 */
static double pressure_pcg(orc_solver *s, int split, int icc) {
  fld *pc = &s->f[ORC_F_P_CORR];
  fld_fill(pc, 0.0);
  bc_pressure(s, pc);
  s->rep.pressure_iterations = 0;
  const int n = s->cfg.nx * s->cfg.ny;
  double *rhs = s->w[11], *x = s->w[12];
  fld pe;
  fld_init(&pe, s->cfg.nx, s->cfg.ny, s->cfg.ghost, 0.0);
  double rho_ref = 1.0;
  if (split) {
    split_extrapolation(s, &pe);
    rho_ref = split_rho_ref(s);
  }
  pressure_system(s, split, rho_ref, split ? &pe : NULL, rhs);
  fld_free(&pe);
  for (int k = 0; k < n; ++k) x[k] = 0.0;
  if (icc) {
    if (!try_icc(&s->pm, &s->ppc)) fail(s, "ICC preconditioner construction failed");
  } else {
    if (!try_ildlt(&s->pm, &s->ppc)) fail(s, "ILDLT preconditioner construction failed");
  }
  for (int k = 0; k < n; ++k) x[k] = 0.0;
  s->mon_active = 1;
  s->mon_count = 0;
  const solve_rep rep = pcg(s, &s->pm, &s->ppc, rhs, s->cfg.poisson_iterations, s->cfg.pressure_tolerance, x,
                            !pressure_has_dirichlet(s));
  s->mon_active = 0;
  s->rep.pressure_iterations = rep.iterations;
  scatter_pressure(s, x);
  if (!pressure_has_dirichlet(s)) subtract_mean(s, pc);
  bc_pressure(s, pc);
  return rep.relative_residual;
}

/* solve_dcdm_conjugate_directions, ch_sparse_krylov.hpp:662-837: conjugate directions from the ICC-applied
 * (or identity) normalised residual, A-orthogonalised against the last history_size stored directions (all
 * stored ones when history_size is 0), at most max(max_stored, history_size, 1) kept, cleared every
 * restart_interval iterations; the residual is recomputed as b - A x after every update. */
static solve_rep dcdm(orc_solver *s, const csr *m, const precond *pc, const double *rhs, int max_it, double tol,
                      double *x, int project) {
  const int n = m->n;
  const double floor_ = 1.0e-30;
  double *ax = s->w[0], *r = s->w[1], *rh = s->w[2], *z = s->w[3], *d = s->w[4], *ad = s->w[5], *y = s->w[6];
  solve_rep rep = {0, 0.0, 0.0, 0.0};
  if (n <= 0) fail(s, "cannot solve an empty linear system");
  spmv(m, x, ax);
  for (int k = 0; k < n; ++k) r[k] = rhs[k] - ax[k];
  if (project) {
    project_mean(r, n);
    project_mean(x, n);
  }
  const double rhs_norm = sqrt(dmax(dot(rhs, rhs, n), 0.0));
  rep.absolute_residual = sqrt(dmax(dot(r, r, n), 0.0));
  rep.relative_residual = rep.absolute_residual / dmax(rhs_norm, 1.0e-30);
  if (rep.relative_residual < tol || rep.absolute_residual < tol) return rep;
  const int hist = s->cfg.dcdm_history_size;
  const int keep_max = (int)dmax((double)s->cfg.dcdm_max_stored_directions, dmax((double)hist, 1.0));
  double **dirs = (double **)calloc((size_t)keep_max + 1, sizeof(double *));
  double **adirs = (double **)calloc((size_t)keep_max + 1, sizeof(double *));
  for (int k = 0; k <= keep_max; ++k) {
    dirs[k] = (double *)malloc((size_t)n * sizeof(double));
    adirs[k] = (double *)malloc((size_t)n * sizeof(double));
  }
  int stored = 0;
  const char *err = NULL;
  const int limit = max_it > 1 ? max_it : 1;
  for (int it = 0; it < limit; ++it) {
    if (s->cfg.dcdm_restart_interval > 0 && it > 0 && (it % s->cfg.dcdm_restart_interval) == 0) stored = 0;
    const double rnorm = sqrt(dmax(dot(r, r, n), 0.0));
    if (rnorm < tol) break;
    for (int k = 0; k < n; ++k) rh[k] = r[k] / dmax(rnorm, floor_);
    if (s->cfg.dcdm_direction_mode == 1)
      memcpy(z, rh, (size_t)n * sizeof(double));
    else
      apply_pc(m, pc, rh, z, y);
    int finite = 1;
    for (int k = 0; k < n && finite; ++k) finite = isfinite(z[k]);
    if (!finite || sqrt(dmax(dot(z, z, n), 0.0)) < floor_) memcpy(z, r, (size_t)n * sizeof(double));
    if (project) project_mean(z, n);
    finite = 1;
    for (int k = 0; k < n && finite; ++k) finite = isfinite(z[k]);
    if (!finite || sqrt(dmax(dot(z, z, n), 0.0)) < floor_) {
      memcpy(z, r, (size_t)n * sizeof(double));
      if (project) project_mean(z, n);
    }
    memcpy(d, z, (size_t)n * sizeof(double));
    const int begin = (hist > 0 && stored > hist) ? stored - hist : 0;
    for (int h = begin; h < stored; ++h) {
      const double den = dot(dirs[h], adirs[h], n);
      if (!isfinite(den) || fabs(den) < floor_) continue;
      const double coeff = dot(d, adirs[h], n) / den;
      for (int k = 0; k < n; ++k) d[k] -= coeff * dirs[h][k];
    }
    if (project) project_mean(d, n);
    spmv(m, d, ad);
    double rd = dot(r, d, n), dad = dot(d, ad, n);
    finite = 1;
    for (int k = 0; k < n && finite; ++k) finite = isfinite(d[k]) && isfinite(ad[k]);
    if (!finite || sqrt(dmax(dot(d, d, n), 0.0)) < floor_ || !isfinite(rd) || rd <= 0.0 || !isfinite(dad) ||
        fabs(dad) < floor_) {
      memcpy(d, r, (size_t)n * sizeof(double));
      if (project) project_mean(d, n);
      spmv(m, d, ad);
      rd = dot(r, d, n);
      dad = dot(d, ad, n);
      if (!isfinite(rd) || rd <= 0.0 || !isfinite(dad) || fabs(dad) < floor_) {
        err = "dcdm breakdown: invalid fallback direction";
        break;
      }
    }
    const double alpha = rd / dad;
    double update_sq = 0.0;
    for (int k = 0; k < n; ++k) {
      const double delta = alpha * d[k];
      x[k] += delta;
      update_sq += delta * delta;
    }
    if (project) project_mean(x, n);
    spmv(m, x, ax);
    for (int k = 0; k < n; ++k) r[k] = rhs[k] - ax[k];
    if (project) project_mean(r, n);
    const double x_norm_sq = dot(x, x, n);
    rep.iterations = it + 1;
    rep.iterate_residual = sqrt(update_sq / dmax(x_norm_sq, 1.0e-30));
    rep.absolute_residual = sqrt(dmax(dot(r, r, n), 0.0));
    rep.relative_residual = rep.absolute_residual / dmax(rhs_norm, 1.0e-30);
    monitor_record(s, it, &rep, alpha);
    /* push_back, then drop the oldest beyond keep_max */
    memcpy(dirs[stored], d, (size_t)n * sizeof(double));
    memcpy(adirs[stored], ad, (size_t)n * sizeof(double));
    ++stored;
    if (stored > keep_max) {
      double *t0 = dirs[0], *t1 = adirs[0];
      for (int h = 0; h < stored - 1; ++h) {
        dirs[h] = dirs[h + 1];
        adirs[h] = adirs[h + 1];
      }
      dirs[stored - 1] = t0;
      adirs[stored - 1] = t1;
      --stored;
    }
    if (rep.relative_residual < tol || rep.absolute_residual < tol) break;
  }
  for (int k = 0; k <= keep_max; ++k) {
    free(dirs[k]);
    free(adirs[k]);
  }
  free(dirs);
  free(adirs);
  if (err) fail(s, err);
  return rep;
}

/* solve_pressure_correction_liu_split_dcdm_icpcg, pressure.cpp:367-468 (icc_preconditioned and identity
 * directions; the neural direction needs an external worker) */
static double pressure_dcdm(orc_solver *s) {
  fld *pc = &s->f[ORC_F_P_CORR];
  fld_fill(pc, 0.0);
  bc_pressure(s, pc);
  s->rep.pressure_iterations = 0;
  const int n = s->cfg.nx * s->cfg.ny;
  double *rhs = s->w[11], *x = s->w[12];
  fld pe;
  fld_init(&pe, s->cfg.nx, s->cfg.ny, s->cfg.ghost, 0.0);
  split_extrapolation(s, &pe);
  pressure_system(s, 1, split_rho_ref(s), &pe, rhs);
  fld_free(&pe);
  for (int k = 0; k < n; ++k) x[k] = 0.0;
  if (!try_icc(&s->pm, &s->ppc)) fail(s, "ICC preconditioner construction failed");
  s->mon_active = 1;
  s->mon_count = 0;
  const solve_rep rep = dcdm(s, &s->pm, &s->ppc, rhs, s->cfg.poisson_iterations, s->cfg.pressure_tolerance, x,
                             !pressure_has_dirichlet(s));
  s->mon_active = 0;
  s->rep.pressure_iterations = rep.iterations;
  scatter_pressure(s, x);
  if (!pressure_has_dirichlet(s)) subtract_mean(s, pc);
  bc_pressure(s, pc);
  return rep.relative_residual;
}

/* solve_pressure_correction_jacobi, pressure.cpp:250-300 */
static double pressure_jacobi(orc_solver *s) {
  fld *pc = &s->f[ORC_F_P_CORR];
  fld_fill(pc, 0.0);
  bc_pressure(s, pc);
  s->rep.pressure_iterations = 0;
  const int n = s->cfg.nx * s->cfg.ny;
  double *rhs = s->w[11], *x = s->w[12], *xn = s->w[13];
  pressure_system(s, 0, 1.0, NULL, rhs);
  const csr *m = &s->pm;
  for (int k = 0; k < n; ++k) {
    x[k] = 0.0;
    xn[k] = 0.0;
  }
  double residual = 0.0;
  for (int it = 0; it < s->cfg.poisson_iterations; ++it) {
    double max_res = 0.0;
    for (int row = 0; row < m->n; ++row) {
      double diag = 0.0, ax = 0.0;
      for (int p = m->row_ptr[row]; p < m->row_ptr[row + 1]; ++p) {
        ax += m->val[p] * x[m->col[p]];
        if (m->col[p] == row) diag = m->val[p];
      }
      const double rr = rhs[row] - ax;
      if (!isfinite(rr) || !isfinite(diag) || fabs(diag) < 1.0e-30) fail(s, "Jacobi pressure solve diverged");
      xn[row] = x[row] + 1.0 * rr / dmax(fabs(diag), 1.0e-30);
      max_res = dmax(max_res, fabs(rr));
    }
    double *t = x;
    x = xn;
    xn = t;
    residual = max_res;
    s->rep.pressure_iterations = it + 1;
    if (residual < s->cfg.pressure_tolerance) break;
  }
  scatter_pressure(s, x);
  if (!pressure_has_dirichlet(s)) subtract_mean(s, pc);
  bc_pressure(s, pc);
  return residual;
}

/* solve_pressure_correction dispatcher, pressure.cpp:1031-1071 */
static double pressure_solve(orc_solver *s) {
  switch (s->cfg.pressure_scheme) {
  case ORC_P_ICPCG: return pressure_pcg(s, 0, 1);
  case ORC_P_ILDLT_PCG: return pressure_pcg(s, 0, 0);
  case ORC_P_SPLIT_ICPCG: return pressure_pcg(s, 1, 1);
  case ORC_P_SPLIT_ILDLT_PCG: return pressure_pcg(s, 1, 0);
  case ORC_P_SPLIT_DCDM_ICPCG: return pressure_dcdm(s);
  case ORC_P_JACOBI: return pressure_jacobi(s);
  default: fail(s, "unsupported pressure scheme"); return 0.0;
  }
}

/* apply_pressure_velocity_correction, operators.cpp:480-534 */
static void velocity_correction(orc_solver *s) {
  fld *u = &s->f[ORC_F_U], *v = &s->f[ORC_F_V], *us = &s->f[ORC_F_U_STAR], *vs = &s->f[ORC_F_V_STAR];
  const fld *rm = &s->f[ORC_F_RHO_MID], *pc = &s->f[ORC_F_P_CORR];
  s->rep.boundary_speed_pre = boundary_speed(s, us, vs);
  fld pe;
  fld_init(&pe, s->cfg.nx, s->cfg.ny, s->cfg.ghost, 0.0);
  const int split = use_split(s);
  const double rho_ref = split ? split_rho_ref(s) : 1.0;
  if (split) split_extrapolation(s, &pe);
  const double dt = s->cfg.dt;
  for (int i = 0; i < u->nx; ++i)
    for (int j = 0; j < u->ny; ++j) {
      const double se = split ? (1.0 / xface(s, rm, i, j) - 1.0 / rho_ref) * gfx(s, &pe, i, j) : 0.0;
      const double si = split ? gfx(s, pc, i, j) / rho_ref : gfx(s, pc, i, j) / xface(s, rm, i, j);
      AT(u, i, j) = AT(us, i, j) - dt * (si + se);
    }
  for (int i = 0; i < v->nx; ++i)
    for (int j = 0; j < v->ny; ++j) {
      const double se = split ? (1.0 / yface(s, rm, i, j) - 1.0 / rho_ref) * gfy(s, &pe, i, j) : 0.0;
      const double si = split ? gfy(s, pc, i, j) / rho_ref : gfy(s, pc, i, j) / yface(s, rm, i, j);
      AT(v, i, j) = AT(vs, i, j) - dt * (si + se);
    }
  bc_u(s, u);
  bc_v(s, v);
  s->rep.boundary_speed_post = boundary_speed(s, u, v);
  fld_copy(&s->f[ORC_F_P_PREV], &s->f[ORC_F_P]);
  fld *p = &s->f[ORC_F_P];
  for (int i = 0; i < s->cfg.nx; ++i)
    for (int j = 0; j < s->cfg.ny; ++j) AT(p, i, j) = AT(pc, i, j);
  if (!pressure_has_dirichlet(s)) subtract_mean(s, p);
  bc_pressure(s, p);
  fld_free(&pe);
}

/* ------------------------------------------------------------------------------------------ */
/* Initialisation (solver.cpp:69-221)                                                          */
/* ------------------------------------------------------------------------------------------ */
static double sd_box(double x, double y, double cx, double cy, double hx, double hy) {
  const double qx = fabs(x - cx) - hx, qy = fabs(y - cy) - hy;
  const double ox = dmax(qx, 0.0), oy = dmax(qy, 0.0);
  return hypot(ox, oy) + dmin(dmax(qx, qy), 0.0);
}

static void init_phase(orc_solver *s) {
  const orc_config *c = &s->cfg;
  fld *cf = &s->f[ORC_F_C];
  if (c->phase_initializer == 1) { /* initialize_zalesak_disk, solver.cpp:152-174 */
    const double cx = c->interface_center_x, cy = c->interface_center_y, radius = c->interface_radius;
    const double shw = 0.5 * c->zalesak_slot_width;
    const double st = cy + radius, sb = st - c->zalesak_slot_depth;
    const double scy = 0.5 * (st + sb), shh = 0.5 * (st - sb);
    const double sm = dmax(2.0 * sqrt(2.0) * c->cn, 1.0e-12);
    for (int i = 0; i < c->nx; ++i)
      for (int j = 0; j < c->ny; ++j) {
        const double x = ((double)i + 0.5) * s->dx, y = ((double)j + 0.5) * s->dy;
        const double dsd = hypot(x - cx, y - cy) - radius;
        const double ssd = sd_box(x, y, cx, scy, shw, shh);
        const double shape = dmax(dsd, -ssd);
        const double value = 0.5 - 0.5 * tanh(shape / sm);
        AT(cf, i, j) = c->invert_phase ? (1.0 - value) : value;
      }
    return;
  }
  for (int i = 0; i < c->nx; ++i)
    for (int j = 0; j < c->ny; ++j) {
      const double x = ((double)i + 0.5) * s->dx, y = ((double)j + 0.5) * s->dy;
      double value = 1.0;
      if (is_single(s)) {
        AT(cf, i, j) = c->invert_phase ? 0.0 : 1.0;
        continue;
      }
      if (!is_adv_only(s)) {
        if (c->interface_radius > 0.0) {
          const double rx = x - c->interface_center_x, ry = y - c->interface_center_y;
          const double r = sqrt(rx * rx + ry * ry);
          value = 0.5 - 0.5 * tanh((r - c->interface_radius) / (2.0 * sqrt(2.0) * c->cn));
        } else {
          const double y0 = c->interface_center_y +
                            c->interface_amplitude * cos(2.0 * M_PI * c->interface_wavenumber * x / dmax(c->lx, 1.0e-12));
          value = 0.5 - 0.5 * tanh((y - y0) / (2.0 * sqrt(2.0) * c->cn));
        }
      }
      AT(cf, i, j) = c->invert_phase ? (1.0 - value) : value;
    }
}

static void init_velocity(orc_solver *s) {
  const orc_config *c = &s->cfg;
  fld *u = &s->f[ORC_F_U], *v = &s->f[ORC_F_V];
  if (c->velocity_profile == 1) { /* fill_solid_body_rotation_velocity, solver.cpp:208-221 */
    for (int i = -u->g; i < u->nx + u->g; ++i)
      for (int j = -u->g; j < u->ny + u->g; ++j) {
        const double y = ((double)j + 0.5) * s->dy;
        AT(u, i, j) = -c->angular_velocity * (y - c->rotation_center_y);
      }
    for (int i = -v->g; i < v->nx + v->g; ++i)
      for (int j = -v->g; j < v->ny + v->g; ++j) {
        const double x = ((double)i + 0.5) * s->dx;
        AT(v, i, j) = c->angular_velocity * (x - c->rotation_center_x);
      }
    return;
  }
  const orc_bc bb = eff_u_bc(s, ORC_BOTTOM), tb = eff_u_bc(s, ORC_TOP);
  const int couette = !c->periodic_y && bb.type == ORC_BC_DIRICHLET && tb.type == ORC_BC_DIRICHLET &&
                      (fabs(tb.value) > 0.0 || fabs(bb.value) > 0.0);
  for (int i = 0; i < u->nx; ++i)
    for (int j = 0; j < u->ny; ++j) {
      if (couette) {
        const double y = ((double)j + 0.5) * s->dy;
        AT(u, i, j) = bb.value + (tb.value - bb.value) * y / dmax(c->ly, 1.0e-30);
      } else {
        AT(u, i, j) = c->advect_u;
      }
    }
  for (int i = 0; i < v->nx; ++i)
    for (int j = 0; j < v->ny; ++j) AT(v, i, j) = c->advect_v;
  bc_u(s, u);
  bc_v(s, v);
}

/* ------------------------------------------------------------------------------------------ */
/* Public API                                                                                  */
/* ------------------------------------------------------------------------------------------ */
orc_solver *orc_create(const orc_config *cfg) {
  orc_solver *s = (orc_solver *)calloc(1, sizeof(orc_solver));
  s->cfg = *cfg;
  const int nx = cfg->nx, ny = cfg->ny, g = cfg->ghost;
  s->dx = cfg->lx / dmax((double)nx, 1.0);
  s->dy = cfg->ly / dmax((double)ny, 1.0);
  for (int k = 0; k < ORC_F_COUNT; ++k) {
    int fx = nx, fy = ny;
    double init = 0.0;
    if (k == ORC_F_U || k == ORC_F_U_PREV || k == ORC_F_U_STAR || k == ORC_F_SFX_U || k == ORC_F_HU_PREV) fx = nx + 1;
    if (k == ORC_F_V || k == ORC_F_V_PREV || k == ORC_F_V_STAR || k == ORC_F_SFY_V || k == ORC_F_HV_PREV) fy = ny + 1;
    if (k == ORC_F_RHO || k == ORC_F_ETA || k == ORC_F_RHO_PREV || k == ORC_F_ETA_PREV || k == ORC_F_RHO_MID ||
        k == ORC_F_ETA_MID)
      init = 1.0;
    fld_init(&s->f[k], fx, fy, g, init);
  }
  s->wn = (nx + 1) * ny + nx * (ny + 1) + 8;
  for (int k = 0; k < 16; ++k) s->w[k] = (double *)calloc((size_t)s->wn, sizeof(double));
  s->ch_cached_alpha0 = -1.0;
  s->rep.ch_preconditioner = -1;
  return s;
}

void orc_set_pressure_monitor(orc_solver *s, int capacity) {
  free(s->mon);
  s->mon = capacity > 0 ? (double *)calloc((size_t)capacity * 4, sizeof(double)) : NULL;
  s->mon_cap = capacity > 0 ? capacity : 0;
  s->mon_count = 0;
}

int orc_pressure_monitor(const orc_solver *s, double *out, int capacity) {
  const int m = s->mon_count < capacity ? s->mon_count : capacity;
  if (m > 0) memcpy(out, s->mon, (size_t)m * 4 * sizeof(double));
  return s->mon_count;
}

void orc_destroy(orc_solver *s) {
  if (!s) return;
  free(s->mon);
  for (int k = 0; k < ORC_F_COUNT; ++k) fld_free(&s->f[k]);
  for (int k = 0; k < 16; ++k) free(s->w[k]);
  csr_free(&s->ch_lap);
  csr_free(&s->ch_biharm);
  csr_free(&s->ch_sys);
  csr_free(&s->pm);
  pc_free(&s->ch_pc);
  pc_free(&s->ppc);
  free(s->rows);
  free(s);
}

const char *orc_last_error(const orc_solver *s) { return s->err; }

double *orc_field(orc_solver *s, int id, int *nx, int *ny, int *ghost) {
  if (id < 0 || id >= ORC_F_COUNT) return NULL;
  if (nx) *nx = s->f[id].nx;
  if (ny) *ny = s->f[id].ny;
  if (ghost) *ghost = s->f[id].g;
  return s->f[id].d;
}

void orc_set_initial_mass(orc_solver *s, double mass) { s->initial_mass = mass; }

#define GUARD_BEGIN                                                                                               \
  jmp_buf jb_;                                                                                                     \
  s->jb = &jb_;                                                                                                    \
  s->err[0] = 0;                                                                                                   \
  if (setjmp(jb_) != 0) {                                                                                          \
    s->jb = NULL;                                                                                                  \
    return 1;                                                                                                      \
  }
#define GUARD_END                                                                                                 \
  s->jb = NULL;                                                                                                    \
  return 0;

int orc_initialize(orc_solver *s) {
  GUARD_BEGIN
  /* validate_boundary_configuration, operators.cpp:11-34 */
  static const char *names[4] = {"left", "right", "bottom", "top"};
  for (int side = 0; side < 4; ++side) {
    const int periodic = (side < 2) ? s->cfg.periodic_x : s->cfg.periodic_y;
    if (!periodic) continue;
    if (s->cfg.p_bc[side].type != ORC_BC_UNSET) fail(s, "pressure_bc_%s cannot be set when the direction is periodic", names[side]);
    if (s->cfg.u_bc[side].type != ORC_BC_UNSET) fail(s, "u_bc_%s cannot be set when the direction is periodic", names[side]);
    if (s->cfg.v_bc[side].type != ORC_BC_UNSET) fail(s, "v_bc_%s cannot be set when the direction is periodic", names[side]);
  }
  if (s->cfg.surface_tension_smoothing_passes < 0) fail(s, "surface_tension_smoothing_passes must be non-negative");
  if (s->cfg.surface_tension_smoothing_weight < 0.0 || s->cfg.surface_tension_smoothing_weight > 0.25)
    fail(s, "surface_tension_smoothing_weight must lie in [0, 0.25]");
  init_phase(s);
  init_velocity(s);
  bc_scalar(s, &s->f[ORC_F_C]);
  fld_copy(&s->f[ORC_F_C_PREV], &s->f[ORC_F_C]);
  fld_copy(&s->f[ORC_F_C_PREV2], &s->f[ORC_F_C]);
  fld_copy(&s->f[ORC_F_U_PREV], &s->f[ORC_F_U]);
  fld_copy(&s->f[ORC_F_V_PREV], &s->f[ORC_F_V]);
  update_materials(s);
  fld_copy(&s->f[ORC_F_RHO_PREV], &s->f[ORC_F_RHO]);
  fld_copy(&s->f[ORC_F_ETA_PREV], &s->f[ORC_F_ETA]);
  fld_copy(&s->f[ORC_F_RHO_MID], &s->f[ORC_F_RHO]);
  fld_copy(&s->f[ORC_F_ETA_MID], &s->f[ORC_F_ETA]);
  refresh_mu(s);
  clear_surface_force(s);
  s->initial_mass = mass_of(s, &s->f[ORC_F_C]);
  fld_fill(&s->f[ORC_F_P], 0.0);
  bc_pressure(s, &s->f[ORC_F_P]);
  fld_copy(&s->f[ORC_F_P_PREV], &s->f[ORC_F_P]);
  fld_fill(&s->f[ORC_F_E_PREV], 0.0);
  GUARD_END
}

int orc_begin_step(orc_solver *s, int step) {
  s->current_step_index = step;
  fld_copy(&s->f[ORC_F_C_PREV2], &s->f[ORC_F_C_PREV]);
  fld_copy(&s->f[ORC_F_C_PREV], &s->f[ORC_F_C]);
  fld_copy(&s->f[ORC_F_RHO_PREV], &s->f[ORC_F_RHO]);
  fld_copy(&s->f[ORC_F_ETA_PREV], &s->f[ORC_F_ETA]);
  fld_copy(&s->f[ORC_F_U_PREV], &s->f[ORC_F_U]);
  fld_copy(&s->f[ORC_F_V_PREV], &s->f[ORC_F_V]);
  return 0;
}

int orc_phase(orc_solver *s, int step) {
  GUARD_BEGIN
  if (solve_ch(s)) {
    s->rep.ch_residual = ch_semi_implicit(s, &s->f[ORC_F_U], &s->f[ORC_F_V], step);
    update_materials(s);
    update_midpoint(s);
    surface_force(s, &s->f[ORC_F_C_PREV], &s->f[ORC_F_C]);
    s->rep.coupling_iterations = 1;
  } else {
    update_materials(s);
    update_midpoint(s);
    refresh_mu(s);
    surface_force(s, &s->f[ORC_F_C_PREV], &s->f[ORC_F_C]);
    s->rep.ch_iterations = 0;
    s->rep.ch_preconditioner = -1;
    s->rep.ch_equation_residual = 0.0;
    s->rep.ch_residual = 0.0;
    s->rep.coupling_iterations = 0;
  }
  GUARD_END
}

int orc_momentum(orc_solver *s, int step) {
  GUARD_BEGIN
  const int nx = s->cfg.nx, ny = s->cfg.ny, g = s->cfg.ghost;
  fld ua, va;
  fld_init(&ua, nx + 1, ny, g, 0.0);
  fld_init(&va, nx, ny + 1, g, 0.0);
  momentum_fluxes(s, &ua, &va);
  s->rep.momentum_residual = momentum_predictor(s, &ua, &va, step);
  fld_free(&ua);
  fld_free(&va);
  GUARD_END
}

int orc_pressure(orc_solver *s) {
  GUARD_BEGIN
  s->rep.pressure_residual = pressure_solve(s);
  GUARD_END
}

int orc_correct(orc_solver *s) {
  GUARD_BEGIN
  velocity_correction(s);
  GUARD_END
}

int orc_advection(orc_solver *s, const double *c, const double *u, const double *v, double *rhs) {
  GUARD_BEGIN
  const int nx = s->cfg.nx, ny = s->cfg.ny, g = s->cfg.ghost;
  const fld cf = {nx, ny, g, (double *)c}, uf = {nx + 1, ny, g, (double *)u}, vf = {nx, ny + 1, g, (double *)v};
  fld out = {nx, ny, g, rhs}, fx, fy;
  fld_init(&fx, nx + 1, ny, g, 0.0);
  fld_init(&fy, nx, ny + 1, g, 0.0);
  adv_fluxes(s, &cf, &uf, &vf, &fx, &fy, &out);
  fld_free(&fx);
  fld_free(&fy);
  GUARD_END
}

int orc_explicit_operator(orc_solver *s, const double *c, const double *u, const double *v, double *E) {
  GUARD_BEGIN
  const int nx = s->cfg.nx, ny = s->cfg.ny, g = s->cfg.ghost;
  const fld uf = {nx + 1, ny, g, (double *)u}, vf = {nx, ny + 1, g, (double *)v};
  fld cw, out = {nx, ny, g, E};
  fld_init(&cw, nx, ny, g, 0.0);
  memcpy(cw.d, c, fld_size(&cw) * sizeof(double));
  bc_scalar(s, &cw);
  phase_explicit(s, &cw, &uf, &vf, &out);
  fld_free(&cw);
  GUARD_END
}

int orc_finish_step(orc_solver *s) {
  GUARD_BEGIN
  refresh_mu(s);
  GUARD_END
}

int orc_step(orc_solver *s, int step) {
  orc_begin_step(s, step);
  if (is_adv_only(s)) {
    GUARD_BEGIN
    s->rep.ch_residual = advection_only(s);
    update_materials(s);
    fld_fill(&s->f[ORC_F_MU], 0.0);
    bc_scalar(s, &s->f[ORC_F_MU]);
    s->rep.ch_iterations = 3;
    s->rep.momentum_iterations = 0;
    s->rep.pressure_iterations = 0;
    s->rep.coupling_iterations = 0;
    s->rep.boundary_speed_pre = 0.0;
    s->rep.boundary_speed_post = 0.0;
    s->rep.ch_equation_residual = 0.0;
    GUARD_END
  }
  if (orc_phase(s, step)) return 1;
  if (orc_momentum(s, step)) return 1;
  if (orc_pressure(s)) return 1;
  if (orc_correct(s)) return 1;
  return orc_finish_step(s);
}

int orc_ch_linear_solve(orc_solver *s, const double *rhs_field, double alpha0, double *c_state,
                        double *iterate_residual, double *equation_residual) {
  GUARD_BEGIN
  fld rf, cs;
  rf.nx = cs.nx = s->cfg.nx;
  rf.ny = cs.ny = s->cfg.ny;
  rf.g = cs.g = s->cfg.ghost;
  rf.d = (double *)rhs_field;
  cs.d = c_state;
  ch_linear_solve(s, &rf, alpha0, &cs, iterate_residual, equation_residual);
  GUARD_END
}

/* restart-load rebuild of the derived fields, io.cpp:412-436 */
int orc_refresh_derived(orc_solver *s) {
  GUARD_BEGIN
  bc_scalar(s, &s->f[ORC_F_C]);
  bc_scalar(s, &s->f[ORC_F_C_PREV]);
  bc_scalar(s, &s->f[ORC_F_C_PREV2]);
  bc_pressure(s, &s->f[ORC_F_P]);
  bc_pressure(s, &s->f[ORC_F_P_PREV]);
  bc_u(s, &s->f[ORC_F_U]);
  bc_v(s, &s->f[ORC_F_V]);
  bc_u(s, &s->f[ORC_F_U_PREV]);
  bc_v(s, &s->f[ORC_F_V_PREV]);
  update_materials(s);
  materials_from(s, &s->f[ORC_F_C_PREV], &s->f[ORC_F_RHO_PREV], &s->f[ORC_F_ETA_PREV]);
  update_midpoint(s);
  refresh_mu(s);
  GUARD_END
}

void orc_get_report(const orc_solver *s, orc_report *r) { *r = s->rep; }

double orc_compute_mass(orc_solver *s, int field_id) { return mass_of(s, &s->f[field_id]); }

/* compute_free_energy / populate_timestep_limits / compute_diagnostics, diagnostics.cpp:34-167 */
void orc_diagnostics(orc_solver *s, orc_diag *dg) {
  const fld *c = &s->f[ORC_F_C], *u = &s->f[ORC_F_U], *v = &s->f[ORC_F_V], *mu = &s->f[ORC_F_MU];
  const fld *rho = &s->f[ORC_F_RHO], *eta = &s->f[ORC_F_ETA];
  const int nx = s->cfg.nx, ny = s->cfg.ny;
  memset(dg, 0, sizeof(*dg));
  dg->mass = mass_of(s, c);
  dg->mass_drift = fabs(dg->mass - s->initial_mass);
  double div_sq = 0.0, div_max = 0.0, mu_max = 0.0, vel_max = 0.0, ke = 0.0;
  double rmin = INFINITY, rmax = 0.0, emin = INFINITY, emax = 0.0;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      const double dv = div_cell(s, u, v, i, j);
      const double uc = ccu(u, i, j), vc = ccv(v, i, j);
      div_sq += dv * dv;
      div_max = dmax(div_max, fabs(dv));
      mu_max = dmax(mu_max, fabs(AT(mu, i, j)));
      vel_max = dmax(vel_max, sqrt(uc * uc + vc * vc));
      ke += 0.5 * AT(rho, i, j) * (uc * uc + vc * vc) * s->dx * s->dy;
      rmin = dmin(rmin, AT(rho, i, j));
      rmax = dmax(rmax, AT(rho, i, j));
      emin = dmin(emin, AT(eta, i, j));
      emax = dmax(emax, AT(eta, i, j));
    }
  dg->divergence_l2 = sqrt(div_sq / (double)(nx * ny));
  dg->max_divergence = div_max;
  dg->max_abs_mu = mu_max;
  dg->max_velocity = vel_max;
  dg->kinetic_energy = ke;
  double energy = 0.0;
  const double alpha = 6.0 * sqrt(2.0);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      const double cc = AT(c, i, j);
      const double bulk = 0.25 * cc * cc * sq(1.0 - cc) / s->cfg.cn;
      const double grad_sq = sq(gcx(s, c, i, j)) + sq(gcy(s, c, i, j));
      energy += alpha * (bulk + 0.5 * s->cfg.cn * grad_sq) * s->dx * s->dy;
    }
  dg->total_free_energy = energy;
  dg->rho_min = rmin;
  dg->rho_max = rmax;
  dg->eta_min = emin;
  dg->eta_max = emax;
  const double h = dmin(s->dx, s->dy), tiny = 1.0e-30;
  double mar = 0.0;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      const double uc = ccu(u, i, j), vc = ccv(v, i, j);
      mar = dmax(mar, fabs(uc) / dmax(s->dx, tiny) + fabs(vc) / dmax(s->dy, tiny));
    }
  dg->dt_limit_advective = mar > tiny ? 0.5 / mar : INFINITY;
  dg->dt_limit_capillary = INFINITY;
  dg->dt_limit_ch_explicit = INFINITY;
  if (solve_ch(s)) {
    const double rs = dmax(dg->rho_max, tiny);
    dg->dt_limit_capillary = 0.5 * sqrt(dmax(s->cfg.re * s->cfg.ca * h * h * h / rs, 0.0));
    double mobility_max = 0.0, max_abs_wpp = 0.0;
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j) {
        const double cc = AT(c, i, j);
        mobility_max = dmax(mobility_max, dmax(0.0, cc * (1.0 - cc)));
        const double wpp = 0.5 - 3.0 * cc + 3.0 * cc * cc;
        max_abs_wpp = dmax(max_abs_wpp, fabs(wpp));
      }
    if (mobility_max > tiny) {
      const double coeff = alpha * mobility_max * max_abs_wpp / dmax(s->cfg.pe * s->cfg.cn, tiny);
      dg->dt_limit_ch_explicit = coeff > tiny ? 0.25 * h * h / coeff : INFINITY;
    }
  }
  dg->dt_limit_active = dg->dt_limit_advective;
  if (dg->dt_limit_capillary < dg->dt_limit_active) dg->dt_limit_active = dg->dt_limit_capillary;
  if (dg->dt_limit_ch_explicit < dg->dt_limit_active) dg->dt_limit_active = dg->dt_limit_ch_explicit;
  if (!isfinite(dg->dt_limit_active) || dg->dt_limit_active <= tiny)
    dg->dt_limit_ratio = 0.0;
  else
    dg->dt_limit_ratio = s->cfg.dt / dg->dt_limit_active;
}
