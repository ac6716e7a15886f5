/*
 * adrt_oracle.c -- TEST INFRASTRUCTURE (the oracle).  An FP64 CPU
 * restatement of the reference's adding-doubling column solver, written in
 * plain C for runtime N.  Each function cites the reference code it follows
 * (paths relative to the NewStrangeWorlds/AddingDoublingRT checkout).  Used
 * only by tests/, bench.py's CPU-baseline leg and __graft_entry__.smoke() as
 * the checker; the engine never calls it.
 *
 * Matrices are row-major N x N doubles, N <= 32.
 */
#include "adrt_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define OR_NMAX 32
#define OR_PI 3.14159265358979323846 /* src/constants.hpp:8 */

static _Thread_local char g_err[256];
static char g_err_shared[256];

const char* oracle_last_error(void) { return g_err_shared; }

static void set_err(const char* msg) {
  snprintf(g_err, sizeof g_err, "%s", msg);
  snprintf(g_err_shared, sizeof g_err_shared, "%s", msg);
}

/* ------------------------------------------------------------------ quadrature */

/* Gauss-Legendre nodes/weights on [0,1] by Newton iteration on P_n
 * (src/quadrature.cpp:11-51). */
void oracle_gauss_legendre(int n, double* nodes, double* weights) {
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double z = cos(OR_PI * (i + 0.75) / (n + 0.5));
    double pp = 0.0;
    for (int iter = 0; iter < 100; ++iter) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; ++k) {
        double pk = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = pk;
      }
      pp = n * (z * p1 - p0) / (z * z - 1.0);
      double dz = -p1 / pp;
      z += dz;
      if (fabs(dz) < 1e-15) break;
    }
    double w = 2.0 / ((1.0 - z * z) * pp * pp);
    nodes[i] = (1.0 - z) / 2.0;
    nodes[n - 1 - i] = (1.0 + z) / 2.0;
    weights[i] = w / 2.0;
    weights[n - 1 - i] = w / 2.0;
  }
}

/* P_l(x_i), l < L, by the three-term recurrence (src/quadrature.cpp:53-76).
 * Output Pl[l * nx + i]. */
static void legendre_table(int L, int nx, const double* x, double* Pl) {
  for (int i = 0; i < nx; ++i) Pl[i] = 1.0;
  if (L > 1)
    for (int i = 0; i < nx; ++i) Pl[nx + i] = x[i];
  for (int l = 2; l < L; ++l)
    for (int i = 0; i < nx; ++i)
      Pl[l * nx + i] =
          ((2 * l - 1) * x[i] * Pl[(l - 1) * nx + i] - (l - 1) * Pl[(l - 2) * nx + i]) / l;
}

/* ------------------------------------------------------------------ Planck */

/* Constants of src/planck.cpp:13-24. */
#define PL_C2 1.438786
#define PL_SIGMA 5.67032E-8
#define PL_VCUT 1.5
#define PL_A1 (1.0 / 3.0)
#define PL_A2 (-1.0 / 8.0)
#define PL_A3 (1.0 / 60.0)
#define PL_A4 (-1.0 / 5040.0)
#define PL_A5 (1.0 / 272160.0)
#define PL_A6 (-1.0 / 13305600.0)

static double planck_kernel(double v) { return v * v * v / (exp(v) - 1.0); }

/* Band-integrated Planck function: Simpson refinement for narrow bands,
 * small-v polynomial / large-v exponential series otherwise
 * (src/planck.cpp:35-131).  Returns -1 on invalid arguments (the reference
 * throws std::invalid_argument). */
double oracle_planck(double wnumlo, double wnumhi, double temp) {
  if (temp < 0.0 || wnumhi < wnumlo || wnumlo < 0.0) return -1.0;
  if (temp < 1.e-4) return 0.0;
  if (wnumhi == wnumlo) {
    double arg = exp(-PL_C2 * wnumhi / temp);
    return 1.1911e-8 * wnumhi * wnumhi * wnumhi * arg / (1.0 - arg);
  }
  const double vmax = log(DBL_MAX);
  const double sigdpi = PL_SIGMA / OR_PI;
  const double conc = 15.0 / pow(OR_PI, 4.0);
  double v[2] = {PL_C2 * wnumlo / temp, PL_C2 * wnumhi / temp};

  if (v[0] > DBL_EPSILON && v[1] < vmax && (wnumhi - wnumlo) / wnumhi < 1.e-2) {
    double hh = v[1] - v[0];
    double oldval = 0.0;
    double val0 = planck_kernel(v[0]) + planck_kernel(v[1]);
    for (int n = 1; n <= 10; ++n) {
      double del = hh / (2.0 * n);
      double val = val0;
      for (int k = 1; k <= 2 * n - 1; ++k) val += 2.0 * (1 + k % 2) * planck_kernel(v[0] + k * del);
      val *= del * PL_A1;
      if (fabs((val - oldval) / val) <= 1.e-6) return sigdpi * pow(temp, 4.0) * conc * val;
      oldval = val;
    }
    return sigdpi * pow(temp, 4.0) * conc * oldval;
  }

  double p[2] = {0.0, 0.0}, d[2] = {0.0, 0.0};
  int smallv = 0;
  static const double vcp[7] = {10.25, 5.7, 3.9, 2.9, 2.3, 1.9, 0.0};
  for (int i = 0; i < 2; ++i) {
    if (v[i] < PL_VCUT) {
      smallv++;
      double vsq = v[i] * v[i];
      p[i] = conc * vsq * v[i] *
             (PL_A1 + v[i] * (PL_A2 + v[i] * (PL_A3 + vsq * (PL_A4 + vsq * (PL_A5 + vsq * PL_A6)))));
    } else {
      int mmax = 1;
      while (v[i] < vcp[mmax - 1]) mmax++;
      double ex = exp(-v[i]);
      double exm = 1.0;
      d[i] = 0.0;
      for (int m = 1; m <= mmax; ++m) {
        double mv = m * v[i];
        exm *= ex;
        d[i] += exm * (6.0 + mv * (6.0 + mv * (3.0 + mv))) / (double)(m * m * m * m);
      }
      d[i] *= conc;
    }
  }
  double ans;
  if (smallv == 2)
    ans = p[1] - p[0];
  else if (smallv == 1)
    ans = 1.0 - p[0] - d[1];
  else
    ans = d[0] - d[1];
  ans *= sigdpi * pow(temp, 4.0);
  return (ans == 0.0) ? 0.0 : ans;
}

/* dB/dT of the band-integrated Planck function (src/planck.cpp:135-175). */
double oracle_planck_deriv(double wnumlo, double wnumhi, double temp) {
  if (temp < 0.0 || wnumhi < wnumlo || wnumlo < 0.0) return -1.0;
  if (temp < 1.e-4) return 0.0;
  if (wnumhi == wnumlo) {
    double x = PL_C2 * wnumhi / temp;
    double em = exp(-x);
    double b = 1.1911e-8 * wnumhi * wnumhi * wnumhi * em / (1.0 - em);
    return b * (x / temp) / (1.0 - em);
  }
  const double sigdpi = PL_SIGMA / OR_PI;
  const double conc = 15.0 / pow(OR_PI, 4.0);
  double v0 = PL_C2 * wnumlo / temp, v1 = PL_C2 * wnumhi / temp;
  double f0, f1;
  if (v0 < 1.e-6) f0 = v0 * v0; else { double em = exp(-v0); f0 = v0 * v0 * v0 * em / (1.0 - em); }
  if (v1 < 1.e-6) f1 = v1 * v1; else { double em = exp(-v1); f1 = v1 * v1 * v1 * em / (1.0 - em); }
  double B = oracle_planck(wnumlo, wnumhi, temp);
  double boundary = sigdpi * conc * temp * temp * temp * (v1 * f1 - v0 * f0);
  return 4.0 * B / temp - boundary;
}

/* ------------------------------------------------------------------ small dense algebra */

typedef struct {
  int n;
} dims_t;

static void mat_mul(int n, const double* A, const double* B, double* C) { /* C = A B */
  double tmp[OR_NMAX * OR_NMAX];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int k = 0; k < n; ++k) s += A[i * n + k] * B[k * n + j];
      tmp[i * n + j] = s;
    }
  memcpy(C, tmp, sizeof(double) * n * n);
}

static void mat_vec(int n, const double* A, const double* x, double* y) { /* y = A x */
  double tmp[OR_NMAX];
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int k = 0; k < n; ++k) s += A[i * n + k] * x[k];
    tmp[i] = s;
  }
  memcpy(y, tmp, sizeof(double) * n);
}

/* LU with partial pivoting (largest |entry| in the column), in place:
 * the factorisation Eigen::PartialPivLU performs for matrix.hpp:108-124. */
static void lu_factor(int n, double* A, int* perm) {
  for (int i = 0; i < n; ++i) perm[i] = i;
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = fabs(A[k * n + k]);
    for (int i = k + 1; i < n; ++i) {
      double v = fabs(A[i * n + k]);
      if (v > best) { best = v; p = i; }
    }
    if (p != k) {
      for (int j = 0; j < n; ++j) { double t = A[k * n + j]; A[k * n + j] = A[p * n + j]; A[p * n + j] = t; }
      int t = perm[k]; perm[k] = perm[p]; perm[p] = t;
    }
    double piv = A[k * n + k];
    if (piv != 0.0)
      for (int i = k + 1; i < n; ++i) A[i * n + k] /= piv;
    for (int i = k + 1; i < n; ++i) {
      double lik = A[i * n + k];
      if (lik == 0.0) continue;
      for (int j = k + 1; j < n; ++j) A[i * n + j] -= lik * A[k * n + j];
    }
  }
}

static void lu_solve_vec(int n, const double* LU, const int* perm, const double* b, double* x) {
  double y[OR_NMAX];
  for (int i = 0; i < n; ++i) y[i] = b[perm[i]];
  for (int i = 0; i < n; ++i) {
    double s = y[i];
    for (int k = 0; k < i; ++k) s -= LU[i * n + k] * y[k];
    y[i] = s;
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = y[i];
    for (int k = i + 1; k < n; ++k) s -= LU[i * n + k] * y[k];
    y[i] = s / LU[i * n + i];
  }
  memcpy(x, y, sizeof(double) * n);
}

/* x = A^{-1} b (matrix.hpp:106-108). */
static void solve_vec(int n, const double* A, const double* b, double* x) {
  double LU[OR_NMAX * OR_NMAX];
  int perm[OR_NMAX];
  memcpy(LU, A, sizeof(double) * n * n);
  lu_factor(n, LU, perm);
  lu_solve_vec(n, LU, perm, b, x);
}

/* X = B A^{-1}: LU of A^T, then A^T X^T = B^T (Matrix::rightSolveMatrix,
 * src/matrix.hpp:120-124). */
static void right_solve(int n, const double* A, const double* B, double* X) {
  double LU[OR_NMAX * OR_NMAX];
  int perm[OR_NMAX];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) LU[i * n + j] = A[j * n + i];
  lu_factor(n, LU, perm);
  double col[OR_NMAX], sol[OR_NMAX];
  for (int r = 0; r < n; ++r) { /* row r of X = column r of X^T */
    for (int k = 0; k < n; ++k) col[k] = B[r * n + k];
    lu_solve_vec(n, LU, perm, col, sol);
    for (int k = 0; k < n; ++k) X[r * n + k] = sol[k];
  }
}

/* ------------------------------------------------------------------ layers */

/* LayerMatrices<N> (src/layer.hpp:19-49); j_p/j_q are not needed here. */
typedef struct {
  double R_ab[OR_NMAX * OR_NMAX], R_ba[OR_NMAX * OR_NMAX];
  double T_ab[OR_NMAX * OR_NMAX], T_ba[OR_NMAX * OR_NMAX];
  double s_up[OR_NMAX], s_down[OR_NMAX], s_up_solar[OR_NMAX], s_down_solar[OR_NMAX];
  int is_scattering;
} layer_t;

static void layer_init(int n, layer_t* L) { /* default: R=0, T=I, s=0 (layer.hpp:42-46) */
  memset(L, 0, sizeof *L);
  for (int i = 0; i < n; ++i) L->T_ab[i * n + i] = L->T_ba[i * n + i] = 1.0;
}

/* Extra doublings from the single-scattering albedo (src/doubling.hpp:20-26). */
int oracle_ipow0(double omega) {
  if (omega < 0.01) return 4;
  if (omega < 0.1) return 10;
  return 16;
}

/* Number of doublings nn = max(1, trunc(ln tau / ln 2) + ipow0) (src/doubling.hpp:107-109). */
int oracle_num_doublings(double tau, double omega) {
  int nn = (int)(log(tau) / log(2.0)) + oracle_ipow0(omega);
  return nn < 1 ? 1 : nn;
}

/* One homogeneous layer: pure-absorption closed form, or first-order thin
 * layer initialisation followed by nn doublings of R, T and the thermal
 * (y, z) and solar sources (src/doubling.hpp:29-230). */
static void doubling(int n, double tau, double omega, double B_top, double B_bottom,
                     const double* Ppp, const double* Ppm, const double* mu, const double* wt,
                     double solar_flux, double solar_mu, double tau_cumulative,
                     const double* p_plus, const double* p_minus, layer_t* out) {
  layer_init(n, out);
  double B_bar = (B_bottom + B_top) / 2.0;
  double B_d = (tau > 0.0) ? (B_bottom - B_top) / tau : 0.0;
  if (tau <= 0.0) return;

  if (omega <= 0.0) { /* pure absorption, doubling.hpp:56-77 */
    memset(out->T_ab, 0, sizeof out->T_ab);
    memset(out->T_ba, 0, sizeof out->T_ba);
    for (int i = 0; i < n; ++i) {
      double tex = -tau / mu[i];
      double trans = (tex > -200.0) ? exp(tex) : 0.0;
      out->T_ab[i * n + i] = trans;
      out->T_ba[i * n + i] = trans;
      double omt = 1.0 - trans;
      double slope = mu[i] * omt - 0.5 * tau * (1.0 + trans);
      out->s_up[i] = B_bar * omt + B_d * slope;
      out->s_down[i] = B_bar * omt - B_d * slope;
    }
    return;
  }

  out->is_scattering = 1;
  if (omega > 1.0) omega = 1.0; /* std::clamp(omega, 0, 1), doubling.hpp:81 */
  const double con = 2.0 * omega * OR_PI;

  double Gpp[OR_NMAX * OR_NMAX], Gpm[OR_NMAX * OR_NMAX];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double pppc = Ppp[i * n + j] * wt[j];
      double temp = ((i == j) ? 1.0 : 0.0) + (-con) * pppc; /* I.add(PppC, -con) */
      Gpp[i * n + j] = temp / mu[i];
      Gpm[i * n + j] = con * (Ppm[i * n + j] * wt[j]) / mu[i];
    }

  int nn = oracle_num_doublings(tau, omega);
  double xfac = 1.0 / pow(2.0, nn);
  double tau0 = tau * xfac;

  int has_solar = (solar_flux > 0.0 && solar_mu > 0.0 && p_plus && p_minus);
  double F_top = has_solar ? solar_flux * exp(-tau_cumulative / solar_mu) : 0.0;

  double R[OR_NMAX * OR_NMAX], T[OR_NMAX * OR_NMAX];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      T[i * n + j] = ((i == j) ? 1.0 : 0.0) - tau0 * Gpp[i * n + j];
      R[i * n + j] = tau0 * Gpm[i * n + j];
    }
  double y[OR_NMAX], z[OR_NMAX], su[OR_NMAX], sd[OR_NMAX];
  for (int i = 0; i < n; ++i) {
    y[i] = (1.0 - omega) * tau0 / mu[i];
    z[i] = 0.0;
    su[i] = sd[i] = 0.0;
  }
  if (has_solar)
    for (int i = 0; i < n; ++i) {
      double base = omega * tau0 / mu[i] * F_top;
      su[i] = base * p_minus[i];
      sd[i] = base * p_plus[i];
    }
  double g = 0.5 * tau0;
  double gamma = has_solar ? exp(-tau0 / solar_mu) : 0.0;

  double R2[OR_NMAX * OR_NMAX], TG[OR_NMAX * OR_NMAX], TGR[OR_NMAX * OR_NMAX];
  double tmp[OR_NMAX * OR_NMAX];
  for (int k = 0; k < nn; ++k) { /* doubling.hpp:149-209 */
    mat_mul(n, R, R, R2);
    for (int i = 0; i < n * n; ++i) R2[i] = -R2[i];
    for (int i = 0; i < n; ++i) R2[i * n + i] += 1.0; /* I - R^2 */
    right_solve(n, R2, T, TG);                        /* TG = T (I - R^2)^{-1} */
    mat_mul(n, TG, R, TGR);
    double zpgy[OR_NMAX], a[OR_NMAX], b[OR_NMAX], c[OR_NMAX], d[OR_NMAX];
    for (int i = 0; i < n; ++i) zpgy[i] = z[i] + g * y[i];
    mat_vec(n, TG, zpgy, a);
    mat_vec(n, TGR, zpgy, b);
    mat_vec(n, TG, y, c);
    mat_vec(n, TGR, y, d);
    double nsu[OR_NMAX], nsd[OR_NMAX];
    if (has_solar) {
      double Rsd[OR_NMAX], Rsu[OR_NMAX], ru[OR_NMAX], rd[OR_NMAX];
      mat_vec(n, R, sd, Rsd);
      mat_vec(n, R, su, Rsu);
      for (int i = 0; i < n; ++i) {
        ru[i] = Rsd[i] + gamma * su[i];
        rd[i] = gamma * Rsu[i] + sd[i];
      }
      double tu[OR_NMAX], td[OR_NMAX];
      mat_vec(n, TG, ru, tu);
      mat_vec(n, TG, rd, td);
      for (int i = 0; i < n; ++i) {
        nsu[i] = tu[i] + su[i];
        nsd[i] = td[i] + gamma * sd[i];
      }
      gamma = gamma * gamma;
    } else {
      for (int i = 0; i < n; ++i) nsu[i] = nsd[i] = 0.0;
    }
    mat_mul(n, TGR, T, tmp);
    for (int i = 0; i < n * n; ++i) R[i] = R[i] + tmp[i]; /* R + TGR T */
    mat_mul(n, TG, T, T);                                 /* T = TG T */
    for (int i = 0; i < n; ++i) {
      double zn = (a[i] - b[i]) + z[i] - g * y[i];
      double yn = c[i] + d[i] + y[i];
      z[i] = zn;
      y[i] = yn;
      su[i] = nsu[i];
      sd[i] = nsd[i];
    }
    g = 2.0 * g;
  }
  memcpy(out->R_ab, R, sizeof(double) * n * n);
  memcpy(out->R_ba, R, sizeof(double) * n * n);
  memcpy(out->T_ab, T, sizeof(double) * n * n);
  memcpy(out->T_ba, T, sizeof(double) * n * n);
  for (int i = 0; i < n; ++i) {
    out->s_up[i] = y[i] * B_bar + z[i] * B_d;
    out->s_down[i] = y[i] * B_bar - z[i] * B_d;
    out->s_up_solar[i] = su[i];
    out->s_down_solar[i] = sd[i];
  }
}

/* Adding of two layers (src/adding.hpp:263-490): general case with two
 * coupling solves, or the non-scattering top / bottom shortcuts. */
static void add_layers(int n, const layer_t* top, const layer_t* bot, layer_t* ans) {
  layer_init(n, ans);
  if (!top->is_scattering) { /* addLayersNonscatTop, adding.hpp:349-406 */
    ans->is_scattering = bot->is_scattering;
    double t[OR_NMAX];
    for (int i = 0; i < n; ++i) t[i] = top->T_ab[i * n + i];
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        ans->R_ab[i * n + j] = t[i] * bot->R_ab[i * n + j] * t[j];
        ans->R_ba[i * n + j] = bot->R_ba[i * n + j];
        ans->T_ab[i * n + j] = bot->T_ab[i * n + j] * t[j];
        ans->T_ba[i * n + j] = t[i] * bot->T_ba[i * n + j];
      }
    for (int pass = 0; pass < 2; ++pass) {
      const double* s1u = pass ? top->s_up_solar : top->s_up;
      const double* s1d = pass ? top->s_down_solar : top->s_down;
      const double* s2u = pass ? bot->s_up_solar : bot->s_up;
      const double* s2d = pass ? bot->s_down_solar : bot->s_down;
      double* au = pass ? ans->s_up_solar : ans->s_up;
      double* ad = pass ? ans->s_down_solar : ans->s_down;
      double Rs[OR_NMAX], Ts[OR_NMAX];
      mat_vec(n, bot->R_ab, s1d, Rs);
      mat_vec(n, bot->T_ab, s1d, Ts);
      for (int i = 0; i < n; ++i) {
        au[i] = s1u[i] + t[i] * (s2u[i] + Rs[i]);
        ad[i] = s2d[i] + Ts[i];
      }
    }
    return;
  }
  if (!bot->is_scattering) { /* addLayersNonscatBot, adding.hpp:413-471 */
    ans->is_scattering = top->is_scattering;
    double t[OR_NMAX];
    for (int i = 0; i < n; ++i) t[i] = bot->T_ab[i * n + i];
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        ans->R_ab[i * n + j] = top->R_ab[i * n + j];
        ans->R_ba[i * n + j] = t[i] * top->R_ba[i * n + j] * t[j];
        ans->T_ab[i * n + j] = t[i] * top->T_ab[i * n + j];
        ans->T_ba[i * n + j] = top->T_ba[i * n + j] * t[j];
      }
    for (int pass = 0; pass < 2; ++pass) {
      const double* s1u = pass ? top->s_up_solar : top->s_up;
      const double* s1d = pass ? top->s_down_solar : top->s_down;
      const double* s2u = pass ? bot->s_up_solar : bot->s_up;
      const double* s2d = pass ? bot->s_down_solar : bot->s_down;
      double* au = pass ? ans->s_up_solar : ans->s_up;
      double* ad = pass ? ans->s_down_solar : ans->s_down;
      double Ts[OR_NMAX], Rs[OR_NMAX];
      mat_vec(n, top->T_ba, s2u, Ts);
      mat_vec(n, top->R_ba, s2u, Rs);
      for (int i = 0; i < n; ++i) {
        au[i] = s1u[i] + Ts[i];
        ad[i] = s2d[i] + t[i] * (s1d[i] + Rs[i]);
      }
    }
    return;
  }
  /* addLayersGeneral, adding.hpp:301-342 */
  ans->is_scattering = 1;
  double A1[OR_NMAX * OR_NMAX], A2[OR_NMAX * OR_NMAX];
  double D1[OR_NMAX * OR_NMAX], D2[OR_NMAX * OR_NMAX], tmp[OR_NMAX * OR_NMAX];
  mat_mul(n, bot->R_ab, top->R_ba, A1);
  mat_mul(n, top->R_ba, bot->R_ab, A2);
  for (int i = 0; i < n * n; ++i) { A1[i] = -A1[i]; A2[i] = -A2[i]; }
  for (int i = 0; i < n; ++i) { A1[i * n + i] += 1.0; A2[i * n + i] += 1.0; }
  right_solve(n, A1, top->T_ba, D1); /* T_ba_D1 = top.T_ba A1^{-1} */
  right_solve(n, A2, bot->T_ab, D2); /* T_bc_D2 = bot.T_ab A2^{-1} */
  mat_mul(n, D1, bot->R_ab, tmp);
  mat_mul(n, tmp, top->T_ab, tmp);
  for (int i = 0; i < n * n; ++i) ans->R_ab[i] = top->R_ab[i] + tmp[i];
  mat_mul(n, D2, top->R_ba, tmp);
  mat_mul(n, tmp, bot->T_ba, tmp);
  for (int i = 0; i < n * n; ++i) ans->R_ba[i] = bot->R_ba[i] + tmp[i];
  mat_mul(n, D2, top->T_ab, ans->T_ab);
  mat_mul(n, D1, bot->T_ba, ans->T_ba);
  for (int pass = 0; pass < 2; ++pass) { /* addSources, adding.hpp:263-294 */
    const double* s1u = pass ? top->s_up_solar : top->s_up;
    const double* s1d = pass ? top->s_down_solar : top->s_down;
    const double* s2u = pass ? bot->s_up_solar : bot->s_up;
    const double* s2d = pass ? bot->s_down_solar : bot->s_down;
    double* au = pass ? ans->s_up_solar : ans->s_up;
    double* ad = pass ? ans->s_down_solar : ans->s_down;
    double v[OR_NMAX], rhs[OR_NMAX], r[OR_NMAX];
    mat_vec(n, bot->R_ab, s1d, v);
    for (int i = 0; i < n; ++i) rhs[i] = s2u[i] + v[i];
    mat_vec(n, D1, rhs, r);
    for (int i = 0; i < n; ++i) au[i] = s1u[i] + r[i];
    mat_vec(n, top->R_ba, s2u, v);
    for (int i = 0; i < n; ++i) rhs[i] = s1d[i] + v[i];
    mat_vec(n, D2, rhs, r);
    for (int i = 0; i < n; ++i) ad[i] = s2d[i] + r[i];
  }
}

/* ------------------------------------------------------------------ phase */

/* m=0 phase matrices with Hansen column renormalisation
 * (src/phase_matrix.hpp:61-111); Pl is [L][N]. */
static void phase_matrices(int n, int L, const double* chi, const double* Pl, const double* wt,
                           double* Ppp, double* Ppm) {
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double spp = 0.0, spm = 0.0, sign = 1.0;
      for (int l = 0; l < L; ++l) {
        double term = (2 * l + 1) * chi[l] * Pl[l * n + i] * Pl[l * n + j];
        spp += term;
        spm += sign * term;
        sign = -sign;
      }
      Ppp[i * n + j] = spp / (2.0 * OR_PI);
      Ppm[i * n + j] = spm / (2.0 * OR_PI);
    }
  for (int j = 0; j < n; ++j) {
    double sum = 0.0;
    for (int i = 0; i < n; ++i) sum += (Ppp[i * n + j] + Ppm[i * n + j]) * wt[i];
    if (sum > 0.0) {
      double corr = 1.0 / (2.0 * OR_PI * sum);
      for (int i = 0; i < n; ++i) { Ppp[i * n + j] *= corr; Ppm[i * n + j] *= corr; }
    }
  }
}

/* Solar phase vectors p+/p- at mu0 (src/phase_matrix.hpp:131-181). */
static void solar_vectors(int n, int L, const double* chi, const double* Pl, const double* wt,
                          double mu0, double* pp, double* pm) {
  double Plm[256];
  Plm[0] = 1.0;
  if (L > 1) Plm[1] = mu0;
  for (int l = 2; l < L; ++l) Plm[l] = ((2 * l - 1) * mu0 * Plm[l - 1] - (l - 1) * Plm[l - 2]) / l;
  for (int i = 0; i < n; ++i) {
    double sp = 0.0, sm = 0.0, sign = 1.0;
    for (int l = 0; l < L; ++l) {
      double term = (2 * l + 1) * chi[l] * Pl[l * n + i] * Plm[l];
      sp += term;
      sm += sign * term;
      sign = -sign;
    }
    pp[i] = sp / (2.0 * OR_PI);
    pm[i] = sm / (2.0 * OR_PI);
  }
  double sum = 0.0;
  for (int i = 0; i < n; ++i) sum += (pp[i] + pm[i]) * wt[i];
  if (sum > 0.0) {
    double corr = 1.0 / (2.0 * OR_PI * sum);
    for (int i = 0; i < n; ++i) { pp[i] *= corr; pm[i] *= corr; }
  }
}

/* ------------------------------------------------------------------ column */

typedef struct {
  int nlay, n, nmom;
  int thermal, delta_m, diffusion, from_bottom;
  double albedo, surf_emission, surf_temp, top_emission, top_temp;
  double F0, mu0, wlo, whi;
  double *dtau, *ssa, *chi; /* chi [nlay][nmom] */
  double *temp, *planck;    /* [nlay+1] or NULL */
} column_t;

/* ADConfig::validate (src/adding_doubling.hpp:123-174). */
static int validate(const column_t* c) {
  if (c->nlay <= 0) { set_err("ADConfig: num_layers must be > 0"); return -1; }
  if (c->n < 2) { set_err("ADConfig: num_quadrature must be >= 2"); return -1; }
  for (int l = 0; l < c->nlay; ++l) {
    if (c->dtau[l] < 0.0) { set_err("ADConfig: delta_tau < 0"); return -1; }
    if (c->ssa[l] < 0.0 || c->ssa[l] > 1.0) { set_err("ADConfig: single_scat_albedo out of [0,1]"); return -1; }
  }
  if (c->albedo < 0.0 || c->albedo > 1.0) { set_err("ADConfig: surface_albedo out of [0,1]"); return -1; }
  if (c->F0 > 0.0 && (c->mu0 <= 0.0 || c->mu0 > 1.0)) { set_err("ADConfig: solar_mu must be in (0,1] when solar_flux > 0"); return -1; }
  if (c->thermal) {
    if (!c->temp) { set_err("ADConfig: temperature size must be num_layers+1"); return -1; }
    for (int l = 0; l <= c->nlay; ++l)
      if (c->temp[l] < 0.0) { set_err("ADConfig: temperature < 0"); return -1; }
    if (c->wlo < 0.0 || c->whi < c->wlo) { set_err("ADConfig: invalid wavenumber range"); return -1; }
  } else if (c->surf_temp >= 0.0) {
    set_err("ADConfig: surface_temperature requires use_thermal_emission"); return -1;
  } else if (c->top_temp >= 0.0) {
    set_err("ADConfig: top_temperature requires use_thermal_emission"); return -1;
  }
  if (c->diffusion && !c->thermal && !c->planck) {
    set_err("ADConfig: use_diffusion_lower_bc requires use_thermal_emission or planck_levels");
    return -1;
  }
  return 0;
}

typedef struct {
  double *fu, *fd, *fdir, *J, *divF; /* [nlay+1] each */
} colout_t;

/* The column solver, solveImpl<N> (src/solver.cpp:348-722), for runtime N. */
static int solve_column(column_t* c, colout_t* o) {
  if (validate(c)) return -1;
  const int n = c->n, nlay = c->nlay;
  if (n > OR_NMAX) { set_err("oracle: num_quadrature > 32"); return -1; }
  if (c->from_bottom) { /* solver.cpp:362-372 */
    for (int a = 0, b = nlay - 1; a < b; ++a, --b) {
      double t = c->dtau[a]; c->dtau[a] = c->dtau[b]; c->dtau[b] = t;
      t = c->ssa[a]; c->ssa[a] = c->ssa[b]; c->ssa[b] = t;
      for (int m = 0; m < c->nmom; ++m) {
        t = c->chi[a * c->nmom + m]; c->chi[a * c->nmom + m] = c->chi[b * c->nmom + m]; c->chi[b * c->nmom + m] = t;
      }
    }
    for (int a = 0, b = nlay; a < b; ++a, --b) {
      double t;
      if (c->thermal) { t = c->temp[a]; c->temp[a] = c->temp[b]; c->temp[b] = t; }
      if (c->planck) { t = c->planck[a]; c->planck[a] = c->planck[b]; c->planck[b] = t; }
    }
  }
  double mu[OR_NMAX], wt[OR_NMAX];
  oracle_gauss_legendre(n, mu, wt);
  double xs = 0.0;
  for (int i = 0; i < n; ++i) xs += mu[i] * wt[i];
  const double xfac = 0.5 / xs;

  /* Planck levels (solver.cpp:385-420) */
  double* B = calloc(nlay + 1, sizeof(double));
  double B_surface = 0.0, B_top = 0.0;
  if (c->thermal) {
    for (int l = 0; l <= nlay; ++l) B[l] = oracle_planck(c->wlo, c->whi, c->temp[l]);
    B_surface = (c->surf_temp >= 0.0) ? oracle_planck(c->wlo, c->whi, c->surf_temp) : B[nlay];
    B_top = (c->top_temp >= 0.0) ? oracle_planck(c->wlo, c->whi, c->top_temp) : B[0];
  } else if (c->planck) {
    for (int l = 0; l <= nlay; ++l) B[l] = c->planck[l];
    B_surface = c->surf_emission;
    B_top = c->top_emission;
  } else {
    B_surface = c->surf_emission;
    B_top = c->top_emission;
  }

  const int has_solar = (c->F0 > 0.0 && c->mu0 > 0.0);
  const int two_M = 2 * n;
  layer_t* lay = malloc(sizeof(layer_t) * (nlay + 1));
  double* tau_used = calloc(nlay, sizeof(double));
  double* Pl = malloc(sizeof(double) * (size_t)(c->nmom > two_M ? c->nmom : two_M) * n);
  double chi_star[256];
  double tau_cum = 0.0;

  for (int l = 0; l < nlay; ++l) { /* layer loop, solver.cpp:430-514 */
    double tau_l = c->dtau[l], om_l = c->ssa[l];
    double Ppp[OR_NMAX * OR_NMAX] = {0}, Ppm[OR_NMAX * OR_NMAX] = {0};
    double pp[OR_NMAX] = {0}, pm[OR_NMAX] = {0};
    int has_sp = 0;
    if (om_l > 0.0 && tau_l > 0.0) {
      const double* full = c->chi + (size_t)l * c->nmom;
      const double* use = full;
      int nuse = c->nmom;
      if (c->delta_m) {
        double f = (c->nmom > two_M) ? full[two_M] : 0.0;
        if (f > 1e-12 && f < 1.0 - 1e-12) { /* delta-M, solver.cpp:445-468 */
          double of = om_l * f;
          tau_l = (1.0 - of) * c->dtau[l];
          om_l = om_l * (1.0 - f) / (1.0 - of);
          double inv = 1.0 / (1.0 - f);
          for (int m = 0; m < two_M; ++m) chi_star[m] = (full[m] - f) * inv;
          use = chi_star;
          nuse = two_M;
        } else {
          nuse = c->nmom < two_M ? c->nmom : two_M;
        }
      }
      legendre_table(nuse, n, mu, Pl);
      phase_matrices(n, nuse, use, Pl, wt, Ppp, Ppm);
      if (has_solar) {
        solar_vectors(n, nuse, use, Pl, wt, c->mu0, pp, pm);
        has_sp = 1;
      }
    }
    tau_used[l] = tau_l;
    doubling(n, tau_l, om_l, B[l], B[l + 1], Ppp, Ppm, mu, wt, c->F0, c->mu0, tau_cum,
             has_sp ? pp : NULL, has_sp ? pm : NULL, &lay[l]);
    tau_cum += tau_l;
  }

  int ltot = nlay;
  const int has_surface = !c->diffusion && (c->albedo > 0.0 || B_surface > 0.0);
  if (has_surface) { /* Lambertian surface pseudo-layer, solver.cpp:516-551 */
    layer_t* s = &lay[nlay];
    layer_init(n, s);
    memset(s->T_ab, 0, sizeof s->T_ab);
    memset(s->T_ba, 0, sizeof s->T_ba);
    double A = c->albedo;
    for (int i = 0; i < n; ++i) {
      for (int j = 0; j < n; ++j) {
        double r = 2.0 * A * mu[j] * wt[j] * xfac;
        s->R_ab[i * n + j] = r;
        s->R_ba[i * n + j] = r;
      }
      s->s_up[i] = (1.0 - A) * B_surface;
      s->s_down[i] = 0.0;
      if (has_solar && A > 0.0) s->s_up_solar[i] = (A / OR_PI) * c->F0 * c->mu0 * exp(-tau_cum / c->mu0);
    }
    s->is_scattering = (A > 0.0);
    ltot++;
  }

  /* rbase (bottom-up) and rtop (top-down) composites, solver.cpp:553-583 */
  layer_t* rbase = malloc(sizeof(layer_t) * (ltot + 1));
  layer_t* rtop = malloc(sizeof(layer_t) * (ltot + 1));
  rbase[1] = lay[ltot - 1];
  for (int l = 1; l < ltot; ++l) add_layers(n, &lay[ltot - 1 - l], &rbase[l], &rbase[l + 1]);
  rtop[1] = lay[0];
  for (int l = 1; l < ltot; ++l) add_layers(n, &rtop[l], &lay[l], &rtop[l + 1]);

  /* boundary intensities, solver.cpp:585-603 */
  double Itop[OR_NMAX], Ibot[OR_NMAX];
  for (int i = 0; i < n; ++i) { Itop[i] = B_top; Ibot[i] = 0.0; }
  if (c->diffusion) {
    double dt = tau_used[nlay - 1];
    double dB = (dt > 0.0) ? (B[nlay] - B[nlay - 1]) / dt : 0.0;
    for (int i = 0; i < n; ++i) Ibot[i] = B[nlay] + mu[i] * dB;
  } else if (!has_surface) {
    for (int i = 0; i < n; ++i) Ibot[i] = B_surface;
  }

  const int nint = nlay + 1;
  for (int l = 0; l < nint; ++l) o->fu[l] = o->fd[l] = o->J[l] = o->divF[l] = o->fdir[l] = 0.0;
  if (has_solar) { /* direct beam with the (delta-M scaled) tau, solver.cpp:615-626 */
    double tc = 0.0;
    o->fdir[0] = c->F0 * c->mu0;
    for (int l = 0; l < nlay; ++l) {
      tc += tau_used[l];
      o->fdir[l + 1] = c->F0 * c->mu0 * exp(-tc / c->mu0);
    }
  }
  { /* TOA, solver.cpp:628-641 */
    layer_t* f = &rbase[ltot];
    double a[OR_NMAX], b[OR_NMAX], Iup[OR_NMAX];
    mat_vec(n, f->R_ab, Itop, a);
    mat_vec(n, f->T_ba, Ibot, b);
    for (int i = 0; i < n; ++i) Iup[i] = a[i] + (b[i] + f->s_up[i] + f->s_up_solar[i]);
    for (int i = 0; i < n; ++i) {
      o->fu[0] += 2.0 * OR_PI * wt[i] * mu[i] * Iup[i];
      o->fd[0] += 2.0 * OR_PI * wt[i] * mu[i] * Itop[i];
      o->J[0] += 0.5 * wt[i] * (Iup[i] + Itop[i]);
    }
  }
  for (int l = 1; l <= nlay; ++l) { /* interfaces, solver.cpp:644-678 and :24-73 */
    int n_top = l, n_base = ltot - l;
    double Iup[OR_NMAX], Idn[OR_NMAX];
    if (n_base > 0 && n_top > 0) {
      const layer_t* tp = &rtop[n_top];
      const layer_t* bs = &rbase[n_base];
      double M[OR_NMAX * OR_NMAX], t1[OR_NMAX], t2[OR_NMAX], t3[OR_NMAX], v[OR_NMAX], rhs[OR_NMAX];
      /* computeIup */
      mat_mul(n, bs->R_ab, tp->R_ba, M);
      for (int i = 0; i < n * n; ++i) M[i] = -M[i];
      for (int i = 0; i < n; ++i) M[i * n + i] += 1.0;
      mat_vec(n, bs->T_ba, Ibot, t1);
      mat_vec(n, tp->T_ab, Itop, v);
      mat_vec(n, bs->R_ab, v, t2);
      for (int i = 0; i < n; ++i) v[i] = tp->s_down[i] + tp->s_down_solar[i];
      mat_vec(n, bs->R_ab, v, t3);
      for (int i = 0; i < n; ++i) rhs[i] = t1[i] + t2[i] + t3[i] + bs->s_up[i] + bs->s_up_solar[i];
      solve_vec(n, M, rhs, Iup);
      /* computeIdown */
      mat_mul(n, tp->R_ba, bs->R_ab, M);
      for (int i = 0; i < n * n; ++i) M[i] = -M[i];
      for (int i = 0; i < n; ++i) M[i * n + i] += 1.0;
      mat_vec(n, tp->T_ab, Itop, t1);
      mat_vec(n, bs->T_ba, Ibot, v);
      mat_vec(n, tp->R_ba, v, t2);
      for (int i = 0; i < n; ++i) v[i] = bs->s_up[i] + bs->s_up_solar[i];
      mat_vec(n, tp->R_ba, v, t3);
      for (int i = 0; i < n; ++i) rhs[i] = t1[i] + t2[i] + t3[i] + tp->s_down[i] + tp->s_down_solar[i];
      solve_vec(n, M, rhs, Idn);
    } else if (n_base == 0) {
      const layer_t* tp = &rtop[n_top];
      double a[OR_NMAX], b[OR_NMAX];
      mat_vec(n, tp->T_ab, Itop, a);
      mat_vec(n, tp->R_ba, Ibot, b);
      for (int i = 0; i < n; ++i) {
        Idn[i] = a[i] + (b[i] + tp->s_down[i] + tp->s_down_solar[i]);
        Iup[i] = Ibot[i];
      }
    } else {
      for (int i = 0; i < n; ++i) { Iup[i] = 0.0; Idn[i] = Itop[i]; }
    }
    for (int i = 0; i < n; ++i) {
      o->fu[l] += 2.0 * OR_PI * wt[i] * mu[i] * Iup[i];
      o->fd[l] += 2.0 * OR_PI * wt[i] * mu[i] * Idn[i];
      o->J[l] += 0.5 * wt[i] * (Iup[i] + Idn[i]);
    }
  }
  if (has_solar) { /* beam term of J, solver.cpp:684-689 */
    double inv = 1.0 / (4.0 * OR_PI * c->mu0);
    for (int l = 0; l < nint; ++l) o->J[l] += o->fdir[l] * inv;
  }
  for (int l = 0; l < nint; ++l) { /* divF with the unscaled omega, solver.cpp:695-700 */
    int lyr = (l == 0) ? 0 : l - 1;
    o->divF[l] = 4.0 * OR_PI * (1.0 - c->ssa[lyr]) * (o->J[l] - B[l]);
  }
  if (c->from_bottom) { /* solver.cpp:711-719 */
    double* arr[5] = {o->fu, o->fd, o->J, o->divF, o->fdir};
    for (int k = 0; k < 5; ++k)
      for (int a = 0, b = nlay; a < b; ++a, --b) { double t = arr[k][a]; arr[k][a] = arr[k][b]; arr[k][b] = t; }
  }
  free(B); free(lay); free(tau_used); free(Pl); free(rbase); free(rtop);
  return 0;
}

/* ------------------------------------------------------------------ batch driver */

static int gather_column(const adrt_batch_desc* d, const adrt_inputs* in, int w, column_t* c) {
  const int L = d->num_layers, M = d->num_moments;
  memset(c, 0, sizeof *c);
  c->nlay = L; c->n = d->num_quadrature; c->nmom = M;
  c->thermal = d->use_thermal_emission; c->delta_m = d->use_delta_m;
  c->diffusion = d->use_diffusion_lower_bc; c->from_bottom = d->index_from_bottom;
  c->albedo = in->surface_albedo ? in->surface_albedo[w] : d->surface_albedo;
  c->surf_emission = in->surface_emission ? in->surface_emission[w] : d->surface_emission;
  c->surf_temp = d->surface_temperature;
  c->top_emission = in->top_emission ? in->top_emission[w] : d->top_emission;
  c->top_temp = d->top_temperature;
  c->F0 = d->solar_flux;
  c->mu0 = in->solar_mu ? in->solar_mu[w] : d->solar_mu;
  c->wlo = in->wavenumber_low ? in->wavenumber_low[w] : d->wavenumber_low;
  c->whi = in->wavenumber_high ? in->wavenumber_high[w] : d->wavenumber_high;
  c->dtau = malloc(sizeof(double) * L);
  c->ssa = malloc(sizeof(double) * L);
  c->chi = malloc(sizeof(double) * (size_t)L * M);
  memcpy(c->dtau, in->delta_tau + (size_t)w * L, sizeof(double) * L);
  memcpy(c->ssa, in->single_scat_albedo + (size_t)w * L, sizeof(double) * L);
  for (int l = 0; l < L; ++l) {
    const double* src;
    if (d->moment_layout == ADRT_MOMENTS_SHARED) src = in->phase_moments + (size_t)l * M;
    else if (d->moment_layout == ADRT_MOMENTS_PER_WAVENUMBER) src = in->phase_moments + (size_t)w * M;
    else src = in->phase_moments + ((size_t)w * L + l) * M;
    memcpy(c->chi + (size_t)l * M, src, sizeof(double) * M);
  }
  if (c->thermal && in->temperature) {
    c->temp = malloc(sizeof(double) * (L + 1));
    memcpy(c->temp, in->temperature + (d->temperature_per_wavenumber ? (size_t)w * (L + 1) : 0),
           sizeof(double) * (L + 1));
  }
  if (in->planck_levels) {
    c->planck = malloc(sizeof(double) * (L + 1));
    memcpy(c->planck, in->planck_levels + (size_t)w * (L + 1), sizeof(double) * (L + 1));
  }
  return 0;
}

static void free_column(column_t* c) {
  free(c->dtau); free(c->ssa); free(c->chi); free(c->temp); free(c->planck);
}

static int solve_one(const adrt_batch_desc* d, const adrt_inputs* in, const adrt_outputs* out, int w) {
  column_t c;
  gather_column(d, in, w, &c);
  const int nint = d->num_layers + 1;
  double* buf = malloc(sizeof(double) * 5 * nint);
  colout_t o = {buf, buf + nint, buf + 2 * nint, buf + 3 * nint, buf + 4 * nint};
  int rc = solve_column(&c, &o);
  if (rc == 0) {
    size_t off = (size_t)w * nint;
    if (out->flux_up) memcpy(out->flux_up + off, o.fu, sizeof(double) * nint);
    if (out->flux_down) memcpy(out->flux_down + off, o.fd, sizeof(double) * nint);
    if (out->flux_direct) memcpy(out->flux_direct + off, o.fdir, sizeof(double) * nint);
    if (out->mean_intensity) memcpy(out->mean_intensity + off, o.J, sizeof(double) * nint);
    if (out->flux_divergence) memcpy(out->flux_divergence + off, o.divF, sizeof(double) * nint);
    /* outputs are in the caller's level order: TOA is the last level when
       the arrays are indexed from the bottom */
    const int toa = d->index_from_bottom ? nint - 1 : 0, boa = d->index_from_bottom ? 0 : nint - 1;
    if (out->toa_flux_up) out->toa_flux_up[w] = o.fu[toa] * d->spectrum_scaling;
    if (out->toa_flux_down) out->toa_flux_down[w] = o.fd[toa];
    if (out->boa_flux_direct) out->boa_flux_direct[w] = o.fdir[boa];
  }
  free(buf);
  free_column(&c);
  return rc;
}

typedef struct {
  const adrt_batch_desc* d;
  const adrt_inputs* in;
  const adrt_outputs* out;
  atomic_int next;
  atomic_int failed;
  int w1;
} pool_t;

static void* worker(void* arg) {
  pool_t* p = arg;
  for (;;) {
    int w = atomic_fetch_add(&p->next, 1);
    if (w >= p->w1 || atomic_load(&p->failed)) break;
    if (solve_one(p->d, p->in, p->out, w)) atomic_store(&p->failed, 1);
  }
  return NULL;
}

int oracle_solve_batch_range(const adrt_batch_desc* desc, const adrt_inputs* in,
                             const adrt_outputs* out, int w0, int w1, int nthreads) {
  if (!desc || !in || !out) { set_err("null argument"); return -1; }
  if (desc->num_quadrature > OR_NMAX || desc->num_quadrature < 2) {
    set_err("ADConfig: num_quadrature must be in 2..32"); return -1;
  }
  if (desc->num_moments > 256) { set_err("oracle: num_moments > 256"); return -1; }
  pool_t p;
  p.d = desc; p.in = in; p.out = out; p.w1 = w1;
  atomic_init(&p.next, w0);
  atomic_init(&p.failed, 0);
  if (nthreads < 1) nthreads = 1;
  pthread_t th[256];
  int nt = nthreads > 256 ? 256 : nthreads;
  for (int t = 1; t < nt; ++t) pthread_create(&th[t], NULL, worker, &p);
  worker(&p);
  for (int t = 1; t < nt; ++t) pthread_join(th[t], NULL);
  return atomic_load(&p.failed) ? -1 : 0;
}

int oracle_solve_batch(const adrt_batch_desc* desc, const adrt_inputs* in,
                       const adrt_outputs* out, int nthreads) {
  return oracle_solve_batch_range(desc, in, out, 0, desc ? desc->num_wavenumbers : 0, nthreads);
}

/* ------------------------------------------------------------------ flop model */

/* Algorithmic flops of one wavenumber-solve, counting only the branch the
 * reference takes (conventions: GEMM 2N^3, LU 2N^3/3, triangular solve 2N^2
 * per right-hand side, mat-vec 2N^2):
 *   doubling: nn * (32/3 N^3 + (solar ? 16 : 8) N^2) + 6N^2 per scattering layer, 6N otherwise
 *             (src/doubling.hpp:56-209)
 *   adding:   (64/3 N^3 + 16 N^2) general, 14 N^2 shortcut, per add, two sweeps
 *             (src/adding.hpp:301-471)
 *   interfaces: (L-1)(16/3 N^3 + 24 N^2) + 2N^2  (src/solver.cpp:24-73, 628-678)
 *   phase build: L (4 N^2 M + 4 N^2) when moments vary per wavenumber
 *             (src/phase_matrix.hpp:73-110). */
double oracle_flops_batch(const adrt_batch_desc* d, const adrt_inputs* in, int w0, int w1) {
  const double N = d->num_quadrature;
  const int L = d->num_layers, M = d->num_moments, two_M = 2 * d->num_quadrature;
  const int solar = d->solar_flux > 0.0;
  double total = 0.0;
  int* scat = malloc(sizeof(int) * (L + 1));
  for (int w = w0; w < w1; ++w) {
    double F = 0.0;
    for (int l = 0; l < L; ++l) {
      double tau = in->delta_tau[(size_t)w * L + l];
      double om = in->single_scat_albedo[(size_t)w * L + l];
      int s = (om > 0.0 && tau > 0.0);
      if (s && d->use_delta_m && M > two_M) {
        const double* chi;
        if (d->moment_layout == ADRT_MOMENTS_SHARED) chi = in->phase_moments + (size_t)l * M;
        else if (d->moment_layout == ADRT_MOMENTS_PER_WAVENUMBER) chi = in->phase_moments + (size_t)w * M;
        else chi = in->phase_moments + ((size_t)w * L + l) * M;
        double f = chi[two_M];
        if (f > 1e-12 && f < 1.0 - 1e-12) {
          double of = om * f;
          tau = (1.0 - of) * tau;
          om = om * (1.0 - f) / (1.0 - of);
        }
      }
      scat[l] = s;
      if (s) F += oracle_num_doublings(tau, om) * (32.0 / 3.0 * N * N * N + (solar ? 16.0 : 8.0) * N * N) + 6.0 * N * N;
      else F += 6.0 * N;
    }
    double A = in->surface_albedo ? in->surface_albedo[w] : d->surface_albedo;
    int has_surface = !d->use_diffusion_lower_bc && (A > 0.0 || d->use_thermal_emission ||
                                                     d->surface_emission > 0.0);
    int ltot = L;
    if (has_surface) { scat[L] = A > 0.0; ltot++; }
    /* bottom-up sweep: composite scattering flag accumulates */
    int comp = scat[ltot - 1];
    for (int l = 1; l < ltot; ++l) {
      int top = scat[ltot - 1 - l];
      F += (top && comp) ? (64.0 / 3.0 * N * N * N + 16.0 * N * N) : 14.0 * N * N;
      comp = comp || top;
    }
    comp = scat[0];
    for (int l = 1; l < ltot; ++l) {
      int bot = scat[l];
      F += (comp && bot) ? (64.0 / 3.0 * N * N * N + 16.0 * N * N) : 14.0 * N * N;
      comp = comp || bot;
    }
    F += (L - 1) * (16.0 / 3.0 * N * N * N + 24.0 * N * N) + 2.0 * N * N;
    if (d->moment_layout != ADRT_MOMENTS_SHARED) F += L * (4.0 * N * N * M + 4.0 * N * N);
    total += F;
  }
  free(scat);
  return total;
}
