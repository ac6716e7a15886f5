// adrt_tpw.cuh -- the thread-per-wavenumber mapping: one thread solves one
// wavenumber end to end, its matrices in per-thread (local) memory.
//
// This is the mapping of the reference's GPU kernel solveKernel<N>
// (src_cuda/cuda_solver.cu:131-493: one thread per wavenumber, 128-thread
// blocks, every matrix a per-thread array), applied to this engine's scheme
// and outputs: FP64, the first-order thin-layer start and reference-order
// doubling (src/doubling.hpp:29-230), adding (src/adding.hpp:263-490), the
// downward interface pass and per-interface fluxes, exactly the steps of
// wav_body (adrt_kernel.cuh) written for one thread.  The right-solves are
// the Gauss-Jordan column elimination with the reference's pivot rule
// (largest |entry| of the pivot row, the LU of A^T of src/matrix.hpp:120-124).
//
// It serves as the fixed mapping the autotuned uneven launch is measured
// against and as one of the mappings the autotuner chooses from (at small N
// a thread owns a whole matrix in few registers).  Per-interface records of
// the downward pass live in each thread's HBM slot, interleaved over the
// threads of the launch (element e of slot s at e * nslots + s).
#pragma once

#include "adrt_kernel.cuh"

namespace adrt_dev {
namespace tpw {

// Per-thread record of interface l: R, T, R_base (NP x NP row-major), s_dn,
// U_base (NP), the layer's scattering flag and the composite's reflects flag.
template <int NP>
struct Rec {
  static constexpr int R = 0, T = NP * NP, RB = 2 * NP * NP, SDN = 3 * NP * NP;
  static constexpr int UB = SDN + NP, SCAT = UB + NP, CS = SCAT + 1, SIZE = CS + 1;
};
constexpr int kLev = 5;  // level arrays: B, tau_cum, tau', omega', omega (unscaled)

template <int NP>
__host__ __device__ inline size_t slot_doubles(int lmax) {
  return (size_t)kLev * (lmax + 1) + (size_t)(lmax + 1) * Rec<NP>::SIZE;
}

// Interleaved per-thread HBM storage.
struct Slot {
  double* base;
  long long stride;  // nslots
  __device__ __forceinline__ double& operator[](long long e) const { return base[e * stride]; }
};

template <int NP>
__device__ __forceinline__ void mat_mul(const double (&A)[NP][NP], const double (&B)[NP][NP],
                                        double (&C)[NP][NP]) {
#pragma unroll 1
  for (int i = 0; i < NP; ++i)
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < NP; ++k) s = fma(A[i][k], B[k][j], s);
      C[i][j] = s;
    }
}

template <int NP>
__device__ __forceinline__ void mat_vec(const double (&A)[NP][NP], const double (&v)[NP],
                                        double (&y)[NP]) {
#pragma unroll 1
  for (int i = 0; i < NP; ++i) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < NP; ++k) s = fma(A[i][k], v[k], s);
    y[i] = s;
  }
}

// X = B A^{-1} (A and B are overwritten): column elimination with the pivot
// on the largest |entry| of the pivot row among the unused columns.  Returns
// nonzero if a pivot was exactly 0.
template <int NP>
__device__ int right_solve(double (&A)[NP][NP], double (&B)[NP][NP], double (&X)[NP][NP]) {
  int q[NP];
  unsigned used = 0;
  int singular = 0;
#pragma unroll 1
  for (int k = 0; k < NP; ++k) {
    int p = -1;
    double best = -1.0;
#pragma unroll 1
    for (int c = 0; c < NP; ++c)
      if (!((used >> c) & 1u) && fabs(A[k][c]) > best) {
        best = fabs(A[k][c]);
        p = c;
      }
    used |= 1u << p;
    singular |= (A[k][p] == 0.0);
    const double inv = recip(A[k][p]);
    double rv[NP];
#pragma unroll
    for (int c = 0; c < NP; ++c) rv[c] = A[k][c];
#pragma unroll 1
    for (int r = 0; r < NP; ++r) {
      const double ca = A[r][p] * inv, cb = B[r][p] * inv;
#pragma unroll
      for (int c = 0; c < NP; ++c) {
        if (c == p) continue;
        A[r][c] = fma(-ca, rv[c], A[r][c]);
        B[r][c] = fma(-cb, rv[c], B[r][c]);
      }
      A[r][p] = ca;
      B[r][p] = cb;
    }
    q[p] = k;
  }
#pragma unroll 1
  for (int c = 0; c < NP; ++c)
#pragma unroll 1
    for (int r = 0; r < NP; ++r) X[r][q[c]] = B[r][c];
  return singular;
}

// x^T = b^T A^{-1}, i.e. A^T x = b, for one right-hand side (A overwritten).
template <int NP>
__device__ int vec_right_solve(double (&A)[NP][NP], const double (&b)[NP], double (&x)[NP]) {
  double B[NP][NP], X[NP][NP];
#pragma unroll 1
  for (int r = 0; r < NP; ++r)
#pragma unroll
    for (int c = 0; c < NP; ++c) B[r][c] = (r == 0) ? b[c] : 0.0;
  const int s = right_solve<NP>(A, B, X);
#pragma unroll
  for (int c = 0; c < NP; ++c) x[c] = X[0][c];
  return s;
}

// Phase matrices P++ / P+- (Hansen-normalised, src/phase_matrix.hpp:61-111)
// and, with a solar beam, the normalised phase vectors at mu0 (:131-181).
template <int NP>
__device__ void phase(const double* chi, int nuse, double f, int N, const double* pl,
                      const double (&wt)[NP], bool solar, double mu0, double (&Ppp)[NP][NP],
                      double (&Ppm)[NP][NP], double (&pp)[NP], double (&pm)[NP]) {
  const double inv_1mf = (f >= 0.0) ? 1.0 / (1.0 - f) : 1.0;
#pragma unroll 1
  for (int r = 0; r < NP; ++r)
#pragma unroll 1
    for (int c = 0; c < NP; ++c) {
      double spp = 0.0, spm = 0.0;
      if (r < N && c < N) {
        double sign = 1.0;
        for (int l = 0; l < nuse; ++l) {
          const double cl = (f >= 0.0) ? (chi[l] - f) * inv_1mf : chi[l];
          const double term = (2 * l + 1) * cl * pl[l * N + r] * pl[l * N + c];
          spp += term;
          spm += sign * term;
          sign = -sign;
        }
        spp /= (2.0 * kPi);
        spm /= (2.0 * kPi);
      }
      Ppp[r][c] = spp;
      Ppm[r][c] = spm;
    }
#pragma unroll 1
  for (int c = 0; c < N; ++c) {
    double sum = 0.0;
    for (int i = 0; i < N; ++i) sum += (Ppp[i][c] + Ppm[i][c]) * wt[i];
    if (sum > 0.0) {
      const double corr = 1.0 / (2.0 * kPi * sum);
      for (int i = 0; i < N; ++i) {
        Ppp[i][c] *= corr;
        Ppm[i][c] *= corr;
      }
    }
  }
  if (!solar) return;
#pragma unroll 1
  for (int t = 0; t < NP; ++t) {
    double sp = 0.0, sm = 0.0;
    if (t < N) {
      double sign = 1.0, p0 = 1.0, p1 = mu0;
      for (int l = 0; l < nuse; ++l) {
        double plm;
        if (l == 0) {
          plm = 1.0;
        } else if (l == 1) {
          plm = mu0;
        } else {
          plm = ((2 * l - 1) * mu0 * p1 - (l - 1) * p0) * recip((double)l);
          p0 = p1;
          p1 = plm;
        }
        const double cl = (f >= 0.0) ? (chi[l] - f) * inv_1mf : chi[l];
        const double term = (2 * l + 1) * cl * pl[l * N + t] * plm;
        sp += term;
        sm += sign * term;
        sign = -sign;
      }
      sp /= (2.0 * kPi);
      sm /= (2.0 * kPi);
    }
    pp[t] = sp;
    pm[t] = sm;
  }
  double sum = 0.0;
  for (int i = 0; i < N; ++i) sum += (pp[i] + pm[i]) * wt[i];
  const double corr = (sum > 0.0) ? 1.0 / (2.0 * kPi * sum) : 1.0;
  for (int i = 0; i < N; ++i) {
    pp[i] *= corr;
    pm[i] *= corr;
  }
}

// Doubling of one scattering layer (reference order, src/doubling.hpp:79-229):
// R, T and the combined thermal + solar sources s_up / s_dn.
template <int NP>
__device__ int doubling(double tau, double om, double Bt, double Bb, double tcum, int N,
                        bool solar, double F0, double mu0, const double (&mu)[NP],
                        const double (&wt)[NP], const double (&Ppp)[NP][NP],
                        const double (&Ppm)[NP][NP], const double (&pp)[NP],
                        const double (&pm)[NP], double (&R)[NP][NP], double (&T)[NP][NP],
                        double (&sup)[NP], double (&sdn)[NP]) {
  om = om > 1.0 ? 1.0 : om;
  const double con = 2.0 * om * kPi;
  const int nn = num_doublings(tau, om);
  const double tau0 = ldexp(tau, -nn);
  const double Ftop = solar ? F0 * exp(-tcum / mu0) : 0.0;
#pragma unroll 1
  for (int r = 0; r < NP; ++r)
#pragma unroll 1
    for (int c = 0; c < NP; ++c) {
      double tv = (r == c) ? 1.0 : 0.0, rv = 0.0;
      if (r < N && c < N) {
        const double pppc = Ppp[r][c] * wt[c];
        const double temp = ((r == c) ? 1.0 : 0.0) + (-con) * pppc;
        const double gpp = temp / mu[r];
        tv = ((r == c) ? 1.0 : 0.0) - tau0 * gpp;
        const double gpm = con * (Ppm[r][c] * wt[c]) / mu[r];
        rv = tau0 * gpm;
      }
      T[r][c] = tv;
      R[r][c] = rv;
    }
  double y[NP], z[NP], su[NP], sd[NP];
#pragma unroll
  for (int i = 0; i < NP; ++i) {
    y[i] = z[i] = su[i] = sd[i] = 0.0;
    if (i < N) {
      y[i] = (1.0 - om) * tau0 / mu[i];
      if (solar) {
        const double base = om * tau0 / mu[i] * Ftop;
        su[i] = base * pm[i];
        sd[i] = base * pp[i];
      }
    }
  }
  double g = 0.5 * tau0;
  double gam = solar ? exp(-tau0 / mu0) : 0.0;
  int singular = 0;
  double A[NP][NP], TG[NP][NP], TGR[NP][NP], W[NP][NP];
#pragma unroll 1
  for (int k = 0; k < nn; ++k) {
    double ru[NP], rd[NP];
    if (solar) {
      double a[NP], b[NP];
      mat_vec<NP>(R, sd, a);
      mat_vec<NP>(R, su, b);
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        ru[i] = a[i] + gam * su[i];
        rd[i] = gam * b[i] + sd[i];
      }
    }
    mat_mul<NP>(R, R, A);
#pragma unroll 1
    for (int r = 0; r < NP; ++r)
#pragma unroll
      for (int c = 0; c < NP; ++c) {
        A[r][c] = ((r == c) ? 1.0 : 0.0) - A[r][c];
        W[r][c] = T[r][c];
      }
    singular |= right_solve<NP>(A, W, TG);  // TG = T (I - R^2)^{-1}
    mat_mul<NP>(TG, R, TGR);
    double v[NP], tg0[NP], tg1[NP], tr0[NP], tr1[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) v[i] = z[i] + g * y[i];
    mat_vec<NP>(TG, v, tg0);
    mat_vec<NP>(TG, y, tg1);
    mat_vec<NP>(TGR, v, tr0);
    mat_vec<NP>(TGR, y, tr1);
    double tu0[NP], tu1[NP];
    if (solar) {
      mat_vec<NP>(TG, ru, tu0);
      mat_vec<NP>(TG, rd, tu1);
    }
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      const double zn = (tg0[i] - tr0[i]) + z[i] - g * y[i];
      const double yn = tg1[i] + tr1[i] + y[i];
      z[i] = zn;
      y[i] = yn;
      if (solar) {
        su[i] = tu0[i] + su[i];
        sd[i] = tu1[i] + gam * sd[i];
      }
    }
    mat_mul<NP>(TGR, T, W);  // R <- R + TGR T
#pragma unroll 1
    for (int r = 0; r < NP; ++r)
#pragma unroll
      for (int c = 0; c < NP; ++c) R[r][c] += W[r][c];
    mat_mul<NP>(TG, T, W);  // T <- TG T
#pragma unroll 1
    for (int r = 0; r < NP; ++r)
#pragma unroll
      for (int c = 0; c < NP; ++c) T[r][c] = W[r][c];
    gam = gam * gam;
    g = 2.0 * g;
  }
  const double Bbar = (Bb + Bt) / 2.0;
  const double Bd = (Bb - Bt) / tau;
#pragma unroll
  for (int i = 0; i < NP; ++i) {
    sup[i] = (i < N) ? (y[i] * Bbar + z[i] * Bd) + su[i] : 0.0;
    sdn[i] = (i < N) ? (y[i] * Bbar - z[i] * Bd) + sd[i] : 0.0;
  }
  return singular;
}

// One wavenumber w of column C, by one thread.
template <int NP>
__device__ void solve_wavenumber(const ColumnDev* C, int w, const Slot& S, int lmax,
                                 unsigned* status) {
  const int N = C->N, nL = C->L, M = C->M, layout = C->moment_layout;
  const int from_bottom = C->from_bottom;
  const long long lev = lmax + 1;
  const long long oB = 0, oTC = lev, oTAU = 2 * lev, oOM = 3 * lev, oOMU = 4 * lev;
  const long long oREC = (long long)kLev * lev;
  using RC = Rec<NP>;
  const double wlo = C->wlo_w ? C->wlo_w[w] : C->wn_lo;
  const double whi = C->whi_w ? C->whi_w[w] : C->wn_hi;
  double mu[NP], wt[NP], cw[NP], hw[NP];
#pragma unroll
  for (int i = 0; i < NP; ++i) {
    mu[i] = (i < N) ? C->quad.mu[i] : 1.0;
    wt[i] = (i < N) ? C->quad.wt[i] : 0.0;
    cw[i] = 2.0 * kPi * wt[i] * mu[i];
    hw[i] = 0.5 * wt[i];
  }
  // ---- prologue: Planck levels, delta-M scaled layers, cumulative tau
  unsigned bad = 0;
  for (int l = 0; l <= nL; ++l) {
    const int ul = from_bottom ? nL - l : l;
    double Bv = 0.0;
    if (C->thermal) {
      const double Tv = C->temperature[(C->temp_per_wav ? (size_t)w * (nL + 1) : 0) + ul];
      if (!(Tv >= 0.0)) bad = 1;
      Bv = planck_band(wlo, whi, Tv);
    } else if (C->planck) {
      Bv = C->planck[(size_t)w * (nL + 1) + ul];
    }
    S[oB + l] = Bv;
  }
  double tc = 0.0;
  S[oTC] = 0.0;
  for (int l = 0; l < nL; ++l) {
    const int u = from_bottom ? nL - 1 - l : l;
    double tau = C->dtau[(size_t)w * nL + u];
    double om = C->ssa[(size_t)w * nL + u];
    if (!(tau >= 0.0 && tau < 1e300) || !(om >= 0.0 && om <= 1.0)) bad = 1;
    S[oOMU + l] = om;
    if (om > 0.0 && tau > 0.0 && C->delta_m && M > 2 * N) {
      const double* chi = C->moments + (layout == 0 ? (size_t)u * M
                                        : layout == 1 ? (size_t)w * M
                                                      : ((size_t)w * nL + u) * M);
      const double f = chi[2 * N];
      if (f > 1e-12 && f < 1.0 - 1e-12) {
        const double of = om * f;
        tau = (1.0 - of) * tau;
        om = om * (1.0 - f) / (1.0 - of);
      }
    }
    if (tau > 0.0 && om > 0.0 && tau >= ldexp(1.0, kMaxDoublings + 1 - ipow0(om > 1.0 ? 1.0 : om)))
      bad = 1;  // beyond the doubling bound (as the warp kernels)
    S[oTAU + l] = tau;
    S[oOM + l] = om;
    tc += tau;
    S[oTC + l + 1] = tc;
  }
  if (bad) atomicOr(status, 4u);
  double Bs, Btop;
  if (C->thermal) {
    Bs = (C->surface_temperature >= 0.0) ? planck_band(wlo, whi, C->surface_temperature)
                                         : S[oB + nL];
    Btop = (C->top_temperature >= 0.0) ? planck_band(wlo, whi, C->top_temperature) : S[oB];
  } else {
    Bs = C->semis_w ? C->semis_w[w] : C->surface_emission;
    Btop = C->temis_w ? C->temis_w[w] : C->top_emission;
  }
  const double A = C->albedo_w ? C->albedo_w[w] : C->surface_albedo;
  const double mu0 = C->mu0_w ? C->mu0_w[w] : C->solar_mu;
  const double F0 = C->solar_flux;
  const bool solar = (F0 > 0.0 && mu0 > 0.0);
  const bool has_surface = !C->diffusion && (A > 0.0 || Bs > 0.0);
  auto moments = [&](int l, int& nuse, double& f) -> const double* {
    const int u = from_bottom ? nL - 1 - l : l;
    const double* chi = C->moments + (layout == 0 ? (size_t)u * M
                                      : layout == 1 ? (size_t)w * M
                                                    : ((size_t)w * nL + u) * M);
    nuse = M;
    f = -1.0;
    if (C->delta_m) {
      const double ff = (M > 2 * N) ? chi[2 * N] : 0.0;
      if (ff > 1e-12 && ff < 1.0 - 1e-12) {
        f = ff;
        nuse = 2 * N;
      } else {
        nuse = (M < 2 * N) ? M : 2 * N;
      }
    }
    return chi;
  };
  double Ppp[NP][NP], Ppm[NP][NP], pp[NP], pm[NP];
  if (layout == 1) {
    int nuse;
    double f;
    const double* chi = moments(0, nuse, f);
    phase<NP>(chi, nuse, f, N, C->quad.pl, wt, solar, mu0, Ppp, Ppm, pp, pm);
  }
  // ---- bottom composite: surface, or the lower boundary intensity
  double Rb[NP][NP], Ub[NP];
  {
    const double dt = C->diffusion ? S[oTAU + nL - 1] : 0.0;
    const double dB = (C->diffusion && dt > 0.0) ? (S[oB + nL] - S[oB + nL - 1]) / dt : 0.0;
    const long long rb = oREC + (long long)nL * RC::SIZE;
#pragma unroll 1
    for (int r = 0; r < NP; ++r)
#pragma unroll 1
      for (int c = 0; c < NP; ++c) {
        double v = 0.0;
        if (has_surface && r < N && c < N) v = 2.0 * A * mu[c] * wt[c] * C->quad.xfac;
        Rb[r][c] = v;
        S[rb + RC::RB + r * NP + c] = v;
      }
#pragma unroll 1
    for (int i = 0; i < NP; ++i) {
      double u = 0.0;
      if (i < N) {
        if (has_surface) {
          u = (1.0 - A) * Bs;
          if (solar && A > 0.0) u = u + (A / kPi) * F0 * mu0 * exp(-S[oTC + nL] / mu0);
        } else if (C->diffusion) {
          u = S[oB + nL] + mu[i] * dB;
        } else {
          u = Bs;
        }
      }
      Ub[i] = u;
      S[rb + RC::UB + i] = u;
    }
  }
  int cs = (has_surface && A > 0.0) ? 1 : 0;
  S[oREC + (long long)nL * RC::SIZE + RC::CS] = cs;
  // ---- upward: doubling + adding onto the composite below
  int singular = 0;
  double R[NP][NP], T[NP][NP], X1[NP][NP], X2[NP][NP], sup[NP], sdn[NP], tv[NP];
#pragma unroll 1
  for (int l = nL - 1; l >= 0; --l) {
    const double tau = S[oTAU + l], om = S[oOM + l];
    const double Bt = S[oB + l], Bb = S[oB + l + 1];
    const int scat = (tau > 0.0 && om > 0.0);
    const long long rp = oREC + (long long)l * RC::SIZE;
    if (!scat) {
      // transparent or pure absorption (src/doubling.hpp:49-77)
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        double t1 = 1.0, up = 0.0, dn = 0.0;
        if (i < N && tau > 0.0) {
          const double Bbar = (Bb + Bt) / 2.0;
          const double Bd = (Bb - Bt) / tau;
          const double tex = -tau / mu[i];
          t1 = (tex > -200.0) ? exp(tex) : 0.0;
          const double omt = 1.0 - t1;
          const double slope = mu[i] * omt - 0.5 * tau * (1.0 + t1);
          up = Bbar * omt + Bd * slope;
          dn = Bbar * omt - Bd * slope;
        }
        tv[i] = t1;
        sup[i] = up;
        sdn[i] = dn;
      }
#pragma unroll 1
      for (int r = 0; r < NP; ++r)
#pragma unroll 1
        for (int c = 0; c < NP; ++c) {
          S[rp + RC::R + r * NP + c] = 0.0;
          S[rp + RC::T + r * NP + c] = (r == c) ? tv[r] : 0.0;
        }
    } else {
      if (layout != 1) {
        int nuse;
        double f;
        const double* chi = moments(l, nuse, f);
        phase<NP>(chi, nuse, f, N, C->quad.pl, wt, solar, mu0, Ppp, Ppm, pp, pm);
      }
      singular |= doubling<NP>(tau, om, Bt, Bb, S[oTC + l], N, solar, F0, mu0, mu, wt, Ppp, Ppm,
                               pp, pm, R, T, sup, sdn);
#pragma unroll 1
      for (int r = 0; r < NP; ++r)
#pragma unroll 1
        for (int c = 0; c < NP; ++c) {
          S[rp + RC::R + r * NP + c] = R[r][c];
          S[rp + RC::T + r * NP + c] = T[r][c];
        }
    }
#pragma unroll 1
    for (int i = 0; i < NP; ++i) S[rp + RC::SDN + i] = sdn[i];
    S[rp + RC::SCAT] = scat;
    // adding: top = this layer, bottom = composite (src/adding.hpp:478-490)
    if (!scat) {
      // R_b <- t R_b t, U_b <- s_up + t (U_b + R_b s_dn)
      double y[NP];
      mat_vec<NP>(Rb, sdn, y);
#pragma unroll
      for (int i = 0; i < NP; ++i) Ub[i] = sup[i] + tv[i] * (Ub[i] + y[i]);
#pragma unroll 1
      for (int r = 0; r < NP; ++r)
#pragma unroll 1
        for (int c = 0; c < NP; ++c) Rb[r][c] = tv[r] * Rb[r][c] * tv[c];
    } else if (!cs) {
      // R_b <- R, U_b <- s_up + T U_b
      double y[NP];
      mat_vec<NP>(T, Ub, y);
#pragma unroll
      for (int i = 0; i < NP; ++i) Ub[i] = sup[i] + y[i];
#pragma unroll 1
      for (int r = 0; r < NP; ++r)
#pragma unroll 1
        for (int c = 0; c < NP; ++c) Rb[r][c] = R[r][c];
      cs = 1;
    } else {
      // A1 = I - R_b R, D1 = T A1^{-1}, U_b <- s_up + D1 (U_b + R_b s_dn),
      // R_b <- R + (D1 R_b) T
      double y[NP], v[NP];
      mat_vec<NP>(Rb, sdn, y);
#pragma unroll
      for (int i = 0; i < NP; ++i) v[i] = Ub[i] + y[i];
      mat_mul<NP>(Rb, R, X1);
#pragma unroll 1
      for (int r = 0; r < NP; ++r)
#pragma unroll
        for (int c = 0; c < NP; ++c) {
          X1[r][c] = ((r == c) ? 1.0 : 0.0) - X1[r][c];
          X2[r][c] = T[r][c];
        }
      double D1[NP][NP];
      singular |= right_solve<NP>(X1, X2, D1);
      mat_vec<NP>(D1, v, y);
#pragma unroll
      for (int i = 0; i < NP; ++i) Ub[i] = sup[i] + y[i];
      mat_mul<NP>(D1, Rb, X1);
      mat_mul<NP>(X1, T, X2);
#pragma unroll 1
      for (int r = 0; r < NP; ++r)
#pragma unroll
        for (int c = 0; c < NP; ++c) Rb[r][c] = R[r][c] + X2[r][c];
    }
#pragma unroll 1
    for (int r = 0; r < NP; ++r)
#pragma unroll 1
      for (int c = 0; c < NP; ++c) S[rp + RC::RB + r * NP + c] = Rb[r][c];
#pragma unroll 1
    for (int i = 0; i < NP; ++i) S[rp + RC::UB + i] = Ub[i];
    S[rp + RC::CS] = cs;
  }
  // ---- downward pass and interface fluxes
  double Id[NP], Iu[NP];
  auto emit = [&](int l) {
    double fu = 0.0, fd = 0.0, J = 0.0;
    for (int i = 0; i < N; ++i) {
      fu += cw[i] * Iu[i];
      fd += cw[i] * Id[i];
      J += hw[i] * (Iu[i] + Id[i]);
    }
    double fdir = 0.0;
    if (solar) {
      fdir = (l == 0) ? F0 * mu0 : F0 * mu0 * exp(-S[oTC + l] / mu0);
      J += fdir * (1.0 / (4.0 * kPi * mu0));
    }
    const int lyr = (l == 0) ? 0 : l - 1;
    const double divF = 4.0 * kPi * (1.0 - S[oOMU + lyr]) * (J - S[oB + l]);
    const size_t oi = (size_t)w * (nL + 1) + (from_bottom ? nL - l : l);
    if (C->fu) C->fu[oi] = fu;
    if (C->fd) C->fd[oi] = fd;
    if (C->fdir) C->fdir[oi] = fdir;
    if (C->J) C->J[oi] = J;
    if (C->divF) C->divF[oi] = divF;
    if (l == 0) {
      if (C->toa_fu) C->toa_fu[w] = fu * C->spectrum_scaling;
      if (C->toa_fd) C->toa_fd[w] = fd;
    }
    if (l == nL && C->boa_fdir) C->boa_fdir[w] = fdir;
    if (!isfinite(fu) || !isfinite(fd) || !isfinite(J)) atomicOr(status, 2u);
  };
  {
    const long long r0 = oREC;
#pragma unroll 1
    for (int r = 0; r < NP; ++r)
#pragma unroll 1
      for (int c = 0; c < NP; ++c) Rb[r][c] = S[r0 + RC::RB + r * NP + c];
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      Id[i] = (i < N) ? Btop : 0.0;
      Ub[i] = S[r0 + RC::UB + i];
    }
    double y[NP];
    mat_vec<NP>(Rb, Id, y);
#pragma unroll
    for (int i = 0; i < NP; ++i) Iu[i] = y[i] + Ub[i];
    emit(0);
  }
#pragma unroll 1
  for (int l = 0; l < nL; ++l) {
    const long long rl = oREC + (long long)l * RC::SIZE;
    const long long rb = oREC + (long long)(l + 1) * RC::SIZE;
    const int scat = S[rl + RC::SCAT] != 0.0;
    const int cbase = S[rb + RC::CS] != 0.0;
#pragma unroll 1
    for (int r = 0; r < NP; ++r)
#pragma unroll 1
      for (int c = 0; c < NP; ++c) {
        R[r][c] = S[rl + RC::R + r * NP + c];
        T[r][c] = S[rl + RC::T + r * NP + c];
        Rb[r][c] = S[rb + RC::RB + r * NP + c];
      }
    double rhs[NP], a0[NP], a1[NP], x[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      Ub[i] = S[rb + RC::UB + i];
      sdn[i] = S[rl + RC::SDN + i];
    }
    // rhs = T I_dn + R U_base + s_dn
    mat_vec<NP>(T, Id, a0);
    mat_vec<NP>(R, Ub, a1);
#pragma unroll
    for (int i = 0; i < NP; ++i) rhs[i] = (a0[i] + a1[i]) + sdn[i];
    if (scat && cbase) {
      // (I - R R_base) x = rhs, as x^T = rhs^T (I - R R_base)^{-T}
      mat_mul<NP>(R, Rb, X1);
#pragma unroll 1
      for (int r = 0; r < NP; ++r)
#pragma unroll
        for (int c = 0; c < NP; ++c) X2[c][r] = ((r == c) ? 1.0 : 0.0) - X1[r][c];
      singular |= vec_right_solve<NP>(X2, rhs, x);
    } else {
#pragma unroll
      for (int i = 0; i < NP; ++i) x[i] = rhs[i];
    }
    double y[NP];
    mat_vec<NP>(Rb, x, y);
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      Id[i] = x[i];
      Iu[i] = y[i] + Ub[i];
    }
    emit(l + 1);
  }
  if (singular) atomicOr(status, 1u);
}

// The persistent thread-per-wavenumber launch over a column table (tasks
// flattened in column order as for solve_kernel_multi); a thread takes the
// next task from the work counter.  Columns of padded order above NP are not
// this kernel's (the host sends each column to the kernel of its order).
template <int NP>
__global__ void __launch_bounds__(128) solve_kernel_tpw(SolveParams P) {
  const long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= P.nslots) return;
  const Slot S{reinterpret_cast<double*>(P.scratch) + slot, (long long)P.nslots};
  for (;;) {
    const long long task = (long long)atomicAdd(P.counter, 1ull);
    if (task >= P.ntasks) break;
    int lo = 0, hi = P.ncols - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (P.cols[mid].task_begin <= task) lo = mid; else hi = mid - 1;
    }
    const ColumnDev* C = &P.cols[lo];
    solve_wavenumber<NP>(C, (int)(task - C->task_begin), S, P.max_layers, P.status);
  }
}

}  // namespace tpw
}  // namespace adrt_dev
