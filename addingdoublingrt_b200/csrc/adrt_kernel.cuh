// adrt_kernel.cuh -- per-wavenumber solve and the persistent batch kernel.
#pragma once

#include "adrt_solver.cuh"

namespace adrt_dev {

// Per-slot HBM scratch of one thread group: level scalars, the phase
// matrices of the current moment set, then one record per interface l =
// 0..L (the layer below it: R, T, s_down; the composite of everything below
// it: R_base, U_base) for the downward pass.
template <class Gm>
struct SlotLayout {
  using Real = typename Gm::Real;
  static constexpr int NP = Gm::NP;
  static constexpr int TILE = Gm::G * Gm::TE;  // Reals per matrix in tile order
  static constexpr int REC_RAW = 3 * TILE + 2 * NP + 2;
  static constexpr int RALIGN = 16 / (int)sizeof(Real);
  static constexpr int REC = (REC_RAW + RALIGN - 1) / RALIGN * RALIGN;
  static __host__ __device__ size_t level_bytes(int lmax) {
    return ((size_t)5 * (lmax + 1) * sizeof(double) + 255) & ~size_t(255);
  }
  static __host__ __device__ size_t phase_bytes() {
    return ((size_t)2 * NP * NP * sizeof(double) + 255) & ~size_t(255);
  }
  static __host__ __device__ size_t bytes(int lmax) {
    return level_bytes(lmax) + phase_bytes() + (size_t)(lmax + 1) * REC * sizeof(Real);
  }
};

// Pointers into one group's shared memory.  Built inside every function
// from the group's byte offset `goff` into adrt_smem, so the compiler sees
// shared-space pointers; non-inlined calls receive (goff, t, bar).
template <class Gm>
struct Ctx {
  using Real = typename Gm::Real;
  using SL = SmemLayout<Gm>;
  static constexpr int NP = Gm::NP, MAT = Gm::MAT;
  unsigned goff;
  int t, lane, warp, bar;
  Real *vec, *gjbuf;
  double* dvec;
  ColumnDev* col;
  unsigned* red;
  double* dmisc;
  __device__ __forceinline__ Ctx(unsigned goff_, int t_, int bar_)
      : goff(goff_), t(t_), lane(t_ & 31), warp(t_ >> 5), bar(bar_) {
    vec = sp<Real>(goff + SL::vecs);
    gjbuf = sp<Real>(goff + SL::gj);
    dvec = sp<double>(goff + SL::dvecs);
    col = sp<ColumnDev>(goff + SL::col);
    red = sp<unsigned>(goff + SL::misc);
    dmisc = sp<double>(goff + SL::misc + 32);
  }
  __device__ __forceinline__ unsigned mo(int i) const {
    return goff + (unsigned)(SL::mats + (size_t)i * MAT * sizeof(Real));
  }
  __device__ __forceinline__ Real* m(int i) const { return sp<Real>(mo(i)); }
  __device__ __forceinline__ unsigned vo(int s) const {
    return goff + (unsigned)(SL::vecs + (size_t)s * NP * sizeof(Real));
  }
  __device__ __forceinline__ unsigned gjo() const { return goff + (unsigned)SL::gj; }
  __device__ __forceinline__ unsigned redo() const { return goff + (unsigned)SL::misc; }
  __device__ __forceinline__ Real* V(int s) const { return vec + s * NP; }
  __device__ __forceinline__ double* DV(int s) const { return dvec + s * NP; }
  __device__ __forceinline__ void sync() const { gsync<Gm::G>(bar); }
};

// ------------------------------------------------------------- phase matrices
// P++/P+- from Legendre moments with Hansen column renormalisation
// (src/phase_matrix.hpp:61-111) into the slot (row-major NP x NP doubles)
// and, with a solar beam, the phase vectors at mu0 (src/phase_matrix.hpp:
// 131-181) into D_PP / D_PM.  chi_l = (chi[l] - f) / (1 - f) when delta-M
// truncation applies (f >= 0), chi[l] otherwise.
template <class Gm>
__device__ __noinline__ void build_phase(unsigned goff, int t_, int bar, const double* chi,
                                         int nuse, double f, int N, const double* pl, bool solar,
                                         double mu0, double* Ppp, double* Ppm) {
  constexpr int NP = Gm::NP, G = Gm::G;
  const Ctx<Gm> X(goff, t_, bar);
  const int t = X.t;
  const double inv_1mf = (f >= 0.0) ? 1.0 / (1.0 - f) : 1.0;
  const double* wt = X.DV(D_WT);
  for (int e = t; e < NP * NP; e += G) {
    const int r = e / NP, c = e % NP;
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
    Ppp[e] = spp;
    Ppm[e] = spm;
  }
  X.sync();
  if (t < N) {
    const int c = t;
    double sum = 0.0;
    for (int i = 0; i < N; ++i) sum += (Ppp[i * NP + c] + Ppm[i * NP + c]) * wt[i];
    if (sum > 0.0) {
      const double corr = 1.0 / (2.0 * kPi * sum);
      for (int i = 0; i < N; ++i) {
        Ppp[i * NP + c] *= corr;
        Ppm[i * NP + c] *= corr;
      }
    }
  }
  if (solar) {
    double* pp = X.DV(D_PP);
    double* pm = X.DV(D_PM);
    if (t < NP) {
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
            plm = ((2 * l - 1) * mu0 * p1 - (l - 1) * p0) / l;
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
    X.sync();
    double corr = 1.0;
    {
      double sum = 0.0;
      for (int i = 0; i < N; ++i) sum += (pp[i] + pm[i]) * wt[i];
      if (sum > 0.0) corr = 1.0 / (2.0 * kPi * sum);
    }
    X.sync();
    if (t < N) {
      pp[t] *= corr;
      pm[t] *= corr;
    }
  }
  X.sync();
}

// ------------------------------------------------------------- doubling
// One homogeneous scattering layer (src/doubling.hpp:79-229): first-order
// thin-layer start at tau0 = tau 2^-nn, then nn doublings of R, T and of the
// thermal (y, z) and solar sources.  On return R is in m[0] (row-major) and
// m[1] (column-major), T in m[return value] (row-major, 2 or 3), and the
// combined thermal + solar sources in V_SUP / V_SDN.
template <class Gm>
__device__ __noinline__ int doubling(unsigned goff, int t_, int bar, double tau, double om,
                                     double Bt, double Bb, double tcum, int N, bool solar,
                                     double F0, double mu0, const double* Ppp, const double* Ppm,
                                     int* singular) {
  using Real = typename Gm::Real;
  const Ctx<Gm> X(goff, t_, bar);
  constexpr int NP = Gm::NP, TR = Gm::TR, TC = Gm::TC;
  const int t = X.t;
  const double* mu = X.DV(D_MU);
  const double* wt = X.DV(D_WT);
  om = om > 1.0 ? 1.0 : om;
  const double con = 2.0 * om * kPi;
  const int nn = num_doublings(tau, om);
  const double tau0 = ldexp(tau, -nn);
  const double Ftop = solar ? F0 * exp(-tcum / mu0) : 0.0;
  const unsigned oR = X.mo(0), oRc = X.mo(1), oA = X.mo(4), oTG = X.mo(5);
  const unsigned oT[2] = {X.mo(2), X.mo(3)};
  Real* Rrm = sp<Real>(oR);
  Real* Rcm = sp<Real>(oRc);
  Real* Am = sp<Real>(oA);  // I - R R, then TG R (column-major)
  Real* TGcm = sp<Real>(oTG);
  // thin-layer start (FP64): T = I - tau0 Gpp, R = tau0 Gpm
  {
    const Tile<Gm> tl(t);
    if (tl.valid()) {
      Real Rt[TR][TC], Tt[TR][TC];
#pragma unroll
      for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) {
          const int r = tl.row(a), c = tl.col(b);
          double tv = (r == c) ? 1.0 : 0.0, rv = 0.0;
          if (r < N && c < N) {
            const double pppc = Ppp[r * NP + c] * wt[c];
            const double temp = ((r == c) ? 1.0 : 0.0) + (-con) * pppc;
            const double gpp = temp / mu[r];
            tv = ((r == c) ? 1.0 : 0.0) - tau0 * gpp;
            const double gpm = con * (Ppm[r * NP + c] * wt[c]) / mu[r];
            rv = tau0 * gpm;
          }
          Tt[a][b] = static_cast<Real>(tv);
          Rt[a][b] = static_cast<Real>(rv);
        }
      tl.store_rm(Rt, Rrm);
      tl.store_cm(Rt, Rcm);
      tl.store_rm(Tt, sp<Real>(oT[0]));
    }
  }
  if (X.warp == 0 && X.lane < NP) {
    const int i = X.lane;
    double y = 0.0, su = 0.0, sd = 0.0;
    if (i < N) {
      y = (1.0 - om) * tau0 / mu[i];
      if (solar) {
        const double base = om * tau0 / mu[i] * Ftop;
        su = base * X.DV(D_PM)[i];
        sd = base * X.DV(D_PP)[i];
      }
    }
    X.V(V_Y0)[i] = static_cast<Real>(y);
    X.V(V_Z0)[i] = Real(0);
    X.V(V_SU0)[i] = static_cast<Real>(su);
    X.V(V_SD0)[i] = static_cast<Real>(sd);
  }
  Real g = static_cast<Real>(0.5 * tau0);
  Real gam = solar ? static_cast<Real>(exp(-tau0 / mu0)) : Real(0);
  int cur = 0;
  for (int k = 0; k < nn; ++k) {
    const int par = k & 1;
    Real* y = X.V(V_Y0 + par);
    Real* z = X.V(V_Z0 + par);
    Real* su = X.V(V_SU0 + par);
    Real* sd = X.V(V_SD0 + par);
    const unsigned oTc = oT[cur];
    X.sync();  // R, T and the vectors of the previous step are complete
    if (solar && X.warp == 0) {  // ru = R sd + gam su, rd = gam R su + sd (old R)
      const Real* vv[2] = {sd, su};
      Real yv[2];
      matvec<Gm, true, 2>(Rcm, vv, yv, X.lane);
      if (X.lane < NP) {
        X.V(V_RU)[X.lane] = yv[0] + gam * su[X.lane];
        X.V(V_RD)[X.lane] = gam * yv[1] + sd[X.lane];
      }
    }
    op_gemm<Gm>(oRc, oR, kNoMat, 1, oA, kNoMat, t);  // I - R^2
    X.sync();
    *singular |= op_gj<Gm>(oA, oTc, kNoMat, oTG, X.gjo(), X.redo(), t, X.bar);  // TG = T (I-R^2)^-1
    X.sync();
    op_gemm<Gm>(oTG, oR, kNoMat, 0, kNoMat, oA, t);  // TGR = TG R (column-major)
    X.sync();
    op_gemm<Gm>(oA, oTc, oR, 0, oR, oRc, t);                 // R <- R + TGR T
    op_gemm<Gm>(oTG, oTc, kNoMat, 0, oT[cur ^ 1], kNoMat, t);  // T <- TG T
    if (X.warp == 0) {
      Real* yn = X.V(V_Y0 + 1 - par);
      Real* zn = X.V(V_Z0 + 1 - par);
      Real* sun = X.V(V_SU0 + 1 - par);
      Real* sdn = X.V(V_SD0 + 1 - par);
      if (X.lane < NP) X.V(V_TMP)[X.lane] = z[X.lane] + g * y[X.lane];
      __syncwarp();
      const Real* va[2] = {X.V(V_TMP), y};
      Real tg[2], tgr[2];
      matvec<Gm, true, 2>(TGcm, va, tg, X.lane);
      matvec<Gm, true, 2>(Am, va, tgr, X.lane);
      Real tu[2] = {Real(0), Real(0)};
      if (solar) {
        const Real* vs[2] = {X.V(V_RU), X.V(V_RD)};
        matvec<Gm, true, 2>(TGcm, vs, tu, X.lane);
      }
      if (X.lane < NP) {
        const int i = X.lane;
        zn[i] = (tg[0] - tgr[0]) + z[i] - g * y[i];
        yn[i] = tg[1] + tgr[1] + y[i];
        sun[i] = solar ? tu[0] + su[i] : Real(0);
        sdn[i] = solar ? tu[1] + gam * sd[i] : Real(0);
      }
    }
    gam = gam * gam;
    g = Real(2) * g;
    cur ^= 1;
  }
  X.sync();
  if (X.warp == 0 && X.lane < NP) {
    const int i = X.lane, par = nn & 1;
    const double Bbar = (Bb + Bt) / 2.0;
    const double Bd = (Bb - Bt) / tau;
    const double y = X.V(V_Y0 + par)[i], z = X.V(V_Z0 + par)[i];
    const double su = X.V(V_SU0 + par)[i], sd = X.V(V_SD0 + par)[i];
    double up = 0.0, dn = 0.0;
    if (i < N) {
      up = (y * Bbar + z * Bd) + su;
      dn = (y * Bbar - z * Bd) + sd;
    }
    X.V(V_SUP)[i] = static_cast<Real>(up);
    X.V(V_SDN)[i] = static_cast<Real>(dn);
  }
  return 2 + cur;
}

// ------------------------------------------------------------- interface output
template <class Gm>
__device__ __forceinline__ void emit_interface(const Ctx<Gm>& X, const ColumnDev* C, int w, int l,
                                               int N, bool solar, double F0, double mu0,
                                               const double* lvTc, const double* lvOmu,
                                               const double* lvB, unsigned* status) {
  const typename Gm::Real* iu = X.V(V_IU);
  const typename Gm::Real* id = X.V(V_ID);
  const double* cw = X.DV(D_CW);
  const double* hw = X.DV(D_HW);
  double fu = 0.0, fd = 0.0, J = 0.0;
  for (int i = 0; i < N; ++i) {
    const double u = iu[i], d = id[i];
    fu += cw[i] * u;
    fd += cw[i] * d;
    J += hw[i] * (u + d);
  }
  double fdir = 0.0;
  if (solar) {
    fdir = (l == 0) ? F0 * mu0 : F0 * mu0 * exp(-lvTc[l] / mu0);
    J += fdir * (1.0 / (4.0 * kPi * mu0));
  }
  const int nL = C->L;
  const int lyr = (l == 0) ? 0 : l - 1;
  const double divF = 4.0 * kPi * (1.0 - lvOmu[lyr]) * (J - lvB[l]);
  const size_t oi = (size_t)w * (nL + 1) + (C->from_bottom ? nL - l : l);
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
}

// ------------------------------------------------------------- one wavenumber
template <class Gm>
__device__ __noinline__ void solve_one(unsigned goff, int t_, int bar, int w, char* slot, int lmax,
                                       unsigned* status) {
  using Real = typename Gm::Real;
  const Ctx<Gm> X(goff, t_, bar);
  using SLay = SlotLayout<Gm>;
  constexpr int NP = Gm::NP, G = Gm::G, TR = Gm::TR, TC = Gm::TC, LD = Gm::LD;
  constexpr int TILE = SLay::TILE;
  const ColumnDev* C = X.col;
  const int t = X.t;
  const int N = C->N, nL = C->L, M = C->M, layout = C->moment_layout;
  const int from_bottom = C->from_bottom;

  const double A = C->albedo_w ? C->albedo_w[w] : C->surface_albedo;
  const double mu0 = C->mu0_w ? C->mu0_w[w] : C->solar_mu;
  const double wlo = C->wlo_w ? C->wlo_w[w] : C->wn_lo;
  const double whi = C->whi_w ? C->whi_w[w] : C->wn_hi;
  const double F0 = C->solar_flux;
  const bool solar = (F0 > 0.0 && mu0 > 0.0);

  double* lvB = reinterpret_cast<double*>(slot);
  double* lvTc = lvB + (lmax + 1);
  double* lvTau = lvTc + (lmax + 1);
  double* lvOm = lvTau + (lmax + 1);
  double* lvOmu = lvOm + (lmax + 1);
  double* Ppp = reinterpret_cast<double*>(slot + SLay::level_bytes(lmax));
  double* Ppm = Ppp + NP * NP;
  Real* recs = reinterpret_cast<Real*>(slot + SLay::level_bytes(lmax) + SLay::phase_bytes());
  const double* chi_base = C->moments;

  // ---------------- quadrature constants for this column
  if (t < NP) {
    double mu = 1.0, wt = 0.0;
    if (t < N) {
      mu = C->quad.mu[t];
      wt = C->quad.wt[t];
    }
    X.DV(D_MU)[t] = mu;
    X.DV(D_WT)[t] = wt;
    X.DV(D_CW)[t] = 2.0 * kPi * wt * mu;
    X.DV(D_HW)[t] = 0.5 * wt;
  }

  // ---------------- prologue: Planck levels, scaled optical properties
  unsigned bad = 0;
  for (int l = t; l <= nL; l += G) {
    const int ul = from_bottom ? nL - l : l;
    double Bv = 0.0;
    if (C->thermal) {
      const double Tv = C->temperature[(C->temp_per_wav ? (size_t)w * (nL + 1) : 0) + ul];
      if (!(Tv >= 0.0)) bad = 1;
      Bv = planck_band(wlo, whi, Tv);
    } else if (C->planck) {
      Bv = C->planck[(size_t)w * (nL + 1) + ul];
    }
    lvB[l] = Bv;
  }
  for (int l = t; l < nL; l += G) {
    const int u = from_bottom ? nL - 1 - l : l;
    double tau = C->dtau[(size_t)w * nL + u];
    double om = C->ssa[(size_t)w * nL + u];
    if (!(tau >= 0.0 && tau < 1e300) || !(om >= 0.0 && om <= 1.0)) bad = 1;
    lvOmu[l] = om;
    if (om > 0.0 && tau > 0.0 && C->delta_m && M > 2 * N) {
      const double* chi = chi_base + (layout == 0 ? (size_t)u * M
                                      : layout == 1 ? (size_t)w * M
                                                    : ((size_t)w * nL + u) * M);
      const double f = chi[2 * N];
      if (f > 1e-12 && f < 1.0 - 1e-12) {
        const double of = om * f;
        tau = (1.0 - of) * tau;
        om = om * (1.0 - f) / (1.0 - of);
      }
    }
    lvTau[l] = tau;
    lvOm[l] = om;
  }
  if (bad) atomicOr(status, 4u);
  X.sync();
  if (t == 0) {
    double tc = 0.0;
    lvTc[0] = 0.0;
    for (int l = 0; l < nL; ++l) {
      tc += lvTau[l];
      lvTc[l + 1] = tc;
    }
    double Bs, Btop;
    if (C->thermal) {
      Bs = (C->surface_temperature >= 0.0) ? planck_band(wlo, whi, C->surface_temperature) : lvB[nL];
      Btop = (C->top_temperature >= 0.0) ? planck_band(wlo, whi, C->top_temperature) : lvB[0];
    } else {
      Bs = C->semis_w ? C->semis_w[w] : C->surface_emission;
      Btop = C->temis_w ? C->temis_w[w] : C->top_emission;
    }
    X.dmisc[0] = Bs;
    X.dmisc[1] = Btop;
  }
  X.sync();
  const double Bs = X.dmisc[0], Btop = X.dmisc[1];
  const bool has_surface = !C->diffusion && (A > 0.0 || Bs > 0.0);

  // moment set of internal layer l: pointer, effective count, delta-M fraction
  auto moments = [&](int l, int& nuse, double& f) -> const double* {
    const int u = from_bottom ? nL - 1 - l : l;
    const double* chi = chi_base + (layout == 0 ? (size_t)u * M
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
  if (layout == 1) {  // one moment set per wavenumber: phase matrices once
    int nuse;
    double f;
    const double* chi = moments(0, nuse, f);
    build_phase<Gm>(X.goff, t, X.bar, chi, nuse, f, N, C->quad.pl, solar, mu0, Ppp, Ppm);
  }

  // ---------------- bottom composite: surface, or the lower boundary intensity
  int cs = 0;
  {
    const double* mu = X.DV(D_MU);
    const double* wt = X.DV(D_WT);
    double dB = 0.0;
    if (C->diffusion) {
      const double dt = lvTau[nL - 1];
      dB = (dt > 0.0) ? (lvB[nL] - lvB[nL - 1]) / dt : 0.0;
    }
    Real* rp = recs + (size_t)nL * SLay::REC;
    const Tile<Gm> tl(t);
    if (tl.valid()) {
      Real* p = rp + 2 * TILE + t * Gm::TE;
#pragma unroll
      for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) {
          const int r = tl.row(a), c = tl.col(b);
          double v = 0.0;
          if (has_surface && r < N && c < N) v = 2.0 * A * mu[c] * wt[c] * C->quad.xfac;
          p[a * TC + b] = static_cast<Real>(v);
        }
    }
    if (X.warp == 0 && X.lane < NP) {
      const int i = X.lane;
      double u = 0.0;
      if (i < N) {
        if (has_surface) {
          u = (1.0 - A) * Bs;
          if (solar && A > 0.0) u = u + (A / kPi) * F0 * mu0 * exp(-lvTc[nL] / mu0);
        } else if (C->diffusion) {
          u = lvB[nL] + mu[i] * dB;
        } else {
          u = Bs;
        }
      }
      X.V(V_UB)[i] = static_cast<Real>(u);
      rp[3 * TILE + NP + i] = static_cast<Real>(u);
    }
    cs = (has_surface && A > 0.0) ? 1 : 0;
    if (t == 0) rp[3 * TILE + 2 * NP + 1] = Real(cs);
  }

  // ---------------- upward: doubling + adding onto the composite below
  int singular = 0;
  for (int l = nL - 1; l >= 0; --l) {
    const double tau = lvTau[l], om = lvOm[l];
    const double Bt = lvB[l], Bb = lvB[l + 1];
    const int scat = (tau > 0.0 && om > 0.0);
    Real* rp = recs + (size_t)l * SLay::REC;
    Real* rb_below = recs + (size_t)(l + 1) * SLay::REC + 2 * TILE;
    X.sync();
    int tcur = 2;
    if (!scat) {
      // transparent (tau <= 0) or pure absorption (src/doubling.hpp:49-77)
      if (X.warp == 0 && X.lane < NP) {
        const int i = X.lane;
        double tv = 1.0, up = 0.0, dn = 0.0;
        if (i < N && tau > 0.0) {
          const double mui = X.DV(D_MU)[i];
          const double Bbar = (Bb + Bt) / 2.0;
          const double Bd = (Bb - Bt) / tau;
          const double tex = -tau / mui;
          tv = (tex > -200.0) ? exp(tex) : 0.0;
          const double omt = 1.0 - tv;
          const double slope = mui * omt - 0.5 * tau * (1.0 + tv);
          up = Bbar * omt + Bd * slope;
          dn = Bbar * omt - Bd * slope;
        }
        X.V(V_T)[i] = static_cast<Real>(tv);
        X.V(V_SUP)[i] = static_cast<Real>(up);
        X.V(V_SDN)[i] = static_cast<Real>(dn);
      }
      X.sync();
      const Tile<Gm> tl(t);
      if (tl.valid()) {  // record R = 0, T = diag(t)
        Real* pR = rp + t * Gm::TE;
        Real* pT = rp + TILE + t * Gm::TE;
#pragma unroll
        for (int a = 0; a < TR; ++a)
#pragma unroll
          for (int b = 0; b < TC; ++b) {
            pR[a * TC + b] = Real(0);
            pT[a * TC + b] = (tl.row(a) == tl.col(b)) ? X.V(V_T)[tl.row(a)] : Real(0);
          }
      }
    } else {
      if (layout != 1) {
        int nuse;
        double f;
        const double* chi = moments(l, nuse, f);
        build_phase<Gm>(X.goff, t, X.bar, chi, nuse, f, N, C->quad.pl, solar, mu0, Ppp, Ppm);
      }
      tcur = doubling<Gm>(X.goff, t, X.bar, tau, om, Bt, Bb, lvTc[l], N, solar, F0, mu0, Ppp, Ppm,
                          &singular);
      X.sync();
      op_s2g<Gm>(X.mo(0), rp, t);
      op_s2g<Gm>(X.mo(tcur), rp + TILE, t);
    }
    if (X.warp == 0 && X.lane < NP) rp[3 * TILE + X.lane] = X.V(V_SDN)[X.lane];
    if (t == 0) rp[3 * TILE + 2 * NP] = Real(scat);

    // adding: top = this layer, bottom = composite (src/adding.hpp:478-490)
    const unsigned oTl = X.mo(tcur);       // layer T (row-major)
    const unsigned oSp = X.mo(tcur ^ 1);   // spare matrix
    Real* Rtm = sp<Real>(oTl);
    if (!scat) {
      // non-scattering top (src/adding.hpp:349-406):
      // R_b <- t R_b t, U_b <- s_up + t (U_b + R_b s_dn)
      op_g2s<Gm>(rb_below, kNoMat, X.mo(4), t);
      X.sync();
      if (X.warp == 0) {
        const Real* vv[1] = {X.V(V_SDN)};
        Real yv[1];
        matvec<Gm, true, 1>(X.m(4), vv, yv, X.lane);
        if (X.lane < NP) {
          const int i = X.lane;
          X.V(V_UB)[i] = X.V(V_SUP)[i] + X.V(V_T)[i] * (X.V(V_UB)[i] + yv[0]);
        }
      }
      const Tile<Gm> tl(t);
      if (tl.valid()) {
        const Real* src = rb_below + t * Gm::TE;
        Real* dst = rp + 2 * TILE + t * Gm::TE;
#pragma unroll
        for (int a = 0; a < TR; ++a)
#pragma unroll
          for (int b = 0; b < TC; ++b)
            dst[a * TC + b] = X.V(V_T)[tl.row(a)] * src[a * TC + b] * X.V(V_T)[tl.col(b)];
      }
    } else if (!cs) {
      // non-scattering bottom (src/adding.hpp:413-471): R_b <- R, U_b <- s_up + T U_b
      if (X.warp == 0) {
        const Real* vv[1] = {X.V(V_UB)};
        Real yv[1];
        matvec<Gm, false, 1>(Rtm, vv, yv, X.lane);
        __syncwarp();
        if (X.lane < NP) X.V(V_UB)[X.lane] = X.V(V_SUP)[X.lane] + yv[0];
      }
      op_s2g<Gm>(X.mo(0), rp + 2 * TILE, t);
      cs = 1;
    } else {
      // general (src/adding.hpp:301-342): A1 = I - R_b R, D1 = T A1^{-1},
      // U_b <- s_up + D1 (U_b + R_b s_dn), R_b <- R + (D1 R_b) T
      op_g2s<Gm>(rb_below, X.mo(5), X.mo(4), t);  // R_b row-major (m5), column-major (m4)
      X.sync();
      if (X.warp == 0) {
        const Real* vv[1] = {X.V(V_SDN)};
        Real yv[1];
        matvec<Gm, true, 1>(X.m(4), vv, yv, X.lane);
        if (X.lane < NP) X.V(V_TMP)[X.lane] = X.V(V_UB)[X.lane] + yv[0];
      }
      op_gemm<Gm>(X.mo(4), X.mo(0), kNoMat, 1, oSp, kNoMat, t);  // A1
      X.sync();
      singular |= op_gj<Gm>(oSp, oTl, kNoMat, X.mo(1), X.gjo(), X.redo(), t, X.bar);  // D1 (cm)
      X.sync();
      if (X.warp == 0) {
        const Real* vv[1] = {X.V(V_TMP)};
        Real yv[1];
        matvec<Gm, true, 1>(X.m(1), vv, yv, X.lane);
        if (X.lane < NP) X.V(V_UB)[X.lane] = X.V(V_SUP)[X.lane] + yv[0];
      }
      op_gemm<Gm>(X.mo(1), X.mo(5), kNoMat, 0, kNoMat, oSp, t);  // D1 R_b (cm)
      X.sync();
      op_gemm<Gm>(oSp, oTl, X.mo(0), 0, X.mo(4), kNoMat, t);  // R + (D1 R_b) T
      op_s2g<Gm>(X.mo(4), rp + 2 * TILE, t);
    }
    if (X.warp == 0) {
      __syncwarp();
      if (X.lane < NP) rp[3 * TILE + NP + X.lane] = X.V(V_UB)[X.lane];
    }
    if (t == 0) rp[3 * TILE + 2 * NP + 1] = Real(cs);
  }

  // ---------------- downward pass and interface fluxes
  X.sync();
  op_g2s<Gm>(recs + 2 * TILE, kNoMat, X.mo(0), t);  // R_base at the TOA (column-major)
  X.sync();
  if (X.warp == 0) {
    if (X.lane < NP) X.V(V_ID)[X.lane] = (X.lane < N) ? static_cast<Real>(Btop) : Real(0);
    __syncwarp();
    const Real* vv[1] = {X.V(V_ID)};
    Real yv[1];
    matvec<Gm, true, 1>(X.m(0), vv, yv, X.lane);
    if (X.lane < NP) X.V(V_IU)[X.lane] = yv[0] + X.V(V_UB)[X.lane];
    __syncwarp();
    if (X.lane == 0) emit_interface<Gm>(X, C, w, 0, N, solar, F0, mu0, lvTc, lvOmu, lvB, status);
  }
  for (int l = 0; l < nL; ++l) {
    const Real* rl = recs + (size_t)l * SLay::REC;
    const Real* rb = recs + (size_t)(l + 1) * SLay::REC;
    const int scat = rl[3 * TILE + 2 * NP] != Real(0);
    const int cbase = rb[3 * TILE + 2 * NP + 1] != Real(0);
    X.sync();
    op_g2s<Gm>(rl + TILE, kNoMat, X.mo(0), t);      // T (cm)
    op_g2s<Gm>(rl, kNoMat, X.mo(1), t);             // R (cm)
    op_g2s<Gm>(rb + 2 * TILE, X.mo(2), kNoMat, t);  // R_base (rm)
    if (X.warp == 0 && X.lane < NP) {
      X.V(V_UB)[X.lane] = rb[3 * TILE + NP + X.lane];
      X.V(V_SDN)[X.lane] = rl[3 * TILE + X.lane];
    }
    X.sync();
    // rhs = T I_dn + R U_base + s_dn
    if (X.warp == 0) {
      const Real* v0[1] = {X.V(V_ID)};
      const Real* v1[1] = {X.V(V_UB)};
      Real a0[1], a1[1];
      matvec<Gm, true, 1>(X.m(0), v0, a0, X.lane);
      matvec<Gm, true, 1>(X.m(1), v1, a1, X.lane);
      if (X.lane < NP) X.V(V_RHS)[X.lane] = (a0[0] + a1[0]) + X.V(V_SDN)[X.lane];
    }
    X.sync();
    const Real* xsol = X.V(V_RHS);
    int xstride = 1;
    if (scat && cbase) {
      // (I - R R_base) x = rhs, as x^T = rhs^T (I - R R_base)^{-T}
      op_gemm<Gm>(X.mo(2), X.mo(1), kNoMat, 1, X.mo(3), kNoMat, t);  // (I - R R_base)^T
      X.sync();
      singular |= op_gj<Gm>(X.mo(3), kNoMat, X.vo(V_RHS), X.mo(4), X.gjo(), X.redo(), t, X.bar);
      X.sync();
      xsol = X.m(4);
      xstride = LD;
    }
    if (X.warp == 0) {
      if (X.lane < NP) X.V(V_X)[X.lane] = xsol[X.lane * xstride];
      __syncwarp();
      const Real* vv[1] = {X.V(V_X)};
      Real yv[1];
      matvec<Gm, false, 1>(X.m(2), vv, yv, X.lane);
      __syncwarp();
      if (X.lane < NP) {
        X.V(V_ID)[X.lane] = X.V(V_X)[X.lane];
        X.V(V_IU)[X.lane] = yv[0] + X.V(V_UB)[X.lane];
      }
      __syncwarp();
      if (X.lane == 0)
        emit_interface<Gm>(X, C, w, l + 1, N, solar, F0, mu0, lvTc, lvOmu, lvB, status);
    }
  }
  if (singular && t == 0) atomicOr(status, 1u);
  X.sync();
}

// ------------------------------------------------------------- persistent kernel
template <int NP, typename Real>
__global__ void __launch_bounds__(128) solve_kernel(SolveParams P, ColumnDev col0) {
  using Gm = Geo<NP, Real>;
  constexpr int G = Gm::G;
  const int gib = threadIdx.x / G;
  const int t = threadIdx.x % G;
  const unsigned goff = (unsigned)(gib * SmemLayout<Gm>::bytes);
  const int slot = blockIdx.x * (blockDim.x / G) + gib;
  char* sl = P.scratch + (size_t)slot * P.slot_bytes;
  const Ctx<Gm> X(goff, t, 1 + gib);
  for (int i = t; i < 6 * Gm::DIM + 4; i += G) X.gjbuf[i] = Real(0);
  if (P.ncols <= 1 && t == 0) *X.col = col0;
  long long* task_s = sp<long long>(goff + SmemLayout<Gm>::misc + 48);
  int cur_col = -1;
  for (;;) {
    long long task;
    if constexpr (G == 32) {
      unsigned long long v = 0;
      if (t == 0) v = atomicAdd(P.counter, 1ull);
      task = (long long)__shfl_sync(0xffffffffu, v, 0);
    } else {
      gsync<G>(1 + gib);
      if (t == 0) *task_s = (long long)atomicAdd(P.counter, 1ull);
      gsync<G>(1 + gib);
      task = *task_s;
    }
    if (task >= P.ntasks) break;
    int w = (int)task;
    if (P.ncols > 1) {
      int lo = 0, hi = P.ncols - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (P.cols[mid].task_begin <= task) lo = mid; else hi = mid - 1;
      }
      if (lo != cur_col) {
        gsync<G>(1 + gib);
        if (t == 0) *X.col = P.cols[lo];
        cur_col = lo;
      }
      w = (int)(task - P.cols[lo].task_begin);
    }
    gsync<G>(1 + gib);
    solve_one<Gm>(goff, t, 1 + gib, w, sl, P.max_layers, P.status);
  }
}

}  // namespace adrt_dev
