// adrt_kernel.cuh -- per-wavenumber solve and the persistent batch kernel.
#pragma once

#include "adrt_solver.cuh"

namespace adrt_dev {

// Per-slot HBM scratch of one thread group: level scalars, then one record
// per layer (layer R, T, s_down and the composite R_base, U_base below the
// layer's top interface) for the downward pass.
template <class Gm>
struct SlotLayout {
  using Real = typename Gm::Real;
  static constexpr int TILE = Gm::G * Gm::TE;  // Reals per matrix in tile order
  static constexpr int REC_RAW = 3 * TILE + 2 * Gm::NP + 2;
  static constexpr int RALIGN = 16 / (int)sizeof(Real);
  static constexpr int REC = (REC_RAW + RALIGN - 1) / RALIGN * RALIGN;
  static __host__ __device__ size_t level_bytes(int lmax) {
    return ((size_t)5 * (lmax + 1) * sizeof(double) + 255) & ~size_t(255);
  }
  static __host__ __device__ size_t bytes(int lmax) {
    return level_bytes(lmax) + (size_t)(lmax + 1) * REC * sizeof(Real);
  }
};

template <class Gm>
struct Ctx {
  using Real = typename Gm::Real;
  using SL = SmemLayout<Gm>;
  static constexpr int NP = Gm::NP, LD = Gm::LD, MAT = Gm::MAT;
  TileOps<Gm> ops;
  int lane, warp;
  Real *m0, *m1, *m2, *m3, *gjbuf, *vec;
  double *Ppp, *Ppm, *dvec, *dmisc;
  unsigned* red;
  __device__ Ctx(char* smem, int t, int bar) : ops(t, bar) {
    lane = t & 31;
    warp = t >> 5;
    m0 = reinterpret_cast<Real*>(smem + SL::mats);
    m1 = m0 + MAT;
    m2 = m1 + MAT;
    m3 = m2 + MAT;
    gjbuf = reinterpret_cast<Real*>(smem + SL::gj);
    vec = reinterpret_cast<Real*>(smem + SL::vecs);
    Ppp = reinterpret_cast<double*>(smem + SL::dmats);
    Ppm = Ppp + NP * NP;
    dvec = reinterpret_cast<double*>(smem + SL::dvecs);
    red = reinterpret_cast<unsigned*>(smem + SL::misc);
    dmisc = reinterpret_cast<double*>(smem + SL::misc + 32);
  }
  __device__ __forceinline__ Real* V(int s) const { return vec + s * NP; }
  __device__ __forceinline__ double* DV(int s) const { return dvec + s * NP; }
};

// ------------------------------------------------------------- phase matrices
// P++/P+- from Legendre moments with Hansen column renormalisation
// (src/phase_matrix.hpp:61-111) and, with a solar beam, the phase vectors at
// mu0 (src/phase_matrix.hpp:131-181).  chi_l is (chi[l] - f) / (1 - f) when
// delta-M truncation applies (f >= 0), chi[l] otherwise.
template <class Gm>
__device__ void build_phase(const Ctx<Gm>& X, const double* chi, int nuse, double f, int N,
                            const QuadDev& q, bool solar, double mu0) {
  constexpr int NP = Gm::NP, TR = Gm::TR, TC = Gm::TC;
  const auto& o = X.ops;
  const double inv_1mf = (f >= 0.0) ? 1.0 / (1.0 - f) : 1.0;
#pragma unroll
  for (int a = 0; a < TR; ++a)
#pragma unroll
    for (int b = 0; b < TC; ++b) {
      const int r = o.row(a), c = o.col(b);
      if (r < NP && c < NP) {
        double spp = 0.0, spm = 0.0;
        if (r < N && c < N) {
          double sign = 1.0;
          for (int l = 0; l < nuse; ++l) {
            const double cl = (f >= 0.0) ? (chi[l] - f) * inv_1mf : chi[l];
            const double term = (2 * l + 1) * cl * q.pl[l * N + r] * q.pl[l * N + c];
            spp += term;
            spm += sign * term;
            sign = -sign;
          }
          spp /= (2.0 * kPi);
          spm /= (2.0 * kPi);
        }
        X.Ppp[r * NP + c] = spp;
        X.Ppm[r * NP + c] = spm;
      }
    }
  o.sync();
  const int t = o.t;
  if (t < N) {
    const int c = t;
    double sum = 0.0;
    for (int i = 0; i < N; ++i) sum += (X.Ppp[i * NP + c] + X.Ppm[i * NP + c]) * q.wt[i];
    if (sum > 0.0) {
      const double corr = 1.0 / (2.0 * kPi * sum);
      for (int i = 0; i < N; ++i) {
        X.Ppp[i * NP + c] *= corr;
        X.Ppm[i * NP + c] *= corr;
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
          if (l == 0)
            plm = 1.0;
          else if (l == 1)
            plm = mu0;
          else {
            plm = ((2 * l - 1) * mu0 * p1 - (l - 1) * p0) / l;
            p0 = p1;
            p1 = plm;
          }
          const double cl = (f >= 0.0) ? (chi[l] - f) * inv_1mf : chi[l];
          const double term = (2 * l + 1) * cl * q.pl[l * N + t] * plm;
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
    o.sync();
    double corr = 1.0;
    {
      double sum = 0.0;
      for (int i = 0; i < N; ++i) sum += (pp[i] + pm[i]) * q.wt[i];
      if (sum > 0.0) corr = 1.0 / (2.0 * kPi * sum);
    }
    o.sync();
    if (t < N) {
      pp[t] *= corr;
      pm[t] *= corr;
    }
  }
  o.sync();
}

// ------------------------------------------------------------- doubling
// One homogeneous scattering layer (src/doubling.hpp:79-229): first-order
// thin-layer start at tau0 = tau 2^-nn, then nn doublings of R, T and of the
// thermal (y, z) and solar sources.  Leaves R, T in the tiles and the
// combined thermal + solar sources in V_SUP / V_SDN.
template <class Gm>
__device__ int doubling(const Ctx<Gm>& X, double tau, double om, double Bt, double Bb,
                        double tcum, int N, const QuadDev& q, bool solar, double F0, double mu0,
                        typename TileOps<Gm>::Tile& R, typename TileOps<Gm>::Tile& T) {
  using Real = typename Gm::Real;
  constexpr int NP = Gm::NP, TR = Gm::TR, TC = Gm::TC;
  const auto& o = X.ops;
  om = om > 1.0 ? 1.0 : om;
  const double con = 2.0 * om * kPi;
  const int nn = num_doublings(tau, om);
  const double tau0 = ldexp(tau, -nn);
  const double Ftop = solar ? F0 * exp(-tcum / mu0) : 0.0;
  // thin-layer start (FP64)
#pragma unroll
  for (int a = 0; a < TR; ++a)
#pragma unroll
    for (int b = 0; b < TC; ++b) {
      const int r = o.row(a), c = o.col(b);
      double tv = (r == c) ? 1.0 : 0.0, rv = 0.0;
      if (r < N && c < N) {
        const double pppc = X.Ppp[r * NP + c] * q.wt[c];
        const double temp = ((r == c) ? 1.0 : 0.0) + (-con) * pppc;
        const double gpp = temp / q.mu[r];
        tv = ((r == c) ? 1.0 : 0.0) - tau0 * gpp;
        const double gpm = con * (X.Ppm[r * NP + c] * q.wt[c]) / q.mu[r];
        rv = tau0 * gpm;
      }
      T[a][b] = static_cast<Real>(tv);
      R[a][b] = static_cast<Real>(rv);
    }
  if (X.warp == 0 && X.lane < NP) {
    const int i = X.lane;
    double y = 0.0, su = 0.0, sd = 0.0;
    if (i < N) {
      y = (1.0 - om) * tau0 / q.mu[i];
      if (solar) {
        const double base = om * tau0 / q.mu[i] * Ftop;
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
  int singular = 0;
  for (int k = 0; k < nn; ++k) {
    const int par = k & 1;
    Real* y = X.V(V_Y0 + par);
    Real* z = X.V(V_Z0 + par);
    Real* su = X.V(V_SU0 + par);
    Real* sd = X.V(V_SD0 + par);
    Real* yn = X.V(V_Y0 + 1 - par);
    Real* zn = X.V(V_Z0 + 1 - par);
    Real* sun = X.V(V_SU0 + 1 - par);
    Real* sdn = X.V(V_SD0 + 1 - par);
    o.sync();  // previous readers of m0..m3 are done
    o.stage_rm(R, X.m0);
    o.stage_cm(R, X.m1);
    o.stage_rm(T, X.m2);
    o.sync();
    if (solar && X.warp == 0) {  // ru = R sd + gam su, rd = gam R su + sd
      const Real* vv[2] = {sd, su};
      Real yv[2];
      matvec_cm<Gm, 2>(X.m1, vv, yv, X.lane);
      if (X.lane < NP) {
        X.V(V_RU)[X.lane] = yv[0] + gam * su[X.lane];
        X.V(V_RD)[X.lane] = gam * yv[1] + sd[X.lane];
      }
    }
    typename TileOps<Gm>::Tile Am, Bm;
    o.template gemm<false>(Am, X.m1, X.m0);  // R R
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) Am[a][b] = ((o.row(a) == o.col(b)) ? Real(1) : Real(0)) - Am[a][b];
    o.copy(Bm, T);
    singular |= o.gj_right_solve(Am, Bm, X.m3, X.gjbuf, X.red);  // TG = T (I - R^2)^{-1}
    o.sync();
    o.template gemm<false>(Am, X.m3, X.m0);  // TGR = TG R
    o.stage_cm(Am, X.m1);
    o.sync();
    o.template gemm<true>(R, X.m1, X.m2);  // R + TGR T
    o.template gemm<false>(T, X.m3, X.m2);  // TG T
    if (X.warp == 0) {
      if (X.lane < NP) X.V(V_TMP)[X.lane] = z[X.lane] + g * y[X.lane];
      __syncwarp();
      const Real* va[2] = {X.V(V_TMP), y};
      Real tg[2], tgr[2];
      matvec_cm<Gm, 2>(X.m3, va, tg, X.lane);
      matvec_cm<Gm, 2>(X.m1, va, tgr, X.lane);
      Real tu[2] = {Real(0), Real(0)};
      if (solar) {
        const Real* vs[2] = {X.V(V_RU), X.V(V_RD)};
        matvec_cm<Gm, 2>(X.m3, vs, tu, X.lane);
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
  }
  o.sync();
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
  return singular;
}

// ------------------------------------------------------------- one wavenumber
template <class Gm>
__device__ void solve_one(const ColumnDev& C, int w, char* slot, int lmax, const Ctx<Gm>& X,
                          unsigned* status) {
  using Real = typename Gm::Real;
  using Tile = typename TileOps<Gm>::Tile;
  using SLay = SlotLayout<Gm>;
  constexpr int NP = Gm::NP, G = Gm::G, TR = Gm::TR, TC = Gm::TC, LD = Gm::LD;
  const auto& o = X.ops;
  const int t = o.t;
  const int N = C.N, nL = C.L, M = C.M;
  const QuadDev& q = C.quad;

  const double A = C.albedo_w ? C.albedo_w[w] : C.surface_albedo;
  const double mu0 = C.mu0_w ? C.mu0_w[w] : C.solar_mu;
  const double wlo = C.wlo_w ? C.wlo_w[w] : C.wn_lo;
  const double whi = C.whi_w ? C.whi_w[w] : C.wn_hi;
  const double semis = C.semis_w ? C.semis_w[w] : C.surface_emission;
  const double temis = C.temis_w ? C.temis_w[w] : C.top_emission;
  const double F0 = C.solar_flux;
  const bool solar = (F0 > 0.0 && mu0 > 0.0);

  double* lvB = reinterpret_cast<double*>(slot);
  double* lvTc = lvB + (lmax + 1);
  double* lvTau = lvTc + (lmax + 1);
  double* lvOm = lvTau + (lmax + 1);
  double* lvOmu = lvOm + (lmax + 1);
  Real* recs = reinterpret_cast<Real*>(slot + SLay::level_bytes(lmax));
  auto rec = [&](int l) { return recs + (size_t)l * SLay::REC; };
  constexpr int TILE = SLay::TILE;

  auto src_layer = [&](int l) { return C.from_bottom ? nL - 1 - l : l; };
  auto src_level = [&](int l) { return C.from_bottom ? nL - l : l; };
  auto chi_of = [&](int l) -> const double* {
    const int u = src_layer(l);
    if (C.moment_layout == 0) return C.moments + (size_t)u * M;
    if (C.moment_layout == 1) return C.moments + (size_t)w * M;
    return C.moments + ((size_t)w * nL + u) * M;
  };

  // ---------------- prologue: Planck levels, scaled optical properties
  unsigned bad = 0;
  for (int l = t; l <= nL; l += G) {
    double Bv = 0.0;
    if (C.thermal) {
      const double* Tl = C.temperature + (C.temp_per_wav ? (size_t)w * (nL + 1) : 0);
      const double Tv = Tl[src_level(l)];
      if (Tv < 0.0) bad = 1;
      Bv = planck_band(wlo, whi, Tv);
    } else if (C.planck) {
      Bv = C.planck[(size_t)w * (nL + 1) + src_level(l)];
    }
    lvB[l] = Bv;
  }
  for (int l = t; l < nL; l += G) {
    const int u = src_layer(l);
    double tau = C.dtau[(size_t)w * nL + u];
    double om = C.ssa[(size_t)w * nL + u];
    if (!(tau >= 0.0 && tau < 1e300) || !(om >= 0.0 && om <= 1.0)) bad = 1;
    lvOmu[l] = om;
    if (om > 0.0 && tau > 0.0 && C.delta_m && M > 2 * N) {
      const double f = chi_of(l)[2 * N];
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
  o.sync();
  if (t == 0) {
    double tc = 0.0;
    lvTc[0] = 0.0;
    for (int l = 0; l < nL; ++l) {
      tc += lvTau[l];
      lvTc[l + 1] = tc;
    }
    double Bs, Btop;
    if (C.thermal) {
      Bs = (C.surface_temperature >= 0.0) ? planck_band(wlo, whi, C.surface_temperature) : lvB[nL];
      Btop = (C.top_temperature >= 0.0) ? planck_band(wlo, whi, C.top_temperature) : lvB[0];
    } else {
      Bs = semis;
      Btop = temis;
    }
    X.dmisc[0] = Bs;
    X.dmisc[1] = Btop;
  }
  o.sync();
  const double Bs = X.dmisc[0], Btop = X.dmisc[1];
  const bool has_surface = !C.diffusion && (A > 0.0 || Bs > 0.0);

  // moment set of a layer: effective count and delta-M fraction
  auto moment_setup = [&](int l, int& nuse, double& f) {
    const double* chi = chi_of(l);
    nuse = M;
    f = -1.0;
    if (C.delta_m) {
      const double ff = (M > 2 * N) ? chi[2 * N] : 0.0;
      if (ff > 1e-12 && ff < 1.0 - 1e-12) {
        f = ff;
        nuse = 2 * N;
      } else {
        nuse = (M < 2 * N) ? M : 2 * N;
      }
    }
  };
  if (C.moment_layout == 1) {  // one moment set per wavenumber: phase matrices once
    int nuse;
    double f;
    moment_setup(0, nuse, f);
    build_phase<Gm>(X, chi_of(0), nuse, f, N, q, solar, mu0);
  }

  // ---------------- bottom composite: surface or the lower boundary intensity
  Tile Rb;
  int cs = 0;
  {
    double dB = 0.0;
    if (C.diffusion) {
      const double dt = lvTau[nL - 1];
      dB = (dt > 0.0) ? (lvB[nL] - lvB[nL - 1]) / dt : 0.0;
    }
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) {
        const int r = o.row(a), c = o.col(b);
        double v = 0.0;
        if (has_surface && r < N && c < N) v = 2.0 * A * q.mu[c] * q.wt[c] * q.xfac;
        Rb[a][b] = static_cast<Real>(v);
      }
    if (X.warp == 0 && X.lane < NP) {
      const int i = X.lane;
      double u = 0.0;
      if (i < N) {
        if (has_surface) {
          u = (1.0 - A) * Bs;
          if (solar && A > 0.0) u = u + (A / kPi) * F0 * mu0 * exp(-lvTc[nL] / mu0);
        } else if (C.diffusion) {
          u = lvB[nL] + q.mu[i] * dB;
        } else {
          u = Bs;
        }
      }
      X.V(V_UB)[i] = static_cast<Real>(u);
      X.DV(D_IBOT)[i] = u;
    }
    cs = (has_surface && A > 0.0) ? 1 : 0;
    Real* rp = rec(nL);
    o.store_g(Rb, rp + 2 * TILE);
    __syncwarp();
    if (X.warp == 0 && X.lane < NP) rp[3 * TILE + NP + X.lane] = X.V(V_UB)[X.lane];
    if (t == 0) rp[3 * TILE + 2 * NP + 1] = Real(cs);
  }

  // ---------------- upward: doubling + adding onto the composite below
  int singular = 0;
  for (int l = nL - 1; l >= 0; --l) {
    const double tau = lvTau[l], om = lvOm[l];
    const double Bt = lvB[l], Bb = lvB[l + 1];
    const int scat = (tau > 0.0 && om > 0.0);
    Tile R, T;
    o.sync();
    if (!scat) {
      // transparent (tau <= 0) or pure absorption (src/doubling.hpp:49-77)
      if (X.warp == 0 && X.lane < NP) {
        const int i = X.lane;
        double tv = 1.0, up = 0.0, dn = 0.0;
        if (i < N && tau > 0.0) {
          const double Bbar = (Bb + Bt) / 2.0;
          const double Bd = (Bb - Bt) / tau;
          const double tex = -tau / q.mu[i];
          tv = (tex > -200.0) ? exp(tex) : 0.0;
          const double omt = 1.0 - tv;
          const double slope = q.mu[i] * omt - 0.5 * tau * (1.0 + tv);
          up = Bbar * omt + Bd * slope;
          dn = Bbar * omt - Bd * slope;
        }
        X.V(V_T)[i] = static_cast<Real>(tv);
        X.V(V_SUP)[i] = static_cast<Real>(up);
        X.V(V_SDN)[i] = static_cast<Real>(dn);
      }
      o.sync();
#pragma unroll
      for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) {
          const int r = o.row(a), c = o.col(b);
          R[a][b] = Real(0);
          T[a][b] = (r == c && r < NP) ? X.V(V_T)[r] : Real(0);
        }
    } else {
      if (C.moment_layout != 1) {
        int nuse;
        double f;
        moment_setup(l, nuse, f);
        build_phase<Gm>(X, chi_of(l), nuse, f, N, q, solar, mu0);
      }
      singular |= doubling<Gm>(X, tau, om, Bt, Bb, lvTc[l], N, q, solar, F0, mu0, R, T);
    }
    // layer record for the downward pass
    Real* rp = rec(l);
    o.store_g(R, rp);
    o.store_g(T, rp + TILE);
    o.sync();
    if (X.warp == 0 && X.lane < NP) rp[3 * TILE + X.lane] = X.V(V_SDN)[X.lane];
    if (t == 0) rp[3 * TILE + 2 * NP] = Real(scat);

    // adding: top = this layer, bottom = composite (src/adding.hpp:478-490)
    if (!scat) {
      // non-scattering top (src/adding.hpp:349-406): R_b <- t R_b t,
      // U_b <- s_up + t (U_b + R_b s_dn)
      o.stage_cm(Rb, X.m0);
      o.sync();
      if (X.warp == 0) {
        const Real* vv[1] = {X.V(V_SDN)};
        Real yv[1];
        matvec_cm<Gm, 1>(X.m0, vv, yv, X.lane);
        if (X.lane < NP) {
          const int i = X.lane;
          X.V(V_UB)[i] = X.V(V_SUP)[i] + X.V(V_T)[i] * (X.V(V_UB)[i] + yv[0]);
        }
      }
#pragma unroll
      for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) {
          const int r = o.row(a), c = o.col(b);
          if (r < NP && c < NP) Rb[a][b] = X.V(V_T)[r] * Rb[a][b] * X.V(V_T)[c];
        }
    } else if (!cs) {
      // non-scattering bottom (src/adding.hpp:413-471): R_b <- R, U_b <- s_up + T U_b
      o.stage_cm(T, X.m0);
      o.sync();
      if (X.warp == 0) {
        const Real* vv[1] = {X.V(V_UB)};
        Real yv[1];
        matvec_cm<Gm, 1>(X.m0, vv, yv, X.lane);
        __syncwarp();
        if (X.lane < NP) X.V(V_UB)[X.lane] = X.V(V_SUP)[X.lane] + yv[0];
      }
      o.copy(Rb, R);
      cs = 1;
    } else {
      // general (src/adding.hpp:301-342): A1 = I - R_b R, D1 = T A1^{-1},
      // U_b <- s_up + D1 (U_b + R_b s_dn), R_b <- R + (D1 R_b) T
      o.stage_cm(Rb, X.m0);
      o.stage_rm(R, X.m1);
      o.stage_rm(T, X.m2);
      o.sync();
      if (X.warp == 0) {
        const Real* vv[1] = {X.V(V_SDN)};
        Real yv[1];
        matvec_cm<Gm, 1>(X.m0, vv, yv, X.lane);
        if (X.lane < NP) X.V(V_TMP)[X.lane] = X.V(V_UB)[X.lane] + yv[0];
      }
      Tile Am, Bm;
      o.template gemm<false>(Am, X.m0, X.m1);
#pragma unroll
      for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) Am[a][b] = ((o.row(a) == o.col(b)) ? Real(1) : Real(0)) - Am[a][b];
      o.sync();
      o.stage_rm(Rb, X.m1);
      o.copy(Bm, T);
      singular |= o.gj_right_solve(Am, Bm, X.m3, X.gjbuf, X.red);
      o.sync();
      if (X.warp == 0) {
        const Real* vv[1] = {X.V(V_TMP)};
        Real yv[1];
        matvec_cm<Gm, 1>(X.m3, vv, yv, X.lane);
        if (X.lane < NP) X.V(V_UB)[X.lane] = X.V(V_SUP)[X.lane] + yv[0];
      }
      o.template gemm<false>(Am, X.m3, X.m1);  // D1 R_b
      o.stage_cm(Am, X.m0);
      o.sync();
      o.copy(Rb, R);
      o.template gemm<true>(Rb, X.m0, X.m2);  // R + (D1 R_b) T
    }
    o.store_g(Rb, rp + 2 * TILE);
    o.sync();
    if (X.warp == 0 && X.lane < NP) rp[3 * TILE + NP + X.lane] = X.V(V_UB)[X.lane];
    if (t == 0) rp[3 * TILE + 2 * NP + 1] = Real(cs);
  }

  // ---------------- downward pass and interface fluxes
  const size_t ob = (size_t)w * (nL + 1);
  const double inv4pimu0 = solar ? 1.0 / (4.0 * kPi * mu0) : 0.0;
  auto emit = [&](int l) {  // thread 0: reductions of V_IU / V_ID at internal interface l
    double fu = 0.0, fd = 0.0, J = 0.0;
    for (int i = 0; i < N; ++i) {
      const double iu = X.V(V_IU)[i], id = X.V(V_ID)[i];
      const double cw = 2.0 * kPi * q.wt[i] * q.mu[i];
      fu += cw * iu;
      fd += cw * id;
      J += 0.5 * q.wt[i] * (iu + id);
    }
    double fdir = 0.0;
    if (solar) {
      fdir = (l == 0) ? F0 * mu0 : F0 * mu0 * exp(-lvTc[l] / mu0);
      J += fdir * inv4pimu0;
    }
    const int lyr = (l == 0) ? 0 : l - 1;
    const double divF = 4.0 * kPi * (1.0 - lvOmu[lyr]) * (J - lvB[l]);
    const size_t oi = ob + (C.from_bottom ? nL - l : l);
    if (C.fu) C.fu[oi] = fu;
    if (C.fd) C.fd[oi] = fd;
    if (C.fdir) C.fdir[oi] = fdir;
    if (C.J) C.J[oi] = J;
    if (C.divF) C.divF[oi] = divF;
    if (l == 0) {
      if (C.toa_fu) C.toa_fu[w] = fu * C.spectrum_scaling;
      if (C.toa_fd) C.toa_fd[w] = fd;
    }
    if (l == nL && C.boa_fdir) C.boa_fdir[w] = fdir;
    if (!isfinite(fu) || !isfinite(fd) || !isfinite(J)) atomicOr(status, 2u);
  };

  // TOA: I_up = R_base I_top + U_base
  o.sync();
  o.stage_cm(Rb, X.m0);
  o.sync();
  if (X.warp == 0) {
    if (X.lane < NP) X.V(V_ID)[X.lane] = (X.lane < N) ? static_cast<Real>(Btop) : Real(0);
    __syncwarp();
    const Real* vv[1] = {X.V(V_ID)};
    Real yv[1];
    matvec_cm<Gm, 1>(X.m0, vv, yv, X.lane);
    if (X.lane < NP) X.V(V_IU)[X.lane] = yv[0] + X.V(V_UB)[X.lane];
    __syncwarp();
    if (X.lane == 0) emit(0);
  }
  for (int l = 0; l < nL; ++l) {
    const Real* rl = rec(l);
    const Real* rb = rec(l + 1);
    const int scat = rl[3 * TILE + 2 * NP] != Real(0);
    const int cb_ = rb[3 * TILE + 2 * NP + 1] != Real(0);
    Tile R, T, B2;
    o.load_g(R, rl);
    o.load_g(T, rl + TILE);
    o.load_g(B2, rb + 2 * TILE);
    o.sync();
    o.stage_cm(T, X.m0);
    o.stage_cm(R, X.m1);
    o.stage_rm(B2, X.m2);
    if (X.warp == 0 && X.lane < NP) {
      X.V(V_UB)[X.lane] = rb[3 * TILE + NP + X.lane];
      X.V(V_SDN)[X.lane] = rl[3 * TILE + X.lane];
    }
    o.sync();
    // rhs = T I_dn + R U_base + s_dn
    if (X.warp == 0) {
      const Real* v0[1] = {X.V(V_ID)};
      const Real* v1[1] = {X.V(V_UB)};
      Real a0[1], a1[1];
      matvec_cm<Gm, 1>(X.m0, v0, a0, X.lane);
      matvec_cm<Gm, 1>(X.m1, v1, a1, X.lane);
      if (X.lane < NP) X.V(V_RHS)[X.lane] = (a0[0] + a1[0]) + X.V(V_SDN)[X.lane];
    }
    o.sync();
    const Real* xsol = X.V(V_RHS);
    int xstride = 1;
    if (scat && cb_) {
      // (I - R R_base) x = rhs, as x^T = rhs^T (I - R R_base)^{-T}
      Tile Am, Bm;
      o.template gemm<false>(Am, X.m2, X.m1);  // R_base^T R^T = (R R_base)^T
#pragma unroll
      for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) {
          Am[a][b] = ((o.row(a) == o.col(b)) ? Real(1) : Real(0)) - Am[a][b];
          Bm[a][b] = (o.row(a) == 0 && o.col(b) < NP) ? X.V(V_RHS)[o.col(b)] : Real(0);
        }
      singular |= o.gj_right_solve(Am, Bm, X.m3, X.gjbuf, X.red);
      o.sync();
      xsol = X.m3;
      xstride = LD;
    }
    if (X.warp == 0) {
      if (X.lane < NP) X.V(V_X)[X.lane] = xsol[X.lane * xstride];
      __syncwarp();
      const Real* vv[1] = {X.V(V_X)};
      Real yv[1];
      matvec_rm<Gm, 1>(X.m2, vv, yv, X.lane);
      __syncwarp();
      if (X.lane < NP) {
        X.V(V_ID)[X.lane] = X.V(V_X)[X.lane];
        X.V(V_IU)[X.lane] = yv[0] + X.V(V_UB)[X.lane];
      }
      __syncwarp();
      if (X.lane == 0) emit(l + 1);
    }
  }
  if (singular && t == 0) atomicOr(status, 1u);
  o.sync();
}

// ------------------------------------------------------------- persistent kernel
template <int NP, typename Real>
__global__ void __launch_bounds__(128) solve_kernel(SolveParams P, ColumnDev col0) {
  using Gm = Geo<NP, Real>;
  constexpr int G = Gm::G;
  extern __shared__ __align__(16) char smem_raw[];
  const int gib = threadIdx.x / G;
  const int t = threadIdx.x % G;
  char* smem = smem_raw + gib * SmemLayout<Gm>::bytes;
  const int slot = blockIdx.x * (blockDim.x / G) + gib;
  char* sl = P.scratch + (size_t)slot * P.slot_bytes;
  Ctx<Gm> X(smem, t, 1 + gib);
  // zero the Gauss-Jordan buffers once so padded lanes never read garbage
  for (int i = t; i < 6 * Gm::DIM + 4; i += G) X.gjbuf[i] = Real(0);
  long long* task_s = reinterpret_cast<long long*>(smem + SmemLayout<Gm>::misc + 48);
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
    if (P.ncols <= 1) {
      solve_one<Gm>(col0, (int)task, sl, P.max_layers, X, P.status);
    } else {
      int lo = 0, hi = P.ncols - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (P.cols[mid].task_begin <= task) lo = mid; else hi = mid - 1;
      }
      const ColumnDev& C = P.cols[lo];
      solve_one<Gm>(C, (int)(task - C.task_begin), sl, P.max_layers, X, P.status);
    }
  }
}

}  // namespace adrt_dev
