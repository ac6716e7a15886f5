// adrt_kernel.cuh -- per-wavenumber solve and the persistent batch kernel.
//
// Two precision forms share this code:
//
//   FP64    every operation in FP64, the doubling in the reference's own order
//           (T-form: T <- T (I - R^2)^{-1} T, src/doubling.hpp:149-209).
//   MIXED   per wavenumber, one of two classes (decided in the prologue):
//     S     no ill-conditioned layer: every doubling in the FP32 Lambda-split
//           form below, adding and interfaces in FP32;
//     D     at least one ill-conditioned layer: those layers double in FP64
//           (T-form), all others in FP32 Lambda-split form, and the adding,
//           the composites and the interface solves run in FP64.
//   A layer is ill-conditioned for FP32 when its first-order start is
//   unstable (tau0 = tau 2^-nn above half the smallest quadrature cosine, so
//   1 - tau0/mu is near zero or negative and the doubling amplifies
//   round-off), when it is thick and near-conservative (1 - omega < 1e-2 with
//   tau > 1: I - R^2 nearly singular), or when it needs more than 20
//   doublings.
//
// Lambda-split doubling.  Write the layer transmission as T = Lambda + T'
// with Lambda = diag((1 - tau0/mu_i)^(2^k)) (the first-order direct term,
// squared exactly in FP64 at every doubling) and T' >= 0 the diffuse part.
// With A = I - R^2 and G' = TG - Lambda = (Lambda R^2 + T') A^{-1}:
//     TGR = Lambda R + G' R,      R <- R + TGR T,
//     T'  <- G' T + Lambda T',    Lambda <- Lambda^2,   T = Lambda + T'.
// The thermal recurrences (src/doubling.hpp:186-197) are carried in
// a = z + g y >= 0 and b = z - g y <= 0, whose updates
//     a <- TG (2a - b) - TGR b + a,   b <- TG b - TGR (2a - b) + 2b - a
// and the solar ones are sums of same-signed terms, and the layer sources
// follow as s_up = (a B_bot - b B_top)/tau + s_sol_up, s_dn = (a B_top -
// b B_bot)/tau + s_sol_dn.  This is the reference's recurrence rewritten
// exactly (equal in exact arithmetic); its FP32 evaluation keeps every
// entry to FP32 relative accuracy for thin and thick streams alike, where
// the reference-order FP32 evaluation loses (1 - T) for thin layers and the
// small T of thick ones.  The beam factor gamma = exp(-tau0/mu0)^(2^k) is
// squared in FP64.
#pragma once

#include "adrt_solver.cuh"

namespace adrt_dev {

constexpr int kFp64MaxDoublings = 20;           // more doublings -> FP64 layer
constexpr double kFp64StartRatio = 0.5;         // tau0 > ratio * mu_min -> FP64 layer
constexpr double kFp64NearConservative = 1e-2;  // 1 - omega below this ...
constexpr double kFp64ThickTau = 1.0;           // ... with tau above this -> FP64 layer

enum SolveMode { MODE_FP64 = 0, MODE_MIX_S = 1, MODE_MIX_D = 2 };
#ifndef ADRT_MIX_FORCE_D
#define ADRT_MIX_FORCE_D 1  // every mixed wavenumber takes class D (FP64 adding)
#endif
// Scattering depth tau omega above which a layer doubles in FP64 in the mixed
// form.  An FP32 doubling carries about 3e-7 of the largest entry of R and T
// as round-off whatever the precision of its products (the rounding of R, T'
// and the sources at each of the nn steps), so a layer's FP32 error in the
// fluxes scales with its reflection and diffuse transmission, which grow with
// tau omega: only weakly scattering layers double in FP32.
#ifndef ADRT_MIX_SCAT_DEPTH
#define ADRT_MIX_SCAT_DEPTH 0.003
#endif
enum KernelKind { KIND_FP64 = 0, KIND_MIXED = 1 };
constexpr int kLevelArrays = 6;  // B, tau_cum, tau', omega', omega, FP64-layer flag

// Per-slot HBM scratch of one thread group: level scalars, the phase
// matrices of the current moment set, then one record per interface l =
// 0..L (the layer below it: R, T, s_down; the composite of everything below
// it: R_base, U_base) for the downward pass.
template <class Gm>
struct SlotLayout {
  using Real = typename Gm::Real;
  static constexpr int NP = Gm::NP;
  static constexpr int TILE = Gm::G * Gm::TE;  // Reals per matrix in tile order
  // R, T, R_base tiles; s_dn, U_base; scat flag, base-reflects flag; s_up
  static constexpr int REC_RAW = 3 * TILE + 3 * NP + 2;
  static constexpr int RALIGN = 16 / (int)sizeof(Real);
  static constexpr int REC = (REC_RAW + RALIGN - 1) / RALIGN * RALIGN;
  static __host__ __device__ size_t level_bytes(int lmax) {
    return ((size_t)kLevelArrays * (lmax + 1) * sizeof(double) + 255) & ~size_t(255);
  }
  static __host__ __device__ size_t phase_bytes() {
    return ((size_t)2 * NP * NP * sizeof(double) + 255) & ~size_t(255);
  }
  static __host__ __device__ size_t bytes(int lmax) {
    return level_bytes(lmax) + phase_bytes() + (size_t)(lmax + 1) * REC * sizeof(Real);
  }
};

// One step of the adjoint's doubling record (per layer, nn steps): R, T, TG
// tiles (TG taken from its column-major buffer, i.e. TG^T in tile order),
// (I - R^2)^{-1}, then y, z, s_up, s_dn and gamma, and with a solar beam the
// step's r_up = R s_dn + gamma s_up, r_dn = gamma R s_up + s_dn and R s_up
// (unwritten without one).  After the nn steps, a tail holds the final y and
// z of the chain.
template <class Gm>
struct TapeLayout {
  static constexpr int NP = Gm::NP;
  static constexpr int TILE = Gm::G * Gm::TE;
  static constexpr int OFF_R = 0, OFF_T = TILE, OFF_TG = 2 * TILE, OFF_AI = 3 * TILE;
  static constexpr int OFF_VEC = 4 * TILE;  // y, z, s_up, s_dn (NP each), gamma
  static constexpr int OFF_SOL = OFF_VEC + 4 * NP + 2;  // r_up, r_dn, R s_up
  static constexpr int STEP = (OFF_SOL + 3 * NP + 1) / 2 * 2;
  static constexpr int TAIL = 2 * NP;
  static __host__ __device__ long long layer(int nn) { return (long long)nn * STEP + TAIL; }
};


// Shared-memory bytes of one group for a kernel kind: the common prefix and
// one typed region (FP64), or for the mixed kind the larger of the FP32
// class-S layout and the class-D layout (FP64 vectors and buffers followed
// by room for both the FP64 matrices and the FP32 Lambda-split region).
template <int NP, int KIND>
struct GroupLayout {
  using GD = Geo<NP, double>;
  using GF = Geo<NP, float>;
  static constexpr size_t cbytes = CommonLayout<NP>::bytes;
  static constexpr size_t fp64 = TypedLayout<GD, kMatsTForm>::bytes;
  static constexpr size_t lamF = TypedLayout<GF, kMatsLam>::bytes;
  static constexpr size_t dmats = TypedLayout<GD, kMatsTForm>::bytes - TypedLayout<GD, 0>::bytes;
  static constexpr size_t classD = TypedLayout<GD, 0>::bytes + (dmats > lamF ? dmats : lamF);
  static constexpr size_t typed = (KIND == KIND_FP64) ? fp64 : (classD > lamF ? classD : lamF);
  static constexpr size_t bytes = align16(cbytes + typed);
  // typed-region offset of the FP32 region inside a class-D group
  static constexpr size_t lamF_in_D = TypedLayout<GD, 0>::bytes;
};

// Pointers into one group's shared memory: the common prefix at `goff`, the
// typed region (Real view) at `tb` (both absolute byte offsets into
// adrt_smem).  Built inside every function so the compiler sees
// shared-space pointers; non-inlined calls receive (goff, tb, t, bar).
template <class Gm>
struct Ctx {
  using Real = typename Gm::Real;
  using CL = CommonLayout<Gm::NP>;
  using TL = TypedLayout<Gm, 0>;
  static constexpr int NP = Gm::NP, MAT = Gm::MAT;
  unsigned goff, tb;
  int t, lane, warp, bar;
  Real *vec, *gjbuf;
  double* dvec;
  ColumnDev* col;
  unsigned* red;
  double* sc;
  __device__ __forceinline__ Ctx(unsigned goff_, unsigned tb_, int t_, int bar_)
      : goff(goff_), tb(tb_), t(t_), lane(t_ & 31), warp(t_ >> 5), bar(bar_) {
    vec = sp<Real>(tb + TL::vecs);
    gjbuf = sp<Real>(tb + TL::gj);
    dvec = sp<double>(goff + CL::dvecs);
    col = sp<ColumnDev>(goff + CL::col);
    red = sp<unsigned>(goff + CL::misc);
    sc = sp<double>(goff + CL::misc + 48);
  }
  __device__ __forceinline__ unsigned mo(int i) const {
    return tb + (unsigned)(TL::mats + (size_t)i * MAT * sizeof(Real));
  }
  __device__ __forceinline__ Real* m(int i) const { return sp<Real>(mo(i)); }
  __device__ __forceinline__ unsigned vo(int s) const {
    return tb + (unsigned)(TL::vecs + (size_t)s * NP * sizeof(Real));
  }
  __device__ __forceinline__ unsigned dvo(int s) const {
    return goff + (unsigned)(CL::dvecs + (size_t)s * NP * sizeof(double));
  }
  __device__ __forceinline__ unsigned gjo() const { return tb + (unsigned)TL::gj; }
  __device__ __forceinline__ unsigned redo() const { return goff + (unsigned)CL::misc; }
  __device__ __forceinline__ Real* V(int s) const { return vec + s * NP; }
  __device__ __forceinline__ double* DV(int s) const { return dvec + s * NP; }
  __device__ __forceinline__ void sync() const { gsync<Gm::G>(bar); }
};

// Level arrays of one slot.
struct Levels {
  double *B, *tc, *tau, *om, *omu, *flag;
  __device__ __forceinline__ Levels(char* slot, int lmax) {
    B = reinterpret_cast<double*>(slot);
    tc = B + (lmax + 1);
    tau = tc + (lmax + 1);
    om = tau + (lmax + 1);
    omu = om + (lmax + 1);
    flag = omu + (lmax + 1);
  }
};

// ------------------------------------------------------------- phase matrices
// P++/P+- from Legendre moments with Hansen column renormalisation
// (src/phase_matrix.hpp:61-111) into the slot (row-major NP x NP doubles)
// and, with a solar beam, the phase vectors at mu0 (src/phase_matrix.hpp:
// 131-181) into D_PP / D_PM.  chi_l = (chi[l] - f) / (1 - f) when delta-M
// truncation applies (f >= 0), chi[l] otherwise.
//
// On the FP64 tensor cores (NP >= 8) the double sum is two products over the
// even and the odd moments, E = A_e B_e and O = A_o B_o with
// A[r][k] = d_l P_l(mu_r), B[k][c] = P_l(mu_c), d_l = (2l+1) chi_l, so that
// P++ = (E + O) / 2pi and P+- = (E - O) / 2pi; rows and columns >= N are zero.
#ifndef ADRT_PHASE_MMA
#define ADRT_PHASE_MMA 1
#endif
#ifndef ADRT_UNSTABLE_PIVOT
#define ADRT_UNSTABLE_PIVOT 1  // tuning: 0 leaves unstable starts to the weak-pivot check
#endif
#ifndef ADRT_PHASE_TABLE
#define ADRT_PHASE_TABLE 1  // tuning: 0 rebuilds shared phase matrices per wavenumber
#endif

template <class Gm>
struct UsePhaseMMA {
  static constexpr int NT = Gm::NP / 8, NW = Gm::G / 32;
  static constexpr bool value = ADRT_PHASE_MMA && Gm::NP >= 8 && (NT * NT) % NW == 0;
};

// Q+- (as above) into qpp / qpm with row stride ldq; with NORM, already
// Hansen-normalised: column c scaled by 1 / (2 pi s_c), s_c = sum_r (Q++ +
// Q+-)[r][c] w_r = sum_r E[r][c] w_r / pi, reduced from the fragments (wt:
// the quadrature weights, red: NW x NP doubles of scratch).
template <class Gm, bool NORM = false>
__device__ __forceinline__ void phase_products(const double* chi, int nuse, double f, int N,
                                               const double* pl, double* qpp, double* qpm,
                                               int ldq, int t, const double* wt = nullptr,
                                               double* red = nullptr, int bar = 0) {
  constexpr int NT = UsePhaseMMA<Gm>::NT, NW = UsePhaseMMA<Gm>::NW, TPW = NT * NT / NW;
  const int warp = t >> 5, lane = t & 31, g = lane >> 2, q = lane & 3;
  const double inv_1mf = (f >= 0.0) ? 1.0 / (1.0 - f) : 1.0;
  const int kh = (nuse + 1) >> 1;  // even moments (odd ones: nuse / 2)
  double ev[TPW][2], od[TPW][2];
#pragma unroll
  for (int u = 0; u < TPW; ++u) ev[u][0] = ev[u][1] = od[u][0] = od[u][1] = 0.0;
  for (int k0 = 0; k0 < kh; k0 += 4) {
    const int le = 2 * (k0 + q), lo = le + 1;
    double de = 0.0, dd = 0.0;
    if (le < nuse) de = (2 * le + 1) * ((f >= 0.0) ? (chi[le] - f) * inv_1mf : chi[le]);
    if (lo < nuse) dd = (2 * lo + 1) * ((f >= 0.0) ? (chi[lo] - f) * inv_1mf : chi[lo]);
#pragma unroll
    for (int u = 0; u < TPW; ++u) {
      const int tau = warp * TPW + u, r = 8 * (tau / NT) + g, c = 8 * (tau % NT) + g;
      const double ae = (r < N && le < nuse) ? de * pl[le * N + r] : 0.0;
      const double be = (c < N && le < nuse) ? pl[le * N + c] : 0.0;
      const double ao = (r < N && lo < nuse) ? dd * pl[lo * N + r] : 0.0;
      const double bo = (c < N && lo < nuse) ? pl[lo * N + c] : 0.0;
      mma_f64_m8n8k4(ev[u][0], ev[u][1], ae, be);
      mma_f64_m8n8k4(od[u][0], od[u][1], ao, bo);
    }
  }
  const double s = 1.0 / (2.0 * kPi);
  double corr[NT][2];
#pragma unroll
  for (int j = 0; j < NT; ++j) corr[j][0] = corr[j][1] = 1.0;
  if constexpr (NORM) {
    double cp[NT][2];  // this warp's part of the column sums of E w
#pragma unroll
    for (int j = 0; j < NT; ++j) cp[j][0] = cp[j][1] = 0.0;
#pragma unroll
    for (int u = 0; u < TPW; ++u) {
      const int tau = warp * TPW + u, r = 8 * (tau / NT) + g, j = tau % NT;
      const double wr = (r < N) ? wt[r] : 0.0;
      cp[j][0] += ev[u][0] * wr;
      cp[j][1] += ev[u][1] * wr;
    }
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int o = 4; o < 32; o <<= 1) {
        cp[j][0] += __shfl_xor_sync(0xffffffffu, cp[j][0], o);
        cp[j][1] += __shfl_xor_sync(0xffffffffu, cp[j][1], o);
      }
    if constexpr (NW > 1) {
      constexpr int NP = Gm::NP;
      if (g == 0) {
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          red[warp * NP + 8 * j + 2 * q] = cp[j][0];
          red[warp * NP + 8 * j + 2 * q + 1] = cp[j][1];
        }
      }
      gsync<Gm::G>(bar);
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        double a = 0.0, b = 0.0;
#pragma unroll
        for (int w2 = 0; w2 < NW; ++w2) {
          a += red[w2 * NP + 8 * j + 2 * q];
          b += red[w2 * NP + 8 * j + 2 * q + 1];
        }
        cp[j][0] = a;
        cp[j][1] = b;
      }
      gsync<Gm::G>(bar);
    }
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const double sc = cp[j][e] / kPi;
        corr[j][e] = (sc > 0.0) ? 1.0 / (2.0 * kPi * sc) : 1.0;
      }
  }
#pragma unroll
  for (int u = 0; u < TPW; ++u) {
    const int tau = warp * TPW + u, r = 8 * (tau / NT) + g, j = tau % NT, c = 8 * j + 2 * q;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      qpp[r * ldq + c + e] = (ev[u][e] + od[u][e]) * s * corr[j][e];
      qpm[r * ldq + c + e] = (ev[u][e] - od[u][e]) * s * corr[j][e];
    }
  }
}

// Phase matrices P++ / P+- (normalised, row-major, pitch NP) into Ppp / Ppm
// and, with `solar`, the solar phase vectors into D_PP / D_PM.  With PL0,
// plm0[l] = P_l(mu0) for l < nuse (formed once per wavenumber by the same
// recurrence) and the un-normalised solar vectors also go to D_LAM0 / D_LAM1.
// With a table (the call's shared-moment phase table row of this layer: the
// normalised P++ then P+-) the matrices are copied from it and only the solar
// vectors are formed.
template <class Gm, bool PL0 = false>
__device__ __noinline__ void build_phase(unsigned goff, unsigned tb, int t_, int bar,
                                         const double* chi, int nuse, double f, int N,
                                         const double* pl, bool solar, double mu0, double* Ppp,
                                         double* Ppm, const double* plm0 = nullptr,
                                         const double* table = nullptr) {
  constexpr int NP = Gm::NP, G = Gm::G;
  const Ctx<Gm> X(goff, tb, t_, bar);
  const int t = X.t;
  const double inv_1mf = (f >= 0.0) ? 1.0 / (1.0 - f) : 1.0;
  const double* wt = X.DV(D_WT);
  const bool mats = table == nullptr;
  if (!mats) {
    for (int e = t; e < NP * NP; e += G) {
      Ppp[e] = __ldg(table + e);
      Ppm[e] = __ldg(table + NP * NP + e);
    }
  } else if constexpr (UsePhaseMMA<Gm>::value) {
    // scratch: D_PP .. D_LAM1 (4 NP doubles; the solar vectors are built below)
    phase_products<Gm, true>(chi, nuse, f, N, pl, Ppp, Ppm, NP, t, wt, X.DV(D_PP), bar);
  } else {
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
  }
  X.sync();
  if (mats && !UsePhaseMMA<Gm>::value && t < N) {  // Hansen renormalisation (scalar path)
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
        if constexpr (PL0) {
          // the same sums, their loads issued eight at a time (these small
          // tables mostly miss L1 beside the adjoint's shared memory)
          for (int l0 = 0; l0 < nuse; l0 += 8) {
            double c[8], p[8], q[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const int l = (l0 + j < nuse) ? l0 + j : 0;
              c[j] = chi[l];
              p[j] = pl[l * N + t];
              q[j] = plm0[l];
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const int l = l0 + j;
              if (l < nuse) {
                const double cl = (f >= 0.0) ? (c[j] - f) * inv_1mf : c[j];
                const double term = (2 * l + 1) * cl * p[j] * q[j];
                sp += term;
                sm += (l & 1) ? -term : term;
              }
            }
          }
        } else {
          double sign = 1.0, p0 = 1.0, p1 = mu0;
          for (int l = 0; l < nuse; ++l) {
            double plm;
            if (l == 0) {
              plm = 1.0;
            } else if (l == 1) {
              plm = mu0;
            } else {
              plm = ((2 * l - 1) * mu0 * p1 - (l - 1) * p0) * recip((double)l);  // off the chain
              p0 = p1;
              p1 = plm;
            }
            const double cl = (f >= 0.0) ? (chi[l] - f) * inv_1mf : chi[l];
            const double term = (2 * l + 1) * cl * pl[l * N + t] * plm;
            sp += term;
            sm += sign * term;
            sign = -sign;
          }
        }
        sp /= (2.0 * kPi);
        sm /= (2.0 * kPi);
      }
      pp[t] = sp;
      pm[t] = sm;
      if constexpr (PL0) {
        X.DV(D_LAM0)[t] = sp;
        X.DV(D_LAM1)[t] = sm;
      }
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

// ------------------------------------------------------------- doubling (reference order)
// One homogeneous scattering layer (src/doubling.hpp:79-229): first-order
// thin-layer start at tau0 = tau 2^-nn, then nn doublings of R, T and of the
// thermal (y, z) and solar sources.  Buffers: m0 R (row-major), m1 / m2 T
// (row-major, ping-pong), m3 I - R^2 then TG R (column-major), m4 TG
// (column-major).  On return T is in m[return value] (1 or 2) and the
// combined thermal + solar sources in V_SUP / V_SDN.  With a tape, every step
// is recorded for the adjoint (TapeLayout, matrices in the tile order of the
// forward kernel's geometry whatever the group size): R, T, TG, and
// (I - R^2)^{-1}, which the taping step solves for (straight to the record)
// and multiplies into TG.
template <class Gm, bool TAPE = false>
__device__ __noinline__ int doubling(unsigned goff, unsigned tb, int t_, int bar, double tau,
                                     double om, double Bt, double Bb, double tcum, int N,
                                     bool solar, double F0, double mu0, const double* Ppp,
                                     const double* Ppm, int* singular,
                                     typename Gm::Real* tape = nullptr) {
  using Real = typename Gm::Real;
  const Ctx<Gm> X(goff, tb, t_, bar);
  constexpr int NP = Gm::NP, TR = Gm::TR, TC = Gm::TC;
  const int t = X.t;
  const double* mu = X.DV(D_MU);
  const double* wt = X.DV(D_WT);
  om = om > 1.0 ? 1.0 : om;
  const double con = 2.0 * om * kPi;
  const int nn = num_doublings(tau, om);
  const double tau0 = ldexp(tau, -nn);
  const double Ftop = solar ? F0 * exp(-tcum / mu0) : 0.0;
  const unsigned oR = X.mo(0), oA = X.mo(3), oTG = X.mo(4);
  const unsigned oT[2] = {X.mo(1), X.mo(2)};
  constexpr bool taping = TAPE;
  // An unstable first-order start (tau0 beyond half the smallest quadrature
  // cosine: T = I - tau0 Gpp with large negative diagonal entries) leaves
  // I - R^2 outside the diagonally dominant class the pivot-free solve is
  // argued for; its solves use the reference's partial pivoting, as every
  // solve does in the re-solve of a wavenumber that met a weak pivot (the
  // group's S_PIVALL flag: the re-solve pass, or wav_body_checked).
  const int pivot = X.sc[S_PIVALL] != 0.0 || (ADRT_UNSTABLE_PIVOT && tau0 > 0.5 * mu[0]);
  using GC = Geo<NP, Real>;  // record order
  using Tp = TapeLayout<Gm>;
  Real* Rrm = sp<Real>(oR);
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
      matvec<Gm, false, 2>(Rrm, vv, yv, X.lane);
      if (X.lane < NP) {
        const Real ru = yv[0] + gam * su[X.lane], rd = gam * yv[1] + sd[X.lane];
        X.V(V_RU)[X.lane] = ru;
        X.V(V_RD)[X.lane] = rd;
        if constexpr (taping) {
          Real* tv = tape + (size_t)k * Tp::STEP + Tp::OFF_SOL;
          tv[X.lane] = ru;
          tv[NP + X.lane] = rd;
          tv[2 * NP + X.lane] = yv[1];
        }
      }
    }
    int steps = -1;  // product-form steps of (I - R^2)^{-1}, or -1: Gauss-Jordan
    if constexpr (UseNS<Gm>::value) {
      op_gemm<Gm, true>(oR, oR, kNoMat, 0, oA, kNoMat, t);  // S = R^2 (X = R row-major)
      X.sync();
      steps = pivot ? -1 : ns_steps(ns_norm_inf<Gm>(Am, t));
      if (steps < 0) {
        op_id_plus<Gm>(oA, oA, -1.0, t);  // A = I - S (each thread its own tile)
        X.sync();
      }
    } else {
      op_gemm<Gm, true>(oR, oR, kNoMat, 1, oA, kNoMat, t);  // I - R^2 (X = R row-major)
      X.sync();
    }
    if (steps == 0 && !taping) {
      // (I - S)^{-1} = I + S to round-off: TG = T + T S
      op_gemm<Gm, true>(oTc, oA, oTc, 0, kNoMat, oTG, t);
    } else if (steps >= 0) {
      // X = (I + S)(I + S^2)...: S, E and X rotate through the S buffer, the
      // free T buffer and the TG buffer, ending outside the TG buffer
      const bool odd = (steps & 1) || steps == 0;
      unsigned e = oA, x = odd ? oT[cur ^ 1] : oTG, f = odd ? oTG : oT[cur ^ 1];
      op_id_plus<Gm>(oA, x, 1.0, t);  // X_0 = I + S
      X.sync();
      for (int j = 0; j < steps; ++j) {
        op_gemm<Gm, true>(e, e, kNoMat, 0, f, kNoMat, t);  // E <- E^2
        X.sync();
        op_gemm<Gm, true>(x, f, x, 0, e, kNoMat, t);  // X <- X + X E (into the old E)
        X.sync();
        const unsigned ne = f, nx = e;
        f = x;
        e = ne;
        x = nx;
      }
      if constexpr (taping) op_s2g<Gm, GC>(x, tape + (size_t)k * Tp::STEP + Tp::OFF_AI, t);
      op_gemm<Gm, true>(oTc, x, kNoMat, 0, kNoMat, oTG, t);  // TG = T X (column-major)
    } else if constexpr (taping) {
      // (I - R^2)^{-1} into the free T buffer and the record, then TG = T (I - R^2)^{-1}
      Real* tk = tape + (size_t)k * Tp::STEP;
      *singular |= op_gj<Gm, GC, true>(oA, kIdentity, kNoMat, kNoMat, X.gjo(), X.redo(), t,
                                       X.bar, oT[cur ^ 1], tk + Tp::OFF_AI, pivot);
      X.sync();
      op_gemm<Gm, true>(oTc, oT[cur ^ 1], kNoMat, 0, kNoMat, oTG, t);
    } else {
      *singular |= op_gj<Gm>(oA, oTc, kNoMat, oTG, X.gjo(), X.redo(), t, X.bar, kNoMat, nullptr,
                             pivot);  // TG = T (I-R^2)^-1
    }
    X.sync();
    if constexpr (taping) {  // the adjoint's record of this step
      Real* tk = tape + (size_t)k * Tp::STEP;
      op_s2g<Gm, GC>(oR, tk + Tp::OFF_R, t);
      op_s2g<Gm, GC>(oTc, tk + Tp::OFF_T, t);
      op_s2g<Gm, GC>(oTG, tk + Tp::OFF_TG, t);  // from column-major: TG^T
      X.sync();
      if (X.warp == 0 && X.lane < NP) {
        tk[Tp::OFF_VEC + X.lane] = y[X.lane];
        tk[Tp::OFF_VEC + NP + X.lane] = z[X.lane];
        tk[Tp::OFF_VEC + 2 * NP + X.lane] = su[X.lane];
        tk[Tp::OFF_VEC + 3 * NP + X.lane] = sd[X.lane];
      }
      if (t == 0) tk[Tp::OFF_VEC + 4 * NP] = gam;
    }
    op_gemm<Gm>(oTG, oR, kNoMat, 0, kNoMat, oA, t);  // TGR = TG R (column-major)
    X.sync();
    op_gemm<Gm>(oA, oTc, oR, 0, oR, kNoMat, t);              // R <- R + TGR T
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
  if constexpr (taping) {  // tail: the chain's final y, z
    if (X.warp == 0 && X.lane < NP) {
      Real* tl_ = tape + (size_t)nn * Tp::STEP;
      tl_[X.lane] = X.V(V_Y0 + (nn & 1))[X.lane];
      tl_[NP + X.lane] = X.V(V_Z0 + (nn & 1))[X.lane];
    }
  }
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
  return 1 + cur;
}

// ------------------------------------------------------------- doubling (Lambda-split, FP32)
// Same layer, same discrete scheme, evaluated in the Lambda-split form
// described at the top of this file.  Buffers: m0/m1 R (row/column-major),
// m2/m3 T (row-major, ping-pong), m4 I - R^2 then TGR (column-major), m5 G'
// (column-major), m6/m7 T' (row-major, ping-pong), m8 the right-hand side
// Lambda R^2 + T'.  Returns the T buffer index like doubling(); the layer
// sources are left in V_SUP / V_SDN (Real) and, when src64 is given, also in
// FP64 in src64[0..NP) (up) and src64[NP..2NP) (down).
template <class Gm>
__device__ __noinline__ int doubling_lam(unsigned goff, unsigned tb, int t_, int bar, double tau,
                                         double om, double Bt, double Bb, double tcum, int N,
                                         bool solar, double F0, double mu0, const double* Ppp,
                                         const double* Ppm, int* singular, double* src64) {
  using Real = typename Gm::Real;
  const Ctx<Gm> X(goff, tb, t_, bar);
  constexpr int NP = Gm::NP, TR = Gm::TR, TC = Gm::TC;
  const int t = X.t;
  const double* mu = X.DV(D_MU);
  const double* wt = X.DV(D_WT);
  om = om > 1.0 ? 1.0 : om;
  const double con = 2.0 * om * kPi;
  const int nn = num_doublings(tau, om);
  const double tau0 = ldexp(tau, -nn);
  const double Ftop = solar ? F0 * exp(-tcum / mu0) : 0.0;
  const unsigned oR = X.mo(0), oRc = X.mo(1), oA = X.mo(4), oG = X.mo(5), oRHS = X.mo(8);
  const unsigned oT[2] = {X.mo(2), X.mo(3)};
  const unsigned oTp[2] = {X.mo(6), X.mo(7)};
  const unsigned oLam[2] = {X.dvo(D_LAM0), X.dvo(D_LAM1)};
  // first-order start: R = tau0 Gpm, T' = tau0 con Ppp w / mu, Lambda = 1 - tau0/mu
  {
    const Tile<Gm> tl(t);
    if (tl.valid()) {
      Real Rt[TR][TC], Tp[TR][TC], Tt[TR][TC];
#pragma unroll
      for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) {
          const int r = tl.row(a), c = tl.col(b);
          double rv = 0.0, tp = 0.0, tv = (r == c) ? 1.0 : 0.0;
          if (r < N && c < N) {
            rv = tau0 * (con * (Ppm[r * NP + c] * wt[c]) / mu[r]);
            tp = tau0 * (con * (Ppp[r * NP + c] * wt[c]) / mu[r]);
            tv = tp + ((r == c) ? 1.0 - tau0 / mu[r] : 0.0);
          }
          Rt[a][b] = static_cast<Real>(rv);
          Tp[a][b] = static_cast<Real>(tp);
          Tt[a][b] = static_cast<Real>(tv);
        }
      tl.store_rm(Rt, sp<Real>(oR));
      tl.store_cm(Rt, sp<Real>(oRc));
      tl.store_rm(Tp, sp<Real>(oTp[0]));
      tl.store_rm(Tt, sp<Real>(oT[0]));
    }
  }
  if (X.warp == 0 && X.lane < NP) {
    const int i = X.lane;
    double a = 0.0, su = 0.0, sd = 0.0, lam = 1.0;
    if (i < N) {
      lam = 1.0 - tau0 / mu[i];
      a = 0.5 * tau0 * ((1.0 - om) * tau0 / mu[i]);  // g y at the start
      if (solar) {
        const double base = om * tau0 / mu[i] * Ftop;
        su = base * X.DV(D_PM)[i];
        sd = base * X.DV(D_PP)[i];
      }
    }
    X.DV(D_LAM0)[i] = lam;
    X.V(V_Y0)[i] = static_cast<Real>(a);
    X.V(V_Z0)[i] = static_cast<Real>(-a);
    X.V(V_SU0)[i] = static_cast<Real>(su);
    X.V(V_SD0)[i] = static_cast<Real>(sd);
  }
  double gam = solar ? exp(-tau0 / mu0) : 0.0;
  int cur = 0;
  for (int k = 0; k < nn; ++k) {
    const int par = k & 1;
    Real* av = X.V(V_Y0 + par);
    Real* bv = X.V(V_Z0 + par);
    Real* su = X.V(V_SU0 + par);
    Real* sd = X.V(V_SD0 + par);
    const double* lam = X.DV(D_LAM0 + par);
    const Real gm = static_cast<Real>(gam);
    X.sync();  // R, T, T', Lambda and the vectors of the previous step are complete
    if (solar && X.warp == 0) {  // ru = R sd + gam su, rd = gam R su + sd (old R)
      const Real* vv[2] = {sd, su};
      Real yv[2];
      matvec<Gm, true, 2>(sp<Real>(oRc), vv, yv, X.lane);
      if (X.lane < NP) {
        X.V(V_RU)[X.lane] = yv[0] + gm * su[X.lane];
        X.V(V_RD)[X.lane] = gm * yv[1] + sd[X.lane];
      }
    }
    // A = I - R^2, RHS = Lambda R^2 + T'
    op_gemm_lam<Gm>(oRc, oR, oTp[cur], oLam[par], kLamR2, oA, kNoMat, oRHS, t);
    X.sync();
    *singular |= op_gj<Gm>(oA, oRHS, kNoMat, oG, X.gjo(), X.redo(), t, X.bar);  // G' (cm)
    X.sync();
    op_gemm_lam<Gm>(oG, oR, oR, oLam[par], kLamAdd, kNoMat, oA, kNoMat, t);  // TGR (cm)
    X.sync();
    op_gemm<Gm>(oA, oT[cur], oR, 0, oR, oRc, t);  // R <- R + TGR T
    // T' <- G' T + Lambda T', T <- T' + Lambda^2
    op_gemm_lam<Gm>(oG, oT[cur], oTp[cur], oLam[par], kLamAdd, oTp[cur ^ 1], kNoMat, oT[cur ^ 1],
                    t);
    if (X.warp == 0) {
      Real* an = X.V(V_Y0 + 1 - par);
      Real* bn = X.V(V_Z0 + 1 - par);
      Real* sun = X.V(V_SU0 + 1 - par);
      Real* sdn = X.V(V_SD0 + 1 - par);
      if (X.lane < NP) X.V(V_TMP)[X.lane] = Real(2) * av[X.lane] - bv[X.lane];
      __syncwarp();
      const Real* vc[2] = {X.V(V_TMP), bv};
      Real gv[2], rv[2];
      matvec<Gm, true, 2>(sp<Real>(oG), vc, gv, X.lane);  // G' c, G' b
      matvec<Gm, true, 2>(sp<Real>(oA), vc, rv, X.lane);  // TGR c, TGR b
      Real gs[2] = {Real(0), Real(0)};
      if (solar) {
        const Real* vs[2] = {X.V(V_RU), X.V(V_RD)};
        matvec<Gm, true, 2>(sp<Real>(oG), vs, gs, X.lane);
      }
      if (X.lane < NP) {
        const int i = X.lane;
        const Real l = static_cast<Real>(lam[i]);
        const Real c = X.V(V_TMP)[i], a = av[i], b = bv[i];
        an[i] = ((l * c + gv[0]) - rv[1]) + a;
        bn[i] = ((l * b + gv[1]) - rv[0]) + (Real(2) * b - a);
        if (solar) {
          sun[i] = (l * X.V(V_RU)[i] + gs[0]) + su[i];
          sdn[i] = (l * X.V(V_RD)[i] + gs[1]) + gm * sd[i];
        } else {
          sun[i] = Real(0);
          sdn[i] = Real(0);
        }
        X.DV(D_LAM0 + 1 - par)[i] = lam[i] * lam[i];
      }
    }
    gam = gam * gam;
    cur ^= 1;
  }
  X.sync();
  if (X.warp == 0 && X.lane < NP) {
    const int i = X.lane, par = nn & 1;
    const double a = X.V(V_Y0 + par)[i], b = X.V(V_Z0 + par)[i];
    const double su = X.V(V_SU0 + par)[i], sd = X.V(V_SD0 + par)[i];
    double up = 0.0, dn = 0.0;
    if (i < N) {
      up = (a * Bb - b * Bt) / tau + su;
      dn = (a * Bt - b * Bb) / tau + sd;
    }
    X.V(V_SUP)[i] = static_cast<Real>(up);
    X.V(V_SDN)[i] = static_cast<Real>(dn);
    if (src64) {
      src64[i] = up;
      src64[NP + i] = dn;
    }
  }
  return 2 + cur;
}

// ------------------------------------------------------------- doubling (Lambda-split, FP32 tensor cores)
// doubling_lam with its four products on the tensor cores (tc32_tile: three
// TF32 products each, FP32 accumulation) and the right-solve as the row-
// parallel Gauss-Jordan without pivoting (op_gj_rows), for NP = 16 (one warp)
// and NP = 32 (four warps, a 16 x 16 output tile each).  Each product reads
// its left operand row-major and its right operand column-major.  Buffers:
// m0 / m1 R (row- / column-major), m2 / m3 T (column-major, ping-pong), m4
// I - R^2 then TGR (row-major), m5 G' (row-major), m6 / m7 T' (row-major,
// ping-pong), m8 the right-hand side Lambda R^2 + T' and at the end T
// row-major.  Returns 8 (the buffer of the row-major T); the layer sources
// are left as by doubling_lam.
template <class Gm>
__device__ __noinline__ int doubling_tc(unsigned goff, unsigned tb, unsigned tbD, int t_,
                                        int bar, double tau, double om, double Bt, double Bb,
                                        double tcum, int N, bool solar, double F0, double mu0,
                                        const double* Ppp, const double* Ppm, int* singular,
                                        double* src64) {
  static_assert(UseTC32<Gm>::value && UseGjRows<Gm>::value, "tensor-core FP32 geometry");
  using Real = float;
  const Ctx<Gm> X(goff, tb, t_, bar);
  // the source vectors (a, b, s_up, s_dn and the solar ru, rd) in FP64, in
  // the class-D group's FP64 vector slots (idle while a layer doubles in
  // FP32; V_UB, the composite's source, is not touched)
  const Ctx<Geo<Gm::NP, double, Gm::G>> XV(goff, tbD, t_, bar);
  constexpr int NP = Gm::NP, TR = Gm::TR, TC = Gm::TC, LD = Gm::LD;
  const int t = X.t;
  const double* mu = X.DV(D_MU);
  const double* wt = X.DV(D_WT);
  om = om > 1.0 ? 1.0 : om;
  const double con = 2.0 * om * kPi;
  const int nn = num_doublings(tau, om);
  const double tau0 = ldexp(tau, -nn);
  const double Ftop = solar ? F0 * exp(-tcum / mu0) : 0.0;
  float* Rr = X.m(0);
  float* Rc = X.m(1);
  float* Tc[2] = {X.m(2), X.m(3)};
  float* Am = X.m(4);
  float* Gp = X.m(5);
  float* Tp[2] = {X.m(6), X.m(7)};
  float* RHS = X.m(8);
  // first-order start: R = tau0 Gpm, T' = tau0 con Ppp w / mu, Lambda = 1 - tau0/mu
  {
    const Tile<Gm> tl(t);
    if (tl.valid()) {
      Real Rt[TR][TC], Tpt[TR][TC], Tt[TR][TC];
#pragma unroll
      for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) {
          const int r = tl.row(a), c = tl.col(b);
          double rv = 0.0, tp = 0.0, tv = (r == c) ? 1.0 : 0.0;
          if (r < N && c < N) {
            rv = tau0 * (con * (Ppm[r * NP + c] * wt[c]) / mu[r]);
            tp = tau0 * (con * (Ppp[r * NP + c] * wt[c]) / mu[r]);
            tv = tp + ((r == c) ? 1.0 - tau0 / mu[r] : 0.0);
          }
          Rt[a][b] = static_cast<Real>(rv);
          Tpt[a][b] = static_cast<Real>(tp);
          Tt[a][b] = static_cast<Real>(tv);
        }
      tl.store_rm(Rt, Rr);
      tl.store_cm(Rt, Rc);
      tl.store_rm(Tpt, Tp[0]);
      tl.store_cm(Tt, Tc[0]);
    }
  }
  if (X.warp == 0 && X.lane < NP) {
    const int i = X.lane;
    double a = 0.0, su = 0.0, sd = 0.0, lam = 1.0;
    if (i < N) {
      lam = 1.0 - tau0 / mu[i];
      a = 0.5 * tau0 * ((1.0 - om) * tau0 / mu[i]);  // g y at the start
      if (solar) {
        const double base = om * tau0 / mu[i] * Ftop;
        su = base * X.DV(D_PM)[i];
        sd = base * X.DV(D_PP)[i];
      }
    }
    X.DV(D_LAM0)[i] = lam;
    XV.V(V_Y0)[i] = a;
    XV.V(V_Z0)[i] = -a;
    XV.V(V_SU0)[i] = su;
    XV.V(V_SD0)[i] = sd;
  }
  int r0, c0;
  tc32_origin<Gm>(t, r0, c0);
  const int g = X.lane >> 2, q = X.lane & 3;
  double gam = solar ? exp(-tau0 / mu0) : 0.0;
  int cur = 0;
  for (int k = 0; k < nn; ++k) {
    const int par = k & 1;
    double* av = XV.V(V_Y0 + par);
    double* bv = XV.V(V_Z0 + par);
    double* su = XV.V(V_SU0 + par);
    double* sd = XV.V(V_SD0 + par);
    const double* lam = X.DV(D_LAM0 + par);
    X.sync();  // R, T, T', Lambda and the vectors of the previous step are complete
    if (solar && X.warp == 0) {  // ru = R sd + gam su, rd = gam R su + sd (old R)
      const double* vv[2] = {sd, su};
      double yv[2];
      matvec_fd<Gm, true, 2>(Rc, vv, yv, X.lane);
      if (X.lane < NP) {
        XV.V(V_RU)[X.lane] = yv[0] + gam * su[X.lane];
        XV.V(V_RD)[X.lane] = gam * yv[1] + sd[X.lane];
      }
    }
    {  // A = I - R^2, RHS = Lambda R^2 + T'
      float acc[2][4];
      tc32_tile<NP, LD>(Rr, Rc, r0, c0, X.lane, acc);
      const float* tpc = Tp[cur];
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = r0 + g + 8 * h, c = c0 + 8 * j + 2 * q;
          const float l = static_cast<float>(lam[r]);
          const float v0 = acc[j][2 * h], v1 = acc[j][2 * h + 1];
          const float2 tp = *reinterpret_cast<const float2*>(tpc + r * LD + c);
          *reinterpret_cast<float2*>(Am + r * LD + c) =
              make_float2(((r == c) ? 1.f : 0.f) - v0, ((r == c + 1) ? 1.f : 0.f) - v1);
          *reinterpret_cast<float2*>(RHS + r * LD + c) = make_float2(fmaf(l, v0, tp.x), fmaf(l, v1, tp.y));
        }
    }
    X.sync();
    *singular |= op_gj_rows<Gm>(X.mo(4), X.mo(8), X.mo(5), t, X.bar);  // G' (row-major)
    X.sync();
    {  // TGR = G' R + Lambda R (row-major, over I - R^2)
      float acc[2][4];
      tc32_tile<NP, LD>(Gp, Rc, r0, c0, X.lane, acc);
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = r0 + g + 8 * h, c = c0 + 8 * j + 2 * q;
          const float l = static_cast<float>(lam[r]);
          const float2 rv = *reinterpret_cast<const float2*>(Rr + r * LD + c);
          *reinterpret_cast<float2*>(Am + r * LD + c) =
              make_float2(fmaf(l, rv.x, acc[j][2 * h]), fmaf(l, rv.y, acc[j][2 * h + 1]));
        }
    }
    X.sync();
    {  // R <- R + TGR T;  T' <- G' T + Lambda T',  T <- T' + Lambda^2
      float acc[2][4], acc2[2][4];
      tc32_tile<NP, LD>(Am, Tc[cur], r0, c0, X.lane, acc);
      tc32_tile<NP, LD>(Gp, Tc[cur], r0, c0, X.lane, acc2);
      const float* tpc = Tp[cur];
      float* tpn = Tp[cur ^ 1];
      float* tcn = Tc[cur ^ 1];
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = r0 + g + 8 * h, c = c0 + 8 * j + 2 * q;
          const float2 rv = *reinterpret_cast<const float2*>(Rr + r * LD + c);
          const float n0 = rv.x + acc[j][2 * h], n1 = rv.y + acc[j][2 * h + 1];
          *reinterpret_cast<float2*>(Rr + r * LD + c) = make_float2(n0, n1);
          Rc[c * LD + r] = n0;
          Rc[(c + 1) * LD + r] = n1;
          const double ld = lam[r];
          const float l = static_cast<float>(ld), l2 = static_cast<float>(ld * ld);
          const float2 tp = *reinterpret_cast<const float2*>(tpc + r * LD + c);
          const float p0 = fmaf(l, tp.x, acc2[j][2 * h]), p1 = fmaf(l, tp.y, acc2[j][2 * h + 1]);
          *reinterpret_cast<float2*>(tpn + r * LD + c) = make_float2(p0, p1);
          tcn[c * LD + r] = (r == c) ? p0 + l2 : p0;
          tcn[(c + 1) * LD + r] = (r == c + 1) ? p1 + l2 : p1;
        }
    }
    if (X.warp == 0) {
      double* an = XV.V(V_Y0 + 1 - par);
      double* bn = XV.V(V_Z0 + 1 - par);
      double* sun = XV.V(V_SU0 + 1 - par);
      double* sdn = XV.V(V_SD0 + 1 - par);
      if (X.lane < NP) XV.V(V_TMP)[X.lane] = 2.0 * av[X.lane] - bv[X.lane];
      __syncwarp();
      const double* vc[2] = {XV.V(V_TMP), bv};
      double gv[2], rv[2];
      matvec_fd<Gm, false, 2>(Gp, vc, gv, X.lane);  // G' c, G' b
      matvec_fd<Gm, false, 2>(Am, vc, rv, X.lane);  // TGR c, TGR b
      double gs[2] = {0.0, 0.0};
      if (solar) {
        const double* vs[2] = {XV.V(V_RU), XV.V(V_RD)};
        matvec_fd<Gm, false, 2>(Gp, vs, gs, X.lane);
      }
      if (X.lane < NP) {
        const int i = X.lane;
        const double l = lam[i];
        const double c = XV.V(V_TMP)[i], a = av[i], b = bv[i];
        an[i] = ((l * c + gv[0]) - rv[1]) + a;
        bn[i] = ((l * b + gv[1]) - rv[0]) + (2.0 * b - a);
        if (solar) {
          sun[i] = (l * XV.V(V_RU)[i] + gs[0]) + su[i];
          sdn[i] = (l * XV.V(V_RD)[i] + gs[1]) + gam * sd[i];
        } else {
          sun[i] = 0.0;
          sdn[i] = 0.0;
        }
        X.DV(D_LAM0 + 1 - par)[i] = lam[i] * lam[i];
      }
    }
    gam = gam * gam;
    cur ^= 1;
  }
  X.sync();
  {  // T row-major (into the right-hand-side buffer) for the adding
    const Tile<Gm> tl(t);
    if (tl.valid()) {
      Real Tt[TR][TC];
#pragma unroll
      for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) Tt[a][b] = Tc[cur][tl.col(b) * LD + tl.row(a)];
      tl.store_rm(Tt, RHS);
    }
  }
  if (X.warp == 0 && X.lane < NP) {
    const int i = X.lane, par = nn & 1;
    const double a = XV.V(V_Y0 + par)[i], b = XV.V(V_Z0 + par)[i];
    const double su = XV.V(V_SU0 + par)[i], sd = XV.V(V_SD0 + par)[i];
    double up = 0.0, dn = 0.0;
    if (i < N) {
      up = (a * Bb - b * Bt) / tau + su;
      dn = (a * Bt - b * Bb) / tau + sd;
    }
    X.V(V_SUP)[i] = static_cast<Real>(up);
    X.V(V_SDN)[i] = static_cast<Real>(dn);
    if (src64) {
      src64[i] = up;
      src64[NP + i] = dn;
    }
  }
  return 8;
}

// Class-D layers that double in FP32: run doubling_lam in the FP32 region
// at `tbF` (which overlays this group's FP64 matrices), then widen R, T and
// the sources into the FP64 buffers the adding reads (R -> m0 row-major,
// T -> m2 row-major, sources -> V_SUP / V_SDN).  src64 is 2 NP doubles of
// global scratch that carry the FP64 sources across.
template <class GmD>
__device__ __noinline__ int doubling_lam_wide(unsigned goff, unsigned tbD, unsigned tbF, int t_,
                                              int bar, double tau, double om, double Bt,
                                              double Bb, double tcum, int N, bool solar,
                                              double F0, double mu0, const double* Ppp,
                                              const double* Ppm, int* singular,
                                              double* src64) {
  using GmF = Geo<GmD::NP, float, GmD::G>;
  constexpr int TR = GmD::TR, TC = GmD::TC, NP = GmD::NP;
  static_assert(GmF::TR == TR && GmF::TC == TC && GmF::G == GmD::G, "tile maps must agree");
  int tF;
  if constexpr (UseTC32<GmF>::value && UseGjRows<GmF>::value)
    tF = doubling_tc<GmF>(goff, tbF, tbD, t_, bar, tau, om, Bt, Bb, tcum, N, solar, F0, mu0, Ppp,
                          Ppm, singular, src64);
  else
    tF = doubling_lam<GmF>(goff, tbF, t_, bar, tau, om, Bt, Bb, tcum, N, solar, F0, mu0, Ppp,
                           Ppm, singular, src64);
  (void)tF;
  const Ctx<GmF> XF(goff, tbF, t_, bar);
  const Ctx<GmD> XD(goff, tbD, t_, bar);
  XD.sync();
  const Tile<GmF> tf(XF.t);
  const Tile<GmD> td(XD.t);
  // T = Lambda + T' is widened as its two parts: the diffuse T' (FP32, the
  // buffer 6 + (nn & 1) of both FP32 doublings) plus the direct diagonal
  // Lambda kept in FP64, so that 1 - T of a thin layer keeps FP64 accuracy
  // in the adding (T rounded to FP32 as a whole loses it: 6e-8 of 1 per layer)
  const int nn = num_doublings(tau, om > 1.0 ? 1.0 : om);
  const double* lam = XF.DV(D_LAM0 + (nn & 1));
  float Rf[TR][TC], Tf[TR][TC];
  if (tf.valid()) {
    tf.load_rm(Rf, XF.m(0));
    tf.load_rm(Tf, XF.m(6 + (nn & 1)));
  }
  XD.sync();  // the FP64 buffers overlay the FP32 region
  if (td.valid()) {
    double Rd[TR][TC], Td[TR][TC];
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) {
        Rd[a][b] = Rf[a][b];
        Td[a][b] = (double)Tf[a][b] + ((td.row(a) == td.col(b)) ? lam[td.row(a)] : 0.0);
      }
    td.store_rm(Rd, XD.m(0));
    td.store_rm(Td, XD.m(1));
  }
  if (XD.warp == 0 && XD.lane < NP) {
    XD.V(V_SUP)[XD.lane] = src64[XD.lane];
    XD.V(V_SDN)[XD.lane] = src64[NP + XD.lane];
  }
  return 1;
}

// ------------------------------------------------------------- interface output
template <class Gm>
__device__ __forceinline__ void emit_interface(const Ctx<Gm>& X, const ColumnDev* C, int w, int l,
                                               int N, bool solar, double F0, double mu0,
                                               const Levels& lv, unsigned* status) {
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
    fdir = (l == 0) ? F0 * mu0 : F0 * mu0 * exp(-lv.tc[l] / mu0);
    J += fdir * (1.0 / (4.0 * kPi * mu0));
  }
  const int nL = C->L;
  const int lyr = (l == 0) ? 0 : l - 1;
  const double divF = 4.0 * kPi * (1.0 - lv.omu[lyr]) * (J - lv.B[l]);
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

// ------------------------------------------------------------- prologue
// Quadrature constants, Planck levels, delta-M scaled optical properties
// (src/solver.cpp:385-514), cumulative scaled tau and the boundary sources;
// with `mixed`, also the per-layer FP64 flags of the mixed form.  Returns
// (group-uniform) whether any layer is flagged.
template <int NP, int GS = default_group<NP>()>
__device__ __noinline__ int wav_prologue(unsigned goff, int t_, int bar, int w, char* slot,
                                         int lmax, unsigned* status, int mixed) {
  using Gm = Geo<NP, double, GS>;
  constexpr int G = Gm::G;
  const Ctx<Gm> X(goff, goff, t_, bar);  // common prefix only
  const ColumnDev* C = X.col;
  const int t = X.t;
  const int N = C->N, nL = C->L, M = C->M, layout = C->moment_layout;
  const int from_bottom = C->from_bottom;
  const double wlo = C->wlo_w ? C->wlo_w[w] : C->wn_lo;
  const double whi = C->whi_w ? C->whi_w[w] : C->wn_hi;
  const Levels lv(slot, lmax);
  // raw coefficients (src_cuda/cuda_solver.cu:175-221, 1131-1186): levels and
  // layers counted from the bottom, single-wavenumber Planck levels
  const bool raw = (C->raw_abs != nullptr);
  const double nu = raw ? C->raw_wn[w] : 0.0;

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
  unsigned bad = 0;
  for (int l = t; l <= nL; l += G) {
    const int ul = from_bottom ? nL - l : l;
    double Bv = 0.0;
    if (raw) {
      const double Tv = C->raw_temp[nL - l];
      if (!(Tv >= 0.0)) bad = 1;
      Bv = planck_single(Tv, nu);
    } else if (C->thermal) {
      const double Tv = C->temperature[(C->temp_per_wav ? (size_t)w * (nL + 1) : 0) + ul];
      if (!(Tv >= 0.0)) bad = 1;
      Bv = planck_band(wlo, whi, Tv);
    } else if (C->planck) {
      Bv = C->planck[(size_t)w * (nL + 1) + ul];
    }
    lv.B[l] = Bv;
  }
  const double mu_min = C->quad.mu[0];
  unsigned flagged = 0;
  for (int l = t; l < nL; l += G) {
    const int u = from_bottom ? nL - 1 - l : l;
    double tau, om;
    if (raw) {
      // trapezoid over the layer's two levels, plus the cloud's optical depth
      const int b = nL - 1 - l;
      const size_t W = C->W;
      const double dz = (double)C->raw_alt[b + 1] - (double)C->raw_alt[b];
      const double ab = C->raw_abs[b * W + w], at = C->raw_abs[(b + 1) * W + w];
      const double sb = C->raw_scat[b * W + w], st = C->raw_scat[(b + 1) * W + w];
      tau = dz * ((at + st) + (ab + sb)) * 0.5;
      const double sdep = dz * (st + sb) * 0.5;
      if (C->raw_cloud) tau += C->raw_cloud[b * W + w];
      if (tau < 0.0) tau = 0.0;
      om = (tau > 0.0) ? sdep / tau : 0.0;
    } else {
      tau = C->dtau[(size_t)w * nL + u];
      om = C->ssa[(size_t)w * nL + u];
    }
    if (!(tau >= 0.0 && tau < 1e300) || !(om >= 0.0 && om <= 1.0)) bad = 1;
    lv.omu[l] = om;
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
    // the reference's rule would take more doublings than the device's bound
    // (tau of order 1e15 and beyond): the layer is solved at the bound, flagged
    if (tau > 0.0 && om > 0.0 && tau >= ldexp(1.0, kMaxDoublings + 1 - ipow0(om > 1.0 ? 1.0 : om)))
      bad = 1;
    lv.tau[l] = tau;
    lv.om[l] = om;
    double fl = 0.0;
    if (mixed && tau > 0.0 && om > 0.0) {
      const double omc = om > 1.0 ? 1.0 : om;
      const int nn = num_doublings(tau, omc);
      const double tau0 = ldexp(tau, -nn);
      if (nn > kFp64MaxDoublings || tau0 > kFp64StartRatio * mu_min ||
          (1.0 - omc < kFp64NearConservative && tau > kFp64ThickTau) ||
          tau * omc > ADRT_MIX_SCAT_DEPTH) {
        fl = 1.0;
        flagged = 1;
      }
    }
    lv.flag[l] = fl;
  }
  if (bad) atomicOr(status, 4u);
  const unsigned any = gmax_u32<G>(flagged, X.red, 0, bar);
  X.sync();
  if (t == 0) {
    double tc = 0.0;
    lv.tc[0] = 0.0;
    for (int l = 0; l < nL; ++l) {
      tc += lv.tau[l];
      lv.tc[l + 1] = tc;
    }
    double Bs, Btop;
    if (raw) {
      Bs = (C->surface_temperature >= 0.0) ? planck_single(C->surface_temperature, nu) : lv.B[nL];
      Btop = (C->top_temperature >= 0.0) ? planck_single(C->top_temperature, nu) : lv.B[0];
    } else if (C->thermal) {
      Bs = (C->surface_temperature >= 0.0) ? planck_band(wlo, whi, C->surface_temperature)
                                           : lv.B[nL];
      Btop = (C->top_temperature >= 0.0) ? planck_band(wlo, whi, C->top_temperature) : lv.B[0];
    } else {
      Bs = C->semis_w ? C->semis_w[w] : C->surface_emission;
      Btop = C->temis_w ? C->temis_w[w] : C->top_emission;
    }
    X.sc[S_BS] = Bs;
    X.sc[S_BTOP] = Btop;
    X.sc[S_PIVALL] = 0.0;
  }
  X.sync();
  return any != 0u;
}

// ------------------------------------------------------------- one wavenumber
// Everything after the prologue, in the Real type of Gm: phase matrices,
// bottom composite, upward doubling + adding, downward pass and fluxes.
// MODE picks the doubling form per layer (see the top of this file); tbF is
// the FP32 region of a class-D group.
template <class Gm, int MODE>
__device__ __noinline__ int wav_body(unsigned goff, unsigned tb, unsigned tbF, int t_, int bar,
                                     int w, char* slot, int lmax, unsigned* status,
                                     double* ivec = nullptr, double* tape_all = nullptr,
                                     long long tape_cap = 0, long long* toff = nullptr) {
  using Real = typename Gm::Real;
  const Ctx<Gm> X(goff, tb, t_, bar);
  using SLay = SlotLayout<Gm>;
  constexpr int NP = Gm::NP, TR = Gm::TR, TC = Gm::TC;
  constexpr int TILE = SLay::TILE;
  const ColumnDev* C = X.col;
  const int t = X.t;
  const int N = C->N, nL = C->L, M = C->M, layout = C->moment_layout;
  const int from_bottom = C->from_bottom;

  const double A = C->albedo_w ? C->albedo_w[w] : C->surface_albedo;
  const double mu0 = C->mu0_w ? C->mu0_w[w] : C->solar_mu;
  const double F0 = C->solar_flux;
  const bool solar = (F0 > 0.0 && mu0 > 0.0);
  const Levels lv(slot, lmax);
  double* const Pslot = reinterpret_cast<double*>(slot + SLay::level_bytes(lmax));
  const double* const Ppp = Pslot;
  const double* const Ppm = Pslot + NP * NP;
  Real* recs = reinterpret_cast<Real*>(slot + SLay::level_bytes(lmax) + SLay::phase_bytes());
  const double* chi_base = C->moments;
  const double Bs = X.sc[S_BS], Btop = X.sc[S_BTOP];
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
    build_phase<Gm>(X.goff, X.tb, t, X.bar, chi, nuse, f, N, C->quad.pl, solar, mu0, Pslot,
                    Pslot + NP * NP);
  }

  // ---------------- bottom composite: surface, or the lower boundary intensity
  int cs = 0;
  {
    const double* mu = X.DV(D_MU);
    const double* wt = X.DV(D_WT);
    double dB = 0.0;
    if (C->diffusion) {
      const double dt = lv.tau[nL - 1];
      dB = (dt > 0.0) ? (lv.B[nL] - lv.B[nL - 1]) / dt : 0.0;
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
          if (solar && A > 0.0) u = u + (A / kPi) * F0 * mu0 * exp(-lv.tc[nL] / mu0);
        } else if (C->diffusion) {
          u = lv.B[nL] + mu[i] * dB;
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
  // With toff (the adjoint's forward, FP64), the doubling chains of the
  // layers are recorded back to back from the bottom into tape_all while they
  // fit in tape_cap doubles; toff[l] is the offset of layer l's record or -1.
  int singular = 0;
  long long tape_used = 0;
  for (int l = nL - 1; l >= 0; --l) {
    const double tau = lv.tau[l], om = lv.om[l];
    const double Bt = lv.B[l], Bb = lv.B[l + 1];
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
        // moments per layer; a set shared by every wavenumber (layout 0) has
        // its matrices in the call's table, copied into the slot (the doubling
        // reads them at a fixed place), and only the solar vectors, which
        // depend on this wavenumber's mu0, are formed here
        int nuse;
        double f;
        const double* chi = moments(l, nuse, f);
        const double* table =
            (ADRT_PHASE_TABLE && layout == 0 && C->ptab)
                ? C->ptab + (size_t)(from_bottom ? nL - 1 - l : l) * 2 * NP * NP
                : nullptr;
        build_phase<Gm>(X.goff, X.tb, t, X.bar, chi, nuse, f, N, C->quad.pl, solar, mu0, Pslot,
                        Pslot + NP * NP, nullptr, table);
      }
      if constexpr (MODE == MODE_FP64) {
        Real* tape_l = nullptr;
        if (toff) {
          const long long need = TapeLayout<Gm>::layer(num_doublings(tau, om > 1.0 ? 1.0 : om));
          if (tape_all && tape_used + need <= tape_cap) {
            tape_l = tape_all + tape_used;
            if (t == 0) toff[l] = tape_used;
            tape_used += need;
          } else if (t == 0) {
            toff[l] = -1;
          }
        }
        if (tape_l)
          tcur = doubling<Gm, true>(X.goff, X.tb, t, X.bar, tau, om, Bt, Bb, lv.tc[l], N, solar,
                                    F0, mu0, Ppp, Ppm, &singular, tape_l);
        else
          tcur = doubling<Gm>(X.goff, X.tb, t, X.bar, tau, om, Bt, Bb, lv.tc[l], N, solar, F0,
                              mu0, Ppp, Ppm, &singular);
      } else if constexpr (MODE == MODE_MIX_S) {
        tcur = doubling_lam<Gm>(X.goff, X.tb, t, X.bar, tau, om, Bt, Bb, lv.tc[l], N, solar, F0,
                                mu0, Ppp, Ppm, &singular, nullptr);
      } else if (lv.flag[l] != 0.0) {
        tcur = doubling<Gm>(X.goff, X.tb, t, X.bar, tau, om, Bt, Bb, lv.tc[l], N, solar, F0, mu0,
                            Ppp, Ppm, &singular);
      } else {
        // the record's two source vectors (written later in this step) carry
        // the FP64 layer sources out of the FP32 region
        tcur = doubling_lam_wide<Gm>(X.goff, X.tb, tbF, t, X.bar, tau, om, Bt, Bb, lv.tc[l], N,
                                     solar, F0, mu0, Ppp, Ppm, &singular,
                                     reinterpret_cast<double*>(rp + 3 * TILE));
      }
      X.sync();
      op_s2g<Gm>(X.mo(0), rp, t);
      op_s2g<Gm>(X.mo(tcur), rp + TILE, t);
    }
    if (X.warp == 0 && X.lane < NP) {
      rp[3 * TILE + X.lane] = X.V(V_SDN)[X.lane];
      rp[3 * TILE + 2 * NP + 2 + X.lane] = X.V(V_SUP)[X.lane];
    }
    if (t == 0) rp[3 * TILE + 2 * NP] = Real(scat);

    // adding: top = this layer, bottom = composite (src/adding.hpp:478-490).
    // The layer's T is one of the doubling's two T buffers (1 / 2 for the
    // FP64 forms, 2 / 3 for the FP32 Lambda-split form); the other is spare,
    // and the two buffers after them take R_b and D1.
    constexpr int tb0 = (MODE == MODE_MIX_S) ? 2 : 1;
    if (!scat) tcur = tb0;
    const unsigned oTl = X.mo(tcur);                 // layer T (row-major)
    const unsigned oSp = X.mo(2 * tb0 + 1 - tcur);   // spare matrix
    const unsigned oRb = X.mo(tb0 + 2), oD1 = X.mo(tb0 + 3);
    Real* Rtm = sp<Real>(oTl);
    if (!scat) {
      // non-scattering top (src/adding.hpp:349-406):
      // R_b <- t R_b t, U_b <- s_up + t (U_b + R_b s_dn)
      op_g2s<Gm>(rb_below, oRb, kNoMat, t);
      X.sync();
      if (X.warp == 0) {
        const Real* vv[1] = {X.V(V_SDN)};
        Real yv[1];
        matvec<Gm, false, 1>(sp<Real>(oRb), vv, yv, X.lane);
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
      op_g2s<Gm>(rb_below, oRb, kNoMat, t);  // R_b (row-major)
      X.sync();
      if (X.warp == 0) {
        const Real* vv[1] = {X.V(V_SDN)};
        Real yv[1];
        matvec<Gm, false, 1>(sp<Real>(oRb), vv, yv, X.lane);
        if (X.lane < NP) X.V(V_TMP)[X.lane] = X.V(V_UB)[X.lane] + yv[0];
      }
      op_gemm<Gm, true>(oRb, X.mo(0), kNoMat, 1, oSp, kNoMat, t);  // A1 = I - R_b R
      X.sync();
      singular |= op_gj<Gm>(oSp, oTl, kNoMat, oD1, X.gjo(), X.redo(), t, X.bar, kNoMat, nullptr,
                            X.sc[S_PIVALL] != 0.0);  // D1 (cm)
      X.sync();
      if (X.warp == 0) {
        const Real* vv[1] = {X.V(V_TMP)};
        Real yv[1];
        matvec<Gm, true, 1>(sp<Real>(oD1), vv, yv, X.lane);
        if (X.lane < NP) X.V(V_UB)[X.lane] = X.V(V_SUP)[X.lane] + yv[0];
      }
      op_gemm<Gm>(oD1, oRb, kNoMat, 0, kNoMat, oSp, t);  // D1 R_b (cm)
      X.sync();
      op_gemm<Gm>(oSp, oTl, X.mo(0), 0, oRb, kNoMat, t);  // R + (D1 R_b) T
      // the tensor-core product writes in fragment order, the copy reads in
      // tile order: other threads' elements must be complete
      X.sync();
      op_s2g<Gm>(oRb, rp + 2 * TILE, t);
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
    if (ivec && X.lane < NP) {  // interface intensities for the adjoint
      ivec[X.lane] = X.V(V_ID)[X.lane];
      ivec[NP + X.lane] = X.V(V_IU)[X.lane];
    }
    if (X.lane == 0) emit_interface<Gm>(X, C, w, 0, N, solar, F0, mu0, lv, status);
  }
  for (int l = 0; l < nL; ++l) {
    const Real* rl = recs + (size_t)l * SLay::REC;
    const Real* rb = recs + (size_t)(l + 1) * SLay::REC;
    const int scat = rl[3 * TILE + 2 * NP] != Real(0);
    const int cbase = rb[3 * TILE + 2 * NP + 1] != Real(0);
    X.sync();
    {  // T (cm), R (cm), R_base (rm), every load before the first store
      const Real* g[3] = {rl + TILE, rl, rb + 2 * TILE};
      const unsigned orm[3] = {kNoMat, kNoMat, X.mo(2)};
      const unsigned ocm[3] = {X.mo(0), X.mo(1), kNoMat};
      g2s_n<Gm, Gm, 3, 7u>(g, orm, ocm, t);
    }
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
      singular |= op_gj<Gm>(X.mo(3), kNoMat, X.vo(V_RHS), X.mo(4), X.gjo(), X.redo(), t, X.bar,
                            kNoMat, nullptr, X.sc[S_PIVALL] != 0.0);
      X.sync();
      xsol = X.m(4);
      xstride = Gm::LD;
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
      if (ivec && X.lane < NP) {
        ivec[(size_t)(l + 1) * 2 * NP + X.lane] = X.V(V_ID)[X.lane];
        ivec[(size_t)(l + 1) * 2 * NP + NP + X.lane] = X.V(V_IU)[X.lane];
      }
      if (X.lane == 0)
        emit_interface<Gm>(X, C, w, l + 1, N, solar, F0, mu0, lv, status);
    }
  }
  if (singular && t == 0) atomicOr(status, status_bits(singular));
  X.sync();
  return singular;
}

// The wavenumber with the tensor-core solves, and once more at once with
// partial pivoting in every solve (the group's S_PIVALL flag) when one of
// them met a weak pivot; its status then carries the pivoted re-solve bit.
// The body only reads what the prologue left, so the second pass starts from
// the same state.  For the adjoint's taping forward; the forward kernels list
// such wavenumbers for a second launch instead, which keeps a second call of
// the body (and its registers) out of them.
template <class Gm, int MODE>
__device__ __forceinline__ void wav_body_checked(unsigned goff, unsigned tb, unsigned tbF, int t,
                                                 int bar, int w, char* slot, int lmax,
                                                 unsigned* status, double* ivec = nullptr,
                                                 double* tape_all = nullptr,
                                                 long long tape_cap = 0,
                                                 long long* toff = nullptr) {
  const int fl = wav_body<Gm, MODE>(goff, tb, tbF, t, bar, w, slot, lmax, status, ivec, tape_all,
                                    tape_cap, toff);
  if (ADRT_GJ_FALLBACK && (fl & kGjWeakPivot)) {
    const Ctx<Gm> X(goff, tb, t, bar);
    if (t == 0) X.sc[S_PIVALL] = 1.0;  // the next prologue clears it
    X.sync();
    wav_body<Gm, MODE>(goff, tb, tbF, t, bar, w, slot, lmax, status, ivec, tape_all, tape_cap,
                       toff);
  }
}

// ------------------------------------------------------------- persistent kernel
// ------------------------------------------------------------- re-solve pass
// A launch's tasks: its own, or in the re-solve pass the ones the first pass
// listed (at most redo_cap), each taken from that pass's work counter.
__device__ __forceinline__ long long pass_tasks(const SolveParams& P) {
  if (!P.redo_pass) return P.ntasks;
  const long long n = (long long)P.redo[0];
  return n < P.redo_cap ? n : P.redo_cap;
}
__device__ __forceinline__ unsigned long long* pass_counter(const SolveParams& P) {
  return P.redo_pass ? P.redo + 1 : P.counter;
}
__device__ __forceinline__ long long pass_task(const SolveParams& P, long long i) {
  return P.redo_pass ? (long long)P.redo[2 + i] : i;
}
// In the re-solve pass (or with ADRT_PIVOTING_PARTIAL), after the prologue:
// every solve of the wavenumber with partial pivoting (the group's S_PIVALL
// flag; the next prologue clears it).
template <int G>
__device__ __forceinline__ void pass_pivot_all(const SolveParams& P, unsigned goff, int t,
                                               int bar, int np_common_misc) {
  if (!P.redo_pass && !P.pivot_all) return;
  if (t == 0) sp<double>(goff + (unsigned)np_common_misc + 48)[S_PIVALL] = 1.0;
  gsync<G>(bar);
}
// In the first pass, after the body: a wavenumber whose pivot-free solve met
// a weak pivot goes on the re-solve list (ADRT_FLAG_PIVOT_UNRESOLVED when
// the list is full: that wavenumber keeps the pivot-free result).
__device__ __forceinline__ void pass_list_weak(const SolveParams& P, int flags, long long task,
                                               int t) {
  if (!ADRT_GJ_FALLBACK || P.redo_pass || !(flags & kGjWeakPivot) || t != 0) return;
  const unsigned long long k = P.redo ? atomicAdd(P.redo, 1ull) : ~0ull;
  if (P.redo && k < (unsigned long long)P.redo_cap)
    P.redo[2 + k] = (unsigned long long)task;
  else
    atomicOr(P.status, 16u);
}

template <int NP, int KIND>
__global__ void __launch_bounds__(128, 3) solve_kernel(SolveParams P, ColumnDev col0) {
  using GD = Geo<NP, double>;
  using GF = Geo<NP, float>;
  using GL = GroupLayout<NP, KIND>;
  constexpr int G = GD::G;
  const int gib = threadIdx.x / G;
  const int t = threadIdx.x % G;
  const int bar = 1 + gib;
  const unsigned goff = (unsigned)(gib * GL::bytes);
  const unsigned tb = goff + (unsigned)CommonLayout<NP>::bytes;
  const int slot = blockIdx.x * (blockDim.x / G) + gib;
  char* sl = P.scratch + (size_t)slot * P.slot_bytes;
  for (unsigned i = (unsigned)t * 4u; i < (unsigned)GL::bytes; i += (unsigned)G * 4u)
    *sp<unsigned>(goff + i) = 0u;
  gsync<G>(bar);
  ColumnDev* colp = sp<ColumnDev>(goff + CommonLayout<NP>::col);
  if (P.ncols <= 1 && t == 0) *colp = col0;
  long long* task_s = sp<long long>(goff + CommonLayout<NP>::misc + 32);
  int cur_col = -1;
  const long long ntasks = pass_tasks(P);
  unsigned long long* const counter = pass_counter(P);
  for (;;) {
    long long task;
    if constexpr (G == 32) {
      unsigned long long v = 0;
      if (t == 0) v = atomicAdd(counter, 1ull);
      task = (long long)__shfl_sync(0xffffffffu, v, 0);
    } else {
      gsync<G>(bar);
      if (t == 0) *task_s = (long long)atomicAdd(counter, 1ull);
      gsync<G>(bar);
      task = *task_s;
    }
    if (task >= ntasks) break;
    task = pass_task(P, task);
    int w = (int)task;
    if (P.ncols > 1) {
      int lo = 0, hi = P.ncols - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (P.cols[mid].task_begin <= task) lo = mid; else hi = mid - 1;
      }
      if (lo != cur_col) {
        gsync<G>(bar);
        if (t == 0) *colp = P.cols[lo];
        cur_col = lo;
      }
      w = (int)(task - P.cols[lo].task_begin);
    }
    gsync<G>(bar);
    const int any =
        wav_prologue<NP>(goff, t, bar, w, sl, P.max_layers, P.status, KIND == KIND_MIXED);
    pass_pivot_all<G>(P, goff, t, bar, (int)CommonLayout<NP>::misc);
    int fl = 0;
    if constexpr (KIND == KIND_FP64) {
      fl = wav_body<GD, MODE_FP64>(goff, tb, 0u, t, bar, w, sl, P.max_layers, P.status);
    } else if (colp->precision == 0) {  // an FP64 column of an uneven batch
      fl = wav_body<GD, MODE_FP64>(goff, tb, 0u, t, bar, w, sl, P.max_layers, P.status);
    } else if (!any && !ADRT_MIX_FORCE_D) {
      fl = wav_body<GF, MODE_MIX_S>(goff, tb, 0u, t, bar, w, sl, P.max_layers, P.status);
    } else {
      fl = wav_body<GD, MODE_MIX_D>(goff, tb, tb + (unsigned)GL::lamF_in_D, t, bar, w, sl,
                                    P.max_layers, P.status);
    }
    pass_list_weak(P, fl, task, t);
  }
}

// ------------------------------------------------------------- uneven batches
// Columns of any N <= 16 (padded orders 4, 8, 16: one warp per wavenumber in
// every case) and either precision form in ONE persistent launch: each task
// is dispatched on its column's padded order and precision.  The group's
// shared memory and slot are sized for the largest order.
template <int NP>
__device__ __noinline__ int multi_task(unsigned goff, int t, int bar, int w, char* sl, int lmax,
                                       unsigned* status, int precision, int pivot_all) {
  using GD = Geo<NP, double>;
  using GF = Geo<NP, float>;
  using GL = GroupLayout<NP, KIND_MIXED>;
  const unsigned tb = goff + (unsigned)CommonLayout<NP>::bytes;
  const int any = wav_prologue<NP>(goff, t, bar, w, sl, lmax, status, precision != 0);
  if (pivot_all) {  // the re-solve pass
    if (t == 0) sp<double>(goff + (unsigned)CommonLayout<NP>::misc + 48)[S_PIVALL] = 1.0;
    __syncwarp();
  }
  if (precision == 0) return wav_body<GD, MODE_FP64>(goff, tb, 0u, t, bar, w, sl, lmax, status);
  if (!any && !ADRT_MIX_FORCE_D)
    return wav_body<GF, MODE_MIX_S>(goff, tb, 0u, t, bar, w, sl, lmax, status);
  return wav_body<GD, MODE_MIX_D>(goff, tb, tb + (unsigned)GL::lamF_in_D, t, bar, w, sl, lmax,
                                  status);
}

constexpr size_t cmax(size_t a, size_t b) { return a > b ? a : b; }
constexpr size_t kMultiGroupBytes =
    cmax(GroupLayout<16, KIND_MIXED>::bytes,
         cmax(GroupLayout<8, KIND_MIXED>::bytes, GroupLayout<4, KIND_MIXED>::bytes));

template <int kUnused = 0>  // a template, so only the translation units that launch it hold it
__global__ void __launch_bounds__(128) solve_kernel_multi(SolveParams P) {
  constexpr int G = 32;
  const int gib = threadIdx.x / G;
  const int t = threadIdx.x % G;
  const int bar = 1 + gib;
  const unsigned goff = (unsigned)(gib * kMultiGroupBytes);
  const int slot = blockIdx.x * (blockDim.x / G) + gib;
  char* sl = P.scratch + (size_t)slot * P.slot_bytes;
  for (unsigned i = (unsigned)t * 4u; i < (unsigned)kMultiGroupBytes; i += (unsigned)G * 4u)
    *sp<unsigned>(goff + i) = 0u;
  __syncwarp();
  ColumnDev* colp = sp<ColumnDev>(goff);
  int cur_col = -1;
  const long long ntasks = pass_tasks(P);
  unsigned long long* const counter = pass_counter(P);
  for (;;) {
    unsigned long long v = 0;
    if (t == 0) v = atomicAdd(counter, 1ull);
    long long task = (long long)__shfl_sync(0xffffffffu, v, 0);
    if (task >= ntasks) break;
    task = pass_task(P, task);
    int lo = 0, hi = P.ncols - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (P.cols[mid].task_begin <= task) lo = mid; else hi = mid - 1;
    }
    if (lo != cur_col) {
      __syncwarp();
      if (t == 0) *colp = P.cols[lo];
      cur_col = lo;
    }
    __syncwarp();
    const int w = (int)(task - colp->task_begin);
    const int np = colp->NP, prec = colp->precision;
    int fl;
    if (np <= 4) {
      fl = multi_task<4>(goff, t, bar, w, sl, P.max_layers, P.status, prec,
                         P.redo_pass | P.pivot_all);
    } else if (np <= 8) {
      fl = multi_task<8>(goff, t, bar, w, sl, P.max_layers, P.status, prec,
                         P.redo_pass | P.pivot_all);
    } else {
      fl = multi_task<16>(goff, t, bar, w, sl, P.max_layers, P.status, prec,
                         P.redo_pass | P.pivot_all);
    }
    pass_list_weak(P, fl, task, t);
  }
}

}  // namespace adrt_dev
