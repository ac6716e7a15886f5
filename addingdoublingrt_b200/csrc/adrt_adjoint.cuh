// adrt_adjoint.cuh -- hand-written reverse-mode adjoint of the column solve.
//
// Gradients of a loss L = sum over interfaces of c_up F_up + c_dn F_dn +
// c_J J + c_dir F_dir (cotangents supplied per wavenumber and interface) with
// respect to delta_tau, single_scat_albedo, the phase moments and the level
// temperatures (or Planck levels), for the reference's discrete scheme at
// fixed doubling counts nn (src/doubling.hpp:107-109 is piecewise constant).
// FP64 throughout.  Per wavenumber, one thread group:
//
//   1. the forward solve (wav_body), which keeps every layer's R, T, s_up,
//      s_dn, every composite R_base, U_base and the interface intensities
//      (the per-layer checkpoints of the adding);
//   2. the downward-pass adjoint, interface L-1 .. 0.  Every matrix
//      cotangent it produces is rank one (b_rhs x^T), so it stores only two
//      vectors per interface;
//   3. the adding adjoint, layer 0 .. L-1 (reverse of the bottom-up build),
//      which completes each layer's (dR, dT, ds_up, ds_dn); then that layer's
//      doubling chain is recomputed with a record of every step (the chain is
//      not stored across layers) and run backwards, then the phase matrices'
//      adjoint and the Planck / beam chain rules.
#pragma once

#include "adrt_kernel.cuh"

namespace adrt_dev {

// dB/dT of the band integral in closed form: 4B/T minus the boundary terms of
// d/dT of the integration limits v = c2 nu / T (the construction of the
// reference's planckFunctionDeriv, src/planck.cpp:135-175).
__host__ __device__ inline double planck_band_deriv(double lo, double hi, double T) {
  const double C2 = 1.438786, SIGMA = 5.67032E-8;
  if (T < 0.0 || hi < lo || lo < 0.0) return -1.0;
  if (T < 1.e-4) return 0.0;
  if (hi == lo) {
    const double x = C2 * hi / T, em = exp(-x);
    const double b = 1.1911e-8 * hi * hi * hi * em / (1.0 - em);
    return b * (x / T) / (1.0 - em);
  }
  const double conc = 15.0 / (kPi * kPi * kPi * kPi);
  const double v0 = C2 * lo / T, v1 = C2 * hi / T;
  double f0, f1;
  if (v0 < 1.e-6) {
    f0 = v0 * v0;
  } else {
    const double em = exp(-v0);
    f0 = v0 * v0 * v0 * em / (1.0 - em);
  }
  if (v1 < 1.e-6) {
    f1 = v1 * v1;
  } else {
    const double em = exp(-v1);
    f1 = v1 * v1 * v1 * em / (1.0 - em);
  }
  const double B = planck_band(lo, hi, T);
  return 4.0 * B / T - (SIGMA / kPi) * conc * T * T * T * (v1 * f1 - v0 * f0);
}

// Sum of a double over the group (every thread gets the total).
template <int G>
__device__ __forceinline__ double gsum(double v, double* red, int bar) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if constexpr (G == 32) {
    return v;
  } else {
    constexpr int NW = G / 32;
    const int t = threadIdx.x % G;
    gsync<G>(bar);
    if ((t & 31) == 0) red[t >> 5] = v;
    gsync<G>(bar);
    double r = 0.0;
#pragma unroll
    for (int i = 0; i < NW; ++i) r += red[i];
    gsync<G>(bar);
    return r;
  }
}

// out (row-major and/or column-major) += sum_p alpha_p u_p v_p^T, with the
// vectors u_p, v_p in shared memory (Real, NP entries; kNoMat = unused pair).
template <class Gm>
__device__ __noinline__ void op_rank(unsigned orm, unsigned ocm, unsigned u0, unsigned v0,
                                     double a0, unsigned u1, unsigned v1, double a1, unsigned u2,
                                     unsigned v2, double a2, unsigned u3, unsigned v3, double a3,
                                     int t) {
  using Real = typename Gm::Real;
  constexpr int TR = Gm::TR, TC = Gm::TC, LD = Gm::LD;
  const Tile<Gm> tl(t);
  if (!tl.valid()) return;
  const unsigned us[4] = {u0, u1, u2, u3}, vs[4] = {v0, v1, v2, v3};
  const double al[4] = {a0, a1, a2, a3};
  Real d[TR][TC];
#pragma unroll
  for (int a = 0; a < TR; ++a)
#pragma unroll
    for (int b = 0; b < TC; ++b) d[a][b] = Real(0);
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    if (us[p] == kNoMat) continue;
    const Real* u = sp<Real>(us[p]);
    const Real* v = sp<Real>(vs[p]);
#pragma unroll
    for (int a = 0; a < TR; ++a) {
      const Real ua = static_cast<Real>(al[p]) * u[tl.row(a)];
#pragma unroll
      for (int b = 0; b < TC; ++b) d[a][b] = fma(ua, v[tl.col(b)], d[a][b]);
    }
  }
  if (orm != kNoMat) {
    Real* o = sp<Real>(orm);
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) o[tl.row(a) * LD + tl.col(b)] += d[a][b];
  }
  if (ocm != kNoMat) {
    Real* o = sp<Real>(ocm);
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) o[tl.col(b) * LD + tl.row(a)] += d[a][b];
  }
}

// out = sum_s X_s Y_s [+ add] [+ sum_p a_p u_p v_p^T]: up to three products
// (X_s column-major, Y_s row-major, K = NP each), an added row-major matrix
// and up to four rank-one terms (vectors in smem) in one pass, so that a
// step of the doubling adjoint needs one barrier per dependent product.
struct GemmX {
  unsigned x[3], y[3];
  int nseg;
  unsigned add, orm, ocm;
  unsigned u[4], v[4];
  double a[4];
  int nrank;
};

template <class Gm, int NSEG, int NRANK>
__device__ __forceinline__ void op_gemm_x(const GemmX g, int t) {
  using Real = typename Gm::Real;
  constexpr int NP = Gm::NP, LD = Gm::LD;
  const Real* add = (g.add == kNoMat) ? nullptr : sp<Real>(g.add);
  Real* out_rm = (g.orm == kNoMat) ? nullptr : sp<Real>(g.orm);
  Real* out_cm = (g.ocm == kNoMat) ? nullptr : sp<Real>(g.ocm);
  const Real* ru[NRANK > 0 ? NRANK : 1];
  const Real* rv[NRANK > 0 ? NRANK : 1];
#pragma unroll
  for (int p = 0; p < NRANK; ++p) {
    ru[p] = sp<Real>(g.u[p]);
    rv[p] = sp<Real>(g.v[p]);
  }
  auto rank = [&](int r, int c) {
    Real v = Real(0);
#pragma unroll
    for (int p = 0; p < NRANK; ++p) v += static_cast<Real>(g.a[p]) * ru[p][r] * rv[p][c];
    return v;
  };
  if constexpr (UseMMA<Gm>::value) {
    constexpr int NT = NP / 8;
    constexpr int TPW = NT * NT / (Gm::G / 32);
    constexpr int WR = (TPW >= 4) ? 2 : 1, WC = (TPW >= 2) ? 2 : 1;
    constexpr int WPC = NT / WC;
    // a warp with one output tile keeps two partial sums (even / odd k-steps)
    // so that consecutive DMMAs do not wait on each other
    constexpr int NA = (WR * WC == 1) ? ((NSEG > 1) ? 4 : 2) : 1;
    const int warp = t >> 5, lane = t & 31, gg = lane >> 2, q = lane & 3;
    const int r0 = (warp / WPC) * WR * 8, c0 = (warp % WPC) * WC * 8;
    double acc[NA][WR][WC][2];
#pragma unroll
    for (int h = 0; h < NA; ++h)
#pragma unroll
      for (int i = 0; i < WR; ++i)
#pragma unroll
        for (int j = 0; j < WC; ++j) acc[h][i][j][0] = acc[h][i][j][1] = 0.0;
#pragma unroll
    for (int sg = 0; sg < NSEG; ++sg) {
      const double* XT = sp<double>(g.x[sg]);
      const double* Y = sp<double>(g.y[sg]);
#pragma unroll
      for (int ks = 0; ks < NP / 4; ++ks) {
        const int k = ks * 4 + q;
        const int h = (sg * (NP / 4) + ks) % NA;
        double a[WR], b[WC];
#pragma unroll
        for (int i = 0; i < WR; ++i) a[i] = XT[k * LD + r0 + i * 8 + gg];
#pragma unroll
        for (int j = 0; j < WC; ++j) b[j] = Y[k * LD + c0 + j * 8 + gg];
#pragma unroll
        for (int i = 0; i < WR; ++i)
#pragma unroll
          for (int j = 0; j < WC; ++j)
            mma_f64_m8n8k4(acc[h][i][j][0], acc[h][i][j][1], a[i], b[j]);
      }
    }
#pragma unroll
    for (int i = 0; i < WR; ++i)
#pragma unroll
      for (int j = 0; j < WC; ++j) {
        const int r = r0 + i * 8 + gg, c = c0 + j * 8 + 2 * q;
        double v0 = acc[0][i][j][0], v1 = acc[0][i][j][1];
#pragma unroll
        for (int h = 1; h < NA; ++h) {
          v0 += acc[h][i][j][0];
          v1 += acc[h][i][j][1];
        }
        if (add) {
          const double2 ad = *reinterpret_cast<const double2*>(add + r * LD + c);
          v0 = ad.x + v0;
          v1 = ad.y + v1;
        }
        if constexpr (NRANK > 0) {
          v0 += rank(r, c);
          v1 += rank(r, c + 1);
        }
        if (out_rm) *reinterpret_cast<double2*>(out_rm + r * LD + c) = make_double2(v0, v1);
        if (out_cm) {
          out_cm[c * LD + r] = v0;
          out_cm[(c + 1) * LD + r] = v1;
        }
      }
  } else {
    constexpr int TR = Gm::TR, TC = Gm::TC;
    const Tile<Gm> tl(t);
    if (!tl.valid()) return;
    Real acc[TR][TC];
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) acc[a][b] = Real(0);
#pragma unroll
    for (int sg = 0; sg < NSEG; ++sg) {
      const Real* xp = sp<Real>(g.x[sg]) + tl.rb * TR;
      const Real* yp = sp<Real>(g.y[sg]) + tl.cb * TC;
      for (int k = 0; k < NP; ++k) {
        Real xa[TR], yb[TC];
        lds_vec<Real, TR>(xa, xp + k * LD);
        lds_vec<Real, TC>(yb, yp + k * LD);
#pragma unroll
        for (int a = 0; a < TR; ++a)
#pragma unroll
          for (int b = 0; b < TC; ++b) acc[a][b] = fma(xa[a], yb[b], acc[a][b]);
      }
    }
    if (add) {
      Real ad[TR][TC];
      tl.load_rm(ad, add);
#pragma unroll
      for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) acc[a][b] = ad[a][b] + acc[a][b];
    }
    if constexpr (NRANK > 0) {
#pragma unroll
      for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) acc[a][b] += rank(tl.row(a), tl.col(b));
    }
    if (out_rm) tl.store_rm(acc, out_rm);
    if (out_cm) tl.store_cm(acc, out_cm);
  }
}

// Copy a row-major matrix into row-major and/or column-major buffers, scaled.
template <class Gm>
__device__ __noinline__ void op_copy(unsigned in_rm, unsigned orm, unsigned ocm, double scale,
                                     int t) {
  using Real = typename Gm::Real;
  constexpr int TR = Gm::TR, TC = Gm::TC;
  const Tile<Gm> tl(t);
  if (!tl.valid()) return;
  Real X[TR][TC];
  tl.load_rm(X, sp<Real>(in_rm));
#pragma unroll
  for (int a = 0; a < TR; ++a)
#pragma unroll
    for (int b = 0; b < TC; ++b) X[a][b] *= static_cast<Real>(scale);
  if (orm != kNoMat) tl.store_rm(X, sp<Real>(orm));
  if (ocm != kNoMat) tl.store_cm(X, sp<Real>(ocm));
}

// ---------------------------------------------------------------- buffers
// Matrix buffers of the adjoint's typed region (row-major "r", column-major "c").
enum AdjMat {
  J_R = 0, J_Rc, J_Tc, J_TG, J_TGc, J_TGR, J_Ac, J_bR0, J_bR0c, J_bT0, J_bT0c, J_bR1, J_bR1c,
  J_bT1, J_bT1c, J_bTGR, J_bTGRc, J_bTG, J_W, J_C, J_Cc, J_T1, J_T2, J_VEC,
  kMatsAdj = J_VEC + 2  // J_VEC spans two buffers (18 vectors even at NP = 8)
};
// The record pool of a chunk holds kTapeStepsPerLayer doubling steps per
// layer and wavenumber on average (nn = trunc(log2 tau) + 4 / 10 / 16, so
// 12 covers tau up to 2^-4 .. 2^8 depending on omega; the pool is shared, so
// thin layers leave room for thick ones).  A wavenumber whose chains do not
// fit is recomputed in the reverse.  kAdjointMemory bounds the adjoint's
// work memory when the engine has no workspace limit.
constexpr int kTapeStepsPerLayer = 12;
constexpr size_t kAdjointMemory = size_t(16) << 30;
// Moment sets shared by every wavenumber: the reverse sums their phase-matrix
// cotangents per block (2 NP^2 doubles per set and block) when that fits here.
constexpr size_t kPhaseSumMemory = size_t(1) << 30;

// Vector slots inside the J_VEC buffers (each NP Reals; 2 DIM LD >= 20 NP).
enum AdjVec {
  A_BY = 0, A_BZ, A_BSU, A_BSD, A_H, A_RU, A_RD, A_BRU, A_BRD, A_BH, A_Y, A_Z, A_SU, A_SD,
  A_BUP, A_BDN, A_T0, A_T1,
  A_CUB,  // the adding adjoint's carried d U_base (not touched by the layer adjoints)
  A_X4, A_X5, A_X6,  // a doubling-adjoint step's TGR^T bsd, TGR^T bsu, R su
  kAdjVecs
};
// Partial products of one doubling-adjoint step, in slots that are scratch
// inside the step loop (z is only needed for h; T0 / T1 are written after it).
constexpr int A_X0 = A_BH, A_X1 = A_T0, A_X2 = A_T1, A_X3 = A_Z;

// Per-wavenumber state that the taping forward (tape_kernel, the forward
// kernel's geometry GC) leaves for the reverse (adjoint_kernel): the forward
// slot (levels, phase, records in GC's tile order), the interface
// intensities, and the offsets of the layers' doubling records (toff[l],
// relative to the wavenumber's block of the record pool, or -1; toff[L] is
// that block's offset in the pool, or -1).
template <class GC>
struct WavState {
  static __host__ __device__ size_t fwd(int lmax) {
    return (SlotLayout<GC>::bytes(lmax) + 255) & ~size_t(255);
  }
  static __host__ __device__ size_t ivec(int lmax) {
    return ((size_t)(lmax + 1) * 2 * GC::NP * sizeof(double) + 255) & ~size_t(255);
  }
  static __host__ __device__ size_t toff_at(int lmax) { return fwd(lmax) + ivec(lmax); }
  static __host__ __device__ size_t bytes(int lmax) {
    return toff_at(lmax) + (((size_t)(lmax + 1) * sizeof(long long) + 255) & ~size_t(255));
  }
};

// Per-group scratch of the reverse: the downward-pass vectors, one layer's
// doubling record (layers without a record are recomputed into it), the
// layout-1 phase-cotangent accumulators, the carried d R_base (own tile
// order), the level accumulators and 32 scalars.
template <class Gm>
struct AdjScratch {
  using Tp = TapeLayout<Gm>;
  static constexpr int NP = Gm::NP;
  static __host__ __device__ size_t dvec(int lmax) {
    return ((size_t)(lmax + 1) * 2 * NP * sizeof(double) + 255) & ~size_t(255);
  }
  static __host__ __device__ size_t tape() {
    return ((size_t)Tp::layer(kMaxDoublings) * sizeof(double) + 255) & ~size_t(255);
  }
  // two matrices in tile order (Tp::TILE Reals each: the thread grid can be
  // wider than NP x NP) and two vectors
  static __host__ __device__ size_t pacc() {
    return ((size_t)2 * Tp::TILE * sizeof(double) + 2 * NP * sizeof(double) + 255) & ~size_t(255);
  }
  static __host__ __device__ size_t brb() { return (Tp::TILE * sizeof(double) + 255) & ~size_t(255); }
  static __host__ __device__ size_t acc(int lmax) {
    return ((size_t)4 * (lmax + 1) * sizeof(double) + 255) & ~size_t(255);
  }
  static __host__ __device__ size_t plm(int m) {  // P_l(mu0), l < M
    return ((size_t)m * sizeof(double) + 255) & ~size_t(255);
  }
  static __host__ __device__ size_t svec(int lmax) {  // per layer: p+, p-, q+, q-
    return ((size_t)lmax * 4 * NP * sizeof(double) + 255) & ~size_t(255);
  }
  static __host__ __device__ size_t bytes(int lmax, int m) {
    return dvec(lmax) + tape() + pacc() + brb() + acc(lmax) + 256 + plm(m) + svec(lmax);
  }
};

// The adjoint holds 25 matrices per wavenumber, so few groups fit on an SM;
// at NP = 16 a group is four warps (one 8x8 product tile each) so that the SM
// still runs as many warps as the forward kernel.
template <int NP>
constexpr int adjoint_group() { return (NP == 16) ? 128 : default_group<NP>(); }
template <int NP>
using AdjGeo = Geo<NP, double, adjoint_group<NP>()>;

template <int NP>
struct AdjGroup {
  using GD = AdjGeo<NP>;
  static constexpr size_t bytes =
      align16(CommonLayout<NP>::bytes + TypedLayout<GD, kMatsAdj>::bytes);
};

// Cotangent / gradient pointers of one batch (device).
struct AdjDev {
  const double *c_fu, *c_fd, *c_J, *c_fdir;  // [W*(L+1)] each, or null
  double *g_tau, *g_ssa, *g_mom, *g_temp, *g_planck, *g_semis;
  // one chunk of wavenumbers [w0, w0 + P.ntasks): per-wavenumber states
  // (WavState, state_bytes apart) and the pool of doubling records
  long long w0;
  char* state;
  size_t state_bytes;
  double* pool;
  long long pool_cap;               // doubles
  unsigned long long* pool_used;    // zeroed before each chunk
  // moment sets shared by all wavenumbers (one per layer): their phase
  // matrices ([set][P++, P+-], row-major, pitch NP; null: built per layer),
  // and the per-block sums of the phase-matrix cotangents ([set][block]
  // [P++, P+-] in the reverse group's tile order; null: per layer)
  const double* ptab;
  double* pacc;
  int pacc_blocks;
};

// ---------------------------------------------------------------- doubling adjoint
// Reverse of doubling<Gm> for one layer.  On entry the layer cotangents are
// in (J_bR0, J_bR0c), (J_bT0, J_bT0c) and vectors A_BUP / A_BDN; the phase
// matrices in Ppp / Ppm and the solar phase vectors in D_PP / D_PM.  Writes
// the phase-matrix cotangents to J_T1 (P++) and J_T2 (P+-), the solar phase
// vector cotangents to A_T0 (p+) / A_T1 (p-), and returns the scalar
// cotangents through out[0..4] = d tau, d omega, d B_top, d B_bot, d F_top.
template <class Gm>
__device__ __noinline__ void doubling_adjoint(unsigned goff, unsigned tb, int t_, int bar,
                                              double tau, double om, double Bt, double Bb,
                                              double tcum, int N, bool solar, double F0,
                                              double mu0, const double* Ppp, const double* Ppm,
                                              double* tape, bool recompute, double* out,
                                              int* singular) {
  using Real = typename Gm::Real;
  static_assert(sizeof(Real) == 8, "the adjoint runs in FP64");
  static_assert(kAdjVecs * Gm::NP <= 2 * Gm::MAT, "vector slots fit the two J_VEC buffers");
  using Tp = TapeLayout<Gm>;
  using GC = Geo<Gm::NP, double>;  // record order
  const Ctx<Gm> X(goff, tb, t_, bar);
  constexpr int NP = Gm::NP, TR = Gm::TR, TC = Gm::TC, G = Gm::G;
  constexpr int NWG = G / 32;  // warps of the group (vector work is spread over them)
  const int t = X.t;
  double* red = reinterpret_cast<double*>(X.gjbuf) + 4;  // 4 doubles of reduction scratch
  // 1. the record of this layer's chain: taped by the forward pass, or the
  //    chain again now (buffers 0..5 and V_*)
  const int nn = num_doublings(tau, om > 1.0 ? 1.0 : om);
  if (recompute) {
    int fl = 0;
    doubling<Gm, true>(goff, tb, t_, bar, tau, om, Bt, Bb, tcum, N, solar, F0, mu0, Ppp, Ppm,
                       &fl, tape);
    if (ADRT_GJ_FALLBACK && (fl & kGjWeakPivot)) {  // the chain again, pivoted
      if (t == 0) X.sc[S_PIVALL] = 1.0;
      X.sync();
      fl = kGjWeakPivot;
      doubling<Gm, true>(goff, tb, t_, bar, tau, om, Bt, Bb, tcum, N, solar, F0, mu0, Ppp, Ppm,
                         &fl, tape);
      X.sync();
      if (t == 0) X.sc[S_PIVALL] = 0.0;
    }
    *singular |= fl;
  }
  X.sync();
  const double* mu = X.DV(D_MU);
  const double* wt = X.DV(D_WT);
  const double omc = om > 1.0 ? 1.0 : om;
  const double con = 2.0 * omc * kPi;
  const double tau0 = ldexp(tau, -nn);
  const double Ftop = solar ? F0 * exp(-tcum / mu0) : 0.0;
  Real* vb = X.m(J_VEC);
  auto VA = [&](int s) { return vb + s * NP; };
  auto vo = [&](int s) { return X.mo(J_VEC) + (unsigned)(s * NP * sizeof(Real)); };
  // 2. sources: up = y Bbar + z Bd + su, dn = y Bbar - z Bd + sd
  const double Bbar = 0.5 * (Bb + Bt), Bd = (Bb - Bt) / tau;
  const double* yF = nullptr;
  (void)yF;
  double pBbar = 0.0, pBd = 0.0;
  {
    // final y, z of the chain: the tape's tail
    const double* tail = tape + (size_t)nn * Tp::STEP;
    if (X.warp == 0 && X.lane < NP) {
      const int i = X.lane;
      const double bu = VA(A_BUP)[i], bd = VA(A_BDN)[i];
      const double y = tail[i], z = tail[NP + i];
      VA(A_BY)[i] = (bu + bd) * Bbar;
      VA(A_BZ)[i] = (bu - bd) * Bd;
      VA(A_BSU)[i] = bu;
      VA(A_BSD)[i] = bd;
      pBbar = (bu + bd) * y;
      pBd = (bu - bd) * z;
    }
  }
  pBbar = gsum<G>(pBbar, red, bar);
  pBd = gsum<G>(pBd, red, bar);
  double d_tau = -pBd * Bd / tau;
  const double d_Bb = 0.5 * pBbar + pBd / tau, d_Bt = 0.5 * pBbar - pBd / tau;
  double bg = 0.0, bgam = 0.0;
  int cs = 0;  // which cotangent set holds the current dR, dT
  // the record of step k - 1 is fetched into registers while step k runs
  const Tile<Gm> tlp(t);
  Real nR[TR][TC], nT[TR][TC], nG[TR][TC], nA[TR][TC];
  double nv[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, ngam = 0.0;
  auto fetch = [&](int k) {
    const double* tk = tape + (size_t)k * Tp::STEP;
    if (tlp.valid()) {
#pragma unroll
      for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) {
          const int e = tile_index<GC>(tlp.row(a), tlp.col(b));
          nR[a][b] = tk[Tp::OFF_R + e];
          nT[a][b] = tk[Tp::OFF_T + e];
          nG[a][b] = tk[Tp::OFF_TG + e];
          nA[a][b] = tk[Tp::OFF_AI + e];
        }
    }
    if (X.warp == 0 && X.lane < NP) {
#pragma unroll
      for (int j = 0; j < 4; ++j) nv[j] = tk[Tp::OFF_VEC + j * NP + X.lane];
      if (solar) {
#pragma unroll
        for (int j = 0; j < 3; ++j) nv[4 + j] = tk[Tp::OFF_SOL + j * NP + X.lane];
      }
    }
    ngam = tk[Tp::OFF_VEC + 4 * NP];
  };
  fetch(nn - 1);
  for (int k = nn - 1; k >= 0; --k) {
    const double g = ldexp(tau0, k - 1);
    const double gam = ngam;
    const unsigned bRr = X.mo(cs ? J_bR1 : J_bR0), bRc = X.mo(cs ? J_bR1c : J_bR0c);
    const unsigned bTr = X.mo(cs ? J_bT1 : J_bT0), bTc = X.mo(cs ? J_bT1c : J_bT0c);
    const unsigned nRr = X.mo(cs ? J_bR0 : J_bR1), nRc = X.mo(cs ? J_bR0c : J_bR1c);
    const unsigned nTr = X.mo(cs ? J_bT0 : J_bT1), nTc = X.mo(cs ? J_bT0c : J_bT1c);
    auto gx = [&](unsigned x0, unsigned y0, unsigned x1, unsigned y1, unsigned x2, unsigned y2,
                  unsigned add, unsigned orm, unsigned ocm) {
      GemmX a{};
      a.x[0] = x0; a.y[0] = y0; a.x[1] = x1; a.y[1] = y1; a.x[2] = x2; a.y[2] = y2;
      a.nseg = (x1 == kNoMat) ? 1 : (x2 == kNoMat) ? 2 : 3;
      a.add = add; a.orm = orm; a.ocm = ocm;
      a.nrank = 0;
      return a;
    };
    auto rk = [&](GemmX& a, int s_u, int s_v, double al) {
      a.u[a.nrank] = vo(s_u); a.v[a.nrank] = vo(s_v); a.a[a.nrank] = al; ++a.nrank;
    };
    // 1. this step's record; h = z + g y
    X.sync();
    // the step's record (fetched during the step before): R (rm + cm), T (cm),
    // TG^T (rm + cm), (I - R R)^{-1} (cm) and y, z, s_up, s_dn
    if (tlp.valid()) {
      tlp.store_rm(nR, X.m(J_R));
      tlp.store_cm(nR, X.m(J_Rc));
      tlp.store_cm(nT, X.m(J_Tc));
      tlp.store_rm(nG, X.m(J_TGc));
      tlp.store_cm(nG, X.m(J_TG));
      tlp.store_cm(nA, X.m(J_Ac));
    }
    if (X.warp == 0 && X.lane < NP) {
      const int i = X.lane;
      VA(A_Y)[i] = nv[0];
      VA(A_Z)[i] = nv[1];
      VA(A_H)[i] = nv[1] + g * nv[0];
      VA(A_SU)[i] = nv[2];
      VA(A_SD)[i] = nv[3];
      VA(A_RU)[i] = nv[4];  // R sd + gam su
      VA(A_RD)[i] = nv[5];  // gam R su + sd
      VA(A_X6)[i] = nv[6];  // R su
    }
    if (k > 0) fetch(k - 1);
    X.sync();
    // 2. TGR = TG R;  dTGR = dR T^T - bz h^T + by y^T
    op_gemm_x<Gm, 1, 0>(gx(X.mo(J_TGc), X.mo(J_R), kNoMat, kNoMat, kNoMat, kNoMat, kNoMat,
                           X.mo(J_TGR), kNoMat), t);
    {
      GemmX a = gx(bRc, X.mo(J_Tc), kNoMat, kNoMat, kNoMat, kNoMat, kNoMat, X.mo(J_bTGR),
                   X.mo(J_bTGRc));
      rk(a, A_BZ, A_H, -1.0);
      rk(a, A_BY, A_Y, 1.0);
      op_gemm_x<Gm, 1, 2>(a, t);
    }
    X.sync();
    // 3. dTG = dTGR R^T + dT T^T + bz h^T + by y^T + bsu ru^T + bsd rd^T (column-major)
    {
      GemmX a = gx(X.mo(J_bTGRc), X.mo(J_Rc), bTc, X.mo(J_Tc), kNoMat, kNoMat, kNoMat, kNoMat,
                   X.mo(J_bTG));
      rk(a, A_BZ, A_H, 1.0);
      rk(a, A_BY, A_Y, 1.0);
      rk(a, A_BSU, A_RU, 1.0);
      rk(a, A_BSD, A_RD, 1.0);
      op_gemm_x<Gm, 2, 4>(a, t);
    }
    X.sync();
    // 4. W = dTG A^{-T} = dTG ((I - R R)^{-1})^T
    op_gemm_x<Gm, 1, 0>(gx(X.mo(J_bTG), X.mo(J_Ac), kNoMat, kNoMat, kNoMat, kNoMat, kNoMat,
                           X.mo(J_W), kNoMat), t);
    X.sync();
    // 5. C = TG^T W (= -dA);  dT' = TG^T dT + TGR^T dR + W;  the vector cotangents
    op_gemm_x<Gm, 1, 0>(gx(X.mo(J_TG), X.mo(J_W), kNoMat, kNoMat, kNoMat, kNoMat, kNoMat,
                           X.mo(J_C), X.mo(J_Cc)), t);
    op_gemm_x<Gm, 2, 0>(gx(X.mo(J_TG), bTr, X.mo(J_TGR), bRr, kNoMat, kNoMat, X.mo(J_W), nTr,
                           nTc), t);
    // the vector cotangents' products, one warp each; R^T TG^T = TGR^T turns
    // the next phase's R^T brd, R^T bru into TGR^T bsd, TGR^T bsu, here
    if (X.warp == 0) {
      const Real* v0[2] = {VA(A_BSD), VA(A_BSU)};
      Real rt[2];
      matvec<Gm, true, 2>(X.m(J_TGR), v0, rt, X.lane);
      if (X.lane < NP) {
        VA(A_X4)[X.lane] = rt[0];
        VA(A_X5)[X.lane] = rt[1];
      }
    }
    if (X.warp == 1 % NWG) {
      const Real* v1[2] = {VA(A_BSU), VA(A_BSD)};
      Real tgs[2];
      matvec<Gm, true, 2>(X.m(J_TG), v1, tgs, X.lane);  // TG^T bsu, TG^T bsd
      if (X.lane < NP) {
        VA(A_BRU)[X.lane] = tgs[0];
        VA(A_BRD)[X.lane] = tgs[1];
      }
    }
    if (X.warp == 2 % NWG) {
      const Real* v2[2] = {VA(A_BZ), VA(A_BY)};
      Real tgz[2];
      matvec<Gm, true, 2>(X.m(J_TG), v2, tgz, X.lane);  // TG^T bz, TG^T by
      if (X.lane < NP) {
        VA(A_X0)[X.lane] = tgz[0];
        VA(A_X1)[X.lane] = tgz[1];
      }
    }
    if (X.warp == 3 % NWG) {
      const Real* v2[2] = {VA(A_BZ), VA(A_BY)};
      Real trz[2];
      matvec<Gm, true, 2>(X.m(J_TGR), v2, trz, X.lane);  // TGR^T bz, TGR^T by
      if (X.lane < NP) {
        VA(A_X2)[X.lane] = trz[0];
        VA(A_X3)[X.lane] = trz[1];
      }
    }
    X.sync();
    // 6. dR' = TG^T dTGR + C R^T + R^T C + dR + bru sd^T + gam brd su^T; the
    //    vector cotangents of the step before (reductions read after the next barrier)
    {
      GemmX a = gx(X.mo(J_TG), X.mo(J_bTGR), X.mo(J_Cc), X.mo(J_Rc), X.mo(J_R), X.mo(J_C), bRr,
                   nRr, nRc);
      rk(a, A_BRU, A_SD, 1.0);
      rk(a, A_BRD, A_SU, gam);
      op_gemm_x<Gm, 3, 2>(a, t);
    }
    if (X.warp == 1 % NWG && X.lane < NP) {
      // g and gamma's cotangents obey bg' = pg + 2 bg, bgam' = pgam + 2 gam bgam,
      // linear in the per-row terms: each lane carries its rows' share, summed
      // after the chain
      const int i = X.lane;
      const double bz = VA(A_BZ)[i], by = VA(A_BY)[i];
      const double bh = VA(A_X0)[i] - VA(A_X2)[i];    // (TG - TGR)^T bz
      const double bt0 = VA(A_X1)[i] + VA(A_X3)[i];   // (TG + TGR)^T by
      const double bsu = VA(A_BSU)[i], bsd = VA(A_BSD)[i];
      const double y = VA(A_Y)[i], su = VA(A_SU)[i], sd = VA(A_SD)[i];
      const double bru = VA(A_BRU)[i], brd = VA(A_BRD)[i];
      const double rtd = VA(A_X4)[i], rtu = VA(A_X5)[i], rsu = VA(A_X6)[i];
      bg = (-y * bz + y * bh) + 2.0 * bg;
      bgam = (sd * bsd + su * bru + rsu * brd) + 2.0 * gam * bgam;
      VA(A_BZ)[i] = bz + bh;
      VA(A_BY)[i] = -g * bz + bt0 + by + g * bh;
      VA(A_BSU)[i] = bsu + gam * bru + gam * rtd;
      VA(A_BSD)[i] = gam * bsd + rtu + brd;
    }
    cs ^= 1;
  }
  X.sync();
  bg = gsum<G>(bg, red, bar);
  bgam = gsum<G>(bgam, red, bar);
  // 3. first-order start: T0 = I - tau0 Gpp, R0 = tau0 Gpm, y0 = (1-om) tau0/mu,
  //    su0 / sd0 = om tau0 Ftop p-/p+ / mu, g0 = tau0/2, gam0 = exp(-tau0/mu0)
  const unsigned bRr = X.mo(cs ? J_bR1 : J_bR0), bTr = X.mo(cs ? J_bT1 : J_bT0);
  double p_tau0 = 0.0, p_con = 0.0;
  {
    const Tile<Gm> tl(t);
    if (tl.valid()) {
      const Real* dR = sp<Real>(bRr);
      const Real* dT = sp<Real>(bTr);
      Real* dPpp = X.m(J_T1);
      Real* dPpm = X.m(J_T2);
#pragma unroll
      for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) {
          const int r = tl.row(a), c = tl.col(b);
          double gp = 0.0, gm = 0.0;
          if (r < N && c < N) {
            const double dt = dT[r * Gm::LD + c], dr = dR[r * Gm::LD + c];
            const double fw = wt[c] / mu[r];
            const double pp = Ppp[r * NP + c], pm = Ppm[r * NP + c];
            p_tau0 += dt * (con * pp * fw - ((r == c) ? 1.0 / mu[r] : 0.0)) + dr * con * pm * fw;
            p_con += tau0 * fw * (dt * pp + dr * pm);
            gp = dt * tau0 * con * fw;
            gm = dr * tau0 * con * fw;
          }
          dPpp[r * Gm::LD + c] = gp;
          dPpm[r * Gm::LD + c] = gm;
        }
    }
  }
  double p_om = 0.0, p_ftop = 0.0;
  if (X.warp == 0 && X.lane < NP) {
    const int i = X.lane;
    double dpp = 0.0, dpm = 0.0;
    if (i < N) {
      const double by = VA(A_BY)[i];
      p_tau0 += by * (1.0 - omc) / mu[i];
      p_om -= by * tau0 / mu[i];
      if (solar) {
        const double bsu = VA(A_BSU)[i], bsd = VA(A_BSD)[i];
        const double pm = X.DV(D_PM)[i], pp = X.DV(D_PP)[i];
        const double bb = bsu * pm + bsd * pp;
        p_om += bb * tau0 * Ftop / mu[i];
        p_tau0 += bb * omc * Ftop / mu[i];
        p_ftop += bb * omc * tau0 / mu[i];
        const double base = omc * tau0 / mu[i] * Ftop;
        dpm = bsu * base;
        dpp = bsd * base;
      }
    }
    VA(A_T0)[i] = dpp;
    VA(A_T1)[i] = dpm;
  }
  p_tau0 = gsum<G>(p_tau0, red, bar);
  p_con = gsum<G>(p_con, red, bar);
  p_om = gsum<G>(p_om, red, bar);
  p_ftop = gsum<G>(p_ftop, red, bar);
  p_tau0 += 0.5 * bg;
  if (solar) p_tau0 += bgam * (-exp(-tau0 / mu0) / mu0);
  p_om += 2.0 * kPi * p_con;
  d_tau += p_tau0 * ldexp(1.0, -nn);
  if (t == 0) {
    out[0] = d_tau;
    out[1] = (om > 1.0) ? 0.0 : p_om;
    out[2] = d_Bt;
    out[3] = d_Bb;
    out[4] = p_ftop;
  }
  X.sync();
}

// ---------------------------------------------------------------- phase adjoint
// Cotangents of the phase moments from those of P++ (J_T1), P+- (J_T2) and of
// the solar phase vectors (A_T0 = p+, A_T1 = p-), through the Hansen column
// renormalisation (src/phase_matrix.hpp:61-111, 131-181).  Adds into dchi[l]
// for l < nuse (global, atomically).  The two parts are linear in their
// cotangents and independent: MAT the matrices' (which, for a moment set
// shared by all wavenumbers, runs once on the cotangents summed over them),
// SOL the solar vectors' (which depend on each wavenumber's mu0; plm0[l] =
// P_l(mu0) for l < nuse, the un-normalised vectors in D_LAM0 / D_LAM1 as
// build_phase<Gm, true> leaves them).
//
// With delta-M truncation (f >= 0: the forward used chi*_l = (chi_l - f) /
// (1 - f) for l < nuse = 2N, f = chi_2N, src/solver.cpp:441-501) the cotangent
// of chi*_l reaches chi_l as 1 / (1 - f) and chi_2N as (chi_l - 1) / (1 - f)^2.
template <class Gm, bool MAT = true, bool SOL = true>
__device__ __noinline__ void phase_adjoint(unsigned goff, unsigned tb, int t_, int bar,
                                           const double* chi, int nuse, int N, const double* pl,
                                           bool solar, double mu0, double* dchi,
                                           const double* plm0, double f = -1.0) {
  using Real = typename Gm::Real;
  const Ctx<Gm> X(goff, tb, t_, bar);
  constexpr int NP = Gm::NP, G = Gm::G, LD = Gm::LD;
  const int t = X.t;
  const double* wt = X.DV(D_WT);
  Real* dPpp = X.m(J_T1);
  Real* dPpm = X.m(J_T2);
  Real* Qpp = X.m(J_W);
  Real* Qpm = X.m(J_C);
  Real* vb = X.m(J_VEC);
  Real* sarr = vb + A_BY * NP;   // column sums s_j
  Real* carr = vb + A_BZ * NP;   // corr_j
  Real* bsar = vb + A_BSU * NP;  // d s_j
  Real* qp = vb + A_H * NP;
  Real* qm = vb + A_RU * NP;
  solar = SOL && solar;
  const double inv_1mf = (f >= 0.0) ? 1.0 / (1.0 - f) : 1.0;
  // the cotangent v of the effective moment l, into the inputs' moments
  auto add_moment = [&](int l, double v) {
    if (f >= 0.0) {
      atomicAdd(&dchi[l], v * inv_1mf);
      atomicAdd(&dchi[nuse], v * (chi[l] - 1.0) * inv_1mf * inv_1mf);
    } else {
      atomicAdd(&dchi[l], v);
    }
  };
  if constexpr (MAT) {
    // un-normalised Q
    if constexpr (UsePhaseMMA<Gm>::value)
      phase_products<Gm>(chi, nuse, f, N, pl, Qpp, Qpm, LD, t);
    else
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
      }
      Qpp[r * LD + c] = spp / (2.0 * kPi);
      Qpm[r * LD + c] = spm / (2.0 * kPi);
    }
    X.sync();
    if (t < NP) {
      const int c = t;
      double s = 0.0, bc = 0.0;
      for (int i = 0; i < N; ++i) s += (Qpp[i * LD + c] + Qpm[i * LD + c]) * wt[i];
      const double corr = (s > 0.0) ? 1.0 / (2.0 * kPi * s) : 1.0;
      for (int i = 0; i < N; ++i)
        bc += dPpp[i * LD + c] * Qpp[i * LD + c] + dPpm[i * LD + c] * Qpm[i * LD + c];
      sarr[c] = s;
      carr[c] = corr;
      bsar[c] = (s > 0.0) ? -bc * corr / s : 0.0;
    }
    X.sync();
    for (int e = t; e < NP * NP; e += G) {  // dQ = dP corr_j + w_i ds_j (in place)
      const int r = e / NP, c = e % NP;
      dPpp[r * LD + c] = dPpp[r * LD + c] * carr[c] + wt[r] * bsar[c];
      dPpm[r * LD + c] = dPpm[r * LD + c] * carr[c] + wt[r] * bsar[c];
    }
  }
  double bqscale = 0.0;
  if (solar) {
    // the un-normalised solar vectors (left in D_LAM0 / D_LAM1 by the build)
    // and their normalisation
    const double* qpu = X.DV(D_LAM0);
    const double* qmu = X.DV(D_LAM1);
    const Real* dpp = vb + A_T0 * NP;
    const Real* dpm = vb + A_T1 * NP;
    double ss = 0.0, bcs = 0.0;
#pragma unroll
    for (int i = 0; i < NP; ++i)
      if (i < N) ss += (qpu[i] + qmu[i]) * wt[i];
    const double cs = (ss > 0.0) ? 1.0 / (2.0 * kPi * ss) : 1.0;
#pragma unroll
    for (int i = 0; i < NP; ++i)
      if (i < N) bcs += dpp[i] * qpu[i] + dpm[i] * qmu[i];
    bqscale = (ss > 0.0) ? -bcs * cs / ss : 0.0;
    X.sync();
    if (t < NP) {  // dq = dp cs + w dss
      qp[t] = dpp[t] * cs + wt[t] * bqscale;
      qm[t] = dpm[t] * cs + wt[t] * bqscale;
    }
  }
  X.sync();
  // dchi_l = (2l+1)/(2 pi) [P_l^T (dQpp + s_l dQpm) P_l + p0_l P_l . (dqp + s_l dqm)]
  bool forms_done = !MAT;
  if constexpr (MAT && UsePhaseMMA<Gm>::value) {
    // the quadratic forms on the tensor cores: V = S B with S = dQpp + dQpm
    // (even l) or dQpp - dQpm (odd l) and B[j][k] = P_l(k)(mu_j), l(k) = 2k or
    // 2k + 1; the form of moment l(k) is column k of V dotted with P_l(k)(mu_.)
    constexpr int NT = NP / 8, NW = G / 32;
    const int warp = t >> 5, lane = t & 31, g = lane >> 2, q = lane & 3;
    const int kt = (((nuse + 1) >> 1) + 7) >> 3;  // 8-column tiles of moments per parity
    for (int tau = warp; tau < 2 * NT * kt; tau += NW) {
      const int par = tau / (NT * kt), i = (tau % (NT * kt)) / kt, jt = tau % kt;
      const double sg = par ? -1.0 : 1.0;
      const int r = 8 * i + g, lb = 2 * (8 * jt + g) + par;
      double v0 = 0.0, v1 = 0.0;
#pragma unroll
      for (int ks = 0; ks < NP / 4; ++ks) {
        const int j = 4 * ks + q;
        const double a = dPpp[r * LD + j] + sg * dPpm[r * LD + j];
        const double b = (j < N && lb < nuse) ? pl[lb * N + j] : 0.0;
        mma_f64_m8n8k4(v0, v1, a, b);
      }
      const int l0 = 2 * (8 * jt + 2 * q) + par, l1 = l0 + 2;  // columns 2q, 2q + 1
      double s0 = (r < N && l0 < nuse) ? v0 * pl[l0 * N + r] : 0.0;
      double s1 = (r < N && l1 < nuse) ? v1 * pl[l1 * N + r] : 0.0;
#pragma unroll
      for (int o = 4; o < 32; o <<= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      }
      if (g == 0) {
        if (l0 < nuse) add_moment(l0, (2 * l0 + 1) * s0 / (2.0 * kPi));
        if (l1 < nuse) add_moment(l1, (2 * l1 + 1) * s1 / (2.0 * kPi));
      }
    }
    forms_done = true;
  }
  if (!forms_done || solar) {
    for (int l = t; l < nuse; l += G) {
      const double sg = (l & 1) ? -1.0 : 1.0;
      double acc = 0.0;
      if (!forms_done) {
        for (int i = 0; i < N; ++i) {
          double ri = 0.0;
          for (int j = 0; j < N; ++j)
            ri += (dPpp[i * LD + j] + sg * dPpm[i * LD + j]) * pl[l * N + j];
          acc += pl[l * N + i] * ri;
        }
      }
      if (solar) {
        const double plm = plm0[l];
        double sv = 0.0;
#pragma unroll
        for (int i = 0; i < NP; ++i)
          if (i < N) sv += pl[l * N + i] * (qp[i] + sg * qm[i]);
        acc += plm * sv;
      }
      add_moment(l, (2 * l + 1) * acc / (2.0 * kPi));
    }
  }
  X.sync();
}


// Effective moment count and delta-M fraction of a moment set, as the forward
// pass forms them (f < 0: no truncation scaling).
__device__ __forceinline__ void moment_use(const ColumnDev* C, const double* chi, int& nuse,
                                           double& f) {
  const int N = C->N, M = C->M;
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
}

// ---------------------------------------------------------------- one wavenumber
// Runs on the state a taping forward left for wavenumber w (WavState: the
// slot with levels, phase matrices and records in GC's tile order, the
// interface intensities, the record offsets), with the group's scratch.
template <int NP>
__device__ __noinline__ void wav_adjoint(unsigned goff, unsigned tb, int t_, int bar, int w,
                                         char* slot, char* scr, int lmax, unsigned* status,
                                         AdjDev AD) {
  using Gm = AdjGeo<NP>;
  using GC = Geo<NP, double>;  // the taping forward's geometry: record order
  using Real = double;
  using SLay = SlotLayout<Gm>;
  using WS = WavState<GC>;
  using AS = AdjScratch<Gm>;
  constexpr int TILE = SLay::TILE, REC = SLay::REC, G = Gm::G, TR = Gm::TR, TC = Gm::TC;
  constexpr int LD = Gm::LD;
  const Ctx<Gm> X(goff, tb, t_, bar);
  const ColumnDev* C = X.col;
  const int t = X.t;
  const int N = C->N, nL = C->L, M = C->M, layout = C->moment_layout, fb = C->from_bottom;
  const double Aalb = C->albedo_w ? C->albedo_w[w] : C->surface_albedo;
  const double mu0 = C->mu0_w ? C->mu0_w[w] : C->solar_mu;
  const double wlo = C->wlo_w ? C->wlo_w[w] : C->wn_lo;
  const double whi = C->whi_w ? C->whi_w[w] : C->wn_hi;
  const double F0 = C->solar_flux;
  const bool solar = (F0 > 0.0 && mu0 > 0.0);
  const Levels lv(slot, lmax);
  double* Ppp = reinterpret_cast<double*>(slot + SLay::level_bytes(lmax));
  double* Ppm = Ppp + NP * NP;
  double* recs = reinterpret_cast<double*>(slot + SLay::level_bytes(lmax) + SLay::phase_bytes());
  double* iv = reinterpret_cast<double*>(slot + WS::fwd(lmax));   // [L+1][Id, Iu]
  const long long* toff = reinterpret_cast<const long long*>(slot + WS::toff_at(lmax));
  char* p = scr;
  double* dv = reinterpret_cast<double*>(p);                      // [L+1][brhs, u]
  double* tape = reinterpret_cast<double*>(p += AS::dvec(lmax));
  double* pacc = reinterpret_cast<double*>(p += AS::tape());      // dPpp, dPpm, dpp, dpm
  double* brb = reinterpret_cast<double*>(p += AS::pacc());       // carried d R_base (tiles)
  double* acc = reinterpret_cast<double*>(p += AS::brb());        // bB, btc, dtau, dom
  double* scal = reinterpret_cast<double*>(p += AS::acc(lmax));   // 32 doubles
  double* plm0 = reinterpret_cast<double*>(p += 256);              // P_l(mu0), l < M
  double* svec = reinterpret_cast<double*>(p += AS::plm(M));       // [L][p+, p-, q+, q-]
  const long long tbase = toff[nL];                               // this wavenumber's records
  double* tape_all = (tbase >= 0) ? AD.pool + tbase : nullptr;
  double* bB = acc;
  double* btc = acc + (lmax + 1);
  double* gtau = acc + 2 * (lmax + 1);
  double* gom = acc + 3 * (lmax + 1);
  const double Bs = X.sc[S_BS], Btop = X.sc[S_BTOP];
  const bool has_surface = !C->diffusion && (Aalb > 0.0 || Bs > 0.0);
  const double* cw = X.DV(D_CW);
  const double* hw = X.DV(D_HW);
  const size_t wo = (size_t)w * (nL + 1);
  auto ui = [&](int l) { return fb ? nL - l : l; };  // user level index
  // moment set of internal layer l, its effective count and delta-M fraction
  auto moments = [&](int l, int& nuse, double& f) -> const double* {
    const int u = fb ? nL - 1 - l : l;
    const double* chi = C->moments + (layout == 0 ? (size_t)u * M
                                      : layout == 1 ? (size_t)w * M
                                                    : ((size_t)w * nL + u) * M);
    moment_use(C, chi, nuse, f);
    return chi;
  };
  auto cot = [&](const double* a, int l) { return a ? a[wo + ui(l)] : 0.0; };
  Real* vb = X.m(J_VEC);
  auto VA = [&](int s) { return vb + s * NP; };
  auto vo = [&](int s) { return X.mo(J_VEC) + (unsigned)(s * NP * sizeof(Real)); };
  const Tile<Gm> tl(t);
  int singular = 0;
  const bool table = (layout == 0) && (AD.ptab != nullptr);

  for (int l = t; l <= nL; l += G) {
    bB[l] = 0.0;
    btc[l] = 0.0;
    gtau[l] = 0.0;
    gom[l] = 0.0;
  }
  for (int e = t; e < 2 * TILE + 2 * NP; e += G) pacc[e] = 0.0;
  if (solar && t == 0) {  // P_l(mu0) by the recurrence the phase vectors use
    double p0 = 1.0, p1 = mu0;
    for (int l = 0; l < M; ++l) {
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
      plm0[l] = plm;
    }
  }
  X.sync();
  if (table && solar) {
    // every layer's solar phase vectors at once (they depend on the layer's
    // moments and this wavenumber's mu0): q = sum_k (2k+1) chi_k P_k(mu_i)
    // P_k(mu0) / 2 pi with the sign (-1)^k for q-, then p = q / (2 pi s)
    for (int e = t; e < nL * NP; e += G) {
      const int l = e / NP, i = e - l * NP;
      double sp = 0.0, sm = 0.0;
      if (i < N) {
        int nuse;
        double f;
        const double* chi = moments(l, nuse, f);
        const double inv_1mf = (f >= 0.0) ? 1.0 / (1.0 - f) : 1.0;
        for (int k0 = 0; k0 < nuse; k0 += 8) {
          double c[8], pk[8], q[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int k = (k0 + j < nuse) ? k0 + j : 0;
            c[j] = chi[k];
            pk[j] = C->quad.pl[k * N + i];
            q[j] = plm0[k];
          }
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int k = k0 + j;
            if (k < nuse) {
              const double cl = (f >= 0.0) ? (c[j] - f) * inv_1mf : c[j];
              const double term = (2 * k + 1) * cl * pk[j] * q[j];
              sp += term;
              sm += (k & 1) ? -term : term;
            }
          }
        }
        sp /= (2.0 * kPi);
        sm /= (2.0 * kPi);
      }
      svec[(size_t)l * 4 * NP + 2 * NP + i] = sp;
      svec[(size_t)l * 4 * NP + 3 * NP + i] = sm;
    }
    X.sync();
    const double* wq = X.DV(D_WT);
    for (int l = t; l < nL; l += G) {
      double* q = svec + (size_t)l * 4 * NP;
      double qp[NP], qm[NP];
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        qp[i] = q[2 * NP + i];
        qm[i] = q[3 * NP + i];
      }
      double ss = 0.0;
#pragma unroll
      for (int i = 0; i < NP; ++i)
        if (i < N) ss += (qp[i] + qm[i]) * wq[i];
      const double cs = (ss > 0.0) ? 1.0 / (2.0 * kPi * ss) : 1.0;
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        q[i] = (i < N) ? qp[i] * cs : qp[i];
        q[NP + i] = (i < N) ? qm[i] * cs : qm[i];
      }
    }
    X.sync();
  }

  // ======== 1. downward-pass adjoint (interface L-1 .. 0); bId carried in A_BDN
  if (X.warp == 0 && X.lane < NP) {
    const int i = X.lane;
    VA(A_BDN)[i] = (i < N) ? cot(AD.c_fd, nL) * cw[i] + cot(AD.c_J, nL) * hw[i] : 0.0;
  }
  for (int l = nL - 1; l >= 0; --l) {
    const double* rl = recs + (size_t)l * REC;
    const double* rb = recs + (size_t)(l + 1) * REC;
    const int scat = rl[3 * TILE + 2 * NP] != 0.0;
    const int cb = rb[3 * TILE + 2 * NP + 1] != 0.0;
    X.sync();
    {  // R_base(l+1), R_l, T_l (rm)
      const double* g[3] = {rb + 2 * TILE, rl, rl + TILE};
      const unsigned orm[3] = {X.mo(J_TGR), X.mo(J_R), X.mo(J_TG)};
      const unsigned ocm[3] = {X.mo(J_TGc), X.mo(J_Rc), kNoMat};
      g2s_n<Gm, GC, 3, 0u>(g, orm, ocm, t);
    }
    X.sync();
    if (X.warp == 0) {  // bIu(l+1), bx = Rb^T bIu + bId
      if (X.lane < NP) {
        const int i = X.lane;
        VA(A_BUP)[i] = (i < N) ? cot(AD.c_fu, l + 1) * cw[i] + cot(AD.c_J, l + 1) * hw[i] : 0.0;
      }
      __syncwarp();
      const Real* vv[1] = {VA(A_BUP)};
      Real yv[1];
      matvec<Gm, true, 1>(X.m(J_TGR), vv, yv, X.lane);  // Rb^T bIu
      if (X.lane < NP) VA(A_Y)[X.lane] = yv[0] + VA(A_BDN)[X.lane];
    }
    X.sync();
    const Real* brhs = VA(A_Y);
    int bstride = 1;
    if (scat && cb) {  // b_rhs = M^{-T} bx with M = I - R Rb, as b_rhs^T = bx^T M^{-1}
      op_gemm<Gm>(X.mo(J_Rc), X.mo(J_TGR), kNoMat, 1, X.mo(J_T1), kNoMat, t);
      X.sync();
      singular |= op_gj_safe<Gm>(X.mo(J_T1), kNoMat, vo(A_Y), X.mo(J_T2), X.gjo(), X.redo(), t, X.bar);
      X.sync();
      brhs = X.m(J_T2);
      bstride = LD;
    }
    if (X.warp == 0) {
      if (X.lane < NP) VA(A_Z)[X.lane] = brhs[X.lane * bstride];
      __syncwarp();
      const Real* vv[1] = {VA(A_Z)};
      Real rt[1], tt[1];
      matvec<Gm, true, 1>(X.m(J_R), vv, rt, X.lane);   // R^T b_rhs
      matvec<Gm, true, 1>(X.m(J_TG), vv, tt, X.lane);  // T^T b_rhs
      if (X.lane < NP) {
        const int i = X.lane;
        const double br = VA(A_Z)[i];
        dv[(size_t)l * 2 * NP + i] = br;
        dv[(size_t)(l + 1) * 2 * NP + NP + i] = VA(A_BUP)[i] + (scat ? rt[0] : 0.0);
        VA(A_BDN)[i] = tt[0] + ((i < N) ? cot(AD.c_fd, l) * cw[i] + cot(AD.c_J, l) * hw[i] : 0.0);
      }
    }
  }
  X.sync();
  // interface 0: Iu0 = Rb0 Id0 + Ub0, Id0 = Btop
  op_g2s<Gm, GC>(recs + 2 * TILE, X.mo(J_TGR), kNoMat, t);
  X.sync();
  double pBtop = 0.0;
  if (X.warp == 0) {
    if (X.lane < NP) {
      const int i = X.lane;
      VA(A_BUP)[i] = (i < N) ? cot(AD.c_fu, 0) * cw[i] + cot(AD.c_J, 0) * hw[i] : 0.0;
      dv[NP + i] = VA(A_BUP)[i];
    }
    __syncwarp();
    const Real* vv[1] = {VA(A_BUP)};
    Real yv[1];
    matvec<Gm, true, 1>(X.m(J_TGR), vv, yv, X.lane);
    if (X.lane < N) pBtop = VA(A_BDN)[X.lane] + yv[0];
  }
  pBtop = gsum<G>(pBtop, reinterpret_cast<double*>(X.gjbuf) + 4, bar);
  // beam outputs: F_dir and the beam term of J depend on the cumulative tau
  if (solar && t == 0) {
    for (int l = 1; l <= nL; ++l) {
      const double e = F0 * mu0 * exp(-lv.tc[l] / mu0);
      btc[l] += (cot(AD.c_fdir, l) + cot(AD.c_J, l) / (4.0 * kPi * mu0)) * e * (-1.0 / mu0);
    }
  }

  // ======== 2. adding adjoint, layer 0 .. L-1, with each layer's own chain
  // carried: d R_base(l) in brb (tiles), d U_base(l) in A_CUB
  {  // interface 0: d Rb0 = u0 Id0^T, d Ub0 = u0
    double* tu = VA(A_BUP);
    if (X.warp == 0 && X.lane < NP) {
      tu[X.lane] = dv[NP + X.lane];
      VA(A_CUB)[X.lane] = dv[NP + X.lane];
      VA(A_SD)[X.lane] = iv[X.lane];  // Id0
    }
    X.sync();
    if (tl.valid()) {
      double* pb = brb + t * Gm::TE;
#pragma unroll
      for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) pb[a * TC + b] = tu[tl.row(a)] * VA(A_SD)[tl.col(b)];
    }
  }
  int nuse_l1 = M;
  double f_l1 = -1.0;
  if (layout == 1) {  // one moment set per wavenumber: the solar phase vectors once
    int nuse;
    double f;
    const double* chi = moments(0, nuse, f);
    nuse_l1 = nuse;
    f_l1 = f;
    build_phase<Gm, true>(X.goff, X.tb, t, X.bar, chi, nuse, f, N, C->quad.pl, solar, mu0, Ppp,
                          Ppm, plm0);
  }
  for (int l = 0; l < nL; ++l) {
    const double* rl = recs + (size_t)l * REC;
    const double* rb = recs + (size_t)(l + 1) * REC;
    const int scat = rl[3 * TILE + 2 * NP] != 0.0;
    const int cb = rb[3 * TILE + 2 * NP + 1] != 0.0;
    const double tau = lv.tau[l], om = lv.om[l];
    X.sync();
    {  // R_l, T_l, R_base(l+1) (records) and the carried d R_base (own order)
      const double* g[4] = {rl, rl + TILE, rb + 2 * TILE, brb};
      const unsigned orm[4] = {X.mo(J_R), X.mo(J_TG), X.mo(J_TGR), X.mo(J_bTGR)};
      const unsigned ocm[4] = {X.mo(J_Rc), X.mo(J_Tc), X.mo(J_TGc), X.mo(J_bTGRc)};
      g2s_n<Gm, GC, 4, 8u>(g, orm, ocm, t);
    }
    if (X.warp == 0 && X.lane < NP) {
      const int i = X.lane;
      VA(A_Y)[i] = dv[(size_t)l * 2 * NP + i];                           // b_rhs(l)
      VA(A_Z)[i] = iv[(size_t)l * 2 * NP + i];                           // Id(l)
      VA(A_H)[i] = (scat && cb) ? iv[(size_t)(l + 1) * 2 * NP + NP + i]  // b_l
                                : rb[3 * TILE + NP + i];
      VA(A_RU)[i] = rb[3 * TILE + NP + i];  // U_base(l+1)
      VA(A_RD)[i] = rl[3 * TILE + i];       // s_dn(l)
      VA(A_BH)[i] = rl[3 * TILE + 2 * NP + 2 + i];  // s_up(l)
      VA(A_BDN)[i] = VA(A_Y)[i];            // d s_dn starts at b_rhs
      VA(A_BUP)[i] = VA(A_CUB)[i];           // d s_up = d U_base(l)
    }
    X.sync();
    if (scat && cb) {
      // ---- general: A1 = I - Rb R, D1 = T A1^{-1}
      op_gemm<Gm>(X.mo(J_TGc), X.mo(J_R), kNoMat, 1, X.mo(J_bR1), X.mo(J_bR1c), t);
      X.sync();
      singular |= op_gj_safe<Gm>(X.mo(J_bR1), X.mo(J_TG), kNoMat, X.mo(J_bT1c), X.gjo(), X.redo(), t,
                            X.bar, X.mo(J_bT1));
      X.sync();
      op_gemm<Gm>(X.mo(J_TGc), X.mo(J_TG), kNoMat, 0, X.mo(J_W), X.mo(J_Ac), t);   // Q = Rb T
      op_gemm<Gm>(X.mo(J_bT1), X.mo(J_bTGR), kNoMat, 0, X.mo(J_C), X.mo(J_Cc), t);  // E = D1^T dRb
      op_gemm<Gm>(X.mo(J_bT1c), X.mo(J_TGR), kNoMat, 0, X.mo(J_T1), kNoMat, t);     // F = D1 Rb
      if (X.warp == 0) {
        const Real* v1[1] = {VA(A_RD)};
        Real rbd[1];
        matvec<Gm, true, 1>(X.m(J_TGc), v1, rbd, X.lane);  // Rb s_dn
        const Real* v2[1] = {VA(A_CUB)};
        Real bvv[1];
        matvec<Gm, true, 1>(X.m(J_bT1), v2, bvv, X.lane);  // bv = D1^T dUb
        if (X.lane < NP) {
          VA(A_T0)[X.lane] = VA(A_RU)[X.lane] + rbd[0];  // v = Ub1 + Rb s_dn
          VA(A_T1)[X.lane] = bvv[0];
        }
        __syncwarp();
        const Real* v3[1] = {VA(A_T1)};
        Real rtb[1];
        matvec<Gm, true, 1>(X.m(J_TGR), v3, rtb, X.lane);  // Rb^T bv
        if (X.lane < NP) VA(A_BDN)[X.lane] += rtb[0];
      }
      X.sync();
      // dD1 = dRb Q^T + dUb v^T
      op_gemm<Gm>(X.mo(J_bTGRc), X.mo(J_Ac), kNoMat, 0, X.mo(J_bTG), kNoMat, t);
      X.sync();
      op_rank<Gm>(X.mo(J_bTG), kNoMat, vo(A_CUB), vo(A_T0), 1.0, kNoMat, kNoMat, 0.0, kNoMat,
                  kNoMat, 0.0, kNoMat, kNoMat, 0.0, t);
      X.sync();
      // W = dD1 A1^{-T}
      singular |= op_gj_safe<Gm>(X.mo(J_bR1c), X.mo(J_bTG), kNoMat, kNoMat, X.gjo(), X.redo(), t,
                            X.bar, X.mo(J_T2));
      X.sync();
      // G1 = D1^T W (= -dA1);  dT = F^T dRb + W + b_rhs Id^T
      op_gemm<Gm>(X.mo(J_bT1), X.mo(J_T2), kNoMat, 0, X.mo(J_W), X.mo(J_Ac), t);
      op_gemm<Gm>(X.mo(J_T1), X.mo(J_bTGR), X.mo(J_T2), 0, X.mo(J_bT0), X.mo(J_bT0c), t);
      X.sync();
      // dRb(l+1) = E T^T + G1 R^T + bv s_dn^T (+ u(l+1) Id(l+1)^T below)
      op_gemm<Gm>(X.mo(J_Cc), X.mo(J_Tc), kNoMat, 0, X.mo(J_T1), kNoMat, t);
      X.sync();
      op_gemm<Gm>(X.mo(J_Ac), X.mo(J_Rc), X.mo(J_T1), 0, X.mo(J_bR1), kNoMat, t);
      // dR = dRb + Rb^T G1 + b_rhs b_l^T
      op_gemm<Gm>(X.mo(J_TGR), X.mo(J_W), X.mo(J_bTGR), 0, X.mo(J_bR0), X.mo(J_bR0c), t);
      X.sync();
      op_rank<Gm>(X.mo(J_bR1), kNoMat, vo(A_T1), vo(A_RD), 1.0, kNoMat, kNoMat, 0.0, kNoMat,
                  kNoMat, 0.0, kNoMat, kNoMat, 0.0, t);
      if (X.warp == 0 && X.lane < NP) VA(A_CUB)[X.lane] = VA(A_T1)[X.lane];  // d Ub(l+1) = bv
    } else if (scat) {
      // ---- base below reflects nothing: Ub = s_up + T Ub1, Rb = R
      op_copy<Gm>(X.mo(J_bTGR), X.mo(J_bR0), X.mo(J_bR0c), 1.0, t);
      op_copy<Gm>(X.mo(J_bTGR), X.mo(J_bT0), X.mo(J_bT0c), 0.0, t);
      if (X.warp == 0) {
        const Real* v1[1] = {VA(A_CUB)};
        Real ttb[1];
        matvec<Gm, true, 1>(X.m(J_TG), v1, ttb, X.lane);  // T^T dUb
        __syncwarp();
        if (X.lane < NP) VA(A_T1)[X.lane] = ttb[0];
      }
      X.sync();
      op_rank<Gm>(X.mo(J_bT0), X.mo(J_bT0c), vo(A_CUB), vo(A_RU), 1.0, kNoMat, kNoMat, 0.0,
                  kNoMat, kNoMat, 0.0, kNoMat, kNoMat, 0.0, t);
      op_copy<Gm>(X.mo(J_bTGR), X.mo(J_bR1), kNoMat, 0.0, t);  // no dependence on Rb below
      X.sync();  // the rank update above reads A_CUB
      if (X.warp == 0 && X.lane < NP) VA(A_CUB)[X.lane] = VA(A_T1)[X.lane];
    } else {
      // ---- non-scattering layer: Ub = s_up + t (Ub1 + Rb s_dn), Rb = t Rb1 t
      // its T is diagonal: only diag(dT) = dt is kept (in A_T0)
      if (X.warp == 0) {
        const Real* v1[1] = {VA(A_RD)};
        Real rbd[1];
        matvec<Gm, true, 1>(X.m(J_TGc), v1, rbd, X.lane);  // Rb s_dn
        if (X.lane < NP) {
          const int i = X.lane;
          const double tv = X.m(J_TG)[i * LD + i];
          const double v = VA(A_RU)[i] + rbd[0];
          double dt = VA(A_CUB)[i] * v + VA(A_Y)[i] * VA(A_Z)[i];  // + b_rhs Id (diag)
          const Real* dRb = X.m(J_bTGR);
          const Real* Rb1 = X.m(J_TGR);
          for (int j = 0; j < NP; ++j) {
            const double tj = X.m(J_TG)[j * LD + j];
            dt += dRb[i * LD + j] * Rb1[i * LD + j] * tj + dRb[j * LD + i] * Rb1[j * LD + i] * tj;
          }
          VA(A_T0)[i] = dt;
          VA(A_T1)[i] = tv * VA(A_CUB)[i];  // bv
        }
        __syncwarp();
        const Real* v3[1] = {VA(A_T1)};
        Real rtb[1];
        matvec<Gm, true, 1>(X.m(J_TGR), v3, rtb, X.lane);  // Rb^T bv
        if (X.lane < NP) VA(A_BDN)[X.lane] += rtb[0];
      }
      X.sync();
      if (tl.valid()) {  // dRb(l+1) = t dRb t (+ bv s_dn^T below)
        const Real* dRb = X.m(J_bTGR);
        Real* o = X.m(J_bR1);
#pragma unroll
        for (int a = 0; a < TR; ++a)
#pragma unroll
          for (int b = 0; b < TC; ++b) {
            const int r = tl.row(a), c = tl.col(b);
            o[r * LD + c] = X.m(J_TG)[r * LD + r] * dRb[r * LD + c] * X.m(J_TG)[c * LD + c];
          }
      }
      X.sync();
      op_rank<Gm>(X.mo(J_bR1), kNoMat, vo(A_T1), vo(A_RD), 1.0, kNoMat, kNoMat, 0.0, kNoMat,
                  kNoMat, 0.0, kNoMat, kNoMat, 0.0, t);
      if (X.warp == 0 && X.lane < NP) VA(A_CUB)[X.lane] = VA(A_T1)[X.lane];
    }
    X.sync();
    // downward-pass contributions of interface l+1: dRb += u Id^T, dUb += u
    if (X.warp == 0 && X.lane < NP) {
      const int i = X.lane;
      VA(A_SD)[i] = dv[(size_t)(l + 1) * 2 * NP + NP + i];      // u(l+1)
      VA(A_BRU)[i] = iv[(size_t)(l + 1) * 2 * NP + i];          // Id(l+1)
      VA(A_CUB)[i] += VA(A_SD)[i];
    }
    X.sync();
    op_rank<Gm>(X.mo(J_bR1), kNoMat, vo(A_SD), vo(A_BRU), 1.0, kNoMat, kNoMat, 0.0, kNoMat,
                kNoMat, 0.0, kNoMat, kNoMat, 0.0, t);
    X.sync();
    op_s2g<Gm>(X.mo(J_bR1), brb, t);
    // layer cotangents from the downward pass: dR += b_rhs b_l^T, dT += b_rhs Id^T
    if (scat) {
      op_rank<Gm>(X.mo(J_bR0), X.mo(J_bR0c), vo(A_Y), vo(A_H), 1.0, kNoMat, kNoMat, 0.0, kNoMat,
                  kNoMat, 0.0, kNoMat, kNoMat, 0.0, t);
      op_rank<Gm>(X.mo(J_bT0), X.mo(J_bT0c), vo(A_Y), vo(A_Z), 1.0, kNoMat, kNoMat, 0.0, kNoMat,
                  kNoMat, 0.0, kNoMat, kNoMat, 0.0, t);
    }
    X.sync();
    // ---- this layer's own construction
    const double Bt = lv.B[l], Bb = lv.B[l + 1];
    if (scat) {
      int nuse;
      double f;
      const double* chi = moments(l, nuse, f);
      const size_t set = (size_t)(chi - C->moments) / (size_t)M;
      nuse_l1 = nuse;
      const double* lPpp = Ppp;
      const double* lPpm = Ppm;
      if (table) {  // shared moments: the layer's matrices from the table
        lPpp = AD.ptab + set * 2 * NP * NP;
        lPpm = lPpp + NP * NP;
        if (solar) {  // and its solar vectors from this wavenumber's start
          if (t < 4 * NP) X.DV(D_PP)[t] = svec[(size_t)l * 4 * NP + t];
          X.sync();
        }
      } else if (layout != 1) {
        build_phase<Gm, true>(X.goff, X.tb, t, X.bar, chi, nuse, f, N, C->quad.pl, solar, mu0,
                              Ppp, Ppm, plm0);
      }
      const long long to = tape_all ? toff[l] : -1;
      doubling_adjoint<Gm>(X.goff, X.tb, t, X.bar, tau, om, Bt, Bb, lv.tc[l], N, solar, F0, mu0,
                           lPpp, lPpm, to >= 0 ? tape_all + to : tape, to < 0, scal, &singular);
      if (t == 0) {  // every load first: the regions are disjoint
        const double s0 = scal[0], s1 = scal[1], s2 = scal[2], s3 = scal[3], s4 = scal[4];
        const double a0 = gtau[l], a1 = gom[l], a2 = bB[l], a3 = bB[l + 1], a4 = btc[l];
        const double tc = lv.tc[l];
        gtau[l] = a0 + s0;
        gom[l] = a1 + s1;
        bB[l] = a2 + s2;
        bB[l + 1] = a3 + s3;
        if (solar) btc[l] = a4 + s4 * F0 * exp(-tc / mu0) * (-1.0 / mu0);
      }
      if (layout != 1) {
        double* dchi = AD.g_mom ? AD.g_mom + (chi - C->moments) : nullptr;
        if (dchi && table && AD.pacc) {
          // the matrix part is linear in the cotangents: summed per block and
          // set here (no return value: fire-and-forget reductions), run once
          // per set after the last chunk; the solar part now
          if (tl.valid()) {
            double* a = AD.pacc + (set * AD.pacc_blocks + blockIdx.x) * 2 * TILE + t * Gm::TE;
#pragma unroll
            for (int i = 0; i < TR; ++i)
#pragma unroll
              for (int j = 0; j < TC; ++j) {
                atomicAdd(a + i * TC + j, X.m(J_T1)[tl.row(i) * LD + tl.col(j)]);
                atomicAdd(a + TILE + i * TC + j, X.m(J_T2)[tl.row(i) * LD + tl.col(j)]);
              }
          }
          if (solar)
            phase_adjoint<Gm, false, true>(X.goff, X.tb, t, X.bar, chi, nuse, N, C->quad.pl,
                                           solar, mu0, dchi, plm0, f);
        } else if (dchi) {
          phase_adjoint<Gm>(X.goff, X.tb, t, X.bar, chi, nuse, N, C->quad.pl, solar, mu0, dchi,
                            plm0, f);
        }
      } else {  // one moment set per wavenumber: accumulate the phase cotangents
        if (tl.valid()) {
          double* aP = pacc + t * Gm::TE;
          double* aM = pacc + TILE + t * Gm::TE;
#pragma unroll
          for (int a = 0; a < TR; ++a)
#pragma unroll
            for (int b = 0; b < TC; ++b) {
              aP[a * TC + b] += X.m(J_T1)[tl.row(a) * LD + tl.col(b)];
              aM[a * TC + b] += X.m(J_T2)[tl.row(a) * LD + tl.col(b)];
            }
        }
        if (X.warp == 0 && X.lane < NP) {
          pacc[2 * TILE + X.lane] += VA(A_T0)[X.lane];
          pacc[2 * TILE + NP + X.lane] += VA(A_T1)[X.lane];
        }
      }
    } else if (tau > 0.0) {
      // pure absorption (src/doubling.hpp:56-77): t = exp(-tau/mu), linear-in-tau source
      double pbar = 0.0, pd = 0.0, pt = 0.0;
      const double Bbar = 0.5 * (Bb + Bt), Bd = (Bb - Bt) / tau;
      if (X.warp == 0 && X.lane < N) {
        const int i = X.lane;
        const double mui = X.DV(D_MU)[i];
        const double tex = -tau / mui;
        const double tv = (tex > -200.0) ? exp(tex) : 0.0;
        const double omt = 1.0 - tv, slope = mui * omt - 0.5 * tau * (1.0 + tv);
        const double bu = VA(A_BUP)[i], bd = VA(A_BDN)[i];
        double btv = VA(A_T0)[i];
        pbar = (bu + bd) * omt;
        pd = (bu - bd) * slope;
        double bomt = (bu + bd) * Bbar;
        const double bslope = (bu - bd) * Bd;
        bomt += bslope * mui;
        btv += bslope * (-0.5 * tau);
        pt = bslope * (-0.5 * (1.0 + tv));
        btv += -bomt;
        pt += btv * tv * (-1.0 / mui);
      }
      double* red = reinterpret_cast<double*>(X.gjbuf) + 4;
      pbar = gsum<G>(pbar, red, bar);
      pd = gsum<G>(pd, red, bar);
      pt = gsum<G>(pt, red, bar);
      if (t == 0) {
        bB[l + 1] += 0.5 * pbar + pd / tau;
        bB[l] += 0.5 * pbar - pd / tau;
        gtau[l] += pt - pd * Bd / tau;
      }
    }
    X.sync();
  }
  // one moment set per wavenumber: its adjoint once
  if (layout == 1 && AD.g_mom) {
    op_g2s<Gm>(pacc, X.mo(J_T1), kNoMat, t);
    op_g2s<Gm>(pacc + TILE, X.mo(J_T2), kNoMat, t);
    if (X.warp == 0 && X.lane < NP) {
      VA(A_T0)[X.lane] = pacc[2 * TILE + X.lane];
      VA(A_T1)[X.lane] = pacc[2 * TILE + NP + X.lane];
    }
    X.sync();
    const double* chi = C->moments + (size_t)w * M;
    phase_adjoint<Gm>(X.goff, X.tb, t, X.bar, chi, nuse_l1, N, C->quad.pl, solar, mu0,
                      AD.g_mom + (size_t)w * M, plm0, f_l1);
  }
  // ======== 3. lower boundary, beam and Planck chain rules
  double pub = 0.0, pubmu = 0.0;
  if (X.warp == 0 && X.lane < N) {
    pub = VA(A_CUB)[X.lane];
    pubmu = VA(A_CUB)[X.lane] * X.DV(D_MU)[X.lane];
  }
  double* red = reinterpret_cast<double*>(X.gjbuf) + 4;
  pub = gsum<G>(pub, red, bar);
  pubmu = gsum<G>(pubmu, red, bar);
  if (t == 0) {
    double bBs = 0.0;
    if (has_surface) {
      bBs = (1.0 - Aalb) * pub;
      if (solar && Aalb > 0.0)
        btc[nL] += pub * (Aalb / kPi) * F0 * mu0 * exp(-lv.tc[nL] / mu0) * (-1.0 / mu0);
    } else if (C->diffusion) {
      const double dt = lv.tau[nL - 1];
      bB[nL] += pub;
      if (dt > 0.0) {
        const double dB = (lv.B[nL] - lv.B[nL - 1]) / dt;
        bB[nL] += pubmu / dt;
        bB[nL - 1] -= pubmu / dt;
        gtau[nL - 1] += -pubmu * dB / dt;
      }
    } else {
      bBs = pub;
    }
    if (C->thermal) {
      if (C->surface_temperature < 0.0)
        bB[nL] += bBs;  // the surface emits B(T_L)
      else if (AD.g_semis)
        AD.g_semis[w] = bBs;  // d L / d B(surface_temperature)
      if (C->top_temperature < 0.0) bB[0] += pBtop;
    } else if (AD.g_semis) {
      AD.g_semis[w] = bBs;
    }
    // cumulative tau: tc(l) = sum_{j<l} tau_j
    double s = 0.0;
    for (int l = nL; l >= 1; --l) {
      s += btc[l];
      gtau[l - 1] += s;
    }
  }
  X.sync();
  for (int l = t; l < nL; l += G) {
    const int ul = fb ? nL - 1 - l : l;
    const double om = lv.om[l];
    double gt = gtau[l], go = (om > 0.0 && om <= 1.0) ? gom[l] : 0.0;
    // delta-M scaling (src/solver.cpp:441-501): tau' = (1 - omega f) tau,
    // omega' = omega (1 - f) / (1 - omega f), f = chi_2N of the layer's set;
    // the cotangents above are those of tau' and omega'
    const double om_u = lv.omu[l];
    const double tau_u = C->dtau[(size_t)w * nL + ul];
    if (C->delta_m && M > 2 * N && om_u > 0.0 && tau_u > 0.0) {
      int nuse;
      double f;
      const double* chi = moments(l, nuse, f);
      if (f >= 0.0) {
        const double d = 1.0 - om_u * f;
        const double gtu = gt * d;
        const double gou = -gt * f * tau_u + go * (1.0 - f) / (d * d);
        const double gf = -gt * om_u * tau_u + go * om_u * (om_u - 1.0) / (d * d);
        if (AD.g_mom) atomicAdd(&AD.g_mom[(size_t)(chi - C->moments) + 2 * N], gf);
        gt = gtu;
        go = gou;
      }
    }
    if (AD.g_tau) AD.g_tau[(size_t)w * nL + ul] = gt;
    if (AD.g_ssa) AD.g_ssa[(size_t)w * nL + ul] = (om_u > 0.0 && om_u <= 1.0) ? go : 0.0;
  }
  for (int l = t; l <= nL; l += G) {
    const int ul = fb ? nL - l : l;
    if (C->thermal && AD.g_temp) {
      const double Tv = C->temperature[(C->temp_per_wav ? wo : 0) + ul];
      atomicAdd(&AD.g_temp[(C->temp_per_wav ? wo : 0) + ul], bB[l] * planck_band_deriv(wlo, whi, Tv));
    } else if (!C->thermal && C->planck && AD.g_planck) {
      AD.g_planck[wo + ul] = bB[l];
    }
  }
  if (singular && t == 0) atomicOr(status, status_bits(singular));
  X.sync();
}

// ---------------------------------------------------------------- kernel
template <int NP>
struct AdjKern {
  using GD = AdjGeo<NP>;
  static constexpr size_t kMaxSmem = 227 * 1024;
  static constexpr int G = GD::G;
  static constexpr int kGroups =
      (AdjGroup<NP>::bytes * 4 <= kMaxSmem) ? 4
      : (AdjGroup<NP>::bytes * 3 <= kMaxSmem) ? 3
      : (AdjGroup<NP>::bytes * 2 <= kMaxSmem) ? 2 : 1;
  static constexpr int kThreads = kGroups * G;
};

// Taping forward of one chunk, in the forward kernel's geometry and shared
// memory (one-warp groups at NP <= 16): prologue, a claim on the record pool
// for all of the wavenumber's doubling chains (none when the pool is full:
// the reverse then recomputes them), and the forward solve recording the
// chains, the records and the interface intensities into the wavenumber's
// WavState.
template <int NP>
__global__ void __launch_bounds__(128, 3) tape_kernel(SolveParams P, ColumnDev col0, AdjDev AD) {
  using GD = Geo<NP, double>;
  using GL = GroupLayout<NP, KIND_FP64>;
  using WS = WavState<GD>;
  constexpr int G = GD::G;
  const int gib = threadIdx.x / G;
  const int t = threadIdx.x % G;
  const int bar = 1 + gib;
  const unsigned goff = (unsigned)(gib * GL::bytes);
  const unsigned tb = goff + (unsigned)CommonLayout<NP>::bytes;
  for (unsigned i = (unsigned)t * 4u; i < (unsigned)GL::bytes; i += (unsigned)G * 4u)
    *sp<unsigned>(goff + i) = 0u;
  gsync<G>(bar);
  if (t == 0) *sp<ColumnDev>(goff + CommonLayout<NP>::col) = col0;
  long long* task_s = sp<long long>(goff + CommonLayout<NP>::misc + 32);
  double* red = sp<double>(goff + CommonLayout<NP>::misc + 64);
  const int lmax = P.max_layers, nL = col0.L;
  for (;;) {
    long long task;
    if constexpr (G == 32) {
      unsigned long long v = 0;
      if (t == 0) v = atomicAdd(P.counter, 1ull);
      task = (long long)__shfl_sync(0xffffffffu, v, 0);
    } else {
      gsync<G>(bar);
      if (t == 0) *task_s = (long long)atomicAdd(P.counter, 1ull);
      gsync<G>(bar);
      task = *task_s;
    }
    if (task >= P.ntasks) break;
    const int w = (int)(AD.w0 + task);
    char* st = AD.state + (size_t)task * AD.state_bytes;
    long long* toff = reinterpret_cast<long long*>(st + WS::toff_at(lmax));
    gsync<G>(bar);
    wav_prologue<NP>(goff, t, bar, w, st, lmax, P.status, 0);
    const Levels lv(st, lmax);
    double need = 0.0;  // doubles of this wavenumber's records (exact in FP64)
    for (int l = t; l < nL; l += G) {
      const double tau = lv.tau[l], om = lv.om[l];
      if (tau > 0.0 && om > 0.0)
        need += (double)TapeLayout<GD>::layer(num_doublings(tau, om > 1.0 ? 1.0 : om));
    }
    need = gsum<G>(need, red, bar);
    if (t == 0) {
      const unsigned long long n = (unsigned long long)need;
      const unsigned long long base = atomicAdd(AD.pool_used, n);
      toff[nL] = (base + n <= (unsigned long long)AD.pool_cap) ? (long long)base : -1ll;
    }
    if (P.pivot_all && t == 0)
      sp<double>(goff + (unsigned)CommonLayout<NP>::misc + 48)[S_PIVALL] = 1.0;
    gsync<G>(bar);
    const long long base = toff[nL];
    wav_body_checked<GD, MODE_FP64>(goff, tb, 0u, t, bar, w, st, lmax, P.status,
                                    reinterpret_cast<double*>(st + WS::fwd(lmax)),
                                    base >= 0 ? AD.pool + base : nullptr,
                                    base >= 0 ? (long long)need : 0, toff);
  }
}

// Reverse of one chunk (after its tape_kernel): per wavenumber, the prologue
// again for the group's shared constants, then wav_adjoint on the state the
// forward left.
template <int NP>
__global__ void __launch_bounds__(AdjKern<NP>::kThreads) adjoint_kernel(SolveParams P, ColumnDev col0, AdjDev AD) {
  using GD = AdjGeo<NP>;
  constexpr int G = GD::G;
  const int gib = threadIdx.x / G;
  const int t = threadIdx.x % G;
  const int bar = 1 + gib;
  const unsigned goff = (unsigned)(gib * AdjGroup<NP>::bytes);
  const unsigned tb = goff + (unsigned)CommonLayout<NP>::bytes;
  const int slot = blockIdx.x * (blockDim.x / G) + gib;
  char* scr = P.scratch + (size_t)slot * P.slot_bytes;
  for (unsigned i = (unsigned)t * 4u; i < (unsigned)AdjGroup<NP>::bytes; i += (unsigned)G * 4u)
    *sp<unsigned>(goff + i) = 0u;
  gsync<G>(bar);
  if (t == 0) *sp<ColumnDev>(goff + CommonLayout<NP>::col) = col0;
  long long* task_s = sp<long long>(goff + CommonLayout<NP>::misc + 32);
  for (;;) {
    long long task;
    if constexpr (G == 32) {
      unsigned long long v = 0;
      if (t == 0) v = atomicAdd(P.counter, 1ull);
      task = (long long)__shfl_sync(0xffffffffu, v, 0);
    } else {
      gsync<G>(bar);
      if (t == 0) *task_s = (long long)atomicAdd(P.counter, 1ull);
      gsync<G>(bar);
      task = *task_s;
    }
    if (task >= P.ntasks) break;
    const int w = (int)(AD.w0 + task);
    char* st = AD.state + (size_t)task * AD.state_bytes;
    gsync<G>(bar);
    wav_prologue<NP, adjoint_group<NP>()>(goff, t, bar, w, st, P.max_layers, P.status, 0);
    wav_adjoint<NP>(goff, tb, t, bar, w, st, scr, P.max_layers, P.status, AD);
  }
}

// One reverse-geometry group per block, for the per-moment-set kernels below:
// cleared shared memory, the column and the quadrature constants.
template <int NP>
__device__ __forceinline__ Ctx<AdjGeo<NP>> set_group(const ColumnDev& col0, int t) {
  using Gm = AdjGeo<NP>;
  constexpr int G = Gm::G;
  for (unsigned i = (unsigned)t * 4u; i < (unsigned)AdjGroup<NP>::bytes; i += (unsigned)G * 4u)
    *sp<unsigned>(i) = 0u;
  gsync<G>(1);
  if (t == 0) *sp<ColumnDev>(CommonLayout<NP>::col) = col0;
  const Ctx<Gm> X(0u, (unsigned)CommonLayout<NP>::bytes, t, 1);
  if (t < NP) {
    const bool q = t < col0.N;
    const double mu = q ? col0.quad.mu[t] : 1.0, wt = q ? col0.quad.wt[t] : 0.0;
    X.DV(D_MU)[t] = mu;
    X.DV(D_WT)[t] = wt;
    X.DV(D_CW)[t] = 2.0 * kPi * wt * mu;
    X.DV(D_HW)[t] = 0.5 * wt;
  }
  gsync<G>(1);
  return X;
}

// Phase matrices of the moment sets that every wavenumber shares (one per
// layer), once per adjoint call instead of once per wavenumber and layer:
// block u forms set u's normalised P++ / P+- into tab[u] (row-major, pitch NP).
template <int NP>
__global__ void __launch_bounds__(AdjGeo<NP>::G) phase_table_kernel(ColumnDev col0, double* tab) {
  using Gm = AdjGeo<NP>;
  const int t = threadIdx.x;
  const Ctx<Gm> X = set_group<NP>(col0, t);
  const size_t u = blockIdx.x;
  const double* chi = col0.moments + u * col0.M;
  int nuse;
  double f;
  moment_use(&col0, chi, nuse, f);
  double* P = tab + u * 2 * NP * NP;
  build_phase<Gm>(X.goff, X.tb, t, X.bar, chi, nuse, f, col0.N, col0.quad.pl, false, 1.0, P,
                  P + NP * NP);
}

// The moment gradients of the shared sets from the phase-matrix cotangents
// that the reverse pass summed per block: block u adds the blocks' sums of
// set u and runs the matrix part of phase_adjoint once.
template <int NP>
__global__ void __launch_bounds__(AdjGeo<NP>::G) phase_finish_kernel(ColumnDev col0, AdjDev AD) {
  using Gm = AdjGeo<NP>;
  constexpr int TR = Gm::TR, TC = Gm::TC, TE = Gm::TE, TILE = Gm::G * Gm::TE;
  const int t = threadIdx.x;
  const Ctx<Gm> X = set_group<NP>(col0, t);
  const size_t u = blockIdx.x;
  const Tile<Gm> tl(t);
  if (tl.valid()) {
    double sP[TR][TC], sM[TR][TC];
#pragma unroll
    for (int i = 0; i < TR; ++i)
#pragma unroll
      for (int j = 0; j < TC; ++j) sP[i][j] = sM[i][j] = 0.0;
    const double* a = AD.pacc + u * AD.pacc_blocks * 2 * TILE + t * TE;
#pragma unroll 4
    for (int b = 0; b < AD.pacc_blocks; ++b, a += 2 * TILE)
#pragma unroll
      for (int i = 0; i < TR; ++i)
#pragma unroll
        for (int j = 0; j < TC; ++j) {
          sP[i][j] += a[i * TC + j];
          sM[i][j] += a[TILE + i * TC + j];
        }
    tl.store_rm(sP, X.m(J_T1));
    tl.store_rm(sM, X.m(J_T2));
  }
  X.sync();
  const double* chi = col0.moments + u * col0.M;
  int nuse;
  double f;
  moment_use(&col0, chi, nuse, f);
  phase_adjoint<Gm, true, false>(X.goff, X.tb, t, X.bar, chi, nuse, col0.N, col0.quad.pl, false,
                                 1.0, AD.g_mom + u * col0.M, nullptr, f);
}

}  // namespace adrt_dev
