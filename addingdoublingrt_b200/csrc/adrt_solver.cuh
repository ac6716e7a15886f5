// adrt_solver.cuh -- the fused per-wavenumber adding-doubling solver.
//
// One thread group (a warp for N <= 16, four warps for N = 32) solves one
// wavenumber column end to end:
//
//   prologue   Planck levels, delta-M scaled tau/omega, scaled cumulative tau
//              (src/solver.cpp:385-514, src/planck.cpp:35-131)
//   upward     for each layer from the bottom: phase matrices
//              (src/phase_matrix.hpp:61-181), thin-layer init and doubling
//              (src/doubling.hpp:29-230), then adding onto the composite of
//              everything below it (src/adding.hpp:263-490).  The composite
//              keeps only R_ab and the upward source with the lower boundary
//              intensity folded in (T_ba I_bot + s_up), which is all the
//              interface formulas of src/solver.cpp:24-73 read from rbase.
//   downward   from the top: the downward intensity below layer l solves
//              (I - R_l R_base) I_dn = T_l I_dn(above) + R_l U_base + s_dn_l, and
//              I_up = R_base I_dn + U_base -- the same linear system the
//              reference solves with its rtop composites (computeIdown /
//              computeIup), without building rtop.
//   fluxes     F = 2 pi sum w mu I, J (+ beam), divF (src/solver.cpp:605-700).
//
// Matrices are NP x NP (NP = N rounded up to 4, 8, 16 or 32; padded with the
// identity/zero blocks, which the algebra keeps exact).  Each thread of the
// group owns a TR x TC register tile of every matrix.  FP64 products C = A B
// run on the FP64 tensor cores (mma.sync m8n8k4) from operands staged in
// shared memory; FP32 products are register-tile FFMA loops.  The
// (I - R R')^{-1} right-solves are, in FP64, a blocked Gauss-Jordan without
// pivoting on the tensor cores (gj_mma; the matrices are diagonally dominant),
// and in FP32 a register-tile Gauss-Jordan with the reference's pivot rule
// (column pivoting on the largest |entry| of the pivot row, the LU of the
// transpose of src/matrix.hpp:120-124).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "adrt_types.cuh"

namespace adrt_dev {

#ifndef ADRT_GEMM_MMA
#define ADRT_GEMM_MMA 1
#endif

// The block's dynamic shared memory.  Non-inlined operations take 32-bit
// byte offsets into it (not pointers) and rebuild their pointers from this
// symbol, so every shared access compiles to a 32-bit LDS/STS.
extern __shared__ __align__(16) char adrt_smem[];

template <typename T>
__device__ __forceinline__ T* sp(unsigned off) {
  return reinterpret_cast<T*>(adrt_smem + off);
}
__device__ __forceinline__ unsigned soff(const void* p) {
  return static_cast<unsigned>(static_cast<const char*>(p) - adrt_smem);
}

// ============================================================== geometry
// Threads that solve one wavenumber: a warp up to NP = 16, four warps at 32.
template <int NP>
constexpr int default_group() { return (NP <= 16) ? 32 : 128; }

template <int NP_, typename Real_, int G_ = default_group<NP_>()>
struct Geo {
  static constexpr int NP = NP_;
  using Real = Real_;
  static constexpr int G = G_;  // threads per wavenumber (32, 64 or 128)
  static_assert(G == 32 || G == 64 || G == 128, "group of one, two or four warps");
  static constexpr int RB = (G == 32) ? 4 : 8;      // thread-grid rows
  static constexpr int CB = G / RB;                 // thread-grid cols
  static constexpr int TR = (NP + RB - 1) / RB;     // tile rows per thread
  static constexpr int TC = (NP + CB - 1) / CB;     // tile cols per thread
  static constexpr int TE = TR * TC;
  static constexpr int DIM = (RB * TR > CB * TC) ? RB * TR : CB * TC;
  // Row padding keeps rows 16-byte aligned and spreads rows over the shared-
  // memory banks: an FP64 pitch of DIM + 4 puts the four k-rows of an m8n8k4
  // operand load 8 banks apart (row- or column-major), so those loads are
  // conflict-free.  NP = 32 keeps DIM + 2 so the adjoint's 25 matrices fit.
  static constexpr int PAD = (sizeof(Real) == 8) ? ((NP_ <= 16) ? 4 : 2) : 4;
  static constexpr int LD = DIM + PAD;
  static constexpr int MAT = DIM * LD;                // Reals per smem matrix
  static constexpr int NW = G / 32;                   // warps per group
  // matvec lanes: warp 0 only; LPR lanes per row
  static constexpr int LPR = (32 / NP < NP) ? (32 / NP) : NP;
  static constexpr int KCH = NP / LPR;
  static_assert(NP % TR == 0 && NP % TC == 0, "tiles must divide the padded order");
};

constexpr size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// Shared memory of one thread group = a precision-independent prefix
// (CommonLayout: the column descriptor, scalars and FP64 vectors) followed by
// one or two typed regions (TypedLayout: Real vectors, the Gauss-Jordan
// buffers, then NMAT matrices).  Because the prefix is shared, an FP32 and an
// FP64 view of the same group see the same column, quadrature and scalars,
// which lets an FP64-adding wavenumber run FP32 doublings in a second typed
// region placed over its own matrices.
template <int NP>
struct CommonLayout {
  static constexpr size_t col = 0;
  static constexpr size_t misc = align16(sizeof(ColumnDev));
  // misc: [0,32) reduction words, [32,40) task index, [48,112) eight FP64
  //       per-wavenumber scalars (MiscSlot)
  static constexpr size_t dvecs = misc + 128;
  static constexpr int NDVEC = 8;  // double vectors of NP (DVecSlot)
  static constexpr size_t bytes = align16(dvecs + sizeof(double) * NDVEC * NP);
};

template <class Gm, int NMAT>
struct TypedLayout {
  using Real = typename Gm::Real;
  static constexpr int NVEC = 20;  // Real vectors of NP (VecSlot)
  static constexpr size_t vecs = 0;
  static constexpr size_t gj = align16(vecs + sizeof(Real) * NVEC * Gm::NP);
  static constexpr size_t mats = align16(gj + sizeof(Real) * (6 * Gm::DIM + 4));
  static constexpr size_t bytes = align16(mats + (size_t)NMAT * sizeof(Real) * Gm::MAT);
};

// Matrix buffers of the reference-order (T-form) doubling and the adding,
// and of the FP32 Lambda-split doubling.
constexpr int kMatsTForm = 5;
constexpr int kMatsLam = 9;

// Vector slots (Real) inside TypedLayout::vecs.
enum VecSlot {
  V_Y0 = 0, V_Y1, V_Z0, V_Z1, V_SU0, V_SU1, V_SD0, V_SD1,
  V_RU, V_RD, V_UB, V_SDN, V_SUP, V_ID, V_IU, V_RHS, V_TMP, V_T, V_X
};
// Double vector slots inside CommonLayout::dvecs: quadrature, solar phase and
// the direct-transmission diagonal of the Lambda-split doubling (ping-pong).
enum DVecSlot { D_MU = 0, D_WT, D_CW, D_HW, D_PP, D_PM, D_LAM0, D_LAM1 };
// FP64 per-wavenumber scalars inside CommonLayout::misc (+48).
// S_PIVALL: nonzero while a wavenumber is solved again with partial pivoting
// in every solve (after a weak pivot of the tensor-core solve).
enum MiscSlot { S_BS = 0, S_BTOP, S_PIVALL };

// ============================================================== sync / reductions
template <int G>
__device__ __forceinline__ void gsync(int bar) {
  if constexpr (G == 32) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(bar), "n"(G) : "memory");
  }
}

// Max of a 32-bit key over the group.  red: 2*NW unsigned in smem (double
// buffered by `parity`).
template <int G>
__device__ __forceinline__ unsigned gmax_u32(unsigned key, unsigned* red, int parity, int bar) {
  unsigned m = __reduce_max_sync(0xffffffffu, key);
  if constexpr (G == 32) {
    return m;
  } else {
    constexpr int NW = G / 32;
    const int t = threadIdx.x % G;
    if ((t & 31) == 0) red[parity * NW + (t >> 5)] = m;
    gsync<G>(bar);
    unsigned r = red[parity * NW];
#pragma unroll
    for (int i = 1; i < NW; ++i) r = max(r, red[parity * NW + i]);
    return r;
  }
}

__device__ __forceinline__ double recip(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float recip(float x) { return __frcp_rn(x); }

// ============================================================== vector smem access
template <typename Real, int CNT>
__device__ __forceinline__ void lds_vec(Real* dst, const Real* src) {
  if constexpr (sizeof(Real) * CNT % 16 == 0) {
#pragma unroll
    for (int i = 0; i < CNT; i += 16 / (int)sizeof(Real)) {
      if constexpr (sizeof(Real) == 8) {
        const double2 v = *reinterpret_cast<const double2*>(src + i);
        dst[i] = v.x;
        dst[i + 1] = v.y;
      } else {
        const float4 v = *reinterpret_cast<const float4*>(src + i);
        dst[i] = v.x;
        dst[i + 1] = v.y;
        dst[i + 2] = v.z;
        dst[i + 3] = v.w;
      }
    }
  } else if constexpr (sizeof(Real) == 4 && CNT == 2) {
    const float2 v = *reinterpret_cast<const float2*>(src);
    dst[0] = v.x;
    dst[1] = v.y;
  } else {
#pragma unroll
    for (int i = 0; i < CNT; ++i) dst[i] = src[i];
  }
}

template <typename Real, int CNT>
__device__ __forceinline__ void sts_vec(Real* dst, const Real* src) {
  if constexpr (sizeof(Real) * CNT % 16 == 0) {
#pragma unroll
    for (int i = 0; i < CNT; i += 16 / (int)sizeof(Real)) {
      if constexpr (sizeof(Real) == 8) {
        *reinterpret_cast<double2*>(dst + i) = make_double2(src[i], src[i + 1]);
      } else {
        *reinterpret_cast<float4*>(dst + i) = make_float4(src[i], src[i + 1], src[i + 2], src[i + 3]);
      }
    }
  } else if constexpr (sizeof(Real) == 4 && CNT == 2) {
    *reinterpret_cast<float2*>(dst) = make_float2(src[0], src[1]);
  } else {
#pragma unroll
    for (int i = 0; i < CNT; ++i) dst[i] = src[i];
  }
}

// ============================================================== tile algebra
// Every matrix lives in shared memory (row-major "rm": s[r*LD + c], or
// column-major "cm": s[c*LD + r]).  Thread t of the group owns the TR x TC
// tile at rows rb*TR.., cols cb*TC.. of every operation's output; the
// operations are non-inlined so each exists once in the binary.
template <class Gm>
struct Tile {
  using Real = typename Gm::Real;
  static constexpr int TR = Gm::TR, TC = Gm::TC, LD = Gm::LD, NP = Gm::NP;
  int rb, cb;
  __device__ __forceinline__ explicit Tile(int t) : rb(t / Gm::CB), cb(t % Gm::CB) {}
  __device__ __forceinline__ bool valid() const { return rb * TR < NP && cb * TC < NP; }
  __device__ __forceinline__ int row(int a) const { return rb * TR + a; }
  __device__ __forceinline__ int col(int b) const { return cb * TC + b; }
  __device__ __forceinline__ void load_rm(Real (&X)[TR][TC], const Real* s) const {
#pragma unroll
    for (int a = 0; a < TR; ++a) lds_vec<Real, TC>(X[a], s + row(a) * LD + cb * TC);
  }
  __device__ __forceinline__ void store_rm(const Real (&X)[TR][TC], Real* s) const {
#pragma unroll
    for (int a = 0; a < TR; ++a) sts_vec<Real, TC>(s + row(a) * LD + cb * TC, X[a]);
  }
  __device__ __forceinline__ void store_cm(const Real (&X)[TR][TC], Real* s) const {
#pragma unroll
    for (int b = 0; b < TC; ++b) {
      Real colv[TR];
#pragma unroll
      for (int a = 0; a < TR; ++a) colv[a] = X[a][b];
      sts_vec<Real, TR>(s + col(b) * LD + rb * TR, colv);
    }
  }
};

// Offset of element (r, c) of an NP x NP matrix stored in the tile order of
// geometry GO (thread t of GO owns TE contiguous Reals).
template <class GO>
__host__ __device__ __forceinline__ int tile_index(int r, int c) {
  return ((r / GO::TR) * GO::CB + c / GO::TC) * GO::TE + (r % GO::TR) * GO::TC + c % GO::TC;
}

// FP64 products on the tensor cores: mma.sync m8n8k4 f64 (the FP64 tensor
// path of sm_100a; tcgen05 has no f64 kind).  Each warp owns WR x WC output
// tiles of 8x8; lane (g = lane/4, q = lane%4) holds rows g, columns 2q, 2q+1
// of each tile (the m8n8k4 accumulator fragment).
template <class Gm>
struct UseMMA {
  static constexpr bool value =
      ADRT_GEMM_MMA && sizeof(typename Gm::Real) == 8 && Gm::NP >= 8 &&
      (Gm::NP / 8) * (Gm::NP / 8) >= Gm::G / 32;  // at least one 8x8 tile per warp
};

__device__ __forceinline__ void mma_f64_m8n8k4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <class Gm, bool XRM = false>
__device__ __forceinline__ void gemm_mma(const double* __restrict__ XT, const double* __restrict__ Y,
                                         const double* add, int id_minus, double* out_rm,
                                         double* out_cm, int t) {
  constexpr int NP = Gm::NP, LD = Gm::LD;
  constexpr int NT = NP / 8;
  constexpr int TPW = NT * NT / (Gm::G / 32);  // 8x8 output tiles per warp
  constexpr int WR = (TPW >= 4) ? 2 : 1, WC = (TPW >= 2) ? 2 : 1;
  constexpr int WPC = NT / WC;  // warps per tile-row band
  static_assert(TPW >= 1 && (NT / WR) * WPC == Gm::G / 32, "warp grid must cover the tiles");
  const int warp = t >> 5, lane = t & 31, g = lane >> 2, q = lane & 3;
  const int r0 = (warp / WPC) * WR * 8, c0 = (warp % WPC) * WC * 8;
  // a warp with one output tile keeps two partial sums (even / odd k-steps)
  constexpr int NA = (WR * WC == 1 && NP >= 16) ? 2 : 1;
  double acc[NA][WR][WC][2];
#pragma unroll
  for (int h = 0; h < NA; ++h)
#pragma unroll
    for (int i = 0; i < WR; ++i)
#pragma unroll
      for (int j = 0; j < WC; ++j) acc[h][i][j][0] = acc[h][i][j][1] = 0.0;
  constexpr int sk = XRM ? 1 : LD, sr = XRM ? LD : 1;  // X element (r, k) at XT[k sk + r sr]
#pragma unroll
  for (int ks = 0; ks < NP / 4; ++ks) {
    const int k = ks * 4 + q;
    double a[WR], b[WC];
#pragma unroll
    for (int i = 0; i < WR; ++i) a[i] = XT[k * sk + (r0 + i * 8 + g) * sr];
#pragma unroll
    for (int j = 0; j < WC; ++j) b[j] = Y[k * LD + c0 + j * 8 + g];
#pragma unroll
    for (int i = 0; i < WR; ++i)
#pragma unroll
      for (int j = 0; j < WC; ++j)
        mma_f64_m8n8k4(acc[ks % NA][i][j][0], acc[ks % NA][i][j][1], a[i], b[j]);
  }
#pragma unroll
  for (int i = 0; i < WR; ++i)
#pragma unroll
    for (int j = 0; j < WC; ++j) {
      const int r = r0 + i * 8 + g, c = c0 + j * 8 + 2 * q;
      double v0 = acc[0][i][j][0], v1 = acc[0][i][j][1];
      if constexpr (NA == 2) {
        v0 += acc[1][i][j][0];
        v1 += acc[1][i][j][1];
      }
      if (id_minus == 1) {
        v0 = ((r == c) ? 1.0 : 0.0) - v0;
        v1 = ((r == c + 1) ? 1.0 : 0.0) - v1;
      } else if (id_minus == 2) {
        v0 = -v0;
        v1 = -v1;
      }
      if (add) {
        const double2 ad = *reinterpret_cast<const double2*>(add + r * LD + c);
        v0 = ad.x + v0;
        v1 = ad.y + v1;
      }
      if (out_rm) *reinterpret_cast<double2*>(out_rm + r * LD + c) = make_double2(v0, v1);
      if (out_cm) {
        out_cm[c * LD + r] = v0;
        out_cm[(c + 1) * LD + r] = v1;
      }
    }
}

// out = [I -] X Y [+ add] (id_minus = 1), or -X Y [+ add] (id_minus = 2):
// X column-major (XT[k*LD + r] = X[r][k]), Y and add row-major.  Writes out_rm and/or out_cm (either may be null).  `add` may
// alias out_rm (each thread reads its own tile before writing it).
// Marks an absent optional operand (add / out_rm / out_cm / B / bvec).
constexpr unsigned kNoMat = 0xffffffffu;
// As op_gj's right-hand side: the identity (X = A^{-1}).
constexpr unsigned kIdentity = 0xfffffffeu;


// XRM: X given row-major (a separate instantiation; the common product keeps
// one body).
template <class Gm, bool XRM = false>
__device__ __noinline__ void op_gemm(unsigned xt_off, unsigned y_off, unsigned add_off,
                                     int id_minus, unsigned orm_off, unsigned ocm_off, int t) {
  using Real = typename Gm::Real;
  constexpr int TR = Gm::TR, TC = Gm::TC, LD = Gm::LD, NP = Gm::NP;
  const Real* __restrict__ XT = sp<Real>(xt_off);
  const Real* __restrict__ Y = sp<Real>(y_off);
  const Real* add = (add_off == kNoMat) ? nullptr : sp<Real>(add_off);
  Real* out_rm = (orm_off == kNoMat) ? nullptr : sp<Real>(orm_off);
  Real* out_cm = (ocm_off == kNoMat) ? nullptr : sp<Real>(ocm_off);
  if constexpr (UseMMA<Gm>::value) {
    gemm_mma<Gm, XRM>(XT, Y, add, id_minus, out_rm, out_cm, t);
    return;
  }
  const Tile<Gm> tl(t);
  if (!tl.valid()) return;
  Real acc[TR][TC];
#pragma unroll
  for (int a = 0; a < TR; ++a)
#pragma unroll
    for (int b = 0; b < TC; ++b) acc[a][b] = Real(0);
  const Real* xp = XT + tl.rb * TR;
  const Real* yp = Y + tl.cb * TC;
#pragma unroll 8
  for (int k = 0; k < NP; ++k) {
    Real xa[TR], yb[TC];
    if constexpr (XRM) {
#pragma unroll
      for (int a = 0; a < TR; ++a) xa[a] = XT[tl.row(a) * LD + k];
    } else {
      lds_vec<Real, TR>(xa, xp + k * LD);
    }
    lds_vec<Real, TC>(yb, yp + k * LD);
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) acc[a][b] = fma(xa[a], yb[b], acc[a][b]);
  }
  if (id_minus) {
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b)
        acc[a][b] = (id_minus == 2) ? -acc[a][b]
                                    : ((tl.row(a) == tl.col(b)) ? Real(1) : Real(0)) - acc[a][b];
  }
  if (add) {
    Real ad[TR][TC];
    tl.load_rm(ad, add);
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) acc[a][b] = ad[a][b] + acc[a][b];
  }
  if (out_rm) tl.store_rm(acc, out_rm);
  if (out_cm) tl.store_cm(acc, out_cm);
}

// Products of the Lambda-split doubling (FP32, register tiles).  lam is the
// FP64 diagonal Lambda (smem byte offset of NP doubles); Z a row-major matrix.
//   kLamR2:  acc = X Y;  out_rm = I - acc;  out2_rm = Lambda acc + Z
//   kLamAdd: v = X Y + Lambda Z;  out_rm / out_cm = v;
//            out2_rm (optional) = v + Lambda^2 on the diagonal
// Every term is a sum of non-negative products for a non-negative phase
// function, so each entry keeps FP32 relative accuracy.
constexpr int kLamR2 = 0, kLamAdd = 1;

template <class Gm>
__device__ __noinline__ void op_gemm_lam(unsigned xt_off, unsigned y_off, unsigned z_off,
                                         unsigned lam_off, int mode, unsigned orm_off,
                                         unsigned ocm_off, unsigned o2_off, int t) {
  using Real = typename Gm::Real;
  constexpr int TR = Gm::TR, TC = Gm::TC, LD = Gm::LD, NP = Gm::NP;
  const Real* __restrict__ XT = sp<Real>(xt_off);
  const Real* __restrict__ Y = sp<Real>(y_off);
  const Real* Z = sp<Real>(z_off);
  const double* lam = sp<double>(lam_off);
  Real* out_rm = (orm_off == kNoMat) ? nullptr : sp<Real>(orm_off);
  Real* out_cm = (ocm_off == kNoMat) ? nullptr : sp<Real>(ocm_off);
  Real* out2 = (o2_off == kNoMat) ? nullptr : sp<Real>(o2_off);
  const Tile<Gm> tl(t);
  if (!tl.valid()) return;
  Real acc[TR][TC];
#pragma unroll
  for (int a = 0; a < TR; ++a)
#pragma unroll
    for (int b = 0; b < TC; ++b) acc[a][b] = Real(0);
  const Real* xp = XT + tl.rb * TR;
  const Real* yp = Y + tl.cb * TC;
#pragma unroll 8
  for (int k = 0; k < NP; ++k) {
    Real xa[TR], yb[TC];
    lds_vec<Real, TR>(xa, xp + k * LD);
    lds_vec<Real, TC>(yb, yp + k * LD);
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) acc[a][b] = fma(xa[a], yb[b], acc[a][b]);
  }
  Real zt[TR][TC];
  tl.load_rm(zt, Z);
  Real lr[TR];
#pragma unroll
  for (int a = 0; a < TR; ++a) lr[a] = static_cast<Real>(lam[tl.row(a)]);
  if (mode == kLamR2) {
    Real o1[TR][TC], o2[TR][TC];
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) {
        o1[a][b] = ((tl.row(a) == tl.col(b)) ? Real(1) : Real(0)) - acc[a][b];
        o2[a][b] = fma(lr[a], acc[a][b], zt[a][b]);
      }
    tl.store_rm(o1, out_rm);
    tl.store_rm(o2, out2);
  } else {
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) acc[a][b] = fma(lr[a], zt[a][b], acc[a][b]);
    if (out_rm) tl.store_rm(acc, out_rm);
    if (out_cm) tl.store_cm(acc, out_cm);
    if (out2) {
#pragma unroll
      for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b)
          if (tl.row(a) == tl.col(b)) {
            const double l = lam[tl.row(a)];
            acc[a][b] = acc[a][b] + static_cast<Real>(l * l);
          }
      tl.store_rm(acc, out2);
    }
  }
}

// ============================================================== (I - S)^{-1} by products
// For the doubling's A = I - R^2 with S = R^2 small, the inverse is the
// product form of the Neumann series, (I - S)^{-1} = (I + S)(I + S^2)(I + S^4)
// ..., i.e. X_0 = I + S, E_0 = S^2, X_{j+1} = X_j + X_j E_{j+1} with E_{j+1} =
// E_j^2 (the Newton-Schulz iteration X <- X (2I - A X) from X_0 = 2I - A):
// after k steps the residual is I - A X_k = S^(2^(k+1)), of norm at most
// ||S||^(2^(k+1)).  With ||S||_inf <= 1e-8 / 1e-4 / 1e-2 / 0.1, k = 0 / 1 / 2 /
// 3 steps bring it below 1e-16: 1 + 2k FP64 tensor-core products against the
// ~950 instructions of the blocked Gauss-Jordan.  Beyond 0.1 the solve stays
// the Gauss-Jordan.  One-warp groups only (the products' buffers rotate, never
// in place).  Off by default: on config 2 (N = 16) and config 5 the solve
// takes the same time with it as without (3 steps at most) and longer with
// fewer steps allowed, since the norm and the extra products cost what the
// shorter elimination saves; it is kept as a tuning option.
#ifndef ADRT_NS_INVERSE
#define ADRT_NS_INVERSE 0
#endif
template <class Gm>
struct UseNS {
  static constexpr bool value = ADRT_NS_INVERSE && UseMMA<Gm>::value && Gm::G == 32;
};

// ||S||_inf (the largest row sum of |S|) of a row-major smem matrix over the
// one-warp group, every lane ending with it.
template <class Gm>
__device__ __forceinline__ double ns_norm_inf(const double* S, int t) {
  static_assert(Gm::G == 32, "one-warp groups");
  constexpr int TR = Gm::TR, TC = Gm::TC, CB = Gm::CB;
  const Tile<Gm> tl(t);
  double X[TR][TC];
  if (tl.valid()) {
    tl.load_rm(X, S);
  } else {
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) X[a][b] = 0.0;
  }
  double m = 0.0;
#pragma unroll
  for (int a = 0; a < TR; ++a) {
    double r = 0.0;
#pragma unroll
    for (int b = 0; b < TC; ++b) r += fabs(X[a][b]);
#pragma unroll
    for (int o = 1; o < CB; o <<= 1) r += __shfl_xor_sync(0xffffffffu, r, o);  // the row's sum
    m = fmax(m, r);
  }
#pragma unroll
  for (int o = CB; o < 32; o <<= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  return m;
}

// Product-form steps for ||S||_inf = nrm, or -1 when the Gauss-Jordan serves
// (at most ADRT_NS_MAX_STEPS: a longer chain of dependent products is no
// shorter than the elimination).
#ifndef ADRT_NS_MAX_STEPS
#define ADRT_NS_MAX_STEPS 3
#endif
__device__ __forceinline__ int ns_steps(double nrm) {
  const int k = !(nrm <= 0.1) ? -1 : nrm <= 1e-8 ? 0 : nrm <= 1e-4 ? 1 : nrm <= 1e-2 ? 2 : 3;
  return k > ADRT_NS_MAX_STEPS ? -1 : k;
}

// dst = I + sign * src (row-major, tile order).
template <class Gm>
__device__ __noinline__ void op_id_plus(unsigned src_off, unsigned dst_off, double sign, int t) {
  constexpr int TR = Gm::TR, TC = Gm::TC;
  const Tile<Gm> tl(t);
  if (!tl.valid()) return;
  double X[TR][TC];
  tl.load_rm(X, sp<double>(src_off));
#pragma unroll
  for (int a = 0; a < TR; ++a)
#pragma unroll
    for (int b = 0; b < TC; ++b)
      X[a][b] = ((tl.row(a) == tl.col(b)) ? 1.0 : 0.0) + sign * X[a][b];
  tl.store_rm(X, sp<double>(dst_off));
}

// FP64 right-solve X = B A^{-1} on the tensor cores, without pivoting.
//
// Every matrix the solver inverts is I - R R' with R, R' reflection matrices
// (non-negative, row sums <= 1): I - R^2 in the doubling, I - R_b R in the
// adding, (I - R R_b)^T at the interfaces and their transposes in the adjoint.
// Such a matrix is diagonally dominant by rows (or, transposed, by columns),
// so elimination without pivoting is backward stable, and partial pivoting
// -- the reference's LU of A^T (src/matrix.hpp:120-124) -- would choose the
// diagonal at every step.
//
// The stacked matrix M = [A; B] (2NP x NP) lives in m8n8k4 accumulator
// fragments.  Columns are eliminated four at a time: for the panel of pivot
// rows/columns 4j..4j+3 with 4x4 pivot block P, the panel columns become
// M[:, panel] P^{-1} (each row's four entries times P^{-1}, computed from the
// published pivot rows by every thread) and every other column c becomes
// M[:, c] - (M[:, panel] P^{-1}) M[pivot rows, c], one k = 4 DMMA per 8x8
// tile.  After NP/4 panels the A part is I and the B part is B A^{-1}.
// lbuf (8 NP doubles) and rbuf (4 (NP + 4) doubles) are scratch.
#ifndef ADRT_GJ_MMA
#define ADRT_GJ_MMA 1
#endif

template <class Gm>
struct UseGjMMA {
  static constexpr int NP = Gm::NP, NW = Gm::G / 32;
  static constexpr bool value = ADRT_GJ_MMA && sizeof(typename Gm::Real) == 8 && NP >= 8 &&
                                2 * NP <= Gm::G &&  // one thread per row of [A; B]
                                ((2 * NP / 8) * (NP / 8)) % NW == 0;
};

// The pivot-free solve's safety net: a pivot below kGjMinPivot in magnitude
// (or not finite) means the matrix is not the diagonally dominant one the
// argument above covers; gj_mma then returns kGjWeakPivot and the caller
// solves again with partial pivoting.  Every such matrix here is I minus a product
// of reflection matrices with O(1) entries, so the bound is absolute.
#ifndef ADRT_GJ_FALLBACK
#define ADRT_GJ_FALLBACK 1  // tuning: 0 leaves out the pivoted re-solve
#endif
#ifndef ADRT_GJ_MIN_PIVOT
#define ADRT_GJ_MIN_PIVOT 1e-10  // tuning
#endif
constexpr double kGjMinPivot = ADRT_GJ_MIN_PIVOT;
constexpr int kGjWeakPivot = 2;  // op_gj result bit: solved again with pivoting

// Device status bits of op_gj results (adrt_device_flag): an exactly zero
// pivot (1), a pivoted re-solve (8).
__device__ __forceinline__ unsigned status_bits(int gj) {
  return ((gj & 1) ? 1u : 0u) | ((gj & kGjWeakPivot) ? 8u : 0u);
}

template <class Gm, class GO = Gm, bool OUTG = false>
__device__ __forceinline__ int gj_mma(const double* A_rm, const double* B_rm, const double* bvec,
                                      double* out_cm, double* out_rm, double* lbuf, double* rbuf,
                                      int t, int bar, double* out_g = nullptr) {
  constexpr int NP = Gm::NP, LD = Gm::LD, G = Gm::G, NW = G / 32;
  constexpr int NTR = 2 * NP / 8, NTC = NP / 8, TPW = NTR * NTC / NW;
  constexpr int RS = NP + 4;  // rbuf row stride (conflict-free B-fragment loads)
  constexpr int NROW = 2 * NP;
  const int warp = t >> 5, lane = t & 31, g = lane >> 2, q = lane & 3;
  double acc[TPW][2];
#pragma unroll
  for (int u = 0; u < TPW; ++u) {
    const int tau = warp * TPW + u, i = tau / NTC, jt = tau % NTC;
    const int r = 8 * i + g, c = 8 * jt + 2 * q;
    double2 v;
    if (r < NP) {
      v = *reinterpret_cast<const double2*>(A_rm + r * LD + c);
    } else if (B_rm) {
      v = *reinterpret_cast<const double2*>(B_rm + (r - NP) * LD + c);
    } else if (bvec) {
      v = (r == NP) ? make_double2(bvec[c], bvec[c + 1]) : make_double2(0.0, 0.0);
    } else {  // identity right-hand side
      v = make_double2((r - NP == c) ? 1.0 : 0.0, (r - NP == c + 1) ? 1.0 : 0.0);
    }
    acc[u][0] = v.x;
    acc[u][1] = v.y;
  }
  int singular = 0, weak = 0;
#pragma unroll
  for (int j = 0; j < NP / 4; ++j) {
    const int pt = j >> 1, half = j & 1;  // tile row/column holding the panel, and which half
    // 1. publish the panel columns (lbuf, 2NP x 4) and the pivot rows (rbuf, 4 x NP)
#pragma unroll
    for (int u = 0; u < TPW; ++u) {
      const int tau = warp * TPW + u, i = tau / NTC, jt = tau % NTC;
      if (jt == pt && (q >> 1) == half)
        *reinterpret_cast<double2*>(lbuf + (8 * i + g) * 4 + 2 * (q & 1)) =
            make_double2(acc[u][0], acc[u][1]);
      if (i == pt && (g >> 2) == half)
        *reinterpret_cast<double2*>(rbuf + (g & 3) * RS + 8 * jt + 2 * q) =
            make_double2(acc[u][0], acc[u][1]);
    }
    gsync<G>(bar);
    // 2. row t of the panel times P^{-1} (every thread reduces P, so the
    //    singular flag is group-uniform; rows < 2NP are stored)
    {
      double P[4][4], x[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const double2 p0 = *reinterpret_cast<const double2*>(rbuf + a * RS + 4 * j);
        const double2 p1 = *reinterpret_cast<const double2*>(rbuf + a * RS + 4 * j + 2);
        P[a][0] = p0.x;
        P[a][1] = p0.y;
        P[a][2] = p1.x;
        P[a][3] = p1.y;
      }
      if (t < NROW) {
        const double2 x0 = *reinterpret_cast<const double2*>(lbuf + t * 4);
        const double2 x1 = *reinterpret_cast<const double2*>(lbuf + t * 4 + 2);
        x[0] = x0.x;
        x[1] = x0.y;
        x[2] = x1.x;
        x[3] = x1.y;
      } else {
        x[0] = x[1] = x[2] = x[3] = 0.0;
      }
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const double piv = P[s][s];
        singular |= (piv == 0.0);
        weak |= !(fabs(piv) >= kGjMinPivot);  // tiny or non-finite
        const double inv = recip(piv);
        const double fx = x[s] * inv;
#pragma unroll
        for (int c = 0; c < 4; ++c)
          if (c != s) x[c] = fma(-fx, P[s][c], x[c]);
        x[s] = fx;
#pragma unroll
        for (int s2 = s + 1; s2 < 4; ++s2) {
          const double f = P[s2][s] * inv;
#pragma unroll
          for (int c = 0; c < 4; ++c)
            if (c != s) P[s2][c] = fma(-f, P[s][c], P[s2][c]);
          P[s2][s] = f;
        }
      }
      const int pr = t - 4 * j;  // pivot rows take the exact unit rows
      if (pr >= 0 && pr < 4) {
#pragma unroll
        for (int c = 0; c < 4; ++c) x[c] = (c == pr) ? 1.0 : 0.0;
      }
      if (t < NROW) {  // each thread reads and writes only its own row
        *reinterpret_cast<double2*>(lbuf + t * 4) = make_double2(x[0], x[1]);
        *reinterpret_cast<double2*>(lbuf + t * 4 + 2) = make_double2(x[2], x[3]);
      }
    }
    gsync<G>(bar);
    // 3. rank-4 update of every tile, then the panel columns take their new values
#pragma unroll
    for (int u = 0; u < TPW; ++u) {
      const int tau = warp * TPW + u, i = tau / NTC, jt = tau % NTC;
      const double a = -lbuf[(8 * i + g) * 4 + q];
      const double b = rbuf[q * RS + 8 * jt + g];
      mma_f64_m8n8k4(acc[u][0], acc[u][1], a, b);
      if (jt == pt && (q >> 1) == half) {
        const double2 l = *reinterpret_cast<const double2*>(lbuf + (8 * i + g) * 4 + 2 * (q & 1));
        acc[u][0] = l.x;
        acc[u][1] = l.y;
      }
    }
    gsync<G>(bar);  // the next panel overwrites lbuf / rbuf
  }
#pragma unroll
  for (int u = 0; u < TPW; ++u) {
    const int tau = warp * TPW + u, i = tau / NTC, jt = tau % NTC;
    const int r = 8 * i + g - NP, c = 8 * jt + 2 * q;
    if (r >= 0) {
      if (out_rm) *reinterpret_cast<double2*>(out_rm + r * LD + c) = make_double2(acc[u][0], acc[u][1]);
      if (out_cm) {
        out_cm[c * LD + r] = acc[u][0];
        out_cm[(c + 1) * LD + r] = acc[u][1];
      }
      if constexpr (OUTG) {  // HBM, in the tile order of GO
        out_g[tile_index<GO>(r, c)] = acc[u][0];
        out_g[tile_index<GO>(r, c + 1)] = acc[u][1];
      }
    }
  }
  return singular | (weak ? kGjWeakPivot : 0);
}

// X = B A^{-1} by Gauss-Jordan column elimination, with column pivoting on
// the largest |entry| of the pivot row -- the pivot rule of the LU with
// partial pivoting of A^T that the reference's right-solve performs
// (src/matrix.hpp:120-124).  A and B are row-major in smem; when B is kNoMat
// the right-hand side is the single row `bvec` (a vector solve), when it is
// kIdentity the result is A^{-1}.  The result is written column-major to
// out_cm and/or row-major to out_rm.  FP64 orders >= 8 take gj_mma (above).
// Returns bit 0 if a pivot was exactly 0, and kGjWeakPivot when the
// tensor-core solve met a weak pivot and the pivoted elimination was used
// instead; `pivot` requests the pivoted elimination from the start.
// OUTG: the result also into HBM (out_g), in the tile order of GO.
template <class Gm, class GO = Gm, bool OUTG = false>
__device__ __noinline__ int gj_pivoted(unsigned a_off, unsigned b_off, unsigned bvec_off,
                                       unsigned ocm_off, unsigned gj_off, unsigned red_off, int t,
                                       int bar, unsigned orm_off, typename Gm::Real* out_g) {
  using Real = typename Gm::Real;
  const Real* A_rm = sp<Real>(a_off);
  const Real* B_rm = (b_off == kNoMat || b_off == kIdentity) ? nullptr : sp<Real>(b_off);
  const Real* bvec = (bvec_off == kNoMat || b_off == kIdentity) ? nullptr : sp<Real>(bvec_off);
  Real* out_cm = sp<Real>(ocm_off);
  Real* gjbuf = sp<Real>(gj_off);
  unsigned* red = sp<unsigned>(red_off);
  constexpr int TR = Gm::TR, TC = Gm::TC, LD = Gm::LD, NP = Gm::NP, DIM = Gm::DIM;
  constexpr int G = Gm::G;
  const Tile<Gm> tl(t);
  const bool tv = tl.valid();
  Real A[TR][TC], B[TR][TC];
  if (tv) {
    tl.load_rm(A, A_rm);
    if (B_rm) {
      tl.load_rm(B, B_rm);
    } else if (bvec) {
#pragma unroll
      for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) B[a][b] = (tl.row(a) == 0) ? bvec[tl.col(b)] : Real(0);
    } else {
#pragma unroll
      for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) B[a][b] = (tl.row(a) == tl.col(b)) ? Real(1) : Real(0);
    }
  } else {
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) A[a][b] = B[a][b] = Real(0);
  }
  unsigned used = 0;
  int q[TC];
#pragma unroll
  for (int b = 0; b < TC; ++b) q[b] = 0;
  int singular = 0;
  for (int kr = 0; kr * TR < NP; ++kr) {
#pragma unroll
    for (int ka = 0; ka < TR; ++ka) {
      const int k = kr * TR + ka;
      const int par = k & 1;
      Real* rowb = gjbuf + par * DIM;
      Real* colA = gjbuf + 2 * DIM + par * DIM;
      Real* colB = gjbuf + 4 * DIM + par * DIM;
      Real* invb = gjbuf + 6 * DIM + par;
      const bool own_row = tv && (tl.rb == kr);
      // 1. pivot: largest |A[k][c]| over unused columns c
      unsigned key = 0;
      if (own_row) {
#pragma unroll
        for (int b = 0; b < TC; ++b) {
          const int c = tl.col(b);
          if (!((used >> c) & 1u)) {
            const unsigned bits = __float_as_uint(fabsf(static_cast<float>(A[ka][b])));
            key = max(key, (bits & ~63u) | 32u | (unsigned)c);
          }
        }
      }
      key = gmax_u32<G>(key, red, par, bar);
      const int p = (int)(key & 31u);
      singular |= ((key >> 6) == 0u);
      used |= 1u << p;
      const int pb = p % TC;
      const bool own_col = tv && (tl.cb == p / TC);
      // 2. publish row k, column p and 1/pivot
      if (own_row) {
        sts_vec<Real, TC>(rowb + tl.cb * TC, A[ka]);
        if (own_col) {
          Real piv = A[ka][0];
#pragma unroll
          for (int b = 1; b < TC; ++b)
            if (pb == b) piv = A[ka][b];
          *invb = recip(piv);
        }
      }
      if (own_col) {
        Real va[TR], vb[TR];
#pragma unroll
        for (int a = 0; a < TR; ++a) {
          va[a] = A[a][0];
          vb[a] = B[a][0];
#pragma unroll
          for (int b = 1; b < TC; ++b)
            if (pb == b) {
              va[a] = A[a][b];
              vb[a] = B[a][b];
            }
        }
        sts_vec<Real, TR>(colA + tl.rb * TR, va);
        sts_vec<Real, TR>(colB + tl.rb * TR, vb);
      }
      gsync<G>(bar);
      // 3. eliminate column p from every other column
      if (tv) {
        const Real inv = *invb;
        Real cA[TR], cB[TR], rv[TC];
        lds_vec<Real, TR>(cA, colA + tl.rb * TR);
        lds_vec<Real, TR>(cB, colB + tl.rb * TR);
        lds_vec<Real, TC>(rv, rowb + tl.cb * TC);
#pragma unroll
        for (int a = 0; a < TR; ++a) {
          cA[a] *= inv;
          cB[a] *= inv;
        }
#pragma unroll
        for (int b = 0; b < TC; ++b) {
          const bool isp = (tl.col(b) == p);
#pragma unroll
          for (int a = 0; a < TR; ++a) {
            const Real na = fma(-cA[a], rv[b], A[a][b]);
            const Real nb = fma(-cB[a], rv[b], B[a][b]);
            A[a][b] = isp ? cA[a] : na;
            B[a][b] = isp ? cB[a] : nb;
          }
          if (isp) q[b] = k;
        }
      }
    }
  }
  // column c of the reduced B is column q[c] of B A^{-1}
  if (tv) {
#pragma unroll
    for (int b = 0; b < TC; ++b) {
      Real colv[TR];
#pragma unroll
      for (int a = 0; a < TR; ++a) colv[a] = B[a][b];
      if (ocm_off != 0xffffffffu) sts_vec<Real, TR>(out_cm + q[b] * LD + tl.rb * TR, colv);
      if (orm_off != 0xffffffffu) {
        Real* out_rm = sp<Real>(orm_off);
#pragma unroll
        for (int a = 0; a < TR; ++a) out_rm[tl.row(a) * LD + q[b]] = colv[a];
      }
      if constexpr (OUTG) {
#pragma unroll
        for (int a = 0; a < TR; ++a) out_g[tile_index<GO>(tl.row(a), q[b])] = colv[a];
      }
    }
  }
  return singular;
}

// ============================================================== FP32 on the tensor cores
// FP32 products as three TF32 tensor-core products (mma.sync m16n8k8 tf32,
// FP32 accumulation): x = x_hi + x_lo with x_hi = tf32(x) and x_lo =
// tf32(x - x_hi) (both rounded to nearest), and X Y = X_lo Y_hi + X_hi Y_lo +
// X_hi Y_hi (the X_lo Y_lo term, 2^-22 relative, is dropped).  The error per
// product is about 2^-21 of |X| |Y|, close to an FP32 product's; the tensor
// pipe issues the 16x16x16 product in 12 instructions against 128 FFMA.
template <class Gm>
struct UseTC32 {
  static constexpr bool value = ADRT_GEMM_MMA && sizeof(typename Gm::Real) == 4 &&
                                ((Gm::NP == 16 && Gm::G == 32) || (Gm::NP == 32 && Gm::G == 128));
};

__device__ __forceinline__ unsigned tf32_rna(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void mma_tf32_m16n8k8(float (&d)[4], const unsigned (&a)[4],
                                                 const unsigned (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// The warp's 16 x 16 output tile at (r0, c0) of C = X Y: X row-major, Y given
// column-major (YT[n * LD + k] = Y[k][n]), both FP32 in smem with pitch LD.
// acc[j][e] is element (r0 + g + 8 (e >> 1), c0 + 8 j + 2 q + (e & 1)) with
// g = lane / 4, q = lane % 4 (the m16n8 accumulator fragment of column tile j).
// With LD = NP + 4 every operand load is free of bank conflicts.
template <int NP, int LD>
__device__ __forceinline__ void tc32_tile(const float* __restrict__ X, const float* __restrict__ YT,
                                          int r0, int c0, int lane, float (&acc)[2][4]) {
  const int g = lane >> 2, q = lane & 3;
  float hi[2][4], lo[2][4];  // X_hi Y_hi and the two correction products, apart
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) hi[j][e] = lo[j][e] = 0.f;
#pragma unroll
  for (int k0 = 0; k0 < NP; k0 += 8) {
    float xa[4], yb[2][2];
    xa[0] = X[(r0 + g) * LD + k0 + q];
    xa[1] = X[(r0 + g + 8) * LD + k0 + q];
    xa[2] = X[(r0 + g) * LD + k0 + q + 4];
    xa[3] = X[(r0 + g + 8) * LD + k0 + q + 4];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      yb[j][0] = YT[(c0 + 8 * j + g) * LD + k0 + q];
      yb[j][1] = YT[(c0 + 8 * j + g) * LD + k0 + q + 4];
    }
    unsigned ah[4], al[4], bh[2][2], bl[2][2];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      ah[e] = tf32_rna(xa[e]);
      al[e] = tf32_rna(xa[e] - __uint_as_float(ah[e]));
    }
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        bh[j][e] = tf32_rna(yb[j][e]);
        bl[j][e] = tf32_rna(yb[j][e] - __uint_as_float(bh[j][e]));
      }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      mma_tf32_m16n8k8(lo[j], al, bh[j]);
      mma_tf32_m16n8k8(lo[j], ah, bl[j]);
      mma_tf32_m16n8k8(hi[j], ah, bh[j]);
    }
  }
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[j][e] = hi[j][e] + lo[j][e];
}

// The warp's output tile origin in a group of NP x NP products: one 16 x 16
// tile per warp (one warp at NP = 16, four at NP = 32).
template <class Gm>
__device__ __forceinline__ void tc32_origin(int t, int& r0, int& c0) {
  const int warp = t >> 5;
  r0 = (Gm::NP == 32) ? 16 * (warp >> 1) : 0;
  c0 = (Gm::NP == 32) ? 16 * (warp & 1) : 0;
}

// FP32 right-solve X = B A^{-1} without pivoting, one row of [A; B] per
// thread (two threads per row, each half of the columns, at NP = 32).  The
// matrices inverted are diagonally dominant (I - R R' with reflection
// matrices R, R'), so elimination without pivoting is backward stable (see
// gj_mma).  Columns are eliminated four at a time: the panel's pivot rows and
// every row's panel entries are published, each thread forms its row's panel
// entries times the 4 x 4 pivot block's inverse, x' = x P^{-1}, and updates
// its other columns c by x' P[:, c].  A and B are row-major (pitch LD); the
// result goes row-major to `out`, whose buffer is also the scratch of the
// publication (2NP x 4 panel entries, then 4 pivot rows).  Returns nonzero if
// a pivot was exactly 0.
template <class Gm>
struct UseGjRows {
  static constexpr int NP = Gm::NP, G = Gm::G;
  static constexpr bool value = sizeof(typename Gm::Real) == 4 && (NP == 16 || NP == 32) &&
                                G % (2 * NP) == 0 && NP / (G / (2 * NP)) >= 4;
};

template <class Gm, int PART>
__device__ __forceinline__ int gj_rows_part(const float* A, const float* B, float* out, int row,
                                            int bar) {
  constexpr int NP = Gm::NP, LD = Gm::LD, G = Gm::G;
  constexpr int ROWS = 2 * NP, TPR = G / ROWS, CPT = NP / TPR, C0 = PART * CPT;
  constexpr int RS = NP + 4;  // pivot-row pitch
  float* lbuf = out;
  float* rbuf = out + ROWS * 4;
  float v[CPT];
  const float* src = (row < NP) ? A + row * LD : B + (row - NP) * LD;
  lds_vec<float, CPT>(v, src + C0);
  int singular = 0;
#pragma unroll
  for (int j = 0; j < NP / 4; ++j) {
    const int pc = 4 * j;
    // 1. publish this row's panel entries and, on the pivot rows, the row
    if (pc >= C0 && pc < C0 + CPT)
      *reinterpret_cast<float4*>(lbuf + row * 4) =
          make_float4(v[(pc - C0) & (CPT - 1)], v[(pc - C0 + 1) & (CPT - 1)],
                      v[(pc - C0 + 2) & (CPT - 1)], v[(pc - C0 + 3) & (CPT - 1)]);
    if (row >= pc && row < pc + 4) sts_vec<float, CPT>(rbuf + (row - pc) * RS + C0, v);
    gsync<G>(bar);
    // 2. x' = x P^{-1} (every thread factors the pivot block itself)
    float P[4][4], x[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) lds_vec<float, 4>(P[a], rbuf + a * RS + pc);
    lds_vec<float, 4>(x, lbuf + row * 4);
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const float piv = P[s][s];
      singular |= (piv == 0.f);
      const float inv = recip(piv);
      const float fx = x[s] * inv;
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (c != s) x[c] = fmaf(-fx, P[s][c], x[c]);
      x[s] = fx;
#pragma unroll
      for (int s2 = s + 1; s2 < 4; ++s2) {
        const float f = P[s2][s] * inv;
#pragma unroll
        for (int c = 0; c < 4; ++c)
          if (c != s) P[s2][c] = fmaf(-f, P[s][c], P[s2][c]);
        P[s2][s] = f;
      }
    }
    if (row >= pc && row < pc + 4) {  // pivot rows take the exact unit rows
#pragma unroll
      for (int c = 0; c < 4; ++c) x[c] = (c == row - pc) ? 1.f : 0.f;
    }
    // 3. the row's columns: panel columns take x', the others lose x' P[:, c]
#pragma unroll
    for (int c4 = 0; c4 < CPT; c4 += 4) {
      const int c = C0 + c4;
      if (c == pc) {
#pragma unroll
        for (int e = 0; e < 4; ++e) v[c4 + e] = x[e];
      } else {
        float pr[4][4];
#pragma unroll
        for (int s = 0; s < 4; ++s) lds_vec<float, 4>(pr[s], rbuf + s * RS + c);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          float a = v[c4 + e];
#pragma unroll
          for (int s = 0; s < 4; ++s) a = fmaf(-x[s], pr[s][e], a);
          v[c4 + e] = a;
        }
      }
    }
    gsync<G>(bar);  // the next panel (or the result) overwrites the publication
  }
  if (row >= NP) sts_vec<float, CPT>(out + (row - NP) * LD + C0, v);
  return singular;
}

template <class Gm>
__device__ __noinline__ int op_gj_rows(unsigned a_off, unsigned b_off, unsigned out_off, int t,
                                       int bar) {
  static_assert(UseGjRows<Gm>::value, "row-parallel Gauss-Jordan geometry");
  constexpr int ROWS = 2 * Gm::NP;
  const float* A = sp<float>(a_off);
  const float* B = sp<float>(b_off);
  float* out = sp<float>(out_off);
  // warp-uniform halves at NP = 32 (rows t % 64, column half t / 64)
  const int row = t % ROWS, part = t / ROWS;
  if constexpr (Gm::G / ROWS == 1) {
    return gj_rows_part<Gm, 0>(A, B, out, row, bar);
  } else {
    return part == 0 ? gj_rows_part<Gm, 0>(A, B, out, row, bar)
                     : gj_rows_part<Gm, 1>(A, B, out, row, bar);
  }
}

// The right-solve X = B A^{-1} (arguments as gj_pivoted): FP64 orders >= 8
// on the tensor cores without pivoting (gj_mma), and the pivoted
// elimination (a function of its own, so that the tensor-core path keeps its
// registers) when `pivot` asks for it, or for the other orders and FP32.
// Returns bit 0 if a pivot was exactly 0, and kGjWeakPivot when the
// tensor-core solve met a weak pivot: its result is then not to be used, and
// the caller solves again with pivoting (op_gj_safe below for one solve; the
// forward solves the whole wavenumber again in a second pass).
template <class Gm, class GO = Gm, bool OUTG = false>
__device__ __noinline__ int op_gj(unsigned a_off, unsigned b_off, unsigned bvec_off,
                                  unsigned ocm_off, unsigned gj_off, unsigned red_off, int t,
                                  int bar, unsigned orm_off = 0xffffffffu,
                                  typename Gm::Real* out_g = nullptr, int pivot = 0) {
  using Real = typename Gm::Real;
  if constexpr (UseGjMMA<Gm>::value) {
    constexpr int NP = Gm::NP, LD = Gm::LD, DIM = Gm::DIM;
    static_assert(4 * (NP + 4) <= 6 * DIM + 4 && 8 * NP <= NP * LD, "gj_mma scratch");
    if (!pivot) {
      const Real* A_rm = sp<Real>(a_off);
      const Real* B_rm = (b_off == kNoMat || b_off == kIdentity) ? nullptr : sp<Real>(b_off);
      const Real* bvec = (bvec_off == kNoMat || b_off == kIdentity) ? nullptr : sp<Real>(bvec_off);
      Real* out_rm = (orm_off == kNoMat) ? nullptr : sp<Real>(orm_off);
      Real* o_cm = (ocm_off == kNoMat) ? nullptr : sp<Real>(ocm_off);
      // scratch: the output buffer, or the one matrix buffer the call names
      Real* lbuf = o_cm ? o_cm : out_rm;
      const int r = gj_mma<Gm, GO, OUTG>(A_rm, B_rm, bvec, o_cm, out_rm, lbuf, sp<Real>(gj_off),
                                         t, bar, out_g);
      return ADRT_GJ_FALLBACK ? r : (r & 1);
    }
  }
  return gj_pivoted<Gm, GO, OUTG>(a_off, b_off, bvec_off, ocm_off, gj_off, red_off, t, bar,
                                  orm_off, out_g);
}

// op_gj with its own safety net, for solves outside the forward's wavenumber
// pass (whose re-solve covers the whole wavenumber): on a weak pivot the same
// solve again with partial pivoting (A and B are intact), kGjWeakPivot set.
template <class Gm, class GO = Gm, bool OUTG = false>
__device__ __noinline__ int op_gj_safe(unsigned a_off, unsigned b_off, unsigned bvec_off,
                                       unsigned ocm_off, unsigned gj_off, unsigned red_off, int t,
                                       int bar, unsigned orm_off = 0xffffffffu,
                                       typename Gm::Real* out_g = nullptr) {
  const int r = op_gj<Gm, GO, OUTG>(a_off, b_off, bvec_off, ocm_off, gj_off, red_off, t, bar,
                                    orm_off, out_g);
  if (!ADRT_GJ_FALLBACK || !(r & kGjWeakPivot)) return r & ~kGjWeakPivot;
  gsync<Gm::G>(bar);
  return op_gj<Gm, GO, OUTG>(a_off, b_off, bvec_off, ocm_off, gj_off, red_off, t, bar, orm_off,
                             out_g, 1) | kGjWeakPivot;
}

// Tile copies between the HBM scratch and smem.  The HBM side is in the tile
// order of GO: the group's own (thread t owns TE contiguous Reals) or, for
// records written by a kernel of another group size, that kernel's order.
template <class Gm, class GO = Gm>
__device__ __noinline__ void op_g2s(const typename Gm::Real* g, unsigned orm_off,
                                    unsigned ocm_off, int t) {
  using Real = typename Gm::Real;
  Real* out_rm = (orm_off == kNoMat) ? nullptr : sp<Real>(orm_off);
  Real* out_cm = (ocm_off == kNoMat) ? nullptr : sp<Real>(ocm_off);
  constexpr int TR = Gm::TR, TC = Gm::TC;
  const Tile<Gm> tl(t);
  if (!tl.valid()) return;
  Real X[TR][TC];
  if constexpr (GO::G == Gm::G) {
    const Real* p = g + t * Gm::TE;
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) X[a][b] = p[a * TC + b];
  } else {
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) X[a][b] = g[tile_index<GO>(tl.row(a), tl.col(b))];
  }
  if (out_rm) tl.store_rm(X, out_rm);
  if (out_cm) tl.store_cm(X, out_cm);
}

// N matrices from global memory into shared memory (row- and / or
// column-major; kNoMat skips), every load issued before the first store so
// that their latencies overlap.  Bit n of OWN: matrix n is in this group's
// own tile order, else in GO's (a record of the taping forward).
template <class Gm, class GO, int N, unsigned OWN>
__device__ __forceinline__ void g2s_n(const typename Gm::Real* const (&g)[N],
                                      const unsigned (&orm)[N], const unsigned (&ocm)[N], int t) {
  using Real = typename Gm::Real;
  constexpr int TR = Gm::TR, TC = Gm::TC;
  const Tile<Gm> tl(t);
  if (!tl.valid()) return;
  Real X[N][TR][TC];
#pragma unroll
  for (int n = 0; n < N; ++n)
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b)
        X[n][a][b] = ((OWN >> n) & 1u) ? g[n][t * Gm::TE + a * TC + b]
                                       : g[n][tile_index<GO>(tl.row(a), tl.col(b))];
#pragma unroll
  for (int n = 0; n < N; ++n) {
    if (orm[n] != kNoMat) tl.store_rm(X[n], sp<Real>(orm[n]));
    if (ocm[n] != kNoMat) tl.store_cm(X[n], sp<Real>(ocm[n]));
  }
}

template <class Gm, class GO = Gm>
__device__ __noinline__ void op_s2g(unsigned in_off, typename Gm::Real* g, int t) {
  using Real = typename Gm::Real;
  const Real* in_rm = sp<Real>(in_off);
  constexpr int TR = Gm::TR, TC = Gm::TC;
  const Tile<Gm> tl(t);
  if (!tl.valid()) return;
  Real X[TR][TC];
  tl.load_rm(X, in_rm);
  if constexpr (GO::G == Gm::G) {
    Real* p = g + t * Gm::TE;
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) p[a * TC + b] = X[a][b];
  } else {
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) g[tile_index<GO>(tl.row(a), tl.col(b))] = X[a][b];
  }
}

// ============================================================== matvec (warp 0)
// y = X v (NV vectors) with X in smem, column-major (CM) or row-major.
// Executed by warp 0 of the group; every lane ends with the full sums of
// row lane % NP.
template <class Gm, bool CM, int NV>
__device__ __forceinline__ void matvec(const typename Gm::Real* S,
                                       const typename Gm::Real* const (&v)[NV],
                                       typename Gm::Real (&y)[NV], int lane) {
  using Real = typename Gm::Real;
  constexpr int NP = Gm::NP, LPR = Gm::LPR, KCH = Gm::KCH, LD = Gm::LD;
  const int i = lane % NP, part = lane / NP;
#pragma unroll
  for (int n = 0; n < NV; ++n) y[n] = Real(0);
  if (part < LPR) {
    if constexpr (!CM && KCH % 2 == 0) {
      // row-major: two k per 16-byte (8-byte for FP32) load, half the loads
      // and half the bank conflicts of single elements (rows 4 apart share
      // banks at a pitch of 20 doubles); the same k order
      using R2 = typename std::conditional<sizeof(Real) == 8, double2, float2>::type;
#pragma unroll
      for (int kk = 0; kk < KCH; kk += 2) {
        const int k = part * KCH + kk;
        const R2 x2 = *reinterpret_cast<const R2*>(S + i * LD + k);
#pragma unroll
        for (int n = 0; n < NV; ++n) {
          y[n] = fma(x2.x, v[n][k], y[n]);
          y[n] = fma(x2.y, v[n][k + 1], y[n]);
        }
      }
    } else {
#pragma unroll
      for (int kk = 0; kk < KCH; ++kk) {
        const int k = part * KCH + kk;
        const Real x = CM ? S[k * LD + i] : S[i * LD + k];
#pragma unroll
        for (int n = 0; n < NV; ++n) y[n] = fma(x, v[n][k], y[n]);
      }
    }
  }
#pragma unroll
  for (int off = NP; off < NP * LPR; off <<= 1)
#pragma unroll
    for (int n = 0; n < NV; ++n) y[n] += __shfl_xor_sync(0xffffffffu, y[n], off);
}

// y = X v with X an FP32 smem matrix and the vectors in FP64 (accumulated in
// FP64): the source recurrences of the FP32 doubling, whose vectors are
// carried in FP64.  Lane layout as matvec.
template <class Gm, bool CM, int NV>
__device__ __forceinline__ void matvec_fd(const float* S, const double* const (&v)[NV],
                                          double (&y)[NV], int lane) {
  constexpr int NP = Gm::NP, LPR = Gm::LPR, KCH = Gm::KCH, LD = Gm::LD;
  const int i = lane % NP, part = lane / NP;
#pragma unroll
  for (int n = 0; n < NV; ++n) y[n] = 0.0;
  if (part < LPR) {
#pragma unroll
    for (int kk = 0; kk < KCH; ++kk) {
      const int k = part * KCH + kk;
      const double x = CM ? S[k * LD + i] : S[i * LD + k];
#pragma unroll
      for (int n = 0; n < NV; ++n) y[n] = fma(x, v[n][k], y[n]);
    }
  }
#pragma unroll
  for (int off = NP; off < NP * LPR; off <<= 1)
#pragma unroll
    for (int n = 0; n < NV; ++n) y[n] += __shfl_xor_sync(0xffffffffu, y[n], off);
}

// ============================================================== Planck (device)
// Band-integrated Planck function, DisORT method: Simpson refinement for
// narrow bands, small-v polynomial / large-v exponential series otherwise.
// Same algorithm and constants as the reference (src/planck.cpp:13-131) so
// that the level sources agree to round-off.
__host__ __device__ __forceinline__ double planck_kernel_v(double v) { return v * v * v / (exp(v) - 1.0); }

// Host and device: the host copy serves adrt_planck_band().
__host__ __device__ inline double planck_band(double wnumlo, double wnumhi, double temp) {
  const double C2 = 1.438786, SIGMA = 5.67032E-8, VCUT = 1.5;
  const double A1 = 1.0 / 3.0, A2 = -1.0 / 8.0, A3 = 1.0 / 60.0, A4 = -1.0 / 5040.0;
  const double A5 = 1.0 / 272160.0, A6 = -1.0 / 13305600.0;
  if (temp < 0.0 || wnumhi < wnumlo || wnumlo < 0.0) return -1.0;
  if (temp < 1.e-4) return 0.0;
  if (wnumhi == wnumlo) {
    double arg = exp(-C2 * wnumhi / temp);
    return 1.1911e-8 * wnumhi * wnumhi * wnumhi * arg / (1.0 - arg);
  }
  const double vmax = 709.782712893384;  // log(DBL_MAX)
  const double sigdpi = SIGMA / kPi;
  const double conc = 15.0 / pow(kPi, 4.0);
  const double v0 = C2 * wnumlo / temp, v1 = C2 * wnumhi / temp;
  if (v0 > 2.220446049250313e-16 && v1 < vmax && (wnumhi - wnumlo) / wnumhi < 1.e-2) {
    const double hh = v1 - v0;
    double oldval = 0.0;
    const double val0 = planck_kernel_v(v0) + planck_kernel_v(v1);
    for (int n = 1; n <= 10; ++n) {
      const double del = hh / (2.0 * n);
      double val = val0;
      for (int k = 1; k <= 2 * n - 1; ++k) val += 2.0 * (1 + k % 2) * planck_kernel_v(v0 + k * del);
      val *= del * A1;
      if (fabs((val - oldval) / val) <= 1.e-6) return sigdpi * pow(temp, 4.0) * conc * val;
      oldval = val;
    }
    return sigdpi * pow(temp, 4.0) * conc * oldval;
  }
  const double vcp[7] = {10.25, 5.7, 3.9, 2.9, 2.3, 1.9, 0.0};
  double v[2] = {v0, v1}, p[2] = {0.0, 0.0}, d[2] = {0.0, 0.0};
  int smallv = 0;
  for (int i = 0; i < 2; ++i) {
    if (v[i] < VCUT) {
      smallv++;
      const double vsq = v[i] * v[i];
      p[i] = conc * vsq * v[i] * (A1 + v[i] * (A2 + v[i] * (A3 + vsq * (A4 + vsq * (A5 + vsq * A6)))));
    } else {
      int mmax = 1;
      while (v[i] < vcp[mmax - 1]) mmax++;
      const double ex = exp(-v[i]);
      double exm = 1.0;
      double s = 0.0;
      for (int m = 1; m <= mmax; ++m) {
        const double mv = m * v[i];
        exm *= ex;
        s += exm * (6.0 + mv * (6.0 + mv * (3.0 + mv))) / (double)(m * m * m * m);
      }
      d[i] = s * conc;
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

// Single-wavenumber Planck function of the raw-coefficient entry point,
// B(T, nu) = c1 nu^3 / (exp(c2 nu / T) - 1) with c1 = 2 h c^2 = 1.19105e-8
// W m^-2 cm (CGS with the 1e-3 unit factor) and c2 = h c / k = 1.43879 cm K,
// zero below 1e-5 K (src_cuda/cuda_planck_single.cuh:19-35; evaluated in FP64).
__host__ __device__ inline double planck_single(double temp, double nu) {
  const double c1 = 1.19105e-08, c2 = 1.43879;
  if (temp < 1e-5) return 0.0;
  return c1 * nu * nu * nu / (exp(c2 * nu / temp) - 1.0);
}

// Extra doublings from omega (src/doubling.hpp:20-26).
__device__ __forceinline__ int ipow0(double omega) {
  return omega < 0.01 ? 4 : (omega < 0.1 ? 10 : 16);
}

// nn = max(1, trunc(ln tau / ln 2) + ipow0) (src/doubling.hpp:107-109).  An
// exact power of two takes its exponent directly, so that the truncation
// agrees with the host library on the inputs where ln(tau)/ln(2) is integral.
// Non-finite or absurdly large optical depths are clamped to 64 doublings so a
// bad input can never run the loop unbounded (the prologue flags it).
constexpr int kMaxDoublings = 64;
__device__ __forceinline__ int num_doublings(double tau, double omega) {
  if (!(tau < 1e300)) return kMaxDoublings;
  int e;
  const double m = frexp(tau, &e);
  int lg;
  if (m == 0.5)
    lg = e - 1;
  else
    lg = (int)(log(tau) / log(2.0));
  const int nn = lg + ipow0(omega);
  return nn < 1 ? 1 : (nn > kMaxDoublings ? kMaxDoublings : nn);
}

}  // namespace adrt_dev
