// PMCHWT system-matrix assembly on sm_100a.
//
// Replaces sysmat_pmchwt / computeD / computeH / computeK (sysmat.f90:18-519)
// with the intK1/intK2/intK4 source integrals (srcint.f90:57-448), the
// Green's functions (green.f90:40-151) and the closed-form singular terms
// (int.f90:15-407).
//
// Formulation.  For a test face m (centroid c_m, points r = c_m + rho) and a
// source face n (centroid c_n, points r' = c_n + rho'), with d = c_m - c_n,
// one pass over the NQ x NQ point pairs evaluates G = e^{ikR}/(4 pi R) and
// the gradient phasor phi = e^{ikR}(1/R^3 - ik/R^2)/(4 pi) once per pair and
// reduces them into 18 complex moments; the 3 x 3 edge-pair blocks of D+H
// and K follow in closed form from those moments (the RWG functions are
// affine in the point), e.g.
//   D(p,q) = c1 sl_p sl_q / 4 * sum_r w_r (rho - mu_p).sum_r' w' G (rho' - nu_q)
// with mu_p, nu_q the free RWG vertices relative to the centroids and
// sl = sign * edge length.  The reference evaluates intK2 per test point
// (srcint.f90:158) and contracts afterwards (sysmat.f90:326-343); the sums
// are the same, only the rounding order differs.
//
// Kernels:
//   pair_kernel<T>    all face pairs with the regular G (T = double for the
//                     FP64 path, float for the mixed path in units of the
//                     domain's average edge length);
//   near_static_kernel  once per geometry: the wavelength-independent
//                     closed-form integrals (int.f90) of every near pair,
//                     contracted with the test functions;
//   near_kernel       per wavelength, FP64: the smoothed-G quadrature of the
//                     near pairs plus the closed-form terms scaled by
//                     1/(4 pi) and k^2/(8 pi) (srcint.f90:21-53,121-154,
//                     330-366); overwrites the near blocks;
//   gather_kernel     sums the (up to) four face-pair blocks of every
//                     edge pair and adds them to A with the Zsi and sign
//                     factors of sysmat.f90:70-99.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include <type_traits>

#include "mom_internal.h"

namespace mom {

__constant__ double c_qw[kMaxQ];
__constant__ double c_qn[kMaxQ][3];

namespace {

constexpr int kPairThreads = 128;
constexpr int kTestPerCta = 8;
constexpr double kOofpi = 1.0 / (4.0 * kPi);  // green.f90:20-21

template <typename T>
struct Cx {
  T re, im;
};

__device__ __forceinline__ void fsincos(double x, double *s, double *c) { sincos(x, s, c); }
__device__ __forceinline__ void fsincos(float x, float *s, float *c) { __sincosf(x, s, c); }
__device__ __forceinline__ double fexp(double x) { return exp(x); }
__device__ __forceinline__ float fexp(float x) { return __expf(x); }
__device__ __forceinline__ double frsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float frsqrt(float x) { return rsqrtf(x); }

// The 18 moments of one face pair (without the 1/(4 pi) factor).
template <typename T>
struct Moments {
  Cx<T> TA, TD, KG;
  Cx<T> TB[3], TC[3], KC[3], KE[3], KF[3];
};

// The moments of the face pair with the two faces' roles exchanged (test <->
// source): G and the gradient phasor depend on |r - r'| only, so TB <-> TC,
// KC <-> KF, KE -> -KE, and TA, TD, KG stay (the centroid offset of the
// exchanged pair is the negated one).  Both faces use the same point rule.
template <typename T>
__device__ __forceinline__ void exchange_roles(Moments<T> &M) {
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const Cx<T> tb = M.TB[i], kc = M.KC[i];
    M.TB[i] = M.TC[i];
    M.TC[i] = tb;
    M.KC[i] = M.KF[i];
    M.KF[i] = kc;
    M.KE[i].re = -M.KE[i].re;
    M.KE[i].im = -M.KE[i].im;
  }
}

template <typename T>
__device__ __forceinline__ void zero(Cx<T> &a) {
  a.re = 0;
  a.im = 0;
}

// Point-pair loop.  rho_t: test point offsets (stride 3), rho_s: source
// offsets with stride sstride between coordinates; w from constant memory.
// SMOOTH selects the singularity-subtracted kernels (green.f90:40-97).  The
// geometry has its own types (the value type T by default): G for the test
// points, GS for the source points, GD for the centroid offset; the adjoint
// runs T = dual numbers on plain FP64 geometry (permittivity) or on one dual
// and one plain face (vertex coordinates).
template <typename T, int NQ, bool SMOOTH, bool LOSSLESS = false, typename G = T, typename GS = G, typename GD = G>
__device__ __forceinline__ void pair_moments(const G *rho_t, const GS *rho_s, int sstride, const GD d[3], T kr, T ki,
                                             Moments<T> &M) {
  zero(M.TA);
  zero(M.TD);
  zero(M.KG);
#pragma unroll
  for (int i = 0; i < 3; i++) {
    zero(M.TB[i]);
    zero(M.TC[i]);
    zero(M.KC[i]);
    zero(M.KE[i]);
    zero(M.KF[i]);
  }
  // k^2 for the smoothed kernels
  const T k2r = kr * kr - ki * ki, k2i = 2 * kr * ki;
#pragma unroll 1
  for (int t = 0; t < NQ; t++) {
    const G rx = rho_t[3 * t], ry = rho_t[3 * t + 1], rz = rho_t[3 * t + 2];
    const G wt = (G)c_qw[t];
    const auto ax = d[0] + rx, ay = d[1] + ry, az = d[2] + rz;
    Cx<T> G0 = {0, 0}, P0 = {0, 0}, G1[3] = {{0, 0}, {0, 0}, {0, 0}}, P1[3] = {{0, 0}, {0, 0}, {0, 0}};
#pragma unroll
    for (int s = 0; s < NQ; s++) {
      const GS sx = rho_s[(3 * s) * sstride], sy = rho_s[(3 * s + 1) * sstride], sz = rho_s[(3 * s + 2) * sstride];
      const GS ws = (GS)c_qw[s];
      const auto dx = ax - sx, dy = ay - sy, dz = az - sz;
      const auto R2 = dx * dx + dy * dy + dz * dz;
      T gre, gim, pre, pim;
      if (R2 > 0) {
        const auto iR = frsqrt(R2);
        const auto R = R2 * iR;
        T sn, cs;
        fsincos(kr * R, &sn, &cs);
        const T ea = LOSSLESS ? (T)1 : fexp(-ki * R);  // real k: no decay factor
        const T er = ea * cs, ei = ea * sn;  // e^{ikR}
        const auto iR2 = iR * iR;
        const auto iR3 = iR2 * iR;
        // q = 1/R^3 - i k / R^2 = (iR3 + ki iR2) - i kr iR2
        const T qr = iR3 + ki * iR2, qi = -kr * iR2;
        if (SMOOTH) {
          // Gs*4pi = (e - 1)/R + k^2 R / 2 ; phis*4pi = e q - 1/R^3 - k^2/(2R)
          gre = ((er - (T)1) * iR + (T)0.5 * k2r * R) * ws;
          gim = (ei * iR + (T)0.5 * k2i * R) * ws;
          pre = (er * qr - ei * qi - iR3 - (T)0.5 * k2r * iR) * ws;
          pim = (er * qi + ei * qr - (T)0.5 * k2i * iR) * ws;
        } else {
          const auto g = iR * ws;
          gre = er * g;
          gim = ei * g;
          pre = (er * qr - ei * qi) * ws;
          pim = (er * qi + ei * qr) * ws;
        }
      } else {
        if (SMOOTH) {  // R = 0 limits: Gs = ik/(4 pi), grad Gs = 0
          gre = -ki * ws;
          gim = kr * ws;
        } else {
          gre = 0;
          gim = 0;
        }
        pre = 0;
        pim = 0;
      }
      G0.re += gre;
      G0.im += gim;
      P0.re += pre;
      P0.im += pim;
      G1[0].re += gre * sx; G1[0].im += gim * sx;
      G1[1].re += gre * sy; G1[1].im += gim * sy;
      G1[2].re += gre * sz; G1[2].im += gim * sz;
      P1[0].re += pre * sx; P1[0].im += pim * sx;
      P1[1].re += pre * sy; P1[1].im += pim * sy;
      P1[2].re += pre * sz; P1[2].im += pim * sz;
    }
    // Test-side sums.
    const G rr[3] = {rx, ry, rz};
    M.TA.re += wt * (rx * G1[0].re + ry * G1[1].re + rz * G1[2].re);
    M.TA.im += wt * (rx * G1[0].im + ry * G1[1].im + rz * G1[2].im);
    M.TD.re += wt * G0.re;
    M.TD.im += wt * G0.im;
    M.KG.re += wt * P0.re;
    M.KG.im += wt * P0.im;
#pragma unroll
    for (int i = 0; i < 3; i++) {
      M.TB[i].re += wt * G0.re * rr[i];
      M.TB[i].im += wt * G0.im * rr[i];
      M.TC[i].re += wt * G1[i].re;
      M.TC[i].im += wt * G1[i].im;
      M.KC[i].re += wt * P0.re * rr[i];
      M.KC[i].im += wt * P0.im * rr[i];
      M.KF[i].re += wt * P1[i].re;
      M.KF[i].im += wt * P1[i].im;
    }
    // KE += w rho x P1
    M.KE[0].re += wt * (ry * P1[2].re - rz * P1[1].re);
    M.KE[0].im += wt * (ry * P1[2].im - rz * P1[1].im);
    M.KE[1].re += wt * (rz * P1[0].re - rx * P1[2].re);
    M.KE[1].im += wt * (rz * P1[0].im - rx * P1[2].im);
    M.KE[2].re += wt * (rx * P1[1].re - ry * P1[0].re);
    M.KE[2].im += wt * (rx * P1[1].im - ry * P1[0].im);
  }
}

struct Cd {
  double re, im;
};
__device__ __forceinline__ Cd cmul(Cd a, Cd b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

template <typename R>
struct Cr {
  R re, im;
};
template <typename R>
__device__ __forceinline__ Cr<R> cmul(Cr<R> a, Cr<R> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}

// Closed-form 3x3 blocks from the moments, in the real type R (FP64, or FP32
// for FP32 moments).  mu[p][3], nu[q][3], d in the kernel's length unit; fD,
// fH, fK carry c1, c2, 1/(16 pi) and the unit scale.  Writes S = D + H and K,
// interleaved, 18 double2 values.
template <typename T, typename R = double>
__device__ __forceinline__ void blocks_from_moments(const Moments<T> &Mt, const double mu[3][3], const double nu[3][3],
                                                    const double slp[3], const double slq[3], const double d_[3],
                                                    Cd fD_, Cd fH_, double fK_, bool self, double2 *out) {
  using Cd = Cr<R>;
  const R d[3] = {(R)d_[0], (R)d_[1], (R)d_[2]};
  const Cd fD = {(R)fD_.re, (R)fD_.im}, fH = {(R)fH_.re, (R)fH_.im};
  const R fK = (R)fK_;
  auto cv = [](const Cx<T> &a) -> Cd { return {(R)a.re, (R)a.im}; };
  Cd TA = cv(Mt.TA), TD = cv(Mt.TD), KG = cv(Mt.KG);
  Cd TB[3], TC[3], KC[3], KE[3], KF[3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    TB[i] = cv(Mt.TB[i]);
    TC[i] = cv(Mt.TC[i]);
    KC[i] = cv(Mt.KC[i]);
    KE[i] = cv(Mt.KE[i]);
    KF[i] = cv(Mt.KF[i]);
  }
  // K helpers: KBv = d x KF + KE, KDv = d KG + KC, dKE = d . KE
  Cd KBv[3], KDmF[3];
  KBv[0] = {d[1] * KF[2].re - d[2] * KF[1].re + KE[0].re, d[1] * KF[2].im - d[2] * KF[1].im + KE[0].im};
  KBv[1] = {d[2] * KF[0].re - d[0] * KF[2].re + KE[1].re, d[2] * KF[0].im - d[0] * KF[2].im + KE[1].im};
  KBv[2] = {d[0] * KF[1].re - d[1] * KF[0].re + KE[2].re, d[0] * KF[1].im - d[1] * KF[0].im + KE[2].im};
#pragma unroll
  for (int i = 0; i < 3; i++)
    KDmF[i] = {d[i] * KG.re + KC[i].re - KF[i].re, d[i] * KG.im + KC[i].im - KF[i].im};
  Cd dKE = {d[0] * KE[0].re + d[1] * KE[1].re + d[2] * KE[2].re, d[0] * KE[0].im + d[1] * KE[1].im + d[2] * KE[2].im};
  // per q: beta_q = nu.TB, bq = (d x nu).KC, cq = nu.KE
  Cd beta[3], bq[3], cq[3];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const R v[3] = {(R)nu[q][0], (R)nu[q][1], (R)nu[q][2]};
    beta[q] = {v[0] * TB[0].re + v[1] * TB[1].re + v[2] * TB[2].re, v[0] * TB[0].im + v[1] * TB[1].im + v[2] * TB[2].im};
    R dn[3] = {d[1] * v[2] - d[2] * v[1], d[2] * v[0] - d[0] * v[2], d[0] * v[1] - d[1] * v[0]};
    bq[q] = {dn[0] * KC[0].re + dn[1] * KC[1].re + dn[2] * KC[2].re, dn[0] * KC[0].im + dn[1] * KC[1].im + dn[2] * KC[2].im};
    cq[q] = {v[0] * KE[0].re + v[1] * KE[1].re + v[2] * KE[2].re, v[0] * KE[0].im + v[1] * KE[1].im + v[2] * KE[2].im};
  }
#pragma unroll
  for (int p = 0; p < 3; p++) {
    const R u[3] = {(R)mu[p][0], (R)mu[p][1], (R)mu[p][2]};
    Cd alpha = {u[0] * TC[0].re + u[1] * TC[1].re + u[2] * TC[2].re, u[0] * TC[0].im + u[1] * TC[1].im + u[2] * TC[2].im};
    Cd ap = {u[0] * KBv[0].re + u[1] * KBv[1].re + u[2] * KBv[2].re, u[0] * KBv[0].im + u[1] * KBv[1].im + u[2] * KBv[2].im};
    // Z_p = mu_p x (KDv - KF)
    Cd Z[3] = {{u[1] * KDmF[2].re - u[2] * KDmF[1].re, u[1] * KDmF[2].im - u[2] * KDmF[1].im},
               {u[2] * KDmF[0].re - u[0] * KDmF[2].re, u[2] * KDmF[0].im - u[0] * KDmF[2].im},
               {u[0] * KDmF[1].re - u[1] * KDmF[0].re, u[0] * KDmF[1].im - u[1] * KDmF[0].im}};
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const R v[3] = {(R)nu[q][0], (R)nu[q][1], (R)nu[q][2]};
      const R uv = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
      const R ss = (R)slp[p] * (R)slq[q];
      Cd cD = {TA.re - beta[q].re - alpha.re + uv * TD.re, TA.im - beta[q].im - alpha.im + uv * TD.im};
      Cd S1 = cmul(fD, cD), S2 = cmul(fH, TD);
      double2 sv = make_double2((double)(ss * (S1.re + S2.re)), (double)(ss * (S1.im + S2.im)));
      double2 kv = make_double2(0.0, 0.0);
      if (!self) {
        Cd cK = {-dKE.re - ap.re - bq[q].re + cq[q].re + v[0] * Z[0].re + v[1] * Z[1].re + v[2] * Z[2].re,
                 -dKE.im - ap.im - bq[q].im + cq[q].im + v[0] * Z[0].im + v[1] * Z[1].im + v[2] * Z[2].im};
        kv = make_double2((double)(ss * fK * cK.re), (double)(ss * fK * cK.im));
      }
      out[2 * (3 * p + q)] = sv;
      out[2 * (3 * p + q) + 1] = kv;
    }
  }
}

struct PairArgs {
  int F;
  const double *qrel;  // [F][NQ][3]  source faces
  const double *cp;    // [F][3]
  const double *mu;    // [F][3][3]
  const double *sl;    // [F][3]
  const double *tqrel, *tcp, *tmu;  // test faces (mapped by J^T for a group action g != identity)
  int ident;           // identity action: the self pair m == n has no K term
  int sym;             // identity action: each unordered pair once, both blocks written
  double inv_unit;     // 1/L0
  double kr, ki;       // k * L0
  Cd fD, fH;
  double fK;
  double2 *blk;        // [F source][F test][18]
};

// One thread per source face n; the CTA walks kTestPerCta test faces.  In the
// FP32 kernel the source face's FP64 geometry (centroid, edge vectors, edge
// lengths) waits in shared memory while the point-pair loop runs, so it holds
// no registers there (the FP64 kernel's point sources already fill the 48 KB
// of static shared memory and keep it in registers).  MINB CTAs of 128
// threads share an SM (the register cap follows).
template <typename T, int NQ, bool LOSSLESS, int MINB = 3, bool E32 = false>
__global__ void __launch_bounds__(kPairThreads, MINB) pair_kernel(PairArgs a) {
  using R = typename std::conditional<E32, float, double>::type;  // the block contraction's type
  constexpr bool kGeoShared = sizeof(T) == sizeof(float);
  __shared__ T s_src[NQ * 3][kPairThreads];
  __shared__ T s_tst[NQ * 3];
  __shared__ double s_tmu[9], s_tsl[3], s_tcp[3];
  // per source face: cp[3], mu[3][3] / L0, sl[3] / L0
  __shared__ double s_ngeo[kGeoShared ? 15 : 1][kPairThreads];
  double r_ngeo[kGeoShared ? 1 : 15];
  const int tid = threadIdx.x;
  auto ngeo = [&](int i) -> double {
    if constexpr (kGeoShared) return s_ngeo[i][tid];
    else return r_ngeo[i];
  };
  const int n = blockIdx.x * kPairThreads + tid;
  const bool active = n < a.F;
  if (active) {
#pragma unroll
    for (int i = 0; i < NQ * 3; i++) s_src[i][tid] = (T)(a.qrel[(size_t)n * NQ * 3 + i] * a.inv_unit);
    double g[15];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      g[i] = a.cp[3 * n + i];
      g[12 + i] = a.sl[3 * n + i] * a.inv_unit;
#pragma unroll
      for (int j = 0; j < 3; j++) g[3 + 3 * i + j] = a.mu[9 * n + 3 * i + j] * a.inv_unit;
    }
#pragma unroll
    for (int i = 0; i < 15; i++) {
      if constexpr (kGeoShared) s_ngeo[i][tid] = g[i];
      else r_ngeo[i] = g[i];
    }
  }
  const int m0 = blockIdx.y * kTestPerCta;
  // with sym, a CTA whose test faces all come after its source faces has no work
  if (a.sym && (int64_t)m0 > (int64_t)blockIdx.x * kPairThreads + kPairThreads - 1) return;
  for (int mi = 0; mi < kTestPerCta; mi++) {
    const int m = m0 + mi;
    if (m >= a.F) break;
    __syncthreads();
    if (tid < NQ * 3) s_tst[tid] = (T)(a.tqrel[(size_t)m * NQ * 3 + tid] * a.inv_unit);
    if (tid < 9) s_tmu[tid] = a.tmu[9 * m + tid] * a.inv_unit;
    if (tid < 3) {
      s_tsl[tid] = a.sl[3 * m + tid] * a.inv_unit;
      s_tcp[tid] = a.tcp[3 * m + tid];
    }
    __syncthreads();
    if (!active || (a.sym && m > n)) continue;
    T dT[3];
#pragma unroll
    for (int i = 0; i < 3; i++) dT[i] = (T)((s_tcp[i] - ngeo(i)) * a.inv_unit);
    Moments<T> Mt;
    pair_moments<T, NQ, false, LOSSLESS>(s_tst, &s_src[0][tid], kPairThreads, dT, (T)a.kr, (T)a.ki, Mt);
    double mu[3][3], slp[3], nu[3][3], slq[3], dd[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      slp[i] = s_tsl[i];
      slq[i] = ngeo(12 + i);
      dd[i] = (s_tcp[i] - ngeo(i)) * a.inv_unit;
#pragma unroll
      for (int j = 0; j < 3; j++) {
        mu[i][j] = s_tmu[3 * i + j];
        nu[i][j] = ngeo(3 + 3 * i + j);
      }
    }
    blocks_from_moments<T, R>(Mt, mu, nu, slp, slq, dd, a.fD, a.fH, a.fK, a.ident && m == n,
                              a.blk + ((size_t)n * a.F + m) * 18);
    if (a.sym && m < n) {
      // the block of test face n and source face m from the same point pairs
      Moments<T> Ms = Mt;
      exchange_roles(Ms);
#pragma unroll
      for (int i = 0; i < 3; i++) dd[i] = -dd[i];
      blocks_from_moments<T, R>(Ms, nu, mu, slq, slp, dd, a.fD, a.fH, a.fK, false, a.blk + ((size_t)m * a.F + n) * 18);
    }
  }
}

// ---- closed-form static integrals (int.f90), FP64 ------------------------

// The closed-form integrals below are templates on the scalar type S: double
// for the matrix, and a forward-mode dual number for the adjoint gradients.
template <typename S>
struct FaceGeoT {
  S v[3][3];   // vertices
  S s[3][3];   // edge unit vectors s(:,e)
  S mm[3][3];  // in-plane edge normals m(:,e)
  S n[3];      // unit normal
};
using FaceGeo = FaceGeoT<double>;

template <typename S>
__device__ __forceinline__ S dot3(const S *a, const S *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
template <typename S>
__device__ __forceinline__ S norm3(const S *a) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

// int.f90:15-53 intLm1
template <typename S>
__device__ S d_intLm1(const S *r, const FaceGeoT<S> &g, int e) {
  const S *p1 = g.v[e], *p2 = g.v[(e + 1) % 3], *s = g.s[e];
  S a[3] = {r[0] - p2[0], r[1] - p2[1], r[2] - p2[2]}, b[3] = {r[0] - p1[0], r[1] - p1[1], r[2] - p1[2]};
  S Rp = norm3(a), Rm = norm3(b);
  S sp = -dot3(a, s), sm = -dot3(b, s);
  S div1 = Rp - sp, div2 = Rm + sm;
  if (fabs(div1) > fabs(div2)) return log((Rm - sm) / div1);
  return log((Rp + sp) / div2);
}

// int.f90:55-96 intL1 and 98-135 intL3 together (they share R02, Rp, Rm).
template <typename S>
__device__ void d_intL13(const S *r, const FaceGeoT<S> &g, int e, const S *n, S lm1, S *L1, S *L3) {
  const S *p1 = g.v[e], *p2 = g.v[(e + 1) % 3], *s = g.s[e];
  S rp[3];
#pragma unroll
  for (int i = 0; i < 3; i++) rp[i] = r[i] - 0.5 * (p1[i] + p2[i]);
  S h = dot3(n, rp), t = dot3(g.mm[e], rp);
  S R02 = t * t + h * h;
  S a[3] = {r[0] - p2[0], r[1] - p2[1], r[2] - p2[2]}, b[3] = {r[0] - p1[0], r[1] - p1[1], r[2] - p1[2]};
  S Rp = norm3(a), Rm = norm3(b);
  S sp = -dot3(a, s), sm = -dot3(b, s);
  S l1 = (R02 == 0) ? 0.5 * (sp * Rp - sm * Rm) : 0.5 * R02 * lm1 + 0.5 * (sp * Rp - sm * Rm);
  *L1 = l1;
  *L3 = 0.75 * R02 * l1 + 0.25 * (sp * (Rp * Rp * Rp) - sm * (Rm * Rm * Rm));
}

// int.f90:137-162 intSm3h
template <typename S>
__device__ S d_intSm3h(const S *r, const FaceGeoT<S> &g) {
  S a[3][3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    S v[3] = {g.v[k][0] - r[0], g.v[k][1] - r[1], g.v[k][2] - r[2]};
    S l = norm3(v);
#pragma unroll
    for (int i = 0; i < 3; i++) a[k][i] = v[i] / l;
  }
  S x = 1.0 + dot3(a[0], a[1]) + dot3(a[0], a[2]) + dot3(a[1], a[2]);
  S c[3] = {a[1][1] * a[2][2] - a[1][2] * a[2][1], a[1][2] * a[2][0] - a[1][0] * a[2][2],
            a[1][0] * a[2][1] - a[1][1] * a[2][0]};
  S y = fabs(dot3(a[0], c));
  S om = 2.0 * atan2(y, x);
  S rp1[3] = {r[0] - g.v[0][0], r[1] - g.v[0][1], r[2] - g.v[0][2]};
  return dot3(g.n, rp1) > 0.0 ? fabs(om) : -fabs(om);
}

// The closed-form static integrals of face g at one point r that the
// singular parts need (int.f90:137-407 and the intK*singular routines of
// srcint.f90): Sm1 and S1 (intSm1, intS1), rho = r - h n, the edge sums
// mL1 = sum_e m_e L1_e and mL3, and the gradient integrals K3m1 (intK3m1)
// and K31 (intK31).
template <typename S>
struct PointStatic {
  S Sm1, S1, rho[3], mL1[3], mL3[3], K3m1[3], K31[3];
};
template <typename S>
__device__ __forceinline__ void point_static(const S *r, const FaceGeoT<S> &g, PointStatic<S> &o) {
  S Lm1[3], L1[3], L3[3];
  // intSm1 (int.f90:181-226) decides per edge whether intLm1 is needed
  // when h == 0; intL1 always calls intLm1 unless R02 == 0.
  S r1[3] = {r[0] - g.v[0][0], r[1] - g.v[0][1], r[2] - g.v[0][2]};
  S h = dot3(g.n, r1);
#pragma unroll
  for (int e = 0; e < 3; e++) {
    Lm1[e] = d_intLm1(r, g, e);
    d_intL13(r, g, e, g.n, Lm1[e], &L1[e], &L3[e]);
  }
  S tt[3];
#pragma unroll
  for (int e = 0; e < 3; e++) {
    S re[3] = {r[0] - g.v[e][0], r[1] - g.v[e][1], r[2] - g.v[e][2]};
    tt[e] = dot3(g.mm[e], re);
  }
  S Sm3h = d_intSm3h(r, g);
  S Sm1;
  if (h == 0) {
    S e1 = tt[0] == 0 ? S(0.0) : Lm1[0], e2 = tt[1] == 0 ? S(0.0) : Lm1[1], e3 = tt[2] == 0 ? S(0.0) : Lm1[2];
    Sm1 = -(tt[0] * e1 + tt[1] * e2 + tt[2] * e3);
  } else {
    Sm1 = -h * Sm3h - (tt[0] * Lm1[0] + tt[1] * Lm1[1] + tt[2] * Lm1[2]);
  }
  o.Sm1 = Sm1;
  o.S1 = (h * h) / 3.0 * Sm1 - 1.0 / 3.0 * (tt[0] * L1[0] + tt[1] * L1[1] + tt[2] * L1[2]);
#pragma unroll
  for (int i = 0; i < 3; i++) {
    o.rho[i] = r[i] - h * g.n[i];
    o.mL1[i] = g.mm[0][i] * L1[0] + g.mm[1][i] * L1[1] + g.mm[2][i] * L1[2];
    o.mL3[i] = g.mm[0][i] * L3[0] + g.mm[1][i] * L3[1] + g.mm[2][i] * L3[2];
    o.K3m1[i] = g.mm[0][i] * Lm1[0] + g.mm[1][i] * Lm1[1] + g.mm[2][i] * Lm1[2] + g.n[i] * Sm3h;
    o.K31[i] = (h == 0) ? o.mL1[i] : o.mL1[i] - h * g.n[i] * Sm1;
  }
}

// The k-independent closed-form integrals of source face n (geometry g,
// area An, RWG sl and free vertices bnn) at the NQ test points qm of face m
// (area Am, sl slm, free vertices bnm), contracted with the test RWG
// functions: out[0..5] = Dm1, D1, Hm1, H1, Km1, K1 (each 3x3, row p = test
// edge; K terms zero for the self pair).
template <typename S, int NQ>
__device__ void static_terms(const S (*qm)[3], S Am, const S *slm, const S (*bnm)[3], const FaceGeoT<S> &g, S An,
                             const S *sln, const S (*bnn)[3], bool self, S out[6][9]) {
  S acc[6][9];
#pragma unroll
  for (int o = 0; o < 6; o++)
#pragma unroll
    for (int i = 0; i < 9; i++) acc[o][i] = 0.0;
  for (int t = 0; t < NQ; t++) {
    const S *r = qm[t];
    const double wt = c_qw[t];
    PointStatic<S> ps;
    point_static(r, g, ps);
    const S Sm1 = ps.Sm1, S1 = ps.S1;
    const S *rho = ps.rho, *K3m1 = ps.K3m1, *K31 = ps.K31, *mL1 = ps.mL1, *mL3 = ps.mL3;
    // test functions at r: f_p = sl_p/(2 Am) (r - u_p), div f_p = sl_p / Am
    S fp[3][3], dvp[3];
#pragma unroll
    for (int p = 0; p < 3; p++) {
      const S slp = slm[p];
      const S *u = bnm[p];
#pragma unroll
      for (int i = 0; i < 3; i++) fp[p][i] = slp / (2.0 * Am) * (r[i] - u[i]);
      dvp[p] = slp / Am;
    }
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const S slq = sln[q];
      const S cq = slq / (2.0 * An);
      const S *pq = bnn[q];
      S K2m1[3], K21[3], K4m1[3], K41[3], rpq[3];
#pragma unroll
      for (int i = 0; i < 3; i++) {
        K2m1[i] = cq * (mL1[i] + (rho[i] - pq[i]) * Sm1);
        K21[i] = cq * (1.0 / 3.0 * mL3[i] + (rho[i] - pq[i]) * S1);
        rpq[i] = r[i] - pq[i];
      }
      K4m1[0] = -cq * (rpq[1] * K3m1[2] - rpq[2] * K3m1[1]);
      K4m1[1] = -cq * (rpq[2] * K3m1[0] - rpq[0] * K3m1[2]);
      K4m1[2] = -cq * (rpq[0] * K3m1[1] - rpq[1] * K3m1[0]);
      K41[0] = -cq * (rpq[1] * K31[2] - rpq[2] * K31[1]);
      K41[1] = -cq * (rpq[2] * K31[0] - rpq[0] * K31[2]);
      K41[2] = -cq * (rpq[0] * K31[1] - rpq[1] * K31[0]);
      const S K1m1 = slq / An * Sm1, K11 = slq / An * S1;
#pragma unroll
      for (int p = 0; p < 3; p++) {
        const int pq_ = 3 * p + q;
        acc[0][pq_] += wt * dot3(fp[p], K2m1);
        acc[1][pq_] += wt * dot3(fp[p], K21);
        acc[2][pq_] += wt * dvp[p] * K1m1;
        acc[3][pq_] += wt * dvp[p] * K11;
        acc[4][pq_] += wt * dot3(fp[p], K4m1);
        acc[5][pq_] += wt * dot3(fp[p], K41);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 6; k++)
#pragma unroll
    for (int i = 0; i < 9; i++) out[k][i] = (self && k >= 4) ? S(0.0) : acc[k][i] * Am;
}

struct StaticArgs {
  int64_t nnear;
  const int *near_m, *near_n;
  const FaceGeo *geo;  // [F]
  const double *qabs;  // [F][NQ][3]  test points (mapped by J^T for a group action)
  const double *area;  // [F]
  const double *sl;    // [F][3]
  const double *bn;    // [F][3][3] free vertex (absolute) of local edge e, source faces
  const double *tbn;   // the same of the test faces (mapped by J^T for a group action)
  int ident;           // identity action: the self pair has no K term
  double *out;         // [nnear][6][9]
};

// One thread per near pair: the k-independent closed-form integrals of
// source face n at the test points of face m, contracted with the test RWG
// functions: Dm1, D1, Hm1, H1, Km1, K1 (each 3x3, row p = test edge).
template <int NQ>
__global__ void __launch_bounds__(128) near_static_kernel(StaticArgs a) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.nnear) return;
  const int m = a.near_m[j], n = a.near_n[j];
  const FaceGeo g = a.geo[n];
  const double(*qm)[3] = reinterpret_cast<const double(*)[3]>(a.qabs + (size_t)m * NQ * 3);
  const double(*bnm)[3] = reinterpret_cast<const double(*)[3]>(a.tbn + 9 * (size_t)m);
  const double(*bnn)[3] = reinterpret_cast<const double(*)[3]>(a.bn + 9 * (size_t)n);
  double out[6][9];
  static_terms<double, NQ>(qm, a.area[m], a.sl + 3 * m, bnm, g, a.area[n], a.sl + 3 * n, bnn, a.ident && m == n,
                           out);
  double *o = a.out + j * 54;
#pragma unroll
  for (int k = 0; k < 6; k++)
#pragma unroll
    for (int i = 0; i < 9; i++) o[9 * k + i] = out[k][i];
}

struct NearArgs {
  int64_t nnear;
  int F;
  const int *near_m, *near_n;
  const double *qrel, *cp, *mu, *sl;
  const double *tqrel, *tcp, *tmu;  // test faces (mapped by J^T for a group action)
  int ident;
  const double *stat;  // [nnear][54]
  double kr, ki;
  Cd c1, c2;           // -i w mu0, -1/(i w eps0 n^2)
  Cd k2;               // k^2
  double2 *blk;
};

// Per wavelength, FP64: smoothed-G quadrature of each near pair (one thread
// per pair) plus the closed-form terms; overwrites the pair's block.
template <int NQ>
__global__ void __launch_bounds__(128) near_kernel(NearArgs a) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.nnear) return;
  const int m = a.near_m[j], n = a.near_n[j];
  double d[3], mu[3][3], nu[3][3], slp[3], slq[3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    d[i] = a.tcp[3 * m + i] - a.cp[3 * n + i];
    slp[i] = a.sl[3 * m + i];
    slq[i] = a.sl[3 * n + i];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      mu[i][k] = a.tmu[9 * m + 3 * i + k];
      nu[i][k] = a.mu[9 * n + 3 * i + k];
    }
  }
  Moments<double> Mt;
  pair_moments<double, NQ, true>(a.tqrel + (size_t)m * NQ * 3, a.qrel + (size_t)n * NQ * 3, 1, d, a.kr, a.ki, Mt);
  double2 out[18];
  const Cd fD = {a.c1.re * kOofpi / 4.0, a.c1.im * kOofpi / 4.0};
  const Cd fH = {a.c2.re * kOofpi, a.c2.im * kOofpi};
  blocks_from_moments<double>(Mt, mu, nu, slp, slq, d, fD, fH, kOofpi / 4.0, a.ident && m == n, out);
  // closed-form parts: (1/(4 pi)) X_m1 - (k^2/(8 pi)) X_1
  const double *st = a.stat + j * 54;
  const double f4 = 1.0 / (4.0 * kPi);
  const Cd f8 = {a.k2.re / (8.0 * kPi), a.k2.im / (8.0 * kPi)};
  double2 *dst = a.blk + ((size_t)n * a.F + m) * 18;
#pragma unroll
  for (int i = 0; i < 9; i++) {
    Cd dterm = {f4 * st[i] - f8.re * st[9 + i], -f8.im * st[9 + i]};
    Cd hterm = {f4 * st[18 + i] - f8.re * st[27 + i], -f8.im * st[27 + i]};
    Cd kterm = {f4 * st[36 + i] - f8.re * st[45 + i], -f8.im * st[45 + i]};
    Cd sD = cmul(a.c1, dterm), sH = cmul(a.c2, hterm);
    double2 s = out[2 * i], k = out[2 * i + 1];
    s.x += sD.re + sH.re;
    s.y += sD.im + sH.im;
    k.x += kterm.re;
    k.y += kterm.im;
    dst[2 * i] = s;
    dst[2 * i + 1] = k;
  }
}

struct GatherArgs {
  int F, Nd, N;
  const int *eh;    // [Nd][2]
  const int *epar;  // [Nd]
  const double2 *blk;
  // coefficients of the four PMCHWT blocks (sysmat.f90:70-99): [J,J] += cJJ S,
  // [M,M] += cMM S, [M,J] += cMJ K, [J,M] += cJM K; for the identity action
  // 1, Zsi, 1, -1; for group action g in representation r, with its field
  // action e = ef_g(r): e, e det J Zsi, e det J, -e (K here being the mapped
  // pair's K, det J times the reference's).
  Cd cJJ, cMM, cMJ, cJM;
  double2 *A;
  int64_t lda;
};

// Thread per domain edge pair (e1 fastest): S = sum of the face-pair blocks
// over the (+,-) halves of e1 and e2, then the four PMCHWT blocks.
__global__ void __launch_bounds__(256) gather_kernel(GatherArgs a) {
  const int e1 = blockIdx.x * blockDim.x + threadIdx.x;
  const int e2 = blockIdx.y;
  if (e1 >= a.Nd) return;
  const int h1[2] = {a.eh[2 * e1], a.eh[2 * e1 + 1]};
  const int h2[2] = {a.eh[2 * e2], a.eh[2 * e2 + 1]};
  double sr = 0, si = 0, kr = 0, ki = 0;
#pragma unroll
  for (int i = 0; i < 2; i++) {
    if (h1[i] < 0) continue;
#pragma unroll
    for (int j = 0; j < 2; j++) {
      if (h2[j] < 0) continue;
      const int m = h1[i] / 3, p = h1[i] % 3, n = h2[j] / 3, q = h2[j] % 3;
      const double4 v = *reinterpret_cast<const double4 *>(a.blk + ((size_t)n * a.F + m) * 18 + 2 * (3 * p + q));
      sr += v.x;
      si += v.y;
      kr += v.z;
      ki += v.w;
    }
  }
  const int64_t r = a.epar[e1], c = a.epar[e2];
  const int64_t N = a.N;
  double2 *A = a.A;
  double2 t;
  t = A[r + c * a.lda];
  t.x += a.cJJ.re * sr - a.cJJ.im * si;
  t.y += a.cJJ.re * si + a.cJJ.im * sr;
  A[r + c * a.lda] = t;
  t = A[(r + N) + (c + N) * a.lda];
  t.x += a.cMM.re * sr - a.cMM.im * si;
  t.y += a.cMM.re * si + a.cMM.im * sr;
  A[(r + N) + (c + N) * a.lda] = t;
  t = A[(r + N) + c * a.lda];
  t.x += a.cMJ.re * kr - a.cMJ.im * ki;
  t.y += a.cMJ.re * ki + a.cMJ.im * kr;
  A[(r + N) + c * a.lda] = t;
  t = A[r + (c + N) * a.lda];
  t.x += a.cJM.re * kr - a.cJM.im * ki;
  t.y += a.cJM.re * ki + a.cJM.im * kr;
  A[r + (c + N) * a.lda] = t;
}

constexpr int kGatherDoms = 8;

struct GatherAllArgs {
  int N, ndom;
  const int *dmap;  // [ndom][N]: domain edge of each global edge, -1 if none
  const double2 *blk[kGatherDoms];
  const int *eh[kGatherDoms];
  int F[kGatherDoms];
  Cd Zsi[kGatherDoms];
  double2 *A;       // FP64 matrix, written (not accumulated)
  float2 *A32;      // FP32 copy, or null
  int64_t lda;
};

// Thread per global edge pair (g1 fastest): the four PMCHWT blocks summed
// over the domains in order (sysmat.f90:70-99, identity group), each domain's
// S and K from its face-pair blocks over the (+,-) halves of both edges;
// written once into A (and its FP32 copy), so the matrix needs no clearing,
// no read-modify-write per domain and no separate conversion.
__global__ void __launch_bounds__(256) gather_all_kernel(GatherAllArgs a) {
  const int g1 = blockIdx.x * blockDim.x + threadIdx.x;
  const int g2 = blockIdx.y;
  if (g1 >= a.N) return;
  double2 jj = make_double2(0, 0), mm = jj, mj = jj, jm = jj;
  for (int d = 0; d < a.ndom; d++) {
    const int e1 = a.dmap[(size_t)d * a.N + g1], e2 = a.dmap[(size_t)d * a.N + g2];
    if (e1 < 0 || e2 < 0) continue;
    const int *eh = a.eh[d];
    const int h1[2] = {eh[2 * e1], eh[2 * e1 + 1]};
    const int h2[2] = {eh[2 * e2], eh[2 * e2 + 1]};
    double sr = 0, si = 0, kr = 0, ki = 0;
#pragma unroll
    for (int i = 0; i < 2; i++) {
      if (h1[i] < 0) continue;
#pragma unroll
      for (int j = 0; j < 2; j++) {
        if (h2[j] < 0) continue;
        const int m = h1[i] / 3, p = h1[i] % 3, n = h2[j] / 3, q = h2[j] % 3;
        const double4 v =
            *reinterpret_cast<const double4 *>(a.blk[d] + ((size_t)n * a.F[d] + m) * 18 + 2 * (3 * p + q));
        sr += v.x;
        si += v.y;
        kr += v.z;
        ki += v.w;
      }
    }
    // the coefficients of the identity action: 1, Zsi, 1, -1
    const Cd z = a.Zsi[d];
    jj.x += 1.0 * sr - 0.0 * si;
    jj.y += 1.0 * si + 0.0 * sr;
    mm.x += z.re * sr - z.im * si;
    mm.y += z.re * si + z.im * sr;
    mj.x += 1.0 * kr - 0.0 * ki;
    mj.y += 1.0 * ki + 0.0 * kr;
    jm.x += -1.0 * kr - 0.0 * ki;
    jm.y += -1.0 * ki + 0.0 * kr;
  }
  const int64_t r = g1, c = g2, N = a.N, ld = a.lda;
  a.A[r + c * ld] = jj;
  a.A[(r + N) + (c + N) * ld] = mm;
  a.A[(r + N) + c * ld] = mj;
  a.A[r + (c + N) * ld] = jm;
  if (a.A32) {
    a.A32[r + c * ld] = make_float2((float)jj.x, (float)jj.y);
    a.A32[(r + N) + (c + N) * ld] = make_float2((float)mm.x, (float)mm.y);
    a.A32[(r + N) + c * ld] = make_float2((float)mj.x, (float)mj.y);
    a.A32[r + (c + N) * ld] = make_float2((float)jm.x, (float)jm.y);
  }
}

// The padding rows and columns 2N..n-1 of a matrix the gather writes
// without clearing: zero, with ones on the diagonal.  Thread per (row,
// padding index) of both strips.
template <class T>
__global__ void pad_strips_kernel(T *A, int64_t lda, int64_t n2, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t k = n2 + blockIdx.y;
  if (i >= n) return;
  T z{};
  A[i + k * lda] = z;  // column k
  A[k + i * lda] = z;  // row k
  if (i == k) {
    T one{};
    one.x = 1;
    A[k + k * lda] = one;
  }
}

// Rows/columns 2N..n-1 pad the matrix to a multiple of the panel width with
// an identity block, which leaves the LU of the leading 2N x 2N part as is.
__global__ void pad_identity(double2 *A, int64_t lda, int64_t n2, int64_t n) {
  const int64_t i = n2 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) A[i + i * lda] = make_double2(1.0, 0.0);
}

__global__ void convert_to_fp32(const double2 *__restrict__ A, float2 *__restrict__ B, int64_t count) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (; i < count; i += stride) {
    double2 v = A[i];
    B[i] = make_float2((float)v.x, (float)v.y);
  }
}

template <typename T, bool LOSSLESS>
int launch_pair_k(Ctx *c, int nq, dim3 grid, const PairArgs &a) {
  switch (nq) {
    case 1: pair_kernel<T, 1, LOSSLESS><<<grid, kPairThreads, 0, c->stream>>>(a); break;
    case 3: pair_kernel<T, 3, LOSSLESS><<<grid, kPairThreads, 0, c->stream>>>(a); break;
    case 4: pair_kernel<T, 4, LOSSLESS><<<grid, kPairThreads, 0, c->stream>>>(a); break;
    case 7: pair_kernel<T, 7, LOSSLESS><<<grid, kPairThreads, 0, c->stream>>>(a); break;
    case 13:
      // the FP64 kernel keeps 3 CTAs per SM (168 registers, no spills)
      if (sizeof(T) == sizeof(float) && c->pair_ctas == 4 && c->pair_e32)
        pair_kernel<T, 13, LOSSLESS, 4, true><<<grid, kPairThreads, 0, c->stream>>>(a);
      else if (sizeof(T) == sizeof(float) && c->pair_ctas == 4)
        pair_kernel<T, 13, LOSSLESS, 4><<<grid, kPairThreads, 0, c->stream>>>(a);
      else if (sizeof(T) == sizeof(float) && c->pair_e32)
        pair_kernel<T, 13, LOSSLESS, 3, true><<<grid, kPairThreads, 0, c->stream>>>(a);
      else
        pair_kernel<T, 13, LOSSLESS, 3><<<grid, kPairThreads, 0, c->stream>>>(a);
      break;
    default: return fail(c, MOM_ERR_ARG, "unsupported number of quadrature points");
  }
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  return MOM_OK;
}

// A lossless medium (real k) skips the decay factor e^{-Im(k) R}.
template <typename T>
int launch_pair(Ctx *c, int nq, dim3 grid, const PairArgs &a) {
  return a.ki == 0.0 ? launch_pair_k<T, true>(c, nq, grid, a) : launch_pair_k<T, false>(c, nq, grid, a);
}

}  // namespace


int upload_quadrature(Ctx *c) {
  MOM_CUDA(c, cudaMemcpyToSymbolAsync(c_qw, c->qw, sizeof(c->qw), 0, cudaMemcpyHostToDevice, c->stream));
  MOM_CUDA(c, cudaMemcpyToSymbolAsync(c_qn, c->qn, sizeof(c->qn), 0, cudaMemcpyHostToDevice, c->stream));
  return MOM_OK;
}

// Near pairs of one domain (sysmat.f90:233-260: |cp_m - J cp_n|^2 <
// (3 avelen)^2 with the domain's own average edge length, here as
// |J^T cp_m - cp_n| with the test centroids tcp already mapped) and their
// closed-form terms, from the test points tqabs and free vertices tbn (device,
// mapped likewise).  The list is wavelength independent, built once per
// geometry.
int near_setup(Ctx *c, DomDev &D, const double *tcp, const double *tqabs, const double *tbn, bool ident,
               int64_t *nnear, int **near_m, int **near_n, double **near_static) {
  const int F = D.F;
  const double thr = D.avelen * 3;
  // near_faces (sysmat.f90:233-260): |cp_m - cp_n| < 3 avelen.  The source
  // centroids are binned in cubes of side 3 avelen, so the partners of a test
  // face lie in the 27 cubes around its own; the pairs come out in the order
  // of the all-pairs loop (m, then n ascending) with the same distance test.
  std::vector<int> nm, nn;
  auto cell = [&](double v) { return (int64_t)std::floor(v / thr); };
  auto key = [](int64_t i, int64_t j, int64_t k) {
    return ((i & 0x1FFFFF) << 42) | ((j & 0x1FFFFF) << 21) | (k & 0x1FFFFF);
  };
  std::vector<std::pair<int64_t, int>> bins(F);
  for (int n = 0; n < F; n++) {
    const double *cn = &D.h_cp[3 * (size_t)n];
    bins[n] = {key(cell(cn[0]), cell(cn[1]), cell(cn[2])), n};
  }
  std::sort(bins.begin(), bins.end());
  std::vector<int> cand;
  for (int m = 0; m < F; m++) {
    const double *cm = tcp + 3 * (size_t)m;
    const int64_t ci = cell(cm[0]), cj = cell(cm[1]), ck = cell(cm[2]);
    cand.clear();
    for (int64_t a = -1; a <= 1; a++)
      for (int64_t b = -1; b <= 1; b++)
        for (int64_t e = -1; e <= 1; e++) {
          const int64_t k = key(ci + a, cj + b, ck + e);
          auto it = std::lower_bound(bins.begin(), bins.end(), std::make_pair(k, -1));
          for (; it != bins.end() && it->first == k; ++it) {
            const int n = it->second;
            const double *cn = &D.h_cp[3 * (size_t)n];
            const double d0 = cm[0] - cn[0], d1 = cm[1] - cn[1], d2 = cm[2] - cn[2];
            const double distsq = d0 * d0 + d1 * d1 + d2 * d2;
            if (distsq < thr * thr) cand.push_back(n);
          }
        }
    std::sort(cand.begin(), cand.end());
    for (int n : cand) {
      nm.push_back(m);
      nn.push_back(n);
    }
  }
  *nnear = (int64_t)nm.size();
  const size_t cap = (size_t)std::max<int64_t>(1, *nnear);
  MOM_CUDA(c, cudaMalloc(near_m, sizeof(int) * cap));
  MOM_CUDA(c, cudaMalloc(near_n, sizeof(int) * cap));
  MOM_CUDA(c, cudaMalloc(near_static, sizeof(double) * 54 * cap));
  if (*nnear == 0) return MOM_OK;
  MOM_CUDA(c, cudaMemcpyAsync(*near_m, nm.data(), sizeof(int) * *nnear, cudaMemcpyHostToDevice, c->stream));
  MOM_CUDA(c, cudaMemcpyAsync(*near_n, nn.data(), sizeof(int) * *nnear, cudaMemcpyHostToDevice, c->stream));
  std::vector<FaceGeo> geo(F);
  for (int f = 0; f < F; f++) {
    FaceGeo &g = geo[f];
    for (int k = 0; k < 3; k++)
      for (int i = 0; i < 3; i++) {
        g.v[k][i] = D.h_fv[9 * (size_t)f + 3 * k + i];
        g.s[k][i] = D.h_fs[9 * (size_t)f + 3 * k + i];
        g.mm[k][i] = D.h_fm[9 * (size_t)f + 3 * k + i];
      }
    for (int i = 0; i < 3; i++) g.n[i] = D.h_nrm[3 * (size_t)f + i];
  }
  FaceGeo *dgeo = nullptr;
  double *dbn = nullptr;
  MOM_CUDA(c, cudaMalloc(&dgeo, sizeof(FaceGeo) * F));
  MOM_CUDA(c, cudaMalloc(&dbn, sizeof(double) * 9 * F));
  MOM_CUDA(c, cudaMemcpyAsync(dgeo, geo.data(), sizeof(FaceGeo) * F, cudaMemcpyHostToDevice, c->stream));
  MOM_CUDA(c, cudaMemcpyAsync(dbn, D.h_bn.data(), sizeof(double) * 9 * F, cudaMemcpyHostToDevice, c->stream));
  StaticArgs a;
  a.nnear = *nnear;
  a.near_m = *near_m;
  a.near_n = *near_n;
  a.geo = dgeo;
  a.qabs = tqabs;
  a.area = D.area;
  a.sl = D.sl;
  a.bn = dbn;
  a.tbn = tbn ? tbn : dbn;
  a.ident = ident ? 1 : 0;
  a.out = *near_static;
  const unsigned blocks = (unsigned)((*nnear + 127) / 128);
  switch (c->nq) {
    case 1: near_static_kernel<1><<<blocks, 128, 0, c->stream>>>(a); break;
    case 3: near_static_kernel<3><<<blocks, 128, 0, c->stream>>>(a); break;
    case 4: near_static_kernel<4><<<blocks, 128, 0, c->stream>>>(a); break;
    case 7: near_static_kernel<7><<<blocks, 128, 0, c->stream>>>(a); break;
    case 13: near_static_kernel<13><<<blocks, 128, 0, c->stream>>>(a); break;
    default: return fail(c, MOM_ERR_ARG, "unsupported number of quadrature points");
  }
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  cudaFree(dgeo);
  cudaFree(dbn);
  return MOM_OK;
}

int near_precompute(Ctx *c, int d) {
  DomDev &D = c->dom[d];
  return near_setup(c, D, D.h_cp.data(), D.qabs, nullptr, true, &D.nnear, &D.near_m, &D.near_n, &D.near_static);
}

void free_actions(DomDev &D) {
  for (ActDev &A : D.act) {
    cudaFree(A.qrel);
    cudaFree(A.cp);
    cudaFree(A.mu);
    cudaFree(A.near_m);
    cudaFree(A.near_n);
    cudaFree(A.near_static);
    A = ActDev();
  }
  D.act.clear();
}

// Test faces of domain d mapped by J^T of group action g: points relative
// to the mapped centroid, mapped centroids and free vertices, their near
// pairs and closed-form terms.
int action_precompute(Ctx *c, int d, int g) {
  DomDev &D = c->dom[d];
  ActDev &A = D.act[g];
  const double *J = c->ga[g].j;
  auto jt = [&](const double *v, double *o) {
    for (int i = 0; i < 3; i++) o[i] = J[i] * v[0] + J[3 + i] * v[1] + J[6 + i] * v[2];
  };
  const int F = D.F, nq = c->nq;
  std::vector<double> qrel((size_t)F * nq * 3), qabs((size_t)F * nq * 3), cp(3 * (size_t)F), mu(9 * (size_t)F),
      bn(9 * (size_t)F);
  for (size_t i = 0; i < (size_t)F * nq; i++) {
    jt(&D.h_qrel[3 * i], &qrel[3 * i]);
    jt(&D.h_qabs[3 * i], &qabs[3 * i]);
  }
  for (size_t f = 0; f < (size_t)F; f++) {
    jt(&D.h_cp[3 * f], &cp[3 * f]);
    for (int e = 0; e < 3; e++) {
      jt(&D.h_mu[9 * f + 3 * e], &mu[9 * f + 3 * e]);
      jt(&D.h_bn[9 * f + 3 * e], &bn[9 * f + 3 * e]);
    }
  }
  double *dqabs = nullptr, *dbn = nullptr;
  auto up = [&](double **dst, const std::vector<double> &h) -> int {
    MOM_CUDA(c, cudaMalloc(dst, sizeof(double) * h.size()));
    MOM_CUDA(c, cudaMemcpyAsync(*dst, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, c->stream));
    return MOM_OK;
  };
  MOM_TRY(up(&A.qrel, qrel));
  MOM_TRY(up(&A.cp, cp));
  MOM_TRY(up(&A.mu, mu));
  MOM_TRY(up(&dqabs, qabs));
  MOM_TRY(up(&dbn, bn));
  const int rc = near_setup(c, D, cp.data(), dqabs, dbn, false, &A.nnear, &A.near_m, &A.near_n, &A.near_static);
  cudaStreamSynchronize(c->stream);
  cudaFree(dqabs);
  cudaFree(dbn);
  return rc;
}

// sysmat_pmchwt (sysmat.f90:18-105): A = 0, then for every domain and every
// admissible group action the face-pair blocks (far pairs in the requested
// precision, near pairs in FP64) are gathered into the four PMCHWT blocks of
// every representation (sysmat.f90:56-100; the identity group has one
// action and one representation).
int assemble_begin(Ctx *c) {
  const int64_t n = c->n, lda = c->lda;
  const size_t mat = (size_t)lda * n;
  const int nga = c->nga;
  MOM_CUDA(c, cudaMemsetAsync(c->A_all, 0, sizeof(double2) * mat * nga, c->stream));
  const int64_t n2 = 2 * (int64_t)c->N;
  if (n > n2)
    for (int r = 0; r < nga; r++) {
      pad_identity<<<(unsigned)((n - n2 + 127) / 128), 128, 0, c->stream>>>(c->A_all + r * mat, lda, n2, n);
      c->launches++;
    }
  return MOM_OK;
}

// Medium constants of domain d: k = ri omega / c0, c1 = -i omega mu0,
// c2 = -1/(i omega eps0 ri^2), Zsi = ri^2/eta0^2.
struct MediumConsts {
  double kr, ki;
  Cd c1, c2, Zsi;
};

MediumConsts medium_consts(double omega, const double *ri, int d) {
  const Cd rid = {ri[2 * d], ri[2 * d + 1]};
  MediumConsts m;
  m.kr = rid.re * omega / kC0;
  m.ki = rid.im * omega / kC0;
  m.c1 = {0.0, -omega * kMu0};
  const Cd ri2 = {rid.re * rid.re - rid.im * rid.im, 2 * rid.re * rid.im};
  const Cd den = {-omega * kEps0 * ri2.im, omega * kEps0 * ri2.re};  // i omega eps0 ri^2
  const double dn2 = den.re * den.re + den.im * den.im;
  m.c2 = {-den.re / dn2, den.im / dn2};
  m.Zsi = {ri2.re / (kEta0 * kEta0), ri2.im / (kEta0 * kEta0)};
  return m;
}

// The face-pair blocks of domain d under group action g (pair_kernel for
// every pair, then near_kernel over the near pairs) into blk.
int domain_blocks(Ctx *c, int d, int g, double omega, const double *ri, int precision, double2 *blk) {
  DomDev &D = c->dom[d];
  const MediumConsts mc = medium_consts(omega, ri, d);
  const double kr = mc.kr, ki = mc.ki;
  const Cd c1 = mc.c1, c2 = mc.c2;
  const double L0 = (precision == MOM_PREC_MIXED) ? D.avelen : 1.0;
  {
    {
      const bool ident = g == 0;
      const double *tqrel = ident ? D.qrel : D.act[g].qrel, *tcp = ident ? D.cp : D.act[g].cp,
                   *tmu = ident ? D.mu : D.act[g].mu;
      const int64_t nnear = ident ? D.nnear : D.act[g].nnear;
      PairArgs pa;
      pa.F = D.F;
      pa.qrel = D.qrel;
      pa.cp = D.cp;
      pa.mu = D.mu;
      pa.sl = D.sl;
      pa.tqrel = tqrel;
      pa.tcp = tcp;
      pa.tmu = tmu;
      pa.ident = ident ? 1 : 0;
      pa.sym = ident && c->pair_sym ? 1 : 0;
      pa.inv_unit = 1.0 / L0;
      pa.kr = kr * L0;
      pa.ki = ki * L0;
      pa.fD = {c1.re * L0 * L0 * L0 * kOofpi / 4.0, c1.im * L0 * L0 * L0 * kOofpi / 4.0};
      pa.fH = {c2.re * L0 * kOofpi, c2.im * L0 * kOofpi};
      pa.fK = L0 * L0 * kOofpi / 4.0;
      pa.blk = blk;
      dim3 grid((D.F + kPairThreads - 1) / kPairThreads, (D.F + kTestPerCta - 1) / kTestPerCta);
      {
        ProfScope ps(c, kProfPair);
        if (precision == MOM_PREC_MIXED) {
          MOM_TRY(launch_pair<float>(c, c->nq, grid, pa));
        } else {
          MOM_TRY(launch_pair<double>(c, c->nq, grid, pa));
        }
      }
      if (nnear > 0) {
        NearArgs na;
        na.nnear = nnear;
        na.F = D.F;
        na.near_m = ident ? D.near_m : D.act[g].near_m;
        na.near_n = ident ? D.near_n : D.act[g].near_n;
        na.qrel = D.qrel;
        na.cp = D.cp;
        na.mu = D.mu;
        na.sl = D.sl;
        na.tqrel = tqrel;
        na.tcp = tcp;
        na.tmu = tmu;
        na.ident = ident ? 1 : 0;
        na.stat = ident ? D.near_static : D.act[g].near_static;
        na.kr = kr;
        na.ki = ki;
        na.c1 = c1;
        na.c2 = c2;
        na.k2 = {kr * kr - ki * ki, 2 * kr * ki};
        na.blk = blk;
        const unsigned blocks = (unsigned)((nnear + 127) / 128);
        ProfScope ps(c, kProfNear);
        switch (c->nq) {
          case 1: near_kernel<1><<<blocks, 128, 0, c->stream>>>(na); break;
          case 3: near_kernel<3><<<blocks, 128, 0, c->stream>>>(na); break;
          case 4: near_kernel<4><<<blocks, 128, 0, c->stream>>>(na); break;
          case 7: near_kernel<7><<<blocks, 128, 0, c->stream>>>(na); break;
          case 13: near_kernel<13><<<blocks, 128, 0, c->stream>>>(na); break;
          default: return fail(c, MOM_ERR_ARG, "unsupported number of quadrature points");
        }
        c->launches++;
        MOM_CUDA(c, cudaGetLastError());
      }
    }
  }
  return MOM_OK;
}

int assemble_domain(Ctx *c, int d, double omega, const double *ri, int precision) {
  const int64_t n = c->n, lda = c->lda;
  const size_t mat = (size_t)lda * n;
  const int nga = c->nga;
  {
    DomDev &D = c->dom[d];
    const Cd Zsi = medium_consts(omega, ri, d).Zsi;
    for (int g = 0; g < nga; g++) {
      if (g > 0 && !D.act[g].admissible) continue;
      MOM_TRY(domain_blocks(c, d, g, omega, ri, precision, c->blk));
      const double detj = c->ga[g].detj;
      for (int r = 0; r < nga; r++) {
        const double e = c->ga[g].ef[r];
        GatherArgs ga;
        ga.F = D.F;
        ga.Nd = D.Nd;
        ga.N = c->N;
        ga.eh = D.eh;
        ga.epar = D.epar;
        ga.blk = c->blk;
        ga.cJJ = {e, 0.0};
        ga.cMM = {e * detj * Zsi.re, e * detj * Zsi.im};
        ga.cMJ = {e * detj, 0.0};
        ga.cJM = {-e, 0.0};
        ga.A = c->A_all + r * mat;
        ga.lda = lda;
        dim3 gg((D.Nd + 255) / 256, D.Nd);
        ProfScope ps(c, kProfGather);
        gather_kernel<<<gg, 256, 0, c->stream>>>(ga);
        c->launches++;
        MOM_CUDA(c, cudaGetLastError());
      }
    }
  }
  return MOM_OK;
}

int assemble_end(Ctx *c, int precision) {
  const size_t mat = (size_t)c->lda * c->n;
  const int nga = c->nga;
  for (int r = 0; r < nga && nga > 1; r++) MOM_TRY(apply_bc_matrix(c, r));
  if (precision == MOM_PREC_MIXED) {
    convert_to_fp32<<<c->nsm * 8, 256, 0, c->stream>>>(c->A_all, c->A32_all, (int64_t)mat * nga);
    c->launches++;
    MOM_CUDA(c, cudaGetLastError());
  }
  c->assembled = 1;
  c->factored = -1;
  return MOM_OK;
}

// The identity-group assembly when every domain's face-pair blocks fit at
// once: pair and near kernels per domain into its own block buffer, then one
// gather over the global edge pairs that writes A (and A32) once.
int assemble_fused(Ctx *c, double omega, const double *ri, int precision) {
  GatherAllArgs ga;
  ga.N = c->N;
  ga.ndom = c->ndom;
  ga.dmap = c->dmap;
  for (int d = 0; d < c->ndom; d++) {
    double2 *blk = c->blk + c->blk_off[d];
    MOM_TRY(domain_blocks(c, d, 0, omega, ri, precision, blk));
    ga.blk[d] = blk;
    ga.eh[d] = c->dom[d].eh;
    ga.F[d] = c->dom[d].F;
    ga.Zsi[d] = medium_consts(omega, ri, d).Zsi;
  }
  ga.A = c->A_all;
  ga.A32 = precision == MOM_PREC_MIXED ? c->A32_all : nullptr;
  ga.lda = c->lda;
  {
    ProfScope ps(c, kProfGather);
    gather_all_kernel<<<dim3((c->N + 255) / 256, c->N), 256, 0, c->stream>>>(ga);
    c->launches++;
    MOM_CUDA(c, cudaGetLastError());
  }
  const int64_t n = c->n, n2 = 2 * (int64_t)c->N;
  if (n > n2) {
    const dim3 pg((unsigned)((n + 255) / 256), (unsigned)(n - n2));
    pad_strips_kernel<double2><<<pg, 256, 0, c->stream>>>(c->A_all, c->lda, n2, n);
    c->launches++;
    if (ga.A32) {
      pad_strips_kernel<float2><<<pg, 256, 0, c->stream>>>(c->A32_all, c->lda, n2, n);
      c->launches++;
    }
    MOM_CUDA(c, cudaGetLastError());
  }
  c->assembled = 1;
  c->factored = -1;
  return MOM_OK;
}

int assemble(Ctx *c, double omega, const double *ri, int precision) {
  if (c->blk_fused && c->nga == 1 && c->ndom <= kGatherDoms) return assemble_fused(c, omega, ri, precision);
  MOM_TRY(assemble_begin(c));
  for (int d = 0; d < c->ndom; d++) MOM_TRY(assemble_domain(c, d, omega, ri, precision));
  return assemble_end(c, precision);
}

// A caller's 2N x 2N matrix (host, column-major, lda) in place of an
// assembled one: the same padding and FP32 copy as assemble().
int load_matrix(Ctx *c, const double *A_host, int64_t ldh, int precision) {
  const int64_t n = c->n, lda = c->lda, n2 = 2 * (int64_t)c->N;
  MOM_CUDA(c, cudaMemsetAsync(c->A, 0, sizeof(double2) * (size_t)lda * n, c->stream));
  MOM_CUDA(c, cudaMemcpy2DAsync(c->A, sizeof(double2) * lda, A_host, sizeof(double2) * ldh, sizeof(double2) * n2, n2,
                                cudaMemcpyHostToDevice, c->stream));
  if (n > n2) {
    pad_identity<<<(unsigned)((n - n2 + 127) / 128), 128, 0, c->stream>>>(c->A, lda, n2, n);
    c->launches++;
  }
  if (precision == MOM_PREC_MIXED) {
    convert_to_fp32<<<c->nsm * 8, 256, 0, c->stream>>>(c->A, c->A32, (int64_t)lda * n);
    c->launches++;
  }
  MOM_CUDA(c, cudaGetLastError());
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  c->assembled = 1;
  c->factored = -1;
  return MOM_OK;
}

#include "adjoint_impl.cuh"
#include "nfields_impl.cuh"

namespace {

template <typename V>
int upload_vec(Ctx *c, V **dst, const std::vector<V> &src) {
  MOM_CUDA(c, cudaMalloc(dst, sizeof(V) * std::max<size_t>(1, src.size())));
  if (!src.empty())
    MOM_CUDA(c, cudaMemcpyAsync(*dst, src.data(), sizeof(V) * src.size(), cudaMemcpyHostToDevice, c->stream));
  return MOM_OK;
}

// Topology of domain d for the geometry derivatives: nodes, face and edge
// node indices, the near-pair bitmap and the (vertex, face) incidences.
int adjoint_setup(Ctx *c, int d) {
  DomDev &D = c->dom[d];
  if (D.adj_ready) return MOM_OK;
  const int F = D.F;
  MOM_TRY(upload_vec(c, &D.nodes, D.h_nodes));
  MOM_TRY(upload_vec(c, &D.fsign, D.h_fsign));
  MOM_TRY(upload_vec(c, &D.fnode, D.h_fnode));
  MOM_TRY(upload_vec(c, &D.fea, D.h_fea));
  MOM_TRY(upload_vec(c, &D.feb, D.h_feb));
  MOM_TRY(upload_vec(c, &D.fbn, D.h_fbn));
  const size_t words = ((size_t)F * F + 31) / 32;
  MOM_CUDA(c, cudaMalloc(&D.near_bits, sizeof(unsigned) * words));
  MOM_CUDA(c, cudaMemsetAsync(D.near_bits, 0, sizeof(unsigned) * words, c->stream));
  if (D.nnear > 0) {
    near_bits_kernel<<<(unsigned)((D.nnear + 255) / 256), 256, 0, c->stream>>>(D.nnear, F, D.near_m, D.near_n,
                                                                                D.near_bits);
    c->launches++;
    MOM_CUDA(c, cudaGetLastError());
  }
  std::vector<int> inode, iface;
  std::vector<std::vector<int>> byn(D.nnodes);
  for (int f = 0; f < F; f++)
    for (int k = 0; k < 3; k++) byn[D.h_fnode[3 * (size_t)f + k]].push_back(f);
  for (int v = 0; v < D.nnodes; v++)
    for (int f : byn[v]) {
      inode.push_back(v);
      iface.push_back(f);
    }
  D.ninc = (int)inode.size();
  MOM_TRY(upload_vec(c, &D.inc_node, inode));
  MOM_TRY(upload_vec(c, &D.inc_face, iface));
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  D.adj_ready = true;
  return MOM_OK;
}

AdjTopo topo_of(const Ctx *c, const DomDev &D) {
  AdjTopo t;
  t.F = D.F;
  t.N = c->N;
  t.nodes = D.nodes;
  t.fnode = D.fnode;
  t.fea = D.fea;
  t.feb = D.feb;
  t.fbn = D.fbn;
  t.fsign = D.fsign;
  t.hpar = D.hpar;
  t.near_bits = D.near_bits;
  return t;
}

Cd cdiv(Cd a, Cd b) {
  const double d = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
Cd cmulh(Cd a, Cd b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

// Medium constants of domain d (sysmat.f90:40-60) as dual numbers, with the
// derivative along Re(eps) when seed is set.
void medium_duals(double omega, const double *ri, int d, bool seed, AdjPairArgs &a) {
  const Cd n = {ri[2 * d], ri[2 * d + 1]};
  const double k0 = omega / kC0;
  const Cd eps = cmulh(n, n);
  const Cd dk = seed ? cdiv({k0, 0.0}, {2.0 * n.re, 2.0 * n.im}) : Cd{0.0, 0.0};  // dk/deps = k0 / (2 n)
  a.kr = Dual(n.re * k0, dk.re);
  a.ki = Dual(n.im * k0, dk.im);
  a.c1 = {Dual(0.0), Dual(-omega * kMu0)};
  const Cd den = {-omega * kEps0 * eps.im, omega * kEps0 * eps.re};  // i omega eps0 eps
  const Cd c2 = cdiv({-1.0, 0.0}, den);
  const Cd dc2 = seed ? cdiv({-c2.re, -c2.im}, eps) : Cd{0.0, 0.0};  // dc2/deps = -c2 / eps
  a.c2 = {Dual(c2.re, dc2.re), Dual(c2.im, dc2.im)};
  const double ie2 = 1.0 / (kEta0 * kEta0);
  a.Zsi = {Dual(eps.re * ie2, seed ? ie2 : 0.0), Dual(eps.im * ie2, 0.0)};
}

int adj_launch_pair(Ctx *c, const dim3 &grid, const AdjPairArgs &a) {
  switch (c->nq) {
    case 1: launch_adj_pair<1>(grid, c->stream, a); break;
    case 3: launch_adj_pair<3>(grid, c->stream, a); break;
    case 4: launch_adj_pair<4>(grid, c->stream, a); break;
    case 7: launch_adj_pair<7>(grid, c->stream, a); break;
    case 13: launch_adj_pair<13>(grid, c->stream, a); break;
    default: return fail(c, MOM_ERR_ARG, "unsupported number of quadrature points");
  }
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  return MOM_OK;
}

}  // namespace

int adjoint_eps(Ctx *c, double omega, const double *ri, int d, int R, const double2 *lam, const double2 *xv,
                const double2 *W, double *out) {
  if (R < 0 || R > kAdjMaxObj) return fail(c, MOM_ERR_ARG, "too many adjoint objectives");
  MOM_TRY(adjoint_setup(c, d));
  DomDev &D = c->dom[d];
  AdjPairArgs a;
  a.t = topo_of(c, D);
  a.n = c->n;
  medium_duals(omega, ri, d, true, a);
  a.mode = 0;
  a.inc_node = a.inc_face = nullptr;
  a.qrel = D.qrel;
  a.cp = D.cp;
  a.mu = D.mu;
  a.sl = D.sl;
  a.R = R;
  a.lam = lam;
  a.xv = xv;
  a.W = W;
  const int nobj = R == 0 ? 1 : R;
  const dim3 grid((D.F + kAdjThreads - 1) / kAdjThreads, D.F);
  const size_t nvals = (size_t)grid.x * grid.y * nobj * 2;
  MOM_TRY(ensure_buffer(c, &c->adj_part, &c->adj_part_bytes, sizeof(double) * nvals));
  a.part = (double *)c->adj_part;
  if (c->adj_eps_plain) {
    // the same sums with FP64 geometry and dual numbers only where k enters
    MOM_TRY(nfield_geometry(c, D));
    AdjEpsArgs e;
    e.F = D.F;
    e.n = c->n;
    e.N = c->N;
    e.qrel = D.qrel;
    e.qabs = D.qabs;
    e.cp = D.cp;
    e.area = D.area;
    e.mu = D.mu;
    e.sl = D.sl;
    e.bn = D.nf_bn;
    e.geo = reinterpret_cast<const FaceGeo *>(D.nf_geo);
    e.hpar = D.hpar;
    e.near_bits = D.near_bits;
    e.kr = a.kr;
    e.ki = a.ki;
    e.c1 = a.c1;
    e.c2 = a.c2;
    e.Zsi = a.Zsi;
    e.R = R;
    e.lam = lam;
    e.xv = xv;
    e.W = W;
    e.part = a.part;
    switch (c->nq) {
      case 1: launch_adj_eps<1>(grid, c->stream, e); break;
      case 3: launch_adj_eps<3>(grid, c->stream, e); break;
      case 4: launch_adj_eps<4>(grid, c->stream, e); break;
      case 7: launch_adj_eps<7>(grid, c->stream, e); break;
      case 13: launch_adj_eps<13>(grid, c->stream, e); break;
      default: return fail(c, MOM_ERR_ARG, "unsupported number of quadrature points");
    }
    c->launches++;
    MOM_CUDA(c, cudaGetLastError());
  } else {
    MOM_TRY(adj_launch_pair(c, grid, a));
  }
  std::vector<double> h(nvals);
  MOM_CUDA(c, cudaMemcpyAsync(h.data(), a.part, sizeof(double) * nvals, cudaMemcpyDeviceToHost, c->stream));
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  for (int o = 0; o < nobj; o++) {
    double re = 0, im = 0;
    for (size_t b = 0; b < (size_t)grid.x * grid.y; b++) {
      re += h[(b * nobj + o) * 2];
      im += h[(b * nobj + o) * 2 + 1];
    }
    out[2 * o] = re;
    out[2 * o + 1] = im;
  }
  return MOM_OK;
}

int adjoint_nodes(Ctx *c, double omega, const double *ri, int R, const double2 *lam, const double2 *xv,
                  const int *obj_src, const int *obj_kind, int nsrc, const mom_src *src, double *out) {
  if (R < 1 || R > kAdjMaxObj) return fail(c, MOM_ERR_ARG, "1 to 8 adjoint objectives");
  int total = 0;
  std::vector<int> off(c->ndom);
  for (int d = 0; d < c->ndom; d++) {
    off[d] = total;
    total += c->dom[d].nnodes;
  }
  std::fill(out, out + (size_t)R * total * 3, 0.0);
  // - Re(lambda^T dA x) of every domain's blocks
  for (int d = 0; d < c->ndom; d++) {
    MOM_TRY(adjoint_setup(c, d));
    DomDev &D = c->dom[d];
    if (D.ninc == 0) continue;
    AdjPairArgs a;
    a.t = topo_of(c, D);
    a.n = c->n;
    medium_duals(omega, ri, d, false, a);
    a.mode = 1;
    a.inc_node = D.inc_node;
    a.inc_face = D.inc_face;
    a.R = R;
    a.lam = lam;
    a.xv = xv;
    a.W = nullptr;
    a.qrel = D.qrel;
    a.cp = D.cp;
    a.mu = D.mu;
    a.sl = D.sl;
    const dim3 grid((D.F + kAdjThreads - 1) / kAdjThreads, 3 * D.ninc);
    const size_t nvals = (size_t)grid.x * grid.y * R * 2;
    MOM_TRY(ensure_buffer(c, &c->adj_part, &c->adj_part_bytes, sizeof(double) * nvals));
    a.part = (double *)c->adj_part;
    if (c->adj_vertex_plain) {
      switch (c->nq) {
        case 1: launch_adj_vertex<1>(grid, c->stream, a); break;
        case 3: launch_adj_vertex<3>(grid, c->stream, a); break;
        case 4: launch_adj_vertex<4>(grid, c->stream, a); break;
        case 7: launch_adj_vertex<7>(grid, c->stream, a); break;
        case 13: launch_adj_vertex<13>(grid, c->stream, a); break;
        default: return fail(c, MOM_ERR_ARG, "unsupported number of quadrature points");
      }
      c->launches++;
      MOM_CUDA(c, cudaGetLastError());
    } else {
      MOM_TRY(adj_launch_pair(c, grid, a));
    }
    std::vector<double> h(nvals);
    std::vector<int> inode(D.ninc);
    MOM_CUDA(c, cudaMemcpyAsync(h.data(), a.part, sizeof(double) * nvals, cudaMemcpyDeviceToHost, c->stream));
    MOM_CUDA(c, cudaMemcpyAsync(inode.data(), D.inc_node, sizeof(int) * D.ninc, cudaMemcpyDeviceToHost, c->stream));
    MOM_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int item = 0; item < 3 * D.ninc; item++) {
      const int v = inode[item / 3], k = item % 3;
      for (int o = 0; o < R; o++) {
        double re = 0;
        for (unsigned b = 0; b < grid.x; b++) re += h[(((size_t)item * grid.x + b) * R + o) * 2];
        out[((size_t)o * total + off[d] + v) * 3 + k] -= re;
      }
    }
  }
  // Re(lambda^T dq) and the explicit term of sigma on the exterior surface
  {
    MOM_TRY(adjoint_setup(c, 0));
    DomDev &D = c->dom[0];
    std::vector<AdjSrc> hs(nsrc);
    for (int s = 0; s < nsrc; s++) {
      if (src[s].type != MOM_SRC_PW && src[s].type != MOM_SRC_PW_ELLIPTIC)
        return fail(c, MOM_ERR_ARG, "unsupported source type (only pw and pw_elliptic)");
      src_geometry(src[s], hs[s].dir, hs[s].pol);
      hs[s].ph_re = src[s].phase_re;
      hs[s].ph_im = src[s].phase_im;
      hs[s].type = src[s].type;
    }
    const size_t items = 3 * (size_t)D.ninc;
    const size_t b_src = ((sizeof(AdjSrc) * nsrc + 255) / 256) * 256, b_obj = 512,
                 b_out = sizeof(double) * items * R;
    MOM_TRY(ensure_buffer(c, &c->adj_part, &c->adj_part_bytes, b_src + 2 * b_obj + b_out));
    char *base = (char *)c->adj_part;
    AdjFaceArgs f;
    f.t = topo_of(c, D);
    f.n = c->n;
    f.ninc = D.ninc;
    f.inc_node = D.inc_node;
    f.inc_face = D.inc_face;
    f.R = R;
    f.src = (const AdjSrc *)base;
    f.obj_src = (const int *)(base + b_src);
    f.obj_kind = (const int *)(base + b_src + b_obj);
    f.lam = lam;
    f.xv = xv;
    f.k = {ri[0] * omega / kC0, ri[1] * omega / kC0};
    f.omega = omega;
    f.cc = 2.0 / (kEps0 * kC0 * ri[0]);  // cs.f90:38
    f.out = (double *)(base + b_src + 2 * b_obj);
    MOM_CUDA(c, cudaMemcpyAsync((void *)f.src, hs.data(), sizeof(AdjSrc) * nsrc, cudaMemcpyHostToDevice, c->stream));
    MOM_CUDA(c, cudaMemcpyAsync((void *)f.obj_src, obj_src, sizeof(int) * R, cudaMemcpyHostToDevice, c->stream));
    MOM_CUDA(c, cudaMemcpyAsync((void *)f.obj_kind, obj_kind, sizeof(int) * R, cudaMemcpyHostToDevice, c->stream));
    const int blocks = (int)((items + 63) / 64);
    switch (c->nq) {
      case 1: launch_adj_face<1>(blocks, c->stream, f); break;
      case 3: launch_adj_face<3>(blocks, c->stream, f); break;
      case 4: launch_adj_face<4>(blocks, c->stream, f); break;
      case 7: launch_adj_face<7>(blocks, c->stream, f); break;
      case 13: launch_adj_face<13>(blocks, c->stream, f); break;
      default: return fail(c, MOM_ERR_ARG, "unsupported number of quadrature points");
    }
    c->launches++;
    MOM_CUDA(c, cudaGetLastError());
    std::vector<double> h(items * R);
    std::vector<int> inode(D.ninc);
    MOM_CUDA(c, cudaMemcpyAsync(h.data(), f.out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream));
    MOM_CUDA(c, cudaMemcpyAsync(inode.data(), D.inc_node, sizeof(int) * D.ninc, cudaMemcpyDeviceToHost, c->stream));
    MOM_CUDA(c, cudaStreamSynchronize(c->stream));
    for (size_t item = 0; item < items; item++) {
      const int v = inode[item / 3], k = (int)(item % 3);
      for (int o = 0; o < R; o++) out[((size_t)o * total + off[0] + v) * 3 + k] += h[item * R + o];
    }
  }
  return MOM_OK;
}

}  // namespace mom
