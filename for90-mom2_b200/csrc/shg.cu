// Second-harmonic generation from centrosymmetric surface nonlinearities on
// sm_100a (FP64): the nonlinear branch of solve_batch (solver.f90:143-217)
// for the identity symmetry group.
//
//   nls_face_kernel    efield, Pnls_invmap and the first loop of nlsurf_coef
//                      (nlsurf.f90:22-51, 76-103, 181-217): per face and
//                      source, the surface polarisation of the fundamental
//                      field at the quadrature points and its three moments
//                      per local edge;
//   nls_edge_kernel    per domain edge: the moments of its two faces summed,
//                      src_vec (E0, H0) into the right-hand side and the
//                      right-hand sides of the Gram systems;
//   gram_*_kernel      rwg_moments (rwgf.f90:148-221) as a 5-entry ELL matrix;
//   gram_cg_kernel     the Gram systems <f_m, f_n> c = b (the reference's
//                      dense LU, solve_multi_linsys) by Jacobi-preconditioned
//                      conjugate gradients: the matrix is real, symmetric,
//                      positive definite and sparse (an edge couples to the
//                      four other edges of its two faces), so each real and
//                      imaginary part is one CG on one CTA;
//   nls_cm_kernel      the expansion method's <f_m, n x sum_p coef_p f_p>
//                      (nlsurf.f90:276-300);
//   nls_scatter_kernel the source coefficients (cJ, cM) on the global unknowns;
// then sysmat_pmchwt_nls (sysmat.f90:112-229): the matrix at 2 omega with the
// second-harmonic indices, the domains' own blocks applied to their source
// coefficients (nlx -= A_d c_d) while the matrix is being accumulated, and
// the solve.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <set>
#include <vector>

#include "mom_internal.h"

namespace mom {

namespace {

struct Z {
  double re, im;
};
__device__ __forceinline__ Z zmul(Z a, Z b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ Z zadd(Z a, Z b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ Z zsub(Z a, Z b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ Z zrs(Z a, double s) { return {a.re * s, a.im * s}; }
__device__ __forceinline__ Z zdiv(Z a, Z b) {
  const double d = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}

constexpr int kEll = 5;        // Gram matrix entries per row: the diagonal, then up to four neighbours
constexpr int kCgThreads = 1024;

// RWG function of local edge q of a face (rwg, rwgf.f90:13-32):
// sign * L / (2 A) * (r - free vertex).
__device__ __forceinline__ void rwg_at(const double *r, const double *bn, double slq, double A, double *f) {
  const double s = slq / (2.0 * A);
  for (int i = 0; i < 3; i++) f[i] = s * (r[i] - bn[i]);
}

// The symmetry group as kernel argument (point actions J row-major, det J,
// field actions ef[g][r]: real for the mirror groups).
struct ShgGroup {
  int nga;
  double j[kMaxGroup][9];
  double detj[kMaxGroup];
  double ef[kMaxGroup][kMaxGroup];
};

struct FaceArgs {
  double w[kMaxQ];
  int F, nq, N, nsrc;
  int64_t ldx, xrep;    // solutions: source s, representation m at X + m xrep + s ldx
  const double *qabs, *area, *nrm, *sl, *bn;
  const int *hpar;
  const double2 *X;     // fundamental solutions
  const double2 *epsp;  // [F] selvedge permittivity
  Z iwe;                // i omega eps of the medium at the fundamental
  Z chi_nnn, chi_ntt, chi_ttn;
  ShgGroup G;
  double2 *half;        // [nga][nsrc][F][3][3]: int1 A / epsp, int3 A, int2 A
};

// efield (nlsurf.f90:22-51) of solution x on face f at a point: n x M + n
// div J / (i omega eps), with the RWG values fq at the point.
__device__ __forceinline__ void face_efield(const FaceArgs &a, const double2 *x, int f, const double *nor,
                                            const double slq[3], double A, const double fq[3][3], Z *e) {
  Z divj = {0, 0}, ms[3] = {{0, 0}, {0, 0}, {0, 0}};
  for (int q = 0; q < 3; q++) {
    const int g = a.hpar[3 * f + q];
    const Z xj = {x[g].x, x[g].y}, xm = {x[a.N + g].x, x[a.N + g].y};
    divj = zadd(divj, zrs(xj, slq[q] / A));
    for (int i = 0; i < 3; i++) ms[i] = zadd(ms[i], zrs(xm, fq[q][i]));
  }
  const Z en0 = zdiv(divj, a.iwe);
  e[0] = zadd(zsub(zrs(ms[2], nor[1]), zrs(ms[1], nor[2])), zrs(en0, nor[0]));
  e[1] = zadd(zsub(zrs(ms[0], nor[2]), zrs(ms[2], nor[0])), zrs(en0, nor[1]));
  e[2] = zadd(zsub(zrs(ms[1], nor[0]), zrs(ms[0], nor[1])), zrs(en0, nor[2]));
}

// Pnls_invmap's polarisation (nlsurf.f90:76-103) of the field e with the
// normal nn: eps0 (chi_nnn En^2 + chi_ntt Et.Et) nn + 2 eps0 chi_ttn Et En.
__device__ __forceinline__ void surface_polarisation(const FaceArgs &a, const Z *e, const double *nn, Z *P) {
  Z en = {0, 0};
  for (int i = 0; i < 3; i++) en = zadd(en, zrs(e[i], nn[i]));
  Z et[3];
  for (int i = 0; i < 3; i++) et[i] = zsub(e[i], zrs(en, nn[i]));
  Z ett = {0, 0};
  for (int i = 0; i < 3; i++) ett = zadd(ett, zmul(et[i], et[i]));
  const Z pn = zrs(zadd(zmul(a.chi_nnn, zmul(en, en)), zmul(a.chi_ntt, ett)), kEps0);
  const Z ttn = zrs(a.chi_ttn, 2.0 * kEps0);
  for (int i = 0; i < 3; i++) P[i] = zadd(zmul(zmul(ttn, et[i]), en), zrs(pn, nn[i]));
}

// Thread per (face, source, representation nf): the polarisation of
// representation nf (Pnls_frag, nlsurf.f90:106-125: for every element n the
// field of the image point, sum_m ef_n(m) J_n^T E_m, with the normal
// J_n^T n, and the sum over n of ef_n(nf) J_n P_n / nga; for the identity
// group simply P(E)) and its three moments per local edge.
__global__ void nls_face_kernel(FaceArgs a) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y, nf = blockIdx.z;
  if (f >= a.F) return;
  const int nga = a.G.nga;
  const double A = a.area[f];
  const double nor[3] = {a.nrm[3 * f], a.nrm[3 * f + 1], a.nrm[3 * f + 2]};
  double slq[3];
  for (int q = 0; q < 3; q++) slq[q] = a.sl[3 * f + q];
  Z i1[3] = {{0, 0}, {0, 0}, {0, 0}}, i2[3] = {{0, 0}, {0, 0}, {0, 0}}, i3[3] = {{0, 0}, {0, 0}, {0, 0}};
  for (int r = 0; r < a.nq; r++) {
    const double *pt = a.qabs + ((size_t)f * a.nq + r) * 3;
    double fq[3][3];
    for (int q = 0; q < 3; q++) rwg_at(pt, a.bn + 9 * (size_t)f + 3 * q, slq[q], A, fq[q]);
    Z P[3];
    if (nga == 1) {
      Z e[3];
      face_efield(a, a.X + (size_t)s * a.ldx, f, nor, slq, A, fq, e);
      surface_polarisation(a, e, nor, P);
    } else {
      Z Em[kMaxGroup][3];
      for (int m = 0; m < nga; m++) face_efield(a, a.X + (size_t)m * a.xrep + (size_t)s * a.ldx, f, nor, slq, A, fq, Em[m]);
      for (int i = 0; i < 3; i++) P[i] = {0, 0};
      for (int n = 0; n < nga; n++) {
        const double *J = a.G.j[n];
        Z e[3] = {{0, 0}, {0, 0}, {0, 0}};
        for (int m = 0; m < nga; m++) {
          const double c = a.G.ef[n][m];  // conj of a real character
          for (int i = 0; i < 3; i++)  // (J^T E)_i = sum_k J[k][i] E_k
            e[i] = zadd(e[i], zrs(zadd(zadd(zrs(Em[m][0], J[i]), zrs(Em[m][1], J[3 + i])), zrs(Em[m][2], J[6 + i])), c));
        }
        double nn[3];
        for (int i = 0; i < 3; i++) nn[i] = J[i] * nor[0] + J[3 + i] * nor[1] + J[6 + i] * nor[2];
        Z Pn_[3];
        surface_polarisation(a, e, nn, Pn_);
        const double c = a.G.ef[n][nf];
        for (int i = 0; i < 3; i++)  // J P
          P[i] = zadd(P[i], zrs(zadd(zadd(zrs(Pn_[0], J[3 * i]), zrs(Pn_[1], J[3 * i + 1])), zrs(Pn_[2], J[3 * i + 2])), c));
      }
      for (int i = 0; i < 3; i++) P[i] = zrs(P[i], 1.0 / nga);
    }
    // nlsurf_coef: Pn = n . P, Pt = P - Pn n
    Z Pn = {0, 0};
    for (int i = 0; i < 3; i++) Pn = zadd(Pn, zrs(P[i], nor[i]));
    Z Pt[3];
    for (int i = 0; i < 3; i++) Pt[i] = zsub(P[i], zrs(Pn, nor[i]));
    // Pt x n
    Z ptn[3];
    ptn[0] = zsub(zrs(Pt[1], nor[2]), zrs(Pt[2], nor[1]));
    ptn[1] = zsub(zrs(Pt[2], nor[0]), zrs(Pt[0], nor[2]));
    ptn[2] = zsub(zrs(Pt[0], nor[1]), zrs(Pt[1], nor[0]));
    const double wr = a.w[r];
    for (int q = 0; q < 3; q++) {
      const double div = slq[q] / A;
      i1[q] = zsub(i1[q], zrs(Pn, wr * div));
      Z d2 = {0, 0}, d3 = {0, 0};
      for (int i = 0; i < 3; i++) {
        d2 = zadd(d2, zrs(ptn[i], fq[q][i]));
        d3 = zadd(d3, zrs(Pt[i], fq[q][i]));
      }
      i2[q] = zadd(i2[q], zrs(d2, wr));
      i3[q] = zadd(i3[q], zrs(d3, wr));
    }
  }
  const Z ep = {a.epsp[f].x, a.epsp[f].y};
  double2 *o = a.half + (((size_t)nf * a.nsrc + s) * a.F + f) * 9;
  for (int q = 0; q < 3; q++) {
    const Z c = zdiv(zrs(i1[q], A), ep);
    o[3 * q] = make_double2(c.re, c.im);
    o[3 * q + 1] = make_double2(i3[q].re * A, i3[q].im * A);
    o[3 * q + 2] = make_double2(i2[q].re * A, i2[q].im * A);
  }
}

struct EdgeArgs {
  int F, Nd, N;
  int64_t ldb;
  const int *eh, *epar;
  const double2 *half;  // [nsrc][F][3][3]
  double omega_sh;
  double2 *B;           // second-harmonic right-hand sides [nsrc][ldb]
  double *rhs;          // [nsrc][4][Nd]: coef re, im; J-coefficient right-hand side re, im
};

// Thread per (domain edge, source): the sums over the edge's two faces and
// the closing scalings of the first loop of nlsurf_coef (nlsurf.f90:219-225).
__global__ void nls_edge_kernel(EdgeArgs a) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (e >= a.Nd) return;
  Z coef = {0, 0}, cj = {0, 0}, hv = {0, 0};
  for (int k = 0; k < 2; k++) {
    const int h = a.eh[2 * e + k];
    if (h < 0) continue;
    const double2 *o = a.half + ((size_t)s * a.F + h / 3) * 9 + 3 * (h % 3);
    coef = zadd(coef, {o[0].x, o[0].y});
    cj = zadd(cj, {o[1].x, o[1].y});
    hv = zadd(hv, {o[2].x, o[2].y});
  }
  // src_coef(J) = -src_coef * i * omega_sh; src_vec = (coef / 2, i omega_sh H / 2)
  const Z cjr = zrs(Z{cj.im, -cj.re}, a.omega_sh);
  const double h2 = 0.5 * a.omega_sh;
  double2 *b = a.B + (size_t)s * a.ldb;
  const int g = a.epar[e];
  b[g].x += 0.5 * coef.re;
  b[g].y += 0.5 * coef.im;
  b[a.N + g].x += -h2 * hv.im;
  b[a.N + g].y += h2 * hv.re;
  double *r = a.rhs + (size_t)s * 4 * a.Nd;
  r[e] = coef.re;
  r[a.Nd + e] = coef.im;
  r[2 * a.Nd + e] = cjr.re;
  r[3 * a.Nd + e] = cjr.im;
}

struct GramArgs {
  double w[kMaxQ];
  int F, Nd, nq;
  const double *qabs, *area, *sl, *bn;
  const int *eh, *fedge;
  double *G;      // [F][3][3]
  int *col;       // [Nd][kEll]
  double *val;    // [Nd][kEll]
};

// Thread per face: A sum_r w_r f_q(r) . f_p(r) for the face's nine pairs.
__global__ void gram_face_kernel(GramArgs a) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= a.F) return;
  const double A = a.area[f];
  double acc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int r = 0; r < a.nq; r++) {
    const double *pt = a.qabs + ((size_t)f * a.nq + r) * 3;
    double fq[3][3];
    for (int q = 0; q < 3; q++) rwg_at(pt, a.bn + 9 * (size_t)f + 3 * q, a.sl[3 * f + q], A, fq[q]);
    for (int q = 0; q < 3; q++)
      for (int p = 0; p < 3; p++)
        acc[q][p] += a.w[r] * (fq[q][0] * fq[p][0] + fq[q][1] * fq[p][1] + fq[q][2] * fq[p][2]);
  }
  for (int q = 0; q < 3; q++)
    for (int p = 0; p < 3; p++) a.G[9 * (size_t)f + 3 * q + p] = acc[q][p] * A;
}

// Thread per domain edge: its row (the diagonal over both faces, then the
// other two edges of each face).
__global__ void gram_ell_kernel(GramArgs a) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.Nd) return;
  int *col = a.col + (size_t)e * kEll;
  double *val = a.val + (size_t)e * kEll;
  for (int k = 0; k < kEll; k++) {
    col[k] = e;
    val[k] = 0;
  }
  double diag = 0;
  int k = 1;
  for (int side = 0; side < 2; side++) {
    const int h = a.eh[2 * e + side];
    if (h < 0) continue;
    const int f = h / 3, q = h % 3;
    diag += a.G[9 * (size_t)f + 4 * q];
    for (int p = 0; p < 3; p++) {
      if (p == q) continue;
      col[k] = a.fedge[3 * f + p];
      val[k] = a.G[9 * (size_t)f + 3 * q + p];
      k++;
    }
  }
  val[0] = diag;
}

struct CgArgs {
  int Nd, maxit;
  double tol;
  const int *col;
  const double *val;
  const double *b;   // [nv][Nd]
  double *x;         // [nv][Nd]
  double *work;      // [nv][3][Nd]: r, p, q
  int *status;       // [nv]: iterations, or -1 if the residual did not reach tol ||b||
  // Symmetry-plane boundary conditions (edge_bc): keep[rep][Nd] = 0 removes
  // an unknown (identity row and column, zero right-hand side, so it stays
  // 0, as reduce_system / expand_solution leave it); vector v belongs to
  // representation (v / vec_per_col) / nsrc.  Null: nothing removed.
  const unsigned char *keep;
  int vec_per_col, nsrc;
};

__device__ __forceinline__ void block_sum2(double &a, double &b, double *red) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) {
    red[wid] = a;
    red[32 + wid] = b;
  }
  __syncthreads();
  a = 0;
  b = 0;
  for (int i = 0; i < nw; i++) {
    a += red[i];
    b += red[32 + i];
  }
}

// One CTA per real right-hand side: Jacobi-preconditioned conjugate
// gradients with at most maxit iterations (the loop always ends).
__global__ void __launch_bounds__(kCgThreads) gram_cg_kernel(CgArgs a) {
  __shared__ double red[64];
  const int v = blockIdx.x, n = a.Nd;
  const double *b = a.b + (size_t)v * n;
  double *x = a.x + (size_t)v * n;
  double *r = a.work + (size_t)v * 3 * n, *p = r + n, *q = p + n;
  const unsigned char *km = a.keep ? a.keep + (size_t)((v / a.vec_per_col) / a.nsrc) * n : nullptr;
  auto kept = [&](int i) { return km == nullptr || km[i] != 0; };
  auto diag = [&](int i) { return kept(i) ? a.val[(size_t)i * kEll] : 1.0; };
  double rz = 0, bb = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double bi = kept(i) ? b[i] : 0.0, zi = bi / diag(i);
    x[i] = 0;
    r[i] = bi;
    p[i] = zi;
    rz += bi * zi;
    bb += bi * bi;
  }
  block_sum2(rz, bb, red);
  int it = 0;
  bool done = bb == 0.0;  // a zero right-hand side: x = 0; a NaN one never converges
  const double lim = a.tol * a.tol * bb;
  while (!done && it < a.maxit) {
    __syncthreads();  // p complete before the product reads neighbours
    double pq = 0, dummy = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int *ci = a.col + (size_t)i * kEll;
      const double *vi = a.val + (size_t)i * kEll;
      double s = 0;
      if (km == nullptr) {
#pragma unroll
        for (int k = 0; k < kEll; k++) s += vi[k] * p[ci[k]];
      } else if (km[i]) {
#pragma unroll
        for (int k = 0; k < kEll; k++) s += km[ci[k]] ? vi[k] * p[ci[k]] : 0.0;
      } else {
        s = p[i];
      }
      q[i] = s;
      pq += p[i] * s;
    }
    block_sum2(pq, dummy, red);
    const double alpha = rz / pq;
    double rr = 0, rzn = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      x[i] += alpha * p[i];
      const double ri = r[i] - alpha * q[i];
      r[i] = ri;
      rr += ri * ri;
      rzn += ri * ri / diag(i);
    }
    block_sum2(rr, rzn, red);
    it++;
    if (rr <= lim || !(pq > 0)) {
      done = rr <= lim;
      break;
    }
    const double beta = rzn / rz;
    rz = rzn;
    for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = r[i] / diag(i) + beta * p[i];
  }
  if (threadIdx.x == 0) a.status[v] = done ? it : -1;
}

struct CmArgs {
  double w[kMaxQ];
  int F, Nd, nq;
  const double *qabs, *area, *nrm, *sl, *bn;
  const int *fedge;
  const double *coef;  // solved coefficients [nsrc][4][Nd] (re, im first)
  double2 *half;       // [nsrc][F][3]
};

// Thread per (face, source): A sum_r w_r f_q . (n x sum_p f_p coef_p).
__global__ void nls_cm_kernel(CmArgs a) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (f >= a.F) return;
  const double A = a.area[f];
  const double nor[3] = {a.nrm[3 * f], a.nrm[3 * f + 1], a.nrm[3 * f + 2]};
  const double *cre = a.coef + (size_t)s * 4 * a.Nd, *cim = cre + a.Nd;
  Z cf[3];
  for (int p = 0; p < 3; p++) {
    const int e = a.fedge[3 * f + p];
    cf[p] = {cre[e], cim[e]};
  }
  Z acc[3] = {{0, 0}, {0, 0}, {0, 0}};
  for (int r = 0; r < a.nq; r++) {
    const double *pt = a.qabs + ((size_t)f * a.nq + r) * 3;
    double fq[3][3];
    for (int q = 0; q < 3; q++) rwg_at(pt, a.bn + 9 * (size_t)f + 3 * q, a.sl[3 * f + q], A, fq[q]);
    Z ex[3] = {{0, 0}, {0, 0}, {0, 0}};
    for (int p = 0; p < 3; p++)
      for (int i = 0; i < 3; i++) ex[i] = zadd(ex[i], zrs(cf[p], fq[p][i]));
    Z ncr[3];
    ncr[0] = zsub(zrs(ex[2], nor[1]), zrs(ex[1], nor[2]));
    ncr[1] = zsub(zrs(ex[0], nor[2]), zrs(ex[2], nor[0]));
    ncr[2] = zsub(zrs(ex[1], nor[0]), zrs(ex[0], nor[1]));
    for (int q = 0; q < 3; q++) {
      Z d = {0, 0};
      for (int i = 0; i < 3; i++) d = zadd(d, zrs(ncr[i], fq[q][i]));
      acc[q] = zadd(acc[q], zrs(d, a.w[r]));
    }
  }
  for (int q = 0; q < 3; q++)
    a.half[((size_t)s * a.F + f) * 3 + q] = make_double2(acc[q].re * A, acc[q].im * A);
}

// Thread per (domain edge, source): the right-hand side of the M-coefficient
// Gram system, [nsrc][2][Nd].
__global__ void nls_cm_edge_kernel(int F, int Nd, const int *eh, const double2 *half, double *rhs) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (e >= Nd) return;
  double re = 0, im = 0;
  for (int k = 0; k < 2; k++) {
    const int h = eh[2 * e + k];
    if (h < 0) continue;
    const double2 v = half[(size_t)s * F * 3 + h];
    re += v.x;
    im += v.y;
  }
  rhs[(size_t)s * 2 * Nd + e] = re;
  rhs[(size_t)s * 2 * Nd + Nd + e] = im;
}

// Thread per (domain edge, source): c[epar] = cJ, c[N + epar] = cM.
__global__ void nls_scatter_kernel(int Nd, int N, int64_t ldc, const int *epar, const double *cj, const double *cm,
                                   double2 *C) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (e >= Nd) return;
  const double *j = cj + (size_t)s * 4 * Nd + 2 * Nd;  // J coefficients: vectors 2, 3 of the first system
  const double *m = cm + (size_t)s * 2 * Nd;
  double2 *c = C + (size_t)s * ldc;
  c[epar[e]] = make_double2(j[e], j[Nd + e]);
  c[N + epar[e]] = make_double2(m[e], m[Nd + e]);
}

template <class T>
int shg_upload(Ctx *c, T **dst, const std::vector<T> &src) {
  MOM_CUDA(c, cudaMalloc(dst, sizeof(T) * std::max<size_t>(src.size(), 1)));
  MOM_CUDA(c, cudaMemcpyAsync(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice, c->stream));
  return MOM_OK;
}

// Free vertices, face-local to domain edge map and the Gram matrix of domain
// d (geometry only; made once per problem).
int shg_setup(Ctx *c, int d) {
  DomDev &D = c->dom[d];
  if (D.gram_val) return MOM_OK;
  std::vector<int> fedge(3 * (size_t)D.F, -1);
  for (int e = 0; e < D.Nd; e++)
    for (int k = 0; k < 2; k++)
      if (D.h_eh[2 * e + k] >= 0) fedge[D.h_eh[2 * e + k]] = e;
  for (int v : fedge)
    if (v < 0) return fail(c, MOM_ERR_MESH, "a face edge without a domain edge");
  MOM_TRY(shg_upload(c, &D.shg_bn, D.h_bn));
  MOM_TRY(shg_upload(c, &D.shg_fedge, fedge));
  MOM_CUDA(c, cudaMalloc(&D.gram_col, sizeof(int) * kEll * (size_t)D.Nd));
  MOM_CUDA(c, cudaMalloc(&D.gram_val, sizeof(double) * kEll * (size_t)D.Nd));
  double *G = nullptr;
  MOM_CUDA(c, cudaMalloc(&G, sizeof(double) * 9 * (size_t)D.F));
  GramArgs g;
  for (int i = 0; i < kMaxQ; i++) g.w[i] = c->qw[i];
  g.F = D.F;
  g.Nd = D.Nd;
  g.nq = c->nq;
  g.qabs = D.qabs;
  g.area = D.area;
  g.sl = D.sl;
  g.bn = D.shg_bn;
  g.eh = D.eh;
  g.fedge = D.shg_fedge;
  g.G = G;
  g.col = D.gram_col;
  g.val = D.gram_val;
  gram_face_kernel<<<(D.F + 127) / 128, 128, 0, c->stream>>>(g);
  gram_ell_kernel<<<(D.Nd + 127) / 128, 128, 0, c->stream>>>(g);
  c->launches += 2;
  const cudaError_t le = cudaGetLastError();
  const cudaError_t se = cudaStreamSynchronize(c->stream);
  cudaFree(G);
  MOM_CUDA(c, le);
  MOM_CUDA(c, se);
  return MOM_OK;
}

// determine_epsp (solver.f90:393-433): per face of domain d, eps0 ri^2 of
// the first other domain that has the same face (the same three master
// edges).
int face_epsp(Ctx *c, int d, const double *ri, std::vector<double2> &epsp) {
  auto key = [&](const DomDev &D, int f) {
    std::array<int, 3> k = {D.h_hpar[3 * (size_t)f], D.h_hpar[3 * (size_t)f + 1], D.h_hpar[3 * (size_t)f + 2]};
    std::sort(k.begin(), k.end());
    return k;
  };
  std::vector<std::set<std::array<int, 3>>> faces(c->ndom);
  for (int d2 = 0; d2 < c->ndom; d2++)
    if (d2 != d)
      for (int f = 0; f < c->dom[d2].F; f++) faces[d2].insert(key(c->dom[d2], f));
  const DomDev &D = c->dom[d];
  epsp.assign(D.F, make_double2(0, 0));
  for (int f = 0; f < D.F; f++) {
    const std::array<int, 3> k = key(D, f);
    int found = -1;
    for (int d2 = 0; d2 < c->ndom && found < 0; d2++)
      if (d2 != d && faces[d2].count(k)) found = d2;
    if (found < 0) return fail(c, MOM_ERR_ARG, "Could not find epsp! (a face of a nonlinear domain is in no other domain)");
    const double a = ri[2 * found], b = ri[2 * found + 1];
    epsp[f] = make_double2((a * a - b * b) * kEps0, 2 * a * b * kEps0);
  }
  return MOM_OK;
}

struct ShgBuf {
  size_t off_half, off_rhs, off_x1, off_rhs2, off_x2, off_work, off_st, off_epsp, total;
};

ShgBuf shg_layout(int F, int Nd, int nsrc) {
  auto al = [](size_t b) { return (b + 255) / 256 * 256; };
  ShgBuf L;
  size_t o = 0;
  L.off_half = o;
  o += al(sizeof(double2) * 9 * (size_t)F * nsrc);
  L.off_rhs = o;
  o += al(sizeof(double) * 4 * (size_t)Nd * nsrc);
  L.off_x1 = o;
  o += al(sizeof(double) * 4 * (size_t)Nd * nsrc);
  L.off_rhs2 = o;
  o += al(sizeof(double) * 2 * (size_t)Nd * nsrc);
  L.off_x2 = o;
  o += al(sizeof(double) * 2 * (size_t)Nd * nsrc);
  L.off_work = o;
  o += al(sizeof(double) * 3 * 4 * (size_t)Nd * nsrc);
  L.off_st = o;
  o += al(sizeof(int) * 4 * (size_t)nsrc);
  L.off_epsp = o;
  o += al(sizeof(double2) * (size_t)F);
  L.total = o;
  return L;
}

constexpr int kCgMaxIt = 20000;
constexpr double kCgTol = 1e-14;

int run_cg(Ctx *c, const DomDev &D, int nv, const double *b, double *x, double *work, int *status,
           const unsigned char *keep, int vec_per_col, int nsrc) {
  CgArgs g;
  g.keep = keep;
  g.vec_per_col = vec_per_col;
  g.nsrc = nsrc;
  g.Nd = D.Nd;
  g.maxit = kCgMaxIt;
  g.tol = kCgTol;
  g.col = D.gram_col;
  g.val = D.gram_val;
  g.b = b;
  g.x = x;
  g.work = work;
  g.status = status;
  gram_cg_kernel<<<nv, kCgThreads, 0, c->stream>>>(g);
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  std::vector<int> st(nv);
  MOM_CUDA(c, cudaMemcpyAsync(st.data(), status, sizeof(int) * nv, cudaMemcpyDeviceToHost, c->stream));
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  for (int v : st)
    if (v < 0) return fail(c, MOM_ERR_NOCONV, "the RWG Gram system of the surface polarisation did not converge");
  return MOM_OK;
}

}  // namespace

void free_shg(DomDev &D) {
  cudaFree(D.shg_bn);
  cudaFree(D.shg_fedge);
  cudaFree(D.gram_col);
  cudaFree(D.gram_val);
  D.shg_bn = nullptr;
  D.shg_fedge = nullptr;
  D.gram_col = nullptr;
  D.gram_val = nullptr;
}

int shg_solve(Ctx *c, double omega, const double *ri, const double *shri, const mom_nls *nls, int precision,
              double tol, int maxit, int *iters) {
  const int nsrc = c->nsrc, nga = c->nga;
  const int ncol = nga * nsrc;  // (representation, source) columns: column r nsrc + s at X, B + (r nsrc + s) n
  const int64_t n = c->n;
  const double omega_sh = 2.0 * omega;
  std::vector<int> nl;
  c->shg_slot.assign(c->ndom, -1);
  for (int d = 0; d < c->ndom; d++)
    if (nls[d].active) {
      c->shg_slot[d] = (int)nl.size();
      nl.push_back(d);
    }
  // source coefficients of every nonlinear domain, [nl][ncol][n]
  MOM_TRY(ensure_buffer(c, &c->shg_c, &c->shg_c_bytes, sizeof(double2) * (size_t)n * ncol * std::max<size_t>(nl.size(), 1)));
  double2 *Call = (double2 *)c->shg_c;
  MOM_CUDA(c, cudaMemsetAsync(Call, 0, sizeof(double2) * (size_t)n * ncol * nl.size(), c->stream));
  MOM_CUDA(c, cudaMemsetAsync(c->B, 0, sizeof(double2) * (size_t)n * ncol, c->stream));
  ShgGroup G;
  std::memset(&G, 0, sizeof G);
  G.nga = nga;
  for (int g = 0; g < nga; g++) {
    for (int i = 0; i < 9; i++) G.j[g][i] = c->ga[g].j[i];
    G.detj[g] = c->ga[g].detj;
    for (int r = 0; r < nga; r++) G.ef[g][r] = c->ga[g].ef[r];
  }
  for (size_t k = 0; k < nl.size(); k++) {
    const int d = nl[k];
    MOM_TRY(shg_setup(c, d));
    const DomDev &D = c->dom[d];
    std::vector<double2> epsp;
    MOM_TRY(face_epsp(c, d, ri, epsp));
    // edge_bc on the domain mesh per representation: the E-type unknowns (coef
    // and cJ) and the H-type ones (cM) that the symmetry planes remove
    std::vector<unsigned char> keep;
    if (nga > 1) {
      keep.assign(2 * (size_t)nga * D.Nd, 1);
      for (int r = 0; r < nga; r++) {
        std::vector<char> rem(2 * (size_t)c->N, 0);
        for (int u : c->removed[r]) rem[u] = 1;
        for (int e = 0; e < D.Nd; e++) {
          keep[(size_t)r * D.Nd + e] = !rem[D.h_epar[e]];
          keep[((size_t)nga + r) * D.Nd + e] = !rem[c->N + D.h_epar[e]];
        }
      }
    }
    const ShgBuf L = shg_layout(D.F, D.Nd, ncol);
    const size_t keep_off = (L.total + 255) / 256 * 256;
    MOM_TRY(ensure_buffer(c, &c->shg_ws, &c->shg_ws_bytes, keep_off + keep.size() + 256));
    char *ws = (char *)c->shg_ws;
    double2 *half = (double2 *)(ws + L.off_half), *dep = (double2 *)(ws + L.off_epsp);
    double *rhs = (double *)(ws + L.off_rhs), *x1 = (double *)(ws + L.off_x1), *rhs2 = (double *)(ws + L.off_rhs2),
           *x2 = (double *)(ws + L.off_x2), *work = (double *)(ws + L.off_work);
    int *st = (int *)(ws + L.off_st);
    unsigned char *dkeep = keep.empty() ? nullptr : (unsigned char *)(ws + keep_off);
    MOM_CUDA(c, cudaMemcpyAsync(dep, epsp.data(), sizeof(double2) * D.F, cudaMemcpyHostToDevice, c->stream));
    if (dkeep) MOM_CUDA(c, cudaMemcpyAsync(dkeep, keep.data(), keep.size(), cudaMemcpyHostToDevice, c->stream));
    const mom_nls &m = nls[d];
    FaceArgs fa;
    for (int i = 0; i < kMaxQ; i++) fa.w[i] = c->qw[i];
    fa.F = D.F;
    fa.nq = c->nq;
    fa.N = c->N;
    fa.nsrc = nsrc;
    fa.ldx = n;
    fa.xrep = (int64_t)nsrc * n;
    fa.qabs = D.qabs;
    fa.area = D.area;
    fa.nrm = D.nrm;
    fa.sl = D.sl;
    fa.bn = D.shg_bn;
    fa.hpar = D.hpar;
    fa.X = c->X;
    fa.epsp = dep;
    // i omega eps0 ri^2 of domain d at the fundamental
    const double a = ri[2 * d], b = ri[2 * d + 1];
    const double e_re = (a * a - b * b) * kEps0, e_im = 2 * a * b * kEps0;
    fa.iwe = {-omega * e_im, omega * e_re};
    fa.chi_nnn = {m.chi_nnn[0], m.chi_nnn[1]};
    fa.chi_ntt = {m.chi_ntt[0], m.chi_ntt[1]};
    fa.chi_ttn = {m.chi_ttn[0], m.chi_ttn[1]};
    fa.G = G;
    fa.half = half;
    {
      ProfScope ps(c, kProfPost);
      nls_face_kernel<<<dim3((D.F + 127) / 128, nsrc, nga), 128, 0, c->stream>>>(fa);
      c->launches++;
      MOM_CUDA(c, cudaGetLastError());
    }
    EdgeArgs ea;
    ea.F = D.F;
    ea.Nd = D.Nd;
    ea.N = c->N;
    ea.ldb = n;
    ea.eh = D.eh;
    ea.epar = D.epar;
    ea.half = half;
    ea.omega_sh = omega_sh;
    ea.B = c->B;
    ea.rhs = rhs;
    nls_edge_kernel<<<dim3((D.Nd + 127) / 128, ncol), 128, 0, c->stream>>>(ea);
    c->launches++;
    MOM_CUDA(c, cudaGetLastError());
    MOM_TRY(run_cg(c, D, 4 * ncol, rhs, x1, work, st, dkeep, 4, nsrc));
    CmArgs ca;
    for (int i = 0; i < kMaxQ; i++) ca.w[i] = c->qw[i];
    ca.F = D.F;
    ca.Nd = D.Nd;
    ca.nq = c->nq;
    ca.qabs = D.qabs;
    ca.area = D.area;
    ca.nrm = D.nrm;
    ca.sl = D.sl;
    ca.bn = D.shg_bn;
    ca.fedge = D.shg_fedge;
    ca.coef = x1;
    ca.half = half;
    nls_cm_kernel<<<dim3((D.F + 127) / 128, ncol), 128, 0, c->stream>>>(ca);
    nls_cm_edge_kernel<<<dim3((D.Nd + 127) / 128, ncol), 128, 0, c->stream>>>(D.F, D.Nd, D.eh, half, rhs2);
    c->launches += 2;
    MOM_CUDA(c, cudaGetLastError());
    MOM_TRY(run_cg(c, D, 2 * ncol, rhs2, x2, work, st, dkeep ? dkeep + (size_t)nga * D.Nd : nullptr, 2, nsrc));
    nls_scatter_kernel<<<dim3((D.Nd + 127) / 128, ncol), 128, 0, c->stream>>>(D.Nd, c->N, n, D.epar, x1, x2,
                                                                               Call + k * (size_t)n * ncol);
    c->launches++;
    MOM_CUDA(c, cudaGetLastError());
  }
  // sysmat_pmchwt_nls: the nonlinear domains first, each block applied to
  // its own coefficients as A_after c - A_before c in every representation,
  // then the other domains.
  const size_t col_rep = (size_t)nsrc * n;
  auto apply = [&](const double2 *Ck, double sign) -> int {
    for (int r = 0; r < nga; r++) {
      select_rep(c, r);
      MOM_TRY(matvec_acc(c, Ck + r * col_rep, nsrc, c->B + r * col_rep, sign));
    }
    select_rep(c, 0);
    return MOM_OK;
  };
  select_rep(c, 0);
  MOM_TRY(assemble_begin(c));
  for (size_t k = 0; k < nl.size(); k++) {
    const double2 *Ck = Call + k * (size_t)n * ncol;
    if (k > 0) MOM_TRY(apply(Ck, 1.0));
    MOM_TRY(assemble_domain(c, nl[k], omega_sh, shri, precision));
    MOM_TRY(apply(Ck, -1.0));
  }
  for (int d = 0; d < c->ndom; d++)
    if (!nls[d].active) MOM_TRY(assemble_domain(c, d, omega_sh, shri, precision));
  MOM_TRY(assemble_end(c, precision));
  c->omega_rhs = omega_sh;
  c->ri1[0] = shri[0];
  c->ri1[1] = shri[1];
  // solve_systems per representation: the removed unknowns' right-hand
  // sides are zero (identity rows), one factorisation and solve each
  int it = 0;
  for (int r = 0; r < nga && nga > 1; r++) MOM_TRY(apply_bc_rhs(c, r, c->B + r * col_rep, nsrc));
  for (int r = 0; r < nga; r++) {
    select_rep(c, r);
    const int rc = lu_factor(c, precision);
    if (rc != MOM_OK) {
      select_rep(c, 0);
      return rc;
    }
  }
  for (int r = 0; r < nga; r++) {
    select_rep(c, r);
    int itr = 0;
    const int rc = lu_solve_ex(c, precision, 0, c->B + r * col_rep, c->X + r * col_rep, nsrc, tol, maxit, &itr);
    if (rc != MOM_OK) {
      select_rep(c, 0);
      return rc;
    }
    it = std::max(it, itr);
  }
  select_rep(c, 0);
  if (iters) *iters = it;
  if (precision == MOM_PREC_FP64) c->assembled = 0;
  return MOM_OK;
}

}  // namespace mom
