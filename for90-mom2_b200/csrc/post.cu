// Excitation and post-processing reductions on sm_100a (FP64):
//   rhs      -> srcvec / src_field_frags / pw_fields(_elliptic)
//               (source.f90:84-125, 136-315) for identity symmetry;
//   cs       -> cs_prtsrf (cs.f90:14-104);
//   farfield -> far_fields / rcs_ext / rcs (ffields.f90:16-122, 203-266).
// Each edge receives contributions from its two faces; those are computed
// per half-edge and summed per edge in a second pass, so results are
// deterministic (the reference adds them in face order).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "mom_internal.h"

namespace mom {

namespace {

}  // namespace

// get_dir / get_pol (aux.f90:245-261), evaluated on the host in FP64.
void src_geometry(const mom_src &s, double dir[3], double pol[3]) {
  const double th = s.theta, ph = s.phi, ps = (s.type == MOM_SRC_PW) ? s.psi : 0.0;
  dir[0] = sin(th) * cos(ph);
  dir[1] = sin(th) * sin(ph);
  dir[2] = cos(th);
  pol[0] = cos(ps) * sin(ph) - sin(ps) * cos(th) * cos(ph);
  pol[1] = -cos(ps) * cos(ph) - sin(ps) * cos(th) * sin(ph);
  pol[2] = sin(ps) * sin(th);
}

namespace {

struct SrcDev {
  double dir[3], pol[3];
  double ph_re, ph_im;  // pw_elliptic phase
  int type;
};

struct Z {
  double re, im;
};
__device__ __forceinline__ Z zmul(Z a, Z b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ Z zadd(Z a, Z b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ Z zsub(Z a, Z b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ Z zscale(Z a, double s) { return {a.re * s, a.im * s}; }
__device__ __forceinline__ Z zconj(Z a) { return {a.re, -a.im}; }
__device__ __forceinline__ void zcross(const Z *a, const Z *b, Z *r) {
  r[0] = zsub(zmul(a[1], b[2]), zmul(a[2], b[1]));
  r[1] = zsub(zmul(a[2], b[0]), zmul(a[0], b[2]));
  r[2] = zsub(zmul(a[0], b[1]), zmul(a[1], b[0]));
}
__device__ __forceinline__ Z zexp_i(Z k, double s) {  // exp(i k s)
  double sn, cs;
  sincos(k.re * s, &sn, &cs);
  const double a = exp(-k.im * s);
  return {a * cs, a * sn};
}

// pw_fields / pw_fields_elliptic (source.f90:84-125) at point pt.
__device__ void src_fields(const SrcDev &S, Z k, double omega, const double *pt, Z *ef, Z *hf) {
  if (S.type == MOM_SRC_NONE) {  // no incident field (src_fields, source.f90:328-329)
    for (int i = 0; i < 3; i++) ef[i] = hf[i] = {0, 0};
    return;
  }
  const double kd = S.dir[0] * pt[0] + S.dir[1] * pt[1] + S.dir[2] * pt[2];
  const Z ph = zexp_i(k, kd);
  Z dc[3] = {{S.dir[0], 0}, {S.dir[1], 0}, {S.dir[2], 0}};
  if (S.type == MOM_SRC_PW) {
    for (int i = 0; i < 3; i++) ef[i] = zscale(ph, S.pol[i]);
  } else {
    Z efx[3], efy[3];
    for (int i = 0; i < 3; i++) efx[i] = zscale(ph, S.pol[i]);
    zcross(dc, efx, efy);
    const Z phase = {S.ph_re, S.ph_im};
    double nn = 0;
    for (int i = 0; i < 3; i++) {
      ef[i] = zadd(efx[i], zmul(phase, efy[i]));
      nn += ef[i].re * ef[i].re + ef[i].im * ef[i].im;
    }
    nn = sqrt(nn);
    for (int i = 0; i < 3; i++) ef[i] = {ef[i].re / nn, ef[i].im / nn};
  }
  Z c[3];
  zcross(dc, ef, c);
  const Z kk = {k.re / (omega * kMu0), k.im / (omega * kMu0)};
  for (int i = 0; i < 3; i++) hf[i] = zmul(kk, c[i]);
}

struct RhsArgs {
  double w[kMaxQ];
  int F, nq;
  const double *qabs, *area, *sl, *mu, *cp;
  const SrcDev *src;
  int nsrc;
  Z k;
  double omega;
  double2 *half;  // [nsrc][F][3][2]  (E part, H part)
};

// Thread per (face, source): <f_p, E_inc>, <f_p, H_inc> for the three RWG
// halves of the face (source.f90:214-246).
__global__ void rhs_half_kernel(RhsArgs a) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (f >= a.F) return;
  const SrcDev S = a.src[s];
  Z Ie[3] = {{0, 0}, {0, 0}, {0, 0}}, Ih[3] = {{0, 0}, {0, 0}, {0, 0}};
  const double Am = a.area[f];
  for (int r = 0; r < a.nq; r++) {
    const double *pt = a.qabs + ((size_t)f * a.nq + r) * 3;
    Z ef[3], hf[3];
    src_fields(S, a.k, a.omega, pt, ef, hf);
    const double w = a.w[r];
    for (int p = 0; p < 3; p++) {
      // f_p(r) = sl_p / (2 Am) (r - v_p),  v_p = cp + mu_p
      const double cc = a.sl[3 * f + p] / (2.0 * Am);
      double fm[3];
      for (int i = 0; i < 3; i++) fm[i] = cc * (pt[i] - (a.cp[3 * f + i] + a.mu[9 * f + 3 * p + i]));
      Z de = {0, 0}, dh = {0, 0};
      for (int i = 0; i < 3; i++) {
        de = zadd(de, zscale(ef[i], fm[i]));
        dh = zadd(dh, zscale(hf[i], fm[i]));
      }
      Ie[p] = zadd(Ie[p], zscale(de, w));
      Ih[p] = zadd(Ih[p], zscale(dh, w));
    }
  }
  double2 *o = a.half + (((size_t)s * a.F + f) * 3) * 2;
  for (int p = 0; p < 3; p++) {
    o[2 * p] = make_double2(Ie[p].re * Am, Ie[p].im * Am);
    o[2 * p + 1] = make_double2(Ih[p].re * Am, Ih[p].im * Am);
  }
}

// Per domain edge: q[J] = sum of the halves' E parts, q[M] = H parts.
__global__ void rhs_edge_kernel(int Nd, int F, int N, int64_t ldb, const int *eh, const int *epar,
                                const double2 *half, double2 *B) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (e >= Nd) return;
  double2 qe = make_double2(0, 0), qh = make_double2(0, 0);
  int h[2] = {eh[2 * e], eh[2 * e + 1]};
  if (h[0] >= 0 && h[1] >= 0 && h[1] < h[0]) {  // face order, as the reference accumulates
    int t = h[0];
    h[0] = h[1];
    h[1] = t;
  }
  for (int i = 0; i < 2; i++) {
    if (h[i] < 0) continue;
    const double2 *v = half + (((size_t)s * F) * 3 + h[i]) * 2;
    qe.x += v[0].x;
    qe.y += v[0].y;
    qh.x += v[1].x;
    qh.y += v[1].y;
  }
  const int64_t r = epar[e];
  B[(size_t)s * ldb + r] = qe;
  B[(size_t)s * ldb + r + N] = qh;
}

struct CsArgs {
  double w[kMaxQ];
  int F, nq, N;
  const double *qabs, *area, *sl, *mu, *cp, *nrm;
  const int *hpar;
  const SrcDev *src;
  const double2 *x;
  int64_t ldx;
  Z k;
  double omega;
  double *part;  // [nsrc][gridDim.x][2]
};

// cs_prtsrf: per face the Poynting flux of total and scattered tangential
// fields at the quadrature points; block partial sums.
__global__ void __launch_bounds__(256) cs_kernel(CsArgs a) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  double i1 = 0, i2 = 0;
  if (f < a.F) {
    const SrcDev S = a.src[s];
    const double2 *x = a.x + (size_t)s * a.ldx;
    const double An = a.area[f];
    const double *nor = a.nrm + 3 * f;
    const Z nc[3] = {{nor[0], 0}, {nor[1], 0}, {nor[2], 0}};
    Z al[3], be[3];
    for (int p = 0; p < 3; p++) {
      const int idx = a.hpar[3 * f + p];
      al[p] = {x[idx].x, x[idx].y};
      be[p] = {x[idx + a.N].x, x[idx + a.N].y};
    }
    double int1 = 0, int2 = 0;
    for (int t = 0; t < a.nq; t++) {
      const double *pt = a.qabs + ((size_t)f * a.nq + t) * 3;
      Z Et[3] = {{0, 0}, {0, 0}, {0, 0}}, Ht[3] = {{0, 0}, {0, 0}, {0, 0}};
      for (int p = 0; p < 3; p++) {
        const double cc = a.sl[3 * f + p] / (2.0 * An);
        double fr[3], fn[3];
        for (int i = 0; i < 3; i++) fr[i] = cc * (pt[i] - (a.cp[3 * f + i] + a.mu[9 * f + 3 * p + i]));
        fn[0] = nor[1] * fr[2] - nor[2] * fr[1];
        fn[1] = nor[2] * fr[0] - nor[0] * fr[2];
        fn[2] = nor[0] * fr[1] - nor[1] * fr[0];
        for (int i = 0; i < 3; i++) {
          Ht[i] = zsub(Ht[i], zscale(al[p], fn[i]));
          Et[i] = zadd(Et[i], zscale(be[p], fn[i]));
        }
      }
      Z einc[3], hinc[3], t1[3], Eti[3], Hti[3], Ets[3], Hts[3], cr[3], cj[3];
      src_fields(S, a.k, a.omega, pt, einc, hinc);
      zcross(nc, hinc, t1);
      zcross(t1, nc, Hti);
      zcross(nc, einc, t1);
      zcross(t1, nc, Eti);
      for (int i = 0; i < 3; i++) {
        Hts[i] = zsub(Ht[i], Hti[i]);
        Ets[i] = zsub(Et[i], Eti[i]);
        cj[i] = zconj(Ht[i]);
      }
      zcross(Et, cj, cr);
      double Sn = 0.5 * (cr[0].re * nor[0] + cr[1].re * nor[1] + cr[2].re * nor[2]);
      const double w = a.w[t];
      int1 += w * Sn;
      for (int i = 0; i < 3; i++) cj[i] = zconj(Hts[i]);
      zcross(Ets, cj, cr);
      Sn = 0.5 * (cr[0].re * nor[0] + cr[1].re * nor[1] + cr[2].re * nor[2]);
      int2 += w * Sn;
    }
    i1 = int1 * An;
    i2 = int2 * An;
  }
  // deterministic block reduction
  __shared__ double r1[256], r2[256];
  r1[threadIdx.x] = i1;
  r2[threadIdx.x] = i2;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      r1[threadIdx.x] += r1[threadIdx.x + w];
      r2[threadIdx.x] += r2[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    a.part[((size_t)s * gridDim.x + blockIdx.x) * 2] = r1[0];
    a.part[((size_t)s * gridDim.x + blockIdx.x) * 2 + 1] = r2[0];
  }
}

// d sigma / dx of cs_prtsrf, d sigma = Re(G^T dx), per face and source:
// with E = sum_p beta_p (n x f_p) and H = -sum_p alpha_p (n x f_p),
// d/dbeta_p 0.5 Re[(E x H*).n] = 0.5 (n x f_p) x H* . n and
// d/dalpha_p = -0.5 E* x (n x f_p) . n; sigma_abs uses the total fields,
// sigma_sca the scattered ones.  Output per half: [s][F][3][ext alpha,
// ext beta, abs alpha, abs beta].
__global__ void __launch_bounds__(128) cs_grad_half_kernel(CsArgs a, double cc, double2 *half) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (f >= a.F) return;
  const SrcDev S = a.src[s];
  const double2 *x = a.x + (size_t)s * a.ldx;
  const double An = a.area[f];
  const double *nor = a.nrm + 3 * f;
  const Z nc[3] = {{nor[0], 0}, {nor[1], 0}, {nor[2], 0}};
  Z al[3], be[3];
  for (int p = 0; p < 3; p++) {
    const int idx = a.hpar[3 * f + p];
    al[p] = {x[idx].x, x[idx].y};
    be[p] = {x[idx + a.N].x, x[idx + a.N].y};
  }
  Z g[3][4];
  for (int p = 0; p < 3; p++)
    for (int k = 0; k < 4; k++) g[p][k] = {0, 0};
  for (int t = 0; t < a.nq; t++) {
    const double *pt = a.qabs + ((size_t)f * a.nq + t) * 3;
    double fn[3][3];
    Z Et[3] = {{0, 0}, {0, 0}, {0, 0}}, Ht[3] = {{0, 0}, {0, 0}, {0, 0}};
    for (int p = 0; p < 3; p++) {
      const double c0 = a.sl[3 * f + p] / (2.0 * An);
      double fr[3];
      for (int i = 0; i < 3; i++) fr[i] = c0 * (pt[i] - (a.cp[3 * f + i] + a.mu[9 * f + 3 * p + i]));
      fn[p][0] = nor[1] * fr[2] - nor[2] * fr[1];
      fn[p][1] = nor[2] * fr[0] - nor[0] * fr[2];
      fn[p][2] = nor[0] * fr[1] - nor[1] * fr[0];
      for (int i = 0; i < 3; i++) {
        Ht[i] = zsub(Ht[i], zscale(al[p], fn[p][i]));
        Et[i] = zadd(Et[i], zscale(be[p], fn[p][i]));
      }
    }
    Z einc[3], hinc[3], t1[3], Eti[3], Hti[3], Es[3], Hs[3];
    src_fields(S, a.k, a.omega, pt, einc, hinc);
    zcross(nc, hinc, t1);
    zcross(t1, nc, Hti);
    zcross(nc, einc, t1);
    zcross(t1, nc, Eti);
    for (int i = 0; i < 3; i++) {
      Hs[i] = zsub(Ht[i], Hti[i]);
      Es[i] = zsub(Et[i], Eti[i]);
    }
    const double w = 0.5 * a.w[t] * An;
    for (int p = 0; p < 3; p++) {
      const Z fz[3] = {{fn[p][0], 0}, {fn[p][1], 0}, {fn[p][2], 0}};
      Z hc[3], ec[3], cr[3];
      // total fields
      for (int i = 0; i < 3; i++) {
        hc[i] = zconj(Ht[i]);
        ec[i] = zconj(Et[i]);
      }
      zcross(fz, hc, cr);
      const Z gbt = zadd(zadd(zscale(cr[0], nor[0]), zscale(cr[1], nor[1])), zscale(cr[2], nor[2]));
      zcross(ec, fz, cr);
      const Z gat = zscale(zadd(zadd(zscale(cr[0], nor[0]), zscale(cr[1], nor[1])), zscale(cr[2], nor[2])), -1.0);
      // scattered fields
      for (int i = 0; i < 3; i++) {
        hc[i] = zconj(Hs[i]);
        ec[i] = zconj(Es[i]);
      }
      zcross(fz, hc, cr);
      const Z gbs = zadd(zadd(zscale(cr[0], nor[0]), zscale(cr[1], nor[1])), zscale(cr[2], nor[2]));
      zcross(ec, fz, cr);
      const Z gas = zscale(zadd(zadd(zscale(cr[0], nor[0]), zscale(cr[1], nor[1])), zscale(cr[2], nor[2])), -1.0);
      // sigma_ext = cc (I_sca - I_tot), sigma_abs = -cc I_tot
      g[p][0] = zadd(g[p][0], zscale(zsub(gas, gat), cc * w));
      g[p][1] = zadd(g[p][1], zscale(zsub(gbs, gbt), cc * w));
      g[p][2] = zadd(g[p][2], zscale(gat, -cc * w));
      g[p][3] = zadd(g[p][3], zscale(gbt, -cc * w));
    }
  }
  double2 *o = half + (((size_t)s * a.F + f) * 3) * 4;
  for (int p = 0; p < 3; p++)
    for (int k = 0; k < 4; k++) o[4 * p + k] = make_double2(g[p][k].re, g[p][k].im);
}

// G[2 s] (ext) and G[2 s + 1] (abs): sums of the halves of each edge.
__global__ void cs_grad_edge_kernel(int Nd, int F, int N, int64_t n, const int *eh, const int *epar,
                                    const double2 *half, double2 *G) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (e >= Nd) return;
  double2 v[4] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
  for (int i = 0; i < 2; i++) {
    const int h = eh[2 * e + i];
    if (h < 0) continue;
    const double2 *src = half + (((size_t)s * F) * 3 + h) * 4;
    for (int k = 0; k < 4; k++) {
      v[k].x += src[k].x;
      v[k].y += src[k].y;
    }
  }
  const int64_t r = epar[e];
  double2 *ge = G + (size_t)(2 * s) * n, *ga = G + (size_t)(2 * s + 1) * n;
  ge[r] = v[0];
  ge[r + N] = v[1];
  ga[r] = v[2];
  ga[r + N] = v[3];
}

struct FfArgs {
  double w[kMaxQ];
  int F, nq, N;
  const double *qabs, *area, *sl, *mu, *cp;
  const int *hpar;
  const double2 *x;
  double4 *cur;  // [F*nq][3]: (J re, J im, M re, M im) per component, weighted by w A
  double *pos;   // [F*nq][3]
};

// Weighted surface currents at every quadrature point (ffields.f90:70-80):
// J = sum_q alpha_q f_q, M = sum_q beta_q f_q, times w_t A_n.
__global__ void ff_current_kernel(FfArgs a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.F * a.nq) return;
  const int f = j / a.nq, t = j % a.nq;
  const double *pt = a.qabs + (size_t)j * 3;
  const double An = a.area[f];
  const double w = a.w[t] * An;
  double J[3][2] = {{0, 0}, {0, 0}, {0, 0}}, M[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  for (int q = 0; q < 3; q++) {
    const int idx = a.hpar[3 * f + q];
    const double2 al = a.x[idx], be = a.x[idx + a.N];
    const double cc = a.sl[3 * f + q] / (2.0 * An);
    for (int i = 0; i < 3; i++) {
      const double fi = cc * (pt[i] - (a.cp[3 * f + i] + a.mu[9 * f + 3 * q + i]));
      J[i][0] += fi * al.x;
      J[i][1] += fi * al.y;
      M[i][0] += fi * be.x;
      M[i][1] += fi * be.y;
    }
  }
  for (int i = 0; i < 3; i++) {
    a.cur[(size_t)j * 3 + i] = make_double4(w * J[i][0], w * J[i][1], w * M[i][0], w * M[i][1]);
    a.pos[(size_t)j * 3 + i] = pt[i];
  }
}

constexpr int kFfThreads = 128;
constexpr int kFfTile = 128;

// One thread per direction, the points split over blockIdx.y: partial N and
// L radiation vectors (theta, phi components) by the phasor sum over the
// split's weighted quadrature points, into part[split][direction][4].
__global__ void __launch_bounds__(kFfThreads) ff_dir_kernel(int npts, int per_split, const double4 *cur,
                                                            const double *pos, int ntheta, int nphi, Z k,
                                                            double2 *part) {
  __shared__ double4 s_cur[kFfTile][3];
  __shared__ double s_pos[kFfTile][3];
  const int dirx = blockIdx.x * blockDim.x + threadIdx.x;
  const int p0 = blockIdx.y * per_split, p1 = min(npts, p0 + per_split);
  const int nd = ntheta * nphi;
  const int it = dirx % ntheta, ip = dirx / ntheta;
  const double theta = kPi * (double)it / (double)(ntheta - 1);
  const double phi = 2.0 * kPi * (double)ip / (double)(nphi - 1);
  double st, ct, sp, cp;
  sincos(theta, &st, &ct);
  sincos(phi, &sp, &cp);
  const double ux = st * cp, uy = st * sp, uz = ct;
  Z Nt = {0, 0}, Np = {0, 0}, Lt = {0, 0}, Lp = {0, 0};
  for (int base = p0; base < p1; base += kFfTile) {
    __syncthreads();
    for (int i = threadIdx.x; i < kFfTile; i += blockDim.x) {
      const int j = base + i;
      for (int c = 0; c < 3; c++) {
        s_cur[i][c] = (j < p1) ? cur[(size_t)j * 3 + c] : make_double4(0, 0, 0, 0);
        s_pos[i][c] = (j < p1) ? pos[(size_t)j * 3 + c] : 0.0;
      }
    }
    __syncthreads();
    const int cnt = min(kFfTile, p1 - base);
    for (int i = 0; i < cnt; i++) {
      const double s = s_pos[i][0] * ux + s_pos[i][1] * uy + s_pos[i][2] * uz;
      // phasor = exp(-i k s)
      double sn, cs;
      sincos(-k.re * s, &sn, &cs);
      const double am = exp(k.im * s);
      const Z ph = {am * cs, am * sn};
      const double4 jx = s_cur[i][0], jy = s_cur[i][1], jz = s_cur[i][2];
      // theta and phi projections
      const Z jt = {ct * cp * jx.x + ct * sp * jy.x - st * jz.x, ct * cp * jx.y + ct * sp * jy.y - st * jz.y};
      const Z jp = {-sp * jx.x + cp * jy.x, -sp * jx.y + cp * jy.y};
      const Z mt = {ct * cp * jx.z + ct * sp * jy.z - st * jz.z, ct * cp * jx.w + ct * sp * jy.w - st * jz.w};
      const Z mp = {-sp * jx.z + cp * jy.z, -sp * jx.w + cp * jy.w};
      Nt = zadd(Nt, zmul(jt, ph));
      Np = zadd(Np, zmul(jp, ph));
      Lt = zadd(Lt, zmul(mt, ph));
      Lp = zadd(Lp, zmul(mp, ph));
    }
  }
  if (dirx >= nd) return;
  double2 *o = part + ((size_t)blockIdx.y * nd + dirx) * 4;
  o[0] = make_double2(Nt.re, Nt.im);
  o[1] = make_double2(Np.re, Np.im);
  o[2] = make_double2(Lt.re, Lt.im);
  o[3] = make_double2(Lp.re, Lp.im);
}

// Thread per direction: the splits' partial radiation vectors summed in
// split order, then E_theta, E_phi at r = 1 m and the RCS.
__global__ void ff_finish_kernel(int nd, int nsplit, const double2 *part, int ntheta, Z k, Z ri, double *rcs) {
  const int dirx = blockIdx.x * blockDim.x + threadIdx.x;
  if (dirx >= nd) return;
  Z Nt = {0, 0}, Np = {0, 0}, Lt = {0, 0}, Lp = {0, 0};
  for (int sp = 0; sp < nsplit; sp++) {
    const double2 *o = part + ((size_t)sp * nd + dirx) * 4;
    Nt = zadd(Nt, Z{o[0].x, o[0].y});
    Np = zadd(Np, Z{o[1].x, o[1].y});
    Lt = zadd(Lt, Z{o[2].x, o[2].y});
    Lp = zadd(Lp, Z{o[3].x, o[3].y});
  }
  const int it = dirx % ntheta, ip = dirx / ntheta;
  // prefix = i k exp(i k r) / (4 pi r), r = 1
  const Z e = zexp_i(k, 1.0);
  const Z ik = {-k.im, k.re};
  Z prefix = zmul(ik, e);
  prefix = zscale(prefix, 1.0 / (4.0 * kPi * 1.0));
  // eta0 / ri
  const double rr = ri.re * ri.re + ri.im * ri.im;
  const Z er = {kEta0 * ri.re / rr, -kEta0 * ri.im / rr};
  const Z et = zmul(prefix, zadd(Lp, zmul(er, Nt)));
  const Z ep = zscale(zmul(prefix, zsub(Lt, zmul(er, Np))), -1.0);
  const double a = hypot(et.re, et.im), b = hypot(ep.re, ep.im);
  rcs[(size_t)it + (size_t)ip * ntheta] = a * a + b * b;
}

// ---- symmetry groups (nga > 1) ----

// The group as kernel argument: point actions J (row-major), det J and the
// field actions ef[g][r] (real for mirror groups).
struct GroupArg {
  int nga;
  double j[kMaxGroup][9];
  double detj[kMaxGroup];
  double ef[kMaxGroup][kMaxGroup];
};

__device__ __forceinline__ void jvec(const double *J, const double *v, double *o) {
  for (int i = 0; i < 3; i++) o[i] = J[3 * i] * v[0] + J[3 * i + 1] * v[1] + J[3 * i + 2] * v[2];
}
__device__ __forceinline__ void jtvec(const double *J, const double *v, double *o) {
  for (int i = 0; i < 3; i++) o[i] = J[i] * v[0] + J[3 + i] * v[1] + J[6 + i] * v[2];
}
__device__ __forceinline__ void jzvec(const double *J, const Z *v, Z *o) {
  for (int i = 0; i < 3; i++)
    o[i] = zadd(zadd(zscale(v[0], J[3 * i]), zscale(v[1], J[3 * i + 1])), zscale(v[2], J[3 * i + 2]));
}

// srcvec with a group (source.f90:136-247 with src_field_frags 250-315):
// thread per (face, source, representation r); the incident fields at the
// test point seen by every element g (at J^T r, mapped back by J, H with
// det J), projected on representation r with ef[g][r] / nga.
__global__ void rhs_half_sym_kernel(RhsArgs a, GroupArg G) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y, r = blockIdx.z;
  if (f >= a.F) return;
  const SrcDev S = a.src[s];
  Z Ie[3] = {{0, 0}, {0, 0}, {0, 0}}, Ih[3] = {{0, 0}, {0, 0}, {0, 0}};
  const double Am = a.area[f];
  for (int t = 0; t < a.nq; t++) {
    const double *pt = a.qabs + ((size_t)f * a.nq + t) * 3;
    Z ef[3] = {{0, 0}, {0, 0}, {0, 0}}, hf[3] = {{0, 0}, {0, 0}, {0, 0}};
    for (int g = 0; g < G.nga; g++) {
      double pp[3];
      jtvec(G.j[g], pt, pp);
      Z e[3], h[3], je[3], jh[3];
      src_fields(S, a.k, a.omega, pp, e, h);
      jzvec(G.j[g], e, je);
      jzvec(G.j[g], h, jh);
      const double ce = G.ef[g][r], ch = G.ef[g][r] * G.detj[g];
      for (int i = 0; i < 3; i++) {
        ef[i] = zadd(ef[i], zscale(je[i], ce));
        hf[i] = zadd(hf[i], zscale(jh[i], ch));
      }
    }
    for (int i = 0; i < 3; i++) {
      ef[i] = zscale(ef[i], 1.0 / G.nga);
      hf[i] = zscale(hf[i], 1.0 / G.nga);
    }
    const double w = a.w[t];
    for (int p = 0; p < 3; p++) {
      const double cc = a.sl[3 * f + p] / (2.0 * Am);
      double fm[3];
      for (int i = 0; i < 3; i++) fm[i] = cc * (pt[i] - (a.cp[3 * f + i] + a.mu[9 * f + 3 * p + i]));
      Z de = {0, 0}, dh = {0, 0};
      for (int i = 0; i < 3; i++) {
        de = zadd(de, zscale(ef[i], fm[i]));
        dh = zadd(dh, zscale(hf[i], fm[i]));
      }
      Ie[p] = zadd(Ie[p], zscale(de, w));
      Ih[p] = zadd(Ih[p], zscale(dh, w));
    }
  }
  double2 *o = a.half + ((((size_t)r * a.nsrc + s) * a.F + f) * 3) * 2;
  for (int p = 0; p < 3; p++) {
    o[2 * p] = make_double2(Ie[p].re * Am, Ie[p].im * Am);
    o[2 * p + 1] = make_double2(Ih[p].re * Am, Ih[p].im * Am);
  }
}

// cs_prtsrf with a group (cs.f90:14-104): per face and source, the Poynting
// fluxes on every image J(face) of the fragment, with the image's fields
// built from all representations' currents; x of representation r, source
// s at x + r xrep + s ldx.
__global__ void __launch_bounds__(256) cs_sym_kernel(CsArgs a, GroupArg G, int64_t xrep) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  double i1 = 0, i2 = 0;
  if (f < a.F) {
    const SrcDev S = a.src[s];
    const double An = a.area[f];
    const double *n0 = a.nrm + 3 * f;
    double int1 = 0, int2 = 0;
    for (int t = 0; t < a.nq; t++) {
      const double *qp = a.qabs + ((size_t)f * a.nq + t) * 3;
      double fn0[3][3];
      for (int p = 0; p < 3; p++) {
        const double cc = a.sl[3 * f + p] / (2.0 * An);
        double fr[3];
        for (int i = 0; i < 3; i++) fr[i] = cc * (qp[i] - (a.cp[3 * f + i] + a.mu[9 * f + 3 * p + i]));
        fn0[p][0] = n0[1] * fr[2] - n0[2] * fr[1];
        fn0[p][1] = n0[2] * fr[0] - n0[0] * fr[2];
        fn0[p][2] = n0[0] * fr[1] - n0[1] * fr[0];
      }
      for (int g = 0; g < G.nga; g++) {
        const double *J = G.j[g];
        double nor[3], pt[3], fn[3][3];
        jvec(J, n0, nor);
        jvec(J, qp, pt);
        for (int p = 0; p < 3; p++) jvec(J, fn0[p], fn[p]);
        Z Et[3] = {{0, 0}, {0, 0}, {0, 0}}, Ht[3] = {{0, 0}, {0, 0}, {0, 0}};
        for (int r = 0; r < G.nga; r++) {
          const double gae = G.ef[g][r];
          const double2 *x = a.x + (size_t)r * xrep + (size_t)s * a.ldx;
          for (int p = 0; p < 3; p++) {
            const int idx = a.hpar[3 * f + p];
            const Z xj = {x[idx].x, x[idx].y}, xm = {x[idx + a.N].x, x[idx + a.N].y};
            for (int i = 0; i < 3; i++) {
              Ht[i] = zsub(Ht[i], zscale(xj, fn[p][i] * gae * G.detj[g]));
              Et[i] = zadd(Et[i], zscale(xm, fn[p][i] * gae));
            }
          }
        }
        const Z nc[3] = {{nor[0], 0}, {nor[1], 0}, {nor[2], 0}};
        Z einc[3], hinc[3], t1[3], Eti[3], Hti[3], Ets[3], Hts[3], cr[3], cj[3];
        src_fields(S, a.k, a.omega, pt, einc, hinc);
        zcross(nc, hinc, t1);
        zcross(t1, nc, Hti);
        zcross(nc, einc, t1);
        zcross(t1, nc, Eti);
        for (int i = 0; i < 3; i++) {
          Hts[i] = zsub(Ht[i], Hti[i]);
          Ets[i] = zsub(Et[i], Eti[i]);
          cj[i] = zconj(Ht[i]);
        }
        zcross(Et, cj, cr);
        const double w = a.w[t];
        int1 += w * 0.5 * (cr[0].re * nor[0] + cr[1].re * nor[1] + cr[2].re * nor[2]);
        for (int i = 0; i < 3; i++) cj[i] = zconj(Hts[i]);
        zcross(Ets, cj, cr);
        int2 += w * 0.5 * (cr[0].re * nor[0] + cr[1].re * nor[1] + cr[2].re * nor[2]);
      }
    }
    i1 = int1 * An;
    i2 = int2 * An;
  }
  __shared__ double r1[256], r2[256];
  r1[threadIdx.x] = i1;
  r2[threadIdx.x] = i2;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      r1[threadIdx.x] += r1[threadIdx.x + w];
      r2[threadIdx.x] += r2[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    a.part[((size_t)s * gridDim.x + blockIdx.x) * 2] = r1[0];
    a.part[((size_t)s * gridDim.x + blockIdx.x) * 2 + 1] = r2[0];
  }
}

// far_fields with a group (ffields.f90:52-91): the weighted currents at the
// images J r of every quadrature point, J f times the representations'
// coefficients with ef[g][r] (M also with det J); point index
// (g F + f) nq + t.  x of representation r at x + r xrep.
__global__ void ff_current_sym_kernel(FfArgs a, GroupArg G, int64_t xrep) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int per = a.F * a.nq;
  if (j >= per * G.nga) return;
  const int g = j / per, ft = j % per, f = ft / a.nq, t = ft % a.nq;
  const double *pt = a.qabs + (size_t)ft * 3;
  const double An = a.area[f];
  const double w = a.w[t] * An;
  const double *J = G.j[g];
  double Jr[3][2] = {{0, 0}, {0, 0}, {0, 0}}, Mr[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  for (int q = 0; q < 3; q++) {
    const int idx = a.hpar[3 * f + q];
    const double cc = a.sl[3 * f + q] / (2.0 * An);
    double fq[3], jf[3];
    for (int i = 0; i < 3; i++) fq[i] = cc * (pt[i] - (a.cp[3 * f + i] + a.mu[9 * f + 3 * q + i]));
    jvec(J, fq, jf);
    for (int r = 0; r < G.nga; r++) {
      const double gae = G.ef[g][r];
      const double2 al = a.x[(size_t)r * xrep + idx], be = a.x[(size_t)r * xrep + idx + a.N];
      for (int i = 0; i < 3; i++) {
        Jr[i][0] += jf[i] * gae * al.x;
        Jr[i][1] += jf[i] * gae * al.y;
        Mr[i][0] += jf[i] * gae * G.detj[g] * be.x;
        Mr[i][1] += jf[i] * gae * G.detj[g] * be.y;
      }
    }
  }
  double pos[3];
  jvec(J, pt, pos);
  for (int i = 0; i < 3; i++) {
    a.cur[(size_t)j * 3 + i] = make_double4(w * Jr[i][0], w * Jr[i][1], w * Mr[i][0], w * Mr[i][1]);
    a.pos[(size_t)j * 3 + i] = pos[i];
  }
}

// field_mesh (nfpost.f90:167-262): the fields on the boundary of a domain
// at the centroid of every face of every image J_g(face), from the surface
// currents alone (the jump conditions): with the image normal n = J n0 and
// f' = J (n0 x f_q(cp)),
//   E = sum_r ef[g][r] sum_q (beta_q f' + n div f_q alpha_q / (i w eps)),
//   H = sum_r ef[g][r] det J sum_q (-alpha_q f' + n div f_q beta_q / (i w mu0)).
// Thread per (element g, face f), output index g F + f.
__global__ void surface_field_kernel(int F, int N, const double *cp, const double *nrm, const double *area,
                                     const double *sl, const double *mu, const int *hpar, const double2 *x,
                                     int64_t xrep, GroupArg G, Z iwe, Z iwm, double2 *E, double2 *H) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= F * G.nga) return;
  const int g = j / F, f = j % F;
  const double *J = G.j[g], *n0 = nrm + 3 * f;
  const double An = area[f];
  double nor[3];
  jvec(J, n0, nor);
  Z et[3] = {{0, 0}, {0, 0}, {0, 0}}, ht[3] = {{0, 0}, {0, 0}, {0, 0}}, en = {0, 0}, hn = {0, 0};
  for (int r = 0; r < G.nga; r++) {
    const double gae = G.ef[g][r];
    for (int q = 0; q < 3; q++) {
      const int idx = hpar[3 * f + q];
      const double2 al = x[(size_t)r * xrep + idx], be = x[(size_t)r * xrep + idx + N];
      // rwg at the centroid: sl/(2A) (cp - v_q) = -sl/(2A) mu_q
      const double cc = -sl[3 * f + q] / (2.0 * An);
      double fr[3], fn0[3], fn[3];
      for (int i = 0; i < 3; i++) fr[i] = cc * mu[9 * f + 3 * q + i];
      fn0[0] = n0[1] * fr[2] - n0[2] * fr[1];
      fn0[1] = n0[2] * fr[0] - n0[0] * fr[2];
      fn0[2] = n0[0] * fr[1] - n0[1] * fr[0];
      jvec(J, fn0, fn);
      const double dv = sl[3 * f + q] / An;
      for (int i = 0; i < 3; i++) {
        ht[i] = zsub(ht[i], zscale(Z{al.x, al.y}, fn[i] * gae * G.detj[g]));
        et[i] = zadd(et[i], zscale(Z{be.x, be.y}, fn[i] * gae));
      }
      hn = zadd(hn, zscale(Z{be.x, be.y}, dv * gae * G.detj[g]));
      en = zadd(en, zscale(Z{al.x, al.y}, dv * gae));
    }
  }
  // en / (i w eps), hn / (i w mu0)
  auto zdiv = [](Z a, Z b) -> Z {
    const double d = b.re * b.re + b.im * b.im;
    return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
  };
  en = zdiv(en, iwe);
  hn = zdiv(hn, iwm);
  for (int i = 0; i < 3; i++) {
    const Z e = zadd(et[i], zscale(en, nor[i])), h = zadd(ht[i], zscale(hn, nor[i]));
    E[(size_t)j * 3 + i] = make_double2(e.re, e.im);
    H[(size_t)j * 3 + i] = make_double2(h.re, h.im);
  }
}

GroupArg group_arg(const Ctx *c) {
  GroupArg G;
  std::memset(&G, 0, sizeof G);
  G.nga = c->nga;
  for (int g = 0; g < c->nga; g++) {
    for (int i = 0; i < 9; i++) G.j[g][i] = c->ga[g].j[i];
    G.detj[g] = c->ga[g].detj;
    for (int r = 0; r < c->nga; r++) G.ef[g][r] = c->ga[g].ef[r];
  }
  return G;
}

void make_src(const mom_src &s, SrcDev &d) {
  src_geometry(s, d.dir, d.pol);
  d.ph_re = s.phase_re;
  d.ph_im = s.phase_im;
  d.type = s.type;
}

int upload_sources(Ctx *c, int nsrc, const mom_src *src, SrcDev **out) {
  std::vector<SrcDev> h(nsrc);
  for (int i = 0; i < nsrc; i++) {
    if (src[i].type != MOM_SRC_PW && src[i].type != MOM_SRC_PW_ELLIPTIC && src[i].type != MOM_SRC_NONE)
      return fail(c, MOM_ERR_ARG, "unsupported source type (only pw, pw_elliptic and none)");
    make_src(src[i], h[i]);
  }
  const size_t bytes = sizeof(SrcDev) * nsrc;
  char *ws = (char *)c->ws;
  *out = reinterpret_cast<SrcDev *>(ws);
  MOM_CUDA(c, cudaMemcpyAsync(*out, h.data(), bytes, cudaMemcpyHostToDevice, c->stream));
  return MOM_OK;
}

}  // namespace

// srcvec for all sources on domain 1's mesh: B[:, s] (2N each, ld = n).
int rhs_build(Ctx *c, double omega, const double *ri1, int nsrc, const mom_src *src) {
  const DomDev &D = c->dom[0];
  const size_t src_bytes = ((sizeof(SrcDev) * nsrc + 255) / 256) * 256;
  const size_t half_bytes = sizeof(double2) * 6 * (size_t)D.F * nsrc * c->nga;
  MOM_TRY(ensure_buffer(c, &c->ws, &c->ws_bytes, src_bytes + half_bytes));
  SrcDev *dsrc = nullptr;
  MOM_TRY(upload_sources(c, nsrc, src, &dsrc));
  RhsArgs a;
  for (int i = 0; i < kMaxQ; i++) a.w[i] = c->qw[i];
  a.F = D.F;
  a.nq = c->nq;
  a.qabs = D.qabs;
  a.area = D.area;
  a.sl = D.sl;
  a.mu = D.mu;
  a.cp = D.cp;
  a.src = dsrc;
  a.nsrc = nsrc;
  a.k = {ri1[0] * omega / kC0, ri1[1] * omega / kC0};
  a.omega = omega;
  a.half = reinterpret_cast<double2 *>((char *)c->ws + src_bytes);
  MOM_CUDA(c, cudaMemsetAsync(c->B, 0, sizeof(double2) * c->n * nsrc * c->nga, c->stream));
  ProfScope ps(c, kProfPost);
  if (c->nga > 1) {
    // one block of right-hand sides per representation: B + r nsrc n
    rhs_half_sym_kernel<<<dim3((D.F + 127) / 128, nsrc, c->nga), 128, 0, c->stream>>>(a, group_arg(c));
    c->launches++;
    MOM_CUDA(c, cudaGetLastError());
    for (int r = 0; r < c->nga; r++) {
      double2 *Br = c->B + (size_t)r * nsrc * c->n;
      rhs_edge_kernel<<<dim3((D.Nd + 127) / 128, nsrc), 128, 0, c->stream>>>(
          D.Nd, D.F, c->N, c->n, D.eh, D.epar, a.half + (size_t)r * nsrc * D.F * 6, Br);
      c->launches++;
      MOM_CUDA(c, cudaGetLastError());
      MOM_TRY(apply_bc_rhs(c, r, Br, nsrc));
    }
    return MOM_OK;
  }
  rhs_half_kernel<<<dim3((D.F + 127) / 128, nsrc), 128, 0, c->stream>>>(a);
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  rhs_edge_kernel<<<dim3((D.Nd + 127) / 128, nsrc), 128, 0, c->stream>>>(D.Nd, D.F, c->N, c->n, D.eh, D.epar, a.half,
                                                                           c->B);
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  return MOM_OK;
}

int cross_sections(Ctx *c, int dom, double omega, const double *ri, int nsrc, const mom_src *src,
                   const double2 *xdev, int64_t ldx, double *csca, double *cabs, int64_t xrep) {
  const DomDev &D = c->dom[dom];
  const int blocks = (D.F + 255) / 256;
  const size_t src_bytes = ((sizeof(SrcDev) * nsrc + 255) / 256) * 256;
  const size_t part_bytes = sizeof(double) * 2 * (size_t)blocks * nsrc;
  MOM_TRY(ensure_buffer(c, &c->ws, &c->ws_bytes, src_bytes + part_bytes));
  SrcDev *dsrc = nullptr;
  MOM_TRY(upload_sources(c, nsrc, src, &dsrc));
  CsArgs a;
  for (int i = 0; i < kMaxQ; i++) a.w[i] = c->qw[i];
  a.F = D.F;
  a.nq = c->nq;
  a.N = c->N;
  a.qabs = D.qabs;
  a.area = D.area;
  a.sl = D.sl;
  a.mu = D.mu;
  a.cp = D.cp;
  a.nrm = D.nrm;
  a.hpar = D.hpar;
  a.src = dsrc;
  a.x = xdev;
  a.ldx = ldx;
  a.k = {ri[0] * omega / kC0, ri[1] * omega / kC0};
  a.omega = omega;
  a.part = reinterpret_cast<double *>((char *)c->ws + src_bytes);
  {
  ProfScope ps(c, kProfPost);
  if (c->nga > 1) cs_sym_kernel<<<dim3(blocks, nsrc), 256, 0, c->stream>>>(a, group_arg(c), xrep);
  else cs_kernel<<<dim3(blocks, nsrc), 256, 0, c->stream>>>(a);
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  }
  std::vector<double> part(2 * (size_t)blocks * nsrc);
  MOM_CUDA(c, cudaMemcpyAsync(part.data(), a.part, part_bytes, cudaMemcpyDeviceToHost, c->stream));
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  const double cc = 2.0 / (kEps0 * kC0 * ri[0]);  // cs.f90:38
  for (int s = 0; s < nsrc; s++) {
    double ab = 0, sc = 0;
    for (int b = 0; b < blocks; b++) {
      ab += part[((size_t)s * blocks + b) * 2];
      sc += part[((size_t)s * blocks + b) * 2 + 1];
    }
    cabs[s] = -cc * ab;
    csca[s] = cc * sc;
  }
  return MOM_OK;
}

// d sigma_ext / dx and d sigma_abs / dx on domain dom for nsrc sources into
// G (2 nsrc columns of length n, zero outside the domain's unknowns).
int cs_gradient(Ctx *c, int dom, double omega, const double *ri, int nsrc, const mom_src *src, const double2 *xdev,
                int64_t ldx, double2 *G) {
  const DomDev &D = c->dom[dom];
  const size_t src_bytes = ((sizeof(SrcDev) * nsrc + 255) / 256) * 256;
  const size_t half_bytes = sizeof(double2) * 12 * (size_t)D.F * nsrc;
  MOM_TRY(ensure_buffer(c, &c->ws, &c->ws_bytes, src_bytes + half_bytes));
  SrcDev *dsrc = nullptr;
  MOM_TRY(upload_sources(c, nsrc, src, &dsrc));
  CsArgs a;
  for (int i = 0; i < kMaxQ; i++) a.w[i] = c->qw[i];
  a.F = D.F;
  a.nq = c->nq;
  a.N = c->N;
  a.qabs = D.qabs;
  a.area = D.area;
  a.sl = D.sl;
  a.mu = D.mu;
  a.cp = D.cp;
  a.nrm = D.nrm;
  a.hpar = D.hpar;
  a.src = dsrc;
  a.x = xdev;
  a.ldx = ldx;
  a.k = {ri[0] * omega / kC0, ri[1] * omega / kC0};
  a.omega = omega;
  a.part = nullptr;
  double2 *half = reinterpret_cast<double2 *>((char *)c->ws + src_bytes);
  const double cc = 2.0 / (kEps0 * kC0 * ri[0]);  // cs.f90:38
  MOM_CUDA(c, cudaMemsetAsync(G, 0, sizeof(double2) * (size_t)c->n * 2 * nsrc, c->stream));
  cs_grad_half_kernel<<<dim3((D.F + 127) / 128, nsrc), 128, 0, c->stream>>>(a, cc, half);
  cs_grad_edge_kernel<<<dim3((D.Nd + 127) / 128, nsrc), 128, 0, c->stream>>>(D.Nd, D.F, c->N, c->n, D.eh, D.epar,
                                                                             half, G);
  c->launches += 2;
  MOM_CUDA(c, cudaGetLastError());
  return MOM_OK;
}

int far_field(Ctx *c, int dom, double omega, const double *ri, const double2 *xdev, int ntheta, int nphi,
              double *rcs, int64_t xrep) {
  const DomDev &D = c->dom[dom];
  const int npts = D.F * c->nq * c->nga;
  const int nd = ntheta * nphi;
  const size_t cur_bytes = sizeof(double4) * 3 * (size_t)npts;
  const size_t pos_bytes = sizeof(double) * 3 * (size_t)npts;
  const size_t out_bytes = ((sizeof(double) * (size_t)nd + 255) / 256) * 256;
  // split the points so that about 8 CTAs per SM are in flight, at least
  // 1024 points per split
  const int dir_ctas = (nd + kFfThreads - 1) / kFfThreads;
  int nsplit = std::max(1, (8 * c->nsm + dir_ctas - 1) / dir_ctas);
  nsplit = std::min(nsplit, std::max(1, npts / 1024));
  const int per_split = (npts + nsplit - 1) / nsplit;
  nsplit = (npts + per_split - 1) / per_split;
  const size_t part_bytes = sizeof(double2) * 4 * (size_t)nd * nsplit;
  MOM_TRY(ensure_buffer(c, &c->ws, &c->ws_bytes, cur_bytes + pos_bytes + out_bytes + part_bytes + 512));
  FfArgs a;
  for (int i = 0; i < kMaxQ; i++) a.w[i] = c->qw[i];
  a.F = D.F;
  a.nq = c->nq;
  a.N = c->N;
  a.qabs = D.qabs;
  a.area = D.area;
  a.sl = D.sl;
  a.mu = D.mu;
  a.cp = D.cp;
  a.hpar = D.hpar;
  a.x = xdev;
  a.cur = reinterpret_cast<double4 *>(c->ws);
  a.pos = reinterpret_cast<double *>((char *)c->ws + cur_bytes);
  double *dout = reinterpret_cast<double *>((char *)c->ws + cur_bytes + pos_bytes);
  double2 *dpart = reinterpret_cast<double2 *>((char *)c->ws + cur_bytes + pos_bytes + out_bytes);
  {
  ProfScope ps(c, kProfPost);
  if (c->nga > 1) ff_current_sym_kernel<<<(npts + 127) / 128, 128, 0, c->stream>>>(a, group_arg(c), xrep);
  else ff_current_kernel<<<(npts + 127) / 128, 128, 0, c->stream>>>(a);
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  const Z k = {ri[0] * omega / kC0, ri[1] * omega / kC0};
  const Z rz = {ri[0], ri[1]};
  ff_dir_kernel<<<dim3(dir_ctas, nsplit), kFfThreads, 0, c->stream>>>(npts, per_split, a.cur, a.pos, ntheta, nphi,
                                                                       k, dpart);
  ff_finish_kernel<<<(nd + 127) / 128, 128, 0, c->stream>>>(nd, nsplit, dpart, ntheta, k, rz, dout);
  c->launches += 2;
  MOM_CUDA(c, cudaGetLastError());
  }
  MOM_CUDA(c, cudaMemcpyAsync(rcs, dout, sizeof(double) * (size_t)nd, cudaMemcpyDeviceToHost, c->stream));
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  return MOM_OK;
}

// Surface fields (field_mesh) of domain dom for one solution column: x at
// xdev (representation r at xdev + r xrep), E, H device [nga F][3].
int surface_fields(Ctx *c, int dom, double omega, const double *ri, const double2 *xdev, int64_t xrep, double2 *E,
                   double2 *H) {
  const DomDev &D = c->dom[dom];
  const Z n = {ri[0], ri[1]};
  const Z eps = {kEps0 * (n.re * n.re - n.im * n.im), kEps0 * 2.0 * n.re * n.im};
  const Z iwe = {-omega * eps.im, omega * eps.re};  // i omega eps
  const Z iwm = {0.0, omega * kMu0};                // i omega mu0
  const int total = D.F * c->nga;
  ProfScope ps(c, kProfPost);
  surface_field_kernel<<<(total + 127) / 128, 128, 0, c->stream>>>(D.F, c->N, D.cp, D.nrm, D.area, D.sl, D.mu,
                                                                   D.hpar, xdev, xrep, group_arg(c), iwe, iwm, E, H);
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  return MOM_OK;
}

namespace {

// Thread per (point, source): E, H += the source's plane-wave fields at the point.
__global__ void incident_kernel(const SrcDev *src, Z k, double omega, const double *pts, int npts, double2 *E,
                                double2 *H) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (i >= npts) return;
  Z ef[3], hf[3];
  src_fields(src[s], k, omega, pts + 3 * i, ef, hf);
  double2 *e = E + ((size_t)s * npts + i) * 3, *h = H + ((size_t)s * npts + i) * 3;
  for (int c = 0; c < 3; c++) {
    e[c].x += ef[c].re;
    e[c].y += ef[c].im;
    h[c].x += hf[c].re;
    h[c].y += hf[c].im;
  }
}

}  // namespace

int add_incident_fields(Ctx *c, double omega, const double *ri, int nsrc, const mom_src *src, int npts,
                        const double *pts, double2 *E, double2 *H, void *srcbuf) {
  static_assert(sizeof(SrcDev) <= 128, "source record larger than the caller's scratch");
  std::vector<SrcDev> h(nsrc);
  for (int i = 0; i < nsrc; i++) {
    if (src[i].type != MOM_SRC_PW && src[i].type != MOM_SRC_PW_ELLIPTIC && src[i].type != MOM_SRC_NONE)
      return fail(c, MOM_ERR_ARG, "unsupported source type (only pw, pw_elliptic and none)");
    make_src(src[i], h[i]);
  }
  SrcDev *d = reinterpret_cast<SrcDev *>(srcbuf);
  MOM_CUDA(c, cudaMemcpyAsync(d, h.data(), sizeof(SrcDev) * nsrc, cudaMemcpyHostToDevice, c->stream));
  const Z k = {ri[0] * omega / kC0, ri[1] * omega / kC0};
  incident_kernel<<<dim3((npts + 127) / 128, nsrc), 128, 0, c->stream>>>(d, k, omega, pts, npts, E, H);
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  return MOM_OK;
}

}  // namespace mom
