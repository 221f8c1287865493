// Adjoint gradients of the cross sections (no counterpart in the reference).
//
// Included once, at the end of assemble.cu, so that the face-pair templates
// (pair_moments, static_terms) and the quadrature in constant memory are
// shared with the matrix assembly.
//
// sigma is a real function of the solution x of A x = q.  With
// G = d sigma / dx in the sense d sigma = Re(G^T dx) (from the cs_prtsrf
// formula, cs.f90:14-104) and the adjoint currents lambda, A^T lambda = G,
//   d sigma = Re(lambda^T (dq - dA x)) + (explicit geometry term of sigma).
// dA is never stored: the kernels below re-evaluate every face-pair block
// in forward-mode dual arithmetic (value, directional derivative) and
// contract its derivative with lambda and x on the fly.  Directions:
//   permittivity eps of one interior domain (A is holomorphic in eps:
//     k = sqrt(eps) k0, c2 ~ 1/eps, Zsi ~ eps), derivative along Re(eps);
//     d/dIm(eps) = i d/dRe(eps);
//   one coordinate of one mesh vertex: the face geometry, quadrature
//     points, RWG functions and the closed-form singular integrals of the
//     faces that touch the vertex.
// The near-pair classification (sysmat.f90:233-260) is held fixed at the
// unperturbed geometry.

namespace {

// ---- forward-mode dual numbers ------------------------------------------

struct Dual {
  double v, d;
  __host__ __device__ Dual() {}
  __host__ __device__ Dual(double a) : v(a), d(0.0) {}
  __host__ __device__ Dual(double a, double b) : v(a), d(b) {}
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  const double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
__device__ __forceinline__ Dual operator+(Dual a, double b) { return Dual(a.v + b, a.d); }
__device__ __forceinline__ Dual operator+(double a, Dual b) { return Dual(a + b.v, b.d); }
__device__ __forceinline__ Dual operator-(Dual a, double b) { return Dual(a.v - b, a.d); }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return Dual(a - b.v, -b.d); }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return Dual(a.v * b, a.d * b); }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return Dual(a * b.v, a * b.d); }
__device__ __forceinline__ Dual operator/(Dual a, double b) { return Dual(a.v / b, a.d / b); }
__device__ __forceinline__ Dual operator/(double a, Dual b) {
  const double q = a / b.v;
  return Dual(q, -q * b.d / b.v);
}
__device__ __forceinline__ Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__device__ __forceinline__ Dual &operator+=(Dual &a, Dual b) {
  a.v += b.v;
  a.d += b.d;
  return a;
}
__device__ __forceinline__ Dual &operator-=(Dual &a, Dual b) {
  a.v -= b.v;
  a.d -= b.d;
  return a;
}
__device__ __forceinline__ bool operator>(Dual a, Dual b) { return a.v > b.v; }
__device__ __forceinline__ bool operator>(Dual a, double b) { return a.v > b; }
__device__ __forceinline__ bool operator<(Dual a, double b) { return a.v < b; }
__device__ __forceinline__ bool operator==(Dual a, double b) { return a.v == b; }
__device__ __forceinline__ Dual sqrt(Dual a) {
  const double s = ::sqrt(a.v);
  return Dual(s, a.d / (2.0 * s));
}
__device__ __forceinline__ Dual frsqrt(Dual a) {
  const double r = ::rsqrt(a.v);
  return Dual(r, -0.5 * a.d * r * r * r);
}
__device__ __forceinline__ Dual fexp(Dual a) {
  const double e = ::exp(a.v);
  return Dual(e, e * a.d);
}
__device__ __forceinline__ void fsincos(Dual a, Dual *s, Dual *c) {
  double sn, cs;
  ::sincos(a.v, &sn, &cs);
  *s = Dual(sn, cs * a.d);
  *c = Dual(cs, -sn * a.d);
}
__device__ __forceinline__ Dual log(Dual a) { return Dual(::log(a.v), a.d / a.v); }
__device__ __forceinline__ Dual fabs(Dual a) { return a.v < 0.0 ? -a : a; }
__device__ __forceinline__ Dual atan2(Dual y, Dual x) {
  const double r2 = x.v * x.v + y.v * y.v;
  return Dual(::atan2(y.v, x.v), (x.v * y.d - y.v * x.d) / r2);
}

// complex helpers on Cx<S>
template <typename S>
__device__ __forceinline__ Cx<S> cxm(Cx<S> a, Cx<S> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename S>
__device__ __forceinline__ Cx<S> cxa(Cx<S> a, Cx<S> b) {
  return {a.re + b.re, a.im + b.im};
}
template <typename S>
__device__ __forceinline__ Cx<S> cxs(Cx<S> a, Cx<S> b) {
  return {a.re - b.re, a.im - b.im};
}
template <typename S>
__device__ __forceinline__ Cx<S> cxr(Cx<S> a, S r) {
  return {a.re * r, a.im * r};
}
// derivative part of a dual complex value
__device__ __forceinline__ Cd dpart(Cx<Dual> a) { return {a.re.d, a.im.d}; }

// ---- face geometry from the vertices (compute_basis_data, mesh.f90:1265) --

struct AdjTopo {
  int F, N;
  const double *nodes;  // [nnodes][3] domain submesh nodes
  const int *fnode;     // [F][3] vertices of the face
  const int *fea, *feb; // [F][3] end points of local edge e
  const int *fbn;       // [F][3] free vertex of local edge e
  const double *fsign;  // [F][3] +1 / -1: the face is the + / - face of edge e
  const int *hpar;      // [F][3] global edge index of local edge e
  const unsigned *near_bits;  // [F*F] bits: pair (m, n) is near
};

template <typename S, int NQ>
struct FaceAll {
  FaceGeoT<S> g;
  S area, cp[3], sl[3], bn[3][3], mu[3][3];
  S qa[NQ][3], qr[NQ][3];  // quadrature points, absolute and minus the centroid
};

template <typename S>
__device__ __forceinline__ void cross3(const S *a, const S *b, S *r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}

// Geometry of face f with the derivative seeded on coordinate scoord of node
// snode (snode < 0: no geometric seed).
template <int NQ>
__device__ void face_build(const AdjTopo &t, int f, int snode, int scoord, FaceAll<Dual, NQ> &o) {
  auto node = [&](int id, int k) { return Dual(t.nodes[3 * id + k], (id == snode && k == scoord) ? 1.0 : 0.0); };
  Dual p[3][3];
#pragma unroll
  for (int v = 0; v < 3; v++)
#pragma unroll
    for (int i = 0; i < 3; i++) p[v][i] = node(t.fnode[3 * f + v], i);
  Dual a[3], cc[3], b[3], p21[3], p32[3], p13[3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    a[i] = p[1][i] - p[0][i];
    cc[i] = p[2][i] - p[0][i];
    p21[i] = p[1][i] - p[0][i];
    p32[i] = p[2][i] - p[1][i];
    p13[i] = p[0][i] - p[2][i];
  }
  cross3(a, cc, b);
  const Dual nb = norm3(b);
#pragma unroll
  for (int i = 0; i < 3; i++) o.g.n[i] = b[i] / nb;
  const Dual l21 = norm3(p21), l32 = norm3(p32), l13 = norm3(p13);
#pragma unroll
  for (int i = 0; i < 3; i++) {
    o.g.s[0][i] = p21[i] / l21;
    o.g.s[1][i] = p32[i] / l32;
    o.g.s[2][i] = p13[i] / l13;
  }
#pragma unroll
  for (int e = 0; e < 3; e++) {
    cross3(o.g.s[e], o.g.n, o.g.mm[e]);
    const Dual l = norm3(o.g.mm[e]);
#pragma unroll
    for (int i = 0; i < 3; i++) o.g.mm[e][i] = o.g.mm[e][i] / l;
  }
  Dual mp13[3] = {-p13[0], -p13[1], -p13[2]}, cr[3];
  cross3(mp13, p32, cr);
  o.area = 0.5 * norm3(cr);
#pragma unroll
  for (int i = 0; i < 3; i++) o.cp[i] = (p[0][i] + p[1][i] + p[2][i]) / 3.0;
#pragma unroll
  for (int v = 0; v < 3; v++)
#pragma unroll
    for (int i = 0; i < 3; i++) o.g.v[v][i] = p[v][i];
  for (int q = 0; q < NQ; q++)
#pragma unroll
    for (int i = 0; i < 3; i++) {
      o.qa[q][i] = c_qn[q][2] * p[0][i] + c_qn[q][0] * p[1][i] + c_qn[q][1] * p[2][i];
      o.qr[q][i] = o.qa[q][i] - o.cp[i];
    }
#pragma unroll
  for (int e = 0; e < 3; e++) {
    const int ea = t.fea[3 * f + e], eb = t.feb[3 * f + e], bn = t.fbn[3 * f + e];
    Dual dl[3];
#pragma unroll
    for (int i = 0; i < 3; i++) dl[i] = node(ea, i) - node(eb, i);
    o.sl[e] = t.fsign[3 * f + e] * norm3(dl);
#pragma unroll
    for (int i = 0; i < 3; i++) {
      o.bn[e][i] = node(bn, i);
      o.mu[e][i] = o.bn[e][i] - o.cp[i];
    }
  }
}

// blocks_from_moments in the scalar type S, with the test face's geometry in
// type GM, the source face's in GN and the centroid offset in GD (S by
// default).
template <typename S, typename GM = S, typename GN = GM, typename GD = GM>
__device__ void blocks_generic(const Moments<S> &M, const GM mu[3][3], const GN nu[3][3], const GM slp[3],
                               const GN slq[3], const GD d[3], Cx<S> fD, Cx<S> fH, double fK, bool self, Cx<S> *Sb,
                               Cx<S> *Kb) {
  Cx<S> KBv[3], KDmF[3];
  KBv[0] = {d[1] * M.KF[2].re - d[2] * M.KF[1].re + M.KE[0].re, d[1] * M.KF[2].im - d[2] * M.KF[1].im + M.KE[0].im};
  KBv[1] = {d[2] * M.KF[0].re - d[0] * M.KF[2].re + M.KE[1].re, d[2] * M.KF[0].im - d[0] * M.KF[2].im + M.KE[1].im};
  KBv[2] = {d[0] * M.KF[1].re - d[1] * M.KF[0].re + M.KE[2].re, d[0] * M.KF[1].im - d[1] * M.KF[0].im + M.KE[2].im};
#pragma unroll
  for (int i = 0; i < 3; i++)
    KDmF[i] = {d[i] * M.KG.re + M.KC[i].re - M.KF[i].re, d[i] * M.KG.im + M.KC[i].im - M.KF[i].im};
  const Cx<S> dKE = {d[0] * M.KE[0].re + d[1] * M.KE[1].re + d[2] * M.KE[2].re,
                     d[0] * M.KE[0].im + d[1] * M.KE[1].im + d[2] * M.KE[2].im};
  Cx<S> beta[3], bq[3], cq[3];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const GN *v = nu[q];
    beta[q] = {v[0] * M.TB[0].re + v[1] * M.TB[1].re + v[2] * M.TB[2].re,
               v[0] * M.TB[0].im + v[1] * M.TB[1].im + v[2] * M.TB[2].im};
    const auto dn0 = d[1] * v[2] - d[2] * v[1], dn1 = d[2] * v[0] - d[0] * v[2], dn2 = d[0] * v[1] - d[1] * v[0];
    bq[q] = {dn0 * M.KC[0].re + dn1 * M.KC[1].re + dn2 * M.KC[2].re,
             dn0 * M.KC[0].im + dn1 * M.KC[1].im + dn2 * M.KC[2].im};
    cq[q] = {v[0] * M.KE[0].re + v[1] * M.KE[1].re + v[2] * M.KE[2].re,
             v[0] * M.KE[0].im + v[1] * M.KE[1].im + v[2] * M.KE[2].im};
  }
#pragma unroll
  for (int p = 0; p < 3; p++) {
    const GM *u = mu[p];
    const Cx<S> alpha = {u[0] * M.TC[0].re + u[1] * M.TC[1].re + u[2] * M.TC[2].re,
                         u[0] * M.TC[0].im + u[1] * M.TC[1].im + u[2] * M.TC[2].im};
    const Cx<S> ap = {u[0] * KBv[0].re + u[1] * KBv[1].re + u[2] * KBv[2].re,
                      u[0] * KBv[0].im + u[1] * KBv[1].im + u[2] * KBv[2].im};
    const Cx<S> Z[3] = {{u[1] * KDmF[2].re - u[2] * KDmF[1].re, u[1] * KDmF[2].im - u[2] * KDmF[1].im},
                        {u[2] * KDmF[0].re - u[0] * KDmF[2].re, u[2] * KDmF[0].im - u[0] * KDmF[2].im},
                        {u[0] * KDmF[1].re - u[1] * KDmF[0].re, u[0] * KDmF[1].im - u[1] * KDmF[0].im}};
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const GN *v = nu[q];
      const auto uv = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
      const auto ss = slp[p] * slq[q];
      const Cx<S> cD = {M.TA.re - beta[q].re - alpha.re + uv * M.TD.re, M.TA.im - beta[q].im - alpha.im + uv * M.TD.im};
      const Cx<S> s12 = cxa(cxm(fD, cD), cxm(fH, M.TD));
      Sb[3 * p + q] = cxr(s12, S(ss));
      Cx<S> kv = {S(0.0), S(0.0)};
      if (!self) {
        const Cx<S> cK = {-dKE.re - ap.re - bq[q].re + cq[q].re + v[0] * Z[0].re + v[1] * Z[1].re + v[2] * Z[2].re,
                          -dKE.im - ap.im - bq[q].im + cq[q].im + v[0] * Z[0].im + v[1] * Z[1].im + v[2] * Z[2].im};
        kv = cxr(cK, S(ss * fK));
      }
      Kb[3 * p + q] = kv;
    }
  }
}

// Blocks S = D + H and K of the face pair (test m, source n) in FP64 dual
// arithmetic: regular G for far pairs; smoothed G plus the closed-form
// terms (1/(4 pi)) X_m1 - (k^2/(8 pi)) X_1 for near pairs, as the matrix
// assembly does.
template <int NQ>
__device__ void pair_eval(const FaceAll<Dual, NQ> &fm, const FaceAll<Dual, NQ> &fn, bool near, bool self, Dual kr,
                          Dual ki, Cx<Dual> c1, Cx<Dual> c2, Cx<Dual> *Sb, Cx<Dual> *Kb) {
  Dual d[3];
#pragma unroll
  for (int i = 0; i < 3; i++) d[i] = fm.cp[i] - fn.cp[i];
  Moments<Dual> M;
  if (near) pair_moments<Dual, NQ, true>(&fm.qr[0][0], &fn.qr[0][0], 1, d, kr, ki, M);
  else pair_moments<Dual, NQ, false>(&fm.qr[0][0], &fn.qr[0][0], 1, d, kr, ki, M);
  const Cx<Dual> fD = {c1.re * (kOofpi / 4.0), c1.im * (kOofpi / 4.0)};
  const Cx<Dual> fH = {c2.re * kOofpi, c2.im * kOofpi};
  blocks_generic<Dual>(M, fm.mu, fn.mu, fm.sl, fn.sl, d, fD, fH, kOofpi / 4.0, self, Sb, Kb);
  if (!near) return;
  Dual st[6][9];
  static_terms<Dual, NQ>(fm.qa, fm.area, fm.sl, fm.bn, fn.g, fn.area, fn.sl, fn.bn, self, st);
  const double f4 = 1.0 / (4.0 * kPi);
  const Cx<Dual> f8 = {(kr * kr - ki * ki) / (8.0 * kPi), (2.0 * kr * ki) / (8.0 * kPi)};
#pragma unroll
  for (int i = 0; i < 9; i++) {
    const Cx<Dual> dterm = {f4 * st[0][i] - f8.re * st[1][i], -f8.im * st[1][i]};
    const Cx<Dual> hterm = {f4 * st[2][i] - f8.re * st[3][i], -f8.im * st[3][i]};
    const Cx<Dual> kterm = {f4 * st[4][i] - f8.re * st[5][i], -f8.im * st[5][i]};
    Sb[i] = cxa(Sb[i], cxa(cxm(c1, dterm), cxm(c2, hterm)));
    Kb[i] = cxa(Kb[i], kterm);
  }
}

constexpr int kAdjThreads = 64;
constexpr int kAdjMaxObj = 8;

struct AdjPairArgs {
  AdjTopo t;
  int64_t n;       // matrix order (leading dimension of the objective vectors)
  Dual kr, ki;     // k of the domain (derivative seeded in eps mode)
  Cx<Dual> c1, c2, Zsi;
  int mode;        // 0: eps, item = test face; 1: vertex, item = 3 * incidence + coordinate
  const int *inc_node, *inc_face;
  int R;           // objectives (lambda_o, x_o) pairs; 0: dense W
  const double2 *lam, *xv;  // [R][n]
  const double2 *W;         // [n][n] column-major, W(r, c) = sum_o lambda_o[r] x_o[c]
  double *part;    // [gridDim.y][gridDim.x][max(R,1)][2]
  // the assembly's FP64 geometry (partner faces that carry no derivative)
  const double *qrel, *cp, *mu, *sl;
};

__device__ __forceinline__ Cd cdm(Cd a, double2 b) { return {a.re * b.x - a.im * b.y, a.re * b.y + a.im * b.x}; }

// Adds the derivative blocks Sb, Kb of the pair (test m, source n) contracted
// with the objectives into acc (the loop of pair_contract).
__device__ __forceinline__ void contract_blocks(const AdjPairArgs &a, int m, int n, const Cx<Dual> *Sb,
                                                const Cx<Dual> *Kb, Cd *acc) {
  const int64_t N = a.t.N, ld = a.n;
#pragma unroll 1
  for (int p = 0; p < 3; p++) {
    const int64_t r = a.t.hpar[3 * m + p];
#pragma unroll 1
    for (int q = 0; q < 3; q++) {
      const int64_t cI = a.t.hpar[3 * n + q];
      const Cd dS = dpart(Sb[3 * p + q]), dZ = dpart(cxm(a.Zsi, Sb[3 * p + q])), dK = dpart(Kb[3 * p + q]);
      for (int o = 0; o < a.R; o++) {
        const double2 *l = a.lam + (size_t)o * ld, *x = a.xv + (size_t)o * ld;
        const double2 lr = l[r], lrN = l[r + N], xc = x[cI], xcN = x[cI + N];
        const double2 jj = make_double2(lr.x * xc.x - lr.y * xc.y, lr.x * xc.y + lr.y * xc.x);
        const double2 mm = make_double2(lrN.x * xcN.x - lrN.y * xcN.y, lrN.x * xcN.y + lrN.y * xcN.x);
        const double2 mj = make_double2(lrN.x * xc.x - lrN.y * xc.y, lrN.x * xc.y + lrN.y * xc.x);
        const double2 jm = make_double2(lr.x * xcN.x - lr.y * xcN.y, lr.x * xcN.y + lr.y * xcN.x);
        const Cd t1 = cdm(dS, jj), t2 = cdm(dZ, mm), t3 = cdm(dK, make_double2(mj.x - jm.x, mj.y - jm.y));
        acc[o].re += t1.re + t2.re + t3.re;
        acc[o].im += t1.im + t2.im + t3.im;
      }
    }
  }
}

// Adds d/dp (lambda_o^T A x_o) of pair (m, n) into acc[o] for the four
// PMCHWT blocks [JJ] S, [MM] Zsi S, [MJ] K, [JM] -K (sysmat.f90:70-99).
template <int NQ>
__device__ void pair_contract(const AdjPairArgs &a, int m, int n, const FaceAll<Dual, NQ> &fm,
                              const FaceAll<Dual, NQ> &fn, Cd *acc) {
  const int64_t bit = (int64_t)m * a.t.F + n;
  const bool near = (a.t.near_bits[bit >> 5] >> (bit & 31)) & 1u;
  Cx<Dual> Sb[9], Kb[9];
  pair_eval<NQ>(fm, fn, near, m == n, a.kr, a.ki, a.c1, a.c2, Sb, Kb);
  const int64_t N = a.t.N, ld = a.n;
#pragma unroll 1
  for (int p = 0; p < 3; p++) {
    const int64_t r = a.t.hpar[3 * m + p];
#pragma unroll 1
    for (int q = 0; q < 3; q++) {
      const int64_t cI = a.t.hpar[3 * n + q];
      const Cd dS = dpart(Sb[3 * p + q]), dZ = dpart(cxm(a.Zsi, Sb[3 * p + q])), dK = dpart(Kb[3 * p + q]);
      if (a.R == 0) {
        const double2 wjj = a.W[r + cI * ld], wmm = a.W[(r + N) + (cI + N) * ld];
        const double2 wmj = a.W[(r + N) + cI * ld], wjm = a.W[r + (cI + N) * ld];
        const Cd t1 = cdm(dS, wjj), t2 = cdm(dZ, wmm), t3 = cdm(dK, make_double2(wmj.x - wjm.x, wmj.y - wjm.y));
        acc[0].re += t1.re + t2.re + t3.re;
        acc[0].im += t1.im + t2.im + t3.im;
      } else {
        for (int o = 0; o < a.R; o++) {
          const double2 *l = a.lam + (size_t)o * ld, *x = a.xv + (size_t)o * ld;
          const double2 lr = l[r], lrN = l[r + N], xc = x[cI], xcN = x[cI + N];
          const double2 jj = make_double2(lr.x * xc.x - lr.y * xc.y, lr.x * xc.y + lr.y * xc.x);
          const double2 mm = make_double2(lrN.x * xcN.x - lrN.y * xcN.y, lrN.x * xcN.y + lrN.y * xcN.x);
          const double2 mj = make_double2(lrN.x * xc.x - lrN.y * xc.y, lrN.x * xc.y + lrN.y * xc.x);
          const double2 jm = make_double2(lr.x * xcN.x - lr.y * xcN.y, lr.x * xcN.y + lr.y * xcN.x);
          const Cd t1 = cdm(dS, jj), t2 = cdm(dZ, mm), t3 = cdm(dK, make_double2(mj.x - jm.x, mj.y - jm.y));
          acc[o].re += t1.re + t2.re + t3.re;
          acc[o].im += t1.im + t2.im + t3.im;
        }
      }
    }
  }
}

// One thread per partner face x: eps mode evaluates (f, x); vertex mode
// evaluates (f, x) and, when x does not touch the seeded vertex, (x, f),
// so that every pair touching the vertex is taken once.
template <int NQ>
__global__ void __launch_bounds__(kAdjThreads) adj_pair_kernel(AdjPairArgs a) {
  const int item = blockIdx.y;
  int f, snode = -1, scoord = 0;
  if (a.mode == 0) {
    f = item;
  } else {
    f = a.inc_face[item / 3];
    snode = a.inc_node[item / 3];
    scoord = item % 3;
  }
  const int x = blockIdx.x * kAdjThreads + threadIdx.x;
  Cd acc[kAdjMaxObj];
#pragma unroll
  for (int o = 0; o < kAdjMaxObj; o++) acc[o] = {0.0, 0.0};
  if (x < a.t.F) {
    FaceAll<Dual, NQ> ff, fx;
    face_build<NQ>(a.t, f, snode, scoord, ff);
    face_build<NQ>(a.t, x, snode, scoord, fx);
    pair_contract<NQ>(a, f, x, ff, fx, acc);
    if (a.mode == 1 && a.t.fnode[3 * x] != snode && a.t.fnode[3 * x + 1] != snode && a.t.fnode[3 * x + 2] != snode)
      pair_contract<NQ>(a, x, f, fx, ff, acc);
  }
  // deterministic block reduction per objective
  __shared__ double red[kAdjThreads][2];
  const int nobj = a.R == 0 ? 1 : a.R;
  for (int o = 0; o < nobj; o++) {
    red[threadIdx.x][0] = acc[o].re;
    red[threadIdx.x][1] = acc[o].im;
    __syncthreads();
    for (int w = kAdjThreads / 2; w > 0; w >>= 1) {
      if (threadIdx.x < w) {
        red[threadIdx.x][0] += red[threadIdx.x + w][0];
        red[threadIdx.x][1] += red[threadIdx.x + w][1];
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      double *out = a.part + (((size_t)blockIdx.y * gridDim.x + blockIdx.x) * nobj + o) * 2;
      out[0] = red[0][0];
      out[1] = red[0][1];
    }
    __syncthreads();
  }
}

// ---- vertex mode with one dual face ---------------------------------------
//
// Item (vertex v, incident face f, axis): only the faces that touch v carry a
// derivative.  The CTA builds f's dual record once in shared memory; a
// partner x that does not touch v is read as FP64 from the assembly's arrays
// and the far pairs (f, x) and (x, f) run with one dual and one plain face.
// Partners that touch v, and near pairs (closed-form singular terms), take
// the all-dual evaluation of adj_pair_kernel.  Same pairs, same contraction
// and the same deterministic block sums.

template <int NQ>
__device__ __noinline__ void vertex_pairs_dual(const AdjPairArgs &a, int f, int x, int snode, int scoord,
                                               const FaceAll<Dual, NQ> &ff, bool touches, Cd *acc) {
  FaceAll<Dual, NQ> fx;
  face_build<NQ>(a.t, x, snode, scoord, fx);
  pair_contract<NQ>(a, f, x, ff, fx, acc);
  if (!touches) pair_contract<NQ>(a, x, f, fx, ff, acc);
}

template <int NQ>
__global__ void __launch_bounds__(kAdjThreads) adj_vertex_kernel(AdjPairArgs a) {
  // the seeded face's dual record, built once per CTA (raw storage: Dual has
  // a constructor, which a __shared__ object may not run)
  __shared__ __align__(16) unsigned char ff_raw[sizeof(FaceAll<Dual, NQ>)];
  FaceAll<Dual, NQ> &ff = *reinterpret_cast<FaceAll<Dual, NQ> *>(ff_raw);
  const int item = blockIdx.y;
  const int f = a.inc_face[item / 3], snode = a.inc_node[item / 3], scoord = item % 3;
  if (threadIdx.x == 0) face_build<NQ>(a.t, f, snode, scoord, ff);
  __syncthreads();
  const int x = blockIdx.x * kAdjThreads + threadIdx.x;
  Cd acc[kAdjMaxObj];
#pragma unroll
  for (int o = 0; o < kAdjMaxObj; o++) acc[o] = {0.0, 0.0};
  if (x < a.t.F) {
    const bool touches = a.t.fnode[3 * x] == snode || a.t.fnode[3 * x + 1] == snode || a.t.fnode[3 * x + 2] == snode;
    const int64_t b1 = (int64_t)f * a.t.F + x, b2 = (int64_t)x * a.t.F + f;
    const bool near = ((a.t.near_bits[b1 >> 5] >> (b1 & 31)) & 1u) || ((a.t.near_bits[b2 >> 5] >> (b2 & 31)) & 1u);
    if (touches || near) {
      vertex_pairs_dual<NQ>(a, f, x, snode, scoord, ff, touches, acc);
    } else {
      const double *qx = a.qrel + (size_t)x * NQ * 3;
      const double *mux = a.mu + 9 * (size_t)x, *slx = a.sl + 3 * (size_t)x;
      const Cx<Dual> fD = {a.c1.re * (kOofpi / 4.0), a.c1.im * (kOofpi / 4.0)};
      const Cx<Dual> fH = {a.c2.re * kOofpi, a.c2.im * kOofpi};
      Dual d[3];
      Cx<Dual> Sb[9], Kb[9];
      Moments<Dual> M;
      // (f, x): dual test face, plain source
#pragma unroll
      for (int i = 0; i < 3; i++) d[i] = ff.cp[i] - a.cp[3 * x + i];
      pair_moments<Dual, NQ, false, false, Dual, double, Dual>(&ff.qr[0][0], qx, 1, d, a.kr, a.ki, M);
      blocks_generic<Dual, Dual, double, Dual>(M, ff.mu, reinterpret_cast<const double(*)[3]>(mux), ff.sl, slx, d, fD,
                                               fH, kOofpi / 4.0, false, Sb, Kb);
      contract_blocks(a, f, x, Sb, Kb, acc);
      // (x, f): plain test face, dual source; the same point pairs, so its
      // moments are those of (f, x) with the faces' roles exchanged
#pragma unroll
      for (int i = 0; i < 3; i++) d[i] = -d[i];
      exchange_roles(M);
      blocks_generic<Dual, double, Dual, Dual>(M, reinterpret_cast<const double(*)[3]>(mux), ff.mu, slx, ff.sl, d, fD,
                                               fH, kOofpi / 4.0, false, Sb, Kb);
      contract_blocks(a, x, f, Sb, Kb, acc);
    }
  }
  __shared__ double red[kAdjThreads][2];
  for (int o = 0; o < a.R; o++) {
    red[threadIdx.x][0] = acc[o].re;
    red[threadIdx.x][1] = acc[o].im;
    __syncthreads();
    for (int w = kAdjThreads / 2; w > 0; w >>= 1) {
      if (threadIdx.x < w) {
        red[threadIdx.x][0] += red[threadIdx.x + w][0];
        red[threadIdx.x][1] += red[threadIdx.x + w][1];
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      double *out = a.part + (((size_t)blockIdx.y * gridDim.x + blockIdx.x) * a.R + o) * 2;
      out[0] = red[0][0];
      out[1] = red[0][1];
    }
    __syncthreads();
  }
}

template <int NQ>
void launch_adj_vertex(const dim3 &grid, cudaStream_t s, const AdjPairArgs &a) {
  adj_vertex_kernel<NQ><<<grid, kAdjThreads, 0, s>>>(a);
}

// ---- permittivity mode on plain geometry ---------------------------------
//
// The permittivity moves only k, c2 and Zsi: the geometry carries no
// derivative, so the face data come as FP64 from the assembly's arrays and
// only the values that depend on k are dual numbers.  Same pairs, same
// contraction and the same deterministic block sums as adj_pair_kernel in
// eps mode, without the dual face records (which spill at 255 registers).

struct AdjEpsArgs {
  int F;
  int64_t n, N;
  const double *qrel, *qabs, *cp, *area, *mu, *sl, *bn;  // assembly geometry; bn: [F][3][3] free vertices
  const FaceGeo *geo;  // [F] vertices, edge vectors and normals
  const int *hpar;
  const unsigned *near_bits;
  Dual kr, ki;
  Cx<Dual> c1, c2, Zsi;
  int R;
  const double2 *lam, *xv, *W;
  double *part;  // [gridDim.y][gridDim.x][max(R,1)][2]
};

// The closed-form singular terms of a near pair: geometry only, scaled by
// the dual coefficients (as pair_eval does for near pairs).
template <int NQ>
__device__ __noinline__ void eps_near_terms(const AdjEpsArgs &a, int m, int n, Cx<Dual> *Sb, Cx<Dual> *Kb) {
  double st[6][9];
  static_terms<double, NQ>(reinterpret_cast<const double(*)[3]>(a.qabs + (size_t)m * NQ * 3), a.area[m], a.sl + 3 * m,
                           reinterpret_cast<const double(*)[3]>(a.bn + 9 * (size_t)m), a.geo[n], a.area[n],
                           a.sl + 3 * n, reinterpret_cast<const double(*)[3]>(a.bn + 9 * (size_t)n), m == n, st);
  const double f4 = 1.0 / (4.0 * kPi);
  const Cx<Dual> f8 = {(a.kr * a.kr - a.ki * a.ki) / (8.0 * kPi), (2.0 * a.kr * a.ki) / (8.0 * kPi)};
#pragma unroll
  for (int i = 0; i < 9; i++) {
    const Cx<Dual> dterm = {f4 * st[0][i] - f8.re * st[1][i], -f8.im * st[1][i]};
    const Cx<Dual> hterm = {f4 * st[2][i] - f8.re * st[3][i], -f8.im * st[3][i]};
    const Cx<Dual> kterm = {f4 * st[4][i] - f8.re * st[5][i], -f8.im * st[5][i]};
    Sb[i] = cxa(Sb[i], cxa(cxm(a.c1, dterm), cxm(a.c2, hterm)));
    Kb[i] = cxa(Kb[i], kterm);
  }
}

// One thread per source face, one CTA row per test face.  A far pair is
// evaluated once, by the thread with m < x, which contracts both its blocks
// ((m, x) and, with the faces' roles exchanged, (x, m)); near pairs (their
// closed-form terms are not symmetric in the two faces) and the self pair
// are evaluated in each order.
template <int NQ>
__global__ void __launch_bounds__(kAdjThreads) adj_eps_kernel(AdjEpsArgs a) {
  const int m = blockIdx.y;
  const int x = blockIdx.x * kAdjThreads + threadIdx.x;
  Cd acc[kAdjMaxObj];
#pragma unroll
  for (int o = 0; o < kAdjMaxObj; o++) acc[o] = {0.0, 0.0};
  // dZ/deps-weighted blocks of test face tm, source face tx into acc
  auto contract = [&](int tm, int tx, const Cx<Dual> *Sb, const Cx<Dual> *Kb) {
    const int64_t N = a.N, ld = a.n;
#pragma unroll 1
    for (int p = 0; p < 3; p++) {
      const int64_t r = a.hpar[3 * tm + p];
#pragma unroll 1
      for (int q = 0; q < 3; q++) {
        const int64_t cI = a.hpar[3 * tx + q];
        const Cd dS = dpart(Sb[3 * p + q]), dZ = dpart(cxm(a.Zsi, Sb[3 * p + q])), dK = dpart(Kb[3 * p + q]);
        if (a.R == 0) {
          const double2 wjj = a.W[r + cI * ld], wmm = a.W[(r + N) + (cI + N) * ld];
          const double2 wmj = a.W[(r + N) + cI * ld], wjm = a.W[r + (cI + N) * ld];
          const Cd t1 = cdm(dS, wjj), t2 = cdm(dZ, wmm), t3 = cdm(dK, make_double2(wmj.x - wjm.x, wmj.y - wjm.y));
          acc[0].re += t1.re + t2.re + t3.re;
          acc[0].im += t1.im + t2.im + t3.im;
        } else {
          for (int o = 0; o < a.R; o++) {
            const double2 *l = a.lam + (size_t)o * ld, *xo = a.xv + (size_t)o * ld;
            const double2 lr = l[r], lrN = l[r + N], xc = xo[cI], xcN = xo[cI + N];
            const double2 jj = make_double2(lr.x * xc.x - lr.y * xc.y, lr.x * xc.y + lr.y * xc.x);
            const double2 mm = make_double2(lrN.x * xcN.x - lrN.y * xcN.y, lrN.x * xcN.y + lrN.y * xcN.x);
            const double2 mj = make_double2(lrN.x * xc.x - lrN.y * xc.y, lrN.x * xc.y + lrN.y * xc.x);
            const double2 jm = make_double2(lr.x * xcN.x - lr.y * xcN.y, lr.x * xcN.y + lr.y * xcN.x);
            const Cd t1 = cdm(dS, jj), t2 = cdm(dZ, mm), t3 = cdm(dK, make_double2(mj.x - jm.x, mj.y - jm.y));
            acc[o].re += t1.re + t2.re + t3.re;
            acc[o].im += t1.im + t2.im + t3.im;
          }
        }
      }
    }
  };
  const int64_t bit = (int64_t)m * a.F + x;
  const bool near = x < a.F && ((a.near_bits[bit >> 5] >> (bit & 31)) & 1u);
  if (x < a.F && (near || m <= x)) {
    double d[3];
#pragma unroll
    for (int i = 0; i < 3; i++) d[i] = a.cp[3 * m + i] - a.cp[3 * x + i];
    Moments<Dual> M;
    if (near)
      pair_moments<Dual, NQ, true, false, double>(a.qrel + (size_t)m * NQ * 3, a.qrel + (size_t)x * NQ * 3, 1, d, a.kr,
                                                  a.ki, M);
    else
      pair_moments<Dual, NQ, false, false, double>(a.qrel + (size_t)m * NQ * 3, a.qrel + (size_t)x * NQ * 3, 1, d,
                                                   a.kr, a.ki, M);
    const Cx<Dual> fD = {a.c1.re * (kOofpi / 4.0), a.c1.im * (kOofpi / 4.0)};
    const Cx<Dual> fH = {a.c2.re * kOofpi, a.c2.im * kOofpi};
    Cx<Dual> Sb[9], Kb[9];
    blocks_generic<Dual, double>(M, reinterpret_cast<const double(*)[3]>(a.mu + 9 * (size_t)m),
                                 reinterpret_cast<const double(*)[3]>(a.mu + 9 * (size_t)x), a.sl + 3 * m,
                                 a.sl + 3 * x, d, fD, fH, kOofpi / 4.0, m == x, Sb, Kb);
    if (near) eps_near_terms<NQ>(a, m, x, Sb, Kb);
    contract(m, x, Sb, Kb);
    if (!near && m < x) {
      exchange_roles(M);
#pragma unroll
      for (int i = 0; i < 3; i++) d[i] = -d[i];
      blocks_generic<Dual, double>(M, reinterpret_cast<const double(*)[3]>(a.mu + 9 * (size_t)x),
                                   reinterpret_cast<const double(*)[3]>(a.mu + 9 * (size_t)m), a.sl + 3 * x,
                                   a.sl + 3 * m, d, fD, fH, kOofpi / 4.0, false, Sb, Kb);
      contract(x, m, Sb, Kb);
    }
  }
  __shared__ double red[kAdjThreads][2];
  const int nobj = a.R == 0 ? 1 : a.R;
  for (int o = 0; o < nobj; o++) {
    red[threadIdx.x][0] = acc[o].re;
    red[threadIdx.x][1] = acc[o].im;
    __syncthreads();
    for (int w = kAdjThreads / 2; w > 0; w >>= 1) {
      if (threadIdx.x < w) {
        red[threadIdx.x][0] += red[threadIdx.x + w][0];
        red[threadIdx.x][1] += red[threadIdx.x + w][1];
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      double *out = a.part + (((size_t)blockIdx.y * gridDim.x + blockIdx.x) * nobj + o) * 2;
      out[0] = red[0][0];
      out[1] = red[0][1];
    }
    __syncthreads();
  }
}

template <int NQ>
void launch_adj_eps(const dim3 &grid, cudaStream_t s, const AdjEpsArgs &a) {
  adj_eps_kernel<NQ><<<grid, kAdjThreads, 0, s>>>(a);
}

// ---- explicit geometry terms of the exterior surface: q and sigma --------

struct AdjSrc {
  double dir[3], pol[3];
  double ph_re, ph_im;
  int type;
};

// pw_fields / pw_fields_elliptic (source.f90:84-125) at a dual point.
__device__ void src_fields_dual(const AdjSrc &S, Cd k, double omega, const Dual *pt, Cx<Dual> *ef, Cx<Dual> *hf) {
  const Dual kd = S.dir[0] * pt[0] + S.dir[1] * pt[1] + S.dir[2] * pt[2];
  // exp(i k kd)
  Dual sn, cs;
  fsincos(k.re * kd, &sn, &cs);
  const Dual ea = fexp(-k.im * kd);
  const Cx<Dual> ph = {ea * cs, ea * sn};
  if (S.type == MOM_SRC_PW) {
    for (int i = 0; i < 3; i++) ef[i] = cxr(ph, Dual(S.pol[i]));
  } else {
    // the elliptic field is normalised pointwise, which removes |e^{ik d.r}|:
    // E = e^{i Re(k) d.r} (p + phase d x p) / |p + phase d x p|
    const Cx<Dual> phu = {cs, sn};
    const double dp[3] = {S.dir[1] * S.pol[2] - S.dir[2] * S.pol[1], S.dir[2] * S.pol[0] - S.dir[0] * S.pol[2],
                          S.dir[0] * S.pol[1] - S.dir[1] * S.pol[0]};
    double e[3][2], nn = 0;
    for (int i = 0; i < 3; i++) {
      e[i][0] = S.pol[i] + S.ph_re * dp[i];
      e[i][1] = S.ph_im * dp[i];
      nn += e[i][0] * e[i][0] + e[i][1] * e[i][1];
    }
    nn = ::sqrt(nn);
    for (int i = 0; i < 3; i++) ef[i] = cxm(phu, Cx<Dual>{Dual(e[i][0] / nn), Dual(e[i][1] / nn)});
  }
  const Cx<Dual> kk = {Dual(k.re / (omega * kMu0)), Dual(k.im / (omega * kMu0))};
  Cx<Dual> c[3];
  c[0] = cxs(cxr(ef[2], Dual(S.dir[1])), cxr(ef[1], Dual(S.dir[2])));
  c[1] = cxs(cxr(ef[0], Dual(S.dir[2])), cxr(ef[2], Dual(S.dir[0])));
  c[2] = cxs(cxr(ef[1], Dual(S.dir[0])), cxr(ef[0], Dual(S.dir[1])));
  for (int i = 0; i < 3; i++) hf[i] = cxm(kk, c[i]);
}

struct AdjFaceArgs {
  AdjTopo t;
  int64_t n;
  int ninc;
  const int *inc_node, *inc_face;
  int R;
  const int *obj_src;  // [R] source of objective o
  const int *obj_kind; // [R] 0: sigma_ext, 1: sigma_abs
  const AdjSrc *src;
  const double2 *lam, *xv;  // [R][n]
  Cd k;                      // exterior wavenumber
  double omega, cc;          // cc = 2 / (eps0 c0 Re n1)  (cs.f90:38)
  double *out;               // [3 * ninc][R]
};

// Per (exterior face touching a vertex, coordinate) and objective:
// Re(lambda^T dq) (srcvec, source.f90:214-246) plus the explicit derivative
// of the face's cs_prtsrf term (cs.f90:40-100) at fixed x.
template <int NQ>
__global__ void __launch_bounds__(64) adj_face_kernel(AdjFaceArgs a) {
  const int item = blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= 3 * a.ninc) return;
  const int f = a.inc_face[item / 3], snode = a.inc_node[item / 3], scoord = item % 3;
  FaceAll<Dual, NQ> g;
  face_build<NQ>(a.t, f, snode, scoord, g);
  const int64_t N = a.t.N;
  for (int o = 0; o < a.R; o++) {
    const AdjSrc S = a.src[a.obj_src[o]];
    const double2 *l = a.lam + (size_t)o * a.n, *x = a.xv + (size_t)o * a.n;
    Cx<Dual> Ie[3], Ih[3];
    for (int p = 0; p < 3; p++) Ie[p] = Ih[p] = Cx<Dual>{Dual(0.0), Dual(0.0)};
    Dual int1 = 0.0, int2 = 0.0;
    Cd al[3], be[3];
    for (int p = 0; p < 3; p++) {
      const int64_t idx = a.t.hpar[3 * f + p];
      al[p] = {x[idx].x, x[idx].y};
      be[p] = {x[idx + N].x, x[idx + N].y};
    }
    for (int t = 0; t < NQ; t++) {
      const Dual *pt = g.qa[t];
      Cx<Dual> ef[3], hf[3];
      src_fields_dual(S, a.k, a.omega, pt, ef, hf);
      const double w = c_qw[t];
      Cx<Dual> Et[3], Ht[3];
      for (int i = 0; i < 3; i++) Et[i] = Ht[i] = Cx<Dual>{Dual(0.0), Dual(0.0)};
      for (int p = 0; p < 3; p++) {
        const Dual cc = g.sl[p] / (2.0 * g.area);
        Dual fr[3], fnv[3];
        for (int i = 0; i < 3; i++) fr[i] = cc * (pt[i] - g.bn[p][i]);
        // srcvec: <f_p, E_inc>, <f_p, H_inc>
        Cx<Dual> de = {Dual(0.0), Dual(0.0)}, dh = {Dual(0.0), Dual(0.0)};
        for (int i = 0; i < 3; i++) {
          de = cxa(de, cxr(ef[i], fr[i]));
          dh = cxa(dh, cxr(hf[i], fr[i]));
        }
        Ie[p] = cxa(Ie[p], cxr(de, Dual(w)));
        Ih[p] = cxa(Ih[p], cxr(dh, Dual(w)));
        // cs_prtsrf: tangential fields n x f_p
        cross3(g.g.n, fr, fnv);
        for (int i = 0; i < 3; i++) {
          Ht[i] = cxs(Ht[i], Cx<Dual>{al[p].re * fnv[i], al[p].im * fnv[i]});
          Et[i] = cxa(Et[i], Cx<Dual>{be[p].re * fnv[i], be[p].im * fnv[i]});
        }
      }
      // incident tangential fields (n x F) x n
      Cx<Dual> Eti[3], Hti[3], t1[3];
      auto ncross = [&](const Cx<Dual> *v, Cx<Dual> *r) {
        const Dual *nn = g.g.n;
        r[0] = cxs(cxr(v[2], nn[1]), cxr(v[1], nn[2]));
        r[1] = cxs(cxr(v[0], nn[2]), cxr(v[2], nn[0]));
        r[2] = cxs(cxr(v[1], nn[0]), cxr(v[0], nn[1]));
      };
      auto crossn = [&](const Cx<Dual> *v, Cx<Dual> *r) {
        const Dual *nn = g.g.n;
        r[0] = cxs(cxr(v[1], nn[2]), cxr(v[2], nn[1]));
        r[1] = cxs(cxr(v[2], nn[0]), cxr(v[0], nn[2]));
        r[2] = cxs(cxr(v[0], nn[1]), cxr(v[1], nn[0]));
      };
      ncross(hf, t1);
      crossn(t1, Hti);
      ncross(ef, t1);
      crossn(t1, Eti);
      // 0.5 Re[(E x H*) . n] for total and scattered fields
      auto flux = [&](const Cx<Dual> *E, const Cx<Dual> *H) {
        Cx<Dual> hc[3], cr[3];
        for (int i = 0; i < 3; i++) hc[i] = {H[i].re, -H[i].im};
        cr[0] = cxs(cxm(E[1], hc[2]), cxm(E[2], hc[1]));
        cr[1] = cxs(cxm(E[2], hc[0]), cxm(E[0], hc[2]));
        cr[2] = cxs(cxm(E[0], hc[1]), cxm(E[1], hc[0]));
        return 0.5 * (cr[0].re * g.g.n[0] + cr[1].re * g.g.n[1] + cr[2].re * g.g.n[2]);
      };
      Cx<Dual> Es[3], Hs[3];
      for (int i = 0; i < 3; i++) {
        Es[i] = cxs(Et[i], Eti[i]);
        Hs[i] = cxs(Ht[i], Hti[i]);
      }
      int1 += w * flux(Et, Ht);
      int2 += w * flux(Es, Hs);
    }
    // Re(lambda^T dq): q[J] = A Ie, q[M] = A Ih
    double dq = 0.0;
    for (int p = 0; p < 3; p++) {
      const int64_t idx = a.t.hpar[3 * f + p];
      const Cd qe = dpart(cxr(Ie[p], g.area)), qh = dpart(cxr(Ih[p], g.area));
      const double2 le = l[idx], lh = l[idx + N];
      dq += le.x * qe.re - le.y * qe.im + lh.x * qh.re - lh.y * qh.im;
    }
    const double i1 = (int1 * g.area).d, i2 = (int2 * g.area).d;
    const double dsig = a.obj_kind[o] == 0 ? a.cc * (i2 - i1) : -a.cc * i1;
    a.out[(size_t)item * a.R + o] = dq + dsig;
  }
}

// Near-pair bitmap of a domain from its near list.
__global__ void near_bits_kernel(int64_t nnear, int F, const int *nm, const int *nn, unsigned *bits) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nnear) return;
  const int64_t b = (int64_t)nm[j] * F + nn[j];
  atomicOr(bits + (b >> 5), 1u << (b & 31));
}

template <int NQ>
void launch_adj_pair(const dim3 &grid, cudaStream_t s, const AdjPairArgs &a) {
  adj_pair_kernel<NQ><<<grid, kAdjThreads, 0, s>>>(a);
}
template <int NQ>
void launch_adj_face(int blocks, cudaStream_t s, const AdjFaceArgs &a) {
  adj_face_kernel<NQ><<<blocks, 64, 0, s>>>(a);
}

}  // namespace
