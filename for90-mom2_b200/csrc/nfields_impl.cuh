// Scattered near fields of a domain's surface currents at arbitrary points
// (scat_fields, nfields.f90:29-49, with scat_fields_frags 109-197, identity
// group).  Included once, at the end of assemble.cu, so that the field
// kernel shares the closed-form static integrals (point_static) and the
// quadrature weights (c_qw) of the assembly (inside namespace mom).
//
// For point r and source face f with RWG functions f_q = c_q (r' - p_q)
// (c_q = s_q l_q / (2 A_f), div f_q = s_q l_q / A_f) the kernel needs
//   K2_q = int G f_q,  K3_q = int grad'G div'f_q,  K4_q = int grad'G x f_q
// (intK2, intK3, intK4 of srcint.f90 with no test face).  With
// grad'G = (r - r') phi / (4 pi), phi = e^{ikR} (1/R^3 - ik/R^2), one
// quadrature pass over the face gives the sums
//   SG = sum w g,  SGr = sum w g r',  SPd = sum w phi (r - r')
// and then  K2_q = c_q (SGr - p_q SG),  K3_q = div_q SPd,
// K4_q = -c_q (r - p_q) x SPd   (all times A_f / (4 pi); SPd = sum w phi (r - r'),
// using (r - r') x r' = -(r x (r - r'))).  Within three
// average edge lengths of the face centroid the smoothed kernels are used and
// the closed-form parts (1/(4 pi)) X_m1 - (k^2/(8 pi)) X_1 are added, as in
// the reference.  The currents then give (c1 = i w mu0, c2 = 1/(i w eps0 n^2))
//   E += x_J (c1 K2 + c2 K3) + x_M K4,   H += x_M (K2/c2 + K3/c1) - x_J K4.

namespace {

constexpr int kNfThreads = 128;

struct NfArgs {
  int F, N;
  const double *qabs;    // [F][NQ][3]
  const double *cp;      // [F][3]
  const double *area;    // [F]
  const double *sl;      // [F][3]
  const int *hpar;       // [F][3] global edge of local edge q
  const FaceGeo *geo;    // [F]
  const double *bn;      // [F][3][3] free vertex of local edge q
  double thr2;           // (3 avelen)^2
  double kr, ki;         // k = ri w / c0
  Cd k2;                 // k^2
  Cd c1, c2;             // i w mu0, 1 / (i w eps0 n^2)
  const double2 *X;      // [nsrc][ldx]: J in 0..N-1, M in N..2N-1
  int64_t ldx;
  int nsrc;              // sources in this launch (<= NS)
  const double *pts;     // [npts][3]
  double2 *E, *H;        // [nsrc][npts][3] (the launch's first source at E)
  int npts;
};

__device__ __forceinline__ Cd cadd(Cd a, Cd b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ Cd csc(Cd a, double s) { return {a.re * s, a.im * s}; }
__host__ __device__ __forceinline__ Cd cdivd(Cd a, Cd b) {
  const double d = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}

// One CTA per point; threads stride over the faces and reduce at the end.
template <int NQ, int NS>
__global__ void __launch_bounds__(kNfThreads) nfield_kernel(NfArgs a) {
  const int ip = blockIdx.x;
  const double r[3] = {a.pts[3 * ip], a.pts[3 * ip + 1], a.pts[3 * ip + 2]};
  Cd e[NS][3], h[NS][3];
#pragma unroll
  for (int s = 0; s < NS; s++)
#pragma unroll
    for (int i = 0; i < 3; i++) e[s][i] = h[s][i] = Cd{0, 0};
  const double k2r = a.k2.re, k2i = a.k2.im;
  for (int f = threadIdx.x; f < a.F; f += blockDim.x) {
    const double *cp = a.cp + 3 * f;
    const double dc[3] = {r[0] - cp[0], r[1] - cp[1], r[2] - cp[2]};
    const bool near = dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2] < a.thr2;
    Cd SG = {0, 0}, SGr[3] = {{0, 0}, {0, 0}, {0, 0}}, SPd[3] = {{0, 0}, {0, 0}, {0, 0}};
    const double *q = a.qabs + (size_t)f * NQ * 3;
#pragma unroll 1
    for (int t = 0; t < NQ; t++) {
      const double rp[3] = {q[3 * t], q[3 * t + 1], q[3 * t + 2]};
      const double w = c_qw[t];
      const double dx = r[0] - rp[0], dy = r[1] - rp[1], dz = r[2] - rp[2];
      const double R2 = dx * dx + dy * dy + dz * dz;
      Cd g, p;
      if (R2 > 0) {
        const double R = ::sqrt(R2), iR = 1.0 / R, iR2 = iR * iR, iR3 = iR2 * iR;
        double sn, cs;
        ::sincos(a.kr * R, &sn, &cs);
        const double ea = ::exp(-a.ki * R);
        const double er = ea * cs, ei = ea * sn;
        const double qr = iR3 + a.ki * iR2, qi = -a.kr * iR2;  // 1/R^3 - i k / R^2
        if (near) {  // green.f90 vGs / vgradGs: (e - 1)/R + k^2 R / 2, e q - 1/R^3 - k^2/(2R)
          g = {(er - 1.0) * iR + 0.5 * k2r * R, ei * iR + 0.5 * k2i * R};
          p = {er * qr - ei * qi - iR3 - 0.5 * k2r * iR, er * qi + ei * qr - 0.5 * k2i * iR};
        } else {
          g = {er * iR, ei * iR};
          p = {er * qr - ei * qi, er * qi + ei * qr};
        }
      } else if (near) {  // R = 0: Gs = i k / (4 pi), grad Gs = 0
        g = {-a.ki, a.kr};
        p = {0, 0};
      } else {
        g = {0, 0};
        p = {0, 0};
      }
      const double dd[3] = {dx, dy, dz};
      SG = cadd(SG, csc(g, w));
#pragma unroll
      for (int i = 0; i < 3; i++) {
        SGr[i] = cadd(SGr[i], csc(g, w * rp[i]));
        SPd[i] = cadd(SPd[i], csc(p, w * dd[i]));
      }
    }
    const double An = a.area[f], sc = An * kOofpi;
    SG = csc(SG, sc);
    Cd grad[3];  // int grad'G over the face (+ its closed-form part when near)
#pragma unroll
    for (int i = 0; i < 3; i++) {
      SGr[i] = csc(SGr[i], sc);
      grad[i] = csc(SPd[i], sc);
    }
    PointStatic<double> ps;
    const double f4 = 1.0 / (4.0 * kPi);
    const Cd f8 = {k2r / (8.0 * kPi), k2i / (8.0 * kPi)};
    if (near) {
      // intK3singular (srcint.f90:227-260): (1/(4 pi)) K3m1 - (k^2/(8 pi)) K31
      point_static(r, a.geo[f], ps);
#pragma unroll
      for (int i = 0; i < 3; i++) grad[i] = cadd(grad[i], {f4 * ps.K3m1[i] - f8.re * ps.K31[i], -f8.im * ps.K31[i]});
    }
#pragma unroll
    for (int qe = 0; qe < 3; qe++) {
      const double slq = a.sl[3 * f + qe];
      const double cq = slq / (2.0 * An), dq = slq / An;
      const double *pq = a.bn + 9 * f + 3 * qe;
      const double rpq[3] = {r[0] - pq[0], r[1] - pq[1], r[2] - pq[2]};
      Cd K2[3], K3[3], K4[3];
#pragma unroll
      for (int i = 0; i < 3; i++) {
        K2[i] = csc({SGr[i].re - pq[i] * SG.re, SGr[i].im - pq[i] * SG.im}, cq);
        K3[i] = csc(grad[i], dq);
      }
      // K4 = -c_q (r - p_q) x grad (intK4singular, srcint.f90:330-366, has the same form)
      K4[0] = csc({rpq[1] * grad[2].re - rpq[2] * grad[1].re, rpq[1] * grad[2].im - rpq[2] * grad[1].im}, -cq);
      K4[1] = csc({rpq[2] * grad[0].re - rpq[0] * grad[2].re, rpq[2] * grad[0].im - rpq[0] * grad[2].im}, -cq);
      K4[2] = csc({rpq[0] * grad[1].re - rpq[1] * grad[0].re, rpq[0] * grad[1].im - rpq[1] * grad[0].im}, -cq);
      if (near) {
        // intK2singular (srcint.f90:121-154)
#pragma unroll
        for (int i = 0; i < 3; i++) {
          const double k2m1 = cq * (ps.mL1[i] + (ps.rho[i] - pq[i]) * ps.Sm1);
          const double k21 = cq * (1.0 / 3.0 * ps.mL3[i] + (ps.rho[i] - pq[i]) * ps.S1);
          K2[i] = cadd(K2[i], {f4 * k2m1 - f8.re * k21, -f8.im * k21});
        }
      }
      const int idx = a.hpar[3 * f + qe];
#pragma unroll
      for (int s = 0; s < NS; s++) {
        if (s >= a.nsrc) break;
        const double2 xj2 = a.X[(size_t)s * a.ldx + idx], xm2 = a.X[(size_t)s * a.ldx + idx + a.N];
        const Cd xj = {xj2.x, xj2.y}, xm = {xm2.x, xm2.y};
#pragma unroll
        for (int i = 0; i < 3; i++) {
          const Cd ee = cadd(cadd(cmul(a.c1, K2[i]), cmul(a.c2, K3[i])), Cd{0, 0});
          e[s][i] = cadd(e[s][i], cadd(cmul(xj, ee), cmul(xm, K4[i])));
          const Cd hh = cadd(cdivd(K2[i], a.c2), cdivd(K3[i], a.c1));
          const Cd hx = cmul(xm, hh), hj = cmul(xj, K4[i]);
          h[s][i] = cadd(h[s][i], {hx.re - hj.re, hx.im - hj.im});
        }
      }
    }
  }
  // CTA reduction: warp shuffles, then one value per warp through shared memory
  __shared__ double red[kNfThreads / 32][NS * 12];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int s = 0; s < NS; s++)
#pragma unroll
    for (int i = 0; i < 3; i++) {
      double v[4] = {e[s][i].re, e[s][i].im, h[s][i].re, h[s][i].im};
#pragma unroll
      for (int c = 0; c < 4; c++) {
        for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_down_sync(0xffffffffu, v[c], o);
        if (lane == 0) red[wid][s * 12 + i * 4 + c] = v[c];
      }
    }
  __syncthreads();
  for (int j = threadIdx.x; j < NS * 12; j += blockDim.x) {
    const int s = j / 12, i = (j % 12) / 4, c = j % 4;
    if (s >= a.nsrc) continue;
    double t = 0;
    for (int w = 0; w < kNfThreads / 32; w++) t += red[w][j];
    double2 *dst = (c < 2 ? a.E : a.H) + ((size_t)s * a.npts + ip) * 3 + i;
    if (c % 2 == 0) dst->x = t;
    else dst->y = t;
  }
}

template <int NQ>
void launch_nfield(int ns, int npts, cudaStream_t st, const NfArgs &a) {
  if (ns == 1) nfield_kernel<NQ, 1><<<npts, kNfThreads, 0, st>>>(a);
  else if (ns == 2) nfield_kernel<NQ, 2><<<npts, kNfThreads, 0, st>>>(a);
  else nfield_kernel<NQ, 4><<<npts, kNfThreads, 0, st>>>(a);
}

}  // namespace

// Face geometry of domain d for the field kernel (uploaded once per geometry).
static int nfield_geometry(Ctx *c, DomDev &D) {
  if (D.nf_geo) return MOM_OK;
  const int F = D.F;
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
  void *pg = nullptr;
  double *pb = nullptr;
  if (cudaMalloc(&pg, sizeof(FaceGeo) * F) != cudaSuccess || cudaMalloc(&pb, sizeof(double) * 9 * F) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(pg);
    return fail(c, MOM_ERR_ALLOC, "near-field geometry allocation failed");
  }
  D.nf_geo = pg;
  D.nf_bn = pb;
  MOM_CUDA(c, cudaMemcpyAsync(pg, geo.data(), sizeof(FaceGeo) * F, cudaMemcpyHostToDevice, c->stream));
  MOM_CUDA(c, cudaMemcpyAsync(pb, D.h_bn.data(), sizeof(double) * 9 * F, cudaMemcpyHostToDevice, c->stream));
  return MOM_OK;
}

int scat_fields(Ctx *c, int d, double omega, const double *ri, int nsrc, const double2 *X, int64_t ldx, int npts,
                const double *pts, double2 *E, double2 *H) {
  if (d < 0 || d >= c->ndom) return fail(c, MOM_ERR_ARG, "domain index out of range");
  DomDev &D = c->dom[d];
  MOM_TRY(nfield_geometry(c, D));
  const double k0 = omega / kC0;
  NfArgs a;
  a.F = D.F;
  a.N = c->N;
  a.qabs = D.qabs;
  a.cp = D.cp;
  a.area = D.area;
  a.sl = D.sl;
  a.hpar = D.hpar;
  a.geo = reinterpret_cast<const FaceGeo *>(D.nf_geo);
  a.bn = D.nf_bn;
  a.thr2 = (D.avelen * 3) * (D.avelen * 3);
  a.kr = ri[0] * k0;
  a.ki = ri[1] * k0;
  a.k2 = {a.kr * a.kr - a.ki * a.ki, 2 * a.kr * a.ki};
  a.c1 = {0.0, omega * kMu0};
  const Cd n2 = {ri[0] * ri[0] - ri[1] * ri[1], 2 * ri[0] * ri[1]};
  const Cd den = {-omega * kEps0 * n2.im, omega * kEps0 * n2.re};  // i w eps0 n^2
  a.c2 = cdivd({1.0, 0.0}, den);
  a.ldx = ldx;
  a.pts = pts;
  a.npts = npts;
  for (int s0 = 0; s0 < nsrc; s0 += 4) {
    const int ns = std::min(4, nsrc - s0);
    a.nsrc = ns;
    a.X = X + (size_t)s0 * ldx;
    a.E = E + (size_t)s0 * npts * 3;
    a.H = H + (size_t)s0 * npts * 3;
    const int nl = ns == 1 ? 1 : (ns == 2 ? 2 : 4);
    switch (c->nq) {
      case 1: launch_nfield<1>(nl, npts, c->stream, a); break;
      case 3: launch_nfield<3>(nl, npts, c->stream, a); break;
      case 4: launch_nfield<4>(nl, npts, c->stream, a); break;
      case 7: launch_nfield<7>(nl, npts, c->stream, a); break;
      case 13: launch_nfield<13>(nl, npts, c->stream, a); break;
      default: return fail(c, MOM_ERR_ARG, "unsupported number of quadrature points");
    }
    c->launches++;
    MOM_CUDA(c, cudaGetLastError());
  }
  return MOM_OK;
}
