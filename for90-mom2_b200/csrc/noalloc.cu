// Allocation-free variant of the cross-section reduction (cs_prtsrf).
//
// Some callers cannot allocate device memory when they ask for cross
// sections: applications whose device memory is reserved up front by
// another allocator (a framework's caching allocator that owns the whole
// pool), and latency-sensitive callers that cannot accept the implicit
// device-wide synchronisation of cudaMalloc / cudaFree.  For them this file
// provides mom_gpu_cross_sections_noalloc: the same computation as
// mom_gpu_cross_sections, with every scratch byte (source parameters,
// per-block partial sums, the reduced results) in one file-scope
// __device__ array of fixed size.  The caller passes the solutions as a
// device pointer and receives the results in host arrays; the function
// calls no cudaMalloc, cudaFree or other allocating routine.
//
// Limits: at most kNaMaxSrc sources per call and at most
// kNaMaxBlocks * kNaThreads faces in the domain (scratch ~263 KB, held by
// every device that loads the library until the process exits).
//
// Set-up: every call looks up the array's device address in the current
// context with cudaGetSymbolAddress (host code must not use the symbol
// itself as a device address).  With lazy module loading (the CUDA
// default) the first call on a device may load this module, which
// allocates the array and can synchronise the device; callers that must
// not allocate at all make one warm-up call at set-up.  Every call copies
// its sources to the device and synchronises the context's stream before
// returning, so it must not be called while a stream capture is open.
// Sharing: every call on a device uses the same array and it keeps the last
// call's contents.  Calls on one context are serialised by its mutex; calls
// from different contexts (or processes sharing a context) that overlap on
// the GPU race on the array.  No part of the scratch needs to start at zero:
// each call writes every partial sum and result it later reads.
#include <cuda_runtime.h>

#include <cmath>

#include "mom_internal.h"

namespace mom {
namespace {

constexpr int kNaMaxSrc = 64;
constexpr int kNaThreads = 256;
constexpr int kNaMaxBlocks = 256;

struct NaSrc {
  double dir[3], pol[3];
  double ph_re, ph_im;
  int type;
};

struct NaScratch {
  NaSrc src[kNaMaxSrc];
  double part[kNaMaxSrc][kNaMaxBlocks][2];
  double result[kNaMaxSrc][2];
};

static __device__ __align__(256) NaScratch g_na_scratch;

struct Zc {
  double re, im;
};
__device__ __forceinline__ Zc za(Zc a, Zc b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ Zc zs(Zc a, Zc b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ Zc zm(Zc a, Zc b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ Zc zr(Zc a, double s) { return {a.re * s, a.im * s}; }
__device__ __forceinline__ void zx(const Zc *a, const Zc *b, Zc *r) {
  r[0] = zs(zm(a[1], b[2]), zm(a[2], b[1]));
  r[1] = zs(zm(a[2], b[0]), zm(a[0], b[2]));
  r[2] = zs(zm(a[0], b[1]), zm(a[1], b[0]));
}

// pw_fields / pw_fields_elliptic (source.f90:84-125)
__device__ void na_fields(const NaSrc &S, Zc k, double omega, const double *pt, Zc *ef, Zc *hf) {
  if (S.type == MOM_SRC_NONE) {  // no incident field
    for (int i = 0; i < 3; i++) ef[i] = hf[i] = {0, 0};
    return;
  }
  const double kd = S.dir[0] * pt[0] + S.dir[1] * pt[1] + S.dir[2] * pt[2];
  double sn, cs;
  sincos(k.re * kd, &sn, &cs);
  const double am = exp(-k.im * kd);
  const Zc ph = {am * cs, am * sn};
  const Zc dc[3] = {{S.dir[0], 0}, {S.dir[1], 0}, {S.dir[2], 0}};
  if (S.type == MOM_SRC_PW) {
    for (int i = 0; i < 3; i++) ef[i] = zr(ph, S.pol[i]);
  } else {
    Zc efx[3], efy[3];
    for (int i = 0; i < 3; i++) efx[i] = zr(ph, S.pol[i]);
    zx(dc, efx, efy);
    const Zc phase = {S.ph_re, S.ph_im};
    double nn = 0;
    for (int i = 0; i < 3; i++) {
      ef[i] = za(efx[i], zm(phase, efy[i]));
      nn += ef[i].re * ef[i].re + ef[i].im * ef[i].im;
    }
    nn = sqrt(nn);
    for (int i = 0; i < 3; i++) ef[i] = {ef[i].re / nn, ef[i].im / nn};
  }
  Zc c[3];
  zx(dc, ef, c);
  const Zc kk = {k.re / (omega * kMu0), k.im / (omega * kMu0)};
  for (int i = 0; i < 3; i++) hf[i] = zm(kk, c[i]);
}

struct NaArgs {
  double w[kMaxQ];
  int F, nq, N;
  const double *qabs, *area, *sl, *mu, *cp, *nrm;
  const int *hpar;
  const double2 *x;
  int64_t ldx;
  Zc k;
  double omega;
  NaScratch *scr;
};

// cs_prtsrf (cs.f90:14-104) per face, block partial sums into the scratch.
__global__ void __launch_bounds__(kNaThreads) na_cs_kernel(NaArgs a) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  double i1 = 0, i2 = 0;
  if (f < a.F) {
    const NaSrc S = a.scr->src[s];
    const double2 *x = a.x + (size_t)s * a.ldx;
    const double An = a.area[f];
    const double *nor = a.nrm + 3 * f;
    const Zc nc[3] = {{nor[0], 0}, {nor[1], 0}, {nor[2], 0}};
    Zc al[3], be[3];
    for (int p = 0; p < 3; p++) {
      const int idx = a.hpar[3 * f + p];
      al[p] = {x[idx].x, x[idx].y};
      be[p] = {x[idx + a.N].x, x[idx + a.N].y};
    }
    double int1 = 0, int2 = 0;
    for (int t = 0; t < a.nq; t++) {
      const double *pt = a.qabs + ((size_t)f * a.nq + t) * 3;
      Zc Et[3] = {{0, 0}, {0, 0}, {0, 0}}, Ht[3] = {{0, 0}, {0, 0}, {0, 0}};
      for (int p = 0; p < 3; p++) {
        const double cc = a.sl[3 * f + p] / (2.0 * An);
        double fr[3], fn[3];
        for (int i = 0; i < 3; i++) fr[i] = cc * (pt[i] - (a.cp[3 * f + i] + a.mu[9 * f + 3 * p + i]));
        fn[0] = nor[1] * fr[2] - nor[2] * fr[1];
        fn[1] = nor[2] * fr[0] - nor[0] * fr[2];
        fn[2] = nor[0] * fr[1] - nor[1] * fr[0];
        for (int i = 0; i < 3; i++) {
          Ht[i] = zs(Ht[i], zr(al[p], fn[i]));
          Et[i] = za(Et[i], zr(be[p], fn[i]));
        }
      }
      Zc einc[3], hinc[3], t1[3], Eti[3], Hti[3], Ets[3], Hts[3], cr[3], cj[3];
      na_fields(S, a.k, a.omega, pt, einc, hinc);
      zx(nc, hinc, t1);
      zx(t1, nc, Hti);
      zx(nc, einc, t1);
      zx(t1, nc, Eti);
      for (int i = 0; i < 3; i++) {
        Hts[i] = zs(Ht[i], Hti[i]);
        Ets[i] = zs(Et[i], Eti[i]);
        cj[i] = {Ht[i].re, -Ht[i].im};
      }
      zx(Et, cj, cr);
      const double w = a.w[t];
      int1 += w * 0.5 * (cr[0].re * nor[0] + cr[1].re * nor[1] + cr[2].re * nor[2]);
      for (int i = 0; i < 3; i++) cj[i] = {Hts[i].re, -Hts[i].im};
      zx(Ets, cj, cr);
      int2 += w * 0.5 * (cr[0].re * nor[0] + cr[1].re * nor[1] + cr[2].re * nor[2]);
    }
    i1 = int1 * An;
    i2 = int2 * An;
  }
  __shared__ double r1[kNaThreads], r2[kNaThreads];
  r1[threadIdx.x] = i1;
  r2[threadIdx.x] = i2;
  __syncthreads();
  for (int h = kNaThreads / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      r1[threadIdx.x] += r1[threadIdx.x + h];
      r2[threadIdx.x] += r2[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    a.scr->part[s][blockIdx.x][0] = r1[0];
    a.scr->part[s][blockIdx.x][1] = r2[0];
  }
}

// Sum the block partials of each source in block order.
__global__ void na_reduce_kernel(NaScratch *scr, int nblocks, int nsrc) {
  const int s = threadIdx.x;
  if (s >= nsrc) return;
  double ab = 0, sc = 0;
  for (int b = 0; b < nblocks; b++) {
    ab += scr->part[s][b][0];
    sc += scr->part[s][b][1];
  }
  scr->result[s][0] = ab;
  scr->result[s][1] = sc;
}

// Device address of the scratch array in the current CUDA context, looked
// up on every call: the address belongs to the context, and a context
// recreated after a device reset places the array elsewhere.
int na_scratch_address(Ctx *c, NaScratch **out) {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_na_scratch);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaGetSymbolAddress(g_na_scratch)");
  *out = reinterpret_cast<NaScratch *>(p);
  return MOM_OK;
}

}  // namespace
}  // namespace mom

using namespace mom;

struct mom_ctx : public Ctx {};

extern "C" int mom_gpu_cross_sections_noalloc(mom_ctx *c, int32_t dom, double omega, const double *ri, int32_t nsrc,
                                              const mom_src *src, const void *x_dev, int64_t ldx, double *csca,
                                              double *cabs) {
  if (!c) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  if (!c->have_problem) return fail(c, MOM_ERR_STATE, "set the problem first");
  if (dom < 0 || dom >= c->ndom || !src || !ri || !csca || !cabs || !x_dev || !(omega > 0) ||
      ldx < 2 * (int64_t)c->N)
    return fail(c, MOM_ERR_ARG, "invalid cross-section arguments");
  if (nsrc < 1 || nsrc > kNaMaxSrc)
    return fail(c, MOM_ERR_ARG, "allocation-free cross sections take 1 to 64 sources per call");
  if (c->nga > 1) return fail(c, MOM_ERR_ARG, "allocation-free cross sections take the identity group only");
  const DomDev &D = c->dom[dom];
  const int blocks = (D.F + kNaThreads - 1) / kNaThreads;
  if (blocks > kNaMaxBlocks)
    return fail(c, MOM_ERR_ARG, "allocation-free cross sections support at most 65536 faces per domain");
  MOM_CUDA(c, cudaSetDevice(c->device));
  NaScratch *scr = nullptr;
  MOM_TRY(na_scratch_address(c, &scr));
  NaSrc hs[kNaMaxSrc];
  for (int i = 0; i < nsrc; i++) {
    const mom_src &s = src[i];
    if (s.type != MOM_SRC_PW && s.type != MOM_SRC_PW_ELLIPTIC && s.type != MOM_SRC_NONE)
      return fail(c, MOM_ERR_ARG, "unsupported source type (only pw, pw_elliptic and none)");
    // get_dir / get_pol (aux.f90:245-261)
    const double th = s.theta, ph = s.phi, ps = (s.type == MOM_SRC_PW) ? s.psi : 0.0;
    hs[i].dir[0] = sin(th) * cos(ph);
    hs[i].dir[1] = sin(th) * sin(ph);
    hs[i].dir[2] = cos(th);
    hs[i].pol[0] = cos(ps) * sin(ph) - sin(ps) * cos(th) * cos(ph);
    hs[i].pol[1] = -cos(ps) * cos(ph) - sin(ps) * cos(th) * sin(ph);
    hs[i].pol[2] = sin(ps) * sin(th);
    hs[i].ph_re = s.phase_re;
    hs[i].ph_im = s.phase_im;
    hs[i].type = s.type;
  }
  MOM_CUDA(c, cudaMemcpyAsync(scr->src, hs, sizeof(NaSrc) * nsrc, cudaMemcpyHostToDevice, c->stream));
  NaArgs a;
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
  a.x = reinterpret_cast<const double2 *>(x_dev);
  a.ldx = ldx;
  a.k = {ri[0] * omega / kC0, ri[1] * omega / kC0};
  a.omega = omega;
  a.scr = scr;
  na_cs_kernel<<<dim3(blocks, nsrc), kNaThreads, 0, c->stream>>>(a);
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  na_reduce_kernel<<<1, kNaMaxSrc, 0, c->stream>>>(scr, blocks, nsrc);
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  double res[kNaMaxSrc][2];
  MOM_CUDA(c, cudaMemcpyAsync(res, scr->result, sizeof(double) * 2 * nsrc, cudaMemcpyDeviceToHost, c->stream));
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  const double cc = 2.0 / (kEps0 * kC0 * ri[0]);  // cs.f90:38
  for (int s = 0; s < nsrc; s++) {
    cabs[s] = -cc * res[s][0];
    csca[s] = cc * res[s][1];
  }
  return MOM_OK;
}
