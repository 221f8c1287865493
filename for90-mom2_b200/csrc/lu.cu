// Dense complex LU with partial pivoting and triangular solves on sm_100a.
//
// Replaces ZGETRF + ZGETRS of solve_multi_linsys (linalg.f90:159-180).
// Right-looking blocked LU, panel width nb:
//   panel_kernel   cooperative, one CTA per SM, the panel held in shared
//                  memory; per column one bounded grid barrier, pivot =
//                  first row of largest |re|+|im| (izamax), FP64 arithmetic;
//   laswp_kernel   the panel's row interchanges on the other columns;
//   diag_inv       inverses of the unit-lower and upper diagonal blocks;
//   TRSM as GEMM   U12 = inv(L11) A12, then A22 -= L21 U12 (plain library
//                  GEMMs: cuBLAS ZGEMM for FP64, CGEMM on TF32 tensor cores
//                  for the mixed path).
// The mixed path factors an FP32 copy and refines in FP64 against the FP64
// matrix (iterative refinement; residual GEMV kernel below).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "mom_internal.h"

namespace mom {
namespace {

__device__ __forceinline__ double2 ld2(const double2 *p) { return *p; }
__device__ __forceinline__ double2 ld2(const float2 *p) {
  float2 v = *p;
  return make_double2(v.x, v.y);
}
__device__ __forceinline__ void st2(double2 *p, double2 v) { *p = v; }
__device__ __forceinline__ void st2(float2 *p, double2 v) { *p = make_float2((float)v.x, (float)v.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double cabs1(double2 a) { return fabs(a.x) + fabs(a.y); }

constexpr int kPanelThreads = 256;
constexpr long long kSpinLimit = 1LL << 24;  // bounded barrier wait (~seconds)

struct PanelArgs {
  void *A;
  int64_t lda, n, j0;
  int nb, rpc, P;
  int *ipiv;
  int *info;      // first zero pivot (1-based), 0 if none
  int *timeout;   // set when a barrier wait ran out
  unsigned *bar;  // arrival counter, zeroed before launch
  double *cand_abs;   // [2][P]
  int *cand_row;      // [2][P]
  double2 *cand_data; // [2][P][nb]
  double2 *col_data;  // [2][nb]
};

__device__ bool grid_barrier(unsigned *bar, unsigned target, int *timeout) {
  __syncthreads();
  bool ok = true;
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(bar, 1u);
    long long it = 0;
    while (true) {
      unsigned v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
      if (v >= target) break;
      if (*(volatile int *)timeout) { ok = false; break; }
      if (++it > kSpinLimit) {
        atomicExch(timeout, 1);
        ok = false;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
  }
  __shared__ int s_ok;
  if (threadIdx.x == 0) s_ok = ok;
  __syncthreads();
  return s_ok != 0;
}

template <typename T>
__global__ void __launch_bounds__(kPanelThreads, 1) panel_kernel(PanelArgs a) {
  extern __shared__ double2 slab[];  // [nb][rpc] column-major within the CTA
  __shared__ double red_abs[kPanelThreads];
  __shared__ int red_row[kPanelThreads];
  __shared__ int s_prow, s_pcta;
  const int tid = threadIdx.x, cta = blockIdx.x;
  const int nb = a.nb, rpc = a.rpc;
  T *A = reinterpret_cast<T *>(a.A);
  const int64_t row0 = a.j0 + (int64_t)cta * rpc;
  const int64_t rem = a.n - row0;
  const int nrow = rem <= 0 ? 0 : (rem < rpc ? (int)rem : rpc);
  for (int idx = tid; idx < nb * rpc; idx += kPanelThreads) {
    const int c = idx / rpc, i = idx % rpc;
    slab[idx] = (i < nrow) ? ld2(A + (row0 + i) + (a.j0 + c) * a.lda) : make_double2(0, 0);
  }
  __syncthreads();
  for (int c = 0; c < nb; c++) {
    const int64_t col = a.j0 + c;
    const int par = c & 1;
    // local pivot candidate in column c over owned rows >= col
    double best = -1.0;
    int brow = 0x7fffffff;
    for (int i = tid; i < nrow; i += kPanelThreads) {
      const int64_t g = row0 + i;
      if (g < col) continue;
      const double v = cabs1(slab[c * rpc + i]);
      if (v > best || (v == best && g < brow)) {
        best = v;
        brow = (int)g;
      }
    }
    red_abs[tid] = best;
    red_row[tid] = brow;
    __syncthreads();
    for (int w = kPanelThreads / 2; w > 0; w >>= 1) {
      if (tid < w) {
        const double ov = red_abs[tid + w];
        const int orow = red_row[tid + w];
        if (ov > red_abs[tid] || (ov == red_abs[tid] && orow < red_row[tid])) {
          red_abs[tid] = ov;
          red_row[tid] = orow;
        }
      }
      __syncthreads();
    }
    const int my_row = red_row[0];
    if (tid == 0) {
      a.cand_abs[par * a.P + cta] = red_abs[0];
      a.cand_row[par * a.P + cta] = my_row;
    }
    if (red_abs[0] >= 0.0) {
      const int li = my_row - (int)row0;
      for (int j = tid; j < nb; j += kPanelThreads) a.cand_data[((size_t)par * a.P + cta) * nb + j] = slab[j * rpc + li];
    }
    if (col >= row0 && col < row0 + nrow) {
      const int li = (int)(col - row0);
      for (int j = tid; j < nb; j += kPanelThreads) a.col_data[(size_t)par * nb + j] = slab[j * rpc + li];
    }
    if (!grid_barrier(a.bar, (unsigned)(c + 1) * a.P, a.timeout)) return;
    // global pivot: largest cabs1, first row on ties (izamax)
    if (tid == 0) {
      double gb = -1.0;
      int gr = 0x7fffffff, gc = -1;
      for (int p = 0; p < a.P; p++) {
        const double v = __ldcg(a.cand_abs + par * a.P + p);
        const int r = __ldcg(a.cand_row + par * a.P + p);
        if (v > gb || (v == gb && r < gr)) {
          gb = v;
          gr = r;
          gc = p;
        }
      }
      s_prow = gr;
      s_pcta = gc;
      if (cta == 0) {
        a.ipiv[col] = gr;
        if (gb == 0.0) atomicCAS(a.info, 0, (int)col + 1);
      }
    }
    __syncthreads();
    const int prow = s_prow, pcta = s_pcta;
    const double2 *pdat = a.cand_data + ((size_t)par * a.P + pcta) * nb;
    const double2 *cdat = a.col_data + (size_t)par * nb;
    // swap rows col <-> prow inside the panel
    if (prow != col && prow >= row0 && prow < row0 + nrow) {
      const int li = prow - (int)row0;
      for (int j = tid; j < nb; j += kPanelThreads) slab[j * rpc + li] = __ldcg(cdat + j);
    }
    if (col >= row0 && col < row0 + nrow) {
      const int li = (int)(col - row0);
      for (int j = tid; j < nb; j += kPanelThreads) slab[j * rpc + li] = __ldcg(pdat + j);
    }
    __syncthreads();
    const double2 piv = __ldcg(pdat + c);
    const double pa = piv.x * piv.x + piv.y * piv.y;
    if (pa != 0.0) {
      const double2 rp = make_double2(piv.x / pa, -piv.y / pa);  // 1 / pivot
      for (int i = tid; i < nrow; i += kPanelThreads) {
        const int64_t g = row0 + i;
        if (g <= col) continue;
        const double2 l = cmul(slab[c * rpc + i], rp);
        slab[c * rpc + i] = l;
        for (int j = c + 1; j < nb; j++) {
          const double2 u = __ldcg(pdat + j);
          double2 v = slab[j * rpc + i];
          v.x -= l.x * u.x - l.y * u.y;
          v.y -= l.x * u.y + l.y * u.x;
          slab[j * rpc + i] = v;
        }
      }
    }
    __syncthreads();
  }
  for (int idx = tid; idx < nb * rpc; idx += kPanelThreads) {
    const int c = idx / rpc, i = idx % rpc;
    if (i < nrow) st2(A + (row0 + i) + (a.j0 + c) * a.lda, slab[idx]);
  }
}

// Row interchanges ipiv[j0 .. j0+nb) applied, in order, to the columns
// outside the panel.
template <typename T>
__global__ void laswp_kernel(T *A, int64_t lda, int64_t n, int64_t j0, int nb, const int *ipiv) {
  int64_t col = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= n - nb) return;
  if (col >= j0) col += nb;
  T *a = A + col * lda;
  for (int c = 0; c < nb; c++) {
    const int64_t r = ipiv[j0 + c];
    if (r != j0 + c) {
      T t = a[j0 + c];
      a[j0 + c] = a[r];
      a[r] = t;
    }
  }
}

// Inverses of the unit-lower L11 and upper U11 diagonal blocks of the panel
// (FP64), stored as inv[0] = inv(L11), inv[1] = inv(U11), column-major nb x nb.
// One CTA, thread j computes column j.
template <typename T>
__global__ void diag_inv_kernel(const T *A, int64_t lda, int64_t j0, int nb, double2 *invL, double2 *invU,
                                float2 *invL32) {
  extern __shared__ double2 D[];  // nb x nb
  const int j = threadIdx.x;
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    const int r = idx % nb, c = idx / nb;
    D[idx] = ld2(A + (j0 + r) + (j0 + c) * lda);
  }
  __syncthreads();
  if (j >= nb) return;
  // inv(L): solve L x = e_j (unit diagonal)
  for (int i = 0; i < nb; i++) {
    double2 v = make_double2(i == j ? 1.0 : 0.0, 0.0);
    if (i > j) {
      for (int k = j; k < i; k++) {
        const double2 l = D[i + k * nb], x = invL[k + j * nb];
        v.x -= l.x * x.x - l.y * x.y;
        v.y -= l.x * x.y + l.y * x.x;
      }
    } else if (i < j) {
      v = make_double2(0, 0);
    }
    invL[i + j * nb] = v;
    if (invL32) invL32[i + j * nb] = make_float2((float)v.x, (float)v.y);
  }
  // inv(U): solve U x = e_j, i from j down to 0
  for (int i = nb - 1; i >= 0; i--) {
    double2 v = make_double2(0, 0);
    if (i <= j) {
      v = make_double2(i == j ? 1.0 : 0.0, 0.0);
      for (int k = i + 1; k <= j; k++) {
        const double2 u = D[i + k * nb], x = invU[k + j * nb];
        v.x -= u.x * x.x - u.y * x.y;
        v.y -= u.x * x.y + u.y * x.x;
      }
      const double2 d = D[i + i * nb];
      const double dd = d.x * d.x + d.y * d.y;
      v = (dd != 0.0) ? make_double2((v.x * d.x + v.y * d.y) / dd, (v.y * d.x - v.x * d.y) / dd) : make_double2(0, 0);
    }
    invU[i + j * nb] = v;
  }
}

// Forward / backward block substitution step (one launch per block):
//   y_k = Inv_k x_k   (every CTA recomputes it; CTA 0 stores it in Y)
//   x_i -= M[i, k-block] y_k for the rows i of the remaining range.
// lower: rows i >= (k+1) nb ; upper: rows i < k nb.  nrhs <= 8 per launch.
template <typename T>
__global__ void __launch_bounds__(256) trsv_step_kernel(const T *M, int64_t lda, int64_t n, int64_t k0, int nb,
                                                        const double2 *inv, double2 *X, double2 *Y, int64_t ldx,
                                                        int nrhs, int lower) {
  extern __shared__ double2 yk[];  // [nrhs][nb]
  for (int idx = threadIdx.x; idx < nb * nrhs; idx += blockDim.x) {
    const int r = idx % nb, s = idx / nb;
    double2 acc = make_double2(0, 0);
    for (int j = 0; j < nb; j++) {
      const double2 iv = inv[r + j * nb];
      const double2 xv = X[(size_t)s * ldx + k0 + j];
      acc.x += iv.x * xv.x - iv.y * xv.y;
      acc.y += iv.x * xv.y + iv.y * xv.x;
    }
    yk[s * nb + r] = acc;
  }
  __syncthreads();
  if (blockIdx.x == 0)
    for (int idx = threadIdx.x; idx < nb * nrhs; idx += blockDim.x) {
      const int r = idx % nb, s = idx / nb;
      Y[(size_t)s * ldx + k0 + r] = yk[s * nb + r];
    }
  const int64_t lo = lower ? k0 + nb : 0, hi = lower ? n : k0;
  for (int64_t i = lo + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += (int64_t)gridDim.x * blockDim.x) {
    double2 acc[8];
    for (int s = 0; s < nrhs; s++) acc[s] = make_double2(0, 0);
    for (int j = 0; j < nb; j++) {
      const double2 m = ld2(M + i + (k0 + j) * lda);
      for (int s = 0; s < nrhs; s++) {
        const double2 y = yk[s * nb + j];
        acc[s].x += m.x * y.x - m.y * y.y;
        acc[s].y += m.x * y.y + m.y * y.x;
      }
    }
    for (int s = 0; s < nrhs; s++) {
      double2 v = X[(size_t)s * ldx + i];
      v.x -= acc[s].x;
      v.y -= acc[s].y;
      X[(size_t)s * ldx + i] = v;
    }
  }
}

// X = P B (row interchanges of the whole factorisation, in order).
__global__ void apply_pivots_kernel(double2 *X, int64_t ldx, int64_t n, const int *ipiv, int nrhs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nrhs) return;
  double2 *x = X + (size_t)s * ldx;
  for (int64_t i = 0; i < n; i++) {
    const int64_t r = ipiv[i];
    if (r != i) {
      double2 t = x[i];
      x[i] = x[r];
      x[r] = t;
    }
  }
}

constexpr int kGemvRows = 256;
constexpr int kGemvCols = 256;

// partial[chunk][s][i] = sum_{j in chunk} A[i, j] x_s[j]  (FP64 matrix)
__global__ void __launch_bounds__(kGemvRows) gemv_partial_kernel(const double2 *A, int64_t lda, int64_t n,
                                                                 const double2 *X, int64_t ldx, int nrhs,
                                                                 double2 *partial) {
  __shared__ double2 xs[8][kGemvCols];
  const int64_t i = (int64_t)blockIdx.x * kGemvRows + threadIdx.x;
  const int64_t j0 = (int64_t)blockIdx.y * kGemvCols;
  const int cnt = (n - j0) < kGemvCols ? (int)(n - j0) : kGemvCols;
  for (int idx = threadIdx.x; idx < cnt * nrhs; idx += kGemvRows) {
    const int j = idx % cnt, s = idx / cnt;
    xs[s][j] = X[(size_t)s * ldx + j0 + j];
  }
  __syncthreads();
  if (i >= n) return;
  double2 acc[8];
  for (int s = 0; s < nrhs; s++) acc[s] = make_double2(0, 0);
  for (int j = 0; j < cnt; j++) {
    const double2 m = A[i + (j0 + j) * lda];
    for (int s = 0; s < nrhs; s++) {
      const double2 x = xs[s][j];
      acc[s].x += m.x * x.x - m.y * x.y;
      acc[s].y += m.x * x.y + m.y * x.x;
    }
  }
  for (int s = 0; s < nrhs; s++) partial[((size_t)blockIdx.y * nrhs + s) * n + i] = acc[s];
}

// R = B - sum of partials; per-column squared norms of R into rn (block partials).
__global__ void residual_kernel(const double2 *B, int64_t ldb, const double2 *partial, int nchunk, int64_t n,
                                int nrhs, double2 *R, int64_t ldr, double *rn2) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  double v2 = 0;
  if (i < n) {
    double2 acc = B[(size_t)s * ldb + i];
    for (int c = 0; c < nchunk; c++) {
      const double2 p = partial[((size_t)c * nrhs + s) * n + i];
      acc.x -= p.x;
      acc.y -= p.y;
    }
    R[(size_t)s * ldr + i] = acc;
    v2 = acc.x * acc.x + acc.y * acc.y;
  }
  __shared__ double red[256];
  red[threadIdx.x] = v2;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) rn2[(size_t)s * gridDim.x + blockIdx.x] = red[0];
}

__global__ void axpy_kernel(double2 *X, const double2 *D, int64_t count) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t st = (int64_t)gridDim.x * blockDim.x;
  for (; i < count; i += st) {
    X[i].x += D[i].x;
    X[i].y += D[i].y;
  }
}

struct LuWork {
  unsigned *bar;
  int *info, *timeout;
  double *cand_abs;
  int *cand_row;
  double2 *cand_data, *col_data;
  double2 *W;      // nb x n workspace for the TRSM product
  float2 *invL32;  // nb x nb
};

int lu_workspace(Ctx *c, int precision, LuWork &w) {
  const int nb = c->nb, P = c->nsm;
  const size_t esz = precision == MOM_PREC_MIXED ? sizeof(float2) : sizeof(double2);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) / 256 * 256;
    return o;
  };
  const size_t o_bar = take(sizeof(unsigned) * 4);
  const size_t o_ca = take(sizeof(double) * 2 * P);
  const size_t o_cr = take(sizeof(int) * 2 * P);
  const size_t o_cd = take(sizeof(double2) * 2 * P * nb);
  const size_t o_cl = take(sizeof(double2) * 2 * nb);
  const size_t o_w = take(esz * (size_t)nb * c->n);
  const size_t o_i32 = take(sizeof(float2) * nb * nb);
  MOM_TRY(ensure_buffer(c, &c->ws, &c->ws_bytes, off));
  char *b = (char *)c->ws;
  w.bar = (unsigned *)(b + o_bar);
  w.info = c->dinfo;
  w.timeout = c->dinfo + 1;
  w.cand_abs = (double *)(b + o_ca);
  w.cand_row = (int *)(b + o_cr);
  w.cand_data = (double2 *)(b + o_cd);
  w.col_data = (double2 *)(b + o_cl);
  w.W = (double2 *)(b + o_w);
  w.invL32 = (float2 *)(b + o_i32);
  return MOM_OK;
}

template <typename T>
int lu_factor_t(Ctx *c, T *A, int precision) {
  const int64_t n = c->n, lda = c->lda;
  const int nb = c->nb;
  if (n % nb != 0) return fail(c, MOM_ERR_ARG, "matrix order must be a multiple of the panel width");
  LuWork w;
  MOM_TRY(lu_workspace(c, precision, w));
  MOM_CUDA(c, cudaMemsetAsync(c->dinfo, 0, sizeof(int) * 4, c->stream));
  const bool mixed = precision == MOM_PREC_MIXED;
  MOM_BLAS(c, cublasSetMathMode(c->blas, mixed ? CUBLAS_TF32_TENSOR_OP_MATH : CUBLAS_DEFAULT_MATH));
  const int nblk = (int)(n / nb);
  for (int kb = 0; kb < nblk; kb++) {
    const int64_t j0 = (int64_t)kb * nb;
    const int64_t m = n - j0;
    int P = (int)std::min<int64_t>(c->nsm, (m + 31) / 32);
    int rpc = (int)((m + P - 1) / P);
    P = (int)((m + rpc - 1) / rpc);
    const size_t smem = sizeof(double2) * (size_t)nb * rpc;
    if (smem > 227 * 1024) return fail(c, MOM_ERR_ARG, "panel does not fit in shared memory");
    PanelArgs pa;
    pa.A = A;
    pa.lda = lda;
    pa.n = n;
    pa.j0 = j0;
    pa.nb = nb;
    pa.rpc = rpc;
    pa.P = P;
    pa.ipiv = c->ipiv;
    pa.info = w.info;
    pa.timeout = w.timeout;
    pa.bar = w.bar;
    pa.cand_abs = w.cand_abs;
    pa.cand_row = w.cand_row;
    pa.cand_data = w.cand_data;
    pa.col_data = w.col_data;
    MOM_CUDA(c, cudaMemsetAsync(w.bar, 0, sizeof(unsigned), c->stream));
    MOM_CUDA(c, cudaFuncSetAttribute(panel_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    void *args[] = {&pa};
    MOM_CUDA(c, cudaLaunchCooperativeKernel((void *)panel_kernel<T>, dim3(P), dim3(kPanelThreads), args, smem,
                                            c->stream));
    c->launches++;
    if (n > nb) {
      laswp_kernel<T><<<(unsigned)((n - nb + 255) / 256), 256, 0, c->stream>>>(A, lda, n, j0, nb, c->ipiv);
      c->launches++;
    }
    double2 *invL = c->invd + (size_t)kb * 2 * nb * nb, *invU = invL + (size_t)nb * nb;
    MOM_CUDA(c, cudaFuncSetAttribute(diag_inv_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(sizeof(double2) * nb * nb)));
    diag_inv_kernel<T><<<1, std::max(nb, 64), sizeof(double2) * nb * nb, c->stream>>>(A, lda, j0, nb, invL, invU,
                                                                                     mixed ? w.invL32 : nullptr);
    c->launches++;
    MOM_CUDA(c, cudaGetLastError());
    const int64_t nc = n - j0 - nb;  // trailing columns
    if (nc > 0) {
      T *A12 = A + j0 + (j0 + nb) * lda;
      T *L21 = A + (j0 + nb) + j0 * lda;
      T *A22 = A + (j0 + nb) + (j0 + nb) * lda;
      if (!mixed) {
        const cuDoubleComplex one = make_cuDoubleComplex(1, 0), zero = make_cuDoubleComplex(0, 0),
                              mone = make_cuDoubleComplex(-1, 0);
        MOM_BLAS(c, cublasZgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, nb, (int)nc, nb, &one, (cuDoubleComplex *)invL, nb,
                                (cuDoubleComplex *)A12, (int)lda, &zero, (cuDoubleComplex *)w.W, nb));
        MOM_CUDA(c, cudaMemcpy2DAsync(A12, sizeof(T) * lda, w.W, sizeof(T) * nb, sizeof(T) * nb, nc,
                                      cudaMemcpyDeviceToDevice, c->stream));
        MOM_BLAS(c, cublasZgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)(m - nb), (int)nc, nb, &mone,
                                (cuDoubleComplex *)L21, (int)lda, (cuDoubleComplex *)A12, (int)lda, &one,
                                (cuDoubleComplex *)A22, (int)lda));
      } else {
        const cuComplex one = make_cuComplex(1, 0), zero = make_cuComplex(0, 0), mone = make_cuComplex(-1, 0);
        MOM_BLAS(c, cublasCgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, nb, (int)nc, nb, &one, (cuComplex *)w.invL32, nb,
                                (cuComplex *)A12, (int)lda, &zero, (cuComplex *)w.W, nb));
        MOM_CUDA(c, cudaMemcpy2DAsync(A12, sizeof(T) * lda, w.W, sizeof(T) * nb, sizeof(T) * nb, nc,
                                      cudaMemcpyDeviceToDevice, c->stream));
        MOM_BLAS(c, cublasCgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)(m - nb), (int)nc, nb, &mone,
                                (cuComplex *)L21, (int)lda, (cuComplex *)A12, (int)lda, &one, (cuComplex *)A22,
                                (int)lda));
      }
      c->launches += 3;
    }
  }
  MOM_BLAS(c, cublasSetMathMode(c->blas, CUBLAS_DEFAULT_MATH));
  int hinfo[2] = {0, 0};
  MOM_CUDA(c, cudaMemcpyAsync(hinfo, c->dinfo, sizeof(int) * 2, cudaMemcpyDeviceToHost, c->stream));
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  if (hinfo[1]) return fail(c, MOM_ERR_TIMEOUT, "panel factorisation barrier timed out");
  if (hinfo[0]) {
    c->factored = -1;
    return fail(c, MOM_ERR_SINGULAR, "Matrix factorization failed! (zero pivot at column " + std::to_string(hinfo[0]) + ")");
  }
  c->factored = precision;
  return MOM_OK;
}

// X (n x nrhs, ld n) <- A^{-1} X with the factors in place; Y is scratch.
template <typename T>
int getrs_t(Ctx *c, const T *A, double2 *X, double2 *Y, int nrhs) {
  const int64_t n = c->n, lda = c->lda;
  const int nb = c->nb, nblk = (int)(n / nb);
  apply_pivots_kernel<<<(nrhs + 31) / 32, 32, 0, c->stream>>>(X, n, n, c->ipiv, nrhs);
  c->launches++;
  for (int s0 = 0; s0 < nrhs; s0 += 8) {
    const int ns = std::min(8, nrhs - s0);
    double2 *x = X + (size_t)s0 * n, *y = Y + (size_t)s0 * n;
    const size_t smem = sizeof(double2) * nb * ns;
    for (int kb = 0; kb < nblk; kb++) {
      const int64_t k0 = (int64_t)kb * nb;
      const int64_t rows = n - k0 - nb;
      const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>((rows + 255) / 256, 2 * c->nsm));
      trsv_step_kernel<T><<<g, 256, smem, c->stream>>>(A, lda, n, k0, nb, c->invd + (size_t)kb * 2 * nb * nb, x, y, n,
                                                       ns, 1);
      c->launches++;
    }
    for (int kb = nblk - 1; kb >= 0; kb--) {
      const int64_t k0 = (int64_t)kb * nb;
      const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>((k0 + 255) / 256, 2 * c->nsm));
      trsv_step_kernel<T><<<g, 256, smem, c->stream>>>(A, lda, n, k0, nb,
                                                       c->invd + (size_t)kb * 2 * nb * nb + (size_t)nb * nb, y, x, n,
                                                       ns, 0);
      c->launches++;
    }
  }
  MOM_CUDA(c, cudaGetLastError());
  return MOM_OK;
}

}  // namespace

int lu_factor(Ctx *c, int precision) {
  if (precision == MOM_PREC_MIXED) return lu_factor_t<float2>(c, c->A32, precision);
  return lu_factor_t<double2>(c, c->A, precision);
}

// Solve for the nsrc right-hand sides in c->B into c->X.
int lu_solve(Ctx *c, int precision, double tol, int maxit, int *iters) {
  const int64_t n = c->n;
  const int nrhs = c->nsrc;
  if (c->factored != precision) return fail(c, MOM_ERR_STATE, "matrix not factored in this precision");
  const size_t vec = sizeof(double2) * (size_t)n * nrhs;
  if (precision == MOM_PREC_FP64) {
    MOM_CUDA(c, cudaMemcpyAsync(c->X, c->B, vec, cudaMemcpyDeviceToDevice, c->stream));
    MOM_TRY(ensure_buffer(c, &c->ws, &c->ws_bytes, vec));
    MOM_TRY(getrs_t<double2>(c, c->A, c->X, (double2 *)c->ws, nrhs));
    if (iters) *iters = 0;
    return MOM_OK;
  }
  // Mixed: x = 0, r = b; repeat d = LU32^{-1} r, x += d, r = b - A x.
  const int nchunk = (int)((n + kGemvCols - 1) / kGemvCols);
  const int rblocks = (int)((n + 255) / 256);
  const size_t off_r = 0, off_d = vec, off_y = 2 * vec, off_p = 3 * vec;
  const size_t part = sizeof(double2) * (size_t)nchunk * 8 * n;
  const size_t off_n = off_p + part;
  MOM_TRY(ensure_buffer(c, &c->ws, &c->ws_bytes, off_n + sizeof(double) * rblocks * nrhs + 256));
  char *ws = (char *)c->ws;
  double2 *R = (double2 *)(ws + off_r), *Dv = (double2 *)(ws + off_d), *Yv = (double2 *)(ws + off_y),
          *Pp = (double2 *)(ws + off_p);
  double *rn2 = (double *)(ws + off_n);
  // ||b|| per column
  std::vector<double> bn(nrhs), h(rblocks * (size_t)nrhs);
  MOM_CUDA(c, cudaMemsetAsync(c->X, 0, vec, c->stream));
  MOM_CUDA(c, cudaMemcpyAsync(R, c->B, vec, cudaMemcpyDeviceToDevice, c->stream));
  residual_kernel<<<dim3(rblocks, nrhs), 256, 0, c->stream>>>(c->B, n, Pp, 0, n, nrhs, R, n, rn2);
  c->launches++;
  MOM_CUDA(c, cudaMemcpyAsync(h.data(), rn2, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream));
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  for (int s = 0; s < nrhs; s++) {
    double t = 0;
    for (int b = 0; b < rblocks; b++) t += h[(size_t)s * rblocks + b];
    bn[s] = std::sqrt(t);
  }
  int it = 0;
  double worst = 1.0;
  for (it = 1; it <= maxit; it++) {
    MOM_CUDA(c, cudaMemcpyAsync(Dv, R, vec, cudaMemcpyDeviceToDevice, c->stream));
    MOM_TRY(getrs_t<float2>(c, c->A32, Dv, Yv, nrhs));
    axpy_kernel<<<c->nsm * 4, 256, 0, c->stream>>>(c->X, Dv, (int64_t)n * nrhs);
    c->launches++;
    for (int s0 = 0; s0 < nrhs; s0 += 8) {
      const int ns = std::min(8, nrhs - s0);
      gemv_partial_kernel<<<dim3(rblocks, nchunk), kGemvRows, 0, c->stream>>>(c->A, c->lda, n, c->X + (size_t)s0 * n,
                                                                               n, ns, Pp);
      residual_kernel<<<dim3(rblocks, ns), 256, 0, c->stream>>>(c->B + (size_t)s0 * n, n, Pp, nchunk, n, ns,
                                                                R + (size_t)s0 * n, n, rn2 + (size_t)s0 * rblocks);
      c->launches += 2;
    }
    MOM_CUDA(c, cudaGetLastError());
    MOM_CUDA(c, cudaMemcpyAsync(h.data(), rn2, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream));
    MOM_CUDA(c, cudaStreamSynchronize(c->stream));
    worst = 0;
    for (int s = 0; s < nrhs; s++) {
      double t = 0;
      for (int b = 0; b < rblocks; b++) t += h[(size_t)s * rblocks + b];
      worst = std::max(worst, bn[s] > 0 ? std::sqrt(t) / bn[s] : 0.0);
    }
    if (worst <= tol) break;
  }
  if (iters) *iters = std::min(it, maxit);
  if (worst > tol) {
    char buf[160];
    snprintf(buf, sizeof buf, "iterative refinement stopped at relative residual %.3e > %.3e", worst, tol);
    return fail(c, MOM_ERR_NOCONV, buf);
  }
  return MOM_OK;
}

}  // namespace mom
