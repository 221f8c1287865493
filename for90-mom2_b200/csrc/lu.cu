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
#include <chrono>
#include <cmath>
#include <cstdlib>
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
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double cabs1(float2 a) { return (double)(fabsf(a.x) + fabsf(a.y)); }
__device__ __forceinline__ void st2(float2 *p, float2 v) { *p = v; }
__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2(v.x, v.y); }
template <typename E> __device__ __forceinline__ E from_d2(double2 v);
template <> __device__ __forceinline__ double2 from_d2<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 from_d2<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }
template <typename E> __device__ __forceinline__ E ld_slab(const double2 *p) { return from_d2<E>(*p); }
template <typename E> __device__ __forceinline__ E ld_slab(const float2 *p);
template <> __device__ __forceinline__ float2 ld_slab<float2>(const float2 *p) { return *p; }
template <> __device__ __forceinline__ double2 ld_slab<double2>(const float2 *p) { return to_d2(*p); }

// Element type of a panel's shared-memory slab: the FP64 factorisation works
// in FP64; the mixed path's FP32 factors are factored in FP32 arithmetic
// (what the tensor-core trailing updates keep), which halves the slab and so
// the CTAs a panel needs.
template <typename T> struct SlabOf { using type = double2; };
template <> struct SlabOf<float2> { using type = float2; };
// Rows per CTA that fit a 64-column slab in the 222 KB the panel kernel gets.
template <typename T> constexpr int64_t kPanelMaxRows = sizeof(typename SlabOf<T>::type) == 8 ? 416 : 208;

constexpr int kPanelThreads = 512;
constexpr long long kSpinLimit = 1LL << 26;  // default bound of a barrier wait (a few seconds)

struct PanelArgs {
  void *A;
  int64_t lda, n, j0;
  int nb, rpc, P;
  int *ipiv;
  int *info;      // first zero pivot (1-based), 0 if none
  int *timeout;   // set when a barrier wait ran out
  long long spin; // polls before a wait is declared timed out
  unsigned long long *rec;  // [2][P] candidate records, zeroed before launch
  double2 *cand_data;       // [2][P][nb]
  double2 *col_data;        // [2][nb]
};

// A CTA's pivot candidate for one column as one 64-bit word, so that seeing
// the arrival and reading the candidate is a single load:
//   bits 63..32  float bits of |re|+|im| plus one (0: no candidate),
//   bits 31..8   0xffffff - (row - j0)  (ties go to the smaller row),
//   bits  7..0   column epoch c + 1.
// Comparing words >> 8 as unsigned integers orders candidates by magnitude,
// then by the smaller row.  Within a CTA the magnitude is compared in FP64;
// across CTAs in its FP32 rounding.
__device__ __forceinline__ unsigned long long pack_candidate(double v, int64_t row, int64_t j0, int epoch) {
  const unsigned long long mag = v >= 0.0 ? (unsigned long long)__float_as_uint((float)v) + 1ull : 0ull;
  return (mag << 32) | ((unsigned long long)((0xffffffu - (unsigned)(row - j0)) & 0xffffffu) << 8) |
         (unsigned)epoch;
}

// (value, row) pair reduction: larger |re|+|im| wins, the first row on ties.
__device__ __forceinline__ void argmax_warp(double &v, int &r, int &w) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_down_sync(0xffffffffu, v, o);
    const int orow = __shfl_down_sync(0xffffffffu, r, o);
    const int ow = __shfl_down_sync(0xffffffffu, w, o);
    if (ov > v || (ov == v && orow < r)) {
      v = ov;
      r = orow;
      w = ow;
    }
  }
}

// Largest packed candidate over a warp: the magnitude word first, then the
// row word among the lanes that hold that magnitude (two warp reductions).
__device__ __forceinline__ unsigned long long warp_max_key(unsigned long long k) {
  const unsigned hi = (unsigned)(k >> 32);
  const unsigned mh = __reduce_max_sync(0xffffffffu, hi);
  const unsigned ml = __reduce_max_sync(0xffffffffu, hi == mh ? (unsigned)k : 0u);
  return ((unsigned long long)mh << 32) | ml;
}

// Panel factorisation (unblocked, partial pivoting) of columns j0 .. j0+nb
// over rows j0 .. n, cooperative over P CTAs; CTA p holds rows
// [j0 + p rpc, j0 + (p+1) rpc) of the panel in shared memory.  Thread t
// works on row t % rpc and on the columns j = t / rpc (mod S), S = 256 / rpc
// threads per row, so short panels keep every thread busy.  Per column:
// CTA argmax, one packed record per CTA exchanged through global memory,
// row swap, scaling and the rank-1 update of the CTA's rows.
template <typename T>
__global__ void __launch_bounds__(kPanelThreads, 1) panel_kernel(PanelArgs a) {
  using E = typename SlabOf<T>::type;
  extern __shared__ __align__(16) unsigned char panel_smem[];
  E *slab = reinterpret_cast<E *>(panel_smem);  // [nb][rpc] column-major within the CTA
  __shared__ unsigned long long w_key[kPanelThreads / 32];
  __shared__ E s_prow_data[64];
  __shared__ E s_rpc[64];  // 1 / pivot of each column (0: failed pivot)
  __shared__ E s_rp;
  __shared__ int s_ok;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, cta = blockIdx.x;
  const int nb = a.nb, rpc = a.rpc;
  T *A = reinterpret_cast<T *>(a.A);
  const int64_t row0 = a.j0 + (int64_t)cta * rpc;
  const int64_t rem = a.n - row0;
  const int nrow = rem <= 0 ? 0 : (rem < rpc ? (int)rem : rpc);
  for (int base = tid; base < nb * rpc; base += 8 * kPanelThreads) {
    E v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * kPanelThreads;
      const int c = idx / rpc, i = idx % rpc;
      v[u] = (idx < nb * rpc && i < nrow) ? ld_slab<E>(A + (row0 + i) + (a.j0 + c) * a.lda)
                                          : from_d2<E>(make_double2(0, 0));
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * kPanelThreads;
      if (idx < nb * rpc) slab[idx] = v[u];
    }
  }
  __syncthreads();
  const int S = kPanelThreads / rpc;  // threads per row (rpc <= kPanelThreads)
  const int i = tid % rpc, sph = tid / rpc;
  const bool mine = sph < S && i < nrow;
  const int64_t g = row0 + i;  // global row of this thread
  double cv = (mine && sph == 0) ? cabs1(slab[i]) : -1.0;  // candidate for column 0
  for (int c = 0; c < nb; c++) {
    const int64_t col = a.j0 + c;
    const int par = c & 1;
    // 1. CTA candidate (packed: magnitude, then the smaller row)
    const unsigned long long wk = warp_max_key(cv >= 0.0 ? pack_candidate(cv, g, a.j0, 0) : 0ull);
    if (lane == 0) w_key[wid] = wk;
    __syncthreads();
    if (wid == 0) {
      const unsigned long long bkey = warp_max_key(lane < kPanelThreads / 32 ? w_key[lane] : 0ull);
      // 2. publish the candidate row data (and row col, if owned), then the
      //    record; the release store orders the whole warp's stores before it
      if (bkey != 0ull) {
        const int li = (int)(0xffffffu - (unsigned)((bkey >> 8) & 0xffffffu)) - (int)(row0 - a.j0);
        for (int j = lane; j < nb; j += 32) a.cand_data[((size_t)par * a.P + cta) * nb + j] = to_d2(slab[j * rpc + li]);
      }
      if (col >= row0 && col < row0 + nrow) {
        const int li = (int)(col - row0);
        for (int j = lane; j < nb; j += 32) a.col_data[(size_t)par * nb + j] = to_d2(slab[j * rpc + li]);
      }
      __syncwarp();
      unsigned long long *rec = a.rec + (size_t)par * a.P;
      if (lane == 0) {
        const unsigned long long word = bkey | (unsigned)(c + 1);
        asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(rec + cta), "l"(word) : "memory");
      }
      // 3. wait for all P records of this column (acquire loads); lane l
      //    keeps the best of records l, l + 32, ...
      unsigned long long best = 0;
      int bw = -1;
      unsigned pending = 0;
      for (int q = 0; q < 8; q++)
        if (lane + 32 * q < a.P) pending |= 1u << q;
      long long it = 0;
      int ok = 1;
      // the row of the best record seen so far is fetched while the others
      // arrive (its data is visible once its record is: release / acquire)
      unsigned long long pf_key = 0;
      double2 pf0 = make_double2(0, 0), pf1 = make_double2(0, 0);
      while (true) {
#pragma unroll
        for (int q = 0; q < 8; q++) {
          if (!(pending >> q & 1u)) continue;
          unsigned long long wv;
          asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(wv) : "l"(rec + lane + 32 * q) : "memory");
          if ((int)(wv & 0xffu) == c + 1) {
            pending &= ~(1u << q);
            if (bw < 0 || (wv >> 8) > (best >> 8)) {
              best = wv;
              bw = lane + 32 * q;
            }
          }
        }
        const bool done = __all_sync(0xffffffffu, pending == 0);
        const unsigned long long rk = warp_max_key(bw >= 0 ? (best & ~0xffull) : 0ull);
        if (rk != 0ull && rk != pf_key) {
          const int rw = __ffs(__ballot_sync(0xffffffffu, bw >= 0 && (best & ~0xffull) == rk)) - 1;
          const int rcta = __shfl_sync(0xffffffffu, bw, rw);
          const double2 *pd = a.cand_data + ((size_t)par * a.P + rcta) * nb;
          pf0 = __ldcg(pd + lane);
          pf1 = __ldcg(pd + lane + 32);
          pf_key = rk;
        }
        if (done) break;
        if ((++it & 255) == 0 || it > a.spin) {
          int stop = 0;
          if (lane == 0) {
            if (*(volatile int *)a.timeout) stop = 1;
            else if (it > a.spin) {
              atomicExch(a.timeout, 1);
              stop = 1;
            }
          }
          if (__shfl_sync(0xffffffffu, stop, 0)) {
            ok = 0;
            break;
          }
        }
      }
      if (ok) {
        // global pivot: the largest record; its CTA index travels with it
        const unsigned long long gkey = warp_max_key(bw >= 0 ? (best & ~0xffull) : 0ull);
        const int gw = __ffs(__ballot_sync(0xffffffffu, bw >= 0 && (best & ~0xffull) == gkey)) - 1;
        const int gcta = gw < 0 ? 0 : __shfl_sync(0xffffffffu, bw, gw);
        // no candidate at all (every entry of the column NaN): no interchange,
        // reported as a failed pivot, so ipiv stays within the panel's rows
        const bool none = gkey == 0ull;
        const int gr = none ? (int)col : (int)a.j0 + (int)(0xffffffu - (unsigned)((gkey >> 8) & 0xffffffu));
        const double2 *pdat = a.cand_data + ((size_t)par * a.P + gcta) * nb;
        const double2 *cdat = a.col_data + (size_t)par * nb;
        const bool own_p = gr != col && gr >= row0 && gr < row0 + nrow;
        const bool own_c = col >= row0 && col < row0 + nrow;
        const bool have = pf_key == gkey;  // the final best was prefetched
        for (int j = lane; j < nb; j += 32) {
          const double2 pv = none ? __ldcg(cdat + j) : have ? (j < 32 ? pf0 : pf1) : __ldcg(pdat + j);
          const double2 cvv = own_p ? __ldcg(cdat + j) : make_double2(0, 0);
          s_prow_data[j] = from_d2<E>(pv);
          if (own_p) slab[j * rpc + (gr - (int)row0)] = from_d2<E>(cvv);  // row prow <- old row col
          if (own_c) slab[j * rpc + (int)(col - row0)] = from_d2<E>(pv);  // row col  <- pivot row
          if (j == c) {
            // 1 / pivot, formed in FP64 (|pivot|^2 cannot underflow)
            const double pa = none ? 0.0 : pv.x * pv.x + pv.y * pv.y;
            s_rp = from_d2<E>(pa != 0.0 ? make_double2(pv.x / pa, -pv.y / pa) : make_double2(0, 0));
            s_rpc[c] = s_rp;
            if (cta == 0 && pa == 0.0) atomicCAS(a.info, 0, (int)col + 1);
          }
        }
        if (lane == 0 && cta == 0) a.ipiv[col] = gr;
      }
      if (lane == 0) s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) return;
    // 4. rank-1 update of columns c+1 .. nb, S threads per row, with the
    //    multiplier l = a(i, c) / pivot formed by each of them; column c keeps
    //    a(i, c) until the final store scales it (the same product, so the
    //    factors are unchanged) and needs no barrier of its own
    const E rp = s_rp;
    const bool live = mine && g > col && (rp.x != 0 || rp.y != 0);
    cv = -1.0;
    const int own = (c + 1) % S;  // phase of the thread that holds column c+1
    if (mine && g > col) {
      const int jst = c + 1 + ((sph - (c + 1)) % S + S) % S;
      if (live) {
        const E l = cmul(slab[c * rpc + i], rp);
        for (int j = jst; j < nb; j += 4 * S) {
          E x[4];
#pragma unroll
          for (int u = 0; u < 4; u++)
            if (j + u * S < nb) x[u] = slab[(j + u * S) * rpc + i];
#pragma unroll
          for (int u = 0; u < 4; u++)
            if (j + u * S < nb) {
              const E uu = s_prow_data[j + u * S];
              x[u].x -= l.x * uu.x - l.y * uu.y;
              x[u].y -= l.x * uu.y + l.y * uu.x;
              slab[(j + u * S) * rpc + i] = x[u];
            }
        }
      }
      if (sph == own && c + 1 < nb) cv = cabs1(slab[(c + 1) * rpc + i]);
    }
  }
  __syncthreads();
  // L below the diagonal scaled by its column's 1 / pivot on the way out
  for (int idx = tid; idx < nb * rpc; idx += kPanelThreads) {
    const int c = idx / rpc, ii = idx % rpc;
    if (ii < nrow) {
      const E v = slab[idx], rp = s_rpc[c];
      const bool low = row0 + ii > a.j0 + c && (rp.x != 0 || rp.y != 0);
      st2(A + (row0 + ii) + (a.j0 + c) * a.lda, low ? cmul(v, rp) : v);
    }
  }
}

// ---- short panels: one thread-block cluster, exchange in distributed shared memory ----

constexpr int kMaxCluster = 16;
// rows per CTA of a cluster panel (slab + pushed rows in shared memory): 176
// with the FP64 slab, 352 with the FP32 slab of the mixed path
template <typename T> constexpr int kClusterRows = sizeof(typename SlabOf<T>::type) == 8 ? 352 : 176;

__device__ __forceinline__ unsigned map_shared(const void *p, unsigned rank) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_cluster_u64(unsigned addr, unsigned long long v) {
  asm volatile("st.shared::cluster.u64 [%0], %1;" ::"r"(addr), "l"(v) : "memory");
}
__device__ __forceinline__ double2 ld_cluster_d2(unsigned addr) {
  double2 v;
  asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(addr) : "memory");
  return v;
}
// Every thread of every CTA of the cluster; orders shared-memory accesses
// across the cluster (release / acquire).
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ void st_cluster_d2(unsigned addr, double2 v) {
  asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(addr), "d"(v.x), "d"(v.y) : "memory");
}
__device__ __forceinline__ void st_cluster_d2(unsigned addr, float2 v) {
  asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(v.x), "f"(v.y) : "memory");
}

// The same panel factorisation as panel_kernel for panels of at most
// kClusterRows<T> * kMaxCluster rows, on a grid that is exactly one cluster of
// P CTAs (all co-scheduled by the hardware).  Per column each CTA pushes
// its packed candidate key and the candidate row (and the owner of row col
// that row) into every CTA's shared memory, then one cluster barrier; the
// winner, the pivot row and the displaced row are then read locally.  The
// pushed buffers alternate by column parity, so one barrier per column
// suffices.  No global memory round trip and no spin-wait: every thread of
// the cluster executes the same sequence of cluster barriers.
template <typename T>
__global__ void __launch_bounds__(kPanelThreads, 1) panel_cluster_kernel(PanelArgs a) {
  using E = typename SlabOf<T>::type;
  extern __shared__ __align__(16) unsigned char cluster_smem[];
  E *slab = reinterpret_cast<E *>(cluster_smem);  // [nb][rpc] column-major, then the pushed rows
  __shared__ unsigned long long w_key[kPanelThreads / 32];
  __shared__ unsigned long long c_key[2][kMaxCluster];
  __shared__ E s_prow_data[64];
  __shared__ E s_rpc[64];  // 1 / pivot of each column (0: failed pivot)
  __shared__ E s_rp;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, cta = blockIdx.x;  // cta == cluster rank
  const int nb = a.nb, rpc = a.rpc, P = a.P;
  E *recv_row = slab + (size_t)nb * rpc;           // [2][P][nb] candidate rows by sender
  E *recv_col = recv_row + (size_t)2 * P * nb;    // [2][nb] row col, from its owner
  T *A = reinterpret_cast<T *>(a.A);
  const int64_t row0 = a.j0 + (int64_t)cta * rpc;
  const int64_t rem = a.n - row0;
  const int nrow = rem <= 0 ? 0 : (rem < rpc ? (int)rem : rpc);
  for (int base = tid; base < nb * rpc; base += 8 * kPanelThreads) {
    E v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * kPanelThreads;
      const int c = idx / rpc, i = idx % rpc;
      v[u] = (idx < nb * rpc && i < nrow) ? ld_slab<E>(A + (row0 + i) + (a.j0 + c) * a.lda)
                                          : from_d2<E>(make_double2(0, 0));
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * kPanelThreads;
      if (idx < nb * rpc) slab[idx] = v[u];
    }
  }
  __syncthreads();
  const int S = kPanelThreads / rpc;  // threads per row (rpc <= kPanelThreads)
  const int i = tid % rpc, sph = tid / rpc;
  const bool mine = sph < S && i < nrow;
  const int64_t g = row0 + i;  // global row of this thread
  double cv = (mine && sph == 0) ? cabs1(slab[i]) : -1.0;  // candidate for column 0
  for (int c = 0; c < nb; c++) {
    const int64_t col = a.j0 + c;
    const int par = c & 1;
    // 1. CTA candidate; push key and row (and row col, if owned) to every CTA
    const unsigned long long wk = warp_max_key(cv >= 0.0 ? pack_candidate(cv, g, a.j0, 0) : 0ull);
    if (lane == 0) w_key[wid] = wk;
    __syncthreads();
    if (wid == 0) {
      const unsigned long long bkey = warp_max_key(lane < kPanelThreads / 32 ? w_key[lane] : 0ull);
      if (lane < P) st_cluster_u64(map_shared(&c_key[par][cta], (unsigned)lane), bkey);
      if (bkey != 0ull) {
        const int li = (int)(0xffffffu - (unsigned)((bkey >> 8) & 0xffffffu)) - (int)(row0 - a.j0);
        const E v0 = slab[lane * rpc + li], v1 = slab[(lane + 32) * rpc + li];
        E *dst = recv_row + ((size_t)par * P + cta) * nb;
        for (int t = 0; t < P; t++) {
          const unsigned base = map_shared(dst, (unsigned)t);
          st_cluster_d2(base + (unsigned)(lane * sizeof(E)), v0);
          st_cluster_d2(base + (unsigned)((lane + 32) * sizeof(E)), v1);
        }
      }
      if (col >= row0 && col < row0 + nrow) {
        const int li = (int)(col - row0);
        const E v0 = slab[lane * rpc + li], v1 = slab[(lane + 32) * rpc + li];
        E *dst = recv_col + (size_t)par * nb;
        for (int t = 0; t < P; t++) {
          const unsigned base = map_shared(dst, (unsigned)t);
          st_cluster_d2(base + (unsigned)(lane * sizeof(E)), v0);
          st_cluster_d2(base + (unsigned)((lane + 32) * sizeof(E)), v1);
        }
      }
    }
    cluster_sync();
    // 2. the winner, read locally; swap
    if (wid == 0) {
      const unsigned long long k = lane < P ? c_key[par][lane] : 0ull;
      const unsigned long long gkey = warp_max_key(k);
      const int gw = __ffs(__ballot_sync(0xffffffffu, lane < P && k == gkey)) - 1;
      const int gsrc = gw < 0 ? 0 : gw;
      // no candidate (every entry of the column NaN): no interchange, failed pivot
      const bool none = gkey == 0ull;
      const int gr = none ? (int)col : (int)a.j0 + (int)(0xffffffu - (unsigned)((gkey >> 8) & 0xffffffu));
      const bool own_p = gr != col && gr >= row0 && gr < row0 + nrow;
      const bool own_c = col >= row0 && col < row0 + nrow;
      const E *prow = recv_row + ((size_t)par * P + gsrc) * nb, *crow = recv_col + (size_t)par * nb;
      for (int j = lane; j < nb; j += 32) {
        const E pv = none ? crow[j] : prow[j];
        s_prow_data[j] = pv;
        if (own_p) slab[j * rpc + (gr - (int)row0)] = crow[j];  // row prow <- old row col
        if (own_c) slab[j * rpc + (int)(col - row0)] = pv;      // row col  <- pivot row
        if (j == c) {
          // 1 / pivot, formed in FP64
          const double2 pd = to_d2(pv);
          const double pa = none ? 0.0 : pd.x * pd.x + pd.y * pd.y;
          s_rp = from_d2<E>(pa != 0.0 ? make_double2(pd.x / pa, -pd.y / pa) : make_double2(0, 0));
          s_rpc[c] = s_rp;
          if (cta == 0 && pa == 0.0) atomicCAS(a.info, 0, (int)col + 1);
        }
      }
      if (lane == 0 && cta == 0) a.ipiv[col] = gr;
    }
    __syncthreads();
    // 3. rank-1 update of columns c+1 .. with l = a(i, c) / pivot formed by
    //    each thread of the row (column c is scaled at the final store)
    const E rp = s_rp;
    const bool live = mine && g > col && (rp.x != 0 || rp.y != 0);
    cv = -1.0;
    const int own = (c + 1) % S;
    if (mine && g > col) {
      const int jst = c + 1 + ((sph - (c + 1)) % S + S) % S;
      if (live) {
        const E l = cmul(slab[c * rpc + i], rp);
        for (int j = jst; j < nb; j += 4 * S) {
          E x[4];
#pragma unroll
          for (int u = 0; u < 4; u++)
            if (j + u * S < nb) x[u] = slab[(j + u * S) * rpc + i];
#pragma unroll
          for (int u = 0; u < 4; u++)
            if (j + u * S < nb) {
              const E uu = s_prow_data[j + u * S];
              x[u].x -= l.x * uu.x - l.y * uu.y;
              x[u].y -= l.x * uu.y + l.y * uu.x;
              slab[(j + u * S) * rpc + i] = x[u];
            }
        }
      }
      if (sph == own && c + 1 < nb) cv = cabs1(slab[(c + 1) * rpc + i]);
    }
  }
  __syncthreads();
  for (int idx = tid; idx < nb * rpc; idx += kPanelThreads) {
    const int c = idx / rpc, ii = idx % rpc;
    if (ii < nrow) {
      const E v = slab[idx], rp = s_rpc[c];
      const bool low = row0 + ii > a.j0 + c && (rp.x != 0 || rp.y != 0);
      st2(A + (row0 + ii) + (a.j0 + c) * a.lda, low ? cmul(v, rp) : v);
    }
  }
  cluster_sync();  // no CTA leaves while another may still address its shared memory
}

// The nb row interchanges of a panel (ipiv[j0 .. j0+nb), applied in order)
// composed into one permutation of the at most 2 nb rows they touch:
// after the swaps, row dst[i] holds the old row src[i], i < *count.
// One warp: rows inside the panel are tracked in a direct array, rows below
// it (at most nb distinct) in a list searched by the whole warp at once, so
// each interchange costs a few warp-wide steps.  Requires nb <= 64.
__global__ void pivot_map_kernel(const int *ipiv, int64_t j0, int nb, int *dst, int *src, int *count) {
  __shared__ int piv[64], in_orig[64], out_row[64], out_orig[64];
  const int lane = threadIdx.x;
  for (int i = lane; i < nb; i += 32) {
    piv[i] = ipiv[j0 + i];
    in_orig[i] = (int)j0 + i;
  }
  __syncwarp();
  int nout = 0;  // warp-uniform
  for (int c = 0; c < nb; c++) {
    const int b = piv[c];
    const int a = (int)j0 + c;
    if (b == a) continue;
    int *slot;
    if (b < j0 + nb) {
      slot = &in_orig[b - j0];
    } else {
      const unsigned m0 = __ballot_sync(0xffffffffu, lane < nout && out_row[lane] == b);
      const unsigned m1 = __ballot_sync(0xffffffffu, lane + 32 < nout && out_row[lane + 32] == b);
      int s;
      if (m0) s = __ffs(m0) - 1;
      else if (m1) s = 32 + __ffs(m1) - 1;
      else {
        s = nout++;
        if (lane == 0) {
          out_row[s] = b;
          out_orig[s] = b;
        }
      }
      slot = &out_orig[s];
    }
    if (lane == 0) {
      const int t = in_orig[c];
      in_orig[c] = *slot;
      *slot = t;
    }
    __syncwarp();
  }
  // compact the rows whose content changed: inside rows first, then the list
  int k = 0;
  for (int base = 0; base < nb + nout; base += 32) {
    const int i = base + lane;
    int r = -1, o = -1;
    if (i < nb) {
      r = (int)j0 + i;
      o = in_orig[i];
    } else if (i < nb + nout) {
      r = out_row[i - nb];
      o = out_orig[i - nb];
    }
    const bool moved = r >= 0 && o != r;
    const unsigned m = __ballot_sync(0xffffffffu, moved);
    if (moved) {
      const int at = k + __popc(m & ((1u << lane) - 1u));
      dst[at] = r;
      src[at] = o;
    }
    k += __popc(m);
  }
  if (lane == 0) *count = k;
}

// Apply the composed panel permutation to every column outside the panel:
// one warp per column, all source rows loaded before any store.
template <typename T>
__global__ void laswp_kernel(T *A, int64_t lda, int64_t n, int64_t j0, int nb, const int *dst, const int *src,
                             const int *count) {
  const int lane = threadIdx.x & 31;
  int64_t col = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (col >= n - nb) return;
  if (col >= j0) col += nb;
  const int k = *count;
  T *a = A + col * lda;
  T v[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = lane + 32 * q;
    if (i < k) v[q] = a[src[i]];
  }
  __syncwarp();
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = lane + 32 * q;
    if (i < k) a[dst[i]] = v[q];
  }
}

// The same interchanges on the columns [c0, c0 + ncols) outside the panel
// [j0, j0 + nb): one warp per column.
template <typename T>
__global__ void laswp_range_kernel(T *A, int64_t lda, int64_t c0, int64_t ncols, int64_t j0, int nb, const int *dst,
                                   const int *src, const int *count) {
  const int lane = threadIdx.x & 31;
  const int64_t idx = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (idx >= ncols) return;
  const int64_t col = c0 + idx;
  if (col >= j0 && col < j0 + nb) return;
  const int k = *count;
  T *a = A + col * lda;
  T v[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = lane + 32 * q;
    if (i < k) v[q] = a[src[i]];
  }
  __syncwarp();
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = lane + 32 * q;
    if (i < k) a[dst[i]] = v[q];
  }
}

// The interchanges of the np panels of an outer block [J0, J0 + NBc), in
// panel order, on the columns outside that block: one warp per column, maps
// at pm + 260 p (dst[128], src[128], count).  The outside columns are
// numbered 0 .. n - NBc - 1 (those right of the block shifted by NBc); the
// launch covers [c_lo, c_hi) of that numbering without [s_lo, s_hi).
template <typename T>
__global__ void laswp_block_kernel(T *A, int64_t lda, int64_t n, int64_t J0, int64_t NBc, const int *pm, int np,
                                   int64_t c_lo, int64_t c_hi, int64_t s_lo, int64_t s_hi) {
  const int lane = threadIdx.x & 31;
  int64_t col = c_lo + (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (col >= c_hi || col >= n - NBc) return;
  if (col >= s_lo && col < s_hi) return;
  if (col >= J0) col += NBc;
  T *a = A + col * lda;
  for (int p = 0; p < np; p++) {
    const int *dst = pm + 260 * p, *src = dst + 128;
    const int k = dst[256];
    T v[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = lane + 32 * q;
      if (i < k) v[q] = a[src[i]];
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = lane + 32 * q;
      if (i < k) a[dst[i]] = v[q];
    }
    __syncwarp();
  }
}

// Inverses of the unit-lower L11 and upper U11 diagonal blocks of a panel
// (FP64), stored as inv[0] = inv(L11), inv[1] = inv(U11), column-major
// 64 x 64.  One CTA of 512 threads (256 per triangle), all in shared memory,
// by recursive doubling: the sixteen 8 x 8 diagonal blocks are inverted by
// substitution, then neighbouring inverses are joined for block sizes 8, 16
// and 32,
//   inv([L11 0; L21 L22]) = [X11 0; -X22 L21 X11, X22],
//   inv([U11 U12; 0 U22]) = [Y11, -Y11 U12 Y22; 0 Y22],
// each join as two small triangular-times-dense products.  The dependent
// chain is 8 substitution steps and six products instead of 64 substitution
// steps.  Product temporaries sit in the half of each inverse that is zero
// (above the diagonal of inv(L), below it for inv(U)); the triangular k
// ranges below never read those halves, and the final store masks them.
constexpr int kDiagNb = 64;
constexpr int kDiagThreads = 512;

__device__ __forceinline__ void cfma(double2 &acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}

// For the 32 / B joins of one triangle (join p works on rows and columns
// from o = 2 B p): C(o+cr.., o+cc..) = s * A(o+ar.., o+ac..) * B(o+br.., o+bc..),
// B x B blocks of 64 x 64 column-major shared arrays, with k restricted to
// the non-zero part of the triangular factor: MODE 0 k >= col, 1 k <= row,
// 2 k <= col, 3 k >= row.  NT threads (u < NT) share the 32 B outputs.
template <int B, int MODE, int NT>
__device__ __forceinline__ void join_product(int u, double s, const double2 *Am, int ar, int ac, const double2 *Bm,
                                             int br, int bc, double2 *Cm, int cr, int cc) {
#pragma unroll
  for (int i = 0; i < (32 * B + NT - 1) / NT; i++) {
    const int e = u + NT * i;
    if (e >= 32 * B) break;
    const int p = e / (B * B), rem = e % (B * B);
    const int col = rem / B, row = rem % B;
    const int o = 2 * B * p;
    const double2 *a = Am + (o + ar + row) + (o + ac) * kDiagNb;
    const double2 *b = Bm + (o + br) + (o + bc + col) * kDiagNb;
    const int k0 = MODE == 0 ? col : (MODE == 3 ? row : 0);
    const int k1 = MODE == 1 ? row + 1 : (MODE == 2 ? col + 1 : B);
    double2 acc = make_double2(0, 0);
    for (int k = k0; k < k1; k++) cfma(acc, a[k * kDiagNb], b[k]);
    Cm[(o + cr + row) + (o + cc + col) * kDiagNb] = make_double2(s * acc.x, s * acc.y);
  }
}

// L: T = L21 X11 into the upper slot, then X21 = -X22 T;
// U: T = U12 Y22 into the lower slot, then Y12 = -Y11 T.
// TRI 0: L only, 1: U only (all threads on one triangle), 2: both.
template <int B, int TRI>
__device__ __forceinline__ void join_level(int t, const double2 *D, double2 *XL, double2 *XU) {
  if (TRI == 0) {
    join_product<B, 0, kDiagThreads>(t, 1.0, D, B, 0, XL, 0, 0, XL, 0, B);
    __syncthreads();
    join_product<B, 1, kDiagThreads>(t, -1.0, XL, B, B, XL, 0, B, XL, B, 0);
  } else if (TRI == 1) {
    join_product<B, 2, kDiagThreads>(t, 1.0, D, 0, B, XU, B, B, XU, B, 0);
    __syncthreads();
    join_product<B, 3, kDiagThreads>(t, -1.0, XU, 0, 0, XU, B, 0, XU, 0, B);
  } else {
    if (t < 256) join_product<B, 0, 256>(t, 1.0, D, B, 0, XL, 0, 0, XL, 0, B);
    else join_product<B, 2, 256>(t - 256, 1.0, D, 0, B, XU, B, B, XU, B, 0);
    __syncthreads();
    if (t < 256) join_product<B, 1, 256>(t, -1.0, XL, B, B, XL, 0, B, XL, B, 0);
    else join_product<B, 3, 256>(t - 256, -1.0, XU, 0, 0, XU, B, 0, XU, 0, B);
  }
  __syncthreads();
}

// CTA b inverts the diagonal block kb = kb0 + b (rows and columns 64 kb ..)
// of the factors in A: inv(L11) into invd[kb][0] (and FP32 into
// invL32[kb]), inv(U11) into invd[kb][1], for the triangles TRI selects.
template <typename T, int TRI>
__global__ void __launch_bounds__(kDiagThreads) diag_inv_kernel(const T *A, int64_t lda, int kb0, double2 *invd,
                                                                float2 *invL32) {
  extern __shared__ double2 sm[];
  constexpr int nb = kDiagNb, nn = kDiagNb * kDiagNb;
  const int kb = kb0 + blockIdx.x;
  const int64_t j0 = (int64_t)kb * nb;
  double2 *invL = invd + (size_t)kb * 2 * nn, *invU = invL + nn;
  double2 *D = sm, *XL = sm + nn, *XU = sm + 2 * nn, *rinv = sm + 3 * nn;
  const int t = threadIdx.x;
  // eight independent loads in flight per thread before the shared stores
  {
    double2 v[nn / kDiagThreads];
#pragma unroll
    for (int u = 0; u < nn / kDiagThreads; u++) {
      const int idx = t + u * kDiagThreads;
      v[u] = ld2(A + (j0 + idx % nb) + (j0 + idx / nb) * lda);
    }
#pragma unroll
    for (int u = 0; u < nn / kDiagThreads; u++) D[t + u * kDiagThreads] = v[u];
  }
  __syncthreads();
  if (TRI != 0 && t < nb) {  // 1 / U_ii (0 for a zero pivot; the panel reports it)
    const double2 d = D[t + t * nb];
    const double dd = d.x * d.x + d.y * d.y;
    rinv[t] = dd != 0.0 ? make_double2(d.x / dd, -d.y / dd) : make_double2(0, 0);
  }
  __syncthreads();
  // the 8 x 8 diagonal blocks: thread (block q, column c) by substitution
  const int tl = TRI == 2 ? 256 : 0;  // first thread of the U triangle
  if (TRI != 1 && t < 64) {
    const int q = t >> 3, c = t & 7, o = 8 * q;
    double2 x[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      double2 v = make_double2(i == c ? 1.0 : 0.0, 0.0);
#pragma unroll
      for (int k = 0; k < i; k++)
        if (k >= c) {
          const double2 l = D[(o + i) + (o + k) * nb];
          v.x -= l.x * x[k].x - l.y * x[k].y;
          v.y -= l.x * x[k].y + l.y * x[k].x;
        }
      x[i] = i >= c ? v : make_double2(0, 0);
    }
#pragma unroll
    for (int i = 0; i < 8; i++) XL[(o + i) + (o + c) * nb] = x[i];
  } else if (TRI != 0 && t >= tl && t < tl + 64) {
    const int q = (t - tl) >> 3, c = t & 7, o = 8 * q;
    double2 y[8];
#pragma unroll
    for (int i = 7; i >= 0; i--) {
      double2 v = make_double2(i == c ? 1.0 : 0.0, 0.0);
#pragma unroll
      for (int k = i + 1; k < 8; k++)
        if (k <= c) {
          const double2 u = D[(o + i) + (o + k) * nb];
          v.x -= u.x * y[k].x - u.y * y[k].y;
          v.y -= u.x * y[k].y + u.y * y[k].x;
        }
      y[i] = i <= c ? cmul(v, rinv[o + i]) : make_double2(0, 0);
    }
#pragma unroll
    for (int i = 0; i < 8; i++) XU[(o + i) + (o + c) * nb] = y[i];
  }
  __syncthreads();
  join_level<8, TRI>(t, D, XL, XU);
  join_level<16, TRI>(t, D, XL, XU);
  join_level<32, TRI>(t, D, XL, XU);
  for (int idx = t; idx < nn; idx += kDiagThreads) {
    const int r = idx % nb, c = idx / nb;
    if (TRI != 1) {
      const double2 l = r > c ? XL[idx] : make_double2(r == c ? 1.0 : 0.0, 0.0);
      invL[idx] = l;
      if (invL32) invL32[(size_t)kb * nn + idx] = make_float2((float)l.x, (float)l.y);
    }
    if (TRI != 0) invU[idx] = r <= c ? XU[idx] : make_double2(0, 0);
  }
}

// The row interchanges of the whole factorisation, in order, composed into
// one permutation: perm[i] = source row of row i of P*B.  One thread walks
// the swaps in shared memory (once per factorisation).
__global__ void compose_pivots_kernel(const int *ipiv, int n, int *perm) {
  extern __shared__ int p[];
  for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = i;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int i = 0; i < n; i++) {
      const int r = ipiv[i];
      if (r != i) {
        const int t = p[i];
        p[i] = p[r];
        p[r] = t;
      }
    }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = p[i];
}

__global__ void inv_to_fp32_kernel(const double2 *a, float2 *b, int64_t count) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = make_float2((float)a[i].x, (float)a[i].y);
}

struct TrsvArgs {
  const void *M;     // LU factors (T)
  int64_t lda, n;
  int nb, P, rpc, ns;
  const void *inv;   // [nblk][2][nb][nb] (T): inv(L_kk), inv(U_kk)
  const int *perm;
  double2 *X, *Y, *Z;  // [ns][n]: right-hand sides in X (solution returned there); the solved
                       // blocks of the forward pass are published in Y, of the backward pass in Z
                       // (both zeroed before the launch; published words carry a mark bit)
  int *timeout;
  long long spin;  // polls before a wait is declared timed out
  int direct;  // 1: factor tiles do not fit in shared memory; read them from global memory
  int stages;  // prefetch stages (1 or 2) of factor tile + diagonal-block inverse
};

// Complex multiply-add in the factor's precision (FP32 for the mixed
// path's correction solves, as the single-precision solves of classical
// mixed-precision refinement; FP64 otherwise).
__device__ __forceinline__ float fma_t(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return __fma_rn(a, b, c); }
template <typename T>
__device__ __forceinline__ void cmac(T &acc, T m, T y) {
  acc.x = fma_t(m.x, y.x, acc.x);
  acc.x = fma_t(-m.y, y.y, acc.x);
  acc.y = fma_t(m.x, y.y, acc.y);
  acc.y = fma_t(m.y, y.x, acc.y);
}
template <typename T>
__device__ __forceinline__ T cadd(T a, T b) {
  a.x += b.x;
  a.y += b.y;
  return a;
}
// sum over groups of g adjacent lanes (g a power of two <= 32, all lanes present)
template <typename T>
__device__ __forceinline__ T group_sum(T v, int g) {
  for (int o = g >> 1; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}

// ys = Inv * xs for an nb x nb block (column-major, element type T) and NS
// vectors xs[sv * nb + j] (type T); `parts` adjacent lanes share one output
// and reduce with shuffles.  The result goes to ys (FP64) and ysc (T).
// tr: apply the transpose.  Requires nb a multiple of 64.
template <typename T, int NS>
__device__ void block_apply(const T *inv, int nb, const T *xs, double2 *ys, T *ysc, bool tr) {
  const int O = nb * NS;
  int parts = 1;
  while (parts * 2 * O <= (int)blockDim.x && parts < 16) parts *= 2;
  for (int base = 0; base < O * parts; base += blockDim.x) {
    const int g = base + threadIdx.x;
    const bool valid = g < O * parts;
    const int o = valid ? g / parts : 0, part = g % parts;
    const int r = o % nb, sv = o / nb;
    T a0 = {0, 0}, a1 = {0, 0}, a2 = {0, 0}, a3 = {0, 0};
    if (valid) {
      for (int j = part; j < nb; j += 4 * parts) {
        const T *i0 = tr ? inv + j + (size_t)r * nb : inv + r + (size_t)j * nb;
        const size_t st = tr ? (size_t)parts : (size_t)parts * nb;
        cmac(a0, i0[0], xs[sv * nb + j]);
        cmac(a1, i0[st], xs[sv * nb + j + parts]);
        cmac(a2, i0[2 * st], xs[sv * nb + j + 2 * parts]);
        cmac(a3, i0[3 * st], xs[sv * nb + j + 3 * parts]);
      }
    }
    const T acc = group_sum(cadd(cadd(a0, a1), cadd(a2, a3)), parts);
    if (valid && part == 0) {
      ys[o] = make_double2(acc.x, acc.y);
      ysc[o] = acc;
    }
  }
  __syncthreads();
}

__device__ __forceinline__ void cp_async(void *smem, const void *gmem, int bytes_is_16) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  if (bytes_is_16)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Row range of CTA-owned rows that block kb updates in pass 0 (below the
// block) or pass 1 (above it).
__device__ __forceinline__ void upd_range(int pass, int64_t k0, int nb, int64_t r0, int64_t r1, int64_t *lo,
                                          int64_t *hi) {
  *lo = pass == 0 ? max(r0, k0 + nb) : r0;
  *hi = pass == 0 ? r1 : min(r1, k0);
}

// Published solution words: the lowest mantissa bit is forced to 1 (a
// change of at most one unit in the last place), so that a word of a
// buffer zeroed before the launch is known to be written once it reads
// odd.  Each 64-bit word is single-copy atomic; no fence or flag is needed.
__device__ __forceinline__ void publish_word2(double2 *p, double2 v) {
  const unsigned long long x = (unsigned long long)__double_as_longlong(v.x) | 1ull;
  const unsigned long long y = (unsigned long long)__double_as_longlong(v.y) | 1ull;
  asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(x), "l"(y) : "memory");
}
__device__ __forceinline__ bool read_word2(const double2 *p, double2 *v) {
  unsigned long long x, y;
  asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(x), "=l"(y) : "l"(p) : "memory");
  *v = make_double2(__longlong_as_double((long long)x), __longlong_as_double((long long)y));
  return (x & y & 1ull) != 0ull;
}

// Forward (unit lower) and backward (upper) substitution of P A = L U for
// NS right-hand sides in one cooperative launch, scheduled by data flow.
// CTA c owns whole 64-row blocks, rows [c rpc, (c+1) rpc), and keeps its
// rows of the vector in shared memory for both passes.  The owner of a
// block solves it (y_k = inv_k x_k) and publishes y_k (pass 0 in Y, pass 1
// in Z) as marked words; every other CTA with rows to update polls those
// words until all are marked and updates its own rows with the factor tile
// of block k (prefetched with cp.async while it waits, double-buffered when
// shared memory allows).  A CTA that owns the next block updates that
// block's rows first, solves and publishes it, and only then updates the
// rest, so the critical path per block is one flag hand-off, one L2 read of
// y_k, a 64-row update and one 64 x 64 apply; between consecutive blocks of
// one CTA there is no hand-off at all.  The steps of both passes form one
// sequence t = 0 .. 2 nblk - 1 (pass 0 block t, then pass 1 block
// 2 nblk - 1 - t); the last block of pass 0 is the first of pass 1 and
// stays with its owner.  TR solves A^T x = b: forward with U^T, backward
// with L^T (unit), x = P^T z; its tile is the block row of U (L) right
// (left) of the diagonal, row by row with a padded stride.
template <typename T, int NS, bool TR>
__global__ void __launch_bounds__(256, 1) trsv_flow_kernel(TrsvArgs a) {
  __shared__ double2 ysb[2][NS * 64];  // y of the current / next block (FP64)
  __shared__ T ysc[2][NS * 64];        // the same in the factor's precision
  __shared__ T xsc[NS * 64];           // the block being solved, in the factor's precision
  __shared__ int s_ok;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const T *M = reinterpret_cast<const T *>(a.M);
  const T *inv = reinterpret_cast<const T *>(a.inv);
  const int64_t n = a.n, lda = a.lda;
  const int nb = a.nb, nblk = (int)(n / nb), rpc = a.rpc, S = a.stages;
  const int nsteps = 2 * nblk;
  const int64_t r0 = (int64_t)blockIdx.x * rpc;
  const int64_t r1 = min(n, r0 + rpc);
  // shared memory: own rows [NS][rpc] (double2) | inverses [S][nb][nb] | tiles [S]
  double2 *xo = reinterpret_cast<double2 *>(smem_raw);
  T *sinv = reinterpret_cast<T *>(smem_raw + sizeof(double2) * (size_t)NS * rpc);
  // tile element (row i, column j of the block): TR i * (nb + 1) + j, else
  // j * cs + i with the column stride cs padded by 64 bytes, so that the
  // lanes of a warp reading 4 columns of 8 rows hit distinct banks
  const int cs = rpc + 64 / (int)sizeof(T);
  const size_t tile_elems = TR ? (size_t)rpc * (nb + 1) : (size_t)nb * cs;
  const size_t tile_stride = ((sizeof(T) * tile_elems + 15) / 16) * 16 / sizeof(T);
  T *tiles = sinv + (size_t)S * nb * nb;
  auto blk_of = [&](int t) { return t < nblk ? t : nsteps - 1 - t; };
  auto pass_of = [&](int t) { return t < nblk ? 0 : 1; };
  auto owns = [&](int kb) { return (int64_t)kb * nb >= r0 && (int64_t)kb * nb < r1; };
  // prefetch group of step t: the factor tile of block t (stage t % S) and,
  // when this CTA solves the block of step t + 1, its inverse (stage (t + 1) % S)
  auto issue = [&](int t) {
    if (t >= 0 && t < nsteps && !a.direct) {
      const int pass = pass_of(t);
      const int64_t k0 = (int64_t)blk_of(t) * nb;
      int64_t lo, hi;
      upd_range(pass, k0, nb, r0, r1, &lo, &hi);
      const int cnt = hi <= lo ? 0 : (int)(hi - lo);
      T *tile = tiles + (size_t)(t % S) * tile_stride;
      if (TR) {
        for (int idx = threadIdx.x; idx < cnt * nb; idx += blockDim.x) {
          const int j = idx % nb, i = idx / nb;
          cp_async(tile + (size_t)i * (nb + 1) + j, M + (k0 + j) + (lo + i) * lda, sizeof(T) == 16);
        }
      } else {
        for (int idx = threadIdx.x; idx < cnt * nb; idx += blockDim.x) {
          const int i = idx % cnt, j = idx / cnt;
          cp_async(tile + (size_t)j * cs + i, M + (lo + i) + (k0 + j) * lda, sizeof(T) == 16);
        }
      }
    }
    const int u = t + 1;
    if (u < nsteps && owns(blk_of(u))) {
      // pass 0 applies inv(L) (or inv(U)^T), pass 1 inv(U) (or inv(L)^T)
      const int pu = pass_of(u);
      const T *ib = inv + ((size_t)blk_of(u) * 2 + (TR ? 1 - pu : pu)) * nb * nb;
      T *dst = sinv + (size_t)(u % S) * nb * nb;
      for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) cp_async(dst + idx, ib + idx, sizeof(T) == 16);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  auto wait_stage = [&]() {
    if (S == 2) asm volatile("cp.async.wait_group 1;" ::: "memory");
    else asm volatile("cp.async.wait_group 0;" ::: "memory");
  };
  // xo[i] -= sum_j M(i, block k0) y[j] for own rows i in [lo, hi); tl holds
  // the tile rows from tlo.  G adjacent lanes share a row when there are few
  // rows (shuffle reduction); products and the 64-term sums in the factor's
  // precision, the running vector in FP64.  No barrier inside.
  auto update = [&](int64_t k0, int64_t lo, int64_t hi, int64_t tlo, const T *tl, const T *y) {
    const int rows = hi > lo ? (int)(hi - lo) : 0;
    if (rows == 0) return;  // uniform over the CTA
    const int G = NS > 2 ? 1 : (rows <= 64 ? 4 : (rows <= 128 ? 2 : 1));
    const int part = threadIdx.x % G, rpr = (int)blockDim.x / G;
    const int64_t mstride = TR ? 1 : (a.direct ? lda : cs);
    for (int base = 0; base < rows; base += rpr) {
      const int ri = base + (int)threadIdx.x / G;
      const bool valid = ri < rows;
      T a0[NS], a1[NS];
#pragma unroll
      for (int sv = 0; sv < NS; sv++) a0[sv] = a1[sv] = T{0, 0};
      if (valid) {
        const int64_t i = lo + ri;
        const T *mp = TR ? (a.direct ? M + k0 + i * lda : tl + (size_t)(i - tlo) * (nb + 1))
                         : (a.direct ? M + i + k0 * lda : tl + (i - tlo));
#pragma unroll 2
        for (int j = part; j < nb; j += 2 * G) {
          const T m0 = mp[(size_t)j * mstride], m1 = mp[(size_t)(j + G) * mstride];
#pragma unroll
          for (int sv = 0; sv < NS; sv++) {
            cmac(a0[sv], m0, y[sv * nb + j]);
            cmac(a1[sv], m1, y[sv * nb + j + G]);
          }
        }
      }
#pragma unroll
      for (int sv = 0; sv < NS; sv++) {
        const T acc = group_sum(cadd(a0[sv], a1[sv]), G);
        if (valid && part == 0) {
          const int64_t li = lo + ri - r0;
          double2 v = xo[(size_t)sv * rpc + li];
          v.x -= (double)acc.x;
          v.y -= (double)acc.y;
          xo[(size_t)sv * rpc + li] = v;
        }
      }
    }
  };
  // solve the own block of step u from xo and publish it
  auto solve_publish = [&](int u) {
    const int kb = blk_of(u), pu = pass_of(u);
    const int64_t l0 = (int64_t)kb * nb - r0;
    for (int idx = threadIdx.x; idx < nb * NS; idx += blockDim.x) {
      const int j = idx % nb, sv = idx / nb;
      st2(xsc + sv * nb + j, xo[(size_t)sv * rpc + l0 + j]);
    }
    __syncthreads();
    double2 *y = ysb[u & 1];
    block_apply<T, NS>(sinv + (size_t)(u % S) * nb * nb, nb, xsc, y, ysc[u & 1], TR);
    double2 *E = pu == 0 ? a.Y : a.Z;
    for (int idx = threadIdx.x; idx < nb * NS; idx += blockDim.x) {
      const int j = idx % nb, sv = idx / nb;
      const double2 v = y[sv * nb + j];
      xo[(size_t)sv * rpc + l0 + j] = v;
      publish_word2(E + (size_t)sv * n + (int64_t)kb * nb + j, v);
    }
    __syncthreads();
  };
  // own rows of P X (TR: X)
  const int nrow = (int)(r1 - r0);
  for (int idx = threadIdx.x; idx < NS * nrow; idx += blockDim.x) {
    const int li = idx % nrow, sv = idx / nrow;
    const int64_t i = r0 + li;
    xo[(size_t)sv * rpc + li] = a.X[(size_t)sv * n + (TR ? i : a.perm[i])];
  }
  for (int t = -1; t <= S - 2; t++) issue(t);
  wait_stage();
  __syncthreads();
  if (owns(blk_of(0))) solve_publish(0);
  __syncthreads();
  issue(S - 1);
  for (int t = 0; t < nsteps; t++) {
    const int kb = blk_of(t), pass = pass_of(t);
    const int64_t k0 = (int64_t)kb * nb;
    int64_t lo, hi;
    upd_range(pass, k0, nb, r0, r1, &lo, &hi);
    const int u = t + 1;
    const bool own_next = u < nsteps && owns(blk_of(u));
    if ((hi > lo || own_next) && !owns(kb)) {
      // poll the published words of block kb until all are marked (bounded)
      const double2 *E = pass == 0 ? a.Y : a.Z;
      long long it = 0;
      while (true) {
        int ok = 1;
        for (int idx = threadIdx.x; idx < nb * NS; idx += blockDim.x) {
          const int j = idx % nb, sv = idx / nb;
          double2 v;
          if (read_word2(E + (size_t)sv * n + k0 + j, &v)) {
            st2(&ysc[t & 1][sv * nb + j], v);
          } else {
            ok = 0;
          }
        }
        if (__syncthreads_and(ok)) break;
        if ((++it & 255) == 0 || it > a.spin) {
          if (threadIdx.x == 0) {
            int go = 1;
            if (*(volatile int *)a.timeout) go = 0;
            else if (it > a.spin) {
              atomicExch(a.timeout, 1);
              go = 0;
            }
            s_ok = go;
          }
          __syncthreads();
          if (!s_ok) {
            cp_async_wait_all();
            return;
          }
        }
      }
    }
    wait_stage();
    __syncthreads();
    const T *tl = tiles + (size_t)(t % S) * tile_stride;
    const T *yc = ysc[t & 1];
    if (own_next) {
      const int64_t a0 = (int64_t)blk_of(u) * nb;
      const bool same = pass_of(u) == pass;
      if (same) {
        update(k0, a0, a0 + nb, lo, tl, yc);
        __syncthreads();
      }
      solve_publish(u);
      if (same) {
        update(k0, lo, a0, lo, tl, yc);
        update(k0, a0 + nb, hi, lo, tl, yc);
      } else {
        update(k0, lo, hi, lo, tl, yc);
      }
    } else {
      update(k0, lo, hi, lo, tl, yc);
    }
    __syncthreads();
    issue(t + S);
  }
  cp_async_wait_all();
  // the solution of the own rows; TR: X = P^T Z
  for (int idx = threadIdx.x; idx < NS * nrow; idx += blockDim.x) {
    const int li = idx % nrow, sv = idx / nrow;
    const int64_t i = r0 + li;
    a.X[(size_t)sv * n + (TR ? a.perm[i] : i)] = xo[(size_t)sv * rpc + li];
  }
}

constexpr int kGemvRows = 256;
constexpr int kGemvCols = 256;

// partial[chunk][s][i] = sum_{j in chunk} A[i, j] x_s[j]  (FP64 matrix)
template <int NS>
__global__ void __launch_bounds__(kGemvRows) gemv_partial_kernel(const double2 *A, int64_t lda, int64_t n,
                                                                 const double2 *X, int64_t ldx, double2 *partial) {
  __shared__ double2 xs[NS][kGemvCols];
  const int64_t i = (int64_t)blockIdx.x * kGemvRows + threadIdx.x;
  const int64_t j0 = (int64_t)blockIdx.y * kGemvCols;
  const int cnt = (n - j0) < kGemvCols ? (int)(n - j0) : kGemvCols;
  for (int idx = threadIdx.x; idx < cnt * NS; idx += kGemvRows) {
    const int j = idx % cnt, s = idx / cnt;
    xs[s][j] = X[(size_t)s * ldx + j0 + j];
  }
  __syncthreads();
  if (i >= n) return;
  double2 acc[NS];
#pragma unroll
  for (int s = 0; s < NS; s++) acc[s] = make_double2(0, 0);
#pragma unroll 8
  for (int j = 0; j < cnt; j++) {
    const double2 m = A[i + (j0 + j) * lda];
#pragma unroll
    for (int s = 0; s < NS; s++) {
      const double2 x = xs[s][j];
      acc[s].x += m.x * x.x - m.y * x.y;
      acc[s].y += m.x * x.y + m.y * x.x;
    }
  }
#pragma unroll
  for (int s = 0; s < NS; s++) partial[((size_t)blockIdx.y * NS + s) * n + i] = acc[s];
}

// Y[s][j] = sum_i A[i, j] x_s[i] (FP64 matrix, transposed product): one
// warp per column, lanes stride down the column.
template <int NS>
__global__ void __launch_bounds__(256) gemv_t_kernel(const double2 *A, int64_t lda, int64_t n, const double2 *X,
                                                     int64_t ldx, double2 *Y) {
  const int lane = threadIdx.x & 31;
  const int64_t j = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  if (j >= n) return;
  const double2 *col = A + j * lda;
  double2 acc[NS];
#pragma unroll
  for (int s = 0; s < NS; s++) acc[s] = make_double2(0, 0);
  for (int64_t i = lane; i < n; i += 32) {
    const double2 m = __ldcs(col + i);
#pragma unroll
    for (int s = 0; s < NS; s++) {
      const double2 x = X[(size_t)s * ldx + i];
      acc[s].x += m.x * x.x - m.y * x.y;
      acc[s].y += m.x * x.y + m.y * x.x;
    }
  }
#pragma unroll
  for (int s = 0; s < NS; s++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      acc[s].x += __shfl_xor_sync(0xffffffffu, acc[s].x, o);
      acc[s].y += __shfl_xor_sync(0xffffffffu, acc[s].y, o);
    }
    if (lane == 0) Y[(size_t)s * n + j] = acc[s];
  }
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

// Y[s] += sign * (sum of partials)
__global__ void acc_partials_kernel(double2 *Y, int64_t ldy, const double2 *partial, int nchunk, int64_t n, int nrhs,
                                    double sign) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (i >= n) return;
  double2 acc = make_double2(0, 0);
  for (int c = 0; c < nchunk; c++) {
    const double2 p = partial[((size_t)c * nrhs + s) * n + i];
    acc.x += p.x;
    acc.y += p.y;
  }
  double2 y = Y[(size_t)s * ldy + i];
  y.x += sign * acc.x;
  y.y += sign * acc.y;
  Y[(size_t)s * ldy + i] = y;
}

__global__ void axpy_kernel(double2 *X, const double2 *D, int64_t count) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t st = (int64_t)gridDim.x * blockDim.x;
  for (; i < count; i += st) {
    X[i].x += D[i].x;
    X[i].y += D[i].y;
  }
}

// U12 of an outer block in one launch: B <- inv(L11) B for the np panels'
// rows [J0, J0 + np nb) and the columns [c0, c0 + ncol), L11 unit lower
// triangular.  Per panel p: X_p = inv(L_pp) B_p with the diagonal block's
// inverse (diag_inv_kernel), then B_q -= L_qp X_p for every panel q below.
// One CTA per kBtCols columns keeps its np nb x kBtCols tile in shared
// memory; the 64 x 64 factor blocks are staged one at a time.  FP32 complex
// products with FP32 accumulation, as the library CGEMM it replaces.
constexpr int kBtCols = 32;
constexpr int kBtThreads = 256;
constexpr int kBtMaxPanels = 4;
constexpr int kBtLd = 65;             // padded row stride of the staged factor block
constexpr int kBtLdB = kBtCols + 1;   // padded row stride of the column tile
constexpr size_t kBtSmem = sizeof(float2) * ((size_t)kBtMaxPanels * 64 * kBtLdB + 64 * kBtLd);

__global__ void __launch_bounds__(kBtThreads) block_trsm_kernel(float2 *A, int64_t lda, int64_t J0, int np,
                                                                int64_t c0, int ncol, const float2 *invL) {
  extern __shared__ float2 bt_smem[];
  float2 *Bs = bt_smem;                                  // [np * 64][kBtLdB]
  float2 *Ms = bt_smem + (size_t)kBtMaxPanels * 64 * kBtLdB;  // [64][kBtLd], row-major
  const int t = threadIdx.x, j = t % kBtCols, rg = t / kBtCols;  // 8 rows per thread
  const int jc = blockIdx.x * kBtCols;
  const int rows = np * 64;
  for (int idx = t; idx < rows * kBtCols; idx += kBtThreads) {
    const int r = idx % rows, cc = idx / rows;
    Bs[r * kBtLdB + cc] = (jc + cc < ncol) ? A[(J0 + r) + (c0 + jc + cc) * lda] : make_float2(0.f, 0.f);
  }
  for (int p = 0; p < np; p++) {
    // X_p = inv(L_pp) B_p
    __syncthreads();
    const float2 *inv = invL + (size_t)p * 64 * 64;  // column-major 64 x 64
    for (int idx = t; idx < 64 * 64; idx += kBtThreads) Ms[(idx % 64) * kBtLd + idx / 64] = inv[idx];
    __syncthreads();
    float2 acc[8];
#pragma unroll
    for (int r = 0; r < 8; r++) acc[r] = make_float2(0.f, 0.f);
    for (int k = 0; k < 64; k++) {
      const float2 b = Bs[(p * 64 + k) * kBtLdB + j];
#pragma unroll
      for (int r = 0; r < 8; r++) {
        const float2 m = Ms[(rg * 8 + r) * kBtLd + k];
        acc[r].x = fmaf(m.x, b.x, fmaf(-m.y, b.y, acc[r].x));
        acc[r].y = fmaf(m.x, b.y, fmaf(m.y, b.x, acc[r].y));
      }
    }
    __syncthreads();  // every read of B_p done
#pragma unroll
    for (int r = 0; r < 8; r++) Bs[(p * 64 + rg * 8 + r) * kBtLdB + j] = acc[r];
    // B_q -= L_qp X_p
    for (int q = p + 1; q < np; q++) {
      __syncthreads();
      const float2 *L = A + (J0 + q * 64) + (J0 + p * 64) * lda;
      for (int idx = t; idx < 64 * 64; idx += kBtThreads) Ms[(idx % 64) * kBtLd + idx / 64] = L[(idx % 64) + (idx / 64) * lda];
      __syncthreads();
#pragma unroll
      for (int r = 0; r < 8; r++) acc[r] = make_float2(0.f, 0.f);
      for (int k = 0; k < 64; k++) {
        const float2 x = Bs[(p * 64 + k) * kBtLdB + j];
#pragma unroll
        for (int r = 0; r < 8; r++) {
          const float2 m = Ms[(rg * 8 + r) * kBtLd + k];
          acc[r].x = fmaf(m.x, x.x, fmaf(-m.y, x.y, acc[r].x));
          acc[r].y = fmaf(m.x, x.y, fmaf(m.y, x.x, acc[r].y));
        }
      }
#pragma unroll
      for (int r = 0; r < 8; r++) {
        float2 &v = Bs[(q * 64 + rg * 8 + r) * kBtLdB + j];
        v.x -= acc[r].x;
        v.y -= acc[r].y;
      }
    }
  }
  __syncthreads();
  for (int idx = t; idx < rows * kBtCols; idx += kBtThreads) {
    const int r = idx % rows, cc = idx / rows;
    if (jc + cc < ncol) A[(J0 + r) + (c0 + jc + cc) * lda] = Bs[r * kBtLdB + cc];
  }
}

struct LuWork {
  int *info, *timeout;
  unsigned long long *rec;
  double2 *cand_data, *col_data;
  double2 *W;      // nb x n workspace for the TRSM product
  float2 *invL32;  // nb x nb
  float *tcw;      // tensor-core GEMM operands (mixed path)
  int *pmap;       // [257]: composed panel permutation (dst[128], src[128], count)
  int *pmb;        // [2][16][260]: the composed permutations of every panel of an outer block, double-buffered
  void *W2;        // nb x 16 nb workspace of the look-ahead stream's block TRSM
};

// The panel kernel's exchange buffers (records polled by every CTA once per
// column, candidate rows) can sit at kXSlots placements kXSlotBytes apart.
// Their physical placement changes the exchange latency: at 15,360 rows on
// 96 CTAs one B200 measured 5.2 to 6.5 us per column across eight 64 KB
// steps, constant in 128 KB pairs; so the autotuner times each placement.
constexpr int kXSlots = 16;
constexpr size_t kXSlotBytes = 128 << 10;

// slot < 0: the tuned placement (0 without a table)
int lu_workspace(Ctx *c, int precision, LuWork &w, int slot = -1) {
  const int nb = c->nb, P = c->nsm;
  const size_t esz = precision == MOM_PREC_MIXED ? sizeof(float2) : sizeof(double2);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) / 256 * 256;
    return o;
  };
  if (slot < 0) slot = c->tune ? c->tune->xslot : 0;
  const size_t x_rec = 0, x_cd = x_rec + ((sizeof(unsigned long long) * 2 * P + 255) / 256) * 256;
  const size_t x_cl = x_cd + sizeof(double2) * 2 * P * nb, x_end = x_cl + sizeof(double2) * 2 * nb;
  const size_t o_x = take(kXSlots * kXSlotBytes + x_end);
  const size_t o_w = take(esz * (size_t)nb * c->n);
  const size_t o_i32 = take(sizeof(float2) * (size_t)nb * c->n);
  const size_t o_pm = take(sizeof(int) * 260);
  const size_t o_pmb = take(sizeof(int) * 260 * 2 * 16);
  const size_t o_w2 = take(esz * (size_t)nb * 16 * nb);
  const size_t o_tc =
      take(precision == MOM_PREC_MIXED ? tc_cgemm_work_bytes((int)c->n, (int)c->n, c->outer_panels * nb) : 0);
  MOM_TRY(ensure_buffer(c, &c->ws, &c->ws_bytes, off));
  char *b = (char *)c->ws;
  char *x = b + o_x + (size_t)slot * kXSlotBytes;
  w.info = c->dinfo;
  w.timeout = c->dinfo + 1;
  w.rec = (unsigned long long *)(x + x_rec);
  w.cand_data = (double2 *)(x + x_cd);
  w.col_data = (double2 *)(x + x_cl);
  w.W = (double2 *)(b + o_w);
  w.invL32 = (float2 *)(b + o_i32);
  w.tcw = (float *)(b + o_tc);
  w.pmap = (int *)(b + o_pm);
  w.pmb = (int *)(b + o_pmb);
  w.W2 = (void *)(b + o_w2);
  return MOM_OK;
}

// Identity of the panel table in use (part of the LU graph key).
uint64_t tune_hash(const Ctx *c) {
  uint64_t h = 1469598103934665603ull ^ (uint64_t)c->panel_cap_env;
  if (c->tune) h = (h ^ (uint64_t)(c->tune->xslot + 1)) * 1099511628211ull;
  if (c->tune)
    for (size_t i = 0; i < c->tune->m.size(); i++) h = (h ^ (uint64_t)(c->tune->m[i] * 1000 + c->tune->P[i])) * 1099511628211ull;
  return h;
}

// CTAs for a panel of m rows: the autotuned table's entry at the nearest
// probed height (log scale), else a cap, else one CTA per SM; never fewer
// than needed for rpc <= max_rows rows (what one CTA's slab holds).
int panel_ctas(const Ctx *c, int64_t m, int64_t max_rows) {
  int P = c->nsm;
  if (c->panel_cap_env > 0) {
    P = std::min(c->panel_cap_env, c->nsm);
  } else if (c->tune && !c->tune->m.empty()) {
    double bd = 1e30;
    for (size_t i = 0; i < c->tune->m.size(); i++) {
      const double d = std::fabs(std::log((double)m / (double)c->tune->m[i]));
      if (d < bd) {
        bd = d;
        P = c->tune->P[i];
      }
    }
  }
  P = (int)std::min<int64_t>(P, (m + 7) / 8);
  return (int)std::min<int64_t>(c->nsm, std::max<int64_t>(P, (m + max_rows - 1) / max_rows));
}

// One panel (rows j0 .. n of columns j0 .. j0+nb) on P CTAs.
template <typename T>
int launch_panel(Ctx *c, T *A, int64_t lda, int64_t n, int64_t j0, int P, int *ipiv, int *info, const LuWork &w,
                 cudaStream_t st = nullptr) {
  if (!st) st = c->stream;
  const int nb = c->nb;
  const int64_t m = n - j0;
  if (c->panel_cluster > 0 && m <= (int64_t)kClusterRows<T> * c->panel_cluster) {
    // short panel: one cluster, the smallest power of two with <= kClusterRows rows per CTA
    int CL = 1;
    while ((int64_t)kClusterRows<T> * CL < m) CL *= 2;
    const int rpc = (int)((m + CL - 1) / CL);
    PanelArgs pa;
    pa.A = A;
    pa.lda = lda;
    pa.n = n;
    pa.j0 = j0;
    pa.nb = nb;
    pa.rpc = rpc;
    pa.P = CL;
    pa.ipiv = ipiv;
    pa.info = info;
    pa.timeout = w.timeout;
    pa.spin = wait_polls(c, 0);
    pa.rec = nullptr;
    pa.cand_data = nullptr;
    pa.col_data = nullptr;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CL);
    cfg.blockDim = dim3(kPanelThreads);
    cfg.dynamicSmemBytes = sizeof(typename SlabOf<T>::type) * ((size_t)nb * rpc + (size_t)2 * CL * nb + 2 * nb);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = CL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    MOM_CUDA(c, cudaLaunchKernelEx(&cfg, panel_cluster_kernel<T>, pa));
    c->launches++;
    return MOM_OK;
  }
  const int rpc = (int)((m + P - 1) / P);
  P = (int)((m + rpc - 1) / rpc);
  const size_t smem = sizeof(typename SlabOf<T>::type) * (size_t)nb * rpc;
  if (smem > 222 * 1024 || rpc > kPanelThreads || nb > 64 || P > 256)
    return fail(c, MOM_ERR_ARG, "panel does not fit in shared memory (matrix order too large)");
  PanelArgs pa;
  pa.A = A;
  pa.lda = lda;
  pa.n = n;
  pa.j0 = j0;
  pa.nb = nb;
  pa.rpc = rpc;
  pa.P = P;
  pa.ipiv = ipiv;
  pa.info = info;
  pa.timeout = w.timeout;
  pa.spin = wait_polls(c, 0);
  pa.rec = w.rec;
  pa.cand_data = w.cand_data;
  pa.col_data = w.col_data;
  MOM_CUDA(c, cudaMemsetAsync(w.rec, 0, sizeof(unsigned long long) * 2 * P, st));
  void *args[] = {&pa};
  MOM_CUDA(c, cudaLaunchCooperativeKernel((void *)panel_kernel<T>, dim3(P), dim3(kPanelThreads), args, smem, st));
  c->launches++;
  return MOM_OK;
}

// Issues every launch of the factorisation on the context stream (eagerly,
// or into an open capture).
template <typename T>
int lu_enqueue(Ctx *c, T *A, int precision, const LuWork &w) {
  const int64_t n = c->n, lda = c->lda;
  const int nb = c->nb;
  MOM_CUDA(c, cudaMemsetAsync(c->dinfo, 0, sizeof(int) * 4, c->stream));
  const bool mixed = precision == MOM_PREC_MIXED;
  // The small GEMMs (block TRSM, updates inside an outer block) stay in full FP32 / FP64.
  MOM_BLAS(c, cublasSetMathMode(c->blas, CUBLAS_DEFAULT_MATH));
  // C <- alpha * A(m x k) * B(k x nc) + beta * C, column-major with lda
  auto gemm = [&](int64_t m, int64_t ncol, int64_t k, double alpha, const T *Am, int64_t la, const T *Bm, int64_t lb,
                  double beta, T *Cm, int64_t lc) -> int {
    if (m <= 0 || ncol <= 0 || k <= 0) return MOM_OK;
    c->blas_calls++;
    if (!mixed) {
      const cuDoubleComplex al = make_cuDoubleComplex(alpha, 0), be = make_cuDoubleComplex(beta, 0);
      MOM_BLAS(c, cublasZgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)m, (int)ncol, (int)k, &al,
                              (const cuDoubleComplex *)Am, (int)la, (const cuDoubleComplex *)Bm, (int)lb, &be,
                              (cuDoubleComplex *)Cm, (int)lc));
    } else {
      const cuComplex al = make_cuComplex((float)alpha, 0), be = make_cuComplex((float)beta, 0);
      MOM_BLAS(c, cublasCgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)m, (int)ncol, (int)k, &al,
                              (const cuComplex *)Am, (int)la, (const cuComplex *)Bm, (int)lb, &be, (cuComplex *)Cm,
                              (int)lc));
    }
    return MOM_OK;
  };
  // C(m x ncol) -= L(m x nb) U(nb x ncol): the rank-64 updates; on the
  // tensor cores (3xTF32) in the mixed path, as the trailing update
  auto update64 = [&](int64_t m, int64_t ncol, const T *Lm, const T *Um, T *Cm) -> int {
    if (m <= 0 || ncol <= 0) return MOM_OK;
    if (mixed && c->small_tc)
      return tc_cgemm_update(c, reinterpret_cast<float2 *>(Cm), lda, reinterpret_cast<const float2 *>(Lm), lda,
                             reinterpret_cast<const float2 *>(Um), lda, (int)m, (int)ncol, nb, w.tcw, c->dinfo + 2);
    return gemm(m, ncol, nb, -1.0, Lm, lda, Um, lda, 1.0, Cm, lda);
  };
  // B(nb x ncol, at A + j0 + col*lda) <- inv(L_jj) B, through the workspace
  auto trsm_l = [&](int64_t j0, int64_t col, int64_t ncol, int kb) -> int {
    if (ncol <= 0) return MOM_OK;
    const T *inv = mixed ? (const T *)(w.invL32 + (size_t)kb * nb * nb) : (const T *)(c->invd + (size_t)kb * 2 * nb * nb);
    T *B = A + j0 + col * lda;
    MOM_TRY(gemm(nb, ncol, nb, 1.0, inv, nb, B, lda, 0.0, (T *)w.W, nb));
    MOM_CUDA(c, cudaMemcpy2DAsync(B, sizeof(T) * lda, w.W, sizeof(T) * nb, sizeof(T) * nb, ncol,
                                  cudaMemcpyDeviceToDevice, c->stream));
    return MOM_OK;
  };
  const int NB = c->outer_panels * nb;  // outer block: trailing updates run with K = NB
  for (int64_t J0 = 0; J0 < n; J0 += NB) {
    const int64_t NBc = std::min<int64_t>(NB, n - J0);
    for (int64_t j0 = J0; j0 < J0 + NBc; j0 += nb) {
      const int kb = (int)(j0 / nb);
      const int64_t m = n - j0;
      {
        ProfScope ps(c, kProfPanel);
        MOM_TRY(launch_panel<T>(c, A, lda, n, j0, panel_ctas(c, m, kPanelMaxRows<T>), c->ipiv, w.info, w));
      }
      {
        ProfScope pz(c, kProfPivotAux);
        if (n > nb) {
          pivot_map_kernel<<<1, 32, 0, c->stream>>>(c->ipiv, j0, nb, w.pmap, w.pmap + 128, w.pmap + 256);
          laswp_kernel<T><<<(unsigned)(((n - nb) * 32 + 255) / 256), 256, 0, c->stream>>>(A, lda, n, j0, nb, w.pmap,
                                                                                          w.pmap + 128, w.pmap + 256);
          c->launches += 2;
        }
      }
      {
        // inv(L11) now (the block TRSM needs it); inv(U11) of all blocks after the loop
        ProfScope pd(c, kProfDiagInv);
        diag_inv_kernel<T, 0><<<1, kDiagThreads, sizeof(double2) * (3 * nb * nb + nb), c->stream>>>(
            A, lda, kb, c->invd, mixed ? w.invL32 : nullptr);
        c->launches++;
        MOM_CUDA(c, cudaGetLastError());
      }
      // update the rest of the outer block: U = inv(L_jj) A_j,rest ; A_below,rest -= L_below,j U
      const int64_t rest = J0 + NBc - (j0 + nb);
      if (rest > 0) {
        ProfScope pg(c, kProfGemm);
        MOM_TRY(trsm_l(j0, j0 + nb, rest, kb));
        MOM_TRY(update64(n - j0 - nb, rest, A + (j0 + nb) + j0 * lda, A + j0 + (j0 + nb) * lda,
                         A + (j0 + nb) + (j0 + nb) * lda));
      }
    }
    // trailing columns: block-row TRSM with L_JJ, then A22 -= L21 U12 with K = NBc
    const int64_t t0 = J0 + NBc, nc = n - t0;
    if (nc > 0) {
      ProfScope pg(c, kProfGemm);
      for (int64_t j0 = J0; j0 < J0 + NBc; j0 += nb) {
        MOM_TRY(trsm_l(j0, t0, nc, (int)(j0 / nb)));
        const int64_t below = J0 + NBc - (j0 + nb);
        MOM_TRY(update64(below, nc, A + (j0 + nb) + j0 * lda, A + j0 + t0 * lda, A + (j0 + nb) + t0 * lda));
      }
      if (mixed) {
        // the large update on the tensor cores (3xTF32, FP32-accurate)
        MOM_TRY(tc_cgemm_update(c, reinterpret_cast<float2 *>(A + t0 + t0 * lda), lda,
                                reinterpret_cast<const float2 *>(A + t0 + J0 * lda), lda,
                                reinterpret_cast<const float2 *>(A + J0 + t0 * lda), lda, (int)(n - t0), (int)nc,
                                (int)NBc, w.tcw, c->dinfo + 2));
      } else {
        MOM_TRY(gemm(n - t0, nc, NBc, -1.0, A + t0 + J0 * lda, lda, A + J0 + t0 * lda, lda, 1.0, A + t0 + t0 * lda,
                     lda));
      }
    }
  }
  MOM_BLAS(c, cublasSetMathMode(c->blas, CUBLAS_DEFAULT_MATH));
  {
    // inv(U11) of every diagonal block (only the solves need them), one CTA per block
    ProfScope pd(c, kProfDiagInv);
    diag_inv_kernel<T, 1><<<(unsigned)(n / nb), kDiagThreads, sizeof(double2) * (3 * nb * nb + nb), c->stream>>>(
        A, lda, 0, c->invd, nullptr);
    c->launches++;
    MOM_CUDA(c, cudaGetLastError());
    if (mixed) {
      // FP32 copy of all inverses for the solves with the FP32 factors
      inv_to_fp32_kernel<<<c->nsm * 4, 256, 0, c->stream>>>(c->invd, c->inv32, 2 * (int64_t)nb * n);
      c->launches++;
      MOM_CUDA(c, cudaGetLastError());
    }
  }
  compose_pivots_kernel<<<1, 256, sizeof(int) * n, c->stream>>>(c->ipiv, (int)n, c->perm);
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  return MOM_OK;
}

// The mixed-precision factorisation with look-ahead.  Right-looking over
// outer blocks of NB = outer_panels * 64 columns as lu_enqueue, reordered so
// that the next outer block is factored on the second stream while the
// trailing update of the current one runs:
//   stream 1: J's interchanges on every column outside J; the block-row
//             TRSM and update of J on the next block's columns (L), then
//             record eL; the same on the rest (R), its tensor-core GEMM on
//             fewer SMs; then wait for eF;
//   stream 2: wait eL; factor block J+1 (panels, interchanges inside the
//             block only, diagonal inverses, in-block TRSM and updates on its
//             own cuBLAS handle); record eF.
// Interchanges commute with the row-wise trailing update, so applying a
// block's interchanges to the columns outside it after its factorisation
// (instead of panel by panel) gives the same factors; the columns left of
// the block are swapped at the same time (they hold L of earlier blocks,
// which nothing reads any more).  Blocks whose trailing height is above
// la_from * n, or whose panels need more than half of the SMs (over about
// 30,800 rows: at most 416 rows per FP32 panel CTA), run without the overlap
// (the panel would take too many SMs from the larger GEMM).
template <typename T>
int lu_enqueue_la(Ctx *c, T *A, const LuWork &w) {
  const int64_t n = c->n, lda = c->lda;
  const int nb = c->nb;
  const int NB = c->outer_panels * nb;
  cudaStream_t sa = c->stream, sb = c->stream2;
  if (sizeof(T) != sizeof(float2)) return fail(c, MOM_ERR_ARG, "the look-ahead schedule serves the mixed path");
  MOM_CUDA(c, cudaMemsetAsync(c->dinfo, 0, sizeof(int) * 4, sa));
  MOM_BLAS(c, cublasSetMathMode(c->blas, CUBLAS_DEFAULT_MATH));
  MOM_BLAS(c, cublasSetMathMode(c->blas2, CUBLAS_DEFAULT_MATH));
  auto gemm = [&](cublasHandle_t h, int64_t m, int64_t ncol, int64_t k, float alpha, const T *Am, int64_t la,
                  const T *Bm, int64_t lb, float beta, T *Cm, int64_t lc) -> int {
    if (m <= 0 || ncol <= 0 || k <= 0) return MOM_OK;
    c->blas_calls++;
    const cuComplex al = make_cuComplex(alpha, 0), be = make_cuComplex(beta, 0);
    MOM_BLAS(c, cublasCgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, (int)m, (int)ncol, (int)k, &al, (const cuComplex *)Am, (int)la,
                            (const cuComplex *)Bm, (int)lb, &be, (cuComplex *)Cm, (int)lc));
    return MOM_OK;
  };
  // B(nb x ncol at rows j0, columns col) <- inv(L_jj) B through the workspace Wk
  auto trsm_l = [&](cublasHandle_t h, cudaStream_t st, T *Wk, int64_t j0, int64_t col, int64_t ncol) -> int {
    if (ncol <= 0) return MOM_OK;
    const T *inv = (const T *)(w.invL32 + (size_t)(j0 / nb) * nb * nb);
    T *B = A + j0 + col * lda;
    MOM_TRY(gemm(h, nb, ncol, nb, 1.0f, inv, nb, B, lda, 0.0f, Wk, nb));
    MOM_CUDA(c, cudaMemcpy2DAsync(B, sizeof(T) * lda, Wk, sizeof(T) * nb, sizeof(T) * nb, ncol, cudaMemcpyDeviceToDevice,
                                  st));
    return MOM_OK;
  };
  // factor the outer block at J0 on stream st (panel CTAs capped at pcap > 0)
  auto factor_block = [&](int64_t J0, cudaStream_t st, cublasHandle_t h, int *pm, int pcap) -> int {
    const int64_t NBc = std::min<int64_t>(NB, n - J0);
    for (int64_t j0 = J0; j0 < J0 + NBc; j0 += nb) {
      const int p = (int)((j0 - J0) / nb), kb = (int)(j0 / nb);
      const int64_t m = n - j0;
      int P = panel_ctas(c, m, kPanelMaxRows<T>);
      if (pcap > 0) P = (int)std::max<int64_t>(std::min(P, pcap), (m + kPanelMaxRows<T> - 1) / kPanelMaxRows<T>);
      {
        ProfScope ps(c, kProfPanel, st);
        MOM_TRY(launch_panel<T>(c, A, lda, n, j0, P, c->ipiv, w.info, w, st));
      }
      {
        ProfScope pz(c, kProfPivotAux, st);
        int *mp = pm + 260 * p;
        pivot_map_kernel<<<1, 32, 0, st>>>(c->ipiv, j0, nb, mp, mp + 128, mp + 256);
        if (NBc > nb)
          laswp_range_kernel<T><<<(unsigned)((NBc * 32 + 255) / 256), 256, 0, st>>>(A, lda, J0, NBc, j0, nb, mp,
                                                                                      mp + 128, mp + 256);
        c->launches += NBc > nb ? 2 : 1;
      }
      {
        ProfScope pd(c, kProfDiagInv, st);
        diag_inv_kernel<T, 0><<<1, kDiagThreads, sizeof(double2) * (3 * nb * nb + nb), st>>>(A, lda, kb, c->invd,
                                                                                              w.invL32);
        c->launches++;
        MOM_CUDA(c, cudaGetLastError());
      }
      const int64_t rest = J0 + NBc - (j0 + nb);
      if (rest > 0) {
        ProfScope pg(c, kProfGemm, st);
        if (c->fused_trsm != 0 && nb == 64) {
          block_trsm_kernel<<<(unsigned)((rest + kBtCols - 1) / kBtCols), kBtThreads, kBtSmem, st>>>(
              reinterpret_cast<float2 *>(A), lda, j0, 1, j0 + nb, (int)rest, w.invL32 + (size_t)kb * nb * nb);
          c->launches++;
          MOM_CUDA(c, cudaGetLastError());
        } else {
          MOM_TRY(trsm_l(h, st, (T *)w.W2, j0, j0 + nb, rest));
        }
        MOM_TRY(gemm(h, n - j0 - nb, rest, nb, -1.0f, A + (j0 + nb) + j0 * lda, lda, A + j0 + (j0 + nb) * lda, lda,
                     1.0f, A + (j0 + nb) + (j0 + nb) * lda, lda));
      }
    }
    return MOM_OK;
  };
  // trailing update of block J0 on columns [c0, c0 + ncol), stream 1;
  // reuse_a: the previous trailing call was for the same block (its expanded
  // L21 is still in the work buffer: nothing between them writes L21 or it)
  auto trailing = [&](int64_t J0, int64_t c0, int64_t ncol, int gemm_ctas, bool reuse_a) -> int {
    if (ncol <= 0) return MOM_OK;
    const int64_t NBc = std::min<int64_t>(NB, n - J0), t0 = J0 + NBc;
    ProfScope pg(c, kProfGemm);
    if ((c->fused_trsm == 1 || (c->fused_trsm == 2 && ncol <= NB)) && NBc <= (int64_t)kBtMaxPanels * nb &&
        nb == 64) {
      block_trsm_kernel<<<(unsigned)((ncol + kBtCols - 1) / kBtCols), kBtThreads, kBtSmem, sa>>>(
          reinterpret_cast<float2 *>(A), lda, J0, (int)(NBc / nb), c0, (int)ncol, w.invL32 + (size_t)(J0 / nb) * nb * nb);
      c->launches++;
      MOM_CUDA(c, cudaGetLastError());
    } else {
      for (int64_t j0 = J0; j0 < t0; j0 += nb) {
        MOM_TRY(trsm_l(c->blas, sa, (T *)w.W, j0, c0, ncol));
        const int64_t below = t0 - (j0 + nb);
        MOM_TRY(gemm(c->blas, below, ncol, nb, -1.0f, A + (j0 + nb) + j0 * lda, lda, A + j0 + c0 * lda, lda, 1.0f,
                     A + (j0 + nb) + c0 * lda, lda));
      }
    }
    MOM_TRY(tc_cgemm_update(c, reinterpret_cast<float2 *>(A + t0 + c0 * lda), lda,
                            reinterpret_cast<const float2 *>(A + t0 + J0 * lda), lda,
                            reinterpret_cast<const float2 *>(A + J0 + c0 * lda), lda, (int)(n - t0), (int)ncol,
                            (int)NBc, w.tcw, c->dinfo + 2, gemm_ctas, reuse_a));
    return MOM_OK;
  };
  // stream 2 joins the stream (and any capture open on it)
  MOM_CUDA(c, cudaEventRecord(c->la_ev[0], sa));
  MOM_CUDA(c, cudaStreamWaitEvent(sb, c->la_ev[0], 0));
  MOM_TRY(factor_block(0, sa, c->blas, w.pmb, 0));
  for (int64_t J0 = 0; J0 < n; J0 += NB) {
    const int J = (int)(J0 / NB);
    const int64_t NBc = std::min<int64_t>(NB, n - J0), t0 = J0 + NBc, nc = n - t0;
    int *pmJ = w.pmb + 260 * 16 * (J & 1), *pmN = w.pmb + 260 * 16 * ((J + 1) & 1);
    const int64_t L = std::min<int64_t>(NB, nc);
    // block J's interchanges: first on the next block's L columns (outside
    // numbering [J0, J0 + L)), which its panels need; the other columns follow
    // beside those panels
    auto swaps = [&](int64_t lo, int64_t hi, int64_t slo, int64_t shi) -> int {
      if (hi <= lo) return MOM_OK;
      ProfScope pz(c, kProfPivotAux);
      laswp_block_kernel<T><<<(unsigned)(((hi - lo) * 32 + 255) / 256), 256, 0, sa>>>(A, lda, n, J0, NBc, pmJ,
                                                                                      (int)(NBc / nb), lo, hi, slo, shi);
      c->launches++;
      MOM_CUDA(c, cudaGetLastError());
      return MOM_OK;
    };
    if (nc <= 0) {
      MOM_TRY(swaps(0, n - NBc, 0, 0));
      break;
    }
    MOM_TRY(swaps(J0, J0 + L, 0, 0));
    MOM_TRY(trailing(J0, t0, L, 0, false));
    // overlap only where the next block's panels leave the GEMM at least half
    // of the SMs
    constexpr int64_t R = kPanelMaxRows<T>;
    const bool overlap = (double)nc < c->la_from * (double)n && nc > L && (nc + R - 1) / R <= c->nsm / 2;
    if (overlap) {
      // panel CTAs of the next block (the tallest of its panels), the GEMM gets the rest
      int P = panel_ctas(c, nc, R);
      const int pcap = c->la_ctas > 0 ? c->la_ctas : 1;
      P = (int)std::max<int64_t>(std::min(P, pcap), (nc + R - 1) / R);
      if (c->panel_cluster > 0 && nc <= (int64_t)kClusterRows<T> * c->panel_cluster) P = c->panel_cluster;
      MOM_CUDA(c, cudaEventRecord(c->la_ev[1], sa));
      MOM_CUDA(c, cudaStreamWaitEvent(sb, c->la_ev[1], 0));
      MOM_TRY(factor_block(t0, sb, c->blas2, pmN, pcap));
      MOM_CUDA(c, cudaEventRecord(c->la_ev[2], sb));
      MOM_TRY(swaps(0, n - NBc, J0, J0 + L));
      MOM_TRY(trailing(J0, t0 + L, nc - L, std::max(8, c->nsm - P), true));
      MOM_CUDA(c, cudaStreamWaitEvent(sa, c->la_ev[2], 0));
    } else {
      MOM_TRY(swaps(0, n - NBc, J0, J0 + L));
      MOM_TRY(trailing(J0, t0 + L, nc - L, 0, true));
      MOM_TRY(factor_block(t0, sa, c->blas, pmN, 0));
    }
  }
  // stream 2 rejoins stream 1 (closes any capture branch it holds)
  MOM_CUDA(c, cudaEventRecord(c->la_ev[2], sb));
  MOM_CUDA(c, cudaStreamWaitEvent(sa, c->la_ev[2], 0));
  {
    ProfScope pd(c, kProfDiagInv);
    diag_inv_kernel<T, 1><<<(unsigned)(n / nb), kDiagThreads, sizeof(double2) * (3 * nb * nb + nb), sa>>>(
        A, lda, 0, c->invd, nullptr);
    c->launches++;
    MOM_CUDA(c, cudaGetLastError());
    inv_to_fp32_kernel<<<c->nsm * 4, 256, 0, sa>>>(c->invd, c->inv32, 2 * (int64_t)nb * n);
    c->launches++;
    MOM_CUDA(c, cudaGetLastError());
  }
  compose_pivots_kernel<<<1, 256, sizeof(int) * n, sa>>>(c->ipiv, (int)n, c->perm);
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  return MOM_OK;
}

// The look-ahead schedule serves the mixed path (tensor-core trailing
// updates) with at least two outer blocks.
bool use_lookahead(const Ctx *c, int precision) {
  return c->lookahead && precision == MOM_PREC_MIXED && !c->small_tc && c->outer_panels <= 16 &&
         c->n > 2 * (int64_t)c->outer_panels * c->nb;
}

// Captures the factorisation of this precision into g (replacing what g held).
template <typename T>
int lu_capture(Ctx *c, T *A, int precision, const LuWork &w, Ctx::LuGraph &g, const std::vector<uintptr_t> &key) {
  g.reset();
  const int64_t l0 = c->launches, b0 = c->blas_calls;
  const double f0 = c->tc_flops;
  MOM_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  c->capturing = true;
  const int st = use_lookahead(c, precision) ? lu_enqueue_la<T>(c, A, w) : lu_enqueue<T>(c, A, precision, w);
  c->capturing = false;
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
  g.ev.swap(c->cap_ev);
  c->cap_ev.clear();
  g.launches = c->launches - l0;
  g.blas_calls = c->blas_calls - b0;
  g.tc_flops = c->tc_flops - f0;
  c->launches = l0;  // counted again on every replay
  c->blas_calls = b0;
  c->tc_flops = f0;
  if (st != MOM_OK || e != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    g.reset();
    return st != MOM_OK ? st : cuda_fail(c, e, "cudaStreamEndCapture (LU factorisation)");
  }
  const cudaError_t ei = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ei != cudaSuccess) {
    g.exec = nullptr;
    g.reset();
    return cuda_fail(c, ei, "cudaGraphInstantiate (LU factorisation)");
  }
  g.key = key;
  return MOM_OK;
}

template <typename T>
int lu_factor_t(Ctx *c, T *A, int precision) {
  const int64_t n = c->n;
  const int nb = c->nb;
  if (n % nb != 0) return fail(c, MOM_ERR_ARG, "matrix order must be a multiple of the panel width");
  if (nb != kDiagNb) return fail(c, MOM_ERR_ARG, "panel width must be 64");
  LuWork w;
  MOM_TRY(lu_workspace(c, precision, w));
  Ctx::LuGraph *g = nullptr;
  // the whole factorisation on the context stream (its wall time, with the
  // look-ahead stream joined in before the end event)
  {
  ProfScope pl(c, kProfLu);
  if (c->use_graph) {
    // Everything the captured launches bake in: sizes, buffer addresses, the
    // SM count (panel grid) and whether timing events are part of the graph.
    const std::vector<uintptr_t> key = {(uintptr_t)n,         (uintptr_t)c->lda,   (uintptr_t)nb,
                                        (uintptr_t)A,         (uintptr_t)c->ws,    (uintptr_t)c->ws_bytes,
                                        (uintptr_t)c->ipiv,   (uintptr_t)c->invd,  (uintptr_t)c->perm,
                                        (uintptr_t)c->dinfo,  (uintptr_t)c->nsm,   (uintptr_t)c->prof,
                                        (uintptr_t)tune_hash(c), (uintptr_t)c->outer_panels, (uintptr_t)c->inv32,
                                        (uintptr_t)wait_polls(c, 0), (uintptr_t)wait_polls(c, 1),
                                        (uintptr_t)use_lookahead(c, precision), (uintptr_t)c->la_ctas,
                                        (uintptr_t)(c->la_from * 1e6), (uintptr_t)c->fused_trsm};
    for (Ctx::LuGraph *h : c->lu_graphs)
      if (h->exec && h->key == key) g = h;
    if (!g) {
      // one graph per (precision, representation); the oldest goes first
      if (c->lu_graphs.size() >= 2 * (size_t)kMaxGroup) {
        c->lu_graphs.front()->reset();
        delete c->lu_graphs.front();
        c->lu_graphs.erase(c->lu_graphs.begin());
      }
      g = new Ctx::LuGraph();
      c->lu_graphs.push_back(g);
      const int rc = lu_capture<T>(c, A, precision, w, *g, key);
      if (rc != MOM_OK) {
        delete g;
        c->lu_graphs.pop_back();
        return rc;
      }
    }
    MOM_CUDA(c, cudaGraphLaunch(g->exec, c->stream));
    c->launches += g->launches;
    c->blas_calls += g->blas_calls;
    c->tc_flops += g->tc_flops;
  } else {
    MOM_TRY(use_lookahead(c, precision) ? lu_enqueue_la<T>(c, A, w) : lu_enqueue<T>(c, A, precision, w));
  }
  }
  int hinfo[3] = {0, 0, 0};
  MOM_CUDA(c, cudaMemcpyAsync(hinfo, c->dinfo, sizeof(int) * 3, cudaMemcpyDeviceToHost, c->stream));
  MOM_CUDA(c, cudaStreamSynchronize(c->stream));
  if (g && c->prof) {
    for (auto &e : g->ev) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, std::get<1>(e), std::get<2>(e)) == cudaSuccess) c->prof_ms[std::get<0>(e)] += ms;
      c->prof_launch[std::get<0>(e)]++;
    }
  }
  if (hinfo[1]) return fail(c, MOM_ERR_TIMEOUT, "panel factorisation barrier timed out");
  if (hinfo[2]) return fail(c, MOM_ERR_TIMEOUT, "tensor-core GEMM wait timed out");
  if (hinfo[0]) {
    c->factored = -1;
    return fail(c, MOM_ERR_SINGULAR, "Matrix factorization failed! (zero pivot at column " + std::to_string(hinfo[0]) + ")");
  }
  c->factored = precision;
  return MOM_OK;
}

// X (n x nrhs, ld n) <- A^{-1} X (TR: A^{-T} X) with the factors in place;
// Y is scratch.
template <typename T, bool TR = false>
int getrs_t(Ctx *c, const T *A, double2 *X, double2 *Y, double2 *Z, int nrhs) {
  const int64_t n = c->n;
  const int nb = c->nb;
  ProfScope ps(c, kProfTrsv);
  // whole 64-row blocks per CTA (each block has exactly one owner)
  const int nblk = (int)(n / nb);
  const int bpc = (nblk + c->nsm - 1) / c->nsm;
  const int rpc = bpc * nb;
  const int P = (nblk + bpc - 1) / bpc;
  auto kernel_of = [](int ns) -> void * {
    return ns == 1 ? (void *)trsv_flow_kernel<T, 1, TR>
           : ns == 2 ? (void *)trsv_flow_kernel<T, 2, TR>
           : ns == 4 ? (void *)trsv_flow_kernel<T, 4, TR>
                     : (void *)trsv_flow_kernel<T, 8, TR>;
  };
  const size_t tile_elems = TR ? (size_t)rpc * (nb + 1) : (size_t)nb * (rpc + 64 / sizeof(T));
  const size_t tile_bytes = ((sizeof(T) * tile_elems + 15) / 16) * 16, inv_bytes = sizeof(T) * nb * nb;
  const T *inv = sizeof(T) == sizeof(float2) ? (const T *)c->inv32 : (const T *)c->invd;
  for (int s0 = 0, ns = 0; s0 < nrhs; s0 += ns) {
    ns = 8;
    while (ns > nrhs - s0) ns >>= 1;  // chunks of 8, 4, 2, 1 vectors
    // shared memory: own rows, then per stage one inverse and (unless direct) one tile
    int stages = 0, direct = 0;
    size_t smem = 0;
    for (;;) {
      cudaFuncAttributes fa;
      MOM_CUDA(c, cudaFuncGetAttributes(&fa, kernel_of(ns)));
      const size_t cap = (size_t)fa.maxDynamicSharedSizeBytes, own = sizeof(double2) * (size_t)ns * rpc;
      const size_t opt[3][2] = {{2, 0}, {1, 0}, {1, 1}};
      for (int o = 0; o < 3 && !stages; o++) {
        const size_t need = own + opt[o][0] * (inv_bytes + (opt[o][1] ? 0 : tile_bytes));
        if (need <= cap) {
          stages = (int)opt[o][0];
          direct = (int)opt[o][1];
          smem = need;
        }
      }
      if (stages || ns == 1) break;
      ns >>= 1;
    }
    if (!stages) return fail(c, MOM_ERR_ARG, "matrix order too large for the triangular solve");
    TrsvArgs ta;
    ta.M = A;
    ta.lda = c->lda;
    ta.n = n;
    ta.nb = nb;
    ta.P = P;
    ta.rpc = rpc;
    ta.ns = ns;
    ta.inv = inv;
    ta.perm = c->perm;
    ta.X = X + (size_t)s0 * n;
    ta.Y = Y + (size_t)s0 * n;
    ta.Z = Z + (size_t)s0 * n;
    ta.timeout = c->dinfo + 1;
    ta.spin = wait_polls(c, 2);
    ta.direct = direct;
    ta.stages = stages;
    MOM_CUDA(c, cudaMemsetAsync(ta.Y, 0, sizeof(double2) * ns * n, c->stream));
    MOM_CUDA(c, cudaMemsetAsync(ta.Z, 0, sizeof(double2) * ns * n, c->stream));
    void *args[] = {&ta};
    MOM_CUDA(c, cudaLaunchCooperativeKernel(kernel_of(ns), dim3(P), dim3(256), args, smem, c->stream));
    c->launches++;
  }
  return MOM_OK;
}


// Opt a kernel in to all the dynamic shared memory the device allows next to
// its static shared memory.
template <typename T>
cudaError_t set_smem(T *fn) {
  int dev = 0, optin = 0;
  cudaFuncAttributes fa;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

}  // namespace

// Shared-memory opt-in of the LU kernels, once per context (outside any
// stream capture and off the factorisation's critical path).
// Largest cluster (power of two <= 16) with one panel CTA per SM that the
// device can schedule; 0 when clusters are unavailable.
template <typename T>
int max_panel_cluster() {
  if (cudaFuncSetAttribute(panel_cluster_kernel<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
    cudaGetLastError();
    return 8;
  }
  for (int cl = kMaxCluster; cl >= 2; cl /= 2) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cl);
    cfg.blockDim = dim3(kPanelThreads);
    cfg.dynamicSmemBytes = sizeof(typename SlabOf<T>::type) * (64 * kClusterRows<T> + 2 * cl * 64 + 2 * 64);
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, panel_cluster_kernel<T>, &cfg) == cudaSuccess && nclusters >= 1)
      return cl;
    cudaGetLastError();
  }
  return 0;
}

int lu_init_kernels(Ctx *c) {
  MOM_CUDA(c, set_smem(panel_kernel<double2>));
  MOM_CUDA(c, set_smem(panel_kernel<float2>));
  MOM_CUDA(c, set_smem(panel_cluster_kernel<double2>));
  MOM_CUDA(c, set_smem(panel_cluster_kernel<float2>));
  c->panel_cluster = std::min(max_panel_cluster<double2>(), max_panel_cluster<float2>());
  const char *ec = std::getenv("MOM_PANEL_CLUSTER");
  if (ec) c->panel_cluster = std::max(0, std::min(c->panel_cluster, std::atoi(ec)));
  MOM_CUDA(c, set_smem(diag_inv_kernel<double2, 0>));
  MOM_CUDA(c, set_smem(diag_inv_kernel<float2, 0>));
  MOM_CUDA(c, set_smem(diag_inv_kernel<double2, 1>));
  MOM_CUDA(c, set_smem(diag_inv_kernel<float2, 1>));
  MOM_CUDA(c, set_smem(compose_pivots_kernel));
  MOM_CUDA(c, cudaFuncSetAttribute(block_trsm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBtSmem));
  MOM_CUDA(c, set_smem(trsv_flow_kernel<double2, 1, false>));
  MOM_CUDA(c, set_smem(trsv_flow_kernel<double2, 2, false>));
  MOM_CUDA(c, set_smem(trsv_flow_kernel<double2, 4, false>));
  MOM_CUDA(c, set_smem(trsv_flow_kernel<double2, 8, false>));
  MOM_CUDA(c, set_smem(trsv_flow_kernel<float2, 1, false>));
  MOM_CUDA(c, set_smem(trsv_flow_kernel<float2, 2, false>));
  MOM_CUDA(c, set_smem(trsv_flow_kernel<float2, 4, false>));
  MOM_CUDA(c, set_smem(trsv_flow_kernel<float2, 8, false>));
  MOM_CUDA(c, set_smem(trsv_flow_kernel<double2, 1, true>));
  MOM_CUDA(c, set_smem(trsv_flow_kernel<double2, 2, true>));
  MOM_CUDA(c, set_smem(trsv_flow_kernel<double2, 4, true>));
  MOM_CUDA(c, set_smem(trsv_flow_kernel<double2, 8, true>));
  MOM_CUDA(c, set_smem(trsv_flow_kernel<float2, 1, true>));
  MOM_CUDA(c, set_smem(trsv_flow_kernel<float2, 2, true>));
  MOM_CUDA(c, set_smem(trsv_flow_kernel<float2, 4, true>));
  MOM_CUDA(c, set_smem(trsv_flow_kernel<float2, 8, true>));
  return MOM_OK;
}

namespace {
}  // namespace

namespace {


// Autotuner of the panel parallelism.  The panel is latency bound: one
// device-wide pivot exchange per column, whose cost grows with the number of
// CTAs, against per-CTA update work that shrinks with it.  For panel heights
// m = n, n/2, n/4, ... (>= 128) the first 64 columns of the matrix, rows
// 0 .. m, are copied to a scratch panel and factored once per candidate CTA
// count (CUDA-event timed, best of two); the fastest count per height forms
// the table panel_ctas() interpolates (nearest height on a log scale).
template <typename T>
int tune_panels(Ctx *c, const T *A, Ctx::Tuned &t) {
  const int64_t n = c->n, lda = c->lda;
  const int nb = c->nb;
  LuWork w;
  MOM_TRY(lu_workspace(c, t.precision, w, 0));
  T *S = nullptr;
  int *ip = nullptr;
  if (cudaMalloc(&S, sizeof(T) * (size_t)n * nb) != cudaSuccess || cudaMalloc(&ip, sizeof(int) * 2 * nb) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(S);
    return fail(c, MOM_ERR_ALLOC, "autotune scratch allocation failed");
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int rc = MOM_OK;
  const int cands[] = {148, 120, 96, 80, 64, 48, 40, 32, 24, 16, 12, 8};
  // one panel of height m on P CTAs, best of two (milliseconds)
  auto trial = [&](int64_t m, int P, const LuWork &wk) -> double {
    double ms_min = 1e30;
    for (int rep = 0; rep < 2 && rc == MOM_OK; rep++) {
      const cudaError_t ce = cudaMemcpy2DAsync(S, sizeof(T) * m, A, sizeof(T) * lda, sizeof(T) * m, nb,
                                               cudaMemcpyDeviceToDevice, c->stream);
      if (ce != cudaSuccess) {
        rc = cuda_fail(c, ce, "panel autotune copy");
        break;
      }
      cudaEventRecord(e0, c->stream);
      rc = launch_panel<T>(c, S, m, m, 0, P, ip, ip + nb, wk);
      cudaEventRecord(e1, c->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) rc = cuda_fail(c, cudaGetLastError(), "panel autotune trial");
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      ms_min = std::min(ms_min, (double)ms);
    }
    return ms_min;
  };
  for (int64_t m = n; m >= 128 && rc == MOM_OK; m /= 2) {
    int best = c->nsm, last = -1;
    double best_ms = 1e30;
    // heights that run on one cluster have nothing to tune: one timed trial
    const bool clustered = c->panel_cluster > 0 && m <= (int64_t)kClusterRows<T> * c->panel_cluster;
    for (int cand : cands) {
      if (clustered && cand != cands[0]) break;
      const int P0 = (int)std::min<int64_t>(
          c->nsm, std::max<int64_t>(std::min<int64_t>(cand, (m + 7) / 8), (m + kPanelMaxRows<T> - 1) / kPanelMaxRows<T>));
      const int rpc = (int)((m + P0 - 1) / P0);
      const int P = (int)((m + rpc - 1) / rpc);
      if (P == last) continue;
      last = P;
      const double ms_min = trial(m, P, w);
      if (rc == MOM_OK && ms_min < best_ms) {
        best_ms = ms_min;
        best = P;
      }
    }
    if (m == n && !clustered && rc == MOM_OK) {
      // placement of the exchange buffers, at the tallest height with its best P
      for (int sl = 0; sl < kXSlots && rc == MOM_OK; sl++) {
        LuWork ws;
        rc = lu_workspace(c, t.precision, ws, sl);
        const double ms = sl == 0 ? best_ms : trial(m, best, ws);
        t.xslot_us.push_back(ms * 1e3 / nb);
        if (rc == MOM_OK && ms < best_ms) {
          best_ms = ms;
          t.xslot = sl;
        }
      }
      if (rc == MOM_OK) rc = lu_workspace(c, t.precision, w, t.xslot);
    }
    t.m.push_back(m);
    t.P.push_back(best);
    t.us.push_back(best_ms * 1e3 / nb);
  }
  int tmo = 0;
  cudaMemcpy(&tmo, c->dinfo + 1, sizeof(int), cudaMemcpyDeviceToHost);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(S);
  cudaFree(ip);
  if (rc == MOM_OK && tmo) rc = fail(c, MOM_ERR_TIMEOUT, "panel autotune trial timed out");
  return rc;
}

int lu_autotune(Ctx *c, int precision) {
  c->tune = nullptr;
  if (c->panel_cap_env > 0 || !c->autotune) return MOM_OK;
  for (const auto &t : c->tuned)
    if (t.n == c->n && t.precision == precision) {
      c->tune = &t;
      return MOM_OK;
    }
  Ctx::Tuned t;
  t.n = c->n;
  t.precision = precision;
  const bool prof = c->prof;
  c->prof = false;
  const int64_t l0 = c->launches;
  const auto t0 = std::chrono::steady_clock::now();
  MOM_CUDA(c, cudaMemsetAsync(c->dinfo, 0, sizeof(int) * 4, c->stream));
  const int rc = precision == MOM_PREC_MIXED ? tune_panels<float2>(c, c->A32, t) : tune_panels<double2>(c, c->A, t);
  c->prof = prof;
  c->launches = l0;
  if (rc != MOM_OK) return rc;
  t.ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  c->tuned.push_back(t);
  c->tune = &c->tuned.back();
  return MOM_OK;
}

}  // namespace

int lu_factor(Ctx *c, int precision) {
  MOM_TRY(lu_autotune(c, precision));
  if (precision == MOM_PREC_MIXED) return lu_factor_t<float2>(c, c->A32, precision);
  return lu_factor_t<double2>(c, c->A, precision);
}

namespace {

constexpr int kMultiRhs = 16;  // from this many right-hand sides on, the solves are GEMM based
constexpr int kMultiTc = 64;   // ... and with the FP32 factors, the block updates on the tensor cores

// Y = P X (mode 0), Y = X (mode 1) or Y[perm[i]] = X[i] (mode 2), with a
// type conversion, for nrhs columns.
template <typename TI, typename TO>
__global__ void permute_rows_kernel(const TI *X, int64_t ldx, TO *Y, int64_t ldy, int64_t n, const int *perm,
                                    int mode) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (i >= n) return;
  const int64_t src = mode == 0 ? perm[i] : i, dst = mode == 2 ? perm[i] : i;
  const TI v = X[(size_t)s * ldx + src];
  TO o;
  o.x = v.x;
  o.y = v.y;
  Y[(size_t)s * ldy + dst] = o;
}

template <typename T>
int blas_gemm(Ctx *c, cublasOperation_t ta, int m, int nn, int k, double alpha, const T *A, int64_t lda, const T *B,
              int64_t ldb, double beta, T *C, int64_t ldc);
template <>
int blas_gemm<double2>(Ctx *c, cublasOperation_t ta, int m, int nn, int k, double alpha, const double2 *A,
                       int64_t lda, const double2 *B, int64_t ldb, double beta, double2 *C, int64_t ldc) {
  const cuDoubleComplex al = make_cuDoubleComplex(alpha, 0), be = make_cuDoubleComplex(beta, 0);
  MOM_BLAS(c, cublasZgemm(c->blas, ta, CUBLAS_OP_N, m, nn, k, &al, (const cuDoubleComplex *)A, (int)lda,
                          (const cuDoubleComplex *)B, (int)ldb, &be, (cuDoubleComplex *)C, (int)ldc));
  c->blas_calls++;
  return MOM_OK;
}
template <>
int blas_gemm<float2>(Ctx *c, cublasOperation_t ta, int m, int nn, int k, double alpha, const float2 *A, int64_t lda,
                      const float2 *B, int64_t ldb, double beta, float2 *C, int64_t ldc) {
  const cuComplex al = make_cuComplex((float)alpha, 0), be = make_cuComplex((float)beta, 0);
  MOM_BLAS(c, cublasCgemm(c->blas, ta, CUBLAS_OP_N, m, nn, k, &al, (const cuComplex *)A, (int)lda,
                          (const cuComplex *)B, (int)ldb, &be, (cuComplex *)C, (int)ldc));
  c->blas_calls++;
  return MOM_OK;
}

// Many right-hand sides: blocked substitution with the diagonal-block
// inverses, every step a library GEMM (64-row blocks; the updates of the
// rows below / above are tall GEMMs with K = 64).  X (n x nrhs, ld n) is
// overwritten with A^{-1} X (trans: A^{-T} X).  T = float2 works on the FP32
// factors in FP32 (no TF32), T = double2 on the FP64 factors.
template <typename T>
int getrs_multi(Ctx *c, const T *F, double2 *X, int nrhs, int trans) {
  const int64_t n = c->n, lda = c->lda;
  const int nb = c->nb, nblk = (int)(n / nb);
  const bool f32 = sizeof(T) == sizeof(float2);
  // FP32 factors and many right-hand sides: 256-row blocks whose updates run
  // on the tensor cores (3xTF32, FP32-accurate like the rest of the solve)
  const bool tc = f32 && nrhs >= kMultiTc;
  const int64_t NBt = 4 * (int64_t)nb;
  const size_t ybytes = sizeof(T) * (size_t)n * nrhs, tbytes = sizeof(T) * (size_t)nb * nrhs;
  const size_t o_t = ((ybytes + 255) / 256) * 256, o_w = o_t + ((tbytes + 255) / 256) * 256;
  const size_t wbytes = tc ? tc_cgemm_work_bytes((int)n, nrhs, (int)NBt) : 0;
  MOM_TRY(ensure_buffer(c, &c->ws2, &c->ws2_bytes, o_w + wbytes + 1024));
  T *Y = (T *)c->ws2;
  T *Tm = (T *)((char *)c->ws2 + o_t);
  float *tw = (float *)((char *)c->ws2 + o_w);
  const T *inv = f32 ? (const T *)c->inv32 : (const T *)c->invd;
  ProfScope ps(c, kProfTrsv);
  const dim3 pg((unsigned)((n + 255) / 256), nrhs);
  permute_rows_kernel<double2, T><<<pg, 256, 0, c->stream>>>(X, n, Y, n, n, c->perm, trans ? 1 : 0);
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  MOM_BLAS(c, cublasSetMathMode(c->blas, CUBLAS_DEFAULT_MATH));
  const cublasOperation_t op = trans ? CUBLAS_OP_T : CUBLAS_OP_N;
  // block k of the pass: y_k <- inv_k y_k (through Tm), then the update
  auto diag = [&](int kb, int which) -> int {
    const int64_t k0 = (int64_t)kb * nb;
    MOM_TRY(blas_gemm<T>(c, op, nb, nrhs, nb, 1.0, inv + ((size_t)kb * 2 + which) * nb * nb, nb, Y + k0, n, 0.0, Tm,
                         nb));
    MOM_CUDA(c, cudaMemcpy2DAsync(Y + k0, sizeof(T) * n, Tm, sizeof(T) * nb, sizeof(T) * nb, nrhs,
                                  cudaMemcpyDeviceToDevice, c->stream));
    return MOM_OK;
  };
  if (tc) {
    // forward: L (unit lower), or U^T; 64-row blocks inside a 256-row block
    // with the library GEMM, the rows below the 256-row block on the tensor cores
    for (int64_t K0 = 0; K0 < n; K0 += NBt) {
      const int64_t K1 = std::min<int64_t>(K0 + NBt, n);
      for (int64_t k0 = K0; k0 < K1; k0 += nb) {
        MOM_TRY(diag((int)(k0 / nb), trans ? 1 : 0));
        const int64_t mi = K1 - k0 - nb;
        if (mi > 0) {
          const T *Ab = trans ? F + k0 + (k0 + nb) * lda : F + (k0 + nb) + k0 * lda;
          MOM_TRY(blas_gemm<T>(c, op, (int)mi, nrhs, nb, -1.0, Ab, lda, Tm, nb, 1.0, Y + k0 + nb, n));
        }
      }
      if (K1 < n) {
        const T *Ab = trans ? F + K0 + K1 * lda : F + K1 + K0 * lda;
        MOM_TRY(tc_cgemm_update(c, reinterpret_cast<float2 *>(Y + K1), n, reinterpret_cast<const float2 *>(Ab), lda,
                                reinterpret_cast<const float2 *>(Y + K0), n, (int)(n - K1), nrhs, (int)(K1 - K0), tw,
                                c->dinfo + 2, 0, false, trans != 0));
      }
    }
    // backward: U, or L^T (unit upper)
    for (int64_t K0 = ((n - 1) / NBt) * NBt; K0 >= 0; K0 -= NBt) {
      const int64_t K1 = std::min<int64_t>(K0 + NBt, n);
      for (int64_t k0 = K1 - nb; k0 >= K0; k0 -= nb) {
        MOM_TRY(diag((int)(k0 / nb), trans ? 0 : 1));
        if (k0 > K0) {
          const T *Ab = trans ? F + k0 + K0 * lda : F + K0 + k0 * lda;
          MOM_TRY(blas_gemm<T>(c, op, (int)(k0 - K0), nrhs, nb, -1.0, Ab, lda, Tm, nb, 1.0, Y + K0, n));
        }
      }
      if (K0 > 0) {
        const T *Ab = trans ? F + K0 : F + K0 * lda;
        MOM_TRY(tc_cgemm_update(c, reinterpret_cast<float2 *>(Y), n, reinterpret_cast<const float2 *>(Ab), lda,
                                reinterpret_cast<const float2 *>(Y + K0), n, (int)K0, nrhs, (int)(K1 - K0), tw,
                                c->dinfo + 2, 0, false, trans != 0));
      }
    }
    permute_rows_kernel<T, double2><<<pg, 256, 0, c->stream>>>(Y, n, X, n, n, c->perm, trans ? 2 : 1);
    c->launches++;
    MOM_CUDA(c, cudaGetLastError());
    return MOM_OK;
  }
  // forward: L (unit lower), or U^T; backward: U, or L^T (unit upper)
  for (int kb = 0; kb < nblk; kb++) {
    const int64_t k0 = (int64_t)kb * nb, m = n - k0 - nb;
    MOM_TRY(diag(kb, trans ? 1 : 0));
    if (m > 0) {
      const T *Ab = trans ? F + k0 + (k0 + nb) * lda : F + (k0 + nb) + k0 * lda;
      MOM_TRY(blas_gemm<T>(c, op, (int)m, nrhs, nb, -1.0, Ab, lda, Tm, nb, 1.0, Y + k0 + nb, n));
    }
  }
  for (int kb = nblk - 1; kb >= 0; kb--) {
    const int64_t k0 = (int64_t)kb * nb;
    MOM_TRY(diag(kb, trans ? 0 : 1));
    if (k0 > 0) {
      const T *Ab = trans ? F + k0 : F + k0 * lda;
      MOM_TRY(blas_gemm<T>(c, op, (int)k0, nrhs, nb, -1.0, Ab, lda, Tm, nb, 1.0, Y, n));
    }
  }
  permute_rows_kernel<T, double2><<<pg, 256, 0, c->stream>>>(Y, n, X, n, n, c->perm, trans ? 2 : 1);
  c->launches++;
  MOM_CUDA(c, cudaGetLastError());
  return MOM_OK;
}

}  // namespace

// Solve A X = B (trans: A^T X = B) for nrhs columns (ld n) with the factors
// of `precision` in place.  FP64: one triangular solve.  Mixed: x = 0,
// r = b; repeat d = LU32^{-1} r, x += d, r = b - A x with the FP64 matrix
// until max_s ||r_s|| / ||b_s|| <= tol.
int lu_solve_ex(Ctx *c, int precision, int trans, const double2 *B, double2 *X, int nrhs, double tol, int maxit,
                int *iters) {
  const int64_t n = c->n;
  if (c->factored != precision) return fail(c, MOM_ERR_STATE, "matrix not factored in this precision");
  const size_t vec = sizeof(double2) * (size_t)n * nrhs;
  if (precision == MOM_PREC_FP64) {
    if (X != B) MOM_CUDA(c, cudaMemcpyAsync(X, B, vec, cudaMemcpyDeviceToDevice, c->stream));
    if (nrhs >= kMultiRhs) {
      MOM_TRY(getrs_multi<double2>(c, c->A, X, nrhs, trans));
    } else {
      MOM_TRY(ensure_buffer(c, &c->ws, &c->ws_bytes, 2 * vec));
      double2 *Yw = (double2 *)c->ws, *Zw = (double2 *)((char *)c->ws + vec);
      if (trans) MOM_TRY((getrs_t<double2, true>(c, c->A, X, Yw, Zw, nrhs)));
      else MOM_TRY((getrs_t<double2, false>(c, c->A, X, Yw, Zw, nrhs)));
    }
    if (iters) *iters = 0;
    int tmo = 0;
    MOM_CUDA(c, cudaMemcpyAsync(&tmo, c->dinfo + 1, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    MOM_CUDA(c, cudaStreamSynchronize(c->stream));
    if (tmo) return fail(c, MOM_ERR_TIMEOUT, "triangular solve barrier timed out");
    return MOM_OK;
  }
  const int nchunk = (int)((n + kGemvCols - 1) / kGemvCols);
  const int rblocks = (int)((n + 255) / 256);
  const size_t off_r = 0, off_d = vec, off_y = 2 * vec, off_p = 3 * vec;
  const size_t part = sizeof(double2) * (size_t)nchunk * 8 * n;
  const size_t off_n = off_p + part;
  const size_t off_z = off_n + ((sizeof(double) * rblocks * nrhs + 255) / 256) * 256;
  MOM_TRY(ensure_buffer(c, &c->ws, &c->ws_bytes, off_z + vec + 256));
  char *ws = (char *)c->ws;
  double2 *R = (double2 *)(ws + off_r), *Dv = (double2 *)(ws + off_d), *Yv = (double2 *)(ws + off_y),
          *Pp = (double2 *)(ws + off_p), *Zv = (double2 *)(ws + off_z);
  double *rn2 = (double *)(ws + off_n);
  // ||b|| per column
  std::vector<double> bn(nrhs), h(rblocks * (size_t)nrhs);
  MOM_CUDA(c, cudaMemsetAsync(X, 0, vec, c->stream));
  MOM_CUDA(c, cudaMemcpyAsync(R, B, vec, cudaMemcpyDeviceToDevice, c->stream));
  residual_kernel<<<dim3(rblocks, nrhs), 256, 0, c->stream>>>(B, n, Pp, 0, n, nrhs, R, n, rn2);
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
    const bool multi = nrhs >= kMultiRhs;
    if (multi) MOM_TRY(getrs_multi<float2>(c, c->A32, Dv, nrhs, trans));
    else if (trans) MOM_TRY((getrs_t<float2, true>(c, c->A32, Dv, Yv, Zv, nrhs)));
    else MOM_TRY((getrs_t<float2, false>(c, c->A32, Dv, Yv, Zv, nrhs)));
    axpy_kernel<<<c->nsm * 4, 256, 0, c->stream>>>(X, Dv, (int64_t)n * nrhs);
    c->launches++;
    ProfScope pr(c, kProfResidual);
    if (multi) {
      // R = B - op(A) X as one FP64 library GEMM, then the column norms
      MOM_CUDA(c, cudaMemcpyAsync(R, B, vec, cudaMemcpyDeviceToDevice, c->stream));
      MOM_TRY(blas_gemm<double2>(c, trans ? CUBLAS_OP_T : CUBLAS_OP_N, (int)n, nrhs, (int)n, -1.0, c->A, c->lda, X,
                                 n, 1.0, R, n));
      residual_kernel<<<dim3(rblocks, nrhs), 256, 0, c->stream>>>(R, n, Pp, 0, n, nrhs, R, n, rn2);
      c->launches++;
    }
    for (int s0 = 0, ns = 0; !multi && s0 < nrhs; s0 += ns) {
      ns = 8;
      while (ns > nrhs - s0) ns >>= 1;
      const double2 *xs0 = X + (size_t)s0 * n;
      int nch = nchunk;
      if (trans) {
        const unsigned gb = (unsigned)((n + 7) / 8);
        if (ns == 1) gemv_t_kernel<1><<<gb, 256, 0, c->stream>>>(c->A, c->lda, n, xs0, n, Pp);
        else if (ns == 2) gemv_t_kernel<2><<<gb, 256, 0, c->stream>>>(c->A, c->lda, n, xs0, n, Pp);
        else if (ns == 4) gemv_t_kernel<4><<<gb, 256, 0, c->stream>>>(c->A, c->lda, n, xs0, n, Pp);
        else gemv_t_kernel<8><<<gb, 256, 0, c->stream>>>(c->A, c->lda, n, xs0, n, Pp);
        nch = 1;
      } else {
        const dim3 gg(rblocks, nchunk);
        if (ns == 1) gemv_partial_kernel<1><<<gg, kGemvRows, 0, c->stream>>>(c->A, c->lda, n, xs0, n, Pp);
        else if (ns == 2) gemv_partial_kernel<2><<<gg, kGemvRows, 0, c->stream>>>(c->A, c->lda, n, xs0, n, Pp);
        else if (ns == 4) gemv_partial_kernel<4><<<gg, kGemvRows, 0, c->stream>>>(c->A, c->lda, n, xs0, n, Pp);
        else gemv_partial_kernel<8><<<gg, kGemvRows, 0, c->stream>>>(c->A, c->lda, n, xs0, n, Pp);
      }
      residual_kernel<<<dim3(rblocks, ns), 256, 0, c->stream>>>(B + (size_t)s0 * n, n, Pp, nch, n, ns,
                                                                R + (size_t)s0 * n, n, rn2 + (size_t)s0 * rblocks);
      c->launches += 2;
    }
    MOM_CUDA(c, cudaGetLastError());
    MOM_CUDA(c, cudaMemcpyAsync(h.data(), rn2, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream));
    int tmo[2] = {0, 0};
    MOM_CUDA(c, cudaMemcpyAsync(tmo, c->dinfo + 1, sizeof(int) * 2, cudaMemcpyDeviceToHost, c->stream));
    MOM_CUDA(c, cudaStreamSynchronize(c->stream));
    if (tmo[0]) return fail(c, MOM_ERR_TIMEOUT, "triangular solve barrier timed out");
    if (tmo[1]) return fail(c, MOM_ERR_TIMEOUT, "tensor-core GEMM wait timed out");
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

int matvec_acc(Ctx *c, const double2 *X, int nrhs, double2 *Y, double sign) {
  const int64_t n = c->n;
  const int nchunk = (int)((n + kGemvCols - 1) / kGemvCols);
  const int rblocks = (int)((n + kGemvRows - 1) / kGemvRows);
  MOM_TRY(ensure_buffer(c, &c->ws, &c->ws_bytes, sizeof(double2) * (size_t)nchunk * 8 * n));
  double2 *Pp = (double2 *)c->ws;
  for (int s0 = 0, ns = 0; s0 < nrhs; s0 += ns) {
    ns = 8;
    while (ns > nrhs - s0) ns >>= 1;
    const double2 *xs0 = X + (size_t)s0 * n;
    const dim3 gg(rblocks, nchunk);
    if (ns == 1) gemv_partial_kernel<1><<<gg, kGemvRows, 0, c->stream>>>(c->A, c->lda, n, xs0, n, Pp);
    else if (ns == 2) gemv_partial_kernel<2><<<gg, kGemvRows, 0, c->stream>>>(c->A, c->lda, n, xs0, n, Pp);
    else if (ns == 4) gemv_partial_kernel<4><<<gg, kGemvRows, 0, c->stream>>>(c->A, c->lda, n, xs0, n, Pp);
    else gemv_partial_kernel<8><<<gg, kGemvRows, 0, c->stream>>>(c->A, c->lda, n, xs0, n, Pp);
    acc_partials_kernel<<<dim3((unsigned)((n + 255) / 256), ns), 256, 0, c->stream>>>(Y + (size_t)s0 * n, n, Pp,
                                                                                     nchunk, n, ns, sign);
    c->launches += 2;
    MOM_CUDA(c, cudaGetLastError());
  }
  return MOM_OK;
}

// Solve for the nsrc right-hand sides in c->B into c->X.
int lu_solve(Ctx *c, int precision, double tol, int maxit, int *iters) {
  return lu_solve_ex(c, precision, 0, c->B, c->X, c->nsrc, tol, maxit, iters);
}

}  // namespace mom
