// Trailing-update GEMM of the mixed-precision LU on the sm_100a tensor cores.
//
//   C  -=  L21 * U12      (complex FP32, C = A22 of the LU, in place)
//
// Complex products are built from real ones: with C viewed as a real matrix
// (re/im interleaved rows, 2m x nc), L21 expanded to the real 2m x 2k matrix
//   Ahat[2i][2l] = Re L, Ahat[2i][2l+1] = -Im L, Ahat[2i+1][2l] = Im L,
//   Ahat[2i+1][2l+1] = Re L
// and U12 viewed as real 2k x nc (its own interleaved storage), C -= Ahat B.
// Accuracy: each operand is split into a TF32 high part and an FP32 low
// remainder, and the MMA accumulates hi*hi + hi*lo + lo*hi (three
// kind::tf32 passes into one FP32 TMEM accumulator), which keeps the
// factorisation close to FP32 accuracy so FP64 refinement converges in a
// few steps.
//
// Kernel: persistent, one CTA per SM, 128 x 256 output tiles, K blocks of
// 32 floats (one 128-byte swizzle atom) staged by TMA in a 2-deep ring.
//   warp 0   TMA producer (one elected lane)
//   warp 1   MMA issuer (one elected lane; tcgen05.mma cta_group::1)
//   warp 2   TMEM allocator (512 columns = two 128 x 256 accumulators)
//   warps 4-7 epilogue: tcgen05.ld the accumulator, C -= acc (coalesced)
// Every mbarrier wait is bounded; on timeout the kernel records the error,
// stops issuing work, waits (bounded) for its own copies and for the MMAs
// already issued, frees TMEM and exits.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "mom_internal.h"

namespace mom {
namespace {

constexpr int kBM = 128, kBN = 256, kBK = 32, kStages = 2;
constexpr int kTileA = kBM * kBK * 4;  // bytes of one A tile (hi or lo)
constexpr int kTileB = kBN * kBK * 4;  // bytes of one B tile
constexpr int kStageBytes = 2 * kTileA + 2 * kTileB;
constexpr int kTcThreads = 256;
constexpr long long kDrainPolls = 1LL << 22;  // bound of the waits for work already issued

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Bounded parity wait; returns false (and raises *abort) after `limit` polls,
// or when another warp of the CTA has raised *abort.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, volatile int *abort, long long limit) {
  const uint32_t a = smem_u32(bar);
  for (long long it = 0;; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 1023) == 1023 || it >= limit) {
      if (*abort) return false;
      if (it >= limit) {
        *abort = 1;
        return false;
      }
    }
  }
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// K-major, 128-byte swizzled operand tile: rows of 128 bytes, 8-row atoms of
// 1024 bytes (SBO), LBO unused (1), descriptor version 1, layout SWIZZLE_128B.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;            // LBO (16-byte units)
  d |= (uint64_t)(1024 >> 4) << 32;  // SBO
  d |= (uint64_t)1 << 46;            // version
  d |= (uint64_t)2 << 61;            // SWIZZLE_128B
  return d;
}

// kind::tf32 instruction descriptor: D f32, A/B tf32, both K-major, M=128, N=256.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kBN >> 3) << 17) |
                            ((uint32_t)(kBM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

struct TcArgs {
  float *C;        // real view of the complex FP32 C block
  int64_t ldc;     // in floats
  int Mr, Nc, Kr;  // real rows of C, columns, real K
  int *err;        // device error word (timeout)
  long long spin;  // polls before an mbarrier wait is declared timed out
};

__global__ void __launch_bounds__(kTcThreads, 1)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap mAhi, const __grid_constant__ CUtensorMap mAlo,
                   const __grid_constant__ CUtensorMap mBhi, const __grid_constant__ CUtensorMap mBlo, TcArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte aligned stage buffers (SWIZZLE_128B atoms need it)
  unsigned char *smem = reinterpret_cast<unsigned char *>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ uint64_t full[kStages], empty[kStages], acc_full[2], acc_empty[2], drain;
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int numM = a.Mr / kBM, numN = (a.Nc + kBN - 1) / kBN, ntiles = numM * numN, nk = a.Kr / kBK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 4);  // one arrival per epilogue warp
    }
    mbar_init(&drain, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  volatile int *abort = &abort_flag;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      int s = 0;
      unsigned ph = 0;
      unsigned last_ph[kStages];
      bool pending[kStages];
      for (int i = 0; i < kStages; i++) pending[i] = false;
      for (int t = blockIdx.x; t < ntiles && !*abort; t += gridDim.x) {
        const int tm = t % numM, tn = t / numM;
        for (int kb = 0; kb < nk; kb++) {
          if (!mbar_wait(&empty[s], ph ^ 1, abort, a.spin)) break;
          unsigned char *st = smem + (size_t)s * kStageBytes;
          mbar_expect_tx(&full[s], kStageBytes);
          tma_load_2d(st, &mAhi, &full[s], kb * kBK, tm * kBM);
          tma_load_2d(st + kTileA, &mAlo, &full[s], kb * kBK, tm * kBM);
          tma_load_2d(st + 2 * kTileA, &mBhi, &full[s], kb * kBK, tn * kBN);
          tma_load_2d(st + 2 * kTileA + kTileB, &mBlo, &full[s], kb * kBK, tn * kBN);
          pending[s] = true;
          last_ph[s] = ph;
          if (++s == kStages) {
            s = 0;
            ph ^= 1;
          }
        }
      }
      // wait (bounded) until the last copy into every stage has landed: the
      // MMA warp may give up on a stage whose copy is still in flight, and
      // the CTA must not exit before its shared memory is written
      volatile int dummy = 0;
      for (int i = 0; i < kStages; i++)
        if (pending[i]) mbar_wait(&full[i], last_ph[i], &dummy, kDrainPolls);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      int s = 0;
      unsigned ph = 0;
      int it = 0;
      for (int t = blockIdx.x; t < ntiles && !*abort; t += gridDim.x, it++) {
        const int acc = it & 1;
        const unsigned acc_ph = (it >> 1) & 1;
        if (!mbar_wait(&acc_empty[acc], acc_ph ^ 1, abort, a.spin)) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + (uint32_t)(acc * kBN);
        bool ok = true;
        for (int kb = 0; kb < nk; kb++) {
          if (!mbar_wait(&full[s], ph, abort, a.spin)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t base = smem_u32(smem + (size_t)s * kStageBytes);
          const uint32_t ahi = base, alo = base + kTileA, bhi = base + 2 * kTileA, blo = base + 2 * kTileA + kTileB;
#pragma unroll
          for (int k = 0; k < kBK / 8; k++) {
            const uint32_t off = (uint32_t)k * 32;  // 8 tf32 = 32 bytes along K inside the swizzle atom
            mma_tf32(d, sw128_desc(ahi + off), sw128_desc(bhi + off), (kb | k) != 0);
            mma_tf32(d, sw128_desc(ahi + off), sw128_desc(blo + off), 1);
            mma_tf32(d, sw128_desc(alo + off), sw128_desc(bhi + off), 1);
          }
          mma_commit(&empty[s]);  // frees the stage when these MMAs complete
          if (++s == kStages) {
            s = 0;
            ph ^= 1;
          }
        }
        if (!ok) break;
        mma_commit(&acc_full[acc]);
      }
      // on abort, wait (bounded) until every MMA issued so far has completed
      // (they read the stage buffers and write TMEM, both released below)
      if (*abort) {
        volatile int dummy = 0;
        mma_commit(&drain);
        mbar_wait(&drain, 0, &dummy, kDrainPolls);
      }
    }
  } else if (warp >= 4) {
    // ---------------- epilogue ----------------
    const int ew = warp - 4;  // TMEM lanes 32*ew .. 32*ew+31
    int it = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
      const int acc = it & 1;
      const unsigned acc_ph = (it >> 1) & 1;
      int ok = 1;
      if (lane == 0) ok = mbar_wait(&acc_full[acc], acc_ph, abort, a.spin) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int tm = t % numM, tn = t / numM;
      const int64_t row = (int64_t)tm * kBM + ew * 32 + lane;
      float *crow = a.C + row;
#pragma unroll 1
      for (int c0 = 0; c0 < kBN; c0 += 16) {
        uint32_t v[16];
        const uint32_t taddr = tmem + ((uint32_t)(ew * 32) << 16) + (uint32_t)(acc * kBN + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int col0 = tn * kBN + c0;
        // all 16 loads in flight before the stores (the stores could alias them otherwise)
        float cv[16];
#pragma unroll
        for (int j = 0; j < 16; j++) cv[j] = (col0 + j < a.Nc) ? __ldcs(crow + (int64_t)(col0 + j) * a.ldc) : 0.0f;
#pragma unroll
        for (int j = 0; j < 16; j++)
          if (col0 + j < a.Nc) __stcs(crow + (int64_t)(col0 + j) * a.ldc, cv[j] - __uint_as_float(v[j]));
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[acc]);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && abort_flag) atomicExch(a.err, 1);
  if (warp == 2) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
}

// Ahat_hi / Ahat_lo (Mr x Kr, row-major) from the complex block L (m x k, ld),
// or (tr) from the transpose of a k x m block: L(i, l) = P[l + i ld].  In
// 32 x 32 tiles through shared memory: the complex block is read along its
// contiguous direction and the expanded rows are written as FP32 pairs
// (block 32 x 8 threads).
__global__ void __launch_bounds__(256) expand_a_tiled_kernel(const float2 *L, int64_t ld, int m, int k, float *hi,
                                                             float *lo, bool tr) {
  __shared__ float2 t[32][33];  // [l][i] of the tile
  const int i0 = blockIdx.y * 32, l0 = blockIdx.x * 32, tx = threadIdx.x;
  for (int r = threadIdx.y; r < 32; r += 8) {
    if (!tr) {
      const int i = i0 + tx, l = l0 + r;
      t[r][tx] = (i < m && l < k) ? L[i + (int64_t)l * ld] : make_float2(0.f, 0.f);
    } else {
      const int l = l0 + tx, i = i0 + r;
      t[tx][r] = (i < m && l < k) ? L[l + (int64_t)i * ld] : make_float2(0.f, 0.f);
    }
  }
  __syncthreads();
  const int64_t Kr = 2 * (int64_t)k;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int i = i0 + r, l = l0 + tx;
    if (i >= m || l >= k) continue;
    const float2 z = t[tx][r];
    const float v[4] = {z.x, -z.y, z.y, z.x};  // rows 2i and 2i + 1, columns 2l and 2l + 1
    float h[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      uint32_t u;
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(u) : "f"(v[q]));
      h[q] = __uint_as_float(u);
    }
    const int64_t p0 = (2 * (int64_t)i) * Kr + 2 * l, p1 = p0 + Kr;
    *reinterpret_cast<float2 *>(hi + p0) = make_float2(h[0], h[1]);
    *reinterpret_cast<float2 *>(hi + p1) = make_float2(h[2], h[3]);
    *reinterpret_cast<float2 *>(lo + p0) = make_float2(v[0] - h[0], v[1] - h[1]);
    *reinterpret_cast<float2 *>(lo + p1) = make_float2(v[2] - h[2], v[3] - h[3]);
  }
}

// B_hi / B_lo (Nc x Kr, K contiguous) from the complex block U (k x nc, ld).
__global__ void split_b_kernel(const float2 *U, int64_t ld, int k, int nc, float *hi, float *lo) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)k * nc) return;
  const int l = (int)(idx % k), j = (int)(idx / k);
  const float2 z = U[l + (int64_t)j * ld];
  const int64_t base = (int64_t)j * 2 * k + 2 * l;
  const float vals[2] = {z.x, z.y};
#pragma unroll
  for (int q = 0; q < 2; q++) {
    uint32_t h;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(vals[q]));
    const float hf = __uint_as_float(h);
    hi[base + q] = hf;
    lo[base + q] = vals[q] - hf;
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// 2-D FP32 tensor map over a row-major rows x cols matrix (cols contiguous),
// box = 32 columns (128 bytes) x box_rows rows, 128-byte swizzle.
int make_map(Ctx *c, CUtensorMap *m, const float *base, int64_t rows, int64_t cols, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return fail(c, MOM_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(cols * sizeof(float))};
  cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(c, MOM_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return MOM_OK;
}

}  // namespace

// C (m x nc complex FP32, ldc) -= L (m x k, ldl) * U (k x nc, ldu) with the
// 3xTF32 tensor-core kernel.  m must be a multiple of 64, k of 16.
// work: >= (4 m k + 4 k nc) * 4 bytes of device scratch.  max_ctas > 0
// caps the persistent grid.  reuse_a: work already holds the expansion of
// this L (the previous call on the same stream had the same L, m and k).
// trans_l: L is given as its k x m transpose at L (ld ldl).
int tc_cgemm_update(Ctx *c, float2 *C, int64_t ldc, const float2 *L, int64_t ldl, const float2 *U, int64_t ldu, int m,
                    int nc, int k, float *work, int *err, int max_ctas, bool reuse_a, bool trans_l) {
  if (m <= 0 || nc <= 0 || k <= 0) return MOM_OK;
  if ((2 * m) % kBM != 0 || (2 * k) % kBK != 0) return fail(c, MOM_ERR_ARG, "tc_cgemm_update: unsupported shape");
  const int Mr = 2 * m, Kr = 2 * k;
  float *ahi = work, *alo = ahi + (size_t)Mr * Kr, *bhi = alo + (size_t)Mr * Kr, *blo = bhi + (size_t)nc * Kr;
  if (!reuse_a) {
    expand_a_tiled_kernel<<<dim3((unsigned)((k + 31) / 32), (unsigned)((m + 31) / 32)), dim3(32, 8), 0, c->stream>>>(
        L, ldl, m, k, ahi, alo, trans_l);
    c->launches++;
  }
  split_b_kernel<<<(unsigned)(((int64_t)k * nc + 255) / 256), 256, 0, c->stream>>>(U, ldu, k, nc, bhi, blo);
  c->launches++;
  CUtensorMap mAhi, mAlo, mBhi, mBlo;
  MOM_TRY(make_map(c, &mAhi, ahi, Mr, Kr, kBM));
  MOM_TRY(make_map(c, &mAlo, alo, Mr, Kr, kBM));
  MOM_TRY(make_map(c, &mBhi, bhi, nc, Kr, kBN));
  MOM_TRY(make_map(c, &mBlo, blo, nc, Kr, kBN));
  TcArgs ta;
  ta.C = reinterpret_cast<float *>(C);
  ta.ldc = 2 * ldc;
  ta.Mr = Mr;
  ta.Nc = nc;
  ta.Kr = Kr;
  ta.err = err;
  ta.spin = wait_polls(c, 1);
  const int ntiles = (Mr / kBM) * ((nc + kBN - 1) / kBN);
  // persistent: one CTA per SM, or fewer when another kernel (the look-ahead
  // panel) is to run beside it
  const int cap = (max_ctas > 0 && max_ctas < c->nsm) ? max_ctas : c->nsm;
  const int grid = ntiles < cap ? ntiles : cap;
  const size_t smem = (size_t)kStages * kStageBytes + 1024;
  {
    ProfScope ps(c, kProfTc);
    tc_gemm_kernel<<<grid, kTcThreads, smem, c->stream>>>(mAhi, mAlo, mBhi, mBlo, ta);
  }
  c->launches++;
  c->tc_flops += 6.0 * Mr * (double)nc * Kr;  // three TF32 passes, 2 FLOP per real MAC
  MOM_CUDA(c, cudaGetLastError());
  return MOM_OK;
}

int tc_init_kernels(Ctx *c) {
  MOM_CUDA(c, cudaFuncSetAttribute(tc_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   kStages * kStageBytes + 1024));
  return MOM_OK;
}

size_t tc_cgemm_work_bytes(int m, int nc, int k) { return ((size_t)8 * m * k + (size_t)4 * k * nc) * sizeof(float); }

}  // namespace mom

using namespace mom;
struct mom_ctx : public Ctx {};

// Diagnostics: C -= L U (host arrays, complex FP32 interleaved, column-major,
// leading dimensions m, k, m) through the tensor-core kernel above.
extern "C" int mom_gpu_selftest_cgemm(mom_ctx *c, int32_t m, int32_t nc, int32_t k, const float *L, const float *U,
                                      float *C) {
  if (!c || !L || !U || !C || m <= 0 || nc <= 0 || k <= 0) return MOM_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  MOM_CUDA(c, cudaSetDevice(c->device));
  const size_t bl = sizeof(float2) * (size_t)m * k, bu = sizeof(float2) * (size_t)k * nc,
               bc = sizeof(float2) * (size_t)m * nc, bw = tc_cgemm_work_bytes(m, nc, k);
  char *buf = nullptr;
  if (cudaMalloc(&buf, bl + bu + bc + bw + 4096) != cudaSuccess) {
    cudaGetLastError();
    return fail(c, MOM_ERR_ALLOC, "selftest allocation failed");
  }
  float2 *dL = (float2 *)buf, *dU = (float2 *)(buf + bl), *dC = (float2 *)(buf + bl + bu);
  float *dw = (float *)(buf + ((bl + bu + bc + 255) / 256) * 256);
  int rc = MOM_OK;
  cudaMemcpyAsync(dL, L, bl, cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(dU, U, bu, cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(dC, C, bc, cudaMemcpyHostToDevice, c->stream);
  cudaMemsetAsync(c->dinfo + 2, 0, sizeof(int), c->stream);
  rc = tc_cgemm_update(c, dC, m, dL, m, dU, k, m, nc, k, dw, c->dinfo + 2);
  int err = 0;
  if (rc == MOM_OK) {
    cudaMemcpyAsync(C, dC, bc, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(&err, c->dinfo + 2, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) rc = fail(c, MOM_ERR_CUDA, "selftest failed");
    else if (err) rc = fail(c, MOM_ERR_TIMEOUT, "tensor-core GEMM wait timed out");
  }
  cudaStreamSynchronize(c->stream);
  cudaFree(buf);
  return rc;
}
