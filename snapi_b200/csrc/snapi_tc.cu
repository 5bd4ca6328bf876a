// snapi_tc.cu -- batched Gram matrices G_p = M_p M_p^T of many small matrices M_p [16][K] on the
// 5th-generation tensor cores (tcgen05, sm_100a), FP32 accuracy from TF32 by a three-product split.
//
// Use: the LM normal equations.  Row i < npar of M_p is pixel p's scaled Jacobian row
// dS/dnode_i * scale_i * w_s * mask / I_c over the 4 x nlambda Stokes samples, row npar its scaled
// residual; G_p then holds J^T J (rows / columns < npar) and J^T r (column npar) -- the two
// products stokes_lm_fit forms at atmos_fit.cc:135-137.
//
// One CTA (4 warps) takes 8 matrices: A = [M_0; ...; M_7] is 128 x K, and one MMA chain computes
// D = A A^T (128 x 128, FP32 in TMEM); the 8 diagonal 16 x 16 blocks are the Gram matrices (the
// off-diagonal blocks are wasted work, negligible here).  Per stage of 64 K values all threads
// write the TF32 split hi = rna(A), lo = A - hi into shared memory in the canonical K-major layout
// without swizzle (8-row x 16-byte core matrices; SBO = 128 B between row groups, LBO = 2 KB between
// K chunks), one thread issues 8 K-steps x 3 tcgen05.mma (hi hi^T, hi lo^T, lo hi^T) and commits
// to an mbarrier; every wait on it is bounded.  Each warp then reads its 32 TMEM lanes
// (tcgen05.ld 32x32b.x32), which contain the diagonal blocks of matrices 2w and 2w + 1.
#include <cstdint>
#include <cstdio>

#include "snapi_internal.cuh"

namespace {

constexpr int kGramThreads = 128;
constexpr int kGramRows = 16;                 // rows of each small matrix
constexpr int kGramPerCta = 8;                // 8 x 16 = 128 = UMMA M = N
constexpr int kStageK = 64;                   // K values per shared-memory stage
constexpr int kTileBytes = 128 * kStageK * 4; // one operand split (hi or lo): 32 KB
constexpr uint32_t kCoreBytes = 128;          // 8 rows x 16 bytes
constexpr uint32_t kSBO = kCoreBytes;         // between 8-row groups
constexpr uint32_t kLBO = 16 * kCoreBytes;    // between 4-element K chunks (16 row groups)
constexpr long long kGramWaitLimit = 1LL << 24;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor: K-major, no swizzle, Blackwell version 1
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((kLBO >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((kSBO >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: D F32, A/B TF32, both K-major, M = N = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(acc));
}

__device__ __forceinline__ bool mbar_wait(uint32_t mb, uint32_t parity) {
  uint32_t done = 0;
  for (long long it = 0; it < kGramWaitLimit && !done; ++it)
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(mb), "r"(parity)
        : "memory");
  return done != 0;
}

__global__ void __launch_bounds__(kGramThreads, 1) k_gram_tf32(const float *M, int nmat, int K, float *G,
                                                                int *status) {
  extern __shared__ __align__(1024) unsigned char smem[];
  float *hi = reinterpret_cast<float *>(smem);
  float *lo = reinterpret_cast<float *>(smem + kTileBytes);
  uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + 2 * kTileBytes);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(smem + 2 * kTileBytes + 8);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kGramPerCta;
  const uint32_t mb = smem_addr(mbar);
  if (warp == 0) {  // 128 TMEM columns: D is 128 lanes x 128 FP32 columns
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                 "r"(128u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  const uint32_t hi_a = smem_addr(hi), lo_a = smem_addr(lo);
  const int nst = (K + kStageK - 1) / kStageK;
  bool ok = true;
  for (int s = 0; s < nst && ok; ++s) {
    for (int e = tid; e < 128 * kStageK; e += kGramThreads) {
      const int kk = e % kStageK, row = e / kStageK;
      const int mat = m0 + row / kGramRows, k = s * kStageK + kk;
      const float v = (mat < nmat && k < K) ? M[((size_t)mat * kGramRows + row % kGramRows) * K + k] : 0.0f;
      uint32_t h;
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(v));
      const float hv = __uint_as_float(h);
      const int off = ((kk >> 2) * 16 + (row >> 3)) * 32 + (row & 7) * 4 + (kk & 3);
      hi[off] = hv;
      lo[off] = v - hv;
    }
    // the tensor cores read shared memory through the async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int j = 0; j < kStageK / 8; ++j) {
        const uint32_t koff = (uint32_t)j * 2u * kLBO;  // 8 K values = 2 core-matrix chunks
        const uint64_t dh = umma_desc(hi_a + koff), dl = umma_desc(lo_a + koff);
        mma_tf32(tmem, dh, dh, (s > 0 || j > 0) ? 1u : 0u);
        mma_tf32(tmem, dh, dl, 1u);
        mma_tf32(tmem, dl, dh, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb)
                   : "memory");
    }
    ok = mbar_wait(mb, (uint32_t)(s & 1));
    ok = __syncthreads_and(ok) != 0;  // every thread takes the same decision
  }
  if (ok) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    uint32_t r[32];
    const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(32 * warp);
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    // lane l holds row 32w + l of D, columns 32w .. 32w + 31: matrix 2w + l / 16, its row l % 16
    const int mat = m0 + 2 * warp + (lane >> 4), i = lane & 15;
    if (mat < nmat) {
      float *g = G + ((size_t)mat * kGramRows + i) * kGramRows;
#pragma unroll
      for (int j = 0; j < 16; ++j) g[j] = __uint_as_float(lane < 16 ? r[j] : r[16 + j]);
    }
  } else if (tid == 0) {
    atomicExch(status, SNAPI_ETIMEOUT);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u));
}

constexpr size_t kGramSmem = 2 * kTileBytes + 16;

}  // namespace

namespace snapi {

cudaError_t launch_gram_tf32(const float *M, int nmat, int K, float *G, int *status, cudaStream_t st) {
  static bool attr[64] = {};  // the shared-memory opt-in, once per device
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64 || !attr[dev]) {
    e = cudaFuncSetAttribute(k_gram_tf32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGramSmem);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) attr[dev] = true;
  }
  if (nmat <= 0) return cudaSuccess;
  k_gram_tf32<<<(nmat + kGramPerCta - 1) / kGramPerCta, kGramThreads, kGramSmem, st>>>(M, nmat, K, G, status);
  return cudaGetLastError();
}

}  // namespace snapi

namespace {
// the bounded-wait status word of snapi_batched_gram (one per device that loads the library;
// calls that overlap on a GPU share it)
__device__ int g_gram_status;
}  // namespace

extern "C" {

int snapi_batched_gram(int nmat, int K, const float *M, float *G, void *stream) {
  if (nmat < 0 || K < 1 || (nmat > 0 && (!M || !G))) return SNAPI_EINVAL;
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  int *status = nullptr;
  if (cudaGetSymbolAddress(reinterpret_cast<void **>(&status), g_gram_status) != cudaSuccess) return SNAPI_ECUDA;
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), st);
  if (e == cudaSuccess) e = snapi::launch_gram_tf32(M, nmat, K, G, status, st);
  int word = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&word, status, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return SNAPI_ECUDA;
  return word ? word : SNAPI_OK;
}

}  // extern "C"
