// path_gram.cu — G = X Y^T over the path dimension on the tensor cores.
//
// G[i][j] = sum_p X[i][p] Y[j][p] for i < m <= 128, j < n <= 128, where X
// and Y are row-major [rows][paths] with paths contiguous — the layout every
// per-path array of this library has.  It is the contraction behind the
// Longstaff–Schwartz normal equations (X = basis functions and target,
// gold/LS_regression.h:431-530: E[phi phi^T], E[phi y]) and behind the
// adjoint's pseudo-root sensitivities (sums over paths of outer products of
// per-path vectors).
//
// Precision: split TF32 ("3xTF32").  Each value x is split into
// hi = tf32(x) (round to nearest) and lo = x - hi; the tensor cores form
// hi*hi + hi*lo + lo*hi with FP32 accumulation in tensor memory, which
// recovers FP32-level products.  The tensor cores' FP32 accumulation does
// not round to nearest: measured here, a chain of 512 K-steps over
// same-sign products drifted by 4e-5 relative, about 2^-23.5 per step.  So
// the accumulator covers kDrain paths only (16 K-steps, a drift of about
// 1e-6 at most): after each such group every thread adds its row of the
// accumulator into FP32 registers and the next group starts from zero.
// Each CTA covers kChunk paths; the per-CTA partials are summed in FP64
// with Kahan compensation in a fixed order.
//
// Structure (one CTA of 128 threads per chunk):
//   * tensor memory for the 128 x N accumulator is allocated by warp 0;
//   * all threads stage 32-path slices of X and Y into shared memory in
//     the canonical K-major no-swizzle layout (8-row x 16-byte core
//     matrices; leading-dimension offset 128 B between the two 16-byte K
//     halves of an 8-element K step, stride offset 1 KB between row groups),
//     already split into hi and lo parts, double-buffered;
//   * one thread issues tcgen05.mma (kind::tf32, M = 128, N = 16..128,
//     K = 8 per instruction) and commits each stage to an mbarrier;
//   * every kDrain paths the threads read the accumulator with tcgen05.ld
//     (lane = row) into registers; the last read gives the CTA's partial.
// Every wait on an mbarrier is bounded (one second of elapsed time); on
// timeout the CTA sets the lowest bit (value 1) of *status, skips the
// remaining work, lets the tensor cores finish what it has issued (one more
// bounded wait) and still frees its tensor memory.
#include "lmm_common.cuh"

#include <algorithm>
#include <cstdint>

using namespace lmm;

namespace {

constexpr int kThreads = 128;
constexpr int kKT = 32;                 // paths per stage
constexpr int kKC = kKT / 4;            // 16-byte K chunks per row
constexpr int kChunk = 2048;            // paths per CTA
constexpr int kDrain = 128;             // paths per accumulation group
constexpr int kTilesPerDrain = kDrain / kKT;
constexpr uint32_t kSpinLimit = 1u << 30;  // backstop of the timed waits
constexpr uint64_t kWaitNs = 1000000000ull;  // bound of one mbarrier wait: 1 s

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Canonical K-major, no-swizzle shared-memory matrix descriptor.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo,
                                              uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  return d;                // base offset 0, no swizzle
}

// Instruction descriptor: D f32, A/B tf32, both K-major, M x N.
__host__ __device__ constexpr uint32_t make_idesc(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc,
                                         uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u),
      "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

// Bounded wait for the given phase parity; returns false when it runs out.
// The bound is elapsed time (kWaitNs on the %globaltimer nanosecond clock,
// sampled every 64 polls), with a poll count as a backstop, so a wait ends
// after about a second however long each try_wait blocks.
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          uint64_t limit_ns = kWaitNs) {
  const uint32_t a = smem_u32(bar);
  const uint64_t t0 = global_ns();
  for (uint32_t i = 0; i < kSpinLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((i & 63u) == 63u && global_ns() - t0 > limit_ns) return false;
  }
  return false;
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
        "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
        "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}

}  // namespace

// One CTA: paths [blockIdx.x*kChunk, +kChunk).  NP = n rounded up to 16.
template <int NP>
__global__ void __launch_bounds__(kThreads, 1)
    path_gram_kernel(int m, int n, int paths, const float* __restrict__ X,
                     int ldx, const float* __restrict__ Y, int ldy, int same,
                     float* __restrict__ part, int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ __align__(8) uint64_t bar_drain;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const size_t a_bytes = 128 * kKT * sizeof(float);              // one A tile
  const size_t b_bytes = same ? 0 : (size_t)NP * kKT * sizeof(float);
  const size_t stage_bytes = 2 * a_bytes + 2 * b_bytes;
  unsigned char* base = smem_raw;
  // zero both stages (rows beyond m / n stay zero)
  for (size_t i = tid * 16; i < 2 * stage_bytes; i += kThreads * 16)
    *reinterpret_cast<uint4*>(base + i) = make_uint4(0, 0, 0, 0);
  constexpr uint32_t ncols = NP <= 32 ? 32 : NP <= 64 ? 64 : 128;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tmem_slot;
  const uint32_t idesc = make_idesc(128, NP);
  const int p_begin = blockIdx.x * kChunk;
  const int p_end = min(paths, p_begin + kChunk);
  const int ntiles = (p_end - p_begin + kKT - 1) / kKT;
  float acc[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) acc[j] = 0.0f;

  for (int t = 0; t < ntiles; ++t) {
    const int st = t & 1;
    if (t >= 2) {
      if (!mbar_wait(&bar[st], (uint32_t)(((t >> 1) - 1) & 1))) {
        if (tid == 0) atomicOr(status, 1);
        abort_flag = 1;
      }
    }
    __syncthreads();
    if (abort_flag) break;
    unsigned char* sbase = base + st * stage_bytes;
    float* Ahi = reinterpret_cast<float*>(sbase);
    float* Alo = reinterpret_cast<float*>(sbase + a_bytes);
    float* Bhi = same ? Ahi : reinterpret_cast<float*>(sbase + 2 * a_bytes);
    float* Blo = same ? Alo : reinterpret_cast<float*>(sbase + 2 * a_bytes + b_bytes);
    const int p0 = p_begin + t * kKT;
    // stage X rows (and Y rows): item = (row, kc), kc fastest
    const int rows_total = same ? m : m + n;
    for (int it = tid; it < rows_total * kKC; it += kThreads) {
      const int rr = it / kKC, kc = it - rr * kKC;
      const bool isx = rr < m;
      const int r = isx ? rr : rr - m;
      const float* src = isx ? X + (size_t)r * ldx : Y + (size_t)r * ldy;
      const int p = p0 + 4 * kc;
      float4 v;
      if (p + 3 < p_end) {
        v = __ldg(reinterpret_cast<const float4*>(src + p));
      } else {
        v.x = p < p_end ? src[p] : 0.0f;
        v.y = p + 1 < p_end ? src[p + 1] : 0.0f;
        v.z = p + 2 < p_end ? src[p + 2] : 0.0f;
        v.w = p + 3 < p_end ? src[p + 3] : 0.0f;
      }
      uint4 hi, lo;
      hi.x = tf32_rna(v.x);
      hi.y = tf32_rna(v.y);
      hi.z = tf32_rna(v.z);
      hi.w = tf32_rna(v.w);
      lo.x = __float_as_uint(v.x - __uint_as_float(hi.x));
      lo.y = __float_as_uint(v.y - __uint_as_float(hi.y));
      lo.z = __float_as_uint(v.z - __uint_as_float(hi.z));
      lo.w = __float_as_uint(v.w - __uint_as_float(hi.w));
      const size_t off = ((size_t)((r >> 3) * kKC + kc) * 128 + (r & 7) * 16) / sizeof(float);
      float* dh = isx ? Ahi : Bhi;
      float* dl = isx ? Alo : Blo;
      *reinterpret_cast<uint4*>(dh + off) = hi;
      *reinterpret_cast<uint4*>(dl + off) = lo;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    const bool group_start = (t % kTilesPerDrain) == 0;
    if (tid == 0) {
      fence_after_sync();
      const uint32_t ah = smem_u32(Ahi), al = smem_u32(Alo);
      const uint32_t bh = smem_u32(Bhi), bl = smem_u32(Blo);
#pragma unroll
      for (int k0 = 0; k0 < kKT / 8; ++k0) {
        const uint32_t koff = k0 * 2 * 128;
        const uint64_t dAh = make_desc(ah + koff, 128, kKC * 128);
        const uint64_t dAl = make_desc(al + koff, 128, kKC * 128);
        const uint64_t dBh = make_desc(bh + koff, 128, kKC * 128);
        const uint64_t dBl = make_desc(bl + koff, 128, kKC * 128);
        mma_tf32(tmem, dAh, dBh, idesc, (group_start && k0 == 0) ? 0u : 1u);
        mma_tf32(tmem, dAh, dBl, idesc, 1u);
        mma_tf32(tmem, dAl, dBh, idesc, 1u);
      }
      mma_commit(&bar[st]);
    }
    // end of a group: wait for its MMAs, add the accumulator into registers
    if ((t % kTilesPerDrain) == kTilesPerDrain - 1 || t == ntiles - 1) {
      if (!mbar_wait(&bar[st], (uint32_t)((t >> 1) & 1))) {
        if (tid == 0) atomicOr(status, 1);
        abort_flag = 1;
      }
      __syncthreads();
      if (abort_flag) break;
      fence_after_sync();
#pragma unroll
      for (int c0 = 0; c0 < NP; c0 += 16) {
        uint32_t v[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[c0 + j] += __uint_as_float(v[j]);
      }
      fence_before_sync();
    }
  }
  if (abort_flag) {
    // a wait ran out: let every MMA this CTA issued finish (bounded) before
    // its tensor memory is freed
    if (tid == 0) {
      mbar_init(&bar_drain, 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      mma_commit(&bar_drain);
      if (!mbar_wait(&bar_drain, 0u)) atomicOr(status, 2);
    }
  } else {
    const int row = warp * 32 + lane;
    if (row < m) {
      float* dst = part + ((size_t)blockIdx.x * m + row) * n;
#pragma unroll
      for (int j = 0; j < NP; ++j)
        if (j < n) dst[j] = acc[j];
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols)
                 : "memory");
}

// FP64 Kahan sum of the per-CTA partials, fixed order, times `scale`.
__global__ void path_gram_reduce_kernel(int m, int n, int nblocks,
                                        const float* __restrict__ part,
                                        double scale, double* __restrict__ G,
                                        int ldg) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= m * n) return;
  const int i = idx / n, j = idx - i * n;
  double s = 0.0, c = 0.0;
  for (int b = 0; b < nblocks; ++b) {
    const double y = (double)part[((size_t)b * m + i) * n + j] - c;
    const double t = s + y;
    c = (t - s) - y;
    s = t;
  }
  G[(size_t)i * ldg + j] = s * scale;
}

namespace lmm {
int path_gram_blocks(int paths) { return (paths + kChunk - 1) / kChunk; }

size_t path_gram_workspace(int m, int n, int paths) {
  return (size_t)path_gram_blocks(paths) * m * n * sizeof(float);
}

size_t path_gram_smem(int n, int same) {
  const int NP = ((n + 15) / 16) * 16;
  const size_t a = 128 * kKT * sizeof(float);
  const size_t b = same ? 0 : (size_t)NP * kKT * sizeof(float);
  return 2 * (2 * a + 2 * b);
}

int path_gram_launch(int m, int n, int paths, const float* X, int ldx,
                     const float* Y, int ldy, double scale, double* G, int ldg,
                     float* part, int* status, cudaStream_t s) {
  const int same = (X == Y && ldx == ldy && m == n) ? 1 : 0;
  const int NP = ((n + 15) / 16) * 16;
  const int nb = path_gram_blocks(paths);
  const size_t smem = path_gram_smem(n, same);
  auto go = [&](auto kern) -> int {
    int st = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem),
                        "lmm_path_gram: smem attribute");
    if (st) return st;
    kern<<<nb, kThreads, smem, s>>>(m, n, paths, X, ldx, Y, ldy, same, part, status);
    return check_launch("path_gram_kernel");
  };
  int st;
  switch (NP) {
    case 16: st = go(path_gram_kernel<16>); break;
    case 32: st = go(path_gram_kernel<32>); break;
    case 48: st = go(path_gram_kernel<48>); break;
    case 64: st = go(path_gram_kernel<64>); break;
    case 80: st = go(path_gram_kernel<80>); break;
    case 96: st = go(path_gram_kernel<96>); break;
    case 112: st = go(path_gram_kernel<112>); break;
    default: st = go(path_gram_kernel<128>); break;
  }
  if (st) return st;
  path_gram_reduce_kernel<<<div_up(m * n, 128), 128, 0, s>>>(m, n, nb, part, scale, G, ldg);
  return check_launch("path_gram_reduce_kernel");
}
}  // namespace lmm

extern "C" size_t lmm_path_gram_workspace_bytes(int m, int n, int paths) {
  if (m < 1 || n < 1 || paths < 1) return 0;
  return (size_t)lmm::path_gram_blocks(paths) * m * n * sizeof(float);
}

extern "C" int lmm_path_gram(int m, int n, int paths, const float* d_X, int ldx,
                             const float* d_Y, int ldy, double scale, double* d_G,
                             void* d_workspace, size_t workspace_bytes,
                             int* d_status, lmm_stream_t stream) {
  LMM_REQUIRE(m >= 1 && m <= 128 && n >= 1 && n <= 128 && paths >= 1,
              "lmm_path_gram: need 1 <= m, n <= 128 and paths >= 1");
  LMM_REQUIRE(d_X && d_Y && d_G && d_workspace && d_status, "lmm_path_gram: null pointer");
  LMM_REQUIRE(ldx >= paths && ldy >= paths && ldx % 4 == 0 && ldy % 4 == 0,
              "lmm_path_gram: leading dimensions must be >= paths and multiples of 4");
  LMM_REQUIRE(reinterpret_cast<uintptr_t>(d_X) % 16 == 0 &&
                  reinterpret_cast<uintptr_t>(d_Y) % 16 == 0,
              "lmm_path_gram: X and Y must be 16-byte aligned");
  LMM_REQUIRE(workspace_bytes >= lmm_path_gram_workspace_bytes(m, n, paths),
              "lmm_path_gram: workspace too small");
  return lmm::path_gram_launch(m, n, paths, d_X, ldx, d_Y, ldy, scale, d_G, n,
                               (float*)d_workspace, d_status, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// The reference's outer-product reductions (reduceOuterProduct_gpu and
// reduceOuterProductSymmetric_gpu, outerProduct_gpu.cu:205-700), which make
// one pass over the data per matrix entry, as batches of the tensor-core
// contraction above: answer[r][c] = sum_p in1[r][p] in2[c][p] (FP32
// output, FP64 running sum over the batches).  The workspace holds the
// FP64 running sum, one batch's FP64 result and the per-CTA partials of a
// batch; a batch takes as many paths as the partials allow, so any
// workspace of at least lmm_outer_product_workspace_bytes(rows, cols, 1)
// works, a larger one in fewer launches.
// ---------------------------------------------------------------------------
namespace {

__global__ void outer_accumulate_kernel(int mn, const double* __restrict__ batch,
                                        double* __restrict__ acc, int first) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < mn) acc[i] = first ? batch[i] : acc[i] + batch[i];
}

__global__ void outer_store_kernel(int mn, const double* __restrict__ acc,
                                   float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < mn) out[i] = (float)acc[i];
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

extern "C" size_t lmm_outer_product_workspace_bytes(int rows, int cols, int paths) {
  if (rows < 1 || cols < 1 || paths < 1) return 0;
  const size_t mn = (size_t)rows * cols;
  return 2 * align256(mn * sizeof(double)) + align256(sizeof(int)) +
         lmm_path_gram_workspace_bytes(rows, cols, paths);
}

extern "C" int lmm_outer_product(int paths, int rows, int cols, const float* d_in1,
                                 const float* d_in2, float* d_answer, void* d_workspace,
                                 size_t workspace_bytes, int* d_status, lmm_stream_t stream) {
  LMM_REQUIRE(paths >= 1 && rows >= 1 && rows <= 128 && cols >= 1 && cols <= 128,
              "lmm_outer_product: need 1 <= rows, cols <= 128 and paths >= 1");
  LMM_REQUIRE(paths % 4 == 0, "lmm_outer_product: paths (the row stride) must be a multiple of 4");
  LMM_REQUIRE(d_in1 && d_in2 && d_answer && d_workspace && d_status,
              "lmm_outer_product: null pointer");
  const size_t mn = (size_t)rows * cols;
  const size_t fixed = 2 * align256(mn * sizeof(double)) + align256(sizeof(int));
  LMM_REQUIRE(workspace_bytes >= lmm_outer_product_workspace_bytes(rows, cols, 1),
              "lmm_outer_product: workspace %zu < %zu", workspace_bytes,
              lmm_outer_product_workspace_bytes(rows, cols, 1));
  char* base = (char*)d_workspace;
  double* acc = (double*)base;
  double* batch = (double*)(base + align256(mn * sizeof(double)));
  void* part = base + fixed;
  const size_t part_bytes = workspace_bytes - fixed;
  const long long chunks = (long long)(part_bytes / (mn * sizeof(float)));
  const long long per_batch = std::min<long long>((long long)paths, chunks * kChunk);
  cudaStream_t s = (cudaStream_t)stream;
  int st = check_cuda(cudaMemsetAsync(d_status, 0, sizeof(int), s), "lmm_outer_product: status");
  if (st) return st;
  int first = 1;
  for (long long p0 = 0; p0 < paths; p0 += per_batch, first = 0) {
    const int np = (int)std::min<long long>(per_batch, paths - p0);
    st = lmm_path_gram(rows, cols, np, d_in1 + p0, paths, d_in2 + p0, paths, 1.0, batch, part,
                       part_bytes, d_status, stream);
    if (st) return st;
    outer_accumulate_kernel<<<div_up((long long)mn, 256), 256, 0, s>>>((int)mn, batch, acc,
                                                                       first);
    st = check_launch("lmm_outer_product: accumulate");
    if (st) return st;
  }
  outer_store_kernel<<<div_up((long long)mn, 256), 256, 0, s>>>((int)mn, acc, d_answer);
  return check_launch("lmm_outer_product: store");
}

// ---------------------------------------------------------------------------
// Self-test of the bounded-wait path of the tensor-core kernels: one CTA
// allocates tensor memory, waits on an mbarrier that nothing will signal
// (nothing else is in flight), reports the timeout in *status (value 1)
// and frees the tensor memory, leaving the context usable.
// ---------------------------------------------------------------------------
namespace {
__global__ void __launch_bounds__(32, 1)
    tensor_wait_selftest_kernel(int* __restrict__ status, unsigned long long limit_ns) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(&tmem_slot)),
               "r"(32u)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (threadIdx.x == 0 && !mbar_wait(&bar, 0u, (uint64_t)limit_ns)) atomicOr(status, 1);
  fence_before_sync();
  __syncthreads();
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_slot), "r"(32u)
               : "memory");
}
}  // namespace

extern "C" int lmm_tensor_wait_selftest(unsigned long long limit_ns, int* d_status,
                                        lmm_stream_t stream) {
  LMM_REQUIRE(d_status, "lmm_tensor_wait_selftest: null status");
  LMM_REQUIRE(limit_ns <= kWaitNs, "lmm_tensor_wait_selftest: limit above one second");
  tensor_wait_selftest_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(d_status, limit_ns);
  return check_launch("lmm_tensor_wait_selftest");
}
