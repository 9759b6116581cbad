// tc_evolve.cuh — the fused evolution with its per-step contractions on the
// tensor cores (included by pipeline.cu after fused_kernels.cuh).
//
// Per step s the spot-measure drift of every alive rate is a lower-triangular
// matrix product: mu_r = sum_{j<=r} C_rj g_j with C = A_s A_s^T (the factor
// form of the reference, e_f(r) = sum_{j<=r} g_j A_jf and mu_r =
// sum_f A_rf e_f(r), LMM_evolver_all.cu:690-741, regrouped), and the
// correlated increment is dW_r = sum_f A_rf z_f.  For a CTA of 128 paths
// these are GEMMs with M = 128 paths:
//   D1 = [g | z] [C | A]^T          (mu + dW of the start rates)
//   D2 = (gp - g) C^T               (mu(predicted) - mu(start))
// so the predictor-corrector step is
//   lp = lf + D1 + fixed,  gp = G(lp),  ln = lp + D2 / 2
// (identical to lf + (mu + mu_p)/2 + dW + fixed).  Each MMA runs in split
// FP16: every operand x is stored as hi = fp16(x s) and lo = fp16(x s - hi)
// with a power-of-two scale s, and the tensor cores form hi*hi + hi*lo +
// lo*hi in FP32 (about 22 significant bits); the accumulators live in tensor
// memory.  The B operand [C | A] of every step (and its scales) is built
// once per call by tc_b_image_kernel in the exact shared-memory image and
// copied per step with one bulk copy.  The log-rates of the CTA's paths live
// in tensor memory too (one lane per path), which leaves shared memory for
// the operands and allows two CTAs per SM.  Waits on mbarriers are bounded
// (one second of elapsed time); a timeout sets the lowest bit (value 1) of
// the library's device error word, the CTA stops issuing work, lets the
// tensor cores drain (bounded) and still frees its tensor memory.
#pragma once
#include "fused_kernels.cuh"

#include <cuda_fp16.h>

namespace lmm {

namespace tc {

constexpr int kThreads = 128;
constexpr uint32_t kSpinLimit = 1u << 30;  // backstop of the timed waits
constexpr uint64_t kWaitNs = 1000000000ull;  // bound of one mbarrier wait: 1 s
// operand scales (powers of two): g in (0, 1), C ~ var * dt, A ~ vol * sqrt(dt)
constexpr float kSG = 16.0f;     // g and gp
constexpr float kSC = 64.0f;     // C
constexpr float kSZ = 1.0f;      // z
constexpr float kSA = kSG * kSC / kSZ;  // A, so that z A and g C share one scale
constexpr float kSD = 1024.0f;   // gp - g
constexpr float kInvD1 = 1.0f / (kSG * kSC);
constexpr float kInvD2 = 1.0f / (kSD * kSC);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// K-major, no-swizzle shared-memory descriptor: core matrices of 8 rows x
// 16 bytes, LBO between the two 16-byte K chunks of one MMA, SBO between
// row groups.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// kind::f16 instruction descriptor: D f32, A/B f16, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N) {
  return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t a, uint64_t b,
                                        uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
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

// Bulk copy global -> shared (contiguous, 16-byte aligned, multiple of 16
// bytes) completing on an mbarrier that expects `bytes`.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Byte offset of element (row, k) in a K-major no-swizzle image with KC8
// 16-byte chunks (8 fp16) per row group.
__host__ __device__ __forceinline__ uint32_t img_off(int row, int k, int KC8) {
  return (uint32_t)(((row >> 3) * KC8 + (k >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

}  // namespace tc

// Geometry of the tensor-core form for n rates and F factors.
struct TcGeom {
  int NB;    // rates rounded up to 16: B rows and drift K columns
  int KT;    // drift columns + 16 factor columns
  int KC8;   // 16-byte chunks per row of an image (KT / 8)
  int b_bytes;   // one step's B image (hi then lo)
  int a_bytes;   // the A tile (hi then lo), 128 rows
  int tmem_cols; // D1 | D2 | log-rates, rounded up to a power of two
  __host__ __device__ static TcGeom make(int n) {
    TcGeom g;
    g.NB = (n + 15) & ~15;
    g.KT = g.NB + 16;
    g.KC8 = g.KT / 8;
    g.b_bytes = 2 * g.NB * g.KT * 2;
    g.a_bytes = 2 * 128 * g.KT * 2;
    int c = 32;
    while (c < 3 * g.NB) c <<= 1;
    g.tmem_cols = c;
    return g;
  }
};

// B images of every step: rows r < NB (rates), columns k < KT; k < NB is
// C_s[r][k] kSC for s <= k <= r < n (zero elsewhere), k = NB + f is
// A_s[r][f] kSA for f < F and s <= r < n.  hi image then lo image, each in
// the K-major core-matrix layout of the shared-memory operand.  Grid
// (NB, steps), block KT threads.
__global__ void tc_b_image_kernel(int n, int F, const float* __restrict__ A,
                                  unsigned char* __restrict__ img) {
  const TcGeom G = TcGeom::make(n);
  const int r = blockIdx.x, s = blockIdx.y, k = threadIdx.x;
  if (k >= G.KT) return;
  const float* As = A + (size_t)s * n * F;
  double v = 0.0;
  if (r >= s && r < n) {
    if (k < G.NB) {
      if (k >= s && k <= r) {
        for (int f = 0; f < F; ++f) v += (double)As[r * F + f] * (double)As[k * F + f];
        v *= tc::kSC;
      }
    } else if (k - G.NB < F) {
      v = (double)As[r * F + (k - G.NB)] * tc::kSA;
    }
  }
  const __half hi = __double2half(v);
  const __half lo = __double2half(v - (double)__half2float(hi));
  unsigned char* base = img + (size_t)s * G.b_bytes;
  const uint32_t off = tc::img_off(r, k, G.KC8);
  *reinterpret_cast<__half*>(base + off) = hi;
  *reinterpret_cast<__half*>(base + G.b_bytes / 2 + off) = lo;
}


// G(x) = tau e^x / (c0 + tau e^x), the spot drift factor of a displaced rate
__device__ __forceinline__ float drift_factor(float lf, float tau, float c0) {
  const float Fr = exp_ftz(lf) * tau;
  return Fr * rcp_ftz(c0 + Fr);
}

namespace tc {

__device__ __forceinline__ void tmem_ld16_nw(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_st16_nw(uint32_t taddr, const float* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
          taddr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
      "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
      "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
      "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
      "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
      "r"(__float_as_uint(v[15]))
      : "memory");
}

__device__ __forceinline__ void tmem_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// 16 values x * scale split into fp16 hi and lo (packed conversions), stored
// as two 16-byte chunks each at hi + off and lo + off (next chunk +128 B).
__device__ __forceinline__ void split_store16(unsigned char* hi, unsigned char* lo,
                                              uint32_t off, const float* x, float scale) {
  uint32_t h[8], l[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const float a = x[2 * i] * scale, b = x[2 * i + 1] * scale;
    const __half2 hh = __floats2half2_rn(a, b);
    const float2 back = __half22float2(hh);
    const __half2 ll = __floats2half2_rn(a - back.x, b - back.y);
    h[i] = *reinterpret_cast<const uint32_t*>(&hh);
    l[i] = *reinterpret_cast<const uint32_t*>(&ll);
  }
  *reinterpret_cast<uint4*>(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<uint4*>(hi + off + 128) = make_uint4(h[4], h[5], h[6], h[7]);
  *reinterpret_cast<uint4*>(lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
  *reinterpret_cast<uint4*>(lo + off + 128) = make_uint4(l[4], l[5], l[6], l[7]);
}

}  // namespace tc

// Fused evolution with tensor-core contractions; MODE kModeInputs or
// kModeRule as fused_evolve_kernel (same outputs, same product epilogue).
// One CTA of 128 threads per 128 paths; thread = path = tensor-memory lane.
// Tensor memory per lane: D (the MMA accumulator, NB columns), LF (the
// log-rates, then the predicted log-rates within a step) and G (the drift
// factor of the start rates, formed at the end of the previous step from
// the same exp and reciprocal as the discount factor 1 / (1 + tau f)).
template <int MODE>
__global__ void __launch_bounds__(tc::kThreads, 2)
    tc_evolve_kernel(int paths, const float* __restrict__ Z, int F,
                     const unsigned char* __restrict__ bimg,
                     const float* __restrict__ fixed,
                     const __grid_constant__ ModelConst mc,
                     const __grid_constant__ ProductConst pc,
                     const __grid_constant__ RuleConst rc,
                     const LsRuleView rule, int total, int col0,
                     float* __restrict__ o_vars, float* __restrict__ o_ex,
                     float* __restrict__ o_cf, float* __restrict__ o_num,
                     float* __restrict__ o_payoff, unsigned int* __restrict__ errors) {
  using namespace tc;
  const int n = mc.n;
  const TcGeom G = TcGeom::make(n);
  const int tid = threadIdx.x, warp = tid >> 5;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* Ahi = smem;                         // [128][KT] fp16 image
  unsigned char* Alo = Ahi + G.a_bytes / 2;
  unsigned char* Bimg = Alo + G.a_bytes / 2;         // hi image then lo image
  float* fx = reinterpret_cast<float*>(Bimg + G.b_bytes);  // [NB]
  __shared__ __align__(8) uint64_t bar_b, bar_m;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_s;
  if (tid == 0) {
    mbar_init(&bar_b, 1);
    mbar_init(&bar_m, 1);
    abort_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_slot)),
                 "r"((uint32_t)G.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = tmem_slot;
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
  const uint32_t tD = lane_base, tLF = lane_base + G.NB, tG = lane_base + 2 * G.NB;
  // parities of the copy and the MMA group thread 0 has in flight (-1: none)
  int cp_par = -1, mm_par = -1;
  if (tid == 0) {
    bulk_load(Bimg, bimg, (uint32_t)G.b_bytes, &bar_b);
    cp_par = 0;
  }
  const int p = blockIdx.x * kThreads + tid;
  const bool valid = p < paths;
  // initial log-rates and drift factors into tensor memory
  for (int cb = 0; cb < G.NB; cb += 16) {
    float v[16], g[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int r = cb + j;
      v[j] = r < n ? mc.logf0[r] : 0.0f;
      g[j] = r < n ? drift_factor(v[j], mc.tau[r], mc.c0[r]) : 0.0f;
    }
    tmem_st16_nw(tLF + cb, v);
    tmem_st16_nw(tG + cb, g);
  }
  tmem_wait_st();
  float N = 1.0f, f_first = 0.0f, cf_acc = 0.0f, N_bucket = 1.0f;
  int bucket = -1;
  double payoff = 0.0;
  float tarn_paid = 0.0f;
  bool tarn_over = false;
  bool done = !valid;
  const int col = col0 + p;
  const uint32_t a_hi = smem_u32(Ahi), a_lo = smem_u32(Alo);
  const uint32_t b_hi = smem_u32(Bimg), b_lo = b_hi + G.b_bytes / 2;
  const uint32_t sbo = (uint32_t)G.KC8 * 128u;
  // this thread's row of the A tile: byte offset of column k is rowoff + (k / 8) * 128
  const uint32_t rowoff = (uint32_t)(tid >> 3) * sbo + (uint32_t)(tid & 7) * 16u;
  for (int s = 0; s < n; ++s) {
    const int rb = s & ~15;
    const int N_mma = G.NB - rb;
    __syncthreads();  // the previous step's readers of fx are done
    for (int i = tid; i < G.NB; i += kThreads) fx[i] = i < n ? __ldg(fixed + (size_t)s * n + i) : 0.0f;
    // ---- P1: g of the start rates and z into the A tile ----
    for (int cb = rb; cb < G.NB; cb += 16) {
      float g[16];
      tmem_ld16_nw(tG + cb, g);
      tmem_wait_ld();
#pragma unroll
      for (int j = 0; j < 16; ++j)
        if (cb + j < s || cb + j >= n) g[j] = 0.0f;
      split_store16(Ahi, Alo, rowoff + (uint32_t)(cb >> 3) * 128u, g, kSG);
    }
    {
      float z[16];
#pragma unroll
      for (int f = 0; f < 16; ++f)
        z[f] = (valid && f < F) ? __ldg(Z + ((size_t)s * F + f) * paths + p) : 0.0f;
      split_store16(Ahi, Alo, rowoff + (uint32_t)(G.NB >> 3) * 128u, z, kSZ);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    fence_before();
    __syncthreads();
    fence_after();
    // ---- P2: D = [g | z] [C | A]^T ----
    if (tid == 0) {
      if (mbar_wait(&bar_b, (uint32_t)(s & 1)))
        cp_par = -1;
      else
        abort_s = 1;
      if (!abort_s) {
        const uint32_t idesc = idesc_f16(128, N_mma);
        const uint32_t brow = (uint32_t)(rb >> 3) * sbo;
        for (int ks = rb >> 4; ks < G.KT >> 4; ++ks) {
          const uint32_t ko = (uint32_t)ks * 256u;
          const uint64_t dAh = make_desc(a_hi + ko, 128, sbo), dAl = make_desc(a_lo + ko, 128, sbo);
          const uint64_t dBh = make_desc(b_hi + brow + ko, 128, sbo);
          const uint64_t dBl = make_desc(b_lo + brow + ko, 128, sbo);
          mma_f16(tmem, dAh, dBh, idesc, ks > (rb >> 4) ? 1u : 0u);
          mma_f16(tmem, dAh, dBl, idesc, 1u);
          mma_f16(tmem, dAl, dBh, idesc, 1u);
        }
        mma_commit(&bar_m);
        mm_par = 0;
      }
    }
    __syncthreads();
    if (abort_s) break;
    if (mbar_wait(&bar_m, 0u))
      mm_par = -1;
    else
      abort_s = 1;
    __syncthreads();
    if (abort_s) break;
    fence_after();
    // ---- P3: predicted log-rates (kept in LF), gp - g into the A tile ----
    for (int cb = rb; cb < G.NB; cb += 16) {
      float lf[16], d[16], g[16];
      tmem_ld16_nw(tLF + cb, lf);
      tmem_ld16_nw(tD + (cb - rb), d);
      tmem_ld16_nw(tG + cb, g);
      tmem_wait_ld();
      float dg[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int r = cb + j;
        dg[j] = 0.0f;
        if (r >= s && r < n) {
          const float lp = lf[j] + (d[j] * kInvD1 + fx[r]);
          lf[j] = lp;
          dg[j] = drift_factor(lp, mc.tau[r], mc.c0[r]) - g[j];
        }
      }
      split_store16(Ahi, Alo, rowoff + (uint32_t)(cb >> 3) * 128u, dg, kSD);
      tmem_st16_nw(tLF + cb, lf);
    }
    tmem_wait_st();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    fence_before();
    __syncthreads();
    fence_after();
    // ---- P4: D = (gp - g) C^T ----
    if (tid == 0) {
      const uint32_t idesc = idesc_f16(128, N_mma);
      const uint32_t brow = (uint32_t)(rb >> 3) * sbo;
      for (int ks = rb >> 4; ks < G.NB >> 4; ++ks) {
        const uint32_t ko = (uint32_t)ks * 256u;
        const uint64_t dAh = make_desc(a_hi + ko, 128, sbo), dAl = make_desc(a_lo + ko, 128, sbo);
        const uint64_t dBh = make_desc(b_hi + brow + ko, 128, sbo);
        const uint64_t dBl = make_desc(b_lo + brow + ko, 128, sbo);
        mma_f16(tmem, dAh, dBh, idesc, ks > (rb >> 4) ? 1u : 0u);
        mma_f16(tmem, dAh, dBl, idesc, 1u);
        mma_f16(tmem, dAl, dBh, idesc, 1u);
      }
      mma_commit(&bar_m);
      mm_par = 1;
    }
    if (mbar_wait(&bar_m, 1u))
      mm_par = -1;
    else
      abort_s = 1;
    __syncthreads();
    if (abort_s) break;
    fence_after();
    // the B image of the next step can come in while this one finishes
    if (tid == 0 && s + 1 < n) {
      bulk_load(Bimg, bimg + (size_t)(s + 1) * G.b_bytes, (uint32_t)G.b_bytes, &bar_b);
      cp_par = (s + 1) & 1;
    }
    // ---- P5: corrected rates, the next drift factors, the curve at T_s ----
    if (s > 0) N = N * (1.0f + mc.tau[s - 1] * f_first);
    const int e = pc.ex_index[s];
    const bool curve = (e >= 0) || (pc.kind != LMM_PRODUCT_SWAPTION);
    float Prun = 1.0f, ann = 0.0f, P1 = 1.0f;
    for (int cb = rb; cb < G.NB; cb += 16) {
      float lp[16], d[16], g[16];
      tmem_ld16_nw(tLF + cb, lp);
      tmem_ld16_nw(tD + (cb - rb), d);
      tmem_ld16_nw(tG + cb, g);
      tmem_wait_ld();
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int r = cb + j;
        if (r >= s && r < n) {
          const float ln = fminf(lp[j] + 0.5f * (d[j] * kInvD2), mc.cutoff);
          lp[j] = ln;
          // one exp and one reciprocal give f, 1 / (1 + tau f) = 1 / (c0 + tau F)
          // and the drift factor tau F / (c0 + tau F) of the next step
          const float Fd = exp_ftz(ln);
          const float tF = mc.tau[r] * Fd;
          const float q = rcp_ftz(mc.c0[r] + tF);
          g[j] = tF * q;
          if (r == s) f_first = Fd - mc.disp[r];
          if (curve) {
            Prun = Prun * q;
            ann += mc.tau[r] * Prun;
            if (r == s) P1 = Prun;
          }
        }
      }
      tmem_st16_nw(tLF + cb, lp);
      tmem_st16_nw(tG + cb, g);
    }
    tmem_wait_st();
    if (done) continue;
    if (pc.kind == LMM_PRODUCT_TARN) {
      payoff += (double)(tarn_flow(pc, s, n, mc.tau[s], f_first, tarn_paid, tarn_over) * P1) /
                (double)N;
      continue;
    }
    if (pc.kind == LMM_PRODUCT_EUROPEAN) {
      const float tau = mc.tau[s];
      const float cap = tau * fmaxf(f_first - pc.cap_strike, 0.0f);
      const float swp = tau * (f_first - pc.strike) * pc.pay_receive;
      payoff += (double)((cap + swp) * P1) / (double)N;
      continue;
    }
    float coupon = 0.0f;
    if (pc.kind == LMM_PRODUCT_CANCELLABLE_SWAP)
      coupon = mc.tau[s] * (f_first - pc.strike) * pc.pay_receive * P1;
    if (e >= 0) {
      float v[kMaxVars], exv = 0.0f;
      const float Pn = Prun;
      if (pc.kind == LMM_PRODUCT_SWAPTION) {
        const float sr = (1.0f - Pn) / ann;
        v[0] = f_first;
        v[1] = sr;
        v[2] = ann;
        exv = fmaxf((sr - pc.strike) * ann, 0.0f);
      } else {
        float sr;
        if (s + 1 < n) {
          const float ann2 = ann - mc.tau[s] * P1;
          sr = (P1 - Pn) / ann2;
        } else {
          sr = (1.0f - Pn) / ann;
        }
        v[0] = f_first;
        v[1] = sr;
        v[2] = mc.tau[n - 1] * Pn;
      }
      if (MODE == kModeInputs) {
        if (bucket >= 0) o_cf[(size_t)bucket * total + col] = cf_acc;
        bucket = e;
        cf_acc = coupon;
#pragma unroll
        for (int k = 0; k < kMaxVars; ++k)
          o_vars[((size_t)e * kMaxVars + k) * total + col] = v[k];
        o_ex[(size_t)e * total + col] = exv;
        o_num[(size_t)e * total + col] = N;
      } else {
        const double est = rule_estimate(rc, e, v, exv, rule);
        if ((double)exv > est) {
          payoff += (double)exv / (double)N;
          done = true;
          continue;
        }
        payoff += (double)coupon / (double)N;
      }
      N_bucket = N;
    } else if (coupon != 0.0f) {
      if (MODE == kModeInputs) {
        if (bucket >= 0) cf_acc += coupon * (N_bucket / N);
      } else {
        payoff += (double)coupon / (double)N;
      }
    }
  }
  // a timed-out wait: report, let the tensor cores drain (bounded), free
  if (abort_s) {
    if (tid == 0) {
      atomicOr(errors, 1u);
      mbar_wait(&bar_m, 0u);
      mbar_wait(&bar_m, 1u);
    }
  }
  fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"((uint32_t)G.tmem_cols)
                 : "memory");
  if (!valid || abort_s) return;
  if (MODE == kModeInputs) {
    if (pc.kind != LMM_PRODUCT_EUROPEAN && bucket >= 0)
      o_cf[(size_t)bucket * total + col] = cf_acc;
    if ((pc.kind == LMM_PRODUCT_EUROPEAN || pc.kind == LMM_PRODUCT_TARN) && o_payoff)
      o_payoff[p] = (float)payoff;
  } else {
    o_payoff[p] = (float)payoff;
  }
}

// Shared memory of tc_evolve_kernel.
inline size_t tc_evolve_smem(int n) {
  const TcGeom G = TcGeom::make(n);
  return (size_t)G.a_bytes + G.b_bytes + (size_t)G.NB * sizeof(float);
}

}  // namespace lmm
