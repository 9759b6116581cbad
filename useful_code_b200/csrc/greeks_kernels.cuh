// greeks_kernels.cuh — pathwise adjoint of the fused pricing pass (included
// by pipeline.cu after fused_kernels.cuh).
//
// The price with a frozen exercise rule is V = P(0,T_0) mean_p Phi_p, where
// Phi_p is the sum of the path's numeraire-deflated flows up to its
// exercise step.  The exercise step of each path is recorded in the forward
// pass and held fixed (the pathwise method: the decision boundary has
// measure zero), so Phi_p is a smooth function of the initial log-rates and
// of the pseudo-roots A_s along the path.  The adjoint runs the steps
// backwards.  Log-rate checkpoints every k steps come from the recording
// forward pass; a segment kernel recomputes k steps from a checkpoint
// (pc_rate, the pricing kernels' own arithmetic) and stores the drift
// factors g (start rates) and gp (predicted rates) and the new log-rates ln
// of each step; then one reverse kernel per step:
//   * adds the adjoint of the step's flow (exercise value, coupon, caplet)
//     and of the numeraire factor (1 + tau_s f_s), which scales every later
//     flow, to a_r = dPhi/dln_r (zero where the log-rate cap applied);
//   * reverses the predictor-corrector step in one descending sweep:
//       L_r     = a_r + gp_r (1 - gp_r) sum_f A_rf h_f(r),
//                 h_f(r) = sum_{j >= r} a_j A_jf / 2     (adjoint of lp_r)
//       mubar_r = L_r - a_r / 2                          (adjoint of mu_r)
//       lam_r   = L_r + g_r (1 - g_r) sum_f A_rf k_f(r),
//                 k_f(r) = sum_{j >= r} mubar_j A_jf     (adjoint of lf_r)
//     with G'(x) = G (1 - G) for G(x) = tau e^x / (c0 + tau e^x);
//   * accumulates dV/dA_s.  With M_rj = sum_p (mubar_r g_j + a_r gp_j / 2)
//     (j <= r), N_rf = sum_p L_r z_f and l_r = sum_p L_r,
//       dV/dA_s[k][f] = sum_{j<=k} M_kj A_jf + sum_{i>=k} M_ik A_if + N_kf
//                       - A_kf l_k
//     (mu_r = sum_{j<=r} C_rj g_j with C = A A^T, dW = A z, fixed drift
//     -|A_r|^2 / 2).  The row and column sums against A are the prefix and
//     suffix factor sums the sweep already carries, so each path adds its
//     row of dV/dA_s in O(F) per rate and M (O(n^2) per path) is never
//     formed.
// Deltas: dV/df0_r = P(0,T_0) mean_p lam_r(0) / (f0_r + d_r), plus the
// derivative of P(0,T_0) = 1 / (1 + f0_0 T_0) for r = 0.
#pragma once
#include "fused_kernels.cuh"

namespace lmm {

// Paths are ordered for the reverse sweep within chunks of this many
// consecutive paths (a multiple of every CTA tile below; see
// greeks_sort_kernel).
constexpr int kSortChunk = 4096;

// Positions per CTA tile of the segment and reverse kernels.
constexpr int kRevThreads = 128;
// The segment kernel's per-rate output for one tile of kRevThreads
// positions: g, gp and ln (NaN where the cap applied) side by side, so that
// one pointer per rate reaches all three at fixed offsets.
constexpr int kSegRow = 3 * kRevThreads;

// Recompute steps [s0, s1) from the checkpoint at s0 (log-rates ckpt [n][P],
// rates r >= s0, and the numeraire ckptN [P]; the normals of step s at row
// s - zs0 of Z) and store, per step k = s - s0,
// what the reverse sweep reads: drift factors g, gp and new log-rates ln (NaN
// where the cap applied) in seg [k][n][tile][kSegRow] for rates r >= s
// (the CTA is one tile of kRevThreads positions), and seg_info
// [k][2F + 3][P] = (sum_r g_r A_rf, sum_r gp_r A_rf,
// numeraire at T_s, P(T_s, T_n), annuity of T_s).  Paths past their
// exercise step write nothing; with an order (cnt not null, [step][chunk])
// the positions of a chunk from cnt[s0][chunk] on have no work in the
// segment, and CTAs that hold only such positions return at once.
template <int FT>
__global__ void __launch_bounds__(kRevThreads, (FT > 0 && FT <= 10) ? 5 : 4)
    greeks_segment_kernel(int paths, int s0, int s1, const float* __restrict__ Z, int zs0,
                          const int* __restrict__ cnt, int chunks,
                          const float* __restrict__ A,
                          const float* __restrict__ fixed,
                          const __grid_constant__ ModelConst mc,
                          const float* __restrict__ ckpt,
                          const float* __restrict__ ckptN,
                          const int* __restrict__ ex_step, int stop_rule,
                          float* __restrict__ seg, float* __restrict__ seg_info) {
  constexpr int FM = FPad<FT>::FM;
  constexpr int FP = FPad<FT>::FP;
  const int F = FT > 0 ? FT : mc.F;
  const int n = mc.n;
  const int T = blockDim.x, tid = threadIdx.x;
  if (cnt) {  // the whole CTA (a tile of T positions never straddles chunks)
    const int q0 = blockIdx.x * T, c = q0 / kSortChunk;
    if (q0 - c * kSortChunk >= cnt[(size_t)s0 * chunks + c]) return;
  }
  extern __shared__ __align__(16) float sm[];
  float* As = sm;
  float* fx = As + n * FP;
  float* lfs = fx + ((n + 3) & ~3);
  const int p = blockIdx.x * T + tid;
  const bool valid = p < paths;
  // stop_rule 0: a path runs to its exercise step; 1 (the swaption): paths
  // never exercised have no flows and are not needed; 2 (the swaption-plus-
  // cap portfolio): every path runs to the last step for its caplets
  int stop = valid ? ex_step[p] : -1;
  // the step's discount curve (P(T_s, T_n), annuity) is read by the reverse
  // sweep only at the path's exercise step
  const int curve_step = stop;
  if (stop_rule == 1 && stop >= n) stop = -1;
  if (stop_rule == 2 && valid) stop = n - 1;
  const size_t P = (size_t)paths;
  for (int r = s0; r < n; ++r)
    lfs[r * T + tid] = valid ? ckpt[(size_t)r * P + p] : 0.0f;
  float N = valid ? ckptN[p] : 1.0f, f_first = 0.0f;
  for (int s = s0; s < s1; ++s) {
    __syncthreads();
    for (int i = tid; i < n * FP; i += T) {
      const int r = i / FP, f = i - r * FP;
      As[i] = f < F ? __ldg(A + ((size_t)s * n + r) * F + f) : 0.0f;
    }
    for (int i = tid; i < n; i += T) fx[i] = __ldg(fixed + (size_t)s * n + i);
    __syncthreads();
    if (!valid || s > stop) continue;
    if (s > s0) N = N * (1.0f + mc.tau[s - 1] * f_first);
    const size_t k = (size_t)(s - s0);
    float z[FP];
#pragma unroll
    for (int f = 0; f < FP; ++f)
      z[f] = (f < F) ? __ldg(Z + ((size_t)(s - zs0) * F + f) * P + p) : 0.0f;
    // w, v: pc_rate's running vectors; at the end of the step w = z + E and
    // v = EP - E with the step's totals E = sum_r g_r A_r and
    // EP = sum_r gp_r A_r, which the reverse sweep reads
    float2 w[FP / 2], v[FP / 2];
    step_start<FP>(z, w, v);
    const bool curve = s == curve_step;
    float Prun = 1.0f, ann = 0.0f, ln_first = 0.0f;
    const size_t seg_rate = (size_t)gridDim.x * kSegRow;  // floats between two rates
    float* sg = seg + ((k * n + s) * gridDim.x + blockIdx.x) * kSegRow + tid;
#pragma unroll 4
    for (int r = s; r < n; ++r) {
      float g, gp;
      bool capped;
      const float ln = pc_rate<FM, FP>(lfs[r * T + tid], mc.l2tau[r], mc.c0[r], fx[r],
                                       As + r * FP, w, v, mc.cutoff, g, gp, capped);
      lfs[r * T + tid] = ln;
      sg[0] = g;
      sg[kRevThreads] = gp;
      sg[2 * kRevThreads] = capped ? __int_as_float(0x7fc00000) : ln;  // NaN marks the cap
      sg += seg_rate;
      if (r == s) ln_first = ln;
      if (curve) {
        const float fn = exp_ftz(ln) - mc.disp[r];
        Prun = Prun * rcp_ftz(1.0f + mc.tau[r] * fn);
        ann += mc.tau[r] * Prun;
      }
    }
    f_first = exp_ftz(ln_first) - mc.disp[s];
    float2 e_[FP / 2], ep[FP / 2];
#pragma unroll
    for (int k = 0; k < FP / 2; ++k) {
      e_[k] = make_float2(w[k].x - z[2 * k], w[k].y - z[2 * k + 1]);
      ep[k] = make_float2(v[k].x + e_[k].x, v[k].y + e_[k].y);
    }
    float* info = seg_info + k * (2 * F + 3) * P + p;
#pragma unroll
    for (int f = 0; f < FM; ++f)
      if (f < F) {
        info[(size_t)f * P] = (f & 1) ? e_[f >> 1].y : e_[f >> 1].x;
        info[(size_t)(F + f) * P] = (f & 1) ? ep[f >> 1].y : ep[f >> 1].x;
      }
    info[(size_t)(2 * F) * P] = N;
    info[(size_t)(2 * F + 1) * P] = Prun;
    info[(size_t)(2 * F + 2) * P] = ann;
  }
}

// ---------------------------------------------------------------------------
// Paths ordered by the last step at which they carry adjoint work.
//
// A path's adjoint runs from its last step with a flow (its exercise step, or
// the last step for products that never stop) down to step 0; the paths of a
// warp run in lockstep, so with paths in simulation order a warp works at a
// step as long as any of its 32 paths does (with the c3 rule 99.7% of the
// warp-steps are live against 67% of the path-steps).  The paths of each
// chunk of kSortChunk consecutive paths are therefore put in the order of a
// stable counting sort on b = n - 1 - run_end (run_end = -1, bucket n, for
// paths with no flow at all), and every per-path buffer of the reverse
// sweep is held in that order: at step s the live paths of chunk c are the
// first cnt[s][c] positions of the chunk.  The order stays inside a chunk
// so that a chunk's row of any per-path array fits in shared memory: the
// gather into the order reads and writes whole rows coalesced.  The ranks
// are taken in path order (warp match masks and per-warp counts), so the
// order is deterministic.
constexpr int kSortThreads = 1024;

__device__ __forceinline__ int greeks_bucket(int ex, int n, int stop_rule) {
  int run_end = ex;
  if (stop_rule == 1 && ex >= n) run_end = -1;
  if (run_end > n - 1) run_end = n - 1;
  return run_end < 0 ? n : n - 1 - run_end;
}

// One CTA per chunk: perm[c C + j] = the path at position j of chunk c's
// order, ex_sorted the same for its exercise step, cnt[s][c] = the chunk's
// paths with work at step s (s < n).
__global__ void __launch_bounds__(kSortThreads)
    greeks_sort_kernel(int paths, int n, int stop_rule, const int* __restrict__ ex_step,
                       int chunks, int* __restrict__ perm, int* __restrict__ ex_sorted,
                       int* __restrict__ cnt) {
  constexpr int NWARP = kSortThreads / 32;
  __shared__ int hist[kMaxRates + 2];  // bucket sizes, then their running offsets
  __shared__ int wcnt[NWARP][kMaxRates + 1];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int c0 = blockIdx.x * kSortChunk;
  const int len = min(kSortChunk, paths - c0);
  for (int b = tid; b <= n + 1; b += kSortThreads) hist[b] = 0;
  __syncthreads();
  for (int j = tid; j < len; j += kSortThreads)
    atomicAdd(&hist[greeks_bucket(ex_step[c0 + j], n, stop_rule)], 1);
  __syncthreads();
  if (tid == 0) {
    int run = 0;
    for (int b = 0; b <= n; ++b) {
      const int h = hist[b];
      hist[b] = run;
      run += h;
    }
    hist[n + 1] = run;
  }
  __syncthreads();
  // paths with work at step s: buckets b <= n - 1 - s
  for (int st = tid; st < n; st += kSortThreads)
    cnt[(size_t)st * chunks + blockIdx.x] = hist[n - st];
  // ranks, one round of kSortThreads paths at a time, in path order
  for (int j0 = 0; j0 < len; j0 += kSortThreads) {
    for (int i = tid; i < NWARP * (kMaxRates + 1); i += kSortThreads) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const int j = j0 + tid;
    const bool valid = j < len;
    const int ex = valid ? ex_step[c0 + j] : 0;
    const int b = valid ? greeks_bucket(ex, n, stop_rule) : n + 1;  // n + 1: no path
    const unsigned peers = __match_any_sync(0xffffffffu, b);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    if (valid && rank == 0) wcnt[warp][b] = __popc(peers);
    __syncthreads();
    if (valid) {
      int pre = 0;
      for (int w = 0; w < warp; ++w) pre += wcnt[w][b];
      const int dest = c0 + hist[b] + pre + rank;
      perm[dest] = c0 + j;
      ex_sorted[dest] = ex;
    }
    __syncthreads();
    // advance the running offsets by this round's counts
    for (int bb = tid; bb <= n; bb += kSortThreads) {
      int t = 0;
      for (int w = 0; w < NWARP; ++w) t += wcnt[w][bb];
      hist[bb] += t;
    }
    __syncthreads();
  }
}

// Per segment [s0, s1): the checkpoint's log-rates (rows r >= s0) and
// numeraire, and the segment's normals, gathered into the order for the
// positions that have work.  Row y: y < n - s0 the log-rate of rate s0 + y
// (live at s0); y = n - s0 the numeraire (live at s0); above, normal (s, f)
// in step order (live at s).  One CTA per (chunk, group of rows): the chunk's
// positions are read once, then each row of the chunk is staged in shared
// memory by a coalesced read and written in the order by a coalesced write.
constexpr int kGatherThreads = 512;
constexpr int kGatherRows = 16;

__global__ void __launch_bounds__(kGatherThreads)
    greeks_gather_kernel(int paths, int n, int F, int s0, int s1, int chunks,
                         const int* __restrict__ perm, const int* __restrict__ cnt,
                         const float* __restrict__ ckpt, const float* __restrict__ ckptN,
                         const float* __restrict__ Z, float* __restrict__ ckS,
                         float* __restrict__ ckNS, float* __restrict__ Zs) {
  constexpr int PER = kSortChunk / kGatherThreads;
  __shared__ float row_s[kSortChunk];
  const int c = blockIdx.x, tid = threadIdx.x;
  const int c0 = c * kSortChunk;
  const int len = min(kSortChunk, paths - c0);
  const size_t P = (size_t)paths;
  const int rows = (n - s0) + 1 + (s1 - s0) * F;
  int src[PER];
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const int j = tid + i * kGatherThreads;
    src[i] = j < len ? perm[c0 + j] - c0 : 0;
  }
  // row y: its source, destination and number of live positions
  auto row_of = [&](int y, const float*& in, float*& out) -> int {
    int st;
    if (y < n - s0) {
      in = ckpt + (size_t)(s0 + y) * P;
      out = ckS + (size_t)(s0 + y) * P;
      st = s0;
    } else if (y == n - s0) {
      in = ckptN;
      out = ckNS;
      st = s0;
    } else {
      const int jr = y - (n - s0) - 1;
      st = s0 + jr / F;
      const int f = jr - (jr / F) * F;
      in = Z + ((size_t)st * F + f) * P;
      out = Zs + ((size_t)(st - s0) * F + f) * P;
    }
    return cnt[(size_t)st * chunks + c];  // uniform over the CTA
  };
  // the next row's values are read into registers while the current row is
  // written out of shared memory
  const int y0 = blockIdx.y * kGatherRows;
  const int y1 = min(rows, y0 + kGatherRows);
  float nxt[PER];
  const float* in;
  float* out;
  int lim = y0 < y1 ? row_of(y0, in, out) : 0;
  if (y0 < y1 && lim > 0)
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int j = tid + i * kGatherThreads;
      nxt[i] = j < len ? in[c0 + j] : 0.0f;
    }
  for (int y = y0; y < y1; ++y) {
    float* cur_out = out;
    const int cur_lim = lim;
    if (cur_lim > 0) {
      __syncthreads();  // the previous row's reads of row_s are done
#pragma unroll
      for (int i = 0; i < PER; ++i) row_s[tid + i * kGatherThreads] = nxt[i];
      __syncthreads();
    }
    if (y + 1 < y1) {
      lim = row_of(y + 1, in, out);
      if (lim > 0)
#pragma unroll
        for (int i = 0; i < PER; ++i) {
          const int j = tid + i * kGatherThreads;
          nxt[i] = j < len ? in[c0 + j] : 0.0f;
        }
    }
    if (cur_lim > 0)
#pragma unroll
      for (int i = 0; i < PER; ++i) {
        const int j = tid + i * kGatherThreads;
        if (j < cur_lim) cur_out[c0 + j] = row_s[src[i]];
      }
  }
}

// Doubles of one warp's (and one CTA's) partial sums in the reverse sweep:
// the rows of dV/dA_s [n][F], the rate adjoints [n] (read at step 0) and
// l_r = sum_p L_r [n].
__host__ __device__ constexpr int greeks_part_width(int n, int F) { return n * F + 2 * n; }

// Buffers of the reverse sweep.
struct GreeksStepBufs {
  float* lam;     // [n][P] adjoint of the log-rates (in: end of step, out: start)
  double* later;  // [P] sum of the flows after the step (deflated)
  double* part;   // [CTA][greeks_part_width] per-CTA sums of the step's
                  // dV/dA_s rows, rate adjoints and l_r
};

// The sums of the step after (the launch before): a reverse launch first
// turns the previous launch's per-CTA partials into dV/dA of that step
// (part null: nothing to do).
struct GreeksPrevSums {
  const double* part;  // the previous launch's partials (a buffer of its own)
  int s;               // their step
  int nblocks;         // CTAs of the previous launch
  double scale;        // P(0,T_0) / paths
  double* abar;        // [steps][rates][factors] output
};

// One warp: entry idx (n F + n of them) of step s from the per-CTA
// partials, summed in a fixed order (lane l adds the partials of CTAs l,
// l + 32, ..., a fixed shuffle tree adds the lanes) and scaled by
// P(0,T_0) / paths.  An entry (r, f) of dV/dA_s also sums l_r = sum_p L_r
// and subtracts A_s[r][f] l_r; the rate adjoints (idx >= n F) are kept at
// step 0 only, in lam_sum.
__device__ __forceinline__ void greeks_abar_entry(int n, int F, int s, int idx, int lane,
                                                  int nblocks, double scale,
                                                  const double* __restrict__ part,
                                                  const float* __restrict__ A,
                                                  double* __restrict__ abar,
                                                  double* __restrict__ lam_sum) {
  const int accw = greeks_part_width(n, F);
  const int lidx = idx < n * F ? n * F + n + idx / F : -1;  // l_r of the entry's rate
  double v = 0.0, l = 0.0;
  for (int c = lane; c < nblocks; c += 32) {
    v += part[(size_t)c * accw + idx];
    if (lidx >= 0) l += part[(size_t)c * accw + lidx];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_down_sync(0xffffffffu, v, o);
    l += __shfl_down_sync(0xffffffffu, l, o);
  }
  if (lane != 0) return;
  if (lidx >= 0) v -= (double)A[(size_t)s * n * F + idx] * l;
  v *= scale;
  if (idx < n * F)
    abar[(size_t)s * n * F + idx] = (idx / F >= s) ? v : 0.0;
  else if (s == 0)
    lam_sum[idx - n * F] = v;
}

// One step's forward quantities, written by the segment kernel.
struct GreeksStepIn {
  const float* seg;   // [n][tiles][kSegRow]: g, gp, ln of rates r >= s
  const float* info;  // [2F + 3][P] factor totals, numeraire, P(T_s,T_n), annuity
};

// Row stride of a warp's stage in the reverse kernel: the lanes' rows of
// dV/dA (factor pairs 0 .. NP-1, NP = (FM + 1) / 2), the rate adjoint in
// column 2 NP and L_r in column 2 NP + 1; even (8-byte aligned pair stores)
// with an odd number of pairs, so the 16 lanes of a half-warp's pair store
// hit distinct bank pairs.  Lanes 16..31 write 16 floats further on, so the
// two halves of the column sums read disjoint banks (16 NC is a multiple of
// 32 banks).
__host__ __device__ constexpr int rev_stage_cols(int FM) {
  return (((FM + 1) / 2 + 1) & 1) ? 2 * ((FM + 1) / 2) + 2 : 2 * ((FM + 1) / 2) + 4;
}
__host__ __device__ constexpr int rev_stage_floats(int FM) { return 32 * rev_stage_cols(FM) + 16; }

// Live tiles of each step in the order (a chunk's live tiles at step s are
// its first ceil(cnt[s][c] / T)): live[s] = their number and
// tile_list[s][0 .. live[s]) = the tiles, chunk by chunk.  One warp per
// step.
__global__ void __launch_bounds__(32)
    greeks_live_tiles_kernel(int chunks, int tiles, const int* __restrict__ cnt,
                             int* __restrict__ live, int* __restrict__ tile_list) {
  constexpr int TPC = kSortChunk / kRevThreads;  // tiles per chunk
  const int st = blockIdx.x, lane = threadIdx.x;
  int* list = tile_list + (size_t)st * tiles;
  int carry = 0;
  for (int c0 = 0; c0 < chunks; c0 += 32) {
    const int c = c0 + lane;
    const int x = c < chunks ? (cnt[(size_t)st * chunks + c] + kRevThreads - 1) / kRevThreads
                             : 0;
    int incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int base = carry + incl - x;
    for (int i = 0; i < x; ++i) list[base + i] = c * TPC + i;
    carry += __shfl_sync(0xffffffffu, incl, 31);
  }
  if (lane == 0) live[st] = carry;
}

// Reverse of step s (one launch per step, steps descending; persistent CTAs
// walk the step's live tiles of kRevThreads positions, NPATH tiles at a
// time: each thread carries the paths at its position in NPATH tiles).  Per
// path and rate r (descending) the contribution to dV/dA_s[r][f] is
//   mubar_r e_f(r) + a_r ep_f(r) / 2 + g_r k_f(r) + gp_r h_f(r)
//   + L_r z_f   (and - A_rf L_r)
// with the prefix sums e_f(r) = sum_{j<=r} g_j A_jf (and ep with gp) taken
// as the step total minus the suffix beyond r, and the suffix sums k, h of
// the sweep: the row and column sums of M = sum_p (mubar g^T + a gp^T / 2)
// against A without forming M.  The last term's path sum is A_rf l_r with
// l_r = sum_p L_r, so the sweep sums L_r as one more column and
// greeks_abar_kernel subtracts A_rf l_r once per entry.  A thread adds the
// rows of its paths in registers; the sums over the lanes of a warp go
// through a shared-memory transpose (two lanes per column, 16 rows each,
// one shuffle); each warp keeps FP64 sums in shared memory, and the CTA
// writes its partial in a fixed order.  Warps whose paths all have work at the step (the common case
// once the paths are ordered) and none of which exercises at the step run
// the sweep without per-lane predicates and without the exercise value's
// discount curve.
template <int FT>
struct RevShape {
  static constexpr int NPATH = (FT > 0 && FT <= 10) ? 2 : 1;  // paths per thread
  static constexpr int MINB = (FT > 0 && FT <= 5) ? 4 : (FT == 10 ? 3 : 1);
};

template <int FT>
__global__ void __launch_bounds__(kRevThreads, RevShape<FT>::MINB)
    greeks_reverse_kernel(int paths, int s, const float* __restrict__ Z, int zs0,
                          const int* __restrict__ live_n, const int* __restrict__ tile_list,
                          const float* __restrict__ A,
                          const __grid_constant__ ModelConst mc,
                          const __grid_constant__ ProductConst pc,
                          const GreeksStepIn in, const int* __restrict__ ex_step,
                          const GreeksStepBufs b, const GreeksPrevSums prev) {
  constexpr int FM = FPad<FT>::FM;
  constexpr int FP = FPad<FT>::FP;
  constexpr int T = kRevThreads, NW = kRevThreads / 32;
  constexpr int NP = (FM + 1) / 2;  // factor pairs that hold factors
  constexpr int NC = rev_stage_cols(FM);
  constexpr int NS = FM + 2;        // summed columns: FM factors, the adjoint, L
  constexpr int LAMC = 2 * NP;      // stage column of the rate adjoint
  constexpr int NPATH = RevShape<FT>::NPATH;
  const int F = FT > 0 ? FT : mc.F;
  const int n = mc.n;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tiles = (paths + T - 1) / T;
  extern __shared__ __align__(16) float sm[];
  double* acc = reinterpret_cast<double*>(sm);        // [NW][n F + n + n]
  const int accw = greeks_part_width(n, F);            // doubles per warp
  float* As = reinterpret_cast<float*>(acc + (size_t)NW * accw);  // [n][FP]
  float* stage = As + (size_t)n * FP + (size_t)warp * rev_stage_floats(FM);
  for (int i = tid; i < n * FP; i += T) {
    const int r = i / FP, f = i - r * FP;
    As[i] = f < F ? __ldg(A + ((size_t)s * n + r) * F + f) : 0.0f;
  }
  for (int i = tid; i < NW * accw; i += T) acc[i] = 0.0;
  // dV/dA of the step after (prev.s > 0, so no rate adjoints), from the
  // previous launch's partials: one entry per warp of the grid, looping
  // while the grid has fewer warps than entries
  if (prev.part) {
    for (int idx = blockIdx.x * NW + warp; idx < n * F + n; idx += gridDim.x * NW)
      greeks_abar_entry(n, F, prev.s, idx, lane, prev.nblocks, prev.scale, prev.part, A,
                        prev.abar, nullptr);
  }
  __syncthreads();
  double* myacc = acc + (size_t)warp * accw;
  // this lane's row of the stage, and the column it sums.  With 2 NS <= 32
  // lanes [0, NS) add rows 0..15 and lanes [NS, 2 NS) rows 16..31 (one
  // shuffle joins them); otherwise lanes [0, NS) add all 32 rows.  The other
  // lanes repeat lane 0's reads (same addresses: no bank conflict) and
  // discard them.
  float* wrow = stage + lane * NC + (lane >> 4) * 16;
  constexpr bool kSplit = 2 * NS <= 32;
  const int csum = lane < NS ? lane : (kSplit && lane < 2 * NS ? lane - NS : 0);
  const float* rd = stage + (kSplit && lane >= NS && lane < 2 * NS ? 16 * NC + 16 : 0) +
                    (csum < FM ? csum : LAMC + (csum - FM));
  const bool row_lane = lane < F;                // adds dV/dA_s[r][lane]
  const bool lam_lane = (s == 0) && lane == FM;  // adds the adjoint at step 0
  const bool l_lane = lane == FM + 1;            // adds l_r = sum_p L_r
  const size_t P = (size_t)paths;
  const size_t seg_rate = (size_t)tiles * kSegRow;  // floats between two rates
  const int* tl = tile_list ? tile_list + (size_t)s * tiles : nullptr;
  const int live = tl ? live_n[s] : tiles;
  const int e_s = pc.ex_index[s];
  const float tau_s = mc.tau[s];
  const float strike = pc.strike;
  for (int t0 = blockIdx.x * NPATH; t0 < live; t0 += gridDim.x * NPATH) {
    // ---- per path: the flow at step s and the step's factor vectors ----
    int p[NPATH];
    bool act[NPATH];
    const float* seg_s[NPATH];
    float2 z2[NPATH][NP], eg[NPATH][NP], ef[NPATH][NP];
    float Pn[NPATH], ex_scale[NPATH], dterm_fs[NPATH];
    bool any = false, all = true;
#pragma unroll
    for (int q = 0; q < NPATH; ++q) {
      const bool has = t0 + q < live;
      const int tile = has ? (tl ? tl[t0 + q] : t0 + q) : 0;
      p[q] = tile * T + tid;
      // every per-position load below reads an allocated position (pv), so
      // they all issue at once; the values of positions without work at the
      // step are discarded by act
      const int pv = p[q] < paths ? p[q] : paths - 1;
      const int stop = (has && p[q] < paths) ? ex_step[pv] : -1;
      // a path contributes at step s if it is still running there and has a
      // flow at or after s (a swaption only at its exercise step; the
      // swaption-plus-cap portfolio runs every path to the last step)
      // (an inactive path's adjoint rows keep the zeros of the start of the
      // call until its exercise step: nothing writes them before)
      const int run_end = (pc.kind == LMM_PRODUCT_BERMUDAN_CAP) ? n - 1 : stop;
      bool a_ = has && p[q] < paths && s <= run_end;
      if (pc.kind == LMM_PRODUCT_SWAPTION && stop >= n) a_ = false;
      act[q] = a_;
      any = any || a_;
      all = all && a_;
      seg_s[q] = in.seg + ((size_t)s * tiles + tile) * kSegRow + tid;  // rate s
      // z: the step's normals; eg, ef: the prefix sums sum_{j<=r} g_j A_j and
      // sum_{j<=r} gp_j A_j, from the step totals down (the sweep subtracts
      // each rate after its row)
#pragma unroll
      for (int k = 0; k < NP; ++k) {
        float zz[2], ee[2], eq[2];
#pragma unroll
        for (int h2 = 0; h2 < 2; ++h2) {
          const int f = 2 * k + h2;
          zz[h2] = f < F ? __ldg(Z + ((size_t)(s - zs0) * F + f) * P + pv) : 0.0f;
          ee[h2] = f < F ? in.info[(size_t)f * P + pv] : 0.0f;
          eq[h2] = f < F ? in.info[(size_t)(F + f) * P + pv] : 0.0f;
          if (!a_) zz[h2] = ee[h2] = eq[h2] = 0.0f;
        }
        z2[q][k] = make_float2(zz[0], zz[1]);
        eg[q][k] = make_float2(ee[0], ee[1]);
        ef[q][k] = make_float2(eq[0], eq[1]);
      }
      float N = in.info[(size_t)(2 * F) * P + pv];
      float Pnq = in.info[(size_t)(2 * F + 1) * P + pv];
      float ann = in.info[(size_t)(2 * F + 2) * P + pv];
      const float l0 = seg_s[q][2 * kRevThreads];
      const double later_in = b.later[pv];
      if (!a_) {
        N = 1.0f;
        Pnq = 1.0f;
        ann = 0.0f;
      }
      float f_s = 0.0f, P1 = 1.0f;
      if (a_) {
        f_s = exp_ftz(l0 != l0 ? mc.cutoff : l0) - mc.disp[s];
        P1 = 1.0f / (1.0f + tau_s * f_s);
      }
      const bool is_ex = a_ && (s == stop) && (e_s >= 0) && pc.kind != LMM_PRODUCT_EUROPEAN;
      const float invN = 1.0f / N;
      float term = 0.0f;  // flow / N at step s
      float dts = 0.0f;   // d(term)/d f_s from the flows that depend on f_s only
      bool swaption_ex = false;
      if (!a_) {
      } else if (pc.kind == LMM_PRODUCT_EUROPEAN) {
        const float cap = tau_s * fmaxf(f_s - pc.cap_strike, 0.0f);
        const float swp = tau_s * (f_s - pc.strike) * pc.pay_receive;
        term = (cap + swp) * P1 * invN;
        const float dv = tau_s * ((f_s > pc.cap_strike ? 1.0f : 0.0f) + pc.pay_receive);
        dts = (dv * P1 - (cap + swp) * P1 * tau_s * P1) * invN;
      } else if (pc.kind == LMM_PRODUCT_BERMUDAN_CAP) {
        // caplet on f_s paid at T_{s+1}, plus the swaption at its exercise
        const float cap = tau_s * fmaxf(f_s - pc.cap_strike, 0.0f);
        term = cap * P1 * invN;
        dts = (tau_s * (f_s > pc.cap_strike ? 1.0f : 0.0f) * P1 - cap * P1 * tau_s * P1) *
              invN;
        if (is_ex) {
          const float v = (1.0f - Pnq) - pc.strike * ann;
          if (v > 0.0f) {
            term += v * invN;
            swaption_ex = true;
          }
        }
      } else if (pc.kind == LMM_PRODUCT_CANCELLABLE_SWAP) {
        if (!is_ex) {
          const float c = tau_s * (f_s - pc.strike) * pc.pay_receive;
          term = c * P1 * invN;
          dts = (tau_s * pc.pay_receive * P1 - c * P1 * tau_s * P1) * invN;
        }
      } else if (is_ex) {
        const float v = (1.0f - Pnq) - pc.strike * ann;
        if (v > 0.0f) {
          term = v * invN;
          swaption_ex = true;
        }
      }
      if (a_) {
        // the numeraire factor (1 + tau_s f_s) divides every later flow
        dts += -(float)later_in * tau_s / (1.0f + tau_s * f_s);
        b.later[p[q]] = later_in + (double)term;
      }
      dterm_fs[q] = dts;
      Pn[q] = Pnq;
      // the exercise value's derivative with respect to f_r, r >= s, is
      // tau_r / (1 + tau_r f_r) (P(T_s,T_n) + K sum_{k>=r} tau_k
      // P(T_s,T_{k+1})) / N: its scale, zero where the path does not
      // exercise here
      ex_scale[q] = swaption_ex ? invN : 0.0f;
    }
    // a warp with no active path adds exact zeros to every sum: skip it
    if (!__any_sync(0xffffffffu, any)) continue;
    // ---- descending sweep (every lane of the warp, for the warp sums) ----
    // Factor vectors are held in pairs (f = 2k, 2k + 1) and updated with
    // packed FP32x2 FMAs, as in the forward rate step; the two halves of a
    // dot product are added at the end.
    // EX: a path of the warp exercises at step s, so the exercise value's
    // derivative reaches every rate; without one only the step's own rate
    // carries a flow derivative, and the other rates need neither their
    // rate nor the discount curve
    auto sweep = [&](auto all_tag, auto ex_tag) {
      constexpr bool ALL = decltype(all_tag)::value;  // every path of the warp active
      constexpr bool EX = decltype(ex_tag)::value;
      float2 h[NPATH][NP], kk[NPATH][NP];
      float Pr[NPATH], ann_suf[NPATH];
      const float* sp[NPATH];
      float* lp[NPATH];
      // each rate's inputs are loaded two iterations ahead (a and b: the
      // next two rates); rates below s and the adjoint of rate s (no input
      // from the later step) read as zero
      float a_g[NPATH], a_gp[NPATH], a_ln[NPATH], a_lam[NPATH];
      float b_g[NPATH], b_gp[NPATH], b_ln[NPATH], b_lam[NPATH];
#pragma unroll
      for (int q = 0; q < NPATH; ++q) {
#pragma unroll
        for (int k = 0; k < NP; ++k) h[q][k] = kk[q][k] = make_float2(0.0f, 0.0f);
        Pr[q] = Pn[q];
        ann_suf[q] = 0.0f;
        sp[q] = seg_s[q] + (size_t)(n - 1 - s) * seg_rate;  // rate n - 1
        lp[q] = b.lam + (size_t)(n - 1) * P + (p[q] < paths ? p[q] : 0);
        a_g[q] = a_gp[q] = a_ln[q] = a_lam[q] = 0.0f;
        b_g[q] = b_gp[q] = b_ln[q] = b_lam[q] = 0.0f;
        if (ALL || act[q]) {
          a_g[q] = sp[q][0];
          a_gp[q] = sp[q][kRevThreads];
          a_ln[q] = sp[q][2 * kRevThreads];
          a_lam[q] = (n - 1 > s) ? *lp[q] : 0.0f;
          if (n - 2 >= s) {
            b_g[q] = sp[q][-(ptrdiff_t)seg_rate];
            b_gp[q] = sp[q][kRevThreads - (ptrdiff_t)seg_rate];
            b_ln[q] = sp[q][2 * kRevThreads - (ptrdiff_t)seg_rate];
            b_lam[q] = (n - 2 > s) ? lp[q][-(ptrdiff_t)P] : 0.0f;
          }
        }
      }
      const float* arow = As + (n - 1) * FP;
      double* ar = myacc + (n - 1) * F + lane;
      double* al = myacc + (size_t)n * F + (n - 1);  // adjoint sums; l_r n further on
      // two rates per iteration: the row and the column sums of one rate
      // overlap the adjoint chain of the next
#pragma unroll 2
      for (int r = n - 1; r >= s; --r) {
        const float4* a4 = reinterpret_cast<const float4*>(arow);
        float2 av[FP / 2];
#pragma unroll
        for (int qq = 0; qq < FP / 4; ++qq) {
          const float4 v4 = a4[qq];
          av[2 * qq] = make_float2(v4.x, v4.y);
          av[2 * qq + 1] = make_float2(v4.z, v4.w);
        }
        const float tr = mc.tau[r], dr = mc.disp[r];
        float2 row[NP];
        float lam_sum_r = 0.0f, l_sum_r = 0.0f;
#pragma unroll
        for (int q = 0; q < NPATH; ++q) {
          const float ln_raw = a_ln[q], lam_in = a_lam[q], g_in = a_g[q], gp_in = a_gp[q];
          a_g[q] = b_g[q];
          a_gp[q] = b_gp[q];
          a_ln[q] = b_ln[q];
          a_lam[q] = b_lam[q];
          sp[q] -= seg_rate;
          if (r - 2 >= s && (ALL || act[q])) {
            b_g[q] = sp[q][-(ptrdiff_t)seg_rate];
            b_gp[q] = sp[q][kRevThreads - (ptrdiff_t)seg_rate];
            b_ln[q] = sp[q][2 * kRevThreads - (ptrdiff_t)seg_rate];
            b_lam[q] = (r - 2 > s) ? lp[q][-2 * (ptrdiff_t)P] : 0.0f;
          }
          const bool capped = ln_raw != ln_raw;
          float a;
          if (EX) {
            const float Fd = exp_ftz(capped ? mc.cutoff : ln_raw);  // f_r + d_r = df_r / dln_r
            const float onep = 1.0f + tr * (Fd - dr);
            // Pr = P(T_s, T_{r+1}); ann_suf = sum_{k >= r} tau_k P(T_s, T_{k+1})
            ann_suf[q] = fmaf(tr, Pr[q], ann_suf[q]);
            float dphi_df = tr * rcp_ftz(onep) * (Pn[q] + strike * ann_suf[q]) * ex_scale[q];
            if (r == s) dphi_df += dterm_fs[q];
            a = capped ? 0.0f : fmaf(dphi_df, Fd, lam_in);
            Pr[q] = Pr[q] * onep;  // P(T_s, T_r)
          } else if (r == s) {
            const float Fd = exp_ftz(capped ? mc.cutoff : ln_raw);
            a = capped ? 0.0f : fmaf(dterm_fs[q], Fd, lam_in);
          } else {
            a = capped ? 0.0f : lam_in;
          }
          float g = g_in, gp = gp_in;
          if (!ALL && !act[q]) a = g = gp = 0.0f;
          const float ha = 0.5f * a;
          const float2 ha2 = make_float2(ha, ha);
          // dot products in two packed accumulators (even and odd pairs)
          float2 s1a = make_float2(0.0f, 0.0f), s1b = s1a;
#pragma unroll
          for (int k = 0; k < NP; ++k) {
            h[q][k] = __ffma2_rn(ha2, av[k], h[q][k]);
            if (k & 1)
              s1b = __ffma2_rn(av[k], h[q][k], s1b);
            else
              s1a = __ffma2_rn(av[k], h[q][k], s1a);
          }
          const float L = a + gp * (1.0f - gp) * ((s1a.x + s1a.y) + (s1b.x + s1b.y));
          const float mubar = L - ha;
          const float2 mb2 = make_float2(mubar, mubar);
          float2 s2a = make_float2(0.0f, 0.0f), s2b = s2a;
#pragma unroll
          for (int k = 0; k < NP; ++k) {
            kk[q][k] = __ffma2_rn(mb2, av[k], kk[q][k]);
            if (k & 1)
              s2b = __ffma2_rn(av[k], kk[q][k], s2b);
            else
              s2a = __ffma2_rn(av[k], kk[q][k], s2a);
          }
          const float lam_out = L + g * (1.0f - g) * ((s2a.x + s2a.y) + (s2b.x + s2b.y));
          if (ALL || act[q]) *lp[q] = lam_out;
          lam_sum_r += lam_out;
          l_sum_r += L;
          // this path's row r of dV/dA_s without its - A_r L_r term, added to
          // the thread's row (eg, ef: the prefix sums through r)
          const float2 g2 = make_float2(g, g), gp2 = make_float2(gp, gp);
          const float2 L2 = make_float2(L, L);
          const float2 ng2 = make_float2(-g, -g), ngp2 = make_float2(-gp, -gp);
#pragma unroll
          for (int k = 0; k < NP; ++k) {
            float2 x = q == 0 ? __fmul2_rn(mb2, eg[q][k]) : __ffma2_rn(mb2, eg[q][k], row[k]);
            x = __ffma2_rn(ha2, ef[q][k], x);
            x = __ffma2_rn(g2, kk[q][k], x);
            x = __ffma2_rn(gp2, h[q][k], x);
            row[k] = __ffma2_rn(L2, z2[q][k], x);
            eg[q][k] = __ffma2_rn(ng2, av[k], eg[q][k]);
            ef[q][k] = __ffma2_rn(ngp2, av[k], ef[q][k]);
          }
          lp[q] -= P;
        }
#pragma unroll
        for (int k = 0; k < NP; ++k) reinterpret_cast<float2*>(wrow)[k] = row[k];
        // column LAMC holds the rate adjoint (for the step-0 sums), LAMC + 1
        // the paths' L_r
        wrow[LAMC] = lam_sum_r;
        wrow[LAMC + 1] = l_sum_r;
        __syncwarp();
        float t0s = 0.0f, t1s = 0.0f, tsum;
        if constexpr (kSplit) {
#pragma unroll
          for (int l = 0; l < 16; l += 2) {
            t0s += rd[l * NC];
            t1s += rd[(l + 1) * NC];
          }
          tsum = t0s + t1s;
          tsum += __shfl_down_sync(0xffffffffu, tsum, NS);
        } else {
#pragma unroll
          for (int l = 0; l < 16; ++l) {
            t0s += rd[l * NC];
            t1s += rd[16 * NC + 16 + l * NC];
          }
          tsum = t0s + t1s;
        }
        if (row_lane) *ar += (double)tsum;
        if (lam_lane) *al += (double)tsum;
        if (l_lane) al[n] += (double)tsum;
        __syncwarp();
        arow -= FP;
        ar -= F;
        al -= 1;
      }
    };
    bool ex_here = false;
#pragma unroll
    for (int q = 0; q < NPATH; ++q) ex_here = ex_here || ex_scale[q] != 0.0f;
    const bool all_w = __all_sync(0xffffffffu, all);
    const bool ex_w = __any_sync(0xffffffffu, ex_here);
    // the common case (every path of the warp live, none exercising here)
    // runs without predicates and without the curve; any other warp runs
    // the general sweep
    if (all_w && !ex_w)
      sweep(std::true_type(), std::false_type());
    else
      sweep(std::false_type(), std::true_type());
  }
  // fixed-order sum over the warps, one partial per CTA
  __syncthreads();
  double* out = b.part + (size_t)blockIdx.x * accw;
  for (int i = tid; i < accw; i += T) {
    double v = 0.0;
    for (int w = 0; w < NW; ++w) v += acc[(size_t)w * accw + i];
    out[i] = v;
  }
}

// dV/dA_s (and at step 0 the adjoint sums behind the deltas) from the
// per-CTA partials, summed in a fixed order and scaled by P(0,T_0) / paths:
// one warp per entry (n F + n of them), lane l adds the partials of CTAs l,
// l + 32, ... and a fixed shuffle tree adds the lanes.  An entry (r, f) of
// dV/dA_s also sums l_r = sum_p L_r and subtracts A_s[r][f] l_r.
constexpr int kAbarThreads = 256;
__global__ void __launch_bounds__(kAbarThreads)
    greeks_abar_kernel(int n, int F, int s, int nblocks, double scale,
                       const double* __restrict__ part, const float* __restrict__ A,
                       double* __restrict__ abar, double* __restrict__ lam_sum) {
  const int idx = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;  // warp-uniform
  if (idx >= n * F + n) return;
  greeks_abar_entry(n, F, s, idx, threadIdx.x & 31, nblocks, scale, part, A, abar, lam_sum);
}

// Price, deltas and per-rate vegas.  lam_sum[r] = P(0,T_0) mean_p lam_r(0);
// mean_payoff = mean_p Phi_p.  vega_rate[r] = sum_{s,f} abar A (derivative
// with respect to a scaling of row r of every pseudo-root).
__global__ void greeks_finish_kernel(int n, int F, const __grid_constant__ ModelConst mc,
                                     float f0_0, float T0, const double* __restrict__ lam_sum,
                                     const double* __restrict__ mean_payoff,
                                     const float* __restrict__ A,
                                     const double* __restrict__ abar,
                                     double* __restrict__ price, double* __restrict__ delta,
                                     double* __restrict__ vega_rate) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const double P0 = 1.0 / (1.0 + (double)f0_0 * (double)T0);
  if (r == 0 && price) price[0] = P0 * mean_payoff[0];
  if (r >= n) return;
  const double Fd = exp((double)mc.logf0[r]);  // f0_r + d_r
  double d = lam_sum[r] / Fd;
  if (r == 0) d += -(double)T0 * P0 * P0 * mean_payoff[0];
  delta[r] = d;
  if (vega_rate) {
    double v = 0.0;
    for (int s = 0; s < n; ++s)
      for (int f = 0; f < F; ++f)
        v += abar[((size_t)s * n + r) * F + f] * (double)A[((size_t)s * n + r) * F + f];
    vega_rate[r] = v;
  }
}

// Shared memory of the reverse kernel.
inline size_t greeks_reverse_smem(int n, int F) {
  const int FP = launched_row_pad(F);
  const size_t acc = (size_t)(kRevThreads / 32) * greeks_part_width(n, F) * sizeof(double);
  const size_t stage = (size_t)(kRevThreads / 32) * rev_stage_floats(launched_fm(F)) *
                       sizeof(float);
  return acc + (size_t)n * FP * sizeof(float) + stage;
}

}  // namespace lmm
