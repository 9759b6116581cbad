// lmm_oracle.cpp — CPU restatement of the reference's LMM pricing path.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels.  Only tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs load
// this library; the product never does.  Each routine restates, in plain
// scalar C++ templated on the arithmetic type R (float or double), the
// reference routine cited in its comment (paths relative to the Kooderive
// r256 tree).  Instantiated with R = double and fed the same Sobol integers
// it is the FP64 oracle for prices.  Parity pinning: the stage functions are
// checked against the reference's own gold code (oracle/_ref/libkooref.so)
// and against fixtures under tests/golden/ generated from it.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#define ORC extern "C" __attribute__((visibility("default")))

namespace {

// --- Sobol ----------------------------------------------------------------
// Bratley–Fox direction numbers (gold/sobol_gold.cpp:118-164).
void directions(int dims, const uint32_t* degree, const uint32_t* a,
                const uint32_t* m, int mstride, uint32_t* out) {
  for (int d = 0; d < dims; ++d) {
    uint32_t* v = out + 32 * (size_t)d;
    if (d == 0) {
      for (int i = 0; i < 32; ++i) v[i] = 1u << (31 - i);
      continue;
    }
    const int s = (int)degree[d];
    for (int i = 0; i < s; ++i) v[i] = m[(size_t)d * mstride + i] << (31 - i);
    for (int i = s; i < 32; ++i) {
      v[i] = v[i - s] ^ (v[i - s] >> s);
      for (int k = 1; k < s; ++k)
        v[i] ^= ((a[d] >> (s - 1 - k)) & 1u) * v[i - k];
    }
  }
}

// Point n of dimension d: XOR of v[k] over the set bits k of gray(n)
// (sobol_int_gpu.cu:76-121, same values as the recurrence of
// gold/sobol_gold.cpp:168-204 which skips point 0).
inline uint32_t sobol_point(const uint32_t* v, uint32_t n) {
  uint32_t g = n ^ (n >> 1), x = 0;
  for (int k = 0; g; ++k, g >>= 1)
    if (g & 1u) x ^= v[k];
  return x;
}

// --- inverse cumulative normal ---------------------------------------------
// Shaw–Brickman rational form (inverseCumulatives.h:146-172), evaluated in R.
template <class R>
R icdf_sb(R v) {
  const R P1 = 1.2533136835212087879, P2 = 1.9797154223229267471,
          P3 = 0.80002295072483916762, P4 = 0.087403248265958578062,
          P5 = 0.0020751409553756572917, P6 = 4.744820732427972462e-6;
  const R Q1 = 1.0, Q2 = 2.0795584360534589311, Q3 = 1.2499328117341603014,
          Q4 = 0.23668431621373705623, Q5 = 0.0120098270559197768,
          Q6 = 0.00010590620919921025259;
  const R sgn = v >= R(0.5) ? R(1) : R(-1);
  R t = R(1) - sgn * ((R(2) * v) - R(1));
  if (t < R(2.3283064365386963e-10)) t = R(2.3283064365386963e-10);
  const R z = -std::log(t);
  const R p = P1 + z * (P2 + z * (P3 + z * (P4 + (P5 + P6 * z) * z)));
  const R q = Q1 + z * (Q2 + z * (Q3 + z * (Q4 + (Q5 + Q6 * z) * z)));
  return sgn * z * p / q;
}

// FP32 path: u = float(i) * 2^-32 as the reference.
inline float icdf_f(uint32_t i) { return icdf_sb<float>((float)i * 2.3283064E-10f); }

// FP32 path of the pipelines: the same rational form on the tail
// probability t = min(i, 2^32 - i) * 2^-31 taken from the integer (the
// device's icdf_sb_tails), which avoids the 2^-24 quantisation of
// 1 - |2u - 1| in single precision.
inline float icdf_f_tails(uint32_t i) {
  const bool upper = i >= 0x80000000u;
  const float sgn = upper ? 1.0f : -1.0f;
  const uint32_t m = upper ? (0u - i) : i;
  float t = (float)m * 4.656612873077392578125e-10f;
  if (t < 2.3283064365386963e-10f) t = 2.3283064365386963e-10f;
  const float z = -std::log(t);
  const float p = 1.2533136835212087879f +
                  z * (1.9797154223229267471f +
                       z * (0.80002295072483916762f +
                            z * (0.087403248265958578062f +
                                 (0.0020751409553756572917f + 4.744820732427972462e-6f * z) * z)));
  const float q = 1.0f +
                  z * (2.0795584360534589311f +
                       z * (1.2499328117341603014f +
                            z * (0.23668431621373705623f +
                                 (0.0120098270559197768f + 0.00010590620919921025259f * z) * z)));
  return sgn * z * p / q;
}

// FP64 path: exact u = i * 2^-32 (clamped like the FP32 path at the two
// ends), Shaw–Brickman start refined by Newton steps on Phi(x) - u with
// Phi(x) = erfc(-x/sqrt2)/2, which converge to double precision.
inline double icdf_d(uint32_t i) {
  double u = (double)i * 2.3283064365386963e-10;
  const double lo = 1.1641532182693481e-10;  // 2^-33
  if (u < lo) u = lo;
  if (u > 1.0 - lo) u = 1.0 - lo;
  double x = icdf_sb<double>(u);
  for (int it = 0; it < 3; ++it) {
    const double cdf = 0.5 * std::erfc(-x * 0.70710678118654752440);
    const double pdf = 0.39894228040143267794 * std::exp(-0.5 * x * x);
    if (!(pdf > 0)) break;
    x -= (cdf - u) / pdf;
  }
  return x;
}

// --- Brownian bridge ---------------------------------------------------------
// Construction tables (brownian_bridge.cu:639-697, t_i = i + 1).
template <class R>
struct Bridge {
  int S;
  std::vector<R> lw, rw, sd;
  std::vector<int> left, right, bidx;
  explicit Bridge(int steps)
      : S(steps), lw(steps), rw(steps), sd(steps), left(steps), right(steps),
        bidx(steps) {
    std::vector<R> t(S);
    for (int i = 0; i < S; ++i) t[i] = R(i + 1);
    std::vector<int> map(S, 0);
    map[S - 1] = 1;
    bidx[0] = S - 1;
    sd[0] = std::sqrt(t[S - 1]);
    lw[0] = rw[0] = R(0);
    for (int j = 0, i = 1; i < S; ++i) {
      while (map[j]) ++j;
      int k = j;
      while (!map[k]) ++k;
      int l = j + ((k - 1 - j) >> 1);
      map[l] = i;
      bidx[i] = l;
      left[i] = j;
      right[i] = k;
      if (j != 0) {
        lw[i] = (t[k] - t[l]) / (t[k] - t[j - 1]);
        rw[i] = (t[l] - t[j - 1]) / (t[k] - t[j - 1]);
        sd[i] = std::sqrt(((t[l] - t[j - 1]) * (t[k] - t[l])) / (t[k] - t[j - 1]));
      } else {
        lw[i] = (t[k] - t[l]) / t[k];
        rw[i] = t[l] / t[k];
        sd[i] = std::sqrt(t[l] * (t[k] - t[l]) / t[k]);
      }
      j = k + 1;
      if (j >= S) j = 0;
    }
  }
  // One factor of one path: z indexed by bridge stage, out = increments.
  void path(const R* z, R* w, R* inc) const {
    w[S - 1] = sd[0] * z[0];
    for (int i = 1; i < S; ++i) {
      const int j = left[i], k = right[i], l = bidx[i];
      R x = (j != 0) ? lw[i] * w[j - 1] : R(0);
      x += rw[i] * w[k];
      x += sd[i] * z[i];
      w[l] = x;
    }
    R prev = 0;
    for (int s = 0; s < S; ++s) {
      inc[s] = w[s] - prev;
      prev = w[s];
    }
  }
};

// Diagonal allocation (gold/Bridge_allocator_gold.cpp:38-76).
void alloc_diagonal(int F, int S, int* idx) {
  int i0 = 0, j0 = 0, i = 0, j = 0;
  for (int c = 0; c < F * S; ++c) {
    idx[i * S + j] = c;
    if (i == 0 || j == S - 1) {
      if (i0 < F - 1) {
        ++i0;
        j0 = 0;
      } else {
        i0 = F - 1;
        ++j0;
      }
      i = i0;
      j = j0;
    } else {
      --i;
      ++j;
    }
  }
}

// --- spot-measure drift (gold/LMM_evolver_gold.h:178-203) ------------------
template <class R>
void spot_drift(const R* A, const R* f, const R* tau, const R* disp, int n,
                int F, R* mu) {
  std::vector<R> e(F, R(0));
  for (int r = 0; r < n; ++r) {
    const R g = (f[r] + disp[r]) * tau[r] / (R(1) + f[r] * tau[r]);
    R x = 0;
    for (int k = 0; k < F; ++k) {
      e[k] += A[r * F + k] * g;
      x += A[r * F + k] * e[k];
    }
    mu[r] = x;
  }
}

// Predictor-corrector step over all rates (gold/LMM_evolver_gold.h:315-387):
// predictor drift from the rates at the start of the step, corrector drift
// from the predicted rates, log-rates capped at cutoff.
template <class R>
void pc_step(const R* A, const R* corr, const R* tau, const R* disp, int n,
             int F, R cutoff, R* f, R* lf, R* mu, R* mup) {
  spot_drift(A, f, tau, disp, n, F, mu);
  for (int r = 0; r < n; ++r) {
    lf[r] += mu[r] + corr[r];
    f[r] = std::exp(lf[r]) - disp[r];
  }
  spot_drift(A, f, tau, disp, n, F, mup);
  for (int r = 0; r < n; ++r) {
    R x = (lf[r] += R(0.5) * (mup[r] - mu[r]));
    if (x > cutoff) lf[r] = x = cutoff;
    f[r] = std::exp(lf[r]) - disp[r];
  }
}

// --- pipeline description ---------------------------------------------------
// kBermudanCap: the Bermudan payer swaption plus a cap strip paid on every
// period whatever the exercise (no reference product; the portfolio of the
// differentiation form).
enum Product { kSwaption = 0, kCancellableSwap = 1, kEuropean = 2, kTarn = 3, kBermudanCap = 4 };

// One TARN period (TARN_gold::getCashFlows, gold/cashFlowGeneration_product_gold.h:
// 106-146): floating flow tau f, inverse-floater coupon max(K - m f, 0) tau paid
// until the coupons reach the total (then paid - total and the note ends; the
// last period pays paid - total).  Returns flow1 + flow2.
template <class R>
R tarn_period(R f, R tau, int s, int n, R total, R strike, R mult, R& paid, bool& over) {
  if (over) return R(0);
  const R flow2 = tau * f;
  R flow1;
  if (s + 1 == n) {
    flow1 = paid - total;
    over = true;
  } else {
    R c = (strike - mult * f) * tau;
    if (c < R(0)) c = R(0);
    const R t = paid + c;
    if (t >= total) {
      flow1 = paid - total;
      over = true;
    } else {
      flow1 = -c;
      paid = t;
    }
  }
  return flow1 + flow2;
}

struct Spec {
  int n, F, P;            // rates (= steps), factors, paths
  uint32_t path_offset;   // Sobol point offset
  int scramble_dims;      // leading dims that are XOR-scrambled
  int product;            // Product
  double strike, pay_receive, cap_strike, cutoff;
  double tarn_total = 0, tarn_mult = 0;
  int n_ex;               // exercise dates (steps)
  int K;                  // basis functions
  int normalise;
};

// Per-path evolution and per-step products shared by the first and second
// passes.  Writes per exercise date: vars[e][3], ex[e], cf[e] (deflated to
// the exercise time), num[e]; and for the European product the per-path
// discounted payoff.
template <class R>
struct Evolver {
  const Spec& sp;
  const uint32_t* dirs;
  const uint32_t* scr;
  const R* A;        // [S][n][F]
  const R* fixed;    // [S][n]
  const R* tau;
  const R* disp;
  const R* f0;
  const R* lf0;
  const int* ex_steps;  // [n_ex]
  std::vector<int> alloc;
  Bridge<R> bridge;
  Evolver(const Spec& s, const uint32_t* d, const uint32_t* sc, const R* a,
          const R* fx, const R* t, const R* dp, const R* f, const R* l,
          const int* ex)
      : sp(s), dirs(d), scr(sc), A(a), fixed(fx), tau(t), disp(dp), f0(f),
        lf0(l), ex_steps(ex), alloc(s.F * s.n), bridge(s.n) {
    alloc_diagonal(sp.F, sp.n, alloc.data());
  }

  // increments[s][f] for path p.
  void variates(int p, std::vector<R>& inc) const {
    const int S = sp.n, F = sp.F;
    std::vector<R> z(S), w(S), o(S);
    inc.assign((size_t)S * F, R(0));
    const uint32_t n = sp.path_offset + 1u + (uint32_t)p;
    for (int f = 0; f < F; ++f) {
      for (int i = 0; i < S; ++i) {
        const int d = alloc[f * S + i];
        uint32_t x = sobol_point(dirs + 32 * (size_t)d, n);
        if (d < sp.scramble_dims) x ^= scr[d];
        z[i] = sizeof(R) == 4 ? (R)icdf_f_tails(x) : (R)icdf_d(x);
      }
      bridge.path(z.data(), w.data(), o.data());
      for (int s = 0; s < S; ++s) inc[(size_t)s * F + f] = o[s];
    }
  }

  // Evolves path p; fills per-exercise-date outputs.  Returns the discounted
  // (by numeraire, units of the T_0 numeraire) payoff of the European
  // product or the TARN, the cap strip of the swaption-plus-cap portfolio,
  // or 0.
  R path(int p, R* vars, R* exv, R* cf, R* num, R* rates_sn = nullptr) const {
    const int S = sp.n, n = sp.n, F = sp.F;
    std::vector<R> inc, f(f0, f0 + n), lf(lf0, lf0 + n), mu(n), mup(n),
        corr(n), P(n + 1);
    variates(p, inc);
    R N = 1, payoff = 0;
    int e = 0;
    R tarn_paid = 0;
    bool tarn_over = false;
    for (int s = 0; s < S; ++s) {
      if (s > 0) N = N * (R(1) + tau[s - 1] * f[s - 1]);
      const R* As = A + (size_t)s * n * F;
      for (int r = 0; r < n; ++r) {
        R x = 0;
        for (int k = 0; k < F; ++k) x += As[r * F + k] * inc[(size_t)s * F + k];
        corr[r] = x + fixed[s * n + r];
      }
      pc_step(As, corr.data(), tau, disp, n, F, (R)sp.cutoff, f.data(),
              lf.data(), mu.data(), mup.data());
      if (rates_sn)
        for (int r = 0; r < n; ++r) rates_sn[(size_t)s * n + r] = f[r];
      // discount ratios P(T_s, T_r), r >= s
      P[s] = 1;
      for (int r = s; r < n; ++r) P[r + 1] = P[r] / (R(1) + tau[r] * f[r]);
      if (sp.product == kTarn) {
        // TARN period (TARN_gold::getCashFlows, accruals = tau), paid at T_{s+1}
        payoff += tarn_period<R>(f[s], tau[s], s, n, (R)sp.tarn_total, (R)sp.strike,
                                 (R)sp.tarn_mult, tarn_paid, tarn_over) *
                  P[s + 1] / N;
        continue;
      }
      if (sp.product == kEuropean) {
        // caplet on f_s plus a payer swaplet, paid at T_{s+1}
        const R cap = tau[s] * std::max(f[s] - (R)sp.cap_strike, R(0));
        const R swp = tau[s] * (f[s] - (R)sp.strike) * (R)sp.pay_receive;
        payoff += (cap + swp) * P[s + 1] / N;
        continue;
      }
      if (sp.product == kBermudanCap) {
        // the portfolio's caplet on f_s, paid at T_{s+1}
        payoff += tau[s] * std::max(f[s] - (R)sp.cap_strike, R(0)) * P[s + 1] / N;
      }
      if (e < sp.n_ex && ex_steps[e] == s) {
        R ann = 0;
        for (int r = n - 1; r >= s; --r) ann += tau[r] * P[r + 1];
        const R sr = (P[s] - P[n]) / ann;
        R v1 = f[s], v2 = sr, v3 = ann;
        R x = 0, c = 0;
        if (sp.product == kSwaption || sp.product == kBermudanCap) {
          x = (sr - (R)sp.strike) * ann;
          if (x < 0) x = 0;
        } else {  // cancellable payer swap: coupon of this period
          const int j = std::min(s + 1, n - 1);
          R ann2 = 0;
          for (int r = n - 1; r >= j; --r) ann2 += tau[r] * P[r + 1];
          v2 = (P[j] - P[n]) / ann2;
          v3 = tau[n - 1] * P[n];
          c = tau[s] * (f[s] - (R)sp.strike) * (R)sp.pay_receive * P[s + 1];
        }
        vars[(size_t)e * 3 + 0] = v1;
        vars[(size_t)e * 3 + 1] = v2;
        vars[(size_t)e * 3 + 2] = v3;
        exv[e] = x;
        cf[e] = c;
        num[e] = N;
        ++e;
      }
    }
    return payoff;
  }
};

template <class R>
void basis_eval(const R* x, int nvars, const uint8_t* mono, int K, R* phi) {
  for (int k = 0; k < K; ++k) {
    R v = 1;
    for (int j = 0; j < nvars && j < 3; ++j)
      for (int t = 0; t < mono[k * 3 + j]; ++t) v *= x[j];
    phi[k] = v;
  }
}

// Symmetric positive definite solve by Cholesky with the same jitter policy
// as the device solver; falls back to zeros.
void chol_solve(std::vector<double> G, std::vector<double> b, int K,
                double* beta) {
  double maxd = 0;
  for (int i = 0; i < K; ++i) maxd = std::max(maxd, std::fabs(G[i * K + i]));
  for (int k = 0; k < K; ++k) beta[k] = 0;
  if (!(maxd > 0)) return;
  std::vector<double> L(K * K, 0.0);
  double jitter = 0;
  bool ok = false;
  for (int att = 0; att < 6 && !ok; ++att) {
    ok = true;
    for (int i = 0; i < K && ok; ++i)
      for (int j = 0; j <= i; ++j) {
        double s = G[i * K + j] + (i == j ? jitter : 0.0);
        for (int k = 0; k < j; ++k) s -= L[i * K + k] * L[j * K + k];
        if (i == j) {
          if (!(s > 1e-300)) {
            ok = false;
            break;
          }
          L[i * K + i] = std::sqrt(s);
        } else
          L[i * K + j] = s / L[j * K + j];
      }
    if (!ok) jitter = jitter == 0 ? 1e-14 * maxd : jitter * 100;
  }
  if (!ok) return;
  std::vector<double> z(K);
  for (int i = 0; i < K; ++i) {
    double s = b[i];
    for (int k = 0; k < i; ++k) s -= L[i * K + k] * z[k];
    z[i] = s / L[i * K + i];
  }
  for (int i = K - 1; i >= 0; --i) {
    double s = z[i];
    for (int k = i + 1; k < K; ++k) s -= L[k * K + i] * beta[k];
    beta[i] = s / L[i * K + i];
  }
}

// Backward LS at depth 1 (gold/MultiLS_regression.cpp:101-417 with the
// regression matrix of gold/LS_regression.h:431-530): R is the type of the
// stored path data; sums and the solve are FP64.  vars [E][3][P], beta
// [E][16].  Returns mean_p y_p / N_0(p).
template <class R>
double ls_regress(int E, int P, const R* vars, const int* nvars,
                  const uint8_t* mono /*[E][16][3]*/, const int* nbasis,
                  const R* cf, const R* ex, const R* num, int normalise,
                  double* beta, double* means, double* sds, double* gram) {
  std::vector<double> y(P, 0.0);
  std::vector<double> phi(16), x(3);
  for (int e = E - 1; e >= 0; --e) {
    const int K = nbasis[e], V = nvars[e];
    double m[3] = {0, 0, 0}, sd[3] = {1, 1, 1};
    if (normalise) {
      for (int v = 0; v < V; ++v) {
        double s = 0, s2 = 0;
        for (int p = 0; p < P; ++p) {
          const double t = vars[((size_t)e * 3 + v) * P + p];
          s += t;
          s2 += t * t;
        }
        m[v] = s / P;
        double var = s2 / P - m[v] * m[v];
        sd[v] = var > 0 ? std::sqrt(var) : 1.0;
      }
    }
    for (int v = 0; v < 3; ++v) {
      if (means) means[e * 3 + v] = m[v];
      if (sds) sds[e * 3 + v] = sd[v];
    }
    std::vector<double> G(K * K, 0.0), b(K, 0.0);
    for (int p = 0; p < P; ++p) {
      for (int v = 0; v < 3; ++v)
        x[v] = v < V ? (vars[((size_t)e * 3 + v) * P + p] - m[v]) / sd[v] : 0.0;
      basis_eval<double>(x.data(), V, mono + (size_t)e * 48, K, phi.data());
      const double t = (cf ? (double)cf[(size_t)e * P + p] : 0.0) + y[p];
      for (int i = 0; i < K; ++i) {
        for (int j = 0; j <= i; ++j) G[i * K + j] += phi[i] * phi[j];
        b[i] += t * phi[i];
      }
    }
    for (int i = 0; i < K; ++i) {
      b[i] /= P;
      for (int j = 0; j <= i; ++j) {
        G[i * K + j] /= P;
        G[j * K + i] = G[i * K + j];
      }
    }
    if (gram)
      for (int i = 0; i < K; ++i) {
        for (int j = 0; j < K; ++j) gram[(size_t)e * 272 + i * 17 + j] = G[i * K + j];
        gram[(size_t)e * 272 + i * 17 + K] = b[i];
      }
    double* be = beta + e * 16;
    chol_solve(G, b, K, be);
    for (int k = K; k < 16; ++k) be[k] = 0;
    for (int p = 0; p < P; ++p) {
      for (int v = 0; v < 3; ++v)
        x[v] = v < V ? (vars[((size_t)e * 3 + v) * P + p] - m[v]) / sd[v] : 0.0;
      basis_eval<double>(x.data(), V, mono + (size_t)e * 48, K, phi.data());
      double est = 0;
      for (int k = 0; k < K; ++k) est += phi[k] * be[k];
      const double exv = ex ? (double)ex[(size_t)e * P + p] : 0.0;
      if (exv > est)
        y[p] = exv;
      else
        y[p] += cf ? (double)cf[(size_t)e * P + p] : 0.0;
      if (e > 0) y[p] *= (double)num[(size_t)(e - 1) * P + p] / (double)num[(size_t)e * P + p];
    }
  }
  double res = 0;
  for (int p = 0; p < P; ++p) res += y[p] / (double)num[p];
  return res / P;
}

// Second pass with a frozen rule: per path, walk the exercise dates; stop at
// the first date where the exercise value exceeds the estimated
// continuation (MultiLSExerciseStrategy::decide and
// SecondPassPriceLSAMultiUsingAggregatedFlows_gold,
// gold/MultiLS_regression.h:190-289, regression depth 1).
template <class R>
double second_pass_path(int E, const R* vars, const int* nvars,
                        const uint8_t* mono, const int* nbasis, const R* cf,
                        const R* ex, const R* num, const double* beta,
                        const double* means, const double* sds) {
  double total = 0;
  double x[3], phi[16];
  for (int e = 0; e < E; ++e) {
    const int K = nbasis[e], V = nvars[e];
    for (int v = 0; v < 3; ++v)
      x[v] = v < V ? ((double)vars[e * 3 + v] - (means ? means[e * 3 + v] : 0.0)) /
                         (sds ? sds[e * 3 + v] : 1.0)
                   : 0.0;
    basis_eval<double>(x, V, mono + (size_t)e * 48, K, phi);
    double est = 0;
    for (int k = 0; k < K; ++k) est += phi[k] * beta[e * 16 + k];
    const double exv = (double)ex[e];
    if (exv > est) {
      total += exv / (double)num[e];
      return total;
    }
    total += (double)cf[e] / (double)num[e];
  }
  return total;
}

// --- regression at depth > 1 --------------------------------------------
// Nested regressions with path selection (generateRegressionCoefficientsVia
// LSMulti_gold, gold/MultiLS_regression.cpp:101-417): at each exercise date
// the depth-0 regression runs over all paths; the paths whose net
// continuation value (estimate minus exercise value) lies within a cut
// [-c, c] chosen by the fraction selector are regressed again, and so on up
// to D regressions.  The decision walks the chain: it moves to depth d + 1
// while the net value at depth d lies strictly inside that depth's cuts
// (updateDeflatedNextStepValuesMulti_gold and MultiLSExerciseStrategy::
// decide, gold/MultiLS_regression.h:42-99, 190-231).

struct SelectOpts {
  double lower_frac, upper_frac, sds, multiplier;
  int min_paths;
};

// Status bit: a cut-off search stopped at its evaluation limit.
constexpr int kSelectCapped = 8;
// Count evaluations allowed per search.  The reference's loops are
// unbounded and do not end when more than the upper target of net values
// are exactly zero; here the search keeps its current cut-off instead.
constexpr int kSelectMaxCounts = 512;

// Fraction selector (RegressionSelector_gold_Fraction::Select,
// gold/Regression_Selector_concrete_gold.cpp:58-205): with n preselected
// paths the targets are floor(n * lower_frac) and floor(n * upper_frac); the
// half-width starts at `sds` standard deviations of the net values, grows by
// 1 / multiplier until at least the lower target lies within it, shrinks by
// multiplier while more than the upper target do, then bisects to 1e-6.
// Returns the paths selected (pre[p] and |net[p]| <= cut) and the cut.
int frac_select(const SelectOpts& o, const std::vector<double>& net,
                const std::vector<uint8_t>& pre, int n_pre, double* cut, int* status) {
  const int P = (int)net.size();
  int evals = 0;
  auto count = [&](double g) {
    ++evals;
    int c = 0;
    for (int p = 0; p < P; ++p)
      if (pre[p] && net[p] >= -g && net[p] <= g) ++c;
    return c;
  };
  auto capped = [&]() {
    if (evals < kSelectMaxCounts) return false;
    *status |= kSelectCapped;
    return true;
  };
  const int lo_t = (int)(n_pre * o.lower_frac), hi_t = (int)(n_pre * o.upper_frac);
  if (n_pre > lo_t && n_pre < hi_t) {
    *cut = 1e4;
    return count(*cut);
  }
  double s1 = 0, s2 = 0;
  for (int p = 0; p < P; ++p)
    if (pre[p]) {
      s1 += net[p];
      s2 += net[p] * net[p];
    }
  const double mean = s1 / n_pre;
  double g = std::sqrt(s2 / n_pre - mean * mean) * o.sds;
  int c = count(g);
  while (c < lo_t && !capped()) {
    g /= o.multiplier;
    c = count(g);
  }
  if (c < hi_t) {
    *cut = g;
    return c;
  }
  double lo = g * o.multiplier;
  c = count(lo);
  while (c > hi_t && !capped()) {
    lo *= o.multiplier;
    c = count(lo);
  }
  if (c > lo_t) {
    *cut = lo;
    return c;
  }
  double hi = g;
  g = 0.5 * (lo + hi);
  c = count(g);
  while ((c < lo_t || c > hi_t) && (hi - lo) > 1e-6 && !capped()) {
    if (c < lo_t)
      lo = g;
    else
      hi = g;
    g = 0.5 * (lo + hi);
    c = count(g);
  }
  *cut = g;
  return c;
}

// A frozen exercise rule at depth D: beta [E][D][16], means / sds [E][D][3]
// (null: raw variables), cuts [E][D][2] (lower, upper; null at D = 1),
// shifts [E] (Andersen shifts added to every estimate; null: none).
struct MultiRule {
  int D;
  const double* beta;
  const double* means;
  const double* sds;
  const double* cuts;
  const double* shifts;
};

// Continuation estimate at date e by the depth chain; x_raw: the date's
// basis variables.
double chain_estimate(const MultiRule& r, int e, const double* x_raw, int V,
                      const uint8_t* mono_e, int K, double exv) {
  double est = 0, x[3], phi[16];
  for (int d = 0; d < r.D; ++d) {
    const size_t md = ((size_t)e * r.D + d) * 3;
    for (int v = 0; v < 3; ++v)
      x[v] = v < V ? (x_raw[v] - (r.means ? r.means[md + v] : 0.0)) /
                         (r.sds ? r.sds[md + v] : 1.0)
                   : 0.0;
    basis_eval<double>(x, V, mono_e, K, phi);
    est = r.shifts ? r.shifts[e] : 0.0;
    const double* b = r.beta + ((size_t)e * r.D + d) * 16;
    for (int k = 0; k < K; ++k) est += phi[k] * b[k];
    if (d + 1 >= r.D || !r.cuts) break;
    const double net = est - exv;
    const double* c = r.cuts + ((size_t)e * r.D + d) * 2;
    if (!(net > c[0] && net < c[1])) break;
  }
  return est;
}

// Backward LS with nested regressions.  Layouts as MultiRule; the cuts of
// the last depth are never read and stay zero.  Returns mean_p y_p / N_0(p).
template <class R>
double ls_regress_multi(int E, int P, const R* vars, const int* nvars,
                        const uint8_t* mono, const int* nbasis, const R* cf,
                        const R* ex, const R* num, int normalise, int D,
                        const SelectOpts& o, double* beta, double* means, double* sds,
                        double* cuts, int* status) {
  std::vector<double> y(P, 0.0), net(P, 0.0);
  std::vector<uint8_t> pre(P), sel(P);
  std::vector<double> phi(16), x(3);
  std::fill(beta, beta + (size_t)E * D * 16, 0.0);
  std::fill(cuts, cuts + (size_t)E * D * 2, 0.0);
  MultiRule rule{D, beta, means, sds, cuts, nullptr};
  for (int e = E - 1; e >= 0; --e) {
    const int K = nbasis[e], V = nvars[e];
    const uint8_t* mono_e = mono + (size_t)e * 48;
    std::fill(pre.begin(), pre.end(), 1);
    int n_pre = P;
    for (int d = 0; d < D; ++d) {
      const size_t md = ((size_t)e * D + d) * 3;
      double m[3] = {0, 0, 0}, sd[3] = {1, 1, 1};
      if (normalise)
        for (int v = 0; v < V; ++v) {
          double s1 = 0, s2 = 0;
          for (int p = 0; p < P; ++p)
            if (pre[p]) {
              const double t = vars[((size_t)e * 3 + v) * P + p];
              s1 += t;
              s2 += t * t;
            }
          m[v] = s1 / n_pre;
          const double var = s2 / n_pre - m[v] * m[v];
          sd[v] = var > 0 ? std::sqrt(var) : 1.0;
        }
      for (int v = 0; v < 3; ++v) {
        means[md + v] = m[v];
        sds[md + v] = sd[v];
      }
      std::vector<double> G(K * K, 0.0), b(K, 0.0);
      for (int p = 0; p < P; ++p) {
        if (!pre[p]) continue;
        for (int v = 0; v < 3; ++v)
          x[v] = v < V ? (vars[((size_t)e * 3 + v) * P + p] - m[v]) / sd[v] : 0.0;
        basis_eval<double>(x.data(), V, mono_e, K, phi.data());
        const double t = (cf ? (double)cf[(size_t)e * P + p] : 0.0) + y[p];
        for (int i = 0; i < K; ++i) {
          for (int j = 0; j <= i; ++j) G[i * K + j] += phi[i] * phi[j];
          b[i] += t * phi[i];
        }
      }
      for (int i = 0; i < K; ++i) {
        b[i] /= n_pre;
        for (int j = 0; j <= i; ++j) {
          G[i * K + j] /= n_pre;
          G[j * K + i] = G[i * K + j];
        }
      }
      double* be = beta + ((size_t)e * D + d) * 16;
      chol_solve(G, b, K, be);
      if (d + 1 == D) break;
      // net continuation values of the selected paths at this depth
      double nmax = -1e300, nmin = 1e300;
      for (int p = 0; p < P; ++p) {
        if (!pre[p]) continue;
        for (int v = 0; v < 3; ++v)
          x[v] = v < V ? (vars[((size_t)e * 3 + v) * P + p] - m[v]) / sd[v] : 0.0;
        basis_eval<double>(x.data(), V, mono_e, K, phi.data());
        double est = 0;
        for (int k = 0; k < K; ++k) est += phi[k] * be[k];
        net[p] = est - (ex ? (double)ex[(size_t)e * P + p] : 0.0);
        nmax = std::max(nmax, net[p]);
        nmin = std::min(nmin, net[p]);
      }
      // all net values of one sign: no nested regression at this date
      if (d == 0 && (nmax <= 0.0 || nmin >= 0.0)) break;
      double c = 0;
      const int after = frac_select(o, net, pre, n_pre, &c, status);
      if (after <= o.min_paths) break;
      cuts[((size_t)e * D + d) * 2 + 0] = -c;
      cuts[((size_t)e * D + d) * 2 + 1] = c;
      for (int p = 0; p < P; ++p) pre[p] = pre[p] && net[p] >= -c && net[p] <= c;
      n_pre = after;
    }
    double xr[3];
    for (int p = 0; p < P; ++p) {
      for (int v = 0; v < 3; ++v) xr[v] = v < V ? (double)vars[((size_t)e * 3 + v) * P + p] : 0.0;
      const double exv = ex ? (double)ex[(size_t)e * P + p] : 0.0;
      const double est = chain_estimate(rule, e, xr, V, mono_e, K, exv);
      if (exv > est)
        y[p] = exv;
      else
        y[p] += cf ? (double)cf[(size_t)e * P + p] : 0.0;
      if (e > 0) y[p] *= (double)num[(size_t)(e - 1) * P + p] / (double)num[(size_t)e * P + p];
    }
  }
  double res = 0;
  for (int p = 0; p < P; ++p) res += y[p] / (double)num[p];
  return res / P;
}

// Second pass of one path with a frozen depth-D rule
// (SecondPassPriceLSAMultiUsingAggregatedFlows_gold with
// MultiLSExerciseStrategy, gold/MultiLS_regression.h:190-289).
template <class R>
double second_pass_path_multi(int E, const R* vars, const int* nvars, const uint8_t* mono,
                              const int* nbasis, const R* cf, const R* ex, const R* num,
                              const MultiRule& rule) {
  double total = 0, xr[3];
  for (int e = 0; e < E; ++e) {
    const int V = nvars[e];
    for (int v = 0; v < 3; ++v) xr[v] = v < V ? (double)vars[e * 3 + v] : 0.0;
    const double exv = (double)ex[e];
    const double est = chain_estimate(rule, e, xr, V, mono + (size_t)e * 48, nbasis[e], exv);
    if (exv > est) return total + exv / (double)num[e];
    total += (double)cf[e] / (double)num[e];
  }
  return total;
}

// --- Andersen–Broadie duality gap ----------------------------------------
// ABDualityGapEstimateNonZeroRebate (root tree gold/Andersen_Broadie_gold.cpp:
// 121-187) and, with no payoffs, ABDualityGapEstimateZeroRebate (:59-119).
// ex [steps][paths] (the frozen rule's decision at every date, 0/1), payoffs
// [steps][paths] (deflated exercise values) or null, means [paths][steps]
// (continuation estimates from the inner simulations), is_ex [steps].
// Per path: the maximum over exercise dates of the payoff minus the
// martingale built from the continuation estimates, floored at zero; the
// result is the mean and standard error over paths.
void ab_gap(int steps, int paths, const int* ex, const double* payoffs, const double* means,
            const int* is_ex, double* out) {
  double total = 0, total_sq = 0;
  const int last = payoffs ? steps - 1 : steps;
  for (int p = 0; p < paths; ++p) {
    double best = 0, balance = 0;
    for (int s = 0; s < last; ++s) {
      if (!is_ex[s]) continue;
      const double z = payoffs ? payoffs[(size_t)s * paths + p] : 0.0;
      const double m = means[(size_t)p * steps + s];
      double x;
      if (ex[(size_t)s * paths + p] == 1) {
        x = -balance;
        balance += z - m;
      } else {
        x = z - m - balance;
      }
      best = std::max(best, x);
    }
    best = std::max(best, -balance);
    total += best;
    total_sq += best * best;
  }
  const double mean = total / paths;
  out[0] = mean;
  out[1] = std::sqrt((total_sq / paths - mean * mean) / paths);
}

// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror and Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC 2011): ten rounds of two
// 32x32 -> 64-bit multiplications with a Weyl-sequence key schedule.
inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int round = 0; round < 10; ++round) {
    if (round) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint64_t a = (uint64_t)0xD2511F53u * c[0];
    const uint64_t b = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t n0 = (uint32_t)(b >> 32) ^ c[1] ^ k0;
    const uint32_t n2 = (uint32_t)(a >> 32) ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = (uint32_t)b;
    c[2] = n2;
    c[3] = (uint32_t)a;
  }
}

// Normal increment of factor f at step s for inner path i of outer path p
// and exercise date e: Philox on the counter (i, p, 4s + f/4, e) with key
// (seed low, seed high), word f % 4, through the exact-tail inverse normal.
template <class R>
R inner_normal(uint64_t seed, int i, int p, int s, int f, int e) {
  uint32_t c[4] = {(uint32_t)i, (uint32_t)p, (uint32_t)(4 * s + f / 4), (uint32_t)e};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const uint32_t u = c[f % 4];
  return sizeof(R) == 4 ? (R)icdf_f_tails(u) : (R)icdf_d(u);
}

// Inner path of an Andersen–Broadie sub-simulation (Bermudan swaption):
// from the state at the start of step s0 (log-rates lf_start[r], r >= s0,
// numeraire N0), evolve steps s0..n-1 with increments z(s, f) and stop at
// the first exercise date where the frozen rule exercises; returns the
// exercise value deflated by the path's numeraire (0 if never).  As
// Evolver::path from step s0 on.
template <class R, class Normals>
double inner_path(const Evolver<R>& ev, int s0, const R* lf_start, R N0, Normals z,
                  const MultiRule& rule, const int* nvars, const uint8_t* mono,
                  const int* nbasis) {
  const Spec& sp = ev.sp;
  const int n = sp.n, F = sp.F;
  std::vector<R> f(n, R(0)), lf(n, R(0)), mu(n), mup(n), corr(n), P(n + 1), zs(F);
  for (int r = s0; r < n; ++r) {
    lf[r] = lf_start[r];
    f[r] = std::exp(lf[r]) - ev.disp[r];
  }
  R N = N0;
  int e = 0;
  while (e < sp.n_ex && ev.ex_steps[e] < s0) ++e;
  for (int s = s0; s < n; ++s) {
    if (s > s0) N = N * (R(1) + ev.tau[s - 1] * f[s - 1]);
    for (int k = 0; k < F; ++k) zs[k] = z(s, k);
    const R* As = ev.A + (size_t)s * n * F;
    for (int r = 0; r < n; ++r) {
      R x = 0;
      for (int k = 0; k < F; ++k) x += As[r * F + k] * zs[k];
      corr[r] = x + ev.fixed[s * n + r];
    }
    pc_step(As, corr.data(), ev.tau, ev.disp, n, F, (R)sp.cutoff, f.data(), lf.data(),
            mu.data(), mup.data());
    P[s] = 1;
    for (int r = s; r < n; ++r) P[r + 1] = P[r] / (R(1) + ev.tau[r] * f[r]);
    if (e < sp.n_ex && ev.ex_steps[e] == s) {
      R ann = 0;
      for (int r = n - 1; r >= s; --r) ann += ev.tau[r] * P[r + 1];
      const R sr = (P[s] - P[n]) / ann;
      R x = (sr - (R)sp.strike) * ann;
      if (x < 0) x = 0;
      const double xr[3] = {(double)f[s], (double)sr, (double)ann};
      const double est = chain_estimate(rule, e, xr, nvars[e], mono + (size_t)e * 48,
                                        nbasis[e], (double)x);
      if ((double)x > est) return (double)x / (double)N;
      ++e;
    }
  }
  return 0.0;
}

template <class R>
struct PipelineIO {
  const uint32_t* dirs;
  const uint32_t* scr;
  const R* A;
  const R* fixed;
  const R* tau;
  const R* disp;
  const R* f0;
  const R* lf0;
  const int* ex_steps;
  const int* nvars;
  const uint8_t* mono;
  const int* nbasis;
};

}  // namespace

// ===================== extern "C" surface ==================================

ORC void orc_sobol_directions(int dims, const uint32_t* degree,
                              const uint32_t* a, const uint32_t* m,
                              int mstride, uint32_t* out) {
  directions(dims, degree, a, m, mstride, out);
}

ORC void orc_sobol_ints(int paths, int dims, uint32_t offset,
                        const uint32_t* dirs, uint32_t* out) {
  for (int d = 0; d < dims; ++d)
    for (int p = 0; p < paths; ++p)
      out[(size_t)d * paths + p] = sobol_point(dirs + 32 * (size_t)d, offset + 1u + (uint32_t)p);
}

// scramble_gold (gold/scramble_gold.cpp:11-27)
ORC void orc_scramble(uint32_t* data, const uint32_t* scr, int dims, int paths) {
  for (int d = 0; d < dims; ++d)
    for (int p = 0; p < paths; ++p) data[(size_t)d * paths + p] ^= scr[d];
}

ORC void orc_icdf_f(const uint32_t* in, float* out, long n) {
  for (long i = 0; i < n; ++i) out[i] = icdf_f(in[i]);
}
ORC void orc_icdf_tails_f(const uint32_t* in, float* out, long n) {
  for (long i = 0; i < n; ++i) out[i] = icdf_f_tails(in[i]);
}
ORC void orc_icdf_d(const uint32_t* in, double* out, long n) {
  for (long i = 0; i < n; ++i) out[i] = icdf_d(in[i]);
}

ORC void orc_bridge_allocate_diagonal(int F, int S, int* idx) {
  alloc_diagonal(F, S, idx);
}

// brownian_bridge::transformCPU (brownian_bridge.cu:401-455): in [F*S][P],
// out [S][F][P]; alloc NULL = diagonal.
template <class R>
static void bridge_t(const R* in, R* out, int P, int S, int F, const int* alloc) {
  std::vector<int> al(F * S);
  if (alloc)
    std::copy(alloc, alloc + F * S, al.begin());
  else
    alloc_diagonal(F, S, al.data());
  Bridge<R> b(S);
  std::vector<R> z(S), w(S), o(S);
  for (int p = 0; p < P; ++p)
    for (int f = 0; f < F; ++f) {
      for (int i = 0; i < S; ++i) z[i] = in[(size_t)al[f * S + i] * P + p];
      b.path(z.data(), w.data(), o.data());
      for (int s = 0; s < S; ++s) out[((size_t)s * F + f) * P + p] = o[s];
    }
}
ORC void orc_bridge_f(const float* in, float* out, int P, int S, int F, const int* alloc) {
  bridge_t<float>(in, out, P, S, F, alloc);
}
ORC void orc_bridge_d(const double* in, double* out, int P, int S, int F, const int* alloc) {
  bridge_t<double>(in, out, P, S, F, alloc);
}

// correlate_drift_paths_gold (gold/correlate_drift_gold.h:22-60); layout 0:
// in [S][P][F], 1: in [S][F][P]; writes every rate.
ORC void orc_correlate_drift_f(const float* in, float* out, const float* A,
                               int A_step, const float* drift, int F, int n,
                               int P, int S, int layout) {
  for (int s = 0; s < S; ++s)
    for (int p = 0; p < P; ++p)
      for (int r = 0; r < n; ++r) {
        float t = 0;
        for (int f = 0; f < F; ++f) {
          const float z = layout == 0 ? in[((size_t)s * P + p) * F + f]
                                      : in[((size_t)s * F + f) * P + p];
          t += A[(size_t)s * A_step + r * F + f] * z;
        }
        t += drift[s * n + r];
        out[((size_t)s * n + r) * P + p] = t;
      }
}

// LMM_evolver_pc_gold (gold/LMM_evolver_gold.h:391-455)
template <class R>
static void pc_t(const R* f0, const R* tau, const R* corr, const R* A,
                 const R* disp, int P, int F, int S, int n, R cutoff, R* ro,
                 R* lo) {
  std::vector<R> f(n), lf(n), mu(n), mup(n), c(n);
  for (int p = 0; p < P; ++p) {
    for (int r = 0; r < n; ++r) {
      f[r] = f0[r];
      lf[r] = std::log(f0[r] + disp[r]);
    }
    for (int s = 0; s < S; ++s) {
      for (int r = 0; r < n; ++r) c[r] = corr[((size_t)s * n + r) * P + p];
      pc_step(A + (size_t)s * n * F, c.data(), tau, disp, n, F, cutoff, f.data(),
              lf.data(), mu.data(), mup.data());
      for (int r = 0; r < n; ++r) {
        ro[((size_t)s * n + r) * P + p] = f[r];
        lo[((size_t)s * n + r) * P + p] = lf[r];
      }
    }
  }
}
ORC void orc_pc_f(const float* f0, const float* tau, const float* corr,
                  const float* A, const float* disp, int P, int F, int S,
                  int n, float cutoff, float* ro, float* lo) {
  pc_t<float>(f0, tau, corr, A, disp, P, F, S, n, cutoff, ro, lo);
}
ORC void orc_pc_d(const double* f0, const double* tau, const double* corr,
                  const double* A, const double* disp, int P, int F, int S,
                  int n, double cutoff, double* ro, double* lo) {
  pc_t<double>(f0, tau, corr, A, disp, P, F, S, n, cutoff, ro, lo);
}

// spotDriftComputer::getDrifts (gold/LMM_evolver_gold.h:178-203)
ORC void orc_spot_drift_d(const double* A, const double* f, const double* tau,
                          const double* disp, int n, int F, double* mu) {
  spot_drift<double>(A, f, tau, disp, n, F, mu);
}

// discount ratios / annuities / swap rates / numeraires
// (gold/LMM_evolver_gold.h:460-553,617-666)
ORC void orc_discount_ratios_f(const float* fr, const float* tau,
                               const int* alive, int P, int S, int n,
                               float* out) {
  for (int s = 0; s < S; ++s)
    for (int p = 0; p < P; ++p) {
      float df = 1;
      out[((size_t)s * (n + 1) + alive[s]) * P + p] = df;
      for (int r = alive[s]; r < n; ++r) {
        df /= 1 + tau[r] * fr[((size_t)s * n + r) * P + p];
        out[((size_t)s * (n + 1) + r + 1) * P + p] = df;
      }
    }
}
ORC void orc_annuities_f(const float* disc, const float* tau, const int* alive,
                         int P, int S, int n, float* out) {
  for (int s = 0; s < S; ++s)
    for (int p = 0; p < P; ++p) {
      float a = 0;
      for (int r = n - 1; r >= alive[s]; --r) {
        a += tau[r] * disc[((size_t)s * (n + 1) + r + 1) * P + p];
        out[((size_t)s * n + r) * P + p] = a;
      }
    }
}
ORC void orc_swap_rates_f(const float* disc, const float* ann, const int* alive,
                          int P, int S, int n, float* out) {
  for (int s = 0; s < S; ++s)
    for (int p = 0; p < P; ++p)
      for (int r = alive[s]; r < n; ++r)
        out[((size_t)s * n + r) * P + p] =
            (disc[((size_t)s * (n + 1) + r) * P + p] -
             disc[((size_t)s * (n + 1) + n) * P + p]) /
            ann[((size_t)s * n + r) * P + p];
}
ORC void orc_numeraires_f(const float* disc, int P, int n, float* out) {
  for (int p = 0; p < P; ++p) {
    out[p] = 1;
    for (int r = 1; r < n; ++r)
      out[(size_t)r * P + p] = out[(size_t)(r - 1) * P + p] *
                               disc[((size_t)(r - 1) * (n + 1) + r - 1) * P + p] /
                               disc[((size_t)(r - 1) * (n + 1) + r) * P + p];
  }
}

// cashFlowDiscounting_gold (gold/cashFlowDiscounting_gold.h:20-92)
ORC void orc_discounting_f(const int* first, const int* second,
                           const float* theta, const float* disc,
                           const float* flows, const float* num, int P, int S,
                           float* out, float* summed) {
  for (int p = 0; p < P; ++p) {
    float total = 0;
    for (int s = 0; s < S; ++s) {
      const float b = disc[((size_t)s * (S + 1) + s) * P + p];
      const float r1 = disc[((size_t)s * (S + 1) + first[s]) * P + p] / b;
      const float r2 = disc[((size_t)s * (S + 1) + second[s]) * P + p] / b;
      const float df = std::pow(r1, 1.0f - theta[s]) * std::pow(r2, theta[s]);
      float cf = flows[(size_t)s * P + p] * df;
      cf /= num[(size_t)s * P + p];
      out[(size_t)s * P + p] = cf;
      total += cf;
    }
    summed[p] = total;
  }
}

// adjoinExerciseValues_Bermudan_swaption_gold value max((SR-K)A, 0)
// (gold/early_exercise_value_generator_gold.h:93-130)
// TARN flows (cashFlowGeneratorCallerTARN_gold, gold/cashFlowGeneration_product_gold.h:
// 171; generator loop gold/cashFlowGeneration_gold.h:8-60): aux = {total, K, m,
// accruals1[steps], accruals2[steps]}; flows [steps][paths].
ORC void orc_tarn_flows_f(float* f1, float* f2, const float* aux, int paths, int steps,
                          const float* rate1, const float* rate2) {
  for (int p = 0; p < paths; ++p) {
    float paid = 0.0f;
    bool over = false;
    for (int i = 0; i < steps; ++i) {
      float a = 0.0f, b = 0.0f;
      if (!over) {
        b = aux[3 + steps + i] * rate2[(size_t)i * paths + p];
        if (i + 1 == steps) {
          a = paid - aux[0];
          over = true;
        } else {
          float c = (aux[1] - aux[2] * rate1[(size_t)i * paths + p]) * aux[3 + i];
          if (c < 0.0f) c = 0.0f;
          const float t = paid + c;
          if (t >= aux[0]) {
            a = paid - aux[0];
            over = true;
          } else {
            a = -c;
            paid = t;
          }
        }
      }
      f1[(size_t)i * paths + p] = a;
      f2[(size_t)i * paths + p] = b;
    }
  }
}

ORC void orc_payer_swaption_values_f(float K, const float* sr, const float* ann,
                                     int P, int E, float* out) {
  for (size_t i = 0; i < (size_t)P * E; ++i) {
    const float v = (sr[i] - K) * ann[i];
    out[i] = v > 0 ? v : 0;
  }
}

// Backward LS (double sums) on float or double data.
ORC double orc_ls_regress_f(int E, int P, const float* vars, const int* nvars,
                            const uint8_t* mono, const int* nbasis,
                            const float* cf, const float* ex, const float* num,
                            int normalise, double* beta, double* means,
                            double* sds, double* gram) {
  return ls_regress<float>(E, P, vars, nvars, mono, nbasis, cf, ex, num,
                           normalise, beta, means, sds, gram);
}
ORC double orc_ls_regress_d(int E, int P, const double* vars, const int* nvars,
                            const uint8_t* mono, const int* nbasis,
                            const double* cf, const double* ex,
                            const double* num, int normalise, double* beta,
                            double* means, double* sds, double* gram) {
  return ls_regress<double>(E, P, vars, nvars, mono, nbasis, cf, ex, num,
                            normalise, beta, means, sds, gram);
}

// Regression at depth D (ls_regress_multi).  opts = {lower_frac,
// upper_frac, sds, multiplier, min_paths}.  beta [E][D][16], means / sds
// [E][D][3], cuts [E][D][2]; status receives kSelectCapped when a cut-off
// search stopped at its limit.
#define MULTI_ARGS(R)                                                          \
  int E, int P, const R *vars, const int *nvars, const uint8_t *mono,          \
      const int *nbasis, const R *cf, const R *ex, const R *num, int normalise, \
      int D, const double *opts, double *beta, double *means, double *sds,     \
      double *cuts, int *status
ORC double orc_ls_regress_multi_f(MULTI_ARGS(float)) {
  const SelectOpts o{opts[0], opts[1], opts[2], opts[3], (int)opts[4]};
  return ls_regress_multi<float>(E, P, vars, nvars, mono, nbasis, cf, ex, num, normalise, D,
                                 o, beta, means, sds, cuts, status);
}
ORC double orc_ls_regress_multi_d(MULTI_ARGS(double)) {
  const SelectOpts o{opts[0], opts[1], opts[2], opts[3], (int)opts[4]};
  return ls_regress_multi<double>(E, P, vars, nvars, mono, nbasis, cf, ex, num, normalise, D,
                                  o, beta, means, sds, cuts, status);
}

// Andersen–Broadie duality gap (ab_gap); payoffs null = zero rebate.
ORC void orc_ab_gap(int steps, int paths, const int* ex, const double* payoffs,
                    const double* means, const int* is_ex, double* out) {
  ab_gap(steps, paths, ex, payoffs, means, is_ex, out);
}

ORC void orc_philox4x32_10(uint32_t* ctr, uint32_t k0, uint32_t k1, int n) {
  for (int i = 0; i < n; ++i) philox4x32_10(ctr + 4 * i, k0, k1);
}

// Continuation estimates of Andersen–Broadie outer paths (Bermudan payer
// swaption).  For outer path p and exercise date e (step s = ex_steps[e],
// e < E - 1): `inner` paths from the state at the start of step s + 1
// (lf_ckpt [n][n][K]: log-rates at the start of each step, numeraire
// N_ckpt [n][K]) with the Philox normals of inner_normal, priced with the
// frozen rule (depth, beta, means, sds, cuts; shifts null) from date e + 1.
// Q [E][K] = mean deflated value, se [E][K] its standard error; the last
// date has no continuation (0).  spec as orc_pipeline_*; rows e of Q and
// se with e < e_begin or e >= e_end are left untouched.
template <class R>
static void ab_inner_t(const int* si, const double* sd, const PipelineIO<R>& io, int depth,
                       const double* beta, const double* means, const double* sds,
                       const double* cuts, const R* lf_ckpt, const R* N_ckpt, int K, int inner,
                       uint64_t seed, int e_begin, int e_end, double* Q, double* se) {
  Spec sp;
  sp.n = si[0];
  sp.F = si[1];
  sp.P = si[2];
  sp.path_offset = (uint32_t)si[3];
  sp.scramble_dims = si[4];
  sp.product = si[5];
  sp.n_ex = si[6];
  sp.normalise = si[7];
  const int threads = std::max(1, si[8]);
  sp.strike = sd[0];
  sp.pay_receive = sd[1];
  sp.cap_strike = sd[2];
  sp.cutoff = sd[3];
  sp.K = 0;
  Evolver<R> ev(sp, io.dirs, io.scr, io.A, io.fixed, io.tau, io.disp, io.f0, io.lf0,
                io.ex_steps);
  const MultiRule rule{depth, beta, means, sds, cuts, nullptr};
  const int n = sp.n, E = sp.n_ex;
  auto work = [&](int lo, int hi) {
    std::vector<R> lfs(n);
    for (int job = lo; job < hi; ++job) {
      const int e = e_begin + job / K, p = job % K;
      double m = 0, m2 = 0;
      if (e + 1 < E) {
        const int s0 = io.ex_steps[e] + 1;
        for (int r = 0; r < n; ++r) lfs[r] = lf_ckpt[((size_t)s0 * n + r) * K + p];
        const R N0 = N_ckpt[(size_t)s0 * K + p];
        for (int i = 0; i < inner; ++i) {
          auto z = [&](int s, int f) { return inner_normal<R>(seed, i, p, s, f, e); };
          const double v = inner_path<R>(ev, s0, lfs.data(), N0, z, rule, io.nvars, io.mono,
                                         io.nbasis);
          m += v;
          m2 += v * v;
        }
        m /= inner;
        m2 = std::sqrt(std::max(0.0, m2 / inner - m * m) / inner);
      }
      Q[(size_t)e * K + p] = m;
      se[(size_t)e * K + p] = m2;
    }
  };
  const int jobs = (e_end - e_begin) * K;
  std::vector<std::thread> pool;
  const int chunk = (jobs + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    const int lo = t * chunk, hi = std::min(jobs, lo + chunk);
    if (lo < hi) pool.emplace_back(work, lo, hi);
  }
  for (auto& th : pool) th.join();
}

#define AB_ARGS(R)                                                                         \
  const int *si, const double *sd, const uint32_t *dirs, const uint32_t *scr, const R *A,  \
      const R *fixed, const R *tau, const R *disp, const R *f0, const R *lf0,              \
      const int *ex_steps, const int *nvars, const uint8_t *mono, const int *nbasis,       \
      int depth, const double *beta, const double *means, const double *sds,               \
      const double *cuts, const R *lf_ckpt, const R *N_ckpt, int K, int inner,             \
      uint64_t seed, int e_begin, int e_end, double *Q, double *se
ORC void orc_ab_inner_f(AB_ARGS(float)) {
  PipelineIO<float> io{dirs, scr, A, fixed, tau, disp, f0, lf0, ex_steps, nvars, mono, nbasis};
  ab_inner_t<float>(si, sd, io, depth, beta, means, sds, cuts, lf_ckpt, N_ckpt, K, inner, seed,
                    e_begin, e_end, Q, se);
}
ORC void orc_ab_inner_d(AB_ARGS(double)) {
  PipelineIO<double> io{dirs, scr, A, fixed, tau, disp, f0, lf0, ex_steps, nvars, mono, nbasis};
  ab_inner_t<double>(si, sd, io, depth, beta, means, sds, cuts, lf_ckpt, N_ckpt, K, inner,
                     seed, e_begin, e_end, Q, se);
}

// Mean second-pass value of stored paths (vars [E][3][P], cf / ex / num
// [E][P]) under a depth-D rule with Andersen shifts (null: none).
ORC double orc_ls_second_pass_multi_d(int E, int P, const double* vars, const int* nvars,
                                      const uint8_t* mono, const int* nbasis,
                                      const double* cf, const double* ex, const double* num,
                                      int D, const double* beta, const double* means,
                                      const double* sds, const double* cuts,
                                      const double* shifts) {
  const MultiRule rule{D, beta, means, sds, cuts, shifts};
  std::vector<double> v((size_t)E * 3), c(E), x(E), n(E);
  double total = 0;
  for (int p = 0; p < P; ++p) {
    for (int e = 0; e < E; ++e) {
      for (int k = 0; k < 3; ++k) v[e * 3 + k] = vars[((size_t)e * 3 + k) * P + p];
      c[e] = cf[(size_t)e * P + p];
      x[e] = ex[(size_t)e * P + p];
      n[e] = num[(size_t)e * P + p];
    }
    total += second_pass_path_multi<double>(E, v.data(), nvars, mono, nbasis, c.data(),
                                            x.data(), n.data(), rule);
  }
  return total / P;
}

// Whole-path pipeline.  spec_i = {n, F, P, path_offset, scramble_dims,
// product, n_ex, normalise, threads}; spec_d = {strike, pay_receive,
// cap_strike, cutoff}.  mode 0: evolve only, writing vars [E][3][P], ex, cf,
// num [E][P] (or, for the European product, payoff[P]).  mode 1: evolve and
// price with the frozen rule beta/means/sds, writing payoff[P] (units of the
// T_0 numeraire).  Paths are split over `threads` std::threads.
template <class R>
static void pipeline_t(const int* si, const double* sd, const PipelineIO<R>& io,
                       int mode, const double* beta, const double* means,
                       const double* sds, R* vars, R* ex, R* cf, R* num,
                       double* payoff, const MultiRule* multi = nullptr) {
  Spec sp;
  sp.n = si[0];
  sp.F = si[1];
  sp.P = si[2];
  sp.path_offset = (uint32_t)si[3];
  sp.scramble_dims = si[4];
  sp.product = si[5];
  sp.n_ex = si[6];
  sp.normalise = si[7];
  const int threads = std::max(1, si[8]);
  sp.strike = sd[0];
  sp.pay_receive = sd[1];
  sp.cap_strike = sd[2];
  sp.cutoff = sd[3];
  if (sp.product == kTarn) {
    sp.tarn_total = sd[4];
    sp.tarn_mult = sd[5];
  }
  sp.K = 0;
  Evolver<R> ev(sp, io.dirs, io.scr, io.A, io.fixed, io.tau, io.disp, io.f0,
                io.lf0, io.ex_steps);
  const int E = sp.n_ex, P = sp.P;
  auto work = [&](int lo, int hi) {
    std::vector<R> v((size_t)E * 3 + 3), x(E + 1), c(E + 1), nm(E + 1);
    for (int p = lo; p < hi; ++p) {
      const R pay = ev.path(p, v.data(), x.data(), c.data(), nm.data());
      if (sp.product == kEuropean || sp.product == kTarn) {
        if (payoff) payoff[p] = (double)pay;
        continue;
      }
      if (mode == 0) {
        for (int e = 0; e < E; ++e) {
          for (int k = 0; k < 3; ++k) vars[((size_t)e * 3 + k) * P + p] = v[e * 3 + k];
          ex[(size_t)e * P + p] = x[e];
          cf[(size_t)e * P + p] = c[e];
          num[(size_t)e * P + p] = nm[e];
        }
      } else if (multi) {
        payoff[p] = second_pass_path_multi<R>(E, v.data(), io.nvars, io.mono, io.nbasis,
                                              c.data(), x.data(), nm.data(), *multi);
      } else {
        payoff[p] = second_pass_path<R>(E, v.data(), io.nvars, io.mono, io.nbasis,
                                        c.data(), x.data(), nm.data(), beta,
                                        means, sds);
      }
      if (mode != 0 && sp.product == kBermudanCap) payoff[p] += (double)pay;
    }
  };
  std::vector<std::thread> pool;
  const int chunk = (P + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    const int lo = t * chunk, hi = std::min(P, lo + chunk);
    if (lo < hi) pool.emplace_back(work, lo, hi);
  }
  for (auto& th : pool) th.join();
}

#define PIPE_ARGS(R)                                                          \
  const int *si, const double *sd, const uint32_t *dirs, const uint32_t *scr, \
      const R *A, const R *fixed, const R *tau, const R *disp, const R *f0,   \
      const R *lf0, const int *ex_steps, const int *nvars,                    \
      const uint8_t *mono, const int *nbasis, int mode, const double *beta,   \
      const double *means, const double *sds, R *vars, R *ex, R *cf, R *num,  \
      double *payoff

ORC void orc_pipeline_f(PIPE_ARGS(float)) {
  PipelineIO<float> io{dirs, scr, A, fixed, tau, disp, f0, lf0, ex_steps, nvars, mono, nbasis};
  pipeline_t<float>(si, sd, io, mode, beta, means, sds, vars, ex, cf, num, payoff);
}
ORC void orc_pipeline_d(PIPE_ARGS(double)) {
  PipelineIO<double> io{dirs, scr, A, fixed, tau, disp, f0, lf0, ex_steps, nvars, mono, nbasis};
  pipeline_t<double>(si, sd, io, mode, beta, means, sds, vars, ex, cf, num, payoff);
}

// Second pass (mode 1) with a nested rule: depth rows per date, cuts
// [E][depth][2], Andersen shifts [E] (null: none); other arguments as
// orc_pipeline_*.
ORC void orc_pipeline_rule_f(PIPE_ARGS(float), int depth, const double* cuts,
                             const double* shifts) {
  PipelineIO<float> io{dirs, scr, A, fixed, tau, disp, f0, lf0, ex_steps, nvars, mono, nbasis};
  const MultiRule rule{depth, beta, means, sds, cuts, shifts};
  pipeline_t<float>(si, sd, io, mode, beta, means, sds, vars, ex, cf, num, payoff, &rule);
}
ORC void orc_pipeline_rule_d(PIPE_ARGS(double), int depth, const double* cuts,
                             const double* shifts) {
  PipelineIO<double> io{dirs, scr, A, fixed, tau, disp, f0, lf0, ex_steps, nvars, mono, nbasis};
  const MultiRule rule{depth, beta, means, sds, cuts, shifts};
  pipeline_t<double>(si, sd, io, mode, beta, means, sds, vars, ex, cf, num, payoff, &rule);
}

// Forward rates of every step along the pipeline's paths: rates_out
// [S][n][P] holds f_r after step s (rates r < s keep their last value);
// spec as orc_pipeline_* (the product fields are unused).
template <class R>
static void path_rates_t(const int* si, const double* sd, const PipelineIO<R>& io,
                         R* rates_out) {
  Spec sp;
  sp.n = si[0];
  sp.F = si[1];
  sp.P = si[2];
  sp.path_offset = (uint32_t)si[3];
  sp.scramble_dims = si[4];
  sp.product = kEuropean;
  sp.n_ex = 0;
  sp.normalise = 0;
  const int threads = std::max(1, si[8]);
  sp.strike = sd[0];
  sp.pay_receive = sd[1];
  sp.cap_strike = sd[2];
  sp.cutoff = sd[3];
  sp.K = 0;
  Evolver<R> ev(sp, io.dirs, io.scr, io.A, io.fixed, io.tau, io.disp, io.f0, io.lf0,
                io.ex_steps);
  const int n = sp.n, P = sp.P;
  auto work = [&](int lo, int hi) {
    std::vector<R> v(3), x(1), c(1), nm(1), fr((size_t)n * n);
    for (int p = lo; p < hi; ++p) {
      ev.path(p, v.data(), x.data(), c.data(), nm.data(), fr.data());
      for (size_t i = 0; i < fr.size(); ++i) rates_out[i * P + p] = fr[i];
    }
  };
  std::vector<std::thread> pool;
  const int chunk = (P + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    const int lo = t * chunk, hi = std::min(P, lo + chunk);
    if (lo < hi) pool.emplace_back(work, lo, hi);
  }
  for (auto& th : pool) th.join();
}

#define RATES_ARGS(R)                                                         \
  const int *si, const double *sd, const uint32_t *dirs, const uint32_t *scr, \
      const R *A, const R *fixed, const R *tau, const R *disp, const R *f0,   \
      const R *lf0, R *rates_out

ORC void orc_path_rates_f(RATES_ARGS(float)) {
  PipelineIO<float> io{dirs, scr, A, fixed, tau, disp, f0, lf0, nullptr, nullptr, nullptr,
                       nullptr};
  path_rates_t<float>(si, sd, io, rates_out);
}
ORC void orc_path_rates_d(RATES_ARGS(double)) {
  PipelineIO<double> io{dirs, scr, A, fixed, tau, disp, f0, lf0, nullptr, nullptr, nullptr,
                        nullptr};
  path_rates_t<double>(si, sd, io, rates_out);
}

// Frozen-exercise payoff (FP64 path): the path's flows up to its given
// exercise date ex_at[p] (an exercise index; n_ex = never), deflated by the
// numeraire: the function whose derivatives the pathwise adjoint computes.
// Central differences of this function on the same Sobol points are the
// reference for the adjoint Greeks.  Arguments as orc_pipeline_d.
ORC void orc_frozen_payoff_d(const int* si, const double* sd, const uint32_t* dirs,
                             const uint32_t* scr, const double* A, const double* fixed,
                             const double* tau, const double* disp, const double* f0,
                             const double* lf0, const int* ex_steps, const int* ex_at,
                             double* payoff) {
  Spec sp;
  sp.n = si[0];
  sp.F = si[1];
  sp.P = si[2];
  sp.path_offset = (uint32_t)si[3];
  sp.scramble_dims = si[4];
  sp.product = si[5];
  sp.n_ex = si[6];
  sp.normalise = si[7];
  const int threads = std::max(1, si[8]);
  sp.strike = sd[0];
  sp.pay_receive = sd[1];
  sp.cap_strike = sd[2];
  sp.cutoff = sd[3];
  sp.K = 0;
  Evolver<double> ev(sp, dirs, scr, A, fixed, tau, disp, f0, lf0, ex_steps);
  const int E = sp.n_ex, P = sp.P;
  auto work = [&](int lo, int hi) {
    std::vector<double> v((size_t)E * 3 + 3), x(E + 1), c(E + 1), nm(E + 1);
    for (int p = lo; p < hi; ++p) {
      const double pay = ev.path(p, v.data(), x.data(), c.data(), nm.data());
      if (sp.product == kEuropean || sp.product == kTarn) {
        payoff[p] = pay;
        continue;
      }
      double total = sp.product == kBermudanCap ? pay : 0.0;
      for (int e = 0; e < E; ++e) {
        if (e == ex_at[p]) {
          total += x[e] / nm[e];
          break;
        }
        total += c[e] / nm[e];
      }
      payoff[p] = total;
    }
  };
  std::vector<std::thread> pool;
  const int chunk = (P + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    const int lo = t * chunk, hi = std::min(P, lo + chunk);
    if (lo < hi) pool.emplace_back(work, lo, hi);
  }
  for (auto& th : pool) th.join();
}

// MT19937 (Matsumoto & Nishimura 1998; init_genrand seeding, seed 0 -> 1 as
// MersenneTwisterUniformRng::seedInitialization, gold/Mersenne_gold.cpp:51)
ORC void orc_mt19937(uint32_t seed, int n, uint32_t* out) {
  uint32_t mt[624];
  mt[0] = seed ? seed : 1u;
  for (int i = 1; i < 624; ++i)
    mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (uint32_t)i;
  int idx = 624;
  for (int k = 0; k < n; ++k) {
    if (idx >= 624) {
      for (int i = 0; i < 624; ++i) {
        const uint32_t y = (mt[i] & 0x80000000u) | (mt[(i + 1) % 624] & 0x7fffffffu);
        mt[i] = mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
      }
      idx = 0;
    }
    uint32_t y = mt[idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    out[k] = y;
  }
}
