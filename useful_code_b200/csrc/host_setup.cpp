// host_setup.cpp — host-side (FP64) model set-up: pseudo-roots of the
// per-step covariance matrices, fixed and initial drifts, and scrambler
// words.  Negligible cost next to the path simulation; results are the
// small device inputs of the pipeline.
//
// Reference behaviour followed:
//   abcd covariance integral   gold/volstructs_gold.cpp:271-307
//                              (Abcdprimitive, covarianceABCD)
//   ABCD + exp correlation     gold/volstructs_gold.cpp:311-360
//   flat vols                  gold/volstructs_gold.cpp:177-255
//   rank-F pseudo-root         gold/math/pseudoSquareRoot.cpp:76-110
//                              (eigen-decomposition, descending eigenvalues,
//                              rows rescaled to the input variances)
//   fixed drift -1/2 |A_r|^2   kooexample/bermudanIRDPricer.cu:403-417
//   initial spot drift         gold/LMM_evolver_gold.h:178-203
//   scrambler words            MT19937 as gold/Mersenne_gold.cpp:51-110
// The eigen-decomposition is a cyclic Jacobi iteration written here; the
// sign of each eigenvector is fixed so that its first non-negligible
// component is positive.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "../../include/lmm_c.h"

namespace lmm {
int fail(int code, const char* fmt, ...);
}

namespace {

// Cyclic Jacobi: a (n x n, row-major, destroyed), eigenvalues w, vectors
// in the columns of v.
void jacobi_eigen(std::vector<double>& a, int n, std::vector<double>& w,
                  std::vector<double>& v) {
  v.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) v[(size_t)i * n + i] = 1.0;
  double scale = 0.0;
  for (int i = 0; i < n * n; ++i) scale = std::max(scale, std::fabs(a[i]));
  if (scale == 0.0) {
    w.assign(n, 0.0);
    return;
  }
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += a[(size_t)p * n + q] * a[(size_t)p * n + q];
    if (off <= 1e-30 * scale * scale) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a[(size_t)p * n + q];
        if (std::fabs(apq) <= 1e-300) continue;
        const double app = a[(size_t)p * n + p], aqq = a[(size_t)q * n + q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) /
                         (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          const double akp = a[(size_t)k * n + p], akq = a[(size_t)k * n + q];
          a[(size_t)k * n + p] = c * akp - s * akq;
          a[(size_t)k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = a[(size_t)p * n + k], aqk = a[(size_t)q * n + k];
          a[(size_t)p * n + k] = c * apk - s * aqk;
          a[(size_t)q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = v[(size_t)k * n + p], vkq = v[(size_t)k * n + q];
          v[(size_t)k * n + p] = c * vkp - s * vkq;
          v[(size_t)k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  w.resize(n);
  for (int i = 0; i < n; ++i) w[i] = a[(size_t)i * n + i];
}

// Rank-F pseudo-square-root of the covariance c (n x n) into out (n x F).
void pseudo_root(const std::vector<double>& c, int n, int F, double* out) {
  std::vector<double> a(c), w, v;
  jacobi_eigen(a, n, w, v);
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return w[x] > w[y]; });
  const double wmax = n ? std::max(w[order[0]], 0.0) : 0.0;
  for (int f = 0; f < F; ++f) {
    const int col = f < n ? order[f] : -1;
    double lam = col >= 0 ? w[col] : 0.0;
    if (wmax > 0 && std::fabs(lam / wmax) < 1e-16) lam = 0.0;
    const double root = lam > 0 ? std::sqrt(lam) : 0.0;
    double sign = 1.0;
    if (col >= 0) {
      double vmax = 0.0;
      for (int i = 0; i < n; ++i) vmax = std::max(vmax, std::fabs(v[(size_t)i * n + col]));
      for (int i = 0; i < n; ++i) {
        const double x = v[(size_t)i * n + col];
        if (std::fabs(x) > 1e-9 * vmax) {
          sign = x < 0 ? -1.0 : 1.0;
          break;
        }
      }
    }
    for (int i = 0; i < n; ++i)
      out[(size_t)i * F + f] = col >= 0 ? sign * v[(size_t)i * n + col] * root : 0.0;
  }
  for (int i = 0; i < n; ++i) {
    double norm = 0.0;
    for (int f = 0; f < F; ++f) norm += out[(size_t)i * F + f] * out[(size_t)i * F + f];
    if (norm > 0.0) {
      const double adj = std::sqrt(c[(size_t)i * n + i] / norm);
      for (int f = 0; f < F; ++f) out[(size_t)i * F + f] *= adj;
    }
  }
}

// Integral of (a + b(S-s)) e^{-c(S-s)} + d times the same for T, from 0 to t
// (the abcd instantaneous covariance primitive).
double abcd_primitive(double a, double b, double c, double d, double t,
                      double S, double T) {
  if (T < t || S < t) return 0.0;
  if (std::fabs(c) < 1e-9) {
    const double v = a + d;
    return t * (v * v + v * b * S + v * b * T - v * b * t + b * b * S * T -
                0.5 * b * b * t * (S + T) + b * b * t * t / 3.0);
  }
  const double k1 = std::exp(c * t), k2 = std::exp(c * S), k3 = std::exp(c * T);
  return (b * b * (-1 - 2 * c * c * S * T - c * (S + T) +
                   k1 * k1 * (1 + c * (S + T - 2 * t) + 2 * c * c * (S - t) * (T - t))) +
          2 * c * c *
              (2 * d * a * (k2 + k3) * (k1 - 1) + a * a * (k1 * k1 - 1) +
               2 * c * d * d * k2 * k3 * t) +
          2 * b * c *
              (a * (-1 - c * (S + T) + k1 * k1 * (1 + c * (S + T - 2 * t))) -
               2 * d *
                   (k3 * (1 + c * S) + k2 * (1 + c * T) - k1 * k3 * (1 + c * (S - t)) -
                    k1 * k2 * (1 + c * (T - t))))) /
         (4 * c * c * c * k2 * k3);
}

double abcd_covariance(double a, double b, double c, double d, double t1,
                       double t2, double S, double T) {
  const double stop = std::min(std::min(S, T), t2);
  if (t1 >= stop) return 0.0;
  return abcd_primitive(a, b, c, d, t2, S, T) - abcd_primitive(a, b, c, d, t1, S, T);
}

}  // namespace

extern "C" int lmm_abcd_pseudo_roots(double a, double b, double c, double d,
                                     const double* h_evolution_times, int steps,
                                     const double* h_rate_starts, int rates,
                                     const double* h_multipliers, int factors,
                                     double L, double beta, double* h_out) {
  if (steps < 1 || rates < 1 || factors < 1 || factors > rates ||
      !h_evolution_times || !h_rate_starts || !h_multipliers || !h_out)
    return lmm::fail(LMM_EINVAL, "lmm_abcd_pseudo_roots: bad arguments");
  std::vector<double> cov((size_t)rates * rates);
  double start = 0.0;
  for (int s = 0; s < steps; ++s) {
    const double stop = h_evolution_times[s];
    for (int r = 0; r < rates; ++r) {
      const double kr = h_multipliers[r];
      cov[(size_t)r * rates + r] =
          abcd_covariance(a, b, c, d, start, stop, h_rate_starts[r], h_rate_starts[r]) * kr * kr;
      for (int q = 0; q < r; ++q) {
        const double rho =
            std::exp(-beta * std::fabs(h_rate_starts[q] - h_rate_starts[r])) * (1 - L) + L;
        const double x = abcd_covariance(a, b, c, d, start, stop, h_rate_starts[r],
                                         h_rate_starts[q]) *
                         rho * h_multipliers[q] * kr;
        cov[(size_t)r * rates + q] = cov[(size_t)q * rates + r] = x;
      }
    }
    start = stop;
    pseudo_root(cov, rates, factors, h_out + (size_t)s * rates * factors);
  }
  return LMM_OK;
}

// Chain rule from dV/dA (lmm_greeks) to the abcd parameters: central
// differences of the pseudo-root construction above, contracted with abar.
// The construction's eigenvector sign rule (first non-negligible component
// positive) keeps the bumped roots on the same branch.
extern "C" int lmm_abcd_vegas(double a, double b, double c, double d,
                              const double* h_evolution_times, int steps,
                              const double* h_rate_starts, int rates,
                              const double* h_multipliers, int factors, double L,
                              double beta, const double* h_abar, double rel_bump,
                              double* h_out) {
  if (!h_abar || !h_out || !(rel_bump > 0.0))
    return lmm::fail(LMM_EINVAL, "lmm_abcd_vegas: bad arguments");
  const size_t nA = (size_t)steps * rates * factors;
  std::vector<double> up(nA), dn(nA);
  double par[4] = {a, b, c, d};
  for (int k = 0; k < 4; ++k) {
    const double h = rel_bump * std::max(std::fabs(par[k]), 1e-3);
    double pu[4] = {a, b, c, d}, pd[4] = {a, b, c, d};
    pu[k] += h;
    pd[k] -= h;
    int st = lmm_abcd_pseudo_roots(pu[0], pu[1], pu[2], pu[3], h_evolution_times, steps,
                                   h_rate_starts, rates, h_multipliers, factors, L, beta,
                                   up.data());
    if (st) return st;
    st = lmm_abcd_pseudo_roots(pd[0], pd[1], pd[2], pd[3], h_evolution_times, steps,
                               h_rate_starts, rates, h_multipliers, factors, L, beta,
                               dn.data());
    if (st) return st;
    double v = 0.0;
    for (size_t i = 0; i < nA; ++i) v += h_abar[i] * (up[i] - dn[i]);
    h_out[k] = v / (2.0 * h);
  }
  return LMM_OK;
}

extern "C" int lmm_flat_pseudo_roots(const double* h_rate_times, int rates,
                                     const double* h_evolution_times, int steps,
                                     const double* h_vols, int factors,
                                     double L, double beta, double* h_out) {
  if (steps < 1 || rates < 1 || factors < 1 || factors > rates ||
      !h_rate_times || !h_evolution_times || !h_vols || !h_out)
    return lmm::fail(LMM_EINVAL, "lmm_flat_pseudo_roots: bad arguments");
  std::vector<double> cov((size_t)rates * rates);
  double start = 0.0;
  for (int s = 0; s < steps; ++s) {
    const double stop = h_evolution_times[s];
    for (int r = 0; r < rates; ++r) {
      const double tr = std::min(stop, h_rate_times[r]) - std::min(start, h_rate_times[r]);
      cov[(size_t)r * rates + r] = h_vols[r] * h_vols[r] * tr;
      for (int q = 0; q < r; ++q) {
        const double tq = std::min(stop, h_rate_times[q]) - std::min(start, h_rate_times[q]);
        const double rho =
            L + (1.0 - L) * std::exp(-beta * std::fabs(h_rate_times[r] - h_rate_times[q]));
        cov[(size_t)r * rates + q] = cov[(size_t)q * rates + r] =
            rho * h_vols[r] * h_vols[q] * std::min(tr, tq);
      }
    }
    start = stop;
    pseudo_root(cov, rates, factors, h_out + (size_t)s * rates * factors);
  }
  return LMM_OK;
}

extern "C" int lmm_fixed_drifts(const float* h_A, int steps, int rates,
                                int factors, float* h_out) {
  if (!h_A || !h_out || steps < 1 || rates < 1 || factors < 1)
    return lmm::fail(LMM_EINVAL, "lmm_fixed_drifts: bad arguments");
  for (int s = 0; s < steps; ++s)
    for (int r = 0; r < rates; ++r) {
      float x = 0.0f;
      for (int f = 0; f < factors; ++f) {
        const float a = h_A[((size_t)s * rates + r) * factors + f];
        x += a * a;
      }
      h_out[(size_t)s * rates + r] = -0.5f * x;
    }
  return LMM_OK;
}

extern "C" int lmm_spot_drifts(const float* h_A, const float* h_rates,
                               const float* h_taus, const float* h_disp,
                               int rates, int factors, float* h_out) {
  if (!h_A || !h_rates || !h_taus || !h_disp || !h_out || rates < 1 || factors < 1)
    return lmm::fail(LMM_EINVAL, "lmm_spot_drifts: bad arguments");
  std::vector<float> e(factors, 0.0f);
  for (int r = 0; r < rates; ++r) {
    const float g = (h_rates[r] + h_disp[r]) * h_taus[r] / (1.0f + h_rates[r] * h_taus[r]);
    float x = 0.0f;
    for (int f = 0; f < factors; ++f) {
      e[f] += h_A[(size_t)r * factors + f] * g;
      x += h_A[(size_t)r * factors + f] * e[f];
    }
    h_out[r] = x;
  }
  return LMM_OK;
}

extern "C" int lmm_mt19937_words(uint32_t seed, int n, uint32_t* h_out) {
  if (n < 0 || (n > 0 && !h_out))
    return lmm::fail(LMM_EINVAL, "lmm_mt19937_words: bad arguments");
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
    h_out[k] = y;
  }
  return LMM_OK;
}
