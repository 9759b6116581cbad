// lmm_device.cuh — device helpers shared by the staged and fused kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace lmm {

// Hardware approximations with denormals flushed (PTX ex2/rcp/lg2.approx.ftz).
// The arguments and results where the evolution and the inverse normal use
// them are normal numbers (log-rates capped at 10, accruals and displaced
// rates of order 1e-3..1e2, tail probabilities >= 2^-32), where flushing
// changes no value; the non-flushing forms carry a denormal fix-up around
// each approximation.  exp(x) = 2^(x log2 e), log(x) = log2(x) ln 2.
__device__ __forceinline__ float ex2_ftz(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_ftz(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float lg2_ftz(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float exp_ftz(float x) { return ex2_ftz(x * 1.44269504088896341f); }
__device__ __forceinline__ float log_ftz(float x) { return lg2_ftz(x) * 0.693147180559945309f; }

// Shaw & Brickman (2009) rational approximation of the inverse cumulative
// normal in the form used by inverseCumulativeShawBrickmanUnsignedInt
// (inverseCumulatives.h:146-172): u = float(i) * 2^-32,
// z = -log(1 - |2u - 1|), x = sign(u - 1/2) z P(z)/Q(z).
// The reference evaluates log(0) = -inf for the 129 integers that round to
// u = 0 or u = 1 and returns NaN there; this version clamps the log argument
// at 2^-32 so those points map to the finite tail value (|x| ~ 6.23).
__device__ __forceinline__ float icdf_sb_u(float v) {
  const float P1 = 1.2533136835212087879f;
  const float P2 = 1.9797154223229267471f;
  const float P3 = 0.80002295072483916762f;
  const float P4 = 0.087403248265958578062f;
  const float P5 = 0.0020751409553756572917f;
  const float P6 = 4.744820732427972462e-6f;
  const float Q1 = 1.0f;
  const float Q2 = 2.0795584360534589311f;
  const float Q3 = 1.2499328117341603014f;
  const float Q4 = 0.23668431621373705623f;
  const float Q5 = 0.0120098270559197768f;
  const float Q6 = 0.00010590620919921025259f;
  const float sgn = (v >= 0.5f) ? 1.0f : -1.0f;
  float t = 1.0f - sgn * ((2.0f * v) - 1.0f);
  t = fmaxf(t, 2.3283064365386963e-10f);
  const float z = -logf(t);
  const float p = P1 + z * (P2 + z * (P3 + z * (P4 + (P5 + P6 * z) * z)));
  const float q = Q1 + z * (Q2 + z * (Q3 + z * (Q4 + (Q5 + Q6 * z) * z)));
  return sgn * z * p / q;
}

__device__ __forceinline__ float icdf_sb(uint32_t vi) {
  return icdf_sb_u(__uint2float_rn(vi) * 2.3283064E-10f);
}

// Tail probability of the Shaw–Brickman form, t = 2 min(u, 1 - u), taken
// from the integer: t = min(i, 2^32 - i) * 2^-31.  The reference forms
// 1 - |2 float(i) 2^-32 - 1| in single precision, which quantises t in
// steps of 2^-24 (about 6% of t at u = 2^-20, and t = 0 below 2^-25); this
// form keeps t to 24 significant bits everywhere.  sgn = +1 for i >= 2^31.
__device__ __forceinline__ float icdf_tail_t(uint32_t vi, float* sgn) {
  const bool upper = vi >= 0x80000000u;
  *sgn = upper ? 1.0f : -1.0f;
  const uint32_t m = upper ? (0u - vi) : vi;
  return fmaxf(__uint2float_rn(m) * 4.656612873077392578125e-10f,
               2.3283064365386963e-10f);
}

// Shaw–Brickman rational form on the exact tail probability.
__device__ __forceinline__ float icdf_sb_tails(uint32_t vi) {
  float sgn;
  const float t = icdf_tail_t(vi, &sgn);
  const float z = -logf(t);
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

// Small fixed-capacity tables passed by value as kernel parameters.
template <int N>
struct IntTab {
  int v[N];
};
template <int N>
struct FloatTab {
  float v[N];
};

}  // namespace lmm
