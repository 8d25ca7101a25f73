// Counter-based random numbers shared bit-for-bit by host and device code.
//
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): a keyed bijection of a 128-bit counter.  Every random
// draw in this library is a pure function of (seed, stream, step, atom id), so
// a replica's noise does not depend on storage order, batch composition, or the
// number of steps taken per launch.  This replaces the reference's per-atom
// cuRAND state (integrate/langevin.cu:7-13, 64-66), which costs 128 B of state
// traffic per atom-step.
//
// Normal deviates use the Box-Muller transform.  Its log and sin/cos are written
// here from their series (atanh series for log; Taylor series for sin/cos on
// [0, pi/4] after an exact quadrant split) using only correctly rounded IEEE
// operations with every fused multiply-add explicit, so the host and the GPU
// produce identical bits.  That is what makes single-step parity against the
// CPU oracle exact rather than statistical.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define FMD_HD __host__ __device__ __forceinline__
#else
#define FMD_HD inline
#endif

#if defined(__CUDA_ARCH__)
#define FMD_DMUL(a, b) __dmul_rn((a), (b))
#define FMD_DADD(a, b) __dadd_rn((a), (b))
#define FMD_DSUB(a, b) __dsub_rn((a), (b))
#define FMD_DFMA(a, b, c) __fma_rn((a), (b), (c))
#define FMD_DDIV(a, b) __ddiv_rn((a), (b))
#define FMD_DSQRT(a) __dsqrt_rn((a))
#else
#include <cmath>
#define FMD_DMUL(a, b) ((a) * (b))
#define FMD_DADD(a, b) ((a) + (b))
#define FMD_DSUB(a, b) ((a) - (b))
#define FMD_DFMA(a, b, c) std::fma((a), (b), (c))
#define FMD_DDIV(a, b) ((a) / (b))
#define FMD_DSQRT(a) std::sqrt((a))
#endif

namespace fmd {

// Stream identifiers (the fourth counter word) keep independent uses apart.
enum : uint32_t {
  kStreamLangevin = 0x4C414E47u,  // "LANG": per-atom thermostat noise
  kStreamGenWalk = 0x47454E57u,   // "GENW": melt generator random walk
  kStreamGenVel = 0x47454E56u,    // "GENV": melt generator initial velocities
  kStreamPushoff = 0x50555348u,   // "PUSH": push-off thermostat noise
};

struct U32x4 {
  uint32_t x, y, z, w;
};

FMD_HD uint32_t philox_mulhi(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
#endif
}

// Philox4x32 with 10 rounds.  Multipliers and Weyl key increments are the ones
// published with the algorithm.
FMD_HD U32x4 philox4x32_10(U32x4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint32_t lo0 = 0xD2511F53u * c.x;
    const uint32_t hi0 = philox_mulhi(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z;
    const uint32_t hi1 = philox_mulhi(0xCD9E8D57u, c.z);
    U32x4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
  }
  return c;
}

// Natural log of x in (0, 1] (x > 0 finite, normal).  x = m * 2^e with
// m in [sqrt(1/2), sqrt(2)); ln m = 2 atanh(s), s = (m - 1) / (m + 1), summed
// as s * sum_k s^(2k) / (2k + 1) to 12 terms (|s| < 0.1716, truncation < 1e-19).
FMD_HD double rng_log(double x) {
  union {
    double d;
    uint64_t u;
  } b;
  b.d = x;
  int e = (int)((b.u >> 52) & 0x7FFu) - 1023;
  b.u = (b.u & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull;
  double m = b.d;
  if (m > 1.4142135623730951) {
    m = FMD_DMUL(m, 0.5);
    e += 1;
  }
  const double s = FMD_DDIV(FMD_DSUB(m, 1.0), FMD_DADD(m, 1.0));
  const double z = FMD_DMUL(s, s);
  double p = 1.0 / 23.0;
  p = FMD_DFMA(p, z, 1.0 / 21.0);
  p = FMD_DFMA(p, z, 1.0 / 19.0);
  p = FMD_DFMA(p, z, 1.0 / 17.0);
  p = FMD_DFMA(p, z, 1.0 / 15.0);
  p = FMD_DFMA(p, z, 1.0 / 13.0);
  p = FMD_DFMA(p, z, 1.0 / 11.0);
  p = FMD_DFMA(p, z, 1.0 / 9.0);
  p = FMD_DFMA(p, z, 1.0 / 7.0);
  p = FMD_DFMA(p, z, 1.0 / 5.0);
  p = FMD_DFMA(p, z, 1.0 / 3.0);
  // ln m = 2 s + 2 s z p(z)
  const double two_s = FMD_DMUL(2.0, s);
  const double lnm = FMD_DFMA(FMD_DMUL(two_s, z), p, two_s);
  // ln 2 split so that e * ln2_hi is exact for |e| < 2^28.
  const double ln2_hi = 0x1.62e42f0000000p-1;
  const double ln2_lo = 0x1.df473de6af279p-26;
  const double de = (double)e;
  return FMD_DFMA(de, ln2_hi, FMD_DFMA(de, ln2_lo, lnm));
}

// sin and cos of (pi/2) * g for g in [0, 1/2] via Taylor series through the
// 17th / 18th power (truncation below 2e-17 on [0, pi/4]).
FMD_HD void rng_sincos_quarter(double g, double* s_out, double* c_out) {
  const double pio2_hi = 0x1.921fb50000000p+0;
  const double pio2_lo = 0x1.110b4611a6263p-26;
  const double t = FMD_DFMA(g, pio2_hi, FMD_DMUL(g, pio2_lo));
  const double t2 = FMD_DMUL(t, t);
  double ps = -1.0 / 355687428096000.0;  // -1/17!
  ps = FMD_DFMA(ps, t2, 1.0 / 1307674368000.0);
  ps = FMD_DFMA(ps, t2, -1.0 / 6227020800.0);
  ps = FMD_DFMA(ps, t2, 1.0 / 39916800.0);
  ps = FMD_DFMA(ps, t2, -1.0 / 362880.0);
  ps = FMD_DFMA(ps, t2, 1.0 / 5040.0);
  ps = FMD_DFMA(ps, t2, -1.0 / 120.0);
  ps = FMD_DFMA(ps, t2, 1.0 / 6.0);
  // sin t = t - t^3 ps'(t^2) written as t - t*t2*ps
  *s_out = FMD_DFMA(-FMD_DMUL(t, t2), ps, t);
  double pc = 1.0 / 6402373705728000.0;  // 1/18!
  pc = FMD_DFMA(pc, t2, -1.0 / 20922789888000.0);
  pc = FMD_DFMA(pc, t2, 1.0 / 87178291200.0);
  pc = FMD_DFMA(pc, t2, -1.0 / 479001600.0);
  pc = FMD_DFMA(pc, t2, 1.0 / 3628800.0);
  pc = FMD_DFMA(pc, t2, -1.0 / 40320.0);
  pc = FMD_DFMA(pc, t2, 1.0 / 720.0);
  pc = FMD_DFMA(pc, t2, -1.0 / 24.0);
  pc = FMD_DFMA(pc, t2, 0.5);
  *c_out = FMD_DFMA(-t2, pc, 1.0);
}

// Box-Muller pair from two 32-bit words: u1 = (a + 1) 2^-32 in (0, 1];
// the angle 2 pi u2 is split exactly into quadrant q = top two bits of b and
// fraction f = (low 30 bits) 2^-30.
FMD_HD void rng_normal_pair(uint32_t a, uint32_t b, double* z0, double* z1) {
  const double u1 = FMD_DMUL((double)a + 1.0, 0x1.0p-32);
  const double r = FMD_DSQRT(FMD_DMUL(-2.0, rng_log(u1)));
  const uint32_t q = b >> 30;
  double f = FMD_DMUL((double)(b & 0x3FFFFFFFu), 0x1.0p-30);
  double s, c;
  if (f > 0.5) {
    rng_sincos_quarter(FMD_DSUB(1.0, f), &c, &s);
  } else {
    rng_sincos_quarter(f, &s, &c);
  }
  double cs, sn;
  switch (q) {
    case 0: cs = c; sn = s; break;
    case 1: cs = -s; sn = c; break;
    case 2: cs = -c; sn = -s; break;
    default: cs = s; sn = -c; break;
  }
  *z0 = FMD_DMUL(r, cs);
  *z1 = FMD_DMUL(r, sn);
}

// Three standard normal deviates for (seed, stream, step, id).
FMD_HD void rng_normal3(uint64_t seed, uint32_t stream, uint64_t step, uint32_t id,
                        double* n0, double* n1, double* n2) {
  U32x4 c;
  c.x = id;
  c.y = (uint32_t)step;
  c.z = (uint32_t)(step >> 32);
  c.w = stream;
  const U32x4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  double z3;
  rng_normal_pair(r.x, r.y, n0, n1);
  rng_normal_pair(r.z, r.w, n2, &z3);
}

// Uniform double in [0, 1) with 53 random bits from words (a, b).
FMD_HD double rng_uniform53(uint32_t a, uint32_t b) {
  const uint64_t v = ((uint64_t)a << 21) ^ (uint64_t)(b >> 11);
  return (double)(v & ((1ull << 53) - 1)) * 0x1.0p-53;
}

}  // namespace fmd
