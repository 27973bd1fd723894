// akmc_common.cuh -- arithmetic shared by the host layer and the sm_100a kernels.
//
// Every routine here runs the same IEEE-754 operation sequence on the host and
// on the GPU: multiplies and adds round separately (the library is compiled
// with -fmad=false / -ffp-contract=off) and fused multiply-adds are explicit.
// That is what lets the GPU reproduce the CPU semantics bit for bit.
#pragma once

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define AK_HD __host__ __device__ __forceinline__
#else
#define AK_HD inline
#endif

#if !defined(__CUDA_ARCH__)
#include <cmath>
#include <limits>
#endif

namespace akmc {

// Boltzmann constant in eV/K (models/abvi/rate/rates_types.h:16).
constexpr double kBoltzmann = 8.617330350E-5;

// Sector ring of the synchronous sublattice: 0,7,2,5,3,4,1,6
// (src/algorithms/sl/sublattice.h:21-30); bit 0 = high x half, bit 1 = high y, bit 2 = high z.
AK_HD int sector_of_round(int64_t round) {
  constexpr uint32_t packed = 0u | (7u << 3) | (2u << 6) | (5u << 9) | (3u << 12) | (4u << 15) | (1u << 18) | (6u << 21);
  return static_cast<int>((packed >> (3 * (round & 7))) & 7u);
}

// Species codes of the occupancy array (src/lattice/lattice_types.h:20-36).
enum : uint8_t { kV = 0, kFe = 1, kCu = 2, kNi = 4, kMn = 8 };

AK_HD bool is_atom(uint8_t c) { return c == kFe || c == kCu || c == kNi || c == kMn; }
// Fe, Cu, Ni, Mn -> 0..3 (V -> -1)
AK_HD int species_index(uint8_t c) {
  return c == kFe ? 0 : c == kCu ? 1 : c == kNi ? 2 : c == kMn ? 3 : -1;
}
// The same for a code known to be an atom (1, 2, 4, 8 -> 0..3), without the compare chain.
AK_HD int atom_index(uint8_t c) { return (c >> 1) - (c >> 3); }
// V, Fe, Cu, Ni, Mn -> 0..4 (pair-bond table index)
AK_HD int bond_index(uint8_t c) { return c == kV ? 0 : species_index(c) + 1; }

// Migration energy prefactor e0 by moving species (vacancy_rates_solver.cpp:14-27).
AK_HD double e0_of(uint8_t c) {
  return c == kFe ? 0.62 : c == kCu ? 0.54 : c == kNi ? 0.68 : c == kMn ? 1.03 : 0.0;
}

// ---------------------------------------------------------------------------
AK_HD double fma_d(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}
AK_HD float fma_f(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
  return __fmaf_rn(a, b, c);
#else
  return std::fmaf(a, b, c);
#endif
}
AK_HD double bits_to_double(uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double(static_cast<long long>(b));
#else
  double d;
  memcpy(&d, &b, 8);
  return d;
#endif
}
AK_HD uint64_t double_to_bits(double d) {
#if defined(__CUDA_ARCH__)
  return static_cast<uint64_t>(__double_as_longlong(d));
#else
  uint64_t b;
  memcpy(&b, &d, 8);
  return b;
#endif
}
AK_HD double rint_d(double x) {
#if defined(__CUDA_ARCH__)
  return rint(x);
#else
  return std::rint(x);
#endif
}

// exp(x): Cody & Waite reduction x = k ln2 + r with ln2 split into a 32-bit head and a tail,
// then the Taylor polynomial of degree 13 for e^r (|r| <= ln2/2, truncation < 5e-18) as
// e^r = 1 + (r + r^2 T(r)), with T(r) = sum_{i=2..13} r^(i-2)/i! in Estrin's scheme (pairs
// 1/i! + r/(i+1)!, then r^2, r^4, r^8), and scaling by 2^k through the exponent field.  The
// dependent chain of the polynomial is 6 operations instead of Horner's 14 (a rate is one long
// FP64 chain per jump); max error 0.92 ulp against a correctly rounded exp over the range used.
AK_HD double port_exp(double x) {
  if (x != x) return x;
  if (x > 709.782712893384) return bits_to_double(0x7ff0000000000000ULL);
  if (x < -745.1332191019412) return 0.0;
  const double kd = rint_d(x * 0x1.71547652b82fep+0);
  const int k = static_cast<int>(kd);
  double r = fma_d(-kd, 0x1.62e42fee00000p-1, x);
  r = fma_d(-kd, 0x1.a39ef35793c76p-33, r);
  const double r2 = r * r, r4 = r2 * r2, r8 = r4 * r4;
  const double p23 = fma_d(0x1.5555555555555p-3, r, 0.5);                     // 1/2! + r/3!
  const double p45 = fma_d(0x1.1111111111111p-7, r, 0x1.5555555555555p-5);    // 1/4!, 1/5!
  const double p67 = fma_d(0x1.a01a01a01a01ap-13, r, 0x1.6c16c16c16c17p-10);  // 1/6!, 1/7!
  const double p89 = fma_d(0x1.71de3a556c734p-19, r, 0x1.a01a01a01a01ap-16);  // 1/8!, 1/9!
  const double p1011 = fma_d(0x1.ae64567f544e4p-26, r, 0x1.27e4fb7789f5cp-22);  // 1/10!, 1/11!
  const double p1213 = fma_d(0x1.6124613a86d09p-33, r, 0x1.1eed8eff8d898p-29);  // 1/12!, 1/13!
  const double t0 = fma_d(p45, r2, p23), t1 = fma_d(p89, r2, p67), t2 = fma_d(p1213, r2, p1011);
  const double T = fma_d(t2, r8, fma_d(t1, r4, t0));
  const double p = 1.0 + fma_d(r2, T, r);
  if (k > 1023) return p * bits_to_double(2046ULL << 52) * bits_to_double(static_cast<uint64_t>(k) << 52);
  if (k < -1022) return p * bits_to_double(1ULL << 52) * bits_to_double(static_cast<uint64_t>(k + 2045) << 52);
  return p * bits_to_double(static_cast<uint64_t>(k + 1023) << 52);
}

// log(x): x = m 2^e, m in [sqrt(1/2), sqrt(2)); log m = 2 atanh(s) with
// s = (m-1)/(m+1), odd series to s^25 (|s| <= 0.1716, truncation < 3e-18).
AK_HD double port_log(double x) {
  if (x != x || x < 0.0) return bits_to_double(0x7ff8000000000000ULL);
  if (x == 0.0) return bits_to_double(0xfff0000000000000ULL);
  if (double_to_bits(x) == 0x7ff0000000000000ULL) return x;
  uint64_t b = double_to_bits(x);
  int e = static_cast<int>((b >> 52) & 0x7ff);
  if (e == 0) {
    x = x * 0x1p54;
    b = double_to_bits(x);
    e = static_cast<int>((b >> 52) & 0x7ff) - 54;
  }
  e -= 1023;
  double m = bits_to_double((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
  if (m > 0x1.6a09e667f3bcdp+0) {
    m = m * 0.5;
    e += 1;
  }
  const double s = (m - 1.0) / (m + 1.0);
  const double z = s * s;
  double p = 0x1.47ae147ae147bp-5;       // 1/25
  p = fma_d(p, z, 0x1.642c8590b2164p-5);  // 1/23
  p = fma_d(p, z, 0x1.8618618618618p-5);  // 1/21
  p = fma_d(p, z, 0x1.af286bca1af28p-5);  // 1/19
  p = fma_d(p, z, 0x1.e1e1e1e1e1e1ep-5);  // 1/17
  p = fma_d(p, z, 0x1.1111111111111p-4);  // 1/15
  p = fma_d(p, z, 0x1.3b13b13b13b14p-4);  // 1/13
  p = fma_d(p, z, 0x1.745d1745d1746p-4);  // 1/11
  p = fma_d(p, z, 0x1.c71c71c71c71cp-4);  // 1/9
  p = fma_d(p, z, 0x1.2492492492492p-3);  // 1/7
  p = fma_d(p, z, 0x1.999999999999ap-3);  // 1/5
  p = fma_d(p, z, 0x1.5555555555555p-2);  // 1/3
  const double t = s + s;
  const double logm = fma_d(t * z, p, t);
  const double ed = static_cast<double>(e);
  return fma_d(ed, 0x1.62e42fee00000p-1, fma_d(ed, 0x1.a39ef35793c76p-33, logm));
}

// Arrhenius rate nu exp(-Ea / (kB T)), Ea = e0 + dE/2 (rates_solver.cpp:12-26).
AK_HD double arrhenius(double nu, double kT, uint8_t moving, double dE) {
  const double Ea = e0_of(moving) + dE / 2;
  return nu * port_exp(-Ea / kT);
}

// a / b rounded to nearest from y = RN(1 / b), by Markstein's correction (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
// Dev. 34(1), 1990): when y is the correctly rounded reciprocal and q lies within one ulp of
// a / b, the remainder r = a - b q is exact under a fused multiply-add and RN(q + r y) is the
// correctly rounded quotient.  q0 = RN(a y) may lie up to 1.5 ulp away, so a first correction
// brings it within one ulp (its error becomes about half an ulp) and a second one gives RN(a / b),
// the same bits as an IEEE division.  Valid away from overflow and underflow of q and r: the
// rates' exponent arguments are a few eV over kT in (0, 1) eV.  Five dependent operations in
// place of a division on the latency chain of every rate.
AK_HD double div_rn_recip(double a, double b, double y) {
  const double q0 = a * y;
  const double r0 = fma_d(-q0, b, a);
  const double q1 = fma_d(r0, y, q0);
  const double r1 = fma_d(-q1, b, a);
  return fma_d(r1, y, q1);
}

// arrhenius() with the exponent argument -Ea / kT formed by div_rn_recip (rkT = RN(1 / kT)):
// the same bits.
AK_HD double arrhenius_rk(double nu, double kT, double rkT, uint8_t moving, double dE) {
  const double Ea = e0_of(moving) + dE / 2;
  return nu * port_exp(div_rn_recip(-Ea, kT, rkT));
}

// ---------------------------------------------------------------------------
// xoshiro256** (Blackman & Vigna 2018); streams seeded through splitmix64.
// Stream (seed, tag, index): tag 1 alloy types, 2 vacancies, 3 event selection,
// 4 residence time, 5 EAM parameters; index = domain block.
enum : uint64_t { kTagTypes = 1, kTagVacancy = 2, kTagSelect = 3, kTagTime = 4, kTagPotential = 5 };

AK_HD uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
AK_HD uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
AK_HD uint64_t xoshiro_next(uint64_t s[4]) {
  const uint64_t r = rotl64(s[1] * 5, 7) * 9;
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl64(s[3], 45);
  return r;
}
AK_HD void xoshiro_seed(uint64_t s[4], uint64_t seed, uint64_t tag, uint64_t index) {
  uint64_t h = mix64(seed ^ (tag * 0xD1B54A32D192ED03ULL));
  h = mix64(h ^ (index * 0x9E3779B97F4A7C15ULL + 0x632BE59BD9B4E019ULL));
  for (int i = 0; i < 4; ++i) {
    h += 0x9E3779B97F4A7C15ULL;
    s[i] = mix64(h);
  }
  if ((s[0] | s[1] | s[2] | s[3]) == 0) s[0] = 1;
}
// selection uniform in [0, 1)
AK_HD double uniform_co(uint64_t s[4]) { return static_cast<double>(xoshiro_next(s) >> 11) * 0x1p-53; }
// residence-time uniform in (0, 1]: -log(u) stays finite
AK_HD double uniform_oc(uint64_t s[4]) { return static_cast<double>((xoshiro_next(s) >> 11) + 1) * 0x1p-53; }

// ---------------------------------------------------------------------------
// EAM embedding function F(rho) on the fixed-point density (Q.24, cell = r >> 17,
// rho step 2^-7): Catmull-Rom cubic per cell, c0 + p(c1 + p(c2 + p c3)).
constexpr int kRhoCellShift = 17;
constexpr int kRhoFracMask = (1 << kRhoCellShift) - 1;
constexpr int kTabN = 5000;

struct alignas(32) FCell32 {  // single-precision cell: node value split hi+lo, then c1..c3
  float hi, lo, c1, c2, c3, pad0, pad1, pad2;
};

AK_HD double cubic_d(double c0, double c1, double c2, double c3, double p) {
  return fma_d(fma_d(fma_d(c3, p, c2), p, c1), p, c0);
}
// F(r1) - F(r0) in FP32: the node difference (hi1 - hi0) is exact for nearby
// nodes, the tails and the polynomial parts are small, so the result carries
// an absolute error of a few 1e-8 eV instead of the 1e-7 of two F values.
AK_HD float dF32(const FCell32& a1, const FCell32& a0, int32_t r1, int32_t r0) {
  const float p1 = static_cast<float>(r1 & kRhoFracMask) * 0x1p-17f;
  const float p0 = static_cast<float>(r0 & kRhoFracMask) * 0x1p-17f;
  const float q1 = fma_f(fma_f(a1.c3, p1, a1.c2), p1, a1.c1) * p1;
  const float q0 = fma_f(fma_f(a0.c3, p0, a0.c2), p0, a0.c1) * p0;
  const float node = (a1.hi - a0.hi) + (a1.lo - a0.lo);
  return node + (q1 - q0);
}

// Kahan-compensated FP32 sum and its merge (two-sum of the heads, tails added);
// the merge is commutative, so a xor-shuffle butterfly is order independent.
struct Comp32 {
  float s, c;
};
AK_HD void kahan_add(Comp32& a, float v) {
  const float y = v - a.c;
  const float t = a.s + y;
  a.c = (t - a.s) - y;
  a.s = t;
}
AK_HD Comp32 comp_merge(Comp32 a, Comp32 b) {
  const float s = a.s + b.s;
  const float bb = s - a.s;
  const float e = (a.s - (s - bb)) + (b.s - bb);
  Comp32 r;
  r.s = s;
  r.c = (a.c + b.c) - e;
  return r;
}

}  // namespace akmc
