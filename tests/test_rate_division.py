"""The hop kernels form each rate's exponent argument -Ea / kT as div_rn_recip(-Ea, kT, RN(1/kT))
(akmc_common.cuh): Markstein's correction from the rounded reciprocal, which must give the
bits of an IEEE division, the oracle's `-Ea / (kB T)` (rates_solver.cpp:12-26).  This test
compiles the same header for the host (explicit fused multiply-adds through std::fma, no
contraction) and compares the two on every temperature the configurations use and on random
arguments over the whole range the rates reach, and beyond it."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "misa-akmc-gpu_b200", "csrc")

PROGRAM = r"""
#include <cstdio>
#include <cstdint>
#include "akmc_common.cuh"
using namespace akmc;
static uint64_t s[4] = {0x9E3779B97F4A7C15ull, 0xD1B54A32D192ED03ull, 0x8CB92BA72F3D8DD7ull, 42ull};
static uint64_t nxt() {  // xoshiro256**
  const uint64_t r = rotl64(s[1] * 5, 7) * 9, t = s[1] << 17;
  s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl64(s[3], 45);
  return r;
}
static double u01() { return static_cast<double>(nxt() >> 11) * 0x1p-53; }
int main() {
  long long bad = 0, n = 0;
  auto check = [&](double a, double b) {
    const double y = 1.0 / b;
    const double q = div_rn_recip(a, b, y), want = a / b;
    ++n;
    if (double_to_bits(q) != double_to_bits(want)) {
      if (bad < 5) std::printf("mismatch a=%a b=%a got=%a want=%a\n", a, b, q, want);
      ++bad;
    }
  };
  // every whole temperature from 1 K to 3000 K, arguments -Ea from the jumps' range
  for (int T = 1; T <= 3000; ++T) {
    const double kT = kBoltzmann * static_cast<double>(T);
    for (int i = 0; i < 2000; ++i) check(-(0.3 + 1.2 * u01()), kT);
    for (int i = 0; i < 200; ++i) check(-(6.0 * u01() - 3.0), kT);
  }
  // random significands and exponents: a in +-[2^-40, 2^40], b in [2^-30, 2^30]
  for (int i = 0; i < 20000000; ++i) {
    const double a = (nxt() & 1 ? -1.0 : 1.0) * (1.0 + u01()) * std::ldexp(1.0, static_cast<int>(nxt() % 81) - 40);
    const double b = (1.0 + u01()) * std::ldexp(1.0, static_cast<int>(nxt() % 61) - 30);
    check(a, b);
  }
  // quotients on and next to exact values
  for (int i = 1; i < 200000; ++i) {
    const double b = (1.0 + u01()) * 0.05;
    const double q = static_cast<double>(i) * 0x1p-12;
    const double a = q * b;
    check(a, b);
    check(std::nextafter(a, 0.0), b);
    check(std::nextafter(a, 10.0), b);
  }
  std::printf("%lld %lld\n", n, bad);
  return bad != 0;
}
"""


def test_markstein_quotient_is_the_ieee_quotient(tmp_path):
    src = tmp_path / "div.cpp"
    exe = tmp_path / "div"
    src.write_text(PROGRAM)
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I" + CSRC, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    n, bad = map(int, out.stdout.split()[-2:])
    assert n > 20_000_000
    assert bad == 0 and out.returncode == 0, out.stdout
