"""port_exp of the product (akmc_common.cuh, one definition for the host layer and the kernels),
compiled for the host here, must give the oracle's exp bit for bit (oracle/akmc_oracle.cpp
port_exp, a restatement of the same algorithm) on random arguments over the whole double range
that reaches the polynomial and on every special case: NaN, infinities, overflow, underflow to
zero, and results below 2^-1022.  tests/test_gpu_parity.py checks the kernels' exp against the
oracle on the same kinds of arguments."""
import os
import struct
import subprocess

import numpy as np

import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "misa-akmc-gpu_b200", "csrc")

PROGRAM = r"""
#include <cstdio>
#include <cstdint>
#include "akmc_common.cuh"
int main() {
  uint64_t b;
  while (std::fread(&b, 8, 1, stdin) == 1) {
    const uint64_t e = akmc::double_to_bits(akmc::port_exp(akmc::bits_to_double(b)));
    std::fwrite(&e, 8, 1, stdout);
  }
  return 0;
}
"""


def edge_arguments():
    inf = float("inf")
    return [float("nan"), inf, -inf, 0.0, -0.0, 1.0, -1.0, 709.0, 709.782712893384, 709.7827128933841, 709.79, 710.0,
            711.0, 1e300, -700.0, -708.3, -708.4, -708.5, -720.0, -744.0, -745.0, -745.1332191019411,
            -745.1332191019412, -745.1332191019413, -745.2, -746.0, -747.0, -1e300, 2.0 ** -1074, -(2.0 ** -1074)]


def test_host_exp_equals_the_oracle_bit_for_bit(tmp_path):
    src = tmp_path / "exp.cpp"
    exe = tmp_path / "exp"
    src.write_text(PROGRAM)
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I" + CSRC, str(src), "-o", str(exe)], check=True)
    rng = np.random.default_rng(11)
    x = np.concatenate([np.array(edge_arguments()), rng.uniform(-750, 715, 200000), rng.uniform(-60, 0, 100000),
                        rng.uniform(-746, -708, 50000)])
    out = subprocess.run([str(exe)], input=x.astype("<f8").tobytes(), capture_output=True, check=True).stdout
    got = np.frombuffer(out, "<u8")
    want = np.array([struct.unpack("<Q", struct.pack("<d", po.port_exp(float(v))))[0] for v in x], np.uint64)
    nan = np.isnan(x)
    assert np.array_equal(got[~nan], want[~nan])
    assert np.all(np.isnan(np.frombuffer(out, "<f8")[nan]))
