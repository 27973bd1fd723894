"""The reference-side binding (misa-akmc-gpu_b200/integration/gpu_simulate_b200.cpp).

CPU: the shim compiles against the reference's own gpu/gpu_simulate.h and lattice-store
headers (with stand-ins for HIP, libcomm and kiwi) and defines every function that header
declares.

GPU: a PeriodLatticeList of the reference, filled through its occupancy hash sets, is driven
through the shim the way ABVIModel and SubLattice::startTimeLoop drive the HIP backend
(models/abvi/kmc.cpp:118-211, src/algorithms/sl/sublattice.inl:61-140), with the selection and
time draws of the oracle's streams.  Every sector total the shim returns must equal the oracle's,
and after every sector the hash sets must hold the oracle's lattice: the shim uploads the real
alloy and applies every hop to the host lattice.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

import pyoracle as po
from helpers import QUATERNARY, oracle_job

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "shim"))
import build_shim  # noqa: E402

# the free functions of the reference's gpu/gpu_simulate.h:31-66, as declared there
DECLARED = ["firstSectLocalToGpu", "first_calculate_GPU", "calculate_GPU", "selectAndPerformEventGPU",
            "calculateNextAdvRegion", "sector_final", "initialize_gpu", "gpu_final", "gpu_prepare", "getType",
            "exchange_lattices", "add_ghost", "initInfo", "add_surface"]


def _declared_in_reference_header():
    text = open(os.path.join(build_shim.REFERENCE, "gpu", "gpu_simulate.h")).read()
    return sorted(n for n in DECLARED if (n + "(") in text)


@pytest.mark.skipif(not build_shim.available(), reason="the reference sources are not present")
def test_shim_compiles_against_the_reference_header_and_defines_every_declaration():
    assert _declared_in_reference_header() == sorted(DECLARED)
    lib = build_shim.build()
    out = subprocess.run(["nm", "-D", "-C", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    defined = {line.split(" ", 2)[2].split("(")[0] for line in out.splitlines() if " T " in line}
    missing = [n for n in DECLARED if n not in defined]
    assert not missing, missing


def _shim():
    import akmc_b200 as ak

    ak.lib()  # the engine, loaded from its in-tree path first
    if not os.path.exists(build_shim.OUT):
        raise FileNotFoundError("%s is built by __graft_entry__.build() (needs the reference sources)" % build_shim.OUT)
    L = C.CDLL(build_shim.OUT)
    L.shim_prepare.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_double]
    L.shim_prepare.restype = C.c_int
    L.shim_calculate.argtypes = [C.c_int, C.c_int]
    L.shim_calculate.restype = C.c_double
    L.shim_select.argtypes = [C.c_double, C.c_int, C.c_uint]
    L.shim_sector_final.argtypes = [C.c_int]
    L.shim_occupancy.argtypes = [C.c_void_p]
    L.shim_occupancy.restype = C.c_int64
    return L


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [9, 23])
def test_shim_drives_the_reference_loop_and_keeps_the_hash_sets_live(seed):
    box = (16, 16, 16)
    rounds = 32
    o = oracle_job(box=box, model=po.MODEL_PAIRBOND, alloy=QUATERNARY, n_vacancies=8, seed=seed, temperature=563.0)
    occ0 = o.occupancy()
    L = _shim()
    assert L.shim_prepare(occ0.ctypes.data, *box, 2, 6e12, 563.0) == 0
    got = np.empty_like(occ0)
    assert L.shim_occupancy(got.ctypes.data) == 0
    assert np.array_equal(got, occ0)  # the hash sets hold the alloy the engine was given

    # the oracle, sector by sector, as the reference of what the host lattice must hold
    ref = oracle_job(box=box, model=po.MODEL_PAIRBOND, alloy=QUATERNARY, n_vacancies=8, seed=seed,
                     temperature=563.0)
    o.run_rounds(rounds)
    want_events = o.events()
    sel = iter(po.xoshiro_stream(seed, 3, 0, 1 << 16))
    tim = iter(po.xoshiro_stream(seed, 4, 0, 1 << 16))
    ring = (0, 7, 2, 5, 3, 4, 1, 6)
    evo = [0.0] * 8
    totals = []
    for rnd in range(rounds):
        sect = rnd % 8
        sector_id = ring[sect]
        thr = float(rnd // 8 + 1) * 3e-7 - evo[sector_id]
        t, first = 0.0, 1
        while t < thr:  # SubLattice::startTimeLoop, sublattice.inl:82-124
            total = L.shim_calculate(sect, first)
            first = 0
            if total == 0.0 or abs(total) < np.finfo(float).eps:
                t = thr
                continue
            u = float(int(next(sel)) >> 11) * 2.0 ** -53
            L.shim_select(u, sect, sector_id)
            u2 = float((int(next(tim)) >> 11) + 1) * 2.0 ** -53
            t += -po.port_log(u2) / total
            totals.append(total)
        L.shim_sector_final(sect)
        evo[sector_id] += t
        ref.run_rounds(1)
        assert L.shim_occupancy(got.ctypes.data) == 0  # no site in two hash sets
        assert np.array_equal(got, ref.occupancy()), "host lattice differs after round %d" % rnd
    L.shim_final()
    assert len(want_events) > 20
    assert np.array_equal(np.array(totals).view(np.uint64), np.ascontiguousarray(want_events["total"]).view(np.uint64))
    assert np.array_equal(got, o.occupancy())
