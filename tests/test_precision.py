"""Precision report (akmc_b200.precision): the window cut keeps a vacancy's jumps exactly (CPU,
against the oracle), and on the GPU the FP32-compensated form stays within 1e-5 eV of FP64."""
import os
import sys

import numpy as np
import pytest

import pyoracle as po
from helpers import QUATERNARY, oracle_job

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "misa-akmc-gpu_b200",
                                "python"))
from akmc_b200.precision import WINDOW, window  # noqa: E402


@pytest.mark.parametrize("precision", [po.FP64, po.FP32C])
def test_window_keeps_every_jump_of_its_centre_vacancy(precision):
    box = (32, 28, 30)
    o = oracle_job(box=box, precision=precision, alloy=QUATERNARY, n_vacancies=40, seed=3, log_events=0)
    w_job = oracle_job(box=(WINDOW,) * 3, precision=precision, alloy=QUATERNARY, n_vacancies=1, seed=3,
                       log_events=0)
    occ = o.occupancy()
    sites = np.flatnonzero(occ == 0)
    assert len(sites) == 40
    for s in sites[:12]:
        w, c = window(occ, box, int(s))
        assert w[c] == 0 and w.size == 2 * WINDOW ** 3
        w_job.set_occupancy(w)
        a0, r0, d0 = o.vacancy_rates(int(s))
        a1, r1, d1 = w_job.vacancy_rates(int(c))
        assert a0 == a1
        assert np.array_equal(r0.view(np.uint64), r1.view(np.uint64))
        for b in range(8):
            if (a0 >> b) & 1:
                assert d0[b].view(np.uint64) == d1[b].view(np.uint64)


def test_window_wraps_the_periodic_box():
    box = (24, 20, 22)
    occ = np.arange(2 * 24 * 20 * 22, dtype=np.int64)
    w, c = window(occ, box, 1)  # site x=1 (cell 0, body centre), y=0, z=0
    assert w[c] == 1
    w3 = w.reshape(WINDOW, WINDOW, 2 * WINDOW)
    # the window's first row starts 10 cells back in x, y and z, wrapped
    assert w3[0, 0, 0] == (2 * 24 - 20) + 2 * 24 * ((20 - 10) + 20 * (22 - 10))


@pytest.mark.gpu
def test_fp32c_report_on_a_small_lattice():
    import akmc_b200.precision as pr

    r = pr.report(box=(64, 64, 64), blocks=(4, 4, 4), vacancy_fraction=1e-4, n_hops=20000, chunk_rounds=16,
                  log_capacity=1 << 18)
    assert r["hops"]["fp64"] >= 20000
    for k in ("jumps_start", "jumps_end_fp64"):
        j = r[k]
        assert j["jumps"] > 0.5 * 8 * j["vacancies"]
        assert 0.0 < j["max_abs_de_ev"] <= 1e-5
        assert j["max_rel_rate"] <= 1e-3
    d = r["first_divergence"]
    assert (d["hop"] is None) != (d["hops_compared"] is None)
