"""The asynchronous round order against the synchronous one, on the oracle.

A block's round may run once every neighbour has completed its latest earlier round
whose staged region (sector plus a 2-cell halo) overlaps this round's region; rounds of
other blocks may run in any order.  These tests run the oracle in random orders that
respect that rule and require the same events, lattice, densities and clocks as the
round-by-round schedule of SubLattice::startTimeLoop (sublattice.inl:61-179).
"""
import numpy as np
import pytest

import pyoracle as po
from helpers import QUATERNARY, oracle_job, sort_events

CASES = [
    dict(box=(32, 32, 32), blocks=(2, 2, 2), model=po.MODEL_EAM, alloy=QUATERNARY, n_vacancies=60, seed=7,
         temperature=563.0),
    dict(box=(25, 17, 19), blocks=(3, 2, 1), model=po.MODEL_EAM, precision=po.FP32C, alloy=QUATERNARY,
         n_vacancies=30, seed=11),
    dict(box=(48, 32, 40), blocks=(6, 4, 5), model=po.MODEL_PAIRBOND, alloy=QUATERNARY, n_vacancies=80, seed=3),
    dict(box=(40, 40, 40), blocks=(5, 5, 5), model=po.MODEL_EAM, alloy=QUATERNARY, n_vacancies=150, seed=5),
]


def _state(o):
    ev = sort_events(o.events())
    evo, hops = o.block_state()
    rho = o.rho() if o._cfg.energy_model == po.MODEL_EAM else None
    return ev, o.occupancy(), rho, evo, hops, o.hops


@pytest.mark.parametrize("case", range(len(CASES)))
def test_dependency_order_equals_round_order(case):
    kw = CASES[case]
    rounds = 48
    ref = oracle_job(**kw)
    ref.run_rounds(rounds)
    want = _state(ref)
    assert want[5] > 100
    for order_seed in (0, 1, 2):  # 0: the ready block furthest ahead first
        o = oracle_job(**kw)
        o.run_rounds_flow(rounds, order_seed)
        got = _state(o)
        assert got[5] == want[5]
        ev_g, ev_w = got[0], want[0]
        for f in ("round", "hop", "from_site", "to_site", "block", "species", "n_act", "n_dirty"):
            assert np.array_equal(ev_g[f], ev_w[f]), f
        for f in ("u", "total", "dt"):
            assert np.array_equal(ev_g[f].view(np.uint64), ev_w[f].view(np.uint64)), f
        assert np.array_equal(got[1], want[1])
        if want[2] is not None:
            assert np.array_equal(got[2], want[2])
        assert np.array_equal(got[3].view(np.uint64), want[3].view(np.uint64))
        assert np.array_equal(got[4], want[4])
