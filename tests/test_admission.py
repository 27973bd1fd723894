"""Continuous batching in one context: akmc_admit_job / akmc_retire_job.

Jobs admitted into a prepared context that is already running rounds start at round 0 and
must follow exactly the trajectory they have alone (the oracle's): events, lattice, densities,
block clocks.  Retiring a job leaves the others untouched, and its slot can take a new job.
Both round schedules are run, and a context may start with no jobs at all.
"""
import numpy as np
import pytest

import pyoracle as po
from helpers import QUATERNARY, oracle_job

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ak():
    import os
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "misa-akmc-gpu_b200"))
    import build

    build.build()
    import akmc_b200

    return akmc_b200


def _cfg(ak, o, kw, hop_budget=0):
    model = kw.get("model", po.MODEL_EAM)
    eam = ak.eam_johnson(kw.get("pot_seed", 42)) if model == po.MODEL_EAM else None
    return ak.job_config(kw["box"], blocks=kw.get("blocks", (1, 1, 1)), energy_model=model,
                         precision=kw.get("precision", po.FP64), seed=kw.get("seed", 42),
                         temperature=kw.get("temperature", 573.0), eam=eam, hop_budget=hop_budget)


def _check(eng, slot, o, ev, eam=True):
    mine = ev[ev["job"] == slot]
    mine = mine[np.lexsort((mine["hop"], mine["block"], mine["round"]))]
    want = o.events()
    assert len(mine) == len(want) and len(want) > 0
    for f in ("round", "hop", "from_site", "to_site", "block", "species"):
        assert np.array_equal(mine[f], want[f]), f
    for f in ("u", "total", "dt"):
        assert np.array_equal(np.ascontiguousarray(mine[f]).view(np.uint64),
                              np.ascontiguousarray(want[f]).view(np.uint64)), f
    assert np.array_equal(eng.occupancy(slot), o.occupancy())
    if eam:
        assert np.array_equal(eng.rho(slot), o.rho())
    evo_d, hops_d = eng.block_clocks(slot)
    evo_o, hops_o = o.block_state()
    assert np.array_equal(hops_d, hops_o)
    assert np.array_equal(evo_d.view(np.uint64), evo_o.view(np.uint64))
    st = eng.job_state(slot)
    assert st["round"] == o.round and st["hops"] == o.hops


JOBS = [
    dict(box=(32, 32, 32), blocks=(2, 2, 2), alloy=QUATERNARY, n_vacancies=40, temperature=563.0, seed=51),
    dict(box=(16, 16, 16), precision=po.FP32C, alloy=QUATERNARY, n_vacancies=4, temperature=620.0, seed=52),
    dict(box=(24, 16, 16), blocks=(2, 1, 1), model=po.MODEL_PAIRBOND, alloy=QUATERNARY, n_vacancies=10, seed=53),
    dict(box=(20, 20, 20), n_vacancies=8, seed=54, pot_seed=7),  # a potential the context has not seen
    dict(box=(24, 24, 24), blocks=(2, 2, 2), precision=po.FP32C, alloy=QUATERNARY, n_vacancies=20,
         temperature=500.0, seed=55),
]


@pytest.mark.parametrize("schedule", [1, 2])  # round by round; dependency-driven
def test_admitted_jobs_follow_their_own_trajectories(ak, schedule):
    with ak.Engine(event_log_capacity=1 << 20, max_jobs=4, max_blocks=32, max_vacancies=256) as eng:
        eng.set_round_schedule(schedule)
        ors = [oracle_job(**JOBS[k]) for k in range(5)]
        s0 = eng.add_job(_cfg(ak, ors[0], JOBS[0]), ors[0].occupancy())
        eng.prepare()
        eng.run_rounds(40)
        s1 = eng.admit_job(_cfg(ak, ors[1], JOBS[1]), ors[1].occupancy())
        s2 = eng.admit_job(_cfg(ak, ors[2], JOBS[2]), ors[2].occupancy())
        eng.run_rounds(33)
        eng.sync()
        ev1 = eng.events()
        ors[0].run_rounds(73)
        _check(eng, s0, ors[0], ev1)
        eng.retire_job(s0)  # its slot and blocks go back to the context
        with pytest.raises(ak.AkmcError) as e:
            eng.job_state(s0)
        assert e.value.status == -9
        s3 = eng.admit_job(_cfg(ak, ors[3], JOBS[3]), ors[3].occupancy())
        s4 = eng.admit_job(_cfg(ak, ors[4], JOBS[4]), ors[4].occupancy())
        assert s3 == s0 and len({s1, s2, s3, s4}) == 4
        eng.run_rounds(27)
        eng.sync()
        ev2 = eng.events()
        for o, n in ((ors[1], 60), (ors[2], 60), (ors[3], 27), (ors[4], 27)):
            o.run_rounds(n)
        both = np.concatenate([ev1, ev2])
        _check(eng, s1, ors[1], both)
        _check(eng, s2, ors[2], both, eam=False)
        _check(eng, s3, ors[3], ev2)  # the slot's earlier events belong to the retired job
        _check(eng, s4, ors[4], ev2)


def test_admission_into_an_empty_context_and_room_checks(ak):
    with ak.Engine(event_log_capacity=1 << 18, max_jobs=2, max_blocks=9, max_vacancies=64,
                   max_block_edge=16) as eng:
        eng.prepare()  # no jobs yet
        o = oracle_job(**JOBS[1])
        s = eng.admit_job(_cfg(ak, o, JOBS[1]), o.occupancy())
        eng.run_rounds(50)
        eng.sync()
        o.run_rounds(50)
        _check(eng, s, o, eng.events())
        big = dict(box=(40, 16, 16), n_vacancies=4, seed=3)  # one 40-cell block: over max_block_edge
        ob = oracle_job(**big)
        with pytest.raises(ak.AkmcError) as e:
            eng.admit_job(_cfg(ak, ob, big), ob.occupancy())
        assert e.value.status == -1
        o2 = oracle_job(**JOBS[0])  # 8 blocks: 1 + 8 fit in 9
        eng.admit_job(_cfg(ak, o2, JOBS[0]), o2.occupancy())
        o3 = oracle_job(**JOBS[1])
        with pytest.raises(ak.AkmcError) as e:  # a third job: no slot left
            eng.admit_job(_cfg(ak, o3, JOBS[1]), o3.occupancy())
        assert e.value.status == -5
        eng.run_rounds(8)
        eng.sync()
