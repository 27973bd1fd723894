"""GPU parity at the benchmark sizes: the 256^3 lattice and the 512 batched boxes.

The oracle keeps pace with these sizes for a few hundred sector rounds (256 rounds of the
256^3 lattice, about 214K hops, take it under a second after a 3 s set-up), so the comparison
is the small cases' own: every event field, the final occupancy, the per-block clocks and the
density cache, identical bit for bit.  A longer run of the 256^3 lattice is checked through
properties that hold at any size:

- species counts are conserved;
- the event log, replayed on the starting lattice in (round, block, hop) order, moves a vacancy
  at every step onto a site of the logged species and ends on the final lattice;
- the density cache kept by the per-hop refresh equals the oracle's from-scratch density sum
  over the final lattice;
- the job's hop count equals the number of logged events.
"""
import os
import sys

import numpy as np
import pytest

import pyoracle as po
from helpers import QUATERNARY, assert_same_events, device_job, oracle_job, sort_events

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EDGE = 256
BLOCKS = (16, 16, 16)
N_VAC = int(round(2e-5 * 2 * EDGE ** 3))  # 671


@pytest.fixture(scope="module")
def ak():
    sys.path.insert(0, os.path.join(ROOT, "misa-akmc-gpu_b200"))
    import build

    build.build()
    import akmc_b200

    return akmc_b200


def scale_oracle(**kw):
    args = dict(box=(EDGE,) * 3, blocks=BLOCKS, alloy=QUATERNARY, n_vacancies=N_VAC, temperature=563.0, seed=42)
    args.update(kw)
    return oracle_job(**args)


def check(eng, o, j, ev, rho=True):
    assert_same_events(ev[ev["job"] == j], o.events())
    assert np.array_equal(eng.occupancy(j), o.occupancy())
    evo_d, hops_d = eng.block_clocks(j)
    evo_o, hops_o = o.block_state()
    assert np.array_equal(hops_d, hops_o)
    assert np.array_equal(evo_d.view(np.uint64), evo_o.view(np.uint64))
    st = eng.job_state(j)
    assert st["hops"] == o.hops and st["round"] == o.round
    if rho:
        assert np.array_equal(eng.rho(j), o.rho())


@pytest.mark.parametrize("schedule", [1, 2])
def test_256_cubed_fp64_matches_oracle(ak, schedule):
    # one launch of the benchmark's 256^3 workload (256 sector rounds), both schedules
    o = scale_oracle()
    with ak.Engine(event_log_capacity=1 << 19) as eng:
        eng.set_round_schedule(schedule)
        device_job(eng, o, (EDGE,) * 3, blocks=BLOCKS, temperature=563.0)
        eng.prepare()
        assert eng.round_schedule() == schedule
        o.run_rounds(256)
        eng.run_rounds(256)
        eng.sync()
        assert o.hops > 150_000
        check(eng, o, 0, eng.events(1 << 19))


@pytest.mark.parametrize("model,prec", [(po.MODEL_EAM, po.FP32C), (po.MODEL_PAIRBOND, po.FP64)])
def test_256_cubed_fp32c_and_pairbond_match_oracle(ak, model, prec):
    o = scale_oracle(model=model, precision=prec)
    with ak.Engine(event_log_capacity=1 << 18) as eng:
        device_job(eng, o, (EDGE,) * 3, blocks=BLOCKS, model=model, precision=prec, temperature=563.0)
        eng.prepare()
        o.run_rounds(96)
        eng.run_rounds(96)
        eng.sync()
        assert o.hops > 50_000
        check(eng, o, 0, eng.events(1 << 18), rho=model == po.MODEL_EAM)


def test_512_batched_boxes_match_oracle(ak):
    # the batched workload as the benchmark runs it: 512 boxes of 16-48 cells, FP32-comp, one
    # engine, on the block edge the autotuner picks for it (20 cells)
    sys.path.insert(0, ROOT)
    import bench
    from akmc_b200.autotune import blocks_for

    jobs = bench.workload_jobs("batched")
    assert len(jobs) == 512
    oracles = []
    with ak.Engine(event_log_capacity=1 << 20) as eng:
        for j in jobs:
            nb = tuple(blocks_for(e, 20) for e in j["box"])
            o = oracle_job(box=j["box"], blocks=nb, precision=j["precision"], seed=j["seed"],
                           temperature=j["temperature"], alloy=j["alloy"], n_vacancies=j["n_vacancies"])
            device_job(eng, o, j["box"], blocks=nb, precision=j["precision"], seed=j["seed"],
                       temperature=j["temperature"])
            oracles.append(o)
        eng.prepare()
        for o in oracles:
            o.run_rounds(64)
        eng.run_rounds(64)
        eng.sync()
        assert sum(o.hops for o in oracles) > 100_000
        ev = eng.events(1 << 20)
        for j, o in enumerate(oracles):
            check(eng, o, j, ev)
        # every job's lattice once more, through the whole-context read
        occ = eng.occupancies()
        assert np.array_equal(occ, np.concatenate([o.occupancy() for o in oracles]))


def replay(occ0, ev):
    """The event log applied to the starting lattice; every step is checked as it is applied."""
    occ = bytearray(occ0.tobytes())
    ev = sort_events(ev)
    frm = ev["from_site"].tolist()
    to = ev["to_site"].tolist()
    sp = ev["species"].tolist()
    for k, (f, t, x) in enumerate(zip(frm, to, sp)):
        if occ[f] != 0 or occ[t] != x:
            raise AssertionError("event %d: site %d holds %d, site %d holds %d, logged species %d"
                                 % (k, f, occ[f], t, occ[t], x))
        occ[f], occ[t] = x, 0
    return np.frombuffer(bytes(occ), np.uint8)


def test_256_cubed_long_run_properties(ak):
    # 1024 sector rounds (128 time steps, about 850K hops) under the default schedule
    box = (EDGE,) * 3
    occ0 = ak.create_lattice(box, QUATERNARY, N_VAC, 42)
    with ak.Engine(event_log_capacity=1 << 21) as eng:
        eng.add_job(ak.job_config(box, blocks=BLOCKS, temperature=563.0, seed=42, eam=ak.eam_johnson(42)), occ0)
        eng.prepare()
        eng.run_rounds(1024)
        eng.sync()
        st = eng.job_state(0)
        ev = eng.events(1 << 21)
        occ = eng.occupancy(0)
        rho = eng.rho(0)
    assert st["round"] == 1024
    assert len(ev) == st["hops"] > 500_000
    assert np.array_equal(np.bincount(occ, minlength=9), np.bincount(occ0, minlength=9))
    assert np.array_equal(replay(occ0, ev), occ)
    o = scale_oracle(log_events=0)
    o.set_occupancy(occ)
    assert np.array_equal(rho, o.rho())
