"""Restart snapshots (akmc_save_snapshot / akmc_restore_snapshot): a run saved after R1 rounds
and continued from the snapshot in a fresh context gives the events, lattice, clocks and
counters of the uninterrupted run, bit for bit."""
import numpy as np
import pytest

QUATERNARY = ((1, 9766), (2, 134), (4, 70), (8, 30))


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


def _ordered(ev):
    return ev[np.lexsort((ev["hop"], ev["block"], ev["round"]))]


def _run(ak, cfg, occ, schedule, rounds, snapshot=None):
    with ak.Engine(event_log_capacity=1 << 20, graph_rounds=8) as eng:
        eng.add_job(cfg, occ)
        eng.set_round_schedule(schedule)
        eng.prepare()
        if snapshot is not None:
            eng.restore_snapshot(0, snapshot)
        eng.run_rounds(rounds)
        eng.sync()
        st = eng.job_state(0)
        return dict(events=_ordered(eng.events()), occ=eng.occupancy(0), clocks=eng.block_clocks(0),
                    state=st, snap=eng.save_snapshot(0), cluster=eng.cluster_stats(0, 32))


@pytest.mark.gpu
@pytest.mark.parametrize("box,blocks,schedule,budget", [((32, 32, 32), (2, 2, 2), 1, 0),
                                                         ((32, 32, 32), (2, 2, 2), 2, 0),
                                                         ((24, 20, 20), (1, 1, 1), 0, 8000)])
def test_continued_run_equals_uninterrupted(ak, box, blocks, schedule, budget):
    occ = ak.create_lattice(box, QUATERNARY, 24, 11)
    cfg = ak.job_config(box, blocks=blocks, energy_model=ak.MODEL_EAM, eam=ak.eam_johnson(42), temperature=563.0,
                        seed=11, hop_budget=budget)
    r1, r2 = 40, 56
    whole = _run(ak, cfg, occ, schedule, r1 + r2)
    first = _run(ak, cfg, occ, schedule, r1)
    rest = _run(ak, cfg, occ, schedule, r2, snapshot=first["snap"])
    assert len(first["events"]) > 0 and len(rest["events"]) > 0
    both = _ordered(np.concatenate([first["events"], rest["events"]]))
    assert np.array_equal(both.view(np.uint8), whole["events"].view(np.uint8))
    assert np.array_equal(rest["occ"], whole["occ"])
    assert np.array_equal(rest["clocks"][0].view(np.uint64), whole["clocks"][0].view(np.uint64))
    assert np.array_equal(rest["clocks"][1], whole["clocks"][1])
    assert rest["state"] == whole["state"]
    assert rest["snap"] == whole["snap"]
    assert rest["cluster"][0] == whole["cluster"][0] and np.array_equal(rest["cluster"][1], whole["cluster"][1])


@pytest.mark.gpu
def test_restore_rejects_damaged_or_foreign_snapshots(ak):
    box = (20, 20, 20)
    occ = ak.create_lattice(box, QUATERNARY, 10, 3)
    eam = ak.eam_johnson(42)
    cfg = ak.job_config(box, energy_model=ak.MODEL_EAM, eam=eam, temperature=563.0, seed=3)
    snap = _run(ak, cfg, occ, 0, 8)["snap"]
    other = ak.job_config(box, energy_model=ak.MODEL_EAM, eam=eam, temperature=600.0, seed=3)
    damaged = bytearray(snap)
    damaged[-5] ^= 1
    with ak.Engine() as eng:
        eng.add_job(cfg, occ)
        eng.add_job(other, occ)
        eng.prepare()
        for job, data in ((0, bytes(damaged)), (1, snap), (0, snap[:-1]), (0, b"x" * 64)):
            with pytest.raises(ak.AkmcError) as e:
                eng.restore_snapshot(job, data)
            assert e.value.status == -1
        eng.restore_snapshot(0, snap)
        assert eng.job_state(0)["round"] == 8


@pytest.mark.gpu
def test_flow_watchdog_gives_up_and_a_snapshot_recovers(ak):
    # one sweep per CTA cannot finish 64 rounds of 8 blocks holding 24 vacancies: the launch
    # gives up with AKMC_ETIMEOUT, the context keeps answering, and the snapshot taken before
    # the failure continues to the uninterrupted result
    box = (32, 32, 32)
    occ = ak.create_lattice(box, QUATERNARY, 24, 11)
    cfg = ak.job_config(box, blocks=(2, 2, 2), energy_model=ak.MODEL_EAM, eam=ak.eam_johnson(42),
                        temperature=563.0, seed=11)
    whole = _run(ak, cfg, occ, 2, 64)
    with ak.Engine(event_log_capacity=1 << 20, graph_rounds=8, flow_sweep_limit=1) as eng:
        eng.add_job(cfg, occ)
        eng.set_round_schedule(2)
        eng.prepare()
        snap = eng.save_snapshot(0)
        with pytest.raises(ak.AkmcError) as e:
            eng.run_rounds(64)
            eng.sync()
        assert e.value.status == -4
        assert eng.job_state(0)["n_blocks"] == 8
        assert eng.occupancy(0).shape == occ.shape
    rest = _run(ak, cfg, occ, 2, 64, snapshot=snap)
    assert np.array_equal(rest["events"].view(np.uint8), whole["events"].view(np.uint8))
    assert np.array_equal(rest["occ"], whole["occ"])
