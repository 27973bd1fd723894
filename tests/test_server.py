"""The job server (akmc_server_*): validation on the CPU; on the GPU, every served job's result
equals the oracle's run of the same job alone -- hop count, rounds, final lattice and the
sector clocks of every block (their checksum) -- while jobs are admitted into, and retired from,
the lanes' running contexts."""
import numpy as np
import pytest

import pyoracle as po
from helpers import QUATERNARY, oracle_job


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


def _job(ak, box, model, seed, budget=0, max_rounds=0, blocks=(1, 1, 1), precision=0):
    o = oracle_job(box=box, blocks=blocks, model=model, precision=precision, seed=seed, temperature=563.0,
                   alloy=QUATERNARY, n_vacancies=max(2, int(2e-4 * 2 * np.prod(box))), log_events=0)
    eam = ak.eam_johnson(42) if model == ak.MODEL_EAM else None
    cfg = ak.job_config(box, blocks=blocks, energy_model=model, precision=precision, seed=seed, temperature=563.0,
                        eam=eam, hop_budget=budget, max_rounds=max_rounds)
    return cfg, o.occupancy(), o


def test_submit_rejects_jobs_that_cannot_run(ak):
    with ak.Server(lanes=1) as srv:
        cfg, occ, _ = _job(ak, (16, 16, 16), ak.MODEL_PAIRBOND, 1)  # neither hop budget nor max_rounds
        with pytest.raises(ak.AkmcError) as e:
            srv.submit(cfg, occ)
        assert e.value.status == -1
        cfg, occ, _ = _job(ak, (16, 16, 16), ak.MODEL_PAIRBOND, 1, max_rounds=8)
        with pytest.raises(ak.AkmcError):
            srv.submit(cfg, occ[:-2])  # wrong lattice size
        cfg, occ, _ = _job(ak, (32, 16, 16), ak.MODEL_PAIRBOND, 1, max_rounds=8)  # one 32-cell block
        with pytest.raises(ak.AkmcError) as e:
            srv.submit(cfg, occ)
        assert e.value.status == -1
        assert srv.stats() == dict(queued=0, running=0, done=0)
        prof = srv.profile()  # an idle server has run nothing
        assert prof["chunks"] == 0 and prof["run_s"] == 0.0


SPECS = [((16, 16, 16), po.MODEL_EAM, 1, 3000, 0, (1, 1, 1), 0),
         ((24, 20, 16), po.MODEL_PAIRBOND, 2, 0, 40, (1, 1, 1), 0),
         ((32, 32, 32), po.MODEL_EAM, 3, 5000, 0, (2, 2, 2), 0),
         ((20, 20, 20), po.MODEL_EAM, 4, 0, 64, (1, 1, 1), 1),
         ((16, 24, 20), po.MODEL_EAM, 5, 800, 0, (1, 1, 1), 0),
         ((40, 16, 16), po.MODEL_PAIRBOND, 6, 2000, 0, (2, 1, 1), 0),
         ((18, 18, 18), po.MODEL_EAM, 7, 1500, 0, (1, 1, 1), 1)]


@pytest.mark.gpu
# max_batch bounds the jobs a lane runs at once, so finished jobs' slots take queued ones;
# order 1 admits the smallest hop budget first
@pytest.mark.parametrize("lanes,max_batch,order", [(2, 3, 0), (1, 2, 0), (1, 2, 1), (1, 0, 0)])
def test_served_jobs_equal_the_oracle_alone(ak, lanes, max_batch, order):
    jobs = [_job(ak, *sp) for sp in SPECS]
    with ak.Server(lanes=lanes, max_batch_jobs=max_batch, chunk_rounds=8, order=order) as srv:
        tickets = [srv.submit(cfg, occ) for cfg, occ, _ in jobs]
        got = [srv.wait(t, timeout=300.0) for t in tickets]
        prof = srv.profile()
    assert prof["builds"] == lanes  # one context per lane for the server's life
    for sp, (cfg, occ, o), (res, out) in zip(SPECS, jobs, got):
        assert res["status"] == 0, res["error"]
        assert res["submit_s"] <= res["start_s"] <= res["finish_s"]
        budget, max_rounds = sp[3], sp[4]
        if budget:
            o.run(budget, 1 << 30)
        else:
            o.run_rounds(max_rounds)
        assert res["hops"] == o.hops and res["rounds"] == o.round
        assert np.array_equal(out, o.occupancy())
        evo, hops = o.block_state()
        assert res["clocks_fnv"] == ak.clocks_fnv(evo, hops)
