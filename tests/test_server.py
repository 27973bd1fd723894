"""The job server (akmc_server_*): validation on the CPU; on the GPU, every job's result
equals the same job run alone in its own context: jobs of a batch do not interact, and a job
carried through a batch refill (snapshot, rebuilt context, restore) continues exactly."""
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


def _job(ak, box, model, seed, budget=0, max_rounds=0, blocks=(1, 1, 1), precision=0):
    occ = ak.create_lattice(box, QUATERNARY, max(2, int(2e-4 * 2 * np.prod(box))), seed)
    eam = ak.eam_johnson(42) if model == ak.MODEL_EAM else None
    cfg = ak.job_config(box, blocks=blocks, energy_model=model, precision=precision, seed=seed, temperature=563.0,
                        eam=eam, hop_budget=budget, max_rounds=max_rounds)
    return cfg, occ


def test_submit_rejects_jobs_that_cannot_run(ak):
    with ak.Server(lanes=1) as srv:
        cfg, occ = _job(ak, (16, 16, 16), ak.MODEL_PAIRBOND, 1)  # neither hop budget nor max_rounds
        with pytest.raises(ak.AkmcError) as e:
            srv.submit(cfg, occ)
        assert e.value.status == -1
        cfg, occ = _job(ak, (16, 16, 16), ak.MODEL_PAIRBOND, 1, max_rounds=8)
        with pytest.raises(ak.AkmcError):
            srv.submit(cfg, occ[:-2])  # wrong lattice size
        assert srv.stats() == dict(queued=0, running=0, done=0)
        prof = srv.profile()  # an idle server has built nothing and run nothing
        assert prof["builds"] == 0 and prof["chunks"] == 0 and prof["run_s"] == 0.0


@pytest.mark.gpu
# (1, 2): every finish refills the batch; order 1 admits the smallest hop budget first
@pytest.mark.parametrize("lanes,max_batch,order", [(2, 3, 0), (1, 2, 0), (1, 2, 1)])
def test_server_results_equal_jobs_run_alone(ak, lanes, max_batch, order):
    specs = [((16, 16, 16), ak.MODEL_EAM, 1, 3000, 0, (1, 1, 1), 0),
             ((24, 20, 16), ak.MODEL_PAIRBOND, 2, 0, 40, (1, 1, 1), 0),
             ((32, 32, 32), ak.MODEL_EAM, 3, 5000, 0, (2, 2, 2), 0),
             ((20, 20, 20), ak.MODEL_EAM, 4, 0, 64, (1, 1, 1), 1),
             ((16, 24, 20), ak.MODEL_EAM, 5, 800, 0, (1, 1, 1), 0),
             ((40, 16, 16), ak.MODEL_PAIRBOND, 6, 2000, 0, (2, 1, 1), 0)]
    jobs = [_job(ak, *sp) for sp in specs]
    with ak.Server(lanes=lanes, max_batch_jobs=max_batch, chunk_rounds=8, order=order) as srv:
        tickets = [srv.submit(cfg, occ) for cfg, occ in jobs]
        got = [srv.wait(t, timeout=300.0) for t in tickets]
    for (cfg, occ), (res, out) in zip(jobs, got):
        assert res["status"] == 0, res["error"]
        assert res["submit_s"] <= res["start_s"] <= res["finish_s"]
        with ak.Engine(graph_rounds=8) as eng:
            eng.add_job(cfg, occ)
            eng.prepare()
            eng.run(0)
            st = eng.job_state(0)
            assert st["done"]
            assert res["hops"] == st["hops"] and res["rounds"] == st["round"]
            assert np.array_equal(out, eng.occupancy(0))
