"""akmc_run_rounds_noalloc against akmc_run_rounds, through the C ABI.

akmc_run_rounds_noalloc serves callers that must not allocate device memory once
their jobs are admitted: a serving loop that admits jobs against a fixed memory
budget, or a process whose device memory is already held by another caching
allocator.  It keeps the per-round scratch in a fixed device array of the
library instead of context memory.  Everything else (kernels, context state) is
shared with akmc_run_rounds under the round-by-round schedule, so the two must
give the same trajectory bit for bit: occupancy, densities, event fields, the
floating-point draws, totals, residence times and the block clocks.  The free
device memory must not change across the no-allocation calls.
The file is named to be collected last: it must pass alone and after every other
GPU test (the scratch is a process-wide device array).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

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


def _jobs(ak):
    """An 8-block EAM FP64 job, a pair-bond job and a 2-block EAM FP32-comp job."""
    specs = [
        dict(box=(32, 32, 32), blocks=(2, 2, 2), energy_model=ak.MODEL_EAM, precision=ak.FP64, seed=11,
             temperature=563.0, n_vac=40),
        dict(box=(16, 24, 18), blocks=(1, 1, 1), energy_model=ak.MODEL_PAIRBOND, precision=ak.FP64, seed=12,
             temperature=500.0, n_vac=9),
        dict(box=(32, 16, 16), blocks=(2, 1, 1), energy_model=ak.MODEL_EAM, precision=ak.FP32C, seed=13,
             temperature=650.0, n_vac=12),
    ]
    out = []
    for s in specs:
        occ = ak.create_lattice(s["box"], QUATERNARY, s["n_vac"], s["seed"])
        eam = ak.eam_johnson(42) if s["energy_model"] == ak.MODEL_EAM else None
        cfg = ak.job_config(s["box"], blocks=s["blocks"], energy_model=s["energy_model"], precision=s["precision"],
                            seed=s["seed"], temperature=s["temperature"], eam=eam)
        out.append((cfg, occ))
    return out


def _engine(ak, jobs):
    eng = ak.Engine(event_log_capacity=1 << 20)
    # the no-allocation entry point runs the rounds one by one; the reference path runs the
    # same kernels in the same order
    eng.set_round_schedule(ak.SCHEDULE_ROUNDS)
    for cfg, occ in jobs:
        eng.add_job(cfg, occ)
    eng.prepare()
    return eng


def _state(eng, n_jobs):
    st = []
    for j in range(n_jobs):
        evo, hops = eng.block_clocks(j)
        st.append(dict(occ=eng.occupancy(j), rho=eng.rho(j) if j != 1 else None, evo=evo, hops=hops,
                       job=eng.job_state(j)))
    ev = eng.events()
    ev = ev[np.lexsort((ev["hop"], ev["block"], ev["job"], ev["round"]))]
    return st, ev


def _assert_same(a, b):
    (sa, ea), (sb, eb) = a, b
    for x, y in zip(sa, sb):
        assert np.array_equal(x["occ"], y["occ"])
        if x["rho"] is not None:
            assert np.array_equal(x["rho"], y["rho"])
        assert np.array_equal(x["hops"], y["hops"])
        assert np.array_equal(x["evo"].view(np.uint64), y["evo"].view(np.uint64))
        assert x["job"] == y["job"]
    assert len(ea) == len(eb) and len(ea) > 0
    for f in ("round", "job", "hop", "from_site", "to_site", "block", "species", "n_act", "n_dirty"):
        assert np.array_equal(ea[f], eb[f]), f
    for f in ("u", "total", "dt"):
        assert np.array_equal(np.ascontiguousarray(ea[f]).view(np.uint64), np.ascontiguousarray(eb[f]).view(np.uint64)), f


def _free_bytes():
    import torch

    torch.cuda.synchronize()
    return torch.cuda.mem_get_info(0)[0]


def test_noalloc_rounds_match_run_rounds_on_two_calls(ak):
    jobs = _jobs(ak)
    ref = _engine(ak, jobs)
    dut = _engine(ak, jobs)
    try:
        for n in (40, 24):  # two calls in a row, each compared with the same rounds of akmc_run_rounds
            ref.run_rounds(n)
            ref.sync()
            free0 = _free_bytes()
            dut.run_rounds_noalloc(n)
            dut.sync()
            assert _free_bytes() == free0  # nothing allocated on the device by the call
            _assert_same(_state(dut, len(jobs)), _state(ref, len(jobs)))
        # the context stays usable by the allocating entry point afterwards
        ref.run_rounds(8)
        dut.run_rounds(8)
        ref.sync()
        dut.sync()
        _assert_same(_state(dut, len(jobs)), _state(ref, len(jobs)))
    finally:
        ref.close()
        dut.close()


def test_noalloc_rejects_more_blocks_than_its_scratch(ak):
    box = (8 * 24, 8 * 24, 8 * 15)  # 24 * 24 * 15 = 8640 blocks > NOALLOC_MAX_BLOCKS
    occ = ak.create_lattice(box, QUATERNARY, 64, 7)
    cfg = ak.job_config(box, blocks=(24, 24, 15), energy_model=ak.MODEL_PAIRBOND, seed=7, temperature=563.0)
    with ak.Engine() as eng:
        eng.add_job(cfg, occ)
        eng.prepare()
        with pytest.raises(ak.AkmcError) as e:
            eng.run_rounds_noalloc(1)
        assert e.value.status == -1  # AKMC_EINVAL
        assert "AKMC_NOALLOC_MAX_BLOCKS" in str(e.value)
