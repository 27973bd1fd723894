"""Cu cluster statistics of a resident lattice, computed on the device
(akmc_job_cluster_stats), against the host count of akmc_cluster_stats, which the oracle
pins (test_boundary.py)."""
import numpy as np
import pytest


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


@pytest.mark.gpu
def test_device_cluster_stats_match_host(ak):
    # 1.34 % Cu in an odd box (13,566 sites: the last 14 are past the 16-byte loads), 25 % Cu
    # (clusters span the box), and a larger box after a smaller one (the scratch grows)
    cases = [((17, 19, 21), 134, 7), ((20, 20, 20), 2500, 5), ((32, 24, 16), 1500, 9)]
    with ak.Engine() as eng:
        with pytest.raises(ak.AkmcError) as e:  # before akmc_prepare
            eng.cluster_stats(0, 8)
        assert e.value.status == -6
        occs = []
        for box, cu, seed in cases:
            occ = ak.create_lattice(box, ((ak.FE, 10000 - cu), (ak.CU, cu)), 6, seed)
            eng.add_job(ak.job_config(box, energy_model=ak.MODEL_PAIRBOND, seed=seed), occ)
            occs.append(occ)
        eng.prepare()
        with pytest.raises(ak.AkmcError) as e:
            eng.cluster_stats(0, 4097)
        assert e.value.status == -1
        for j, (box, _, _) in enumerate(cases):
            for bins in (1, 64, 4096):
                iso, hist = eng.cluster_stats(j, bins)
                iso_h, hist_h = ak.cluster_stats(occs[j], box, bins)
                assert iso == iso_h and np.array_equal(hist, hist_h)
            assert hist.sum() > 0
        # the statistics follow the lattice as the device changes it
        eng.run_rounds(24)
        eng.sync()
        moved = 0
        for j, (box, _, _) in enumerate(cases):
            occ = eng.occupancy(j)
            moved += int((occ != occs[j]).sum())
            iso, hist = eng.cluster_stats(j, 64)
            iso_h, hist_h = ak.cluster_stats(occ, box, 64)
            assert iso == iso_h and np.array_equal(hist, hist_h)
        assert moved > 0
