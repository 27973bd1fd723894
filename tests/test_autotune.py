"""Autotuner of the domain-block edge (akmc_b200.autotune)."""
import os
import sys

import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "misa-akmc-gpu_b200",
                                "python"))
from akmc_b200.autotune import blocks_for  # noqa: E402


def test_blocks_for_keeps_blocks_within_the_edge_and_at_least_8_cells():
    assert blocks_for(16, 24) == 1 and blocks_for(24, 24) == 1 and blocks_for(25, 24) == 2
    assert blocks_for(48, 16) == 3 and blocks_for(48, 8) == 6
    assert blocks_for(20, 8) == 2  # 3 blocks would be under 8 cells
    assert blocks_for(8, 8) == 1 and blocks_for(12, 8) == 1
    for edge in range(8, 97):
        for c in (8, 12, 16, 20, 24):
            nb = blocks_for(edge, c)
            assert 1 <= nb and edge // nb >= 8  # every block at least 8 cells
            if nb == -(-edge // c):  # not limited by the 8-cell minimum: blocks of at most c cells
                assert -(-edge // nb) <= c


@pytest.mark.gpu
def test_tuner_searches_edge_warps_and_takes():
    import akmc_b200 as ak
    from akmc_b200.autotune import tune

    jobs = [dict(box=(e, e, e), precision=1, temperature=563.0, seed=3 + i) for i, e in enumerate((16, 24, 32, 40))]
    lats = [ak.create_lattice(j["box"], ((ak.FE, 9766), (ak.CU, 134), (ak.NI, 70), (ak.MN, 30)),
                              max(2, int(2e-4 * 2 * j["box"][0] ** 3)), j["seed"]) for j in jobs]
    choice, table = tune(jobs, lats, ak.eam_johnson(42), candidates=(8, 16), takes=(0, 1), rounds=16, warmup=8)
    e = choice["block_edge"]
    # every edge with the default shape, then 4 warps and a take of 1 at the chosen edge
    assert {"edge=8 warps=8 take=0", "edge=16 warps=8 take=0", "edge=%d warps=4 take=0" % e} <= set(table)
    assert "edge=%d warps=%d take=1" % (e, choice["eval_warps"]) in table
    key = "edge=%d warps=%d take=%d" % (e, choice["eval_warps"], choice["flow_take"])
    assert table[key] == max(table.values()) and all(v > 0 for v in table.values())


@pytest.mark.gpu
def test_tuner_raises_on_a_failing_candidate():
    import akmc_b200 as ak
    from akmc_b200.autotune import tune_block_edge

    jobs = [dict(box=(16, 16, 16), precision=1, temperature=563.0, seed=3)]
    lats = [ak.create_lattice((16, 16, 16), ((ak.FE, 1),), 2, 3)[:-1]]  # a lattice one site short
    with pytest.raises(ak.AkmcError):
        tune_block_edge(jobs, lats, ak.eam_johnson(42), candidates=(8, 16), rounds=4, warmup=1)


@pytest.mark.gpu
def test_tuner_returns_the_fastest_candidate():
    import akmc_b200 as ak
    from akmc_b200.autotune import tune_block_edge

    jobs = [dict(box=(e, e, e), precision=1, temperature=563.0, seed=3 + i) for i, e in enumerate((16, 24, 32, 40))]
    lats = [ak.create_lattice(j["box"], ((ak.FE, 9766), (ak.CU, 134), (ak.NI, 70), (ak.MN, 30)),
                              max(2, int(2e-4 * 2 * j["box"][0] ** 3)), j["seed"]) for j in jobs]
    best, table = tune_block_edge(jobs, lats, ak.eam_johnson(42), candidates=(8, 16, 24), rounds=16, warmup=8)
    assert set(table) == {8, 16, 24} and best in table
    assert all(v > 0 for v in table.values()) and table[best] == max(table.values())
