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
def test_tuner_returns_the_fastest_candidate():
    import akmc_b200 as ak
    from akmc_b200.autotune import tune_block_edge

    jobs = [dict(box=(e, e, e), precision=1, temperature=563.0, seed=3 + i) for i, e in enumerate((16, 24, 32, 40))]
    lats = [ak.create_lattice(j["box"], ((ak.FE, 9766), (ak.CU, 134), (ak.NI, 70), (ak.MN, 30)),
                              max(2, int(2e-4 * 2 * j["box"][0] ** 3)), j["seed"]) for j in jobs]
    best, table = tune_block_edge(jobs, lats, ak.eam_johnson(42), candidates=(8, 16, 24), rounds=16, warmup=8)
    assert set(table) == {8, 16, 24} and best in table
    assert all(v > 0 for v in table.values()) and table[best] == max(table.values())
