"""The C-ABI library: loads, exports every declared symbol, and its host-side
model construction matches the oracle bit for bit.  No GPU calls."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def ak():
    import sys

    sys.path.insert(0, os.path.join(ROOT, "misa-akmc-gpu_b200"))
    import build

    build.build()
    import akmc_b200

    akmc_b200.lib()
    return akmc_b200


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "akmc.h")).read()
    return sorted(set(re.findall(r"AKMC_API\s+[\w\s\*]+?\b(akmc_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(ak):
    L = C.CDLL(ak.lib_path())
    syms = declared_symbols()
    assert len(syms) >= 24
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(ak.SIGNATURES), "binding and header disagree"


def test_status_strings(ak):
    assert ak.lib().akmc_status_string(0) == b"ok"
    assert ak.lib().akmc_status_string(-7) == b"overflow"


def test_eam_tables_match_oracle(ak):
    t = ak.eam_johnson(42, 2.855, 5.6)
    o = po.Oracle(po.make_config(box=(8, 8, 8), n_vacancies=1))
    ref = o.eam_tables()
    f = np.ctypeslib.as_array(t.f_shell)
    phi = np.ctypeslib.as_array(t.phi_shell)
    assert t.n_shells == 5
    assert np.array_equal(f.view(np.uint64), ref["f_sh"].view(np.uint64))
    assert np.array_equal(phi.view(np.uint64), ref["phi_sh"].view(np.uint64))
    F = np.ctypeslib.as_array(t.F)
    assert np.array_equal(F, -np.sqrt(np.arange(5000) * 2.0 ** -7))


@pytest.mark.parametrize("box,alloy,nv,seed", [
    ((20, 20, 20), ((po.FE, 9866), (po.CU, 134)), 20, 42),
    ((16, 24, 18), ((po.FE, 9766), (po.CU, 134), (po.NI, 70), (po.MN, 30)), 7, 1234),
])
def test_lattice_creation_matches_oracle(ak, box, alloy, nv, seed):
    occ = ak.create_lattice(box, alloy, nv, seed)
    o = po.Oracle(po.make_config(box=box, alloy=alloy, n_vacancies=nv, seed=seed))
    assert np.array_equal(occ, o.occupancy())
    assert int((occ == 0).sum()) == nv


def test_cluster_stats_match_oracle(ak):
    box = (16, 16, 16)
    o = po.Oracle(po.make_config(box=box, alloy=((po.FE, 90), (po.CU, 10)), n_vacancies=3))
    iso, hist = ak.cluster_stats(o.occupancy(), box, 32)
    iso_o, hist_o = o.cluster_stats(32)
    assert iso == iso_o and np.array_equal(hist, hist_o)


def test_invalid_inputs_are_rejected_without_gpu(ak):
    with pytest.raises(ak.AkmcError):
        ak.create_lattice((8, 8, 8), ((po.FE, 0),), 0, 1)  # no atoms to draw from
    with pytest.raises(ak.AkmcError):
        ak.eam_johnson(1, 2.855, 6.0)  # cutoff beyond the 5th shell


def test_engine_fails_loudly_without_a_gpu(ak):
    # no CPU fallback: with no CUDA device, creating a context is an error, not a slower path
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(ak.AkmcError) as ei:
        ak.Engine()
    assert ei.value.status == -3  # AKMC_ECUDA
