"""Host layer without a GPU: config.yaml reader (schema of the reference's
profiles/config/config_parsing.cpp:54-230), lattice creation in the reference's
draw order, the lattice dump format."""
import os

import numpy as np
import pytest

import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CONFIG = """
# parallel kMC configure file (keys of the reference schema)
title: "parallel kMC configure file"
version: "0.1.0"

box:
  size: [12, 10, 14]
  lattice_const: 2.85532   # lattice constance
  cutoff_radius: 5.6

create:
  random:
    enable: true
    va_count: 7
    alloy:
      Fe: 9598
      Cu: 134
      Mn: 134
      Ni: 134
      FeFe: 0
      CuCu: 0
  pipe:
    enable: false
    input_box: last_frame.xyz
  restart:
    enable: false
    file_path: 1072.xyz

seeds:
  seeds_file: ""
  create_types: 100565
  create_vacancy: 16650
  event_selection: 563264
  time_inc: 594689

simulation:
  temperature: 673
  physics_time: 8e4
  steps_limit: 1000
  attempt_freq: 6e12
  isgenr: false
  dpasm1: 3e-9

output:
  dump:
    interval: 100
    file_path: "kmc.{}.out"
  logs:
    interval: 10
    logs_file: ""
"""


@pytest.fixture(scope="module")
def ak():
    import sys

    sys.path.insert(0, os.path.join(ROOT, "misa-akmc-gpu_b200"))
    import build

    build.build()
    import akmc_b200

    return akmc_b200


def test_config_reader_fields(ak):
    c = ak.config_parse(CONFIG)
    assert list(c.box) == [12, 10, 14]
    assert c.lattice_const == 2.85532 and c.cutoff_radius == 5.6
    assert c.create_random == 1 and c.va_count == 7
    assert c.n_types == 4
    assert list(c.type_codes) == [po.FE, po.CU, po.MN, po.NI]  # YAML order, as yaml-cpp iterates
    assert list(c.ratio) == [9598, 134, 134, 134]
    assert (c.seed_create_types, c.seed_create_vacancy, c.seed_event_selection, c.seed_time_inc) == (
        100565, 16650, 563264, 594689)
    assert c.temperature == 673.0 and c.physics_time == 8e4 and c.attempt_freq == 6e12
    assert c.steps_limit == 1000 and c.isgenr == 0 and c.dpasm1 == 3e-9
    assert c.dump_interval == 100 and c.dump_file_path == b"kmc.{}.out" and c.logs_interval == 10
    assert c.energy_model == 0 and list(c.blocks) == [1, 1, 1] and c.sector_window == 3e-7


def test_config_kmc_block(ak):
    c = ak.config_parse(CONFIG + "\nkmc:\n  energy_model: eam\n  precision: fp32c\n  blocks: [2, 1, 1]\n"
                                 "  hop_budget: 5000\n  seed: 9\n")
    assert c.energy_model == 1 and c.precision == 1 and list(c.blocks) == [2, 1, 1]
    assert c.hop_budget == 5000 and c.seed == 9
    job = ak.config_job(c, ak.eam_johnson(42))
    assert job.max_rounds == 8 * int(np.ceil(8e4 / 3e-7))


@pytest.mark.parametrize("bad,msg", [
    ("box:\n  size: [1, 2]\n", "box size must be 3"),
    (CONFIG.replace("enable: true", "enable: false"), "no create option"),
    (CONFIG.replace("FeFe: 0", "FeFe: 5"), "dumbbell"),
])
def test_config_errors(ak, bad, msg):
    with pytest.raises(ak.AkmcError) as e:
        ak.config_parse(bad)
    assert msg in str(e.value)


def test_reference_order_creation_matches_oracle(ak):
    # the product host code and the oracle both draw with libstdc++ distributions
    c = ak.config_parse(CONFIG)
    occ = ak.config_lattice(c)
    cfg = po.make_config(box=(12, 10, 14), creation_mode=po.CREATE_MT19937_REF, seed=100565, seed_vacancy=16650,
                         alloy=((po.FE, 9598), (po.CU, 134), (po.MN, 134), (po.NI, 134)), n_vacancies=7,
                         lattice_const=2.85532, energy_model=po.MODEL_PAIRBOND)
    o = po.Oracle(cfg)
    assert np.array_equal(occ, o.occupancy())
    assert int((occ == 0).sum()) == 7
    fr = np.bincount(occ, minlength=9)
    assert fr[po.CU] > 0 and fr[po.MN] > 0 and fr[po.NI] > 0


def test_dump_format(ak, tmp_path):
    box = (4, 4, 4)
    occ = np.full(2 * 64, po.FE, np.uint8)
    occ[0] = po.V
    occ[1] = po.CU
    p = tmp_path / "d.xyz"
    ak.dump_lattice(occ, box, str(p), ghost=2)
    lines = p.read_text().splitlines()
    assert lines[0] == "128" and lines[1] == ""
    assert lines[2] == "V\t2\t2\t2"          # corner site (0,0,0) at local ghost offset 2
    assert lines[3] == "Cu\t2.5\t2.5\t2.5"   # centre site
    assert len(lines) == 2 + 128


def _pipe_config(path):
    # create.random disabled, create.pipe enabled: the reference still takes the alloy from
    # create.random.alloy (config_parsing.cpp:177)
    return CONFIG.replace("    enable: true\n    va_count: 7", "    enable: false\n    va_count: 7").replace(
        "  pipe:\n    enable: false\n    input_box: last_frame.xyz", "  pipe:\n    enable: true\n    input_box: %s" % path)


def test_pipe_creation_matches_oracle(ak, tmp_path):
    # vacancy positions (x doubled): inside the box, a repeat, and two outside it (skipped)
    pile = [(0, 0, 0), (5, 3, 7), (23, 9, 13), (5, 3, 7), (24, 0, 0), (-1, 2, 2), (10, 2, 11)]
    p = tmp_path / "last_frame.xyz"
    p.write_text("".join("%d %d %d\n" % xyz for xyz in pile))
    c = ak.config_parse(_pipe_config(str(p)))
    assert c.create_pipe == 1 and c.create_random == 0 and c.pipe_input_box == str(p).encode()
    assert list(c.type_codes) == [po.FE, po.CU, po.MN, po.NI] and list(c.ratio) == [9598, 134, 134, 134]
    occ = ak.config_lattice(c)
    cfg = po.make_config(box=(12, 10, 14), creation_mode=po.CREATE_MT19937_PILE, seed=100565,
                         alloy=((po.FE, 9598), (po.CU, 134), (po.MN, 134), (po.NI, 134)), n_vacancies=0,
                         lattice_const=2.85532, energy_model=po.MODEL_PAIRBOND, pile=pile)
    o = po.Oracle(cfg)
    assert np.array_equal(occ, o.occupancy())
    sx, sy = 24, 10
    want = sorted({x + sx * (y + sy * z) for x, y, z in pile if 0 <= x < 24 and 0 <= y < 10 and 0 <= z < 14})
    assert list(np.flatnonzero(occ == 0)) == want
    # the alloy is the random creation's (same mt19937 draws) away from the listed sites
    rnd = ak.config_lattice(ak.config_parse(CONFIG))
    keep = np.ones(occ.size, bool)
    keep[want] = False
    keep[rnd == 0] = False
    assert np.array_equal(occ[keep], rnd[keep])


def test_pipe_file_missing_and_restart(ak, tmp_path):
    c = ak.config_parse(_pipe_config(str(tmp_path / "nowhere.xyz")))
    with pytest.raises(ak.AkmcError) as e:
        ak.config_lattice(c)
    assert e.value.status == -1
    restart = CONFIG.replace("    enable: true\n    va_count: 7", "    enable: false\n    va_count: 7").replace(
        "  restart:\n    enable: false", "  restart:\n    enable: true")
    with pytest.raises(ak.AkmcError) as e:
        ak.config_parse(restart)
    assert "akmc_restore_snapshot" in str(e.value)
