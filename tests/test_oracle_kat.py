"""Pins the oracle against the reference's own known-answer tests.

Restated from the reference's gtest suites (panzhija/MISA-AKMC-GPU):
  tests/unit/lattices_list_test.cpp:16-140          neighbour ids and orders
  tests/unit-abvi/rate/bonds/bonds_counter_test.cpp:17-100   bond sums
  tests/unit-abvi/rate/vac_rates_solver_test.cpp:20-106      dE and rate
Those suites run on NormalLatticeList (open boundaries, every 2nn counted); the
path under test is PeriodLatticeList, whose 2nn status is 0x2F
(src/lattice/period_lattice_list.cpp:15-18), so the expected bond sums below
count 5 of the 6 second neighbours.  The dE cases are unaffected because the
solute sits in a counted shell (bit 3 = z+1, or a first neighbour).
"""
import math
import struct

import numpy as np
import pytest

import pyoracle as po

B1 = {  # bonds_counter.cpp:13-22 (1nn), Vincent et al. 2006 table 7
    "FeFe": -0.778, "VV": 0.315, "CuCu": -0.581, "NiNi": -0.793, "MnMn": -0.438,
    "VFe": -0.161, "FeCu": -0.609, "FeNi": -0.821, "FeMn": -0.648,
    "VCu": -0.103, "VNi": -0.234, "VMn": -0.151, "CuNi": -0.692, "CuMn": -0.519, "NiMn": -0.831,
}
B2 = {  # bonds_counter.cpp:24-33 (2nn)
    "FeFe": -0.389, "VV": -0.214, "CuCu": -0.389, "NiNi": -0.389, "MnMn": -0.389,
    "VFe": -0.161, "FeCu": -0.344, "FeNi": -0.399, "FeMn": -0.364,
    "VCu": -0.206, "VNi": -0.351, "VMn": -0.206, "CuNi": -0.344, "CuMn": -0.249, "NiMn": -0.464,
}
KB = 8.617330350e-5  # rates_types.h:16


def pure_fe(box, model=po.MODEL_PAIRBOND, temperature=700.0):
    cfg = po.make_config(box=box, energy_model=model, n_vacancies=0, alloy=((po.FE, 1),),
                         temperature=temperature, attempt_freq=6e12)
    return po.Oracle(cfg)


def sid(box, x, y, z):
    return x + 2 * box[0] * (y + box[1] * z)


# --- lattices_list_test.cpp -------------------------------------------------

def test_1nn_ids_even_site():
    # lattice_list_get1nn_1 (lattices_list_test.cpp:16-44), box 4x4x4, ID = x + 8y + 32z
    o = pure_fe((4, 4, 4))
    nn1, _ = o.neighbours(sid((4, 4, 4), 2, 1, 1))
    want = [(1, 0, 0), (1, 0, 1), (1, 1, 0), (1, 1, 1), (3, 0, 0), (3, 0, 1), (3, 1, 0), (3, 1, 1)]
    assert list(nn1) == [x + 8 * y + 32 * z for x, y, z in want]


def test_1nn_ids_odd_site():
    # second half of lattice_list_get1nn_1: site (1,1,1), odd x
    o = pure_fe((4, 4, 4))
    nn1, _ = o.neighbours(sid((4, 4, 4), 1, 1, 1))
    want = [(0, 1, 1), (0, 1, 2), (0, 2, 1), (0, 2, 2), (2, 1, 1), (2, 1, 2), (2, 2, 1), (2, 2, 2)]
    assert list(nn1) == [x + 8 * y + 32 * z for x, y, z in want]


def test_1nn_ids_interior_high():
    # lattice_list_get1nn_5 (lattices_list_test.cpp:81-98): site (4,3,3)
    o = pure_fe((4, 4, 4))
    nn1, _ = o.neighbours(sid((4, 4, 4), 4, 3, 3))
    want = [(3, 2, 2), (3, 2, 3), (3, 3, 2), (3, 3, 3), (5, 2, 2), (5, 2, 3), (5, 3, 2), (5, 3, 3)]
    # periodic list: z+0 = 3, y+0 = 3 stay inside; ids as in the reference test
    assert list(nn1) == [x + 8 * y + 32 * z for x, y, z in want]


def test_2nn_ids_order():
    # lattice_list_get2nn_1 (lattices_list_test.cpp:101-114): site (2,1,1)
    o = pure_fe((4, 4, 4))
    _, nn2 = o.neighbours(sid((4, 4, 4), 2, 1, 1))
    want = [(0, 1, 1), (2, 0, 1), (2, 1, 0), (2, 1, 2), (2, 2, 1), (4, 1, 1)]
    assert list(nn2) == [x + 8 * y + 32 * z for x, y, z in want]


def test_periodic_wrap_at_low_corner():
    # lattice_list_get2nn_2 tests the open boundary at (0,0,0); the periodic list wraps instead
    o = pure_fe((4, 4, 4))
    _, nn2 = o.neighbours(0)
    want = [(6, 0, 0), (0, 3, 0), (0, 0, 3), (0, 0, 1), (0, 1, 0), (2, 0, 0)]
    assert list(nn2) == [x + 8 * y + 32 * z for x, y, z in want]


# --- bonds_counter_test.cpp -------------------------------------------------

def test_bond_count_pure_fe():
    # bonds_counter_count_test case 1 (bonds_counter_test.cpp:17-32), masked 2nn shell
    o = pure_fe((4, 4, 4))
    e = o.bond_count(sid((4, 4, 4), 4, 2, 2), po.FE)
    assert e == pytest.approx(B1["FeFe"] * 8 + B2["FeFe"] * 5, abs=1e-12)


def _src_tar_ni(box=(4, 4, 4), ni=(3, 1, 2), vac="src"):
    o = pure_fe(box)
    occ = o.occupancy()
    src, tar = sid(box, 4, 2, 2), sid(box, 5, 2, 2)
    occ[sid(box, *ni)] = po.NI
    occ[src if vac == "src" else tar] = po.V
    o.set_occupancy(occ)
    return o, src, tar


def test_bond_count_with_vacancy():
    # bonds_counter_count_test_with_V (bonds_counter_test.cpp:36-66)
    o, src, tar = _src_tar_ni()
    assert o.bond_count(src, po.V) == pytest.approx(B1["VFe"] * 7 + B1["VNi"] + B2["VFe"] * 5, abs=1e-12)
    assert o.bond_count(tar, po.FE) == pytest.approx(B1["VFe"] + B1["FeFe"] * 7 + B2["FeFe"] * 5, abs=1e-12)


def test_bond_count_after_exchange():
    # bonds_counter_count_test_with_V_2 (bonds_counter_test.cpp:70-100)
    o, src, tar = _src_tar_ni(vac="tar")
    assert o.bond_count(src, po.FE) == pytest.approx(
        B1["FeFe"] * 6 + B1["VFe"] + B1["FeNi"] + B2["FeFe"] * 5, abs=1e-12)
    assert o.bond_count(tar, po.V) == pytest.approx(B1["VFe"] + B1["VFe"] * 7 + B2["VFe"] * 5, abs=1e-12)


# --- vac_rates_solver_test.cpp ----------------------------------------------

def _direction(o, src, tar):
    nn1, _ = o.neighbours(src)
    return int(np.nonzero(nn1 == tar)[0][0])


def test_delta_e_null_and_rate():
    # vac_deltaE_test_null (vac_rates_solver_test.cpp:20-43): pure Fe, T=700, nu=6e12
    o = pure_fe((4, 4, 4))
    occ = o.occupancy()
    src, tar = sid((4, 4, 4), 4, 1, 1), sid((4, 4, 4), 5, 1, 1)
    occ[src] = po.V
    o.set_occupancy(occ)
    avail, rates, de = o.vacancy_rates(src)
    b = _direction(o, src, tar)
    assert avail == 0xFF
    assert de[b] == pytest.approx(0.0, abs=1e-10)
    expected = 6e12 * math.exp(-0.62 / (KB * 700.0))
    assert rates[b] / expected == pytest.approx(1.0, abs=1e-10)


def test_delta_e_src_1nn_neighbour():
    # vac_deltaE_test_src_1nn_neighbour (vac_rates_solver_test.cpp:81-106)
    o, src, tar = _src_tar_ni()
    _, _, de = o.vacancy_rates(src)
    want = (B1["VFe"] + B1["FeNi"]) - (B1["VNi"] + B1["FeFe"])
    assert de[_direction(o, src, tar)] == pytest.approx(want, abs=1e-10)


def test_delta_e_both_neighbour():
    # vac_deltaE_test_both_neighbour (vac_rates_solver_test.cpp:49-76), box 6x6x6, Ni at (4,2,3)
    o, src, tar = _src_tar_ni(box=(6, 6, 6), ni=(4, 2, 3))
    _, _, de = o.vacancy_rates(src)
    want = (B1["FeFe"] + B1["VNi"] + B2["FeNi"] + B2["VFe"]
            - B1["VFe"] - B1["FeNi"] - B2["VNi"] - B2["FeFe"])
    assert de[_direction(o, src, tar)] == pytest.approx(want, abs=1e-10)


def test_unavailable_directions_are_zero():
    # VacancyHash::beforeRatesUpdate2 (vac_hash.cpp:18-25): V neighbours are not jump targets
    o = pure_fe((6, 6, 6))
    occ = o.occupancy()
    src = sid((6, 6, 6), 4, 2, 2)
    occ[src] = po.V
    nn1, _ = o.neighbours(src)
    occ[nn1[3]] = po.V
    o.set_occupancy(occ)
    avail, rates, _ = o.vacancy_rates(src)
    assert avail == 0xFF & ~(1 << 3)
    assert rates[3] == 0.0 and np.all(rates[np.arange(8) != 3] > 0)


# --- RNG known answers --------------------------------------------------------

def test_mt19937_standard_check_value():
    # The C++ standard's check value for a default-constructed mt19937: the
    # 10000th draw is 4123659995.  The reference's selection stream r::rng is
    # a default-constructed (never seeded) mt19937 (src/utils/random/rand_generators.cpp:8).
    d = po.mt19937_draws(0, 10000, default_seed=True)
    assert round(d[-1] * 4294967295.0) == 4123659995


def _xoshiro_py(s, n):
    """Independent restatement of xoshiro256** (Blackman & Vigna 2018)."""
    M = (1 << 64) - 1
    rotl = lambda x, k: ((x << k) | (x >> (64 - k))) & M
    s = list(s)
    out = []
    for _ in range(n):
        out.append(rotl((s[1] * 5) & M, 7) * 9 & M)
        t = (s[1] << 17) & M
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t
        s[3] = rotl(s[3], 45)
    return out


def _splitmix_stream_py(seed, tag, index):
    M = (1 << 64) - 1

    def mix(z):
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        return z ^ (z >> 31)

    h = mix(seed ^ ((tag * 0xD1B54A32D192ED03) & M))
    h = mix(h ^ ((index * 0x9E3779B97F4A7C15 + 0x632BE59BD9B4E019) & M))
    st = []
    for _ in range(4):
        h = (h + 0x9E3779B97F4A7C15) & M
        st.append(mix(h))
    return st


def test_xoshiro_known_answer():
    # hand-derivable first outputs of xoshiro256** from state (1, 2, 3, 4)
    assert _xoshiro_py([1, 2, 3, 4], 2) == [11520, 0]


@pytest.mark.parametrize("seed,tag,index", [(42, 3, 0), (42, 4, 7), (0, 1, 0), (2**64 - 1, 5, 123)])
def test_xoshiro_streams_match_independent_restatement(seed, tag, index):
    got = po.xoshiro_stream(seed, tag, index, 64)
    want = _xoshiro_py(_splitmix_stream_py(seed, tag, index), 64)
    assert [int(v) for v in got] == want


# --- portable exp / log ----------------------------------------------------------

def _ulp_diff(a, b):
    ia = struct.unpack("<q", struct.pack("<d", a))[0]
    ib = struct.unpack("<q", struct.pack("<d", b))[0]
    return abs(ia - ib)


def test_portable_exp_within_one_ulp_of_libm():
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(-40, 0, 20000), rng.uniform(-700, 700, 5000), [0.0, -1e-300, 1e-20]])
    worst = max(_ulp_diff(po.port_exp(x), math.exp(x)) for x in xs)
    assert worst <= 1


def test_portable_log_within_two_ulp_of_libm():
    rng = np.random.default_rng(2)
    xs = np.concatenate([rng.uniform(0, 1, 20000), 10.0 ** rng.uniform(-300, 300, 5000), [1.0, 2**-1074, 0.5]])
    worst = max(_ulp_diff(po.port_log(x), math.log(x)) for x in xs if x > 0)
    assert worst <= 2
    assert po.port_log(1.0) == 0.0


@pytest.mark.parametrize("model", [po.MODEL_PAIRBOND, po.MODEL_EAM])
def test_libm_and_portable_math_give_the_same_events(model):
    # the GPU path computes exp/log with the portable routines; the reference uses libm
    evs = []
    for mm in (po.MATH_PORTABLE, po.MATH_LIBM):
        o = po.Oracle(po.make_config(energy_model=model, math_mode=mm))
        o.run(20000, 100000)
        evs.append(o.events())
    a, b = evs
    assert len(a) == len(b)
    for f in ("round", "from_site", "to_site", "species", "block"):
        assert np.array_equal(a[f], b[f])
    np.testing.assert_allclose(a["total"], b["total"], rtol=1e-14)
