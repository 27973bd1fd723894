"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Integer results (event sites, species, block, round, hop index, final
occupancy, density cache) must be identical; the floating-point results of
the same arithmetic (selection draw, total rate, residence time, per-sector
clocks) must be identical bit for bit, because host and device execute the
same IEEE operation sequence.
"""
import numpy as np
import pytest

import pyoracle as po
from helpers import CU_134, QUATERNARY, assert_same_events, device_job, oracle_job

pytestmark = pytest.mark.gpu


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


def run_pair(ak, rounds, jobs, schedule=0):
    """jobs: list of dicts of oracle_job/device_job kwargs; returns (engine, oracles)."""
    eng = ak.Engine(event_log_capacity=1 << 21)
    eng.set_round_schedule(schedule)
    oracles = []
    for kw in jobs:
        o = oracle_job(**kw)
        dkw = {k: kw[k] for k in ("box", "blocks", "model", "precision", "seed", "temperature", "pot_seed", "window")
               if k in kw}
        device_job(eng, o, **dkw)
        oracles.append(o)
    eng.prepare()
    for o in oracles:
        o.run_rounds(rounds)
    eng.run_rounds(rounds)
    eng.sync()
    return eng, oracles


def check_job(eng, o, j, dev_events):
    ev = dev_events[dev_events["job"] == j]
    assert_same_events(ev, o.events())
    assert np.array_equal(eng.occupancy(j), o.occupancy())
    evo_d, hops_d = eng.block_clocks(j)
    evo_o, hops_o = o.block_state()
    assert np.array_equal(hops_d, hops_o)
    assert np.array_equal(evo_d.view(np.uint64), evo_o.view(np.uint64))
    st = eng.job_state(j)
    assert st["hops"] == o.hops and st["round"] == o.round


def test_device_exp_log_bit_exact(ak):
    rng = np.random.default_rng(7)
    inf = float("inf")
    x = np.concatenate([rng.uniform(-60, 0, 4000), rng.uniform(1e-300, 1, 4000), rng.uniform(-700, 700, 2000),
                        rng.uniform(-746, -708, 2000), rng.uniform(-750, 715, 2000),
                        [0.0, 1.0, 0.5, 2.0 ** -1074, 709.0, -745.0, float("nan"), inf, -inf, 709.782712893384,
                         709.79, 710.0, 1e300, -745.1332191019412, -745.2, -1e300]])
    with ak.Engine() as eng:
        e, l = eng.device_math(x)
    want_e = np.array([po.port_exp(v) for v in x])
    want_l = np.array([po.port_log(v) if v > 0 else np.nan for v in x])
    assert np.array_equal(e.view(np.uint64), want_e.view(np.uint64))
    pos = x > 0
    assert np.array_equal(l[pos].view(np.uint64), want_l[pos].view(np.uint64))


@pytest.mark.parametrize("model,prec", [(po.MODEL_EAM, po.FP64), (po.MODEL_EAM, po.FP32C),
                                        (po.MODEL_PAIRBOND, po.FP64)])
def test_single_domain_20_cubed(ak, model, prec):
    eng, (o,) = run_pair(ak, 400, [dict(box=(20, 20, 20), model=model, precision=prec)])
    assert o.hops > 1000
    check_job(eng, o, 0, eng.events())
    if model == po.MODEL_EAM:
        assert np.array_equal(eng.rho(0), o.rho())
    eng.close()


def test_serial_box_20_cubed_to_1e5_hops(ak):
    # The plain serial workload at its stated length: BCC 20^3 cells, Fe-1.34Cu, 20 vacancies,
    # T = 573 K, seed 42, EAM in FP64, single domain, run until past 1e5 hops (3328 sector
    # rounds, 416 sublattice time steps of SubLattice::startTimeLoop, sublattice.inl:61-179).
    # Every event (sites, species, u, total, dt), the final occupancy, the density cache, the 8
    # sector clocks and the hop count must equal the oracle's bit for bit.
    rounds = 3328
    eng, (o,) = run_pair(ak, rounds, [dict(box=(20, 20, 20), model=po.MODEL_EAM, precision=po.FP64, seed=42,
                                           temperature=573.0, alloy=CU_134, n_vacancies=20)])
    assert o.hops >= 100000, o.hops
    assert o.round == rounds
    check_job(eng, o, 0, eng.events())
    assert np.array_equal(eng.rho(0), o.rho())
    eng.close()


@pytest.mark.parametrize("schedule", [1, 2])  # round by round; dependency-driven
def test_domain_blocks_quaternary(ak, schedule):
    kw = dict(box=(32, 32, 32), blocks=(2, 2, 2), model=po.MODEL_EAM, alloy=QUATERNARY, n_vacancies=60,
              temperature=563.0, seed=7)
    eng, (o,) = run_pair(ak, 160, [kw], schedule)
    assert o.hops > 500
    check_job(eng, o, 0, eng.events())
    assert np.array_equal(eng.rho(0), o.rho())
    eng.close()


def test_uneven_blocks_and_odd_edges(ak):
    kw = dict(box=(25, 17, 19), blocks=(3, 2, 1), model=po.MODEL_EAM, precision=po.FP32C, alloy=QUATERNARY,
              n_vacancies=30, seed=11)
    eng, (o,) = run_pair(ak, 120, [kw])
    check_job(eng, o, 0, eng.events())
    eng.close()


@pytest.mark.parametrize("model,prec", [(po.MODEL_EAM, po.FP64), (po.MODEL_PAIRBOND, po.FP64)])
def test_single_domain_24_cubed_wrapped_bulk_staging(ak, model, prec):
    # rows of 48 sites: every sector's halo wraps in x, and each staged row goes in two bulk copies
    eng, (o,) = run_pair(ak, 320, [dict(box=(24, 24, 24), model=model, precision=prec, alloy=QUATERNARY,
                                        n_vacancies=12, temperature=563.0, seed=17)])
    assert o.hops > 500
    check_job(eng, o, 0, eng.events())
    if model == po.MODEL_EAM:
        assert np.array_equal(eng.rho(0), o.rho())
    eng.close()


@pytest.mark.parametrize("schedule", [1, 2])
def test_uneven_blocks_with_bulk_staging(ak, schedule):
    # rows of 80 sites (a multiple of 16): regions that do not wrap in x are staged by bulk
    # copies; the x split 14/13/13 gives sectors of 7 and 6 cells, staged with one row pitch
    kw = dict(box=(40, 24, 56), blocks=(3, 2, 3), model=po.MODEL_EAM, alloy=QUATERNARY, n_vacancies=40,
              temperature=563.0, seed=13)
    eng, (o,) = run_pair(ak, 128, [kw], schedule)
    assert o.hops > 500
    check_job(eng, o, 0, eng.events())
    assert np.array_equal(eng.rho(0), o.rho())
    eng.close()


@pytest.mark.parametrize("warps,take,schedule", [(4, 0, 1), (4, 0, 2), (8, 1, 2), (4, 4, 2)])
def test_kernel_shapes_and_takes_give_the_same_trajectories(ak, warps, take, schedule):
    # the autotuner's knobs: 4 evaluator warps (two jumps each, two CTAs per SM) and the rounds
    # a CTA takes per sweep must not change a bit of any trajectory
    jobs = [dict(box=(32, 32, 32), blocks=(2, 2, 2), model=po.MODEL_EAM, alloy=QUATERNARY, n_vacancies=50,
                 temperature=563.0, seed=71),
            dict(box=(24, 24, 24), blocks=(2, 1, 1), model=po.MODEL_EAM, precision=po.FP32C, alloy=QUATERNARY,
                 n_vacancies=12, seed=72),
            dict(box=(16, 24, 18), model=po.MODEL_PAIRBOND, alloy=QUATERNARY, n_vacancies=9, temperature=500.0,
                 seed=73),
            dict(box=(20, 20, 20), model=po.MODEL_EAM, n_vacancies=8, seed=74)]
    eng = ak.Engine(event_log_capacity=1 << 21, eval_warps=warps, flow_take=take)
    eng.set_round_schedule(schedule)
    oracles = []
    for kw in jobs:
        o = oracle_job(**kw)
        dkw = {k: kw[k] for k in ("box", "blocks", "model", "precision", "seed", "temperature") if k in kw}
        device_job(eng, o, **dkw)
        oracles.append(o)
    eng.prepare()
    for o in oracles:
        o.run_rounds(120)
    eng.run_rounds(120)
    eng.sync()
    ev = eng.events()
    for j, o in enumerate(oracles):
        check_job(eng, o, j, ev)
    assert np.array_equal(eng.rho(0), oracles[0].rho())
    eng.close()


def test_batched_jobs_of_different_shapes(ak):
    jobs = [
        dict(box=(20, 20, 20), model=po.MODEL_EAM, seed=1, temperature=573.0),
        dict(box=(16, 24, 18), model=po.MODEL_PAIRBOND, seed=2, alloy=QUATERNARY, n_vacancies=9, temperature=500.0),
        dict(box=(32, 16, 16), blocks=(2, 1, 1), model=po.MODEL_EAM, precision=po.FP32C, seed=3, n_vacancies=12,
             temperature=650.0, pot_seed=5),
    ]
    eng, oracles = run_pair(ak, 96, jobs)
    ev = eng.events()
    for j, o in enumerate(oracles):
        check_job(eng, o, j, ev)
    eng.close()


def test_hop_budget_stops_at_time_step_boundary(ak):
    o = oracle_job(box=(20, 20, 20))
    with ak.Engine(event_log_capacity=1 << 20) as eng:
        device_job(eng, o, (20, 20, 20), hop_budget=2000)
        eng.prepare()
        o.run(2000, 100000)
        eng.run(100000)
        st = eng.job_state(0)
        assert st["done"] and st["hops"] == o.hops and st["round"] == o.round
        assert o.hops >= 2000 and o.round % 8 == 0
        assert np.array_equal(eng.occupancy(0), o.occupancy())


@pytest.mark.parametrize("schedule", [1, 2])
def test_hop_budgets_under_both_schedules(ak, schedule):
    # a multi-block job with a budget next to one without, 93 rounds requested (not a multiple
    # of 8): the budget job stops at a time-step boundary, the other runs all 93 rounds
    kws = [dict(box=(32, 32, 32), blocks=(2, 2, 2), model=po.MODEL_EAM, alloy=QUATERNARY, n_vacancies=40,
                temperature=563.0, seed=21),
           dict(box=(24, 24, 24), blocks=(2, 1, 1), model=po.MODEL_EAM, precision=po.FP32C, n_vacancies=10, seed=22)]
    budget = 2500
    with ak.Engine(event_log_capacity=1 << 20) as eng:
        eng.set_round_schedule(schedule)
        oracles = [oracle_job(**kw) for kw in kws]
        for k, (kw, o) in enumerate(zip(kws, oracles)):
            dkw = {key: kw[key] for key in ("box", "blocks", "model", "precision", "seed", "temperature") if key in kw}
            device_job(eng, o, hop_budget=budget if k == 0 else 0, **dkw)
        eng.prepare()
        assert eng.round_schedule() == schedule
        eng.run_rounds(93)
        eng.sync()
        oracles[0].run(budget, 93)
        oracles[1].run_rounds(93)
        ev = eng.events()
        for k, o in enumerate(oracles):
            check_job(eng, o, k, ev)
        st = eng.job_state(0)
        assert st["done"] and st["round"] % 8 == 0 and st["round"] < 93 and st["hops"] >= budget
        assert eng.job_state(1)["round"] == 93


def test_single_block_budget_jobs_under_flow(ak):
    # single-block jobs run their rounds back to back in one CTA under the dependency-driven
    # schedule, and the kernel itself stops each at the first time-step boundary at which its
    # hops reached its budget; a multi-block job without budget shares the launches.  Each job
    # must equal the oracle, budgets and rounds alike, over calls that end between boundaries.
    kws = [dict(box=(16, 16, 16), model=po.MODEL_EAM, precision=po.FP32C, alloy=QUATERNARY, n_vacancies=4,
                temperature=600.0, seed=41),
           dict(box=(20, 20, 20), model=po.MODEL_EAM, n_vacancies=6, seed=42),
           dict(box=(18, 17, 16), model=po.MODEL_PAIRBOND, alloy=QUATERNARY, n_vacancies=5, seed=43),
           dict(box=(32, 32, 32), blocks=(2, 2, 2), model=po.MODEL_EAM, alloy=QUATERNARY, n_vacancies=40,
                temperature=563.0, seed=44)]
    budgets = [300, 700, 150, 0]
    calls = (37, 100, 63, 5)
    with ak.Engine(event_log_capacity=1 << 20) as eng:
        eng.set_round_schedule(ak.SCHEDULE_FLOW)
        oracles = [oracle_job(**kw) for kw in kws]
        for kw, o, b in zip(kws, oracles, budgets):
            dkw = {key: kw[key] for key in ("box", "blocks", "model", "precision", "seed", "temperature") if key in kw}
            device_job(eng, o, hop_budget=b, **dkw)
        eng.prepare()
        assert eng.round_schedule() == ak.SCHEDULE_FLOW
        for n in calls:
            eng.run_rounds(n)
        eng.sync()
        total = sum(calls)
        for o, b in zip(oracles, budgets):
            if b:
                o.run(b, total)
            else:
                o.run_rounds(total)
        ev = eng.events()
        for k, (o, b) in enumerate(zip(oracles, budgets)):
            check_job(eng, o, k, ev)
            st = eng.job_state(k)
            if b:
                assert st["done"] and st["round"] % 8 == 0 and st["hops"] >= b and st["round"] < total, st
            else:
                assert st["round"] == total


def test_time_boxed_calls_follow_the_oracle(ak):
    # akmc_run_for: launches that take no new round after 200 us, so every job ends each call at
    # its own round; repeated until the budget jobs are done and the round-limited ones at their
    # limit.  A multi-block budget job (its blocks meet at each time-step boundary), single-block
    # budget jobs, a round-limited multi-block job and a pair-bond job: each equals the oracle.
    kws = [dict(box=(32, 32, 32), blocks=(2, 2, 2), model=po.MODEL_EAM, alloy=QUATERNARY, n_vacancies=40,
                temperature=563.0, seed=61),
           dict(box=(16, 16, 16), model=po.MODEL_EAM, precision=po.FP32C, alloy=QUATERNARY, n_vacancies=4,
                temperature=620.0, seed=62),
           dict(box=(24, 16, 16), blocks=(2, 1, 1), model=po.MODEL_PAIRBOND, alloy=QUATERNARY, n_vacancies=10, seed=63),
           dict(box=(20, 20, 20), model=po.MODEL_EAM, n_vacancies=6, seed=64)]
    budgets = [3000, 400, 0, 900]
    max_rounds = [0, 0, 150, 0]
    with ak.Engine(event_log_capacity=1 << 20) as eng:
        oracles = [oracle_job(**kw) for kw in kws]
        for kw, o, b, m in zip(kws, oracles, budgets, max_rounds):
            dkw = {key: kw[key] for key in ("box", "blocks", "model", "precision", "seed", "temperature") if key in kw}
            device_job(eng, o, hop_budget=b, max_rounds=m, **dkw)
        eng.prepare()
        eng.set_round_schedule(ak.SCHEDULE_FLOW)
        calls = 0
        while not all(st["done"] for st in eng.job_states()):
            eng.run_for(1 << 20, 200)
            eng.sync()
            calls += 1
            assert calls < 20000
        assert calls > 3  # the time box cut the runs into several calls
        for o, b, m in zip(oracles, budgets, max_rounds):
            if b:
                o.run(b, 1 << 30)
            else:
                o.run_rounds(m)
        ev = eng.events()
        for k, o in enumerate(oracles):
            check_job(eng, o, k, ev)
            assert eng.job_state(k)["done"]


def test_schedule_switch_between_calls(ak):
    # the job server switches a context between the two schedules from one chunk to the next:
    # the trajectory must not notice.  A budget job (it stops at a time-step boundary inside the
    # third call), a job without budget and a single-block job, 40 + 56 + 24 + 7 rounds under
    # flow, rounds (a captured graph and eager rounds), flow, rounds
    kws = [dict(box=(32, 32, 32), blocks=(2, 2, 2), model=po.MODEL_EAM, alloy=QUATERNARY, n_vacancies=40,
                temperature=563.0, seed=31),
           dict(box=(24, 24, 24), blocks=(2, 1, 1), model=po.MODEL_EAM, precision=po.FP32C, n_vacancies=10, seed=32),
           dict(box=(16, 16, 16), model=po.MODEL_EAM, precision=po.FP32C, n_vacancies=4, seed=33)]
    budget = 5700  # the oracle reaches it in the time step that ends at round 112
    with ak.Engine(event_log_capacity=1 << 20) as eng:
        oracles = [oracle_job(**kw) for kw in kws]
        for k, (kw, o) in enumerate(zip(kws, oracles)):
            dkw = {key: kw[key] for key in ("box", "blocks", "model", "precision", "seed", "temperature") if key in kw}
            device_job(eng, o, hop_budget=budget if k == 0 else 0, **dkw)
        eng.prepare()
        for schedule, n in ((2, 40), (1, 56), (2, 24), (1, 7)):
            eng.set_round_schedule(schedule)
            assert eng.round_schedule() == schedule
            eng.run_rounds(n)
        eng.sync()
        oracles[0].run(budget, 127)
        oracles[1].run_rounds(127)
        oracles[2].run_rounds(127)
        ev = eng.events()
        for k, o in enumerate(oracles):
            check_job(eng, o, k, ev)
        st = eng.job_state(0)
        assert st["done"] and st["round"] % 8 == 0 and 96 < st["round"] < 120, st
        assert eng.job_state(1)["round"] == 127 and eng.job_state(2)["round"] == 127


def test_job_without_vacancies_only_advances_clocks(ak):
    o = oracle_job(box=(16, 16, 16), n_vacancies=0)
    with ak.Engine() as eng:
        device_job(eng, o, (16, 16, 16))
        eng.prepare()
        o.run_rounds(24)
        eng.run_rounds(24)
        evo_d, hops_d = eng.block_clocks(0)
        evo_o, _ = o.block_state()
        assert hops_d.sum() == 0
        assert np.array_equal(evo_d.view(np.uint64), evo_o.view(np.uint64))


def _host_driven_loop(eng, o_cfg_seed, window, rounds, job=0):
    """SubLattice::startTimeLoop (sublattice.inl:61-140) driven from the host over
    the per-hop entry points, with the host drawing the xoshiro streams."""
    sel = iter(po.xoshiro_stream(o_cfg_seed, 3, 0, 1 << 20))
    tim = iter(po.xoshiro_stream(o_cfg_seed, 4, 0, 1 << 20))
    evo = [0.0] * 8
    events = []
    hops = 0
    for rnd in range(rounds):
        sector = ak_sector(rnd)
        step = rnd // 8
        thr = float(step + 1) * window - evo[sector]
        t = 0.0
        while t < thr:
            total = eng.calculate(job, sector)
            if total == 0.0 or abs(total) < np.finfo(float).eps:
                t = thr
                continue
            u = float(int(next(sel)) >> 11) * 2.0 ** -53
            ev = eng.select_and_perform(job, sector, u)
            u2 = float((int(next(tim)) >> 11) + 1) * 2.0 ** -53
            dt = -po.port_log(u2) / total
            t += dt
            if ev.from_site >= 0:
                events.append((rnd, hops, ev.from_site, ev.to_site, ev.species, u, total, dt))
                hops += 1
        evo[sector] += t
    return events, evo


def ak_sector(rnd):
    return (0, 7, 2, 5, 3, 4, 1, 6)[rnd % 8]


@pytest.mark.parametrize("model", [po.MODEL_PAIRBOND, po.MODEL_EAM])
def test_per_hop_entry_points_follow_the_reference_loop(ak, model):
    o = oracle_job(box=(16, 16, 16), model=model, n_vacancies=6, seed=9)
    with ak.Engine() as eng:
        device_job(eng, o, (16, 16, 16), model=model, seed=9)
        eng.prepare()
        rounds = 24
        events, evo = _host_driven_loop(eng, 9, 3e-7, rounds)
        o.run_rounds(rounds)
        oe = o.events()
        assert len(events) == len(oe) and len(oe) > 20
        for a, b in zip(events, oe):
            assert a[0] == b["round"] and a[2] == b["from_site"] and a[3] == b["to_site"] and a[4] == b["species"]
            assert a[5] == b["u"] and a[6] == b["total"] and a[7] == b["dt"]
        evo_o, _ = o.block_state()
        assert np.array_equal(np.array(evo).view(np.uint64), evo_o[0].view(np.uint64))
        assert np.array_equal(eng.occupancy(0), o.occupancy())


@pytest.mark.parametrize("model,precision", [(po.MODEL_PAIRBOND, po.FP64), (po.MODEL_EAM, po.FP64),
                                             (po.MODEL_EAM, po.FP32C)])
def test_calculated_rates_match_oracle_jump_by_jump(ak, model, precision):
    # every sector of a quaternary 20^3 box with 40 vacancies: each vacancy's 8 jumps
    o = oracle_job(model=model, precision=precision, alloy=QUATERNARY, n_vacancies=40, seed=5)
    with ak.Engine() as eng:
        device_job(eng, o, (20, 20, 20), model=model, precision=precision, seed=5)
        eng.prepare()
        seen = 0
        for sector in range(8):
            total = eng.calculate(0, sector)
            sites, de, rates = eng.calculated_rates()
            want_total = 0.0
            for i in np.argsort(sites, kind="stable"):  # the ordered total runs in site order
                for b in range(8):
                    want_total += float(rates[i, b])
            assert total == want_total
            for i, s in enumerate(sites):
                assert s >= 0
                avail, r, d = o.vacancy_rates(int(s))
                assert np.array_equal(rates[i].view(np.uint64), r.view(np.uint64))
                for b in range(8):
                    if (avail >> b) & 1:
                        assert de[i, b].view(np.uint64) == d[b].view(np.uint64)
                    else:
                        assert rates[i, b] == 0.0 and de[i, b] == 0.0
                seen += 1
            assert (total > 0.0) == (len(sites) > 0)
        assert seen == 40


def test_sector_overflow_is_reported(ak):
    # 200 vacancies in a 16^3 box: more than 64 in one sector
    o = oracle_job(box=(16, 16, 16), n_vacancies=600, model=po.MODEL_PAIRBOND, alloy=((po.FE, 1),))
    with ak.Engine() as eng:
        device_job(eng, o, (16, 16, 16), model=po.MODEL_PAIRBOND)
        eng.prepare()
        eng.run_rounds(1)
        with pytest.raises(ak.AkmcError) as ei:
            eng.sync()
        assert ei.value.status == -7


def test_cpp_host_time_loop_matches_oracle(ak):
    # akmc_host_time_loop: SubLattice::startTimeLoop in C++ over the per-hop entry points
    o = oracle_job(box=(16, 16, 16), n_vacancies=6, seed=9)
    with ak.Engine() as eng:
        device_job(eng, o, (16, 16, 16), seed=9)
        eng.prepare()
        ev, evo = eng.host_time_loop(0, 40, 9)
        o.run_rounds(40)
        oe = o.events()
        assert len(ev) == len(oe) > 20
        for f in ("round", "from_site", "to_site", "species"):
            assert np.array_equal(ev[f], oe[f]), f
        for f in ("u", "total", "dt"):
            assert np.array_equal(ev[f].view(np.uint64), np.ascontiguousarray(oe[f]).view(np.uint64)), f
        evo_o, _ = o.block_state()
        assert np.array_equal(evo.view(np.uint64), evo_o[0].view(np.uint64))
        assert np.array_equal(eng.occupancy(0), o.occupancy())


def test_load_occupancies_restarts_every_job(ak):
    jobs = [dict(box=(20, 20, 20), model=po.MODEL_EAM, seed=1),
            dict(box=(17, 19, 21), model=po.MODEL_PAIRBOND, seed=2, alloy=QUATERNARY, n_vacancies=7),
            dict(box=(32, 16, 16), blocks=(2, 1, 1), model=po.MODEL_EAM, precision=po.FP32C, seed=3,
                 n_vacancies=12)]
    starts = [oracle_job(**kw).occupancy() for kw in jobs]  # the initial lattices
    order = ["job", "round", "block", "hop"]
    eng, oracles = run_pair(ak, 48, jobs)
    first = np.sort(eng.events(), order=order)
    ends = [eng.occupancy(j) for j in range(len(jobs))]
    assert len(first) > 100
    assert np.array_equal(eng.occupancies(), np.concatenate(ends))
    eng.load_occupancies(np.concatenate(starts))  # every job restarts
    eng.run_rounds(48)
    eng.sync()
    second = np.sort(eng.events(), order=order)
    assert first.tobytes() == second.tobytes()
    assert np.array_equal(eng.occupancies(), np.concatenate(ends))
    bad = np.concatenate(starts)
    bad[np.nonzero(bad == 0)[0][-1]] = 1  # the last job holds one vacancy fewer
    with pytest.raises(ak.AkmcError) as e:
        eng.load_occupancies(bad)
        eng.sync()
    assert e.value.status == -1
    eng.close()


def test_load_occupancy_restarts_the_trajectory(ak):
    o = oracle_job(box=(20, 20, 20), seed=5)
    occ0 = o.occupancy()
    with ak.Engine(event_log_capacity=1 << 18) as eng:
        device_job(eng, o, (20, 20, 20), seed=5)
        eng.prepare()
        eng.run_rounds(64)
        first = eng.events()
        occ1 = eng.occupancy(0)
        eng.load_occupancy(0, occ0)
        assert np.array_equal(eng.occupancy(0), occ0)
        assert eng.job_state(0)["round"] == 0
        eng.run_rounds(64)
        second = eng.events()
        assert len(first) > 100
        assert_same_events(second, np.sort(first, order=["round", "block", "hop"]))
        assert np.array_equal(eng.occupancy(0), occ1)
        bad = occ0.copy()
        bad[np.nonzero(bad == 0)[0][0]] = 1  # one vacancy fewer than the job holds
        with pytest.raises(ak.AkmcError) as e:  # reported by the next synchronising call
            eng.load_occupancy(0, bad)
            eng.sync()
        assert e.value.status == -1
        eng.load_occupancy(0, occ0)  # the context stays usable
        eng.sync()
        assert np.array_equal(eng.occupancy(0), occ0)


@pytest.mark.parametrize("schedule", [1, 2])
@pytest.mark.parametrize("edge,nvac", [(5, 150), (7, 400)])
def test_many_blocks_both_schedules(ak, schedule, edge, nvac):
    # edge^3 blocks of 8 cells: under the dependency-driven schedule blocks run rounds apart;
    # both schedules must give the oracle's trajectory.  343 blocks are more than two per SM,
    # so the dependency-driven kernel runs two CTAs per SM.
    kw = dict(box=(8 * edge,) * 3, blocks=(edge,) * 3, model=po.MODEL_EAM, alloy=QUATERNARY, n_vacancies=nvac,
              temperature=563.0, seed=5)
    eng, (o,) = run_pair(ak, 96, [kw], schedule)
    assert o.hops > 1000
    check_job(eng, o, 0, eng.events())
    assert np.array_equal(eng.rho(0), o.rho())
    eng.close()
