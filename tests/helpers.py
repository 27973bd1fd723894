"""Shared set-up for the parity tests: one oracle job and the matching device job."""
import numpy as np

import pyoracle as po

CU_134 = ((po.FE, 9866), (po.CU, 134))
QUATERNARY = ((po.FE, 9766), (po.CU, 134), (po.NI, 70), (po.MN, 30))


def oracle_job(box=(20, 20, 20), blocks=(1, 1, 1), model=po.MODEL_EAM, precision=po.FP64, seed=42,
               temperature=573.0, alloy=CU_134, n_vacancies=20, pot_seed=42, log_events=1, window=3e-7):
    cfg = po.make_config(box=box, blocks=blocks, energy_model=model, precision=precision, seed=seed,
                         temperature=temperature, alloy=alloy, n_vacancies=n_vacancies, pot_seed=pot_seed,
                         log_events=log_events, window=window)
    return po.Oracle(cfg)


def device_job(engine, oracle, box, blocks=(1, 1, 1), model=po.MODEL_EAM, precision=po.FP64, seed=42,
               temperature=573.0, pot_seed=42, hop_budget=0, max_rounds=0, window=3e-7):
    import akmc_b200 as ak

    eam = ak.eam_johnson(pot_seed) if model == po.MODEL_EAM else None
    cfg = ak.job_config(box, blocks=blocks, energy_model=model, precision=precision, seed=seed,
                        temperature=temperature, hop_budget=hop_budget, max_rounds=max_rounds, eam=eam,
                        window=window)
    return engine.add_job(cfg, oracle.occupancy())


def sort_events(ev):
    return ev[np.lexsort((ev["hop"], ev["block"], ev["round"]))]


def assert_same_events(dev, ora, fields_exact=("round", "hop", "from_site", "to_site", "block", "species",
                                                "n_act", "n_dirty"), fields_bits=("u", "total", "dt")):
    dev = sort_events(dev)
    assert len(dev) == len(ora), "event counts differ: device %d oracle %d" % (len(dev), len(ora))
    for f in fields_exact:
        if not np.array_equal(dev[f], ora[f]):
            i = int(np.nonzero(dev[f] != ora[f])[0][0])
            raise AssertionError("field %s first differs at event %d: device %r oracle %r" % (f, i, dev[i], ora[i]))
    for f in fields_bits:
        a = dev[f].view(np.uint64)
        b = np.ascontiguousarray(ora[f]).view(np.uint64)
        if not np.array_equal(a, b):
            i = int(np.nonzero(a != b)[0][0])
            raise AssertionError("field %s first differs at event %d: device %r oracle %r" % (f, i, dev[f][i], ora[f][i]))
