"""Precision report: the FP32-compensated form against the FP64 form, same lattice, same seed.

The FP64 form reproduces the CPU restatement of the reference bit for bit, so its numbers stand
for the reference's.  Reported:

- jump errors: every vacancy's 8 jumps in sampled lattice states, each state evaluated by both
  forms on identical occupancy and density cache: max |dE_fp32c - dE_fp64| in eV and the max
  relative rate error (jumps onto a vacancy carry no rate and are left out);
- first divergence: the two runs advance together round by round; their event sequences, each in
  (round, block, hop) order, are compared as they arrive, and the index of the first hop that
  differs (site, species, round or block) is reported, with its round;
- cluster statistics of the two final lattices (isolated-Cu count and Cu cluster-size histogram
  by 1nn connectivity, as MEventHook::onStepFinished counts them in profiles/m_event_hook.cpp).

Jump errors on a large lattice are taken in windows: each sampled vacancy is cut out with the
20^3 cells around it as a periodic box of its own.  A jump's dE reads the occupancy within the
cutoff (1.96 a) of both end sites, 0.87 a apart, and the densities of those sites, which read
their own cutoff neighbourhoods: under 5 cells from the vacancy, while the window reaches 9 cells
on every side.  So the window holds the vacancy's whole environment, and its density cache is
the large lattice's, value for value.

Run: python -m akmc_b200.precision [--hops 1e7] [--out report.json]
"""
import argparse
import json
import sys
import time

import numpy as np

from . import FE, CU, NI, MN, FP32C, FP64, Engine, cluster_stats, create_lattice, eam_johnson, job_config

QUATERNARY = ((FE, 9766), (CU, 134), (NI, 70), (MN, 30))
WINDOW = 20  # cells per side; the vacancy sits at cell (10, 10, 10), in sector 7
_KEYS = ("round", "block", "hop", "from_site", "to_site", "species")


def window(occ, box, site, edge=WINDOW):
    """Occupancy of the periodic edge^3-cell box around `site` of a box-sized lattice (site ids
    x + 2 nx (y + ny z), x doubled), and the id of `site` inside it."""
    nx, ny, nz = (int(b) for b in box)
    if min(nx, ny, nz) < edge:
        raise ValueError("lattice smaller than the window")
    occ3 = np.asarray(occ).reshape(nz, ny, 2 * nx)
    X = site % (2 * nx)
    t = site // (2 * nx)
    y, z = t % ny, t // ny
    h = edge // 2
    xs = (2 * ((X >> 1) - h) + np.arange(2 * edge)) % (2 * nx)
    ys = (y - h + np.arange(edge)) % ny
    zs = (z - h + np.arange(edge)) % nz
    w = np.ascontiguousarray(occ3[np.ix_(zs, ys, xs)]).reshape(-1)
    return w, (2 * h + (X & 1)) + 2 * edge * (h + edge * h)


def jump_rates(occ, box, sites, eam, temperature, precision, device=0):
    """dE (eV) and rates (Hz) of the 8 jumps of each vacancy in `sites`, evaluated by the form
    `precision` on windows of `occ`; arrays of shape (len(sites), 8)."""
    wins = [window(occ, box, int(s)) for s in sites]
    de = np.zeros((len(wins), 8))
    rates = np.zeros((len(wins), 8))
    with Engine(device=device) as eng:
        for w, _ in wins:
            eng.add_job(job_config((WINDOW,) * 3, precision=precision, temperature=temperature, eam=eam), w)
        eng.prepare()
        for j, (_, centre) in enumerate(wins):
            eng.calculate(j, 7)
            s, d, r = eng.calculated_rates()
            k = np.flatnonzero(s == centre)
            if len(k) != 1:
                raise RuntimeError("window %d: the centre vacancy is not in sector 7" % j)
            de[j], rates[j] = d[k[0]], r[k[0]]
    return de, rates


def jump_errors(occ, box, eam, temperature, max_vacancies=1024, device=0):
    """Errors of the FP32-compensated jumps against FP64 over the vacancies of `occ`."""
    sites = np.flatnonzero(np.asarray(occ) == 0)[:max_vacancies]
    d64, r64 = jump_rates(occ, box, sites, eam, temperature, FP64, device)
    d32, r32 = jump_rates(occ, box, sites, eam, temperature, FP32C, device)
    on = r64 > 0.0
    if not np.array_equal(on, r32 > 0.0):
        raise RuntimeError("the two forms disagree on which jumps are open")
    dde = np.abs(d32 - d64)[on]
    rel = (np.abs(r32 - r64)[on] / r64[on]) if on.any() else np.zeros(0)
    return dict(vacancies=int(len(sites)), jumps=int(on.sum()),
                max_abs_de_ev=float(dde.max(initial=0.0)), mean_abs_de_ev=float(dde.mean()) if len(dde) else 0.0,
                max_rel_rate=float(rel.max(initial=0.0)), mean_rel_rate=float(rel.mean()) if len(rel) else 0.0,
                max_abs_de_fp64_ev=float(np.abs(d64[on]).max(initial=0.0)))


def _ordered(ev):
    ev = ev[np.lexsort((ev["hop"], ev["block"], ev["round"]))]
    return np.stack([ev[k].astype(np.int64) for k in _KEYS], axis=1)


def report(box=(256, 256, 256), blocks=(16, 16, 16), alloy=QUATERNARY, vacancy_fraction=2e-5, temperature=563.0,
           seed=42, pot_seed=42, n_hops=10_000_000, chunk_rounds=32, log_capacity=1 << 21, device=0,
           max_window_vacancies=1024):
    """Side-by-side run of both forms from one lattice and seed until the FP64 run has made
    n_hops hops, with the jump errors of the start and end lattices and the cluster statistics."""
    t0 = time.time()
    nv = max(1, int(round(vacancy_fraction * 2 * np.prod(box))))
    occ0 = create_lattice(box, alloy, nv, seed)
    eam = eam_johnson(pot_seed)
    matched, diverged, div_round = 0, None, None
    with Engine(device=device, event_log_capacity=log_capacity, graph_rounds=chunk_rounds) as eng:
        for prec in (FP64, FP32C):
            eng.add_job(job_config(box, blocks=blocks, precision=prec, temperature=temperature, seed=seed, eam=eam),
                        occ0)
        eng.prepare()
        schedule = eng.round_schedule()
        while eng.job_state(0)["hops"] < n_hops:
            eng.run_rounds(chunk_rounds)
            eng.sync()
            ev = eng.events(log_capacity)
            if diverged is not None:
                continue
            a, b = _ordered(ev[ev["job"] == 0]), _ordered(ev[ev["job"] == 1])
            n = min(len(a), len(b))
            diff = np.flatnonzero((a[:n] != b[:n]).any(axis=1))
            if len(diff) or len(a) != len(b):
                i = int(diff[0]) if len(diff) else n
                diverged = matched + i
                div_round = int(min(a[i, 0] if i < len(a) else 1 << 62, b[i, 0] if i < len(b) else 1 << 62))
            else:
                matched += n
        st64, st32 = eng.job_state(0), eng.job_state(1)
        occ64, occ32 = eng.occupancy(0), eng.occupancy(1)
    iso0, h0 = cluster_stats(occ0, box)
    iso64, h64 = cluster_stats(occ64, box)
    iso32, h32 = cluster_stats(occ32, box)
    cu_atoms = int((occ0 == CU).sum())
    out = dict(
        lattice=dict(box=list(box), blocks=list(blocks), sites=int(occ0.size), vacancies=nv,
                     temperature=temperature, seed=seed, schedule="flow" if schedule == 2 else "rounds"),
        hops=dict(fp64=int(st64["hops"]), fp32c=int(st32["hops"]), rounds=int(st64["round"])),
        first_divergence=dict(hop=diverged, round=div_round, hops_compared=matched if diverged is None else None),
        jumps_start=jump_errors(occ0, box, eam, temperature, max_window_vacancies, device),
        jumps_end_fp64=jump_errors(occ64, box, eam, temperature, max_window_vacancies, device),
        clusters=dict(cu_atoms=cu_atoms, isolated_cu_start=iso0, isolated_cu_fp64=iso64, isolated_cu_fp32c=iso32,
                      isolated_cu_rel_diff=abs(iso32 - iso64) / max(1, iso64),
                      hist_fp64=[int(x) for x in h64[:16]], hist_fp32c=[int(x) for x in h32[:16]],
                      hist_rel_l1=float(np.abs(h32 - h64).sum() / max(1, h64.sum())),
                      hist_start=[int(x) for x in h0[:16]]),
        seconds=round(time.time() - t0, 1),
    )
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--edge", type=int, default=256)
    ap.add_argument("--block", type=int, default=16)
    ap.add_argument("--hops", type=float, default=1e7)
    ap.add_argument("--vacancy-fraction", type=float, default=2e-5)
    ap.add_argument("--temperature", type=float, default=563.0)
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default="")
    a = ap.parse_args(argv)
    nb = a.edge // a.block
    r = report(box=(a.edge,) * 3, blocks=(nb,) * 3, vacancy_fraction=a.vacancy_fraction, temperature=a.temperature,
               seed=a.seed, n_hops=int(a.hops), device=a.device)
    s = json.dumps(r)
    print(s)
    if a.out:
        with open(a.out, "w") as f:
            f.write(s + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
