"""Autotuner for batched and served runs: domain-block edge, threads per vacancy, rounds per CTA.

The knobs, all of which leave every trajectory unchanged except the block edge (see below):

- block edge: one CTA runs one domain block's active sector at a time, so the edge sets the work
  a CTA carries -- the vacancies its hop loop selects among (vacancies per CTA) and the region it
  stages into shared memory (sector plus a 2-cell halo).  Small blocks stage little per round but
  pay the per-round scheduling cost more often; large blocks carry more hops per round but stage
  regions that most hops never touch.  A box of edge n gets ceil(n / edge) blocks per dimension,
  at most n // 8 (blocks are at least 8 cells).  Different blocks give different (equally valid)
  trajectories, so the choice is made once, before the run it serves;
- threads per vacancy (eval_warps): the hop kernels evaluate a vacancy's 8 jumps with 8 warps
  (one jump each, one CTA per SM) or 4 warps (two jumps each, two CTAs per SM);
- rounds per CTA (flow_take): how many ready rounds with vacancies a CTA of the
  dependency-driven schedule takes per sweep (0: all it finds).

The sector window is part of the model (3e-7 s, src/simulation.h:73-74), not a knob.

tune() runs short trials on the actual job set: first every candidate edge with the default
shape, then the other thread count and round takes at the best edge, and returns the fastest.
"""
import time

from . import MODEL_EAM, AkmcError, Engine, job_config

CANDIDATES = (8, 12, 16, 20, 24)
WARPS = (8, 4)
TAKES = (0, 1, 4)


def blocks_for(edge, max_block_edge):
    """Domain blocks along a box edge of `edge` cells for blocks of at most max_block_edge."""
    return max(1, min(-(-edge // max_block_edge), edge // 8))


def _trial(jobs, lattices, eam, max_block_edge, rounds, warmup, device, eval_warps=8, flow_take=0):
    with Engine(device=device, eval_warps=eval_warps, flow_take=flow_take) as eng:
        for j, occ in zip(jobs, lattices):
            nb = tuple(blocks_for(e, max_block_edge) for e in j["box"])
            model = j.get("model", MODEL_EAM)
            eng.add_job(job_config(j["box"], blocks=nb, energy_model=model, precision=j["precision"],
                                   temperature=j["temperature"], seed=j["seed"],
                                   eam=eam if model == MODEL_EAM else None), occ)
        eng.prepare()
        eng.run_rounds(warmup)
        eng.sync()
        h0 = eng.counters()["hops"]
        t0 = time.perf_counter()
        eng.run_rounds(rounds)
        eng.sync()
        dt = time.perf_counter() - t0
        return (eng.counters()["hops"] - h0) / dt


# akmc_prepare's answer to a decomposition whose sector regions the hop kernels cannot stage
_REGION_TOO_LARGE = ("does not fit in shared memory", "wider than 28 cells")


def _region_too_large(e):
    return isinstance(e, AkmcError) and e.status == -1 and any(m in str(e) for m in _REGION_TOO_LARGE)


def tune_block_edge(jobs, lattices, eam, candidates=CANDIDATES, rounds=64, warmup=16, device=0):
    """jobs: dicts with box, precision, temperature, seed (as bench.py builds them); lattices:
    their occupancy arrays.  Returns (best edge, {edge: hops/s}) with the default kernel shape.
    A candidate whose regions do not fit the hop kernels is left out of the table; any other
    failure raises, and so does a candidate list with no runnable entry."""
    table = {}
    for c in candidates:
        try:
            table[c] = _trial(jobs, lattices, eam, c, rounds, warmup, device)
        except AkmcError as e:
            if not _region_too_large(e):
                raise
    if not table:
        raise RuntimeError("autotune: no candidate block edge of %r can run these jobs" % (tuple(candidates),))
    best = max(table, key=lambda c: table[c])
    return best, table


def tune(jobs, lattices, eam, candidates=CANDIDATES, warps=WARPS, takes=TAKES, rounds=64, warmup=16, device=0):
    """Staged search: the block edge with the default shape (8 warps, every round taken), then
    the other thread counts at that edge, then the round takes at the best (edge, warps).
    Returns ({"block_edge", "eval_warps", "flow_take"}, {"edge=E warps=W take=T": hops/s})."""
    edge, by_edge = tune_block_edge(jobs, lattices, eam, candidates, rounds, warmup, device)
    table = {"edge=%d warps=%d take=%d" % (e, 8, 0): v for e, v in by_edge.items()}
    best = (edge, 8, 0)
    for w in warps:
        if w == 8:
            continue
        v = _trial(jobs, lattices, eam, edge, rounds, warmup, device, eval_warps=w)
        table["edge=%d warps=%d take=%d" % (edge, w, 0)] = v
        if v > table["edge=%d warps=%d take=%d" % best]:
            best = (edge, w, 0)
    for t in takes:
        if t == 0:
            continue
        v = _trial(jobs, lattices, eam, edge, rounds, warmup, device, eval_warps=best[1], flow_take=t)
        table["edge=%d warps=%d take=%d" % (edge, best[1], t)] = v
        if v > table["edge=%d warps=%d take=%d" % best]:
            best = (edge, best[1], t)
    return dict(block_edge=best[0], eval_warps=best[1], flow_take=best[2]), table
