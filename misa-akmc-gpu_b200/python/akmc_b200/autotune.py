"""Autotuner for batched and served runs: the domain-block edge.

One CTA runs one domain block's active sector at a time, so the block edge sets the work a CTA
carries: the vacancies its hop loop selects among (vacancies per CTA) and the region it stages
into shared memory (sector plus a 2-cell halo).  Small blocks stage little per round but pay
the per-round scheduling cost more often; large blocks carry more hops per round but stage
regions that most hops never touch.  The threads per vacancy are fixed by the kernel (one warp
per jump direction, 8 warps), and the sector window is part of the model (3e-7 s), not a knob.

tune_block_edge() runs every candidate edge on the actual job set for a short trial and returns
the fastest.  A box of edge n gets ceil(n / edge) blocks per dimension, at most n // 8 (blocks
are at least 8 cells).  Different blocks give different (equally valid) trajectories, so the
choice is made once, before the run it serves.
"""
import time

from . import MODEL_EAM, AkmcError, Engine, job_config

CANDIDATES = (8, 12, 16, 20, 24)


def blocks_for(edge, max_block_edge):
    """Domain blocks along a box edge of `edge` cells for blocks of at most max_block_edge."""
    return max(1, min(-(-edge // max_block_edge), edge // 8))


def _trial(jobs, lattices, eam, max_block_edge, rounds, warmup, device):
    with Engine(device=device) as eng:
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
    their occupancy arrays.  Returns (best edge, {edge: hops/s}).  A candidate whose regions
    do not fit the hop kernels is left out of the table; any other failure raises, and so does
    a candidate list with no runnable entry."""
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
