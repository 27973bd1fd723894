"""Cu cluster statistics of a synthetic lattice, computed on the device.

    python -m akmc_b200.stats [--edge 256] [--repeat 3] [--bins 64]

Builds a BCC lattice of edge^3 cells (Fe-1.34Cu-0.7Ni-0.3Mn at.%, vacancy fraction 2e-5, seed
42), loads it as a job, and prints the isolated-Cu count (MEventHook::onStepFinished,
profiles/m_event_hook.cpp:17-55), the number of Cu clusters and the host wall time of each
akmc_job_cluster_stats call; the last result is checked against the host count.
"""
import argparse
import sys
import time

import numpy as np

from . import CU, FE, MN, NI, MODEL_PAIRBOND, Engine, cluster_stats, create_lattice, job_config


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--edge", type=int, default=256)
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--bins", type=int, default=64)
    a = ap.parse_args(argv)
    box = (a.edge,) * 3
    nvac = max(1, int(round(2e-5 * 2 * a.edge ** 3)))
    occ = create_lattice(box, ((FE, 9766), (CU, 134), (NI, 70), (MN, 30)), nvac, 42)
    nb = max(1, a.edge // 16)
    with Engine() as eng:
        eng.add_job(job_config(box, blocks=(nb,) * 3, energy_model=MODEL_PAIRBOND, seed=42), occ)
        eng.prepare()
        for _ in range(a.repeat):
            t0 = time.perf_counter()
            iso, hist = eng.cluster_stats(0, a.bins)
            dt = time.perf_counter() - t0
            print("isolated Cu %d, clusters %d, %.3f ms" % (iso, int(hist.sum()), 1e3 * dt))
    iso_h, hist_h = cluster_stats(occ, box, a.bins)
    if iso != iso_h or not np.array_equal(hist, hist_h):
        print("device and host counts differ")
        return 1
    print("equal to the host count")
    return 0


if __name__ == "__main__":
    sys.exit(main())
