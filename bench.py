"""Benchmark of the vacancy-hop path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload scale|scale32|batched|serial]
                    [--rounds-per-step R] [--impl b200|reference]

One step = R sector rounds of the synchronous sublattice (R/8 sublattice time
steps of window 3e-7 s) over the workload's jobs.  `value` is whole-job vacancy
hops per second with the lattices resident in HBM; `e2e` is the same metric
through the public C ABI with the lattice uploaded from pinned host memory and
read back every step.  N > 1 runs independent replicas (one per GPU, seed 42 +
rank): the path has no exchange step between jobs.
"""
import argparse
import datetime
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "misa-akmc-gpu_b200"))
sys.path.insert(0, os.path.join(ROOT, "misa-akmc-gpu_b200", "python"))

METRIC = "vacancy hops/s on 1 B200: plain FP64 vs batched FP32-comp; p50/p99 job latency"
FE, CU, NI, MN = 1, 2, 4, 8
QUATERNARY = ((FE, 9766), (CU, 134), (NI, 70), (MN, 30))


# ---------------------------------------------------------------------------
# workloads
def _xoshiro(seed, tag):
    M = (1 << 64) - 1

    def mix(z):
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        return z ^ (z >> 31)

    h = mix(seed ^ ((tag * 0xD1B54A32D192ED03) & M))
    h = mix(h ^ (0x632BE59BD9B4E019))
    s = []
    for _ in range(4):
        h = (h + 0x9E3779B97F4A7C15) & M
        s.append(mix(h))

    def rotl(x, k):
        return ((x << k) | (x >> (64 - k))) & M

    def nxt():
        r = rotl((s[1] * 5) & M, 7) * 9 & M
        t = (s[1] << 17) & M
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = rotl(s[3], 45)
        return (r >> 11) * 2.0 ** -53

    return nxt


def workload_jobs(name, rank=0):
    """List of job dicts: box, blocks, alloy, n_vacancies, temperature, precision, seed."""
    seed = 42 + rank
    if name in ("scale", "scale32"):
        n = 256
        nv = int(round(2e-5 * 2 * n ** 3))
        return [dict(box=(n, n, n), blocks=(16, 16, 16), alloy=QUATERNARY, n_vacancies=nv, temperature=563.0,
                     precision=0 if name == "scale" else 1, seed=seed)]
    if name == "serial":
        return [dict(box=(20, 20, 20), blocks=(1, 1, 1), alloy=((FE, 9866), (CU, 134)), n_vacancies=20,
                     temperature=573.0, precision=0, seed=seed)]
    if name == "batched":
        draw = _xoshiro(seed, 7)
        jobs = []
        for i in range(512):
            edge = int(round(math.exp(math.log(16) + (math.log(48) - math.log(16)) * draw())))
            cu = 50 + int(round(100 * draw()))      # 0.5-1.5 at.% in 1e-4 units
            ni = int(round(100 * draw()))           # 0-1 at.%
            mn = int(round(50 * draw()))            # 0-0.5 at.%
            temp = 473.0 + 200.0 * draw()
            nb = 1 if edge <= 24 else 2
            nv = max(1, int(round(1e-4 * 2 * edge ** 3)))
            jobs.append(dict(box=(edge, edge, edge), blocks=(nb, nb, nb),
                             alloy=((FE, 10000 - cu - ni - mn), (CU, cu), (NI, ni), (MN, mn)), n_vacancies=nv,
                             temperature=temp, precision=1, seed=42 + i + 1000 * rank))
        return jobs
    raise SystemExit("unknown workload %s" % name)


def with_model(jobs, model):
    """The jobs in the named energy model: the synthetic EAM (as generated), or the reference's
    own pair-bond model, which has one precision (FP64)."""
    if model == "pairbond":
        for j in jobs:
            j["model"] = 0
            j["precision"] = 0
    return jobs


def serve_jobs(rate, seconds, rank=0):
    """Job stream of the serving workload: Poisson arrivals at `rate` per second for `seconds`,
    box edge log-uniform in [16, 96] cells, hop budget log-uniform in [1e4, 1e6], the batched
    workload's composition ranges, vacancy fraction 1e-4, seed 42 + job index."""
    draw = _xoshiro(42 + rank, 11)
    t, out, i = 0.0, [], 0
    while True:
        t += -math.log(1.0 - draw()) / rate
        if t >= seconds:
            return out
        edge = int(round(math.exp(math.log(16) + (math.log(96) - math.log(16)) * draw())))
        budget = int(round(math.exp(math.log(1e4) + (math.log(1e6) - math.log(1e4)) * draw())))
        cu = 50 + int(round(100 * draw()))
        ni = int(round(100 * draw()))
        mn = int(round(50 * draw()))
        nb = -(-edge // 24)  # blocks of at most 24 cells: the staged sector region fits in shared memory
        out.append(dict(t=t, box=(edge, edge, edge), blocks=(nb, nb, nb),
                        alloy=((FE, 10000 - cu - ni - mn), (CU, cu), (NI, ni), (MN, mn)),
                        n_vacancies=max(2, int(round(1e-4 * 2 * edge ** 3))), temperature=473.0 + 200.0 * draw(),
                        precision=1, seed=42 + i + 100000 * rank, hop_budget=budget))
        i += 1


def run_serve(args, ak, device):
    """Serving workload through akmc_server: arrivals replayed in real time, every job waited
    for; latency = result published - submitted."""
    jobs = serve_jobs(args.serve_rate, args.serve_seconds)
    eam = ak.eam_johnson(42)
    prepared = []
    for j in jobs:
        occ = ak.create_lattice(j["box"], j["alloy"], j["n_vacancies"], j["seed"])
        cfg = ak.job_config(j["box"], blocks=j["blocks"], energy_model=ak.MODEL_EAM, precision=j["precision"],
                            temperature=j["temperature"], seed=j["seed"], eam=eam, hop_budget=j["hop_budget"])
        prepared.append((j["t"], cfg, occ))
    srv = ak.Server(device=device, lanes=args.serve_lanes, chunk_rounds=args.serve_chunk,
                    order=1 if args.serve_order == "smallest" else 0)
    t0 = time.perf_counter()
    tickets = []
    for t, cfg, occ in prepared:
        while time.perf_counter() - t0 < t:
            time.sleep(0.0005)
        tickets.append(srv.submit(cfg, occ))
    lat, hops = [], 0
    for tk in tickets:
        res, _ = srv.wait(tk, timeout=3600.0)
        if res["status"] != 0:
            raise SystemExit("serving job failed with status %d: %s" % (res["status"], res["error"]))
        lat.append(res["finish_s"] - res["submit_s"])
        hops += res["hops"]
    wall = time.perf_counter() - t0
    prof = srv.profile()
    srv.close()
    lat = np.array(lat)
    line = {
        "metric": METRIC, "value": hops / wall, "unit": "hops/s", "n_gpus": 1, "steps": 1, "warmup": 0,
        "ms_per_step": 1e3 * wall, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32c",
        "data": "synthetic",
        "config": {"workload": "serving: Poisson arrivals %.0f/s for %.0f s, edge log-uniform 16-96 cells, hop "
                               "budget log-uniform 1e4-1e6, EAM FP32-compensated" % (args.serve_rate, args.serve_seconds),
                   "jobs": len(jobs), "lanes": args.serve_lanes, "chunk_rounds": args.serve_chunk,
                   "order": args.serve_order,
                   "offered_hops_per_s": sum(j["hop_budget"] for j in jobs) / args.serve_seconds},
        "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
        "latency_max_s": float(lat.max()), "wall_s": wall, "server_profile": prof,
    }
    print(json.dumps(line))


def reduce_over_ranks(dist, t, hops, device):
    """Whole-job figures over the ranks of a replica run: the slowest rank's time and the hops
    of all ranks (every rank takes the same two collectives in the same order)."""
    import torch

    v = torch.tensor([float(t), float(hops)], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(v[0:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(v[1:2], op=dist.ReduceOp.SUM)
    return float(v[0]), float(v[1])


def run_one_at_a_time(args, ak, jobs, device, stream, torch):
    """The plain form of a multi-job workload: the first N jobs in FP64, each alone in its own
    context, R rounds each after one untimed step; hops/s = all hops / all device time."""
    eam = ak.eam_johnson(42)
    hops, ms = 0, 0.0
    sample = jobs[: args.one_at_a_time]
    for j in sample:
        occ = ak.create_lattice(j["box"], j["alloy"], j["n_vacancies"], j["seed"])
        cfg = ak.job_config(j["box"], blocks=j["blocks"], energy_model=j.get("model", 1), precision=ak.FP64,
                            temperature=j["temperature"], seed=j["seed"], eam=eam if j.get("model", 1) else None)
        with ak.Engine(device=device, stream=stream.cuda_stream) as eng:
            eng.add_job(cfg, occ)
            eng.prepare()
            eng.run_rounds(args.rounds_per_step)
            eng.sync()
            h0 = eng.counters()["hops"]
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            eng.run_rounds(args.rounds_per_step)
            e1.record(stream)
            eng.sync()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            hops += eng.counters()["hops"] - h0
    line = {"metric": METRIC, "impl": "b200 plain FP64, one job at a time", "value": hops / (ms / 1e3),
            "unit": "hops/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": config_of(args, jobs)["workload"], "jobs_timed": len(sample),
                       "rounds_per_job": args.rounds_per_step, "note": "each job alone in its own context"},
            "hops_timed": int(hops), "ms": ms}
    print(json.dumps(line))


def algorithmic_bytes(hops, evals, nact_sum, eam=True):
    """Canonical bytes of the path: per vacancy evaluation the 145-site footprint
    (occupancy byte + int32 density) and 8 FP64 rates; per hop the 78-site density
    refresh (read + write), the occupancy swap and the event; per hop the selection
    scan over the sector's rates (64 B per vacancy)."""
    if eam:
        return evals * (145 + 145 * 4 + 64) + hops * (78 * 2 * 4 + 2 + 16) + 64 * nact_sum
    return evals * (113 + 64) + hops * (2 + 16) + 64 * nact_sum


# ---------------------------------------------------------------------------
class Clocks:
    """nvidia-smi samples (every 200 ms) around the timed region.  The sampler starts before
    the warm-up, so short timed regions still get samples; samples taken between mark_start
    and mark_stop (plus 250 ms either side) are kept, else the two nearest."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None
        self.t0 = self.t1 = None
        self.path = os.path.join("/tmp", "akmc_clocks_%d_%d.csv" % (os.getpid(), device))

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(self.device)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def mark_start(self):
        self.t0 = time.time()

    def mark_stop(self):
        self.t1 = time.time()

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.3)  # one more sample after the timed region
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.close()
        rows = []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((ts, float(parts[2]), float(parts[3]), parts[6:10]))
            except ValueError:
                continue
        if not rows:
            return None
        t0, t1 = (self.t0 or rows[0][0]), (self.t1 or rows[-1][0])
        sel = [r for r in rows if t0 - 0.25 <= r[0] <= t1 + 0.25]
        if not sel:
            sel = sorted(rows, key=lambda r: min(abs(r[0] - t0), abs(r[0] - t1)))[:2]
        reasons = set()
        for r in sel:
            for n, v in zip(names, r[3]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median([r[1] for r in sel]), "sm_max_mhz": sel[-1][2],
                "reasons": sorted(reasons), "samples": len(sel)}


def peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_per_launch(workload, schedule, rounds):
    """DRAM bytes per hop-kernel launch from the committed ncu summary, if any: per launch
    of one round (round by round) or per round of a flow launch, scaled to its rounds."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "k_hop_traffic.json")))
        v = d.get(schedule, {}).get(workload)
        if v is None:
            return None
        return v * rounds if schedule == "flow" else v
    except Exception:
        return None


# ---------------------------------------------------------------------------
def build_engine(ak, jobs, device, stream, log=0, schedule=0):
    eng = ak.Engine(device=device, stream=stream, event_log_capacity=log)
    eng.set_round_schedule(schedule)
    lattices = []
    eam = ak.eam_johnson(42)
    for j in jobs:
        occ = ak.create_lattice(j["box"], j["alloy"], j["n_vacancies"], j["seed"])
        cfg = ak.job_config(j["box"], blocks=j["blocks"], energy_model=j.get("model", 1), precision=j["precision"],
                            temperature=j["temperature"], seed=j["seed"], eam=eam if j.get("model", 1) else None)
        eng.add_job(cfg, occ)
        lattices.append(occ)
    eng.prepare()
    return eng, lattices


def cpu_baseline(jobs, seconds=15.0, rounds_per_chunk=8):
    """The oracle (the reference CPU path restated) on a bounded sample of the workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po

    j = jobs[0]
    cfg = po.make_config(box=j["box"], blocks=j["blocks"], energy_model=j.get("model", 1), precision=j["precision"],
                         temperature=j["temperature"], seed=j["seed"], pot_seed=42, alloy=j["alloy"],
                         n_vacancies=j["n_vacancies"], log_events=0)
    o = po.Oracle(cfg)
    t0 = time.perf_counter()
    rounds = 0
    while time.perf_counter() - t0 < seconds:
        o.run_rounds(rounds_per_chunk)
        rounds += rounds_per_chunk
    dt = time.perf_counter() - t0
    return {"value": o.hops / dt, "unit": "hops/s", "cores": os.cpu_count(), "kind": "port",
            "sample": "oracle, job 0 of the workload (%s cells, %d blocks), first %d sector rounds, %d hops, %.1f s"
                      % ("x".join(map(str, j["box"])), int(np.prod(j["blocks"])), rounds, o.hops, dt)}


def run_reference(args, jobs):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po

    j = jobs[0]
    cfg = po.make_config(box=j["box"], blocks=j["blocks"], energy_model=j.get("model", 1), precision=j["precision"],
                         temperature=j["temperature"], seed=j["seed"], pot_seed=42, alloy=j["alloy"],
                         n_vacancies=j["n_vacancies"], log_events=0)
    o = po.Oracle(cfg)
    rounds = args.rounds_per_step
    for _ in range(args.warmup):
        o.run_rounds(rounds)
    h0 = o.hops
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.run_rounds(rounds)
    dt = time.perf_counter() - t0
    value = (o.hops - h0) / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "hops/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if j["precision"] == 0 else "f32c",
        "data": "synthetic", "config": config_of(args, jobs),
        "cpu_baseline": {"value": value, "unit": "hops/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": "oracle (reference CPU path restated, OpenMP over domain blocks), job 0, "
                                   "%d timed steps of %d sector rounds" % (args.steps, rounds)},
        "e2e": {"value": value, "unit": "hops/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def config_of(args, jobs):
    j = jobs[0]
    c = {"workload": {"scale": "BCC 256^3 cells Fe-1.34Cu-0.7Ni-0.3Mn, 16^3-cell domain blocks x 8 sectors, "
                               "671 vacancies, EAM, T=563 K",
                      "scale32": "BCC 256^3 cells Fe-1.34Cu-0.7Ni-0.3Mn, 16^3-cell blocks, 671 vacancies, EAM "
                                 "FP32-compensated, T=563 K",
                      "batched": "512 boxes, edge log-uniform 16-48 cells, Cu 0.5-1.5 / Ni 0-1 / Mn 0-0.5 at.%, "
                                 "vacancy fraction 1e-4, T 473-673 K, EAM FP32-compensated",
                      "serial": "BCC 20^3 cells Fe-1.34Cu, 20 vacancies, single domain, EAM, T=573 K"}[args.workload],
         "jobs": len(jobs), "sites": int(sum(2 * np.prod(x["box"]) for x in jobs)),
         "vacancies": int(sum(x["n_vacancies"] for x in jobs)), "rounds_per_step": args.rounds_per_step,
         "sector_window_s": 3e-7,
         "energy_model": "synthetic Johnson EAM (5 shells, rc 5.6 A)" if j.get("model", 1) else
                         "pair bond (the reference's model: 1nn and masked 2nn bond energies)",
         "parallelism": "replicas x%d" % args.gpus,
         "l2": "inputs larger than L2 (occupancy + int32 density cache of %.0f MB)"
               % (5 * sum(2 * np.prod(x["box"]) for x in jobs) / 1e6)}
    if not j.get("model", 1):
        c["workload"] = c["workload"].replace("EAM FP32-compensated", "pair bond, FP64").replace("EAM", "pair bond")
    if len(jobs) == 1:
        c["box"] = list(j["box"])
        c["blocks"] = list(j["blocks"])
    return c


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="scale", choices=["scale", "scale32", "batched", "serial", "serve"])
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-seconds", type=float, default=10.0)
    ap.add_argument("--serve-lanes", type=int, default=2)
    ap.add_argument("--serve-chunk", type=int, default=16, help="sector rounds per server chunk")
    ap.add_argument("--serve-order", default="fifo", choices=["fifo", "smallest"],
                    help="admission order: arrival, or smallest hop budget first")
    ap.add_argument("--rounds-per-step", type=int, default=256)
    ap.add_argument("--one-at-a-time", type=int, default=0, metavar="N",
                    help="time the first N jobs of the workload in plain FP64, each alone (the baseline of "
                         "the batched form)")
    ap.add_argument("--model", default="eam", choices=["eam", "pairbond"],
                    help="energy model: the synthetic EAM, or the reference's own pair-bond model (FP64)")
    ap.add_argument("--schedule", default="auto", choices=["auto", "rounds", "flow"],
                    help="round schedule of the context (auto: dependency-driven where allowed)")
    ap.add_argument("--block-edge", type=int, default=0,
                    help="batched workload: blocks of at most this many cells; 0 = autotune before timing")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "serve":
        if rank == 0 and args.impl != "reference":
            import build as akbuild
            import akmc_b200 as ak

            akbuild.build()
            run_serve(args, ak, local)
        elif rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the serving workload has no CPU reference arm"}))
        return
    jobs = with_model(workload_jobs(args.workload, rank), args.model)

    if args.impl == "reference":
        if rank == 0:
            run_reference(args, with_model(workload_jobs(args.workload, 0), args.model))
        return

    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import build as akbuild
    import akmc_b200 as ak

    if rank == 0 or not os.path.exists(ak.lib_path()):
        akbuild.build()
    if dist:
        dist.barrier()
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream(device=local)
    if args.one_at_a_time:
        run_one_at_a_time(args, ak, jobs, local, stream, torch)
        return
    tuned = None
    if args.workload == "batched":
        import akmc_b200.autotune as at

        edge = args.block_edge
        if edge <= 0:  # autotune on the actual job set, outside the timed region
            lats = [ak.create_lattice(j["box"], j["alloy"], j["n_vacancies"], j["seed"]) for j in jobs]
            edge, table = at.tune_block_edge(jobs, lats, ak.eam_johnson(42), device=local)
            tuned = {"block_edge": edge, "trial_hops_per_s": {str(k): round(v) for k, v in table.items()}}
        else:
            tuned = {"block_edge": edge}
        for j in jobs:
            j["blocks"] = tuple(at.blocks_for(e, edge) for e in j["box"])
    eng, lattices = build_engine(ak, jobs, local, stream.cuda_stream,
                                 schedule={"auto": 0, "rounds": 1, "flow": 2}[args.schedule])
    R = args.rounds_per_step
    eam = jobs[0].get("model", 1) == 1

    def sync_all():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    clocks = Clocks(local)
    clocks.start()
    # warm-up
    for _ in range(args.warmup):
        eng.run_rounds(R)
    eng.sync()
    sync_all()
    c0 = eng.counters()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    sync_all()
    clocks.mark_start()
    ev0.record(stream)
    for _ in range(args.steps):
        eng.run_rounds(R)
    ev1.record(stream)
    eng.sync()
    sync_all()
    clocks.mark_stop()
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    c1 = eng.counters()
    hops = c1["hops"] - c0["hops"]
    ms_all, hops_all = reduce_over_ranks(dist, ms, hops, "cuda")
    value = hops_all / (ms_all / 1e3)

    # kernels launched per timed step: round by round, k_bucket + k_hop + k_finalize per round
    # (captured in CUDA graphs); dependency-driven, per launch of up to 1024 rounds k_flow_prep,
    # k_flow_slots, k_flow and k_flow_finalize (plus two memsets)
    sched = eng.round_schedule()
    sched_name = "flow" if sched == ak.SCHEDULE_FLOW else "rounds"
    launches_per_step = 4 * ((R + 1023) // 1024) if sched == ak.SCHEDULE_FLOW else 3 * R

    # roofline pass: same workload continued, hop kernel timed with events around every launch
    eng.set_kernel_timing(True)
    r0 = eng.counters()
    for _ in range(max(1, args.steps // 2)):
        eng.run_rounds(R)
    eng.sync()
    r1 = eng.counters()
    hop_ms, launches = eng.kernel_timing()
    eng.set_kernel_timing(False)
    rh = r1["hops"] - r0["hops"]
    bytes_alg = algorithmic_bytes(rh, r1["evaluations"] - r0["evaluations"], r1["n_act_sum"] - r0["n_act_sum"], eam)
    peak, peak_kind = peaks()
    achieved = bytes_alg / (hop_ms / 1e3) / 1e9 if hop_ms > 0 else 0.0
    traffic = traffic_per_launch(args.workload, sched_name, R)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_kind": peak_kind, "kernel": "k_flow" if sched_name == "flow" else "k_hop",
                "bytes_per_launch": bytes_alg / max(1, launches), "avg_launch_us": 1e3 * hop_ms / max(1, launches),
                "hops_per_launch": rh / max(1, launches),
                "e_hop": (r1["evaluations"] - r0["evaluations"]) / max(1, rh),
                "n_act_per_hop": (r1["n_act_sum"] - r0["n_act_sum"]) / max(1, rh)}

    # end to end through the C ABI: lattices from pinned host memory, R rounds, lattices back
    # (one job: akmc_load_occupancy / akmc_get_occupancy; several: the all-jobs forms)
    whole = torch.from_numpy(np.concatenate(lattices)).pin_memory()
    whole_out = torch.empty(whole.numel(), dtype=torch.uint8).pin_memory()
    for step in range(args.steps + 1):  # step 0 untimed: the first transfer sets up its buffers
        if step == 1:
            sync_all()
            e0 = eng.counters()
            t0 = time.perf_counter()
        if len(lattices) == 1:
            eng.load_occupancy(0, whole.numpy())
        else:
            eng.load_occupancies(whole.numpy())
        eng.run_rounds(R)
        eng.sync()
        if len(lattices) == 1:
            eng.occupancy(0, out=whole_out.numpy())
        else:
            eng.occupancies(out=whole_out.numpy())
    sync_all()
    e_dt = time.perf_counter() - t0
    e1 = eng.counters()
    e_hops = e1["hops"] - e0["hops"]
    e_dt_all, e_hops_all = reduce_over_ranks(dist, e_dt, e_hops, "cuda")
    e2e = {"value": e_hops_all / e_dt_all, "unit": "hops/s",
           "h2d_bytes_per_step": int(sum(o.size for o in lattices)), "d2h_bytes_per_step": int(sum(o.size for o in lattices)),
           "note": "each step restarts the jobs from the host lattices (upload, density rebuild), runs R rounds and "
                   "reads the lattices back"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "hops/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_all / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if jobs[0]["precision"] == 0 else "f32c", "data": "synthetic",
            "config": config_of(args, jobs), "roofline": roofline, "e2e": e2e,
            "gpu_launches": launches_per_step * args.steps, "schedule": sched_name, "clocks": clk,
            "hops_timed": int(hops_all),
        }
        if tuned:
            line["config"]["autotune"] = tuned
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(jobs)
        print(json.dumps(line))
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
