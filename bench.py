"""Benchmark of the vacancy-hop path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload scale|scale32|batched|serial|serve]
                    [--rounds-per-step R] [--impl b200|reference] [--no-extras]

One step = R sector rounds of the synchronous sublattice (R/8 sublattice time
steps of window 3e-7 s) over the workload's jobs.  `value` is whole-job vacancy
hops per second with the lattices resident in HBM; `e2e` is the same metric
through the public C ABI with the lattice uploaded from pinned host memory and
read back every step.  N > 1 runs independent replicas (one per GPU, seed 42 +
rank): the path has no exchange step between jobs.

The default run (workload `scale`, one GPU) measures the whole metric in one
JSON line: the 256^3 lattice in plain FP64 is `value`; the same lattice in
FP32-comp (`scale32`), the 512 batched boxes in FP32-comp (`batched`), the same
boxes in plain FP64 one job at a time (`plain_one_at_a_time`, a seeded sample),
their ratio (`batched_over_plain`) and the served Poisson job stream with its
p50/p99 latency (`serve`) are extra keys, each with its own clock record.
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
# sector rounds per timed step: 1024 rounds of the 256^3 lattice are about 0.86M hops, so the
# default 20 timed steps cover about 1.7e7 hops
DEFAULT_ROUNDS = {"scale": 1024, "scale32": 1024, "batched": 256, "serial": 256, "serve": 0}


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


def plain_sample(n_jobs, n, seed=42):
    """Indices of the jobs the plain form times one at a time: a seeded uniform sample without
    replacement, in ascending order."""
    if n >= n_jobs:
        return list(range(n_jobs))
    return sorted(int(i) for i in np.random.default_rng(seed).choice(n_jobs, size=n, replace=False))


# ---------------------------------------------------------------------------
class Clocks:
    """nvidia-smi samples (every 200 ms) over the whole run.  Each timed region is marked with
    mark(name) before and end(name) after it; report() gives, per region, the median SM clock,
    the maximum and the throttle reasons active in the samples taken inside it (plus 250 ms
    either side), else the two nearest samples."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None
        self.regions = {}
        self.rows = None
        self.path = os.path.join("/tmp", "akmc_clocks_%d_%d.csv" % (os.getpid(), device))

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(self.device)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def mark(self, name):
        self.regions[name] = [time.time(), None]

    def end(self, name):
        self.regions[name][1] = time.time()

    def stop(self):
        if self.p is None:
            return
        time.sleep(0.3)  # one more sample after the last timed region
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((ts, float(parts[2]), float(parts[3]), float(parts[4]), parts[6:10]))
            except ValueError:
                continue
        self.rows = rows
        self.p = None

    def report(self, name):
        if not self.rows or name not in self.regions:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0, t1 = self.regions[name]
        t1 = t1 or t0
        sel = [r for r in self.rows if t0 - 0.25 <= r[0] <= t1 + 0.25]
        if not sel:
            sel = sorted(self.rows, key=lambda r: min(abs(r[0] - t0), abs(r[0] - t1)))[:2]
        reasons = set()
        for r in sel:
            for n, v in zip(names, r[4]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median([r[1] for r in sel]), "sm_max_mhz": sel[-1][2],
                "power_w_max": max(r[3] for r in sel), "reasons": sorted(reasons), "samples": len(sel)}


def peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


TRAFFIC_FILE = os.path.join("profiles", "k_hop_traffic.json")


def traffic_per_launch(workload, schedule, rounds):
    """DRAM bytes per hop-kernel launch from the committed ncu summary, if it holds an entry
    for this workload and schedule: per launch of one round (round by round) or per round of a
    flow launch, scaled to its rounds.  None when there is no such entry."""
    try:
        d = json.load(open(os.path.join(ROOT, TRAFFIC_FILE)))
        v = d.get(schedule, {}).get(workload)
        if v is None:
            return None
        return v * rounds if schedule == "flow" else v
    except Exception:
        return None


def algorithmic_bytes(hops, evals, nact_sum, eam=True):
    """Canonical bytes of the path: per vacancy evaluation the 145-site footprint
    (occupancy byte + int32 density) and 8 FP64 rates; per hop the 78-site density
    refresh (read + write), the occupancy swap and the event; per hop the selection
    scan over the sector's rates (64 B per vacancy)."""
    if eam:
        return evals * (145 + 145 * 4 + 64) + hops * (78 * 2 * 4 + 2 + 16) + 64 * nact_sum
    return evals * (113 + 64) + hops * (2 + 16) + 64 * nact_sum


# ---------------------------------------------------------------------------
def build_engine(ak, jobs, device, stream, log=0, schedule=0, shape=None):
    """An engine with the jobs added and prepared; shape: the tuner's eval_warps / flow_take."""
    shape = shape or {}
    eng = ak.Engine(device=device, stream=stream, event_log_capacity=log, eval_warps=shape.get("eval_warps", 0),
                    flow_take=shape.get("flow_take", 0))
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


def reduce_over_ranks(dist, t, hops, device):
    """Whole-job figures over the ranks of a replica run: the slowest rank's time and the hops
    of all ranks (every rank takes the same two collectives in the same order)."""
    import torch

    v = torch.tensor([float(t), float(hops)], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(v[0:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(v[1:2], op=dist.ReduceOp.SUM)
    return float(v[0]), float(v[1])


class Runner:
    """Timed passes over one engine; `sync_all` is the barrier + device synchronise that
    brackets every timed region."""

    def __init__(self, torch, stream, dist, clocks):
        self.torch = torch
        self.stream = stream
        self.dist = dist
        self.clocks = clocks

    def sync_all(self):
        self.torch.cuda.synchronize()
        if self.dist:
            self.dist.barrier()

    def device_rate(self, eng, R, steps, warmup, name):
        """W untimed steps, then K steps of R rounds between CUDA events on the engine's
        stream; (ms, hops) of this rank."""
        torch = self.torch
        for _ in range(warmup):
            eng.run_rounds(R)
        eng.sync()
        self.sync_all()
        c0 = eng.counters()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        self.sync_all()
        self.clocks.mark(name)
        ev0.record(self.stream)
        for _ in range(steps):
            eng.run_rounds(R)
        ev1.record(self.stream)
        eng.sync()
        self.sync_all()
        self.clocks.end(name)
        return ev0.elapsed_time(ev1), eng.counters()["hops"] - c0["hops"]

    def roofline(self, eng, R, steps, eam, workload):
        """The hop kernel timed with CUDA events around every launch (same workload,
        continued): algorithmic bytes per launch over the launch time, against the measured
        copy peak."""
        eng.set_kernel_timing(True)
        r0 = eng.counters()
        for _ in range(max(1, steps)):
            eng.run_rounds(R)
        eng.sync()
        r1 = eng.counters()
        hop_ms, launches = eng.kernel_timing()
        eng.set_kernel_timing(False)
        rh = r1["hops"] - r0["hops"]
        evals = r1["evaluations"] - r0["evaluations"]
        bytes_alg = algorithmic_bytes(rh, evals, r1["n_act_sum"] - r0["n_act_sum"], eam)
        staged = (r1["staged_sites"] - r0["staged_sites"]) * (5 if eam else 1)
        ws = r1["written_sites"] - r0["written_sites"]  # 2 occupancy bytes per hop, plus 78 densities (EAM)
        written = 4 * (ws - 2 * rh) + 2 * rh if eam else ws
        peak, peak_kind = peaks()
        achieved = bytes_alg / (hop_ms / 1e3) / 1e9 if hop_ms > 0 else 0.0
        sched = "flow" if eng.round_schedule() == 2 else "rounds"
        traffic = traffic_per_launch(workload, sched, R)
        n = max(1, launches)
        return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic,
                "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one full 1024-round "
                                   "launch of this command (1 pass, warm L2), per round, scaled to the launch's "
                                   "rounds; stored in %s" % TRAFFIC_FILE
                                   if sched == "flow" else
                                   "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, 16-round capture "
                                   "with a cold L2; stored in %s" % TRAFFIC_FILE)
                if traffic is not None else None,
                "peak_kind": peak_kind, "kernel": "k_flow" if sched == "flow" else "k_hop",
                "bytes_per_launch": bytes_alg / n, "avg_launch_us": 1e3 * hop_ms / n, "launches": launches,
                "hops_per_launch": rh / n, "e_hop": evals / max(1, rh),
                "n_act_per_hop": (r1["n_act_sum"] - r0["n_act_sum"]) / max(1, rh),
                "staged_bytes_per_launch": (staged + written) / n,
                "staged_bytes_note": "measured in this run by the kernel's own counters: sector regions "
                                     "staged into shared memory and sites written through, per launch"}

    def end_to_end(self, eng, lattices, R, steps, name):
        """Every step: the lattices from pinned host memory through the C ABI (one job:
        akmc_load_occupancy / akmc_get_occupancy; several: the all-jobs forms), R rounds, the
        lattices read back; (seconds, hops, bytes each way per step) of this rank."""
        torch = self.torch
        whole = torch.from_numpy(np.concatenate(lattices)).pin_memory()
        whole_out = torch.empty(whole.numel(), dtype=torch.uint8).pin_memory()
        t0 = e0 = None
        for step in range(steps + 1):  # step 0 untimed: the first transfer sets up its buffers
            if step == 1:
                self.sync_all()
                e0 = eng.counters()
                self.clocks.mark(name)
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
        self.sync_all()
        dt = time.perf_counter() - t0
        self.clocks.end(name)
        return dt, eng.counters()["hops"] - e0["hops"], int(whole.numel())


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


WORKLOAD_TEXT = {
    "scale": "BCC 256^3 cells Fe-1.34Cu-0.7Ni-0.3Mn, 16^3-cell domain blocks x 8 sectors, 671 vacancies, EAM, "
             "T=563 K",
    "scale32": "BCC 256^3 cells Fe-1.34Cu-0.7Ni-0.3Mn, 16^3-cell blocks, 671 vacancies, EAM FP32-compensated, "
               "T=563 K",
    "batched": "512 boxes, edge log-uniform 16-48 cells, Cu 0.5-1.5 / Ni 0-1 / Mn 0-0.5 at.%, vacancy fraction "
               "1e-4, T 473-673 K, EAM FP32-compensated",
    "serial": "BCC 20^3 cells Fe-1.34Cu, 20 vacancies, single domain, EAM, T=573 K",
}


def config_of(args, jobs, workload=None, rounds=None):
    workload = workload or args.workload
    j = jobs[0]
    c = {"workload": WORKLOAD_TEXT[workload],
         "jobs": len(jobs), "sites": int(sum(2 * np.prod(x["box"]) for x in jobs)),
         "vacancies": int(sum(x["n_vacancies"] for x in jobs)),
         "rounds_per_step": rounds if rounds is not None else args.rounds_per_step,
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


# ---------------------------------------------------------------------------
def autotune_batched(ak, jobs, device, block_edge):
    """The batched jobs' decomposition and kernel shape: the fastest of the tuner's candidates
    on this job set (outside any timed region), or the fixed edge given with the default shape."""
    import akmc_b200.autotune as at

    if block_edge <= 0:
        lats = [ak.create_lattice(j["box"], j["alloy"], j["n_vacancies"], j["seed"]) for j in jobs]
        choice, table = at.tune(jobs, lats, ak.eam_johnson(42), device=device)
        tuned = dict(choice, trial_hops_per_s={k: round(v) for k, v in table.items()})
    else:
        tuned = {"block_edge": block_edge, "eval_warps": 8, "flow_take": 0}
    for j in jobs:
        j["blocks"] = tuple(at.blocks_for(e, tuned["block_edge"]) for e in j["box"])
    return tuned


def plain_one_at_a_time(ak, jobs, idx, R, device, stream, torch, clocks, name):
    """The plain form of a multi-job workload: the sampled jobs in FP64, each alone in its own
    context, R rounds each after one untimed step of R rounds; hops/s = all hops / all device
    time between CUDA events."""
    eam = ak.eam_johnson(42)
    hops, ms = 0, 0.0
    clocks.mark(name)
    for i in idx:
        j = jobs[i]
        occ = ak.create_lattice(j["box"], j["alloy"], j["n_vacancies"], j["seed"])
        cfg = ak.job_config(j["box"], blocks=j["blocks"], energy_model=j.get("model", 1), precision=ak.FP64,
                            temperature=j["temperature"], seed=j["seed"], eam=eam if j.get("model", 1) else None)
        with ak.Engine(device=device, stream=stream.cuda_stream) as eng:
            eng.add_job(cfg, occ)
            eng.prepare()
            eng.run_rounds(R)
            eng.sync()
            h0 = eng.counters()["hops"]
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            eng.run_rounds(R)
            e1.record(stream)
            eng.sync()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            hops += eng.counters()["hops"] - h0
    clocks.end(name)
    return ms, hops


def serve_stream(ak, device, rate, seconds, lanes, chunk, order, clocks=None, name="serve"):
    """Serving workload through akmc_server: arrivals replayed in real time, every job waited
    for; latency = result published - submitted."""
    jobs = serve_jobs(rate, seconds)
    eam = ak.eam_johnson(42)
    prepared = []
    for j in jobs:
        occ = ak.create_lattice(j["box"], j["alloy"], j["n_vacancies"], j["seed"])
        cfg = ak.job_config(j["box"], blocks=j["blocks"], energy_model=ak.MODEL_EAM, precision=j["precision"],
                            temperature=j["temperature"], seed=j["seed"], eam=eam, hop_budget=j["hop_budget"])
        prepared.append((j["t"], cfg, occ))
    srv = ak.Server(device=device, lanes=lanes, chunk_rounds=chunk, order=1 if order == "smallest" else 0)
    if clocks:
        clocks.mark(name)
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
    if clocks:
        clocks.end(name)
    prof = srv.profile()
    srv.close()
    lat = np.array(lat)
    return {
        "value": hops / wall, "unit": "hops/s", "dtype": "f32c", "wall_s": wall,
        "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
        "latency_max_s": float(lat.max()),
        "config": {"workload": "serving: Poisson arrivals %.0f/s for %.0f s, edge log-uniform 16-96 cells, hop "
                               "budget log-uniform 1e4-1e6, EAM FP32-compensated" % (rate, seconds),
                   "jobs": len(jobs), "lanes": lanes, "chunk_rounds": chunk, "order": order,
                   "offered_hops_per_s": sum(j["hop_budget"] for j in jobs) / seconds},
        "server_profile": prof,
    }


def run_serve(args, ak, device):
    """--workload serve: one JSON line for the served stream."""
    clocks = Clocks(device)
    clocks.start()
    s = serve_stream(ak, device, args.serve_rate, args.serve_seconds, args.serve_lanes, args.serve_chunk,
                     args.serve_order, clocks)
    clocks.stop()
    line = {"metric": METRIC, "value": s["value"], "unit": "hops/s", "n_gpus": 1, "steps": 1, "warmup": 0,
            "ms_per_step": 1e3 * s["wall_s"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32c", "data": "synthetic", "config": s["config"], "clocks": clocks.report("serve")}
    for k in ("latency_p50_s", "latency_p99_s", "latency_max_s", "wall_s", "server_profile"):
        line[k] = s[k]
    print(json.dumps(line))


def extras(args, ak, device, stream, torch, runner, clocks):
    """The rest of the metric on the same GPU, each part with its own clock record: the 256^3
    lattice in FP32-comp, the 512 batched boxes in FP32-comp (autotuned), a seeded sample of the
    same boxes in plain FP64 one job at a time, their ratio, and the served job stream."""
    out = {}
    # FP32-comp on the same 256^3 lattice and seed as `value`
    jobs = workload_jobs("scale32")
    eng, _ = build_engine(ak, jobs, device, stream.cuda_stream)
    ms, hops = runner.device_rate(eng, args.rounds_per_step, args.steps, args.warmup, "scale32")
    out["scale32"] = {"value": hops / (ms / 1e3), "unit": "hops/s", "dtype": "f32c", "steps": args.steps,
                      "ms_per_step": ms / args.steps, "hops_timed": int(hops),
                      "config": config_of(args, jobs, "scale32"), "clocks": None}
    eng.close()

    # batched FP32-comp: 512 boxes in one context, autotuned decomposition
    R = args.batched_rounds
    jobs = workload_jobs("batched")
    tuned = autotune_batched(ak, jobs, device, args.block_edge)
    eng, lattices = build_engine(ak, jobs, device, stream.cuda_stream, shape=tuned)
    ms, hops = runner.device_rate(eng, R, args.steps, args.warmup, "batched")
    e_dt, e_hops, nbytes = runner.end_to_end(eng, lattices, R, max(3, args.steps // 2), "batched_e2e")
    cfg = config_of(args, jobs, "batched", R)
    cfg["autotune"] = tuned
    batched = {"value": hops / (ms / 1e3), "unit": "hops/s", "dtype": "f32c", "steps": args.steps,
               "ms_per_step": ms / args.steps, "hops_timed": int(hops), "config": cfg,
               "e2e": {"value": e_hops / e_dt, "unit": "hops/s", "h2d_bytes_per_step": nbytes,
                       "d2h_bytes_per_step": nbytes}, "clocks": None}
    out["batched"] = batched
    eng.close()

    # the same boxes in plain FP64, each alone (the configuration's default decomposition)
    jobs = workload_jobs("batched")
    idx = plain_sample(len(jobs), args.plain_sample)
    ms, hops = plain_one_at_a_time(ak, jobs, idx, R, device, stream, torch, clocks, "plain")
    out["plain_one_at_a_time"] = {
        "value": hops / (ms / 1e3), "unit": "hops/s", "dtype": "f64", "hops_timed": int(hops), "ms": ms,
        "config": {"workload": WORKLOAD_TEXT["batched"].replace("EAM FP32-compensated", "EAM FP64"),
                   "jobs_timed": len(idx), "sample": "seeded uniform sample of the 512 boxes without replacement "
                                                     "(numpy default_rng(42)), job indices %s" % idx,
                   "rounds_per_job": R, "note": "each job alone in its own context, after one untimed step"},
        "clocks": None}
    out["batched_over_plain"] = out["batched"]["value"] / out["plain_one_at_a_time"]["value"]

    # the served Poisson job stream
    if args.serve_seconds > 0:
        out["serve"] = serve_stream(ak, device, args.serve_rate, args.serve_seconds, args.serve_lanes,
                                    args.serve_chunk, args.serve_order, clocks, "serve")
        out["serve"]["clocks"] = None
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="scale", choices=["scale", "scale32", "batched", "serial", "serve"])
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-seconds", type=float, default=None,
                    help="arrival window of the serving stream (default 10 s; 5 s as an extra of the default run)")
    ap.add_argument("--serve-lanes", type=int, default=2)
    ap.add_argument("--serve-chunk", type=int, default=16, help="sector rounds per server chunk")
    ap.add_argument("--serve-order", default="fifo", choices=["fifo", "smallest"],
                    help="admission order: arrival, or smallest hop budget first")
    ap.add_argument("--rounds-per-step", type=int, default=0, help="0: the workload's default")
    ap.add_argument("--batched-rounds", type=int, default=256, help="rounds per step of the batched extra")
    ap.add_argument("--plain-sample", type=int, default=64,
                    help="batched boxes the plain FP64 form times one at a time (seeded sample)")
    ap.add_argument("--one-at-a-time", type=int, default=0, metavar="N",
                    help="only time N sampled jobs of the workload in plain FP64, each alone")
    ap.add_argument("--model", default="eam", choices=["eam", "pairbond"],
                    help="energy model: the synthetic EAM, or the reference's own pair-bond model (FP64)")
    ap.add_argument("--schedule", default="auto", choices=["auto", "rounds", "flow"],
                    help="round schedule of the context (auto: dependency-driven where allowed)")
    ap.add_argument("--block-edge", type=int, default=0,
                    help="batched workload: blocks of at most this many cells; 0 = autotune before timing")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="default run: only the 256^3 FP64 line, without the other parts of the metric")
    args = ap.parse_args()
    if args.rounds_per_step <= 0:
        args.rounds_per_step = DEFAULT_ROUNDS[args.workload]
    if args.serve_seconds is None:
        args.serve_seconds = 10.0 if args.workload == "serve" else 5.0

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
    clocks = Clocks(local)
    clocks.start()
    runner = Runner(torch, stream, dist, clocks)
    if args.one_at_a_time:
        idx = plain_sample(len(jobs), args.one_at_a_time)
        ms, hops = plain_one_at_a_time(ak, jobs, idx, args.rounds_per_step, local, stream, torch, clocks, "plain")
        clocks.stop()
        print(json.dumps({"metric": METRIC, "impl": "b200 plain FP64, one job at a time", "value": hops / (ms / 1e3),
                          "unit": "hops/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f64",
                          "data": "synthetic", "config": {"workload": WORKLOAD_TEXT[args.workload],
                                                          "jobs_timed": len(idx), "job_indices": idx,
                                                          "rounds_per_job": args.rounds_per_step},
                          "hops_timed": int(hops), "ms": ms, "clocks": clocks.report("plain")}))
        return
    tuned = None
    if args.workload == "batched":
        tuned = autotune_batched(ak, jobs, local, args.block_edge)
    eng, lattices = build_engine(ak, jobs, local, stream.cuda_stream,
                                 schedule={"auto": 0, "rounds": 1, "flow": 2}[args.schedule], shape=tuned)
    R = args.rounds_per_step
    eam = jobs[0].get("model", 1) == 1

    ms, hops = runner.device_rate(eng, R, args.steps, args.warmup, "main")
    ms_all, hops_all = reduce_over_ranks(dist, ms, hops, "cuda")
    value = hops_all / (ms_all / 1e3)

    # kernels launched per timed step: round by round, k_bucket + k_hop + k_finalize per round
    # (captured in CUDA graphs); dependency-driven, per launch of up to 1024 rounds k_flow_begin
    # once per step, then k_flow_prep, k_flow_slots, k_flow and k_flow_finalize
    sched = eng.round_schedule()
    sched_name = "flow" if sched == ak.SCHEDULE_FLOW else "rounds"
    launches_per_step = (1 + 4 * ((R + 1023) // 1024)) if sched == ak.SCHEDULE_FLOW else 3 * R

    roofline = runner.roofline(eng, R, max(1, args.steps // 2), eam, args.workload)
    e_dt, e_hops, nbytes = runner.end_to_end(eng, lattices, R, args.steps, "e2e")
    e_dt_all, e_hops_all = reduce_over_ranks(dist, e_dt, e_hops, "cuda")
    e2e = {"value": e_hops_all / e_dt_all, "unit": "hops/s", "h2d_bytes_per_step": nbytes,
           "d2h_bytes_per_step": nbytes,
           "note": "each step restarts the jobs from the host lattices (upload, density rebuild), runs R rounds and "
                   "reads the lattices back"}
    eng.close()

    more = None
    if rank == 0 and world == 1 and args.workload == "scale" and args.model == "eam" and not args.no_extras:
        more = extras(args, ak, local, stream, torch, runner, clocks)
    clocks.stop()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "hops/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_all / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if jobs[0]["precision"] == 0 else "f32c", "data": "synthetic",
            "config": config_of(args, jobs), "roofline": roofline, "e2e": e2e,
            "gpu_launches": launches_per_step * args.steps, "schedule": sched_name, "clocks": clocks.report("main"),
            "hops_timed": int(hops_all),
        }
        line["e2e"]["clocks"] = clocks.report("e2e")
        if tuned:
            line["config"]["autotune"] = tuned
        if more:
            for k in ("scale32", "batched", "plain_one_at_a_time", "serve"):
                if k in more:
                    more[k]["clocks"] = clocks.report(k if k != "plain_one_at_a_time" else "plain")
            if "batched" in more:
                more["batched"]["e2e"]["clocks"] = clocks.report("batched_e2e")
            line.update(more)
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(jobs)
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
