"""ctypes binding of libakmc_b200.so (include/akmc.h).

The compute path is the CUDA library; this module only marshals arguments.
There is no CPU fallback: loading fails with an error when the library has not
been built, and every non-zero status raises AkmcError.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(os.path.dirname(HERE))  # misa-akmc-gpu_b200/
LIB_PATH = os.path.join(PKG, "lib", "libakmc_b200.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "akmc.h")

MODEL_PAIRBOND, MODEL_EAM = 0, 1
FP64, FP32C = 0, 1
SERVE_FIFO, SERVE_SMALLEST_BUDGET = 0, 1
RNG_XOSHIRO = 0
V, FE, CU, NI, MN = 0, 1, 2, 4, 8
MAX_SECTOR_VACANCIES = 64
NOALLOC_MAX_BLOCKS = 8192
SCHEDULE_AUTO, SCHEDULE_ROUNDS, SCHEDULE_FLOW = 0, 1, 2
SECTOR_ORDER = (0, 7, 2, 5, 3, 4, 1, 6)

STATUS = {
    0: "AKMC_OK",
    -1: "AKMC_EINVAL",
    -2: "AKMC_ENOMEM",
    -3: "AKMC_ECUDA",
    -4: "AKMC_ETIMEOUT",
    -5: "AKMC_EBUSY",
    -6: "AKMC_ESTATE",
    -7: "AKMC_EOVERFLOW",
    -8: "AKMC_ERANGE",
    -9: "AKMC_ENOTFOUND",
}


class AkmcError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__("%s (%d): %s" % (STATUS.get(status, "?"), status, msg))


class EamTables(C.Structure):
    _fields_ = [
        ("n_shells", C.c_int32),
        ("reserved", C.c_int32),
        ("f_shell", (C.c_double * 5) * 4),
        ("phi_shell", ((C.c_double * 5) * 4) * 4),
        ("F", C.c_double * 5000),
    ]


class JobConfig(C.Structure):
    _fields_ = [
        ("box", C.c_int64 * 3),
        ("blocks", C.c_int32 * 3),
        ("energy_model", C.c_int32),
        ("precision", C.c_int32),
        ("rng", C.c_int32),
        ("lattice_const", C.c_double),
        ("cutoff_radius", C.c_double),
        ("attempt_freq", C.c_double),
        ("temperature", C.c_double),
        ("sector_window", C.c_double),
        ("seed", C.c_uint64),
        ("hop_budget", C.c_int64),
        ("max_rounds", C.c_int64),
        ("eam", C.POINTER(EamTables)),
    ]


class Event(C.Structure):
    _fields_ = [
        ("round", C.c_int64),
        ("hop", C.c_int64),
        ("from_site", C.c_int64),
        ("to_site", C.c_int64),
        ("block", C.c_int32),
        ("species", C.c_int32),
        ("u", C.c_double),
        ("total", C.c_double),
        ("dt", C.c_double),
        ("n_act", C.c_int32),
        ("n_dirty", C.c_int32),
        ("job", C.c_int32),
        ("reserved", C.c_int32),
    ]


EVENT_DTYPE = np.dtype(
    [
        ("round", "<i8"),
        ("hop", "<i8"),
        ("from_site", "<i8"),
        ("to_site", "<i8"),
        ("block", "<i4"),
        ("species", "<i4"),
        ("u", "<f8"),
        ("total", "<f8"),
        ("dt", "<f8"),
        ("n_act", "<i4"),
        ("n_dirty", "<i4"),
        ("job", "<i4"),
        ("reserved", "<i4"),
    ]
)
assert EVENT_DTYPE.itemsize == C.sizeof(Event)


class JobState(C.Structure):
    _fields_ = [
        ("round", C.c_int64),
        ("hops", C.c_int64),
        ("done", C.c_int32),
        ("n_blocks", C.c_int32),
        ("n_sites", C.c_int64),
        ("n_vacancies", C.c_int64),
    ]


class ContextConfig(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("graph_rounds", C.c_int32),
        ("stream", C.c_void_p),
        ("event_log_capacity", C.c_int64),
        ("hop_cap_per_round", C.c_int64),
        ("flow_sweep_limit", C.c_int64),
        ("max_jobs", C.c_int32),
        ("max_block_edge", C.c_int32),
        ("max_blocks", C.c_int64),
        ("max_vacancies", C.c_int64),
        ("eval_warps", C.c_int32),
        ("flow_take", C.c_int32),
    ]


class ServerConfig(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("lanes", C.c_int32),
        ("budget_bytes", C.c_int64),
        ("max_batch_jobs", C.c_int32),
        ("chunk_rounds", C.c_int32),
        ("order", C.c_int32),
        ("chunk_us", C.c_int32),
    ]


class JobResult(C.Structure):
    _fields_ = [
        ("hops", C.c_int64),
        ("rounds", C.c_int64),
        ("submit_s", C.c_double),
        ("start_s", C.c_double),
        ("finish_s", C.c_double),
        ("status", C.c_int32),
        ("n_blocks", C.c_int32),
        ("error", C.c_char * 128),
        ("clocks_fnv", C.c_uint64),
    ]


class RunConfig(C.Structure):
    _fields_ = [
        ("box", C.c_int64 * 3),
        ("lattice_const", C.c_double),
        ("cutoff_radius", C.c_double),
        ("create_random", C.c_int32),
        ("n_types", C.c_int32),
        ("type_codes", C.c_int32 * 4),
        ("ratio", C.c_int64 * 4),
        ("va_count", C.c_int64),
        ("seed_create_types", C.c_int64),
        ("seed_create_vacancy", C.c_int64),
        ("seed_event_selection", C.c_int64),
        ("seed_time_inc", C.c_int64),
        ("temperature", C.c_double),
        ("physics_time", C.c_double),
        ("attempt_freq", C.c_double),
        ("dpasm1", C.c_double),
        ("steps_limit", C.c_int64),
        ("isgenr", C.c_int32),
        ("energy_model", C.c_int32),
        ("precision", C.c_int32),
        ("creation", C.c_int32),
        ("blocks", C.c_int32 * 3),
        ("reserved", C.c_int32),
        ("sector_window", C.c_double),
        ("hop_budget", C.c_int64),
        ("seed", C.c_uint64),
        ("pot_seed", C.c_uint64),
        ("dump_interval", C.c_int64),
        ("logs_interval", C.c_int64),
        ("dump_file_path", C.c_char * 256),
        ("logs_file", C.c_char * 256),
        ("create_pipe", C.c_int32),
        ("reserved2", C.c_int32),
        ("pipe_input_box", C.c_char * 256),
    ]


# every symbol include/akmc.h declares, with (restype, argtypes)
_vp, _i32, _i64, _u64, _d = C.c_void_p, C.c_int32, C.c_int64, C.c_uint64, C.c_double
SIGNATURES = {
    "akmc_status_string": (C.c_char_p, [C.c_int]),
    "akmc_last_error": (C.c_int, [_vp, C.c_char_p, _i32]),
    "akmc_initialize_gpu": (C.c_int, [_i32, C.POINTER(_i32)]),
    "akmc_create": (C.c_int, [C.POINTER(ContextConfig), C.POINTER(_vp)]),
    "akmc_destroy": (C.c_int, [_vp]),
    "akmc_add_job": (C.c_int, [_vp, C.POINTER(JobConfig), _vp, _i64, C.POINTER(_i32)]),
    "akmc_prepare": (C.c_int, [_vp]),
    "akmc_admit_job": (C.c_int, [_vp, C.POINTER(JobConfig), _vp, _i64, C.POINTER(_i32)]),
    "akmc_retire_job": (C.c_int, [_vp, _i32]),
    "akmc_run_for": (C.c_int, [_vp, _i64, _i64]),
    "akmc_run_rounds": (C.c_int, [_vp, _i64]),
    "akmc_run_rounds_noalloc": (C.c_int, [_vp, _i64]),
    "akmc_set_round_schedule": (C.c_int, [_vp, _i32]),
    "akmc_get_round_schedule": (C.c_int, [_vp, C.POINTER(_i32)]),
    "akmc_run": (C.c_int, [_vp, _i64]),
    "akmc_sync": (C.c_int, [_vp]),
    "akmc_stream": (_vp, [_vp]),
    "akmc_gpu_final": (C.c_int, [_vp]),
    "akmc_get_job_state": (C.c_int, [_vp, _i32, C.POINTER(JobState)]),
    "akmc_get_job_states": (C.c_int, [_vp, _vp, _i32]),
    "akmc_load_occupancies": (C.c_int, [_vp, _vp, _i64]),
    "akmc_get_occupancies": (C.c_int, [_vp, _vp, _i64]),
    "akmc_get_occupancy": (C.c_int, [_vp, _i32, _vp, _i64]),
    "akmc_get_rho": (C.c_int, [_vp, _i32, _vp, _i64]),
    "akmc_get_block_clocks": (C.c_int, [_vp, _i32, _vp, _vp, _i32]),
    "akmc_get_events": (C.c_int, [_vp, _vp, _i64, C.POINTER(_i64)]),
    "akmc_get_counters": (C.c_int, [_vp, _vp]),
    "akmc_calculate": (C.c_int, [_vp, _i32, _i32, C.POINTER(_d)]),
    "akmc_select_and_perform": (C.c_int, [_vp, _i32, _i32, _d, C.POINTER(Event)]),
    "akmc_get_calculated_rates": (C.c_int, [_vp, _vp, _vp, _vp, _i64, C.POINTER(_i64)]),
    "akmc_eam_johnson": (C.c_int, [_u64, _d, _d, C.POINTER(EamTables)]),
    "akmc_create_lattice": (C.c_int, [_vp, _vp, _vp, _i64, _u64, _vp, _i64]),
    "akmc_cluster_stats": (C.c_int, [_vp, _vp, C.POINTER(_i64), _vp, _i64]),
    "akmc_job_cluster_stats": (C.c_int, [_vp, _i32, C.POINTER(_i64), _vp, _i64]),
    "akmc_snapshot_size": (C.c_int, [_vp, _i32, C.POINTER(_i64)]),
    "akmc_save_snapshot": (C.c_int, [_vp, _i32, _vp, _i64, C.POINTER(_i64)]),
    "akmc_restore_snapshot": (C.c_int, [_vp, _i32, _vp, _i64]),
    "akmc_device_math": (C.c_int, [_vp, _vp, _i64, _vp, _vp]),
    "akmc_server_create": (C.c_int, [_vp, C.POINTER(_vp)]),
    "akmc_server_submit": (C.c_int, [_vp, _vp, _vp, _i64, C.POINTER(_i64)]),
    "akmc_server_poll": (C.c_int, [_vp, _i64, _vp, _vp, _i64, C.POINTER(_i32)]),
    "akmc_server_wait": (C.c_int, [_vp, _i64, _d, _vp, _vp, _i64]),
    "akmc_server_profile": (C.c_int, [_vp, _vp, _vp]),
    "akmc_server_stats": (C.c_int, [_vp, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64)]),
    "akmc_server_shutdown": (C.c_int, [_vp]),
    "akmc_load_occupancy": (C.c_int, [_vp, _i32, _vp, _i64]),
    "akmc_get_phase_cycles": (C.c_int, [_vp, _vp]),
    "akmc_set_kernel_timing": (C.c_int, [_vp, _i32]),
    "akmc_get_kernel_timing": (C.c_int, [_vp, C.POINTER(_d), C.POINTER(_i64)]),
    "akmc_config_parse": (C.c_int, [C.c_char_p, C.POINTER(RunConfig), C.c_char_p, _i32]),
    "akmc_config_lattice": (C.c_int, [C.POINTER(RunConfig), _vp, _i64]),
    "akmc_config_job": (C.c_int, [C.POINTER(RunConfig), C.POINTER(EamTables), C.POINTER(JobConfig)]),
    "akmc_host_time_loop": (C.c_int, [_vp, _i32, _i64, _u64, _d, _vp, _i64, C.POINTER(_i64), _vp]),
    "akmc_dump_lattice": (C.c_int, [_vp, _vp, _i32, C.c_char_p]),
}


def config_parse(text):
    cfg = RunConfig()
    err = C.create_string_buffer(256)
    rc = lib().akmc_config_parse(text.encode() if isinstance(text, str) else text, C.byref(cfg), err, 256)
    if rc:
        raise AkmcError(rc, err.value.decode())
    return cfg


def config_lattice(cfg):
    n = int(2 * cfg.box[0] * cfg.box[1] * cfg.box[2])
    occ = np.empty(n, np.uint8)
    _check(lib().akmc_config_lattice(C.byref(cfg), _ptr(occ), n))
    return occ


def config_job(cfg, eam=None):
    out = JobConfig()
    _check(lib().akmc_config_job(C.byref(cfg), C.byref(eam) if eam is not None else None, C.byref(out)))
    out._eam_ref = eam
    return out


def dump_lattice(occ, box, path, ghost=2):
    occ = np.ascontiguousarray(occ, np.uint8)
    box = np.asarray(box, np.int64)
    _check(lib().akmc_dump_lattice(_ptr(occ), _ptr(box), ghost, path.encode()))

_lib = None


def lib_path():
    return LIB_PATH


def lib():
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "libakmc_b200.so not built (%s); run python misa-akmc-gpu_b200/build.py" % LIB_PATH
            )
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _check(rc, ctx=None):
    if rc != 0:
        msg = ""
        if ctx:
            buf = C.create_string_buffer(512)
            lib().akmc_last_error(ctx, buf, 512)
            msg = buf.value.decode(errors="replace")
        raise AkmcError(rc, msg)


def eam_johnson(seed=42, lattice_const=2.855, cutoff=5.6):
    t = EamTables()
    _check(lib().akmc_eam_johnson(seed, lattice_const, cutoff, C.byref(t)))
    return t


def create_lattice(box, alloy, n_vacancies, seed):
    box = np.asarray(box, np.int64)
    codes = np.array([a[0] for a in alloy] + [FE] * (4 - len(alloy)), np.int32)
    ratio = np.array([a[1] for a in alloy] + [0] * (4 - len(alloy)), np.int64)
    occ = np.empty(int(2 * box[0] * box[1] * box[2]), np.uint8)
    _check(lib().akmc_create_lattice(_ptr(box), _ptr(codes), _ptr(ratio), n_vacancies, seed, _ptr(occ), occ.size))
    return occ


def cluster_stats(occ, box, hist_len=64):
    occ = np.ascontiguousarray(occ, np.uint8)
    box = np.asarray(box, np.int64)
    iso = C.c_int64(0)
    hist = np.zeros(hist_len, np.int64)
    _check(lib().akmc_cluster_stats(_ptr(occ), _ptr(box), C.byref(iso), _ptr(hist), hist_len))
    return int(iso.value), hist


def job_config(
    box,
    blocks=(1, 1, 1),
    energy_model=MODEL_EAM,
    precision=FP64,
    lattice_const=2.855,
    cutoff=5.6,
    attempt_freq=6e12,
    temperature=573.0,
    window=3.0e-7,
    seed=42,
    hop_budget=0,
    max_rounds=0,
    eam=None,
):
    c = JobConfig()
    c.box[:] = list(box)
    c.blocks[:] = list(blocks)
    c.energy_model = energy_model
    c.precision = precision
    c.rng = RNG_XOSHIRO
    c.lattice_const = lattice_const
    c.cutoff_radius = cutoff
    c.attempt_freq = attempt_freq
    c.temperature = temperature
    c.sector_window = window
    c.seed = seed
    c.hop_budget = hop_budget
    c.max_rounds = max_rounds
    c._eam_ref = eam
    c.eam = C.pointer(eam) if eam is not None else C.POINTER(EamTables)()
    return c


class Engine:
    """One akmc_ctx: a set of jobs advanced together on one GPU."""

    def __init__(self, device=0, stream=None, event_log_capacity=0, graph_rounds=32, hop_cap_per_round=0,
                 flow_sweep_limit=0, max_jobs=0, max_block_edge=0, max_blocks=0, max_vacancies=0, eval_warps=0,
                 flow_take=0):
        """max_jobs > 0 leaves room for jobs admitted after prepare (admit_job): that many jobs,
        max_blocks domain blocks and max_vacancies vacancies held at once, blocks of at most
        max_block_edge cells."""
        cfg = ContextConfig()
        cfg.device = device
        cfg.graph_rounds = graph_rounds
        cfg.stream = stream
        cfg.event_log_capacity = event_log_capacity
        cfg.hop_cap_per_round = hop_cap_per_round
        cfg.flow_sweep_limit = flow_sweep_limit
        cfg.max_jobs = max_jobs
        cfg.max_block_edge = max_block_edge
        cfg.max_blocks = max_blocks
        cfg.max_vacancies = max_vacancies
        cfg.eval_warps = eval_warps
        cfg.flow_take = flow_take
        h = C.c_void_p()
        _check(lib().akmc_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self.jobs = []

    def close(self):
        if self.h:
            lib().akmc_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        _check(rc, self.h)

    def add_job(self, cfg, occ):
        occ = np.ascontiguousarray(occ, np.uint8)
        jid = C.c_int32(-1)
        self._ck(lib().akmc_add_job(self.h, C.byref(cfg), _ptr(occ), occ.size, C.byref(jid)))
        self.jobs.append((cfg, occ.size))
        return jid.value

    def prepare(self):
        self._ck(lib().akmc_prepare(self.h))

    def admit_job(self, cfg, occ):
        """akmc_admit_job: a job added to the prepared, running context; returns its slot id."""
        occ = np.ascontiguousarray(occ, np.uint8)
        jid = C.c_int32(-1)
        self._ck(lib().akmc_admit_job(self.h, C.byref(cfg), _ptr(occ), occ.size, C.byref(jid)))
        while len(self.jobs) <= jid.value:
            self.jobs.append(None)
        self.jobs[jid.value] = (cfg, occ.size)
        return jid.value

    def run_for(self, n, max_us):
        """akmc_run_for: up to n more rounds per job, taking no new round after max_us."""
        self._ck(lib().akmc_run_for(self.h, n, max_us))

    def retire_job(self, job):
        """akmc_retire_job: frees the job's slots; its id may be given out again."""
        self._ck(lib().akmc_retire_job(self.h, job))
        self.jobs[job] = None

    def run_rounds(self, n):
        self._ck(lib().akmc_run_rounds(self.h, n))

    def run_rounds_noalloc(self, n):
        """akmc_run_rounds without allocation: round scratch in a fixed device array
        (at most NOALLOC_MAX_BLOCKS domain blocks; calls on one device must not overlap)."""
        self._ck(lib().akmc_run_rounds_noalloc(self.h, n))

    def set_round_schedule(self, schedule):
        """SCHEDULE_AUTO, SCHEDULE_ROUNDS (round by round) or SCHEDULE_FLOW (dependency-driven)."""
        self._ck(lib().akmc_set_round_schedule(self.h, schedule))

    def round_schedule(self):
        """The schedule run_rounds uses: SCHEDULE_ROUNDS or SCHEDULE_FLOW."""
        v = _i32(0)
        self._ck(lib().akmc_get_round_schedule(self.h, C.byref(v)))
        return v.value

    def run(self, max_rounds=0):
        self._ck(lib().akmc_run(self.h, max_rounds))

    def sync(self):
        self._ck(lib().akmc_sync(self.h))

    @property
    def stream(self):
        return lib().akmc_stream(self.h)

    def job_state(self, job=0):
        st = JobState()
        self._ck(lib().akmc_get_job_state(self.h, job, C.byref(st)))
        return dict(round=st.round, hops=st.hops, done=bool(st.done), n_blocks=st.n_blocks,
                    n_sites=st.n_sites, n_vacancies=st.n_vacancies)

    def job_states(self):
        """job_state of every job, read from the device at once."""
        arr = (JobState * len(self.jobs))()
        self._ck(lib().akmc_get_job_states(self.h, C.cast(arr, C.c_void_p), len(self.jobs)))
        return [dict(round=st.round, hops=st.hops, done=bool(st.done), n_blocks=st.n_blocks, n_sites=st.n_sites,
                     n_vacancies=st.n_vacancies) for st in arr]

    def occupancy(self, job=0, out=None):
        """The job's lattice; into `out` (a contiguous uint8 array, pinned memory for a fast
        copy) when given."""
        n = self.jobs[job][1]
        if out is None:
            out = np.empty(n, np.uint8)
        elif out.dtype != np.uint8 or out.size != n or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a contiguous uint8 array of %d sites" % n)
        self._ck(lib().akmc_get_occupancy(self.h, job, _ptr(out), n))
        return out

    def rho(self, job=0):
        n = self.jobs[job][1]
        out = np.empty(n, np.int32)
        self._ck(lib().akmc_get_rho(self.h, job, _ptr(out), n))
        return out

    def block_clocks(self, job=0):
        nb = self.job_state(job)["n_blocks"]
        evo = np.empty((nb, 8), np.float64)
        hops = np.empty(nb, np.int64)
        self._ck(lib().akmc_get_block_clocks(self.h, job, _ptr(evo), _ptr(hops), nb))
        return evo, hops

    def events(self, capacity=1 << 22):
        out = np.empty(capacity, EVENT_DTYPE)
        n = C.c_int64(0)
        self._ck(lib().akmc_get_events(self.h, _ptr(out), capacity, C.byref(n)))
        return out[: n.value].copy()

    def counters(self):
        out = np.zeros(8, np.int64)
        self._ck(lib().akmc_get_counters(self.h, _ptr(out)))
        return dict(hops=int(out[0]), evaluations=int(out[1]), rounds=int(out[2]), blocks=int(out[3]),
                    n_act_sum=int(out[4]), staged_sites=int(out[5]), written_sites=int(out[6]))

    def phase_cycles(self):
        out = np.zeros(16, np.int64)
        self._ck(lib().akmc_get_phase_cycles(self.h, _ptr(out)))
        return out

    def load_occupancy(self, job, occ):
        occ = np.ascontiguousarray(occ, np.uint8)
        self._ck(lib().akmc_load_occupancy(self.h, job, _ptr(occ), occ.size))

    def load_occupancies(self, occ):
        """akmc_load_occupancies: every job's lattice, back to back in job order."""
        occ = np.ascontiguousarray(occ, np.uint8)
        self._ck(lib().akmc_load_occupancies(self.h, _ptr(occ), occ.size))

    def occupancies(self, out=None):
        """akmc_get_occupancies: every job's lattice, back to back in job order (into `out`)."""
        n = sum(j[1] for j in self.jobs if j is not None)
        if out is None:
            out = np.empty(n, np.uint8)
        elif out.dtype != np.uint8 or out.size != n or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a contiguous uint8 array of %d sites" % n)
        self._ck(lib().akmc_get_occupancies(self.h, _ptr(out), n))
        return out

    def set_kernel_timing(self, enable):
        self._ck(lib().akmc_set_kernel_timing(self.h, int(enable)))

    def kernel_timing(self):
        ms = C.c_double(0.0)
        n = C.c_int64(0)
        self._ck(lib().akmc_get_kernel_timing(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def save_snapshot(self, job=0):
        """Restart snapshot of the job (bytes)."""
        n = C.c_int64(0)
        self._ck(lib().akmc_snapshot_size(self.h, job, C.byref(n)))
        buf = np.empty(n.value, np.uint8)
        w = C.c_int64(0)
        self._ck(lib().akmc_save_snapshot(self.h, job, _ptr(buf), n.value, C.byref(w)))
        return buf[: w.value].tobytes()

    def restore_snapshot(self, job, data):
        buf = np.frombuffer(data, np.uint8)
        self._ck(lib().akmc_restore_snapshot(self.h, job, _ptr(buf), len(buf)))

    def cluster_stats(self, job=0, hist_len=64):
        """(isolated-Cu count, Cu cluster-size histogram) of the job's lattice, on the device."""
        iso = C.c_int64(0)
        hist = np.zeros(hist_len, np.int64)
        self._ck(lib().akmc_job_cluster_stats(self.h, job, C.byref(iso), _ptr(hist), hist_len))
        return int(iso.value), hist

    def calculate(self, job, sector_id):
        t = C.c_double(0.0)
        self._ck(lib().akmc_calculate(self.h, job, sector_id, C.byref(t)))
        return t.value

    def calculated_rates(self, capacity=MAX_SECTOR_VACANCIES):
        """(sites int32[n], delta_e float64[n, 8] in eV, rates float64[n, 8] in Hz) of the
        jumps behind the last calculate(), in the sector's list order."""
        sites = np.empty(capacity, np.int32)
        de = np.empty((capacity, 8), np.float64)
        rates = np.empty((capacity, 8), np.float64)
        n = C.c_int64(0)
        self._ck(lib().akmc_get_calculated_rates(self.h, _ptr(sites), _ptr(de), _ptr(rates), capacity, C.byref(n)))
        k = n.value
        return sites[:k].copy(), de[:k].copy(), rates[:k].copy()

    def select_and_perform(self, job, sector_id, u):
        ev = Event()
        self._ck(lib().akmc_select_and_perform(self.h, job, sector_id, u, C.byref(ev)))
        return ev

    def host_time_loop(self, job, n_rounds, seed, window=3e-7, capacity=1 << 20):
        ev = np.empty(capacity, EVENT_DTYPE)
        n = C.c_int64(0)
        evo = np.zeros(8, np.float64)
        self._ck(lib().akmc_host_time_loop(self.h, job, n_rounds, seed, window, _ptr(ev), capacity, C.byref(n),
                                           _ptr(evo)))
        return ev[: n.value].copy(), evo

    def device_math(self, x):
        x = np.ascontiguousarray(x, np.float64)
        e = np.empty_like(x)
        l = np.empty_like(x)
        self._ck(lib().akmc_device_math(self.h, _ptr(x), x.size, _ptr(e), _ptr(l)))
        return e, l


def _result(r):
    return dict(hops=r.hops, rounds=r.rounds, submit_s=r.submit_s, start_s=r.start_s, finish_s=r.finish_s,
                status=r.status, n_blocks=r.n_blocks, error=r.error.decode(errors="replace"),
                clocks_fnv=r.clocks_fnv)


def clocks_fnv(evo, hops):
    """The job result's clocks_fnv of block clocks evo[nblocks][8] (FP64) and hops[nblocks]."""
    h = 0xCBF29CE484222325
    for b in range(len(hops)):
        data = np.ascontiguousarray(evo[b], np.float64).tobytes() + np.int64(hops[b]).tobytes()
        for x in data:
            h = ((h ^ x) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


class Server:
    """akmc_server: queued jobs admitted into the lanes' running contexts as room frees up,
    results as each job ends."""

    def __init__(self, device=0, lanes=0, budget_bytes=0, max_batch_jobs=0, chunk_rounds=0, order=0, chunk_us=0):
        cfg = ServerConfig(device, lanes, budget_bytes, max_batch_jobs, chunk_rounds, order, chunk_us)
        h = C.c_void_p()
        _check(lib().akmc_server_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self.sizes = {}

    def submit(self, cfg, occ):
        occ = np.ascontiguousarray(occ, np.uint8)
        t = C.c_int64(0)
        _check(lib().akmc_server_submit(self.h, C.byref(cfg), _ptr(occ), occ.size, C.byref(t)))
        self.sizes[t.value] = occ.size
        return t.value

    def poll(self, ticket):
        """(result, final lattice) once the job is done, else None."""
        n = self.sizes.get(ticket, 0)
        out = np.empty(n, np.uint8)
        r = JobResult()
        ready = C.c_int32(0)
        _check(lib().akmc_server_poll(self.h, ticket, C.byref(r), _ptr(out), n, C.byref(ready)))
        if not ready.value:
            return None
        self.sizes.pop(ticket, None)
        return _result(r), out

    def wait(self, ticket, timeout=60.0):
        n = self.sizes.get(ticket, 0)
        out = np.empty(n, np.uint8)
        r = JobResult()
        _check(lib().akmc_server_wait(self.h, ticket, timeout, C.byref(r), _ptr(out), n))
        self.sizes.pop(ticket, None)
        return _result(r), out

    def profile(self):
        """akmc_server_profile: lane seconds (job-set changes, run, publish, wait) and counts."""
        t = np.zeros(8, np.float64)
        c = np.zeros(3, np.int64)
        _check(lib().akmc_server_profile(self.h, _ptr(t), _ptr(c)))
        return dict(build_s=float(t[0]), run_s=float(t[1]), publish_s=float(t[2]), wait_s=float(t[3]),
                    admit_s=float(t[4]), create_s=float(t[5]), retire_s=float(t[6]),
                    chunks=int(c[0]), mean_batch=float(c[1]) / max(1, int(c[0])), builds=int(c[2]))

    def stats(self):
        q, r, d = C.c_int64(0), C.c_int64(0), C.c_int64(0)
        _check(lib().akmc_server_stats(self.h, C.byref(q), C.byref(r), C.byref(d)))
        return dict(queued=q.value, running=r.value, done=d.value)

    def close(self):
        if self.h:
            lib().akmc_server_shutdown(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
