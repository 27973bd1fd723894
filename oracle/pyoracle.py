"""ctypes binding of the CPU oracle (oracle/akmc_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
the cpu_baseline leg of bench.py, always as the checker.  The product never
imports this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libakmc_oracle.so")

MODEL_PAIRBOND, MODEL_EAM = 0, 1
FP64, FP32C = 0, 1
RNG_XOSHIRO, RNG_MT19937_REF = 0, 1
MATH_PORTABLE, MATH_LIBM = 0, 1
CREATE_XOSHIRO, CREATE_MT19937_REF, CREATE_EXTERNAL, CREATE_MT19937_PILE = 0, 1, 2, 3

V, FE, CU, NI, MN = 0, 1, 2, 4, 8


class AoConfig(C.Structure):
    _fields_ = [
        ("box", C.c_int64 * 3),
        ("blocks", C.c_int32 * 3),
        ("energy_model", C.c_int32),
        ("precision", C.c_int32),
        ("rng_mode", C.c_int32),
        ("math_mode", C.c_int32),
        ("creation_mode", C.c_int32),
        ("log_events", C.c_int32),
        ("lattice_const", C.c_double),
        ("cutoff", C.c_double),
        ("attempt_freq", C.c_double),
        ("temperature", C.c_double),
        ("window", C.c_double),
        ("seed", C.c_uint64),
        ("seed_vacancy", C.c_uint64),
        ("seed_time_inc", C.c_uint64),
        ("pot_seed", C.c_uint64),
        ("type_codes", C.c_int32 * 4),
        ("ratio", C.c_int64 * 4),
        ("n_vacancies", C.c_int64),
        ("pile_xyz", C.c_void_p),
        ("pile_n", C.c_int64),
    ]


class AoEvent(C.Structure):
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
    ]
)
assert EVENT_DTYPE.itemsize == C.sizeof(AoEvent)

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, i64, i32, dp = C.c_void_p, C.c_int64, C.c_int32, C.c_void_p
        L.ao_create.restype = vp
        L.ao_create.argtypes = [C.POINTER(AoConfig), C.c_char_p, C.c_int]
        L.ao_destroy.argtypes = [vp]
        L.ao_nsites.restype = i64
        L.ao_nsites.argtypes = [vp]
        L.ao_nblocks.restype = i32
        L.ao_nblocks.argtypes = [vp]
        for name, args in [
            ("ao_set_occupancy", [vp, dp, i64]),
            ("ao_get_occupancy", [vp, dp]),
            ("ao_get_rho", [vp, dp]),
            ("ao_run_rounds", [vp, i64]),
            ("ao_run_rounds_flow", [vp, i64, C.c_uint64]),
            ("ao_run", [vp, i64, i64]),
            ("ao_get_events", [vp, dp, i64, i64]),
            ("ao_get_block_state", [vp, dp, dp]),
            ("ao_stats", [vp, dp]),
            ("ao_vacancy_rates", [vp, i64, dp, dp]),
            ("ao_eam_export", [vp, dp, dp, dp, dp, dp]),
            ("ao_cluster_stats", [vp, dp, dp, i64]),
            ("ao_neighbours", [vp, i64, dp, dp]),
            ("ao_xoshiro_stream", [C.c_uint64, C.c_uint64, C.c_uint64, dp, i64]),
            ("ao_mt19937_draws", [C.c_uint64, C.c_int, C.c_int, dp, i64]),
        ]:
            f = getattr(L, name)
            f.restype = C.c_int
            f.argtypes = args
        for name in ("ao_round", "ao_total_hops", "ao_num_events"):
            getattr(L, name).restype = i64
            getattr(L, name).argtypes = [vp]
        L.ao_bond_count.restype = C.c_double
        L.ao_bond_count.argtypes = [vp, i64, i32]
        L.ao_exp.restype = C.c_double
        L.ao_exp.argtypes = [C.c_double]
        L.ao_log.restype = C.c_double
        L.ao_log.argtypes = [C.c_double]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def make_config(
    box=(20, 20, 20),
    blocks=(1, 1, 1),
    energy_model=MODEL_EAM,
    precision=FP64,
    rng_mode=RNG_XOSHIRO,
    math_mode=MATH_PORTABLE,
    creation_mode=CREATE_XOSHIRO,
    log_events=1,
    lattice_const=2.855,
    cutoff=5.6,
    attempt_freq=6e12,
    temperature=573.0,
    window=3.0e-7,
    seed=42,
    seed_vacancy=0,
    seed_time_inc=0,
    pot_seed=42,
    alloy=((FE, 9866), (CU, 134)),
    n_vacancies=20,
    pile=None,
):
    """pile: vacancy positions (x doubled, y, z) for creation_mode CREATE_MT19937_PILE."""
    c = AoConfig()
    c.box[:] = list(box)
    c.blocks[:] = list(blocks)
    c.energy_model = energy_model
    c.precision = precision
    c.rng_mode = rng_mode
    c.math_mode = math_mode
    c.creation_mode = creation_mode
    c.log_events = log_events
    c.lattice_const = lattice_const
    c.cutoff = cutoff
    c.attempt_freq = attempt_freq
    c.temperature = temperature
    c.window = window
    c.seed = seed
    c.seed_vacancy = seed_vacancy
    c.seed_time_inc = seed_time_inc
    c.pot_seed = pot_seed
    codes = [a[0] for a in alloy] + [FE] * (4 - len(alloy))
    ratios = [a[1] for a in alloy] + [0] * (4 - len(alloy))
    c.type_codes[:] = codes
    c.ratio[:] = ratios
    c.n_vacancies = n_vacancies
    if pile is not None:
        arr = np.ascontiguousarray(np.asarray(pile, np.int64).reshape(-1, 3))
        c._pile = arr  # keeps the positions alive with the config
        c.pile_xyz = arr.ctypes.data
        c.pile_n = len(arr)
    return c


class Oracle:
    """One oracle job (a periodic box split into domain blocks)."""

    def __init__(self, cfg):
        L = lib()
        err = C.create_string_buffer(256)
        self._cfg = cfg
        self.h = L.ao_create(C.byref(cfg), err, 256)
        if not self.h:
            raise ValueError(err.value.decode())
        self.nsites = L.ao_nsites(self.h)
        self.nblocks = L.ao_nblocks(self.h)

    def close(self):
        if self.h:
            lib().ao_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def occupancy(self):
        out = np.empty(self.nsites, np.uint8)
        lib().ao_get_occupancy(self.h, _ptr(out))
        return out

    def set_occupancy(self, occ):
        occ = np.ascontiguousarray(occ, np.uint8)
        rc = lib().ao_set_occupancy(self.h, _ptr(occ), occ.size)
        if rc:
            raise ValueError("ao_set_occupancy failed %d" % rc)

    def rho(self):
        out = np.empty(self.nsites, np.int32)
        if lib().ao_get_rho(self.h, _ptr(out)):
            raise ValueError("no density cache in this model")
        return out

    def run_rounds(self, n):
        rc = lib().ao_run_rounds(self.h, n)
        if rc:
            raise RuntimeError("oracle run failed %d" % rc)

    def run_rounds_flow(self, n, order_seed):
        rc = lib().ao_run_rounds_flow(self.h, n, order_seed)
        if rc:
            raise RuntimeError("oracle run failed %d" % rc)

    def run(self, hop_budget, max_rounds):
        rc = lib().ao_run(self.h, hop_budget, max_rounds)
        if rc:
            raise RuntimeError("oracle run failed %d" % rc)

    @property
    def round(self):
        return lib().ao_round(self.h)

    @property
    def hops(self):
        return lib().ao_total_hops(self.h)

    def events(self):
        n = lib().ao_num_events(self.h)
        out = np.empty(n, EVENT_DTYPE)
        if n:
            lib().ao_get_events(self.h, _ptr(out), 0, n)
        return out

    def block_state(self):
        evo = np.empty((self.nblocks, 8), np.float64)
        hops = np.empty(self.nblocks, np.int64)
        lib().ao_get_block_state(self.h, _ptr(evo), _ptr(hops))
        return evo, hops

    def stats(self):
        out = np.empty(4, np.int64)
        lib().ao_stats(self.h, _ptr(out))
        return dict(hops=int(out[0]), n_act_sum=int(out[1]), dirty_sum=int(out[2]), start_evals=int(out[3]))

    def vacancy_rates(self, site):
        r = np.empty(8, np.float64)
        d = np.empty(8, np.float64)
        avail = lib().ao_vacancy_rates(self.h, site, _ptr(r), _ptr(d))
        if avail < 0:
            raise ValueError("site %d is not a vacancy" % site)
        return avail, r, d

    def bond_count(self, site, code):
        return lib().ao_bond_count(self.h, site, code)

    def eam_tables(self):
        params = np.empty((4, 5), np.float64)
        f_sh = np.empty((4, 5), np.float64)
        phi = np.empty((4, 4, 5), np.float64)
        fq = np.empty((4, 7), np.int32)
        coef = np.empty((5000, 4), np.float64)
        if lib().ao_eam_export(self.h, _ptr(params), _ptr(f_sh), _ptr(phi), _ptr(fq), _ptr(coef)):
            raise ValueError("not an EAM job")
        return dict(params=params, f_sh=f_sh, phi_sh=phi, fq=fq, coef=coef)

    def neighbours(self, site):
        nn1 = np.empty(8, np.int64)
        nn2 = np.empty(6, np.int64)
        lib().ao_neighbours(self.h, site, _ptr(nn1), _ptr(nn2))
        return nn1, nn2

    def cluster_stats(self, hist_len=64):
        iso = C.c_int64(0)
        hist = np.zeros(hist_len, np.int64)
        lib().ao_cluster_stats(self.h, C.byref(iso), _ptr(hist), hist_len)
        return int(iso.value), hist


def port_exp(x):
    return lib().ao_exp(float(x))


def port_log(x):
    return lib().ao_log(float(x))


def xoshiro_stream(seed, tag, index, n):
    out = np.empty(n, np.uint64)
    lib().ao_xoshiro_stream(seed, tag, index, _ptr(out), n)
    return out


def mt19937_draws(seed, n, default_seed=False, canonical=False):
    out = np.empty(n, np.float64)
    lib().ao_mt19937_draws(seed, int(default_seed), int(canonical), _ptr(out), n)
    return out
