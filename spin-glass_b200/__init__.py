"""Python mirror of libcsg.so, the B200 parallel-tempering engine.

The product is the C ABI in ``include/csg.h`` (and the ``csg`` command built
on it).  This module binds that ABI with ctypes so that tests and the
benchmark drive exactly the entry points a C/C++ caller would.  It never
computes anything itself: if ``libcsg.so`` is missing or fails to load, every
call raises.

Arrays use the canonical layout of ``include/csg.h``:

* spins ``uint32[W, C, T//4, N, 4]`` — checkerboard site slots,
* bonds ``uint32[W, 3, N]``.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib

import numpy as np

PKG_DIR = pathlib.Path(__file__).resolve().parent
# the library built beside this file, or another build named by $CSG_LIBRARY
LIB_PATH = pathlib.Path(os.environ.get("CSG_LIBRARY") or PKG_DIR / "libcsg.so")

CSG_MEASURE_M = 1
CSG_ENGINE_STREAM = 2
CSG_STREAM_FUSED = 4
_lib = None


class Dims(C.Structure):
    _fields_ = [("L", C.c_int32), ("n_words", C.c_int32), ("n_copies", C.c_int32),
                ("n_temps", C.c_int32)]


class Schedule(C.Structure):
    _fields_ = [("sweeps_per_swap", C.c_int32), ("sweeps_per_meas", C.c_int32),
                ("meas_start", C.c_int64)]


class Config(C.Structure):
    _fields_ = [("dims", Dims), ("sched", Schedule), ("H", C.c_double), ("seed", C.c_uint64),
                ("betas", C.c_void_p), ("flags", C.c_int32), ("swap_log_rounds", C.c_int32),
                ("word0", C.c_int32)]


class ObservablesC(C.Structure):
    _fields_ = [("e_sum", C.c_void_p), ("m_sum", C.c_void_p), ("q_sum", C.c_void_p),
                ("q2_sum", C.c_void_p), ("q4_sum", C.c_void_p), ("hist", C.c_void_p),
                ("e_last", C.c_void_p), ("m_last", C.c_void_p), ("d_last", C.c_void_p),
                ("swap_acc", C.c_void_p), ("swap_log", C.c_void_p),
                ("swap_log_rounds", C.c_int64), ("swap_rounds", C.c_int64),
                ("n_meas", C.c_int64), ("boundary", C.c_uint64)]


class DeviceObs(C.Structure):
    _fields_ = [("e_sum", C.c_void_p), ("m_sum", C.c_void_p), ("q_sum", C.c_void_p),
                ("q2_sum", C.c_void_p), ("q4_sum", C.c_void_p), ("hist", C.c_void_p),
                ("e_last", C.c_void_p), ("m_last", C.c_void_p), ("d_last", C.c_void_p),
                ("swap_acc", C.c_void_p), ("swap_log", C.c_void_p),
                ("swap_log_rounds", C.c_int64), ("swap_round0", C.c_int64),
                ("boundary", C.c_void_p)]


class Plan(C.Structure):
    _fields_ = [("quads_per_cta", C.c_int32), ("ctas_per_word", C.c_int32),
                ("threads_per_quad", C.c_int32), ("smem_bytes", C.c_int32)]


class CsgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"csg error {code}: {msg}")
        self.code = code


def lib():
    """Load libcsg.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run spin-glass_b200/build.py")
        L = C.CDLL(str(LIB_PATH))
        vp, i64, sz = C.c_void_p, C.c_int64, C.c_size_t
        pcfg = C.POINTER(Config)
        L.csg_last_error.restype = C.c_char_p
        L.csg_last_error.argtypes = []
        sig = {
            "csg_engine_create": [pcfg, C.POINTER(vp)],
            "csg_engine_destroy": [vp],
            "csg_init_lattice": [vp],
            "csg_set_state": [vp, vp, sz, vp, sz, i64],
            "csg_get_state": [vp, vp, sz, vp, sz, C.POINTER(i64)],
            "csg_run": [vp, i64],
            "csg_get_observables": [vp, C.POINTER(ObservablesC)],
            "csg_reset_observables": [vp],
            "csg_obs_records": [vp, vp, sz],
            "csg_save_checkpoint": [vp, vp, sz],
            "csg_load_checkpoint": [vp, vp, sz, i64],
            "csg_pt_run_device": [pcfg, vp, vp, C.POINTER(DeviceObs), i64, i64, vp],
            "csg_init_device": [pcfg, vp, vp, vp],
            "csg_query_plan": [pcfg, C.POINTER(Plan)],
            "csg_set_plan_override": [C.POINTER(Plan)],
            "csg_batch_create": [C.POINTER(Config), C.c_int32, C.POINTER(vp)],
            "csg_batch_destroy": [vp],
            "csg_batch_engine": [vp, C.c_int32, C.POINTER(vp)],
            "csg_batch_run": [vp, i64],
            "csg_batch_run_sequential": [vp, i64],
            "csg_batch_tune": [vp, i64, vp],
            "csg_batch_set_plan": [vp, vp],
            "csg_batch_member_plan": [vp, C.c_int32, C.POINTER(Plan)],
            "csg_batch_launch": [vp, i64, C.c_int32, vp],
            "csg_batch_set_member_plan": [vp, C.c_int32, C.POINTER(Plan)],
            "csg_engine_footprint": [C.POINTER(Config), C.POINTER(sz)],
            "csg_server_create": [sz, C.c_int32, C.c_int32, C.POINTER(vp)],
            "csg_server_destroy": [vp],
            "csg_server_submit": [vp, C.POINTER(Config), i64, C.POINTER(i64)],
            "csg_server_poll": [vp, vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                C.POINTER(C.c_int32)],
            "csg_server_result": [vp, i64, C.POINTER(ObservablesC), vp, sz],
            "csg_analyze_records": [vp, i64, C.c_int32, C.c_int32, C.c_int32, vp, vp],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise CsgError(rc, lib().csg_last_error().decode())


def _p(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data_as(C.c_void_p)
    return C.c_void_p(a)  # raw device pointer


def make_config(L: int, n_words: int, n_copies: int, betas, *, H: float = 0.0, seed: int = 1,
                sweeps_per_swap: int = 1, sweeps_per_meas: int = 0, meas_start: int = 0,
                flags: int = 0, swap_log_rounds: int = 0, word0: int = 0):
    """Build a csg_config; returns (config, betas array that must stay alive)."""
    b = np.ascontiguousarray(betas, dtype=np.float64)
    cfg = Config(dims=Dims(L, n_words, n_copies, b.size),
                 sched=Schedule(sweeps_per_swap, sweeps_per_meas, meas_start),
                 H=float(H), seed=seed, betas=b.ctypes.data, flags=flags,
                 swap_log_rounds=swap_log_rounds, word0=word0)
    return cfg, b


class Observables:
    """Host copies of the engine's accumulators (shapes as in include/csg.h)."""

    def __init__(self, L: int, W: int, C_: int, T: int, log_rounds: int = 0, alloc=np.zeros):
        """alloc(shape, dtype) makes each array (e.g. in page-locked memory, for
        faster device-to-host copies when the same object is refilled)."""
        N = L ** 3
        two = C_ == 2
        self.e_sum = alloc((W, C_, T, 32), np.int64)
        self.m_sum = alloc((W, C_, T, 32), np.int64)
        self.q_sum = alloc((W, T, 32) if two else (0,), np.int64)
        self.q2_sum = alloc((W, T, 32) if two else (0,), np.int64)
        self.q4_sum = alloc((W, T, 32, 2) if two else (0,), np.uint64)
        self.hist = alloc((T, N + 1) if two else (0,), np.uint32)
        self.e_last = alloc((W, C_, T, 32), np.int32)
        self.m_last = alloc((W, C_, T, 32), np.int32)
        self.d_last = alloc((W, T, 32) if two else (0,), np.int32)
        self.swap_acc = alloc((C_, T), np.uint64)
        self.swap_log = alloc((max(log_rounds, 1), W, C_, T), np.uint32)
        self.c = ObservablesC()
        for f in ("e_sum", "m_sum", "q_sum", "q2_sum", "q4_sum", "hist", "e_last", "m_last",
                  "d_last", "swap_acc", "swap_log"):
            setattr(self.c, f, _p(getattr(self, f)))
        self.c.swap_log_rounds = log_rounds
        if log_rounds == 0:
            self.c.swap_log = None

    n_meas = property(lambda self: int(self.c.n_meas))
    swap_rounds = property(lambda self: int(self.c.swap_rounds))
    boundary = property(lambda self: int(self.c.boundary))

    def q4(self) -> np.ndarray:
        lo = self.q4_sum[..., 0].astype(object)
        hi = self.q4_sum[..., 1].astype(object)
        return lo + hi * (1 << 64)


class Engine:
    """One simulation on the current CUDA device (csg_engine_* entry points)."""

    def __init__(self, L: int, n_words: int, n_copies: int, betas, **kw):
        self.cfg, self._betas = make_config(L, n_words, n_copies, betas, **kw)
        self.L, self.W, self.C, self.T = L, n_words, n_copies, self._betas.size
        self.N = L ** 3
        self._log_rounds = kw.get("swap_log_rounds", 0)
        h = C.c_void_p()
        _check(lib().csg_engine_create(C.byref(self.cfg), C.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().csg_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def spin_shape(self):
        return (self.W, self.C, self.T // 4, self.N, 4)

    @property
    def bond_shape(self):
        return (self.W, 3, self.N)

    def init_lattice(self) -> None:
        _check(lib().csg_init_lattice(self._h))

    def set_state(self, spins: np.ndarray, bonds: np.ndarray, sweep: int = 0) -> None:
        s = np.ascontiguousarray(spins, np.uint32)
        b = np.ascontiguousarray(bonds, np.uint32)
        _check(lib().csg_set_state(self._h, _p(s), s.size, _p(b), b.size, sweep))

    def get_state(self):
        s = np.zeros(self.spin_shape, np.uint32)
        b = np.zeros(self.bond_shape, np.uint32)
        sw = C.c_int64()
        _check(lib().csg_get_state(self._h, _p(s), s.size, _p(b), b.size, C.byref(sw)))
        return s, b, int(sw.value)

    def run(self, n_sweeps: int) -> None:
        _check(lib().csg_run(self._h, n_sweeps))

    def observables(self, out: Observables | None = None) -> Observables:
        """The accumulated observables (into `out`, made by new_observables, when given)."""
        o = out if out is not None else self.new_observables()
        _check(lib().csg_get_observables(self._h, C.byref(o.c)))
        return o

    def new_observables(self, alloc=np.zeros) -> Observables:
        return Observables(self.L, self.W, self.C, self.T, self._log_rounds, alloc=alloc)

    def reset_observables(self) -> None:
        _check(lib().csg_reset_observables(self._h))

    def obs_records(self) -> np.ndarray:
        rec = np.zeros((32 * self.W, self.T, 11), np.float32)
        _check(lib().csg_obs_records(self._h, _p(rec), rec.size))
        return rec

    def save_checkpoint(self) -> np.ndarray:
        ref = np.zeros((64 * self.W, self.N), np.uint32)
        _check(lib().csg_save_checkpoint(self._h, _p(ref), ref.size))
        return ref

    def load_checkpoint(self, ref: np.ndarray, sweep: int = 0) -> None:
        r = np.ascontiguousarray(ref, np.uint32)
        _check(lib().csg_load_checkpoint(self._h, _p(r), r.size, sweep))


def query_plan(L: int, n_words: int, n_copies: int, betas, **kw) -> Plan:
    cfg, _b = make_config(L, n_words, n_copies, betas, **kw)
    p = Plan()
    _check(lib().csg_query_plan(C.byref(cfg), C.byref(p)))
    return p


def set_plan_override(quads_per_cta: int | None, threads_per_quad: int = 0) -> None:
    """Force quads per CTA and/or threads per quad (0: automatic) of later
    resident-kernel launches; None restores the automatic plan."""
    if quads_per_cta is None and not threads_per_quad:
        _check(lib().csg_set_plan_override(None))
    else:
        p = Plan(quads_per_cta or 0, 0, threads_per_quad, 0)
        _check(lib().csg_set_plan_override(C.byref(p)))


def run_device(cfg: Config, spins_ptr: int, bonds_ptr: int, obs: DeviceObs | None,
               sweep0: int, n_sweeps: int, stream: int = 0) -> None:
    """csg_pt_run_device on raw device pointers (e.g. torch tensors' data_ptr())."""
    _check(lib().csg_pt_run_device(C.byref(cfg), C.c_void_p(spins_ptr), C.c_void_p(bonds_ptr),
                                   C.byref(obs) if obs is not None else None, sweep0, n_sweeps,
                                   C.c_void_p(stream) if stream else None))


def init_device(cfg: Config, spins_ptr: int, bonds_ptr: int, stream: int = 0) -> None:
    _check(lib().csg_init_device(C.byref(cfg), C.c_void_p(spins_ptr), C.c_void_p(bonds_ptr),
                                 C.c_void_p(stream) if stream else None))


def geometric_betas(T: int, t_min: float, t_max: float) -> np.ndarray:
    """Inverse temperatures with T geometric in [t_min, t_max]; plane 0 coldest."""
    temps = t_min * (t_max / t_min) ** (np.arange(T) / (T - 1))
    return 1.0 / temps


def reference_betas(T: int = 24) -> np.ndarray:
    """beta_r = 2 (2^(-4/(T-1)))^r stored as float32, as eamsim.cu:728-737."""
    ratio = 2.0 ** (-4.0 / (T - 1.0))
    return np.array([np.float32(ratio ** r * 2.0) for r in range(T)], dtype=np.float64)


class _Member(Engine):
    """A batch member: an Engine view whose handle the batch owns."""

    def __init__(self, handle, cfg, betas, log_rounds):
        self.cfg, self._betas = cfg, betas
        d = cfg.dims
        self.L, self.W, self.C, self.T = d.L, d.n_words, d.n_copies, d.n_temps
        self.N = d.L ** 3
        self._log_rounds = log_rounds
        self._h = handle

    def close(self) -> None:  # the batch destroys its members
        self._h = None


class Batch:
    """Several simulations advanced together (csg_batch_* entry points).

    members: list of dicts with the keyword arguments of Engine
    (L, n_words, n_copies, betas, and optional H, seed, schedule...)."""

    def __init__(self, members):
        made = [make_config(m["L"], m["n_words"], m["n_copies"], m["betas"],
                            **{k: v for k, v in m.items()
                               if k not in ("L", "n_words", "n_copies", "betas")})
                for m in members]
        self._betas = [b for _, b in made]
        arr = (Config * len(made))(*[c for c, _ in made])
        self._cfgs = arr
        h = C.c_void_p()
        _check(lib().csg_batch_create(arr, len(made), C.byref(h)))
        self._h = h
        self.members = []
        for i, m in enumerate(members):
            eh = C.c_void_p()
            _check(lib().csg_batch_engine(self._h, i, C.byref(eh)))
            self.members.append(_Member(eh, arr[i], self._betas[i], m.get("swap_log_rounds", 0)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            for m in self.members:
                m._h = None
            lib().csg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def run(self, n_sweeps: int) -> None:
        _check(lib().csg_batch_run(self._h, n_sweeps))

    def run_sequential(self, n_sweeps: int) -> None:
        _check(lib().csg_batch_run_sequential(self._h, n_sweeps))

    def launch(self, n_sweeps: int, stream: int = 0, plain: bool = False) -> None:
        """Queue n_sweeps sweeps of every member on a CUDA stream (handle as an
        int, e.g. torch.cuda.current_stream().cuda_stream) without waiting."""
        _check(lib().csg_batch_launch(self._h, n_sweeps, 1 if plain else 0, C.c_void_p(stream)))

    def tune(self, probe_sweeps: int = 64):
        out = np.zeros(len(self.members), np.int32)
        _check(lib().csg_batch_tune(self._h, probe_sweeps, _p(out)))
        return out

    def set_plan(self, quads_per_cta) -> None:
        q = np.ascontiguousarray(quads_per_cta, np.int32)
        _check(lib().csg_batch_set_plan(self._h, _p(q)))

    def set_member_plan(self, i: int, quads_per_cta: int, threads_per_quad: int = 0) -> None:
        """Fix member i's tile (0: automatic)."""
        p = Plan(quads_per_cta, 0, threads_per_quad, 0)
        _check(lib().csg_batch_set_member_plan(self._h, i, C.byref(p)))

    def member_plan(self, i: int) -> "Plan":
        """Launch plan member i runs with (the tuned one after tune())."""
        out = Plan()
        _check(lib().csg_batch_member_plan(self._h, i, C.byref(out)))
        return out


def footprint(L: int, n_words: int, n_copies: int, betas, **kw) -> int:
    """Device bytes an engine of this configuration allocates."""
    cfg, _b = make_config(L, n_words, n_copies, betas, **kw)
    out = C.c_size_t()
    _check(lib().csg_engine_footprint(C.byref(cfg), C.byref(out)))
    return int(out.value)


class Server:
    """Continuous-batching request server (csg_server_* entry points)."""

    def __init__(self, memory_budget_bytes: int, max_active: int = 64,
                 sweeps_per_launch: int = 1024):
        h = C.c_void_p()
        _check(lib().csg_server_create(memory_budget_bytes, max_active, sweeps_per_launch,
                                       C.byref(h)))
        self._h = h
        self._req = {}

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().csg_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, n_sweeps: int, L: int, n_words: int, n_copies: int, betas, **kw) -> int:
        cfg, b = make_config(L, n_words, n_copies, betas, **kw)
        rid = C.c_int64()
        _check(lib().csg_server_submit(self._h, C.byref(cfg), n_sweeps, C.byref(rid)))
        self._req[rid.value] = (L, n_words, n_copies, b.size)
        return rid.value

    def poll(self, max_completed: int = 256):
        ids = np.zeros(max_completed, np.int64)
        nc, na, nq = C.c_int32(), C.c_int32(), C.c_int32()
        _check(lib().csg_server_poll(self._h, _p(ids), max_completed, C.byref(nc), C.byref(na),
                                     C.byref(nq)))
        return [int(i) for i in ids[:min(nc.value, max_completed)]], na.value, nq.value

    def result(self, rid: int, with_spins: bool = False):
        if rid not in self._req:  # the library reports the unknown id
            _check(lib().csg_server_result(self._h, rid, None, None, 0))
            return None
        L, W, C_, T = self._req.pop(rid)
        o = Observables(L, W, C_, T)
        spins = np.zeros((W, C_, T // 4, L ** 3, 4), np.uint32) if with_spins else None
        _check(lib().csg_server_result(self._h, rid, C.byref(o.c), _p(spins),
                                       spins.size if with_spins else 0))
        return (o, spins) if with_spins else o
