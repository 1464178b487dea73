"""ctypes front-end of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs use
this module.  It loads ``oracle/_build/libcsg_oracle.so`` (built by
``oracle/Makefile``) and exposes the oracle's entry points on numpy arrays in
the engine's canonical layout:

* spins  ``uint32[W, C, T//4, N, 4]`` (site axis = checkerboard slot)
* bonds  ``uint32[W, 3, N]``          (bit 1 = antiferromagnetic bond)
"""
from __future__ import annotations

import ctypes as C
import pathlib
import subprocess

import numpy as np

_HERE = pathlib.Path(__file__).resolve().parent
_LIB_PATH = _HERE / "_build" / "libcsg_oracle.so"
_lib = None


def build() -> pathlib.Path:
    """Compile the oracle library (idempotent)."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


class Params(C.Structure):
    _fields_ = [
        ("L", C.c_int32), ("W", C.c_int32), ("C", C.c_int32), ("T", C.c_int32),
        ("sweeps_per_swap", C.c_int32), ("sweeps_per_meas", C.c_int32),
        ("meas_start", C.c_int64),
        ("H", C.c_double),
        ("seed", C.c_uint64),
        ("betas", C.c_void_p),
        ("thr", C.c_void_p),
        ("n_threads", C.c_int32),
        ("word0", C.c_int32),
    ]


class Obs(C.Structure):
    _fields_ = [
        ("e_sum", C.c_void_p), ("m_sum", C.c_void_p),
        ("q_sum", C.c_void_p), ("q2_sum", C.c_void_p), ("q4_sum", C.c_void_p),
        ("hist", C.c_void_p),
        ("e_last", C.c_void_p), ("m_last", C.c_void_p), ("d_last", C.c_void_p),
        ("swap_acc", C.c_void_p),
        ("swap_log", C.c_void_p), ("swap_log_rounds", C.c_int64),
        ("swap_rounds", C.c_int64), ("n_meas", C.c_int64),
        ("boundary", C.c_uint64),
    ]


def lib():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        L = C.CDLL(str(_LIB_PATH))
        vp = C.c_void_p
        L.orc_philox4x32_10.argtypes = [vp, vp, vp]
        L.orc_philox4x32_10.restype = None
        L.orc_thresholds.argtypes = [C.c_int32, vp, C.c_double, vp]
        L.orc_init.argtypes = [C.c_int32] * 4 + [C.c_uint64, C.c_int32, vp, vp]
        L.orc_run.argtypes = [C.POINTER(Params), vp, vp, C.c_int64, C.c_int64, C.POINTER(Obs)]
        L.orc_run_multispin.argtypes = L.orc_run.argtypes
        L.orc_energies.argtypes = [C.c_int32] * 4 + [vp, vp, vp, vp]
        L.orc_overlaps.argtypes = [C.c_int32] * 3 + [vp, vp, vp]
        L.orc_obs_records.argtypes = [C.c_int32] * 3 + [C.c_float, vp, vp, vp]
        L.orc_to_ref_lattice.argtypes = [C.c_int32] * 3 + [vp, vp, vp]
        L.orc_from_ref_lattice.argtypes = [C.c_int32] * 3 + [vp, vp, vp]
        for f in ("orc_thresholds", "orc_init", "orc_run", "orc_run_multispin", "orc_energies",
                  "orc_overlaps",
                  "orc_obs_records", "orc_to_ref_lattice", "orc_from_ref_lattice"):
            getattr(L, f).restype = C.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"oracle {what} failed with status {rc}")


def philox(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, np.uint32)
    lib().orc_philox4x32_10(_p(c), _p(k), _p(out))
    return out


def thresholds(betas, H: float) -> np.ndarray:
    b = np.ascontiguousarray(betas, dtype=np.float64)
    thr = np.zeros((b.size, 2, 7), np.uint64)
    _check(lib().orc_thresholds(b.size, _p(b), float(H), _p(thr)), "thresholds")
    return thr


def init(L: int, W: int, C_: int, T: int, seed: int, word0: int = 0):
    N = L ** 3
    spins = np.zeros((W, C_, T // 4, N, 4), np.uint32)
    bonds = np.zeros((W, 3, N), np.uint32)
    _check(lib().orc_init(L, W, C_, T, seed, word0, _p(spins), _p(bonds)), "init")
    return spins, bonds


class Observables:
    """Accumulators of the measurement schedule (same meaning as the engine's)."""

    def __init__(self, L: int, W: int, C_: int, T: int, log_rounds: int = 0):
        N = L ** 3
        self.e_sum = np.zeros((W, C_, T, 32), np.int64)
        self.m_sum = np.zeros((W, C_, T, 32), np.int64)
        self.q_sum = np.zeros((W, T, 32), np.int64)
        self.q2_sum = np.zeros((W, T, 32), np.int64)
        self.q4_sum = np.zeros((W, T, 32, 2), np.uint64)
        self.hist = np.zeros((T, N + 1), np.uint32)
        self.e_last = np.zeros((W, C_, T, 32), np.int32)
        self.m_last = np.zeros((W, C_, T, 32), np.int32)
        self.d_last = np.zeros((W, T, 32), np.int32)
        self.swap_acc = np.zeros((C_, T), np.uint64)
        self.swap_log = np.zeros((max(log_rounds, 1), W, C_, T), np.uint32)
        self.c = Obs()
        for f in ("e_sum", "m_sum", "q_sum", "q2_sum", "q4_sum", "hist", "e_last", "m_last",
                  "d_last", "swap_acc", "swap_log"):
            setattr(self.c, f, _p(getattr(self, f)))
        self.c.swap_log_rounds = log_rounds
        if log_rounds == 0:
            self.c.swap_log = None

    @property
    def n_meas(self) -> int:
        return int(self.c.n_meas)

    @property
    def swap_rounds(self) -> int:
        return int(self.c.swap_rounds)

    @property
    def boundary(self) -> int:
        return int(self.c.boundary)

    def q4(self) -> np.ndarray:
        """Sum of Q^4 as Python ints (object array)."""
        lo = self.q4_sum[..., 0].astype(object)
        hi = self.q4_sum[..., 1].astype(object)
        return lo + hi * (1 << 64)


def run(spins: np.ndarray, bonds: np.ndarray, *, L: int, betas, H: float, seed: int,
        sweep0: int, n_sweeps: int, sweeps_per_swap: int = 1, sweeps_per_meas: int = 0,
        meas_start: int = 0, obs: Observables | None = None, n_threads: int = 0,
        word0: int = 0, multispin: bool = False) -> Observables:
    """n_sweeps sweeps from global sweep sweep0.  multispin: the Metropolis
    step for all 32 samples of a word at once (orc_run_multispin, the timing
    baseline); the default is the one-sample-at-a-time restatement."""
    W, C_, Q = spins.shape[:3]
    T = 4 * Q
    b = np.ascontiguousarray(betas, dtype=np.float64)
    thr = thresholds(b, H)
    if obs is None:
        obs = Observables(L, W, C_, T)
    p = Params(L=L, W=W, C=C_, T=T, sweeps_per_swap=sweeps_per_swap,
               sweeps_per_meas=sweeps_per_meas, meas_start=meas_start, H=float(H),
               seed=seed, betas=_p(b).value, thr=_p(thr).value, n_threads=n_threads,
               word0=word0)
    fn = lib().orc_run_multispin if multispin else lib().orc_run
    _check(fn(C.byref(p), _p(spins), _p(bonds), sweep0, n_sweeps, C.byref(obs.c)), "run")
    return obs


def energies(spins: np.ndarray, bonds: np.ndarray, L: int):
    W, C_, Q = spins.shape[:3]
    e = np.zeros((W, C_, 4 * Q, 32), np.int32)
    m = np.zeros_like(e)
    _check(lib().orc_energies(L, W, C_, 4 * Q, _p(spins), _p(bonds), _p(e), _p(m)), "energies")
    return e, m


def overlaps(spins: np.ndarray, L: int, planes: bool = False):
    W, C_, Q = spins.shape[:3]
    T = 4 * Q
    d = np.zeros((W, T, 32), np.int32)
    dpl = np.zeros((W, T, 32, 3, L), np.int32) if planes else None
    _check(lib().orc_overlaps(L, W, T, _p(spins), _p(d), _p(dpl) if planes else None),
           "overlaps")
    return (d, dpl) if planes else d


def obs_records(spins: np.ndarray, bonds: np.ndarray, L: int, H: float) -> np.ndarray:
    W, C_, Q = spins.shape[:3]
    T = 4 * Q
    rec = np.zeros((32 * W, T, 11), np.float32)
    _check(lib().orc_obs_records(L, W, T, float(H), _p(spins), _p(bonds), _p(rec)), "obs")
    return rec


def to_ref_lattice(spins: np.ndarray, bonds: np.ndarray, L: int) -> np.ndarray:
    W, C_, Q = spins.shape[:3]
    ref = np.zeros((64 * W, L ** 3), np.uint32)
    _check(lib().orc_to_ref_lattice(L, W, 4 * Q, _p(spins), _p(bonds), _p(ref)), "to_ref")
    return ref


def from_ref_lattice(ref: np.ndarray, L: int, T: int):
    W = ref.shape[0] // 64
    N = L ** 3
    spins = np.zeros((W, 2, T // 4, N, 4), np.uint32)
    bonds = np.zeros((W, 3, N), np.uint32)
    ref = np.ascontiguousarray(ref, dtype=np.uint32)
    _check(lib().orc_from_ref_lattice(L, W, T, _p(ref), _p(spins), _p(bonds)), "from_ref")
    return spins, bonds


def geometric_betas(T: int, t_min: float, t_max: float) -> np.ndarray:
    """Temperatures geometric in [t_min, t_max]; plane 0 is the coldest."""
    temps = t_min * (t_max / t_min) ** (np.arange(T) / (T - 1))
    return 1.0 / temps


def reference_betas(T: int = 24) -> np.ndarray:
    """The reference ladder beta_r = 2 (2^(-4/(T-1)))^r stored as float32
    (eamsim.cu:728-737)."""
    ratio = 2.0 ** (-4.0 / (T - 1.0))
    return np.array([np.float32(ratio ** r * 2.0) for r in range(T)], dtype=np.float64)
