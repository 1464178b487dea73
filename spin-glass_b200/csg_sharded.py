"""The `csg <sim_dir> <H>` command over several GPUs, one rank per GPU.

    torchrun --nproc-per-node G --master-addr 127.0.0.1 spin-glass_b200/csg_sharded.py <sim_dir> <H>

It takes the same arguments, files, csg.conf keys, resume sidecar, log file and
exit codes as the single-GPU command (spin-glass_b200/csrc/csg_main.cpp, itself
the reference program's Program/src/main.cu:8-84).
The NDIS/32 sample words are split into contiguous ranges, one per rank
(distributed.shard).  Each rank's engine carries its range's first word as
word0, so every file is bit-identical to the single-GPU command's with the same
seed.  After every section the ranks' obs_s records go to rank 0 in sample
order, and rank 0 appends them to <H>-obs.bin.  At the end the checkpoint rows
are gathered the same way.  Only rank 0 writes files or logs.

A failure on any rank (configuration, device, file) ends every rank with exit
code 1 at the next agreement point, and rank 0 logs that rank's message; no
rank is left waiting in a collective.
"""
from __future__ import annotations

import importlib
import importlib.util
import os
import pathlib
import re
import socket
import sys
import time

import numpy as np

PKG_DIR = pathlib.Path(__file__).resolve().parent
RESUME_MAGIC = "csg-resume-v1"


def _package():
    """The engine package (this directory) imported as spin_glass_b200."""
    if "spin_glass_b200" in sys.modules:
        return sys.modules["spin_glass_b200"]
    spec = importlib.util.spec_from_file_location(
        "spin_glass_b200", PKG_DIR / "__init__.py", submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["spin_glass_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


class Failure(RuntimeError):
    pass


# ------------------------------------------------------------ the C library's parsing
_INT = re.compile(r"\s*([+-]?\d+)")
_INT_AUTO = re.compile(r"\s*([+-]?)(0[xX][0-9a-fA-F]+|0[0-7]*|[1-9]\d*)")
_FLOAT = re.compile(r"\s*([+-]?(\d+\.?\d*([eE][+-]?\d+)?|\.\d+([eE][+-]?\d+)?|inf(inity)?|nan))",
                    re.IGNORECASE)


def _stoi(v: str) -> int:
    """std::stoi / std::stoll: the leading decimal integer, else an error."""
    m = _INT.match(v)
    if not m:
        raise Failure("stoi")
    return int(m.group(1))


def _stoull_auto(v: str) -> int:
    """std::stoull(v, nullptr, 0): 0x… hexadecimal, 0… octal, else decimal."""
    m = _INT_AUTO.match(v)
    if not m:
        raise Failure("stoull")
    digits = m.group(2)
    x = int(digits, 16) if digits[:2].lower() == "0x" else int(digits, 8 if digits[0] == "0" else 10)
    return ((-x) % (1 << 64)) if m.group(1) == "-" else x


def _stod(v: str) -> float:
    m = _FLOAT.match(v)
    if not m:
        raise Failure("stod")
    return float(m.group(1))


def read_settings(sim_dir: str) -> dict:
    """Defaults are the reference's compile-time constants (eamsim.cuh:13-22);
    <sim_dir>/csg.conf (key = value lines, # comments) changes them.  Same keys
    and checks as the single-GPU command."""
    st = dict(L=16, NDIS=2048, NREP=24, SBSHFL=16, SBMEAS=1024, SPFILE=262144, seed=None,
              beta_max=2.0, beta_min=0.125)
    path = pathlib.Path(sim_dir) / "csg.conf"
    if not path.is_file():
        return st
    for line in path.read_text().splitlines():
        line = line.split("#", 1)[0]
        if "=" not in line:
            continue
        k, v = line.split("=", 1)
        k, v = k.strip(" \t"), v.strip(" \t\r")
        if k in ("L", "NDIS", "NREP", "SBSHFL", "SBMEAS", "SPFILE"):
            st[k] = _stoi(v)
        elif k == "seed":
            st[k] = _stoull_auto(v)
        elif k in ("beta_max", "beta_min"):
            st[k] = _stod(v)
        else:
            raise Failure("unknown key in csg.conf: " + k)
    if st["NDIS"] % 32 or st["NDIS"] <= 0:
        raise Failure("NDIS must be a positive multiple of 32")
    if st["SBMEAS"] <= 0 or st["SPFILE"] % st["SBMEAS"]:
        raise Failure("SPFILE must be a multiple of SBMEAS")
    return st


def ladder(nrep: int, beta_max: float, beta_min: float) -> np.ndarray:
    """beta_r = beta_max (beta_min/beta_max)^(r/(NREP-1)), stored as float32 as
    the reference does (eamsim.cu:728-737)."""
    ratio = (beta_min / beta_max) ** (1.0 / (nrep - 1))
    return np.array([np.float32(ratio ** r * beta_max) for r in range(nrep)], np.float64)


def parse_field(arg: str) -> float:
    """std::stof of the command's second argument."""
    return float(np.float32(_stod(arg)))


# ------------------------------------------------------------------- the command
class _Log:
    """Timestamped lines to stdout and <unix time>.log (util.cu:22-47); rank 0 only."""

    def __init__(self, path: pathlib.Path | None):
        self.path, self.f = path, None
        if path is not None:
            try:  # as the single-GPU command: no log file is no error
                self.f = open(path, "a")
            except OSError:
                pass

    def record(self, msg: str) -> None:
        if self.path is None:
            return
        line = time.strftime("[%d/%m/%y %H:%M:%S] ") + msg
        if self.f is not None:
            try:
                self.f.write(line + "\n")
                self.f.flush()
            except OSError:
                pass
        print(line, flush=True)

    def progress(self, pc: float) -> None:
        if self.path is not None:
            print(f"progress: {pc:05.1f}%", end="\r", flush=True)

    def close(self, remove: bool) -> None:
        if self.f is not None:
            try:
                self.f.close()
                if remove:
                    self.path.unlink()
            except OSError:
                pass


def run(sim_dir: str, h_arg: str, *, group=None, engine_factory=None, log_dir: str = ".") -> int:
    """One invocation of the command on every rank of the process group;
    returns the exit code (the same on every rank)."""
    import torch.distributed as dist
    distributed = importlib.import_module(_package().__name__ + ".distributed")
    rank = dist.get_rank(group)
    lead = rank == 0

    def agree(err):
        """Every rank's error message (or None) to every rank; raises on every
        rank when one of them failed, with the first failing rank's message."""
        msgs = [None] * dist.get_world_size(group)
        dist.all_gather_object(msgs, None if err is None else str(err), group=group)
        bad = [(r, m) for r, m in enumerate(msgs) if m is not None]
        if bad:
            r, m = bad[0]
            raise Failure(m if r == rank else f"rank {r}: {m}")

    def step(fn):
        """fn() on every rank, then agreement; its result on success."""
        res, err = None, None
        try:
            res = fn()
        except Exception as e:  # noqa: BLE001 - any local failure ends every rank
            err = e if str(e) else type(e).__name__
        agree(err)
        return res

    try:
        H = parse_field(h_arg)
    except Failure:
        if lead:
            print("invalid H", flush=True)
        return 1
    base = f"{sim_dir}/{H:06.4f}-"
    # one start time for every rank: it names the log and seeds a fresh run
    t_s = [int(time.time())]
    dist.broadcast_object_list(t_s, src=0, group=group)
    t_s = t_s[0]
    log = _Log(pathlib.Path(log_dir) / f"{t_s}.log" if lead else None)
    sh = out = None
    try:
        if not (0.0 <= H <= 4.0):
            raise Failure("H out of range")
        log.record(f"H = {H:06.4f}")
        st = step(lambda: read_settings(sim_dir))
        betas = ladder(st["NREP"], st["beta_max"], st["beta_min"])
        N = st["L"] ** 3

        def resume():
            sweep, seed = 0, st["seed"] if st["seed"] is not None else t_s
            prev = os.path.isfile(base + "chkpt.bin")
            if prev and os.path.isfile(base + "chkpt.csg"):
                f = pathlib.Path(base + "chkpt.csg").read_text().split()
                try:
                    ok = len(f) >= 3 and f[0] == RESUME_MAGIC and int(f[1]) >= 0
                    if ok:
                        sweep, seed = int(f[1]), int(f[2])
                except ValueError:
                    ok = False
                if not ok:
                    raise Failure("bad resume sidecar")
            return prev, sweep, seed

        prev, sweep, seed = step(resume)
        pkg = _package()
        factory = engine_factory if engine_factory is not None else pkg.Engine
        sh = step(lambda: distributed.ShardedEngine(
            st["L"], st["NDIS"] // 32, 2, betas, group=group, engine_factory=factory, H=H,
            seed=seed, sweeps_per_swap=st["SBSHFL"], sweeps_per_meas=st["SBMEAS"],
            flags=pkg.CSG_MEASURE_M))
        log.record("eamsim initialized")
        if not prev:
            step(sh.init_lattice)
            log.record("lattice array initialized")
        else:
            def load():
                nref = 2 * st["NDIS"] * N
                ref = np.fromfile(base + "chkpt.bin", dtype=np.uint32, count=nref)
                if ref.size != nref:
                    raise Failure("checkpoint is truncated")
                sh.load_checkpoint(ref.reshape(2 * st["NDIS"], N), sweep)
            step(load)
            log.record("checkpoint loaded")
        out = step(lambda: open(base + "obs.bin", "ab") if lead else None)
        spfile, sbmeas = st["SPFILE"], st["SBMEAS"]
        t0 = time.perf_counter()

        def write(rec):
            out.write(np.ascontiguousarray(rec, np.float32).tobytes())
            out.flush()

        # run only queues a section on the GPU.  Each step takes a section's
        # records and queues the next section before the collectives, and
        # rank 0 writes the previous section's records while the GPU works.
        step(lambda: sh.run(sbmeas))
        last = None  # records of the previous section (rank 0)
        for done in range(0, spfile, sbmeas):
            log.progress(100.0 * done / spfile)

            def take(last=last, done=done):
                if lead and last is not None:
                    write(last)
                rec = sh.engine.obs_records()
                if done + sbmeas < spfile:
                    sh.run(sbmeas)
                return rec
            last = sh.gather_rows(step(take))
        step(lambda: (write(last), out.close()) if lead else None)
        secs = time.perf_counter() - t0
        t_e = secs * 1e12 / (spfile * N * 2 * st["NDIS"] * st["NREP"])
        log.record(f"t_e = {t_e:07.4f} ps")
        log.record("simulation ended")
        chk = sh.gather_rows(step(sh.engine.save_checkpoint))

        def save():
            if lead:
                np.ascontiguousarray(chk, np.uint32).tofile(base + "chkpt.bin")
                with open(base + "chkpt.csg", "w") as f:
                    f.write(f"{RESUME_MAGIC} {sweep + spfile} {seed}\n")
        step(save)
        log.record("checkpoint saved")
    except Exception as e:  # noqa: BLE001 - the command reports and exits 1
        log.record(str(e) if str(e) else type(e).__name__)
        log.close(remove=False)
        if out is not None and not out.closed:
            out.close()
        _close(sh)
        return 1
    log.close(remove=True)
    _close(sh)
    return 0


def _close(sh) -> None:
    close = getattr(getattr(sh, "engine", None), "close", None)
    if close is not None:
        close()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) < 2:
        print("missing arguments")
        return 1
    if len(argv) > 2:
        print("extra arguments")
        return 1
    import datetime

    import torch
    import torch.distributed as dist
    if "WORLD_SIZE" not in os.environ:  # started without torchrun: one rank
        os.environ.update(RANK="0", WORLD_SIZE="1", MASTER_ADDR="127.0.0.1",
                          MASTER_PORT=str(_free_port()))
    cuda = torch.cuda.is_available()
    if cuda:
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dist.init_process_group("nccl" if cuda else "gloo", timeout=datetime.timedelta(seconds=300))
    try:
        return run(argv[0], argv[1])
    finally:
        dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
