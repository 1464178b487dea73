"""Sample sharding over GPUs: one process per GPU, no collective on the data path.

Disorder samples never interact, and the replica exchange is per sample, so a
simulation of W sample words splits into contiguous word ranges, one per rank.
Each rank runs its range as an ordinary engine whose ``word0`` is the range's
first global word, which keeps every Philox counter equal to the unsplit
run's: the union of the shards is bit-identical to running all words on one
GPU.  The only communication is gathers to rank 0 over the process group (NCCL
on GPUs, gloo on CPUs): the observable accumulators, the reference-format
records after a section, and the reference-format checkpoint.  csg_sharded.py
builds the reference program's command on these.
"""
from __future__ import annotations

import numpy as np
import torch.distributed as dist


def shard(n_words: int, world: int, rank: int) -> tuple[int, int]:
    """(first global word, number of words) of a rank; sizes differ by <= 1."""
    if not (0 <= rank < world) or n_words < world:
        raise ValueError("need at least one word per rank")
    base, extra = divmod(n_words, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


_PER_WORD = ("e_sum", "m_sum", "q_sum", "q2_sum", "q4_sum", "e_last", "m_last", "d_last")
_SUMMED = ("hist", "swap_acc")


class ShardedEngine:
    """This rank's shard of one simulation.

    engine_factory(L, n_words, n_copies, betas, word0=..., **kw) builds the
    per-rank engine; the default is the CUDA engine on the current device."""

    def __init__(self, L, n_words, n_copies, betas, *, group=None, engine_factory=None, **kw):
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.n_words = n_words
        self.word_first, self.n_local = shard(n_words, self.world, self.rank)
        if engine_factory is None:
            from . import Engine as engine_factory  # noqa: N813
        word0 = kw.pop("word0", 0)
        self.engine = engine_factory(L, self.n_local, n_copies, betas,
                                     word0=word0 + self.word_first, **kw)

    def init_lattice(self) -> None:
        self.engine.init_lattice()

    def run(self, n_sweeps: int) -> None:
        self.engine.run(n_sweeps)

    def gather_observables(self):
        """Observables of the whole simulation on rank 0 (None on other ranks):
        per-word arrays concatenated in word order, histograms and exchange
        counts summed, boundary counts summed."""
        o = self.engine.observables()
        mine = {f: getattr(o, f) for f in _PER_WORD + _SUMMED}
        mine.update(n_meas=o.n_meas, swap_rounds=o.swap_rounds, boundary=o.boundary,
                    first=self.word_first)
        parts = [None] * self.world if self.rank == 0 else None
        dist.gather_object(mine, parts, dst=0, group=self.group)
        if self.rank != 0:
            return None
        parts.sort(key=lambda p: p["first"])
        out = {f: np.concatenate([p[f] for p in parts], axis=0) for f in _PER_WORD
               if parts[0][f].size}
        for f in _SUMMED:
            out[f] = sum(p[f] for p in parts)
        if len({p["n_meas"] for p in parts}) != 1 or len({p["swap_rounds"] for p in parts}) != 1:
            raise RuntimeError("shards disagree on the schedule")
        out.update(n_meas=parts[0]["n_meas"], swap_rounds=parts[0]["swap_rounds"],
                   boundary=sum(p["boundary"] for p in parts))
        return out

    def gather_records(self):
        """The obs_s records of every sample on rank 0 (None on other ranks):
        float32 [32 W][T][11] in sample order, the block the reference program
        appends to <H>-obs.bin after each section (eamsim.cu:704-708)."""
        return self.gather_rows(self.engine.obs_records())

    def gather_checkpoint(self):
        """The reference checkpoint of the whole simulation on rank 0 (None on
        other ranks): uint32 [64 W][N], lattice 2*sample+copy (eamsim.cu:655-676)."""
        return self.gather_rows(self.engine.save_checkpoint())

    def load_checkpoint(self, ref, sweep: int = 0) -> None:
        """Load this rank's rows of a whole-simulation reference checkpoint."""
        ref = np.asarray(ref)
        if ref.ndim != 2 or ref.shape[0] != 64 * self.n_words:
            raise ValueError("checkpoint rows do not match the simulation's samples")
        rows = ref[64 * self.word_first:64 * (self.word_first + self.n_local)]
        self.engine.load_checkpoint(np.ascontiguousarray(rows, np.uint32), sweep)

    def gather_rows(self, mine):
        """This rank's array, whose rows follow its sample words, stacked with
        the other ranks' on rank 0 in word order (None on other ranks)."""
        parts = [None] * self.world if self.rank == 0 else None
        dist.gather_object((self.word_first, mine), parts, dst=0, group=self.group)
        if self.rank != 0:
            return None
        parts.sort(key=lambda p: p[0])
        return np.concatenate([p[1] for p in parts], axis=0)
