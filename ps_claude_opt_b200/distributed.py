"""Period scan over several GPUs: one process per GPU, disjoint frequencies.

Every (frequency, pole) fit is independent -- the reference's batches of
frequencies (start_CUDA.cu:792-1245) share nothing but the object -- so the
scan shards without a data-path collective.  Each rank takes whole
frequencies (all 10 poles of a frequency on one rank, so the best-pole choice
of start_CUDA.cu:1200-1229 stays local) in contiguous blocks dealt
round-robin -- by default eight blocks per rank, so frequencies whose fits
converge early or late (stop condition < 1 makes iteration counts ragged)
spread over all ranks instead of piling onto one -- fits them through its own
engine, and only the finished lines travel: one gather of (first frequency,
lines) pairs to rank 0.

The convexity-weight search (CUDAPrecalc, start_CUDA.cu:400-789) runs on rank
0 and its conw_r is broadcast, so every rank scans with the same weight.

Every rank takes the same collective steps in the same order on the error
path too: a rank whose engine fails still joins the broadcast and the gather,
carrying its error, and then every rank raises ScanError naming the failed
ranks -- nobody waits for a peer that has given up.
"""
from __future__ import annotations

import traceback

import numpy as np


class ScanError(RuntimeError):
    """A rank of a distributed scan failed; .failures maps rank -> message."""

    def __init__(self, failures):
        self.failures = dict(failures)
        super().__init__("scan failed on rank(s) %s: %s" % (
            sorted(self.failures), "; ".join(f"{r}: {m}" for r, m in sorted(self.failures.items()))))


BLOCKS_PER_RANK = 8


def frequency_blocks(n_start: int, n_last: int, world: int, rank: int, block: int | None = None):
    """Blocks (first frequency, count) of frequencies n_start..n_last that
    `rank` of `world` fits.  Blocks of `block` frequencies go round-robin;
    the default interleaves BLOCKS_PER_RANK blocks per rank (one block when
    there is one rank)."""
    total = max(0, n_last - n_start + 1)
    if total == 0:
        return []
    if block is None:
        block = total if world == 1 else -(-total // (world * BLOCKS_PER_RANK))
    if block < 1:
        raise ValueError("block must be >= 1")
    out = []
    for i, lo in enumerate(range(n_start, n_last + 1, block)):
        if i % world == rank:
            out.append((lo, min(block, n_last - lo + 1)))
    return out


def _default_engine(obj, device):
    from . import native

    return native.Engine(obj, device)


def scan(obj, n_start: int = 1, max_freq: int | None = None, block: int | None = None, quirks: int = 0,
         engine_factory=None, device: int | None = None, group=None):
    """The reference's main flow (convexity-weight search, then the scan)
    spread over the ranks of the default process group (or `group`).

    Returns (lines, conw_r) on rank 0 -- lines in frequency order, as one
    process would write them -- and (None, conw_r) on the other ranks.
    Without an initialised process group it runs as a single rank.

    engine_factory(obj, device) must return an object with set_quirks(q),
    precalc(conw_r) -> (conw_r, new_conw), start(conw_r, n_start_from,
    max_lines) -> lines array and close(); the default is the GPU engine
    (native.Engine) on `device` (default: this rank's local GPU).
    """
    import os

    import torch.distributed as dist

    distributed = dist.is_available() and dist.is_initialized()
    rank = dist.get_rank(group) if distributed else 0
    world = dist.get_world_size(group) if distributed else 1
    if device is None:
        device = int(os.environ.get("LOCAL_RANK", "0"))
    factory = engine_factory or _default_engine
    n_last = obj.grid.n_max if max_freq is None else min(obj.grid.n_max, n_start + max_freq - 1)

    eng, error = None, None
    try:
        eng = factory(obj, device)
        eng.set_quirks(quirks)
    except Exception:  # reported to every rank below
        error = traceback.format_exc(limit=3)

    # convexity-weight search on rank 0 (period_search_BOINC.cpp:646-770)
    conw_r = obj.conw_r
    if rank == 0 and error is None:
        try:
            new_conw = 0
            while new_conw != 1 and conw_r * obj.escl * obj.escl < 10.0:
                conw_r, new_conw = eng.precalc(conw_r)
        except Exception:
            error = traceback.format_exc(limit=3)
    state = [conw_r, error if rank == 0 else None]
    if distributed:
        dist.broadcast_object_list(state, src=0, group=group)
    conw_r = state[0]
    failures = {0: state[1]} if state[1] else {}

    parts = []
    if not failures and error is None:
        try:
            for lo, cnt in frequency_blocks(n_start, n_last, world, rank, block):
                parts.append((lo, np.asarray(eng.start(conw_r, n_start_from=lo, max_lines=cnt))))
        except Exception:
            error = traceback.format_exc(limit=3)
    mine = (rank, error, parts)
    if distributed:
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(mine, gathered, dst=0, group=group)
        # rank 0 tells everybody whether the scan as a whole succeeded
        verdict = [None]
        if rank == 0:
            verdict[0] = {r: e for r, e, _ in gathered if e}
        dist.broadcast_object_list(verdict, src=0, group=group)
        failures.update(verdict[0])
    else:
        gathered = [mine]
        if error:
            failures[rank] = error
    if eng is not None:
        try:
            eng.close()
        except Exception:
            pass
    if failures:
        raise ScanError(failures)
    if rank != 0:
        return None, conw_r
    blocks = sorted(((lo, arr) for _, _, p in gathered for lo, arr in p), key=lambda b: b[0])
    lines = np.concatenate([a for _, a in blocks]) if blocks else np.zeros((0, 6))
    return lines, conw_r
