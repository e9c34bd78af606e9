"""The multi-GPU scan's host logic on CPU ranks (gloo, world size 2), with
the oracle standing in for each rank's GPU engine: sharded and gathered
lines equal a single process's, whatever the blocking; an engine failure on
one rank raises on every rank; a rank that dies ends its peer's next
collective with an error instead of a hang."""
import os
import socket

import numpy as np
import pytest

from conftest import prepared


class OracleEngine:
    """The engine interface of distributed.scan over the CPU oracle."""

    fail_on_rank = None     # rank whose start() raises
    die_on_rank = None      # rank whose start() kills its process

    def __init__(self, obj, device):
        self.obj = obj
        self.quirks = 0

    def set_quirks(self, q):
        self.quirks = q

    def precalc(self, conw_r):
        import oracle

        g = self.obj.grid
        return oracle.OracleModel(self.obj, conw_r=conw_r).precalc(g.freq_start, g.freq_step, conw_r,
                                                                   quirks=self.quirks, threads=2)

    def start(self, conw_r, n_start_from=1, max_lines=None):
        import oracle
        import torch.distributed as dist

        rank = dist.get_rank() if dist.is_initialized() else 0
        if rank == self.fail_on_rank:
            raise RuntimeError("injected engine failure")
        if rank == self.die_on_rank:
            os._exit(3)
        g = self.obj.grid
        lines = oracle.OracleModel(self.obj, conw_r=conw_r).scan(g.freq_start, g.freq_end, g.freq_step,
                                                                 n_start=n_start_from, max_lines=max_lines,
                                                                 threads=2)
        if n_start_from == 1 and len(lines):
            lines[0, 3] = conw_r * self.obj.escl ** 2    # the scan's first line (start_CUDA.cu:1218-1222)
        return lines

    def close(self):
        pass


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir, block, fail_on, die_on, timeout_s):
    import datetime

    import torch.distributed as dist

    from ps_claude_opt_b200 import distributed

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=timeout_s))
    OracleEngine.fail_on_rank = fail_on
    OracleEngine.die_on_rank = die_on
    obj = prepared("tiny")
    try:
        lines, conw_r = distributed.scan(obj, block=block, engine_factory=OracleEngine)
        if rank == 0:
            np.save(os.path.join(out_dir, "lines.npy"), lines)
        with open(os.path.join(out_dir, f"ok{rank}"), "w") as f:
            f.write(repr(conw_r))
    except distributed.ScanError as e:
        with open(os.path.join(out_dir, f"scanerror{rank}"), "w") as f:
            f.write(repr(sorted(e.failures)))
    except Exception as e:  # a collective that ended with an error
        with open(os.path.join(out_dir, f"error{rank}"), "w") as f:
            f.write(type(e).__name__)
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _spawn(tmp_path, block=None, fail_on=None, die_on=None, timeout_s=60):
    import torch.multiprocessing as mp

    ctx = mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path), block, fail_on, die_on, timeout_s),
                             nprocs=2, join=False, start_method="spawn")
    for p in ctx.processes:
        p.join(180)
    codes = [p.exitcode for p in ctx.processes]
    for p in ctx.processes:
        if p.is_alive():
            p.kill()
    return codes


def _single_process_lines():
    from ps_claude_opt_b200 import distributed

    return distributed.scan(prepared("tiny"), engine_factory=OracleEngine)


def test_frequency_blocks_cover_each_frequency_once():
    from ps_claude_opt_b200.distributed import frequency_blocks

    for n_start, n_last, world, block in [(1, 5000, 8, None), (1, 5000, 8, 64), (7, 10, 4, None), (3, 3, 2, 1),
                                          (1, 13, 3, 2)]:
        seen = []
        for r in range(world):
            for lo, cnt in frequency_blocks(n_start, n_last, world, r, block):
                assert cnt >= 1
                seen.extend(range(lo, lo + cnt))
        assert sorted(seen) == list(range(n_start, n_last + 1))
    assert frequency_blocks(5, 4, 2, 0) == []
    # default: BLOCKS_PER_RANK interleaved blocks per rank; one block on one rank
    assert frequency_blocks(1, 10, 1, 0) == [(1, 10)]
    assert frequency_blocks(1, 10, 2, 0) == [(1, 1), (3, 1), (5, 1), (7, 1), (9, 1)]
    assert frequency_blocks(1, 5000, 8, 3) == [(lo, 79) for lo in range(1 + 3 * 79, 5001, 8 * 79)][:8]
    assert sum(c for r in range(8) for _, c in frequency_blocks(1, 5000, 8, r)) == 5000


@pytest.mark.parametrize("block", [None, 1, 4])
def test_two_rank_scan_equals_single_process(block, tmp_path):
    ref, conw_ref = _single_process_lines()
    codes = _spawn(tmp_path, block=block)
    assert codes == [0, 0]
    got = np.load(tmp_path / "lines.npy")
    assert np.array_equal(got, ref)
    for r in range(2):
        assert float((tmp_path / f"ok{r}").read_text()) == conw_ref


def test_engine_failure_raises_on_every_rank(tmp_path):
    codes = _spawn(tmp_path, fail_on=1)
    assert codes == [0, 0]
    for r in range(2):
        assert (tmp_path / f"scanerror{r}").read_text() == "[1]"


def test_dead_rank_ends_peer_collective_with_error(tmp_path):
    codes = _spawn(tmp_path, die_on=1, timeout_s=20)
    assert codes[1] == 3
    assert codes[0] == 0                       # rank 0 returned: no hang
    assert (tmp_path / "error0").exists()     # its gather ended with an error
