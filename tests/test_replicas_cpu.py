"""The multi-rank path of bench.py on the CPU: two ranks over gloo
(127.0.0.1) run lightspeed_b200.replicas exactly as the benchmark does --
join the group, barrier, take each timing's maximum over the ranks in one
all-reduce, compute the whole-job rate, leave -- and the reference arm's
non-zero ranks exit without work. A rank that never joins turns into an
error on the other within the group timeout (failure made on the host)."""
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out, timeout_s, skip_rank):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    try:
        if rank == skip_rank:
            out.put((rank, "skipped"))
            return
        from lightspeed_b200 import replicas
        replicas.init("gloo", timeout_s=timeout_s)
        replicas.barrier()
        # rank r "took" (r + 1) ms, (10 - r) ms and 5 ms for three phases
        m = replicas.max_over_ranks([rank + 1.0, 10.0 - rank, 5.0])
        replicas.barrier()
        rate = replicas.whole_job_rate(100.0, world, m[0] * 1e-3)
        replicas.finish()
        out.put((rank, {"max": m, "rate": rate}))
    except Exception as e:   # reported to the parent
        out.put((rank, "error: %s" % type(e).__name__))


def _run(world, timeout_s=60, skip_rank=-1):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, world, port, q, timeout_s, skip_rank)) for r in range(world)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=180) for _ in range(world))
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return res


def test_two_ranks_max_over_ranks_and_rate():
    res = _run(2)
    for r in (0, 1):
        assert res[r]["max"] == [2.0, 10.0, 5.0]
        assert abs(res[r]["rate"] - 2 * 100.0 / 2e-3) < 1e-6


def test_single_rank_needs_no_group():
    from lightspeed_b200 import replicas
    assert replicas.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
    assert replicas.whole_job_rate(10.0, 1, 2.0) == 5.0
    replicas.barrier()   # no group: nothing to wait for
    replicas.finish()


def test_missing_rank_fails_on_the_host():
    """Rank 1 never joins: rank 0's join (or first collective) ends with an
    error inside the short timeout instead of waiting for good."""
    res = _run(2, timeout_s=5, skip_rank=1)
    assert res[1] == "skipped"
    assert isinstance(res[0], str) and res[0].startswith("error")


def test_reference_arm_nonzero_rank_exits_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
