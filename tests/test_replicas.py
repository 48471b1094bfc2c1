"""Multi-GPU replica plumbing (kwave/replicas.py) on CPU: two gloo ranks on 127.0.0.1.

`bench.py --gpus N` runs one independent replica per GPU under torchrun; the only cross-rank steps
are the barriers around the timed region and the slowest rank's time. These tests run the same
helpers with world size 2 on the gloo backend: the rendezvous, max / sum over ranks, the split of
independent simulations between ranks, a rank that raises before a collective (the other rank's
collective ends with an error within the process-group timeout instead of hanging), and the
reference arm, where only rank 0 does work.
"""
import os
import socket
import subprocess
import sys
import textwrap

import pytest

from kwave.replicas import own_range

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "k-wave-swift_b200")


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_ranks(body: str, world: int = 2, timeout: int = 120) -> list[subprocess.CompletedProcess]:
    port = _free_port()
    script = textwrap.dedent(body)
    procs = []
    for rank in range(world):
        env = dict(os.environ, WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), PYTHONPATH=PKG)
        procs.append(subprocess.Popen([sys.executable, "-c", script], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    out = []
    for p in procs:
        try:
            so, se = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            p.kill()
            so, se = p.communicate()
        out.append(subprocess.CompletedProcess(p.args, p.returncode, so, se))
    return out


def test_own_range_covers_every_item_once():
    for n in (0, 1, 5, 64, 65):
        for world in (1, 2, 3, 8):
            got = [i for r in range(world) for i in own_range(n, world, r)]
            assert got == list(range(n))
            sizes = [len(own_range(n, world, r)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1


def test_two_gloo_ranks_reduce_and_split():
    res = _run_ranks("""
        from kwave import replicas
        rep = replicas.init("gloo", timeout_s=60)
        assert rep.world == 2
        rep.barrier()
        ms = 10.0 + 5.0 * rep.rank           # rank 1 is the slowest
        slow = rep.max_over_ranks(ms)
        total = rep.sum_over_ranks(len(rep.my_items(65)))
        print("RESULT", rep.rank, slow, total, rep.my_items(65)[0])
        rep.close()
    """)
    for r in res:
        assert r.returncode == 0, r.stderr
    lines = sorted(l for r in res for l in r.stdout.splitlines() if l.startswith("RESULT"))
    assert lines == ["RESULT 0 15.0 65.0 0", "RESULT 1 15.0 65.0 33"]


def test_a_failing_rank_does_not_hang_the_other():
    # rank 1 raises before the collective; rank 0's all-reduce ends with an error (the peer's
    # connection closes) within the process-group timeout
    res = _run_ranks("""
        import sys
        from kwave import replicas
        rep = replicas.init("gloo", timeout_s=20)
        if rep.rank == 1:
            raise SystemExit(3)
        try:
            rep.max_over_ranks(1.0)
        except Exception as e:
            print("PEER_LOST", type(e).__name__)
            sys.exit(0)
        sys.exit(5)
    """, timeout=90)
    assert res[1].returncode == 3
    assert res[0].returncode == 0, (res[0].returncode, res[0].stderr[-500:])
    assert "PEER_LOST" in res[0].stdout


@pytest.mark.parametrize("workload", ["hetero3d_256", "batch2d_64", "adjoint2d_512"])
def test_reference_arm_runs_on_rank_zero_only(workload):
    # under torchrun only rank 0 times the CPU reference and prints its line; rank 1 exits at once
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(_free_port()))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--workload", workload, "--steps", "1"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-500:]
    assert r.stdout.strip() == ""
