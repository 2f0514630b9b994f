"""The N>1 bench path is replicas only: every rank renders its own copy and
the timing is the max over ranks, with no collective on the data path.
These world-size-2 gloo runs on the CPU cover bench.py's process-group
setup and its max-over-ranks reduction."""
import os
import socket
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_max_over_ranks_two_gloo_ranks(tmp_path):
    script = tmp_path / "rank.py"
    script.write_text(textwrap.dedent("""
        import os, sys, types
        sys.path.insert(0, %r)
        import bench
        args = types.SimpleNamespace(impl="reference")   # gloo backend
        world, rank, local, pg = bench.dist_setup(args)
        assert world == 2 and pg is not None
        # per-rank step times; the bench reports the slowest rank
        ms = 10.0 + 5.0 * rank
        out = bench.max_over_ranks(ms, pg, "cpu")
        assert out == 15.0, out
        pg.barrier()
        pg.destroy_process_group()
        print("rank", rank, "ok", out)
    """ % ROOT))
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        try:
            out, _ = p.communicate(timeout=180)
        except subprocess.TimeoutExpired:
            p.kill()
            out, _ = p.communicate()
        outs.append(out)
        assert p.returncode == 0, out
    assert all("ok 15.0" in o for o in outs), outs


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    import types
    env_keys = ("WORLD_SIZE", "RANK", "LOCAL_RANK")
    saved = {k: os.environ.pop(k, None) for k in env_keys}
    try:
        world, rank, local, pg = bench.dist_setup(types.SimpleNamespace(impl="ours"))
        assert (world, rank, local, pg) == (1, 0, 0, None)
        assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    finally:
        for k, v in saved.items():
            if v is not None:
                os.environ[k] = v


def test_reference_arm_names_every_workload():
    """Every workload has a reference arm; the adjoint one reports that the
    reference has no differentiable render."""
    sys.path.insert(0, ROOT)
    import bench
    import types
    out = bench.run_adjoint_reference(types.SimpleNamespace(steps=1, warmup=3))
    assert out["impl"] == "reference" and "unavailable" in out
    for name in ("run_render_reference", "run_trace_reference", "run_batch_reference", "run_adjoint_reference"):
        assert callable(getattr(bench, name))
    s = bench._batch_sample(8, [14, 26])
    assert "8 threads" in s and "14, 26" in s
