"""Multi-process logic of bench.py on the CPU: world_size-2 gloo ranks run
independent replicas (the path does not shard) and agree on the max-over-ranks
time; a rank that fails before the reduction makes the others fail on the
process-group timeout instead of hanging."""
import os
import socket
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


SCRIPT = textwrap.dedent("""
    import os, sys, json
    sys.path.insert(0, {root!r})
    import bench
    d = bench.Dist()
    assert d.world == 2 and d.pg
    d.barrier()
    if os.environ.get("FAIL_RANK") == str(d.rank):
        raise SystemExit(3)
    t = d.max(1.0 + d.rank)
    print(json.dumps({{"rank": d.rank, "max": t}}), flush=True)
    d.close()
""")


def _launch(tmp_path, extra_env=None, timeout=120):
    script = tmp_path / "rank.py"
    script.write_text(SCRIPT.format(root=ROOT))
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="", **(extra_env or {}))
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            out, err = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            p.kill()
            out, err = p.communicate()
        outs.append((p.returncode, out, err))
    return outs


def test_two_gloo_ranks_agree_on_max_time(tmp_path):
    outs = _launch(tmp_path)
    for rc, out, err in outs:
        assert rc == 0, err[-2000:]
        assert '"max": 2.0' in out


@pytest.mark.timeout(400)
def test_failed_rank_does_not_hang_the_other(tmp_path, monkeypatch):
    # rank 1 exits before the reduction; rank 0 must end with an error, not hang
    outs = _launch(tmp_path, {"FAIL_RANK": "1", "ZSPH_PG_TIMEOUT": "20"}, timeout=300)
    assert outs[1][0] == 3
    assert outs[0][0] != 0


def test_a_failing_secondary_leg_is_reported_not_fatal(capsys):
    sys.path.insert(0, ROOT)
    import bench

    def boom():
        raise RuntimeError("leg exploded")

    assert bench.guarded_leg("learned", lambda: {"value": 1.0}) == {"value": 1.0}
    r = bench.guarded_leg("learned", boom)
    assert r == {"error": "RuntimeError: leg exploded"}
    assert "the learned leg failed" in capsys.readouterr().err
