"""The N > 1 launch of bench.py: one independent replica per rank, started
by torch.distributed.run. The ranks meet only on the host, over gloo: a
barrier around the timed region, the maximum of the step times and the sum of
the particles. Two ranks on 127.0.0.1, CPU only. The reference arm runs on
rank 0 alone; the other ranks exit at once."""
import json
import os
import socket
import subprocess
import sys
import textwrap
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

RANK_CODE = textwrap.dedent(f"""
    import json, sys
    sys.path.insert(0, {str(ROOT)!r})
    import bench
    ws, rank, local = bench.dist_info()
    d = bench.Dist(ws)
    d.barrier()
    out = {{"rank": rank, "ws": ws, "max": d.max(1.5 + rank), "sum": d.sum(10.0 * (rank + 1))}}
    d.barrier()
    d.close()
    print(json.dumps(out))
""")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, ws, port):
    return dict(os.environ, WORLD_SIZE=str(ws), RANK=str(rank), LOCAL_RANK=str(rank),
                MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))


def test_two_ranks_barrier_max_sum():
    port = _free_port()
    procs = [subprocess.Popen([sys.executable, "-c", RANK_CODE], env=_env(r, 2, port),
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
             for r in range(2)]
    outs = []
    try:
        for p in procs:
            outs.append(p.communicate(timeout=180))
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    for p, (_, err) in zip(procs, outs):
        assert p.returncode == 0, err[-2000:]
    res = sorted((json.loads(o.strip().splitlines()[-1]) for o, _ in outs), key=lambda r: r["rank"])
    assert [r["rank"] for r in res] == [0, 1]
    for r in res:
        assert r["ws"] == 2
        assert r["max"] == 2.5          # max over ranks of 1.5 + rank
        assert r["sum"] == 30.0         # 10 + 20


def test_reference_arm_runs_on_rank_zero_only():
    # rank 1 of two leaves without work and without output
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference"],
                         env=_env(1, 2, _free_port()), capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.strip() == ""
