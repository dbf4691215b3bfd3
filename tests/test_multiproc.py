"""The multi-rank plumbing of bench.py on CPU: two ranks over gloo, launched the way the driver
launches the GPU runs (torch.distributed.run, rendezvous on 127.0.0.1).  Chains are replicas, so
the only collectives are the timing barrier and the max/sum of per-rank scalars."""
import json
import os
import re
import socket
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _torchrun(args, timeout):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={_port()}"] + args
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    return subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, cwd=ROOT, env=env)


def test_two_ranks_reduce_max_and_sum(tmp_path):
    probe = tmp_path / "probe.py"
    probe.write_text(textwrap.dedent(f"""
        import json, sys
        sys.path.insert(0, {ROOT!r})
        import bench
        d = bench.Dist(2)
        d.barrier()
        out = {{"rank": d.rank, "world": d.world, "max": d.max(10.0 + d.rank), "sum": d.sum(1.5 * (d.rank + 1))}}
        print("RESULT " + json.dumps(out), flush=True)
        d.close()
    """))
    r = _torchrun([str(probe)], timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    # the two ranks share stdout, so their lines may interleave
    res = [json.loads(m) for m in re.findall(r"RESULT (\{[^}]*\})", r.stdout)]
    assert sorted(x["rank"] for x in res) == [0, 1]
    for x in res:
        assert x["world"] == 2 and x["max"] == 11.0 and x["sum"] == 4.5


def test_reference_arm_under_two_ranks_prints_one_line():
    r = _torchrun(["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1"], timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    res = json.loads(lines[0])
    assert res["impl"] == "reference" and res["n_gpus"] == 2 and res["value"] > 0
    assert res["cpu_baseline"]["kind"] == "port" and res["e2e"]["h2d_bytes_per_step"] == 0
