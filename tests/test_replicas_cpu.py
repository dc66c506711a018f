"""The replica protocol of multi-GPU runs on CPU: one process, and two
processes over gloo (barrier, maximum of the ranks' times, clean shutdown).
The same class runs over NCCL with one process per GPU."""
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_RANK_SCRIPT = r'''
import sys
sys.path.insert(0, sys.argv[1])
from n2p2_b200.replicas import Replicas
rep = Replicas("gloo", timeout_s=60)
rep.barrier()
t = rep.max(1.5 * (rep.rank + 1))
rep.barrier()
with open(sys.argv[2], "w") as fh:
    fh.write(f"{rep.rank} {rep.world} {t!r}\n")
rep.close()
'''


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_single_process(monkeypatch):
    from n2p2_b200.replicas import Replicas
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    rep = Replicas("gloo")
    assert (rep.rank, rep.world, rep.local) == (0, 1, 0)
    rep.barrier()
    assert rep.max(2.5) == 2.5
    rep.close()


def test_two_ranks_over_gloo(tmp_path):
    script = tmp_path / "rank.py"
    script.write_text(_RANK_SCRIPT)
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen(
            [sys.executable, str(script), ROOT, str(tmp_path / f"r{r}.txt")],
            env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
            text=True))
    try:
        outs = [p.communicate(timeout=180) for p in procs]
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    for p, (_, err) in zip(procs, outs):
        assert p.returncode == 0, err
    rows = sorted(open(tmp_path / f"r{r}.txt").read().split()
                  for r in range(2))
    assert rows == [["0", "2", "3.0"], ["1", "2", "3.0"]]
