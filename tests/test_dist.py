"""bench.py's multi-process plumbing on CPU with gloo, world size 2: each rank is an
independent replica (its own seeded scene), ranks meet only at the barrier and in the
max-over-ranks of the timed region; the aggregate sums every rank's particle-updates."""
import os
import socket
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = textwrap.dedent('''
    import os, sys, json
    sys.path.insert(0, {root!r})
    import bench
    d = bench.Dist(2, backend="gloo")
    assert d.world == 2
    sc = bench.make_scene("dam_break_sph", seed_offset=d.rank)
    d.barrier()
    t_rank = 10.0 + 5.0 * d.rank            # this rank's device time, ms
    t_max = d.max(t_rank)
    total = d.sum(float(sc.n) * 3)
    first = float(sc.positions[0, 0])
    firsts = [d.sum(first if r == d.rank else 0.0) for r in range(2)]
    print(json.dumps(dict(rank=d.rank, t_max=t_max, total=total, firsts=firsts, n=sc.n)))
    d.close()
''')


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_gloo_replicas(tmp_path):
    script = tmp_path / "rank.py"
    script.write_text(SCRIPT.format(root=ROOT))
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), PYTHONPATH=ROOT)
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err
        outs.append(out.strip().splitlines()[-1])
    import json
    res = [json.loads(o) for o in outs]
    for r in res:
        assert r["t_max"] == 15.0                    # max over ranks, not the local time
        assert r["total"] == 2 * 3 * r["n"]          # every rank's updates are counted
        assert r["firsts"][0] != r["firsts"][1]      # replicas are different seeded scenes


def test_bench_cli_launches_its_own_ranks():
    """`python bench.py --gpus 2` outside torchrun starts two ranks itself; --dry-run runs the
    replica path on CPU oracle samples over gloo. One line, from rank 0, with n_gpus 2 and the
    aggregate of both ranks."""
    import json
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "LOCAL_RANK", "WORLD_SIZE")}
    r = subprocess.run([sys.executable, "bench.py", "--gpus", "2", "--dry-run", "--steps", "2", "--warmup", "1",
                        "--workload", "dam_break_pcisph"], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and d["dry_run"] is True and d["config"]["parallelism"] == "replicas x2"
    assert abs(d["value"] - 2 * d["particles_per_rank"] * d["steps"] / (d["ms_per_step"] * d["steps"] / 1e3)) \
        <= 1e-6 * d["value"]
