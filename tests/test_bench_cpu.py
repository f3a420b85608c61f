"""CPU tests of bench.py's multi-rank plumbing (gloo, world size 2).

bench.py runs one process per GPU; the ranks are independent replicas and
meet only in the host-side barrier and the max-over-ranks of the timed
region.  These tests run that plumbing on CPU: the max over two gloo ranks,
and the reference arm under torchrun with two ranks (rank 0 times the
reference's CPU path and prints the one JSON line, rank 1 exits 0).
"""
import json
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


def _max_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    w, r, _, pg = bench.dist_setup()
    assert (w, r) == (world, rank)
    out[rank] = bench.max_over_ranks(pg, 1.5 + rank)
    pg.barrier()
    pg.destroy_process_group()


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp
    mgr = mp.Manager()
    out = mgr.dict()
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_max_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    assert dict(out) == {0: 2.5, 1: 2.5}


def test_reference_arm_two_ranks():
    from oracle import refsim
    if not os.path.exists(refsim.LIB_PATH) and not os.path.isdir(refsim.REFERENCE_SOURCE):
        pytest.skip("oracle/_ref not built and reference sources absent")
    refsim.lib()
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--gpus", "2", "--impl", "reference", "--workload", "cylinder", "--steps", "1", "--warmup", "0"]
    env = dict(os.environ, OMP_NUM_THREADS="4")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["value"] > 0


def test_reference_arm_ensemble_workload():
    """The reference arm of the ensemble workload: the compiled reference on
    the first members, one JSON line on the ensemble's name."""
    from oracle import refsim
    if not os.path.exists(refsim.LIB_PATH) and not os.path.isdir(refsim.REFERENCE_SOURCE):
        pytest.skip("oracle/_ref not built and reference sources absent")
    refsim.lib()
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "ensemble",
           "--members", "2", "--steps", "2", "--warmup", "0"]
    env = dict(os.environ, OMP_NUM_THREADS="4")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["config"]["workload"] == "ensemble2_seed0_fp64"
    assert line["steps"] == 2 and line["value"] > 0


def test_ensemble_members_are_drawn_reproducibly():
    from cubismup_2d_b200.synthetic import ENSEMBLE_GRIDS, ensemble_configs, fish_length_ok
    from cubismup_2d_b200.abi import parse_args
    a, b = ensemble_configs(64, seed=0), ensemble_configs(64, seed=0)
    assert a == b and a != ensemble_configs(64, seed=1)
    kinds = set()
    for line in a:
        cfg, shapes = parse_args(line)
        assert (cfg.bpdx, cfg.bpdy) in ENSEMBLE_GRIDS and len(shapes) == 1
        kind, sp = shapes[0]
        kinds.add(kind)
        h = 1.0 / (32 * max(cfg.bpdx, cfg.bpdy))
        if kind == 0:
            assert 0.02 <= sp.radius <= 0.05
            re = 0.2 * 2 * sp.radius / cfg.nu
        else:
            assert 0.15 <= sp.L <= 0.25 and fish_length_ok(sp.L, h)
            re = sp.L * sp.L / cfg.nu
        assert 100 * (1 - 1e-12) <= re <= 1000 * (1 + 1e-12)
    assert kinds == {0, 1}
