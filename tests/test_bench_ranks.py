"""World-size-2 checks of bench.py's rank logic on CPU (gloo): the timing
reduction takes the maximum over ranks, ensemble runs shard across ranks with
every run on exactly one rank, and the reference arm under torchrun prints
one line from rank 0 while the other rank exits without work."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, 'oracle'))


def free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup(None)
    try:
        m = bench.max_over_ranks(float(r + 1) * 0.5, w)
        bench.barrier(w)
        specs = bench.ensemble_specs(37)
        mine = list(range(37))[r::w]
        q.put((r, m, mine, [specs[i] for i in mine]))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_ensemble_sharding():
    world = 2
    ctx = mp.get_context('spawn')
    q = ctx.SimpleQueue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get() for _ in range(world))
    assert all(m == 1.0 for _, m, _, _ in res)            # max of 0.5, 1.0
    ids = sorted(i for _, _, mine, _ in res for i in mine)
    assert ids == list(range(37))                          # every run on exactly one rank
    import bench
    full = bench.ensemble_specs(37)
    for _, _, mine, specs in res:
        assert specs == [full[i] for i in mine]            # same seeded draw on every rank


def test_reference_arm_two_ranks():
    from em2d_oracle import ref_available
    if not (ref_available('avx2') or ref_available('scalar')):
        pytest.skip('reference build oracle/_ref not present')
    cmd = [sys.executable, '-m', 'torch.distributed.run', '--nnodes=1', '--nproc-per-node', '2',
           '--master-addr', '127.0.0.1', '--master-port', str(free_port()),
           os.path.join(ROOT, 'bench.py'), '--impl', 'reference', '--gpus', '2',
           '--steps', '2', '--warmup', '3', '--ref-cells', '64']
    env = dict(os.environ, OMP_NUM_THREADS='2')
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith('{')]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d['impl'] == 'reference' and d['n_gpus'] == 2
    assert d['value'] > 0 and d['cpu_baseline']['kind'] == 'reference'
    assert d['e2e']['h2d_bytes_per_step'] == 0
