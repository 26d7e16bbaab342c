"""CPU checks of bench.py: the multi-rank plumbing (world size 2 over gloo)
and the output contract of the reference arm (the compiled reference on the
host cores)."""
import importlib.util
import json
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _load_bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    bench = _load_bench()
    bench.barrier(world)
    # each rank reports its own timing; the job takes the slowest
    out[rank] = bench.allreduce_max(world, 10.0 + rank)
    out[10 + rank] = bench.allreduce_sum(world, 1.5 + rank)
    bench.barrier(world)
    dist.destroy_process_group()


def _shard_rank_main(rank, world, port, out):
    """One rank of the sharded batched mix, run end to end on the CPU: the
    rank takes its share of a small seeded mix (batch.shard_runs, no
    exchange), advances each of its runs to its end time with the oracle
    (the reference main loop), and joins the job's reductions: cell-updates
    summed over ranks, time the slowest rank's."""
    import time

    import numpy as np
    import torch.distributed as dist

    sys.path.insert(0, os.path.join(ROOT, "mhd2d-solver_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from mhd2d_b200 import batch as B
    from mhd2d_b200 import problems as P
    from pyoracle import Oracle

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    bench = _load_bench()
    mix = B.mixed_runs(12, seed=3, side_min=8, side_max=24)
    costs = np.array([m.run.nx * m.run.ny for m in mix], dtype=np.float64)
    mine = B.shard_runs(costs, world, rank)
    t0 = time.perf_counter()
    cell_updates = 0.0
    for i in mine:
        r = mix[i].run
        p = P.explosion(r.nx, r.ny) if mix[i].kind == "explosion" else \
            P.random_smooth(r.nx, r.ny, seed=i)
        o = Oracle(r.nx, r.ny, p.dx, p.dy, r.gamma, r.bc, scheme=r.scheme, dt_min=r.dt_min,
                   dt_max=r.dt_max, cfl=r.cfl)
        U = p.U.copy()
        res = o.run(U, r.dt0, t_max=0.02)
        cell_updates += float(r.nx * r.ny * res["steps"])
    ms = (time.perf_counter() - t0) * 1e3
    out[rank] = (sorted(mine), cell_updates)
    out[10 + rank] = bench.allreduce_sum(world, cell_updates)
    out[20 + rank] = bench.allreduce_max(world, ms)
    out[30 + rank] = ms
    bench.barrier(world)
    dist.destroy_process_group()


def test_sharded_batched_mix_two_ranks_gloo():
    """The instance-sharded batched path end to end on two gloo ranks: the
    shares partition the runs, the summed cell-updates equal the sum of the
    ranks' own counts, and the job time is the slower rank's."""
    world, port = 2, 29533
    with mp.Manager() as man:
        out = man.dict()
        mp.start_processes(_shard_rank_main, args=(world, port, out), nprocs=world, join=True,
                           start_method="spawn")
        shares = [out[r][0] for r in range(world)]
        assert sorted(shares[0] + shares[1]) == list(range(12))
        assert not set(shares[0]) & set(shares[1])
        total = out[0][1] + out[1][1]
        assert total > 0 and out[10] == total and out[11] == total
        assert out[20] == out[21] == max(out[30], out[31])


def test_batched_runs_shard_without_overlap_and_balanced():
    """Instance sharding of the batched runs (no exchange between GPUs): the
    shares of all ranks partition the runs, one rank takes all, and the
    greedy assignment keeps every rank within one run's cost of the others."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "mhd2d-solver_b200"))
    from mhd2d_b200 import batch as B

    mix = B.mixed_runs(512, seed=0)
    costs = np.array([m.run.nx * m.run.ny for m in mix], dtype=np.float64)
    assert B.shard_runs(costs, 1, 0) == list(range(512))
    for world in (2, 3, 4, 8):
        shares = [B.shard_runs(costs, world, r) for r in range(world)]
        flat = sorted(i for sh in shares for i in sh)
        assert flat == list(range(512))
        loads = [costs[sh].sum() for sh in shares]
        assert max(loads) - min(loads) <= costs.max()
        assert shares == [B.shard_runs(costs, world, r) for r in range(world)]  # deterministic
    with pytest.raises(ValueError):
        B.shard_runs(costs, 2, 2)


def test_two_rank_max_over_ranks_gloo():
    world, port = 2, 29531
    with mp.Manager() as man:
        out = man.dict()
        mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, join=True,
                           start_method="spawn")
        assert out[0] == 11.0 and out[1] == 11.0
        assert out[10] == 4.0 and out[11] == 4.0


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_bench")),
                    reason="oracle/_ref not built")
def test_reference_arm_prints_one_json_line():
    """The reference arm on a small grid (the bench's default is 4096^2, ~19
    GB and ~35 s per step per copy): one JSON line naming the same config
    as the GPU arm, the requested steps spread over the copies."""
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--n", "96", "--steps", "3", "--warmup", "2"], capture_output=True,
                       text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "cell-updates/s"
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["higher_is_better"] is True
    assert d["steps"] == 3 and d["warmup"] == 2
    assert d["config"] == _load_bench().bench_config(96, "roe")
    assert "3 timed steps" in d["cpu_baseline"]["sample"]


def test_reference_copies_bounded_by_host_memory():
    bench = _load_bench()
    copies, avail, per = bench.ref_copies(4096, 16)
    assert 1 <= copies <= 16
    if avail is not None:
        assert copies == 1 or copies * per <= avail - 8e9
    # the timed and warm-up steps are spread over the copies without loss
    for total, parts in ((20, 9), (3, 8), (10, 10)):
        assert sum(bench._split(total, parts, c) for c in range(parts)) == total
