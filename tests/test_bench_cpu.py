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
    bench.barrier(world)
    dist.destroy_process_group()


def test_two_rank_max_over_ranks_gloo():
    world, port = 2, 29531
    with mp.Manager() as man:
        out = man.dict()
        mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, join=True,
                           start_method="spawn")
        assert out[0] == 11.0 and out[1] == 11.0


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_bench")),
                    reason="oracle/_ref not built")
def test_reference_arm_prints_one_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "1"], capture_output=True, text=True,
                       timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "cell-updates/s"
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["higher_is_better"] is True
