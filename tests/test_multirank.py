"""Multi-rank path sharding on CPU: two gloo ranks each track a contiguous
path range (the CPU restatement stands in for each rank's GPU here), the
records are gathered in path order and finished by the library's host
bookkeeping (phc_finish_solve); the result must equal a single-process
solve of the restatement (same counts, indices, solutions)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, name, outdir):
    import torch.distributed as dist
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    from oracle import oracle as O
    import polyhomocont_b200 as P
    from polyhomocont_b200 import shard
    from polyhomocont_b200 import workloads as W
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n, eqs = {"cyclic5": lambda: W.cyclic(5), "katsura4": lambda: W.katsura(4),
                  "mixed": lambda: (2, [([1, -1], [[1, 0], [1, 0]]),
                                        ([1, -3, 2], [[3, 1, 0], [0, 0, 0]])])}[name]()
        so = W.build(O.SparseSystem, n, eqs)
        sp = W.build(P.SparseSystem, n, eqs)

        def runner(k0, count):
            p, z, x, st = O.solve_paths(so, k0=k0, count=count)
            assert st == 0
            return p, z, x

        res = shard.solve_sharded(sp, rank, world, runner=runner)
        if rank == 0:
            np.savez(os.path.join(outdir, f"{name}.npz"), paths=res.paths, sols=res.solutions,
                     ssols=res.singular_solutions, mult=res.multiplicities,
                     counts=np.array([res.nsolutions, res.nreal, res.nsingular, res.ninfinite,
                                      res.nfailed, res.nduplicates]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", ["cyclic5", "katsura4", "mixed"])
@pytest.mark.parametrize("world", [2, 3])
def test_sharded_solve_matches_single_process(orc, tmp_path, name, world):
    from polyhomocont_b200 import build as B
    B.build()
    mp.start_processes(_worker, args=(world, _free_port(), name, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    got = np.load(os.path.join(tmp_path, f"{name}.npz"))
    from polyhomocont_b200 import workloads as W
    n, eqs = {"cyclic5": lambda: W.cyclic(5), "katsura4": lambda: W.katsura(4),
              "mixed": lambda: (2, [([1, -1], [[1, 0], [1, 0]]),
                                    ([1, -3, 2], [[3, 1, 0], [0, 0, 0]])])}[name]()
    ref, st = orc.solve(W.build(orc.SparseSystem, n, eqs))
    assert list(got["counts"]) == [ref.nsolutions, ref.nreal, ref.nsingular, ref.ninfinite,
                                   ref.nfailed, ref.nduplicates]
    assert np.array_equal(got["paths"]["solution_index"], ref.paths["solution_index"])
    assert np.array_equal(got["paths"]["singular_index"], ref.paths["singular_index"])
    assert np.array_equal(got["sols"], ref.solutions)
    assert np.array_equal(got["ssols"], ref.singular_solutions)
    assert list(got["mult"]) == list(ref.multiplicities)


def test_path_ranges_partition():
    from polyhomocont_b200.shard import path_range
    for npaths in (1, 7, 1024, 65536):
        for world in (1, 2, 3, 8):
            ks = [path_range(npaths, r, world) for r in range(world)]
            assert ks[0][0] == 1
            for (a, ca), (b, _) in zip(ks, ks[1:]):
                assert a + ca == b
            assert sum(c for _, c in ks) == npaths
            assert max(c for _, c in ks) - min(c for _, c in ks) <= 1


def _worker_failing(rank, world, port, mode, outdir):
    """Rank 1 fails; rank 0 must learn of it (an error, never a hang)."""
    import time
    import sys
    from datetime import timedelta
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    from oracle import oracle as O
    import polyhomocont_b200 as P
    from polyhomocont_b200 import shard
    from polyhomocont_b200 import workloads as W
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=5))
    n, eqs = W.katsura(3)
    so = W.build(O.SparseSystem, n, eqs)
    sp = W.build(P.SparseSystem, n, eqs)

    def runner(k0, count):
        if rank == 1:
            if mode == "exit":
                os._exit(0)  # the rank dies without a word
            raise RuntimeError("injected tracking failure")
        p, z, x, st = O.solve_paths(so, k0=k0, count=count)
        return p, z, x

    t0 = time.time()
    outcome = "returned"
    try:
        shard.solve_sharded(sp, rank, world, runner=runner)
    except Exception as e:  # noqa: BLE001 - the outcome is the test's subject
        outcome = f"{type(e).__name__}: {e}"
    with open(os.path.join(outdir, f"rank{rank}.txt"), "w") as f:
        f.write(f"{time.time() - t0:.3f}\n{outcome}\n")
    try:
        dist.destroy_process_group()
    except Exception:  # noqa: BLE001 - the peer may be gone
        pass


@pytest.mark.parametrize("mode", ["raise", "exit"])
def test_failed_rank_is_detected(tmp_path, mode):
    from polyhomocont_b200 import build as B
    B.build()
    mp.start_processes(_worker_failing, args=(2, _free_port(), mode, str(tmp_path)), nprocs=2,
                       join=True, start_method="spawn")
    t0, out0 = open(os.path.join(tmp_path, "rank0.txt")).read().split("\n", 1)
    assert float(t0) < 60.0
    assert out0.startswith(("ShardFailure", "RuntimeError", "DistBackendError")), out0
    if mode == "raise":
        assert "ranks failed: 1" in out0 and "injected tracking failure" in out0
        t1, out1 = open(os.path.join(tmp_path, "rank1.txt")).read().split("\n", 1)
        assert out1.startswith("ShardFailure")


def test_single_rank_needs_no_process_group(orc):
    """world == 1 (bench.py on one GPU with a path subset): solve_sharded
    gathers nothing and finishes the first npaths paths directly."""
    import polyhomocont_b200 as P
    from polyhomocont_b200 import shard
    from polyhomocont_b200 import workloads as W
    n, eqs = W.cyclic(5)
    so = W.build(orc.SparseSystem, n, eqs)
    sp = W.build(P.SparseSystem, n, eqs)

    def runner(k0, count):
        p, z, x, st = orc.solve_paths(so, k0=k0, count=count)
        assert st == 0
        return p, z, x

    res = shard.solve_sharded(sp, 0, 1, runner=runner, npaths=40)
    p, z, x, st = orc.solve_paths(so, k0=1, count=40)
    ref = P.result_from_arrays(n, p, x)
    assert res.npaths == 40
    assert np.array_equal(res.paths["solution_index"], ref.paths["solution_index"])
    assert res.nsolutions == ref.nsolutions and res.ninfinite == ref.ninfinite
