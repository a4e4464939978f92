"""Data-parallel views (multiview.py): the sharding arithmetic, and the split
iteration over two gloo ranks with the oracle as each rank's compute, against
the oracle's single-process iteration over all views."""
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from nanotracer_b200.multiview import chunk_range, expected_shards, shard_size, split_views


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("n,world", [(1, 1), (5, 2), (1000, 2), (1000, 3), (64 * 8, 8), (100, 8), (10**6, 8)])
def test_chunks_tile_the_splats(n, world):
    shard = shard_size(n, world)
    assert shard % 64 == 0 and shard * world >= n
    chunks = expected_shards(n, world)
    covered = np.zeros(n, np.int32)
    for r, (lo, count) in enumerate(chunks):
        assert 0 <= count <= shard and (count == 0 or lo == r * shard)
        covered[lo:lo + count] += 1
    assert np.all(covered == 1)
    assert chunk_range(n, shard, world - 1)[0] <= n


@pytest.mark.parametrize("total,world", [(8, 1), (8, 2), (8, 3), (3, 2), (8, 8)])
def test_views_are_split_in_contiguous_blocks(total, world):
    blocks = [split_views(total, world, r) for r in range(world)]
    assert sum(blocks, []) == list(range(total))
    assert max(map(len, blocks)) - min(map(len, blocks)) <= 1


def _oracle_reference(O, steps, n, V, densify_at):
    from tests.oracle_view_backend import LRS, problem
    from nanotracer_b200.adam_gpu import DENSIFY_GRAD_THRESHOLD, PRUNE_OPACITY_LOGIT, SPLIT_SCALE_THRESHOLD
    scene, cams, tl, tgt = problem(n=n, V=V)
    s = O.OSplats.from_buffer(scene, 4 * n)
    m, v = O.OSplats.zeros(n, 4 * n), O.OSplats.zeros(n, 4 * n)
    acc = np.zeros(4 * n, np.float32)
    losses = []
    for t in range(1, steps + 1):
        loss, _ = O.train_step(s, m, v, acc, cams, tgt, tl, 1, LRS, t)
        losses.append(loss)
        if densify_at and t == densify_at:
            O.prune(s, m, v, acc, PRUNE_OPACITY_LOGIT)
            O.densify(s, m, v, acc, t, DENSIFY_GRAD_THRESHOLD, SPLIT_SCALE_THRESHOLD, 2 * n, t)
            acc[:] = 0.0
    return s, m, v, acc, losses


def _spawn(tmp_path, world, steps, n, V, densify_at):
    from tests.oracle_view_backend import run_rank
    mp.start_processes(run_rank, args=(world, _free_port(), str(tmp_path), steps, n, V, densify_at), nprocs=world,
                       join=True, start_method="spawn")
    return [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]


@pytest.mark.parametrize("world,V,n", [(2, 4, 300), (2, 3, 257)])
def test_two_rank_split_iteration_matches_single_process(oracle, tmp_path, world, V, n):
    steps = 2
    outs = _spawn(tmp_path, world, steps, n, V, 0)
    # every rank ends with the same parameters
    for o in outs[1:]:
        assert np.array_equal(o["params"], outs[0]["params"])
    assert sorted(sum((list(o["views"]) for o in outs), [])) == list(range(V))
    s, m, v, acc, losses = _oracle_reference(oracle, steps, n, V, 0)
    # the cross-rank sum reassociates the per-view gradient sum: float rounding only
    assert np.allclose(outs[0]["losses"], losses, rtol=1e-6)
    want = s.flat()
    got = outs[0]["params"]
    assert np.mean(np.abs(got - want) <= 1e-6 + 1e-6 * np.abs(want)) > 0.995
    # each rank updated only its chunk of the moments; together they are the full moments
    shard = shard_size(n, world)
    mg = np.concatenate([outs[r]["m"][r * shard:(r + 1) * shard] for r in range(world)])
    assert np.allclose(mg, m.flat(), rtol=1e-4, atol=1e-9)
    ag = np.concatenate([outs[r]["acc"][r * shard:(r + 1) * shard] for r in range(world)])
    assert np.allclose(ag, acc[:n], rtol=1e-4, atol=1e-9)


def test_two_rank_state_gather_then_densify_and_prune(oracle, tmp_path):
    n, V, world, steps = 300, 4, 2, 3
    outs = _spawn(tmp_path, world, steps, n, V, 2)
    for o in outs[1:]:
        assert np.array_equal(o["params"], outs[0]["params"])
    s, m, v, acc, losses = _oracle_reference(oracle, steps, n, V, 2)
    got, want = outs[0]["params"], s.flat()
    # the same splat count on every rank and in the oracle, and the schedule did densify
    assert got.shape == want.shape and s.n > n
    assert np.mean(np.abs(got - want) <= 1e-5 + 1e-5 * np.abs(want)) > 0.99
    assert np.allclose(outs[0]["losses"], losses, rtol=1e-5)


def test_a_rank_that_leaves_makes_the_others_fail_not_hang(tmp_path):
    from tests.oracle_view_backend import run_rank_leaving
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=run_rank_leaving, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, "a rank hung"
    assert (tmp_path / "rank1.txt").read_text() == "left"
    outcome, secs = (tmp_path / "rank0.txt").read_text().split()
    assert outcome.startswith("error:") and float(secs) < 60


def test_multiview_data_plane_imports_no_torch():
    """The product exchange (multiview + nccl) is the C ABI and NCCL's C API
    only: importing it loads no torch."""
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    code = ("import sys; sys.path.insert(0, %r); import nanotracer_b200.multiview, nanotracer_b200.nccl; "
            "print('torch' in sys.modules)" % str(root))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True)
    assert out.stdout.strip() == "False"


def _rendezvous_rank(rank, world, port, q):
    from nanotracer_b200.nccl import rendezvous_bytes
    payload = bytes(range(128)) if rank == 0 else None
    q.put((rank, rendezvous_bytes(payload, rank, world, "127.0.0.1", port, timeout=20.0)))


def test_unique_id_rendezvous_reaches_every_rank():
    """The NCCL unique id's TCP rendezvous: rank 0's 128 bytes reach every rank."""
    import multiprocessing as pmp
    ctx = pmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rendezvous_rank, args=(r, 3, port, q)) for r in range(3)]
    for p in ps:
        p.start()
    got = dict(q.get(timeout=60) for _ in ps)
    for p in ps:
        p.join(timeout=30)
    assert all(got[r] == bytes(range(128)) for r in range(3))


def test_rendezvous_without_rank0_errors_instead_of_hanging():
    from nanotracer_b200.nccl import NcclError, rendezvous_bytes
    import time
    t0 = time.time()
    with pytest.raises(NcclError):
        rendezvous_bytes(None, 1, 2, "127.0.0.1", _free_port(), timeout=1.0)
    assert time.time() - t0 < 10
