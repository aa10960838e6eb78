"""Multi-GPU sweep logic on the CPU: two gloo ranks each sweep their own rows of a grid (through
the fake device seam) and the assembled map equals the one-process sweep; max-over-ranks timing."""

import os
import socket

import numpy as np
import pytest

from gqis.shard import shard_rows, weak_axis


def test_shard_rows_cover_the_grid_once():
    for n in (1, 7, 8, 2048):
        for ws in (1, 2, 3, 8):
            if ws > n:
                continue
            ranges = [shard_rows(n, ws, r) for r in range(ws)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
            assert max(e - b for b, e in ranges) - min(e - b for b, e in ranges) <= 1
    np.testing.assert_array_equal(weak_axis(np.arange(8), 2, 1), [4, 5, 6, 7])
    with pytest.raises(ValueError):
        weak_axis(np.arange(7), 2, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _sweep(var):
    """mesolve_2D of a two-level model on the fake device, whose result is a function of (eps, A)."""
    import sympy as sp
    import gqis
    from fake_device import fake_device
    eps, A, t, Drive = sp.symbols("eps A t Drive", real=True)
    H = eps / 2 * sp.Matrix([[1, 0], [0, -1]]) + Drive * sp.Matrix([[0, 1], [1, 0]])

    def values(launch):
        X, Y = np.meshgrid(launch.par_x, launch.par_y, indexing="ij")
        return np.stack([X.ravel() * 10 + Y.ravel(), X.ravel() - Y.ravel()], 1)
    with fake_device(values):
        return gqis.mesolve_2D(H, A * sp.cos(t), [], sp.diag(0, 1), np.linspace(0, 1, 5),
                               var_arrays={eps: var[0], A: var[1]}, fp64=True)


def _rank(rank, ws, port, out):
    import sys
    import torch.distributed as dist
    here = os.path.dirname(os.path.abspath(__file__))
    for sub in (here, os.path.join(here, "..", "gpu-quantum-interferometry-solver_b200"), os.path.join(here, "..", "oracle")):
        sys.path.insert(0, sub)
    from gqis.shard import gather_rows, max_over_ranks, shard_rows
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=ws)
    try:
        eps_full, a_axis = np.linspace(-1, 1, 7), np.linspace(0, 2, 3)
        b, e = shard_rows(len(eps_full), ws, rank)
        local = _sweep((eps_full[b:e], a_axis))
        full = gather_rows(local, len(eps_full))
        slowest = max_over_ranks(1.0 + rank)
        np.save(os.path.join(out, f"rank{rank}.npy"), full)
        np.save(os.path.join(out, f"max{rank}.npy"), np.array(slowest))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_assemble_the_one_process_map(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    single = _sweep((np.linspace(-1, 1, 7), np.linspace(0, 2, 3)))
    for r in range(2):
        np.testing.assert_array_equal(np.load(tmp_path / f"rank{r}.npy"), single)
        assert float(np.load(tmp_path / f"max{r}.npy")) == 2.0
