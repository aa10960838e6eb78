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


def _fit_maps():
    """A synthetic 7 x 5 model map, its gradient in 3 parameters and a measured map."""
    rng = np.random.default_rng(3)
    return rng.random((7, 5)), rng.standard_normal((7, 5, 3)), rng.random((7, 5))


def _fit_rank(rank, ws, port, out):
    import sys
    import torch.distributed as dist
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "..", "gpu-quantum-interferometry-solver_b200"))
    from gqis.shard import fit_loss_gradient, shard_rows
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=ws)
    try:
        m, g, y = _fit_maps()
        b, e = shard_rows(m.shape[0], ws, rank)
        loss, grad = fit_loss_gradient(m[b:e], g[b:e], y[b:e])
        np.save(os.path.join(out, f"fit{rank}.npy"), np.concatenate([[loss], grad]))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_sharded_fit_gradient_is_the_one_process_gradient(tmp_path):
    """Two gloo ranks each own rows of the map; one all-reduce of loss + 3 gradient sums gives every
    rank the whole grid's least-squares loss and gradient."""
    import torch.multiprocessing as mp
    from gqis.shard import fit_loss_gradient
    m, g, y = _fit_maps()
    loss, grad = fit_loss_gradient(m, g, y)  # no process group: this process's sums
    np.testing.assert_allclose(loss, np.sum((m - y) ** 2), rtol=1e-14)
    np.testing.assert_allclose(grad, [2 * np.sum((m - y) * g[..., k]) for k in range(3)], rtol=1e-12)
    port = _free_port()
    mp.start_processes(_fit_rank, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    for r in range(2):
        np.testing.assert_allclose(np.load(tmp_path / f"fit{r}.npy"), np.concatenate([[loss], grad]), rtol=1e-12)
