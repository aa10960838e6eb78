"""GPU tests of the phase-space rasteriser (gqis.render, csrc/gqis_render.cu) against the reference
kernels' golden outputs and the NumPy oracle."""

from pathlib import Path

import numpy as np
import pytest

import render_oracle

GOLDEN = Path(__file__).resolve().parent / "golden"


def _rasterizer(g, **kw):
    from gqis.render import PhaseRasterizer
    return PhaseRasterizer(g["colors"], x_range=tuple(g["x_range"]), v_range=tuple(g["v_range"]),
                           bins=tuple(int(b) for b in g["bins"]), **kw)


@pytest.mark.gpu
def test_raster_matches_reference_binning_and_oracle_means():
    g = np.load(GOLDEN / "render_raster.npz")
    got = _rasterizer(g).render(g["points"])
    ref, counts = render_oracle.bin_raster(g["points"], g["colors"], g["bins"], g["x_range"], g["v_range"])
    np.testing.assert_array_equal(np.isnan(got), np.isnan(g["raster"]))  # same occupied pixels as the reference
    occ = ~np.isnan(ref)
    np.testing.assert_array_max_ulp(got[occ], ref[occ], maxulp=1)     # FP64 sums, any atomic order
    assert np.max(np.abs(got[occ] - g["raster"][occ])) < 2e-4           # vs the reference's FP32 sums


@pytest.mark.gpu
def test_device_fp64_points_partitions_and_trace_views_give_the_same_raster():
    import torch
    g = np.load(GOLDEN / "render_raster.npz")
    host = _rasterizer(g).render(g["points"])
    pts64 = torch.as_tensor(g["points"], dtype=torch.float64, device="cuda")
    dev = _rasterizer(g, partitions=1).render(pts64, return_device=True).cpu().numpy()
    np.testing.assert_array_max_ulp(dev[~np.isnan(dev)], host[~np.isnan(host)], maxulp=1)
    n = len(g["points"])
    trace = torch.zeros((n, 4, 3), dtype=torch.float64, device="cuda")  # (points, samples, state)
    trace[:, 2, 1:3] = pts64
    via_trace = _rasterizer(g).render_trace(trace, 2, components=(1, 2))
    np.testing.assert_array_max_ulp(via_trace[~np.isnan(via_trace)], host[~np.isnan(host)], maxulp=1)


@pytest.mark.gpu
def test_display_rgba_matches_reference_kernel():
    from gqis.render import GPUDisplayImage
    g = np.load(GOLDEN / "render_display.npz")
    lo, hi = g["color_range"]
    for k, ((w, h, linear), view) in enumerate(zip(g["cases"], g["views"])):
        disp = GPUDisplayImage(g["lut"], lo, hi, "bilinear" if linear else "nearest")
        img = disp.render(g["raster"], (int(w), int(h), *[float(v) for v in view]))
        np.testing.assert_array_equal(img, g[f"image_{k}"], err_msg=f"case {k}")


@pytest.mark.gpu
def test_odesolve_trace_is_binned_in_place():
    """Fused path: a Duffing sweep's state trace stays on the device and is binned sample by sample."""
    import gqis
    from gqis.render import PhaseRasterizer
    from test_support_calls import duffing_case
    _, args, kwargs = duffing_case(side=16, solver="rk4", return_device=True)
    kwargs.pop("adaptive_options")
    args = args[:3] + (np.linspace(0.0, 50.0, 1001),)  # RK4 needs dt well below the grid's 0.98 here
    final, trace, _ = gqis.odesolve_2D(*args, **kwargs)
    colors = np.linspace(0.0, 1.0, 256, dtype=np.float32)
    r = PhaseRasterizer(colors, x_range=(-2, 2), v_range=(-2, 2), bins=(48, 40))
    host = trace.cpu().numpy().reshape(256, trace.shape[-2], 2)
    for k in (0, trace.shape[-2] // 2, trace.shape[-2] - 1):
        got = r.render_trace(trace, k)
        ref, _ = render_oracle.bin_raster(host[:, k], colors, (48, 40), (-2, 2), (-2, 2))
        np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
        np.testing.assert_array_max_ulp(got[~np.isnan(got)], ref[~np.isnan(ref)], maxulp=1)
