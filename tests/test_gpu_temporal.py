"""Temporal multi-sample resolve: jittered layers rendered on the device equal
the oracle's jittered renders with the same seeds, and their resolve equals
the oracle's resolve (renderer/triangle.frag)."""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

import frep
import oracle
from frep import scenes
from parity import device_tree, oracle_tree

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = frep.Context(0, hbm_budget_bytes=8 << 30)
    yield c
    c.close()


@pytest.mark.parametrize("n_samples", [1, 4, 7])
def test_temporal_resolve_matches_oracle(ctx, n_samples):
    import torch
    sc = scenes.random_csg(30, seed=17, grid_dims=[16, 8], width=120, height=80)
    vs = device_tree(ctx, sc, rounding=1)
    orc = oracle_tree(sc, vs.tape, rounding=1)
    lights = frep.Lights(shadow_mask=1)
    rt = frep.Raytracer(ctx, vs)
    rt.lights = lights
    cam = dataclasses.replace(sc.camera, jitter_seed=3.25)
    rgba, layers = rt.trace_temporal(cam, 0.0, sc.width, sc.height, n_samples)
    torch.cuda.synchronize()
    o_layers = []
    for i in range(n_samples):
        ci = dataclasses.replace(cam, jitter=True, jitter_seed=cam.jitter_seed + i)
        o_rgba, _ = orc.render(oracle.camera_vector(ci, sc.width, sc.height), lights, 0.0)
        o_layers.append(o_rgba)
    o_layers = np.stack(o_layers)
    np.testing.assert_array_equal(layers.cpu().numpy(), o_layers)
    np.testing.assert_array_equal(rgba.cpu().numpy(), oracle.resolve_layers(o_layers))
    if n_samples > 1:  # jitter moves rays: the layers differ somewhere
        assert (o_layers[0] != o_layers[1]).any()
    # the stand-alone resolve of the same layers
    again = frep.resolve_layers(layers)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(again.cpu().numpy(), rgba.cpu().numpy())


def test_resolve_rounding_edges(ctx):
    """Exact mean, ties rounded up, alpha 255."""
    import torch
    vals = np.array([[0, 1], [1, 2], [254, 255], [255, 255], [3, 4]], np.uint8)  # pairs of layer values
    layers = np.zeros((2, 1, len(vals), 4), np.uint8)
    layers[0, 0, :, :3] = vals[:, :1]
    layers[1, 0, :, :3] = vals[:, 1:]
    layers[..., 3] = 7
    out = frep.resolve_layers(torch.from_numpy(layers).cuda())
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    np.testing.assert_array_equal(got, oracle.resolve_layers(layers))
    np.testing.assert_array_equal(got[0, :, 0], [1, 2, 255, 255, 4])
    assert (got[..., 3] == 255).all()
