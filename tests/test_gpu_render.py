"""Headless render (LiquidModel<3>::Render, LiquidModel.cpp:1138-1159, with
Shader/Scene3D_vertex.glsl) on the GPU against the oracle's restatement:
the vertex shader's coordinates and the drawn image, bit for bit."""
import numpy as np
import pytest

from liquidhairinteration_b200 import scenes

from helpers import assert_bitwise, gpu_model

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("size,w,h", [(5.0, 480, 480), (4.0, 200, 120), (1.0, 64, 64), (7.5, 333, 211)])
def test_render_matches_oracle(oracle_mod, lhi, prec, size, w, h):
    spec = scenes.dam(32)
    g = gpu_model(spec, prec)
    pos, vel = scenes.seed(spec, "fp64" if prec == "fp64" else "fp32")
    ps = g.GetParticleSystem()
    ps.SetParticles(pos, vel)
    g.PreStep(spec.dt)
    g.Step(spec.dt)
    # a few particles off the domain (clipped by the rasteriser) and on its faces
    pos, vel, aff = ps.GetParticles()
    pos[:5, 0] = [-0.2, 1.3, 0.999, 0.0, 1.0]
    ps.SetParticles(pos, vel, aff)
    g.sort_particles()  # device order = the cell sort; NDC come back in the caller's order
    img, ndc = g.Render(w, h, size, color=(10, 20, 230, 255), background=(255, 250, 240, 255), ndc=True)
    p = g.GetParticleSystem().GetPositions().astype(np.float32)
    img_o, ndc_o = oracle_mod.render(p, (0, 0, 0), (1, 1, 1), w, h, size, (10, 20, 230, 255), (255, 250, 240, 255))
    assert_bitwise(ndc, ndc_o, "ndc")
    assert np.array_equal(img, img_o), int((img != img_o).any(axis=2).sum())
    assert (img[..., 2] == 230).any() and (img[..., 2] == 240).any()


def test_render_without_particles(lhi):
    spec = scenes.dam(16)
    g = gpu_model(spec, "fp32")
    img = g.Render(32, 16)
    assert img.shape == (16, 32, 4) and (img == 255).all()
