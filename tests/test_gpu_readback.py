"""Render data on the GPU (prep_readback.rs, headless) against the oracle: the
ReadbackData records of every mode after a few steps, in particle-id order on
block-ordered storage too, the device-buffer form, and the rigid particles."""
import numpy as np
import pytest

from nexus_b200 import scenes
from nexus_b200.mpm import (MpmPipeline, state_from_scene, RENDER_VOLUME, RENDER_CDF_NORMALS, RENDER_CDF_SIGNS,
                            RENDER_DEFAULT, RENDER_VELOCITY)

pytestmark = pytest.mark.gpu


def _decorated(sc, seed=3):
    """Varied group ids and phases, a few disabled particles."""
    p = sc.particles
    rng = np.random.default_rng(seed)
    p.group_id = rng.integers(0, 11, p.n).astype(np.uint32)
    p.phase = rng.uniform(0.0, 1.0, p.n).astype(np.float32)
    p.enabled[::97] = 0
    return sc


def _run(sc, deterministic, steps, use_cpic=False):
    from oracle.oracle import OracleScene
    st = state_from_scene(sc, deterministic=deterministic, use_cpic=use_cpic)
    pipe = MpmPipeline()
    for _ in range(steps):
        pipe.step(st)
    st.synchronize()
    o = OracleScene(sc)
    o.set_use_cpic(use_cpic)
    o.step(steps)
    return st, o


@pytest.mark.parametrize("deterministic", [True, False])
def test_prep_readback_matches_oracle(gpu_lib, oracle_built, deterministic):
    sc = _decorated(scenes.elastic_cube(n_side=16))
    st, o = _run(sc, deterministic, 20)
    pal = np.random.default_rng(9).uniform(0, 1, (7, 4)).astype(np.float32)
    pos = st.read_positions()
    for mode in range(7):
        g, w = st.prep_readback(mode, pal), o.prep_readback(mode, pal)
        # the records follow particle ids, wherever the fast mode stores them
        np.testing.assert_array_equal(g["position"], pos)
        np.testing.assert_allclose(g["position"], w["position"], rtol=0, atol=1e-5)
        np.testing.assert_allclose(g["deformation"], w["deformation"], rtol=0, atol=1e-6)
        tol = 2e-3 if mode == RENDER_VOLUME else 1e-5  # singular values are scaled by 1 / 0.005
        np.testing.assert_allclose(g["color"], w["color"], rtol=0, atol=tol)
        assert (g["color"][::97] == np.array([1, 0, 0, 1], np.float32)).all()  # disabled: red


def test_prep_readback_cdf_modes_match_oracle(gpu_lib, oracle_built):
    sc = scenes.cpic_trimesh()
    st, o = _run(sc, True, 60, use_cpic=True)
    for mode in range(RENDER_CDF_NORMALS, RENDER_CDF_SIGNS + 1):
        g, w = st.prep_readback(mode), o.prep_readback(mode)
        # the fitted normals and distances after 60 steps: a few ill-conditioned
        # fits amplify the last-bit differences of the positions
        np.testing.assert_allclose(g["color"], w["color"], rtol=0, atol=1e-3)
        assert (np.abs(g["color"] - w["color"]).max(1) <= 1e-5).mean() > 0.99
    signs = st.prep_readback(RENDER_CDF_SIGNS)["color"]
    assert (signs[:, 1] == 1.0).sum() > 100  # particles with an affinity and no sign bit


def test_prep_render_fills_device_buffers(gpu_lib):
    import torch
    sc = _decorated(scenes.elastic_cube(n_side=12))
    st = state_from_scene(sc)
    pipe = MpmPipeline()
    for _ in range(5):
        pipe.step(st)
    n = sc.n
    pos = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    dfm = torch.empty((n, 9), dtype=torch.float32, device="cuda")
    col = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    st.prep_render(RENDER_VELOCITY, pos.data_ptr(), dfm.data_ptr(), col.data_ptr())
    st.synchronize()
    r = st.prep_readback(RENDER_VELOCITY)
    np.testing.assert_array_equal(pos.cpu().numpy(), r["position"])
    np.testing.assert_array_equal(dfm.cpu().numpy().reshape(n, 3, 3), r["deformation"][:, :3, :3])
    np.testing.assert_array_equal(col.cpu().numpy(), r["color"])


def test_prep_readback_rigid_matches_oracle(gpu_lib, oracle_built):
    sc = scenes.cpic_trimesh()
    st, o = _run(sc, True, 10, use_cpic=True)
    g, w = st.prep_readback_rigid(), o.prep_readback_rigid()
    assert len(g["position"]) == len(w["position"]) > 10000
    np.testing.assert_allclose(g["position"], w["position"], rtol=0, atol=1e-5)
    np.testing.assert_array_equal(g["color"], w["color"])
    np.testing.assert_array_equal(g["deformation"], w["deformation"])
    cols = np.random.default_rng(2).uniform(0, 1, (len(g["position"]), 4)).astype(np.float32)
    np.testing.assert_array_equal(st.prep_readback_rigid(colors=cols)["color"], cols)
    st2 = state_from_scene(sc, use_cpic=True)  # before any step: the local samples
    np.testing.assert_array_equal(st2.prep_readback_rigid()["position"], st2.read_rigid_particles()["local"])
    assert st.prep_readback(RENDER_DEFAULT)["color"].shape == (sc.n, 4)
