"""The thin-lens camera, the normal integrator and the command-line renderer on the GPU,
against the oracle."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

import oracle
import pbrt_b200 as pb
from conftest import ROOT, fixture_mesh_loader, stage_text
from oracle.stage import load_stage
from test_image_cli import read_png

pytestmark = pytest.mark.gpu

THIN = """camera thin_lens pos -1.5 0.3 1.5 look 0 0 0 up 0 1 0 radius 0.08 focal_length 2.1
scene
  object transformed object simple sphere 0.4 metal 0.2 color 0 0.65 1 transform { translate -1 0 0 }
  object transformed object simple sphere 0.4 lambertian color 0.8 0.3 0.3 transform { translate 0 0 0 }
  object transformed object simple sphere 0.4 lambertian color 0.3 0.8 0.3 transform { translate 1 0 -1 }
  object transformed object simple rectangle 6 6
    lambertian checkerboard 0.65 0.0 0.0 0.65 0.65 0.65 2.0
    transform { translate 0 -0.4 0 }
"""


def relmse(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref * ref + 1e-2)))


def test_thin_lens_render_matches_oracle(golden_meshes):
    st = pb.Stage(THIN, width=64, height=48)
    assert st.camera["kind"] == "thin_lens"
    scene = st.scene()
    want = load_stage(THIN, fixture_mesh_loader(golden_meshes), width=64, height=48)
    img = scene.render(st.camera, spp=32, max_depth=6, seed=2)
    ref = oracle.Scene(want, np.float32).render(want["camera"], 32, 6, seed=2)
    assert relmse(img, ref) < 5e-3
    # the lens blurs: the pinhole render of the same scene differs
    pin = dict(st.camera)
    pin.pop("kind")
    sharp = scene.render(pin, spp=32, max_depth=6, seed=2)
    assert relmse(sharp, img) > 1e-3


def test_thin_lens_of_radius_zero_is_a_pinhole_up_to_rounding(golden_meshes):
    st = pb.Stage(THIN.replace("radius 0.08", "radius 0"), width=48, height=36)
    scene = st.scene()
    pin = dict(st.camera)
    pin.pop("kind")
    a = scene.render(st.camera, spp=4, max_depth=1, seed=5, integrator="normal")
    b = scene.render(pin, spp=4, max_depth=1, seed=5, integrator="normal")
    assert np.abs(a - b).mean() < 1e-3


# many_spheres.stage (445 objects) takes the persistent extend walk, the others one thread per path
@pytest.mark.parametrize("name", ["default.stage", "cornell_box_canonical.stage", "cube_mesh.stage",
                                  "many_spheres.stage"])
def test_normal_integrator_matches_oracle(name, golden_meshes, mesh_dir):
    opts = dict(width=64, height=48, fov_deg=60.0, far=2000.0)
    st = pb.Stage(stage_text(name), base_dir=mesh_dir, **opts)
    want = load_stage(stage_text(name), fixture_mesh_loader(golden_meshes), **opts)
    img = st.scene().render(st.camera, spp=4, max_depth=5, seed=3, integrator="normal")
    ref = oracle.Scene(want, np.float32).render(want["camera"], 4, 5, seed=3, integrator="normal")
    assert np.all((img >= 0) & (img <= 1.0 + 1e-6))
    np.testing.assert_allclose(img, ref, rtol=0, atol=1e-5)


def test_cli_renders_a_scene_file(tmp_path, mesh_dir):
    stage = tmp_path / "scene.stage"
    stage.write_text(stage_text("cornell_box_canonical.stage"))
    out = tmp_path / "out.png"
    cli = os.path.join(ROOT, "pbrt_b200", "pbrt")
    r = subprocess.run([cli, "--input", str(stage), "--output", str(out), "--fov", "60", "--far", "2000",
                        "--output_width", "40", "--output_height", "30", "--samples_ppx", "8", "--max_depth", "4",
                        "--threads", "8", "--seed", "7"], capture_output=True, text=True, cwd=mesh_dir)
    assert r.returncode == 0, r.stderr
    got = read_png(str(out))
    scene, cam = pb.load_scene(stage_text("cornell_box_canonical.stage"), base_dir=mesh_dir, width=40, height=30,
                               fov_deg=60.0, far=2000.0)
    film = scene.render(cam, spp=8, max_depth=4, seed=7)
    np.testing.assert_array_equal(got, pb.film_to_rgba8(film))
