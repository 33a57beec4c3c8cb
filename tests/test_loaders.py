"""Scene loaders (delta_ray_b200.loaders): Mitsuba .serialized meshes, OBJ
files and Mitsuba XML scenes.

The .serialized reader is checked against the reference's own reader
(load_serialized.cpp, compiled by `make -C oracle ref`) on files this test
writes, and on the reference's test scene when its sources are mounted."""
import glob
import importlib.util
import os

import numpy as np
import pytest

from conftest import ROOT
from refpath import reference_dir

REF_SCENES = os.path.join(reference_dir(), "test", "scenes")


def _reference_reader():
    cands = glob.glob(os.path.join(ROOT, "oracle", "_ref", "load_serialized*.so"))
    if not cands:
        pytest.skip("reference mesh reader not built (make -C oracle ref)")
    spec = importlib.util.spec_from_file_location("load_serialized", cands[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _meshes(rng):
    out = []
    for k, (nv, nt) in enumerate([(5, 3), (9, 7), (4, 2)]):
        v = rng.normal(size=(nv, 3)).astype(np.float32)
        f = rng.integers(0, nv, size=(nt, 3)).astype(np.int32)
        n = rng.normal(size=(nv, 3)).astype(np.float32) if k != 1 else None
        uv = rng.uniform(size=(nv, 2)).astype(np.float32) if k != 2 else None
        out.append((f, v, uv, n, f"mesh{k}"))
    return out


@pytest.mark.parametrize("version,double", [(4, False), (4, True), (3, False)])
def test_serialized_roundtrip_and_reference_reader(tmp_path, version, double):
    from delta_ray_b200.loaders import load_serialized, write_serialized
    meshes = _meshes(np.random.default_rng(version + 10 * double))
    path = str(tmp_path / "m.serialized")
    write_serialized(path, meshes, version=version, double_precision=double)
    ref = _reference_reader()
    for i, (f, v, uv, n, _) in enumerate(meshes):
        idx, vtx, uvs, nrm = load_serialized(path, i)
        assert np.array_equal(idx, f)
        assert np.array_equal(vtx, v)
        assert (uvs.shape[0] == 0) if uv is None else np.array_equal(uvs, uv)
        assert (nrm.shape[0] == 0) if n is None else np.array_equal(nrm, n)
        r_idx, r_vtx, r_uv, r_n = ref.load_serialized(path, i)
        assert np.array_equal(idx, np.asarray(r_idx))
        assert np.array_equal(vtx, np.asarray(r_vtx))
        if uv is not None:
            assert np.array_equal(uvs, np.asarray(r_uv))
        if n is not None:
            assert np.array_equal(nrm, np.asarray(r_n))


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_SCENES, "bunny_box.serialized")),
                    reason="reference test scenes not mounted")
def test_serialized_matches_reference_reader_on_reference_scene():
    from delta_ray_b200.loaders import load_serialized
    ref = _reference_reader()
    path = os.path.join(REF_SCENES, "bunny_box.serialized")
    for i in range(6):
        mine = load_serialized(path, i)
        theirs = ref.load_serialized(path, i)
        for a, b in zip(mine, theirs):
            b = np.asarray(b)
            if b.size == 0:
                assert a.shape[0] == 0
            else:
                assert np.array_equal(a, b)


def test_obj_loader(tmp_path):
    from delta_ray_b200.loaders import load_obj
    path = tmp_path / "q.obj"
    path.write_text("""# a quad and a triangle
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
vt 0 0
vt 1 0
vt 1 1
vt 0 1
vn 0 0 1
f 1/1/1 2/2/1 3/3/1 4/4/1
f -4/-4/-1 -2/-2/-1 -1/-1/-1
""")
    idx, v, uv, n = load_obj(str(path))
    assert idx.tolist() == [[0, 1, 2], [0, 2, 3], [0, 2, 3]]  # the second face reuses the first's vertices
    assert v.shape == (4, 3) and uv.shape == (4, 2) and n.shape == (4, 3)
    assert np.allclose(v[2], [1, 1, 0]) and np.allclose(uv[3], [0, 1])


def _write_scene(tmp_path):
    from delta_ray_b200.loaders import write_serialized
    ground_v = np.array([[-5, 0, -5], [5, 0, -5], [-5, 0, 5], [5, 0, 5]], np.float32)
    ground_f = np.array([[0, 2, 1], [1, 2, 3]], np.int32)
    box_v = np.array([[-1, 1, -1], [1, 1, -1], [0, 1, 1], [0, 2, 0]], np.float32)
    box_f = np.array([[0, 1, 3], [1, 2, 3], [2, 0, 3]], np.int32)
    write_serialized(str(tmp_path / "scene.serialized"), [(box_f, box_v, None, None, "box"),
                                                          (ground_f, ground_v, None, None, "ground")])
    (tmp_path / "scene.xml").write_text("""<?xml version='1.0' encoding='utf-8'?>
<scene version="0.5.0">
  <sensor type="perspective">
    <float name="fov" value="45"/>
    <transform name="toWorld">
      <lookat origin="0, 6, -6" target="0, 0, 0" up="0, 1, 0"/>
    </transform>
    <film type="hdrfilm">
      <integer name="width" value="24"/>
      <integer name="height" value="20"/>
    </film>
  </sensor>
  <bsdf type="diffuse" id="grey">
    <rgb name="reflectance" value="0.5 0.5 0.5"/>
  </bsdf>
  <bsdf type="twosided" id="red">
    <bsdf type="diffuse">
      <rgb name="reflectance" value="0.6, 0.1, 0.1"/>
      <rgb name="specular" value="0.2 0.2 0.2"/>
      <float name="roughness" value="0.3"/>
    </bsdf>
  </bsdf>
  <shape type="serialized">
    <string name="filename" value="scene.serialized"/>
    <integer name="shapeIndex" value="1"/>
    <ref name="bsdf" id="grey"/>
  </shape>
  <shape type="serialized">
    <string name="filename" value="scene.serialized"/>
    <integer name="shapeIndex" value="0"/>
    <transform name="toWorld">
      <translate x="0" y="0.25" z="0"/>
    </transform>
    <ref name="bsdf" id="red"/>
  </shape>
  <shape type="rectangle">
    <transform name="toWorld">
      <scale x="1" y="1" z="1"/>
      <matrix value="1 0 0 0  0 0 -1 5  0 1 0 0  0 0 0 1"/>
    </transform>
    <ref name="bsdf" id="grey"/>
    <emitter type="area">
      <spectrum name="radiance" value="15"/>
    </emitter>
  </shape>
</scene>
""")
    return str(tmp_path / "scene.xml")


def test_mitsuba_scene(tmp_path):
    from delta_ray_b200.loaders import load_mitsuba
    cam, materials, shapes, lights, res = load_mitsuba(_write_scene(tmp_path))
    assert res == [24, 20] and cam.resolution == [24, 20]
    assert len(materials) == 2 and materials[1].two_sided
    assert np.allclose(materials[1].diffuse_reflectance.numpy(), [0.6, 0.1, 0.1])
    assert np.allclose(materials[1].roughness.numpy(), [0.3])
    assert [s.mat_id for s in shapes] == [0, 1, 0]
    assert np.allclose(shapes[1].vertices.numpy()[3], [0, 2.25, 0])  # translated
    assert np.allclose(shapes[2].vertices.numpy()[:, 1], 5.0)         # the rectangle moved to y = 5
    assert len(lights) == 1 and lights[0].shape_id == 2
    assert np.allclose(lights[0].intensity.numpy(), [15, 15, 15])


def test_mitsuba_scene_renders_in_the_oracle(tmp_path):
    """A loaded scene goes through serialize_scene / the C ABI descriptors."""
    import oracle
    from delta_ray_b200.loaders import load_mitsuba
    from delta_ray_b200.workloads import Workload
    cam, materials, shapes, lights, res = load_mitsuba(_write_scene(tmp_path))
    wl = Workload("mitsuba", cam, materials, shapes, lights, res, 4, 1)
    o = oracle.oracle_render(wl, 3, np.ones((res[1], res[0], 3), np.float32), rng_mode=oracle.PHILOX)
    assert np.isfinite(o["image"]).all() and o["image"].max() > 0
    assert np.isfinite(o["grad"]).all() and np.abs(o["grad"]).max() > 0


@pytest.mark.gpu
def test_mitsuba_scene_gpu_matches_oracle(tmp_path):
    """A loaded scene on the CUDA library, forward and backward, against the
    oracle on the same Philox streams."""
    import oracle
    from delta_ray_b200.loaders import load_mitsuba
    from delta_ray_b200.workloads import Workload
    from conftest import assert_grad_parity, assert_image_parity
    from test_forward_gpu import product_scene
    import torch
    cam, materials, shapes, lights, res = load_mitsuba(_write_scene(tmp_path))
    wl = Workload("mitsuba", cam, materials, shapes, lights, res, 4, 1)
    W, H = res
    sc = product_scene(wl)
    img = sc.forward(W, H, 4, 1, 3).cpu().numpy()
    grad, _ = sc.backward(W, H, 4, 1, 3, torch.ones((H, W, 3), device="cuda"))
    o = oracle.oracle_render(wl, 3, np.ones((H, W, 3), np.float32), rng_mode=oracle.PHILOX)
    assert_image_parity(img, o["image"])
    assert_grad_parity(grad.cpu().numpy(), o["grad"])
    sc.close()
