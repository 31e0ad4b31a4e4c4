"""rkscene ingestion on the host (prt_scene_file_load): the loader against files written by the
reference's own rkscene::save (through the oracle), instances, default materials, and the
errors rkscene::load reports.

Exact bars: geometry arrays, textures and the material fields the reference's writer keeps are
equal to the source scene's bit for bit; flattened instances equal the affine map of the
positions (and the inverse transpose for normals) to float rounding.
"""
import json

import numpy as np
import pytest

import prt_cuda
import prt_scenes
import prt_types as T

REF = pytest.importorskip("ref")


def reference_written(scene, tmp_path):
    if not REF.ref_available():
        pytest.skip("oracle/_ref is not built")
    return REF.write_rkscene(scene, tmp_path)


SCENES = {
    "cornell": lambda: prt_scenes.cornell(seed=0, width=16, height=16),
    "textured": lambda: prt_scenes.cornell_inverse(seed=0, width=16, height=16, tex_size=32)[0],
    "lobes": lambda: prt_scenes.cornell_lobes(seed=0, width=16, height=16),
    "terrain": lambda: prt_scenes.terrain(seed=1, grid=64, n_spheres=8, width=16, height=16, spp=1),
}


@pytest.mark.parametrize("name", list(SCENES))
def test_reference_written_file_loads_exactly(name, tmp_path):
    s = SCENES[name]()
    r = prt_cuda.SceneFile(reference_written(s, tmp_path))
    meshes = r.meshes()
    assert len(meshes) == len(s.meshes)
    for a, b in zip(meshes, s.meshes):
        assert np.array_equal(a["positions"], b["positions"])
        assert np.array_equal(a["indices"], b["indices"])
        for key in ("normals", "texcoords"):
            assert (a[key] is None) == (b[key] is None)
            if b[key] is not None:
                assert np.array_equal(a[key], b[key])
        assert a["material"] == b["material"]
    for a, b in zip(r.textures(), s.textures):
        assert np.array_equal(a, b)
    mats = r.materials()
    assert len(mats) == len(s.materials)
    for a, b in zip(mats, s.materials):
        for f in ("base_color_texture", "metalness", "specular_weight", "transmission_weight", "coat_weight",
                  "sheen_weight", "emission_luminance", "thin_walled", "opacity"):
            assert getattr(a, f) == getattr(b, f), f
        if not (b.metalness == 0.0 and b.transmission_weight == 1.0):
            assert list(a.base_color) == list(b.base_color)
        if b.emission_luminance != 0.0:
            assert list(a.emission_color) == list(b.emission_color)
    r.close()


def test_own_writer_round_trip(tmp_path):
    s = prt_scenes.cornell_inverse(seed=2, width=16, height=16, tex_size=16)[0]
    r = prt_cuda.SceneFile(prt_scenes.write_rkscene(s, tmp_path / "room.rkscene"))
    for a, b in zip(r.meshes(), s.meshes):
        assert np.array_equal(a["positions"], b["positions"]) and np.array_equal(a["indices"], b["indices"])
    assert all(bytes(a) == bytes(b) for a, b in zip(r.materials(), s.materials))
    for a, b in zip(r.textures(), s.textures):
        assert np.array_equal(a, b)


def small_scene():
    s = prt_scenes.Scene()
    m = s.add_material(T.material(base_color=(0.5, 0.6, 0.7)))
    quad_p = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    quad_i = np.array([[0, 1, 2], [0, 2, 3]], np.int32)
    s.add_mesh(quad_p, quad_i, m, normals=np.tile([0, 0, 1], (4, 1)))
    s.add_mesh(quad_p + 2.0, quad_i, m)
    return s


def test_instances_are_flattened(tmp_path):
    s = small_scene()
    rng = np.random.default_rng(3)
    xfs = []
    for _ in range(3):
        lin = rng.normal(size=(3, 3)).astype(np.float32) + 2 * np.eye(3, dtype=np.float32)
        xfs.append(np.concatenate([lin, rng.normal(size=(3, 1)).astype(np.float32)], 1))
    path = prt_scenes.write_rkscene(s, tmp_path / "inst.rkscene", objects=[([0, 1], xfs)])
    meshes = prt_cuda.SceneFile(path).meshes()
    assert len(meshes) == 6  # instance-major: (inst 0: geom 0, geom 1), (inst 1: ...), ...
    for k, mesh in enumerate(meshes):
        xf, src = xfs[k // 2], s.meshes[k % 2]
        want = src["positions"].astype(np.float64) @ xf[:, :3].T.astype(np.float64) + xf[:, 3]
        assert np.allclose(mesh["positions"], want, rtol=1e-5, atol=1e-5)
        assert np.array_equal(mesh["indices"], src["indices"])
        if src["normals"] is not None:
            nt = src["normals"].astype(np.float64) @ np.linalg.inv(xf[:, :3].astype(np.float64))
            assert np.allclose(mesh["normals"], nt, rtol=1e-4, atol=1e-5)
        else:
            assert mesh["normals"] is None


def test_missing_and_unknown_materials_get_the_default(tmp_path):
    s = small_scene()
    s.meshes[0]["material"] = -1
    s.meshes[1]["material"] = 7
    r = prt_cuda.SceneFile(prt_scenes.write_rkscene(s, tmp_path / "d.rkscene"))
    mats = r.materials()
    assert len(mats) == 2 and mats[1].model == T.PRT_MATERIAL_PRINCIPLED
    assert [m["material"] for m in r.meshes()] == [1, 1]


def edit(path, fn):
    doc = json.loads(path.read_text())
    fn(doc)
    path.write_text(json.dumps(doc))
    return path


@pytest.mark.parametrize("change,kind,text", [
    (lambda d: d.pop("buffers"), ValueError, "no buffers"),
    (lambda d: d["buffers"].append(d["buffers"][0]), ValueError, "single buffer"),
    (lambda d: d["geometries"][0]["positions"].update(count=10 ** 6), ValueError, "out of bounds"),
    (lambda d: d["geometries"][0]["positions"].update(type="float2"), ValueError, "buffer type"),
    (lambda d: d["geometries"][0].update(type="curve"), ValueError, "geom type"),
    (lambda d: d.update(lights=[{"type": "spot"}]), ValueError, "light type"),
    (lambda d: d["materials"][0].update(specularRoughness="rough.pfm"), ValueError, "baseColor only"),
    (lambda d: d["materials"][0].update(baseColor={"image": "t.pfm", "transform": {"scale": [2, 2]}}), ValueError,
     "transform"),
    (lambda d: d["materials"][0].update(normal={"image": "n.pfm"}), ValueError, "normal"),
    (lambda d: d["materials"][0].update(baseColor=0.5), ValueError, "array of 3"),
    (lambda d: d["objects"][0].update(geometries=[5]), ValueError, "out of range"),
    (lambda d: d["buffers"][0].update(uri="missing.rkbin"), OSError, "failed to open"),
    (lambda d: d["materials"][0].update(baseColor="missing.pfm"), OSError, "failed to open image"),
])
def test_errors(tmp_path, change, kind, text):
    path = edit(prt_scenes.write_rkscene(small_scene(), tmp_path / "e.rkscene"), change)
    with pytest.raises(kind, match=text):
        prt_cuda.SceneFile(path)


def test_index_out_of_range(tmp_path):
    s = small_scene()
    s.meshes[1]["indices"] = s.meshes[1]["indices"] + 10
    with pytest.raises(ValueError, match="index out of range"):
        prt_cuda.SceneFile(prt_scenes.write_rkscene(s, tmp_path / "i.rkscene"))


@pytest.mark.parametrize("text", ["", "{", "[1,]", '{"a" 1}', '{"a": tru}', '{"a": "\\x"}', '{"a": 01}',
                                  '{"a": "\\ud800"}', "{} {}"])
def test_malformed_json(tmp_path, text):
    p = tmp_path / "bad.rkscene"
    p.write_text(text)
    with pytest.raises(ValueError, match="invalid JSON|document"):
        prt_cuda.SceneFile(p)


def test_json_details(tmp_path):
    path = prt_scenes.write_rkscene(small_scene(), tmp_path / "j.rkscene")
    doc = json.loads(path.read_text())
    doc["name"] = "café \U0001F600 \"q\""
    doc["materials"][0]["name"] = "m\\u00e9"
    doc["lights"] = None
    doc["extra"] = {"nested": [1, 2.5e-3, -0.0, True, False, None]}
    path.write_text(json.dumps(doc, ensure_ascii=True))
    assert len(prt_cuda.SceneFile(path).meshes()) == 2


def test_gzip_buffers_are_reported(tmp_path):
    path = prt_scenes.write_rkscene(small_scene(), tmp_path / "z.rkscene")
    binp = path.with_suffix(".rkbin")
    binp.rename(binp.with_name(binp.name + ".gz"))
    with pytest.raises(OSError, match="gzip"):
        prt_cuda.SceneFile(path)


# -- .mesh + .mtl ------------------------------------------------------------------------------

def test_mesh_file_loads_exactly(tmp_path):
    s = prt_scenes.cornell_inverse(seed=0, width=16, height=16, tex_size=16)[0]
    f = prt_cuda.SceneFile(prt_scenes.write_mesh(s, tmp_path / "room.mesh"))
    mats = f.materials()
    # write_mesh puts the first non-emissive material first, then the emissive ones.
    n = len(s.materials)
    emissive = [i for i in range(n) if s.materials[i].emission_luminance > 0.0]
    others = [i for i in range(n) if i not in emissive]
    order = others[:1] + emissive + others[1:]
    assert len(mats) == n
    assert mats[0].model == T.PRT_MATERIAL_MISS  # id 0: the stream renderer's miss bucket
    for k in range(1, n):
        assert bytes(mats[k]) == bytes(s.materials[order[k]]), k
    # One mesh per material, the source triangles in order, shared vertex arrays.
    P = np.concatenate([m["positions"] for m in s.meshes])
    base = np.cumsum([0] + [m["positions"].shape[0] for m in s.meshes])
    meshes = f.meshes()
    for mesh in meshes:
        assert np.array_equal(mesh["positions"], P)
        src = [(k, m) for k, m in enumerate(s.meshes) if order[mesh["material"]] == m["material"]]
        want = np.concatenate([m["indices"] + base[k] for k, m in src])
        assert np.array_equal(mesh["indices"], want)
    assert sum(m["indices"].shape[0] for m in meshes) == s.tri_count
    for a, b in zip(f.textures(), s.textures):
        assert np.array_equal(a, b)


def test_mesh_obj_materials_map_to_principled(tmp_path):
    s = small_scene()
    s.meshes[1]["material"] = s.add_material(T.material(base_color=(0.9, 0.9, 0.9)))
    path = prt_scenes.write_mesh(s, tmp_path / "obj.mesh")
    mtl = path.with_suffix(".mtl")
    mtl.write_text("newmtl mat0\nKd 0.2 0.3 0.4\n"
                   "newmtl mat1\nKd 0.5 0.6 0.7\nNs 62\nKs 1 1 1\nTf 0.25 0.5 1\n")
    mats = prt_cuda.SceneFile(path).materials()
    m = mats[1]
    assert m.model == T.PRT_MATERIAL_PRINCIPLED
    assert np.allclose(list(m.base_color), [0.5, 0.6, 0.7])
    rough = np.sqrt(np.sqrt(np.float32(2.0) / (np.float32(62.0) + np.float32(2.0))))
    assert np.isclose(m.specular_roughness, rough, rtol=1e-6)
    f0 = np.float32(1.0) * np.float32(0.08)
    assert np.isclose(m.specular_ior, (1 + np.sqrt(f0)) / (1 - np.sqrt(f0)), rtol=1e-6)
    assert m.transmission_weight == 1.0 and np.allclose(list(m.transmission_color), [0.75, 0.5, 0.0])


def test_mesh_errors(tmp_path):
    s = small_scene()
    path = prt_scenes.write_mesh(s, tmp_path / "e.mesh")
    data = path.read_bytes()
    bad = tmp_path / "bad.mesh"
    bad.write_bytes(b"\x00\x00\x00\x00" + data[4:])
    with pytest.raises(ValueError, match="blob ID"):
        prt_cuda.SceneFile(bad)
    bad.write_bytes(data[:40])
    with pytest.raises(OSError, match="end of stream"):
        prt_cuda.SceneFile(bad)
    path.with_suffix(".mtl").write_text("newmtl mat0\ntype CarPaint\n")
    with pytest.raises(ValueError, match="not supported"):
        prt_cuda.SceneFile(path)
    with pytest.raises(ValueError, match="unknown scene format"):
        prt_cuda.SceneFile(tmp_path / "x.obj")


def test_mesh_emissive_materials_must_come_first(tmp_path):
    """Scene::Scene needs the emissive materials at ids 1..k (render/scene.cpp:119-130)."""
    s = small_scene()
    s.add_material(T.material(base_color=(0.1, 0.2, 0.3)))
    s.add_material(T.material(emission_luminance=5.0))
    s.meshes[1]["material"] = 2
    path = prt_scenes.write_mesh(s, tmp_path / "l.mesh")  # the writer puts the emissive one at id 1
    assert len(prt_cuda.SceneFile(path).meshes()) == 2
    # Swap the library's definitions of ids 1 and 2: the emissive material now sits at id 2.
    text = path.with_suffix(".mtl").read_text()
    text = text.replace("newmtl mat1", "newmtl X").replace("newmtl mat2", "newmtl mat1").replace("newmtl X", "newmtl mat2")
    path.with_suffix(".mtl").write_text(text)
    with pytest.raises(ValueError, match="remapped"):
        prt_cuda.SceneFile(path)
