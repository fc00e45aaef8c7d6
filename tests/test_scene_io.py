"""Scene files, checkpoints and particle export.

- The reference's JSON scenes (SceneLoader) map onto AsimSceneDesc; a file describing the
  benchmark dam break gives the same seeded particles as the built-in description.
- A checkpoint holds everything a step reads from the previous one: a handle loaded from it
  continues bit-identically.
- The particle export (Scene::ExportParticles' Partio branch) writes FLUID particles with
  position in grid units, v and id, under the frame-numbered name.
"""
import json
import os

import numpy as np
import pytest

from ariel_b200 import _abi as A
from ariel_b200.flipsim import Batch, state_bytes
from ariel_b200.sceneloader import SceneError, load_scene

from helpers import assert_bits, dambreak, params


def _scene_json(n=64, rotation=None, meshfile=None, dim=None):
    box = {"id": "tank", "mesh_gen": "box", "point0": {"x": 0, "y": 0, "z": 0},
           "point1": {"x": 0.4 * n, "y": 0.6 * n, "z": 1.0 * n}}
    ball = {"id": "ball", "mesh_gen": "sphere", "center": {"x": 0, "y": 0, "z": 0}, "radius": 0.15 * n}
    moved = {"id": "moved", "translation": {"x": 0.6 * n, "y": 0.3 * n, "z": 0.5 * n}}
    if rotation:
        moved["rotation"] = rotation
    return {
        "settings": [{"density": 0.5, "step_size": 1.0 / 480.0,
                      "dim": dim or {"x": n, "y": n, "z": n}, "partio_output": "out/particles.geo"}],
        "camera": [{"resolution": {"x": 640, "y": 480}}],
        "globalforces": [{"x": 0.0, "y": -9.8, "z": 0.0}],
        "transforms": [{"id": "identity"}, moved],
        "meshfiles": [meshfile or box, ball],
        "geoms": [{"id": "water", "type": "mesh", "geom_frames": ["tank"], "transform_frames": ["identity"]},
                  {"id": "rock", "type": "mesh", "geom_frames": ["ball"], "transform_frames": ["moved"]}],
        "sim": [{"geom": "water", "type": "liquid"}, {"geom": "rock", "type": "solid"}],
    }


def test_scene_file_matches_builtin_description(tmp_path):
    p = tmp_path / "dambreak.json"
    p.write_text(json.dumps(_scene_json(64)))
    d, info = load_scene(str(p))
    ref = A.scene_dambreak(64, liquid_hi=(0.4, 0.6, 1.0), dt=1.0 / 480.0, seed=1, jitter=0.0,
                           spheres=[((0.6, 0.3, 0.5), 0.15)])
    assert info["dim"] == 64 and info["partio_output"] == "out/particles.geo"
    assert d.dim == ref.dim and d.density == ref.density and d.stepsize == ref.stepsize
    assert d.n_forces == 1 and abs(d.forces[0][1] + 9.8) < 1e-6
    assert d.n_liquid == 1 and d.n_solid == 1 and d.jitter == 0.0
    for a in range(3):
        assert abs(d.liquid[0].hi[a] - ref.liquid[0].hi[a]) < 1e-7
        assert abs(d.solid[0].center[a] - ref.solid[0].center[a]) < 1e-7
    assert abs(d.solid[0].radius - ref.solid[0].radius) < 1e-7
    # the seeded lattice (host-side) is the same: equal device footprints, particle for particle
    prm = params(precision=A.PREC_MIXED)
    assert state_bytes([d], prm) == state_bytes([ref], prm)


@pytest.mark.parametrize("bad", ["rotation", "file", "grid"])
def test_scene_file_refuses_what_it_cannot_represent(tmp_path, bad):
    kw = {"rotation": dict(rotation={"x": 0, "y": 30, "z": 0}),
          "file": dict(meshfile={"id": "tank", "file": "tank.obj"}),
          "grid": dict(dim={"x": 64, "y": 32, "z": 64})}[bad]
    p = tmp_path / "bad.json"
    p.write_text(json.dumps(_scene_json(64, **kw)))
    # (the "file" case: a liquid read from an OBJ file; only box liquids are seeded)
    (tmp_path / "tank.obj").write_text(_CUBE_OBJ)
    with pytest.raises(SceneError):
        load_scene(str(p))


_CUBE_OBJ = """# unit cube, quads
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
v 0 0 1
v 1 0 1
v 1 1 1
v 0 1 1
f 1 4 3 2
f 5 6 7 8
f 1 2 6 5
f 2 3 7 6
f 3 4 8 7
f 4 1 5 8
"""


def test_scene_file_mesh_solids(tmp_path):
    """A solid read from an OBJ file (translated and scaled) and a box solid become static solid
    meshes of the scene; the sphere stays analytic."""
    from ariel_b200.sceneloader import read_obj
    (tmp_path / "rock.obj").write_text(_CUBE_OBJ)
    v, t = read_obj(str(tmp_path / "rock.obj"))
    assert len(v) == 8 and len(t) == 12
    root = _scene_json(64)
    root["meshfiles"].append({"id": "rockfile", "file": "rock.obj"})
    root["meshfiles"].append({"id": "slab", "mesh_gen": "box", "point0": {"x": 40, "y": 0, "z": 10},
                              "point1": {"x": 50, "y": 8, "z": 20}})
    root["transforms"].append({"id": "placed", "translation": {"x": 44, "y": 10, "z": 40},
                               "scale": {"x": 6, "y": 6, "z": 6}})
    root["geoms"].append({"id": "r2", "type": "mesh", "geom_frames": ["rockfile"], "transform_frames": ["placed"]})
    root["geoms"].append({"id": "s2", "type": "mesh", "geom_frames": ["slab"], "transform_frames": ["identity"]})
    root["sim"] += [{"geom": "r2", "type": "solid"}, {"geom": "s2", "type": "solid"}]
    p = tmp_path / "meshes.json"
    p.write_text(json.dumps(root))
    d, info = load_scene(str(p))
    assert d.n_solid == 1 and d.n_mesh == 2 and len(info["meshes"]) == 2
    m = info["meshes"][0]
    assert abs(m.scale - 6.0 / 64) < 1e-7 and abs(float(m.translate[0]) - 44.0 / 64) < 1e-7
    prm = params(precision=A.PREC_MIXED)
    base = A.scene_dambreak(64, liquid_hi=(0.4, 0.6, 1.0), dt=1.0 / 480.0, seed=1, jitter=0.0,
                            spheres=[((0.6, 0.3, 0.5), 0.15)])
    assert state_bytes([d], prm) > state_bytes([base], prm)  # the meshes' trees and their solids


def test_native_loader_reads_json_as_the_reference_files_write_it(tmp_path):
    """The library's own JSON reader: escapes in ids and paths, exponents, a repeated key (the
    last value counts, as Python's json keeps it), numbers given as strings, and the same scene
    whether read from the file or from its text."""
    from ariel_b200.sceneloader import scene_from_json
    text = json.dumps(_scene_json(64)).replace('"tank"', '"t\\u00e4nk"')  # an escaped id, used twice
    text = text.replace('"step_size": 0.0020833333333333333', '"step_size": 2.0833333333333333e-3, "step_size": "0.0020833333333333333"')
    p = tmp_path / "escaped.json"
    p.write_text(text)
    d, info = load_scene(str(p))
    ref, _ = scene_from_json(_scene_json(64))
    assert bytes(d) == bytes(ref)
    assert info["step_size"] == 1.0 / 480.0
    d2, _ = scene_from_json(json.loads(text))
    assert bytes(d2) == bytes(d)


@pytest.mark.parametrize("bad", ["json", "unknown_mesh", "unknown_geom", "too_many_meshes", "missing_file"])
def test_native_loader_refusals(tmp_path, bad):
    from ariel_b200.sceneloader import scene_from_json
    root = _scene_json(64)
    if bad == "unknown_mesh":
        root["geoms"][0]["geom_frames"] = ["nothing"]
    elif bad == "unknown_geom":
        root["sim"][0]["geom"] = "nothing"
    elif bad == "too_many_meshes":
        for k in range(A.MAX_MESHES + 1):
            root["meshfiles"].append({"id": "b%d" % k, "mesh_gen": "box", "point0": {"x": k, "y": 0, "z": 0},
                                      "point1": {"x": k + 1, "y": 1, "z": 1}})
            root["geoms"].append({"id": "g%d" % k, "type": "mesh", "geom_frames": ["b%d" % k],
                                  "transform_frames": ["identity"]})
            root["sim"].append({"geom": "g%d" % k, "type": "solid"})
    elif bad == "missing_file":
        root["meshfiles"].append({"id": "gone", "file": "gone.obj"})
    if bad == "json":
        p = tmp_path / "broken.json"
        p.write_text(json.dumps(root)[:-3])
        with pytest.raises(SceneError, match="JSON"):
            load_scene(str(p))
    else:
        with pytest.raises(SceneError):
            scene_from_json(root, base_dir=str(tmp_path))
    with pytest.raises(SceneError, match="cannot read"):
        load_scene(str(tmp_path / "no_such_scene.json"))


def test_native_loader_error_buffer(tmp_path):
    """The reason is cut to the caller's buffer (NUL-terminated), and no buffer is needed."""
    import ctypes as C
    from ariel_b200 import _lib
    L = _lib.lib()
    d, info = A.AsimSceneDesc(), A.AsimSceneInfo()
    text = json.dumps(_scene_json(64, rotation={"x": 0, "y": 30, "z": 0})).encode()
    buf = C.create_string_buffer(b"#" * 16, 16)
    assert L.ariel_scene_parse(text, b".", 0.0, 1, C.byref(d), C.byref(info), buf, 8) == A.ARIEL_ERR_INVALID_ARG
    assert buf.raw[:8] == b"rotated\0" and buf.raw[8:] == b"#" * 8
    assert L.ariel_scene_parse(text, b".", 0.0, 1, C.byref(d), None, None, 0) == A.ARIEL_ERR_INVALID_ARG
    assert L.ariel_scene_parse(None, b".", 0.0, 1, C.byref(d), None, None, 0) == A.ARIEL_ERR_INVALID_ARG
    ok = json.dumps(_scene_json(64)).encode()
    assert L.ariel_scene_parse(ok, None, 0.0, 1, C.byref(d), None, None, 0) == A.ARIEL_OK
    assert d.dim == 64 and d.n_liquid == 1


def test_cpp_host_loads_a_scene_file(tmp_path):
    """ariel::LoadScene from a C++ program (tests/cpp/scene_load_main.cpp), no GPU needed: the
    same description as the Python loader, mesh solids registered, and a refusal's reason."""
    import subprocess
    from test_cpp_wrapper import _build
    (tmp_path / "rock.obj").write_text(_CUBE_OBJ)
    root = _scene_json(64)
    root["meshfiles"].append({"id": "rockfile", "file": "rock.obj"})
    root["transforms"].append({"id": "placed", "translation": {"x": 44, "y": 10, "z": 40},
                               "scale": {"x": 6, "y": 6, "z": 6}})
    root["geoms"].append({"id": "r2", "type": "mesh", "geom_frames": ["rockfile"], "transform_frames": ["placed"]})
    root["sim"].append({"geom": "r2", "type": "solid"})
    good, bad = tmp_path / "scene.json", tmp_path / "rotated.json"
    good.write_text(json.dumps(root))
    bad.write_text(json.dumps(_scene_json(64, rotation={"x": 0, "y": 30, "z": 0})))
    r = subprocess.run([_build(tmp_path, "scene_load_main"), str(good), str(bad)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "dim 64 density 0.500 step 0.002083 partio out/particles.geo" in r.stdout
    assert ("liquids 1 box 0.400 0.600 1.000 solids 1 sphere 0.6000 0.3000 0.5000 r 0.1500 meshes 1 forces 1"
            in r.stdout), r.stdout
    assert "mesh 0 vertices 8 triangles 12 scale 0.093750" in r.stdout
    assert "refused: LoadScene(" in r.stdout and "rotated geometry" in r.stdout


@pytest.mark.gpu
def test_checkpoint_continues_bit_identically(tmp_path):
    descs = [dambreak(16, seed=1), dambreak(20, seed=3, spheres=[((0.6, 0.3, 0.5), 0.15)])]
    prm = params(precision=A.PREC_MIXED, stop=A.STOP_REL, tol=1e-5, graph=1)
    a = Batch(descs, prm)
    a.init()
    a.step(4)
    ck = tmp_path / "state.ck"
    a.checkpoint_save(ck)
    a.step(3)
    b = Batch(descs, prm)
    b.checkpoint_load(ck)
    assert b.stats(1).frame == 4
    b.step(3)
    for i in range(2):
        pa, pb = a.get_particles(i), b.get_particles(i)
        assert_bits("scene %d pos" % i, pb["pos"], pa["pos"])
        assert_bits("scene %d vel" % i, pb["vel"], pa["vel"])
        assert_bits("scene %d P" % i, b.get_grid(A.GRID_P, i), a.get_grid(A.GRID_P, i))
    other = Batch([dambreak(16, seed=2)], prm)
    with pytest.raises(Exception):
        other.checkpoint_load(ck)
    for h in (a, b, other):
        h.close()


@pytest.mark.gpu
def test_particle_export(tmp_path):
    d = dambreak(16, seed=1, spheres=[((0.6, 0.3, 0.5), 0.15)])
    b = Batch([d], params())
    b.init()
    b.step(2)
    path = b.export_particles(tmp_path / "parts.geo", 7)
    assert os.path.basename(path) == "parts.0007.geo"
    st = b.get_particles()
    b.close()
    fl = st["type"] == A.FLUID
    lines = open(path).read().splitlines()
    assert lines[0] == "PGEOMETRY V5"
    assert lines[1] == "NPoints %d NPrims 1" % fl.sum()
    rows = [l for l in lines if l.endswith(")") and "(" in l]
    assert len(rows) == fl.sum()
    pos = np.array([[float(x) for x in r.split("(")[0].split()[:3]] for r in rows], np.float32)
    rest = np.array([[float(x) for x in r.split("(")[1].rstrip(")").split()] for r in rows])
    np.testing.assert_array_equal(pos, st["pos"][fl] * np.float32(16))
    np.testing.assert_array_equal(rest[:, :3].astype(np.float32), st["vel"][fl])
    np.testing.assert_array_equal(rest[:, 3], np.arange(fl.sum()))
    # the same file gzip-compressed for a ".geo.gz" path, frame number before ".geo.gz"
    import gzip
    b = Batch([d], params())
    b.init()
    b.step(2)
    gzpath = b.export_particles(tmp_path / "parts.geo.gz", 7)
    b.close()
    assert os.path.basename(gzpath) == "parts.0007.geo.gz"
    assert gzip.open(gzpath, "rt").read().splitlines() == lines
