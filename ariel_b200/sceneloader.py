"""Reads the reference's JSON scene files into AsimSceneDesc (SceneLoader,
src/scene/sceneloader.cpp:11-131, 346-443), through the library's native loader
(``ariel_scene_load`` / ``ariel_scene_parse``, csrc/sceneload.cu).

Supported, as the reference reads them:
- ``settings[0]``: ``density`` (default .5), ``step_size`` (.005), ``dim`` {x,y,z} (32 each;
  the grid must be cubic), ``partio_output`` (returned for ``ariel_export_particles``);
- ``globalforces``: [{x,y,z}], applied in order;
- ``transforms``: {id, translation, rotation, scale};
- ``meshfiles``: {id, mesh_gen: "box", point0, point1} and {id, mesh_gen: "sphere", center,
  radius} -- coordinates in grid cells, as the reference's mesh generators take them;
- ``geoms``: {id, type: "mesh", geom_frames, transform_frames, frame_offset, ...}: the geometry
  of frame 0 (its first mesh under its first transform);
- ``sim``: {geom, type: "liquid" | "solid", velocity}.

A liquid becomes an AsimBox.  A sphere solid becomes an analytic AsimSphere; a box solid and a
solid read from an OBJ file (``meshfiles`` {id, file}, src/geom/obj/obj.cpp) become static solid
meshes registered with the library (``ariel_mesh_create``, uniform scale and translation), so
the returned ``info["meshes"]`` (which own them) must stay alive while handles are created
from the scene.
Anything the path cannot represent -- liquids from meshes, animated meshes, rotations,
non-uniform scaling of spheres or meshes, geometry that appears after frame 0, non-cubic grids,
more boxes, spheres, meshes or forces than the ABI holds -- raises ``SceneError`` rather than
being approximated.  Camera settings are ignored (no viewer).
"""
import ctypes as C
import json
import os

from . import _abi as A
from ._lib import check, lib


class SceneError(ValueError):
    pass


def read_obj(path):
    """Vertices and triangles of an OBJ file (``v`` and ``f`` records; 1-based or negative
    indices, ``a/b/c`` forms; polygons split into fans, so a quad v0 v1 v2 v3 gives the two
    triangles the reference tests, Obj::QuadTest obj.cpp:344-352)."""
    verts, tris = [], []
    with open(path) as f:
        for line in f:
            parts = line.split()
            if not parts:
                continue
            if parts[0] == "v" and len(parts) >= 4:
                verts.append([float(parts[1]), float(parts[2]), float(parts[3])])
            elif parts[0] == "f" and len(parts) >= 4:
                idx = []
                for tok in parts[1:]:
                    i = int(tok.split("/")[0])
                    idx.append(i - 1 if i > 0 else len(verts) + i)
                for j in range(1, len(idx) - 1):
                    tris.append([idx[0], idx[j], idx[j + 1]])
    if not verts or not tris:
        raise SceneError("OBJ file %r has no triangles" % path)
    return verts, tris


def _finish(st, d, info, err):
    if st == A.ARIEL_ERR_INVALID_ARG:
        raise SceneError(err.value.decode(errors="replace") or "invalid scene")
    check(st, "ariel_scene_load")
    from .flipsim import Mesh
    meshes = [Mesh.adopt(d.mesh[i]) for i in range(d.n_mesh)]
    return d, {"dim": info.dim, "density": info.density, "step_size": info.step_size,
               "partio_output": info.partio_output.decode(), "vdb_output": info.vdb_output.decode(),
               "mesh_output": info.mesh_output.decode(), "meshes": meshes}


def load_scene(path, jitter=0.0, seed=1):
    """Returns (AsimSceneDesc, info) for the scene file at `path`.  `info` holds the grid size,
    density, step size, the output paths of the settings block and the scene's solid meshes.
    The reference seeds liquid particles at lattice-cell centres, so `jitter` defaults to 0."""
    d, info, err = A.AsimSceneDesc(), A.AsimSceneInfo(), C.create_string_buffer(512)
    st = lib().ariel_scene_load(os.fsencode(path), float(jitter), int(seed), C.byref(d), C.byref(info), err, 512)
    return _finish(st, d, info, err)


def scene_from_json(root, jitter=0.0, seed=1, base_dir=""):
    """The same for an already parsed scene (a dict); OBJ paths resolve against `base_dir`."""
    d, info, err = A.AsimSceneDesc(), A.AsimSceneInfo(), C.create_string_buffer(512)
    st = lib().ariel_scene_parse(json.dumps(root).encode(), os.fsencode(base_dir or "."), float(jitter), int(seed),
                                 C.byref(d), C.byref(info), err, 512)
    return _finish(st, d, info, err)
