"""Reads the reference's JSON scene files into AsimSceneDesc (SceneLoader,
src/scene/sceneloader.cpp:11-131, 346-443).

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
the returned ``info["meshes"]`` must stay alive while handles are created from the scene.
Anything the path cannot represent -- liquids from meshes, animated meshes, rotations,
non-uniform scaling of spheres or meshes, geometry that appears after frame 0, non-cubic grids,
more boxes, spheres, meshes or forces than the ABI holds -- raises ``SceneError`` rather than
being approximated.  Camera settings are ignored (no viewer).
"""
import json
import os

from . import _abi as A


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


def _box_mesh(lo, hi):
    v = [[(lo, hi)[x][0], (lo, hi)[y][1], (lo, hi)[z][2]] for x in (0, 1) for y in (0, 1) for z in (0, 1)]
    i = lambda x, y, z: x * 4 + y * 2 + z
    quads = [(i(0, 0, 0), i(0, 1, 0), i(0, 1, 1), i(0, 0, 1)), (i(1, 0, 0), i(1, 0, 1), i(1, 1, 1), i(1, 1, 0)),
             (i(0, 0, 0), i(0, 0, 1), i(1, 0, 1), i(1, 0, 0)), (i(0, 1, 0), i(1, 1, 0), i(1, 1, 1), i(0, 1, 1)),
             (i(0, 0, 0), i(1, 0, 0), i(1, 1, 0), i(0, 1, 0)), (i(0, 0, 1), i(0, 1, 1), i(1, 1, 1), i(1, 0, 1))]
    tris = []
    for a, b, c, d in quads:
        tris += [[a, b, c], [a, c, d]]
    return v, tris


def _vec(obj, key, default):
    if key not in obj:
        return list(default)
    v = obj[key]
    return [float(v.get("x", 0.0)), float(v.get("y", 0.0)), float(v.get("z", 0.0))]


def load_scene(path, jitter=0.0, seed=1):
    """Returns (AsimSceneDesc, info) for the scene file at `path`.  `info` holds the grid size,
    density, step size and the output paths of the settings block.  The reference seeds liquid
    particles at lattice-cell centres, so `jitter` defaults to 0."""
    with open(path) as f:
        root = json.load(f)
    return scene_from_json(root, jitter=jitter, seed=seed, base_dir=os.path.dirname(os.path.abspath(path)))


def scene_from_json(root, jitter=0.0, seed=1, base_dir=""):
    settings = root.get("settings", [{}])
    settings = settings[0] if settings else {}
    density = float(settings.get("density", 0.5))
    step = float(settings.get("step_size", 0.005))
    dim = settings.get("dim", {"x": 32, "y": 32, "z": 32})
    dims = [int(dim.get("x", 32)), int(dim.get("y", 32)), int(dim.get("z", 32))]
    if not (dims[0] == dims[1] == dims[2]):
        raise SceneError("non-cubic grid %s: the step treats every axis as the largest one" % dims)
    n = dims[0]

    transforms = {}
    for t in root.get("transforms", []):
        if "id" not in t or t["id"] in transforms:
            continue  # the reference skips nodes without an id and repeated ids
        transforms[t["id"]] = (_vec(t, "translation", (0, 0, 0)), _vec(t, "rotation", (0, 0, 0)),
                               _vec(t, "scale", (1, 1, 1)))
    meshes = {}
    for m in root.get("meshfiles", []):
        if "id" not in m or m["id"] in meshes:
            continue
        if "file" in m:
            meshes[m["id"]] = ("obj",) + tuple(read_obj(os.path.join(base_dir, m["file"])))
            continue
        gen = m.get("mesh_gen")
        if gen == "box":
            meshes[m["id"]] = ("box", _vec(m, "point0", (0, 0, 0)), _vec(m, "point1", (0, 0, 0)))
        elif gen == "sphere":
            meshes[m["id"]] = ("sphere", _vec(m, "center", (0, 0, 0)), float(m.get("radius", 0.0)))
        else:
            raise SceneError("mesh generator %r is not supported" % gen)
    if root.get("animatedmeshes"):
        raise SceneError("animated meshes are not supported")
    geoms = {}
    for g in root.get("geoms", []):
        if "id" not in g or g["id"] in geoms:
            continue
        if g.get("type") != "mesh":
            raise SceneError("geom type %r is not supported" % g.get("type"))
        frames, tframes = g.get("geom_frames", []), g.get("transform_frames", [])
        if not frames or not tframes:
            raise SceneError("geom %r has no frame-0 mesh or transform" % g["id"])
        geoms[g["id"]] = dict(mesh=meshes[frames[0]], transform=transforms[tframes[0]],
                              offset=int(g.get("frame_offset", 0)))

    def placed(geom):
        (tx, ty, tz), rot, scale = geom["transform"]
        if any(abs(r) > 0.0 for r in rot):
            raise SceneError("rotated geometry is not supported (boxes and spheres stay axis-aligned)")
        if any(s <= 0.0 for s in scale):
            raise SceneError("non-positive scale")
        mesh = geom["mesh"]
        t = (tx, ty, tz)
        if mesh[0] == "obj":
            if not (scale[0] == scale[1] == scale[2]):
                raise SceneError("non-uniformly scaled mesh")
            return ("obj", mesh[1], mesh[2], t, scale[0])
        if mesh[0] == "box":
            lo = [t[a] + scale[a] * min(mesh[1][a], mesh[2][a]) for a in range(3)]
            hi = [t[a] + scale[a] * max(mesh[1][a], mesh[2][a]) for a in range(3)]
            return ("box", lo, hi)
        if not (scale[0] == scale[1] == scale[2]):
            raise SceneError("non-uniformly scaled sphere")
        return ("sphere", [t[a] + scale[a] * mesh[1][a] for a in range(3)], scale[0] * mesh[2])

    d = A.AsimSceneDesc()
    d.dim = n
    d.density = density
    d.stepsize = step
    forces = root.get("globalforces", [])
    if len(forces) > A.MAX_FORCES:
        raise SceneError("more than %d global forces" % A.MAX_FORCES)
    d.n_forces = len(forces)
    for i, fo in enumerate(forces):
        for a, key in enumerate("xyz"):
            d.forces[i][a] = float(fo.get(key, 0.0))
    nl = ns = 0
    meshes_alive = []
    for node in root.get("sim", []):
        geom = geoms[node["geom"]]
        if geom["offset"] != 0:
            raise SceneError("geometry that appears after frame 0 is not supported")
        kind, *shape = placed(geom)
        if node.get("type") == "liquid":
            if kind != "box":
                raise SceneError("only box liquids are supported")
            if nl >= A.MAX_BOXES:
                raise SceneError("more than %d liquids" % A.MAX_BOXES)
            lo, hi = shape
            vel = _vec(node, "velocity", (0, 0, 0))
            for a in range(3):
                d.liquid[nl].lo[a] = lo[a] / n
                d.liquid[nl].hi[a] = hi[a] / n
                d.liquid[nl].vel[a] = vel[a]
            nl += 1
        elif node.get("type") == "solid":
            if kind == "sphere":
                if ns >= A.MAX_SPHERES:
                    raise SceneError("more than %d sphere solids" % A.MAX_SPHERES)
                c, r = shape
                for a in range(3):
                    d.solid[ns].center[a] = c[a] / n
                d.solid[ns].radius = r / n
                ns += 1
            else:
                # a box or OBJ solid: a static mesh in grid units, placed in the unit cube
                if d.n_mesh >= A.MAX_MESHES:
                    raise SceneError("more than %d mesh solids" % A.MAX_MESHES)
                from .flipsim import Mesh
                if kind == "box":
                    verts, tris = _box_mesh(*shape)
                    mesh = Mesh(verts, tris, translate=(0.0, 0.0, 0.0), scale=1.0 / n)
                else:
                    verts, tris, t, sc = shape
                    mesh = Mesh(verts, tris, translate=[x / n for x in t], scale=sc / n)
                meshes_alive.append(mesh)
                A.add_mesh(d, mesh.id)
        else:
            raise SceneError("sim node type %r is not supported" % node.get("type"))
    d.n_liquid = nl
    d.n_solid = ns
    d.seed = seed
    d.jitter = jitter
    info = {"dim": n, "density": density, "step_size": step,
            "partio_output": settings.get("partio_output", ""),
            "vdb_output": settings.get("vdb_output", ""), "mesh_output": settings.get("mesh_output", ""),
            "meshes": meshes_alive}
    return d, info
