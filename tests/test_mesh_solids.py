"""Static solid meshes (the reference's mesh solids, src/scene/scene.cpp:362-434 and
src/spatial/bvh.inl, generalising the analytic spheres of the solid constraints).

The CUDA library places every mesh of a scene in one bounding volume hierarchy; the oracle loops
over all triangles.  Both use the reference's ray-triangle test (src/geom/obj/obj.cpp:354-398),
the inside rule of Scene::CheckPointInsideSolidGeom (odd number of hits along +z,
scene.cpp:382-402) and tie-breaks by triangle order, so seeding, cell flags and every stage agree
bit for bit.  The closest surface point (the reference asks OpenVDB, levelset.cpp:175-193) is
the exact one on both sides.
"""
import numpy as np
import pytest

from ariel_b200 import _abi as A
from oracle.pyoracle import RefSim

from helpers import assert_bits, box_mesh, dambreak, icosphere, params, stage_parity

SPHERE_C, SPHERE_R = (0.6, 0.3, 0.5), 0.15


def _mesh_scene(n, kind, seed=7):
    desc = dambreak(n, seed=seed, hi=(0.35, 0.5, 1.0))
    if kind == "icosphere":
        v, t = icosphere(2)
        return desc, v, t, SPHERE_C, SPHERE_R
    v, t = box_mesh()
    return desc, v, t, (0.62, 0.25, 0.45), 0.1


def test_mesh_registry_checks_arguments():
    import ctypes as C
    from ariel_b200._lib import lib
    L = lib()
    v, t = box_mesh()
    tr = np.zeros(3, np.float32)
    mid = C.c_int32()
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    assert L.ariel_mesh_create(p(v), 8, p(t), 12, p(tr), 0.1, C.byref(mid)) == A.ARIEL_OK
    bad = t.copy()
    bad[0, 0] = 8
    other = C.c_int32()
    assert L.ariel_mesh_create(p(v), 8, p(bad), 12, p(tr), 0.1, C.byref(other)) == A.ARIEL_ERR_INVALID_ARG
    assert L.ariel_mesh_create(p(v), 8, p(t), 12, p(tr), 0.0, C.byref(other)) == A.ARIEL_ERR_INVALID_ARG
    assert L.ariel_mesh_destroy(mid.value) == A.ARIEL_OK
    assert L.ariel_mesh_destroy(mid.value) == A.ARIEL_ERR_INVALID_ARG
    # a scene naming an unknown mesh is refused before any device work
    d = dambreak(16)
    A.add_mesh(d, mid.value)
    prm = A.params_default()
    h = C.c_void_p()
    assert L.ariel_create(C.byref(d), C.byref(prm), C.byref(h)) in (A.ARIEL_ERR_INVALID_ARG, A.ARIEL_ERR_NO_DEVICE)


def test_oracle_icosphere_seeds_like_the_sphere():
    """The oracle's brute-force mesh test against the analytic sphere it approximates: lattice
    points well inside or outside agree; the SOLID particles and flags of the mesh scene differ
    from the sphere scene's only near the surface."""
    n = 32
    desc, v, t, c, r = _mesh_scene(n, "icosphere")
    mesh = RefSim(desc, params())
    mesh.add_mesh(v, t, translate=c, scale=r)
    mesh.init()
    sph = RefSim(dambreak(n, seed=7, hi=(0.35, 0.5, 1.0), spheres=[(c, r)]), params())
    sph.init()
    pm, ps = mesh.get_particles(), sph.get_particles()
    solid_m = pm["pos"][pm["type"] == A.SOLID]
    solid_s = ps["pos"][ps["type"] == A.SOLID]
    assert len(solid_m) > 0 and abs(len(solid_m) - len(solid_s)) < 0.15 * len(solid_s)
    d = np.linalg.norm(solid_m - np.array(c, np.float32), axis=1)
    assert d.max() < r * 1.01  # the inscribed mesh never reaches beyond the sphere
    fm, fs = mesh.get_grid(A.GRID_A), sph.get_grid(A.GRID_A)
    assert ((fm == A.SOLID) != (fs == A.SOLID)).sum() < 0.2 * (fs == A.SOLID).sum()
    mesh.step(2)
    p = mesh.get_particles()
    fl = p["type"] == A.FLUID
    inside = np.linalg.norm(p["pos"][fl] - np.array(c, np.float32), axis=1) < r * 0.9
    assert not inside.any()  # the solid constraints keep the liquid out of the mesh
    mesh.close()
    sph.close()


CASES = [("icosphere20", 20, "icosphere", 0), ("box20_evolved", 20, "box", 4), ("icosphere64_evolved", 64, "icosphere", 3)]


@pytest.mark.gpu
@pytest.mark.parametrize("name,n,kind,steps", CASES, ids=[c[0] for c in CASES])
def test_mesh_solid_stage_parity(name, n, kind, steps):
    from ariel_b200.flipsim import Batch, Mesh
    desc, v, t, c, r = _mesh_scene(n, kind)
    prm = params(stop=A.STOP_REL, tol=1e-6, resample_every=1)
    m = Mesh(v, t, translate=c, scale=r)
    A.add_mesh(desc, m.id)
    ora = RefSim(desc, prm)
    ora.add_mesh(v, t, translate=c, scale=r)
    ora.init()
    gpu = Batch([desc], prm)
    gpu.init()
    # seeding with the mesh (liquid outside it, SOLID particles inside) and the first flags
    assert_bits("init pos", gpu.get_particles()["pos"], ora.get_particles()["pos"])
    assert_bits("init type", gpu.get_particles()["type"], ora.get_particles()["type"])
    assert_bits("init flags", gpu.get_grid(A.GRID_A), ora.get_grid(A.GRID_A))
    assert (ora.get_grid(A.GRID_A) == A.SOLID).any()
    if steps:
        ora.step(steps)
        st = ora.get_particles()
        P, P64 = ora.get_grid(A.GRID_P), ora.get_grid(A.GRID_P64)
        ora.close()
        gpu.close()
        ora = RefSim(desc, prm)
        ora.add_mesh(v, t, translate=c, scale=r)
        ora.set_particles(st["pos"], st["vel"], st["mass"], st["type"])
        ora.set_grid(A.GRID_P, P)
        ora.set_grid(A.GRID_P64, P64)
        gpu = Batch([desc], prm)
        gpu.set_particles(st["pos"], st["vel"], st["mass"], st["type"])
        gpu.set_grid(A.GRID_P, P)
        gpu.set_grid(A.GRID_P64, P64)
    stage_parity(name, gpu, ora)
    ora.close()
    gpu.close()
    m.close()


@pytest.mark.gpu
def test_mesh_and_sphere_together_whole_steps():
    """A sphere and a mesh box in one scene, a few whole steps on each side: flags bit-exact
    before every solve, particle state to the solve's tolerance."""
    from ariel_b200.flipsim import Batch, Mesh
    desc = dambreak(24, seed=5, hi=(0.5, 0.6, 1.0), spheres=[((0.7, 0.25, 0.3), 0.12)])
    v, t = box_mesh()
    m = Mesh(v, t, translate=(0.7, 0.2, 0.72), scale=0.1)
    A.add_mesh(desc, m.id)
    prm = params(stop=A.STOP_REL, tol=1e-7)
    ora = RefSim(desc, prm)
    ora.add_mesh(v, t, translate=(0.7, 0.2, 0.72), scale=0.1)
    ora.init()
    gpu = Batch([desc], prm)
    gpu.init()
    assert_bits("init type", gpu.get_particles()["type"], ora.get_particles()["type"])
    ora.step(1)
    gpu.step(1)
    assert_bits("step-1 flags", gpu.get_grid(A.GRID_A), ora.get_grid(A.GRID_A))
    gp, op = gpu.get_particles(), ora.get_particles()
    np.testing.assert_allclose(gp["pos"], op["pos"], rtol=0, atol=1e-5)
    ora.close()
    gpu.close()
    m.close()
