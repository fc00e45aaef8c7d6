"""The oracle pinned to the reference's own code.

oracle/_ref/ holds betajippity/Ariel's FLIP step compiled from its unmodified sources
(src/sim/flip.cpp and everything it includes, src/grid/particlegrid.cpp) with stand-in headers for
the libraries absent here (oracle/refshim/, oracle/ref_driver.cpp).  These CPU tests hold the C++
restatement in oracle/ariel_oracle.cpp bit-identical to it: whole FlipSim::Step calls from Init,
and every stage from identical evolved states.  The oracle runs with the parameters the reference
hard-codes (fp32 PCG, the reference preconditioner, the absolute stop rule, resampling every step).

Since the CUDA library is tested against the oracle (and against fixtures of this reference build,
tests/golden/), this closes the chain GPU = oracle = reference.  The reference's sources exist only
in the build container; elsewhere these tests skip.
"""
import numpy as np
import pytest

from ariel_b200 import _abi as A
from oracle import pyref
from oracle.pyoracle import RefSim, philox as oracle_philox

from helpers import assert_bits

pytestmark = pytest.mark.skipif(not pyref.available(), reason="reference sources not present (oracle/_ref unbuilt)")

FIELDS = ("pos", "vel", "density", "mass", "type")
GRIDS = (A.GRID_UX, A.GRID_UY, A.GRID_UZ, A.GRID_PREV_UX, A.GRID_PREV_UY, A.GRID_PREV_UZ,
         A.GRID_D, A.GRID_P, A.GRID_L, A.GRID_A)


def scene(n, seed, hi=(0.4, 0.6, 1.0), spheres=(), density=0.5, dt=1.0 / 240.0):
    d = A.scene_dambreak(n, liquid_hi=hi, seed=seed, spheres=spheres, density=density, dt=dt)
    return d


def compare_all(tag, ref, ora, grids=GRIDS):
    pr, po = ref.get_particles(), ora.get_particles()
    for f in FIELDS:
        assert_bits("%s %s" % (tag, f), pr[f], po[f])
    for w in grids:
        assert_bits("%s grid %d" % (tag, w), ref.get_grid(w), ora.get_grid(w))


WHOLE = [
    ("dambreak16", scene(16, 3), 6),
    ("dambreak24", scene(24, 11), 10),
    ("sphere20", scene(20, 7, hi=(0.35, 0.5, 1.0), spheres=[((0.6, 0.3, 0.5), 0.15)]), 5),
    ("sphere32_dt480", scene(32, 9, hi=(0.35, 0.5, 1.0), spheres=[((0.6, 0.3, 0.5), 0.15)], dt=1.0 / 480.0), 3),
    ("density1_n13", scene(13, 13, density=1.0), 4),
    ("density025_n10", scene(10, 17, density=0.25), 2),
    ("two_spheres18", scene(18, 19, hi=(0.5, 0.7, 1.0), spheres=[((0.7, 0.25, 0.3), 0.12), ((0.7, 0.25, 0.7), 0.12)]), 4),
    # the 64^3 dam break (502,656 particles), two steps from Init
    ("dambreak64", scene(64, 1), 2),
]


@pytest.mark.parametrize("name,desc,steps", WHOLE, ids=[w[0] for w in WHOLE])
def test_whole_steps_match_reference(name, desc, steps):
    prm = pyref.reference_params()
    ora = RefSim(desc, prm)
    ora.init()
    ref = pyref.ReferenceSim(desc, prm.rng_seed)
    ref.init_with(ora.get_particles())
    assert ref.max_density() == ora.max_density()
    assert_bits(name + " init flags", ref.get_grid(A.GRID_A), ora.get_grid(A.GRID_A))
    for s in range(steps):
        ora.step(1)
        ref.step(1)
        compare_all("%s step %d" % (name, s + 1), ref, ora)
    assert ref.frame() == steps
    ora.close()
    ref.close()


@pytest.mark.parametrize("name,desc,steps", [WHOLE[0], WHOLE[2]], ids=["dambreak16", "sphere20"])
def test_glm096_minmax_gives_the_same_steps(name, desc, steps):
    """glm's two min/max conventions differ only for NaN and signed zeros; neither occurs here."""
    prm = pyref.reference_params()
    ora = RefSim(desc, prm)
    ora.init()
    ref = pyref.ReferenceSim(desc, prm.rng_seed, variant="glm096")
    ref.init_with(ora.get_particles())
    for s in range(steps):
        ora.step(1)
        ref.step(1)
        compare_all("%s glm096 step %d" % (name, s + 1), ref, ora)
    ora.close()
    ref.close()


def _evolved_pair(desc, steps):
    prm = pyref.reference_params()
    src = RefSim(desc, prm)
    src.init()
    src.step(steps)
    st = src.get_particles()
    P = src.get_grid(A.GRID_P)
    ora = RefSim(desc, prm)
    ora.set_particles(st["pos"], st["vel"], st["mass"], st["type"])
    ora.set_grid(A.GRID_P, P)
    ref = pyref.ReferenceSim(desc, prm.rng_seed)
    ref.set_particles(st["pos"], st["vel"], st["mass"], st["type"])
    ref.set_grid(A.GRID_P, P)
    src.close()
    return ora, ref


STAGE_CASES = [
    ("dambreak16_evolved", scene(16, 5), 6),
    ("sphere20_evolved", scene(20, 7, hi=(0.35, 0.5, 1.0), spheres=[((0.6, 0.3, 0.5), 0.15)]), 4),
]


@pytest.mark.parametrize("name,desc,steps", STAGE_CASES, ids=[c[0] for c in STAGE_CASES])
def test_each_stage_matches_reference(name, desc, steps):
    """Every stage from identical state.  The reference computes the divergence inside Project,
    so the oracle's BOUNDARY_DIV is checked in two parts: the face grids against the reference's
    StorePreviousGrid + EnforceBoundaryVelocity, and D against Project's (on a second pair)."""
    ora, ref = _evolved_pair(desc, steps)
    assert ref.max_density() == ora.max_density()
    for stage in range(A.STAGE_COUNT):
        tag = "%s/%s" % (name, A.STAGE_NAMES[stage])
        if stage == A.STAGE_SOLVE:
            # The reference's Solve starts with FlipGrid: hand it the divergence before the flip.
            ref.set_grid(A.GRID_D, -ora.get_grid(A.GRID_D))
            ora.stage(stage)
            ref.stage(pyref.STAGE_SOLVE_WITH_FLIP)
        else:
            ora.stage(stage)
            ref.stage(stage)
        if stage == A.STAGE_BOUNDARY_DIV:
            grids = (A.GRID_UX, A.GRID_UY, A.GRID_UZ, A.GRID_PREV_UX, A.GRID_PREV_UY, A.GRID_PREV_UZ)
        elif stage == A.STAGE_SORT:
            rc, rn = ref.get_cells()
            oc, on = ora.get_cells()
            assert_bits(tag + " particle->cell", rc, oc)
            assert_bits(tag + " per-cell counts", rn, on)
            grids = ()
        else:
            grids = GRIDS
        compare_all(tag, ref, ora, grids)
    ora.close()
    ref.close()

    # D, P and faces through the reference's Project (StorePreviousGrid .. EnforceBoundaryVelocity)
    ora, ref = _evolved_pair(desc, steps)
    for stage in range(A.STAGE_BOUNDARY_DIV):
        ora.stage(stage)
        ref.stage(stage)
    for stage in (A.STAGE_BOUNDARY_DIV, A.STAGE_SOLVE, A.STAGE_GRADIENT):
        ora.stage(stage)
    ref.stage(pyref.STAGE_PROJECT)
    compare_all(name + "/project", ref, ora)
    ora.close()
    ref.close()


def test_rand_stand_in_serves_the_oracle_stream():
    rng = np.random.default_rng(5)
    for _ in range(64):
        c = rng.integers(0, 2 ** 32, 4, dtype=np.uint64).astype(np.uint32)
        k = rng.integers(0, 2 ** 32, 2, dtype=np.uint64).astype(np.uint32)
        assert (pyref.philox(c, k) == oracle_philox(c, k)).all()
    # Salmon et al.'s published known answer for a zero counter and key
    z = pyref.philox(np.zeros(4, np.uint32), np.zeros(2, np.uint32))
    assert [int(v) for v in z] == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]


def _ray_triangle_cases(rng):
    """Triangles and rays for the mesh queries' ray-triangle test: rays aimed at random points,
    vertices and edge midpoints of random triangles (grid units), random rays, the +z rays of
    the inside test against axis-aligned faces (rays in the triangle's plane included), rays hitting
    from behind, and degenerate triangles."""
    cases = []
    for _ in range(3000):
        v = rng.uniform(0.0, 64.0, (3, 3)).astype(np.float32)
        o = rng.uniform(-8.0, 72.0, 3).astype(np.float32)
        w = rng.dirichlet((1.0, 1.0, 1.0))
        targets = [w @ v, v[0], v[1], v[2], 0.5 * (v[0] + v[1]), 0.5 * (v[1] + v[2])]
        for tgt in targets:
            d = (np.asarray(tgt, np.float64) - o).astype(np.float32)
            n = np.sqrt(np.float32(np.dot(d, d)))
            if n > 0:
                cases.append((v, o, (d / n).astype(np.float32)))
        d = rng.normal(size=3).astype(np.float32)
        cases.append((v, o, (d / np.sqrt(np.dot(d, d))).astype(np.float32)))
        cases.append((v, o, -cases[-2][2]))  # the aimed ray reversed: a hit behind the origin
    z = np.array([0.0, 0.0, 1.0], np.float32)
    for _ in range(2000):
        a, b = sorted(rng.integers(0, 32, 2))
        c = rng.integers(0, 32)
        quad = np.array([[a, a, c], [b, a, c], [b, b, c]], np.float32)  # a face normal to z
        side = np.array([[a, c, a], [b, c, a], [b, c, b]], np.float32)  # a face containing z
        o = np.array([rng.integers(0, 32) + 0.5, rng.integers(0, 32) + 0.5, rng.integers(-4, 4)], np.float32)
        cases += [(quad, o, z), (side, o, z)]
    for _ in range(200):
        p = rng.uniform(0.0, 64.0, 3).astype(np.float32)
        cases.append((np.stack([p, p, p]), rng.uniform(0.0, 64.0, 3).astype(np.float32), z))
    return cases


def test_ray_triangle_matches_reference():
    """The mesh queries' ray-triangle test (the CUDA library's mesh.cuh, held bit-exact to the
    oracle by tests/test_mesh_solids.py) against Obj::RayTriangleTest (src/geom/obj/obj.cpp:354-398)
    compiled from the reference's sources: the same hits, and the same hit points bit for bit."""
    from oracle.pyoracle import tri_ray
    rng = np.random.default_rng(11)
    cases = _ray_triangle_cases(rng)
    hits = 0
    for v, o, d in cases:
        rh, rp = pyref.ray_triangle(v, o, d)
        oh, op = tri_ray(v, o, d)
        assert rh == oh, (v.tolist(), o.tolist(), d.tolist())
        if rh:
            hits += 1
            assert np.array_equal(rp.view(np.uint32), op.view(np.uint32)), (v.tolist(), o.tolist(), d.tolist())
    assert hits > len(cases) // 4
