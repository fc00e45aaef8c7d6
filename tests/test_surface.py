"""Liquid surface for output (the reference's particle level set and its mesh,
src/grid/levelset.cpp:101-172 through OpenVDB, called by Scene::ExportParticles).

The CUDA library rasterises the FLUID particles as spheres of radius 0.5 cells into a level set
(scatter with an order-free atomic minimum) and meshes it by surface nets; the oracle does the
same with serial loops.  Level set, vertices and quads must agree bit for bit.  OpenVDB is absent,
so the reference's own level set and mesh are not reproduced (its particle trails and 3-cell band
are not); CPU tests check what a surface must be: closed, consistently wound, enclosing the
liquid's volume.
"""
import numpy as np
import pytest

from ariel_b200 import _abi as A
from oracle.pyoracle import RefSim

from helpers import assert_bits, dambreak, params


def _closed_and_volume(v, q, manifold=False):
    """The quad mesh has no boundary: every edge is walked as often in one direction as in the
    other (closed and consistently wound; where two sheets of the surface touch, surface nets
    shares an edge among four quads).  With `manifold`, exactly once each way.  Returns the
    enclosed volume (divergence theorem over the quads split in two triangles)."""
    from collections import Counter
    edges = Counter()
    for a, b, c, d in q:
        for x, y in ((a, b), (b, c), (c, d), (d, a)):
            edges[(x, y)] += 1
    for (x, y), cnt in edges.items():
        assert edges.get((y, x), 0) == cnt, "open or inconsistently wound edge %s" % ((x, y),)
        assert not manifold or cnt == 1, "edge %s shared by more than two quads" % ((x, y),)
    v = v.astype(np.float64)
    tri = np.concatenate([q[:, [0, 1, 2]], q[:, [0, 2, 3]]])
    a, b, c = v[tri[:, 0]], v[tri[:, 1]], v[tri[:, 2]]
    return np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0


def test_oracle_surface_of_a_block():
    n = 16
    r = RefSim(dambreak(n, seed=1, jitter=0.0), params())
    r.init()
    phi = r.level_set()
    assert phi.shape == (n + 5,) * 3
    g = lambda x, y, z: phi[x + 2, y + 2, z + 2]
    assert g(3, 4, 8) < 0 and g(12, 14, 8) > 0  # inside the block / in the air
    v, q = r.surface_mesh()
    vol = _closed_and_volume(v, q, manifold=True)
    p = r.get_particles()["pos"] * n
    inner = np.prod(p.max(0) - p.min(0))        # the box of the particle centres
    outer = np.prod(p.max(0) - p.min(0) + 1.0)  # the spheres' union reaches 0.5 beyond them
    assert inner < vol < outer, (inner, vol, outer)
    r.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n,steps", [(16, 0), (32, 6), (64, 3)])
def test_surface_matches_oracle(n, steps, tmp_path):
    from ariel_b200.flipsim import Batch
    desc = dambreak(n, seed=3)
    prm = params()
    ora = RefSim(desc, prm)
    ora.init()
    if steps:
        ora.step(steps)
    st = ora.get_particles()
    gpu = Batch([desc], prm)
    gpu.set_particles(st["pos"], st["vel"], st["mass"], st["type"])
    ora2 = RefSim(desc, prm)
    ora2.set_particles(st["pos"], st["vel"], st["mass"], st["type"])
    assert_bits("level set", gpu.level_set(), ora2.level_set())
    gv, gq = gpu.surface_mesh()
    ov, oq = ora2.surface_mesh()
    assert_bits("vertices", gv, ov)
    assert_bits("quads", gq, oq)
    _closed_and_volume(gv, gq)
    gpu.export_surface(tmp_path / "surface.obj", 7)
    lines = (tmp_path / "surface.0007.obj").read_text().splitlines()
    assert sum(l.startswith("v ") for l in lines) == len(gv) and sum(l.startswith("f ") for l in lines) == len(gq)
    for h in (gpu, ora, ora2):
        h.close()
