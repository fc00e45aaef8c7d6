"""Generates tests/golden/stages_n8.npz: golden inputs and outputs for the first FLIP stages,
computed by an independent numpy restatement of the reference source (pure float32 scalar
arithmetic in the reference's expression order), not by the C++ oracle or the CUDA library.

Stages restated (one scene, n = 8, 600 particles of which 40 SOLID):
  ParticleGrid::Sort          src/grid/particlegrid.cpp:140-172  -> per-particle cell, counts
  FlipSim::ComputeDensity     src/sim/flip.cpp:697-733            -> density
  ApplyExternalForces         src/sim/flip.cpp:682-695            -> velocity
  SplatParticlesToMACGrid     src/sim/particlegridoperations.inl:146-249 -> face velocities
  MarkCellTypes / BuildSDF    src/grid/particlegrid.cpp:75-138    -> flags, L
  StorePrev + EnforceBoundary + divergence + FlipGrid (flip.cpp:324-437, pgo.inl:45-104,
                              solver.inl:42-56)                  -> prev faces, faces, D
The normaliser m_max_density (flip.cpp:42-70) is restated too.

Run:  python tests/golden/make_golden.py
"""
import os

import numpy as np

F = np.float32
HERE = os.path.dirname(os.path.abspath(__file__))
FLUID, SOLID, AIR = 1, 2, 0


def gmin(x, y):
    return y if y < x else x


def gmax(x, y):
    return y if x < y else x


def sqrlength(p0, p1):
    a = F(p0[0] - p1[0])
    b = F(p0[1] - p1[1])
    c = F(p0[2] - p1[2])
    return F(F(F(a * a) + F(b * b)) + F(c * c))


def smooth(r2, h):
    return gmax(F(F(1.0) - F(r2 / F(h * h))), F(0.0))


def sharpen(r2, h):
    return gmax(F(F(F(h * h) / gmax(r2, F(1.0e-5))) - F(1.0)), F(0.0))


def cell_coord(maxd, x):
    return int(gmax(F(0.0), gmin(F(F(int(maxd)) - F(1.0)), F(F(int(maxd)) * x))))


def sort_cells(pos, n):
    maxd = F(n)
    cells = {}
    pcell = np.zeros(len(pos), np.int64)
    for i, p in enumerate(pos):
        c = (cell_coord(maxd, p[0]), cell_coord(maxd, p[1]), cell_coord(maxd, p[2]))
        cells.setdefault(c, []).append(i)
        pcell[i] = (c[0] * n + c[1]) * n + c[2]
    return cells, pcell


def neighbours(cells, n, lo, hi):
    out = []
    for sx in range(lo[0], hi[0] + 1):
        for sy in range(lo[1], hi[1] + 1):
            for sz in range(lo[2], hi[2] + 1):
                if 0 <= sx < n and 0 <= sy < n and 0 <= sz < n:
                    out.extend(cells.get((sx, sy, sz), []))
    return out


def density(pos, mass, typ, cells, n, density_param, max_density):
    maxd = F(n)
    h = F(F(F(4.0) * F(density_param)) / maxd)
    out = np.zeros(len(pos), np.float32)
    for i in range(len(pos)):
        if typ[i] == SOLID:
            out[i] = F(1.0)
            continue
        c = [cell_coord(maxd, pos[i][a]) for a in range(3)]
        ws = F(0.0)
        for m in neighbours(cells, n, [c[0] - 1, c[1] - 1, c[2] - 1], [c[0] + 1, c[1] + 1, c[2] + 1]):
            ws = F(ws + F(mass[m] * smooth(sqrlength(pos[m], pos[i]), h)))
        out[i] = F(ws / F(max_density))
    return out


def max_density(n, density_param):
    maxd = F(n)
    h = F(F(density_param) / maxd)
    pos = np.array([[F(F(F(i) + F(0.5)) * h), F(F(F(j) + F(0.5)) * h), F(F(F(k) + F(0.5)) * h)]
                    for i in range(10) for j in range(10) for k in range(10)], np.float32)
    cells, _ = sort_cells(pos, n)
    d = density(pos, np.ones(1000, np.float32), np.full(1000, FLUID), cells, n, density_param, 1.0)
    m = F(0.0)
    for v in d:
        m = gmax(m, v)
    return m


def p2g(pos, vel, mass, typ, cells, n):
    RE = F(1.4)
    maxd = F(n)
    ux = np.zeros((n + 1, n, n), np.float32)
    uy = np.zeros((n, n + 1, n), np.float32)
    uz = np.zeros((n, n, n + 1), np.float32)
    gp = [[gmax(F(0.0), gmin(maxd, F(maxd * pos[m][a]))) for a in range(3)] for m in range(len(pos))]
    for i in range(n + 1):
        for j in range(n + 1):
            for k in range(n + 1):
                for axis, grid, ok, fc, lo, hi in (
                        (0, ux, j < n and k < n, (F(i), F(F(j) + F(0.5)), F(F(k) + F(0.5))),
                         (i - 1, j - 2, k - 2), (i, j + 1, k + 1)),
                        (1, uy, i < n and k < n, (F(F(i) + F(0.5)), F(j), F(F(k) + F(0.5))),
                         (i - 2, j - 1, k - 2), (i + 1, j, k + 1)),
                        (2, uz, i < n and j < n, (F(F(i) + F(0.5)), F(F(j) + F(0.5)), F(k)),
                         (i - 2, j - 2, k - 1), (i + 1, j + 1, k))):
                    if not ok:
                        continue
                    sw, su = F(0.0), F(0.0)
                    for m in neighbours(cells, n, lo, hi):
                        if typ[m] != FLUID:
                            continue
                        w = F(mass[m] * sharpen(sqrlength(gp[m], fc), RE))
                        su = F(su + F(w * vel[m][axis]))
                        sw = F(sw + w)
                    grid[i, j, k] = F(su / sw) if sw > 0 else F(0.0)
    return ux, uy, uz


def classify(cells, dens, typ, n, density_param):
    flags = np.zeros((n, n, n), np.int32)
    L = np.zeros((n, n, n), np.float32)
    n0 = F(F(1.0) / F(F(F(density_param) * F(density_param)) * F(density_param)))
    for i in range(n):
        for j in range(n):
            for k in range(n):
                lst = cells.get((i, j, k), [])
                accm = F(0.0)
                sdf = None
                for a in lst:
                    if typ[a] == FLUID:
                        accm = F(accm + dens[a])
                    else:
                        sdf = F(1.0)
                        break
                if sdf is None:
                    sdf = F(F(F(0.2) * n0) - accm)
                L[i, j, k] = sdf
                if any(typ[a] == SOLID for a in lst):
                    flags[i, j, k] = SOLID
                else:
                    flags[i, j, k] = FLUID if sdf < 0.0 else AIR
    return flags, L


def boundary_div(ux, uy, uz, flags, n):
    pux, puy, puz = ux.copy(), uy.copy(), uz.copy()
    wall = lambda a, b, c: F(1.0) if flags[a, b, c] == SOLID else F(-1.0)
    ux, uy, uz = ux.copy(), uy.copy(), uz.copy()
    for i in range(n + 1):
        for j in range(n):
            for k in range(n):
                if i == 0 or i == n or (wall(i, j, k) * wall(i - 1, j, k) < 0):
                    ux[i, j, k] = F(0.0)
    for i in range(n):
        for j in range(n + 1):
            for k in range(n):
                if j == 0 or j == n or (wall(i, j, k) * wall(i, j - 1, k) < 0):
                    uy[i, j, k] = F(0.0)
    for i in range(n):
        for j in range(n):
            for k in range(n + 1):
                if k == 0 or k == n or (wall(i, j, k) * wall(i, j, k - 1) < 0):
                    uz[i, j, k] = F(0.0)
    h = F(F(1.0) / F(n))
    D = np.zeros((n, n, n), np.float32)
    for i in range(n):
        for j in range(n):
            for k in range(n):
                d = F(ux[i + 1, j, k] - ux[i, j, k])
                d = F(d + uy[i, j + 1, k])
                d = F(d - uy[i, j, k])
                d = F(d + uz[i, j, k + 1])
                d = F(d - uz[i, j, k])
                D[i, j, k] = F(-F(d / h))
    return pux, puy, puz, ux, uy, uz, D


def main():
    n = 8
    density_param = 0.5
    dt = F(1.0 / 240.0)
    rng = np.random.default_rng(20261203)
    nf, ns = 560, 40
    pos = np.concatenate([rng.uniform(0.02, 0.7, (nf, 3)), rng.uniform(0.6, 0.95, (ns, 3))]).astype(np.float32)
    vel = np.concatenate([rng.normal(0, 0.3, (nf, 3)), np.zeros((ns, 3))]).astype(np.float32)
    typ = np.array([FLUID] * nf + [SOLID] * ns, np.int32)
    mass = np.array([1.0] * nf + [10.0] * ns, np.float32)
    md = max_density(n, density_param)
    cells, pcell = sort_cells(pos, n)
    counts = np.zeros(n ** 3, np.int32)
    for c, lst in cells.items():
        counts[(c[0] * n + c[1]) * n + c[2]] = len(lst)
    dens = density(pos, mass, typ, cells, n, density_param, md)
    g = (F(0.0), F(-9.8), F(0.0))
    fdt = [F(g[a] * dt) for a in range(3)]
    vel_f = np.array([[F(v[a] + fdt[a]) for a in range(3)] for v in vel], np.float32)
    ux, uy, uz = p2g(pos, vel_f, mass, typ, cells, n)
    flags, L = classify(cells, dens, typ, n, density_param)
    pux, puy, puz, ex, ey, ez, D = boundary_div(ux, uy, uz, flags, n)
    np.savez_compressed(os.path.join(HERE, "stages_n8.npz"), n=n, density=density_param, dt=dt, pos=pos, vel=vel,
                        type=typ, mass=mass, max_density=md, particle_cell=pcell, cell_count=counts, dens=dens,
                        vel_forced=vel_f, ux=ux, uy=uy, uz=uz, flags=flags, L=L, pux=pux, puy=puy, puz=puz,
                        ex=ex, ey=ey, ez=ez, D=D)
    print("max_density", md, "fluid cells", int((flags == FLUID).sum()), "solid cells", int((flags == SOLID).sum()))


if __name__ == "__main__":
    main()
