"""Generates tests/golden/reference_<case>.npz: stage-by-stage outputs of betajippity/Ariel's own
FLIP step (compiled from its sources into oracle/_ref/, see oracle/ref_driver.cpp), so that the
CUDA library can be checked against the reference's arithmetic on a machine without the
reference's sources (tests/test_reference_golden.py).

Each case: a seeded scene is seeded by the oracle (the reference's GenerateParticles lives in
scene.cpp, which needs meshes and OpenVDB), the reference runs FlipSim::Init and `steps` whole
steps, and the resulting particles and pressure are handed to a fresh reference FlipSim.  That sim
then runs one step cut into the stages of include/ariel.h, and the outputs of every stage are
stored:

  begin          pos, vel                 (AdjustParticlesStuckInSolids, StoreTemp)
  sort           particle_cell, cell_count
  density        density
  forces         vel
  p2g            ux, uy, uz
  classify       A, L
  boundary_div   pux, puy, puz, ux, uy, uz (StorePreviousGrid + EnforceBoundaryVelocity), D
  solve          P   (the reference's fp32 PCG to its absolute stop rule)
  gradient       ux, uy, uz
  extrapolate    ux, uy, uz, pux, puy, puz
  g2p_advect     pos, vel
  resample       pos, vel

The reference computes the divergence inside Project, so D, P and the gradient's faces come from
a Project run on the boundary stage's input state (the face grids are restored first).

Run (in the build container, where the reference's sources are):
    python tests/golden/make_reference_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ariel_b200 import _abi as A  # noqa: E402
from oracle import pyref  # noqa: E402
from oracle.pyoracle import RefSim  # noqa: E402

CASES = {
    # 16^3 dam break, evolved 5 steps from Init
    "dambreak16": dict(n=16, seed=5, hi=(0.4, 0.6, 1.0), spheres=(), dt=1.0 / 240.0, steps=5),
    # 16^3 block beside a static solid sphere, dt 1/480 (the 256^3 sphere scene's shape), evolved 4 steps
    "sphere16": dict(n=16, seed=7, hi=(0.35, 0.5, 1.0), spheres=(((0.6, 0.3, 0.5), 0.15),), dt=1.0 / 480.0,
                     steps=4),
}


def desc_of(c):
    return A.scene_dambreak(c["n"], liquid_hi=c["hi"], seed=c["seed"], spheres=c["spheres"], dt=c["dt"])


def generate(name, c):
    desc = desc_of(c)
    prm = pyref.reference_params()
    seed_src = RefSim(desc, prm)
    seed_src.init()
    ref0 = pyref.ReferenceSim(desc, prm.rng_seed)
    ref0.init_with(seed_src.get_particles())
    ref0.step(c["steps"])
    st = ref0.get_particles()
    P0 = ref0.get_grid(A.GRID_P)
    ref0.close()
    seed_src.close()

    def fresh():
        r = pyref.ReferenceSim(desc, prm.rng_seed)
        r.set_particles(st["pos"], st["vel"], st["mass"], st["type"])
        r.set_grid(A.GRID_P, P0)
        return r

    out = dict(n=c["n"], seed=c["seed"], hi=np.array(c["hi"], np.float32), dt=np.float32(c["dt"]),
               spheres=np.array([[*cc, r] for cc, r in c["spheres"]], np.float32).reshape(-1, 4),
               rng_seed=np.uint64(prm.rng_seed), in_pos=st["pos"], in_vel=st["vel"], in_mass=st["mass"],
               in_type=st["type"], in_P=P0)
    r = fresh()
    out["max_density"] = np.float32(r.max_density())
    g = {A.GRID_UX: "ux", A.GRID_UY: "uy", A.GRID_UZ: "uz", A.GRID_PREV_UX: "pux", A.GRID_PREV_UY: "puy",
         A.GRID_PREV_UZ: "puz", A.GRID_D: "D", A.GRID_P: "P", A.GRID_L: "L", A.GRID_A: "A"}

    def grids(tag, which):
        for w in which:
            out["%s_%s" % (tag, g[w])] = r.get_grid(w)

    faces = (A.GRID_UX, A.GRID_UY, A.GRID_UZ)
    prev = (A.GRID_PREV_UX, A.GRID_PREV_UY, A.GRID_PREV_UZ)
    r.stage(A.STAGE_BEGIN)
    p = r.get_particles()
    out["begin_pos"], out["begin_vel"] = p["pos"], p["vel"]
    r.stage(A.STAGE_SORT)
    out["sort_particle_cell"], out["sort_cell_count"] = r.get_cells()
    r.stage(A.STAGE_DENSITY)
    out["density_density"] = r.get_particles()["density"]
    r.stage(A.STAGE_FORCES)
    out["forces_vel"] = r.get_particles()["vel"]
    r.stage(A.STAGE_P2G)
    grids("p2g", faces)
    r.stage(A.STAGE_CLASSIFY)
    grids("classify", (A.GRID_A, A.GRID_L))
    saved = {w: r.get_grid(w) for w in faces}
    r.stage(pyref.STAGE_BOUNDARY)
    grids("boundary_div", faces + prev)
    for w in faces:
        r.set_grid(w, saved[w])
    r.stage(pyref.STAGE_PROJECT)
    out["boundary_div_D"] = r.get_grid(A.GRID_D)
    out["solve_P"] = r.get_grid(A.GRID_P)
    grids("gradient", faces)
    r.stage(A.STAGE_EXTRAPOLATE)
    grids("extrapolate", faces + prev)
    r.stage(A.STAGE_G2P_ADVECT)
    p = r.get_particles()
    out["g2p_advect_pos"], out["g2p_advect_vel"] = p["pos"], p["vel"]
    r.stage(A.STAGE_RESAMPLE)
    p = r.get_particles()
    out["resample_pos"], out["resample_vel"] = p["pos"], p["vel"]
    r.close()
    path = os.path.join(HERE, "reference_%s.npz" % name)
    np.savez_compressed(path, **out)
    return path, len(st["mass"])


if __name__ == "__main__":
    if not pyref.available():
        raise SystemExit("the reference's sources are needed (oracle/_ref)")
    for name, c in CASES.items():
        path, npart = generate(name, c)
        print("%s: %d particles -> %s (%d bytes)" % (name, npart, path, os.path.getsize(path)))
