"""Generate the golden fixtures in this directory from the REFERENCE Aster CPU
code, compiled unmodified from its sources (oracle/Makefile ->
oracle/_ref/libaster_ref.so). Run here, where the reference sources exist:

    make -C oracle REF=<reference source tree> && python tests/golden/make_golden.py

The fixtures are committed; the tests read them on machines without the
reference. Inputs come from the seeded generators in aster_b200/gen.py.

Fixtures:
  allpairs_plummer512.npz   Parallelized::compute_forces (Newton, and Newton+PN1
                            with c=100 and boosted velocities), eps2=1e-4,
                            reference get_total_energy.
  leapfrog_plummer4096.npz  C1 setup (N=4096 Plummer, eps=0.01, dt=1e-3):
                            update_leapfrog x 100 with Parallelized; accelerations
                            after steps 1, 10, 50, 100; final x, v; energies.
  tree_plummer4096.npz      Barnes_Hut::make_tree + unite on a lognormal-mass
                            Plummer sphere with 64 duplicated positions (forces
                            Morton ties): codes, left, right, node masses/COMs.
  tree_small.npz            the same for n = 2, 3, 5, 33 and an all-equal set.
  pn_pairs.npz              compute_gravitational on 64 seeded pairs (c = 10,
                            eps2 = 1e-4) for force laws NEWTON|PN1, NEWTON|PN2,
                            NEWTON|PN25 and all four terms: the force on body 1.

  allpairs_pn_plummer256.npz  Parallelized::compute_forces on a lognormal-mass
                            N=256 Plummer sphere with velocities x5, c = 10,
                            eps2 = 1e-4, for NEWTON and the four PN force laws
                            of pn_pairs.npz.
  saba_plummer256.npz       update_SABA1..10 with Parallelized: 4 steps each from one
                            N=256 Plummer state (eps2 = 1e-4, dt = 1e-3), and the
                            reference coefficient tables (GPU::saba_coeffs).

  kepler_drift.npz          update_WH_planetary under a zero-force solver (so the
                            reference's update_kepler drift alone, two half-steps
                            a step) on 400 massless bodies about a unit mass
                            (gen.kepler_orbits: elliptic, near-parabolic and
                            hyperbolic), dt = 0.05, 40 steps: final x, v.

  opencl_tree.npz           the reference's OpenCL tree construction (its kernel
                            text for gen_mortons, the bitonic sort and build_tree,
                            run on the CPU: oracle/ref_cl -> libaster_refcl.so) on
                            Plummer spheres of n = 2, 3, 100, 257, 1000, 3000 with a
                            duplicated position and a coordinate at +B: per-body
                            codes, sorted codes, body order, left/right/parent.

`python tests/golden/make_golden.py pn_pairs` regenerates one fixture only.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from aster_b200 import gen  # noqa: E402
from oracle.oracle import NEWTON, PN1, PN2, PN25, Ref, RefCL  # noqa: E402

OUT = Path(__file__).resolve().parent


def allpairs_fixture(ref: Ref):
    pos, vel, m = gen.plummer(512, 1001)
    B = gen.bounding_cube(pos)
    ref.setup(pos, vel, m, G=1.0, eps2=1e-4, box=B)
    acc = ref.forces()
    e_ref = ref.energy()
    vb = vel * 30.0
    ref.setup(pos, vb, m, G=1.0, c=100.0, eps2=1e-4, box=B, force_law=NEWTON | PN1)
    acc_pn = ref.forces()
    np.savez_compressed(OUT / "allpairs_plummer512.npz", pos=pos, vel=vel, m=m, eps2=1e-4, acc=acc,
                        energy_ref_form=e_ref, vel_pn=vb, c_pn=100.0, acc_pn1=acc_pn)


def leapfrog_fixture(ref: Ref):
    pos, vel, m = gen.plummer(4096, 1001)
    B = gen.bounding_cube(pos)
    eps2, dt = 1e-4, 1e-3
    ref.setup(pos, vel, m, G=1.0, dt=dt, eps2=eps2, box=B)
    e0 = ref.energy()
    keep = [0, 9, 49, 99]
    accs = []
    for k in range(100):
        a = ref.leapfrog(1, record_acc=True)[0]
        if k in keep:
            accs.append(a)
    p1, v1, _ = ref.state()
    e1 = ref.energy()
    np.savez_compressed(OUT / "leapfrog_plummer4096.npz", pos=pos, vel=vel, m=m, eps2=eps2, dt=dt, steps=100,
                        acc_steps=np.array(keep) + 1, acc=np.stack(accs), pos_final=p1, vel_final=v1,
                        energy0_ref_form=e0, energy1_ref_form=e1)


def tree_case(ref: Ref, pos, m):
    vel = np.zeros_like(pos)
    B = gen.bounding_cube(pos)
    ref.setup(pos, vel, m, G=1.0, eps2=2.5e-5, theta=0.5, box=B, solver="bh")
    t = ref.bh_tree()
    return dict(pos=pos, m=m, box=B, codes=t["codes"], left=t["left"], right=t["right"],
                node_mass=t["node_mass"], node_com=t["node_com"])


def tree_fixture(ref: Ref):
    pos, _, m = gen.plummer(4096, 1002, masses="lognormal")
    rng = np.random.default_rng(7)
    src = rng.choice(4096, 64, replace=False)
    dst = rng.choice(np.setdiff1d(np.arange(4096), src), 64, replace=False)
    pos[dst] = pos[src]  # exact duplicates: equal codes, tie-break exercised
    d = tree_case(ref, pos, m)
    np.savez_compressed(OUT / "tree_plummer4096.npz", **d)
    small = {}
    for n in (2, 3, 5, 33):
        p, _, mm = gen.plummer(n, 2000 + n)
        for k, v in tree_case(ref, p, mm).items():
            small[f"n{n}_{k}"] = v
    p = np.tile(np.array([[0.25, -0.5, 0.125]]), (9, 1))
    p[0] = [1.0, 1.0, 1.0]  # one distinct body so the cube is not degenerate
    for k, v in tree_case(ref, p, np.full(9, 1.0 / 9)).items():
        small[f"eq9_{k}"] = v
    np.savez_compressed(OUT / "tree_small.npz", **small)


PN_LAWS = {"pn1": NEWTON | PN1, "pn2": NEWTON | PN2, "pn25": NEWTON | PN25, "all": NEWTON | PN1 | PN2 | PN25}


def pn_fixture(ref: Ref):
    rng = np.random.default_rng(1006)
    npair, c, eps2 = 64, 10.0, 1e-4
    m = rng.lognormal(0.0, 0.5, (npair, 2))
    p1 = rng.normal(0.0, 1.0, (npair, 3))
    p2 = p1 + rng.normal(0.0, 0.5, (npair, 3))
    v1 = rng.normal(0.0, 1.0, (npair, 3))
    v2 = rng.normal(0.0, 1.0, (npair, 3))
    out = dict(m=m, p1=p1, p2=p2, v1=v1, v2=v2, c=c, eps2=eps2)
    for name, law in PN_LAWS.items():
        ref.setup(np.stack([p1[0], p2[0]]), np.stack([v1[0], v2[0]]), m[0], G=1.0, c=c, eps2=eps2, force_law=law)
        out[f"force_{name}"] = np.stack([ref.pair_force(m[k, 0], m[k, 1], v1[k], v2[k], p1[k], p2[k])
                                         for k in range(npair)])
    np.savez_compressed(OUT / "pn_pairs.npz", **out)


def allpairs_pn_fixture(ref: Ref):
    pos, vel, m = gen.plummer(256, 1015, masses="lognormal")
    vb = vel * 5.0
    B = gen.bounding_cube(pos)
    c, eps2 = 10.0, 1e-4
    out = dict(pos=pos, vel=vb, m=m, c=c, eps2=eps2)
    for name, law in {"newton": NEWTON, **PN_LAWS}.items():
        ref.setup(pos, vb, m, G=1.0, c=c, eps2=eps2, box=B, force_law=law)
        out[f"acc_{name}"] = ref.forces()
    np.savez_compressed(OUT / "allpairs_pn_plummer256.npz", **out)


def saba_fixture(ref: Ref):
    pos, vel, m = gen.plummer(256, 1008)
    eps2, dt, steps = 1e-4, 1e-3, 4
    out = dict(pos=pos, vel=vel, m=m, eps2=eps2, dt=dt, steps=steps)
    for order in range(1, 11):
        ref.setup(pos, vel, m, G=1.0, dt=dt, eps2=eps2)
        ref.saba(order, steps)
        p1, v1, _ = ref.state()
        out[f"pos_{order}"], out[f"vel_{order}"] = p1, v1
        out[f"coeffs_{order}"] = ref.saba_coeffs(order)
    np.savez_compressed(OUT / "saba_plummer256.npz", **out)


def kepler_fixture(ref: Ref):
    pos, vel, m, e = gen.kepler_orbits(400, 1025)
    dt, nsteps = 0.05, 40
    ref.setup(pos, vel, m, G=1.0, dt=dt)
    ref.wh_drift_only(nsteps)
    rp, rv, _ = ref.state()
    np.savez_compressed(OUT / "kepler_drift.npz", pos=pos, vel=vel, m=m, e=e, dt=dt, steps=nsteps,
                        ref_pos=rp, ref_vel=rv)


def opencl_cases():
    """The inputs of opencl_tree.npz: (n, positions, masses, B)."""
    for n, seed in ((2, 1), (3, 2), (100, 3), (257, 6), (1000, 7), (3000, 8)):
        pos, _, m = gen.plummer(n, seed)
        if n > 10:
            pos[7] = pos[9]                     # equal codes: tie broken by body index
            pos[3, 0] = np.abs(pos).max()       # a coordinate at +B (1024 wraps to 0)
        yield n, pos, m, float(np.abs(pos).max())


def opencl_fixture(ref: Ref):
    cl = RefCL()
    out = {}
    for n, pos, m, B in opencl_cases():
        r = cl.build(pos, m, B)
        out[f"n{n}_pos"], out[f"n{n}_m"], out[f"n{n}_B"] = pos, m, B
        for k, v in r.items():
            out[f"n{n}_{k}"] = v
    np.savez_compressed(OUT / "opencl_tree.npz", **out)


FIXTURES = {"allpairs": allpairs_fixture, "leapfrog": leapfrog_fixture, "tree": tree_fixture,
            "pn_pairs": pn_fixture, "saba": saba_fixture, "allpairs_pn": allpairs_pn_fixture,
            "kepler": kepler_fixture, "opencl": opencl_fixture}


def main():
    ref = Ref()
    for name in (sys.argv[1:] or FIXTURES):
        FIXTURES[name](ref)
    for f in sorted(OUT.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
