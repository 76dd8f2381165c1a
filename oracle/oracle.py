"""ctypes front end for the two CPU checkers. TEST INFRASTRUCTURE ONLY.

* ``Ref``: the reference Aster CPU code compiled unmodified from its sources
  (oracle/Makefile -> oracle/_ref/libaster_ref.so). Exists where the reference
  sources were available at build time; the library travels prebuilt.
* ``Orc``: the CPU restatement in oracle/aster_oracle.c
  (oracle/build_oracle.sh -> oracle/_build/libaster_oracle.so).

Only tests/, the golden-fixture script, ``__graft_entry__.smoke`` and the
CPU-baseline leg of bench.py may use this module, and only as the checker.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libaster_ref.so"
REFCL_LIB = HERE / "_ref" / "libaster_refcl.so"
ORC_LIB = HERE / "_build" / "libaster_oracle.so"

_D = ctypes.POINTER(ctypes.c_double)
_F = ctypes.POINTER(ctypes.c_float)
_I32 = ctypes.POINTER(ctypes.c_int32)
_U32 = ctypes.POINTER(ctypes.c_uint32)
_U64 = ctypes.POINTER(ctypes.c_uint64)
_L = ctypes.POINTER(ctypes.c_long)

NEWTON = 0x1
PN1 = 0x10
PN2 = 0x100
PN25 = 0x1000
EIH = 0x10000  # with PN1: the N-body Einstein-Infeld-Hoffmann 1PN acceleration (ensembles)


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Ref:
    """The reference CPU implementation (one Simulation per process)."""

    _lib = None

    def __init__(self):
        if Ref._lib is None:
            if not REF_LIB.exists():
                raise FileNotFoundError(f"{REF_LIB} missing: run `make -C oracle REF=<reference source tree>`")
            lib = ctypes.CDLL(str(REF_LIB))
            lib.ref_setup.argtypes = [ctypes.c_int, _D, _D, _D] + [ctypes.c_double] * 6 + [ctypes.c_int, ctypes.c_int]
            lib.ref_get_state.argtypes = [_D, _D, _D]
            lib.ref_compute_forces.argtypes = [_D]
            lib.ref_set_bounds.argtypes = [ctypes.c_int, ctypes.c_int]
            lib.ref_leapfrog.argtypes = [ctypes.c_int, _D]
            lib.ref_energy.restype = ctypes.c_double
            lib.ref_bh_tree.argtypes = [_U32, _I32, _I32, _D, _D]
            lib.ref_bh_node_extra.argtypes = [_D, _D]
            lib.ref_set_temps.argtypes = [_D]
            lib.ref_pair_force.argtypes = [ctypes.c_double, ctypes.c_double, _D, _D, _D, _D, _D]
            lib.ref_saba.argtypes = [ctypes.c_int, ctypes.c_int]
            lib.ref_wh.argtypes = [ctypes.c_int]
            lib.ref_wh_drift_only.argtypes = [ctypes.c_int]
            lib.ref_saba_coeffs.argtypes = [ctypes.c_int, _D]
            Ref._lib = lib
        self.lib = Ref._lib
        self.n = 0

    @staticmethod
    def available() -> bool:
        return REF_LIB.exists()

    def threads(self) -> int:
        return self.lib.ref_threads()

    def setup(self, pos, vel, m, G=1.0, c=299792458.0, dt=1e-3, eps2=0.0, theta=0.5,
              box=None, force_law=NEWTON, solver="allpairs"):
        pos, vel, m = _c64(pos), _c64(vel), _c64(m)
        if box is None:
            box = float(np.abs(pos).max())
        kind = {"allpairs": 1, "bh": 2}[solver]
        self.n = len(m)
        rc = self.lib.ref_setup(self.n, _p(pos, _D), _p(vel, _D), _p(m, _D), G, c, dt, eps2, theta,
                                box, force_law, kind)
        if rc != 0:
            raise RuntimeError(f"ref_setup failed: {rc}")
        return self

    def forces(self):
        acc = np.zeros((self.n, 3))
        self.lib.ref_compute_forces(_p(acc, _D))
        return acc

    def leapfrog(self, nsteps, record_acc=False):
        acc = np.zeros((nsteps, self.n, 3)) if record_acc else None
        self.lib.ref_leapfrog(nsteps, _p(acc, _D))
        return acc

    def state(self):
        pos, vel, acc = (np.zeros((self.n, 3)) for _ in range(3))
        self.lib.ref_get_state(_p(pos, _D), _p(vel, _D), _p(acc, _D))
        return pos, vel, acc

    def energy(self) -> float:
        return self.lib.ref_energy()

    def bh_tree(self):
        n = self.n
        codes = np.zeros(n, np.uint32)
        left = np.zeros(2 * n - 1, np.int32)
        right = np.zeros(2 * n - 1, np.int32)
        nm = np.zeros(2 * n - 1)
        nc = np.zeros((2 * n - 1, 3))
        rc = self.lib.ref_bh_tree(_p(codes, _U32), _p(left, _I32), _p(right, _I32), _p(nm, _D), _p(nc, _D))
        if rc != 0:
            raise RuntimeError(f"ref_bh_tree failed: {rc}")
        nv = np.zeros((2 * n - 1, 3))
        nt = np.zeros(2 * n - 1)
        self.lib.ref_bh_node_extra(_p(nv, _D), _p(nt, _D))
        return dict(codes=codes, left=left, right=right, node_mass=nm, node_com=nc, node_vel=nv, node_temp=nt)

    def set_temps(self, temps):
        """BodyArray::temps of the current bodies."""
        self.lib.ref_set_temps(_p(_c64(temps), _D))
        return self

    def saba(self, order, nsteps):
        """nsteps of the reference CPU SABA_order (update_SABA1..10)."""
        if self.lib.ref_saba(order, nsteps) != 0:
            raise RuntimeError("ref_saba failed")

    def wh(self, nsteps):
        """nsteps of the reference CPU update_WH_planetary (body 0 central)."""
        if self.lib.ref_wh(nsteps) != 0:
            raise RuntimeError("ref_wh failed")

    def wh_drift_only(self, nsteps):
        """nsteps of update_WH_planetary under a zero-force solver: the
        reference's update_kepler drift of every body about body 0 (two
        half-steps per step), with no kick."""
        if self.lib.ref_wh_drift_only(nsteps) != 0:
            raise RuntimeError("ref_wh_drift_only failed")

    def saba_coeffs(self, order):
        """The reference's SABA table for the order: (d, c) slot pairs."""
        out = np.zeros(22)
        ln = self.lib.ref_saba_coeffs(order, _p(out, _D))
        return out[:ln].copy()

    def set_bounds(self, lower, upper=-1):
        """Solver::set_bounds on the current solver (reset by every setup)."""
        if self.lib.ref_set_bounds(lower, upper) != 0:
            raise RuntimeError("ref_set_bounds failed")
        return self

    def pair_force(self, m1, m2, v1, v2, p1, p2):
        f = np.zeros(3)
        args = [_c64(v1), _c64(v2), _c64(p1), _c64(p2)]
        self.lib.ref_pair_force(m1, m2, *[_p(a, _D) for a in args], _p(f, _D))
        return f


class RefCL:
    """The reference's OpenCL tree construction (gen_mortons, the bitonic
    sort, build_tree) compiled from its kernel text and run on the CPU under a
    work-group emulator (oracle/ref_cl; oracle/Makefile ->
    oracle/_ref/libaster_refcl.so), launched as BH_hyper's host code launches
    it (src/solvers/full_GPU.cpp:52-112, 312-338)."""

    _lib = None

    def __init__(self):
        if RefCL._lib is None:
            if not REFCL_LIB.exists():
                raise FileNotFoundError(f"{REFCL_LIB} missing: run `make -C oracle REF=<reference source tree>`")
            lib = ctypes.CDLL(str(REFCL_LIB))
            lib.refcl_build.argtypes = [ctypes.c_long, _D, _D, _D, _U32, _U32, _I32, _I32, _I32, _I32]
            lib.refcl_build.restype = ctypes.c_int
            RefCL._lib = lib
        self.lib = RefCL._lib

    @staticmethod
    def available() -> bool:
        return REFCL_LIB.exists()

    def build(self, pos, m, bd):
        """pos (n, 3), masses (n,), bd: the bounding half-sizes (3,). Returns
        the per-body codes, the sorted codes and body order of the sort's
        first n entries, and the 2n - 1 node links (left, right, parent)."""
        pos, m = _c64(pos), _c64(m)
        bd = _c64(np.broadcast_to(np.asarray(bd, dtype=np.float64), (3,)))
        n = len(m)
        out = dict(codes=np.zeros(n, np.uint32), sorted_codes=np.zeros(n, np.uint32), perm=np.zeros(n, np.int32),
                   left=np.zeros(2 * n - 1, np.int32), right=np.zeros(2 * n - 1, np.int32),
                   parent=np.zeros(2 * n - 1, np.int32))
        st = self.lib.refcl_build(n, _p(pos, _D), _p(m, _D), _p(bd, _D), _p(out["codes"], _U32),
                                  _p(out["sorted_codes"], _U32), _p(out["perm"], _I32), _p(out["left"], _I32),
                                  _p(out["right"], _I32), _p(out["parent"], _I32))
        if st != 0:
            raise ValueError("refcl_build needs n >= 2")
        return out


class Orc:
    """The CPU restatement (oracle/aster_oracle.c)."""

    _lib = None

    def __init__(self):
        if Orc._lib is None:
            if not ORC_LIB.exists():
                raise FileNotFoundError(f"{ORC_LIB} missing: run oracle/build_oracle.sh")
            lib = ctypes.CDLL(str(ORC_LIB))
            lib.orc_pair_acc.argtypes = [ctypes.c_double] * 3 + [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                                 _D, _D, _D, _D, _D]
            lib.orc_allpairs.argtypes = [ctypes.c_long, _D, _D, _D, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, ctypes.c_long, _L, _D]
            lib.orc_energy.argtypes = [ctypes.c_long, _D, _D, _D, ctypes.c_double, ctypes.c_double, ctypes.c_int]
            lib.orc_energy.restype = ctypes.c_double
            lib.orc_momentum.argtypes = [ctypes.c_long, _D, _D, _D]
            lib.orc_saba_coeffs.argtypes = [ctypes.c_int, _D, _D]
            lib.orc_saba.argtypes = [ctypes.c_long, _D, _D, _D, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, _D]
            lib.orc_wh.argtypes = [ctypes.c_long, _D, _D, _D, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_int]
            lib.orc_kepler.argtypes = [_D, _D, ctypes.c_double, ctypes.c_double]
            lib.orc_saba_seq.argtypes = [ctypes.c_long, _D, _D, _D, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int, _D, _D,
                                         ctypes.c_int, _D]
            lib.orc_kdk.argtypes = [ctypes.c_long, _D, _D, _D, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_int, ctypes.c_double, ctypes.c_int, _D, ctypes.c_int, _D]
            lib.orc_morton30.argtypes = [ctypes.c_long, _D, ctypes.c_double, _U32]
            lib.orc_morton30_compat.argtypes = [ctypes.c_long, _D, ctypes.c_double, _U32]
            lib.orc_morton63.argtypes = [ctypes.c_long, _D, ctypes.c_double, _U64]
            lib.orc_sort_codes.argtypes = [ctypes.c_long, _U64, ctypes.c_int, ctypes.c_int, _U64, _I32]
            lib.orc_karras.argtypes = [ctypes.c_long, _U64, _I32, ctypes.c_int, ctypes.c_int,
                                       _I32, _I32, _I32, _I32, _I32]
            lib.orc_bottom_up.argtypes = [ctypes.c_long, _I32, _I32, _I32, _D, _D, ctypes.c_double,
                                          _D, _D, _F, _F, _F]
            lib.orc_lbvh_forces.argtypes = [ctypes.c_long, ctypes.c_int, _I32, _I32, _I32, _I32, _I32, _I32,
                                            _D, _D, _D, _F, ctypes.c_double, ctypes.c_double, _D, _I32]
            lib.orc_node_velocities.argtypes = [ctypes.c_long, _I32, _I32, _I32, _D, _D, _D]
            lib.orc_lbvh_forces_pn.argtypes = [ctypes.c_long, ctypes.c_int, _I32, _I32, _I32, _I32, _I32, _I32,
                                               _D, _D, _D, _D, _D, _F, ctypes.c_double, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_int, _D, _I32]
            lib.orc_groups.argtypes = [ctypes.c_long, ctypes.c_int, _I32, _I32, _I32, _I32, _I32]
            lib.orc_groups.restype = ctypes.c_long
            lib.orc_set_threads.argtypes = [ctypes.c_int]
            _I64 = ctypes.POINTER(ctypes.c_int64)
            lib.orc_ens_run.argtypes = [ctypes.c_long, _I64, _D, _D, _D, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_long]
            lib.orc_eih_acc.argtypes = [ctypes.c_long, _D, _D, _D, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, _D]
            lib.orc_ens_energy.argtypes = [ctypes.c_long, _I64, _D, _D, _D, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_int, _D]
            Orc._lib = lib
        self.lib = Orc._lib

    def set_threads(self, t: int):
        self.lib.orc_set_threads(int(t))

    def pair_acc(self, G, inv_c, eps2, pn, m1, m2, v1, v2, p1, p2):
        a = np.zeros(3)
        args = [_c64(v1), _c64(v2), _c64(p1), _c64(p2)]
        self.lib.orc_pair_acc(G, inv_c, eps2, pn, m1, m2, *[_p(x, _D) for x in args], _p(a, _D))
        return a

    def allpairs(self, pos, m, G=1.0, eps2=0.0, vel=None, inv_c=0.0, pn=NEWTON, targets=None):
        pos, m = _c64(pos), _c64(m)
        vel = _c64(vel) if vel is not None else None
        n = len(m)
        tg = None if targets is None else np.ascontiguousarray(targets, dtype=np.int64)
        nt = n if tg is None else len(tg)
        acc = np.zeros((nt, 3))
        self.lib.orc_allpairs(n, _p(pos, _D), _p(vel, _D), _p(m, _D), G, inv_c, eps2, pn, nt,
                              _p(tg, _L) if tg is not None else None, _p(acc, _D))
        return acc

    def energy(self, pos, vel, m, G=1.0, eps2=0.0, ref_form=False):
        pos, vel, m = _c64(pos), _c64(vel), _c64(m)
        return self.lib.orc_energy(len(m), _p(pos, _D), _p(vel, _D), _p(m, _D), G, eps2, int(ref_form))

    def momentum(self, vel, m):
        vel, m = _c64(vel), _c64(m)
        p = np.zeros(3)
        self.lib.orc_momentum(len(m), _p(vel, _D), _p(m, _D), _p(p, _D))
        return p

    def saba_coeffs(self, order):
        """(drifts c[0..n], kicks d[0..n-1]) of SABA_order; order 1 is Euler."""
        c, d = np.zeros(11), np.zeros(10)
        nk = self.lib.orc_saba_coeffs(order, _p(c, _D), _p(d, _D))
        if nk < 0:
            raise ValueError("order must be 1..10")
        return c[:nk + 1].copy(), d[:nk].copy()

    def saba(self, pos, vel, m, dt, order, nsteps, G=1.0, eps2=0.0, inv_c=0.0, pn=NEWTON):
        """nsteps of SABA_order (the reference update_SABAn) with all-pairs
        forces; returns new (pos, vel)."""
        n = len(m)
        pos, vel, m = _c64(pos).copy(), _c64(vel).copy(), _c64(m)
        acc = np.zeros((n, 3))
        self.lib.orc_saba(n, _p(pos, _D), _p(vel, _D), _p(m, _D), G, inv_c, eps2, pn, dt, order, nsteps, _p(acc, _D))
        return pos, vel

    def wh(self, pos, vel, m, dt, nsteps, G=1.0, eps2=0.0):
        """nsteps of Wisdom-Holman (democratic heliocentric, body 0 central);
        returns new (pos, vel). Raises if a Kepler drift fails."""
        pos, vel, m = _c64(pos).copy(), _c64(vel).copy(), _c64(m)
        if self.lib.orc_wh(len(m), _p(pos, _D), _p(vel, _D), _p(m, _D), G, eps2, dt, nsteps) != 0:
            raise RuntimeError("orc_wh: Kepler drift failed or bad input")
        return pos, vel

    def kepler(self, r, v, mu, dt):
        r, v = _c64(r).copy(), _c64(v).copy()
        if self.lib.orc_kepler(_p(r, _D), _p(v, _D), mu, dt) != 0:
            raise RuntimeError("orc_kepler failed")
        return r, v

    def saba_seq(self, pos, vel, m, dt, c, d, nsteps, G=1.0, eps2=0.0, inv_c=0.0, pn=NEWTON):
        """nsteps of an explicit drift/kick sequence: drift c[0], then
        (forces, kick d[k], drift c[k+1]) for every k."""
        n = len(m)
        c, d = _c64(c), _c64(d)
        assert len(c) == len(d) + 1
        pos, vel, m = _c64(pos).copy(), _c64(vel).copy(), _c64(m)
        acc = np.zeros((n, 3))
        self.lib.orc_saba_seq(n, _p(pos, _D), _p(vel, _D), _p(m, _D), G, inv_c, eps2, pn, dt, len(d), _p(c, _D),
                              _p(d, _D), nsteps, _p(acc, _D))
        return pos, vel

    def kdk(self, pos, vel, m, dt, nsteps, G=1.0, eps2=0.0, inv_c=0.0, pn=NEWTON, record_acc=False):
        pos, vel, m = _c64(pos).copy(), _c64(vel).copy(), _c64(m)
        n = len(m)
        acc = np.zeros((n, 3))
        accs = np.zeros((nsteps, n, 3)) if record_acc else None
        self.lib.orc_kdk(n, _p(pos, _D), _p(vel, _D), _p(m, _D), G, inv_c, eps2, pn, dt, nsteps,
                         _p(acc, _D), 0, _p(accs, _D))
        return pos, vel, acc, accs

    def morton30(self, pos, B, compat=False):
        pos = _c64(pos)
        codes = np.zeros(len(pos), np.uint32)
        fn = self.lib.orc_morton30_compat if compat else self.lib.orc_morton30
        fn(len(pos), _p(pos, _D), B, _p(codes, _U32))
        return codes

    def morton63(self, pos, B):
        pos = _c64(pos)
        codes = np.zeros(len(pos), np.uint64)
        self.lib.orc_morton63(len(pos), _p(pos, _D), B, _p(codes, _U64))
        return codes

    def sort_codes(self, codes, bits=30, descending=False):
        c = np.ascontiguousarray(codes, dtype=np.uint64)
        n = len(c)
        s = np.zeros(n, np.uint64)
        perm = np.zeros(n, np.int32)
        self.lib.orc_sort_codes(n, _p(c, _U64), bits, int(descending), _p(s, _U64), _p(perm, _I32))
        return s, perm

    def karras(self, sorted_codes, perm, bits=30, compat=False):
        sc = np.ascontiguousarray(sorted_codes, dtype=np.uint64)
        perm = np.ascontiguousarray(perm, dtype=np.int32)
        n = len(sc)
        out = {k: np.zeros(2 * n - 1, np.int32) for k in ("left", "right", "parent", "range_lo", "range_hi")}
        self.lib.orc_karras(n, _p(sc, _U64), _p(perm, _I32), bits, int(compat),
                            *[_p(out[k], _I32) for k in ("left", "right", "parent", "range_lo", "range_hi")])
        return out

    def bottom_up(self, left, right, perm, pos, m, theta):
        n = len(m)
        pos, m = _c64(pos), _c64(m)
        nm = np.zeros(2 * n - 1)
        nc = np.zeros((2 * n - 1, 3))
        bmin = np.zeros((2 * n - 1, 3), np.float32)
        bmax = np.zeros((2 * n - 1, 3), np.float32)
        rc2 = np.zeros(2 * n - 1, np.float32)
        args = [np.ascontiguousarray(a, dtype=np.int32) for a in (left, right, perm)]
        self.lib.orc_bottom_up(n, *[_p(a, _I32) for a in args], _p(pos, _D), _p(m, _D), theta,
                               _p(nm, _D), _p(nc, _D), _p(bmin, _F), _p(bmax, _F), _p(rc2, _F))
        return dict(node_mass=nm, node_com=nc, bmin=bmin, bmax=bmax, rcrit2=rc2)

    def lbvh_forces(self, tree, perm, pos, G, eps2, group=64):
        """Group walk; returns (acc per body, list length per body), input order."""
        n = len(perm)
        pos = _c64(pos)
        acc = np.zeros((n, 3))
        cnt = np.zeros(n, np.int32)
        args = [np.ascontiguousarray(a, dtype=np.int32)
                for a in (tree["left"], tree["right"], tree["parent"], tree["range_lo"], tree["range_hi"], perm)]
        self.lib.orc_lbvh_forces(n, group, *[_p(a, _I32) for a in args], _p(pos, _D),
                                 _p(tree["node_mass"], _D), _p(tree["node_com"], _D), _p(tree["rcrit2"], _F),
                                 G, eps2, _p(acc, _D), _p(cnt, _I32))
        return acc, cnt

    def node_velocities(self, tree, perm, vel):
        """Per node (2n - 1, node order): leaves the sorted body velocities,
        internal nodes the mass-weighted mean of their children (unite form)."""
        n = len(perm)
        out = np.zeros((max(2 * n - 1, 1), 3))
        args = [np.ascontiguousarray(a, dtype=np.int32) for a in (tree["left"], tree["right"], perm)]
        self.lib.orc_node_velocities(n, *[_p(a, _I32) for a in args], _p(_c64(vel), _D),
                                     _p(np.ascontiguousarray(tree["node_mass"], dtype=np.float64), _D), _p(out, _D))
        return out

    def lbvh_forces_pn(self, tree, perm, pos, vel, G, eps2, inv_c, pn, group=64):
        """Group walk with a post-Newtonian force law (node velocities as
        node_velocities); returns (acc per body, list length per body)."""
        n = len(perm)
        pos, vel = _c64(pos), _c64(vel)
        nv = self.node_velocities(tree, perm, vel)
        acc = np.zeros((n, 3))
        cnt = np.zeros(n, np.int32)
        args = [np.ascontiguousarray(a, dtype=np.int32)
                for a in (tree["left"], tree["right"], tree["parent"], tree["range_lo"], tree["range_hi"], perm)]
        self.lib.orc_lbvh_forces_pn(n, group, *[_p(a, _I32) for a in args], _p(pos, _D), _p(vel, _D),
                                    _p(tree["node_mass"], _D), _p(tree["node_com"], _D), _p(nv, _D),
                                    _p(tree["rcrit2"], _F), G, inv_c, eps2, pn, _p(acc, _D), _p(cnt, _I32))
        return acc, cnt

    def groups(self, tree, group=64):
        n = (len(tree["left"]) + 1) // 2
        start = np.zeros(n, np.int32)
        count = np.zeros(n, np.int32)
        args = [np.ascontiguousarray(tree[k], dtype=np.int32) for k in ("parent", "range_lo", "range_hi")]
        ng = self.lib.orc_groups(n, group, *[_p(a, _I32) for a in args], _p(start, _I32), _p(count, _I32))
        return start[:ng], count[:ng]

    def lbvh(self, pos, m, theta, B=None, bits=30):
        """Full CPU LBVH build (Morton -> stable sort -> Karras -> bottom-up)."""
        if B is None:
            B = float(np.abs(pos).max())
        codes = self.morton30(pos, B).astype(np.uint64) if bits == 30 else self.morton63(pos, B)
        sc, perm = self.sort_codes(codes, bits=bits)
        t = self.karras(sc, perm, bits=bits)
        t.update(self.bottom_up(t["left"], t["right"], perm, pos, m, theta))
        t.update(codes=codes, sorted_codes=sc, perm=perm, box=B)
        return t

    # -- batched ensembles --------------------------------------------------
    def ens_run(self, offsets, pos, vel, m, dt, nsteps, G=1.0, c=None, eps2=0.0, integrator=1, pn=None):
        """Advance every system nsteps (integrator 1 = Yoshida-4, 0 = leapfrog).
        Force law `pn` (NEWTON | PN1 | PN2 | PN25); default NEWTON, plus PN1
        when c is given. Returns new (pos, vel)."""
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        pos, vel, m = _c64(pos).copy(), _c64(vel).copy(), _c64(m)
        if pn is None:
            pn = NEWTON | (PN1 if c else 0)
        inv_c = 1.0 / c if c else 0.0
        self.lib.orc_ens_run(len(off) - 1, off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), _p(pos, _D),
                             _p(vel, _D), _p(m, _D), G, inv_c, eps2, pn, integrator, dt, nsteps)
        return pos, vel

    def eih_acc(self, pos, vel, m, G=1.0, c=100.0, eps2=0.0):
        """Accelerations of one system (n <= 64) under Newton + the N-body
        Einstein-Infeld-Hoffmann 1PN terms."""
        pos, vel, m = _c64(pos), _c64(vel), _c64(m)
        acc = np.zeros((len(m), 3))
        self.lib.orc_eih_acc(len(m), _p(pos, _D), _p(vel, _D), _p(m, _D), G, 1.0 / c, eps2, _p(acc, _D))
        return acc

    def ens_energy(self, offsets, pos, vel, m, G=1.0, c=None, eps2=0.0, pn=None):
        """Newtonian energy, plus the 1PN energy when c is given: the sum of
        two-body terms for the pairwise law, the N-body EIH energy when pn
        carries EIH."""
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        pos, vel, m = _c64(pos), _c64(vel), _c64(m)
        e = np.zeros(len(off) - 1)
        if pn is None:
            pn = NEWTON | (PN1 if c else 0)
        inv_c = 1.0 / c if c else 0.0
        self.lib.orc_ens_energy(len(off) - 1, off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), _p(pos, _D),
                                _p(vel, _D), _p(m, _D), G, inv_c, eps2, pn, _p(e, _D))
        return e

    # -- adjoint -------------------------------------------------------------
    def adjoint(self, x0, v0, m, target, dt, nsteps, G=1.0, eps2=0.0):
        """FP64 reverse mode: (loss, dL/dx0, dL/dv0, dL/dm) of
        L = mean_i |x_T,i - target_i|^2 after nsteps KDK steps."""
        x0, v0, m, tg = _c64(x0), _c64(v0), _c64(m), _c64(target)
        n = len(m)
        gx, gv, gm = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n)
        f = self.lib.orc_adjoint
        f.restype = ctypes.c_double
        f.argtypes = [ctypes.c_long, _D, _D, _D, _D, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                      ctypes.c_long, _D, _D, _D]
        loss = f(n, _p(x0, _D), _p(v0, _D), _p(m, _D), _p(tg, _D), G, eps2, dt, nsteps, _p(gx, _D), _p(gv, _D),
                 _p(gm, _D))
        return loss, gx, gv, gm
