"""Python host side over the C ABI (include/aster_cuda.h), mirroring the
reference's Simulation / Solver / Updater interface for the hot path
(include/Aster/simulations/sim_obj.h:34-197).

* ``Context``: one-to-one wrapper of the C entry points (status codes become
  ``AsterError``).
* ``Simulation``: the slice of the reference Simulation the hot path touches:
  bodies (positions/velocities/masses/accs, AoS FP64 like BodyArray), G, c,
  dt, softening (= eps^2, added to r^2 exactly as the reference does), theta,
  force_law, solver/updater, step(), integrate(n, precision_test).
* ``CudaAllPairs`` / ``CudaLBVH`` (Solver) and ``CudaKDK`` (Updater): drop-in
  for Parallelized/SimpleGPU, Barnes_Hut/BH_hyper and update_leapfrog.

There is no CPU fallback: loading fails loudly if libaster_cuda.so or a CUDA
device is missing.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libaster_cuda.so"

OK = 0
NEWTON = 0x0001
PN1 = 0x0010
PN2 = 0x0100   # all-pairs solver and ensemble
PN25 = 0x1000  # all-pairs solver and ensemble
EIH = 0x10000  # with PN1, ensembles only: the N-body Einstein-Infeld-Hoffmann 1PN acceleration
UPDATER_KDK, UPDATER_SABA, UPDATER_WH = 0, 1, 2
COLLECT_ENERGY, COLLECT_ENERGY_ERROR, COLLECT_MOMENTUM, COLLECT_CENTER, COLLECT_DISTANCE = 0x1, 0x2, 0x4, 0x8, 0x10
FP64 = 0
MIXED = 1
SOLVER_ALLPAIRS = 0
SOLVER_LBVH = 1
LEAPFROG = 0
YOSHIDA4 = 1
ERR_CANCELLED = 8

EXPORTS = [
    "aster_strerror", "aster_version", "aster_ctx_create", "aster_ctx_destroy", "aster_state_upload",
    "aster_state_upload_acc", "aster_kdk_steps_host",
    "aster_state_download", "aster_state_size", "aster_allpairs", "aster_allpairs_range", "aster_allpairs_targets",
    "aster_lbvh_build",
    "aster_lbvh_forces", "aster_kdk_steps", "aster_saba_steps", "aster_wh_steps", "aster_record",
    "aster_record_columns", "aster_energy", "aster_get_stats", "aster_ensemble_upload",
    "aster_ensemble_download", "aster_ensemble_run", "aster_ensemble_energy", "aster_ensemble_cancel",
    "aster_adjoint_leapfrog",
]


class AsterError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: status {status} ({msg})")
        self.status = status


class CParams(ctypes.Structure):
    _fields_ = [("G", ctypes.c_double), ("c", ctypes.c_double), ("eps2", ctypes.c_double),
                ("theta", ctypes.c_double), ("dt", ctypes.c_double), ("force_law", ctypes.c_int32),
                ("morton_bits", ctypes.c_int32), ("compat_mode", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class CTreeView(ctypes.Structure):
    _fields_ = [("codes", ctypes.c_void_p), ("sorted_codes", ctypes.c_void_p), ("perm", ctypes.c_void_p),
                ("left", ctypes.c_void_p), ("right", ctypes.c_void_p), ("parent", ctypes.c_void_p),
                ("range_lo", ctypes.c_void_p), ("range_hi", ctypes.c_void_p), ("node_mass", ctypes.c_void_p),
                ("node_com", ctypes.c_void_p), ("node_bmin", ctypes.c_void_p), ("node_bmax", ctypes.c_void_p),
                ("node_rcrit2", ctypes.c_void_p), ("box", ctypes.c_double)]


class CEnsembleConfig(ctypes.Structure):
    _fields_ = [("warps_per_block", ctypes.c_int32), ("unroll", ctypes.c_int32), ("check_every", ctypes.c_int32),
                ("use_graph", ctypes.c_int32), ("schedule", ctypes.c_int32)]


class CRecordConfig(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int32) for k in ("updater", "order", "solver", "precision", "rate", "collect",
                                             "ref_form", "reserved")]


class CStats(ctypes.Structure):
    _fields_ = [("ms_total", ctypes.c_double), ("ms_force", ctypes.c_double), ("ms_build", ctypes.c_double),
                ("interactions", ctypes.c_double), ("max_stack", ctypes.c_int32), ("kernels", ctypes.c_int32)]


@dataclass
class Params:
    G: float = 1.0
    c: float = 299792458.0
    eps2: float = 0.0
    theta: float = 0.5
    dt: float = 1e-3
    force_law: int = NEWTON
    morton_bits: int = 30
    compat_mode: int = 0

    def c_struct(self) -> CParams:
        return CParams(self.G, self.c, self.eps2, self.theta, self.dt, self.force_law, self.morton_bits,
                       self.compat_mode, 0)


_lib = None


def load_library(path: Path | str | None = None) -> ctypes.CDLL:
    """Load libaster_cuda.so (raises if it is missing: no fallback path)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} not built: run `python -m aster_b200.build` (nvcc, sm_100a)")
    lib = ctypes.CDLL(str(p))
    vp, i32, i64, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    lib.aster_strerror.restype = ctypes.c_char_p
    lib.aster_strerror.argtypes = [ctypes.c_int]
    lib.aster_ctx_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, vp]
    lib.aster_ctx_destroy.argtypes = [vp]
    lib.aster_state_upload.argtypes = [vp, i64, vp, vp, vp]
    lib.aster_state_upload_acc.argtypes = [vp, i64, vp, vp, vp, vp]
    lib.aster_kdk_steps_host.argtypes = [vp, ctypes.POINTER(CParams), ctypes.c_int, ctypes.c_int, ctypes.c_int, i64,
                                         vp, vp, vp, vp]
    lib.aster_state_download.argtypes = [vp, vp, vp, vp]
    lib.aster_state_size.argtypes = [vp, ctypes.POINTER(i64)]
    lib.aster_allpairs.argtypes = [vp, ctypes.POINTER(CParams), ctypes.c_int, vp]
    lib.aster_allpairs_range.argtypes = [vp, ctypes.POINTER(CParams), ctypes.c_int, ctypes.c_int64, ctypes.c_int64,
                                         vp]
    lib.aster_allpairs_targets.argtypes = [vp, ctypes.POINTER(CParams), ctypes.c_int, i64, vp, vp]
    lib.aster_lbvh_build.argtypes = [vp, ctypes.POINTER(CParams), ctypes.POINTER(CTreeView)]
    lib.aster_lbvh_forces.argtypes = [vp, ctypes.POINTER(CParams), ctypes.c_int, vp, vp]
    lib.aster_kdk_steps.argtypes = [vp, ctypes.POINTER(CParams), ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.aster_saba_steps.argtypes = [vp, ctypes.POINTER(CParams), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int]
    lib.aster_wh_steps.argtypes = [vp, ctypes.POINTER(CParams), ctypes.c_int, ctypes.c_int]
    lib.aster_record_columns.restype = ctypes.c_int64
    lib.aster_record_columns.argtypes = [ctypes.POINTER(CRecordConfig), ctypes.c_int64]
    lib.aster_record.argtypes = [vp, ctypes.POINTER(CParams), ctypes.POINTER(CRecordConfig), ctypes.c_int64, vp]
    lib.aster_energy.argtypes = [vp, ctypes.POINTER(CParams), ctypes.c_int, ctypes.POINTER(dbl), vp]
    lib.aster_get_stats.argtypes = [vp, ctypes.POINTER(CStats)]
    lib.aster_ensemble_upload.argtypes = [vp, ctypes.c_int32, vp, vp, vp, vp]
    lib.aster_ensemble_download.argtypes = [vp, vp, vp]
    lib.aster_ensemble_run.argtypes = [vp, ctypes.POINTER(CParams), ctypes.c_int, ctypes.c_int, i64,
                                       ctypes.POINTER(CEnsembleConfig)]
    lib.aster_ensemble_energy.argtypes = [vp, ctypes.POINTER(CParams), vp]
    lib.aster_ensemble_cancel.argtypes = [vp]
    lib.aster_adjoint_leapfrog.argtypes = [vp, ctypes.POINTER(CParams), ctypes.c_int, i64, ctypes.c_int32, vp,
                                           ctypes.POINTER(dbl), vp, vp, vp]
    for name in EXPORTS:
        if not hasattr(lib, name):
            raise ImportError(f"{p} lacks {name}")
    if path is None:
        _lib = lib
    return lib


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _aos(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if n is not None and a.shape != (n, 3):
        raise ValueError(f"expected ({n}, 3), got {a.shape}")
    return a


class Context:
    """A device context holding one body state (one GPU, one stream)."""

    def __init__(self, device: int = 0, stream: int | None = None, lib=None):
        self.lib = lib or load_library()
        h = ctypes.c_void_p()
        self._check(self.lib.aster_ctx_create(ctypes.byref(h), device, stream), "aster_ctx_create")
        self.h = h
        self.n = 0
        self.device = device

    def _check(self, st: int, where: str):
        if st != OK:
            raise AsterError(st, where, self.lib.aster_strerror(st).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.aster_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state -----------------------------------------------------------
    def upload(self, pos, vel, mass, acc=None):
        """State to the device; acc (the bodies' current accelerations) becomes
        the cached acceleration when given."""
        n = len(mass)
        pos = _aos(pos, n)
        vel = None if vel is None else _aos(vel, n)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        if acc is None:
            self._check(self.lib.aster_state_upload(self.h, n, _ptr(pos), _ptr(vel), _ptr(mass)), "aster_state_upload")
        else:
            acc = _aos(acc, n)
            self._check(self.lib.aster_state_upload_acc(self.h, n, _ptr(pos), _ptr(vel), _ptr(mass), _ptr(acc)),
                        "aster_state_upload_acc")
        self.n = n
        return self

    def download(self):
        pos, vel, acc = (np.empty((self.n, 3)) for _ in range(3))
        self._check(self.lib.aster_state_download(self.h, _ptr(pos), _ptr(vel), _ptr(acc)), "aster_state_download")
        return pos, vel, acc

    # -- forces ----------------------------------------------------------
    def allpairs(self, p: Params, precision: int = FP64):
        acc = np.empty((self.n, 3))
        cp = p.c_struct()
        self._check(self.lib.aster_allpairs(self.h, ctypes.byref(cp), precision, _ptr(acc)), "aster_allpairs")
        return acc

    def allpairs_range(self, p: Params, lower: int, upper: int = -1, precision: int = FP64):
        """Accelerations of every body from the sources [lower, upper) only
        (upper = -1: to the end), as Parallelized sums over set_bounds."""
        acc = np.empty((self.n, 3))
        cp = p.c_struct()
        self._check(self.lib.aster_allpairs_range(self.h, ctypes.byref(cp), precision, lower, upper, _ptr(acc)),
                    "aster_allpairs_range")
        return acc

    def allpairs_targets(self, p: Params, targets, precision: int = FP64):
        tg = np.ascontiguousarray(targets, dtype=np.int32)
        acc = np.empty((len(tg), 3))
        cp = p.c_struct()
        self._check(self.lib.aster_allpairs_targets(self.h, ctypes.byref(cp), precision, len(tg), _ptr(tg),
                                                    _ptr(acc)), "aster_allpairs_targets")
        return acc

    def lbvh_build(self, p: Params, export: bool = True):
        n, m = self.n, 2 * self.n - 1
        cp = p.c_struct()
        if not export:
            self._check(self.lib.aster_lbvh_build(self.h, ctypes.byref(cp), None), "aster_lbvh_build")
            return None
        out = dict(codes=np.empty(n, np.uint64), sorted_codes=np.empty(n, np.uint64), perm=np.empty(n, np.int32),
                   left=np.empty(m, np.int32), right=np.empty(m, np.int32), parent=np.empty(m, np.int32),
                   range_lo=np.empty(m, np.int32), range_hi=np.empty(m, np.int32), node_mass=np.empty(m),
                   node_com=np.empty((m, 3)), node_bmin=np.empty((m, 3), np.float32),
                   node_bmax=np.empty((m, 3), np.float32), node_rcrit2=np.empty(m, np.float32))
        v = CTreeView(**{k: a.ctypes.data for k, a in out.items()}, box=0.0)
        self._check(self.lib.aster_lbvh_build(self.h, ctypes.byref(cp), ctypes.byref(v)), "aster_lbvh_build")
        out["box"] = v.box
        return out

    def lbvh_forces(self, p: Params, precision: int = MIXED, list_counts: bool = False):
        """Accelerations (n,3); with list_counts also the interaction-list
        length of each body's group (n,), input order."""
        acc = np.empty((self.n, 3))
        gc = np.empty(self.n, np.int32) if list_counts else None
        cp = p.c_struct()
        self._check(self.lib.aster_lbvh_forces(self.h, ctypes.byref(cp), precision, _ptr(acc), _ptr(gc)),
                    "aster_lbvh_forces")
        return (acc, gc) if list_counts else acc

    def kdk_steps(self, p: Params, nsteps: int, solver: int = SOLVER_ALLPAIRS, precision: int = FP64):
        cp = p.c_struct()
        self._check(self.lib.aster_kdk_steps(self.h, ctypes.byref(cp), solver, precision, nsteps), "aster_kdk_steps")

    def record(self, p: Params, nsteps: int, *, updater: int = UPDATER_KDK, order: int = 4,
               solver: int = SOLVER_ALLPAIRS, precision: int = FP64, rate: int = 1,
               collect: int = COLLECT_ENERGY, ref_form: bool = True):
        """Step nsteps on the device, sampling every `rate` steps (and at step
        0). Returns (rows, names): rows[k] = [step, columns...] as in the
        reference's Graph CSV files; names are the column names."""
        cfg = CRecordConfig(updater, order, solver, precision, rate, collect, int(ref_form), 0)
        ncol = self.lib.aster_record_columns(ctypes.byref(cfg), self.n)
        if ncol < 1:
            raise AsterError(1, "aster_record_columns", "invalid argument")
        rows = np.empty((nsteps // max(rate, 1) + 1, ncol))
        cp = p.c_struct()
        self._check(self.lib.aster_record(self.h, ctypes.byref(cp), ctypes.byref(cfg), nsteps, _ptr(rows)),
                    "aster_record")
        names = ["time"]
        if collect & COLLECT_ENERGY:
            names.append("energy")
        if collect & COLLECT_ENERGY_ERROR:
            names.append("energy_error")
        if collect & COLLECT_MOMENTUM:
            names += ["px", "py", "pz"]
        if collect & COLLECT_CENTER:
            names += ["x_cm", "y_cm", "z_cm"]
        if collect & COLLECT_DISTANCE:
            names += [f"Body{i}" for i in range(self.n)]
        return rows, names

    def wh_steps(self, p: Params, nsteps: int, precision: int = FP64):
        """nsteps of the Wisdom-Holman planetary integrator (body 0 central)."""
        cp = p.c_struct()
        self._check(self.lib.aster_wh_steps(self.h, ctypes.byref(cp), precision, nsteps), "aster_wh_steps")

    def kdk_steps_host(self, p: Params, nsteps: int, pos, vel, acc, mass, solver: int = SOLVER_ALLPAIRS,
                       precision: int = FP64):
        """Host-resident loop in one call: uploads (pos, vel, mass, acc), takes
        nsteps KDK steps and writes pos, vel, acc back in place (float64
        C-contiguous (n, 3) arrays; acc = the accelerations of pos)."""
        n = len(mass)
        for a in (pos, vel, acc):
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.shape != (n, 3):
                raise ValueError("pos, vel, acc must be C-contiguous float64 (n, 3) arrays")
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        cp = p.c_struct()
        self._check(self.lib.aster_kdk_steps_host(self.h, ctypes.byref(cp), solver, precision, nsteps, n, _ptr(pos),
                                                  _ptr(vel), _ptr(acc), _ptr(mass)), "aster_kdk_steps_host")
        self.n = n

    def saba_steps(self, p: Params, order: int, nsteps: int, solver: int = SOLVER_ALLPAIRS, precision: int = FP64):
        """nsteps of SABA_order (1..10; order 1 is the reference's Euler step)."""
        cp = p.c_struct()
        self._check(self.lib.aster_saba_steps(self.h, ctypes.byref(cp), solver, precision, order, nsteps),
                    "aster_saba_steps")

    def energy(self, p: Params, ref_form: bool = False):
        e = ctypes.c_double()
        mom = np.empty(3)
        cp = p.c_struct()
        self._check(self.lib.aster_energy(self.h, ctypes.byref(cp), int(ref_form), ctypes.byref(e), _ptr(mom)),
                    "aster_energy")
        return e.value, mom

    def stats(self) -> dict:
        s = CStats()
        self._check(self.lib.aster_get_stats(self.h, ctypes.byref(s)), "aster_get_stats")
        return {k: getattr(s, k) for k, _ in CStats._fields_}

    # -- batched ensembles ---------------------------------------------------
    def ensemble_upload(self, offsets, pos, vel, mass):
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        nb = int(off[-1])
        pos = _aos(pos, nb)
        vel = None if vel is None else _aos(vel, nb)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        self._check(self.lib.aster_ensemble_upload(self.h, len(off) - 1, _ptr(off), _ptr(pos), _ptr(vel),
                                                   _ptr(mass)), "aster_ensemble_upload")
        self.ens_nsys, self.ens_nbodies = len(off) - 1, nb
        self._ens_mass = mass.copy()
        return self

    def ensemble_download(self):
        pos, vel = np.empty((self.ens_nbodies, 3)), np.empty((self.ens_nbodies, 3))
        self._check(self.lib.aster_ensemble_download(self.h, _ptr(pos), _ptr(vel)), "aster_ensemble_download")
        return pos, vel

    def ensemble_run(self, p: Params, nsteps: int, integrator: int = YOSHIDA4, precision: int = MIXED,
                     config: dict | None = None):
        cp = p.c_struct()
        cfg = None
        if config is not None:
            cfg = CEnsembleConfig(config.get("warps_per_block", 0), config.get("unroll", 0),
                                  config.get("check_every", 0), int(config.get("use_graph", 1)),
                                  int(config.get("schedule", 0)))
        self._check(self.lib.aster_ensemble_run(self.h, ctypes.byref(cp), integrator, precision, nsteps,
                                                ctypes.byref(cfg) if cfg is not None else None),
                    "aster_ensemble_run")

    def ensemble_energy(self, p: Params):
        e = np.empty(self.ens_nsys)
        cp = p.c_struct()
        self._check(self.lib.aster_ensemble_energy(self.h, ctypes.byref(cp), _ptr(e)), "aster_ensemble_energy")
        return e

    def ensemble_cancel(self):
        self._check(self.lib.aster_ensemble_cancel(self.h), "aster_ensemble_cancel")

    # -- adjoint ---------------------------------------------------------------
    def adjoint(self, p: Params, nsteps: int, target, precision: int = MIXED, checkpoint_every: int = 32):
        """Loss L = mean_i |x_T,i - target_i|^2 after nsteps KDK steps from the
        uploaded state and (dL/dx0, dL/dv0, dL/dm). The state is unchanged."""
        tg = _aos(target, self.n)
        gx, gv, gm = np.empty((self.n, 3)), np.empty((self.n, 3)), np.empty(self.n)
        loss = ctypes.c_double()
        cp = p.c_struct()
        self._check(self.lib.aster_adjoint_leapfrog(self.h, ctypes.byref(cp), precision, nsteps, checkpoint_every,
                                                    _ptr(tg), ctypes.byref(loss), _ptr(gx), _ptr(gv), _ptr(gm)),
                    "aster_adjoint_leapfrog")
        return loss.value, gx, gv, gm


# ---------------------------------------------------------------------------
# Reference-shaped interface (sim_obj.h): Simulation, Solver, Updater
# ---------------------------------------------------------------------------
class BodyArray:
    """AoS FP64 body state (include/Aster/physics/body.h:9-24)."""

    def __init__(self, positions, velocities, masses):
        self.positions = _aos(positions).copy()
        self.velocities = _aos(velocities).copy()
        self.masses = np.ascontiguousarray(masses, dtype=np.float64).copy()
        self.accs = np.zeros_like(self.positions)


class Solver:
    """Mirror of Aster::Solver (sim_obj.h:34-61): load(), compute_forces()
    fills sim.bodies.accs with ACCELERATIONS, force_law bitmask."""

    precision = FP64

    def __init__(self, sim: "Simulation", precision: int | None = None):
        self._s = sim
        self.force_law = sim.force_law
        if precision is not None:
            self.precision = precision

    def load(self):
        self._s._ensure_uploaded()

    def compute_forces(self):
        raise NotImplementedError


class CudaAllPairs(Solver):
    """Replaces Parallelized / SimpleGPU (builder_endpoint.cpp:729-757,
    SimpleGPU.cpp:17-71)."""

    kind = SOLVER_ALLPAIRS

    def compute_forces(self):
        s = self._s
        s._ensure_uploaded()
        s.bodies.accs[:] = s.ctx.allpairs(s.params(self.force_law), self.precision)


class CudaLBVH(Solver):
    """Replaces Barnes_Hut / BH_hyper (barnes_hut.cpp:402-418,
    full_GPU.cpp:519-527). Mixed precision by default."""

    kind = SOLVER_LBVH
    precision = MIXED

    def compute_forces(self):
        s = self._s
        s._ensure_uploaded()
        s.bodies.accs[:] = s.ctx.lbvh_forces(s.params(self.force_law), self.precision)


class Updater:
    """Mirror of Aster::Updater (sim_obj.h:64-77)."""

    def __init__(self, sim: "Simulation"):
        self._s = sim

    def update_bodies(self):
        raise NotImplementedError


class CudaKDK(Updater):
    """Replaces update_leapfrog(_gpu_3d) (tool_chain_impl.cpp:169-185,
    updater.cpp:53-87): one kick-drift-kick step, force evaluated once."""

    def update_bodies(self, nsteps: int = 1):
        s = self._s
        s._ensure_uploaded()
        sol = s.solver
        s.ctx.kdk_steps(s.params(sol.force_law), nsteps, sol.kind, sol.precision)
        s._device_newer = True


class CudaSABA(Updater):
    """Replaces update_SABA1..10 (src/integrators/SABA.cpp:14-553) and the
    OpenCL SABA updater (tc_impl_cl.cpp:269-299) for order 1..10, the
    Laskar-Robutel sequence with n force evaluations per step."""

    def __init__(self, sim: "Simulation", order: int = 4):
        super().__init__(sim)
        if not 1 <= order <= 10:
            raise ValueError("SABA order must be 1..10")
        self.order = order

    def update_bodies(self, nsteps: int = 1):
        s = self._s
        s._ensure_uploaded()
        sol = s.solver
        s.ctx.saba_steps(s.params(sol.force_law), self.order, nsteps, sol.kind, sol.precision)
        s._device_newer = True


class CudaWH(Updater):
    """Replaces update_WH_planetary (tool_chain_impl.cpp:186-290) and its
    OpenCL form (WH_planetary.cl.h): Wisdom-Holman with body 0 as the central
    mass, the interaction from the solver's all-pairs kernel at its precision."""

    def update_bodies(self, nsteps: int = 1):
        s = self._s
        s._ensure_uploaded()
        s.ctx.wh_steps(s.params(NEWTON), nsteps, s.solver.precision)
        s._device_newer = True


class Simulation:
    """The part of Aster::Simulation that the hot path touches."""

    def __init__(self, positions, velocities, masses, G=1.0, c=299792458.0, dt=1e-3, softening=0.0,
                 theta=0.5, force_law=NEWTON, device=0):
        self.bodies = BodyArray(positions, velocities, masses)
        self.G, self.c, self.dt = G, c, dt
        self.softening, self.theta, self.force_law = softening, theta, force_law
        self.morton_bits, self.compat_mode = 30, 0
        self.always_read_pos = True
        self.ctx = Context(device)
        self.solver: Solver = CudaAllPairs(self)
        self.updater: Updater = CudaKDK(self)
        self._uploaded = False
        self._device_newer = False
        self.time_passed = 0

    def params(self, force_law=None) -> Params:
        return Params(G=self.G, c=self.c, eps2=self.softening, theta=self.theta, dt=self.dt,
                      force_law=self.force_law if force_law is None else force_law,
                      morton_bits=self.morton_bits, compat_mode=self.compat_mode)

    def _ensure_uploaded(self):
        if not self._uploaded:
            b = self.bodies
            self.ctx.upload(b.positions, b.velocities, b.masses)
            self._uploaded = True

    def load(self):
        self.solver.load()
        return self

    def read_bodies_gpu(self):
        if self._device_newer:
            pos, vel, acc = self.ctx.download()
            self.bodies.positions[:], self.bodies.velocities[:], self.bodies.accs[:] = pos, vel, acc
            self._device_newer = False
        return self

    def step(self):
        self.updater.update_bodies()
        if self.always_read_pos:
            self.read_bodies_gpu()
        self.time_passed += 1

    def get_total_energy(self) -> float:
        self._ensure_uploaded()
        return self.ctx.energy(self.params())[0]

    def integrate(self, n: int, precision_test: bool = False) -> dict:
        """n steps in one call (device resident); returns the reference's
        IntegrationReport fields (sim_obj.h:80-87)."""
        self._ensure_uploaded()
        e0 = self.get_total_energy() if precision_test else 0.0
        self.updater.update_bodies(n)
        st = self.ctx.stats()
        e1 = self.get_total_energy() if precision_test else 0.0
        self.read_bodies_gpu()
        self.time_passed += n
        prec = abs(e1 - e0) / abs(e0) if (precision_test and e0) else 0.0
        return dict(total_time=st["ms_total"], time_per_step=st["ms_total"] / max(n, 1), initial_energy=e0,
                    final_energy=e1, precision=prec, tested_precision=precision_test)


def graph_csv(times, values) -> str:
    """CSV text in the layout of the reference's Graph files
    (src/utils/graph_collection.cpp:60-150): one value per sample ->
    "time,data" rows; one value per body per sample (FOR_EACH) -> header
    "time,Body0,...,Body{n-1}," and rows "t,v0,...,v{n-1}"."""
    times = np.asarray(times)
    values = np.asarray(values)
    out = []
    if values.ndim == 1:
        out.append("time,data\n")
        out += [f"{int(t)},{v!r}\n" for t, v in zip(times, values.tolist())]
    else:
        out.append("time," + "".join(f"Body{i}," for i in range(values.shape[1])) + "\n")
        out += [f"{int(t)}," + ",".join(repr(x) for x in row) + "\n" for t, row in zip(times, values.tolist())]
    return "".join(out)
