"""ctypes binding of libcipc_gpu.so (include/cipc_gpu.h) and the synthetic
scene builders of the benchmark configurations.

The library is the product; this module is the thin host-side front end the
tests, bench.py and the headless runner use.  Loading fails loudly when the
shared library is missing - there is no CPU fallback.
"""
import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcipc_gpu.so")

CIPC_OK = 0
ERRORS = {1: "invalid argument", 2: "runtime error", 3: "CUDA error", 4: "PCG not converged", 5: "device status"}
LINEAR_GPU_PCG = 3
PRECISION = {"fp64": 0, "mixed": 1}
PRECOND = {"jacobi": 0, "learned": 1, "fsai": 2}
MOTION_NONE, MOTION_TWIST_X = 0, 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class LinearOptions(C.Structure):
    _fields_ = [("backend", C.c_int), ("precision", C.c_int), ("preconditioner", C.c_int),
                ("relativeTolerance", C.c_double), ("maximumIterations", C.c_int)]


class SceneDesc(C.Structure):
    _fields_ = [
        ("nv", C.c_int), ("nt", C.c_int), ("nf", C.c_int),
        ("x", _dp), ("vel", _dp), ("tets", _ip), ("tris", _ip), ("btype", _ip), ("tetE", _dp),
        ("density", C.c_double), ("cloth_density", C.c_double), ("thickness", C.c_double), ("E", C.c_double),
        ("nu", C.c_double), ("clothE", C.c_double), ("shearE", C.c_double), ("bendE", C.c_double),
        ("strainRate", C.c_double), ("friction", C.c_double),
        ("dt", C.c_double), ("drag", C.c_double), ("newtonThr", C.c_double), ("relDhat", C.c_double),
        ("use_barrier", C.c_int), ("apply_gravity", C.c_int), ("quasi_static", C.c_int), ("quad_bending", C.c_int),
        ("bboxMin", C.c_double * 3), ("bboxMax", C.c_double * 3),
        ("nsoft", C.c_int), ("softIdx", _ip), ("softW", C.c_double), ("softMotion", C.c_int), ("softRate", C.c_double),
        ("ndir", C.c_int), ("dirIdx", _ip), ("dirMotion", C.c_int), ("dirRate", C.c_double),
        ("nsf", C.c_int), ("nsv", C.c_int), ("nse", C.c_int),
        ("surfFaces", _ip), ("surfVerts", _ip), ("surfEdges", _ip),
    ]


class StepStats(C.Structure):
    _fields_ = [
        ("frame", C.c_int), ("newtonIterations", C.c_int), ("kappaIterations", C.c_int), ("lineSearchBacktracks", C.c_int),
        ("energyBacktracks", C.c_int), ("intersectionBacktracks", C.c_int), ("maximumEnergyBacktracksPerNewton", C.c_int),
        ("newtonStepsWithMoreThanTwoBacktracks", C.c_int),
        ("stepMilliseconds", C.c_double), ("assemblyMilliseconds", C.c_double), ("linearSolveMilliseconds", C.c_double),
        ("ccdMilliseconds", C.c_double), ("lineSearchMilliseconds", C.c_double), ("postLineSearchMilliseconds", C.c_double),
        ("collisions", C.c_double), ("kappa", C.c_double), ("minConstraintDistance2", C.c_double),
        ("acceptedStepSum", C.c_double), ("minimumAcceptedStep", C.c_double), ("maximumAcceptedStep", C.c_double),
        ("groundContacts", C.c_longlong), ("selfContacts", C.c_longlong), ("mollifiedContacts", C.c_longlong),
        ("matrixBlocks", C.c_longlong), ("pcgIterations", C.c_longlong), ("pcgRelativeResidual", C.c_double),
    ]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


_lib = None


def lib():
    """Load libcipc_gpu.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with python cpu-ipc_b200/build.py")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.cipc_gpu_create.argtypes = [C.POINTER(SceneDesc), C.POINTER(LinearOptions), C.POINTER(vp)]
        L.cipc_gpu_destroy.argtypes = [vp]
        L.cipc_gpu_last_error.restype = C.c_char_p
        L.cipc_gpu_last_error.argtypes = [vp]
        L.cipc_gpu_create_error.restype = C.c_char_p
        L.cipc_gpu_step.argtypes = [vp, C.POINTER(StepStats)]
        L.cipc_gpu_get_state.argtypes = [vp, C.c_int, _dp]
        L.cipc_gpu_set_state.argtypes = [vp, C.c_int, _dp]
        L.cipc_gpu_get_scalars.argtypes = [vp, _dp]
        L.cipc_gpu_set_kappa.argtypes = [vp, C.c_double]
        L.cipc_gpu_set_intersection_rule.argtypes = [vp, C.c_int]
        L.cipc_gpu_set_broad_phase.argtypes = [vp, C.c_int]
        L.cipc_gpu_set_online_training.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.c_ulonglong]
        L.cipc_gpu_set_system_dump.argtypes = [vp, C.c_char_p]
        L.cipc_gpu_hook_systems.argtypes = [vp, C.POINTER(C.c_longlong)]
        L.cipc_gpu_host_syncs.argtypes = [vp, C.POINTER(C.c_longlong)]
        L.cipc_gpu_get_counts.argtypes = [vp, C.POINTER(C.c_longlong)]
        L.cipc_gpu_get_surface.argtypes = [vp, _ip, _ip, _ip]
        L.cipc_gpu_build_collision_sets.argtypes = [vp, C.POINTER(C.c_longlong)]
        L.cipc_gpu_get_active_sets.argtypes = [vp, _ip, _ip, _ip, _ip, _ip]
        L.cipc_gpu_friction_init.argtypes = [vp]
        L.cipc_gpu_assemble.argtypes = [vp, _dp, _ip]
        L.cipc_gpu_export_matrix.argtypes = [vp, C.POINTER(C.c_longlong), _ip, _ip, _dp]
        L.cipc_gpu_solve.argtypes = [vp, _dp, _ip, _dp]
        L.cipc_gpu_energy.argtypes = [vp, C.c_double, _dp]
        L.cipc_gpu_step_bounds.argtypes = [vp, _dp, C.c_double, _dp]
        L.cipc_gpu_intersected.argtypes = [vp, _ip]
        L.cipc_gpu_pcg_bsr.argtypes = [C.c_int, _ip, _ip, _dp, _dp, _dp, C.POINTER(LinearOptions), _ip, _dp, C.c_char_p, C.c_int]
        L.cipc_gpu_accd.argtypes = [C.c_int, _ip, _dp, _dp, C.c_double, _dp, C.c_char_p, C.c_int]
        L.cipc_gpu_timed_steps.argtypes = [vp, C.c_int, C.POINTER(StepStats), _dp]
        L.cipc_gpu_profile.argtypes = [vp, C.c_int, C.c_int]
        L.cipc_gpu_profile_read.argtypes = [vp, C.POINTER(C.c_longlong), _dp]
        L.cipc_gpu_kernel_launches.restype = C.c_longlong
        _fp = C.POINTER(C.c_float)
        L.cipc_gpu_export_bsr.argtypes = [vp, _ip, _ip, _ip, _dp, _ip, _ip, _ip, _dp, _dp]
        L.cipc_gpu_precond_num_params.restype = C.c_int
        L.cipc_gpu_precond_set_weights.argtypes = [vp, _fp, C.c_int]
        L.cipc_gpu_precond_get_weights.argtypes = [vp, _fp, C.c_int]
        L.cipc_gpu_precond_loss.argtypes = [vp, C.c_int, _fp, C.c_ulonglong, _dp, _fp]
        L.cipc_gpu_precond_train.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.c_ulonglong, _dp, _dp]
        L.cipc_gpu_precond_stats.argtypes = [vp, C.POINTER(C.c_longlong)]
        L.cipc_gpu_precond_factor.argtypes = [vp, C.c_int, _fp, _fp]
        L.cipc_gpu_pcg_bsr_noalloc.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int,
                                               C.c_void_p, _ip, _dp]
        _lib = L
    return _lib


EXPORTED_SYMBOLS = [
    "cipc_gpu_create", "cipc_gpu_destroy", "cipc_gpu_last_error", "cipc_gpu_create_error", "cipc_gpu_step",
    "cipc_gpu_get_state", "cipc_gpu_set_state", "cipc_gpu_get_scalars", "cipc_gpu_set_kappa", "cipc_gpu_set_intersection_rule", "cipc_gpu_set_broad_phase", "cipc_gpu_get_counts",
    "cipc_gpu_get_surface", "cipc_gpu_build_collision_sets", "cipc_gpu_get_active_sets", "cipc_gpu_friction_init",
    "cipc_gpu_assemble", "cipc_gpu_export_matrix", "cipc_gpu_solve", "cipc_gpu_energy", "cipc_gpu_step_bounds",
    "cipc_gpu_intersected", "cipc_gpu_accd", "cipc_gpu_pcg_bsr", "cipc_gpu_timed_steps", "cipc_gpu_profile", "cipc_gpu_profile_read",
    "cipc_gpu_kernel_launches", "cipc_gpu_pcg_bsr_noalloc", "cipc_gpu_export_bsr", "cipc_gpu_precond_num_params",
    "cipc_gpu_precond_set_weights", "cipc_gpu_precond_get_weights", "cipc_gpu_precond_loss", "cipc_gpu_precond_train",
    "cipc_gpu_precond_stats", "cipc_gpu_precond_factor", "cipc_gpu_set_online_training", "cipc_gpu_set_system_dump",
    "cipc_gpu_hook_systems", "cipc_gpu_host_syncs",
]
NOALLOC_MAX_ROWS = 32768

PROFILE_KINDS = {"spmv": 1, "tet": 2, "tri": 3, "slot": 4, "barrier": 5, "active": 6, "fullccd": 7, "pcg": 8}


def kernel_launches():
    return int(lib().cipc_gpu_kernel_launches())


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class CipcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, 'error')} ({code}): {msg}")
        self.code = code


def linear_options(precision="fp64", precond="jacobi", tol=1e-6, max_iter=10000):
    return LinearOptions(LINEAR_GPU_PCG, PRECISION[precision], PRECOND[precond], tol, max_iter)


def scene_desc(scene, surface=None):
    """Build the cipc_scene_desc of a scene dict; returns (desc, arrays to keep alive)."""
    keep = []
    d = SceneDesc()
    x = np.ascontiguousarray(scene["x"], np.float64).reshape(-1)
    tets = np.ascontiguousarray(scene.get("tets", np.zeros((0, 4))), np.int32).reshape(-1)
    tris = np.ascontiguousarray(scene.get("tris", np.zeros((0, 3))), np.int32).reshape(-1)
    bt = np.ascontiguousarray(scene["btype"], np.int32)
    keep += [x, tets, tris, bt]
    d.nv, d.nt, d.nf = len(x) // 3, len(tets) // 4, len(tris) // 3
    d.x, d.tets, d.tris, d.btype = _d(x), _i(tets), _i(tris), _i(bt)
    if scene.get("vel") is not None:
        v = np.ascontiguousarray(scene["vel"], np.float64).reshape(-1)
        keep.append(v)
        d.vel = _d(v)
    if scene.get("tetE") is not None:
        te = np.ascontiguousarray(scene["tetE"], np.float64)
        keep.append(te)
        d.tetE = _d(te)
    p = scene["params"]
    for k in ("density", "cloth_density", "thickness", "E", "nu", "clothE", "shearE", "bendE", "strainRate",
              "friction", "dt", "drag", "newtonThr", "relDhat"):
        setattr(d, k, float(p[k]))
    d.use_barrier = int(p.get("use_barrier", 1))
    d.apply_gravity = int(p.get("apply_gravity", 1))
    d.quasi_static = int(p.get("quasi_static", 0))
    d.quad_bending = int(p.get("quad_bending", 1))
    for k in range(3):
        d.bboxMin[k] = scene["bbox_min"][k]
        d.bboxMax[k] = scene["bbox_max"][k]
    soft = scene.get("soft")
    if soft:
        si = np.ascontiguousarray(soft["idx"], np.int32)
        keep.append(si)
        d.nsoft, d.softIdx, d.softW = len(si), _i(si), float(soft["weight"])
        d.softMotion, d.softRate = int(soft.get("motion", 0)), float(soft.get("rate", 0.0))
    dirc = scene.get("dirichlet")
    if dirc:
        di = np.ascontiguousarray(dirc["idx"], np.int32)
        keep.append(di)
        d.ndir, d.dirIdx = len(di), _i(di)
        d.dirMotion, d.dirRate = int(dirc.get("motion", 0)), float(dirc.get("rate", 0.0))
    if surface is not None:
        f, sv, e = [np.ascontiguousarray(a, np.int32).reshape(-1) for a in surface]
        keep += [f, sv, e]
        d.nsf, d.nsv, d.nse = len(f) // 3, len(sv), len(e) // 2
        d.surfFaces, d.surfVerts, d.surfEdges = _i(f), _i(sv), _i(e)
    return d, keep


class Simulator:
    """One GPU context (FEMSimulator + IPCSolverContext equivalent)."""

    STATE = {"x": 0, "vel": 1, "vprev": 2, "xtilde": 3, "rest": 4}

    def __init__(self, scene, precision="fp64", precond="jacobi", tol=1e-6, max_iter=10000, surface=None):
        L = lib()
        self.L = L
        d, self._keep = scene_desc(scene, surface)
        self.opts = linear_options(precision, precond, tol, max_iter)
        h = C.c_void_p()
        rc = L.cipc_gpu_create(C.byref(d), C.byref(self.opts), C.byref(h))
        if rc != CIPC_OK:
            raise CipcError(rc, L.cipc_gpu_create_error().decode())
        self.h = h
        c = self.counts()
        self.nv, self.nsf, self.nsv, self.nse, self.nbend, self.nt, self.nf, self.nnzb = c[:8]

    def counts(self):
        """[nv, nsf, nsv, nse, nbend, nt, nf, static BSR blocks, contact BSR blocks]"""
        c = (C.c_longlong * 9)()
        self._chk(self.L.cipc_gpu_get_counts(self.h, c))
        return [int(v) for v in c]

    def _chk(self, rc):
        if rc != CIPC_OK:
            raise CipcError(rc, self.L.cipc_gpu_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.cipc_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def step(self):
        st = StepStats()
        self._chk(self.L.cipc_gpu_step(self.h, C.byref(st)))
        return st.as_dict()

    def timed_steps(self, n):
        """Run n steps; returns (device milliseconds from CUDA events on the context's stream, last stats)."""
        st = StepStats()
        ms = C.c_double(0)
        self._chk(self.L.cipc_gpu_timed_steps(self.h, int(n), C.byref(st), C.byref(ms)))
        return ms.value, st.as_dict()

    def profile(self, kind, capacity=100000):
        self._chk(self.L.cipc_gpu_profile(self.h, PROFILE_KINDS.get(kind, 0) if isinstance(kind, str) else int(kind), int(capacity)))

    def profile_read(self):
        n = C.c_longlong(0); ms = C.c_double(0)
        self._chk(self.L.cipc_gpu_profile_read(self.h, C.byref(n), C.byref(ms)))
        return n.value, ms.value

    def get(self, name):
        o = np.zeros((self.nv, 3))
        self._chk(self.L.cipc_gpu_get_state(self.h, self.STATE[name], _d(o)))
        return o

    def set(self, name, arr):
        a = np.ascontiguousarray(arr, np.float64).reshape(self.nv, 3)
        self._chk(self.L.cipc_gpu_set_state(self.h, self.STATE[name], _d(a)))

    def scalars(self):
        o = np.zeros(14)
        self._chk(self.L.cipc_gpu_get_scalars(self.h, _d(o)))
        keys = ["kappa", "Hhat", "Fhat", "dTol", "bboxDiag2", "meanMass", "avgEdge", "lengthRate", "volumeRate",
                "stretchS", "shearS", "plateRigidity", "dt", "newtonThr"]
        return dict(zip(keys, o.tolist()))

    def set_kappa(self, k):
        self._chk(self.L.cipc_gpu_set_kappa(self.h, float(k)))

    def set_online_training(self, iterations, probes=4, lr=1e-3, seed=0):
        """Adam iterations of the network on every Newton system as it is
        assembled (0 turns it off)."""
        self._chk(self.L.cipc_gpu_set_online_training(self.h, int(iterations), int(probes), float(lr), int(seed)))

    def set_system_dump(self, directory):
        """Write every Newton system to `directory` (None turns it off)."""
        self._chk(self.L.cipc_gpu_set_system_dump(self.h, None if directory is None else str(directory).encode()))

    def host_syncs(self):
        """Host waits on the context's stream since creation."""
        n = C.c_longlong(0)
        self._chk(self.L.cipc_gpu_host_syncs(self.h, C.byref(n)))
        return n.value

    def hook_systems(self):
        n = C.c_longlong(0)
        self._chk(self.L.cipc_gpu_hook_systems(self.h, C.byref(n)))
        return n.value

    def set_broad_phase(self, backend):
        """'lbvh' (default) or 'spatial-hash'."""
        self._chk(self.L.cipc_gpu_set_broad_phase(self.h, {"lbvh": 0, "spatial-hash": 1}[backend]))

    def set_intersection_rule(self, rule):
        """'tolerant' (default) or 'reference' (the reference's exact
        segment-triangle coplanarity rule)."""
        self._chk(self.L.cipc_gpu_set_intersection_rule(self.h, {"tolerant": 0, "reference": 1}[rule]))

    def surface(self):
        f = np.zeros((self.nsf, 3), np.int32); v = np.zeros(self.nsv, np.int32); e = np.zeros((self.nse, 2), np.int32)
        self._chk(self.L.cipc_gpu_get_surface(self.h, _i(f), _i(v), _i(e)))
        return f, v, e

    def collision_sets(self):
        c = (C.c_longlong * 4)()
        self._chk(self.L.cipc_gpu_build_collision_sets(self.h, c))
        ns, nm, nc, ng = [int(v) for v in c]
        sa = np.zeros((ns, 4), np.int32); see = np.zeros((nm, 4), np.int32); eeie = np.zeros((nm, 2), np.int32)
        ccd = np.zeros((nc, 2), np.int32); gr = np.zeros(ng, np.int32)
        self._chk(self.L.cipc_gpu_get_active_sets(self.h, _i(sa), _i(see), _i(eeie), _i(ccd), _i(gr)))
        return dict(self_active=sa, self_ee=see, ee_ie=eeie, ccd=ccd, ground=gr)

    def friction_init(self):
        self._chk(self.L.cipc_gpu_friction_init(self.h))

    def assemble(self):
        g = np.zeros((self.nv, 3))
        coll = C.c_int(0)
        self._chk(self.L.cipc_gpu_assemble(self.h, _d(g), C.byref(coll)))
        return g, coll.value

    def export_matrix(self):
        """Full symmetric scalar COO (rows, cols, vals) of the last assembled system."""
        n = C.c_longlong(0)
        self._chk(self.L.cipc_gpu_export_matrix(self.h, C.byref(n), None, None, None))
        r = np.zeros(n.value, np.int32); c = np.zeros(n.value, np.int32); v = np.zeros(n.value)
        self._chk(self.L.cipc_gpu_export_matrix(self.h, C.byref(n), _i(r), _i(c), _d(v)))
        k = n.value
        return r[:k], c[:k], v[:k]

    def solve(self):
        d = np.zeros((self.nv, 3))
        it = C.c_int(0); rr = C.c_double(0)
        self._chk(self.L.cipc_gpu_solve(self.h, _d(d), C.byref(it), C.byref(rr)))
        return d, it.value, rr.value

    def energy(self, kappa):
        e = C.c_double(0)
        self._chk(self.L.cipc_gpu_energy(self.h, float(kappa), C.byref(e)))
        return e.value

    def step_bounds(self, direction, alpha_in=1.0):
        dd = np.ascontiguousarray(direction, np.float64).reshape(-1)
        o = np.zeros(4)
        self._chk(self.L.cipc_gpu_step_bounds(self.h, _d(dd), float(alpha_in), _d(o)))
        return dict(ground=o[0], partial=o[1], cfl=o[2], full=o[3])

    def intersected(self):
        r = C.c_int(0)
        self._chk(self.L.cipc_gpu_intersected(self.h, C.byref(r)))
        return bool(r.value)

    # ---- system dump and learned preconditioner ----
    def export_bsr(self):
        """The last assembled Newton matrix in the device block layout (a dict)."""
        sz = np.zeros(2, np.int32)
        self._chk(self.L.cipc_gpu_export_bsr(self.h, _i(sz), None, None, None, None, None, None, None, None))
        nnzb, ndyn = int(sz[0]), int(sz[1])
        nv = self.nv
        rp = np.zeros(nv + 1, np.int32); col = np.zeros(max(nnzb, 1), np.int32); val = np.zeros((max(nnzb, 1), 9))
        drs = np.zeros(nv, np.int32); dre = np.zeros(nv, np.int32)
        dcol = np.zeros(max(ndyn, 1), np.int32); dval = np.zeros((max(ndyn, 1), 9)); dx = np.zeros((nv, 9))
        self._chk(self.L.cipc_gpu_export_bsr(self.h, _i(sz), _i(rp), _i(col), _d(val), _i(drs), _i(dre), _i(dcol), _d(dval), _d(dx)))
        return dict(nv=nv, rowPtr=rp, col=col[:nnzb], val=val[:nnzb], dRowS=drs, dRowE=dre, dCol=dcol[:ndyn], dVal=dval[:ndyn],
                    diagExtra=dx)

    def precond_weights(self):
        n = self.L.cipc_gpu_precond_num_params()
        w = np.zeros(n, np.float32)
        self._chk(self.L.cipc_gpu_precond_get_weights(self.h, _f(w), n))
        return w

    def set_precond_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        self._chk(self.L.cipc_gpu_precond_set_weights(self.h, _f(w), len(w)))

    def precond_loss(self, probes=None, nprobes=4, seed=0, grad=False):
        """(loss, gradient or None) on the last assembled system."""
        pv = None
        if probes is not None:
            pv = np.ascontiguousarray(probes, np.float32).reshape(-1)
            nprobes = len(pv) // (3 * self.nv)
        loss = C.c_double(0)
        g = np.zeros(self.L.cipc_gpu_precond_num_params(), np.float32) if grad else None
        self._chk(self.L.cipc_gpu_precond_loss(self.h, nprobes, _f(pv) if pv is not None else None, seed, C.byref(loss),
                                               _f(g) if grad else None))
        return loss.value, g

    def precond_train(self, iterations, probes=4, lr=1e-3, seed=0):
        a = C.c_double(0); b = C.c_double(0)
        self._chk(self.L.cipc_gpu_precond_train(self.h, iterations, probes, lr, seed, C.byref(a), C.byref(b)))
        return a.value, b.value

    def precond_factor(self, which="fsai"):
        """The factor G on the last assembled system, slot-aligned with export_bsr:
        (static blocks (nnzb, 9), contact blocks (ndyn, 9))."""
        sz = np.zeros(2, np.int32)
        self._chk(self.L.cipc_gpu_export_bsr(self.h, _i(sz), None, None, None, None, None, None, None, None))
        gs = np.zeros((max(int(sz[0]), 1), 9), np.float32)
        gd = np.zeros((max(int(sz[1]), 1), 9), np.float32)
        self._chk(self.L.cipc_gpu_precond_factor(self.h, PRECOND[which], _f(gs), _f(gd)))
        return gs[:int(sz[0])], gd[:int(sz[1])]

    def precond_stats(self):
        o = (C.c_longlong * 3)()
        self._chk(self.L.cipc_gpu_precond_stats(self.h, o))
        return dict(fallbacks=o[0], adam_steps=o[1], last_launch_iterations=o[2])


def pcg_bsr(row_ptr, col_idx, vals, rhs, precision="fp64", tol=1e-6, max_iter=10000):
    """Stand-alone GPU PCG on a full symmetric 3x3-block CSR matrix."""
    L = lib()
    nv = len(row_ptr) - 1
    rp = np.ascontiguousarray(row_ptr, np.int32); ci = np.ascontiguousarray(col_idx, np.int32)
    va = np.ascontiguousarray(vals, np.float64).reshape(-1); b = np.ascontiguousarray(rhs, np.float64).reshape(-1)
    sol = np.zeros(3 * nv)
    it = C.c_int(0); rr = C.c_double(0)
    err = C.create_string_buffer(512)
    opts = linear_options(precision, "jacobi", tol, max_iter)
    rc = L.cipc_gpu_pcg_bsr(nv, _i(rp), _i(ci), _d(va), _d(b), _d(sol), C.byref(opts), C.byref(it), C.byref(rr), err, 512)
    if rc != CIPC_OK:
        raise CipcError(rc, err.value.decode())
    return sol, it.value, rr.value


def read_system(path):
    """A Newton system written by Simulator.set_system_dump (file layout in
    include/cipc_gpu.h, cipc_gpu_set_system_dump)."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] != b"CIPCSYS1":
        raise ValueError(f"{path} is not a dumped Newton system")
    nv, nnzb, ndyn, vb, frame, newton = np.frombuffer(buf, np.int32, 6, 8)
    off = 32
    def take(dtype, n):
        nonlocal off
        a = np.frombuffer(buf, dtype, n, off)
        off += a.nbytes
        return a
    vt = np.float32 if vb == 4 else np.float64
    out = dict(frame=int(frame), newton=int(newton))
    out["row_ptr"] = take(np.int32, nv + 1)
    out["col"] = take(np.int32, nnzb)
    out["val"] = take(vt, 9 * nnzb).reshape(nnzb, 3, 3)
    out["dyn_row_start"] = take(np.int32, nv)
    out["dyn_row_end"] = take(np.int32, nv)
    out["dyn_col"] = take(np.int32, ndyn) if ndyn else np.zeros(0, np.int32)
    out["dyn_val"] = take(vt, 9 * ndyn).reshape(ndyn, 3, 3) if ndyn else np.zeros((0, 3, 3), vt)
    out["diag_extra"] = take(np.float64, 9 * nv).reshape(nv, 3, 3)
    out["rhs"] = take(np.float64, 3 * nv).reshape(nv, 3)
    out["x"] = take(np.float64, 3 * nv).reshape(nv, 3)
    out["btype"] = take(np.int32, nv)
    if off != len(buf):
        raise ValueError(f"{path}: {len(buf) - off} trailing bytes")
    return out


def accd(kind, positions, displacements, eta=0.2):
    """Conservative time of impact of independent candidate pairs on the GPU
    (kind 0 point-triangle, 1 edge-edge; positions and displacements n x 4 x 3)."""
    L = lib()
    k = np.ascontiguousarray(kind, np.int32).reshape(-1)
    p = np.ascontiguousarray(positions, np.float64).reshape(-1)
    d = np.ascontiguousarray(displacements, np.float64).reshape(-1)
    n = len(k)
    if p.size != 12 * n or d.size != 12 * n:
        raise ValueError("positions and displacements need 12 values per pair")
    out = np.zeros(n)
    err = C.create_string_buffer(512)
    rc = L.cipc_gpu_accd(n, _i(k), _d(p), _d(d), float(eta), _d(out), err, 512)
    if rc != CIPC_OK:
        raise CipcError(rc, err.value.decode())
    return out


# ---------------------------------------------------------------------------
# Synthetic scenes (structured Kuhn 6-tet cubes, triangle-grid cloth)
# ---------------------------------------------------------------------------
def cube_mesh(n, size=1.0, center=(0.0, 0.0, 0.0)):
    """Regular n x n x n cell cube, each cell split into 6 tets sharing the main diagonal."""
    g = np.linspace(-0.5 * size, 0.5 * size, n + 1)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    x = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1) + np.asarray(center)
    idx = np.arange((n + 1) ** 3).reshape(n + 1, n + 1, n + 1)
    c = np.array([[i, j, k] for i in range(n) for j in range(n) for k in range(n)])
    v = lambda di, dj, dk: idx[c[:, 0] + di, c[:, 1] + dj, c[:, 2] + dk]
    v0, v1, v2, v3 = v(0, 0, 0), v(1, 0, 0), v(0, 1, 0), v(1, 1, 0)
    v4, v5, v6, v7 = v(0, 0, 1), v(1, 0, 1), v(0, 1, 1), v(1, 1, 1)
    # six tets around the diagonal v0-v7 (positively oriented)
    tl = [(v0, v1, v3, v7), (v0, v1, v7, v5), (v0, v2, v7, v3), (v0, v2, v6, v7), (v0, v4, v5, v7), (v0, v4, v7, v6)]
    tets = np.concatenate([np.stack(t, 1) for t in tl]).astype(np.int32)
    # orient every tet positively
    a = x[tets[:, 1]] - x[tets[:, 0]]; b = x[tets[:, 2]] - x[tets[:, 0]]; cc = x[tets[:, 3]] - x[tets[:, 0]]
    neg = np.einsum("ij,ij->i", np.cross(a, b), cc) < 0
    tets[neg, 2], tets[neg, 3] = tets[neg, 3].copy(), tets[neg, 2].copy()
    return x, tets


def grid_cloth(n, size=1.0, y=0.0):
    """n x n vertex square triangle grid in the xz-plane at height y."""
    g = np.linspace(-0.5 * size, 0.5 * size, n)
    X, Z = np.meshgrid(g, g, indexing="ij")
    x = np.stack([X.ravel(), np.full(X.size, y), Z.ravel()], 1)
    idx = np.arange(n * n).reshape(n, n)
    a, b, c, d = idx[:-1, :-1].ravel(), idx[1:, :-1].ravel(), idx[:-1, 1:].ravel(), idx[1:, 1:].ravel()
    # winding with +y normals: the rest-shape map rotates each normal onto +y,
    # which is singular for a normal of exactly -y
    tris = np.concatenate([np.stack([a, d, b], 1), np.stack([a, c, d], 1)]).astype(np.int32)
    return x, tris


def base_params(**kw):
    p = dict(density=1000.0, cloth_density=200.0, thickness=1e-3, E=1e5, nu=0.4, clothE=1e4, shearE=10.0,
             bendE=1e4, strainRate=100.0, friction=0.2, dt=0.01, drag=0.0, newtonThr=1e-2, relDhat=1e-3,
             use_barrier=1, apply_gravity=1, quasi_static=0, quad_bending=1)
    p.update(kw)
    return p


def _bbox(x):
    return x.min(0).tolist(), x.max(0).tolist()


def scene_two_cubes(cells=8, gap=0.05, newton_thr=1e-6):
    """Two unit cubes (cells^3 cells, 6 tets/cell) stacked with a gap, lowest one `gap` above the ground y=-1."""
    xa, ta = cube_mesh(cells, 1.0, (0.0, -1.0 + gap + 0.5, 0.0))
    xb, tb = cube_mesh(cells, 1.0, (0.0, -1.0 + gap + 1.0 + gap + 0.5, 0.0))
    x = np.concatenate([xa, xb]); tets = np.concatenate([ta, tb + len(xa)])
    lo, hi = _bbox(x)
    return dict(x=x, tets=tets, tris=np.zeros((0, 3), np.int32), btype=np.zeros(len(x), np.int32),
                params=base_params(E=1e5, nu=0.4, density=1000.0, friction=0.2, dt=0.01, newtonThr=newton_thr, relDhat=1e-3),
                bbox_min=lo, bbox_max=hi, name=f"two_cubes_{cells}")


def scene_cloth_drape(n=128, cube_cells=10, newton_thr=1e-2):
    """n x n vertex 1 m cloth 0.1 m above a fixed 0.5 m tet cube (external collider)."""
    xc, tc = cube_mesh(cube_cells, 0.5, (0.0, 0.0, 0.0))
    xs, ts = grid_cloth(n, 1.0, 0.25 + 0.1)
    x = np.concatenate([xs, xc]); tets = tc + len(xs)
    bt = np.zeros(len(x), np.int32); bt[len(xs):] = 2
    # plate rigidity k_b = 1e-3 with t = 1e-3, nu = 0.3
    nu = 0.3
    bendE = 1e-3 * 12 * (1 - nu * nu) / (1e-3) ** 3
    lo, hi = _bbox(x)
    return dict(x=x, tets=tets, tris=ts, btype=bt,
                params=base_params(E=1e5, nu=nu, clothE=1e4, shearE=10.0, bendE=bendE, thickness=1e-3, cloth_density=200.0,
                                   friction=0.3, dt=0.005, newtonThr=newton_thr, relDhat=1e-3),
                bbox_min=lo, bbox_max=hi, name=f"cloth_drape_{n}")


def _rand_rot(rng):
    u1, u2, u3 = rng.random(3)
    q = np.array([math.sqrt(1 - u1) * math.sin(2 * math.pi * u2), math.sqrt(1 - u1) * math.cos(2 * math.pi * u2),
                  math.sqrt(u1) * math.sin(2 * math.pi * u3), math.sqrt(u1) * math.cos(2 * math.pi * u3)])
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def scene_pile(n_cubes=64, cells=12, seed=0, box=1.5, newton_thr=1e-2):
    """Cubes of 0.2 m at seeded random rotations, dropped into a static open
    box (5 quads).  Positions are seeded uniform jitters of the points of a
    k x k x k lattice that fills the box (k = ceil(n_cubes^(1/3)); n_cubes of
    its cells, chosen at random): every cube's bounding sphere stays inside
    its own cell, so no two cubes touch whatever their rotations.  (Rejection
    sampling of free positions cannot place 64 such spheres in a 1.5 m box:
    that packing is past the random-sequential-addition limit.)"""
    rng = np.random.default_rng(seed)
    r = 0.1 * math.sqrt(3) + 1e-3
    k = 1
    while k ** 3 < n_cubes:
        k += 1
    cell = box / k
    slack = 0.5 * cell - r
    if slack < 0:
        raise ValueError(f"{n_cubes} cubes of 0.2 m do not fit a {box} m box")
    base = np.array([-0.5 * box, -1.0 + 0.05, -0.5 * box])
    slots = rng.permutation(k ** 3)[:n_cubes]
    centers = []
    for sl in slots:
        ijk = np.array([sl % k, (sl // k) % k, sl // (k * k)], float)
        centers.append(base + (ijk + 0.5) * cell + rng.uniform(-slack, slack, 3))
    xs, ts, te = [], [], []
    off = 0
    Es = rng.uniform(5e4, 5e5, n_cubes)
    for k, c in enumerate(centers):
        x, t = cube_mesh(cells, 0.2)
        x = x @ _rand_rot(rng).T + c
        xs.append(x); ts.append(t + off); te.append(np.full(len(t), Es[k])); off += len(x)
    x = np.concatenate(xs); tets = np.concatenate(ts)
    # open box: floor + 4 walls as triangle pairs (external collider, cloth-type triangles)
    h = 0.5 * box + 0.05
    y0, y1 = -1.0 + 0.02, -1.0 + 0.05 + box
    q = [
        [(-h, y0, -h), (-h, y0, h), (h, y0, h), (h, y0, -h)],  # +y normal (see grid_cloth)
        [(-h, y0, -h), (-h, y1, -h), (h, y1, -h), (h, y0, -h)],
        [(-h, y0, h), (h, y0, h), (h, y1, h), (-h, y1, h)],
        [(-h, y0, -h), (-h, y0, h), (-h, y1, h), (-h, y1, -h)],
        [(h, y0, -h), (h, y1, -h), (h, y1, h), (h, y0, h)],
    ]
    bx = np.array([p for quad in q for p in quad], float)
    btris = []
    for i in range(5):
        b = len(x) + 4 * i
        btris += [[b, b + 1, b + 2], [b, b + 2, b + 3]]
    x = np.concatenate([x, bx])
    bt = np.zeros(len(x), np.int32); bt[-len(bx):] = 2
    lo, hi = _bbox(x)
    return dict(x=x, tets=tets, tris=np.array(btris, np.int32), btype=bt, tetE=np.concatenate(te),
                params=base_params(E=float(np.mean(Es)), nu=0.4, friction=0.2, dt=0.01, newtonThr=newton_thr, relDhat=1e-3),
                bbox_min=lo, bbox_max=hi, name=f"pile_{n_cubes}x{cells}")


def scene_twist(radial=8, angular=16, axial=32, radius=0.1, length=1.0, rate=2 * math.pi, newton_thr=1e-2):
    """Structured cylindrical tet mesh (wedge prisms split into 3 tets) with both end caps Dirichlet-twisted."""
    pts = [(0.0, 0.0)]
    for ir in range(1, radial + 1):
        for ia in range(angular):
            a = 2 * math.pi * ia / angular
            pts.append((radius * ir / radial * math.cos(a), radius * ir / radial * math.sin(a)))
    pts = np.array(pts)
    ring = lambda ir, ia: 0 if ir == 0 else 1 + (ir - 1) * angular + (ia % angular)
    tri2 = []
    for ir in range(radial):
        for ia in range(angular):
            if ir == 0:
                tri2.append((ring(0, 0), ring(1, ia), ring(1, ia + 1)))
            else:
                a, b, c, d = ring(ir, ia), ring(ir, ia + 1), ring(ir + 1, ia), ring(ir + 1, ia + 1)
                tri2 += [(a, c, d), (a, d, b)]
    npl = len(pts)
    xs = np.linspace(-0.5 * length, 0.5 * length, axial + 1)
    x = np.array([[xx, p[0], p[1]] for xx in xs for p in pts])
    tets = []
    for k in range(axial):
        for (a, b, c) in tri2:
            A, B, Cc = a + k * npl, b + k * npl, c + k * npl
            D, E, F = A + npl, B + npl, Cc + npl
            # prism split with global vertex-order rule to keep faces conforming
            v = sorted([(A, D), (B, E), (Cc, F)], key=lambda e: e[0])
            (a0, a1), (b0, b1), (c0, c1) = v
            tets += [(a0, b0, c0, a1), (b0, c0, a1, b1), (c0, a1, b1, c1)]
    tets = np.array(tets, np.int32)
    p0 = x[tets[:, 0]]
    neg = np.einsum("ij,ij->i", np.cross(x[tets[:, 1]] - p0, x[tets[:, 2]] - p0), x[tets[:, 3]] - p0) < 0
    tets[neg, 2], tets[neg, 3] = tets[neg, 3].copy(), tets[neg, 2].copy()
    bt = np.zeros(len(x), np.int32)
    caps = np.nonzero((np.abs(x[:, 0]) > 0.5 * length - 1e-9))[0].astype(np.int32)
    bt[caps] = 1
    lo, hi = _bbox(x)
    return dict(x=x, tets=tets, tris=np.zeros((0, 3), np.int32), btype=bt,
                params=base_params(E=1e5, nu=0.45, friction=0.1, dt=0.01, newtonThr=newton_thr, relDhat=1e-3, apply_gravity=0),
                dirichlet=dict(idx=caps, motion=MOTION_TWIST_X, rate=rate),
                bbox_min=lo, bbox_max=hi, name=f"twist_{radial}x{angular}x{axial}")


SCENES = {"two_cubes": scene_two_cubes, "cloth_drape": scene_cloth_drape, "pile": scene_pile, "twist": scene_twist}
