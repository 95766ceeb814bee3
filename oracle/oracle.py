"""Test infrastructure only: ctypes front-end of the FP64 CPU oracle.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs (cpu_baseline
and --impl reference) import this module; the shipped library never uses
it.  It loads ``liboracle.so`` (built from the sources beside it by
``make``) and exposes the oracle's scene set-up, time step and per-stage
evaluations.
"""
import ctypes as C
import hashlib
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

MOTION_NONE = 0
MOTION_TWIST_X = 1


def build():
    """Compile liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class Scene(C.Structure):
    _fields_ = [
        ("nv", C.c_int), ("nt", C.c_int), ("nf", C.c_int),
        ("x", C.POINTER(C.c_double)), ("vel", C.POINTER(C.c_double)),
        ("tets", C.POINTER(C.c_int)), ("tris", C.POINTER(C.c_int)), ("btype", C.POINTER(C.c_int)),
        ("tetE", C.POINTER(C.c_double)),
        ("density", C.c_double), ("cloth_density", C.c_double), ("thickness", C.c_double),
        ("E", C.c_double), ("nu", C.c_double), ("clothE", C.c_double), ("shearE", C.c_double),
        ("bendE", C.c_double), ("strainRate", C.c_double), ("friction", C.c_double),
        ("dt", C.c_double), ("drag", C.c_double), ("newtonThr", C.c_double), ("relDhat", C.c_double),
        ("use_barrier", C.c_int), ("apply_gravity", C.c_int), ("quasi_static", C.c_int), ("quad_bending", C.c_int),
        ("bboxMin", C.c_double * 3), ("bboxMax", C.c_double * 3),
        ("nsoft", C.c_int), ("softIdx", C.POINTER(C.c_int)), ("softW", C.c_double),
        ("softMotion", C.c_int), ("softRate", C.c_double),
        ("ndir", C.c_int), ("dirIdx", C.POINTER(C.c_int)), ("dirMotion", C.c_int), ("dirRate", C.c_double),
        ("linear", C.c_int), ("pcgRelTol", C.c_double), ("threads", C.c_int),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("frame", C.c_int), ("newton", C.c_int), ("kappaIters", C.c_int), ("backtracks", C.c_int),
        ("energyBacktracks", C.c_int), ("intersectionBacktracks", C.c_int),
        ("maxEnergyBacktracksPerNewton", C.c_int), ("newtonOverTwo", C.c_int),
        ("collisions", C.c_double), ("kappa", C.c_double), ("minDist2", C.c_double),
        ("acceptedStepSum", C.c_double), ("minStep", C.c_double), ("maxStep", C.c_double),
        ("groundContacts", C.c_longlong), ("selfContacts", C.c_longlong),
        ("mollifiedContacts", C.c_longlong), ("matrixNnz", C.c_longlong), ("pcgIterations", C.c_longlong),
        ("linearSolves", C.c_longlong),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        dp, ip, vp = C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_void_p
        L.cipc_oracle_create.restype = vp
        L.cipc_oracle_create.argtypes = [C.POINTER(Scene), C.c_char_p, C.c_int]
        L.cipc_oracle_destroy.argtypes = [vp]
        L.cipc_oracle_step.argtypes = [vp, C.POINTER(Stats), C.c_char_p, C.c_int]
        L.cipc_oracle_info.argtypes = [vp, C.POINTER(C.c_longlong)]
        L.cipc_oracle_scalars.argtypes = [vp, dp]
        L.cipc_oracle_set_kappa.argtypes = [vp, C.c_double]
        L.cipc_oracle_set_intersection_rule.argtypes = [vp, C.c_int]
        L.cipc_oracle_get.argtypes = [vp, C.c_int, dp]
        L.cipc_oracle_set.argtypes = [vp, C.c_int, dp]
        L.cipc_oracle_surface.argtypes = [vp, ip, ip, ip]
        L.cipc_oracle_rest.argtypes = [vp, dp, dp, dp, dp, ip, dp]
        L.cipc_oracle_collision_sets.argtypes = [vp, C.POINTER(C.c_longlong)]
        L.cipc_oracle_get_sets.argtypes = [vp, ip, ip, ip, ip, ip]
        L.cipc_oracle_friction_init.argtypes = [vp]
        L.cipc_oracle_system.restype = C.c_longlong
        L.cipc_oracle_system.argtypes = [vp, dp, ip, ip, dp, dp]
        L.cipc_oracle_energy.restype = C.c_double
        L.cipc_oracle_energy.argtypes = [vp, C.c_double]
        L.cipc_oracle_total_energy.restype = C.c_double
        L.cipc_oracle_total_energy.argtypes = [vp]
        L.cipc_oracle_step_bounds.argtypes = [vp, dp, C.c_double, dp]
        L.cipc_oracle_intersected.restype = C.c_int
        L.cipc_oracle_intersected.argtypes = [vp]
        L.cipc_oracle_pt_ccd.restype = C.c_double
        L.cipc_oracle_pt_ccd.argtypes = [dp, dp, C.c_double]
        L.cipc_oracle_ee_ccd.restype = C.c_double
        L.cipc_oracle_ee_ccd.argtypes = [dp, dp, C.c_double]
        L.cipc_oracle_snh.argtypes = [dp, C.c_double, C.c_double, dp, dp, dp]
        L.cipc_oracle_distance.restype = C.c_double
        L.cipc_oracle_distance.argtypes = [C.c_int, dp, dp, dp]
        L.cipc_oracle_hinge.restype = C.c_double
        L.cipc_oracle_hinge.argtypes = [dp, dp, C.c_double, dp, dp]
        L.cipc_oracle_linear_solve.restype = C.c_int
        L.cipc_oracle_linear_solve.argtypes = [C.c_int, ip, ip, dp, dp, dp, C.c_int, C.c_double, C.c_int, ip, dp, C.c_int, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class Oracle:
    """One oracle simulation context built from a scene dictionary.

    The dictionary is the raw scene format shared with the CUDA path (see
    ``cpu-ipc_b200/cipc.py``): positions, tets, cloth triangles, boundary
    codes, material and solver parameters and the bounding box.
    """

    def __init__(self, scene, linear="direct", pcg_tol=1e-6, threads=1):
        self._keep = []
        L = lib()
        s = Scene()
        x = np.ascontiguousarray(scene["x"], dtype=np.float64).reshape(-1)
        tets = np.ascontiguousarray(scene.get("tets", np.zeros((0, 4))), dtype=np.int32).reshape(-1)
        tris = np.ascontiguousarray(scene.get("tris", np.zeros((0, 3))), dtype=np.int32).reshape(-1)
        btype = np.ascontiguousarray(scene["btype"], dtype=np.int32)
        self._keep += [x, tets, tris, btype]
        s.nv, s.nt, s.nf = len(x) // 3, len(tets) // 4, len(tris) // 3
        s.x, s.tets, s.tris, s.btype = _dp(x), _ip(tets), _ip(tris), _ip(btype)
        if scene.get("vel") is not None:
            vel = np.ascontiguousarray(scene["vel"], dtype=np.float64).reshape(-1)
            self._keep.append(vel)
            s.vel = _dp(vel)
        if scene.get("tetE") is not None:
            te = np.ascontiguousarray(scene["tetE"], dtype=np.float64)
            self._keep.append(te)
            s.tetE = _dp(te)
        p = scene["params"]
        for k in ("density", "cloth_density", "thickness", "E", "nu", "clothE", "shearE", "bendE",
                  "strainRate", "friction", "dt", "drag", "newtonThr", "relDhat"):
            setattr(s, k, float(p[k]))
        s.use_barrier = int(p.get("use_barrier", 1))
        s.apply_gravity = int(p.get("apply_gravity", 1))
        s.quasi_static = int(p.get("quasi_static", 0))
        s.quad_bending = int(p.get("quad_bending", 1))
        for i in range(3):
            s.bboxMin[i] = scene["bbox_min"][i]
            s.bboxMax[i] = scene["bbox_max"][i]
        soft = scene.get("soft")
        if soft:
            si = np.ascontiguousarray(soft["idx"], dtype=np.int32)
            self._keep.append(si)
            s.nsoft, s.softIdx, s.softW = len(si), _ip(si), float(soft["weight"])
            s.softMotion, s.softRate = int(soft.get("motion", 0)), float(soft.get("rate", 0.0))
        dirc = scene.get("dirichlet")
        if dirc:
            di = np.ascontiguousarray(dirc["idx"], dtype=np.int32)
            self._keep.append(di)
            s.ndir, s.dirIdx = len(di), _ip(di)
            s.dirMotion, s.dirRate = int(dirc.get("motion", 0)), float(dirc.get("rate", 0.0))
        s.linear = {"direct": 0, "pcg": 1, "multifrontal": 2}[linear]
        s.pcgRelTol = pcg_tol
        s.threads = threads
        err = C.create_string_buffer(512)
        h = L.cipc_oracle_create(C.byref(s), err, 512)
        if not h:
            raise RuntimeError("oracle scene set-up failed: " + err.value.decode())
        self.h = C.c_void_p(h)
        self.L = L
        c = (C.c_longlong * 7)()
        L.cipc_oracle_info(self.h, c)
        self.nv, self.nsf, self.nsv, self.nse, self.nbend, self.nt, self.nf = [int(v) for v in c]

    def __del__(self):
        if getattr(self, "h", None):
            self.L.cipc_oracle_destroy(self.h)
            self.h = None

    def step(self):
        st = Stats()
        err = C.create_string_buffer(512)
        if self.L.cipc_oracle_step(self.h, C.byref(st), err, 512) != 0:
            raise RuntimeError(err.value.decode())
        return st.as_dict()

    def scalars(self):
        o = np.zeros(14)
        self.L.cipc_oracle_scalars(self.h, _dp(o))
        keys = ["kappa", "Hhat", "Fhat", "dTol", "bboxDiag2", "meanMass", "avgEdge", "lengthRate", "volumeRate",
                "stretchS", "shearS", "plateRigidity", "dt", "newtonThr"]
        return dict(zip(keys, o.tolist()))

    def set_kappa(self, k):
        self.L.cipc_oracle_set_kappa(self.h, float(k))

    def set_intersection_rule(self, rule):
        """'tolerant' (default): near-coplanar segments within a 1e-12
        relative tolerance count as coplanar; 'reference': the reference's
        exact rule (ContactMechanics.h:47-71)."""
        self.L.cipc_oracle_set_intersection_rule(self.h, {"tolerant": 0, "reference": 1}[rule])

    _FIELDS = {"x": 0, "vel": 1, "vprev": 2, "xtilde": 3, "rest": 4}

    def get(self, name):
        if name == "mass":
            o = np.zeros(self.nv)
            self.L.cipc_oracle_get(self.h, 5, _dp(o))
            return o
        o = np.zeros((self.nv, 3))
        self.L.cipc_oracle_get(self.h, self._FIELDS[name], _dp(o))
        return o

    def set(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(self.nv, 3)
        self.L.cipc_oracle_set(self.h, self._FIELDS[name], _dp(a))

    def rest_digest(self):
        """SHA-256 of the rest positions: names the scene a saved state belongs to."""
        return hashlib.sha256(self.get("rest").tobytes()).hexdigest()

    def save_state(self, path, frame):
        """Write what the next step starts from: positions, velocities, kappa.

        After every step V_prev equals x and x_tilde = V_prev + dt v + dt^2 g
        (updateInertialTarget, IPCSolver.cpp:55-70), so restore_state rebuilds
        those two; this checks the rebuild against the oracle's own x_tilde.
        """
        x, vel = self.get("x"), self.get("vel")
        if not np.array_equal(self.get("vprev"), x):
            raise RuntimeError("save_state must follow a completed step (V_prev != x)")
        xt = self.get("xtilde")
        g = next((g for g in (-9.8, 0.0) if np.array_equal(xt, self._xtilde(x, vel, g))), None)
        if g is None:
            raise RuntimeError("x_tilde does not follow V_prev + dt v + dt^2 g")
        np.savez_compressed(path, x=x, vel=vel, kappa=self.scalars()["kappa"], gravity=g, frame=frame,
                            rest_sha256=self.rest_digest())

    def restore_state(self, path):
        """Load a state written by save_state; returns its frame number.

        The collision sets are rebuilt at the restored positions: a step
        leaves them built at its final positions, and the next step's lagged
        friction starts from them (frictionInitialize, Friction.cpp:81-156).
        Raises ValueError when the state belongs to another scene."""
        s = np.load(path)
        if str(s["rest_sha256"]) != self.rest_digest():
            raise ValueError(f"{path} was saved from another scene")
        x, vel = s["x"], s["vel"]
        self.set("x", x)
        self.set("vprev", x)
        self.set("vel", vel)
        self.set("xtilde", self._xtilde(x, vel, float(s["gravity"])))
        self.set_kappa(float(s["kappa"]))
        self.collision_sets()
        return int(s["frame"])

    def _xtilde(self, vprev, vel, g):
        # componentwise as the oracle: (V_prev + v dt) + (0, g dt dt, 0)
        dt = self.scalars()["dt"]
        return vprev + vel * dt + np.array([0.0, g * dt * dt, 0.0])

    def surface(self):
        f = np.zeros((self.nsf, 3), np.int32)
        v = np.zeros(self.nsv, np.int32)
        e = np.zeros((self.nse, 2), np.int32)
        self.L.cipc_oracle_surface(self.h, _ip(f), _ip(v), _ip(e))
        return f, v, e

    def rest(self):
        dm = np.zeros((self.nt, 3, 3)); vol = np.zeros(self.nt)
        dm2 = np.zeros((self.nf, 2, 2)); area = np.zeros(self.nf)
        bv = np.zeros((self.nbend, 4), np.int32); bq = np.zeros((self.nbend, 4, 4))
        self.L.cipc_oracle_rest(self.h, _dp(dm), _dp(vol), _dp(dm2), _dp(area), _ip(bv), _dp(bq))
        return dict(DmInv=dm, vol=vol, DmInv2=dm2, area=area, bend_v=bv, bend_Q=bq)

    def collision_sets(self):
        c = (C.c_longlong * 4)()
        self.L.cipc_oracle_collision_sets(self.h, c)
        na, nee, nccd, ng = [int(v) for v in c]
        sa = np.zeros((na, 4), np.int32); see = np.zeros((nee, 4), np.int32)
        eeie = np.zeros((nee, 2), np.int32); ccd = np.zeros((nccd, 2), np.int32); gr = np.zeros(ng, np.int32)
        self.L.cipc_oracle_get_sets(self.h, _ip(sa), _ip(see), _ip(eeie), _ip(ccd), _ip(gr))
        return dict(self_active=sa, self_ee=see, ee_ie=eeie, ccd=ccd, ground=gr)

    def friction_init(self):
        self.L.cipc_oracle_friction_init(self.h)

    def system(self):
        """Gradient and the lower-triangular free-vertex scalar CSR of the Newton matrix."""
        nnz = self.L.cipc_oracle_system(self.h, None, None, None, None, None)
        g = np.zeros((self.nv, 3))
        rp = np.zeros(3 * self.nv + 1, np.int32)
        col = np.zeros(nnz, np.int32)
        val = np.zeros(nnz)
        rhs = np.zeros(3 * self.nv)
        self.L.cipc_oracle_system(self.h, _dp(g), _ip(rp), _ip(col), _dp(val), _dp(rhs))
        return g, rp, col, val, rhs

    def energy(self, kappa=None):
        if kappa is None:
            return self.L.cipc_oracle_total_energy(self.h)
        return self.L.cipc_oracle_energy(self.h, float(kappa))

    def step_bounds(self, direction, alpha_in=1.0):
        d = np.ascontiguousarray(direction, dtype=np.float64).reshape(-1)
        o = np.zeros(4)
        self.L.cipc_oracle_step_bounds(self.h, _dp(d), float(alpha_in), _dp(o))
        return dict(ground=o[0], partial=o[1], cfl=o[2], full=o[3])

    def intersected(self):
        return bool(self.L.cipc_oracle_intersected(self.h))


def pt_ccd(p, d, eta):
    p = np.ascontiguousarray(p, dtype=np.float64).reshape(-1)
    d = np.ascontiguousarray(d, dtype=np.float64).reshape(-1)
    return lib().cipc_oracle_pt_ccd(_dp(p), _dp(d), eta)


def ee_ccd(p, d, eta):
    p = np.ascontiguousarray(p, dtype=np.float64).reshape(-1)
    d = np.ascontiguousarray(d, dtype=np.float64).reshape(-1)
    return lib().cipc_oracle_ee_ccd(_dp(p), _dp(d), eta)


def snh(F, u, r):
    F = np.ascontiguousarray(F, dtype=np.float64).reshape(-1)
    P = np.zeros(9); H = np.zeros(81); psi = np.zeros(1)
    lib().cipc_oracle_snh(_dp(F), u, r, _dp(P), _dp(H), _dp(psi))
    return P.reshape(3, 3), H.reshape(9, 9), psi[0]


def distance(kind, pts):
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1)
    n = {0: 6, 1: 9}.get(kind, 12)
    g = np.zeros(n); H = np.zeros(n * n)
    d = lib().cipc_oracle_distance(kind, _dp(pts), _dp(g), _dp(H))
    return d, g, H.reshape(n, n)


def hinge(x, rest, k):
    """One hinge bending element (4 x 3 positions and rest positions: edge
    start, edge end, first and second opposite vertex): energy, gradient (12)
    and the PSD-projected Hessian (12 x 12)."""
    x = np.ascontiguousarray(x, np.float64).reshape(12)
    r = np.ascontiguousarray(rest, np.float64).reshape(12)
    g = np.zeros(12)
    H = np.zeros((12, 12))
    e = lib().cipc_oracle_hinge(_dp(x), _dp(r), float(k), _dp(g), _dp(H))
    return e, g, H


def linear_solve(nv, rowptr, col, val, rhs, method="pcg", tol=1e-6, max_iter=10000, threads=1, xyz=None):
    rowptr = np.ascontiguousarray(rowptr, np.int32); col = np.ascontiguousarray(col, np.int32)
    val = np.ascontiguousarray(val, np.float64); rhs = np.ascontiguousarray(rhs, np.float64)
    sol = np.zeros(3 * nv)
    it = C.c_int(0); rr = C.c_double(0)
    if xyz is not None:
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(3 * nv)
    rc = lib().cipc_oracle_linear_solve(nv, _ip(rowptr), _ip(col), _dp(val), _dp(rhs), _dp(sol),
                                       {"direct": 0, "pcg": 1, "multifrontal": 2}[method], tol, max_iter, C.byref(it), C.byref(rr),
                                       threads, None if xyz is None else _dp(xyz))
    if rc != 0:
        raise RuntimeError("oracle linear solve failed")
    return sol, it.value, rr.value
