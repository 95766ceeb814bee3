"""Test infrastructure only: the reference's own demo scenes as raw scene dicts.

Restates the scene builders of CPU IPC/Simulator.cpp:265-399, the parameter
file Assets/scene/parameterSetting.txt and the Gmsh/OBJ loaders of
CPU IPC/SimulationMesh.cpp:174-362, 545-716, so the oracle can be pinned
against the known answers the reference's documentation quotes.  The meshes
are read from tests/golden/assets (copies of the reference's Assets files,
MPL-2.0, see the NOTICE there); CIPC_REFERENCE_ASSETS names another Assets
directory instead.  Nothing here is shipped or used by the library.
"""
import math
import os

import numpy as np

BUNDLED_ASSETS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden", "assets")
REFERENCE_ASSETS = os.environ.get("CIPC_REFERENCE_ASSETS", BUNDLED_ASSETS)

SCENE_FILES = {
    "twisting_mat": ["tetrahedraMesh/ipcmesh/mat40x40.msh"],
    "cloth_bunny": ["triangleMesh/planes/plane1024.obj", "tetrahedraMesh/bunny.msh"],
    "bunny2": ["tetrahedraMesh/bunny2.msh"],
}


def assets_available(scene="twisting_mat"):
    """Whether the mesh files of a reference scene are present."""
    return all(os.path.isfile(os.path.join(REFERENCE_ASSETS, f)) for f in SCENE_FILES[scene])


def load_gmsh(path, scale=1.0, offset=(0.0, 0.0, 0.0)):
    """mesh3D::load_tetrahedraMesh: compact 3-field or Gmsh 2.2 4-field nodes,
    compact 5-field or typed (type 4) tetrahedron rows."""
    verts, tets = [], []
    node_index = {}
    nfields = 0
    with open(path) as f:
        lines = [ln.rstrip("\r\n") for ln in f]
    i = 0
    while i < len(lines):
        line = lines[i].rstrip("\r")
        if line == "$Nodes":
            n = int(lines[i + 1].split()[0])
            for k in range(n):
                fields = lines[i + 2 + k].split()
                if nfields == 0:
                    nfields = len(fields)
                if len(fields) == 3:
                    nid, xyz = k + 1, [float(v) for v in fields]
                else:
                    nid, xyz = int(fields[0]), [float(v) for v in fields[1:4]]
                node_index[nid] = k
                verts.append([scale * xyz[0] + offset[0], scale * xyz[1] + offset[1], scale * xyz[2] + offset[2]])
            i += 2 + n
            continue
        if line == "$Elements":
            n = int(lines[i + 1].split()[0])
            for k in range(n):
                fields = [int(v) for v in lines[i + 2 + k].split()]
                if nfields == 3 and len(fields) == 5:
                    ids = fields[1:5]
                else:
                    if fields[1] != 4:
                        continue
                    ids = fields[-4:]
                tets.append([node_index[v] for v in ids])
            break
        i += 1
    return np.array(verts, dtype=np.float64), np.array(tets, dtype=np.int32)


def load_obj(path, scale=1.0, offset=(0.0, 0.0, 0.0)):
    """mesh3D::load_triangleMesh: 'v' rows and fan-triangulated 'f' rows."""
    verts, tris = [], []
    with open(path) as f:
        for line in f:
            if len(line) <= 1:
                continue
            key = line[:2]
            if key == "v ":
                x, y, z = [float(v) for v in line[2:].split()[:3]]
                verts.append([scale * x + offset[0], scale * y + offset[1], scale * z + offset[2]])
            elif key == "f ":
                toks = line.split()
                for j in range(3, len(toks)):
                    tri = [toks[1], toks[j - 1], toks[j]]
                    tris.append([int(t.split("/")[0]) - 1 for t in tri])
    return np.array(verts, dtype=np.float64), np.array(tris, dtype=np.int32)


def parameter_settings():
    """Assets/scene/parameterSetting.txt as loadSettings() reads it."""
    return dict(density=1000.0, E=1e4, nu=0.49, friction=0.4, thickness=0.001, clothE=1e4, shearE=1e1,
                bendE=1e4, cloth_density=200.0, strainRate=1e2, use_barrier=1, drag=0.0, dt=0.01,
                newtonThr=1e-2, relDhat=1e-3, apply_gravity=1, quasi_static=0, quad_bending=1)


def twisting_mat(soft=False):
    """buildTwistingMatScene (Simulator.cpp:265-330), hard Dirichlet or soft targets."""
    p = parameter_settings()
    p["E"] = 1e6
    p["quasi_static"] = 1
    p["apply_gravity"] = 0
    x, tets = load_gmsh(os.path.join(REFERENCE_ASSETS, "tetrahedraMesh/ipcmesh/mat40x40.msh"))
    lo, hi = x.min(axis=0), x.max(axis=0)
    eps = 1e-4
    sel = np.nonzero((x[:, 0] < lo[0] + eps) | (x[:, 0] > hi[0] - eps))[0].astype(np.int32)
    btype = np.zeros(len(x), np.int32)
    scene = dict(x=x, tets=tets, tris=np.zeros((0, 3), np.int32), btype=btype, params=p,
                 bbox_min=lo.tolist(), bbox_max=hi.tolist())
    rate = 3.14 / 5
    if soft:
        scene["soft"] = dict(idx=sel, weight=100.0, motion=1, rate=rate)
    else:
        btype[sel] = 1
        scene["dirichlet"] = dict(idx=sel, motion=1, rate=rate)
    return scene


def cloth_bunny(hinge=False):
    """buildClothOverBunnyScene (Simulator.cpp:332-382); hinge=True selects the
    dihedral-angle bending the reference builds without USE_QUADRATIC_BENDING."""
    p = parameter_settings()
    p["E"] = 1e4
    if hinge:
        p["quad_bending"] = 2
    xc, tris = load_obj(os.path.join(REFERENCE_ASSETS, "triangleMesh/planes/plane1024.obj"))
    a = math.pi / 2
    R = np.array([[1, 0, 0], [0, math.cos(a), -math.sin(a)], [0, math.sin(a), math.cos(a)]])
    xc = np.array([R @ v for v in xc])
    lo, hi = xc.min(axis=0), xc.max(axis=0)
    xb, tets = load_gmsh(os.path.join(REFERENCE_ASSETS, "tetrahedraMesh/bunny.msh"), 0.5, (0.0, -0.5, 0.0))
    lo = np.minimum(lo, xb.min(axis=0))
    hi = np.maximum(hi, xb.max(axis=0))
    x = np.concatenate([xc, xb])
    tets = tets + len(xc)
    btype = np.zeros(len(x), np.int32)
    return dict(x=x, tets=tets, tris=tris, btype=btype, params=p, bbox_min=lo.tolist(), bbox_max=hi.tolist())


def bunny2():
    """buildBunny2Scene (Simulator.cpp:382-399): two copies of bunny2.msh at
    scale 0.2, offset (0, 0.65, 0) and (0, 0, 0), Young's modulus 1e5, the
    rest from parameterSetting.txt."""
    p = parameter_settings()
    p["E"] = 1e5
    path = os.path.join(REFERENCE_ASSETS, "tetrahedraMesh/bunny2.msh")
    xa, ta = load_gmsh(path, 0.2, (0.0, 0.65, 0.0))
    xb, tb = load_gmsh(path, 0.2, (0.0, 0.0, 0.0))
    x = np.concatenate([xa, xb])
    tets = np.concatenate([ta, tb + len(xa)]).astype(np.int32)
    btype = np.zeros(len(x), np.int32)
    return dict(x=x, tets=tets, tris=np.zeros((0, 3), np.int32), btype=btype, params=p,
                bbox_min=x.min(axis=0).tolist(), bbox_max=x.max(axis=0).tolist())
