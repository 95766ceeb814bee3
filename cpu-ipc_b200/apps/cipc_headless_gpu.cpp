// cipc_headless_gpu: the reference's headless runner (apps/cipc_headless.cpp)
// on the GPU pipeline.  Same command-line shape, the same scenes where the
// reference's assets are supplied (--assets DIR: twisting-mat,
// twisting-mat-soft, cloth-bunny, bunny2, built as Simulator.cpp:265-399 builds them
// from Assets/scene/parameterSetting.txt and the Gmsh/OBJ meshes), plus the
// synthetic benchmark scenes (two-cubes, cloth-drape).  Writes metrics.csv
// with the reference's columns (IPCSolver.cpp:1286-1315; the PARDISO columns
// are zero, the PCG iteration count and residual are appended), the
// reference's timeCost.txt summary and, with --write-checkpoints, its
// checkpoint files every tenth step; --resume restarts from such a checkpoint
// (the reference's or this runner's).  Prints the reference's RESULT line
// (cipc_headless.cpp:146-175).
//
// Links only against libcipc_gpu.so through include/cipc_gpu.h.
#include "cipc_gpu.h"
#include "runtime_files.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <vector>

namespace {

struct Options {
    std::string scene = "cloth-drape";
    std::string assets;
    std::string output;
    std::string weights;
    int steps = 1;
    int cloth = 128;
    int cells = 10;
    int precision = CIPC_PRECISION_MIXED;
    int precond = CIPC_PRECOND_BLOCK_JACOBI;
    int broadPhase = CIPC_BROAD_PHASE_LBVH;  // cipc_headless --broad-phase
    bool writeOutput = true;
    bool verbose = false;
    bool disableBarrier = false;
    bool resume = false;            // cipc_headless --resume
    bool writeCheckpoints = false;  // cipc_headless --write-checkpoints
    bool hingeBending = false;      // the reference built without USE_QUADRATIC_BENDING
};

void usage(const char* exe) {
    std::cout << "Usage: " << exe << " [options]\n"
              << "  --scene cloth-drape|two-cubes|twisting-mat|twisting-mat-soft|cloth-bunny|bunny2 (default cloth-drape)\n"
              << "  --assets DIRECTORY      the reference's Assets/ tree (twisting-mat, cloth-bunny, bunny2)\n"
              << "  --steps N\n"
              << "  --cloth N               cloth-drape: N x N cloth vertices (default 128)\n"
              << "  --cells N               cube cells per side (default 10 cloth-drape, 8 two-cubes)\n"
              << "  --linear-solver gpu-pcg\n"
              << "  --precision fp64|mixed  (default mixed)\n"
              << "  --precond jacobi|learned|fsai (default jacobi)\n"
              << "  --broad-phase lbvh|spatial-hash (default lbvh)\n"
              << "  --weights FILE          learned-preconditioner weights (raw float32)\n"
              << "  --output DIRECTORY      metrics.csv, timeCost.txt and tempData/ go here\n"
              << "  --resume                start from the checkpoint in DIRECTORY/tempData\n"
              << "  --write-checkpoints     write a checkpoint to DIRECTORY/tempData every tenth step\n"
              << "  --hinge-bending         dihedral-angle bending instead of quadratic bending\n"
              << "  --disable-barrier\n"
              << "  --no-output\n"
              << "  --verbose\n"
              << "  --help\n";
}

int nonNegative(const std::string& v, const char* opt) {
    size_t used = 0;
    int r = std::stoi(v, &used);
    if (used != v.size() || r < 0) throw std::invalid_argument(std::string(opt) + " expects a non-negative integer");
    return r;
}

Options parse(int argc, char** argv) {
    Options o;
    bool cellsGiven = false;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto value = [&](const char* opt) -> std::string {
            if (++i >= argc) throw std::invalid_argument(std::string(opt) + " requires a value");
            return argv[i];
        };
        if (a == "--scene") o.scene = value("--scene");
        else if (a == "--assets") o.assets = value("--assets");
        else if (a == "--steps") o.steps = nonNegative(value("--steps"), "--steps");
        else if (a == "--cloth") o.cloth = nonNegative(value("--cloth"), "--cloth");
        else if (a == "--cells") { o.cells = nonNegative(value("--cells"), "--cells"); cellsGiven = true; }
        else if (a == "--output") o.output = value("--output");
        else if (a == "--weights") o.weights = value("--weights");
        else if (a == "--linear-solver") {
            std::string v = value("--linear-solver");
            if (v != "gpu-pcg") throw std::invalid_argument("linear solver " + v + " is not part of this build (use gpu-pcg)");
        } else if (a == "--precision") {
            std::string v = value("--precision");
            if (v == "fp64") o.precision = CIPC_PRECISION_FP64;
            else if (v == "mixed") o.precision = CIPC_PRECISION_MIXED;
            else throw std::invalid_argument("unknown precision: " + v);
        } else if (a == "--precond") {
            std::string v = value("--precond");
            if (v == "jacobi") o.precond = CIPC_PRECOND_BLOCK_JACOBI;
            else if (v == "learned") o.precond = CIPC_PRECOND_LEARNED;
            else if (v == "fsai") o.precond = CIPC_PRECOND_FSAI;
            else throw std::invalid_argument("unknown preconditioner: " + v);
        } else if (a == "--broad-phase") {
            std::string v = value("--broad-phase");
            if (v == "lbvh") o.broadPhase = CIPC_BROAD_PHASE_LBVH;
            else if (v == "spatial-hash") o.broadPhase = CIPC_BROAD_PHASE_SPATIAL_HASH;
            else throw std::invalid_argument("unknown broad phase: " + v);
        } else if (a == "--disable-barrier") o.disableBarrier = true;
        else if (a == "--resume") o.resume = true;
        else if (a == "--write-checkpoints") o.writeCheckpoints = true;
        else if (a == "--hinge-bending") o.hingeBending = true;
        else if (a == "--no-output") o.writeOutput = false;
        else if (a == "--verbose") o.verbose = true;
        else if (a == "--help" || a == "-h") { usage(argv[0]); std::exit(0); }
        else throw std::invalid_argument("unknown option: " + a);
    }
    if (!cellsGiven && o.scene == "two-cubes") o.cells = 8;
    return o;
}

// ---------------------------------------------------------------------------
// scene data
// ---------------------------------------------------------------------------
struct Params {
    double density = 1000, E = 1e4, nu = 0.49, friction = 0.4, thickness = 1e-3, clothE = 1e4, shearE = 10, bendE = 1e4;
    double cloth_density = 200, strainRate = 100, drag = 0, dt = 0.01, newtonThr = 1e-2, relDhat = 1e-3;
    int use_barrier = 1, apply_gravity = 1, quasi_static = 0;
};

struct Scene {
    std::vector<double> x;
    std::vector<int> tets, tris, btype;
    std::vector<int> softIdx, dirIdx;
    double softW = 0, motionRate = 0;
    int softMotion = CIPC_MOTION_NONE, dirMotion = CIPC_MOTION_NONE;
    Params p;
    int firstMeshVertices = 0;  // the RESULT line sums over the first mesh, as the reference does
};

// Assets/scene/parameterSetting.txt: key value pairs (loadSettings,
// Simulator.cpp:174-263); unknown keys are rejected like the reference does.
Params loadSettings(const std::string& path) {
    Params p;
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::map<std::string, double*> d = {
        {"volume_mesh_density", &p.density}, {"volume_mesh_YoungsModulus", &p.E}, {"poisson_rate", &p.nu},
        {"friction_rate", &p.friction}, {"triangle(cloth)_mesh_thickness", &p.thickness},
        {"triangle(cloth)_mesh_YoungsModulus", &p.clothE}, {"triangle(cloth)_mesh_shearYoungsModulus", &p.shearE},
        {"triangle(cloth)_mesh_bendingYoungsModulus", &p.bendE}, {"triangle(cloth)_mesh_density", &p.cloth_density},
        {"strainRate", &p.strainRate}, {"drag_coeff", &p.drag}, {"ipc_time_step", &p.dt},
        {"Newton_solver_threshold", &p.newtonThr}, {"IPC_ralative_dHat", &p.relDhat}};
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream in(line);
        std::string key;
        double v;
        if (!(in >> key)) continue;
        if (!(in >> v)) throw std::runtime_error("missing value for " + key + " in " + path);
        if (key == "enable_collision_handling") { p.use_barrier = v != 0; continue; }
        auto it = d.find(key);
        if (it == d.end()) throw std::runtime_error("unknown setting " + key + " in " + path);
        *it->second = v;
    }
    return p;
}

// Gmsh tetrahedral mesh (mesh3D::load_tetrahedraMesh, SimulationMesh.cpp:174-280):
// compact 3-field or indexed 4-field node rows, compact 5-field or typed
// (element type 4) tetrahedron rows.
void loadGmsh(const std::string& path, double scale, const double off[3], std::vector<double>& x, std::vector<int>& tets) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::vector<std::string> lines;
    std::string line;
    while (std::getline(f, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        lines.push_back(line);
    }
    std::map<long long, int> index;
    int base = (int)(x.size() / 3);
    size_t nfields = 0;
    for (size_t i = 0; i < lines.size(); ++i) {
        if (lines[i] == "$Nodes") {
            int n = std::stoi(lines[i + 1]);
            for (int k = 0; k < n; ++k) {
                std::istringstream in(lines[i + 2 + k]);
                std::vector<double> v;
                double t;
                while (in >> t) v.push_back(t);
                if (nfields == 0) nfields = v.size();
                long long id = v.size() == 3 ? k + 1 : (long long)v[0];
                const double* xyz = v.size() == 3 ? &v[0] : &v[1];
                index[id] = k;
                for (int q = 0; q < 3; ++q) x.push_back(scale * xyz[q] + off[q]);
            }
            i += 1 + n;
        } else if (lines[i] == "$Elements") {
            int n = std::stoi(lines[i + 1]);
            for (int k = 0; k < n; ++k) {
                std::istringstream in(lines[i + 2 + k]);
                std::vector<long long> v;
                long long t;
                while (in >> t) v.push_back(t);
                const long long* ids;
                if (nfields == 3 && v.size() == 5) ids = &v[1];
                else if (v.size() >= 6 && v[1] == 4) ids = &v[v.size() - 4];
                else continue;
                for (int q = 0; q < 4; ++q) tets.push_back(base + index.at(ids[q]));
            }
            break;
        }
    }
    if (tets.empty()) throw std::runtime_error("no tetrahedra in " + path);
}

// OBJ triangle mesh (mesh3D::load_triangleMesh, SimulationMesh.cpp:300-362):
// 'v' rows and fan-triangulated 'f' rows.
void loadObj(const std::string& path, std::vector<double>& x, std::vector<int>& tris) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open " + path);
    int base = (int)(x.size() / 3);
    std::string line;
    while (std::getline(f, line)) {
        if (line.size() < 2) continue;
        if (line[0] == 'v' && line[1] == ' ') {
            std::istringstream in(line.substr(2));
            double a, b, c;
            in >> a >> b >> c;
            x.push_back(a); x.push_back(b); x.push_back(c);
        } else if (line[0] == 'f' && line[1] == ' ') {
            std::istringstream in(line.substr(2));
            std::vector<int> ids;
            std::string tok;
            while (in >> tok) ids.push_back(std::stoi(tok.substr(0, tok.find('/'))) - 1);
            for (size_t j = 2; j < ids.size(); ++j) {
                tris.push_back(base + ids[0]); tris.push_back(base + ids[j - 1]); tris.push_back(base + ids[j]);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// synthetic benchmark meshes (the same generators as cpu-ipc_b200/cipc.py)
// ---------------------------------------------------------------------------
double lin(double a, double b, int n, int i) { return i == n ? b : a + i * ((b - a) / n); }

// n^3 cells, 6 tets per cell around the v0-v7 diagonal, positively oriented
void cubeMesh(int n, double size, const double c[3], std::vector<double>& x, std::vector<int>& tets) {
    int base = (int)(x.size() / 3), m = n + 1;
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j)
            for (int k = 0; k < m; ++k) {
                x.push_back(lin(-0.5 * size, 0.5 * size, n, i) + c[0]);
                x.push_back(lin(-0.5 * size, 0.5 * size, n, j) + c[1]);
                x.push_back(lin(-0.5 * size, 0.5 * size, n, k) + c[2]);
            }
    auto id = [&](int i, int j, int k) { return base + (i * m + j) * m + k; };
    const int pat[6][4] = {{0, 1, 3, 7}, {0, 1, 7, 5}, {0, 2, 7, 3}, {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 7, 6}};
    for (int t = 0; t < 6; ++t)
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < n; ++k) {
                    int v[8] = {id(i, j, k), id(i + 1, j, k), id(i, j + 1, k), id(i + 1, j + 1, k),
                                id(i, j, k + 1), id(i + 1, j, k + 1), id(i, j + 1, k + 1), id(i + 1, j + 1, k + 1)};
                    int q[4] = {v[pat[t][0]], v[pat[t][1]], v[pat[t][2]], v[pat[t][3]]};
                    const double* p0 = &x[3 * q[0]];
                    double a[3], b[3], d[3];
                    for (int r = 0; r < 3; ++r) { a[r] = x[3 * q[1] + r] - p0[r]; b[r] = x[3 * q[2] + r] - p0[r]; d[r] = x[3 * q[3] + r] - p0[r]; }
                    double vol = (a[1] * b[2] - a[2] * b[1]) * d[0] + (a[2] * b[0] - a[0] * b[2]) * d[1] + (a[0] * b[1] - a[1] * b[0]) * d[2];
                    if (vol < 0) std::swap(q[2], q[3]);
                    for (int r = 0; r < 4; ++r) tets.push_back(q[r]);
                }
}

// n x n vertex cloth in the xz-plane at height y, triangles wound for +y normals
void gridCloth(int n, double size, double y, std::vector<double>& x, std::vector<int>& tris) {
    int base = (int)(x.size() / 3);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k) {
            x.push_back(lin(-0.5 * size, 0.5 * size, n - 1, i));
            x.push_back(y);
            x.push_back(lin(-0.5 * size, 0.5 * size, n - 1, k));
        }
    auto id = [&](int i, int k) { return base + i * n + k; };
    for (int pass = 0; pass < 2; ++pass)
        for (int i = 0; i + 1 < n; ++i)
            for (int k = 0; k + 1 < n; ++k) {
                int a = id(i, k), b = id(i + 1, k), c = id(i, k + 1), d = id(i + 1, k + 1);
                if (pass == 0) { tris.push_back(a); tris.push_back(d); tris.push_back(b); }
                else { tris.push_back(a); tris.push_back(c); tris.push_back(d); }
            }
}

Scene buildScene(const Options& o) {
    Scene s;
    if (o.scene == "cloth-drape") {
        // n x n 1 m cloth 0.1 m above a fixed 0.5 m tet cube (external collider)
        gridCloth(o.cloth, 1.0, 0.25 + 0.1, s.x, s.tris);
        s.firstMeshVertices = (int)(s.x.size() / 3);
        const double c[3] = {0, 0, 0};
        cubeMesh(o.cells, 0.5, c, s.x, s.tets);
        s.btype.assign(s.x.size() / 3, 0);
        for (size_t v = s.firstMeshVertices; v < s.btype.size(); ++v) s.btype[v] = 2;
        Params& p = s.p;
        p.E = 1e5; p.nu = 0.3; p.clothE = 1e4; p.shearE = 10; p.thickness = 1e-3; p.cloth_density = 200;
        p.bendE = 1e-3 * 12 * (1 - p.nu * p.nu) / 1e-9;  // plate rigidity 1e-3
        p.friction = 0.3; p.dt = 0.005; p.newtonThr = 1e-2; p.relDhat = 1e-3; p.density = 1000; p.strainRate = 100;
    } else if (o.scene == "two-cubes") {
        const double gap = 0.05;
        const double ca[3] = {0, -1.0 + gap + 0.5, 0}, cb[3] = {0, -1.0 + gap + 1.0 + gap + 0.5, 0};
        cubeMesh(o.cells, 1.0, ca, s.x, s.tets);
        s.firstMeshVertices = (int)(s.x.size() / 3);
        cubeMesh(o.cells, 1.0, cb, s.x, s.tets);
        s.btype.assign(s.x.size() / 3, 0);
        Params& p = s.p;
        p.E = 1e5; p.nu = 0.4; p.density = 1000; p.friction = 0.2; p.dt = 0.01; p.newtonThr = 1e-6; p.relDhat = 1e-3;
    } else if (o.scene == "twisting-mat" || o.scene == "twisting-mat-soft" || o.scene == "cloth-bunny" || o.scene == "bunny2") {
        if (o.assets.empty()) throw std::invalid_argument("--scene " + o.scene + " needs --assets (the reference's Assets directory)");
        s.p = loadSettings(o.assets + "/scene/parameterSetting.txt");
        const double zero[3] = {0, 0, 0};
        if (o.scene == "bunny2") {
            // buildBunny2Scene (Simulator.cpp:382-399): two copies of bunny2.msh at
            // scale 0.2, the upper one raised by 0.65
            s.p.E = 1e5;
            const double up[3] = {0.0, 0.65, 0.0};
            loadGmsh(o.assets + "/tetrahedraMesh/bunny2.msh", 0.2, up, s.x, s.tets);
            s.firstMeshVertices = (int)(s.x.size() / 3);
            loadGmsh(o.assets + "/tetrahedraMesh/bunny2.msh", 0.2, zero, s.x, s.tets);
            s.btype.assign(s.x.size() / 3, 0);
        } else if (o.scene == "cloth-bunny") {
            // buildClothOverBunnyScene (Simulator.cpp:332-382): plane1024 rotated by pi/2
            // about x, bunny.msh scaled 0.5 and lowered by 0.5
            s.p.E = 1e4;
            std::vector<double> xc;
            loadObj(o.assets + "/triangleMesh/planes/plane1024.obj", xc, s.tris);
            const double a = 3.14159265358979323846 / 2;
            for (size_t v = 0; v < xc.size() / 3; ++v) {
                double y = xc[3 * v + 1], z = xc[3 * v + 2];
                s.x.push_back(xc[3 * v]);
                s.x.push_back(std::cos(a) * y - std::sin(a) * z);
                s.x.push_back(std::sin(a) * y + std::cos(a) * z);
            }
            s.firstMeshVertices = (int)(s.x.size() / 3);
            const double off[3] = {0.0, -0.5, 0.0};
            loadGmsh(o.assets + "/tetrahedraMesh/bunny.msh", 0.5, off, s.x, s.tets);
            s.btype.assign(s.x.size() / 3, 0);
        } else {
            // buildTwistingMatScene (Simulator.cpp:265-330): both x-ends rotate about x
            s.p.E = 1e6; s.p.quasi_static = 1; s.p.apply_gravity = 0;
            loadGmsh(o.assets + "/tetrahedraMesh/ipcmesh/mat40x40.msh", 1.0, zero, s.x, s.tets);
            s.firstMeshVertices = (int)(s.x.size() / 3);
            int nv = s.firstMeshVertices;
            double lo = 1e300, hi = -1e300;
            for (int v = 0; v < nv; ++v) { lo = std::min(lo, s.x[3 * v]); hi = std::max(hi, s.x[3 * v]); }
            s.btype.assign(nv, 0);
            std::vector<int> sel;
            for (int v = 0; v < nv; ++v)
                if (s.x[3 * v] < lo + 1e-4 || s.x[3 * v] > hi - 1e-4) sel.push_back(v);
            s.motionRate = 3.14 / 5;
            if (o.scene == "twisting-mat-soft") {
                s.softIdx = sel; s.softW = 100.0; s.softMotion = CIPC_MOTION_TWIST_X;
            } else {
                s.dirIdx = sel; s.dirMotion = CIPC_MOTION_TWIST_X;
                for (int v : sel) s.btype[v] = 1;
            }
        }
    } else {
        throw std::invalid_argument("unknown scene: " + o.scene);
    }
    if (o.disableBarrier) s.p.use_barrier = 0;
    return s;
}

void check(int rc, cipc_gpu_context* ctx, const char* what) {
    if (rc == CIPC_OK) return;
    std::string msg = ctx ? cipc_gpu_last_error(ctx) : cipc_gpu_create_error();
    // the reference throws std::invalid_argument / std::runtime_error
    if (rc == CIPC_ERR_INVALID_ARGUMENT) throw std::invalid_argument(std::string(what) + ": " + msg);
    throw std::runtime_error(std::string(what) + ": " + msg);
}

}  // namespace

int main(int argc, char** argv) {
    cipc_gpu_context* ctx = nullptr;
    try {
        const Options o = parse(argc, argv);
        Scene s = buildScene(o);
        const int nv = (int)(s.x.size() / 3);
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int v = 0; v < nv; ++v)
            for (int q = 0; q < 3; ++q) { lo[q] = std::min(lo[q], s.x[3 * v + q]); hi[q] = std::max(hi[q], s.x[3 * v + q]); }

        cipc_scene_desc d{};
        d.nv = nv; d.nt = (int)(s.tets.size() / 4); d.nf = (int)(s.tris.size() / 3);
        d.x = s.x.data(); d.tets = s.tets.data(); d.tris = s.tris.data(); d.btype = s.btype.data();
        const Params& p = s.p;
        d.density = p.density; d.cloth_density = p.cloth_density; d.thickness = p.thickness; d.E = p.E; d.nu = p.nu;
        d.clothE = p.clothE; d.shearE = p.shearE; d.bendE = p.bendE; d.strainRate = p.strainRate; d.friction = p.friction;
        d.dt = p.dt; d.drag = p.drag; d.newtonThr = p.newtonThr; d.relDhat = p.relDhat;
        d.use_barrier = p.use_barrier; d.apply_gravity = p.apply_gravity; d.quasi_static = p.quasi_static; d.quad_bending = o.hingeBending ? 2 : 1;
        for (int q = 0; q < 3; ++q) { d.bboxMin[q] = lo[q]; d.bboxMax[q] = hi[q]; }
        d.nsoft = (int)s.softIdx.size(); d.softIdx = s.softIdx.data(); d.softW = s.softW; d.softMotion = s.softMotion; d.softRate = s.motionRate;
        d.ndir = (int)s.dirIdx.size(); d.dirIdx = s.dirIdx.data(); d.dirMotion = s.dirMotion; d.dirRate = s.motionRate;

        cipc_linear_options lo_{};
        lo_.backend = CIPC_LINEAR_GPU_PCG;
        lo_.precision = o.precision;
        lo_.preconditioner = o.precond;
        lo_.relativeTolerance = 1e-6;
        lo_.maximumIterations = 10000;
        check(cipc_gpu_create(&d, &lo_, &ctx), nullptr, "cipc_gpu_create");
        if (o.broadPhase != CIPC_BROAD_PHASE_LBVH) check(cipc_gpu_set_broad_phase(ctx, o.broadPhase), ctx, "cipc_gpu_set_broad_phase");

        if (!o.weights.empty()) {
            int n = cipc_gpu_precond_num_params();
            std::vector<float> w(n);
            std::ifstream f(o.weights, std::ios::binary);
            if (!f.read(reinterpret_cast<char*>(w.data()), sizeof(float) * (size_t)n))
                throw std::runtime_error("weights file " + o.weights + " must hold " + std::to_string(n) + " float32 values");
            check(cipc_gpu_precond_set_weights(ctx, w.data(), n), ctx, "cipc_gpu_precond_set_weights");
        }

        const std::string outDir = o.output.empty() ? "headless_output" : o.output;
        cipc_io::RunTotals totals;
        // resume: positions and inertial target from tempData (V_prev = x),
        // then the collision sets at those positions (Simulator.cpp:510-519);
        // the running totals, step index and kappa as the first step reads
        // them (IPCSolver.cpp:1085-1101)
        bool resumed = false;
        if (o.resume) {
            std::vector<double> xr, xt;
            resumed = cipc_io::loadVertexState(outDir, nv, xr, xt);
            if (resumed) {
                check(cipc_gpu_set_state(ctx, 0, xr.data()), ctx, "cipc_gpu_set_state");
                check(cipc_gpu_set_state(ctx, 2, xr.data()), ctx, "cipc_gpu_set_state");
                check(cipc_gpu_set_state(ctx, 3, xt.data()), ctx, "cipc_gpu_set_state");
                long long counts[4];
                check(cipc_gpu_build_collision_sets(ctx, counts), ctx, "cipc_gpu_build_collision_sets");
                if (cipc_io::loadCheckpointTotals(outDir, totals))
                    check(cipc_gpu_set_kappa(ctx, totals.kappa), ctx, "cipc_gpu_set_kappa");
            }
            if (o.verbose) std::cout << (resumed ? "load temp data" : "no temp data") << std::endl;
        }

        std::ofstream metrics;
        if (o.writeOutput) {
            if (!cipc_io::makeDirectories(outDir)) throw std::runtime_error("invalid output directory " + outDir);
            // a resumed run appends to the metrics it continues (IPCSolver.cpp:1275-1285)
            bool hasContent = false;
            if (resumed) {
                std::ifstream existing(cipc_io::joinPath(outDir, "metrics.csv"));
                hasContent = existing && existing.peek() != std::ifstream::traits_type::eof();
            }
            metrics.open(cipc_io::joinPath(outDir, "metrics.csv"), resumed ? std::ios::out | std::ios::app : std::ios::out | std::ios::trunc);
            if (!metrics) throw std::runtime_error("invalid output directory " + outDir);
            if (!hasContent)
                metrics << "frame,step_ms,assembly_ms,linear_ms,ccd_ms,line_search_ms,post_ms,"
                           "newton,kappa_loops,backtracks,energy_backtracks,intersection_backtracks,"
                           "max_energy_backtracks_per_newton,newton_steps_over_two_backtracks,"
                           "mean_alpha,min_alpha,max_alpha,collisions,kappa,min_distance2,"
                           "ground_contacts,self_contacts,mollified_contacts,matrix_nnz,"
                           "symbolic_analyses,numeric_factorizations,pardiso_analysis_ms,"
                           "pardiso_factorization_ms,pardiso_solve_ms,linear_solver_threads,"
                           "factor_nnz,pcg_iterations,pcg_relative_residual\n";
        }
        cipc_step_stats st{};
        std::vector<double> xs(3 * (size_t)nv), xts(3 * (size_t)nv);
        for (int step = 0; step < o.steps; ++step) {
            check(cipc_gpu_step(ctx, &st), ctx, "cipc_gpu_step");
            const int frame = totals.stepIndex;  // IPCSolver.cpp:1104-1106
            totals.stageMs[0] += st.assemblyMilliseconds;
            totals.stageMs[1] += st.linearSolveMilliseconds;
            totals.stageMs[2] += st.ccdMilliseconds;
            totals.stageMs[3] += st.lineSearchMilliseconds;
            totals.stageMs[4] += st.postLineSearchMilliseconds;
            totals.stepMs += st.stepMilliseconds;
            totals.newtonIterations += st.newtonIterations;
            totals.collisions += st.collisions;
            totals.kappa = st.kappa;
            ++totals.stepIndex;
            if (o.verbose)
                std::cout << "step " << frame << " newton " << st.newtonIterations << " pcg " << st.pcgIterations << " ms " << st.stepMilliseconds
                          << std::endl;
            if (o.writeOutput) {
                if (!cipc_io::writeTimeSummary(outDir, totals)) throw std::runtime_error("cannot write timeCost.txt in " + outDir);
                metrics << std::setprecision(17) << frame << ',' << st.stepMilliseconds << ',' << st.assemblyMilliseconds << ','
                        << st.linearSolveMilliseconds << ',' << st.ccdMilliseconds << ',' << st.lineSearchMilliseconds << ','
                        << st.postLineSearchMilliseconds << ',' << st.newtonIterations << ',' << st.kappaIterations << ','
                        << st.lineSearchBacktracks << ',' << st.energyBacktracks << ',' << st.intersectionBacktracks << ','
                        << st.maximumEnergyBacktracksPerNewton << ',' << st.newtonStepsWithMoreThanTwoBacktracks << ','
                        << (st.newtonIterations > 0 ? st.acceptedStepSum / st.newtonIterations : 0.0) << ',' << st.minimumAcceptedStep << ','
                        << st.maximumAcceptedStep << ',' << st.collisions << ',' << st.kappa << ',' << st.minConstraintDistance2 << ','
                        << st.groundContacts << ',' << st.selfContacts << ',' << st.mollifiedContacts << ',' << 9 * st.matrixBlocks
                        << ",0,0,0,0,0,0,0," << st.pcgIterations << ',' << st.pcgRelativeResidual << '\n';
                metrics.flush();
                // checkpoint every tenth step (IPCSolver.cpp:1318-1332)
                if (o.writeCheckpoints && totals.stepIndex % 10 == 0) {
                    check(cipc_gpu_get_state(ctx, 0, xs.data()), ctx, "cipc_gpu_get_state");
                    check(cipc_gpu_get_state(ctx, 3, xts.data()), ctx, "cipc_gpu_get_state");
                    if (!cipc_io::writeCheckpointTotals(outDir, totals) || !cipc_io::writeVertexState(outDir, xs, xts, nv))
                        std::cerr << "Warning: failed to save simulation checkpoint" << std::endl;
                }
            }
        }
        // RESULT line over the first mesh (cipc_headless.cpp:146-175)
        std::vector<double> x(3 * (size_t)nv);
        check(cipc_gpu_get_state(ctx, 0, x.data()), ctx, "cipc_gpu_get_state");
        double sum[3] = {0, 0, 0}, sq = 0;
        for (int v = 0; v < s.firstMeshVertices; ++v)
            for (int q = 0; q < 3; ++q) { sum[q] += x[3 * v + q]; sq += x[3 * v + q] * x[3 * v + q]; }
        std::cout << std::setprecision(17) << "RESULT steps=" << o.steps << " vertices=" << s.firstMeshVertices << " sum_x=" << sum[0]
                  << " sum_y=" << sum[1] << " sum_z=" << sum[2] << " squared_norm_sum=" << sq;
        if (o.steps > 0)
            std::cout << " last_step_ms=" << st.stepMilliseconds << " last_newton=" << st.newtonIterations
                      << " last_min_distance2=" << st.minConstraintDistance2 << " last_matrix_blocks=" << st.matrixBlocks
                      << " last_pcg_iterations=" << st.pcgIterations;
        std::cout << std::endl;
        cipc_gpu_destroy(ctx);
    } catch (const std::exception& e) {
        if (ctx) cipc_gpu_destroy(ctx);
        std::cerr << "cipc_headless_gpu: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
