// Runtime files of the headless runner, in the reference's formats, so a run
// can be resumed from the reference's checkpoints and its outputs diffed
// against the reference's:
//
//   <output>/timeCost.txt           cumulative stage times, rewritten every step
//                                   (IPCSolver.cpp:1261-1273)
//   <output>/tempData/timeCost.txt  checkpoint totals: five cumulative stage ms,
//                                   cumulative step ms, Newton iterations, step
//                                   index, kappa, one per line at the stream's
//                                   default precision (IPCSolver.cpp:1318-1328)
//   <output>/tempData/vertex.txt    positions, "x y z" per vertex, 17 digits
//   <output>/tempData/vertexXtile.txt  inertial target, same layout
//                                   (mesh3D::output_tetTempData,
//                                   SimulationMesh.cpp:516-543)
//
// Loading follows mesh3D::load_tetTempData (SimulationMesh.cpp:470-514): both
// files must hold exactly nv vertices; anything short, unparsable or longer
// rejects the checkpoint.  The checkpoint totals are read as solveIPCStep
// reads them on the first step after a resume (IPCSolver.cpp:1085-1101).
// Host-only C++: no CUDA types.
#pragma once

#include <fstream>
#include <iomanip>
#include <string>
#include <vector>

#include <sys/stat.h>

namespace cipc_io {

// IPCSolverContext's running totals (IPCSolver.h:46-61)
struct RunTotals {
    double stageMs[5] = {0, 0, 0, 0, 0};  // assembly, linear, CCD, line search, post
    double stepMs = 0;
    long long newtonIterations = 0;
    int stepIndex = 0;
    double kappa = 0;
    double collisions = 0;
};

inline std::string joinPath(const std::string& dir, const std::string& name) {
    if (dir.empty()) return name;
    return dir.back() == '/' ? dir + name : dir + "/" + name;
}

inline bool makeDirectories(const std::string& dir) {
    if (dir.empty()) return true;
    std::string partial;
    for (size_t i = 0; i <= dir.size(); ++i) {
        if (i == dir.size() || dir[i] == '/') {
            if (!partial.empty()) {
                struct stat sb;
                if (stat(partial.c_str(), &sb) != 0 && mkdir(partial.c_str(), 0755) != 0) return false;
            }
        }
        if (i < dir.size()) partial += dir[i];
    }
    struct stat sb;
    return stat(dir.c_str(), &sb) == 0 && S_ISDIR(sb.st_mode);
}

inline std::string tempDirectory(const std::string& output) { return joinPath(output, "tempData"); }

inline bool writeVertexFile(const std::string& path, const std::vector<double>& v, int nv) {
    std::ofstream f(path);
    if (!f) return false;
    f << std::setprecision(17);
    for (int i = 0; i < nv; ++i) f << v[3 * i] << " " << v[3 * i + 1] << " " << v[3 * i + 2] << std::endl;
    f.flush();
    return f.good();
}

// positions and inertial target (3 nv doubles each)
inline bool writeVertexState(const std::string& output, const std::vector<double>& x, const std::vector<double>& xTilde, int nv) {
    const std::string dir = tempDirectory(output);
    if (!makeDirectories(dir)) return false;
    return writeVertexFile(joinPath(dir, "vertex.txt"), x, nv) && writeVertexFile(joinPath(dir, "vertexXtile.txt"), xTilde, nv);
}

inline bool loadVertexState(const std::string& output, int nv, std::vector<double>& x, std::vector<double>& xTilde) {
    const std::string dir = tempDirectory(output);
    std::ifstream f1(joinPath(dir, "vertex.txt")), f2(joinPath(dir, "vertexXtile.txt"));
    if (!f1 || !f2 || nv < 0) return false;
    std::vector<double> a(3 * (size_t)nv), b(3 * (size_t)nv);
    for (size_t i = 0; i < a.size(); ++i)
        if (!(f1 >> a[i])) return false;
    for (size_t i = 0; i < b.size(); ++i)
        if (!(f2 >> b[i])) return false;
    double extra;
    if (f1 >> extra || f2 >> extra) return false;  // a checkpoint of another mesh
    x.swap(a);
    xTilde.swap(b);
    return true;
}

inline bool writeCheckpointTotals(const std::string& output, const RunTotals& t) {
    const std::string dir = tempDirectory(output);
    if (!makeDirectories(dir)) return false;
    std::ofstream f(joinPath(dir, "timeCost.txt"));
    if (!f) return false;
    for (double ms : t.stageMs) f << ms << std::endl;
    f << t.stepMs << std::endl;
    f << t.newtonIterations << std::endl;
    f << t.stepIndex << std::endl;
    f << t.kappa << std::endl;
    return f.good();
}

// returns false (and leaves t alone) when the file is absent; a short file
// fills the leading fields, as the reference's extraction chain does
inline bool loadCheckpointTotals(const std::string& output, RunTotals& t) {
    std::ifstream f(joinPath(tempDirectory(output), "timeCost.txt"));
    if (!f) return false;
    f >> t.stageMs[0] >> t.stageMs[1] >> t.stageMs[2] >> t.stageMs[3] >> t.stageMs[4] >> t.stepMs >> t.newtonIterations >>
        t.stepIndex >> t.kappa;
    return true;
}

// the per-step summary <output>/timeCost.txt
inline bool writeTimeSummary(const std::string& output, const RunTotals& t) {
    if (!makeDirectories(output)) return false;
    std::ofstream f(joinPath(output, "timeCost.txt"));
    if (!f) return false;
    const double averageCollision = t.newtonIterations > 0 ? t.collisions / t.newtonIterations : 0.0;
    for (int k = 0; k < 5; ++k) f << "time" << k << ": " << t.stageMs[k] / 1000.0 << std::endl;
    f << "timeAll: " << t.stepMs / 1000.0 << std::endl;
    f << "total iter: " << t.newtonIterations << std::endl;
    f << "frames: " << t.stepIndex << std::endl;
    f << "totalCollisionNum: " << t.collisions << std::endl;
    f << "averageCollision: " << averageCollision << std::endl;
    return f.good();
}

}  // namespace cipc_io
