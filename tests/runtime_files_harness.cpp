// Host harness around cpu-ipc_b200/apps/runtime_files.h (the headless
// runner's checkpoint and summary files) for tests/test_runtime_files.py.
#include "runtime_files.h"

#include <vector>

extern "C" {

int rf_write_state(const char* out, const double* x, const double* xt, int nv) {
    std::vector<double> a(x, x + 3 * (size_t)nv), b(xt, xt + 3 * (size_t)nv);
    return cipc_io::writeVertexState(out, a, b, nv) ? 1 : 0;
}

int rf_load_state(const char* out, int nv, double* x, double* xt) {
    std::vector<double> a, b;
    if (!cipc_io::loadVertexState(out, nv, a, b)) return 0;
    for (size_t i = 0; i < a.size(); ++i) { x[i] = a[i]; xt[i] = b[i]; }
    return 1;
}

static cipc_io::RunTotals totals(const double* stage5, double stepMs, long long newton, int stepIndex, double kappa, double collisions) {
    cipc_io::RunTotals t;
    for (int k = 0; k < 5; ++k) t.stageMs[k] = stage5[k];
    t.stepMs = stepMs;
    t.newtonIterations = newton;
    t.stepIndex = stepIndex;
    t.kappa = kappa;
    t.collisions = collisions;
    return t;
}

int rf_write_totals(const char* out, const double* stage5, double stepMs, long long newton, int stepIndex, double kappa) {
    return cipc_io::writeCheckpointTotals(out, totals(stage5, stepMs, newton, stepIndex, kappa, 0.0)) ? 1 : 0;
}

int rf_load_totals(const char* out, double* stage5, double* stepMs, long long* newton, int* stepIndex, double* kappa) {
    cipc_io::RunTotals t;
    if (!cipc_io::loadCheckpointTotals(out, t)) return 0;
    for (int k = 0; k < 5; ++k) stage5[k] = t.stageMs[k];
    *stepMs = t.stepMs;
    *newton = t.newtonIterations;
    *stepIndex = t.stepIndex;
    *kappa = t.kappa;
    return 1;
}

int rf_write_summary(const char* out, const double* stage5, double stepMs, long long newton, int stepIndex, double collisions) {
    return cipc_io::writeTimeSummary(out, totals(stage5, stepMs, newton, stepIndex, 0.0, collisions)) ? 1 : 0;
}

}  // extern "C"
