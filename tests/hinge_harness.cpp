// Host build of the library's hinge bending element math
// (cpu-ipc_b200/csrc/hinge_bending.cuh) for tests/test_hinge_math.py.
#include "hinge_bending.cuh"

extern "C" double hinge_element(const double* x, const double* rest, double k, double* g, double* H) {
    return cipc::hinge::energyGradHess(x, cipc::hinge::restWeight(rest), cipc::hinge::angle(rest), k, g, H);
}
extern "C" double hinge_angle(const double* x) { return cipc::hinge::angle(x); }
extern "C" void hinge_hess_column(const double* x, int j, double* col) { cipc::hinge::angleHessColumn(x, j, col); }
extern "C" double hinge_angle_hess_full(const double* x, double* H) {
    // hess(theta) from the 12-direction forward mode (k w = 1, d = 1, minus grad grad^T)
    double g[12];
    double th0 = cipc::hinge::angle(x) - 1.0;
    cipc::hinge::energyGradHess(x, 1.0, th0, 1.0, g, H);
    for (int i = 0; i < 12; ++i)
        for (int j = 0; j < 12; ++j) H[12 * i + j] -= g[i] * g[j];
    return 0.0;
}
