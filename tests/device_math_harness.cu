// Host build of device math the kernels run, for the host tests
// (test_distance_derivs.py, test_svd3.py): the generated contact-distance
// derivatives (cpu-ipc_b200/csrc/distance_derivs.cuh) and the rotation-aware
// 3x3 SVD of the elastic kernels (cpu-ipc_b200/csrc/cipc_device.cuh).  Only
// host functions are called.
#include "distance_derivs.cuh"

extern "C" int dd_grad_hess(int kind, const double* v, double* g, double* H) {
    switch (kind) {
    case 1: g_PE(v, g); H_PE(v, H); return 9;
    case 2: g_PT(v, g); H_PT(v, H); return 12;
    case 3: g_EE(v, g); H_EE(v, H); return 12;
    case 4: g_EECross(v, g); H_EECross(v, H); return 12;
    default: return 0;
    }
}

// F, U, V row-major 3x3
extern "C" void svd3_host(const double* F9, double* U9, double* s3, double* V9) {
    double F[3][3], U[3][3], V[3][3];
    for (int i = 0; i < 9; ++i) F[i / 3][i % 3] = F9[i];
    svd3<double>(F, U, s3, V);
    for (int i = 0; i < 9; ++i) { U9[i] = U[i / 3][i % 3]; V9[i] = V[i / 3][i % 3]; }
}
