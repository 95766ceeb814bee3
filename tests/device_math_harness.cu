// Host build of device math the kernels run, for the host tests
// (test_distance_derivs.py, test_svd3.py): the generated contact-distance
// derivatives (cpu-ipc_b200/csrc/distance_derivs.cuh, distance_rows.cuh) and the rotation-aware
// 3x3 SVD of the elastic kernels (cpu-ipc_b200/csrc/cipc_device.cuh).  Only
// host functions are called.
#include "distance_derivs.cuh"
#include "distance_rows.cuh"

extern "C" int dd_grad_hess(int kind, const double* v, double* g, double* H) {
    switch (kind) {
    case 1: g_PE(v, g); H_PE(v, H); return 9;
    case 2: g_PT(v, g); H_PT(v, H); return 12;
    case 3: g_EE(v, g); H_EE(v, H); return 12;
    case 4: g_EECross(v, g); H_EECross(v, H); return 12;
    default: return 0;
    }
}

// the Hessian assembled row by row (distance_rows.cuh), kinds as above (1-3)
extern "C" int dd_hess_rows(int kind, const double* v, double* H) {
    const int n = kind == 1 ? 9 : 12;
    for (int r = 0; r < n; ++r) {
        switch (kind) {
        case 1: Hrow_PE(v, r, H + n * r); break;
        case 2: Hrow_PT(v, r, H + n * r); break;
        case 3: Hrow_EE(v, r, H + n * r); break;
        default: return 0;
        }
    }
    return n;
}

// F, U, V row-major 3x3
extern "C" void svd3_host(const double* F9, double* U9, double* s3, double* V9) {
    double F[3][3], U[3][3], V[3][3];
    for (int i = 0; i < 9; ++i) F[i / 3][i % 3] = F9[i];
    svd3<double>(F, U, s3, V);
    for (int i = 0; i < 9; ++i) { U9[i] = U[i / 3][i % 3]; V9[i] = V[i / 3][i % 3]; }
}
