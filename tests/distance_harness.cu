// Host build of the generated contact-distance derivatives
// (cpu-ipc_b200/csrc/distance_derivs.cuh, the code the barrier kernels run)
// for tests/test_distance_derivs.py.  Only host functions are called.
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
