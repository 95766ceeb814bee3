// Deterministic device reductions (the partition depends only on n, so the
// summation order is reproducible) and the status-word check.
#include "cipc_device.cuh"
#include "cipc_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdio>

namespace cipc {

namespace {
constexpr int RB = 256;

template <int OP>
__device__ __forceinline__ double combine(double a, double b) {
    if (OP == 0) return a + b;
    // max and min carry a NaN forward whatever the order of the operands
    if (OP == 1) return (a > b || a != a) ? a : b;
    if (OP == 2) return (a < b || a != a) ? a : b;
    return a + b;
}
template <int OP>
__device__ __forceinline__ double ident() { return OP == 2 ? 1e308 : (OP == 1 ? -1e308 : 0.0); }

// OP: 0 sum, 1 max, 2 min, 3 dot(a,b), 4 max |a|
template <int OP>
__global__ void partialKernel(const double* a, const double* b, int n, int chunk, double* part) {
    const int OPC = (OP == 3 ? 0 : (OP == 4 ? 1 : OP));
    double acc = ident<OPC>();
    int beg = blockIdx.x * chunk, end = min(n, beg + chunk);
    for (int i = beg + threadIdx.x; i < end; i += blockDim.x) {
        double v = OP == 3 ? a[i] * b[i] : (OP == 4 ? fabs(a[i]) : a[i]);
        acc = combine<OPC>(acc, v);
    }
    __shared__ double sh[RB];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = RB / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = combine<OPC>(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

template <int OPC>
__global__ void finalKernel(const double* part, int np, double* out) {
    __shared__ double sh[RB];
    double acc = ident<OPC>();
    for (int i = threadIdx.x; i < np; i += RB) acc = combine<OPC>(acc, part[i]);
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = RB / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = combine<OPC>(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sh[0];
}

template <int OP>
double reduce(Ctx& c, const double* a, const double* b, int n) {
    const int OPC = (OP == 3 ? 0 : (OP == 4 ? 1 : OP));
    if (n <= 0) return OPC == 2 ? 1e308 : (OPC == 1 ? -1e308 : 0.0);
    int nb = std::min(1024, (n + 4 * RB - 1) / (4 * RB));
    int chunk = (n + nb - 1) / nb;
    c.scratch.reserve(nb + 8);
    launch(partialKernel<OP>, nb, RB, 0, c.s, a, b, n, chunk, c.scratch.p + 8);
    launch(finalKernel<OPC>, 1, RB, 0, c.s, c.scratch.p + 8, nb, c.scratch.p);
    double h;
    CIPC_CUDA(cudaMemcpyAsync(&h, c.scratch.p, sizeof(double), cudaMemcpyDeviceToHost, c.s));
    hostSync(c);
    return h;
}
}  // namespace

double deviceSum(Ctx& c, const double* v, int n) { return reduce<0>(c, v, nullptr, n); }

// The same two-pass sum as deviceSum, left on the device in slot `slot` of
// c.sums (no host synchronisation); fetchSums reads the slots back at once.
void deviceSumTo(Ctx& c, const double* v, int n, int slot) {
    c.sums.reserve(SUM_SLOTS);
    if (n <= 0) {
        CIPC_CUDA(cudaMemsetAsync(c.sums.p + slot, 0, sizeof(double), c.s));
        return;
    }
    int nb = std::min(1024, (n + 4 * RB - 1) / (4 * RB));
    int chunk = (n + nb - 1) / nb;
    c.scratch.reserve(nb + 8);
    launch(partialKernel<0>, nb, RB, 0, c.s, v, (const double*)nullptr, n, chunk, c.scratch.p + 8);
    launch(finalKernel<0>, 1, RB, 0, c.s, (const double*)(c.scratch.p + 8), nb, c.sums.p + slot);
}
// Minimum / maximum of v[0..n) into the device scalar *dst without a host
// synchronisation (the identity, +-1e308, for n <= 0).
void deviceMinTo(Ctx& c, const double* v, int n, double* dst) {
    int nb = n > 0 ? std::min(1024, (n + 4 * RB - 1) / (4 * RB)) : 0;
    int chunk = n > 0 ? (n + nb - 1) / nb : 0;
    c.scratch.reserve(nb + 8);
    if (nb) launch(partialKernel<2>, nb, RB, 0, c.s, v, (const double*)nullptr, n, chunk, c.scratch.p + 8);
    launch(finalKernel<2>, 1, RB, 0, c.s, (const double*)(c.scratch.p + 8), nb, dst);
}
void deviceMaxTo(Ctx& c, const double* v, int n, double* dst) {
    int nb = n > 0 ? std::min(1024, (n + 4 * RB - 1) / (4 * RB)) : 0;
    int chunk = n > 0 ? (n + nb - 1) / nb : 0;
    c.scratch.reserve(nb + 8);
    if (nb) launch(partialKernel<1>, nb, RB, 0, c.s, v, (const double*)nullptr, n, chunk, c.scratch.p + 8);
    launch(finalKernel<1>, 1, RB, 0, c.s, (const double*)(c.scratch.p + 8), nb, dst);
}

void fetchSums(Ctx& c, double* h, int nslots) {
    CIPC_CUDA(cudaMemcpyAsync(h, c.sums.p, sizeof(double) * nslots, cudaMemcpyDeviceToHost, c.s));
    hostSync(c);
}
double deviceMax(Ctx& c, const double* v, int n) { return reduce<1>(c, v, nullptr, n); }
double deviceMin(Ctx& c, const double* v, int n, double init) { return std::min(init, reduce<2>(c, v, nullptr, n)); }
double deviceDot(Ctx& c, const double* a, const double* b, int n) { return reduce<3>(c, a, b, n); }
double deviceInfNorm(Ctx& c, const double* v, int n) {
    const double m = reduce<4>(c, v, nullptr, n);
    if (!std::isfinite(m)) throw std::runtime_error("non-finite entry in a search direction or vector norm");
    return std::max(0.0, m);
}

bool debugAlloc() {
    static int v = -1;
    if (v < 0) { const char* e = std::getenv("CIPC_DEBUG_ALLOC"); v = (e && *e == '1') ? 1 : 0; }
    return v == 1;
}
void reportAlloc(size_t oldBytes, size_t newBytes, double ms) {
    std::fprintf(stderr, "[alloc] %zu -> %zu bytes in %.3f ms\n", oldBytes, newBytes, ms);
}

void checkStatus(Ctx& c, const char* stage) {
    int st = 0;
    CIPC_CUDA(cudaMemcpyAsync(&st, c.status.p, sizeof(int), cudaMemcpyDeviceToHost, c.s));
    hostSync(c);
    if (st) {
        CIPC_CUDA(cudaMemsetAsync(c.status.p, 0, sizeof(int), c.s));
        std::string msg = std::string("device status in ") + stage + ":";
        if (st & CIPC_ST_NONFINITE) msg += " non-finite value;";
        if (st & CIPC_ST_STACK_OVERFLOW) msg += " BVH traversal stack overflow;";
        if (st & CIPC_ST_CAPACITY) msg += " candidate buffer capacity exceeded;";
        if (st & CIPC_ST_CCD_CAP) msg += " CCD iteration cap;";
        if (st & CIPC_ST_JACOBI_CAP) msg += " eigen-solver sweep cap;";
        if (st & CIPC_ST_TC_TIMEOUT) {
            // a late tensor-core operation may have written freed tensor
            // memory: no further network pass runs on this context
            c.tcFault = true;
            msg += " tensor-core completion wait timed out (the learned preconditioner is disabled for this context);";
        }
        throw std::runtime_error(msg);
    }
}

}  // namespace cipc
