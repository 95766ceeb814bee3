// GPU harness for the PSD projections of the contact kernels
// (cpu-ipc_b200/csrc/cipc_device.cuh): the half-warp one-sided Jacobi sweep
// in registers (halfWarpPsdProject12, two matrices per warp) and the warp
// shared-memory two-sided sweep (warpPsdProject), each applied to n row-major 12 x 12 matrices.
#include "cipc_device.cuh"

namespace {

constexpr int WPB = 4;

__global__ void halfKernel(int n, const double* in, double* out, int* capHits) {
    __shared__ double sA[2 * WPB][144], sV[2 * WPB][144], sL[2 * WPB][12];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, half = lane >> 4, hl = lane & 15;
    const int slot = 2 * w + half;
    for (int i0 = 2 * (blockIdx.x * WPB + w); i0 < n; i0 += 2 * gridDim.x * WPB) {
        const int i = i0 + half;
        const bool act = i < n;
        if (act)
            for (int e = hl; e < 144; e += 16) sA[slot][e] = in[144 * (size_t)i + e];
        __syncwarp();
        const bool ok = halfWarpPsdProject12(sA[slot], sV[slot], sL[slot], hl, act);
        if (act && hl == 0 && !ok) atomicAdd(capHits, 1);
        if (act)
            for (int e = hl; e < 144; e += 16) out[144 * (size_t)i + e] = sA[slot][e];
        __syncwarp();
    }
}

__global__ void warpKernel(int n, const double* in, double* out, int* capHits) {
    __shared__ JacobiSmem sm[WPB];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    JacobiSmem& S = sm[w];
    for (int i = blockIdx.x * WPB + w; i < n; i += gridDim.x * WPB) {
        for (int e = lane; e < 144; e += 32) S.A[e] = in[144 * (size_t)i + e];
        __syncwarp();
        const bool ok = warpPsdProject(S, 12, lane);
        if (lane == 0 && !ok) atomicAdd(capHits, 1);
        for (int e = lane; e < 144; e += 32) out[144 * (size_t)i + e] = S.A[e];
        __syncwarp();
    }
}

}  // namespace

// which = 0: half-warp register sweep, 1: warp shared-memory sweep.  Returns
// the number of matrices that hit the sweep cap, or -1 on a CUDA error.
extern "C" int psd12_project(int which, int n, const double* hIn, double* hOut) {
    double *dIn = nullptr, *dOut = nullptr;
    int* dCap = nullptr;
    const size_t bytes = sizeof(double) * 144 * (size_t)n;
    if (cudaMalloc(&dIn, bytes) != cudaSuccess || cudaMalloc(&dOut, bytes) != cudaSuccess || cudaMalloc(&dCap, sizeof(int)) != cudaSuccess)
        return -1;
    cudaMemcpy(dIn, hIn, bytes, cudaMemcpyHostToDevice);
    cudaMemset(dCap, 0, sizeof(int));
    const int blocks = which == 0 ? (n + 2 * WPB - 1) / (2 * WPB) : (n + WPB - 1) / WPB;
    if (which == 0) halfKernel<<<blocks > 0 ? blocks : 1, 32 * WPB>>>(n, dIn, dOut, dCap);
    else warpKernel<<<blocks > 0 ? blocks : 1, 32 * WPB>>>(n, dIn, dOut, dCap);
    int cap = 0;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(hOut, dOut, bytes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&cap, dCap, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(dIn);
    cudaFree(dOut);
    cudaFree(dCap);
    return e == cudaSuccess ? cap : -1;
}
