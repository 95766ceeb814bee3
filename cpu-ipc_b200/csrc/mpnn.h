// Learned preconditioner: parameter layout and host entry points (mpnn.cu).
#pragma once

#include "cipc_internal.h"

namespace cipc {

constexpr int MPNN_H = 32;   // width
constexpr int MPNN_L = 3;    // message-passing layers
constexpr int MPNN_NF = 6;   // node features
constexpr int MPNN_EF = 9;   // edge features (the scaled 3x3 block)

// Parameter offsets (FP32 master and BF16 copy share the layout); weight
// matrices are row-major [out][in].
constexpr int MP_WN0 = 0;
constexpr int MP_BN0 = MP_WN0 + MPNN_H * MPNN_NF;
constexpr int MP_WE0 = MP_BN0 + MPNN_H;
constexpr int MP_BE0 = MP_WE0 + MPNN_H * MPNN_EF;
constexpr int MP_LAYERS = MP_BE0 + MPNN_H;
constexpr int MP_LAYER = 2 * (MPNN_H * 2 * MPNN_H + MPNN_H);
__host__ __device__ constexpr int mpWe(int l) { return MP_LAYERS + l * MP_LAYER; }
__host__ __device__ constexpr int mpBe(int l) { return mpWe(l) + MPNN_H * 2 * MPNN_H; }
__host__ __device__ constexpr int mpWh(int l) { return mpBe(l) + MPNN_H; }
__host__ __device__ constexpr int mpBh(int l) { return mpWh(l) + MPNN_H * 2 * MPNN_H; }
constexpr int MP_WD = MP_LAYERS + MPNN_L * MP_LAYER;  // diagonal head [6][H]
constexpr int MP_BD = MP_WD + 6 * MPNN_H;
constexpr int MP_WO = MP_BD + 6;                      // off-diagonal head [9][H + 9]
constexpr int MP_BO = MP_WO + 9 * (MPNN_H + MPNN_EF);
constexpr int MP_NPARAM = MP_BO + 9;

void mpnnInitWeights(Ctx& c, unsigned long long seed);
void mpnnSetWeights(Ctx& c, const float* w, int n);
void mpnnGetWeights(Ctx& c, float* w);
// Scaling, mirror slots and (with features) the network inputs of the
// current assembled system.
void mpnnPrepare(Ctx& c, bool features = true);
// Network forward: factor G into c.mpGS / c.mpGD (activations kept).
void mpnnForward(Ctx& c);
// Kaporin loss on the current factor; with backward, the weight gradient
// into c.mpG.  probes: host array (nprobes x 3 nv) or null for the device
// generator seeded by seed.
double mpnnLoss(Ctx& c, int nprobes, const float* probes, unsigned long long seed, bool backward);
void mpnnAdam(Ctx& c, double lr);
void mpnnGetGrad(Ctx& c, float* g);

}  // namespace cipc
