// Dense layer of the preconditioner network on the 5th-generation tensor
// cores: for every item (edge or vertex) y = bf16(x) W^T + b, x the item's
// IN gathered FP32 inputs rounded to BF16 (round to nearest even), W the
// layer's OUT x IN BF16 weights, FP32 accumulation.
//
// One CTA of 128 threads per tile of 128 items: each thread gathers one
// item's inputs and stores them as BF16 in shared memory in the canonical
// K-major, no-swizzle operand layout (8-row x 16-byte core matrices), one
// thread issues the IN/16 tcgen05.mma (M=128, N=OUT, K=16, kind::f16) into an
// FP32 accumulator in tensor memory, the commit arrives on an mbarrier, and
// each warp reads its 32 accumulator lanes back with tcgen05.ld (thread t
// gets item t's OUT outputs).  Waits are bounded: on timeout the kernel sets
// timeoutBit in *status, frees its tensor memory and returns.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace cipc {
namespace tc {

constexpr int M = 128;            // items per tile (MMA M, accumulator lanes)
constexpr int THREADS = 128;
constexpr long long SPIN_MAX = 1ll << 24;

// byte offset of element (row, k) in a K-major no-swizzle operand of `rows`
// rows: core matrix (k/8, row/8) is 128 contiguous bytes, row r of it at 16 r
__host__ __device__ constexpr uint32_t coreOffset(int row, int k, int rows) {
    return (uint32_t)(((k >> 3) * (rows >> 3) + (row >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: start, leading-dimension byte offset
// (between the two 8-element K halves of one MMA), stride byte offset
// (between 8-row groups), descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t smemDesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) |
           (1ull << 46);
}

// instruction descriptor of kind::f16: D FP32, A and B BF16, both K-major
__host__ __device__ constexpr uint32_t instrDesc(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ uint32_t smemAddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mbarInit(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbarTryWait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smemAddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait for the phase with the given parity to complete
__device__ __forceinline__ bool mbarWait(uint64_t* bar, unsigned parity) {
    for (long long i = 0; i < SPIN_MAX; ++i)
        if (mbarTryWait(bar, parity)) return true;
    return false;
}

// warp-wide (all 32 lanes): allocate `cols` tensor-memory columns, address into *dst
__device__ __forceinline__ void tmemAlloc(uint32_t* dst, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddr(dst)), "r"(cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmemFree(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// D (tensor memory) = A B^T (+ D when accumulate)
__device__ __forceinline__ void mmaBf16(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(dTmem),
        "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate ? 1u : 0u)
        : "memory");
}
// the completion of every MMA this thread issued arrives once on bar
__device__ __forceinline__ void mmaCommit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smemAddr(bar)) : "memory");
}

// 32 consecutive 32-bit columns of this warp's 32 lanes (one lane per thread)
__device__ __forceinline__ void tmemLoad32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, "
        "%20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]),
          "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
          "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t packBf16(float a, float b) {
    const __nv_bfloat162 p = __floats2bfloat162_rn(a, b);  // a in the low half
    return *reinterpret_cast<const uint32_t*>(&p);
}

// Layers of IN = 64 inputs made of two 32-wide halves.  G::Idx holds what
// locates an item's inputs (G::index(item)); G::pair(idx, lane) gives inputs
// lane and 32 + lane, so that a warp gathers one item with coalesced 128-byte
// loads; G::shfl(idx, src) broadcasts lane src's Idx.  E::emit32(item, const
// float v[32]) stores one item's OUT = 32 pre-activation outputs.  Shared
// memory: 128 x 64 + 32 x 64 BF16 operands.
template <class G, class E>
__global__ void __launch_bounds__(THREADS) denseTcKernel(int n, G gather, E emit, const __nv_bfloat16* W, const __nv_bfloat16* bias, int* status,
                                                         int timeoutBit) {
    constexpr int IN = 64, OUT = 32;
    __shared__ __align__(1024) unsigned char sA[M * IN * 2];
    __shared__ __align__(1024) unsigned char sB[OUT * IN * 2];
    __shared__ float sBias[OUT];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmemBase;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // weights: W is OUT x IN row-major, i.e. B = W in N x K, K-major; each
    // thread moves two 8-element K chunks (16 bytes each)
    for (int c = tid; c < OUT * IN / 8; c += THREADS) {
        const int o = c / (IN / 8), k0 = (c % (IN / 8)) * 8;
        *reinterpret_cast<uint4*>(sB + coreOffset(o, k0, OUT)) = *reinterpret_cast<const uint4*>(W + (size_t)o * IN + k0);
    }
    for (int t = tid; t < OUT; t += THREADS) sBias[t] = __bfloat162float(bias[t]);
    if (tid == 0) {
        mbarInit(&mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");  // visible to the tensor core's arrive
    }
    if (warp == 0) tmemAlloc(&tmemBase, OUT);
    fenceProxyAsync();
    fenceBeforeSync();
    __syncthreads();
    fenceAfterSync();
    const uint32_t dTmem = tmemBase;
    constexpr uint32_t idesc = instrDesc(M, OUT);
    constexpr uint32_t lboA = (M / 8) * 128, lboB = (OUT / 8) * 128, sbo = 128;
    unsigned phase = 0;
    for (int base = blockIdx.x * M; base < n; base += gridDim.x * M) {
        // warp w gathers the 32 items of its accumulator lanes: each lane
        // reads one item's index (coalesced), then the warp walks the items,
        // inputs lane and 32 + lane from each lane (zeros past the end)
        const int mine = base + warp * 32 + lane;
        const typename G::Idx myIdx = gather.index(mine < n ? mine : n - 1);
#pragma unroll 8
        for (int j = 0; j < 32; ++j) {
            const int row = warp * 32 + j, item = base + row;
            const typename G::Idx idx = G::shfl(myIdx, j);
            const float2 v = item < n ? gather.pair(idx, lane) : make_float2(0.f, 0.f);
            *reinterpret_cast<__nv_bfloat16*>(sA + coreOffset(row, lane, M)) = __float2bfloat16_rn(v.x);
            *reinterpret_cast<__nv_bfloat16*>(sA + coreOffset(row, 32 + lane, M)) = __float2bfloat16_rn(v.y);
        }
        fenceProxyAsync();
        fenceBeforeSync();
        __syncthreads();
        fenceAfterSync();
        if (tid == 0) {
#pragma unroll
            for (int s = 0; s < IN / 16; ++s) {
                const uint64_t a = smemDesc(smemAddr(sA) + s * 2 * lboA, lboA, sbo);
                const uint64_t b = smemDesc(smemAddr(sB) + s * 2 * lboB, lboB, sbo);
                mmaBf16(dTmem, a, b, idesc, s > 0);
            }
            mmaCommit(&mbar);
        }
        const bool done = mbarWait(&mbar, phase);
        // one decision for the whole CTA, so that no thread is left at a barrier
        if (!__syncthreads_and(done)) {
            // the committed MMAs may still read sA/sB and write the
            // accumulator: a second bounded wait lets a late completion drain
            // before the tensor memory is freed below.  The host treats the
            // status bit as fatal for the context either way.
            if (tid == 0) {
                atomicOr(status, timeoutBit);
                mbarWait(&mbar, phase);
            }
            break;
        }
        phase ^= 1u;
        fenceAfterSync();
        float acc[32];
        tmemLoad32(dTmem + ((uint32_t)(warp * 32) << 16), acc);
        const int item = base + tid;  // accumulator lane tid holds item base + tid
        if (item < n) {
#pragma unroll
            for (int o = 0; o < 32; ++o) acc[o] += sBias[o];
            emit.emit32(item, acc);
        }
        // every thread's tensor-memory reads and shared-memory uses are done
        // before the next tile's MMAs overwrite them
        fenceBeforeSync();
        __syncthreads();
        fenceAfterSync();
    }
    fenceBeforeSync();
    __syncthreads();
    fenceAfterSync();
    if (warp == 0) tmemFree(dTmem, OUT);
}

// Weight gradient of a 64 -> 32 layer on the tensor cores:
//   dW^T (64 x 32) = sum over items of x_item^T d_item, db = sum of d_item,
// x the item's 64 BF16-exact inputs ([X1 | X2], 32 + 32 FP32 values already
// rounded to BF16 by the forward's rule), d its 32 FP32 output gradients.
// One tile of 128 items is one K = 128 slab of the contraction: the operand
// A (M = 128 x K, K-major) holds x^T in rows 0-63, ones in row 64 (the bias
// gradient comes out as row 64 of the product) and zeros below; B (N = 32 x
// K) holds d^T split into two BF16 terms, hi = bf16(d) and lo = bf16(d - hi),
// so that the two MMAs per K step carry d to about 16 bits and every product
// is exact in the FP32 accumulator.  Each CTA accumulates its tiles in
// tensor memory and writes one partial (OUT * 64 weights then OUT biases, the
// layout of the CUDA-core kernel's partials); items with mask 0 contribute
// nothing.  Dynamic shared memory: WG_SMEM bytes.  Waits are bounded as in
// denseTcKernel.
constexpr int WG_K = 128;  // items per tile
constexpr int WG_SMEM = M * WG_K * 2 + 2 * 32 * WG_K * 2;

__global__ void __launch_bounds__(THREADS) weightGradTcKernel(int items, const float* D, const float* X1, const float* X2, const unsigned char* mask,
                                                              float* partial, int* status, int timeoutBit) {
    constexpr int IN = 64, OUT = 32, NW = OUT * IN + OUT;
    extern __shared__ __align__(1024) unsigned char wgSmem[];
    unsigned char* sA = wgSmem;                  // M x WG_K
    unsigned char* sBh = wgSmem + M * WG_K * 2;  // OUT x WG_K
    unsigned char* sBl = sBh + OUT * WG_K * 2;
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmemBase;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // rows 65-127 of A stay zero
    for (int r = 65 + warp; r < M; r += THREADS / 32)
        for (int k = lane; k < WG_K; k += 32) *reinterpret_cast<__nv_bfloat16*>(sA + coreOffset(r, k, M)) = __float2bfloat16_rn(0.f);
    if (tid == 0) {
        mbarInit(&mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tmemAlloc(&tmemBase, OUT);
    fenceProxyAsync();
    fenceBeforeSync();
    __syncthreads();
    fenceAfterSync();
    const uint32_t dTmem = tmemBase;
    constexpr uint32_t idesc = instrDesc(M, OUT);
    constexpr uint32_t lboA = (M / 8) * 128, lboB = (OUT / 8) * 128, sbo = 128;
    unsigned phase = 0;
    bool any = false, ok = true;
    for (int base = blockIdx.x * WG_K; base < items; base += gridDim.x * WG_K) {
        // thread t stores item base + t as column t of A and of the two B terms
        const int it = base + tid;
        const bool on = it < items && (!mask || mask[it]);
        const float4* x1 = reinterpret_cast<const float4*>(X1 + (size_t)(on ? it : 0) * 32);
        const float4* x2 = reinterpret_cast<const float4*>(X2 + (size_t)(on ? it : 0) * 32);
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const float4 v = on ? (q < 8 ? x1[q] : x2[q - 8]) : make_float4(0.f, 0.f, 0.f, 0.f);
            const float e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int u = 0; u < 4; ++u) *reinterpret_cast<__nv_bfloat16*>(sA + coreOffset(4 * q + u, tid, M)) = __float2bfloat16_rn(e[u]);
        }
        *reinterpret_cast<__nv_bfloat16*>(sA + coreOffset(64, tid, M)) = __float2bfloat16_rn(on ? 1.f : 0.f);
        const float4* dv = reinterpret_cast<const float4*>(D + (size_t)(on ? it : 0) * OUT);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float4 v = on ? dv[q] : make_float4(0.f, 0.f, 0.f, 0.f);
            const float e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const __nv_bfloat16 hi = __float2bfloat16_rn(e[u]);
                const __nv_bfloat16 lo = __float2bfloat16_rn(e[u] - __bfloat162float(hi));
                *reinterpret_cast<__nv_bfloat16*>(sBh + coreOffset(4 * q + u, tid, OUT)) = hi;
                *reinterpret_cast<__nv_bfloat16*>(sBl + coreOffset(4 * q + u, tid, OUT)) = lo;
            }
        }
        fenceProxyAsync();
        fenceBeforeSync();
        __syncthreads();
        fenceAfterSync();
        if (tid == 0) {
#pragma unroll
            for (int s = 0; s < WG_K / 16; ++s) {
                const uint64_t a = smemDesc(smemAddr(sA) + s * 2 * lboA, lboA, sbo);
                mmaBf16(dTmem, a, smemDesc(smemAddr(sBh) + s * 2 * lboB, lboB, sbo), idesc, any || s > 0);
                mmaBf16(dTmem, a, smemDesc(smemAddr(sBl) + s * 2 * lboB, lboB, sbo), idesc, true);
            }
            mmaCommit(&mbar);
        }
        any = true;
        const bool done = mbarWait(&mbar, phase);
        if (!__syncthreads_and(done)) {
            // as in denseTcKernel: a second bounded wait before the tensor
            // memory is freed; the host treats the bit as fatal
            if (tid == 0) {
                atomicOr(status, timeoutBit);
                mbarWait(&mbar, phase);
            }
            ok = false;
            break;
        }
        phase ^= 1u;
        fenceAfterSync();
    }
    if (ok) {
        // accumulator lane m = row m of the product: weights for m < 64, biases at m = 64
        float acc[32];
        if (any) {
            tmemLoad32(dTmem + ((uint32_t)(warp * 32) << 16), acc);
        } else {
#pragma unroll
            for (int o = 0; o < 32; ++o) acc[o] = 0.f;
        }
        float* P = partial + (size_t)blockIdx.x * NW;
        if (tid < IN) {
#pragma unroll
            for (int o = 0; o < OUT; ++o) P[o * IN + tid] = acc[o];
        } else if (tid == IN) {
#pragma unroll
            for (int o = 0; o < OUT; ++o) P[OUT * IN + o] = acc[o];
        }
    }
    fenceBeforeSync();
    __syncthreads();
    fenceAfterSync();
    if (warp == 0) tmemFree(dTmem, OUT);
}

}  // namespace tc
}  // namespace cipc
