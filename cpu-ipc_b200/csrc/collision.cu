// Broad phase and step bounds on the GPU.
//
// * LBVH build: primitive boxes -> scene box -> 30-bit Morton keys with the
//   primitive id in the low word -> radix sort -> Karras internal nodes ->
//   bottom-up boxes (first-arrival flags).  Topology follows
//   CPULinearBVH::build, CPU IPC/LBVH.cpp:163-250.
// * Active sets: one thread per query traverses the tree with the inclusive
//   overlaps(gap) test (LBVH.cpp:157-161), applies the collider / incidence
//   filters of SpatialHash::calculateActivateSet
//   (CPU IPC/CollisionBroadPhase.cpp:765-1059), classifies and emits 64-bit
//   pair keys.  Keys are radix-sorted, so every list comes out in the
//   reference's order (query ascending, then primitive ascending); PP/PE
//   duplicates are merged by sort + run-length encoding, the job of the
//   reference's std::map.
// * Partial CCD, full (swept) CCD, ground bound, CFL bound and the
//   edge-triangle intersection test (IPCSolver.cpp:476-542, 943-990;
//   ContactMechanics.cpp:3704-3867; FeasibleStep.cpp:8-40).
#include "../../include/cipc_gpu.h"
#include "cipc_internal.h"
#include "geometry.cuh"

#include <cooperative_groups.h>
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <cstdlib>

namespace cipc {

namespace cg = cooperative_groups;

namespace {

constexpr int TB = 128;
inline int blocksFor(int n, int tb = TB) { return std::max(1, std::min((n + tb - 1) / tb, 148 * 32)); }

__device__ __forceinline__ void boxInit(double lo[3], double hi[3]) {
    for (int k = 0; k < 3; ++k) { lo[k] = 1.7976931348623157e308; hi[k] = -1.7976931348623157e308; }
}
__device__ __forceinline__ void boxAdd(double lo[3], double hi[3], d3 p) {
    lo[0] = fmin(lo[0], p.x); lo[1] = fmin(lo[1], p.y); lo[2] = fmin(lo[2], p.z);
    hi[0] = fmax(hi[0], p.x); hi[1] = fmax(hi[1], p.y); hi[2] = fmax(hi[2], p.z);
}
// (query lo, hi).overlaps(node lo, hi, gap), inclusive.
__device__ __forceinline__ bool overlaps(const double* qlo, const double* qhi, const double* nlo, const double* nhi, double gap) {
    return !((nlo[0] - qhi[0] > gap) || (nlo[1] - qhi[1] > gap) || (nlo[2] - qhi[2] > gap) || (qlo[0] - nhi[0] > gap) ||
             (qlo[1] - nhi[1] > gap) || (qlo[2] - nhi[2] > gap));
}

// Swept point box: combine(p) then combine(p - step * d).
__device__ __forceinline__ void sweptAdd(double lo[3], double hi[3], d3 p, d3 d, double step) {
    boxAdd(lo, hi, p);
    boxAdd(lo, hi, p - step * d);
}

__global__ void faceBoxKernel(int n, const int* faces, const double* x, const double* d, double stepVal, const double* stepPtr, int swept,
                              double* lo, double* hi) {
    const double step = stepPtr ? *stepPtr : stepVal;
    CIPC_KERNEL_LOOP(f, n) {
        double l[3], h[3];
        boxInit(l, h);
        for (int k = 0; k < 3; ++k) {
            int v = faces[3 * f + k];
            if (swept) sweptAdd(l, h, ld3(x, v), ld3(d, v), step);
            else boxAdd(l, h, ld3(x, v));
        }
        for (int k = 0; k < 3; ++k) { lo[3 * f + k] = l[k]; hi[3 * f + k] = h[k]; }
    }
}
__global__ void edgeBoxKernel(int n, const int* edges, const double* x, const double* d, double stepVal, const double* stepPtr, int swept,
                              double* lo, double* hi) {
    const double step = stepPtr ? *stepPtr : stepVal;
    CIPC_KERNEL_LOOP(e, n) {
        double l[3], h[3];
        boxInit(l, h);
        for (int k = 0; k < 2; ++k) {
            int v = edges[2 * e + k];
            if (swept) sweptAdd(l, h, ld3(x, v), ld3(d, v), step);
            else boxAdd(l, h, ld3(x, v));
        }
        for (int k = 0; k < 3; ++k) { lo[3 * e + k] = l[k]; hi[3 * e + k] = h[k]; }
    }
}

// Scene box in two passes: each block reduces a strided share of the
// primitive boxes into 6 partials, one block reduces the partials (min and
// max do not depend on the order).  n lo/hi triples, stride 3.
__global__ void sceneBoxKernel(int n, const double* lo, const double* hi, double* out) {
    double l[3], h[3];
    boxInit(l, h);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += blockDim.x * gridDim.x)
        for (int k = 0; k < 3; ++k) { l[k] = fmin(l[k], lo[3 * i + k]); h[k] = fmax(h[k], hi[3 * i + k]); }
    for (int k = 0; k < 3; ++k) {
        l[k] = blockReduce(l[k], MinOp(), 1.7976931348623157e308);
        __syncthreads();
        h[k] = blockReduce(h[k], MaxOp(), -1.7976931348623157e308);
        __syncthreads();
        if (threadIdx.x == 0) { out[6 * blockIdx.x + k] = l[k]; out[6 * blockIdx.x + 3 + k] = h[k]; }
    }
}
// partials (6 per block, lo then hi) of nb blocks -> box
__global__ void sceneBoxFinalKernel(int nb, const double* part, double* out) {
    double l[3], h[3];
    boxInit(l, h);
    for (int i = threadIdx.x; i < nb; i += blockDim.x)
        for (int k = 0; k < 3; ++k) { l[k] = fmin(l[k], part[6 * i + k]); h[k] = fmax(h[k], part[6 * i + 3 + k]); }
    for (int k = 0; k < 3; ++k) {
        l[k] = blockReduce(l[k], MinOp(), 1.7976931348623157e308);
        __syncthreads();
        h[k] = blockReduce(h[k], MaxOp(), -1.7976931348623157e308);
        __syncthreads();
        if (threadIdx.x == 0) { out[k] = l[k]; out[3 + k] = h[k]; }
    }
}

__device__ __forceinline__ uint32_t expandBits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
__device__ __forceinline__ uint32_t quantize(double v) {
    v = fmax(0.0, fmin(v * 1024.0, 1023.0));
    return (uint32_t)v;
}

// Morton keys (30-bit code << 32 | index).  A primitive whose box spans
// more than bigExtent along an axis (the walls of a container, a fast swept
// primitive) gets bit 62 instead: the sort moves it past the others, the
// tree is built over the rest, and every query tests the few large ones
// directly - a large box would otherwise widen all its ancestors' boxes and
// draw every query down their paths.  *nbig counts them.
__global__ void mortonKernel(int n, const double* lo, const double* hi, const double* scene, double bigExtent, uint64_t* keys, int* nbig) {
    CIPC_KERNEL_LOOP(i, n) {
        bool big = false;
        for (int k = 0; k < 3; ++k) big = big || (hi[3 * i + k] - lo[3 * i + k] > bigExtent);
        if (big) {
            atomicAdd(nbig, 1);
            keys[i] = (1ull << 62) | (uint32_t)i;
            continue;
        }
        double c[3], q[3];
        for (int k = 0; k < 3; ++k) {
            c[k] = 0.5 * (lo[3 * i + k] + hi[3 * i + k]);
            double ext = scene[3 + k] - scene[k];
            double off = c[k] - scene[k];
            q[k] = ext > 0.0 ? off / ext : 0.0;
        }
        uint32_t code = (expandBits(quantize(q[0])) << 2) | (expandBits(quantize(q[1])) << 1) | expandBits(quantize(q[2]));
        keys[i] = ((uint64_t)code << 32) | (uint32_t)i;
    }
}

__device__ __forceinline__ int prefixLen(const uint64_t* k, int n, int a, int b) {
    if (b < 0 || b >= n) return -1;
    uint64_t x = k[a] ^ k[b];
    return x == 0 ? 64 : __clzll(x);
}

__global__ void karrasKernel(int nAll, const int* nbig, const uint64_t* keys, int* left, int* right, int* parent) {
    const int n = nAll - *nbig;  // leaves of the tree (the large primitives stay out)
    CIPC_KERNEL_LOOP(in, n - 1) {
        int first, last;
        if (in == 0) { first = 0; last = n - 1; }
        else {
            int lp = prefixLen(keys, n, in, in - 1), rp = prefixLen(keys, n, in, in + 1);
            int dir = rp > lp ? 1 : -1;
            int minp = min(lp, rp);
            int maxLen = 2;
            while (prefixLen(keys, n, in, in + dir * maxLen) > minp) maxLen <<= 1;
            int len = 0;
            for (int step = maxLen >> 1; step > 0; step >>= 1)
                if (prefixLen(keys, n, in, in + dir * (len + step)) > minp) len += step;
            int other = in + dir * len;
            first = min(in, other); last = max(in, other);
        }
        int split;
        uint64_t fc = keys[first], lc = keys[last];
        if (fc == lc) split = (first + last) >> 1;
        else {
            int common = __clzll(fc ^ lc);
            split = first;
            unsigned step = (unsigned)(last - first);
            do {
                step = (step + 1) >> 1;
                int cand = split + (int)step;
                if (cand < last && __clzll(fc ^ keys[cand]) > common) split = cand;
            } while (step > 1);
        }
        int l = split, r = split + 1;
        if (split == first) l += n - 1;
        if (split + 1 == last) r += n - 1;
        left[in] = l; right[in] = r;
        parent[l] = in; parent[r] = in;
    }
}

__global__ void leafKernel(int nAll, const int* nbig, const uint64_t* keys, const double* plo, const double* phi, int* leafPrim, double* lo,
                           double* hi, int* flags, int* parent) {
    const int n = nAll - *nbig;
    CIPC_KERNEL_LOOP(s, n) {
        int prim = (int)(keys[s] & 0xffffffffu);
        leafPrim[s] = prim;
        int node = s + n - 1;
        for (int k = 0; k < 3; ++k) { lo[3 * node + k] = plo[3 * prim + k]; hi[3 * node + k] = phi[3 * prim + k]; }
        if (s < n - 1) flags[s] = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) parent[0] = -1;
}

__device__ __forceinline__ int atomAddAcqRel(int* p, int v) {
    int old;
    asm volatile("atom.add.acq_rel.gpu.s32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Bottom-up box merge: the second child to arrive at a node combines both
// child boxes (left first, then right, as the reference's post-order merge).
// The arrival is an acquire-release atomic: it publishes the box this thread
// wrote for the child it came from and, for the second arrival, makes the
// sibling's box visible.  The same thread writes the node's traversal
// record: the boxes of both children rounded outward to FP32 (lo down, hi
// up) and the children's node indices, 64 bytes, so that one load tests
// both children.
__global__ void refitKernel(int nAll, const int* nbig, const int* left, const int* right, const int* parent, double* lo, double* hi, int* flags,
                            float* rec) {
    const int n = nAll - *nbig;
    if (n <= 1) return;
    CIPC_KERNEL_LOOP(s, n) {
        int node = s + n - 1;
        int p = parent[node];
        for (int guard = 0; guard < 64 && p >= 0; ++guard) {
            if (atomAddAcqRel(&flags[p], 1) == 0) break;
            const int ch[2] = {left[p], right[p]};
            double cb[2][6];
            for (int q = 0; q < 2; ++q)
                for (int k = 0; k < 3; ++k) {
                    cb[q][k] = __ldcg(&lo[3 * ch[q] + k]);
                    cb[q][3 + k] = __ldcg(&hi[3 * ch[q] + k]);
                }
            for (int k = 0; k < 3; ++k) {
                double a = fmin(1.7976931348623157e308, cb[0][k]);
                a = fmin(a, cb[1][k]);
                double b = fmax(-1.7976931348623157e308, cb[0][3 + k]);
                b = fmax(b, cb[1][3 + k]);
                lo[3 * p + k] = a; hi[3 * p + k] = b;
            }
            float r[16];
            for (int q = 0; q < 2; ++q)
                for (int k = 0; k < 3; ++k) {
                    r[6 * q + k] = __double2float_rd(cb[q][k]);
                    r[6 * q + 3 + k] = __double2float_ru(cb[q][3 + k]);
                }
            r[12] = __int_as_float(ch[0]);
            r[13] = __int_as_float(ch[1]);
            r[14] = r[15] = 0.f;
            float4* o = reinterpret_cast<float4*>(rec) + 4 * (size_t)p;
            for (int q = 0; q < 4; ++q) o[q] = make_float4(r[4 * q], r[4 * q + 1], r[4 * q + 2], r[4 * q + 3]);
            node = p;
            p = parent[node];
        }
    }
}

// Escape (rope) index of every node: the next node of a depth-first walk
// once the node's subtree is done - the right sibling of the node or of its
// nearest ancestor that is a left child; -1 past the last leaf.  One thread
// per node walks up the parent links (at most the tree's depth, which the
// 64-bit keys bound by 64).
__global__ void escapeKernel(int nAll, const int* nbig, const int* left, const int* right, const int* parent, int* escape) {
    const int n = nAll - *nbig;
    CIPC_KERNEL_LOOP(node, 2 * n - 1) {
        int cur = node, e = -1;
        for (int guard = 0; guard < 128; ++guard) {
            const int p = parent[cur];
            if (p < 0) break;
            if (left[p] == cur) { e = right[p]; break; }
            cur = p;
        }
        escape[node] = e;
    }
}

struct BvhView {
    static constexpr bool kSplitsBig = true;  // large primitives are kept out of the tree (see traverse2)
    double bigExtent;  // a box wider than this along an axis is large
    int nAll;         // primitives; the tree holds nAll - *nbig of them
    const int* nbig;  // primitives kept out of the tree (their keys sort last)
    const uint64_t* keys;
    const int *left, *right, *leafPrim, *escape;
    const double *lo, *hi;
    const double *plo, *phi;  // primitive boxes
    const float4* rec;
};
BvhView view(const DevBvh& t) {
    return BvhView{t.bigExtent, t.n, t.bigCount.p, t.keys, t.left, t.right, t.leafPrim, t.escape, t.lo, t.hi, t.primLo, t.primHi,
                   reinterpret_cast<const float4*>(t.rec.p)};
}

__device__ __forceinline__ bool isLargeBox(const double* lo, const double* hi, double ext) {
    return (hi[0] - lo[0] > ext) || (hi[1] - lo[1] > ext) || (hi[2] - lo[2] > ext);
}

// Stack-less depth-first traversal along escape indices; calls f(prim) once
// for every leaf whose box overlaps the query box with the gap (inclusive
// test, in FP64).  At an internal node one 64-byte record tests both
// children on their outward-rounded FP32 boxes, which contain the FP64
// boxes: a hit internal left child is entered directly (its sibling is
// reached later by the escape index and tested on its own FP64 box); a hit
// leaf is tested on its FP64 box and reported unless the walk entered its
// left sibling, in which case the escape index brings the walk to it.  The
// set of leaves reported is exactly that of a walk on the FP64 boxes (the
// order of the calls differs, and every caller sorts or reduces what it
// collects).  The walk visits each node at most once; a count past the node
// count raises a status bit.
template <class F>
__device__ __forceinline__ void traverseTree(const BvhView& t, int n, const double* qlo, const double* qhi, double gap, int* status, F& f) {
    if (n <= 0) return;
    if (!overlaps(qlo, qhi, t.lo, t.hi, gap)) return;  // the root (node 0)
    if (n == 1) { f(t.leafPrim[0]); return; }
    const int firstLeaf = n - 1;
    int cur = 0;  // an internal node whose box overlaps the query
    for (int visits = 0; cur >= 0; ++visits) {
        if (visits > 2 * n) { raiseStatus(status, CIPC_ST_STACK_OVERFLOW); return; }
        const float4* r = t.rec + 4 * (size_t)cur;
        const float4 a = r[0], b = r[1], cc = r[2], d = r[3];
        const double lo0[3] = {a.x, a.y, a.z}, hi0[3] = {a.w, b.x, b.y};
        const double lo1[3] = {b.z, b.w, cc.x}, hi1[3] = {cc.y, cc.z, cc.w};
        const int c0 = __float_as_int(d.x), c1 = __float_as_int(d.y);
        const bool h0 = overlaps(qlo, qhi, lo0, hi0, gap), h1 = overlaps(qlo, qhi, lo1, hi1, gap);
        if (h0 && c0 < firstLeaf) { cur = c0; continue; }
        if (h0 && overlaps(qlo, qhi, t.lo + 3 * c0, t.hi + 3 * c0, gap)) f(t.leafPrim[c0 - firstLeaf]);
        if (h1 && c1 < firstLeaf) { cur = c1; continue; }
        if (h1 && overlaps(qlo, qhi, t.lo + 3 * c1, t.hi + 3 * c1, gap)) f(t.leafPrim[c1 - firstLeaf]);
        // both children done: follow escape indices to the next node to test
        int e = t.escape[cur];
        while (e >= 0) {
            if (++visits > 2 * n) { raiseStatus(status, CIPC_ST_STACK_OVERFLOW); return; }
            const bool hit = overlaps(qlo, qhi, t.lo + 3 * e, t.hi + 3 * e, gap);
            if (e >= firstLeaf) {
                if (hit) f(t.leafPrim[e - firstLeaf]);
            } else if (hit) {
                break;
            }
            e = t.escape[e];
        }
        cur = e;
    }
}

template <class F>
__device__ __forceinline__ void traverse(const BvhView& t, const double* qlo, const double* qhi, double gap, int* status, F f) {
    if (t.nAll <= 0) return;
    const int nb = *t.nbig, n = t.nAll - nb;
    traverseTree(t, n, qlo, qhi, gap, status, f);
    for (int b = 0; b < nb; ++b) {
        const int p = (int)(t.keys[n + b] & 0xffffffffu);
        if (overlaps(qlo, qhi, t.plo + 3 * p, t.phi + 3 * p, gap)) f(p);
    }
}

// For queries over the tree's own primitive set (edges against edges): a
// large query does not walk the tree; it meets only the large primitives.
// Its pairs with the tree's primitives are reported from their side, through
// their own loop over the large primitives, which therefore sees every large
// primitive whatever the indices.  f(prim, fromLargeList).
template <class F>
__device__ __forceinline__ void traverse2(const BvhView& t, const double* qlo, const double* qhi, double gap, bool largeQuery, int* status, F f) {
    if (t.nAll <= 0) return;
    const int nb = *t.nbig, n = t.nAll - nb;
    if (!largeQuery) {
        auto g = [&](int p) { f(p, false); };
        traverseTree(t, n, qlo, qhi, gap, status, g);
    }
    for (int b = 0; b < nb; ++b) {
        const int p = (int)(t.keys[n + b] & 0xffffffffu);
        if (overlaps(qlo, qhi, t.plo + 3 * p, t.phi + 3 * p, gap)) f(p, true);
    }
}

// ---------------------------------------------------------------------------
// Spatial-hash backend (the reference's SpatialHash, CollisionBroadPhase.cpp:
// 11-763, as an A/B alternative to the LBVH): every primitive box is entered
// in the cubic cells of edge `h` (the mean surface edge length, as the
// reference's sh.build(mesh, averageEdgeLenth)) that it touches, as
// (cell key, primitive) pairs sorted by key.  A query visits the cells of its
// box grown by the gap (and one cell more on each side, against rounding),
// finds each cell's run by binary search, and reports a primitive only in the
// lowest cell it shares with the query, after the same inclusive FP64 box
// test as the LBVH walk - so both backends report the same set.  Primitives
// touching more than HASH_MAX_CELLS cells are kept in a list that every query
// tests; a query touching more than HASH_MAX_QUERY cells tests all
// primitives.
// ---------------------------------------------------------------------------
constexpr int HASH_MAX_CELLS = 64;
constexpr long long HASH_MAX_QUERY = 4096;
constexpr int HASH_BIAS = 1 << 20;  // cell coordinates are offset into [0, 2^21)

struct HashView {
    static constexpr bool kSplitsBig = false;
    double bigExtent;
    int n, pairs;
    double inv;
    const uint64_t* key;
    const int* prim;
    const int* big;
    const int* nbig;
    const double *plo, *phi;
};

__device__ __forceinline__ int hashCell(double v, double inv) {
    const double c = floor(v * inv) + (double)HASH_BIAS;
    return (int)fmin(fmax(c, 0.0), (double)(2 * HASH_BIAS - 1));
}
__device__ __forceinline__ uint64_t hashKeyOf(int ix, int iy, int iz) {
    return ((uint64_t)ix << 42) | ((uint64_t)iy << 21) | (uint64_t)iz;
}

template <class F>
__device__ __forceinline__ void traverse(const HashView& t, const double* qlo, const double* qhi, double gap, int* status, F f) {
    if (t.n <= 0) return;
    int lo[3], hi[3];
    long long cells = 1;
    for (int k = 0; k < 3; ++k) {
        lo[k] = max(hashCell(qlo[k] - gap, t.inv) - 1, 0);
        hi[k] = min(hashCell(qhi[k] + gap, t.inv) + 1, 2 * HASH_BIAS - 1);
        cells *= (long long)(hi[k] - lo[k] + 1);
    }
    if (cells > HASH_MAX_QUERY) {  // a large query box: test every primitive
        for (int p = 0; p < t.n; ++p)
            if (overlaps(qlo, qhi, t.plo + 3 * p, t.phi + 3 * p, gap)) f(p);
        return;
    }
    for (int iz = lo[2]; iz <= hi[2]; ++iz)
        for (int iy = lo[1]; iy <= hi[1]; ++iy)
            for (int ix = lo[0]; ix <= hi[0]; ++ix) {
                const uint64_t key = hashKeyOf(ix, iy, iz);
                int a = 0, b = t.pairs;  // first pair with a key >= key
                while (a < b) {
                    const int m = (a + b) >> 1;
                    if (t.key[m] < key) a = m + 1;
                    else b = m;
                }
                for (int k = a; k < t.pairs && t.key[k] == key; ++k) {
                    const int p = t.prim[k];
                    const double* pl = t.plo + 3 * p;
                    // the lowest cell the primitive shares with the query
                    if (max(hashCell(pl[0], t.inv), lo[0]) != ix || max(hashCell(pl[1], t.inv), lo[1]) != iy ||
                        max(hashCell(pl[2], t.inv), lo[2]) != iz)
                        continue;
                    if (overlaps(qlo, qhi, pl, t.phi + 3 * p, gap)) f(p);
                }
            }
    const int nb = *t.nbig;
    for (int b = 0; b < nb; ++b) {
        const int p = t.big[b];
        if (overlaps(qlo, qhi, t.plo + 3 * p, t.phi + 3 * p, gap)) f(p);
    }
}

template <class F>
__device__ __forceinline__ void traverse2(const HashView& t, const double* qlo, const double* qhi, double gap, bool, int* status, F f) {
    traverse(t, qlo, qhi, gap, status, [&](int p) { f(p, false); });
}

__global__ void hashCountKernel(int n, const double* plo, const double* phi, double inv, int* count, int* bigFlag) {
    CIPC_KERNEL_LOOP(p, n) {
        long long cells = 1;
        for (int k = 0; k < 3; ++k) cells *= (long long)(hashCell(phi[3 * p + k], inv) - hashCell(plo[3 * p + k], inv) + 1);
        const bool big = cells > HASH_MAX_CELLS;
        count[p] = big ? 0 : (int)cells;
        bigFlag[p] = big ? 1 : 0;
    }
}

__global__ void hashEmitKernel(int n, const double* plo, const double* phi, double inv, const int* offset, const int* count, uint64_t* key, int* prim) {
    CIPC_KERNEL_LOOP(p, n) {
        if (count[p] == 0) continue;
        int lo[3], hi[3];
        for (int k = 0; k < 3; ++k) { lo[k] = hashCell(plo[3 * p + k], inv); hi[k] = hashCell(phi[3 * p + k], inv); }
        int o = offset[p];
        for (int iz = lo[2]; iz <= hi[2]; ++iz)
            for (int iy = lo[1]; iy <= hi[1]; ++iy)
                for (int ix = lo[0]; ix <= hi[0]; ++ix) { key[o] = hashKeyOf(ix, iy, iz); prim[o] = p; ++o; }
    }
}

__device__ __forceinline__ bool isCollider(int t) { return t >= 2; }

// Packed PP/PE key: lexicographic order of (c0 = -v-1, c1, c2) with c3 = -1.
constexpr uint64_t M21 = (1ull << 21) - 1;
__device__ __forceinline__ uint64_t ppeKey(int c0, int c1, int c2) {
    uint64_t v = (uint64_t)(-c0 - 1);
    return ((M21 - v) << 42) | ((uint64_t)c1 << 21) | (uint64_t)(c2 + 1);
}

// Appends a key to a list: the lanes of a warp that emit at the same point
// take one atomic for all of them (the leader reserves the group's slots and
// broadcasts the base).  The list is sorted afterwards, so the order of the
// slots does not matter.
struct Emit {
    uint64_t* buf;
    int cap;
    int* counter;
    __device__ void operator()(uint64_t k, int* status) const {
        cg::coalesced_group g = cg::coalesced_threads();
        int base = 0;
        if (g.thread_rank() == 0) base = atomicAdd(counter, (int)g.size());
        const int i = g.shfl(base, 0) + (int)g.thread_rank();
        if (i < cap) buf[i] = k;
        else raiseStatus(status, CIPC_ST_CAPACITY);
    }
};

// Active sets in two kernels per kind, so that the distance classification
// runs one thread per candidate instead of inside the divergent tree walk:
// the walk emits every candidate pair (the partial-CCD set), then one thread
// per stored candidate classifies it and emits the contact keys.  The sets
// are sorted afterwards, so the order of emission does not matter.
template <class View>
__global__ void activePTKernel(int nsv, const int* surfVerts, const int* faces, const int* btype, const double* x, View tree, double sq, Emit ccd,
                               int* status) {
    CIPC_KERNEL_LOOP(svI, nsv) {
        int vI = surfVerts[svI];
        d3 p = ld3(x, vI);
        double lo[3] = {p.x, p.y, p.z};
        traverse(tree, lo, lo, sq, status, [&](int sfI) {
            int f0 = faces[3 * sfI], f1 = faces[3 * sfI + 1], f2 = faces[3 * sfI + 2];
            if (isCollider(btype[vI]) && isCollider(btype[f0]) && isCollider(btype[f1]) && isCollider(btype[f2])) return;
            if (vI == f0 || vI == f1 || vI == f2) return;
            ccd(((uint64_t)svI << 32) | (uint32_t)sfI, status);
        });
    }
}

// the point-triangle candidates (svI << 32 | sfI) stored by activePTKernel
__global__ void activePTClassKernel(const uint64_t* cand, const int* count, int cap, const int* surfVerts, const int* faces, const double* x,
                                    double Hhat, Emit ptk, Emit ppe, int* status) {
    const int n = min(*count, cap);
    CIPC_KERNEL_LOOP(k, n) {
        const uint64_t key = cand[k];
        const int svI = (int)(key >> 32), sfI = (int)(key & 0xffffffffu);
        const int vI = surfVerts[svI];
        const int f0 = faces[3 * sfI], f1 = faces[3 * sfI + 1], f2 = faces[3 * sfI + 2];
        const d3 p = ld3(x, vI), a = ld3(x, f0), b = ld3(x, f1), c = ld3(x, f2);
        double d;
        switch (dTypePT(p, a, b, c)) {
        case 0: d = dPP(p, a); if (d < Hhat) ppe(ppeKey(-vI - 1, f0, -1), status); break;
        case 1: d = dPP(p, b); if (d < Hhat) ppe(ppeKey(-vI - 1, f1, -1), status); break;
        case 2: d = dPP(p, c); if (d < Hhat) ppe(ppeKey(-vI - 1, f2, -1), status); break;
        case 3: d = dPE(p, a, b); if (d < Hhat) ppe(ppeKey(-vI - 1, f0, f1), status); break;
        case 4: d = dPE(p, b, c); if (d < Hhat) ppe(ppeKey(-vI - 1, f1, f2), status); break;
        case 5: d = dPE(p, c, a); if (d < Hhat) ppe(ppeKey(-vI - 1, f2, f0), status); break;
        default: d = dPT(p, a, b, c); if (d < Hhat) ptk(key, status); break;
        }
    }
}

template <class View>
__global__ void activeEEKernel(int ne, const int* edges, const int* btype, const double* x, View tree, double sq, Emit ccd, int* status) {
    CIPC_KERNEL_LOOP(self, ne) {
        double lo[3], hi[3];
        boxInit(lo, hi);
        boxAdd(lo, hi, ld3(x, edges[2 * self])); boxAdd(lo, hi, ld3(x, edges[2 * self + 1]));
        const bool large = View::kSplitsBig && isLargeBox(lo, hi, tree.bigExtent);
        // the pair (eI, eJ), eI < eJ, as the reference forms it
        auto pair = [&](int eI, int eJ) {
            int e0 = edges[2 * eI], e1 = edges[2 * eI + 1];
            int g0 = edges[2 * eJ], g1 = edges[2 * eJ + 1];
            if (isCollider(btype[e0]) && isCollider(btype[e1]) && isCollider(btype[g0]) && isCollider(btype[g1])) return;
            if (e0 == g0 || e0 == g1 || e1 == g0 || e1 == g1) return;
            ccd(((uint64_t)eI << 32) | (uint32_t)eJ, status);
        };
        traverse2(tree, lo, hi, sq, large, status, [&](int other, bool fromLarge) {
            // a pair is handled once: by its lower index, except that a
            // small edge handles its pairs with the large ones either way
            if (!fromLarge || large) {
                if (other > self) pair(self, other);
            } else if (other != self) {
                if (other > self) pair(self, other);
                else pair(other, self);
            }
        });
    }
}

// the edge-edge candidates (eI << 32 | eJ) stored by activeEEKernel,
// classified as the reference does with eI's points first
__global__ void activeEEClassKernel(const uint64_t* cand, const int* count, int cap, const int* edges, const double* x, const double* rest,
                                    double Hhat, Emit eek, Emit moll, Emit ppe, int* status) {
    const int n = min(*count, cap);
    CIPC_KERNEL_LOOP(k, n) {
        const uint64_t key = cand[k];
        const int eI = (int)(key >> 32), eJ = (int)(key & 0xffffffffu);
        const int e0 = edges[2 * eI], e1 = edges[2 * eI + 1];
        const int g0 = edges[2 * eJ], g1 = edges[2 * eJ + 1];
        const d3 p0 = ld3(x, e0), p1 = ld3(x, e1), q0 = ld3(x, g0), q1 = ld3(x, g1);
        const int t = dTypeEE(p0, p1, q0, q1);
        const double cs = crossSqNormEE(p0, p1, q0, q1);
        const double ex = 1e-3 * sqn(ld3(rest, e0) - ld3(rest, e1)) * sqn(ld3(rest, g0) - ld3(rest, g1));
        const bool mol = cs < ex;
        double d;
        int c0 = 0, c1 = 0, c2 = -1;
        switch (t) {
        case 0: d = dPP(p0, q0); c0 = -e0 - 1; c1 = g0; break;
        case 1: d = dPP(p0, q1); c0 = -e0 - 1; c1 = g1; break;
        case 2: d = dPE(p0, q0, q1); c0 = -e0 - 1; c1 = g0; c2 = g1; break;
        case 3: d = dPP(p1, q0); c0 = -e1 - 1; c1 = g0; break;
        case 4: d = dPP(p1, q1); c0 = -e1 - 1; c1 = g1; break;
        case 5: d = dPE(p1, q0, q1); c0 = -e1 - 1; c1 = g0; c2 = g1; break;
        case 6: d = dPE(q0, p0, p1); c0 = -g0 - 1; c1 = e0; c2 = e1; break;
        case 7: d = dPE(q1, p0, p1); c0 = -g1 - 1; c1 = e0; c2 = e1; break;
        default: d = dEE(p0, p1, q0, q1); break;
        }
        if (!(d < Hhat)) continue;
        if (mol) moll(((uint64_t)eI << 34) | ((uint64_t)eJ << 4) | (uint64_t)t, status);
        else if (t == 8) eek(key, status);
        else ppe(ppeKey(c0, c1, c2), status);
    }
}

__global__ void decodeSelfKernel(int nPT, int nEE, int nPPE, const uint64_t* kPT, const uint64_t* kEE, const uint64_t* uniq, const int* counts,
                                 const int* surfVerts, const int* faces, const int* edges, int* out) {
    int n = nPT + nEE + nPPE;
    CIPC_KERNEL_LOOP(i, n) {
        int c[4];
        if (i < nPT) {
            int svI = (int)(kPT[i] >> 32), sfI = (int)(kPT[i] & 0xffffffffu);
            c[0] = -surfVerts[svI] - 1; c[1] = faces[3 * sfI]; c[2] = faces[3 * sfI + 1]; c[3] = faces[3 * sfI + 2];
        } else if (i < nPT + nEE) {
            uint64_t k = kEE[i - nPT];
            int eI = (int)(k >> 32), eJ = (int)(k & 0xffffffffu);
            c[0] = edges[2 * eI]; c[1] = edges[2 * eI + 1]; c[2] = edges[2 * eJ]; c[3] = edges[2 * eJ + 1];
        } else {
            int j = i - nPT - nEE;
            uint64_t k = uniq[j];
            int v = (int)(M21 - (k >> 42));
            c[0] = -v - 1; c[1] = (int)((k >> 21) & M21); c[2] = (int)(k & M21) - 1; c[3] = -counts[j];
        }
        for (int q = 0; q < 4; ++q) out[4 * i + q] = c[q];
    }
}

__global__ void decodeMollKernel(int n, const uint64_t* k, const int* edges, int* selfEE, int* eeIe) {
    CIPC_KERNEL_LOOP(i, n) {
        uint64_t key = k[i];
        int eI = (int)(key >> 34), eJ = (int)((key >> 4) & ((1u << 30) - 1)), t = (int)(key & 15);
        int e0 = edges[2 * eI], e1 = edges[2 * eI + 1], g0 = edges[2 * eJ], g1 = edges[2 * eJ + 1];
        int c[4] = {0, 0, -1, -1};
        switch (t) {
        case 0: c[0] = -e0 - 1; c[1] = g0; break;
        case 1: c[0] = -e0 - 1; c[1] = g1; break;
        case 2: c[0] = -e0 - 1; c[1] = g0; c[2] = g1; break;
        case 3: c[0] = -e1 - 1; c[1] = g0; break;
        case 4: c[0] = -e1 - 1; c[1] = g1; break;
        case 5: c[0] = -e1 - 1; c[1] = g0; c[2] = g1; break;
        case 6: c[0] = -g0 - 1; c[1] = e0; c[2] = e1; break;
        case 7: c[0] = -g1 - 1; c[1] = e0; c[2] = e1; break;
        default: c[0] = e0; c[1] = e1; c[2] = g0; c[3] = g1; break;
        }
        for (int q = 0; q < 4; ++q) selfEE[4 * i + q] = c[q];
        eeIe[2 * i] = t == 8 ? -1 : eI;
        eeIe[2 * i + 1] = t == 8 ? -1 : eJ;
    }
}

__global__ void groundFlagKernel(int nsv, const int* surfVerts, const double* x, double nx, double ny, double nz, double D, double Hhat, int* flags) {
    CIPC_KERNEL_LOOP(i, nsv) {
        d3 p = ld3(x, surfVerts[i]);
        double dist = nx * p.x + ny * p.y + nz * p.z - D;
        flags[i] = dist * dist < Hhat ? 1 : 0;
    }
}

// ---- step bounds ----
__global__ void groundBoundKernel(int nsv, const int* surfVerts, const double* x, const double* dir, double nx, double ny, double nz, double D,
                                  double slack, double* out) {
    CIPC_KERNEL_LOOP(i, nsv) {
        int v = surfVerts[i];
        d3 p = ld3(x, v), d = ld3(dir, v);
        double r = 1.0;
        double nm = nx * -d.x + ny * -d.y + nz * -d.z;
        if (nm < 0.0) {
            double dist = nx * p.x + ny * p.y + nz * p.z - D;
            double cand = -dist / nm * slack;
            if (cand >= 0.0) r = cand;
        }
        out[i] = r;
    }
}

__global__ void surfMoveKernel(int nsv, const int* surfVerts, const double* dir, double* out) {
    CIPC_KERNEL_LOOP(i, nsv) out[i] = sqrt(sqn(ld3(dir, surfVerts[i])));
}

__global__ void partialCCDKernel(int nPT, int nEE, const uint64_t* ccdPT, const uint64_t* ccdEE, const int* surfVerts, const int* faces,
                                 const int* edges, const double* x, const double* dir, double eta, double* out, int* status) {
    CIPC_KERNEL_LOOP(i, nPT + nEE) {
        double a;
        if (i < nPT) {
            int svI = (int)(ccdPT[i] >> 32), sfI = (int)(ccdPT[i] & 0xffffffffu);
            int p = surfVerts[svI], f0 = faces[3 * sfI], f1 = faces[3 * sfI + 1], f2 = faces[3 * sfI + 2];
            a = pointTriangleCCD(ld3(x, p), ld3(x, f0), ld3(x, f1), ld3(x, f2), -ld3(dir, p), -ld3(dir, f0), -ld3(dir, f1), -ld3(dir, f2), eta, status);
        } else {
            uint64_t k = ccdEE[i - nPT];
            int eI = (int)(k >> 32), eJ = (int)(k & 0xffffffffu);
            int a0 = edges[2 * eI], a1 = edges[2 * eI + 1], b0 = edges[2 * eJ], b1 = edges[2 * eJ + 1];
            a = edgeEdgeCCD(ld3(x, a0), ld3(x, a1), ld3(x, b0), ld3(x, b1), -ld3(dir, a0), -ld3(dir, a1), -ld3(dir, b0), -ld3(dir, b1), eta, status);
        }
        out[i] = a;
    }
}

// Full point-triangle CCD in two kernels (as the edge-edge one below): the
// walk of each surface vertex's swept box emits (vertex, face) pairs that do
// not share a vertex and are not all colliders, then one thread per pair
// runs the additive CCD.
template <class View>
__global__ void fullPTPairsKernel(int nsv, const int* surfVerts, const int* faces, const int* btype, const double* x, const double* dir,
                                  double stepVal, const double* stepPtr, View tree, int2* pairs, int cap, int* count, int* status) {
    const double step = stepPtr ? *stepPtr : stepVal;
    CIPC_KERNEL_LOOP(svI, nsv) {
        const int vI = surfVerts[svI];
        const d3 p = ld3(x, vI), dp = ld3(dir, vI);
        double lo[3], hi[3];
        boxInit(lo, hi);
        sweptAdd(lo, hi, p, dp, step);
        traverse(tree, lo, hi, 0.0, status, [&](int sfI) {
            const int f0 = faces[3 * sfI], f1 = faces[3 * sfI + 1], f2 = faces[3 * sfI + 2];
            if (isCollider(btype[vI]) && isCollider(btype[f0]) && isCollider(btype[f1]) && isCollider(btype[f2])) return;
            if (vI == f0 || vI == f1 || vI == f2) return;
            cg::coalesced_group g = cg::coalesced_threads();
            int base = 0;
            if (g.thread_rank() == 0) base = atomicAdd(count, (int)g.size());
            const int i = g.shfl(base, 0) + (int)g.thread_rank();
            if (i < cap) pairs[i] = make_int2(vI, sfI);
        });
    }
}

__global__ void fullPTAccdKernel(const int2* pairs, const int* count, int cap, const int* faces, const double* x, const double* dir, double eta,
                                 double* outMin, int* status) {
    const int n = min(*count, cap);
    double best = 1.0;
    CIPC_KERNEL_LOOP(k, n) {
        const int2 pr = pairs[k];
        const int vI = pr.x, f0 = faces[3 * pr.y], f1 = faces[3 * pr.y + 1], f2 = faces[3 * pr.y + 2];
        best = fmin(pointTriangleCCD(ld3(x, vI), ld3(x, f0), ld3(x, f1), ld3(x, f2), -ld3(dir, vI), -ld3(dir, f0), -ld3(dir, f1), -ld3(dir, f2), eta,
                                     status),
                    best);
    }
    best = blockReduce(best, MinOp(), 1.0);
    if (threadIdx.x == 0) atomicMin(reinterpret_cast<unsigned long long*>(outMin), (unsigned long long)__double_as_longlong(best));
}

// Full edge-edge CCD in two kernels, so that the additive CCD runs one
// thread per candidate pair instead of inside the divergent tree walk.  The
// walk emits (query eJ, candidate eI > eJ) as the reference forms its pairs
// (Self_largestFeasibleStepSize_CCD): no two colliders, no shared vertex, and
// swept boxes at the entry step that overlap.  Pairs past `cap` are counted
// but not stored; the caller grows the buffer and runs again.
template <class View>
__global__ void fullEEPairsKernel(int ne, const int* edges, const int* btype, const double* x, const double* dir, const double* treeBoxLo,
                                  const double* treeBoxHi, double eeStepVal, const double* eeStepPtr, View tree, int2* pairs, int cap, int* count,
                                  int* status) {
    const double eeStep = eeStepPtr ? *eeStepPtr : eeStepVal;
    CIPC_KERNEL_LOOP(self, ne) {
        double qlo[3], qhi[3];
        for (int k = 0; k < 3; ++k) { qlo[k] = treeBoxLo[3 * self + k]; qhi[k] = treeBoxHi[3 * self + k]; }
        const bool large = View::kSplitsBig && isLargeBox(qlo, qhi, tree.bigExtent);
        auto pair = [&](int eJ, int eI) {
            int g0 = edges[2 * eJ], g1 = edges[2 * eJ + 1];
            int e0 = edges[2 * eI], e1 = edges[2 * eI + 1];
            if (isCollider(btype[e0]) && isCollider(btype[e1]) && isCollider(btype[g0]) && isCollider(btype[g1])) return;
            if (e0 == g0 || e0 == g1 || e1 == g0 || e1 == g1) return;
            double blo[3], bhi[3], clo[3], chi[3];
            boxInit(blo, bhi);
            sweptAdd(blo, bhi, ld3(x, g0), ld3(dir, g0), eeStep);
            sweptAdd(blo, bhi, ld3(x, g1), ld3(dir, g1), eeStep);
            boxInit(clo, chi);
            sweptAdd(clo, chi, ld3(x, e0), ld3(dir, e0), eeStep);
            sweptAdd(clo, chi, ld3(x, e1), ld3(dir, e1), eeStep);
            if (!overlaps(blo, bhi, clo, chi, 0.0)) return;
            cg::coalesced_group g = cg::coalesced_threads();
            int base = 0;
            if (g.thread_rank() == 0) base = atomicAdd(count, (int)g.size());
            const int i = g.shfl(base, 0) + (int)g.thread_rank();
            if (i < cap) pairs[i] = make_int2(eJ, eI);
        };
        traverse2(tree, qlo, qhi, 0.0, large, status, [&](int other, bool fromLarge) {
            if (!fromLarge || large) {
                if (other > self) pair(self, other);
            } else if (other != self) {
                if (other > self) pair(self, other);
                else pair(other, self);
            }
        });
    }
}

// The additive CCD of every stored pair (eI's points first, as the
// reference calls it); the minimum of 1 and every time of impact goes into
// *outMin by an atomic minimum on the bit pattern (non-negative doubles order
// as their bits), so the result does not depend on the order of the pairs.
__global__ void fullEEAccdKernel(const int2* pairs, const int* count, int cap, const int* edges, const double* x, const double* dir, double eta,
                                 double* outMin, int* status) {
    const int n = min(*count, cap);
    double best = 1.0;
    CIPC_KERNEL_LOOP(k, n) {
        const int2 pr = pairs[k];
        const int g0 = edges[2 * pr.x], g1 = edges[2 * pr.x + 1];
        const int e0 = edges[2 * pr.y], e1 = edges[2 * pr.y + 1];
        const d3 q0 = ld3(x, g0), q1 = ld3(x, g1), dq0 = ld3(dir, g0), dq1 = ld3(dir, g1);
        const d3 p0 = ld3(x, e0), p1 = ld3(x, e1), dp0 = ld3(dir, e0), dp1 = ld3(dir, e1);
        best = fmin(edgeEdgeCCD(p0, p1, q0, q1, -dp0, -dp1, -dq0, -dq1, eta, status), best);
    }
    best = blockReduce(best, MinOp(), 1.0);
    if (threadIdx.x == 0) atomicMin(reinterpret_cast<unsigned long long*>(outMin), (unsigned long long)__double_as_longlong(best));
}

__global__ void setDoubleKernel(double* p, double v) { *p = v; }
__global__ void copyCountKernel(const int* count, double* out) { *out = (double)*count; }

// The segment-triangle test of one (face, edge) pair (the filters of
// checkEdgeTriIntersectionIfAny, IPCSolver.cpp:514-542).
__device__ __forceinline__ bool faceEdgeHit(const int* faces, const int* edges, const int* btype, const double* x, int f, int e, double coplanarTol) {
    int f0 = faces[3 * f], f1 = faces[3 * f + 1], f2 = faces[3 * f + 2];
    int e0 = edges[2 * e], e1 = edges[2 * e + 1];
    if (e0 == f0 || e0 == f1 || e0 == f2 || e1 == f0 || e1 == f1 || e1 == f2) return false;
    if (isCollider(btype[e0]) && isCollider(btype[e1]) && isCollider(btype[f0]) && isCollider(btype[f1]) && isCollider(btype[f2])) return false;
    return segTriIntersect(ld3(x, e0), ld3(x, e1), ld3(x, f0), ld3(x, f1), ld3(x, f2), coplanarTol);
}

// Faces against the edge tree.  A large face (one the face tree keeps out of
// its tree) meets only the edge tree's large edges here; its pairs with the
// other edges are tested by largeFaceKernel from the edges' side.
// Intersection test in two kernels, as the full CCD: each face's walk over
// the edge tree emits its candidate (face, edge) pairs, then one thread per
// pair runs the segment-triangle test (faceEdgeHit) and raises the flag.
template <class View>
__global__ void intersectPairsKernel(int nsf, const int* faces, const double* x, View tree, int2* pairs, int cap, int* count, int* status) {
    CIPC_KERNEL_LOOP(f, nsf) {
        double lo[3], hi[3];
        boxInit(lo, hi);
        for (int k = 0; k < 3; ++k) boxAdd(lo, hi, ld3(x, faces[3 * f + k]));
        const bool large = View::kSplitsBig && isLargeBox(lo, hi, tree.bigExtent);
        traverse2(tree, lo, hi, 0.0, large, status, [&](int e, bool) {
            cg::coalesced_group g = cg::coalesced_threads();
            int base = 0;
            if (g.thread_rank() == 0) base = atomicAdd(count, (int)g.size());
            const int i = g.shfl(base, 0) + (int)g.thread_rank();
            if (i < cap) pairs[i] = make_int2(f, e);
        });
    }
}

__global__ void intersectTestKernel(const int2* pairs, const int* count, int cap, const int* faces, const int* edges, const int* btype,
                                    const double* x, double coplanarTol, int* flag) {
    const int n = min(*count, cap);
    bool hit = false;
    CIPC_KERNEL_LOOP(k, n) {
        const int2 pr = pairs[k];
        if (!hit && faceEdgeHit(faces, edges, btype, x, pr.x, pr.y, coplanarTol)) hit = true;
    }
    if (hit) atomicOr(flag, 1);
}

// The edges that are not large (the edge tree's own) against the large faces
// of the face tree (the last *nbig keys of its sorted order).
__global__ void largeFaceKernel(int ne, const int* faces, const int* edges, const int* btype, const double* x, BvhView faceTree, BvhView edgeTree,
                                double coplanarTol, int* flag) {
    const int nbf = *faceTree.nbig;
    if (nbf == 0) return;
    const int nf = faceTree.nAll - nbf;
    CIPC_KERNEL_LOOP(e, ne) {
        const double* elo = edgeTree.plo + 3 * e;
        const double* ehi = edgeTree.phi + 3 * e;
        if (isLargeBox(elo, ehi, edgeTree.bigExtent)) continue;  // met by the large faces' own queries
        bool hit = false;
        for (int b = 0; b < nbf && !hit; ++b) {
            const int f = (int)(faceTree.keys[nf + b] & 0xffffffffu);
            if (overlaps(faceTree.plo + 3 * f, faceTree.phi + 3 * f, elo, ehi, 0.0) && faceEdgeHit(faces, edges, btype, x, f, e, coplanarTol)) hit = true;
        }
        if (hit) atomicOr(flag, 1);
    }
}

__global__ void groundIntersectKernel(int n, const int* ground, const double* x, double nx, double ny, double nz, double D, int* flag) {
    CIPC_KERNEL_LOOP(i, n) {
        d3 p = ld3(x, ground[i]);
        double dist = nx * p.x + ny * p.y + nz * p.z - D;
        if (dist * dist <= 0.0) atomicOr(flag, 1);
    }
}

// Stable radix sort of 64-bit keys on bits [beginBit, endBit): the bits
// outside the range are either zero for every key or already in order.
void sortKeys(Ctx& c, uint64_t* in, uint64_t* tmp, int n, int endBit, int beginBit = 0) {
    if (n <= 1) return;
    size_t bytes = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, bytes, in, tmp, n, beginBit, endBit, c.s);
    c.sortTmp.reserve(bytes + 16);
    CIPC_CUDA(cub::DeviceRadixSort::SortKeys(c.sortTmp.p, bytes, in, tmp, n, beginBit, endBit, c.s));
    CIPC_CUDA(cudaMemcpyAsync(in, tmp, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, c.s));
}

// bits needed for the values 0 .. m - 1
int bitsFor(int m) {
    int b = 1;
    while (b < 31 && (1 << b) < m) ++b;
    return b;
}

}  // namespace

// Primitive boxes of the face / edge tree at x, or swept from x to
// x - step * d (step read from *stepPtr on the device when it is given).
void computeFaceBoxes(Ctx& c, const double* x, const double* d, double step, bool swept, const double* stepPtr) {
    c.faceTree.primLo.reserve(3 * std::max(1, c.nsf));
    c.faceTree.primHi.reserve(3 * std::max(1, c.nsf));
    if (c.nsf) launch(faceBoxKernel, blocksFor(c.nsf), TB, 0, c.s, c.nsf, c.faces, x, d, step, stepPtr, swept, c.faceTree.primLo, c.faceTree.primHi);
}
void computeEdgeBoxes(Ctx& c, const double* x, const double* d, double step, bool swept, const double* stepPtr) {
    c.edgeTree.primLo.reserve(3 * std::max(1, c.nse));
    c.edgeTree.primHi.reserve(3 * std::max(1, c.nse));
    if (c.nse) launch(edgeBoxKernel, blocksFor(c.nse), TB, 0, c.s, c.nse, c.edges, x, d, step, stepPtr, swept, c.edgeTree.primLo, c.edgeTree.primHi);
}

void buildBvh(Ctx& c, DevBvh& t, int n) {
    t.n = n;
    if (n <= 0) return;
    int nn = 2 * n - 1;
    t.keys.reserve(n); t.keysAlt.reserve(n);
    t.left.reserve(nn); t.right.reserve(nn); t.parent.reserve(nn); t.escape.reserve(nn); t.leafPrim.reserve(n); t.flags.reserve(n);
    t.lo.reserve(3 * nn); t.hi.reserve(3 * nn); t.sceneBox.reserve(6);
    const int nbBox = std::max(1, std::min(148, (n + 255) / 256));
    t.boxPart.reserve(6 * (size_t)nbBox);
    launch(sceneBoxKernel, nbBox, 256, 0, c.s, n, t.primLo, t.primHi, t.boxPart);
    launch(sceneBoxFinalKernel, 1, 256, 0, c.s, nbBox, (const double*)t.boxPart, t.sceneBox);
    t.bigCount.reserve(1);
    CIPC_CUDA(cudaMemsetAsync(t.bigCount.p, 0, sizeof(int), c.s));
    const double bigExtent = t.bigExtent = 0.1 * std::sqrt(c.P.bboxDiag2);
    launch(mortonKernel, blocksFor(n), TB, 0, c.s, n, t.primLo, t.primHi, t.sceneBox, bigExtent, t.keys, t.bigCount.p);
    // keys are (code << 32) | index (bit 62: kept out of the tree), written in
    // index order: a stable sort on bits 32-62 gives the order of a sort on
    // the whole key
    sortKeys(c, t.keys, t.keysAlt, n, 63, 32);
    const int* nbig = t.bigCount.p;
    if (n > 1) launch(karrasKernel, blocksFor(n - 1), TB, 0, c.s, n, nbig, t.keys, t.left, t.right, t.parent);
    launch(leafKernel, blocksFor(n), TB, 0, c.s, n, nbig, t.keys, t.primLo, t.primHi, t.leafPrim, t.lo, t.hi, t.flags, t.parent);
    t.rec.reserve(16 * (size_t)std::max(1, n - 1));
    if (n > 1) launch(refitKernel, blocksFor(n), TB, 0, c.s, n, nbig, t.left, t.right, t.parent, t.lo, t.hi, t.flags, t.rec.p);
    if (n > 1) launch(escapeKernel, blocksFor(nn), TB, 0, c.s, n, nbig, t.left, t.right, t.parent, t.escape);
    CIPC_CUDA(cudaGetLastError());
}

// The spatial-hash tables of one primitive set from its boxes (primLo/Hi).
void buildHash(Ctx& c, DevBvh& t, int n) {
    t.n = n;
    t.hashPairs = 0;
    t.hashBig.reserve(std::max(1, n)); t.hashBigFlag.reserve(std::max(1, n));
    t.hashCount.reserve(std::max(1, n)); t.hashOffset.reserve(std::max(1, n));
    c.counters.reserve(16);
    if (n <= 0) return;
    const double inv = 1.0 / c.P.avgEdge;
    launch(hashCountKernel, blocksFor(n), TB, 0, c.s, n, t.primLo, t.primHi, inv, t.hashCount, t.hashBigFlag);
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, t.hashCount.p, t.hashOffset.p, n, c.s);
    size_t b2 = 0;
    cub::DeviceSelect::Flagged(nullptr, b2, thrust::counting_iterator<int>(0), t.hashBigFlag.p, t.hashBig.p, c.counters.p + 11, n, c.s);
    t.hashTmp.reserve(std::max(bytes, b2) + 16);
    CIPC_CUDA(cub::DeviceScan::ExclusiveSum(t.hashTmp.p, bytes, t.hashCount.p, t.hashOffset.p, n, c.s));
    int last[2];
    CIPC_CUDA(cudaMemcpyAsync(&last[0], t.hashOffset.p + n - 1, sizeof(int), cudaMemcpyDeviceToHost, c.s));
    CIPC_CUDA(cudaMemcpyAsync(&last[1], t.hashCount.p + n - 1, sizeof(int), cudaMemcpyDeviceToHost, c.s));
    hostSync(c);
    const int pairs = last[0] + last[1];
    t.hashPairs = pairs;
    t.hashKey.reserve(std::max(1, pairs)); t.hashKeyAlt.reserve(std::max(1, pairs));
    t.hashPrim.reserve(std::max(1, pairs)); t.hashPrimAlt.reserve(std::max(1, pairs));
    launch(hashEmitKernel, blocksFor(n), TB, 0, c.s, n, t.primLo, t.primHi, inv, (const int*)t.hashOffset, (const int*)t.hashCount, t.hashKeyAlt,
           t.hashPrimAlt);
    if (pairs > 0) {
        size_t b3 = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, b3, t.hashKeyAlt.p, t.hashKey.p, t.hashPrimAlt.p, t.hashPrim.p, pairs, 0, 63, c.s);
        t.hashTmp.reserve(b3 + 16);
        CIPC_CUDA(cub::DeviceRadixSort::SortPairs(t.hashTmp.p, b3, t.hashKeyAlt.p, t.hashKey.p, t.hashPrimAlt.p, t.hashPrim.p, pairs, 0, 63, c.s));
    }
    // the primitives too large for the cells (their ids in order)
    thrust::counting_iterator<int> ids(0);
    size_t b4 = 0;
    cub::DeviceSelect::Flagged(nullptr, b4, ids, t.hashBigFlag.p, t.hashBig.p, c.counters.p + (&t == &c.edgeTree ? 14 : 11), n, c.s);
    t.hashTmp.reserve(b4 + 16);
    CIPC_CUDA(cub::DeviceSelect::Flagged(t.hashTmp.p, b4, ids, t.hashBigFlag.p, t.hashBig.p, c.counters.p + (&t == &c.edgeTree ? 14 : 11), n,
                                         c.s));
    CIPC_CUDA(cudaGetLastError());
}

HashView hview(Ctx& c, const DevBvh& t) {
    return HashView{t.bigExtent, t.n, t.hashPairs, 1.0 / c.P.avgEdge, t.hashKey, t.hashPrim, t.hashBig, c.counters.p + (&t == &c.edgeTree ? 14 : 11),
                    t.primLo, t.primHi};
}

// The broad-phase structure of one primitive set, LBVH or spatial hash.
void buildBroad(Ctx& c, DevBvh& t, int n) {
    if (c.broadPhase == CIPC_BROAD_PHASE_SPATIAL_HASH) buildHash(c, t, n);
    else buildBvh(c, t, n);
}

// Calls k(view) with the selected backend's view of tree t.
template <class K>
void withView(Ctx& c, const DevBvh& t, K k) {
    if (c.broadPhase == CIPC_BROAD_PHASE_SPATIAL_HASH) k(hview(c, t));
    else k(view(t));
}

static void buildStaticTrees(Ctx& c) {
    computeFaceBoxes(c, c.x, c.x, 0.0, false);
    buildBroad(c, c.faceTree, c.nsf);
    computeEdgeBoxes(c, c.x, c.x, 0.0, false);
    buildBroad(c, c.edgeTree, c.nse);
}

// Ground::calculateActivateSet: the surface vertices within dHat of the
// ground, in order, into c.ground; their count lands in counters[15] (read
// back by the caller).
void groundActiveSetLaunch(Ctx& c) {
    c.ground.reserve(std::max(1, c.nsv));
    c.counts.reserve(std::max(1, c.nsv) + 1);
    c.counters.reserve(16);
    if (c.nsv == 0) {
        CIPC_CUDA(cudaMemsetAsync(c.counters.p + 15, 0, sizeof(int), c.s));
        return;
    }
    launch(groundFlagKernel, blocksFor(c.nsv), TB, 0, c.s, c.nsv, c.surfVerts, c.x, c.P.groundN[0], c.P.groundN[1], c.P.groundN[2], c.P.groundD,
                                                       c.P.Hhat, c.counts);
    size_t bytes = 0;
    cub::DeviceSelect::Flagged(nullptr, bytes, c.surfVerts.p, c.counts.p, c.ground.p, c.counters.p + 15, c.nsv, c.s);
    c.groundTmp.reserve(bytes + 16);
    CIPC_CUDA(cub::DeviceSelect::Flagged(c.groundTmp.p, bytes, c.surfVerts.p, c.counts.p, c.ground.p, c.counters.p + 15, c.nsv, c.s));
}

void groundActiveSet(Ctx& c) {
    groundActiveSetLaunch(c);
    int n = 0;
    CIPC_CUDA(cudaMemcpyAsync(&n, c.counters.p + 15, sizeof(int), cudaMemcpyDeviceToHost, c.s));
    hostSync(c);
    c.nGround = n;
}

// SpatialHash::calculateActivateSet with the LBVH backend, then
// Ground::calculateActivateSet (IPCSolver.cpp:544-556).
void buildCollisionSets(Ctx& c, bool rehash) {
    if (c.P.useBarrier) {
        if (rehash) buildStaticTrees(c);
        double sq = sqrt(c.P.Hhat);
        int caps[6] = {(int)std::max<size_t>(c.ccdPT.cap, 1024), (int)std::max<size_t>(c.kPT.cap, 1024), (int)std::max<size_t>(c.kPPE.cap, 1024),
                       (int)std::max<size_t>(c.ccdEE.cap, 1024), (int)std::max<size_t>(c.kEE.cap, 1024), (int)std::max<size_t>(c.kMoll.cap, 1024)};
        int cnt[6];
        int stWord = 0;
        bool fits = false;
        for (int attempt = 0; attempt < 4; ++attempt) {
            c.ccdPT.reserve(caps[0]); c.kPT.reserve(caps[1]); c.kPPE.reserve(caps[2]);
            c.ccdEE.reserve(caps[3]); c.kEE.reserve(caps[4]); c.kMoll.reserve(caps[5]);
            c.counters.reserve(16);
            CIPC_CUDA(cudaMemsetAsync(c.counters.p, 0, 8 * sizeof(int), c.s));
            Emit eCcdPT{c.ccdPT, caps[0], c.counters.p + 0}, ePT{c.kPT, caps[1], c.counters.p + 1}, ePPE{c.kPPE, caps[2], c.counters.p + 2};
            Emit eCcdEE{c.ccdEE, caps[3], c.counters.p + 3}, eEE{c.kEE, caps[4], c.counters.p + 4}, eMoll{c.kMoll, caps[5], c.counters.p + 5};
            profBegin(c, PROF_ACTIVE);
            if (c.nsv) {
                withView(c, c.faceTree, [&](auto v) {
                    launch(activePTKernel<decltype(v)>, blocksFor(c.nsv), TB, 0, c.s, c.nsv, c.surfVerts, c.faces, c.btype, c.x, v, sq, eCcdPT, c.status);
                });
                launch(activePTClassKernel, 148 * 8, TB, 0, c.s, (const uint64_t*)c.ccdPT.p, (const int*)c.counters.p + 0, caps[0], c.surfVerts, c.faces,
                       c.x, c.P.Hhat, ePT, ePPE, c.status);
            }
            if (c.nse) {
                withView(c, c.edgeTree, [&](auto v) {
                    launch(activeEEKernel<decltype(v)>, blocksFor(c.nse), TB, 0, c.s, c.nse, c.edges, c.btype, c.x, v, sq, eCcdEE, c.status);
                });
                launch(activeEEClassKernel, 148 * 8, TB, 0, c.s, (const uint64_t*)c.ccdEE.p, (const int*)c.counters.p + 3, caps[3], c.edges, c.x, c.rest,
                       c.P.Hhat, eEE, eMoll, ePPE, c.status);
            }
            profEnd(c, PROF_ACTIVE);
            CIPC_CUDA(cudaGetLastError());
            CIPC_CUDA(cudaMemcpyAsync(cnt, c.counters.p, 6 * sizeof(int), cudaMemcpyDeviceToHost, c.s));
            CIPC_CUDA(cudaMemcpyAsync(&stWord, c.status.p, sizeof(int), cudaMemcpyDeviceToHost, c.s));
            hostSync(c);
            fits = true;
            for (int k = 0; k < 6; ++k)
                if (cnt[k] > caps[k]) { caps[k] = cnt[k] + cnt[k] / 2 + 1024; fits = false; }
            if (fits || attempt == 3) break;
            int st = 0;  // clear the capacity bit before retrying (only when another attempt follows)
            CIPC_CUDA(cudaMemcpyAsync(c.status.p, &st, sizeof(int), cudaMemcpyHostToDevice, c.s));
        }
        if (stWord) checkStatus(c, "active set");
        // the counts size the sorts and decodes below: never past what the
        // last launch could write
        if (!fits) throw std::runtime_error("active-set candidate counts exceed their buffers after four attempts");
        c.nCcdPT = cnt[0]; c.nPT = cnt[1]; c.nPPERaw = cnt[2]; c.nCcdEE = cnt[3]; c.nEE = cnt[4]; c.nMoll = cnt[5];
        int mx = std::max(std::max(std::max(cnt[0], cnt[1]), std::max(cnt[2], cnt[3])), std::max(cnt[4], cnt[5]));
        c.kTmp.reserve(std::max(mx, 1));
        // pair keys (query << 32 | primitive), mollified (eI << 34 | eJ << 4 | type)
        const int ptBits = 32 + bitsFor(c.nsv), eeBits = 32 + bitsFor(c.nse), mollBits = std::min(64, 34 + bitsFor(c.nse));
        sortKeys(c, c.ccdPT, c.kTmp, cnt[0], ptBits);
        sortKeys(c, c.kPT, c.kTmp, cnt[1], ptBits);
        sortKeys(c, c.kPPE, c.kTmp, cnt[2], 63);
        sortKeys(c, c.ccdEE, c.kTmp, cnt[3], eeBits);
        sortKeys(c, c.kEE, c.kTmp, cnt[4], eeBits);
        sortKeys(c, c.kMoll, c.kTmp, cnt[5], mollBits);
        // merge PP/PE duplicates (multiplicity)
        int nu = 0;
        c.uniq.reserve(std::max(cnt[2], 1));
        c.runs.reserve(std::max(cnt[2], 1));
        if (cnt[2] > 0) {
            size_t bytes = 0;
            cub::DeviceRunLengthEncode::Encode(nullptr, bytes, c.kPPE.p, c.uniq.p, c.runs.p, c.counters.p + 6, cnt[2], c.s);
            c.sortTmp.reserve(bytes + 16);
            CIPC_CUDA(cub::DeviceRunLengthEncode::Encode(c.sortTmp.p, bytes, c.kPPE.p, c.uniq.p, c.runs.p, c.counters.p + 6, cnt[2], c.s));
        } else {
            CIPC_CUDA(cudaMemsetAsync(c.counters.p + 6, 0, sizeof(int), c.s));
        }
        // the ground set is selected meanwhile; both counts come back at once
        groundActiveSetLaunch(c);
        {
            int h[10];
            CIPC_CUDA(cudaMemcpyAsync(h, c.counters.p + 6, 10 * sizeof(int), cudaMemcpyDeviceToHost, c.s));
            hostSync(c);
            nu = h[0];
            c.nGround = h[9];
        }
        c.nPPE = nu;
        c.nSelf = c.nPT + c.nEE + c.nPPE;
        c.selfActive.reserve(4 * std::max(c.nSelf, 1));
        if (c.nSelf)
            launch(decodeSelfKernel, blocksFor(c.nSelf), TB, 0, c.s, c.nPT, c.nEE, c.nPPE, c.kPT, c.kEE, c.uniq, c.runs, c.surfVerts, c.faces, c.edges,
                                                                 c.selfActive);
        c.selfEE.reserve(4 * std::max(c.nMoll, 1));
        c.eeIe.reserve(2 * std::max(c.nMoll, 1));
        if (c.nMoll) launch(decodeMollKernel, blocksFor(c.nMoll), TB, 0, c.s, c.nMoll, c.kMoll, c.edges, c.selfEE, c.eeIe);
        CIPC_CUDA(cudaGetLastError());
    } else {
        groundActiveSet(c);
    }
}

// the candidate-pair buffer shared by the intersection test and the full CCD
static int ccdPairsReserve(Ctx& c);

bool isIntersected(Ctx& c) {
    c.counters.reserve(16);
    CIPC_CUDA(cudaMemsetAsync(c.counters.p + 7, 0, sizeof(int), c.s));
    if (c.nGround)
        launch(groundIntersectKernel, blocksFor(c.nGround), TB, 0, c.s, c.nGround, c.ground, c.x, c.P.groundN[0], c.P.groundN[1], c.P.groundN[2],
                                                                   c.P.groundD, c.counters.p + 7);
    if (c.nse && c.nsf && c.broadPhase == CIPC_BROAD_PHASE_LBVH)
        launch(largeFaceKernel, blocksFor(c.nse), TB, 0, c.s, c.nse, c.faces, c.edges, c.btype, c.x, view(c.faceTree), view(c.edgeTree), c.coplanarTol,
               c.counters.p + 7);
    for (;;) {
        int cap = 0;
        if (c.nsf) {
            cap = ccdPairsReserve(c);
            CIPC_CUDA(cudaMemsetAsync(c.ccdPairCount.p, 0, sizeof(int), c.s));
            withView(c, c.edgeTree, [&](auto v) {
                launch(intersectPairsKernel<decltype(v)>, blocksFor(c.nsf), TB, 0, c.s, c.nsf, c.faces, c.x, v, c.ccdPairs.p, cap, c.ccdPairCount.p,
                       c.status);
            });
            launch(intersectTestKernel, 148 * 8, TB, 0, c.s, (const int2*)c.ccdPairs.p, (const int*)c.ccdPairCount.p, cap, c.faces, c.edges, c.btype,
                   c.x, c.coplanarTol, c.counters.p + 7);
        }
        int h[3] = {0, 0, 0};
        CIPC_CUDA(cudaMemcpyAsync(&h[0], c.counters.p + 7, sizeof(int), cudaMemcpyDeviceToHost, c.s));
        CIPC_CUDA(cudaMemcpyAsync(&h[1], c.status.p, sizeof(int), cudaMemcpyDeviceToHost, c.s));
        if (c.nsf) CIPC_CUDA(cudaMemcpyAsync(&h[2], c.ccdPairCount.p, sizeof(int), cudaMemcpyDeviceToHost, c.s));
        hostSync(c);
        if (h[1]) checkStatus(c, "intersection test");
        // a hit among the stored pairs stands; otherwise every pair must have been tested
        if (h[0] != 0 || h[2] <= cap) return h[0] != 0;
        c.ccdPairs.reserve((size_t)h[2]);
    }
}

// Rebuild the static trees at the current positions (sh.build in the line search).
void rebuildTrees(Ctx& c) { buildStaticTrees(c); }

double groundStepBound(Ctx& c) {
    if (c.nsv == 0) return 1.0;
    c.energyBuf.reserve(std::max(c.nsv, 1));
    launch(groundBoundKernel, blocksFor(c.nsv), TB, 0, c.s, c.nsv, c.surfVerts, c.x, c.dir, c.P.groundN[0], c.P.groundN[1], c.P.groundN[2], c.P.groundD,
                                                        0.8, c.energyBuf);
    return deviceMin(c, c.energyBuf, c.nsv, 1e308);
}

double partialCCD(Ctx& c, double alpha) {
    int n = c.nCcdPT + c.nCcdEE;
    if (n == 0) return alpha;
    c.energyBuf.reserve(n);
    launch(partialCCDKernel, blocksFor(n), TB, 0, c.s, c.nCcdPT, c.nCcdEE, c.ccdPT, c.ccdEE, c.surfVerts, c.faces, c.edges, c.x, c.dir, 1.0 - 0.8,
                                                  c.energyBuf, c.status);
    double mn = deviceMin(c, c.energyBuf, n, 1e308);
    checkStatus(c, "partial CCD");
    return std::min(alpha, mn);
}

double cflBound(Ctx& c) {
    if (c.nsv == 0) return 1.0;
    c.energyBuf.reserve(c.nsv);
    launch(surfMoveKernel, blocksFor(c.nsv), TB, 0, c.s, c.nsv, c.surfVerts, c.dir, c.energyBuf);
    double mx = std::max(0.0, deviceMax(c, c.energyBuf, c.nsv));
    return mx > 0.0 ? sqrt(c.P.Hhat) / (mx * 2.0) : 1.0;
}

// The full edge-edge CCD over the swept edge tree (built with the entry
// step stepVal, or *stepPtr when given): candidate pairs, then one thread per
// pair; min(1, every time of impact) into the device scalar *outMin.  The
// pair count stays on the device (ccdPairCount): a caller that finds it above
// the buffer's capacity grows the buffer and runs again.
// First size of the pair buffer: 8 pairs per query, or CIPC_CCD_PAIRS_INITIAL
// pairs (a small value exercises the grow-and-rerun path).
static size_t ccdPairsInitial(const Ctx& c) {
    static long long v = -2;
    if (v == -2) { const char* e = std::getenv("CIPC_CCD_PAIRS_INITIAL"); v = e ? std::atoll(e) : -1; }
    return v > 0 ? (size_t)v : std::max<size_t>(1024, 8 * (size_t)std::max(c.nse, c.nsv));
}
static int ccdPairsReserve(Ctx& c) {
    c.ccdPairCount.reserve(2);
    c.ccdPairs.reserve(ccdPairsInitial(c));
    return (int)std::min<size_t>(c.ccdPairs.cap, 0x7fffffff);
}
static void fullEEDevice(Ctx& c, const double* d, double stepVal, const double* stepPtr, double* outMin) {
    const int cap = ccdPairsReserve(c);
    CIPC_CUDA(cudaMemsetAsync(c.ccdPairCount.p + 1, 0, sizeof(int), c.s));
    launch(setDoubleKernel, 1, 1, 0, c.s, outMin, 1.0);
    withView(c, c.edgeTree, [&](auto v) {
        launch(fullEEPairsKernel<decltype(v)>, blocksFor(c.nse), TB, 0, c.s, c.nse, c.edges, c.btype, c.x, d, c.edgeTree.primLo, c.edgeTree.primHi,
               stepVal, stepPtr, v, c.ccdPairs.p, cap, c.ccdPairCount.p + 1, c.status);
    });
    launch(fullEEAccdKernel, 148 * 8, TB, 0, c.s, (const int2*)c.ccdPairs.p, (const int*)c.ccdPairCount.p + 1, cap, c.edges, c.x, d, 1.0 - 0.8,
           outMin, c.status);
}
// The same for the point-triangle pairs (surface vertices against the swept
// face tree), count in ccdPairCount[0].
static void fullPTDevice(Ctx& c, const double* d, double stepVal, const double* stepPtr, double* outMin) {
    const int cap = ccdPairsReserve(c);
    CIPC_CUDA(cudaMemsetAsync(c.ccdPairCount.p, 0, sizeof(int), c.s));
    launch(setDoubleKernel, 1, 1, 0, c.s, outMin, 1.0);
    withView(c, c.faceTree, [&](auto v) {
        launch(fullPTPairsKernel<decltype(v)>, blocksFor(c.nsv), TB, 0, c.s, c.nsv, c.surfVerts, c.faces, c.btype, c.x, d, stepVal, stepPtr, v,
               c.ccdPairs.p, cap, c.ccdPairCount.p, c.status);
    });
    launch(fullPTAccdKernel, 148 * 8, TB, 0, c.s, (const int2*)c.ccdPairs.p, (const int*)c.ccdPairCount.p, cap, c.faces, c.x, d, 1.0 - 0.8, outMin,
           c.status);
}

// Swept build with the entry step, then Self_largestFeasibleStepSize_CCD.
double fullCCDDir(Ctx& c, const double* d, double alpha) {
    double step = alpha;
    computeFaceBoxes(c, c.x, d, step, true);
    buildBroad(c, c.faceTree, c.nsf);
    computeEdgeBoxes(c, c.x, d, step, true);
    buildBroad(c, c.edgeTree, c.nse);
    c.stepScal.reserve(16);
    double* sm = c.stepScal.p + 12;  // [12] minimum, [13] pair count
    // one pass (point-triangle or edge-edge) with the host's entry step; a
    // pair buffer that was too small is grown and the pass runs again
    auto pass = [&](bool pt) {
        for (;;) {
            profBegin(c, PROF_FULLCCD);
            if (pt) fullPTDevice(c, d, step, nullptr, sm);
            else fullEEDevice(c, d, step, nullptr, sm);
            profEnd(c, PROF_FULLCCD);
            launch(copyCountKernel, 1, 1, 0, c.s, (const int*)c.ccdPairCount.p + (pt ? 0 : 1), sm + 1);
            double h[2];
            CIPC_CUDA(cudaMemcpyAsync(h, sm, sizeof(h), cudaMemcpyDeviceToHost, c.s));
            hostSync(c);
            if (h[1] <= (double)c.ccdPairs.cap) { step = std::min(step, h[0]); return; }
            c.ccdPairs.reserve((size_t)h[1]);
        }
    };
    if (c.nsv) pass(true);
    if (c.nse) pass(false);
    checkStatus(c, "full CCD");
    return step;
}

double fullCCD(Ctx& c, double alpha) { return fullCCDDir(c, c.dir, alpha); }

namespace {
// Scalars of the chained step bounds (stepBoundsDevice), one thread each.
// s: 0 ground min, 1 partial-CCD min, 2 max surface move, 3 entry step,
// 4 full point-triangle min, 5 edge-edge entry step, 6 full edge-edge min,
// 7 merged step, 8 status word, 9 and 10 point-triangle and edge-edge
// CCD pair counts.
__global__ void stepEntryKernel(double* s, int nsv) {
    double a = nsv ? s[0] : 1.0;
    a = fmin(1.0, a);
    if (a <= 0) a = 1;
    s[3] = a;
    s[5] = a;
}
__global__ void stepEeEntryKernel(double* s) { s[5] = fmin(s[3], s[4]); }
__global__ void stepMergeKernel(double* s, int nsv, int nse, int nPartial, int barrier, double sqrtHhat, const int* status) {
    const double alpha = s[3];
    double a = alpha;
    if (barrier) {
        const double partial = nPartial ? fmin(alpha, s[1]) : alpha;
        const double mx = nsv ? fmax(0.0, s[2]) : 0.0;
        const double aCFL = mx > 0.0 ? sqrtHhat / (mx * 2.0) : 1.0;
        double full = alpha;
        if (nsv) full = fmin(full, s[4]);
        if (nse) full = fmin(full, s[6]);
        a = fmin(a, aCFL);
        if (partial > 2.0 * aCFL) {
            a = fmin(partial, full);
            a = fmax(a, aCFL);
        }
        s[1] = partial; s[2] = aCFL; s[6] = full;
    }
    s[7] = a;
    s[8] = (double)*status;
}
}  // namespace

// The step bound of one Newton iteration (IPCSolver.cpp:943-990) without
// host round trips between its stages: the ground bound gives the entry step,
// the partial CCD, CFL bound and the swept full CCD (entry step read on the
// device, the edge-edge pass starting from the point-triangle result) write
// device scalars, and one kernel applies the merge rule.  One read-back.
double stepBoundsDevice(Ctx& c) {
    c.stepScal.reserve(16);
    double* s = c.stepScal.p;
    const int nPartial = c.nCcdPT + c.nCcdEE;
    c.energyBuf.reserve(std::max(std::max(std::max(c.nsv, c.nse), nPartial), 1));
    if (c.nsv) {
        launch(groundBoundKernel, blocksFor(c.nsv), TB, 0, c.s, c.nsv, c.surfVerts, c.x, c.dir, c.P.groundN[0], c.P.groundN[1], c.P.groundN[2],
               c.P.groundD, 0.8, c.energyBuf);
        deviceMinTo(c, c.energyBuf, c.nsv, s + 0);
    }
    launch(stepEntryKernel, 1, 1, 0, c.s, s, c.nsv);
    if (c.P.useBarrier) {
        if (nPartial) {
            launch(partialCCDKernel, blocksFor(nPartial), TB, 0, c.s, c.nCcdPT, c.nCcdEE, c.ccdPT, c.ccdEE, c.surfVerts, c.faces, c.edges, c.x, c.dir,
                   1.0 - 0.8, c.energyBuf, c.status);
            deviceMinTo(c, c.energyBuf, nPartial, s + 1);
        }
        if (c.nsv) {
            launch(surfMoveKernel, blocksFor(c.nsv), TB, 0, c.s, c.nsv, c.surfVerts, c.dir, c.energyBuf);
            deviceMaxTo(c, c.energyBuf, c.nsv, s + 2);
        }
        computeFaceBoxes(c, c.x, c.dir, 0.0, true, s + 3);
        buildBroad(c, c.faceTree, c.nsf);
        computeEdgeBoxes(c, c.x, c.dir, 0.0, true, s + 3);
        buildBroad(c, c.edgeTree, c.nse);
        ccdPairsReserve(c);
        CIPC_CUDA(cudaMemsetAsync(c.ccdPairCount.p, 0, 2 * sizeof(int), c.s));
        if (c.nsv) {
            profBegin(c, PROF_FULLCCD);
            fullPTDevice(c, c.dir, 0.0, s + 3, s + 4);
            profEnd(c, PROF_FULLCCD);
            launch(stepEeEntryKernel, 1, 1, 0, c.s, s);
        }
        if (c.nse) {
            profBegin(c, PROF_FULLCCD);
            fullEEDevice(c, c.dir, 0.0, s + 5, s + 6);
            profEnd(c, PROF_FULLCCD);
        }
        launch(copyCountKernel, 1, 1, 0, c.s, (const int*)c.ccdPairCount.p, s + 9);
        launch(copyCountKernel, 1, 1, 0, c.s, (const int*)c.ccdPairCount.p + 1, s + 10);
    }
    launch(stepMergeKernel, 1, 1, 0, c.s, s, c.nsv, c.nse, nPartial, c.P.useBarrier ? 1 : 0, std::sqrt(c.P.Hhat), (const int*)c.status.p);
    CIPC_CUDA(cudaGetLastError());
    double h[11];
    CIPC_CUDA(cudaMemcpyAsync(h, s, sizeof(h), cudaMemcpyDeviceToHost, c.s));
    hostSync(c);
    if (h[8] != 0.0) checkStatus(c, "step bounds");
    const double pairs = std::max(h[9], h[10]);
    if (c.P.useBarrier && pairs > (double)c.ccdPairs.cap) {
        // more CCD candidates than the pair buffer holds: grow it and
        // recompute the bounds (every input is unchanged)
        c.ccdPairs.reserve((size_t)pairs);
        return stepBoundsDevice(c);
    }
    return h[7];
}


// Additive CCD on a batch of independent candidate pairs (the per-pair time
// of impact of Self_largestFeasibleStepSize, ContactMechanics.cpp:3704-3752,
// AdditiveCCD.cpp:221-329): kind 0 point-triangle (point, t0, t1, t2), kind 1
// edge-edge (a0, a1, b0, b1); 12 positions and 12 displacements per pair.
namespace {
__global__ void accdBatchKernel(int n, const int* kind, const double* p, const double* d, double eta, double* toi, int* status) {
    CIPC_KERNEL_LOOP(k, n) {
        const double* q = p + 12 * (size_t)k;
        const double* m = d + 12 * (size_t)k;
        d3 x[4], v[4];
        for (int a = 0; a < 4; ++a) {
            x[a] = mk(q[3 * a], q[3 * a + 1], q[3 * a + 2]);
            v[a] = mk(m[3 * a], m[3 * a + 1], m[3 * a + 2]);
        }
        toi[k] = kind[k] == 0 ? pointTriangleCCD(x[0], x[1], x[2], x[3], v[0], v[1], v[2], v[3], eta, status)
                              : edgeEdgeCCD(x[0], x[1], x[2], x[3], v[0], v[1], v[2], v[3], eta, status);
    }
}
}  // namespace

void accdBatch(int n, const int* kind, const double* p, const double* d, double eta, double* toi) {
    DBuf<int> dk, st;
    DBuf<double> dp, dd, dt;
    try {
        dk.reserve(n); dp.reserve(12 * (size_t)n); dd.reserve(12 * (size_t)n); dt.reserve(n); st.reserve(1);
        CIPC_CUDA(cudaMemcpy(dk.p, kind, sizeof(int) * n, cudaMemcpyHostToDevice));
        CIPC_CUDA(cudaMemcpy(dp.p, p, sizeof(double) * 12 * (size_t)n, cudaMemcpyHostToDevice));
        CIPC_CUDA(cudaMemcpy(dd.p, d, sizeof(double) * 12 * (size_t)n, cudaMemcpyHostToDevice));
        CIPC_CUDA(cudaMemset(st.p, 0, sizeof(int)));
        launch(accdBatchKernel, blocksFor(n), TB, 0, (cudaStream_t)0, n, (const int*)dk.p, (const double*)dp.p, (const double*)dd.p, eta,
               dt.p, st.p);
        CIPC_CUDA(cudaGetLastError());
        int hs = 0;
        CIPC_CUDA(cudaMemcpy(toi, dt.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
        CIPC_CUDA(cudaMemcpy(&hs, st.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (hs & CIPC_ST_CCD_CAP) throw std::runtime_error("a pair reached the CCD iteration cap");
    } catch (...) {
        dk.free(); dp.free(); dd.free(); dt.free(); st.free();
        throw;
    }
    dk.free(); dp.free(); dd.free(); dt.free(); st.free();
}

}  // namespace cipc
