// GPU BVH builder: binned-SAH binary tree, collapsed into an 8-wide BVH with
// quantized (compressed) child boxes.  Replaces optixAccelBuild
// (libWR/src/internal/scene.cpp:493-550 in trianglestrip/OfflineRenderer).
//
// Binary build, level by level over all open tasks at once:
//   bin     -- every primitive adds its AABB to its task's 16 bins on each axis
//              (atomics on order-preserving integer encodings of floats, merged per
//              block in shared memory when the block lies in one task)
//   split   -- one thread per task sweeps the 3x15 candidate planes for the lowest
//              SAH cost (object median when all centroids share a bin); allocates the
//              two children; children of <= kSmallTask primitives go to the small list
//   flags + exclusive scan + scatter -- stable partition of each task's range,
//              accumulating child boxes and centroid bounds with atomics.
// Small tasks are finished by one thread each with a sorted SAH sweep.
//
// Collapse: top-down, one thread per 8-wide node.  The binary child with the
// largest surface area is opened until 8 children; children go to slots by
// corner (octant) so traversal can visit them front-to-back by XOR with the ray's
// octant; child boxes are quantized to 8 bits against the node box, widened by one
// quantization step so decoding never shrinks a box.  Leaves' triangles are copied
// into leaf order as (v0|prim, v1-v0|material, v2-v0) records.
#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <vector>

#include "wrk_internal.h"

namespace wrk {
namespace {

constexpr int kBins = 16;
constexpr uint32_t kSmallTask = 16;
constexpr uint32_t kMaxLeaf = 3;
// BVH levels (and collapse depths) enqueued between two host reads of the counts.
constexpr int kLevelsPerSync = 4;
constexpr uint32_t kMaxLevels = 256;

__host__ __device__ __forceinline__ uint32_t f2o(float f) {
#ifdef __CUDA_ARCH__
    uint32_t u = __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, 4);
#endif
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

struct BNode {
    float lo[3];
    uint32_t left;  // internal: left child (right = left+1); leaf: first primitive position
    float hi[3];
    uint32_t count;  // 0 = internal
};
struct OBox {
    uint32_t lo[3], hi[3];
};  // order-encoded floats, for atomic min/max
struct Task {
    uint32_t node, begin, end, pad;
};
struct Bin {
    uint32_t cnt;
    uint32_t lo[3], hi[3];
    uint32_t pad;
};
struct Split {
    int axis, bin;
    uint32_t nLeft;
    int leftTask, rightTask;  // >= 0 next-level task id, -1 prims finished
    uint32_t leftNode;
    uint32_t pad[2];
};
struct SmallTask {
    uint32_t node, begin, end, pad;
};
// cur: open tasks of the level being built (set on the device from nextTasks at the
// start of each level, so the host need not read it back between levels).
struct BuildCtr {
    uint32_t nodes, nextTasks, small, cur;
};
struct CollapseCtr {
    uint32_t nodes, tris, next, maxDepth, cur;
};

__device__ __forceinline__ void obox_empty(OBox& b) {
    for (int k = 0; k < 3; ++k) { b.lo[k] = f2o(FLT_MAX); b.hi[k] = f2o(-FLT_MAX); }
}

__global__ void k_prim_bounds(const float* __restrict__ vtx, const uint32_t* __restrict__ idx, uint32_t n,
                              float4* __restrict__ blo, float4* __restrict__ bhi, OBox* rootBox, OBox* rootCen) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    float c[3] = {0, 0, 0};
    bool valid = i < n;
    if (valid) {
        for (int v = 0; v < 3; ++v) {
            uint32_t k = idx[3 * i + v];
            for (int a = 0; a < 3; ++a) {
                float x = vtx[3 * k + a];
                lo[a] = fminf(lo[a], x);
                hi[a] = fmaxf(hi[a], x);
            }
        }
        blo[i] = make_float4(lo[0], lo[1], lo[2], 0.0f);
        bhi[i] = make_float4(hi[0], hi[1], hi[2], 0.0f);
        for (int a = 0; a < 3; ++a) c[a] = 0.5f * (lo[a] + hi[a]);
    }
    // block-reduce to a few atomics
    typedef cub::BlockReduce<float, 256> BR;
    __shared__ typename BR::TempStorage tmp;
    for (int a = 0; a < 3; ++a) {
        float m = BR(tmp).Reduce(lo[a], cub::Min());
        __syncthreads();
        float M = BR(tmp).Reduce(hi[a], cub::Max());
        __syncthreads();
        float cm = BR(tmp).Reduce(valid ? c[a] : FLT_MAX, cub::Min());
        __syncthreads();
        float cM = BR(tmp).Reduce(valid ? c[a] : -FLT_MAX, cub::Max());
        __syncthreads();
        if (threadIdx.x == 0) {
            atomicMin(&rootBox->lo[a], f2o(m));
            atomicMax(&rootBox->hi[a], f2o(M));
            atomicMin(&rootCen->lo[a], f2o(cm));
            atomicMax(&rootCen->hi[a], f2o(cM));
        }
    }
}

// One thread, at the start of a level: the tasks the last level opened become this
// level's (the device keeps the count; the host reads it only every few levels).
__global__ void k_level_begin(BuildCtr* ctr) {
    ctr->cur = ctr->nextTasks;
    ctr->nextTasks = 0;
}

__global__ void k_init_bins(Bin* bins, const BuildCtr* __restrict__ ctr) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ctr->cur * 3u * kBins) return;
    Bin b;
    b.cnt = 0;
    for (int k = 0; k < 3; ++k) { b.lo[k] = f2o(FLT_MAX); b.hi[k] = f2o(-FLT_MAX); }
    b.pad = 0;
    bins[i] = b;
}

__device__ __forceinline__ int bin_of(float c, float lo, float ext) {
    if (!(ext > 0.0f)) return 0;
    int b = (int)((c - lo) * ((float)kBins / ext));
    return min(kBins - 1, max(0, b));
}

// A block's primitives occupy consecutive positions and a task's primitives one
// contiguous range, so when the block's first and last positions share an open
// task, all of them do.  The block then merges into shared-memory copies of the
// task's bins / child boxes first and each field takes one global atomic per block
// instead of one per primitive (near the root every primitive of the scene would
// otherwise hit the same few addresses).  min / max / add give the same result in
// any order, so the tree does not change.
__device__ __forceinline__ int block_task(uint32_t n, const int* __restrict__ taskOf) {
    const uint32_t i0 = blockIdx.x * blockDim.x, i1 = min(n, i0 + blockDim.x) - 1;
    const int a = taskOf[i0], b = taskOf[i1];
    return a >= 0 && a == b ? a : -1;
}

__global__ void k_bin(uint32_t n, const uint32_t* __restrict__ ref, const int* __restrict__ taskOf,
                      const OBox* __restrict__ tcen, const float4* __restrict__ blo, const float4* __restrict__ bhi,
                      Bin* bins) {
    __shared__ uint32_t sCnt[3 * kBins], sLo[3 * kBins][3], sHi[3 * kBins][3];
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const int bt = block_task(n, taskOf);
    if (bt >= 0) {
        for (uint32_t k = threadIdx.x; k < 3 * kBins; k += blockDim.x) {
            sCnt[k] = 0;
            for (int c = 0; c < 3; ++c) { sLo[k][c] = 0xffffffffu; sHi[k][c] = 0u; }
        }
        __syncthreads();
        if (i < n) {
            const uint32_t p = ref[i];
            const float4 l = blo[p], h = bhi[p];
            const float lo[3] = {l.x, l.y, l.z}, hi[3] = {h.x, h.y, h.z};
            const OBox cb = tcen[bt];
            for (int a = 0; a < 3; ++a) {
                const float cl = o2f(cb.lo[a]), ch = o2f(cb.hi[a]);
                const int k = a * kBins + bin_of(0.5f * (lo[a] + hi[a]), cl, ch - cl);
                atomicAdd(&sCnt[k], 1u);
                for (int c = 0; c < 3; ++c) {
                    atomicMin(&sLo[k][c], f2o(lo[c]));
                    atomicMax(&sHi[k][c], f2o(hi[c]));
                }
            }
        }
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < 3 * kBins; k += blockDim.x) {
            if (!sCnt[k]) continue;
            Bin* bn = bins + (size_t)bt * 3 * kBins + k;
            atomicAdd(&bn->cnt, sCnt[k]);
            for (int c = 0; c < 3; ++c) {
                atomicMin(&bn->lo[c], sLo[k][c]);
                atomicMax(&bn->hi[c], sHi[k][c]);
            }
        }
        return;
    }
    if (i >= n) return;
    int t = taskOf[i];
    if (t < 0) return;
    uint32_t p = ref[i];
    float4 l = blo[p], h = bhi[p];
    float lo[3] = {l.x, l.y, l.z}, hi[3] = {h.x, h.y, h.z};
    OBox cb = tcen[t];
    for (int a = 0; a < 3; ++a) {
        float cl = o2f(cb.lo[a]), ch = o2f(cb.hi[a]);
        int b = bin_of(0.5f * (lo[a] + hi[a]), cl, ch - cl);
        Bin* bn = bins + ((size_t)t * 3 + a) * kBins + b;
        atomicAdd(&bn->cnt, 1u);
        for (int k = 0; k < 3; ++k) {
            atomicMin(&bn->lo[k], f2o(lo[k]));
            atomicMax(&bn->hi[k], f2o(hi[k]));
        }
    }
}

__device__ __forceinline__ float half_area(const float lo[3], const float hi[3]) {
    float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    if (!(dx >= 0.0f)) return 0.0f;
    return dx * dy + dy * dz + dz * dx;
}

__global__ void k_split(const Task* __restrict__ tasks, const Bin* __restrict__ bins, Split* splits, Task* nextTasks,
                        OBox* nextCen, SmallTask* small, BNode* nodes, OBox* nbox, BuildCtr* ctr) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ctr->cur) return;
    Task tk = tasks[t];
    uint32_t cnt = tk.end - tk.begin;
    float bestCost = FLT_MAX;
    int bestAxis = -1, bestBin = -1;
    uint32_t bestLeft = 0;
    for (int a = 0; a < 3; ++a) {
        const Bin* B = bins + ((size_t)t * 3 + a) * kBins;
        float rA[kBins];
        uint32_t rN[kBins];
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        uint32_t c = 0;
        for (int b = kBins - 1; b > 0; --b) {
            c += B[b].cnt;
            if (B[b].cnt)
                for (int k = 0; k < 3; ++k) { lo[k] = fminf(lo[k], o2f(B[b].lo[k])); hi[k] = fmaxf(hi[k], o2f(B[b].hi[k])); }
            rA[b] = half_area(lo, hi);
            rN[b] = c;
        }
        for (int k = 0; k < 3; ++k) { lo[k] = FLT_MAX; hi[k] = -FLT_MAX; }
        c = 0;
        for (int b = 0; b < kBins - 1; ++b) {
            c += B[b].cnt;
            if (B[b].cnt)
                for (int k = 0; k < 3; ++k) { lo[k] = fminf(lo[k], o2f(B[b].lo[k])); hi[k] = fmaxf(hi[k], o2f(B[b].hi[k])); }
            if (c == 0 || rN[b + 1] == 0) continue;
            float cost = half_area(lo, hi) * (float)c + rA[b + 1] * (float)rN[b + 1];
            if (cost < bestCost) { bestCost = cost; bestAxis = a; bestBin = b; bestLeft = c; }
        }
    }
    Split sp;
    sp.axis = bestAxis;
    sp.bin = bestBin;
    sp.nLeft = bestAxis >= 0 ? bestLeft : cnt / 2;  // object median when no plane separates
    uint32_t child = atomicAdd(&ctr->nodes, 2u);
    sp.leftNode = child;
    BNode nd;
    nd.left = child;
    nd.count = 0;
    nodes[tk.node] = nd;  // box filled from nbox at the end
    uint32_t nn[2] = {sp.nLeft, cnt - sp.nLeft};
    uint32_t beg[2] = {tk.begin, tk.begin + sp.nLeft};
    int tid[2];
    for (int s = 0; s < 2; ++s) {
        OBox e;
        obox_empty(e);
        nbox[child + s] = e;
        if (nn[s] > kSmallTask) {
            uint32_t q = atomicAdd(&ctr->nextTasks, 1u);
            Task nt;
            nt.node = child + s;
            nt.begin = beg[s];
            nt.end = beg[s] + nn[s];
            nt.pad = 0;
            nextTasks[q] = nt;
            nextCen[q] = e;
            tid[s] = (int)q;
        } else {
            uint32_t q = atomicAdd(&ctr->small, 1u);
            SmallTask st;
            st.node = child + s;
            st.begin = beg[s];
            st.end = beg[s] + nn[s];
            st.pad = 0;
            small[q] = st;
            tid[s] = -1;
        }
    }
    sp.leftTask = tid[0];
    sp.rightTask = tid[1];
    splits[t] = sp;
}

__device__ __forceinline__ bool goes_left(const Split& sp, const Task& tk, uint32_t i, const OBox& cb, float4 l,
                                          float4 h) {
    if (sp.axis < 0) return (i - tk.begin) < sp.nLeft;
    float lo = sp.axis == 0 ? l.x : (sp.axis == 1 ? l.y : l.z);
    float hi = sp.axis == 0 ? h.x : (sp.axis == 1 ? h.y : h.z);
    float cl = o2f(cb.lo[sp.axis]), ch = o2f(cb.hi[sp.axis]);
    return bin_of(0.5f * (lo + hi), cl, ch - cl) <= sp.bin;
}

__global__ void k_flags(uint32_t n, const uint32_t* __restrict__ ref, const int* __restrict__ taskOf,
                        const Task* __restrict__ tasks, const OBox* __restrict__ tcen, const Split* __restrict__ splits,
                        const float4* __restrict__ blo, const float4* __restrict__ bhi, uint32_t* flags) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int t = taskOf[i];
    uint32_t f = 0;
    if (t >= 0) {
        uint32_t p = ref[i];
        f = goes_left(splits[t], tasks[t], i, tcen[t], blo[p], bhi[p]) ? 1u : 0u;
    }
    flags[i] = f;
}

__global__ void k_scatter(uint32_t n, const uint32_t* __restrict__ ref, const int* __restrict__ taskOf,
                          const Task* __restrict__ tasks, const OBox* __restrict__ tcen,
                          const Split* __restrict__ splits, const float4* __restrict__ blo,
                          const float4* __restrict__ bhi, const uint32_t* __restrict__ flags,
                          const uint32_t* __restrict__ scan, uint32_t* ref2, int* taskOf2, OBox* nextCen, OBox* nbox) {
    // [side][lo xyz | hi xyz] of the two children's boxes and centroid bounds when
    // the block lies in one task (block_task); otherwise global atomics per primitive
    __shared__ uint32_t sBox[2][6], sCen[2][6];
    const int bt = block_task(n, taskOf);
    if (bt >= 0) {
        if (threadIdx.x < 24) {
            const uint32_t side = threadIdx.x / 12, k = threadIdx.x % 12;
            (k < 6 ? sBox[side][k] : sCen[side][k - 6]) = (k % 6) < 3 ? 0xffffffffu : 0u;
        }
        __syncthreads();
    }
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int t = taskOf[i];
        const uint32_t p = ref[i];
        if (t < 0) {
            ref2[i] = p;
            taskOf2[i] = -1;
        } else {
            const Task tk = tasks[t];
            const Split sp = splits[t];
            const uint32_t base = scan[tk.begin];
            const uint32_t lr = scan[i] - base;
            const bool left = flags[i] != 0;
            const uint32_t np = left ? tk.begin + lr : tk.begin + sp.nLeft + ((i - tk.begin) - lr);
            ref2[np] = p;
            const int nt = left ? sp.leftTask : sp.rightTask;
            taskOf2[np] = nt;
            const uint32_t node = sp.leftNode + (left ? 0 : 1);
            const float4 l = blo[p], h = bhi[p];
            const float lo[3] = {l.x, l.y, l.z}, hi[3] = {h.x, h.y, h.z};
            uint32_t* bx = bt >= 0 ? sBox[left ? 0 : 1] : nullptr;
            uint32_t* cx = bt >= 0 ? sCen[left ? 0 : 1] : nullptr;
            for (int k = 0; k < 3; ++k) {
                atomicMin(bx ? &bx[k] : &nbox[node].lo[k], f2o(lo[k]));
                atomicMax(bx ? &bx[3 + k] : &nbox[node].hi[k], f2o(hi[k]));
            }
            if (nt >= 0) {
                for (int k = 0; k < 3; ++k) {
                    const float c = 0.5f * (lo[k] + hi[k]);
                    atomicMin(cx ? &cx[k] : &nextCen[nt].lo[k], f2o(c));
                    atomicMax(cx ? &cx[3 + k] : &nextCen[nt].hi[k], f2o(c));
                }
            }
        }
    }
    if (bt >= 0) {
        __syncthreads();
        if (threadIdx.x < 24) {
            const uint32_t side = threadIdx.x / 12, k = threadIdx.x % 12;
            const Split sp = splits[bt];
            const bool lo = (k % 6) < 3;
            const uint32_t v = k < 6 ? sBox[side][k] : sCen[side][k - 6];
            const bool any = v != (lo ? 0xffffffffu : 0u);  // the side received a primitive
            if (any) {
                uint32_t* dst;
                if (k < 6) {
                    OBox& o = nbox[sp.leftNode + side];
                    dst = lo ? &o.lo[k % 3] : &o.hi[k % 3];
                } else {
                    const int nt = side ? sp.rightTask : sp.leftTask;
                    dst = nt >= 0 ? (lo ? &nextCen[nt].lo[k % 3] : &nextCen[nt].hi[k % 3]) : nullptr;
                }
                if (dst) {
                    if (lo) atomicMin(dst, v);
                    else atomicMax(dst, v);
                }
            }
        }
    }
}

// One thread finishes a small task: recursive SAH over sorted centroids.
__global__ void k_small(uint32_t numSmall, const SmallTask* __restrict__ small, uint32_t* ref,
                        const float4* __restrict__ blo, const float4* __restrict__ bhi, BNode* nodes, OBox* nbox,
                        BuildCtr* ctr) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= numSmall) return;
    SmallTask st = small[s];
    struct Item {
        uint32_t node, begin, end;
    };
    Item stk[2 * kSmallTask];
    int sp = 0;
    stk[sp++] = {st.node, st.begin, st.end};
    while (sp > 0) {
        Item it = stk[--sp];
        uint32_t cnt = it.end - it.begin;
        float nlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, nhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        uint32_t ids[kSmallTask];
        for (uint32_t k = 0; k < cnt; ++k) {
            ids[k] = ref[it.begin + k];
            float4 l = blo[ids[k]], h = bhi[ids[k]];
            nlo[0] = fminf(nlo[0], l.x); nlo[1] = fminf(nlo[1], l.y); nlo[2] = fminf(nlo[2], l.z);
            nhi[0] = fmaxf(nhi[0], h.x); nhi[1] = fmaxf(nhi[1], h.y); nhi[2] = fmaxf(nhi[2], h.z);
        }
        BNode nd;
        for (int k = 0; k < 3; ++k) { nd.lo[k] = nlo[k]; nd.hi[k] = nhi[k]; }
        // best split over the three sorted orders
        float bestCost = FLT_MAX;
        int bestAxis = -1;
        uint32_t bestPos = 0;
        float parentA = half_area(nlo, nhi);
        if (cnt > 1) {
            for (int a = 0; a < 3; ++a) {
                uint32_t ord[kSmallTask];
                for (uint32_t k = 0; k < cnt; ++k) ord[k] = ids[k];
                for (uint32_t k = 1; k < cnt; ++k) {  // insertion sort by centroid
                    uint32_t v = ord[k];
                    float4 l = blo[v], h = bhi[v];
                    float cv = a == 0 ? l.x + h.x : (a == 1 ? l.y + h.y : l.z + h.z);
                    int j = (int)k - 1;
                    while (j >= 0) {
                        float4 l2 = blo[ord[j]], h2 = bhi[ord[j]];
                        float cj = a == 0 ? l2.x + h2.x : (a == 1 ? l2.y + h2.y : l2.z + h2.z);
                        if (cj <= cv) break;
                        ord[j + 1] = ord[j];
                        --j;
                    }
                    ord[j + 1] = v;
                }
                float rA[kSmallTask];
                float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
                for (int k = (int)cnt - 1; k > 0; --k) {
                    float4 l = blo[ord[k]], h = bhi[ord[k]];
                    lo[0] = fminf(lo[0], l.x); lo[1] = fminf(lo[1], l.y); lo[2] = fminf(lo[2], l.z);
                    hi[0] = fmaxf(hi[0], h.x); hi[1] = fmaxf(hi[1], h.y); hi[2] = fmaxf(hi[2], h.z);
                    rA[k] = half_area(lo, hi);
                }
                for (int k = 0; k < 3; ++k) { lo[k] = FLT_MAX; hi[k] = -FLT_MAX; }
                for (uint32_t k = 0; k + 1 < cnt; ++k) {
                    float4 l = blo[ord[k]], h = bhi[ord[k]];
                    lo[0] = fminf(lo[0], l.x); lo[1] = fminf(lo[1], l.y); lo[2] = fminf(lo[2], l.z);
                    hi[0] = fmaxf(hi[0], h.x); hi[1] = fmaxf(hi[1], h.y); hi[2] = fmaxf(hi[2], h.z);
                    float cost = half_area(lo, hi) * (float)(k + 1) + rA[k + 1] * (float)(cnt - k - 1);
                    if (cost < bestCost) {
                        bestCost = cost;
                        bestAxis = a;
                        bestPos = k + 1;
                    }
                }
                if (bestAxis == a)
                    for (uint32_t k = 0; k < cnt; ++k) ref[it.begin + k] = ord[k];
            }
        }
        // leaf when small enough and the split does not pay for a traversal step,
        // priced at half a triangle test (SAH with Ct/Ci = 0.5: an 8-wide node test
        // is shared by up to eight children; showcase extension traversal ran 3.5 % faster
        // than with Ct/Ci = 1)
        bool leaf = cnt <= 1 ||
                    (cnt <= kMaxLeaf && (parentA <= 0.0f || (float)cnt * parentA <= 0.5f * parentA + bestCost));
        if (bestAxis < 0) leaf = cnt <= kMaxLeaf;
        if (leaf) {
            nd.left = it.begin;
            nd.count = cnt;
            nodes[it.node] = nd;
            continue;
        }
        if (bestAxis < 0) bestPos = cnt / 2;
        uint32_t child = atomicAdd(&ctr->nodes, 2u);
        nd.left = child;
        nd.count = 0;
        nodes[it.node] = nd;
        OBox e;
        obox_empty(e);
        nbox[child] = e;
        nbox[child + 1] = e;
        stk[sp++] = {child, it.begin, it.begin + bestPos};
        stk[sp++] = {child + 1, it.begin + bestPos, it.end};
    }
}

// Boxes of level-built nodes live in nbox (atomics); small-task nodes wrote theirs.
__global__ void k_fix_boxes(uint32_t numNodes, BNode* nodes, const OBox* __restrict__ nbox,
                            const uint8_t* __restrict__ fromLevels) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= numNodes || !fromLevels[i]) return;
    for (int k = 0; k < 3; ++k) {
        nodes[i].lo[k] = o2f(nbox[i].lo[k]);
        nodes[i].hi[k] = o2f(nbox[i].hi[k]);
    }
}

__global__ void k_mark_level_nodes(const BuildCtr* __restrict__ ctr, const Task* __restrict__ tasks,
                                   const Split* __restrict__ splits, uint8_t* fromLevels) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ctr->cur) return;
    fromLevels[tasks[t].node] = 1;
    fromLevels[splits[t].leftNode] = 1;
    fromLevels[splits[t].leftNode + 1] = 1;
}

// ---------------------------------------------------------------------------
// Collapse to 8-wide compressed nodes.
struct CItem {
    uint32_t bnode, onode;
};

__device__ __forceinline__ float node_area(const BNode& b) {
    float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    return dx * dy + dy * dz + dz * dx;
}

// One thread, before each collapse depth: last depth's new nodes become this one's items.
__global__ void k_collapse_begin(CollapseCtr* ctr) {
    ctr->cur = ctr->next;
    ctr->next = 0;
}

__global__ void k_collapse(const CItem* __restrict__ items, const BNode* __restrict__ bn,
                           const uint32_t* __restrict__ ref, const float* __restrict__ vtx,
                           const uint32_t* __restrict__ idx, const uint32_t* __restrict__ triMat, uint4* onodes,
                           float4* otris, CItem* next, CollapseCtr* ctr, uint32_t depth) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ctr->cur) return;
    CItem it = items[i];
    uint32_t kids[8];
    int n = 0;
    BNode root = bn[it.bnode];
    if (root.count > 0) {
        kids[n++] = it.bnode;
    } else {
        kids[n++] = root.left;
        kids[n++] = root.left + 1;
    }
    while (n < 8) {
        int best = -1;
        float bestA = -1.0f;
        for (int j = 0; j < n; ++j) {
            BNode b = bn[kids[j]];
            if (b.count == 0) {
                float a = node_area(b);
                if (a > bestA) { bestA = a; best = j; }
            }
        }
        if (best < 0) break;
        BNode b = bn[kids[best]];
        kids[best] = b.left;
        kids[n++] = b.left + 1;
    }
    // node box and child centroids
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    BNode kb[8];
    for (int j = 0; j < n; ++j) {
        kb[j] = bn[kids[j]];
        for (int k = 0; k < 3; ++k) { lo[k] = fminf(lo[k], kb[j].lo[k]); hi[k] = fmaxf(hi[k], kb[j].hi[k]); }
    }
    float ctr3[3] = {0.5f * (lo[0] + hi[0]), 0.5f * (lo[1] + hi[1]), 0.5f * (lo[2] + hi[2])};
    // slot s holds the child lying furthest toward corner s (bit k set = negative side of axis k)
    int slotOf[8];
    int kidIn[8];
    for (int s = 0; s < 8; ++s) kidIn[s] = -1;
    for (int j = 0; j < n; ++j) slotOf[j] = -1;
    float cost[8][8];
    for (int j = 0; j < n; ++j) {
        float c[3];
        for (int k = 0; k < 3; ++k) c[k] = 0.5f * (kb[j].lo[k] + kb[j].hi[k]) - ctr3[k];
        for (int s = 0; s < 8; ++s)
            cost[j][s] = ((s & 1) ? -c[0] : c[0]) + ((s & 2) ? -c[1] : c[1]) + ((s & 4) ? -c[2] : c[2]);
    }
    for (int round = 0; round < n; ++round) {
        float bc = -FLT_MAX;
        int bj = -1, bs = -1;
        for (int j = 0; j < n; ++j) {
            if (slotOf[j] >= 0) continue;
            for (int s = 0; s < 8; ++s)
                if (kidIn[s] < 0 && cost[j][s] > bc) { bc = cost[j][s]; bj = j; bs = s; }
        }
        slotOf[bj] = bs;
        kidIn[bs] = bj;
    }
    uint32_t imask = 0, nInternal = 0, nTris = 0;
    for (int s = 0; s < 8; ++s) {
        int j = kidIn[s];
        if (j < 0) continue;
        if (kb[j].count == 0) { imask |= 1u << s; ++nInternal; }
        else nTris += kb[j].count;
    }
    uint32_t childBase = nInternal ? atomicAdd(&ctr->nodes, nInternal) : 0;
    uint32_t triBase = nTris ? atomicAdd(&ctr->tris, nTris) : 0;
    if (nInternal) atomicMax(&ctr->maxDepth, depth + 1);
    // quantization frame: step >= 2^-20 of the coordinate magnitude
    int ex[3];
    for (int k = 0; k < 3; ++k) {
        double ext = (double)hi[k] - (double)lo[k];
        double mag = fmax(fabs((double)lo[k]), fabs((double)hi[k]));
        int e = -126;
        if (ext > 0.0) e = (int)ceil(log2(ext / 255.0));
        if (mag > 0.0) e = max(e, (int)floor(log2(mag)) - 20);
        e = max(-126, min(127, e));
        while (e < 127 && ext / ldexp(1.0, e) > 253.0) ++e;  // room for the one-step widening
        ex[k] = e;
    }
    uint8_t meta[8], qlo[3][8], qhi[3][8];
    uint32_t triOff = 0;
    for (int s = 0; s < 8; ++s) {
        int j = kidIn[s];
        meta[s] = 0;
        if (j < 0) {
            for (int k = 0; k < 3; ++k) { qlo[k][s] = 255; qhi[k][s] = 0; }
            continue;
        }
        for (int k = 0; k < 3; ++k) {
            double sc = ldexp(1.0, ex[k]);
            double ql = floor(((double)kb[j].lo[k] - (double)lo[k]) / sc) - 1.0;
            double qh = ceil(((double)kb[j].hi[k] - (double)lo[k]) / sc) + 1.0;
            qlo[k][s] = (uint8_t)fmax(0.0, fmin(255.0, ql));
            qhi[k][s] = (uint8_t)fmax(0.0, fmin(255.0, qh));
        }
        if (kb[j].count == 0) {
            uint32_t rank = __popc(imask & ((1u << s) - 1u));
            uint32_t q = atomicAdd(&ctr->next, 1u);
            next[q] = {kids[j], childBase + rank};
        } else {
            meta[s] = (uint8_t)(triOff | ((kb[j].count - 1u) << 5));
            for (uint32_t k = 0; k < kb[j].count; ++k) {
                uint32_t p = ref[kb[j].left + k];
                uint32_t i0 = idx[3 * p], i1 = idx[3 * p + 1], i2 = idx[3 * p + 2];
                float ax = vtx[3 * i0], ay = vtx[3 * i0 + 1], az = vtx[3 * i0 + 2];
                float bx = vtx[3 * i1], by = vtx[3 * i1 + 1], bz = vtx[3 * i1 + 2];
                float cx = vtx[3 * i2], cy = vtx[3 * i2 + 1], cz = vtx[3 * i2 + 2];
                float4* o = otris + 3 * (size_t)(triBase + triOff + k);
                o[0] = make_float4(ax, ay, az, __uint_as_float(p));
                o[1] = make_float4(__fsub_rn(bx, ax), __fsub_rn(by, ay), __fsub_rn(bz, az), __uint_as_float(triMat[p]));
                o[2] = make_float4(__fsub_rn(cx, ax), __fsub_rn(cy, ay), __fsub_rn(cz, az), 0.0f);
            }
            triOff += kb[j].count;
        }
    }
    auto pack4 = [](const uint8_t* b) -> uint32_t {
        return (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
    };
    uint4* o = onodes + 5 * (size_t)it.onode;
    uint32_t eb = (uint32_t)(ex[0] + 127) | ((uint32_t)(ex[1] + 127) << 8) | ((uint32_t)(ex[2] + 127) << 16) |
                  (imask << 24);
    o[0] = make_uint4(__float_as_uint(lo[0]), __float_as_uint(lo[1]), __float_as_uint(lo[2]), eb);
    o[1] = make_uint4(childBase, triBase, pack4(meta), pack4(meta + 4));
    o[2] = make_uint4(pack4(qlo[0]), pack4(qlo[0] + 4), pack4(qlo[1]), pack4(qlo[1] + 4));
    o[3] = make_uint4(pack4(qlo[2]), pack4(qlo[2] + 4), pack4(qhi[0]), pack4(qhi[0] + 4));
    o[4] = make_uint4(pack4(qhi[1]), pack4(qhi[1] + 4), pack4(qhi[2]), pack4(qhi[2] + 4));
}

inline unsigned grid_for(uint64_t n, unsigned b) { return (unsigned)((n + b - 1) / b); }

// SAH cost of the 8-wide tree: one node test for the root plus, for every child
// box, its surface area over the root's times the work a ray entering it does
// (one node test, or the leaf's triangle tests).  One thread per node decodes the
// node's quantized child boxes; sums[0] += area x work, sums[1] = the root's area
// (the union of its children).
__global__ void k_sah(const uint4* __restrict__ nodes, uint32_t numNodes, double* sums) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= numNodes) return;
    const uint4* n = nodes + 5 * (size_t)i;
    const uint4 n0 = n[0], n1 = n[1], n2 = n[2], n3 = n[3], n4 = n[4];
    const float p[3] = {__uint_as_float(n0.x), __uint_as_float(n0.y), __uint_as_float(n0.z)};
    float sc[3];
    for (int a = 0; a < 3; ++a) sc[a] = ldexpf(1.0f, (int)((n0.w >> (8 * a)) & 0xffu) - 127);
    const uint32_t imask = n0.w >> 24;
    const uint32_t qlo[3][2] = {{n2.x, n2.y}, {n2.z, n2.w}, {n3.x, n3.y}};
    const uint32_t qhi[3][2] = {{n3.z, n3.w}, {n4.x, n4.y}, {n4.z, n4.w}};
    float ulo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, uhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    double acc = 0.0;
    for (int s = 0; s < 8; ++s) {
        float lo[3], hi[3];
        bool empty = false;
        for (int a = 0; a < 3; ++a) {
            const uint32_t bl = (qlo[a][s >> 2] >> (8 * (s & 3))) & 0xffu, bh = (qhi[a][s >> 2] >> (8 * (s & 3))) & 0xffu;
            if (bl > bh) empty = true;
            lo[a] = p[a] + (float)bl * sc[a];
            hi[a] = p[a] + (float)bh * sc[a];
        }
        if (empty) continue;
        const uint32_t meta = ((s < 4 ? n1.z : n1.w) >> (8 * (s & 3))) & 0xffu;
        const double work = ((imask >> s) & 1u) ? 1.0 : (double)((meta >> 5) + 1u);
        acc += (double)half_area(lo, hi) * work;
        for (int a = 0; a < 3; ++a) { ulo[a] = fminf(ulo[a], lo[a]); uhi[a] = fmaxf(uhi[a], hi[a]); }
    }
    atomicAdd(&sums[0], acc);
    if (i == 0) sums[1] = (double)half_area(ulo, uhi);
}

}  // namespace

// The build's scratch (primitive references, tasks, bins, the binary tree, ...: a few
// hundred MB for a 2.4M-triangle scene) comes from a stream-ordered memory pool of
// the library's own, one per device, that keeps its memory between builds: no
// cudaMalloc / cudaFree in the build, and a scene built after another reuses the
// same memory.  The finished tree (nodes, triangle records) is allocated with
// cudaMalloc, as it lives with the scene.
cudaError_t scratch_pool(cudaMemPool_t* out) {
    static std::mutex m;
    static cudaMemPool_t pools[64] = {nullptr};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(m);
    if (!pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        if ((e = cudaMemPoolCreate(&p, &props)) != cudaSuccess) return e;
        unsigned long long keep = ~0ull;  // never hand memory back at synchronisation
        if ((e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) return e;
        pools[dev] = p;
    }
    *out = pools[dev];
    return cudaSuccess;
}

template <class T>
cudaError_t scratch_alloc(T** p, cudaMemPool_t pool, cudaStream_t st, size_t bytes) {
    return cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), bytes, pool, st);
}

#define WRK_BCHECK(x)                                                                               \
    do {                                                                                            \
        cudaError_t e_ = (x);                                                                       \
        if (e_ != cudaSuccess) {                                                                    \
            snprintf(err, errlen, "BVH build: %s at %s:%d", cudaGetErrorString(e_), __FILE__, __LINE__); \
            goto fail;                                                                              \
        }                                                                                           \
    } while (0)

int build_bvh8(const float* d_vtx, const uint32_t* d_idx, const uint32_t* d_triMat, uint32_t n, cudaStream_t st,
               BvhBuildResult* out, char* err, size_t errlen) {
    // scratch
    float4 *blo = nullptr, *bhi = nullptr;
    uint32_t *ref = nullptr, *ref2 = nullptr, *flags = nullptr, *scan = nullptr;
    int *taskOf = nullptr, *taskOf2 = nullptr;
    Task *tasks = nullptr, *ntasks = nullptr;
    OBox *tcen = nullptr, *ncen = nullptr, *nbox = nullptr;
    Bin* bins = nullptr;
    Split* splits = nullptr;
    SmallTask* small = nullptr;
    BNode* nodes = nullptr;
    BuildCtr* ctr = nullptr;
    uint8_t* fromLevels = nullptr;
    void* cubTmp = nullptr;
    size_t cubBytes = 0;
    CItem *items = nullptr, *items2 = nullptr;
    CollapseCtr* cctr = nullptr;
    uint4* onodes = nullptr;
    float4* otris = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BuildCtr hc{};
    uint32_t numTasks = 1, numBinary = 0, smallCount = 0;
    uint32_t maxTasks = n / (kSmallTask + 1) + 2;
    uint32_t maxNodes = 2 * n + 1;
    int rc = WRK_ERR_CUDA;
    std::vector<uint32_t> iota;

    cudaMemPool_t pool = nullptr;
    WRK_BCHECK(scratch_pool(&pool));
    WRK_BCHECK(cudaEventCreate(&e0));
    WRK_BCHECK(cudaEventCreate(&e1));
    WRK_BCHECK(cudaEventRecord(e0, st));
    WRK_BCHECK(scratch_alloc(&blo, pool, st, sizeof(float4) * n));
    WRK_BCHECK(scratch_alloc(&bhi, pool, st, sizeof(float4) * n));
    WRK_BCHECK(scratch_alloc(&ref, pool, st, sizeof(uint32_t) * n));
    WRK_BCHECK(scratch_alloc(&ref2, pool, st, sizeof(uint32_t) * n));
    WRK_BCHECK(scratch_alloc(&flags, pool, st, sizeof(uint32_t) * n));
    WRK_BCHECK(scratch_alloc(&scan, pool, st, sizeof(uint32_t) * std::max<uint32_t>(n, 4u)));  // also the SAH sums (2 doubles)
    WRK_BCHECK(scratch_alloc(&taskOf, pool, st, sizeof(int) * n));
    WRK_BCHECK(scratch_alloc(&taskOf2, pool, st, sizeof(int) * n));
    WRK_BCHECK(scratch_alloc(&tasks, pool, st, sizeof(Task) * maxTasks));
    WRK_BCHECK(scratch_alloc(&ntasks, pool, st, sizeof(Task) * maxTasks));
    WRK_BCHECK(scratch_alloc(&tcen, pool, st, sizeof(OBox) * maxTasks));
    WRK_BCHECK(scratch_alloc(&ncen, pool, st, sizeof(OBox) * maxTasks));
    WRK_BCHECK(scratch_alloc(&bins, pool, st, sizeof(Bin) * 3 * kBins * (size_t)maxTasks));
    WRK_BCHECK(scratch_alloc(&splits, pool, st, sizeof(Split) * maxTasks));
    WRK_BCHECK(scratch_alloc(&small, pool, st, sizeof(SmallTask) * (size_t)(n + 1)));
    WRK_BCHECK(scratch_alloc(&nodes, pool, st, sizeof(BNode) * maxNodes));
    WRK_BCHECK(scratch_alloc(&nbox, pool, st, sizeof(OBox) * maxNodes));
    WRK_BCHECK(scratch_alloc(&fromLevels, pool, st, maxNodes));
    WRK_BCHECK(scratch_alloc(&ctr, pool, st, sizeof(BuildCtr)));
    WRK_BCHECK(cudaMemsetAsync(fromLevels, 0, maxNodes, st));
    WRK_BCHECK(cudaMemsetAsync(ctr, 0, sizeof(BuildCtr), st));
    WRK_BCHECK(cub::DeviceScan::ExclusiveSum(nullptr, cubBytes, flags, scan, (int)n, st));
    WRK_BCHECK(scratch_alloc(&cubTmp, pool, st, cubBytes));

    iota.resize(n);
    for (uint32_t i = 0; i < n; ++i) iota[i] = i;
    WRK_BCHECK(cudaMemcpyAsync(ref, iota.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st));
    WRK_BCHECK(cudaMemsetAsync(taskOf, 0, sizeof(int) * n, st));
    {
        OBox e;
        for (int k = 0; k < 3; ++k) { e.lo[k] = f2o(FLT_MAX); e.hi[k] = f2o(-FLT_MAX); }
        WRK_BCHECK(cudaMemcpyAsync(nbox, &e, sizeof(OBox), cudaMemcpyHostToDevice, st));
        WRK_BCHECK(cudaMemcpyAsync(tcen, &e, sizeof(OBox), cudaMemcpyHostToDevice, st));
        Task root{0, 0, n, 0};
        WRK_BCHECK(cudaMemcpyAsync(tasks, &root, sizeof(Task), cudaMemcpyHostToDevice, st));
        BuildCtr c0{1, 1, 0, 0};  // the root task is the first level's one task
        WRK_BCHECK(cudaMemcpyAsync(ctr, &c0, sizeof(BuildCtr), cudaMemcpyHostToDevice, st));
    }
    k_prim_bounds<<<grid_for(n, 256), 256, 0, st>>>(d_vtx, d_idx, n, blo, bhi, nbox, tcen);
    WRK_BCHECK(cudaGetLastError());
    if (n <= kSmallTask) {
        SmallTask s0{0, 0, n, 0};
        WRK_BCHECK(cudaMemcpyAsync(small, &s0, sizeof(SmallTask), cudaMemcpyHostToDevice, st));
        BuildCtr c1{1, 0, 1, 0};
        WRK_BCHECK(cudaMemcpyAsync(ctr, &c1, sizeof(BuildCtr), cudaMemcpyHostToDevice, st));
        uint8_t one = 1;
        WRK_BCHECK(cudaMemcpyAsync(fromLevels, &one, 1, cudaMemcpyHostToDevice, st));
        numTasks = 0;
    }
    // Levels run kLevelsPerSync at a time without a host round trip: the device keeps
    // each level's task count (k_level_begin) and the kernels read it there; the host
    // sizes grids for an upper bound (a task opens at most two child tasks) and reads
    // the count back only between batches.  A level with no open task passes every
    // primitive through unchanged, so the batch may overshoot the last level.
    for (uint32_t bound = numTasks, levels = 0; numTasks > 0;) {
        for (int k = 0; k < kLevelsPerSync; ++k, ++levels) {
            k_level_begin<<<1, 1, 0, st>>>(ctr);
            k_init_bins<<<grid_for(bound * 3 * kBins, 256), 256, 0, st>>>(bins, ctr);
            k_bin<<<grid_for(n, 256), 256, 0, st>>>(n, ref, taskOf, tcen, blo, bhi, bins);
            k_split<<<grid_for(bound, 128), 128, 0, st>>>(tasks, bins, splits, ntasks, ncen, small, nodes, nbox, ctr);
            k_mark_level_nodes<<<grid_for(bound, 128), 128, 0, st>>>(ctr, tasks, splits, fromLevels);
            k_flags<<<grid_for(n, 256), 256, 0, st>>>(n, ref, taskOf, tasks, tcen, splits, blo, bhi, flags);
            WRK_BCHECK(cub::DeviceScan::ExclusiveSum(cubTmp, cubBytes, flags, scan, (int)n, st));
            k_scatter<<<grid_for(n, 256), 256, 0, st>>>(n, ref, taskOf, tasks, tcen, splits, blo, bhi, flags, scan,
                                                         ref2, taskOf2, ncen, nbox);
            WRK_BCHECK(cudaGetLastError());
            std::swap(ref, ref2);
            std::swap(taskOf, taskOf2);
            std::swap(tasks, ntasks);
            std::swap(tcen, ncen);
            bound = std::min(maxTasks, 2 * bound);
        }
        WRK_BCHECK(cudaMemcpyAsync(&hc, ctr, sizeof(BuildCtr), cudaMemcpyDeviceToHost, st));
        WRK_BCHECK(cudaStreamSynchronize(st));
        numTasks = hc.nextTasks;
        bound = numTasks;
        if (numTasks > maxTasks || levels > kMaxLevels) {
            snprintf(err, errlen, "BVH build: task overflow or level limit (%u tasks, %u levels)", numTasks, levels);
            rc = WRK_ERR_DEVICE;
            goto fail;
        }
    }
    WRK_BCHECK(cudaMemcpyAsync(&hc, ctr, sizeof(BuildCtr), cudaMemcpyDeviceToHost, st));
    WRK_BCHECK(cudaStreamSynchronize(st));
    smallCount = hc.small;
    k_fix_boxes<<<grid_for(hc.nodes, 256), 256, 0, st>>>(hc.nodes, nodes, nbox, fromLevels);
    if (smallCount) k_small<<<grid_for(smallCount, 64), 64, 0, st>>>(smallCount, small, ref, blo, bhi, nodes, nbox, ctr);
    WRK_BCHECK(cudaGetLastError());
    WRK_BCHECK(cudaMemcpyAsync(&hc, ctr, sizeof(BuildCtr), cudaMemcpyDeviceToHost, st));
    WRK_BCHECK(cudaStreamSynchronize(st));
    numBinary = hc.nodes;

    // ---- collapse ----
    WRK_BCHECK(scratch_alloc(&items, pool, st, sizeof(CItem) * numBinary));
    WRK_BCHECK(scratch_alloc(&items2, pool, st, sizeof(CItem) * numBinary));
    WRK_BCHECK(scratch_alloc(&cctr, pool, st, sizeof(CollapseCtr)));
    WRK_BCHECK(cudaMalloc(&onodes, sizeof(uint4) * 5 * (size_t)numBinary));
    WRK_BCHECK(cudaMalloc(&otris, sizeof(float4) * 3 * (size_t)n));
    {
        CItem r{0, 0};
        WRK_BCHECK(cudaMemcpyAsync(items, &r, sizeof(CItem), cudaMemcpyHostToDevice, st));
        CollapseCtr c0{1, 0, 1, 1, 0};  // the root item is the first depth's one item
        WRK_BCHECK(cudaMemcpyAsync(cctr, &c0, sizeof(CollapseCtr), cudaMemcpyHostToDevice, st));
    }
    {
        // as the binary levels: the item count stays on the device, read back every
        // kLevelsPerSync depths; an 8-wide node opens at most 8 items
        uint32_t cnt = 1, depth = 1;
        CollapseCtr hcc{};
        while (cnt > 0) {
            uint32_t bound = cnt;
            for (int k = 0; k < kLevelsPerSync; ++k) {
                k_collapse_begin<<<1, 1, 0, st>>>(cctr);
                k_collapse<<<grid_for(bound, 64), 64, 0, st>>>(items, nodes, ref, d_vtx, d_idx, d_triMat, onodes,
                                                               otris, items2, cctr, depth);
                WRK_BCHECK(cudaGetLastError());
                std::swap(items, items2);
                ++depth;
                bound = std::min(numBinary, 8 * bound);
            }
            WRK_BCHECK(cudaMemcpyAsync(&hcc, cctr, sizeof(CollapseCtr), cudaMemcpyDeviceToHost, st));
            WRK_BCHECK(cudaStreamSynchronize(st));
            cnt = hcc.next;
            if (depth > 256) {
                snprintf(err, errlen, "BVH collapse: depth limit exceeded");
                rc = WRK_ERR_DEVICE;
                goto fail;
            }
        }
        WRK_BCHECK(cudaEventRecord(e1, st));
        // SAH cost of the finished tree (outside the timed build)
        double hs[2] = {0.0, 0.0};
        WRK_BCHECK(cudaMemsetAsync(scan, 0, 2 * sizeof(double), st));
        if (hcc.nodes) k_sah<<<grid_for(hcc.nodes, 256), 256, 0, st>>>(onodes, hcc.nodes, (double*)scan);
        WRK_BCHECK(cudaGetLastError());
        WRK_BCHECK(cudaMemcpyAsync(hs, scan, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
        WRK_BCHECK(cudaStreamSynchronize(st));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (hcc.tris != n) {
            snprintf(err, errlen, "BVH collapse: %u triangles emitted, expected %u", hcc.tris, n);
            rc = WRK_ERR_DEVICE;
            goto fail;
        }
        out->nodes = onodes;
        out->tris = otris;
        out->numNodes = hcc.nodes;
        out->numBinary = numBinary;
        out->depth = hcc.maxDepth;
        out->ms = ms;
        out->sah = hs[1] > 0.0 ? (float)(1.0 + hs[0] / hs[1]) : 0.0f;
        onodes = nullptr;
        otris = nullptr;
        rc = WRK_OK;
    }
fail:
    for (void* p : {(void*)blo, (void*)bhi, (void*)ref, (void*)ref2, (void*)flags, (void*)scan, (void*)taskOf,
                    (void*)taskOf2, (void*)tasks, (void*)ntasks, (void*)tcen, (void*)ncen, (void*)bins, (void*)splits,
                    (void*)small, (void*)nodes, (void*)nbox, (void*)fromLevels, (void*)ctr, cubTmp, (void*)items,
                    (void*)items2, (void*)cctr})
        if (p) cudaFreeAsync(p, st);
    cudaFree(onodes);
    cudaFree(otris);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return rc;
}

}  // namespace wrk
