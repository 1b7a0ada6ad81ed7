// The scene build on the GPU: the steps of lambda_host::BuildAccel, each giving the
// host loop's results float for float and byte for byte.
//
//  - Instance bounds (Instance::min/max/center, src/scene/instance.h:54-101): one
//    block per instance transforms every object's eight box corners and takes the
//    per-axis minimum and maximum, then sums the transformed object centres in
//    object order.
//  - The binned-SAH build (BVH::buildRecursive, src/scene/bvh.h:111-246): level by
//    level, every node of a level at once. Per node: bounds of its items, 16
//    centroid bins per axis, the SAH sweep, the split or leaf decision, then the
//    partition. A final pass numbers the nodes in the depth-first order the host
//    recursion writes them.
//
// Reductions follow the host's std::fmin/std::fmax exactly. Those keep their first
// argument when the two compare equal (+0 against -0), so a running minimum keeps
// the first of several equal values in sequence order and ignores NaN. Here every
// minimum or maximum is a 64-bit atomic on a key (order-preserving float bits, with
// -0 and +0 mapped together, then the sequence index), which picks the same
// element; its exact bits are then read back from that element. The partition
// reproduces std::partition's swaps (libstdc++'s bidirectional form: the k-th
// element that fails the predicate, from the left, trades places with the k-th
// element that passes it, from the right) with prefix sums.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "engine.h"
#include "lambda_gpu.h"
#include "scene.h"

namespace {

constexpr float kEps = 1e-4f;   // constants.h:5
constexpr float kBig = 1e30f;   // constants.h:16
constexpr int kBinN = 16;       // constants.h:9
constexpr int kDepthCap = 20;   // constants.h:10

struct F3 {
    float x, y, z;
};

__device__ __forceinline__ float comp(const F3 &v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// std::fmin / std::fmax as the host's C library computes them: the first argument
// when they compare equal, the other when one is NaN.
__device__ __forceinline__ float lib_fmin(float a, float b) { return (isnan(b) || a <= b) ? a : b; }
__device__ __forceinline__ float lib_fmax(float a, float b) { return (isnan(b) || a >= b) ? a : b; }
__device__ __forceinline__ F3 vmin3(const F3 &a, const F3 &b) {
    return F3{lib_fmin(a.x, b.x), lib_fmin(a.y, b.y), lib_fmin(a.z, b.z)};
}
__device__ __forceinline__ F3 vmax3(const F3 &a, const F3 &b) {
    return F3{lib_fmax(a.x, b.x), lib_fmax(a.y, b.y), lib_fmax(a.z, b.z)};
}
__device__ __forceinline__ F3 add3(const F3 &a, const F3 &b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 sub3(const F3 &a, const F3 &b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }

// Float bits ordered as unsigned integers, -0 and +0 alike.
__device__ __forceinline__ uint32_t order_bits(float f) {
    uint32_t b = __float_as_uint(f);
    if ((b << 1) == 0) b = 0;
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
// Key of value v at sequence index i: the smallest key is the smallest value, and of
// equal values the first.
__device__ __forceinline__ unsigned long long min_key(float v, uint32_t i) {
    return (static_cast<unsigned long long>(order_bits(v)) << 32) | i;
}
// The largest key is the largest value, and of equal values the first.
__device__ __forceinline__ unsigned long long max_key(float v, uint32_t i) {
    return (static_cast<unsigned long long>(order_bits(v)) << 32) | (0xFFFFFFFFu - i);
}
constexpr unsigned long long kNoMin = ~0ull, kNoMax = 0ull;
__device__ __forceinline__ uint32_t min_index(unsigned long long k) { return uint32_t(k); }
__device__ __forceinline__ uint32_t max_index(unsigned long long k) { return 0xFFFFFFFFu - uint32_t(k); }

// --- Object and instance geometry (object.h:166-176, utils.h:89-95) -----------

struct ObjG {
    int type;
    F3 c, h, v;
    float r;
};

__device__ __forceinline__ ObjG load_obj(const lambda_object &o) {
    ObjG g;
    g.type = o.type;
    g.c = F3{o.g[0], o.g[1], o.g[2]};
    g.h = F3{o.g[3], o.g[4], o.g[5]};
    g.v = F3{o.g[6], o.g[7], o.g[8]};
    g.r = o.g[3];
    return g;
}

__device__ __forceinline__ F3 obj_min(const ObjG &g) {
    const F3 e{kEps, kEps, kEps};
    if (g.type == LAMBDA_OBJECT_SPHERE) return sub3(g.c, F3{g.r, g.r, g.r});
    if (g.type == LAMBDA_OBJECT_QUAD)
        return sub3(vmin3(g.c, vmin3(add3(g.c, g.h), vmin3(add3(g.c, g.v), add3(add3(g.c, g.h), g.v)))), e);
    return sub3(vmin3(g.c, vmin3(add3(g.c, g.h), add3(g.c, g.v))), e);
}

__device__ __forceinline__ F3 obj_max(const ObjG &g) {
    const F3 e{kEps, kEps, kEps};
    if (g.type == LAMBDA_OBJECT_SPHERE) return add3(g.c, F3{g.r, g.r, g.r});
    if (g.type == LAMBDA_OBJECT_QUAD)
        return add3(vmax3(g.c, vmax3(add3(g.c, g.h), vmax3(add3(g.c, g.v), add3(add3(g.c, g.h), g.v)))), e);
    return add3(vmax3(g.c, vmax3(add3(g.c, g.h), add3(g.c, g.v))), e);
}

__device__ __forceinline__ F3 obj_center(const ObjG &g) {
    if (g.type == LAMBDA_OBJECT_SPHERE) return g.c;
    if (g.type == LAMBDA_OBJECT_QUAD) {
        const F3 a{0.5f * g.h.x, 0.5f * g.h.y, 0.5f * g.h.z}, b{0.5f * g.v.x, 0.5f * g.v.y, 0.5f * g.v.z};
        return add3(add3(g.c, a), b);
    }
    const F3 s = add3(g.h, g.v);
    return add3(g.c, F3{s.x / 3.0f, s.y / 3.0f, s.z / 3.0f});
}

// Point transform with projective divide (utils.h:89-95), w = 1.
__device__ __forceinline__ F3 xform_point(const float *m, const F3 &p) {
    float den = m[12] * p.x + m[13] * p.y + m[14] * p.z + m[15] * 1.0f;
    if (fabsf(den) < kEps) den = 1;
    const float x = m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3] * 1.0f;
    const float y = m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7] * 1.0f;
    const float z = m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11] * 1.0f;
    return F3{x / den, y / den, z / den};
}

// Corner k of the box (a, c), in the host's order: a, c, (a a c), (a c a), (a c c),
// (c a a), (c a c), (c c a).
__device__ __forceinline__ F3 box_corner(const F3 &a, const F3 &c, int k) {
    switch (k) {
        case 0: return a;
        case 1: return c;
        case 2: return F3{a.x, a.y, c.z};
        case 3: return F3{a.x, c.y, a.z};
        case 4: return F3{a.x, c.y, c.z};
        case 5: return F3{c.x, a.y, a.z};
        case 6: return F3{c.x, a.y, c.z};
        default: return F3{c.x, c.y, a.z};
    }
}

__device__ __forceinline__ F3 instance_corner(const lambda_instance &in, const lambda_object *objs, uint32_t seq) {
    const ObjG g = load_obj(objs[in.object + int(seq >> 3)]);
    return xform_point(in.transform, box_corner(obj_min(g), obj_max(g), int(seq & 7)));
}

// Warp then block reduction of a key (min when kMin, else max); the result is valid in thread 0.
template <bool kMin>
__device__ __forceinline__ unsigned long long block_reduce(unsigned long long k, unsigned long long *scratch) {
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long v = __shfl_down_sync(0xffffffffu, k, o);
        k = kMin ? (v < k ? v : k) : (v > k ? v : k);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) scratch[warp] = k;
    __syncthreads();
    if (warp == 0) {
        k = lane < int(blockDim.x >> 5) ? scratch[lane] : (kMin ? kNoMin : kNoMax);
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long v = __shfl_down_sync(0xffffffffu, k, o);
            k = kMin ? (v < k ? v : k) : (v > k ? v : k);
        }
    }
    return k;
}

constexpr int kBoundsThreads = 256;
constexpr int kCenterChunk = 1024;

// One block per instance: out9[i] = lo xyz, hi xyz, centroid xyz.
__global__ void __launch_bounds__(kBoundsThreads) k_instance_bounds(const lambda_object *__restrict__ objs,
                                                                     const lambda_instance *__restrict__ insts,
                                                                     int n_inst, float *__restrict__ out9) {
    __shared__ unsigned long long scratch[kBoundsThreads / 32];
    __shared__ F3 centers[kCenterChunk];
    __shared__ unsigned long long win[6];
    for (int i = blockIdx.x; i < n_inst; i += gridDim.x) {
        const lambda_instance in = insts[i];
        unsigned long long lo[3] = {kNoMin, kNoMin, kNoMin}, hi[3] = {kNoMax, kNoMax, kNoMax};
        const uint32_t n_corner = uint32_t(in.count) * 8u;
        for (uint32_t s = threadIdx.x; s < n_corner; s += blockDim.x) {
            const F3 w = instance_corner(in, objs, s);
            for (int a = 0; a < 3; a++) {
                const float v = comp(w, a);
                if (isnan(v)) continue;
                const unsigned long long kl = min_key(v, s), kh = max_key(v, s);
                lo[a] = kl < lo[a] ? kl : lo[a];
                hi[a] = kh > hi[a] ? kh : hi[a];
            }
        }
        for (int a = 0; a < 3; a++) {
            const unsigned long long l = block_reduce<true>(lo[a], scratch);
            if (threadIdx.x == 0) win[a] = l;
            const unsigned long long h = block_reduce<false>(hi[a], scratch);
            if (threadIdx.x == 0) win[3 + a] = h;
        }
        // the centroid: the transformed centres summed in object order, a chunk at a time
        F3 sum{0, 0, 0};
        for (int base = 0; base < in.count; base += kCenterChunk) {
            __syncthreads();
            for (int j = threadIdx.x; j < kCenterChunk && base + j < in.count; j += blockDim.x)
                centers[j] = xform_point(in.transform, obj_center(load_obj(objs[in.object + base + j])));
            __syncthreads();
            if (threadIdx.x == 0) {
                const int n = min(kCenterChunk, in.count - base);
                for (int j = 0; j < n; j++) sum = add3(sum, centers[j]);
            }
        }
        if (threadIdx.x == 0) {
            float *o = out9 + size_t(i) * 9;
            for (int a = 0; a < 3; a++) {
                // fmin(kMax, ...) in sequence: the initial kMax wins ties and beats larger values
                float v = kBig;
                if (win[a] != kNoMin) {
                    const float w = comp(instance_corner(in, objs, min_index(win[a])), a);
                    if (w < kBig) v = w;
                }
                o[a] = v;
                float u = -kBig;
                if (win[3 + a] != kNoMax) {
                    const float w = comp(instance_corner(in, objs, max_index(win[3 + a])), a);
                    if (w > -kBig) u = w;
                }
                o[3 + a] = u;
            }
            const float n = float(in.count);
            o[6] = sum.x / n;
            o[7] = sum.y / n;
            o[8] = sum.z / n;
        }
        __syncthreads();
    }
}

// --- Binned-SAH build ------------------------------------------------------------

// Per-task key slots: lo xyz, hi xyz, centroid lo xyz, centroid hi xyz.
constexpr int kTaskKeys = 12;
// Per-task, per-axis, per-bin slots: lo xyz, hi xyz keys, then the count.
constexpr int kBinKeys = 6;

struct Task {
    int start, end, depth, rec;
};

// What the build knows about each node (task) once its level is done.
struct Rec {
    float lo[3], hi[3];
    int start, count;   // the item range; a leaf keeps it
    int left, right;    // child records, -1 for a leaf
    int level;
};

struct Split {
    int axis;       // -1: leaf
    float plane;
};

__device__ __forceinline__ const float *item(const float *items, int id) { return items + size_t(id) * 9; }

// Task of each position of the level's ranges (tasks sorted by start), -1 outside.
__global__ void k_assign(const Task *tasks, int n_tasks, int lo_pos, int hi_pos, int *pos_task) {
    const int p = lo_pos + blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= hi_pos) return;
    int a = 0, b = n_tasks - 1, t = -1;
    while (a <= b) {
        const int m = (a + b) >> 1;
        if (tasks[m].start <= p) {
            t = m;
            a = m + 1;
        } else {
            b = m - 1;
        }
    }
    pos_task[p - lo_pos] = (t >= 0 && p < tasks[t].end) ? t : -1;
}

__global__ void k_init_keys(unsigned long long *keys, int n_tasks) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_tasks * kTaskKeys) return;
    keys[i] = (i % kTaskKeys) % 6 < 3 ? kNoMin : kNoMax;
}

// Item bounds and centroid bounds of every task: one position per thread, with the
// keys of a warp whose positions share one task combined before the atomics.
__global__ void k_task_bounds(const float *items, const int *order, const int *pos_task, int lo_pos, int hi_pos,
                              unsigned long long *keys) {
    const int p = lo_pos + blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = p < hi_pos;
    const int t = in ? pos_task[p - lo_pos] : -1;
    const float *it = (t >= 0) ? item(items, order[p]) : nullptr;
    const int t0 = __shfl_sync(0xffffffffu, t, 0);
    const bool uniform = __all_sync(0xffffffffu, t == t0) && t0 >= 0;
    for (int s = 0; s < kTaskKeys; s++) {
        // slots 0-2 min of the item lo, 3-5 max of its hi, 6-8 min and 9-11 max of its centroid
        const bool is_min = (s % 6) < 3;
        const int src = s < 6 ? s : 6 + (s % 3);
        unsigned long long k = is_min ? kNoMin : kNoMax;
        if (it) {
            const float v = it[src];
            if (!isnan(v)) k = is_min ? min_key(v, uint32_t(p)) : max_key(v, uint32_t(p));
        }
        if (uniform) {
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long w = __shfl_down_sync(0xffffffffu, k, o);
                k = is_min ? (w < k ? w : k) : (w > k ? w : k);
            }
            if ((threadIdx.x & 31) == 0 && k != (is_min ? kNoMin : kNoMax)) {
                if (is_min) atomicMin(&keys[size_t(t0) * kTaskKeys + s], k);
                else atomicMax(&keys[size_t(t0) * kTaskKeys + s], k);
            }
        } else if (t >= 0 && k != (is_min ? kNoMin : kNoMax)) {
            if (is_min) atomicMin(&keys[size_t(t) * kTaskKeys + s], k);
            else atomicMax(&keys[size_t(t) * kTaskKeys + s], k);
        }
    }
}

// The value a key picked: the winning item's own float (its exact bits), clamped as
// fmin(kMax, ...) / fmax(-kMax, ...) in sequence are.
__device__ __forceinline__ float key_value(const float *items, const int *order, unsigned long long k, int field,
                                           bool is_min) {
    if (is_min) {
        if (k == kNoMin) return kBig;
        const float v = item(items, order[min_index(k)])[field];
        return v < kBig ? v : kBig;
    }
    if (k == kNoMax) return -kBig;
    const float v = item(items, order[max_index(k)])[field];
    return v > -kBig ? v : -kBig;
}

struct TaskBox {
    float lo[3], hi[3], clo[3], chi[3];
};

// Decodes each task's bounds and clears its bins.
__global__ void k_task_decode(const float *items, const int *order, const unsigned long long *keys, int n_tasks,
                              TaskBox *boxes, unsigned long long *bin_keys, int *bin_n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tasks) return;
    TaskBox b;
    const unsigned long long *k = keys + size_t(t) * kTaskKeys;
    for (int a = 0; a < 3; a++) {
        b.lo[a] = key_value(items, order, k[a], a, true);
        b.hi[a] = key_value(items, order, k[3 + a], 3 + a, false);
        b.clo[a] = key_value(items, order, k[6 + a], 6 + a, true);
        b.chi[a] = key_value(items, order, k[9 + a], 6 + a, false);
    }
    boxes[t] = b;
    for (int i = 0; i < 3 * kBinN; i++) {
        unsigned long long *bk = bin_keys + (size_t(t) * 3 * kBinN + i) * kBinKeys;
        for (int j = 0; j < kBinKeys; j++) bk[j] = j < 3 ? kNoMin : kNoMax;
        bin_n[size_t(t) * 3 * kBinN + i] = 0;
    }
}

// int(x) as the host's x86 conversion gives it: out-of-range and NaN become INT_MIN.
__device__ __forceinline__ int host_int(float x) {
    return (x >= -2147483648.0f && x < 2147483648.0f) ? int(x) : INT_MIN;
}

__device__ __forceinline__ int bin_of(float c, float clo, float extent) {
    const int b = host_int(float(kBinN) * (c - clo) / extent);
    return b < 0 ? 0 : (b > kBinN - 1 ? kBinN - 1 : b);
}

// Bins of every task: per position and axis (with extent >= 1e-4), the item's box
// into its centroid bin.
__global__ void k_task_bins(const float *items, const int *order, const int *pos_task, int lo_pos, int hi_pos,
                            const TaskBox *boxes, unsigned long long *bin_keys, int *bin_n) {
    const int p = lo_pos + blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= hi_pos) return;
    const int t = pos_task[p - lo_pos];
    if (t < 0) return;
    const TaskBox &b = boxes[t];
    const float *it = item(items, order[p]);
    for (int a = 0; a < 3; a++) {
        const float extent = b.chi[a] - b.clo[a];
        if (!(extent >= kEps)) continue;
        const int bin = bin_of(it[6 + a], b.clo[a], extent);
        const size_t slot = size_t(t) * 3 * kBinN + size_t(a) * kBinN + size_t(bin);
        unsigned long long *bk = bin_keys + slot * kBinKeys;
        for (int j = 0; j < 3; j++) {
            const float l = it[j], h = it[3 + j];
            if (!isnan(l)) atomicMin(&bk[j], min_key(l, uint32_t(p)));
            if (!isnan(h)) atomicMax(&bk[3 + j], max_key(h, uint32_t(p)));
        }
        atomicAdd(&bin_n[slot], 1);
    }
}

__device__ __forceinline__ float half_area3(const F3 &e) { return 2 * (e.x * e.y + e.x * e.z + e.y * e.z); }

// The SAH sweep and the leaf-or-split decision of every task (bvh.h:111-246).
__global__ void k_task_split(const float *items, const int *order, const Task *tasks, int n_tasks,
                             const TaskBox *boxes, const unsigned long long *bin_keys, const int *bin_n,
                             Split *splits) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tasks) return;
    const TaskBox &b = boxes[t];
    const Task tk = tasks[t];
    float best_cost = kBig;
    int best_axis = 0, best_split = -1;
    for (int a = 0; a < 3; a++) {
        const float extent = b.chi[a] - b.clo[a];
        if (!(extent >= kEps)) continue;
        F3 blo[kBinN], bhi[kBinN];
        int bn[kBinN];
        for (int j = 0; j < kBinN; j++) {
            const size_t slot = size_t(t) * 3 * kBinN + size_t(a) * kBinN + size_t(j);
            const unsigned long long *bk = bin_keys + slot * kBinKeys;
            blo[j] = F3{key_value(items, order, bk[0], 0, true), key_value(items, order, bk[1], 1, true),
                        key_value(items, order, bk[2], 2, true)};
            bhi[j] = F3{key_value(items, order, bk[3], 3, false), key_value(items, order, bk[4], 4, false),
                        key_value(items, order, bk[5], 5, false)};
            bn[j] = bin_n[slot];
        }
        F3 llo[kBinN], lhi[kBinN], rlo_[kBinN], rhi_[kBinN];
        int ln[kBinN], rn_[kBinN];
        F3 rlo{kBig, kBig, kBig}, rhi{-kBig, -kBig, -kBig};
        int rn = 0;
        for (int j = 0; j < kBinN; j++) {
            rlo = vmin3(rlo, blo[j]);
            rhi = vmax3(rhi, bhi[j]);
            rn += bn[j];
            llo[j] = rlo;
            lhi[j] = rhi;
            ln[j] = rn;
        }
        rlo = F3{kBig, kBig, kBig};
        rhi = F3{-kBig, -kBig, -kBig};
        rn = 0;
        for (int j = kBinN - 1; j >= 0; j--) {
            rlo = vmin3(rlo, blo[j]);
            rhi = vmax3(rhi, bhi[j]);
            rn += bn[j];
            rlo_[j] = rlo;
            rhi_[j] = rhi;
            rn_[j] = rn;
        }
        const float total_area = half_area3(F3{b.hi[0] - b.lo[0], b.hi[1] - b.lo[1], b.hi[2] - b.lo[2]});
        for (int j = 0; j < kBinN - 1; j++) {
            if (ln[j] == 0 || rn_[j + 1] == 0) continue;
            const float la = half_area3(sub3(lhi[j], llo[j]));
            const float ra = half_area3(sub3(rhi_[j + 1], rlo_[j + 1]));
            const float cost = la / total_area * float(ln[j]) + ra / total_area * float(rn_[j + 1]);
            if (cost < best_cost) {
                best_cost = cost;
                best_axis = a;
                best_split = j;
            }
        }
    }
    const int n = tk.end - tk.start;
    Split s;
    if (n == 1 || tk.depth >= kDepthCap || best_cost >= float(n) || best_split == -1) {
        s.axis = -1;
        s.plane = 0;
    } else {
        s.axis = best_axis;
        s.plane = b.clo[best_axis] + float(best_split + 1) * (b.chi[best_axis] - b.clo[best_axis]) / float(kBinN);
    }
    splits[t] = s;
}

// 1 where the item at a position of a splitting task goes left (centroid < plane).
__global__ void k_flags(const float *items, const int *order, const int *pos_task, int lo_pos, int hi_pos,
                        const Split *splits, int *flags) {
    const int p = lo_pos + blockIdx.x * blockDim.x + threadIdx.x;
    if (p > hi_pos) return;
    int f = 0;
    if (p < hi_pos) {
        const int t = pos_task[p - lo_pos];
        if (t >= 0 && splits[t].axis >= 0) f = item(items, order[p])[6 + splits[t].axis] < splits[t].plane ? 1 : 0;
    }
    flags[p - lo_pos] = f;
}

// Positions of the elements std::partition swaps, per splitting task with T passing
// elements: the k-th failing element of the left part [start, start + T), counted
// from the left, goes to fail_pos[start + k] (k_fail_list); the m-th passing element
// of the right part [start + T, end), counted from the left, to pass_pos[start + m]
// (k_pass_list). Both lists are F long, F the failing count of the left part.
__global__ void k_pass_list(const int *pos_task, int lo_pos, int hi_pos, const Task *tasks, const Split *splits,
                            const int *flags, const int *prefix, int *pass_pos) {
    const int p = lo_pos + blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= hi_pos) return;
    const int t = pos_task[p - lo_pos];
    if (t < 0 || splits[t].axis < 0) return;
    const int s = tasks[t].start;
    const int base = prefix[s - lo_pos];
    const int T = prefix[tasks[t].end - lo_pos] - base;
    if (p < s + T || flags[p - lo_pos] == 0) return;
    const int m = prefix[p - lo_pos] - prefix[s + T - lo_pos];  // passing elements in [s + T, p)
    pass_pos[s - lo_pos + m] = p;
}

__global__ void k_fail_list(const int *pos_task, int lo_pos, int hi_pos, const Task *tasks, const Split *splits,
                            const int *flags, const int *prefix, int *fail_pos) {
    const int p = lo_pos + blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= hi_pos) return;
    const int t = pos_task[p - lo_pos];
    if (t < 0 || splits[t].axis < 0) return;
    const int s = tasks[t].start;
    const int base = prefix[s - lo_pos];
    const int T = prefix[tasks[t].end - lo_pos] - base;
    if (p >= s + T || flags[p - lo_pos] != 0) return;
    const int k = (p - s) - (prefix[p - lo_pos] - base);  // failing elements before p in [s, p)
    fail_pos[s - lo_pos + k] = p;
}

// The swaps: the k-th failing element of the left part with the k-th passing element
// of the right part counted from the right.
__global__ void k_swap(const int *pos_task, int lo_pos, int hi_pos, const Task *tasks, const Split *splits,
                       const int *prefix, const int *fail_pos, const int *pass_pos, int *order) {
    const int p = lo_pos + blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= hi_pos) return;
    const int t = pos_task[p - lo_pos];
    if (t < 0 || splits[t].axis < 0) return;
    const int s = tasks[t].start;
    const int base = prefix[s - lo_pos];
    const int T = prefix[tasks[t].end - lo_pos] - base;
    const int F = T - (prefix[s + T - lo_pos] - base);  // failing elements in the left part
    const int k = p - s;
    if (k >= F) return;
    const int a = fail_pos[s - lo_pos + k], b = pass_pos[s - lo_pos + F - 1 - k];
    const int x = order[a];
    order[a] = order[b];
    order[b] = x;
}

// Records the level's tasks and emits the next level's: a leaf keeps its range; a
// split task gets its two children at 2 * (split tasks before it) (child_base, an
// exclusive prefix over is_split), left then right, so the next level stays sorted.
__global__ void k_children(const Task *tasks, int n_tasks, const TaskBox *boxes, const Split *splits,
                           const int *prefix, int lo_pos, const int *child_base, int level, int rec_base, Rec *recs,
                           Task *next) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tasks) return;
    const Task tk = tasks[t];
    Rec r;
    for (int a = 0; a < 3; a++) {
        r.lo[a] = boxes[t].lo[a];
        r.hi[a] = boxes[t].hi[a];
    }
    r.start = tk.start;
    r.count = tk.end - tk.start;
    r.level = level;
    r.left = r.right = -1;
    if (splits[t].axis >= 0) {
        const int T = prefix[tk.end - lo_pos] - prefix[tk.start - lo_pos];
        int mid = tk.start + T;
        if (mid == tk.start || mid == tk.end) mid = tk.start + (tk.end - tk.start) / 2;
        const int c = 2 * child_base[t];
        r.left = rec_base + c;
        r.right = rec_base + c + 1;
        next[c] = Task{tk.start, mid, tk.depth + 1, rec_base + c};
        next[c + 1] = Task{mid, tk.end, tk.depth + 1, rec_base + c + 1};
    }
    recs[tk.rec] = r;
}

__global__ void k_is_split(const Split *splits, int n, int *out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t <= n) out[t] = (t < n && splits[t].axis >= 0) ? 1 : 0;
}

// Subtree node counts, one level at a time from the deepest.
__global__ void k_sizes(const Rec *recs, int lo, int hi, int *size) {
    const int r = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= hi) return;
    size[r] = recs[r].left < 0 ? 1 : 1 + size[recs[r].left] + size[recs[r].right];
}

// Depth-first (preorder) node indices, one level at a time from the root, and the
// node of each record: the host recursion writes a node, then its left subtree, then
// its right subtree.
__global__ void k_number(const Rec *recs, int lo, int hi, const int *size, int *index, int node_base,
                         lambda_bvh_node *nodes) {
    const int r = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= hi) return;
    const Rec &x = recs[r];
    const int self = index[r];
    lambda_bvh_node n;
    for (int a = 0; a < 3; a++) {
        n.min[a] = x.lo[a];
        n.max[a] = x.hi[a];
    }
    if (x.left < 0) {
        n.index = x.start;
        n.count = x.count;
    } else {
        index[x.left] = self + 1;
        index[x.right] = self + 1 + size[x.left];
        n.index = node_base + self + 1 + size[x.left];
        n.count = 0;
    }
    nodes[self] = n;
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side: the BuildAccel steps on a context's device and stream.
// ---------------------------------------------------------------------------

namespace {

struct BuildError {
    cudaError_t e;
    const char *what;
};

void ck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw BuildError{e, what};
}

// Temporary device memory of one build step, freed on every exit.
struct Scratch {
    std::vector<void *> ptrs;
    template <typename T>
    T *get(size_t n) {
        void *p = nullptr;
        ck(cudaMalloc(&p, std::max<size_t>(n * sizeof(T), 16)), "allocate build memory");
        ptrs.push_back(p);
        return static_cast<T *>(p);
    }
    ~Scratch() {
        for (void *p : ptrs) cudaFree(p);
    }
};

int blocks(int64_t n, int b) { return int(std::max<int64_t>(1, (n + b - 1) / b)); }

void gpu_instance_bounds(lambda_ctx *ctx, const lambda_host::HostScene &s, std::vector<float> &out) {
    const int n = int(s.instances.size());
    out.assign(size_t(n) * 9, 0.0f);
    if (n == 0) return;
    ck(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t st = ctx->stream;
    Scratch sc;
    auto *objs = sc.get<lambda_object>(s.objects.size());
    auto *insts = sc.get<lambda_instance>(size_t(n));
    auto *o9 = sc.get<float>(size_t(n) * 9);
    ck(cudaMemcpyAsync(objs, s.objects.data(), s.objects.size() * sizeof(lambda_object), cudaMemcpyHostToDevice, st),
       "upload objects");
    ck(cudaMemcpyAsync(insts, s.instances.data(), size_t(n) * sizeof(lambda_instance), cudaMemcpyHostToDevice, st),
       "upload instances");
    const int grid = std::min(n, 8 * ctx->sm_count * 8);
    k_instance_bounds<<<grid, kBoundsThreads, 0, st>>>(objs, insts, n, o9);
    ck(cudaGetLastError(), "launch instance bounds");
    ck(cudaMemcpyAsync(out.data(), o9, out.size() * sizeof(float), cudaMemcpyDeviceToHost, st), "read instance bounds");
    ck(cudaStreamSynchronize(st), "instance bounds");
}

void gpu_build(lambda_ctx *ctx, const std::vector<float> &items9, std::vector<int> &order, int start, int end,
               std::vector<lambda_bvh_node> &nodes) {
    const int n = end - start;
    if (n <= 0) return;
    ck(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t st = ctx->stream;
    Scratch sc;
    const size_t n_items = items9.size() / 9;
    float *items = sc.get<float>(items9.size());
    int *d_order = sc.get<int>(n_items);
    ck(cudaMemcpyAsync(items, items9.data(), items9.size() * sizeof(float), cudaMemcpyHostToDevice, st), "upload items");
    ck(cudaMemcpyAsync(d_order, order.data(), n_items * sizeof(int), cudaMemcpyHostToDevice, st), "upload order");
    // per position of [start, end) (one extra for the prefix sums' end)
    int *pos_task = sc.get<int>(size_t(n));
    int *flags = sc.get<int>(size_t(n) + 1);
    int *prefix = sc.get<int>(size_t(n) + 1);
    int *fail_pos = sc.get<int>(size_t(n));
    int *pass_pos = sc.get<int>(size_t(n));
    // a level's tasks (at most n), processed in chunks of at most `cap` tasks: the
    // per-task keys, boxes and bins (about 2.6 KB a task) are sized for one chunk
    const size_t max_tasks = size_t(n);
    const size_t cap = std::min<size_t>(max_tasks, size_t(1) << 16);
    Task *tasks = sc.get<Task>(max_tasks);
    Task *next = sc.get<Task>(max_tasks);
    auto *keys = sc.get<unsigned long long>(cap * kTaskKeys);
    TaskBox *boxes = sc.get<TaskBox>(cap);
    auto *bin_keys = sc.get<unsigned long long>(cap * 3 * kBinN * kBinKeys);
    int *bin_n = sc.get<int>(cap * 3 * kBinN);
    Split *splits = sc.get<Split>(cap);
    int *is_split = sc.get<int>(cap + 1);
    int *child_base = sc.get<int>(cap + 1);
    // records: at most 2n - 1 nodes
    const size_t max_recs = 2 * size_t(n);
    Rec *recs = sc.get<Rec>(max_recs);
    int *size = sc.get<int>(max_recs);
    int *index = sc.get<int>(max_recs);
    lambda_bvh_node *d_nodes = sc.get<lambda_bvh_node>(max_recs);
    // CUB scan scratch, sized for the larger of the two scans
    size_t scan_bytes = 0, b2 = 0;
    ck(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, flags, prefix, n + 1, st), "size scan");
    ck(cub::DeviceScan::ExclusiveSum(nullptr, b2, is_split, child_base, int(cap) + 1, st), "size scan");
    void *scan_tmp = sc.get<uint8_t>(std::max(scan_bytes, b2));
    const size_t scan_cap = std::max(scan_bytes, b2);

    const Task root{start, end, 1, 0};
    ck(cudaMemcpyAsync(tasks, &root, sizeof(Task), cudaMemcpyHostToDevice, st), "upload root");
    int n_tasks = 1, n_recs = 1;
    std::vector<int> level_lo{0}, level_hi{1};  // record ranges per level
    std::vector<Task> htasks;
    const int B = 256;
    for (int level = 0; n_tasks > 0; level++) {
        // the level's task ranges, which give each chunk its positions
        htasks.resize(size_t(n_tasks));
        ck(cudaMemcpyAsync(htasks.data(), tasks, size_t(n_tasks) * sizeof(Task), cudaMemcpyDeviceToHost, st),
           "read level");
        ck(cudaStreamSynchronize(st), "read level");
        int next_count = 0;
        for (int c0 = 0; c0 < n_tasks; c0 += int(cap)) {
            const int c1 = std::min(n_tasks, c0 + int(cap)), nt = c1 - c0;
            const int P0 = htasks[size_t(c0)].start, P1 = htasks[size_t(c1 - 1)].end, np = P1 - P0;
            const size_t off = size_t(P0 - start);
            int *pt = pos_task + off, *fl = flags + off, *pf = prefix + off, *fp = fail_pos + off, *pp = pass_pos + off;
            const Task *tk = tasks + c0;
            const int PB = blocks(np, B);
            k_assign<<<PB, B, 0, st>>>(tk, nt, P0, P1, pt);
            k_init_keys<<<blocks(int64_t(nt) * kTaskKeys, B), B, 0, st>>>(keys, nt);
            k_task_bounds<<<PB, B, 0, st>>>(items, d_order, pt, P0, P1, keys);
            k_task_decode<<<blocks(nt, 128), 128, 0, st>>>(items, d_order, keys, nt, boxes, bin_keys, bin_n);
            k_task_bins<<<PB, B, 0, st>>>(items, d_order, pt, P0, P1, boxes, bin_keys, bin_n);
            k_task_split<<<blocks(nt, 64), 64, 0, st>>>(items, d_order, tk, nt, boxes, bin_keys, bin_n, splits);
            k_flags<<<blocks(np + 1, B), B, 0, st>>>(items, d_order, pt, P0, P1, splits, fl);
            size_t tb = scan_cap;
            ck(cub::DeviceScan::ExclusiveSum(scan_tmp, tb, fl, pf, np + 1, st), "scan flags");
            k_fail_list<<<PB, B, 0, st>>>(pt, P0, P1, tk, splits, fl, pf, fp);
            k_pass_list<<<PB, B, 0, st>>>(pt, P0, P1, tk, splits, fl, pf, pp);
            k_swap<<<PB, B, 0, st>>>(pt, P0, P1, tk, splits, pf, fp, pp, d_order);
            k_is_split<<<blocks(nt + 1, B), B, 0, st>>>(splits, nt, is_split);
            tb = scan_cap;
            ck(cub::DeviceScan::ExclusiveSum(scan_tmp, tb, is_split, child_base, nt + 1, st), "scan splits");
            k_children<<<blocks(nt, B), B, 0, st>>>(tk, nt, boxes, splits, pf, P0, child_base, level,
                                                    n_recs + next_count, recs, next + next_count);
            ck(cudaGetLastError(), "launch build level");
            int splits_n = 0;
            ck(cudaMemcpyAsync(&splits_n, child_base + nt, sizeof(int), cudaMemcpyDeviceToHost, st), "read level");
            ck(cudaStreamSynchronize(st), "build level");
            next_count += 2 * splits_n;
        }
        std::swap(tasks, next);
        n_tasks = next_count;
        if (n_tasks > 0) {
            if (size_t(n_recs + n_tasks) > max_recs) throw BuildError{cudaErrorUnknown, "build exceeded its node bound"};
            level_lo.push_back(n_recs);
            level_hi.push_back(n_recs + n_tasks);
            n_recs += n_tasks;
        }
    }
    for (int l = int(level_lo.size()) - 1; l >= 0; l--)
        k_sizes<<<blocks(level_hi[l] - level_lo[l], B), B, 0, st>>>(recs, level_lo[l], level_hi[l], size);
    const int zero = 0;
    ck(cudaMemcpyAsync(index, &zero, sizeof(int), cudaMemcpyHostToDevice, st), "number nodes");
    const int node_base = int(nodes.size());
    for (size_t l = 0; l < level_lo.size(); l++)
        k_number<<<blocks(level_hi[l] - level_lo[l], B), B, 0, st>>>(recs, level_lo[l], level_hi[l], size, index,
                                                                      node_base, d_nodes);
    ck(cudaGetLastError(), "launch node numbering");
    nodes.resize(size_t(node_base) + size_t(n_recs));
    ck(cudaMemcpyAsync(nodes.data() + node_base, d_nodes, size_t(n_recs) * sizeof(lambda_bvh_node), cudaMemcpyDeviceToHost, st),
       "read nodes");
    ck(cudaMemcpyAsync(order.data() + start, d_order + start, size_t(n) * sizeof(int), cudaMemcpyDeviceToHost, st),
       "read order");
    ck(cudaStreamSynchronize(st), "build");
}

}  // namespace

// The BuildAccel of a context: both GPU steps, ranges of at least min_items items
// to the GPU builder. A CUDA failure becomes a SceneError with status LAMBDA_ERR_CUDA.
lambda_host::BuildAccel gpu_build_accel(lambda_ctx *ctx, int min_items) {
    lambda_host::BuildAccel a;
    a.instance_bounds = [ctx](const lambda_host::HostScene &s, std::vector<float> &out) {
        try {
            gpu_instance_bounds(ctx, s, out);
        } catch (const BuildError &e) {
            cudaGetLastError();
            throw lambda_host::SceneError(LAMBDA_ERR_CUDA, std::string(e.what) + " (" + cudaGetErrorString(e.e) + ")");
        }
    };
    a.build = [ctx](const std::vector<float> &items, std::vector<int> &order, int start, int end,
                    std::vector<lambda_bvh_node> &nodes) {
        try {
            gpu_build(ctx, items, order, start, end, nodes);
        } catch (const BuildError &e) {
            cudaGetLastError();
            throw lambda_host::SceneError(LAMBDA_ERR_CUDA, std::string(e.what) + " (" + cudaGetErrorString(e.e) + ")");
        }
    };
    a.build_min_items = std::max(1, min_items);
    return a;
}

extern "C" lambda_status lambda_parse_lrd_gpu(lambda_ctx *ctx, const char *path, int32_t gpu_min_items,
                                              lambda_host_scene **out, char *err, size_t err_len) {
    if (!ctx) return LAMBDA_ERR_INVALID_ARGUMENT;
    if (gpu_min_items < 0) return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "gpu_min_items must be >= 0");
    const lambda_host::BuildAccel accel = gpu_build_accel(ctx, gpu_min_items > 0 ? gpu_min_items : 1 << 16);
    return lambda_host::parse_into(path, out, err, err_len, &accel);
}
