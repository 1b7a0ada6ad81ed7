// Two-level binned-SAH BVH build and light list for the host scene.
//
// The split rule is the reference's (src/scene/bvh.h:111-246): 16 centroid bins
// per axis, SAH cost without a traversal term, a leaf when one item is left, at
// depth 20, when no split beats the item count, or when no axis has centroid
// extent >= 1e-4; partition by centroid < plane with std::partition, falling back
// to the middle when one side is empty. The tree, and with it the reordering of
// objects and instances, must come out identical, because hit object/instance
// ids are indices into the reordered arrays.
//
// Unlike the reference, every item's bounds and centroid are computed once and
// cached: the reference re-derives an instance's bounds from all of its objects'
// eight transformed corners on every visit (instance.h:54-101), which makes the
// build quadratic for instanced scenes. Caching changes no value.
#include <algorithm>
#include <cmath>
#include <map>
#include <numeric>
#include <thread>
#include <vector>

#include "hmath.h"
#include "scene.h"

namespace lambda_host {

namespace {

V3 load3(const float *p) { return v3(p[0], p[1], p[2]); }

struct ObjectGeom {
    const lambda_object &o;
    V3 corner() const { return load3(o.g); }
    V3 horizontal() const { return load3(o.g + 3); }
    V3 vertical() const { return load3(o.g + 6); }
    V3 normal() const { return load3(o.g + 9); }
    float radius_param() const { return o.g[3]; }

    // object.h:166-172
    V3 min() const {
        const V3 e = v3(kEpsilon, kEpsilon, kEpsilon);
        switch (o.type) {
            case LAMBDA_OBJECT_SPHERE: {
                float r = radius_param();
                return corner() - v3(r, r, r);
            }
            case LAMBDA_OBJECT_QUAD: {
                V3 c = corner(), h = horizontal(), v = vertical();
                return vmin(c, vmin(c + h, vmin(c + v, c + h + v))) - e;
            }
            default: {
                V3 c = corner(), h = horizontal(), v = vertical();
                return vmin(c, vmin(c + h, c + v)) - e;
            }
        }
    }
    V3 max() const {
        const V3 e = v3(kEpsilon, kEpsilon, kEpsilon);
        switch (o.type) {
            case LAMBDA_OBJECT_SPHERE: {
                float r = radius_param();
                return corner() + v3(r, r, r);
            }
            case LAMBDA_OBJECT_QUAD: {
                V3 c = corner(), h = horizontal(), v = vertical();
                return vmax(c, vmax(c + h, vmax(c + v, c + h + v))) + e;
            }
            default: {
                V3 c = corner(), h = horizontal(), v = vertical();
                return vmax(c, vmax(c + h, c + v)) + e;
            }
        }
    }
    // object.h:174-176
    V3 center() const {
        switch (o.type) {
            case LAMBDA_OBJECT_SPHERE: return corner();
            case LAMBDA_OBJECT_QUAD: return corner() + 0.5f * horizontal() + 0.5f * vertical();
            default: return corner() + (horizontal() + vertical()) / 3.0f;
        }
    }
    // object.h:178-195
    float bounding_radius() const {
        switch (o.type) {
            case LAMBDA_OBJECT_SPHERE: return radius_param();
            case LAMBDA_OBJECT_QUAD: {
                float d1 = length_sq(horizontal() + vertical());
                float d2 = length_sq(horizontal() - vertical());
                return 0.5f * std::sqrt(std::fmax(d1, d2));
            }
            default: {
                V3 c = center();
                float d1 = length_sq(corner() - c);
                float d2 = length_sq(corner() + horizontal() - c);
                float d3 = length_sq(corner() + vertical() - c);
                return std::sqrt(std::fmax(d1, std::fmax(d2, d3)));
            }
        }
    }
    // object.h:197-199
    float area() const {
        switch (o.type) {
            case LAMBDA_OBJECT_SPHERE: return 4.0f * kPi * radius_param() * radius_param();
            case LAMBDA_OBJECT_QUAD: return length(normal());
            default: return length(normal()) / 2.0f;
        }
    }
};

struct ItemBounds {
    V3 lo, hi, centroid;
};

V3 col0(const lambda_instance &in) { return v3(in.transform[0], in.transform[4], in.transform[8]); }

// Instance::min/max/center (instance.h:54-101): world bounds of the eight corners
// of every object's box, and the mean of the objects' transformed centres.
ItemBounds instance_bounds(const HostScene &s, const lambda_instance &in) {
    ItemBounds b;
    b.lo = v3(kMax, kMax, kMax);
    b.hi = v3(-kMax, -kMax, -kMax);
    V3 sum = v3(0, 0, 0);
    for (int i = 0; i < in.count; i++) {
        ObjectGeom g{s.objects[in.object + i]};
        V3 a = g.min(), c = g.max();
        const V3 corners[8] = {a, c, v3(a[0], a[1], c[2]), v3(a[0], c[1], a[2]), v3(a[0], c[1], c[2]),
                               v3(c[0], a[1], a[2]), v3(c[0], a[1], c[2]), v3(c[0], c[1], a[2])};
        for (const V3 &k : corners) {
            V3 w = transform(in.transform, k, 1);
            b.lo = vmin(b.lo, w);
            b.hi = vmax(b.hi, w);
        }
        sum = sum + transform(in.transform, g.center(), 1);
    }
    b.centroid = sum / float(in.count);
    return b;
}

ItemBounds object_bounds(const lambda_object &o) {
    ObjectGeom g{o};
    return ItemBounds{g.min(), g.max(), g.center()};
}

float half_area(const V3 &e) { return 2 * (e[0] * e[1] + e[0] * e[2] + e[1] * e[2]); }

// Subtrees of at least this many items are split across threads (see build_range).
constexpr int kParallelItems = 1024;

// Levels of the build that hand their right subtree to another thread: enough for
// every host thread.
int spawn_levels() {
    int levels = 0;
    for (unsigned t = std::max(1u, std::thread::hardware_concurrency()); t > 1; t >>= 1) levels++;
    return levels;
}

// Runs fn(i) for i in [0, n) on all host threads, in contiguous blocks. Each i is
// computed by one thread alone, so results do not depend on the thread count.
template <class F>
void parallel_for(size_t n, F fn) {
    const size_t threads = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), std::max<size_t>(n / 64, 1));
    if (threads <= 1) {
        for (size_t i = 0; i < n; i++) fn(i);
        return;
    }
    std::vector<std::thread> pool;
    for (size_t t = 0; t < threads; t++)
        pool.emplace_back([&, t] {
            for (size_t i = n * t / threads; i < n * (t + 1) / threads; i++) fn(i);
        });
    for (auto &th : pool) th.join();
}

// One recursive binned-SAH build over order[start, end) (bvh.h:111-246). Returns
// the node index of the subtree root.
int build_range(const std::vector<ItemBounds> &items, std::vector<int> &order, int start, int end,
                std::vector<lambda_bvh_node> &nodes, int depth, int spawn = 0) {
    V3 lo = v3(kMax, kMax, kMax), hi = v3(-kMax, -kMax, -kMax);
    V3 clo = lo, chi = hi;
    for (int i = start; i < end; i++) {
        const ItemBounds &b = items[order[i]];
        lo = vmin(lo, b.lo);
        hi = vmax(hi, b.hi);
        clo = vmin(clo, b.centroid);
        chi = vmax(chi, b.centroid);
    }

    float best_cost = kMax;
    int best_axis = 0, best_split = -1;
    for (int axis = 0; axis < 3; axis++) {
        const float extent = chi[axis] - clo[axis];
        if (!(extent >= kEpsilon)) continue;
        V3 bin_lo[kBinCount], bin_hi[kBinCount];
        int bin_n[kBinCount];
        for (int j = 0; j < kBinCount; j++) {
            bin_lo[j] = v3(kMax, kMax, kMax);
            bin_hi[j] = v3(-kMax, -kMax, -kMax);
            bin_n[j] = 0;
        }
        for (int j = start; j < end; j++) {
            const ItemBounds &b = items[order[j]];
            int bin = int(float(kBinCount) * (b.centroid[axis] - clo[axis]) / extent);
            bin = std::clamp(bin, 0, kBinCount - 1);
            bin_lo[bin] = vmin(bin_lo[bin], b.lo);
            bin_hi[bin] = vmax(bin_hi[bin], b.hi);
            bin_n[bin]++;
        }
        // prefix (left) and suffix (right) sweeps
        V3 left_lo[kBinCount], left_hi[kBinCount], right_lo[kBinCount], right_hi[kBinCount];
        int left_n[kBinCount], right_n[kBinCount];
        V3 rlo = v3(kMax, kMax, kMax), rhi = v3(-kMax, -kMax, -kMax);
        int rn = 0;
        for (int j = 0; j < kBinCount; j++) {
            rlo = vmin(rlo, bin_lo[j]);
            rhi = vmax(rhi, bin_hi[j]);
            rn += bin_n[j];
            left_lo[j] = rlo;
            left_hi[j] = rhi;
            left_n[j] = rn;
        }
        rlo = v3(kMax, kMax, kMax);
        rhi = v3(-kMax, -kMax, -kMax);
        rn = 0;
        for (int j = kBinCount - 1; j >= 0; j--) {
            rlo = vmin(rlo, bin_lo[j]);
            rhi = vmax(rhi, bin_hi[j]);
            rn += bin_n[j];
            right_lo[j] = rlo;
            right_hi[j] = rhi;
            right_n[j] = rn;
        }
        const float total_area = half_area(hi - lo);
        for (int j = 0; j < kBinCount - 1; j++) {
            if (left_n[j] == 0 || right_n[j + 1] == 0) continue;
            float la = half_area(left_hi[j] - left_lo[j]);
            float ra = half_area(right_hi[j + 1] - right_lo[j + 1]);
            float cost = la / total_area * float(left_n[j]) + ra / total_area * float(right_n[j + 1]);
            if (cost < best_cost) {
                best_cost = cost;
                best_axis = axis;
                best_split = j;
            }
        }
    }

    if (end - start == 1 || depth >= kMaxDepth || best_cost >= float(end - start) || best_split == -1) {
        lambda_bvh_node leaf{};
        for (int k = 0; k < 3; k++) {
            leaf.min[k] = lo[k];
            leaf.max[k] = hi[k];
        }
        leaf.index = start;
        leaf.count = end - start;
        nodes.push_back(leaf);
        return int(nodes.size()) - 1;
    }

    const float plane = clo[best_axis] + float(best_split + 1) * (chi[best_axis] - clo[best_axis]) / float(kBinCount);
    auto split = std::partition(order.begin() + start, order.begin() + end,
                                [&](int i) { return items[i].centroid[best_axis] < plane; });
    int mid = int(split - order.begin());
    if (mid == start || mid == end) mid = start + (end - start) / 2;

    const int self = int(nodes.size());
    lambda_bvh_node inner{};
    for (int k = 0; k < 3; k++) {
        inner.min[k] = lo[k];
        inner.max[k] = hi[k];
    }
    inner.index = -1;
    inner.count = 0;
    nodes.push_back(inner);
    if (spawn > 0 && end - start >= kParallelItems) {
        // The right subtree reorders only order[mid, end), so it is built on another
        // thread into its own array (node links relative to that array) while the left
        // one is built here; it is then appended after the left subtree with its links
        // shifted, which is the array the sequential build writes.
        std::vector<lambda_bvh_node> right_nodes;
        right_nodes.reserve(size_t(2 * (end - mid)));
        std::thread t([&] { build_range(items, order, mid, end, right_nodes, depth + 1, spawn - 1); });
        build_range(items, order, start, mid, nodes, depth + 1, spawn - 1);
        t.join();
        const int offset = int(nodes.size());
        for (lambda_bvh_node &n : right_nodes) {
            if (n.count == 0) n.index += offset;  // interior: link to its right child
            nodes.push_back(n);
        }
        nodes[self].index = offset;
        return self;
    }
    build_range(items, order, start, mid, nodes, depth + 1, spawn);
    const int right = build_range(items, order, mid, end, nodes, depth + 1, spawn);
    nodes[self].index = right;
    return self;
}

// Items as the 9 floats per item (lo, hi, centroid) a BuildAccel step takes.
std::vector<float> flatten(const std::vector<ItemBounds> &items) {
    std::vector<float> f(items.size() * 9);
    for (size_t i = 0; i < items.size(); i++)
        for (int k = 0; k < 3; k++) {
            f[9 * i + k] = items[i].lo[k];
            f[9 * i + 3 + k] = items[i].hi[k];
            f[9 * i + 6 + k] = items[i].centroid[k];
        }
    return f;
}

// One build over order[start, end): on the GPU when a BuildAccel takes ranges this
// large, else the host recursion. Both write the same nodes.
void build_items(const std::vector<ItemBounds> &items, const std::vector<float> *flat, std::vector<int> &order,
                 int start, int end, std::vector<lambda_bvh_node> &nodes, const BuildAccel *accel) {
    if (accel && accel->build && flat && end - start >= accel->build_min_items) {
        accel->build(*flat, order, start, end, nodes);
        return;
    }
    build_range(items, order, start, end, nodes, 1, spawn_levels());
}

}  // namespace

void build_bvh(HostScene &s, const std::vector<int> &group_offsets, const BuildAccel *accel,
               std::vector<float> *instance_boxes) {
    s.nodes.clear();
    if (instance_boxes) instance_boxes->clear();
    if (s.objects.empty()) return;
    s.nodes.reserve(2 * s.objects.size());

    // TLAS over instances
    // An instance's bounds visit all its objects (O(instances x objects)); instances
    // are independent, so they run on all host threads, or on the GPU.
    std::vector<ItemBounds> inst_bounds(s.instances.size());
    if (accel && accel->instance_bounds) {
        std::vector<float> f;
        accel->instance_bounds(s, f);
        for (size_t i = 0; i < inst_bounds.size(); i++)
            inst_bounds[i] = ItemBounds{v3(f[9 * i], f[9 * i + 1], f[9 * i + 2]), v3(f[9 * i + 3], f[9 * i + 4], f[9 * i + 5]),
                                        v3(f[9 * i + 6], f[9 * i + 7], f[9 * i + 8])};
    } else {
        parallel_for(s.instances.size(), [&](size_t i) { inst_bounds[i] = instance_bounds(s, s.instances[i]); });
    }
    std::vector<int> order(s.instances.size());
    std::iota(order.begin(), order.end(), 0);
    {
        const bool big = accel && accel->build && int(s.instances.size()) >= accel->build_min_items;
        const std::vector<float> flat = big ? flatten(inst_bounds) : std::vector<float>{};
        build_items(inst_bounds, big ? &flat : nullptr, order, 0, int(s.instances.size()), s.nodes, accel);
    }
    {
        std::vector<lambda_instance> reordered;
        reordered.reserve(s.instances.size());
        for (int i : order) reordered.push_back(s.instances[i]);
        s.instances.swap(reordered);
    }
    if (instance_boxes) {
        instance_boxes->resize(order.size() * 6);
        for (size_t i = 0; i < order.size(); i++)
            for (int k = 0; k < 3; k++) {
                (*instance_boxes)[6 * i + k] = inst_bounds[size_t(order[i])].lo[k];
                (*instance_boxes)[6 * i + 3 + k] = inst_bounds[size_t(order[i])].hi[k];
            }
    }

    // one BLAS per object group, over a shared object order
    std::vector<ItemBounds> obj_bounds(s.objects.size());
    parallel_for(s.objects.size(), [&](size_t i) { obj_bounds[i] = object_bounds(s.objects[i]); });
    std::vector<int> obj_order(s.objects.size());
    std::iota(obj_order.begin(), obj_order.end(), 0);
    std::map<int, int> root_of_group;
    std::vector<float> obj_flat;
    for (size_t g = 0; g + 1 < group_offsets.size(); g++) {
        root_of_group[group_offsets[g]] = int(s.nodes.size());
        const bool big = accel && accel->build && group_offsets[g + 1] - group_offsets[g] >= accel->build_min_items;
        if (big && obj_flat.empty()) obj_flat = flatten(obj_bounds);
        build_items(obj_bounds, big ? &obj_flat : nullptr, obj_order, group_offsets[g], group_offsets[g + 1], s.nodes,
                    accel);
    }
    for (auto &in : s.instances) in.node = root_of_group.at(in.object);
    {
        std::vector<lambda_object> reordered;
        reordered.reserve(s.objects.size());
        for (int i : obj_order) reordered.push_back(s.objects[i]);
        s.objects.swap(reordered);
    }
}

namespace {

// Whether every object sphere of an instance leaves the scene sphere (C, R) of the
// light-list merge unchanged, shown from the instance's world box alone: all of its
// objects' transformed centres lie in the box (up to rounding) and their radii are
// at most r_max, so if the box's farthest corner from C plus r_max stays below R by
// a margin far wider than float rounding, the merge's "grow" test fails for each of
// them, and since R exceeds every object radius its "replace" test fails too. The
// margins (1e-5 relative, plus an absolute term for the centres' rounding) dwarf
// the float error of the merge's own arithmetic (about 1e-7 relative).
bool instance_leaves_sphere(const float *box, double r_max, const V3 &C, float R) {
    const double c[3] = {C[0], C[1], C[2]};
    double far = 0, mag = std::fabs(c[0]) + std::fabs(c[1]) + std::fabs(c[2]) + 1.0;
    for (int k = 0; k < 8; k++) {
        double d2 = 0;
        for (int a = 0; a < 3; a++) {
            const double v = (k >> a) & 1 ? box[3 + a] : box[a];
            mag = std::max(mag, std::fabs(v));
            d2 += (v - c[a]) * (v - c[a]);
        }
        far = std::max(far, std::sqrt(d2));
    }
    const double tol = 1e-5;
    const double reach = (far + 4.0 * tol * mag) * (1 + tol) + r_max * (1 + tol);
    return std::isfinite(reach) && reach <= double(R) * (1 - tol) && double(R) > r_max * (1 + tol);
}

}  // namespace

void build_lights(HostScene &s, const std::vector<float> *instance_boxes) {
    V3 scene_center = v3(0, 0, 0);
    float scene_radius = 0;
    // The merge below is sequential in instance and object order. The transformed
    // centres and radii it consumes are not, so they are computed ahead on all host
    // threads, an instance at a time. An instance whose box shows that it changes
    // neither the sphere (instance_leaves_sphere) nor the light list (no emissive
    // material) is passed over: the merge's state is the same after it either way.
    struct Sphere {
        V3 c;
        float r;
    };
    // per object group (first object, count): the largest bounding radius and
    // whether any object's own material is emissive
    std::map<std::pair<int, int>, std::pair<float, bool>> groups;
    auto group_of = [&](const lambda_instance &in) {
        auto it = groups.find({in.object, in.count});
        if (it != groups.end()) return it->second;
        float r = 0;
        bool emits = false;
        for (int j = 0; j < in.count; j++) {
            ObjectGeom g{s.objects[in.object + j]};
            r = std::fmax(r, g.bounding_radius());
            emits = emits || s.materials[s.objects[in.object + j].material].type == LAMBDA_MATERIAL_EMISSIVE;
        }
        return groups[{in.object, in.count}] = {r, emits};
    };
    const bool can_skip = instance_boxes && instance_boxes->size() == s.instances.size() * 6;
    std::vector<Sphere> pre;
    for (int i = 0; i < int(s.instances.size()); i++) {
        const lambda_instance &in = s.instances[i];
        if (can_skip && scene_radius > 0) {
            const auto [r_max, group_emits] = group_of(in);
            const bool emits =
                in.material >= 0 ? s.materials[in.material].type == LAMBDA_MATERIAL_EMISSIVE : group_emits;
            if (!emits && instance_leaves_sphere(instance_boxes->data() + 6 * size_t(i),
                                                 double(r_max) * double(length(col0(in))), scene_center, scene_radius))
                continue;
        }
        const float scale = length(col0(in));
        pre.resize(size_t(in.count));
        parallel_for(size_t(in.count), [&](size_t j) {
            ObjectGeom g{s.objects[in.object + int(j)]};
            pre[j] = Sphere{transform(in.transform, g.center(), 1), g.bounding_radius() * scale};
        });
        const float scale_sq = length_sq(col0(in));
        for (int j = 0; j < in.count; j++) {
            const int object_index = in.object + j;
            ObjectGeom g{s.objects[object_index]};
            const V3 object_center = pre[size_t(j)].c;
            const float object_radius = pre[size_t(j)].r;
            const V3 to_object = object_center - scene_center;
            const float distance = length(to_object);
            if (distance + scene_radius <= object_radius) {
                scene_center = object_center;
                scene_radius = object_radius;
            } else if (distance + object_radius > scene_radius) {
                const float grown = 0.5f * (distance + scene_radius + object_radius);
                scene_center = scene_center + (grown - scene_radius) * to_object / distance;
                scene_radius = grown;
            }
            const int material = in.material >= 0 ? in.material : s.objects[object_index].material;
            const lambda_material &m = s.materials[material];
            if (m.type == LAMBDA_MATERIAL_EMISSIVE) {
                s.light_instances.push_back(i);
                s.light_objects.push_back(object_index);
                const float power = g.area() * scale_sq * spectrum_texture_average(s, m.p[0]);
                s.light_powers.push_back(power);
                s.total_light_power += power;
            }
        }
    }
    s.light_instances.push_back(-1);
    s.light_objects.push_back(-1);
    const float background_power =
        4.0f * kPi * scene_radius * scene_radius * spectrum_texture_average(s, s.background_texture);
    s.light_powers.push_back(background_power);
    s.total_light_power += background_power;
}

}  // namespace lambda_host
