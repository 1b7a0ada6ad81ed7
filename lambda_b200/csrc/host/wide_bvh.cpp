// Wide BVH construction (see wide_bvh.h for why traversal results do not change).
#include "wide_bvh.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <utility>

namespace lambda_host {
namespace {

struct Builder {
    const lambda_bvh_node *n;
    int num_nodes;
    int width;
    WideBvh &out;
    std::vector<std::vector<int>> children;  // per wide node: its child binary nodes in visiting order

    static float area(const lambda_bvh_node &b) {
        const float x = b.max[0] - b.min[0], y = b.max[1] - b.min[1], z = b.max[2] - b.min[2];
        return x * y + x * z + y * z;
    }
    bool leaf(int i) const { return n[i].count > 0; }

    // Code of binary node i, making its wide node (and those below) on first use.
    int code_of(int i) {
        if (out.code[i] != std::numeric_limits<int32_t>::min()) return out.code[i];
        if (leaf(i)) {
            const int id = int(out.leaves.size() / 2);
            out.leaves.push_back(n[i].index);
            out.leaves.push_back(n[i].count);
            return out.code[i] = -1 - id;
        }
        // frontier in visiting order: right child (index) before left (i + 1)
        std::vector<int> f = {n[i].index, i + 1};
        while (int(f.size()) < width) {
            int pick = -1;
            float best = -1;
            for (int k = 0; k < int(f.size()); k++)
                if (!leaf(f[k]) && area(n[f[k]]) > best) {
                    best = area(n[f[k]]);
                    pick = k;
                }
            if (pick < 0) break;
            const int c = f[pick];
            f[pick] = n[c].index;                    // its right child keeps its place
            f.insert(f.begin() + pick + 1, c + 1);  // then its left child
        }
        const int w = int(children.size());
        out.code[i] = w;
        children.push_back(f);
        for (int c : f) code_of(c);
        return w;
    }

    void emit() {
        const size_t W = children.size();
        out.records.assign(W * size_t(width) * 8, 0.0f);
        const float inf = std::numeric_limits<float>::infinity();
        for (size_t w = 0; w < W; w++)
            for (int k = 0; k < width; k++) {
                float *r = &out.records[(w * width + k) * 8];
                if (k < int(children[w].size())) {
                    const lambda_bvh_node &b = n[children[w][k]];
                    const int32_t c = out.code[children[w][k]];
                    r[0] = b.min[0];
                    r[1] = b.min[1];
                    r[2] = b.min[2];
                    std::memcpy(&r[3], &c, 4);
                    r[4] = b.max[0];
                    r[5] = b.max[1];
                    r[6] = b.max[2];
                } else {
                    r[0] = r[1] = r[2] = inf;
                    r[4] = r[5] = r[6] = -inf;
                    const int32_t c = -1;
                    std::memcpy(&r[3], &c, 4);
                }
            }
    }

    // Most entries a traversal from root binary node r holds at once if every child
    // passes: an entry popped with `pend` entries below it pushes its m children,
    // and the child visited k-th (k = 0 first) is later popped above pend + m - 1 - k.
    int stack_need(int r) const {
        int need = 1;
        std::vector<std::pair<int, int>> todo = {{out.code[r], 0}};
        while (!todo.empty()) {
            const auto [c, pend] = todo.back();
            todo.pop_back();
            if (c < 0) continue;
            const std::vector<int> &f = children[size_t(c)];
            const int m = int(f.size());
            need = std::max(need, pend + m);
            for (int k = 0; k < m; k++) todo.push_back({out.code[f[k]], pend + m - 1 - k});
        }
        return need;
    }
};

// One child bound quantized against origin o with scale s: the largest q in
// [0, 255] whose decoded value o + q * s is <= v (lower bound), or the smallest
// whose decoded value is >= v (upper bound); -1 when none fits.
int quant_bound(float v, float o, float s, bool upper) {
    const double x = (double(v) - double(o)) / double(s);
    int q = upper ? int(std::ceil(x)) : int(std::floor(x));
    q = std::clamp(q, 0, 255);
    auto dec = [&](int k) { return o + float(k) * s; };  // the device's FP32 decode
    if (upper) {
        while (q <= 255 && !(dec(q) >= v)) q++;
        return q <= 255 ? q : -1;
    }
    while (q >= 0 && !(dec(q) <= v)) q--;
    return q;
}

// The compressed records of every wide node (see WideBvh::quant).
void quantize(WideBvh &out, const std::vector<std::vector<int>> &children, int width) {
    const int stride = 1 + (6 * width + 15) / 16;
    out.quant_stride = stride;
    const size_t W = children.size();
    out.quant.assign(W * size_t(stride) * 4, 0u);
    for (size_t w = 0; w < W; w++) {
        uint32_t *q = &out.quant[w * size_t(stride) * 4];
        const int m = int(children[w].size());
        const float *rec = &out.records[w * size_t(width) * 8];
        float o[3];
        bool ok = true;
        for (int a = 0; a < 3; a++) {
            o[a] = std::numeric_limits<float>::infinity();
            for (int k = 0; k < m; k++) o[a] = std::min(o[a], rec[k * 8 + a]);
            ok = ok && std::isfinite(o[a]);
        }
        uint8_t bytes[6 * 8] = {0};
        uint32_t exps = 0;
        for (int a = 0; a < 3 && ok; a++) {
            double span = 0;
            for (int k = 0; k < m; k++) {
                const float lo = rec[k * 8 + a], hi = rec[k * 8 + 4 + a];
                ok = ok && std::isfinite(lo) && std::isfinite(hi);
                span = std::max(span, double(hi) - double(o[a]));
            }
            if (!ok) break;
            int e = 1;  // biased exponent: s = 2^(e - 127), the smallest normal power of two first
            while (e < 254 && std::ldexp(1.0, e - 127) * 255.0 < span) e++;
            bool fit = false;
            for (; e < 254 && !fit; e++) {
                const float sc = std::ldexp(1.0f, e - 127);
                fit = true;
                for (int k = 0; k < m && fit; k++) {
                    const int lo = quant_bound(rec[k * 8 + a], o[a], sc, false);
                    const int hi = quant_bound(rec[k * 8 + 4 + a], o[a], sc, true);
                    fit = lo >= 0 && hi >= 0;
                    if (fit) {
                        bytes[6 * k + a] = uint8_t(lo);
                        bytes[6 * k + 3 + a] = uint8_t(hi);
                    }
                }
                if (fit) exps |= uint32_t(e) << (8 * a);
            }
            ok = fit;
        }
        uint32_t packed = exps | (uint32_t(m) << 24);
        if (!ok) packed = (uint32_t(m) << 24) | 0x80000000u;
        std::memcpy(&q[0], &o[0], 4);
        std::memcpy(&q[1], &o[1], 4);
        std::memcpy(&q[2], &o[2], 4);
        q[3] = packed;
        if (ok) std::memcpy(&q[4], bytes, size_t(6 * m));
    }
}

}  // namespace

WideBvh build_wide_bvh(const lambda_bvh_node *nodes, int num_nodes, const lambda_instance *instances,
                       int num_instances, int width) {
    WideBvh out;
    out.width = width;
    out.code.assign(size_t(num_nodes), std::numeric_limits<int32_t>::min());
    Builder b{nodes, num_nodes, width, out, {}};
    b.code_of(0);
    for (int i = 0; i < num_instances; i++) b.code_of(instances[i].node);
    b.emit();
    quantize(out, b.children, width);
    out.stack_tlas = b.stack_need(0);
    out.stack_blas = 1;
    // one walk per distinct BLAS root: instances of one mesh share its tree
    std::vector<char> seen(size_t(num_nodes), 0);
    for (int i = 0; i < num_instances; i++) {
        const int r = instances[i].node;
        if (seen[size_t(r)]) continue;
        seen[size_t(r)] = 1;
        out.stack_blas = std::max(out.stack_blas, b.stack_need(r));
    }
    return out;
}

}  // namespace lambda_host
