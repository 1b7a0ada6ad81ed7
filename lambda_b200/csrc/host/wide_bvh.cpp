// Wide BVH construction (see wide_bvh.h for why traversal results do not change).
#include "wide_bvh.h"

#include <algorithm>
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
