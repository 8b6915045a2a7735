// Host BVH construction: binned SAH → compressed 8-wide nodes (see
// bvh_build.h). The reference builds its acceleration structures through the
// Vulkan driver (crates/cenote/src/gpu/accel.rs:82-140); this build replaces
// that library call for traversal without RT cores.
#include "bvh_build.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <deque>
#include <future>
#include <limits>

namespace cn {
namespace {

struct Box {
    float lo[3] = {std::numeric_limits<float>::max(), std::numeric_limits<float>::max(),
                   std::numeric_limits<float>::max()};
    float hi[3] = {-std::numeric_limits<float>::max(), -std::numeric_limits<float>::max(),
                   -std::numeric_limits<float>::max()};
    void grow(const Box& b) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], b.lo[a]);
            hi[a] = std::max(hi[a], b.hi[a]);
        }
    }
    void grow(const float* p) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], p[a]);
            hi[a] = std::max(hi[a], p[a]);
        }
    }
    // Half the surface area, in double: boxes of very large triangles
    // (extents near FLT_MAX) keep finite, ordered costs.
    double area() const {
        double d[3];
        for (int a = 0; a < 3; ++a) d[a] = std::max(double(hi[a]) - double(lo[a]), 0.0);
        return d[0] * d[1] + d[1] * d[2] + d[2] * d[0];
    }
};

struct Node2 {
    Box box;
    uint32_t left = 0, right = 0;  // children when count == 0
    uint32_t first = 0, count = 0; // leaf range into the index array
    uint32_t tris = 0;             // triangles in the subtree
};

struct Builder {
    const std::vector<BuildTri>& in;
    std::vector<Box> tri_box;
    std::vector<float> cen;  // 3 per triangle
    std::vector<uint32_t> idx;
    std::vector<Node2> nodes;
    std::atomic<uint32_t> next{1};

    explicit Builder(const std::vector<BuildTri>& t) : in(t) {
        size_t n = t.size();
        tri_box.resize(n);
        cen.resize(3 * n);
        idx.resize(n);
        nodes.resize(std::max<size_t>(2 * n, 1));
        for (size_t i = 0; i < n; ++i) {
            for (int k = 0; k < 3; ++k) tri_box[i].grow(t[i].v[k]);
            for (int a = 0; a < 3; ++a) cen[3 * i + a] = 0.5f * (tri_box[i].lo[a] + tri_box[i].hi[a]);
            idx[i] = uint32_t(i);
        }
    }

    // Exact SAH for ranges of at most SWEEP_MAX triangles: sort the range by
    // centroid along each axis (stable, so ties keep their order and the
    // build stays deterministic), cost every split between two different
    // centroids from prefix and suffix bounds, and leave the range sorted
    // along the winning axis. Like the binned split, equal centroids stay on
    // one side; a range whose centroids all coincide splits by index.
    // Returns the index of the first triangle of the right child.
    static constexpr uint32_t SWEEP_MAX = 65536;

    uint32_t sweep_split(uint32_t first, uint32_t count, const Box& cbox) {
        auto begin = idx.begin() + first, end = begin + count;
        std::vector<double> right_area(count);
        double best_cost = std::numeric_limits<double>::max();
        int best_axis = -1, sorted_axis = -1;
        uint32_t best_left = 0;
        for (int axis = 0; axis < 3; ++axis) {
            if (!(cbox.hi[axis] > cbox.lo[axis])) continue;
            auto key = [&](uint32_t x) { return cen[3 * x + axis]; };
            std::stable_sort(begin, end, [&](uint32_t x, uint32_t y) { return key(x) < key(y); });
            sorted_axis = axis;
            Box acc;
            for (uint32_t i = count; i-- > 1;) {
                acc.grow(tri_box[idx[first + i]]);
                right_area[i] = acc.area();
            }
            Box left;
            for (uint32_t i = 1; i < count; ++i) {
                left.grow(tri_box[idx[first + i - 1]]);
                if (!(key(idx[first + i - 1]) < key(idx[first + i]))) continue;
                double cost = left.area() * double(i) + right_area[i] * double(count - i);
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = axis;
                    best_left = i;
                }
            }
        }
        if (best_axis < 0) return first + count / 2;  // coincident centroids
        if (best_axis != sorted_axis)
            std::stable_sort(begin, end, [&](uint32_t x, uint32_t y) {
                return cen[3 * x + best_axis] < cen[3 * y + best_axis];
            });
        return first + best_left;
    }

    // Past SAH_DEPTH_MAX binary levels the split is the object median along
    // the centroid box's longest axis (ties by triangle index), which halves
    // the range every level: an SAH that peels one triangle off per level
    // (nested triangles of geometrically growing size) cannot make the
    // binary tree, the recursion or the wide tree deeper than
    // SAH_DEPTH_MAX + log2(n) levels.
    static constexpr int SAH_DEPTH_MAX = 48;

    uint32_t median_split(uint32_t first, uint32_t count, const Box& cbox) {
        int axis = 0;
        for (int a = 1; a < 3; ++a)
            if (cbox.hi[a] - cbox.lo[a] > cbox.hi[axis] - cbox.lo[axis]) axis = a;
        auto begin = idx.begin() + first;
        std::nth_element(begin, begin + count / 2, begin + count, [&](uint32_t x, uint32_t y) {
            float a = cen[3 * x + axis], b = cen[3 * y + axis];
            return a < b || (a == b && x < y);
        });
        return first + count / 2;
    }

    void build(uint32_t ni, uint32_t first, uint32_t count, int depth) {
        Node2& n = nodes[ni];
        Box box, cbox;
        for (uint32_t i = first; i < first + count; ++i) {
            box.grow(tri_box[idx[i]]);
            cbox.grow(&cen[3 * idx[i]]);
        }
        n.box = box;
        n.tris = count;
        if (count == 1) {
            n.first = first;
            n.count = 1;
            return;
        }
        uint32_t mid;
        if (depth >= SAH_DEPTH_MAX) {
            mid = median_split(first, count, cbox);
        } else if (count <= SWEEP_MAX) {
            mid = sweep_split(first, count, cbox);
        } else {
            constexpr int NB = 32;
            double best_cost = std::numeric_limits<double>::max();
            int best_axis = -1, best_split = 0;
            for (int axis = 0; axis < 3; ++axis) {
                float ext = cbox.hi[axis] - cbox.lo[axis];
                if (!(ext > 0.0f)) continue;
                float scale = float(NB) / ext;
                Box bb[NB];
                uint32_t bn[NB] = {};
                for (uint32_t i = first; i < first + count; ++i) {
                    int b = std::min(NB - 1, std::max(0, int((cen[3 * idx[i] + axis] - cbox.lo[axis]) * scale)));
                    bb[b].grow(tri_box[idx[i]]);
                    bn[b]++;
                }
                double rarea[NB];
                uint32_t rcount[NB];
                Box acc;
                uint32_t c = 0;
                for (int b = NB - 1; b > 0; --b) {
                    acc.grow(bb[b]);
                    c += bn[b];
                    rarea[b] = acc.area();
                    rcount[b] = c;
                }
                Box lacc;
                uint32_t lc = 0;
                for (int s = 1; s < NB; ++s) {
                    lacc.grow(bb[s - 1]);
                    lc += bn[s - 1];
                    if (!lc || !rcount[s]) continue;
                    double cost = lacc.area() * double(lc) + rarea[s] * double(rcount[s]);
                    if (cost < best_cost) {
                        best_cost = cost;
                        best_axis = axis;
                        best_split = s;
                    }
                }
            }
            if (best_axis >= 0) {
                float ext = cbox.hi[best_axis] - cbox.lo[best_axis];
                float scale = float(NB) / ext;
                float lo = cbox.lo[best_axis];
                auto it = std::partition(idx.begin() + first, idx.begin() + first + count, [&](uint32_t t) {
                    int b = std::min(NB - 1, std::max(0, int((cen[3 * t + best_axis] - lo) * scale)));
                    return b < best_split;
                });
                mid = uint32_t(it - idx.begin());
                if (mid == first || mid == first + count) mid = first + count / 2;
            } else {
                mid = first + count / 2;  // coincident centroids: split by index
            }
        }
        uint32_t l = next.fetch_add(2);
        n.left = l;
        n.right = l + 1;
        n.count = 0;
        uint32_t lc = mid - first, rc = first + count - mid;
        if (depth < 4 && count > 65536) {
            auto f = std::async(std::launch::async, [&, l, first, lc, depth] { build(l, first, lc, depth + 1); });
            build(l + 1, mid, rc, depth + 1);
            f.get();
        } else {
            build(l, first, lc, depth + 1);
            build(l + 1, mid, rc, depth + 1);
        }
    }

    void gather(uint32_t ni, std::vector<uint32_t>& out) const {
        const Node2& n = nodes[ni];
        if (n.count) {
            for (uint32_t i = n.first; i < n.first + n.count; ++i) out.push_back(idx[i]);
            return;
        }
        gather(n.left, out);
        gather(n.right, out);
    }
};

void put_tri(std::vector<float>& out, const BuildTri& t) {
    float rec[12];
    for (int k = 0; k < 3; ++k)
        for (int a = 0; a < 3; ++a) rec[4 * k + a] = t.v[k][a];
    std::memcpy(&rec[3], &t.instance, 4);
    std::memcpy(&rec[7], &t.primitive, 4);
    std::memcpy(&rec[11], &t.flags, 4);
    out.insert(out.end(), rec, rec + 12);
}

}  // namespace

WideBvh build_wide_bvh(const std::vector<BuildTri>& tris, unsigned threads) {
    WideBvh out;
    if (tris.empty()) return out;
    Builder b(tris);
    (void)threads;
    b.build(0, 0, uint32_t(tris.size()), 0);

    // Cost-optimal collapse (Ylitie, Karras & Laine 2017, "Efficient
    // incoherent ray traversal on GPUs through compressed wide BVHs", §3.1):
    // bottom-up, cost[n][i] is the cheapest SAH cost of covering n's subtree
    // with at most i child slots of the parent (i = 1..7); a slot is either a
    // leaf of up to three triangles or an 8-wide node whose own children are
    // distributed over its 8 slots. c_node = 1 per node visit, c_prim = 0.3
    // per triangle test, each weighted by the node's surface area.
    constexpr float C_NODE = 1.0f, C_PRIM = 0.3f;
    constexpr float INF = std::numeric_limits<float>::infinity();
    const uint32_t n2 = b.next.load();
    // Areas relative to the root's, so the float costs stay finite for any
    // finite geometry.
    const double inv_root = 1.0 / std::max(b.nodes[0].box.area(), 1e-300);
    std::vector<float> cost(size_t(n2) * 8, INF);  // [n][i], i = 1..7 used
    std::vector<uint8_t> how(size_t(n2) * 8, 0);    // i=1: 0 leaf / 1 node; i>1: 0 = as i-1, k = left gets k
    std::vector<uint8_t> split8(n2, 0);             // left's share when n is an 8-wide node
    for (uint32_t ni = n2; ni-- > 0;) {
        const Node2& n = b.nodes[ni];
        float* c = &cost[size_t(ni) * 8];
        uint8_t* h = &how[size_t(ni) * 8];
        const float area = float(n.box.area() * inv_root);
        const float leaf = n.tris <= 3 ? area * C_PRIM * float(n.tris) : INF;
        if (n.count) {
            for (int i = 1; i < 8; ++i) c[i] = leaf;
            continue;
        }
        const float* cl = &cost[size_t(n.left) * 8];
        const float* cr = &cost[size_t(n.right) * 8];
        float dist[9];
        uint8_t dsplit[9] = {};
        for (int j = 2; j <= 8; ++j) {
            dist[j] = INF;
            for (int k = 1; k < j; ++k) {
                float v = cl[k] + cr[j - k];
                if (v < dist[j]) {
                    dist[j] = v;
                    dsplit[j] = uint8_t(k);
                }
            }
        }
        split8[ni] = dsplit[8];
        const float node = dist[8] + area * C_NODE;
        c[1] = std::min(leaf, node);
        h[1] = leaf <= node ? 0 : 1;
        for (int i = 2; i < 8; ++i) {
            if (dist[i] < c[i - 1]) {
                c[i] = dist[i];
                h[i] = dsplit[i];
            } else {
                c[i] = c[i - 1];
                h[i] = 0;
            }
        }
    }
    auto is_leaf = [&](uint32_t ni) { return b.nodes[ni].count || how[size_t(ni) * 8 + 1] == 0; };
    auto collect = [&](auto&& self, uint32_t ni, int i, std::vector<uint32_t>& kids) -> void {
        while (i > 1 && how[size_t(ni) * 8 + i] == 0) --i;
        if (i == 1) {
            kids.push_back(ni);
            return;
        }
        int k = how[size_t(ni) * 8 + i];
        self(self, b.nodes[ni].left, k, kids);
        self(self, b.nodes[ni].right, i - k, kids);
    };

    struct Pending {
        uint32_t n2, wide, depth;
    };
    std::deque<Pending> queue;
    out.nodes.emplace_back();
    queue.push_back({0, 0, 1});
    out.tris.reserve(tris.size() * 12);
    while (!queue.empty()) {
        Pending job = queue.front();
        queue.pop_front();
        out.depth = std::max(out.depth, job.depth);
        std::vector<uint32_t> kids;
        const Node2& root = b.nodes[job.n2];
        if (root.count || root.tris <= 3) kids.push_back(job.n2);
        else {
            int k = split8[job.n2];
            collect(collect, root.left, k, kids);
            collect(collect, root.right, 8 - k, kids);
        }
        // Octant slot assignment: child i's centre offset from the node centre
        // scored against slot s's direction (bit 2 ↔ +x, 1 ↔ +y, 0 ↔ +z);
        // greedy best-pair matching.
        Box nb;
        for (uint32_t k : kids) nb.grow(b.nodes[k].box);
        float nc[3];
        for (int a = 0; a < 3; ++a) nc[a] = 0.5f * (nb.lo[a] + nb.hi[a]);
        int slot_of[8];
        bool slot_used[8] = {};
        bool kid_done[8] = {};
        float score[8][8];
        for (size_t i = 0; i < kids.size(); ++i) {
            const Box& kb = b.nodes[kids[i]].box;
            for (int s = 0; s < 8; ++s) {
                float d = 0.0f;
                for (int a = 0; a < 3; ++a) {
                    float off = 0.5f * (kb.lo[a] + kb.hi[a]) - nc[a];
                    d += ((s >> (2 - a)) & 1) ? off : -off;
                }
                score[i][s] = d;
            }
        }
        for (size_t round = 0; round < kids.size(); ++round) {
            float best = -std::numeric_limits<float>::max();
            int bi = -1, bs = -1;
            for (size_t i = 0; i < kids.size(); ++i) {
                if (kid_done[i]) continue;
                for (int s = 0; s < 8; ++s) {
                    if (slot_used[s]) continue;
                    if (score[i][s] > best) {
                        best = score[i][s];
                        bi = int(i);
                        bs = s;
                    }
                }
            }
            kid_done[bi] = true;
            slot_used[bs] = true;
            slot_of[bi] = bs;
        }
        int kid_in_slot[8];
        for (int s = 0; s < 8; ++s) kid_in_slot[s] = -1;
        for (size_t i = 0; i < kids.size(); ++i) kid_in_slot[slot_of[i]] = int(i);

        // Quantisation frame.
        WideNode wn;
        std::memset(&wn, 0, sizeof wn);
        int exps[3];
        for (int a = 0; a < 3; ++a) {
            wn.p[a] = nb.lo[a];
            double ext = double(nb.hi[a]) - double(nb.lo[a]);
            int e = ext > 0.0 ? int(std::ceil(std::log2(ext / 254.0))) : -126;
            exps[a] = std::max(-126, std::min(127, e));
        }
        for (;;) {  // widen an axis' step until every child box fits in 8 bits
            bool ok = true;
            for (size_t i = 0; i < kids.size() && ok; ++i) {
                const Box& kb = b.nodes[kids[i]].box;
                for (int a = 0; a < 3; ++a) {
                    double sc = std::ldexp(1.0, exps[a]);
                    double hi = std::ceil((double(kb.hi[a]) - double(wn.p[a])) / sc + 1e-4);
                    if (hi > 255.0) {
                        exps[a]++;
                        ok = false;
                        break;
                    }
                }
            }
            if (ok) break;
        }
        for (int a = 0; a < 3; ++a) wn.e[a] = uint8_t(exps[a] + 127);

        uint32_t inner = 0;
        for (size_t i = 0; i < kids.size(); ++i) {
            if (!is_leaf(kids[i])) inner++;
        }
        wn.base_child = uint32_t(out.nodes.size());
        wn.base_tri = uint32_t(out.tris.size() / 12);
        uint32_t next_child = wn.base_child;
        uint32_t tri_off = 0;
        std::vector<Pending> spawn;
        for (int s = 0; s < 8; ++s) {
            int i = kid_in_slot[s];
            if (i < 0) continue;
            const Node2& k = b.nodes[kids[i]];
            for (int a = 0; a < 3; ++a) {
                double sc = std::ldexp(1.0, exps[a]);
                double lo = std::floor((double(k.box.lo[a]) - double(wn.p[a])) / sc - 1e-4);
                double hi = std::ceil((double(k.box.hi[a]) - double(wn.p[a])) / sc + 1e-4);
                uint8_t ql = uint8_t(std::max(0.0, std::min(255.0, lo)));
                uint8_t qh = uint8_t(std::max(0.0, std::min(255.0, hi)));
                if (a == 0) { wn.qlo_x[s] = ql; wn.qhi_x[s] = qh; }
                if (a == 1) { wn.qlo_y[s] = ql; wn.qhi_y[s] = qh; }
                if (a == 2) { wn.qlo_z[s] = ql; wn.qhi_z[s] = qh; }
            }
            if (is_leaf(kids[i])) {
                std::vector<uint32_t> leaf;
                b.gather(kids[i], leaf);
                uint32_t cnt = uint32_t(leaf.size());  // 1..3
                wn.meta[s] = uint8_t((((1u << cnt) - 1u) << 5) | tri_off);
                for (uint32_t t : leaf) put_tri(out.tris, tris[t]);
                tri_off += cnt;
            } else {
                wn.imask |= uint8_t(1u << s);
                wn.meta[s] = uint8_t((1u << 5) | (24u + uint32_t(s)));
                spawn.push_back({kids[i], next_child++, job.depth + 1});
            }
        }
        out.nodes.resize(out.nodes.size() + inner);
        out.nodes[job.wide] = wn;
        for (const Pending& p : spawn) queue.push_back(p);
    }
    // Stack entries a walk's node groups can need: a node with two or more
    // inner children may leave a group on the stack while one child is
    // walked. Children follow their parents (breadth first), so one pass
    // from the back sees every child before its parent.
    std::vector<uint32_t> need(out.nodes.size(), 0);
    for (size_t i = out.nodes.size(); i-- > 0;) {
        const WideNode& w = out.nodes[i];
        const uint32_t inner = uint32_t(__builtin_popcount(w.imask));
        uint32_t m = 0;
        for (uint32_t k = 0; k < inner; ++k) m = std::max(m, need[w.base_child + k]);
        need[i] = m + (inner >= 2 ? 1u : 0u);
    }
    out.stack_need = need.empty() ? 0u : need[0];
    return out;
}

}  // namespace cn
