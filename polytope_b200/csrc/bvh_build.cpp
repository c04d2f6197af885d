// bvh_build.cpp -- host SAH build that reproduces the reference tree node for node.
//
// Reference: poly::bvh::bound (src/cpu/acceleration/bvh.cpp:36-395) and poly::bvh::compact /
// compact_helper (bvh.cpp:652-698).  The reference builds breadth-first, copying every node's
// index vector several times; this builder partitions one index array in place (a stable
// counting sort by bucket keeps each child's element order equal to the reference's
// bucket-concatenation order) and builds large subtrees on several host threads.  Every float
// expression that decides the tree is evaluated with the reference's operand order, and the
// build is compiled with -ffp-contract=off, so decisions and boxes are bit-identical.  Min/max
// folds use the reference's ternaries in the reference's element order ("last equal wins" also
// for +0/-0), so even signed zeros in the boxes match.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <future>
#include <limits>
#include <memory>
#include <thread>

#include "pt_internal.h"

namespace pt {

namespace {

constexpr float kInf = std::numeric_limits<float>::infinity();
constexpr float kFloatMax = std::numeric_limits<float>::max();

inline float sum_prod(float a, float b, float c, float d) {  // constants.h:128-133
    const float cd = c * d;
    const float sop = std::fma(a, b, cd);
    const float err = std::fma(c, d, -cd);
    return sop + err;
}

struct Box {
    float lo[3], hi[3];
};

inline void box_empty(Box& b) {
    for (int k = 0; k < 3; ++k) { b.lo[k] = kInf; b.hi[k] = -kInf; }
}
// BoundingBox::UnionInPlace(const BoundingBox&) (BoundingBox.cpp:136-144): the running value is
// kept only when strictly smaller (larger), so ties take the incoming value.
inline void box_union(Box& a, const Box& b) {
    for (int k = 0; k < 3; ++k) {
        a.lo[k] = a.lo[k] < b.lo[k] ? a.lo[k] : b.lo[k];
        a.hi[k] = a.hi[k] > b.hi[k] ? a.hi[k] : b.hi[k];
    }
}
// BoundingBox::surface_area (BoundingBox.cpp:146-152)
inline float box_area(const Box& b) {
    const float x = b.hi[0] - b.lo[0], y = b.hi[1] - b.lo[1], z = b.hi[2] - b.lo[2];
    return (2 * x * y) + (2 * y * z) + (2 * z * x);
}

struct Node {  // trivial, so the 2n-node pool is allocated without being initialised
    Box bb;
    int32_t low, high;            // -1: leaf
    uint16_t axis;
    uint32_t begin, end;          // element range
};

inline void node_init(Node& n, const Box& bb, uint32_t begin, uint32_t end) {
    n.bb = bb;
    n.low = n.high = -1;
    n.axis = 0;
    n.begin = begin;
    n.end = end;
}

struct Builder {
    const WorldMeshes& w;
    std::vector<Box> pbox;        // face box by prim id (bvh.cpp:84-97)
    std::vector<float> pcen;      // 3 * prim: box centroid (bvh.cpp:110-113)
    std::vector<uint32_t> idx;    // element order (prim ids)
    std::vector<uint32_t> tmp;
    std::vector<uint8_t> bkt;
    std::unique_ptr<Node[]> nodes;
    std::atomic<uint32_t> next{0};
    int spawn_depth = 0;

    explicit Builder(const WorldMeshes& wm) : w(wm) {}

    uint32_t alloc2() { return next.fetch_add(2, std::memory_order_relaxed); }

    // One node of the breadth-first loop of bvh::bound (bvh.cpp:133-391), applied to the
    // element range [b, e).  Returns true when the node was split.
    bool split(uint32_t ni, uint32_t& low, uint32_t& high) {
        Node& node = nodes[ni];
        const uint32_t b = node.begin, e = node.end;
        const uint32_t n = e - b;
        if (n == 1) return false;                          // stop case 1
        const float sa = box_area(node.bb);
        if (sa == 0.f) return false;                       // stop case 2
        const float inv_sa = 1.f / sa;
        float cmin[3] = {kInf, kInf, kInf}, cmax[3] = {-kInf, -kInf, -kInf};
        for (uint32_t i = b; i < e; ++i) {
            const float* c = &pcen[3 * (size_t)idx[i]];
            for (int k = 0; k < 3; ++k) {
                cmin[k] = cmin[k] < c[k] ? cmin[k] : c[k];
                cmax[k] = cmax[k] > c[k] ? cmax[k] : c[k];
            }
        }
        const float ext[3] = {cmax[0] - cmin[0], cmax[1] - cmin[1], cmax[2] - cmin[2]};
        if (ext[0] == ext[1] && ext[1] == ext[2] && ext[2] == 0.f) return false;  // stop case 3
        int axis;
        if (ext[0] >= ext[1] && ext[0] >= ext[2]) axis = 0;
        else if (ext[1] >= ext[0] && ext[1] >= ext[2]) axis = 1;
        else axis = 2;
        const float width = ext[axis] / (float)12;
        const float amin = cmin[axis];
        // bucket assignment (bvh.cpp:231-244) + per-bucket boxes folded in element order
        uint32_t count[12] = {0};
        Box bbox[12];
        for (int k = 0; k < 12; ++k) box_empty(bbox[k]);
        for (uint32_t i = b; i < e; ++i) {
            const uint32_t p = idx[i];
            const float raw = (pcen[3 * (size_t)p + axis] - amin) / (float)width;
            unsigned bi = (unsigned)raw;
            if (bi >= 12) bi = 11;  // 12 at the top edge (the reference's bi--); NaN centroids stay in range
            bkt[i] = (uint8_t)bi;
            count[bi]++;
            box_union(bbox[bi], pbox[p]);
        }
        // forward scan (bvh.cpp:251-287) and backward scan (bvh.cpp:289-317)
        float fwd[12], bwd[12];
        Box lowbb[12], highbb[12];
        Box run;
        box_empty(run);
        float cnt = 0.f;
        for (int k = 0; k < 12; ++k) {
            box_union(run, bbox[k]);
            lowbb[k] = run;
            cnt += (float)count[k];
            const float cost = box_area(run) * inv_sa * cnt * 1.f;
            fwd[k] = cost == 0 ? kInf : cost;
        }
        box_empty(run);
        cnt = 0.f;
        for (int k = 11; k >= 0; --k) {
            box_union(run, bbox[k]);
            highbb[k] = run;
            cnt += (float)count[k];
            const float cost = box_area(run) * inv_sa * cnt * 1.f;
            bwd[11 - k] = cost == 0 ? kInf : cost;
        }
        float total[11];
        for (int k = 0; k < 11; ++k) total[k] = 1.f + fwd[k] + bwd[10 - k];
        const float leaf_cost = (float)n * 1.f;
        bool make_leaf = true;
        for (int k = 0; k < 11; ++k)
            if (leaf_cost > total[k]) make_leaf = false;
        if (make_leaf && n <= 4) return false;             // stop case 5
        int best = 0;
        float best_cost = kFloatMax;
        for (int k = 0; k < 11; ++k)
            if (total[k] < best_cost) { best_cost = total[k]; best = k; }
        uint32_t nlow = 0;
        for (int k = 0; k <= best; ++k) nlow += count[k];
        node.axis = (uint16_t)axis;
        if (nlow == n || nlow == 0) return false;          // no progress (bvh.cpp:366-369)
        // stable partition by bucket (children keep the reference's concatenation order)
        uint32_t start[12];
        uint32_t s = b;
        for (int k = 0; k < 12; ++k) { start[k] = s; s += count[k]; }
        for (uint32_t i = b; i < e; ++i) tmp[start[bkt[i]]++] = idx[i];
        std::memcpy(&idx[b], &tmp[b], sizeof(uint32_t) * n);
        const uint32_t c = alloc2();
        high = c;
        low = c + 1;
        node_init(nodes[high], highbb[best + 1], b + nlow, e);
        node_init(nodes[low], lowbb[best], b, b + nlow);
        node.high = (int32_t)high;
        node.low = (int32_t)low;
        return true;
    }

    void build_subtree(uint32_t root, int depth) {
        std::vector<uint32_t> stack{root};
        while (!stack.empty()) {
            const uint32_t ni = stack.back();
            stack.pop_back();
            uint32_t lo, hi;
            if (!split(ni, lo, hi)) continue;
            const uint32_t nlo = nodes[lo].end - nodes[lo].begin;
            const uint32_t nhi = nodes[hi].end - nodes[hi].begin;
            if (depth < spawn_depth && nlo > 20000 && nhi > 20000) {
                auto fut = std::async(std::launch::async, [this, lo, depth]() { build_subtree(lo, depth + 1); });
                build_subtree(hi, depth + 1);
                fut.get();
                continue;
            }
            stack.push_back(lo);
            stack.push_back(hi);
        }
    }
};

// The reference's in-leaf comparator (bvh.cpp:666-671), kept verbatim in behaviour: when the mesh
// indices differ it compares lhs.first with lhs.second.  It is not a strict weak order, so the
// leaf order it produces is whatever libstdc++'s std::sort makes of it -- the same call is used
// here so that the order is the reference's.
struct LeafLess {
    bool operator()(const std::pair<uint32_t, uint32_t>& l, const std::pair<uint32_t, uint32_t>& r) const {
        if (l.first == r.first) return l.second < r.second;
        return l.first < l.second;
    }
};

}  // namespace

void apply_point(const float* m, float p[3]) {  // Transform::ApplyInPlace(Point&), Transform.cpp:69-91
    const float x = p[0], y = p[1], z = p[2];
    const float nx = sum_prod(x, m[0], y, m[1]) + std::fma(z, m[2], m[3]);
    const float ny = sum_prod(x, m[4], y, m[5]) + std::fma(z, m[6], m[7]);
    const float nz = sum_prod(x, m[8], y, m[9]) + std::fma(z, m[10], m[11]);
    const float w = sum_prod(x, m[12], y, m[13]) + std::fma(z, m[14], m[15]);
    if (w == 1) {
        p[0] = nx; p[1] = ny; p[2] = nz;
    } else {
        const float div = 1.f / w;
        p[0] = nx * div; p[1] = ny * div; p[2] = nz * div;
    }
}

void apply_normal(const float* inv, float n[3]) {  // Transform::ApplyInPlace(Normal&), Transform.cpp:135-143
    const float x = n[0], y = n[1], z = n[2];
    n[0] = x * inv[0] + y * inv[4] + z * inv[8];
    n[1] = x * inv[1] + y * inv[5] + z * inv[9];
    n[2] = x * inv[2] + y * inv[6] + z * inv[10];
}

int bake_world(const pt_mesh_desc* meshes, uint32_t num_meshes, WorldMeshes& out) {
    uint64_t total = 0;
    out.prim_base.assign(num_meshes, 0);
    for (uint32_t m = 0; m < num_meshes; ++m) {
        const pt_mesh_desc& d = meshes[m];
        if (d.num_faces && (!d.x || !d.y || !d.z || !d.fv0 || !d.fv1 || !d.fv2))
            return fail(PT_EINVAL, "mesh " + std::to_string(m) + ": NULL vertex or face array");
        out.prim_base[m] = (uint32_t)total;
        total += d.num_faces;
        if (total >= 0xFFFFFFFFull) return fail(PT_EINVAL, "more than 2^32-2 faces");
    }
    out.num_prims = (uint32_t)total;
    out.tri.resize(9 * total);
    out.prim_mesh.resize(total);
    // every face independently, in parallel; the first bad face in prim order is the one reported
    std::atomic<uint64_t> first_bad{~0ull};
    parallel_ranges((size_t)total, 0, [&](size_t pb, size_t pe) {
        uint32_t m = (uint32_t)(std::upper_bound(out.prim_base.begin(), out.prim_base.end(), (uint32_t)pb) -
                                out.prim_base.begin()) - 1;
        for (size_t p = pb; p < pe; ++p) {
            while (m + 1 < num_meshes && p >= out.prim_base[m + 1]) ++m;
            const pt_mesh_desc& d = meshes[m];
            const uint32_t f = (uint32_t)(p - out.prim_base[m]);
            const uint32_t vi[3] = {d.fv0[f], d.fv1[f], d.fv2[f]};
            float* t = &out.tri[9 * p];
            for (int k = 0; k < 3; ++k) {
                if (vi[k] >= d.num_vertices) {
                    uint64_t cur = first_bad.load();
                    while (p < cur && !first_bad.compare_exchange_weak(cur, p)) {}
                    return;
                }
                t[3 * k + 0] = d.x[vi[k]];
                t[3 * k + 1] = d.y[vi[k]];
                t[3 * k + 2] = d.z[vi[k]];
                apply_point(d.object_to_world, &t[3 * k]);
            }
            out.prim_mesh[p] = m;
        }
    });
    if (first_bad.load() != ~0ull) {
        const uint64_t p = first_bad.load();
        const uint32_t m = (uint32_t)(std::upper_bound(out.prim_base.begin(), out.prim_base.end(), (uint32_t)p) -
                                      out.prim_base.begin()) - 1;
        return fail(PT_EINVAL, "mesh " + std::to_string(m) + " face " + std::to_string(p - out.prim_base[m]) +
                                   ": vertex index out of range");
    }
    return PT_OK;
}

int build_bvh(const pt_mesh_desc* meshes, uint32_t num_meshes, const WorldMeshes& w, int threads, BuiltTree& out) {
    const uint32_t n = w.num_prims;
    if (n == 0) return fail(PT_EINVAL, "scene has no faces (the reference's bvh::bound is undefined for it)");
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    Builder B(w);
    B.pbox.resize(n);
    B.pcen.resize(3 * (size_t)n);
    // face boxes and centroids (bvh.cpp:53-121), each face on its own, in parallel
    parallel_ranges(n, threads, [&](size_t pb, size_t pe) {
        for (size_t p = pb; p < pe; ++p) {
            const float* t = &w.tri[9 * p];
            Box& b = B.pbox[p];
            for (int k = 0; k < 3; ++k) {
                float mn = t[k] < t[3 + k] ? t[k] : t[3 + k];
                mn = mn < t[6 + k] ? mn : t[6 + k];
                float mx = t[k] > t[3 + k] ? t[k] : t[3 + k];
                mx = mx > t[6 + k] ? mx : t[6 + k];
                b.lo[k] = mn;
                b.hi[k] = mx;
                B.pcen[3 * p + k] = (mn + mx) * .5f;
            }
        }
    });
    // the root box folds the face boxes in element order, on one thread, so that ties (and signed
    // zeros, and NaN) resolve exactly as in the reference's sequential loop
    Box root_bb;
    box_empty(root_bb);
    for (uint32_t p = 0; p < n; ++p) {
        const Box& b = B.pbox[p];
        for (int k = 0; k < 3; ++k) {
            root_bb.lo[k] = root_bb.lo[k] < b.lo[k] ? root_bb.lo[k] : b.lo[k];
            root_bb.hi[k] = root_bb.hi[k] > b.hi[k] ? root_bb.hi[k] : b.hi[k];
        }
    }
    B.idx.resize(n);
    for (uint32_t p = 0; p < n; ++p) B.idx[p] = p;  // master_indices order (mesh, then face)
    B.tmp.resize(n);
    B.bkt.resize(n);
    B.nodes.reset(new Node[2 * (size_t)n]);
    node_init(B.nodes[0], root_bb, 0, n);
    B.next.store(1);
    int sd = 0;
    while ((1 << sd) < threads) ++sd;
    B.spawn_depth = threads > 1 ? sd + 1 : 0;
    B.build_subtree(0, 0);

    // compact_helper (bvh.cpp:652-693): pre-order DFS, low child at index + 1, high child at
    // index + high_child_offset; leaves append their (sorted) pairs to leaf_ordered_indices.
    // Every node's output position is known up front -- its pre-order index follows from the
    // subtree sizes, and a leaf's pairs start at its first element (the stable partition keeps the
    // leaves' elements in pre-order), so subtrees are written in parallel with the same result.
    const uint32_t total_nodes = B.next.load();
    out.nodes.assign(total_nodes, pt_bvh_node{});
    out.leaf_pairs.assign(2 * (size_t)n, 0u);
    std::vector<uint32_t> sub(total_nodes, 0);
    // subtree sizes (descendant counts) by a reverse pass: children are always allocated after
    // their parent, so a descending sweep sees children first.
    for (uint32_t i = total_nodes; i-- > 0;) {
        const Node& nd = B.nodes[i];
        if (nd.low >= 0) sub[i] = 2 + sub[nd.low] + sub[nd.high];
    }
    struct Item { uint32_t tn, index, depth; };
    std::atomic<bool> leaf_too_big{false};
    // writes one node; returns true for an interior node, whose children the caller visits
    auto emit = [&](const Item& it, std::vector<std::pair<uint32_t, uint32_t>>& leaf) {
        const Node& nd = B.nodes[it.tn];
        pt_bvh_node& cn = out.nodes[it.index];
        for (int k = 0; k < 3; ++k) { cn.bb_min[k] = nd.bb.lo[k]; cn.bb_max[k] = nd.bb.hi[k]; }
        cn.axis = nd.axis;
        if (nd.low < 0) {
            cn.offset = nd.begin;
            leaf.clear();
            for (uint32_t i = nd.begin; i < nd.end; ++i) {
                const uint32_t p = B.idx[i];
                const uint32_t m = w.prim_mesh[p];
                leaf.emplace_back(m, p - w.prim_base[m]);
            }
            if (leaf.size() > 65535) {  // the 16-bit num_faces of the record cannot hold it
                leaf_too_big.store(true);
                return false;
            }
            // LeafLess is not a strict weak order when meshes differ.  libstdc++'s std::sort only
            // runs its bounds-safe insertion sort on 16 elements or fewer; on a longer leaf that
            // mixes meshes its unguarded partition can step past the leaf (undefined behaviour in
            // the reference, which crashes on such scenes), so those leaves are sorted by (mesh,
            // face) instead.
            bool mixed = false;
            for (const auto& pr : leaf) mixed = mixed || pr.first != leaf[0].first;
            if (leaf.size() > 16 && mixed) std::sort(leaf.begin(), leaf.end());
            else std::sort(leaf.begin(), leaf.end(), LeafLess());
            uint32_t* dst = &out.leaf_pairs[2 * (size_t)nd.begin];
            for (const auto& pr : leaf) { *dst++ = pr.first; *dst++ = pr.second; }
            cn.num_faces = (uint16_t)leaf.size();
            return false;
        }
        cn.offset = 2 + sub[nd.low];
        cn.num_faces = 0;
        return true;
    };
    auto children = [&](const Item& it, Item& lo, Item& hi) {
        const Node& nd = B.nodes[it.tn];
        lo = {(uint32_t)nd.low, it.index + 1, it.depth + 1};
        hi = {(uint32_t)nd.high, it.index + 2 + sub[nd.low], it.depth + 1};
    };
    // the top of the tree on this thread, down to subtrees of at most `grain` nodes
    const uint32_t grain = std::max<uint32_t>(4096, total_nodes / (uint32_t)(8 * threads));
    std::vector<Item> tasks, st{{0, 0, 0}};
    std::vector<std::pair<uint32_t, uint32_t>> leaf;
    uint32_t max_depth = 0;
    while (!st.empty()) {
        const Item it = st.back();
        st.pop_back();
        if (sub[it.tn] + 1 <= grain) { tasks.push_back(it); continue; }
        max_depth = std::max(max_depth, it.depth);
        if (!emit(it, leaf)) continue;
        Item lo, hi;
        children(it, lo, hi);
        st.push_back(hi);
        st.push_back(lo);
    }
    std::atomic<size_t> next_task{0};
    std::atomic<uint32_t> deepest{max_depth};
    auto worker = [&]() {
        std::vector<Item> stack;
        std::vector<std::pair<uint32_t, uint32_t>> lp;
        uint32_t dmax = 0;
        for (size_t t; (t = next_task.fetch_add(1)) < tasks.size();) {
            stack.assign(1, tasks[t]);
            while (!stack.empty()) {
                const Item it = stack.back();
                stack.pop_back();
                dmax = std::max(dmax, it.depth);
                if (!emit(it, lp)) continue;
                Item lo, hi;
                children(it, lo, hi);
                stack.push_back(hi);
                stack.push_back(lo);
            }
        }
        uint32_t cur = deepest.load();
        while (dmax > cur && !deepest.compare_exchange_weak(cur, dmax)) {}
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (std::thread& th : pool) th.join();
    max_depth = deepest.load();
    if (leaf_too_big.load())
        return fail(PT_EINVAL, "a leaf would hold more than 65535 faces (faces whose centroids coincide)");
    out.max_depth = max_depth;
    (void)meshes;
    (void)num_meshes;
    return PT_OK;
}

int validate_tree(const pt_bvh_node* nodes, uint32_t num_nodes, uint32_t num_leaf_entries, uint32_t* max_depth_out) {
    if (num_nodes == 0) return fail(PT_EINVAL, "empty tree");
    std::vector<uint32_t> depth(num_nodes, 0);
    std::vector<uint8_t> seen(num_nodes, 0);
    seen[0] = 1;
    uint32_t max_depth = 0;
    // Pre-order layout: every child index is larger than its parent's, so one forward sweep
    // visits parents first.
    for (uint32_t i = 0; i < num_nodes; ++i) {
        if (!seen[i]) continue;
        const pt_bvh_node& n = nodes[i];
        max_depth = std::max(max_depth, depth[i]);
        if (n.num_faces > 0) {
            if ((uint64_t)n.offset + n.num_faces > num_leaf_entries)
                return fail(PT_EINVAL, "leaf " + std::to_string(i) + " face range out of bounds");
            continue;
        }
        if (n.axis > 2) return fail(PT_EINVAL, "node " + std::to_string(i) + ": bad split axis");
        const uint64_t lo = (uint64_t)i + 1, hi = (uint64_t)i + n.offset;
        if (n.offset < 2 || hi >= num_nodes || lo >= num_nodes)
            return fail(PT_EINVAL, "node " + std::to_string(i) + ": child index out of bounds");
        seen[lo] = seen[hi] = 1;
        depth[lo] = depth[hi] = depth[i] + 1;
    }
    if (max_depth_out) *max_depth_out = max_depth;
    return PT_OK;
}

}  // namespace pt
