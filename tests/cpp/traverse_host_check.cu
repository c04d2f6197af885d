// traverse_host_check.cu -- runs the ray-query device code (traverse.cuh) on the CPU.
//
// The traversal functions are host/device code; this program compiles them for the host (nvcc,
// host code only: no kernel is launched, no device is needed) and traces a ray set with both
// device forms of the walk -- traverse() (one thread per ray: the fused path kernels, the
// one-thread-per-ray query kernel) and the resumable walk_begin / walk_step / walk_leaf (the
// persistent kernels) -- so that tests/test_traverse_host_cpu.py can compare both, bit for bit and
// count for count, with the oracle.  exact_tree = 1 forces the compare-and-select box test on
// every ray (the form a tree with a NaN box takes).
//
// usage: traverse_host_check NODES TRIS RAYS OUT EXACT_TREE
//   NODES  32-byte node records (pt_bvh_node), TRIS 48-byte leaf-ordered face records,
//   RAYS   32-byte pt_ray records; OUT receives per ray, for traverse() then for the walk:
//          {prim, t bits, u bits, v bits, node tests, face tests} as 6 x uint32.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "traverse.cuh"

using namespace pt;

template <class T>
static bool read_all(const char* path, std::vector<T>& v) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    v.resize((size_t)n / sizeof(T));
    const bool ok = std::fread(v.data(), sizeof(T), v.size(), f) == v.size();
    std::fclose(f);
    return ok;
}

struct Ray {
    float o[3], tmax, d[3];
    uint32_t flags;
};

int main(int argc, char** argv) {
    if (argc != 6) {
        std::fprintf(stderr, "usage: %s NODES TRIS RAYS OUT EXACT_TREE\n", argv[0]);
        return 2;
    }
    std::vector<uint4> nodes;
    std::vector<float4> tris;
    std::vector<Ray> rays;
    if (!read_all(argv[1], nodes) || !read_all(argv[2], tris) || !read_all(argv[3], rays)) {
        std::fprintf(stderr, "cannot read the inputs\n");
        return 2;
    }
    const bool exact = std::atoi(argv[5]) != 0;
    const uint32_t num_nodes = (uint32_t)(nodes.size() / 2);
    std::vector<uint32_t> out(12 * rays.size());
    for (size_t i = 0; i < rays.size(); ++i) {
        const Ray& ry = rays[i];
        const bool any = (ry.flags & 1u) != 0;
        RayState r;
        ray_setup(r, ry.o[0], ry.o[1], ry.o[2], ry.d[0], ry.d[1], ry.d[2]);
        const TraceResult t = traverse<true>(nodes.data(), tris.data(), num_nodes, r, ry.tmax, any, exact);
        uint32_t* o = &out[12 * i];
        o[0] = t.overflow ? 0xFFFFFFFEu : t.prim;
        o[1] = fbits(t.t);
        o[2] = fbits(t.u);
        o[3] = fbits(t.v);
        o[4] = t.nodes;
        o[5] = t.tris;
        RayWalkT<kStackCap, 0> k;
        walk_begin(k, ry.o[0], ry.o[1], ry.o[2], ry.d[0], ry.d[1], ry.d[2], ry.tmax, any, exact);
        bool ok = true;
        while (ok && !k.done && k.sp > 0) {
            uint32_t off = 0, cnt = 0;
            const int st = walk_step<true>(k, nodes.data(), num_nodes, off, cnt);
            if (st < 0) ok = false;
            else if (st > 0) walk_leaf<true>(k, tris.data(), off, cnt);
        }
        o[6] = ok ? k.prim : 0xFFFFFFFEu;
        o[7] = fbits(k.min_t);
        o[8] = fbits(k.u);
        o[9] = fbits(k.v);
        o[10] = k.nodes;
        o[11] = k.tris;
    }
    FILE* f = std::fopen(argv[4], "wb");
    if (!f || std::fwrite(out.data(), sizeof(uint32_t), out.size(), f) != out.size()) {
        std::fprintf(stderr, "cannot write %s\n", argv[4]);
        return 2;
    }
    std::fclose(f);
    return 0;
}
