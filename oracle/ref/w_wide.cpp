// The reference's N-wide collapse (rt/bvh/BVH.h: recomputeCostsWide,
// collapseWide, collapseAdaptiveWide), compiled on the host from its source
// tree (test infrastructure only). Around it, restated:
//   * BVHCollapser::convert (rt/bvh/BVHCollapser.cpp:339-413): the binary tree
//     (left/right children, node boxes, leaf j = n-1+p holding sorted reference
//     p) becomes a host BVH, and writeTriangleIndices (:497-519) renumbers the
//     references in left-first depth-first order;
//   * BVHConverter::convert (rt/bvh/BVHConverter.cpp:13-89): breadth-first
//     numbering into the reference's own HipBVHNodeN<N> records (unused words
//     zero here; the reference leaves them uninitialised).
// Headers that BVH.h includes for other purposes (HipBVH.h, the environment,
// the logger) are skipped through their include guards; Bvh.ct / Bvh.ci come
// from the stand-in Environment below.
#define _HIP_BVH_H_
#define _APP_ENVIRONMENT_H_
#define _LOGGER_H_
#include <algorithm>
#include <cstring>
#include <vector>

#define CT 3.0f
#define CI 3.0f
#define Q_ASSERT(x) ((void)0)
template <typename T> inline const T& qMax(const T& a, const T& b) { return std::max(a, b); }
template <typename T> inline const T& qMin(const T& a, const T& b) { return std::min(a, b); }

static float g_ct = 3.0f, g_ci = 2.0f;
class Environment {
public:
    static Environment* getInstance() {
        static Environment e;
        return &e;
    }
    bool getFloatValue(const char* name, float& v) {
        v = std::strcmp(name, "Bvh.ct") == 0 ? g_ct : (std::strcmp(name, "Bvh.ci") == 0 ? g_ci : 0.0f);
        return true;
    }
};

#include "util/AABB.h"
#include "rt/bvh/BVH.h"
#include "rt/bvh/HipBVHNode.h"

// Named as one of BVH's friends to reach its private tree.
class BVHImporter {
public:
    static BVH* from_binary(int n, const int* left, const int* right, const float* bmin4, const float* bmax4,
                            const int* sorted_tri) {
        BVH* bvh = new BVH();
        bvh->root = new BVH::InteriorNode();
        bvh->numberOfInteriorNodes = n - 1;
        bvh->numberOfLeafNodes = n;
        std::vector<std::pair<int, BVH::Node*>> stack{{0, bvh->root}};
        while (!stack.empty()) {
            const int v = stack.back().first;
            BVH::Node* node = stack.back().second;
            stack.pop_back();
            node->box = AABB(Vec3f(bmin4[4 * v], bmin4[4 * v + 1], bmin4[4 * v + 2]),
                             Vec3f(bmax4[4 * v], bmax4[4 * v + 1], bmax4[4 * v + 2]));
            if (v >= n - 1) {
                node->begin = v - (n - 1);
                node->end = v - (n - 1) + 1;
            } else {
                BVH::InteriorNode* in = dynamic_cast<BVH::InteriorNode*>(node);
                const int c[2] = {left[v], right[v]};
                for (int i = 0; i < 2; ++i) {
                    if (c[i] >= n - 1) in->children[i] = new BVH::LeafNode();
                    else in->children[i] = new BVH::InteriorNode();
                    stack.push_back({c[i], in->children[i]});
                }
            }
        }
        bvh->recomputeDepth();
        bvh->recomputeIDs();
        bvh->recomputeParents();
        bvh->recomputeBounds();
        int offset = 0;
        bvh->triangleIndices.resize(n);
        write(bvh->root, sorted_tri, bvh->triangleIndices.data(), offset);
        return bvh;
    }

    static void write(BVH::Node* node, const int* src, int* dst, int& offset) {
        if (node->isLeaf()) {
            const int o = offset;
            for (int i = node->begin; i < node->end; ++i) dst[offset++] = src[i];
            node->begin = o;
            node->end = offset;
        } else {
            BVH::InteriorNode* in = dynamic_cast<BVH::InteriorNode*>(node);
            node->begin = offset;
            for (int i = 0; i < 2; ++i) write(in->children[i], src, dst, offset);
            node->end = offset;
        }
    }

    template <typename HipBVHNode>
    static void dump(const BVH& bvh, int* nodes_out) {
        struct E {
            const BVH::Node* node;
            int index, parent;
        };
        std::vector<E> queue{{bvh.getRoot(), 0, -1}};
        int next_int = 1, next_leaf = bvh.getNumberOfInteriorNodes();
        for (size_t h = 0; h < queue.size(); ++h) {
            const E e = queue[h];
            HipBVHNode node;
            std::memset(&node, 0, sizeof(node));
            int size = e.node->end - e.node->begin, ccnt = 0;
            if (e.node->isLeaf()) {
                size = ~size;
                node.setBoundingBox(e.node->box);
                node.setBegin(e.node->begin);
                node.setEnd(e.node->end);
            } else {
                ccnt = e.node->getNumberOfChildNodes();
                for (int i = 0; i < ccnt; ++i) {
                    const BVH::Node* c = e.node->getChildNode(i);
                    const int idx = c->isLeaf() ? next_leaf++ : next_int++;
                    queue.push_back({c, idx, e.index});
                    node.setChildBoundingBox(i, c->box);
                    node.setChildIndex(i, c->isLeaf() ? ~idx : idx);
                }
                const AABB dummy(node.getChildBoundingBox(0).mn, node.getChildBoundingBox(0).mn);
                const int dummy_index = node.getChildIndex(0);
                for (int i = ccnt; i < HipBVHNode::N; ++i) {
                    node.setChildBoundingBox(i, dummy);
                    node.setChildIndex(i, dummy_index);
                }
            }
            node.setNumberOfChildren(ccnt);
            node.setSize(size);
            node.setParentIndex(e.parent);
            std::memcpy(nodes_out + (size_t)e.index * 8 * HipBVHNode::N, &node, sizeof(node));
        }
    }

    static int root_is_leaf(const BVH& bvh) { return bvh.getRoot()->count[0].x < 0; }
};

// Returns the node count (counts[0] interior, counts[1] leaves), or -1 when the
// root's best choice is a leaf (the reference's collapseWide then reads
// outside its count arrays).
extern "C" int hpref_wide_collapse(int n, const int* left, const int* right, const float* bmin4,
                                   const float* bmax4, const int* sorted_tri, int width, float ct, float ci,
                                   int adaptive, int max_leaf, int* nodes_out, int* tri_out, int* counts) {
    if (n < 2 || (width != 4 && width != 8)) return 0;
    g_ct = ct;
    g_ci = ci;
    BVH* bvh = BVHImporter::from_binary(n, left, right, bmin4, bmax4, sorted_tri);
    bvh->recomputeIDs();
    bvh->recomputeCostsWide(width, adaptive ? MAX_INT : max_leaf);
    if (BVHImporter::root_is_leaf(*bvh)) {
        delete bvh;
        return -1;
    }
    if (adaptive) bvh->collapseAdaptiveWide(width);
    else bvh->collapseWide(width, max_leaf);
    if (width == 4) BVHImporter::dump<HipBVHNodeN<4>>(*bvh, nodes_out);
    else BVHImporter::dump<HipBVHNodeN<8>>(*bvh, nodes_out);
    std::memcpy(tri_out, bvh->getTriangleIndices().data(), sizeof(int) * n);
    counts[0] = bvh->getNumberOfInteriorNodes();
    counts[1] = bvh->getNumberOfLeafNodes();
    const int total = counts[0] + counts[1];
    delete bvh;
    return total;
}
