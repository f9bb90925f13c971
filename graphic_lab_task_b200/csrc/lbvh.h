// lbvh.h — the device tree builder used for the BUILD_LOW build quality.
#pragma once
#include <stdint.h>

#include <functional>
#include <vector>

namespace lrt {

// Inner node i of the binary radix tree over the Morton-sorted boxes.  kid[c]
// is an inner node index, or a leaf (a position in the sorted order) with
// the top bit set.  [first, last] is the node's range of sorted positions;
// lo/hi its box (the union of its boxes).
struct LbvhInner {
  float lo[3], hi[3];
  uint32_t kid[2];
  uint32_t first, last;
};

// Builds the tree over n boxes (n x {lo.xyz, hi.xyz}, host memory) on the
// current CUDA device and returns it to the host: order[p] is the box at
// sorted position p, inner has n - 1 nodes with the root at 0 (none when
// n == 1).  Returns nullptr on success, else a message.
const char* lbvh_build(const float* boxes6, uint32_t n, std::vector<uint32_t>& order, std::vector<LbvhInner>& inner);

// One BLAS node pair as the reference stores it (BVHNodePair, cbvh.h:21-33):
// per child {boxMin.xyz, leftOffset, boxMax.xyz, escapeIndex}.
struct LbvhPairOut {
  float node[2][8];
};

// Builds the tree as lbvh_build does and emits a triangle BLAS from it on the
// device, exactly as the host emitter would from the same tree with inner
// nodes of at most maxLeaf boxes collapsed into leaves: the pairs (relative
// child indices; copied to pairsAt(count), which the caller makes room for),
// the leaf table entries Pack(start, count) in leaf-id order (`startCount`)
// and the box order of the leaves (`order`: position -> box).  Needs
// n > maxLeaf (a root that is one leaf has no pairs to emit).  Returns nullptr
// on success, else a message.
const char* lbvh_build_blas(const float* boxes6, uint32_t n, uint32_t maxLeaf,
                            const std::function<LbvhPairOut*(size_t)>& pairsAt, std::vector<uint32_t>& startCount,
                            std::vector<uint32_t>& order);

} // namespace lrt
