// scene.cpp — host half of the scene object: geometry adders, instancing,
// TLAS commit, the drop-in array upload/export and structural validation.
//
// The adders reproduce how BVHRT's host code flattens geometry
// (MultiRenderer/BVH2Common_host.cpp: AddGeom_Triangles3f :307-359,
// AddGeom_AABB :441-459, AddGeom_SdfFrameOctree :501-534 with
// add_border_nodes_rec :1348-1390, AddGeom_SdfSVS :536-599,
// AddGeom_SdfSBS :601-695, AddInstance :1264-1301, CommitScene :1230-1262),
// so the arrays have the reference's meaning field by field.  The BVH
// topology comes from this file's own binned-SAH builder instead of Embree
// (utils/raytracing/cbvh_embree2.cpp); it emits the reference's layouts: fat
// node pairs in depth-first pre-order for BLAS (CreateFatTreeArray,
// cbvh_fat.cpp:128-142) and the pair-aligned escape-index array for the TLAS
// (AlignNodes2, cbvh.cpp:143-169).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>

#include "lbvh.h"
#include "scene.h"

namespace lrt {

lrt_status fail(lrt_scene* s, lrt_status code, const char* fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (s) s->err = buf;
  return code;
}

namespace {

// ---------------------------------------------------------------------------
// Binned-SAH BVH2 builder over boxes
// ---------------------------------------------------------------------------
struct Aabb {
  float lo[3], hi[3];
  void reset()
  {
    for (int k = 0; k < 3; k++) { lo[k] = FLT_MAX; hi[k] = -FLT_MAX; }
  }
  void grow(const Aabb& b)
  {
    for (int k = 0; k < 3; k++) { lo[k] = std::min(lo[k], b.lo[k]); hi[k] = std::max(hi[k], b.hi[k]); }
  }
  float area() const
  {
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    if (!(dx >= 0 && dy >= 0 && dz >= 0)) return 0.0f;
    return 2.0f * (dx * dy + dy * dz + dz * dx);
  }
};

struct BNode {
  Aabb box;
  int32_t kid[2] = {-1, -1};
  uint32_t start = 0, count = 0; // leaf range in `ids`
  bool leaf() const { return kid[0] < 0; }
};

struct SahBuilder {
  const std::vector<Aabb>& prim;
  std::vector<float> cent[3];
  std::vector<uint32_t> ids;
  std::vector<BNode> nodes;
  uint32_t maxLeaf;

  SahBuilder(const std::vector<Aabb>& p, uint32_t max_leaf) : prim(p), maxLeaf(std::max(1u, max_leaf))
  {
    const size_t n = p.size();
    for (int k = 0; k < 3; k++) cent[k].resize(n);
    ids.resize(n);
    for (size_t i = 0; i < n; i++) {
      for (int k = 0; k < 3; k++) cent[k][i] = 0.5f * (p[i].lo[k] + p[i].hi[k]);
      ids[i] = uint32_t(i);
    }
    nodes.reserve(2 * n + 1);
  }

  int32_t build(uint32_t b, uint32_t e)
  {
    const int32_t me = int32_t(nodes.size());
    nodes.emplace_back();
    Aabb box;
    box.reset();
    for (uint32_t i = b; i < e; i++) box.grow(prim[ids[i]]);
    nodes[me].box = box;
    if (e - b <= maxLeaf) {
      nodes[me].start = b;
      nodes[me].count = e - b;
      return me;
    }
    const uint32_t m = split(b, e);
    const int32_t l = build(b, m);
    const int32_t r = build(m, e);
    nodes[me].kid[0] = l;
    nodes[me].kid[1] = r;
    return me;
  }

  uint32_t split(uint32_t b, uint32_t e)
  {
    constexpr int NB = 32;
    float cmin[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, cmax[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = b; i < e; i++)
      for (int k = 0; k < 3; k++) {
        cmin[k] = std::min(cmin[k], cent[k][ids[i]]);
        cmax[k] = std::max(cmax[k], cent[k][ids[i]]);
      }
    float best = FLT_MAX;
    int bestAxis = -1, bestBin = 0;
    for (int k = 0; k < 3; k++) {
      const float ext = cmax[k] - cmin[k];
      if (!(ext > 0.0f)) continue;
      const float scale = NB / ext;
      Aabb bb[NB];
      uint32_t cnt[NB] = {0};
      for (int i = 0; i < NB; i++) bb[i].reset();
      for (uint32_t i = b; i < e; i++) {
        const int bin = std::min(NB - 1, std::max(0, int((cent[k][ids[i]] - cmin[k]) * scale)));
        cnt[bin]++;
        bb[bin].grow(prim[ids[i]]);
      }
      float rArea[NB];
      uint32_t rCnt[NB];
      Aabb acc;
      acc.reset();
      uint32_t c = 0;
      for (int i = NB - 1; i > 0; i--) {
        acc.grow(bb[i]);
        c += cnt[i];
        rArea[i] = acc.area();
        rCnt[i] = c;
      }
      acc.reset();
      c = 0;
      for (int i = 0; i < NB - 1; i++) {
        acc.grow(bb[i]);
        c += cnt[i];
        if (c == 0 || rCnt[i + 1] == 0) continue;
        const float cost = acc.area() * float(c) + rArea[i + 1] * float(rCnt[i + 1]);
        if (cost < best) { best = cost; bestAxis = k; bestBin = i; }
      }
    }
    if (bestAxis < 0) return b + (e - b) / 2;
    const float ext = cmax[bestAxis] - cmin[bestAxis];
    const float scale = NB / ext;
    auto mid = std::partition(ids.begin() + b, ids.begin() + e, [&](uint32_t id) {
      const int bin = std::min(NB - 1, std::max(0, int((cent[bestAxis][id] - cmin[bestAxis]) * scale)));
      return bin <= bestBin;
    });
    uint32_t m = uint32_t(mid - ids.begin());
    if (m == b || m == e) m = b + (e - b) / 2;
    return m;
  }
};

// The BUILD_LOW tree: a linear BVH built on the device (lbvh.cu) in the
// node form the emitters read (nodes[0] the root, leaf ranges in `ids`).
// Inner nodes of at most maxLeaf primitives become leaves, as SahBuilder
// stops at maxLeaf.
struct RadixTree {
  std::vector<uint32_t> ids;
  std::vector<BNode> nodes;

  // nullptr on success, else the device builder's message
  const char* build(const std::vector<Aabb>& prim, uint32_t maxLeaf)
  {
    maxLeaf = std::max(1u, maxLeaf);
    std::vector<LbvhInner> inner;
    static_assert(sizeof(Aabb) == 6 * sizeof(float), "Aabb is lo.xyz, hi.xyz");
    const char* err = lbvh_build(reinterpret_cast<const float*>(prim.data()), uint32_t(prim.size()), ids, inner);
    if (err) return err;
    nodes.clear();
    nodes.reserve(2 * prim.size());
    nodes.emplace_back();
    if (inner.empty()) { // one primitive
      nodes[0].box = prim[ids[0]];
      nodes[0].count = 1;
      return nullptr;
    }
    // depth-first from the root; `tree` is an inner index or a leaf position with the top bit set
    struct Item {
      uint32_t tree;
      int32_t node;
    };
    std::vector<Item> todo{{0u, 0}};
    while (!todo.empty()) {
      const Item it = todo.back();
      todo.pop_back();
      BNode& n = nodes[it.node];
      if (it.tree & 0x80000000u) {
        const uint32_t pos = it.tree & 0x7FFFFFFFu;
        n.box = prim[ids[pos]];
        n.start = pos;
        n.count = 1;
        continue;
      }
      const LbvhInner& in = inner[it.tree];
      for (int k = 0; k < 3; k++) {
        n.box.lo[k] = in.lo[k];
        n.box.hi[k] = in.hi[k];
      }
      if (in.last - in.first + 1 <= maxLeaf) {
        n.start = in.first;
        n.count = in.last - in.first + 1;
        continue;
      }
      for (int c = 0; c < 2; c++) {
        const int32_t id = int32_t(nodes.size());
        nodes[it.node].kid[c] = id; // `n` may move when nodes grows
        nodes.emplace_back();
        todo.push_back({in.kid[c], id});
      }
    }
    return nullptr;
  }
};

lrt_bvh_node make_node(const Aabb& b, uint32_t left, uint32_t esc)
{
  lrt_bvh_node n;
  for (int k = 0; k < 3; k++) { n.boxMin[k] = b.lo[k]; n.boxMax[k] = b.hi[k]; }
  n.leftOffset = left;
  n.escapeIndex = esc;
  return n;
}

// DummyNode, utils/raytracing/cbvh.cpp:49-57
lrt_bvh_node dummy_node()
{
  lrt_bvh_node n;
  for (int k = 0; k < 3; k++) { n.boxMin[k] = 0.0f; n.boxMax[k] = 0.0f; }
  n.leftOffset = 0x80000000u;
  n.escapeIndex = 0xFFFFFFFFu;
  return n;
}

// Emits a built tree as BLAS fat pairs (depth-first pre-order, children of the
// node stored in pair k are pair `leftOffset`).  `leafWord(node)` gives the
// packed leftOffset of a leaf.  escapeIndex follows the aligned-array
// convention of AlignNodes2 (left -> its right sibling, right -> parent's).
template <class Tree, class LeafWord>
void emit_pairs(const Tree& B, std::vector<lrt_bvh_node_pair>& out, LeafWord leafWord)
{
  const BNode& root = B.nodes[0];
  if (root.leaf()) {
    lrt_bvh_node_pair p;
    p.left = make_node(root.box, leafWord(0), 1);
    p.right = dummy_node();
    out.push_back(p);
    return;
  }
  struct Rec {
    static uint32_t go(const Tree& B, std::vector<lrt_bvh_node_pair>& out, int32_t node, uint32_t base,
                       uint32_t parentEsc, LeafWord& lw)
    {
      const BNode& n = B.nodes[node];
      const uint32_t k = uint32_t(out.size()) - base;
      out.emplace_back();
      const BNode& l = B.nodes[n.kid[0]];
      const BNode& r = B.nodes[n.kid[1]];
      out[base + k].left = make_node(l.box, l.leaf() ? lw(n.kid[0]) : 0u, 2 * k + 1);
      out[base + k].right = make_node(r.box, r.leaf() ? lw(n.kid[1]) : 0u, parentEsc);
      if (!l.leaf()) {
        const uint32_t c = go(B, out, n.kid[0], base, 2 * k + 1, lw);
        out[base + k].left.leftOffset = c;
      }
      if (!r.leaf()) {
        const uint32_t c = go(B, out, n.kid[1], base, parentEsc, lw);
        out[base + k].right.leftOffset = c;
      }
      return k;
    }
  };
  Rec::go(B, out, 0, uint32_t(out.size()), kEscapeRoot, leafWord);
}

// Emits a built tree as the TLAS node array: aligned pairs in depth-first
// pre-order, node 0/1 are the root's children, inner nodes point at their
// left child, escapeIndex gives the next node of a stackless traversal.
template <class Tree>
void emit_tlas(const Tree& B, std::vector<lrt_bvh_node>& out)
{
  struct Rec {
    static void go(const Tree& B, std::vector<lrt_bvh_node>& out, int32_t node, uint32_t parentEsc)
    {
      const BNode& n = B.nodes[node];
      const uint32_t k = uint32_t(out.size());
      out.push_back(lrt_bvh_node{});
      out.push_back(lrt_bvh_node{});
      for (int j = 0; j < 2; j++) {
        const BNode& c = B.nodes[n.kid[j]];
        const uint32_t esc = j == 0 ? k + 1 : parentEsc;
        out[k + j] = make_node(c.box, 0, esc);
        if (c.leaf()) out[k + j].leftOffset = pack_offset_and_size(B.ids[c.start], 1);
      }
      for (int j = 0; j < 2; j++) {
        const BNode& c = B.nodes[n.kid[j]];
        if (!c.leaf()) {
          out[k + j].leftOffset = uint32_t(out.size());
          go(B, out, n.kid[j], out[k + j].escapeIndex);
        }
      }
    }
  };
  Rec::go(B, out, 0, kEscapeRoot);
}

Aabb box_of(const float* mn, const float* mx)
{
  Aabb b;
  for (int k = 0; k < 3; k++) { b.lo[k] = mn[k]; b.hi[k] = mx[k]; }
  return b;
}

// AddGeom_AABB's BLAS part: one box per leaf, leaf word = Pack(boxIndex, 1)
// (BuildBVH(boxes), cbvh.cpp:650-660), identity leaf table (:451-453).
// BLAS of custom boxes, one box per leaf; BUILD_LOW builds the tree on the
// device.  ~0u if that build failed (the message is the scene's last error).
uint32_t add_aabb_blas(lrt_scene* s, uint32_t tag, const std::vector<Aabb>& boxes, uint32_t flags = 0)
{
  HostArrays& h = s->h;
  auto emit = [&](const auto& B) {
    emit_pairs(B, h.allNodePairs, [&](int32_t node) { return pack_offset_and_size(B.ids[B.nodes[node].start], 1); });
  };
  if (flags & LRT_BUILD_LOW) {
    RadixTree R;
    if (const char* err = R.build(boxes, 1)) {
      fail(s, LRT_ERR_CUDA, "AddGeom_AABB (BUILD_LOW): %s", err);
      return ~0u;
    }
    emit(R);
  } else {
    SahBuilder B(boxes, 1);
    B.build(0, uint32_t(boxes.size()));
    emit(B);
  }
  const uint32_t old = uint32_t(h.primIdCount.size());
  for (uint32_t i = 0; i < boxes.size(); i++) h.primIdCount.push_back(i);
  h.startEnd.push_back(old);
  h.startEnd.push_back(uint32_t(h.primIdCount.size()));
  h.geomTags.push_back(tag);
  return uint32_t(h.startEnd.size() / 2 - 1);
}

lrt_geom_data unit_cube_geom(uint32_t bvhOffset, uint32_t type, uint32_t sdfId)
{
  lrt_geom_data g;
  std::memset(&g, 0, sizeof(g));
  const float mn[4] = {-1, -1, -1, 1}, mx[4] = {1, 1, 1, 1};
  std::memcpy(g.boxMin, mn, sizeof(mn));
  std::memcpy(g.boxMax, mx, sizeof(mx));
  g.bvhOffset = bvhOffset;
  g.type = type;
  g.offset[0] = sdfId;
  return g;
}

// add_border_nodes_rec (BVH2Common_host.cpp:1348-1381): leaves whose corner
// values change sign, with the box arithmetic of the reference.
void border_nodes(const lrt_sdf_frame_octree_node* nodes, size_t count, std::vector<lrt_bvh_node>& out, unsigned idx,
                  const float p[3], float d, int depth)
{
  if (idx >= count || depth > 32) return;
  const unsigned ofs = nodes[idx].offset;
  if (ofs == 0) {
    bool less = false, more = false;
    for (int i = 0; i < 8; i++) {
      if (nodes[idx].values[i] <= 0) less = true;
      else if (nodes[idx].values[i] >= 0) more = true;
    }
    if (less && more) {
      lrt_bvh_node n;
      for (int k = 0; k < 3; k++) {
        n.boxMin[k] = 2.0f * (d * p[k]) - 1.0f;
        n.boxMax[k] = n.boxMin[k] + 2.0f * d * 1.0f;
      }
      n.leftOffset = idx;
      n.escapeIndex = 0;
      out.push_back(n);
    }
  } else {
    for (int i = 0; i < 8; i++) {
      const float ch_d = d / 2;
      const float ch_p[3] = {2 * p[0] + float((i & 4) >> 2), 2 * p[1] + float((i & 2) >> 1), 2 * p[2] + float(i & 1)};
      border_nodes(nodes, count, out, ofs + i, ch_p, ch_d, depth + 1);
    }
  }
}

// Node box of an SVS / SBS node (BVH2Common_host.cpp:588-596, 676-684).
Aabb lod_box(uint32_t pos_xy, uint32_t pos_z_lod_size)
{
  const float px = float(pos_xy >> 16), py = float(pos_xy & 0x0000FFFF);
  const float pz = float(pos_z_lod_size >> 16), sz = float(pos_z_lod_size & 0x0000FFFF);
  Aabb b;
  const float p[3] = {px, py, pz};
  for (int k = 0; k < 3; k++) {
    b.lo[k] = -1.0f + 2.0f * p[k] / sz;
    b.hi[k] = b.lo[k] + 2.0f * 1.0f / sz;
  }
  return b;
}

// Inverse of a column-major 4x4 in float, by cofactors, rounding exactly like
// LiteMath's inverse4x4 (dependencies/1st-party/LiteMath/LiteMath.h:2070-2153),
// which BVHRT::AddInstance and UpdateInstance use for transformInv
// (BVH2Common_host.cpp:1295-1296, 1333): the instance matrices must be the
// reference's floats, or rays enter the BLAS at other points and hits drift.
//
// 2x2 products p[k] = a(i, u_k) * a(j, v_k) are formed for the row pairs
// (i, j) = (2, 3) (output columns 0, 1) and (0, 1) (columns 2, 3).  Each
// cofactor is (three products) - (three products), each triple summed left to
// right, with the terms in the order of kCof; the result is scaled by
// 1 / (row 0 of the input . column 0 of the cofactors).  Returns false for a
// matrix whose determinant is zero or not finite (the reference would return
// infinities and NaNs).
bool invert4(const float* m, float* out)
{
  auto a = [m](int r, int c) { return m[c * 4 + r]; };
  // the column pairs (u_k, v_k) of the 12 products of one row pair
  static const uint8_t kPairCols[12][2] = {{2, 3}, {3, 2}, {1, 3}, {3, 1}, {1, 2}, {2, 1},
                                           {0, 3}, {3, 0}, {0, 2}, {2, 0}, {0, 1}, {1, 0}};
  // cofactor (r, c): six {product index, column of the multiplying row} terms,
  // three added then three subtracted; the multiplying row of output column
  // c is kRowOf[c]
  static const uint8_t kRowOf[4] = {1, 0, 3, 2};
  static const uint8_t kCof[4][4][6][2] = {
      // output column 0
      {{{0, 1}, {3, 2}, {4, 3}, {1, 1}, {2, 2}, {5, 3}},
       {{1, 0}, {6, 2}, {9, 3}, {0, 0}, {7, 2}, {8, 3}},
       {{2, 0}, {7, 1}, {10, 3}, {3, 0}, {6, 1}, {11, 3}},
       {{5, 0}, {8, 1}, {11, 2}, {4, 0}, {9, 1}, {10, 2}}},
      // output column 1
      {{{1, 1}, {2, 2}, {5, 3}, {0, 1}, {3, 2}, {4, 3}},
       {{0, 0}, {7, 2}, {8, 3}, {1, 0}, {6, 2}, {9, 3}},
       {{3, 0}, {6, 1}, {11, 3}, {2, 0}, {7, 1}, {10, 3}},
       {{4, 0}, {9, 1}, {10, 2}, {5, 0}, {8, 1}, {11, 2}}},
      // output column 2
      {{{0, 1}, {3, 2}, {4, 3}, {1, 1}, {2, 2}, {5, 3}},
       {{1, 0}, {6, 2}, {9, 3}, {0, 0}, {7, 2}, {8, 3}},
       {{2, 0}, {7, 1}, {10, 3}, {3, 0}, {6, 1}, {11, 3}},
       {{5, 0}, {8, 1}, {11, 2}, {4, 0}, {9, 1}, {10, 2}}},
      // output column 3
      {{{2, 2}, {5, 3}, {1, 1}, {4, 3}, {0, 1}, {3, 2}},
       {{8, 3}, {0, 0}, {7, 2}, {6, 2}, {9, 3}, {1, 0}},
       {{6, 1}, {11, 3}, {3, 0}, {10, 3}, {2, 0}, {7, 1}},
       {{10, 2}, {4, 0}, {9, 1}, {8, 1}, {11, 2}, {5, 0}}},
  };
  float p[2][12];
  for (int half = 0; half < 2; half++) {
    const int i = half ? 0 : 2, j = i + 1;
    for (int k = 0; k < 12; k++) p[half][k] = a(i, kPairCols[k][0]) * a(j, kPairCols[k][1]);
  }
  float cof[4][4]; // cof[r][c]
  for (int c = 0; c < 4; c++) {
    const float* t = p[c >> 1];
    const int row = kRowOf[c];
    for (int r = 0; r < 4; r++) {
      const uint8_t(*q)[2] = kCof[c][r];
      float v = t[q[0][0]] * a(row, q[0][1]) + t[q[1][0]] * a(row, q[1][1]) + t[q[2][0]] * a(row, q[2][1]);
      v -= t[q[3][0]] * a(row, q[3][1]) + t[q[4][0]] * a(row, q[4][1]) + t[q[5][0]] * a(row, q[5][1]);
      cof[r][c] = v;
    }
  }
  const float det = a(0, 0) * cof[0][0] + a(0, 1) * cof[1][0] + a(0, 2) * cof[2][0] + a(0, 3) * cof[3][0];
  if (det == 0.0f || !std::isfinite(det)) return false;
  const float k = 1.0f / det;
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) out[c * 4 + r] = cof[r][c] * k;
  return true;
}

uint32_t prims_in_leaf_from_name(const char* name)
{
  // BuilderPresetsFromString (cbvh.cpp:57-69): trailing digit, default 2
  if (!name || !*name) return 2;
  const char last = name[std::strlen(name) - 1];
  if (last >= '0' && last <= '9') return uint32_t(last - '0');
  return 2;
}

bool need_normal(const lrt_preset& p)
{
  const uint32_t m = p.render_mode; // BVH2Common.cpp:19-32
  return m == 1 || m == 8 || m == 12 || m == 17 || m == 20 || m == 7 || m == 18 || m == 23 || m == 21 || m == 11 ||
         m == 27;
}

} // namespace

// ---------------------------------------------------------------------------
// Structural validation: every index the kernels follow is in bounds, every
// tree pointer points forward (so the stackless TLAS loop and the BLAS loop
// terminate), and the BLAS depth fits the traversal stack.
// ---------------------------------------------------------------------------
lrt_status validate(lrt_scene* s, SceneInfo* info)
{
  const HostArrays& h = s->h;
  SceneInfo I;
  const size_t G = h.geomData.size();
  if (h.instanceData.empty()) return fail(s, LRT_ERR_BAD_SCENE, "scene has no instances");
  if (h.nodesTLAS.empty()) return fail(s, LRT_ERR_BAD_SCENE, "TLAS is empty (CommitScene not called?)");
  if (h.geomTags.size() != G || h.startEnd.size() != 2 * G)
    return fail(s, LRT_ERR_BAD_SCENE, "geomData/geomTags/startEnd sizes differ (%zu/%zu/%zu)", G, h.geomTags.size(),
                h.startEnd.size() / 2);
  if (h.vertPos.size() % 4 != 0) return fail(s, LRT_ERR_BAD_SCENE, "vertPos is not float4");
  // TLAS: the pair-aligned layout of AlignNodes2 (cbvh.cpp:143-169).  Every
  // node is reached exactly once from the root pair, children of an inner
  // node sit at leftOffset and leftOffset+1, and each escape index is the
  // next node of a depth-first walk (left -> right sibling, right -> the
  // parent's escape).  This makes the stackless loop of RayQuery_NearestHit
  // finite on every uploaded TLAS.
  const size_t T = h.nodesTLAS.size();
  for (size_t i = 0; i < T; i++) {
    const lrt_bvh_node& n = h.nodesTLAS[i];
    if ((n.leftOffset & kLeafBit) && (n.leftOffset & kStartMask) >= h.instanceData.size())
      return fail(s, LRT_ERR_BAD_SCENE, "TLAS leaf %zu names instance %u of %zu", i, n.leftOffset & kStartMask,
                  h.instanceData.size());
  }
  if (T == 1) {
    if (!(h.nodesTLAS[0].leftOffset & kLeafBit) || h.nodesTLAS[0].escapeIndex < kEscapeRoot)
      return fail(s, LRT_ERR_BAD_SCENE, "one-node TLAS must be a leaf with an out-of-tree escape");
  } else {
    std::vector<uint8_t> seen(T, 0);
    std::vector<std::pair<uint32_t, uint32_t>> st{{0u, kEscapeRoot}};
    size_t reached = 0;
    while (!st.empty()) {
      const auto [a, esc] = st.back();
      st.pop_back();
      if (uint64_t(a) + 1 >= T || seen[a] || seen[a + 1])
        return fail(s, LRT_ERR_BAD_SCENE, "TLAS pair at %u is out of range or reached twice", a);
      seen[a] = seen[a + 1] = 1;
      reached += 2;
      if (h.nodesTLAS[a].escapeIndex != a + 1 || h.nodesTLAS[a + 1].escapeIndex != esc)
        return fail(s, LRT_ERR_BAD_SCENE, "TLAS pair at %u has escape indices (%u,%u), expected (%u,%u)", a,
                    h.nodesTLAS[a].escapeIndex, h.nodesTLAS[a + 1].escapeIndex, a + 1, esc);
      for (uint32_t j = 0; j < 2; j++) {
        const lrt_bvh_node& n = h.nodesTLAS[a + j];
        if (!(n.leftOffset & kLeafBit)) st.push_back({n.leftOffset, n.escapeIndex});
      }
    }
    (void)reached;
  }
  I.tlasNodes = uint32_t(T);
  for (size_t i = 0; i < h.instanceData.size(); i++)
    if (h.instanceData[i].geomId >= G)
      return fail(s, LRT_ERR_BAD_SCENE, "instance %zu names geometry %u of %zu", i, h.instanceData[i].geomId, G);
  // geometries: checked once per geometry version; a commit after instance
  // changes only keeps what the last check found
  const bool geomChecked = s->validatedGeomVersion == s->geomVersion;
  if (geomChecked) {
    const SceneInfo& c = s->geomInfo;
    I.maxBlasDepth = c.maxBlasDepth;
    I.hasTriangles = c.hasTriangles;
    I.hasSbs = c.hasSbs;
    I.hasFrameOctree = c.hasFrameOctree;
    I.hasSvs = c.hasSvs;
    I.hasSbsNeighbours = c.hasSbsNeighbours;
  }
  const size_t P = geomChecked ? 0 : h.allNodePairs.size();
  std::vector<uint8_t> pairSeen(P, 0);
  for (size_t g = 0; g < G && !geomChecked; g++) {
    const lrt_geom_data& gd = h.geomData[g];
    const uint32_t tag = h.geomTags[g];
    const uint32_t a0 = h.startEnd[2 * g], a1 = h.startEnd[2 * g + 1];
    if (a0 > a1 || a1 > h.primIdCount.size())
      return fail(s, LRT_ERR_BAD_SCENE, "geometry %zu leaf table [%u,%u) outside primIdCount", g, a0, a1);
    if (gd.bvhOffset >= P) return fail(s, LRT_ERR_BAD_SCENE, "geometry %zu bvhOffset %u >= %zu", g, gd.bvhOffset, P);
    // BLAS: walk the pairs reachable from the root, checking forward pointers
    // and leaf ids, and measure depth.
    uint32_t maxDepth = 0;
    std::vector<std::pair<uint32_t, uint32_t>> st{{0u, 1u}};
    while (!st.empty()) {
      const auto [k, dpt] = st.back();
      st.pop_back();
      maxDepth = std::max(maxDepth, dpt);
      if (dpt > 4096) return fail(s, LRT_ERR_BAD_SCENE, "geometry %zu BLAS deeper than 4096", g);
      const uint64_t abs = uint64_t(gd.bvhOffset) + k;
      if (abs >= P) return fail(s, LRT_ERR_BAD_SCENE, "geometry %zu pair %u beyond allNodePairs", g, k);
      if (pairSeen[abs]) return fail(s, LRT_ERR_BAD_SCENE, "geometry %zu pair %u is reached twice", g, k);
      pairSeen[abs] = 1;
      const lrt_bvh_node* ch[2] = {&h.allNodePairs[abs].left, &h.allNodePairs[abs].right};
      for (int j = 0; j < 2; j++) {
        const uint32_t lo = ch[j]->leftOffset;
        if (lo & kLeafBit) {
          if (lo == kLeafNormal) continue; // empty leaf (BVH2Common.cpp:3290)
          const uint32_t aabb = lo & kStartMask;
          if (uint64_t(a0) + aabb >= a1)
            return fail(s, LRT_ERR_BAD_SCENE, "geometry %zu leaf aabb %u outside its %u leaves", g, aabb, a1 - a0);
        } else {
          if (lo <= k) return fail(s, LRT_ERR_BAD_SCENE, "geometry %zu pair %u child %u is not a later pair", g, k, lo);
          st.push_back({lo, dpt + 1});
        }
      }
    }
    I.maxBlasDepth = std::max(I.maxBlasDepth, maxDepth);
    // leaf payloads
    if (tag == LRT_TAG_TRIANGLE) {
      I.hasTriangles = true;
      if (gd.type != LRT_TYPE_MESH_TRIANGLE) return fail(s, LRT_ERR_BAD_SCENE, "triangle geometry %zu has type %u", g, gd.type);
      if (gd.offset[0] % 3 != 0) return fail(s, LRT_ERR_BAD_SCENE, "geometry %zu index offset not a multiple of 3", g);
      for (uint32_t a = a0; a < a1; a++) {
        const uint32_t pk = h.primIdCount[a];
        const uint64_t st0 = pk & kStartMask, cnt = (pk & kSizeMask) >> 28;
        const uint64_t lastIdx = uint64_t(gd.offset[0]) + (st0 + cnt) * 3;
        if (cnt && lastIdx > h.indices.size())
          return fail(s, LRT_ERR_BAD_SCENE, "geometry %zu leaf %u triangles beyond indices", g, a - a0);
        if (cnt && uint64_t(gd.offset[0]) / 3 + st0 + cnt > h.primIndices.size())
          return fail(s, LRT_ERR_BAD_SCENE, "geometry %zu leaf %u triangles beyond primIndices", g, a - a0);
        for (uint64_t t = st0; t < st0 + cnt; t++)
          for (int c = 0; c < 3; c++) {
            const uint64_t vi = uint64_t(gd.offset[1]) + h.indices[gd.offset[0] + 3 * t + c];
            if (vi >= h.vertPos.size() / 4)
              return fail(s, LRT_ERR_BAD_SCENE, "geometry %zu triangle %llu vertex beyond vertPos", g,
                          (unsigned long long)t);
          }
      }
    } else if (tag == LRT_TAG_SDF_BRICK) {
      I.hasSbs = true;
      const uint32_t sid = gd.offset[0];
      if (sid >= h.sdfSBSRoots.size() || sid >= h.sdfSBSHeaders.size())
        return fail(s, LRT_ERR_BAD_SCENE, "SBS geometry %zu names SBS %u", g, sid);
      const lrt_sdf_sbs_header& hd = h.sdfSBSHeaders[sid];
      const uint32_t layout = hd.aux_data & LRT_SBS_LAYOUT_MASK;
      if (hd.brick_size == 0 || hd.brick_size > 16)
        return fail(s, LRT_ERR_BAD_SCENE, "SBS %u brick_size %u", sid, hd.brick_size);
      const bool idx = layout == LRT_SBS_LAYOUT_ID32F_IRGB32F || layout == LRT_SBS_LAYOUT_ID32F_IRGB32F_IN;
      if (layout == LRT_SBS_LAYOUT_ID32F_IRGB32F_IN) I.hasSbsNeighbours = true;
      if (!idx && !(hd.bytes_per_value == 1 || hd.bytes_per_value == 2 || hd.bytes_per_value == 4))
        return fail(s, LRT_ERR_BAD_SCENE, "SBS %u bytes_per_value %u", sid, hd.bytes_per_value);
      const uint64_t v = hd.brick_size + 2 * hd.brick_pad + 1, v3 = v * v * v;
      // this model's nodes run from its root to the next larger root
      uint64_t nodeEnd = h.sdfSBSNodes.size();
      for (uint32_t r : h.sdfSBSRoots)
        if (r > h.sdfSBSRoots[sid]) nodeEnd = std::min<uint64_t>(nodeEnd, r);
      for (uint32_t a = a0; a < a1; a++) {
        const uint64_t nodeId = uint64_t(h.primIdCount[a] & kStartMask) + h.sdfSBSRoots[sid];
        // AddGeom_SdfSBS pads one-brick models with a box that names a node
        // past the model (BVH2Common_host.cpp:686-693); the kernels skip it.
        if (nodeId >= nodeEnd) continue;
        const uint64_t off = h.sdfSBSNodes[nodeId].data_offset;
        if (idx) {
          if (off + v3 + 8 > h.sdfSBSData.size())
            return fail(s, LRT_ERR_BAD_SCENE, "SBS node %llu data beyond sdfSBSData", (unsigned long long)nodeId);
          for (uint64_t q = 0; q < v3; q++)
            if (h.sdfSBSData[off + q] >= h.sdfSBSDataF.size())
              return fail(s, LRT_ERR_BAD_SCENE, "SBS node %llu value index beyond sdfSBSDataF",
                          (unsigned long long)nodeId);
          for (uint64_t q = 0; q < 8; q++)
            if (uint64_t(h.sdfSBSData[off + v3 + q]) + 3 > h.sdfSBSDataF.size())
              return fail(s, LRT_ERR_BAD_SCENE, "SBS node %llu colour index beyond sdfSBSDataF",
                          (unsigned long long)nodeId);
        } else {
          const uint64_t vpi = 4 / hd.bytes_per_value;
          if (off + (v3 + vpi - 1) / vpi > h.sdfSBSData.size())
            return fail(s, LRT_ERR_BAD_SCENE, "SBS node %llu data beyond sdfSBSData", (unsigned long long)nodeId);
        }
      }
    } else if (tag == LRT_TAG_SDF_NODE) {
      const uint32_t sid = gd.offset[0];
      if (gd.type == LRT_TYPE_SDF_FRAME_OCTREE) {
        I.hasFrameOctree = true;
        if (sid >= h.sdfFrameOctreeRoots.size())
          return fail(s, LRT_ERR_BAD_SCENE, "frame-octree geometry %zu names octree %u", g, sid);
        // The reference indexes the single, last-written origNodes array with
        // the leaf id (BVH2Common_host.cpp:531); leaves beyond it are unusable.
        for (uint32_t a = a0; a < a1; a++) {
          const uint32_t b = h.primIdCount[a] & kStartMask;
          if (b >= h.origNodes.size())
            return fail(s, LRT_ERR_BAD_SCENE,
                        "frame-octree geometry %zu leaf %u beyond origNodes (%zu); the reference keeps only the last "
                        "octree's boxes",
                        g, b, h.origNodes.size());
          const uint64_t nodeId = uint64_t(h.origNodes[b].leftOffset) + h.sdfFrameOctreeRoots[sid];
          if (nodeId >= h.sdfFrameOctreeNodes.size())
            return fail(s, LRT_ERR_BAD_SCENE, "frame-octree geometry %zu leaf %u node beyond nodes", g, b);
        }
      } else if (gd.type == LRT_TYPE_SDF_SVS) {
        I.hasSvs = true;
        if (sid >= h.sdfSVSRoots.size()) return fail(s, LRT_ERR_BAD_SCENE, "SVS geometry %zu names SVS %u", g, sid);
        for (uint32_t a = a0; a < a1; a++) {
          const uint64_t nodeId = uint64_t(h.primIdCount[a] & kStartMask) + h.sdfSVSRoots[sid];
          if (nodeId >= h.sdfSVSNodes.size())
            return fail(s, LRT_ERR_BAD_SCENE, "SVS geometry %zu leaf %u node beyond nodes", g, a - a0);
        }
      } else {
        return fail(s, LRT_ERR_UNSUPPORTED, "SDF-node geometry %zu has type %u (frame octree and SVS are supported)",
                    g, gd.type);
      }
    } else if (tag != LRT_TAG_NONE) {
      return fail(s, LRT_ERR_UNSUPPORTED, "geometry %zu tag %u is outside the ray-query path", g, tag);
    }
  }
  if (I.maxBlasDepth > kMaxStack)
    return fail(s, LRT_ERR_BAD_SCENE, "BLAS depth %u exceeds the %u-entry traversal stack", I.maxBlasDepth, kMaxStack);
  s->geomInfo = I;
  s->validatedGeomVersion = s->geomVersion;
  *info = I;
  return LRT_OK;
}

// Presets the kernels implement: the ST, ANALYTIC, NEWTON, BBOX and IT node
// solvers (only ST and BBOX where sphere_tracing_only: the batched, render
// and adjoint kernels), trilinear, geometric triangle normals; any render mode.
lrt_status check_preset(lrt_scene* s, bool sphere_tracing_only)
{
  const lrt_preset& p = s->preset;
  const SceneInfo& I = s->info;
  const bool sdf = I.hasSbs || I.hasFrameOctree || I.hasSvs;
  if (sdf && p.sdf_node_intersect > 4)
    return fail(s, LRT_ERR_UNSUPPORTED, "sdf_node_intersect %u is not a node solver (0..4)", p.sdf_node_intersect);
  if (sdf && sphere_tracing_only && p.sdf_node_intersect != 0 && p.sdf_node_intersect != 3)
    return fail(s, LRT_ERR_UNSUPPORTED,
                "sdf_node_intersect %u: this call implements ST (0) and BBOX (3); lrt_trace_nearest has all five",
                p.sdf_node_intersect);
  if (I.hasSbs && p.interpolation_mode != 0)
    return fail(s, LRT_ERR_UNSUPPORTED, "interpolation_mode %u: only TRILINEAR is implemented", p.interpolation_mode);
  if (I.hasTriangles && need_normal(p) && p.normal_mode != 0)
    return fail(s, LRT_ERR_UNSUPPORTED, "normal_mode %u for triangles: only GEOMETRY is implemented", p.normal_mode);
  if (I.hasSbsNeighbours && need_normal(p) && p.normal_mode == 2)
    return fail(s, LRT_ERR_UNSUPPORTED, "normal_mode SDF_SMOOTHED is not implemented");
  if (p.render_mode == 26)
    return fail(s, LRT_ERR_UNSUPPORTED, "render_mode INTERSECTION_COUNT is not implemented");
  return LRT_OK;
}

} // namespace lrt

using namespace lrt;

extern "C" {

static thread_local std::string g_create_error;

lrt_status lrt_default_preset(lrt_preset* out)
{
  if (!out) return LRT_ERR_INVALID_ARGUMENT;
  // getDefaultPreset(), core/render_settings.h:139-160
  out->render_mode = 1;
  out->sdf_node_intersect = 1;
  out->normal_mode = 1;
  out->ray_gen_mode = 0;
  out->interpolation_mode = 0;
  out->representation_mode = 1;
  out->spp = 1;
  out->fixed_lod = 1;
  out->level_of_detail = 16.0f;
  out->compact_sdf_eps = 0.05f;
  out->LOD_distance = 10.0f;
  out->channel_render_mode = 0;
  out->channel_id = 0;
  out->component_id = 0;
  out->CTF_id = 0;
  return LRT_OK;
}

lrt_status lrt_scene_create(const char* build_name, const char* layout_name, lrt_scene** out)
{
  (void)layout_name; // the layout string selects Embree treelet layouts; this builder has one layout
  if (!out) {
    g_create_error = "lrt_scene_create: out is NULL";
    return LRT_ERR_INVALID_ARGUMENT;
  }
  lrt_scene* s = new (std::nothrow) lrt_scene();
  if (!s) {
    g_create_error = "lrt_scene_create: out of host memory";
    return LRT_ERR_OUT_OF_MEMORY;
  }
  lrt_default_preset(&s->preset);
  s->primsInLeaf = prims_in_leaf_from_name(build_name);
  if (s->primsInLeaf == 0 || s->primsInLeaf > 7) s->primsInLeaf = 2;
  *out = s;
  return LRT_OK;
}

lrt_status lrt_scene_destroy(lrt_scene* s)
{
  if (!s) return LRT_OK;
  device_release(s);
  delete s;
  return LRT_OK;
}

const char* lrt_last_error(const lrt_scene* s)
{
  if (!s) return g_create_error.c_str();
  return s->err.c_str();
}

lrt_status lrt_set_preset(lrt_scene* s, const lrt_preset* p)
{
  if (!s || !p) return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_set_preset: NULL argument");
  s->preset = *p;
  return LRT_OK;
}

lrt_status lrt_clear_geom(lrt_scene* s)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  s->geomVersion++;
  const lrt_preset keep = s->preset;
  s->h = HostArrays();
  s->preset = keep;
  s->committed = false;
  return LRT_OK;
}

lrt_status lrt_add_geom_triangles3f(lrt_scene* s, const float* vpos, size_t nvert, const uint32_t* tri,
                                    size_t nidx, uint32_t flags, size_t stride, uint32_t* geom_id_out)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  s->geomVersion++;
  if (!vpos || !tri || nvert == 0 || nidx == 0 || nidx % 3 != 0)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "AddGeom_Triangles3f: empty input or index count %zu not a multiple of 3",
                nidx);
  if ((flags & LRT_BUILD_LOW) && nidx / 3 >= (size_t(1) << 28))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "AddGeom_Triangles3f (BUILD_LOW): %zu triangles", nidx / 3);
  if (stride == 0) stride = 12;
  if (stride % 4 != 0 || stride < 12)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "AddGeom_Triangles3f: vertex byte stride %zu", stride);
  // The per-element loops below run on the host's cores (OpenMP); each
  // element's result is what the sequential loop computes, and the geometry
  // box combines the chunks' boxes in chunk order (std::min/max keep the
  // first of equal values, so signed zeros come out as in one pass).
  size_t firstBad = nidx;
#pragma omp parallel for reduction(min : firstBad) schedule(static)
  for (size_t i = 0; i < nidx; i++)
    if (tri[i] >= nvert && i < firstBad) firstBad = i;
  if (firstBad < nidx)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "AddGeom_Triangles3f: index %u >= vertex count %zu", tri[firstBad],
                nvert);
  HostArrays& h = s->h;
  const size_t vs = stride / 4;
  const uint32_t geomId = uint32_t(h.geomData.size());
  const size_t oldV = h.vertPos.size() / 4, oldI = h.indices.size();
  lrt_geom_data g;
  std::memset(&g, 0, sizeof(g));
  for (int k = 0; k < 4; k++) { g.boxMin[k] = FLT_MAX; g.boxMax[k] = -FLT_MAX; }
  h.vertPos.resize(4 * (oldV + nvert));
  {
    float* dst = h.vertPos.data() + 4 * oldV;
    constexpr size_t kChunks = 64;
    float cmin[kChunks][4], cmax[kChunks][4];
#pragma omp parallel for schedule(static)
    for (size_t c = 0; c < kChunks; c++) {
      for (int k = 0; k < 4; k++) { cmin[c][k] = FLT_MAX; cmax[c][k] = -FLT_MAX; }
      const size_t lo = nvert * c / kChunks, hi = nvert * (c + 1) / kChunks;
      for (size_t i = lo; i < hi; i++) {
        const float v[4] = {vpos[i * vs + 0], vpos[i * vs + 1], vpos[i * vs + 2], 1.0f};
        for (int k = 0; k < 4; k++) {
          dst[4 * i + k] = v[k];
          cmin[c][k] = std::min(cmin[c][k], v[k]);
          cmax[c][k] = std::max(cmax[c][k], v[k]);
        }
      }
    }
    for (size_t c = 0; c < kChunks; c++)
      for (int k = 0; k < 4; k++) {
        g.boxMin[k] = std::min(g.boxMin[k], cmin[c][k]);
        g.boxMax[k] = std::max(g.boxMax[k], cmax[c][k]);
      }
  }
  g.offset[0] = uint32_t(oldI);
  g.offset[1] = uint32_t(oldV);
  g.bvhOffset = uint32_t(h.allNodePairs.size());
  g.type = LRT_TYPE_MESH_TRIANGLE;
  h.geomData.push_back(g);
  h.geomTags.push_back(LRT_TAG_TRIANGLE);

  const size_t nt = nidx / 3;
  std::vector<Aabb> boxes(nt);
  const float* V = h.vertPos.data() + 4 * oldV;
#pragma omp parallel for schedule(static)
  for (size_t t = 0; t < nt; t++) {
    boxes[t].reset();
    for (int c = 0; c < 3; c++) {
      const float* p = V + 4 * size_t(tri[3 * t + c]);
      for (int k = 0; k < 3; k++) {
        boxes[t].lo[k] = std::min(boxes[t].lo[k], p[k]);
        boxes[t].hi[k] = std::max(boxes[t].hi[k], p[k]);
      }
    }
  }
  // leaves numbered in emission order; each leaf word is Pack(leafId, 1) and
  // its triangle range goes to primIdCount as Pack(start, count)
  // (cbvh.cpp:516-525, AppendTreeData BVH2Common_host.cpp:287-301).
  std::vector<uint32_t> startCount;
  std::vector<uint32_t> reordered;
  reordered.reserve(nt);
  auto emit = [&](const auto& B) {
    emit_pairs(B, h.allNodePairs, [&](int32_t node) {
      const BNode& n = B.nodes[node];
      const uint32_t leafId = uint32_t(startCount.size());
      startCount.push_back(pack_offset_and_size(uint32_t(reordered.size()), n.count));
      for (uint32_t i = n.start; i < n.start + n.count; i++) reordered.push_back(B.ids[i]);
      return pack_offset_and_size(leafId, 1);
    });
  };
  if (flags & LRT_BUILD_LOW) {
    // the device builds the tree and, when the root is not a single leaf,
    // also emits the pairs, leaf table and triangle order (lbvh_build_blas:
    // the arrays the host emitter makes from the same tree)
    const char* err = nullptr;
    if (nt > s->primsInLeaf) {
      static_assert(sizeof(LbvhPairOut) == sizeof(lrt_bvh_node_pair), "a pair is 64 bytes");
      const size_t base = h.allNodePairs.size();
      err = lbvh_build_blas(
          reinterpret_cast<const float*>(boxes.data()), uint32_t(nt), s->primsInLeaf,
          [&](size_t count) {
            h.allNodePairs.resize(base + count);
            return reinterpret_cast<LbvhPairOut*>(h.allNodePairs.data() + base);
          },
          startCount, reordered);
      if (err) h.allNodePairs.resize(base);
    } else {
      RadixTree R;
      err = R.build(boxes, s->primsInLeaf);
      if (!err) emit(R);
    }
    if (err) {
      h.vertPos.resize(4 * oldV);
      h.geomData.pop_back();
      h.geomTags.pop_back();
      return fail(s, LRT_ERR_CUDA, "AddGeom_Triangles3f (BUILD_LOW): %s", err);
    }
  } else {
    SahBuilder B(boxes, s->primsInLeaf);
    B.build(0, uint32_t(nt));
    emit(B);
  }
  h.primIndices.insert(h.primIndices.end(), reordered.begin(), reordered.end());
  h.indices.resize(oldI + 3 * reordered.size());
  uint32_t* idx = h.indices.data() + oldI;
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < reordered.size(); i++)
    for (int c = 0; c < 3; c++) idx[3 * i + c] = tri[3 * size_t(reordered[i]) + c];
  const uint32_t old = uint32_t(h.primIdCount.size());
  h.primIdCount.insert(h.primIdCount.end(), startCount.begin(), startCount.end());
  h.startEnd.push_back(old);
  h.startEnd.push_back(uint32_t(h.primIdCount.size()));
  s->committed = false;
  if (geom_id_out) *geom_id_out = uint32_t(h.startEnd.size() / 2 - 1);
  (void)geomId;
  return LRT_OK;
}

lrt_status lrt_add_geom_aabb(lrt_scene* s, uint32_t tag, const float* boxes8, size_t n, uint32_t flags,
                             uint32_t* geom_id_out)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  s->geomVersion++;
  if (!boxes8 || n == 0) return fail(s, LRT_ERR_INVALID_ARGUMENT, "AddGeom_AABB: no boxes");
  if ((flags & LRT_BUILD_LOW) && n >= (size_t(1) << 28))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "AddGeom_AABB (BUILD_LOW): %zu boxes", n);
  std::vector<Aabb> boxes(n);
  for (size_t i = 0; i < n; i++) boxes[i] = box_of(boxes8 + 8 * i, boxes8 + 8 * i + 4);
  const uint32_t id = add_aabb_blas(s, tag, boxes, flags);
  if (id == ~0u) return LRT_ERR_CUDA;
  s->committed = false;
  if (geom_id_out) *geom_id_out = id;
  return LRT_OK;
}

lrt_status lrt_add_geom_sdf_frame_octree(lrt_scene* s, const lrt_sdf_frame_octree_node* nodes, size_t count,
                                         uint32_t* geom_id_out)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  s->geomVersion++;
  if (!nodes || count == 0 || count >= (1u << 28))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "AddGeom_SdfFrameOctree: %zu nodes", count);
  HostArrays& h = s->h;
  std::vector<lrt_bvh_node> orig;
  const float p0[3] = {0, 0, 0};
  border_nodes(nodes, count, orig, 0, p0, 1.0f, 0);
  if (orig.empty()) return fail(s, LRT_ERR_INVALID_ARGUMENT, "AddGeom_SdfFrameOctree: octree has no surface leaves");
  h.geomData.push_back(unit_cube_geom(uint32_t(h.allNodePairs.size()), LRT_TYPE_SDF_FRAME_OCTREE,
                                      uint32_t(h.sdfFrameOctreeRoots.size())));
  const uint32_t n_off = uint32_t(h.sdfFrameOctreeNodes.size());
  h.sdfFrameOctreeRoots.push_back(n_off);
  h.sdfFrameOctreeNodes.insert(h.sdfFrameOctreeNodes.end(), nodes, nodes + count);
  for (size_t i = n_off; i < h.sdfFrameOctreeNodes.size(); i++) h.sdfFrameOctreeNodes[i].offset += n_off;
  h.origNodes = orig; // one array for all octrees, as in the reference (:531)
  std::vector<Aabb> boxes(orig.size());
  for (size_t i = 0; i < orig.size(); i++) boxes[i] = box_of(orig[i].boxMin, orig[i].boxMax);
  const uint32_t id = add_aabb_blas(s, LRT_TAG_SDF_NODE, boxes);
  s->committed = false;
  if (geom_id_out) *geom_id_out = id;
  return LRT_OK;
}

lrt_status lrt_add_geom_sdf_svs(lrt_scene* s, const lrt_sdf_svs_node* nodes, size_t count, uint32_t* geom_id_out)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  s->geomVersion++;
  if (!nodes || count == 0 || count >= (1u << 28))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "AddGeom_SdfSVS: %zu nodes", count);
  HostArrays& h = s->h;
  h.geomData.push_back(
      unit_cube_geom(uint32_t(h.allNodePairs.size()), LRT_TYPE_SDF_SVS, uint32_t(h.sdfSVSRoots.size())));
  h.sdfSVSRoots.push_back(uint32_t(h.sdfSVSNodes.size()));
  h.sdfSVSNodes.insert(h.sdfSVSNodes.end(), nodes, nodes + count);
  std::vector<Aabb> boxes(count);
  for (size_t i = 0; i < count; i++) boxes[i] = lod_box(nodes[i].pos_xy, nodes[i].pos_z_lod_size);
  const uint32_t id = add_aabb_blas(s, LRT_TAG_SDF_NODE, boxes);
  s->committed = false;
  if (geom_id_out) *geom_id_out = id;
  return LRT_OK;
}

lrt_status lrt_add_geom_sdf_sbs(lrt_scene* s, const lrt_sdf_sbs_header* header, const lrt_sdf_sbs_node* nodes,
                                size_t count, const uint32_t* values, size_t values_count, const float* values_f,
                                size_t values_f_count, uint32_t* geom_id_out)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  s->geomVersion++;
  if (!header || !nodes || count == 0 || !values || values_count == 0 || count >= (1u << 28) ||
      values_count >= (1u << 28))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "AddGeom_SdfSBS: %zu nodes, %zu values", count, values_count);
  HostArrays& h = s->h;
  const uint32_t layout = header->aux_data & LRT_SBS_LAYOUT_MASK;
  uint32_t type = LRT_TYPE_SDF_SBS;
  if (layout == LRT_SBS_LAYOUT_UNDEFINED || layout == LRT_SBS_LAYOUT_DX) type = LRT_TYPE_SDF_SBS;
  else if (layout == LRT_SBS_LAYOUT_DX_UV16) type = LRT_TYPE_SDF_SBS_TEX;
  else if (layout == LRT_SBS_LAYOUT_DX_RGB8 || layout == LRT_SBS_LAYOUT_ID32F_IRGB32F ||
           layout == LRT_SBS_LAYOUT_ID32F_IRGB32F_IN)
    type = LRT_TYPE_SDF_SBS_COL;
  else
    return fail(s, LRT_ERR_UNSUPPORTED, "AddGeom_SdfSBS: node layout %u", layout >> 24);
  const bool indexed = layout == LRT_SBS_LAYOUT_ID32F_IRGB32F || layout == LRT_SBS_LAYOUT_ID32F_IRGB32F_IN;
  if (indexed && (!values_f || values_f_count == 0))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "AddGeom_SdfSBS: indexed layout without float values");
  h.geomData.push_back(unit_cube_geom(uint32_t(h.allNodePairs.size()), type, uint32_t(h.sdfSBSRoots.size())));
  const uint32_t n_off = uint32_t(h.sdfSBSNodes.size()), v_off = uint32_t(h.sdfSBSData.size());
  h.sdfSBSRoots.push_back(n_off);
  h.sdfSBSHeaders.push_back(*header);
  h.sdfSBSNodes.insert(h.sdfSBSNodes.end(), nodes, nodes + count);
  h.sdfSBSData.insert(h.sdfSBSData.end(), values, values + values_count);
  for (size_t i = n_off; i < h.sdfSBSNodes.size(); i++) h.sdfSBSNodes[i].data_offset += v_off;
  if (indexed) {
    const uint32_t f_off = uint32_t(h.sdfSBSDataF.size());
    h.sdfSBSDataF.insert(h.sdfSBSDataF.end(), values_f, values_f + values_f_count);
    for (size_t i = v_off; i < h.sdfSBSData.size(); i++) h.sdfSBSData[i] += f_off;
  }
  std::vector<Aabb> boxes(count);
  for (size_t i = 0; i < count; i++) boxes[i] = lod_box(nodes[i].pos_xy, nodes[i].pos_z_lod_size);
  if (boxes.size() == 1) {
    // the reference adds a tiny second box for one-brick models (:686-693)
    Aabb b;
    for (int k = 0; k < 3; k++) { b.lo[k] = boxes[0].lo[k] - 0.001f * 1.0f; b.hi[k] = boxes[0].lo[k]; }
    boxes.push_back(b);
  }
  const uint32_t id = add_aabb_blas(s, LRT_TAG_SDF_BRICK, boxes);
  s->committed = false;
  if (geom_id_out) *geom_id_out = id;
  return LRT_OK;
}

// ---- SDF model files (the formats of sdf/simple/sdf_simple.cpp:50-142) ----
namespace {
struct FileReader {
  FILE* f = nullptr;
  long size = 0;
  explicit FileReader(const char* path)
  {
    f = path ? std::fopen(path, "rb") : nullptr;
    if (f && std::fseek(f, 0, SEEK_END) == 0) {
      size = std::ftell(f);
      std::fseek(f, 0, SEEK_SET);
    }
  }
  ~FileReader()
  {
    if (f) std::fclose(f);
  }
  long left() const { return f ? size - std::ftell(f) : 0; }
  bool read(void* dst, size_t bytes) { return f && left() >= long(bytes) && std::fread(dst, 1, bytes, f) == bytes; }
  bool u32(uint32_t* v) { return read(v, sizeof(uint32_t)); }
};
} // namespace

// load_sdf_frame_octree (:58-66): u32 count, count 36-byte nodes.
lrt_status lrt_add_geom_sdf_frame_octree_file(lrt_scene* s, const char* path, uint32_t* geom_id_out)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  FileReader r(path);
  uint32_t n = 0;
  if (!r.f) return fail(s, LRT_ERR_INVALID_ARGUMENT, "frame-octree file %s cannot be opened", path ? path : "(null)");
  if (!r.u32(&n) || r.left() < long(n) * long(sizeof(lrt_sdf_frame_octree_node)))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "frame-octree file %s is shorter than its %u nodes", path, n);
  std::vector<lrt_sdf_frame_octree_node> nodes(n);
  if (n && !r.read(nodes.data(), n * sizeof(lrt_sdf_frame_octree_node)))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "frame-octree file %s: read error", path);
  return lrt_add_geom_sdf_frame_octree(s, nodes.data(), n, geom_id_out);
}

// load_sdf_SVS (:88-96): u32 count, count 16-byte nodes.
lrt_status lrt_add_geom_sdf_svs_file(lrt_scene* s, const char* path, uint32_t* geom_id_out)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  FileReader r(path);
  uint32_t n = 0;
  if (!r.f) return fail(s, LRT_ERR_INVALID_ARGUMENT, "SVS file %s cannot be opened", path ? path : "(null)");
  if (!r.u32(&n) || r.left() < long(n) * long(sizeof(lrt_sdf_svs_node)))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "SVS file %s is shorter than its %u nodes", path, n);
  std::vector<lrt_sdf_svs_node> nodes(n);
  if (n && !r.read(nodes.data(), n * sizeof(lrt_sdf_svs_node)))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "SVS file %s: read error", path);
  return lrt_add_geom_sdf_svs(s, nodes.data(), n, geom_id_out);
}

// load_sdf_SBS (:122-142): header, u32 count, nodes, u32 value count, values,
// then u32 float count and floats; files written before the float trailer
// existed end after the values.
lrt_status lrt_add_geom_sdf_sbs_file(lrt_scene* s, const char* path, uint32_t* geom_id_out)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  FileReader r(path);
  if (!r.f) return fail(s, LRT_ERR_INVALID_ARGUMENT, "SBS file %s cannot be opened", path ? path : "(null)");
  lrt_sdf_sbs_header hdr;
  uint32_t n = 0, cnt = 0, cnt_f = 0;
  if (!r.read(&hdr, sizeof(hdr)) || !r.u32(&n) || r.left() < long(n) * long(sizeof(lrt_sdf_sbs_node)))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "SBS file %s is shorter than its header and %u nodes", path, n);
  std::vector<lrt_sdf_sbs_node> nodes(n);
  if (n && !r.read(nodes.data(), n * sizeof(lrt_sdf_sbs_node)))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "SBS file %s: read error", path);
  if (!r.u32(&cnt) || r.left() < long(cnt) * 4)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "SBS file %s is shorter than its %u values", path, cnt);
  std::vector<uint32_t> values(cnt);
  if (cnt && !r.read(values.data(), cnt * sizeof(uint32_t)))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "SBS file %s: read error", path);
  std::vector<float> values_f;
  if (r.left() >= 4) {
    if (!r.u32(&cnt_f) || r.left() < long(cnt_f) * 4)
      return fail(s, LRT_ERR_INVALID_ARGUMENT, "SBS file %s is shorter than its %u float values", path, cnt_f);
    values_f.resize(cnt_f);
    if (cnt_f && !r.read(values_f.data(), cnt_f * sizeof(float)))
      return fail(s, LRT_ERR_INVALID_ARGUMENT, "SBS file %s: read error", path);
  }
  return lrt_add_geom_sdf_sbs(s, &hdr, nodes.data(), n, values.data(), values.size(),
                              values_f.empty() ? nullptr : values_f.data(), values_f.size(), geom_id_out);
}

lrt_status lrt_clear_scene(lrt_scene* s)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  s->h.instanceData.clear();
  s->h.nodesTLAS.clear();
  s->committed = false;
  return LRT_OK;
}

lrt_status lrt_add_instance(lrt_scene* s, uint32_t geom_id, const float* m, uint32_t* inst_id_out)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  if (!m) return fail(s, LRT_ERR_INVALID_ARGUMENT, "AddInstance: NULL matrix");
  geom_id &= 0x7fffffffu; // CRT_GEOM_MASK_AABB_BIT (BVH2Common_host.cpp:1266-1267)
  HostArrays& h = s->h;
  if (geom_id >= h.geomData.size())
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "AddInstance: geometry %u of %zu", geom_id, h.geomData.size());
  lrt_instance_data inst;
  std::memset(&inst, 0, sizeof(inst));
  const float* bmin = h.geomData[geom_id].boxMin;
  const float* bmax = h.geomData[geom_id].boxMax;
  for (int k = 0; k < 4; k++) { inst.boxMin[k] = FLT_MAX; inst.boxMax[k] = -FLT_MAX; }
  for (int c = 0; c < 8; c++) {
    const float v[4] = {(c & 1) ? bmax[0] : bmin[0], (c & 2) ? bmax[1] : bmin[1], (c & 4) ? bmax[2] : bmin[2], 1.0f};
    for (int r = 0; r < 4; r++) {
      const float x = v[0] * m[r] + v[1] * m[4 + r] + v[2] * m[8 + r] + v[3] * m[12 + r];
      inst.boxMin[r] = std::min(inst.boxMin[r], x);
      inst.boxMax[r] = std::max(inst.boxMax[r], x);
    }
  }
  inst.geomId = geom_id;
  std::memcpy(inst.transform, m, sizeof(inst.transform));
  if (!invert4(m, inst.transformInv)) return fail(s, LRT_ERR_INVALID_ARGUMENT, "AddInstance: singular matrix");
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) inst.transformInvTransposed[c * 4 + r] = inst.transformInv[r * 4 + c];
  h.instanceData.push_back(inst);
  s->committed = false;
  if (inst_id_out) *inst_id_out = uint32_t(h.instanceData.size() - 1);
  return LRT_OK;
}

lrt_status lrt_commit_scene(lrt_scene* s, uint32_t flags)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  HostArrays& h = s->h;
  if (h.instanceData.empty()) return fail(s, LRT_ERR_INVALID_ARGUMENT, "CommitScene: no instances");
  h.nodesTLAS.clear();
  if (h.instanceData.size() > 1) {
    std::vector<Aabb> boxes(h.instanceData.size());
    for (size_t i = 0; i < boxes.size(); i++) boxes[i] = box_of(h.instanceData[i].boxMin, h.instanceData[i].boxMax);
    if (flags & LRT_BUILD_LOW) {
      RadixTree R;
      if (const char* err = R.build(boxes, 1)) return fail(s, LRT_ERR_CUDA, "CommitScene (BUILD_LOW): %s", err);
      emit_tlas(R, h.nodesTLAS);
    } else {
      SahBuilder B(boxes, 1);
      B.build(0, uint32_t(boxes.size()));
      emit_tlas(B, h.nodesTLAS);
    }
  } else {
    // a single instance needs no TLAS: one leaf node (:1245-1252)
    lrt_bvh_node n;
    for (int k = 0; k < 3; k++) {
      n.boxMin[k] = h.instanceData[0].boxMin[k];
      n.boxMax[k] = h.instanceData[0].boxMax[k];
    }
    n.leftOffset = kLeafBit;
    n.escapeIndex = kLeafNormal;
    h.nodesTLAS.push_back(n);
  }
  lrt_status st = validate(s, &s->info);
  if (st != LRT_OK) return st;
  if (flags & LRT_COMMIT_HOST_ONLY) return LRT_OK;
  if (s->dev && s->uploadedGeomVersion == s->geomVersion) {
    // only instances changed since the last upload (UpdateInstance,
    // ClearScene + AddInstance): the BLAS data on the device stays
    st = device_update_instances(s);
  } else {
    st = device_upload(s);
    if (st == LRT_OK) s->uploadedGeomVersion = s->geomVersion;
  }
  if (st != LRT_OK) return st;
  s->committed = true;
  return LRT_OK;
}

lrt_status lrt_update_instance(lrt_scene* s, uint32_t inst_id, const float* m, uint32_t flags)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  if (!m) return fail(s, LRT_ERR_INVALID_ARGUMENT, "UpdateInstance: NULL matrix");
  HostArrays& h = s->h;
  // the reference accepts inst_id == size (BVH2Common_host.cpp:1305) and writes past the array
  if (inst_id >= h.instanceData.size())
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "UpdateInstance: instance %u of %zu", inst_id, h.instanceData.size());
  lrt_instance_data& inst = h.instanceData[inst_id];
  float inv[16];
  if (!invert4(m, inv)) return fail(s, LRT_ERR_INVALID_ARGUMENT, "UpdateInstance: singular matrix");
  // the box of the geometry box's 8 corners (:1311-1329); min/max do not depend on their order
  const float* bmin = h.geomData[inst.geomId].boxMin;
  const float* bmax = h.geomData[inst.geomId].boxMax;
  for (int k = 0; k < 4; k++) { inst.boxMin[k] = FLT_MAX; inst.boxMax[k] = -FLT_MAX; }
  for (int c = 0; c < 8; c++) {
    const float v[4] = {(c & 1) ? bmax[0] : bmin[0], (c & 2) ? bmax[1] : bmin[1], (c & 4) ? bmax[2] : bmin[2], 1.0f};
    for (int r = 0; r < 4; r++) {
      const float x = v[0] * m[r] + v[1] * m[4 + r] + v[2] * m[8 + r] + v[3] * m[12 + r];
      inst.boxMin[r] = std::min(inst.boxMin[r], x);
      inst.boxMax[r] = std::max(inst.boxMax[r], x);
    }
  }
  std::memcpy(inst.transform, m, sizeof(inst.transform));
  std::memcpy(inst.transformInv, inv, sizeof(inst.transformInv));
  // the reference leaves transformInvTransposed as it was (:1333-1334)
  if (flags & LRT_UPDATE_NORMAL_MATRIX)
    for (int r = 0; r < 4; r++)
      for (int c = 0; c < 4; c++) inst.transformInvTransposed[c * 4 + r] = inst.transformInv[r * 4 + c];
  s->committed = false;
  return LRT_OK;
}

lrt_status lrt_scene_upload(lrt_scene* s, const lrt_scene_arrays* a)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  if (!a) return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_scene_upload: NULL arrays");
  HostArrays h;
#define CP(field, T, mult)                                                                                       \
  if (a->field##_count && !a->field) return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_scene_upload: " #field " is NULL"); \
  h.field.assign(reinterpret_cast<const T*>(a->field), reinterpret_cast<const T*>(a->field) + a->field##_count * mult);
  CP(nodesTLAS, lrt_bvh_node, 1)
  CP(allNodePairs, lrt_bvh_node_pair, 1)
  CP(instanceData, lrt_instance_data, 1)
  CP(geomData, lrt_geom_data, 1)
  CP(geomTags, uint32_t, 1)
  CP(startEnd, uint32_t, 2)
  CP(primIdCount, uint32_t, 1)
  CP(indices, uint32_t, 1)
  CP(vertPos, float, 4)
  CP(primIndices, uint32_t, 1)
  CP(origNodes, lrt_bvh_node, 1)
  CP(sdfFrameOctreeNodes, lrt_sdf_frame_octree_node, 1)
  CP(sdfFrameOctreeRoots, uint32_t, 1)
  CP(sdfSVSNodes, lrt_sdf_svs_node, 1)
  CP(sdfSVSRoots, uint32_t, 1)
  CP(sdfSBSNodes, lrt_sdf_sbs_node, 1)
  CP(sdfSBSData, uint32_t, 1)
  CP(sdfSBSDataF, float, 1)
  CP(sdfSBSRoots, uint32_t, 1)
  CP(sdfSBSHeaders, lrt_sdf_sbs_header, 1)
#undef CP
  s->h = std::move(h);
  s->committed = false;
  s->geomVersion++;
  lrt_status st = validate(s, &s->info);
  if (st != LRT_OK) return st;
  st = device_upload(s);
  if (st != LRT_OK) return st;
  s->uploadedGeomVersion = s->geomVersion;
  s->committed = true;
  return LRT_OK;
}

lrt_status lrt_scene_export(const lrt_scene* s, lrt_scene_arrays* a)
{
  if (!s || !a) return LRT_ERR_INVALID_ARGUMENT;
  const HostArrays& h = s->h;
  std::memset(a, 0, sizeof(*a));
#define EX(field, T, div)                                          \
  a->field = reinterpret_cast<const T*>(h.field.data());           \
  a->field##_count = h.field.size() / div;
  EX(nodesTLAS, lrt_bvh_node, 1)
  EX(allNodePairs, lrt_bvh_node_pair, 1)
  EX(instanceData, lrt_instance_data, 1)
  EX(geomData, lrt_geom_data, 1)
  EX(geomTags, uint32_t, 1)
  EX(startEnd, uint32_t, 2)
  EX(primIdCount, uint32_t, 1)
  EX(indices, uint32_t, 1)
  EX(vertPos, float, 4)
  EX(primIndices, uint32_t, 1)
  EX(origNodes, lrt_bvh_node, 1)
  EX(sdfFrameOctreeNodes, lrt_sdf_frame_octree_node, 1)
  EX(sdfFrameOctreeRoots, uint32_t, 1)
  EX(sdfSVSNodes, lrt_sdf_svs_node, 1)
  EX(sdfSVSRoots, uint32_t, 1)
  EX(sdfSBSNodes, lrt_sdf_sbs_node, 1)
  EX(sdfSBSData, uint32_t, 1)
  EX(sdfSBSDataF, float, 1)
  EX(sdfSBSRoots, uint32_t, 1)
  EX(sdfSBSHeaders, lrt_sdf_sbs_header, 1)
#undef EX
  return LRT_OK;
}

} // extern "C"
