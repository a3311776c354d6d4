// Host check of the 8-wide copy of a 4-wide BVH (ebg::widenBvh8, ebgeometry_b200/csrc/mesh_wide.cpp),
// compiled by tests/test_wide_host.py together with the library's host sources.  For seeded random
// primitive sets, both build methods and several leaf sizes it checks that the copy
//  - holds every leaf of the 4-wide tree exactly once, with its triangle range, leaf id and box;
//  - gives every 8-wide node the leaves of the 4-wide node it was made from, and that node's
//    oriented box;
//  - keeps every interior child's box and oriented-box flag as the 4-wide parent slot stored them;
//  - has in-range child indices, empty slots as the traversal expects them, and no more levels
//    than the 4-wide tree;
//  - answers a scalar nearest-box search (the traversal's pruning on the boxes alone) exactly as
//    the 4-wide tree does.
// Prints one "ok ..." line per case, or "FAIL ..." and exits 1.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <random>
#include <set>
#include <string>
#include <tuple>
#include <vector>

#include "mesh_host.h"

using namespace ebg;

namespace {

int g_fail = 0;

void fail(const std::string& what)
{
  std::printf("FAIL %s\n", what.c_str());
  g_fail = 1;
}

using Leaf = std::tuple<uint32_t, uint32_t>; // (child word, count word)
struct Box
{
  float lo[3], hi[3];
  bool  operator==(const Box& o) const { return std::memcmp(this, &o, sizeof(Box)) == 0; }
};

template <int W, class N>
Box slotBox(const N& nd, int k)
{
  return Box{{nd.lox[k], nd.loy[k], nd.loz[k]}, {nd.hix[k], nd.hiy[k], nd.hiz[k]}};
}

template <int W, class N>
void leavesBelow(const std::vector<N>& nodes, uint32_t x, std::vector<Leaf>& out)
{
  for (int k = 0; k < W; k++) {
    const uint32_t c = nodes[x].child[k];
    if (c & EBG_LEAF_BIT) {
      out.emplace_back(c, nodes[x].count[k]);
    }
    else if (c != 0u) {
      leavesBelow<W>(nodes, c, out);
    }
  }
}

float boxD2(const Box& b, const float* p)
{
  float s = 0.f;
  for (int a = 0; a < 3; a++) {
    const float d = std::fmax(std::fmax(b.lo[a] - p[a], p[a] - b.hi[a]), 0.f);
    s += d * d;
  }
  return s;
}

// Smallest box distance over the leaves, by branch and bound from the root (strict pruning).
template <int W, class N>
float nearestLeafBox(const std::vector<N>& nodes, const float* p, uint32_t& leafOut)
{
  float                 best = std::numeric_limits<float>::infinity();
  std::vector<uint32_t> stack{0u};
  while (!stack.empty()) {
    const uint32_t x = stack.back();
    stack.pop_back();
    for (int k = 0; k < W; k++) {
      const uint32_t c = nodes[x].child[k];
      if (c == 0u) {
        continue;
      }
      const float d = boxD2(slotBox<W>(nodes[x], k), p);
      if (d > best) {
        continue;
      }
      if (c & EBG_LEAF_BIT) {
        if (d < best || (d == best && c < leafOut)) {
          best    = d;
          leafOut = c;
        }
      }
      else {
        stack.push_back(c);
      }
    }
  }
  return best;
}

void checkCase(uint32_t seed, int n, int build, int leafSize)
{
  std::mt19937_64                        rng(seed);
  std::uniform_real_distribution<double> u(-1.0, 1.0), s(0.001, 0.05);
  std::vector<double>                    lo(3 * size_t(n)), hi(3 * size_t(n)), c(3 * size_t(n));
  for (int i = 0; i < n; i++) {
    // clustered on a sphere-like shell plus a uniform part, as meshes and scenes are
    const bool   shell = (i % 4) != 0;
    double       x = u(rng), y = u(rng), z = u(rng);
    const double r = std::sqrt(x * x + y * y + z * z) + 1e-12;
    if (shell) {
      x /= r, y /= r, z /= r;
    }
    const double h = s(rng);
    const double p[3] = {x, y, z};
    for (int a = 0; a < 3; a++) {
      c[3 * size_t(i) + a]  = p[a];
      lo[3 * size_t(i) + a] = p[a] - h;
      hi[3 * size_t(i) + a] = p[a] + h;
    }
  }
  Bvh4        t4;
  std::string msg;
  const std::string tag = "seed " + std::to_string(seed) + " n " + std::to_string(n) + " build " +
                          std::to_string(build) + " leaf " + std::to_string(leafSize);
  if (!buildBvh4(lo, hi, c, build, leafSize, t4, msg)) {
    fail(tag + ": build: " + msg);
    return;
  }
  if (t4.rootRef & EBG_LEAF_BIT) {
    std::printf("ok %s: root is a leaf\n", tag.c_str());
    return;
  }
  const size_t        n4 = t4.nodes.size();
  std::vector<EbgObb> o4(n4);
  for (size_t i = 0; i < n4; i++) {
    std::memset(&o4[i], 0, sizeof(EbgObb));
    o4[i].pad = float(i); // marks the source node
    o4[i].hn  = float(i % 7);
  }
  std::vector<EbgNode8> n8;
  std::vector<EbgObb>   o8;
  int                   depth8 = 0;
  if (!widenBvh8(t4.nodes, o4, int64_t(n), t4.numLeaves, n8, o8, depth8, msg)) {
    fail(tag + ": widen: " + msg);
    return;
  }
  if (o8.size() != n8.size() || n8.empty()) {
    fail(tag + ": sizes");
    return;
  }
  // slot boxes and words of every child as the 4-wide parents store them
  std::map<uint32_t, std::pair<Box, uint32_t>> childSlot4; // 4-wide node -> (box, count word)
  std::map<uint32_t, Box>                      leafSlot4;  // leaf child word -> box
  for (size_t x = 0; x < n4; x++) {
    for (int k = 0; k < 4; k++) {
      const uint32_t ch = t4.nodes[x].child[k];
      if (ch & EBG_LEAF_BIT) {
        leafSlot4[ch] = slotBox<4>(t4.nodes[x], k);
      }
      else if (ch != 0u) {
        childSlot4[ch] = {slotBox<4>(t4.nodes[x], k), t4.nodes[x].count[k]};
      }
    }
  }
  // every 4-wide leaf exactly once in the copy
  std::vector<Leaf> all4, all8;
  leavesBelow<4>(t4.nodes, 0u, all4);
  leavesBelow<8>(n8, 0u, all8);
  std::sort(all4.begin(), all4.end());
  std::sort(all8.begin(), all8.end());
  if (all4 != all8 || int64_t(all4.size()) != t4.numLeaves) {
    fail(tag + ": leaf sets differ");
  }
  const float inf = std::numeric_limits<float>::infinity();
  for (size_t j = 0; j < n8.size(); j++) {
    const uint32_t x = uint32_t(o8[j].pad);
    if (x >= n4 || o8[j].hn != float(x % 7)) {
      fail(tag + ": oriented box of node " + std::to_string(j));
      continue;
    }
    std::vector<Leaf> a, b;
    leavesBelow<4>(t4.nodes, x, a);
    leavesBelow<8>(n8, uint32_t(j), b);
    std::sort(a.begin(), a.end());
    std::sort(b.begin(), b.end());
    if (a != b) {
      fail(tag + ": leaves below node " + std::to_string(j));
    }
    for (int k = 0; k < 8; k++) {
      const uint32_t ch = n8[j].child[k], cw = n8[j].count[k];
      const Box      bx = slotBox<8>(n8[j], k);
      if (ch == 0u) {
        if (cw != 0u || !(bx.lo[0] == inf && bx.hi[0] == -inf && bx.lo[1] == inf && bx.hi[2] == -inf)) {
          fail(tag + ": empty slot");
        }
      }
      else if (ch & EBG_LEAF_BIT) {
        if (!(leafSlot4.count(ch) && leafSlot4[ch] == bx)) {
          fail(tag + ": leaf slot box");
        }
      }
      else {
        if (ch >= n8.size()) {
          fail(tag + ": child index out of range");
          continue;
        }
        const uint32_t src = uint32_t(o8[ch].pad);
        if (!(childSlot4.count(src) && childSlot4[src].first == bx && childSlot4[src].second == cw)) {
          fail(tag + ": interior slot box or flag");
        }
      }
    }
  }
  if (depth8 > t4.depth + 1) {
    fail(tag + ": depth " + std::to_string(depth8));
  }
  // the pruned nearest-box search agrees
  std::mt19937_64                       qr(seed + 1);
  std::uniform_real_distribution<float> q(-1.5f, 1.5f);
  for (int i = 0; i < 2000; i++) {
    const float p[3] = {q(qr), q(qr), q(qr)};
    uint32_t    l4 = 0xffffffffu, l8 = 0xffffffffu;
    const float d4 = nearestLeafBox<4>(t4.nodes, p, l4);
    const float d8 = nearestLeafBox<8>(n8, p, l8);
    if (!(d4 == d8 && l4 == l8)) {
      fail(tag + ": nearest-box search differs");
      break;
    }
  }
  std::printf("ok %s: %zu 4-wide nodes (depth %d) -> %zu 8-wide nodes (depth %d)\n", tag.c_str(), n4, t4.depth,
              n8.size(), depth8);
}

} // namespace

int main()
{
  for (int build : {0, 1}) {
    for (int leaf : {1, 4, 8, 16}) {
      checkCase(11, 20000, build, leaf);
    }
    checkCase(12, 3, build, 4);   // root is a leaf
    checkCase(13, 9, build, 2);   // a few nodes
    checkCase(14, 200000, build, 8);
  }
  return g_fail;
}
