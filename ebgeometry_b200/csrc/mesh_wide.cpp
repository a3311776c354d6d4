// The 8-wide copy of a mesh's 4-wide BVH (host side).
//
// The reference makes its tree's branching ratio a compile-time constant (DefaultBranchingRatio,
// BVH.hpp:89-111; the packed tree's K, BVHImplem.hpp:425-548).  Here the 4-wide tree is the one
// every kernel reads; an 8-wide copy is an option of the plain FP32 traversal, so that the
// autotuner can time both widths on the caller's queries.  The copy is made from the 4-wide tree,
// not from a second build: each 8-wide node starts as one 4-wide node's slots and repeatedly
// replaces its largest-area interior slot by that child's own slots, while the slots still fit in
// eight.  Every leaf (its triangle range and leaf id) and every FP32 child box is carried over
// unchanged, so a query meets the same triangles with the same arithmetic and its answer is the same
// bit for bit; only the number of levels and the order of the tests change.
#include <algorithm>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "mesh_host.h"

namespace ebg {

namespace {

struct Slot
{
  float    lo[3], hi[3];
  uint32_t child, count;
};

// The non-empty slots of 4-wide node `x` (an empty slot has child 0 and is not a leaf: the root,
// node 0, is nobody's child).
void slotsOf(const EbgNode4& nd, std::vector<Slot>& out)
{
  for (int k = 0; k < 4; k++) {
    if (nd.child[k] == 0u) {
      continue;
    }
    out.push_back(Slot{{nd.lox[k], nd.loy[k], nd.loz[k]}, {nd.hix[k], nd.hiy[k], nd.hiz[k]}, nd.child[k], nd.count[k]});
  }
}

double area(const Slot& s)
{
  const double dx = double(s.hi[0]) - s.lo[0], dy = double(s.hi[1]) - s.lo[1], dz = double(s.hi[2]) - s.lo[2];
  return dx * dy + dy * dz + dz * dx;
}

int nonEmpty(const EbgNode4& nd)
{
  int c = 0;
  for (int k = 0; k < 4; k++) {
    c += nd.child[k] != 0u;
  }
  return c;
}

} // namespace

bool widenBvh8(const std::vector<EbgNode4>& n4,
               const std::vector<EbgObb>&   obb4,
               int64_t                      numTris,
               int64_t                      numLeaves,
               std::vector<EbgNode8>&       n8,
               std::vector<EbgObb>&         obb8,
               int&                         depth8,
               std::string&                 msg)
{
  n8.clear();
  obb8.clear();
  depth8 = 0;
  if (n4.empty() || obb4.size() < n4.size()) {
    msg = "widen: the 4-wide tree has no interior nodes";
    return false;
  }
  // breadth first, so that the top levels come first; queue entries are (4-wide node, level)
  std::vector<uint32_t> src{0u};
  std::vector<int>      level{1};
  std::vector<Slot>     slots;
  for (size_t j = 0; j < src.size(); j++) {
    const uint32_t x = src[j];
    if (x >= n4.size()) {
      msg = "widen: child index out of range in the 4-wide tree";
      return false;
    }
    slots.clear();
    slotsOf(n4[x], slots);
    // absorb the largest interior slot whose children still fit
    while (true) {
      int    pick = -1;
      double bestArea = -1.0;
      for (int i = 0; i < int(slots.size()); i++) {
        const Slot& s = slots[size_t(i)];
        if ((s.child & EBG_LEAF_BIT) || s.child >= n4.size()) {
          continue;
        }
        if (int(slots.size()) - 1 + nonEmpty(n4[s.child]) > 8) {
          continue;
        }
        const double a = area(s);
        if (a > bestArea) {
          bestArea = a;
          pick     = i;
        }
      }
      if (pick < 0) {
        break;
      }
      const uint32_t c = slots[size_t(pick)].child;
      slots.erase(slots.begin() + pick);
      slotsOf(n4[c], slots);
    }
    EbgNode8 out;
    for (int k = 0; k < 8; k++) {
      // empty slot: child 0, count 0 and an empty box, whose point distance is +inf
      out.lox[k] = out.loy[k] = out.loz[k] = std::numeric_limits<float>::infinity();
      out.hix[k] = out.hiy[k] = out.hiz[k] = -std::numeric_limits<float>::infinity();
      out.child[k] = 0u;
      out.count[k] = 0u;
    }
    for (int k = 0; k < int(slots.size()); k++) {
      const Slot& s = slots[size_t(k)];
      out.lox[k]    = s.lo[0];
      out.loy[k]    = s.lo[1];
      out.loz[k]    = s.lo[2];
      out.hix[k]    = s.hi[0];
      out.hiy[k]    = s.hi[1];
      out.hiz[k]    = s.hi[2];
      out.count[k]  = s.count;
      if (s.child & EBG_LEAF_BIT) {
        const uint64_t t0 = s.child & ~EBG_LEAF_BIT, cnt = s.count & EBG_COUNT_MASK, leaf = s.count >> EBG_COUNT_BITS;
        if (cnt == 0 || t0 + cnt > uint64_t(numTris) || leaf >= uint64_t(numLeaves)) {
          msg = "widen: leaf out of range in the 4-wide tree";
          return false;
        }
        out.child[k] = s.child;
      }
      else {
        // the child keeps its oriented-box flag; its 8-wide node is built from the same 4-wide node
        out.child[k] = uint32_t(src.size());
        src.push_back(s.child);
        level.push_back(level[j] + 1);
      }
    }
    n8.push_back(out);
    obb8.push_back(obb4[x]);
    depth8 = std::max(depth8, level[j] + 1); // + the leaf level
  }
  // Stack entries the traversal can hold at once: a node pops its own entry and pushes at most its
  // non-empty slots; descending into one of them leaves the others waiting.  So a subtree needs
  // need(x) = slots(x) - 1 + max(1, need(c) over its interior children c), computed children first
  // (breadth-first order puts every child after its parent).  The margin of 4 matches the 4-wide
  // builder's rule (3 x depth + 4).
  std::vector<int> need(n8.size(), 0);
  for (size_t j = n8.size(); j-- > 0;) {
    int slotsJ = 0, below = 1;
    for (int k = 0; k < 8; k++) {
      const uint32_t c = n8[j].child[k];
      slotsJ += c != 0u;
      if (c != 0u && !(c & EBG_LEAF_BIT)) {
        below = std::max(below, need[c]);
      }
    }
    need[j] = slotsJ - 1 + below;
  }
  if (need[0] + 4 > EBG_STACK_DEPTH) {
    msg = "widen: the 8-wide tree is too deep for the traversal stack (" + std::to_string(need[0]) +
          " entries on its deepest path, depth " + std::to_string(depth8) + ")";
    return false;
  }
  return true;
}

} // namespace ebg
