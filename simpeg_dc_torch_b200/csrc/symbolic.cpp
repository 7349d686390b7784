// Symbolic analysis: nested dissection, assembly tree, front structures.
//
// Replaces the reordering + symbolic factorization that the reference obtains
// from cuDSS's `DirectSolver.plan()` (dctorch/solver.py:103-109, 204-207).
//
// Ordering.  The graph of the (structurally symmetric) pattern is split
// recursively.  With integer grid coordinates (the tensor meshes of the DC
// engines) a subdomain is cut by the coordinate plane through the middle of
// its longest axis; nodes of one side that still touch the other side are
// moved into the separator, so any graph is handled correctly.  Without
// coordinates, the cut is the middle level of a breadth-first level structure
// rooted at a pseudo-peripheral node.  Recursion stops at `leaf_size` nodes.
// Unknowns are numbered in postorder: left subtree, right subtree, separator.
//
// Assembly tree.  Every non-empty separator and every leaf subdomain is one
// supernode (a block of contiguous pivot columns, factored as a dense front).
// With T(s) the subtree of s, its front rows are its own pivots followed by
// B(s) = the later-numbered nodes adjacent to T(s); no fill entry of L can
// fall outside that set, because a path from a column of s through earlier
// nodes cannot leave T(s) without crossing an ancestor separator.  B(s) is
// formed bottom-up from the children's B and the pivots' neighbours, and
// every row of B(s) is a row of the parent's front, which is what makes the
// extend-add map well defined.
#include "symbolic.h"

#include <algorithm>
#include <cstring>
#include <numeric>

namespace dct {
namespace {

struct Graph {
  int n = 0;
  std::vector<int64_t> ptr;
  std::vector<int32_t> adj;
};

struct NDNode {
  std::vector<int32_t> sep;
  int left = -1;
  int right = -1;
};

class Dissector {
 public:
  Dissector(const Graph& g, const int32_t* coords, int ndim, int leaf)
      : g_(g), coords_(coords), ndim_(ndim), leaf_(std::max(leaf, 2)),
        mark_(g.n, -1), side_(g.n, 0) {}

  int build(std::vector<int32_t> nodes) {
    std::vector<int32_t> L, R, S;
    bool cut = static_cast<int>(nodes.size()) > leaf_ && split(nodes, L, R, S);
    int idx = static_cast<int>(tree_.size());
    tree_.emplace_back();
    if (!cut) {
      std::sort(nodes.begin(), nodes.end());
      tree_[idx].sep = std::move(nodes);
      return idx;
    }
    nodes.clear();
    nodes.shrink_to_fit();
    std::sort(S.begin(), S.end());
    tree_[idx].sep = std::move(S);
    int l = L.empty() ? -1 : build(std::move(L));
    int r = R.empty() ? -1 : build(std::move(R));
    tree_[idx].left = l;
    tree_[idx].right = r;
    return idx;
  }

  std::vector<NDNode>& tree() { return tree_; }

 private:
  bool split(const std::vector<int32_t>& nodes, std::vector<int32_t>& L,
             std::vector<int32_t>& R, std::vector<int32_t>& S) {
    if (component_split(nodes, L, R)) return true;
    L.clear();
    R.clear();
    if (coords_ != nullptr && plane_split(nodes, L, R, S)) return true;
    L.clear();
    R.clear();
    S.clear();
    return level_split(nodes, L, R, S);
  }

  bool plane_split(const std::vector<int32_t>& nodes, std::vector<int32_t>& L,
                   std::vector<int32_t>& R, std::vector<int32_t>& S) {
    int lo[8], hi[8];
    for (int d = 0; d < ndim_; ++d) {
      lo[d] = INT32_MAX;
      hi[d] = INT32_MIN;
    }
    for (int32_t v : nodes)
      for (int d = 0; d < ndim_; ++d) {
        int c = coords_[int64_t(v) * ndim_ + d];
        lo[d] = std::min(lo[d], c);
        hi[d] = std::max(hi[d], c);
      }
    int ax = 0;
    for (int d = 1; d < ndim_; ++d)
      if (hi[d] - lo[d] > hi[ax] - lo[ax]) ax = d;
    if (hi[ax] - lo[ax] < 2) return false;
    int mid = lo[ax] + (hi[ax] - lo[ax]) / 2;
    ++stamp_;
    for (int32_t v : nodes) {
      mark_[v] = stamp_;
      int c = coords_[int64_t(v) * ndim_ + ax];
      side_[v] = c < mid ? 0 : (c > mid ? 1 : 2);
    }
    // a left node with a right neighbour joins the separator
    for (int32_t v : nodes) {
      if (side_[v] != 0) continue;
      for (int64_t p = g_.ptr[v]; p < g_.ptr[v + 1]; ++p) {
        int32_t u = g_.adj[p];
        if (mark_[u] == stamp_ && side_[u] == 1) {
          side_[v] = 2;
          break;
        }
      }
    }
    for (int32_t v : nodes) {
      if (side_[v] == 0) L.push_back(v);
      else if (side_[v] == 1) R.push_back(v);
      else S.push_back(v);
    }
    return !(L.empty() && R.empty());
  }

  // A disconnected subset (several independent systems assembled side by
  // side, e.g. a batch of surveys) splits between its components with an
  // empty separator: the components are dealt largest first to the lighter
  // side, so the two halves carry about the same number of nodes.
  bool component_split(const std::vector<int32_t>& nodes, std::vector<int32_t>& L,
                       std::vector<int32_t>& R) {
    ++stamp_;
    for (int32_t v : nodes) mark_[v] = stamp_;
    if (cmark_.empty()) cmark_.assign(g_.n, -1);
    ++cstamp_;
    std::vector<std::vector<int32_t>> comps;
    for (int32_t v0 : nodes) {
      if (cmark_[v0] == cstamp_) continue;
      std::vector<int32_t> c{v0};
      cmark_[v0] = cstamp_;
      for (size_t h = 0; h < c.size(); ++h) {
        const int32_t v = c[h];
        for (int64_t p = g_.ptr[v]; p < g_.ptr[v + 1]; ++p) {
          const int32_t u = g_.adj[p];
          if (mark_[u] == stamp_ && cmark_[u] != cstamp_) {
            cmark_[u] = cstamp_;
            c.push_back(u);
          }
        }
      }
      if (comps.empty() && c.size() == nodes.size()) return false;   // connected
      comps.push_back(std::move(c));
    }
    std::stable_sort(comps.begin(), comps.end(),
                     [](const std::vector<int32_t>& x, const std::vector<int32_t>& y) {
                       return x.size() > y.size();
                     });
    size_t nl = 0, nr = 0;
    for (const auto& c : comps) {
      if (nl <= nr) {
        L.insert(L.end(), c.begin(), c.end());
        nl += c.size();
      } else {
        R.insert(R.end(), c.begin(), c.end());
        nr += c.size();
      }
    }
    return true;
  }

  // breadth-first levels within the current subset; returns the depth
  int bfs(int32_t root, std::vector<int32_t>& order, std::vector<int32_t>& lev) {
    ++stamp2_;
    order.clear();
    order.push_back(root);
    seen(root) = stamp2_;
    lev_of(root) = 0;
    size_t head = 0;
    int depth = 0;
    while (head < order.size()) {
      int32_t v = order[head++];
      int lv = lev_of(v);
      depth = std::max(depth, lv);
      for (int64_t p = g_.ptr[v]; p < g_.ptr[v + 1]; ++p) {
        int32_t u = g_.adj[p];
        if (mark_[u] != stamp_ || seen(u) == stamp2_) continue;
        seen(u) = stamp2_;
        lev_of(u) = lv + 1;
        order.push_back(u);
      }
    }
    lev.resize(order.size());
    for (size_t i = 0; i < order.size(); ++i) lev[i] = lev_of(order[i]);
    return depth;
  }

  int32_t& seen(int32_t v) {
    if (seen_.empty()) seen_.assign(g_.n, -1);
    return seen_[v];
  }
  int32_t& lev_of(int32_t v) {
    if (levv_.empty()) levv_.assign(g_.n, 0);
    return levv_[v];
  }

  bool level_split(const std::vector<int32_t>& nodes, std::vector<int32_t>& L,
                   std::vector<int32_t>& R, std::vector<int32_t>& S) {
    ++stamp_;
    for (int32_t v : nodes) mark_[v] = stamp_;
    std::vector<int32_t> order, lev;
    int depth = bfs(nodes[0], order, lev);
    if (order.size() < nodes.size()) {
      // disconnected: the reached component against the rest, no separator
      for (int32_t v : order) side_[v] = 0;
      for (int32_t v : nodes) {
        if (seen(v) == stamp2_) L.push_back(v);
        else R.push_back(v);
      }
      return true;
    }
    // pseudo-peripheral root: restart from a far node while depth grows
    for (int it = 0; it < 4; ++it) {
      int32_t far = order.back();
      int64_t best_deg = INT64_MAX;
      for (size_t i = order.size(); i-- > 0 && lev[i] == depth;) {
        int64_t d = g_.ptr[order[i] + 1] - g_.ptr[order[i]];
        if (d < best_deg) {
          best_deg = d;
          far = order[i];
        }
      }
      std::vector<int32_t> o2, l2;
      int d2 = bfs(far, o2, l2);
      if (d2 <= depth) break;
      depth = d2;
      order.swap(o2);
      lev.swap(l2);
    }
    if (depth < 2) return false;
    std::vector<int64_t> cnt(depth + 1, 0);
    for (int l : lev) ++cnt[l];
    int64_t half = static_cast<int64_t>(nodes.size()) / 2, acc = 0;
    int m = 1;
    for (int l = 0; l <= depth; ++l) {
      if (acc + cnt[l] > half) {
        m = l;
        break;
      }
      acc += cnt[l];
    }
    m = std::min(std::max(m, 1), depth - 1);
    for (size_t i = 0; i < order.size(); ++i) {
      if (lev[i] < m) L.push_back(order[i]);
      else if (lev[i] > m) R.push_back(order[i]);
      else S.push_back(order[i]);
    }
    return true;
  }

  const Graph& g_;
  const int32_t* coords_;
  int ndim_, leaf_;
  std::vector<int32_t> mark_, side_, seen_, levv_, cmark_;
  int stamp_ = 0, stamp2_ = 0, cstamp_ = 0;
  std::vector<NDNode> tree_;
};

}  // namespace

std::string analyse(int n, const int32_t* crow, const int32_t* col,
                    const int32_t* coords, int ndim,
                    const SymbolicOptions& opt, Symbolic* out) {
  if (n <= 0) return "empty matrix";
  if (coords != nullptr && (ndim < 1 || ndim > 8)) return "bad ndim";
  Symbolic& S = *out;
  S = Symbolic();
  S.n = n;
  const int64_t nnz = crow[n];
  S.nnz_in = nnz;
  if (crow[0] != 0) return "crow[0] must be 0";
  for (int i = 0; i < n; ++i)
    if (crow[i + 1] < crow[i]) return "crow not monotone";
  for (int64_t e = 0; e < nnz; ++e)
    if (col[e] < 0 || col[e] >= n) return "column index out of range";
  S.in_crow.assign(crow, crow + n + 1);
  S.in_col.assign(col, col + nnz);

  // structural symmetry check (sorted copies of each row)
  {
    std::vector<int32_t> sorted(col, col + nnz);
    for (int i = 0; i < n; ++i)
      std::sort(sorted.begin() + crow[i], sorted.begin() + crow[i + 1]);
    for (int i = 0; i < n; ++i)
      for (int64_t e = crow[i]; e < crow[i + 1]; ++e) {
        int j = sorted[e];
        if (j == i) continue;
        if (!std::binary_search(sorted.begin() + crow[j],
                                sorted.begin() + crow[j + 1], i))
          return "pattern is not structurally symmetric";
      }
  }

  // adjacency without self loops
  Graph g;
  g.n = n;
  g.ptr.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    int64_t c = 0;
    for (int64_t e = crow[i]; e < crow[i + 1]; ++e) c += (col[e] != i);
    g.ptr[i + 1] = g.ptr[i] + c;
  }
  g.adj.resize(g.ptr[n]);
  for (int i = 0; i < n; ++i) {
    int64_t w = g.ptr[i];
    for (int64_t e = crow[i]; e < crow[i + 1]; ++e)
      if (col[e] != i) g.adj[w++] = col[e];
  }

  // ---- nested dissection tree
  Dissector dis(g, coords, ndim, opt.leaf_size);
  std::vector<int32_t> all(n);
  std::iota(all.begin(), all.end(), 0);
  int root = dis.build(std::move(all));
  std::vector<NDNode>& tree = dis.tree();

  // ---- postorder numbering; non-empty ND nodes become supernodes
  S.perm.reserve(n);
  S.sn_first.push_back(0);
  std::vector<int32_t> parent;
  // explicit stack to avoid deep recursion on degenerate graphs
  struct Frame {
    int nd;
    int state;
    std::vector<int32_t> tops;
  };
  std::vector<Frame> stack;
  std::vector<int32_t> roots;
  stack.push_back({root, 0, {}});
  std::vector<std::vector<int32_t>> ret;  // return values of finished frames
  while (!stack.empty()) {
    Frame& f = stack.back();
    NDNode& nd = tree[f.nd];
    if (f.state == 0) {
      f.state = 1;
      if (nd.left >= 0) {
        stack.push_back({nd.left, 0, {}});
        continue;
      }
    }
    if (f.state == 1) {
      if (nd.left >= 0) {
        f.tops.insert(f.tops.end(), ret.back().begin(), ret.back().end());
        ret.pop_back();
      }
      f.state = 2;
      if (nd.right >= 0) {
        stack.push_back({nd.right, 0, {}});
        continue;
      }
    }
    if (f.state == 2) {
      if (nd.right >= 0) {
        f.tops.insert(f.tops.end(), ret.back().begin(), ret.back().end());
        ret.pop_back();
      }
      std::vector<int32_t> result;
      if (!nd.sep.empty()) {
        int s = static_cast<int>(parent.size());
        parent.push_back(-1);
        for (int32_t t : f.tops) parent[t] = s;
        for (int32_t v : nd.sep) S.perm.push_back(v);
        S.sn_first.push_back(static_cast<int32_t>(S.perm.size()));
        result.push_back(s);
      } else {
        result = f.tops;
      }
      std::vector<int32_t>().swap(nd.sep);
      stack.pop_back();
      ret.push_back(std::move(result));
    }
  }
  if (static_cast<int>(S.perm.size()) != n) return "ordering lost nodes";
  S.nsuper = static_cast<int>(parent.size());
  S.sn_parent = parent;
  S.iperm.assign(n, -1);
  for (int i = 0; i < n; ++i) S.iperm[S.perm[i]] = i;

  const int ns_total = S.nsuper;
  std::vector<int32_t> owner(n);
  for (int s = 0; s < ns_total; ++s)
    for (int j = S.sn_first[s]; j < S.sn_first[s + 1]; ++j) owner[j] = s;

  // children lists
  S.child_ptr.assign(ns_total + 1, 0);
  for (int s = 0; s < ns_total; ++s)
    if (parent[s] >= 0) ++S.child_ptr[parent[s] + 1];
  for (int s = 0; s < ns_total; ++s) S.child_ptr[s + 1] += S.child_ptr[s];
  S.child.resize(S.child_ptr[ns_total]);
  S.child_slot.assign(ns_total, 0);
  {
    std::vector<int32_t> fill(S.child_ptr.begin(), S.child_ptr.end() - 1);
    for (int s = 0; s < ns_total; ++s)
      if (parent[s] >= 0) {
        int p = parent[s];
        S.child_slot[s] = fill[p] - S.child_ptr[p];
        S.child[fill[p]++] = s;
      }
  }

  // ---- boundary sets, bottom-up (supernode ids are a postorder)
  std::vector<std::vector<int32_t>> B(ns_total);
  std::vector<int32_t> mk(n, -1);
  for (int s = 0; s < ns_total; ++s) {
    const int first = S.sn_first[s], last = S.sn_first[s + 1] - 1;
    std::vector<int32_t>& lst = B[s];
    for (int ci = S.child_ptr[s]; ci < S.child_ptr[s + 1]; ++ci) {
      int c = S.child[ci];
      for (int32_t b : B[c]) {
        if (b < first) return "invalid dissection (child boundary below parent)";
        if (b > last && mk[b] != s) {
          mk[b] = s;
          lst.push_back(b);
        }
      }
    }
    for (int j = first; j <= last; ++j) {
      int v = S.perm[j];
      for (int64_t p = g.ptr[v]; p < g.ptr[v + 1]; ++p) {
        int u = S.iperm[g.adj[p]];
        if (u > last && mk[u] != s) {
          mk[u] = s;
          lst.push_back(u);
        }
      }
    }
    std::sort(lst.begin(), lst.end());
  }

  // ---- front rows, sizes, offsets, levels, statistics
  S.rows_ptr.assign(ns_total + 1, 0);
  S.front_n.assign(ns_total, 0);
  S.front_off.assign(ns_total, 0);
  S.sn_level.assign(ns_total, 0);
  int64_t off = 0;
  for (int s = 0; s < ns_total; ++s) {
    const int ns = S.ns(s);
    const int N = ns + static_cast<int>(B[s].size());
    S.front_n[s] = N;
    S.front_off[s] = off;
    off += int64_t(N) * N;
    S.rows_ptr[s + 1] = S.rows_ptr[s] + N;
    S.max_front = std::max(S.max_front, N);
    S.max_ns = std::max(S.max_ns, ns);
    S.nnz_L += int64_t(ns) * N - int64_t(ns) * (ns - 1) / 2;
    for (int k = 0; k < ns; ++k) {
      double m = double(N - k - 1);
      S.flops_factor += 1.0 + m + m * (m + 1.0);
    }
    int lv = 0;
    for (int ci = S.child_ptr[s]; ci < S.child_ptr[s + 1]; ++ci)
      lv = std::max(lv, S.sn_level[S.child[ci]] + 1);
    S.sn_level[s] = lv;
  }
  S.front_total = off;
  S.rows.resize(S.rows_ptr[ns_total]);
  for (int s = 0; s < ns_total; ++s) {
    int64_t w = S.rows_ptr[s];
    for (int j = S.sn_first[s]; j < S.sn_first[s + 1]; ++j) S.rows[w++] = j;
    for (int32_t b : B[s]) S.rows[w++] = b;
  }

  // ---- extend-add maps: boundary row of s -> row of the parent front
  S.rel_ptr.assign(ns_total + 1, 0);
  for (int s = 0; s < ns_total; ++s)
    S.rel_ptr[s + 1] = S.rel_ptr[s] + (parent[s] >= 0 ? int64_t(B[s].size()) : 0);
  S.rel.resize(S.rel_ptr[ns_total]);
  for (int s = 0; s < ns_total; ++s) {
    int p = parent[s];
    if (p < 0) {
      if (!B[s].empty()) return "root supernode with a boundary";
      continue;
    }
    const int pf = S.sn_first[p], pl = S.sn_first[p + 1] - 1, pns = pl - pf + 1;
    int64_t w = S.rel_ptr[s];
    for (int32_t b : B[s]) {
      int pos;
      if (b <= pl) {
        pos = b - pf;
      } else {
        auto it = std::lower_bound(B[p].begin(), B[p].end(), b);
        if (it == B[p].end() || *it != b) return "boundary row missing from parent front";
        pos = pns + static_cast<int>(it - B[p].begin());
      }
      S.rel[w++] = pos;
    }
  }

  // ---- entry scatter map (lower triangle in the new order), grouped by front
  {
    std::vector<int32_t> ent_s;
    std::vector<int32_t> ent_e, ent_pos;
    ent_s.reserve(nnz / 2 + n);
    ent_e.reserve(nnz / 2 + n);
    ent_pos.reserve(nnz / 2 + n);
    for (int i = 0; i < n; ++i) {
      const int pi = S.iperm[i];
      for (int64_t e = crow[i]; e < crow[i + 1]; ++e) {
        const int pj = S.iperm[col[e]];
        if (pi < pj) continue;
        const int s = owner[pj];
        const int first = S.sn_first[s], last = S.sn_first[s + 1] - 1;
        const int ns = last - first + 1;
        int lrow;
        if (pi <= last) {
          lrow = pi - first;
        } else {
          auto it = std::lower_bound(B[s].begin(), B[s].end(), pi);
          if (it == B[s].end() || *it != pi) return "entry outside its front";
          lrow = ns + static_cast<int>(it - B[s].begin());
        }
        const int64_t pos = int64_t(lrow) + int64_t(pj - first) * S.front_n[s];
        if (pos > INT32_MAX) return "front too large for 32-bit positions";
        ent_s.push_back(s);
        ent_e.push_back(static_cast<int32_t>(e));
        ent_pos.push_back(static_cast<int32_t>(pos));
      }
    }
    S.amap_ptr.assign(ns_total + 1, 0);
    for (int32_t s : ent_s) ++S.amap_ptr[s + 1];
    for (int s = 0; s < ns_total; ++s) S.amap_ptr[s + 1] += S.amap_ptr[s];
    S.amap_e.resize(ent_s.size());
    S.amap_pos.resize(ent_s.size());
    std::vector<int64_t> fill(S.amap_ptr.begin(), S.amap_ptr.end() - 1);
    for (size_t k = 0; k < ent_s.size(); ++k) {
      int64_t w = fill[ent_s[k]]++;
      S.amap_e[w] = ent_e[k];
      S.amap_pos[w] = ent_pos[k];
    }
  }

  // ---- level schedule
  S.nlevels = 0;
  for (int s = 0; s < ns_total; ++s) S.nlevels = std::max(S.nlevels, S.sn_level[s] + 1);
  S.level_ptr.assign(S.nlevels + 1, 0);
  for (int s = 0; s < ns_total; ++s) ++S.level_ptr[S.sn_level[s] + 1];
  for (int l = 0; l < S.nlevels; ++l) S.level_ptr[l + 1] += S.level_ptr[l];
  S.level_sn.resize(ns_total);
  {
    std::vector<int32_t> fill(S.level_ptr.begin(), S.level_ptr.end() - 1);
    for (int s = 0; s < ns_total; ++s) S.level_sn[fill[S.sn_level[s]]++] = s;
  }
  return std::string();
}

}  // namespace dct
