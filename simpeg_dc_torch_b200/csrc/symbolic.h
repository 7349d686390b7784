// Symbolic analysis for the supernodal multifrontal Cholesky factorization:
// nested-dissection ordering, the assembly tree of dense fronts, the maps that
// scatter matrix entries and children's update matrices into fronts, and the
// level / panel schedules the GPU kernels walk.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace dct {

// Pivot columns are processed in panels of this width (factor and solve).
constexpr int kPanel = 64;

struct SymbolicOptions {
  int leaf_size = 64;      // nested dissection stops at subdomains this small
};

// Work item of a panel step: supernode s, panel p (columns p*kPanel ...),
// and a tile index whose meaning depends on the kernel.
struct PanelTask {
  int32_t s;
  int32_t p;
  int32_t t0;
  int32_t t1;
};

struct Symbolic {
  int n = 0;
  int64_t nnz_in = 0;                 // entries of the input CSR pattern
  std::vector<int32_t> in_crow;       // the input pattern (n+1)
  std::vector<int32_t> in_col;        // (nnz_in)
  std::vector<int32_t> perm;          // perm[new] = old
  std::vector<int32_t> iperm;         // iperm[old] = new

  // supernodes (contiguous pivot columns in the new order, postordered)
  int nsuper = 0;
  std::vector<int32_t> sn_first;      // nsuper+1
  std::vector<int32_t> sn_parent;     // -1 at roots
  std::vector<int32_t> sn_level;      // 0 at leaves
  std::vector<int32_t> front_n;       // front order N = ns + nb
  std::vector<int64_t> front_off;     // element offset of the (N x N, column-major) front
  int64_t front_total = 0;            // elements per system
  std::vector<int64_t> rows_ptr;      // nsuper+1
  std::vector<int32_t> rows;          // front rows (new indices); first ns are the pivots
  std::vector<int32_t> child_ptr, child;  // children of each supernode
  std::vector<int32_t> child_slot;    // position of s among its parent's children
  std::vector<int64_t> rel_ptr;       // nsuper+1 ; rel of s: nb_s entries
  std::vector<int32_t> rel;           // parent-front row of each boundary row of s

  // entry scatter: CSR entry e (lower triangle in the new order) -> front pos
  std::vector<int64_t> amap_ptr;      // nsuper+1
  std::vector<int32_t> amap_e;        // input CSR entry index
  std::vector<int32_t> amap_pos;      // local position row + col*N

  // level schedule
  int nlevels = 0;
  std::vector<int32_t> level_ptr;     // nlevels+1, into level_sn
  std::vector<int32_t> level_sn;      // supernodes sorted by level

  // statistics
  int64_t nnz_L = 0;                  // stored factor entries (lower, incl. zeros)
  double flops_factor = 0.0;          // dense front flops (Cholesky + updates)
  int max_front = 0;
  int max_ns = 0;

  int ns(int s) const { return sn_first[s + 1] - sn_first[s]; }
  int nb(int s) const { return front_n[s] - ns(s); }
};

// Builds the analysis.  `coords` (n x ndim, may be null) are integer grid
// coordinates used for geometric bisection; without them the graph is
// bisected with breadth-first level structures.  Returns an empty string on
// success, else the reason the pattern was rejected.
std::string analyse(int n, const int32_t* crow, const int32_t* col,
                    const int32_t* coords, int ndim,
                    const SymbolicOptions& opt, Symbolic* out);

}  // namespace dct
