// C ABI of libdct: symbolic analysis handles, numeric plans (device buffers
// and launch schedules), factorize / solve with float64 iterative refinement.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>

#include "dct_internal.h"

using dct::Launch;
using dct::PanelTask;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail(e == cudaErrorMemoryAllocation ? DCT_ERR_OOM : DCT_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

#define DCT_CUDA(call, what)                              \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(e_, what);    \
  } while (0)

template <typename V>
int upload(dct_plan* P, const std::vector<V>& h, const V** out) {
  void* d = nullptr;
  size_t bytes = std::max<size_t>(1, h.size() * sizeof(V));
  cudaError_t e = cudaMalloc(&d, bytes);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc (symbolic arrays)");
  P->owned.push_back(d);
  if (!h.empty()) {
    e = cudaMemcpy(d, h.data(), h.size() * sizeof(V), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy (symbolic arrays)");
  }
  *out = static_cast<const V*>(d);
  return DCT_OK;
}

int alloc(dct_plan* P, size_t bytes, void** out, const char* what) {
  void* d = nullptr;
  cudaError_t e = cudaMalloc(&d, std::max<size_t>(bytes, 16));
  if (e != cudaSuccess) return cuda_fail(e, what);
  P->owned.push_back(d);
  *out = d;
  return DCT_OK;
}

int ceil_div(int a, int b) { return (a + b - 1) / b; }

// Tiles of a trailing update start at `base` (float64) or at base & ~7
// (float32: the 8-row grid of the split panel images, update_tc.cu).
int update_origin(int base, bool align8) { return align8 ? (base & ~7) : base; }

// ---- schedules ------------------------------------------------------------
// Algorithmic work of each launch (see dct::Schedule).  es = element size.
void account_factor(const dct::Symbolic& S, dct::Schedule* sc, double es,
                    int utile, int bpan, bool align8) {
  sc->flops.assign(sc->launches.size(), 0.0);
  sc->bytes.assign(sc->launches.size(), 0.0);
  sc->bytes_rhs.assign(sc->launches.size(), 0.0);
  for (size_t li = 0; li < sc->launches.size(); ++li) {
    const Launch& l = sc->launches[li];
    double f = 0, b = 0;
    for (int64_t q = l.first; q < l.first + l.count; ++q) {
      const PanelTask& t = sc->tasks[q];
      const int s = t.s, N = S.front_n[s], ns = S.ns(s);
      const int c0 = t.p * dct::kPanel, w = std::min(dct::kPanel, ns - c0);
      switch (l.kind) {
        case dct::kSmallFront: {
          for (int k = 0; k < ns; ++k) {
            double m = N - k - 1;
            f += 1 + m + m * (m + 1);
          }
          double upd = 0;
          for (int ci = S.child_ptr[s]; ci < S.child_ptr[s + 1]; ++ci) {
            double nbc = S.nb(S.child[ci]);
            upd += nbc * (nbc + 1) / 2;
          }
          double nent = double(S.amap_ptr[s + 1] - S.amap_ptr[s]);
          b += es * (double(N) * N + upd) + nent * (es + 8);
          break;
        }
        case dct::kLargeScatter:
          b += double(S.amap_ptr[s + 1] - S.amap_ptr[s]) * (2 * es + 8);
          break;
        case dct::kLargeExtendAdd: {
          const int nbc = S.nb(t.t0);
          double cols = std::min(8, nbc - t.t1), el = 0;
          for (int j = t.t1; j < t.t1 + cols; ++j) el += nbc - j;
          f += el;
          b += el * 3 * es;
          break;
        }
        case dct::kLargePanel: {
          const int r0 = c0 + w + (t.t0 - 1) * dct::kPanel;
          const double nr = std::min(dct::kPanel, N - r0);
          f += nr * w * w;
          b += es * (2 * nr * w + w * w / 2.0);
          break;
        }
        case dct::kLargeUpdate: {
          if (t.t0 < 0) {
            f += 2.0 * double(w) * w * w / 3.0;
            b += es * 2.0 * w * w;
            break;
          }
          const int base = c0 + w;
          const dct::UpdateRange R = dct::update_range(t.p, ns, N, bpan);
          const double kk = base - R.ka;
          // the tile's rows and columns from `base` on that it updates
          const int R0 = update_origin(base, align8);
          const int ri = std::max(base, R0 + t.t0 * utile);
          const int rj = std::max(base, R0 + t.t1 * utile);
          const double ni = std::min(R0 + (t.t0 + 1) * utile, N) - ri;
          const double nj = std::min(R0 + (t.t1 + 1) * utile, R.cend) - rj;
          if (t.t0 == t.t1) {
            // a diagonal tile: only its lower triangle (nj <= ni columns,
            // column c from row c down) is algorithmic work
            const double tri = nj * ni - nj * (nj - 1) / 2;
            f += 2 * tri * kk;
            b += es * (ni * kk + 2 * tri);
          } else {
            f += 2 * ni * nj * kk;
            b += es * ((ni + nj) * kk + 2 * ni * nj);
          }
          if (t.t0 == 0 && t.t1 == 0 && base < ns) {
            const double w2 = std::min(dct::kPanel, ns - base);
            f += 2.0 * w2 * w2 * w2 / 3.0;
          }
          break;
        }
        default:
          break;
      }
    }
    sc->flops[li] = f;
    sc->bytes[li] = b;
  }
}

// Tensor-core substitution tasks: one 128-row output tile t and a K range
// [k0, k1) per task (PanelTask {s, k0, t, k1}).  K ranges are split into
// pieces of at most kTcSplitK columns; a launch with fewer than
// kTcTargetCtas tasks halves the piece (down to kTcSplitMin) so that the top
// levels of the tree, which hold few supernodes, still fill the GPU.  Within
// a launch the longest tasks come first.
constexpr int kTcTile = 128;
#ifndef DCT_TC_SPLITK
#define DCT_TC_SPLITK 512
#endif
#ifndef DCT_TC_TARGET_CTAS
#define DCT_TC_TARGET_CTAS 592   // four waves of 148 SMs
#endif
#ifndef DCT_TC_SPLIT_MIN
#define DCT_TC_SPLIT_MIN 128
#endif
constexpr int kTcSplitK = DCT_TC_SPLITK;
constexpr int kTcTargetCtas = DCT_TC_TARGET_CTAS;
constexpr int kTcSplitMin = DCT_TC_SPLIT_MIN;

// The measured defaults of the schedule shapes (see dct_tuning in dct.h),
// and a user tuning with its zero fields defaulted and the rest clamped to
// what the kernels support.
// largest front the single-CTA kernel holds in shared memory (N^2 values)
int small_front_limit(int dtype) {
  return dtype == DCT_F64 ? dct::kSmallFrontF64
                          : (dtype == DCT_C128 ? dct::kSmallFrontC128 : dct::kSmallFrontF32);
}

dct_tuning default_tuning(int dtype) {
  dct_tuning t;
  t.small_front_max = small_front_limit(dtype);
  t.update_block = dtype == DCT_F32 ? dct::kUpdateBlockPanels : 1;
  t.solve_target = kTcTargetCtas;
  t.solve_split_max = kTcSplitK;
  t.solve_split_min = kTcSplitMin;
  t.small_tc = 0;
  return t;
}

dct_tuning resolve_tuning(int dtype, const dct_tuning* in) {
  dct_tuning t = default_tuning(dtype);
  if (in == nullptr) return t;
  const int smax = small_front_limit(dtype);
  if (in->small_front_max > 0) t.small_front_max = std::max(32, std::min(smax, in->small_front_max));
  // float64 fronts update after every panel (no blocking)
  if (in->update_block > 0 && dtype == DCT_F32) t.update_block = std::min(4, in->update_block);
  if (in->solve_target > 0) t.solve_target = in->solve_target;
  if (in->solve_split_max > 0) t.solve_split_max = std::max(16, in->solve_split_max);
  if (in->solve_split_min > 0) t.solve_split_min = std::max(16, in->solve_split_min);
  t.solve_split_min = std::min(t.solve_split_min, t.solve_split_max);
  if (in->small_tc > 0) t.small_tc = std::min(2, in->small_tc);
  return t;
}


void account_solve(const dct::Symbolic& S, dct::Schedule* sc, double es) {
  sc->flops.assign(sc->launches.size(), 0.0);
  sc->bytes.assign(sc->launches.size(), 0.0);
  sc->bytes_rhs.assign(sc->launches.size(), 0.0);
  for (size_t li = 0; li < sc->launches.size(); ++li) {
    const Launch& l = sc->launches[li];
    double f = 0, bf = 0, br = 0;
    for (int64_t q = l.first; q < l.first + l.count; ++q) {
      const PanelTask& t = sc->tasks[q];
      const int s = t.s, N = S.front_n[s], ns = S.ns(s);
      const double nbd = N - ns;
      if (l.kind == dct::kFwdSmall || l.kind == dct::kBwdSmall) {
        f += double(ns) * ns + 2 * nbd * ns;
        bf += es * (ns * (ns + 1) / 2.0 + nbd * ns);
        br += es * (2.0 * ns + (l.kind == dct::kFwdSmall ? 2 : 1) * nbd);
      } else if (l.kind == dct::kFwdLinv || l.kind == dct::kBwdLinv) {
        const double nr = std::min(dct::kPanel, ns - t.t0 * dct::kPanel);
        const double kk = l.kind == dct::kFwdLinv ? (t.t0 * dct::kPanel + nr)
                                                   : (ns - t.t0 * dct::kPanel);
        f += 2 * nr * kk;
        bf += es * nr * kk;
        br += es * (nr + kk);
      } else if (l.kind == dct::kFwdBnd) {
        const double nr = std::min(dct::kPanel, N - (ns + t.t0 * dct::kPanel));
        f += 2 * nr * ns;
        bf += es * nr * ns;
        br += es * (2 * nr + ns);
      } else if (l.kind == dct::kBwdGemm) {
        const double w = std::min(dct::kPanel, ns - t.p * dct::kPanel);
        f += 2 * nbd * w;
        bf += es * nbd * w;
        br += es * (nbd + 2.0 * w);
      } else if (l.kind >= dct::kFwdLinvTc && l.kind <= dct::kBwdLinvTc) {
        // entries of the A tile that are used (the inverses are triangular)
        const int m0 = t.t0 * kTcTile;
        const int mr = std::min(kTcTile, (l.kind == dct::kFwdBndTc ? N - ns : ns) - m0);
        double used = 0;
        if (l.kind == dct::kFwdLinvTc || l.kind == dct::kBwdLinvTc) {
          for (int m = m0; m < m0 + mr; ++m)
            used += l.kind == dct::kFwdLinvTc
                        ? std::max(0, std::min(t.t1, m + 1) - t.p)
                        : std::max(0, t.t1 - std::max(t.p, m));
        } else {
          used = double(mr) * (t.t1 - t.p);
        }
        f += 2 * used;
        bf += es * used;
        br += es * ((t.t1 - t.p) + 2.0 * mr);
      }
    }
    sc->flops[li] = f;
    sc->bytes[li] = bf;
    sc->bytes_rhs[li] = br;
  }
}

// trailing-update tile: 64 for float64 (CUDA cores), 128 for float32
// (tcgen05 tensor-core tiles, M = N = 128)
int update_tile(int dtype) { return dtype == DCT_F32 ? 128 : dct::kUpdateTile; }

#ifndef DCT_SMALL_BUCKETS
#define DCT_SMALL_BUCKETS 1
#endif
constexpr int kSmallBucketMin = 256;   // fronts: about two CTAs per SM of a B200

void build_factor_schedule(const dct::Symbolic& S, int small_max, int utile, int bpan,
                           bool align8, dct::Schedule* out) {
  auto& T = out->tasks;
  auto& L = out->launches;
  for (int lv = 0; lv < S.nlevels; ++lv) {
    std::vector<int> small, large;
    for (int q = S.level_ptr[lv]; q < S.level_ptr[lv + 1]; ++q) {
      int s = S.level_sn[q];
      (S.front_n[s] <= small_max ? small : large).push_back(s);
    }
    if (!small.empty()) {
      // The single-CTA kernel's shared memory is set by the largest front of
      // its launch, so the level's small fronts go into launches by order
      // (bounds at multiples of 32 rows): the smaller fronts then fit more
      // CTAs per SM.  A launch of fewer than kSmallBucketMin fronts would
      // leave most SMs idle and joins the next larger bucket.
      std::stable_sort(small.begin(), small.end(),
                       [&](int a, int b) { return S.front_n[a] < S.front_n[b]; });
      size_t i0 = 0;
      while (i0 < small.size()) {
        size_t i1 = small.size();
        if (DCT_SMALL_BUCKETS) {
          int bound = (S.front_n[small[i0]] + 31) / 32 * 32;
          for (;;) {
            i1 = i0;
            while (i1 < small.size() && S.front_n[small[i1]] <= bound) ++i1;
            if (i1 == small.size() || i1 - i0 >= size_t(kSmallBucketMin)) break;
            bound += 32;
          }
          // a last bucket too small to stand alone joins this one
          if (small.size() - i1 < size_t(kSmallBucketMin)) i1 = small.size();
        }
        Launch l{dct::kSmallFront, lv, int64_t(T.size()), int64_t(i1 - i0), 0};
        for (size_t i = i0; i < i1; ++i) {
          T.push_back({small[i], 0, 0, 0});
          l.arg = std::max(l.arg, S.front_n[small[i]]);
        }
        L.push_back(l);
        i0 = i1;
      }
    }
    if (large.empty()) continue;
    {
      Launch l{dct::kLargeScatter, lv, int64_t(T.size()), int64_t(large.size()), 0};
      for (int s : large) T.push_back({s, 0, 0, 0});
      L.push_back(l);
    }
    int max_children = 0;
    for (int s : large)
      max_children = std::max(max_children, S.child_ptr[s + 1] - S.child_ptr[s]);
    for (int slot = 0; slot < max_children; ++slot) {
      Launch l{dct::kLargeExtendAdd, lv, int64_t(T.size()), 0, slot};
      for (int s : large) {
        int nch = S.child_ptr[s + 1] - S.child_ptr[s];
        if (slot >= nch) continue;
        int c = S.child[S.child_ptr[s] + slot];
        int nbc = S.nb(c);
        for (int j = 0; j < nbc; j += 8) T.push_back({s, 0, c, j});
      }
      l.count = int64_t(T.size()) - l.first;
      L.push_back(l);
    }
    {
      // the first panel's diagonal block of every large front
      Launch ld{dct::kLargeUpdate, lv, int64_t(T.size()), int64_t(large.size()), 0};
      for (int s : large) T.push_back({s, 0, -1, 0});
      L.push_back(ld);
    }
    int max_panels = 0;
    for (int s : large) max_panels = std::max(max_panels, ceil_div(S.ns(s), dct::kPanel));
    for (int p = 0; p < max_panels; ++p) {
      Launch lp{dct::kLargePanel, lv, int64_t(T.size()), 0, p};
      for (int s : large) {
        int ns = S.ns(s), N = S.front_n[s];
        int c0 = p * dct::kPanel;
        if (c0 >= ns) continue;
        int w = std::min(dct::kPanel, ns - c0);
        int nt = ceil_div(N - c0 - w, dct::kPanel);
        for (int t = 1; t <= nt; ++t) T.push_back({s, p, t, 0});
      }
      lp.count = int64_t(T.size()) - lp.first;
      L.push_back(lp);
      Launch lu{dct::kLargeUpdate, lv, int64_t(T.size()), 0, p};
      for (int s : large) {
        int ns = S.ns(s), N = S.front_n[s];
        int c0 = p * dct::kPanel;
        if (c0 >= ns) continue;
        int w = std::min(dct::kPanel, ns - c0);
        const dct::UpdateRange R = dct::update_range(p, ns, N, bpan);
        const int R0 = update_origin(c0 + w, align8);
        // no tile when nothing lies beyond the panel (R0 may sit above it)
        int nti = N > c0 + w ? ceil_div(N - R0, utile) : 0;
        int ntj = R.cend > c0 + w ? ceil_div(R.cend - R0, utile) : 0;
        for (int i = 0; i < nti; ++i)
          for (int j = 0; j <= i && j < ntj; ++j) T.push_back({s, p, i, j});
      }
      lu.count = int64_t(T.size()) - lu.first;
      L.push_back(lu);
    }
  }
}

// Forward and backward substitution schedules.  Per level of the assembly
// tree: single-panel supernodes run one CTA each (kFwdSmall / kBwdSmall);
// larger ones multiply by their precomputed inverse L_ss^{-1}
// (kFwdLinv / kBwdLinv, 64-row tiles) and exchange with their boundary rows
// once (kFwdBnd[Tc] after, kBwdGemm before).  A pass is a few launches per
// level, independent of the supernodes' widths.
void push_split(std::vector<PanelTask>& T, int s, int t, int k0, int k1, int split) {
  for (int a = k0; a < k1; a += split) T.push_back({s, a, t, std::min(k1, a + split)});
}

void build_solve_schedules(const dct::Symbolic& S, int dtype, const dct_tuning& tu,
                           dct::Schedule* fwd, dct::Schedule* bwd) {
  const bool tc = dtype == DCT_F32;
  // Single-panel supernodes run in one CTA each (k_fwd_small / k_bwd_small),
  // except in float32 plans whose single-panel fronts are mostly large (at
  // least kTcSmallFront rows hold most of their substitution work, as in 3-D
  // grids): there they all take the tensor-core products with every right-
  // hand side in one CTA.  For small fronts (2-D grids) a one-CTA-per-SM
  // tensor-core task costs more than it saves.
  constexpr int kTcSmallFront = 128;
  bool small_tc = false;
  if (tc && tu.small_tc == 1) {
    small_tc = true;
  } else if (tc && tu.small_tc != 2) {
    double big = 0, all = 0;
    for (int s = 0; s < S.nsuper; ++s) {
      const double ns = S.ns(s), nb = S.nb(s);
      if (ns > dct::kPanel) continue;
      const double wk = ns * ns + 2 * nb * ns;
      all += wk;
      if (S.front_n[s] >= kTcSmallFront) big += wk;
    }
    small_tc = all > 0 && big >= 0.5 * all;
  }
  auto is_small = [&](int s) { return S.ns(s) <= dct::kPanel && !small_tc; };
  int split = tu.solve_split_max;   // K piece of the tensor-core tasks being filled
  std::vector<PanelTask> tmp;
  auto add = [&](dct::Schedule* sc, int kind, int lv, auto&& fill) {
    Launch l{kind, lv, int64_t(sc->tasks.size()), 0, 0};
    for (split = tu.solve_split_max;; split /= 2) {
      tmp.clear();
      fill(tmp);
      if (!tc || int64_t(tmp.size()) >= tu.solve_target || split / 2 < tu.solve_split_min)
        break;
    }
    sc->tasks.insert(sc->tasks.end(), tmp.begin(), tmp.end());
    l.count = int64_t(sc->tasks.size()) - l.first;
    if (tc && l.count)
      std::stable_sort(sc->tasks.begin() + l.first, sc->tasks.end(),
                       [](const PanelTask& x, const PanelTask& y) {
                         return x.t1 - x.p > y.t1 - y.p;
                       });
    if (l.count) sc->launches.push_back(l);
  };
  for (int lv = 0; lv < S.nlevels; ++lv) {
    const int q0 = S.level_ptr[lv], q1 = S.level_ptr[lv + 1];
    add(fwd, dct::kFwdSmall, lv, [&](std::vector<PanelTask>& T) {
      for (int q = q0; q < q1; ++q)
        if (is_small(S.level_sn[q])) T.push_back({S.level_sn[q], 0, 0, 0});
    });
    add(fwd, tc ? dct::kFwdLinvTc : dct::kFwdLinv, lv, [&](std::vector<PanelTask>& T) {
      for (int q = q0; q < q1; ++q) {
        const int s = S.level_sn[q], ns = S.ns(s);
        if (is_small(s)) continue;
        if (tc) {
          for (int t = 0; t * kTcTile < ns; ++t)
            push_split(T, s, t, 0, std::min(ns, (t + 1) * kTcTile), split);
        } else {
          for (int t = 0; t * dct::kPanel < ns; ++t) T.push_back({s, 0, t, 0});
        }
      }
    });
    add(fwd, tc ? dct::kFwdBndTc : dct::kFwdBnd, lv, [&](std::vector<PanelTask>& T) {
      for (int q = q0; q < q1; ++q) {
        const int s = S.level_sn[q];
        if (is_small(s)) continue;
        if (tc) {
          for (int t = 0; t < ceil_div(S.nb(s), kTcTile); ++t) push_split(T, s, t, 0, S.ns(s), split);
        } else {
          for (int t = 0; t < ceil_div(S.nb(s), dct::kPanel); ++t) T.push_back({s, 0, t, 0});
        }
      }
    });
  }
  for (int lv = S.nlevels - 1; lv >= 0; --lv) {
    const int q0 = S.level_ptr[lv], q1 = S.level_ptr[lv + 1];
    add(bwd, dct::kBwdSmall, lv, [&](std::vector<PanelTask>& T) {
      for (int q = q0; q < q1; ++q)
        if (is_small(S.level_sn[q])) T.push_back({S.level_sn[q], 0, 0, 0});
    });
    add(bwd, tc ? dct::kBwdGemmTc : dct::kBwdGemm, lv, [&](std::vector<PanelTask>& T) {
      for (int q = q0; q < q1; ++q) {
        const int s = S.level_sn[q], ns = S.ns(s);
        if (is_small(s) || S.nb(s) == 0) continue;
        if (tc) {
          for (int t = 0; t * kTcTile < ns; ++t) push_split(T, s, t, 0, S.nb(s), split);
        } else {
          for (int p = 0; p * dct::kPanel < ns; ++p) T.push_back({s, p, 0, 0});
        }
      }
    });
    add(bwd, tc ? dct::kBwdLinvTc : dct::kBwdLinv, lv, [&](std::vector<PanelTask>& T) {
      for (int q = q0; q < q1; ++q) {
        const int s = S.level_sn[q], ns = S.ns(s);
        if (is_small(s)) continue;
        if (tc) {
          for (int t = 0; t * kTcTile < ns; ++t) push_split(T, s, t, t * kTcTile, ns, split);
        } else {
          for (int t = 0; t * dct::kPanel < ns; ++t) T.push_back({s, 0, t, 0});
        }
      }
    });
  }
}

// Supernode inverses L_ss^{-1} (ns > 64) by recursive doubling from the
// 64-column panel inverses: with L = [[A, 0], [C, D]] over blocks of h and
// h' <= h columns, L^{-1} = [[A^{-1}, 0], [-D^{-1} C A^{-1}, D^{-1}]].  Level h
// runs two launches over every pair of blocks: T = C A^{-1}, then
// X = -D^{-1} T, on 64 x 64 output tiles (t0 = tile row, t1 = tile column,
// p = pair index, launch arg = h).  Offsets: ns^2 elements per supernode.
// Float32 plans keep an inverse for every supernode (single-panel ones too:
// their substitution runs on the same tensor-core products); float64 plans
// only for supernodes wider than one panel.
void build_linv_schedule(const dct::Symbolic& S, int dtype, dct::Schedule* sc,
                         std::vector<int64_t>* off, int64_t* total) {
  const int min_ns = dtype == DCT_F32 ? 1 : dct::kPanel + 1;
  off->assign(S.nsuper, -1);
  int64_t acc = 0;
  int max_ns = 0;
  for (int s = 0; s < S.nsuper; ++s) {
    const int ns = S.ns(s);
    if (ns < min_ns) continue;
    (*off)[s] = acc;
    acc += int64_t(ns) * ns;
    max_ns = std::max(max_ns, ns);
  }
  *total = acc;
  {
    Launch l{dct::kLinvInit, 0, int64_t(sc->tasks.size()), 0, 0};
    for (int s = 0; s < S.nsuper; ++s)
      if (S.ns(s) >= min_ns)
        for (int p = 0; p * dct::kPanel < S.ns(s); ++p) sc->tasks.push_back({s, p, 0, 0});
    l.count = int64_t(sc->tasks.size()) - l.first;
    if (l.count) sc->launches.push_back(l);
  }
  for (int h = dct::kPanel; h < max_ns; h *= 2) {
    for (int kind : {int(dct::kLinvT), int(dct::kLinvX)}) {
      Launch l{kind, 0, int64_t(sc->tasks.size()), 0, h};
      for (int s = 0; s < S.nsuper; ++s) {
        const int ns = S.ns(s);
        if (ns <= dct::kPanel) continue;
        for (int i = 0; 2 * i * h + h < ns; ++i) {
          const int d0 = 2 * i * h + h;
          const int hd = std::min(h, ns - d0);
          for (int r = 0; r < ceil_div(hd, dct::kPanel); ++r)
            for (int c = 0; c < h / dct::kPanel; ++c) sc->tasks.push_back({s, i, r, c});
        }
      }
      l.count = int64_t(sc->tasks.size()) - l.first;
      if (l.count) sc->launches.push_back(l);
    }
  }
}

// diagonal-block inverse of every panel, and where each supernode's panel
// inverses start (sum over earlier panels of w^2)
void build_inverse_schedule(const dct::Symbolic& S, int small_max,
                            dct::Schedule* inv, std::vector<int64_t>* off,
                            int64_t* total) {
  off->assign(S.nsuper, 0);
  int64_t acc = 0;
  for (int s = 0; s < S.nsuper; ++s) {
    (*off)[s] = acc;
    const int ns = S.ns(s);
    for (int p = 0; p * dct::kPanel < ns; ++p) {
      const int64_t w = std::min(dct::kPanel, ns - p * dct::kPanel);
      // large fronts store their inverses while factoring
      if (S.front_n[s] <= small_max) inv->tasks.push_back({s, p, 0, 0});
      acc += w * w;
    }
  }
  *total = acc;
  inv->launches.push_back({dct::kPanelInverse, 0, 0, int64_t(inv->tasks.size()), 0});
}

// Float32 plans of one system: the trailing-update launches with many tiles
// and few fronts run persistent CTAs (update_tc.cu), which need the diagonal
// tile of every front -- the one whose CTA then factors the next diagonal
// block -- ahead of the other tiles.  The tiles of one launch are
// independent, so the order inside a launch is free.
#ifndef DCT_U_PERSISTENT
#define DCT_U_PERSISTENT 1
#endif
#ifndef DCT_U_PERSIST_MAX_FRONTS
#define DCT_U_PERSIST_MAX_FRONTS 32
#endif
void plan_persistent_updates(dct_plan* P) {
  P->update_nspec.assign(P->fact.launches.size(), -1);
  if (!DCT_U_PERSISTENT || P->dtype != DCT_F32 || P->nbatch != 1) return;
  auto diagonal = [](const PanelTask& t) { return t.t0 < 0 || (t.t0 == 0 && t.t1 == 0); };
  for (size_t li = 0; li < P->fact.launches.size(); ++li) {
    const Launch& L = P->fact.launches[li];
    if (L.kind != dct::kLargeUpdate || L.count <= 0) continue;
    auto b = P->fact.tasks.begin() + L.first;
    auto e = b + L.count;
    const int64_t nspec = std::count_if(b, e, diagonal);
    const int64_t pers = int64_t(P->sm_count) - nspec;
    // each persistent CTA takes two tiles or more
    if (nspec > DCT_U_PERSIST_MAX_FRONTS || pers < 1 || L.count - nspec < 2 * pers) continue;
    std::stable_partition(b, e, diagonal);
    P->update_nspec[li] = static_cast<int32_t>(nspec);
  }
}

int upload_schedule(dct_plan* P, dct::Schedule* sch) {
  const PanelTask* d = nullptr;
  int rc = upload(P, sch->tasks, &d);
  sch->d_tasks = const_cast<PanelTask*>(d);
  return rc;
}

size_t esize(int dtype) { return dtype == DCT_F64 ? 8 : (dtype == DCT_C128 ? 16 : 4); }
bool valid_dtype(int dtype) { return dtype == DCT_F64 || dtype == DCT_F32 || dtype == DCT_C128; }

int set_device(int device) {
  int cur = -1;
  cudaError_t e = cudaGetDevice(&cur);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (cur != device) {
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  }
  return DCT_OK;
}

}  // namespace

void dct::set_last_error(const char* msg) { g_err = msg; }

cudaError_t dct::Profiler::begin(int kind, double flops, double bytes,
                                 cudaStream_t st) {
  if (!on) return cudaSuccess;
  Rec r{kind, nullptr, nullptr, flops, bytes};
  for (cudaEvent_t* ev : {&r.a, &r.b}) {
    if (!pool.empty()) {
      *ev = pool.back();
      pool.pop_back();
    } else {
      cudaError_t e = cudaEventCreate(ev);
      if (e != cudaSuccess) return e;
    }
  }
  recs.push_back(r);
  return cudaEventRecord(r.a, st);
}

cudaError_t dct::Profiler::end(cudaStream_t st) {
  if (!on || recs.empty()) return cudaSuccess;
  return cudaEventRecord(recs.back().b, st);
}

cudaError_t dct::Profiler::collect() {
  for (Rec& r : recs) {
    cudaError_t e = cudaEventSynchronize(r.b);
    if (e != cudaSuccess) return e;
    float t = 0.f;
    e = cudaEventElapsedTime(&t, r.a, r.b);
    if (e != cudaSuccess) return e;
    ms[r.kind] += t;
    fl[r.kind] += r.flops;
    by[r.kind] += r.bytes;
    n[r.kind] += 1;
    log_kind.push_back(r.kind);
    log_ms.push_back(t);
    pool.push_back(r.a);
    pool.push_back(r.b);
  }
  recs.clear();
  return cudaSuccess;
}

void dct::Profiler::reset() {
  for (int k = 0; k < kNumKinds; ++k) {
    ms[k] = fl[k] = by[k] = 0.0;
    n[k] = 0;
  }
  log_kind.clear();
  log_ms.clear();
}

extern "C" {

int dct_version(void) { return 10000; }

const char* dct_last_error(void) { return g_err.c_str(); }

int dct_symbolic_create(int32_t n, const int32_t* crow, const int32_t* col,
                        const int32_t* coords, int32_t ndim, int32_t leaf_size,
                        dct_symbolic** out) {
  if (!out || !crow || !col || n <= 0) return fail(DCT_ERR_ARG, "bad arguments");
  *out = nullptr;
  auto* h = new (std::nothrow) dct_symbolic();
  if (!h) return fail(DCT_ERR_OOM, "host allocation");
  dct::SymbolicOptions opt;
  if (leaf_size > 0) opt.leaf_size = leaf_size;
  std::string why;
  try {
    why = dct::analyse(n, crow, col, coords, ndim, opt, &h->sym);
  } catch (const std::exception& ex) {
    delete h;
    return fail(DCT_ERR_OOM, std::string("symbolic analysis: ") + ex.what());
  }
  if (!why.empty()) {
    delete h;
    return fail(DCT_ERR_BAD_PATTERN, why);
  }
  *out = h;
  return DCT_OK;
}

void dct_symbolic_destroy(dct_symbolic* sym) { delete sym; }

int dct_symbolic_get_info(const dct_symbolic* h, dct_symbolic_info* out) {
  if (!h || !out) return fail(DCT_ERR_ARG, "null argument");
  const dct::Symbolic& S = h->sym;
  out->n = S.n;
  out->nnz_in = S.nnz_in;
  out->nsuper = S.nsuper;
  out->nlevels = S.nlevels;
  out->max_front = S.max_front;
  out->max_ns = S.max_ns;
  out->nnz_L = S.nnz_L;
  out->front_total = S.front_total;
  out->flops_factor = S.flops_factor;
  return DCT_OK;
}

int dct_symbolic_get_array(const dct_symbolic* h, const char* name, void* dst,
                           int64_t capacity_bytes, int64_t* size_bytes) {
  if (!h || !name) return fail(DCT_ERR_ARG, "null argument");
  const dct::Symbolic& S = h->sym;
  const void* src = nullptr;
  int64_t bytes = 0;
  auto pick32 = [&](const std::vector<int32_t>& v) {
    src = v.data();
    bytes = int64_t(v.size()) * 4;
  };
  auto pick64 = [&](const std::vector<int64_t>& v) {
    src = v.data();
    bytes = int64_t(v.size()) * 8;
  };
  std::string nm(name);
  if (nm == "perm") pick32(S.perm);
  else if (nm == "iperm") pick32(S.iperm);
  else if (nm == "sn_first") pick32(S.sn_first);
  else if (nm == "sn_parent") pick32(S.sn_parent);
  else if (nm == "sn_level") pick32(S.sn_level);
  else if (nm == "front_n") pick32(S.front_n);
  else if (nm == "front_off") pick64(S.front_off);
  else if (nm == "rows_ptr") pick64(S.rows_ptr);
  else if (nm == "rows") pick32(S.rows);
  else if (nm == "child_ptr") pick32(S.child_ptr);
  else if (nm == "child") pick32(S.child);
  else if (nm == "rel_ptr") pick64(S.rel_ptr);
  else if (nm == "rel") pick32(S.rel);
  else if (nm == "amap_ptr") pick64(S.amap_ptr);
  else if (nm == "amap_e") pick32(S.amap_e);
  else if (nm == "amap_pos") pick32(S.amap_pos);
  else return fail(DCT_ERR_ARG, "unknown array " + nm);
  if (size_bytes) *size_bytes = bytes;
  if (dst) {
    if (capacity_bytes < bytes) return fail(DCT_ERR_ARG, "destination too small");
    if (bytes) std::memcpy(dst, src, bytes);
  }
  return DCT_OK;
}

int dct_symbolic_get_schedule(const dct_symbolic* h, int32_t dtype, int32_t which,
                              int32_t* tasks, int64_t* ntasks, int64_t* launches,
                              int64_t* nlaunches) {
  if (!h || !ntasks || !nlaunches || which < 0 || which > 4 || !valid_dtype(dtype))
    return fail(DCT_ERR_ARG, "bad arguments");
  dct::Schedule f, fw, bw, iv;
  const dct_tuning tu = default_tuning(dtype);
  const int small_max = tu.small_front_max;
  build_factor_schedule(h->sym, small_max, update_tile(dtype), tu.update_block,
                        dtype == DCT_F32, &f);
  build_solve_schedules(h->sym, dtype, tu, &fw, &bw);
  std::vector<int64_t> off;
  int64_t tot = 0;
  build_inverse_schedule(h->sym, small_max, &iv, &off, &tot);
  dct::Schedule lv;
  std::vector<int64_t> loff;
  int64_t ltot = 0;
  build_linv_schedule(h->sym, dtype, &lv, &loff, &ltot);
  const dct::Schedule& sc =
      which == 0 ? f : (which == 1 ? fw : (which == 2 ? bw : (which == 3 ? iv : lv)));
  const int64_t nt = int64_t(sc.tasks.size()), nl = int64_t(sc.launches.size());
  if (tasks) {
    if (*ntasks < nt) return fail(DCT_ERR_ARG, "task buffer too small");
    for (int64_t i = 0; i < nt; ++i) {
      tasks[4 * i + 0] = sc.tasks[i].s;
      tasks[4 * i + 1] = sc.tasks[i].p;
      tasks[4 * i + 2] = sc.tasks[i].t0;
      tasks[4 * i + 3] = sc.tasks[i].t1;
    }
  }
  if (launches) {
    if (*nlaunches < nl) return fail(DCT_ERR_ARG, "launch buffer too small");
    for (int64_t i = 0; i < nl; ++i) {
      const Launch& l = sc.launches[i];
      launches[5 * i + 0] = l.kind;
      launches[5 * i + 1] = l.level;
      launches[5 * i + 2] = l.first;
      launches[5 * i + 3] = l.count;
      launches[5 * i + 4] = l.arg;
    }
  }
  *ntasks = nt;
  *nlaunches = nl;
  return DCT_OK;
}

void dct_plan_destroy(dct_plan* P) {
  if (!P) return;
  int cur = -1;
  cudaGetDevice(&cur);
  cudaSetDevice(P->device);
  for (void* p : P->owned) cudaFree(p);
  if (cur >= 0) cudaSetDevice(cur);
  delete P;
}

int dct_tuning_default(int32_t dtype, dct_tuning* out) {
  if (!out || !valid_dtype(dtype)) return fail(DCT_ERR_ARG, "bad arguments");
  *out = default_tuning(dtype);
  return DCT_OK;
}

int dct_plan_get_tuning(const dct_plan* P, dct_tuning* out) {
  if (!P || !out) return fail(DCT_ERR_ARG, "null argument");
  *out = P->tune;
  return DCT_OK;
}

int dct_plan_create(const dct_symbolic* h, int32_t nbatch, int32_t max_rhs,
                    int32_t dtype, int32_t device, dct_plan** out) {
  return dct_plan_create_tuned(h, nbatch, max_rhs, dtype, device, nullptr, out);
}

int dct_plan_create_tuned(const dct_symbolic* h, int32_t nbatch, int32_t max_rhs,
                          int32_t dtype, int32_t device, const dct_tuning* tuning,
                          dct_plan** out) {
  if (!h || !out || nbatch < 1 || max_rhs < 1 ||
      !valid_dtype(dtype))
    return fail(DCT_ERR_ARG, "bad arguments");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(DCT_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(DCT_ERR_ARG, "bad device");
  int rc = set_device(device);
  if (rc) return rc;
  auto* P = new (std::nothrow) dct_plan();
  if (!P) return fail(DCT_ERR_OOM, "host allocation");
  P->sym = h->sym;
  P->device = device;
  P->nbatch = nbatch;
  P->max_rhs = max_rhs;
  P->dtype = dtype;
  const dct::Symbolic& S = P->sym;
  auto bail = [&](int code) {
    dct_plan_destroy(P);
    return code;
  };
  dct::DevSym& D = P->ds;
  if ((rc = upload(P, S.sn_first, &D.sn_first)) || (rc = upload(P, S.front_n, &D.front_n)) ||
      (rc = upload(P, S.front_off, &D.front_off)) || (rc = upload(P, S.rows_ptr, &D.rows_ptr)) ||
      (rc = upload(P, S.rows, &D.rows)) || (rc = upload(P, S.amap_ptr, &D.amap_ptr)) ||
      (rc = upload(P, S.amap_e, &D.amap_e)) || (rc = upload(P, S.amap_pos, &D.amap_pos)) ||
      (rc = upload(P, S.child_ptr, &D.child_ptr)) || (rc = upload(P, S.child, &D.child)) ||
      (rc = upload(P, S.rel_ptr, &D.rel_ptr)) || (rc = upload(P, S.rel, &D.rel)) ||
      (rc = upload(P, S.perm, &D.perm)) || (rc = upload(P, S.iperm, &D.iperm)) ||
      (rc = upload(P, S.in_crow, &D.crow)) || (rc = upload(P, S.in_col, &D.col)))
    return bail(rc);
  P->tune = resolve_tuning(dtype, tuning);
  const int small_max = P->tune.small_front_max;
  build_factor_schedule(S, small_max, update_tile(dtype), P->tune.update_block,
                        dtype == DCT_F32, &P->fact);
  P->update_bpan = P->tune.update_block;
  {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess &&
        sms > 0)
      P->sm_count = sms;
  }
  plan_persistent_updates(P);
  build_solve_schedules(S, dtype, P->tune, &P->fwd, &P->bwd);
  std::vector<int64_t> dinv_off;
  build_inverse_schedule(S, small_max, &P->inv, &dinv_off, &P->dinv_stride);
  {
    const int64_t* d = nullptr;
    if ((rc = upload(P, dinv_off, &d))) return bail(rc);
    P->d_dinv_off = d;
  }
  std::vector<int64_t> linv_off;
  build_linv_schedule(S, dtype, &P->linv_sched, &linv_off, &P->linv_stride);
  {
    const int64_t* d = nullptr;
    if ((rc = upload(P, linv_off, &d))) return bail(rc);
    P->d_linv_off = d;
  }
  if (dtype == DCT_F32) {
    // split images of every panel of the large fronts (update_tc.cu)
    std::vector<int32_t> pan_first(S.nsuper + 1, 0);
    std::vector<int64_t> img_off;
    int64_t acc = 0;
    for (int s = 0; s < S.nsuper; ++s) {
      pan_first[s] = int32_t(img_off.size());
      const int ns = S.ns(s), N = S.front_n[s];
      for (int q = 0; q * dct::kPanel < ns; ++q) {
        img_off.push_back(acc);
        if (N > small_max) acc += dct::img_floats(dct::img_groups(q, ns, N));
      }
    }
    pan_first[S.nsuper] = int32_t(img_off.size());
    img_off.push_back(acc);
    const int64_t* d_off = nullptr;
    const int32_t* d_pf = nullptr;
    if ((rc = upload(P, img_off, &d_off)) || (rc = upload(P, pan_first, &d_pf))) return bail(rc);
    void* img = nullptr;
    if ((rc = alloc(P, sizeof(float) * size_t(acc) * nbatch, &img, "panel images")))
      return bail(rc);
    // padding rows and the columns beyond a narrow panel are never written
    if (cudaMemset(img, 0, sizeof(float) * size_t(acc) * nbatch) != cudaSuccess)
      return bail(fail(DCT_ERR_CUDA, "cudaMemset (panel images)"));
    P->img = dct::ImgArgs{static_cast<float*>(img), d_off, d_pf, acc};
  }
  account_factor(S, &P->fact, double(esize(dtype)), update_tile(dtype),
                 P->update_bpan, dtype == DCT_F32);
  account_solve(S, &P->fwd, double(esize(dtype)));
  account_solve(S, &P->bwd, double(esize(dtype)));
  if ((rc = upload_schedule(P, &P->fact)) || (rc = upload_schedule(P, &P->fwd)) ||
      (rc = upload_schedule(P, &P->bwd)) || (rc = upload_schedule(P, &P->inv)) ||
      (rc = upload_schedule(P, &P->linv_sched)))
    return bail(rc);
  const size_t es = esize(dtype);
  P->front_stride = S.front_total;
  const size_t work = size_t(nbatch) * S.n * max_rhs;
  void* p = nullptr;
  if ((rc = alloc(P, es * S.front_total * nbatch, &P->fronts, "front storage")))
    return bail(rc);
  if ((rc = alloc(P, es * P->dinv_stride * nbatch, &P->dinv, "panel inverses")))
    return bail(rc);
  if ((rc = alloc(P, es * P->linv_stride * nbatch, &P->linv, "supernode inverses")))
    return bail(rc);
  if ((rc = alloc(P, es * P->linv_stride * nbatch, &P->ltmp, "inverse products")))
    return bail(rc);
  if ((rc = alloc(P, es * work, &P->bufA, "work buffer A"))) return bail(rc);
  if ((rc = alloc(P, es * work, &P->bufB, "work buffer B"))) return bail(rc);
  if (dtype == DCT_F32) {
    if ((rc = alloc(P, 8 * work, &p, "refinement iterate"))) return bail(rc);
    P->x64 = static_cast<double*>(p);
    if ((rc = alloc(P, 8 * work, &p, "refinement rhs"))) return bail(rc);
    P->b64 = static_cast<double*>(p);
    if ((rc = alloc(P, 8 * size_t(nbatch) * S.nnz_in, &p, "float64 values")))
      return bail(rc);
    P->vals64 = static_cast<double*>(p);
  }
  if ((rc = alloc(P, 64, &p, "status"))) return bail(rc);
  P->status = static_cast<int*>(p);
  if ((rc = alloc(P, 16, &p, "residual"))) return bail(rc);
  P->resid_bits = static_cast<unsigned long long*>(p);
  if ((rc = alloc(P, sizeof(dct::IrState), &p, "refinement state"))) return bail(rc);
  P->ir = static_cast<dct::IrState*>(p);
  if (cudaMemset(P->status, 0, 64) != cudaSuccess ||
      cudaMemset(P->resid_bits, 0, 16) != cudaSuccess ||
      cudaMemset(P->ir, 0, sizeof(dct::IrState)) != cudaSuccess)
    return bail(fail(DCT_ERR_CUDA, "cudaMemset"));
  *out = P;
  return DCT_OK;
}

int dct_plan_create_general(const dct_symbolic* h, int32_t nbatch, int32_t max_rhs,
                            int32_t device, dct_plan** out) {
  if (!h || !out) return fail(DCT_ERR_ARG, "bad arguments");
  *out = nullptr;
  // the transpose map: entry (i, j) -> entry (j, i) of the input pattern,
  // which must hold both (structurally symmetric)
  const dct::Symbolic& S0 = h->sym;
  const int n = S0.n;
  std::vector<int32_t> tr(S0.in_col.size(), -1);
  for (int i = 0; i < n; ++i)
    for (int64_t e = S0.in_crow[i]; e < S0.in_crow[i + 1]; ++e) {
      const int j = S0.in_col[e];
      if (j < 0 || j >= n) return fail(DCT_ERR_BAD_PATTERN, "column out of range");
      for (int64_t f = S0.in_crow[j]; f < S0.in_crow[j + 1]; ++f)
        if (S0.in_col[f] == i) {
          tr[e] = static_cast<int32_t>(f);
          break;
        }
      if (tr[e] < 0)
        return fail(DCT_ERR_BAD_PATTERN, "pattern not structurally symmetric: (i, j) without (j, i)");
    }
  dct_plan* P = nullptr;
  int rc = dct_plan_create_tuned(h, nbatch, max_rhs, DCT_F64, device, nullptr, &P);
  if (rc) return rc;
  auto bail = [&](int code) {
    dct_plan_destroy(P);
    return code;
  };
  P->lu = 1;
  // static pivoting at sqrt(eps) of the block's largest entry
  P->pivot_floor = 1.4901161193847656e-08;
  const int32_t* d_tr = nullptr;
  if ((rc = upload(P, tr, &d_tr))) return bail(rc);
  P->d_tr = d_tr;
  if ((rc = alloc(P, 8 * size_t(P->sym.front_total) * nbatch, &P->fronts2, "front storage (U^T)")))
    return bail(rc);
  if ((rc = alloc(P, 8 * size_t(P->dinv_stride) * nbatch, &P->dinv2, "panel inverses (U^T)")))
    return bail(rc);
  if ((rc = alloc(P, 8 * size_t(P->linv_stride) * nbatch, &P->linv2,
                  "supernode inverses (U^T)")))
    return bail(rc);
  *out = P;
  return DCT_OK;
}

int dct_plan_static_pivots(dct_plan* P, void* stream, int32_t* count) {
  if (!P || !count) return fail(DCT_ERR_ARG, "bad arguments");
  int rc = set_device(P->device);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int h = 0;
  DCT_CUDA(cudaMemcpyAsync(&h, P->status + 4, sizeof(int), cudaMemcpyDeviceToHost, st),
           "status read");
  DCT_CUDA(cudaStreamSynchronize(st), "stream synchronize");
  *count = h;
  return DCT_OK;
}

int dct_plan_set_refinement(dct_plan* P, int32_t iterations) {
  if (!P || iterations < 0 || iterations > 64) return fail(DCT_ERR_ARG, "bad arguments");
  P->ir_iters = iterations;
  return DCT_OK;
}

int dct_plan_set_refinement_tolerance(dct_plan* P, double tol) {
  if (!P || !(tol >= 0.0)) return fail(DCT_ERR_ARG, "bad arguments");
  P->ir_tol = tol;
  return DCT_OK;
}

int dct_plan_refinement_info(dct_plan* P, void* stream, int32_t* iters,
                             int32_t* converged, double* est_error, double* rho,
                             int32_t capacity) {
  if (!P || capacity < 0) return fail(DCT_ERR_ARG, "bad arguments");
  int rc = set_device(P->device);
  if (rc) return rc;
  dct::IrState h{};
  if (P->ir != nullptr) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    DCT_CUDA(cudaMemcpyAsync(&h, P->ir, sizeof(h), cudaMemcpyDeviceToHost, st),
             "refinement state read");
    DCT_CUDA(cudaStreamSynchronize(st), "stream synchronize");
  }
  if (iters) *iters = h.iters;
  if (converged) *converged = h.converged;
  if (est_error) *est_error = h.est;
  if (rho)
    for (int i = 0; i < capacity && i < h.iters && i < dct::kIrHistory; ++i) rho[i] = h.rho[i];
  return DCT_OK;
}

int dct_plan_iperm(const dct_plan* P, const int32_t** d_iperm) {
  if (!P || !d_iperm) return fail(DCT_ERR_ARG, "null argument");
  *d_iperm = P->ds.iperm;
  return DCT_OK;
}

int64_t dct_plan_stamp(const dct_plan* P) { return P ? P->stamp : -1; }

int dct_factorize(dct_plan* P, const void* d_vals, int32_t vals_dtype,
                  int64_t vals_batch_stride, void* stream) {
  if (!P || !d_vals || !valid_dtype(vals_dtype) ||
      ((vals_dtype == DCT_C128) != (P->dtype == DCT_C128)))
    return fail(DCT_ERR_ARG, "bad arguments (complex values need a complex plan and back)");
  if (P->lu && vals_dtype != DCT_F64)
    return fail(DCT_ERR_ARG, "general plans take float64 values");
  int rc = set_device(P->device);
  if (rc) return rc;
  if (P->lu)
    DCT_CUDA(cudaMemsetAsync(P->status + 4, 0, sizeof(int), static_cast<cudaStream_t>(stream)),
             "static pivot count reset");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (P->dtype == DCT_F32) {
    // keep float64 values for the refinement residual
    DCT_CUDA(dct::launch_convert_any(d_vals, vals_dtype, vals_batch_stride,
                                     P->sym.nnz_in, P->nbatch, P->vals64,
                                     DCT_F64, st),
             "value copy");
  }
  DCT_CUDA(dct::run_factor(P, d_vals, vals_dtype, vals_batch_stride, st),
           "factorization launch");
  P->factored = 1;
  ++P->stamp;
  return DCT_OK;
}

namespace {

// f32 plans: solve bp -> xp (both float64, permuted) with refinement.
int solve_refined(dct_plan* P, const double* bp, int64_t bstride, int k,
                  double* xp, cudaStream_t st) {
  const int n = P->sym.n;
  const int64_t per = int64_t(n) * k;
  DCT_CUDA(cudaMemsetAsync(P->resid_bits, 0, 16, st), "memset");
  DCT_CUDA(cudaMemsetAsync(P->ir, 0, sizeof(dct::IrState), st), "memset");
  DCT_CUDA(dct::launch_convert_any(bp, DCT_F64, bstride, per, P->nbatch, P->bufA,
                                   DCT_F32, st),
           "rhs conversion");
  DCT_CUDA(dct::run_solve_f32(P, k, st), "solve launch");
  DCT_CUDA(dct::launch_ir_update(P, xp, k, 1, st), "refinement update");
  // corrections until the estimated error is below the tolerance, the
  // iterations stagnate or ir_iters are spent; the decision is taken on the
  // device (k_ir_decide), so the launches of the corrections that are not
  // needed return at entry and the host never waits
  for (int it = 0; it < P->ir_iters; ++it) {
    DCT_CUDA(dct::launch_residual(P, bp, bstride, xp, k, st), "residual");
    DCT_CUDA(dct::run_solve_f32(P, k, st), "solve launch");
    DCT_CUDA(dct::launch_ir_update(P, xp, k, 0, st), "refinement update");
    DCT_CUDA(dct::launch_ir_decide(P, it + 1, st), "refinement decision");
  }
  return DCT_OK;
}

}  // namespace

int dct_solve_permuted(dct_plan* P, const double* d_bp, int32_t b_batched,
                       int32_t k, double* d_xp, void* stream) {
  if (!P || !d_bp || !d_xp || k < 1 || k > P->max_rhs)
    return fail(DCT_ERR_ARG, "bad arguments");
  if (!P->factored) return fail(DCT_ERR_NOT_FACTORED, "solve before factorize");
  if (P->dtype == DCT_C128)
    return fail(DCT_ERR_ARG, "dct_solve_permuted takes float64 plans; use dct_solve");
  if (P->dtype == DCT_F32 && d_bp == d_xp)
    return fail(DCT_ERR_ARG, "float32 plans refine against the right-hand side: "
                             "d_bp must not alias d_xp");
  int rc = set_device(P->device);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t per = int64_t(P->sym.n) * k;
  const int64_t bstride = b_batched ? per : 0;
  if (P->dtype == DCT_F64) {
    if (d_bp != d_xp || !b_batched)
      DCT_CUDA(dct::launch_convert_any(d_bp, DCT_F64, bstride, per, P->nbatch,
                                       d_xp, DCT_F64, st),
               "rhs copy");
    DCT_CUDA(dct::run_solve_f64(P, d_xp, k, st), "solve launch");
    return DCT_OK;
  }
  return solve_refined(P, d_bp, bstride, k, d_xp, st);
}

namespace {
int solve_common(dct_plan* P, const void* d_b, int32_t io_dtype, int32_t b_batched,
                 int32_t k, void* d_x, void* stream, bool transposed);
}  // namespace

int dct_solve(dct_plan* P, const void* d_b, int32_t io_dtype, int32_t b_batched,
              int32_t k, void* d_x, void* stream) {
  return solve_common(P, d_b, io_dtype, b_batched, k, d_x, stream, false);
}

int dct_solve_transposed(dct_plan* P, const void* d_b, int32_t io_dtype, int32_t b_batched,
                         int32_t k, void* d_x, void* stream) {
  if (P && !P->lu) return dct_solve(P, d_b, io_dtype, b_batched, k, d_x, stream);
  return solve_common(P, d_b, io_dtype, b_batched, k, d_x, stream, true);
}

namespace {
int solve_common(dct_plan* P, const void* d_b, int32_t io_dtype, int32_t b_batched,
                 int32_t k, void* d_x, void* stream, bool transposed) {
  if (!P || !d_b || !d_x || k < 1 || k > P->max_rhs || !valid_dtype(io_dtype) ||
      ((io_dtype == DCT_C128) != (P->dtype == DCT_C128)))
    return fail(DCT_ERR_ARG, "bad arguments");
  if (!P->factored) return fail(DCT_ERR_NOT_FACTORED, "solve before factorize");
  int rc = set_device(P->device);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int n = P->sym.n;
  const int64_t per = int64_t(n) * k;
  const int64_t bstride = b_batched ? per : 0;
  if (P->dtype == DCT_C128) {
    DCT_CUDA(dct::launch_perm_in_any(d_b, DCT_C128, bstride, P->ds.perm, n, k,
                                     P->nbatch, P->bufA, DCT_C128, st),
             "permute rhs");
    DCT_CUDA(dct::run_solve_c128(P, static_cast<dct::cplx*>(P->bufA), k, st),
             "solve launch");
    DCT_CUDA(dct::launch_perm_out_any(P->bufA, DCT_C128, P->ds.perm, n, k,
                                      P->nbatch, d_x, DCT_C128, st),
             "permute solution");
    return DCT_OK;
  }
  if (P->dtype == DCT_F64) {
    DCT_CUDA(dct::launch_perm_in_any(d_b, io_dtype, bstride, P->ds.perm, n, k,
                                     P->nbatch, P->bufA, DCT_F64, st),
             "permute rhs");
    DCT_CUDA(dct::run_solve_f64(P, static_cast<double*>(P->bufA), k, st, transposed),
             "solve launch");
    DCT_CUDA(dct::launch_perm_out_any(P->bufA, DCT_F64, P->ds.perm, n, k,
                                      P->nbatch, d_x, io_dtype, st),
             "permute solution");
    return DCT_OK;
  }
  DCT_CUDA(dct::launch_perm_in_any(d_b, io_dtype, bstride, P->ds.perm, n, k,
                                   P->nbatch, P->b64, DCT_F64, st),
           "permute rhs");
  rc = solve_refined(P, P->b64, per, k, P->x64, st);
  if (rc) return rc;
  DCT_CUDA(dct::launch_perm_out_any(P->x64, DCT_F64, P->ds.perm, n, k, P->nbatch,
                                    d_x, io_dtype, st),
           "permute solution");
  return DCT_OK;
}
}  // namespace

int dct_plan_profile(dct_plan* P, int32_t enable, int32_t reset) {
  if (!P) return fail(DCT_ERR_ARG, "null plan");
  int rc = set_device(P->device);
  if (rc) return rc;
  DCT_CUDA(P->prof.collect(), "profile collect");
  if (reset) P->prof.reset();
  P->prof.on = enable != 0;
  return DCT_OK;
}

int dct_plan_profile_get(dct_plan* P, int32_t kind, double* ms, int64_t* launches,
                         double* flops, double* bytes) {
  if (!P || kind < 0 || kind >= dct::kNumKinds) return fail(DCT_ERR_ARG, "bad arguments");
  int rc = set_device(P->device);
  if (rc) return rc;
  DCT_CUDA(P->prof.collect(), "profile collect");
  if (ms) *ms = P->prof.ms[kind];
  if (launches) *launches = P->prof.n[kind];
  if (flops) *flops = P->prof.fl[kind];
  if (bytes) *bytes = P->prof.by[kind];
  return DCT_OK;
}

int dct_plan_profile_log(dct_plan* P, int64_t capacity, int32_t* kinds, double* ms,
                         int64_t* count) {
  if (!P || !count) return fail(DCT_ERR_ARG, "bad arguments");
  int rc = set_device(P->device);
  if (rc) return rc;
  DCT_CUDA(P->prof.collect(), "profile collect");
  const int64_t n = int64_t(P->prof.log_ms.size());
  *count = n;
  for (int64_t i = 0; i < n && i < capacity; ++i) {
    if (kinds) kinds[i] = P->prof.log_kind[i];
    if (ms) ms[i] = P->prof.log_ms[i];
  }
  return DCT_OK;
}

int dct_check_status(dct_plan* P, void* stream, int32_t* code, int32_t* where,
                     double* residual) {
  if (!P) return fail(DCT_ERR_ARG, "null plan");
  int rc = set_device(P->device);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int hs[16] = {0};
  unsigned long long rb[2] = {0, 0};
  DCT_CUDA(cudaMemcpyAsync(hs, P->status, sizeof(hs), cudaMemcpyDeviceToHost, st),
           "status read");
  DCT_CUDA(cudaMemcpyAsync(rb, P->resid_bits, sizeof(rb), cudaMemcpyDeviceToHost, st),
           "status read");
  DCT_CUDA(cudaStreamSynchronize(st), "stream synchronize");
  // the error words; the static-pivot count (status[4]) lives until the
  // next factorization
  DCT_CUDA(cudaMemsetAsync(P->status, 0, 4 * sizeof(int), st), "status reset");
  if (code) *code = hs[0];
  if (where) *where = hs[0] ? hs[1] : -1;
  if (residual) {
    double r, b;
    std::memcpy(&r, &rb[0], 8);
    std::memcpy(&b, &rb[1], 8);
    *residual = b > 0 ? r / b : 0.0;
  }
  return DCT_OK;
}

}  // extern "C"
