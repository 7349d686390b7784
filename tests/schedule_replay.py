"""CPU replay of libdct's factor / solve launch schedules (test infrastructure).

The schedules are exported through the C ABI (`dct_symbolic_get_schedule`)
and every task is executed with numpy exactly as the corresponding kernel
does it (same tiles, same reads and writes, same buffers A/B).  Each launch
is replayed twice, in forward and in reversed task order, from the same
starting state: since the kernels of one launch run in any order on the GPU,
the two results must agree to round-off, which catches a task that reads
what another task of the same launch writes.  Every index is bounds-checked.
"""
from __future__ import annotations

import numpy as np

PANEL = 64
UTILE = 64
TCTILE = 128
IMG_K = 32           # columns of one K stage of the panel images (DCT_IMG_K)
(SMALL, LSCATTER, LEXTEND, LPANEL, LUPDATE, PINV, LINVINIT, LINVT, LINVX,
 FWDSMALL, FWDLINV, FWDBND, BWDSMALL, BWDGEMM, BWDLINV, FWDLINVTC, FWDBNDTC,
 BWDGEMMTC, BWDLINVTC) = range(19)


class Struct:
    def __init__(self, sym):
        for name in ("perm", "iperm", "sn_first", "front_n", "front_off",
                     "rows_ptr", "rows", "child_ptr", "child", "rel_ptr",
                     "rel", "amap_ptr", "amap_e", "amap_pos", "sn_parent"):
            setattr(self, name, sym.array(name))
        self.nsuper = len(self.front_n)
        self.front_total = int((self.front_n.astype(np.int64) ** 2).sum())

    def ns(self, s):
        return int(self.sn_first[s + 1] - self.sn_first[s])

    def front(self, buf, s):
        N = int(self.front_n[s])
        off = int(self.front_off[s])
        assert 0 <= off and off + N * N <= buf.size
        return buf[off:off + N * N].reshape(N, N, order="F")


def _chol_lower(D):
    w = D.shape[0]
    D = np.tril(D).copy()
    for k in range(w):
        piv = D[k, k]
        assert piv > 0, "non-positive pivot in replay"
        d = np.sqrt(piv)
        D[k + 1:, k] /= d
        D[k + 1:, k + 1:] -= np.tril(np.outer(D[k + 1:, k], D[k + 1:, k]))
        D[k, k] = d
    return D


def _factor_diag(S, F, s, c0, w, dinv):
    L = _chol_lower(F[c0:c0 + w, c0:c0 + w])
    blk = F[c0:c0 + w, c0:c0 + w]
    blk[np.tril(np.ones((w, w), bool))] = L[np.tril(np.ones((w, w), bool))]
    dinv[(s, c0 // PANEL)] = np.linalg.inv(L)


SMALL_F32 = 224      # largest front of the single-CTA float32 kernel


def img_origin(q, ns):
    """First row of panel q's split image (libdct's dct::img_origin)."""
    c0 = q * PANEL
    return c0 + (min(PANEL, ns - c0) & ~7)


def img_groups(q, ns, N):
    return (N - img_origin(q, ns) + 7) // 8 + 16


def img_index(G, hl, stage, g, k, r8):
    return (((hl * (PANEL // IMG_K) + stage) * G + g) * (8 * IMG_K) + (k >> 2) * 32 + r8 * 4
            + (k & 3))


def image_offsets(S):
    """{(s, q): first float of panel q's image} of the large fronts and the
    total size (the plan's layout, capi.cu)."""
    off, acc = {}, 0
    for s in range(S.nsuper):
        ns, N = S.ns(s), int(S.front_n[s])
        for q in range(-(-ns // PANEL)):
            off[(s, q)] = acc
            if N > SMALL_F32:
                acc += 2 * PANEL * 8 * img_groups(q, ns, N)
    return off, acc


# element (m, k) of a 128-row x IMG_K-column image chunk
_CHUNK_M, _CHUNK_K = np.meshgrid(np.arange(128), np.arange(IMG_K), indexing="ij")
_CHUNK_IDX = ((_CHUNK_M // 8) * (8 * IMG_K) + (_CHUNK_K // 4) * 32 + (_CHUNK_M % 8) * 4
              + _CHUNK_K % 4)


def _image_operand(dinv, s, ns, N, row0, ka, nst):
    """The (128, IMG_K nst) operand the tensor-core update streams from the
    panel images for tile rows row0 .. row0 + 127 and K stages of IMG_K columns
    from ka, with every chunk bounds-checked against its panel's image."""
    img = dinv[("img", 0)]
    parts = []
    for st in range(nst):
        kcol = ka + IMG_K * st
        q, h = kcol // PANEL, (kcol % PANEL) // IMG_K
        G, R0q = img_groups(q, ns, N), img_origin(q, ns)
        assert row0 >= R0q and (row0 - R0q) % 8 == 0
        off = dinv[("imgoff", s, q)]
        lo = off + img_index(G, 0, h, 0, 0, 0)
        start = off + img_index(G, 0, h, (row0 - R0q) // 8, 0, 0)
        assert lo <= start and start + 128 * IMG_K <= lo + G * 8 * IMG_K, \
            "chunk outside its image"
        parts.append(img[start + _CHUNK_IDX])
    return np.hstack(parts)


def update_range(p, ns, N, bpan):
    """K columns [ka, base) and last column cend of the trailing update after
    panel p when panels are grouped in blocks of bpan (libdct's
    dct::update_range): a block's last panel updates everything beyond the
    block with all of its panels, the others only the rest of their block."""
    npan = -(-ns // PANEL)
    blk = p // bpan
    last = p % bpan == bpan - 1 or p == npan - 1
    ka = (blk * bpan if last else p) * PANEL
    cend = N if last else min((blk + 1) * bpan * PANEL, ns)
    return ka, cend


def _task_factor(S, kind, tk, fronts, vals, arg, dinv, utile=UTILE, bpan=1):
    s, p, t0, t1 = (int(v) for v in tk)
    N = int(S.front_n[s])
    ns = S.ns(s)
    F = S.front(fronts, s)
    if kind == SMALL:
        assert N <= arg
        a0, a1 = S.amap_ptr[s], S.amap_ptr[s + 1]
        pos = S.amap_pos[a0:a1]
        assert pos.size == 0 or (pos.min() >= 0 and pos.max() < N * N)
        flat = np.zeros(N * N)
        flat[pos] = vals[S.amap_e[a0:a1]]
        G = flat.reshape(N, N, order="F")
        for ci in range(S.child_ptr[s], S.child_ptr[s + 1]):
            c = int(S.child[ci])
            nc, nsc = int(S.front_n[c]), S.ns(c)
            U = S.front(fronts, c)[nsc:, nsc:]
            rel = S.rel[S.rel_ptr[c]:S.rel_ptr[c + 1]]
            assert rel.size == nc - nsc and (rel.size == 0 or rel.max() < N)
            G[np.ix_(rel, rel)] += np.tril(U)
        for k in range(ns):
            piv = G[k, k]
            assert piv > 0, f"non-positive pivot at supernode {s}"
            d = np.sqrt(piv)
            G[k + 1:, k] /= d
            G[k + 1:, k + 1:] -= np.tril(np.outer(G[k + 1:, k], G[k + 1:, k]))
            G[k, k] = d
        F[:, :] = G
    elif kind == LSCATTER:
        a0, a1 = S.amap_ptr[s], S.amap_ptr[s + 1]
        flat = fronts[int(S.front_off[s]):int(S.front_off[s]) + N * N]
        flat[S.amap_pos[a0:a1]] = vals[S.amap_e[a0:a1]]
    elif kind == LEXTEND:
        c = t0
        nc, nsc = int(S.front_n[c]), S.ns(c)
        nbc = nc - nsc
        U = S.front(fronts, c)
        rel = S.rel[S.rel_ptr[c]:S.rel_ptr[c + 1]]
        for j in range(t1, min(t1 + 8, nbc)):
            i = np.arange(j, nbc)
            F[rel[i], rel[j]] += U[nsc + i, nsc + j]
    elif kind == LPANEL:
        c0 = p * PANEL
        w = min(PANEL, ns - c0)
        assert w > 0 and t0 >= 1
        Di = dinv[(s, p)]           # stored when the diagonal was factored
        r0 = c0 + w + (t0 - 1) * PANEL
        nr = min(PANEL, N - r0)
        assert nr > 0
        F[r0:r0 + nr, c0:c0 + w] = F[r0:r0 + nr, c0:c0 + w] @ Di.T
        if utile == TCTILE:
            # float32 plans: the split image of these rows (hi part; the
            # replay is exact, so lo stays zero)
            img, off = dinv[("img", 0)], dinv[("imgoff", s, p)]
            G, R0q = img_groups(p, ns, N), img_origin(p, ns)
            rr, cc = np.meshgrid(np.arange(nr), np.arange(w), indexing="ij")
            gr = r0 + rr - R0q
            assert gr.min() >= 0 and gr.max() < 8 * (G - 16)
            idx = off + img_index(G, 0, cc // IMG_K, gr >> 3, cc % IMG_K, gr & 7)
            assert idx.max() < off + PANEL * 8 * G
            img[idx] = F[r0:r0 + nr, c0:c0 + w]
    elif kind == LUPDATE:
        c0 = p * PANEL
        w = min(PANEL, ns - c0)
        base = c0 + w
        if t0 < 0:
            _factor_diag(S, F, s, c0, w, dinv)
            return
        ka, cend = update_range(p, ns, N, bpan)
        # float32 plans (128-row tensor-core tiles) start the tiles at
        # base & ~7, the 8-row grid of the split panel images, and update
        # only the rows and columns from base on (update_tc.cu)
        R0 = base & ~7 if utile == TCTILE else base
        ri, rj = R0 + t0 * utile, R0 + t1 * utile
        assert ri < N and rj < cend and t0 >= t1
        ri, rj = max(ri, base), max(rj, base)
        ni = min(R0 + (t0 + 1) * utile, N) - ri
        nj = min(R0 + (t1 + 1) * utile, cend) - rj
        assert ni > 0 and nj > 0
        upd = F[ri:ri + ni, ka:base] @ F[rj:rj + nj, ka:base].T
        if utile == TCTILE:
            # the tensor-core kernel's operands come from the panel images:
            # they must hold exactly these rows of L
            nst = (base - ka + IMG_K - 1) // IMG_K
            Ai = _image_operand(dinv, s, ns, N, R0 + t0 * utile, ka, nst)
            Bj = _image_operand(dinv, s, ns, N, R0 + t1 * utile, ka, nst)
            full = Ai @ Bj.T
            a0, b0 = ri - (R0 + t0 * utile), rj - (R0 + t1 * utile)
            img_upd = full[a0:a0 + ni, b0:b0 + nj]
            assert np.allclose(img_upd, upd, rtol=1e-12,
                               atol=1e-12 * max(1.0, np.abs(upd).max())), \
                "tensor-core update operands differ from the factor rows"
            upd = img_upd
            if t0 == t1:
                # diagonal tiles: the lower triangle only
                upd = np.where(np.arange(ri, ri + ni)[:, None]
                               >= np.arange(rj, rj + nj)[None, :], upd, 0.0)
        F[ri:ri + ni, rj:rj + nj] -= upd
        if t0 == 0 and t1 == 0 and base < ns:
            _factor_diag(S, F, s, base, min(PANEL, ns - base), dinv)
    elif kind == PINV:
        c0 = p * PANEL
        w = min(PANEL, ns - c0)
        dinv[(s, p)] = np.linalg.inv(np.tril(F[c0:c0 + w, c0:c0 + w]))
    elif kind == LINVINIT:
        c0 = p * PANEL
        w = min(PANEL, ns - c0)
        dinv[("linv", s)][c0:c0 + w, c0:c0 + w] = dinv[(s, p)]
    elif kind in (LINVT, LINVX):
        # supernode inverse by doubling: pair p of blocks of h = arg columns
        h = arg
        X, Tt = dinv[("linv", s)], dinv[("ltmp", s)]
        a0 = 2 * p * h
        d0 = a0 + h
        hd = min(h, ns - d0)
        r0, cc0 = t0 * PANEL, t1 * PANEL
        nr = min(PANEL, hd - r0)
        assert hd > 0 and nr > 0 and cc0 + PANEL <= h
        rs = slice(d0 + r0, d0 + r0 + nr)
        cs = slice(a0 + cc0, a0 + cc0 + PANEL)
        if kind == LINVT:
            Tt[rs, cs] = F[rs, a0 + cc0:a0 + h] @ X[a0 + cc0:a0 + h, cs]
        else:
            X[rs, cs] = -X[rs, d0:d0 + r0 + nr] @ Tt[d0:d0 + r0 + nr, cs]
    else:
        raise AssertionError(f"unexpected kind {kind}")


def replay_factor(sym, S, vals, dtype=0):
    """Returns (fronts, dinv) with dinv[(s, p)] the stored panel inverses."""
    fronts = np.zeros(S.front_total)
    dinv = {}
    # supernode inverses and their scratch start as NaN: a read of an entry
    # that no earlier launch wrote poisons the result
    # (float32 plans keep one for every supernode, float64 plans for those
    # wider than one panel)
    min_ns = 1 if dtype == 1 else PANEL + 1
    for s in range(S.nsuper):
        if S.ns(s) >= min_ns:
            dinv[("linv", s)] = np.full((S.ns(s), S.ns(s)), np.nan)
            dinv[("ltmp", s)] = np.full((S.ns(s), S.ns(s)), np.nan)
    utile = UTILE if dtype == 0 else 128
    bpan = 1 if dtype == 0 else 4
    if dtype == 1:
        off, total = image_offsets(S)
        dinv[("img", 0)] = np.zeros(total)
        for (s, q), o in off.items():
            dinv[("imgoff", s, q)] = o

    def snapshot(d):
        return {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}

    for which in (0, 3, 4):
        tasks, launches = sym.schedule(dtype, which)
        for kind, lv, first, count, arg in launches:
            chunk = tasks[first:first + count]
            snap, dsnap = fronts.copy(), snapshot(dinv)
            for tk in chunk:
                _task_factor(S, kind, tk, fronts, vals, arg, dinv, utile, bpan)
            fwd_result, fwd_dinv = fronts.copy(), snapshot(dinv)
            fronts[:], dinv = snap, dsnap
            for tk in chunk[::-1]:
                _task_factor(S, kind, tk, fronts, vals, arg, dinv, utile, bpan)
            scale = max(1.0, np.abs(fwd_result).max())
            assert np.abs(fronts - fwd_result).max() <= 1e-9 * scale, \
                f"launch kind {kind} level {lv}: result depends on task order"
            assert fwd_dinv.keys() == dinv.keys()
            for key, v in dinv.items():
                u = fwd_dinv[key]
                if not isinstance(v, np.ndarray):
                    assert u == v
                    continue
                assert np.array_equal(np.isnan(u), np.isnan(v))
                ok = ~np.isnan(u)
                assert np.abs(u[ok] - v[ok]).max(initial=0.0) <= 1e-9 * max(
                    1.0, np.abs(u[ok]).max(initial=0.0)), \
                    f"launch kind {kind}: {key} depends on task order"
    npanels = sum((S.ns(s) + PANEL - 1) // PANEL for s in range(S.nsuper))
    assert len([k for k in dinv if k[0] not in ("linv", "ltmp", "img", "imgoff")]) == npanels, \
        "a panel inverse was never stored"
    for s in range(S.nsuper):
        if S.ns(s) >= min_ns:
            X = dinv[("linv", s)]
            low = np.tril(np.ones_like(X, dtype=bool))
            assert not np.isnan(X[low]).any(), f"supernode {s}: inverse incomplete"
    return fronts, dinv


def _task_solve(S, kind, tk, fronts, A, B, dinv):
    s, p, t0, t1 = (int(v) for v in tk)
    N = int(S.front_n[s])
    ns = S.ns(s)
    first = int(S.sn_first[s])
    F = S.front(fronts, s)
    rows = S.rows[S.rows_ptr[s]:S.rows_ptr[s + 1]]
    assert rows.size == N
    if kind == FWDSMALL:
        assert ns <= PANEL and p == 0
        y = dinv[(s, 0)] @ A[first:first + ns]
        B[first:first + ns] = y
        A[rows[ns:]] -= F[ns:, :ns] @ y
    elif kind == BWDSMALL:
        assert ns <= PANEL and p == 0
        y = B[first:first + ns] - F[ns:, :ns].T @ A[rows[ns:]]
        A[first:first + ns] = dinv[(s, 0)].T @ y
    elif kind == FWDBND:
        r0 = ns + t0 * PANEL
        r1 = min(r0 + PANEL, N)
        assert ns < r0 + 1 <= r1
        A[rows[r0:r1]] -= F[r0:r1, :ns] @ B[first:first + ns]
    elif kind == BWDGEMM:
        c0 = p * PANEL
        w = min(PANEL, ns - c0)
        assert w > 0
        B[first + c0:first + c0 + w] -= F[ns:, c0:c0 + w].T @ A[rows[ns:]]
    elif kind == FWDLINV:
        assert ns > PANEL and p == 0
        X = dinv[("linv", s)]
        r0 = t0 * PANEL
        nr = min(PANEL, ns - r0)
        assert nr > 0
        B[first + r0:first + r0 + nr] = X[r0:r0 + nr, :r0 + nr] @ A[first:first + r0 + nr]
    elif kind == BWDLINV:
        assert ns > PANEL and p == 0
        X = dinv[("linv", s)]
        r0 = t0 * PANEL
        nr = min(PANEL, ns - r0)
        assert nr > 0
        A[first + r0:first + r0 + nr] = X[r0:ns, r0:r0 + nr].T @ B[first + r0:first + ns]
    elif kind in (FWDLINVTC, FWDBNDTC, BWDGEMMTC, BWDLINVTC):
        # tensor-core products: 128-row output tile t0, K range [p, t1),
        # accumulated (other tasks may add to the same rows)
        k0, k1, m0 = p, t1, t0 * TCTILE
        assert 0 <= k0 < k1
        if kind == FWDBNDTC:
            mr = min(TCTILE, N - ns - m0)
            assert mr > 0 and k1 <= ns
            A[rows[ns + m0:ns + m0 + mr]] -= F[ns + m0:ns + m0 + mr, k0:k1] @ B[first + k0:first + k1]
        elif kind == BWDGEMMTC:
            mr = min(TCTILE, ns - m0)
            assert mr > 0 and k1 <= N - ns
            B[first + m0:first + m0 + mr] -= (F[ns + k0:ns + k1, m0:m0 + mr].T
                                             @ A[rows[ns + k0:ns + k1]])
        else:
            X = dinv[("linv", s)]
            mr = min(TCTILE, ns - m0)
            assert mr > 0 and k1 <= ns
            m = np.arange(m0, m0 + mr)[:, None]
            k = np.arange(k0, k1)[None, :]
            if kind == FWDLINVTC:
                T = np.where(k <= m, X[m0:m0 + mr, k0:k1], 0.0)
                B[first + m0:first + m0 + mr] += T @ A[first + k0:first + k1]
            else:
                T = np.where(k >= m, X[k0:k1, m0:m0 + mr].T, 0.0)
                A[first + m0:first + m0 + mr] += T @ B[first + k0:first + k1]
    else:
        raise AssertionError(f"unexpected kind {kind}")


def replay_solve(sym, S, fronts, bp, dinv, dtype=0):
    """bp: permuted rhs (n, k).  Returns the permuted solution."""
    A = np.array(bp, dtype=float, copy=True)
    B = np.zeros_like(A)
    for which in (1, 2):
        if dtype == 1:
            # float32 plans clear the destination of the accumulating
            # tensor-core products before each pass
            (B if which == 1 else A)[:] = 0.0
        tasks, launches = sym.schedule(dtype, which)
        for kind, lv, first, count, arg in launches:
            chunk = tasks[first:first + count]
            sa, sb = A.copy(), B.copy()
            for tk in chunk:
                _task_solve(S, kind, tk, fronts, A, B, dinv)
            ra, rb = A.copy(), B.copy()
            A[:], B[:] = sa, sb
            for tk in chunk[::-1]:
                _task_solve(S, kind, tk, fronts, A, B, dinv)
            scale = max(1.0, np.abs(ra).max(), np.abs(rb).max())
            assert max(np.abs(A - ra).max(), np.abs(B - rb).max()) <= 1e-9 * scale, \
                f"solve launch kind {kind} level {lv}: depends on task order"
    return A
