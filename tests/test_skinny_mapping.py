"""CPU replay of the skinny kernel's index arithmetic
(tccg_b200/csrc/skinny_gett.cuh): the jobs (block x pass x k slice) and a
persistent CTA's walk over them, the block boxes over the W positions, the
three P load walks and both Q load walks of a k chunk, the epilogue's row
staging, and the three C store walks with their stepping of positions and
rows. Each element is touched exactly once, and every store instruction of a
whole run covers 32 consecutive C addresses.
"""
import itertools

import pytest

BW, KC, LDP, SUB, THREADS = 256, 32, 260, 32, 256  # positions per block = threads
WG, SG = BW // 4, 4  # a thread owns 4 positions of one of 4 row groups
P_X, P_Y, P_K = 0, 1, 2
C_XS, C_XY, C_SX = 0, 1, 2


def pos(p_walk, tx, ty, xl, yl):
    return yl + ty * xl if p_walk == P_Y else xl + tx * yl


def box(p_walk, tx, ty, bxn, ex, ey, b):
    """skinny_box: {position: (x, y)} of block b (valid positions only)."""
    ix, iy = b % bxn, b // bxn
    out = {}
    for w in range(BW):
        if p_walk == P_Y:
            yl, xl = w % ty, w // ty
        else:
            xl, yl = w % tx, w // tx
        x, y = ix * tx + xl, iy * ty + yl
        if w < tx * ty and x < ex and y < ey:
            out[w] = (x, y)
    return out


@pytest.mark.parametrize("p_walk", [P_X, P_Y, P_K])
@pytest.mark.parametrize("ex,ey,tx,ty", [(19, 262, 19, 13), (2627, 3, 256, 1), (10, 250, 10, 25),
                                         (300, 300, 16, 16), (7, 5, 7, 5), (1, 40, 1, 40)])
def test_boxes_cover_each_position_once(p_walk, ex, ey, tx, ty):
    bxn = -(-ex // tx)
    nblk = bxn * -(-ey // ty)
    seen = {}
    for b in range(nblk):
        for w, xy in box(p_walk, tx, ty, bxn, ex, ey, b).items():
            assert xy not in seen
            seen[xy] = (b, w)
            xl, yl = xy[0] - (b % bxn) * tx, xy[1] - (b // bxn) * ty
            assert pos(p_walk, tx, ty, xl, yl) == w  # the store walks' numbering
    assert len(seen) == ex * ey


def p_loads(p_walk, kr_log2, kc, valid):
    """skinny_load, P part: (k, w) of every copy or zero fill, per thread."""
    out = []
    for tid in range(THREADS):
        if p_walk == P_K:
            kl = tid & ((1 << kr_log2) - 1)
            if kl < kc:
                w = tid >> kr_log2
                while w < BW:
                    out.append((kl, w))
                    w += THREADS >> kr_log2
        else:
            for k in range(kc):
                out.append((k, tid))
    return out


def p_vec_loads(kc):
    """skinny_issue, 16-byte copies: thread tid takes positions 4 (tid % WG)
    .. + 3 at k = tid / WG, tid / WG + SG, ..."""
    out = []
    for tid in range(THREADS):
        g = 4 * (tid % WG)
        k = tid // WG
        while k < kc:
            out += [(k, g + e) for e in range(4)]
            k += SG
    return out


@pytest.mark.parametrize("kc", [1, 3, 4, 17, 32])
def test_p_vector_loads_each_element_once(kc):
    got = p_vec_loads(kc)
    assert sorted(got) == [(k, w) for k in range(kc) for w in range(BW)]
    # a warp's threads share k (the shuffled k offset comes from one lane)
    for w0 in range(0, THREADS, 32):
        assert len({tid // WG for tid in range(w0, w0 + 32)}) == 1


@pytest.mark.parametrize("p_walk", [P_X, P_Y, P_K])
@pytest.mark.parametrize("K", [1, 3, 8, 13, 20, 32, 45, 100])
def test_p_chunk_loads_each_element_once(p_walk, K):
    kr_log2 = 0
    while (1 << kr_log2) < min(K, KC):
        kr_log2 += 1
    for c in range(-(-K // KC)):
        kc = min(KC, K - c * KC)
        got = p_loads(p_walk, kr_log2, kc, None)
        assert sorted(got) == [(k, w) for k in range(kc) for w in range(BW)]
        # lanes of a warp: along k (one 32-lane run of a position's k) or
        # along consecutive positions
        if p_walk == P_K and kc >= 8:
            lanes = [(tid & ((1 << kr_log2) - 1), tid >> kr_log2) for tid in range(32)]
            assert [k for k, _ in lanes[: 1 << kr_log2]] == list(range(1 << kr_log2))


QLD = 52


def q_loads(q_kfast, sp, kc):
    out = []
    for tid in range(THREADS):
        if q_kfast:
            lane = tid & 31
            if lane < kc:
                out += [(lane, r) for r in range(tid >> 5, sp, THREADS // 32)]
        else:
            r, k = tid % sp, tid // sp
            while k < kc:
                out.append((k, r))
                r += THREADS % sp
                k += THREADS // sp
                if r >= sp:
                    r -= sp
                    k += 1
    return out


@pytest.mark.parametrize("q_kfast", [0, 1])
@pytest.mark.parametrize("sp", [16, 32, 48])
@pytest.mark.parametrize("kc", [1, 7, 20, 32])
def test_q_chunk_loads_each_element_once(q_kfast, sp, kc):
    got = q_loads(q_kfast, sp, kc)
    assert sorted(got) == [(k, r) for k in range(kc) for r in range(sp)]
    assert all(k * QLD + r < KC * QLD for k, r in got)  # inside one Q stage


def jobs(nblk, npass, ksplit, nchunks, cps):
    """skinny_job over J in [0, nblk npass ksplit): (b, p, z, c0, c1)."""
    out = []
    for J in range(nblk * npass * ksplit):
        z = J % ksplit
        r = J // ksplit
        p, b = r % npass, r // npass
        c0 = z * cps
        out.append((b, p, z, c0, min(c0 + cps, nchunks)))
    return out


@pytest.mark.parametrize("nblk,npass,ksplit,nchunks", [(7, 1, 1, 1), (3, 5, 1, 1), (2, 1, 16, 77),
                                                       (18, 1, 16, 3075), (5, 4, 1, 40), (1, 1, 3, 3)])
def test_jobs_cover_blocks_passes_and_chunks(nblk, npass, ksplit, nchunks):
    cps = -(-nchunks // ksplit)
    js = jobs(nblk, npass, ksplit, nchunks, cps)
    seen = {}
    for b, p, z, c0, c1 in js:
        assert c0 < c1  # no empty slice (the host picks ksplit = ceil(nchunks / cps))
        for c in range(c0, c1):
            assert (b, p, c) not in seen
            seen[(b, p, c)] = z
    assert len(seen) == nblk * npass * nchunks
    # the passes of a block are neighbouring jobs (one slice): their P chunks
    # are read by CTAs that run at the same time
    if ksplit == 1:
        assert [(b, p) for b, p, *_ in js] == [(b, p) for b in range(nblk) for p in range(npass)]


@pytest.mark.parametrize("njobs,grid", [(1, 296), (296, 296), (1000, 296), (20198, 296), (5, 2)])
def test_persistent_steps(njobs, grid):
    """skinny_loop: CTA j0 takes jobs j0, j0 + grid, ...; its job slot
    alternates per job and its stage per step (chunk), so the next step's
    copies never land in the stage or slot the current step reads."""
    chunks = lambda J: 1 + (J * 7) % 3
    taken = []
    for cta in range(min(grid, njobs)):
        jg, slot, st, steps = cta, 0, 0, []
        c, c1 = 0, chunks(jg)
        while True:
            last = c + 1 >= c1
            jn = jg + grid if last else jg
            has_next = jn < njobs
            steps.append((jg, c, st, slot))
            taken.append((jg, c))
            if not has_next:
                break
            nslot = slot ^ 1 if last else slot
            assert (st ^ 1) != st and (not last or nslot != slot)
            if last:
                slot, jg, c, c1 = nslot, jn, 0, chunks(jn)
            else:
                c += 1
            st ^= 1
        for (j1, _, s1, l1), (j2, _, s2, l2) in zip(steps, steps[1:]):
            assert s1 != s2 and (l1 == l2) == (j1 == j2)
    assert sorted(taken) == sorted((J, c) for J in range(njobs) for c in range(chunks(J)))


def stage_rows(rs, S, p):
    """skinny_finish of pass p: thread row (sg, i) -> staged (s0, r, stored)."""
    sp = 4 * rs
    out = {}
    for h in range(0, sp, SUB):
        s0 = p * sp + h
        if s0 >= S:
            break
        ns = min(sp - h, SUB, S - s0)
        for sg in range(4):
            for i in range(rs):
                r = sg * rs + i - h
                if 0 <= r < SUB:
                    assert (sg, i) not in out
                    out[(sg, i)] = (s0, r, r < ns, h + r)  # cs index within the pass
    return out


@pytest.mark.parametrize("rs,S,npass", [(4, 1, 1), (4, 16, 1), (8, 20, 1), (12, 40, 1), (12, 48, 1),
                                        (8, 49, 2), (8, 64, 2), (8, 150, 5), (8, 256, 8),
                                        (8, 65, 3)])
def test_epilogue_stages_every_row_once(rs, S, npass):
    sp = 4 * rs
    stored = []
    for p in range(npass):
        for (s0, r, ok, ci) in stage_rows(rs, S, p).values():
            if ok:
                stored.append(s0 + r)
                assert ci < sp and p * sp + ci == s0 + r  # the slot's row offsets
    assert sorted(stored) == list(range(S))


def plane(L0, L1, w0, wi, wj, r0, ri, rj, warp, out):
    """skinny_plane: the (w, r) of every lane and step, stepped incrementally."""
    total, di, dj = L0 * L1, 32 % L0, 32 // L0
    dw, dr = wi * di + wj * dj, ri * di + rj * dj
    cwc, crc = wj - wi * L0, rj - ri * L0
    for lane in range(32):
        i, j = lane % L0, lane // L0
        w, r = w0 + wi * i + wj * j, r0 + ri * i + rj * j
        f, step = lane, 0
        while f < total:
            fi, fj = f % L0, f // L0
            assert (w, r) == (w0 + wi * fi + wj * fj, r0 + ri * fi + rj * fj)
            out.append((warp, (w, r), step, lane))
            i += di
            w += dw
            r += dr
            if i >= L0:
                i -= L0
                w += cwc
                r += crc
            f += 32
            step += 1


def xparts(n, tx, nw):
    """skinny_xparts: pieces of the x range per plane."""
    if n >= 2 * nw:
        return 1
    return min(-(-2 * nw // n), -(-tx // 32))


def store_walk(c_walk, p_walk, tx, ty, s_run, s0, ns, NW=THREADS // 32):
    """skinny_store: [(warp plane, (w, r), step, lane)] of one staged step."""
    out = []
    py = p_walk == P_Y
    xs = ty if py else 1
    for warp in range(NW):
        if c_walk == C_XS:
            parts = xparts(ty, tx, NW)
            xp = -(-tx // parts)
            for job in range(warp, ty * parts, NW):
                yl, x0 = job // parts, (job % parts) * xp
                xn = min(xp, tx - x0)
                if xn > 0:
                    plane(xn, ns, (yl if py else tx * yl) + x0 * xs, xs, 0, 0, 0, 1, (warp, job), out)
        elif c_walk == C_XY:
            for r in range(warp, ns, NW):
                plane(tx, ty, 0, xs, 1 if py else tx, r, 0, 0, (warp, r), out)
        else:
            e0 = s_run
            first = (s0 // e0) * e0
            nruns = (s0 + ns - first + e0 - 1) // e0
            parts = xparts(nruns * ty, tx, NW)
            xp = -(-tx // parts)
            for job in range(warp, nruns * ty * parts, NW):
                part, rj = job % parts, job // parts
                run, yl = rj % nruns, rj // nruns
                rs_ = first + run * e0
                ra, rb = max(rs_, s0), min(rs_ + e0, s0 + ns)
                x0 = part * xp
                xn = min(xp, tx - x0)
                if rb <= ra or xn <= 0:
                    continue
                plane(rb - ra, xn, (yl if py else tx * yl) + x0 * xs, 0, xs, ra - s0, 1, 0,
                      (warp, job), out)
    return out


GEOMS = [(19, 13), (10, 25), (16, 16), (256, 1), (3, 5), (1, 1)]


@pytest.mark.parametrize("c_walk", [C_XS, C_XY, C_SX])
@pytest.mark.parametrize("p_walk", [P_X, P_Y])
@pytest.mark.parametrize("tx,ty", GEOMS)
@pytest.mark.parametrize("s0,ns,s_run", [(0, 32, 10), (32, 8, 10), (0, 20, 8), (64, 32, 19),
                                         (0, 1, 1), (96, 22, 64)])
@pytest.mark.parametrize("nw", [8, 4])
def test_store_walk_covers_each_element_once(c_walk, p_walk, tx, ty, s0, ns, s_run, nw):
    st = store_walk(c_walk, p_walk, tx, ty, s_run, s0, ns, nw)
    got = sorted(e for _, e, _, _ in st)
    assert got == sorted((pos(p_walk, tx, ty, xl, yl), r)
                         for xl in range(tx) for yl in range(ty) for r in range(ns))


def test_flat_boxes_give_every_warp_work():
    """A box of 256 x 1 positions (one y): the (x, s) planes and the runs of
    C's stride-one S mode are split along x so that all 8 warps store (before
    the split 1 of 8, resp. 4 of 8 warps had work and the rest waited at the
    barrier after the stores)."""
    for c_walk, ns, s_run in ((C_XS, 32, 0), (C_SX, 32, 10)):
        st = store_walk(c_walk, P_X, 256, 1, s_run, 0, ns)
        per_warp = {}
        for (warp, _), _, _, _ in st:
            per_warp[warp] = per_warp.get(warp, 0) + 1
        assert len(per_warp) == 8 and max(per_warp.values()) <= 2 * min(per_warp.values())


def test_store_instructions_are_contiguous():
    """C(x, y, s) = x + 19 s + 760 y (item-69-like: X of 19, then S of 40):
    the (x, s) walk's full steps write 32 consecutive addresses; the (s, x)
    walk with C(x, s) = s + 10 x (a run of 10 rows, then X) likewise."""
    tx, ty = 19, 13
    st = store_walk(C_XS, P_Y, tx, ty, 0, 0, 32)
    inv = {pos(P_Y, tx, ty, xl, yl): (xl, yl) for xl in range(tx) for yl in range(ty)}
    steps = {}
    for warp, (w, r), step, lane in st:
        xl, yl = inv[w]
        steps.setdefault((warp, step), []).append(xl + 19 * r + 760 * yl)
    full = [sorted(a) for a in steps.values() if len(a) == 32]
    assert full and all(a == list(range(a[0], a[0] + 32)) for a in full)
    st = store_walk(C_SX, P_X, 256, 1, 10, 0, 30)
    steps = {}
    for warp, (w, r), step, lane in st:
        steps.setdefault((warp, step), []).append(r + 10 * w)
    full = [sorted(a) for a in steps.values() if len(a) == 32]
    assert full and all(a == list(range(a[0], a[0] + 32)) for a in full)


@pytest.mark.parametrize("p_walk", [P_X, P_Y])
@pytest.mark.parametrize("tx,ty,xn", [(37, 6, 37), (256, 1, 256), (256, 1, 44), (19, 13, 7), (4, 64, 4)])
@pytest.mark.parametrize("e0,ns", [(10, 30), (8, 32), (10, 20), (3, 30), (32, 32)])
@pytest.mark.parametrize("nt", [256, 128])
def test_run_ranges_copy_each_element_once(p_walk, tx, ty, xn, e0, ns, nt):
    """skinny_copy_runs: range (u, yl) element f = x e0 + o reads staged row
    u e0 + o of position (x, yl) at (u e0 + o) LDP + pos and writes C range
    offset f; (x, o) and the staging index step by fs with one carry --
    every (row, position) with x < xn copied once, to its own address."""
    nw = nt // 32
    n, nr = xn * e0, (ns // e0) * ty
    per_warp = nr >= nw
    wx = ty if p_walk == P_Y else 1
    seen = {}
    for tid in range(nt):
        g0, gs = (tid >> 5, nw) if per_warp else (0, 1)
        f0, fs = (tid & 31, 32) if per_warp else (tid, nt)
        dx, dox = fs // e0, fs % e0
        x0, o0 = f0 // e0, f0 % e0
        dsi, csi = dox * LDP + dx * wx, wx - e0 * LDP
        for g in range(g0, nr, gs):
            u, yl = g // ty, g % ty
            wy = yl if p_walk == P_Y else tx * yl
            o, si = o0, (u * e0 + o0) * LDP + wy + x0 * wx
            for f in range(f0, n, fs):
                x = f // e0
                assert o == f % e0
                assert si == (u * e0 + o) * LDP + pos(p_walk, tx, ty, x, yl)
                assert (u, yl, f) not in seen
                seen[(u, yl, f)] = si
                o += dox
                si += dsi
                if o >= e0:
                    o -= e0
                    si += csi
    assert len(seen) == nr * n
    assert len(set(seen.values())) == len(seen)


def test_partial_slices_round_trip():
    """k-split: the job of slice z, block b, pass p writes row r, position w
    at (((z nblk + b) npass + p) SP + r) BW + w; the reduction CTA of (b, p)
    (index b npass + p) reads slice z at (b npass + p) SP BW + r BW + w +
    z slice -- the same element, for every (z, b, p, r, w)."""
    for nblk, npass, sp, splits in itertools.product((1, 3, 7), (1, 2, 5), (16, 32), (2, 5)):
        slice_ = nblk * npass * sp * BW
        for z, b, p, r in itertools.product(range(splits), range(nblk), range(npass), range(sp)):
            w = (z * 7 + r) % BW
            wr = (((z * nblk + b) * npass + p) * sp + r) * BW + w
            cta = b * npass + p
            assert (cta // npass, cta % npass) == (b, p)
            rd = cta * sp * BW + w + r * BW + z * slice_
            assert wr == rd
