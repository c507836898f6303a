"""Index mapping of the k-block packs, on the CPU. A restatement of
the plan-time tile choice (tccg_abi.cu: ``kblock_tiles``, ``kblock_quads``)
and of ``pack_kblock_quad`` (pack.cuh) -- 256 threads copy 4 consecutive u
of one (row, l) as one 16-byte chunk into a shared tile whose chunks are
rotated by l / 4, then each thread reads 4 consecutive l of one u back out
into K-major rows -- replayed with numpy on the layouts the GPU tests use:
every chunk lands inside the tile and is written once, every 16-byte copy
reads 4 source elements that are k, k + lo, k + 2 lo, k + 3 lo of the
operand, every slot the write-out reads was written, and the packed rows
equal the operand gathered through its offset tables (zeros past K). Likewise the
element-wise tiles (``pack_kblock`` and its division-free ``KbWalk``): every
(row, l, u) copied once into its padded slot inside the kernel's shared
tile, the run's column shortcut (including runs that wrap into the next
value of the higher modes and u of stride -1) reading the right element, and
each quad of the write-out inside one 32-element group. The kernels
themselves are checked on a B200 by test_pack_kblock.py."""
import numpy as np
import pytest

PACK_KB_ELEMS = 4096  # rows x k elements of one CTA's tile at most
THREADS = 256


def offsets(ext, stride):
    """Column-major offsets of every index of the modes (first mode fastest)."""
    out = np.zeros(int(np.prod(ext)) if len(ext) else 1, dtype=np.int64)
    idx = [0] * len(ext)
    off = 0
    for n in range(len(out)):
        out[n] = off
        for i in range(len(ext)):
            idx[i] += 1
            off += stride[i]
            if idx[i] < ext[i]:
                break
            off -= idx[i] * stride[i]
            idx[i] = 0
    return out


def kblock_tiles(kext, kstr):
    """(lo, run, rows, ext of u, step of u) or None, as chosen at plan time."""
    first = u = -1
    for i, e in enumerate(kext):
        if e <= 1:
            continue
        if first < 0:
            first = i
        if abs(kstr[i]) == 1:
            u = i
    if u < 0 or u == first or kext[u] < 8:
        return None
    lo = int(np.prod(kext[:u]))
    if lo > 128:
        return None
    run = min(kext[u], 1024 // lo)
    t = lo * run
    if run < 8 or t % 4:
        return None
    return lo, run, max(1, min(32, PACK_KB_ELEMS // t)), kext[u], 1 if kstr[u] > 0 else -1


def kblock_quads(kext, kstr, coff):
    """True when the k-block tiles may move 16-byte quads along u."""
    kb = kblock_tiles(kext, kstr)
    if kb is None:
        return False
    lo, run, _, ext, step = kb
    if lo % 4 or run % 4 or ext % 4 or step != 1:
        return False
    for k in range(len(coff)):
        if ((k // lo) % ext) % 4:
            continue
        if coff[k] % 4:
            return False
        for j in range(1, 4):
            if k + j * lo < len(coff) and coff[k + j * lo] != coff[k] + j:
                return False
    return True


def replay(rext, rstr, kext, kstr, kcover_multiple):
    """Runs the pack's two phases over every CTA of the operand; returns the
    packed rows and the (lo, run, rows) tile shape."""
    roff, coff = offsets(rext, rstr), offsets(kext, kstr)
    R, K = len(roff), len(coff)
    assert kblock_quads(kext, kstr, coff) and all(o % 4 == 0 for o in roff)
    lo, run, rows, ext, _ = kblock_tiles(kext, kstr)
    T, nch = lo * run, run // 4
    kcover = -(-K // kcover_multiple) * kcover_multiple
    src = np.random.default_rng(0).standard_normal(int(roff.max() + coff.max() + 1))
    out = np.full((R, kcover), np.nan)
    nq = PACK_KB_ELEMS // 4 // THREADS

    def chunk(r, l, c):  # raw position of chunk c of tile row (r, l)
        return (r * lo + l) * run + 4 * ((c + (l >> 2)) % nch)

    for kt in range(-(-kcover // T)):
        for rt in range(-(-R // rows)):
            k0, r0 = kt * T, rt * rows
            u0 = (kt * run) % ext
            assert u0 % 4 == 0
            tile = np.full(rows * T, np.nan)
            written = np.zeros(rows * T, dtype=int)
            for tid in range(THREADS):  # phase 1: 16-byte copies into the tile
                for i in range(nq):
                    f = tid + THREADS * i
                    if f >= rows * lo * nch:
                        break
                    c, rl = f % nch, f // nch
                    l, r = rl % lo, rl // lo
                    u = 4 * c
                    row, k = r0 + r, k0 + l + lo * u
                    d = chunk(r, l, c)
                    assert 0 <= d and d + 4 <= rows * T and d % 4 == 0
                    if row < R and k + 3 * lo < K:
                        base = roff[row] + (coff[k0 + l] + u if u0 + u < ext else coff[k])
                        assert base % 4 == 0  # 16-byte aligned source
                        for j in range(4):
                            assert base + j == roff[row] + coff[k + j * lo]
                        tile[d:d + 4] = src[base:base + 4]
                    else:
                        for j in range(4):
                            kj = k + lo * j
                            tile[d + j] = src[roff[row] + coff[kj]] if row < R and kj < K else 0.0
                    written[d:d + 4] += 1
            assert written.max() <= 1
            q = T // 4
            for tid in range(THREADS):  # phase 2: 4 consecutive l of one u per thread
                for f in range(tid, rows * q, THREADS):
                    r, kq = f // q, (f % q) * 4
                    row, k = r0 + r, k0 + kq
                    if row >= R or k >= kcover:
                        continue
                    l, u = kq % lo, kq // lo
                    for j in range(4):
                        pos = chunk(r, l + j, u >> 2) + (u & 3)
                        assert written[pos] == 1
                        out[row, k + j] = tile[pos]
    ref = np.zeros((R, kcover))
    ref[:, :K] = src[roff[:, None] + coff[None, :]]
    return out, ref, (lo, run, rows)


def _strides(labels, sizes):
    s, acc = {}, 1
    for label in labels:
        s[label] = acc
        acc *= sizes[label]
    return s


# (operand labels in memory order, extents, row modes, K modes in K order,
#  expected tile lo x run x rows)
CASES = {
    # configuration 4's B[k1, j1, k0, j0] at reduced extents: unit stride on
    # k1, the second K mode
    "cfg4_small": (["k1", "j1", "k0", "j0"], dict(j0=8, j1=40, k0=32, k1=32), ["j0", "j1"],
                   ["k0", "k1"], (32, 32, 4)),
    # runs of 64 over an extent of 100 wrap into the next k2
    "wrap": (["k1", "k0", "k2", "n"], dict(n=130, k0=16, k1=100, k2=2), ["n"],
             ["k0", "k1", "k2"], (16, 64, 4)),
    # unit stride on the third K mode
    "third": (["k2", "k0", "k1", "n"], dict(n=75, k0=4, k1=16, k2=12), ["n"],
              ["k0", "k1", "k2"], (64, 12, 5)),
    # short runs (12) and lo = 8, K tail inside the last tile
    "short_run": (["k1", "j1", "k0", "j0"], dict(j0=4, j1=3, k0=8, k1=12), ["j0", "j1"],
                  ["k0", "k1"], (8, 12, 32)),
    # lo = 12 (two K modes below u), few rows
    "lo12": (["k2", "n", "k1", "k0"], dict(n=5, k0=4, k1=3, k2=16), ["n"], ["k0", "k1", "k2"],
             (12, 16, 21)),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("kcover_multiple", [32, 64])  # BF16x3 rows / BF16 rows
def test_kblock_quad_mapping(name, kcover_multiple):
    labels, sizes, rows, ks, shape = CASES[name]
    st = _strides(labels, sizes)
    out, ref, got = replay([sizes[m] for m in rows], [st[m] for m in rows],
                           [sizes[k] for k in ks], [st[k] for k in ks], kcover_multiple)
    assert got == shape
    assert np.array_equal(out, ref)


def test_quads_refused_where_a_copy_would_straddle():
    # u's extent not a multiple of 4: the element-wise k-block tiles only
    kext, kstr = [16, 10], [10, 1]
    assert kblock_tiles(kext, kstr) is not None
    assert not kblock_quads(kext, kstr, offsets(kext, kstr))
    # u on the first K mode is the streaming pass, not a k-block tile
    assert kblock_tiles([16, 8], [1, 16]) is None


def kb_walk(f, step, lo, run):
    """KbWalk: (r, l, u) of element f = r lo run + l run + u, then steps of
    ``step`` elements without divisions."""
    T = lo * run
    r = f // T
    l = (f - r * T) // run
    u = f - r * T - l * run
    dr = step // T
    dl = (step - dr * T) // run
    du = step - dr * T - dl * run
    while True:
        yield r, l, u
        u += du
        l += dl
        if u >= run:
            u -= run
            l += 1
        if l >= lo:
            l -= lo
            r += 1
        r += dr


def replay_elementwise(rext, rstr, kext, kstr, kcover_multiple):
    """``pack_kblock``: one 4-byte copy per (r, l, u) into the padded slot of
    k_local = l + lo u, then quads of k_local read back out."""
    roff, coff = offsets(rext, rstr), offsets(kext, kstr)
    R, K = len(roff), len(coff)
    lo, run, rows, ext, step = kblock_tiles(kext, kstr)
    T, TP = lo * run, lo * run + lo * run // 32
    assert rows * TP <= 128 * 33  # the kernel's shared tile
    kcover = -(-K // kcover_multiple) * kcover_multiple
    # negative strides give negative offsets: index from the lowest element
    base0 = -int(roff.min() + coff.min())
    src = np.random.default_rng(1).standard_normal(int(roff.max() + coff.max()) + base0 + 1)
    out = np.full((R, kcover), np.nan)
    for kt in range(-(-kcover // T)):
        for rt in range(-(-R // rows)):
            k0, r0 = kt * T, rt * rows
            u0 = (kt * run) % ext
            tile = np.full(128 * 33, np.nan)
            written = np.zeros(128 * 33, dtype=int)
            for tid in range(THREADS):
                w = kb_walk(tid, THREADS, lo, run)
                for i in range(PACK_KB_ELEMS // THREADS):
                    r, l, u = next(w)
                    assert (r * lo + l) * run + u == tid + THREADS * i
                    if r >= rows:
                        continue
                    row, k = r0 + r, k0 + l + lo * u
                    kl = l + lo * u
                    slot = r * TP + kl + kl // 32
                    if k >= K or row >= R:
                        tile[slot] = 0.0
                    else:
                        co = coff[k0 + l] + step * u if u0 + u < ext else coff[k]
                        assert co == coff[k]  # the run's shortcut reads the right element
                        tile[slot] = src[base0 + roff[row] + co]
                    written[slot] += 1
            assert written.max() <= 1
            q = T // 4
            for f in range(rows * q):
                r, kq = f // q, (f % q) * 4
                row, k = r0 + r, k0 + kq
                if row >= R or k >= kcover:
                    continue
                base = r * TP + kq + kq // 32
                assert (kq + 3) // 32 == kq // 32  # a quad stays inside one 32-group
                assert written[base:base + 4].tolist() == [1, 1, 1, 1]
                out[row, k:k + 4] = tile[base:base + 4]
    ref = np.zeros((R, kcover))
    ref[:, :K] = src[base0 + roff[:, None] + coff[None, :]]
    return out, ref


# (row extents, row strides, K extents in K order, K strides): u = the K
# mode of stride +-1 after the first
ELEMENTWISE = {
    "u_extent_10": ([37], [10 * 16 * 3], [16, 10, 3], [10, 1, 160]),
    "wrap": ([5], [3200], [16, 100, 2], [100, 1, 1600]),
    "negative_step": ([9], [2000], [6, 24], [24, -1]),
    "cfg4_small": ([8, 40], [32 * 40 * 32, 32], [32, 32], [32 * 40, 1]),
}


@pytest.mark.parametrize("name", sorted(ELEMENTWISE))
def test_kblock_elementwise_mapping(name):
    rext, rstr, kext, kstr = ELEMENTWISE[name]
    out, ref = replay_elementwise(rext, rstr, kext, kstr, 32)
    assert np.array_equal(out, ref)
