"""Index walk of the streaming K-major pack, on the CPU. A restatement of
``pack_kstream`` (pack.cuh) -- quad q = blk * 4 * 256 + i * 256 + tid is
(row, k-quad) = divmod(q, Kcover / 4), stepped without divisions -- and of
its grid size (tccg_abi.cu, ``pack_geometry``: cdiv(Rcover * Kcover / 4,
1024) CTAs), replayed for row widths below, at and above 256 quads,
including widths that do not divide 256: every (row, quad) of the packed
operand is visited exactly once, the step never leaves [0, Kcover / 4), and
the read and write phases visit the same quads. Also ``k_quads``, the
plan-time test that every quad of k is 4 consecutive, 16-byte-aligned source
elements. The kernel itself is checked on a B200 by the GPU parity tests."""
import pytest

THREADS, QUADS_PER_THREAD = 256, 4


def cdiv(a, b):
    return -(-a // b)


def walk(blk, tid, qr):
    """The (row, k-quad) sequence one thread visits."""
    q0 = blk * QUADS_PER_THREAD * THREADS + tid
    row0, drow = q0 // qr, THREADS // qr
    kq0, dkq = q0 - row0 * qr, THREADS - drow * qr
    row, kq, out = row0, kq0, []
    for _ in range(QUADS_PER_THREAD):
        assert 0 <= kq < qr
        out.append((row, kq))
        kq += dkq
        row += drow
        if kq >= qr:
            kq -= qr
            row += 1
    return out


def k_quads(coff):
    if len(coff) < 4:
        return False
    for k in range(0, len(coff) - 3, 4):
        if coff[k] % 4:
            return False
        if any(coff[k + j] != coff[k] + j for j in range(1, 4)):
            return False
    return True


@pytest.mark.parametrize("rcover,kcover", [
    (1, 32), (7, 96), (37, 160), (100, 1024), (33, 1056), (3, 4096), (130, 64), (5, 8192)])
def test_every_quad_once(rcover, kcover):
    qr = kcover // 4
    tiles = cdiv(rcover * qr, THREADS * QUADS_PER_THREAD)
    seen = {}
    for blk in range(tiles):
        for tid in range(THREADS):
            read = walk(blk, tid, qr)
            # the write phase restarts from (row0, kq0) and takes the same steps
            assert read == walk(blk, tid, qr)
            for i, (row, kq) in enumerate(read):
                assert row * qr + kq == blk * QUADS_PER_THREAD * THREADS + i * THREADS + tid
                if row < rcover:
                    seen[(row, kq)] = seen.get((row, kq), 0) + 1
    assert len(seen) == rcover * qr and set(seen.values()) == {1}


def test_k_quads():
    # unit stride on the first K mode, extent a multiple of 4: eligible
    assert k_quads([k + 64 * b for b in range(3) for k in range(16)])
    # a K mode of extent 6 leaves quads straddling two values of the next mode
    assert not k_quads([k + 64 * b for b in range(4) for k in range(6)])
    # a quad that does not start 16-byte aligned
    assert not k_quads([1 + k for k in range(8)])
    assert not k_quads([0, 1, 2])
