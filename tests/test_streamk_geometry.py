"""The FP64 stream-K schedule's piece geometry, restated from csrc/fp64_gemm.cu (sk_begin,
sk_owner, walk_next and the slot rule of the stream-K epilogue) and checked without a GPU: the
CTAs' shares cover every tile's K range exactly once, in order, the piece index and partial slot
each CTA computes for its segments are the ones the finishing warp looks up, and the slots stay
inside the workspace (two per CTA)."""
import pytest


def sk_begin(c, U, G):
    return c * U // G


def sk_owner(u, U, G):
    return ((u + 1) * G + U - 1) // U - 1


def segments(c, tiles, kblocks, G):
    """walk_next in stream-K mode: (tile, kb_begin, kb_end) of CTA c's share."""
    U = tiles * kblocks
    u, end = sk_begin(c, U, G), sk_begin(c + 1, U, G)
    while u < end:
        t = u // kblocks
        kb0 = u - t * kblocks
        kb1 = kblocks if kblocks - kb0 < end - u else kb0 + (end - u)
        yield t, kb0, kb1, u
        u += kb1 - kb0


@pytest.mark.parametrize("tiles", [1, 2, 3, 7, 64, 128, 130, 200, 1000])
@pytest.mark.parametrize("kblocks", [1, 2, 5, 32, 33, 100])
@pytest.mark.parametrize("sms", [1, 7, 148, 300])
def test_shares_cover_every_tile_once_in_k_order(tiles, kblocks, sms):
    U = tiles * kblocks
    G = min(sms, U)          # streamk_grid: no more CTAs than units
    for u in range(0, U, max(1, U // 997)):
        c = sk_owner(u, U, G)
        assert 0 <= c < G and sk_begin(c, U, G) <= u < sk_begin(c + 1, U, G)
    pieces = {}
    for c in range(G):
        for t, kb0, kb1, u in segments(c, tiles, kblocks, G):
            t0 = t * kblocks
            c0 = sk_owner(t0, U, G)
            n = sk_owner(t0 + kblocks - 1, U, G) - c0 + 1
            j = c - c0
            slot = 0 if t0 + kb0 == sk_begin(c, U, G) else 1
            assert 0 <= j < n and slot in (0, 1)
            # the finishing warp's lookup: piece 0 in slot 0 iff its CTA's share starts the tile,
            # every later piece in slot 0 of CTA c0 + j
            want_slot = (0 if sk_begin(c0, U, G) == t0 else 1) if j == 0 else 0
            assert slot == want_slot
            pieces.setdefault(t, []).append((kb0, kb1, j, n))
    assert sorted(pieces) == list(range(tiles))
    for t, segs in pieces.items():
        segs.sort()
        assert segs[0][0] == 0 and segs[-1][1] == kblocks
        assert all(a[1] == b[0] for a, b in zip(segs, segs[1:]))
        assert [s[2] for s in segs] == list(range(len(segs))) and all(s[3] == len(segs) for s in segs)
