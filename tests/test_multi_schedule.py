"""The multi-spectrum kernel's tile schedule, restated on the CPU.

search_ws_multi (cs_search_ws.cuh, walk_begin / walk_block / walk_next)
walks rounds of grid x block consecutive tiles of the concatenated tile
list: in a full round CTA b takes the b-th block, the last partial round is
split evenly over the CTAs.  Every tile must be taken exactly once, by one
CTA, in increasing order per CTA (each role's spectrum cursor only moves
forward), with the work per CTA within one block of the mean (one tile in
the partial round), and at any time all CTAs inside one round: a window of
grid x block tiles of the list.
"""
import numpy as np
import pytest


def walk(b, G, ntiles, block):
    out = []
    base = 0
    while base < ntiles:
        rem = ntiles - base
        if rem >= G * block:
            g, end = base + b * block, base + b * block + block
        else:
            g, end = base + (b * rem) // G, base + ((b + 1) * rem) // G
        if g >= end:
            break
        out.extend(range(g, end))
        base += G * block
    return out


@pytest.mark.parametrize("ntiles,G,block", [(1, 148, 64), (147, 148, 64), (148, 148, 64),
                                            (9471, 148, 64), (9472, 148, 64), (9473, 148, 64),
                                            (8_821_000, 148, 64), (100_000, 148, 1),
                                            (100_000, 148, 256), (5, 3, 2)])
def test_walk_covers_every_tile_once(ntiles, G, block):
    seen = np.zeros(ntiles, dtype=np.int32)
    counts = []
    for b in range(G):
        tiles = walk(b, G, ntiles, block)
        assert all(x < y for x, y in zip(tiles, tiles[1:]))      # increasing per CTA
        assert not tiles or (0 <= tiles[0] and tiles[-1] < ntiles)
        np.add.at(seen, np.asarray(tiles, dtype=np.int64), 1)
        counts.append(len(tiles))
    assert np.all(seen == 1)
    full = ntiles // (G * block)
    # full rounds give every CTA the same count; the last round +-1 tile
    assert max(counts) - min(counts) <= 1
    assert min(counts) >= full * block


def test_walk_rounds_keep_ctas_together():
    """In round k every CTA's block lies in [k G block, (k+1) G block)."""
    G, block, ntiles = 148, 64, 1_000_000
    for b in (0, 73, 147):
        tiles = np.asarray(walk(b, G, ntiles, block))
        rounds = tiles // (G * block)
        assert np.all(np.diff(rounds) >= 0)
        for k in np.unique(rounds)[:-1]:
            assert np.sum(rounds == k) == block
