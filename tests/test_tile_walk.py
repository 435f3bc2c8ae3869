"""The tensor-core GEMM's tile walk (tc_gemm.cu decode_tile and the host's band
prefix counts), restated: row tiles in bands of 2,048 rows, each band column by
column, only the tiles that reach the lower part when C is triangular. Every
tile that holds a written element is visited exactly once, in full and lower
products, on single CTAs (128 x 256 tiles) and CTA pairs (256 x 256)."""
import pytest

TBN = 256
BAND_ROWS = 2048
MAX_BANDS = 64


def first_mt(nt, tile_m, lower, diag_off=0):
    if not lower:
        return 0
    num = nt * TBN - diag_off - (tile_m - 1)
    return 0 if num <= 0 else (num + tile_m - 1) // tile_m


def plan(M, N, tile_m, lower):
    tiles_m = (M + tile_m - 1) // tile_m
    tiles_n = (N + TBN - 1) // TBN
    band = max(BAND_ROWS // tile_m, (tiles_m + MAX_BANDS - 1) // MAX_BANDS)
    nbands = (tiles_m + band - 1) // band
    starts, total = [], 0
    for b in range(nbands):
        starts.append(total)
        r0, r1 = b * band, min(b * band + band, tiles_m)
        for nt in range(tiles_n):
            total += max(0, r1 - max(r0, first_mt(nt, tile_m, lower)))
    starts += [total] * (MAX_BANDS + 1 - nbands)
    return dict(tiles_m=tiles_m, tiles_n=tiles_n, band=band, starts=starts, total=total,
                tile_m=tile_m, lower=lower)


def decode(p, v):
    b = 0
    while (b + 1 < MAX_BANDS and p["starts"][b + 1] <= v
           and b + 1 < (p["tiles_m"] + p["band"] - 1) // p["band"]):
        b += 1
    v -= p["starts"][b]
    r0 = b * p["band"]
    r1 = min(r0 + p["band"], p["tiles_m"])
    h = r1 - r0
    full = p["tiles_n"]
    if p["lower"]:
        num = r0 * p["tile_m"] + p["tile_m"] - 1
        full = 0 if num < 0 else min(p["tiles_n"], num // TBN + 1)
    if v < full * h:
        return r0 + v % h, v // h
    v -= full * h
    for c in range(full, p["tiles_n"]):
        f = max(r0, first_mt(c, p["tile_m"], p["lower"]))
        cnt = max(0, r1 - f)
        if v < cnt or c == p["tiles_n"] - 1:
            return f + v, c
        v -= cnt
    return r0, p["tiles_n"] - 1


@pytest.mark.parametrize("tile_m", [128, 256])
@pytest.mark.parametrize("M,N,lower", [(300, 200, False), (2600, 2600, False), (5944, 47552, False),
                                       (4700, 4700, True), (46528, 46528, True), (1000, 77, False),
                                       (2048, 2048, True), (130, 5000, False)])
def test_every_written_tile_once(tile_m, M, N, lower):
    p = plan(M, N, tile_m, lower)
    seen = [decode(p, v) for v in range(p["total"])]
    assert len(set(seen)) == len(seen), "a tile visited twice"
    want = {(mt, nt) for nt in range(p["tiles_n"]) for mt in range(p["tiles_m"])
            if not lower or (mt + 1) * tile_m - 1 >= nt * TBN}
    assert set(seen) == want


def test_bands_are_walked_in_order():
    """Within a wave of 148 consecutive tiles the walk stays inside one or two
    bands: the rows a wave touches stay near 2,048."""
    p = plan(47552, 47552, 128, True)
    for w0 in range(0, p["total"] - 148, 148 * 37):
        rows = {decode(p, v)[0] // p["band"] for v in range(w0, w0 + 148)}
        assert len(rows) <= 2
