"""Host-side plans of the uneven-batch launch (sigpde_b200.torch.ragged), without a GPU.

plan(): the rows per lane of every pair (the vectorised rule equals the scalar
rows_per_lane), its bands, its boundary-row offsets and the work order (pairs
longest first, each pair's bands consecutive and in order).
tc_plan(): the tensor-core plan the GEMM and the wavefront read: operand-image
rows aligned to 8 (bulk copies of whole 8-row groups), every pair's increment
block covered by exactly one tile per element, offsets inside the block buffer,
the largest pairs first."""
import numpy as np
import pytest

rg = pytest.importorskip("sigpde_b200.torch.ragged")


def _batch(seed, npairs, lmax=700):
    rng = np.random.default_rng(seed)
    lx = rng.integers(2, lmax, npairs)
    ly = rng.integers(2, lmax, npairs)
    od = rng.integers(0, 5, npairs)
    return lx, ly, od


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("dim,tsize,staged", [(3, 8, True), (32, 8, True), (32, 4, True), (17, 8, False)])
def test_plan_rows_bands_and_order(seed, dim, tsize, staged):
    lx, ly, od = _batch(seed, 60)
    pl = rg.plan(lx, ly, od, dim, tsize, staged=staged)
    n = (np.minimum(lx, ly) - 1) << od
    m = (np.maximum(lx, ly) - 1) << od
    for b in range(len(lx)):
        assert pl["rows"][b] == rg.rows_per_lane(int(n[b]), dim, int(od[b]), tsize, staged)
    R = pl["rows"]
    assert set(np.unique(R)) <= {2, 4, 8, 16}
    assert np.all(pl["bands"] == (n + 32 * R - 1) // (32 * R))
    assert np.all(32 * R * pl["bands"] >= n) and np.all(32 * R * (pl["bands"] - 1) < n)
    sizes = (pl["bands"] - 1) * (m + 1)
    assert pl["bnd_elems"] == sizes.sum()
    assert np.all(pl["bnd_off"] == np.concatenate([[0], np.cumsum(sizes)[:-1]]))
    # work items: each pair's bands consecutive and in order, pairs by decreasing cells (stable)
    ip, ib = pl["item_pair"], pl["item_band"]
    assert len(ip) == len(ib) == pl["bands"].sum()
    starts = np.nonzero(ib == 0)[0]
    assert list(ip[starts]) == list(np.argsort(-(n * m).astype(np.float64), kind="stable"))
    for s, b in zip(starts, ip[starts]):
        k = int(pl["bands"][b])
        assert np.all(ip[s:s + k] == b) and list(ib[s:s + k]) == list(range(k))


@pytest.mark.parametrize("seed", range(3))
@pytest.mark.parametrize("tile_n", [128, 256])
def test_tc_plan_tiles_cover_every_block_once(seed, tile_n):
    lx, ly, _ = _batch(100 + seed, 25, lmax=400)
    tp = rg.tc_plan(lx, ly, tile_n=tile_n)
    rows = np.minimum(lx, ly) - 1
    cols = np.maximum(lx, ly) - 1
    r8, c8 = (rows + 7) // 8 * 8, (cols + 7) // 8 * 8
    ld = (rows + 3) // 4 * 4
    assert np.all(tp["a_row0"] % 8 == 0) and np.all(tp["b_row0"] % 8 == 0)
    assert np.all(np.diff(tp["a_row0"]) == r8[:-1]) and np.all(np.diff(tp["b_row0"]) == c8[:-1])
    assert tp["a_rows"] == r8.sum() + 128 and tp["b_rows"] == c8.sum() + tile_n
    blk = cols * ld
    assert tp["inc_elems"] == blk.sum()
    assert np.all(np.diff(tp["inc_off"]) == blk[:-1])
    tiles = tp["tiles"]
    assert tiles.shape[1] == 6
    cover = [np.zeros((int(cols[b]), int(ld[b])), np.int32) for b in range(len(lx))]
    seen = []
    for a_row, b_row, mv, nv, off, tld in tiles:
        b = int(np.searchsorted(tp["a_row0"], a_row, side="right") - 1)
        i, rem = divmod(int(a_row - tp["a_row0"][b]), 128)
        assert rem == 0 and a_row % 8 == 0 and b_row % 8 == 0
        j, rem = divmod(int(b_row - tp["b_row0"][b]), tile_n)
        assert rem == 0 and tld == ld[b] and tld % 4 == 0
        assert mv == min(128, rows[b] - 128 * i) > 0 and nv == min(tile_n, cols[b] - tile_n * j) > 0
        assert off == tp["inc_off"][b] + tile_n * j * ld[b] + 128 * i
        # the tile's block region: columns tile_n j .. +nv, rows 128 i .. +mv (column-major, ld rows a column)
        assert off + (nv - 1) * tld + mv <= tp["inc_off"][b] + blk[b]
        cover[b][tile_n * j:tile_n * j + nv, 128 * i:128 * i + mv] += 1
        seen.append(b)
    for b in range(len(lx)):
        assert np.all(cover[b][:, :rows[b]] == 1), b
    # largest pairs first (by coarse cells)
    firsts = list(dict.fromkeys(seen))
    assert firsts == list(np.argsort(-(rows * cols).astype(np.float64), kind="stable"))
