"""The bulk-copy staging geometry, checked on the CPU for every block and sector of the box and
block layouts the host accepts.

The hop kernels stage a sector region (the sector plus a 2-cell halo) by bulk copies of whole
rows when the lattice rows hold a multiple of 16 sites (make_region and the staging in
csrc/akmc_kernels.cu): each row's span is rounded out to 16-site boundaries from the region's
unwrapped origin, and a span that runs past the row's end, or starts before it (the halo of a
sector on the box's face in x), goes in two pieces, one from each end of the row.  The host sizes
shared memory for the widest region (region_sites in csrc/akmc_api.cu).  A bulk copy wants a
16-byte aligned source, destination and size, and must stay inside the lattice array.  This test
restates that geometry and checks, for each piece: alignment in both arrays (occupancy bytes,
int32 densities), sizes that are multiples of 16 bytes, a place inside the lattice row, pieces
of one row that cover disjoint sites and land where the unwrapped span puts them, a shared-memory
row pitch that holds the span and keeps every row 16-byte aligned, a layout within the host's
sizing, a transaction count within the mbarrier's limit, and the x halo the hop loop uses for its
"still inside the sector" test.
"""
import itertools

import pytest


def splits(n, nb):
    # block_split in csrc/akmc_model.cpp: nb blocks of n cells, the first n % nb one cell wider
    return [k * (n // nb) + min(k, n % nb) for k in range(nb + 1)]


def host_accepts(sp):
    # akmc_prepare: staged rows hold at most 64 sites in the row-load form
    return all(2 * ((sp[k + 1] - sp[k]) - (sp[k + 1] - sp[k]) // 2 + 4) <= 64 for k in range(len(sp) - 1))


def region_sites(sp3, bulk):
    mx = 1
    for d in range(3):
        sp = sp3[d]
        wmax = max((sp[k + 1] - sp[k]) - (sp[k + 1] - sp[k]) // 2 for k in range(len(sp) - 1))
        ext = (wmax + 4) * (2 if d == 0 else 1)
        if bulk and d == 0:
            ext = (ext + 14 + 15) & ~15
        mx *= ext
    return mx


def regions(n, nb):
    """(block, sector, region dict) for every block and sector of an n^3 box in nb^3 blocks."""
    sp = splits(n, nb)
    sx = 2 * n
    for bz, by, bx in itertools.product(range(nb), repeat=3):
        c0 = (sp[bx], sp[by], sp[bz])
        c1 = (sp[bx + 1], sp[by + 1], sp[bz + 1])
        for sec in range(8):
            slo, w = [], []
            for d in range(3):
                half = (c1[d] - c0[d]) // 2
                if (sec >> d) & 1:
                    slo.append(c0[d] + half)
                    w.append(c1[d] - c0[d] - half)
                else:
                    slo.append(c0[d])
                    w.append(half)
            R = dict(ox=2 * (slo[0] - 2), LX=2 * (w[0] + 4), LY=w[1] + 4, LZ=w[2] + 4, bulk=False)
            R["LXt"], R["xo"] = R["LX"], 0
            x0 = R["ox"] & ~15  # Python's & rounds negative origins down too
            bo = (R["ox"] - x0 + R["LXt"] + 15) & ~15
            if sx % 16 == 0 and bo <= sx:
                R["xo"] = R["ox"] - x0
                R["ox"] = x0
                R["LX"] = (R["LXt"] + 14 + 15) & ~15
                R["bo"] = bo
                R["br"] = (R["xo"] + R["LXt"] + 3) & ~3
                R["bulk"] = True
            R["hx"] = slo[0] - R["ox"] // 2
            R["n"] = R["LX"] * R["LY"] * R["LZ"]
            yield (bx, by, bz), sec, R


def pieces(ox, length, sx):
    """The bulk copies of one row's span of `length` sites from the unwrapped origin ox, as the
    staging issues them: (row position, sites, shared position)."""
    n1 = -ox if ox < 0 else min(length, sx - ox)
    out = [(ox + sx if ox < 0 else ox, n1, 0)]
    if length > n1:
        out.append((0, length - n1, n1))
    return out


LAYOUTS = [(n, nb) for n in (8, 16, 17, 20, 24, 25, 31, 32, 40, 47, 48, 56, 64, 96)
           for nb in sorted({1, 2, 3, max(1, n // 16), max(1, n // 8)})
           if (nb == 1 or n // nb >= 8) and host_accepts(splits(n, nb))] + [(128, 8), (256, 16), (256, 32)]


@pytest.mark.parametrize("n,nb", LAYOUTS)
def test_every_bulk_copy_is_aligned_and_in_bounds(n, nb):
    sx = 2 * n
    sp3 = [splits(n, nb)] * 3
    limit = region_sites(sp3, sx % 16 == 0)
    n_bulk = 0
    for blk, sec, R in regions(n, nb):
        assert R["n"] <= limit, (blk, sec)
        assert R["xo"] % 2 == 0 and R["hx"] == 2 + R["xo"] // 2, (blk, sec)
        if not R["bulk"]:
            assert R["LX"] <= 64
            continue
        n_bulk += 1
        ox, LX, bo, br = R["ox"], R["LX"], R["bo"], R["br"]
        assert sx % 16 == 0 and ox % 16 == 0 and -16 <= ox < sx
        for length, es in ((bo, 1), (br, 4)):  # occupancy bytes, int32 densities
            for piece_at, piece_len, dst in pieces(ox, length, sx):
                # every row starts at a multiple of sx (a multiple of 16 sites)
                assert (es * piece_at) % 16 == 0 and (es * piece_len) % 16 == 0 and (es * dst) % 16 == 0
                assert 0 <= piece_at and piece_at + piece_len <= sx and piece_len > 0
                # the piece holds the sites the unwrapped span puts at shared positions dst..
                assert (ox + dst) % sx == piece_at
            got = sorted(x for a, m, _ in pieces(ox, length, sx) for x in range(a, a + m))
            assert got == sorted((ox + k) % sx for k in range(length)) and len(set(got)) == length
        # shared rows: the pitch holds both spans and the region, and keeps rows aligned
        assert LX % 16 == 0 and bo <= LX and br <= LX and R["xo"] + R["LXt"] <= LX
        assert R["n"] % 2 == 0
        # the mbarrier's transaction count
        assert R["LY"] * R["LZ"] * (bo + 4 * br) < (1 << 20)
    if sx % 16 == 0 and nb > 1:
        assert n_bulk > 0


def test_256_cubed_stages_every_round_by_bulk_copies():
    # rows of 512 sites: regions on the box's faces in x go in two pieces per row
    regs = [R for _, _, R in regions(256, 16)]
    assert all(R["bulk"] for R in regs)
    wrapped = [R for R in regs if R["ox"] < 0 or R["ox"] + R["bo"] > 512]
    assert len(wrapped) * 16 == len(regs)


@pytest.mark.parametrize("n", [24, 32, 40, 48])
def test_single_block_boxes_with_16_site_rows_stage_by_bulk_copies(n):
    # one block: every sector's halo wraps in x
    assert all(R["bulk"] for _, _, R in regions(n, 1))


def test_a_span_longer_than_the_row_stays_on_row_loads():
    # a 16-cell box: rows of 32 sites, but the 24-site region rounds out to a 48-site span
    assert not any(R["bulk"] for _, _, R in regions(16, 1))
