"""The bulk-copy staging geometry, checked on the CPU for every block and sector of the box and
block layouts the host accepts.

The hop kernels stage a sector region (the sector plus a 2-cell halo) by one bulk copy per row
and array when the lattice rows hold a multiple of 16 sites and the region does not wrap in x
(make_region in csrc/akmc_kernels.cu); the host sizes shared memory for the widest such region
(region_sites in csrc/akmc_api.cu).  A bulk copy wants a 16-byte aligned source, destination and
size, and must stay inside the lattice array.  This test restates that geometry and checks, for
each copy: alignment of the row start in both arrays (occupancy bytes, int32 densities), sizes
that are multiples of 16 bytes, an end inside the lattice row, a shared-memory row pitch that
holds the copy and keeps every row 16-byte aligned, a layout within the host's sizing, a
transaction count within the mbarrier's limit, and the x halo the hop loop uses for its
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
            if sx % 16 == 0 and R["ox"] >= 0 and R["ox"] + R["LX"] <= sx:
                x0 = R["ox"] & ~15
                R["xo"] = R["ox"] - x0
                R["ox"] = x0
                R["LX"] = (R["LXt"] + 14 + 15) & ~15
                R["bo"] = (R["xo"] + R["LXt"] + 15) & ~15
                R["br"] = (R["xo"] + R["LXt"] + 3) & ~3
                R["bulk"] = True
            R["hx"] = slo[0] - R["ox"] // 2
            R["n"] = R["LX"] * R["LY"] * R["LZ"]
            yield (bx, by, bz), sec, R


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
        # sources: every row starts at a multiple of sx (a multiple of 16 sites), plus ox
        assert sx % 16 == 0 and ox % 16 == 0
        assert (4 * ox) % 16 == 0
        # sizes, ends inside the lattice row
        assert bo % 16 == 0 and (4 * br) % 16 == 0
        assert 0 <= ox and ox + bo <= sx and ox + br <= sx
        # shared rows: the pitch holds both copies and the region, and keeps rows aligned
        assert LX % 16 == 0 and bo <= LX and br <= LX and R["xo"] + R["LXt"] <= LX
        assert R["n"] % 2 == 0
        # the mbarrier's transaction count
        assert R["LY"] * R["LZ"] * (bo + 4 * br) < (1 << 20)
    if sx % 16 == 0 and nb > 1:
        assert n_bulk > 0


def test_256_cubed_stages_fifteen_of_sixteen_rounds_by_bulk_copies():
    flags = [R["bulk"] for _, _, R in regions(256, 16)]
    assert sum(flags) * 16 == len(flags) * 15
