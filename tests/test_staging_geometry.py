"""The bulk-copy staging geometry and the device lattice's halo layout, checked on the CPU for
every block and sector of the box and block layouts the host accepts.  (A region that does not
wrap in y or z is staged instead by one tensor copy per array of the job's box; the box check
below restates that sizing.)

The device stores each x row of a job's lattice (sx sites) with a periodic halo
(lattice_pitch, lattice_put in csrc/akmc_device.h): kHaloL = 16 entries on the left hold copies
of the row's last sites, kHaloR = 32 on the right copies of its first ones, in a row of a pitch
rounded up to 16 entries; entry p holds site (p - kHaloL) mod sx, and a write of a site writes
every entry that holds it.  The hop kernels stage a sector region (the sector plus a 2-cell halo)
by one bulk copy per row and array (make_region, stage_rows in csrc/akmc_kernels.cu): the row's
span is rounded out to 16-site boundaries from the region's unwrapped origin x0, and entries
kHaloL + x0 .. kHaloL + x0 + bo are copied.  The host sizes shared memory for the widest region
(region_sites in csrc/akmc_api.cu).  A bulk copy wants a 16-byte aligned source, destination and
size, and must stay inside the row.  This test restates that geometry and checks, for each
copy: alignment in both arrays (occupancy bytes, int32 densities), sizes that are multiples of
16 bytes, a span inside the row's entries, entries that hold the sites the unwrapped span puts
at each shared position, a shared-memory row pitch that holds the span and keeps every row
16-byte aligned, a layout within the host's sizing, a transaction count within the mbarrier's
limit, and the x halo the hop loop uses for its "still inside the sector" test.
"""
import itertools

import pytest

HALO_L, HALO_R = 16, 32


def pitch(sx):
    # lattice_pitch in csrc/akmc_device.h
    return (HALO_L + sx + HALO_R + 15) & ~15


def row_layout(sx):
    """The sites a row's entries hold, as lattice_put leaves them (None: padding)."""
    row = [None] * pitch(sx)
    for x in range(sx):
        writes = [HALO_L + x]
        if x < HALO_R or x >= sx - HALO_L:
            writes += list(range(HALO_L + x - sx, -1, -sx))
            writes += list(range(HALO_L + x + sx, HALO_L + sx + HALO_R, sx))
        for p in writes:
            assert row[p] is None
            row[p] = x
    return row


def splits(n, nb):
    # block_split in csrc/akmc_model.cpp: nb blocks of n cells, the first n % nb one cell wider
    return [k * (n // nb) + min(k, n % nb) for k in range(nb + 1)]


def host_accepts(sp):
    # akmc_prepare: staged rows hold at most 64 sites in the row-load form
    return all(2 * ((sp[k + 1] - sp[k]) - (sp[k + 1] - sp[k]) // 2 + 4) <= 64 for k in range(len(sp) - 1))


def region_sites(sp3):
    mx = 1
    for d in range(3):
        sp = sp3[d]
        wmax = max((sp[k + 1] - sp[k]) - (sp[k + 1] - sp[k]) // 2 for k in range(len(sp) - 1))
        ext = (wmax + 4) * (2 if d == 0 else 1)
        if d == 0:
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
            if x0 >= -HALO_L and x0 + bo <= sx + HALO_R:
                R["xo"] = R["ox"] - x0
                R["ox"] = x0
                R["LX"] = (R["LXt"] + 14 + 15) & ~15
                R["bo"] = bo
                R["br"] = (R["xo"] + R["LXt"] + 3) & ~3
                R["bulk"] = True
            R["hx"] = slo[0] - R["ox"] // 2
            R["n"] = R["LX"] * R["LY"] * R["LZ"]
            yield (bx, by, bz), sec, R


LAYOUTS = [(n, nb) for n in (8, 9, 10, 16, 17, 20, 23, 24, 25, 31, 32, 40, 47, 48, 56, 64, 96)
           for nb in sorted({1, 2, 3, max(1, n // 16), max(1, n // 8)})
           if (nb == 1 or n // nb >= 8) and host_accepts(splits(n, nb))] + [(128, 8), (256, 16), (256, 32)]


@pytest.mark.parametrize("sx", [16, 18, 20, 30, 32, 34, 46, 48, 50, 64, 96, 512])
def test_every_site_and_halo_entry_holds_its_site(sx):
    row = row_layout(sx)
    px = pitch(sx)
    assert px % 16 == 0 and px >= HALO_L + sx + HALO_R
    for p in range(HALO_L + sx + HALO_R):
        assert row[p] == (p - HALO_L) % sx, p
    assert all(v is None for v in row[HALO_L + sx + HALO_R:])


@pytest.mark.parametrize("n,nb", LAYOUTS)
def test_every_bulk_copy_is_aligned_and_in_bounds(n, nb):
    sx = 2 * n
    px = pitch(sx)
    row = row_layout(sx)
    sp3 = [splits(n, nb)] * 3
    limit = region_sites(sp3)
    for blk, sec, R in regions(n, nb):
        # every region of a block of >= 8 cells fits the halo: one copy per row and array
        assert R["bulk"], (blk, sec)
        assert R["n"] <= limit, (blk, sec)
        assert R["xo"] % 2 == 0 and R["hx"] == 2 + R["xo"] // 2, (blk, sec)
        x0, LX, bo, br = R["ox"], R["LX"], R["bo"], R["br"]
        first = HALO_L + x0  # entry of the span's first site in its row
        assert x0 % 16 == 0 and first >= 0
        for length, es in ((bo, 1), (br, 4)):  # occupancy bytes, int32 densities
            # rows start on multiples of px (a multiple of 16 entries)
            assert (es * first) % 16 == 0 and (es * length) % 16 == 0
            assert first + length <= px
            # the entries hold the sites the unwrapped span puts at shared positions 0..length
            assert all(row[first + k] == (x0 + k) % sx for k in range(length)), (blk, sec)
        # the region's own sites lie inside both spans
        assert R["xo"] + R["LXt"] <= min(bo, br)
        # shared rows: the pitch holds both spans and the region, and keeps rows aligned
        assert LX % 16 == 0 and bo <= LX and br <= LX
        assert R["n"] % 2 == 0
        # the mbarrier's transaction count
        assert R["LY"] * R["LZ"] * (bo + 4 * br) < (1 << 20)


@pytest.mark.parametrize("n,nb", LAYOUTS)
def test_tensor_box_holds_every_region(n, nb):
    # the job's tensor box (setup_job: the widest region, x rounded as the bulk form rounds it)
    # is every region's shared-memory pitch: each region's bulk row span and its rows fit it, the
    # box's x extent is a multiple of 16 entries, and its volume is the host's shared-memory sizing
    sp = splits(n, nb)
    wmax = max((sp[k + 1] - sp[k]) - (sp[k + 1] - sp[k]) // 2 for k in range(nb))
    box = ((2 * (wmax + 4) + 14 + 15) & ~15, wmax + 4, wmax + 4)
    assert box[0] % 16 == 0 and all(1 <= b <= 256 for b in box)
    assert box[0] * box[1] * box[2] == region_sites([sp] * 3)
    for _, _, R in regions(n, nb):
        assert R["LX"] <= box[0] and R["bo"] <= box[0] and R["br"] <= box[0]
        assert R["LY"] <= box[1] and R["LZ"] <= box[2]
        # a region staged by the tensor copy starts on a 16-entry boundary of its row
        assert (HALO_L + R["ox"]) % 16 == 0


def test_256_cubed_regions_on_the_box_faces_in_x_use_the_halo():
    # rows of 512 sites: the regions of the blocks on the box's faces in x reach into the halo
    regs = [R for _, _, R in regions(256, 16)]
    assert all(R["bulk"] for R in regs)
    over = [R for R in regs if R["ox"] < 0 or R["ox"] + R["bo"] > 512]
    assert len(over) * 16 == len(regs)


@pytest.mark.parametrize("n", [8, 10, 16, 17, 23, 24, 32, 40, 48])
def test_single_block_boxes_stage_by_bulk_copies(n):
    # one block: every sector's halo wraps in x, into the row's halo entries
    assert all(R["bulk"] for _, _, R in regions(n, 1))
