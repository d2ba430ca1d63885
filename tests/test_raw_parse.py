"""The RAW tile parser on the host (tdp_raw_check, the parser every upload and
attach uses): counts on generated tiles, checked against the independent
numpy reader, and the first error in file order for malformed bytes -- both
when the size fields are broken (the sequential walk) and when only the voxel
tables are (the parallel pass), where the lowest bad object must be named."""
import struct

import numpy as np
import pytest

from rawdt import read_tile


def test_counts_match_independent_reader(pkg):
    for nv, npv in ((1, 3), (10, 200)):          # the second has enough objects for the parallel pass
        nb, vb = pkg.tdp.gen_tiles(nv, npv, seed=5)
        for raw in (nb, vb):
            n_obj, n_vox = pkg.tdp.raw_check(raw)
            objs = read_tile(raw)
            assert n_obj == len(objs)
            assert n_vox == sum(len(o.voxels) for o in objs)


def corrupt_box(raw, off, obj):
    """invert the x extent of the first voxel box of object `obj`"""
    b = raw.copy()
    p = int(off[obj])
    (ds,) = struct.unpack_from("<Q", b, p)
    q = p + 8 + ds + 8 + 40          # first voxel record
    lo_x = struct.unpack_from("<f", b, q)[0]
    struct.pack_into("<f", b, q + 12, lo_x - 1.0)  # high x below low x
    return b


@pytest.mark.parametrize("bad", [[7], [1500, 40], [1999]])
def test_content_errors_name_the_lowest_object(pkg, bad):
    nb, _ = pkg.tdp.gen_tiles(10, 200, seed=5)
    off = pkg.tdp.raw_object_offsets(nb)
    b = nb
    for o in bad:
        b = corrupt_box(b, off, o)
    with pytest.raises(pkg.TdpError) as e:
        pkg.tdp.raw_check(b)
    assert e.value.code == 4
    assert str(e.value).endswith("inverted voxel box in object %d" % min(bad))


def test_lod_range_error(pkg):
    nb, _ = pkg.tdp.gen_tiles(10, 200, seed=5)
    off = pkg.tdp.raw_object_offsets(nb)
    b = nb.copy()
    p = int(off[321])
    (ds,) = struct.unpack_from("<Q", b, p)
    q = p + 8 + ds + 8 + 40 + 36      # lod table of the first voxel
    struct.pack_into("<Q", b, q, ds + 4)   # offset past the data block
    with pytest.raises(pkg.TdpError) as e:
        pkg.tdp.raw_check(b)
    assert str(e.value).endswith("voxel lod range outside data block in object 321")


def test_structural_errors(pkg):
    nb, _ = pkg.tdp.gen_tiles(10, 200, seed=5)
    off = pkg.tdp.raw_object_offsets(nb)
    p = int(off[500])
    (ds,) = struct.unpack_from("<Q", nb, p)
    cases = [
        (nb[:p + 8 + ds // 2], "bad data_size of object 500"),            # cut inside the data block
        (nb[:p + 8 + ds + 8 + 40 + 20], "truncated voxel record of object 500"),
        (nb[:p + 8 + ds + 8 + 40 + 50], "truncated voxel lod table"),
        (nb[:int(off[501]) - 6], "truncated transform of object 500"),
    ]
    b = nb.copy()
    struct.pack_into("<Q", b, p + 8 + ds, 0)                               # a zero voxel count
    cases.append((b, "bad voxel count of object 500"))
    # a box error before a structural error: the box error comes first in file order
    cases.append((corrupt_box(nb, off, 100)[: int(off[501]) - 6], "inverted voxel box in object 100"))
    for raw, want in cases:
        with pytest.raises(pkg.TdpError) as e:
            pkg.tdp.raw_check(raw)
        assert e.value.code == 4
        assert str(e.value).endswith(want), (str(e.value), want)
    with pytest.raises(pkg.TdpError):
        pkg.tdp.raw_check(np.array([2, 0, 0], np.uint8))   # not RAW
