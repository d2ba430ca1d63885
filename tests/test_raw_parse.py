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


# Tiles of many equal-size records: the parser's threads walk chunks from
# starts guessed at the first record's stride.  Two record kinds share one
# size -- A: one voxel with 29 triangles (5+5+6+6+7 over the LODs), B: twelve
# voxels without triangles (44 * 29 + 116 == 116 * 12) -- so the voxel count
# tells whether every record was found where the serial walk finds it.
def _record(kind, extra_voxels=0):
    if kind == "A":
        counts, nv = (5, 5, 6, 6, 7), 1
    else:
        counts, nv = (0, 0, 0, 0, 0), 12
    nv += extra_voxels
    data = bytearray(44 * sum(counts))
    for i in range(0, len(data), 4):
        struct.pack_into("<f", data, i, float(i % 97))
    rec = bytearray(struct.pack("<Q", len(data))) + data + struct.pack("<Q", nv)
    rec += struct.pack("<10f", *([1.0] * 10))
    off = 0
    for v in range(nv):
        rec += struct.pack("<9f", 0, 0, 0, 1, 1, 1, 0.5, 0.5, 0.5)
        for li in range(5):
            c = counts[li] if v == 0 else 0
            rec += struct.pack("<QQ", off, c)
            off += 44 * c
    rec += struct.pack("<3f", 0, 0, 0)
    return bytes(rec)


def _uniform_tile(n, seed, odd=None):
    """(bytes, voxels per record, record offsets); record `odd` gets one more voxel"""
    rng = np.random.default_rng(seed)
    kinds = rng.integers(0, 2, n)
    recs = {"A": _record("A"), "B": _record("B")}
    parts, nvox, offs = [b"\x01"], [], []
    pos = 1
    for i, k in enumerate(kinds):
        r = _record("AB"[k], 1) if odd == i else recs["AB"[k]]
        offs.append(pos)
        parts.append(r)
        pos += len(r)
        nvox.append((1 if k == 0 else 12) + (1 if odd == i else 0))
    return np.frombuffer(b"".join(parts), np.uint8).copy(), np.array(nvox), np.array(offs)


def test_uniform_records_found_by_the_parallel_walk(pkg):
    assert len(_record("A")) == len(_record("B"))
    raw, nvox, offs = _uniform_tile(20000, 3)
    assert pkg.tdp.raw_check(raw) == (20000, nvox.sum())
    # the tile ends 77 records early: the last chunk stops at the end
    assert pkg.tdp.raw_check(raw[:offs[-77]]) == (20000 - 77, nvox[:-77].sum())


@pytest.mark.parametrize("odd", [1, 7000, 19999])
def test_a_longer_record_breaks_the_guessed_starts(pkg, odd):
    raw, nvox, _ = _uniform_tile(20000, 4, odd=odd)
    assert pkg.tdp.raw_check(raw) == (20000, nvox.sum())


def test_errors_inside_guessed_chunks(pkg):
    raw, _, offs = _uniform_tile(20000, 5)
    b = raw.copy()
    p = int(offs[17000])
    (ds,) = struct.unpack_from("<Q", b, p)
    struct.pack_into("<Q", b, p + 8 + ds, 0)                 # a zero voxel count
    with pytest.raises(pkg.TdpError) as e:
        pkg.tdp.raw_check(b)
    assert str(e.value).endswith("bad voxel count of object 17000")
    b = raw.copy()
    for o in (19000, 12345):                                   # inverted boxes: the lowest is named
        p = int(offs[o])
        (ds,) = struct.unpack_from("<Q", b, p)
        struct.pack_into("<f", b, p + 8 + ds + 8 + 40 + 12, -1.0)
    with pytest.raises(pkg.TdpError) as e:
        pkg.tdp.raw_check(b)
    assert str(e.value).endswith("inverted voxel box in object 12345")


def test_host_block_cache_recycles_and_trims(pkg):
    """The parser's arrays of 1 MiB and up go back to the process-wide block
    cache when a parse ends, are reused by the next parse of the same tile,
    and are handed back to the system on request."""
    raw, nvox, _ = _uniform_tile(40000, 6)      # ~260k voxels: the per-voxel offset arrays exceed 1 MiB
    pkg.tdp.host_cache_trim()
    assert pkg.tdp.host_cache_bytes() == 0
    assert pkg.tdp.raw_check(raw) == (40000, nvox.sum())
    held = pkg.tdp.host_cache_bytes()
    assert held > 0
    assert pkg.tdp.raw_check(raw) == (40000, nvox.sum())
    assert pkg.tdp.host_cache_bytes() == held    # the second parse took its blocks from the cache and gave them back
    pkg.tdp.host_cache_trim()
    assert pkg.tdp.host_cache_bytes() == 0


def _record_table(raw):
    """(record offsets plus the end, voxels per record) of RAW tile bytes"""
    offs, pos = [], 1
    nvox = []
    while pos < len(raw):
        offs.append(pos)
        (ds,) = struct.unpack_from("<Q", raw, pos)
        (vn,) = struct.unpack_from("<Q", raw, pos + 8 + ds)
        nvox.append(vn)
        pos += 8 + ds + 8 + 40 + 116 * vn + 12
    return np.array(offs + [pos]), np.array(nvox)


@pytest.mark.parametrize("tile", ["equal-size records", "generated nuclei"])
def test_random_corruptions_report_what_a_sequential_read_finds(pkg, tile):
    """Random byte changes, some with the tile cut short after them: the
    parser reports the first problem a sequential read meets, or the counts
    it reads.  Equal-size records are walked by the parser's threads from
    guessed starts; the generated tile's records differ in size."""
    from rawdt import first_problem
    if tile == "equal-size records":
        raw, _, _ = _uniform_tile(12000, 7)
    else:
        raw, _ = pkg.tdp.gen_tiles(3, 200, seed=8)
        raw = np.array(raw)
    ends, nvox = _record_table(raw)
    offs, n = ends[:-1], len(ends) - 1
    rng = np.random.default_rng(11)
    for trial in range(200):
        r = int(rng.integers(0, n))
        p, q = int(offs[r]), int(ends[r + 1])
        (ds,) = struct.unpack_from("<Q", raw, p)
        if trial % 2:   # a field outside the data block: sizes, bounds, voxel records, lod tables, transform
            at = p + int(rng.choice([0, 8 + ds + int(rng.integers(0, q - p - 8 - ds))]))
        else:
            at = p + int(rng.integers(0, q - p))
        old = int(raw[at])
        raw[at] = (old + int(rng.integers(1, 256))) % 256   # changed in place, restored below
        cut = trial % 5 == 4
        b = raw[: int(rng.integers(at + 1, len(raw) + 1))] if cut else raw
        # records after the changed byte are intact up to the end (or the cut)
        resume = None if cut else {int(o): i for i, o in enumerate(offs) if o > at}
        want = first_problem(b, p, r, resume)
        if want[0] == "error":
            with pytest.raises(pkg.TdpError) as e:
                pkg.tdp.raw_check(b)
            assert e.value.code == 4
            assert str(e.value).endswith(want[1]), (trial, str(e.value), want)
        else:
            k = want[3]
            objs = r + want[1] + (n - k if k is not None else 0)
            vox = int(nvox[:r].sum()) + want[2] + (int(nvox[k:].sum()) if k is not None else 0)
            assert pkg.tdp.raw_check(b) == (objs, vox), (trial, want)
        raw[at] = old


def test_concurrent_parses_share_the_block_cache(pkg):
    """Parses on several threads at once (as request submissions to a server
    run): each returns its own tile's counts while they take blocks from,
    and give them back to, the one process-wide cache."""
    import threading
    tiles = [_uniform_tile(n, seed) for n, seed in ((9000, 31), (12000, 32), (3000, 33), (20000, 34))]
    want = [(len(offs), int(nvox.sum())) for _, nvox, offs in tiles]
    errors = []

    def worker(k):
        try:
            for i in range(6):
                j = (k + i) % len(tiles)
                got = pkg.tdp.raw_check(tiles[j][0])
                if got != want[j]:
                    errors.append((k, j, got))
        except Exception as e:  # noqa: BLE001 -- reported below
            errors.append((k, repr(e)))

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(8)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    assert not errors, errors[:3]
    pkg.tdp.host_cache_trim()
    assert pkg.tdp.host_cache_bytes() == 0


@pytest.mark.filterwarnings("ignore:This process .* is multi-threaded")
def test_parallel_parse_on_the_host_pool_survives_fork(pkg):
    """The parser's parallel loops (the chunked walk, the voxel tables, the
    prefix sums) run on one process-wide pool of host threads; a child
    forked from a process that has started the pool starts its own."""
    import os
    import signal
    import time
    nb, _ = pkg.tdp.gen_tiles(50, 200, seed=31, only="nuclei")  # 10,000 equal records
    first = pkg.tdp.raw_check(nb)
    assert first == (10000, 130000)
    assert pkg.tdp.raw_check(nb) == first
    pid = os.fork()
    if pid == 0:
        code = 3
        try:
            code = 0 if pkg.tdp.raw_check(nb) == first else 2
        finally:
            os._exit(code)
    deadline = time.time() + 120
    while True:
        done, status = os.waitpid(pid, os.WNOHANG)
        if done:
            break
        if time.time() > deadline:
            os.kill(pid, signal.SIGKILL)
            os.waitpid(pid, 0)
            pytest.fail("the forked child did not finish parsing")
        time.sleep(0.05)
    assert os.WIFEXITED(status) and os.WEXITSTATUS(status) == 0
