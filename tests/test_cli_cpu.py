"""The `tdbase join` command line (3dpipe_b200/bin/tdbase) on the host: the
reference's operator surface (src/tools/tdbase.cpp:482-549, options
src/include/query_context.h:145-167) with status codes instead of exit() deep
inside the library -- usage errors exit 2, missing inputs and an absent
device exit 1 with a message, nothing crashes."""
import subprocess
from pathlib import Path

import pytest


@pytest.fixture(scope="module")
def exe(pkg):
    p = Path(pkg.__file__).parent / "bin" / "tdbase"
    assert p.exists(), "the CLI is built by __graft_entry__.build()"
    return str(p)


@pytest.fixture(scope="module")
def tile_files(pkg, tmp_path_factory):
    d = tmp_path_factory.mktemp("tiles")
    nb, vb = pkg.tdp.gen_tiles(2, 4, seed=21)
    p1, p2 = d / "n.dt", d / "v.dt"
    nb.tofile(p1)
    vb.tofile(p2)
    return str(p1), str(p2)


def run(exe, *args):
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=120)


def test_usage_errors(exe, tile_files):
    n, v = tile_files
    cases = [
        ((), "usage: tdbase join"),
        (("convert",), "usage: tdbase join"),
        (("join", "--tile1", n), "usage: tdbase join"),                       # no query
        (("join", "--tile1", n, "-q", "nn", "--bogus"), "unknown option --bogus"),
        (("join", "--tile1", n, "-q"), "missing value for -q"),
        (("join", "--tile1", n, "-q", "closest"), "error query type: closest"),
        (("join", "--tile1", n, "-q", "nn", "--form", "fast"), "unknown form fast"),
        (("join", "--tile1", n, "-q", "nn") + ("-l", "20") * 9, "at most 8 LODs"),
    ]
    for args, msg in cases:
        out = run(exe, *args)
        assert out.returncode == 2, (args, out.returncode, out.stderr)
        assert msg in out.stderr, (args, out.stderr)


def test_missing_tile_file(exe, tile_files, tmp_path):
    n, _ = tile_files
    missing = str(tmp_path / "none.dt")
    for args in (("--tile1", missing), ("--tile1", n, "--tile2", missing)):
        out = run(exe, "join", *args, "-q", "nn", "--knn", "2")
        assert out.returncode == 1
        assert f"{missing} does not exist" in out.stderr


def test_no_device_is_a_message_not_a_crash(exe, tile_files):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present: the join itself is covered by the GPU tests")
    n, v = tile_files
    out = run(exe, "join", "--tile1", n, "--tile2", v, "-q", "within", "--within_dist", "100", "-g",
              "--print_result")
    assert out.returncode == 1
    assert "cannot open device 0 (status 7)" in out.stderr
    assert out.stdout == ""
