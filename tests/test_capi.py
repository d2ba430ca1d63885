"""The C-ABI library loads on CPU and exports every symbol include/tdp.h declares."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    txt = (ROOT / "include" / "tdp.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(tdp_[a-z0-9_]+)\s*\(", txt)))


def test_header_symbols_exported(pkg):
    L = pkg.tdp.lib()
    names = declared_symbols()
    assert names, "no declarations found"
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(pkg.tdp.EXPORTED)


def test_no_device_is_an_error_not_a_crash(pkg):
    import torch
    if torch.cuda.is_available():
        return
    L = pkg.tdp.lib()
    h = ctypes.c_void_p()
    rc = L.tdp_ctx_create(0, 0, 0, ctypes.byref(h))
    assert rc == 7  # TDP_ERR_NODEV


NULL_CALLS = r'''
import ctypes as C, importlib, sys
sys.path.insert(0, sys.argv[1])
tdp = importlib.import_module("3dpipe_b200").tdp
L = tdp.lib()
z, i0, i1, f0 = C.c_size_t(0), C.c_int(0), C.c_int(1), C.c_float(0)
calls = {
    "tdp_ctx_create": (i0, z, C.c_uint(0), None),
    "tdp_ctx_destroy": (None,),
    "tdp_ctx_memory": (None, None, None),
    "tdp_last_stats": (None, None),
    "tdp_fp32_peak": (None, None),
    "tdp_refine_config_info": (C.c_int(99), None, None),
    "tdp_set_refine_config": (None, i0),
    "tdp_get_refine_config": (None, None),
    "tdp_get_refine_config_lod": (None, C.c_int(20), None),
    "tdp_set_lod_graph": (None, i0),
    "tdp_tile_upload": (None, None, z, C.c_long(0), None),
    "tdp_tile_attach": (None, None, z, C.c_long(0), None),
    "tdp_host_alloc": (C.c_size_t(16), None),
    "tdp_host_free": (None,),
    "tdp_tile_free": (None, None),
    "tdp_tile_get_info": (None, None),
    "tdp_tile_compute_bounds": (None, None, None),
    "tdp_raw_compute_bounds": (None, None, z, None, None),
    "tdp_join": (None, None, None, None, None),
    "tdp_result_count": (None, None),
    "tdp_result_copy": (None, None, None, None),
    "tdp_result_copy_f64": (None, None),
    "tdp_result_free": (None,),
    "tdp_autotune": (None, None, None, None, None, None),
    "tdp_join_chunked": (None, None, z, None, z, None, C.c_long(0), None, None),
    "tdp_server_create": (None, None, None, None),
    "tdp_server_submit": (None, None, z, i0, i1, f0, None),
    "tdp_server_wait": (None, C.c_uint64(0), i0, None, None),
    "tdp_server_get_stats": (None, None),
    "tdp_server_destroy": (None,),
    "tdp_refine_batch": (None, None, None, z, None, C.c_uint32(0), i0, None),
    "tdp_gen_tiles": (None, None, z, None, None, z, None, None, z),
    "tdp_partition_queries": (None, None, None, C.c_long(0), None, None, None, C.c_long(0), i0, i0, i1, f0,
                              C.c_int(2), None, None),
    "tdp_raw_partition": (None, z, None, z, i0, i1, f0, C.c_int(2), None, None, None, z),
    "tdp_raw_prep_bound": (None, C.c_long(1), C.c_int(100), None),
    "tdp_raw_from_meshes": (None, None, None, None, None, C.c_long(0), C.c_int(100), None, z, None, None),
    "tdp_gen_meshes": (None, i0, None, z, None, None, z, None, None, None, None, None, z),
}
for name, args in calls.items():
    print(name, getattr(L, name)(*args))
L.tdp_raw_check.restype = C.c_int
print("tdp_raw_check", L.tdp_raw_check(None, z, None, None, None, z))
for name, args in (("tdp_candidates", (None, None, C.c_long(0), None, None, C.c_long(0), i0, i1, i1, f0, None, None,
                                       C.c_long(0))),
                   ("tdp_tile_candidates", (None, None, None, i1, i1, f0, None, None, C.c_long(0)))):
    f = getattr(L, name)
    f.restype = C.c_long
    print(name, f(*args))
L.tdp_last_error.restype = C.c_char_p
print("tdp_last_error", L.tdp_last_error(None).decode().replace(" ", "_"))
L.tdp_ctx_stream.restype = C.c_void_p
print("tdp_ctx_stream", L.tdp_ctx_stream(None))
# an empty batch is nothing to do
print("tdp_refine_batch_noalloc", L.tdp_refine_batch_noalloc(None, None, z, None, C.c_uint32(0), None, None, None, z))
for name in ("tdp_join_default_params", "tdp_server_default_params", "tdp_gen_default_params"):
    getattr(L, name).restype = None
    getattr(L, name)(None)
    print(name, "returned")
L.tdp_host_cache_trim.restype = None
L.tdp_host_cache_trim()
print("tdp_host_cache_trim", "returned")
L.tdp_host_cache_bytes.restype = C.c_size_t
print("tdp_host_cache_bytes", L.tdp_host_cache_bytes())
print("tdp_refine_config_count", L.tdp_refine_config_count())
'''


def test_null_arguments_are_errors_not_crashes(pkg, tmp_path):
    """Every entry point given null handles and pointers returns its documented
    error (TDP_ERR_ARG, or LONG_MIN for the candidate counts), or does nothing
    for the parameter fillers, without touching a device or crashing; run in a
    child process so a crash fails only this test."""
    import subprocess
    import sys
    script = tmp_path / "null_calls.py"
    script.write_text(NULL_CALLS)
    out = subprocess.run([sys.executable, str(script), str(ROOT)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    got = dict(line.split() for line in out.stdout.splitlines())
    for name, value in got.items():
        if name in ("tdp_candidates", "tdp_tile_candidates"):
            assert int(value) == -(2 ** 63), (name, value)
        elif name == "tdp_raw_check":
            assert int(value) == 4, value                      # an empty buffer is malformed bytes
        elif name == "tdp_last_error":
            assert value == "null_context"
        elif name == "tdp_ctx_stream":
            assert value == "None"
        elif name == "tdp_refine_batch_noalloc":
            assert int(value) == 0
        elif name.endswith("_default_params") or name == "tdp_host_cache_trim":
            assert value == "returned"
        elif name == "tdp_host_cache_bytes":
            assert int(value) == 0                             # trimmed just before
        elif name == "tdp_refine_config_count":
            assert int(value) == 18
        else:
            assert int(value) == 1, (name, value)              # TDP_ERR_ARG
    assert set(got) == set(declared_symbols()), sorted(set(declared_symbols()) ^ set(got))
