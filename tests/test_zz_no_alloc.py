"""The allocation-free refine entry point (tdp_refine_batch_noalloc), through the C ABI.

It serves callers that cannot allocate device memory, so the test hands it
device buffers it allocated itself and checks, on two calls in a row with
different batches (the second call must not see the first one's leftovers),
that it returns what the ordinary entry point tdp_refine_batch returns for the
same inputs and what the FP64 oracle gives, both within the refine tests'
FP32 tolerance; that an empty row starting at the end of the batch is valid;
and that batches over its fixed limits are rejected with the limit named.
This file is collected last so a failure here never hides the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from test_refine_gpu import ERR_C, U, check, local_scale, make_batch, oracle_batch

pytestmark = pytest.mark.gpu


def call_noalloc(pkg, data, hd, osz, stream=None):
    import torch
    L = pkg.tdp.lib()
    L.tdp_refine_batch_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_uint32, C.c_void_p,
                                           C.c_void_p, C.c_char_p, C.c_size_t]
    d_data = torch.from_numpy(np.ascontiguousarray(data, np.float32)).cuda()
    d_hd = None if hd is None else torch.from_numpy(np.ascontiguousarray(hd, np.float32)).cuda()
    d_osz = torch.from_numpy(np.ascontiguousarray(osz, np.uint64).view(np.int64)).cuda()
    d_out = torch.empty((len(osz), 3), dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream()
    err = C.create_string_buffer(256)
    rc = L.tdp_refine_batch_noalloc(d_data.data_ptr(), None if d_hd is None else d_hd.data_ptr(), len(data),
                                    d_osz.data_ptr(), len(osz), d_out.data_ptr(), s.cuda_stream, err, 256)
    s.synchronize()
    return rc, err.value.decode(), d_out.cpu().numpy()


def test_noalloc_matches_refine_batch_on_two_calls(pkg, ctx):
    rng = np.random.default_rng(2026)
    for call in range(2):
        tri, hd, osz = make_batch(rng, 120 + 40 * call, sizes=(1, 120), gap=(0.0, 40.0))
        rc, msg, got = call_noalloc(pkg, tri, hd, osz)
        assert rc == 0, msg
        want = ctx.refine_batch(tri, hd, osz, form=pkg.FORM_TUNED)
        tol = ERR_C * U * np.maximum(local_scale(tri, osz), 1e-30)
        assert (np.abs(got[:, 0] - want[:, 0]) <= tol).all(), call
        assert (np.abs(got[:, 1:] - want[:, 1:]) <= tol[:, None] + 1e-5 * np.abs(want[:, 1:])).all(), call
        # and directly against the FP64 oracle
        check(got, oracle_batch(tri, hd, osz), tri, hd, osz)


def test_noalloc_without_hausdorff_and_bad_rows(pkg, ctx):
    rng = np.random.default_rng(7)
    tri, _, osz = make_batch(rng, 30)
    osz[3] = (len(tri) + 5, 4, 0, 2)  # points outside the batch
    rc, msg, got = call_noalloc(pkg, tri, None, osz)
    assert rc == 0, msg
    assert np.isnan(got[3]).all()
    ok = np.ones(len(osz), bool)
    ok[3] = False
    want = ctx.refine_batch(tri, None, osz[ok], form=pkg.FORM_TUNED)
    np.testing.assert_array_equal(got[ok][:, 1:], want[:, 1:])
    tol = ERR_C * U * np.maximum(local_scale(tri, osz[ok]), 1e-30)
    assert (np.abs(got[ok][:, 0] - want[:, 0]) <= tol).all()


def test_noalloc_rejects_oversized_batches(pkg):
    tri = np.zeros((300_000, 9), np.float32)
    osz = np.array([[0, 1, 1, 1]], np.uint64)
    rc, msg, _ = call_noalloc(pkg, tri, None, osz)
    assert rc == 1 and "262144" in msg


def test_noalloc_empty_row_at_the_end_of_the_batch(pkg, ctx):
    rng = np.random.default_rng(11)
    tri, hd, osz = make_batch(rng, 12)
    osz = np.concatenate([osz, np.array([[len(tri), 0, 0, 5]], np.uint64)])  # n1 = 0 at offset == element_num
    rc, msg, got = call_noalloc(pkg, tri, hd, osz)
    assert rc == 0, msg
    want = ctx.refine_batch(tri, hd, osz, form=pkg.FORM_TUNED)
    assert not np.isnan(got[-1]).any()
    np.testing.assert_array_equal(got[-1], want[-1])
    check(got[:-1], oracle_batch(tri, hd, osz[:-1]), tri, hd, osz[:-1])


def test_noalloc_rejects_too_many_pairs(pkg):
    tri = np.zeros((4, 9), np.float32)
    osz = np.tile(np.array([[0, 1, 1, 1]], np.uint64), (65537, 1))
    rc, msg, _ = call_noalloc(pkg, tri, None, osz)
    assert rc == 1 and "65536" in msg
