"""The allocation-free collision entry point against the allocating one.

avbd_collide_noalloc serves callers that may not allocate device memory
during a call (fixed budgets, custom pools, hosts where cudaMalloc/cudaFree
would synchronise or fail): its scratch is one fixed device array shared by
every call.  This file is collected last so a failure here leaves every other
test already run.  It must pass alone in a fresh process and after the rest.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scene(Solver, n_pairs, seed):
    rng = np.random.default_rng(seed)
    s = Solver()
    pairs = []
    for i in range(n_pairs):
        sa = rng.uniform(0.3, 2.0, 3).astype(np.float32)
        sb = rng.uniform(0.3, 2.0, 3).astype(np.float32)
        qa = rng.normal(size=4)
        qb = rng.normal(size=4)
        qa = (qa / np.linalg.norm(qa)).astype(np.float32)
        qb = (qb / np.linalg.norm(qb)).astype(np.float32)
        pa = rng.uniform(-1, 1, 3).astype(np.float32) + np.float32(10.0 * i)
        pb = pa + (rng.normal(size=3) * 0.4 * (sa.mean() + sb.mean())).astype(np.float32)
        a = s.add_body(0, 1.0, 0.5, pa, sa, quat=qa)
        b = s.add_body(0, 1.0, 0.5, pb, sb, quat=qb)
        pairs.append((a, b))
    return s, np.array(pairs, np.int32)


def _call_noalloc(lib, handle, pairs):
    n = len(pairs)
    a = np.ascontiguousarray(pairs[:, 0])
    b = np.ascontiguousarray(pairs[:, 1])
    ids = np.zeros((n, 8), np.uint32)
    data = np.zeros((n, 8, 13), np.float32)
    counts = np.zeros(n, np.int32)
    ip = C.POINTER(C.c_int32)
    rc = lib.avbd_collide_noalloc(handle, n, a.ctypes.data_as(ip), b.ctypes.data_as(ip),
                                  ids.ctypes.data_as(C.POINTER(C.c_uint32)),
                                  data.ctypes.data_as(C.POINTER(C.c_float)), counts.ctypes.data_as(ip))
    return rc, ids, data, counts


def test_noalloc_matches_collide_two_calls():
    from skyephyx_b200 import Solver, load
    lib = load()
    s, pairs = _scene(Solver, 300, 99)
    # the allocating entry point (uploads the world on first use)
    ref = [s.collide(int(a), int(b)) for a, b in pairs]
    # two calls in a row over different pair sets: the second must not see the first's contents
    first, second = pairs[:300], pairs[::-1][:120]
    for batch in (first, second):
        rc, ids, data, counts = _call_noalloc(lib, s.handle, batch)
        assert rc == 0
        for i, (a, b) in enumerate(batch):
            j = int(np.nonzero((pairs[:, 0] == a) & (pairs[:, 1] == b))[0][0])
            r_ids, r_data = ref[j]
            k = len(r_ids)
            assert counts[i] == k
            assert [int(x) for x in ids[i, :k]] == r_ids
            assert np.all(ids[i, k:] == 0xFFFFFFFF)
            # bit-exact, the tolerance of every narrowphase test here
            assert np.array_equal(data[i, :k].view(np.uint32), r_data.view(np.uint32))
            assert np.all(data[i, k:] == 0.0)
    assert sum(len(r[0]) > 0 for r in ref) > 40


def test_noalloc_rejects_oversized_request():
    from skyephyx_b200 import Solver, load
    lib = load()
    s, pairs = _scene(Solver, 4, 7)
    s.collide(0, 1)   # uploads the world
    big = np.zeros((4097, 2), np.int32)
    big[:, 1] = 1
    rc, *_ = _call_noalloc(lib, s.handle, big)
    assert rc == -1   # AVBD_ERR_INVALID: more pairs than AVBD_COLLIDE_NOALLOC_MAX_PAIRS
