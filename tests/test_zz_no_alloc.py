"""mg_neighbor_lists_noalloc: the neighbour-list build with no allocation, against the existing
entry point mg_probe_neighbor_lists on the same points.

Neighbour lists are integer (index) results, so the tolerance is exact equality. The buffers the
entry point reads and writes are caller-owned device memory; the test allocates them with torch
(the entry point itself allocates nothing). Collected last (file name) so it runs both after the
other GPU tests and alone in a fresh process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from milldynamics3_b200.sim import probe_neighbor_lists

pytestmark = pytest.mark.gpu

MAX_POINTS = 16384  # the entry point's stated limit


def _bind(lib):
    fn = lib.dll.mg_neighbor_lists_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_uint32, C.c_float, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                   C.c_void_p]
    return fn


def _cloud(seed, n, spread):
    rng = np.random.default_rng(seed)
    return rng.uniform(-spread, spread, size=(n, 2)).astype(np.float32)


def _run_noalloc(fn, torch, pts, h, cap, stream):
    n = pts.shape[0]
    xy = torch.from_numpy(np.ascontiguousarray(pts).reshape(-1)).cuda()
    off = torch.full((n + 1,), 0xDEAD, dtype=torch.int32, device="cuda")
    nbrs = torch.full((max(cap, 1),), 0xBEEF, dtype=torch.int32, device="cuda")
    ne = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = torch.full((1,), 0x77, dtype=torch.int32, device="cuda")
    rc = fn(C.c_void_p(xy.data_ptr()), n, h, C.c_void_p(off.data_ptr()), C.c_void_p(nbrs.data_ptr()), cap,
            C.c_void_p(ne.data_ptr()), C.c_void_p(st.data_ptr()), C.c_void_p(stream.cuda_stream))
    stream.synchronize()
    return (rc, off.cpu().numpy().view(np.uint32), nbrs.cpu().numpy().view(np.uint32), int(ne.item()),
            int(st.item()))


# The last case puts one point far outside the cloud: its bounding box then holds far more cells
# than 2 n + 512, so the grid takes the sparse (sorted-key) path instead of the dense one.
@pytest.mark.parametrize("seed,n,h,outlier", [(1, 794, 0.00252, False), (2, 12700, 0.0011, False),
                                              (3, 100, 0.01, False), (4, 16384, 0.0009, False),
                                              (6, 16000, 0.0009, True)])
def test_matches_existing_entry_point_on_two_calls_in_a_row(device_lib, seed, n, h, outlier):
    torch = pytest.importorskip("torch")
    fn = _bind(device_lib)
    pts = _cloud(seed, n, 0.03)
    pts[n // 3] = np.nan  # a non-finite point is skipped by both
    if outlier:
        pts[7] = (1.0e3, 1.0e3)
    rc_ref, off_ref, nbrs_ref = probe_neighbor_lists(device_lib, pts, h)
    assert rc_ref == 0
    stream = torch.cuda.Stream()
    cap = int(off_ref[-1]) + 64
    for call in range(2):
        rc, off, nbrs, ne, st = _run_noalloc(fn, torch, pts, h, cap, stream)
        assert rc == 0, f"call {call}: {device_lib.global_last_error().decode()}"
        assert st == 0, f"call {call}: status bits {st:#x}"
        assert ne == int(off_ref[-1])
        assert np.array_equal(off, off_ref), f"call {call}: offsets differ"
        assert np.array_equal(nbrs[:ne], nbrs_ref), f"call {call}: neighbour lists differ"


def test_reports_small_capacity_and_rejects_too_many_points(device_lib):
    torch = pytest.importorskip("torch")
    fn = _bind(device_lib)
    stream = torch.cuda.Stream()
    pts = _cloud(5, 500, 0.01)
    _, off_ref, _ = probe_neighbor_lists(device_lib, pts, 0.002)
    rc, off, _, ne, st = _run_noalloc(fn, torch, pts, 0.002, 3, stream)
    assert rc == 0 and st == 1  # cap too small: reported in the status word, full count still given
    assert ne == int(off_ref[-1]) > 3 and np.array_equal(off, off_ref)
    # the empty input gives one zero offset
    rc, off, _, ne, st = _run_noalloc(fn, torch, np.zeros((0, 2), np.float32), 0.002, 0, stream)
    assert rc == 0 and st == 0 and ne == 0 and off[0] == 0
    # beyond the stated limit: rejected before anything runs, with a clear message
    big = torch.zeros(2 * (MAX_POINTS + 1), dtype=torch.float32, device="cuda")
    dummy = torch.zeros(MAX_POINTS + 2, dtype=torch.int32, device="cuda")
    rc = fn(C.c_void_p(big.data_ptr()), MAX_POINTS + 1, 0.002, C.c_void_p(dummy.data_ptr()),
            C.c_void_p(dummy.data_ptr()), 1, C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()), None)
    assert rc == 4  # MG_ERR_CAPACITY
    assert "no-allocation limit" in device_lib.global_last_error().decode()
