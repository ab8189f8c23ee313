"""cmi_traverse_buffer_noalloc: the allocation-free traversal entry point.

Callers whose GPU memory is owned by someone else (a host code with its own
pool allocator, a plug-in inside another application's process) cannot call
cudaMalloc/cudaFree.  This entry point takes every buffer from the caller
(here: tensors from torch's allocator) and keeps its intermediate photons in
one fixed device array inside the library.  Its results must equal those of
the allocating entry point cmi_traverse_buffer on the same inputs, on two calls
in a row (the second call reuses the array the first one left behind).
"""
import ctypes as C

import numpy as np
import pytest

from conftest import golden

from parallelcmacionize_b200 import GridSpec, TransportEngine, _lib

pytestmark = pytest.mark.gpu


def _bind():
    L = _lib.load()
    f = L.cmi_traverse_buffer_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                  C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_void_p]
    f.restype = C.c_int
    return f


def _noalloc(f, torch, box, ncell, nH_t, xH_t, J_t, in_dir, photons, enabled):
    n = photons.size
    d_in = torch.from_numpy(photons.view(np.uint8).copy()).cuda()
    d_out = torch.zeros(max(n, 1) * 80, dtype=torch.uint8, device="cuda")
    d_cnt = torch.zeros(27, dtype=torch.int32, device="cuda")
    d_done = torch.zeros(1, dtype=torch.int32, device="cuda")
    b = np.ascontiguousarray(box, np.float64)
    nc = np.ascontiguousarray(ncell, np.int32)
    en = None if enabled is None else np.ascontiguousarray(enabled, np.uint8)
    torch.cuda.synchronize()
    rc = f(b.ctypes.data, nc.ctypes.data, nH_t.data_ptr(), xH_t.data_ptr(), J_t.data_ptr(),
           int(in_dir), d_in.data_ptr(), n, en.ctypes.data if en is not None else None,
           d_out.data_ptr(), d_cnt.data_ptr(), d_done.data_ptr(), None)
    _lib.check(rc)
    counts = d_cnt.cpu().numpy().astype(np.uint32)
    out = np.frombuffer(d_out.cpu().numpy().tobytes(), dtype=_lib.PHOTON_DTYPE)
    return out[: int(counts.sum())], counts, int(d_done.item())


def test_noalloc_matches_traverse_buffer_twice():
    torch = pytest.importorskip("torch")
    f = _bind()
    g = golden("walk_interior16.npz")
    box, ncell = g["box"], g["ncell"]
    # the caller's device memory
    nH_t = torch.from_numpy(g["nH"].copy()).cuda()
    xH_t = torch.from_numpy(g["xH"].copy()).cuda()
    J_t = torch.zeros_like(nH_t)
    # the allocating entry point on the same subgrid
    eng = TransportEngine(GridSpec(box=tuple(box), ncell=tuple(int(v) for v in ncell),
                                   num_subgrid=(1, 1, 1)), precision="fp64")
    eng.set_fields(0, g["nH"], g["xH"])

    ph = g["photons"]
    enabled2 = np.ones(27, np.uint8)
    enabled2[0] = 0  # absorbed packets done (reemission off)
    calls = [(ph, None), (ph[:150], enabled2)]  # second call: fewer photons, other flags
    for photons, enabled in calls:
        out_n, cnt_n, done_n = _noalloc(f, torch, box, ncell, nH_t, xH_t, J_t, 0, photons,
                                        enabled)
        out_r, cnt_r, done_r = eng.traverse_buffer(0, 0, 0, photons, enabled=enabled)
        assert np.array_equal(cnt_n, cnt_r)
        assert done_n == done_r
        assert out_n.tobytes() == out_r.tobytes()  # FP64 walk: bit-exact
        _, J_r = eng.get_fields(0)
        np.testing.assert_allclose(J_t.cpu().numpy(), J_r, rtol=1e-13, atol=0)
    eng.close()


def test_noalloc_rejects_oversized_buffers():
    torch = pytest.importorskip("torch")
    f = _bind()
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    box = np.array([0, 0, 0, 1, 1, 1], np.float64)
    nc = np.array([2, 2, 2], np.int32)
    rc = f(box.ctypes.data, nc.ctypes.data, t.data_ptr(), t.data_ptr(), t.data_ptr(), 0,
           t.data_ptr(), 4097, None, t.data_ptr(), t.data_ptr(), t.data_ptr(), None)
    assert rc == _lib.ERR_CAPACITY
    assert b"4096" in _lib.load().cmi_last_error_string()


def test_noalloc_reproduces_reference_photons_all_entry_directions():
    """Straight against the reference's own interact (golden photons of
    walk_entries8: every one of the 27 entry directions), grouped as
    do_photon_traversal groups them, with unchanged free device memory once
    the entry point has been called (no allocation)."""
    torch = pytest.importorskip("torch")
    f = _bind()
    g = golden("walk_entries8.npz")
    box, ncell = g["box"], g["ncell"]
    nH_t = torch.from_numpy(g["nH"].copy()).cuda()
    xH_t = torch.from_numpy(g["xH"].copy()).cuda()
    J_t = torch.zeros_like(nH_t)
    seen = set()
    for d in np.unique(g["in_dirs"]):
        sel = np.nonzero(g["in_dirs"] == d)[0]
        _noalloc(f, torch, box, ncell, nH_t, xH_t, J_t, int(d), g["photons"][sel], None)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        out, counts, done = _noalloc(f, torch, box, ncell, nH_t, xH_t, J_t, int(d),
                                     g["photons"][sel], None)
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0
        res = g["result"][sel]
        expect = np.concatenate([g["out"][sel][res == k] for k in range(27)])
        assert done == 0
        assert np.array_equal(counts, np.bincount(res, minlength=27))
        assert out.tobytes() == expect.tobytes()
        seen.add(int(d))
    assert seen == set(range(27))


def test_noalloc_empty_buffer_and_oversized_subgrid():
    torch = pytest.importorskip("torch")
    f = _bind()
    t = torch.zeros(4096 * 2, dtype=torch.float64, device="cuda")
    cnt = torch.full((27,), 7, dtype=torch.int32, device="cuda")
    done = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    box = np.array([0, 0, 0, 1, 1, 1], np.float64)
    nc = np.array([2, 2, 2], np.int32)
    # n = 0 with no photon buffers: nothing walks, every group is empty
    rc = f(box.ctypes.data, nc.ctypes.data, t.data_ptr(), t.data_ptr(), t.data_ptr(), 0,
           None, 0, None, None, cnt.data_ptr(), done.data_ptr(), None)
    assert rc == _lib.OK
    assert int(cnt.sum().item()) == 0 and int(done.item()) == 0
    # more than 4096 cells per subgrid: refused before any launch
    big = np.array([16, 16, 17], np.int32)
    rc = f(box.ctypes.data, big.ctypes.data, t.data_ptr(), t.data_ptr(), t.data_ptr(), 0,
           t.data_ptr(), 1, None, t.data_ptr(), cnt.data_ptr(), done.data_ptr(), None)
    assert rc == _lib.ERR_NOT_SUPPORTED
    assert b"4096" in _lib.load().cmi_last_error_string()
