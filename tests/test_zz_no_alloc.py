"""The allocation-free Morton sort entry point (nbb_morton_sort_noalloc).

It serves callers that cannot allocate device memory -- hosts that own all
device memory through their own pool or budget and do not let libraries call
cudaMalloc.  Its scratch is a fixed-size device array inside the library, so
this test checks, through the C ABI, that two calls in a row give exactly the
keys and permutation of the ordinary (allocating) entry point nbb_accel, and
that inputs beyond the array's capacity are rejected with a clear error.
Integer output, so the tolerance is exact equality.  The file sorts last so a
run that stops at the first failure has run every other test first; it also
passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(lib):
    fn = lib.nbb_morton_sort_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p] * 3 + [C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p]
    msg = lib.nbb_noalloc_last_error_message
    msg.restype = C.c_char_p
    msg.argtypes = []
    return fn, msg


def _noalloc_sort(nbb_mod, p):
    import torch

    fn, msg = _bind(nbb_mod.load())
    dev = torch.device("cuda:0")
    x, y, z = (torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (p.x, p.y, p.z))
    n = x.numel()
    keys = torch.empty(n, dtype=torch.int32, device=dev)
    idx = torch.empty(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    st = fn(C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), C.c_void_p(z.data_ptr()), n,
            C.c_void_p(keys.data_ptr()), C.c_void_p(idx.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert st == 0, msg().decode()
    return keys.cpu().numpy().view(np.uint32), idx.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_allocating_entry_point_twice(nbb_mod):
    from nbb import ics

    limit = 1 << 18  # NBB_NOALLOC_MAX_PARTICLES
    cases = [ics.plummer(100_000, seed=7), ics.blobs(limit, seed=8)]
    for p in cases:  # two calls in a row share the scratch array
        keys, idx = _noalloc_sort(nbb_mod, p)
        _, _, _, ex = nbb_mod.compute_accelerations(p, 0.5, 0.01, 1.0, export=True)
        assert np.array_equal(keys, ex["keys"])
        assert np.array_equal(idx, ex["idx"])


def test_noalloc_sort_rejects_oversized_input(nbb_mod):
    import torch

    fn, msg = _bind(nbb_mod.load())
    n = (1 << 18) + 1
    dev = torch.device("cuda:0")
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    out = torch.empty(n, dtype=torch.int32, device=dev)
    st = fn(C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), n,
            C.c_void_p(out.data_ptr()), C.c_void_p(out.data_ptr()), None)
    assert st == 1  # NBB_ERR_INVALID_ARGUMENT
    assert "NBB_NOALLOC_MAX_PARTICLES" in msg().decode()


def _raw_call(nbb_mod, x, y, z, keys, idx):
    fn, msg = _bind(nbb_mod.load())
    st = fn(C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), C.c_void_p(z.data_ptr()), x.numel(),
            C.c_void_p(keys.data_ptr()), C.c_void_p(idx.data_ptr()), None)
    return st, msg().decode()


def test_noalloc_sort_reports_non_finite_input_then_recovers(nbb_mod):
    # a NaN position is the reference's domain error; the error word in the
    # shared scratch is cleared again by the next call
    import torch
    from nbb import ics

    p = ics.plummer(5000, seed=11)
    dev = torch.device("cuda:0")
    x, y, z = (torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (p.x, p.y, p.z))
    keys = torch.empty(5000, dtype=torch.int32, device=dev)
    idx = torch.empty(5000, dtype=torch.int32, device=dev)
    bad = x.clone()
    bad[1234] = float("nan")
    st, text = _raw_call(nbb_mod, bad, y, z, keys, idx)
    assert st == 2 and "must be finite" in text  # NBB_ERR_DOMAIN
    st, text = _raw_call(nbb_mod, x, y, z, keys, idx)
    assert st == 0, text
    _, _, _, ex = nbb_mod.compute_accelerations(p, 0.5, 0.01, 1.0, export=True)
    assert np.array_equal(keys.cpu().numpy().view(np.uint32), ex["keys"])
    assert np.array_equal(idx.cpu().numpy().view(np.uint32), ex["idx"])


def test_noalloc_sort_takes_no_device_memory(nbb_mod):
    # free device memory is unchanged across a call (the first call of the
    # process may load the library's device module, so measure a later one)
    import torch
    from nbb import ics

    p = ics.plummer(200_000, seed=12)
    dev = torch.device("cuda:0")
    x, y, z = (torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (p.x, p.y, p.z))
    keys = torch.empty(x.numel(), dtype=torch.int32, device=dev)
    idx = torch.empty(x.numel(), dtype=torch.int32, device=dev)
    st, text = _raw_call(nbb_mod, x, y, z, keys, idx)
    assert st == 0, text
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(dev)
    st, text = _raw_call(nbb_mod, x, y, z, keys, idx)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert st == 0, text
    assert free1 == free0


def test_noalloc_sort_refuses_stream_capture(nbb_mod):
    # the call reads its error word back and synchronises, which a capture
    # forbids: on a capturing stream it returns NBB_ERR_INVALID_ARGUMENT and
    # leaves the capture intact
    import torch

    fn, msg = _bind(nbb_mod.load())
    dev = torch.device("cuda:0")
    x = torch.zeros(1000, dtype=torch.float64, device=dev)
    keys = torch.zeros(1000, dtype=torch.int32, device=dev)
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream(dev)
    with torch.cuda.graph(g, stream=s):
        st = fn(C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), 1000,
                C.c_void_p(keys.data_ptr()), C.c_void_p(keys.data_ptr()), C.c_void_p(s.cuda_stream))
        keys.add_(1)
    assert st == 1 and "captured" in msg().decode()
    g.replay()
    torch.cuda.synchronize()
    assert int(keys.sum()) == 1000
