"""avism_gpu_knn_noalloc: the kNN entry point whose scratch is a static device
array.  Collected last (file name) so that it also runs after every other GPU
test has used the library; it passes alone as well.

Its results must equal avism_gpu_knn's bit for bit, over consecutive calls that
reuse the same static scratch with different inputs."""
import ctypes as C

import numpy as np
import pytest

MAX_N = 1048576   # AVISM_KNN_NOALLOC_MAX_N in include/avism_gpu.h


def _noalloc(lib, dev_arrays, box_l, k, stream):
    import torch
    x, y, z, qx, qy, qz = dev_arrays
    nq = qx.numel()
    idx = torch.empty(nq * k, dtype=torch.int64, device=x.device)
    dist = torch.empty(nq * k, dtype=torch.float32, device=x.device)
    err = C.create_string_buffer(256)
    st = lib.avism_gpu_knn_noalloc(0, C.c_void_p(stream), x.numel(), x.data_ptr(), y.data_ptr(), z.data_ptr(),
                                   box_l, nq, qx.data_ptr(), qy.data_ptr(), qz.data_ptr(), k, idx.data_ptr(),
                                   dist.data_ptr(), err, 256)
    return st, err.value.decode(), idx, dist


def _case(seed, n, nq, box_l, spread):
    rng = np.random.default_rng(seed)
    lo, hi = (-box_l / 2, box_l / 2) if box_l > 0 else (-spread, spread)
    pts = rng.uniform(lo, hi, size=(3, n)).astype(np.float32)
    qs = rng.uniform(lo, hi, size=(3, nq)).astype(np.float32)
    if box_l > 0:
        pts = np.clip(pts, np.float32(lo), np.nextafter(np.float32(hi), np.float32(0)))
        qs = np.clip(qs, np.float32(lo), np.nextafter(np.float32(hi), np.float32(0)))
    return pts, qs


@pytest.mark.gpu
def test_noalloc_matches_knn_over_consecutive_calls(gpu):
    import torch
    from avism_b200 import _lib
    lib = _lib.load()
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev).cuda_stream
    cases = [
        (11, 262144, 200000, 100.0, 0.0, 32),      # periodic, k <= 32
        (12, MAX_N, 150000, 0.0, 37.0, 48),        # non-periodic, the largest n, k <= 64
        (11, 262144, 200000, 100.0, 0.0, 32),      # the first case again after the scratch was reused
    ]
    results = []
    for seed, n, nq, box_l, spread, k in cases:
        pts, qs = _case(seed, n, nq, box_l, spread)
        d = [torch.from_numpy(a.copy()).to(dev) for a in (*pts, *qs)]
        st, msg, idx, dist = _noalloc(lib, d, box_l, k, stream)
        assert st == 0 and msg == "", (st, msg)
        torch.cuda.current_stream(dev).synchronize()
        ref_idx, ref_dist = gpu.knn_search(*pts, *qs, k, box_l=box_l)
        got_idx = idx.cpu().numpy().reshape(nq, k)
        got_dist = dist.cpu().numpy().reshape(nq, k)
        assert np.array_equal(got_idx, ref_idx)
        assert np.array_equal(got_dist.view(np.uint32), ref_dist.view(np.uint32))
        results.append(got_idx)
    assert np.array_equal(results[0], results[2])


@pytest.mark.gpu
def test_noalloc_rejects_oversize_and_host_pointers(gpu):
    import torch
    from avism_b200 import _lib
    lib = _lib.load()
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev).cuda_stream
    big = [torch.zeros(MAX_N + 1, dtype=torch.float32, device=dev) for _ in range(3)]
    q = [torch.zeros(4, dtype=torch.float32, device=dev) for _ in range(3)]
    st, msg, _, _ = _noalloc(lib, big + q, 10.0, 8, stream)
    assert st == 1 and "AVISM_KNN_NOALLOC_MAX_N" in msg, (st, msg)

    hx = np.zeros(16, np.float32)
    idx = torch.empty(4 * 8, dtype=torch.int64, device=dev)
    dist = torch.empty(4 * 8, dtype=torch.float32, device=dev)
    err = C.create_string_buffer(256)
    p = hx.ctypes.data
    st = lib.avism_gpu_knn_noalloc(0, C.c_void_p(stream), 16, p, p, p, 10.0, 4, q[0].data_ptr(),
                                   q[1].data_ptr(), q[2].data_ptr(), 8, idx.data_ptr(), dist.data_ptr(), err, 256)
    assert st == 1 and b"not a device pointer" in err.value, (st, err.value)


@pytest.mark.gpu
@pytest.mark.parametrize("k,box_l", [(8, 0.0), (100, 60.0), (100, 0.0), (200, 60.0), (200, 0.0)])
def test_noalloc_matches_oracle(k, box_l):
    """Against the CPU oracle's kNN (k-d tree, ties by particle index) on the
    same points, over the 32-, 128- and 256-wide instantiations, periodic and
    not; two calls in a row with different inputs."""
    import torch
    from avism_b200 import _lib
    from oracle import oracle as O
    lib = _lib.load()
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev).cuda_stream
    for seed in (k, k + 1):
        pts, qs = _case(seed, 30000, 2000, box_l, 30.0)
        d = [torch.from_numpy(a.copy()).to(dev) for a in (*pts, *qs)]
        st, msg, idx, dist = _noalloc(lib, d, box_l, k, stream)
        assert st == 0 and msg == "", (st, msg)
        torch.cuda.current_stream(dev).synchronize()
        ref_idx, ref_dist = O.knn(*pts, *qs, k, box_l)
        assert np.array_equal(idx.cpu().numpy().reshape(-1, k), ref_idx)
        assert np.array_equal(dist.cpu().numpy().reshape(-1, k).view(np.uint32), ref_dist.view(np.uint32))
