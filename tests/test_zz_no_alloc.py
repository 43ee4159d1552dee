"""The allocation-free score_and_refine entry point, through the C ABI.

id11b_dev_score_and_refine_noalloc serves callers that cannot allocate device
memory (for example a process that has reserved all GPU memory up front for
its own buffers): it keeps its least-squares scratch in a library-owned device
array.  This test gives it the same inputs as the workspace-taking entry point
id11b_dev_score_and_refine and requires the same results, on two calls in a
row (the shared scratch keeps the previous call's contents, which must not leak
into the next result).  The file is named so that pytest collects it last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UBI_RTOL = 1e-12      # the tolerance the drop-in parity tests use
DRLV2_RTOL = 1e-12


def _run(lib, torch, fn, u, gv, tol, with_ws, stream):
    dev = gv.device
    ub = torch.tensor(u, dtype=torch.float64, device=dev).contiguous()
    n = torch.zeros(1, dtype=torch.int32, device=dev)
    m = torch.zeros(1, dtype=torch.float64, device=dev)
    if with_ws:
        wsb = lib.id11b_lsq_workspace_bytes(gv.shape[0])
        ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
        rc = fn(ub.data_ptr(), gv.data_ptr(), float(tol), gv.shape[0], n.data_ptr(),
                m.data_ptr(), ws.data_ptr(), wsb, stream)
    else:
        rc = fn(ub.data_ptr(), gv.data_ptr(), float(tol), gv.shape[0], n.data_ptr(),
                m.data_ptr(), stream)
    assert rc == 0, rc
    torch.cuda.synchronize()
    return int(n.item()), float(m.item()), ub.cpu().numpy()


def test_noalloc_matches_workspace_entry_point(golden, cuda):
    import torch
    from imaged11_b200._lib import lib
    d = golden["scoring"]
    gv = torch.tensor(d["sc_gv"], device=cuda)
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.id11b_noalloc_scratch_bytes() == lib.id11b_lsq_workspace_bytes(gv.shape[0])
    cases = [(d["sc_ubis"][i], t) for i in (0, 5, 21, 33) for t in d["sc_tols"]]
    for _call in range(2):               # two calls in a row over every case
        for u, t in cases:
            n_a, m_a, u_a = _run(lib, torch, lib.id11b_dev_score_and_refine, u, gv, t,
                                 True, stream)
            n_b, m_b, u_b = _run(lib, torch, lib.id11b_dev_score_and_refine_noalloc, u, gv,
                                 t, False, stream)
            assert n_b == n_a
            assert abs(m_b - m_a) <= DRLV2_RTOL * abs(m_a)
            assert np.abs(u_b - u_a).max() <= UBI_RTOL * np.abs(u_a).max()


def test_noalloc_small_and_empty_inputs(cuda):
    """A large call followed by an empty one: stale scratch must not leak."""
    import torch
    from imaged11_b200._lib import lib
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(3)
    u = np.eye(3) * 4.05
    g = torch.tensor(rng.integers(-4, 5, size=(5000, 3)) @ np.linalg.inv(u).T, device=cuda)
    n, m, _ = _run(lib, torch, lib.id11b_dev_score_and_refine_noalloc, u, g, 0.05, False,
                   stream)
    assert n == 5000
    empty = torch.zeros((0, 3), dtype=torch.float64, device=cuda)
    n, m, u2 = _run(lib, torch, lib.id11b_dev_score_and_refine_noalloc, u, empty, 0.05, False,
                    stream)
    assert (n, m) == (0, 0.0) and np.array_equal(u2, u)


def test_noalloc_rejects_sizes_beyond_maximum(cuda):
    from imaged11_b200._lib import lib
    # checked before any device access: the pointers are never used
    rc = lib.id11b_dev_score_and_refine_noalloc(8, 8, 0.1, 2 ** 31, 8, 8, None)
    assert rc == 4   # ID11B_ERR_SIZE
    assert lib.id11b_dev_score_and_refine_noalloc(8, 8, 0.1, -1, 8, 8, None) == 1


def test_noalloc_warmed_call_takes_no_device_memory(golden, cuda):
    """After one warm-up call (which loads the library's module lazily), a call
    leaves the device's free memory unchanged: the entry point allocates nothing."""
    import torch
    from imaged11_b200._lib import lib
    d = golden["scoring"]
    gv = torch.tensor(d["sc_gv"], device=cuda)
    ub = torch.tensor(d["sc_ubis"][5], dtype=torch.float64, device=cuda).contiguous()
    n = torch.zeros(1, dtype=torch.int32, device=cuda)
    m = torch.zeros(1, dtype=torch.float64, device=cuda)
    stream = torch.cuda.current_stream().cuda_stream
    fn = lib.id11b_dev_score_and_refine_noalloc
    assert fn(ub.data_ptr(), gv.data_ptr(), 0.05, gv.shape[0], n.data_ptr(), m.data_ptr(),
              stream) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(cuda)
    for _ in range(3):
        assert fn(ub.data_ptr(), gv.data_ptr(), 0.05, gv.shape[0], n.data_ptr(),
                  m.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(cuda)
    assert free1 == free0
