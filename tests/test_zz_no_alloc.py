"""spq_gmres_dev_noalloc: GMRES for callers that must not allocate device memory
while they run (a service that reserves its GPU memory at start-up, a real-time
loop that may not enter the allocator). Its Krylov workspace comes from one
fixed device array instead of cudaMalloc; the result must equal the allocating
spq_gmres_dev's on the same inputs, call after call.

Collected last (file name) so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from spaqr_public_b200 import Tree, matgen
from spaqr_public_b200._abi import check, lib

pytestmark = pytest.mark.gpu


def _setup():
    import torch
    w = matgen.workload("advdiff2d_32")
    A = matgen.column_normalize(w["A"])
    t = Tree(w["levels"], w["skip"])
    t.set_tol(w["tol"])
    t.set_scale(1)
    t.set_square(1)
    t.set_coords_grid(w["n"], w["d"])
    t.partition(A)
    t.assemble(A)
    t.factorize()
    m, n, rp, ci, va = matgen.to_csr(A)
    dev = dict(rp=torch.tensor(rp, dtype=torch.int32, device="cuda"),
               ci=torch.tensor(ci, dtype=torch.int32, device="cuda"),
               va=torch.tensor(va, dtype=torch.float64, device="cuda"),
               b=torch.tensor(w["b"], dtype=torch.float64, device="cuda"))
    return w, A, t, dev


def _pool_bytes():
    used, reserved = C.c_ulonglong(0), C.c_ulonglong(0)
    check(lib().spq_pool_memory(0, C.byref(used), C.byref(reserved)))
    return used.value, reserved.value


def _gmres(fn, t, A, dev, restart, tol, memory=None):
    """One GMRES call; with memory a list, appends the device pool's (used,
    reserved) bytes and the device's free bytes just before and just after the
    call (nothing else runs in between)."""
    import torch
    x = torch.zeros(A[1], dtype=torch.float64, device="cuda")
    its = C.c_int(0)
    res = C.c_double(0)
    torch.cuda.synchronize()
    if memory is not None:
        memory.append((_pool_bytes(), torch.cuda.mem_get_info()[0]))
    rc = fn(t._h, A[0], C.c_void_p(dev["rp"].data_ptr()), C.c_void_p(dev["ci"].data_ptr()),
            C.c_void_p(dev["va"].data_ptr()), C.c_void_p(dev["b"].data_ptr()), C.c_void_p(x.data_ptr()), 100,
            restart, tol, C.byref(its), C.byref(res))
    if memory is not None:
        torch.cuda.synchronize()
        memory.append((_pool_bytes(), torch.cuda.mem_get_info()[0]))
    return rc, x.cpu().numpy(), its.value, res.value


def test_noalloc_gmres_matches_allocating_gmres(gpu):
    w, A, t, dev = _setup()
    L = lib()
    # before any preconditioner application the solve graph does not exist yet
    rc, _, _, _ = _gmres(L.spq_gmres_dev_noalloc, t, A, dev, 100, w["res"])
    assert rc == 2 and b"apply the preconditioner once" in L.spq_last_error()
    t.solve(w["b"])
    for _ in range(2):  # two calls in a row: the shared workspace keeps old contents
        rc, x_ref, its_ref, res_ref = _gmres(L.spq_gmres_dev, t, A, dev, 100, w["res"])
        check(rc)
        memory = []
        rc, x, its, res = _gmres(L.spq_gmres_dev_noalloc, t, A, dev, 100, w["res"], memory)
        check(rc)
        # nothing taken from the device pool, and no device memory at all
        # (the workspace and the kernels were loaded when the handle bound the device)
        assert memory[0] == memory[1]
        assert its == its_ref
        assert abs(res - res_ref) <= 1e-6 * res_ref
        assert np.linalg.norm(x - x_ref) <= 1e-10 * np.linalg.norm(x_ref)
        true = np.linalg.norm(matgen.spmv(A, x) - w["b"]) / np.linalg.norm(w["b"])
        assert true <= 10 * w["res"]


def test_noalloc_gmres_rejects_oversized_workspace(gpu):
    w, A, t, dev = _setup()
    t.solve(w["b"])
    # m * (restart + 1) doubles beyond the fixed 4 Mi-double workspace
    rc, _, _, _ = _gmres(lib().spq_gmres_dev_noalloc, t, A, dev, 5000, w["res"])
    assert rc == 1
    assert b"fixed workspace holds" in lib().spq_last_error()
