"""The allocation-free PCG entry point (cipc_gpu_pcg_bsr_noalloc).

Some callers cannot allocate device memory at solve time: a host whose GPU
memory is owned by its own allocator (here PyTorch's caching allocator owns
the matrix, right-hand side and solution), or a loop that must not pay
cudaMalloc latency.  This entry point takes device buffers from the caller and
keeps its scratch in a fixed array inside the library.  The test calls it
through the C ABI twice in a row and checks each result against the
allocating entry point, within the residual tolerance the other PCG tests
use.  It runs last so that a failure here cannot hide other failures.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

import cipc

pytestmark = pytest.mark.gpu


def _spd_block_system(nv=400, seed=0):
    rng = np.random.default_rng(seed)
    blocks = {}
    for i in range(nv):
        for j in (i, (i + 1) % nv, (i + 11) % nv):
            B = rng.standard_normal((3, 3)) * 0.1
            blocks.setdefault((i, j), np.zeros((3, 3)))
            blocks[(i, j)] += B
            blocks.setdefault((j, i), np.zeros((3, 3)))
            blocks[(j, i)] += B.T
    for i in range(nv):
        blocks[(i, i)] += 4.0 * np.eye(3)
    keys = sorted(blocks)
    rp = np.zeros(nv + 1, np.int32)
    for (i, _) in keys:
        rp[i + 1] += 1
    rp = np.cumsum(rp).astype(np.int32)
    ci = np.array([j for (_, j) in keys], np.int32)
    vals = np.ascontiguousarray(np.stack([blocks[k] for k in keys]))
    b = rng.standard_normal(3 * nv)
    A = sp.bsr_matrix((vals, ci, rp), shape=(3 * nv, 3 * nv)).tocsr()
    return rp, ci, vals, b, A


def _noalloc_call(rp, ci, vals, b, tol, sol_fill=float("nan")):
    """One call of the allocation-free entry point on device copies of the
    arrays (torch owns them, as the host's own allocator would)."""
    import torch

    nv = len(rp) - 1
    dev = torch.device("cuda", 0)
    d_rp = torch.from_numpy(np.ascontiguousarray(rp, np.int32)).to(dev)
    d_ci = torch.from_numpy(np.ascontiguousarray(ci, np.int32)).to(dev)
    d_vals = torch.from_numpy(np.ascontiguousarray(vals, np.float64).reshape(-1)).to(dev)
    d_b = torch.from_numpy(np.ascontiguousarray(b, np.float64)).to(dev)
    d_sol = torch.full((3 * nv,), sol_fill, dtype=torch.float64, device=dev)
    it = C.c_int(0)
    rr = C.c_double(0)
    stream = torch.cuda.current_stream().cuda_stream
    rc = cipc.lib().cipc_gpu_pcg_bsr_noalloc(nv, d_rp.data_ptr(), d_ci.data_ptr(), d_vals.data_ptr(), d_b.data_ptr(), d_sol.data_ptr(),
                                             tol, 10000, C.c_void_p(stream), C.byref(it), C.byref(rr))
    torch.cuda.synchronize()
    return rc, d_sol.cpu().numpy(), it.value


def _check_against_allocating(nv, seed):
    rp, ci, vals, b, A = _spd_block_system(nv=nv, seed=seed)
    tol = 1e-8
    x_ref, it_ref, _ = cipc.pcg_bsr(rp, ci, vals, b, precision="fp64", tol=tol)
    for call in range(2):
        rc, x, it = _noalloc_call(rp, ci, vals, b, tol)
        assert rc == 0, f"call {call}: rc {rc}"
        assert np.linalg.norm(A @ x - b) <= 1e-6 * np.linalg.norm(b)
        assert it == it_ref
        assert np.allclose(x, x_ref, rtol=1e-9, atol=1e-12 * np.abs(x_ref).max())


def test_noalloc_pcg_matches_allocating_entry_point():
    import torch

    torch.cuda.set_device(0)
    _check_against_allocating(400, 0)


def test_noalloc_at_the_row_limit():
    """A system of exactly CIPC_NOALLOC_MAX_ROWS block rows fills the whole
    scratch array; it matches the allocating entry point, twice in a row."""
    import torch

    torch.cuda.set_device(0)
    _check_against_allocating(cipc.NOALLOC_MAX_ROWS, 3)


def _drop_diagonal(rp, ci, vals, row):
    keep = np.ones(len(ci), bool)
    keep[rp[row] + int(np.nonzero(ci[rp[row]:rp[row + 1]] == row)[0][0])] = False
    rp2 = rp.copy()
    rp2[row + 1:] -= 1
    return rp2, ci[keep], vals[keep]


def test_noalloc_rejects_malformed_structure():
    """A row without its diagonal block, a duplicated diagonal block and a
    column index out of range are refused by both PCG entry points before
    any block is read (the solution buffer stays untouched); a valid call
    afterwards still solves."""
    import torch

    torch.cuda.set_device(0)
    rp, ci, vals, b, A = _spd_block_system(nv=64, seed=5)
    bad = [_drop_diagonal(rp, ci, vals, 17)]
    ci_dup = ci.copy()
    ci_dup[rp[9] + int(np.nonzero(ci[rp[9]:rp[10]] != 9)[0][0])] = 9  # a second diagonal block in row 9
    bad.append((rp, ci_dup, vals))
    ci_oob = ci.copy()
    ci_oob[5] = 64
    bad.append((rp, ci_oob, vals))
    for brp, bci, bvals in bad:
        rc, x, _ = _noalloc_call(brp, bci, bvals, b, 1e-8, sol_fill=7.0)
        assert rc == 1
        assert np.all(x == 7.0)
        with pytest.raises(cipc.CipcError):
            cipc.pcg_bsr(brp, bci, bvals, b, precision="fp64", tol=1e-8)
    rc, x, _ = _noalloc_call(rp, ci, vals, b, 1e-8)
    assert rc == 0 and np.linalg.norm(A @ x - b) <= 1e-6 * np.linalg.norm(b)


def test_noalloc_rejects_oversized_systems():
    L = cipc.lib()
    it = C.c_int(0)
    rr = C.c_double(0)
    rc = L.cipc_gpu_pcg_bsr_noalloc(cipc.NOALLOC_MAX_ROWS + 1, 1, 1, 1, 1, 1, 1e-6, 100, None, C.byref(it), C.byref(rr))
    assert rc == 1
