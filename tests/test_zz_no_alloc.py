"""The cell-list build that allocates no device memory (ctc_clist_build_noalloc).

It exists for callers that cannot call cudaMalloc where they build cell lists
(an allocator hook, which must not re-enter the allocator it implements, or a
service that must not allocate on its steady-state path).  It must give
exactly the result of the allocating entry point (ctc_clist_build): cell
counts, starts, the sorted particles and the input index of each, bit for bit
-- also on the calls after the first, which find the shared scratch array
holding the previous call's leftovers: a larger call after a smaller one, then
a smaller one after it, in both particles and cells, so that stale slots
beyond the current sizes are left in the array.  This file is named so that
pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from ctc_b200 import _lib, systems

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _noalloc(L, pp):
    n = len(pp)
    nc = L[0] * L[1] * L[2]
    P = torch.as_tensor(pp, device="cuda")
    out = torch.zeros_like(P)
    starts = torch.full((nc + 1,), -1, dtype=torch.int32, device="cuda")
    counts = torch.full((nc,), -1, dtype=torch.int32, device="cuda")
    ids = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = lambda t: C.c_void_p(t.data_ptr())
    _lib.check(_lib.lib().ctc_clist_build_noalloc(*L, n, p(P), p(out), p(starts), p(counts), p(ids), st))
    torch.cuda.synchronize()
    nout = int(starts[nc].item())
    return out[:nout].cpu().numpy(), starts.cpu().numpy(), counts.cpu().numpy(), ids[:nout].cpu().numpy()


def _allocating(L, pp):
    import ctc_b200
    out, starts, counts, ids = ctc_b200.Clist(L, len(pp)).build(torch.as_tensor(pp, device="cuda"))
    return out.cpu().numpy(), starts.cpu().numpy(), counts.cpu().numpy(), ids.cpu().numpy()


def test_noalloc_matches_allocating_build_in_a_row():
    # three calls in a row: larger, then smaller in particles and cells
    cases = [((12, 10, 8), 1), ((16, 16, 8), 2), ((10, 6, 8), 3)]
    for L, seed in cases:
        pp = systems.solvent(L, seed=seed)
        extra = systems.solvent(L, n=50, seed=seed + 10)
        extra[:, 1] -= L[1]                             # outside the box: dropped by both
        pp = np.concatenate([pp, extra])
        np.random.default_rng(seed).shuffle(pp)
        got = _noalloc(L, pp)
        ref = _allocating(L, pp)
        for a, b in zip(got, ref):
            assert a.shape == b.shape and np.array_equal(a, b)


def test_noalloc_rejects_oversize():
    """one particle over the limit: refused before any launch (the buffers
    are large enough all the same)"""
    L = (8, 8, 8)
    n = 262144 + 1
    pp = torch.zeros((n, 6), dtype=torch.float32, device="cuda")
    out = torch.zeros_like(pp)
    starts = torch.zeros(8 * 8 * 8 + 1, dtype=torch.int32, device="cuda")
    counts = torch.zeros(8 * 8 * 8, dtype=torch.int32, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())
    rc = _lib.lib().ctc_clist_build_noalloc(*L, n, p(pp), p(out), p(starts), p(counts), None, None)
    assert rc == _lib.CTC_ERR_CAPACITY
    assert b"exceed the fixed scratch" in _lib.lib().ctc_last_error()
