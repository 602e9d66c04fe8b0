"""mg_local_move_noalloc: the local-move sweep for callers that cannot call
cudaMalloc (a process whose HBM budget already belongs to its own pool, or
code that must not enter the CUDA allocator).  Its hash tables live in a
static 16 MiB device array instead of engine allocations.

The test gives it device buffers it did not allocate itself (torch tensors),
calls it through the C ABI twice in a row, and checks each result against
the regular entry point mg_local_move and against the oracle (bit-exact:
integral weights).  One graph has a hub of degree 100,000 among 100,000
low-degree vertices: each vertex's table follows its own degree.  It
also checks that a graph whose maximum degree exceeds the static array is
refused with a clear error.  This file is collected last on purpose.
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(mg):
    L = mg.lib()
    f = L.mg_local_move_noalloc
    f.restype = ct.c_int
    f.argtypes = [ct.c_uint32, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_double, ct.c_void_p, ct.c_void_p,
                  ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p]
    return f


def _dev(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a).astype(dtype)).cuda()


def test_noalloc_matches_local_move(O, mg, ctx):
    import torch

    f = _noalloc(mg)
    base = O.gen_rmat(14, seed=6)
    row = np.repeat(np.arange(base.n), np.diff(base.offsets).astype(np.int64))
    m = row < base.cols
    w = np.random.default_rng(4).integers(1, 6, m.sum()).astype(np.float64)
    leaves = 100_000
    ring = np.arange(1, leaves + 1)
    hub = O.csr_from_pairs(leaves + 1, np.concatenate([np.zeros(leaves, np.int64), ring]),
                           np.concatenate([ring, ring % leaves + 1]))
    for g in (base, O.csr_from_pairs(base.n, row[m], base.cols[m], w), hub):
        n = g.n
        k = O.vertex_weights(g)
        mass = O.mass(g)
        dg = ctx.graph_from_csr(n, g.offsets, g.cols, g.weights)
        d_off = _dev(torch, g.offsets, np.int32)
        d_col = _dev(torch, g.cols, np.int32)
        d_w = None if g.weights is None else _dev(torch, g.weights, np.float64)
        # two calls in a row: phase start, then a later assignment
        C = np.arange(n, dtype=np.uint32)
        sig = k.copy()
        for call in range(2):
            for version, up in ((2, True), (1, False)):
                d_C = _dev(torch, C, np.int32)
                d_s = _dev(torch, sig, np.float64)
                d_k = _dev(torch, k, np.float64)
                d_out = torch.full((n,), -1, dtype=torch.int32, device="cuda")
                st = f(n, d_off.data_ptr(), d_col.data_ptr(), None if d_w is None else d_w.data_ptr(), mass,
                       d_C.data_ptr(), d_s.data_ptr(), d_k.data_ptr(), d_out.data_ptr(), version, int(up), None)
                assert st == 0, mg.lib().mg_last_error(None)
                torch.cuda.synchronize()
                got = d_out.cpu().numpy().view(np.uint32)
                want, _ = dg.local_move(C, sig, k, version, up)
                assert (got == want).all(), (call, version, up, np.nonzero(got != want)[0][:10])
                ref, _ = O.local_move(g, C, sig, k, mass, version, up)
                assert (got == ref).all(), (call, version, up, np.nonzero(got != ref)[0][:10])
            C, _ = O.local_move(g, C, sig, k, mass, 2, True)
            sig = np.zeros(n)
            np.add.at(sig, C, k)


def test_noalloc_rejects_degree_beyond_static_scratch(O, mg):
    import torch

    f = _noalloc(mg)
    leaves = 600_000
    g = O.csr_from_pairs(leaves + 1, np.zeros(leaves, np.int64), np.arange(1, leaves + 1))
    n = g.n
    d_off = _dev(torch, g.offsets, np.int32)
    d_col = _dev(torch, g.cols, np.int32)
    k = O.vertex_weights(g)
    d_C = _dev(torch, np.arange(n), np.int32)
    d_s = _dev(torch, k, np.float64)
    d_k = _dev(torch, k, np.float64)
    d_out = torch.zeros(n, dtype=torch.int32, device="cuda")
    st = f(n, d_off.data_ptr(), d_col.data_ptr(), None, O.mass(g), d_C.data_ptr(), d_s.data_ptr(), d_k.data_ptr(),
           d_out.data_ptr(), 2, 1, None)
    assert st == 6  # MG_ERR_UNSUPPORTED
    assert b"static scratch" in mg.lib().mg_last_error(None)
