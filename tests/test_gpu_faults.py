"""Allocation failures, injected on the host (mg_test_fail_allocation).

The reference ends the process on any CUDA error (include/common.h:53-83).
Here the nth device allocation is made to fail as out-of-memory -- no GPU
fault is involved -- and every entry point that allocates must return
MG_ERR_OOM with text, release what it allocated, and leave its context (or
server) usable: the next call on it gives the oracle's result.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OOM = 3


def _free_mem():
    import torch

    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def _sweep_countdown(mg, attempt):
    """Arm n = 1, 2, ... until the attempt finishes without reaching the
    countdown; returns how many attempts failed (each must be an injected
    MG_ERR_OOM)."""
    failed = 0
    for nth in range(1, 400):
        mg.fail_allocation(nth)
        try:
            attempt()
        except mg.MGError as e:
            assert e.status == OOM and "injected" in str(e), str(e)
            failed += 1
            continue
        finally:
            left = mg.fail_allocation(0)
        # it finished: only possible before the nth allocation (a failure that
        # fired must have surfaced), so every allocation point has been hit
        assert left > 0, f"allocation {nth} failed but the call succeeded"
        return failed
    raise AssertionError("the countdown never ran out")


def test_louvain_and_stages_survive_failed_allocations(O, mg):
    g = O.gen_rmat(13, seed=2)
    ref = O.louvain(g)
    C = ref["assignment"].astype(np.uint32)
    before = _free_mem()
    ctx = mg.Context(0)

    def attempt():
        # a fresh context each time, so that every buffer is allocated anew
        c = mg.Context(0)
        try:
            h = c.graph_from_csr(g.n, g.offsets, g.cols, None)
            try:
                h.coarsen(C)[1].close()
                h.louvain(keep_levels=1)
            finally:
                h.close()
        finally:
            c.close()

    assert _sweep_countdown(mg, attempt) > 10
    # the engine works afterwards, on a context that saw failures as well
    for _ in range(2):
        mg.fail_allocation(3)
        try:
            ctx.graph_from_csr(g.n, g.offsets, g.cols, None).louvain()
        except mg.MGError as e:
            assert e.status == OOM
        mg.fail_allocation(0)
    r = ctx.graph_from_csr(g.n, g.offsets, g.cols, None).louvain()
    assert r["modularity"] == ref["modularity"] and (r["assignment"] == ref["assignment"]).all()
    ctx.close()
    # nothing leaked: device memory back to where it was (allow allocator slack)
    assert before - _free_mem() < 64 << 20


def test_batch_survives_failed_allocations(O, mg):
    gs = [O.gen_sbm(3000, 8, 12.0, 0.8, seed=s) for s in (1, 2, 3)]
    refs = [O.louvain(g) for g in gs]

    def attempt():
        c = mg.Context(0)
        try:
            b = c.batch_from_csr([(g.n, g.offsets, g.cols, None) for g in gs])
            try:
                b.run()
            finally:
                b.close()
        finally:
            c.close()

    assert _sweep_countdown(mg, attempt) > 5
    c = mg.Context(0)
    res = c.batch_from_csr([(g.n, g.offsets, g.cols, None) for g in gs]).run()
    for i, r in enumerate(refs):
        assert res["graphs"]["modularity"][i] == r["modularity"]
    c.close()


def test_server_job_fails_cleanly_and_the_slot_recovers(O, mg):
    g = O.gen_sbm(4000, 8, 12.0, 0.8, seed=5)
    ref = O.louvain(g)
    with mg.Server(device=0, slots=1, hbm_budget_bytes=8 << 30) as srv:
        mg.fail_allocation(1)
        j = srv.submit_csr(g.n, g.offsets, g.cols)
        info = srv.wait(j, timeout=120)
        mg.fail_allocation(0)
        assert info["state"] == mg.JOB_FAILED and info["status"] == OOM
        j2 = srv.submit_csr(g.n, g.offsets, g.cols, keep_assignment=True)
        info2 = srv.wait(j2, timeout=120)
        assert info2["state"] == mg.JOB_DONE
        assert info2["modularity"] == ref["modularity"]
        assert (srv.assignment(j2, g.n) == ref["assignment"]).all()
