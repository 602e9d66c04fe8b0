"""Host logic of the serving loop, without a GPU: admission, cancellation,
refusal of jobs larger than a slot's budget, statistics and shutdown.  (With
no CUDA device the worker slots fail to start, so submitted jobs stay
queued; the GPU tests cover the running path.)"""
import pytest

from conftest import cuda_available


@pytest.fixture
def server(mg):
    if cuda_available():
        pytest.skip("host-only checks: on a GPU machine the workers would run the jobs")
    s = mg.Server(slots=2, hbm_budget_bytes=2 * 10**9)
    yield s
    s.stop()


def test_submit_queue_cancel_stats(mg, server):
    ids = [server.submit(mg.gen_params("sbm", n=1000 + i, blocks=4, seed=i)) for i in range(5)]
    assert len(set(ids)) == 5
    st = server.stats()
    assert st["submitted"] == 5 and st["queued"] == 5 and st["completed"] == 0
    assert server.poll(ids[0])["state"] == mg.JOB_QUEUED
    assert server.cancel(ids[1])
    assert not server.cancel(ids[1])  # only queued jobs can be cancelled
    assert server.poll(ids[1])["state"] == mg.JOB_CANCELLED
    assert server.stats()["queued"] == 4 and server.stats()["cancelled"] == 1
    with pytest.raises(TimeoutError):
        server.wait(ids[0], timeout=0.05)
    assert server.release(ids[1])
    with pytest.raises(mg.MGError):
        server.poll(ids[1])


def test_refuses_jobs_over_a_slot_budget(mg, server):
    # 1 GB per slot: an R-MAT of scale 24 needs far more
    with pytest.raises(mg.MGError) as e:
        server.submit(mg.gen_params("rmat", scale=24))
    assert e.value.status == 3
    with pytest.raises(mg.MGError):
        server.submit(mg.gen_params("sbm", n=10, blocks=20))
    with pytest.raises(mg.MGError):
        server.submit(mg.gen_params("sbm", n=100, blocks=4), precision="fp64", version=7)


def test_csr_jobs_are_copied(mg, server):
    import numpy as np

    off = np.array([0, 1, 2], np.uint64)
    cols = np.array([1, 0], np.uint32)
    jid = server.submit_csr(2, off, cols, keep_assignment=True)
    off[:] = 0  # the server holds its own copy
    assert server.poll(jid)["state"] == mg.JOB_QUEUED


def test_stop_cancels_queued(mg):
    if cuda_available():
        pytest.skip("host-only check")
    s = mg.Server(slots=1, hbm_budget_bytes=10**9)
    jid = s.submit(mg.gen_params("sbm", n=2000, blocks=8))
    s.stop()
    s.stop()  # idempotent
    del jid
