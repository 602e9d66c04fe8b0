"""GPU tests of the serving loop: jobs submitted from several threads while
others run are batched continuously, batches of different slots overlap on
the GPU, and every job's result is the one the single-graph path gives for
its graph alone (bit-exact: the graphs have integral weights)."""
import threading
import time

import numpy as np
import pytest

from conftest import ring_of_cliques, two_cliques

pytestmark = pytest.mark.gpu


def _alone(ctx, mg, job):
    if job.kind == mg.GEN_SBM:
        g = ctx.generate_sbm(job.n, job.blocks, job.mean_degree, job.intra_frac, job.seed)
    else:
        g = ctx.generate_rmat(job.scale, job.edge_factor, job.a, job.b, job.c, job.seed)
    r = g.louvain()
    g.close()
    return r


def _same(info, ref, assignment=None):
    assert info["state"] == 2, info
    assert info["modularity"] == ref["modularity"]
    assert info["communities"] == ref["communities"]
    assert info["phases"] == ref["phases"] and info["levels"] == ref["levels"]
    assert info["iterations"] == ref["iterations"]
    if assignment is not None:
        assert (assignment == ref["assignment"]).all()


def test_continuous_batching_matches_single_runs(O, ctx, mg):
    rng = np.random.default_rng(3)
    jobs = [mg.gen_params("rmat", scale=17, seed=31)]  # a long job first
    for i in range(23):
        if i % 3 == 0:
            jobs.append(mg.gen_params("rmat", scale=int(rng.integers(10, 15)), seed=100 + i))
        else:
            n = int(np.exp(rng.uniform(np.log(1000), np.log(60000))))
            jobs.append(mg.gen_params("sbm", n=n, blocks=int(rng.integers(4, 64)),
                                      mean_degree=float(rng.uniform(8, 32)), intra_frac=float(rng.uniform(0.7, 0.9)),
                                      seed=200 + i))
    with mg.Server(slots=3, hbm_budget_bytes=60 * 10**9, max_batch_jobs=6) as srv:
        ids = [None] * len(jobs)
        ids[0] = srv.submit(jobs[0], keep_assignment=True)
        time.sleep(0.05)

        def producer(lo, hi):
            for i in range(lo, hi):
                ids[i] = srv.submit(jobs[i], keep_assignment=(i % 2 == 0))
                if i % 4 == 0:
                    time.sleep(0.02)

        ts = [threading.Thread(target=producer, args=(1, 12)), threading.Thread(target=producer, args=(12, 24))]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        infos = [srv.wait(j, timeout=600) for j in ids]
        st = srv.stats()
        for i, (job, info) in enumerate(zip(jobs, infos)):
            ref = _alone(ctx, mg, job)
            a = srv.assignment(ids[i], info["n"]) if i % 2 == 0 else None
            _same(info, ref, a)
        assert st["completed"] == len(jobs) and st["failed"] == 0
        assert st["batches"] >= 3
        assert max(i["batch_jobs"] for i in infos) > 1
        # batches of different slots overlapped in time
        span = {}
        for i in infos:
            lo, hi = span.get(i["batch"], (i["started_s"], i["finished_s"]))
            span[i["batch"]] = (min(lo, i["started_s"]), max(hi, i["finished_s"]))
        iv = sorted(span.values())
        assert any(iv[k + 1][0] < iv[k][1] for k in range(len(iv) - 1))
        assert 0 < st["p50_latency_s"] <= st["p99_latency_s"] <= st["max_latency_s"]


def test_csr_jobs_and_weights(O, ctx, mg):
    gs = [O.csr_from_pairs(*two_cliques()), O.csr_from_pairs(*ring_of_cliques()),
          O.gen_sbm(3000, 8, 12.0, 0.8, seed=5)]
    w = np.arange(gs[2].nnz) % 1 + 2.0  # uniform weight 2: integral, not unit
    with mg.Server(slots=2, hbm_budget_bytes=8 * 10**9) as srv:
        ids = [srv.submit_csr(g.n, g.offsets, g.cols, keep_assignment=True) for g in gs[:2]]
        ids.append(srv.submit_csr(gs[2].n, gs[2].offsets, gs[2].cols, w, keep_assignment=True))
        for jid, g, ww in zip(ids, gs, [None, None, w]):
            info = srv.wait(jid, timeout=300)
            ref = O.louvain(type(g)(g.n, g.offsets, g.cols, ww))
            _same(info, ref, srv.assignment(jid, info["n"]))
