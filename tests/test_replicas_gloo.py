"""bench.py's N > 1 path with two ranks on the CPU (gloo).

On the GPU the path runs one independent solve per rank (replicas: the
triangulation has no data exchange) and the ranks only meet to reduce the
timings.  Here each of two gloo ranks takes its own seeded workload, solves
it with the oracle, and the reductions must give the job figure the bench
reports: the points of all ranks over the slowest rank's time."""
import multiprocessing as mp
import os
import socket
import time

import numpy as np


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    from oracle import oracle
    r, w, _ = bench.dist_init("gloo")
    xy, cons = bench.replica_workload(r, scale_points=20000)
    t0 = time.perf_counter()
    rc, tris, adj, cf, _ = oracle.cdt(xy, cons)
    ms = (time.perf_counter() - t0) * 1e3 + 50.0 * r      # rank 1 made slower by a known amount
    total = bench.sum_over_ranks(float(len(xy)), w, "cpu")
    slowest = bench.max_over_ranks(ms, w, "cpu")
    ok, _ = oracle.validate(xy, cons, tris, adj, cf)
    out.put((r, len(xy), ms, total, slowest, bench.job_mpts(total, slowest), rc, ok,
             int(np.asarray(xy, np.int64).sum())))
    bench.dist_done(w)


def test_two_gloo_ranks_reduce_like_the_bench():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, n0, ms0, tot0, slow0, v0, rc0, ok0, h0), (r1, n1, ms1, tot1, slow1, v1, rc1, ok1, h1) = res
    assert (r0, r1) == (0, 1)
    assert rc0 == rc1 == 0 and ok0 and ok1
    assert h0 != h1                                   # each rank has its own instance
    assert tot0 == tot1 == n0 + n1                    # exact points of the job
    assert slow0 == slow1 == max(ms0, ms1)            # the slowest rank's time
    assert abs(v0 - (n0 + n1) / (max(ms0, ms1) * 1e-3) / 1e6) < 1e-9
    assert v0 == v1


def test_replica_workloads_are_seeded_per_rank():
    import bench
    a0, c0 = bench.replica_workload(0, scale_points=20000)
    b0, d0 = bench.replica_workload(0, scale_points=20000)
    a1, _ = bench.replica_workload(1, scale_points=20000)
    assert np.array_equal(a0, b0) and np.array_equal(c0, d0)
    assert not np.array_equal(a0[:1000], a1[:1000])


def test_reference_arm_runs_one_instance_per_thread():
    """The --impl reference leg: every thread solves its own seeded instance
    (reduced here), all of them complete, thread 0's is the headline
    instance, and the step figure is all points over the step."""
    import bench
    runs, desc, (n0, s0) = bench.cpu_oracle_parallel(2, 2, scale_points=30000)
    xy, cons = bench.replica_workload(0, scale_points=30000)
    assert (n0, s0) == (len(xy), len(cons))
    assert len(runs) == 2 and desc.startswith("2 concurrent reduced")
    total = int(desc.split(" points in all")[0].rsplit(" ", 1)[1])
    for v, t in runs:
        assert t > 0 and abs(v - total / t / 1e6) < 1e-9
    assert 1 <= bench.cpu_threads() <= (os.cpu_count() or 1)
