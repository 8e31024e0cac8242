"""The multi-GPU form is replicas only: each rank runs its own workload and only timings and counts cross ranks.
These tests run that host logic as two gloo ranks on the CPU: the job's throughput is every rank's units over the
slowest rank's time, the barrier orders the ranks, and a rank that dies before its reduction makes the other rank's
collective end with an error within the process-group timeout instead of hanging."""
import importlib
import json
import multiprocessing as mp
import os
import socket
import time

import pytest


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, mode, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank))
    rep = importlib.import_module("cuda-wavefront-pathtracer_b200.replicas").Replicas(backend="gloo", timeout_s=10.0)
    res = {"rank": rank, "ws": rep.ws}
    try:
        if mode == "ok":
            units, seconds = (1000.0, 2.0) if rank == 0 else (3000.0, 4.0)
            t0 = time.time()
            if rank == 1:
                time.sleep(0.5)
            rep.barrier()
            res["waited"] = time.time() - t0
            res["throughput"], res["total"], res["slowest"] = rep.throughput(units, seconds)
            rep.close()
        else:   # rank 1 fails before its reduction; rank 0 must get an error, not hang
            if rank == 1:
                os._exit(3)
            t0 = time.time()
            try:
                rep.max(1.0)
                res["error"] = None
            except Exception as e:   # the collective failed: the peer is gone
                res["error"] = type(e).__name__
            res["waited"] = time.time() - t0
    finally:
        with open(out % rank, "w") as f:
            json.dump(res, f)


def _run(tmp_path, mode):
    port = _port()
    out = str(tmp_path / ("r%d_" + mode + ".json"))
    ctx = mp.get_context("spawn")
    ps = [ctx.Process(target=_rank, args=(r, port, mode, out)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
    for p in ps:
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
    res = {}
    for r in range(2):
        if os.path.exists(out % r):
            with open(out % r) as f:
                res[r] = json.load(f)
    return ps, res


def test_job_throughput_is_all_units_over_slowest_rank(tmp_path):
    ps, res = _run(tmp_path, "ok")
    assert all(p.exitcode == 0 for p in ps)
    for r in (0, 1):
        assert res[r]["ws"] == 2
        assert res[r]["total"] == 4000.0 and res[r]["slowest"] == 4.0 and res[r]["throughput"] == 1000.0
    assert res[0]["waited"] >= 0.4   # rank 0 waited at the barrier for the later rank


def test_a_dead_rank_ends_the_collective_with_an_error(tmp_path):
    ps, res = _run(tmp_path, "dead")
    assert ps[1].exitcode == 3
    assert res[0]["error"] is not None and res[0]["waited"] < 60.0


def test_single_process_needs_no_process_group():
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    rep = importlib.import_module("cuda-wavefront-pathtracer_b200.replicas").Replicas()
    assert rep.ws == 1 and rep.dist is None
    assert rep.throughput(10.0, 2.0) == (5.0, 10.0, 2.0)
    rep.close()
