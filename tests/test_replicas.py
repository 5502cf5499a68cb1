"""The replica plumbing of the multi-GPU bench with two gloo ranks on CPU:
the maximum over ranks, barriers, and a rank that never arrives ending the
other with an error (short process-group timeout) instead of a hang."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, mode, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from ed_solver_b200.replicas import Replicas
    try:
        rep = Replicas("gloo", timeout_s=5.0 if mode == "absent" else 60.0)
        if mode == "absent" and rank == 1:
            q.put((rank, "left"))
            q.close()
            q.join_thread()
            os._exit(0)                      # leaves between steps, no collective in flight
        rep.barrier()
        m = rep.max(1.5 + rank)
        q.put((rank, m))
        rep.close()
    except Exception as e:                   # the remaining rank sees the timeout as an error
        q.put((rank, "error:" + type(e).__name__))
    q.close()
    q.join_thread()


def _run(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    out = {}
    while not q.empty():
        r, v = q.get()
        out[r] = v
    for p in procs:
        if p.is_alive():
            p.kill()
    return out


def test_max_over_two_gloo_ranks():
    out = _run("normal")
    assert out == {0: 2.5, 1: 2.5}


def test_a_rank_that_never_arrives_ends_the_other_with_an_error():
    out = _run("absent")
    assert out[1] == "left"
    assert isinstance(out.get(0), str) and out[0].startswith("error:")
