"""The bench's multi-GPU logic on CPU: two gloo ranks (replicas, no data
collective), max-over-ranks timing, whole-job value; the reference arm does
its work on rank 0 only."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist)
    v = bench.replica_value(1000, 20, world, ms)
    out.put((rank, ms, v))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]                 # both ranks see the slowest
    assert res[0][2] == res[1][2] == pytest.approx(2 * 1000 * 20 / 15e-3)


def test_reference_arm_only_on_rank0(capsys):
    class A:
        gpus, steps, warmup = 2, 1, 1
    assert bench.run_reference(A, 1, 2) is None
    assert capsys.readouterr().out == ""


def test_node_step_bytes_is_the_sum_of_the_phases():
    """The whole-step roofline counts, per node-step, the ionic phase, two CN
    half steps (prologue + iterations, predictor passes) and the ECG share."""
    n, nnz = 1000, 15000
    z = nnz / n
    for k, pred in ((4.0, 0), (8.5, 1), (8.5, 2)):
        b = bench.node_step_bytes(n, nnz, k, 4, nstate=19, ne=10, ecg_every=10, cg_predict=pred)
        # the start correction gathered + V saved; x, V, k corrections read, x + k written
        extra = 0 if not pred else (2 + 2 * pred + 3) * 4
        cg = z * 12 + 5 * 4 + extra + k * (z * 8 + 12 * 4)
        assert abs(b - ((2 * 19 * 4 + 16 + 1 + 4 + 4) + 2 * cg + 11 * 4 / 10)) < 1e-9


def test_roofline_traffic_follows_the_cg_kernel():
    """roofline.traffic: the committed ncu bytes of the CG kernel that ran --
    the staged kernel's own entry (measured with predictor 2) for cg_batch 32,
    the gather-width kernels' entry otherwise."""
    import json
    import os
    with open(os.path.join(os.path.dirname(bench.__file__), "profiles", "traffic.json")) as f:
        t = json.load(f)
    st = t["cg_staged"]["predict2_bytes"]
    assert bench._traffic("cg", "surrogate", 5.0, 2, 32) == st["prologue_bytes"] + 5.0 * st["per_iteration_bytes"]
    assert bench._traffic("cg", "surrogate", 5.0, 1, 32) is None          # not captured
    c = t["cg"]
    assert bench._traffic("cg", "surrogate", 5.0, 2, 8) == (c["prologue_bytes"] + c["predict_extra_bytes"]["2"]
                                                             + 5.0 * c["per_iteration_bytes"])
    assert bench._traffic("ionic", "surrogate", 5.0) == t["surrogate"]
