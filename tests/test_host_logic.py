"""Host-side logic that needs no GPU: argument validation of the C ABI, the workload
definitions, and the replica plumbing of bench.py over gloo (world size 2)."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

from exfemus_b200 import _lib, workloads


def test_bad_mesh_descriptor_is_rejected_before_any_device_call():
    L = _lib.load()
    d = _lib.ExfMeshDesc()
    d.dim, d.nlev = 4, 3
    h = C.c_void_p()
    assert L.exf_mesh_create(C.byref(d), C.byref(h)) == _lib.EXF_ERR_ARG
    assert b"bad descriptor" in L.exf_last_error()
    d.dim, d.nlev = 2, 0
    assert L.exf_mesh_create(C.byref(d), C.byref(h)) == _lib.EXF_ERR_ARG


def test_null_handles_return_status():
    L = _lib.load()
    n = C.c_int()
    assert L.exf_sys_ndof(None, 0, C.byref(n)) == _lib.EXF_ERR_ARG
    assert L.exf_mg_solve(None, None, None) == _lib.EXF_ERR_ARG
    assert L.exf_gen_mat_rhs(None, None, 0, 1) == _lib.EXF_ERR_ARG
    assert L.exf_sys_destroy(None) == _lib.EXF_OK


def test_workload_sizes_and_sources():
    w = workloads.WORKLOADS
    assert w["channel3d"]["n0"] == (8, 2, 2) and w["channel3d"]["nlev"] == 4
    assert w["cavity2d"]["nlev"] == 6 and w["bouss2d"]["nlev"] == 7
    q = workloads.heat_source(1024, seed=0)
    assert q.shape == (1024,) and q.min() >= 1.0 and q.max() < 1.1
    ln = workloads.lognormal_source(65536, seed=0)
    assert abs(np.log(ln).std() - 0.5) < 0.01
    s = np.linspace(-1, 1, 7)
    assert np.allclose(workloads.legendre(2, s), 0.5 * (3 * s * s - 1))
    ns, t = workloads.bouss_phys(dict(ra=1e5, pr=0.71))
    assert abs(ns["inv_re"] - np.sqrt(0.71 / 1e5)) < 1e-15
    assert abs(t["inv_re"] * t["inv_prdl"] - 1 / np.sqrt(1e5 * 0.71)) < 1e-15


def test_bench_top_wall_weights_and_flop_count():
    """Simpson weights of the wall y = 1 integrate 1 and x^2 exactly on a quad9 mesh
    row; the per-element flop count of the assembly is the stated sum of its loops."""
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    xs = np.linspace(0.0, 1.0, 9)
    x = np.concatenate([xs, xs])
    y = np.concatenate([np.ones(9), np.zeros(9)])
    w = bench.top_wall_weights((x, y))
    assert abs(w.sum() - 1.0) < 1e-15
    assert abs(w @ x ** 2 - 1.0 / 3.0) < 1e-15
    assert np.all(w[9:] == 0)
    assert bench.ASM_FLOPS_HEX27_NS == 729 * 27 * 47 + 216 * 27 * 7 + 2 * 27 * 27 * 9 * 2 + 3 * 27 * 27 * 2


def test_bouss_pseudo_time_step():
    ns, t = workloads.bouss_phys(workloads.WORKLOADS["bouss2d"])
    assert ns["inv_dt"] == 1.0 and t["inv_dt"] == 1.0
    ns0, _ = workloads.bouss_phys(dict(ra=1e5, pr=0.71))
    assert ns0["inv_dt"] == 0.0


def _replica_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    ws, r, local = bench.dist_setup("gloo")
    v = bench.max_over_ranks(ws, float(rank + 1), device="cpu")
    bench.barrier(ws)
    import torch.distributed as dist
    dist.destroy_process_group()
    out.put((r, v))


def test_bench_replica_max_over_ranks_gloo():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29000 + os.getpid() % 1000
    ps = [ctx.Process(target=_replica_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert res == [(0, 2.0), (1, 2.0)]
