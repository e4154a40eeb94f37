"""Host-side logic of batching and serving (CPU): request streams, the
admission ledger, rank sharding and the max-over-ranks timing reduction
over a 2-rank gloo group."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def test_poisson_stream_seeded():
    from warpflow.serve import poisson_stream
    a = poisson_stream(count=50, seed=3)
    b = poisson_stream(count=50, seed=3)
    assert [(r.n, r.n_steps, r.arrival) for r in a] == [(r.n, r.n_steps, r.arrival) for r in b]
    assert all(32 <= r.n <= 128 and r.n % 16 == 0 for r in a)
    assert all(100 <= r.n_steps <= 2000 for r in a)
    arr = [r.arrival for r in a]
    assert arr == sorted(arr)
    # mean inter-arrival near 1/20 s
    assert 0.02 < arr[-1] / len(arr) < 0.09


def test_levels_for_keeps_coarse_small():
    from warpflow.serve import levels_for
    assert levels_for(80) == 3
    assert levels_for(96) == 3       # coarse 24, with an operator
    assert levels_for(112) == 3      # coarse 28 (14 would be slower)
    assert levels_for(128) == 4      # coarse 16 with an operator, not 32 by sweeps
    assert levels_for(256) == 5      # coarse 16
    assert (256 >> (levels_for(256) - 1)) <= 32


def test_admission_fifo_budget():
    from warpflow.serve import Admission, Request, case_bytes, operator_bytes
    b32, op = case_bytes(32), operator_bytes(32)
    adm = Admission(budget_bytes=int(2.5 * b32) + op)
    reqs = [Request(i, 32, 400.0, 1.0, 10, arrival=0.1 * i) for i in range(4)]
    for r in reqs:
        adm.submit(r)
    assert adm.admit(0.05) == [reqs[0]]
    got = adm.admit(1.0)
    assert got == [reqs[1]]              # third does not fit
    assert adm.used == 2 * b32 + op <= adm.budget
    adm.release(0)
    assert adm.admit(1.0) == [reqs[2]]   # freed memory admits the next, in order
    assert adm.peak <= adm.budget


def test_admission_no_overtaking():
    from warpflow.serve import Admission, Request, case_bytes, operator_bytes
    big, small = case_bytes(128), case_bytes(32)
    adm = Admission(budget_bytes=big + small // 2 + operator_bytes(128) + operator_bytes(32))
    adm.submit(Request(0, 32, 400.0, 1.0, 10, arrival=0.0))
    adm.submit(Request(1, 128, 400.0, 1.0, 10, arrival=0.1))
    adm.submit(Request(2, 32, 400.0, 1.0, 10, arrival=0.2))
    assert [r.rid for r in adm.admit(1.0)] == [0]   # 1 blocks 2 (FIFO)
    adm.release(0)
    assert [r.rid for r in adm.admit(1.0)] == [1]


def test_operator_bytes_and_shared_charge():
    """The shared coarse-level operator (220 representative columns of 4000
    entries plus its integer table at 20^3) is charged once per kind."""
    from warpflow.serve import Admission, Request, case_bytes, operator_bytes
    op = operator_bytes(80, 3, "fp64")
    assert op == 220 * 4000 * 8 + (220 + 4000) * 4
    assert operator_bytes(72, 3, "fp64") == 0          # coarsest 18: sweeps
    adm = Admission(budget_bytes=2 * case_bytes(80, 3, "fp64") + op)
    for rid in range(3):
        adm.submit(Request(rid, 80, 400.0, 1.0, 10, arrival=0.0, precision="fp64"))
    got = [r.rid for r in adm.admit(1.0)]
    assert got == [0, 1]
    assert adm.used == 2 * case_bytes(80, 3, "fp64") + op
    adm.release(0)
    assert [r.rid for r in adm.admit(1.0)] == [2]
    assert adm.used == 2 * case_bytes(80, 3, "fp64") + op   # still charged once


def test_idle_solvers_reused_and_evicted():
    """A finished case's solver stays charged as idle and serves the next
    request of its kind with no new bytes; a request of another kind that
    does not fit evicts idle solvers (largest first)."""
    from warpflow.serve import Admission, Request, case_bytes, operator_bytes
    k32, k48 = (32, 3, "mixed"), (48, 3, "mixed")
    b32, b48 = case_bytes(32), case_bytes(48)
    o32, o48 = operator_bytes(32), operator_bytes(48)
    adm = Admission(budget_bytes=b32 + b48 + o32 + o48)
    adm.submit(Request(0, 32, 400.0, 1.0, 5, arrival=0.0))
    assert [r.rid for r in adm.admit(0.0)] == [0] and not adm.reused
    adm.release(0, keep=k32)
    assert adm.idle[k32] == 1 and adm.used == b32 + o32
    adm.submit(Request(1, 32, 700.0, 0.8, 5, arrival=0.1))
    assert [r.rid for r in adm.admit(0.2)] == [1] and adm.reused == {1}
    assert adm.idle[k32] == 0 and adm.used == b32 + o32     # no new bytes
    adm.release(1, keep=k32)
    # two 48^3 cases need the idle 32^3 solver's memory
    adm.submit(Request(2, 48, 400.0, 1.0, 5, arrival=0.3))
    assert [r.rid for r in adm.admit(0.3)] == [2]
    assert adm.evicted == [] and adm.idle[k32] == 1
    adm.submit(Request(3, 48, 400.0, 1.0, 5, arrival=0.4))
    adm.budget = 2 * b48 + o32 + o48
    assert [r.rid for r in adm.admit(0.4)] == [3]
    assert adm.evicted == [k32] and adm.idle[k32] == 0
    assert adm.used == 2 * b48 + o32 + o48 <= adm.budget
    # keep_idle respects the budget
    assert not adm.keep_idle(k32)


def test_admission_rejects_oversize():
    from warpflow.serve import Admission, Request
    adm = Admission(budget_bytes=1000)
    with pytest.raises(ValueError):
        adm.submit(Request(0, 32, 400.0, 1.0, 10, arrival=0.0))


def test_case_bytes_formula():
    from warpflow.serve import case_bytes
    n = 80
    f = 13 * 86 ** 3 * 8
    vol = 82 ** 3 + 42 ** 3 + 22 ** 3
    mg64 = 2 * 8 * vol + 2 * 8 * vol      # phi, rhs + two-array scratch
    mg32 = 2 * 4 * vol + 2 * 4 * vol
    # coarse-operator scratch: 24 permuted copies of the 4000 even cells and
    # 8 slices x 220 representatives x 24 symmetries of partial sums
    sc = 24 * 4000 + 8 * 220 * 24
    cop64, cop32 = sc * 8, sc * 4
    assert 0 <= case_bytes(n, 3, "fp64") - f - mg64 - cop64 < 4096
    assert 0 <= case_bytes(n, 3, "mixed") - f - 2 * 8 * vol - mg32 - cop32 < 4096
    # a coarsest edge without an operator (18) adds no scratch
    n2 = 72
    f2 = 13 * 78 ** 3 * 8
    vol2 = 74 ** 3 + 38 ** 3 + 20 ** 3
    assert 0 <= case_bytes(n2, 3, "fp64") - f2 - 4 * 8 * vol2 < 4096


def test_shard_round_robin():
    from warpflow.dist import shard
    items = list(range(10))
    parts = [shard(items, r, 3) for r in range(3)]
    assert sorted(sum(parts, [])) == items
    assert parts[1] == [1, 4, 7]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from warpflow.dist import max_over_ranks, shard, sum_over_ranks
    mine = shard(range(7), rank, world)
    tmax = max_over_ranks(1.5 + rank)
    cells = sum_over_ranks(sum(mine))
    out[rank] = (tmax, cells, len(mine))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replica_reductions():
    """The N>1 bench path: each rank times its own replica, rank 0 reports
    the max time and the summed work (gloo, world size 2, CPU)."""
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    assert out[0][0] == out[1][0] == 2.5
    assert out[0][1] == out[1][1] == sum(range(7))
    assert out[0][2] + out[1][2] == 7
