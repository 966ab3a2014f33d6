"""Multi-rank logic on CPU with gloo, world size 2 (no GPU)."""
import os
import socket

import pytest

from tictac_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dims = [24300, 24300, 42300, 42300, 53100, 53100, 56700, 56700]
        parts = shard.lpt_partition(shard.channel_weights(dims), world)
        mine = parts[rank]
        t = 1.0 + rank  # pretend step time
        tmax = shard.max_over_ranks(dist, t)
        got = shard.gather_to_rank0(dist, {c: complex(c, rank) for c in mine})
        if rank == 0:
            q.put((parts, tmax, got))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_and_gather():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    parts, tmax, got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert tmax == 2.0
    assert sorted(parts[0] + parts[1]) == list(range(8))
    # every channel solved exactly once, loads balanced within one channel's cost
    merged = {}
    for d in got:
        merged.update(d)
    assert sorted(merged) == list(range(8))
    w = shard.channel_weights([24300, 24300, 42300, 42300, 53100, 53100, 56700, 56700])
    loads = [sum(w[i] for i in p) for p in parts]
    assert abs(loads[0] - loads[1]) <= max(w)


def test_lpt_single_rank_and_energy_replicas():
    assert shard.lpt_partition([3.0, 1.0, 2.0], 1) == [[0, 1, 2]]
    assert shard.rank_lab_energies(10.0, 0) == 10.0 and shard.rank_lab_energies(10.0, 3) == 28.0


def test_scan_plan_covers_every_item_once():
    dims = [24300, 24300, 42300, 42300, 53100, 53100, 56700, 56700]
    for world in (1, 2, 3, 8):
        for nE, group in ((2, 2), (18, 4), (5, 2)):
            plans = shard.plan(dims, nE, world, group)
            assert len(plans) == world
            cover = sorted((c, j) for p in plans for c, js in p.items() for j in js)
            assert cover == [(c, j) for c in range(len(dims)) for j in range(nE)]
            loads = [shard.rank_load(p, dims) for p in plans]
            assert max(loads) - min(loads) <= group * max(dims) ** 3


def _orchestration_worker(rank, world, port, q, case, tmpdir):
    # one rank of a sharded run on CPU: the items (channel, energies) this rank
    # owns are solved by the oracle from the reference's fixture inputs, the U
    # arrays gathered on rank 0, assembled in the reference's layout and
    # written as U tables
    import sys

    import torch.distributed as dist

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__))))
    from conftest import load_case

    import harness as oracle
    import tictac_b200 as tt

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g, m = load_case(case)
        Np, Nq = m["Np"], m["Nq"]
        nch = int(g["n_chn"])
        pws = [g[f"pw_c{c}"] for c in range(nch)]
        dims = [pw.shape[0] * Np * Nq for pw in pws]
        nE = len(g["q_idx"])
        plans = shard.plan(dims, nE, world, group=1)
        lay_args = (g["V_unco"], g["V_coup"], g["C_unco"], g["C_coup"], g["e_unco"], g["e_coup"],
                    m["tensor_force"], m["iso"])

        def solve(c, js):
            pw = pws[c]
            lay = oracle.layout(pw, Np, *lay_args)
            A = oracle.build_A(lay, pw.shape[0], Nq, Np, g[f"p123_row_c{c}"], g[f"p123_col_c{c}"],
                               g[f"p123_val_c{c}"])
            G = g[f"G_c{c}"].reshape(nE, -1)[js]
            return oracle.dense_solve(A, G, g["q_idx"][js], oracle.deuterons(pw), Nq, Np)

        mine = shard.run_plan(plans[rank], solve)
        got = shard.gather_to_rank0(dist, mine)
        if rank == 0:
            nd = [len(oracle.deuterons(pw)) for pw in pws]
            U = shard.assemble_U(got, nd, nE)
            run = tt.Run(**m["opts"])
            for c in range(nch):
                run.write_U_table(c, U[c], os.path.join(tmpdir, f"sharded_c{c}.txt"))
                run.write_U_table(c, g[f"U_c{c}"], os.path.join(tmpdir, f"reference_c{c}.txt"))
            run.close()
            q.put((plans, {c: U[c] for c in U}))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_run_gathers_reference_U(world, tmp_path):
    # lo_j1_J3_n8: four channels x two on-shell energies as (channel, energy)
    # items over 2 and 3 gloo ranks; the U gathered on rank 0 must equal the
    # reference's per element, and its U tables must have the reference's
    # headers and line count
    import torch.multiprocessing as mp

    from conftest import load_case, rel_elem

    case = "lo_j1_J3_n8"
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_orchestration_worker, args=(r, world, port, q, case, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    plans, U = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    # the items really were spread over the ranks
    assert sum(1 for p in plans if p) == world
    g, _ = load_case(case)
    for c in range(int(g["n_chn"])):
        assert rel_elem(U[c], g[f"U_c{c}"]) <= 1e-10
        a = (tmp_path / f"sharded_c{c}.txt").read_text().splitlines()
        b = (tmp_path / f"reference_c{c}.txt").read_text().splitlines()
        assert len(a) == len(b) and len(a) > 1
        for la, lb in zip(a, b):
            if la.startswith("#") or not la.strip():
                assert la == lb
