"""CPU: the radial batch sharded over ranks (gloo, world size 2), with the oracle as the per-rank
solver, gives the same records in the same order as one serial pass; the partition covers every
run once and balances the estimated cost."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from dft_b200.radial_shard import partition, run_cost, solve_atoms_sharded

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUNS = [(Z, k) for k in (0, 1) for Z in (1, 2, 3, 5, 7, 8)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_solve(Zs, kinds):
    from oracle.bindings import Port
    p = Port()
    return [p.solve_atom(z, k) for z, k in zip(Zs, kinds)]


def _rank_main(rank, world, port, out_dir):
    import json
    import sys

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        Zs, kinds = [z for z, _ in RUNS], [k for _, k in RUNS]
        res = solve_atoms_sharded(Zs, kinds, solve=_oracle_solve)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump(res, f)
    finally:
        dist.destroy_process_group()


def test_partition_covers_and_balances():
    Zs = list(range(1, 31)) * 2
    for world in (1, 2, 3, 4, 8):
        parts = partition(Zs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(Zs)))
        loads = [sum(run_cost(Zs[i]) for i in p) for p in parts]
        assert max(loads) - min(loads) <= run_cost(30)
    assert partition(Zs, 2) == partition(Zs, 2)  # deterministic
    with pytest.raises(ValueError):
        partition(Zs, 0)


def test_sharded_matches_serial_gloo(tmp_path):
    import json
    Zs, kinds = [z for z, _ in RUNS], [k for _, k in RUNS]
    serial = _oracle_solve(Zs, kinds)
    assert solve_atoms_sharded(Zs, kinds, solve=_oracle_solve) == serial  # no process group: one rank
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    want = json.loads(json.dumps(serial))
    for r in range(2):
        got = json.load(open(tmp_path / f"rank{r}.json"))
        assert got == want


@pytest.mark.gpu
def test_sharded_single_rank_on_gpu(engine):
    Zs, kinds = [z for z, _ in RUNS], [k for _, k in RUNS]
    assert solve_atoms_sharded(Zs, kinds, engine=engine) == engine.solve_atoms(Zs, kinds)
