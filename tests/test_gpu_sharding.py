"""Ranks of a sharded sweep build their plans independently: two processes (spawned, each on
cuda:0, neither waiting for the other) build the 40-atom molecule's screened plan from the same
host arrays and must agree on every chunk, segment and quartet, so that the chunk assignment
(no collective on the data path) covers the sweep exactly once."""
import multiprocessing as mpr

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _build(q):
    import sys
    sys.path.insert(0, ROOT)
    import cintx_b200 as cx
    from cintx_b200 import molecules as M
    from cintx_b200.sharding import plan_digest
    mol = M.mol40()
    with cx.Optimizer(mol.atm, mol.bas, mol.env) as opt:
        plan = cx.Plan.screened(opt, 1e-12, sph=True, max_chunk_doubles=1 << 23)
        q.put(plan_digest(plan, 2))
        plan.close()


def test_two_processes_build_identical_plans_and_shards():
    ctx = mpr.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_build, args=(q,)) for _ in range(2)]
    for p in procs:
        p.start()
    d = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert d[0] == d[1]
    dg = d[0]
    assert len(dg["chunk_sizes"]) >= 4 and sum(dg["chunk_sizes"]) == dg["nintegrals"]
    # the two shards are disjoint, cover every chunk, and their integral counts add up to the sweep
    assert sorted(set(dg["owner"])) == [0, 1]
    assert sum(dg["shard_integrals"]) == dg["nintegrals"]
    assert max(dg["shard_integrals"]) < dg["nintegrals"]
