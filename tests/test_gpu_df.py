"""GPU parity of the density-fitting sweep (cintx_plan_int3c2e_screened over an optimizer holding
only orbital pairs): the screened tuple set against Schwarz bounds from the oracle, and the
int3c2e_sph blocks against the oracle (all of them on water3+aux, a seeded sample per chunk on
mol40+aux, which has auxiliary shells of higher l than every orbital shell: swapped classes)."""
import numpy as np
import pytest

from conftest import close
from cintx_b200 import molecules as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cx():
    import cintx_b200
    return cintx_b200


@pytest.fixture(scope="module")
def orc():
    from oracle import Restatement
    return Restatement()


def _block_sizes(mol, tuples):
    ls = mol.bas[:, 1]
    return np.prod([2 * ls[tuples[:, c]] + 1 for c in range(3)], axis=0)


def _sweep(cx, mol, norb, cutoff, max_chunk):
    import torch
    opt = cx.Optimizer(mol.atm, mol.bas, mol.env, pair_shells=norb)
    plan = cx.Plan.screened_3c(opt, norb, cutoff=cutoff, max_chunk_doubles=max_chunk)
    st = plan.stats
    buf = torch.empty(st.max_chunk_doubles, dtype=torch.float64, device="cuda")
    chunks = []
    for c in range(st.nchunks):
        plan.execute(buf.data_ptr(), chunk=c, stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        q = plan.chunk_quartets(c)
        assert (q[:, 3] == -1).all()
        chunks.append((q[:, :3].copy(), buf[:plan.chunk_size(c)].cpu().numpy()))
    return opt, plan, chunks


def test_df_sweep_water3_every_block(cx, orc):
    base = M.water_like()
    mol = M.with_aux(base)
    norb = base.nbas
    opt, plan, chunks = _sweep(cx, mol, norb, 1e-12, 1 << 14)
    assert plan.stats.nchunks > 1
    # Schwarz factors from the oracle
    qab = {}
    for a in range(norb):
        for b in range(a + 1):
            v, _ = orc.int2e((a, b, a, b), mol)
            qab[(a, b)] = np.sqrt(np.abs(v).max())
    qk = {k: np.sqrt(np.abs(orc.int2c2e((k, k), mol)[0]).max()) for k in range(norb, mol.nbas)}
    seen = set()
    for tuples, out in chunks:
        sizes = _block_sizes(mol, tuples)
        offs = np.concatenate([[0], np.cumsum(sizes)])
        assert offs[-1] == out.size
        for i, (a, b, k) in enumerate(tuples):
            assert a < norb and b < norb and k >= norb
            key = (max(a, b), min(a, b), k)
            assert key not in seen
            seen.add(key)
            bound = qab[key[:2]] * qk[k]
            assert bound >= 1e-12 * (1 - 1e-9)
            ref, _ = orc.int3c2e((a, b, k), mol)
            assert close(out[offs[i]:offs[i + 1]], ref), (a, b, k)
    expect = {(a, b, k) for (a, b), q in qab.items() for k, r in qk.items() if q * r >= 1e-12 * (1 + 1e-9)}
    assert expect <= seen
    assert plan.stats.nquartets == len(seen)
    plan.close()
    opt.close()


def test_df_sweep_mol40_sampled_blocks_and_swapped_classes(cx, orc):
    base = M.mol40()
    mol = M.with_aux(base)
    norb = base.nbas
    opt, plan, chunks = _sweep(cx, mol, norb, 1e-12, 1 << 26)
    rng = np.random.default_rng(21)
    ls = mol.bas[:, 1]
    swapped = 0
    for tuples, out in chunks:
        sizes = _block_sizes(mol, tuples)
        offs = np.concatenate([[0], np.cumsum(sizes)])
        pick = rng.choice(len(tuples), size=min(250, len(tuples)), replace=False)
        hi = np.where(ls[tuples[:, 2]] > ls[tuples[:, 0]])[0]
        pick = np.concatenate([pick, hi[:40]])
        for i in pick:
            a, b, k = tuples[i]
            swapped += ls[k] > ls[a]
            ref, _ = orc.int3c2e((a, b, k), mol)
            assert close(out[offs[i]:offs[i + 1]], ref), (a, b, k)
    assert swapped > 0
    plan.close()
    opt.close()


def test_pair_limited_optimizer_rejects_foreign_pairs(cx):
    base = M.water_like()
    mol = M.with_aux(base)
    with cx.Optimizer(mol.atm, mol.bas, mol.env, pair_shells=base.nbas) as opt:
        with pytest.raises(cx.CintxError):
            cx.Plan.shells(opt, cx.INT2E, np.array([[base.nbas, 0, 0, 0]], dtype=np.int32))
        p = cx.Plan.shells(opt, cx.INT3C2E, np.array([[1, 0, base.nbas + 3]], dtype=np.int32))
        p.close()
