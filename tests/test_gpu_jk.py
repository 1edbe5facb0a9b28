"""GPU check of the Coulomb/exchange build over a unique-quartet sweep (cintx_plan_jk) against a
dense ERI tensor assembled from the oracle: J = sum_kl (ij|kl) D_kl, K = sum_jl (ij|kl) D_jl.
Tolerance: 1e-8 of the largest element; each element sums thousands of integrals that individually
meet the parity rule (1e-12 absolute or 1e-10 relative).
"""
import itertools

import numpy as np
import pytest

from cintx_b200 import molecules as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cx():
    import cintx_b200
    return cintx_b200


def _dense_eri(orc, mol, sph):
    loc = mol.ao_loc(cart=not sph)
    n = int(loc[-1])
    quartets = np.array(list(itertools.product(range(mol.nbas), repeat=4)), dtype=np.int32)
    vals, offs = orc.int2e_batch(quartets, mol, sph=sph)
    eri = np.zeros((n, n, n, n))
    for q, (a, b, c, d) in enumerate(quartets):
        ni, nj, nk, nl = (int(loc[s + 1] - loc[s]) for s in (a, b, c, d))
        blk = vals[offs[q]:offs[q] + ni * nj * nk * nl]
        eri[loc[a]:loc[a + 1], loc[b]:loc[b + 1], loc[c]:loc[c + 1], loc[d]:loc[d + 1]] = \
            blk.reshape(nl, nk, nj, ni).transpose(3, 2, 1, 0)
    return eri, n


@pytest.mark.parametrize("name,sph", [("water3", True), ("jk4", True), ("jk4", False)])
def test_jk_matches_dense_eri(cx, name, sph):
    import torch
    from oracle import Restatement
    orc = Restatement()
    mol = M.water_like() if name == "water3" else M.random_molecule("jk4", 9, 4, 5.0, with_f=True)
    eri, n = _dense_eri(orc, mol, sph)
    rng = np.random.default_rng(5)
    D = rng.normal(size=(n, n))
    D = D + D.T
    J = np.einsum("ijkl,kl->ij", eri, D)
    K = np.einsum("ijkl,jl->ik", eri, D)
    with cx.Optimizer(mol.atm, mol.bas, mol.env) as opt:
        plan = cx.Plan.screened(opt, 1e-14, sph=sph, max_chunk_doubles=1 << 12)
        assert plan.stats.nchunks > 1
        d = torch.tensor(D, device="cuda")
        vj = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
        vk = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
        s = torch.cuda.current_stream()
        plan.jk(d.data_ptr(), n, vj.data_ptr(), vk.data_ptr(), stream=s.cuda_stream)
        s.synchronize()
        vj, vk = vj.cpu().numpy(), vk.cpu().numpy()
        assert np.abs(vj - J).max() <= 1e-8 * np.abs(J).max(), np.abs(vj - J).max()
        assert np.abs(vk - K).max() <= 1e-8 * np.abs(K).max(), np.abs(vk - K).max()
        # J only: the exchange output is skipped
        vj2 = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        plan.jk(d.data_ptr(), n, vj2.data_ptr(), 0, stream=s.cuda_stream)
        s.synchronize()
        assert np.allclose(vj2.cpu().numpy(), vj, rtol=0, atol=1e-12 * np.abs(J).max())
        with pytest.raises(cx.CintxError):
            plan.jk(d.data_ptr(), n + 1, vj2.data_ptr(), 0, stream=s.cuda_stream)
        plan.close()


@pytest.mark.parametrize("name", ["water3", "jk4"])
def test_s8_packed_tensor_matches_dense_eri(cx, name):
    """cintx_plan_execute_s8: (1) the scatter is exact: every slot equals the plan's own block
    element placed there by a numpy scatter of the chunk outputs (to the last bits where two
    elements share a slot); (2) every canonical slot
    (p >= q, r >= s, pq >= rs) against the dense oracle tensor within 1e-9 of its largest element
    (the oracle evaluates each permutation of a quartet independently)."""
    import torch
    from oracle import Restatement
    orc = Restatement()
    mol = M.water_like() if name == "water3" else M.random_molecule("jk4", 9, 4, 5.0, with_f=True)
    eri, n = _dense_eri(orc, mol, True)
    npair = n * (n + 1) // 2
    loc = mol.ao_loc()
    with cx.Optimizer(mol.atm, mol.bas, mol.env) as opt:
        plan = cx.Plan.screened(opt, 1e-14, sph=True, max_chunk_doubles=1 << 12)
        buf = torch.full((npair * (npair + 1) // 2,), float("nan"), dtype=torch.float64, device="cuda")
        s = torch.cuda.current_stream()
        plan.execute_s8(buf.data_ptr(), buf.numel(), stream=s.cuda_stream)
        s.synchronize()
        got = buf.cpu().numpy()
        # numpy scatter of the same sweep's blocks
        mine = np.zeros_like(got)
        ring = torch.empty(plan.stats.max_chunk_doubles, dtype=torch.float64, device="cuda")
        for c in range(plan.stats.nchunks):
            plan.execute(ring.data_ptr(), chunk=c, stream=s.cuda_stream)
            s.synchronize()
            vals = ring[:plan.chunk_size(c)].cpu().numpy()
            off = 0
            for a, b, cc, d in plan.chunk_quartets(c):
                ni, nj, nk, nl = (int(loc[x + 1] - loc[x]) for x in (a, b, cc, d))
                blk = vals[off:off + ni * nj * nk * nl].reshape(nl, nk, nj, ni)
                off += blk.size
                L, K, J, I = np.meshgrid(np.arange(nl) + loc[d], np.arange(nk) + loc[cc], np.arange(nj) + loc[b],
                                         np.arange(ni) + loc[a], indexing="ij")
                pq = np.where(I >= J, I * (I + 1) // 2 + J, J * (J + 1) // 2 + I)
                rs = np.where(K >= L, K * (K + 1) // 2 + L, L * (L + 1) // 2 + K)
                idx = np.where(pq >= rs, pq * (pq + 1) // 2 + rs, rs * (rs + 1) // 2 + pq)
                mine[idx.ravel()] = blk.ravel()
        with pytest.raises(cx.CintxError):
            plan.execute_s8(buf.data_ptr(), buf.numel() - 1, stream=s.cuda_stream)
        plan.close()
    assert np.isfinite(got).all()
    # slots a diagonal block fills twice ((ij|kl) and (ji|kl)) hold either of two equal elements
    # computed separately (they differ in the last bits)
    assert np.all(np.abs(got - mine) <= 1e-12 * np.abs(mine) + 1e-14), np.abs(got - mine).max()
    p, q = np.tril_indices(n)
    ref = eri[p[:, None], q[:, None], p[None, :], q[None, :]]  # [pq, rs]
    ii, jj = np.tril_indices(npair)
    want = ref[ii, jj]
    assert np.abs(got - want).max() <= 1e-9 * np.abs(want).max(), np.abs(got - want).max()


@pytest.mark.parametrize("name", ["water3", "jk4"])
def test_s1_and_s4_tensors_match_dense_eri(cx, name):
    """cintx_plan_execute_ao with aosym 1 (every index order of every quartet, nao^4) and aosym 4
    (the pair-pair matrix), slot by slot against the dense oracle tensor (1e-9 of its largest
    element, as for s8) and against each other; a short buffer is rejected."""
    import torch
    from oracle import Restatement
    orc = Restatement()
    mol = M.water_like() if name == "water3" else M.random_molecule("jk4", 9, 4, 5.0, with_f=True)
    eri, n = _dense_eri(orc, mol, True)
    npair = n * (n + 1) // 2
    assert np.array_equal(cx.ao_loc(mol.bas, True), mol.ao_loc())
    tol = 1e-9 * np.abs(eri).max()
    with cx.Optimizer(mol.atm, mol.bas, mol.env) as opt:
        plan = cx.Plan.screened(opt, 1e-14, sph=True, max_chunk_doubles=1 << 12)
        s = torch.cuda.current_stream()
        b1 = torch.full((n ** 4,), float("nan"), dtype=torch.float64, device="cuda")
        plan.execute_ao(b1.data_ptr(), b1.numel(), aosym=1, stream=s.cuda_stream)
        b4 = torch.full((npair * npair,), float("nan"), dtype=torch.float64, device="cuda")
        plan.execute_ao(b4.data_ptr(), b4.numel(), aosym=4, stream=s.cuda_stream)
        s.synchronize()
        with pytest.raises(cx.CintxError):
            plan.execute_ao(b4.data_ptr(), b4.numel() - 1, aosym=4, stream=s.cuda_stream)
        with pytest.raises(cx.CintxError):
            plan.execute_ao(b4.data_ptr(), b4.numel(), aosym=2, stream=s.cuda_stream)
        plan.close()
    g1 = b1.cpu().numpy().reshape(n, n, n, n)
    g4 = b4.cpu().numpy().reshape(npair, npair)
    assert np.isfinite(g1).all() and np.isfinite(g4).all()
    assert np.abs(g1 - eri).max() <= tol, np.abs(g1 - eri).max()
    p, q = np.tril_indices(n)
    assert np.abs(g4 - eri[p[:, None], q[:, None], p[None, :], q[None, :]]).max() <= tol
    # the same block elements fill both (a diagonal shell pair reaches a slot from two elements
    # computed separately, equal to the last bits)
    assert np.abs(g4 - g1[p[:, None], q[:, None], p[None, :], q[None, :]]).max() <= 1e-13 * np.abs(eri).max()
