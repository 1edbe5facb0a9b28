"""GPU tests of the learned Rys-root initializer (cintx_rysnet_* / cintx_rys_learned_batch):
the device training kernel's gradient against the CPU oracle, training, the refined roots
against the FP64 oracle at the 1e-14 relative bar, the fallback contract, and what the trained
network gains over the same refinement started without it."""
import numpy as np
import pytest

from oracle import rysnet_oracle as R

pytestmark = pytest.mark.gpu

XMAX = [0, 40, 52, 60, 64, 72, 76, 84, 92, 100]


@pytest.fixture(scope="module")
def cx():
    import cintx_b200
    return cintx_b200


@pytest.fixture(scope="module")
def trained(cx):
    net = cx.RysNet(seed=0)
    hist = net.train(nsamples=5_000_000, n_lo=5, n_hi=9, epochs=40, batch=16384, lr=3e-3, seed=11)
    return net, hist


def test_device_gradient_matches_cpu_oracle(cx):
    net = cx.RysNet(seed=5)
    feat, tgt, nr, x = net.samples(1000, 1, 9, seed=2)
    assert ((nr >= 1) & (nr <= 9)).all() and (x > 0).all()
    np.testing.assert_allclose(feat, R.features(nr, x), rtol=1e-6, atol=1e-6)
    loss, g = net.loss_grad(feat, tgt, nr)
    loss_ref, g_ref = R.loss_grad(net.params.astype(np.float64), feat, tgt, nr)
    assert abs(loss - loss_ref) <= 1e-5 * loss_ref
    scale = np.abs(g_ref).max()
    assert np.abs(g - g_ref).max() <= 2e-4 * scale, np.abs(g - g_ref).max() / scale


def test_training_reduces_loss_and_guess_is_close(cx, trained):
    net, hist = trained
    assert np.isfinite(hist).all() and hist[-1] < 0.02 * hist[0], hist
    rng = np.random.default_rng(9)
    for n in (5, 7, 9):
        x = np.exp(rng.uniform(np.log(1e-7), np.log(XMAX[n] - 1e-3), size=400))
        t2g, wg, st, _ = net.roots(n, x, mode=2)
        t2, w = cx.rys_t2_batch(n, x)  # the plain (table) path judges the network's residual
        assert (st == 3).all()
        assert np.median(np.abs(t2g / t2 - 1)) < 5e-3
        assert np.median(np.abs(wg / w - 1)) < 2e-2


def test_refined_roots_meet_1e14_and_fallbacks_use_the_table(cx, trained):
    from oracle import Restatement
    orc = Restatement()
    net, _ = trained
    rng = np.random.default_rng(10)
    for n in (5, 6, 7, 8, 9):
        lo = np.exp(rng.uniform(np.log(1e-7), np.log(50.0), size=140))
        hi = rng.uniform(50.0, 3000.0, size=60)
        x = np.concatenate([lo, hi, [0.0, 1e-7, XMAX[n] - 1e-9, float(XMAX[n])]])
        t2, w, st, it = net.roots(n, x, mode=0)
        assert set(np.unique(st)) <= {0, 1, 2}
        assert ((x >= XMAX[n]) == (st == 2)).all()
        tab_t2, tab_w = cx.rys_t2_batch(n, x)
        fb = st == 1
        assert np.array_equal(t2[fb], tab_t2[fb]) and np.array_equal(w[fb], tab_w[fb])
        assert fb.mean() <= 0.01, (n, fb.mean())
        for k in np.where(st == 0)[0]:
            rt, rw = orc.rys_t2(n, x[k])
            assert np.abs(t2[k] / rt - 1).max() <= 1e-14, (n, x[k], np.abs(t2[k] / rt - 1).max())
            assert np.abs(w[k] / rw - 1).max() <= 1e-14, (n, x[k], np.abs(w[k] / rw - 1).max())


def test_network_gain_over_refinement_without_it(cx, trained):
    """Same refinement, started from the network's guess or from the x = 0 roots (the method
    without the network): the network's start leaves far fewer points to the table fallback."""
    net, _ = trained
    rng = np.random.default_rng(12)
    fb = {0: 0, 1: 0}
    total = 0
    for n in (5, 6, 7, 8, 9):
        x = np.exp(rng.uniform(np.log(1e-7), np.log(XMAX[n] - 1e-3), size=500))
        total += x.size
        for mode in (0, 1):
            fb[mode] += int((net.roots(n, x, mode=mode)[2] == 1).sum())
    assert fb[0] <= 0.002 * total and fb[1] >= 10 * max(fb[0], 1), fb


def _g_quartets(mol, n, seed):
    """Seeded quartets containing a g shell whose class needs 5..9 roots (sum of l >= 8)."""
    rng = np.random.default_rng(seed)
    ls = mol.bas[:, 1]
    g = np.where(ls == 4)[0]
    out = []
    while len(out) < n:
        q = rng.integers(0, mol.nbas, size=4)
        q[rng.integers(0, 4)] = rng.choice(g)
        if ls[q].sum() >= 8:
            out.append(q)
    return np.array(out, dtype=np.int32)


def test_learned_roots_feed_the_integrals(cx, trained):
    """g-shell int2e quartets evaluated by the ERI kernels with roots from the learned
    initializer + refinement, against the same kernels with table roots and against libcint."""
    from conftest import close
    from cintx_b200 import molecules as M
    from oracle import RefLibcint
    net, _ = trained
    mol = M.mol20_g()
    quartets = _g_quartets(mol, 400, 31)
    with cx.Optimizer(mol.atm, mol.bas, mol.env) as opt:
        p_tab = cx.Plan.shells(opt, cx.INT2E, quartets)
        out_tab = p_tab.execute_host(np.zeros(p_tab.stats.nintegrals))
        p_lrn = cx.Plan.shells(opt, cx.INT2E, quartets)
        fb, npt = p_lrn.use_learned_roots(net)
        out_lrn = p_lrn.execute_host(np.zeros(p_lrn.stats.nintegrals))
        assert npt > 0 and fb <= 0.01 * npt, (fb, npt)
        assert close(out_lrn, out_tab), np.abs(out_lrn - out_tab).max()
        assert p_lrn.use_learned_roots(None) == (0, 0)  # back to the table: identical output
        assert np.array_equal(p_lrn.execute_host(np.zeros(p_lrn.stats.nintegrals)), out_tab)
        offs = p_lrn.offsets
        if RefLibcint.available():
            ref = RefLibcint()
            for k in range(0, len(quartets), 8):
                r, _ = ref.int2e(quartets[k], mol)
                assert close(out_lrn[offs[k]:offs[k] + r.size], r), quartets[k]
        p_tab.close()
        p_lrn.close()
