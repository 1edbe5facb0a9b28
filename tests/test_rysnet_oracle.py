"""CPU checks of the RysNet gradient oracle (oracle/rysnet_oracle.py): its analytic gradient
against central finite differences of its own loss, in float64."""
import numpy as np

from oracle import rysnet_oracle as R


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.normal(scale=0.3, size=R.NPARAM)
    B = 12
    nroots = rng.integers(1, 10, size=B)
    feat = R.features(nroots, np.exp(rng.uniform(np.log(1e-7), np.log(90.0), size=B)))
    tgt = rng.normal(size=(B, R.OUT))
    loss, g = R.loss_grad(p, feat, tgt, nroots)
    assert loss > 0
    idx = rng.choice(R.NPARAM, size=60, replace=False)
    # make sure every parameter block is probed
    starts = np.cumsum([0] + [int(np.prod(s)) for _, s in R.SIZES])[:-1]
    idx = np.unique(np.concatenate([idx, starts, starts + 1]))
    h = 1e-6
    for i in idx:
        e = np.zeros(R.NPARAM)
        e[i] = h
        fd = (R.loss_grad(p + e, feat, tgt, nroots)[0] - R.loss_grad(p - e, feat, tgt, nroots)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-6 * abs(fd), (i, fd, g[i])


def test_oracle_forward_matches_loss_definition():
    rng = np.random.default_rng(4)
    p = rng.normal(scale=0.3, size=R.NPARAM)
    nroots = np.array([1, 5, 9])
    feat = R.features(nroots, [1e-3, 2.0, 80.0])
    y = R.forward(p, feat)
    loss, _ = R.loss_grad(p, feat, y, nroots)  # targets equal to the outputs: zero loss
    assert loss == 0.0
