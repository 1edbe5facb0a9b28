"""GPU parity: the CUDA path through the C ABI against the oracle and golden vectors.

Tolerance is the reference's parity rule (cintx-oracle tests/two_electron_parity.rs:26-33):
per element |d| <= 1e-12 or |d| <= 1e-10 |ref|.  Return values (screening) must match exactly.
"""
import itertools
import os

import numpy as np
import pytest

from conftest import ROOT, close
from cintx_b200 import molecules as M
from oracle import RefLibcint, Restatement

pytestmark = pytest.mark.gpu
GOLD = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def cx():
    import cintx_b200
    return cintx_b200


@pytest.fixture(scope="module")
def orc():
    return Restatement()


def test_device_roots_vs_mpmath(cx):
    g = np.load(os.path.join(GOLD, "roots_mpmath.npz"))
    for n in range(1, 10):
        t2, w = cx.rys_t2_batch(n, g["x"])
        np.testing.assert_allclose(t2, g["t2_%d" % n], rtol=5e-15, atol=0)
        np.testing.assert_allclose(w, g["w_%d" % n], rtol=5e-15, atol=0)


def test_cintrys_roots_convention(cx, orc):
    rng = np.random.default_rng(3)
    for n in range(1, 10):
        for x in np.concatenate([rng.uniform(0, 120, 30), [0.0, 1e-12, 5e4]]):
            u, w = cx.rys_roots(n, x)
            uo, wo = orc.rys_roots(n, x)
            np.testing.assert_allclose(u, uo, rtol=1e-13)
            np.testing.assert_allclose(w, wo, rtol=1e-13)


def test_int2e_sph_water3_all_quartets(cx, orc):
    """Every one of the 12^4 quartets of the 3-atom molecule, per-call path, with and
    without an optimizer handle."""
    mol = M.water_like()
    quartets = list(itertools.product(range(mol.nbas), repeat=4))
    ref, offs = orc.int2e_batch(quartets, mol, sph=True)
    with cx.Optimizer(mol.atm, mol.bas, mol.env) as opt:
        for n, q in enumerate(quartets):
            out, ret = cx.int2e_sph(q, mol.atm, mol.bas, mol.env, opt=opt if n % 2 else None)
            r = ref[offs[n]:offs[n] + out.size]
            _, rret = orc.int2e(q, mol)
            assert ret == rret, q
            assert close(out, r), (q, np.abs(out - r).max())


def _golden_family(cx, mol, data, fam, fn, opt=None):
    tup, offs, vals, rets = (data[fam + k] for k in ("_tuples", "_offsets", "_values", "_ret"))
    for q, t in enumerate(tup):
        out, ret = fn(t, mol.atm, mol.bas, mol.env, opt=opt)
        ref = vals[offs[q]:offs[q + 1]]
        assert ret == rets[q], (fam, t)
        assert close(out, ref), (fam, t, np.abs(out - ref).max())


def test_golden_water3_all_families(cx):
    mol = M.water_like()
    g = np.load(os.path.join(GOLD, "libcint_water3.npz"))
    for fam in ("int2e_sph", "int2e_cart", "int3c2e_sph", "int3c2e_cart", "int2c2e_sph", "int2c2e_cart"):
        _golden_family(cx, mol, g, fam, getattr(cx, fam))


def test_golden_g_shells(cx):
    mol = M.mol20_g()
    g = np.load(os.path.join(GOLD, "libcint_mol20g.npz"))
    _golden_family(cx, mol, g, "int2e_sph", cx.int2e_sph)


def test_golden_general_contraction(cx):
    g = np.load(os.path.join(GOLD, "libcint_ctr2.npz"))
    mol = M.Molecule("ctr2", g["atm"], g["bas"], g["env"], np.zeros((2, 3)))
    _golden_family(cx, mol, g, "int2e_sph", cx.int2e_sph)
    _golden_family(cx, mol, g, "int2e_cart", cx.int2e_cart)
    _golden_family(cx, mol, g, "int3c2e_sph", cx.int3c2e_sph)


def test_dims_and_expcutoff(cx, orc):
    mol = M.water_like()
    q = (5, 0, 4, 3)  # (d s | p p): counts (5, 1, 3, 3)
    ref, _ = orc.int2e(q, mol)
    dims = (7, 2, 4, 5)
    big = np.full(int(np.prod(dims)), 7.0)
    out, ret = cx.int2e_sph(q, mol.atm, mol.bas, mol.env, dims=dims, out=big)
    view = out.reshape(dims[::-1])  # [l][k][j][i]
    np.testing.assert_allclose(view[:3, :3, :1, :5], ref.reshape(3, 3, 1, 5), atol=1e-12)
    mask = np.ones(dims[::-1], dtype=bool)
    mask[:3, :3, :1, :5] = False
    assert np.all(view[mask] == 7.0)
    # a tight exponent cut-off changes screening identically in oracle and device
    env = mol.env.copy()
    env[0] = 40.0
    for t in [(0, 1, 0, 1), (0, 3, 6, 9), (5, 5, 11, 11)]:
        m2 = M.Molecule("w", mol.atm, mol.bas, env, mol.coords)
        a, ra = orc.int2e(t, m2)
        b, rb = cx.int2e_sph(t, mol.atm, mol.bas, env)
        assert ra == rb and close(b, a)


@pytest.mark.parametrize("sph", [True, False])
def test_explicit_plan_matches_per_call(cx, orc, sph):
    mol = M.water_like()
    rng = np.random.default_rng(11)
    quartets = rng.integers(0, mol.nbas, size=(3000, 4)).astype(np.int32)
    with cx.Optimizer(mol.atm, mol.bas, mol.env) as opt:
        plan = cx.Plan.shells(opt, 0, quartets, sph=sph)
        out = np.zeros(plan.stats.nintegrals)
        plan.execute_host(out)
        ref, offs = orc.int2e_batch(quartets, mol, sph=sph)
        assert np.array_equal(plan.offsets, offs)
        assert close(out, ref), np.abs(out - ref).max()
        plan.close()
    # 3- and 2-centre families through the same plan machinery
    trip = rng.integers(0, mol.nbas, size=(500, 3)).astype(np.int32)
    duo = rng.integers(0, mol.nbas, size=(100, 2)).astype(np.int32)
    with cx.Optimizer(mol.atm, mol.bas, mol.env, family=1) as opt:
        p3 = cx.Plan.shells(opt, 1, trip, sph=sph)
        o3 = p3.execute_host(np.zeros(p3.stats.nintegrals))
        p2 = cx.Plan.shells(opt, 2, duo, sph=sph)
        o2 = p2.execute_host(np.zeros(p2.stats.nintegrals))
        r3 = np.concatenate([orc.int3c2e(t, mol, sph)[0] for t in trip])
        r2 = np.concatenate([orc.int2c2e(t, mol, sph)[0] for t in duo])
        assert close(o3, r3) and close(o2, r2)
        p3.close()
        p2.close()


def test_screened_plan_mol40(cx, orc):
    """Schwarz-screened unique-quartet sweep: count, and every block of a seeded sample of
    quartets checked against the oracle."""
    mol = M.mol40()
    with cx.Optimizer(mol.atm, mol.bas, mol.env) as opt:
        plan = cx.Plan.screened(opt, 1e-12, sph=True, max_chunk_doubles=1 << 26)
        st = plan.stats
        assert st.nchunks >= 1 and st.nquartets > 0
        import torch
        buf = torch.empty(st.max_chunk_doubles, dtype=torch.float64, device="cuda")
        rng = np.random.default_rng(5)
        seen = 0
        for c in range(st.nchunks):
            plan.execute(buf.data_ptr(), chunk=c, stream=torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            quart = plan.chunk_quartets(c)
            seen += len(quart)
            if c % max(1, st.nchunks // 3):
                continue
            host = buf[:plan.chunk_size(c)].cpu().numpy()
            sizes = np.array([orc_block(mol, q) for q in quart])
            offs = np.concatenate([[0], np.cumsum(sizes)])
            for k in rng.choice(len(quart), size=min(300, len(quart)), replace=False):
                r, _ = orc.int2e(quart[k], mol)
                assert close(host[offs[k]:offs[k + 1]], r), (c, quart[k])
        assert seen == st.nquartets
        plan.close()


def test_execute_host_all_chunks_back_to_back(cx):
    """The pipelined host path (two staging buffers, copies on a second stream) returns every
    chunk back to back, bit-identical to the device path chunk by chunk."""
    mol = M.mol40()
    import torch
    with cx.Optimizer(mol.atm, mol.bas, mol.env) as opt:
        plan = cx.Plan.screened(opt, 1e-12, sph=True, max_chunk_doubles=1 << 23)
        st = plan.stats
        assert st.nchunks >= 3
        host = torch.empty(st.nintegrals, dtype=torch.float64, pin_memory=True).numpy()
        host[:] = np.nan
        plan.execute_host(host)
        buf = torch.empty(st.max_chunk_doubles, dtype=torch.float64, device="cuda")
        s = torch.cuda.current_stream().cuda_stream
        off = 0
        for c in range(st.nchunks):
            n = plan.chunk_size(c)
            plan.execute(buf.data_ptr(), chunk=c, stream=s)
            torch.cuda.synchronize()
            assert np.array_equal(host[off:off + n], buf[:n].cpu().numpy()), c
            off += n
        assert off == st.nintegrals
        with pytest.raises(ValueError):
            plan.execute_host(np.zeros(st.nintegrals - 1))
        # the two-slot host ring hands every chunk over in order, each equal to the above
        ring = torch.empty(2 * st.max_chunk_doubles, dtype=torch.float64, pin_memory=True).numpy()
        got = []
        plan.execute_host_ring(ring, on_chunk=lambda c, a: got.append((c, a.copy())))
        assert [c for c, _ in got] == list(range(st.nchunks))
        assert np.array_equal(np.concatenate([a for _, a in got]), host)
        with pytest.raises(cx.CintxError):
            plan.execute_host_ring(np.zeros(2 * st.max_chunk_doubles - 1))
        plan.close()


def test_autotuned_launch_shapes_give_the_same_integrals(cx):
    """The autotuner may change lanes per quartet class by class; every chunk's output stays
    within the parity tolerance of the default shapes, the choice is reported per segment, and a
    second plan picks the cached shapes up."""
    mol = M.mol40()
    import torch
    with cx.Optimizer(mol.atm, mol.bas, mol.env) as opt:
        plan = cx.Plan.screened(opt, 1e-12, sph=True, max_chunk_doubles=1 << 23)
        st = plan.stats
        s = torch.cuda.current_stream().cuda_stream
        ref = torch.empty(st.max_chunk_doubles, dtype=torch.float64, device="cuda")
        got = torch.empty_like(ref)
        default_lanes = [plan.segment_lanes(c) for c in range(st.nchunks)]
        refs = []
        for c in range(st.nchunks):
            plan.execute(ref.data_ptr(), chunk=c, stream=s)
            torch.cuda.synchronize()
            refs.append(ref[:plan.chunk_size(c)].cpu().numpy())
        plan.autotune(got.data_ptr(), chunk=0, stream=s, reps=1)
        tuned_lanes = [plan.segment_lanes(c) for c in range(st.nchunks)]
        assert all(len(a) == len(b) and (b > 0).all() for a, b in zip(default_lanes, tuned_lanes))
        for c in range(st.nchunks):
            plan.execute(got.data_ptr(), chunk=c, stream=s)
            torch.cuda.synchronize()
            assert close(got[:plan.chunk_size(c)].cpu().numpy(), refs[c]), c
        other = cx.Plan.screened(opt, 1e-12, sph=True, max_chunk_doubles=1 << 23)
        assert other.use_tuned_shapes() > 0
        assert all(np.array_equal(other.segment_lanes(c), tuned_lanes[c]) for c in range(st.nchunks))
        other.close()
        # the choices export as records and import back (what a later process loads from a file)
        recs = cx.tuned_shapes()
        assert len(recs) > 0 and all(len(r) == 6 and 0 <= r[5] < 10 for r in recs)
        cx.load_tuned_shapes(recs)
        assert cx.tuned_shapes() == recs
        with pytest.raises(cx.CintxError):
            cx.load_tuned_shapes([[0, 0, 0, 0, 0, 99]])
        plan.close()


def test_every_launch_shape_gives_the_same_integrals(cx):
    """Each launch-shape variant (lane counts, register caps, the sliced shapes whose lanes sit in
    separate warps, the cooperative shapes with split horizontal transfers) run on every class of an
    s/p/d/f molecule matches the default shape."""
    mol = M.random_molecule("spdf10", 11, 10, 9.0, with_f=True)
    import torch
    with cx.Optimizer(mol.atm, mol.bas, mol.env) as opt:
        plan = cx.Plan.screened(opt, 1e-12, sph=True, max_chunk_doubles=1 << 24)
        st = plan.stats
        s = torch.cuda.current_stream().cuda_stream
        buf = torch.empty(st.max_chunk_doubles, dtype=torch.float64, device="cuda")
        outs = {}
        for v in range(12):
            assert plan.set_shape(v) >= 0
            res = []
            for c in range(st.nchunks):
                buf.zero_()
                plan.execute(buf.data_ptr(), chunk=c, stream=s)
                torch.cuda.synchronize()
                res.append(buf[:plan.chunk_size(c)].cpu().numpy())
            outs[v] = np.concatenate(res)
        assert np.abs(outs[0]).max() > 0
        for v in range(1, 12):
            assert close(outs[v], outs[0]), v
        with pytest.raises(cx.CintxError):
            plan.set_shape(12)
        plan.close()


def test_f_shell_classes_match_libcint_in_every_shape(cx):
    """50 quartets of every f-containing class of the 120-atom molecule (the classes of the
    headline sweep, in random index orders) against libcint at the parity rule, in each launch
    shape the autotuner can pick (variants 0..11) and in the shapes it picks for them."""
    mol = M.mol120()
    g = np.load(os.path.join(GOLD, "libcint_mol120f.npz"))
    tup, ref = g["int2e_sph_tuples"], g["int2e_sph_values"]
    cls, labels, offs = g["class_index"], g["class_labels"], g["int2e_sph_offsets"]
    import torch
    with cx.Optimizer(mol.atm, mol.bas, mol.env) as opt:
        plan = cx.Plan.shells(opt, cx.INT2E, tup, sph=True)
        assert np.array_equal(plan.offsets, offs[:-1])
        n = plan.stats.nintegrals
        buf = torch.empty(n, dtype=torch.float64, device="cuda")
        s = torch.cuda.current_stream().cuda_stream
        lanes = set()
        for v in list(range(12)) + ["tuned"]:
            if v == "tuned":
                plan.autotune(buf.data_ptr(), chunk=0, stream=s, reps=1)
            else:
                assert plan.set_shape(v) >= 0
            lanes.add(tuple(plan.segment_lanes(0)))
            buf.fill_(float("nan"))
            plan.execute(buf.data_ptr(), stream=s)
            torch.cuda.synchronize()
            got = buf.cpu().numpy()
            for c, lab in enumerate(labels):
                for q in np.where(cls == c)[0]:
                    a, b = got[offs[q]:offs[q + 1]], ref[offs[q]:offs[q + 1]]
                    assert close(a, b), (v, lab, tup[q], np.abs(a - b).max())
        assert len(lanes) > 1  # the variants did change the launch shapes
        plan.close()
    # the per-call libcint-signature path on a subset of the same blocks
    for q in range(0, len(tup), 9):
        out, ret = cx.int2e_sph(tup[q], mol.atm, mol.bas, mol.env)
        assert ret == g["int2e_sph_ret"][q] and close(out, ref[offs[q]:offs[q + 1]]), tup[q]


def test_graph_replay_matches_direct_execution(cx):
    mol = M.mol40()
    import torch
    with cx.Optimizer(mol.atm, mol.bas, mol.env) as opt:
        plan = cx.Plan.screened(opt, 1e-12, sph=True, max_chunk_doubles=1 << 25)
        st = plan.stats
        a = torch.zeros(st.max_chunk_doubles, dtype=torch.float64, device="cuda")
        b = torch.zeros_like(a)
        s = torch.cuda.current_stream().cuda_stream
        last = st.nchunks - 1
        plan.execute(a.data_ptr(), chunk=last, stream=s)
        plan.graph_build(b.data_ptr(), chunks=[last], nbranch=4)
        plan.graph_launch(s)
        plan.graph_launch(s)
        torch.cuda.synchronize()
        n = plan.chunk_size(last)
        assert torch.equal(a[:n], b[:n])
        plan.close()


def test_mixed_precision_plan_within_budget(cx, orc):
    """Tuned plan with both shortcuts at 5e-11 each (primitive screening and FP32 recurrences
    for quartets whose estimated FP32 error is below the budget): every integral of the checked
    chunks stays within 1e-10 absolute of the FP64 evaluation (the tuned form's budget), and a
    sample is also within that budget of the oracle."""
    mol = M.mol40()
    import torch
    with cx.Optimizer(mol.atm, mol.bas, mol.env) as opt:
        plan = cx.Plan.screened_mixed(opt, 1e-12, fp32_budget=5e-11, prim_budget=5e-11,
                                      max_chunk_doubles=1 << 24)
        st = plan.stats
        assert 0 < st.nquartets_fp32 < st.nquartets
        buf = torch.empty(st.max_chunk_doubles, dtype=torch.float64, device="cuda")
        s = torch.cuda.current_stream().cuda_stream
        worst = 0.0
        rng = np.random.default_rng(8)
        for c in sorted({0, st.nchunks // 2, st.nchunks - 1}):
            plan.execute(buf.data_ptr(), chunk=c, stream=s)
            torch.cuda.synchronize()
            got = buf[:plan.chunk_size(c)].cpu().numpy()
            quart = plan.chunk_quartets(c)
            ref_plan = cx.Plan.shells(opt, cx.INT2E, quart, sph=True)
            ref = ref_plan.execute_host(np.zeros(ref_plan.stats.nintegrals))
            ref_plan.close()
            worst = max(worst, float(np.abs(got - ref).max()))
            offs = ref_plan.offsets
            for k in rng.choice(len(quart), size=50, replace=False):
                r, _ = orc.int2e(quart[k], mol)
                assert np.abs(got[offs[k]:offs[k] + r.size] - r).max() <= 1e-10
        assert worst <= 1e-10, worst
        plan.close()


def orc_block(mol, q):
    n = 1
    for s in q:
        n *= 2 * int(mol.bas[s, 1]) + 1
    return n


@pytest.mark.skipif(not RefLibcint.available(), reason="libcint from the reference sources not built")
def test_against_live_libcint_mol40_sample(cx):
    ref = RefLibcint()
    mol = M.mol40()
    rng = np.random.default_rng(9)
    for t in rng.integers(0, mol.nbas, size=(400, 4)):
        a, ra = cx.int2e_sph(t, mol.atm, mol.bas, mol.env)
        b, rb = ref.int2e(t, mol)
        assert ra == rb and close(a, b), t


def test_unsupported_inputs_report_errors(cx):
    mol = M.water_like()
    env = mol.env.copy()
    env[8] = 0.3  # range-separated Coulomb
    with pytest.raises(cx.CintxError) as e:
        cx.int2e_sph((0, 0, 0, 0), mol.atm, mol.bas, env)
    assert e.value.code == 2


def test_cintrs_eval_matches_libcint_signature(cx):
    """cintx-capi's id dispatch returns the same blocks and not0 as int2e_sph / int2c2e_cart."""
    import ctypes
    from test_abi import _Summary, _dispatch_args
    mol = M.water_like()
    dp = ctypes.POINTER(ctypes.c_double)
    for api, shls, fn in [(10, [5, 0, 4, 3], lambda t: cx.int2e_sph(t, mol.atm, mol.bas, mol.env)),
                          (9, [1, 2, 3, 4], lambda t: cx.int2e_cart(t, mol.atm, mol.bas, mol.env)),
                          (12, [5, 3], lambda t: cx.int2c2e_cart(t, mol.atm, mol.bas, mol.env)),
                          (13, [5, 3], lambda t: cx.int2c2e_sph(t, mol.atm, mol.bas, mol.env))]:
        ref, ret = fn(shls)
        keep, args = _dispatch_args(mol, shls)
        out = np.full(ref.size, np.nan)
        summ = _Summary()
        rc = cx.lib.cintrs_eval(api, out.ctypes.data_as(dp), out.size, None, 0, *args, None, None, 0,
                                ctypes.byref(summ))
        assert rc == 0 and summ.not0 == ret and summ.bytes_written == 8 * ref.size
        assert np.array_equal(out, ref)
