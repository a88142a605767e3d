"""Learned WENO router: the BF16 tensor-core inference and the FP32 training
kernels against the CPU restatement in router_ref.py, label collection from
the plain solver, and the routed sweep at its two limits (every interface to
full WENO reproduces the plain method; every interface to the linear flux is
a stable fifth-order scheme)."""
import numpy as np
import pytest

import router_ref as rr
from howtest import active, rel_l1

pytestmark = pytest.mark.gpu


def _feats(n, seed=0):
    rng = np.random.default_rng(seed)
    x = np.empty((n, 6), np.float32)
    x[:, :5] = rng.uniform(-6.0, 0.5, (n, 5))
    x[:, 5] = rng.integers(0, 2, n)
    return x


@pytest.mark.parametrize("n", [16, 1000, 4101])
def test_router_inference_fp32_and_bf16(n):
    import how_mhd as hm
    w = rr.init_weights(3)
    x = _feats(n, 1)
    lf, lb = hm.router_infer(w, x)
    ref = rr.forward(w, x)
    scale = max(1.0, np.abs(ref).max())
    assert np.abs(lf - ref).max() <= 1e-5 * scale
    refb = rr.forward_bf16(w, x)
    # same BF16 operands; FP32 sums in another order and tanhf vs tanh
    assert np.abs(lb - refb).max() <= 2e-3 * scale, np.abs(lb - refb).max()
    # and BF16 stays close to the FP32 network
    assert np.abs(lb - ref).max() <= 0.1 * scale


def test_router_gradient_vs_cpu():
    import how_mhd as hm
    w = rr.init_weights(5)
    x = _feats(3000, 2)
    y = (np.random.default_rng(3).random(3000) < 0.25).astype(np.float32)
    g, loss = hm.router_grad(w, x, y, pos_weight=3.0)
    lref, gref = rr.loss_and_grad(w, x, y, 3.0)
    assert abs(loss - lref) <= 1e-5 * abs(lref)
    err = np.abs(g - gref).max() / np.abs(gref).max()
    assert err <= 1e-4, err
    idx = [0, 50, 191, 192, 223, 224, 700, 1247, 1248, 1279, 1280, 1311, 1312]
    fd = rr.fd_grad(w, x, y, idx, 3.0)
    np.testing.assert_allclose(g[idx], fd, rtol=2e-3, atol=1e-4 * np.abs(gref).max())


def test_router_training_learns_a_boundary():
    import how_mhd as hm
    x = _feats(20000, 4)
    y = ((x[:, 0] > -2.0) | (x[:, 1] > -1.5)).astype(np.float32)
    w0 = rr.init_weights(7)
    w, hist = hm.router_train(w0, x, y, iters=600, batch=2048, lr=3e-3, pos_weight=1.0, seed=11)
    assert hist[-50:].mean() < 0.5 * hist[:10].mean()
    acc = ((rr.forward(w, x) > 0) == (y > 0.5)).mean()
    assert acc > 0.97, acc
    # deterministic: same seed, same weights
    w2, _ = hm.router_train(w0, x, y, iters=600, batch=2048, lr=3e-3, pos_weight=1.0, seed=11)
    np.testing.assert_array_equal(w, w2)


def _domain(prob, n, tend=100.0, **kw):
    import how_mhd as hm
    p = hm.make_parameters(nx=n[0], ny=n[1], nz=n[2], nt=1, tend=tend, gam=5.0 / 3.0, cour=0.4,
                           problem=prob, **kw)
    return hm.Domain(p)


def test_collect_labels_from_plain_solver():
    with _domain("orszag_tang", (64, 64, 1)) as d:
        d.init_problem()
        d.run(0.0, 20)
        ref = d.get_state(0)
        d.collect_begin(1 << 20, every=1)
        d.run(0.0, 2)
        rec = d.collect_end()
    # 2 steps x 5 stages x 2 directions x 65 faces x 64 lines: every active
    # face once (a face shared by two tiles is recorded by one)
    assert len(rec) == 2 * 5 * 2 * 65 * 64
    assert np.isfinite(rec).all()
    # the weight departure lies in [0, 1]; the flux departure is >= 0, and
    # positive somewhere in the vortex
    assert (rec[:, 6] >= 0).all() and (rec[:, 6] <= 1).all() and (rec[:, 6] > 0.1).any()
    assert (rec[:, 7] >= 0).all() and rec[:, 7].max() > 0
    assert (rec[:, 5] == 0).all()   # the prior-stage feature is held at 0
    assert np.isfinite(ref).all()


def test_collect_matches_plain_run():
    """Collection runs the plain FP64 method: the state is unchanged by it."""
    with _domain("orszag_tang", (64, 64, 1)) as d:
        d.init_problem()
        d.run(0.0, 5)
        a = d.get_state(0)
    with _domain("orszag_tang", (64, 64, 1)) as d:
        d.init_problem()
        d.collect_begin(1 << 16, every=3)
        d.run(0.0, 5)
        d.collect_end()
        b = d.get_state(0)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("prob,n,kw", [
    ("orszag_tang", (128, 128, 1), {}),
    ("blast3d_b", (32, 32, 32), dict(rhomin=1e-6, pgmin=1e-6)),
])
def test_routed_all_full_equals_plain(prob, n, kw):
    with _domain(prob, n, **kw) as d:
        d.init_problem()
        d.run(0.0, 8)
        a = d.get_state(0)
    with _domain(prob, n, **kw) as d:
        d.init_problem()
        d.set_router(rr.init_weights(0), "learned", threshold=-1e30)
        d.run(0.0, 8)
        b = d.get_state(0)
        full, cheap = d.router_stats()
    assert cheap == 0 and full > 0
    # the two paths compile separately and may contract products into FMAs
    # differently: equal to round-off, with components that are round-off
    # noise themselves (Mz of the 2-D vortex) measured against their vector
    err = rel_l1(active(b, *n), active(a, *n))
    assert np.all(err <= 1e-13), err


def test_routed_all_linear_converges_to_plain_on_alfven():
    """Every interface on the linear flux (guard off) on the smooth 1-D
    Alfven wave, one period: the difference from the full method is the gap
    between two fifth-order dissipations, so it shrinks by >= 2^4 per
    refinement."""
    diffs = []
    for n in (32, 64):
        out = []
        for routed in (False, True):
            with _domain("alfven3d", (n, 1, 1), tend=1.0) as d:
                d.init_problem()
                if routed:
                    d.set_router(rr.init_weights(0), "learned", threshold=1e30, guard_jump=1e30, guard_floor=0.0)
                d.run(0.0, 10 ** 6)
                if routed:
                    full, cheap = d.router_stats()
                    assert full == 0 and cheap > 0
                out.append(active(d.get_state(0), n, 1, 1))
        assert np.isfinite(out[1]).all()
        diffs.append(np.abs(out[1][5] - out[0][5]).mean())
    assert diffs[1] > 0 and diffs[0] / diffs[1] >= 16.0, diffs


def _blast_final(n, tend, precision, router=None, mode="learned"):
    import how_mhd as hm
    p = hm.make_parameters(nx=n, ny=n, nz=n, nt=1, tend=tend, gam=5.0 / 3.0, cour=0.4, problem="blast3d_b",
                           rhomin=1e-6, pgmin=1e-6, precision=precision)
    with hm.Domain(p) as d:
        d.init_problem()
        if router is not None:
            w, thr = router
            d.set_router(w, mode, threshold=thr)
        d.run(0.0, -1)
        st = d.router_stats() if router is not None else (0, 0)
        return active(d.get_state(0), n, n, n)[0].copy(), st


def test_trained_router_accuracy_and_ablation():
    """The built-in network on the magnetised blast (64^3 to t = 0.2): mixed
    precision + learned routing stays within density L1 1e-5 of plain FP64
    while sending most interfaces to the linear flux; the same routing without
    the network (guard only) is far less accurate -- what the network adds."""
    import how_mhd as hm
    w, thr = hm.default_router()
    ref, _ = _blast_final(64, 0.2, "fp64")
    learned, (f1, c1) = _blast_final(64, 0.2, "mixed", (w, thr), "learned")
    guard, (f2, c2) = _blast_final(64, 0.2, "mixed", (w, thr), "guard")
    l1 = lambda a: float(np.abs(a - ref).sum() / np.abs(ref).sum())
    e_learned, e_guard = l1(learned), l1(guard)
    assert e_learned <= 1e-5, e_learned
    assert f1 / (f1 + c1) < 0.5, (f1, c1)
    assert e_guard >= 10.0 * e_learned and e_guard > 1e-5, (e_guard, e_learned)


def test_router_on_key_uses_builtin_network():
    import how_mhd as hm
    p = hm.make_parameters(nx=32, ny=32, nz=32, nt=1, tend=100.0, gam=5.0 / 3.0, cour=0.4, problem="blast3d_b",
                           rhomin=1e-6, pgmin=1e-6, precision="mixed", router="on")
    with hm.Domain(p) as d:
        d.init_problem()
        d.run(0.0, 3)
        full, cheap, mma, flat = d.router_stats(groups=True)
    assert full > 0 and cheap > 0 and mma + flat > 0


def test_refresh_every_two_steps():
    """Decisions formed once every two steps (refresh 10) on the magnetised
    blast 64^3 to t = 0.2: within the same density bar as once per step, with
    half the routing passes; a state change in between forms fresh ones."""
    import how_mhd as hm
    w, thr = hm.default_router()
    ref, _ = _blast_final(64, 0.2, "fp64")
    p = hm.make_parameters(nx=64, ny=64, nz=64, nt=1, tend=0.2, gam=5.0 / 3.0, cour=0.4, problem="blast3d_b",
                           rhomin=1e-6, pgmin=1e-6, precision="mixed")
    with hm.Domain(p) as d:
        d.init_problem()
        d.set_router(w, "learned", threshold=thr)
        d.set_router_refresh(10)
        l0 = d.kernel_launches
        t4, _, _ = d.run(0.0, 4)
        launches4 = d.kernel_launches - l0
        d.run(t4, -1)
        got = active(d.get_state(0), 64, 64, 64)[0]
    with hm.Domain(p) as d:
        d.init_problem()
        d.set_router(w, "learned", threshold=thr)
        l0 = d.kernel_launches
        d.run(0.0, 4)
        launches4_step = d.kernel_launches - l0
    # two routing passes (3 launches each) fewer over four steps
    assert launches4_step - launches4 == 2 * 3, (launches4_step, launches4)
    e = float(np.abs(got - ref).sum() / np.abs(ref).sum())
    assert e <= 1e-5, e
    with pytest.raises(Exception):
        with hm.Domain(p) as d:
            d.set_router_refresh(7)
