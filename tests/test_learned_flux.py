"""The learned face flux: the tensor-core network kernels against the CPU
oracle of the same rounded network (oracle/mlp_oracle.py)."""
import numpy as np
import pytest

from oracle import mlp_oracle as M


def test_oracle_gradient_matches_finite_differences():
    """The oracle's backward pass is the derivative of its loss (checked on
    the unrounded network by central differences)."""
    rng = np.random.default_rng(2)
    p = M.init_params(3).astype(np.float64) * 0.5
    X = rng.normal(size=(16, M.NIN))
    Y = rng.normal(size=(16, M.NOUT))
    saved = M.bf16
    M.bf16 = lambda x: np.asarray(x, np.float64)  # exact arithmetic for the check
    try:
        _, g = M.loss_and_grad(p, X, Y)
        for idx in rng.choice(p.size, 40, replace=False):
            h = 1e-6
            pp, pm = p.copy(), p.copy()
            pp[idx] += h
            pm[idx] -= h
            fd = (M.loss_and_grad(pp, X, Y)[0] - M.loss_and_grad(pm, X, Y)[0]) / (2 * h)
            assert abs(fd - g[idx]) <= 1e-6 * max(1.0, abs(fd)), idx
    finally:
        M.bf16 = saved


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7 + 2 ** -9, -3.5, 0.0], np.float32)
    assert M.bf16(x).tolist() == [1.0, 1.0, 1.0 + 2 ** -7, -3.5, 0.0]


def test_f16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -11, 1.0 + 2 ** -10 + 2 ** -12, -3.5, 0.0, 70000.0], np.float32)
    assert M.f16(x).tolist() == [1.0, 1.0, 1.0 + 2 ** -10, -3.5, 0.0, np.inf]


def test_twice_gelu_with_halved_weights_is_the_same_network():
    """The algebra behind the inference kernel's weights image: storing
    2 gelu(x) as the next layer's FP16 input and halving W2, W3 and W4 gives
    the network of gelu(x) and W, because power-of-two scaling commutes with
    FP16 rounding and cancels in each product.  Values in FP16's subnormal
    range (below 2^-14) round on a coarser grid, so the two forms agree to
    the rounding of those small terms, not bit for bit.  This checks the
    algebra in float64 with the oracle's own gelu; the GPU inference test
    bounds the kernel's half-precision evaluation of 2 gelu."""
    rng = np.random.default_rng(4)
    p = M.init_params(9)
    X = rng.normal(size=(257, M.NIN))
    W1, b1, W2, b2, W3, b3, W4, b4 = M.unpack(p)
    a = M.f16(X).astype(np.float64)
    z = a @ M.f16(W1).astype(np.float64).T + b1
    for W, b in ((W2, b2), (W3, b3), (W4, b4)):
        x = M.f16(z).astype(np.float64)
        a = M.f16(M.gelu(x)).astype(np.float64)
        z = a @ M.f16(W).astype(np.float64).T + b
    got = M.infer(p, X)
    assert np.abs(got - z).max() <= 1e-5 * np.abs(z).max()


# Tensor-core inference against the oracle's rounded network: largest error
# per output over the rows, relative to that output's largest magnitude over
# 4096 rows of the same distribution (a few rows alone would make the scale
# the size of whatever values they happen to have).  The kernel differs from
# the oracle by FP32 accumulation order and its GELU epilogue in packed half
# precision (u and the result rounded to FP16, the hardware
# tanh.approx.f16x2): measured at most 1.4e-3.
INFER_RTOL = 3e-3


def output_scale(p):
    X = np.random.default_rng(12345).normal(size=(4096, M.NIN))
    return np.abs(M.infer(p, X)).max(axis=0)


# 148 SMs x 4 tile chains x 128 rows = 75,776 rows per wave: the larger
# cases make every chain run several tiles (input prefetch, buffer and
# tensor-memory reuse, mbarrier phases carried across tiles).
@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 1000, 128 * 400 + 17, 160000, 303 * 512 + 5])
def test_tensor_core_inference_matches_oracle(n):
    import fvmhd3d_b200 as F
    rng = np.random.default_rng(n)
    p = M.init_params(5)
    s = F.System()
    s.mlp_set_weights(p)
    X = rng.normal(size=(n, M.NIN)).astype(np.float32)
    got = s.mlp_eval(X)
    ref = M.infer(p, X)
    err = np.abs(got - ref).max(axis=0) / output_scale(p)
    assert np.isfinite(got).all()
    assert err.max() <= INFER_RTOL, err


@pytest.mark.gpu
def test_tensor_core_inference_with_a_device_row_count():
    """The launch the flux passes make: grid sized for nmax rows, the row
    count read on the device, well below nmax but spanning several tiles per
    chain; rows past the count are left untouched."""
    import fvmhd3d_b200 as F
    nmax, n = 600000, 2 * 75776 + 4099
    rng = np.random.default_rng(8)
    p = M.init_params(6)
    s = F.System()
    s.mlp_set_weights(p)
    X = rng.normal(size=(nmax, M.NIN)).astype(np.float32)
    Y0 = np.full((nmax, M.NOUT), 7.0, np.float32)
    got = s.mlp_eval_counted(X, n, Y0)
    assert (got[n:] == 7.0).all()
    ref = M.infer(p, X[:n])
    err = np.abs(got[:n] - ref).max(axis=0) / output_scale(p)
    assert err.max() <= INFER_RTOL, err


GRAD_RTOL = 1e-2  # measured 1.6e-3 at most


# 300 rows: one output tile per product and a two-way K split of the weight
# gradients; 2500 rows: 20 row tiles and a ten-way split (the products run
# on tcgen05 in 128 x 128 tiles with K in chunks of 64).
@pytest.mark.gpu
@pytest.mark.parametrize("rows", [300, 2500])
def test_training_gradient_matches_oracle(rows):
    """Backward kernels (BF16 tensor-core GEMMs, FP32 accumulation) against
    the oracle's backward pass of the same rounded network: loss to 1e-3,
    each parameter block's gradient to GRAD_RTOL in norm."""
    import fvmhd3d_b200 as F
    rng = np.random.default_rng(11)
    p = M.init_params(7)
    X = rng.normal(size=(rows, M.NIN)).astype(np.float32)
    T = rng.normal(size=(rows, M.NOUT)).astype(np.float32)
    wt = np.linspace(0.5, 2.0, M.NOUT)
    s = F.System()
    s.mlp_set_weights(p)
    loss, g = s.mlp_grad(X, T, wt)
    rloss, rg = M.loss_and_grad(p, X, T, wt)
    assert abs(loss - rloss) <= 1e-3 * rloss
    o = 0
    for shp in M.SHAPES:
        k = int(np.prod(shp))
        a, b = g[o:o + k], rg[o:o + k]
        assert np.linalg.norm(a - b) <= GRAD_RTOL * np.linalg.norm(b), (shp, np.linalg.norm(a - b) / np.linalg.norm(b))
        o += k


@pytest.mark.gpu
def test_training_fits_a_smooth_map():
    """Adam on the GPU fits a smooth 16 -> 8 map far below its variance."""
    import fvmhd3d_b200 as F
    rng = np.random.default_rng(4)
    X = rng.uniform(-1, 1, size=(50000, M.NIN)).astype(np.float32)
    A = rng.normal(size=(M.NIN, M.NOUT)) / 4
    T = (np.tanh(X @ A) + 0.3 * (X[:, :M.NOUT] ** 2)).astype(np.float32)
    s = F.System()
    s.mlp_set_weights(M.init_params(1))
    hist = s.mlp_train(X, T, batch=2048, steps=1500, lr=2e-3, seed=3)
    assert hist[-50:].mean() < 0.02 * T.var()
    Y = s.mlp_eval(X[:4096])  # the tensor-core inference uses the trained weights
    assert np.mean((Y - T[:4096]) ** 2) < 0.03 * T.var()
    assert np.allclose(M.infer(s.mlp_get_weights(), X[:512]), Y[:512], atol=2e-2 * np.abs(T).max())


def test_hlld_flux_is_galilean_covariant_under_normal_boosts():
    """The identity the learned flux relies on to work in the face frame:
    the reference's flux at face speed w equals the flux of the boosted
    states at w = 0, mapped back (mass unchanged, momentum + w F_mass,
    energy + w.F_mom + w^2/2 F_mass, induction - w Bn)."""
    import os
    from common import ORACLE_SO
    if not os.path.exists(ORACLE_SO):
        pytest.skip("oracle not built")
    from oracle.pyoracle import OracleSystem
    rng = np.random.default_rng(1)
    nf = 500
    Wi, Wj = np.zeros((nf, 10)), np.zeros((nf, 10))
    for W in (Wi, Wj):
        W[:, 0] = rng.uniform(0.5, 2, nf)
        W[:, 1:4] = rng.normal(0, 0.3, (nf, 3))
        W[:, 4] = rng.uniform(0.75, 3, nf)
        W[:, 5:8] = rng.normal(0, 0.5, (nf, 3))
        W[:, 9] = 1.0
    n = rng.normal(size=(nf, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    w = rng.normal(0, 0.3, (nf, 1)) * n
    jb = np.zeros(nf, np.int32)
    o = OracleSystem()
    _, Bn, F = o.compute_flux(w, Wi, Wj, jb, n)
    Wi0, Wj0 = Wi.copy(), Wj.copy()
    Wi0[:, 1:4] -= w
    Wj0[:, 1:4] -= w
    _, Bn0, F0 = o.compute_flux(np.zeros_like(w), Wi0, Wj0, jb, n)
    G = F0.copy()
    G[:, 1:4] += F0[:, [0]] * w
    G[:, 4] += (w * F0[:, 1:4]).sum(1) + 0.5 * (w * w).sum(1) * F0[:, 0]
    G[:, 5:8] -= w * Bn0[:, None]
    assert np.array_equal(Bn, Bn0)
    scale = np.abs(F).max(axis=0)
    assert (np.abs(F - G).max(axis=0) <= 1e-13 * np.maximum(scale, 1e-300)).all()


@pytest.fixture(scope="module")
def small_trained():
    """Harvest from small Alfven and blast runs, train briefly on the GPU."""
    from fvmhd3d_b200 import learned as L
    X, Y = L.harvest(scale=0.1)
    model, hist = L.train(X, Y, steps=2000, batch=4096, seed=2)
    return X, Y, model, hist


@pytest.mark.gpu
def test_shipped_network_beats_central_and_llf_on_a_deployed_run():
    """The shipped network on the faces a run actually hands it: the 32^3
    blast, 10 global steps, FP32 bulk, every deferred face judged against the
    exact solver.  Its dissipation error is under half the dissipation
    itself (a central flux, i.e. no dissipation, scores 1), and the state
    after the run is closer to the plain FP64 run than with the central flux
    alone or the local Lax-Friedrichs dissipation on the same faces."""
    import fvmhd3d_b200 as F
    from fvmhd3d_b200 import learned as L
    model = L.load_model()
    pos = F.jittered_lattice(32, 0.1, seed=1)
    m = F.build_periodic(pos[F.sort_local_data(pos, 1.0)], 1.0)
    W = F.problems.blast(m.pos)
    ref = F.System()
    ref.set_mesh(m)
    ref.init_problem(W)
    ref.run(10, shared=True)
    Ua = ref.get_state()["U"]
    rel, judged = {}, {}
    for sur in ("network", "central", "llf"):
        s = F.System(precision=F.FVM_PREC_FP32)
        s.set_mesh(m)
        s.init_problem(W)
        L.apply(s, model)
        s.set_flux_mode(1, judge=1, **L.GATE)
        s.set_flux_surrogate(sur)
        s.run(10, shared=True)
        Ub = s.get_state()["U"]
        d = np.abs(Ub - Ua).sum(axis=0) / np.abs(Ua).sum(axis=0)
        rel[sur] = d[[0, 4]].max()
        st = s.learn_stats()
        judged[sur] = st["judged_rel_l1"]
        assert st["judged"] == st["deferred"] > 0
    assert judged["network"] < 0.5, judged
    assert abs(judged["central"] - 1.0) < 1e-6, judged
    assert rel["network"] < rel["central"] and rel["network"] < rel["llf"], rel


@pytest.mark.gpu
def test_trained_network_beats_the_method_without_it(small_trained):
    """On harvested faces, the trained network's dissipation is closer to
    the exact solver's than the local Lax-Friedrichs dissipation (the
    method without the network), and far closer than the untrained
    network's."""
    import fvmhd3d_b200 as F
    from fvmhd3d_b200 import learned as L
    X, Y, model, hist = small_trained
    assert X.shape[0] > 100000 and np.isfinite(hist).all() and hist[-100:].mean() < hist[:100].mean()
    s = F.System()
    idx = np.random.default_rng(0).choice(X.shape[0], 50000, replace=False)
    w = L.OUTPUT_WEIGHTS.astype(bool)
    L.apply(s, model)
    err = np.abs(L.predict(s, model, X[idx]) - Y[idx])[:, w].mean()
    s.mlp_set_weights(L.init_params(2))
    err0 = np.abs(L.predict(s, model, X[idx]) - Y[idx])[:, w].mean()
    err_llf = np.abs(L.llf_dissipation(X[idx]) - Y[idx])[:, w].mean()
    assert err < 0.5 * err_llf and err < 0.1 * err0, (err, err_llf, err0)


@pytest.mark.gpu
def test_learned_flux_steps_conserve_and_stay_close(small_trained):
    """Learned flux on gated faces (FP32 bulk): mass, momentum and energy
    conserved to round-off (fluxes stay antisymmetric per face), the state
    close to the exact solver's after 10 steps, the judge and gate active."""
    import fvmhd3d_b200 as F
    from fvmhd3d_b200 import learned as L
    model = small_trained[2]
    m = F.build_periodic(F.jittered_lattice(20, 0.1, seed=3), 1.0)
    W = F.problems.blast(m.pos)
    a, b = F.System(precision=F.FVM_PREC_FP32), F.System(precision=F.FVM_PREC_FP32)
    for s in (a, b):
        s.set_mesh(m)
        s.init_problem(W)
    L.apply(b, model)
    b.set_flux_mode(1, judge=8, **L.GATE)
    U0 = b.get_state()["U"].sum(axis=0)
    for _ in range(10):
        a.step(shared=True)
        b.step(shared=True)
    Ua, Ub = a.get_state()["U"], b.get_state()["U"]
    scale = np.abs(Ub).sum(axis=0)
    for k in (0, 1, 2, 3, 4):
        assert abs(Ub[:, k].sum() - U0[k]) <= 1e-9 * scale[k], k
    rel = np.abs(Ub - Ua).sum(axis=0) / np.abs(Ua).sum(axis=0)
    assert rel[0] < 1e-2 and rel[4] < 1e-2, rel
    st = b.learn_stats()
    assert st["deferred"] > 0 and st["judged"] > 0 and st["fallback"] <= st["deferred"]
