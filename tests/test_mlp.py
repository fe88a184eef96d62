"""Learned SGS closure: the CPU oracle's own checks, and the GPU kernels
(tcgen05 forward, training gradients, features, fallback to the dynamic
procedure) against it.

Tolerances: the GPU network uses BF16 operands with FP32 accumulation and
the hardware tanh approximation (relative error below 2^-10.9) inside GELU;
the oracle reproduces the BF16 rounding with an exact tanh, so outputs
differ by the tanh error and by the BF16 roundings of hidden activations it
flips (one BF16 ulp is 2^-8 relative).  Outputs: max |dy| <= 2e-3 * (1 + |y|),
median |dy| <= 2e-4.  Gradients: per parameter block, max |dg| <= 2e-3 *
max |g| of the block.
"""
import numpy as np
import pytest

from oracle import mlp_oracle as M


def _params(seed=0, scale=1.0):
    rng = np.random.default_rng(seed)
    p = np.zeros(M.NP, np.float32)
    p[M.O_W1:M.O_B1] = rng.normal(0, np.sqrt(2 / 72), 512) * scale
    p[M.O_B1:M.O_W2] = rng.normal(0, 0.1, 64)
    p[M.O_W2:M.O_B2] = rng.normal(0, np.sqrt(2 / 128), 4096) * scale
    p[M.O_B2:M.O_W3] = rng.normal(0, 0.1, 64)
    p[M.O_W3:M.O_B3] = rng.normal(0, np.sqrt(2 / 65), 64)
    p[M.O_B3] = 0.1
    return p


def _stats():
    s = np.zeros(M.NS, np.float32)
    s[M.S_SD:M.S_SD + 8] = 1.0
    s[M.S_MIN:M.S_MIN + 8] = -1e30
    s[M.S_MAX:M.S_MAX + 8] = 1e30
    s[M.S_YMU] = 0.0
    s[M.S_YSD] = 1.0
    s[M.S_YMIN] = -1e30
    s[M.S_YMAX] = 1e30
    return s


BLOCKS = {"W1": (M.O_W1, M.O_B1), "b1": (M.O_B1, M.O_W2), "W2": (M.O_W2, M.O_B2), "b2": (M.O_B2, M.O_W3),
          "w3": (M.O_W3, M.O_B3), "b3": (M.O_B3, M.NP)}


# ------------------------------------------------------------------ CPU ----
def test_bf16_rounding_known_answers():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, 1.0 + 2.0 ** -7 + 2.0 ** -8, -2.5, 0.0],
                 np.float32)
    # ties go to even: 1 + 2^-8 -> 1; 1 + 1.5 * 2^-8 -> 1 + 2^-7; 1 + 1.5 * 2^-7 -> 1 + 2^-6
    want = np.array([1.0, 1.0, 1.0 + 2.0 ** -7, 1.0 + 2.0 ** -6, -2.5, 0.0], np.float32)
    np.testing.assert_array_equal(M.bf16(x), want)


def test_oracle_gradient_matches_finite_differences():
    """The backward formulas, in FP64 without BF16 rounding, against central differences."""
    rng = np.random.default_rng(1)
    p = _params(1).astype(np.float64)
    x = rng.normal(size=(37, 8))
    t = rng.normal(size=37)
    g, _ = M.grad(p, x, t, bf16_ops=False)
    idx = np.concatenate([rng.choice(np.arange(a, b), size=min(6, b - a), replace=False)
                          for a, b in BLOCKS.values()])
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp = np.mean((M.forward(pp, x, bf16_ops=False) - t) ** 2)
        lm = np.mean((M.forward(pm, x, bf16_ops=False) - t) ** 2)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-6 * abs(fd), (i, fd, g[i])


def test_bf16_gradient_close_to_exact():
    """The GPU's mixed-precision gradient model stays within BF16 rounding of the exact gradient."""
    rng = np.random.default_rng(2)
    p = _params(2)
    x = rng.normal(size=(256, 8)).astype(np.float32)
    t = rng.normal(size=256).astype(np.float32)
    ge, _ = M.grad(p, x, t, bf16_ops=False)
    gb, _ = M.grad(p, x, t, bf16_ops=True)
    for name, (a, b) in BLOCKS.items():
        assert np.abs(gb[a:b] - ge[a:b]).max() <= 3e-2 * np.abs(ge[a:b]).max(), name


# ------------------------------------------------------------------ GPU ----
def _les(nx=32, ny=32, nz=16, precision="fp64", sgs="mlp", **kw):
    from new_repo_b200 import LES, RunParams

    p = RunParams(nx=nx, ny=ny, nz=nz, dt=1e-4, lbc_dz0=1e-4, pfx=1.0, sgs_model=sgs, cs_count=5, dyn_init=5,
                  lbc_special="wall_law", wall_model="wall_filter", dealias="padd", **kw)
    return LES(p, precision=precision)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 128, 1000, 5000])
def test_mlp_forward_matches_oracle(gpu, n):
    les = _les()
    p = _params(3)
    les.mlp_set_params(np.concatenate([p, _stats()]))
    x = np.random.default_rng(4).normal(size=(n, 8)).astype(np.float32)
    y = les.mlp_forward(x)
    yo = M.forward(p, x)
    err = np.abs(y - yo)
    assert err.max() <= 2e-3 * (1 + np.abs(yo).max()), err.max()
    assert np.median(err) <= 2e-4
    les.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [128, 1000, 40000])
def test_mlp_gradient_matches_oracle(gpu, n):
    les = _les()
    p = _params(5)
    les.mlp_set_params(np.concatenate([p, _stats()]))
    rng = np.random.default_rng(6)
    x = rng.normal(size=(n, 8)).astype(np.float32)
    t = rng.normal(size=n).astype(np.float32)
    g, loss = les.mlp_grad(x, t)
    go, lo = M.grad(p, x, t)
    assert abs(loss - lo) <= 1e-4 * lo
    for name, (a, b) in BLOCKS.items():
        e = np.abs(g[a:b] - go[a:b]).max()
        assert e <= 2e-3 * np.abs(go[a:b]).max(), (name, e, np.abs(go[a:b]).max())
    les.close()


@pytest.mark.gpu
def test_mlp_training_is_deterministic(gpu):
    """The same state, collection and training give the same closure bit for
    bit: collected pairs take slots fixed by the state (no atomic counter),
    and the normalisation sums, the per-CTA weight gradients and the losses
    are added in a fixed order (no floating-point atomics)."""
    from new_repo_b200 import log_law_noise

    def run():
        les = _les(nx=64, ny=64, nz=32, sgs="dyn_LagScaleDep")
        les.set_initial_conditions(*log_law_noise(les.params, seed=7))
        les.mlp_init(0)
        les.mlp_reset_data(1 << 20)
        while les.jt_total < 30:
            les.step(1)
            if les.jt_total >= 5 and les.jt_total % 5 == 0:
                les.mlp_collect(stride=3, seed=les.jt_total, dense_levels=4, wall_repeat=3)
        counts = les.mlp_counts()
        les.mlp_fit_stats()
        losses, val = les.mlp_train(epochs=3, tiles_per_step=4, lr=2e-3)
        params = les.mlp_params().copy()
        # one gradient over fewer tiles than CTAs, twice
        rng = np.random.default_rng(8)
        x = rng.normal(size=(1000, 8)).astype(np.float32)
        t = rng.normal(size=1000).astype(np.float32)
        g1, l1 = les.mlp_grad(x, t)
        g2, l2 = les.mlp_grad(x, t)
        np.testing.assert_array_equal(g1, g2)
        assert l1 == l2
        les.close()
        return counts, losses, val, params

    a, b = run(), run()
    assert a[0] == b[0] and a[0][0] > 10000
    assert list(a[1]) == list(b[1]) and a[2] == b[2]
    np.testing.assert_array_equal(a[3], b[3])


def _fields(les):
    names = ("dudx", "dudy", "dudz", "dvdx", "dvdy", "dvdz", "dwdx", "dwdy", "dwdz")
    return {n: les.download(n) for n in names}


def _oracle_cs(les, p, stats, cs_prev, beta=0.0):
    """Cs^2 and the in-range mask of every level 1..nz+1 from the oracle's
    features (beta != 0: the buoyant run's Richardson-number feature)."""
    rp = les.params
    d = _fields(les)
    dtdz = les.download("dtdz") if beta else None
    delta = (rp.dx * rp.dy * rp.dz) ** (1.0 / 3.0)
    cs, ok = [], []
    for k in range(1, rp.nz + 2):
        t = M.raw_features(d, cs_prev, k, rp.dz, delta, np.log(delta / rp.z0), 1, dtdz=dtdz, beta=beta)
        xn = (t - stats[M.S_MU:M.S_MU + 8]) / stats[M.S_SD:M.S_SD + 8]
        cs.append(M.cs_from_output(M.forward(p, xn.astype(np.float32)), stats, t[:, 5]))
        ok.append(M.in_range(xn, stats))
    return np.array(cs), np.array(ok)


@pytest.mark.gpu
@pytest.mark.parametrize("buoyant", [False, True])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mlp_inference_in_step_matches_oracle(gpu, precision, buoyant):
    """Features from the state's gradients, normalisation and the tcgen05
    forward pass inside sgs_stress, against the oracle on the same fields;
    buoyant: a heated, stratified run whose eighth feature is the gradient
    Richardson number."""
    from oracle import les_oracle as O
    from oracle import scalar_oracle as S
    from new_repo_b200 import log_law_noise

    les = _les(precision=precision)
    les.set_initial_conditions(*log_law_noise(les.params, seed=3))
    beta = 30.0 if buoyant else 0.0
    if buoyant:
        les.scalar_init(surface_flux=0.24, top_gradient=10.0, buoyancy=beta)
        rp = les.params
        les.scalar_set_initial(S.inversion_profile(O.Params(nx=rp.nx, ny=rp.ny, nz=rp.nz), seed=3, z_inv=0.3))
    p = _params(7, scale=0.5)
    st = _stats()
    les.mlp_set_params(np.concatenate([p, st]))
    les.step(4)
    les.compute_vel_grad()
    # a non-uniform previous coefficient
    cs_prev = 0.03 * np.exp(0.3 * np.random.default_rng(1).standard_normal(les.download("cs_opt2").shape))
    les.upload("cs_opt2", cs_prev)
    cs_prev = les.download("cs_opt2")
    les.sgs_stress(10, 10)
    cs = les.download("cs_opt2")[1:les.params.nz + 2]
    cso, _ = _oracle_cs(les, p, st, cs_prev, beta)
    cso = cso.reshape(cs.shape)
    e = np.abs(np.log(cs) - np.log(cso))
    assert e.max() <= 2e-2 and np.median(e) <= 3e-4, (e.max(), np.median(e))
    assert les.mlp_info()["flagged_columns"] == 0
    les.close()


@pytest.mark.gpu
def test_mlp_fallback_equals_dynamic_procedure(gpu):
    """Columns whose invariants leave the training range take the dynamic
    procedure's Cs^2: with an empty range every column falls back, and the
    result equals the LASD update with initial Lagrangian averages."""
    from new_repo_b200 import log_law_noise

    les = _les(sgs="dyn_LagScaleDep")
    les.set_initial_conditions(*log_law_noise(les.params, seed=5))
    les.step(6)
    les.set_sgs_model("mlp")
    st = _stats()
    st[M.S_MIN:M.S_MIN + 8] = 1e3  # no feature can be inside [1e3 - 0.25, 1e3 + 0.25]
    st[M.S_MAX:M.S_MAX + 8] = 1e3
    les.mlp_set_params(np.concatenate([_params(8), st]))
    saved = {n: les.download(n) for n in ("F_LM", "F_MM", "F_QN", "F_NN", "beta")}
    les.compute_vel_grad()
    # the fallback relaxes from the previous coefficient; from 0.03 it is the
    # reference's first (initialising) LASD update
    les.upload("cs_opt2", np.full_like(les.download("cs_opt2"), 0.03))
    les.sgs_stress(10, 10)
    info = les.mlp_info()
    assert info["flagged_columns"] == les.params.nx * les.params.ny
    cs_mlp = les.download("cs_opt2")
    for n, a in saved.items():  # the fallback leaves the Lagrangian history alone
        np.testing.assert_array_equal(les.download(n), a)
    les.set_sgs_model("dyn_LagScaleDep")
    les.f_coeff_init = False
    les.sgs_stress(10, 10)
    cs_dyn = les.download("cs_opt2")
    nz = les.params.nz
    np.testing.assert_allclose(cs_mlp[1:nz + 1], cs_dyn[1:nz + 1], rtol=1e-13, atol=0)
    les.close()


@pytest.mark.gpu
def test_mlp_partial_fallback_only_flagged_columns(gpu):
    """A range that excludes part of the domain: flagged columns carry the
    dynamic value, the others the network's."""
    from new_repo_b200 import log_law_noise

    les = _les(sgs="dyn_LagScaleDep")
    les.set_initial_conditions(*log_law_noise(les.params, seed=6))
    les.step(6)
    les.set_sgs_model("mlp")
    les.compute_vel_grad()
    p = _params(9, scale=0.5)
    st = _stats()
    # feature 6 (vortex stretching): exclude the columns whose largest value lies
    # above about the median of the column maxima (threshold in the widest gap
    # between neighbouring column maxima near the median, so float rounding
    # cannot move a column across it)
    d = _fields(les)
    cs_prev = les.download("cs_opt2")
    rp = les.params
    delta = (rp.dx * rp.dy * rp.dz) ** (1.0 / 3.0)
    f6 = np.stack([M.raw_features(d, cs_prev, k, rp.dz, delta, np.log(delta / rp.z0), 1)[:, 6]
                   for k in range(1, rp.nz + 2)])
    cm = np.sort(f6.max(axis=0))
    mid = cm[cm.size // 2 - 64:cm.size // 2 + 64]
    i = int(np.argmax(np.diff(mid)))
    assert mid[i + 1] - mid[i] > 1e-5
    # the test flags x > MAX + 0.25 + 0.05 (MAX - MIN): put that bound at the gap
    lo6 = float(f6.min()) - 1.0
    bound = 0.5 * (mid[i] + mid[i + 1])
    st[M.S_MIN + 6] = lo6
    st[M.S_MAX + 6] = (bound - 0.25 + 0.05 * lo6) / 1.05
    les.mlp_set_params(np.concatenate([p, st]))
    les.sgs_stress(10, 10)
    info = les.mlp_info()
    cs = les.download("cs_opt2")[1:rp.nz + 2].reshape(rp.nz + 1, -1)
    cso, ok = _oracle_cs(les, p, st, cs_prev)
    col_ok = ok.all(axis=0)
    assert 0 < info["flagged_columns"] < rp.nx * rp.ny
    e = np.abs(np.log(cs[:, col_ok]) - np.log(cso[:, col_ok]))
    assert e.max() <= 2e-2
    les.close()


@pytest.mark.gpu
def test_mlp_training_gain_over_constant_coefficient(gpu):
    """Train on LASD pairs from a running state (128 x 128 x 64), then on a
    later (held-out) update step compare log Cs^2 of the closure and of
    constant coefficients with the LASD value the dynamic procedure computes
    on the same fields, and the device time of the SGS update of that step
    with the closure (wall band of 8 LASD levels) against LASD."""
    from new_repo_b200 import log_law_noise

    les = _les(nx=128, ny=128, nz=64, sgs="dyn_LagScaleDep")
    les.set_initial_conditions(*log_law_noise(les.params, seed=11))
    les.mlp_init(0)
    les.mlp_reset_data(1 << 22)
    while les.jt_total < 60:
        les.step(1)
        if les.jt_total >= 5 and les.jt_total % 5 == 0:  # consecutive updates; the first only records
            les.mlp_collect(stride=4, seed=les.jt_total)
    ntr, nva = les.mlp_counts()
    assert ntr > 100000 and nva > 10000
    les.mlp_fit_stats()
    losses, val = les.mlp_train(epochs=8, tiles_per_step=8, lr=2e-3)
    assert val < 0.8, (losses, val)  # normalised target: variance 1
    les.step(4)  # to jt_total 64; the next step is an update step
    les.step(1)
    cs_lasd = les.download("cs_opt2")[1:les.params.nz + 1]
    les.set_sgs_model("mlp")
    les.sgs_stress(les.jt, les.jt_total)
    flagged = les.mlp_info()["flagged_columns"]
    cs_mlp = les.download("cs_opt2")[1:les.params.nz + 1]
    ref = np.log(cs_lasd)
    e_mlp = np.sqrt(np.mean((np.log(cs_mlp) - ref) ** 2))
    e_mean = np.std(ref)  # the best constant in hindsight: exp(mean log Cs^2) of this very state
    e_smag = np.sqrt(np.mean((np.log(0.16 ** 2) - ref) ** 2))
    print(f"rms log error vs LASD: mlp {e_mlp:.3f}, best constant {e_mean:.3f}, cs0=0.16 {e_smag:.3f}; "
          f"val loss {val:.3f}; flagged columns {flagged}")
    assert e_mlp < 0.8 * e_mean and e_mlp < e_smag
    # time saved: the SGS update of this dynamic-update step, device time
    les.mlp_set_wall_levels(8)
    les.mlp_set_check_every(0)

    def update_ms(model, reps=5):
        les.set_sgs_model(model)
        les.sgs_stress(les.jt, les.jt_total)  # warm
        les.sync()
        les.event_record(0)
        for _ in range(reps):
            les.sgs_stress(les.jt, les.jt_total)
        les.event_record(1)
        return les.event_elapsed(0, 1) / reps

    t_lasd = update_ms("dyn_LagScaleDep")
    t_mlp = update_ms("mlp")
    nflag = les.mlp_info()["flagged_columns"]
    # the same closure with its input range opened: no column falls back.  A
    # column outside the range takes the dynamic procedure, whose test filter
    # is a whole-plane transform, so any fallback costs the LASD update's
    # filters on top of the inference
    p = les.mlp_params()
    p[M.NP + M.S_MIN:M.NP + M.S_MIN + 8] = -1e30
    p[M.NP + M.S_MAX:M.NP + M.S_MAX + 8] = 1e30
    les.mlp_set_params(p)
    t_pure = update_ms("mlp")
    assert les.mlp_info()["flagged_columns"] == 0
    print(f"SGS update at a dynamic step (128x128x64): LASD {t_lasd:.3f} ms; learned closure {t_mlp:.3f} ms "
          f"with {nflag} columns falling back, {t_pure:.3f} ms with none")
    assert t_pure < t_lasd
    les.close()


@pytest.mark.gpu
def test_wall_band_keeps_the_lasd_procedure(gpu):
    """With the wall band covering every level the learned-closure run is the
    LASD run; a 3-level band reproduces LASD's first update on those levels."""
    from new_repo_b200 import log_law_noise

    ref = _les(sgs="dyn_LagScaleDep")
    ic = log_law_noise(ref.params, seed=13)
    ref.set_initial_conditions(*ic)
    full = _les()
    full.set_initial_conditions(*ic)
    full.mlp_set_params(np.concatenate([_params(10, scale=0.5), _stats()]))
    full.mlp_set_wall_levels(full.params.nz + 1)
    band = _les()
    band.set_initial_conditions(*ic)
    band.mlp_set_params(np.concatenate([_params(10, scale=0.5), _stats()]))
    band.mlp_set_wall_levels(3)
    ref.step(5)  # step 5 is the first dynamic update
    full.step(5)
    band.step(5)
    cs_ref = ref.download("cs_opt2")
    np.testing.assert_allclose(band.download("cs_opt2")[1:4], cs_ref[1:4], rtol=1e-13, atol=0)
    ref.step(7)
    full.step(7)
    for n in ("u", "v", "w", "cs_opt2", "F_LM", "F_MM"):
        np.testing.assert_allclose(full.download(n)[1:-1], ref.download(n)[1:-1], rtol=1e-12, atol=1e-14)
    for x in (ref, full, band):
        x.close()
