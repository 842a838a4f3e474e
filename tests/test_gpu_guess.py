"""The learned Newton start (a 6 -> 64 -> 64 -> 1 MLP for twoshock's starting pressure):
GPU training kernels against the CPU reference net, the tensor-core inference against
the same net, the Riemann log against the oracle's two-shock solver, and the solver
with the learned start against the FP64 oracle (plain start) within the parity bar,
with fewer Newton iterations."""
import numpy as np
import pytest

import guess_ref as G
import oracle as O
from ppm_b200 import capi
from ppm_b200 import harness as H
from ppm_b200 import learned as LRN
from parity_util import compare, copy_fields, random_state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    t.cuda.set_device(0)
    return t


@pytest.fixture(scope="module")
def ctx(torch):
    s = torch.cuda.Stream()
    torch.cuda.set_stream(s)
    c = capi.Context(0, stream=s.cuda_stream)
    yield c
    c.close()


def _rand_samples(rng, n):
    s = np.zeros((n, 8), dtype=np.float32)
    s[:, :6] = 0.6 * rng.standard_normal((n, 6))
    s[:, 6] = 0.3 * rng.standard_normal(n)
    s[:, 7] = 1.0
    return s


def test_gpu_gradient_matches_cpu_reference(ctx, torch):
    rng = np.random.default_rng(1)
    w = LRN.init_weights(3)
    w[G.OFF_B1:G.OFF_W2] = 0.1 * rng.standard_normal(64)
    s = _rand_samples(rng, 3000)
    idx = rng.permutation(3000)[:2500].astype(np.int64)
    loss_c, g_c = G.loss_and_grad(w, s[idx], rounding=True)
    wd = torch.from_numpy(w).cuda()
    sd = torch.from_numpy(s).cuda()
    idd = torch.from_numpy(idx).cuda()
    grad = torch.zeros(capi.GUESS_WEIGHTS, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.guess_grad(wd, sd, idd, len(idx), grad, loss)
    torch.cuda.synchronize()
    g = grad.cpu().numpy().astype(np.float64)
    assert abs(loss.item() - loss_c) <= 1e-4 * loss_c
    for lo, hi in ((G.OFF_W1, G.OFF_B1), (G.OFF_B1, G.OFF_W2), (G.OFF_W2, G.OFF_B2),
                   (G.OFF_B2, G.OFF_W3), (G.OFF_W3, G.OFF_B3), (G.OFF_B3, G.NWEIGHTS)):
        scale = np.max(np.abs(g_c[lo:hi]))
        err = np.max(np.abs(g[lo:hi] - g_c[lo:hi]))
        assert err <= 2e-3 * scale + 1e-7, (lo, hi, err, scale)


def test_adam_step_updates_and_clears_gradient(ctx, torch):
    w = torch.ones(capi.GUESS_WEIGHTS, dtype=torch.float32, device="cuda")
    g = torch.full_like(w, 0.5)
    m = torch.zeros_like(w)
    v = torch.zeros_like(w)
    torch.cuda.synchronize()
    ctx.guess_adam(w, g, m, v, 1, 1e-2)
    torch.cuda.synchronize()
    # first Adam step moves every weight by lr against the gradient's sign
    assert torch.allclose(w, torch.full_like(w, 1.0 - 1e-2), atol=1e-6)
    assert float(g.abs().max()) == 0.0


def test_tensor_core_inference_matches_cpu_net(ctx, torch):
    rng = np.random.default_rng(2)
    w = LRN.init_weights(4)
    w[G.OFF_B1:G.OFF_W2] = 0.1 * rng.standard_normal(64)
    w[G.OFF_B2:G.OFF_W3] = 0.1 * rng.standard_normal(64)
    w[G.OFF_B3] = 0.05
    ctx.set_guess(w)
    n = 1000  # not a multiple of 32: the last warp has lanes without a face
    x = (0.6 * rng.standard_normal((n, 6))).astype(np.float32)
    y_c, _ = G.forward(w, x, rounding=True)
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros(n, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    ctx.guess_eval(xd, n, yd)
    torch.cuda.synchronize()
    y = yd.cpu().numpy().astype(np.float64)
    scale = np.max(np.abs(y_c))
    d = np.abs(y - y_c)
    assert np.max(d) <= 1e-2 * scale, (np.max(d), scale)
    assert np.median(d) <= 1e-3 * scale, (np.median(d), scale)


def test_features_match_cpu_reference(ctx, torch):
    rng = np.random.default_rng(5)
    n = 4000
    rec = np.zeros((n, 8))
    rec[:, 0:2] = np.exp(rng.standard_normal((n, 2)))
    rec[:, 2:4] = np.exp(rng.standard_normal((n, 2)))
    rec[:, 4:6] = rng.standard_normal((n, 2))
    rec[:, 6] = np.exp(rng.standard_normal(n)) * rec[:, 2]
    rec[:, 7] = rng.choice([3.0, -7.0], n, p=[0.9, 0.1])
    rec[:10, 1] = rec[:10, 0]  # equal states: no usable target
    rec[:10, 3] = rec[:10, 2]
    rec[:10, 5] = rec[:10, 4]
    s_c = G.samples_from_records(rec, 5.0 / 3.0, 1e-20)
    rd = torch.from_numpy(rec).cuda()
    sd = torch.zeros((n, 8), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    ctx.guess_features(rd, n, 5.0 / 3.0, 1e-20, sd)
    torch.cuda.synchronize()
    s = sd.cpu().numpy()
    assert np.array_equal(s[:, 7], s_c[:, 7])
    assert np.allclose(s[:, :6], s_c[:, :6], rtol=1e-6, atol=1e-6)
    ok = s_c[:, 7] > 0
    assert np.allclose(s[ok, 6], s_c[ok, 6], rtol=1e-5, atol=1e-6)


def test_riemann_log_holds_plain_two_shock_solutions(ctx, torch):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True)
    g = H.Grid.uniform((16, 12, 10))
    f = random_state(g, hp, seed=9)
    rec = torch.zeros((200000, 8), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.riemann_log(rec, 1)
    p = O.compute_pressure(g, hp, f)
    dt = hp.cfl * O.calc_dt(g, hp, f, p, g.cellwidth)
    rc, st = ctx.solve_ppm_de(g, hp, dt, 0, f)
    n = ctx.riemann_log_count()
    ctx.riemann_log(None, 0)
    assert rc == capi.OK
    assert n == st["interfaces"]  # stride 1 logs every face
    r = rec[:n].cpu().numpy()
    for k in np.random.default_rng(0).choice(n, 300, replace=False):
        pb, ub, it = O.twoshock_point(r[k, :6], hp.gamma, hp.tiny_number)
        assert pb == r[k, 6], k
        assert it == int(r[k, 7]), k


def _turb(n, mach, seed, hp):
    g = H.Grid.uniform((n, n, n))
    return g, H.turbulence(g, hp, mach=mach, seed=seed)


def _totals(g, f):
    act = g.active_slices()
    return float(np.sum(f["d"][act])), float(np.sum((f["d"] * f["te"])[act]))


# learned_guess 1: the net inside the Riemann kernel (mma.sync); 2: a tensor-core guess
# pass (tcgen05, TMEM accumulators) over the interface states before it
@pytest.mark.parametrize("mach,steps,mode", [(3.0, 40, 1), (10.0, 25, 1), (3.0, 40, 2),
                                             (10.0, 25, 2)])
def test_learned_start_stays_within_the_parity_bar_and_saves_iterations(ctx, torch, mach,
                                                                          steps, mode):
    w = LRN.default_weights()
    ctx.set_guess(w)
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True)
    g, f0 = _turb(24, mach, 31, hp)
    f_ora = copy_fields(f0)
    f_gpu = copy_fields(f0)
    it_plain = it_learn = n_if = 0
    for cyc in range(steps):
        p = O.compute_pressure(g, hp, f_ora)
        dt = hp.cfl * O.calc_dt(g, hp, f_ora, p, g.cellwidth)
        rc, st_o = O.solve_ppm_de(g, hp, dt, cyc, f_ora, g.cellwidth)
        assert rc == 0
        rc, st_g = ctx.solve_ppm_de(g, hp, dt, cyc, f_gpu, learned_guess=mode)
        assert rc == capi.OK
        it_plain += st_o["newton_iters"]
        it_learn += st_g["newton_iters"]
        n_if += st_g["interfaces"]
        tol = 1e-12 if cyc == 0 else 1e-10
        for k, r in compare(f_gpu, f_ora, g).items():
            assert r["maxrel"] <= tol, (cyc, k, r)
        H.fill_ghosts(g, f_ora, "periodic")
        H.fill_ghosts(g, f_gpu, "periodic")
    # the learned start saves Newton iterations over the plain (acoustic) start
    assert it_learn < it_plain, (it_learn / n_if, it_plain / n_if)
    # mass of the periodic box is conserved to round-off (total energy is not: the
    # dual-energy formalism resets E from the gas energy in cold cells, pgas2d_dual.F)
    m0, _ = _totals(g, f0)
    m1, _ = _totals(g, f_gpu)
    assert abs(m1 - m0) <= 1e-12 * m0


@pytest.mark.parametrize("learned", [False, True])
def test_mass_and_energy_conserved_without_dual_energy(ctx, torch, learned):
    ctx.set_guess(LRN.default_weights())
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=False)
    g, f0 = _turb(20, 2.0, 41, hp)
    f = copy_fields(f0)
    for cyc in range(20):
        dt = ctx.compute_timestep(g, hp, f)
        rc, _ = ctx.solve_ppm_de(g, hp, dt, cyc, f, learned_guess=learned)
        assert rc == capi.OK
        H.fill_ghosts(g, f, "periodic")
    m0, e0 = _totals(g, f0)
    m1, e1 = _totals(g, f)
    assert abs(m1 - m0) <= 1e-12 * m0
    assert abs(e1 - e0) <= 1e-12 * e0


@pytest.mark.parametrize("mode", [1, 2])
def test_learned_start_in_level_batches_matches_per_grid(ctx, torch, mode):
    ctx.set_guess(LRN.default_weights())
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True)
    shapes = [(16, 16, 16), (12, 20, 8), (9, 9, 30)]
    grids = [H.Grid.uniform(s) for s in shapes]
    host = [random_state(gr, hp, seed=60 + k, mach=2.5) for k, gr in enumerate(grids)]
    a = [{k: torch.from_numpy(v.copy()).cuda() for k, v in f.items()} for f in host]
    b = [{k: torch.from_numpy(v.copy()).cuda() for k, v in f.items()} for f in host]
    torch.cuda.synchronize()
    dt = 1e-3
    rc, st = ctx.solve_level(grids, hp, dt, 0, a, want_stats=True, learned_guess=mode)
    assert rc == capi.OK
    for k, gr in enumerate(grids):
        ctx.solve_ppm_de(gr, hp, dt, 0, b[k], memory=capi.MEM_DEVICE, learned_guess=mode)
    torch.cuda.synchronize()
    for k, gr in enumerate(grids):
        for name in a[k]:
            assert torch.equal(a[k][name], b[k][name]), (k, name)


def test_short_training_reduces_the_loss(ctx, torch):
    samples = LRN.collect(ctx, torch, stride_sod=8, stride_turb=16, capacity=400_000,
                          sod_n=16, turb_n=32, sod_steps=10, turb_steps=8, log=lambda *_: None)
    assert samples.shape[0] > 20000
    _, hist = LRN.train(ctx, torch, samples, epochs=6, batch=4096, lr=2e-3,
                        log=lambda *_: None)
    assert hist[-1] < 0.5 * hist[0], hist
