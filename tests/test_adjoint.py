"""The adjoint of the differentiable step (sph_diff_*), on the GPU.

The gradients of a loss on the final state with respect to k_n, k_t,
gamma_n, per-particle and global friction and the starting state are checked
against central finite differences of the same FP64 forward (h = 1e-6
relative), over runs spanning several checkpoint segments on scenes where
contacts stick and slide."""
import numpy as np
import pytest
import torch

from sphere_b200 import adjoint, scenes
from sphere_b200.sphk import SphError, Simulation
from sphere_b200.state import config_from_spherebin, state_from_spherebin

pytestmark = pytest.mark.gpu

STEPS, K = 24, 10


def _scene():
    sb = scenes.collision(n=400, seed=91, periodic=0, vmax=0.2, wmax=50.0)
    sb.mu_s = sb.mu_d = 0.3
    return sb


def _weights(sb, seed=5):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(sb.np, 3)), rng.normal(size=(sb.np, 3)) * 1e-3


def _loss(sb, st, wx, wv):
    # displacements, not absolute positions, keep the sum's rounding far
    # below the finite-difference signal
    return float(np.sum(wx * (st.x[:, :3] - sb.x)) + np.sum(wv * st.vel[:, :3]))


def _run(sb, k_n, k_t, g_n, mu_p, K=K):
    sim, st = adjoint.run_forward(sb, STEPS, k_n, k_t, g_n, mu_p, checkpoint_every=K)
    return sim, st


@pytest.fixture(scope="module")
def grads():
    sb = _scene()
    wx, wv = _weights(sb)
    mu_p = np.full(sb.np, 0.3) + np.random.default_rng(6).uniform(-0.05, 0.05, sb.np)
    sim, st = _run(sb, sb.k_n, sb.k_t, sb.gamma_n, mu_p)
    g = sim.diff_backward(wx, wv)
    after = sim.download()
    sim.close()
    return dict(sb=sb, wx=wx, wv=wv, mu_p=mu_p, g=g, st=st, after=after)


def _fd(G, which, h_rel=1e-6, idx=None):
    sb, wx, wv, mu_p = G["sb"], G["wx"], G["wv"], G["mu_p"]
    th = dict(k_n=sb.k_n, k_t=sb.k_t, gamma_n=sb.gamma_n)
    vals = []
    for sgn in (1.0, -1.0):
        t = dict(th)
        m = mu_p.copy()
        if which in th:
            h = h_rel * th[which]
            t[which] = th[which] + sgn * h
        elif which == "mu_i":
            h = h_rel * mu_p[idx]
            m[idx] += sgn * h
        else:   # every particle's friction
            h = h_rel * 0.3
            m = m + sgn * h
        sim, st = _run(sb, t["k_n"], t["k_t"], t["gamma_n"], m)
        sim.close()
        vals.append(_loss(sb, st, wx, wv))
    return (vals[0] - vals[1]) / (2 * h)


@pytest.mark.parametrize("which", ["k_n", "k_t", "gamma_n"])
def test_parameter_gradients_match_central_differences(grads, which):
    fd = _fd(grads, which)
    got = grads["g"][which]
    assert fd != 0.0
    assert abs(got - fd) <= 1e-6 * abs(fd) + 1e-12 * abs(got), (got, fd)


def test_friction_gradients_match_central_differences(grads):
    g = grads["g"]["mu"]
    # particles whose friction matters most, and the global coefficient
    for i in np.argsort(-np.abs(g))[:3]:
        fd = _fd(grads, "mu_i", idx=int(i))
        assert abs(g[i] - fd) <= 1e-6 * abs(fd), (i, g[i], fd)
    fd = _fd(grads, "mu_all")
    assert abs(g.sum() - fd) <= 1e-6 * abs(fd), (g.sum(), fd)


def test_backward_leaves_the_state_as_it_was(grads):
    st, after = grads["st"], grads["after"]
    for f in ("x", "vel", "angvel", "vel0", "angvel0", "delta_t", "contacts"):
        assert np.array_equal(getattr(st, f), getattr(after, f)), f


def test_checkpoint_interval_does_not_change_gradients(grads):
    sb = grads["sb"]
    sim, _ = _run(sb, sb.k_n, sb.k_t, sb.gamma_n, grads["mu_p"], K=STEPS)
    g = sim.diff_backward(grads["wx"], grads["wv"])
    sim.close()
    for k in ("k_n", "k_t", "gamma_n"):
        assert abs(g[k] - grads["g"][k]) <= 1e-12 * abs(g[k]), k
    assert np.allclose(g["mu"], grads["g"]["mu"], rtol=1e-10, atol=1e-12 * np.abs(g["mu"]).max())


def test_repeated_iterations_on_a_callers_stream_give_the_same_gradients(grads):
    """A calibration loop in one context: the second forward reuses the
    checkpoint buffers of the first, and both run on a stream of the
    caller's, in pieces that do not line up with the checkpoint interval."""
    sb, wx, wv = grads["sb"], grads["wx"], grads["wv"]
    sim = Simulation(adjoint._scene_config(sb, sb.k_n, sb.k_t, sb.gamma_n))
    s = torch.cuda.Stream()
    try:
        for _ in range(2):
            sim.upload(state_from_spherebin(sb))
            sim.diff_begin(mu=grads["mu_p"], checkpoint_every=K)
            for n in (7, 9, STEPS - 16):
                sim.step(n, stream=s.cuda_stream)
            s.synchronize()
            sim.sync()
            st = sim.download()
            assert np.array_equal(st.x, grads["st"].x)
            g = sim.diff_backward(wx, wv)
            sim.diff_end()
            # the reverse pass adds partners' adjoints atomically, so only
            # the order of those additions may differ
            for k in ("k_n", "k_t", "gamma_n"):
                assert abs(g[k] - grads["g"][k]) <= 1e-12 * abs(g[k]), k
            assert np.allclose(g["mu"], grads["g"]["mu"], rtol=1e-10,
                               atol=1e-12 * np.abs(g["mu"]).max())
    finally:
        sim.close()


def test_autograd_function_gives_the_same_gradients(grads):
    sb, wx, wv = grads["sb"], grads["wx"], grads["wv"]
    kn = torch.tensor(sb.k_n, dtype=torch.float64, requires_grad=True)
    kt = torch.tensor(sb.k_t, dtype=torch.float64, requires_grad=True)
    gn = torch.tensor(sb.gamma_n, dtype=torch.float64, requires_grad=True)
    mu = torch.tensor(0.3, dtype=torch.float64, requires_grad=True)
    dmu = torch.tensor(grads["mu_p"] - 0.3, dtype=torch.float64, requires_grad=True)
    x, v = adjoint.simulate(sb, STEPS, kn, kt, gn, mu, dmu, checkpoint_every=K)
    loss = (torch.from_numpy(wx) * (x - torch.from_numpy(sb.x))).sum() + (torch.from_numpy(wv) * v).sum()
    loss.backward()
    g = grads["g"]
    assert abs(kn.grad.item() - g["k_n"]) <= 1e-12 * abs(g["k_n"])
    assert abs(gn.grad.item() - g["gamma_n"]) <= 1e-12 * abs(g["gamma_n"])
    assert np.allclose(dmu.grad.numpy(), g["mu"], rtol=1e-10, atol=1e-14)
    assert abs(mu.grad.item() - g["mu"].sum()) <= 1e-10 * abs(g["mu"].sum())


def test_height_profile_loss_backpropagates():
    sb = _scene()
    kn = torch.tensor(sb.k_n, dtype=torch.float64, requires_grad=True)
    mu = torch.tensor(0.3, dtype=torch.float64, requires_grad=True)
    x, _ = adjoint.simulate(sb, 12, kn, sb.k_t, sb.gamma_n, mu, checkpoint_every=5)
    h = adjoint.height_profile(x, sb.radius, 0.0, float(sb.L[0]), bins=16)
    target = torch.from_numpy(np.random.default_rng(3).uniform(0.02, 0.04, 16))
    loss = ((h - target) ** 2).mean()
    loss.backward()
    assert torch.isfinite(kn.grad) and torch.isfinite(mu.grad)


@pytest.mark.parametrize("patch", [dict(contactmodel=1), dict(nw=1)], ids=["model1", "walls"])
def test_differentiable_mode_rejects_unsupported_scenes(patch):
    sb = scenes.collision(n=200, seed=92, periodic=0, nw=patch.get("nw", 0))
    if "contactmodel" in patch:
        sb.contactmodel = patch["contactmodel"]
    with Simulation(config_from_spherebin(sb)) as sim:
        sim.upload(state_from_spherebin(sb))
        with pytest.raises(SphError) as e:
            sim.diff_begin()
        assert e.value.code == -5
