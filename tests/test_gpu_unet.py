"""The learned initial guess on the GPU: tensor-core convolution forward and
backward against the float64 CPU oracle of the network (activations layer by
layer, parameter gradients), and online training inside the PIC loop next to
the reference's warm start and the per-solve history start."""
import numpy as np
import pytest

import unet_ref
from fopis_b200 import RootGrid, _abi, config
from fopis_b200.config import SpeciesInfo, make_params, plasma_units

pytestmark = pytest.mark.gpu

SLOTS = ["x0", "e0", "d1", "e1", "d2", "e2", "e3", "u1", "a4", "u0", "a5"]


def small_cfg(n, boundary):
    dx, dt = plasma_units()
    sp = [SpeciesInfo("Electron", "ambient", 1.0, -1.0, 1e7, 1.0, 1),
          SpeciesInfo("Ion", "ambient", 100.0, 1.0, 1e7, 1.0, 1)]
    p, norm = make_params((n, n, n), boundary, dx, dt, sp, seed=77)
    return config.SimConfig(params=p, norm=norm, species=sp, objects=[])


def fields(shape, seed):
    rng = np.random.default_rng(seed)
    x = np.linspace(0, 2 * np.pi, shape[0])
    smooth = np.sin(x)[:, None, None] * np.cos(2 * x)[None, :, None] * np.sin(3 * x)[None, None, :]
    rho0 = rng.normal(0.0, 1.0, shape) * 1e-12 + 3e-12 * smooth
    phi1 = 0.3 * smooth + 0.01 * rng.normal(0.0, 1.0, shape)
    phi2 = phi1 - 0.02 * np.roll(smooth, 1, axis=0) - 0.002 * rng.normal(0.0, 1.0, shape)
    tgt = phi1 + 0.015 * np.roll(smooth, 2, axis=1) + 0.003 * rng.normal(0.0, 1.0, shape)
    return rho0, phi1, phi2, tgt


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.fixture(scope="module", params=[(16, "PPPPPP"), (21, "DDDDDD")], ids=["periodic16", "dirichlet21"])
def evaluated(request, gpu_available):
    n, bnd = request.param
    cfg = small_cfg(n, bnd)
    g = RootGrid(cfg)
    rho0, phi1, phi2, tgt = fields(g.shape, 5)
    prm = g.unet_params()
    # non-zero biases and a larger head so that every path carries signal
    rng = np.random.default_rng(3)
    lay, _, total = unet_ref.param_layout()
    for w, b, cin, cout in lay:
        prm[b:b + cout] = rng.normal(0.0, 0.05, cout).astype(np.float32)
    prm[total - 17:] = rng.normal(0.0, 0.3, 17).astype(np.float32)
    g.unet_params(prm)
    pred, loss, grad = g.unet_eval(rho0, phi1, phi2, tgt)
    acts = {name: g.unet_tensor(i) for i, name in enumerate(SLOTS)}
    out = g.unet_tensor(24)
    ref = unet_ref.evaluate(cfg.params, prm, rho0, phi1, phi2, tgt)
    g.close()
    return dict(cfg=cfg, pred=pred, loss=loss, grad=grad, acts=acts, out=out, ref=ref)


def test_forward_activations_match_oracle(evaluated):
    ref = evaluated["ref"]["act"]
    for name in SLOTS:
        r = ref[name]                                   # [ch, n0, n1, n2]
        gpu = evaluated["acts"][name].reshape(r.shape[1:] + (r.shape[0],)).transpose(3, 0, 1, 2)
        assert rel(gpu, r) < 2e-2, (name, rel(gpu, r))
    o = ref["out"]
    assert rel(evaluated["out"].reshape(o.shape), o) < 2e-2


def test_prediction_and_loss_match_oracle(evaluated):
    ref = evaluated["ref"]
    cfg = evaluated["cfg"]
    _, _, _, I = unet_ref.features(cfg.params, *([np.zeros(evaluated["pred"].shape)] * 3))
    assert rel(evaluated["pred"][I], ref["pred"]) < 2e-2
    assert abs(evaluated["loss"] - ref["loss"]) <= 2e-2 * ref["loss"]


def test_gradients_match_oracle(evaluated):
    ref = evaluated["ref"]["grad"]
    gpu = evaluated["grad"]
    lay, _, total = unet_ref.param_layout()
    for l, (w, b, cin, cout) in enumerate(lay):
        e = 27 * cin * cout
        assert rel(gpu[w:w + e], ref[w:w + e]) < 5e-2, ("W", l, rel(gpu[w:w + e], ref[w:w + e]))
        assert rel(gpu[b:b + cout], ref[b:b + cout]) < 5e-2, ("b", l, rel(gpu[b:b + cout], ref[b:b + cout]))
    assert rel(gpu[total - 17:], ref[total - 17:]) < 2e-2


def lockstep(cfg_fn, steps_train, steps_use, with_objects):
    """Three contexts with the same seed stepped together: A starts every solve
    from the current phi (the reference's warm start), B from the per-solve
    history, C trains its network on its own first solves and then seeds them
    with the network's increment on top of the history start."""
    gs = [RootGrid(cfg_fn()) for _ in range(3)]
    for g in gs:
        if with_objects:
            g.initializeObjectsCmatrix(0)
        g.generate_ambient()
        g.initialize()
    gs[1].set_guess_mode(_abi.GUESS_HISTORY)
    gs[2].set_guess_mode(_abi.GUESS_HISTORY)
    gs[2].unet_training(True, 1e-3)
    rec = []
    for t in range(steps_train + steps_use):
        if t == steps_train:
            gs[2].set_guess_mode(_abi.GUESS_LEARNED)
        for g in gs:
            g.mainLoopES(1)
        st = [g.stats() for g in gs]
        warm, guess, msf, mst = gs[2].unet_last()
        rec.append(dict(c=[x.vcycles_step for x in st], used=st[2].learned_used, loss=gs[2].unet_state()[0],
                        warm=warm, guess=guess, msf=msf, mst=mst))
    out = dict(rec=rec, policy=gs[2].unet_policy())
    if with_objects:
        out["V"] = [g.getObject(0)[0] for g in gs]
    out["energy"] = [g.getEnergy() for g in gs]
    for g in gs:
        g.close()
    return out


def report(name, r, steps_train):
    use = r["rec"][steps_train:]
    c = np.mean([x["c"] for x in use], axis=0)
    ratio = [x["guess"] / x["warm"] for x in use if x["used"] and x["warm"] > 0]
    loss = np.array([x["loss"] for x in r["rec"]])
    print(f"\n{name}: V-cycles/step warm {c[0]:.2f} history {c[1]:.2f} learned {c[2]:.2f}; guess/history "
          f"residual {np.median(ratio) if ratio else float('nan'):.3f} over {len(ratio)} used steps; loss "
          f"{loss[2]:.3g} -> {loss[steps_train - 1]:.3g}; forward {r['rec'][-1]['msf']:.3f} ms, train "
          f"{r['rec'][steps_train - 1]['mst']:.3f} ms; policy {r['policy']}")
    return c, ratio, loss


def test_online_training_periodic(gpu_available):
    """Stationary periodic plasma (one solve per step, where the history start
    is the warm start): the loss falls while training on the solver's own
    pairs, a used guess always lowers the initial residual (per-step guard) and
    the V-cycles never exceed the history start's by more than one."""
    r = lockstep(lambda: config.workload("periodic32", ppc=8), 60, 30, False)
    c, ratio, loss = report("periodic32", r, 60)
    assert np.mean(loss[50:60]) < np.mean(loss[2:12])
    assert all(x < 1.0 for x in ratio)
    assert c[2] <= c[1] + 1.0
    (pa, fa) = r["energy"][0]
    for (pb, fb) in r["energy"][1:]:
        assert abs(fb - fa) <= 1e-3 * fa and abs(pb - pa) <= 1e-4 * pa


def test_history_and_learned_starts_keep_spacecraft_potential(gpu_available):
    """cube64 with a conductor: the history start needs fewer V-cycles than the
    reference's warm start at the same tolerance, the learned guess no more than
    the history start (+1), and all three keep the spacecraft potential within
    1 % of the warm-start run."""
    r = lockstep(lambda: config.workload("cube64", ppc=8), 60, 40, True)
    Va = r["V"][0]
    for Vb in r["V"][1:]:
        assert abs(Vb - Va) <= 0.01 * abs(Va)
    c, ratio, loss = report("cube64", r, 60)
    assert c[1] < c[0]
    assert c[2] <= c[1] + 1.0
