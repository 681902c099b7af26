# SPDX-License-Identifier: Apache-2.0
"""The learned warm start inside the solver: feature recording leaves the step bit-exact, a network that predicts
badly is rejected by the first-sweep judge in every world (so the step stays bit-exact against the oracle) and is then
evaluated at doubling intervals, the
solver's in-step predictions equal the standalone tensor-core inference on the same features, and a trained network
keeps every step at the solver's tolerance."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.testing import batched_worlds, dam_break
from alloy_b200.solvers.sph.warmstart import Network, WarmModel, collect_pairs, init_params, statistics, train
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


def _scene(cuda):
    return dam_break(counts=(12, 10, 14), box=(0.5, 0.4, 0.6), device=cuda)


def _run_against_oracle(sc, sol, steps):
    orc = Oracle(sc.model.host(), sc.config)
    a, b = sc.model.state(), sc.model.state()
    for k in range(steps):
        sol.step(a, b, None, None, sc.dt)
        a, b = b, a
        orc.step(sc.dt)
        q, qd = orc.state()
        np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q, err_msg=f"q step {k}")
        np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), qd, err_msg=f"qd step {k}")
        rep, orep = sol.report(), orc.report()
        assert rep.iters_density[0] == orep["iters_density"][0], k
        assert rep.iters_divergence[0] == orep["iters_divergence"][0], k
    return a, b


def test_feature_recording_keeps_the_step_bit_exact(cuda):
    sc = _scene(cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    sol.record_features(True)
    _run_against_oracle(sc, sol, 8)
    f = sol.warm_features().cpu().numpy()
    live = f[:, 1] > 0  # n_eff / n_full of liquid particles
    assert live.sum() == sc.fluid_count and np.isfinite(f).all()
    np.testing.assert_array_equal(f[live, 0], sol.debug_field("ratio")[live] - np.float32(1.0))
    np.testing.assert_array_equal(f[live, 1], sol.debug_field("neff")[live] / np.float32(sol.hc.n_full))
    np.testing.assert_array_equal(f[live, 5], sol.debug_field("alpha")[live])


def test_a_bad_network_is_rejected_and_the_step_stays_plain(cuda):
    """A network whose predictions sit at the cap leaves a larger first-sweep residual than the plain start in every
    world and solve, so each solve continues exactly as the plain solver (bit for bit against the oracle)."""
    sc = _scene(cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    p = init_params(0)
    p[-2:] = 50.0  # output biases: far above any converged kappa
    bad = WarmModel(p, np.zeros(16, np.float32), np.ones(16, np.float32), np.ones(2, np.float32),
                    np.ones(2, np.float32))
    sol.set_warm_model(bad)
    _run_against_oracle(sc, sol, 10)
    d = sol.diagnostics()
    assert d["learned_divergence"].sum() == 0 and d["learned_density"].sum() == 0
    # rejected at steps 1, 3 and 7 (gaps 2, 4, 8 between evaluations), not evaluated at the other steps
    keys = sol.alloy_state_arrays()
    np.testing.assert_array_equal(keys["sph.warm_probe_gap"].cpu().numpy(), [8, 8])
    np.testing.assert_array_equal(keys["sph.warm_probe_wait"].cpu().numpy(), [4, 4])
    pk = sol.debug_field("pred_kd")
    assert (pk[: sc.fluid_count] > 1.0).all()  # the predictions really were at the cap


def test_in_step_predictions_equal_standalone_inference(cuda):
    sc = batched_worlds(worlds=5, lo=800, hi=3000, seed=2, device=cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    a, b = sc.model.state(), sc.model.state()
    sol.record_features(True)
    for _ in range(3):
        sol.step(a, b, None, None, sc.dt)
        a, b = b, a
    f = sol.warm_features()
    live = f[:, 1] > 0
    mu, sd = statistics(f[live].cpu().numpy())
    rng = np.random.default_rng(5)
    p = init_params(4)
    p[-130:-2] = rng.normal(0, 0.3, 128)
    model = WarmModel(p, mu, sd, np.array([1e-4, 1e-6], np.float32), np.array([2e-4, 3e-6], np.float32))
    sol.set_warm_model(model)
    sol.step(a, b, None, None, sc.dt)
    a, b = b, a
    f = sol.warm_features()
    live = (f[:, 1] > 0).cpu().numpy()
    net = Network(p)
    finv = torch.from_numpy(model.norm_vector()[16:32]).to(cuda)  # the solver multiplies by 1 / deviation
    x = ((f - torch.from_numpy(mu).to(cuda)) * finv).contiguous()
    y = net.forward(x).cpu().numpy()
    torch.cuda.synchronize()
    y = y * model.t_std + model.t_mean
    for k, name in enumerate(("pred_kv", "pred_kd")):
        got = sol.debug_field(name)[live]
        ref = y[live, k]
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-4 * float(np.abs(ref).max()), err_msg=name)
    net.status()


def test_trained_network_keeps_every_step_at_tolerance(cuda):
    """Train on the plain solver's pairs from one seed, run another seed with the learned start: every solve
    converges to the same tolerance (or stops at max_iterations, never earlier) and the state stays close to the
    plain run of the same seed (within the drift the tolerance itself allows)."""
    train_sc = batched_worlds(worlds=6, lo=1000, hi=4000, seed=11, device=cuda)
    sol = SolverDFSPH(train_sc.model, train_sc.config)
    f, t, _, _ = collect_pairs(sol, train_sc.model.state(), train_sc.model.state(), train_sc.dt, 40, every=2)
    model = train(f, t, epochs=20, batch=8192, lr=1e-3)
    assert np.isfinite(model.params).all()

    runs = {}
    for learned in (False, True):
        sc = batched_worlds(worlds=6, lo=1000, hi=4000, seed=12, device=cuda)
        s = SolverDFSPH(sc.model, sc.config)
        if learned:
            s.set_warm_model(model)
        a, b = sc.model.state(), sc.model.state()
        its, chose = [], 0
        for _ in range(30):
            s.step(a, b, None, None, sc.dt)
            a, b = b, a
            r = s.report()
            tol = sc.config.max_density_error
            conv = (r.density_err <= tol) | (r.iters_density >= sc.config.max_iterations)
            assert conv.all(), r.density_err
            its.append(int(r.iters_density.sum() + r.iters_divergence.sum()))
            d = s.diagnostics()
            chose += int(d["learned_density"].sum() + d["learned_divergence"].sum())
        runs[learned] = (a.particle_q.cpu().numpy(), its, chose)
    q0, it0, _ = runs[False]
    q1, it1, chose = runs[True]
    # both runs meet the density tolerance every step, so they differ by the tolerance's own drift: a few hundredths
    # of a spacing on average after 30 steps, a fraction of one at the splashiest particle
    dq = np.linalg.norm(q1 - q0, axis=1)
    h = train_sc.config.spacing
    assert dq.mean() < 0.05 * h and dq.max() < 0.5 * h, (dq.mean() / h, dq.max() / h)
    print(f"iterations plain {sum(it0)} learned {sum(it1)}; learned start kept in {chose} of {30 * 6 * 2} solves")
