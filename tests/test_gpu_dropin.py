# SPDX-License-Identifier: Apache-2.0
"""The drop-in surface beyond the step, through the C ABI on the GPU:

- snapshot keys and bitwise replay (the reference's R1, tests/solvers/sph/test_determinism.py:21-33): after 10 steps
  of worlds with spouts and a sink, every ``alloy_state_arrays`` value and the state are saved; 15 steps; restore;
  15 steps again give the same bits, ledger included;
- the port (ports.py): absorb, emit and retire against a host restatement of its per-world stack semantics;
- ``alloy_energy`` and ``alloy_stable_dt`` against host float64 / float32 restatements (runtime.py:55-100, 423-430);
- coupling restarts (coupling_hooks.py:41-72) restore the saved solver state;
- ``notify_model_changed`` leaves a step's bits unchanged.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.build import add_fluid_block, add_particle_box, add_spares
from alloy_b200.solvers.sph.config import PHASE_HELD
from alloy_b200.solvers.sph.model import ModelBuilder
from alloy_b200.solvers.sph.solver import layer_offsets
from alloy_b200.solvers.sph.testing import batched_worlds, benchmark_config, dam_break

pytestmark = pytest.mark.gpu


def _spouts(sc, sol):
    arr = sc.model.host()
    for e in sc.emitters:
        w = e["world"]
        i0 = int(arr["world_start"][w])
        m, rho0 = float(arr["mass"][i0]), float(arr["rest_density"][i0])
        offs = layer_offsets(np.asarray(e["half"], np.float64), np.asarray(e["velocity"], np.float64),
                             sc.config.spacing)
        sol.add_emitter(w, e["centre"], e["half"], len(offs) * (m / rho0) / (5.0 * sc.dt), e["velocity"],
                        pool=e["pool"])


def _run(sol, a, b, steps, dt):
    for _ in range(steps):
        sol.step(a, b, None, None, dt)
        a, b = b, a
    return a, b


def _bits(state) -> bytes:
    return state.particle_q.cpu().numpy().tobytes() + state.particle_qd.cpu().numpy().tobytes()


def test_snapshot_restore_replays_bitwise_with_spouts_and_sink(cuda):
    sc = batched_worlds(worlds=3, lo=400, hi=900, seed=5, device=cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    _spouts(sc, sol)
    h = sc.model.host()
    lo = h["q"][(h["world"] == 1) & (h["phase"] >= 1)].min(0)  # a sink over the bottom corner of world 1's liquid
    sol.add_sink(1, (float(lo[0]) + 0.02, float(lo[1]) + 0.02, float(lo[2]) + 0.01, 0.0, 0.0, 0.0, 1.0),
                 (0.03, 0.03, 0.02))
    a, b = sc.model.state(), sc.model.state()
    a, b = _run(sol, a, b, 10, sc.dt)
    keys = sol.alloy_state_arrays(a)
    for k in ("sph.kappa_v", "sph.kappa_d", "sph.phase", "particle_flags", "sph.mass_in", "sph.mass_out",
              "sph.escaped", "sph.emit_t", "sph.emit_cursor", "sph.port_stack", "sph.port_top"):
        assert k in keys, k
    worlds = sol.alloy_state_worlds()
    assert worlds["sph.emit_t"].shape == keys["sph.emit_t"].shape
    saved = {k: v.clone() for k, v in keys.items()}
    sq, sqd = a.particle_q.clone(), a.particle_qd.clone()
    x, y = _run(sol, a, b, 15, sc.dt)
    first, led1 = _bits(x), sol.mass_ledger()
    assert int(led1["in"].sum()) > int(saved["sph.mass_in"].sum().item())  # the spouts emitted after the snapshot
    assert int(led1["out"][1]) > 0  # the sink retired liquid
    for k, v in sol.alloy_state_arrays(x).items():
        v.copy_(saved[k])
    x.particle_q.copy_(sq)
    x.particle_qd.copy_(sqd)
    x2, _ = _run(sol, x, y, 15, sc.dt)
    assert _bits(x2) == first
    led2 = sol.mass_ledger()
    for k in ("in", "out", "active"):
        np.testing.assert_array_equal(led2[k], led1[k], err_msg=k)


def _port_scene(device):
    cfg = benchmark_config(0.02)
    b = ModelBuilder()
    for w in range(2):
        b.begin_world()
        add_fluid_block(b, cfg, (0.0, 0.0, 0.0), (5, 5, 4 + w), jitter=0.01, seed=w)
        add_spares(b, cfg, 6)
        add_particle_box(b, cfg, (0.0, 0.0, 0.0), (0.2, 0.2, 0.2))
        b.end_world()
    m = b.finalize(device)
    ph = m.sph.phase.cpu().numpy()
    ws = m.particle_world_start.cpu().numpy()
    for w in range(2):  # the second half of each world's spares is the port's reservoir (held particles)
        spares = np.flatnonzero(ph[ws[w]:ws[w + 1]] == 0) + ws[w]
        ph[spares[3:]] = PHASE_HELD
    m.sph.phase.copy_(torch.from_numpy(ph))
    return m, cfg


def test_port_absorb_emit_retire(cuda):
    m, cfg = _port_scene(cuda)
    sol = SolverDFSPH(m, cfg)
    ws = m.particle_world_start.cpu().numpy()
    ph0 = m.sph.phase.cpu().numpy().copy()
    held0 = [list(np.flatnonzero(ph0[ws[w]:ws[w + 1]] == PHASE_HELD) + ws[w]) for w in range(2)]
    assert sol.port.reservoir == sum(len(h) for h in held0) == 6
    np.testing.assert_array_equal(sol.port.counts()["held"], [3, 3])
    a, b = m.state(), m.state()
    a, b = _run(sol, a, b, 3, 1.0e-3)
    led0 = sol.mass_ledger()
    n = m.particle_count
    mask = np.zeros(n, np.int32)
    liquid = [np.flatnonzero(ph0[ws[w]:ws[w + 1]] == 1) + ws[w] for w in range(2)]
    take = [liquid[0][[2, 7, 11]], liquid[1][[0, 5]]]
    for t in take:
        mask[t] = 1
    mask[held0[0][0]] = 1  # not liquid: ignored
    sol.port.absorb(a, torch.from_numpy(mask).to(cuda))
    np.testing.assert_array_equal(sol.port.taken.cpu().numpy(), [3, 2])
    ph, fl = m.sph.phase.cpu().numpy(), m.particle_flags.cpu().numpy()
    for t in take:
        assert np.all(ph[t] == PHASE_HELD) and np.all((fl[t] & 1) == 0)
        assert np.all(a.particle_qd.cpu().numpy()[t] == 0.0)
    mass = m.particle_mass.cpu().numpy()
    fixed = lambda ids: int(sum(int(round(float(mass[i]) * 2.0 ** 40)) for i in ids))  # noqa: E731
    led1 = sol.mass_ledger()
    np.testing.assert_array_equal(led1["out"] - led0["out"], [fixed(take[0]), fixed(take[1])])
    # the stack now holds, top last: the build-time reservoir (popped ascending) then the absorbed ids ascending
    stack = [sorted(held0[w], reverse=True) + sorted(take[w]) for w in range(2)]
    np.testing.assert_array_equal(sol.port.counts()["held"], [len(s) for s in stack])
    R = 4
    pos = torch.zeros((2, R, 3), dtype=torch.float32, device=cuda)
    vel = torch.zeros((2, R, 3), dtype=torch.float32, device=cuda)
    for w in range(2):
        for r in range(R):
            pos[w, r] = torch.tensor([0.05 + 0.02 * r, 0.05, 0.15], device=cuda)
            vel[w, r] = torch.tensor([0.0, 0.0, -0.1 * (r + 1)], device=cuda)
    req = torch.tensor([4, 2], dtype=torch.int32, device=cuda)
    sol.port.emit(a, pos, vel, req)
    np.testing.assert_array_equal(sol.port.granted.cpu().numpy(), [4, 2])
    ph, fl = m.sph.phase.cpu().numpy(), m.particle_flags.cpu().numpy()
    q, qd = a.particle_q.cpu().numpy(), a.particle_qd.cpu().numpy()
    for w in range(2):
        popped = [stack[w][-1 - r] for r in range(int(req[w]))]
        for r, i in enumerate(popped):
            assert ph[i] == 1 and (fl[i] & 1) == 1
            np.testing.assert_array_equal(q[i], pos[w, r].cpu().numpy())
            np.testing.assert_array_equal(qd[i], vel[w, r].cpu().numpy())
    led2 = sol.mass_ledger()
    assert np.all(led2["active"] + led2["out"] == led2["initial"] + led2["in"])
    mask[:] = 0
    gone = liquid[1][[1, 2, 3]]
    mask[gone] = 1
    sol.retire(a, torch.from_numpy(mask).to(cuda))
    ph = m.sph.phase.cpu().numpy()
    assert np.all(ph[gone] == -2)
    np.testing.assert_array_equal(sol.port.counts()["retired"], [0, 3])
    a, b = _run(sol, a, b, 3, 1.0e-3)  # the step runs on the changed liquid
    led3 = sol.mass_ledger()
    np.testing.assert_array_equal(led3["active"] + led3["out"], led3["initial"] + led3["in"])
    sol.reset(a)
    np.testing.assert_array_equal(sol.port.counts()["held"], [3, 3])
    np.testing.assert_array_equal(m.sph.phase.cpu().numpy(), ph0)


def test_energy_and_stable_dt(cuda):
    sc = batched_worlds(worlds=3, lo=400, hi=900, seed=2, device=cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    a, b = sc.model.state(), sc.model.state()
    a, b = _run(sol, a, b, 20, sc.dt)
    W = sc.model.world_count
    z_ref = torch.tensor([0.0, 0.01, -0.02], dtype=torch.float64, device=cuda)
    e = torch.zeros(W, dtype=torch.float64, device=cuda)
    sol.alloy_energy(a, z_ref, e)
    h = sc.model.host()
    q, qd = a.particle_q.cpu().numpy(), a.particle_qd.cpu().numpy()
    fl, ph = sc.model.particle_flags.cpu().numpy(), sc.model.sph.phase.cpu().numpy()
    live = ((fl & 1) != 0) & (ph >= 1)
    want = np.zeros(W)
    for i in np.flatnonzero(live):
        w = h["world"][i]
        g = h["gravity"][w].astype(np.float32)
        v = qd[i]
        dz = np.float32(np.float64(q[i, 2]) - z_ref[w].item())
        vv = np.float32(np.float32(v[0] * v[0]) + np.float32(v[1] * v[1])) + np.float32(v[2] * v[2])
        gd = np.float32(np.float32(g[0] * q[i, 0]) + np.float32(g[1] * q[i, 1])) + np.float32(g[2] * dz)
        want[w] += float(h["mass"][i]) * (0.5 * float(vv) - float(gd))
    np.testing.assert_allclose(e.cpu().numpy(), want, rtol=1e-12, atol=1e-15)
    out = torch.zeros(W, dtype=torch.float32, device=cuda)
    sol.alloy_stable_dt(a, None, out)
    cfg = sc.config
    for w in range(W):
        sel = live & (h["world"] == w)
        v = float(np.max(np.linalg.norm(qd[sel].astype(np.float64), axis=1)))
        dt = cfg.dt_max if v <= 0 else min(max(cfg.cfl * cfg.spacing / v, cfg.dt_min), cfg.dt_max)
        assert abs(out[w].item() - dt) <= 1e-6 * dt, (w, out[w].item(), dt)
    rest = sc.model.state()
    rest.particle_qd.zero_()
    sol.alloy_stable_dt(rest, None, out)
    np.testing.assert_array_equal(out.cpu().numpy(), np.full(W, cfg.dt_max, np.float32))


def test_coupling_restart_and_model_notification(cuda):
    sc = dam_break(counts=(8, 8, 8), box=(0.3, 0.3, 0.3), device=cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    a, b = sc.model.state(), sc.model.state()
    a, b = _run(sol, a, b, 5, sc.dt)
    sol.coupling_notify_input_state_update(a, 3)  # exchange start: save
    kv = sol.alloy_state_arrays()["sph.kappa_v"].clone()
    sq, sqd = a.particle_q.clone(), a.particle_qd.clone()
    x, y = _run(sol, a, b, 3, sc.dt)
    first = _bits(x)
    assert not torch.equal(sol.alloy_state_arrays()["sph.kappa_v"], kv)
    sol.coupling_notify_input_state_update(x, 3, iteration_restart=True)  # a second pass of the same exchange
    assert torch.equal(sol.alloy_state_arrays()["sph.kappa_v"], kv)
    x.particle_q.copy_(sq)
    x.particle_qd.copy_(sqd)
    sol.notify_model_changed(0xFFFF)
    x2, _ = _run(sol, x, y, 3, sc.dt)
    assert _bits(x2) == first
    assert sol.coupling_prepare_proxy_contacts(x2, None) is None
    with pytest.raises(ValueError):
        sol.coupling_harvest_proxy_particle_forces(torch.zeros(3, dtype=torch.int32), None, dt=sc.dt)


def _patch_scene(device):
    cfg = benchmark_config(0.02)
    b = ModelBuilder()
    for w in range(3):
        b.begin_world()
        add_fluid_block(b, cfg, (0.0, 0.0, 0.0), (5, 5, 4), jitter=0.01, seed=w)
        add_spares(b, cfg, 12)
        add_particle_box(b, cfg, (0.0, 0.0, 0.0), (0.2, 0.2, 0.3))
        b.end_world()
    return b.finalize(device), cfg


def test_patch_emitter_trigger_fire_reset(cuda):
    """patch.py: spares reserved at registration (the lowest free ids), nothing before a trigger, one emission per
    armed world at the end of the next step (points, velocity, ACTIVE, liquid, ledger), later triggers of a fired
    world ignored, reset re-arms; the pending and fired flags are snapshot keys."""
    m, cfg = _patch_scene(cuda)
    sol = SolverDFSPH(m, cfg)
    W = 3
    ws = m.particle_world_start.cpu().numpy()
    ph0 = m.sph.phase.cpu().numpy().copy()
    spare = [np.flatnonzero(ph0[ws[w]:ws[w + 1]] == 0) + ws[w] for w in range(W)]
    pts = [np.array([[0.05 + 0.02 * k, 0.1, 0.2] for k in range(5)], np.float32), np.zeros((0, 3), np.float32),
           np.array([[0.1, 0.05 + 0.02 * k, 0.22] for k in range(3)], np.float32)]
    pid = sol.add_patch_emitter([True, True, True], -1, pts, velocity=(0.0, 0.1, -0.5))
    assert pid == 0
    with pytest.raises(ValueError, match="body indices"):
        sol.add_patch_emitter([True, False, False], 0, pts)
    with pytest.raises(Exception, match="free spares"):
        sol.add_patch_emitter([True, False, False], -1, [np.zeros((8, 3), np.float32), [], []])
    a, b = m.state(), m.state()
    a, b = _run(sol, a, b, 2, 1.0e-3)
    np.testing.assert_array_equal(m.sph.phase.cpu().numpy()[spare[0]], 0)  # not triggered: nothing emitted
    led0 = sol.mass_ledger()
    sol.trigger(pid, torch.tensor([1, 1, 0], dtype=torch.int32, device=cuda))
    keys = sol.alloy_state_arrays()
    np.testing.assert_array_equal(keys["sph.patch_pending0"].cpu().numpy(), [1, 0])  # entries: worlds 0 and 2
    a, b = _run(sol, a, b, 1, 1.0e-3)
    ph, fl = m.sph.phase.cpu().numpy(), m.particle_flags.cpu().numpy()
    got = spare[0][:5]
    assert np.all(ph[got] == 1) and np.all((fl[got] & 1) == 1) and np.all(ph[spare[0][5:]] == 0)
    np.testing.assert_array_equal(a.particle_q.cpu().numpy()[got], pts[0])
    np.testing.assert_array_equal(a.particle_qd.cpu().numpy()[got], np.tile(np.float32([0.0, 0.1, -0.5]), (5, 1)))
    mass = m.particle_mass.cpu().numpy()
    led1 = sol.mass_ledger()
    assert int(led1["in"][0] - led0["in"][0]) == sum(int(round(float(mass[i]) * 2.0 ** 40)) for i in got)
    np.testing.assert_array_equal(led1["in"][1:], led0["in"][1:])
    keys = sol.alloy_state_arrays()
    np.testing.assert_array_equal(keys["sph.patch_pending0"].cpu().numpy(), [0, 0])
    np.testing.assert_array_equal(keys["sph.patch_fired0"].cpu().numpy(), [1, 0])
    np.testing.assert_array_equal(sol.alloy_state_worlds()["sph.patch_fired0"].cpu().numpy(), [0, 2])
    sol.trigger(pid, torch.tensor([True, False, True], device=cuda))  # world 0 fired already: ignored
    a, b = _run(sol, a, b, 1, 1.0e-3)
    ph = m.sph.phase.cpu().numpy()
    assert np.all(ph[spare[2][:3]] == 1) and np.all(ph[spare[2][3:]] == 0)
    led2 = sol.mass_ledger()
    np.testing.assert_array_equal(led2["in"][0], led1["in"][0])
    np.testing.assert_array_equal(led2["active"] + led2["out"], led2["initial"] + led2["in"])
    sol.reset(a, torch.tensor([1, 0, 0], dtype=torch.uint8))
    np.testing.assert_array_equal(sol.alloy_state_arrays()["sph.patch_fired0"].cpu().numpy(), [0, 1])
    with pytest.raises(ValueError, match="no patch emitter"):
        sol.trigger(5, torch.zeros(3, dtype=torch.int32, device=cuda))
