"""The learned initial guess on the GPU: the CUDA forward/backward kernels against
the CPU oracle (oracle/gnn_oracle.py, itself checked by finite differences), and
what the trained network gains over Newton's previous-step start."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _small():
    from adh_kraken_b200.mesh import small_delaunay_case
    return small_delaunay_case(n=12, seed=3, nsteps=1)


def test_forward_and_gradients_match_oracle():
    import torch
    from adh_kraken_b200 import learned
    from oracle import gnn_oracle as go
    case = _small()
    n = case.nnodes
    gcpu = go.graph_arrays(case.xyz[:, :2], case.tri)
    graph = learned.DeviceGraph(learned.build_graph(case.xyz[:, :2], case.tri))
    rng = np.random.default_rng(0)
    net = learned.Net(seed=1)
    p = rng.normal(0, 0.15, net.P).astype(np.float32)
    net.w.copy_(torch.tensor(p)); net.sync_bf16()
    F = rng.normal(0, 1, (n, 8)).astype(np.float32)
    T = rng.normal(0, 1, (n, 3)).astype(np.float32)
    M = (rng.uniform(size=n) > 0.2).astype(np.float32)
    ws = learned.Workspace(n, train=True)
    ws.F.copy_(torch.tensor(F)); ws.T.copy_(torch.tensor(T)); ws.M.copy_(torch.tensor(M))
    learned.forward(net, graph, ws, train=True)
    k = learned._L().sw2n_mse(n, learned._p(ws.Y), learned._p(ws.T), learned._p(ws.M), learned._p(ws.dY),
                              learned._p(ws.lpart), None)
    learned.backward(net, graph, ws)
    torch.cuda.synchronize()
    loss_ref, g_ref, Y_ref = go.loss_and_grad(p, gcpu, F, T, bf16=True, M=M)
    Y = ws.Y.cpu().numpy(); g = net.g.cpu().numpy()
    assert np.abs(Y - Y_ref).max() <= 1e-4 * max(1.0, np.abs(Y_ref).max())
    assert abs(float(ws.lpart[:k].sum()) - loss_ref) <= 1e-4 * loss_ref
    # FP32 accumulation in a different order (and fast exp) against numpy: relative 1e-3 of the largest entry
    assert np.abs(g - g_ref).max() <= 1e-3 * np.abs(g_ref).max(), np.abs(g - g_ref).max()


def test_features_targets_and_guess_match_oracle():
    import torch
    from adh_kraken_b200 import learned
    from oracle import gnn_oracle as go
    case = _small()
    n = case.nnodes
    rng = np.random.default_rng(2)
    s0 = case.sol0 + rng.normal(0, 0.01, 3 * n)
    s1 = s0 + rng.normal(0, 0.01, 3 * n)
    s2 = s1 + rng.normal(0, 0.01, 3 * n)
    mu = rng.normal(0, 1, 8).astype(np.float32); sd = rng.uniform(0.5, 2, 8).astype(np.float32)
    scale = np.array([0.01, 0.02, 0.03], np.float32)
    d = lambda a: torch.tensor(a, device="cuda")
    S0, S1, S2, z = d(s0), d(s1), d(s2), d(case.xyz[:, 2].copy())
    Fd = torch.zeros(n, 8, device="cuda"); Td = torch.zeros(n, 3, device="cuda"); Md = torch.zeros(n, device="cuda")
    MU, SD, SC = d(mu), d(sd), d(scale)      # kept alive while the kernels use them
    Ld = learned._L(); P = learned._p
    Ld.sw2n_features(n, P(S1), P(S0), P(z), P(MU), P(SD), P(Fd), None)
    Ld.sw2n_targets(n, P(S2), P(S1), P(S0), P(SC), 0.05, P(Td), P(Md), None)
    Y = torch.tensor(rng.normal(0, 1, (n, 3)).astype(np.float32), device="cuda")
    G = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    Ld.sw2n_apply_guess(n, P(S1), P(S0), P(Y), P(SC), 0.05, P(G), None)
    torch.cuda.synchronize()
    assert np.allclose(Fd.cpu().numpy(), go.features(s1, s0, case.xyz[:, 2], mu, sd), rtol=1e-6, atol=1e-6)
    T_ref, M_ref = go.targets(s2, s1, s0, scale, 0.05)
    assert np.allclose(Td.cpu().numpy(), T_ref, rtol=1e-6, atol=1e-6)
    assert np.array_equal(Md.cpu().numpy(), M_ref)
    ref = (2 * s1 - s0 + (Y.cpu().numpy().astype(np.float64) * scale.astype(np.float64)).ravel()).reshape(-1, 3)
    keep = (s1[0::3] <= 0.05) | (ref[:, 0] <= 0.05)
    ref[keep] = s1.reshape(-1, 3)[keep]
    assert keep.any() and not keep.all()
    assert np.allclose(G.cpu().numpy(), ref.ravel(), rtol=1e-14, atol=1e-14)


def test_trained_guess_beats_previous_step_start():
    """Train on solver trajectories of a small beach strip, then solve held-out steps
    from the same states with and without the guess at identical Newton settings.
    Measured on this strip: where taken, the guess halves the initial residual, but
    Newton from it needs more Krylov iterations than from the previous step."""
    from adh_kraken_b200 import learned
    from adh_kraken_b200.capi import default_opts
    from adh_kraken_b200.timeloop import SW2Simulation
    case = learned.beach_strip(ny=12, nx=400, nsteps=40, seed=5)
    opts = default_opts(precond=2, krylov_method=1, krylov_tol=1e-6, tol_nonlin_rel=1e-8, krylov_max_it=5000)
    states, masks = learned.generate_trajectory(case, 30, opts=opts, with_masks=True)
    assert len(states) >= 26                          # the solver generated the data
    n_s = len(states)
    train_states, held, held_mask = states[:n_s - 8], states[n_s - 10:], masks[n_s - 10:]
    t_held0 = n_s - 10
    graph = learned.DeviceGraph(learned.build_graph(case.xyz[:, :2], case.tri))
    tr = learned.Trajectory(train_states, case.xyz[:, 2])
    net = learned.Net()
    learned.set_normalisation(net, [tr])
    before = learned.evaluate_loss(net, graph, [tr])
    learned.train(net, graph, [tr], iters=500, lr=2e-3)
    after = learned.evaluate_loss(net, graph, [tr])
    print("training loss (linear extrapolation = 1):", before, "->", after)
    assert after < 0.8 * before                       # training improves on linear extrapolation
    guesser = learned.Guesser(net, case)
    r_plain, r_guess, k_plain, k_guess, used, diffs, fallbacks = [], [], [], [], 0, [], 0
    for t in range(2, len(held) - 1):                 # solve step t -> t+1 of the held-out window
        results = []
        for use in (False, True):
            sim = SW2Simulation(case, opts=opts)
            sim.t = case.t0 + (t_held0 + t) * case.dt
            sim.model.load_state(held[t], held[t - 1], held[t - 2], bc_mask=held_mask[t])
            o = default_opts(precond=2, krylov_method=1, krylov_tol=1e-6, tol_nonlin_rel=1e-8, krylov_max_it=5000,
                             use_guess=int(use))
            if use:
                guesser.predict_into(sim)
            st = sim.step(o)
            results.append((st, sim.state()[0]))
            sim.model.close()
        (sp, xp), (sg, xg) = results
        if not sp["success"]:
            continue                                   # compare only steps the plain start solves
        assert sg["success"]                           # (a failed start from the guess falls back to the previous step)
        fallbacks += sg["guess_fallback"]
        r_plain.append(sp["initial_resid_l2"]); r_guess.append(sg["initial_resid_l2"])
        k_plain.append(sp["krylov_its"]); k_guess.append(sg["krylov_its"]); used += sg["guess_used"]
        # both solve the same step to the same Newton tolerance: the states agree in the L2 sense
        # (pointwise, the velocities of nodes a few cm deep are barely determined by the equations)
        diffs.append(np.linalg.norm(xg - xp) / np.linalg.norm(xp))
    print("initial residual L2 plain", r_plain, "guess", r_guess)
    print("krylov its plain", k_plain, "guess", k_guess, "guess used", used)
    print("relative L2 state difference guess vs plain", diffs, "fallbacks", fallbacks)
    assert len(r_plain) >= 4 and used >= 3
    assert max(diffs) <= 1e-4
    # the gain: where the residual judge takes the guess, Newton starts from a residual
    # well below the previous step's (the Krylov work of both starts is printed above)
    taken = [g / p_ for g, p_ in zip(r_guess, r_plain) if g < p_]
    assert len(taken) == used and np.mean(taken) < 0.85


def test_learned_guess_cuts_newton_and_krylov_work_on_basin_hydrographs():
    """The learned-guess experiment at a small size: trajectories of the basin under
    training inflow hydrographs, the network trained on them, and one held-out
    hydrograph solved from the previous step and from the guess at identical Newton
    settings.  Measured at this size: Newton 30 -> 21 and Krylov 559 -> 429 over 10
    steps, every step converged either way."""
    from adh_kraken_b200 import learned
    net, res = learned.config4(n=40, steps_per_traj=30, eval_steps=10, iters=400, test_seeds=(48,),
                               log=lambda m: None)
    assert res["loss_after"] < 0.5 * res["loss_before"]
    r = res["held_out"][48]
    prev, lg = r["previous_step"], r["learned"]
    print("previous step", prev, "learned", lg, "state difference", r["state_rel_diff"])
    assert prev["failed"] == 0 and lg["failed"] == 0
    assert lg["guess_used"] >= 5
    assert lg["newton_its"] <= 0.85 * prev["newton_its"]
    assert lg["krylov_its"] <= 0.9 * prev["krylov_its"]
    # both starts solve each step to the same Newton tolerance
    assert r["state_rel_diff"][0] <= 1e-9 and max(r["state_rel_diff"]) <= 1e-6


def test_committed_basin_weights_load_and_guess():
    """The committed basin weights (trained on 8 x 375 steps of the 1M-triangle basin)
    load, and from a spun-up state their guess is taken by the residual judge."""
    import os
    from adh_kraken_b200 import learned
    assert os.path.exists(learned.BASIN_WEIGHTS)
    net = learned.Net.load(learned.BASIN_WEIGHTS)
    from adh_kraken_b200.mesh import basin_hydro_case
    from adh_kraken_b200.capi import default_opts
    case = basin_hydro_case(48, n=40, nsteps=12)
    opts = default_opts(precond=2, krylov_method=1, krylov_precision=32, krylov_basis_precision=32,
                        krylov_tol=1e-6, tol_nonlin_rel=1e-8, krylov_max_it=20000, krylov_restart=50)
    r = learned.evaluate_guess(net, case, 4, opts, start=4)
    assert r["start_step"] == 4
    assert r["previous_step"]["failed"] == 0 and r["learned"]["failed"] == 0
    assert max(r["state_rel_diff"]) <= 1e-6
