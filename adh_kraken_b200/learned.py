"""Learned Newton initial guess for the SW2 time step.

A per-node message-passing network over the mesh's node graph (encoder 8 -> 64,
three aggregation layers 256 -> 64 with SiLU and residual connections, decoder
64 -> 3 followed by two neighbourhood means; BF16 weights, FP32 accumulation)
predicts the next time step as a correction to linear extrapolation:

    guess = 2 sol_t - sol_{t-1} + scale * net(features(sol_t, sol_{t-1}, z_bed))

on nodes deeper than MIN_DEPTH (shallower nodes keep sol_t, and the loss is
masked the same way).

Forward, backward and Adam run in the library's own CUDA kernels
(csrc/gnn_kernels.cu, C ABI in include/adh_sw2_gnn.h); torch only provides device
memory and streams.  Training data are (h, u, v) trajectories that the solver
itself generates.  The guess reaches Newton through sw2g_set_guess with
use_guess = 1; Newton keeps the previous step when that has the smaller residual
(the residual judges the guess).  There is no reference counterpart: the reference
starts Newton from the previous step (src/newton/newton_tools.c:35-37).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .capi import lib

H = 64
LAYERS = [(8, H), (4 * H, H), (4 * H, H), (4 * H, H), (H, 3)]   # (in, out): encoder, 3 layers, decoder
MIN_DEPTH = 0.05   # m: nodes this shallow keep the previous step in the guess
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "beach_guess.npz")
# trained by config4() on the basin with inflow hydrographs (n = 707, 8 x 375 steps, 2000 iterations)
BASIN_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "basin_guess.npz")

_GNN_FUNCS = ["sw2n_agg_fwd", "sw2n_agg_bwd", "sw2n_dense_fwd", "sw2n_dense_bwd", "sw2n_adam", "sw2n_to_bf16",
              "sw2n_features", "sw2n_targets", "sw2n_mse", "sw2n_apply_guess", "sw2n_smooth3", "sw2n_smooth3_adj"]


_VP, _I, _F = C.c_void_p, C.c_int, C.c_float
_ARGTYPES = {
    "sw2n_agg_fwd": [_I] + [_VP] * 11,
    "sw2n_agg_bwd": [_I] + [_VP] * 11,
    "sw2n_dense_fwd": [_I] * 3 + [_VP] * 4 + [_I] + [_VP] * 3,
    "sw2n_dense_bwd": [_I] * 3 + [_VP] * 4 + [_I] + [_VP] * 2 + [_I] + [_VP] * 3,
    "sw2n_adam": [_I] + [_VP] * 5 + [_F] * 4 + [_I, _VP],
    "sw2n_to_bf16": [_I, _VP, _VP, _VP],
    "sw2n_features": [_I] + [_VP] * 7,
    "sw2n_targets": [_I] + [_VP] * 4 + [C.c_double] + [_VP] * 3,
    "sw2n_mse": [_I] + [_VP] * 6,
    "sw2n_smooth3": [_I] + [_VP] * 5,
    "sw2n_smooth3_adj": [_I] + [_VP] * 5,
    "sw2n_apply_guess": [_I] + [_VP] * 4 + [C.c_double, _VP, _VP],
}


def _L():
    L = lib()
    for f in _GNN_FUNCS:
        fn = getattr(L, f)
        fn.restype = C.c_int
        fn.argtypes = _ARGTYPES[f]
    return L


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _check(rc, what):
    if rc < 0:
        raise RuntimeError(f"{what} failed ({rc})")
    return rc


def param_layout():
    offs, o = [], 0
    for i, j in LAYERS:
        offs.append((o, i, j))
        o += j * i + j
    return offs, o


def build_graph(xy, tri):
    """Symmetric node graph of the triangle edges, CSR by node, with reverse slots
    and the edge weights wx, wy = (x_j - x_i) / (L deg_i)."""
    n = xy.shape[0]
    e = np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]]).astype(np.int64)
    e = np.concatenate([e, e[:, ::-1]])
    key = np.unique(e[:, 0] * n + e[:, 1])
    src, dst = key // n, key % n
    indptr = np.zeros(n + 1, np.int64)
    np.add.at(indptr, src + 1, 1)
    indptr = np.cumsum(indptr)
    deg = np.diff(indptr)
    rev = np.searchsorted(key, dst * n + src)
    d = xy[dst] - xy[src]
    L = float(np.mean(np.hypot(d[:, 0], d[:, 1])))
    wx = d[:, 0] / (L * deg[src])
    wy = d[:, 1] / (L * deg[src])
    swx = np.bincount(src, weights=wx, minlength=n)
    swy = np.bincount(src, weights=wy, minlength=n)
    return {"indptr": indptr, "nbr": dst, "rev": rev, "wx": wx, "wy": wy, "inv_deg": 1.0 / deg, "swx": swx,
            "swy": swy, "L": L}


class DeviceGraph:
    def __init__(self, g, device="cuda"):
        import torch
        self.n = len(g["indptr"]) - 1
        ti = lambda a: torch.tensor(np.asarray(a, np.int32), device=device)
        tf = lambda a: torch.tensor(np.asarray(a, np.float32), device=device)
        self.indptr, self.nbr, self.rev = ti(g["indptr"]), ti(g["nbr"]), ti(g["rev"])
        self.wx, self.wy, self.inv_deg = tf(g["wx"]), tf(g["wy"]), tf(g["inv_deg"])
        self.swx, self.swy = tf(g["swx"]), tf(g["swy"])

    def args(self):
        return (self.n, _p(self.indptr), _p(self.nbr), _p(self.rev), _p(self.wx), _p(self.wy), _p(self.inv_deg),
                _p(self.swx), _p(self.swy))

    def sargs(self):
        return (self.n, _p(self.indptr), _p(self.nbr))


class Net:
    """Parameters (FP32 master + BF16 copy), Adam moments and normalisation."""

    def __init__(self, device="cuda", seed=0):
        import torch
        self.device = device
        offs, P = param_layout()
        self.offs, self.P = offs, P
        rng = np.random.default_rng(seed)
        p = np.zeros(P, np.float32)
        for li, (o, i, j) in enumerate(offs):
            if li < len(offs) - 1:
                p[o:o + i * j] = rng.uniform(-1, 1, i * j) * np.sqrt(3.0 / i)   # unit-variance pre-activations
            # the decoder starts at zero: the untrained net is linear extrapolation
        self.w = torch.tensor(p, device=device)
        self.wb = torch.empty(P, dtype=torch.bfloat16, device=device)
        self.m = torch.zeros(P, device=device)
        self.v = torch.zeros(P, device=device)
        self.g = torch.zeros(P, device=device)
        self.t = 0
        self.mu = torch.zeros(8, device=device)
        self.sd = torch.ones(8, device=device)
        self.scale = torch.ones(3, device=device)
        self.sync_bf16()

    def sync_bf16(self, stream=None):
        _check(_L().sw2n_to_bf16(self.P, _p(self.w), _p(self.wb), stream), "to_bf16")

    def layer(self, li):
        o, i, j = self.offs[li]
        return (self.wb[o:o + i * j], self.w[o + i * j:o + i * j + j], self.g[o:o + i * j + j], i, j)

    def save(self, path, meta=None):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez(path, w=self.w.cpu().numpy(), mu=self.mu.cpu().numpy(), sd=self.sd.cpu().numpy(),
                 scale=self.scale.cpu().numpy(), meta=np.array(str(meta or {})))

    @classmethod
    def load(cls, path, device="cuda"):
        import torch
        z = np.load(path)
        net = cls(device=device)
        net.w.copy_(torch.tensor(z["w"], device=device))
        net.mu.copy_(torch.tensor(z["mu"], device=device))
        net.sd.copy_(torch.tensor(z["sd"], device=device))
        net.scale.copy_(torch.tensor(z["scale"], device=device))
        net.sync_bf16()
        return net


class Workspace:
    """Activations of one forward (and backward) pass over n nodes."""

    def __init__(self, n, train, device="cuda"):
        import torch
        z = lambda *s: torch.zeros(*s, device=device)
        self.n = n
        self.F = z(n, 8)
        self.E = [z(n, H) for _ in range(4)] if train else [z(n, H), z(n, H)]
        self.X = [z(n, 4 * H) for _ in range(3)] if train else [z(n, 4 * H)]
        self.Z = [z(n, H) for _ in range(4)] if train else None
        self.Y = z(n, 3)
        self.Yraw = z(n, 3)
        self.Ys = z(n, 3)
        if train:
            self.T = z(n, 3)
            self.dY = z(n, 3)
            self.dYd = z(n, 3)
            self.dYs = z(n, 3)
            self.dYraw = z(n, 3)
            self.M = z(n)
            self.dE = [z(n, H), z(n, H)]
            self.dX = z(n, 4 * H)
            self.dZ = z(n, H)
            self.npb = 256
            self.part = z(((n + self.npb - 1) // self.npb) * (4 * H * H + H))
            self.lpart = z(148 * 4)


def forward(net, graph, ws, stream=None, train=False):
    """ws.F -> ws.Y through the network (the CUDA kernels)."""
    L = _L()
    n = ws.n
    W, b, _, i, j = net.layer(0)
    _check(L.sw2n_dense_fwd(n, i, j, _p(W), _p(b), _p(ws.F), None, 1, _p(ws.Z[0]) if train else None, _p(ws.E[0]),
                            stream), "encoder")
    for li in (1, 2, 3):
        W, b, _, i, j = net.layer(li)
        e_in = ws.E[li - 1] if train else ws.E[(li - 1) % 2]
        e_out = ws.E[li] if train else ws.E[li % 2]
        X = ws.X[li - 1] if train else ws.X[0]
        _check(L.sw2n_agg_fwd(*graph.args(), _p(e_in), _p(X), stream), "aggregate")
        _check(L.sw2n_dense_fwd(n, i, j, _p(W), _p(b), _p(X), _p(e_in), 1, _p(ws.Z[li]) if train else None,
                                _p(e_out), stream), "layer")
    W, b, _, i, j = net.layer(4)
    e_last = ws.E[3] if train else ws.E[1]
    _check(L.sw2n_dense_fwd(n, i, j, _p(W), _p(b), _p(e_last), None, 0, None, _p(ws.Yraw), stream), "decoder")
    _check(L.sw2n_smooth3(*graph.sargs(), _p(ws.Yraw), _p(ws.Ys), stream), "smooth")
    _check(L.sw2n_smooth3(*graph.sargs(), _p(ws.Ys), _p(ws.Y), stream), "smooth")


def backward(net, graph, ws, stream=None):
    """Gradient of the MSE in ws.dY into net.g (the CUDA kernels)."""
    L = _L()
    n = ws.n
    _check(L.sw2n_smooth3_adj(*graph.sargs(), _p(ws.dY), _p(ws.dYs), stream), "smooth bwd")
    _check(L.sw2n_smooth3_adj(*graph.sargs(), _p(ws.dYs), _p(ws.dYraw), stream), "smooth bwd")
    W, _, gW, i, j = net.layer(4)
    dE = ws.dE[0]
    _check(L.sw2n_dense_bwd(n, i, j, _p(W), _p(ws.E[3]), None, _p(ws.dYraw), 0, _p(ws.dYd), _p(dE), ws.npb,
                            _p(ws.part), _p(gW), stream), "decoder bwd")
    for li in (3, 2, 1):
        W, _, gW, i, j = net.layer(li)
        _check(L.sw2n_dense_bwd(n, i, j, _p(W), _p(ws.X[li - 1]), _p(ws.Z[li]), _p(dE), 1, _p(ws.dZ), _p(ws.dX),
                                ws.npb, _p(ws.part), _p(gW), stream), "layer bwd")
        nxt = ws.dE[1] if dE is ws.dE[0] else ws.dE[0]
        _copy(nxt, dE, stream)                                  # residual path
        _check(L.sw2n_agg_bwd(*graph.args(), _p(ws.dX), _p(nxt), stream), "aggregate bwd")
        dE = nxt
    W, _, gW, i, j = net.layer(0)
    _check(L.sw2n_dense_bwd(n, i, j, _p(W), _p(ws.F), _p(ws.Z[0]), _p(dE), 1, _p(ws.dZ), None, ws.npb, _p(ws.part),
                            _p(gW), stream), "encoder bwd")


def _copy(dst, src, stream):
    import torch
    if stream is None:
        dst.copy_(src)
    else:
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            dst.copy_(src)


class Trajectory:
    """Consecutive solver states of one run, kept on the device (FP64 [T, 3n])."""

    def __init__(self, states, z, device="cuda"):
        import torch
        self.S = torch.tensor(np.asarray(states, np.float64), device=device)
        self.z = torch.tensor(np.asarray(z, np.float64), device=device)

    def __len__(self):
        return self.S.shape[0]


def generate_trajectory(case, nsteps, opts=None, spinup=0, with_masks=False):
    """Run the solver and collect sol after every step (the training data); stops at
    the first step that does not converge.  with_masks: also the Dirichlet masks
    (dry-node marks are permanent, so re-solving a step needs the mask it had)."""
    from .capi import SW2Error
    from .timeloop import SW2Simulation
    sim = SW2Simulation(case, opts=opts)
    s0 = sim.state()
    states, masks = [s0[0]], [s0[3]]
    for _ in range(spinup + nsteps):
        try:
            st = sim.step()
        except SW2Error as e:
            print(f"trajectory stops: {e}", flush=True)
            break
        if not st["success"]:
            print(f"trajectory stops: step not converged ({st})", flush=True)
            break
        s = sim.state()
        states.append(s[0]); masks.append(s[3])
    sim.model.close()
    if with_masks:
        return states[spinup:], masks[spinup:]
    return states[spinup:]


def set_normalisation(net, trajs, stride=1):
    """Feature means / deviations and the correction scale from the trajectories (every
    ``stride``-th snapshot, to bound the host memory on long runs)."""
    import torch
    feats, corr = [], []
    for tr in trajs:
        z = tr.z.cpu().numpy()
        for t in range(1, len(tr) - 1, stride):
            S = {k: tr.S[k].cpu().numpy() for k in (t - 1, t, t + 1)}
            s, p, nx = S[t].reshape(-1, 3), S[t - 1].reshape(-1, 3), S[t + 1].reshape(-1, 3)
            f = np.concatenate([s, s - p, z[:, None], (s[:, :1] > 0).astype(np.float64)], axis=1)
            feats.append(f)
            corr.append(nx - 2 * s + p)
    F = np.concatenate(feats)
    Cr = np.concatenate(corr)
    wet = F[:, 0] > MIN_DEPTH
    if wet.any():
        Cr = Cr[wet]                                   # the correction is used (and trained) on wet nodes only
    mu = F.mean(0); sd = F.std(0) + 1e-6
    mu[7], sd[7] = 0.0, 1.0
    scale = np.sqrt((Cr ** 2).mean(0)) + 1e-12
    net.mu.copy_(torch.tensor(mu, dtype=torch.float32))
    net.sd.copy_(torch.tensor(sd, dtype=torch.float32))
    net.scale.copy_(torch.tensor(scale, dtype=torch.float32))


def train(net, graph, trajs, iters=300, lr=2e-3, seed=0, log_every=0):
    """Adam on the MSE of the predicted correction, one random snapshot per step."""
    import torch
    L = _L()
    rng = np.random.default_rng(seed)
    ws = Workspace(graph.n, train=True)
    samples = [(k, t) for k, tr in enumerate(trajs) for t in range(1, len(tr) - 1)]
    losses = []
    for it in range(iters):
        k, t = samples[rng.integers(len(samples))]
        tr = trajs[k]
        S = tr.S
        _check(L.sw2n_features(graph.n, _p(S[t]), _p(S[t - 1]), _p(tr.z), _p(net.mu), _p(net.sd), _p(ws.F), None), "f")
        _check(L.sw2n_targets(graph.n, _p(S[t + 1]), _p(S[t]), _p(S[t - 1]), _p(net.scale), MIN_DEPTH, _p(ws.T),
                              _p(ws.M), None), "t")
        forward(net, graph, ws, train=True)
        nparts = _check(L.sw2n_mse(graph.n, _p(ws.Y), _p(ws.T), _p(ws.M), _p(ws.dY), _p(ws.lpart), None), "mse")
        backward(net, graph, ws)
        net.t += 1
        _check(L.sw2n_adam(net.P, _p(net.w), _p(net.g), _p(net.m), _p(net.v), _p(net.wb), lr, 0.9, 0.999, 1e-8, net.t,
                           None), "adam")
        if log_every and (it % log_every == 0 or it == iters - 1):
            losses.append((it, float(ws.lpart[:nparts].sum().item())))
    torch.cuda.synchronize()
    return losses


def evaluate_loss(net, graph, trajs):
    L = _L()
    ws = Workspace(graph.n, train=True)
    tot, cnt = 0.0, 0
    for tr in trajs:
        for t in range(1, len(tr) - 1):
            S = tr.S
            L.sw2n_features(graph.n, _p(S[t]), _p(S[t - 1]), _p(tr.z), _p(net.mu), _p(net.sd), _p(ws.F), None)
            L.sw2n_targets(graph.n, _p(S[t + 1]), _p(S[t]), _p(S[t - 1]), _p(net.scale), MIN_DEPTH, _p(ws.T),
                           _p(ws.M), None)
            forward(net, graph, ws, train=True)
            k = L.sw2n_mse(graph.n, _p(ws.Y), _p(ws.T), _p(ws.M), _p(ws.dY), _p(ws.lpart), None)
            tot += float(ws.lpart[:k].sum().item()); cnt += 1
    return tot / max(cnt, 1)


class Guesser:
    """Inference on one mesh: writes the guess for the next step into a model."""

    def __init__(self, net, case, device="cuda"):
        import torch
        self.net = net
        self.graph = DeviceGraph(build_graph(case.xyz[:, :2], case.tri), device)
        self.ws = Workspace(case.nnodes, train=False, device=device)
        self.z = torch.tensor(case.xyz[:, 2].astype(np.float64), device=device)
        self.guess = torch.zeros(3 * case.nnodes, dtype=torch.float64, device=device)
        self.hsol = torch.zeros(3 * case.nnodes, dtype=torch.float64, device=device)
        self.hprev = torch.zeros(3 * case.nnodes, dtype=torch.float64, device=device)

    def predict_ptr(self, sol_ptr, prev_ptr, stream):
        L = _L()
        n = self.graph.n
        _check(L.sw2n_features(n, C.c_void_p(sol_ptr), C.c_void_p(prev_ptr), _p(self.z), _p(self.net.mu),
                               _p(self.net.sd), _p(self.ws.F), C.c_void_p(stream)), "features")
        forward(self.net, self.graph, self.ws, stream=C.c_void_p(stream))
        _check(L.sw2n_apply_guess(n, C.c_void_p(sol_ptr), C.c_void_p(prev_ptr), _p(self.ws.Y), _p(self.net.scale),
                                  MIN_DEPTH, _p(self.guess), C.c_void_p(stream)), "apply_guess")
        return self.guess.data_ptr()

    def predict_into(self, sim):
        """Guess for sim's next step from its resident state (sol_t, sol_{t-1})."""
        m = sim.model
        sol, sol_old, _ = m.device_state()
        g = self.predict_ptr(sol, sol_old, m.stream)
        m.set_guess(device_ptr=g)

    def predict_host(self, model, sol_host, prev_host):
        """Guess from host arrays (the end-to-end path): copy in, predict, hand to the model."""
        import torch
        self.hsol.copy_(torch.from_numpy(sol_host))        # completes before the model stream reads it
        self.hprev.copy_(torch.from_numpy(prev_host))
        torch.cuda.current_stream().synchronize()
        g = self.predict_ptr(self.hsol.data_ptr(), self.hprev.data_ptr(), model.stream)
        model.set_guess(device_ptr=g)


def load_guesser(case, path=WEIGHTS):
    if not os.path.exists(path):
        raise FileNotFoundError(f"no trained weights at {path}: run adh_kraken_b200.learned.main() to train them")
    return Guesser(Net.load(path), case)


def beach_strip(ny=40, nsteps=1, seed=3, nx=2828):
    """A strip of the 4M beach at its full resolution (same spacing, dt and forcing)."""
    from .mesh import beach_case
    return beach_case(nx=nx, ny=ny, nsteps=nsteps, seed=seed, ly=(ny - 1) * 40000.0 / (nx - 1))


def main(out=WEIGHTS, nsteps=12, seed=4, iters=300, nx=2828, ny=707, krylov_tol=1e-6):
    """Train the beach initial-guess network on a solver trajectory of a beach with
    the benchmark's resolution, dt and forcing but another bed (seed), and save the
    weights (the benchmark's own beach, seed 3, is never seen in training)."""
    from .capi import default_opts
    from .mesh import beach_case
    opts = default_opts(precond=2, krylov_method=1, krylov_precision=32, krylov_tol=krylov_tol, tol_nonlin_rel=1e-8,
                        krylov_max_it=20000)
    case = beach_case(nx=nx, ny=ny, nsteps=nsteps + 2, seed=seed)
    states = generate_trajectory(case, nsteps, opts=opts)
    print(f"trajectory: {len(states)} states", flush=True)
    tr = Trajectory(states, case.xyz[:, 2])
    graph = DeviceGraph(build_graph(case.xyz[:, :2], case.tri))
    net = Net()
    set_normalisation(net, [tr])
    before = evaluate_loss(net, graph, [tr])
    log = train(net, graph, [tr], iters=iters, log_every=50)
    after = evaluate_loss(net, graph, [tr])
    print("loss (linear extrapolation = %.4f) -> %.4f" % (before, after), log, flush=True)
    net.save(out, meta={"nx": nx, "ny": ny, "seed": seed, "nsteps": len(states) - 1, "iters": iters,
                        "loss_before": before, "loss_after": after})
    return net, before, after




def device_trajectory(case, nsteps, opts=None):
    """Like generate_trajectory, but each state goes to a device tensor as soon as it is
    read back, so long runs on large meshes need no host memory for the set."""
    import torch
    from .capi import SW2Error
    from .timeloop import SW2Simulation
    sim = SW2Simulation(case, opts=opts)
    S = [torch.tensor(sim.state()[0], device="cuda")]
    for _ in range(nsteps):
        try:
            st = sim.step()
        except SW2Error as e:
            print(f"trajectory stops: {e}", flush=True)
            break
        if not st["success"]:
            print(f"trajectory stops: step not converged", flush=True)
            break
        S.append(torch.tensor(sim.state()[0], device="cuda"))
    sim.model.close()
    tr = Trajectory.__new__(Trajectory)
    tr.S = torch.stack(S)
    tr.z = torch.tensor(case.xyz[:, 2].astype(np.float64), device="cuda")
    return tr


def evaluate_guess(net, case, nsteps, opts, start=0):
    """Runs ``nsteps`` steps of ``case`` twice from the same state: Newton started from
    the previous step (the reference's start) and from the network's guess (use_guess = 1;
    the residual still judges it).  With ``start`` > 0 both runs begin after ``start``
    spin-up steps taken once from the initial state with the previous-step start.  Per
    run: Newton and Krylov iterations, steps the guess started, and device time (CUDA
    events on the model's stream, guess inference included)."""
    import copy
    import torch
    from .timeloop import SW2Simulation
    s0, t0 = None, case.t0
    if start > 0:
        o = copy.copy(opts)
        o.use_guess = 0
        sim = SW2Simulation(case, opts=o)
        for _ in range(start):
            st = sim.step()
            if not st["success"]:
                raise RuntimeError(f"spin-up step at t = {sim.t} did not converge")
        s0, t0 = sim.state(), sim.t
        sim.model.close()
    out = {"start_step": start}
    for mode in ("previous_step", "learned"):
        o = copy.copy(opts)
        o.use_guess = 1 if mode == "learned" else 0
        sim = SW2Simulation(case, opts=o)
        if s0 is not None:
            sim.model.load_state(*s0[:3], bc_mask=s0[3])
            sim.t = t0
        g = Guesser(net, case) if mode == "learned" else None
        s = torch.cuda.ExternalStream(sim.model.stream)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        rec = {"newton_its": 0, "krylov_its": 0, "guess_used": 0, "failed": 0, "steps": 0}
        torch.cuda.synchronize()
        ev0.record(s)
        for k in range(nsteps):
            if g is not None and (k > 0 or s0 is not None):   # the guess needs two states
                g.predict_into(sim)
            st = sim.step()
            rec["newton_its"] += st["newton_its"]; rec["krylov_its"] += st["krylov_its"]
            rec["guess_used"] += st.get("guess_used", 0); rec["failed"] += int(not st["success"])
            rec["steps"] += 1
        ev1.record(s)
        torch.cuda.synchronize()
        rec["ms"] = ev0.elapsed_time(ev1)
        rec["steps_per_s"] = rec["steps"] / (rec["ms"] * 1e-3)
        rec["final_state"] = sim.state()[0]
        sim.model.close()
        out[mode] = rec
    a, b = out["previous_step"]["final_state"], out["learned"]["final_state"]
    out["state_rel_diff"] = [float(np.abs(a[k::3] - b[k::3]).max() / max(np.abs(a[k::3]).max(), 1e-300))
                             for k in range(3)]
    for mode in ("previous_step", "learned"):
        del out[mode]["final_state"]
    return out


def config4(n=707, train_seeds=tuple(range(40, 48)), test_seeds=tuple(range(48, 52)), steps_per_traj=375,
            eval_steps=40, iters=2000, out=None, opts=None, log=print, eval_start=0, net=None):
    """The learned-guess experiment on the basin with inflow hydrographs
    (mesh.basin_hydro_case): trajectories of the solver under the training hydrographs
    (8 x 375 = 3000 steps at the default sizes), the network trained on them by the
    library's kernels, then Newton / Krylov work and device time on the held-out
    hydrographs with and without the learned guess, from step ``eval_start`` of each
    held-out run (the hydrographs rise from base flow, so windows later in the day
    see the different peaks).  A given ``net`` (already trained) skips the training."""
    import time
    from .capi import default_opts
    from .mesh import basin_hydro_case
    opts = opts or default_opts(precond=2, krylov_method=1, krylov_precision=32, krylov_basis_precision=32,
                                krylov_tol=1e-6, tol_nonlin_rel=1e-8, krylov_max_it=20000, krylov_restart=50)
    t0 = time.time()
    res = {"held_out": {}}
    if net is None:
        trajs = []
        for sd in train_seeds:
            case = basin_hydro_case(sd, n=n, nsteps=steps_per_traj + 2)
            trajs.append(device_trajectory(case, steps_per_traj, opts))
            log(f"trajectory {sd}: {len(trajs[-1])} states, {time.time() - t0:.0f} s")
        graph = DeviceGraph(build_graph(case.xyz[:, :2], case.tri))
        net = Net()
        set_normalisation(net, trajs, stride=max(1, steps_per_traj // 25))
        before = evaluate_loss(net, graph, [tr for tr in trajs[:1]])
        losses = train(net, graph, trajs, iters=iters, log_every=max(1, iters // 10))
        after = evaluate_loss(net, graph, [tr for tr in trajs[:1]])
        log(f"trained {iters} iterations: loss {before:.4f} (linear extrapolation) -> {after:.4f}, "
            f"{time.time() - t0:.0f} s")
        del trajs
        res.update({"train_states": sum(1 for _ in train_seeds) * steps_per_traj, "loss_before": before,
                    "loss_after": after, "losses": losses})
    for sd in test_seeds:
        case = basin_hydro_case(sd, n=n, nsteps=eval_start + eval_steps + 2)
        res["held_out"][sd] = evaluate_guess(net, case, eval_steps, opts, start=eval_start)
        res["held_out"][sd]["q_peak"] = case.q_peak
        log(f"held-out {sd}: {res['held_out'][sd]}")
    if out and "loss_after" in res:
        net.save(out, meta={"workload": "basin_hydro", "n": n, "train_seeds": list(train_seeds),
                            "steps_per_traj": steps_per_traj, "iters": iters, "loss_before": res["loss_before"],
                            "loss_after": res["loss_after"]})
    return net, res


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train the learned initial guess")
    ap.add_argument("--config4", action="store_true",
                    help="the basin experiment with 8 training and 4 held-out inflow hydrographs")
    ap.add_argument("--n", type=int, default=707)
    ap.add_argument("--steps-per-traj", type=int, default=375)
    ap.add_argument("--eval-steps", type=int, default=40)
    ap.add_argument("--iters", type=int, default=2000)
    ap.add_argument("--out", default=None, help="weights file")
    ap.add_argument("--report", default=None, help="JSON report of the experiment")
    ap.add_argument("--eval-start", type=int, default=0, help="spin-up steps before each held-out window")
    ap.add_argument("--weights", default=None, help="evaluate these trained weights instead of training")
    a = ap.parse_args()
    if a.config4:
        net = Net.load(a.weights) if a.weights else None
        _, res = config4(n=a.n, steps_per_traj=a.steps_per_traj, eval_steps=a.eval_steps, iters=a.iters, out=a.out,
                         log=lambda m: print(m, flush=True), eval_start=a.eval_start, net=net)
        if a.report:
            with open(a.report, "w") as fh:
                json.dump(res, fh, indent=1, default=float)
    else:
        main(out=a.out or WEIGHTS)
