"""The libtorch autograd binding (behavert_b200.autograd.flock_loss, a
torch::autograd::Function in C++) against the C-ABI adjoint it wraps, and a
short Adam fit through it."""
import numpy as np
import pytest

from behavert_b200 import workloads
from behavert_b200.engine import Engine

pytestmark = pytest.mark.gpu

DT = float(np.float32(0.1))


def _setup(n=4096, L=40.0, T=15):
    import torch
    wl = workloads.adjoint(n=n, L=L, steps=T)
    with Engine(wl.params) as eng:
        eng.set_steering_weights(np.asarray([wl.meta["hidden"]], np.float32))
        eng.set_state(wl.pos, wl.meta["fwd_hidden"], wl.acc)
        eng.step(DT, T)
        target = eng.get_state(features=False)[0][:, :3].copy()
    dev = torch.device("cuda:0")
    pos0 = torch.tensor(wl.pos[:, :3], device=dev)
    vel0 = torch.tensor(wl.fwd[:, :3] * wl.fwd[:, 3:4], device=dev)
    tgt = torch.tensor(target, device=dev)
    return wl, pos0, vel0, tgt


def test_autograd_matches_c_abi_adjoint():
    import torch
    from behavert_b200.autograd import flock_loss
    T, k = 15, 5
    wl, pos0, vel0, tgt = _setup(T=T)
    w = torch.tensor([wl.meta["trial"]], dtype=torch.float32, device="cuda:0", requires_grad=True)
    p = pos0.clone().requires_grad_(True)
    v = vel0.clone().requires_grad_(True)
    with Engine(wl.params) as eng:
        loss = flock_loss(eng, w, p, v, tgt, DT, T, k)
        assert loss.dtype == torch.float64 and loss.shape == (1,)
        (3.0 * loss.sum()).backward()
        # the same rollout through the C-ABI directly
        fwd = np.zeros((wl.num_agents, 4), np.float32)
        vv = vel0.cpu().numpy()
        s = np.linalg.norm(vv, axis=1)
        fwd[:, :3] = vv / s[:, None]
        fwd[:, 3] = s
        eng.set_steering_weights(np.asarray([wl.meta["trial"]], np.float32))
        eng.set_state(wl.pos, fwd, np.zeros_like(wl.acc))
        tgt4 = np.zeros((wl.num_agents, 4), np.float32)
        tgt4[:, :3] = tgt.cpu().numpy()
        ref_loss = eng.adjoint_forward(tgt4, T, k, DT)
        ref = eng.adjoint_backward(loss_scale=[3.0])
    assert np.allclose(loss.detach().cpu().numpy(), ref_loss, rtol=1e-6, atol=0)
    gw = w.grad.cpu().numpy().astype(np.float64)
    assert np.allclose(gw, ref["weights"], rtol=1e-5, atol=0)
    gp = p.grad.cpu().numpy()
    gv = v.grad.cpu().numpy()
    assert np.linalg.norm(gp - ref["pos"][:, :3]) <= 1e-5 * np.linalg.norm(ref["pos"][:, :3])
    assert np.linalg.norm(gv - ref["vel"][:, :3]) <= 1e-5 * np.linalg.norm(ref["vel"][:, :3])


def test_adam_fit_reduces_loss_toward_hidden_weights():
    import torch
    from behavert_b200.autograd import flock_loss
    T, k = 15, 5
    wl, pos0, vel0, tgt = _setup(T=T)
    # targets generated from the unperturbed velocities, fitted from them too
    vel_h = torch.tensor(wl.meta["fwd_hidden"][:, :3] * wl.meta["fwd_hidden"][:, 3:4], device="cuda:0")
    w = torch.tensor([wl.meta["trial"]], dtype=torch.float32, device="cuda:0", requires_grad=True)
    opt = torch.optim.Adam([w], lr=0.05)
    losses = []
    with Engine(wl.params) as eng:
        for _ in range(30):
            opt.zero_grad()
            loss = flock_loss(eng, w, pos0, vel_h, tgt, DT, T, k).sum()
            loss.backward()
            opt.step()
            losses.append(float(loss.detach()))
    hidden = np.asarray(wl.meta["hidden"])
    err0 = np.linalg.norm(np.asarray(wl.meta["trial"]) - hidden)
    err = np.linalg.norm(w.detach().cpu().numpy()[0] - hidden)
    assert losses[-1] < 0.2 * losses[0], losses
    assert err < err0, (w, hidden)
