"""Adjoint gradients: the pair VJP against the oracle's tangent (dot-product
test), whole-run gradients against the oracle's tangent-linear model and
against FP64 central finite differences (<= 1e-6 relative), through the
torch.autograd.Function."""
import numpy as np
import pytest

import nbody_b200 as nb
import oracle as O

pytestmark = pytest.mark.gpu


def t(a):
    import torch
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def xv_of(s):
    return np.stack([s["x"], s["y"], s["z"]]), np.stack([s["vx"], s["vy"], s["vz"]])


def test_pair_vjp_dot_product():
    import torch
    n, eps2 = 300, 1e-2
    s = nb.plummer(n, 5)
    X, V = xv_of(s)
    rng = np.random.default_rng(1)
    ab, jb = rng.normal(size=(3, n)), rng.normal(size=(3, n))
    dx, dv, dm = rng.normal(size=(3, n)), rng.normal(size=(3, n)), rng.normal(size=n) / n
    adj = nb.Adjoint(n, eps2, 1 / 256, 0)
    gx, gv, gm = (torch.empty((3, n), dtype=torch.float64, device="cuda"),
                  torch.empty((3, n), dtype=torch.float64, device="cuda"),
                  torch.empty(n, dtype=torch.float64, device="cuda"))
    adj.vjp_acc_jerk(t(X), t(V), t(s["m"]), t(ab), t(jb), gx, gv, gm,
                     torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    da, dj = O.force_jvp(s, eps2, dx, dv, dm)
    lhs = (gx.cpu().numpy() * dx).sum() + (gv.cpu().numpy() * dv).sum() + (gm.cpu().numpy() * dm).sum()
    rhs = (ab * da).sum() + (jb * dj).sum()
    assert abs(lhs - rhs) <= 1e-11 * abs(rhs), (lhs, rhs)


def loss_and_grad(s, eps2, dt, nsteps, k, sel, target, precision="fp64"):
    import torch
    X, V = xv_of(s)
    x0 = t(X).requires_grad_()
    v0 = t(V).requires_grad_()
    m = t(s["m"]).requires_grad_()
    x1, v1 = nb.hermite_rollout(x0, v0, m, eps2=eps2, dt=dt, nsteps=nsteps, checkpoint_every=k,
                                precision=precision)
    loss = ((x1[:, sel] - t(target)) ** 2).sum()
    loss.backward()
    return loss.item(), x0.grad.cpu().numpy(), v0.grad.cpu().numpy(), m.grad.cpu().numpy(), x1.detach().cpu().numpy()


@pytest.mark.parametrize("nsteps,k", [(24, 8), (20, 7), (5, 16)])
def test_gradient_vs_tangent_linear(nsteps, k):
    n, eps2, dt = 128, 1e-2, 1 / 256
    s = nb.plummer(n, 4)
    rng = np.random.default_rng(2)
    sel = np.sort(rng.choice(n, 16, replace=False))
    ref_X, _, _, _ = O.hermite_tlm(s, eps2, dt, nsteps, np.zeros((3, n)), np.zeros((3, n)), np.zeros(n))
    target = ref_X[:, sel] + rng.normal(scale=1e-3, size=(3, sel.size))
    L, gx, gv, gm, x1 = loss_and_grad(s, eps2, dt, nsteps, k, sel, target)
    assert np.abs(x1 - ref_X).max() < 1e-12
    for trial in range(3):
        dx, dv, dm = rng.normal(size=(3, n)), rng.normal(size=(3, n)), rng.normal(size=n) / n
        X1, _, DX1, _ = O.hermite_tlm(s, eps2, dt, nsteps, dx, dv, dm)
        dL = 2.0 * ((X1[:, sel] - target) * DX1[:, sel]).sum()
        g = (gx * dx).sum() + (gv * dv).sum() + (gm * dm).sum()
        assert abs(g - dL) <= 1e-9 * abs(dL), (trial, g, dL)


def test_n4096_256_step_gradients_vs_finite_differences():
    """N = 4096 Plummer (seed 4), eps = 1e-2, dt = 1/256, 256 steps,
    checkpoint every 16; loss over 64 seeded bodies with targets = final
    positions + N(0, 1e-3).  FP64 central differences on sampled components."""
    import torch
    n, eps2, dt, nsteps, k = 4096, 1e-4, 1 / 256, 256, 16
    s = nb.plummer(n, 4)
    rng = np.random.default_rng(4)
    sel = np.sort(rng.choice(n, 64, replace=False))
    adj = nb.Adjoint(n, eps2, dt, nsteps, k)
    X, V = xv_of(s)
    m = t(s["m"])

    def final_x(X, V, m_):
        x1 = torch.empty((3, n), dtype=torch.float64, device="cuda")
        v1 = torch.empty_like(x1)
        adj.forward(t(X), t(V), m_, x1, v1, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        return x1.cpu().numpy()

    x1 = final_x(X, V, m)
    target = x1[:, sel] + rng.normal(scale=1e-3, size=(3, sel.size))
    L, gx, gv, gm, _ = loss_and_grad(s, eps2, dt, nsteps, k, sel, target)

    def loss_at(X, V, mm):
        xf = final_x(X, V, t(mm))
        return ((xf[:, sel] - target) ** 2).sum()

    def fd(kind, body, comp, h):
        """Central difference of the loss along one input component."""
        if kind == "m":
            mp, mn = s["m"].copy(), s["m"].copy()
            mp[body] += h
            mn[body] -= h
            return (loss_at(X, V, mp) - loss_at(X, V, mn)) / (2 * h)
        A = X if kind == "x" else V
        Ap, An = A.copy(), A.copy()
        Ap[comp, body] += h
        An[comp, body] -= h
        if kind == "x":
            return (loss_at(Ap, V, s["m"]) - loss_at(An, V, s["m"])) / (2 * h)
        return (loss_at(X, Ap, s["m"]) - loss_at(X, An, s["m"])) / (2 * h)

    checks = [("x", sel[0], 0), ("x", sel[5], 2), ("v", sel[3], 1), ("x", 17, 1), ("m", sel[7], 0),
              ("m", 100, 0)]
    # relative error <= 1e-6 per component; each kind (dL/dx, dL/dv, dL/dm,
    # in their own units) is scaled by its own largest gradient only where a
    # component is below 1e-3 of that (its relative error then measures the
    # finite differences' noise, not the gradient)
    scale = {"x": np.abs(gx).max(), "v": np.abs(gv).max(), "m": np.abs(gm).max()}
    for kind, body, comp in checks:
        # steps where truncation (large h) and roundoff (small h) errors both
        # stay below 1e-7 relative on this run; Richardson extrapolation of
        # two central differences removes the h^2 term
        h = 2e-3 * s["m"][body] if kind == "m" else 2e-6
        est = (4.0 * fd(kind, body, comp, h / 2) - fd(kind, body, comp, h)) / 3.0
        g = {"x": gx, "v": gv}[kind][comp, body] if kind != "m" else gm[body]
        floor = 1e-3 * scale[kind]
        print(f"d{kind}[{comp},{body}]: adjoint {g:.12e} fd {est:.12e} rel {abs(g - est) / abs(est):.2e}"
              f"{'' if abs(est) >= floor else ' (below floor)'}")
        assert abs(g - est) <= 1e-6 * max(abs(est), floor), (kind, body, comp, g, est)


def test_mixed_forward_gradients_close_to_fp64():
    n, eps2, dt, nsteps = 1024, 1e-4, 1 / 256, 64
    s = nb.plummer(n, 4)
    rng = np.random.default_rng(7)
    sel = np.sort(rng.choice(n, 32, replace=False))
    X1, _, _, _ = O.hermite_tlm(s, eps2, dt, nsteps, np.zeros((3, n)), np.zeros((3, n)), np.zeros(n))
    target = X1[:, sel] + rng.normal(scale=1e-3, size=(3, sel.size))
    _, gx64, gv64, gm64, _ = loss_and_grad(s, eps2, dt, nsteps, 16, sel, target, "fp64")
    _, gxm, gvm, gmm, _ = loss_and_grad(s, eps2, dt, nsteps, 16, sel, target, "mixed")
    rel = np.linalg.norm(gxm - gx64) / np.linalg.norm(gx64)
    assert rel < 1e-4, rel
