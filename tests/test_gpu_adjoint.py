"""The WLS solve behind the Laplace path and its adjoint (cuphu_b200.autograd):
forward solution against a sparse FP64 direct solve, gradients against the
FP64 reference gradient (direct solves of the same adjoint system) and
against central finite differences (step 1e-3 on seeded random arcs), for
one solve and through IRLS reweighting."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

pytestmark = pytest.mark.gpu

EPS = 1e-12


def _problem(nr, nc, seed, wzero=0.05):
    rng = np.random.default_rng(seed)
    gd = rng.normal(0.0, 0.8, (nr, nc)).astype(np.float32)
    gr = rng.normal(0.0, 0.8, (nr, nc)).astype(np.float32)
    wd = rng.uniform(0.3, 2.0, (nr, nc)).astype(np.float32)
    wr = rng.uniform(0.3, 2.0, (nr, nc)).astype(np.float32)
    wd[rng.random((nr, nc)) < wzero] = 0.0
    wr[rng.random((nr, nc)) < wzero] = 0.0
    wd[-1, :] = 0.0
    wr[:, -1] = 0.0
    return gd, gr, wd, wr


def _D(nr, nc):
    """Arc-node incidence: down arcs (r<nr-1, all c) then right arcs."""
    idx = np.arange(nr * nc).reshape(nr, nc)
    t_d, h_d = idx[:-1, :].ravel(), idx[1:, :].ravel()
    t_r, h_r = idx[:, :-1].ravel(), idx[:, 1:].ravel()
    tail = np.concatenate([t_d, t_r])
    head = np.concatenate([h_d, h_r])
    na = tail.size
    rows = np.concatenate([np.arange(na), np.arange(na)])
    cols = np.concatenate([head, tail])
    vals = np.concatenate([np.ones(na), -np.ones(na)])
    return sp.csr_matrix((vals, (rows, cols)), shape=(na, nr * nc))


def _arcs(pd, pr):
    return np.concatenate([pd[:-1, :].ravel(), pr[:, :-1].ravel()]).astype(np.float64)


def _planes(a, nr, nc):
    nd = (nr - 1) * nc
    pd = np.zeros((nr, nc))
    pr = np.zeros((nr, nc))
    pd[:-1, :] = a[:nd].reshape(nr - 1, nc)
    pr[:, :-1] = a[nd:].reshape(nr, nc - 1)
    return pd, pr


def _reference(gd, gr, wd, wr, c):
    """FP64 direct solves: u, and the gradient of l = sum c (u - mean u)."""
    nr, nc = gd.shape
    D = _D(nr, nc)
    g, w = _arcs(gd, gr), _arcs(wd, wr)
    L = (D.T @ sp.diags(w) @ D + EPS * sp.eye(nr * nc)).tocsc()
    u = spla.spsolve(L, D.T @ (w * g))
    cv = c.ravel().astype(np.float64)
    lam = spla.spsolve(L, cv - cv.mean())
    dl = D @ lam
    ggd, ggr = _planes(w * dl, nr, nc)
    gwd, gwr = _planes(dl * (g - D @ u), nr, nc)
    return u.reshape(nr, nc), (ggd, ggr, gwd, gwr)


def _cuda(torch, *arrs):
    return [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrs]


TIGHT = dict(max_iter=20000, tol=1e-11)


def test_wls_forward_matches_direct_solve(torch_cuda):
    from cuphu_b200.autograd import wls_solve
    gd, gr, wd, wr = _problem(40, 53, 1)
    u_ref, _ = _reference(gd, gr, wd, wr, np.zeros((40, 53)))
    tg = _cuda(torch_cuda, gd, gr, wd, wr)
    for prec, tol_abs in (("fp64", 1e-7), ("mixed", 1e-3)):
        u = wls_solve(*tg, precision=prec, **TIGHT).cpu().numpy()
        d = (u - u.mean()) - (u_ref - u_ref.mean())
        assert np.abs(d).max() < tol_abs, (prec, np.abs(d).max())


def test_wls_adjoint_matches_fp64_reference_gradient(torch_cuda):
    torch = torch_cuda
    from cuphu_b200.autograd import WLSSolve
    nr, nc = 36, 45
    gd, gr, wd, wr = _problem(nr, nc, 2)
    c = np.random.default_rng(3).normal(size=(nr, nc))
    _, ref = _reference(gd, gr, wd, wr, c)
    tg = [t.requires_grad_() for t in _cuda(torch, gd, gr, wd, wr)]
    u = WLSSolve.apply(*tg, None, "fp64", TIGHT["max_iter"], TIGHT["tol"])
    ct = torch.from_numpy(c).cuda()
    loss = (ct * (u - u.mean())).sum()
    loss.backward()
    for t, r, name in zip(tg, ref, ("g_d", "g_r", "w_d", "w_r")):
        got = t.grad.double().cpu().numpy()
        scale = np.abs(r).max()
        assert np.abs(got - r).max() < 1e-5 * scale, (name, np.abs(got - r).max(), scale)


def test_wls_gradient_matches_finite_differences(torch_cuda):
    torch = torch_cuda
    from cuphu_b200.autograd import WLSSolve, wls_solve
    nr, nc = 32, 40
    gd, gr, wd, wr = _problem(nr, nc, 4)
    c = np.random.default_rng(5).normal(size=(nr, nc))
    ct = torch.from_numpy(c).cuda()

    def loss_of(arrs):
        u = wls_solve(*_cuda(torch, *arrs), precision="fp64", **TIGHT)
        return float((ct * (u - u.mean())).sum())

    tg = [t.requires_grad_() for t in _cuda(torch, gd, gr, wd, wr)]
    u = WLSSolve.apply(*tg, None, "fp64", TIGHT["max_iter"], TIGHT["tol"])
    (ct * (u - u.mean())).sum().backward()
    grads = [t.grad.double().cpu().numpy() for t in tg]
    rng = np.random.default_rng(6)
    h = 1e-3
    base = [a.astype(np.float64) for a in (gd, gr, wd, wr)]
    for _ in range(64):
        k = int(rng.integers(0, 4))
        r = int(rng.integers(0, nr - 1 if k in (0, 2) else nr))
        col = int(rng.integers(0, nc if k in (0, 2) else nc - 1))
        if k >= 2 and base[k][r, col] == 0.0:
            continue
        plus = [a.copy() for a in base]
        minus = [a.copy() for a in base]
        plus[k][r, col] += h
        minus[k][r, col] -= h
        fd = (loss_of([p.astype(np.float32) for p in plus]) -
              loss_of([m.astype(np.float32) for m in minus])) / (2 * h)
        # the inputs are float32: the perturbation actually applied
        hp = np.float32(base[k][r, col] + h) - np.float32(base[k][r, col] - h)
        fd = fd * 2 * h / float(hp)
        g = grads[k][r, col]
        assert abs(fd - g) <= 2e-4 * max(1.0, abs(g)), (k, r, col, fd, g)


def test_irls_gradient_matches_finite_differences(torch_cuda):
    torch = torch_cuda
    from cuphu_b200.autograd import irls_solve
    nr, nc = 24, 30
    gd, gr, wd, wr = _problem(nr, nc, 7, wzero=0.0)
    c = np.random.default_rng(8).normal(size=(nr, nc))
    ct = torch.from_numpy(c).cuda()
    kw = dict(n_irls=2, precision="fp64", **TIGHT)

    def loss_of(arrs):
        u = irls_solve(*_cuda(torch, *arrs), **kw)
        return float((ct * (u - u.mean())).sum())

    tg = [t.requires_grad_() for t in _cuda(torch, gd, gr, wd, wr)]
    u = irls_solve(*tg, **kw)
    (ct * (u - u.mean())).sum().backward()
    grads = [t.grad.double().cpu().numpy() for t in tg]
    rng = np.random.default_rng(9)
    h = 1e-3
    base = [a.astype(np.float64) for a in (gd, gr, wd, wr)]
    for _ in range(16):
        k = int(rng.integers(0, 4))
        r = int(rng.integers(0, nr - 1 if k in (0, 2) else nr))
        col = int(rng.integers(0, nc if k in (0, 2) else nc - 1))
        plus = [a.copy() for a in base]
        minus = [a.copy() for a in base]
        plus[k][r, col] += h
        minus[k][r, col] -= h
        hp = np.float32(base[k][r, col] + h) - np.float32(base[k][r, col] - h)
        fd = (loss_of([p.astype(np.float32) for p in plus]) -
              loss_of([m.astype(np.float32) for m in minus])) / float(hp)
        g = grads[k][r, col]
        assert abs(fd - g) <= 1e-3 * max(1.0, abs(g)), (k, r, col, fd, g)


def test_mixed_precision_gradient_close_to_fp64(torch_cuda):
    torch = torch_cuda
    from cuphu_b200.autograd import WLSSolve
    nr, nc = 64, 80
    gd, gr, wd, wr = _problem(nr, nc, 10)
    ct = torch.from_numpy(np.random.default_rng(11).normal(size=(nr, nc))).cuda()
    out = {}
    for prec in ("fp64", "mixed"):
        tg = [t.requires_grad_() for t in _cuda(torch, gd, gr, wd, wr)]
        u = WLSSolve.apply(*tg, None, prec, 5000, 1e-8)
        (ct * (u - u.mean())).sum().backward()
        out[prec] = [t.grad.double().cpu().numpy() for t in tg]
    for a, b in zip(out["fp64"], out["mixed"]):
        assert np.abs(a - b).max() <= 1e-3 * np.abs(a).max()
