"""torch.autograd through the matvec: the gradient of 1/2 ||A x - b||^2 with
respect to x is A^H (A x - b), and with respect to the wavenumber it agrees
with central finite differences (h = 1e-6) of the loss."""
import numpy as np
import pytest

from ifgf_b200 import workloads as W

from .helpers import rel2


def _cf(kappa, pts, order=10):
    import ifgf_b200 as G

    op = G.CombinedFieldHelmholtzIfgfOperator(kappa, 64, order)
    op.init(pts, pts, pts)  # unit-sphere normals = the points
    return op


@pytest.mark.gpu
def test_gradients_of_least_squares_loss():
    import torch

    from ifgf_b200.autograd import matvec

    n = 8000
    kappa = 20.0
    pts = W.sphere_points(n, seed=0)
    x0 = W.densities(n, seed=1)
    b0 = W.densities(n, seed=3)
    op = _cf(kappa, pts)
    dev = torch.device("cuda", 0)
    x = torch.tensor(x0, device=dev, requires_grad=True)
    b = torch.tensor(b0, device=dev)
    k = torch.tensor(kappa, dtype=torch.float64, device=dev, requires_grad=True)
    u = matvec(op, x, k)
    loss = 0.5 * torch.sum(torch.abs(u - b) ** 2)
    loss.backward()
    r = op.mult(x0) - b0
    gx = op.mult_adjoint(r)
    assert rel2(x.grad.cpu().numpy(), gx) <= 1e-12
    gk = float(np.real(np.vdot(r, op.mult_dk(x0))))
    assert abs(k.grad.item() - gk) <= 1e-12 * abs(gk)
    # d loss / d kappa against central finite differences of the loss
    h = 1e-6

    def loss_at(kk):
        return 0.5 * float(np.sum(np.abs(_cf(kk, pts).mult(x0) - b0) ** 2))

    fd = (loss_at(kappa + h) - loss_at(kappa - h)) / (2 * h)
    assert abs(fd - k.grad.item()) <= 1e-5 * abs(fd), (fd, k.grad.item())


@pytest.mark.gpu
def test_autograd_real_kernel_density_gradient():
    import torch

    import ifgf_b200 as G
    from ifgf_b200.autograd import matvec

    n = 5000
    pts = W.sphere_points(n, seed=0)
    tg = W.sphere_points(4000, seed=5) * 1.2
    op = G.LaplaceIfgfOperator(64, 8)
    op.init(pts, tg)
    x0 = np.random.default_rng(2).standard_normal(n)
    x = torch.tensor(x0, device="cuda", requires_grad=True)
    u = matvec(op, x)
    (u.sum()).backward()
    assert rel2(x.grad.cpu().numpy(), op.mult_adjoint(np.ones(4000))) <= 1e-12


@pytest.mark.gpu
def test_config5_gradients_against_central_differences():
    """The differentiation workload: combined field, kappa = 50, N = 500,000
    points on the unit sphere with outward normals, x and b complex N(0,1);
    loss 0.5 ||A x - b||^2.  The x-gradient (adjoint kernel) against the
    central difference of the loss along a random direction, the kappa-
    gradient (dA/dk kernel) against the central difference in kappa, both
    with step 1e-6, to 1e-6."""
    import torch

    from ifgf_b200.autograd import matvec

    n = 500000
    kappa = 50.0
    pts = W.sphere_points(n, seed=0)
    x0 = W.densities(n, seed=1)
    b0 = W.densities(n, seed=3)
    v0 = W.densities(n, seed=4)
    op = _cf(kappa, pts)
    x = torch.tensor(x0, device="cuda", requires_grad=True)
    b = torch.tensor(b0, device="cuda")
    k = torch.tensor(kappa, dtype=torch.float64, device="cuda", requires_grad=True)
    loss = 0.5 * torch.sum(torch.abs(matvec(op, x, k) - b) ** 2)
    loss.backward()
    gx = x.grad.cpu().numpy()
    h = 1e-6

    def loss_of(o, xx):
        return 0.5 * float(np.sum(np.abs(o.mult(xx) - b0) ** 2))

    # along v: d/dh L(x + h v) = Re <grad_x, v>
    fd_x = (loss_of(op, x0 + h * v0) - loss_of(op, x0 - h * v0)) / (2 * h)
    dir_x = float(np.real(np.vdot(gx, v0)))
    assert abs(fd_x - dir_x) <= 1e-6 * abs(fd_x), (fd_x, dir_x)
    fd_k = (loss_of(_cf(kappa + h, pts), x0) - loss_of(_cf(kappa - h, pts), x0)) / (2 * h)
    assert abs(fd_k - k.grad.item()) <= 1e-6 * abs(fd_k), (fd_k, k.grad.item())

