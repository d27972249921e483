"""torch.autograd binding of the matvec u = A w.

The backward pass uses the library's adjoint and k-derivative matvecs:

* with respect to the densities: grad_w = A^H grad_u (torch's convention for
  complex tensors: the gradient is the conjugate Wirtinger derivative times
  two, so a real loss L = 1/2 ||A w - b||^2 gets grad_w = A^H (A w - b));
* with respect to a real wavenumber k: grad_k = Re <grad_u, (dA/dk) w>
  (Helmholtz and combined-field operators, see ``mult_dk``).

Tensors live on the GPU; the matvecs run on the current torch stream.
"""
import torch

from .operators import IfgfOperator

__all__ = ["matvec"]


def _stream(t):
    return torch.cuda.current_stream(t.device).cuda_stream


class _Matvec(torch.autograd.Function):
    @staticmethod
    def forward(ctx, op, w, k):
        w = w.contiguous()
        u = torch.empty(op.n_tgt, dtype=w.dtype, device=w.device)
        op.mult_device(w.data_ptr(), u.data_ptr(), _stream(w))
        ctx.op = op
        ctx.save_for_backward(w)
        return u

    @staticmethod
    def backward(ctx, grad_u):
        op = ctx.op
        (w,) = ctx.saved_tensors
        g = grad_u.contiguous().to(w.dtype)
        grad_w = grad_k = None
        if ctx.needs_input_grad[1]:
            grad_w = torch.empty(op.n_src, dtype=w.dtype, device=w.device)
            op.mult_adjoint_device(g.data_ptr(), grad_w.data_ptr(), _stream(w))
        if ctx.needs_input_grad[2]:
            du = torch.empty(op.n_tgt, dtype=w.dtype, device=w.device)
            op.mult_dk_device(w.data_ptr(), du.data_ptr(), _stream(w))
            grad_k = torch.real(torch.vdot(g, du)).to(torch.float64).reshape(())
        return None, grad_w, grad_k


def matvec(op: IfgfOperator, w: torch.Tensor, k: torch.Tensor = None) -> torch.Tensor:
    """u = A w with autograd.

    op: an initialised operator; w: CUDA tensor of shape (N,), complex128
    (float64 for Laplace); k: optional 0-d float64 tensor equal to the
    operator's wavenumber, to receive dL/dk (the operator itself stays at its
    construction wavenumber; build a new one to move k).
    """
    if not w.is_cuda:
        raise ValueError("w must be a CUDA tensor")
    if w.shape != (op.n_src,):
        raise ValueError(f"w must have shape ({op.n_src},)")
    if k is None:
        k = torch.zeros((), dtype=torch.float64, device=w.device)
    return _Matvec.apply(op, w, k)
