"""PyTorch adapters of litepgo.torch for this package (src/python/torch.py:126-175).

``energy(potential, x)`` and ``response(model, x)`` are first-order outer autograd adapters
like the reference's: only the explicit tensor input is differentiable; an energy saves its
gradient in the forward pass, a response is differentiated through its VJP (reverse mode)
or JVP (forward mode, where the model has one) at a saved copy of the input. The reference
takes one-dimensional CPU float64 tensors; CUDA float64 tensors are accepted here too, and an
energy of a CUDA tensor is evaluated and differentiated on that device without host copies.
``TorchVolumetricMaterial`` (src/python/torch.py:72-94 of the reference) is a
PyVolumetricMaterial whose density W(F, Fp, theta) is written in PyTorch: its derivatives come
from autograd on whatever device F lives on, so with this package's energies they are computed
on the GPU for the whole mesh at once. The shell material class is not part of this path.
"""

import numpy as np
import torch
from torch.autograd.function import once_differentiable

from .energy import QuadraticEnergy, WeightedSumEnergy
from .fem import PyVolumetricMaterial, VolumetricFemEnergyTetP1

__all__ = ["energy", "response", "TorchVolumetricMaterial"]


class TorchVolumetricMaterial(PyVolumetricMaterial):
    """A PyVolumetricMaterial whose density is written in PyTorch.

    Subclass it, set ``num_parameters`` and define ``W(F, Fp, theta)`` as a static or class
    method taking float64 tensors (N,3,3), (N,3,3), (N,k) and returning the (N,) density per
    reference volume; rows must be independent and W twice differentiable in F. ``eval`` takes
    dW/dF by one backward pass, d2W/dF2 by nine more ([n,i,j,k,l] = d2W/dF_ij dF_kl) and
    d2W/dF dtheta by nine more ([n,i,j,a]), on the device of F.
    """

    @classmethod
    def W(cls, F, Fp, theta):
        raise NotImplementedError("TorchVolumetricMaterial subclasses must define W(F, Fp, theta)")

    @classmethod
    def eval(cls, F, Fp, theta, *, outputs):
        need2 = "d2W_dF2" in outputs
        need_th = "d2W_dF_dtheta" in outputs
        need1 = need2 or need_th or "dW_dF" in outputs
        n = F.shape[0]
        with torch.enable_grad():
            Fv = F.detach().clone().requires_grad_(need1)
            th = theta.detach().clone().requires_grad_(need_th)
            W = cls.W(Fv, Fp.detach(), th)
            if tuple(W.shape) != (n,):
                raise ValueError(f"TorchVolumetricMaterial.W must return shape ({n},)")
            out = {"W": W.detach()}
            if need1:
                if not W.requires_grad:
                    dW = torch.zeros_like(Fv)
                else:
                    (dW,) = torch.autograd.grad(W.sum(), Fv, create_graph=need2 or need_th, allow_unused=True)
                    dW = torch.zeros_like(Fv) if dW is None else dW
                out["dW_dF"] = dW.detach()
                if need_th:
                    # [n, i, j, a] = d2W / dF_ij dtheta_a: one backward pass per entry of F.
                    k = th.shape[1]
                    cols = []
                    for i in range(3):
                        for j in range(3):
                            g = None
                            if dW.requires_grad:
                                (g,) = torch.autograd.grad(dW[:, i, j].sum(), th, retain_graph=True, allow_unused=True)
                            cols.append(torch.zeros((n, k), dtype=F.dtype, device=F.device) if g is None else g)
                    out["d2W_dF_dtheta"] = torch.stack(cols, 1).reshape(n, 3, 3, k).detach()
                if need2:
                    rows = []
                    for i in range(3):
                        for j in range(3):
                            if dW.requires_grad:
                                (g,) = torch.autograd.grad(dW[:, i, j].sum(), Fv, retain_graph=True, allow_unused=True)
                            else:
                                g = None
                            rows.append(torch.zeros_like(Fv) if g is None else g)
                    # rows[3 i + j][n, k, l] = d2W / dF_ij dF_kl
                    out["d2W_dF2"] = torch.stack(rows, 1).reshape(n, 3, 3, 3, 3).detach()
        return out


def _check(x):
    if not isinstance(x, torch.Tensor):
        raise TypeError("expected a torch.Tensor")
    if x.dtype != torch.float64 or x.ndim != 1 or x.device.type not in ("cpu", "cuda"):
        raise ValueError("expected a one-dimensional float64 tensor on the CPU or a CUDA device")


def _host(x):
    return x.detach().cpu().numpy().copy()


def _on_device(potential, x, need_gradient):
    """(value, gradient tensor or None) of potential at a CUDA tensor x, on x's device."""
    if isinstance(potential, VolumetricFemEnergyTetP1):
        value, g, _ = potential.eval_device(x.detach(), gradient=need_gradient)
        return value, g
    if isinstance(potential, WeightedSumEnergy):
        fem, w, A, f, c = potential.potential()
        xd = x.detach()
        value, g, _ = fem.eval_device(xd, gradient=need_gradient)
        ft = torch.as_tensor(f, device=x.device)
        value = w * value - float(torch.dot(ft, xd)) + c
        if g is not None:
            g = w * g - ft
        if A is not None:
            A = A.tocsr()
            At = torch.sparse_csr_tensor(torch.as_tensor(A.indptr, dtype=torch.int64),
                                         torch.as_tensor(A.indices, dtype=torch.int64),
                                         torch.as_tensor(A.data, dtype=torch.float64), size=A.shape).to(x.device)
            Ax = torch.mv(At, xd)
            value += 0.5 * float(torch.dot(xd, Ax))
            if g is not None:
                g = g + Ax
        return value, g
    if isinstance(potential, QuadraticEnergy) and potential.is_linear:
        b = torch.as_tensor(potential.b, device=x.device)
        return float(torch.dot(b, x.detach())), (b.clone() if need_gradient else None)
    value, g, _ = potential.eval(_host(x), gradient=need_gradient)
    return value, (torch.as_tensor(np.asarray(g), device=x.device) if need_gradient else None)


class _Energy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, potential, need_gradient):
        if x.is_cuda:
            value, gradient = _on_device(potential, x, need_gradient)
            if need_gradient:
                ctx.save_for_backward(gradient)
        else:
            values = _host(x)
            if need_gradient:
                value, gradient, _ = potential.eval(values, gradient=True)
                ctx.save_for_backward(torch.from_numpy(np.array(gradient, copy=True)))
            else:
                value = potential.eval_value(values)
        return torch.tensor(value, dtype=torch.float64, device=x.device)

    @staticmethod
    @once_differentiable
    def backward(ctx, upstream):
        (gradient,) = ctx.saved_tensors
        return upstream * gradient, None, None


class _Response(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, model):
        ctx.values = _host(x)
        ctx.device = x.device
        ctx.model = model
        value = model.eval_value(ctx.values)
        return torch.as_tensor(np.array(value, dtype=np.float64, copy=True), device=x.device)

    @staticmethod
    @once_differentiable
    def backward(ctx, upstream):
        gradient = ctx.model.eval_vjp(ctx.values, _host(upstream))
        return torch.as_tensor(np.array(gradient, dtype=np.float64, copy=True), device=ctx.device), None

    @staticmethod
    def jvp(ctx, tangent, _model):
        if not hasattr(ctx.model, "eval_jvp"):
            raise NotImplementedError(f"{type(ctx.model).__name__} has no forward-mode product (eval_jvp)")
        product = ctx.model.eval_jvp(ctx.values, _host(tangent))
        return torch.as_tensor(np.array(product, dtype=np.float64, copy=True), device=ctx.device)


def energy(potential, x):
    """Evaluates an Energy at x (CPU or CUDA float64 1-D); differentiates with respect to x only."""
    _check(x)
    return _Energy.apply(x, potential, torch.is_grad_enabled() and x.requires_grad)


def response(model, x):
    """Evaluates a Response; reverse / forward AD use its VJP / JVP, differentiating x only."""
    _check(x)
    return _Response.apply(x, model)
