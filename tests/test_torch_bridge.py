"""litepgo_b200.torch: the energy / response autograd adapters (src/python/torch.py:126-175),
host logic on the CPU with pure-Python models, mirroring tests/python/test_torch.py."""

import numpy as np
import pytest
import scipy.sparse as sp

torch = pytest.importorskip("torch")
from litepgo_b200 import energy  # noqa: E402
from litepgo_b200 import torch as bridge  # noqa: E402


class Square:
    """y = x * x with explicit products (a Response with eval_value / eval_vjp / eval_jvp)."""

    num_inputs = num_outputs = 2

    def __init__(self):
        self.products = []

    def eval_value(self, x):
        return np.asarray(x) ** 2

    def eval_vjp(self, x, w):
        self.products.append("vjp")
        return 2 * np.asarray(x) * np.asarray(w)

    def eval_jvp(self, x, dx):
        self.products.append("jvp")
        return 2 * np.asarray(x) * np.asarray(dx)


def test_energy_and_response_gradcheck():
    x = torch.tensor([0.3, 0.7], dtype=torch.float64, requires_grad=True)
    potential = energy.QuadraticEnergy(sp.eye(2, format="csc"), np.ones(2))
    assert torch.autograd.gradcheck(lambda x: bridge.energy(potential, x), (x,))
    model = Square()
    assert torch.autograd.gradcheck(lambda x: bridge.response(model, x), (x,), check_forward_ad=True)
    a, b = bridge.response(model, x), bridge.response(model, 2 * x)
    (a.sum() + b.sum()).backward()
    torch.testing.assert_close(x.grad, 10 * x)


def test_products_only_when_differentiated():
    model = Square()
    x = torch.tensor([0.3, 0.7], dtype=torch.float64, requires_grad=True)
    with torch.no_grad():
        bridge.response(model, x)
    assert model.products == []
    y = bridge.response(model, x)
    y.sum().backward()
    assert model.products == ["vjp"]
    with torch.no_grad(), torch.autograd.forward_ad.dual_level():
        dual = torch.autograd.forward_ad.make_dual(x.detach(), torch.tensor([0.2, -0.4], dtype=torch.float64))
        primal, tangent = torch.autograd.forward_ad.unpack_dual(bridge.response(model, dual))
    torch.testing.assert_close(tangent, 2 * x.detach() * torch.tensor([0.2, -0.4], dtype=torch.float64))
    assert model.products[-1] == "jvp"


def test_forward_owns_an_input_copy():
    model = Square()
    a = torch.tensor([0.3, 0.4], dtype=torch.float64, requires_grad=True)
    saved = a.detach().clone()
    y = bridge.response(model, a)
    with torch.no_grad():
        a.add_(10)
    (g,) = torch.autograd.grad(y.sum(), a)
    torch.testing.assert_close(g, 2 * saved)


def test_double_backward_is_rejected():
    x = torch.ones(2, dtype=torch.float64, requires_grad=True)
    for f in (lambda x: bridge.response(Square(), x).sum(),
              lambda x: bridge.energy(energy.QuadraticEnergy(sp.eye(2, format="csc")), x)):
        first = torch.autograd.grad(f(x), x, create_graph=True)[0]
        with pytest.raises(RuntimeError):
            torch.autograd.grad(first.sum(), x)


def test_argument_errors():
    model = Square()
    x = torch.tensor([0.3, 0.7], dtype=torch.float64)
    with pytest.raises(TypeError):
        bridge.response(model, [0.3, 0.7])
    with pytest.raises(TypeError):
        bridge.energy(energy.QuadraticEnergy(sp.eye(2, format="csc")), np.ones(2))
    with pytest.raises(ValueError):
        bridge.response(model, x.float())
    with pytest.raises(ValueError):
        bridge.response(model, x.reshape(1, 2))
    with pytest.raises(ValueError):
        bridge.energy(energy.QuadraticEnergy(sp.eye(2, format="csc")), torch.tensor([float("nan"), 1.0],
                                                                                     dtype=torch.float64))
