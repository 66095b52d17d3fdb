"""gato_b200: batched SQP trajectory optimisation on NVIDIA B200 (sm_100a).

Drop-in for the reference's Python solver class `bsqp.interface.BSQP`;
the compute path is the CUDA library libgato_b200.so behind the C ABI in
include/gato_b200.h.
"""
from .interface import BSQP  # noqa: F401
from ._lib import GatoError, builtin_model, load  # noqa: F401

__all__ = ["BSQP", "GatoError", "builtin_model", "load", "solve_differentiable"]


def solve_differentiable(*args, **kwargs):
    """Differentiable batched solve (gato_b200.autograd.solve_differentiable)."""
    from .autograd import solve_differentiable as f
    return f(*args, **kwargs)
