"""Drop-in for stojl/SigPDE's `sigpde.torch` (sigpde/torch/__init__.py:9-16):

    import sigpde_b200.torch as sig
    k = sig.SigPDE(sig.kernels.LinearKernel(), dyadic_order=2)
    k.gram(x, y)
"""
from . import autotune, ragged
from . import static_kernels as kernels
from .kernel import RobustSigPDE, SigPDE, gram_inner_product, log_normalizer, pairwise_inner_product

__all__ = ["SigPDE", "RobustSigPDE", "kernels", "ragged", "autotune", "log_normalizer", "pairwise_inner_product", "gram_inner_product"]
