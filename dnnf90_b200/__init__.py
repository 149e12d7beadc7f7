"""dnnf90_b200: B200 device path of DNNF90's derivative-carrying evaluation.

The forward pass carries every mixed partial derivative of a tanh MLP's
output over a downward-closed multi-index set (the multivariate Faa di Bruno
recursion with partial Bell polynomial tables), and the exact analytic
adjoint returns the weight gradient of any loss seeded on those
derivatives.  The kernels are hand-written CUDA for sm_100a behind a C ABI
(include/dnnf90.h, the reference's 24 entry points, plus the batched and
device-pointer entries of include/dnnf90_b200.h).

Python: ``dnnf90_b200.api`` (ctypes binding and handle objects) and
``dnnf90_b200.autograd`` (torch.autograd.Function over the same ABI).
"""
from .api import (PREC_F64, PREC_SPLIT, SEED_HALFSQ, SEED_JROW, SEED_PINN,  # noqa: F401
                  Dnnf90Error, Grad, Net, SeedRule, TableSet, device_available,
                  jacobian_rows, lib, ngd_step)

__all__ = ["PREC_F64", "PREC_SPLIT", "SEED_HALFSQ", "SEED_PINN", "SEED_JROW",
           "Dnnf90Error", "Grad", "Net", "SeedRule", "TableSet", "device_available",
           "jacobian_rows", "lib", "ngd_step"]
