"""ainv_b200: B200 application phase of the MLD2P4 AINV plugin.

Host-side mirror of the plugin solver types over the C-ABI of
libainv_b200.so (include/ainv_b200.h).
"""
from ._lib import (AINV_ALG, KRYLOV, PREC, AinvError, LIB_PATH, check, last_error, lib)
from .device import DeviceFactors, DeviceOperator, SolveResult
from .solver import (mld_d_ainv_solver_type, mld_d_invk_solver_type,
                     mld_d_invt_solver_type)
from . import pde
from .serve import SolveServer

__all__ = ["AINV_ALG", "KRYLOV", "PREC", "AinvError", "LIB_PATH", "check", "last_error", "lib",
           "DeviceFactors", "DeviceOperator", "SolveResult", "mld_d_ainv_solver_type",
           "mld_d_invk_solver_type", "mld_d_invt_solver_type", "pde", "SolveServer"]
