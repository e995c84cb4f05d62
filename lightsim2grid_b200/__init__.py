"""lightsim2grid_b200: batched AC Newton-Raphson power flow on NVIDIA B200 (sm_100a).

Drop-in for lightsim2grid's Newton-Raphson solver and batch layers: ``SolverType`` /
``ErrorType``, ``GPUNRSolverSingleSlack`` / ``GPUNRSolver`` (method set of
``KLUSolverSingleSlack`` / ``KLUSolver``), ``newtonpf``, ``ContingencyAnalysisCPP`` and
``TimeSeriesCPP``.  The compute path is the native library built from ``csrc/`` (C ABI in
``include/lightsim2grid_b200.h``); nothing falls back to the CPU.
"""
from .solver import (SolverType, ErrorType, FDPFMethod, GPUNRSolver, GPUNRSolverSingleSlack, GPUNRMixedSolver,
                     GPUDCSolver, GPUFDPFSolverXB, GPUFDPFSolverBX, GPUNRMixedSolverSingleSlack, Plan, SOLVER_CLASSES,
                     GPU_SOLVERS)
from .newtonpf import newtonpf, newtonpf_new, newtonpf_old
from .gridmodel import GridModel, Coeff
from .computers import ContingencyAnalysisCPP, TimeSeriesCPP, ContingencyAnalysis, SecurityAnalysis, TimeSerie

__version__ = "0.1.0"

__all__ = ["SolverType", "ErrorType", "FDPFMethod", "GPUDCSolver", "GPUFDPFSolverXB", "GPUFDPFSolverBX", "GPUNRSolver", "GPUNRSolverSingleSlack", "GPUNRMixedSolver",
           "GPUNRMixedSolverSingleSlack", "Plan", "SOLVER_CLASSES", "GPU_SOLVERS", "newtonpf", "newtonpf_new",
           "newtonpf_old", "GridModel", "Coeff", "ContingencyAnalysisCPP", "TimeSeriesCPP", "ContingencyAnalysis",
           "SecurityAnalysis", "TimeSerie"]
