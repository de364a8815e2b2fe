"""hprqp_b200 — B200 (sm_100a) iteration engine for the HPR-QP solver.

The solver runs in libhprqp.so (CUDA kernels + C ABI, include/hprqp.h);
this package holds its Python binding, the reference-style API and the
synthetic workload generators.
"""
from .api import HPRQP_parameters, HPRQP_results, Solver, optimize
from .model import (LASSO_Q_operator_cpu, QAP_Q_operator_cpu, QP_info, SparseQ, build_from_ABST,
                    build_from_Ab_lambda, build_from_QAbc, qp_formulation)

__all__ = ["HPRQP_parameters", "HPRQP_results", "Solver", "optimize", "QP_info", "SparseQ",
           "LASSO_Q_operator_cpu", "QAP_Q_operator_cpu", "build_from_QAbc", "build_from_Ab_lambda",
           "build_from_ABST", "qp_formulation"]
