"""gfk_b200 — B200 (sm_100a) engine for layered-soil Green's-function banks.

The Python side mirrors the reference's Go packages internal/fk, internal/layer,
internal/visco and internal/bank; all computation runs in libgfk (CUDA, C ABI
in include/gfk.h). There is no CPU fallback.
"""
from . import _native
from ._native import DUNKIN, PLAIN_FP64, REFERENCE_DIRECT, SPLIT_INT8
from .fk import (Batch, Engine, FkError, Grid, Integration, Layer, MAX_LAYER_PHASE, Medium, Plan, SLS, Stack,
                 default_engine, prop_shape, uniform)
from .bank import (Bank, DeviceBank, Header, Provenance, RangeGrid, build_bank, open_bank, range_nyquist)
from . import workloads
from . import sobol
from . import surrogate
from . import disp
from . import fdtd

__all__ = ["Batch", "Engine", "FkError", "Grid", "Integration", "Layer", "MAX_LAYER_PHASE", "Medium", "Plan", "SLS",
           "Stack", "default_engine", "prop_shape", "uniform", "Bank", "DeviceBank", "Header", "Provenance", "RangeGrid", "build_bank",
           "open_bank", "range_nyquist", "workloads", "sobol", "surrogate", "disp", "fdtd", "DUNKIN", "REFERENCE_DIRECT", "PLAIN_FP64", "SPLIT_INT8"]
