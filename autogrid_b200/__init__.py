"""AutoGrid-B200: AutoGrid 4 grid maps computed by hand-written sm_100a kernels.

Public API:
    run_gpf(gpf, glg)            drop-in for `autogrid4 -p gpf -l glg`
    Job(gpf, glg)                front end (GPF, receptor, tables, bond vectors)
    Context(device).compute(p)   hot path on one problem (FP32 or FP64 twin)
    Context(device).plan(p)      device-resident plan for repeated runs
    Batch(ctx, problems)         many boxes in one persistent, graph-captured launch
    Diff(ctx, p)                 differentiable mode: linear tables, hand-written adjoint
    torch_maps.GridMaps(job)     torch.autograd binding of the differentiable mode
"""
from ._abi import AutoGridError, load_library  # noqa: F401
from .api import Batch, Context, Diff, Job, MapText, Plan, Problem, Stats, run_gpf  # noqa: F401

__all__ = ["AutoGridError", "Batch", "Context", "Diff", "Job", "MapText", "Plan", "Problem", "Stats", "load_library", "run_gpf"]
