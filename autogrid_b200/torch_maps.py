"""torch.autograd binding of the differentiable mode (optional; needs torch).

    job = Job("rec.gpf")
    maps_fn = GridMaps(job, device=0)                  # FP32 kernels
    coords = torch.tensor(job.problem().arrays["coord"], requires_grad=True)
    charges = torch.tensor(job.problem().arrays["charge"], requires_grad=True)
    maps = maps_fn(coords, charges)                    # [n_maps, n1z, n1y, n1x] on cuda
    loss = (w * maps).sum(); loss.backward()           # coords.grad, charges.grad

Coordinates are in the problem's centred frame.  Everything stays on the
device: the forward hands the coordinates and charges to the engine as device
arrays (ag_diff_set_atoms_device), which rebuilds the bond vectors on the bond
topology found at load time (ag_job_bond_topology) and the cell lists, then
computes the maps into the output tensor; the backward runs the hand-written
adjoint kernels and the bond-vector chain rule on the device
(ag_diff_backward_device).  The closest DS/D1 atom of each grid point is
searched at the first forward and kept afterwards (keep_closest_h=False
searches it at every forward).

Sharded over GPUs (one process per GPU): GridMaps(job, device, zslab=(z0, z1))
computes grid planes [z0, z1) only (autogrid_b200.shard.zslab_ranges gives each
rank its slab); the loss over those planes gives each rank a partial gradient
over all atoms, and autogrid_b200.shard.allreduce_gradients([coords.grad,
charges.grad]) sums them with one all-reduce.
"""
from __future__ import annotations

import torch

from .api import Context, Diff, Job


class GridMaps:
    """Callable (coords [N,3], charges [N]) -> maps, differentiable in both."""

    def __init__(self, job: Job, device: int = 0, precision: str = "fp32", keep_closest_h: bool = True,
                 zslab: tuple | None = None):
        self.job = job
        self.problem = job.problem()
        if zslab is not None:
            from .shard import zslab_problem
            self.problem = zslab_problem(self.problem, int(zslab[0]), int(zslab[1]))
        self.device = torch.device("cuda", device)
        self.ctx = Context(device)
        self.diff = Diff(self.ctx, self.problem, precision)
        self.diff.set_bonds(job)
        self.dtype = torch.float64 if precision == "fp64" else torch.float32
        self.keep_closest_h = keep_closest_h
        self.generation = 0
        self._searched = False

    def __call__(self, coords: torch.Tensor, charges: torch.Tensor) -> torch.Tensor:
        return _GridMapsFn.apply(coords, charges, self)

    def _run(self, coord: torch.Tensor, charge: torch.Tensor, out: torch.Tensor) -> None:
        # the inputs are ready and out may reuse memory torch just released
        torch.cuda.current_stream(self.device).synchronize()
        self.diff.set_atoms_device(coord.data_ptr(), charge.data_ptr())
        self.diff.forward(keep_closest_h=self.keep_closest_h and self._searched, device_out=out.data_ptr())
        self._searched = True
        self.generation += 1


class _GridMapsFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, charges, engine: GridMaps):
        coord = coords.detach().to(engine.device, torch.float64).reshape(-1, 3).contiguous()
        charge = charges.detach().to(engine.device, torch.float64).reshape(-1).contiguous()
        out = torch.empty(engine.diff.shape, dtype=engine.dtype, device=engine.device)
        engine._run(coord, charge, out)
        ctx.engine = engine
        ctx.generation = engine.generation
        ctx.coord, ctx.charge = coord, charge
        ctx.shapes = (coords.shape, coords.dtype, coords.device, charges.shape, charges.dtype, charges.device)
        return out

    @staticmethod
    def backward(ctx, grad):
        engine: GridMaps = ctx.engine
        if engine.generation != ctx.generation:  # another forward ran since: recompute this one
            scratch = torch.empty(engine.diff.shape, dtype=engine.dtype, device=engine.device)
            keep = engine.keep_closest_h
            engine._run(ctx.coord, ctx.charge, scratch)
            engine.keep_closest_h = keep
        g = grad.to(device=engine.device, dtype=engine.dtype).contiguous()
        g_coord = torch.empty((engine.problem.n_atoms, 3), dtype=torch.float64, device=engine.device)
        g_charge = torch.empty((engine.problem.n_atoms,), dtype=torch.float64, device=engine.device)
        torch.cuda.current_stream(engine.device).synchronize()
        engine.diff.backward_device(g.data_ptr(), g_coord.data_ptr(), g_charge.data_ptr())
        cs, cdt, cdev, qs, qdt, qdev = ctx.shapes
        return (g_coord.reshape(cs).to(device=cdev, dtype=cdt), g_charge.reshape(qs).to(device=qdev, dtype=qdt), None)
