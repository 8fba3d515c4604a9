"""PyTorch autograd binding of the batched GFN2-xTB energy and nuclear gradient.

The reference's Python package returns energies and gradients of one molecule as numpy arrays
(crates/axtb-py/src/engine.rs:230-256, through driver::Calculator::compute); it has no autograd.
Here the same single points run batched on the GPU on device tensors, and the gradient is the
engine's analytic one (energy-weighted density and converged potentials contracted with
integral derivatives recomputed on the fly, plus the classical and CN chain terms):

    e = GFN2Energy.apply(positions, batch)      # positions: (natoms, 3) float64 CUDA, bohr
    e.sum().backward()                          # positions.grad = dE/dR

`positions` packs every molecule's atoms in batch order; `batch` is an axtb_b200.Batch set up
for the same molecules. GFN2 (a torch.nn.Module) takes padded [B, Nmax, 3] positions instead.
There is no CPU path: the tensors must live on the GPU the batch runs on.
"""
from __future__ import annotations

import numpy as np
import torch

from .calculator import AxtbError, Batch


def _engine_stream(batch: Batch) -> torch.cuda.ExternalStream:
    return torch.cuda.ExternalStream(batch.stream)


class GFN2Energy(torch.autograd.Function):
    """forward: per-molecule total energies (nmol,); backward: grad_output[mol(atom)] * dE/dR."""

    @staticmethod
    def forward(ctx, positions: torch.Tensor, batch: Batch) -> torch.Tensor:
        if not positions.is_cuda or positions.dtype != torch.float64:
            raise TypeError("positions must be a float64 CUDA tensor (bohr)")
        natoms = int(batch.natoms.sum())
        if tuple(positions.shape) != (natoms, 3):
            raise ValueError(f"positions must be ({natoms}, 3) for this batch, got {tuple(positions.shape)}")
        x = positions.detach().contiguous()
        energy = torch.empty(batch.nmol, dtype=torch.float64, device=x.device)
        grad = torch.empty_like(x)
        eng = _engine_stream(batch)
        eng.wait_stream(torch.cuda.current_stream(x.device))  # positions are ready
        st = batch.run_device(x.data_ptr(), energy.data_ptr(), grad.data_ptr(), gradient=True)
        torch.cuda.current_stream(x.device).wait_stream(eng)  # outputs are ready
        bad = np.nonzero(st)[0]
        if len(bad):
            raise AxtbError(int(st[bad[0]]), f"{len(bad)} molecule(s) failed, first: index {bad[0]}")
        atom_mol = torch.as_tensor(np.repeat(np.arange(batch.nmol), batch.natoms), device=x.device)
        ctx.save_for_backward(grad, atom_mol)
        return energy

    @staticmethod
    def backward(ctx, grad_energy: torch.Tensor):
        grad, atom_mol = ctx.saved_tensors
        return grad_energy.index_select(0, atom_mol).unsqueeze(1) * grad, None


class GFN2(torch.nn.Module):
    """Energies of a fixed set of molecules for padded positions [B, Nmax, 3] (bohr, float64,
    CUDA): atoms beyond a molecule's count are ignored and get zero gradient."""

    def __init__(self, molecules, **options):
        super().__init__()
        self.batch = Batch(molecules, **options)
        counts = torch.as_tensor(self.batch.natoms)
        nmax = int(counts.max())
        mask = torch.arange(nmax)[None, :] < counts[:, None]
        self.register_buffer("flat_index", torch.nonzero(mask.reshape(-1)).reshape(-1), persistent=False)
        self.nmax = nmax

    def forward(self, positions: torch.Tensor) -> torch.Tensor:
        b = self.batch.nmol
        if positions.shape[0] != b or positions.shape[2] != 3 or positions.shape[1] < self.nmax:
            raise ValueError(f"positions must be [{b}, >= {self.nmax}, 3], got {tuple(positions.shape)}")
        flat = positions[:, : self.nmax].reshape(-1, 3).index_select(0, self.flat_index.to(positions.device))
        return GFN2Energy.apply(flat, self.batch)

    def close(self):
        self.batch.close()
