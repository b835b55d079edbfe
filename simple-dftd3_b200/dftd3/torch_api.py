"""PyTorch autograd wrapper of the batched GPU evaluation.

``DispersionEnergy`` is a ``torch.autograd.Function``: when an input requires
a gradient, the forward pass evaluates the energies together with the analytic
gradient, virial and damping parameter derivatives in one pass (keeping those
O(natoms) results, not the pair and triple quantities); otherwise it evaluates
the energies only.  The backward pass applies the chain rule to

* the Cartesian positions (Bohr),
* a per-system strain tensor eps: positions x' = x (I + eps)^T and lattice
  L' = L (I + eps)^T, so dE/deps = sigma(x') (I + eps)^-T with the virial
  sigma of the reference (dE/deps at eps = 0),
* the damping parameters (s6, s8, a1, a2, s9) of rational damping or
  (s6, s8, rs6, rs8, s9) of zero damping.

Tensors live on the current CUDA device in float64; the library runs on the
current torch stream.  ``D3Batch`` is the user-facing module.
"""
from typing import Optional, Sequence

import numpy as np
import torch

from . import library

_PARAM_NAMES = {"rational": ("s6", "s8", "a1", "a2", "s9"), "zero": ("s6", "s8", "rs6", "rs8", "s9")}


class D3Batch:
    """Independent systems with fixed atomic numbers evaluated together.

    numbers: one integer array per system.  lattices (nsys, 3, 3, rows =
    lattice vectors) and periodic (nsys, 3) are optional.  damping is
    "rational" or "zero"; alp is fixed (14 by default); precision is "mixed"
    or "fp64".  Calling the object returns the (nsys,) energy tensor.
    """

    def __init__(self, numbers: Sequence[np.ndarray], lattices: Optional[np.ndarray] = None,
                 periodic: Optional[np.ndarray] = None, damping: str = "rational", alp: float = 14.0,
                 precision: str = "mixed", cutoffs: Optional[Sequence[float]] = None):
        if damping not in _PARAM_NAMES:
            raise ValueError(f"Unknown damping '{damping}'")
        self.damping = damping
        self.alp = float(alp)
        self.natoms = np.ascontiguousarray([len(n) for n in numbers], dtype=np.int32)
        self.offsets = np.concatenate([[0], np.cumsum(self.natoms)]).astype(np.int64)
        nums = np.ascontiguousarray(np.concatenate([np.asarray(n) for n in numbers]), dtype=np.int32)
        self.lattices = None if lattices is None else np.ascontiguousarray(lattices, dtype=float).reshape(-1, 3, 3)
        per = None if periodic is None else np.ascontiguousarray(periodic, dtype=bool)
        self.batch = library.new_batch(self.natoms, nums, self.lattices, per)
        library.set_batch_precision(self.batch, library.PRECISION_MIXED if precision == "mixed"
                                    else library.PRECISION_FP64)
        if cutoffs is not None:
            library.set_batch_realspace_cutoff(self.batch, *cutoffs)
        sys_index = np.repeat(np.arange(len(self.natoms)), self.natoms)
        self._sys_index = torch.as_tensor(sys_index, dtype=torch.long)

    def __len__(self):
        return len(self.natoms)

    def param_handle(self, values):
        s6, s8, p1, p2, s9 = (float(v) for v in values)
        if self.damping == "rational":
            return library.new_rational_damping(s6, s8, s9, p1, p2, self.alp)
        return library.new_zero_damping(s6, s8, s9, p1, p2, self.alp)

    def strained(self, positions: torch.Tensor, strain: Optional[torch.Tensor]):
        """Strained positions and host lattices for a (nsys, 3, 3) strain."""
        if strain is None:
            return positions, self.lattices
        idx = self._sys_index.to(positions.device)
        deform = torch.eye(3, dtype=positions.dtype, device=positions.device) + strain
        pos = torch.einsum("nb,nab->na", positions, deform[idx])
        lat = None
        if self.lattices is not None:
            d = deform.detach().cpu().numpy()
            lat = np.ascontiguousarray(np.einsum("skb,sab->ska", self.lattices, d))
        return pos, lat

    def __call__(self, positions: torch.Tensor, params: torch.Tensor,
                 strain: Optional[torch.Tensor] = None) -> torch.Tensor:
        if strain is None:
            strain = torch.zeros((len(self), 3, 3), dtype=positions.dtype, device=positions.device)
        return DispersionEnergy.apply(positions, params, strain, self)


def _evaluate(model: D3Batch, positions, params, strain, derivatives: bool):
    pos, lat = model.strained(positions.detach(), strain.detach())
    pos = pos.contiguous()
    nsys = len(model)
    dev = positions.device
    energies = torch.zeros(nsys, dtype=torch.float64, device=dev)
    grad = torch.zeros_like(pos) if derivatives else None
    sigma = torch.zeros((nsys, 9), dtype=torch.float64, device=dev) if derivatives else None
    pgrad = torch.zeros((nsys, 5), dtype=torch.float64, device=dev) if derivatives else None
    param = model.param_handle(params.detach().cpu().tolist())
    stream = torch.cuda.current_stream(dev).cuda_stream
    library.get_dispersion_device(model.batch, param, pos.data_ptr(), lat, energies.data_ptr(),
                                  grad.data_ptr() if derivatives else 0,
                                  sigma.data_ptr() if derivatives else 0,
                                  pgrad.data_ptr() if derivatives else 0, stream)
    return energies, grad, sigma, pgrad


class DispersionEnergy(torch.autograd.Function):
    """Per-system D3 energies with the analytic derivatives of the same pass."""

    @staticmethod
    def forward(ctx, positions, params, strain, model):
        derivatives = any(ctx.needs_input_grad[:3])
        energies, grad, sigma, pgrad = _evaluate(model, positions, params, strain, derivatives=derivatives)
        ctx.model = model
        if derivatives:
            ctx.save_for_backward(positions, params, strain, grad, sigma, pgrad)
        return energies

    @staticmethod
    def backward(ctx, grad_e):
        positions, params, strain, grad, sigma, pgrad = ctx.saved_tensors
        model = ctx.model
        idx = model._sys_index.to(positions.device)
        ge = grad_e.to(torch.float64)
        deform = torch.eye(3, dtype=torch.float64, device=positions.device) + strain.detach()
        g_pos = g_params = g_strain = None
        if ctx.needs_input_grad[0]:
            # x' = x (I + eps)^T: dE/dx = dE/dx' (I + eps)
            g_pos = ge[idx, None] * torch.einsum("na,nab->nb", grad, deform[idx])
        if ctx.needs_input_grad[1]:
            g_params = (ge[:, None] * pgrad).sum(0)
        if ctx.needs_input_grad[2]:
            # sigma is stored in the reference's (column-major) order: element (a, b) at a + 3 b
            sig = sigma.reshape(-1, 3, 3).transpose(1, 2)
            g_strain = ge[:, None, None] * (sig @ torch.linalg.inv(deform).transpose(1, 2))
        return g_pos, g_params, g_strain, None
