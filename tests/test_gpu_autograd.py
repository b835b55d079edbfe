"""GPU tests of the torch.autograd wrapper: forward energies and the analytic
backward pass w.r.t. positions, cell strain and damping parameters,
against the FP64 oracle (its energies, gradient and virial) and central finite
differences."""
import numpy as np
import pytest

import oracle_ref as O

pytestmark = pytest.mark.gpu


def _frames(nframes=3, natoms=40, seed=21):
    from dftd3 import synthetic as S
    rng = np.random.default_rng(seed)
    nums, pos, lats = [], [], []
    for _ in range(nframes):
        box = rng.uniform(12.0, 13.0)
        lat = np.eye(3) * box + rng.uniform(-0.4, 0.4, size=(3, 3))
        nums.append(rng.choice([1, 6, 7, 8], size=natoms, p=[0.4, 0.3, 0.15, 0.15]).astype(np.int32))
        pos.append(S.pack_cell(rng, natoms, lat, 1.9))
        lats.append(lat)
    return nums, pos, np.array(lats)


CUT = (20.0, 12.0, 15.0, 0.0, 0.0)   # disp2, disp3, cn, width2, width3 (small cell test)


def _oracle_energy(num, pos, lat, par, strain=None):
    d = np.eye(3) if strain is None else np.eye(3) + strain
    return O.dispersion(num, np.asarray(pos) @ d.T, par, lattice=lat @ d.T, periodic=[True] * 3,
                        cutoff=CUT, grad=False, wrap=False)["energy"]


def _model(nums, lats, precision, damping="rational"):
    from dftd3.torch_api import D3Batch
    return D3Batch(nums, lattices=lats, periodic=np.ones((len(nums), 3), dtype=bool), damping=damping,
                   precision=precision, cutoffs=CUT)


@pytest.mark.parametrize("damping", ["rational", "zero"])
def test_forward_and_position_gradient_fp64(damping):
    import torch
    nums, pos, lats = _frames()
    model = _model(nums, lats, "fp64", damping)
    if damping == "rational":
        pvals = [1.0, 0.7875, 0.4289, 4.4407, 1.0]
        par = dict(damping="rational", s6=1.0, s8=0.7875, a1=0.4289, a2=4.4407, s9=1.0, alp=14.0)
    else:
        pvals = [1.0, 1.703, 1.261, 1.0, 1.0]
        par = dict(damping="zero", s6=1.0, s8=1.703, rs6=1.261, rs8=1.0, s9=1.0, alp=14.0)
    x = torch.tensor(np.concatenate(pos), device="cuda", requires_grad=True)
    params = torch.tensor(pvals, dtype=torch.float64, device="cuda")
    e = model(x, params)
    e.sum().backward()
    off = 0
    for k in range(len(nums)):
        ref = O.dispersion(nums[k], pos[k], par, lattice=lats[k], periodic=[True] * 3, cutoff=CUT, wrap=False)
        assert abs(e[k].item() - ref["energy"]) <= 1e-12 * abs(ref["energy"])
        g = x.grad[off:off + len(nums[k])].cpu().numpy()
        assert np.abs(g - ref["gradient"]).max() <= 1e-12 * np.abs(ref["gradient"]).max()
        off += len(nums[k])


def test_parameter_and_strain_gradients_fp64():
    import torch
    nums, pos, lats = _frames(nframes=2, natoms=30, seed=3)
    model = _model(nums, lats, "fp64")
    pvals = np.array([1.0, 0.7875, 0.4289, 4.4407, 1.0])
    x = torch.tensor(np.concatenate(pos), device="cuda")
    params = torch.tensor(pvals, dtype=torch.float64, device="cuda", requires_grad=True)
    rng = np.random.default_rng(0)
    eps0 = rng.uniform(-0.01, 0.01, size=(2, 3, 3))
    strain = torch.tensor(eps0, device="cuda", requires_grad=True)
    w = torch.tensor([0.7, -1.3], dtype=torch.float64, device="cuda")
    loss = (w * model(x, params, strain)).sum()
    loss.backward()

    def loss_oracle(pv, eps):
        tot = 0.0
        for k in range(2):
            par = dict(damping="rational", s6=pv[0], s8=pv[1], a1=pv[2], a2=pv[3], s9=pv[4], alp=14.0)
            tot += [0.7, -1.3][k] * _oracle_energy(nums[k], pos[k], lats[k], par, eps[k])
        return tot

    # damping parameters: central differences
    for p in range(5):
        h = 1e-5 * max(abs(pvals[p]), 1.0)
        up, dn = pvals.copy(), pvals.copy()
        up[p] += h; dn[p] -= h
        fd = (loss_oracle(up, eps0) - loss_oracle(dn, eps0)) / (2 * h)
        assert abs(params.grad[p].item() - fd) <= 1e-7 * max(abs(fd), 1e-6), (p, params.grad[p].item(), fd)
    # strain: central differences on two components of each frame
    for k in range(2):
        for (a, b) in ((0, 0), (1, 2)):
            h = 1e-6
            ep, em = eps0.copy(), eps0.copy()
            ep[k, a, b] += h; em[k, a, b] -= h
            fd = (loss_oracle(pvals, ep) - loss_oracle(pvals, em)) / (2 * h)
            assert abs(strain.grad[k, a, b].item() - fd) <= 1e-6 * max(abs(fd), 1e-4), (k, a, b)


def test_mixed_forward_backward_finite_differences():
    """Mixed forward + analytic backward, central differences with h = 1e-4 Bohr."""
    import torch
    nums, pos, lats = _frames(nframes=2, natoms=32, seed=8)
    model = _model(nums, lats, "mixed")
    pvals = [1.0, 0.7875, 0.4289, 4.4407, 1.0]
    params = torch.tensor(pvals, dtype=torch.float64, device="cuda")
    x0 = np.concatenate(pos)
    x = torch.tensor(x0, device="cuda", requires_grad=True)
    model(x, params).sum().backward()
    g = x.grad.cpu().numpy()
    h = 1e-4
    rng = np.random.default_rng(1)
    for idx in rng.choice(len(x0), size=6, replace=False):
        for c in range(3):
            xp, xm = x0.copy(), x0.copy()
            xp[idx, c] += h; xm[idx, c] -= h
            fd = 0.0
            for k in range(2):
                par = dict(damping="rational", s6=1.0, s8=0.7875, a1=0.4289, a2=4.4407, s9=1.0, alp=14.0)
                sl = slice(32 * k, 32 * (k + 1))
                fd += (_oracle_energy(nums[k], xp[sl], lats[k], par) - _oracle_energy(nums[k], xm[sl], lats[k], par)) / (2 * h)
            assert abs(g[idx, c] - fd) <= 1e-7 + 1e-5 * abs(fd), (idx, c, g[idx, c], fd)


def test_gradcheck_small_fp64():
    import torch
    nums, pos, lats = _frames(nframes=1, natoms=12, seed=5)
    model = _model(nums, lats, "fp64")
    x = torch.tensor(np.concatenate(pos), device="cuda", requires_grad=True)
    params = torch.tensor([1.0, 0.7875, 0.4289, 4.4407, 1.0], dtype=torch.float64, device="cuda",
                          requires_grad=True)
    strain = torch.zeros((1, 3, 3), dtype=torch.float64, device="cuda", requires_grad=True)
    # the three-body scatter adds with atomics: repeated backward passes agree to rounding
    assert torch.autograd.gradcheck(lambda a, b, c: model(a, b, c), (x, params, strain), eps=1e-6, atol=1e-7,
                                    rtol=1e-5, nondet_tol=1e-12)


def test_s9_derivative_at_zero():
    """dE/ds9 at s9 = 0 is the three-body energy at unit s9."""
    import torch
    nums, pos, lats = _frames(nframes=2, natoms=30, seed=13)
    model = _model(nums, lats, "fp64")
    x = torch.tensor(np.concatenate(pos), device="cuda")
    params = torch.tensor([1.0, 0.7875, 0.4289, 4.4407, 0.0], dtype=torch.float64, device="cuda",
                          requires_grad=True)
    model(x, params).sum().backward()
    e3 = 0.0
    for k in range(2):
        p1 = dict(damping="rational", s6=1.0, s8=0.7875, a1=0.4289, a2=4.4407, s9=1.0, alp=14.0)
        p0 = dict(p1, s9=0.0)
        e3 += _oracle_energy(nums[k], pos[k], lats[k], p1) - _oracle_energy(nums[k], pos[k], lats[k], p0)
    assert abs(params.grad[4].item() - e3) <= 1e-10 * abs(e3)
