"""torch.ops.v2rdm.{Au, ATu, solve, doci_Au, doci_ATu}: the device maps and
the device solve as PyTorch operators on CUDA float64 tensors.

A problem is named by the arguments hilbert builds its tables from (nmo,
nalpha, nbeta, POSITIVITY, CONSTRAIN_SPIN, CONSTRAIN_SZ and the Hubbard
multiplicity convention); the operators build it once per CUDA device and
keep it.  They run on the caller's current stream.  Only CUDA kernels are
registered: a CPU tensor raises, there is no host fallback.

Au and ATu are each other's adjoint, and that is their autograd rule:
d<A x, w>/dx = A^T w and d<A^T y, w>/dy = A w.
"""
import threading

import torch

from .v2rdm import DOCIProblem, Options, V2RDMProblem

_lock = threading.Lock()
_problems = {}


def problem(nmo, nalpha, nbeta, positivity="DQG", constrain_spin=True, constrain_sz=True,
            hubbard_multiplicity=False, device=None):
    """The cached V2RDMProblem for these arguments on this CUDA device."""
    dev = torch.cuda.current_device() if device is None else int(device)
    key = (int(nmo), int(nalpha), int(nbeta), str(positivity), bool(constrain_spin),
           bool(constrain_sz), bool(hubbard_multiplicity), dev)
    with _lock:
        p = _problems.get(key)
        if p is None:
            p = V2RDMProblem(key[0], key[1], key[2], key[3], key[4], key[5],
                             hubbard_multiplicity=key[6])
            _problems[key] = p
    return p


def doci_problem(nmo, nalpha, nbeta, positivity="DQG", device=None):
    """The cached DOCIProblem for these arguments on this CUDA device."""
    dev = torch.cuda.current_device() if device is None else int(device)
    key = ("doci", int(nmo), int(nalpha), int(nbeta), str(positivity), dev)
    with _lock:
        p = _problems.get(key)
        if p is None:
            p = DOCIProblem(key[1], key[2], key[3], key[4])
            _problems[key] = p
    return p


def clear():
    """Release the cached problems (and their device memory)."""
    with _lock:
        items = list(_problems.values())
        _problems.clear()
    for p in items:
        p.close()


def _sizes(nmo, nalpha, nbeta, positivity, constrain_spin, constrain_sz, hubbard_multiplicity):
    # the host tables alone (no device work): n_primal, n_dual
    p = V2RDMProblem(nmo, nalpha, nbeta, positivity, constrain_spin, constrain_sz,
                     hubbard_multiplicity=hubbard_multiplicity)
    try:
        return p.n_primal, p.n_dual
    finally:
        p.close()


@torch.library.custom_op("v2rdm::Au", mutates_args=(), device_types="cuda")
def Au(x: torch.Tensor, nmo: int, nalpha: int, nbeta: int, positivity: str,
       constrain_spin: bool, constrain_sz: bool, hubbard_multiplicity: bool) -> torch.Tensor:
    """A x: hilbert's bpsdp_Au (v2rdm_solver.cc:2995-3050), bit-exact"""
    with torch.cuda.device(x.device):
        p = problem(nmo, nalpha, nbeta, positivity, constrain_spin, constrain_sz,
                    hubbard_multiplicity, x.device.index)
        return p.Au(x.contiguous())


@torch.library.custom_op("v2rdm::ATu", mutates_args=(), device_types="cuda")
def ATu(y: torch.Tensor, nmo: int, nalpha: int, nbeta: int, positivity: str,
        constrain_spin: bool, constrain_sz: bool, hubbard_multiplicity: bool) -> torch.Tensor:
    """A^T y: hilbert's bpsdp_ATu (v2rdm_solver.cc:3054-3108), bit-exact"""
    with torch.cuda.device(y.device):
        p = problem(nmo, nalpha, nbeta, positivity, constrain_spin, constrain_sz,
                    hubbard_multiplicity, y.device.index)
        return p.ATu(y.contiguous())


@torch.library.custom_op("v2rdm::solve", mutates_args=(), device_types="cuda")
def solve(x0: torch.Tensor, b: torch.Tensor, c: torch.Tensor, nmo: int, nalpha: int, nbeta: int,
          positivity: str, constrain_spin: bool, constrain_sz: bool, hubbard_multiplicity: bool,
          r_convergence: float, e_convergence: float, maxiter: int, mu_update_frequency: int,
          cg_convergence: float, cg_maxiter: int) -> torch.Tensor:
    """The converged primal x from x0 (hilbert's outer loop,
    v2rdm_solver.cc:1296-1361, with the device BPSDP solve); x0 is not changed"""
    with torch.cuda.device(x0.device):
        p = problem(nmo, nalpha, nbeta, positivity, constrain_spin, constrain_sz,
                    hubbard_multiplicity, x0.device.index)
        o = Options({"R_CONVERGENCE": r_convergence, "E_CONVERGENCE": e_convergence,
                     "MAXITER": maxiter, "MU_UPDATE_FREQUENCY": mu_update_frequency,
                     "CG_CONVERGENCE": cg_convergence, "CG_MAXITER": cg_maxiter})
        x = x0.contiguous().clone()
        p.solve_device(x, b.contiguous(), c.contiguous(), o)
        return x


@Au.register_fake
def _(x, nmo, nalpha, nbeta, positivity, constrain_spin, constrain_sz, hubbard_multiplicity):
    _, nd = _sizes(nmo, nalpha, nbeta, positivity, constrain_spin, constrain_sz, hubbard_multiplicity)
    return x.new_empty(nd)


@ATu.register_fake
def _(y, nmo, nalpha, nbeta, positivity, constrain_spin, constrain_sz, hubbard_multiplicity):
    npr, _ = _sizes(nmo, nalpha, nbeta, positivity, constrain_spin, constrain_sz, hubbard_multiplicity)
    return y.new_empty(npr)


@solve.register_fake
def _(x0, b, c, *args):
    return torch.empty_like(x0)


@torch.library.custom_op("v2rdm::doci_Au", mutates_args=(), device_types="cuda")
def doci_Au(x: torch.Tensor, nmo: int, nalpha: int, nbeta: int, positivity: str) -> torch.Tensor:
    """A x of v2RDM-DOCI: hilbert's DOCI bpsdp_Au (v2rdm_doci_solver.cc:1509-1537)"""
    with torch.cuda.device(x.device):
        return doci_problem(nmo, nalpha, nbeta, positivity, x.device.index).Au(x.contiguous())


@torch.library.custom_op("v2rdm::doci_ATu", mutates_args=(), device_types="cuda")
def doci_ATu(y: torch.Tensor, nmo: int, nalpha: int, nbeta: int, positivity: str) -> torch.Tensor:
    """A^T y of v2RDM-DOCI: hilbert's DOCI bpsdp_ATu (v2rdm_doci_solver.cc:1539-1566)"""
    with torch.cuda.device(y.device):
        return doci_problem(nmo, nalpha, nbeta, positivity, y.device.index).ATu(y.contiguous())


def _doci_sizes(nmo, nalpha, nbeta, positivity):
    p = DOCIProblem(nmo, nalpha, nbeta, positivity)   # host tables only
    try:
        return p.n_primal, p.n_dual
    finally:
        p.close()


@doci_Au.register_fake
def _(x, nmo, nalpha, nbeta, positivity):
    return x.new_empty(_doci_sizes(nmo, nalpha, nbeta, positivity)[1])


@doci_ATu.register_fake
def _(y, nmo, nalpha, nbeta, positivity):
    return y.new_empty(_doci_sizes(nmo, nalpha, nbeta, positivity)[0])


def _setup(ctx, inputs, output):
    ctx.spec = inputs[1:]


def _Au_backward(ctx, grad):
    return (torch.ops.v2rdm.ATu(grad.contiguous(), *ctx.spec),) + (None,) * len(ctx.spec)


def _ATu_backward(ctx, grad):
    return (torch.ops.v2rdm.Au(grad.contiguous(), *ctx.spec),) + (None,) * len(ctx.spec)


Au.register_autograd(_Au_backward, setup_context=_setup)
ATu.register_autograd(_ATu_backward, setup_context=_setup)


def _doci_Au_backward(ctx, grad):
    return (torch.ops.v2rdm.doci_ATu(grad.contiguous(), *ctx.spec),) + (None,) * len(ctx.spec)


def _doci_ATu_backward(ctx, grad):
    return (torch.ops.v2rdm.doci_Au(grad.contiguous(), *ctx.spec),) + (None,) * len(ctx.spec)


doci_Au.register_autograd(_doci_Au_backward, setup_context=_setup)
doci_ATu.register_autograd(_doci_ATu_backward, setup_context=_setup)
