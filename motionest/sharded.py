"""Shot-sharded JointRecon over several GPUs, one process per GPU.

The reference reconstructs on one device; its normal operator is a sum over shots,
A = M sum_s T_s^H C^H F^H M_s F C T_s (image_estimation.py:106-129), and its LM step is
independent per shot given the image (transform_estimation.py:39-144).  So the shots shard:
every rank holds all coil maps, the image and the CG vectors, and its own contiguous block of
shots.  The exchanges are
- one all-reduce of the image per normal-operator application and one for the right-hand
  side: each rank's partial sum over its shots (already masked, and masking commutes with the
  sum) summed over the ranks;
- after each LM step, the ranks' rows of the transforms, damping and flags, gathered by an
  all-reduce of zero-padded copies (adding zeros is exact), then the mean transform over all
  shots is removed and applied to the image on every rank, as the reference does;
- the objective, a sum of the ranks' residual energies.
The CG scalars come from replicated vectors, but an all-reduce need not give bit-identical
results on every rank, so the CG stopping decision is itself agreed by a collective (a sum of
the ranks' stop votes: every rank stops when any rank would).  Every rank therefore issues the
same collectives in the same order.

The collectives go through a communicator with `rank`, `world` and `all_reduce(tensor)` (a sum,
in place): `TorchComm` wraps torch.distributed (NCCL between GPUs), `SoloComm` is one rank.
"""
import numpy as np
import torch

from . import _lib
from ._lib import ptr
from .image_estimation import cg_solve
from .joint_recon import JointRecon
from .problem import SenseProblem
from .transform_estimation import _JAC, LMState, geodesic_step


class TorchComm:
    """The default torch.distributed process group (or `group`) as a communicator."""

    def __init__(self, group=None):
        import torch.distributed as dist
        if not dist.is_initialized():
            raise RuntimeError("ShardedJointRecon needs an initialised torch.distributed "
                               "process group (or a communicator)")
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def all_reduce(self, t):
        import torch.distributed as dist
        v = torch.view_as_real(t) if t.is_complex() else t
        dist.all_reduce(v, op=dist.ReduceOp.SUM, group=self.group)
        return t


class SoloComm:
    """One rank holding every shot: the all-reduce is the identity."""
    rank, world = 0, 1

    def all_reduce(self, t):
        return t


def shot_range(nshots, rank, world):
    """The contiguous block of shots [lo, hi) that `rank` of `world` reconstructs."""
    return nshots * rank // world, nshots * (rank + 1) // world


def lm_accept_gather(comm, stats, e1, t, t_next, lo, hi, damp, flags, tol):
    """Accept or reject the LM proposal of each of this rank's shots, gather all ranks' rows, and
    remove the mean transform.

    For this rank's shots s in [lo, hi), with e0 = stats[s - lo, 0] (transform_estimation.py:
    138-144): if e1 < e0 the proposal is taken, the damping is divided by 5 (floor 1e-4) and the
    shot is flagged when no parameter moved by tol or more; otherwise the damping is multiplied by
    1.5 (cap 1e16).  t [S, 6], damp [S] and flags [S] are updated in place on every rank; the
    mean of t over all S shots is subtracted from t and returned."""
    tl, dl, fl = t[lo:hi], damp[lo:hi], flags[lo:hi]
    acc = e1 < stats[:, 0]
    conv = acc & ((tl - t_next).abs() < tol).all(dim=1)
    fl.copy_(torch.where(conv, torch.ones_like(fl), fl))
    tl.copy_(torch.where(acc[:, None], t_next, tl))
    # divide by a tensor: a scalar divisor may be applied as a multiplication by its reciprocal,
    # which would round differently from the single-process accept kernel
    five = torch.full_like(dl, 5.0)
    dl.copy_(torch.where(acc, torch.clamp(dl / five, min=1e-4), torch.clamp(dl * 1.5, max=1e16)))
    for buf in (t, damp):
        g = torch.zeros_like(buf)
        g[lo:hi] = buf[lo:hi]
        comm.all_reduce(g)
        buf.copy_(g)
    g = torch.zeros(flags.shape, dtype=torch.float64, device=flags.device)
    g[lo:hi] = flags[lo:hi].to(torch.float64)
    comm.all_reduce(g)
    flags.copy_(g.to(flags.dtype))
    # the shots are summed in shot order, as the single-process accept kernel does, so that one
    # rank holding every shot reproduces it bit for bit
    total = t[0].clone()
    for s in range(1, t.shape[0]):
        total += t[s]
    mean = total / torch.full_like(total, float(t.shape[0]))
    t -= mean
    return mean


class _ReducedProblem:
    """This rank's SENSE problem, with the normal operator and right-hand side summed over the
    ranks; everything else is the rank's own."""

    def __init__(self, pb, comm):
        self._pb = pb
        self._comm = comm

    def __getattr__(self, name):
        return getattr(self._pb, name)

    def normal(self, p, out, **kw):
        self._pb.normal(p, out, **kw)
        return self._comm.all_reduce(out)

    def rhs(self, out, **kw):
        self._pb.rhs(out, **kw)
        return self._comm.all_reduce(out)

    def residual(self, x, out, energies=None, **kw):
        """b - A x summed over the ranks (one all-reduce); the energies stay the rank's own."""
        self._pb.residual(x, out, energies, **kw)
        return self._comm.all_reduce(out)

    def agree_stop(self, stop):
        """Stop CG on every rank when any rank's stopping test passes."""
        return agree_any(self._comm, stop, self._pb.device)


def agree_any(comm, flag, device):
    """True on every rank when `flag` is true on at least one rank (one all-reduce)."""
    v = torch.tensor([1.0 if flag else 0.0], dtype=torch.float64, device=device)
    comm.all_reduce(v)
    return bool(v.item() > 0.0)


class ShardedJointRecon(JointRecon):
    """JointRecon with the shots split over the ranks of `comm` (default: the torch.distributed
    process group).  Same arguments and results as JointRecon; each rank passes the same inputs
    and gets the same image and transforms.  `batch` and `lm_batch` count the rank's shots."""

    def __init__(self, ksp, mps, shot_mask, kgrid, rkgrid, t0=None, max_cg_iter=3,
                 max_nm_iter=1, max_joint_iter=100, xp=np, jacobian="reference", batch=None,
                 lm_batch=None, tol=1e-6, comm=None, use_ga=False, ga_mode="reference",
                 fused_residual=True):
        self.comm = comm if comm is not None else TorchComm()
        super().__init__(ksp, mps, shot_mask, kgrid, rkgrid, t0=t0, max_cg_iter=max_cg_iter,
                         max_nm_iter=max_nm_iter, max_joint_iter=max_joint_iter, xp=xp,
                         jacobian=jacobian, batch=batch, lm_batch=lm_batch, tol=tol,
                         use_ga=use_ga, ga_mode=ga_mode, fused_residual=fused_residual)
        self._reduced = _ReducedProblem(self.pb, self.comm)

    def _make_problem(self, ksp_u, mps_u, planes_u, kgrid, rkgrid, batch, lm_batch):
        if self.num_shots < self.comm.world:
            raise ValueError(f"{self.num_shots} shots cannot be split over {self.comm.world} ranks")
        self._lo, self._hi = shot_range(self.num_shots, self.comm.rank, self.comm.world)
        return SenseProblem(ksp_u, mps_u, planes_u[self._lo:self._hi], kgrid, rkgrid,
                            self.t[self._lo:self._hi], batch=batch, lm_batch=lm_batch,
                            grid=self.grid)

    def _local_t(self):
        return self.t[self._lo:self._hi]

    def step(self):
        """One outer iteration: CG on the rank-summed normal equations, the LM step on this
        rank's shots with the transforms gathered and the mean removed, x *= M."""
        pb = self.pb
        ready = self._r0_ready()  # the same on every rank: all run the same steps
        self._r0_key = None
        pb.set_transforms(self._local_t())
        self.cg_iterations.append(cg_solve(self._reduced, self.x, self.max_cg_iter, self.tol,
                                           fused=self.fused_residual,
                                           r=self._residual_buffer(), r_ready=ready))
        for _ in range(self.max_nm_iter):
            self.x = self._lm_step()
            self.x.mul_(self.M)
        pb.set_transforms(self._local_t())

    def _lm_step(self, tol=1e-6):
        pb, st = self.pb, self._lm
        tl = self._local_t()
        pb.set_transforms(tl)
        pb.lm_stats(self.x, _JAC[self.jacobian], out=st.stats)
        _lib.call("me_lm_propose", ptr(st.stats), ptr(self.damp[self._lo:self._hi]), ptr(tl),
                  ptr(st.t_next), pb.nshots, _lib.stream_ptr())
        if self.use_ga:
            geodesic_step(pb, self.x, tl, self.damp[self._lo:self._hi], st, _JAC[self.jacobian],
                          self.ga_mode)
        pb.residual_norms(self.x, st.t_next, out=st.e1)
        mean = lm_accept_gather(self.comm, st.stats, st.e1, self.t, st.t_next, self._lo,
                                self._hi, self.damp, self.convergence_flags, tol)
        out = torch.empty_like(self.x)
        pb.apply_transform(self.x, mean.contiguous(), out=out)
        return out

    def objective_tensor(self):
        """sum_s ||M_s (F C T_s x - y)||^2 over all shots (joint_recon.py:108-115), as a float64
        device scalar (one all-reduce).  With fused_residual the same pass leaves the next
        solve's initial residual, summed over the ranks (one more all-reduce, which that solve
        then does not make)."""
        pb = self.pb
        if not self.fused_residual:
            e = pb.residual_norms(self.x, self._local_t())
        else:
            pb.set_transforms(self._local_t())
            e = torch.empty(pb.nshots, dtype=torch.float64, device=pb.device)
            self._reduced.residual(self.x, self._residual_buffer(), energies=e)
        total = e.sum().reshape(1)
        self.comm.all_reduce(total)
        if self.fused_residual:
            self._r0_key = self._state_key()
        return total[0]
