"""Joint image + motion driver with the reference's interface (joint_recon.py:10-115)."""
import numpy as np
import torch

from . import _lib
from ._arrays import to_device
from ._lib import ptr
from .image_estimation import CgGraph, _host_mask, cg_solve
from .problem import SenseProblem, hybrid_kspace, max_abs_image, zxy_to_xyz
from .sampling import plane_masks
from .transform_estimation import LMState, lm_step
from .utils import DeviceGrid

AX3 = (-3, -2, -1)


class JointRecon:
    """Alternate CG-SENSE image estimation and per-shot LM motion estimation.

    Constructor arguments as the reference's JointRecon (centred ksp/mps [C, X, Y, Z], masks
    [S, X, Y, 1], grids, t0, max_cg_iter=3, max_nm_iter=1, max_joint_iter=100, xp).  Extras:
    jacobian ('reference' | 'exact'), batch (shots per normal-operator launch, default all;
    "auto" times the candidates once per problem shape and caches the choice, see
    motionest/autotune.py), lm_batch (shots per LM launch), use_ga / ga_mode (geodesic
    acceleration in the motion step, see estimate_transform; the reference's JointRecon never
    turns it on), cg_graph (run each CG solve as one CUDA graph with the stopping test on the
    device; same results, no host round trip inside the solve), fused_residual (default True:
    each CG solve's initial residual b - A x comes from one pass over the shots instead of the
    right-hand side and A x separately, and the objective computed after a step forms that
    residual for the next step at the same time, since both are taken at the same image and
    transforms; False keeps the reference's order of operations).  run() returns (image [X, Y, Z] complex64 centred, t
    [S, 6] float64) as CUDA tensors, with transform_history and objective_history as NumPy
    arrays, like the reference (which returns CuPy arrays)."""

    def __init__(self, ksp, mps, shot_mask, kgrid, rkgrid, t0=None, max_cg_iter=3, max_nm_iter=1,
                 max_joint_iter=100, xp=np, jacobian="reference", batch=None, lm_batch=None,
                 tol=1e-6, use_ga=False, ga_mode="reference", cg_graph=False,
                 fused_residual=True):
        _lib.require_cuda()
        self.fused_residual = fused_residual
        self.kgrid = kgrid
        self.rkgrid = rkgrid
        self.max_cg_iter = max_cg_iter
        self.max_nm_iter = max_nm_iter
        self.max_joint_iter = max_joint_iter
        self.jacobian = jacobian
        self.tol = tol
        self.use_ga = use_ga
        self.ga_mode = ga_mode
        planes = plane_masks(_host_mask(shot_mask))
        self.num_shots = planes.shape[0]
        self.img_shape = tuple(int(v) for v in to_shape(ksp)[1:])
        # uncentre and move to the device (joint_recon.py:62-65)
        ksp_u = torch.fft.ifftshift(to_device(ksp, torch.complex64), dim=AX3).contiguous()
        mps_u = torch.fft.ifftshift(to_device(mps, torch.complex64), dim=AX3).contiguous()
        planes_u = np.fft.ifftshift(planes, axes=(-2, -1))
        dev = ksp_u.device
        # max_norm = max |IFFT3(ksp)| (joint_recon.py:67-68); the hybrid k-space is reused
        kh = hybrid_kspace(ksp_u)
        self.max_norm = float(max_abs_image(kh).item())
        ksp_u.div_(self.max_norm)
        del kh
        if t0 is None:
            self.t = torch.zeros((self.num_shots, 6), dtype=torch.float64, device=dev)
        else:
            self.t = to_device(t0 if isinstance(t0, torch.Tensor) else np.asarray(t0, np.float64),
                               torch.float64).clone()
        self.grid = DeviceGrid(kgrid, rkgrid, self.img_shape)
        self.pb = self._make_problem(ksp_u, mps_u, planes_u, kgrid, rkgrid, batch, lm_batch)
        del ksp_u, mps_u
        self.x = self.pb.empty_image().zero_()
        self.damp = torch.ones(self.num_shots, dtype=torch.float64, device=dev)
        self.convergence_flags = torch.zeros(self.num_shots, dtype=torch.uint8, device=dev)
        self.P = self.pb.P
        self.M = self.pb.M
        self._lm = LMState(self.pb.nshots, dev)
        self.cg_iterations = []
        self.cg_graph = cg_graph
        self._graph = None
        self._pending = False
        # the next solve's initial residual b - A x, left by _compute_objective, and the state
        # (image, transforms) it belongs to
        self._r0 = None
        self._r0_key = None

    def _make_problem(self, ksp_u, mps_u, planes_u, kgrid, rkgrid, batch, lm_batch):
        """The SENSE problem over the shots this object reconstructs (all of them here)."""
        return SenseProblem(ksp_u, mps_u, planes_u, kgrid, rkgrid, self.t, batch=batch,
                            lm_batch=lm_batch, grid=self.grid)

    def step(self, sync=True):
        """One outer iteration (joint_recon.py:93-100): CG image step, LM motion step(s), x *= M.

        With cg_graph and sync=False nothing waits for the GPU: the CG iteration count is read
        later by collect(), so that several reconstructions can be enqueued back to back."""
        pb = self.pb
        ready = self._r0_ready()
        self._r0_key = None
        pb.set_transforms(self.t)
        if self.cg_graph:
            if self._graph is None:
                self._graph = CgGraph(pb, self.x, self.max_cg_iter, self.tol,
                                      fused=self.fused_residual, r=self._residual_buffer())
            self._graph.launch(r_ready=ready)
            if sync:
                self.cg_iterations.append(self._graph.count())
            else:
                self._pending = True
        else:
            self.cg_iterations.append(cg_solve(pb, self.x, self.max_cg_iter, self.tol,
                                               fused=self.fused_residual,
                                               r=self._residual_buffer(), r_ready=ready))
        for _ in range(self.max_nm_iter):
            x = lm_step(pb, self.x, self.t, self.damp, self.convergence_flags, self._lm,
                        jacobian=self.jacobian, use_ga=self.use_ga, ga_mode=self.ga_mode)
            # the image buffer stays the same tensor (a CG graph reads and writes it in place)
            torch.mul(x, self.M, out=self.x)
        pb.set_transforms(self.t)

    def collect(self):
        """Record the CG iteration count of a step(sync=False) (reads it from the device)."""
        if self._pending:
            self.cg_iterations.append(self._graph.count())
            self._pending = False

    def run(self):
        self.transform_history = []
        self.objective_history = []
        for _ in range(self.max_joint_iter):
            self.step()
            self.transform_history.append(self.t.cpu().numpy().copy())
            self.objective_history.append(self._compute_objective())
            _lib.check_waits()
        self.transform_history = np.stack(self.transform_history) if self.transform_history \
            else np.zeros((0, self.num_shots, 6))
        self.objective_history = np.array(self.objective_history)
        return self.image(), self.t

    def image(self):
        x = zxy_to_xyz(self.x) * self.max_norm
        return torch.fft.fftshift(x, dim=AX3)

    def _residual_buffer(self):
        """The buffer of the initial CG residual (None in the reference's order of operations)."""
        if self.fused_residual and self._r0 is None:
            self._r0 = self.pb.empty_image()
        return self._r0

    def _state_key(self):
        """Identifies the image and transforms the next solve starts from: the tensors and their
        in-place versions.  Only step() changes them through the library; any other change
        (from torch, in place or by rebinding) gives another key."""
        return (id(self.x), self.x._version, id(self.t), self.t._version,
                self.pb.transforms.data_ptr(), self.pb.transforms._version)

    def _r0_ready(self):
        return self._r0_key is not None and self._r0_key == self._state_key()

    def _compute_objective(self):
        """sum_s ||M_s (F C T_s x - y)||^2 (joint_recon.py:108-115)."""
        return float(self.objective_tensor().item())

    def objective_tensor(self):
        """The objective as a float64 CUDA scalar, enqueued on the current stream without
        waiting for it.

        With fused_residual the pass that forms the energies also adjoins the sampled residual
        into b - A x at the same image and transforms, the next CG solve's starting residual,
        which that solve then uses instead of forming it again."""
        pb = self.pb
        if not self.fused_residual:
            return pb.residual_norms(self.x, self.t).sum()
        if self._graph is not None and self._graph.r is not self._r0:
            raise RuntimeError("the CG graph does not use the residual buffer")
        pb.set_transforms(self.t)
        e = torch.empty(pb.nshots, dtype=torch.float64, device=pb.device)
        pb.residual(self.x, self._residual_buffer(), energies=e)
        self._r0_key = self._state_key()
        return e.sum()


def to_shape(a):
    return tuple(a.shape)
