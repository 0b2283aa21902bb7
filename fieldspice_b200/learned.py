"""Learned coarse-level preconditioner: a BF16 3-D U-Net inside flexible CG.

Where it sits.  The multigrid V-cycle of the CG plan smooths on the fine
levels and, at one coarse level ``level`` (default 3), asks the network for
that level's correction instead of recursing further ("replace" mode):
z = post-smooth(P U(R pre-smooth(r))).  The network costs ~128 kFLOP per
node of its level per right-hand side (17 GFLOP per application at level 3
of a 256x256x128 grid, 8 RHS); on the fine grid the same network would cost
more than the whole multigrid iteration it replaces.  A "hybrid" mode adds a
V-cycle on the residual of the network's guess.  The network is nonlinear
(ReLU), so the outer iteration is flexible CG; if FCG stalls the plan falls
back to plain multigrid PCG, which also checks its answer (same FP64
stopping rule, same charge integration).

Training data.  Residual-to-error pairs generated by the path's own PCG on
seeded geometries of the layered-box family at 128^3: Jacobi-PCG iterates
x_k after k = 4 .. 512 iterations and the converged x*, so e = x* - x_k are
the smooth errors Krylov iterations leave behind.  Each error is injected
into the coarse level (node I of level l is fine node 2^l I; in that level's
equilibrated variables x_l = e(2^l I) / s_l(I), s_l = diag^-1/2), and its
residual b_l = A~_l x_l is computed with the level operator, so every pair
is exact: the network learns b_l -> A~_l^-1 b_l on realistic inputs.

Training runs on the GPU with the library's own kernels (fs_unet_train_step:
tensor-core forward and data gradients, FP32 weight gradients, Adam).
"""

from __future__ import annotations

import ctypes
import math
import time

import numpy as np

from . import _lib as L
from .device import DeviceOperator, EliminatedSystem, device, h2d

__all__ = ["LearnedPreconditioner", "training_pairs", "init_theta", "param_count"]

CIN = (16, 16, 16, 32, 32, 48, 48, 64, 112, 48, 80, 32, 48, 16)
COUT = (16, 16, 32, 32, 48, 48, 64, 64, 48, 48, 32, 32, 16, 16)


def param_count() -> int:
    n = ctypes.c_longlong()
    L.check("fs_unet_param_count", L.load_library().fs_unet_param_count(ctypes.byref(n)))
    return int(n.value)


def init_theta(seed: int = 0) -> np.ndarray:
    """He-normal convolution weights, zero biases, a small random head."""
    lib = L.load_library()
    rng = np.random.default_rng(seed)
    th = np.zeros(param_count(), np.float32)
    ci, co, wo, bo = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong(), ctypes.c_longlong()
    for l in range(15):
        L.check("fs_unet_layer", lib.fs_unet_layer(l, ctypes.byref(ci), ctypes.byref(co),
                                                    ctypes.byref(wo), ctypes.byref(bo)))
        if l < 14:
            th[wo.value:bo.value] = (rng.standard_normal(bo.value - wo.value)
                                     * math.sqrt(2.0 / (27 * ci.value)))
        else:
            th[wo.value:wo.value + 16] = rng.standard_normal(16) * math.sqrt(1.0 / 16)
    return th


def _level_tensors(plan, system, level):
    """Torch views of one multigrid level's dims, FP32 masses, labels and
    diag^-1/2, all living in the plan's workspace."""
    import torch
    lib = L.lib()
    nlev = ctypes.c_int()
    dims = (ctypes.c_int * 48)()
    L.check("fs_pcg_plan_levels", lib.fs_pcg_plan_levels(plan, ctypes.byref(nlev), dims))
    if level >= nlev.value:
        raise ValueError(f"the plan has {nlev.value} levels, level {level} requested")
    d = (dims[3 * level], dims[3 * level + 1], dims[3 * level + 2])
    em = (ctypes.c_void_p * 3)()
    lab = ctypes.c_void_p()
    sc = ctypes.c_void_p()
    L.check("fs_pcg_plan_level_data", lib.fs_pcg_plan_level_data(
        plan, level, em, ctypes.byref(lab), ctypes.byref(sc)))
    ws = system.workspace
    base = ws.data_ptr()
    n = int(np.prod(d))

    def view(ptr, dtype, count):
        off = ptr - base
        nbytes = count * torch.empty(0, dtype=dtype).element_size()
        if off < 0 or off + nbytes > ws.numel():
            raise RuntimeError("level data outside the plan workspace")
        return ws[off:off + nbytes].view(dtype)
    ems = [view(em[a], torch.float32, n) for a in range(3)]
    labels = view(lab.value, torch.uint8, n)
    scale = view(sc.value, torch.float32, n) if sc.value else None
    return d, ems, labels, scale


def training_pairs(workloads, *, level: int = 3, snapshots=(4, 8, 16, 32, 64, 128, 256, 512),
                   tol: float = 1e-10, log=None):
    """(rhs, em, label, target) device tensors of every pair, planar:
    rhs/target [S][N_l] FP32, em [S][3][N_l] FP32, label [S][N_l] uint8."""
    import torch
    lib = L.lib()
    dev = device()
    out = {"rhs": [], "em": [], "label": [], "target": []}
    dims = None
    for wi, w in enumerate(workloads):
        t0 = time.perf_counter()
        grid = w.grid()
        op = DeviceOperator(grid, w.eps_cell)
        N = op.N
        from .boundaries import dirichlet_nodes
        wall = dirichlet_nodes(w.boundary_spec(), grid)[0].astype(np.int64)
        label = torch.zeros(N, dtype=torch.uint8, device=dev)
        if wall.size:
            label[h2d(wall, torch.int64, dev)] = L.LABEL_FIXED
        group = torch.full((N,), -1, dtype=torch.int16, device=dev)
        for c, t in enumerate(w.terminals):
            idx = h2d(np.asarray(t, np.int64), torch.int64, dev)
            label[idx] = L.LABEL_FIXED
            group[idx] = c
        k = len(w.terminals)
        mg = EliminatedSystem(op, label, k, precision="auto", preconditioner="mg")
        jac = EliminatedSystem(op, label, k, precision="mixed", preconditioner="jacobi")
        nx, ny, nz = op.shape

        def excite(sys_):
            L.check("fs_fill_unit_excitation", lib.fs_fill_unit_excitation(
                L.ptr(group), L.ptr(label), L.ptr(sys_.phi), nx, ny, nz, sys_.k, L.stream_ptr()))
        excite(mg)
        mg.solve(tol)
        phi_star = mg.phi.view(N, mg.k)[:, :k].clone()
        d, ems, lab_l, s_l = _level_tensors(mg._plan, mg, level)
        if dims is None:
            dims = d
        elif d != dims:
            raise ValueError("every training geometry must give the same level dims")
        Nl = int(np.prod(d))
        stride = 2 ** level
        fi = torch.arange(d[0], device=dev) * stride
        fj = torch.arange(d[1], device=dev) * stride
        fk = torch.arange(d[2], device=dev) * stride
        fine = ((fi[:, None, None] * ny + fj[None, :, None]) * nz + fk[None, None, :]).reshape(-1)
        inv_s = torch.where(s_l > 0, 1.0 / s_l.double(), torch.zeros_like(s_l, dtype=torch.float64))
        for it in snapshots:
            excite(jac)
            jac.solve(1e-30, maxiter=it)
            e = phi_star - jac.phi.view(N, jac.k)[:, :k]        # (N, k) FP64
            x_l = (e[fine] * inv_s[:, None]).to(torch.float32)  # (Nl, k)
            kk = jac.k
            xin = torch.zeros((Nl, kk), dtype=torch.float32, device=dev)
            xin[:, :k] = x_l
            b = torch.empty_like(xin)
            L.check("fs_eq_apply", lib.fs_eq_apply(
                L.ptr(xin), L.ptr(b), L.ptr(ems[0]), L.ptr(ems[1]), L.ptr(ems[2]),
                L.ptr(lab_l), d[0], d[1], d[2], kk, L.stream_ptr()))
            em3 = torch.stack(ems).unsqueeze(0).expand(k, 3, Nl)
            out["rhs"].append(b[:, :k].t().contiguous())
            out["target"].append(x_l.t().contiguous())
            out["em"].append(em3.contiguous())
            out["label"].append(lab_l.unsqueeze(0).expand(k, Nl).contiguous())
        mg.close()
        jac.close()
        if log is not None:
            log(f"geometry {wi}: {time.perf_counter() - t0:.2f} s")
    data = {key: torch.cat(v, dim=0) for key, v in out.items()}
    data["dims"] = dims
    return data


def dp_batches(S: int, batch: int, epochs: int, seed: int, rank: int = 0, world: int = 1):
    """Training schedule, one ``(epoch, step, indices)`` per step: every epoch
    one permutation of the S pairs (the same on every rank, from ``seed``)
    cut into slices of ``world * batch``; rank r takes part r of each slice.
    Every rank gets the same number of steps (the collectives line up); with
    one rank this is the plain shuffled mini-batch schedule."""
    rng = np.random.default_rng(seed)
    steps = S // (batch * world)
    for ep in range(epochs):
        perm = rng.permutation(S)
        for bi in range(steps):
            base = (bi * world + rank) * batch
            yield ep, bi, perm[base:base + batch]


def dp_world(group=None) -> tuple[int, int]:
    """(rank, world size) of ``group`` (the default group when one is
    initialised), (0, 1) without torch.distributed."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def allreduce_mean(t, group=None, world: int = 1):
    """In place: the mean of ``t`` over the ranks of ``group``."""
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        t /= world
    return t


class LearnedPreconditioner:
    """A trained U-Net and the multigrid level it replaces.

    ``theta``: FP32 parameters (host array or device tensor); ``level``: the
    V-cycle level whose correction the network computes.
    """

    def __init__(self, theta=None, level: int = 3, seed: int = 0, mode: str = "replace"):
        import torch
        dev = device()
        th = init_theta(seed) if theta is None else theta
        self.theta = torch.as_tensor(np.asarray(th, np.float32) if not isinstance(th, torch.Tensor)
                                     else th, dtype=torch.float32, device=dev).contiguous()
        if self.theta.numel() != param_count():
            raise ValueError(f"theta must have {param_count()} entries")
        if mode not in ("hybrid", "replace"):
            raise ValueError("mode must be 'hybrid' (network + V-cycle on its residual) "
                             "or 'replace' (network only)")
        self.level = int(level)
        self.mode = mode
        self.history: list[float] = []
        self.train_time = 0.0

    def zero(self) -> "LearnedPreconditioner":
        """A network whose output is identically 0 (no coarse correction):
        the same V-cycle truncated at ``level`` without the learned part."""
        import torch
        return LearnedPreconditioner(torch.zeros_like(self.theta), self.level, mode=self.mode)

    def with_mode(self, mode: str) -> "LearnedPreconditioner":
        """The same network (shared parameters) used in another mode."""
        other = LearnedPreconditioner(self.theta, self.level, mode=mode)
        other.history = self.history
        return other

    # -- training ------------------------------------------------------------
    def fit(self, data, *, epochs: int = 3, batch: int = 8, lr: float = 1e-3, seed: int = 0,
            log=None, group=None) -> list[float]:
        """Adam on the relative squared error of the network's coarse
        correction against the injected errors; returns the loss history
        (one entry per 50 steps).

        Data parallel over the ranks of ``group`` (the default process group
        when one is initialised; one rank per GPU, each holding the pairs):
        every rank computes the gradient of its own batch
        (``fs_unet_gradient``), one all-reduce averages the gradients and
        every rank applies the same Adam step (``fs_unet_adam_step``), so
        theta stays identical on all ranks.  The network has ~0.7 M
        parameters: one 2.7 MB all-reduce per step."""
        import torch
        lib = L.lib()
        dims = data["dims"]
        S = data["rhs"].shape[0]
        rank, world = dp_world(group)
        if S < batch * world:
            raise ValueError("fewer training pairs than one batch per rank")
        nb = ctypes.c_size_t()
        L.check("fs_unet_workspace_bytes", lib.fs_unet_workspace_bytes(*dims, batch, 1,
                                                                       ctypes.byref(nb)))
        ws = torch.empty(nb.value, dtype=torch.uint8, device=self.theta.device)
        net = ctypes.c_void_p()
        L.check("fs_unet_create", lib.fs_unet_create(*dims, batch, 1, L.ptr(self.theta), L.ptr(ws),
                                                     nb.value, ctypes.byref(net), L.stream_ptr()))
        loss = torch.zeros(1, dtype=torch.float32, device=self.theta.device)
        grad = (torch.empty_like(self.theta) if world > 1 else None)
        total = epochs * (S // (batch * world))
        hist = []
        t0 = time.perf_counter()
        step = 0
        try:
            for _, _, idx_h in dp_batches(S, batch, epochs, seed, rank, world):
                idx = torch.as_tensor(idx_h, device=self.theta.device)
                rhs = data["rhs"].index_select(0, idx).contiguous()
                em = data["em"].index_select(0, idx).contiguous()
                lab = data["label"].index_select(0, idx).contiguous()
                tgt = data["target"].index_select(0, idx).contiguous()
                # cosine learning-rate decay
                lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * step / max(total, 1)))
                if world == 1:
                    L.check("fs_unet_train_step", lib.fs_unet_train_step(
                        net, L.ptr(rhs), L.ptr(em), L.ptr(lab), L.ptr(tgt),
                        ctypes.c_float(lr_t), L.ptr(loss), L.stream_ptr()))
                else:
                    L.check("fs_unet_gradient", lib.fs_unet_gradient(
                        net, L.ptr(rhs), L.ptr(em), L.ptr(lab), L.ptr(tgt), L.ptr(grad),
                        L.ptr(loss), L.stream_ptr()))
                    allreduce_mean(grad, group, world)
                    L.check("fs_unet_adam_step", lib.fs_unet_adam_step(
                        net, L.ptr(grad), ctypes.c_float(lr_t), L.stream_ptr()))
                step += 1
                if step % 50 == 0 or step == total:
                    allreduce_mean(loss, group, world)
                    hist.append(float(loss.item()))
                    if log is not None:
                        log(f"step {step}/{total} loss {hist[-1]:.4f}")
            flag = ctypes.c_int()
            L.check("fs_unet_error", lib.fs_unet_error(net, ctypes.byref(flag), L.stream_ptr()))
            if flag.value:
                raise RuntimeError("a staged load of the network timed out during training")
        finally:
            lib.fs_unet_destroy(net)
        torch.cuda.synchronize()
        self.train_time += time.perf_counter() - t0
        self.history.extend(hist)
        return hist

    @classmethod
    def train(cls, workloads, *, level: int = 3, epochs: int = 3, batch: int = 8,
              lr: float = 1e-3, seed: int = 0, mode: str = "replace",
              log=None) -> "LearnedPreconditioner":
        """Generate the pairs from ``workloads`` and fit a fresh network."""
        t0 = time.perf_counter()
        data = training_pairs(workloads, level=level, log=log)
        gen = time.perf_counter() - t0
        net = cls(level=level, seed=seed, mode=mode)
        net.fit(data, epochs=epochs, batch=batch, lr=lr, seed=seed, log=log)
        net.data_time = gen
        net.pairs = int(data["rhs"].shape[0])
        return net

    # -- use inside a CG plan ------------------------------------------------------
    def attach(self, plan, system) -> int:
        """Install the network in a mixed-precision multigrid plan at
        ``self.level`` (clamped to the plan's coarsest level); returns the
        level used."""
        import torch
        lib = L.lib()
        nlev = ctypes.c_int()
        L.check("fs_pcg_plan_levels", lib.fs_pcg_plan_levels(plan, ctypes.byref(nlev), None))
        level = min(self.level, nlev.value - 1)
        nb = ctypes.c_size_t()
        L.check("fs_pcg_plan_unet_workspace_bytes",
                lib.fs_pcg_plan_unet_workspace_bytes(plan, level, ctypes.byref(nb)))
        system._net_ws = torch.empty(nb.value, dtype=torch.uint8, device=self.theta.device)
        L.check("fs_pcg_plan_set_unet", lib.fs_pcg_plan_set_unet(
            plan, level, 1 if self.mode == "hybrid" else 0, L.ptr(self.theta),
            L.ptr(system._net_ws), nb.value, L.stream_ptr()))
        return level

    def state(self) -> np.ndarray:
        return self.theta.detach().cpu().numpy()
