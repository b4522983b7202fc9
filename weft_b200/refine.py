"""Gradient refinement of fitted primitive stacks (host side of include/weftk_refine.h).

``StackSet`` holds per-tile stacks on the GPU (parameter rows float32[16]:
geom[0..6], color0[7..9], color1[10..12], alpha[13]); ``StackLoss`` is the
``torch.autograd.Function`` whose forward is ``weftk_stack_loss`` (per-tile MSE
of the rendered stack) and whose backward is the hand-written
``weftk_stack_loss_backward``.  ``refine`` runs a fixed number of Adam steps on
the parameters, projecting them after every step onto what the bitstream can
carry (src/weft/primitives.py:102-177: colours and alpha in [0, 1], coordinates
in [0, 15], thickness in [0, 4]); ``quantize_params`` snaps them to the wire grid
exactly as the reference's ``_quantize_primitive`` (src/weft/encoder.py:211-237).

This path has no reference counterpart (the reference's refinement is discrete
perturbation); its correctness is pinned by central finite differences and a
float64 PyTorch autograd restatement in the tests.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._lib import PRIM_DTYPE

SOFT_TRIANGLES = 2
LOSS_RESIDUAL = 4
MAX_PRIMS = 32
GEOM_LEN = {0: 0, 1: 4, 2: 5, 3: 7, 4: 6, 5: 0}


def records_to_rows(recs: np.ndarray) -> np.ndarray:
    """60-byte primitive records -> float32[n, 16] parameter rows."""
    rows = np.zeros((len(recs), 16), np.float32)
    rows[:, 0:7] = recs["geom"]
    rows[:, 7:10] = recs["color0"]
    rows[:, 10:13] = recs["color1"]
    rows[:, 13] = recs["alpha"]
    return rows


def rows_to_records(rows: np.ndarray, kinds: np.ndarray) -> np.ndarray:
    recs = np.zeros(len(rows), PRIM_DTYPE)
    recs["kind"] = kinds
    recs["geom"] = rows[:, 0:7]
    recs["color0"] = rows[:, 7:10]
    recs["color1"] = rows[:, 10:13]
    recs["alpha"] = rows[:, 13]
    return recs


class StackSet:
    """Per-tile stacks over tile pixels resident on the GPU."""

    def __init__(self, src: torch.Tensor, px_off: torch.Tensor, sizes: torch.Tensor, prim_off: np.ndarray,
                 kinds, device: int = 0, kinds_mask: int | None = None, sizes_host: np.ndarray | None = None,
                 moments: torch.Tensor | None = None):
        """``kinds``: per-row primitive kinds, a numpy array or a device int32 tensor (kept by reference).
        ``kinds_mask`` (bit k = kind k may occur) is derived from a numpy ``kinds``; pass it with a
        device tensor whose contents change later.  ``sizes_host``: the tile sides on the host, when
        the caller has them (saves reading ``sizes`` back).  ``moments``: the tiles' pixel sums
        (``WeftStackSet.moments``, double[n_tiles * 6]) for the one-thread path of lone constant
        layers, or None."""
        self.device = torch.device("cuda", device)
        self.lib = _lib.lib_for_device(device)
        self.n = int(sizes.numel())
        counts = np.diff(prim_off)
        self.max_prims = int(counts.max()) if counts.size else 0
        if self.max_prims > MAX_PRIMS:
            raise ValueError(f"stacks longer than {MAX_PRIMS} primitives are not supported")
        self.src, self.px_off, self.sizes = src, px_off, sizes
        self.prim_off_np = np.asarray(prim_off, np.int64)
        if isinstance(kinds, torch.Tensor):
            self.t_kind = kinds
            self.kinds_np = None
        else:
            self.kinds_np = np.asarray(kinds, np.int32)
            self.t_kind = torch.from_numpy(self.kinds_np).to(self.device)
            if kinds_mask is None:
                kinds_mask = kinds_mask_of(self.kinds_np)
        self.t_prim_off = torch.from_numpy(self.prim_off_np.astype(np.int32)).to(self.device)
        # work split by tile side (largest first): > 32 px eight warps, 17-32 four, 9-16 two, <= 8 one
        sz = np.asarray(sizes_host) if sizes_host is not None else sizes.cpu().numpy()
        classes = [sz > 32, (sz > 16) & (sz <= 32), (sz > 8) & (sz <= 16), sz <= 8]
        order = np.concatenate([np.nonzero(c)[0] for c in classes]).astype(np.int32)
        self.t_order = torch.from_numpy(order).to(self.device)
        n_big, n_mid, n_s16 = (int(c.sum()) for c in classes[:3])
        self.st = _lib.WeftStackSet(self.n, self.max_prims, _lib.ptr(src), _lib.ptr(px_off), _lib.ptr(sizes),
                                    _lib.ptr(self.t_prim_off), _lib.ptr(self.t_kind), _lib.ptr(self.t_order),
                                    n_big, n_mid, n_s16, int(kinds_mask or 0), _lib.ptr(moments))
        self._moments = moments
        # each tile's share of the pixels, float32(side^2) / float32(total) as IEEE single division
        # (the native per-image pipeline computes the same bits)
        px = (sz.astype(np.int64) ** 2)
        w = px.astype(np.float32) / np.float32(px.sum()) if self.n else px.astype(np.float32)
        self.weights = torch.from_numpy(np.ascontiguousarray(w, np.float32)).to(self.device)

    @classmethod
    def from_fit(cls, fit) -> tuple["StackSet", torch.Tensor]:
        """The selected stacks of a ``BatchedFit`` (tiles stay where the fit put them)."""
        recs = fit.selected_records()
        counts = np.array([len(r) for r in recs], np.int64)
        prim_off = np.concatenate([[0], np.cumsum(counts)])
        flat = np.concatenate(recs) if recs else np.zeros(0, PRIM_DTYPE)
        set_ = cls(fit.t_src, fit.t_px_off, fit.t_size, prim_off, flat["kind"], fit.device.index or 0)
        return set_, torch.from_numpy(records_to_rows(flat)).to(set_.device)

    @classmethod
    def from_stacks(cls, patches, stacks, device: int = 0) -> tuple["StackSet", torch.Tensor]:
        """Tiles (ts, ts, 3) and per-tile primitive lists (objects with kind/geom/color0/color1/alpha)."""
        d = torch.device("cuda", device)
        sizes = np.array([p.shape[0] for p in patches], np.int32)
        px = sizes.astype(np.int64) ** 2
        px_off = np.concatenate([[0], np.cumsum(px)[:-1]]).astype(np.int32)
        src = np.zeros((int(px.sum()), 4), np.float32)
        src[:, :3] = np.concatenate([np.asarray(p, np.float32).reshape(-1, 3) for p in patches])
        from .fit import pack_cands

        recs = [pack_cands(s) for s in stacks]
        counts = np.array([len(r) for r in recs], np.int64)
        flat = np.concatenate(recs) if recs else np.zeros(0, PRIM_DTYPE)
        t_src = torch.from_numpy(src).to(d)
        set_ = cls(t_src, torch.from_numpy(px_off).to(d), torch.from_numpy(sizes).to(d),
                   np.concatenate([[0], np.cumsum(counts)]), flat["kind"], device)
        set_._keep = t_src
        return set_, torch.from_numpy(records_to_rows(flat)).to(d)

    def _stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def loss(self, params: torch.Tensor, soft: bool = False, residual: bool = False) -> torch.Tensor:
        """Per-tile loss; ``residual`` scores the error left after the tile's residual grid."""
        params = params.detach().contiguous()
        out = torch.empty(self.n, dtype=torch.float32, device=self.device)
        _lib.check(self.lib.weftk_stack_loss(ctypes_addr(self.st), _lib.ptr(params), _lib.ptr(out),
                                             loss_flags(soft, residual), self._stream()), "weftk_stack_loss")
        return out

    def loss_backward(self, params: torch.Tensor, grad_loss: torch.Tensor, soft: bool = False,
                      residual: bool = False) -> torch.Tensor:
        params = params.detach().contiguous()
        g = grad_loss.detach().to(torch.float32).contiguous()
        out = torch.zeros_like(params)
        _lib.check(self.lib.weftk_stack_loss_backward(ctypes_addr(self.st), _lib.ptr(params), _lib.ptr(g),
                                                      _lib.ptr(out), 0, loss_flags(soft, residual), self._stream()),
                   "weftk_stack_loss_backward")
        return out

    # --------------------------------------------------------------- parameter space
    def project_(self, params: torch.Tensor) -> None:
        """Clamp rows onto what the wire format can represent (in place; no host sync,
        so it can be captured in a CUDA graph)."""
        with torch.no_grad():
            params[:, 7:14].clamp_(0.0, 1.0)
            params[:, 0:7].clamp_(0.0, 15.0)
            k = self.t_kind
            for kind, col in ((2, 4), (3, 6)):
                params[:, col] = torch.where(k == kind, params[:, col].clamp(0.0, 4.0), params[:, col])

    def quantize(self, params: torch.Tensor) -> torch.Tensor:
        """Snap to the wire grid on the device (``weftk_quantize_rows``; no host sync)."""
        params = params.detach().contiguous()
        out = torch.empty_like(params)
        kinds = self.t_kind.to(torch.int32).contiguous()
        _lib.check(self.lib.weftk_quantize_rows(_lib.ptr(params), _lib.ptr(kinds), int(params.shape[0]),
                                                _lib.ptr(out), self._stream()), "weftk_quantize_rows")
        return out

    def to_stacks(self, params: torch.Tensor) -> list[list]:
        """Parameter rows -> per-tile ``Cand`` lists (host)."""
        from .fit import unpack_cands

        kinds = self.kinds_np if self.kinds_np is not None else self.t_kind.cpu().numpy()
        recs = rows_to_records(params.detach().cpu().numpy(), kinds)
        cands = unpack_cands(recs)
        off = self.prim_off_np
        return [cands[off[t]:off[t + 1]] for t in range(self.n)]


def quantize_rows(params: torch.Tensor, kinds: torch.Tensor) -> torch.Tensor:
    """Parameter rows snapped to the wire grid (the reference's ``_quantize_primitive``,
    src/weft/encoder.py:211-237): coordinates u16 over [0, 15], thickness u16 over [0, 4],
    colours u8, alpha u16, half-to-even rounding as Python's ``round``, in float64.  Plain torch
    on any device; ``StackSet.quantize`` is the device kernel of the same rule."""
    p = params.detach().to(torch.float64).clone()
    k = kinds.to(p.device).to(torch.int64)
    p[:, 7:13] = torch.round(p[:, 7:13].clamp(0, 1) * 255.0) / 255.0
    p[:, 13] = torch.round(p[:, 13].clamp(0, 1) * 65535.0) / 65535.0
    g = torch.round((p[:, 0:7] / 15.0).clamp(0, 1) * 65535.0) / 65535.0 * 15.0
    th = torch.where(k == 2, 4, torch.where(k == 3, 6, -1))
    gt = torch.round((p[:, 0:7] / 4.0).clamp(0, 1) * 65535.0) / 65535.0 * 4.0
    col = torch.arange(7, device=p.device)[None, :]
    g = torch.where(col == th[:, None], gt, g)
    ng = torch.tensor([GEOM_LEN.get(i, 0) for i in range(8)], device=p.device)[k.clamp(0, 7)]
    ng = torch.where(k < 0, 0, ng)
    p[:, 0:7] = torch.where((col < ng[:, None]) & (k[:, None] != 0), g, p[:, 0:7])
    return p.to(torch.float32)


def kinds_mask_of(kinds: np.ndarray) -> int:
    """Bit k set when kind k occurs (kinds outside 0..30 are ignored)."""
    k = np.asarray(kinds).astype(np.int64, copy=False).ravel()
    k = k[(k >= 0) & (k < 31)]
    if k.size == 0:
        return 0
    present = np.nonzero(np.bincount(k, minlength=1))[0]
    return int(np.bitwise_or.reduce(np.left_shift(1, present)))


def loss_flags(soft: bool = False, residual: bool = False) -> int:
    return (SOFT_TRIANGLES if soft else 0) | (LOSS_RESIDUAL if residual else 0)


def ctypes_addr(st) -> int:
    import ctypes

    return ctypes.addressof(st)


class StackLoss(torch.autograd.Function):
    """Per-tile losses of the stacks; backward is the hand-written kernel."""

    @staticmethod
    def forward(ctx, params: torch.Tensor, stack_set: StackSet, soft: bool = False, residual: bool = False):
        ctx.stack_set = stack_set
        ctx.soft = soft
        ctx.residual = residual
        ctx.save_for_backward(params)
        return stack_set.loss(params, soft, residual)

    @staticmethod
    def backward(ctx, grad_loss):
        (params,) = ctx.saved_tensors
        return ctx.stack_set.loss_backward(params, grad_loss, ctx.soft, ctx.residual), None, None, None


def refine(stack_set: StackSet, params: torch.Tensor, steps: int = 200, lr: float = 1e-2, residual: bool = False
           ) -> tuple[torch.Tensor, list[float]]:
    """Adam (FP32 parameters and moments) on the pixel-weighted total loss, projecting
    onto the wire-representable box after every step; returns (params, loss history).
    ``residual`` optimises the error left after the tile's residual grid."""
    p = params.detach().clone().contiguous()
    stack_set.project_(p)
    p.requires_grad_(True)
    opt = torch.optim.Adam([p], lr=lr, fused=True)
    w = stack_set.weights
    hist = []
    for _ in range(int(steps)):
        opt.zero_grad(set_to_none=False)
        loss = (StackLoss.apply(p, stack_set, False, residual) * w).sum()
        loss.backward()
        opt.step()
        stack_set.project_(p.data)
        hist.append(loss.detach())
    return p.detach(), [float(h) for h in torch.stack(hist).cpu()] if hist else []


class FusedRefiner:
    """Adam refinement without autograd or a torch optimizer: one launch per step
    (``weftk_refine_step``: loss, gradient, Adam and projection per tile group), or with
    ``single_launch=False`` a loss+gradient launch followed by an Adam+projection launch.
    Same update rule as ``refine`` (PyTorch's Adam, FP32 moments); capturable in a CUDA
    graph."""

    def __init__(self, stack_set: StackSet, params: torch.Tensor, lr: float = 1e-2, betas=(0.9, 0.999),
                 eps: float = 1e-8, residual: bool = False, single_launch: bool = True):
        self.ss = stack_set
        self.single_launch = single_launch
        self.flags = loss_flags(False, residual)
        self.p = params.detach().clone().contiguous()
        stack_set.project_(self.p)
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.loss = torch.zeros(stack_set.n, dtype=torch.float32, device=self.p.device)
        self.step_ctr = torch.zeros(1, dtype=torch.int32, device=self.p.device)
        self.w = stack_set.weights.contiguous()
        self.lr, self.b1, self.b2, self.eps = float(lr), float(betas[0]), float(betas[1]), float(eps)

    def step(self) -> None:
        lib, ss = self.ss.lib, self.ss
        s = ss._stream()
        if self.single_launch:
            _lib.check(lib.weftk_refine_step(ctypes_addr(ss.st), _lib.ptr(self.p), _lib.ptr(self.m), _lib.ptr(self.v),
                                             _lib.ptr(self.w), _lib.ptr(self.loss), 0, self.lr, self.b1, self.b2,
                                             self.eps, self.flags, s), "weftk_refine_step")
            return
        _lib.check(lib.weftk_stack_loss_backward(ctypes_addr(ss.st), _lib.ptr(self.p), _lib.ptr(self.w),
                                                 _lib.ptr(self.g), _lib.ptr(self.loss), self.flags, s),
                   "weftk_stack_loss_backward")
        _lib.check(lib.weftk_adam_step(_lib.ptr(self.p), _lib.ptr(self.g), _lib.ptr(self.m), _lib.ptr(self.v),
                                       _lib.ptr(ss.t_kind), int(self.p.shape[0]), self.lr, self.b1, self.b2, self.eps,
                                       _lib.ptr(self.step_ctr), s), "weftk_adam_step")

    def run(self, steps: int) -> torch.Tensor:
        """``steps`` steps; with ``single_launch`` all of them in ONE launch
        (``weftk_refine_steps``: each tile group loops over the steps on its own rows)."""
        steps = int(steps)
        if steps <= 0:
            return self.p
        if not self.single_launch:
            for _ in range(steps):
                self.step()
            return self.p
        lib, ss = self.ss.lib, self.ss
        _lib.check(lib.weftk_refine_steps(ctypes_addr(ss.st), steps, _lib.ptr(self.p), _lib.ptr(self.m),
                                          _lib.ptr(self.v), _lib.ptr(self.w), _lib.ptr(self.loss), 0, self.lr,
                                          self.b1, self.b2, self.eps, self.flags, ss._stream()), "weftk_refine_steps")
        return self.p

    def restart(self, params: torch.Tensor) -> None:
        """New starting point, fresh moments (device ops only; capturable)."""
        self.p.copy_(params)
        self.ss.project_(self.p)
        self.m.zero_()
        self.v.zero_()
        self.step_ctr.zero_()


class RefinedFit:
    """The refined batched fit as one CUDA graph: init-only candidate scoring over the
    fit's (possibly kind-filtered) pools (with the closed-form init, the tile moments it
    needs first), gather of each tile's selected primitive, ``steps`` fused Adam steps, and
    the refined rows snapped to the wire grid (``q_rows``).  Every launch is device work on
    torch's current stream."""

    def __init__(self, fit, steps: int = 20, lr: float = 1e-2, use_graph: bool = True, residual: bool = False,
                 closed_form_init: bool = True, prelude=None):
        """``prelude`` (optional): a callable that enqueues device work to run first in every run
        (inside the graph), e.g. the generation of the fit's candidate pools."""
        self.fit = fit
        self.prelude = prelude
        fit.use_closed_form_init(closed_form_init)
        dev = fit.device
        has = fit.init_cnt > 0 if fit.init_cnt is not None else np.ones(fit.n, bool)
        self.rows = torch.from_numpy(np.nonzero(has)[0]).to(dev)
        self.rows32 = self.rows.to(torch.int32)
        prim_off = np.concatenate([[0], np.cumsum(has.astype(np.int64))])
        n_rows = int(has.sum())
        self.kinds = torch.zeros(n_rows, dtype=torch.int32, device=dev)
        mask = fit.init_kinds_mask()
        self.ss = StackSet(fit.t_src, fit.t_px_off, fit.t_size, prim_off, self.kinds, dev.index or 0, kinds_mask=mask,
                           sizes_host=fit.sizes, moments=fit.t_moments if fit.st.moments else None)
        self.refiner = FusedRefiner(self.ss, torch.zeros((n_rows, 16), dtype=torch.float32, device=dev), lr=lr,
                                    residual=residual)
        self.steps = int(steps)
        self.q_rows = torch.zeros((n_rows, 16), dtype=torch.float32, device=dev)  # refined rows on the wire grid
        self.pool_off = torch.from_numpy(fit.pool_off).to(dev)
        self.graph = None
        self.use_graph = use_graph

    def _body(self) -> None:
        f = self.fit
        if self.prelude is not None:
            self.prelude()
        f.run_init_only()
        fr = self.refiner
        _lib.check(self.ss.lib.weftk_refine_start(ctypes_addr(f.st), _lib.ptr(self.rows32), int(self.rows32.numel()),
                                                  _lib.ptr(fr.p), _lib.ptr(fr.m), _lib.ptr(fr.v),
                                                  _lib.ptr(self.kinds), self.ss._stream()), "weftk_refine_start")
        fr.run(self.steps)
        _lib.check(self.ss.lib.weftk_quantize_rows(_lib.ptr(fr.p), _lib.ptr(self.kinds), int(self.kinds.numel()),
                                                   _lib.ptr(self.q_rows), self.ss._stream()), "weftk_quantize_rows")

    @property
    def start(self) -> torch.Tensor:
        """The starting rows of the last run (the init round's picks, projected)."""
        f = self.fit
        rows = torch.zeros_like(self.refiner.p)
        m = torch.zeros_like(rows)
        v = torch.zeros_like(rows)
        kinds = torch.zeros_like(self.kinds)
        _lib.check(self.ss.lib.weftk_refine_start(ctypes_addr(f.st), _lib.ptr(self.rows32), int(self.rows32.numel()),
                                                  _lib.ptr(rows), _lib.ptr(m), _lib.ptr(v), _lib.ptr(kinds),
                                                  self.ss._stream()), "weftk_refine_start")
        return rows

    def run(self) -> torch.Tensor:
        if not self.use_graph:
            self._body()
            return self.refiner.p
        if self.graph is None:
            side = torch.cuda.Stream(self.fit.device)
            side.wait_stream(torch.cuda.current_stream(self.fit.device))
            with torch.cuda.stream(side):
                self._body()  # warm-up outside capture (lazy allocations, attributes)
            torch.cuda.current_stream(self.fit.device).wait_stream(side)
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph):
                self._body()
        self.graph.replay()
        return self.refiner.p
