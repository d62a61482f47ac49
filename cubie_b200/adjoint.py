"""Gradients of losses on saved trajectories: discrete adjoint on the GPU.

The reference cannot differentiate its integrations.  Here a ``Solver``
built with ``adjoint=True`` (explicit Runge-Kutta tableaus, and Rosenbrock
tableaus for autonomous systems without drivers) gets two extra kernels (``csrc/device/cbx_adjoint.cuh``):

* the forward launch integrates every run exactly as the persistent kernel
  does, writes the same outputs, and stores the complete per-run loop state
  every ``ckpt_every`` accepted steps (for explicit tableaus also a tape of
  every accepted step's size and flags);
* the backward launch replays each run segment by segment from those
  checkpoints (explicit tableaus: only the step function, driven by the
  tape; Rosenbrock: the whole loop) and back-propagates dL/d(saved state
  rows) through the accepted steps (step sizes held fixed), giving
  dL/d(initial state) and dL/d(parameters) for every run.

:class:`AdjointIntegrator` drives the two launches;
:func:`solve_ivp_adjoint` wraps them in a ``torch.autograd.Function`` so a
torch loss on the returned state tensor back-propagates into the initial
values and parameters.  Memory: ``n_runs * max_ckpts`` checkpoint images,
one replay segment of ``ckpt_every`` records per run and, for explicit
tableaus, ``n_runs * max_ckpts * ckpt_every`` tape entries
(:meth:`AdjointIntegrator.sizes` gives the three sizes in bytes).  A run that
needs more than ``max_ckpts * ckpt_every`` accepted steps stops with
status 32 (step budget), like ``max_steps``.
"""

from __future__ import annotations

from typing import Optional, Tuple

import numpy as np

from . import _native
from .solver import Solver, _torch


class AdjointIntegrator:
    """Forward-with-checkpoints and reverse sweeps for one solver."""

    def __init__(self, solver: Solver, ckpt_every: int = 64, max_ckpts: int = 64):
        if not solver.adjoint:
            raise ValueError("build the Solver with adjoint=True")
        if not solver.output_types or "state" not in solver.output_types:
            raise ValueError("the adjoint differentiates saved state rows: include 'state' in output_types")
        if ckpt_every < 1 or max_ckpts < 1:
            raise ValueError("ckpt_every and max_ckpts must be positive")
        self.solver = solver
        self.ckpt_every = int(ckpt_every)
        self.max_ckpts = int(max_ckpts)

    def sizes(self, prep) -> tuple:
        """(bytes of one checkpoint image, bytes of one replay record, bytes
        of one tape entry or 0 when the configuration keeps no tape)."""
        return prep["module"].adjoint_sizes() + (prep["module"].adjoint_tape_bytes(),)

    def tape_layout(self, tape_entry: int) -> Tuple[int, int]:
        """(entries, 32-bit flag words) of one run's step-size tape."""
        cap = self.max_ckpts * self.ckpt_every
        v = 16 // tape_entry
        return -(-cap // v) * v, -(-cap // 32)

    def _tape_buffers(self, n_runs: int, tape_entry: int, dev):
        torch = _torch()
        entries, words = self.tape_layout(tape_entry)
        return (torch.empty((n_runs * entries * tape_entry // 4,), device=dev, dtype=torch.int32),
                torch.empty((n_runs * words,), device=dev, dtype=torch.int32),
                torch.empty((n_runs,), device=dev, dtype=torch.int32))

    @staticmethod
    def _set_tape(adj, tape) -> None:
        if tape is None:
            adj.tape = adj.tape_flags = adj.step_count = None
        else:
            adj.tape, adj.tape_flags, adj.step_count = (t.data_ptr() for t in tape)

    def forward(self, inits_t, params_t, duration: float, settling_time: float = 0.0, t0: float = 0.0,
                stream=None, tol_scale=None):
        """Integrate with checkpoints.  Returns ``(state, status, saved)``:
        the saved-state tensor ``[rows, n_saved (+time), n_runs]`` on the
        device, the status words and the context :meth:`backward` needs."""
        torch = _torch()
        s = self.solver
        prep = s.prepare(duration, settling_time, t0)
        dev = torch.device("cuda", s.device)
        tdtype = torch.float32 if s.precision == np.float32 else torch.float64
        n_runs = int(inits_t.shape[1])
        inits_t = inits_t.detach().to(device=dev, dtype=tdtype).contiguous()
        params_t = params_t.detach().to(device=dev, dtype=tdtype).contiguous()
        if params_t.numel() == 0:
            params_t = torch.zeros((1, max(n_runs, 1)), device=dev, dtype=tdtype)
        # every clear and the launch go to one stream, ordered after the
        # caller's work on the current stream
        st = stream if stream is not None else torch.cuda.current_stream(dev)
        st.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(st):
            bufs = s.allocate_outputs(prep, n_runs, dev, tdtype)
            tol_t = None if tol_scale is None else torch.as_tensor(tol_scale).to(device=dev, dtype=torch.float64)
            args = s.make_args(prep, bufs, inits_t, params_t, None, n_runs, duration, settling_time, t0,
                               None, tol_t)
        lane, record, tape_entry = self.sizes(prep)
        words = lane // 4
        with torch.cuda.stream(st):
            ckpt = torch.empty((n_runs * self.max_ckpts * words,), device=dev, dtype=torch.int32)
            count = torch.zeros((n_runs,), device=dev, dtype=torch.int32)
            tape = self._tape_buffers(n_runs, tape_entry, dev) if tape_entry > 0 else None
        adj = _native.AdjointArgs()
        adj.ckpt = ckpt.data_ptr()
        adj.ckpt_count = count.data_ptr()
        adj.lane_words = words
        adj.ckpt_every = self.ckpt_every
        adj.max_ckpts = self.max_ckpts
        self._set_tape(adj, tape)
        prep["module"].adjoint_launch(args, adj, 0, s.block_size, 0, st.cuda_stream)
        saved = dict(prep=prep, bufs=bufs, inits=inits_t, params=params_t, tol=tol_t, ckpt=ckpt, count=count,
                     words=words,
                     record=record, tape=tape,
                     n_runs=n_runs, duration=duration, settling_time=settling_time, t0=t0, dev=dev, tdtype=tdtype)
        return bufs["state"], bufs["status"], saved

    def backward(self, saved, grad_state, stream=None) -> Tuple["object", "object"]:
        """dL/d(inits) ``[n_states, n_runs]`` and dL/d(params)
        ``[n_params, n_runs]`` for dL/d(state rows) ``grad_state``."""
        torch = _torch()
        s = self.solver
        prep, bufs = saved["prep"], saved["bufs"]
        dev, tdtype, n_runs = saved["dev"], saved["tdtype"], saved["n_runs"]
        n = s.system.num_states
        npar = s.system.num_parameters
        grad_state = grad_state.detach().to(device=dev, dtype=tdtype).contiguous()
        if tuple(grad_state.shape) != tuple(bufs["state"].shape):
            raise ValueError(f"grad_state shape {tuple(grad_state.shape)} != state {tuple(bufs['state'].shape)}")
        # the work-counter reset and the launch share one stream, ordered
        # after the caller's work (and the forward launch) on the current one
        st = stream if stream is not None else torch.cuda.current_stream(dev)
        st.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(st):
            seg = torch.empty((self.ckpt_every * n_runs * saved["record"] // 4,), device=dev, dtype=torch.int32)
            gi = torch.empty((n, n_runs), device=dev, dtype=tdtype)
            gp = torch.empty((max(npar, 1), n_runs), device=dev, dtype=tdtype)
            args = s.make_args(prep, bufs, saved["inits"], saved["params"], None, n_runs, saved["duration"],
                               saved["settling_time"], saved["t0"], None, saved["tol"])  # zeroes the work counter
        adj = _native.AdjointArgs()
        adj.ckpt = saved["ckpt"].data_ptr()
        adj.ckpt_count = saved["count"].data_ptr()
        adj.seg = seg.data_ptr()
        adj.grad_state = grad_state.data_ptr()
        adj.grad_inits = gi.data_ptr()
        adj.grad_params = gp.data_ptr() if npar > 0 else None
        adj.lane_words = saved["words"]
        adj.ckpt_every = self.ckpt_every
        adj.max_ckpts = self.max_ckpts
        self._set_tape(adj, saved["tape"])
        prep["module"].adjoint_launch(args, adj, 1, s.block_size, 0, st.cuda_stream)
        return gi, (gp if npar > 0 else gp[:0])


def _function():
    torch = _torch()

    class IVPAdjointFunction(torch.autograd.Function):
        """state = integrate(inits, params); backward by the discrete adjoint."""

        @staticmethod
        def forward(ctx, inits, params, integ, duration, settling_time, t0):
            state, status, saved = integ.forward(inits, params, duration, settling_time, t0)
            ctx.integ = integ
            ctx.saved = saved
            ctx.in_dtypes = (inits.dtype, params.dtype)
            ctx.mark_non_differentiable(status)
            return state, status

        @staticmethod
        def backward(ctx, grad_state, grad_status):
            gi, gp = ctx.integ.backward(ctx.saved, grad_state)
            return gi.to(ctx.in_dtypes[0]), gp.to(ctx.in_dtypes[1]), None, None, None, None

    return IVPAdjointFunction


_FN = None


def solve_ivp_adjoint(solver: Solver, inits, params, duration: float, settling_time: float = 0.0,
                      t0: float = 0.0, ckpt_every: int = 64, max_ckpts: int = 64,
                      integrator: Optional[AdjointIntegrator] = None):
    """Differentiable solve: returns ``(state, status)`` where ``state``
    ``[rows, n_saved (+time), n_runs]`` carries gradients back to ``inits``
    ``[n_states, n_runs]`` and ``params`` ``[n_params, n_runs]`` (torch
    tensors on the solver's device)."""
    global _FN
    if _FN is None:
        _FN = _function()
    integ = integrator or AdjointIntegrator(solver, ckpt_every, max_ckpts)
    return _FN.apply(inits, params, integ, float(duration), float(settling_time), float(t0))
