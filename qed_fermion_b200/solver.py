"""Batched persistent PCG on M^dag M x = b (``qedf_pcg_solve``).

Replaces ``preconditioned_cg_fast_test`` (``hmc_sampler_batch.py:751-846``)
and the estimator's multi-RHS solve (``stochastic_estimator.py:427-433``).
Several systems -- lattices of different L and Ltau, each with any number of
right-hand sides that share one gauge field or carry their own -- are solved
in one cooperative launch with a convergence mask per right-hand side.

Precision modes:
  "fp32"  complex64 vectors, float32 angles, float arithmetic;
  "fp64"  complex128 vectors, float64 angles, double arithmetic;
  "mixed" complex128 b and x, float32 angles, float iterations with double
          reliable updates (x accumulated and the true residual recomputed in
          double), so the solution meets rtol down to ~1e-12;
  "mixed_bf16" the same with the search direction p and the preconditioned
          residual z stored as bf16 pairs, 4 bytes per complex number; r,
          M^dag M p and the float part of x stay float, so the residual
          recurrence matches the x updates; convergence is still decided on
          the double-precision true residual;
  "mixed_f16" as "mixed_bf16" with fp16 pairs, each vector scaled by a power
          of two taken from the residual's norm (fp16's 11-bit significand
          instead of bf16's 8 bits, at the same 4 bytes).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Sequence

import torch

from . import _lib
from .ops import ptr, stream_handle

MODES = {"fp32": _lib.QEDF_PCG_PLAIN_F32, "fp64": _lib.QEDF_PCG_PLAIN_F64, "mixed": _lib.QEDF_PCG_MIXED,
         "mixed_bf16": _lib.QEDF_PCG_MIXED_BF16, "mixed_f16": _lib.QEDF_PCG_MIXED_F16}
VEC_DTYPE = {"fp32": torch.complex64, "fp64": torch.complex128, "mixed": torch.complex128,
             "mixed_bf16": torch.complex128, "mixed_f16": torch.complex128}
ANGLE_DTYPE = {"fp32": torch.float32, "fp64": torch.float64, "mixed": torch.float32, "mixed_bf16": torch.float32,
               "mixed_f16": torch.float32}


@dataclass(frozen=True)
class System:
    """One lattice: ``Lx x Lx x Ltau`` with ``nrhs`` right-hand sides."""

    Lx: int
    Ltau: int
    nrhs: int = 1
    shared_boson: bool = False

    @property
    def n(self) -> int:
        return self.Lx * self.Lx * self.Ltau


@dataclass
class SolveResult:
    x: torch.Tensor          # packed solutions (device)
    iters: torch.Tensor      # [nrhs_total] int32 (device)
    relres: torch.Tensor     # [nrhs_total] float64 (device)
    status: torch.Tensor     # [nrhs_total] int32 (device): 0 ok, 4 max_iter, 5 timeout, 6 nan


class PcgSolver:
    """Plans a batch of systems once and solves it repeatedly.

    The device workspace is one torch allocation made here; ``solve`` itself
    allocates only its outputs (or none, given ``out``) and never synchronises
    the host, so it can be captured in a CUDA graph.

    ``l2_persist`` (default on) gives the solver launch an L2 access-policy
    window over its iteration vectors, fitted to the process's persisting
    set-aside as it is (the limit is never changed), and releases the window's
    lines after the solve.  Pass False for no window.

    ``tune`` takes ``by``, ``slab`` and ``stage`` from the autotuner
    (:mod:`qed_fermion_b200.autotune`), which times the candidates once per
    problem shape and caches the winner; explicit ``by`` / ``slab`` win over it.

    ``stage`` lets the single-precision operator passes stage their input
    slices in shared memory by bulk copies where the stages fit (the results
    are the same bit for bit; measured no faster on the benchmark lattice, so
    off by default and left to the autotuner).
    """

    def __init__(self, systems: Sequence[System], mode: str = "mixed", rtol: float = 1e-10,
                 max_iter: int = 10000, dtau: float = 0.1, use_precon: bool = True,
                 ru_interval: int = 100, ru_delta: float = 0.01, by: int = 0, slab: int = 0,
                 chunk: int = 0, timeout_ms: float = 2000.0, profile: bool = False, device=None,
                 l2_persist: bool = True, stage: bool = False, tune: bool = False):
        if mode not in MODES:
            raise ValueError(f"mode must be one of {sorted(MODES)}")
        self.systems = [s if isinstance(s, System) else System(*s) for s in systems]
        self.mode = mode
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        # launch shape: explicit, or timed once per shape by the autotuner
        self.tuned = None
        if tune and by == 0 and slab == 0 and self.device.type == "cuda":
            from . import autotune
            with torch.cuda.device(self.device):
                self.tuned = autotune.pcg_choice(self.systems, mode, use_precon=use_precon, dtau=dtau)
            by, slab, stage = self.tuned["by"], self.tuned["slab"], self.tuned["stage"]
            chunk = self.tuned.get("chunk", chunk)
        n = len(self.systems)
        self._sys = (_lib.QedfSystem * n)(*[_lib.QedfSystem(s.Lx, s.Ltau, s.nrhs, 1 if s.shared_boson else 0)
                                            for s in self.systems])
        # optional per-phase SM cycle counters of the solver kernel (block 0)
        self.profile = torch.zeros(8, dtype=torch.int64, device=self.device) if profile else None
        self._opts = _lib.QedfPcgOpts(MODES[mode], int(max_iter), float(rtol), float(dtau),
                                      1 if use_precon else 0, int(ru_interval), float(ru_delta), int(by),
                                      int(slab), int(chunk), float(timeout_ms),
                                      self.profile.data_ptr() if profile else None,
                                      0 if l2_persist else -1, 1 if stage else 0)
        # the same options with x holding an initial guess on entry
        self._opts_x0 = _lib.QedfPcgOpts.from_buffer_copy(self._opts)
        self._opts_x0.x_init = 1
        nbytes = _lib.load().qedf_pcg_workspace_bytes(self._sys, n, self._opts)
        if nbytes < 0:
            raise ValueError("invalid system description for the PCG solver")
        self.workspace = torch.empty(int(nbytes), dtype=torch.uint8, device=self.device)
        self.nrhs = sum(s.nrhs for s in self.systems)
        self.vec_len = sum(s.n * s.nrhs for s in self.systems)
        self.angle_len = sum(2 * s.n * (1 if s.shared_boson else s.nrhs) for s in self.systems)
        self.vec_dtype = VEC_DTYPE[mode]
        self.angle_dtype = ANGLE_DTYPE[mode]

    def solve(self, boson: torch.Tensor, b: torch.Tensor, out: SolveResult = None,
              x0: torch.Tensor = None) -> SolveResult:
        """``boson``: packed angles; ``b``: packed right-hand sides (any shape
        with the right number of elements).  ``x0``: an optional initial guess
        like ``b``; the solve then starts from the residual ``b - A x0``,
        computed in the high precision (the reference starts from 0)."""
        if boson.dtype != self.angle_dtype or boson.numel() != self.angle_len:
            raise RuntimeError(f"boson must hold {self.angle_len} {self.angle_dtype} angles")
        if b.dtype != self.vec_dtype or b.numel() != self.vec_len:
            raise RuntimeError(f"b must hold {self.vec_len} {self.vec_dtype} entries")
        if not (boson.is_cuda and b.is_cuda):
            raise RuntimeError("PcgSolver.solve needs CUDA tensors (no CPU fallback)")
        boson = boson.contiguous()
        b = b.resolve_conj().contiguous()
        if out is None:
            out = SolveResult(torch.empty(self.vec_len, dtype=self.vec_dtype, device=b.device),
                              torch.empty(self.nrhs, dtype=torch.int32, device=b.device),
                              torch.empty(self.nrhs, dtype=torch.float64, device=b.device),
                              torch.empty(self.nrhs, dtype=torch.int32, device=b.device))
        opts = self._opts
        if x0 is not None:
            if x0.dtype != self.vec_dtype or x0.numel() != self.vec_len:
                raise RuntimeError(f"x0 must hold {self.vec_len} {self.vec_dtype} entries")
            if x0.data_ptr() != out.x.data_ptr():
                out.x.copy_(x0.reshape(out.x.shape))
            opts = self._opts_x0
        _lib.call("qedf_pcg_solve", self._sys, len(self.systems), ptr(boson), ptr(b), ptr(out.x),
                  ptr(out.iters), ptr(out.relres), ptr(out.status), ptr(self.workspace),
                  self.workspace.numel(), opts, stream_handle())
        return out


    PHASES = ("init", "operator", "wait_after_operator", "elementwise", "wait_after_elementwise",
              "reliable_updates", "bookkeeping", "total")

    def phase_cycles(self) -> dict:
        """Accumulated SM cycles per phase (needs ``profile=True``); syncs the device."""
        if self.profile is None:
            raise RuntimeError("construct the solver with profile=True")
        return dict(zip(self.PHASES, self.profile.cpu().tolist()))


def solve_pcg_batched(systems, boson, b, **kw) -> SolveResult:
    """One-shot convenience wrapper of :class:`PcgSolver`."""
    return PcgSolver(systems, device=b.device, **kw).solve(boson, b)
