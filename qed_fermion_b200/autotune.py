"""Autotuner of the launch shapes of the persistent PCG and the operators.

The reference hard-codes its kernels' thread blocks (``BLOCK_SIZE = (4, 8)``,
``hmc_sampler_batch.py:111``).  Here the choices that matter are timed on the
device once per problem shape and remembered:

* PCG (``qedf_pcg_solve``): the tile height ``by`` of the slice engine (2, 4
  or 6 rows of the 2 x by block each thread owns), the tau-slab length of the
  operator units (the library's load-balance search, or explicit lengths that
  give one, two or three rounds of units per thread block), and the engine
  that stages its input slices in shared memory against the one that loads
  them directly, and 16- or 32-site elementwise units.
* M^dag M (``qedf_mhm_vec_*``): tile height and slab length.

Each candidate runs a fixed-iteration solve of 100 iterations (or an
operator application) on seeded synthetic inputs of the same shape, timed
with CUDA events: the fastest of a few calls after an untimed one, all after
about a second of solves that bring the GPU's clocks up.  The fastest
candidate wins.  Every candidate computes the same
iteration (tests check each against the oracle), so the choice only changes
the time.  Results are kept in memory and in a JSON file (``QEDF_TUNE_CACHE``,
default ``~/.cache/qed_fermion_b200/tune.json``), keyed by the device, the
library version and the problem shape.
"""
from __future__ import annotations

import json
import math
import os
import threading
import time

import torch

from . import _lib

_MEM: dict = {}
_LOCK = threading.Lock()
MAX_THREADS = {2: 576, 4: 512, 6: 384}
SMS = 148


def cache_path() -> str:
    return os.environ.get("QEDF_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "qed_fermion_b200", "tune.json"))


def _load_disk() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store_disk(key: str, value: dict) -> None:
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        data = _load_disk()
        data[key] = value
        tmp = path + f".{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # an unwritable cache only costs a re-tune in the next process


def tile_heights(Ls) -> list:
    """Tile heights valid for every lattice side in ``Ls`` (the library's rule:
    L divisible by the height, one thread per 2 x by tile within the block limit)."""
    return [by for by in (2, 4, 6) if all(L % by == 0 and (L // 2) * (L // by) <= MAX_THREADS[by] for L in Ls)]


def slab_candidates(systems, blocks=SMS) -> list:
    """0 (the library's load-balance search) and the slab lengths that deal the
    operator units in about one, two or three rounds over the thread blocks."""
    work = sum(s.nrhs * s.Ltau for s in systems)
    ntmax = max(s.Ltau for s in systems)
    out = [0]
    for rounds in (1, 2, 3):
        T = max(1, min(ntmax, math.ceil(work / (rounds * blocks))))
        if T not in out:
            out.append(T)
    return out


def _key(kind: str, shape) -> str:
    dev = torch.cuda.get_device_name(torch.cuda.current_device())
    return f"{_lib.load().qedf_version().decode()}|{dev}|{kind}|{json.dumps(shape, sort_keys=True)}"


def _lookup(key):
    with _LOCK:
        if key in _MEM:
            return _MEM[key]
    hit = _load_disk().get(key)
    if hit is not None:
        with _LOCK:
            _MEM[key] = hit
    return hit


def _remember(key, value):
    with _LOCK:
        _MEM[key] = value
    _store_disk(key, value)


def _time(fn, reps):
    """Milliseconds of one call: the fastest of ``reps`` calls timed one by
    one with CUDA events, after one untimed call."""
    fn()
    torch.cuda.synchronize()
    best = None
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    return best


def _warm_gpu(fn, seconds):
    """Run ``fn`` for about ``seconds`` of wall time, so that the candidates
    timed next see the clocks of a busy GPU rather than those of an idle one
    (the first candidate of a cold process otherwise reads up to 10x slow)."""
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        fn()
        torch.cuda.synchronize()


def _synthetic(systems, angle_dtype, vec_dtype, device, seed=20261204):
    """Seeded pi-flux angles with noise and Gaussian right-hand sides, packed as the solver wants them."""
    g = torch.Generator(device=device).manual_seed(seed)
    phis, bs = [], []
    for s in systems:
        n = s.Lx * s.Lx * s.Ltau
        x = torch.arange(s.Lx, device=device).view(1, -1, 1)
        y = torch.arange(s.Lx, device=device).view(-1, 1, 1)
        sg = (1 - 2 * ((x + y) % 2)).to(torch.float64) * (math.pi / 4)
        nb = 1 if s.shared_boson else s.nrhs
        ang = torch.stack([sg.expand(s.Lx, s.Lx, 1), -sg.expand(s.Lx, s.Lx, 1)], dim=-1)  # [y, x, 1, 2]
        ang = ang.permute(2, 0, 1, 3).expand(s.Ltau, s.Lx, s.Lx, 2).reshape(1, -1).repeat(nb, 1)
        ang = ang + 0.05 * torch.randn(ang.shape, device=device, dtype=torch.float64, generator=g)
        phis.append(ang.reshape(-1))
        bs.append(torch.randn(s.nrhs * n, device=device, dtype=torch.complex128, generator=g))
    return torch.cat(phis).to(angle_dtype), torch.cat(bs).to(vec_dtype)


def pcg_choice(systems, mode, use_precon=True, dtau=0.1, iters=100, force=False, warm_seconds=1.0) -> dict:
    """The fastest (by, slab, stage) for this batch of systems and precision
    mode, timed once and then cached.  Returns a dict with the choice, its
    microseconds per iteration and the timings of every candidate."""
    from .solver import PcgSolver
    shape = {"systems": [[s.Lx, s.Ltau, s.nrhs, int(s.shared_boson)] for s in systems], "mode": mode,
             "precon": bool(use_precon), "dtau": dtau}
    key = _key("pcg", shape)
    if not force:
        hit = _lookup(key)
        if hit is not None:
            return hit
    device = torch.device("cuda", torch.cuda.current_device())
    stages = [True, False] if mode in ("mixed", "fp32", "mixed_bf16", "mixed_f16") else [False]
    chunks = [16, 32] if mode != "fp64" and max(s.Ltau for s in systems) <= 500 else [16]
    cands = [(by, T, st, ch) for by in tile_heights([s.Lx for s in systems]) for T in slab_candidates(systems)
             for st in stages for ch in chunks]
    phi = b = None
    timings = []
    for by, T, st, ch in cands:
        try:
            s = PcgSolver(systems, mode=mode, rtol=0.0, max_iter=iters, dtau=dtau, use_precon=use_precon,
                          by=by, slab=T, stage=st, chunk=ch, device=device, tune=False)
        except (ValueError, _lib.QedfError):
            continue
        if phi is None:
            phi, b = _synthetic(systems, s.angle_dtype, s.vec_dtype, device)
            try:
                _warm_gpu(lambda: s.solve(phi, b), warm_seconds)
            except _lib.QedfError:
                phi = None
                continue
        try:
            ms = _time(lambda: s.solve(phi, b), reps=3)
        except _lib.QedfError:
            continue  # a shape this launch cannot take (shared memory, threads)
        timings.append({"by": by, "slab": T, "stage": st, "chunk": ch, "us_per_iter": 1e3 * ms / iters})
        del s
    if not timings:
        # no launch shape takes this batch (e.g. a lattice beyond the slice
        # engine's limit): the library's defaults stand, and its solve reports
        # the limit as it would without tuning
        out = {"by": 0, "slab": 0, "stage": False, "chunk": 0, "us_per_iter": None, "candidates": []}
        _remember(key, out)
        return out
    best = min(timings, key=lambda t: t["us_per_iter"])
    out = {"by": best["by"], "slab": best["slab"], "stage": best["stage"], "chunk": best["chunk"],
           "us_per_iter": best["us_per_iter"], "candidates": timings}
    _remember(key, out)
    return out


def operator_choice(L, Ltau, nvec, dtype, rhs_per_boson=1, force=False) -> dict:
    """The fastest (by, slab) of M^dag M for this shape and dtype (complex64 or complex128)."""
    from . import ops
    cdt = torch.complex64 if dtype in (torch.complex64, torch.float32) else torch.complex128
    rdt = torch.float32 if cdt == torch.complex64 else torch.float64
    shape = {"L": L, "Ltau": Ltau, "nvec": nvec, "dtype": str(cdt), "rpb": rhs_per_boson}
    key = _key("mhm", shape)
    if not force:
        hit = _lookup(key)
        if hit is not None:
            return hit
    device = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=device).manual_seed(7)
    N = L * L * Ltau
    phi = (torch.rand((nvec // rhs_per_boson, 2 * N), device=device, dtype=torch.float64, generator=g) * 6.28 - 3.14)
    phi = phi.to(rdt)
    x = torch.randn((nvec, N), device=device, dtype=torch.complex128, generator=g).to(cdt)
    out = torch.empty_like(x)

    class _S:
        def __init__(self, n, lt):
            self.nrhs, self.Ltau = n, lt

    timings = []
    for by in tile_heights([L]):
        for T in slab_candidates([_S(nvec, Ltau)], blocks=2 * SMS):
            try:
                ms = _time(lambda: ops.apply_operator("mhm", phi, x, L, 0.1, out=out, by=by, slab=T,
                                                      rhs_per_boson=rhs_per_boson), reps=5)
            except _lib.QedfError:
                continue
            timings.append({"by": by, "slab": T, "ms": ms})
    if not timings:
        res = {"by": 0, "slab": 0, "ms": None, "candidates": []}
        _remember(key, res)
        return res
    best = min(timings, key=lambda t: t["ms"])
    res = {"by": best["by"], "slab": best["slab"], "ms": best["ms"], "candidates": timings}
    _remember(key, res)
    return res
