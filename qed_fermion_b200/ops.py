"""Tensor-level wrappers of the C ABI (device tensors in, device tensors out).

Layouts follow the reference's native extension (``qed_fermion._C`` call
sites in ``hmc_sampler_batch.py``): vectors ``[bs, Ltau*Ly*Lx]`` complex,
angles ("boson") ``[nphi, Ltau*Ly*Lx*2]`` real in kernel layout
(``boson.permute([0, 4, 3, 2, 1])`` of ``[bs, 2, Lx, Ly, Ltau]``).
Every call launches on ``torch.cuda.current_stream()`` and can be captured
in a CUDA graph (no host synchronisation, no allocation besides the output
tensors from torch's caching allocator).
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib

_PREC = {torch.complex64: ("c64", torch.float32), torch.complex128: ("c128", torch.float64)}


def stream_handle():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr())


def _check_cuda(*ts):
    for t in ts:
        if not isinstance(t, torch.Tensor) or not t.is_cuda:
            raise RuntimeError("qed_fermion_b200 operators need CUDA tensors (no CPU fallback)")


def raw(t: torch.Tensor) -> torch.Tensor:
    """The tensor whose values are the raw storage of ``t``: a lazily
    conjugated view is read without applying the conjugation (the convention
    the reference's ``_C.b_vec_per_tau`` call sites rely on,
    ``hmc_sampler_batch.py:2183-2189``)."""
    return t.conj() if t.is_conj() else t


def _vec(x, name):
    if x.dtype not in _PREC:
        raise RuntimeError(f"{name}: expected complex64 or complex128, got {x.dtype}")
    x = raw(x)
    if not x.is_contiguous():
        x = x.contiguous()
    return x


def lattice_dims(N: int, Lx: int):
    Vs = Lx * Lx
    if Lx < 2 or Lx % 2 or N % Vs:
        raise RuntimeError(f"vector length {N} is not Ltau * Lx^2 for even Lx={Lx}")
    return Vs, N // Vs


def apply_operator(op: str, boson: torch.Tensor, x: torch.Tensor, Lx: int, dtau: float,
                   rhs_per_boson: int = 1, by: int = 0, slab: int = 0, out=None) -> torch.Tensor:
    """``op`` in {"mhm", "mh", "m"}: M^dag M x, M^dag x or M x for every row of x."""
    _check_cuda(boson, x)
    x = _vec(x, op)
    if x.dim() == 1:
        x = x.view(1, -1)
    bs, N = x.shape[0], x.shape[-1]
    x = x.reshape(bs, N)
    Vs, Ltau = lattice_dims(N, Lx)
    prec, rdt = _PREC[x.dtype]
    if boson.dtype != rdt:
        raise RuntimeError(f"{op}_vec: boson must be {rdt} for {x.dtype} vectors, got {boson.dtype}")
    boson = boson.contiguous()
    if boson.numel() != (bs // rhs_per_boson) * N * 2:
        raise RuntimeError(f"{op}_vec: boson has {boson.numel()} angles, expected "
                           f"{(bs // rhs_per_boson) * N * 2}")
    if out is None:
        out = torch.empty_like(x)
    _lib.call(f"qedf_{op}_vec_{prec}", ptr(boson), ptr(x), ptr(out), bs, Lx, Ltau, float(dtau),
              int(rhs_per_boson), int(by), int(slab), stream_handle())
    return out


def b_vec_per_tau(boson_tau: torch.Tensor, v: torch.Tensor, Lx: int, dtau: float, interm: bool) -> torch.Tensor:
    _check_cuda(boson_tau, v)
    v = _vec(v, "b_vec_per_tau")
    prec, rdt = _PREC[v.dtype]
    Vs = Lx * Lx
    if v.numel() % Vs:
        raise RuntimeError("b_vec_per_tau: vector length is not a multiple of Lx^2")
    nvec = v.numel() // Vs
    boson_tau = boson_tau.contiguous()
    if boson_tau.dtype != rdt or boson_tau.numel() != 2 * Vs:
        raise RuntimeError("b_vec_per_tau: boson_tau must hold 2*Lx^2 angles of the matching real dtype")
    shape = (nvec, 6, Vs) if interm else (nvec, Vs)
    out = torch.empty(shape, dtype=v.dtype, device=v.device)
    _lib.call(f"qedf_b_vec_per_tau_{prec}", ptr(boson_tau), ptr(v), ptr(out), nvec, Lx, float(dtau),
              1 if interm else 0, stream_handle())
    if nvec == 1:
        out = out[0]
    return out


def precon_apply(r: torch.Tensor, tau_csr, Lx: int) -> torch.Tensor:
    """z = (P_tau (x) I) r with ``tau_csr = (row_ptr, col, val)`` device tensors."""
    _check_cuda(r)
    r = _vec(r, "precon_vec")
    if r.dim() == 1:
        r = r.view(1, -1)
    bs, N = r.shape
    Vs, Ltau = lattice_dims(N, Lx)
    prec, _ = _PREC[r.dtype]
    row_ptr, col, val = tau_csr
    if row_ptr.numel() != Ltau + 1:
        raise RuntimeError(f"precon_vec: preconditioner has {row_ptr.numel() - 1} tau rows, vector has {Ltau}")
    out = torch.empty_like(r)
    _lib.call(f"qedf_precon_vec_{prec}", ptr(r), ptr(out), bs, Lx, Ltau, ptr(row_ptr), ptr(col), ptr(val),
              stream_handle())
    return out


def fermion_force(boson: torch.Tensor, xi: torch.Tensor, Lx: int, dtau: float, rhs_per_boson: int = 1,
                  by: int = 0, slab: int = 0) -> torch.Tensor:
    """F = -dS_f/dphi (kernel layout ``[bs, Ltau*Vs*2]``) from xi = (M^dag M)^{-1} psi."""
    _check_cuda(boson, xi)
    xi = _vec(xi, "force_f")
    bs, N = xi.shape
    Vs, Ltau = lattice_dims(N, Lx)
    prec, rdt = _PREC[xi.dtype]
    if boson.dtype != rdt:
        raise RuntimeError("force_f: boson dtype does not match xi")
    boson = boson.contiguous()
    F = torch.empty((bs, N * 2), dtype=rdt, device=xi.device)
    _lib.call(f"qedf_force_f_{prec}", ptr(boson), ptr(xi), ptr(F), bs, Lx, Ltau, float(dtau),
              int(rhs_per_boson), int(by), int(slab), stream_handle())
    return F


def cdot(u: torch.Tensor, v: torch.Tensor, out: torch.Tensor = None) -> torch.Tensor:
    """Re sum conj(u) v per row, accumulated in double precision."""
    _check_cuda(u, v)
    u, v = _vec(u, "cdot"), _vec(v, "cdot")
    rows = u.shape[0] if u.dim() > 1 else 1
    n = u.numel() // rows
    prec, _ = _PREC[u.dtype]
    if out is None:
        out = torch.zeros(rows, dtype=torch.float64, device=u.device)
    else:
        out.zero_()
    _lib.call(f"qedf_cdot_{prec}", ptr(u), ptr(v), n, rows, ptr(out), stream_handle())
    return out


BB_KINDS = {"T1": 1, "T21": 21, "T2": 2, "T4": 4}


def bb_pair_fields(kind: str, eta: torch.Tensor, g_eta: torch.Tensor, ephase: torch.Tensor, ps: torch.Tensor,
                   pt: torch.Tensor, Lx: int, fa: torch.Tensor, fb: torch.Tensor) -> None:
    """Fill ``fa``, ``fb`` ``[npairs, Ltau, Ly, Lx]`` with the two fields of the
    bond-bond correlator ``kind`` ("T1", "T21", "T2", "T4") for the noise pairs
    (ps[p], pt[p]); eta, G_eta ``[Nrv, Ltau*Vs]`` (same complex dtype, conj(eta)
    is taken by the kernel), ephase = e^{i phi_x} ``[Ltau, Ly, Lx]``."""
    _check_cuda(eta, g_eta, ephase, ps, pt, fa, fb)
    prec, _ = _PREC[eta.dtype]
    for t in (g_eta, ephase, fa, fb):
        if t.dtype != eta.dtype or not t.is_contiguous() or t.is_conj():
            raise RuntimeError("bb_pair_fields: complex tensors must share eta's dtype and be contiguous")
    if ps.dtype != torch.int32 or pt.dtype != torch.int32 or not ps.is_contiguous() or not pt.is_contiguous():
        raise RuntimeError("bb_pair_fields: pair indices must be contiguous int32")
    if eta.dim() != 2:
        raise RuntimeError("bb_pair_fields: eta must be [Nrv, Ltau * Lx^2]")
    nrv, N = eta.shape
    Vs, Ltau = lattice_dims(N, Lx)
    npairs = ps.numel()
    if (g_eta.numel() != eta.numel() or fa.numel() < npairs * N or fb.numel() < npairs * N
            or ephase.numel() != N or pt.numel() != npairs):
        raise RuntimeError("bb_pair_fields: buffer sizes do not match")
    _lib.call(f"qedf_bb_pair_fields_{prec}", BB_KINDS[kind], ptr(eta), ptr(g_eta), ptr(ephase), ptr(ps), ptr(pt),
              npairs, nrv, Lx, Ltau, ptr(fa), ptr(fb), stream_handle())


def bb_corr(kind: str, eta: torch.Tensor, g_eta: torch.Tensor, ephase: torch.Tensor, ps: torch.Tensor,
            pt: torch.Tensor, Lx: int, S: torch.Tensor) -> bool:
    """S[k] += the pair sum of correlator ``kind`` over the pairs (ps, pt) and
    all slices in one pass (fields and transforms in shared memory).  Returns
    False without launching when the lattice does not fit the fused kernel
    (the caller then takes ``bb_pair_fields`` + FFTs + ``bb_kspace_acc``)."""
    prec, nrv, N, Vs, Ltau = _bb_inputs("bb_corr", eta, g_eta, ephase, Lx)
    _check_cuda(ps, pt, S)
    if ps.dtype != torch.int32 or pt.dtype != torch.int32 or not ps.is_contiguous() or not pt.is_contiguous():
        raise RuntimeError("bb_corr: pair indices must be contiguous int32")
    if S.dtype != torch.complex128 or S.numel() != Vs or not S.is_contiguous() or pt.numel() != ps.numel():
        raise RuntimeError("bb_corr: S must be a contiguous complex128 buffer of Lx^2 entries")
    st = getattr(_lib.load(), f"qedf_bb_corr_{prec}")(BB_KINDS[kind], ptr(eta), ptr(g_eta), ptr(ephase), ptr(ps), ptr(pt),
                                            ps.numel(), nrv, Lx, Ltau, ptr(S), stream_handle())
    if st == _lib.QEDF_ERR_SIZE:
        return False
    if st != _lib.QEDF_OK:
        raise _lib.QedfError("qedf_bb_corr", st, _lib.status_string(st))
    _lib.LAUNCHES["count"] += 1
    return True


def bb_kspace_acc(A: torch.Tensor, B: torch.Tensor, S: torch.Tensor) -> None:
    """S[k] += sum over rows of A[..., k] B[..., k] (the last two dimensions of
    A, B are the spatial modes), accumulated in double precision into the
    complex128 ``S`` of Vs entries."""
    _check_cuda(A, B, S)
    prec, _ = _PREC[A.dtype]
    if B.dtype != A.dtype or S.dtype != torch.complex128 or not (A.is_contiguous() and B.is_contiguous()
                                                                  and S.is_contiguous()):
        raise RuntimeError("bb_kspace_acc: contiguous A, B of one dtype and a complex128 S are required")
    Vs = S.numel()
    if A.numel() != B.numel() or A.numel() % Vs:
        raise RuntimeError("bb_kspace_acc: sizes do not match")
    _lib.call(f"qedf_bb_kspace_acc_{prec}", ptr(A), ptr(B), A.numel() // Vs, Vs, ptr(S), stream_handle())


def _bb_inputs(name, eta, g_eta, ephase, Lx):
    _check_cuda(eta, g_eta, ephase)
    prec, _ = _PREC[eta.dtype]
    for t in (g_eta, ephase):
        if t.dtype != eta.dtype or not t.is_contiguous() or t.is_conj():
            raise RuntimeError(f"{name}: complex tensors must share eta's dtype and be contiguous")
    if eta.dim() != 2 or not eta.is_contiguous() or eta.is_conj():
        raise RuntimeError(f"{name}: eta must be a contiguous [Nrv, Ltau * Lx^2]")
    nrv, N = eta.shape
    Vs, Ltau = lattice_dims(N, Lx)
    if g_eta.numel() != eta.numel() or ephase.numel() != N:
        raise RuntimeError(f"{name}: buffer sizes do not match")
    return prec, nrv, N, Vs, Ltau


def bb_vfield(eta: torch.Tensor, g_eta: torch.Tensor, ephase: torch.Tensor, Lx: int, v: torch.Tensor,
              Tv: torch.Tensor) -> None:
    """Tvv's current field of every noise vector into ``v`` (eta's shape and
    dtype) and its sum over vectors and slices added to the complex128 ``Tv``
    of Lx^2 entries."""
    prec, nrv, N, Vs, Ltau = _bb_inputs("bb_vfield", eta, g_eta, ephase, Lx)
    _check_cuda(v, Tv)
    if v.dtype != eta.dtype or v.numel() != eta.numel() or not v.is_contiguous():
        raise RuntimeError("bb_vfield: v must be a contiguous buffer like eta")
    if Tv.dtype != torch.complex128 or Tv.numel() != Vs or not Tv.is_contiguous():
        raise RuntimeError("bb_vfield: Tv must be a contiguous complex128 buffer of Lx^2 entries")
    _lib.call(f"qedf_bb_vfield_{prec}", ptr(eta), ptr(g_eta), ptr(ephase), nrv, Lx, Ltau, ptr(v), ptr(Tv),
              stream_handle())


def bb_diag(eta: torch.Tensor, g_eta: torch.Tensor, ephase: torch.Tensor, Lx: int) -> torch.Tensor:
    """The short-distance terms of T1, T21/T2 and T4 summed over vectors,
    slices and sites (complex128 [3]; divide by their count for the means)."""
    prec, nrv, N, Vs, Ltau = _bb_inputs("bb_diag", eta, g_eta, ephase, Lx)
    D = torch.zeros(3, dtype=torch.complex128, device=eta.device)
    _lib.call(f"qedf_bb_diag_{prec}", ptr(eta), ptr(g_eta), ptr(ephase), nrv, Lx, Ltau, ptr(D), stream_handle())
    return D


def _rprec(t):
    if t.dtype == torch.float32:
        return "f32"
    if t.dtype == torch.float64:
        return "f64"
    raise RuntimeError(f"expected float32/float64 angles, got {t.dtype}")


def boson_force(boson: torch.Tensor, Lx: int, K_int: float, ctau: float, compact: bool = False,
                out: torch.Tensor = None) -> torch.Tensor:
    """-d(S_plaq + S_tau)/dphi in kernel layout ``[bs, Ltau*Vs*2]``."""
    _check_cuda(boson)
    bs = boson.shape[0]
    Ltau = boson[0].numel() // (2 * Lx * Lx)
    if out is None:
        out = torch.empty_like(boson)
    _lib.call(f"qedf_boson_force_{_rprec(boson)}", ptr(boson), ptr(out), bs, Lx, Ltau, float(K_int),
              float(ctau), 1 if compact else 0, stream_handle())
    return out


def boson_action(boson: torch.Tensor, Lx: int, K_int: float, ctau: float, compact: bool = False,
                 momenta: torch.Tensor = None, mass: float = 1.0, out: torch.Tensor = None) -> torch.Tensor:
    """S_tau + S_plaq (+ sum p^2 / 2m) per chain, double precision."""
    _check_cuda(boson)
    bs = boson.shape[0]
    Ltau = boson[0].numel() // (2 * Lx * Lx)
    if out is None:
        out = torch.zeros(bs, dtype=torch.float64, device=boson.device)
    else:
        out.zero_()
    _lib.call(f"qedf_boson_action_{_rprec(boson)}", ptr(boson),
              ptr(momenta) if momenta is not None else None, ptr(out), bs, Lx, Ltau, float(K_int), float(ctau),
              1 if compact else 0, float(mass), stream_handle())
    return out


def kick_drift(p: torch.Tensor, F, x, dt: torch.Tensor, mask, kick: float, drift: float, Lx: int):
    """p += kick*dt*F*mask; x += drift*dt*p*mask (in place)."""
    _check_cuda(p, dt)
    bs = p.shape[0]
    Ltau = p[0].numel() // (2 * Lx * Lx)
    _lib.call(f"qedf_kick_drift_{_rprec(p)}", ptr(p), ptr(F) if F is not None else None,
              ptr(x) if x is not None else None, ptr(dt), ptr(mask) if mask is not None else None,
              float(kick), float(drift), bs, Lx, Ltau, stream_handle())
