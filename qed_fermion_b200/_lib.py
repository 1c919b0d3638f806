"""ctypes binding of ``libqedf.so`` (the C ABI declared in ``include/qedf.h``).

The shared library is built in-tree (``qed_fermion_b200/libqedf.so``) by
``qed_fermion_b200.build.build()``.  Importing this module does not need a
GPU; calling a compute entry point without the library raises immediately,
there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_float, c_int, c_int64, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqedf.so")

QEDF_OK = 0
QEDF_ERR_ARG = 1
QEDF_ERR_CUDA = 2
QEDF_ERR_SIZE = 3
QEDF_ERR_MAXITER = 4
QEDF_ERR_TIMEOUT = 5
QEDF_ERR_NAN = 6

QEDF_PCG_PLAIN_F32 = 0
QEDF_PCG_PLAIN_F64 = 1
QEDF_PCG_MIXED = 2
QEDF_PCG_MIXED_BF16 = 3
QEDF_PCG_MIXED_F16 = 4


class QedfSystem(ctypes.Structure):
    _fields_ = [("Lx", c_int), ("Ltau", c_int), ("nrhs", c_int), ("shared_boson", c_int)]


class QedfPcgOpts(ctypes.Structure):
    _fields_ = [
        ("mode", c_int),
        ("max_iter", c_int),
        ("rtol", c_double),
        ("dtau", c_double),
        ("use_precon", c_int),
        ("ru_interval", c_int),
        ("ru_delta", c_double),
        ("by", c_int),
        ("slab", c_int),
        ("chunk", c_int),
        ("timeout_ms", c_double),
        ("profile", c_void_p),
        ("l2_persist", c_int),
        ("stage", c_int),
        ("x_init", c_int),
    ]


_vp = c_void_p
# name -> (restype, argtypes)
SIGNATURES = {
    "qedf_version": (ctypes.c_char_p, []),
    "qedf_status_string": (ctypes.c_char_p, [c_int]),
}
for _prec in ("c64", "c128"):
    for _op in ("mhm_vec", "mh_vec", "m_vec", "force_f"):
        SIGNATURES[f"qedf_{_op}_{_prec}"] = (
            c_int, [_vp, _vp, _vp, c_int, c_int, c_int, c_double, c_int, c_int, c_int, _vp])
    SIGNATURES[f"qedf_b_vec_per_tau_{_prec}"] = (c_int, [_vp, _vp, _vp, c_int, c_int, c_double, c_int, _vp])
    SIGNATURES[f"qedf_precon_vec_{_prec}"] = (c_int, [_vp, _vp, c_int, c_int, c_int, _vp, _vp, _vp, _vp])
    SIGNATURES[f"qedf_cdot_{_prec}"] = (c_int, [_vp, _vp, c_int64, c_int, _vp, _vp])
    SIGNATURES[f"qedf_bb_pair_fields_{_prec}"] = (
        c_int, [c_int, _vp, _vp, _vp, _vp, _vp, c_int, c_int, c_int, c_int, _vp, _vp, _vp])
    SIGNATURES[f"qedf_bb_kspace_acc_{_prec}"] = (c_int, [_vp, _vp, c_int64, c_int, _vp, _vp])
    SIGNATURES[f"qedf_bb_corr_{_prec}"] = (
        c_int, [c_int, _vp, _vp, _vp, _vp, _vp, c_int, c_int, c_int, c_int, _vp, _vp])
    SIGNATURES[f"qedf_bb_vfield_{_prec}"] = (c_int, [_vp, _vp, _vp, c_int, c_int, c_int, _vp, _vp, _vp])
    SIGNATURES[f"qedf_bb_diag_{_prec}"] = (c_int, [_vp, _vp, _vp, c_int, c_int, c_int, _vp, _vp])
for _r in ("f32", "f64"):
    SIGNATURES[f"qedf_boson_force_{_r}"] = (c_int, [_vp, _vp, c_int, c_int, c_int, c_double, c_double, c_int, _vp])
    SIGNATURES[f"qedf_boson_action_{_r}"] = (
        c_int, [_vp, _vp, _vp, c_int, c_int, c_int, c_double, c_double, c_int, c_double, _vp])
    SIGNATURES[f"qedf_kick_drift_{_r}"] = (
        c_int, [_vp, _vp, _vp, _vp, _vp, c_double, c_double, c_int, c_int, c_int, _vp])
for _r in ("f32", "f64"):
    SIGNATURES[f"qedf_fm_accumulate_{_r}"] = (c_int, [_vp, _vp, _vp, c_int64, c_double, _vp])
    SIGNATURES[f"qedf_fm_spectrum_{_r}"] = (c_int, [_vp, _vp, c_int64, c_double, _vp])
    SIGNATURES[f"qedf_fm_mass_{_r}"] = (
        c_int, [_vp, _vp, c_int, c_int64, _vp, c_double, c_double, c_double, c_double, c_int, _vp])
    SIGNATURES[f"qedf_fm_noise_{_r}"] = (c_int, [_vp, _vp, _vp, _vp, c_int64, c_int, _vp])
    SIGNATURES[f"qedf_fm_scale_{_r}"] = (c_int, [_vp, _vp, c_int64, _vp])
SIGNATURES["qedf_precon_tau_csr"] = (c_int, [c_int, POINTER(c_int), POINTER(c_int), POINTER(c_double),
                                              POINTER(c_int)])
SIGNATURES["qedf_pcg_workspace_bytes"] = (c_int64, [POINTER(QedfSystem), c_int, POINTER(QedfPcgOpts)])
SIGNATURES["qedf_pcg_solve"] = (c_int, [POINTER(QedfSystem), c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, c_int64,
                                        POINTER(QedfPcgOpts), _vp])
SIGNATURES["qedf_pcg_solve_static"] = (c_int, [POINTER(QedfSystem), c_int, _vp, _vp, _vp, _vp, _vp, _vp,
                                               POINTER(QedfPcgOpts), _vp])
# bytes of the library's own device scratch used by qedf_pcg_solve_static
PCG_STATIC_SCRATCH_BYTES = 64 << 20

_LIB = None
# kernel launches issued through ``call`` (compute entry points launch one
# kernel each; qedf_pcg_solve launches one persistent kernel)
LAUNCHES = {"count": 0}
_HOST_ONLY = {"qedf_version", "qedf_status_string", "qedf_precon_tau_csr", "qedf_pcg_workspace_bytes"}


class QedfError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, fn, status, msg):
        super().__init__(f"{fn} failed: {msg} (status {status})")
        self.status = status


def load():
    """Load (once) and return the ctypes library; raises if it is missing."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with qed_fermion_b200.build.build() "
                "(there is no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def call(name, *args):
    """Call entry point ``name`` and raise ``QedfError`` on a non-zero status."""
    lib = load()
    st = getattr(lib, name)(*args)
    if name not in _HOST_ONLY:
        # qedf_pcg_solve launches a small preparation kernel, the solver and,
        # unless l2_persist is -1, the kernel that releases the L2 window
        if name.startswith("qedf_pcg_solve"):
            opts = next((a for a in args if isinstance(a, QedfPcgOpts)), None)
            LAUNCHES["count"] += 2 if (opts is not None and opts.l2_persist < 0) else 3
        else:
            LAUNCHES["count"] += 1
    if st != QEDF_OK:
        raise QedfError(name, st, lib.qedf_status_string(st).decode())
    return st


def status_string(st):
    return load().qedf_status_string(int(st)).decode()


def exported_symbols():
    return sorted(SIGNATURES)
