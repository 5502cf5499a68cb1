"""ctypes binding of libedk.so (the C-ABI declared in include/edk.h).

The library is the product: every call here goes to CUDA kernels through the
C-ABI.  Importing this module on a machine without the built library raises;
there is no CPU fallback.  Device buffers are torch tensors (plumbing only: the
library sees raw pointers and the current torch stream).
"""
from __future__ import annotations

import ctypes as C
import weakref
import os
from typing import Optional

import numpy as np

from .model import AIMModel

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libedk.so")

EDK_OK = 0
EDK_ERR_INVALID = 1
EDK_ERR_CUDA = 2
EDK_ERR_NOMEM = 3
EDK_KRYLOV_EXHAUSTED = 4
EDK_ERR_ZERO_START = 5
EDK_ERR_CF_ZERO_DEN = 6
EDK_ERR_TIMEOUT = 7
EDK_ERR_NOT_FINITE = 8
EDK_ERR_UNSUPPORTED = 9
EDK_F64 = 0
EDK_F32 = 1


class EdkError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__(f"edk error {code}: {msg}")
        self.code = code


class _Model(C.Structure):
    _fields_ = [("nc", C.c_int32), ("nb", C.c_int32), ("ec", C.c_void_p), ("eb", C.c_void_p),
                ("vbc", C.c_void_p), ("u", C.c_void_p), ("jj", C.c_void_p),
                ("jhund", C.c_double), ("cutoff_hamilt_param", C.c_double)]


class _ModelSz(C.Structure):
    _fields_ = [("base", _Model), ("pb", C.c_void_p), ("pvbc", C.c_void_p), ("on_fly", C.c_int32)]


class _LanczosOpts(C.Structure):
    _fields_ = [("nitermax", C.c_int32), ("neigen", C.c_int32), ("tolerance", C.c_double),
                ("demax", C.c_double), ("cutoff_min_lanczos_vec", C.c_double), ("dtype", C.c_int32),
                ("check_every", C.c_int32), ("ran_tab", C.c_void_p), ("start_dev", C.c_void_p),
                ("use_target", C.c_int32), ("target", C.c_double), ("residual_tol", C.c_double),
                ("keep_basis", C.c_int32)]


class _LanczosResult(C.Structure):
    _fields_ = [("nkept", C.c_int32), ("niter", C.c_int32), ("status", C.c_int32),
                ("E", C.c_double * 64), ("converged", C.c_int32 * 64),
                ("diag", C.c_void_p), ("subdiag", C.c_void_p), ("vecp", C.c_void_p)]


class _SolveOpts(C.Structure):
    _fields_ = [("dtype", C.c_int32), ("nsectors", C.c_int32), ("sectors", C.c_void_p), ("neigen", C.c_int32),
                ("nitermax", C.c_int32), ("tolerance", C.c_double), ("tolerance_lowprec", C.c_double),
                ("check_every", C.c_int32), ("beta", C.c_double), ("demax0", C.c_double),
                ("nitergreen", C.c_int32), ("nw", C.c_int32), ("spin_mask", C.c_int32), ("npairs", C.c_int32),
                ("pairs", C.c_void_p), ("cutoff_dynamic", C.c_double), ("ran_tab", C.c_void_p),
                ("residual_tol", C.c_double), ("green_mode", C.c_int32), ("gs_in", C.c_char_p),
                ("gs_out", C.c_char_p), ("sector_bound_file", C.c_char_p), ("iwindow", C.c_int32),
                ("recompute_pass2", C.c_int32), ("reference_small_sectors", C.c_int32),
                ("lowprec_min_dim", C.c_int64), ("fp32_sums", C.c_int32), ("batch_gs", C.c_int32)]


class _ChilocSectors(C.Structure):
    _fields_ = [("dim", C.c_int32 * 11), ("E", C.c_void_p * 11), ("C", C.c_void_p * 14)]


class _GsEntry(C.Structure):
    _fields_ = [("kind", C.c_int32), ("norbs", C.c_int32), ("nup", C.c_int32), ("ndn", C.c_int32),
                ("val", C.c_double), ("converged", C.c_int32), ("rank", C.c_int32), ("n", C.c_int64),
                ("offset", C.c_int64)]


class _SolveResult(C.Structure):
    _fields_ = [("e0", C.c_double), ("z", C.c_double), ("e0_lowprec", C.c_double), ("residual", C.c_double),
                ("nstates", C.c_int32), ("lanczos_steps", C.c_int32), ("green_steps", C.c_int32),
                ("G", C.c_void_p), ("docc", C.c_void_p), ("energies", C.c_void_p), ("state_sectors", C.c_void_p)]


class _Chain(C.Structure):
    _fields_ = [("target", C.c_void_p), ("start_dev", C.c_void_p), ("e0", C.c_double), ("iph", C.c_int32),
                ("weight", C.c_double), ("out", C.c_int32)]


class _BatchStats(C.Structure):
    _fields_ = [("steps", C.c_int64), ("chains", C.c_int32), ("kernel_ms", C.c_double), ("block", C.c_int32),
                ("rows", C.c_int32), ("blocks_per_sm", C.c_int32), ("tuned_shapes", C.c_int32)]


class _Param(C.Structure):
    _fields_ = [("kind", C.c_int32), ("i", C.c_int32), ("j", C.c_int32), ("spin", C.c_int32)]


class _GreenSpec(C.Structure):
    _fields_ = [("site", C.c_int32), ("spin", C.c_int32), ("dagger", C.c_int32), ("site2", C.c_int32),
                ("sign2", C.c_int32)]


class _GradStats(C.Structure):
    _fields_ = [("forward_steps", C.c_int64), ("replay_steps", C.c_int64), ("reverse_steps", C.c_int64),
                ("cg_iterations", C.c_int32), ("cg_residual", C.c_double), ("stored_vectors", C.c_int32)]


class _BlockOpts(C.Structure):
    _fields_ = [("block", C.c_int32), ("nitermax", C.c_int32), ("neigen", C.c_int32), ("tolerance", C.c_double),
                ("check_every", C.c_int32), ("ran_tab", C.c_void_p)]


PARAM_EC, PARAM_EB, PARAM_VBC, PARAM_U = 0, 1, 2, 3


def star_params(model: AIMModel, spin: int = 2):
    """The parameters of a star model: every bath level Eb(k,k), every nonzero
    hybridisation Vbc(k,c), the impurity levels Ec(c,c) and the on-site U(c,c);
    spin-symmetric (spin=2) by default.  List of (kind, i, j, spin)."""
    p = [(PARAM_EB, k, k, spin) for k in range(model.nb)]
    p += [(PARAM_VBC, k, c, spin) for k in range(model.nb) for c in range(model.nc)
          if np.any(model.vbc[:, k, c] != 0)]
    p += [(PARAM_EC, c, c, spin) for c in range(model.nc)]
    p += [(PARAM_U, c, c, 0) for c in range(model.nc)]
    return p


def perturb(model: AIMModel, param, h: float) -> AIMModel:
    """A copy of the model with one parameter (kind, i, j, spin) moved by h;
    symmetric pairs (i, j), (j, i) move together, as the derivative operators
    assume."""
    import dataclasses
    kind, i, j, spin = param
    m = dataclasses.replace(model, ec=model.ec.copy(), eb=model.eb.copy(), vbc=model.vbc.copy(), u=model.u.copy())
    spins = (0, 1) if spin == 2 else (spin,)
    if kind == PARAM_U:
        m.u[i, j] += h
        if i != j:
            m.u[j, i] += h
        return m
    arr = {PARAM_EC: m.ec, PARAM_EB: m.eb, PARAM_VBC: m.vbc}[kind]
    for s in spins:
        arr[s, i, j] += h
        if kind != PARAM_VBC and i != j:
            arr[s, j, i] += h
    return m


def _params_arr(params):
    arr = (_Param * len(params))()
    for q, (k, i, j, s) in enumerate(params):
        arr[q] = _Param(int(k), int(i), int(j), int(s))
    return arr


_LIB = None


def lib():
    """Loads libedk.so; raises when it is missing (no fallback)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `python -m ed_solver_b200.build`")
    L = C.CDLL(LIB_PATH)
    P, I32, I64, D = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    sig = {
        "edk_binom": (I64, [C.c_int, C.c_int]),
        "edk_basis": (C.c_int, [C.c_int, C.c_int, P]),
        "edk_rank_table": (C.c_int, [C.c_int, P]),
        "edk_build_table": (C.c_int, [P, C.c_int, C.c_int, P, P, P, P, P, P]),
        "edk_default_ran_tab": (C.c_int, [P]),
        "edk_ctx_create": (C.c_int, [C.c_int, P, P]),
        "edk_ctx_destroy": (C.c_int, [P]),
        "edk_ctx_set_stream": (C.c_int, [P, P]),
        "edk_ctx_last_error": (C.c_char_p, [P]),
        "edk_ctx_launch_count": (I64, [P]),
        "edk_ctx_timing": (C.c_int, [P, C.c_int]),
        "edk_ctx_set_kernel_path": (C.c_int, [P, C.c_int]),
        "edk_ctx_set_graphs": (C.c_int, [P, C.c_int]),
        "edk_ctx_timing_elements": (C.c_int, [P, C.c_int, P]),
        "edk_ctx_transfer_bytes": (C.c_int, [P, P, P]),
        "edk_ctx_clear_cache": (C.c_int, [P]),
        "edk_ctx_trim": (C.c_int, [P]),
        "edk_ctx_set_fp32_sums": (C.c_int, [P, C.c_int, C.c_int64]),
        "edk_h_launch_shapes": (C.c_int, [P, C.c_int, P, C.c_int32]),
        "edk_h_launch_shape_chosen": (C.c_int, [P, C.c_int, C.c_int, P]),
        "edk_ctx_set_workspace_limit": (C.c_int, [P, C.c_int64]),
        "edk_ctx_timing_report": (C.c_int, [P, C.c_int, P, P]),
        "edk_h_create": (C.c_int, [P, P, C.c_int, C.c_int, P]),
        "edk_h_destroy": (C.c_int, [P]),
        "edk_h_dims": (C.c_int, [P, P, P, P]),
        "edk_h_table": (C.c_int, [P, C.c_int, P, P, P, P, P]),
        "edk_hmult": (C.c_int, [P, C.c_int, I64, P, P]),
        "edk_hmult_host": (C.c_int, [P, C.c_int, I64, P, P]),
        "edk_hmult_split": (C.c_int, [P, C.c_int, I64, P, P]),
        "edk_lanczos_e0": (C.c_int, [P, P, P]),
        "edk_lanczos_gs": (C.c_int, [P, P, I32, P, P]),
        "edk_apply_c": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P, P, P]),
        "edk_green_chain": (C.c_int, [P, C.c_int, P, I32, D, C.c_int, I32, P, D, P, P, P, P]),
        "edk_cf_eval": (C.c_int, [P, I32, I32, P, P, P, P, P, P, I32, P, P]),
        "edk_double_occ": (C.c_int, [P, C.c_int, P, C.c_int, P, P]),
        "edk_residual": (C.c_int, [P, P, D, P, P]),
        "edk_convert": (C.c_int, [P, C.c_int, C.c_int, I64, P, P]),
        "edk_solve": (C.c_int, [P, P, P, P]),
        "edk_green_batch": (C.c_int, [P, C.c_int, I32, P, I32, I32, P, D, I32, P, I32, P]),
        "edk_dh_bilinear": (C.c_int, [P, P, P, I32, P, P]),
        "edk_block_lanczos": (C.c_int, [P, P, P, P, P, P]),
        "edk_grad_e0": (C.c_int, [P, P, I32, P, P]),
        "edk_grad_green": (C.c_int, [P, P, D, I32, P, I32, I32, P, P, D, I32, P, D, P, P, P]),
        "edk_gs_write": (C.c_int, [C.c_char_p, I32, P, P]),
        "edk_gs_read": (C.c_int, [C.c_char_p, I32, P, P, I64, P, P]),
        "edk_sector_bounds_read": (C.c_int, [C.c_char_p, P, P]),
        "edk_sector_bounds_write": (C.c_int, [C.c_char_p, P]),
        "edk_full_ed": (C.c_int, [P, P, P]),
        "edk_chiloc": (C.c_int, [P, I32, D, D, D, D, I32, I32, I32, P, I32, P, P, P]),
        "edk_chiloc_set_kernel": (C.c_int, [C.c_int]),
        "edk_h_create_sz": (C.c_int, [P, P, C.c_int, P]),
        "edk_apply_cnambu": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P, P, P, P]),
        "edk_h_sz_info": (C.c_int, [P, P, P]),
        "edk_apply_csz_ab": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P, P, P,
                                       P]),
        "edk_apply_csz": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P, P, P,
                                    P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _LIB = L
    return L


def _ptr(a) -> int:
    """Raw address of a numpy array or torch tensor."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


def model_struct(m: AIMModel):
    arrs = m.arrays()
    s = _Model(m.nc, m.nb, *[a.ctypes.data for a in arrs], float(m.jhund), float(m.cutoff))
    return s, arrs


def model_struct_sz(m):
    """edk_model_sz of a NambuModel (keeps the arrays alive through the second value)."""
    base, arrs = model_struct(m.base)
    pb = np.ascontiguousarray(m.pb, np.float64)
    pv = None if m.pvbc is None else np.ascontiguousarray(m.pvbc, np.float64)
    s = _ModelSz(base, pb.ctypes.data, None if pv is None else pv.ctypes.data, int(bool(m.on_fly)))
    return s, (arrs, pb, pv)


# ---------------------------------------------------------------------------
# host-only helpers (no GPU needed)
# ---------------------------------------------------------------------------

def binom(n: int, k: int) -> int:
    return int(lib().edk_binom(n, k))


def basis(ns: int, npart: int) -> np.ndarray:
    out = np.zeros(max(binom(ns, npart), 1), np.uint64)
    rc = lib().edk_basis(ns, npart, out.ctypes.data)
    if rc:
        raise EdkError(rc, "edk_basis")
    return out[:binom(ns, npart)]


def rank_table(ns: int) -> np.ndarray:
    out = np.zeros(1 << ns, np.int32)
    rc = lib().edk_rank_table(ns, out.ctypes.data)
    if rc:
        raise EdkError(rc, "edk_rank_table")
    return out


def default_ran_tab() -> np.ndarray:
    out = np.zeros(10001)
    rc = lib().edk_default_ran_tab(out.ctypes.data)
    if rc:
        raise EdkError(rc, "edk_default_ran_tab")
    return out


def build_table(m: AIMModel, spin: int, npart: int):
    """tab_HAIM2 on the host: (ptr, tgt, val, diag)."""
    ms, keep = model_struct(m)
    dim = C.c_int64()
    nnz = C.c_int64()
    rc = lib().edk_build_table(C.byref(ms), spin, npart, C.byref(dim), C.byref(nnz), None, None, None, None)
    if rc:
        raise EdkError(rc, "edk_build_table")
    ptr = np.zeros(dim.value + 1, np.int64)
    tgt = np.zeros(max(nnz.value, 1), np.int32)
    val = np.zeros(max(nnz.value, 1), np.float64)
    diag = np.zeros(max(dim.value, 1), np.float64)
    rc = lib().edk_build_table(C.byref(ms), spin, npart, C.byref(dim), C.byref(nnz), ptr.ctypes.data,
                               tgt.ctypes.data, val.ctypes.data, diag.ctypes.data)
    if rc:
        raise EdkError(rc, "edk_build_table")
    return ptr, tgt[:nnz.value], val[:nnz.value], diag[:dim.value]


# ---------------------------------------------------------------------------
# device objects
# ---------------------------------------------------------------------------

class Context:
    """Device, stream and scratch buffers (edk_ctx)."""

    def __init__(self, device: int = 0, stream=None):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("ed_solver_b200 needs a CUDA device")
        torch.cuda.set_device(device)
        torch.cuda.init()
        self.device = device
        if stream is None:
            stream = torch.cuda.current_stream(device)
        self._stream = stream
        h = C.c_void_p()
        rc = lib().edk_ctx_create(device, C.c_void_p(stream.cuda_stream), C.byref(h))
        if rc:
            raise EdkError(rc, "edk_ctx_create")
        self.h = h
        # sector Hamiltonians of this context: destroyed before the context is
        self._live = weakref.WeakSet()

    def check(self, rc, what=""):
        if rc not in (EDK_OK,):
            msg = lib().edk_ctx_last_error(self.h)
            raise EdkError(rc, f"{what}: {msg.decode() if msg else ''}")

    @property
    def launches(self) -> int:
        return int(lib().edk_ctx_launch_count(self.h))

    def set_kernel_path(self, path: int):
        """0: fastest applicable row kernel (default); 1: generic row kernel only."""
        self.check(lib().edk_ctx_set_kernel_path(self.h, int(path)), "edk_ctx_set_kernel_path")

    def set_graphs(self, enable: bool):
        """Replay pairs of fused Lanczos steps as CUDA graphs (default on)."""
        self.check(lib().edk_ctx_set_graphs(self.h, int(bool(enable))), "set_graphs")

    def timing(self, enable: bool):
        self.check(lib().edk_ctx_timing(self.h, int(enable)), "edk_ctx_timing")

    def timing_report(self, which: int):
        """(launches, total device ms, summed elements) of row-kernel class `which`."""
        n, ms, el = C.c_int64(), C.c_double(), C.c_double()
        self.check(lib().edk_ctx_timing_report(self.h, which, C.byref(n), C.byref(ms)), "timing_report")
        self.check(lib().edk_ctx_timing_elements(self.h, which, C.byref(el)), "timing_elements")
        return n.value, ms.value, el.value

    def transfer_bytes(self):
        a, b = C.c_int64(), C.c_int64()
        self.check(lib().edk_ctx_transfer_bytes(self.h, C.byref(a), C.byref(b)), "transfer_bytes")
        return a.value, b.value

    def clear_cache(self):
        self.check(lib().edk_ctx_clear_cache(self.h), "clear_cache")

    def set_workspace_limit(self, nbytes: int):
        """Caps the Krylov workspace; a pass needing more fails with EDK_ERR_NOMEM (0: no cap)."""
        self.check(lib().edk_ctx_set_workspace_limit(self.h, int(nbytes)), "set_workspace_limit")

    def set_fp32_sums(self, enable: bool, min_dim: int = 1 << 20):
        """FP32 vectors of sectors with at least min_dim states: sum the hop terms of H*v in FP32."""
        self.check(lib().edk_ctx_set_fp32_sums(self.h, int(bool(enable)), int(min_dim)), "set_fp32_sums")

    def trim(self):
        """Returns the device memory the Krylov-basis pool keeps in reserve."""
        self.check(lib().edk_ctx_trim(self.h), "trim")

    def close(self):
        if getattr(self, "h", None):
            for ham in list(getattr(self, "_live", ())):
                ham.close()
            lib().edk_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _dtype_code(dtype) -> int:
    import torch
    if dtype in (torch.float64, "f64", EDK_F64):
        return EDK_F64
    if dtype in (torch.float32, "f32", EDK_F32):
        return EDK_F32
    raise ValueError(dtype)


def _torch_dtype(code: int):
    import torch
    return torch.float64 if code == EDK_F64 else torch.float32


class Hamiltonian:
    """One (N_up, N_dn) sector Hamiltonian on the device (new_H / delete_H)."""

    def __init__(self, ctx: Context, model: AIMModel, nup: int, ndn: int):
        self.ctx = ctx
        self.model = model
        self.nup, self.ndn = nup, ndn
        ms, self._keep = model_struct(model)
        h = C.c_void_p()
        ctx.check(lib().edk_h_create(ctx.h, C.byref(ms), nup, ndn, C.byref(h)), "edk_h_create")
        self.h = h
        ctx._live.add(self)
        d, du, dd = C.c_int64(), C.c_int64(), C.c_int64()
        lib().edk_h_dims(h, C.byref(d), C.byref(du), C.byref(dd))
        self.dim, self.dup, self.ddn = d.value, du.value, dd.value

    def close(self):
        # a Hamiltonian is destroyed while its context lives (edk_h_destroy uses the context's stream)
        if getattr(self, "h", None) and getattr(self.ctx, "h", None):
            lib().edk_h_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def table(self, spin: int):
        nnz = C.c_int64()
        lib().edk_h_table(self.h, spin, C.byref(nnz), None, None, None, None)
        d = self.dup if spin == 0 else self.ddn
        ptr = np.zeros(d + 1, np.int64)
        tgt = np.zeros(max(nnz.value, 1), np.int32)
        val = np.zeros(max(nnz.value, 1), np.float64)
        diag = np.zeros(max(d, 1), np.float64)
        lib().edk_h_table(self.h, spin, C.byref(nnz), ptr.ctypes.data, tgt.ctypes.data,
                          val.ctypes.data, diag.ctypes.data)
        return ptr, tgt[:nnz.value], val[:nnz.value], diag[:d]

    def launch_shapes(self, dtype="f64"):
        """Feasible launch shapes of the fast row kernels, in the order
        Context.set_kernel_path(16 + i) selects them: dicts with rows per
        group, table bounds, block variant and kernel kind."""
        desc = np.zeros(5 * 32, np.int32)
        n = lib().edk_h_launch_shapes(self.h, _dtype_code(dtype), desc.ctypes.data, 32)
        if n < 0:
            raise EdkError(EDK_ERR_INVALID, "launch_shapes")
        return [dict(zip(("rows", "kmu", "kmd", "variant", "kind"), map(int, desc[5 * i:5 * i + 5])))
                for i in range(min(n, 32))]

    def launch_shape_chosen(self, dtype="f32", fp32_sums=True):
        """The launch shape the timing chose for this sector shape (a dict as
        in launch_shapes), or None when none has been chosen yet."""
        desc = np.zeros(5, np.int32)
        rc = lib().edk_h_launch_shape_chosen(self.h, _dtype_code(dtype), int(bool(fp32_sums)), desc.ctypes.data)
        if rc < 0:
            raise EdkError(rc, "launch_shape_chosen")
        if rc == 0:
            return None
        return dict(zip(("rows", "kmu", "kmd", "variant", "kind"), map(int, desc)))

    def hmult(self, x, out=None):
        """Hmult__: y = H x for a device tensor x (float64 or float32)."""
        import torch
        code = _dtype_code(x.dtype)
        x = x.contiguous()
        y = torch.empty_like(x) if out is None else out
        self.ctx.check(lib().edk_hmult(self.h, code, self.dim, _ptr(x), _ptr(y)), "edk_hmult")
        return y

    def hmult_split(self, x, out=None):
        """HAIMupdo_multr_split (HAIMupdo.f90:1221-1347): y = H x through two
        transposes, without the -JJ density terms; raises where the reference
        STOPs (|Jhund| > 1e-5)."""
        import torch
        code = _dtype_code(x.dtype)
        x = x.contiguous()
        y = torch.empty_like(x) if out is None else out
        self.ctx.check(lib().edk_hmult_split(self.h, code, self.dim, _ptr(x), _ptr(y)), "edk_hmult_split")
        return y

    def hmult_host(self, x: np.ndarray) -> np.ndarray:
        code = EDK_F64 if x.dtype == np.float64 else EDK_F32
        x = np.ascontiguousarray(x)
        y = np.empty_like(x)
        self.ctx.check(lib().edk_hmult_host(self.h, code, self.dim, x.ctypes.data, y.ctypes.data),
                       "edk_hmult_host")
        return y

    # ---- Lanczos -------------------------------------------------------
    def _opts(self, dtype, nitermax, neigen, tolerance, demax, cutoff, check_every, ran_tab, start,
              target=None, residual_tol=0.0, keep_basis=False):
        self._tab = None if ran_tab is None else np.ascontiguousarray(ran_tab, np.float64)
        return _LanczosOpts(int(nitermax), int(neigen), float(tolerance), float(demax), float(cutoff),
                            _dtype_code(dtype), int(check_every),
                            None if self._tab is None else self._tab.ctypes.data,
                            None if start is None else _ptr(start),
                            0 if target is None else 1, 0.0 if target is None else float(target),
                            float(residual_tol), 1 if keep_basis else 0)

    def lanczos_e0(self, dtype="f64", nitermax=1000, neigen=1, tolerance=1e-12, demax=1e300,
                   cutoff=1e-25, check_every=8, ran_tab=None, start=None, target=None, residual_tol=0.0,
                   keep_basis=False):
        """Pass 1 (Lanczos_fast_diagonalize). Returns a dict.  keep_basis: keep
        the Krylov vectors on the device for a following lanczos_gs(keep_basis=True)."""
        o = self._opts(dtype, nitermax, neigen, tolerance, demax, cutoff, check_every, ran_tab, start, target,
                       residual_tol, keep_basis)
        cap = min(self.dim, nitermax) + 2
        diag = np.zeros(cap)
        sub = np.zeros(cap)
        vecp = np.zeros(cap * max(neigen, 1))
        r = _LanczosResult()
        r.diag, r.subdiag, r.vecp = diag.ctypes.data, sub.ctypes.data, vecp.ctypes.data
        self.ctx.check(lib().edk_lanczos_e0(self.h, C.byref(o), C.byref(r)), "edk_lanczos_e0")
        n, k = r.niter, r.nkept
        return dict(E=np.array(r.E[:k]), niter=n, status=r.status, conv=np.array(r.converged[:k]),
                    diag=diag[:n].copy(), subdiag=sub[:n + 1].copy(),
                    vecp=vecp[:k * n].reshape(k, n).copy())

    def lanczos_gs(self, coef, dtype="f64", ran_tab=None, start=None, cutoff=1e-25, keep_basis=False):
        """Pass 2 (Lanczos_get_GS_sector): normalised eigenvector as a device tensor.
        keep_basis: form it from the vectors a lanczos_e0(keep_basis=True) with
        the same start kept (recomputing the recurrence when there are none)."""
        import torch
        code = _dtype_code(dtype)
        o = self._opts(code, 1, 1, 0.0, 0.0, cutoff, 1, ran_tab, start, keep_basis=keep_basis)
        coef = np.ascontiguousarray(coef, np.float64)
        psi = torch.zeros(self.dim, dtype=_torch_dtype(code), device=f"cuda:{self.ctx.device}")
        self.ctx.check(lib().edk_lanczos_gs(self.h, C.byref(o), len(coef), coef.ctypes.data, _ptr(psi)),
                       "edk_lanczos_gs")
        return psi

    def full_ed(self, vectors=True):
        """ED_diago: every eigenpair (E ascending, V columns) of this sector."""
        E = np.zeros(self.dim)
        V = np.zeros((self.dim, self.dim)) if vectors else None
        self.ctx.check(lib().edk_full_ed(self.h, E.ctypes.data, None if V is None else V.ctypes.data),
                       "edk_full_ed")
        return E, V

    # ---- observables ----------------------------------------------------
    def double_occ(self, psi, site=0):
        d, n = C.c_double(), C.c_double()
        self.ctx.check(lib().edk_double_occ(self.h, _dtype_code(psi.dtype), _ptr(psi), site,
                                            C.byref(d), C.byref(n)), "edk_double_occ")
        return d.value, n.value

    def residual(self, psi, e):
        r, n = C.c_double(), C.c_double()
        self.ctx.check(lib().edk_residual(self.h, _ptr(psi), float(e), C.byref(r), C.byref(n)),
                       "edk_residual")
        return r.value, n.value

    # ---- c / c+ ----------------------------------------------------------
    def apply_c(self, vec, site, spin, dagger, site2=-1, sign2=1):
        """apply_Cupdo on vec (this sector) -> (tensor in target sector, (nup', ndn'))."""
        import torch
        ns = self.model.ns
        d = 1 if dagger else -1
        tnup, tndn = (self.nup + d, self.ndn) if spin == 0 else (self.nup, self.ndn + d)
        if not (0 <= tnup <= ns and 0 <= tndn <= ns):
            raise ValueError("target sector outside the Hilbert space")
        n = binom(ns, tnup) * binom(ns, tndn)
        out = torch.empty(n, dtype=vec.dtype, device=vec.device)
        od = C.c_int64()
        self.ctx.check(lib().edk_apply_c(self.h, _dtype_code(vec.dtype), site, spin, int(bool(dagger)),
                                         site2, sign2, _ptr(vec), _ptr(out), C.byref(od)), "edk_apply_c")
        return out, (tnup, tndn)

    def block_lanczos(self, block=2, neigen=4, nitermax=300, tolerance=1e-12, check_every=4, vectors=True,
                      ran_tab=None):
        """Block_Lanczos_diagonalize: lowest eigenvalues (and FP64 eigenvectors
        as a (neigen, dim) device tensor when vectors) by block Lanczos."""
        import torch
        tab = None if ran_tab is None else np.ascontiguousarray(ran_tab, np.float64)
        o = _BlockOpts(int(block), int(nitermax), int(neigen), float(tolerance), int(check_every),
                       None if tab is None else tab.ctypes.data)
        E = np.zeros(neigen)
        V = torch.zeros((neigen, self.dim), dtype=torch.float64, device=f"cuda:{self.ctx.device}") if vectors else None
        it, conv = C.c_int32(), C.c_int32()
        self.ctx.check(lib().edk_block_lanczos(self.h, C.byref(o), E.ctypes.data, _ptr(V), C.byref(it), C.byref(conv)),
                       "edk_block_lanczos")
        return E, V, it.value, bool(conv.value)

    # ---- parameter gradients -----------------------------------------------
    def dh_bilinear(self, a, b, params):
        """<a| dH/dtheta_q |b> for every parameter (FP64 device vectors)."""
        arr = _params_arr(params)
        out = np.zeros(len(params))
        self.ctx.check(lib().edk_dh_bilinear(self.h, _ptr(a.contiguous()), _ptr(b.contiguous()), len(params),
                                             C.cast(arr, C.c_void_p), out.ctypes.data), "edk_dh_bilinear")
        return out

    def grad_e0(self, psi, params):
        """Hellmann-Feynman dE/dtheta_q of the state psi (FP64 device vector)."""
        arr = _params_arr(params)
        out = np.zeros(len(params))
        self.ctx.check(lib().edk_grad_e0(self.h, _ptr(psi.contiguous()), len(params), C.cast(arr, C.c_void_p),
                                         out.ctypes.data), "edk_grad_e0")
        return out

    def grad_green(self, psi, e0, chains, nitergreen, wn, gbar, params, e0bar=0.0, cg_tol=1e-10):
        """VJP of the Green functions of the eigenstate psi (and of E0).

        chains: list of (site, spin, dagger) or (site, spin, dagger, site2, sign2);
        gbar: complex array (nchain, nw) of dL/dRe G + i dL/dIm G.
        Returns (grad (np,), G (nchain, nw) complex, stats dict)."""
        wn = np.ascontiguousarray(wn, np.float64)
        nch = len(chains)
        spec = (_GreenSpec * max(nch, 1))()
        for c, ch in enumerate(chains):
            site, spin, dag = ch[:3]
            site2, sign2 = (ch[3], ch[4]) if len(ch) > 3 else (-1, 1)
            spec[c] = _GreenSpec(int(site), int(spin), int(bool(dag)), int(site2), int(sign2))
        gb = np.zeros((max(nch, 1), len(wn), 2))
        if nch:
            g = np.asarray(gbar, np.complex128).reshape(nch, len(wn))
            gb[:nch, :, 0] = g.real
            gb[:nch, :, 1] = g.imag
        G = np.zeros((max(nch, 1), len(wn), 2))
        arr = _params_arr(params)
        out = np.zeros(len(params))
        st = _GradStats()
        self.ctx.check(lib().edk_grad_green(self.h, _ptr(psi.contiguous()), float(e0), nch, C.cast(spec, C.c_void_p),
                                            int(nitergreen), len(wn), wn.ctypes.data, gb.ctypes.data, float(e0bar),
                                            len(params), C.cast(arr, C.c_void_p), float(cg_tol), out.ctypes.data,
                                            G.ctypes.data, C.byref(st)), "edk_grad_green")
        stats = {f: getattr(st, f) for f, _ in _GradStats._fields_}
        return out, (G[:nch, :, 0] + 1j * G[:nch, :, 1]), stats

    # ---- dynamic correlation ----------------------------------------------
    def green_chain(self, start, nitergreen, e0, iph, wn, cutoff_dynamic=1e-8):
        """compute_dynamic_cpu on this (target) sector. Returns (G, diag, subdiag, niter)."""
        wn = np.ascontiguousarray(wn, np.float64)
        G = np.zeros(2 * len(wn))
        cap = min(nitergreen, self.dim) + 2
        dg = np.zeros(cap)
        sd = np.zeros(cap)
        nd = C.c_int32()
        self.ctx.check(lib().edk_green_chain(self.h, _dtype_code(start.dtype), _ptr(start), int(nitergreen),
                                             float(e0), int(iph), len(wn), wn.ctypes.data,
                                             float(cutoff_dynamic), G.ctypes.data, dg.ctypes.data,
                                             sd.ctypes.data, C.byref(nd)), "edk_green_chain")
        n = nd.value
        return G[0::2] + 1j * G[1::2], dg[:n].copy(), sd[:n].copy(), n


class HamiltonianSz(Hamiltonian):
    """One Nambu (Sz) sector Hamiltonian on the device (new_HAIMsz, HAIMsz.f90:51-82):
    `npart` Nambu particles in 2*ns orbitals.  H*v, both Lanczos passes, Green
    chains, residuals and block Lanczos work as for an (N_up, N_dn) sector;
    physical energies are eigenvalues + ``energy_shift``."""

    def __init__(self, ctx: Context, model, npart: int):
        self.ctx = ctx
        self.model = model
        self.npart = npart
        self.nup = self.ndn = None
        ms, self._keep = model_struct_sz(model)
        h = C.c_void_p()
        ctx.check(lib().edk_h_create_sz(ctx.h, C.byref(ms), npart, C.byref(h)), "edk_h_create_sz")
        self.h = h
        ctx._live.add(self)
        d, du, dd = C.c_int64(), C.c_int64(), C.c_int64()
        lib().edk_h_dims(h, C.byref(d), C.byref(du), C.byref(dd))
        self.dim, self.dup, self.ddn = d.value, du.value, dd.value
        n, sh = C.c_int32(), C.c_double()
        lib().edk_h_sz_info(h, C.byref(n), C.byref(sh))
        self.energy_shift = sh.value

    def apply_c(self, vec, site, spin, dagger, site2=-1, sign2=1, projected=False):
        """apply_Csz_updo (projected: apply_Csz_N_updo) -> (tensor in the target sector, npart')."""
        import torch
        create = bool(dagger) if spin == 0 else not dagger
        npt = self.npart + (1 if create else -1)
        if not 0 <= npt <= 2 * self.model.ns:
            raise ValueError("target sector outside the Hilbert space")
        out = torch.empty(binom(2 * self.model.ns, npt), dtype=vec.dtype, device=vec.device)
        od, on = C.c_int64(), C.c_int32()
        self.ctx.check(lib().edk_apply_csz(self.h, _dtype_code(vec.dtype), site, spin, int(bool(dagger)),
                                           int(bool(projected)), site2, sign2, _ptr(vec), _ptr(out),
                                           C.byref(od), C.byref(on)), "edk_apply_csz")
        return out, on.value

    def apply_c_ab(self, vec, site, proj, site2, proj2, spin, dagger):
        """symmetric_combineAB's start vector: (A_site + B_site2)|vec>, each the
        c[+] of apply_Csz_updo or, projected, of apply_Csz_N_updo (site2 may equal
        site) -> (tensor in the target sector, npart')."""
        import torch
        create = bool(dagger) if spin == 0 else not dagger
        npt = self.npart + (1 if create else -1)
        if not 0 <= npt <= 2 * self.model.ns:
            raise ValueError("target sector outside the Hilbert space")
        out = torch.empty(binom(2 * self.model.ns, npt), dtype=vec.dtype, device=vec.device)
        od, on = C.c_int64(), C.c_int32()
        self.ctx.check(lib().edk_apply_csz_ab(self.h, _dtype_code(vec.dtype), site, int(bool(proj)), site2,
                                              int(bool(proj2)), spin, int(bool(dagger)), _ptr(vec), _ptr(out),
                                              C.byref(od), C.byref(on)), "edk_apply_csz_ab")
        return out, on.value

    def apply_b(self, vec, orb, dagger, orb2=-1, sign2=1):
        """apply_Csz on Nambu impurity orbitals (orb < nc: up, orb >= nc: hole), optionally
        + sign2 * the same on orb2 -> (tensor in the target sector, npart')."""
        import torch
        npt = self.npart + (1 if dagger else -1)
        if not 0 <= npt <= 2 * self.model.ns:
            raise ValueError("target sector outside the Hilbert space")
        out = torch.empty(binom(2 * self.model.ns, npt), dtype=vec.dtype, device=vec.device)
        od, on = C.c_int64(), C.c_int32()
        self.ctx.check(lib().edk_apply_cnambu(self.h, _dtype_code(vec.dtype), orb, int(bool(dagger)), orb2, sign2,
                                              _ptr(vec), _ptr(out), C.byref(od), C.byref(on)), "edk_apply_cnambu")
        return out, on.value


def cf_eval(ctx: Context, chains, wn, ld=None):
    """Device continued fractions. chains: list of dict(diag, subdiag, e, ph, scale)."""
    wn = np.ascontiguousarray(wn, np.float64)
    nch = len(chains)
    ld = ld or max(len(c["diag"]) for c in chains)
    n = np.array([len(c["diag"]) for c in chains], np.int32)
    diag = np.zeros((nch, ld))
    sub = np.zeros((nch, ld))
    for i, c in enumerate(chains):
        diag[i, :len(c["diag"])] = c["diag"]
        sub[i, :len(c["subdiag"])] = c["subdiag"][:ld]
    e = np.array([c["e"] for c in chains], np.float64)
    ph = np.array([c["ph"] for c in chains], np.float64)
    sc = np.array([c["scale"] for c in chains], np.float64)
    G = np.zeros((nch, len(wn), 2))
    ctx.check(lib().edk_cf_eval(ctx.h, nch, ld, n.ctypes.data, diag.ctypes.data, sub.ctypes.data,
                                e.ctypes.data, ph.ctypes.data, sc.ctypes.data, len(wn), wn.ctypes.data,
                                G.ctypes.data), "edk_cf_eval")
    return G[..., 0] + 1j * G[..., 1]


def green_batch(ctx: Context, chains, nitergreen: int, wn, nout: int, mode: int = 0, dtype="f64",
                cutoff_dynamic=1e-8):
    """Many compute_dynamic chains at once (edk_green_batch).

    chains: list of dict(h=Hamiltonian of the start vector's sector, start=device tensor, e0, iph (1 particle,
    2 hole), weight, out).  Returns (G (nout, nw) complex, stats dict)."""
    wn = np.ascontiguousarray(wn, np.float64)
    arr = (_Chain * max(len(chains), 1))()
    for i, c in enumerate(chains):
        arr[i] = _Chain(c["h"].h, _ptr(c["start"]), float(c["e0"]), int(c["iph"]), float(c.get("weight", 1.0)),
                        int(c.get("out", 0)))
    G = np.zeros((nout, len(wn), 2))
    st = _BatchStats()
    ctx.check(lib().edk_green_batch(ctx.h, _dtype_code(dtype), len(chains), C.cast(arr, C.c_void_p),
                                    int(nitergreen), len(wn), wn.ctypes.data, float(cutoff_dynamic), int(nout),
                                    G.ctypes.data, int(mode), C.byref(st)), "edk_green_batch")
    stats = {f: getattr(st, f) for f, _ in _BatchStats._fields_}
    return G[..., 0] + 1j * G[..., 1], stats


def chiloc(ctx: Context, E, M, w, beta: float, Z: float, gs_e: float, sites: int, nup: int, ndn: int,
           ops=(1, 2), phi_eps: float = 1e-5):
    """chi~_loc on the device for frequency triples w (nf x 3 complex): E[11]
    sector energies (None outside the space), M[14] c+ matrices (target x
    source), the reference's sector and matrix order.  Returns (pDNDN, pUPDN)
    as complex arrays (None for an op not asked for)."""
    w = np.asarray(w, np.complex128).reshape(-1, 3)
    nf = len(w)
    wr = np.ascontiguousarray(np.stack([w.real, w.imag], axis=-1).reshape(nf, 6))
    st = _ChilocSectors()
    keep = []
    for q in range(11):
        e = None if E[q] is None else np.ascontiguousarray(E[q], np.float64)
        st.dim[q] = 0 if e is None else len(e)
        st.E[q] = None if e is None else e.ctypes.data
        keep.append(e)
    for m in range(14):
        x = None if M[m] is None else np.ascontiguousarray(M[m], np.float64)
        st.C[m] = None if x is None else x.ctypes.data
        keep.append(x)
    mask = (1 if 1 in ops else 0) | (2 if 2 in ops else 0)
    pd = np.zeros(2 * max(nf, 1))
    pu = np.zeros(2 * max(nf, 1))
    ctx.check(lib().edk_chiloc(ctx.h, mask, float(beta), float(Z), float(gs_e), float(phi_eps), int(sites),
                               int(nup), int(ndn), C.byref(st), nf, wr.ctypes.data, pd.ctypes.data,
                               pu.ctypes.data), "edk_chiloc")
    f = lambda a: a[0:2 * nf:2] + 1j * a[1:2 * nf:2]
    return (f(pd) if mask & 1 else None), (f(pu) if mask & 2 else None)


def chiloc_set_kernel(plain: bool):
    """edk_chiloc's kernel: False = the split kernel (default), True = the per-element one."""
    lib().edk_chiloc_set_kernel(int(bool(plain)))


def gs_write(path: str, entries):
    """write_raw_eigensectorlist: entries = list of dict(kind (0 updo, 1 sz), norbs, nup, ndn,
    val, converged, rank, vec); consecutive entries of one sector form one eigensector."""
    arr = (_GsEntry * max(len(entries), 1))()
    vecs, off = [], 0
    for i, e in enumerate(entries):
        v = np.ascontiguousarray(e["vec"], np.float64)
        arr[i] = _GsEntry(int(e.get("kind", 0)), int(e["norbs"]), int(e["nup"]), int(e.get("ndn", -1)),
                          float(e["val"]), int(bool(e.get("converged", True))), int(e.get("rank", i + 1)),
                          len(v), off)
        vecs.append(v)
        off += len(v)
    pool = np.concatenate(vecs) if vecs else np.zeros(1)
    rc = lib().edk_gs_write(path.encode(), len(entries), C.cast(arr, C.c_void_p), pool.ctypes.data)
    if rc:
        raise EdkError(rc, f"edk_gs_write({path})")


def gs_read(path: str):
    """read_raw_eigensectorlist: the entries of a GS.raw file as dicts with their vectors."""
    n, tot = C.c_int32(), C.c_int64()
    rc = lib().edk_gs_read(path.encode(), 0, None, C.byref(n), 0, None, C.byref(tot))
    if rc:
        raise EdkError(rc, f"edk_gs_read({path})")
    arr = (_GsEntry * max(n.value, 1))()
    pool = np.zeros(max(tot.value, 1))
    rc = lib().edk_gs_read(path.encode(), n.value, C.cast(arr, C.c_void_p), C.byref(n), tot.value,
                           pool.ctypes.data, C.byref(tot))
    if rc:
        raise EdkError(rc, f"edk_gs_read({path})")
    out = []
    for i in range(n.value):
        e = arr[i]
        out.append(dict(kind=e.kind, norbs=e.norbs, nup=e.nup, ndn=e.ndn, val=e.val, converged=bool(e.converged),
                        rank=e.rank, vec=pool[e.offset:e.offset + e.n].copy()))
    return out


def sector_bounds_read(path: str):
    """ed.sector_bound_file: ((nupmin, nupmax), (ndnmin, ndnmax), (szmin, szmax) or None)."""
    b = np.zeros(6, np.int32)
    has = C.c_int32()
    rc = lib().edk_sector_bounds_read(path.encode(), b.ctypes.data, C.byref(has))
    if rc:
        raise EdkError(rc, f"edk_sector_bounds_read({path})")
    return (int(b[0]), int(b[1])), (int(b[2]), int(b[3])), ((int(b[4]), int(b[5])) if has.value else None)


def sector_bounds_write(path: str, nup, ndn, sz=(1000, -1000)):
    b = np.array([nup[0], nup[1], ndn[0], ndn[1], sz[0], sz[1]], np.int32)
    rc = lib().edk_sector_bounds_write(path.encode(), b.ctypes.data)
    if rc:
        raise EdkError(rc, f"edk_sector_bounds_write({path})")


def solve(ctx: Context, model: AIMModel, sectors, beta: float, nw: int, dtype="f64", neigen=1,
          nitermax=1000, tolerance=1e-12, tolerance_lowprec=1e-6, demax0=5.0, nitergreen=200,
          spins=(0, 1), pairs=None, cutoff_dynamic=1e-8, check_every=8, ran_tab=None, residual_tol=0.0,
          green_mode=0, gs_in=None, gs_out=None, sector_bound_file=None, iwindow=1, recompute_pass2=False,
          reference_small_sectors=False, lowprec_min_dim=0, fp32_sums=False, batch_gs=False):
    """One impurity solve through the C-ABI (edk_solve): host inputs, host outputs.
    recompute_pass2: rerun the Lanczos recurrence in pass 2 (the reference's way)
    instead of forming the eigenvectors from the Krylov vectors pass 1 kept.
    reference_small_sectors: target sectors of at most 40 states take the
    reference's Lehmann sum over the eigenstates kept in the window
    (compute_dynamic_full_ed) instead of an exact continued fraction.
    lowprec_min_dim: in mixed precision, the smallest sector that runs FP32
    vectors (0: 2^20).
    fp32_sums: in mixed precision, sum the hop terms of H*v in FP32 in sectors
    of at least 2^20 states (the recurrence, norms and alpha/beta stay FP64).
    batch_gs: the ground states of the small FP64 sectors in persistent
    launches over a work queue (pass 1 of all of them in one launch, pass 2 in
    a second) instead of sector by sector; True batches sectors of at most
    2^14 states, an integer above 1 is that bound.

    Returns dict(e0, z, residual, nstates, lanczos_steps, green_steps, G (2, npairs, nw) complex,
    docc (nc,), energies, sectors, e0_lowprec).
    """
    if pairs is None:
        pairs = [(i, i) for i in range(model.nc)]
    sec = np.ascontiguousarray(np.array(sectors, np.int32).reshape(-1))
    pr = np.ascontiguousarray(np.array(pairs, np.int32).reshape(-1))
    tab = None if ran_tab is None else np.ascontiguousarray(ran_tab, np.float64)
    mask = sum(1 << s for s in spins)
    o = _SolveOpts(_dtype_code(dtype), len(sec) // 2, sec.ctypes.data, int(neigen), int(nitermax), float(tolerance),
                   float(tolerance_lowprec), int(check_every), float(beta), float(demax0), int(nitergreen),
                   int(nw), int(mask), len(pr) // 2, pr.ctypes.data, float(cutoff_dynamic),
                   None if tab is None else tab.ctypes.data, float(residual_tol), int(green_mode),
                   None if gs_in is None else gs_in.encode(), None if gs_out is None else gs_out.encode(),
                   None if sector_bound_file is None else sector_bound_file.encode(), int(iwindow),
                   1 if recompute_pass2 else 0, 1 if reference_small_sectors else 0, int(lowprec_min_dim),
                   1 if fp32_sums else 0, int(batch_gs))
    G = np.zeros((2, len(pr) // 2, nw, 2))
    docc = np.zeros(model.nc)
    en = np.zeros(64)
    ss = np.zeros(128, np.int32)
    r = _SolveResult()
    r.G, r.docc, r.energies, r.state_sectors = G.ctypes.data, docc.ctypes.data, en.ctypes.data, ss.ctypes.data
    ms, keep = model_struct(model)
    ctx.check(lib().edk_solve(ctx.h, C.byref(ms), C.byref(o), C.byref(r)), "edk_solve")
    n = r.nstates
    return dict(e0=r.e0, z=r.z, residual=r.residual, nstates=n, lanczos_steps=r.lanczos_steps,
                green_steps=r.green_steps, G=G[..., 0] + 1j * G[..., 1], docc=docc,
                energies=en[:min(n, 64)].copy(), sectors=[tuple(ss[2 * k:2 * k + 2]) for k in range(min(n, 64))],
                e0_lowprec=r.e0_lowprec)
