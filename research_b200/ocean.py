"""ctypes binding of libocean.so, mirroring the reference's SpGEMM interface.

Reference surface (paths inside the reference project):
  * ``somespgemm::SpGEMM(const Config&)`` / ``run(A, B)`` / ``get_stats()``
    (kernels/SpGEMM.cuh:209-343) -> :class:`SpGEMM`
  * ``Config`` + ``from_json`` (include/Utils.h:17-108, src/Utils.cpp:8-37)
    -> JSON text passed to ``ocean_create``
  * ``CSR`` / ``cuCSR`` and their H2D/D2H ``convert`` (include/CSR.h, src/CSR.cpp)
    -> :class:`HostCSR` / :class:`DeviceCSR`

The product path is the CUDA library; nothing here computes a product. If the
library is missing the import of :func:`lib` raises, there is no fallback.
"""
from __future__ import annotations

import ctypes
import json
import os
from dataclasses import dataclass
from pathlib import Path
from typing import Any, Optional, Union

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("OCEAN_LIB", str(_PKG / "libocean.so")))

OCEAN_OK = 0
STATUS_NAMES = {0: "OK", 1: "CUDA", 2: "CAPACITY", 3: "TIMEOUT", 4: "INVALID", 5: "OOM", 6: "INTERNAL"}

# Entry points declared in include/ocean.h (checked by the ABI test).
EXPORTS = (
    "ocean_create", "ocean_create_from_file", "ocean_destroy", "ocean_spgemm", "ocean_spgemm_host",
    "ocean_csr_free", "ocean_csr_download", "ocean_csr_download_rows", "ocean_symbolic", "ocean_stats_json", "ocean_stage_ms",
    "ocean_murmur3_u32", "ocean_last_error", "ocean_version", "ocean_symbolic_noalloc", "ocean_row_estimates",
    "ocean_mlp_features", "ocean_mlp_forward", "ocean_mlp_grad", "ocean_mlp_adam", "ocean_mlp_builtin",
    "ocean_estimate", "ocean_estimate_metrics",
    "ocean_batch_create", "ocean_batch_run", "ocean_batch_launch", "ocean_batch_results", "ocean_batch_info_json",
    "ocean_batch_destroy", "ocean_spgemm_batched", "ocean_batch_download", "ocean_batch_download_async",
)

MLP_FEATURES = 16
MLP_PARAMS = 5313
MLP_BLOB = 5346


class OceanError(RuntimeError):
    """A failed library call; ``code`` is the ocean_status value."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"ocean error {STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class CsrView(ctypes.Structure):
    _fields_ = [("rows", ctypes.c_uint64), ("cols", ctypes.c_uint64), ("nnz", ctypes.c_uint64),
                ("rowptr", ctypes.c_void_p), ("rowptr_bits", ctypes.c_int32),
                ("col", ctypes.c_void_p), ("val", ctypes.c_void_p)]


class MlpModel(ctypes.Structure):
    """ocean_mlp_model: device pointers of the parameters and the feature
    normalisation, plus the log2 margin."""
    _fields_ = [("params", ctypes.c_void_p), ("mu", ctypes.c_void_p), ("inv_sd", ctypes.c_void_p),
                ("margin", ctypes.c_float)]


class CsrOut(ctypes.Structure):
    _fields_ = [("rows", ctypes.c_uint64), ("cols", ctypes.c_uint64), ("nnz", ctypes.c_uint64),
                ("rowptr", ctypes.c_void_p), ("rowptr_bits", ctypes.c_int32),
                ("col", ctypes.c_void_p), ("val", ctypes.c_void_p),
                ("location", ctypes.c_int32), ("_owner", ctypes.c_void_p)]


_lib: Optional[ctypes.CDLL] = None


def lib() -> ctypes.CDLL:
    """Loads libocean.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise OceanError(4, f"{LIB_PATH} is missing; run research_b200/build.py (or __graft_entry__.build())")
    L = ctypes.CDLL(str(LIB_PATH))
    vp, u64, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int
    P = ctypes.POINTER
    L.ocean_create.argtypes = [P(vp), ctypes.c_char_p]
    L.ocean_create_from_file.argtypes = [P(vp), ctypes.c_char_p]
    L.ocean_destroy.argtypes = [vp]
    L.ocean_destroy.restype = None
    L.ocean_spgemm.argtypes = [vp, P(CsrView), P(CsrView), P(CsrOut), vp]
    L.ocean_spgemm_host.argtypes = [vp, P(CsrView), P(CsrView), P(CsrOut), vp]
    L.ocean_csr_free.argtypes = [P(CsrOut), vp]
    L.ocean_csr_download.argtypes = [P(CsrOut), vp, vp, vp, vp]
    L.ocean_csr_download_rows.argtypes = [P(CsrOut), u64, u64, vp, vp, vp, vp]
    L.ocean_symbolic.argtypes = [vp, P(CsrView), P(CsrView), vp, vp]
    L.ocean_symbolic_noalloc.argtypes = [P(CsrView), P(CsrView), vp, vp]
    L.ocean_row_estimates.argtypes = [vp, P(CsrView), P(CsrView), ctypes.c_int, vp, vp]
    L.ocean_stats_json.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t, P(ctypes.c_size_t)]
    L.ocean_stage_ms.argtypes = [vp, ctypes.c_char_p]
    L.ocean_stage_ms.restype = ctypes.c_double
    L.ocean_murmur3_u32.argtypes = [vp, vp, u64, ctypes.c_uint32, vp]
    f32 = ctypes.c_float
    L.ocean_mlp_features.argtypes = [vp, P(CsrView), P(CsrView), vp, vp]
    L.ocean_mlp_forward.argtypes = [vp, P(MlpModel), vp, u64, vp, vp]
    L.ocean_mlp_grad.argtypes = [vp, P(MlpModel), vp, vp, u64, f32, vp, vp, vp]
    L.ocean_mlp_adam.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int, f32, f32, f32, f32, vp]
    L.ocean_mlp_builtin.argtypes = [vp, ctypes.c_size_t]
    L.ocean_estimate.argtypes = [vp, P(CsrView), P(CsrView), ctypes.c_int, ctypes.c_int, vp, vp]
    L.ocean_estimate_metrics.argtypes = [vp, vp, vp, ctypes.c_uint32, vp, vp]
    L.ocean_batch_create.argtypes = [vp, u64, P(CsrView), P(CsrView), P(vp), vp]
    L.ocean_batch_run.argtypes = [vp, P(CsrOut), vp]
    L.ocean_batch_launch.argtypes = [vp, vp]
    L.ocean_batch_results.argtypes = [vp, P(CsrOut)]
    L.ocean_batch_info_json.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t, P(ctypes.c_size_t)]
    L.ocean_batch_destroy.argtypes = [vp]
    L.ocean_batch_download.argtypes = [vp, vp, vp, vp, vp]
    L.ocean_batch_download_async.argtypes = [vp, vp, vp, vp, vp]
    L.ocean_spgemm_batched.argtypes = [vp, u64, P(CsrView), P(CsrView), P(CsrOut), vp]
    L.ocean_last_error.restype = ctypes.c_char_p
    L.ocean_version.restype = ctypes.c_char_p
    for name in EXPORTS:
        if name not in ("ocean_destroy", "ocean_stage_ms", "ocean_last_error", "ocean_version"):
            getattr(L, name).restype = i32
    _lib = L
    return L


def _check(rc: int) -> None:
    if rc != OCEAN_OK:
        raise OceanError(rc, lib().ocean_last_error().decode(errors="replace"))


def _ptr(a: Any) -> int:
    if a is None:
        return 0
    if isinstance(a, np.ndarray):
        return a.ctypes.data if a.size else 0
    return int(a.data_ptr()) if a.numel() else 0  # torch tensor


@dataclass
class HostCSR:
    """CSR matrix in host memory (numpy). rowptr has rows+1 entries."""
    rows: int
    cols: int
    rowptr: np.ndarray
    col: np.ndarray
    val: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.col.shape[0])

    @property
    def rowptr_bits(self) -> int:
        return 64 if self.rowptr.dtype == np.uint64 else 32

    def view(self) -> CsrView:
        return CsrView(self.rows, self.cols, self.nnz, _ptr(self.rowptr), self.rowptr_bits,
                       _ptr(self.col), _ptr(self.val))

    def widened(self) -> "HostCSR":
        return HostCSR(self.rows, self.cols, self.rowptr.astype(np.uint64), self.col, self.val)


class DeviceCSR:
    """CSR matrix in device memory. Inputs are held as torch CUDA tensors
    (plumbing only); results of the library are owned by the library."""

    def __init__(self, rows: int, cols: int, nnz: int, rowptr: Any, col: Any, val: Any,
                 rowptr_bits: int, owned: Optional[CsrOut] = None):
        self.rows, self.cols, self.nnz = rows, cols, nnz
        self.rowptr, self.col, self.val = rowptr, col, val
        self.rowptr_bits = rowptr_bits
        self._out = owned

    @staticmethod
    def from_host(m: HostCSR, device: str = "cuda") -> "DeviceCSR":
        import torch
        rp = torch.from_numpy(m.rowptr.view(np.int64 if m.rowptr_bits == 64 else np.int32)).to(device)
        col = torch.from_numpy(m.col.view(np.int32)).to(device)
        val = torch.from_numpy(m.val).to(device)
        return DeviceCSR(m.rows, m.cols, m.nnz, rp, col, val, m.rowptr_bits)

    def view(self) -> CsrView:
        if self._out is not None:
            o = self._out
            return CsrView(o.rows, o.cols, o.nnz, o.rowptr, o.rowptr_bits, o.col, o.val)
        return CsrView(self.rows, self.cols, self.nnz, _ptr(self.rowptr), self.rowptr_bits,
                       _ptr(self.col), _ptr(self.val))

    def download(self) -> HostCSR:
        if self._out is None:
            return HostCSR(self.rows, self.cols,
                           self.rowptr.cpu().numpy().view(np.uint64 if self.rowptr_bits == 64 else np.uint32),
                           self.col.cpu().numpy().view(np.uint32), self.val.cpu().numpy())
        o = self._out
        rp = np.empty(o.rows + 1, dtype=np.uint64 if o.rowptr_bits == 64 else np.uint32)
        col = np.empty(o.nnz, dtype=np.uint32)
        val = np.empty(o.nnz, dtype=np.float64)
        _check(lib().ocean_csr_download(ctypes.byref(o), _ptr(rp), _ptr(col), _ptr(val), None))
        return HostCSR(int(o.rows), int(o.cols), rp, col, val)

    def download_rows(self, r0: int, r1: int):
        """(rowptr u64 absolute, col, val) of rows [r0, r1) of a library result."""
        o = self._out
        edge = np.empty(1, np.uint64)
        _check(lib().ocean_csr_download_rows(ctypes.byref(o), r0, r0, _ptr(edge), 0, 0, None))
        b = int(edge[0])
        _check(lib().ocean_csr_download_rows(ctypes.byref(o), r1, r1, _ptr(edge), 0, 0, None))
        e = int(edge[0])
        rp = np.empty(r1 - r0 + 1, np.uint64)
        col = np.empty(max(e - b, 0), np.uint32)
        val = np.empty(max(e - b, 0), np.float64)
        _check(lib().ocean_csr_download_rows(ctypes.byref(o), r0, r1, _ptr(rp), _ptr(col), _ptr(val), None))
        return rp, col, val

    def free(self, stream: int = 0) -> None:
        if self._out is not None:
            _check(lib().ocean_csr_free(ctypes.byref(self._out), stream or None))
            self._out = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


ConfigLike = Union[None, str, dict, os.PathLike]


def _config_text(config: ConfigLike) -> str:
    if config is None:
        return ""
    if isinstance(config, dict):
        return json.dumps(config)
    if isinstance(config, os.PathLike) or (isinstance(config, str) and config.endswith(".json")
                                           and not config.lstrip().startswith("{")):
        return Path(config).read_text()
    return str(config)


class SpGEMM:
    """C = A·B on the B200. Mirrors ``somespgemm::SpGEMM`` (kernels/SpGEMM.cuh:209-343):
    constructed from a config (dict, JSON text or a path to a JSON file with the
    reference's keys); :meth:`run` returns C and fills :meth:`get_stats`."""

    def __init__(self, config: ConfigLike = None):
        self._h = ctypes.c_void_p()
        self.config_text = _config_text(config)
        self.config = json.loads(self.config_text) if self.config_text.strip() else {}
        _check(lib().ocean_create(ctypes.byref(self._h), self.config_text.encode()))

    def close(self) -> None:
        if self._h:
            lib().ocean_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- the reference's call -------------------------------------------------
    def run(self, A: Union[HostCSR, DeviceCSR], B: Union[HostCSR, DeviceCSR, None] = None,
            stream: int = 0) -> Union[HostCSR, DeviceCSR]:
        """Runs warmup_iters + bench_iters multiplies like the reference's run()
        (kernels/SpGEMM.cuh:226-320) and returns the last C. Host inputs give a
        host result, device inputs a device result."""
        B = A if B is None else B
        warm = int(self.config.get("warmup_iters", 10))
        bench = int(self.config.get("bench_iters", 10))
        result = None
        for _ in range(max(1, warm + bench)):
            if result is not None and isinstance(result, DeviceCSR):
                result.free(stream)
            result = self.multiply(A, B, stream)
        return result

    def multiply(self, A: Union[HostCSR, DeviceCSR], B: Union[HostCSR, DeviceCSR, None] = None,
                 stream: int = 0) -> Union[HostCSR, DeviceCSR]:
        """One multiply. Host inputs: ocean_spgemm_host (copies in and out);
        device inputs: ocean_spgemm (C stays on the device)."""
        B = A if B is None else B
        out = CsrOut()
        if isinstance(A, HostCSR):
            av, bv = A.view(), B.view()
            _check(lib().ocean_spgemm_host(self._h, ctypes.byref(av), ctypes.byref(bv), ctypes.byref(out),
                                           stream or None))
            rp_dtype = np.uint64 if out.rowptr_bits == 64 else np.uint32
            rp = np.ctypeslib.as_array(ctypes.cast(out.rowptr, ctypes.POINTER(
                ctypes.c_uint64 if out.rowptr_bits == 64 else ctypes.c_uint32)), (out.rows + 1,)).copy()
            col = (np.ctypeslib.as_array(ctypes.cast(out.col, ctypes.POINTER(ctypes.c_uint32)), (out.nnz,)).copy()
                   if out.nnz else np.empty(0, np.uint32))
            val = (np.ctypeslib.as_array(ctypes.cast(out.val, ctypes.POINTER(ctypes.c_double)), (out.nnz,)).copy()
                   if out.nnz else np.empty(0, np.float64))
            return HostCSR(int(out.rows), int(out.cols), rp.astype(rp_dtype, copy=False), col, val)
        av, bv = A.view(), B.view()
        _check(lib().ocean_spgemm(self._h, ctypes.byref(av), ctypes.byref(bv), ctypes.byref(out), stream or None))
        return DeviceCSR(int(out.rows), int(out.cols), int(out.nnz), None, None, None, int(out.rowptr_bits), out)

    def symbolic(self, A: DeviceCSR, B: Optional[DeviceCSR] = None, stream: int = 0):
        """Exact per-row output counts (device tensor, uint32 stored as int32)."""
        import torch
        B = A if B is None else B
        out = torch.empty(A.rows, dtype=torch.int32, device="cuda")
        av, bv = A.view(), B.view()
        _check(lib().ocean_symbolic(self._h, ctypes.byref(av), ctypes.byref(bv), _ptr(out), stream or None))
        return out

    def row_estimates(self, A: DeviceCSR, B: Optional[DeviceCSR] = None, log2p: int = 6):
        """Raw HLL estimate of every row's output count (device tensor, uint32 as int32)."""
        import torch
        B = A if B is None else B
        out = torch.empty(A.rows, dtype=torch.int32, device="cuda")
        av, bv = A.view(), B.view()
        _check(lib().ocean_row_estimates(self._h, ctypes.byref(av), ctypes.byref(bv), log2p, _ptr(out), None))
        return out

    def get_stats(self) -> dict:
        need = ctypes.c_size_t(0)
        _check(lib().ocean_stats_json(self._h, None, 0, ctypes.byref(need)))
        buf = ctypes.create_string_buffer(need.value)
        _check(lib().ocean_stats_json(self._h, buf, need.value, ctypes.byref(need)))
        return json.loads(buf.value.decode())

    def stage_ms(self, stage: str) -> float:
        return float(lib().ocean_stage_ms(self._h, stage.encode()))


def murmur3_device(keys, seed: int = 1234):
    """MurmurHash3 of a CUDA uint32 tensor (int32 storage) on the device."""
    import torch
    out = torch.empty_like(keys)
    _check(lib().ocean_murmur3_u32(_ptr(keys), _ptr(out), keys.numel(), seed, None))
    return out


class Batch:
    """A batch plan (ocean_batch_*): many independent products run as one
    captured graph. ``A`` and ``B`` are lists of DeviceCSR (B None: A[p]*A[p]);
    they must stay alive as long as the plan."""

    def __init__(self, g: "SpGEMM", A, B=None, stream: int = 0):
        n = len(A)
        self._g = g
        self._inputs = (list(A), None if B is None else list(B))
        self._av = (CsrView * n)(*[a.view() for a in A])
        self._bv = None if B is None else (CsrView * n)(*[b.view() for b in B])
        self._h = ctypes.c_void_p()
        self.n = n
        _check(lib().ocean_batch_create(g._h, n, self._av, self._bv, ctypes.byref(self._h), stream or None))
        self._out = (CsrOut * n)()

    def launch(self, stream: int = 0) -> None:
        _check(lib().ocean_batch_launch(self._h, stream or None))

    def run(self, stream: int = 0) -> list:
        """One run; returns n DeviceCSR views of the results (valid until the next run)."""
        _check(lib().ocean_batch_run(self._h, self._out, stream or None))
        return self._views()

    def results(self) -> list:
        _check(lib().ocean_batch_results(self._h, self._out))
        return self._views()

    def _views(self) -> list:
        views = []
        for o in self._out:
            d = DeviceCSR(int(o.rows), int(o.cols), int(o.nnz), None, None, None, int(o.rowptr_bits), _Lent(o))
            d._plan = self  # the plan owns the memory: keep it alive while a view exists
            views.append(d)
        return views

    def download_into(self, rowptrs: np.ndarray, col: np.ndarray, val: np.ndarray, stream: int = 0,
                      wait: bool = True) -> None:
        """All results of the last run into (pinned) host arrays, concatenated;
        wait=False only queues the copies on `stream`."""
        fn = lib().ocean_batch_download if wait else lib().ocean_batch_download_async
        _check(fn(self._h, _ptr(rowptrs), _ptr(col), _ptr(val), stream or None))

    def info(self) -> dict:
        need = ctypes.c_size_t(0)
        _check(lib().ocean_batch_info_json(self._h, None, 0, ctypes.byref(need)))
        buf = ctypes.create_string_buffer(need.value)
        _check(lib().ocean_batch_info_json(self._h, buf, need.value, ctypes.byref(need)))
        return json.loads(buf.value.decode())

    def close(self) -> None:
        if self._h:
            lib().ocean_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Lent(CsrOut):
    """A result view lent by a batch plan (freeing it only clears the struct)."""

    def __init__(self, o: CsrOut):
        super().__init__()
        ctypes.memmove(ctypes.addressof(self), ctypes.addressof(o), ctypes.sizeof(CsrOut))


def spgemm_batched(g: "SpGEMM", A, B=None, stream: int = 0) -> list:
    """One-shot batch (ocean_spgemm_batched): owned device results."""
    n = len(A)
    av = (CsrView * n)(*[a.view() for a in A])
    bv = None if B is None else (CsrView * n)(*[b.view() for b in B])
    out = (CsrOut * n)()
    _check(lib().ocean_spgemm_batched(g._h, n, av, bv, out, stream or None))
    res = []
    for o in out:
        c = CsrOut()
        ctypes.memmove(ctypes.addressof(c), ctypes.addressof(o), ctypes.sizeof(CsrOut))
        res.append(DeviceCSR(int(c.rows), int(c.cols), int(c.nnz), None, None, None, int(c.rowptr_bits), c))
    return res
