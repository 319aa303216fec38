"""sadmrg -- Python binding of the B200 two-site DMRG library (ctypes over the C ABI).

The shared library ``libsadmrg_b200.so`` next to this file holds the sm_100a
kernels and the host bookkeeping; this module only marshals numpy arrays across
the ``extern "C"`` boundary declared in ``include/sadmrg.h``.  There is no
fallback: if the library or a CUDA device is missing, calls raise.

Block-sparse tensors cross the boundary as :class:`BlockTensorData` (the
reference's BlockTensor: bonds with sector labels / dimensions, the present
blocks by block index, and their column-major data concatenated in block order).
"""
from __future__ import annotations

import ctypes as C
import atexit
import os
import weakref
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("SADMRG_LIB") or os.path.join(_HERE, "libsadmrg_b200.so")

SYM_U1, SYM_SU2 = 0, 1
PREC_FP64, PREC_TF32X3 = 0, 1

EXPORTED = [
    "sadmrg_version", "sadmrg_create", "sadmrg_destroy", "sadmrg_last_error",
    "sadmrg_set_lanczos_tol", "sadmrg_heff_plan", "sadmrg_heff_info", "sadmrg_heff_apply", "sadmrg_heff_apply_device", "sadmrg_heff_apply_noalloc",
    "sadmrg_heff_profile", "sadmrg_heff_lanczos", "sadmrg_heff_lanczos2", "sadmrg_svd_truncate",
    "sadmrg_chain_create", "sadmrg_chain_set_dm", "sadmrg_chain_set_excited", "sadmrg_chain_set_precision", "sadmrg_chain_idmrg", "sadmrg_chain_prepare_sweep",
    "sadmrg_chain_sweep", "sadmrg_chain_read_mps", "sadmrg_chain_save_mps", "sadmrg_chain_freeze", "sadmrg_chain_bond", "sadmrg_chain_stats", "sadmrg_chain_set_tensor",
    "sadmrg_chain_stage_tensor", "sadmrg_chain_env_update", "sadmrg_staged_info", "sadmrg_staged_read",
    "sadmrg_device_status", "sadmrg_heff_launch_profile", "sadmrg_set_matvec_fusion", "sadmrg_heff_graph_bench",
    "sadmrg_heff_set_penalty", "sadmrg_batch_add", "sadmrg_batch_finalize", "sadmrg_batch_clear",
    "sadmrg_batch_info", "sadmrg_batch_apply", "sadmrg_batch_lanczos", "sadmrg_batch_profile",
    "sadmrg_chain_set_mlanc", "sadmrg_chain_save_ww", "sadmrg_chain_read_ww", "sadmrg_chain_save_enr",
    "sadmrg_chain_read_enr", "sadmrg_chain_ww", "sadmrg_heff_graph_steps", "sadmrg_heff_launches_per_matvec",
    "sadmrg_heff_wait_fault_test", "sadmrg_set_autotune", "sadmrg_heff_tiles", "sadmrg_set_tiles",
    "sadmrg_set_svd_precondition", "sadmrg_set_svd_stream", "sadmrg_set_svd_block",
    "sadmrg_chain_bond_flags",
]


class TensorDesc(C.Structure):
    _fields_ = [
        ("nbond", C.c_int), ("locspin", C.c_int),
        ("dir", C.POINTER(C.c_int)), ("nmom", C.POINTER(C.c_int)),
        ("q", C.POINTER(C.c_int)), ("d", C.POINTER(C.c_int)),
        ("nblocks", C.c_int), ("block_index", C.POINTER(C.c_longlong)),
        ("data", C.c_void_p),
    ]


_lib = None


def load(path: str = LIB_PATH):
    """Load the shared library (once) and declare the signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libsadmrg_b200.so not built at {path}; run __graft_entry__.build()")
    lib = C.CDLL(path)
    vp, ip, dp, lp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_longlong)
    td = C.POINTER(TensorDesc)
    sig = {
        "sadmrg_version": ([], C.c_int),
        "sadmrg_create": ([C.c_int, C.c_int, C.c_int, C.POINTER(vp)], C.c_int),
        "sadmrg_destroy": ([vp], C.c_int),
        "sadmrg_last_error": ([vp], C.c_char_p),
        "sadmrg_device_status": ([vp, ip], C.c_int),
        "sadmrg_heff_plan": ([vp, td, td, td, C.c_int, td, C.c_int, ip, ip], C.c_int),
        "sadmrg_set_lanczos_tol": ([vp, C.c_double], C.c_int),
        "sadmrg_set_matvec_fusion": ([vp, C.c_int], C.c_int),
        "sadmrg_heff_info": ([vp, lp, dp, dp, ip], C.c_int),
        "sadmrg_heff_set_penalty": ([vp, C.c_int, vp, dp], C.c_int),
        "sadmrg_batch_add": ([vp, vp], C.c_int),
        "sadmrg_batch_finalize": ([vp], C.c_int),
        "sadmrg_batch_clear": ([vp], C.c_int),
        "sadmrg_batch_info": ([vp, ip, lp, dp, C.c_int, lp], C.c_int),
        "sadmrg_batch_apply": ([vp, vp, vp, C.c_int], C.c_int),
        "sadmrg_batch_lanczos": ([vp, vp, C.c_int, C.c_int, dp, ip, ip], C.c_int),
        "sadmrg_batch_profile": ([vp, C.c_int, C.c_int, dp], C.c_int),
        "sadmrg_heff_apply": ([vp, vp, vp, C.c_int], C.c_int),
        "sadmrg_heff_apply_device": ([vp, vp, vp, C.c_int], C.c_int),
        "sadmrg_heff_apply_noalloc": ([vp, vp, vp, C.c_int], C.c_int),
        "sadmrg_heff_lanczos": ([vp, vp, C.c_int, C.c_int, dp, ip], C.c_int),
        "sadmrg_heff_lanczos2": ([vp, vp, C.c_int, dp, ip], C.c_int),
        "sadmrg_heff_profile": ([vp, C.c_int, C.c_int, vp, vp, dp, dp], C.c_int),
        "sadmrg_heff_launch_profile": ([vp, C.c_int, C.c_int, vp, vp, C.c_int, ip, ip, dp], C.c_int),
        "sadmrg_heff_graph_bench": ([vp, C.c_int, C.c_int, vp, vp, dp], C.c_int),
        "sadmrg_heff_graph_steps": ([vp, C.c_int, C.c_int, vp, vp, vp, C.c_longlong, dp], C.c_int),
        "sadmrg_heff_launches_per_matvec": ([vp, C.c_int, ip], C.c_int),
        "sadmrg_heff_wait_fault_test": ([vp, C.c_longlong, ip], C.c_int),
        "sadmrg_set_autotune": ([vp, C.c_int], C.c_int),
        "sadmrg_set_svd_precondition": ([vp, C.c_int], C.c_int),
        "sadmrg_set_svd_stream": ([vp, C.c_int], C.c_int),
        "sadmrg_set_svd_block": ([vp, C.c_int], C.c_int),
        "sadmrg_heff_tiles": ([vp, C.c_int, dp, ip], C.c_int),
        "sadmrg_set_tiles": ([vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int], C.c_int),
        "sadmrg_svd_truncate": ([vp, td, td, td, C.c_double, C.c_double, C.c_int, ip, dp], C.c_int),
        "sadmrg_chain_create": ([vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double], C.c_int),
        "sadmrg_chain_set_precision": ([vp, C.c_int], C.c_int),
        "sadmrg_chain_set_dm": ([vp, C.c_double], C.c_int),
        "sadmrg_chain_set_excited": ([vp, C.c_int], C.c_int),
        "sadmrg_chain_idmrg": ([vp, dp], C.c_int),
        "sadmrg_chain_prepare_sweep": ([vp], C.c_int),
        "sadmrg_chain_sweep": ([vp, dp], C.c_int),
        "sadmrg_chain_bond": ([vp, C.c_int, C.c_int, ip, ip, ip], C.c_int),
        "sadmrg_chain_read_mps": ([vp, C.c_char_p, C.c_int], C.c_int),
        "sadmrg_chain_save_mps": ([vp, C.c_char_p], C.c_int),
        "sadmrg_chain_set_mlanc": ([vp, C.c_int], C.c_int),
        "sadmrg_chain_save_ww": ([vp, C.c_char_p], C.c_int),
        "sadmrg_chain_read_ww": ([vp, C.c_char_p, C.c_int], C.c_int),
        "sadmrg_chain_save_enr": ([vp, C.c_char_p], C.c_int),
        "sadmrg_chain_read_enr": ([vp, C.c_char_p, C.c_int], C.c_int),
        "sadmrg_chain_ww": ([vp, C.c_int, ip, dp], C.c_int),
        "sadmrg_chain_freeze": ([vp, C.c_int, C.c_char_p], C.c_int),
        "sadmrg_chain_stats": ([vp, dp, C.c_int], C.c_int),
        "sadmrg_chain_bond_flags": ([vp, C.c_int, ip], C.c_int),
        "sadmrg_chain_set_tensor": ([vp, C.c_int, C.c_int, C.c_int, td], C.c_int),
        "sadmrg_chain_stage_tensor": ([vp, C.c_int, C.c_int, C.c_int], C.c_int),
        "sadmrg_chain_env_update": ([vp, C.c_int, C.c_int, C.c_int], C.c_int),
        "sadmrg_staged_info": ([vp, C.c_int, ip, ip, ip, ip, lp], C.c_int),
        "sadmrg_staged_read": ([vp, C.c_int, ip, ip, ip, ip, lp, vp], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


class SadmrgError(RuntimeError):
    pass


# status codes of include/sadmrg.h
STATUS_NAMES = {1: "SADMRG_ERR_ARG", 2: "SADMRG_ERR_CUDA", 3: "SADMRG_ERR_NOMEM", 4: "SADMRG_ERR_STATE",
                5: "SADMRG_ERR_NUMERIC", 6: "SADMRG_ERR_LIMIT", 7: "SADMRG_ERR_DEVICE_FLAG"}


@dataclass
class BlockTensorData:
    """Host image of a BlockTensor: bonds, present blocks, concatenated data."""
    dirs: List[int]
    qs: List[List[int]]
    ds: List[List[int]]
    locspin: int
    blocks: np.ndarray            # int64 block indices, ascending
    data: np.ndarray              # float64 or complex128, all present blocks
    _keep: list = field(default_factory=list, repr=False)

    @property
    def nbond(self) -> int:
        return len(self.dirs)

    def block_labels(self, idx: int):
        """Per-bond sector positions of block `idx` (mixed radix, bond 0 fastest): the
        sector label of bond b is qs[b][pos[b]], its dimension ds[b][pos[b]]."""
        out = []
        for b in range(self.nbond):
            n = len(self.qs[b])
            out.append(idx % n)
            idx //= n
        return out

    def block_dims(self, idx: int):
        sec = self.block_labels(idx)
        return [self.ds[b][s] for b, s in enumerate(sec)]

    def block_views(self):
        """(block index, labels, column-major ndarray view) for every present block."""
        off = 0
        res = []
        for bi in self.blocks:
            sec = self.block_labels(int(bi))
            dims = [self.ds[b][s] for b, s in enumerate(sec)]
            n = int(np.prod(dims))
            arr = self.data[off:off + n].reshape(dims[::-1]).transpose()
            res.append((int(bi), [self.qs[b][s] for b, s in enumerate(sec)], arr))
            off += n
        return res

    def desc(self) -> TensorDesc:
        dirs = np.ascontiguousarray(self.dirs, dtype=np.int32)
        nmom = np.ascontiguousarray([len(q) for q in self.qs], dtype=np.int32)
        q = np.ascontiguousarray([x for qq in self.qs for x in qq], dtype=np.int32)
        d = np.ascontiguousarray([x for dd in self.ds for x in dd], dtype=np.int32)
        blocks = np.ascontiguousarray(self.blocks, dtype=np.int64)
        data = np.ascontiguousarray(self.data)
        self._keep = [dirs, nmom, q, d, blocks, data]
        ip = C.POINTER(C.c_int)
        return TensorDesc(self.nbond, int(self.locspin), dirs.ctypes.data_as(ip), nmom.ctypes.data_as(ip),
                          q.ctypes.data_as(ip), d.ctypes.data_as(ip), len(blocks),
                          blocks.ctypes.data_as(C.POINTER(C.c_longlong)), data.ctypes.data)


_live = weakref.WeakSet()
_atexit_registered = False


def _close_all():
    for h in list(_live):
        try:
            h.close()
        except Exception:
            pass


class Handle:
    """One device + one stream (sadmrg_create)."""

    def __init__(self, sym: int = SYM_U1, cplx: bool = False, device: int = 0):
        self.lib = load()
        self.cplx = bool(cplx)
        self.dtype = np.complex128 if cplx else np.float64
        h = C.c_void_p()
        rc = self.lib.sadmrg_create(int(sym), int(bool(cplx)), int(device), C.byref(h))
        if rc != 0:
            why = " (no usable CUDA device)" if rc == 2 else ""
            raise SadmrgError(f"sadmrg_create failed with status {rc} {STATUS_NAMES.get(rc, '')}{why}")
        self.h = h
        # Handles still open at interpreter exit are destroyed by an exit hook that
        # is registered after the first handle (and so after the CUDA runtime's own
        # exit hook, which then runs later): destroying one after the runtime has
        # shut down would touch freed runtime state.
        global _atexit_registered
        _live.add(self)
        if not _atexit_registered:
            atexit.register(_close_all)
            _atexit_registered = True

    def close(self):
        if getattr(self, "h", None):
            self.lib.sadmrg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc != 0:
            msg = self.lib.sadmrg_last_error(self.h)
            raise SadmrgError(f"{what}: status {rc} {STATUS_NAMES.get(rc, '')}: {msg.decode() if msg else ''}")

    def set_matvec_fusion(self, fused: Optional[bool]):
        """True: the split-precision matvec as one cooperative launch; False: pack + one
        launch per stage; None (the default): one launch for small plans only."""
        self._check(self.lib.sadmrg_set_matvec_fusion(self.h, -1 if fused is None else int(bool(fused))),
                    "set_matvec_fusion")

    def set_lanczos_tol(self, ov_tol: float):
        self._check(self.lib.sadmrg_set_lanczos_tol(self.h, float(ov_tol)), "set_lanczos_tol")

    # -- frozen two-site problem -------------------------------------------
    def heff_plan(self, psi: BlockTensorData, hh_left: Optional[BlockTensorData],
                  hh_right: Optional[BlockTensorData], ops: Sequence[BlockTensorData],
                  terms: Sequence[tuple]):
        self._psi_template = psi
        d_psi = psi.desc()
        d_hl = C.pointer(hh_left.desc()) if hh_left is not None else None
        d_hr = C.pointer(hh_right.desc()) if hh_right is not None else None
        arr = (TensorDesc * max(len(ops), 1))()
        for i, o in enumerate(ops):
            arr[i] = o.desc()
        op1 = np.ascontiguousarray([t[0] for t in terms], dtype=np.int32)
        op2 = np.ascontiguousarray([t[1] for t in terms], dtype=np.int32)
        ip = C.POINTER(C.c_int)
        rc = self.lib.sadmrg_heff_plan(self.h, C.byref(d_psi), d_hl, d_hr, len(ops), arr, len(terms),
                                       op1.ctypes.data_as(ip), op2.ctypes.data_as(ip))
        self._check(rc, "heff_plan")

    def heff_set_penalty(self, vecs, weights):
        """Excited-state penalty: H_eff psi -= sum_k weights[k] <vecs[k]|psi> vecs[k]."""
        v = np.ascontiguousarray(np.asarray(vecs, dtype=self.dtype).reshape(len(weights), -1)) if len(weights) else None
        w = np.ascontiguousarray(weights, dtype=np.float64)
        self._check(self.lib.sadmrg_heff_set_penalty(self.h, len(w), v.ctypes.data if v is not None else None,
                                                     w.ctypes.data_as(C.POINTER(C.c_double))), "heff_set_penalty")

    # -- many instances ---------------------------------------------------------
    def batch_add(self, inst: "Handle"):
        """Append inst's H_eff plan to this handle's batch (inst may be closed afterwards)."""
        self._check(self.lib.sadmrg_batch_add(self.h, inst.h), "batch_add")

    def batch_finalize(self):
        self._check(self.lib.sadmrg_batch_finalize(self.h), "batch_finalize")
        return self.batch_info()

    def batch_clear(self):
        self._check(self.lib.sadmrg_batch_clear(self.h), "batch_clear")

    def batch_info(self):
        ni, n, fl = C.c_int(), C.c_longlong(), C.c_double()
        self._check(self.lib.sadmrg_batch_info(self.h, C.byref(ni), C.byref(n), C.byref(fl), 0, None), "batch_info")
        off = np.zeros(ni.value + 1, dtype=np.int64)
        self._check(self.lib.sadmrg_batch_info(self.h, C.byref(ni), C.byref(n), C.byref(fl), len(off),
                                               off.ctypes.data_as(C.POINTER(C.c_longlong))), "batch_info")
        return {"ninst": ni.value, "n": n.value, "flops": fl.value, "offsets": off}

    def batch_apply(self, psi: np.ndarray, precision: int = PREC_FP64) -> np.ndarray:
        x = np.ascontiguousarray(psi, dtype=self.dtype)
        out = np.empty_like(x)
        self._check(self.lib.sadmrg_batch_apply(self.h, x.ctypes.data, out.ctypes.data, int(precision)), "batch_apply")
        return out

    def batch_profile(self, precision: int = PREC_FP64, reps: int = 20) -> float:
        ms = C.c_double()
        self._check(self.lib.sadmrg_batch_profile(self.h, int(precision), int(reps), C.byref(ms)), "batch_profile")
        return ms.value

    def batch_lanczos(self, psi: np.ndarray, mlanc: int = 40, precision: int = PREC_FP64):
        """(energies, Ritz vectors (all segments), matvecs per instance, batched matvec launches)."""
        info = self.batch_info()
        x = np.array(psi, dtype=self.dtype, copy=True)
        e = np.zeros(info["ninst"])
        mv = np.zeros(info["ninst"], dtype=np.int32)
        bm = C.c_int()
        self._check(self.lib.sadmrg_batch_lanczos(self.h, x.ctypes.data, int(mlanc), int(precision),
                                                  e.ctypes.data_as(C.POINTER(C.c_double)),
                                                  mv.ctypes.data_as(C.POINTER(C.c_int)), C.byref(bm)), "batch_lanczos")
        return e, x, mv, bm.value

    def heff_info(self):
        n = C.c_longlong()
        fl, by = C.c_double(), C.c_double()
        nt = C.c_int()
        self._check(self.lib.sadmrg_heff_info(self.h, C.byref(n), C.byref(fl), C.byref(by), C.byref(nt)), "heff_info")
        return {"n": n.value, "flops": fl.value, "bytes": by.value, "ntasks": nt.value}

    def heff_apply(self, psi: np.ndarray, precision: int = PREC_FP64, out: Optional[np.ndarray] = None) -> np.ndarray:
        x = np.ascontiguousarray(psi, dtype=self.dtype)
        if out is None:
            out = np.empty_like(x)
        assert out.dtype == x.dtype and out.shape == x.shape and out.flags.c_contiguous
        self._check(self.lib.sadmrg_heff_apply(self.h, x.ctypes.data, out.ctypes.data, int(precision)), "heff_apply")
        return out

    def heff_apply_device(self, psi_ptr: int, out_ptr: int, precision: int = PREC_FP64):
        self._check(self.lib.sadmrg_heff_apply_device(self.h, C.c_void_p(psi_ptr), C.c_void_p(out_ptr),
                                                      int(precision)), "heff_apply_device")

    def device_status(self) -> int:
        """Status word of the tcgen05 kernels since the last query (0 = fine); clears it."""
        v = C.c_int(0)
        self._check(self.lib.sadmrg_device_status(self.h, C.byref(v)), "device_status")
        return v.value

    def heff_profile(self, precision: int = PREC_FP64, reps: int = 10, psi_ptr: int = 0, out_ptr: int = 0):
        """per-stage device milliseconds and algorithmic flops of one H_eff*psi"""
        ms = (C.c_double * 2)()
        fl = (C.c_double * 2)()
        self._check(self.lib.sadmrg_heff_profile(self.h, int(precision), int(reps), C.c_void_p(psi_ptr or None),
                                                 C.c_void_p(out_ptr or None), ms, fl), "heff_profile")
        return [ms[0], ms[1]], [fl[0], fl[1]]

    def heff_apply_noalloc(self, psi_ptr: int, out_ptr: int, precision: int = PREC_FP64):
        """H_eff*psi on device pointers without allocating (library's fixed device scratch)."""
        self._check(self.lib.sadmrg_heff_apply_noalloc(self.h, C.c_void_p(psi_ptr), C.c_void_p(out_ptr),
                                                       int(precision)), "heff_apply_noalloc")

    def heff_launch_profile(self, precision: int = PREC_FP64, reps: int = 10, psi_ptr: int = 0, out_ptr: int = 0):
        """[(kind, mean ms)] for every kernel one matvec launches; kind 0: psi -> TF32 panels,
        1 + 2*stage: grouped GEMM of that stage, 2 + 2*stage: its split-K reduction,
        5: the whole matvec in one launch."""
        cap = 64
        n = C.c_int(0)
        kinds = np.zeros(cap, dtype=np.int32)
        ms = np.zeros(cap)
        self._check(self.lib.sadmrg_heff_launch_profile(self.h, int(precision), int(reps), C.c_void_p(psi_ptr),
                                                        C.c_void_p(out_ptr), cap, C.byref(n),
                                                        kinds.ctypes.data_as(C.POINTER(C.c_int)),
                                                        ms.ctypes.data_as(C.POINTER(C.c_double))),
                    "heff_launch_profile")
        return [(int(kinds[i]), float(ms[i])) for i in range(min(n.value, cap))]

    def heff_graph_bench(self, precision: int = PREC_FP64, reps: int = 200, psi_ptr: int = 0, out_ptr: int = 0) -> float:
        """Mean device ms of one matvec replayed `reps` times from a captured CUDA graph."""
        ms = C.c_double()
        self._check(self.lib.sadmrg_heff_graph_bench(self.h, int(precision), int(reps), C.c_void_p(psi_ptr),
                                                     C.c_void_p(out_ptr), C.byref(ms)), "heff_graph_bench")
        return ms.value

    def heff_graph_steps(self, precision: int, steps: int, psi_ptr: int = 0, out_ptr: int = 0, flush_ptr: int = 0,
                         flush_bytes: int = 0) -> np.ndarray:
        """Device ms of `steps` replays of one captured matvec, L2 flushed (flush_bytes written) before each."""
        ms = np.zeros(int(steps))
        self._check(self.lib.sadmrg_heff_graph_steps(self.h, int(precision), int(steps), psi_ptr or None,
                                                     out_ptr or None, flush_ptr or None, int(flush_bytes),
                                                     ms.ctypes.data_as(C.POINTER(C.c_double))), "heff_graph_steps")
        return ms

    def heff_wait_fault_test(self, wait_ns: int = 50_000_000) -> int:
        """One split-precision matvec whose first psi panels never complete (bounded waits of
        wait_ns): returns the status word it left (nonzero: a wait ran out); the plan is reset."""
        st = C.c_int()
        self._check(self.lib.sadmrg_heff_wait_fault_test(self.h, int(wait_ns), C.byref(st)), "heff_wait_fault_test")
        return st.value

    def set_autotune(self, on: bool):
        """Time candidate tcgen05 schedules for every new H_eff plan (default on)."""
        self._check(self.lib.sadmrg_set_autotune(self.h, int(bool(on))), "set_autotune")

    def set_svd_precondition(self, on: int):
        """Householder QRs before the block SVD's Jacobi: 0 never, 1 for calls whose
        widest block has at least 32 columns (the default), 2 always."""
        self._check(self.lib.sadmrg_set_svd_precondition(self.h, int(on)), "set_svd_precondition")

    def set_svd_block(self, b: int):
        """Jacobi column blocks of the block SVD: 8, 16, or 0 for the default rule."""
        self._check(self.lib.sadmrg_set_svd_block(self.h, int(b)), "set_svd_block")

    def set_svd_stream(self, on: bool):
        """Stream every Jacobi visit's rows in chunks (default off: resident where they fit)."""
        self._check(self.lib.sadmrg_set_svd_stream(self.h, int(bool(on))), "set_svd_stream")

    def set_tiles(self, bn: int, kc_min: int = 16, kc_max: int = 0, ctas_per_sm: int = 1, one_launch: int = -1):
        """Fix the tcgen05 schedule of the H_eff plans made from now on (bn = 0: autotune again)."""
        self._check(self.lib.sadmrg_set_tiles(self.h, int(bn), int(kc_min), int(kc_max), int(ctas_per_sm),
                                              int(one_launch)), "set_tiles")

    def heff_tiles(self) -> dict:
        """The current plan's tcgen05 tile choice and the candidates timed for it."""
        out = np.zeros(64)
        n = C.c_int()
        self._check(self.lib.sadmrg_heff_tiles(self.h, 64, out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(n)),
                    "heff_tiles")
        v = out[:n.value]
        cands = [{"bn": int(v[7 + 6 * i]), "kc_min": int(v[8 + 6 * i]), "kc_max": int(v[9 + 6 * i]),
                  "ctas_per_sm": int(v[10 + 6 * i]), "one_launch": bool(v[11 + 6 * i]), "ms": float(v[12 + 6 * i])}
                 for i in range(int(v[6]))]
        return {"bn": int(v[0]), "kc_min": int(v[1]), "kc_max": int(v[2]), "ctas_per_sm": int(v[3]),
                "one_launch": bool(v[4]), "source": ["heuristic", "timed", "cached", "set"][int(v[5])],
                "candidates": cands}

    def heff_launches_per_matvec(self, precision: int) -> int:
        n = C.c_int()
        self._check(self.lib.sadmrg_heff_launches_per_matvec(self.h, int(precision), C.byref(n)),
                    "heff_launches_per_matvec")
        return n.value

    def heff_lanczos(self, psi: np.ndarray, mlanc: int = 40, precision: int = PREC_FP64):
        x = np.array(psi, dtype=self.dtype, copy=True)
        e = C.c_double()
        mv = C.c_int()
        self._check(self.lib.sadmrg_heff_lanczos(self.h, x.ctypes.data, int(mlanc), int(precision), C.byref(e),
                                                 C.byref(mv)), "heff_lanczos")
        return e.value, x, mv.value

    def heff_lanczos2(self, psi: np.ndarray, mlanc: int = 40):
        """Lanczos::lanczos2 (FP64, no convergence checks): (energy, Ritz vector, matvecs)."""
        x = np.array(psi, dtype=self.dtype, copy=True)
        e = C.c_double()
        mv = C.c_int()
        self._check(self.lib.sadmrg_heff_lanczos2(self.h, x.ctypes.data, int(mlanc), C.byref(e), C.byref(mv)),
                    "heff_lanczos2")
        return e.value, x, mv.value

    # -- SVD -------------------------------------------------------------------
    def svd_truncate(self, psi: BlockTensorData, tu: BlockTensorData, tv: BlockTensorData, p1: float, p2: float,
                     max_dcut: int):
        kept = C.c_int()
        dw = C.c_double()
        a, b, c = psi.desc(), tu.desc(), tv.desc()
        self._check(self.lib.sadmrg_svd_truncate(self.h, C.byref(a), C.byref(b), C.byref(c), float(p1), float(p2),
                                                 int(max_dcut), C.byref(kept), C.byref(dw)), "svd_truncate")
        return self.staged(0), self.staged(1), kept.value, dw.value

    def staged(self, which: int) -> Optional[BlockTensorData]:
        nb, ls, ns, nbl = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        ne = C.c_longlong()
        self._check(self.lib.sadmrg_staged_info(self.h, int(which), C.byref(nb), C.byref(ls), C.byref(ns),
                                                C.byref(nbl), C.byref(ne)), "staged_info")
        if nb.value == 0:
            return None
        dirs = np.zeros(nb.value, np.int32)
        nmom = np.zeros(nb.value, np.int32)
        q = np.zeros(ns.value, np.int32)
        d = np.zeros(ns.value, np.int32)
        blocks = np.zeros(nbl.value, np.int64)
        data = np.zeros(ne.value, self.dtype)
        ip = C.POINTER(C.c_int)
        self._check(self.lib.sadmrg_staged_read(self.h, int(which), dirs.ctypes.data_as(ip), nmom.ctypes.data_as(ip),
                                                q.ctypes.data_as(ip), d.ctypes.data_as(ip),
                                                blocks.ctypes.data_as(C.POINTER(C.c_longlong)), data.ctypes.data),
                    "staged_read")
        qs, ds, o = [], [], 0
        for n in nmom:
            qs.append([int(x) for x in q[o:o + n]])
            ds.append([int(x) for x in d[o:o + n]])
            o += n
        return BlockTensorData([int(x) for x in dirs], qs, ds, ls.value, blocks, data)

    # -- chain -----------------------------------------------------------------
    def chain_create(self, lx: int, ly: int, bondd: int, physpn: int = 1, totspin: int = 0, open_bc: bool = True,
                     J2: float = 0.0):
        self._check(self.lib.sadmrg_chain_create(self.h, lx, ly, bondd, physpn, totspin, int(bool(open_bc)),
                                                 float(J2)), "chain_create")

    def chain_set_dm(self, dz: float):
        """Dz (S_a x S_b)_z on every J1 bond (U(1) complex chains, before iDMRG)."""
        self._check(self.lib.sadmrg_chain_set_dm(self.h, float(dz)), "chain_set_dm")

    def chain_set_excited(self, exci: int):
        """Target excited state exci (before chain_read_mps): the lower
        states 0 .. exci-1 and their energies are read with the chain's own files."""
        self._check(self.lib.sadmrg_chain_set_excited(self.h, int(exci)), "chain_set_excited")

    def chain_set_precision(self, prec: int):
        self._check(self.lib.sadmrg_chain_set_precision(self.h, int(prec)), "chain_set_precision")

    def chain_idmrg(self) -> float:
        e = C.c_double()
        self._check(self.lib.sadmrg_chain_idmrg(self.h, C.byref(e)), "chain_idmrg")
        return e.value

    def chain_prepare_sweep(self):
        self._check(self.lib.sadmrg_chain_prepare_sweep(self.h), "chain_prepare_sweep")

    def chain_sweep(self) -> float:
        e = C.c_double()
        self._check(self.lib.sadmrg_chain_sweep(self.h, C.byref(e)), "chain_sweep")
        return e.value

    def chain_read_mps(self, directory: str, bond_read: int):
        self._check(self.lib.sadmrg_chain_read_mps(self.h, directory.encode(), int(bond_read)), "chain_read_mps")

    def chain_save_mps(self, directory: str):
        self._check(self.lib.sadmrg_chain_save_mps(self.h, directory.encode()), "chain_save_mps")

    def chain_set_mlanc(self, mlanc: int):
        """Lanczos length of the chain's solves (the reference's mlanc = 40)."""
        self._check(self.lib.sadmrg_chain_set_mlanc(self.h, int(mlanc)), "chain_set_mlanc")

    def chain_save_ww(self, directory: str):
        self._check(self.lib.sadmrg_chain_save_ww(self.h, directory.encode()), "chain_save_ww")

    def chain_read_ww(self, directory: str, bond_read: int):
        self._check(self.lib.sadmrg_chain_read_ww(self.h, directory.encode(), int(bond_read)), "chain_read_ww")

    def chain_save_enr(self, directory: str):
        self._check(self.lib.sadmrg_chain_save_enr(self.h, directory.encode()), "chain_save_enr")

    def chain_read_enr(self, directory: str, bond_read: int):
        self._check(self.lib.sadmrg_chain_read_enr(self.h, directory.encode(), int(bond_read)), "chain_read_enr")

    def chain_ww(self) -> np.ndarray:
        """The chain's ww array (singular values of the truncations, the reference's layout)."""
        n = C.c_int()
        self._check(self.lib.sadmrg_chain_ww(self.h, 0, C.byref(n), None), "chain_ww")
        out = np.zeros(max(n.value, 1))
        self._check(self.lib.sadmrg_chain_ww(self.h, n.value, C.byref(n), out.ctypes.data_as(C.POINTER(C.c_double))),
                    "chain_ww")
        return out[:n.value]

    def chain_freeze(self, il: int, export_dir: Optional[str] = None) -> BlockTensorData:
        """Freeze the two-site problem at (il, il+1) as the handle's H_eff plan; returns psi."""
        self._check(self.lib.sadmrg_chain_freeze(self.h, int(il), (export_dir or "").encode()), "chain_freeze")
        return self.staged(0)

    def chain_bond(self, site: int):
        cap = 4096
        n = C.c_int()
        q = np.zeros(cap, np.int32)
        d = np.zeros(cap, np.int32)
        ip = C.POINTER(C.c_int)
        self._check(self.lib.sadmrg_chain_bond(self.h, int(site), cap, C.byref(n), q.ctypes.data_as(ip),
                                               d.ctypes.data_as(ip)), "chain_bond")
        return [(int(q[i]), int(d[i])) for i in range(n.value)]

    def chain_bond_flags(self, ns: int) -> List[int]:
        """Per bond il: flags of its last truncation (1 rounding tie, 2 stop-test tie)."""
        f = np.zeros(ns, np.int32)
        self._check(self.lib.sadmrg_chain_bond_flags(self.h, int(ns), f.ctypes.data_as(C.POINTER(C.c_int))),
                    "chain_bond_flags")
        return [int(x) for x in f]

    def chain_stats(self):
        out = np.zeros(14)
        self._check(self.lib.sadmrg_chain_stats(self.h, out.ctypes.data_as(C.POINTER(C.c_double)), 14), "chain_stats")
        keys = ["lanczos_s", "env_s", "svd_s", "prep_s", "matvecs", "heff_flops", "gemm_flops", "launches",
                "discarded", "near_ties", "svd_kernel_s", "svd_sweeps", "plan_s", "stop_ties"]
        return dict(zip(keys, out.tolist()))

    def chain_set_tensor(self, kind: int, site: int, k: int, t: Optional[BlockTensorData]):
        d = C.byref(t.desc()) if t is not None else None
        self._check(self.lib.sadmrg_chain_set_tensor(self.h, int(kind), int(site), int(k), d), "chain_set_tensor")

    def chain_get_tensor(self, kind: int, site: int, k: int = 0) -> Optional[BlockTensorData]:
        self._check(self.lib.sadmrg_chain_stage_tensor(self.h, int(kind), int(site), int(k)), "chain_stage_tensor")
        return self.staged(0)

    def chain_env_update(self, site: int, direction: int, real_env: bool):
        self._check(self.lib.sadmrg_chain_env_update(self.h, int(site), int(direction), int(bool(real_env))),
                    "chain_env_update")


def read_exported_tensor(directory: str, name: str, cplx: bool) -> Optional[BlockTensorData]:
    """A tensor written by sadmrg_chain_freeze(..., export_dir): <name>.txt + <name>.bin."""
    path = os.path.join(directory, name + ".txt")
    if not os.path.exists(path):
        return None
    dirs, qs, ds, blocks, ls = [], [], [], [], 0
    with open(path) as f:
        for line in f:
            t = line.split()
            if not t:
                continue
            if t[0] == "nbond":
                ls = int(t[3])
            elif t[0] == "bond":
                qi, di = t.index("q"), t.index("d")
                dirs.append(int(t[3]))
                qs.append([int(x) for x in t[qi + 1:di]])
                ds.append([int(x) for x in t[di + 1:]])
            elif t[0] == "block":
                blocks.append(int(t[1]))
    data = np.fromfile(os.path.join(directory, name + ".bin"), dtype=np.complex128 if cplx else np.float64)
    return BlockTensorData(dirs, qs, ds, ls, np.array(blocks, np.int64), data)


def write_exported_tensor(directory: str, name: str, t: BlockTensorData) -> None:
    """Write t in the format of sadmrg_chain_freeze's export (<name>.txt + <name>.bin),
    which read_exported_tensor and the reference harness's load mode read back."""
    nb = t.nbond
    sizes = []
    lines = [f"nbond {nb} locspin {t.locspin} nten {int(np.prod([len(q) for q in t.qs]))}"]
    for b in range(nb):
        lines.append(f"bond {b} dir {t.dirs[b]} nmom {len(t.qs[b])} q " + " ".join(str(x) for x in t.qs[b]) +
                     " d " + " ".join(str(x) for x in t.ds[b]))
    off = 0
    for bi in t.blocks:
        lab = t.block_labels(int(bi))
        q = [t.qs[b][lab[b]] for b in range(nb)]
        d = [t.ds[b][lab[b]] for b in range(nb)]
        n = int(np.prod(d))
        lines.append(f"block {int(bi)} q " + " ".join(map(str, q)) + " d " + " ".join(map(str, d)) +
                     f" off {off} n {n}")
        off += n
        sizes.append(n)
    if off != t.data.size:
        raise ValueError(f"{name}: blocks hold {off} elements, data has {t.data.size}")
    with open(os.path.join(directory, name + ".txt"), "w") as f:
        f.write("\n".join(lines) + "\n")
    np.ascontiguousarray(t.data).tofile(os.path.join(directory, name + ".bin"))


def channel_weights(t: BlockTensorData, J: float, dz: float) -> np.ndarray:
    """Per-element coupling of a U(1) operator on a J1 bond with a DM term: J - i dz q / 2,
    q the charge of the block's channel leg (bond 1), as sadmrg_chain_set_dm defines it."""
    w = np.empty(t.data.size, np.complex128)
    off = 0
    for bi in t.blocks:
        lab = t.block_labels(int(bi))
        n = int(np.prod([t.ds[b][lab[b]] for b in range(t.nbond)]))
        w[off:off + n] = J - 0.5j * dz * t.qs[1][lab[1]]
        off += n
    return w


def load_exported_problem(h: "Handle", directory: str) -> BlockTensorData:
    """Plan H_eff*psi on a problem exported by sadmrg_chain_freeze (the reference's operator set)."""
    meta = open(os.path.join(directory, "meta.txt")).read().split("\n")
    kv = meta[0].split()
    m = {kv[i]: kv[i + 1] for i in range(0, len(kv) - 1, 2)}
    il, ir, ns = int(m["il"]), int(m["ir"]), int(m["ns"])
    coup = [float(x) for x in meta[1].split()[1:]]
    dz = float(m.get("dz", 0.0))
    hmap = {}
    for line in meta[2:]:
        t = line.split()
        if t and t[0] == "hmap":
            hmap[(int(t[1]), int(t[2]))] = int(t[3])
    cplx = h.cplx
    psi = read_exported_tensor(directory, "psi", cplx)
    hl = read_exported_tensor(directory, "hh_il", cplx)
    hr = read_exported_tensor(directory, "hh_ir", cplx)
    ops, terms = [], []
    left = il < ns // 2
    m1, m4 = (il + 1, ns - ir) if left else (ns - ir, il + 1)
    for m0 in range(m1):
        acc = None
        for mm in range(m4):
            j, k = (m0, ir + mm) if left else (mm, ir + m0)
            hv = hmap.get((j, k), 0)
            if hv <= 0:
                continue
            t = read_exported_tensor(directory, f"opr_ir_{k}" if left else f"opr_il_{j}", cplx)
            if t is None:
                continue
            w = coup[hv]
            if hv == 1 and dz != 0.0:
                w = channel_weights(t, coup[hv], dz)
            if acc is None:
                acc = BlockTensorData(t.dirs, t.qs, t.ds, t.locspin, t.blocks.copy(), w * t.data)
            else:
                if list(acc.blocks) != list(t.blocks):
                    raise ValueError("summed operators with different block sets are not supported here")
                acc.data = acc.data + w * t.data
        if acc is None:
            continue
        fixed = read_exported_tensor(directory, f"opr_il_{m0}" if left else f"opr_ir_{ir + m0}", cplx)
        if fixed is None:
            continue
        ops += [fixed, acc]
        terms.append((len(ops) - 2, len(ops) - 1) if left else (len(ops) - 1, len(ops) - 2))
    h.heff_plan(psi, hl, hr, ops, terms)
    return psi
