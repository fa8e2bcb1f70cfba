"""Python mirror of the reference's hot-path interface.

Reference (geektrove/GPUSpGEMM)                      here
--------------------------------------------------  ---------------------------------
utils::DeviceCSR<T>            (csr.cuh:22-63)       DeviceCSR (torch CUDA tensors)
HostCSR::to<Device>() / to<Host>() (csr.cuh:193-203) DeviceCSR.from_host / .to_host
proposal::proposal<T>(A, B)    (proposal.cuh:85-124) proposal(A, B)
utils::get_nip(A, B)           (nip.cuh:52-78)       get_nip(A, B)
apps' convert + run + to<Host> (proposal.cu:15-26)   proposal_host(A, B)

Everything calls the C ABI of libspgemm_b200.so (include/spgemm.h); errors
raise SpgemmError like the reference's std::runtime_error.  PyTorch only
provides device memory and streams here.
"""
from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .csr import HostCSR

try:
    import torch
except ImportError:  # pragma: no cover - torch is part of the runtime image
    torch = None


def _require_torch():
    if torch is None or not torch.cuda.is_available():
        raise RuntimeError("a CUDA device is required")


class Handle:
    """Owns one spgemm_handle_t (scratch, side streams, pinned staging)."""

    def __init__(self, device: int | None = None):
        self._h = C.c_void_p()
        dev = -1 if device is None else int(device)
        N.check(N.lib().spgemm_create(C.byref(self._h), dev))

    @property
    def ptr(self) -> C.c_void_p:
        if not self._h:
            raise RuntimeError("handle is closed")
        return self._h

    def close(self) -> None:
        if self._h:
            N.lib().spgemm_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_option(self, option: int, value: int) -> None:
        N.check(N.lib().spgemm_set_option(self.ptr, option, int(value)))

    def get_option(self, option: int) -> int:
        v = C.c_int64()
        N.check(N.lib().spgemm_get_option(self.ptr, option, C.byref(v)))
        return int(v.value)

    def info(self) -> dict:
        inf = N.Info()
        N.check(N.lib().spgemm_last_info(self.ptr, C.byref(inf)))
        return {
            "nip": int(inf.nip),
            "nnz": int(inf.nnz),
            "max_row_nip": int(inf.max_row_nip),
            "max_row_nnz": int(inf.max_row_nnz),
            "sym_bin_rows": list(inf.sym_bin_rows)[: inf.n_sym_bins],
            "num_bin_rows": list(inf.num_bin_rows)[: inf.n_num_bins],
            "sym_fail_rows": int(inf.sym_fail_rows),
            "host_syncs": int(inf.host_syncs),
            "phase_us": [round(float(x), 1) for x in inf.phase_us][:7],
            "one_pass": int(inf.one_pass),
            "esc_mask": int(inf.esc_mask),
        }

    def profile(self) -> list[dict]:
        """Per-launch event-timed durations of the last product
        (requires set_option(OPT_PROFILE, 1))."""
        cnt = C.c_int32()
        N.check(N.lib().spgemm_last_profile(self.ptr, None, 0, C.byref(cnt)))
        arr = (N.KernelTime * max(cnt.value, 1))()
        N.check(N.lib().spgemm_last_profile(self.ptr, arr, cnt.value, C.byref(cnt)))
        return [{"name": k.name.decode(), "phase": k.phase, "bin": k.bin, "rows": k.rows,
                 "ms": k.ms, "start_ms": k.start_ms} for k in arr[: cnt.value]]

    def ladder(self, which: int, dtype_bytes: int = 8) -> list[int]:
        nb = C.c_int()
        lim = (C.c_int64 * 16)()
        N.check(N.lib().spgemm_ladder_info(self.ptr, which, dtype_bytes, C.byref(nb), lim))
        return list(lim)[: nb.value]


_local = threading.local()


def default_handle() -> Handle:
    """One handle per host thread (the C ABI's threading rule)."""
    h = getattr(_local, "handle", None)
    if h is None:
        h = Handle()
        _local.handle = h
    return h


class _LibraryArray:
    """A device array allocated by the library, exposed through
    __cuda_array_interface__ so torch can wrap it without a copy."""

    def __init__(self, owner: "_ResultOwner", ptr: int, n: int, typestr: str):
        self._owner = owner
        self.__cuda_array_interface__ = {
            "shape": (n,),
            "typestr": typestr,
            "data": (ptr, False),
            "version": 2,
        }


class _ResultOwner:
    """Frees a library-allocated result (spgemm_csr_free) once no tensor
    refers to it any more."""

    def __init__(self, out: N.CsrOut):
        self.out = out

    def __del__(self):
        try:
            N.lib().spgemm_csr_free(C.byref(self.out), None)
        except Exception:
            pass


@dataclass
class DeviceCSR:
    """CSR on the device: int32 rpt/col and float32/float64 val torch tensors."""

    m: int
    n: int
    rpt: "torch.Tensor"
    col: "torch.Tensor"
    val: "torch.Tensor"

    @property
    def nnz(self) -> int:
        return int(self.col.numel())

    @property
    def dtype(self):
        return self.val.dtype

    @staticmethod
    def from_host(a: HostCSR, device="cuda", pin: bool = False) -> "DeviceCSR":
        _require_torch()

        def t(x):
            ht = torch.from_numpy(np.ascontiguousarray(x))
            if pin:
                ht = ht.pin_memory()
            return ht.to(device, non_blocking=pin)

        return DeviceCSR(a.m, a.n, t(a.rpt), t(a.col), t(a.val))

    def to_host(self) -> HostCSR:
        return HostCSR(self.m, self.n, self.rpt.cpu().numpy(), self.col.cpu().numpy(),
                       self.val.cpu().numpy())

    def view(self) -> N.CsrView:
        for name, x, dt in (("rpt", self.rpt, torch.int32), ("col", self.col, torch.int32)):
            if x.dtype != dt or not x.is_cuda or not x.is_contiguous():
                raise TypeError(f"{name} must be a contiguous int32 CUDA tensor")
        if self.val.dtype not in (torch.float32, torch.float64) or not self.val.is_cuda:
            raise TypeError("val must be a float32 or float64 CUDA tensor")
        return N.CsrView(self.m, self.n, self.nnz, self.rpt.data_ptr(),
                         self.col.data_ptr() if self.nnz else None,
                         self.val.data_ptr() if self.nnz else None)


def _stream_ptr(stream) -> int | None:
    if stream is None:
        stream = torch.cuda.current_stream()
    return stream.cuda_stream or None


def proposal(A: DeviceCSR, B: DeviceCSR, handle: Handle | None = None,
             stream=None) -> DeviceCSR:
    """C = A * B on the device (reference proposal::proposal, proposal.cuh:85-124).

    A and B must share a dtype (float32 or float64), have int32 indices and
    sorted, duplicate-free columns per row.  Synchronous on return.
    """
    _require_torch()
    if A.dtype != B.dtype:
        raise TypeError("A and B must have the same value dtype")
    h = handle or default_handle()
    out = N.CsrOut()
    va, vb = A.view(), B.view()
    fn = N.lib().spgemm_csr_f64 if A.dtype == torch.float64 else N.lib().spgemm_csr_f32
    N.check(fn(h.ptr, C.byref(va), C.byref(vb), C.byref(out), _stream_ptr(stream)))
    return _wrap_result(out, A.dtype)


def _wrap_result(out: N.CsrOut, dtype) -> DeviceCSR:
    owner = _ResultOwner(out)
    dev = torch.device("cuda", torch.cuda.current_device())
    vt = "<f8" if dtype == torch.float64 else "<f4"
    rpt = torch.as_tensor(_LibraryArray(owner, out.rpt, out.m + 1, "<i4"), device=dev)
    if out.nnz > 0:
        col = torch.as_tensor(_LibraryArray(owner, out.col, out.nnz, "<i4"), device=dev)
        val = torch.as_tensor(_LibraryArray(owner, out.val, out.nnz, vt), device=dev)
    else:
        col = torch.empty(0, dtype=torch.int32, device=dev)
        val = torch.empty(0, dtype=dtype, device=dev)
    return DeviceCSR(out.m, out.n, rpt, col, val)


class _BatchOwner:
    """Frees a batch result (spgemm_batch_free) once no product view refers to it."""

    def __init__(self, out: N.BatchOut):
        self.out = out

    def __del__(self):
        try:
            N.lib().spgemm_batch_free(C.byref(self.out), None)
        except Exception:
            pass


@dataclass
class PackedBatch:
    """A batch of independent products C_i = A_i * B_i as block-diagonal CSR
    operands (global column indices) plus host offset arrays."""

    a_row_off: np.ndarray  # int32 [count + 1]
    b_row_off: np.ndarray  # int32 [count + 1]
    c_col_off: np.ndarray  # int32 [count + 1]
    A: DeviceCSR
    B: DeviceCSR

    @property
    def count(self) -> int:
        return int(self.a_row_off.shape[0] - 1)


def pack_batch(pairs, share: bool = False) -> PackedBatch:
    """Pack [(A_i, B_i)] (DeviceCSR, A_i.n == B_i.m) into block-diagonal operands
    on the operands' device (host logic plus torch ops; no library call).
    share: when every pair is one square matrix times itself, the packed B IS
    the packed A (packed once) -- only for callers that do not update the
    packed operands' values afterwards, as a plan over the batch does."""
    if torch is None:
        raise RuntimeError("torch is required")
    if not pairs:
        raise ValueError("empty batch")
    As = [a for a, _ in pairs]
    Bs = [b for _, b in pairs]
    for a, b in pairs:
        if a.n != b.m:
            raise ValueError("A_i.n must equal B_i.m")
        if a.dtype != As[0].dtype or b.dtype != As[0].dtype:
            raise TypeError("all operands must share one value dtype")
    a_row = np.concatenate([[0], np.cumsum([a.m for a in As])]).astype(np.int32)
    b_row = np.concatenate([[0], np.cumsum([b.m for b in Bs])]).astype(np.int32)
    c_col = np.concatenate([[0], np.cumsum([b.n for b in Bs])]).astype(np.int32)

    dev = As[0].rpt.device

    def pack(mats, col_shift):
        # one concatenation per array; the per-matrix offsets are expanded on
        # the device (repeat_interleave with a known output size: no host sync,
        # nothing nnz-sized on the host).  Packed sizes fit int32 (checked by
        # the caller's row/column sums and by the library).
        nnz = np.array([x.nnz for x in mats], np.int64)
        rows = np.array([x.m for x in mats], np.int64)
        tot_nnz = int(nnz.sum())
        if tot_nnz > np.iinfo(np.int32).max:
            raise ValueError("packed operand has more than 2^31-1 entries")
        small = torch.from_numpy(np.stack([np.cumsum(nnz) - nnz, col_shift[:-1].astype(np.int64),
                                           rows, nnz])).to(dev, non_blocking=True)
        rpt = torch.empty(int(rows.sum()) + 1, dtype=torch.int32, device=dev)
        torch.cat([x.rpt[:-1] for x in mats], out=rpt[:-1])
        rpt[:-1] += torch.repeat_interleave(small[0].to(torch.int32), small[2],
                                            output_size=int(rows.sum()))
        rpt[-1] = tot_nnz
        col = torch.cat([x.col for x in mats])
        col += torch.repeat_interleave(small[1].to(torch.int32), small[3], output_size=tot_nnz)
        val = torch.cat([x.val for x in mats])
        return rpt, col, val

    ar, ac, av = pack(As, b_row)
    A = DeviceCSR(int(a_row[-1]), int(b_row[-1]), ar, ac, av)
    if share and all(a is b for a, b in pairs) and np.array_equal(b_row, c_col):
        # C_i = A_i * A_i with square A_i: the packed B is the packed A (same
        # rows, same column shifts), so it is packed once
        B = A
    else:
        br, bc, bv = pack(Bs, c_col)
        B = DeviceCSR(int(b_row[-1]), int(c_col[-1]), br, bc, bv)
    return PackedBatch(a_row, b_row, c_col, A, B)


def _batch_views(out: N.BatchOut, dtype) -> list[DeviceCSR]:
    """One DeviceCSR per product, as views into the batch's device arrays.
    Products of one group lie one after another in three arrays (row
    pointers, columns, values): each run of such products is wrapped once per
    array and sliced per product -- a tensor slice costs a few microseconds,
    wrapping an array through __cuda_array_interface__ tens, which a batch of
    fifty small products paid 150 times."""
    owner = _BatchOwner(out)
    dev = torch.device("cuda", torch.cuda.current_device())
    vt = "<f8" if dtype == torch.float64 else "<f4"
    vsz = 8 if dtype == torch.float64 else 4
    P = out.products
    count = out.count
    res = []
    i = 0
    while i < count:
        first = P[i]
        # the run: row pointers back to back, and (products with entries)
        # columns and values back to back
        j = i + 1
        rlen = first.m + 1
        clen = first.nnz
        if first.nnz > 0:
            while j < count:
                a, b = P[j - 1], P[j]
                if (b.nnz == 0 or b.rpt != a.rpt + 4 * (a.m + 1) or
                        b.col != a.col + 4 * a.nnz or b.val != a.val + vsz * a.nnz):
                    break
                rlen += b.m + 1
                clen += b.nnz
                j += 1
        rpt_all = torch.as_tensor(_LibraryArray(owner, first.rpt, rlen, "<i4"), device=dev)
        if clen > 0:
            col_all = torch.as_tensor(_LibraryArray(owner, first.col, clen, "<i4"), device=dev)
            val_all = torch.as_tensor(_LibraryArray(owner, first.val, clen, vt), device=dev)
        ro = 0
        co = 0
        for k in range(i, j):
            p = P[k]
            rpt = rpt_all[ro:ro + p.m + 1]
            ro += p.m + 1
            if p.nnz > 0:
                col = col_all[co:co + p.nnz]
                val = val_all[co:co + p.nnz]
                co += p.nnz
            else:
                col = torch.empty(0, dtype=torch.int32, device=dev)
                val = torch.empty(0, dtype=dtype, device=dev)
            res.append(DeviceCSR(int(p.m), int(p.n), rpt, col, val))
        i = j
    return res


def batch(pb: PackedBatch, handle: Handle | None = None, stream=None) -> list[DeviceCSR]:
    """C_i = A_i * B_i for every product of a packed batch, run as one binned
    product of the block-diagonal operands (spgemm_batch_*).  Returns one
    DeviceCSR per product with local indices (views into shared storage)."""
    _require_torch()
    h = handle or default_handle()
    desc = N.BatchDesc(pb.count, pb.a_row_off.ctypes.data, pb.b_row_off.ctypes.data,
                       pb.c_col_off.ctypes.data)
    out = N.BatchOut()
    va, vb = pb.A.view(), pb.B.view()
    fn = N.lib().spgemm_batch_f64 if pb.A.dtype == torch.float64 else N.lib().spgemm_batch_f32
    N.check(fn(h.ptr, C.byref(desc), C.byref(va), C.byref(vb), C.byref(out),
               _stream_ptr(stream)))
    h._last_groups = int(out.n_groups)
    return _batch_views(out, pb.A.dtype)


class Plan:
    """A product (or batch) whose structure is fixed and whose values are
    recomputed on demand by replaying one CUDA graph (spgemm_plan_*).  Keeps
    its operands and result alive; update A's and B's values in place, then
    call execute()."""

    def __init__(self, ptr: C.c_void_p, keep: list, result):
        self._p = ptr
        self._keep = keep          # operands (and packed batch) the graph reads
        self.result = result       # DeviceCSR, or a list of them for a batch

    def execute(self, stream=None) -> None:
        N.check(N.lib().spgemm_plan_execute(self._p, _stream_ptr(stream)))

    def check(self, stream=None) -> None:
        N.check(N.lib().spgemm_plan_check(self._p, _stream_ptr(stream)))

    def info(self) -> dict:
        inf = N.PlanInfo()
        N.check(N.lib().spgemm_plan_get_info(self._p, C.byref(inf)))
        n = int(inf.candidates)
        return {"candidates": [{"team_scale": round(float(inf.team_scale[i]), 3),
                                "cta_scale": round(float(inf.cta_scale[i]), 3),
                                "streams": int(inf.streams[i]), "ms": float(inf.ms[i])}
                               for i in range(n)],
                "chosen": int(inf.chosen)}

    def close(self) -> None:
        if self._p:
            torch.cuda.synchronize()
            N.lib().spgemm_plan_destroy(self._p)
            self._p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def plan(A: DeviceCSR, B: DeviceCSR, tune: bool = False, handle: Handle | None = None,
         stream=None) -> Plan:
    """Plan C = A * B (spgemm_plan_csr_*): runs the product once (Plan.result)
    and captures its fill phase for replays; tune=True picks the fastest of a
    small grid of bin-routing and stream configurations."""
    _require_torch()
    if A.dtype != B.dtype:
        raise TypeError("A and B must have the same value dtype")
    h = handle or default_handle()
    out = N.CsrOut()
    p = C.c_void_p()
    va, vb = A.view(), B.view()
    fn = N.lib().spgemm_plan_csr_f64 if A.dtype == torch.float64 else N.lib().spgemm_plan_csr_f32
    N.check(fn(h.ptr, C.byref(va), C.byref(vb), 1 if tune else 0, C.byref(out), C.byref(p),
               _stream_ptr(stream)))
    return Plan(p, [A, B], _wrap_result(out, A.dtype))


def plan_batch(pb: PackedBatch, tune: bool = False, handle: Handle | None = None,
               stream=None) -> Plan:
    """Plan a packed batch (spgemm_plan_batch_*): every group's fill and split
    become one CUDA graph; Plan.result is the list of per-product results."""
    _require_torch()
    h = handle or default_handle()
    desc = N.BatchDesc(pb.count, pb.a_row_off.ctypes.data, pb.b_row_off.ctypes.data,
                       pb.c_col_off.ctypes.data)
    out = N.BatchOut()
    p = C.c_void_p()
    va, vb = pb.A.view(), pb.B.view()
    fn = (N.lib().spgemm_plan_batch_f64 if pb.A.dtype == torch.float64
          else N.lib().spgemm_plan_batch_f32)
    N.check(fn(h.ptr, C.byref(desc), C.byref(va), C.byref(vb), 1 if tune else 0, C.byref(out),
               C.byref(p), _stream_ptr(stream)))
    return Plan(p, [pb], _batch_views(out, pb.A.dtype))


def batch_groups(handle: Handle) -> int:
    """Groups the last batch on `handle` ran as (kept for reporting)."""
    return getattr(handle, "_last_groups", -1)


def _host_view(a: HostCSR) -> tuple[N.CsrView, list]:
    keep = [np.ascontiguousarray(a.rpt, dtype=np.int32),
            np.ascontiguousarray(a.col, dtype=np.int32),
            np.ascontiguousarray(a.val)]
    v = N.CsrView(a.m, a.n, a.nnz, keep[0].ctypes.data, keep[1].ctypes.data,
                  keep[2].ctypes.data)
    return v, keep


class _HostResultOwner:
    """Returns a host result's page-locked block to the library pool
    (spgemm_host_csr_free) once no array refers to it."""

    def __init__(self, out: N.CsrOut):
        self.out = out

    def __del__(self):
        try:
            N.lib().spgemm_host_csr_free(C.byref(self.out))
        except Exception:
            pass


class _HostLibraryArray:
    """Library-owned host memory exposed through __array_interface__; the numpy
    array built from it keeps it (and so the owner) alive."""

    def __init__(self, owner, ptr: int, n: int, typestr: str):
        self._owner = owner
        self.__array_interface__ = {"shape": (n,), "typestr": typestr,
                                    "data": (ptr, False), "version": 3}


def proposal_host(A: HostCSR, B: HostCSR, handle: Handle | None = None,
                  stream=None) -> HostCSR:
    """C = A * B from host operands to a host result through the C ABI's host
    entry point (copies inside the call, like the apps' convert/run/to<Host>).
    The result arrays are zero-copy views of the library's page-locked block."""
    if A.val.dtype != B.val.dtype:
        raise TypeError("A and B must have the same value dtype")
    h = handle or default_handle()
    va, ka = _host_view(A)
    vb, kb = _host_view(B)
    out = N.CsrOut()
    f64 = A.val.dtype == np.float64
    fn = N.lib().spgemm_csr_host_f64 if f64 else N.lib().spgemm_csr_host_f32
    sp = _stream_ptr(stream) if torch is not None and torch.cuda.is_available() else None
    N.check(fn(h.ptr, C.byref(va), C.byref(vb), C.byref(out), sp))
    del ka, kb
    owner = _HostResultOwner(out)
    m, n, nnz = int(out.m), int(out.n), int(out.nnz)
    rpt = np.asarray(_HostLibraryArray(owner, out.rpt, m + 1, "<i4"))
    col = np.asarray(_HostLibraryArray(owner, out.col, nnz, "<i4"))
    val = np.asarray(_HostLibraryArray(owner, out.val, nnz, "<f8" if f64 else "<f4"))
    return HostCSR(m, n, rpt, col, val)


def get_nip_many(pairs, handle: Handle | None = None, stream=None) -> list[int]:
    """NIP of many (A_i, B_i) pairs with one launch and one host sync
    (spgemm_get_nip_many); the reference sizes one pair per call
    (utils::get_nip, nip.cuh:52-78)."""
    h = handle or default_handle()
    n = len(pairs)
    if n == 0:
        return []
    va = (N.CsrView * n)(*[a.view() for a, _ in pairs])
    vb = (N.CsrView * n)(*[b.view() for _, b in pairs])
    out = (C.c_int64 * n)()
    N.check(N.lib().spgemm_get_nip_many(h.ptr, n, va, vb, out, _stream_ptr(stream)))
    return [int(x) for x in out]


def transpose(A: DeviceCSR, handle: Handle | None = None, stream=None) -> DeviceCSR:
    """A^T on the device, columns sorted (spgemm_transpose_*).  The reference
    has no transpose; its Galerkin use forms R = P^T outside the library."""
    _require_torch()
    h = handle or default_handle()
    out = N.CsrOut()
    va = A.view()
    fn = N.lib().spgemm_transpose_f64 if A.dtype == torch.float64 else \
        N.lib().spgemm_transpose_f32
    N.check(fn(h.ptr, C.byref(va), C.byref(out), _stream_ptr(stream)))
    return _wrap_result(out, A.dtype)


def rap(A: DeviceCSR, P: DeviceCSR, R: DeviceCSR | None = None, handle: Handle | None = None,
        stream=None) -> DeviceCSR:
    """Galerkin triple product C = R * (A * P) (spgemm_rap_*); R = None means
    R = P^T, transposed on the device.  Replaces two proposal calls
    (proposal.cuh:85-124) plus a caller-side transpose."""
    _require_torch()
    if A.dtype != P.dtype or (R is not None and R.dtype != A.dtype):
        raise TypeError("R, A and P must have the same value dtype")
    h = handle or default_handle()
    out = N.CsrOut()
    va, vp = A.view(), P.view()
    vr = R.view() if R is not None else None
    fn = N.lib().spgemm_rap_f64 if A.dtype == torch.float64 else N.lib().spgemm_rap_f32
    N.check(fn(h.ptr, C.byref(vr) if vr is not None else None, C.byref(va), C.byref(vp),
               C.byref(out), _stream_ptr(stream)))
    return _wrap_result(out, A.dtype)


def get_nip(A: DeviceCSR, B: DeviceCSR, handle: Handle | None = None, stream=None) -> int:
    """Total intermediate products (reference utils::get_nip, nip.cuh:52-78)."""
    h = handle or default_handle()
    v = C.c_int64()
    va, vb = A.view(), B.view()
    N.check(N.lib().spgemm_get_nip(h.ptr, C.byref(va), C.byref(vb), C.byref(v),
                                   _stream_ptr(stream)))
    return int(v.value)
