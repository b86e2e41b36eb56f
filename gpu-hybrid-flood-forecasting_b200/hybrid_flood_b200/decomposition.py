"""One domain split into row strips: across GPUs over NCCL, or all in one process.

The reference runs one domain on one device.  A domain too large for one GPU's
step rate is cut into contiguous row strips (rows = y, northward); a strip owns
its rows and also holds the row below and the row above it (halo rows).  Every
step of the whole domain is, per strip: the step over the owned rows, the CFL
maximum over all strips (an NCCL all-reduce of one float), the same dt planned
from it on every strip, and the exchange of the new first and last owned rows
with the neighbours (NCCL point-to-point).  Because each owned cell sees exactly
the neighbours it sees in the whole domain and every strip steps with the
domain-wide dt, the result equals the undivided run bit for bit.

:class:`StripSet` runs all strips of a domain in one process on one GPU (the
maximum is a kernel, the exchange device-to-device copies): the strip kernels
and the exchange pattern can be checked against the undivided run on a single
GPU.  :class:`NcclStrip` is one strip per process and GPU.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .ensemble import _desc
from .solver import LEDGER_KEYS, SWEState, _ptr, _stream


def row_ranges(rows: int, parts: int) -> list[tuple[int, int]]:
    """Contiguous owned row ranges, bottom to top, sizes differing by at most one."""
    if parts < 1 or parts > rows:
        raise ValueError(f"cannot split {rows} rows into {parts} strips")
    base, extra = divmod(rows, parts)
    out, lo = [], 0
    for i in range(parts):
        hi = lo + base + (1 if i < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


def local_rows(rows: int, lo: int, hi: int) -> tuple[int, int]:
    """Global rows [first, last) a strip owning [lo, hi) holds, halo rows included."""
    return (lo - 1 if lo > 0 else 0), (hi + 1 if hi < rows else hi)


def split_state(state, rows: int, ranges) -> list[SWEState]:
    """Per-strip local copies (halo rows included) of a global state."""
    out = []
    for lo, hi in ranges:
        a, b = local_rows(rows, lo, hi)
        out.append(SWEState(*(t[a:b].contiguous().clone() for t in state)))
    return out


def join_state(local_states, rows: int, ranges) -> SWEState:
    """The global state from the strips' owned rows."""
    parts = [[], [], []]
    for st, (lo, hi) in zip(local_states, ranges):
        a, _ = local_rows(rows, lo, hi)
        for q in range(3):
            parts[q].append(st[q][lo - a:hi - a])
    return SWEState(*(torch.cat(p) for p in parts))


def _check_local(states, shapes, device) -> None:
    for st, shape in zip(states, shapes):
        for t in st:
            if not (isinstance(t, torch.Tensor) and t.device == device and t.dtype == torch.float32
                    and tuple(t.shape) == shape and t.stride(-1) == 1):
                raise ValueError(f"strip states must be device float32 {shape} tensors with unit column stride")


def agree_on_errors(err: Exception | None, world: int, group=None, device=None) -> None:
    """Raise on every rank of ``group`` if any rank's local check failed.

    Each rank passes the exception its own checks raised (or ``None``); one
    all-reduce (max) of a flag tells every rank whether any of them failed, so
    either all ranks go on into the collective steps or none does.  The failing
    rank re-raises its own exception, the others a ``ValueError`` naming that
    another rank failed.
    """
    import torch.distributed as dist

    if world > 1:
        flag = torch.tensor([1 if err is not None else 0], dtype=torch.int32)
        if dist.get_backend(group) == "nccl":
            flag = flag.to(device)
        dist.all_reduce(flag, op=dist.ReduceOp.MAX, group=group)
        if int(flag.item()) and err is None:
            raise ValueError("another rank's strip arguments are invalid")
    if err is not None:
        raise err


def _results(res) -> list[tuple]:
    return [(float(r.final_time_s), int(r.steps_used), dict(zip(LEDGER_KEYS, list(r.ledger)))) for r in res]


class _StripBase:
    def _make(self, member: dict, arithmetic: str, lo: int, hi: int):
        keep: list = []
        desc = _desc(member, arithmetic, keep)
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self._lib.swe_strip_create(ctypes.byref(desc), int(lo), int(hi), ctypes.byref(handle)),
                       "swe_strip_create")
        return handle

    def _destroy(self, handles) -> None:
        for h in handles:
            if h is not None and h.value:
                try:
                    self._lib.swe_domain_destroy(h)
                except Exception:  # noqa: BLE001 - interpreter shutdown
                    pass


class StripSet(_StripBase):
    """All row strips of one domain in this process, on one GPU.

    ``member`` holds the :class:`B200ShallowWaterSolver` keyword arguments
    (``bed``, ``manning_n``, ``domain_mask``, ``resolution_m``, ...).
    """

    def __init__(self, member: dict, parts: int, *, arithmetic: str = "fast", device=None) -> None:
        if not torch.cuda.is_available():
            raise RuntimeError("StripSet needs a CUDA device (sm_100a); none is visible.")
        self._lib = _lib.load()
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.rows, self.cols = np.asarray(member["bed"]).shape
        self.ranges = row_ranges(self.rows, parts)
        self._handles = [self._make(member, arithmetic, lo, hi) for lo, hi in self.ranges]
        self.shapes = []
        for lo, hi in self.ranges:
            a, b = local_rows(self.rows, lo, hi)
            self.shapes.append((b - a, self.cols))

    def __del__(self):
        self._destroy(getattr(self, "_handles", []))

    def split(self, state) -> list[SWEState]:
        return split_state(SWEState(*state), self.rows, self.ranges)

    def join(self, local_states) -> SWEState:
        return join_state(local_states, self.rows, self.ranges)

    def advance_(self, local_states, n_steps: int, start_time_s: float = 0.0) -> list[tuple]:
        """``n_steps`` domain-wide steps IN PLACE; per strip ``(final_time_s, steps, ledger of its rows)``."""
        n = len(self._handles)
        if len(local_states) != n:
            raise ValueError(f"expected {n} strip states")
        _check_local(local_states, self.shapes, self.device)
        arr = lambda typ, vals: (typ * n)(*vals)  # noqa: E731
        res = (_lib.RunResult * n)()
        with torch.cuda.device(self.device):
            rc = self._lib.swe_strips_advance(
                arr(ctypes.c_void_p, [h.value for h in self._handles]), n,
                arr(ctypes.c_void_p, [s.h.data_ptr() for s in local_states]),
                arr(ctypes.c_void_p, [s.hu.data_ptr() for s in local_states]),
                arr(ctypes.c_void_p, [s.hv.data_ptr() for s in local_states]),
                arr(ctypes.c_int64, [int(s.h.stride(0)) for s in local_states]), int(n_steps), float(start_time_s),
                res, _stream(self.device))
        _lib.check(rc, "swe_strips_advance")
        return _results(res)


class NcclStrip(_StripBase):
    """This rank's row strip of one domain, one process per GPU, stepping over NCCL.

    Needs an initialised ``torch.distributed`` group (any backend) only to hand
    the NCCL id to every rank; the steps use their own NCCL communicator.
    """

    def __init__(self, member: dict, *, rank: int, world: int, arithmetic: str = "fast", device=None,
                 group=None) -> None:
        import torch.distributed as dist

        self._lib = _lib.load()
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.rows, self.cols = np.asarray(member["bed"]).shape
        self.rank, self.world = int(rank), int(world)
        self._group = group
        self.ranges = row_ranges(self.rows, self.world)
        lo, hi = self.ranges[self.rank]
        self._handle = self._make(member, arithmetic, lo, hi)
        a, b = local_rows(self.rows, lo, hi)
        self.shape = (b - a, self.cols)
        self.below = self.rank - 1 if lo > 0 else -1
        self.above = self.rank + 1 if hi < self.rows else -1
        uid = ctypes.create_string_buffer(_lib.SWE_COMM_ID_BYTES)
        if self.rank == 0:
            _lib.check(self._lib.swe_comm_unique_id(uid), "swe_comm_unique_id")
        if self.world > 1:
            box = [bytes(uid.raw)]
            dist.broadcast_object_list(box, src=0, group=group)
            uid = ctypes.create_string_buffer(box[0], _lib.SWE_COMM_ID_BYTES)
        comm = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self._lib.swe_comm_create(uid, self.world, self.rank, ctypes.byref(comm)), "swe_comm_create")
        self._comm = comm

    def __del__(self):
        c = getattr(self, "_comm", None)
        if c is not None and c.value:
            try:
                self._lib.swe_comm_destroy(c)
            except Exception:  # noqa: BLE001 - interpreter shutdown
                pass
        self._destroy([getattr(self, "_handle", None)])

    def local_state(self, state) -> SWEState:
        return split_state(SWEState(*state), self.rows, [self.ranges[self.rank]])[0]

    def advance_(self, local_state, n_steps: int, start_time_s: float = 0.0) -> tuple:
        """``n_steps`` domain-wide steps of this rank's strip IN PLACE.

        Every rank must call it with the same ``n_steps`` and ``start_time_s``.
        The ranks first agree over the ``torch.distributed`` group that every
        one of them has valid arguments (a rank whose check fails still takes
        part in that agreement), so no rank enters the NCCL steps while another
        has left; the library then agrees once more on its own set-up and
        bounds every later wait (``SWE_NCCL_TIMEOUT_S``).
        """
        err = None
        try:
            _check_local([local_state], [self.shape], self.device)
        except ValueError as e:
            err = e
        agree_on_errors(err, self.world, self._group, self.device)
        res = _lib.RunResult()
        with torch.cuda.device(self.device):
            rc = self._lib.swe_strip_advance_nccl(
                self._handle, self._comm, self.below, self.above, _ptr(local_state.h), _ptr(local_state.hu),
                _ptr(local_state.hv), int(local_state.h.stride(0)), int(n_steps), float(start_time_s),
                ctypes.byref(res), _stream(self.device))
        _lib.check(rc, "swe_strip_advance_nccl")
        return _results([res])[0]
