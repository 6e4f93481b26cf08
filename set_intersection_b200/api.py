"""PyTorch-facing wrappers over the C ABI (torch supplies device memory and
streams; all compute is in libsi_b200.so).

Sets are 1-D contiguous CUDA tensors of dtype int32 or uint32 holding the
uint32 bit patterns of an ascending, duplicate-free set.
"""
from __future__ import annotations

import ctypes

import torch

from ._lib import Status, Technique, check, lib

_TECH_NAMES = {
    "ip": Technique.IP,
    "obs": Technique.OBS,
    "hi": Technique.HI,
    "bitmap": Technique.BITMAP,
    "bitmap_dynamic": Technique.BITMAP,
    "bitmap_naive": Technique.BITMAP_NAIVE,
    "mm": Technique.MM,
    "auto": Technique.AUTO,
}


def technique(t) -> Technique:
    if isinstance(t, Technique):
        return t
    if isinstance(t, int):
        return Technique(t)
    try:
        return _TECH_NAMES[str(t).lower()]
    except KeyError as e:
        raise ValueError(f"unknown technique {t!r}; one of {sorted(_TECH_NAMES)}") from e


def _ptr(t: torch.Tensor | None) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr() if t is not None and t.numel() > 0 else None)


def _stream(stream: torch.cuda.Stream | None) -> ctypes.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _check_set(x: torch.Tensor, name: str) -> None:
    if x.dim() != 1 or not x.is_cuda or not x.is_contiguous():
        raise ValueError(f"{name} must be a 1-D contiguous CUDA tensor")
    if x.dtype not in (torch.int32, torch.uint32):
        raise ValueError(f"{name} must hold uint32 bit patterns (int32 or uint32 dtype)")


class Workspace:
    """Grow-only device scratch buffer reused across calls on one stream."""

    def __init__(self, device=None):
        self.device = torch.device(device if device is not None else "cuda")
        self.buf = torch.empty(0, dtype=torch.uint8, device=self.device)

    def get(self, nbytes: int) -> torch.Tensor:
        nbytes = max(int(nbytes), 256)
        if self.buf.numel() < nbytes:
            self.buf = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        return self.buf

    def check(self, stream=None) -> None:
        """Synchronises and raises if the last call recorded a device error."""
        site, detail = ctypes.c_uint32(0), ctypes.c_uint32(0)
        st = lib.si_workspace_diagnostic(_ptr(self.buf), _stream(stream), ctypes.byref(site), ctypes.byref(detail))
        check(st, f"device (site {site.value}, detail {detail.value})")


def sisi_workspace_size(n_a: int, n_b: int, tech="ip") -> int:
    return int(lib.si_sisi_workspace_size(n_a, n_b, int(technique(tech))))


def sisi_into(a: torch.Tensor, b: torch.Tensor, count: torch.Tensor, out: torch.Tensor | None,
              workspace: Workspace, tech="ip", stream=None) -> None:
    """Asynchronous single-pair call: count (int64[1]) <- |a ∩ b|, out[:count]
    <- the sorted intersection when out is given (len(out) >= min(|a|, |b|))."""
    _check_set(a, "a")
    _check_set(b, "b")
    t = technique(tech)
    n_a, n_b = a.numel(), b.numel()
    ws = workspace.get(lib.si_sisi_workspace_size(n_a, n_b, int(t)))
    cap = out.numel() if out is not None else 0
    st = lib.si_sisi(_ptr(a), n_a, _ptr(b), n_b, int(t), _ptr(count),
                     _ptr(out) if out is not None else ctypes.c_void_p(None), cap,
                     _ptr(ws), ws.numel(), _stream(stream))
    check(st, "si_sisi")


def intersect(a: torch.Tensor, b: torch.Tensor, tech="ip", materialize: bool = True,
              workspace: Workspace | None = None, stream=None):
    """|a ∩ b| and (if materialize) the sorted elements, synchronously.

    Returns (count: int, elements: int32 CUDA tensor or None)."""
    ws = workspace or Workspace(a.device)
    count = torch.zeros(1, dtype=torch.int64, device=a.device)
    out = None
    if materialize:
        out = torch.empty(max(1, min(a.numel(), b.numel())), dtype=torch.int32, device=a.device)
    sisi_into(a, b, count, out, ws, tech, stream)
    ws.check(stream)
    c = int(count.item())
    return c, (out[:c] if out is not None else None)


class HostPair:
    """What intersect_host reuses across calls: the device workspace (the
    device copies of both sets, the output and the per-range scratch) and a
    si_host_ctx (copy streams, per-range events, pinned count and error
    words), so a call allocates nothing once the workspace has grown."""

    def __init__(self, device=None):
        self.device = torch.device(device if device is not None else "cuda")
        self.ws = Workspace(self.device)
        self._ctx = ctypes.c_void_p(None)
        with torch.cuda.device(self.device):
            check(lib.si_host_ctx_create(ctypes.byref(self._ctx)), "si_host_ctx_create")

    def close(self) -> None:
        if self._ctx:
            lib.si_host_ctx_destroy(self._ctx)
            self._ctx = ctypes.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _check_host(x: torch.Tensor, name: str) -> None:
    if x.dim() != 1 or x.is_cuda or not x.is_contiguous():
        raise ValueError(f"{name} must be a 1-D contiguous CPU tensor")
    if x.dtype not in (torch.int32, torch.uint32):
        raise ValueError(f"{name} must hold uint32 bit patterns (int32 or uint32 dtype)")


def intersect_host(a_host: torch.Tensor, b_host: torch.Tensor, tech="ip", out_host: torch.Tensor | None = None,
                   ctx: HostPair | None = None, stream=None, chunks: int | None = None):
    """End-to-end single pair from HOST sets through si_sisi_host: copies a and
    b to the device, intersects, and copies the count and the sorted elements
    back, pipelined over `chunks` value ranges (None: the library's default, 8
    for pairs of 2^22 elements or more).

    a_host/b_host: 1-D int32/uint32 CPU tensors (pinned, for the copies to
    overlap).  out_host: optional int32 CPU buffer of >= min(|a|, |b|)
    elements that receives the result (a pinned one is allocated when None).
    Returns (count, host tensor view)."""
    _check_host(a_host, "a_host")
    _check_host(b_host, "b_host")
    ctx = ctx or HostPair()
    s = stream if stream is not None else torch.cuda.current_stream()
    n_a, n_b = a_host.numel(), b_host.numel()
    if out_host is None:
        out_host = torch.empty(max(min(n_a, n_b), 1), dtype=torch.int32).pin_memory()
    _check_host(out_host, "out_host")
    t = int(technique(tech))
    ch = int(chunks or 0)
    need = lib.si_sisi_host_workspace_size(a_host.data_ptr(), n_a, b_host.data_ptr(), n_b, t, ch)
    ws = ctx.ws.get(need)
    count = ctypes.c_uint64(0)
    with torch.cuda.device(ctx.device):
        st = lib.si_sisi_host_ctx(ctx._ctx, a_host.data_ptr(), n_a, b_host.data_ptr(), n_b, t, ch,
                                  ctypes.byref(count), out_host.data_ptr(), out_host.numel(), _ptr(ws), ws.numel(),
                                  _stream(s))
    check(st, "si_sisi_host_ctx")
    return int(count.value), out_host[:count.value]


class Collection:
    """A collection of sorted sets in CSR form on the device (the reference's
    Dataset after its cudaMemcpy + offset scan, e.g. src/ip.cu:129-137)."""

    def __init__(self, elements: torch.Tensor, offsets: torch.Tensor, universe: int):
        if offsets.dtype != torch.int64 or not offsets.is_cuda or not elements.is_cuda:
            raise ValueError("offsets must be an int64 CUDA tensor and elements a CUDA tensor")
        _check_set(elements, "elements")
        self.elements, self.offsets, self.universe = elements, offsets, int(universe)
        self.k = offsets.numel() - 1

    @classmethod
    def from_dataset(cls, ds, device="cuda"):
        import numpy as np
        el = torch.from_numpy(np.ascontiguousarray(ds.elements, dtype=np.uint32).view(np.int32)).to(device)
        off = torch.from_numpy(ds.offsets.astype(np.int64)).to(device)
        return cls(el, off, ds.universe)


DENSE_DTYPES = {"int8": 0, "fp8": 1, "fp8_e4m3": 1}


def n_pairs(k: int) -> int:
    return k * (k - 1) // 2


def misi_dense_into(col: Collection, counts: torch.Tensor, tech="mm", dtype="int8",
                    workspace: Workspace | None = None, stream=None) -> None:
    """Asynchronous all-pairs call: counts[tri(k, a, b)] <- |S_a ∩ S_b| for
    every a < b (counts: int32/uint32 storage, >= k(k-1)/2 elements)."""
    t = technique(tech)
    k = col.k
    if counts.numel() < n_pairs(k) or not counts.is_cuda:
        raise ValueError("counts must be a CUDA tensor of k(k-1)/2 elements")
    ws = workspace if workspace is not None else Workspace(col.elements.device)
    buf = ws.get(lib.si_misi_dense_workspace_size(k, col.universe, int(t)))
    st = lib.si_misi_dense(_ptr(col.elements), _ptr(col.offsets), k, col.universe, int(t), DENSE_DTYPES[dtype],
                           _ptr(counts), _ptr(buf), buf.numel(), _stream(stream))
    check(st, "si_misi_dense")


def misi_dense(col: Collection, tech="mm", dtype="int8", workspace: Workspace | None = None, stream=None,
               check_errors: bool = True) -> torch.Tensor:
    """uint32 counts (as int32 storage) of every pair a < b, triangular order."""
    ws = workspace or Workspace(col.elements.device)
    counts = torch.empty(max(1, n_pairs(col.k)), dtype=torch.int32, device=col.elements.device)
    misi_dense_into(col, counts, tech, dtype, ws, stream)
    if check_errors:
        ws.check(stream)
    return counts[: n_pairs(col.k)]


def _range(r, k):
    from ._lib import SetRange
    if r is None:
        return SetRange(0, k)
    return SetRange(int(r[0]), int(r[1]))


def misi_count_size(a_range, b_range, stride: int) -> int:
    """Counts written by one tile pair (triangular self-join or quadratic cross)."""
    na = a_range[1] - a_range[0]
    if tuple(a_range) == tuple(b_range):
        if na < 2:
            return 0
        i, j = na - 2, na - 1
        return stride * (stride - 1) // 2 - (stride - i) * (stride - i - 1) // 2 + j - i - 1 + 1
    nb = b_range[1] - b_range[0]
    return (na - 1) * stride + nb if na and nb else 0


def misi_into(col: Collection, counts: torch.Tensor, tech="bitmap", a_range=None, b_range=None,
              stride: int | None = None, workspace: Workspace | None = None, stream=None) -> None:
    """Asynchronous all-pairs call over one tile pair of the collection
    (default: the whole collection as one self-join tile, triangular order)."""
    t = technique(tech)
    a = _range(a_range, col.k)
    b = _range(b_range if b_range is not None else a_range, col.k)
    self_join = (a.start, a.end) == (b.start, b.end)
    if stride is None:
        stride = (a.end - a.start) if self_join else (b.end - b.start)
    need = misi_count_size((a.start, a.end), (b.start, b.end), stride)
    if counts.numel() < need or not counts.is_cuda:
        raise ValueError(f"counts must be a CUDA tensor of >= {need} elements")
    ws = workspace if workspace is not None else Workspace(col.elements.device)
    buf = ws.get(lib.si_misi_workspace_size(a, b, int(t)))
    st = lib.si_misi(_ptr(col.elements), _ptr(col.offsets), a, b, stride, int(t), _ptr(counts), _ptr(buf),
                     buf.numel(), _stream(stream))
    check(st, "si_misi")


def misi(col: Collection, tech="bitmap", a_range=None, b_range=None, stride: int | None = None,
         workspace: Workspace | None = None, stream=None, check_errors: bool = True) -> torch.Tensor:
    """Counts of one tile pair (default: all pairs a < b, triangular order).
    Techniques ip, obs, hi, bitmap, auto; mm and bitmap_naive go to the dense
    path (whole collection only)."""
    t = technique(tech)
    if t in (Technique.MM, Technique.BITMAP_NAIVE):
        if a_range is not None or b_range is not None:
            raise ValueError("dense techniques count the whole collection only")
        return misi_dense(col, tech, workspace=workspace, stream=stream, check_errors=check_errors)
    ws = workspace or Workspace(col.elements.device)
    a = (0, col.k) if a_range is None else tuple(a_range)
    b = a if b_range is None else tuple(b_range)
    if stride is None:
        stride = (a[1] - a[0]) if a == b else (b[1] - b[0])
    n = misi_count_size(a, b, stride)
    counts = torch.empty(max(1, n), dtype=torch.int32, device=col.elements.device)
    misi_into(col, counts, tech, a, b, stride, ws, stream)
    if check_errors:
        ws.check(stream)
    return counts[:n]


# Batched technique codes (the table's bytes) and the table size, as si.h.
BATCH_TABLE_SIZE = 1024
BATCH_MERGE, BATCH_SEARCH, BATCH_HASH_1024, BATCH_HASH_512, BATCH_BITMAP_16K, BATCH_BITMAP_32K = range(6)
BATCH_CODES = 6


def _table(table: bytes | None):
    if table is None:
        return None
    if len(table) != BATCH_TABLE_SIZE:
        raise ValueError(f"a batch table has {BATCH_TABLE_SIZE} bytes")
    return ctypes.create_string_buffer(bytes(table), BATCH_TABLE_SIZE)


def batch_bucket(n_a: int, n_b: int, first_l: int = 0, last_l: int = 0) -> int:
    """The table index of a pair of sizes n_a, n_b whose larger set runs from
    first_l to last_l (density class from its mean gap, as the device
    computes it)."""
    s, l = min(n_a, n_b), max(n_a, n_b)
    if l < 2:
        d = 3
    else:
        gap = ((last_l - first_l) & 0xffffffff) // (l - 1)
        d = 0 if gap < 4 else 1 if gap < 32 else 2 if gap < 256 else 3
    ls = min(15, s.bit_length() - 1) if s else 0
    lr = min(15, (l // s).bit_length() - 1) if s else 15
    return (d << 8) | (ls << 4) | lr


def batch_buckets(elements, offsets, pairs):
    """batch_bucket of every pair of a host CSR collection (numpy arrays:
    uint32 elements, int64 offsets, uint32 pairs [n, 2]): int array [n]."""
    import numpy as np
    off = np.asarray(offsets, dtype=np.int64)
    el = np.asarray(elements, dtype=np.uint32)
    sz = np.diff(off)
    p = np.asarray(pairs, dtype=np.int64)
    na, nb = sz[p[:, 0]], sz[p[:, 1]]
    s, l = np.minimum(na, nb), np.maximum(na, nb)
    larger = np.where(na >= nb, p[:, 0], p[:, 1])
    if el.size:
        first = el[np.minimum(off[larger], el.size - 1)].astype(np.int64)
        last = el[np.clip(off[larger + 1] - 1, 0, el.size - 1)].astype(np.int64)
    else:
        first = last = np.zeros(len(p), np.int64)
    gap = ((last - first) & 0xffffffff) // np.maximum(l - 1, 1)
    d = np.where(l < 2, 3, np.where(gap < 4, 0, np.where(gap < 32, 1, np.where(gap < 256, 2, 3))))
    log2 = lambda x: np.frexp(np.maximum(x, 1).astype(np.float64))[1].astype(np.int64) - 1  # exact floor(log2)
    ls = np.where(s > 0, np.minimum(15, log2(s)), 0)
    lr = np.where(s > 0, np.minimum(15, log2(l // np.maximum(s, 1))), 15)
    return (d << 8) | (ls << 4) | lr


def _pairs(pairs: torch.Tensor) -> int:
    if not pairs.is_cuda or pairs.dtype not in (torch.int32, torch.uint32) or not pairs.is_contiguous() or \
            pairs.dim() != 2 or pairs.shape[1] != 2:
        raise ValueError("pairs must be a contiguous CUDA int32/uint32 tensor of shape [n, 2]")
    return pairs.shape[0]


def batch_count_into(col: Collection, pairs: torch.Tensor, counts: torch.Tensor, tech="auto",
                     table: bytes | None = None, workspace: Workspace | None = None, stream=None) -> None:
    """Asynchronous batched call: counts[p] <- |S_a ∩ S_b| for pair p = pairs[p]
    (tech: "ip" = merge, "obs" = search, "hi" = hash, "bitmap" = window
    bitmaps for every pair; "auto" = per bucket from `table`, the
    BATCH_TABLE_SIZE-byte output of batch_tune, or the default rule)."""
    n = _pairs(pairs)
    if counts.numel() < n or not counts.is_cuda:
        raise ValueError("counts must be a CUDA tensor of len(pairs) elements")
    ws = workspace if workspace is not None else Workspace(col.elements.device)
    buf = ws.get(lib.si_batch_workspace_size(n))
    tb = _table(table)
    st = lib.si_batch_count(_ptr(col.elements), _ptr(col.offsets), col.k, _ptr(pairs), n, int(technique(tech)),
                            tb, _ptr(counts), _ptr(buf), buf.numel(), _stream(stream))
    check(st, "si_batch_count")


def batch_count(col: Collection, pairs: torch.Tensor, tech="auto", table: bytes | None = None,
                workspace: Workspace | None = None, stream=None, check_errors: bool = True) -> torch.Tensor:
    ws = workspace or Workspace(col.elements.device)
    counts = torch.empty(max(1, _pairs(pairs)), dtype=torch.int32, device=col.elements.device)
    batch_count_into(col, pairs, counts, tech, table, ws, stream)
    if check_errors:
        ws.check(stream)
    return counts[:pairs.shape[0]]


def batch_tune(col: Collection, pairs: torch.Tensor, sample: int = 4096, workspace: Workspace | None = None,
               stream=None) -> bytes:
    """Times every batched technique per (density, size, ratio) bucket of
    this batch; returns the BATCH_TABLE_SIZE-byte technique table for
    batch_count(..., "auto", table)."""
    n = _pairs(pairs)
    ws = workspace or Workspace(col.elements.device)
    buf = ws.get(lib.si_batch_workspace_size(n))
    counts = torch.empty(max(1, n), dtype=torch.int32, device=col.elements.device)
    out = ctypes.create_string_buffer(BATCH_TABLE_SIZE)
    st = lib.si_batch_tune(_ptr(col.elements), _ptr(col.offsets), col.k, _ptr(pairs), n, sample, _ptr(counts),
                           _ptr(buf), buf.numel(), _stream(stream), out)
    check(st, "si_batch_tune")
    ws.check(stream)
    return out.raw


class BatchGraph:
    """A batched call captured once into a CUDA graph and replayed by launch()."""

    def __init__(self, col: Collection, pairs: torch.Tensor, counts: torch.Tensor, tech="auto",
                 table: bytes | None = None, workspace: Workspace | None = None):
        n = _pairs(pairs)
        self.ws = workspace or Workspace(col.elements.device)
        self.buf = self.ws.get(lib.si_batch_workspace_size(n))
        self._keep = (col, pairs, counts)  # the graph holds their addresses
        tb = _table(table)
        h = ctypes.c_void_p()
        st = lib.si_batch_graph_create(_ptr(col.elements), _ptr(col.offsets), col.k, _ptr(pairs), n,
                                       int(technique(tech)), tb, _ptr(counts), _ptr(self.buf), self.buf.numel(),
                                       ctypes.byref(h))
        check(st, "si_batch_graph_create")
        self.handle = h

    def launch(self, stream=None) -> None:
        check(lib.si_batch_graph_launch(self.handle, _stream(stream)), "si_batch_graph_launch")

    def check(self, stream=None) -> None:
        self.ws.check(stream)

    def close(self) -> None:
        if self.handle:
            lib.si_batch_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def degree_stats(col: Collection, slots: int, workspace: Workspace | None = None, stream=None,
                 check_errors: bool = True):
    """The degree_cdf tool's per-value and per-set figures on the device:
    (inv, set_sum), inv[v] = number of sets holding v for v < slots (int32
    holding uint32), set_sum[s] = sum of inv over set s's values (int64)."""
    ws = workspace or Workspace(col.elements.device)
    buf = ws.get(lib.si_degree_stats_workspace_size())
    dev = col.elements.device
    inv = torch.empty(max(1, slots), dtype=torch.int32, device=dev)
    set_sum = torch.empty(max(1, col.k), dtype=torch.int64, device=dev)
    n = col.offsets.numel() and int(col.offsets[-1].item())
    st = lib.si_degree_stats(_ptr(col.elements), _ptr(col.offsets), col.k, n, slots, _ptr(inv), _ptr(set_sum),
                             _ptr(buf), buf.numel(), _stream(stream))
    check(st, "si_degree_stats")
    if check_errors:
        ws.check(stream)
    return inv[:slots], set_sum[:col.k]


class HostCollection:
    """Device buffers and workspace reused by misi_dense_host across calls."""

    def __init__(self, device=None):
        self.device = torch.device(device if device is not None else "cuda")
        self.ws = Workspace(self.device)
        self.el = self.off = self.counts = None

    def _fit(self, buf, n, dtype):
        if buf is None or buf.numel() < n:
            buf = torch.empty(max(n, 1), dtype=dtype, device=self.device)
        return buf


def misi_dense_host(elements_host: torch.Tensor, offsets_host: torch.Tensor, universe: int, tech="mm",
                    dtype="int8", counts_host: torch.Tensor | None = None, ctx: HostCollection | None = None,
                    stream=None) -> torch.Tensor:
    """End-to-end all pairs from a HOST collection (CSR: int32/uint32
    elements, int64 offsets[k+1], pinned for asynchronous copies): copies it to
    the device, counts every pair, copies the counts back into counts_host
    (pinned int32[k(k-1)/2]) and returns them."""
    ctx = ctx or HostCollection()
    s = stream if stream is not None else torch.cuda.current_stream()
    k = offsets_host.numel() - 1
    n = elements_host.numel()
    ctx.el = ctx._fit(ctx.el, n, torch.int32)
    ctx.off = ctx._fit(ctx.off, k + 1, torch.int64)
    ctx.counts = ctx._fit(ctx.counts, n_pairs(k), torch.int32)
    if counts_host is None:
        counts_host = torch.empty(max(1, n_pairs(k)), dtype=torch.int32).pin_memory()
    dense = technique(tech) in (Technique.MM, Technique.BITMAP_NAIVE)
    with torch.cuda.stream(s):
        ctx.el[:n].copy_(elements_host.view(torch.int32), non_blocking=True)
        ctx.off[:k + 1].copy_(offsets_host, non_blocking=True)
        col = Collection(ctx.el[:n], ctx.off[:k + 1], universe)
        if dense:
            misi_dense_into(col, ctx.counts, tech, dtype, ctx.ws, s)
        else:
            misi_into(col, ctx.counts, tech, workspace=ctx.ws, stream=s)
        counts_host[:n_pairs(k)].copy_(ctx.counts[:n_pairs(k)], non_blocking=True)
    ctx.ws.check(s)
    return counts_host[:n_pairs(k)]


def misi_host(elements_host: torch.Tensor, offsets_host: torch.Tensor, universe: int, tech="bitmap",
              counts_host: torch.Tensor | None = None, ctx: HostCollection | None = None, stream=None):
    """End-to-end all pairs of a HOST collection with any technique (dense
    ones included): H2D, count every pair a < b, D2H of the counts."""
    return misi_dense_host(elements_host, offsets_host, universe, tech, "int8", counts_host, ctx, stream)


def validate_sorted(x: torch.Tensor, stream=None) -> bool:
    _check_set(x, "x")
    flag = torch.zeros(1, dtype=torch.int32, device=x.device)
    check(lib.si_validate_sorted(_ptr(x), x.numel(), _ptr(flag), _stream(stream)), "si_validate_sorted")
    return bool(flag.item())


def status_string(s: int) -> str:
    return lib.si_status_string(int(s)).decode()


__all__ = ["Status", "Technique", "Workspace", "HostPair", "Collection", "HostCollection", "misi", "misi_into", "misi_dense", "misi_dense_into",
           "misi_dense_host", "misi_host", "batch_count", "batch_count_into",
           "batch_tune", "BatchGraph", "intersect", "intersect_host",
           "sisi_into",
           "sisi_workspace_size",
           "technique", "validate_sorted", "status_string"]
