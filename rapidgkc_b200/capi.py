"""ctypes binding of librapidgkc_b200.so (include/gkc_capi.h).

The Python mirror of the reference's GPU interface:

* ``KmerCounter.add_reads``  <- ``GenSuperkmerGPU`` (gpu_skmgen.h:54-58)
* ``KmerCounter.count``      <- ``kmc_counting_GPU_streams`` (gpu_kmercounting.h:14-17)
* ``KmerCounter.store_stats`` / ``store_export`` <- ``SKMStoreNoncon`` counters
  and bytes (skmstore.hpp:85-87, 222-236)

There is no CPU fallback: constructing a counter without the CUDA library, or
without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "librapidgkc_b200.so")

GKC_OK, GKC_EINVAL, GKC_ECUDA, GKC_ENOMEM, GKC_ESTATE, GKC_EINTERNAL, GKC_ELIMIT = 0, -1, -2, -3, -4, -5, -6
COUNTER_SORT, COUNTER_HASH = 0, 1
MEM_HOST, MEM_DEVICE = 0, 1
FORMATS = {"fastq": 0, "fasta": 1}
UINT32_MAX = 0xFFFFFFFF

# Every symbol declared in include/gkc_capi.h.
EXPORTS = (
    "gkc_default_options", "gkc_create", "gkc_destroy", "gkc_last_error", "gkc_strerror",
    "gkc_set_order", "gkc_add_reads", "gkc_add_reads_batches", "gkc_batch_timings", "gkc_store_stats", "gkc_store_export", "gkc_store_clear",
    "gkc_reserve_host", "gkc_store_pack", "gkc_store_append", "gkc_add_fastx", "gkc_parse_fastx", "gkc_add_skm",
    "gkc_count", "gkc_count_partitions", "gkc_result", "gkc_result_device", "gkc_count_reads", "gkc_count_keys",
    "gkc_last_timings", "gkc_kernel_launches", "gkc_set_stream", "gkc_set_profiling", "gkc_kernel_stats",
    "gkc_mlp_param_count", "gkc_minimizer_loads", "gkc_mlp_grad", "gkc_mlp_train", "gkc_mlp_scores",
    "gkc_mlp_order", "gkc_count_keys_noalloc", "gkc_pack_bases",
    "gkc_init", "gkc_skmgen_batch", "gkc_count_partition", "gkc_set_order_lut", "gkc_shutdown",
)
KERNEL_CLASSES = ("find_superkmers", "scatter_superkmers", "hash_insert", "hash_collect", "sort_extract",
                  "radix_hist", "radix_scatter", "scan", "rle", "bucket_split", "hash_records")


class Options(C.Structure):
    _fields_ = [
        ("k", C.c_int),
        ("p", C.c_int),
        ("partitions", C.c_int),
        ("counter", C.c_int),
        ("radix_bits", C.c_int),
        ("table_slots", C.c_double),
        ("batch_bases", C.c_uint64),
        ("spill_host", C.c_int),
        ("group_keys", C.c_uint64),
        ("hash_l2_only", C.c_int),
        ("hpc", C.c_int),
        ("sort_seg_max", C.c_uint64),
    ]


class GkcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"gkc error {code}: {msg}")
        self.code = code


_lib = None


def load_library(path: str = LIB_PATH):
    """Loads the CUDA library; raises if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with `python -m rapidgkc_b200.build`")
    L = C.CDLL(path)
    vp, u64, u32, i32 = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int
    L.gkc_default_options.argtypes = [C.POINTER(Options)]
    L.gkc_default_options.restype = None
    L.gkc_create.argtypes = [i32, C.POINTER(Options), C.POINTER(vp)]
    L.gkc_destroy.argtypes = [vp]
    L.gkc_last_error.argtypes = [vp]
    L.gkc_last_error.restype = C.c_char_p
    L.gkc_strerror.argtypes = [i32]
    L.gkc_strerror.restype = C.c_char_p
    L.gkc_set_order.argtypes = [vp, vp, u64, i32]
    L.gkc_add_reads.argtypes = [vp, vp, vp, u64, i32]
    L.gkc_add_reads_batches.argtypes = [vp, vp, vp, u64, vp, u64]
    L.gkc_batch_timings.argtypes = [vp, vp, u64, C.POINTER(u64)]
    L.gkc_store_stats.argtypes = [vp, vp, vp, vp]
    L.gkc_store_export.argtypes = [vp, i32, vp, u64, C.POINTER(u64)]
    L.gkc_store_clear.argtypes = [vp]
    L.gkc_reserve_host.argtypes = [vp, u64, C.POINTER(u64)]
    L.gkc_store_pack.argtypes = [vp, i32, i32, vp, u64, vp, vp, u64, vp]
    L.gkc_store_append.argtypes = [vp, i32, i32, vp, vp, vp, vp]
    L.gkc_add_skm.argtypes = [vp, vp, vp, i32]
    L.gkc_add_fastx.argtypes = [vp, vp, u64, i32, i32, C.POINTER(i32), C.POINTER(u64), C.POINTER(u64)]
    L.gkc_parse_fastx.argtypes = [vp, vp, u64, i32, i32, C.POINTER(i32), vp, u64, vp, u64, i32, C.POINTER(u64),
                                  C.POINTER(u64)]
    L.gkc_count.argtypes = [vp, u32, u32, C.POINTER(u64), C.POINTER(u64)]
    L.gkc_count_partitions.argtypes = [vp, vp, u64, u32, u32, C.POINTER(u64), C.POINTER(u64)]
    L.gkc_result.argtypes = [vp, vp, vp, u64, i32]
    L.gkc_result_device.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(u64)]
    L.gkc_count_reads.argtypes = [vp, vp, vp, u64, i32, u32, u32, vp, vp, u64, i32, C.POINTER(u64),
                                  C.POINTER(u64)]
    L.gkc_count_keys.argtypes = [vp, vp, u64, i32, u32, u32, C.POINTER(u64), C.POINTER(u64)]
    L.gkc_last_timings.argtypes = [vp, C.POINTER(C.c_double), i32]
    L.gkc_kernel_launches.argtypes = [vp]
    L.gkc_kernel_launches.restype = u64
    L.gkc_set_stream.argtypes = [vp, vp]
    L.gkc_set_profiling.argtypes = [vp, i32]
    L.gkc_kernel_stats.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(u64), C.POINTER(C.c_double), i32, i32]
    f32 = C.c_float
    L.gkc_mlp_param_count.argtypes = [i32]
    L.gkc_mlp_param_count.restype = u64
    L.gkc_minimizer_loads.argtypes = [vp, vp, u64, i32]
    L.gkc_mlp_grad.argtypes = [vp, vp, vp, u64, vp, vp, f32, vp, C.POINTER(f32)]
    L.gkc_mlp_train.argtypes = [vp, vp, vp, vp, i32, i32, f32, u64, C.POINTER(f32)]
    L.gkc_mlp_scores.argtypes = [vp, vp, vp, i32]
    L.gkc_mlp_order.argtypes = [vp, vp, u64, vp]
    L.gkc_count_keys_noalloc.argtypes = [vp, u64, u32, u32, vp, vp, u64, C.POINTER(u64), C.POINTER(u64), vp]
    L.gkc_pack_bases.argtypes = [vp, u64, vp]
    L.gkc_init.argtypes = [i32, C.POINTER(Options), C.POINTER(vp)]
    L.gkc_skmgen_batch.argtypes = [vp, vp, vp, u64, i32, i32, i32, vp, i32, vp, vp, vp]
    L.gkc_count_partition.argtypes = [vp, i32, u32, u32, vp, vp, u64, i32, C.POINTER(u64), C.POINTER(u64)]
    L.gkc_set_order_lut.argtypes = [vp, vp]
    L.gkc_shutdown.argtypes = [vp]
    for name in EXPORTS:
        if name not in ("gkc_default_options", "gkc_last_error", "gkc_strerror", "gkc_kernel_launches",
                        "gkc_mlp_param_count"):
            getattr(L, name).restype = i32
    _lib = L
    return L


def _ptr(a):
    """(pointer, mem) of a numpy array (host) or a CUDA torch tensor (device)."""
    if a is None:
        return None, MEM_HOST
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return a.ctypes.data_as(C.c_void_p), MEM_HOST
    if hasattr(a, "data_ptr") and hasattr(a, "is_cuda"):
        if not a.is_contiguous():
            raise ValueError("tensors must be contiguous")
        return C.c_void_p(a.data_ptr()), MEM_DEVICE if a.is_cuda else MEM_HOST
    raise TypeError(f"unsupported buffer type {type(a)!r}")


def pack_bases(bases) -> np.ndarray:
    """ASCII bases (a uint8 array or bytes) -> uint32 words of 16 2-bit codes,
    first base highest, with the device's base map (gkc_pack_bases; host
    memory, the library's host threads)."""
    b = np.frombuffer(bases, np.uint8) if isinstance(bases, (bytes, bytearray)) else np.ascontiguousarray(bases,
                                                                                                        np.uint8)
    out = np.zeros(max(1, (len(b) + 15) // 16), np.uint32)
    rc = load_library().gkc_pack_bases(b.ctypes.data if len(b) else None, len(b), out.ctypes.data)
    if rc != 0:
        raise GkcError(rc, "gkc_pack_bases")
    return out[:(len(b) + 15) // 16]


class KmerCounter:
    """A counting context on one CUDA device (reference CLI names in brackets):
    k [-k], p [-p], partitions [-skm], counter 'hash' or 'sort'.

    k <= 32 gives uint64 k-mers.  32 < k <= 64 (the reference's 128-bit
    LONGERKMER build) gives k-mers as (n, 2) uint64 arrays of (low word, high
    word); the sort counter orders them as 128-bit values within a partition,
    the hash counter leaves them unordered, as it does for k <= 32."""

    def __init__(self, k: int = 31, p: int = 11, partitions: int = 512, counter: str = "hash",
                 device: int = 0, radix_bits: int = 0, table_slots: float = 0.35,
                 batch_bases: int = 1 << 30, spill_host: bool = False, group_keys: int = 0,
                 hash_l2_only: bool = False, hpc: bool = False, sort_seg_max: int = 0):
        L = load_library()
        o = Options()
        L.gkc_default_options(C.byref(o))
        o.k, o.p, o.partitions = k, p, partitions
        o.counter = {"hash": COUNTER_HASH, "sort": COUNTER_SORT}[counter]
        default_bits = o.radix_bits
        o.radix_bits, o.table_slots, o.batch_bases = radix_bits, table_slots, batch_bases
        o.spill_host, o.group_keys, o.hash_l2_only = int(spill_host), group_keys, int(hash_l2_only)
        o.hpc = int(hpc)
        o.sort_seg_max = sort_seg_max
        h = C.c_void_p()
        rc = L.gkc_create(device, C.byref(o), C.byref(h))
        if rc != GKC_OK:
            raise GkcError(rc, L.gkc_strerror(rc).decode())
        self._L, self._h = L, h
        self.k, self.p, self.partitions, self.counter = k, p, partitions, counter
        self.radix_bits = radix_bits or default_bits  # the sort counter's digit width
        self.device = device
        self._kw = 1  # u64 words per k-mer of the last result

    def close(self):
        if getattr(self, "_h", None):
            self._L.gkc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc != GKC_OK:
            raise GkcError(rc, self._L.gkc_last_error(self._h).decode())

    # -- phase 1 -------------------------------------------------------------
    def set_order(self, lut):
        """Minimizer order table of 4^p uint32 ranks, or None for the default."""
        if lut is None:
            self._check(self._L.gkc_set_order(self._h, None, 0, MEM_HOST))
            return
        ptr, mem = _ptr(lut)
        self._check(self._L.gkc_set_order(self._h, ptr, len(lut), mem))

    def add_reads(self, reads, offs):
        """Appends the superkmers of a CSR read batch to the partition store."""
        rp, rm = _ptr(reads)
        op, om = _ptr(offs)
        if rm != om:
            raise ValueError("reads and offsets must live in the same memory")
        self._check(self._L.gkc_add_reads(self._h, rp, op, len(offs) - 1, rm))

    def add_reads_batches(self, reads, offs, batch_reads):
        """Phase 1 over host reads in caller-chosen (uneven) batches of reads."""
        reads = np.ascontiguousarray(reads)
        offs = np.ascontiguousarray(offs, np.uint64)
        br = np.ascontiguousarray(batch_reads, np.uint64)
        self._check(self._L.gkc_add_reads_batches(self._h, _ptr(reads)[0], _ptr(offs)[0], len(offs) - 1,
                                                  _ptr(br)[0], len(br)))

    def batch_timings(self) -> np.ndarray:
        """Latency (ms) of each batch of the last add_reads call."""
        n = C.c_uint64(0)
        self._check(self._L.gkc_batch_timings(self._h, None, 0, C.byref(n)))
        out = np.zeros(n.value, np.float64)
        self._check(self._L.gkc_batch_timings(self._h, _ptr(out)[0], len(out), C.byref(n)))
        return out

    def store_stats(self):
        P = self.partitions
        b, s, k = (np.zeros(P, np.uint64) for _ in range(3))
        self._check(self._L.gkc_store_stats(self._h, _ptr(b)[0], _ptr(s)[0], _ptr(k)[0]))
        return b, s, k

    def store_export(self, part: int) -> np.ndarray:
        n = C.c_uint64(0)
        self._check(self._L.gkc_store_export(self._h, part, None, 0, C.byref(n)))
        out = np.zeros(max(1, n.value), np.uint8)
        self._check(self._L.gkc_store_export(self._h, part, _ptr(out)[0], n.value, C.byref(n)))
        return out[: n.value]

    def store_clear(self):
        self._check(self._L.gkc_store_clear(self._h))

    def add_skm(self, data, part_off):
        """Appends superkmers in the reference's .skm byte format: partition p
        is data[part_off[p]:part_off[p+1]] (uint8 array or CUDA tensor)."""
        po = np.ascontiguousarray(np.asarray(part_off, np.uint64))
        if len(po) != self.partitions + 1:
            raise ValueError(f"part_off needs {self.partitions + 1} entries")
        if isinstance(data, (bytes, bytearray)):
            data = np.frombuffer(bytes(data), np.uint8)
        dp, dm = _ptr(data)
        self._check(self._L.gkc_add_skm(self._h, dp, _ptr(po)[0], dm))

    def add_fastx(self, text, fmt: str = "fastq", state: int = 0):
        """Phase 1 from FASTQ / FASTA text (bytes, a uint8 array or a CUDA
        tensor), scanned on the GPU.  Returns (reads, bases, state): state is
        the FASTQ line phase at the text's end, to pass with the next piece."""
        if isinstance(text, (bytes, bytearray)):
            text = np.frombuffer(bytes(text), np.uint8)
        tp, tm = _ptr(text)
        st, nr, nb = C.c_int32(state), C.c_uint64(0), C.c_uint64(0)
        n = text.numel() if hasattr(text, "numel") else len(text)
        self._check(self._L.gkc_add_fastx(self._h, tp, n, tm, FORMATS[fmt], C.byref(st), C.byref(nr), C.byref(nb)))
        return nr.value, nb.value, st.value

    def parse_fastx(self, text, fmt: str = "fastq", state: int = 0):
        """The GPU scan alone: (reads uint8, offs uint64, state) on the host."""
        if isinstance(text, (bytes, bytearray)):
            text = np.frombuffer(bytes(text), np.uint8)
        tp, tm = _ptr(text)
        n = text.numel() if hasattr(text, "numel") else len(text)
        st, nr, nb = C.c_int32(state), C.c_uint64(0), C.c_uint64(0)
        self._check(self._L.gkc_parse_fastx(self._h, tp, n, tm, FORMATS[fmt], C.byref(st), None, 0, None, 0,
                                            MEM_HOST, C.byref(nr), C.byref(nb)))
        reads = np.zeros(max(nb.value, 1), np.uint8)
        offs = np.zeros(nr.value + 1, np.uint64)
        st = C.c_int32(state)
        self._check(self._L.gkc_parse_fastx(self._h, tp, n, tm, FORMATS[fmt], C.byref(st), _ptr(reads)[0],
                                            len(reads), _ptr(offs)[0], len(offs), MEM_HOST, C.byref(nr),
                                            C.byref(nb)))
        return reads[: nb.value], offs, st.value

    def store_pack(self, p0: int = 0, p1: int | None = None):
        """Packs partitions [p0, p1) into new device tensors: (bytes uint8,
        idx int64, keys int32, counts uint64 [3, p1 - p0] of per-partition
        bytes, superkmers, k-mers)."""
        import torch

        p1 = self.partitions if p1 is None else p1
        n = p1 - p0
        counts = np.zeros(3 * max(n, 1), np.uint64)
        L, h = self._L, self._h
        self._check(L.gkc_store_pack(h, p0, p1, None, 0, None, None, 0, _ptr(counts)[0]))
        nb, ns = int(counts[:n].sum()), int(counts[n:2 * n].sum())
        dev = torch.device("cuda", self.device)
        b = torch.empty(max(nb, 1), dtype=torch.uint8, device=dev)
        i = torch.empty(max(ns, 1), dtype=torch.int64, device=dev)
        k = torch.empty(max(ns, 1), dtype=torch.int32, device=dev)
        self._check(L.gkc_store_pack(h, p0, p1, _ptr(b)[0], nb, _ptr(i)[0], _ptr(k)[0], ns, _ptr(counts)[0]))
        return b[:nb], i[:ns], k[:ns], counts[:3 * n].reshape(3, n)

    def store_append(self, p0: int, p1: int, nbytes, idx, keys, counts):
        """Appends a packed range of partitions [p0, p1) (store_pack's layout;
        device tensors or host arrays) as one store chunk."""
        counts = np.ascontiguousarray(np.asarray(counts, np.uint64).reshape(-1))
        if hasattr(nbytes, "is_cuda") and nbytes.is_cuda:
            import torch
            torch.cuda.current_stream(nbytes.device).synchronize()  # the producer's stream, e.g. a collective's
        self._check(self._L.gkc_store_append(self._h, p0, p1, _ptr(nbytes)[0], _ptr(idx)[0], _ptr(keys)[0],
                                             _ptr(counts)[0]))

    def reserve_host(self, nbytes: int) -> int:
        """Pins host memory for spilled chunks until the arena holds `nbytes`
        in all; returns the bytes pinned.  May run on another thread beside
        add_reads."""
        pinned = C.c_uint64(0)
        rc = self._L.gkc_reserve_host(self._h, int(nbytes), C.byref(pinned))
        if rc != 0:
            raise GkcError(rc, f"gkc_reserve_host({nbytes}): {self._L.gkc_strerror(rc).decode()}")
        return pinned.value

    # -- phase 2 -------------------------------------------------------------
    def count(self, cmin: int = 1, cmax: int = UINT32_MAX):
        """Counts the store; returns (kept, distinct)."""
        no, nd = C.c_uint64(0), C.c_uint64(0)
        self._check(self._L.gkc_count(self._h, cmin, cmax, C.byref(no), C.byref(nd)))
        self._kw = 2 if self.k > 32 else 1
        return no.value, nd.value

    def count_partitions(self, parts, cmin: int = 1, cmax: int = UINT32_MAX):
        """Counts only partitions `parts` of the store; returns (kept, distinct)."""
        a = np.ascontiguousarray(parts, np.int32)
        no, nd = C.c_uint64(0), C.c_uint64(0)
        self._check(self._L.gkc_count_partitions(self._h, _ptr(a)[0], len(a), cmin, cmax, C.byref(no),
                                                 C.byref(nd)))
        self._kw = 2 if self.k > 32 else 1
        return no.value, nd.value

    def result(self, n: int | None = None):
        """The last count's (kmers uint64, counts uint32) as host arrays
        (kmers of shape (n, 2) for k > 32)."""
        if n is None:
            kp, cp, nn = C.c_void_p(), C.c_void_p(), C.c_uint64(0)
            self._check(self._L.gkc_result_device(self._h, C.byref(kp), C.byref(cp), C.byref(nn)))
            n = nn.value
        km = np.zeros((max(1, n), 2) if self._kw == 2 else max(1, n), np.uint64)
        ct = np.zeros(max(1, n), np.uint32)
        self._check(self._L.gkc_result(self._h, _ptr(km)[0], _ptr(ct)[0], n, MEM_HOST))
        return km[:n], ct[:n]

    def result_into(self, out_kmers, out_counts) -> int:
        """Copies the last count's result into the given arrays (host or CUDA,
        min(len, n) entries); returns n."""
        kp, km = _ptr(out_kmers)
        cp, _ = _ptr(out_counts)
        self._check(self._L.gkc_result(self._h, kp, cp, len(out_kmers), km))
        return self.result_device()[2]

    def result_device(self):
        kp, cp, nn = C.c_void_p(), C.c_void_p(), C.c_uint64(0)
        self._check(self._L.gkc_result_device(self._h, C.byref(kp), C.byref(cp), C.byref(nn)))
        return kp.value, cp.value, nn.value

    def count_reads(self, reads, offs, cmin: int = 1, cmax: int = UINT32_MAX, out_kmers=None,
                    out_counts=None):
        """reads -> (kept, distinct); fills out_kmers/out_counts when given."""
        rp, rm = _ptr(reads)
        op, _ = _ptr(offs)
        kp, km = _ptr(out_kmers)
        cp, _ = _ptr(out_counts)
        cap = 0 if out_kmers is None else len(out_kmers)
        no, nd = C.c_uint64(0), C.c_uint64(0)
        self._check(self._L.gkc_count_reads(self._h, rp, op, len(offs) - 1, rm, cmin, cmax, kp, cp, cap,
                                            km, C.byref(no), C.byref(nd)))
        self._kw = 2 if self.k > 32 else 1
        return no.value, nd.value

    def count_keys(self, keys, cmin: int = 1, cmax: int = UINT32_MAX):
        """Counts raw uint64 keys (no canonical step); returns (kept, distinct)."""
        kp, km = _ptr(keys)
        no, nd = C.c_uint64(0), C.c_uint64(0)
        self._check(self._L.gkc_count_keys(self._h, kp, len(keys), km, cmin, cmax, C.byref(no), C.byref(nd)))
        self._kw = 1
        return no.value, nd.value

    # -- learned minimizer order --------------------------------------------
    def minimizer_loads(self) -> np.ndarray:
        """k-mer instances of the store per minimizer key (4^p, uint64)."""
        out = np.zeros(4 ** self.p, np.uint64)
        self._check(self._L.gkc_minimizer_loads(self._h, _ptr(out)[0], len(out), MEM_HOST))
        return out

    def mlp_grad(self, params, pmers, targets, weights=None, norm: float = 1.0):
        """(loss, gradient) of one forward/backward pass over the samples."""
        params = np.ascontiguousarray(params, np.float32)
        pmers = np.ascontiguousarray(pmers, np.uint32)
        targets = np.ascontiguousarray(targets, np.float32)
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        grad = np.zeros_like(params)
        loss = C.c_float(0)
        self._check(self._L.gkc_mlp_grad(self._h, _ptr(params)[0], _ptr(pmers)[0], len(pmers), _ptr(targets)[0],
                                         _ptr(w)[0], norm, _ptr(grad)[0], C.byref(loss)))
        return loss.value, grad

    def mlp_train(self, params, targets, weights=None, epochs: int = 4, batch: int = 4096, lr: float = 1e-3,
                  seed: int = 0):
        """Trains a copy of params on all 4^p p-mers; returns (params, last loss)."""
        params = np.array(params, np.float32, copy=True)
        targets = np.ascontiguousarray(targets, np.float32)
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        loss = C.c_float(0)
        self._check(self._L.gkc_mlp_train(self._h, _ptr(params)[0], _ptr(targets)[0], _ptr(w)[0], epochs, batch,
                                          lr, seed, C.byref(loss)))
        return params, loss.value

    def mlp_scores(self, params) -> np.ndarray:
        params = np.ascontiguousarray(params, np.float32)
        out = np.zeros(4 ** self.p, np.float32)
        self._check(self._L.gkc_mlp_scores(self._h, _ptr(params)[0], _ptr(out)[0], MEM_HOST))
        return out

    def mlp_order(self, params, heavy: int = 0) -> np.ndarray:
        """Makes the network's order the context's order (the `heavy` p-mers
        of highest score ranked last; 0 = 4^p / 4); returns the rank table."""
        params = np.ascontiguousarray(params, np.float32)
        lut = np.zeros(4 ** self.p, np.uint32)
        self._check(self._L.gkc_mlp_order(self._h, _ptr(params)[0], heavy, _ptr(lut)[0]))
        return lut

    def timings(self):
        t = (C.c_double * 10)()
        self._check(self._L.gkc_last_timings(self._h, t, 10))
        return {"phase1_ms": t[0], "phase1_search_ms": t[1], "phase2_ms": t[2], "phase2_kernel_ms": t[3],
                "sub_buckets": int(t[4]), "overflowed_sub_buckets": int(t[5]), "phase2_stage_ms": t[6],
                "phase2_groups": int(t[7]), "second_pass_sub_buckets": int(t[8]), "h2d_bytes": int(t[9])}

    def kernel_launches(self) -> int:
        return int(self._L.gkc_kernel_launches(self._h))

    def set_stream(self, stream):
        """Runs on a CUDA stream (an int handle or a torch.cuda.Stream); None = own."""
        h = None
        if stream is not None:
            h = C.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
        self._check(self._L.gkc_set_stream(self._h, h))

    def set_profiling(self, on: bool = True):
        self._check(self._L.gkc_set_profiling(self._h, int(on)))

    def kernel_stats(self, reset: bool = False):
        """{class: (ms, launches, algorithmic bytes)} since the last reset."""
        n = len(KERNEL_CLASSES)
        ms, nl, by = (C.c_double * n)(), (C.c_uint64 * n)(), (C.c_double * n)()
        self._check(self._L.gkc_kernel_stats(self._h, ms, nl, by, n, int(reset)))
        return {KERNEL_CLASSES[i]: (ms[i], int(nl[i]), by[i]) for i in range(n)}
