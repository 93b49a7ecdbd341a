"""pose_b200 — Python host mirror of the reference's GPU labeler C API.

The product is ``libpose_b200.so`` (C11 host code + sm_100a kernels, built
from ``csrc/`` by the Makefile next to this file).  This module is a thin
ctypes layer over its C ABI (``include/gpu_label.h``, ``include/pose_b200.h``)
with the reference's names, argument meaning and error behaviour
(Amodo-Design/PoSE-Memory-Wiping, ``common/include/gpu_label.h:40-100``):
entry points return 0 / -1 (``None`` for a failed topology build) and print
their error to stderr.  Device buffers are raw device pointers (integers);
tests and the bench obtain them from torch, which is only plumbing here.

There is no CPU fallback: if the library cannot be loaded, ``load()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpose_b200.so")
INCLUDE_DIR = os.path.join(os.path.dirname(HERE), "include")

POSE_HASH_BLAKE3 = 0
POSE_HASH_SHA256 = 1
POSE_HASH_AES_PRF = 2
POSE_CHUNK_BLOCKS = 4096
POSE_GRAPH_MAX_M = 1 << 20

_lib = None
_lock = threading.Lock()


class Sched(C.Structure):
    """pose_b200_sched_t: zero fields mean automatic."""

    _fields_ = [("team_warps", C.c_uint32), ("units_per_team", C.c_uint32),
                ("max_teams", C.c_uint32), ("kernel", C.c_uint32),
                ("scratch_cap_bytes", C.c_uint64), ("lane_efficiency", C.c_uint32),
                ("flags", C.c_uint32), ("cluster_ctas", C.c_uint32)]


PACK_CHAIN = 255  # POSE_B200_PACK_CHAIN: pack units while their chain stays within the launch's longest
BATCH_ONE_LAUNCH = 1  # POSE_B200_BATCH_ONE_LAUNCH (Sched.flags): no separate launch for the deepest requests


class Stats(C.Structure):
    """pose_b200_stats_t."""

    _fields_ = [("kernel_ms", C.c_double), ("total_ms", C.c_double),
                ("super_chunks", C.c_uint64), ("units", C.c_uint64), ("nodes", C.c_uint64),
                ("scratch_bytes", C.c_uint64), ("team_warps", C.c_uint32),
                ("units_per_team", C.c_uint32), ("teams", C.c_uint32),
                ("kernel_launches", C.c_uint32), ("used_cv0_table", C.c_uint32),
                ("kernel", C.c_uint32), ("cluster_ctas", C.c_uint32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Request(C.Structure):
    """pose_b200_request_t: one pose_graph_hbm_topo_label-style request."""

    _fields_ = [("topo", C.c_void_p), ("session_seed", C.c_void_p), ("seed_len", C.c_size_t),
                ("hbm_dev_ptr", C.c_void_p), ("hbm_len", C.c_size_t), ("region_block_offset", C.c_uint64)]


_u8p = C.POINTER(C.c_uint8)
_u32p = C.POINTER(C.c_uint32)
SINK_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_size_t, C.c_uint64)
READ_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_size_t, C.c_uint64)


def build(force: bool = False) -> str:
    """Compile libpose_b200.so in place (nvcc for sm_100a + gcc)."""
    args = ["make", "-s", "-C", HERE]
    if force:
        subprocess.run(args + ["clean"], check=True)
    subprocess.run(args, check=True)
    return LIB_PATH


def _declare(L: C.CDLL) -> None:
    L.pose_graph_label_hbm.argtypes = [_u8p, C.c_size_t, C.c_uint32, C.c_void_p, C.c_size_t,
                                       C.c_uint64, C.c_int]
    L.pose_graph_label_hbm.restype = C.c_int
    L.pose_graph_hbm_topo_build.argtypes = [C.c_uint32, C.c_int]
    L.pose_graph_hbm_topo_build.restype = C.c_void_p
    L.pose_graph_hbm_topo_label.argtypes = [C.c_void_p, _u8p, C.c_size_t, C.c_void_p, C.c_size_t,
                                            C.c_uint64]
    L.pose_graph_hbm_topo_label.restype = C.c_int
    L.pose_graph_hbm_topo_free.argtypes = [C.c_void_p]
    L.pose_graph_hbm_topo_free.restype = None
    L.pose_gpu_label_node_single.argtypes = [_u8p, C.c_int, C.c_uint64, _u8p, _u8p, _u8p, _u8p,
                                             _u32p, _u32p]
    L.pose_gpu_label_node_single.restype = C.c_int
    L.pose_b200_topo_build.argtypes = [C.c_uint32, C.c_int]
    L.pose_b200_topo_build.restype = C.c_void_p
    L.pose_b200_topo_label.argtypes = [C.c_void_p, _u8p, C.c_size_t, C.c_void_p, C.c_size_t,
                                       C.c_uint64, C.POINTER(Sched), C.POINTER(Stats)]
    L.pose_b200_topo_label.restype = C.c_int
    L.pose_b200_topo_info.argtypes = [C.c_void_p, _u32p, C.POINTER(C.c_uint64), _u32p, _u32p,
                                      C.POINTER(C.c_uint64)]
    L.pose_b200_topo_info.restype = None
    L.pose_b200_plan.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(Sched), C.POINTER(Sched)]
    L.pose_b200_plan.restype = C.c_int
    L.pose_b200_topo_autotune.argtypes = [C.c_void_p, _u8p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_uint64,
                                          C.c_uint32, C.POINTER(Sched), C.POINTER(Stats)]
    L.pose_b200_topo_autotune.restype = C.c_int
    L.pose_b200_compress_rate.argtypes = [C.c_uint32, C.POINTER(C.c_double)]
    L.pose_b200_compress_rate.restype = C.c_double
    L.pose_b200_topo_label_noalloc.argtypes = [C.c_void_p, _u8p, C.c_size_t, C.c_void_p, C.c_size_t,
                                               C.c_uint64]
    L.pose_b200_topo_label_noalloc.restype = C.c_int
    L.pose_b200_topo_residue.argtypes = [C.c_void_p, C.POINTER(C.c_uint64)]
    L.pose_b200_topo_residue.restype = C.c_int
    L.pose_b200_count_nonzero.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(C.c_uint64)]
    L.pose_b200_count_nonzero.restype = C.c_int
    L.pose_b200_batch_create.argtypes = [C.POINTER(Request), C.c_size_t, C.POINTER(Sched)]
    L.pose_b200_batch_create.restype = C.c_void_p
    L.pose_b200_batch_autotune.argtypes = [C.POINTER(Request), C.c_size_t, C.POINTER(Sched), C.c_uint32,
                                           C.POINTER(Sched), C.POINTER(Stats)]
    L.pose_b200_batch_autotune.restype = C.c_void_p
    L.pose_b200_batch_run.argtypes = [C.c_void_p, C.POINTER(Stats)]
    L.pose_b200_batch_run.restype = C.c_int
    L.pose_b200_batch_destroy.argtypes = [C.c_void_p]
    L.pose_b200_batch_destroy.restype = None
    L.pose_b200_label_batch.argtypes = [C.POINTER(Request), C.c_size_t, C.POINTER(Sched), C.POINTER(Stats)]
    L.pose_b200_label_batch.restype = C.c_int
    L.pose_b200_label_stream.argtypes = [C.c_void_p, _u8p, C.c_size_t, C.c_uint64, C.c_uint64, C.c_uint64,
                                         C.c_size_t, SINK_FN, C.c_void_p, C.POINTER(Sched), C.POINTER(Stats)]
    L.pose_b200_label_stream.restype = C.c_int
    L.pose_b200_server_create.argtypes = [C.c_uint64, C.c_uint32]
    L.pose_b200_server_create.restype = C.c_void_p
    L.pose_b200_server_session.argtypes = [C.c_void_p, _u8p, C.c_size_t]
    L.pose_b200_server_session.restype = C.c_int
    L.pose_b200_server_submit.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_size_t, C.c_uint64]
    L.pose_b200_server_submit.restype = C.c_int64
    L.pose_b200_server_prepare.argtypes = [C.c_void_p, C.c_void_p]
    L.pose_b200_server_prepare.restype = C.c_int
    L.pose_b200_server_wait.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.pose_b200_server_wait.restype = C.c_int
    L.pose_b200_server_query.argtypes = [C.c_void_p, C.c_int64]
    L.pose_b200_server_query.restype = C.c_int
    L.pose_b200_server_stats.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                         C.POINTER(C.c_uint64)]
    L.pose_b200_server_stats.restype = None
    L.pose_b200_server_destroy.argtypes = [C.c_void_p]
    L.pose_b200_server_destroy.restype = None
    L.pose_b200_challenge.argtypes = [C.c_void_p, _u8p, C.c_size_t, C.c_uint64, _u8p]
    L.pose_b200_challenge.restype = C.c_int
    L.pose_b200_challenge_blocks.argtypes = [C.c_void_p, _u8p, C.c_size_t, C.POINTER(C.c_uint64), C.c_size_t,
                                             _u8p, C.POINTER(Sched), C.POINTER(Stats)]
    L.pose_b200_challenge_blocks.restype = C.c_int
    L.pose_b200_verify_sampled.argtypes = [C.c_void_p, _u8p, C.c_size_t, C.c_uint64, C.c_uint64, READ_FN,
                                           C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                           C.POINTER(C.c_uint64), C.POINTER(Sched), C.POINTER(Stats)]
    L.pose_b200_verify_sampled.restype = C.c_int
    L.pose_b200_last_error.argtypes = []
    L.pose_b200_last_error.restype = C.c_char_p


def load() -> C.CDLL:
    """Load the in-tree library, building it first if it is missing."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                build()
            L = C.CDLL(LIB_PATH)
            _declare(L)
            _lib = L
    return _lib


def _bytes_arg(b: bytes | None):
    if b is None:
        return None
    return C.cast(C.create_string_buffer(bytes(b), max(1, len(b))), _u8p)


def count_nonzero(dev_ptr: int, nbytes: int) -> int:
    """pose_b200_count_nonzero: nonzero bytes of a 16-byte aligned device
    buffer of the current device."""
    n = C.c_uint64(0)
    if load().pose_b200_count_nonzero(C.c_void_p(dev_ptr), nbytes, C.byref(n)) != 0:
        raise RuntimeError(last_error())
    return n.value


def last_error() -> str:
    return load().pose_b200_last_error().decode(errors="replace")


class Topology:
    """A resident topology (pose_hbm_topo_t) for one chunk_blocks value."""

    def __init__(self, chunk_blocks: int, algo: int = POSE_HASH_BLAKE3, cv0_table: bool = True):
        L = load()
        if algo != POSE_HASH_BLAKE3:
            h = L.pose_graph_hbm_topo_build(chunk_blocks, algo)
        else:
            h = L.pose_b200_topo_build(chunk_blocks, 1 if cv0_table else 0)
        if not h:
            raise RuntimeError(f"topology build failed: {last_error()}")
        self.handle = h
        self.chunk_blocks = chunk_blocks or POSE_CHUNK_BLOCKS
        self.super_bytes = self.chunk_blocks * 32

    def info(self) -> dict:
        cb = C.c_uint32()
        nodes = C.c_uint64()
        lv = C.c_uint32()
        pool = C.c_uint32()
        dev = C.c_uint64()
        load().pose_b200_topo_info(self.handle, C.byref(cb), C.byref(nodes), C.byref(lv),
                                   C.byref(pool), C.byref(dev))
        return {"chunk_blocks": cb.value, "nodes_per_chunk": nodes.value, "levels": lv.value,
                "pool_slots": pool.value, "device_bytes": dev.value}

    def label(self, seed: bytes, dev_ptr: int, nbytes: int, region_block_offset: int = 0,
              sched: Sched | None = None, stats: bool = False):
        """pose_graph_hbm_topo_label (or the scheduled variant).  Returns the
        C return code, or (rc, stats dict) when stats=True."""
        L = load()
        if sched is None and not stats:
            return L.pose_graph_hbm_topo_label(self.handle, _bytes_arg(seed), len(seed),
                                               C.c_void_p(dev_ptr), nbytes, region_block_offset)
        st = Stats()
        rc = L.pose_b200_topo_label(self.handle, _bytes_arg(seed), len(seed), C.c_void_p(dev_ptr),
                                    nbytes, region_block_offset,
                                    C.byref(sched) if sched is not None else None, C.byref(st))
        return (rc, st.as_dict()) if stats else rc

    def autotune(self, seed: bytes, dev_ptr: int, nbytes: int, region_block_offset: int = 0,
                 trials: int = 4):
        """pose_b200_topo_autotune: time the best modelled schedule of each
        team size on this call and keep the fastest for later calls of the
        same size.  Returns (rc, chosen schedule dict, stats dict); the
        buffer holds the labels afterwards."""
        ch = Sched()
        st = Stats()
        rc = load().pose_b200_topo_autotune(self.handle, _bytes_arg(seed), len(seed), C.c_void_p(dev_ptr), nbytes,
                                            region_block_offset, trials, C.byref(ch), C.byref(st))
        return rc, {k: getattr(ch, k) for k, _ in Sched._fields_}, st.as_dict()

    def label_noalloc(self, seed: bytes, dev_ptr: int, nbytes: int, region_block_offset: int = 0) -> int:
        """pose_b200_topo_label_noalloc: the same bytes as label(), with the
        library's static device scratch instead of memory allocated by the
        call (for callers that cannot allocate while labeling)."""
        return load().pose_b200_topo_label_noalloc(self.handle, _bytes_arg(seed), len(seed),
                                                   C.c_void_p(dev_ptr), nbytes, region_block_offset)

    def residue(self) -> int:
        """pose_b200_topo_residue: nonzero bytes left in the device workspace
        of this topology's labeling calls (0 between calls)."""
        n = C.c_uint64(0)
        if load().pose_b200_topo_residue(self.handle, C.byref(n)) != 0:
            raise RuntimeError(last_error())
        return n.value

    def label_stream(self, seed: bytes, region_bytes: int, sink, region_block_offset: int = 0,
                     byte_offset: int = 0, window_bytes: int = 1 << 30, sched: Sched | None = None):
        """pose_b200_label_stream: label region_bytes worth of super-chunks and
        call sink(memoryview, off) per window (from a worker thread) while the
        next window is labelled.  Returns (rc, stats dict)."""
        def _cb(ctx, buf, n, off):
            try:
                return int(sink(memoryview((C.c_uint8 * n).from_address(buf)), off) or 0)
            except Exception:
                return -1
        cb = SINK_FN(_cb)
        st = Stats()
        rc = load().pose_b200_label_stream(self.handle, _bytes_arg(seed), len(seed), region_bytes,
                                           region_block_offset, byte_offset, window_bytes, cb, None,
                                           C.byref(sched) if sched is not None else None, C.byref(st))
        return rc, st.as_dict()

    def challenge(self, seed: bytes, challenge_idx: int) -> bytes | None:
        """pose_b200_challenge: the label of output rank challenge_idx of the
        chunk graph labelled with `seed` (a 32-byte chunk seed), as the
        reference's pose_graph_challenge; None when the call fails."""
        out = (C.c_uint8 * 32)()
        rc = load().pose_b200_challenge(self.handle, _bytes_arg(seed), len(seed), challenge_idx,
                                        C.cast(out, _u8p))
        return bytes(out) if rc == 0 else None

    def challenge_blocks(self, session_seed: bytes, blocks, sched: Sched | None = None):
        """pose_b200_challenge_blocks: labels of absolute region blocks of one
        session.  Returns (rc, labels as n*32 bytes, stats dict)."""
        blocks = list(blocks)
        arr = (C.c_uint64 * max(1, len(blocks)))(*blocks)
        out = (C.c_uint8 * max(1, 32 * len(blocks)))()
        st = Stats()
        rc = load().pose_b200_challenge_blocks(self.handle, _bytes_arg(session_seed), len(session_seed), arr,
                                               len(blocks), C.cast(out, _u8p),
                                               C.byref(sched) if sched is not None else None, C.byref(st))
        return rc, bytes(out)[:32 * len(blocks)], st.as_dict()

    def verify_sampled(self, session_seed: bytes, wipe_len: int, samples: int, read,
                       sched: Sched | None = None) -> dict:
        """pose_b200_verify_sampled with read(nbytes, off) -> bytes-like giving
        the stored bytes at byte offset off.  Returns a dict with rc, checked,
        mismatched, first_bad (per sample, None where it matched) and stats."""
        def _cb(ctx, buf, n, off):
            try:
                data = read(n, off)
                if data is None or len(data) != n:
                    return -1
                C.memmove(buf, bytes(data), n)
                return 0
            except Exception:
                return -1
        cb = READ_FN(_cb)
        checked, mism = C.c_uint64(), C.c_uint64()
        fb = (C.c_uint64 * max(1, samples))()
        st = Stats()
        rc = load().pose_b200_verify_sampled(self.handle, _bytes_arg(session_seed), len(session_seed), wipe_len,
                                             samples, cb, None, C.byref(checked), C.byref(mism), fb,
                                             C.byref(sched) if sched is not None else None, C.byref(st))
        n = max(1, min(samples, wipe_len // self.super_bytes)) if wipe_len >= self.super_bytes else 0
        return {"rc": rc, "checked": checked.value, "mismatched": mism.value,
                "first_bad": [None if fb[i] == (1 << 64) - 1 else fb[i] for i in range(min(n, samples))],
                "stats": st.as_dict()}

    def plan(self, super_chunks: int, hint: Sched | None = None) -> Sched | None:
        out = Sched()
        rc = load().pose_b200_plan(self.handle, super_chunks,
                                   C.byref(hint) if hint is not None else None, C.byref(out))
        return out if rc == 0 else None

    def free(self) -> None:
        if self.handle:
            load().pose_graph_hbm_topo_free(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.free()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Batch:
    """pose_b200_batch_t: many requests in one persistent launch, captured once
    into a CUDA graph and replayed by run().

    requests: iterable of (topology, seed bytes, device pointer, nbytes, rbo).
    autotune > 0 runs pose_b200_batch_autotune with that many trials; the
    chosen schedule is then in .chosen and its timed replay in .tune_stats."""

    def __init__(self, requests, sched: Sched | None = None, autotune: int = 0):
        reqs = list(requests)
        self._seeds = [C.create_string_buffer(bytes(r[1]), max(1, len(r[1]))) for r in reqs]
        arr = (Request * len(reqs))()
        for i, (topo, seed, ptr, nbytes, rbo) in enumerate(reqs):
            arr[i] = Request(topo.handle, C.cast(self._seeds[i], C.c_void_p), len(seed), ptr, nbytes, rbo)
        self._arr = arr
        self.chosen = None
        self.tune_stats = None
        sp = C.byref(sched) if sched is not None else None
        if autotune:
            ch = Sched()
            st = Stats()
            h = load().pose_b200_batch_autotune(arr, len(reqs), sp, autotune, C.byref(ch), C.byref(st))
            if h:
                self.chosen = {k: getattr(ch, k) for k, _ in ch._fields_}
                self.tune_stats = st.as_dict()
        else:
            h = load().pose_b200_batch_create(arr, len(reqs), sp)
        if not h:
            raise RuntimeError("batch create failed")
        self.handle = h

    def run(self) -> tuple[int, dict]:
        st = Stats()
        rc = load().pose_b200_batch_run(self.handle, C.byref(st))
        return rc, st.as_dict()

    def free(self) -> None:
        if self.handle:
            load().pose_b200_batch_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.free()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Server:
    """pose_b200_server_t: continuous-batching labeling service."""

    def __init__(self, scratch_bytes: int = 0, max_waves: int = 0):
        h = load().pose_b200_server_create(scratch_bytes, max_waves)
        if not h:
            raise RuntimeError("server create failed")
        self.handle = h

    def session(self, seed: bytes) -> int:
        sid = load().pose_b200_server_session(self.handle, _bytes_arg(seed), len(seed))
        if sid < 0:
            raise RuntimeError("session registration failed")
        return sid

    def prepare(self, topo: "Topology") -> None:
        """Build what requests of this topology need before the first one
        arrives (the depth kernel's records of a deep topology)."""
        if load().pose_b200_server_prepare(self.handle, topo.handle) != 0:
            raise RuntimeError("server prepare failed")

    def submit(self, topo: "Topology", session: int, dev_ptr: int, nbytes: int, rbo: int = 0) -> int:
        return load().pose_b200_server_submit(self.handle, topo.handle, session, C.c_void_p(dev_ptr), nbytes, rbo)

    def wait(self, ticket: int) -> tuple[int, float, float]:
        """(rc, queue_ms, total_ms) of one request."""
        q = C.c_double()
        t = C.c_double()
        rc = load().pose_b200_server_wait(self.handle, ticket, C.byref(q), C.byref(t))
        return rc, q.value, t.value

    def query(self, ticket: int) -> int:
        return load().pose_b200_server_query(self.handle, ticket)

    def stats(self) -> dict:
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        load().pose_b200_server_stats(self.handle, C.byref(a), C.byref(b), C.byref(c))
        return {"submitted": a.value, "waves": b.value, "scratch_bytes": c.value}

    def close(self) -> None:
        if self.handle:
            load().pose_b200_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def label_hbm(seed: bytes, chunk_blocks: int, dev_ptr: int, nbytes: int,
              region_block_offset: int = 0, algo: int = POSE_HASH_BLAKE3) -> int:
    """pose_graph_label_hbm: build, label, free."""
    return load().pose_graph_label_hbm(_bytes_arg(seed), len(seed), chunk_blocks, C.c_void_p(dev_ptr),
                                       nbytes, region_block_offset, algo)


def label_node_single(is_source: int, node_index: int, pred0: bytes | None, pred1: bytes | None,
                      seed: bytes, descriptor: bytes, key_src, key_int) -> bytes | None:
    """pose_gpu_label_node_single; returns the 32-byte label or None on error."""
    out = (C.c_uint8 * 32)()
    ks = (C.c_uint32 * 8)(*[int(x) for x in key_src])
    ki = (C.c_uint32 * 8)(*[int(x) for x in key_int])
    rc = load().pose_gpu_label_node_single(C.cast(out, _u8p), int(is_source), node_index,
                                           _bytes_arg(pred0), _bytes_arg(pred1), _bytes_arg(seed),
                                           _bytes_arg(descriptor), C.cast(ks, _u32p), C.cast(ki, _u32p))
    return bytes(out) if rc == 0 else None


def compress_rate(iters: int = 4096) -> tuple[float, float]:
    """(compressions/s with every SM full, dependent cycles per compression)."""
    lat = C.c_double()
    rate = load().pose_b200_compress_rate(iters, C.byref(lat))
    return rate, lat.value


def exported_symbols() -> list[str]:
    """Function names declared in include/*.h (the C ABI this library promises)."""
    import re
    names = []
    for fn in sorted(os.listdir(INCLUDE_DIR)):
        if fn.endswith(".h"):
            src = open(os.path.join(INCLUDE_DIR, fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"\b(pose_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))
