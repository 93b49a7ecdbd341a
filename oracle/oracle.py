"""TEST INFRASTRUCTURE ONLY: ctypes bindings for the CPU oracle.

Two oracles live here, both used only by tests/, ``__graft_entry__.smoke()``
and the bench's CPU-baseline / reference legs, never by the product path:

* ``Oracle`` — ``oracle/_build/liboracle.so``, the C restatement of the
  reference algorithm (``oracle/pose_oracle.c``; reference citations there).
* ``RefCPU`` — ``oracle/_ref/libposeref.so``, the reference's own CPU labeler
  compiled from its sources (``common/src/hash.c``, ``common/src/graph.c``,
  vendored BLAKE3 1.8.5) by ``oracle/Makefile``, driven by
  ``oracle/ref_driver.c`` on N host threads.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libposeref.so")

_u8p = C.POINTER(C.c_uint8)


def _buf(b: bytes | bytearray | np.ndarray | None):
    if b is None:
        return None
    a = np.frombuffer(bytes(b), dtype=np.uint8) if not isinstance(b, np.ndarray) else b
    a = np.ascontiguousarray(a, dtype=np.uint8)
    return a.ctypes.data_as(_u8p), a


def build_oracle() -> None:
    """Compile liboracle.so (always possible: needs only gcc)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


class Oracle:
    """The C restatement (``pose_oracle.c``)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build_oracle()
        L = C.CDLL(path)
        L.oracle_blake3.argtypes = [_u8p, C.c_size_t, _u8p]
        L.oracle_derive_key.argtypes = [C.c_char_p, _u8p, C.c_size_t, _u8p]
        L.oracle_label_keys.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.oracle_label_node.argtypes = [_u8p, C.c_int, C.c_uint64, _u8p, _u8p, _u8p, _u8p]
        L.oracle_descriptor.argtypes = [_u8p, C.c_uint64, C.c_uint64]
        L.oracle_chunk_seed.argtypes = [_u8p, _u8p, C.c_size_t, C.c_uint64]
        L.oracle_parameter_n.argtypes = [C.c_uint64]
        L.oracle_parameter_n.restype = C.c_int
        L.oracle_node_count.argtypes = [C.c_uint64]
        L.oracle_node_count.restype = C.c_uint64
        L.oracle_edges.argtypes = [C.c_uint64, _u8p, C.POINTER(C.c_uint32),
                                   C.POINTER(C.c_uint32), C.POINTER(C.c_int32)]
        L.oracle_edges.restype = C.c_uint64
        L.oracle_label_chunk.argtypes = [_u8p, C.c_uint64, _u8p, _u8p]
        L.oracle_label_chunk.restype = C.c_int
        L.oracle_label_region.argtypes = [_u8p, C.c_size_t, C.c_uint32, _u8p, C.c_uint64, C.c_uint64]
        L.oracle_label_region.restype = C.c_int
        self.L = L

    def blake3(self, data: bytes) -> bytes:
        out = np.zeros(32, np.uint8)
        p, _a = _buf(data) if len(data) else (None, None)
        self.L.oracle_blake3(p, len(data), out.ctypes.data_as(_u8p))
        return out.tobytes()

    def derive_key(self, context: str, material: bytes) -> bytes:
        out = np.zeros(32, np.uint8)
        p, _a = _buf(material) if len(material) else (None, None)
        self.L.oracle_derive_key(context.encode(), p, len(material), out.ctypes.data_as(_u8p))
        return out.tobytes()

    def label_keys(self) -> tuple[np.ndarray, np.ndarray]:
        a = np.zeros(8, np.uint32)
        b = np.zeros(8, np.uint32)
        self.L.oracle_label_keys(a.ctypes.data_as(C.POINTER(C.c_uint32)),
                                 b.ctypes.data_as(C.POINTER(C.c_uint32)))
        return a, b

    def label_node(self, is_source: int, idx: int, p0: bytes | None, p1: bytes | None,
                   seed: bytes, desc: bytes) -> bytes:
        out = np.zeros(32, np.uint8)
        a = _buf(p0)
        b = _buf(p1)
        s = _buf(seed)
        d = _buf(desc)
        self.L.oracle_label_node(out.ctypes.data_as(_u8p), int(is_source), idx,
                                 a[0] if a else None, b[0] if b else None, s[0], d[0])
        return out.tobytes()

    def descriptor(self, m: int, n: int) -> bytes:
        out = np.zeros(32, np.uint8)
        self.L.oracle_descriptor(out.ctypes.data_as(_u8p), m, n)
        return out.tobytes()

    def chunk_seed(self, seed: bytes, chunk_index: int) -> bytes:
        out = np.zeros(32, np.uint8)
        s = _buf(seed)
        self.L.oracle_chunk_seed(out.ctypes.data_as(_u8p), s[0] if s else None, len(seed), chunk_index)
        return out.tobytes()

    def parameter_n(self, m: int) -> int:
        return self.L.oracle_parameter_n(m)

    def node_count(self, m: int) -> int:
        return self.L.oracle_node_count(m)

    def edges(self, m: int):
        cnt = self.node_count(m)
        np_ = np.zeros(cnt, np.uint8)
        p0 = np.zeros(cnt, np.uint32)
        p1 = np.zeros(cnt, np.uint32)
        rk = np.zeros(cnt, np.int32)
        got = self.L.oracle_edges(m, np_.ctypes.data_as(_u8p), p0.ctypes.data_as(C.POINTER(C.c_uint32)),
                                  p1.ctypes.data_as(C.POINTER(C.c_uint32)),
                                  rk.ctypes.data_as(C.POINTER(C.c_int32)))
        assert got == cnt
        return np_, p0, p1, rk

    def label_chunk(self, cseed: bytes, m: int, with_all: bool = False):
        out = np.zeros(m * 32, np.uint8)
        allb = np.zeros(self.node_count(m) * 32, np.uint8) if with_all else None
        s = _buf(cseed)
        rc = self.L.oracle_label_chunk(s[0], m, out.ctypes.data_as(_u8p),
                                       allb.ctypes.data_as(_u8p) if with_all else None)
        assert rc == 0
        return (out, allb) if with_all else out

    def label_region(self, seed: bytes, cb: int, num_super: int, rbo: int = 0,
                     threads: int = 1) -> np.ndarray:
        """Super-chunks of a region, optionally on several host threads (the
        C calls release the GIL)."""
        out = np.zeros(num_super * cb * 32, np.uint8)
        s = _buf(seed)

        def one(j: int) -> int:
            view = out[j * cb * 32:(j + 1) * cb * 32]
            return self.L.oracle_label_region(s[0], len(seed), cb, view.ctypes.data_as(_u8p), 1,
                                              rbo + j * cb)

        if threads <= 1:
            rcs = [one(j) for j in range(num_super)]
        else:
            with ThreadPoolExecutor(threads) as ex:
                rcs = list(ex.map(one, range(num_super)))
        assert all(rc == 0 for rc in rcs)
        return out


class RefCPU:
    """The reference's own CPU path compiled from source (``oracle/_ref``)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = C.CDLL(path)
        L.ref_label_super_chunks.argtypes = [_u8p, C.c_size_t, C.c_uint32, _u8p, C.c_uint64,
                                             C.c_uint64, C.c_int]
        L.ref_label_super_chunks.restype = C.c_int
        L.ref_scaffold_labels.argtypes = [_u8p, C.c_uint32, _u8p, C.c_uint64]
        L.ref_scaffold_labels.restype = C.c_uint64
        L.ref_edges.argtypes = [C.c_uint32, _u8p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                C.POINTER(C.c_int32), C.c_uint64]
        L.ref_edges.restype = C.c_uint64
        L.pose_label_node.argtypes = [_u8p, C.c_int, C.c_uint64, _u8p, _u8p, _u8p, _u8p, C.c_int]
        L.pose_label_node_keys.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.pose_graph_descriptor.argtypes = [_u8p, C.c_uint64, C.c_uint64]
        L.pose_chunk_seed.argtypes = [_u8p, _u8p, C.c_size_t, C.c_uint64]
        L.pose_graph_parameter_n.argtypes = [C.c_uint64]
        L.pose_graph_parameter_n.restype = C.c_int
        L.pose_graph_scaffold_node_count.argtypes = [C.c_uint32]
        L.pose_graph_scaffold_node_count.restype = C.c_uint64
        L.pose_graph_label.argtypes = [_u8p, C.c_size_t, C.c_uint64, _u8p, C.c_int]
        L.pose_graph_label.restype = C.c_int
        L.pose_graph_challenge.argtypes = [_u8p, C.c_size_t, C.c_uint64, C.c_uint64, _u8p, C.c_int]
        L.pose_graph_challenge.restype = C.c_int
        L.pose_graph_slot_map.argtypes = [C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.pose_graph_slot_map.restype = C.c_int
        self.L = L

    def label_super_chunks(self, seed: bytes, cb: int, num_super: int, rbo: int = 0,
                           threads: int | None = None) -> np.ndarray:
        out = np.zeros(num_super * cb * 32, np.uint8)
        s = _buf(seed)
        rc = self.L.ref_label_super_chunks(s[0], len(seed), cb, out.ctypes.data_as(_u8p), num_super,
                                           rbo, threads or os.cpu_count() or 1)
        assert rc == 0
        return out

    def scaffold_labels(self, cseed: bytes, cb: int) -> np.ndarray:
        cnt = self.L.pose_graph_scaffold_node_count(cb)
        out = np.zeros(cnt * 32, np.uint8)
        s = _buf(cseed)
        got = self.L.ref_scaffold_labels(s[0], cb, out.ctypes.data_as(_u8p), cnt)
        assert got == cnt
        return out

    def edges(self, cb: int):
        cnt = self.L.pose_graph_scaffold_node_count(cb)
        np_ = np.zeros(cnt, np.uint8)
        p0 = np.zeros(cnt, np.uint32)
        p1 = np.zeros(cnt, np.uint32)
        rk = np.zeros(cnt, np.int32)
        got = self.L.ref_edges(cb, np_.ctypes.data_as(_u8p), p0.ctypes.data_as(C.POINTER(C.c_uint32)),
                               p1.ctypes.data_as(C.POINTER(C.c_uint32)),
                               rk.ctypes.data_as(C.POINTER(C.c_int32)), cnt)
        assert got == cnt
        return np_, p0, p1, rk

    def label_node(self, is_source: int, idx: int, p0, p1, seed: bytes, desc: bytes) -> bytes:
        out = np.zeros(32, np.uint8)
        a = _buf(p0)
        b = _buf(p1)
        s = _buf(seed)
        d = _buf(desc)
        self.L.pose_label_node(out.ctypes.data_as(_u8p), int(is_source), idx, a[0] if a else None,
                               b[0] if b else None, s[0], d[0], 0)
        return out.tobytes()

    def label_keys(self):
        a = np.zeros(8, np.uint32)
        b = np.zeros(8, np.uint32)
        self.L.pose_label_node_keys(a.ctypes.data_as(C.POINTER(C.c_uint32)),
                                    b.ctypes.data_as(C.POINTER(C.c_uint32)))
        return a, b

    def descriptor(self, m: int, n: int) -> bytes:
        out = np.zeros(32, np.uint8)
        self.L.pose_graph_descriptor(out.ctypes.data_as(_u8p), m, n)
        return out.tobytes()

    def chunk_seed(self, seed: bytes, idx: int) -> bytes:
        out = np.zeros(32, np.uint8)
        s = _buf(seed)
        self.L.pose_chunk_seed(out.ctypes.data_as(_u8p), s[0] if s else None, len(seed), idx)
        return out.tobytes()

    def graph_label(self, seed: bytes, m: int) -> np.ndarray:
        out = np.zeros(m * 32, np.uint8)
        s = _buf(seed)
        assert self.L.pose_graph_label(s[0], len(seed), m, out.ctypes.data_as(_u8p), 0) == 0
        return out

    def challenge(self, seed: bytes, m: int, idx: int) -> bytes | None:
        """The reference's pose_graph_challenge (verifier recompute)."""
        out = np.zeros(32, np.uint8)
        s = _buf(seed)
        rc = self.L.pose_graph_challenge(s[0], len(seed), m, idx, out.ctypes.data_as(_u8p), 0)
        return out.tobytes() if rc == 0 else None
