"""The product's host-side schedule (csrc/topology.c) and host BLAKE3
(csrc/b3_host.c), built without CUDA as _build/libpose_b200_host.so.

Checks: the copy edges reproduce the reference's pose_graph_edges numbering
(via the golden digests), and the recycled slot map is safe for level-parallel
labelling — recomputed independently here the way the reference's own
test_slot_map.c checks live ranges (common/test/test_slot_map.c:50-135).
"""
from __future__ import annotations

import ctypes as C
import hashlib
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG_DIR, golden

u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)


class HostTopo(C.Structure):
    _fields_ = [("cb", C.c_uint32), ("n", C.c_int), ("half_w", C.c_uint32),
                ("retained", C.c_uint32), ("S", C.c_uint32), ("L", C.c_uint32),
                ("pool", C.c_uint32), ("max_width", C.c_uint32), ("lstart", u32p),
                ("recs", u32p), ("orank", u32p), ("desc", C.c_uint8 * 32),
                ("csm", C.c_uint32), ("gpool2", C.c_uint32), ("recs2", u32p)]


@pytest.fixture(scope="module")
def host():
    path = os.path.join(PKG_DIR, "_build", "libpose_b200_host.so")
    if not os.path.exists(path):
        subprocess.run(["make", "-s", "-C", PKG_DIR, "host"], check=True)
    L = C.CDLL(path)
    L.pb_copy_node_count.argtypes = [C.c_uint32]
    L.pb_copy_node_count.restype = C.c_uint64
    L.pb_chunk_node_count.argtypes = [C.c_uint32]
    L.pb_chunk_node_count.restype = C.c_uint64
    L.pb_topo_copy_edges.argtypes = [C.c_uint32, u8p, u32p, u32p, u32p]
    L.pb_topo_copy_edges.restype = C.c_uint64
    L.pb_topo_host_build.argtypes = [C.c_uint32, C.POINTER(HostTopo)]
    L.pb_topo_host_build.restype = C.c_int
    L.pb_topo_host_build_ex.argtypes = [C.c_uint32, C.c_uint32, C.POINTER(HostTopo)]
    L.pb_topo_host_build_ex.restype = C.c_int
    L.pb_topo_host_free.argtypes = [C.POINTER(HostTopo)]
    L.pb_chunk_seed.argtypes = [u8p, u8p, C.c_size_t, C.c_uint64]
    L.pb_graph_descriptor.argtypes = [u8p, C.c_uint64, C.c_uint64]
    L.pb_label_keys.argtypes = [u32p, u32p]
    L.pb_parameter_n.argtypes = [C.c_uint64]
    L.pb_parameter_n.restype = C.c_int
    return L


def copy_edges(L, cb):
    S = L.pb_copy_node_count(cb)
    np_ = np.zeros(S, np.uint8)
    p0 = np.zeros(S, np.uint32)
    p1 = np.zeros(S, np.uint32)
    n = L.pb_parameter_n(cb)
    outs = np.zeros(1 << n, np.uint32)
    assert L.pb_topo_copy_edges(cb, np_.ctypes.data_as(u8p), p0.ctypes.data_as(u32p),
                                p1.ctypes.data_as(u32p), outs.ctypes.data_as(u32p)) == S
    return np_, p0, p1, outs


def chunk_edges(L, cb):
    """Assemble the whole chunk (left copy, right copy shifted by S) in the
    reference's pose_graph_edges format."""
    np_, p0, p1, outs = copy_edges(L, cb)
    S = len(np_)
    n = L.pb_parameter_n(cb)
    hw = 1 << n
    ret = cb - hw
    rp0 = np.concatenate([p0, np.where(np_ >= 1, p0 + S, 0).astype(np.uint32)])
    rp1 = np.concatenate([p1, np.where(np_ == 2, p1 + S, 0).astype(np.uint32)])
    rank = np.full(2 * S, -1, np.int32)
    rank[outs] = np.arange(hw, dtype=np.int32)
    rank[outs[:ret].astype(np.int64) + S] = hw + np.arange(ret, dtype=np.int32)
    return np.concatenate([np_, np_]), rp0, rp1, rank


def test_chunk_edges_match_reference(host):
    for e in golden("edges.json"):
        np_, p0, p1, rk = chunk_edges(host, e["m"])
        assert len(np_) == e["count"] == host.pb_chunk_node_count(e["m"])
        assert hashlib.sha256(np_.tobytes()).hexdigest() == e["np"], e["m"]
        assert hashlib.sha256(p0.tobytes()).hexdigest() == e["p0"], e["m"]
        assert hashlib.sha256(p1.tobytes()).hexdigest() == e["p1"], e["m"]
        assert hashlib.sha256(rk.tobytes()).hexdigest() == e["rank"], e["m"]


def test_host_b3_matches_reference(host):
    k = golden("hash_kats.json")
    a = np.zeros(8, np.uint32)
    b = np.zeros(8, np.uint32)
    host.pb_label_keys(a.ctypes.data_as(u32p), b.ctypes.data_as(u32p))
    assert a.tolist() == k["key_src"] and b.tolist() == k["key_int"]
    for d in k["descriptors"]:
        out = (C.c_uint8 * 32)()
        host.pb_graph_descriptor(C.cast(out, u8p), d["m"], d["n"])
        assert bytes(out).hex() == d["hex"]
        assert host.pb_parameter_n(d["m"]) == d["n"]
    for c in k["chunk_seeds"]:
        seed = bytes.fromhex(c["seed"])
        out = (C.c_uint8 * 32)()
        sbuf = (C.c_uint8 * max(1, len(seed))).from_buffer_copy(seed or b"\0")
        host.pb_chunk_seed(C.cast(out, u8p), C.cast(sbuf, u8p), len(seed), c["index"])
        assert bytes(out).hex() == c["hex"], (len(seed), c["index"])


def schedule(L, cb):
    t = HostTopo()
    assert L.pb_topo_host_build(cb, C.byref(t)) == 0
    lstart = np.ctypeslib.as_array(t.lstart, shape=(t.L + 1,)).copy()
    recs = np.ctypeslib.as_array(t.recs, shape=(t.S, 4)).copy()
    orank = np.ctypeslib.as_array(t.orank, shape=(t.S,)).copy()
    info = {k: getattr(t, k) for k in ("cb", "n", "half_w", "retained", "S", "L", "pool", "max_width")}
    desc = bytes(t.desc)
    L.pb_topo_host_free(C.byref(t))
    return info, lstart, recs, orank, desc


@pytest.mark.parametrize("cb", [1, 2, 3, 5, 16, 17, 100, 1024, 4096])
def test_schedule_is_level_parallel_safe(host, cb):
    info, lstart, recs, orank, desc = schedule(host, cb)
    np_, p0, p1, outs = copy_edges(host, cb)
    S, L, pool = info["S"], info["L"], info["pool"]
    ids = (recs[:, 0] & 0x0FFFFFFF).astype(np.int64)
    npr = (recs[:, 0] >> 28) & 3
    outbit = (recs[:, 0] >> 30) & 1
    # the records are a permutation of the copy's nodes, ordered by level
    assert sorted(ids.tolist()) == list(range(S))
    assert (npr == np_[ids]).all()
    assert outbit.sum() == info["half_w"]
    r = orank[outbit == 1]
    assert sorted(r.tolist()) == list(range(info["half_w"]))
    assert (orank[outbit == 0] == 0xFFFFFFFF).all()
    assert (outs[r] == ids[outbit == 1]).all()
    level = np.zeros(S, np.int64)
    for l in range(L):
        level[ids[lstart[l]:lstart[l + 1]]] = l
    # levels are dependency levels: 1 + max(level(pred))
    want = np.zeros(S, np.int64)
    for i in range(S):
        if np_[i] >= 1:
            want[i] = level[p0[i]] + 1
        if np_[i] == 2:
            want[i] = max(want[i], level[p1[i]] + 1)
    assert (want == level).all()
    # slot safety, simulated level by level: every predecessor read in a level
    # sees its own label, and no slot is written twice within a level nor
    # written while it is read in that level
    slot_of = np.full(S, -1, np.int64)
    content = np.full(pool, -1, np.int64)
    assert recs[:, 3].max() < pool and recs[:, 1].max() < pool and recs[:, 2].max() < pool
    for l in range(L):
        seg = recs[lstart[l]:lstart[l + 1]]
        sid = ids[lstart[l]:lstart[l + 1]]
        for k in range(len(seg)):
            i = sid[k]
            if np_[i] >= 1:
                assert seg[k, 1] == slot_of[p0[i]] and content[seg[k, 1]] == p0[i]
            if np_[i] == 2:
                assert seg[k, 2] == slot_of[p1[i]] and content[seg[k, 2]] == p1[i]
        dst = seg[:, 3].astype(np.int64)
        assert len(set(dst.tolist())) == len(dst)
        reads = set(seg[npr[lstart[l]:lstart[l + 1]] >= 1, 1].tolist()) | \
            set(seg[npr[lstart[l]:lstart[l + 1]] == 2, 2].tolist())
        assert not (reads & set(dst.tolist()))
        content[dst] = sid
        slot_of[sid] = dst
    assert pool <= 8 * (1 << info["n"])


def test_schedule_sizes(host):
    info, lstart, recs, orank, desc = schedule(host, 1 << 17)
    assert info["S"] == 18087935 and 2 * info["S"] == 36175870
    assert info["L"] == 393197
    assert info["pool"] <= 2 * (1 << 16) * 2
    assert lstart[-1] == info["S"]


def test_bad_chunk_blocks(host):
    t = HostTopo()
    assert host.pb_topo_host_build(0, C.byref(t)) == -1
    assert host.pb_topo_host_build((1 << 20) + 1, C.byref(t)) == -1


NO_SLOT = 0xFFFFFFFF
PREV = 1 << 31
SMEM = 1 << 30


def pipelined(L, cb, csm):
    t = HostTopo()
    assert L.pb_topo_host_build_ex(cb, csm, C.byref(t)) == 0
    lstart = np.ctypeslib.as_array(t.lstart, shape=(t.L + 1,)).copy()
    recs2 = np.ctypeslib.as_array(t.recs2, shape=(t.S, 8)).copy()
    recs = np.ctypeslib.as_array(t.recs, shape=(t.S, 4)).copy()
    info = {k: getattr(t, k) for k in ("S", "L", "half_w", "csm", "gpool2", "pool")}
    L.pb_topo_host_free(C.byref(t))
    return info, lstart, recs, recs2


@pytest.mark.parametrize("cb,csm", [(1, 4), (3, 2), (16, 4), (100, 16), (1024, 64), (1024, 4096),
                                    (4096, 32), (4096, 2048),
                                    # the multi-unit depth kernel's 512-slot pools
                                    (3000, 512), (4096, 512), (16384, 512)])
def test_pipelined_records_are_safe(host, cb, csm):
    """Simulate the pipelined schedule level by level with both pools:
    every read sees its predecessor, no slot is written while it is read in the
    same level, and a predecessor fetched one level early (a reference without
    PREV) is not overwritten during the level in which it is fetched."""
    info, lstart, recs, r2 = pipelined(host, cb, csm)
    np_, p0, p1, outs = copy_edges(host, cb)
    S, Lv = info["S"], info["L"]
    assert info["csm"] <= csm
    ids = (r2[:, 0] & 0x0FFFFFFF).astype(np.int64)
    assert (r2[:, 0] == recs[:, 0]).all()
    level = np.zeros(S, np.int64)
    for l in range(Lv):
        level[ids[lstart[l]:lstart[l + 1]]] = l
    gs = r2[:, 3]
    ss = r2[:, 4]
    assert (gs[gs != NO_SLOT] < info["gpool2"]).all()
    assert (ss[ss != NO_SLOT] < info["csm"]).all()
    cg = np.full(max(1, info["gpool2"]), -1, np.int64)
    cs = np.full(max(1, info["csm"]), -1, np.int64)

    def check_ref(ref, pred, lv, early):
        if (ref & PREV) != 0:
            assert not early and level[pred] == lv - 1
            pool = cs if (ref & SMEM) else cg
        else:
            assert level[pred] <= lv - 2
            pool = cg
        assert pool[ref & 0x3FFFFFFF] == pred

    for l in range(Lv):
        a, b = lstart[l], lstart[l + 1]
        for k in range(a, b):
            i = ids[k]
            for e, pp in ((1, p0), (2, p1)):
                if np_[i] >= e:
                    check_ref(int(r2[k, e]), int(pp[i]), l, False)
        # early fetch of the next level's old predecessors happens during level l
        if l + 1 < Lv:
            for k in range(lstart[l + 1], lstart[l + 2]):
                i = ids[k]
                for e, pp in ((1, p0), (2, p1)):
                    if np_[i] >= e and (int(r2[k, e]) & PREV) == 0:
                        check_ref(int(r2[k, e]), int(pp[i]), l + 1, True)
                        assert int(r2[k, e]) not in set(gs[a:b].tolist())
        gw = gs[a:b][gs[a:b] != NO_SLOT]
        sw = ss[a:b][ss[a:b] != NO_SLOT]
        assert len(set(gw.tolist())) == len(gw) and len(set(sw.tolist())) == len(sw)
        reads_g, reads_s = set(), set()
        for k in range(a, b):
            for e in (1, 2):
                if np_[ids[k]] >= e:
                    ref = int(r2[k, e])
                    (reads_s if (ref & PREV) and (ref & SMEM) else reads_g).add(ref & 0x3FFFFFFF)
        assert not (reads_g & set(gw.tolist())) and not (reads_s & set(sw.tolist()))
        for k in range(a, b):
            i = ids[k]
            if gs[k] != NO_SLOT:
                cg[gs[k]] = i
            if ss[k] != NO_SLOT:
                cs[ss[k]] = i
        # outputs keep their rank
        outbit = (r2[a:b, 0] >> 30) & 1
        assert ((r2[a:b, 5] != 0xFFFFFFFF) == (outbit == 1)).all()
    assert info["gpool2"] <= info["pool"]


def cluster_barriers(lstart, split_width):
    """The cluster-barrier sequences of the depth kernel's cluster form
    (label_ws.cu, k_label_wsc), restated: rank 0 passes a cluster barrier at
    boundary b (between levels b - 1 and b) when level b - 1 or b is wider
    than split_width; the other ranks walk the split levels in order and
    pass boundary l before split level l unless l - 1 was split too, and
    boundary l + 1 after it."""
    w = np.diff(np.asarray(lstart, dtype=np.int64))
    L = len(w)
    split = w > split_width
    rank0 = [b for b in range(L + 1)
             if (b > 0 and split[b - 1]) or (b < L and split[b])]
    levels = [int(x) for x in np.nonzero(split)[0]]
    helper = []
    for k, l in enumerate(levels):
        if k == 0 or levels[k - 1] + 1 != l:
            helper.append(l)
        helper.append(l + 1)
    return rank0, helper


@pytest.mark.parametrize("cb", [64, 1024, 3000, 4096, 1 << 14])
def test_cluster_ranks_pass_the_same_barriers(host, cb):
    """Every CTA of a depth-kernel cluster passes the same cluster barriers in
    the same order (a rank that skipped or repeated one would leave the
    others waiting), for the default split width and for the extremes."""
    t = HostTopo()
    assert host.pb_topo_host_build(cb, C.byref(t)) == 0
    try:
        lstart = np.ctypeslib.as_array(t.lstart, shape=(t.L + 1,)).copy()
    finally:
        host.pb_topo_host_free(C.byref(t))
    for sw in (0, 1, 100, 480, 224, 1 << 30):
        rank0, helper = cluster_barriers(lstart, sw)
        assert rank0 == helper, (cb, sw)
        assert helper == sorted(set(helper)), (cb, sw)
        if sw == 0:
            assert rank0 == list(range(len(lstart)))  # every boundary
        if sw == 1 << 30:
            assert rank0 == []
