#!/usr/bin/env python3
"""Benchmark of the PoSE-DB labeling hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload plain_2e17|plain_small|window_2e17|throughput_2e12|
                                latency_2e14|deep_2e20|batched|served] [--no-aux] [--no-cpu-baseline]

One step = one pass of the hot path over one batch: label the workload's
super-chunks (default: 32 consecutive super-chunks at chunk_blocks = 2^17,
key splitmix64(1) — the plain drop-in at write-up depth) through the C ABI
pose_graph_hbm_topo_label with the topology resident, as disk-wipe-bench's
worker does per HBM window.  Metric: persisted label MiB/s
(chunk_blocks*32 bytes per super-chunk / time), the reference's own
definition (common/src/cuda/label_gpu_common.cu:312-315).

At one GPU the default run adds, under their own keys: a full 16 GiB window
at 2^17 (the throughput regime), the 256-session batched workload in one
autotuned persistent launch, and a 120-request Poisson trace through the
continuous-batching server next to the same trace run one request at a time.

Under torchrun each rank labels its own disjoint range of super-chunks
(absolute positions offset by rank): no collective on the data path, weak
scaling; the step time is the max over ranks.

--impl reference times the reference's own CPU labeler
(pose_graph_label_region_pooled_inplace, built from source into oracle/_ref)
on this host's cores on a bounded sample of the same workload; rank 0 only.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import time

# One host-to-device work queue per server slot (the default is 8 queues,
# shared by the server's streams); read when CUDA initialises, so set here.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "pose-memory-wiping_b200")
MIB = float(1 << 20)


def load_pkg():
    if "pose_b200" in sys.modules:
        return sys.modules["pose_b200"]
    spec = importlib.util.spec_from_file_location(
        "pose_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pose_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def workload(name: str) -> dict:
    import pose_b200.workloads as wl
    if name == "plain_2e17":
        w = wl.plain_2e17()
    elif name == "plain_small":
        w = wl.plain_small()
    elif name == "window_2e17":
        # the reference's default 16 GiB HBM window at 2^17 (4096 super-chunks)
        w = dict(wl.plain_2e17(), name="window_2e17", chunks=4096)
    elif name == "throughput_2e12":
        # profiling case: many chunks in flight, ~0.1 s kernel, scratch + store > L2
        w = dict(wl.plain_2e17(), name="throughput_2e12", chunk_blocks=1 << 12, chunks=2048)
    elif name == "deep_2e20":
        # deep-graph stress: 4 chunks at chunk_blocks 2^20, scratch capped at 40 GiB
        w = wl.deep_2e20()
    elif name == "latency_2e14":
        # profiling case: few chunks, depth-bound, ~0.1 s kernel
        w = dict(wl.plain_2e17(), name="latency_2e14", chunk_blocks=1 << 14, chunks=16)
    else:
        raise SystemExit(f"unknown workload {name}")
    w["nodes_per_chunk"] = wl.chunk_nodes(w["chunk_blocks"])
    return w


# ── clocks ──────────────────────────────────────────────────────────────────

CLOCK_Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


class ClockSampler:
    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = f"/tmp/.pose_b200_clocks_{os.getpid()}_{gpu_index}.csv"

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={CLOCK_Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for ln in open(self.path):
            p = [x.strip() for x in ln.split(",")]
            if len(p) >= 9:
                rows.append(p)
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = sorted(sm)[len(sm) // 2:] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


# ── DRAM traffic from the committed ncu summaries ───────────────────────────

KERNEL_NAMES = {1: "k_label", 3: "k_label_ws", 4: "k_label_multi"}


def profiled_traffic(workload_name: str, kernel: int) -> float | None:
    """DRAM bytes (read + write) per launch of the kernel the plan ran, from
    the `bench-traffic: <workload> <kernel> <bytes>` lines of the ncu
    summaries in profiles/ (one ncu capture of the same command); None when
    no capture covers this workload and kernel."""
    name = KERNEL_NAMES.get(kernel)
    pdir = os.path.join(ROOT, "profiles")
    if not name or not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith(".md"):
            continue
        for ln in open(os.path.join(pdir, fn)):
            f = ln.split()
            if len(f) == 4 and f[0] == "bench-traffic:" and f[1] == workload_name and f[2] == name:
                return float(f[3])
    return None


def measured_hbm_gbs() -> float | None:
    """The pool's measured HBM copy bandwidth (MEASURED_PEAKS.json, written
    per GPU pod), or None when the file is absent."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except (OSError, ValueError, KeyError):
        return None


# ── reference CPU leg ───────────────────────────────────────────────────────

def cpu_reference(w: dict, steps: int, warmup: int, cores: int | None = None) -> dict:
    """Time the reference's own CPU in-place labeler (oracle/_ref) on the
    whole workload: every step labels all of its super-chunks, spread over
    every host thread (waves of one super-chunk per thread)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import RefCPU  # test infrastructure: the reference's CPU labeler, CPU legs only
    ref = RefCPU()
    cores = cores or os.cpu_count() or 1
    cb = w["chunk_blocks"]
    n = w["chunks"]
    times = []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        ref.label_super_chunks(w["key"], cb, n, w["rbo"], threads=cores)
        dt = time.perf_counter() - t0
        if i >= warmup:
            times.append(dt)
    sec = sum(times) / len(times)
    return {"value": n * cb * 32 / MIB / sec, "unit": "MiB/s", "cores": cores, "kind": "reference",
            "sample": f"the whole workload per step: {n} super-chunks of chunk_blocks={cb} "
                      f"({n * w['nodes_per_chunk']:.3g} nodes) on {cores} host threads, {steps} timed steps",
            "seconds_per_step": sec}


def golden_parity(w: dict, rbo: int, nsup: int, data) -> dict:
    """Compare the persisted super-chunks in `data` (host bytes, nsup
    super-chunks from block offset rbo) with the reference's digests in
    tests/golden/configs.json (made by the reference's own CPU labeler):
    'bit-exact' when every covered super-chunk matches, 'mismatch' otherwise,
    'unchecked' when no digest covers this range."""
    import hashlib
    path = os.path.join(ROOT, "tests", "golden", "configs.json")
    g = json.load(open(path)).get(w["name"].split(" ")[0]) if os.path.exists(path) else None
    cb = w["chunk_blocks"]
    sb = cb * 32
    if not g or g["key"] != w["key"].hex() or g["chunk_blocks"] != cb or (rbo - g["rbo"]) % cb:
        return {"parity": "unchecked", "checked_super_chunks": 0}
    first = (rbo - g["rbo"]) // cb
    digests = g["super_chunk_sha256"]
    idx = [j for j in range(nsup) if 0 <= first + j < len(digests)]
    if not idx:
        return {"parity": "unchecked", "checked_super_chunks": 0}
    mv = memoryview(data)
    bad = [j for j in idx if hashlib.sha256(mv[j * sb:(j + 1) * sb]).hexdigest() != digests[first + j]]
    return {"parity": "mismatch" if bad else "bit-exact", "checked_super_chunks": len(idx),
            "mismatched_super_chunks": bad[:8]}


def run_reference_arm(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    load_pkg()
    w = workload(args.workload)
    # every step is a bounded sample (one super-chunk per host thread, about
    # 2 s), so the requested K and W are run as given
    steps = max(1, args.steps)
    warm = max(0, args.warmup)
    cb = cpu_reference(w, steps, warm)
    line = {"metric": "label MiB/s (persisted output-set bytes / time)", "value": cb["value"],
            "unit": "MiB/s", "n_gpus": args.gpus, "steps": steps, "warmup": warm,
            "ms_per_step": cb["seconds_per_step"] * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic (splitmix64 session keys)",
            "impl": "reference",
            "config": {"workload": w["name"], "chunk_blocks": w["chunk_blocks"], "super_chunks": w["chunks"],
                       "parallelism": "host threads"},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": "MiB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if w["name"] == "plain_2e17" and not args.no_aux:
        line["reference_gpu_warp_sm100"] = reference_gpu_warp(w)
    print(json.dumps(line), flush=True)


def reference_gpu_warp(w: dict) -> dict:
    """The reference's own CUDA "warp" strategy built for sm_100 from its
    sources (oracle/_ref/libposeref_warp.so, `make -C oracle ref_gpu`), timed
    on this GPU by oracle/ref_gpu_bench.py in its own process (it exports the
    same C symbols as libpose_b200.so): the workload's 32 super-chunks with
    their digests checked, and the reference's default 16 GiB window."""
    so = os.path.join(ROOT, "oracle", "_ref", "libposeref_warp.so")
    if not os.path.exists(so):
        return {"unavailable": "oracle/_ref/libposeref_warp.so not built"}
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no GPU"}
    except ImportError:
        return {"unavailable": "torch absent"}
    out = {"build": "common/src/cuda label_gpu_common.cu + label_gpu_warp.cu + blake3_node.cu, "
                    "-gencode arch=compute_100,code=sm_100, POSE_GPU_WARP_MIN_BLOCKS=3"}
    script = os.path.join(ROOT, "oracle", "ref_gpu_bench.py")
    for name, chunks, extra in (("plain_2e17", w["chunks"], ["--check", "--reps", "2"]),
                                ("window_2e17", 4096, ["--reps", "1"])):
        try:
            with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
                r = subprocess.run([sys.executable, script, "--chunks", str(chunks), "--chunk-blocks",
                                    str(w["chunk_blocks"]), *extra], capture_output=True, text=True, timeout=600,
                                   env=dict(os.environ, POSE_GPU_QUIET="1"))
            lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
            if r.returncode != 0 or not lines:
                out[name] = {"unavailable": f"rc={r.returncode}: {r.stderr.strip()[-300:]}"}
                continue
            d = json.loads(lines[-1])
            d["clocks"] = clk.summary()
            out[name] = d
        except subprocess.TimeoutExpired:
            out[name] = {"unavailable": "timed out after 600 s"}
    return out


# ── B200 arm ────────────────────────────────────────────────────────────────

def run_window(pkg, torch, topo, rate: float, reps: int = 1) -> dict:
    """A full reference-sized HBM window at chunk_blocks 2^17: 4096
    super-chunks (16 GiB, the default window of disk-wipe-bench), key
    splitmix64(1), from absolute position 0 — the throughput regime, where the
    INT32 roofline binds."""
    w = workload("window_2e17")
    nbytes = w["chunks"] * w["chunk_blocks"] * 32
    buf = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    # warm-up: the timed-trial autotuner picks this window's schedule, which
    # the timed pose_graph_hbm_topo_label calls below then use
    rc, chosen, _ = topo.autotune(w["key"], buf.data_ptr(), nbytes, 0, trials=10)
    assert rc == 0, pkg.last_error()
    best = None
    for _ in range(reps):
        rc, st = topo.label(w["key"], buf.data_ptr(), nbytes, 0, stats=True)
        assert rc == 0, pkg.last_error()
        if best is None or st["total_ms"] < best["total_ms"]:
            best = st
    # its first 32 super-chunks are the plain workload's: check them against
    # the reference's digests
    first = 32 * w["chunk_blocks"] * 32
    par = golden_parity(dict(w, name="plain_2e17"), 0, 32, buf[:first].cpu().numpy())
    del buf
    comps = 2 if best["used_cv0_table"] else 3
    achieved = best["nodes"] * comps * 680.0 / (best["kernel_ms"] * 1e-3)
    peak = rate * 680.0
    return {"workload": "window_2e17: 4096 super-chunks of chunk_blocks 2^17 (16 GiB), key splitmix64(1)",
            "value": nbytes / MIB / (best["total_ms"] * 1e-3), "unit": "MiB/s", "ms": best["total_ms"],
            "kernel_ms": best["kernel_ms"], "kernel": best["kernel"],
            "schedule": {"T": best["team_warps"], "G": best["units_per_team"], "teams": best["teams"],
                         "chosen_by": "pose_b200_topo_autotune (10 timed trials)"},
            "roofline": {"bound": "int32", "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "Tops/s",
                         "frac": achieved / peak,
                         "ops_per_node": comps * 680.0},
            "parity": par["parity"], "parity_checked_super_chunks": par["checked_super_chunks"]}


def run_plain_leg(pkg, torch, name: str, rate: float, lat_cycles: float, warm: int = 1, reps: int = 2) -> dict:
    """One more plain workload through pose_graph_hbm_topo_label with its
    topology resident (its scratch cap, if any, on every call): best of
    `reps` timed calls after `warm` untimed ones, its bytes checked against
    the reference's digests, clocks sampled during the timed calls."""
    w = workload(name)
    cb, nsup = w["chunk_blocks"], w["chunks"]
    nbytes = nsup * cb * 32
    cap = pkg.Sched(scratch_cap_bytes=w["scratch_cap_bytes"]) if w.get("scratch_cap_bytes") else None
    topo = pkg.Topology(cb)
    buf = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    for _ in range(warm):
        assert topo.label(w["key"], buf.data_ptr(), nbytes, w["rbo"], sched=cap) == 0, pkg.last_error()
    best = None
    with ClockSampler(torch.cuda.current_device()) as clk:
        for _ in range(reps):
            rc, st = topo.label(w["key"], buf.data_ptr(), nbytes, w["rbo"], sched=cap, stats=True)
            assert rc == 0, pkg.last_error()
            if best is None or st["total_ms"] < best["total_ms"]:
                best = st
    torch.cuda.synchronize()
    par = golden_parity(w, w["rbo"], nsup, buf.cpu().numpy())
    levels = topo.info()["levels"]
    topo.free()
    del buf
    comps = 2 if best["used_cv0_table"] else 3
    clocks = clk.summary()
    sm_hz = (clocks.get("sm_mhz") or 1965.0) * 1e6
    t_depth = levels * comps * lat_cycles / sm_hz
    achieved = best["nodes"] * comps * 680.0 / (best["kernel_ms"] * 1e-3)
    out = {"workload": f"{name}: {nsup} super-chunks of chunk_blocks {cb}, key splitmix64",
           "value": nbytes / MIB / (best["total_ms"] * 1e-3), "unit": "MiB/s", "ms": best["total_ms"],
           "kernel_ms": best["kernel_ms"], "kernel": best["kernel"],
           "schedule": {"T": best["team_warps"], "G": best["units_per_team"], "teams": best["teams"],
                        "scratch_bytes": best["scratch_bytes"]},
           "scratch_cap_bytes": w.get("scratch_cap_bytes"),
           "roofline": {"bound": "int32", "achieved": achieved / 1e12, "peak": rate * 680.0 / 1e12,
                        "unit": "Tops/s", "frac": achieved / (rate * 680.0),
                        "depth_bound_mib_s": nbytes / MIB / t_depth,
                        "depth_frac": t_depth * 1e3 / best["kernel_ms"]},
           "clocks": clocks}
    out.update(par)
    return out


def run_batched(pkg, torch, sched=None, reps: int = 2) -> dict:
    """The batched workload (256 sessions, chunk_blocks 2^12..2^17, 1-8 chunks
    each at random absolute positions) through one persistent launch replayed
    from a captured CUDA graph; MiB/s over the graph's device time."""
    import pose_b200.workloads as wl
    sessions = wl.batched()
    topos = {cb: pkg.Topology(cb) for cb in sorted({s["chunk_blocks"] for s in sessions})}
    total = sum(s["chunk_blocks"] * 32 * len(s["chunk_indices"]) for s in sessions)
    big = torch.empty(total, dtype=torch.uint8, device="cuda")
    reqs, off = [], 0
    for s in sessions:
        for idx in s["chunk_indices"]:
            cb = s["chunk_blocks"]
            reqs.append((topos[cb], s["key"], big.data_ptr() + off, cb * 32, idx * cb))
            off += cb * 32
    best = None
    with pkg.Batch(reqs, sched, autotune=0 if sched is not None else 3) as b:
        chosen = b.chosen
        b.run()  # warm-up replay
        for _ in range(reps):
            rc, st = b.run()
            assert rc == 0
            if best is None or st["total_ms"] < best["total_ms"]:
                best = st
    for t in topos.values():
        t.free()
    return {"workload": "batched: 256 sessions x 1-8 chunks, chunk_blocks 2^12..2^17",
            "value": total / MIB / (best["total_ms"] * 1e-3), "unit": "MiB/s",
            "graph_ms": best["total_ms"], "super_chunks": best["super_chunks"], "units": best["units"],
            "nodes": best["nodes"], "teams": best["teams"], "team_warps": best["team_warps"],
            "max_units_per_team": best["units_per_team"], "kernel_launches_per_replay": best["kernel_launches"],
            "schedule": "autotuned" if chosen else "given",
            "packing": None if not chosen else ("chain-bounded" if chosen["lane_efficiency"] == pkg.PACK_CHAIN
                                                 else f"lane efficiency {chosen['lane_efficiency']}%")}


def run_served(pkg, torch, requests: int = 300, alone: bool = False, rate: float = 200.0) -> dict:
    """Replay a fixed Poisson trace (200 requests/s from 64 sessions,
    chunk_blocks 2^10..2^18, 1-16 chunks each) in real time against the
    continuous-batching server; latency = submit to completion.  With alone,
    the same requests also run one at a time (FIFO, each through
    pose_graph_hbm_topo_label, latency = queueing on the same arrival times +
    its measured service time)."""
    import threading
    import pose_b200.workloads as wl
    trace = wl.served(requests, rate_per_s=rate)
    topos = {cb: pkg.Topology(cb) for cb in sorted({r["chunk_blocks"] for r in trace})}
    sizes = [r["chunks"] * r["chunk_blocks"] * 32 for r in trace]
    big = torch.empty(sum(sizes), dtype=torch.uint8, device="cuda")
    offs, o = [], 0
    for sz in sizes:
        offs.append(o)
        o += sz
    keys = {r["session"]: r["key"] for r in trace}
    lat = [0.0] * len(trace)
    with pkg.Server(scratch_bytes=32 << 30) as srv:  # the library's default wave count
        sid = {s: srv.session(k) for s, k in keys.items()}
        for t in topos.values():  # set-up, before the trace: the depth kernel's records
            srv.prepare(t)
        tickets = [None] * len(trace)
        t0 = time.perf_counter()

        def feeder():
            for i, r in enumerate(trace):
                d = r["arrival_s"] - (time.perf_counter() - t0)
                if d > 0:
                    time.sleep(d)
                tickets[i] = srv.submit(topos[r["chunk_blocks"]], sid[r["session"]], big.data_ptr() + offs[i],
                                        sizes[i], r["first_chunk"] * r["chunk_blocks"])

        th = threading.Thread(target=feeder)
        th.start()
        th.join()
        for i, tk in enumerate(tickets):
            rc, q, tot = srv.wait(tk)
            assert rc == 0
            lat[i] = tot
        wall = time.perf_counter() - t0
        st = srv.stats()
    lat_sorted = sorted(lat)
    out = {"workload": f"served: Poisson {rate:.4g} req/s, 64 sessions, {len(trace)} requests, chunk_blocks 2^10..2^18",
           "value": sum(sizes) / MIB / wall, "unit": "MiB/s", "p50_ms": lat_sorted[len(lat) // 2],
           "p99_ms": lat_sorted[min(len(lat) - 1, int(0.99 * len(lat)))], "waves": st["waves"],
           "offered_mib_s": sum(sizes) / MIB / trace[-1]["arrival_s"], "wall_s": wall,
           "policy": "chunk_blocks 2^17 and up on the depth kernel (3 copies per CTA, SM held alone), "
                     "the rest in up to 5 concurrent lockstep waves (3 with fewer than 16 work queues)",
           "work_queues": int(os.environ.get("CUDA_DEVICE_MAX_CONNECTIONS", "8"))}
    if alone:
        # one request at a time, FIFO, on the same arrival times
        sub = trace
        clock = 0.0
        lat1 = []
        for i, r in enumerate(sub):
            start = max(clock, r["arrival_s"])
            torch.cuda.synchronize()
            a = time.perf_counter()
            rc = topos[r["chunk_blocks"]].label(r["key"], big.data_ptr() + offs[i], sizes[i],
                                                r["first_chunk"] * r["chunk_blocks"])
            torch.cuda.synchronize()
            svc = time.perf_counter() - a
            assert rc == 0
            clock = start + svc
            lat1.append((clock - r["arrival_s"]) * 1e3)
        l1 = sorted(lat1)
        out["one_at_a_time"] = {"requests": len(sub), "value": sum(sizes) / MIB / clock, "unit": "MiB/s",
                                "p50_ms": l1[len(l1) // 2], "p99_ms": l1[min(len(l1) - 1, int(0.99 * len(l1)))]}
    for t in topos.values():
        t.free()
    return out


def run_b200(args) -> None:
    import torch
    pkg = load_pkg()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    os.environ.setdefault("POSE_GPU_QUIET", "1")
    w = workload(args.workload)
    if args.chunks:
        w = dict(w, chunks=args.chunks, name=f"{w['name']} ({args.chunks} super-chunks)")
    cb, nsup = w["chunk_blocks"], w["chunks"]
    sb = cb * 32
    nbytes = nsup * sb
    import pose_b200.workloads as wl
    rbo, nsup = wl.rank_region(w, rank, world)  # each rank: its own disjoint absolute range

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    topo = pkg.Topology(cb, cv0_table=not args.no_cv0)
    buf = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    host = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)

    # roofline denominator: the GPU's compression rate for this instruction mix
    rate, lat_cycles = pkg.compress_rate(2048)

    # a workload with a scratch cap runs every call under it; otherwise the
    # timed-trial autotuner fixes this call size's schedule during warm-up
    # (the timed calls are plain pose_graph_hbm_topo_label calls that reuse it)
    cap = pkg.Sched(scratch_cap_bytes=w["scratch_cap_bytes"]) if w.get("scratch_cap_bytes") else None
    if cap is None:
        rc, _, _ = topo.autotune(w["key"], buf.data_ptr(), nbytes, rbo, trials=3)
        assert rc == 0, pkg.last_error()
    for _ in range(args.warmup):
        rc = topo.label(w["key"], buf.data_ptr(), nbytes, rbo, sched=cap)
        assert rc == 0, pkg.last_error()

    stats = []
    barrier()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            rc, st = topo.label(w["key"], buf.data_ptr(), nbytes, rbo, sched=cap, stats=True)
            assert rc == 0, pkg.last_error()
            stats.append(st)
        barrier()
        # end to end through the public API with host buffers: the session key
        # goes host->device inside the call, the persisted labels come back
        # into pinned host memory
        e2e_times = []
        for _ in range(max(1, args.steps)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rc = topo.label(w["key"], buf.data_ptr(), nbytes, rbo, sched=cap)
            host.copy_(buf, non_blocking=False)
            torch.cuda.synchronize()
            e2e_times.append(time.perf_counter() - t0)
            assert rc == 0
        barrier()
    # the bytes of the last timed call and of the last end-to-end host copy,
    # against the reference's digests
    par_dev = golden_parity(w, rbo, nsup, buf.cpu().numpy())
    par_host = golden_parity(w, rbo, nsup, host.numpy())
    device_ms = sum(s["total_ms"] for s in stats)
    kernel_ms = sum(s["kernel_ms"] for s in stats) / len(stats)
    e2e_s = sum(e2e_times) / len(e2e_times)
    if dist:
        t = torch.tensor([device_ms, e2e_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        device_ms, e2e_s = float(t[0]), float(t[1])
    ms_per_step = device_ms / args.steps
    value = world * nbytes / MIB / (ms_per_step * 1e-3)
    e2e_value = world * nbytes / MIB / e2e_s
    st0 = stats[0]
    comps = 2 if st0["used_cv0_table"] else 3
    nodes = st0["nodes"]
    ops_per_compress = 680.0  # 7 rounds x 8 G x 12 int32 ops + 8 output xors
    achieved_ops = nodes * comps * ops_per_compress / (kernel_ms * 1e-3)
    peak_ops = rate * ops_per_compress
    info = topo.info()
    levels = info["levels"]
    traffic = profiled_traffic(w["name"], st0["kernel"]) if not args.chunks else None
    hbm_gbs = measured_hbm_gbs()
    clocks = clk.summary()
    # depth bound: one label per level on the critical path, each ~comps
    # dependent compressions at the measured compression latency
    sm_hz = (clocks.get("sm_mhz") or 1965.0) * 1e6
    t_depth = levels * comps * lat_cycles / sm_hz
    line = {
        "metric": "label MiB/s (persisted output-set bytes / time)",
        "value": value, "unit": "MiB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic (splitmix64 session keys)", "impl": "b200",
        "config": {"workload": w["name"], "chunk_blocks": cb, "super_chunks": nsup,
                   "nodes_per_step": nsup * w["nodes_per_chunk"], "parallelism": f"chunk-sharded x{world}",
                   "l2": "inputs larger than L2 (topology store %.2f GB read per step)" % (info["device_bytes"] / 1e9),
                   "schedule": {"T": st0["team_warps"], "G": st0["units_per_team"], "teams": st0["teams"],
                                "kernel": st0["kernel"], "scratch_bytes": st0["scratch_bytes"]},
                   "scratch_cap_bytes": w.get("scratch_cap_bytes"),
                   "cv0_table": bool(st0["used_cv0_table"])},
        "roofline": {"bound": "int32", "achieved": achieved_ops / 1e12, "peak": peak_ops / 1e12,
                     "unit": "Tops/s", "frac": achieved_ops / peak_ops, "traffic": traffic,
                     "traffic_source": "profiles/: ncu dram__bytes_read.sum + dram__bytes_write.sum per launch"
                                       if traffic is not None else None,
                     "dram_gbs": traffic / (kernel_ms * 1e-3) / 1e9 if traffic is not None else None,
                     "hbm_peak_gbs": hbm_gbs,
                     "dram_frac_of_hbm_peak": traffic / (kernel_ms * 1e-3) / 1e9 / hbm_gbs
                     if traffic is not None and hbm_gbs else None,
                     "peak_source": "measured in this run: k_compress_bench (every SM full, register-resident compressions)",
                     "ops_per_node": comps * ops_per_compress,
                     "spec_ops_per_node": 3 * ops_per_compress,
                     "depth_bound_mib_s": nsup * sb / MIB / t_depth if t_depth > 0 else None,
                     "depth_frac": (t_depth * 1e3) / kernel_ms if kernel_ms > 0 else None,
                     "compress_latency_cycles": lat_cycles},
        "e2e": {"value": e2e_value, "unit": "MiB/s", "h2d_bytes_per_step": len(w["key"]),
                "d2h_bytes_per_step": nbytes},
        "parity": "mismatch" if "mismatch" in (par_dev["parity"], par_host["parity"]) else par_dev["parity"],
        "parity_checked": {"timed_output": par_dev, "e2e_host_copy": par_host,
                           "against": "tests/golden/configs.json: per-super-chunk SHA-256 of the reference's "
                                      "own CPU labeler on the same key and positions (rank 0's range)"},
        "gpu_launches": int(sum(2 * s["kernel_launches"] for s in stats)),
        "clocks": clocks,
        "kernel_ms": kernel_ms,
    }
    if world == 1 and not args.no_aux and args.workload == "plain_2e17":
        for key, fn in (("window_2e17", lambda: run_window(pkg, torch, topo, rate)),
                        ("batched", lambda: run_batched(pkg, torch)),
                        ("served", lambda: run_served(pkg, torch, requests=120, alone=True))):
            with ClockSampler(local) as aclk:
                line[key] = fn()
            line[key]["clocks"] = aclk.summary()
        # the same trace shape below saturation: arrivals at about 0.7 of the
        # served rate measured above
        sv = line["served"]
        low_rate = 200.0 * 0.7 * sv["value"] / sv["offered_mib_s"]
        with ClockSampler(local) as aclk:
            line["served_0p7"] = run_served(pkg, torch, requests=120, rate=low_rate)
        line["served_0p7"]["clocks"] = aclk.summary()
        line["deep_2e20"] = run_plain_leg(pkg, torch, "deep_2e20", rate, lat_cycles, warm=1, reps=2)
        line["plain_small"] = run_plain_leg(pkg, torch, "plain_small", rate, lat_cycles, warm=3, reps=5)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_reference(w, 3, 1)
            line["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as exc:  # the oracle's reference build may be absent
            line["cpu_baseline"] = {"value": None, "unit": "MiB/s", "cores": os.cpu_count(), "kind": "reference",
                                    "sample": f"unavailable: {exc}"}
    topo.free()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if line["parity"] == "mismatch":
        raise SystemExit("bench: labels differ from the reference's digests")


def run_aux(args) -> None:
    """--workload batched | served: one JSON line for that form alone."""
    import torch
    pkg = load_pkg()
    os.environ.setdefault("POSE_GPU_QUIET", "1")
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if args.workload == "batched":
        r = run_batched(pkg, torch, reps=max(1, args.steps))
    else:
        r = run_served(pkg, torch, requests=args.requests, alone=args.alone)
    r.update({"metric": "label MiB/s", "n_gpus": 1, "impl": "b200", "data": "synthetic (splitmix64 session keys)"})
    print(json.dumps(r), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="plain_2e17")
    ap.add_argument("--chunks", type=int, default=0, help="override the workload's super-chunk count (profiling)")
    ap.add_argument("--no-cv0", action="store_true", help="hash block 0 in every call (no table)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-aux", action="store_true", help="skip the batched and served legs")
    ap.add_argument("--requests", type=int, default=300, help="served: trace length")
    ap.add_argument("--alone", action="store_true", help="served: also run the trace one request at a time")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.workload in ("batched", "served"):
        run_aux(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
