"""Benchmark of the streaming k-mer table's hot path on B200: k-mers/s of upsert + find.

Workload (one step): a map <31, u64, 22> sized for n = 10M keys, emptied, then upsert(c + 1, init 1) of 333,333 reads
of 150 bp (10x over a seeded 5 Mbp genome, 50 % reverse-complemented, 0.5 % substitutions, 0.05 % N), then a
per-position lookup (found + value) of 1M held-out reads of the same model. Unit: k-mer positions per second over
both phases (40.0M + 120.0M positions). Synthetic data stands in for the reference's read sets.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

`value` times the device-resident path (reads already in HBM, kache_b200_upsert_dev / kache_b200_lookup_dev);
`e2e` times the C interface with host buffers (kache_insert / kache_lookup: gather + H2D + kernels + D2H of the
per-position results). With N > 1 each rank runs its own table on its own reads (weak scaling, no collective:
tables are independent objects). `--impl reference` times the reference's own CPU table (oracle/_ref) on the same
workload with all host threads.
"""
import argparse
import ctypes
import json
import os
import re
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "kache-hash_b200"), os.path.join(ROOT, "tests")]

import numpy as np  # noqa: E402

import synth  # noqa: E402

METRIC = "k-mers/s upsert+find (config 1: <31,u64,22> n=10M, 333,333 x 150 bp upsert(c+1) + 1M held-out reads find)"
N_KEYS = 10_000_000


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """SM clock and clock-event reasons sampled through NVML (read-only queries) every 10 ms during the timed region,
    from a thread of this process: the library is initialised before the region starts, so nothing starts up inside
    it. Reports "unavailable" without NVML."""

    NAMES = [("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"), ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
             ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"), ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap")]

    def __init__(self, device):
        import torch
        self.rows, self.h, self.run = [], None, False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            try:
                self.h = pynvml.nvmlDeviceGetHandleByUUID("GPU-" + str(torch.cuda.get_device_properties(device).uuid))
            except Exception:
                self.h = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.h = None

    def _sample(self):
        nv = self.nv
        while self.run:
            try:
                self.rows.append((nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM),
                                  nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)))
            except Exception:
                pass
            time.sleep(0.01)

    def start(self):
        if self.h is None:
            return
        self.run = True
        self.t = threading.Thread(target=self._sample, daemon=True)
        self.t.start()

    def stop(self):
        if self.h is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"]}
        self.run = False
        self.t.join()
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["no samples"]}
        sm = sorted(r[0] for r in self.rows)
        reasons = sorted({name for _, mask in self.rows for name, const in self.NAMES if mask & getattr(self.nv, const)})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": self.max_mhz, "reasons": reasons, "samples": len(self.rows),
                "source": "nvml, 10 ms"}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def rank_seeds(rank):
    """The read seeds of a rank: rank 0 runs the workload itself; each other rank its own reads of the same shape,
    into its own table (weak scaling over independent tables)."""
    return (11, 2) if rank == 0 else (11 + 100 * rank, 2 + 100 * rank)


def workload(rank, scale=1.0):
    g, ins, held = synth.config1(scale)
    if rank:
        s_ins, s_held = rank_seeds(rank)
        ins = synth.reads_fixed(g, int(333_333 * scale), 150, seed=s_ins)
        held = synth.reads_fixed(g, int(1_000_000 * scale), 150, seed=s_held)
    return ins, held


def max_over_ranks(dist, x, device):
    """The largest of the ranks' values (the job's time is its slowest rank's)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def ncu_traffic(kernel):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the kernel on this workload, from the
    committed ncu summary under profiles/, or None."""
    name = {"lookup": "lookup_stream_kernel_config1.md", "upsert": "upsert_lane_kernel_config1.md"}.get(kernel)
    try:
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles", name)) as f:
            m = re.search(r"\| dram bytes per launch \| (\d+) \|", f.read())
        return int(m.group(1)) if m else None
    except (OSError, TypeError):
        return None


def random_roofs(kache, nbytes=1 << 30):
    """The device's random-access roofs (kache_b200_memory_roof): 32-byte sector reads and atomic updates at random
    over `nbytes`, and the dependent-load latency."""
    try:
        _, rd = kache.memory_roof(nbytes, kache.ROOF_RANDOM_READ, 1 << 28)
        _, up = kache.memory_roof(nbytes, kache.ROOF_RANDOM_UPDATE, 1 << 28)
        _, seq = kache.memory_roof(nbytes, kache.ROOF_SEQ_READ, 0)
        threads, per = 148 * 32, 256
        ms, ch = kache.memory_roof(nbytes, kache.ROOF_CHASE, threads * per)
        return {"array_bytes": nbytes, "read_sectors_per_s": rd, "read_gbs": rd * 32 / 1e9, "update_per_s": up,
                "update_gbs_rmw": up * 64 / 1e9, "seq_read_gbs": seq / 1e9, "chase_latency_ns": 1e6 * ms / per}
    except Exception as e:  # noqa: BLE001
        return {"error": str(e)}


def positions(off, k=31):
    lens = np.diff(off).astype(np.int64)
    return int(np.maximum(lens - k + 1, 0).sum())


def cpu_baseline_sample(ins, held, threads):
    """The reference's own table (oracle/_ref) on a bounded sample of the same workload: a tenth of the upsert reads
    into a table sized for a tenth of the keys, then per-position finds over a tenth of the held-out reads."""
    import oracle
    L = oracle.ref()
    if L is None:
        return None
    from kache import Batch
    bi, bh = Batch(*ins), Batch(*held)
    si, sh = bi.slice(0, bi.n // 10), bh.slice(0, bh.n // 10)
    t = L.ref_new(0, N_KEYS // 10, 0.8, 0, threads)
    out = oracle._u64()
    t_up = L.ref_bench_upsert(t, si.bases.ctypes.data, si.off.ctypes.data, si.n, 64, threads, 16, 1, oracle.ctypes.byref(out))
    t_q = ref_lookup_timed(L, t, sh, threads)
    L.ref_free(t)
    p = positions(si.off) + positions(sh.off)
    return {"value": p / (t_up + t_q), "unit": "k-mers/s", "cores": threads, "kind": "reference",
            "sample": f"upsert {si.n} reads + per-position find over {sh.n} held-out reads ({p} positions), batches of 64 reads, {threads} threads"}


def ref_lookup_timed(L, t, b, threads, k=31):
    """Seconds for the reference's per-position find over batch b (found flags and values into host arrays, as
    kache_lookup returns them)."""
    lens = np.diff(b.off).astype(np.int64)
    pos_off = np.zeros(b.n + 1, np.uint64)
    np.cumsum(np.maximum(lens - k + 1, 0), out=pos_off[1:])
    P = int(pos_off[-1])
    found = np.zeros(max(P, 1), np.uint8)
    vals = np.zeros(max(P, 1), np.uint64)
    return L.ref_bench_lookup(t, b.bases.ctypes.data, b.off.ctypes.data, b.n, pos_off.ctypes.data, 64, threads,
                              found.ctypes.data, vals.ctypes.data)


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    import oracle
    L = oracle.ref()
    if L is None:
        print(json.dumps({"impl": "reference", "unavailable": "the reference's table (oracle/_ref) was not built on this machine"}))
        return
    from kache import Batch
    ins, held = workload(0)
    bi, bh = Batch(*ins), Batch(*held)
    threads = min(128, os.cpu_count() or 1)
    P = positions(bi.off) + positions(bh.off)
    out = oracle._u64()
    times = []
    for s in range(args.warmup + args.steps):
        t = L.ref_new(0, N_KEYS, 0.8, 0, threads)
        t_up = L.ref_bench_upsert(t, bi.bases.ctypes.data, bi.off.ctypes.data, bi.n, 64, threads, 16, 1, oracle.ctypes.byref(out))
        t_q = ref_lookup_timed(L, t, bh, threads)
        L.ref_free(t)
        if s >= args.warmup:
            times.append(t_up + t_q)
    T = sum(times)
    v = P * args.steps / T
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "k-mers/s", "n_gpus": ws, "steps": args.steps,
                      "warmup": args.warmup, "ms_per_step": 1000 * T / args.steps, "higher_is_better": True, "scaling": "weak",
                      "vs_baseline": None, "dtype": "u64", "data": "synthetic",
                      "config": {"workload": "config 1: <31,u64,22> n=10M; upsert(c+1, init 1) 333,333 x 150 bp; find 1M x 150 bp held-out",
                                 "upsert_positions": positions(bi.off), "find_positions": positions(bh.off), "find": "per-position found flag and value"},
                      "cpu_baseline": {"value": v, "unit": "k-mers/s", "cores": threads, "kind": "reference",
                                       "sample": "the whole workload per step (upsert, then per-position find), batches of 64 reads round-robin over the threads"},
                      "e2e": {"value": v, "unit": "k-mers/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def pcie_floor(d_found, d_vals, t_found, t_vals, d_bases, t_bases, reps=3):
    """This box's copy floor for the end-to-end step: the find output (found flags and values) copied device to host
    into the same page-locked buffers, and the find's reads host to device, as plain copies with nothing else running
    (the fastest of `reps`)."""
    import torch
    s = torch.cuda.Stream()

    def once(f):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with torch.cuda.stream(s):
            f()
        s.synchronize()
        return 1e3 * (time.perf_counter() - t0)

    def out():
        t_found.copy_(d_found, non_blocking=True)
        t_vals.copy_(d_vals.view(torch.uint8), non_blocking=True)

    d2h = min(once(out) for _ in range(reps))
    h2d = min(once(lambda: d_bases.copy_(t_bases, non_blocking=True)) for _ in range(reps))
    out_bytes = d_found.numel() + d_vals.numel() * d_vals.element_size()
    return {"d2h_ms": d2h, "d2h_gbs": out_bytes / d2h / 1e6, "h2d_ms": h2d, "h2d_gbs": t_bases.numel() / h2d / 1e6,
            "form": "the find output device to host and the find's reads host to device, plain copies on this box"}


def run_b200(args):
    import torch
    import kache
    from kache import Batch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    ins, held = workload(rank)
    bi, bh = Batch(*ins), Batch(*held)
    P_up, P_find = positions(bi.off), positions(bh.off)
    P = P_up + P_find
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()

    d_ins_b = torch.from_numpy(bi.bases).to(dev)
    d_ins_o = torch.from_numpy(bi.off.view(np.int64)).to(dev)
    d_held_b = torch.from_numpy(bh.bases).to(dev)
    d_held_o = torch.from_numpy(bh.off.view(np.int64)).to(dev)
    d_found = torch.empty(P_find, dtype=torch.uint8, device=dev)
    d_vals = torch.empty(P_find, dtype=torch.int64, device=dev)

    T = kache.Table(31, 8, N_KEYS, 0.8, False)
    T.set_stream(stream.cuda_stream)
    u = T.register()

    def step_dev():
        T.clear()
        T.upsert_dev(u, d_ins_b.data_ptr(), d_ins_o.data_ptr(), bi.n, kache.ADD_WRAP, 1, 1)
        T.lookup_dev(d_held_b.data_ptr(), d_held_o.data_ptr(), bh.n, d_found.data_ptr(), d_vals.data_ptr(), None)

    # End-to-end buffers: the reads and the lookup outputs in page-locked host memory, which the library copies
    # to and from directly.
    def pinned(a):
        t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
        v = t.numpy().view(a.dtype)
        v[:] = a
        return t, v

    keep = []
    def pinned_batch(b):
        t, v = pinned(b.bases)
        keep.append(t)
        return Batch(v, b.off)

    pi, ph = pinned_batch(bi), pinned_batch(bh)
    t_held = keep[-1]   # The held-out reads' page-locked bases.
    t_f, found_h = pinned(np.zeros(P_find, np.uint8))
    t_v, vals_h = pinned(np.zeros(P_find, np.uint64))
    found_pg, vals_pg = np.zeros(P_find, np.uint8), np.zeros(P_find, np.uint64)

    e2e_parts = {"clear": 0.0, "insert": 0.0, "lookup": 0.0}

    def step_e2e(ins=pi, held=ph, found=found_h, vals=vals_h):
        t0 = time.perf_counter()
        T.clear()
        t1 = time.perf_counter()
        kache.lib().kache_insert(T.h, u, *ins.args(), kache.ADD, 1, None)
        t2 = time.perf_counter()
        kache.lib().kache_lookup(T.h, *held.args(), found.ctypes.data, vals.ctypes.data, None)
        t3 = time.perf_counter()
        e2e_parts["clear"] += t1 - t0
        e2e_parts["insert"] += t2 - t1
        e2e_parts["lookup"] += t3 - t2

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # Device-resident: warm-up, then exactly `steps` steps between barriers, timed with CUDA events on the stream.
    for _ in range(args.warmup):
        step_dev()
    barrier()
    clocks = Clocks(local) if not args.only_dev else None
    if clocks is not None:
        clocks.start()
    launches0 = kache.kernel_launches()
    T.profile(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step_dev()
    e1.record(stream)
    barrier()
    ms = max_over_ranks(dist, e0.elapsed_time(e1), dev) / args.steps
    launches = kache.kernel_launches() - launches0
    prof = {kind: T.profile_read(i) for i, kind in enumerate(["upsert", "update", "lookup", "reduce", "resize", "other"])}
    T.profile(False)
    clk = clocks.stop() if clocks is not None else None

    # Per-kernel roofline: algorithmic bytes per launch over the kernel's mean event-timed duration.
    st = T.stats()
    inserted = T.size()
    fh = d_found.cpu().numpy()
    hit = float((fh == 1).sum()) / max(1, P_find)
    rho = run_density(kache, bi.slice(0, 5000)) if rank == 0 else 0.0
    b_in_up = float(bi.off[-1]) / P_up
    b_in_find = float(bh.off[-1]) / P_find
    A_up = b_in_up + 32 * rho + 32 * (1 - inserted / P_up) + 32 * 1.0
    A_find = b_in_find + 9 + 32 * rho + 32 * hit
    up_ms, up_n = prof["upsert"]
    lk_ms, lk_n = prof["lookup"]
    peak, peak_kind = load_peaks()
    kernels = {
        "upsert": {"launches": up_n, "ms_total": up_ms, "bytes_per_launch": A_up * P_up / max(1, up_n / args.steps),
                   "algorithmic_bytes_per_kmer": A_up},
        "lookup": {"launches": lk_n, "ms_total": lk_ms, "bytes_per_launch": A_find * P_find / max(1, lk_n / args.steps),
                   "algorithmic_bytes_per_kmer": A_find},
    }
    for kv in kernels.values():
        kv["achieved_gbs"] = kv["bytes_per_launch"] / (kv["ms_total"] / max(1, kv["launches"]) * 1e-3) / 1e9 if kv["ms_total"] else None
    # The random-access roofline: a launch's streamed bytes at the copy peak plus its random slot-sector reads and
    # updates at the device's measured random-sector rates (kache_b200_memory_roof over a 1 GiB array, larger than the
    # table); the checksum sectors (the 32*rho term) are left out, as the checksum array (25 MB) stays in L2.
    roof = random_roofs(kache) if rank == 0 and not args.only_dev else None
    if roof and "error" not in roof:
        streamed = {"upsert": b_in_up * P_up, "lookup": (b_in_find + 9) * P_find}
        reads = {"upsert": P_up * (1 - inserted / P_up), "lookup": P_find * hit}
        updates = {"upsert": P_up * 1.0, "lookup": 0.0}
        for name_, kv in kernels.items():
            t_roof = streamed[name_] / (peak * 1e9) + reads[name_] / roof["read_sectors_per_s"] + updates[name_] / roof["update_per_s"]
            kv["random_roof_ms"] = 1e3 * t_roof
            kv["frac_of_random_roof"] = (1e3 * t_roof) / (kv["ms_total"] / max(1, kv["launches"])) if kv["ms_total"] else None
    dom = max(kernels, key=lambda k_: kernels[k_]["ms_total"])
    d = kernels[dom]

    # End to end through the C interface with host buffers.
    e2e_ms = e2e_pg_ms = float("nan")
    pcie = None
    parts_pinned, pg_steps = {}, 0
    if not args.only_dev:
        for _ in range(max(1, args.warmup // 2)):
            step_e2e()
        barrier()
        for key_ in e2e_parts:
            e2e_parts[key_] = 0.0
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step_e2e()
        barrier()
        e2e_ms = max_over_ranks(dist, (time.perf_counter() - t0) * 1000, dev) / args.steps
        parts_pinned = {key_: 1000 * v_ / args.steps for key_, v_ in e2e_parts.items()}
        # The same calls with pageable host buffers (a few steps): the library stages them through its own pinned
        # memory.
        pg_steps = max(1, min(args.steps, 5))
        step_e2e(bi, bh, found_pg, vals_pg)
        barrier()
        t0 = time.perf_counter()
        for _ in range(pg_steps):
            step_e2e(bi, bh, found_pg, vals_pg)
        barrier()
        e2e_pg_ms = max_over_ranks(dist, (time.perf_counter() - t0) * 1000, dev) / pg_steps
        pcie = pcie_floor(d_found, d_vals, t_f, t_v, d_held_b, t_held)

    if rank == 0:
        line = {
            "metric": METRIC, "value": P * ws / (ms * 1e-3), "unit": "k-mers/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64", "data": "synthetic",
            "config": {"workload": "config 1: <31,u64,22> n=10M; upsert(c+1, init 1) 333,333 x 150 bp; find 1M x 150 bp held-out",
                       "upsert_positions": P_up, "find_positions": P_find, "keys": inserted, "capacity": st.capacity,
                       "placed_pct": [round(st.primary_pct, 3), round(st.secondary_pct, 3), round(st.overflow_pct, 3)],
                       "l2": "inputs larger than L2 (reads 250 MB + table 240 MB per step)", "parallelism": f"{ws} independent tables"},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": d["achieved_gbs"], "peak": peak, "unit": "GB/s",
                         "frac": (d["achieved_gbs"] / peak) if d["achieved_gbs"] else None, "traffic": ncu_traffic(dom),
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch on this workload (profiles/)",
                         "peak_source": peak_kind, "kernels": kernels, "random_roof": roof,
                         "model": "A = b_in + b_out + 32*rho + 32*r_slot + 32*w_slot bytes per k-mer; rho from the describer on 5000 reads"},
            "e2e": {"value": P * ws / (e2e_ms * 1e-3), "unit": "k-mers/s", "ms_per_step": e2e_ms,
                    # The reads' bases and the offsets the library lists them by (n + 1 words a batch).
                    "h2d_bytes_per_step": int(bi.off[-1] + bh.off[-1] + 8 * (bi.n + 1 + bh.n + 1)),
                    "d2h_bytes_per_step": int(P_find * 9),
                    "host_buffers": "page-locked (reads and outputs)", "ms_per_call": parts_pinned,
                    "pageable": {"value": P * ws / (e2e_pg_ms * 1e-3), "ms_per_step": e2e_pg_ms, "steps": pg_steps},
                    "pcie_floor": pcie},
            "clocks": clk,
        }
        if ws == 1 and not args.only_dev and not args.no_sub:
            # Right after the timed phases, while the GPU's clocks are up (the CPU baseline below leaves it idle).
            line["cold_first_call"] = cold_first_call(dev, stream, d_ins_b.data_ptr(), d_ins_o.data_ptr(), bi.n, d_held_b.data_ptr(),
                                                      d_held_o.data_ptr(), bh.n, d_found.data_ptr(), d_vals.data_ptr(), P)
        # The reference on the host cores, at one GPU only (the other ranks would wait for it).
        cb = None if (args.only_dev or ws > 1) else cpu_baseline_sample(ins, held, min(128, os.cpu_count() or 1))
        line["cpu_baseline"] = cb
        if ws == 1 and not args.only_dev and not args.no_sub:
            line["config3_batched"] = sub_config3(dev, stream, local)
            line["config5_served"] = sub_config5(dev, stream, local)
        print(json.dumps(line))
    T.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_density(kache, b, k=31):
    """Minimizer runs per k-mer position (rho): the share of positions whose minimizer hash differs from the previous
    position's in the same sequence, from the describer."""
    t = kache.Table(k, 0, 1000, capi=(k == 31))
    key, h, cs, fwd, valid = t.describe(b)
    t.close()
    pos = b.positions(k)
    starts = np.zeros(len(h), bool)
    o = np.concatenate([[0], np.cumsum(pos)[:-1]]).astype(np.int64)
    starts[o[pos > 0]] = True
    change = np.ones(len(h), bool)
    change[1:] = h[1:] != h[:-1]
    runs = (change | starts) & (valid == 1)
    return float(runs.sum()) / max(1, int(valid.sum()))


# ---- Sub-records of the default line: the north-star forms beside the headline --------------------------------------

def kernel_roofline(name, ms_total, launches, bytes_per_launch, A, peak, peak_kind):
    """The roofline record of one kernel kind: algorithmic bytes per launch over its mean event-timed duration."""
    per = ms_total / max(1, launches)
    ach = bytes_per_launch / (per * 1e-3) / 1e9 if ms_total else None
    return {"bound": "hbm", "kernel": name, "achieved": ach, "peak": peak, "unit": "GB/s",
            "frac": (ach / peak) if ach else None, "peak_source": peak_kind, "launches": launches, "ms_total": ms_total,
            "algorithmic_bytes_per_kmer": A, "bytes_per_launch": bytes_per_launch, "traffic": None,
            "model": "A = b_in + b_out + 32*rho + 32*r_slot + 32*w_slot bytes per k-mer position"}


def sub_config3(dev, stream, device_index):
    """Config 3 at full size (strand map <27, u8, 16>, oriented upsert OR 1/2 then oriented find of every read), its
    reads in batches of 256 as a caller of the plain per-call interface hands them over: one call per batch and kind
    (the plain kernel), against the same batches as one kache_b200_run_dev_batches call per kind (the batched
    persistent path: one segment list, one launch)."""
    import torch
    import kache
    from kache import Batch
    g, reads = synth.config3()
    br = Batch(*reads)
    P1 = positions(br.off, 27)
    T = kache.Table(27, 1, 50_000_000, 0.8, False, capi=False)
    T.set_stream(stream.cuda_stream)
    u = T.register()
    found = torch.empty(P1, dtype=torch.uint8, device=dev)
    vals = torch.empty(P1, dtype=torch.uint8, device=dev)
    fwd = torch.empty(P1, dtype=torch.uint8, device=dev)
    pieces = dev_pieces(br, dev, 256)
    starts = np.concatenate([[0], np.cumsum([int(np.maximum(np.diff(o_.cpu().numpy()) - 26, 0).sum()) for _, o_, _ in pieces])])
    ups = [(b_.data_ptr(), o_.data_ptr(), n_) for b_, o_, n_ in pieces]
    looks = [(b_.data_ptr(), o_.data_ptr(), n_, found[int(starts[i_]):].data_ptr(), vals[int(starts[i_]):].data_ptr(),
              fwd[int(starts[i_]):].data_ptr()) for i_, (b_, o_, n_) in enumerate(pieces)]
    torch.cuda.synchronize()

    def step_plain():
        T.clear()
        for b_, o_, n_ in pieces:
            T.upsert_oriented_dev(u, b_.data_ptr(), o_.data_ptr(), n_, kache.OR, 1, 2)
        for i_, (b_, o_, n_) in enumerate(pieces):
            at = int(starts[i_])
            T.lookup_dev(b_.data_ptr(), o_.data_ptr(), n_, found[at:].data_ptr(), vals[at:].data_ptr(), fwd[at:].data_ptr())

    def step_batched():
        T.clear()
        T.run_dev_batches(kache.RUN_UPSERT_ORIENTED, ups, kache.OR, 1, 2, u)
        T.run_dev_batches(kache.RUN_LOOKUP, looks)

    clocks = Clocks(device_index)
    clocks.start()
    ms_plain = timed_steps(stream, step_plain, 3, 3)
    ms_b = timed_steps(stream, step_batched, 5, 3)
    T.profile(True)
    step_batched()
    torch.cuda.synchronize()
    prof = {kind: T.profile_read(i) for i, kind in enumerate(["upsert", "update", "lookup", "reduce", "resize", "other"])}
    T.profile(False)
    clk = clocks.stop()
    inserted, cap = T.size(), T.capacity()
    hit = float((found.cpu().numpy() == 1).sum()) / max(1, P1)
    rho = run_density(kache, br.slice(0, 200), 27)
    b_in = float(br.off[-1]) / P1
    A_up = b_in + 32 * rho + 32 * (1 - inserted / P1) + 32 * 1.0
    A_lk = b_in + 3 + 32 * rho + 32 * hit
    peak, peak_kind = load_peaks()
    kern = {"upsert_oriented": kernel_roofline("lane_kernel<27,16,Upsert_Visitor> (batched)", prof["upsert"][0], prof["upsert"][1],
                                               A_up * P1 / max(1, prof["upsert"][1]), A_up, peak, peak_kind),
            "lookup": kernel_roofline("stream_kernel<27,16,Lookup_Batches_Visitor> (batched)", prof["lookup"][0], prof["lookup"][1],
                                      A_lk * P1 / max(1, prof["lookup"][1]), A_lk, peak, peak_kind)}
    dom = max(kern, key=lambda k_: kern[k_]["ms_total"])
    roof = dict(kern[dom])
    roof["kernels"] = kern
    T.close()
    t_ref, threads = ref_sample(5, 50_000_000, 0.8, False, [("ref_bench_upsert_oriented", br, (3, 1, 2)), ("lookup", br, (27,))])
    cpu = None if t_ref is None else {"value": 2 * P1 / t_ref, "unit": "k-mers/s", "cores": threads, "kind": "reference",
                                      "sample": "the whole workload once: oriented upsert then per-position find, batches of 64 reads over the threads"}
    return {"workload": f"config 3: {len(g)} bp genome, {br.n} reads lognormal(10 kb, 0.8) clipped 1-100 kb at 5x, 5% errors 3:1:1; "
                        f"<27,u8,16> oriented upsert OR 1/2 then oriented find; {len(pieces)} batches of 256 reads",
            "unit": "k-mers/s", "positions_per_step": 2 * P1, "keys": inserted, "capacity": cap,
            "value": 2 * P1 / (ms_b * 1e-3), "ms_per_step": ms_b, "calls_per_step": 2, "form": "kache_b200_run_dev_batches per kind",
            "plain": {"value": 2 * P1 / (ms_plain * 1e-3), "ms_per_step": ms_plain, "calls_per_step": 2 * len(pieces),
                      "form": "one kache_b200_upsert_oriented_dev / kache_b200_lookup_dev call per batch"},
            "batched_over_plain": ms_plain / ms_b, "target": ">= 2x the plain kernel's k-mers/s",
            "kernel_ms_one_step": {k_: v_[0] for k_, v_ in prof.items()}, "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
            "l2": "inputs larger than L2 (reads 250 MB, table about 3 GB)"}


def sub_config5(dev, stream, device_index, scale=0.05, requests=300):
    """Config 5 at `scale` (a <31, u32, 22> map primed with a genome's 31-mers, then upsert ADD 1 / find / count requests
    at 60/30/10, each of lognormal(2000, 1.5) 150 bp reads) with the requests resident in HBM: the batched persistent
    path (one kache_b200_run_dev_batches call per kind), against the request server fed the same requests from four
    client threads, at once (throughput) and at Poisson arrivals at 60 % of that rate (p50/p99 latency)."""
    import torch
    import kache
    from kache import Batch
    rng = np.random.default_rng(54)
    g, primer, reqs = synth.config5(scale, requests)
    T = kache.Table(31, 4, len(g), 0.8, False)
    u = T.register()
    ib, io, ni = dev_batch(Batch(*primer), dev)
    T.upsert_dev(u, ib.data_ptr(), io.data_ptr(), ni, kache.KEEP, 0, 0)
    torch.cuda.synchronize()
    primed = T.size()
    del ib, io
    P = sum(int(b.positions(31).sum()) for _, b in reqs)
    P_kind = [sum(int(b.positions(31).sum()) for k_, b in reqs if k_ == kind) for kind in range(3)]
    T.set_stream(stream.cuda_stream)
    dreq = []
    for kind, b in reqs:
        db, do, n_ = dev_batch(b, dev)
        p_ = int(b.positions(31).sum())
        o0 = torch.empty(max(p_, 1) if kind == 1 else max(n_, 1) * 8, dtype=torch.uint8, device=dev) if kind else None
        o1 = torch.empty(max(p_, 1) * 4, dtype=torch.uint8, device=dev) if kind == 1 else None
        dreq.append((kind, db, do, n_, o0, o1))
    runs_dev = {kind: [(db.data_ptr(), do.data_ptr(), n_) + ((o0.data_ptr(),) if o0 is not None else ()) + ((o1.data_ptr(),) if o1 is not None else ())
                       for k_, db, do, n_, o0, o1 in dreq if k_ == kind] for kind in range(3)}
    res = {}

    def dev_step():
        res["ins"] = sum(T.run_dev_batches(kache.RUN_UPSERT, runs_dev[0], kache.ADD, 1, 1, u))
        res["found"] = sum(T.run_dev_batches(kache.RUN_LOOKUP, runs_dev[1]))
        T.run_dev_batches(kache.RUN_COUNT, runs_dev[2])

    clocks = Clocks(device_index)
    clocks.start()
    dev_ms = timed_steps(stream, dev_step, 3, 3)
    T.profile(True)
    dev_step()
    torch.cuda.synchronize()
    prof = {kind: T.profile_read(i) for i, kind in enumerate(["upsert", "update", "lookup", "reduce", "resize", "other"])}
    T.profile(False)
    T.set_stream(None)
    torch.cuda.synchronize()
    S = kache.Server(T)

    def serve_dev(arrivals=None):
        tickets = [None] * len(dreq)
        start = time.perf_counter()

        def client(idx):
            for i in idx:
                if arrivals is not None:
                    delay = start + arrivals[i] - time.perf_counter()
                    if delay > 0:
                        time.sleep(delay)
                kind, db, do, n_, o0, o1 = dreq[i]
                tickets[i] = S.submit_dev(kind, db.data_ptr(), do.data_ptr(), n_, op=kache.ADD, x=1, init=1,
                                          out0=None if o0 is None else o0.data_ptr(), out1=None if o1 is None else o1.data_ptr())

        th = [threading.Thread(target=client, args=(range(j, len(dreq), 4),)) for j in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        lat = [S.wait(t)[1] for t in tickets]
        return time.perf_counter() - start, np.array(lat)

    for _ in range(3):
        serve_dev()     # warm-up
    r0, _ = S.stats()
    burst_s, burst_lat = serve_dev()
    r1, _ = S.stats()
    rate = 0.6 * len(dreq) / burst_s
    open_s, open_lat = serve_dev(np.cumsum(rng.exponential(1.0 / rate, size=len(dreq))))
    r2, _ = S.stats()
    clk = clocks.stop()
    S.close()
    st = T.stats()
    T.close()
    del dreq, runs_dev
    # Roofline of the batched form's dominant kernel: a map upsert writes a slot sector per position.
    peak, peak_kind = load_peaks()
    b_in = 150.0 / 120.0
    rho = run_density(kache, reqs[0][1].slice(0, min(5000, reqs[0][1].n)))
    hit = res["found"] / max(1, P_kind[1])
    A_up = b_in + 32 * rho + 32 * (1 - res["ins"] / max(1, P_kind[0])) + 32 * 1.0
    A_lk = b_in + 5 + 32 * rho + 32 * hit
    A_ct = b_in + 32 * rho + 32 * hit
    kern = {"upsert": kernel_roofline("lane_kernel<31,22,Upsert_Visitor> (batched)", prof["upsert"][0], prof["upsert"][1],
                                      A_up * P_kind[0] / max(1, prof["upsert"][1]), A_up, peak, peak_kind),
            "lookup": kernel_roofline("stream_kernel<31,22,Lookup_Batches_Visitor> (batched)", prof["lookup"][0], prof["lookup"][1],
                                      A_lk * P_kind[1] / max(1, prof["lookup"][1]), A_lk, peak, peak_kind),
            "count": kernel_roofline("lane_kernel<31,22,Seq_Reduce_Visitor> (batched)", prof["reduce"][0], prof["reduce"][1],
                                     A_ct * P_kind[2] / max(1, prof["reduce"][1]), A_ct, peak, peak_kind)}
    dom = max(kern, key=lambda k_: kern[k_]["ms_total"])
    roof = dict(kern[dom])
    roof["kernels"] = kern
    cpu = cpu_served_reference(reqs, g, primer)
    pct = lambda a, q: float(np.percentile(a, q))
    return {"workload": f"config 5 at scale {scale}: {len(g)} bp genome primed ({primed} keys); {len(reqs)} requests of 150 bp "
                        "reads (1% errors), lognormal(2000, 1.5) reads each clipped 1-1M, upsert ADD 1 / find / count at 60/30/10, "
                        "resident in HBM", "unit": "k-mers/s", "positions": P,
            "value": P / burst_s, "ms": 1000 * burst_s, "form": "request server, device requests from four threads at once",
            "runs": r1 - r0, "p50_ms": pct(burst_lat, 50), "p99_ms": pct(burst_lat, 99),
            "batched": {"value": P / (dev_ms * 1e-3), "ms": dev_ms, "calls": 3,
                        "form": "kache_b200_run_dev_batches per kind (CUDA events)"},
            "served_over_batched": (dev_ms * 1e-3) / burst_s, "target": "served within 20 % of the batched throughput",
            "poisson": {"offered_requests_per_s": rate, "value": P / open_s, "p50_ms": pct(open_lat, 50),
                        "p99_ms": pct(open_lat, 99), "runs": r2 - r1},
            "kernel_ms_batched": {k_: v_[0] for k_, v_ in prof.items()}, "keys_after": st.keys, "capacity_after": st.capacity,
            "roofline": roof, "cpu_baseline": cpu, "clocks": clk}


def cpu_served_reference(reqs, g, primer, budget_s=20.0):
    """The reference's table (oracle/_ref) primed with the same genome, then the requests served one at a time in
    arrival order on one thread (upserts serialised with queries, as the reference's phase rule requires), until
    `budget_s` seconds of request work are spent."""
    import oracle
    from kache import Batch
    if oracle.ref() is None:
        return None
    R = oracle.RefTable(31, 4, len(g), 0.8, False, workers=min(128, os.cpu_count() or 1))
    u = R.register()
    R.bench_upsert(Batch(*primer), 0, 0, min(128, os.cpu_count() or 1))
    done, P, t = 0, 0, 0.0
    for kind, b in reqs:
        t0 = time.perf_counter()
        if kind == 0:
            R.upsert(u, b, 2, 1)
        elif kind == 1:
            R.lookup(b)
        else:
            R.L.ref_count(R.h, b.bases.ctypes.data, b.off.ctypes.data, b.n)
        t += time.perf_counter() - t0
        P += int(b.positions(31).sum())
        done += 1
        if t > budget_s:
            break
    return {"value": P / t, "unit": "k-mers/s", "cores": 1, "kind": "reference",
            "sample": f"the first {done} of {len(reqs)} requests in arrival order on one thread ({P} positions), "
                      "after priming with all host threads"}


def cold_first_call(dev, stream, d_ins_b, d_ins_o, n_ins, d_held_b, d_held_o, n_held, d_found, d_vals, P):
    """Config 1 on a table just made by kache_new: the first upsert call grows the table from its creation size with
    no rate learned from earlier calls, then the lookup; CUDA events around both calls."""
    import torch
    import kache
    T = kache.Table(31, 8, N_KEYS, 0.8, False)
    T.set_stream(stream.cuda_stream)
    u = T.register()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    T.upsert_dev(u, d_ins_b, d_ins_o, n_ins, kache.ADD_WRAP, 1, 1)
    T.lookup_dev(d_held_b, d_held_o, n_held, d_found, d_vals, None)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    keys = T.size()
    T.close()
    return {"value": P / (ms * 1e-3), "unit": "k-mers/s", "ms": ms, "keys": keys,
            "form": "config 1's upsert then find, once, on a fresh kache_new table (no earlier call to learn from)"}


# ---- The other workloads: one JSON line each, for the record (the default line is config 1) -----------------------

def dev_batch(b, dev):
    """A batch's bases and offsets copied to the device: (tensors, n)."""
    import torch
    return torch.from_numpy(b.bases).to(dev), torch.from_numpy(b.off.view(np.int64)).to(dev), b.n


def dev_pieces(b, dev, per):
    """The batch cut into sub-batches of `per` sequences on the device, each with offsets of its own."""
    import torch
    out = []
    for s in range(0, b.n, per):
        e = min(b.n, s + per)
        o0 = int(b.off[s])
        off = (b.off[s:e + 1] - np.uint64(o0)).view(np.int64)
        out.append((torch.from_numpy(b.bases[o0:int(b.off[e]) + 16].copy()).to(dev), torch.from_numpy(off.copy()).to(dev), e - s))
    return out


def timed_steps(stream, step, steps, warmup):
    """Mean device milliseconds per step, CUDA events on the stream, after `warmup` untimed steps."""
    import torch
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def pinned_copy(b):
    import torch
    from kache import Batch
    t = torch.empty(b.bases.nbytes, dtype=torch.uint8, pin_memory=True)
    t.numpy()[:] = b.bases
    pb = Batch(t.numpy(), b.off)
    pb.keep = t
    return pb


def ref_sample(kind, n, lf, pow2, calls):
    """Seconds the reference's own table (oracle/_ref) takes for `calls`, a list of (function name, batch, args),
    all host threads; None where it was not built."""
    import oracle
    L = oracle.ref()
    if L is None:
        return None, 0
    threads = min(128, os.cpu_count() or 1)
    t = L.ref_new(kind, n, lf, 1 if pow2 else 0, threads)
    out = oracle._u64()
    total = 0.0
    for fn, b, a in calls:
        if fn == "lookup":
            total += ref_lookup_timed(L, t, b, threads, *a)
        else:
            total += getattr(L, fn)(t, b.bases.ctypes.data, b.off.ctypes.data, b.n, 64, threads, *a, oracle.ctypes.byref(out))
    L.ref_free(t)
    return total, threads


def config_line(metric, value, ms, cfg, e2e=None, cpu=None, extra=None):
    line = {"metric": metric, "value": value, "unit": "k-mers/s", "n_gpus": 1, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "data": "synthetic", "config": cfg, "e2e": e2e, "cpu_baseline": cpu}
    line.update(extra or {})
    print(json.dumps(line))


def run_config2(args):
    """Kmer_Set_Counter, <31, u32, 22> at load factor 0.9, power-of-2 capacity: prime with the genome's 31-mers
    (upsert KEEP, initial 0), count the reads (present-only wrapping +1), histogram(10000)."""
    import torch
    import kache
    from kache import Batch
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    g, index, reads = synth.config2(args.scale)
    bi, br = Batch(*index), Batch(*reads)
    n = int(100_000_000 * args.scale)
    P = positions(bi.off) + positions(br.off)
    T = kache.Table(31, 4, n, 0.9, True)
    T.set_stream(stream.cuda_stream)
    u = T.register()
    (ib, io, ni), (rb, ro, nr) = dev_batch(bi, dev), dev_batch(br, dev)
    hist = {}

    def step():
        T.clear()
        T.upsert_dev(u, ib.data_ptr(), io.data_ptr(), ni, kache.KEEP, 0, 0)
        hist["found"] = T.update_dev(rb.data_ptr(), ro.data_ptr(), nr, kache.ADD_WRAP, 1)
        hist["h"] = T.histogram(10000)

    ms = timed_steps(stream, step, args.steps, args.warmup)
    size, cap = T.size(), T.capacity()
    T.close()
    # End to end through the counter's C interface with page-locked host batches: a first pass on the new counter
    # (its staging buffers allocated as it goes), the counter's table emptied (kache_b200_clear keeps them), then
    # the timed pass.
    pi, pr = pinned_copy(bi), pinned_copy(br)
    C = kache.Counter(n, 16, 0.9)

    def e2e_pass():
        t0 = time.perf_counter()
        C.prime_batch(pi)
        C.count_batch(pr)
        C.histogram(10000)
        return 1000 * (time.perf_counter() - t0)

    first_ms = e2e_pass()
    kache._check(kache.lib().kache_b200_clear(kache.lib().kache_counter_table(C.h)), "kache_b200_clear")
    e2e_ms = e2e_pass()
    C.close()
    # The reference on a twentieth of the reads (after priming with the whole genome, untimed for the sample rate).
    rs = br.slice(0, br.n // 20)
    t_ref, threads = ref_sample(1, n, 0.9, True, [("ref_bench_upsert", bi, (0, 0)), ("ref_bench_update", rs, (16, 1))])
    cpu = None if t_ref is None else {"value": (positions(bi.off) + positions(rs.off)) / t_ref, "unit": "k-mers/s", "cores": threads,
                                      "kind": "reference", "sample": f"prime with the whole index, count {rs.n} of {br.n} reads"}
    config_line("k-mers/s prime+count (config 2: Kmer_Set_Counter <31,u32,22>, lf 0.9 pow2)", P / (ms * 1e-3), ms,
                {"workload": f"config 2 at scale {args.scale}: {len(g)} bp genome (5% segmental duplications), {br.n} reads "
                             "lognormal(150, 0.6) clipped 50-1000 bp at 30x", "prime_positions": positions(bi.off),
                 "count_positions": positions(br.off), "keys": size, "capacity": cap, "found": hist["found"],
                 "histogram_sum": int(sum(hist["h"]))},
                e2e={"value": P / (e2e_ms * 1e-3), "unit": "k-mers/s", "ms_per_step": e2e_ms, "host_buffers": "page-locked",
                     "first_pass_ms": first_ms,
                     "calls": "kache_counter_prime_batch, kache_counter_count_batch, kache_counter_histogram"},
                cpu=cpu)


def run_config3(args):
    """Oriented strand map <27, u8, 16>: upsert_oriented(OR, fwd 1, rev 2) of long reads with indels, then per-position
    find with the orientation; all reads in one call, and in calls of 256 reads."""
    import torch
    import kache
    from kache import Batch
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    g, reads = synth.config3(args.scale)
    br = Batch(*reads)
    n = int(50_000_000 * args.scale)
    P1 = positions(br.off, 27)
    T = kache.Table(27, 1, n, 0.8, False)
    T.set_stream(stream.cuda_stream)
    u = T.register()
    rb, ro, nr = dev_batch(br, dev)
    found = torch.empty(P1, dtype=torch.uint8, device=dev)
    vals = torch.empty(P1, dtype=torch.uint8, device=dev)
    fwd = torch.empty(P1, dtype=torch.uint8, device=dev)

    def step():
        T.clear()
        T.upsert_oriented_dev(u, rb.data_ptr(), ro.data_ptr(), nr, kache.OR, 1, 2)
        T.lookup_dev(rb.data_ptr(), ro.data_ptr(), nr, found.data_ptr(), vals.data_ptr(), fwd.data_ptr())

    ms = timed_steps(stream, step, args.steps, args.warmup)
    pieces = dev_pieces(br, dev, 256)
    starts = np.concatenate([[0], np.cumsum([int(np.maximum(np.diff(o_.cpu().numpy()) - 26, 0).sum()) for _, o_, _ in pieces])])

    def step_batched():
        T.clear()
        for b_, o_, n_ in pieces:
            T.upsert_oriented_dev(u, b_.data_ptr(), o_.data_ptr(), n_, kache.OR, 1, 2)
        for i_, (b_, o_, n_) in enumerate(pieces):
            at = int(starts[i_])
            T.lookup_dev(b_.data_ptr(), o_.data_ptr(), n_, found[at:].data_ptr(), vals[at:].data_ptr(), fwd[at:].data_ptr())

    ms_b = timed_steps(stream, step_batched, max(1, args.steps // 3), 1)
    # The same 256-read batches, all of a phase in one kache_b200_run_dev_batches call: one segment list, one launch.
    ups = [(b_.data_ptr(), o_.data_ptr(), n_) for b_, o_, n_ in pieces]
    looks = [(b_.data_ptr(), o_.data_ptr(), n_, found[int(starts[i_]):].data_ptr(), vals[int(starts[i_]):].data_ptr(),
              fwd[int(starts[i_]):].data_ptr()) for i_, (b_, o_, n_) in enumerate(pieces)]

    def step_runs():
        T.clear()
        T.run_dev_batches(kache.RUN_UPSERT_ORIENTED, ups, kache.OR, 1, 2, u)
        T.run_dev_batches(kache.RUN_LOOKUP, looks)

    ms_r = timed_steps(stream, step_runs, args.steps, args.warmup)

    # The lookups of the same 256-read batches (on the table step_runs left): one staged call per batch; the batch
    # shapes prepared once and the 71 launches captured in a CUDA graph, replayed; one batched call.
    def look_calls():
        for i_, (b_, o_, n_) in enumerate(pieces):
            at = int(starts[i_])
            T.lookup_dev(b_.data_ptr(), o_.data_ptr(), n_, found[at:].data_ptr(), vals[at:].data_ptr(), fwd[at:].data_ptr())

    ms_lc = timed_steps(stream, look_calls, args.steps, args.warmup)
    ms_lb = timed_steps(stream, lambda: T.run_dev_batches(kache.RUN_LOOKUP, looks), args.steps, args.warmup)
    preps = [T.prepare_dev(o_.data_ptr(), n_) for _, o_, n_ in pieces]
    cap_stream = torch.cuda.Stream()
    T.set_stream(cap_stream.cuda_stream)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=cap_stream):
        for i_, ((b_, o_, n_), p_) in enumerate(zip(pieces, preps)):
            at = int(starts[i_])
            T.lookup_prepared(p_, b_.data_ptr(), found[at:].data_ptr(), vals[at:].data_ptr(), fwd[at:].data_ptr())
    ms_lg = timed_steps(stream, graph.replay, args.steps, args.warmup)     # replay() runs on the current stream
    del graph
    T.set_stream(stream.cuda_stream)
    for p_ in preps:
        T.prepared_free(p_)

    def profiled(f):
        """Device milliseconds per kernel kind of one run of f (CUDA events around each launch)."""
        T.profile(True)
        f()
        torch.cuda.synchronize()
        p_ = {kind: T.profile_read(i) for i, kind in enumerate(["upsert", "update", "lookup", "reduce", "resize", "other"])}
        T.profile(False)
        return p_

    prof_1 = profiled(step)
    prof_r = profiled(step_runs)
    prof_b = profiled(step_batched)
    size, cap = T.size(), T.capacity()
    T.close()
    t_ref, threads = ref_sample(5, n, 0.8, False, [("ref_bench_upsert_oriented", br, (3, 1, 2)), ("lookup", br, (27,))])
    cpu = None if t_ref is None else {"value": 2 * P1 / t_ref, "unit": "k-mers/s", "cores": threads, "kind": "reference",
                                      "sample": "the whole workload once"}
    config_line("k-mers/s upsert_oriented+find (config 3: <27,u8,16> strand map, long reads)", 2 * P1 / (ms * 1e-3), ms,
                {"workload": f"config 3 at scale {args.scale}: {len(g)} bp genome, {br.n} reads lognormal(10 kb, 0.8) clipped "
                             "1-100 kb at 5x, 5% errors 3:1:1", "positions_per_phase": P1, "keys": size, "capacity": cap},
                cpu=cpu, extra={"kernel_ms_one_step": {k_: v_[0] for k_, v_ in prof_1.items()},
                                "batched_256_reads": {"value": 2 * P1 / (ms_b * 1e-3), "ms_per_step": ms_b, "calls_per_step": 2 * len(pieces),
                                                      "kernel_ms_one_step": {k_: v_[0] for k_, v_ in prof_b.items()}},
                                "run_dev_batches_256_reads": {"value": 2 * P1 / (ms_r * 1e-3), "ms_per_step": ms_r, "calls_per_step": 2,
                                                              "batches_per_call": len(pieces),
                                                              "kernel_ms_one_step": {k_: v_[0] for k_, v_ in prof_r.items()},
                                                              "vs_one_call_per_batch": ms_b / ms_r},
                                "lookups_256_reads": {"positions": P1, "batches": len(pieces), "per_call_ms": ms_lc,
                                                      "cuda_graph_ms": ms_lg, "run_dev_batches_ms": ms_lb,
                                                      "cuda_graph": "kache_b200_prepare_dev once per batch shape, the "
                                                                    "kache_b200_lookup_prepared launches captured in one graph"}})


def run_config4(args):
    """Resize-heavy set <32, void, 20> sized for 1M keys (load factor 0.8, exact capacity): insert a uniform genome
    streamed as 150 bp pieces at 1x, in calls of 65,536 pieces; the table doubles about 9 times per step."""
    import torch
    import kache
    from kache import Batch
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    g, pieces_ = synth.config4(args.scale)
    bs = Batch(*pieces_)
    P = positions(bs.off, 32)
    T = kache.Table(32, 0, 1_000_000, 0.8, False)
    T.set_stream(stream.cuda_stream)
    u = T.register()
    pieces = dev_pieces(bs, dev, 65536)
    ins = {}

    def step():
        T.clear()
        c = 0
        for b_, o_, n_ in pieces:
            c += T.upsert_dev(u, b_.data_ptr(), o_.data_ptr(), n_, kache.KEEP, 0, 0)
        ins["n"] = c

    ms = timed_steps(stream, step, args.steps, args.warmup)
    T.profile(True)
    step()
    torch.cuda.synchronize()
    rz_ms, rz_n = T.profile_read(4)
    up_ms, up_n = T.profile_read(0)
    ot_ms, ot_n = T.profile_read(5)
    T.profile(False)
    size, cap = T.size(), T.capacity()
    T.close()
    t_ref, threads = ref_sample(6, 1_000_000, 0.8, False, [("ref_bench_upsert", bs, (0, 0))])
    cpu = None if t_ref is None else {"value": P / t_ref, "unit": "k-mers/s", "cores": threads, "kind": "reference",
                                      "sample": "the whole stream once, batches of 64 pieces over the threads"}
    config_line("k-mers/s insert (config 4: <32,set,20> n=1M, doubling as it fills)", P / (ms * 1e-3), ms,
                {"workload": f"config 4 at scale {args.scale}: {len(g)} bp genome as {bs.n} pieces of 150 bp, calls of 65,536 pieces",
                 "positions": P, "inserted": ins["n"], "keys": size, "capacity": cap},
                cpu=cpu, extra={"profile_one_step": {"insert_ms": up_ms, "insert_launches": up_n, "rebuild_ms": rz_ms,
                                                     "rebuild_launches": rz_n, "staging_and_other_ms": ot_ms,
                                                     "staging_and_other_launches": ot_n}})


def run_config5(args):
    """Served mixed requests (upsert ADD 1 / find / count at 60/30/10) on a <31, u32, 22> map primed with a genome's
    31-mers: the same requests run one by one through the plain calls, then through the request server submitted at
    once from four client threads (throughput), then through the server at Poisson arrivals at 60 % of that
    throughput (latency)."""
    import threading
    import torch
    import kache
    from kache import Batch
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(54)     # arrival times
    g, primer, reqs = synth.config5(args.scale, args.requests)
    glen = len(g)
    T = kache.Table(31, 4, glen, 0.8, False)
    u = T.register()
    ib, io, ni = dev_batch(Batch(*primer), dev)
    T.upsert_dev(u, ib.data_ptr(), io.data_ptr(), ni, kache.KEEP, 0, 0)
    torch.cuda.synchronize()
    primed = T.size()
    del ib, io
    P = sum(int(b.positions(31).sum()) for _, b in reqs)

    def outputs(kind, b):
        p = int(b.positions(31).sum())
        if kind == 1:
            return np.zeros(max(p, 1), np.uint8), np.zeros(max(p, 1), np.uint32), None
        if kind == 2:
            return np.zeros(max(b.n, 1), np.uint64), None, None
        return None, None, None

    # Plain: one call per request, in order.
    t0 = time.perf_counter()
    for kind, b in reqs:
        if kind == 0:
            T.upsert(u, b, kache.ADD, 1, 1)
        elif kind == 1:
            T.lookup(b, values=True, fwd=False)
        else:
            T.count(b)
    plain_s = time.perf_counter() - t0

    # Batched: the same requests from the same pageable buffers, merged by kind into one call each (all upserts, then
    # all finds, then all counts; the sequences' pointer arrays concatenated, no copy): the best a caller feeding the
    # table from host memory gets, and the throughput the served loop is compared with.
    L_ = kache.lib()
    merged = {}
    for kind in range(3):
        bs_ = [b for k_, b in reqs if k_ == kind and b.n]
        ptrs = np.concatenate([b.ptrs[:b.n] for b in bs_]) if bs_ else np.zeros(1, np.uint64)
        lens = np.concatenate([b.lens[:b.n] for b in bs_]) if bs_ else np.zeros(1, np.uint64)
        n_ = sum(b.n for b in bs_)
        p_ = sum(int(b.positions(31).sum()) for b in bs_)
        merged[kind] = (ptrs, lens, n_, np.zeros(max(p_, 1), np.uint8), np.zeros(max(p_, 1), np.uint32), np.zeros(max(n_, 1), np.uint64))
    r_ = ctypes.c_uint64()
    t0 = time.perf_counter()
    for kind in range(3):
        ptrs, lens, n_, f_, v_, c_ = merged[kind]
        if kind == 0:
            kache._check(L_.kache_b200_upsert(T.h, u, ptrs.ctypes.data, lens.ctypes.data, n_, kache.ADD, 1, 1, ctypes.byref(r_)), "upsert")
        elif kind == 1:
            kache._check(L_.kache_lookup(T.h, ptrs.ctypes.data, lens.ctypes.data, n_, f_.ctypes.data, v_.ctypes.data, None), "lookup")
        else:
            kache._check(L_.kache_count(T.h, ptrs.ctypes.data, lens.ctypes.data, n_, c_.ctypes.data), "count")
    batched_s = time.perf_counter() - t0
    del merged

    # The batched persistent path on the same requests, resident in HBM: each kind's requests as one
    # kache_b200_run_dev_batches call (one segment list, one launch), outputs in HBM, CUDA events on the table's stream.
    stream = torch.cuda.current_stream()
    T.set_stream(stream.cuda_stream)
    dreq = []
    for kind, b in reqs:
        db, do, n_ = dev_batch(b, dev)
        p_ = int(b.positions(31).sum())
        o0 = torch.empty(max(p_, 1) if kind == 1 else max(n_, 1) * 8, dtype=torch.uint8, device=dev) if kind else None
        o1 = torch.empty(max(p_, 1) * 4, dtype=torch.uint8, device=dev) if kind == 1 else None
        dreq.append((kind, db, do, n_, o0, o1))
    runs_dev = {kind: [(db.data_ptr(), do.data_ptr(), n_) + ((o0.data_ptr(),) if o0 is not None else ()) + ((o1.data_ptr(),) if o1 is not None else ())
                       for k_, db, do, n_, o0, o1 in dreq if k_ == kind] for kind in range(3)}

    def dev_step():
        T.run_dev_batches(kache.RUN_UPSERT, runs_dev[0], kache.ADD, 1, 1, u)
        T.run_dev_batches(kache.RUN_LOOKUP, runs_dev[1])
        T.run_dev_batches(kache.RUN_COUNT, runs_dev[2])

    dev_ms = timed_steps(stream, dev_step, 3, 1)
    T.set_stream(None)
    del runs_dev
    torch.cuda.synchronize()

    S = kache.Server(T)

    def serve_dev(arrivals=None):
        """The same requests resident in HBM submitted to the server from four threads, at once or at `arrivals`
        seconds: runs of device requests are kache_b200_run_dev_batches calls. Returns wall seconds and latencies."""
        tickets = [None] * len(dreq)
        start = time.perf_counter()

        def client(idx):
            for i in idx:
                if arrivals is not None:
                    delay = start + arrivals[i] - time.perf_counter()
                    if delay > 0:
                        time.sleep(delay)
                kind, db, do, n_, o0, o1 = dreq[i]
                tickets[i] = S.submit_dev(kind, db.data_ptr(), do.data_ptr(), n_, op=kache.ADD, x=1, init=1,
                                          out0=None if o0 is None else o0.data_ptr(), out1=None if o1 is None else o1.data_ptr())

        th = [threading.Thread(target=client, args=(range(j, len(dreq), 4),)) for j in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        lat = [S.wait(t)[1] for t in tickets]
        return time.perf_counter() - start, np.array(lat)

    serve_dev()     # warm-up
    rd0, _ = S.stats()
    dev_served_s, dev_served_lat = serve_dev()
    rd1, _ = S.stats()
    dev_rate = 0.6 * len(dreq) / dev_served_s
    dev_open_s, dev_open_lat = serve_dev(np.cumsum(rng.exponential(1.0 / dev_rate, size=len(dreq))))
    rd2, _ = S.stats()
    del dreq

    def serve(arrivals):
        """Submits request i at arrivals[i] seconds (all at once if None) from four threads; returns wall seconds and
        latencies."""
        tickets = [None] * len(reqs)
        outs = [outputs(kind, b) for kind, b in reqs]
        start = time.perf_counter()

        def client(idx):
            for i in idx:
                if arrivals is not None:
                    delay = start + arrivals[i] - time.perf_counter()
                    if delay > 0:
                        time.sleep(delay)
                kind, b = reqs[i]
                o = outs[i]
                tickets[i] = S.submit(kind, b, op=kache.ADD, x=1, init=1, out0=o[0], out1=o[1], out2=o[2])

        th = [threading.Thread(target=client, args=(range(j, len(reqs), 4),)) for j in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        lat = [S.wait(t)[1] for t in tickets]
        return time.perf_counter() - start, np.array(lat)

    runs0, _ = S.stats()
    burst_s, burst_lat = serve(None)
    runs1, _ = S.stats()
    rate = 0.6 * len(reqs) / burst_s
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(reqs)))
    open_s, open_lat = serve(arrivals)
    runs2, _ = S.stats()
    S.close()
    st = T.stats()
    T.close()
    pct = lambda a, q: float(np.percentile(a, q))
    config_line("k-mers/s served mix (config 5: <31,u32,22> primed map, upsert ADD 1 / find / count at 60/30/10)",
                P / burst_s, 1000 * burst_s,
                {"workload": f"config 5 at scale {args.scale}: {glen} bp genome primed ({primed} keys); {len(reqs)} requests of "
                             "150 bp reads (1% errors), lognormal(2000, 1.5) reads each, clipped 1-1M",
                 "positions": P, "keys_after": st.keys, "capacity_after": st.capacity},
                extra={"plain": {"value": P / plain_s, "ms": 1000 * plain_s, "calls": len(reqs)},
                       "batched": {"value": P / batched_s, "ms": 1000 * batched_s, "calls": 3,
                                   "host_buffers": "pageable, one call per kind"},
                       "batched_device": {"value": P / (dev_ms * 1e-3), "ms": dev_ms, "calls": 3,
                                          "form": "kache_b200_run_dev_batches per kind, requests resident in HBM",
                                          "served_burst_fraction": dev_ms * 1e-3 / burst_s},
                       "served_device_burst": {"value": P / dev_served_s, "ms": 1000 * dev_served_s,
                                               "p50_ms": pct(dev_served_lat, 50), "p99_ms": pct(dev_served_lat, 99),
                                               "runs": rd1 - rd0, "requests": len(reqs),
                                               "fraction_of_batched_device": dev_ms * 1e-3 / dev_served_s,
                                               "form": "the requests resident in HBM, submitted to the server at once from four threads"},
                       "served_device_poisson": {"offered_requests_per_s": dev_rate, "value": P / dev_open_s,
                                                 "p50_ms": pct(dev_open_lat, 50), "p99_ms": pct(dev_open_lat, 99), "runs": rd2 - rd1},
                       "served_burst": {"value": P / burst_s, "p50_ms": pct(burst_lat, 50), "p99_ms": pct(burst_lat, 99),
                                        "runs": runs1 - runs0, "requests": len(reqs)},
                       "served_poisson": {"offered_requests_per_s": rate, "value": P / open_s, "p50_ms": pct(open_lat, 50),
                                          "p99_ms": pct(open_lat, 99), "runs": runs2 - runs1},
                       "host_buffers": "pageable (the library stages them)"})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", type=int, default=1, choices=[1, 2, 3, 4, 5],
                    help="the workload: 1 (the headline line), or one of the other configurations, printed for the record")
    ap.add_argument("--scale", type=float, default=1.0, help="size of configurations 2-5 relative to their full size")
    ap.add_argument("--requests", type=int, default=300, help="requests of configuration 5")
    ap.add_argument("--only-dev", action="store_true",
                    help="time the device-resident steps only (no e2e, CPU baseline or clock sampling): the profiling case")
    ap.add_argument("--no-sub", action="store_true",
                    help="leave out the sub-records of the default line (config 3 batched, config 5 served, cold first call)")
    args = ap.parse_args()
    if args.config != 1:
        {2: run_config2, 3: run_config3, 4: run_config4, 5: run_config5}[args.config](args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
