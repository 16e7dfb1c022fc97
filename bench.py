"""Benchmark of the Eq. (C7) path (exmarg pe_intrinsic) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (one step = one segment analysed end to end through the public API):
2048-template TaylorF2 bank (chirp mass 10-40, q 0.25-1, chi_eff -0.5..0.5), 53
signal-power nodes of seeded synthetic float32 tables at the production shape
(87 lags x 49 phase planes x 200 beta x 219 Delta, 39.8 GB, resident in HBM), 8 s
H1+L1 segments (20-512 Hz, n_time = 32768) of coloured Gaussian noise with one
injected TaylorF2 signal (chirp mass 25, q 0.8, chi_eff 0.1, network SNR 15), volume
prior, n_loud = n_random = 1024.  The tables (39.8 GB) are far larger than the L2
(126 MB), so no flush is needed between steps.

Under torchrun (N > 1) every rank is an independent replica on its own GPU with its
own segments (weak scaling); ranks meet only in host-side barriers and the max of
their device times (gloo).  --impl reference runs the CPU restatement of the
reference's path (oracle/, float64 gather over the host cores) on rank 0 only.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "segments/s at |dlnB|<=1e-5 (2048 templ, 53 nodes); p50/p99 latency; gather GB/s"
N_TEMPLATES, T_SEG, FMAX = 2048, 8.0, 512.0
N_LOUD = N_RANDOM = 1024
TABLE_SEED, BANK_SEED, SEG_SEED = 2026, 11, 50000


def workload_config(args=None):
    if args is not None and (args.templates != N_TEMPLATES or args.nodes != 53 or args.lags != 87):
        return {"workload": "reduced profiling case: %d templates, %d nodes, %d lags (else as the full workload)"
                            % (args.templates, args.nodes, args.lags), "templates": args.templates,
                "nodes": args.nodes, "lags": args.lags, "segment_s": T_SEG, "n_time": 32768, "table_dtype": "f32"}
    return {"workload": "pe_intrinsic, 1 segment per call: 2048-template TaylorF2 bank, 53 nodes of seeded f32 "
                        "tables 87x49x200x219 (39.8 GB, resident), 8 s H1+L1 segment 20-512 Hz (n_time 32768), "
                        "SNR-15 injection, n_loud=n_random=1024, volume prior",
            "templates": N_TEMPLATES, "nodes": 53, "segment_s": T_SEG, "n_time": 32768,
            "table_dtype": "f32", "l2": "inputs larger than L2 (39.8 GB tables vs 126 MB)"}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def segment_seed(rank):
    """first segment seed of a rank: every replica analyses its own segments"""
    return SEG_SEED + 100000 * rank


def combine_ranks(values, dist):
    """the max over ranks of each value (device and wall seconds): the job ends with its slowest rank"""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def make_inputs(n_seg, rank, n_templates=N_TEMPLATES, n_nodes=53, n_lags=87):
    from exmarg_b200 import synth
    spec = synth.TableSpec(ntau=n_lags)
    s_nodes = synth.S_NODES_PROD
    if n_nodes < s_nodes.size:            # a reduced case keeps nodes every template reaches
        s_nodes = s_nodes[30:30 + n_nodes]
    seg = synth.make_segments(n_seg, segment_seed(rank), T=T_SEG, fmax=FMAX, snr=15.0, mc=25.0, q=0.8, chi=0.1)
    rows = synth.make_bank(n_templates, BANK_SEED)
    return spec, s_nodes, seg, rows


class ClockSampler:
    """nvidia-smi samples of one GPU during the timed region"""

    FIELDS = "timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.window = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self, t0, t1):
        """the timed region, in time.time() seconds: only samples inside it are kept"""
        self.window = (t0, t1)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ts, ln in self.lines:
            if self.window and not (self.window[0] <= ts <= self.window[1] + 0.25):
                continue
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 10:
                continue
            try:
                sm.append(float(parts[2]))
                smax.append(float(parts[3]))
                power.append(float(parts[4]))
            except ValueError:
                continue
            for n, v in zip(names, parts[6:10]):
                if v.lower() == "active":
                    reasons.add(n)
        load = [s for s, p in zip(sm, power) if p > 200.0] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# DRAM traffic of the plane gather, per node-tap, from one ncu capture of a reduced case (one kernel, one
# launch, a few GB on the device: profiles/k_gather_planes_small.md gives the command).  The bytes a launch
# moves scale with its node-taps (the windows staged per (node, lag, template block) and the descriptors
# read per node-tap both do), so the full launch's traffic is this figure times its node-taps.  The capture
# holds only for the kernel sources it was taken on: if they changed since, traffic is reported as null.
GATHER_TRAFFIC = {
    "dram_bytes_per_node_tap": 3.9683,       # (1.8772e9 + 8.92e6) B / 4.7531e8 node-taps (28 warps x 1, 150 %)
    "l2_read_hit_rate": 69.92,             # lts__t_sector_op_read_hit_rate.pct
    "sources_sha256": "6014a92f6f6972047daeb8f5535a10d004f69fd2b89c0258d722db9f213bc2f9",
    "capture": "profiles/k_gather_planes_small.md",
}
GATHER_SOURCES = ("exmarg_b200/csrc/gather.cu", "exmarg_b200/csrc/taps.cu", "exmarg_b200/csrc/kernels.cuh")


def gather_sources_sha256():
    import hashlib
    h = hashlib.sha256()
    for f in GATHER_SOURCES:
        with open(os.path.join(ROOT, f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()


def gather_traffic(node_taps_per_launch):
    """(DRAM bytes per launch scaled from the reduced-case capture, L2 read hit rate, why null)"""
    g = GATHER_TRAFFIC
    if g["dram_bytes_per_node_tap"] is None:
        return None, None, "no capture recorded"
    if g["sources_sha256"] != gather_sources_sha256():
        return None, None, "stale: the gather sources changed since the capture"
    return g["dram_bytes_per_node_tap"] * node_taps_per_launch, g["l2_read_hit_rate"], None


def compulsory_table_bytes(traj, sel, u, spec, s_nodes, lags):
    """A lower bound on the table bytes one segment's gather must read from DRAM: the distinct 32-byte
    sectors of the node tables that the taps of a template sample touch (every tap reads 2 phase planes x
    2 beta rows x 2 Delta columns at every node it reaches), counted on the host for the sampled lags and
    scaled to all lags.  A sample touches no more sectors than the whole bank, so this bounds the full
    workload's compulsory table bytes from below."""
    nphi = 96
    db, dd = spec.beta[1] - spec.beta[0], spec.delta[1] - spec.delta[0]
    nt = traj["lqL"].shape[1]
    lqL = np.take_along_axis(traj["lqL"], sel, 1).astype(np.float64)
    phL = np.take_along_axis(traj["phL"], sel, 1)
    bh0 = lqL * (2.0 / db) - (np.log(u) / db)[:, None]
    ck = (np.log(s_nodes) - spec.beta[0]) / db
    nsec = (spec.nd + 1 + 7) // 8
    touched = 0
    for tau in lags:
        i1 = (sel + int(tau)) % nt
        lqH = np.take_along_axis(traj["lqH"], i1, 1).astype(np.float64)
        x3 = (np.take_along_axis(traj["phH"], i1, 1) - phL).astype(np.float64) * (nphi / (2 * np.pi)) % nphi
        c0 = np.minimum(x3.astype(int), nphi - 1)
        p = np.where(c0 <= 47, c0, nphi - 1 - c0).ravel()
        for k in range(s_nodes.size):
            xb = np.clip(bh0 + ck[k], 0.0, spec.nb - 1 - 1e-6)
            lqc = lqL + (xb - (bh0 + ck[k])) * (db / 2.0)
            xd = np.clip((lqH - lqc) / dd - spec.delta[0] / dd, 0.0, spec.nd - 1 - 1e-6)
            b0, d0 = xb.astype(int).ravel(), xd.astype(int).ravel()
            bm = np.zeros((48 + 1, spec.nb + 1, nsec + 1), bool)
            for dp in (0, 1):
                for db_ in (0, 1):
                    for dd_ in (0, 1):
                        bm[p + dp, b0 + db_, (d0 + dd_) // 8] = True
            touched += int(bm[:49, :spec.nb, :nsec].sum())
    return 32.0 * touched * (spec.ntau / float(len(lags)))


# ----------------------------------------------------------------------------- CPU baseline (oracle port)

def cpu_sample(seg, rows, W, u, lo, n_time, store, n_templates, e=0):
    """the CPU restatement of the reference path (oracle) on a template sample of one segment:
    (seconds, sampled template ids, their ln_lambda)"""
    from oracle import restate
    rng = np.random.default_rng(7)
    idx = np.sort(rng.choice(rows.shape[0], min(n_templates, rows.shape[0]), replace=False))
    s1 = restate.read_segments(seg, rows=[e])
    t0 = time.perf_counter()
    o = restate.pe_intrinsic(s1, W[idx], u[idx], rows[idx, 0], rows[idx, 1], rows[idx, 2], lo, n_time, store,
                             n_loud=N_LOUD, n_random=N_RANDOM, seed=0, precision="ref", bank_rows=idx,
                             n_bank=rows.shape[0])
    return time.perf_counter() - t0, idx, o["ln_lambda"][0]


def host_store(spec, s_nodes):
    from exmarg_b200 import synth
    from oracle import restate
    tables = restate.gen_tables(spec, s_nodes, TABLE_SEED)
    return synth.MemoryStore(spec, s_nodes, TABLE_SEED, tables=tables)


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from exmarg_b200 import bank as bank_mod
    from oracle import restate
    spec, s_nodes, seg, rows = make_inputs(args.warmup + args.steps, 0, args.templates, args.nodes, args.lags)
    store = host_store(spec, s_nodes)
    b = bank_mod.MassBank(rows[:, 0], rows[:, 1], rows[:, 2], seg, "b200")
    n_t = min(args.ref_templates, rows.shape[0])
    times = []
    for i in range(args.warmup + args.steps):
        t, _, _ = cpu_sample(seg, rows, b.W, b.u, b.lo, b.n_time, store, n_t, e=i)
        if i >= args.warmup:
            times.append(t)
    frac = n_t / float(rows.shape[0])
    value = args.steps * frac / sum(times)
    cores = restate.num_threads()
    sample = ("C port of the reference's CPU path (_gather_cpu + select_times + node and distance log-sum-exp, "
              "float64 over %d host threads), timed on %d of %d templates of each 8 s segment (all %d nodes, "
              "%d lags, 2048 walked times) and extrapolated to whole segments by %d/%d; each step analyses %.4f "
              "segment.  The port gives the reference's numba gather's results (to 4e-15) at 0.7-1.0x its time "
              "on the same host" % (cores, n_t, rows.shape[0], len(s_nodes), spec.ntau, rows.shape[0], n_t, frac))
    line = {"metric": METRIC, "value": value, "unit": "segments/s", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sum(times) / args.steps,
            "segments_per_step": frac,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args),
            "cpu_baseline": {"value": value, "unit": "segments/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "segments/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- B200 arm

PREC_SNRS = (5.0, 15.0, 30.0, 50.0)


def precision_legs(args, spec, s_nodes, rows, bank, store, store_h, gather_cfg, local):
    """the full workload on tables kept in HBM as float16 (per-node power-of-two scale) and as bfloat16:
    segments/s, and the ln B error against the float64 oracle on the float32 tables, sampled over
    args.prec_templates templates of one segment at each SNR in PREC_SNRS (float32 tables alongside)"""
    import exmarg_b200 as eb
    from exmarg_b200 import _lib, synth
    from oracle import restate
    n_t = min(args.prec_templates, rows.shape[0])
    idx = np.sort(np.random.default_rng(9).choice(rows.shape[0], n_t, replace=False))
    cell = restate.cell_weights(rows[idx, 0], rows[idx, 1], rows[idx, 2])
    segs = [synth.make_segments(1, 90000 + 17 * i, T=T_SEG, fmax=FMAX, snr=snr, mc=25.0, q=0.8, chi=0.1)
            for i, snr in enumerate(PREC_SNRS)]
    oracle, oracle_ref = [], []      # float64 throughout; the reference's precision (complex64 filter)
    for sg in segs:
        for prec, dst in (("fp64", oracle), ("ref", oracle_ref)):
            o = restate.pe_intrinsic(restate.read_segments(sg), bank.W[idx], bank.u[idx], rows[idx, 0], rows[idx, 1],
                                     rows[idx, 2], bank.lo, bank.n_time, store_h, n_loud=N_LOUD, n_random=N_RANDOM,
                                     seed=0, precision=prec, bank_rows=idx, n_bank=rows.shape[0])
            dst.append(restate.log_mean(o["ln_lambda"][0], cell))
    M, P, Q, S = spec.factors(s_nodes)
    out = {"snr": list(PREC_SNRS), "templates_sampled": n_t,
           "error": "|ln B - ln B_fp64| over the sampled templates; float64 oracle on the float32 tables"}
    for dt in ("f32", "f16", "bf16"):
        ctx, b, st = bank.ctx, bank, store
        if dt != "f32":
            ctx = _lib.Context(local)
            b = bank.clone_for(ctx)
            st = synth.MemoryStore(spec, s_nodes, TABLE_SEED, tables=[None] * len(s_nodes), table_dtype=dt)
            st.generator = (M, P, Q, S, TABLE_SEED)
            eb.prepare(b, st, "volume", 0.1267)
            ctx.set_gather_cfg(*gather_cfg)
        d = {}
        try:
            if dt != "f32":
                seg = make_inputs(args.warmup + args.prec_steps, 0, args.templates, args.nodes, args.lags)[2]
                for i in range(args.warmup):
                    eb.pe_intrinsic(seg, b, st, rows=[i])
                ctx.timing(True)
                for i in range(args.warmup, args.warmup + args.prec_steps):
                    eb.pe_intrinsic(seg, b, st, rows=[i])
                tm = ctx.timing(False)
                d["segments_per_s"] = args.prec_steps / (tm["total_ms"] / 1000.0)
                d["gather_ms"] = tm["gather_ms"] / args.prec_steps
                d["context_hbm_gb"] = ctx.bytes / 1e9   # tables + bank + workspace
            errs, errs_ref = [], []
            for sg, lb, lr in zip(segs, oracle, oracle_ref):
                r = eb.pe_intrinsic(sg, b, st, rows=[0])
                v = restate.log_mean(r["ln_lambda"][0][idx], cell)
                errs.append(abs(v - lb))
                errs_ref.append(abs(v - lr))
            d["max_abs_dlnB"] = float(max(errs))
            d["abs_dlnB_per_snr"] = [float(x) for x in errs]
            if dt == "f32":   # parity with the reference's own precision at every SNR
                d["abs_dlnB_vs_reference_per_snr"] = [float(x) for x in errs_ref]
                d["reference_vs_fp64_per_snr"] = [float(abs(a - c)) for a, c in zip(oracle_ref, oracle)]
        finally:
            if dt != "f32":
                ctx.close()
        out[dt] = d
    # float32 tables with the filter's ln|z| kept to float64 precision (filter_precision='fp64')
    d = {}
    try:
        seg = make_inputs(args.warmup + args.prec_steps, 0, args.templates, args.nodes, args.lags)[2]
        eb.pe_intrinsic(seg, bank, store, rows=[0], filter_precision="fp64")
        bank.ctx.timing(True)
        for i in range(args.warmup, args.warmup + args.prec_steps):
            eb.pe_intrinsic(seg, bank, store, rows=[i], filter_precision="fp64")
        tm = bank.ctx.timing(False)
        d["segments_per_s"] = args.prec_steps / (tm["total_ms"] / 1000.0)
        d["taps_ms"] = tm["taps_ms"] / args.prec_steps
        errs, errs_ref = [], []
        for sg, lb, lr in zip(segs, oracle, oracle_ref):
            r = eb.pe_intrinsic(sg, bank, store, rows=[0], filter_precision="fp64")
            v = restate.log_mean(r["ln_lambda"][0][idx], cell)
            errs.append(abs(v - lb))
            errs_ref.append(abs(v - lr))
        d["abs_dlnB_per_snr"] = [float(x) for x in errs]
        d["abs_dlnB_vs_reference_per_snr"] = [float(x) for x in errs_ref]
    finally:
        bank.ctx.set_filter_precision("reference")
    out["f32_filter_fp64"] = d
    return out


def batched_leg(args, store, bank, local, spec, s_nodes, rows, store_h):
    """the batched workload: args.batch_segments segments (8 s, float32 strain, network SNR drawn from U(0, 30),
    30 % noise-only) of the 2048-template bank on the resident store, as
      graph_replay: one pe_intrinsic call over all of them on a context that replays each segment as a
        captured CUDA graph (one segment on the device at a time);
      native_server: all submitted at once to the native request loop (exm_submit / exm_poll) with
        args.batch_workers workers of the bank, graph replay on each: segments overlap on the device, the
        oldest one's gather leading by stream priority.
    Every served ln Lambda is compared with the graph-replay call's (same bank, segment and seed); ln B of a
    sample of segments is checked against the float64 oracle on a template sample."""
    import exmarg_b200 as eb
    from exmarg_b200 import synth
    from oracle import restate
    n = args.batch_segments
    segs = synth.make_segments(n + 1, segment_seed(0) + 4242, T=T_SEG, fmax=FMAX, snr=(0.0, 30.0), noise_only=0.3,
                               mc=(10.0, 40.0), q=(0.25, 1.0), chi=(-0.5, 0.5), dtype=np.complex64)
    ctx = bank.ctx
    ctx.set_graph(True)
    try:
        eb.pe_intrinsic(segs, bank, store, rows=[0])          # first segment of the shape: runs, then is captured
        ctx.timing(True)
        t0 = time.perf_counter()
        res = eb.pe_intrinsic(segs, bank, store, rows=list(range(1, n + 1)))
        wall = time.perf_counter() - t0
        tm = ctx.timing(False)
    finally:
        ctx.set_graph(False)
    out = {"segments": n, "snr": "U(0, 30), 30% noise-only", "strain": "complex64",
           "graph_replay": {"segments_per_s": n / (tm["total_ms"] / 1000.0), "e2e_segments_per_s": n / wall}}
    # the native request loop, several workers of the one bank
    rd = eb.read_segments(segs)
    ctx.serve_start(hbm_budget=0, max_workers=args.batch_workers, n_loud=N_LOUD, n_random=N_RANDOM, graph=True)
    try:
        bid = ctx.serve_add_bank(bank.W, bank.lo, bank.n_time, bank.u, bank.M, bank.q, bank.chi, 0.1267)
        warm = [ctx.submit(bid, rd["d_H"][0], rd["d_L"][0], rd["sig2_H"], rd["sig2_L"], 0)
                for _ in range(args.batch_workers)]          # opens the workers and captures their graphs
        for h in warm:
            ctx.poll(h, bank.u.size)
        t0 = time.perf_counter()
        hs = [ctx.submit(bid, rd["d_H"][e], rd["d_L"][e], rd["sig2_H"], rd["sig2_L"], e) for e in range(1, n + 1)]
        got = [ctx.poll(h, bank.u.size) for h in hs]
        wall_s = time.perf_counter() - t0
        st = ctx.serve_stats()
    finally:
        ctx.serve_stop()
    same = all(np.array_equal(g[0], res["ln_lambda"][i]) for i, g in enumerate(got))
    out["native_server"] = {"workers": args.batch_workers, "segments_per_s": n / wall_s,
                            "identical_to_plain": bool(same), "workers_opened": st["workers_opened"]}
    # parity: the float64 oracle on a template sample of a few segments
    k_seg = min(args.batch_check_segments, n)
    idx = np.sort(np.random.default_rng(13).choice(rows.shape[0], args.batch_check_templates, replace=False))
    cell = restate.cell_weights(rows[idx, 0], rows[idx, 1], rows[idx, 2])
    errs = []
    for e in np.linspace(1, n, k_seg).astype(int):
        o = restate.pe_intrinsic(restate.read_segments(segs, rows=[int(e)]), bank.W[idx], bank.u[idx], rows[idx, 0],
                                 rows[idx, 1], rows[idx, 2], bank.lo, bank.n_time, store_h, n_loud=N_LOUD,
                                 n_random=N_RANDOM, seed=0, precision="ref", bank_rows=idx, n_bank=rows.shape[0])
        errs.append(abs(restate.log_mean(res["ln_lambda"][e - 1][idx], cell) - restate.log_mean(o["ln_lambda"][0], cell)))
    out["parity"] = {"segments_checked": k_seg, "templates": int(idx.size),
                     "max_abs_dlnB_vs_reference_port": float(max(errs))}
    out["ln_b_range"] = [float(np.min(res["ln_b"])), float(np.max(res["ln_b"]))]
    return out


def redshift_leg(args, store, seg, local):
    """pe_redshift as the reference's published timing runs it: a 120-template equal-mass, zero-spin bank of
    detector-frame total masses, 8 s segments on the resident 53-node store, the default (m1, z) grid of
    1600 x 1600, n_loud = n_random = 1024; ln Lambda on the grid is copied back for every segment.  Total
    masses run 8..150 Msun: above that the inspiral's ISCO frequency (4400 Hz Msun / M) falls below the 20 Hz
    band edge and a template has no power"""
    import exmarg_b200 as eb
    M = np.geomspace(8.0, 150.0, 120)
    bank = eb.MassBank(M, np.ones_like(M), np.zeros_like(M), seg, "b200", device_index=local)
    n = min(args.redshift_segments, seg["d_H"].shape[0] - 1)
    eb.pe_redshift(seg, bank, store, rows=[0])          # grid set-up and first-call costs
    t0 = time.perf_counter()
    res = eb.pe_redshift(seg, bank, store, rows=list(range(1, n + 1)))
    wall = time.perf_counter() - t0
    return {"segments": n, "templates": 120, "grid": "1600 m1 x 1600 z", "s_per_segment": wall / n,
            "segments_per_s": n / wall, "reference_published_s_per_segment": 0.102,
            "reference_published_hardware": "1 L40S, cupy, batches of 16",
            "ln_b_range": [float(np.min(res["ln_b"])), float(np.max(res["ln_b"]))]}


def store_io_leg(args, local):
    """loading a store into HBM: io_nodes production-shape node files (87 x 49 x 200 x 219 float32,
    0.75 GB each) written to a temporary directory, then loaded into a fresh context (created and
    declared before the clock starts) --
      reference_pattern: as the reference does it, `readers` threads read every table into host
        memory, then one pageable copy per node;
      native_files: the native loader streaming the files (buffered reads, reads overlapped with copies);
      native_files_direct: the same with O_DIRECT (the disk's own rate);
      native_from_host: the native loader from tables already in host memory.
    "cold" legs first drop these files' pages from the page cache (fsync, then posix_fadvise
    DONTNEED on each file), so their reads come from the disk; "hot" legs read every file once
    first, so their reads hit the page cache (median of three).
    Every load is checked bit for bit on its first and last node."""
    import shutil
    import tempfile
    import torch
    from exmarg_b200 import _lib, synth
    from exmarg_b200.store import load_redshift_store, store_grid
    n, R = args.io_nodes, args.io_readers
    spec = synth.TableSpec()
    s_nodes = synth.S_NODES_PROD[np.linspace(0, 52, n).astype(int)]
    d = tempfile.mkdtemp(prefix="exmarg_store_", dir=args.io_dir)
    out = {"nodes": n, "node_bytes": int(np.prod(spec.shape)) * 4, "readers": R}
    try:
        T = np.random.default_rng(1).random(spec.shape, dtype=np.float32)
        t0 = time.perf_counter()
        for k, sk in enumerate(s_nodes):
            T.flat[0] = np.float32(k)
            np.savez(os.path.join(d, "bd_n120_s%09.3f.npz" % sk), T=T, beta=spec.beta, delta=spec.delta,
                     tau_idx=spec.tau_idx, alpha=synth.ALPHA, s_node=float(sk))
        out["write_s"] = time.perf_counter() - t0
        total = n * out["node_bytes"]

        h = torch.empty(1 << 30, dtype=torch.uint8).pin_memory()       # the host-to-device ceiling
        g = torch.empty(1 << 30, dtype=torch.uint8, device="cuda:%d" % local)
        g.copy_(h, non_blocking=True)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(4):
            g.copy_(h, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        out["pinned_h2d_GB_per_s"] = 4 * (1 << 30) / (e0.elapsed_time(e1) * 1e-3) / 1e9
        del h, g
        torch.cuda.empty_cache()

        def drop_cached():
            for f in os.listdir(d):
                fd = os.open(os.path.join(d, f), os.O_RDONLY)
                try:
                    os.fsync(fd)
                    os.posix_fadvise(fd, 0, 0, os.POSIX_FADV_DONTNEED)
                finally:
                    os.close(fd)

        def warm_cache():
            for f in os.listdir(d):
                with open(os.path.join(d, f), "rb", buffering=0) as fh:
                    while fh.read(64 << 20):
                        pass

        def check(ctx):
            for k in (0, n - 1):
                T.flat[0] = np.float32(k)
                if not np.array_equal(ctx.store_get_node(k, spec.shape), T):
                    raise RuntimeError("store load: node %d differs from its file" % k)

        meta = load_redshift_store(d, mmap=True)

        def leg(kind, cold):
            ctx = _lib.Context(local)
            b0, db, d0, dd = store_grid(meta)
            ctx.store_init(n, spec.shape, meta.tau_idx, b0, db, d0, dd)
            host = load_redshift_store(d, readers=R) if kind == "host" else None
            if cold:
                drop_cached()
            stats = None
            t0 = time.perf_counter()
            if kind == "reference":
                st = load_redshift_store(d, readers=R)
                for k in range(n):
                    ctx.store_set_node(k, st.s[k], st.alpha_lo[k], st.alpha_hi[k], st.tables[k])
            elif kind == "host":
                stats = ctx.store_load(0, host.s, host.alpha_lo, host.alpha_hi, hosts=host.tables, readers=R)
            else:
                st = load_redshift_store(d, mmap=True)
                stats = ctx.store_load(0, st.s, st.alpha_lo, st.alpha_hi, paths=st.files, offsets=st.t_offsets,
                                       readers=R, direct=(kind == "direct"))
            dt = time.perf_counter() - t0
            check(ctx)
            ctx.close()
            r = {"seconds": dt, "GB_per_s": total / dt / 1e9, "seconds_for_53_nodes": dt * 53.0 / n}
            if stats is not None:
                r["loader_seconds"] = stats["seconds"]
                r["reader_seconds"] = stats["read_seconds"]
                r["issuer_wait_seconds"] = stats["issue_wait_seconds"]
            return r

        def median_of(kind, reps=3):
            runs = []
            for _ in range(reps):
                warm_cache()
                runs.append(leg(kind, False))
            return sorted(runs, key=lambda r: r["seconds"])[reps // 2]

        out["legs"] = {
            "reference_pattern_cold": leg("reference", True),
            "native_files_cold": leg("files", True),
            "native_files_direct": leg("direct", True),
            "reference_pattern_hot": median_of("reference"),
            "native_files_hot": median_of("files"),
            "native_from_host": median_of("host"),
        }
        out["reference_published"] = "23 s for the 53-node store (39.6 GB), load_redshift_store with 6 readers"
    finally:
        shutil.rmtree(d, ignore_errors=True)
    return out


def table_build_leg(args, local):
    """stage 3 of the offline table build for one production-shape node: 121 orders (n_max 120), 87 lags,
    110 magnitudes (200 x 219 table), 49 phases, synthetic lnK edges.  Device: exm_bd_build (kernel time
    and time with the host copies), median of 3.  CPU baseline: the reference's algorithm (numpy, float64,
    the restatement in oracle/) on one lag, scaled by the 87 lags."""
    from scipy.special import gammaln
    from exmarg_b200 import _lib, tables
    nord, ntau, nq, nphif = 121, 87, 110, 49
    rng = np.random.default_rng(5)
    lnq = np.log(np.geomspace(0.05, 100.0, nq))
    n = np.arange(nord, dtype=np.float64)[:, None, None, None]
    t = np.arange(ntau, dtype=np.float64)[None, :, None, None]
    ph = (2 * np.pi * np.arange(nphif) / 96.0)[None, None, None, :]
    dq = np.abs(lnq - lnq[-1])[None, None, :, None]
    base = n * (0.4 * np.cos(ph) + 0.01 * t - 0.3 * dq) - gammaln(n + 1.0)
    col = (2 * n * lnq[-1] + base + 0.01 * rng.standard_normal(base.shape)).astype(np.float32)
    row = (2 * n * lnq[None, None, :, None] + base + 0.01 * rng.standard_normal(base.shape)).astype(np.float32)
    ctx = _lib.context(local)
    beta, _ = tables.bd_grid(lnq)
    runs = []
    for _ in range(4):
        T, bad, ms = ctx.bd_build(col, row, lnq, beta, [nord - 1])
        runs.append(ms)
    runs = sorted(runs[1:], key=lambda m: m[0])
    k_ms, all_ms = runs[1]
    nout = ntau * nphif * beta.size * (2 * nq - 1)
    out = {"orders": nord, "lags": ntau, "table": [ntau, nphif, int(beta.size), 2 * nq - 1], "kernel_ms": k_ms,
           "ms_with_copies": all_ms, "non_finite": bad, "exp_per_s": nout * nord / (k_ms * 1e-3),
           "seconds_for_53_nodes": all_ms * 1e-3 * 53}
    # stage 2 on the lnK edges for the same node shape: synthetic rebinned W of every key (n <= 120) on 87 lags,
    # the production magnitude grid (110) and 96 phases
    from exmarg_b200 import wtable
    keys = np.array(wtable.keys(nord - 1))
    Wd = np.exp(rng.normal(-3.0, 1.0, (keys.shape[0], ntau)))
    coeff, gmo, cosm = tables.k_inputs(keys, 25.0, nord - 1, lnq, 96)
    k_runs = sorted(ctx.k_edges(nord - 1, Wd, coeff, lnq, gmo, cosm)[2] for _ in range(3))
    out["stage2_edges_kernel_ms"] = k_runs[1]
    out["stage2_plus_3_kernel_ms"] = k_runs[1] + k_ms
    if not args.no_cpu:
        from oracle import restate
        phi = np.arange(96) * (2 * np.pi / 96)
        t0 = time.perf_counter()
        restate.k_order(60, 25.0, keys, Wd, lnq, phi)
        one = time.perf_counter() - t0
        scale = sum((n + 1) ** 2 for n in range(nord)) / 61.0 ** 2
        out["cpu_baseline_stage2"] = {"seconds_per_node": one * scale, "cores": "numpy BLAS threads", "kind": "port",
                                      "sample": "order 60 of 121 on the full 110 x 110 x 96 grid (the reference's "
                                                "work), scaled by sum (n+1)^2 / 61^2"}
        t0 = time.perf_counter()
        ref = restate.bd_tables(col[:, :1], row[:, :1], lnq, beta, [nord - 1])[nord - 1]
        cpu_lag = time.perf_counter() - t0
        d = np.abs(ref.astype(np.float64) - T[0, 0].astype(np.float64))
        out["cpu_baseline"] = {"seconds_per_node": cpu_lag * ntau, "cores": 1, "kind": "port",
                               "sample": "lag 0 of 87 (49 phases x 200 x 219 x 121 orders), scaled by 87"}
        out["max_abs_diff_vs_cpu_lag0"] = float(d.max())
    return out


def w_build_leg(args, local):
    """stage 1 of the offline table build at the published settings (n_max 120, nside 32: 12288 pixels,
    257 delays, 53 nodes; 302621 keys, 243 x 123 quadrature points): exm_w_build on w_pixels pixels spread
    over the sky, the whole build projected from the time per pixel (the pixels are independent and
    equally costly).  CPU baseline: the reference's per-key quadrature (numpy, float64) for a sample of
    keys of one pixel, scaled to a pixel."""
    import torch
    from exmarg_b200 import wtable, _lib, synth
    s_nodes = synth.S_NODES_PROD[np.linspace(0, 52, min(53, args.w_nodes)).astype(int)]
    npix = wtable.nside2npix(wtable.NSIDE)
    pix = np.linspace(0, npix - 1, args.w_pixels).astype(int)
    g = wtable.geometry(wtable.NSIDE, wtable.N_MAX, wtable.N_TAU, pix)
    sc = wtable.scales(s_nodes, wtable.N_MAX)
    ctx = _lib.context(local)
    W, ms = ctx.w_build(s_nodes, wtable.N_MAX, g, sc)
    per_px = ms[0] / pix.size
    q = 243 * 123
    fma = s_nodes.size * q * float(sc.shape[1])
    # the FP64 denominator: cuBLAS DGEMM 8192^3, best of 5
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda:%d" % local)
    b = torch.randn_like(a)
    torch.matmul(a, b)
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    dgemm_tf = 2 * 8192.0 ** 3 / (best * 1e-3) / 1e12
    del a, b
    torch.cuda.empty_cache()
    tiles = 0
    for m in range(wtable.N_MAX + 1):
        L = wtable.N_MAX - m + 1
        for x0 in range(0, L, 8):
            tiles += len(range(0, L - x0, 16))
    exec_tf = 2.0 * tiles * 64 * 128 * q / (per_px * 1e-3) / 1e12
    out = {"pixels_run": int(pix.size), "ms_per_pixel": per_px, "projected_build_s": per_px * 1e-3 * npix,
           "reference_published_s": 7.1 * 3600, "reference_published": "7.1 h for the 53 nodes on one GPU (build_w.py:5-6)",
           "nodes": int(s_nodes.size), "fp64_fma_per_pixel": fma, "fp64_tflops_useful": 2 * fma / (per_px * 1e-3) / 1e12,
           "fp64_tflops_executed": exec_tf, "dgemm_tflops_measured": dgemm_tf,
           "frac_of_dgemm": exec_tf / dgemm_tf, "ms_with_copies": ms[1], "finite": bool(np.isfinite(W).all())}
    if not args.no_cpu:
        th, ph = wtable.pix2ang(wtable.NSIDE, pix[:1])
        psi, cg, wq = wtable.quadrature(wtable.N_MAX)
        R = []
        for I in "HL":
            fp, fx = (np.float32(v[0]) for v in wtable.antenna(I, th, ph))
            c2, s2 = np.cos(2 * psi).astype(np.float32), np.sin(2 * psi).astype(np.float32)
            Fp, Fx = fp * c2 - fx * s2, fp * s2 + fx * c2
            R.append((np.float32(0.5) * (1 + cg.astype(np.float32) ** 2)[None, :] * Fp[:, None]
                      + 1j * cg.astype(np.float32)[None, :] * Fx[:, None]).astype(np.complex64).ravel())
        S1, S2 = (np.abs(r).astype(np.float64) ** 2 for r in R)
        dph = (np.angle(R[0]) - np.angle(R[1])).astype(np.float64)
        m1, m2 = np.sqrt(S1 / 2), np.sqrt(S2 / 2)
        wqf = np.broadcast_to(wq[None, :], (psi.size, cg.size)).ravel()
        ks = wtable.keys(wtable.N_MAX)
        sample = ks[::max(1, len(ks) // 200)]
        t0 = time.perf_counter()
        Bw = np.stack([np.exp(-(sj * S1 + sj * S2)) for sj in s_nodes]) * wqf[None, :]
        for (n, a, b) in sample:
            (Bw * np.cos((a - b) * dph)[None, :]) @ (m1 ** (a + b) * m2 ** (2 * n - a - b))
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"seconds_per_pixel": dt * len(ks) / len(sample), "cores": 1, "kind": "port",
                               "sample": "%d of %d keys of one pixel, scaled" % (len(sample), len(ks))}
    return out


def shard_leg(args, store, seg, bank, local):
    """node sharding projected on one GPU: the store's nodes split into 2, 4 and 8 ranges (node_ranges);
    each range's node values for one segment (filter, time selection, taps, gather, lag log-sum-exp) timed
    on a context of its own that holds only that range's tables, one range after another.  The slowest
    range is the per-segment time of an N-GPU node-sharded run before its exchange (one all-reduce of
    54 x 2048 float64 = 0.9 MB) and the node log-sum-exp on the host (timed here).  Timing only: a range's
    tables are generated with range-local seeds (the device generator hashes a node's index in its store),
    so their values differ from the whole store's; the work -- nodes, (node, template) pairs, taps -- is
    the same."""
    import exmarg_b200 as eb
    from exmarg_b200 import _lib, shard as sh, synth
    M, P, Q, S, seed = store.generator
    nn = len(store.s)
    rd = eb.read_segments(seg)

    def time_range(k0, k1):
        sub = synth.MemoryStore(store.spec, store.s[k0:k1], seed, tables=[None] * (k1 - k0))
        sub.generator = (M, P, Q, S[k0:k1], seed)
        if (k0, k1) != (0, nn):
            sub.shard_s_before = float(store.s[k0 - 1]) if k0 > 0 else 0.0
        ctx = _lib.Context(local)
        try:
            b = bank.clone_for(ctx)
            eb.prepare(b, sub, "volume", 0.1267)
            ts, lam = [], None
            for rep in range(3):
                e = rep % rd["rows"].size
                t0 = time.perf_counter()
                ctx.filter(rd["d_H"][e:e + 1], rd["d_L"][e:e + 1], rd["sig2_H"], rd["sig2_L"], want=False)
                ctx.select_times(int(rd["rows"][e]), N_LOUD, N_RANDOM, want=False)
                lam = ctx.node_values(k1 - k0)
                ts.append(time.perf_counter() - t0)
            return min(ts[1:]) * 1e3, lam
        finally:
            ctx.close()

    full_ms, lam = time_range(0, nn)
    lnW = sh.node_weights(store, np.asarray(bank.u, float), 0.1267, "volume")
    t0 = time.perf_counter()
    sh.combine(lam[None], lnW, bank.M, bank.q, bank.chi)
    combine_ms = (time.perf_counter() - t0) * 1e3
    out = {"whole_store_node_values_ms": full_ms, "host_combine_ms": combine_ms,
           "exchange_estimate_ms": 0.02, "exchange": "0.9 MB all-reduce over NVLink (770 GB/s measured peer copy "
           "on this pool), not run: one GPU per call here", "ranges": {}}
    for n in (2, 4, 8):
        ranges = sh.node_ranges(store, np.asarray(bank.u, float), 0.1267, n)
        per = [time_range(k0, k1)[0] for k0, k1 in ranges]
        out["ranges"][str(n)] = {"node_ranges": ranges, "ms_per_range": per, "slowest_ms": max(per),
                                 "projected_segment_ms": max(per) + combine_ms + 0.02}
    return out


def serving_legs(args, store, bank, seg, rows, plain, capacity, local):
    """segments served by exmarg_b200.serve.Server: child contexts sharing the resident tables, three
    banks -- all 2048 templates on 8 s segments, the first 1024 on 16 s segments (n_time 65536), all 2048
    on 4 s segments (n_time 16384) -- in equal parts, graph replay on the workers.  'batched': every request
    queued at once (segments in flight together); 'poisson': arrivals at 80 % of the plain path's
    2048-template 8 s capacity.  Served ln Lambda of the 2048-template 8 s bank is compared bitwise
    with the plain call's."""
    import exmarg_b200 as eb
    from exmarg_b200 import synth
    from exmarg_b200.serve import Request, Server, latency_stats
    # the 16 s and 4 s segments follow the serving config's data: network SNR U(0, 50), 90% noise-only
    seg16 = synth.make_segments(8, segment_seed(0) + 1616, T=16.0, fmax=FMAX, snr=(0.0, 50.0), noise_only=0.9, mc=25.0,
                                q=0.8, chi=0.1)
    long = eb.MassBank(rows[:1024, 0], rows[:1024, 1], rows[:1024, 2], seg16, "b200", device_index=local)
    seg4 = synth.make_segments(8, segment_seed(0) + 777, T=4.0, fmax=FMAX, snr=(0.0, 50.0), noise_only=0.9, mc=25.0,
                               q=0.8, chi=0.1)
    short = eb.MassBank(rows[:, 0], rows[:, 1], rows[:, 2], seg4, "b200", device_index=local)
    banks = {"bank2048": bank, "bank1024_16s": long, "bank2048_4s": short}
    segs = {"bank2048": seg, "bank1024_16s": seg16, "bank2048_4s": seg4}
    first = args.warmup
    n_req = args.serve_requests
    n_rows = len(plain)
    keys = ("bank2048", "bank1024_16s", "bank2048_4s")
    mix = [(keys[i % 3], first + (i % n_rows) if i % 3 == 0 else i % 8) for i in range(n_req)]
    out = {}
    srv = Server(store, banks, device=local, max_workers=args.serve_workers, graph=True)
    try:
        # warm-up with the same mix (workers per bank as the mix needs them: allocation, FFT plans,
        # graph capture happen here)
        srv.serve([Request(-1 - i, k, segs[k], row=0) for i, (k, _) in enumerate(mix[:4 * args.serve_workers])])
        for leg in ("batched", "poisson"):
            reqs = [Request(i, k, segs[k], row=r) for i, (k, r) in enumerate(mix)]
            if leg == "batched":
                arrivals = None
            else:
                rate = 0.8 * capacity
                arrivals = np.cumsum(np.random.default_rng(7).exponential(1.0 / rate, n_req)) - 1.0 / rate
            done = srv.serve(reqs, arrivals)
            same = True
            for r in done:
                lnl, _ = r.future.result()
                if r.key == "bank2048":
                    same &= bool(np.array_equal(lnl, plain[r.row - first]["ln_lambda"][0]))
            st = latency_stats(done)
            d = {"requests": n_req, "workers": args.serve_workers, "segments_per_s": st["segments_per_s"],
                 "latency_ms_p50": st["p50_ms"], "latency_ms_p99": st["p99_ms"],
                 "service_ms_p50": st["service_ms_p50"], "service_ms_max": st["service_ms_max"],
                 "workers_created": srv.n_created, "workers_evicted": srv.n_evicted,
                 "identical_to_plain": same,
                 "banks": "2048 templates / 8 s (SNR 15), 1024 / 16 s and 2048 / 4 s (SNR U(0, 50), 90% noise-only)"}
            if leg == "poisson":
                d["offered_per_s"] = 0.8 * capacity
            out[leg] = d
    finally:
        srv.close()
    return out


SERVE_BANKS = (("b256_4s", 256, 4.0), ("b256_16s", 256, 16.0), ("b2048_8s", 2048, 8.0), ("b2048_16s", 2048, 16.0),
               ("b8192_4s", 8192, 4.0), ("b8192_8s", 8192, 8.0))


def serve_config_leg(args, store, local):
    """The serving workload through the native request loop (exm_submit / exm_poll): banks of 256, 2048 and 8192
    TaylorF2 templates on 4, 8 and 16 s segments (SERVE_BANKS; 2048 Hz strain, 20-512 Hz analysed), segments
    with network SNR U(0, 50) and 90 % noise-only, the 53-node store resident, workers opened and closed within
    the HBM budget.  First args.serve_capacity_requests requests are queued at once: their rate is the mixed
    capacity.  Then args.serve_poisson_requests arrive as a Poisson stream at args.serve_load x that capacity
    (the config's 400 req/s is stated beside it as a multiple of the capacity).  Latency is arrival to result
    (p50 / p99); a sample of served results is compared bitwise with the plain single-segment path."""
    import exmarg_b200 as eb
    from exmarg_b200 import _lib, synth
    ctx = eb.context(local)
    rng = np.random.default_rng(2027)
    banks, segs = {}, {}
    for key, nm, T in SERVE_BANKS:
        sg = synth.make_segments(16, segment_seed(0) + int(T * 1000) + nm, T=T, fmax=FMAX, snr=(0.0, 50.0),
                                 noise_only=0.9, mc=(10.0, 40.0), q=(0.25, 1.0), chi=(-0.5, 0.5))
        rows = synth.make_bank(nm, BANK_SEED + nm)
        banks[key] = eb.MassBank(rows[:, 0], rows[:, 1], rows[:, 2], sg, "b200", device_index=local)
        segs[key] = eb.read_segments(sg)
    keys = [k for k, _, _ in SERVE_BANKS]
    weights = np.array([0.2, 0.2, 0.2, 0.15, 0.15, 0.1])
    n_cap, n_poi = args.serve_capacity_requests, args.serve_poisson_requests
    mix = [(keys[int(rng.choice(len(keys), p=weights))], int(rng.integers(0, 16))) for _ in range(n_cap + n_poi)]
    free0, total0 = _lib.device_memory(local)
    budget = int(args.serve_budget_gb * 1e9) if args.serve_budget_gb > 0 else 0
    ctx.serve_start(hbm_budget=budget, max_workers=args.serve_config_workers, n_loud=N_LOUD, n_random=N_RANDOM,
                    graph=True)
    out = {"banks": {k: {"templates": nm, "segment_s": T} for k, nm, T in SERVE_BANKS},
           "mix_weights": weights.tolist(), "snr": "U(0, 50), 90% noise-only", "workers_max": args.serve_config_workers}
    try:
        ids = {k: ctx.serve_add_bank(b.W, b.lo, b.n_time, b.u, b.M, b.q, b.chi, 0.1267) for k, b in banks.items()}
        stats0 = ctx.serve_stats()
        out["hbm_budget_gb"] = stats0["budget"] / 1e9

        def submit(key, e):
            sg = segs[key]
            return ctx.submit(ids[key], sg["d_H"][e], sg["d_L"][e], sg["sig2_H"], sg["sig2_L"], e)

        # warm-up: one request per bank (opens workers, plans, graphs)
        t_w = time.perf_counter()
        for k in keys:
            ctx.poll(submit(k, 0), banks[k].u.size)
        out["warmup_s"] = time.perf_counter() - t_w
        print("serve-config: workers open (%.1f s)" % out["warmup_s"], file=sys.stderr, flush=True)
        # capacity: everything queued at once
        t0 = time.perf_counter()
        hs = [(submit(k, e), k, e) for k, e in mix[:n_cap]]
        served = [(ctx.poll(h, banks[k].u.size), k, e) for h, k, e in hs]
        cap = n_cap / (time.perf_counter() - t0)
        out["capacity"] = {"requests": n_cap, "segments_per_s": cap}
        print("serve-config: capacity %.2f segments/s" % cap, file=sys.stderr, flush=True)
        # the Poisson stream at a stated fraction of that capacity
        rate = args.serve_load * cap
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n_poi))
        pend, lat, done_t = {}, [], []
        t0 = time.perf_counter()
        i = 0
        while i < n_poi or pend:
            now = time.perf_counter() - t0
            if now > args.serve_max_s and i < n_poi:        # a wall-clock guard: stop offering, drain
                n_poi = i
                print("serve-config: stream cut at %d requests after %.0f s" % (i, now), file=sys.stderr, flush=True)
            while i < n_poi and arrivals[i] <= now:
                k, e = mix[n_cap + i]
                pend[submit(k, e)] = (k, arrivals[i])
                i += 1
            for h in list(pend):
                k, ta = pend[h]
                r = ctx.poll(h, banks[k].u.size, timeout_us=0)
                if r is not None:
                    tn = time.perf_counter() - t0
                    lat.append(tn - ta)
                    done_t.append(tn)
                    del pend[h]
            time.sleep(0.0005)
        st = ctx.serve_stats()
        lat = np.array(lat)
        out["poisson"] = {"requests": n_poi, "requests_planned": args.serve_poisson_requests, "offered_per_s": rate, "offered_fraction_of_capacity": args.serve_load,
                          "segments_per_s": n_poi / (max(done_t) - arrivals[0]),
                          "latency_ms_p50": float(np.percentile(lat, 50) * 1e3),
                          "latency_ms_p99": float(np.percentile(lat, 99) * 1e3),
                          "config_rate_400_per_s_as_multiple_of_capacity": 400.0 / cap}
        out["workers_opened"], out["workers_closed_for_budget"] = st["workers_opened"], st["workers_closed"]
        out["failed"] = st["failed"]
    finally:
        ctx.serve_stop()
    # bitwise check of served results against the plain path on the parent context (a sample)
    same, checked = True, 0
    for (lnl, lnb), k, e in served[:: max(1, len(served) // 12)]:
        r = eb.pe_intrinsic(segs[k], banks[k], store, rows=[e], seed=0)
        same &= bool(np.array_equal(r["ln_lambda"][0], lnl)) and float(r["ln_b"][0]) == lnb
        checked += 1
    out["identical_to_plain"] = {"checked": checked, "bitwise": same}
    out["device_memory_gb"] = {"free_at_start": free0 / 1e9, "total": total0 / 1e9}
    return out


def run_b200(args):
    rank, world, local = dist_env()
    import exmarg_b200 as eb
    from exmarg_b200 import synth, _lib
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    n_seg = args.warmup + args.steps
    spec, s_nodes, seg, rows = make_inputs(n_seg, rank, args.templates, args.nodes, args.lags)
    ctx = eb.context(local)
    bank = eb.MassBank(rows[:, 0], rows[:, 1], rows[:, 2], seg, "b200", device_index=local)
    # the store: every node generated on the device (no 40 GB host copy on the measured path)
    M, P, Q, S = spec.factors(s_nodes)
    store = synth.MemoryStore(spec, s_nodes, TABLE_SEED, tables=[None] * len(s_nodes))
    store.generator = (M, P, Q, S, TABLE_SEED)
    eb.prepare(bank, store, "volume", 0.1267)

    # the clock sampler starts before the warm-up: its start-up (NVML initialisation) holds the
    # driver for a moment and must not fall inside the timed region
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(2.0)
    for i in range(args.warmup):
        eb.pe_intrinsic(seg, bank, store, rows=[i])
    tune = None
    if args.gather_cfg >= 0:
        ctx.set_gather_cfg(args.gather_cfg, args.gather_chunk_pct)
        tune = {"chosen": args.gather_cfg, "chunk_pct": ctx.gather_chunk_pct, "forced": True}
    elif not args.no_tune:
        best, ms = ctx.autotune(N_LOUD, N_RANDOM, reps=2)
        ns = len(_lib.GATHER_SHAPES)
        tune = {"chosen": int(best), "ms_per_shape": [round(float(x), 3) for x in ms[:ns]],
                "chunk_pct_chosen": ctx.gather_chunk_pct,
                "ms_per_chunk_pct": {str(p): round(float(x), 3) for p, x in zip((50, 150, 200), ms[ns:ns + 3])},
                "shapes": list(_lib.GATHER_SHAPES)}
    ctx.timing(True)
    if pg:
        pg.barrier()
    lat = []
    res = []
    tw0 = time.time()
    t0 = time.perf_counter()
    for i in range(args.warmup, n_seg):
        a = time.perf_counter()
        r = eb.pe_intrinsic(seg, bank, store, rows=[i])
        lat.append(time.perf_counter() - a)
        res.append(r)
    wall = time.perf_counter() - t0
    clocks.mark(tw0, time.time())
    clk = clocks.stop()
    tm = ctx.timing(False)
    dev_s = tm["total_ms"] / 1000.0
    if pg:
        dev_s, wall = combine_ranks([dev_s, wall], pg)
        pg.barrier()
    total = args.steps * world
    value = total / dev_s
    e2e = total / wall
    nf = bank.W.shape[1]
    launches = tm["gather_launches"]
    g_ms = tm["gather_ms"] / max(launches, 1)
    bytes_per_launch = (32.0 * tm["node_taps"] + 16.0 * tm["tlw_taps"]) / max(launches, 1)
    peak, peak_kind = measured_peaks()
    achieved = bytes_per_launch / (g_ms / 1000.0) / 1e9
    node_taps_launch = tm["node_taps"] / max(launches, 1)
    traffic, l2_hit, traffic_why = gather_traffic(node_taps_launch)
    dram_gbs = (traffic / (g_ms / 1000.0) / 1e9) if traffic else None
    line = {"metric": METRIC, "value": value, "unit": "segments/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * dev_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": workload_config(args),
            "e2e": {"value": e2e, "unit": "segments/s", "h2d_bytes_per_step": 6 * nf * 8,
                    "d2h_bytes_per_step": rows.shape[0] * 8 + 8 + 4,
                    "latency_ms_p50": 1000.0 * float(np.percentile(lat, 50)),
                    "latency_ms_p99": 1000.0 * float(np.percentile(lat, 99))},
            "gpu_launches": int(tm["launches"]),
            "exact_path_taps_per_step": tm["slow_taps"] / args.steps,
            "boundary_taps_per_step": tm["boundary_taps"] / args.steps,
            "stages_ms_per_step": {k: tm[k] / args.steps for k in ("filter_ms", "select_ms", "taps_ms", "gather_ms",
                                                                    "epilogue_ms")},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "achieved_is": "logical gather bytes (32 B per node-tap + 16 B of trajectory per tap) per "
                                        "launch / CUDA-event launch time; served from shared memory, not DRAM",
                         "traffic": traffic, "traffic_is": "ncu dram read + write bytes per node-tap of a reduced "
                                                           "case x this launch's node-taps" if traffic else traffic_why,
                         "achieved_dram": dram_gbs, "frac_dram": (dram_gbs / peak) if dram_gbs else None,
                         "l2_read_hit_rate": l2_hit,
                         "kernel": "k_gather_planes", "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": bytes_per_launch, "launch_ms": g_ms,
                         "node_taps_per_launch": node_taps_launch},
            "gather_gbs_logical": achieved, "clocks": clk, "autotune": tune}
    if rank == 0 and world == 1 and args.serve_config:
        line["serving_config"] = serve_config_leg(args, store, local)
    if rank == 0 and world == 1 and args.serve_requests > 0:
        line["serving"] = serving_legs(args, store, bank, seg, rows, res, value, local)

    if rank == 0 and world == 1 and args.redshift_segments > 0:
        line["redshift"] = redshift_leg(args, store, seg, local)
    if rank == 0 and world == 1 and args.io_nodes > 0:
        line["store_io"] = store_io_leg(args, local)
    if rank == 0 and world == 1 and args.shard_legs:
        line["node_shards"] = shard_leg(args, store, seg, bank, local)
    if rank == 0 and world == 1 and args.table_build:
        line["table_build"] = table_build_leg(args, local)
    if rank == 0 and world == 1 and args.w_pixels > 0:
        line["w_build"] = w_build_leg(args, local)
    if rank == 0 and world == 1 and not args.no_cpu:
        # CPU baseline and parity: the oracle on a template sample of the first timed segment
        store_h = host_store(spec, s_nodes)
        n_t = min(args.cpu_templates, rows.shape[0])
        t_cpu, idx, lnl_cpu = cpu_sample(seg, rows, bank.W, bank.u, bank.lo, bank.n_time, store_h, n_t,
                                         e=args.warmup)
        from oracle import restate
        frac = n_t / float(rows.shape[0])
        lnl_gpu = res[0]["ln_lambda"][0][idx]
        cell = restate.cell_weights(rows[idx, 0], rows[idx, 1], rows[idx, 2])
        line["cpu_baseline"] = {"value": frac / t_cpu, "unit": "segments/s", "cores": restate.num_threads(),
                                "kind": "port",
                                "sample": "%d of %d templates of one segment (all 53 nodes, 87 lags, 2048 walked "
                                          "times), float64 C gather, %.1f s" % (n_t, N_TEMPLATES, t_cpu)}
        line["parity"] = {"templates": n_t, "max_abs_dlnlambda": float(np.abs(lnl_gpu - lnl_cpu).max()),
                          "sample_dlnB": float(abs(restate.log_mean(lnl_gpu, cell) - restate.log_mean(lnl_cpu, cell)))}
        if args.templates == N_TEMPLATES and args.nodes == 53 and args.lags == 87:
            # the DRAM floor of the gather: table sectors a 64-template sample touches (5 lags, scaled), plus the
            # trajectories read once (2 detectors x nm x n_time x 8 B)
            t0c = time.perf_counter()
            sub = idx[:64]
            s1 = restate.read_segments(seg, rows=[args.warmup])
            traj = restate.trajectories(bank.W[sub], {I: s1["d_" + I][0] for I in "HL"},
                                        {I: s1["sig2_" + I] for I in "HL"}, bank.lo, bank.n_time, "ref")
            sel, _ = restate.select_times(traj, spec.tau_idx, N_LOUD, N_RANDOM, 0, bank_rows=sub,
                                          n_bank=rows.shape[0])
            lags = spec.tau_idx[np.linspace(0, spec.ntau - 1, 5).astype(int)]
            comp = compulsory_table_bytes(traj, sel, bank.u[sub], spec, s_nodes, lags)
            comp += 2.0 * rows.shape[0] * bank.n_time * 8
            rl = line["roofline"]
            rl["compulsory_bytes_per_launch_lower_bound"] = comp
            rl["compulsory_is"] = ("distinct 32-B table sectors touched by a 64-template sample (5 of 87 lags, "
                                   "scaled) + trajectories once; %.1f s on the host" % (time.perf_counter() - t0c))
            rl["dram_floor_ms"] = comp / (peak * 1e9) * 1e3
        if args.batch_segments > 0:
            line["batched"] = batched_leg(args, store, bank, local, spec, s_nodes, rows, store_h)
        if args.prec_templates > 0:
            cfg = (ctx.gather_cfg if ctx.gather_cfg is not None else 0, ctx.gather_chunk_pct)
            line["precision"] = precision_legs(args, spec, s_nodes, rows, bank, store, store_h, cfg, local)
        del store_h
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-templates", type=int, default=128)
    ap.add_argument("--ref-templates", type=int, default=64)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-tune", action="store_true", help="skip the gather launch-shape autotuner")
    ap.add_argument("--templates", type=int, default=N_TEMPLATES, help="bank size (reduced profiling cases)")
    ap.add_argument("--nodes", type=int, default=53, help="store nodes (reduced profiling cases)")
    ap.add_argument("--lags", type=int, default=87, help="table lags (reduced profiling cases; odd)")
    ap.add_argument("--gather-cfg", type=int, default=-1, help="force a gather launch shape (no autotuning)")
    ap.add_argument("--gather-chunk-pct", type=int, default=0,
                    help="with --gather-cfg: templates per gather block in percent of the default (0: 100)")
    ap.add_argument("--prec-templates", type=int, default=64,
                    help="templates of the float64 oracle sample of the 16-bit table legs (0: no such legs)")
    ap.add_argument("--prec-steps", type=int, default=5, help="timed segments of each 16-bit table leg")
    ap.add_argument("--shard-legs", type=int, default=1, help="node-sharding projection leg (0: no)")
    ap.add_argument("--only", choices=("all", "tables"), default="all",
                    help="'tables': only the offline table-build legs (no analysis, no JSON contract line)")
    ap.add_argument("--w-nodes", type=int, default=53, help="nodes of the stage-1 table-build leg")
    ap.add_argument("--w-pixels", type=int, default=4, help="sky pixels of the stage-1 table-build leg (0: none)")
    ap.add_argument("--table-build", type=int, default=1, help="run the table-build (stage 3) leg (0: no)")
    ap.add_argument("--io-nodes", type=int, default=8, help="node files of the store-loading leg (0: none)")
    ap.add_argument("--io-readers", type=int, default=6, help="reader threads of the store-loading leg")
    ap.add_argument("--io-dir", default=None, help="where the store-loading leg writes its files (default: TMPDIR)")
    ap.add_argument("--redshift-segments", type=int, default=8, help="segments of the pe_redshift leg (0: none)")
    ap.add_argument("--batch-segments", type=int, default=256, help="segments of the batched leg (0: none)")
    ap.add_argument("--batch-workers", type=int, default=3, help="native-server workers of the batched leg")
    ap.add_argument("--batch-check-segments", type=int, default=4, help="batched segments checked by the oracle")
    ap.add_argument("--batch-check-templates", type=int, default=32, help="templates of that oracle check")
    ap.add_argument("--serve-requests", type=int, default=24, help="requests of each serving leg (0: none)")
    ap.add_argument("--serve-workers", type=int, default=3, help="serving workers (child contexts)")
    ap.add_argument("--serve-config", action="store_true",
                    help="the serving workload at its stated shape through the native request loop (minutes)")
    ap.add_argument("--serve-capacity-requests", type=int, default=200, help="requests queued at once (capacity)")
    ap.add_argument("--serve-poisson-requests", type=int, default=1000, help="requests of the Poisson stream")
    ap.add_argument("--serve-load", type=float, default=0.8, help="Poisson rate as a fraction of the capacity")
    ap.add_argument("--serve-budget-gb", type=float, default=0.0,
                    help="workspace budget of the serving-config leg's workers, GB (0: 85%% of free memory)")
    ap.add_argument("--serve-config-workers", type=int, default=6, help="worker limit of the serving-config leg")
    ap.add_argument("--serve-max-s", type=float, default=600.0,
                    help="wall-clock limit of the serving-config leg's Poisson stream, s (then it drains)")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    if args.only == "tables":
        return run_tables(args)
    return run_b200(args)


def run_tables(args):
    """the offline table-build legs alone (one GPU, rank 0), one JSON line: for profiling those kernels"""
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    line = {"legs": "tables"}
    if args.table_build:
        line["table_build"] = table_build_leg(args, local)
    if args.w_pixels > 0:
        line["w_build"] = w_build_leg(args, local)
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
