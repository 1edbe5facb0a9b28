"""Benchmark: int2e_sph Gint/s on the seeded synthetic molecules, one JSON line on rank 0.

A step is one full pass of the hot path over the workload: every 8-fold-unique shell quartet
whose Schwarz bound reaches 1e-12 (cintx_plan_int2e_screened), evaluated into a device output
ring chunk by chunk (libcint-layout blocks).  The pair tables are resident in HBM before the
timed region; L2 is flushed (a 512 MiB write) between timed steps outside the step events.

  value      Gint/s = spherical integrals written per second, device time (CUDA events on the
             launching stream), max over ranks
  e2e        the same metric through the C ABI from host arrays: optimizer build (host -> device
             basis and pair tables), screened plan, execution and the device -> host copy of every
             chunk's output into pinned host memory, every step
  roofline   the kernel class with the largest device time in one profiled step: algorithmic FP64
             flops (the plan's flop model) / its event time, against the FP64 FMA peak measured by
             a probe kernel on the same GPU in the same run
  cpu_baseline  libcint 6.1.3 built from the reference sources (oracle/_ref), all host cores,
             on a seeded uniform sample of the same quartet set, extrapolated to the full set

--impl reference times that libcint CPU path alone (rank 0) on the same workload and metric.
Multi-GPU: chunks are distributed over ranks by their flop estimate (strong scaling: the
total work is the molecule's quartet set, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from cintx_b200 import molecules as M  # noqa: E402
from cintx_b200.sharding import assign_chunks, chunks_of, max_over_ranks  # noqa: E402

WORKLOADS = {
    "mol40_spd": (M.mol40, "40 seeded atoms in a 14-bohr cube, 60% light (2s,1p) / 40% heavy "
                           "(3s,2p,1d), exponents log-uniform [0.1,1.2e4]; Schwarz 1e-12"),
    "mol120_spdf": (M.mol120, "120 seeded atoms in a 22-bohr cube, heavy atoms add one f shell; "
                              "Schwarz 1e-12"),
    "water3": (M.water_like, "3-atom water-like molecule (O + 2 H), all quartets above 1e-12"),
}
# density-fitting workloads: the orbital molecule plus a per-atom auxiliary basis
# (6s 5p 4d 3f 2g single primitives, exponents log-uniform in [0.05, 5e3])
DF_WORKLOADS = {
    "mol120_df": (M.mol120, "mol120_spdf plus the per-atom auxiliary basis (9600 aux functions): int3c2e_sph over "
                            "orbital pairs x aux shells with Schwarz bound >= 1e-12, plus the int2c2e_sph metric "
                            "over aux shell pairs k >= l"),
    "mol40_df": (M.mol40, "mol40_spd plus the per-atom auxiliary basis (3200 aux functions): int3c2e_sph over "
                          "orbital pairs x aux shells with Schwarz bound >= 1e-12, plus int2c2e_sph over aux "
                          "pairs k >= l"),
}

SCHWARZ = 1e-12
# tuned form: quartets whose estimated FP32 error is below this use FP32 recurrences; off by default
# (5e-11 selects 0.5% of the mol40 quartets and measures 4.6% slower: the FP64 pipe is not the bound)
FP32_BUDGET = 0.0
PRIM_BUDGET = 5e-11  # tuned form: bound on the skipped primitive terms of one block
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "cint_cpu_bench")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="mol120_spdf",
                    choices=sorted(WORKLOADS) + sorted(DF_WORKLOADS) + ["mol20_g_learned"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--chunk-doubles", type=int, default=1 << 28)
    ap.add_argument("--branches", type=int, default=4)
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--form", default="tuned", choices=["tuned", "plain"])
    ap.add_argument("--no-error", action="store_true")
    ap.add_argument("--error-chunks", type=int, default=4)
    ap.add_argument("--fp32-budget", type=float, default=FP32_BUDGET)
    ap.add_argument("--no-autotune", action="store_true", help="tuned form without the launch-shape autotuner")
    ap.add_argument("--no-jk", action="store_true", help="skip the direct J/K build timing")
    ap.add_argument("--e2e-chunk-doubles", type=int, default=1 << 24,
                    help="chunk size of the end-to-end plan (copies of one chunk overlap the next chunk's kernels)")
    ap.add_argument("--prim-budget", type=float, default=PRIM_BUDGET)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    return ap.parse_args()


# ------------------------------------------------------------------ clocks
class Clocks:
    """SM clock and clock-event reasons sampled every 5 ms through NVML (read-only queries) while
    the timed region runs; the device is matched to the CUDA device by PCI bus id.  Without NVML
    the line reports no samples and the reason."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.stop_flag = None
        self.thread = None
        self.proc = None
        self.err = None

    def _handle(self, nv):
        import torch
        p = torch.cuda.get_device_properties(self.index)
        bus = "%08x:%02x:%02x.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
        try:
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._handle(nv)
            smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        except Exception as e:  # noqa: BLE001 - any NVML failure means "no samples", never a crash
            self.err = "nvml unavailable: %s" % e
            return
        self.stop_flag = threading.Event()

        def run():
            while not self.stop_flag.is_set():
                try:
                    self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), smax,
                                         nv.nvmlDeviceGetCurrentClocksEventReasons(h),
                                         nv.nvmlDeviceGetPowerUsage(h) / 1000.0))
                except Exception:  # noqa: BLE001
                    pass
                self.stop_flag.wait(0.005)

        self.nv = nv
        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()

    def stop(self):
        if self.thread is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "samples": 0, "reasons": [self.err or "no sampler"]}
        self.stop_flag.set()
        self.thread.join()
        reasons = set()
        for _, _, mask, _ in self.samples:
            for name, const in self.REASONS:
                if mask & getattr(self.nv, const):
                    reasons.add(name)
        sm = [x[0] for x in self.samples]
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_min_mhz": min(sm) if sm else None,
                "sm_max_mhz": max(x[1] for x in self.samples) if self.samples else None,
                "power_w_median": statistics.median([x[3] for x in self.samples]) if self.samples else None,
                "samples": len(sm), "sampler": "NVML every 5 ms", "reasons": sorted(reasons)}


# ------------------------------------------------------------------ CPU baseline (libcint)
def write_driver_input(path, mol, quartets):
    with open(path, "wb") as fh:
        np.array([mol.natm, mol.nbas, mol.env.size, len(quartets)], dtype=np.int32).tofile(fh)
        np.ascontiguousarray(mol.atm, dtype=np.int32).tofile(fh)
        np.ascontiguousarray(mol.bas, dtype=np.int32).tofile(fh)
        np.ascontiguousarray(mol.env, dtype=np.float64).tofile(fh)
        np.ascontiguousarray(quartets, dtype=np.int32).tofile(fh)


def run_libcint(mol, quartets, threads):
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "in.bin")
        write_driver_input(p, mol, quartets)
        r = subprocess.run([REF_DRIVER, p, str(threads)], capture_output=True, text=True, check=True)
    return json.loads(r.stdout)


def cpu_rate(mol, sampler, nq_total, nint_total, seconds, threads):
    """libcint time per quartet on a seeded uniform sample, extrapolated to the full set."""
    n = 2000
    res = run_libcint(mol, sampler(n, 1), threads)
    per_q = res["seconds"] / n
    n = int(min(5_000_000, max(n, seconds / max(per_q, 1e-9))))
    res = run_libcint(mol, sampler(n, 2), threads)
    per_q = res["seconds"] / n
    full_s = per_q * nq_total
    return {"value": nint_total / full_s / 1e9, "unit": "Gint/s", "cores": int(res["threads"]),
            "kind": "reference",
            "sample": "%d quartets drawn uniformly (seeded) from the %d-quartet set, %.1f s of libcint "
                      "int2e_sph with an optimizer, OpenMP dynamic; extrapolated by quartet count" %
                      (n, nq_total, res["seconds"]),
            "seconds": res["seconds"]}


# ------------------------------------------------------------------ reference arm
def schwarz_pairs_libcint(mol):
    """Q_ij = sqrt(max |(ij|ij)|) for all pairs i >= j, with libcint on the CPU."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import RefLibcint
    ref = RefLibcint()
    pairs = [(i, j) for i in range(mol.nbas) for j in range(i + 1)]

    def one(p):
        out, _ = ref.int2e((p[0], p[1], p[0], p[1]), mol)
        return np.sqrt(np.abs(out).max())

    with ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        q = np.array(list(ex.map(one, pairs, chunksize=256)))
    return np.array(pairs, dtype=np.int32), q


class UniqueQuartets:
    """The plan's quartet set (unordered pairs of shell pairs with Q_p Q_q >= cutoff), built on
    the host from libcint Schwarz factors, with uniform sampling."""

    def __init__(self, mol, cutoff):
        self.mol = mol
        pairs, q = schwarz_pairs_libcint(mol)
        order = np.argsort(-q, kind="stable")
        self.pairs, self.q = pairs[order], q[order]
        keep = self.q * self.q.max() >= cutoff
        self.pairs, self.q = self.pairs[keep], self.q[keep]
        thr = cutoff / np.maximum(self.q, 1e-300)
        # number of partners j <= i (sorted decreasing) with q_j >= cutoff / q_i
        L = np.searchsorted(-self.q, -thr, side="right")
        self.count = np.minimum(np.arange(len(self.q)) + 1, L)
        l = mol.bas[:, 1]
        ns = (2 * l[self.pairs[:, 0]] + 1) * (2 * l[self.pairs[:, 1]] + 1)
        cum = np.concatenate([[0], np.cumsum(ns)])
        self.nquartets = int(self.count.sum())
        self.nintegrals = int((ns * cum[self.count]).sum())
        self.prob = self.count / self.count.sum()

    def sample(self, n, seed):
        rng = np.random.default_rng(seed)
        i = rng.choice(len(self.q), size=n, p=self.prob)
        j = (rng.random(n) * self.count[i]).astype(np.int64)
        return np.concatenate([self.pairs[i], self.pairs[j]], axis=1).astype(np.int32)


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    fn, desc = WORKLOADS[args.workload]
    if not os.path.exists(REF_DRIVER):
        print(json.dumps({"impl": "reference", "unavailable": "libcint was not built from the reference "
                          "sources (oracle/_ref missing)"}))
        return
    mol = fn()
    uq = UniqueQuartets(mol, SCHWARZ)
    threads = os.cpu_count() or 1
    # per-step sample sized for ~target seconds
    cal = run_libcint(mol, uq.sample(2000, 100), threads)
    per_q = cal["seconds"] / 2000
    nsamp = int(min(2_000_000, max(2000, 8.0 / max(per_q, 1e-9))))
    times = []
    for s in range(args.warmup + args.steps):
        res = run_libcint(mol, uq.sample(nsamp, 1000 + s), threads)
        if s >= args.warmup:
            times.append(res["seconds"] / nsamp * uq.nquartets)  # extrapolated full-step time
    t = statistics.mean(times)
    value = uq.nintegrals / t / 1e9
    line = {"metric": "int2e_sph Gint/s at <=1e-10 abs err (libcint CPU reference)", "value": value,
            "unit": "Gint/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": args.workload, "description": desc, "nquartets": uq.nquartets,
                       "nintegrals": uq.nintegrals, "schwarz_cutoff": SCHWARZ},
            "cpu_baseline": {"value": value, "unit": "Gint/s", "cores": threads, "kind": "reference",
                             "sample": "%d seeded uniform quartets per step, extrapolated by quartet count" % nsamp},
            "e2e": {"value": value, "unit": "Gint/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def df_problem(name):
    fn, desc = DF_WORKLOADS[name]
    base = fn()
    mol = M.with_aux(base)
    norb = base.nbas
    naux = mol.nbas - norb
    kk, ll = np.tril_indices(naux)
    aux_pairs = np.stack([norb + kk, norb + ll], axis=1).astype(np.int32)
    return mol, norb, aux_pairs, desc


class DFTriples:
    """The density-fitting sweep's tuple set ((ab|k), a >= b orbital, k auxiliary, Schwarz bound
    >= cutoff) built on the host from libcint Schwarz factors, with uniform sampling."""

    def __init__(self, mol, norb, cutoff):
        from concurrent.futures import ThreadPoolExecutor
        from oracle import RefLibcint
        ref = RefLibcint()
        pairs = [(i, j) for i in range(norb) for j in range(i + 1)]
        aux = list(range(norb, mol.nbas))
        with ThreadPoolExecutor(os.cpu_count() or 1) as ex:
            q = np.array(list(ex.map(lambda p: np.sqrt(np.abs(ref.int2e((p[0], p[1], p[0], p[1]), mol)[0]).max()),
                                     pairs, chunksize=256)))
            qk = np.array(list(ex.map(lambda k: np.sqrt(np.abs(ref.int2c2e((k, k), mol)[0]).max()), aux)))
        order = np.argsort(-qk, kind="stable")
        self.aux, self.qk = np.array(aux)[order], qk[order]
        self.pairs = np.array(pairs, dtype=np.int32)
        self.count = np.searchsorted(-self.qk, -(cutoff / np.maximum(q, 1e-300)), side="right")
        l = mol.bas[:, 1]
        ns = (2 * l[self.pairs[:, 0]] + 1) * (2 * l[self.pairs[:, 1]] + 1)
        cum = np.concatenate([[0], np.cumsum(2 * l[self.aux] + 1)])
        self.nquartets = int(self.count.sum())
        self.nintegrals = int((ns * cum[self.count]).sum())
        self.prob = self.count / self.count.sum()

    def sample(self, n, seed):
        rng = np.random.default_rng(seed)
        i = rng.choice(len(self.pairs), size=n, p=self.prob)
        k = self.aux[(rng.random(n) * self.count[i]).astype(np.int64)]
        return np.stack([self.pairs[i, 0], self.pairs[i, 1], k, np.full(n, -1)], axis=1).astype(np.int32)


def df_reference_arm(args):
    """libcint int3c2e_sph + int2c2e_sph on the host cores over the DF sweep's tuple set."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if not os.path.exists(REF_DRIVER):
        print(json.dumps({"impl": "reference", "unavailable": "libcint was not built from the reference "
                          "sources (oracle/_ref missing)"}))
        return
    mol, norb, aux_pairs, desc = df_problem(args.workload)
    tri = DFTriples(mol, norb, SCHWARZ)
    threads = os.cpu_count() or 1
    l = mol.bas[:, 1]
    n2int = int(((2 * l[aux_pairs[:, 0]] + 1) * (2 * l[aux_pairs[:, 1]] + 1)).sum())
    two = np.stack([aux_pairs[:, 0], np.full(len(aux_pairs), -1), aux_pairs[:, 1], np.full(len(aux_pairs), -1)],
                   axis=1).astype(np.int32)
    cal = run_libcint(mol, tri.sample(2000, 100), threads)
    per_q = cal["seconds"] / 2000
    nsamp = int(min(2_000_000, max(2000, 8.0 / max(per_q, 1e-9))))
    rng = np.random.default_rng(7)
    times = []
    for s_ in range(args.warmup + args.steps):
        r3 = run_libcint(mol, tri.sample(nsamp, 1000 + s_), threads)
        r2 = run_libcint(mol, two[rng.choice(len(two), size=min(len(two), 20000), replace=False)], threads)
        if s_ >= args.warmup:
            times.append(r3["seconds"] / nsamp * tri.nquartets + r2["seconds"] / min(len(two), 20000) * len(two))
    t = statistics.mean(times)
    value = (tri.nintegrals + n2int) / t / 1e9
    line = {"metric": "int3c2e_sph + int2c2e_sph Gint/s, density fitting (libcint CPU reference)", "value": value,
            "unit": "Gint/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": args.workload, "description": desc, "ntriples": tri.nquartets,
                       "nintegrals": tri.nintegrals + n2int, "schwarz_cutoff": SCHWARZ},
            "cpu_baseline": {"value": value, "unit": "Gint/s", "cores": threads, "kind": "reference",
                             "sample": "%d seeded uniform (ab|k) triples and 20000 (k|l) pairs per step, "
                                       "extrapolated by count" % nsamp},
            "e2e": {"value": value, "unit": "Gint/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ------------------------------------------------------------------ our arm
def fp64_peak(cx, torch):
    """FP64 FMA pipe throughput of this GPU (TFLOP/s), best of 3."""
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    blocks, threads, iters = sms * 8, 256, 2000
    out = torch.empty(blocks * threads, dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream()
    best = 0.0
    for _ in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        rc = cx.lib.cintx_fp64_fma_probe(blocks, threads, iters, out.data_ptr(), st.cuda_stream)
        e1.record()
        e1.synchronize()
        assert rc == 0
        flops = blocks * threads * iters * 16 * 8 * 2.0
        best = max(best, flops / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    return best


def timed_sweep(cx, torch, plan, mine, args, stream, local, world, tune=False):
    """Warm-up, then exactly args.steps timed passes of `plan` over the rank's chunks (one CUDA
    graph per pass unless --no-graph), L2 flushed between passes outside the events.  With
    tune, the plan's launch shapes are autotuned first (each class on its largest segment)."""
    return timed_multi(cx, torch, [(plan, mine)], args, stream, local, world, tune)


def timed_multi(cx, torch, items, args, stream, local, world, tune=False):
    """As timed_sweep for several plans run back to back in one step: items = [(plan, chunks)]."""
    import torch.distributed as dist
    rings = [torch.empty(max(p.stats.max_chunk_doubles, 1), dtype=torch.float64, device="cuda") for p, _ in items]
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    tuning = None
    if tune:
        t0 = time.perf_counter()
        lanes = {}
        for (plan, mine), ring in zip(items, rings):
            if not mine:
                continue
            plan.autotune(ring.data_ptr(), chunk=-1, stream=stream.cuda_stream, reps=2)
            for c in mine:
                for cl, n in zip(plan.segments(c)[0], plan.segment_lanes(c)):
                    lanes["(%d%d|%d%d)" % tuple(cl)] = int(n)
        tuning = {"seconds": time.perf_counter() - t0, "lanes_per_quartet": dict(sorted(lanes.items()))}
    use_graph = not args.no_graph
    if use_graph:
        try:
            for (plan, mine), ring in zip(items, rings):
                if mine:
                    plan.graph_build(ring.data_ptr(), chunks=mine, nbranch=args.branches)
        except cx.CintxError:
            use_graph = False

    def step():
        for (plan, mine), ring in zip(items, rings):
            if not mine:
                continue
            if use_graph:
                plan.graph_launch(stream.cuda_stream)
            else:
                for c in mine:
                    plan.execute(ring.data_ptr(), chunk=c, stream=stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = cx.launch_count()
    t_wall = time.perf_counter()
    step_ms = []
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t_wall = time.perf_counter() - t_wall
    launches = cx.launch_count() - launches0
    clk = clocks.stop()
    ms = max_over_ranks(sum(step_ms), device="cuda") / args.steps
    return {"ms": ms, "launches": launches, "clocks": clk, "wall": t_wall, "graph": use_graph, "ring": rings[0],
            "rings": rings, "tuning": tuning}


def class_profile(torch, plan, mine, ring, stream):
    """One pass with every class segment timed on its own."""
    per_class = {}
    for c in mine:
        cls, nq, fl = plan.segments(c)
        for s in range(len(nq)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plan.execute_segment(ring.data_ptr(), c, s, stream=stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            key = "(%d%d|%d%d)" % tuple(cls[s])
            d = per_class.setdefault(key, {"ms": 0.0, "flops": 0.0, "quartets": 0, "launches": 0, "ints": 0})
            d["ms"] += e0.elapsed_time(e1)
            d["flops"] += float(fl[s])
            d["quartets"] += int(nq[s])
            d["launches"] += 1
            d["ints"] += int(nq[s]) * int(np.prod([2 * l + 1 for l in cls[s]]))
    return per_class


def jk_timing(cx, torch, plan, mol, stream, reps):
    """Direct Coulomb + exchange build over the sweep (cintx_plan_jk): device time per build (CUDA
    events, after one warm-up) and end to end with the density copied in and J, K copied out."""
    nao = int(mol.ao_loc()[-1])
    rng = np.random.default_rng(11)
    dh = rng.normal(size=(nao, nao))
    dh = torch.tensor(dh + dh.T).pin_memory()
    d = torch.empty((nao, nao), dtype=torch.float64, device="cuda")
    vj = torch.empty_like(d)
    vk = torch.empty_like(d)
    hj = torch.empty((nao, nao), dtype=torch.float64).pin_memory()
    hk = torch.empty_like(hj).pin_memory()
    d.copy_(dh, non_blocking=True)
    plan.jk(d.data_ptr(), nao, vj.data_ptr(), vk.data_ptr(), stream=stream.cuda_stream)  # warm-up
    stream.synchronize()
    ms, e2e = [], []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        d.copy_(dh, non_blocking=True)
        e0.record(stream)
        plan.jk(d.data_ptr(), nao, vj.data_ptr(), vk.data_ptr(), stream=stream.cuda_stream)
        e1.record(stream)
        hj.copy_(vj, non_blocking=True)
        hk.copy_(vk, non_blocking=True)
        stream.synchronize()
        e2e.append(time.perf_counter() - t0)
        ms.append(e0.elapsed_time(e1))
    st = plan.stats
    t = statistics.mean(ms)
    return {"ms_per_build": t, "nao": nao, "integrals_contracted_per_s": st.nintegrals / (t * 1e-3),
            "e2e_ms_per_build": statistics.mean(e2e) * 1e3,
            "e2e_bytes": {"h2d": nao * nao * 8, "d2h": 2 * nao * nao * 8},
            "what": "J = (pq|rs) D_rs and K = (pq|rs) D_qs over the same quartet set, each chunk contracted "
                    "on the device right after its kernels (8-fold symmetry); integrals never leave the GPU"}


def tuned_error(cx, torch, opt, plan, ring, stream, max_chunks):
    """Max and RMS absolute difference between the mixed plan and an FP64 evaluation of the same
    quartets (explicit FP64 plan over each checked chunk's quartet list)."""
    st = plan.stats
    chunks = list(range(st.nchunks))
    if len(chunks) > max_chunks:
        chunks = sorted(set(np.linspace(0, st.nchunks - 1, max_chunks).astype(int).tolist()))
    mx, ss, n = 0.0, 0.0, 0
    for c in chunks:
        plan.execute(ring.data_ptr(), chunk=c, stream=stream.cuda_stream)
        stream.synchronize()
        got = ring[:plan.chunk_size(c)]
        ref_plan = cx.Plan.shells(opt, cx.INT2E, plan.chunk_quartets(c), sph=True)
        ref = torch.empty(ref_plan.stats.nintegrals, dtype=torch.float64, device="cuda")
        ref_plan.execute(ref.data_ptr(), stream=stream.cuda_stream)
        stream.synchronize()
        d = (got - ref).abs()
        mx = max(mx, float(d.max()))
        ss += float((d * d).sum())
        n += d.numel()
        ref_plan.close()
    return {"max_abs": mx, "rms_abs": (ss / max(n, 1)) ** 0.5, "integrals_checked": n,
            "chunks_checked": len(chunks), "reference": "the same quartets evaluated by the FP64 kernels"}


def our_arm(args):
    import torch
    import torch.distributed as dist

    import cintx_b200 as cx

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    fn, desc = WORKLOADS[args.workload]
    mol = fn()
    opt = cx.Optimizer(mol.atm, mol.bas, mol.env)
    tuned = args.form == "tuned"

    def make_plan(o, tuned_form):
        if tuned_form:
            return cx.Plan.screened_mixed(o, SCHWARZ, fp32_budget=args.fp32_budget, prim_budget=args.prim_budget,
                                          max_chunk_doubles=args.chunk_doubles)
        return cx.Plan.screened(o, SCHWARZ, sph=True, max_chunk_doubles=args.chunk_doubles)

    plan = make_plan(opt, tuned)
    st = plan.stats
    nchunks = st.nchunks
    chunk_flops = [float(plan.segments(c)[2].sum()) for c in range(nchunks)]
    mine = chunks_of(assign_chunks(chunk_flops, world), rank)
    my_ints = sum(plan.chunk_size(c) for c in mine)
    stream = torch.cuda.Stream()  # a real stream handle: events and kernels share it
    torch.cuda.set_stream(stream)

    main_run = timed_sweep(cx, torch, plan, mine, args, stream, local, world, tune=tuned and not args.no_autotune)
    ms_per_step = main_run["ms"]
    value = st.nintegrals / (ms_per_step * 1e-3) / 1e9
    plain = None
    if tuned:
        pplan = make_plan(opt, False)
        pst = pplan.stats
        pmine = chunks_of(assign_chunks([float(pplan.segments(c)[2].sum()) for c in range(pst.nchunks)], world), rank)
        prun = timed_sweep(cx, torch, pplan, pmine, args, stream, local, world)
        plain = {"value": pst.nintegrals / (prun["ms"] * 1e-3) / 1e9, "ms_per_step": prun["ms"]}
        pplan.close()
        del prun

    per_class = class_profile(torch, plan, mine, main_run["ring"], stream)
    peak64 = fp64_peak(cx, torch)
    top = max(per_class.items(), key=lambda kv: kv[1]["ms"]) if per_class else (None, None)
    roof = None
    if top[0] is not None:
        d = top[1]
        achieved = d["flops"] / (d["ms"] * 1e-3) / 1e12
        prof_total = sum(v["ms"] for v in per_class.values())
        roof = {"bound": "fp64", "kernel": "eri4c_kernel" + top[0], "achieved": achieved, "peak": peak64,
                "unit": "TFLOP/s", "frac": achieved / peak64,
                "peak_source": "FP64 FMA probe kernel on this GPU, this run (MEASURED_PEAKS.json has no FP64 figure)",
                "share_of_step": d["ms"] / prof_total, "traffic": None,
                "whole_step_fp64_frac": (st.flops / (ms_per_step * 1e-3) / 1e12) / peak64}
    err = None
    if tuned and rank == 0 and not args.no_error:
        err = tuned_error(cx, torch, opt, plan, main_run["ring"], stream, args.error_chunks)
    jk = None
    if rank == 0 and world == 1 and not args.no_jk:
        jk = jk_timing(cx, torch, plan, mol, stream, min(args.steps, 5))
    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    hbm = None
    try:
        hbm = json.load(open(PEAKS_FILE))["hbm_gbs"]
    except Exception:
        pass
    form = ("tuned: primitive Schwarz screening (budget %g per integral), FP32 recurrences where the estimated "
            "FP32 error is below %g, %s, graph-batched" % (args.prim_budget, args.fp32_budget,
                                                         "launch shapes autotuned per class" if not args.no_autotune
                                                         else "default launch shapes")) if tuned else \
        "plain FP64 (default launch shapes, libcint screening only)"
    line = {"metric": "int2e_sph Gint/s at <=1e-10 abs err (%s form)" % ("tuned" if tuned else "plain FP64"),
            "value": value, "unit": "Gint/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded molecule; no dataset)",
            "config": {"workload": args.workload, "description": desc, "form": form,
                       "nquartets": st.nquartets, "nquartets_fp32": st.nquartets_fp32,
                       "nintegrals": st.nintegrals, "nchunks": nchunks,
                       "chunk_doubles": args.chunk_doubles, "schwarz_cutoff": SCHWARZ,
                       "nprim_quartets": st.nprim_quartets, "model_flops_per_step": st.flops,
                       "l2": "flushed between steps (512 MiB write outside the step events); each step also "
                             "streams %.1f GB of output through HBM" % (st.nintegrals * 8 / 1e9)},
            "quartets_per_s": st.nquartets / (ms_per_step * 1e-3),
            "gpu_launches": main_run["launches"],
            "clocks": main_run["clocks"], "wall_s_timed_region": main_run["wall"],
            "roofline": roof,
            "output_write_gbs": st.nintegrals * 8 / (ms_per_step * 1e-3) / 1e9,
            "hbm_gbs_measured_peak": hbm,
            "execution": "one CUDA graph per step (%d kernel classes on %d branches)" % (len(per_class), args.branches)
                         if main_run["graph"] else "direct launches",
            "per_class": {k: {"ms": round(v["ms"], 4), "tflops": round(v["flops"] / (v["ms"] * 1e-3) / 1e12, 3),
                              "gint_s": round(v["ints"] / (v["ms"] * 1e-3) / 1e9, 2), "quartets": v["quartets"]}
                          for k, v in sorted(per_class.items(), key=lambda kv: -kv[1]["ms"])[:16]},
            "profiled_step_ms": sum(v["ms"] for v in per_class.values())}
    if main_run["tuning"] is not None:
        line["autotune"] = main_run["tuning"]
    if plain is not None:
        line["plain_fp64"] = plain
        line["tuned_over_plain"] = value / plain["value"]
    if err is not None:
        line["error_vs_fp64"] = err
    if jk is not None:
        line["jk_build"] = jk

    # end-to-end through the C ABI from host arrays (rank 0 measures its own shard when N > 1):
    # optimizer from atm/bas/env, screened plan, evaluation and D2H into page-locked host memory
    if not args.no_e2e:
        e2e_chunk = args.e2e_chunk_doubles

        def e2e_plan(o):
            if tuned:
                return cx.Plan.screened_mixed(o, SCHWARZ, fp32_budget=args.fp32_budget, prim_budget=args.prim_budget,
                                              max_chunk_doubles=e2e_chunk)
            return cx.Plan.screened(o, SCHWARZ, sph=True, max_chunk_doubles=e2e_chunk)

        host = None
        phases = {"optimizer": [], "plan": [], "execute_d2h": []}
        h2d = d2h = 0
        for s in range(1 + max(1, min(args.steps, 3))):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            o2 = cx.Optimizer(mol.atm, mol.bas, mol.env)
            t1 = time.perf_counter()
            p2 = e2e_plan(o2)
            if tuned and not args.no_autotune:
                p2.use_tuned_shapes()  # shapes autotuned once in this process (before the timed sweep)
            t2 = time.perf_counter()
            if host is None or host.size < 2 * p2.stats.max_chunk_doubles:  # two-slot page-locked host ring
                # allocated in the untimed first iteration; later iterations reuse it
                host = torch.empty(2 * max(p2.stats.max_chunk_doubles, 1), dtype=torch.float64,
                                   pin_memory=True).numpy()
            if world == 1:
                p2.execute_host_ring(host)
            else:
                e2e_mine = chunks_of(assign_chunks([float(p2.segments(c)[2].sum()) for c in range(p2.stats.nchunks)],
                                                   world), rank)
                off = 0
                for c in e2e_mine:
                    p2.execute_host(host, chunk=c)
                    off += p2.chunk_size(c)
            t3 = time.perf_counter()
            if s > 0:
                phases["optimizer"].append(t1 - t0)
                phases["plan"].append(t2 - t1)
                phases["execute_d2h"].append(t3 - t2)
            h2d = mol.atm.nbytes + mol.bas.nbytes + mol.env.nbytes + o2.device_bytes + p2.stats.device_bytes
            d2h = (st.nintegrals if world == 1 else off) * 8
            p2.close()
            o2.close()
        te = sum(statistics.mean(v) for v in phases.values())
        line["e2e"] = {"value": st.nintegrals / te / 1e9 if world == 1 else d2h / 8 / te / 1e9 * world,
                       "unit": "Gint/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                       "seconds_per_step": te,
                       "phases_s": {k: statistics.mean(v) for k, v in phases.items()},
                       "chunk_doubles": e2e_chunk,
                       "includes": "int2e_optimizer from host atm/bas/env (pair tables, Schwarz passes) + screened "
                                   "plan + evaluation + D2H of every integral through a two-chunk page-locked "
                                   "host ring (copies overlapped with the next chunk's kernels)"}
    if world == 1 and not args.no_cpu and os.path.exists(REF_DRIVER):
        line["cpu_baseline"] = cpu_rate(mol, lambda n, seed: plan.sample_quartets(n, seed), st.nquartets,
                                        st.nintegrals, args.cpu_seconds, os.cpu_count() or 1)
    elif world == 1 and not args.no_cpu:
        line["cpu_baseline"] = None
    print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    plan.close()
    opt.close()


def df_arm(args):
    """Density-fitting sweep on the GPU: int3c2e_sph (screened (ab|k) plan, chunks sharded over
    ranks by flops) plus the int2c2e_sph metric (rank 0), one CUDA graph each per step."""
    import torch
    import torch.distributed as dist

    import cintx_b200 as cx

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    mol, norb, aux_pairs, desc = df_problem(args.workload)
    tuned = args.form == "tuned"
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)

    def make(o):
        p3 = cx.Plan.screened_3c(o, norb, SCHWARZ, max_chunk_doubles=args.chunk_doubles)
        p2 = cx.Plan.shells(o, cx.INT2C2E, aux_pairs)
        return p3, p2

    opt = cx.Optimizer(mol.atm, mol.bas, mol.env, pair_shells=norb)
    p3, p2 = make(opt)
    s3, s2 = p3.stats, p2.stats
    mine3 = chunks_of(assign_chunks([float(p3.segments(c)[2].sum()) for c in range(s3.nchunks)], world), rank)
    mine2 = [0] if rank == 0 else []
    run = timed_multi(cx, torch, [(p3, mine3), (p2, mine2)], args, stream, local, world,
                      tune=tuned and not args.no_autotune)
    nint = s3.nintegrals + s2.nintegrals
    value = nint / (run["ms"] * 1e-3) / 1e9
    plain = err = None
    if tuned:
        q3, q2 = make(opt)  # default launch shapes
        prun = timed_multi(cx, torch, [(q3, mine3), (q2, mine2)], args, stream, local, world, tune=False)
        plain = {"value": nint / (prun["ms"] * 1e-3) / 1e9, "ms_per_step": prun["ms"]}
        if rank == 0 and mine3:
            c = mine3[0]
            a, b = run["rings"][0], prun["rings"][0]
            p3.execute(a.data_ptr(), chunk=c, stream=stream.cuda_stream)
            q3.execute(b.data_ptr(), chunk=c, stream=stream.cuda_stream)
            stream.synchronize()
            n = p3.chunk_size(c)
            err = {"max_abs": float((a[:n] - b[:n]).abs().max()), "integrals_checked": n,
                   "reference": "the same chunk with the default launch shapes"}
        q3.close()
        q2.close()
    per_class = class_profile(torch, p3, mine3, run["rings"][0], stream)
    peak64 = fp64_peak(cx, torch)
    roof = None
    if per_class:
        top = max(per_class.items(), key=lambda kv: kv[1]["ms"])
        d = top[1]
        achieved = d["flops"] / (d["ms"] * 1e-3) / 1e12
        roof = {"bound": "fp64", "kernel": "eri4c_kernel" + top[0], "achieved": achieved, "peak": peak64,
                "unit": "TFLOP/s", "frac": achieved / peak64,
                "peak_source": "FP64 FMA probe kernel on this GPU, this run (MEASURED_PEAKS.json has no FP64 figure)",
                "share_of_step": d["ms"] / sum(v["ms"] for v in per_class.values()), "traffic": None}
    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    line = {"metric": "int3c2e_sph + int2c2e_sph Gint/s, density fitting (%s form)" % ("tuned" if tuned else "plain"),
            "value": value, "unit": "Gint/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": run["ms"], "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded molecule and auxiliary basis; no dataset)",
            "config": {"workload": args.workload, "description": desc, "ntriples": s3.nquartets,
                       "nintegrals_3c": s3.nintegrals, "nintegrals_2c": s2.nintegrals, "nchunks": s3.nchunks,
                       "norb_shells": norb, "naux_shells": mol.nbas - norb, "schwarz_cutoff": SCHWARZ,
                       "model_flops_per_step": s3.flops + s2.flops,
                       "form": "autotuned launch shapes, graph-batched" if tuned and not args.no_autotune
                               else "default launch shapes, graph-batched",
                       "l2": "flushed between steps (512 MiB write outside the step events)"},
            "quartets_per_s": (s3.nquartets + s2.nquartets) / (run["ms"] * 1e-3),
            "gpu_launches": run["launches"], "clocks": run["clocks"], "roofline": roof,
            "per_class": {k: {"ms": round(v["ms"], 4), "tflops": round(v["flops"] / (v["ms"] * 1e-3) / 1e12, 3),
                              "quartets": v["quartets"]}
                          for k, v in sorted(per_class.items(), key=lambda kv: -kv[1]["ms"])[:12]}}
    if run["tuning"] is not None:
        line["autotune"] = run["tuning"]
    if plain is not None:
        line["plain_fp64"] = plain
        line["tuned_over_plain"] = value / plain["value"]
    if err is not None:
        line["error_vs_default_shapes"] = err
    if not args.no_e2e:
        # end to end from host arrays: optimizer, both plans, evaluation and D2H of every chunk into
        # a page-locked host buffer (one chunk at a time: the 3-centre output exceeds host memory)
        host = torch.empty(max(s3.max_chunk_doubles, s2.nintegrals, 1), dtype=torch.float64, pin_memory=True).numpy()
        times = []
        for s_ in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            o2 = cx.Optimizer(mol.atm, mol.bas, mol.env, pair_shells=norb)
            e3, e2 = make(o2)
            if tuned and not args.no_autotune:
                e3.use_tuned_shapes()
                e2.use_tuned_shapes()
            for c in range(e3.stats.nchunks):
                e3.execute_host(host, chunk=c)
            e2.execute_host(host)
            times.append(time.perf_counter() - t0)
            h2d = mol.atm.nbytes + mol.bas.nbytes + mol.env.nbytes + o2.device_bytes + e3.stats.device_bytes
            e3.close()
            e2.close()
            o2.close()
        te = times[-1]
        line["e2e"] = {"value": nint / te / 1e9, "unit": "Gint/s", "h2d_bytes_per_step": int(h2d),
                       "d2h_bytes_per_step": int(nint * 8), "seconds_per_step": te,
                       "includes": "optimizer from host atm/bas/env, both plans (Schwarz passes), evaluation and "
                                   "D2H of every integral, chunk by chunk"}
    if world == 1 and not args.no_cpu and os.path.exists(REF_DRIVER):
        n3 = min(200000, s3.nquartets)
        r3 = run_libcint(mol, p3.sample_quartets(n3, 1), os.cpu_count() or 1)
        n2 = min(20000, s2.nquartets)
        r2 = run_libcint(mol, p2.sample_quartets(n2, 2), os.cpu_count() or 1)
        t_full = r3["seconds"] / n3 * s3.nquartets + r2["seconds"] / n2 * s2.nquartets
        line["cpu_baseline"] = {"value": nint / t_full / 1e9, "unit": "Gint/s", "cores": int(r3["threads"]),
                                "kind": "reference",
                                "sample": "%d (ab|k) triples and %d (k|l) pairs drawn uniformly from the plans, "
                                          "libcint int3c2e_sph/int2c2e_sph with optimizers, OpenMP dynamic; "
                                          "extrapolated by count" % (n3, n2)}
    print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    p3.close()
    p2.close()
    opt.close()


def g_quartets(mol, n, seed):
    """Seeded shell quartets containing a g shell whose class needs 5..9 Rys roots."""
    rng = np.random.default_rng(seed)
    ls = mol.bas[:, 1]
    g = np.where(ls == 4)[0]
    q = rng.integers(0, mol.nbas, size=(4 * n, 4))
    q[np.arange(len(q)), rng.integers(0, 4, len(q))] = rng.choice(g, len(q))
    q = q[ls[q].sum(axis=1) >= 8][:n]
    return np.ascontiguousarray(q, dtype=np.int32)


def learned_arm(args):
    """the learned Rys-root initializer, trained on the device, its roots on 5e6
    (x, n) points of the configs' distribution, and g-shell int2e quartets evaluated with learned
    roots against the same kernels with table roots."""
    import torch

    import cintx_b200 as cx

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if int(os.environ.get("RANK", "0")) != 0:
        return
    mol = M.mol20_g()
    net = cx.RysNet(seed=0)
    t0 = time.perf_counter()
    hist = net.train(nsamples=5_000_000, n_lo=5, n_hi=9, epochs=40, batch=16384, lr=3e-3, seed=1)
    train_s = time.perf_counter() - t0
    # roots: 5e6 points, n uniform in 5..9, x 70% log-uniform [1e-7, 50], 30% uniform [50, 3000]
    rng = np.random.default_rng(3)
    npts = 5_000_000
    nn = rng.integers(5, 10, npts)
    x = np.where(rng.random(npts) < 0.7, np.exp(rng.uniform(np.log(1e-7), np.log(50.0), npts)),
                 rng.uniform(50.0, 3000.0, npts))
    worst, nfb, nref, ncl, iters = 0.0, 0, 0, 0, []
    t_roots = 0.0
    for n in range(5, 10):
        sel = x[nn == n]
        t1 = time.perf_counter()
        t2, w, st, it = net.roots(n, sel)
        t_roots += time.perf_counter() - t1
        tt2, tw = cx.rys_t2_batch(n, sel)
        ok = st == 0
        if ok.any():
            worst = max(worst, float(np.abs(t2[ok] / tt2[ok] - 1).max()), float(np.abs(w[ok] / tw[ok] - 1).max()))
        nfb += int((st == 1).sum())
        nref += int(ok.sum())
        ncl += int((st == 2).sum())
        iters.append(it[ok])
    # integrals: quartets of the Schwarz-screened set (bound >= 1e-12) with a g shell and 5..9 roots
    opt = cx.Optimizer(mol.atm, mol.bas, mol.env)
    scr = cx.Plan.screened(opt, SCHWARZ, sph=True)
    cand = scr.sample_quartets(2_000_000, 4)
    scr.close()
    ls = mol.bas[:, 1]
    cand = cand[(ls[cand] == 4).any(axis=1) & (ls[cand].sum(axis=1) >= 8)]
    quartets = np.ascontiguousarray(np.unique(cand, axis=0)[:100_000], dtype=np.int32)
    p_tab = cx.Plan.shells(opt, cx.INT2E, quartets)
    p_lrn = cx.Plan.shells(opt, cx.INT2E, quartets)
    fb, npq = p_lrn.use_learned_roots(net)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    run_l = timed_multi(cx, torch, [(p_lrn, [0])], args, stream, 0, 1, tune=False)
    run_t = timed_multi(cx, torch, [(p_tab, [0])], args, stream, 0, 1, tune=False)
    nint = p_lrn.stats.nintegrals
    a, b = run_l["rings"][0], run_t["rings"][0]
    p_lrn.execute(a.data_ptr(), stream=stream.cuda_stream)
    p_tab.execute(b.data_ptr(), stream=stream.cuda_stream)
    stream.synchronize()
    d = (a[:nint] - b[:nint]).abs()
    diff = float(d.max())
    big = b[:nint].abs() > 1e-6
    rel = float((d[big] / b[:nint][big].abs()).max()) if bool(big.any()) else 0.0
    parity = bool(((d <= 1e-12) | (d <= 1e-10 * b[:nint].abs())).all())
    line = {"metric": "int2e_sph Gint/s on g-shell quartets with learned Rys roots (5..9 roots)",
            "value": nint / (run_l["ms"] * 1e-3) / 1e9, "unit": "Gint/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": run_l["ms"], "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded molecule and root test set)",
            "config": {"workload": args.workload, "nquartets": int(len(quartets)), "nintegrals": int(nint),
                       "description": "mol20_g: up to 100000 distinct quartets of the Schwarz-screened set (1e-12) with "
                                      "a g shell and 5..9 roots; "
                                      "root test set 5e6 (x, n) points, n 5..9, x 70% log-uniform [1e-7, 50] "
                                      "and 30% uniform [50, 3000]"},
            "gpu_launches": run_l["launches"], "clocks": run_l["clocks"],
            "table_roots": {"value": nint / (run_t["ms"] * 1e-3) / 1e9, "ms_per_step": run_t["ms"]},
            "learned_roots": {"train_seconds": train_s, "train_samples": 5_000_000, "epochs": 40,
                              "loss_first_last": [float(hist[0]), float(hist[-1])],
                              "root_points": npts, "refined": nref, "fallback": nfb, "closed_form": ncl,
                              "fallback_rate_in_table_range": nfb / max(nref + nfb, 1),
                              "max_rel_err_vs_table": worst,
                              "newton_steps_mean": float(np.concatenate(iters).mean()),
                              "roots_per_s": npts / t_roots,
                              "integral_primitive_quartets": int(npq), "integral_fallback": int(fb),
                              "integral_max_abs_vs_table_roots": diff,
                              "integral_max_rel_vs_table_roots": rel,
                              "integral_parity_rule_vs_table_roots": parity}}
    if os.path.exists(REF_DRIVER) and not args.no_cpu:
        nq = min(20000, len(quartets))
        r = run_libcint(mol, quartets[:nq], os.cpu_count() or 1)
        line["cpu_baseline"] = {"value": r["nintegrals"] / r["seconds"] / 1e9, "unit": "Gint/s",
                                "cores": int(r["threads"]), "kind": "reference",
                                "sample": "the first %d of the quartets, libcint int2e_sph, OpenMP dynamic" % nq}
    print(json.dumps(line))
    p_tab.close()
    p_lrn.close()
    opt.close()


def main():
    args = parse()
    df = args.workload in DF_WORKLOADS
    if args.workload == "mol20_g_learned":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the learned-root workload has no reference "
                              "counterpart (libcint computes roots by its own fits); its cpu_baseline times libcint "
                              "on the same quartets"}))
        else:
            learned_arm(args)
    elif args.impl == "reference":
        (df_reference_arm if df else reference_arm)(args)
    else:
        (df_arm if df else our_arm)(args)


if __name__ == "__main__":
    main()
