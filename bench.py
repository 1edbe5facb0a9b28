"""Benchmark: int2e_sph Gint/s on the seeded synthetic molecules, one JSON line on rank 0.

A step is one full pass of the hot path over the workload: every 8-fold-unique shell quartet
whose Schwarz bound reaches 1e-12 (cintx_plan_int2e_screened), evaluated into a device output
ring chunk by chunk (libcint-layout blocks).  The pair tables are resident in HBM before the
timed region; L2 is flushed (a 512 MiB write) between timed steps outside the step events.

  value      Gint/s = spherical integrals written per second, device time (CUDA events on the
             launching stream), max over ranks
  e2e        the same metric through the C ABI from host arrays: optimizer build (host -> device
             basis and pair tables), screened plan, execution and the device -> host copy of every
             chunk's output into pinned host memory, every step (max over ranks of each rank's
             time, every rank evaluating its own chunks)
  roofline   the kernel class with the largest device time in one profiled step: algorithmic FP64
             flops (the plan's flop model) / its event time, against the FP64 FMA peak measured by
             a probe kernel on the same GPU in the same run
  error_vs_libcint  the tuned output of a class-stratified sample of the sweep (up to 2000
             quartets per class) against libcint 6.1.3 built from the reference sources
  cpu_baseline  libcint 6.1.3 built from the reference sources (oracle/_ref), all host cores,
             on seeded uniform samples of the same quartet set (the procedure of --impl reference)

--impl reference times that libcint CPU path alone (rank 0) on the same workload and metric:
each step is one seeded uniform sample of the quartet set (about 1.5 s of libcint work), and
value = the samples' integrals / their libcint time.
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
from cintx_b200.sharding import assign_chunks, chunk_doubles_for, chunks_of, max_over_ranks  # noqa: E402

WORKLOADS = {
    "mol40_spd": (M.mol40, "40 seeded atoms in a 14-bohr cube, 60% light (2s,1p) / 40% heavy "
                           "(3s,2p,1d), exponents log-uniform [0.1,1.2e4]; Schwarz 1e-12"),
    "mol120_spdf": (M.mol120, "120 seeded atoms in a 22-bohr cube, heavy atoms add one f shell; "
                              "Schwarz 1e-12"),
    "water3": (M.water_like, "3-atom water-like molecule (O + 2 H), all quartets above 1e-12"),
    "spdf24": (lambda: M.random_molecule("spdf24", 21, 24, 12.0, with_f=True),
               "24 seeded atoms in a 12-bohr cube with mol120_spdf's shell rules (heavy atoms carry an f shell); "
               "Schwarz 1e-12: the f-shell classes at a size for profiler captures"),
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
# tuned form: bound on the skipped primitive terms of one block (the rest of the 1e-10 budget covers
# FP64 rounding, ~1e-12 against the oracle)
PRIM_BUDGET = 8e-11
# the north-star record: FP32 recurrences where their estimated error fits, with the primitive
# screening budget lowered so that the two budgets together stay inside 1e-10
NORTH_STAR_FP32_BUDGET = 4e-11
NORTH_STAR_PRIM_BUDGET = 5e-11
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
    ap.add_argument("--chunk-doubles", type=int, default=1 << 30,
                    help="largest chunk of the device sweep (output doubles); with N > 1 ranks chunks shrink "
                         "so that every rank gets about sixteen")
    ap.add_argument("--branches", type=int, default=4)
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--form", default="tuned", choices=["tuned", "plain"])
    ap.add_argument("--no-error", action="store_true")
    ap.add_argument("--error-chunks", type=int, default=2)
    ap.add_argument("--libcint-per-class", type=int, default=None,
                    help="quartets per class in the error_vs_libcint sample (default 2000; mol40_spd: all, "
                         "so that every integral of that sweep is checked against libcint)")
    ap.add_argument("--no-decomposition", action="store_true",
                    help="skip the FP64-autotuned-shapes and north-star-form comparison sweeps")
    ap.add_argument("--shapes", default=None,
                    help="launch shapes saved by --save-shapes: applied instead of autotuning (profiler runs, whose "
                         "serialised launches would distort the autotuner's timings)")
    ap.add_argument("--save-shapes", default=None, help="write the autotuned launch shapes to this JSON file")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip every comparison sweep, the plain FP64 one included (profiler runs)")
    ap.add_argument("--fp32-budget", type=float, default=FP32_BUDGET)
    ap.add_argument("--no-autotune", action="store_true", help="tuned form without the launch-shape autotuner")
    ap.add_argument("--no-jk", action="store_true", help="skip the direct J/K build timing")
    ap.add_argument("--e2e-chunk-doubles", type=int, default=1 << 24,
                    help="chunk size of the end-to-end plan (copies of one chunk overlap the next chunk's kernels)")
    ap.add_argument("--prim-budget", type=float, default=PRIM_BUDGET)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    args = ap.parse_args()
    if args.libcint_per_class is None:
        args.libcint_per_class = 1 << 40 if args.workload == "mol40_spd" else 2000
    return args


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


def libcint_steps(mol, sampler, steps, warmup, threads, target_s=1.5, seed0=1000):
    """libcint on seeded uniform samples of a workload's tuple set: warmup + steps samples of
    the same size (sized by a calibration run for about target_s seconds of libcint work each),
    sample s drawn with seed seed0 + s.  The one CPU procedure of both --impl reference and the
    cpu_baseline record.  value = integrals of the timed samples / their libcint seconds."""
    cal = run_libcint(mol, sampler(4000, seed0 - 1), threads)
    per_q = cal["seconds"] / 4000
    n = int(min(8_000_000, max(20_000, target_s / max(per_q, 1e-9))))
    secs, ints = [], []
    for s_ in range(warmup + steps):
        r = run_libcint(mol, sampler(n, seed0 + s_), threads)
        if s_ >= warmup:
            secs.append(r["seconds"])
            ints.append(r["nintegrals"])
            threads_used = int(r["threads"])
    return {"value": sum(ints) / sum(secs) / 1e9, "unit": "Gint/s", "cores": threads_used, "kind": "reference",
            "sample": "%d steps of %d tuples drawn uniformly (seeded) from the tuple set, libcint 6.1.3 with an "
                      "optimizer, OpenMP dynamic over the tuples; value = sampled integrals / libcint seconds" %
                      (steps, n),
            "tuples_per_step": n, "seconds_per_step": secs, "step_ms_mean": statistics.mean(secs) * 1e3,
            "step_ms_spread": [min(secs) * 1e3, max(secs) * 1e3], "seconds_per_tuple": sum(secs) / (n * len(secs))}


# ------------------------------------------------------------------ reference arm
def schwarz_pairs_libcint(mol):
    """Q_ij = sqrt(max |(ij|ij)|) for all pairs i >= j, with libcint on the CPU."""
    from oracle import RefLibcint
    ii, jj = np.tril_indices(mol.nbas)
    pairs = np.stack([ii, jj], axis=1).astype(np.int32)
    vals, offs, _ = RefLibcint().batch(np.concatenate([pairs, pairs], axis=1), mol)
    return pairs, np.sqrt(np.maximum.reduceat(np.abs(vals), offs[:-1]))


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


METRIC = "int2e_sph Gint/s at <=1e-10 abs err"
DF_METRIC = "int3c2e_sph + int2c2e_sph Gint/s, density fitting"


def reference_line(args, metric, value, steps_rec, cfg):
    """The --impl reference JSON line: the measured sample steps are the timed region."""
    return {"metric": metric, "value": value, "unit": "Gint/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": steps_rec["step_ms_mean"], "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "impl": "reference", "config": cfg,
            "cpu_baseline": {k: steps_rec[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "step_ms_spread": steps_rec["step_ms_spread"],
            "e2e": {"value": value, "unit": "Gint/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


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
    rec = libcint_steps(mol, uq.sample, args.steps, args.warmup, threads)
    cfg = {"workload": args.workload, "description": desc, "form": "libcint 6.1.3 int2e_sph on the host cores",
           "nquartets": uq.nquartets, "nintegrals": uq.nintegrals, "schwarz_cutoff": SCHWARZ,
           "step": "one seeded uniform sample of %d quartets of the set" % rec["tuples_per_step"],
           "extrapolated_full_sweep_ms": rec["seconds_per_tuple"] * uq.nquartets * 1e3}
    print(json.dumps(reference_line(args, METRIC, rec["value"], rec, cfg)))


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
        from oracle import RefLibcint
        ref = RefLibcint()
        ii, jj = np.tril_indices(norb)
        pairs = np.stack([ii, jj], axis=1).astype(np.int32)
        aux = np.arange(norb, mol.nbas, dtype=np.int32)
        v, o, _ = ref.batch(np.concatenate([pairs, pairs], axis=1), mol)
        q = np.sqrt(np.maximum.reduceat(np.abs(v), o[:-1]))
        v, o, _ = ref.batch(np.stack([aux, aux], axis=1), mol)
        qk = np.sqrt(np.maximum.reduceat(np.abs(v), o[:-1]))
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
    sampler = df_sampler(tri, aux_pairs, mol)
    rec = libcint_steps(mol, sampler, args.steps, args.warmup, threads)
    cfg = {"workload": args.workload, "description": desc,
           "form": "libcint 6.1.3 int3c2e_sph + int2c2e_sph on the host cores", "ntriples": tri.nquartets,
           "nintegrals": tri.nintegrals + int(sampler.n2int), "schwarz_cutoff": SCHWARZ,
           "step": "one seeded sample of %d tuples: (ab|k) triples and (k|l) pairs in proportion to their counts"
                   % rec["tuples_per_step"]}
    print(json.dumps(reference_line(args, DF_METRIC, rec["value"], rec, cfg)))


def df_sampler(tri, aux_pairs, mol):
    """Sampler over the DF step's tuples: (ab|k) triples of the sweep and (k|l) metric pairs,
    mixed in proportion to their counts."""
    l = mol.bas[:, 1]
    two = np.stack([aux_pairs[:, 0], np.full(len(aux_pairs), -1), aux_pairs[:, 1], np.full(len(aux_pairs), -1)],
                   axis=1).astype(np.int32)
    frac2 = len(two) / (len(two) + tri.nquartets)

    def sample(n, seed):
        n2 = int(round(n * frac2))
        rng = np.random.default_rng(seed + 7919)
        parts = [tri.sample(n - n2, seed), two[rng.integers(0, len(two), size=n2)]]
        return np.concatenate(parts)

    sample.n2int = int(((2 * l[aux_pairs[:, 0]] + 1) * (2 * l[aux_pairs[:, 1]] + 1)).sum())
    return sample


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


def timed_sweep(cx, torch, plan, mine, args, stream, local, world, tune=False, steps=None, warmup=None):
    """Warm-up, then exactly args.steps timed passes of `plan` over the rank's chunks (one CUDA
    graph per pass unless --no-graph), L2 flushed between passes outside the events.  With
    tune, the plan's launch shapes are autotuned first (each class on its largest segment).
    steps / warmup override args.steps / args.warmup (the comparison sweeps run fewer)."""
    return timed_multi(cx, torch, [(plan, mine)], args, stream, local, world, tune, steps, warmup)


def timed_multi(cx, torch, items, args, stream, local, world, tune=False, steps=None, warmup=None):
    """As timed_sweep for several plans run back to back in one step: items = [(plan, chunks)]."""
    nsteps = args.steps if steps is None else steps
    nwarm = args.warmup if warmup is None else warmup
    import torch.distributed as dist
    rings = [torch.empty(max(p.stats.max_chunk_doubles, 1), dtype=torch.float64, device="cuda") for p, _ in items]
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    tuning = None
    if tune:
        t0 = time.perf_counter()
        lanes = {}
        source = "autotuned in this run"
        if args.shapes:
            cx.load_tuned_shapes(json.load(open(args.shapes)))
            source = "loaded from " + os.path.basename(args.shapes)
        for (plan, mine), ring in zip(items, rings):
            if not mine:
                continue
            if args.shapes:
                plan.use_tuned_shapes()
            else:
                plan.autotune(ring.data_ptr(), chunk=-1, stream=stream.cuda_stream, reps=2)
            for c in mine:
                for cl, n in zip(plan.segments(c)[0], plan.segment_lanes(c)):
                    lanes["(%d%d|%d%d)" % tuple(cl)] = int(n)
        if args.save_shapes:
            with open(args.save_shapes, "w") as fh:
                json.dump(cx.tuned_shapes(), fh)
        tuning = {"seconds": time.perf_counter() - t0, "source": source,
                  "lanes_per_quartet": dict(sorted(lanes.items())),
                  "variant_per_class": {"(%d%d|%d%d)%s" % (r[0], r[1], r[2], r[3], " fp32" if r[4] else ""): r[5]
                                        for r in cx.tuned_shapes()}}
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

    for _ in range(nwarm):
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
    for _ in range(nsteps):
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
    ms = max_over_ranks(sum(step_ms), device="cuda") / nsteps
    return {"ms": ms, "steps": nsteps, "step_ms_spread": [min(step_ms), max(step_ms)], "launches": launches, "clocks": clk, "wall": t_wall, "graph": use_graph, "ring": rings[0],
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
    """Max and RMS absolute difference between the tuned plan and an FP64 evaluation of the same
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
        del ref
    return {"max_abs": mx, "rms_abs": (ss / max(n, 1)) ** 0.5, "integrals_checked": n,
            "chunks_checked": len(chunks), "reference": "the same quartets evaluated by the FP64 kernels"}


def class_codes(quartets, lvals):
    """Kernel class of each int2e quartet as an int: 100*(10 la + lb) + (10 lc + ld), the pairs
    oriented larger l first and the pair of larger (la, lb) first (the class the kernels run)."""
    l = lvals[quartets]
    p1 = 10 * np.maximum(l[:, 0], l[:, 1]) + np.minimum(l[:, 0], l[:, 1])
    p2 = 10 * np.maximum(l[:, 2], l[:, 3]) + np.minimum(l[:, 2], l[:, 3])
    return 100 * np.maximum(p1, p2) + np.minimum(p1, p2)


def class_codes3(triples, lvals):
    """Kernel class of each int3c2e triple (a, b, k): the pair (a, b) oriented larger l first and the
    auxiliary shell as the pair (k, unit), the pair of larger l first (as class_codes)."""
    l = lvals[triples]
    p1 = 10 * np.maximum(l[:, 0], l[:, 1]) + np.minimum(l[:, 0], l[:, 1])
    p2 = 10 * l[:, 2]
    return 100 * np.maximum(p1, p2) + np.minimum(p1, p2)


def code_label(code):
    a, b = divmod(int(code), 100)
    return "(%d%d|%d%d)" % (a // 10, a % 10, b // 10, b % 10)


def error_vs_libcint(torch, plan, mol, ring, stream, per_class, seed):
    """The plan's own output for a class-stratified sample of its quartets against libcint 6.1.3
    built from the reference sources (oracle/_ref).  Every chunk is evaluated into `ring`; each
    quartet of a class with T quartets in the sweep is kept with probability per_class / T (all of
    them when T <= per_class), and its block is read back from the chunk's output.  Reports max
    and RMS absolute error over the sampled integrals, the share within the parity rule
    |d| <= 1e-12 or |d| <= 1e-10 |ref| (cintx-oracle two_electron_parity.rs:26-33) and the worst
    class."""
    from oracle import RefLibcint
    rng = np.random.default_rng(seed)
    st = plan.stats
    lv = mol.bas[:, 1].astype(np.int64)
    nsph = 2 * lv + 1
    three = False  # 3-centre plans report tuples (a, b, k, -1): blocks (ab|k), libcint int3c2e_sph
    totals = {}
    for c in range(st.nchunks):
        cls, nq, _ = plan.segments(c)
        for cl, n in zip(cls, nq):
            code = 100 * (10 * int(cl[0]) + int(cl[1])) + 10 * int(cl[2]) + int(cl[3])
            totals[code] = totals.get(code, 0) + int(n)
    t0 = time.perf_counter()
    tuples, got = [], []
    for c in range(st.nchunks):
        q = plan.chunk_quartets(c)
        if len(q) and (q[:, 3] < 0).all():
            three = True
            q = np.ascontiguousarray(q[:, :3])
        codes = class_codes3(q, lv) if three else class_codes(q, lv)
        prob = np.array([min(1.0, per_class / totals.get(int(k), 1)) for k in range(10000)])
        sel = np.where(rng.random(len(q)) < prob[codes])[0]
        if not len(sel):
            continue
        sizes = np.prod(nsph[q], axis=1)
        offs = np.concatenate([[0], np.cumsum(sizes)])
        lens = sizes[sel]
        starts = offs[sel]
        idx = np.repeat(starts - np.concatenate([[0], np.cumsum(lens)[:-1]]), lens) + np.arange(int(lens.sum()))
        plan.execute(ring.data_ptr(), chunk=c, stream=stream.cuda_stream)
        stream.synchronize()
        got.append(ring[torch.from_numpy(idx).to(ring.device)].cpu().numpy())
        tuples.append(q[sel])
    tuples = np.concatenate(tuples)
    got = np.concatenate(got)
    t1 = time.perf_counter()
    ref, offs, _ = RefLibcint().batch(tuples, mol)
    t2 = time.perf_counter()
    d = np.abs(got - ref)
    ok = (d <= 1e-12) | (d <= 1e-10 * np.abs(ref))
    codes = class_codes3(tuples, lv) if three else class_codes(tuples, lv)
    per = {}
    blk = np.repeat(codes, np.diff(offs))
    order = np.argsort(blk, kind="stable")
    bs, ds = blk[order], d[order]
    cuts = np.flatnonzero(np.diff(bs)) + 1
    for part_b, part_d in zip(np.split(bs, cuts), np.split(ds, cuts)):
        per[code_label(part_b[0])] = float(part_d.max())
    worst = max(per.items(), key=lambda kv: kv[1])
    return {"max_abs": float(d.max()), "rms_abs": float(np.sqrt(np.mean(d * d))), "integrals_checked": int(d.size),
            "quartets_checked": int(len(tuples)), "classes_checked": len(per),
            "classes_in_sweep": len(totals), "per_class_target": per_class,
            "parity_rule_share": float(ok.mean()), "worst_class": {"class": worst[0], "max_abs": worst[1]},
            "within_1e-10": bool(d.max() <= 1e-10),
            "reference": "libcint 6.1.3 built from the reference sources (oracle/_ref), same quartets, CPU",
            "seconds": {"sweep_and_gather": t1 - t0, "libcint": t2 - t1}}


# DRAM bytes per quartet measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum of one
# launch / its quartets) for the classes that have been the dominant kernel, with the profile
# summary each figure comes from.
NCU_TRAFFIC_PER_QUARTET = {
    # (dram__bytes_read.sum + dram__bytes_write.sum) of one captured launch / its quartets
    "(10|00)": ((81397504 + 62672384) / 4594144, "profiles/eri4c_1000_mol120_spdf.md"),
}


def roofline_record(per_class, peak64, st, ms_per_step):
    top = max(per_class.items(), key=lambda kv: kv[1]["ms"])
    d = top[1]
    achieved = d["flops"] / (d["ms"] * 1e-3) / 1e12
    prof_total = sum(v["ms"] for v in per_class.values())
    alg_bytes = 8.0 * d["ints"] / d["launches"]
    tr = NCU_TRAFFIC_PER_QUARTET.get(top[0])
    traffic = tr[0] * d["quartets"] / d["launches"] if tr else None
    return {"bound": "fp64", "kernel": "eri4c_kernel" + top[0], "achieved": achieved, "peak": peak64,
            "unit": "TFLOP/s", "frac": achieved / peak64,
            "peak_source": "FP64 FMA probe kernel on this GPU, this run (MEASURED_PEAKS.json has no FP64 figure)",
            "share_of_step": d["ms"] / prof_total,
            "traffic": traffic, "algorithmic_bytes": alg_bytes,
            "traffic_over_algorithmic": traffic / alg_bytes if traffic else None,
            "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum per quartet (%s) x the class's "
                               "quartets per launch" % tr[1]) if tr else "no ncu capture of this class",
            "whole_step_fp64_frac": (st.flops / (ms_per_step * 1e-3) / 1e12) / peak64}


def d2h_bandwidth(torch, nbytes=1 << 30, reps=4):
    """Device-to-host copy bandwidth into page-locked memory (GB/s, best of reps copies of nbytes):
    the bound of an end-to-end step that brings every integral to the host."""
    src = torch.empty(nbytes // 8, dtype=torch.float64, device="cuda")
    dst = torch.empty(nbytes // 8, dtype=torch.float64, pin_memory=True)
    s = torch.cuda.current_stream()
    best = 0.0
    for _ in range(reps + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        dst.copy_(src, non_blocking=True)
        e1.record(s)
        e1.synchronize()
        best = max(best, nbytes / (e0.elapsed_time(e1) * 1e-3) / 1e9)
    del src, dst
    return best


def ip1_record(cx, torch, plan, mol, n=200_000, seed=91, reps=3):
    """First-derivative integrals int2e_ip1_sph (three components per block) of a seeded uniform
    sample of the sweep's quartets through the batched entry point (cintx_ip1_eval: host set-up,
    kernels, into a device buffer; wall time of the call, best of reps) against libcint 6.1.3's
    int2e_ip1_sph on the same tuples on all host cores."""
    from oracle import RefLibcint
    q = np.unique(plan.sample_quartets(n, seed), axis=0)
    nd = cx.ip1_len(cx.INT2E, q, mol.bas)
    buf = torch.empty(nd, dtype=torch.float64, device="cuda")
    best = 1e300
    for _ in range(reps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cx.ip1_eval(cx.INT2E, q, mol.atm, mol.bas, mol.env, buf.data_ptr())
        torch.cuda.synchronize()
        best = min(best, time.perf_counter() - t0)
    got = buf.cpu().numpy()
    t0 = time.perf_counter()
    ref, _, _ = RefLibcint().batch(q, mol, ip1=True)
    t_lib = time.perf_counter() - t0
    d = np.abs(got - ref)
    return {"quartets": int(len(q)), "integrals": int(nd), "seconds": best, "gint_s": nd / best / 1e9,
            "libcint_seconds": t_lib, "libcint_gint_s": nd / t_lib / 1e9, "cores": os.cpu_count(),
            "max_abs_vs_libcint": float(d.max()),
            "parity_rule_share": float(((d <= 1e-12) | (d <= 1e-10 * np.abs(ref))).mean()),
            "what": "int2e_ip1_sph (3 components per block) of a seeded uniform sample of the sweep's quartets: "
                    "cintx_ip1_eval wall time (host set-up + kernels, output on the device) vs libcint on all "
                    "host cores, same tuples"}


def per_call_latency(cx, reps=3):
    """The drop-in per-call path (int2e_sph with libcint's signature: one block per call, host in
    and out, one device round trip) against libcint's own int2e_sph on the same calls (CPU, one
    thread): every 8-fold-unique quartet of the 3-atom water-like molecule, called one after
    another through ctypes with prepared arguments, with and without an optimizer.  The ctypes
    cost of one call (a call of an empty library function) is reported beside them."""
    import ctypes

    from oracle import RefLibcint
    mol = M.water_like()
    nb = mol.nbas
    quart = [(i, j, k, l) for i in range(nb) for j in range(i + 1) for k in range(i + 1) for l in range(k + 1)
             if (i * (i + 1) // 2 + j) >= (k * (k + 1) // 2 + l)]
    shls = np.ascontiguousarray(quart, dtype=np.int32)
    atm, bas, env = (np.ascontiguousarray(a) for a in (mol.atm, mol.bas, mol.env))
    out = np.zeros(4096)
    P = ctypes.POINTER
    ip = lambda a: a.ctypes.data_as(P(ctypes.c_int))
    dp = lambda a: a.ctypes.data_as(P(ctypes.c_double))
    args = (ip(atm), atm.shape[0], ip(bas), bas.shape[0], dp(env))
    rows = [ip(shls[q]) for q in range(len(shls))]

    def run(f, opt):
        po = dp(out)
        best = 1e300
        for _ in range(reps):
            t0 = time.perf_counter()
            for r in rows:
                f(po, None, r, *args, opt, None)
            best = min(best, time.perf_counter() - t0)
        return 1e6 * best / len(rows)

    ours = cx.lib.int2e_sph
    ref = RefLibcint()
    lcint = ref.lib.int2e_sph
    o = cx.Optimizer(mol.atm, mol.bas, mol.env)
    lopt = ctypes.c_void_p()
    ref.lib.int2e_optimizer(ctypes.byref(lopt), *args)
    run(ours, None)  # warm-up: device state, thread scratch
    rec = {"quartets": len(rows), "molecule": "water-like, 3 atoms, %d shells" % nb,
           "us_per_call_ours": run(ours, None), "us_per_call_ours_opt": run(ours, o.handle),
           "us_per_call_libcint": run(lcint, None), "us_per_call_libcint_opt": run(lcint, lopt)}
    noop = cx.lib.cintx_cuda_last_error_code
    t0 = time.perf_counter()
    for _ in rows:
        noop()
    rec["us_ctypes_call"] = 1e6 * (time.perf_counter() - t0) / len(rows)
    ref.lib.CINTdel_optimizer(ctypes.byref(lopt))
    o.close()
    rec["what"] = ("libcint-signature int2e_sph per call (one block, host in/out: one H2D copy, one kernel, one D2H "
                   "copy and a stream synchronisation per call) vs libcint 6.1.3 int2e_sph on the host, same "
                   "quartets, best of %d passes; both through ctypes with prepared arguments" % reps)
    return rec


def learned_root_sample(cx, torch, opt, plan, mol, stream, n, seed):
    """Learned Rys roots on a seeded uniform sample of the sweep's quartets (an explicit plan: its
    root buffer holds every primitive quartet's roots, which the full sweep's 1e10 primitive
    quartets would not fit): RysNet trained on the device for 1..7 roots, the sample evaluated
    with learned roots and with table roots (same launch shapes), times and errors vs libcint."""
    from oracle import RefLibcint
    quart = plan.sample_quartets(n, seed)
    quart = np.unique(quart, axis=0)
    net = cx.RysNet(seed=0)
    t0 = time.perf_counter()
    net.train(nsamples=5_000_000, n_lo=1, n_hi=7, epochs=40, batch=16384, lr=3e-3, seed=1)
    train_s = time.perf_counter() - t0
    p_tab = cx.Plan.shells(opt, cx.INT2E, quart)
    p_lrn = cx.Plan.shells(opt, cx.INT2E, quart)
    p_tab.use_tuned_shapes()
    p_lrn.use_tuned_shapes()
    fb, npq = p_lrn.use_learned_roots(net)
    nint = p_lrn.stats.nintegrals
    a = torch.empty(nint, dtype=torch.float64, device="cuda")
    b = torch.empty_like(a)
    ms = {}
    for name, p, buf in (("learned", p_lrn, a), ("table", p_tab, b)):
        p.execute(buf.data_ptr(), stream=stream.cuda_stream)
        stream.synchronize()
        times = []
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            p.execute(buf.data_ptr(), stream=stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        ms[name] = statistics.median(times)
    ref, _, _ = RefLibcint().batch(quart, mol)
    got = a.cpu().numpy()
    d = np.abs(got - ref)
    p_tab.close()
    p_lrn.close()
    return {"quartets": int(len(quart)), "integrals": int(nint), "primitive_quartets": int(npq),
            "fallback": int(fb), "fallback_rate": fb / max(npq, 1), "train_seconds": train_s,
            "gint_s_learned": nint / (ms["learned"] * 1e-3) / 1e9, "gint_s_table": nint / (ms["table"] * 1e-3) / 1e9,
            "learned_over_table": ms["table"] / ms["learned"],
            "max_abs_vs_libcint": float(d.max()), "rms_abs_vs_libcint": float(np.sqrt(np.mean(d * d))),
            "what": "seeded uniform sample of the sweep's quartets as an explicit plan; roots from the device-trained "
                    "MLP (1..7 roots) refined in FP64 with table fallback, vs table roots in the same kernels"}


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

    def make_plan(o, form, chunk_doubles):
        if form == "tuned":
            return cx.Plan.screened_mixed(o, SCHWARZ, fp32_budget=args.fp32_budget, prim_budget=args.prim_budget,
                                          max_chunk_doubles=chunk_doubles)
        if form == "fp64_tuned_shapes":
            return cx.Plan.screened_mixed(o, SCHWARZ, fp32_budget=0.0, prim_budget=0.0,
                                          max_chunk_doubles=chunk_doubles)
        if form == "north_star":
            return cx.Plan.screened_mixed(o, SCHWARZ, fp32_budget=NORTH_STAR_FP32_BUDGET,
                                          prim_budget=NORTH_STAR_PRIM_BUDGET, max_chunk_doubles=chunk_doubles)
        return cx.Plan.screened(o, SCHWARZ, sph=True, max_chunk_doubles=chunk_doubles)

    def shard(p):
        return chunks_of(assign_chunks([float(p.segments(c)[2].sum()) for c in range(p.stats.nchunks)], world), rank)

    plan = make_plan(opt, "tuned" if tuned else "plain", args.chunk_doubles)
    cd = chunk_doubles_for(plan.stats.nintegrals, world, args.chunk_doubles)
    if cd != args.chunk_doubles:  # N > 1: about sixteen chunks per rank for the longest-first split
        args.chunk_doubles = cd
        plan = make_plan(opt, "tuned" if tuned else "plain", cd)
    st = plan.stats
    nchunks = st.nchunks
    mine = shard(plan)
    stream = torch.cuda.Stream()  # a real stream handle: events and kernels share it
    torch.cuda.set_stream(stream)

    main_run = timed_sweep(cx, torch, plan, mine, args, stream, local, world, tune=tuned and not args.no_autotune)
    ms_per_step = main_run["ms"]
    value = st.nintegrals / (ms_per_step * 1e-3) / 1e9
    # comparison sweeps (fewer steps; every rank runs them in the same order)
    extra = {}
    if tuned and not args.no_compare:
        forms = ["plain"] + ([] if args.no_decomposition else ["fp64_tuned_shapes", "north_star"])
        for form in forms:
            p = make_plan(opt, form, args.chunk_doubles)
            if form != "plain" and not args.no_autotune:
                p.use_tuned_shapes()
            run = timed_sweep(cx, torch, p, shard(p), args, stream, local, world, steps=max(1, min(args.steps, 5)),
                              warmup=2)
            ps = p.stats
            extra[form] = {"plan": p, "value": ps.nintegrals / (run["ms"] * 1e-3) / 1e9, "ms_per_step": run["ms"],
                           "steps": run["steps"], "nquartets_fp32": ps.nquartets_fp32,
                           "nprim_quartets": ps.nprim_quartets, "ring": run["ring"]}
            del run

    per_class = class_profile(torch, plan, mine, main_run["ring"], stream)
    peak64 = fp64_peak(cx, torch)
    roof = roofline_record(per_class, peak64, st, ms_per_step) if per_class else None
    err = err_lib = None
    ns_rec = None
    if tuned and rank == 0 and not args.no_error:
        err = tuned_error(cx, torch, opt, plan, main_run["ring"], stream, args.error_chunks)
        if os.path.exists(REF_DRIVER):
            err_lib = error_vs_libcint(torch, plan, mol, main_run["ring"], stream, args.libcint_per_class, 2027)
            if "north_star" in extra:
                e = extra["north_star"]
                ns_rec = {"error_vs_libcint": error_vs_libcint(torch, e["plan"], mol, e["ring"], stream, 500, 2028)}
                ns_rec["learned_roots_sample"] = learned_root_sample(cx, torch, opt, plan, mol, stream, 100_000, 77)
    for e in extra.values():
        e["plan"].close()
        e.pop("plan")
        e.pop("ring")
    jk = None
    if rank == 0 and world == 1 and not args.no_jk:
        jk = jk_timing(cx, torch, plan, mol, stream, min(args.steps, 5))
    per_call = ip1 = None
    if rank == 0 and world == 1 and not args.no_cpu and os.path.exists(REF_DRIVER):
        per_call = per_call_latency(cx)
        ip1 = ip1_record(cx, torch, plan, mol)

    # end-to-end through the C ABI from host arrays, measured on every rank over its own chunks:
    # optimizer from atm/bas/env, screened plan, evaluation and D2H into page-locked host memory;
    # the step time is the max over ranks
    e2e = None
    if not args.no_e2e:
        e2e_chunk = args.e2e_chunk_doubles
        host = None
        phases = {"optimizer": [], "plan": [], "execute_d2h": []}
        h2d = d2h = 0
        for s_ in range(1 + max(1, min(args.steps, 3))):
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            o2 = cx.Optimizer(mol.atm, mol.bas, mol.env)
            t1 = time.perf_counter()
            p2 = make_plan(o2, "tuned" if tuned else "plain", e2e_chunk)
            if tuned and not args.no_autotune:
                p2.use_tuned_shapes()  # shapes autotuned once in this process (before the timed sweep)
            t2 = time.perf_counter()
            if host is None or host.size < 2 * p2.stats.max_chunk_doubles:  # two-slot page-locked host ring
                # allocated in the untimed first iteration; later iterations reuse it
                host = torch.empty(2 * max(p2.stats.max_chunk_doubles, 1), dtype=torch.float64,
                                   pin_memory=True).numpy()
            e2e_mine = shard(p2)
            if world == 1:
                p2.execute_host_ring(host)
                mine_ints = p2.stats.nintegrals
            else:
                mine_ints = 0
                for c in e2e_mine:
                    p2.execute_host(host, chunk=c)
                    mine_ints += p2.chunk_size(c)
            t3 = time.perf_counter()
            if s_ > 0:
                phases["optimizer"].append(t1 - t0)
                phases["plan"].append(t2 - t1)
                phases["execute_d2h"].append(t3 - t2)
            h2d = mol.atm.nbytes + mol.bas.nbytes + mol.env.nbytes + o2.device_bytes + p2.stats.device_bytes
            d2h = mine_ints * 8
            p2.close()
            o2.close()
        te_local = sum(statistics.mean(v) for v in phases.values())
        te = max_over_ranks(te_local, device="cuda")
        h2d_all = max_over_ranks(h2d, device="cuda") * world  # every rank uploads the basis and its plan
        d2h_all = st.nintegrals * 8
        bw = d2h_bandwidth(torch)
        e2e = {"value": st.nintegrals / te / 1e9, "unit": "Gint/s", "h2d_bytes_per_step": int(h2d_all),
               "d2h_bytes_per_step": int(d2h_all), "seconds_per_step": te,
               "phases_s": {k: statistics.mean(v) for k, v in phases.items()},
               "d2h_gbs_measured": bw, "d2h_bound_gint_s": bw / 8.0 * world,
               "fraction_of_d2h_bound": (st.nintegrals / te / 1e9) / (bw / 8.0 * world),
               "chunk_doubles": e2e_chunk, "ranks_timed": world,
               "includes": "int2e_optimizer from host atm/bas/env (pair tables, Schwarz passes) + screened "
                           "plan + evaluation + D2H of every integral (each rank its own chunks; a two-chunk "
                           "page-locked host ring overlapping copies with the next chunk's kernels at N=1); "
                           "max over ranks"}
    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        plan.close()
        opt.close()
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
    line = {"metric": METRIC, "value": value, "unit": "Gint/s",
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
            "step_ms_spread": main_run["step_ms_spread"],
            "roofline": roof,
            "output_write_gbs": st.nintegrals * 8 / (ms_per_step * 1e-3) / 1e9,
            "hbm_gbs_measured_peak": hbm,
            "execution": "one CUDA graph per step (%d kernel classes on %d branches)" % (len(per_class), args.branches)
                         if main_run["graph"] else "direct launches",
            "per_class": {k: {"ms": round(v["ms"], 4), "tflops": round(v["flops"] / (v["ms"] * 1e-3) / 1e12, 3),
                              "gint_s": round(v["ints"] / (v["ms"] * 1e-3) / 1e9, 2),
                              "out_gbs": round(8 * v["ints"] / (v["ms"] * 1e-3) / 1e9, 1), "quartets": v["quartets"]}
                          for k, v in sorted(per_class.items(), key=lambda kv: -kv[1]["ms"])[:16]},
            "profiled_step_ms": sum(v["ms"] for v in per_class.values())}
    if main_run["tuning"] is not None:
        line["autotune"] = main_run["tuning"]
    if "plain" in extra:
        line["plain_fp64"] = extra["plain"]
        line["tuned_over_plain"] = value / extra["plain"]["value"]
    if "fp64_tuned_shapes" in extra:
        pv = extra["plain"]["value"]
        sv = extra["fp64_tuned_shapes"]["value"]
        line["decomposition"] = {
            "plain_fp64": pv, "fp64_autotuned_shapes": sv, "tuned": value,
            "autotuner_factor": sv / pv, "primitive_screening_factor": value / sv,
            "what": "plain = default shapes, libcint screening; fp64_autotuned_shapes = the tuned plan's launch shapes "
                    "with no primitive screening and no FP32; tuned = this line's value (autotuned shapes + primitive "
                    "Schwarz screening within %g per integral)" % args.prim_budget}
    if "north_star" in extra:
        e = extra["north_star"]
        rec = {"value": e["value"], "ms_per_step": e["ms_per_step"], "steps": e["steps"],
               "over_plain": e["value"] / extra["plain"]["value"],
               "fp32_budget": NORTH_STAR_FP32_BUDGET, "prim_budget": NORTH_STAR_PRIM_BUDGET,
               "nquartets_fp32": e["nquartets_fp32"],
               "fp32_quartet_share": e["nquartets_fp32"] / max(st.nquartets, 1),
               "form": "autotuned shapes + primitive Schwarz screening + FP32 recurrences where the estimated FP32 "
                       "error is below the budget, table roots in the full sweep (learned roots measured on a sample: "
                       "their per-primitive-quartet root buffer does not fit the full sweep)"}
        if ns_rec:
            rec.update(ns_rec)
            lr = ns_rec["learned_roots_sample"]["learned_over_table"]
            rec["with_learned_roots_over_plain_estimate"] = rec["over_plain"] * lr
            rec["meets_3x_at_1e-10"] = bool(rec["with_learned_roots_over_plain_estimate"] >= 3.0 and
                                            ns_rec["error_vs_libcint"]["max_abs"] <= 1e-10)
        line["north_star_form"] = rec
    if err is not None:
        line["error_vs_fp64"] = err
    if err_lib is not None:
        line["error_vs_libcint"] = err_lib
    if jk is not None:
        line["jk_build"] = jk
    if per_call is not None:
        line["per_call"] = per_call
    if ip1 is not None:
        line["ip1"] = ip1
    if e2e is not None:
        line["e2e"] = e2e
    if world == 1 and not args.no_cpu and os.path.exists(REF_DRIVER):
        uq = UniqueQuartets(mol, SCHWARZ)
        cb = libcint_steps(mol, uq.sample, 3, 1, os.cpu_count() or 1)
        line["cpu_baseline"] = cb
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
    cd = chunk_doubles_for(p3.stats.nintegrals, world, args.chunk_doubles)
    if cd != args.chunk_doubles:  # N > 1: about sixteen chunks per rank for the longest-first split
        args.chunk_doubles = cd
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
    err_lib = None
    if tuned and rank == 0 and world == 1 and not args.no_error and os.path.exists(REF_DRIVER):
        err_lib = error_vs_libcint(torch, p3, mol, run["rings"][0], stream, args.libcint_per_class, 2029)
    per_class = class_profile(torch, p3, mine3, run["rings"][0], stream)
    peak64 = fp64_peak(cx, torch)
    from types import SimpleNamespace
    roof = roofline_record(per_class, peak64, SimpleNamespace(flops=s3.flops + s2.flops), run["ms"]) \
        if per_class else None
    e2e = None
    if not args.no_e2e:
        # end to end from host arrays on every rank: optimizer, both plans, evaluation of the rank's
        # 3-centre chunks (rank 0 also the 2-centre metric) and D2H of each into page-locked host
        # memory; at N = 1 the 3-centre sweep runs in chunks of --e2e-chunk-doubles through a
        # two-slot host ring (copies overlap the next chunk's kernels), as the int2e e2e; max over ranks
        e2e_chunk = args.e2e_chunk_doubles
        ring = host2 = None
        phases = {"optimizer": [], "plan": [], "execute_d2h": []}
        for s_ in range(1 + max(1, min(args.steps, 3))):
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            o2 = cx.Optimizer(mol.atm, mol.bas, mol.env, pair_shells=norb)
            t1 = time.perf_counter()
            e3 = cx.Plan.screened_3c(o2, norb, SCHWARZ, max_chunk_doubles=e2e_chunk)
            e2 = cx.Plan.shells(o2, cx.INT2C2E, aux_pairs)
            if tuned and not args.no_autotune:
                e3.use_tuned_shapes()
                e2.use_tuned_shapes()
            t2 = time.perf_counter()
            if ring is None:  # page-locked host buffers, allocated in the untimed first iteration
                ring = torch.empty(2 * max(e3.stats.max_chunk_doubles, 1), dtype=torch.float64,
                                   pin_memory=True).numpy()
                host2 = torch.empty(max(e2.stats.nintegrals, 1), dtype=torch.float64, pin_memory=True).numpy()
            if world == 1:
                e3.execute_host_ring(ring)
            else:
                for c in chunks_of(assign_chunks([float(e3.segments(c)[2].sum()) for c in range(e3.stats.nchunks)],
                                                 world), rank):
                    e3.execute_host(ring, chunk=c)
            if rank == 0:
                e2.execute_host(host2)
            t3 = time.perf_counter()
            if s_ > 0:
                phases["optimizer"].append(t1 - t0)
                phases["plan"].append(t2 - t1)
                phases["execute_d2h"].append(t3 - t2)
            h2d = mol.atm.nbytes + mol.bas.nbytes + mol.env.nbytes + o2.device_bytes + e3.stats.device_bytes
            e3.close()
            e2.close()
            o2.close()
        te = max_over_ranks(sum(statistics.mean(v) for v in phases.values()), device="cuda")
        e2e = {"value": nint / te / 1e9, "unit": "Gint/s", "h2d_bytes_per_step": int(h2d) * world,
               "d2h_bytes_per_step": int(nint * 8), "seconds_per_step": te,
               "phases_s": {k: statistics.mean(v) for k, v in phases.items()}, "chunk_doubles": e2e_chunk,
               "ranks_timed": world,
               "includes": "optimizer from host atm/bas/env, both plans (Schwarz passes), evaluation and "
                           "D2H of every integral (each rank its own chunks; a two-chunk page-locked host ring "
                           "overlapping copies with the next chunk's kernels at N=1); max over ranks"}
    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    line = {"metric": DF_METRIC, "value": value, "unit": "Gint/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
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
    if err_lib is not None:
        line["error_vs_libcint"] = err_lib
    if e2e is not None:
        line["e2e"] = e2e
    if world == 1 and not args.no_cpu and os.path.exists(REF_DRIVER):
        tri = DFTriples(mol, norb, SCHWARZ)
        line["cpu_baseline"] = libcint_steps(mol, df_sampler(tri, aux_pairs, mol), 3, 1, os.cpu_count() or 1)
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
