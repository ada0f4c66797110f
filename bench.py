"""J+K benchmark of the B200 engine on the C40H82 / cc-pVDZ workload.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one full J + K build (Coulomb operator, thresp = thre_pq = 1e-14,
mixed-precision cutoff thredp = 1e-5) on the converged RHF density of all-trans
C40H82 in cc-pVDZ (970 pure / 1010 Cartesian functions, 1290 primitive
shells). `value` is quartets/s with D, J and K resident in HBM (device entry
points); `e2e` is the same metric through the public host API
(ls.IntBox.coulomb / exchange on host tensors: each call's H2D copy of D and
the D2H copies of J and K are inside the timed region). L2 is flushed between steps
by writing a 256 MiB buffer outside the timed events. For N > 1 each rank
runs an independent replica on its own GPU (weak scaling); the max time over
ranks is used. `--impl reference` times the reference CPU IntBox
(oracle/_ref) on a bounded sample with all host cores.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "J+K ms/iter & quartets/s: mixed vs FP64 GPU at |ΔE|≤1e-6 Eh; CPU ref alongside"
THRE = 1.0e-14
THREDP = 1.0e-5
K_TRAFFIC_C40 = 0.6423e9  # ncu dram__bytes_read.sum + dram__bytes_write.sum, FP64 K build of C40H82
SAMPLE_CARBONS = 8        # CPU baseline sample: C8H18 / cc-pVDZ, full J+K


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--carbons", type=int, default=40)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuned re-timing")
    ap.add_argument("--no-merge", action="store_true",
                    help="alkane: K over the primitives as given (the reference's exact quartet set) instead of "
                         "the merged twins")
    ap.add_argument("--scf-maxiter", type=int, default=60)
    ap.add_argument("--workload", default="alkane",
                    choices=["alkane", "batched", "guess", "many", "eri", "grad", "fshell"],
                    help="alkane: the headline C40H82 J+K step; batched: 64 response-like densities "
                         "of a 32-water cluster per step (one line per operator and precision); guess: "
                         "train the learned SCF guess and time SCFs from it against SAD")
    ap.add_argument("--molecules", type=int, default=512, help="many: number of water clusters")
    ap.add_argument("--waters", type=int, default=16, help="eri: water cluster size (fshell: 4 unless given)")
    ap.add_argument("--active", type=int, default=12, help="eri: active orbitals")
    ap.add_argument("--train-clusters", type=int, default=1000)
    ap.add_argument("--test-clusters", type=int, default=20)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--guess-norm", default="element", choices=["element", "type"])
    ap.add_argument("--profile-step", action="store_true",
                    help="after set-up and warm-up, run one FP64 J+K step between cudaProfilerStart/Stop "
                         "(for ncu --profile-from-start off) and exit")
    return ap.parse_args()


def dist_info():
    # read here (not through lightspeed_b200.replicas) so the reference arm never loads the engine
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload(ls, ncarbon):
    from lightspeed_b200.geometry import alkane
    mol = alkane(ncarbon)
    bas = ls.Basis.from_gbs_file(mol, "cc-pvdz")
    return mol, bas


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        import tempfile
        fd, self.path = tempfile.mkstemp(prefix="lsjk_clocks_", suffix=".csv")
        os.close(fd)

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.remove(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_sample():
    """Bounded CPU sample of the workload: C8H18 / cc-pVDZ (all-trans, the same
    basis, thresholds and operator), full J + K at its converged RHF density
    (tests/golden/c8h18_ccpvdz_cocc.npz, converged by the reference CPU
    IntBox itself). Geometry, basis and density come from oracle/ alone, so
    this path loads no code of the product; quartets are counted by the
    oracle's counting routine (the reference quartet set)."""
    from oracle import port, ref, workloads
    symbols, xyz = workloads.alkane(SAMPLE_CARBONS)
    arrays, prims, nao = workloads.basis(symbols, xyz, "cc-pvdz")
    rb = ref.RefBasis(arrays)
    rp = ref.RefPairs(rb, rb, True, THRE)
    z = np.load(os.path.join(ROOT, "tests", "golden", "c%dh%d_ccpvdz_cocc.npz" % (SAMPLE_CARBONS,
                                                                                2 * SAMPLE_CARBONS + 2)))
    C = z["Cocc"]
    D = C @ C.T
    pb = port.Basis(prims)
    ppl = port.Pairs(pb, pb, True, THRE)
    nj, nk = port.count_quartets(ppl, ppl, D, D, True, THRE)
    desc = ("C%dH%d/cc-pVDZ (%d bf) full J+K, FP64, thre_pq = thresp = 1e-14, at its converged RHF density "
            "(reference CPU IntBox SCF); %.4g quartets per J+K (J %.4g, K %.4g)" % (
                SAMPLE_CARBONS, 2 * SAMPLE_CARBONS + 2, nao, nj + nk, nj, nk))
    return rp, D, nj + nk, desc


def time_reference(rp, D, nthread):
    from oracle import ref
    t0 = time.time()
    ref.coulomb(rp, rp, D, THRE, THRE, nthread=nthread)
    ref.exchange(rp, rp, D, True, THRE, THRE, nthread=nthread)
    return time.time() - t0


def cpu_baseline(nthread):
    """The reference CPU IntBox (oracle/_ref) timed on the bounded sample."""
    from oracle import port, ref
    if not (ref.available() and port.available()):
        return {"error": "oracle/_ref not built"}
    rp, D, nq, desc = cpu_sample()
    time_reference(rp, D, nthread)   # warm-up (J and K)
    dt = time_reference(rp, D, nthread)
    return {"value": nq / dt, "unit": "quartets/s", "cores": nthread, "cpu_model": cpu_model(), "kind": "reference",
            "sample": desc + "; %.2f s" % dt, "seconds": dt}


def workload_config(ncarbon):
    """The workload as both arms name it."""
    return {"workload": "C%dH%d/cc-pVDZ full J+K build at the converged RHF density" % (ncarbon, 2 * ncarbon + 2),
            "thre_pq": THRE, "thresp": THRE, "thredp": THREDP, "operator": "1/r",
            "l2": "flushed between steps (256 MiB write outside the timed events)"}


def run_reference(args):
    rank, world, local = dist_info()
    if rank != 0:
        return 0
    from oracle import port, ref
    if not (ref.available() and port.available()):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference CPU IntBox) is not built"}))
        return 0
    nthread = os.cpu_count() or 1
    rp, D, nq, desc = cpu_sample()
    for _ in range(args.warmup):
        time_reference(rp, D, nthread)
    times = [time_reference(rp, D, nthread) for _ in range(args.steps)]
    T = float(np.sum(times))
    v = nq * args.steps / T
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "quartets/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * T / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.carbons),
        "cpu_baseline": {"value": v, "unit": "quartets/s", "cores": nthread, "cpu_model": cpu_model(),
                         "kind": "reference", "sample": desc},
        "e2e": {"value": v, "unit": "quartets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


def run_ours(args):
    rank, world, local = dist_info()
    import torch
    torch.cuda.set_device(local)
    os.environ.setdefault("LSJK_DEVICE", str(local))
    from lightspeed_b200 import replicas
    replicas.init("nccl", timeout_s=600)
    import lightspeed_b200 as ls
    from lightspeed_b200.scf import RHF
    mol, bas = workload(ls, args.carbons)
    # converged density (FP64 J/K), the state an SCF iteration sees
    ls.set_precision(ls.PREC_FP64)
    t0 = time.time()
    from lightspeed_b200.sad import SAD
    scf = RHF(ls, mol, bas, thre_pq=THRE, thre_sp=THRE, thre_dp=THRE)
    D_sad = SAD(ls, "cc-pvdz").density(mol, bas)
    E_scf = scf.compute(D0=D_sad, maxiter=args.scf_maxiter, g_conv=1e-6)
    t_scf = time.time() - t0
    # the same SCF with mixed-precision J/K (quartets below thredp in FP32, incremental
    # Fock builds on FP64 difference densities): energy error per iteration and at
    # convergence against the FP64 SCF
    scf_mixed = None
    if not args.profile_step:
        ls.set_precision(ls.PREC_MIXED)
        t0 = time.time()
        scf_mx = RHF(ls, mol, bas, thre_pq=THRE, thre_sp=THRE, thre_dp=THREDP)
        E_mx = scf_mx.compute(D0=D_sad, maxiter=args.scf_maxiter, g_conv=1e-6)
        n = min(len(scf.trace), len(scf_mx.trace))
        scf_mixed = {"energy": E_mx, "dE_final_Eh": E_mx - E_scf, "converged": bool(scf_mx.converged),
                     "iterations": len(scf_mx.trace), "seconds": time.time() - t0,
                     "dE_per_iteration_Eh": [scf_mx.trace[k]["E"] - scf.trace[k]["E"] for k in range(n)]}
        ls.set_precision(ls.PREC_FP64)
    D = scf.D
    pl = scf.pairs
    ew = ls.Ewald.coulomb()
    res = ls.ResourceList.build()
    nao = bas.nao
    dev = torch.device("cuda", local)
    stream = torch.cuda.ExternalStream(ls.stream_handle(), device=dev)
    Dd = torch.tensor(D, dtype=torch.float64, device=dev)
    Jd = torch.zeros_like(Dd)
    Kd = torch.zeros_like(Dd)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step(thredp):
        ls.coulomb_device(ew, pl, pl, [Dd.data_ptr()], [Jd.data_ptr()], THRE, thredp)
        ls.exchange_device(ew, pl, pl, [Dd.data_ptr()], True, [Kd.data_ptr()], THRE, thredp)

    def timed(mode, thredp, nsteps):
        ls.set_precision(mode)
        ms_total, ms_k = 0.0, 0.0
        for _ in range(nsteps):
            with torch.cuda.stream(stream):
                flush.zero_()
                Jd.zero_()
                Kd.zero_()
                e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
                e0.record(stream)
                ls.coulomb_device(ew, pl, pl, [Dd.data_ptr()], [Jd.data_ptr()], THRE, thredp)
                e1.record(stream)
                ls.exchange_device(ew, pl, pl, [Dd.data_ptr()], True, [Kd.data_ptr()], THRE, thredp)
                e2.record(stream)
            e2.synchronize()
            ms_total += e0.elapsed_time(e2)
            ms_k += e1.elapsed_time(e2)
        return ms_total, ms_k

    # the headline runs K over the merged twins (shared s exponents computed once);
    # the exact reference quartet set (merging off) is timed beside it
    merge = not args.no_merge
    ls.set_merge(merge)
    # warm-up in both precision modes (and in exact mode, timed below too)
    for mg in ((merge, False) if merge else (False,)):
        ls.set_merge(mg)
        for mode in (ls.PREC_FP64, ls.PREC_MIXED):
            ls.set_precision(mode)
            for _ in range(args.warmup):
                step(THREDP)
    ls.set_merge(merge)
    torch.cuda.synchronize()
    if args.profile_step:
        ls.set_precision(ls.PREC_FP64)
        torch.cuda.profiler.start()
        step(THREDP)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        ls.set_precision(ls.PREC_MIXED)
        torch.cuda.profiler.start()
        step(THREDP)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(json.dumps({"profile_step": True, "workload": "C%dH%d/cc-pVDZ" % (args.carbons, 2 * args.carbons + 2)}))
        return 0
    # quartet/flop counts of one step in each mode (the quartets the merged build computes)
    counts = {}
    for name, mode in (("fp64", ls.PREC_FP64), ("mixed", ls.PREC_MIXED)):
        ls.set_precision(mode)
        ls.reset_stats()
        step(THREDP)
        torch.cuda.synchronize()
        counts[name] = dict(ls.stats())
        counts[name].update({"flops_" + k: v for k, v in ls.flops_split().items()})
    # the workload's quartets in the reference's definition: the same step over the
    # primitives as given (merging off), whose counters equal the reference quartet set
    ls.set_merge(False)
    ls.set_precision(ls.PREC_FP64)
    ls.reset_stats()
    step(THREDP)
    torch.cuda.synchronize()
    st_ref = ls.stats()
    q_ref = st_ref["j_quartets"] + st_ref["k_quartets"]
    ls.set_merge(merge)
    # energies at the converged density: E(D) with FP64 vs mixed J/K, and the
    # headline's FP64 build against the exact reference quartet set
    energies = {}
    for name, mode, mg in (("fp64", ls.PREC_FP64, merge), ("mixed", ls.PREC_MIXED, merge),
                           ("fp64_exact", ls.PREC_FP64, False)):
        ls.set_merge(mg)
        ls.set_precision(mode)
        J = ls.IntBox.coulomb(res, ew, pl, pl, ls.Tensor.array(D), THRE, THREDP).np
        K = ls.IntBox.exchange(res, ew, pl, pl, ls.Tensor.array(D), True, THRE, THREDP).np
        energies[name] = scf.energy(D, J, K)[0]
    ls.set_merge(merge)
    dE = energies["mixed"] - energies["fp64"]
    dE_merge = energies["fp64"] - energies["fp64_exact"]

    # ---- timed region -------------------------------------------------------
    clocks = Clocks(local)
    clocks.start()
    replicas.barrier()
    torch.cuda.synchronize()
    launches0 = ls.stats()["kernel_launches"]
    ms64, msk64 = timed(ls.PREC_FP64, THREDP, args.steps)
    launches_fp64 = ls.stats()["kernel_launches"] - launches0
    msmx, mskmx = timed(ls.PREC_MIXED, THREDP, args.steps)
    torch.cuda.synchronize()
    launches_timed = ls.stats()["kernel_launches"] - launches0
    exact = {}
    if merge:
        ls.set_merge(False)
        ex64, exk64 = timed(ls.PREC_FP64, THREDP, args.steps)
        exmx, exkmx = timed(ls.PREC_MIXED, THREDP, args.steps)
        ls.set_merge(True)
        exact = {"fp64_ms": ex64 / args.steps, "fp64_ms_k": exk64 / args.steps, "mixed_ms": exmx / args.steps,
                 "mixed_ms_k": exkmx / args.steps}
    # the autotuner's value: one tuning build per mode (candidate launch shapes timed per
    # class), then the same timed steps with the tuned table
    tuned = None
    if not args.no_tune:
        ls.set_autotune(True)
        for mode in (ls.PREC_FP64, ls.PREC_MIXED):
            ls.set_precision(mode)
            step(THREDP)
        ls.set_autotune(False)
        torch.cuda.synchronize()
        tu64, tuk64 = timed(ls.PREC_FP64, THREDP, args.steps)
        tumx, tukmx = timed(ls.PREC_MIXED, THREDP, args.steps)
        tuned = {"fp64_ms": tu64 / args.steps, "fp64_ms_k": tuk64 / args.steps, "mixed_ms": tumx / args.steps,
                 "mixed_ms_k": tukmx / args.steps, "default_fp64_ms": ms64 / args.steps,
                 "default_mixed_ms": msmx / args.steps}
    # e2e through the public host API (each call copies D host->device; J and K come back)
    Dt = ls.Tensor.array(D)
    e2e_ms = 0.0
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        torch.cuda.synchronize()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        t_host = time.time()
        ls.IntBox.coulomb(res, ew, pl, pl, Dt, THRE, THREDP)
        ls.IntBox.exchange(res, ew, pl, pl, Dt, True, THRE, THREDP)
        s1.record(stream)
        s1.synchronize()
        e2e_ms += max(s0.elapsed_time(s1), 1e3 * (time.time() - t_host))
    replicas.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()

    # every timing as its maximum over the ranks (one all-reduce)
    ms64, msk64, msmx, mskmx, e2e_ms = replicas.max_over_ranks([ms64, msk64, msmx, mskmx, e2e_ms], device=dev)
    if rank != 0:
        replicas.finish()
        return 0
    # computed quartets (merged twins) and the workload's reference quartet count
    q64 = counts["fp64"]["j_quartets"] + counts["fp64"]["k_quartets"]
    qmx = counts["mixed"]["j_quartets"] + counts["mixed"]["k_quartets"]
    fp64_qps = replicas.whole_job_rate(q_ref * args.steps, world, ms64 * 1e-3)
    mixed_qps = replicas.whole_job_rate(q_ref * args.steps, world, msmx * 1e-3)
    e2e_qps = replicas.whole_job_rate(q_ref * args.steps, world, e2e_ms * 1e-3)
    peak64 = ls.fma_peak_tflops(True)
    peak32 = ls.fma_peak_tflops(False)
    # roofline of the dominant kernel family (the K kernels, FP64 path)
    flops_k = counts["fp64"]["flops_k"]
    achieved = flops_k / (msk64 / args.steps * 1e-3) / 1e12
    cpu = None
    if not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(os.cpu_count() or 1)
        except Exception as ex:  # reported, never silently replaced
            cpu = {"error": str(ex)}
    line = {
        "metric": METRIC,
        "value": mixed_qps,
        "unit": "quartets/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": msmx / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64+f32 (mixed)",
        "data": "synthetic",
        "config": workload_config(args.carbons),
        "system": {"nao": nao, "ncart": bas.ncart, "nprim": bas.nprim,
                   "parallelism": "replicas" if world > 1 else "single-gpu", "scf_iterations": len(scf.trace),
                   "scf_energy": E_scf, "scf_converged": bool(scf.converged), "scf_guess": "SAD",
                   "scf_seconds": t_scf, "scf_mixed": scf_mixed},
        # K over merged twins (shared s exponents computed once; ls.set_merge): the same K up to
        # quartets below thresp (dE_merged_vs_exact_Eh at fixed density); "exact" is the same
        # step over the reference's exact quartet set
        "merged_s_exponents": merge, "dE_merged_vs_exact_Eh": dE_merge if merge else 0.0, "exact": exact,
        # the same steps after one autotuning build (the headline keeps the default schedule)
        "autotuned": tuned,
        # quartets: the reference's quartet set of the step (its J and K screens over the
        # primitives as given); quartets_computed: what the merged build evaluates
        "quartets": q_ref, "quartets_ref_j": st_ref["j_quartets"], "quartets_ref_k": st_ref["k_quartets"],
        "fp64": {"ms_per_iter": ms64 / args.steps, "quartets_per_s": fp64_qps, "ms_k": msk64 / args.steps,
                 "quartets_computed": q64, "computed_per_s": q64 / (ms64 / args.steps * 1e-3),
                 "gpu_launches_per_step": launches_fp64 / max(args.steps, 1)},
        "mixed": {"ms_per_iter": msmx / args.steps, "quartets_per_s": mixed_qps, "ms_k": mskmx / args.steps,
                  "quartets_fp32": counts["mixed"]["quartets_fp32"], "quartets_computed": qmx,
                  "computed_per_s": qmx / (msmx / args.steps * 1e-3),
                  "speedup_vs_fp64": ms64 / msmx, "dE_vs_fp64_Eh": dE},
        "roofline": {"bound": "fp64", "kernel": "k_exchange (K build, FP64)", "achieved": achieved,
                     "peak": peak64, "unit": "TFLOP/s", "frac": achieved / peak64,
                     # DRAM bytes (read + write) of the FP64 K build's 81 launches of this workload,
                     # from one ncu capture (cold cache per launch: an upper bound)
                     "traffic": K_TRAFFIC_C40 if args.carbons == 40 else None,
                     "traffic_unit": "bytes per FP64 K build",
                     "traffic_source": "profiles/dram_jk_C40H82_ccpvdz.md",
                     "peak_source": "FP64 FMA microbenchmark run in bench.py (MEASURED_PEAKS.json has no FP64 figure)",
                     "fp32_peak": peak32,
                     # mixed run: the pipe-bound time of its K flops, sum_prec flops_prec / peak_prec,
                     # over the measured K time
                     "mixed_k_frac": ((counts["mixed"]["flops_k_fp64"] / (peak64 * 1e12) +
                                       counts["mixed"]["flops_k_fp32"] / (peak32 * 1e12)) /
                                      (mskmx / args.steps * 1e-3))},
        "e2e": {"value": e2e_qps, "unit": "quartets/s", "h2d_bytes_per_step": 2 * nao * nao * 8,
                "d2h_bytes_per_step": 2 * nao * nao * 8, "ms_per_step": e2e_ms / args.steps},
        "gpu_launches": int(launches_timed),
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))
    replicas.finish()
    return 0


def run_batched(args):
    """64 non-symmetric densities through one batched J+K step.

    32 H2O (seed 0) in 6-31G* (608 functions), Schwarz 1e-12; densities
    D_k = A_k B_k^T with A_k, B_k 608 x 10 seeded Gaussian factors made
    S-orthonormal (the shape of TDA/CIS trial vectors), symmetric pair list,
    D24symm off. Operators: bare Coulomb and erf-attenuated (omega = 0.3).
    Per operator and precision: one step = J and K for all 64 densities
    through the device entry points (one build: one kernel launch per class and
    precision pass serves all 64 densities), captured
    once as a CUDA graph and replayed; the direct (uncaptured) time is
    reported beside it. Mixed results are compared with FP64 elementwise."""
    rank, world, local = dist_info()
    import torch
    torch.cuda.set_device(local)
    import lightspeed_b200 as ls
    from lightspeed_b200.geometry import water_cluster
    thre = 1.0e-12
    mol = water_cluster(32, seed=0)
    bas = ls.Basis.from_gbs_file(mol, "6-31gs")
    res = ls.ResourceList.build()
    pl = ls.PairList.build_schwarz(bas, bas, True, thre)
    S = ls.IntBox.overlap(res, pl).np.copy()
    nao = bas.nao
    ndens, rank_k = 64, 10
    rng = np.random.default_rng(0)
    def s_orth(X):
        M = X.T @ S @ X
        mw, mU = np.linalg.eigh(M)
        return X @ ((mU / np.sqrt(mw)) @ mU.T)

    Ds = []
    for _ in range(ndens):
        A = s_orth(rng.standard_normal((nao, rank_k)))
        B = s_orth(rng.standard_normal((nao, rank_k)))
        Ds.append(A @ B.T)
    dev = torch.device("cuda", local)
    stream = torch.cuda.ExternalStream(ls.stream_handle(), device=dev)
    Dd = torch.tensor(np.stack(Ds), dtype=torch.float64, device=dev)
    Jd = torch.zeros_like(Dd)
    Kd = torch.zeros_like(Dd)
    dptr = [Dd[k].data_ptr() for k in range(ndens)]
    jptr = [Jd[k].data_ptr() for k in range(ndens)]
    kptr = [Kd[k].data_ptr() for k in range(ndens)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    if args.profile_step:
        # one mixed-precision step of the bare operator between profiler start and stop
        ew = ls.Ewald([1.0], [-1.0])
        ls.set_precision(ls.PREC_MIXED)
        for _ in range(max(args.warmup, 1)):
            ls.coulomb_device(ew, pl, pl, dptr, jptr, thre, THREDP)
            ls.exchange_device(ew, pl, pl, dptr, False, kptr, thre, THREDP)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        ls.coulomb_device(ew, pl, pl, dptr, jptr, thre, THREDP)
        ls.exchange_device(ew, pl, pl, dptr, False, kptr, thre, THREDP)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(json.dumps({"profile_step": True, "workload": "batched, 64 densities, mixed, bare operator"}))
        return 0
    results = {}
    ref = {}
    clocks = Clocks(local)
    clocks.start()
    for opname, (scales, omegas) in (("coulomb", ([1.0], [-1.0])), ("erf_omega0.3", ([1.0], [0.3]))):
        ew = ls.Ewald(scales, omegas)
        for prec, mode, thredp in (("fp64", ls.PREC_FP64, thre), ("mixed", ls.PREC_MIXED, THREDP)):
            ls.set_precision(mode)

            def step():
                ls.coulomb_device(ew, pl, pl, dptr, jptr, thre, thredp)
                ls.exchange_device(ew, pl, pl, dptr, False, kptr, thre, thredp)

            for _ in range(args.warmup):
                with torch.cuda.stream(stream):
                    Jd.zero_()
                    Kd.zero_()
                step()
            torch.cuda.synchronize()
            ls.reset_stats()
            with torch.cuda.stream(stream):
                Jd.zero_()
                Kd.zero_()
            step()
            torch.cuda.synchronize()
            st = ls.stats()
            if prec == "fp64":
                ref[opname] = (Jd.clone(), Kd.clone())
                err = None
            else:
                J64, K64 = ref[opname]
                err = {"max_abs_dJ": (Jd - J64).abs().max().item(), "max_abs_dK": (Kd - K64).abs().max().item()}
            ls.graph_begin()
            step()
            g = ls.graph_end()

            def timed(fn):
                tot = 0.0
                for _ in range(args.steps):
                    with torch.cuda.stream(stream):
                        flush.zero_()
                        Jd.zero_()
                        Kd.zero_()
                        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        e0.record(stream)
                        fn()
                        e1.record(stream)
                    e1.synchronize()
                    tot += e0.elapsed_time(e1)
                return tot / args.steps

            ms_graph = timed(g.launch)
            ms_direct = timed(step)
            del g
            ms_tuned = None
            if not args.no_tune and opname == "coulomb" and prec == "mixed":
                # the autotuner's value on the headline pair: tune once, time the direct
                # step, then put the default table back for the other operators
                table = ls.get_tune_table()
                ls.set_autotune(True)
                step()
                ls.set_autotune(False)
                torch.cuda.synchronize()
                ms_tuned = timed(step)
                ls.set_tune_table(table)
            q = st["j_quartets"] + st["k_quartets"]
            results["%s/%s" % (opname, prec)] = {
                "ms_per_step": ms_graph, "ms_per_step_direct": ms_direct,
                "ms_per_step_direct_autotuned": ms_tuned,
                # the engine's counters count each quartet once per density it serves
                "density_quartets": q,
                "quartets_fp32": st["quartets_fp32"],
                "density_quartets_per_s": q / (ms_graph * 1e-3),
                "ms_per_density": ms_graph / ndens, "error_vs_fp64": err,
                "gpu_launches_per_step": st["kernel_launches"]}
    torch.cuda.synchronize()
    clk = clocks.stop()
    if rank != 0:
        return 0
    head = results["coulomb/mixed"]
    line = {
        "metric": "batched J+K, 64 densities: ms per step and density-quartets/s (mixed vs FP64)",
        "value": head["density_quartets_per_s"], "unit": "density-quartets/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32 (mixed)", "data": "synthetic",
        "config": {"workload": "32 H2O (seed 0) / 6-31G*, 64 non-symmetric rank-10 densities, J+K",
                   "nao": nao, "thresp": thre, "thredp": THREDP, "graph": "one CUDA graph per step",
                   "l2": "flushed between steps (256 MiB write outside the timed events)"},
        "results": results, "gpu_launches": int(head["gpu_launches_per_step"] * args.steps), "clocks": clk}
    print(json.dumps(line))
    return 0


def run_guess(args):
    """Learned SCF guess against SAD on seeded water clusters (6-31G*, FP64 J/K).

    Training: converged densities (orbital gradient 1e-6, from SAD) of
    `--train-clusters` seeded clusters of 4-16 H2O with +-0.05 A bond and
    +-5 degree angle noise (seeds 0..), features and local-frame targets per
    atom pair, `--epochs` epochs of the BF16 network. Evaluation: held-out
    clusters of 20-24 H2O (seeds 100000..), each converged to 1e-8 from SAD
    and from the learned guess (SAD fallback on 1e-3 trace/idempotency
    error); wall time includes building the guess (fastest of two runs per
    cluster and arm). `value` = total SAD SCF
    wall time / total learned-guess SCF wall time."""
    rank, world, local = dist_info()
    import torch
    torch.cuda.set_device(local)
    import lightspeed_b200 as ls
    from lightspeed_b200 import guess as g
    from lightspeed_b200.sad import SAD
    if rank != 0:
        return 0
    ls.set_precision(ls.PREC_FP64)
    sad = SAD(ls, "6-31gs")
    rng = np.random.default_rng(0)
    train = [(int(rng.integers(4, 17)), s) for s in range(args.train_clusters)]
    test = [(int(rng.integers(20, 25)), 100000 + s) for s in range(args.test_clusters)]
    t0 = time.time()
    X, Y, W = g.training_set(ls, train, sad)
    t_data = time.time() - t0
    net = g.MLP(ls, seed=0)
    t0 = time.time()
    hist = net.fit(X, Y, W, epochs=args.epochs, batch=4096, lr=2e-3, norm=args.guess_norm)
    torch.cuda.synchronize()
    t_train = time.time() - t0
    # warm the SCF path once so neither arm pays first-call costs
    g.compare_guesses(ls, g.LearnedGuess(net, sad), [(test[0][0], test[0][1] + 50000)])
    rows = g.compare_guesses(ls, g.LearnedGuess(net, sad), test, repeats=2)
    t_sad = sum(r["sad"]["seconds"] for r in rows)
    t_mlp = sum(r["mlp"]["seconds"] for r in rows)
    line = {
        "metric": "SCF wall time, learned guess vs SAD (water clusters of 20-24 H2O, 6-31G*, to 1e-8)",
        "value": t_sad / t_mlp, "unit": "x (SAD time / learned-guess time)", "n_gpus": 1,
        "higher_is_better": True, "data": "synthetic", "dtype": "bf16 network, f64 SCF",
        "config": {"workload": "learned SCF guess", "train_clusters": len(train), "train_sizes": "4-16 H2O",
                   "test_clusters": len(test), "test_sizes": "20-24 H2O", "noise": "+-0.05 A, +-5 deg",
                   "train_pairs": int(X.shape[0]), "epochs": args.epochs, "network": "3 x 256 SiLU, bf16",
                   "target_scaling": args.guess_norm},
        "seconds_training_data": t_data, "seconds_training": t_train,
        "loss_first_epoch": hist[0], "loss_last_epoch": hist[-1],
        "sad": {"iterations_mean": float(np.mean([r["sad"]["iterations"] for r in rows])), "seconds": t_sad},
        "mlp": {"iterations_mean": float(np.mean([r["mlp"]["iterations"] for r in rows])), "seconds": t_mlp,
                "fallbacks": sum(r["mlp"]["source"] != "mlp" for r in rows)},
        "max_abs_dE_Eh": max(abs(r["dE"]) for r in rows),
        "all_converged": all(r["sad"]["converged"] and r["mlp"]["converged"] for r in rows),
        "rows": rows,
    }
    print(json.dumps(line))
    return 0


def run_grad(args):
    """J and K nuclear gradients (IntBox.coulombGrad / exchangeGrad, the
    reference's fully symmetric calls with D13 = D24 = D) of an alkane
    C_nH_2n+2 / cc-pVDZ (`--carbons`, default here 10) at its SAD density,
    Schwarz and thresp 1e-12, FP64. A step is the two calls through the host
    API (D in, G out, host arrays), timed on the wall clock around the
    synchronous calls; `value` = gradient evaluations (J+K) per second. The
    reference's CPU routines (oracle/_ref, all host cores) are timed on the
    same inputs once, and the two gradients compared elementwise."""
    rank, world, local = dist_info()
    import torch
    torch.cuda.set_device(local)
    import lightspeed_b200 as ls
    from lightspeed_b200.sad import SAD
    from oracle import ref
    if rank != 0:
        return 0
    ncarbon = args.carbons if args.carbons != 40 else 10
    mol, bas = workload(ls, ncarbon)
    thre = 1.0e-12
    res = ls.ResourceList.build()
    pl = ls.PairList.build_schwarz(bas, bas, True, thre)
    D = SAD(ls, "cc-pvdz").density(mol, bas)
    Dt = ls.Tensor.array(D)
    ew = ls.Ewald.coulomb()
    ls.set_precision(ls.PREC_FP64)

    def step():
        GJ = ls.IntBox.coulombGrad(res, ew, pl, Dt, Dt, thre, thre)
        GK = ls.IntBox.exchangeGrad(res, ew, pl, Dt, Dt, True, True, True, thre, thre)
        return GJ.np.copy(), GK.np.copy()

    for _ in range(args.warmup):
        step()
    tj, tk = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        GJ = ls.IntBox.coulombGrad(res, ew, pl, Dt, Dt, thre, thre)
        t1 = time.perf_counter()
        GK = ls.IntBox.exchangeGrad(res, ew, pl, Dt, Dt, True, True, True, thre, thre)
        t2 = time.perf_counter()
        tj.append(t1 - t0)
        tk.append(t2 - t1)
    GJ, GK = GJ.np.copy(), GK.np.copy()
    ms_j, ms_k = 1e3 * float(np.mean(tj)), 1e3 * float(np.mean(tk))
    cpu = None
    if ref.available() and not args.no_cpu_baseline:
        rb = ref.RefBasis(ref.prim_arrays(bas))
        rp = ref.RefPairs(rb, rb, True, thre)
        nthread = os.cpu_count() or 1
        t0 = time.perf_counter()
        RJ = ref.coulomb_grad(rp, D, None, thre, thre, nthread=nthread)
        t1 = time.perf_counter()
        RK = ref.exchange_grad(rp, D, None, True, True, thre, thre, nthread=nthread)
        t2 = time.perf_counter()
        cpu = {"kind": "reference", "cores": nthread, "cpu_model": cpu_model(), "ms_j": 1e3 * (t1 - t0),
               "ms_k": 1e3 * (t2 - t1), "max_abs_dGJ": float(np.max(np.abs(GJ - RJ))),
               "max_abs_dGK": float(np.max(np.abs(GK - RK))), "max_abs_GK": float(np.max(np.abs(RK)))}
    line = {
        "metric": "J+K nuclear gradient: ms per evaluation (FP64) and evaluations/s",
        "value": 1e3 / (ms_j + ms_k), "unit": "gradients/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_j + ms_k, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "C%dH%d/cc-pVDZ J+K nuclear gradient at the SAD density" % (ncarbon, 2 * ncarbon + 2),
                   "nao": bas.nao, "natom": mol.natom, "thresp": thre, "api": "host (D in, G out)"},
        "ms_j": ms_j, "ms_k": ms_k, "cpu_baseline": cpu,
    }
    print(json.dumps(line))
    return 0


def run_fshell(args):
    """Classes with f shells: a water cluster (`--waters`, default here 4, seed 0)
    in cc-pVTZ (spherical f on O, d on H), Schwarz and thresp 1e-12, a symmetric
    density of rank 5 per water (seeded normal columns). A step is one J+K build
    through the host API (D in, J and K out, host arrays) timed on the wall clock
    around the synchronous calls, in FP64 and in mixed precision (thredp 1e-6);
    the J+K nuclear gradients (FP64, the fully symmetric calls) are timed the same
    way. `value` = FP64 J+K builds per second. The reference's CPU routines
    (oracle/_ref, all host cores) run once on the same inputs, and the results are
    compared elementwise."""
    rank, world, local = dist_info()
    import torch
    torch.cuda.set_device(local)
    import lightspeed_b200 as ls
    from lightspeed_b200.geometry import water_cluster
    from oracle import ref
    if rank != 0:
        return 0
    nw = args.waters if args.waters != 16 else 4
    mol = water_cluster(nw, seed=0)
    bas = ls.Basis.from_gbs_file(mol, "cc-pvtz")
    thre = 1.0e-12
    res = ls.ResourceList.build()
    pl = ls.PairList.build_schwarz(bas, bas, True, thre)
    rng = np.random.default_rng(5)
    X = rng.standard_normal((bas.nao, 5 * nw)) / np.sqrt(bas.nao)
    D = X @ X.T
    Dt = ls.Tensor.array(D)
    ew = ls.Ewald.coulomb()

    def build(thredp):
        J = ls.IntBox.coulomb(res, ew, pl, pl, Dt, thre, thredp)
        K = ls.IntBox.exchange(res, ew, pl, pl, Dt, True, thre, thredp)
        return J.np.copy(), K.np.copy()

    def grads():
        GJ = ls.IntBox.coulombGrad(res, ew, pl, Dt, Dt, thre, thre)
        GK = ls.IntBox.exchangeGrad(res, ew, pl, Dt, Dt, True, True, True, thre, thre)
        return GJ.np.copy(), GK.np.copy()

    def timed(fn):
        for _ in range(args.warmup):
            out = fn()
        ts = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            out = fn()
            ts.append(time.perf_counter() - t0)
        return out, 1e3 * float(np.mean(ts))

    ls.set_precision(ls.PREC_FP64)
    (J, K), ms64 = timed(lambda: build(thre))
    # the K phase alone (FP64) against the FP64 FMA peak: K flops of one build / its time
    ls.reset_stats()
    ls.IntBox.exchange(res, ew, pl, pl, Dt, True, thre, thre)
    k_flops = ls.flops_split()["k_fp64"]
    _, ms_k64 = timed(lambda: ls.IntBox.exchange(res, ew, pl, pl, Dt, True, thre, thre).np.copy())
    peak64 = ls.fma_peak_tflops(True)
    ls.set_precision(ls.PREC_MIXED)
    (Jm, Km), msmx = timed(lambda: build(1e-6))
    ls.set_precision(ls.PREC_FP64)
    (GJ, GK), msg = timed(grads)
    cpu = None
    if ref.available() and not args.no_cpu_baseline:
        rb = ref.RefBasis(ref.prim_arrays(bas))
        rp = ref.RefPairs(rb, rb, True, thre)
        nthread = os.cpu_count() or 1
        t0 = time.perf_counter()
        RJ = ref.coulomb(rp, rp, D, thre, thre, nthread=nthread)
        RK = ref.exchange(rp, rp, D, True, thre, thre, nthread=nthread)
        t1 = time.perf_counter()
        RGJ = ref.coulomb_grad(rp, D, None, thre, thre, nthread=nthread)
        RGK = ref.exchange_grad(rp, D, None, True, True, thre, thre, nthread=nthread)
        t2 = time.perf_counter()
        cpu = {"kind": "reference", "cores": nthread, "cpu_model": cpu_model(), "ms_jk": 1e3 * (t1 - t0),
               "ms_grad": 1e3 * (t2 - t1), "max_abs_dJ": float(np.max(np.abs(J - RJ))),
               "max_abs_dK": float(np.max(np.abs(K - RK))), "max_abs_dJ_mixed": float(np.max(np.abs(Jm - RJ))),
               "max_abs_dK_mixed": float(np.max(np.abs(Km - RK))), "max_abs_dGJ": float(np.max(np.abs(GJ - RGJ))),
               "max_abs_dGK": float(np.max(np.abs(GK - RGK)))}
    line = {
        "metric": "J+K build with f shells: ms per build (FP64, mixed) and builds/s; J+K gradient ms",
        "value": 1e3 / ms64, "unit": "builds/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms64, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "%d H2O (seed 0) / cc-pVTZ J+K build and gradient" % nw, "nao": bas.nao,
                   "ncart": bas.ncart, "thresp": thre, "api": "host (D in, J/K or G out)"},
        "ms_mixed": msmx, "ms_grad": msg, "ms_k_fp64": ms_k64,
        "roofline": {"bound": "fp64", "kernel": "K build (FP64; f classes in k_exchange_warp)",
                     "achieved": k_flops / (ms_k64 * 1e-3) / 1e12, "peak": peak64, "unit": "TFLOP/s",
                     "frac": k_flops / (ms_k64 * 1e-3) / 1e12 / peak64, "traffic": None,
                     "timing": "host wall clock around the synchronous call (includes D in, K out)"},
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))
    return 0


def run_eri(args):
    """MO-basis integrals through J builds (IntBox.eriJ, the CASCI integrals):
    a `--waters` H2O cluster (seed 0) in 6-31G*, Schwarz 1e-12, one block of
    `--active` S-orthonormal orbitals (seeded) passed as all four coefficient
    tensors, so n(n+1)/2 J builds per call. A step is one IntBox.eriJ call
    through the host API (C in, I out, both host arrays), timed on the wall
    clock around the synchronous call; FP64 and mixed. `value` = J builds per
    second in FP64 (the faster mode here); the mixed integrals are compared
    with FP64 elementwise. Beside it, the reference's structure on the same
    engine: one host IntBox.coulomb call per (i, j) and a host contraction."""
    rank, world, local = dist_info()
    import torch
    torch.cuda.set_device(local)
    import lightspeed_b200 as ls
    from lightspeed_b200.geometry import water_cluster
    mol = water_cluster(args.waters, seed=0)
    bas = ls.Basis.from_gbs_file(mol, "6-31gs")
    res = ls.ResourceList.build()
    pl = ls.PairList.build_schwarz(bas, bas, True, 1.0e-12)
    S = ls.IntBox.overlap(res, pl).np.copy()
    X = np.random.default_rng(0).standard_normal((bas.nao, args.active))
    w, V = np.linalg.eigh(X.T @ S @ X)
    C = ls.Tensor.array(X @ V / np.sqrt(w))
    ew = ls.Ewald.coulomb()
    nbuild = args.active * (args.active + 1) // 2
    out = {}
    for name, prec in (("fp64", ls.PREC_FP64), ("mixed", ls.PREC_MIXED)):
        ls.set_precision(prec)
        for _ in range(args.warmup):
            ls.IntBox.eriJ(res, ew, pl, pl, C, C, C, C, THRE, THREDP)
        t = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            I = ls.IntBox.eriJ(res, ew, pl, pl, C, C, C, C, THRE, THREDP)
            t.append(time.perf_counter() - t0)
        out[name] = {"ms_per_call": 1e3 * float(np.mean(t)), "builds_per_s": nbuild / float(np.mean(t)),
                     "I": I.np.copy()}
    # the reference's structure on the same engine: one host J call per (i, j) and a host contraction
    ls.set_precision(ls.PREC_FP64)
    Cn = C.np
    t0 = time.perf_counter()
    for i in range(args.active):
        for j in range(i + 1):
            J = ls.IntBox.coulomb(res, ew, pl, pl, ls.Tensor.array(np.outer(Cn[:, i], Cn[:, j])), THRE, THREDP).np
            Cn.T @ J @ Cn
    out["fp64"]["host_loop_ms"] = 1e3 * (time.perf_counter() - t0)
    ls.set_precision(ls.PREC_MIXED)
    err = float(np.max(np.abs(out["mixed"]["I"] - out["fp64"]["I"])))
    for v in out.values():
        del v["I"]
    if rank == 0:
        print(json.dumps({
            "metric": "IntBox.eriJ J builds per second (CASCI active-space integrals)",
            "value": out["fp64"]["builds_per_s"], "unit": "J builds/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": out["fp64"]["ms_per_call"], "higher_is_better": True,
            "data": "synthetic", "dtype": "f64",
            "config": {"workload": "eriJ", "waters": args.waters, "basis": "6-31G*", "nao": bas.nao,
                       "active": args.active, "j_builds_per_call": nbuild, "thresp": THRE, "thredp": THREDP},
            "fp64": out["fp64"], "mixed": out["mixed"], "max_abs_dI_mixed_vs_fp64": err}))
    return 0


def run_many(args):
    """Many-molecule batch: `--molecules` seeded water clusters of 1-12 H2O
    (sizes from default_rng(0), cluster m from seed m), 6-31G*, FP64 J/K,
    each converged from SAD to an orbital gradient of 1e-8. The SCFs run in
    lockstep; per iteration the difference densities of all unconverged
    molecules go to the device in one copy, and their J and K builds run
    either (a) as a sequential per-molecule loop of device calls, or (b) as
    one CUDA graph holding every molecule's builds (captured once per active
    set, replayed while the set is unchanged), then J and K come back in one
    copy; (c) the same builds spread round-robin over 8 extra engine contexts
    (ls.Stream: own CUDA stream and scratch) so small molecules' kernels run
    concurrently; (d) as (c) with the SCF algebra itself batched on the GPU
    (scf_batched.BatchedRHF: molecules grouped by size, FP64 batched DIIS and
    eigensolver), so the densities never leave the device. Reported per mode: molecules/s over the whole run,
    quartets/s over the J/K phases (device events), and the wall time split.
    `value` is the best mode's molecules/s."""
    rank, world, local = dist_info()
    import torch
    torch.cuda.set_device(local)
    import lightspeed_b200 as ls
    from lightspeed_b200.geometry import water_cluster
    from lightspeed_b200.sad import SAD
    from lightspeed_b200.scf import RHF, SCFStepper
    if rank != 0:
        return 0
    ls.set_precision(ls.PREC_FP64)
    thre = 1.0e-12
    sizes = np.random.default_rng(0).integers(1, 13, size=args.molecules)
    sad = SAD(ls, "6-31gs")
    t0 = time.time()
    systems = []
    for m, n in enumerate(sizes):
        mol = water_cluster(int(n), seed=m)
        bas = ls.Basis.from_gbs_file(mol, "6-31gs")
        systems.append((mol, bas, RHF(ls, mol, bas, thre_pq=thre, thre_sp=thre, thre_dp=thre)))
    t_setup = time.time() - t0
    dev = torch.device("cuda", local)
    stream = torch.cuda.ExternalStream(ls.stream_handle(), device=dev)
    ew = ls.Ewald.coulomb()
    naos = [b.nao for _, b, _ in systems]
    offs = np.concatenate([[0], np.cumsum([n * n for n in naos])])
    D_dev = torch.zeros(int(offs[-1]), dtype=torch.float64, device=dev)
    JK_dev = torch.zeros(2, int(offs[-1]), dtype=torch.float64, device=dev)
    D_host = torch.zeros(int(offs[-1]), dtype=torch.float64).pin_memory()
    JK_host = torch.zeros(2, int(offs[-1]), dtype=torch.float64).pin_memory()
    ptr = lambda t, m: t.data_ptr() + 8 * int(offs[m])

    def builds(active):
        for m in active:
            pl = systems[m][2].pairs
            ls.coulomb_device(ew, pl, pl, [ptr(D_dev, m)], [ptr(JK_dev[0], m)], thre, thre)
            ls.exchange_device(ew, pl, pl, [ptr(D_dev, m)], True, [ptr(JK_dev[1], m)], thre, thre)

    # concurrent mode: molecules spread round-robin over extra engine contexts (own streams)
    nstream = 8
    extra = [ls.Stream() for _ in range(nstream)]
    xstreams = [torch.cuda.ExternalStream(x.stream_handle(), device=dev) for x in extra]

    def builds_concurrent(active):
        for k, m in enumerate(active):
            x = extra[k % nstream]
            pl = systems[m][2].pairs
            x.coulomb_device(ew, pl, pl, [ptr(D_dev, m)], [ptr(JK_dev[0], m)], thre, thre)
            x.exchange_device(ew, pl, pl, [ptr(D_dev, m)], True, [ptr(JK_dev[1], m)], thre, thre)

    results = {}
    energies = {}
    # (d) everything on the GPU: batched SCF algebra (scf_batched) on device tensors that the
    # concurrent contexts' builds read and write in place -- no per-iteration host copies
    from lightspeed_b200.scf_batched import BatchedRHF
    t_start = time.time()
    for x in extra:
        x.reset_stats()
    ls.reset_stats()
    bat = BatchedRHF(ls, [r for _, _, r in systems], dev)
    bat.set_guess([sad.density(mol, bas) for mol, bas, _ in systems])
    gpu_ms = 0.0
    cur = torch.cuda.current_stream(dev)
    while not bat.finished() and bat.iteration < 100:
        bat.prepare()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(cur)
        for xs in xstreams:
            xs.wait_event(e0)
        for k, (gi, b) in enumerate(bat.active()):
            dptr, jptr, kptr = bat.targets(gi, b)
            pl = systems[bat.groups[gi]["idx"][b]][2].pairs
            x = extra[k % nstream]
            x.coulomb_device(ew, pl, pl, [dptr], [jptr], thre, thre)
            x.exchange_device(ew, pl, pl, [dptr], True, [kptr], thre, thre)
        for xs in xstreams:
            cur.wait_stream(xs)
        e1.record(cur)
        bat.update(1.0e-8)
        e1.synchronize()
        gpu_ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    wall = time.time() - t_start
    stt = dict(ls.stats())
    for x in extra:
        for key, val in x.stats().items():
            stt[key] += val
    q = stt["j_quartets"] + stt["k_quartets"]
    energies["device"] = bat.energies()
    results["device"] = {"seconds": wall, "molecules_per_s": len(systems) / wall, "lockstep_iterations": bat.iteration,
                         "jk_gpu_seconds": gpu_ms * 1e-3, "quartets": q, "quartets_per_s": q / max(gpu_ms * 1e-3, 1e-12),
                         "converged": int(bat.converged().sum()), "gpu_launches": stt["kernel_launches"]}
    for mode in ("sequential", "graph", "streams"):
        steppers = [SCFStepper(r, sad.density(mol, bas), g_conv=1.0e-8) for mol, bas, r in systems]
        active = list(range(len(systems)))
        graph, graph_set = None, None
        t_start = time.time()
        gpu_ms, iters, q = 0.0, 0, 0
        ls.reset_stats()
        for x in extra:
            x.reset_stats()
        Dh = D_host.numpy()
        JKh = JK_host.numpy()
        while active and iters < 100:
            iters += 1
            for m in active:
                Dh[offs[m]:offs[m + 1]] = steppers[m].build_density().ravel()
            with torch.cuda.stream(stream):
                D_dev.copy_(D_host, non_blocking=True)
                JK_dev.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                if mode == "streams":
                    for xs in xstreams:          # the extra streams start after the copies
                        xs.wait_event(e0)
                    builds_concurrent(active)
                    for xs in xstreams:
                        stream.wait_stream(xs)
                    e1.record(stream)
                elif mode == "graph" and graph is not None and graph_set == active:
                    graph.launch()
                    e1.record(stream)
                else:
                    builds(active)
                    e1.record(stream)
                    if mode == "graph":
                        # a new active set: these builds ran directly; capture them for the next iterations
                        graph = None
                        ls.graph_begin()
                        builds(active)
                        graph = ls.graph_end()
                        graph_set = list(active)
                JK_host.copy_(JK_dev, non_blocking=True)
            stream.synchronize()
            gpu_ms += e0.elapsed_time(e1)
            nxt = []
            for m in active:
                n = naos[m]
                dJ = JKh[0, offs[m]:offs[m + 1]].reshape(n, n)
                dK = JKh[1, offs[m]:offs[m + 1]].reshape(n, n)
                if not steppers[m].update(dJ.copy(), dK.copy()):
                    nxt.append(m)
            active = nxt
        for st in steppers:
            st.finish()
        wall = time.time() - t_start
        stt = dict(ls.stats())
        for x in extra:                    # the extra contexts keep their own counters
            for key, val in x.stats().items():
                stt[key] += val
        q = stt["j_quartets"] + stt["k_quartets"]
        energies[mode] = np.array([r.E for _, _, r in systems])
        results[mode] = {"seconds": wall, "molecules_per_s": len(systems) / wall, "lockstep_iterations": iters,
                         "jk_gpu_seconds": gpu_ms * 1e-3, "quartets": q,
                         "quartets_per_s": q / max(gpu_ms * 1e-3, 1e-12),
                         "converged": int(sum(st.converged for st in steppers)),
                         "gpu_launches": stt["kernel_launches"]}
        del graph
    line = {
        "metric": "many-molecule batch: molecules/s and quartets/s; one CUDA graph per SCF iteration, 8 "
                  "concurrent engine streams, or a GPU-resident batched SCF, vs a sequential per-molecule loop",
        "value": max(r["molecules_per_s"] for r in results.values()), "unit": "molecules/s", "n_gpus": 1,
        "higher_is_better": True, "data": "synthetic", "dtype": "f64",
        "config": {"workload": "%d water clusters of 1-12 H2O (sizes from seed 0, cluster m from seed m), 6-31G*, "
                               "RHF from SAD to 1e-8" % len(systems), "thresp": thre,
                   "total_functions": int(sum(naos)), "setup_seconds": t_setup},
        "sequential": results["sequential"], "graph": results["graph"], "streams": results["streams"],
        "device": results["device"],
        "speedup_device_vs_sequential": results["sequential"]["seconds"] / results["device"]["seconds"],
        "max_abs_dE_device_vs_sequential": float(np.max(np.abs(energies["device"] - energies["sequential"]))),
        "speedup_graph_vs_sequential": results["sequential"]["seconds"] / results["graph"]["seconds"],
        "speedup_streams_vs_sequential": results["sequential"]["seconds"] / results["streams"]["seconds"],
        "max_abs_dE_graph_vs_sequential": float(np.max(np.abs(energies["graph"] - energies["sequential"]))),
        "max_abs_dE_streams_vs_sequential": float(np.max(np.abs(energies["streams"] - energies["sequential"]))),
    }
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "guess":
        return run_guess(args)
    if args.workload == "many":
        return run_many(args)
    if args.workload == "eri":
        return run_eri(args)
    if args.workload == "grad":
        return run_grad(args)
    if args.workload == "fshell":
        return run_fshell(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
