"""J+K benchmark of the B200 engine on the C40H82 / cc-pVDZ workload.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one full J + K build (Coulomb operator, thresp = thre_pq = 1e-14,
mixed-precision cutoff thredp = 1e-5) on the converged RHF density of all-trans
C40H82 in cc-pVDZ (970 pure / 1010 Cartesian functions, 1290 primitive
shells). `value` is quartets/s with D, J and K resident in HBM (device entry
points); `e2e` is the same metric through the public host API
(ls.IntBox.coulomb / exchange on host tensors: the H2D copy of D and the D2H
copies of J and K are inside the timed region). L2 is flushed between steps
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
SAMPLE_CARBONS = 8        # CPU baseline sample: C8H18 / cc-pVDZ, full J+K


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--carbons", type=int, default=40)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scf-maxiter", type=int, default=60)
    ap.add_argument("--profile-step", action="store_true",
                    help="after set-up and warm-up, run one FP64 J+K step between cudaProfilerStart/Stop "
                         "(for ncu --profile-from-start off) and exit")
    return ap.parse_args()


def dist_info():
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
        self.path = os.path.join(ROOT, "gpurun_out" if os.path.isdir(os.path.join(ROOT, "gpurun_out")) else "",
                                 ".clocks_%d.csv" % os.getpid())

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


def cpu_sample():
    """Bounded CPU sample of the workload: C8H18 / cc-pVDZ (all-trans, same
    thresholds) with its core-Hamiltonian density, built from the reference
    CPU IntBox alone (S, T, V) so the reference arm runs no code of ours;
    quartets are counted by the oracle's shared counting routine."""
    import lightspeed_b200 as ls
    from oracle import port, ref
    mol, bas = workload(ls, SAMPLE_CARBONS)
    rb = ref.RefBasis(ref.prim_arrays(bas))
    rp = ref.RefPairs(rb, rb, True, THRE)
    S = ref.overlap(rp)
    H = ref.kinetic(rp) + ref.potential(rp, mol.xyzZ)
    s, U = np.linalg.eigh(S)
    X = U / np.sqrt(s)
    e, C = np.linalg.eigh(X.T @ H @ X)
    nocc = int(round(mol.nuclear_charge)) // 2
    Cocc = (X @ C)[:, :nocc]
    D = Cocc @ Cocc.T
    pb = port.Basis(bas.primitives)
    ppl = port.Pairs(pb, pb, True, THRE)
    nj, nk = port.count_quartets(ppl, ppl, D, D, True, THRE)
    desc = ("C%dH%d/cc-pVDZ (%d bf) full J+K, FP64, thresp 1e-14, core-Hamiltonian density; "
            "%.4g quartets per J+K" % (SAMPLE_CARBONS, 2 * SAMPLE_CARBONS + 2, bas.nao, nj + nk))
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
    dt = time_reference(rp, D, nthread)
    return {"value": nq / dt, "unit": "quartets/s", "cores": nthread, "kind": "reference",
            "sample": desc + "; %.2f s" % dt, "seconds": dt}


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
    from oracle import ref as _r
    for _ in range(args.warmup):
        _r.coulomb(rp, rp, D, THRE, THRE, nthread=nthread)
    times = [time_reference(rp, D, nthread) for _ in range(args.steps)]
    T = float(np.sum(times))
    v = nq * args.steps / T
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "quartets/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * T / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "C40H82/cc-pVDZ J+K, timed on a bounded sample", "sample": desc},
        "cpu_baseline": {"value": v, "unit": "quartets/s", "cores": nthread, "kind": "reference",
                         "sample": desc},
        "e2e": {"value": v, "unit": "quartets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


def run_ours(args):
    rank, world, local = dist_info()
    import torch
    torch.cuda.set_device(local)
    os.environ.setdefault("LSJK_DEVICE", str(local))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    import lightspeed_b200 as ls
    from lightspeed_b200.scf import RHF
    mol, bas = workload(ls, args.carbons)
    # converged density (FP64 J/K), the state an SCF iteration sees
    ls.set_precision(ls.PREC_FP64)
    t0 = time.time()
    scf = RHF(ls, mol, bas, thre_pq=THRE, thre_sp=THRE, thre_dp=THRE)
    E_scf = scf.compute(maxiter=args.scf_maxiter, g_conv=1e-5)
    t_scf = time.time() - t0
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

    # warm-up in both modes
    for mode in (ls.PREC_FP64, ls.PREC_MIXED):
        ls.set_precision(mode)
        for _ in range(args.warmup):
            step(THREDP)
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
    # quartet/flop counts of one step in each mode
    counts = {}
    for name, mode in (("fp64", ls.PREC_FP64), ("mixed", ls.PREC_MIXED)):
        ls.set_precision(mode)
        ls.reset_stats()
        step(THREDP)
        torch.cuda.synchronize()
        counts[name] = ls.stats()
    # energies at the converged density: E(D) with FP64 vs mixed J/K
    energies = {}
    for name, mode in (("fp64", ls.PREC_FP64), ("mixed", ls.PREC_MIXED)):
        ls.set_precision(mode)
        J = ls.IntBox.coulomb(res, ew, pl, pl, ls.Tensor.array(D), THRE, THREDP).np
        K = ls.IntBox.exchange(res, ew, pl, pl, ls.Tensor.array(D), True, THRE, THREDP).np
        energies[name] = scf.energy(D, J, K)[0]
    dE = energies["mixed"] - energies["fp64"]

    # ---- timed region -------------------------------------------------------
    clocks = Clocks(local)
    clocks.start()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ls.stats()["kernel_launches"]
    ms64, msk64 = timed(ls.PREC_FP64, THREDP, args.steps)
    launches_fp64 = ls.stats()["kernel_launches"] - launches0
    msmx, mskmx = timed(ls.PREC_MIXED, THREDP, args.steps)
    torch.cuda.synchronize()
    launches_timed = ls.stats()["kernel_launches"] - launches0
    # e2e through the public host API (H2D of D, D2H of J and K inside)
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
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()

    def agg(x):
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([x], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return x

    ms64, msk64, msmx, mskmx, e2e_ms = (agg(v) for v in (ms64, msk64, msmx, mskmx, e2e_ms))
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return 0
    q64 = counts["fp64"]["j_quartets"] + counts["fp64"]["k_quartets"]
    qmx = counts["mixed"]["j_quartets"] + counts["mixed"]["k_quartets"]
    fp64_qps = world * q64 * args.steps / (ms64 * 1e-3)
    mixed_qps = world * qmx * args.steps / (msmx * 1e-3)
    e2e_qps = world * qmx * args.steps / (e2e_ms * 1e-3)
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
        "config": {"workload": "C%dH%d/cc-pVDZ full J+K build at the converged RHF density" % (
            args.carbons, 2 * args.carbons + 2), "nao": nao, "ncart": bas.ncart, "nprim": bas.nprim,
            "thre_pq": THRE, "thresp": THRE, "thredp": THREDP, "operator": "1/r",
            "l2": "flushed between steps (256 MiB write outside the timed events)",
            "parallelism": "replicas" if world > 1 else "single-gpu", "scf_iterations": len(scf.trace),
            "scf_energy": E_scf, "scf_seconds": t_scf},
        "fp64": {"ms_per_iter": ms64 / args.steps, "quartets_per_s": fp64_qps, "ms_k": msk64 / args.steps,
                 "quartets": q64, "gpu_launches_per_step": launches_fp64 / max(args.steps, 1)},
        "mixed": {"ms_per_iter": msmx / args.steps, "quartets_per_s": mixed_qps, "ms_k": mskmx / args.steps,
                  "quartets_fp32": counts["mixed"]["quartets_fp32"], "quartets": qmx,
                  "speedup_vs_fp64": ms64 / msmx, "dE_vs_fp64_Eh": dE},
        "roofline": {"bound": "fp64", "kernel": "k_exchange (K build, FP64)", "achieved": achieved,
                     "peak": peak64, "unit": "TFLOP/s", "frac": achieved / peak64, "traffic": None,
                     "peak_source": "FP64 FMA microbenchmark run in bench.py (MEASURED_PEAKS.json has no FP64 figure)",
                     "fp32_peak": peak32},
        "e2e": {"value": e2e_qps, "unit": "quartets/s", "h2d_bytes_per_step": nao * nao * 8,
                "d2h_bytes_per_step": 2 * nao * nao * 8, "ms_per_step": e2e_ms / args.steps},
        "gpu_launches": int(launches_timed),
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
