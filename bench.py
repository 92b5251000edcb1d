"""Benchmark of the lapw1 H/S setup (HAMILT + HNS [+ HORB]) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--prec fp64|split]
                    [--impl ours|reference]

One step = the full calkpt.F:153-185 setup of one k-point per GPU.  At one
GPU the workload is the 40-atom 2x2x2 ABO3 supercell (RKmax 7, ~4950 basis
functions, one LO per atom for l<=2, one general k).  With N GPUs each rank
sets up its own k-point of the same cell (k-points are independent: weak
scaling, no collective on the data path).  Prints ONE JSON line (rank 0).
The default arithmetic is the split-precision path (5 int8 slices for the
spherical part, 4 for HNS; the
plain FP64 GPU path on the same k-point is timed beside it in
`fp64_path`, with the split path's per-matrix error against it), after the
autotuner has picked the tile/schedule parameters (untimed).  `batch` is a
captured graph of 16 c2 k-points per GPU.

`value` is ms per k-point of the whole job with inputs resident in HBM
(device timed, CUDA events on the library's stream, max over ranks).
`e2e` is the same metric through the host C-ABI entry point lapw1gpu_setup
(inputs from host memory, HS/HSDIAG copied back into pinned host memory).
The reference arm (--impl reference) times the CPU restatement of the
reference algorithm (the oracle: no Fortran compiler exists here to build
the reference itself) on all host cores over a bounded sample of the same
k-point and reports the extrapolated ms per k-point.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "lapw1 H+S setup ms/k-point"
UNIT = "ms/k-point"


def _env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.rows and time.time() - t0 < 5.0:  # sampling is live before timing starts
                time.sleep(0.02)
            self.rows.clear()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except Exception:
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def fp64_peak_tflops(torch, device):
    """Measured FP64 reference: cuBLAS DGEMM 8192^3 (torch.matmul float64), best of 5."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device=device)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=device)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2 * 8192 ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def int8_peak_tops(torch, device):
    """Measured dense int8 reference: cuBLAS int8 GEMM 8192^3 (torch._int_mm,
    int32 accumulate), best of 5; None when the library has no int8 path."""
    try:
        a = torch.randint(-64, 64, (8192, 8192), dtype=torch.int8, device=device)
        b = torch.randint(-64, 64, (8192, 8192), dtype=torch.int8, device=device)
        for _ in range(2):
            torch._int_mm(a, b)
        torch.cuda.synchronize()
        best = 0.0
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = max(best, 2 * 8192 ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
        del a, b
        torch.cuda.empty_cache()
        return best
    except Exception:
        return None


def baseline_def_flops(p):
    """The benchmark definition's work formula F = sum_atoms (16 N^2 (lmax+1)^2 + 8 N^2 (lmax_ns+1)^2):
    the flops of the A^H T A form the benchmark definition counts."""
    n = p.n
    return p.ndf * (16.0 * n * n * p.ltop ** 2 + 8.0 * n * n * (p.lnsmax + 1) ** 2)


def problem_input_bytes(p):
    cp = p.to_c()
    return int(sum(a.nbytes for a in cp._keep))


def _cpu_sample(p, frac):
    """The oracle over a fraction `frac` of one k-point's work: HAMILT over
    the last plane-wave columns worth `frac` of its work (column I of HAMILT
    costs ~I) and HNS for round(frac * NDF) atoms (each atom costs the
    same).  Returns (extrapolated ms per k-point, description, seconds)."""
    from oracle import oracle as O
    nv = p.nv
    c0 = max(1, int(nv * math.sqrt(1.0 - frac)))
    t = time.perf_counter()
    O.hamilt_sample(p, c0, nv)
    t_h = time.perf_counter() - t
    frac_h = (nv * (nv + 1) / 2 - (c0 - 1) * c0 / 2) / (nv * (nv + 1) / 2)
    na = max(1, min(p.ndf, int(round(frac * p.ndf))))
    t = time.perf_counter()
    O.hns_sample(p, 1, na)
    t_ns = time.perf_counter() - t
    est_s = t_h / frac_h + t_ns * p.ndf / na
    sample = (f"HAMILT PW columns {c0}..{nv} of {nv} ({100 * frac_h:.1f}% of its work) + "
              f"HNS atoms 1..{na} of {p.ndf}; extrapolated to one k-point")
    return est_s * 1e3, sample, t_h + t_ns


def cpu_reference(p, budget_s=8.0):
    """Bounded CPU sample of the reference algorithm (the oracle, OpenMP on
    all host cores) sized to about `budget_s` seconds: a 2% calibration
    sample estimates the full k-point, then a sample of budget_s worth (the
    whole k-point when it fits) is timed."""
    est_ms, _, _ = _cpu_sample(p, 0.02)
    frac = min(1.0, max(0.02, budget_s / (est_ms * 1e-3)))
    return _cpu_sample(p, frac)


def run_reference(args):
    rank, world, _ = _env_rank()
    if rank != 0:
        return 0
    from hack_wein2k_b200 import synth
    p = synth.config("c1")[0]
    cores = os.cpu_count()
    vals = []
    sample = ""
    budget = min(8.0, max(0.5, 120.0 / (args.warmup + args.steps)))  # whole run within a few minutes
    for i in range(args.warmup + args.steps):
        v, sample, _ = cpu_reference(p, budget)
        if i >= args.warmup:
            vals.append(v)
    val = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": val, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": "c1: 2x2x2 ABO3 supercell a=14.8 bohr, 40 atoms, RKmax 7, lmax 10, "
                               "lmax_ns 4, LO l<=2, one general k", "n": p.n, "nv": p.nv, "nlo": p.nlo,
                   "impl": "CPU restatement of HAMILT/HNS (oracle port), OpenMP all cores"},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _timed_loop(torch, stream, fn, steps):
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def _rel_err(torch, a, b, n):
    """per-matrix max relative error of packed HS a against b ([col][row][2])"""
    ca = torch.view_as_complex(a).transpose(0, 1)  # [row][col]
    cb = torch.view_as_complex(b).transpose(0, 1)
    low = torch.tril(torch.ones(n, n, dtype=torch.bool, device=a.device))
    out = {}
    for name, mask in (("H", low), ("S", ~low)):
        d = ((ca - cb).abs() * mask).max().item()
        m = ((cb.abs()) * mask).max().item()
        out[name] = d / m if m > 0 else 0.0
    return out


def hundred_atoms(args):
    """The 100-atom configurations: c4 (16 k-points, RKmax 8, N ~ 12700) as
    one captured batch, split precision (spherical/HNS slices) against the
    plain FP64 GPU path, plus the adjoint forces of 400 bands (c3 for
    accuracy, c4 k-point 0 for time).  One JSON line, rank 0 only."""
    import torch
    from hack_wein2k_b200 import forces as FO
    from hack_wein2k_b200 import lapw1gpu, synth
    from hack_wein2k_b200.seclr import hermitian_from_packed_device, solve
    rank, world, local = _env_rank()
    if rank != 0:
        return 0
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ctx = lapw1gpu.Context(local)
    s_sph, s_hns = args.slices, args.slices_hns

    def use(prec):
        if prec == "fp64":
            ctx.set_precision(lapw1gpu.PREC_FP64)
        else:
            ctx.set_precision(lapw1gpu.PREC_SPLIT, s_sph)
            ctx.set_slices(s_sph, s_hns)

    def window_err(w, w0, lo=-10.0, hi=10.0):
        win = (w0 > lo) & (w0 < hi)
        return float(np.abs(w - w0)[win].max()) if win.any() else None

    out = {"metric": "c4 k-batched setup ms/k-point, split vs plain FP64 GPU; c3/c4 adjoint forces",
           "unit": "ms/k-point", "higher_is_better": False, "data": "synthetic (seeded)",
           "slices": [s_sph, s_hns]}
    # ---- c4 batch ----
    ps = synth.config("c4")
    hs = [torch.empty((q.n, q.n), dtype=torch.complex128, device=dev) for q in ps]
    hd = [torch.empty(q.n, dtype=torch.complex128, device=dev) for q in ps]
    res = {}
    for prec in ("fp64", "split"):
        use(prec)
        kps = [ctx.upload(q) for q in ps]
        ctx.autotune(kps[0], hs[0].data_ptr(), ps[0].n, hd[0].data_ptr())
        a = (kps, [t.data_ptr() for t in hs], [q.n for q in ps], [t.data_ptr() for t in hd])
        ctx.setup_batch(*a)
        ms = min(ctx.setup_batch(*a)["ms_total"] for _ in range(2))
        res[prec] = {"ms_per_batch": ms, "ms_per_kpoint": ms / len(ps)}
        if prec == "fp64":
            ref, refd = hs[0].clone(), hd[0].clone()
        else:
            err = {}
            low = torch.tril(torch.ones(ps[0].n, ps[0].n, dtype=torch.bool, device=dev))
            a0, b0 = hs[0].transpose(0, 1), ref.transpose(0, 1)  # [row][col]
            for name, m in (("H", low), ("S", ~low)):
                err[name] = ((a0 - b0).abs() * m).max().item() / ((b0.abs() * m).max().item())
            res[prec]["rel_error_vs_fp64_k0"] = err
        for k in kps:
            k.free()
    out["c4"] = {"workload": f"c4: 100-atom cell 20^3 bohr, RKmax 8, 16 k-points, N {min(q.n for q in ps)}.."
                             f"{max(q.n for q in ps)}, one CUDA graph per batch", **res,
                 "setup_speedup": res["fp64"]["ms_per_kpoint"] / res["split"]["ms_per_kpoint"]}
    # ---- c4 k-point 0: forces of 400 bands (eigenvectors of the split
    # setup), timed in each precision: FP64 (ZHERKX density matrices, ZGEMM
    # HNS projection) and split (both as int8 slice products); the spherical
    # pair sums are FP64 in both ----
    p4 = ps[0]
    use("split")
    kp = ctx.upload(p4)
    kp.run(hs[0].data_ptr(), p4.n, hd[0].data_ptr(), stats=True)
    H, S = hermitian_from_packed_device(hs[0], hd[0])
    del hs, hd
    torch.cuda.empty_cache()
    w, X = solve(H, S, nmax=400)
    del H, S
    occ = torch.ones(400, dtype=torch.float64, device=dev)
    f_ms = {}
    for prec in ("fp64", "split"):
        use(prec)
        FO.gradient(ctx, kp, X, occ, w)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        FO.gradient(ctx, kp, X, occ, w)
        e1.record()
        torch.cuda.synchronize()
        f_ms[prec] = e0.elapsed_time(e1)
    kp.free()
    del X
    torch.cuda.empty_cache()
    out["c4"]["forces_ms_per_kpoint_400_bands"] = f_ms
    out["c4"]["setup_plus_forces_speedup"] = ((res["fp64"]["ms_per_kpoint"] + f_ms["fp64"]) /
                                             (res["split"]["ms_per_kpoint"] + f_ms["split"]))
    # ---- c3: accuracy of the split path (eigenvalues, forces) ----
    p3 = synth.config("c3")[0]
    acc = {}
    for prec in ("fp64", "split"):
        use(prec)
        kp = ctx.upload(p3)
        h3 = torch.zeros((p3.n, p3.n), dtype=torch.complex128, device=dev)
        d3 = torch.zeros(p3.n, dtype=torch.complex128, device=dev)
        torch.cuda.synchronize()
        st = kp.run(h3.data_ptr(), p3.n, d3.data_ptr(), stats=True)
        H, S = hermitian_from_packed_device(h3, d3)
        w, X = solve(H, S, nmax=400)
        g = FO.gradient(ctx, kp, X, torch.ones(400, dtype=torch.float64, device=dev), w)
        acc[prec] = (w.cpu().numpy(), FO.cartesian_forces(p3, g.cpu().numpy()), st["ms_total"])
        kp.free()
        del H, S, X, h3, d3
    out["c3"] = {"workload": "c3: 100-atom cell 20^3 bohr, RKmax 6, N %d, 400 bands" % p3.n,
                 "eig_err_window_ry": window_err(acc["split"][0], acc["fp64"][0]),
                 "force_err_ry_bohr": float(np.abs(acc["split"][1] - acc["fp64"][1]).max()),
                 "max_force_ry_bohr": float(np.abs(acc["fp64"][1]).max())}
    print(json.dumps(out), flush=True)
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--prec", choices=["fp64", "split"], default="split")
    ap.add_argument("--slices", type=int, default=5)
    ap.add_argument("--slices-hns", type=int, default=4,
                    help="int8 slices of HNS (the non-spherical part is 1-2 orders smaller than the spherical one)")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the FP64 comparator and the k-batch line")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the library's default tuning (profiling runs: timings under a profiler mislead the autotuner)")
    ap.add_argument("--hundred-atoms", action="store_true",
                    help="instead: the 100-atom c4 batch (split vs FP64) and c3/c4 adjoint forces, one JSON line")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.hundred_atoms:
        return hundred_atoms(args)

    import torch
    from hack_wein2k_b200 import lapw1gpu, synth

    rank, world, local = _env_rank()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)

    # workload: c1 at one GPU; rank r of N takes k-point r of the same cell
    if world == 1:
        p = synth.config("c1")[0]
        workload = "c1: 2x2x2 ABO3 supercell a=14.8 bohr, 40 atoms, RKmax 7, lmax 10, lmax_ns 4, LO l<=2, one general k"
    else:
        p = synth.config("c2", nk=max(world, 1))[rank]
        workload = "c2 k-shard: 2x2x2 ABO3 supercell, one seeded wedge k-point per rank"

    prec = lapw1gpu.PREC_SPLIT if args.prec == "split" else lapw1gpu.PREC_FP64
    ctx = lapw1gpu.Context(local, prec=prec, slices=args.slices)
    slices_hns = args.slices_hns if args.slices_hns else args.slices
    if prec == lapw1gpu.PREC_SPLIT:
        ctx.set_slices(args.slices, slices_hns)
    stream = torch.cuda.ExternalStream(ctx.stream_handle, device=device)
    kp = ctx.upload(p)
    n = p.n
    d_hs = torch.empty((n, n, 2), dtype=torch.float64, device=device)  # column-major view: [col][row]
    d_hd = torch.empty((n, 2), dtype=torch.float64, device=device)
    torch.cuda.synchronize()
    if args.no_autotune:
        tuning = ctx.tuning()
    else:
        tuning = ctx.autotune(kp, d_hs.data_ptr(), n, d_hd.data_ptr())  # untimed: picks tile/schedule parameters

    def step(stats=True):
        return kp.run(d_hs.data_ptr(), n, d_hd.data_ptr(), stages=7, stats=stats)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    with ClockSampler(local) as clk:
        # queued on the library's stream, no host sync between k-points
        ms = _timed_loop(torch, stream, lambda: step(stats=False), args.steps)
    if dist is not None:
        dist.barrier()
        t = torch.tensor([ms], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    value = ms_step / world  # ms per k-point of the whole job (world k-points per step)

    # ---- per-stage breakdown (separate pass, synchronised per k-point) ----
    stage_ms = {}
    n_stage = max(1, min(args.steps, 10))
    per_step_launches = 0
    for _ in range(n_stage):
        st = step(stats=True)
        for k, v in st.items():
            stage_ms[k] = stage_ms.get(k, 0.0) + v
        per_step_launches = int(st["kernel_launches"])
    launches = per_step_launches * args.steps

    # ---- e2e through the host entry point ----
    hs_h = torch.empty((n, n, 2), dtype=torch.float64).pin_memory()
    hd_h = torch.empty((n, 2), dtype=torch.float64).pin_memory()
    hs_np = hs_h.numpy().view(np.complex128).reshape(n, n).T  # Fortran-order view of [col][row]
    hd_np = hd_h.numpy().view(np.complex128).reshape(n)
    for _ in range(max(1, args.warmup)):
        ctx.setup(p, hs=hs_np, hsdiag=hd_np)
    if dist is not None:
        dist.barrier()
    e2e_steps = max(1, min(args.steps, 5))
    e2e_ms = _timed_loop(torch, stream, lambda: ctx.setup(p, hs=hs_np, hsdiag=hd_np), e2e_steps)
    if dist is not None:
        t = torch.tensor([e2e_ms], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_val = e2e_ms / e2e_steps / world
    h2d = problem_input_bytes(p)
    d2h = n * n * 16 + n * 16

    # ---- the plain FP64 GPU path on the same k-point, and the split error ----
    fp64_cmp = None
    if args.prec == "split" and not args.no_extras:
        cf = lapw1gpu.Context(local, prec=lapw1gpu.PREC_FP64)
        sf = torch.cuda.ExternalStream(cf.stream_handle, device=device)
        kf = cf.upload(p)
        f_hs = torch.empty_like(d_hs)
        f_hd = torch.empty_like(d_hd)
        tf = cf.autotune(kf, f_hs.data_ptr(), n, f_hd.data_ptr())
        for _ in range(2):
            kf.run(f_hs.data_ptr(), n, f_hd.data_ptr(), stats=True)
        nf = max(3, min(args.steps, 20))
        ms_f = _timed_loop(torch, sf, lambda: kf.run(f_hs.data_ptr(), n, f_hd.data_ptr(), stats=False), nf) / nf
        stf = kf.run(f_hs.data_ptr(), n, f_hd.data_ptr(), stats=True)
        step(stats=True)
        err = _rel_err(torch, d_hs, f_hs, n)
        fp64_cmp = {"ms_per_kpoint": ms_f, "speedup_split_over_fp64": ms_f / ms_step,
                    "stage_ms": {k: v for k, v in stf.items() if k.startswith("ms_")},
                    "split_rel_error_vs_fp64": err, "tuning": tf}
        kf.free()
        cf.close()
        del f_hs, f_hd

    # ---- one captured batch of c2 k-points (uneven N) per rank ----
    batch = None
    if not args.no_extras:
        nkb = 16
        probs = synth.config("c2", nk=nkb * world)[rank::world][:nkb]
        kps = [ctx.upload(q) for q in probs]
        bh = [torch.empty((q.n, q.n, 2), dtype=torch.float64, device=device) for q in probs]
        bd = [torch.empty((q.n, 2), dtype=torch.float64, device=device) for q in probs]
        args_b = (kps, [t.data_ptr() for t in bh], [q.n for q in probs], [t.data_ptr() for t in bd])
        best = None
        for sets in (1, 2, 3):  # the batch schedule is tuned too: concurrent k-point chains
            ctx.set_tuning(batch_sets=sets)
            ctx.setup_batch(*args_b)  # capture
            t_b = min(ctx.setup_batch(*args_b)["ms_total"] for _ in range(2))
            if best is None or t_b < best[1]:
                best = (sets, t_b)
        ctx.set_tuning(batch_sets=best[0])
        reps = 3
        ms_b = min(ctx.setup_batch(*args_b)["ms_total"] for _ in range(reps))
        if dist is not None:
            t = torch.tensor([ms_b], device=device, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_b = float(t.item())
        batch = {"workload": f"c2: {nkb} seeded wedge k-points per GPU of the 40-atom cell, N {min(q.n for q in probs)}"
                             f"..{max(q.n for q in probs)}, one CUDA graph launch",
                 "ms_per_batch": ms_b, "ms_per_kpoint": ms_b / nkb / 1.0, "kpoints_per_s": nkb * world / (ms_b * 1e-3),
                 "batch_sets": best[0]}
        for k in kps:
            k.free()
        del bh, bd

    # ---- roofline of the dominant kernel ----
    clocks = clk.summary()
    avg = {k: v / n_stage for k, v in stage_ms.items()}
    nsl2 = (p.lnsmax + 1) ** 2
    pairs = p.nv * (p.nv + 1) / 2.0
    # spherical: per pair, 6 FMA per (atom type, l), 4 per equivalent atom's
    # phase product, 4 per type to add PHASE * t into S and H
    f_sph = 2.0 * (6.0 * p.ltop * p.nat + 4.0 * p.ndf + 4.0 * p.nat) * pairs
    # HNS: complex rank-K update of the lower triangle, K = 2 NDF (lmax_ns+1)^2
    K_hns = 2.0 * p.ndf * nsl2
    f_hns = 8.0 * K_hns * (n * (n + 1) / 2.0)
    split = args.prec == "split"
    sph_tc = split and bool(tuning.get("sph_tc", 0)) and 4 <= args.slices <= 7
    fp64_peak = fp64_peak_tflops(torch, device)
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {"bf16_tflops": 1590.0}
    # dense int8 reference: the measured library int8 GEMM when it beats
    # twice the measured dense bf16 rate (the nominal int8 : bf16 ratio)
    int8_lib = int8_peak_tops(torch, device)
    int8_2bf16 = 2.0 * peaks.get("bf16_tflops", 1590.0)
    int8_peak = max(int8_lib or 0.0, int8_2bf16)
    # algorithmic work of each main kernel: FP64 flops, or int8 slice-product
    # ops (2 per MAC; S(S+1)/2 products per real MAC of the complex product)
    prods = lambda S: S * (S + 1) / 2.0
    kern = {}
    if sph_tc:
        # per pair and l: 4 real outputs (S, H re/im) x 2 K_c real MACs, K_c = 2 NDF
        ops = 2.0 * pairs * p.ltop * 4.0 * (2.0 * 2 * p.ndf) * prods(args.slices)
        kern["k_sph_tc (K-b, tcgen05)"] = ("tensor", ops, avg.get("ms_sph_main", 0.0), f_sph)
    else:
        kern["k_spherical (K-b, FP64)"] = ("fp64", f_sph, avg.get("ms_sph_main", 0.0), f_sph)
    if split:
        # per lower-triangle element: 2 real outputs x 2 K real MACs
        ops = 2.0 * (n * (n + 1) / 2.0) * 4.0 * K_hns * prods(slices_hns)
        kern["k_split_gemm (K-ns, tcgen05)"] = ("tensor", ops, avg.get("ms_hns_main", 0.0), f_hns)
    else:
        kern["HNS update (K-ns, FP64: k_hns_gemm + ZGEMM panels)"] = ("fp64", f_hns, avg.get("ms_hns_main", 0.0),
                                                                     f_hns)
    dom = max(kern, key=lambda k: kern[k][2])
    bound, work, t_ms, f64eq = kern[dom]
    if bound == "tensor":
        unit, peak = "TOP/s", int8_peak
        peak_src = (("measured here: cuBLAS int8 GEMM 8192^3 (torch._int_mm), best of 5 = %.0f TOP/s; "
                     "2 x measured dense bf16 (MEASURED_PEAKS.json) = %.0f; the larger is the peak; "
                     % (int8_lib or 0.0, int8_2bf16)) +
                    "achieved counts the int8 slice-product ops the kernel must execute")
    else:
        unit, peak = "TFLOP/s", fp64_peak
        peak_src = ("measured here: cuBLAS DGEMM 8192^3, best of 5 (MEASURED_PEAKS.json has no FP64 figure); "
                    "FP64 FMA pipe, not tensor cores or HBM")
    achieved = work / (t_ms * 1e-3) / 1e12 if t_ms > 0 else None
    traffic = None
    tj = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tj):
        try:
            traffic = json.load(open(tj)).get(dom)
        except Exception:
            traffic = None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, sample, _ = cpu_reference(p)
        cpu = {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": sample}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.prec == "fp64" else f"int8 x{args.slices}/x{slices_hns} slices (spherical/HNS), f64 combine",
        "data": "synthetic (seeded)",
        "config": {"workload": workload, "n": n, "nv": p.nv, "nlo": p.nlo, "atoms": p.ndf, "lmax": p.ltop - 1,
                   "lmax_ns": p.lnsmax, "precision": args.prec,
                   "slices": [args.slices, slices_hns] if split else None,
                   "parallelism": f"k-shard x{world}",
                   "l2": "HS output 0.39 GB and HNS operands 0.32 GB per k-point exceed the 126 MB L2"},
        "kpoints_per_s": 1e3 / value,
        "fp64_equiv_tflops": (f_sph + f_hns) / (ms_step * 1e-3) / 1e12,
        "fp64_equiv_tflops_baseline_def": baseline_def_flops(p) / (ms_step * 1e-3) / 1e12,
        "stage_ms": {k: v for k, v in avg.items() if k.startswith("ms_")},
        "tuning": tuning,
        "roofline": {"kernel": dom, "bound": bound,
                     "achieved": achieved, "peak": peak, "unit": unit,
                     "frac": achieved / peak if (peak and achieved) else None, "traffic": traffic,
                     "peak_source": peak_src, "work_per_launch": work, "ms_per_launch": t_ms,
                     "fp64_equiv_tflops": f64eq / (t_ms * 1e-3) / 1e12 if t_ms > 0 else None,
                     "fp64_peak_tflops": fp64_peak, "int8_peak_tops": int8_peak,
                     "kernels": {k: {"bound": b, "work": w, "ms": t,
                                     "achieved": w / (t * 1e-3) / 1e12 if t > 0 else None,
                                     "frac": (w / (t * 1e-3) / 1e12) / (int8_peak if b == "tensor" else fp64_peak)
                                     if t > 0 else None,
                                     "fp64_equiv_tflops": f / (t * 1e-3) / 1e12 if t > 0 else None}
                                 for k, (b, w, t, f) in kern.items()}},
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if fp64_cmp is not None:
        line["fp64_path"] = fp64_cmp
    if batch is not None:
        line["batch"] = batch
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(line), flush=True)
    kp.free()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
