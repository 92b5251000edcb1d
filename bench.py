"""Benchmark of the lapw1 H/S setup (HAMILT + HNS [+ HORB]) and its adjoint forces on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c4|c1] [--fd-report]

Default workload (c4): the 100-atom orthorhombic cell 20 x 20 x 20 bohr
(seeded random positions, min separation 3.8 bohr, Rmt 1.8-2.3), RKmax 8
(N ~ 12700 basis functions, 2.6 GB per packed HS), lmax 10, lmax_ns 4, one
LO per atom for l <= 2, 16 seeded k-points per GPU.  One step = the
calkpt.F:153-185 setup of all 16 k-points in split precision as ONE
captured batch launch (lapw1gpu_setup_batch: int8 Ozaki slices on tcgen05,
5 slices spherical / 4 HNS, FP64 combine) plus the adjoint forces of the
lowest 400 bands at each of the 16 k-points (lapw1gpu_forces_batch; int8
slice products with 6 slices for the density matrices and 4 for the HNS
projections, FP64 pair sums).  The
eigenvectors come from the device eigen-solve of each k-point's split
matrices before timing (the eigen-solve is not part of the step, as SECLR4
is not part of the setup).  With N GPUs each rank takes its own 16 k-points
of the same crystal (k-point sharding, no collective on the data path).

`value` is ms per k-point of setup + forces for the whole job (device
time of K steps, CUDA events on the library's stream, max over ranks, over
16 N k-points per step).  `fp64_path` times the plain FP64 GPU path (FP64
spherical kernel, FP64 HNS with library ZGEMM panels, FP64 density
matrices, every adjoint pair on the FP64 pair kernel) on the same k-points
and eigenvectors, against the split arm (int8 slice products on tcgen05,
the adjoint's cross-block spherical pairs as int8 projections); `setup` and `forces` split
both arms into their parts, with forces/s (3 NDF force components per
k-point per second).  `e2e` runs k-point 0 through the host C ABI: inputs
from host memory, HS/HSDIAG copied back into a caller HS page-locked once
by lapw1gpu_host_register, eigenvectors from pinned host memory and the
gradient read back.  `accuracy` gives the split path's errors against the
FP64 path (per-matrix, eigenvalues in the SECLR4 window, forces) and, on
the 100-atom RKmax 6 cell c3, against central differences of the band
energy (step 1e-4 bohr).  The reference arm (--impl reference) times the
CPU restatement of the reference algorithm (no Fortran compiler exists
here to build the reference itself) on all host cores over bounded samples
of k-point 0 (the reference has no force code in lapw1: its arm is the
setup alone).  `--workload c1` prints the 40-atom single-k-point line
instead; `--fd-report` prints the central-difference check of all 300
force components of c3.
"""
from __future__ import annotations

import os

# OpenMP threads of the CPU legs sleep instead of spinning between parallel
# regions, so that they leave the cores to OpenBLAS's own threads (set
# before any OpenMP runtime is loaded)
os.environ.setdefault("OMP_WAIT_POLICY", "passive")

import argparse  # noqa: E402
import json  # noqa: E402
import math  # noqa: E402
import statistics  # noqa: E402
import subprocess  # noqa: E402
import sys  # noqa: E402
import threading  # noqa: E402
import time  # noqa: E402

import numpy as np  # noqa: E402

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NK = 16          # k-points per GPU and step (c4)
NBANDS = 400     # occupied bands of the adjoint
METRIC = "lapw1 H+S setup + adjoint forces ms/k-point (split precision, 16 batched k-points)"
METRIC_C1 = "lapw1 H+S setup ms/k-point"
UNIT = "ms/k-point"
WORKLOAD_C4 = ("c4: 100-atom cell 20^3 bohr, RKmax 8, lmax 10, lmax_ns 4, LO l<=2, 16 batched k-points per GPU, "
               "split setup + adjoint forces of 400 bands")
WORKLOAD_C1 = "c1: 2x2x2 ABO3 supercell a=14.8 bohr, 40 atoms, RKmax 7, lmax 10, lmax_ns 4, LO l<=2, one general k"


def _env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.live = False
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.rows and time.time() - t0 < 5.0:  # sampling is live before timing starts
                time.sleep(0.02)
            self.rows.clear()
            self.live = True
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        self.live = False
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


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return json.load(open(path)), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# ---------------------------------------------------------------- CPU legs
def _cpu_sample(p, frac, L):
    """The oracle over about `frac` of one k-point's setup work: HAMILT
    over every m-th plane-wave column (column I of HAMILT costs ~I, so the
    sampled share of its work is counted exactly) and HNS for the first
    round(frac NDF) atoms (every atom costs the same).  Returns
    (extrapolated ms per k-point, description, seconds of the sample)."""
    from oracle import oracle as O
    nv = p.nv
    # a contiguous block of columns at the far end of the triangle, whose
    # share of the work is exact: columns c0..nv cost sum_I I
    c0 = max(1, int(nv * math.sqrt(1.0 - frac)))
    t = time.perf_counter()
    O.hamilt_sample(p, c0, nv, L=L)
    t_h = time.perf_counter() - t
    frac_h = (nv * (nv + 1) / 2 - (c0 - 1) * c0 / 2) / (nv * (nv + 1) / 2)
    na = max(1, min(p.ndf, int(round(frac * p.ndf))))
    t = time.perf_counter()
    O.hns_sample(p, 1, na, L=L)
    t_ns = time.perf_counter() - t
    est_s = t_h / frac_h + t_ns * p.ndf / na
    sample = (f"HAMILT PW columns {c0}..{nv} of {nv} ({100 * frac_h:.1f}% of its work) + "
              f"HNS atoms 1..{na} of {p.ndf}; extrapolated to one k-point")
    return est_s * 1e3, sample, t_h + t_ns


def cpu_reference(p, budget_s, L):
    """Bounded CPU sample of the reference algorithm (the oracle, OpenMP and
    OpenBLAS on all host cores) sized to about `budget_s` seconds from a
    small calibration sample."""
    est_ms, _, _ = _cpu_sample(p, 0.005, L)
    frac = min(1.0, max(0.005, budget_s / (est_ms * 1e-3)))
    return _cpu_sample(p, frac, L)


def run_reference(args):
    rank, world, _ = _env_rank()
    if rank != 0:
        return 0
    from hack_wein2k_b200 import synth
    from oracle import oracle as O
    L, build = O.baseline_lib()
    if args.workload == "c1":
        p, workload, metric = synth.config("c1")[0], WORKLOAD_C1, METRIC_C1
    else:
        p, workload, metric = synth.config("c4", nk=1)[0], WORKLOAD_C4, METRIC
    cores = os.cpu_count()
    vals, steps_s = [], []
    sample = ""
    budget = min(8.0, max(0.5, 100.0 / (args.warmup + args.steps)))  # whole run within a few minutes
    for i in range(args.warmup + args.steps):
        v, sample, sec = cpu_reference(p, budget, L)
        if i >= args.warmup:
            vals.append(v)
            steps_s.append(sec)
    val = statistics.median(vals)
    note = ("setup only: the reference lapw1 has no force code (WIEN2k computes forces later, in lapw2's "
            "fomai1.f, a separate program)") if args.workload != "c1" else "setup"
    line = {
        "impl": "reference", "metric": metric, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(steps_s),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": workload, "n": p.n, "nv": p.nv, "nlo": p.nlo, "atoms": p.ndf,
                   "impl": "CPU restatement of HAMILT/HNS (oracle port), OpenMP + OpenBLAS on all host cores",
                   "reference_work": note},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
                         "cpu": cpu_model(), "build": build,
                         "step": "one bounded sample (ms_per_step of work) extrapolated to a whole k-point"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- helpers
def _timed_loop(torch, stream, fn, steps, nvtx=None):
    """CUDA-event time of `steps` calls of fn on `stream`; nvtx: the name of
    an NVTX range around the calls (a profiler can be limited to it)"""
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if nvtx:
        torch.cuda.nvtx.range_push(nvtx)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    if nvtx:
        torch.cuda.nvtx.range_pop()
    return e0.elapsed_time(e1)


def _rel_err_c(torch, a, b):
    """per-matrix max relative error of packed HS a against b (complex
    [col][row] device tensors): H lower + diagonal, S strict upper"""
    ca, cb = a.transpose(0, 1), b.transpose(0, 1)  # [row][col]
    n = ca.shape[0]
    out = {}
    for name, tri in (("H", lambda x: torch.tril(x)), ("S", lambda x: torch.triu(x, 1))):
        d = tri((ca - cb).abs()).max().item()
        m = tri(cb.abs()).max().item()
        out[name] = d / m if m > 0 else 0.0
    return out


def _window_err(w, w0, lo=-10.0, hi=10.0):
    w, w0 = np.asarray(w), np.asarray(w0)
    m = min(len(w), len(w0))
    w, w0 = w[:m], w0[:m]
    win = (w0 > lo) & (w0 < hi)
    return float(np.abs(w - w0)[win].max()) if win.any() else None


def _sph_pairs(p):
    return p.nv * (p.nv - 1) / 2.0


def force_sph_flops(p, block=None):
    """FP64 flops of k_force_sph (FMA = 2): per plane-wave pair J < I and
    atom type, the l = 0 term (6) and 10 per further l (two 2-vector dot
    products weighted into the S and H sums); per pair and atom 21 (phase
    product, the two imaginary parts, the pair term and its dK weighting).
    With the spherical projections (block rows per block) the kernel takes
    the pairs inside a block only."""
    if block:
        pairs = sum(min(block, p.nv - r0) * (min(block, p.nv - r0) - 1) / 2.0 for r0 in range(0, p.nv, block))
    else:
        pairs = _sph_pairs(p)
    return pairs * (p.nat * (6.0 + 10.0 * (p.ltop - 1)) + 21.0 * p.ndf)


def force_proj_ops(p, nb, S):
    """int8 ops of the adjoint's spherical projections: output K x 4 nb
    complex (K = 2 NDF ltop^2 real-harmonic rows), inner NV complex, 8 real
    ops per complex multiply-add, S(S+1)/2 slice products"""
    K = 2.0 * p.ndf * p.ltop ** 2
    return 8.0 * K * 4.0 * nb * p.nv * (S * (S + 1) / 2.0)


def sph_tc_ops(p, S):
    """int8 ops of k_sph_tc: per pair (J <= I) and l, 4 real outputs x
    2 K_c real MACs (K_c = 2 NDF) x S(S+1)/2 slice products x 2"""
    pairs = p.nv * (p.nv + 1) / 2.0
    return 2.0 * pairs * p.ltop * 4.0 * (2.0 * 2 * p.ndf) * (S * (S + 1) / 2.0)


def split_gemm_ops(p, S):
    """int8 ops of the split HNS update: per lower-triangle element 2 real
    outputs x 2 K real MACs, K = 2 NDF (lmax_ns+1)^2, S(S+1)/2 products"""
    n = p.n
    K = 2.0 * p.ndf * (p.lnsmax + 1) ** 2
    return 2.0 * (n * (n + 1) / 2.0) * 4.0 * K * (S * (S + 1) / 2.0)


def ka_bytes(p, S):
    """Algorithmic DRAM bytes of the K-a kernels of the split path:
    k_albl writes AL and BL (and reads |k+G|); the spherical slicers read
    AL, BL and the phases and write the int8 slice operands."""
    nvpad = -(-p.nv // 64) * 64
    albl = 2.0 * p.nat * p.ltop * nvpad * 8 + p.nv * 8
    Kp = 2 * (-(-2 * p.ndf // 16) * 16)
    npA = -(-p.nv // 128) * 128
    IT = {4: 8, 5: 12, 6: 8, 7: 8}.get(S, 12)
    npB = -(-p.nv // IT) * IT
    slices = S * p.ltop * (npA + 4 * npB) * Kp
    slicer = slices + albl + p.ndf * (-(-p.n // 64) * 64) * 16
    return albl, slicer


def kc_bytes(p):
    """k_table writes Theta and WARP (complex) on the box of row differences."""
    k = np.asarray(p.kzz[: p.nv])
    d = k.max(axis=0) - k.min(axis=0)
    return float(np.prod(2 * d + 1)) * 2 * 16


# ---------------------------------------------------------------- the c4 line
def c4_step_line(args):
    import torch

    from hack_wein2k_b200 import forces as FO
    from hack_wein2k_b200 import lapw1gpu, synth
    from hack_wein2k_b200.seclr import hermitian_from_packed_device, solve

    rank, world, local = _env_rank()
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    t_prep = time.time()
    ps = synth.config("c4", nk=NK, kofs=NK * rank)
    ctx = lapw1gpu.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream_handle, device=dev)
    s_sph, s_hns = args.slices, args.slices_hns

    def use(prec):
        if prec == "fp64":
            ctx.set_precision(lapw1gpu.PREC_FP64)
        else:
            ctx.set_precision(lapw1gpu.PREC_SPLIT, s_sph)
            ctx.set_slices(s_sph, s_hns)
            ctx.set_force_slices(*args.force_slices)
            ctx.set_force_projection(*args.force_projection)

    def bar():
        if dist is not None:
            dist.barrier()

    def maxr(x):
        if dist is None:
            return x
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    kps = [ctx.upload(q) for q in ps]
    hs = [torch.empty((q.n, q.n), dtype=torch.complex128, device=dev) for q in ps]  # [col][row] = HS
    hd = [torch.empty(q.n, dtype=torch.complex128, device=dev) for q in ps]
    bargs = (kps, [t.data_ptr() for t in hs], [q.n for q in ps], [t.data_ptr() for t in hd])

    def tune(prec, sets_cand):
        use(prec)
        tun = {} if args.no_autotune else ctx.autotune(kps[0], hs[0].data_ptr(), ps[0].n, hd[0].data_ptr())
        best = None
        for sets in sets_cand:  # the batch schedule is tuned too: concurrent k-point chains
            ctx.set_tuning(batch_sets=sets)
            ctx.setup_batch(*bargs)  # eager pass + capture
            t_b = min(ctx.setup_batch(*bargs)["ms_total"] for _ in range(2))
            if best is None or t_b < best[1]:
                best = (sets, t_b)
        ctx.set_tuning(batch_sets=best[0])
        out = ctx.tuning()
        out.update({k: v for k, v in tun.items() if k == "ms_best"})
        return out

    # ---- split precision: tune, set up once, eigenvectors of every k-point ----
    tun_split = tune("split", (1, 2, 3))
    ctx.setup_batch(*bargs)
    t_eig = time.time()
    Xc, W = [], []
    for i, q in enumerate(ps):
        H, S = hermitian_from_packed_device(hs[i], hd[i])
        w, X = solve(H, S, nmax=NBANDS)
        del H, S
        Xc.append(X.transpose(0, 1).contiguous())  # column-major n x nb (ldc = n)
        W.append(w.contiguous())
        del X
        torch.cuda.empty_cache()
    t_eig = time.time() - t_eig
    hs0_split = hs[0].clone()
    w0_split = W[0].cpu().numpy()
    occ = torch.ones(NBANDS, dtype=torch.float64, device=dev)
    grads = [torch.empty((q.ndf, 3), dtype=torch.float64, device=dev) for q in ps]

    fargs = (kps, [x.data_ptr() for x in Xc], [q.n for q in ps], NBANDS, occ.data_ptr(), [w.data_ptr() for w in W],
             [g.data_ptr() for g in grads])

    def forces_all():
        """the adjoint of all 16 k-points, queued back to back (one library call)"""
        ms_f = ctx.forces_batch(*fargs)
        return ctx.last_launches(), ms_f

    launches = {}
    host = {"setup_wall_ms": [], "setup_dev_ms": [], "forces_wall_ms": [], "forces_dev_ms": []}

    def step():
        t0 = time.perf_counter()
        st_b = ctx.setup_batch(*bargs)
        t1 = time.perf_counter()
        launches["setup"] = ctx.last_launches()
        launches["forces"], ms_f = forces_all()
        t2 = time.perf_counter()
        host["setup_wall_ms"].append((t1 - t0) * 1e3)
        host["setup_dev_ms"].append(st_b["ms_total"])
        host["forces_wall_ms"].append((t2 - t1) * 1e3)
        host["forces_dev_ms"].append(ms_f)

    forces_all()  # the adjoint's scratch reaches its size before the warm-up steps
    for _ in range(args.warmup):
        step()
    bar()
    with ClockSampler(local) as clk:
        ms = _timed_loop(torch, stream, step, args.steps, nvtx="timed")
    bar()
    ms = maxr(ms)
    ms_step = ms / args.steps
    value = ms_step / (NK * world)
    step_parts = {k: float(np.mean(v[args.warmup:])) for k, v in host.items()}
    g0_split = grads[0].cpu().numpy()
    # parts of the split step: the batched setup alone, the forces alone
    ms_setup_split = min(ctx.setup_batch(*bargs)["ms_total"] for _ in range(3)) / NK

    def singles():  # the same k-points as 16 lapw1gpu_kpoint_run calls
        for i, k in enumerate(kps):
            k.run(hs[i].data_ptr(), ps[i].n, hd[i].data_ptr())

    singles()
    ms_setup_singles = _timed_loop(torch, stream, singles, 1) / NK
    ms_forces_split = min(forces_all()[1] for _ in range(2)) / NK
    fst_split = []
    for i, q in enumerate(ps[:4]):
        kps[i].forces(Xc[i].data_ptr(), q.n, NBANDS, occ.data_ptr(), W[i].data_ptr(), grads[i].data_ptr())
        fst_split.append(ctx.forces_stats())
    ms_fsph_split = float(np.mean([f["ms_sph_main"] for f in fst_split]))
    ms_fproj_split = float(np.mean([f["ms_sph_slice"] for f in fst_split]))
    fproj_on = ms_fproj_split > 0.0
    fproj_s = args.force_projection[0] if args.force_projection[0] > 0 else 6
    fproj_b = args.force_projection[1] if fproj_on else None
    # per-kernel times of one split k-point (stats pass)
    st_k = kps[0].run(hs[0].data_ptr(), ps[0].n, hd[0].data_ptr(), stats=True)

    # ---- the plain FP64 GPU path on the same k-points and eigenvectors ----
    tun_fp64 = tune("fp64", (2,))  # FP64 kernels fill the GPU alone: two chains

    def step64():
        ctx.setup_batch(*bargs)
        forces_all()

    step64()
    n64 = max(2, min(args.steps, 3))
    bar()
    ms64 = maxr(_timed_loop(torch, stream, step64, n64)) / n64
    g0_fp64_same = grads[0].cpu().numpy()  # FP64 adjoint, the split path's eigenvectors
    ms_setup_fp64 = min(ctx.setup_batch(*bargs)["ms_total"] for _ in range(2)) / NK
    ms_forces_fp64 = forces_all()[1] / NK
    # accuracy at k-point 0: split against FP64 matrices, eigenvalues, forces
    ctx.setup_batch(*bargs)
    err_hs = _rel_err_c(torch, hs0_split, hs[0])
    del hs0_split
    H, S = hermitian_from_packed_device(hs[0], hd[0])
    w64, X64 = solve(H, S, nmax=NBANDS)
    del H, S
    X64c = X64.transpose(0, 1).contiguous()
    del X64
    g64 = torch.empty((ps[0].ndf, 3), dtype=torch.float64, device=dev)
    kps[0].forces(X64c.data_ptr(), ps[0].n, NBANDS, occ.data_ptr(), w64.data_ptr(), g64.data_ptr())
    w64n = w64.cpu().numpy()
    fsp = FO.cartesian_forces(ps[0], g0_split)
    fsame = FO.cartesian_forces(ps[0], g0_fp64_same)
    m = min(len(w0_split), len(w64n))
    # the seeded RKmax 8 inputs put ghost states (|eps| ~ 1e4-1e5 Ry, from
    # an ill-conditioned overlap) among the lowest 400: the force error of
    # the adjoint's arithmetic is compared on the same eigenvectors, and the
    # eigenvalue error is relative to the largest |eps|
    acc4 = {"rel_error_vs_fp64": err_hs,
            "eig_rel_err_lowest": float(np.abs(w0_split[:m] - w64n[:m]).max() / np.abs(w64n[:m]).max()),
            "eig_range_ry": [float(w64n[0]), float(w64n[m - 1])],
            "eig_err_window_ry": _window_err(w0_split, w64n),
            "force_err_same_eigvecs_ry_bohr": float(np.abs(fsp - fsame).max()),
            "max_force_ry_bohr": float(np.abs(fsame).max())}
    del X64c, g64
    torch.cuda.empty_cache()

    # ---- e2e through the host C ABI (k-point 0, split precision) ----
    use("split")
    p0 = ps[0]
    n0 = p0.n
    hs_host = np.zeros((n0, n0), dtype=np.complex128, order="F")  # the caller's HS (pageable)
    hd_host = np.zeros(n0, dtype=np.complex128)
    ctx.host_register(hs_host)  # once, as a Fortran caller would after INIT_MATRICES
    ctx.host_register(hd_host)
    x_host = torch.empty((NBANDS, n0), dtype=torch.complex128).pin_memory()
    x_host.copy_(Xc[0].cpu())
    w_host = W[0].cpu().pin_memory()
    g_host = torch.empty((p0.ndf, 3), dtype=torch.float64).pin_memory()
    x_dev = torch.empty_like(Xc[0])
    w_dev = torch.empty_like(W[0])
    kp_e = {}

    def e2e_step_sequential():
        ctx.setup(p0, hs=hs_host, hsdiag=hd_host)
        x_dev.copy_(x_host, non_blocking=True)
        w_dev.copy_(w_host, non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        kps[0].forces(x_dev.data_ptr(), n0, NBANDS, occ.data_ptr(), w_dev.data_ptr(), grads[0].data_ptr())
        g_host.copy_(grads[0])
        kp_e["g"] = float(g_host.abs().max())

    def e2e_step():
        # the setup's HS copies to the host run behind the adjoint's kernels
        ctx.setup_async(p0, hs_host, hd_host)
        x_dev.copy_(x_host, non_blocking=True)
        w_dev.copy_(w_host, non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()  # the torch stream's copies only
        kps[0].forces(x_dev.data_ptr(), n0, NBANDS, occ.data_ptr(), w_dev.data_ptr(), grads[0].data_ptr())
        ctx.setup_wait()
        g_host.copy_(grads[0])
        kp_e["g"] = float(g_host.abs().max())

    e2e_step()
    e2e_step_sequential()
    ne = max(1, min(args.steps, 3))
    bar()
    t0 = time.perf_counter()
    e2e_ms = _timed_loop(torch, stream, e2e_step, ne) / ne
    wall_e2e = (time.perf_counter() - t0) * 1e3 / ne
    e2e_ms = maxr(e2e_ms)
    e2e_seq_ms = maxr(_timed_loop(torch, stream, e2e_step_sequential, ne) / ne)
    h2d = sum(a.nbytes for a in p0.to_c()._keep) + x_host.numel() * 16 + w_host.numel() * 8
    d2h = n0 * n0 * 16 + n0 * 16 + p0.ndf * 3 * 8
    # the same through a pageable HS never registered (the copies staged by the driver)
    ctx.host_unregister(hs_host)
    ctx.host_unregister(hd_host)
    hs_pg = np.zeros((n0, n0), dtype=np.complex128, order="F")
    hd_pg = np.zeros(n0, dtype=np.complex128)
    ctx.setup(p0, hs=hs_pg, hsdiag=hd_pg)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.setup(p0, hs=hs_pg, hsdiag=hd_pg)
    pageable_setup_ms = (time.perf_counter() - t0) * 1e3
    del hs_pg, hd_pg, hs_host, hd_host

    # ---- c3: accuracy against the FP64 path and central differences ----
    hs.clear()
    hd.clear()
    Xc.clear()
    for k in kps[1:]:
        k.free()
    torch.cuda.empty_cache()
    acc3 = c3_accuracy(ctx, torch, dev, args.fd_components) if not args.no_extras else None

    # ---- c1: the 40-atom single k-point ----
    c1 = c1_summary(ctx, torch, dev, stream) if not args.no_extras else None
    c2 = c2_batch(ctx, torch, dev, stream) if not args.no_extras else None

    # ---- roofline of the dominant kernel (split arm, per k-point) ----
    clocks = clk.summary()
    peaks, peak_kind = measured_peaks()
    fp64_peak = fp64_peak_tflops(torch, dev)
    int8_lib = int8_peak_tops(torch, dev)
    int8_peak = max(int8_lib or 0.0, 2.0 * peaks.get("bf16_tflops", 1590.0))
    hbm = peaks.get("hbm_gbs", 6650.0)
    albl_b, slicer_b = ka_bytes(p0, s_sph)
    kern = {
        "k_force_sph (adjoint pair sums, FP64)": ("fp64", force_sph_flops(p0, fproj_b), ms_fsph_split, "TFLOP/s",
                                                  fp64_peak),
        "k_sph_tc (K-b, tcgen05 int8)": ("tensor", sph_tc_ops(p0, s_sph), st_k["ms_sph_main"], "TOP/s", int8_peak),
        "k_split_gemm (K-ns, tcgen05 int8)": ("tensor", split_gemm_ops(p0, s_hns), st_k["ms_hns_main"], "TOP/s",
                                              int8_peak),
        "k_albl (K-a)": ("hbm", albl_b, st_k["ms_k_albl"], "GB/s", hbm),
        "k_sph_slice x2 (K-a, split operands)": ("hbm", slicer_b, st_k["ms_sph_slice"], "GB/s", hbm),
        "k_table (K-c)": ("hbm", kc_bytes(p0), st_k["ms_table"], "GB/s", hbm),
    }

    if fproj_on:
        kern["k_split_gemm (adjoint spherical projections, tcgen05 int8, with their operand slicing)"] = (
            "tensor", force_proj_ops(p0, NBANDS, fproj_s), ms_fproj_split, "TOP/s", int8_peak)

    def rate(w, t, unit):
        if t <= 0:
            return None
        return w / (t * 1e-3) / (1e9 if unit == "GB/s" else 1e12)

    kd = {}
    for name, (bnd, w, t, unit, pk) in kern.items():
        a = rate(w, t, unit)
        kd[name] = {"bound": bnd, "work_per_launch": w, "ms": t, "achieved": a, "unit": unit, "peak": pk,
                    "frac": a / pk if a else None}
    dom = max((k for k in kern if kern[k][0] != "hbm"), key=lambda k: kern[k][2])
    tr4 = {}
    tj = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tj):
        try:
            tr4 = json.load(open(tj)).get("c4", {})
        except Exception:
            tr4 = {}
    for name in kd:  # DRAM bytes per launch from the ncu captures (profiles/traffic.json)
        kd[name]["traffic"] = tr4.get(name)
    fs = "k_force_sph (adjoint pair sums, FP64)"
    if fproj_on and kd[fs]["traffic"]:  # the capture covers every pair; with projections it takes the block pairs
        kd[fs]["traffic"] *= force_sph_flops(p0, fproj_b) / force_sph_flops(p0)
    traffic = tr4.get(dom)
    dm = kd[dom]
    roofline = {"kernel": dom, "bound": dm["bound"], "achieved": dm["achieved"], "peak": dm["peak"],
                "unit": dm["unit"], "frac": dm["frac"], "traffic": traffic,
                "peak_source": (f"FP64: cuBLAS DGEMM 8192^3 measured here ({fp64_peak:.1f} TFLOP/s; "
                                "MEASURED_PEAKS.json has no FP64 figure); int8: the larger of cuBLAS int8 8192^3 "
                                f"measured here ({(int8_lib or 0):.0f} TOP/s) and 2 x measured bf16 "
                                f"({2.0 * peaks.get('bf16_tflops', 1590.0):.0f}); HBM: {hbm:.0f} GB/s "
                                f"({peak_kind}, MEASURED_PEAKS.json)"),
                "kernels": kd}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        L, build = O.baseline_lib()
        v, sample, sec = cpu_reference(p0, 12.0, L)
        cpu = {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": sample,
               "cpu": cpu_model(), "build": build, "seconds": sec,
               "note": "setup only (the reference lapw1 has no force code)"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None,
        "dtype": f"int8 x{s_sph}/x{s_hns}/x{args.force_slices[0]}/x{args.force_slices[1]}"
                 + (f"/x{fproj_s}" if fproj_on else "") + " slices (spherical/HNS/adjoint density matrices/"
                 "adjoint HNS projections" + ("/adjoint spherical projections" if fproj_on else "")
                 + ") with f64 combine; f64 force pair sums" + (" inside row blocks" if fproj_on else ""),
        "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD_C4, "kpoints_per_gpu": NK, "n": [q.n for q in ps], "nv0": p0.nv,
                   "nlo": p0.nlo, "atoms": p0.ndf, "bands": NBANDS, "lmax": p0.ltop - 1, "lmax_ns": p0.lnsmax,
                   "slices": [s_sph, s_hns], "parallelism": f"k-shard x{world}",
                   "l2": "inputs larger than L2: each k-point's HS is 2.6 GB (126 MB L2)"},
        "kpoints_per_s": 1e3 / value,
        "setup": {"split_ms_per_kpoint": ms_setup_split, "fp64_ms_per_kpoint": ms_setup_fp64,
                  "split_single_calls_ms_per_kpoint": ms_setup_singles,
                  "speedup": ms_setup_fp64 / ms_setup_split,
                  "split_fp64_equiv_tflops": (16.0 * p0.n ** 2 * p0.ltop ** 2 + 8.0 * p0.n ** 2 * 25) * p0.ndf
                  / (ms_setup_split * 1e-3) / 1e12},
        "forces": {"split_ms_per_kpoint": ms_forces_split, "fp64_ms_per_kpoint": ms_forces_fp64,
                   "split_forces_per_s": 3 * p0.ndf / (ms_forces_split * 1e-3),
                   "fp64_forces_per_s": 3 * p0.ndf / (ms_forces_fp64 * 1e-3),
                   "k_force_sph_ms": ms_fsph_split, "projection_products_ms": ms_fproj_split,
                   "projections": ({"slices": fproj_s, "block_rows": args.force_projection[1]} if fproj_on
                                   else None), "stats_k0": fst_split[0]},
        "fp64_path": {"ms_per_kpoint": ms64 / NK, "speedup_split_over_fp64": (ms64 / NK) / value,
                      "tuning": tun_fp64},
        "tuning": tun_split,
        "stage_ms_k0": {k: v for k, v in st_k.items() if k.startswith("ms_")},
        "accuracy": {"c4_k0": acc4, "c3": acc3},
        "roofline": roofline,
        "e2e": {"value": e2e_ms, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "what": "k-point 0 through lapw1gpu_setup_async (host inputs, HS into a caller buffer page-locked "
                        "once by lapw1gpu_host_register) + eigenvectors H2D from pinned memory + lapw1gpu_forces "
                        "while the HS copies run + lapw1gpu_setup_wait + gradient D2H", "host_wall_ms": wall_e2e,
                "sequential_ms": e2e_seq_ms,
                "setup_into_pageable_hs_ms": pageable_setup_ms},
        "gpu_launches": int((launches.get("setup", 0) + launches.get("forces", 0)) * args.steps),
        "clocks": clocks,
        "prep_s": {"total": time.time() - t_prep, "eigen_solves": t_eig},
        "step_parts_ms": step_parts,
    }
    if c1 is not None:
        line["c1"] = c1
    if c2 is not None:
        line["c2_batch"] = c2
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(line), flush=True)
    kps[0].free()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def _c3_band_energy(ctx, torch, dev, p, nb):
    from hack_wein2k_b200.forces import band_energy
    occ = torch.ones(nb, dtype=torch.float64, device=dev)
    E, w, X, kp = band_energy(ctx, p, occ)
    return float(E), w, X, kp, occ


def c3_fd_component(ctx, torch, dev, p, nb, a, c, h_bohr=1.0e-4):
    """Central difference of E (lowest nb bands, FP64 path) along atom a,
    Cartesian component c, step h_bohr; returns dE/dPOS_c (lattice units)."""
    import dataclasses
    bk = np.asarray(p.bkzz, dtype=np.float64).reshape(3, 3)
    h = h_bohr * bk[c, c] / (2.0 * np.pi)  # lattice step of the orthorhombic cell
    from hack_wein2k_b200.forces import _setup_device
    from hack_wein2k_b200.seclr import eigenvalues, hermitian_from_packed_device
    vals = []
    for sgn in (1.0, -1.0):
        pos = np.array(p.pos, dtype=np.float64, copy=True)
        pos[a, c] += sgn * h
        kp, hs, hd = _setup_device(ctx, dataclasses.replace(p, pos=pos))
        H, S = hermitian_from_packed_device(hs, hd)
        del hs, hd
        vals.append(float(eigenvalues(H, S, nb).sum()))  # the band energy, unit occupations
        del H, S
        kp.free()
    return (vals[0] - vals[1]) / (2.0 * h)


def c3_accuracy(ctx, torch, dev, n_fd):
    """c3 (100 atoms, RKmax 6, N = 5904): the split path's eigenvalues and
    forces against the FP64 path, and the FP64 adjoint against central
    differences of the band energy on n_fd force components."""
    from hack_wein2k_b200 import forces as FO
    from hack_wein2k_b200 import lapw1gpu, synth
    p3 = synth.config("c3")[0]
    res = {}
    nb = NBANDS
    for prec in ("fp64", "split"):
        if prec == "fp64":
            ctx.set_precision(lapw1gpu.PREC_FP64)
        else:
            ctx.set_precision(lapw1gpu.PREC_SPLIT, 5)
            ctx.set_slices(5, 4)
        E, w, X, kp, occ = _c3_band_energy(ctx, torch, dev, p3, nb)
        g = FO.gradient(ctx, kp, X, occ, w).cpu().numpy()
        res[prec] = (w.cpu().numpy(), g)
        kp.free()
        del X
        torch.cuda.empty_cache()
    f64 = FO.cartesian_forces(p3, res["fp64"][1])
    fsp = FO.cartesian_forces(p3, res["split"][1])
    out = {"workload": f"c3: 100-atom cell 20^3 bohr, RKmax 6, N {p3.n}, {nb} bands",
           "eig_err_window_ry": _window_err(res["split"][0], res["fp64"][0]),
           "force_err_ry_bohr": float(np.abs(fsp - f64).max()), "max_force_ry_bohr": float(np.abs(f64).max())}
    ctx.set_precision(lapw1gpu.PREC_FP64)
    bk = np.asarray(p3.bkzz, dtype=np.float64).reshape(3, 3)
    fd = []
    rng = np.random.default_rng(77)
    comps = [(int(rng.integers(p3.ndf)), int(c)) for c in rng.integers(0, 3, size=n_fd)]
    for a, c in comps:
        d = c3_fd_component(ctx, torch, dev, p3, nb, a, c)
        err = abs(d - res["fp64"][1][a, c]) * bk[c, c] / (2.0 * np.pi)  # Ry/bohr
        err_sp = abs(d - res["split"][1][a, c]) * bk[c, c] / (2.0 * np.pi)
        fd.append({"atom": a, "comp": c, "fd_minus_adjoint_ry_bohr": err, "fd_minus_split_adjoint_ry_bohr": err_sp,
                   "force_ry_bohr": float(-res["fp64"][1][a, c] * bk[c, c] / (2.0 * np.pi))})
    out["central_fd_1e-4_bohr"] = fd
    return out


def c1_summary(ctx, torch, dev, stream):
    """c1 (40 atoms, one k-point): split and FP64 setup times with resident inputs."""
    from hack_wein2k_b200 import lapw1gpu, synth
    p = synth.config("c1")[0]
    n = p.n
    out = {"workload": WORKLOAD_C1, "n": n}
    hs = torch.empty((n, n), dtype=torch.complex128, device=dev)
    hd = torch.empty(n, dtype=torch.complex128, device=dev)
    kp = ctx.upload(p)
    for prec in ("split", "fp64"):
        if prec == "fp64":
            ctx.set_precision(lapw1gpu.PREC_FP64)
        else:
            ctx.set_precision(lapw1gpu.PREC_SPLIT, 5)
            ctx.set_slices(5, 4)
        ctx.autotune(kp, hs.data_ptr(), n, hd.data_ptr())
        for _ in range(2):
            kp.run(hs.data_ptr(), n, hd.data_ptr(), stats=True)
        reps = 10
        ms = _timed_loop(torch, stream, lambda: kp.run(hs.data_ptr(), n, hd.data_ptr()), reps) / reps
        st = kp.run(hs.data_ptr(), n, hd.data_ptr(), stats=True)
        out[prec] = {"ms_per_kpoint": ms, "ms_sph_main": st["ms_sph_main"], "ms_hns_main": st["ms_hns_main"]}
        if prec == "split":
            out[prec]["k_sph_tc_int8_tops"] = sph_tc_ops(p, 5) / (st["ms_sph_main"] * 1e-3) / 1e12
    kp.free()
    return out


def c2_batch(ctx, torch, dev, stream):
    """c2 (c1's cell at 64 k-points): the k-list set up as one batch (one
    graph launch, concurrent chains tuned) against 64 single-k-point calls."""
    from hack_wein2k_b200 import lapw1gpu, synth
    ps = synth.config("c2")
    ctx.set_precision(lapw1gpu.PREC_SPLIT, 5)
    ctx.set_slices(5, 4)
    kps = [ctx.upload(q) for q in ps]
    hs = [torch.empty((q.n, q.n), dtype=torch.complex128, device=dev) for q in ps]
    hd = [torch.empty(q.n, dtype=torch.complex128, device=dev) for q in ps]
    bargs = (kps, [t.data_ptr() for t in hs], [q.n for q in ps], [t.data_ptr() for t in hd])
    tun = ctx.autotune(kps[0], hs[0].data_ptr(), ps[0].n, hd[0].data_ptr())
    per_sets = {}
    for sets in (1, 2, 3):
        ctx.set_tuning(batch_sets=sets)
        ctx.setup_batch(*bargs)  # eager pass + capture
        per_sets[sets] = min(ctx.setup_batch(*bargs)["ms_total"] for _ in range(3)) / len(ps)
    best = min(per_sets, key=per_sets.get)
    ctx.set_tuning(batch_sets=best)

    def singles():
        for i, k in enumerate(kps):
            k.run(hs[i].data_ptr(), ps[i].n, hd[i].data_ptr())

    singles()
    ms_single = min(_timed_loop(torch, stream, singles, 1) for _ in range(2)) / len(ps)
    for k in kps:
        k.free()
    del hs, hd
    torch.cuda.empty_cache()
    return {"workload": "c2: c1's cell at 64 seeded k-points, split 5/4", "nk": len(ps),
            "n_range": [min(q.n for q in ps), max(q.n for q in ps)],
            "batch_ms_per_kpoint": per_sets[best], "batch_sets": best,
            "batch_ms_per_kpoint_by_sets": per_sets, "single_calls_ms_per_kpoint": ms_single,
            "gain": ms_single / per_sets[best],
            "tuning": {k: v for k, v in tun.items() if k in ("split_group", "sph_tc", "sph_kblock")}}


def fd_report(args):
    """Central differences (step 1e-4 bohr) of the c3 band energy along all
    3 NDF coordinates against the FP64 adjoint and the split one: one JSON
    line.  The energies come from the eigenvalue-only solve."""
    import torch

    from hack_wein2k_b200 import forces as FO
    from hack_wein2k_b200 import lapw1gpu, synth
    dev = torch.device("cuda", 0)
    ctx = lapw1gpu.Context(0)
    p3 = synth.config("c3")[0]
    nb = NBANDS
    E, w, X, kp, occ = _c3_band_energy(ctx, torch, dev, p3, nb)
    g = FO.gradient(ctx, kp, X, occ, w).cpu().numpy()
    # the split adjoint (bench.py's slice counts) on the same eigenvectors
    ctx.set_precision(lapw1gpu.PREC_SPLIT, args.slices)
    ctx.set_slices(args.slices, args.slices_hns)
    ctx.set_force_slices(*args.force_slices)
    gs = FO.gradient(ctx, kp, X, occ, w).cpu().numpy()
    ctx.set_precision(lapw1gpu.PREC_FP64)
    kp.free()
    del X
    torch.cuda.empty_cache()
    bk = np.asarray(p3.bkzz, dtype=np.float64).reshape(3, 3)
    errs = np.zeros((p3.ndf, 3))
    errs_sp = np.zeros((p3.ndf, 3))
    t0 = time.time()
    for a in range(p3.ndf):
        for c in range(3):
            d = c3_fd_component(ctx, torch, dev, p3, nb, a, c)
            errs[a, c] = abs(d - g[a, c]) * bk[c, c] / (2.0 * np.pi)
            errs_sp[a, c] = abs(d - gs[a, c]) * bk[c, c] / (2.0 * np.pi)
    F = FO.cartesian_forces(p3, g)
    print(json.dumps({"workload": f"c3: 100-atom cell 20^3 bohr, RKmax 6, N {p3.n}, {nb} bands; central "
                                  "differences of the FP64 setup's band energy",
                      "components": int(errs.size), "step_bohr": 1e-4,
                      "fp64_adjoint": {"max_abs_err_ry_bohr": float(errs.max()),
                                       "mean_abs_err_ry_bohr": float(errs.mean()),
                                       "worst": [int(x) for x in np.unravel_index(np.argmax(errs), errs.shape)]},
                      "split_adjoint": {"slices": [args.slices, args.slices_hns] + list(args.force_slices),
                                        "max_abs_err_ry_bohr": float(errs_sp.max()),
                                        "mean_abs_err_ry_bohr": float(errs_sp.mean())},
                      "max_force_ry_bohr": float(np.abs(F).max()), "seconds": time.time() - t0}), flush=True)
    ctx.close()
    return 0


# ---------------------------------------------------------------- the c1 line
def single_c1(args):
    """The 40-atom c1 single-k-point setup (split vs FP64) as its own line."""
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
    p = synth.config("c1")[0] if world == 1 else synth.config("c2", nk=1, kofs=rank)[0]
    ctx = lapw1gpu.Context(local, prec=lapw1gpu.PREC_SPLIT, slices=args.slices)
    ctx.set_slices(args.slices, args.slices_hns)
    stream = torch.cuda.ExternalStream(ctx.stream_handle, device=device)
    kp = ctx.upload(p)
    n = p.n
    d_hs = torch.empty((n, n, 2), dtype=torch.float64, device=device)
    d_hd = torch.empty((n, 2), dtype=torch.float64, device=device)
    torch.cuda.synchronize()
    tuning = ctx.tuning() if args.no_autotune else ctx.autotune(kp, d_hs.data_ptr(), n, d_hd.data_ptr())

    def step(stats=False):
        return kp.run(d_hs.data_ptr(), n, d_hd.data_ptr(), stages=7, stats=stats)

    for _ in range(args.warmup):
        step(True)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    with ClockSampler(local) as clk:
        ms = _timed_loop(torch, stream, step, args.steps)
    if dist is not None:
        dist.barrier()
        t = torch.tensor([ms], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    st = step(True)
    launches = int(st["kernel_launches"]) * args.steps
    hs_h = np.zeros((n, n), dtype=np.complex128, order="F")
    hd_h = np.zeros(n, dtype=np.complex128)
    ctx.host_register(hs_h)
    ctx.host_register(hd_h)
    ctx.setup(p, hs=hs_h, hsdiag=hd_h)
    e2e_steps = max(1, min(args.steps, 5))
    e2e_ms = _timed_loop(torch, stream, lambda: ctx.setup(p, hs=hs_h, hsdiag=hd_h), e2e_steps) / e2e_steps
    h2d = sum(a.nbytes for a in p.to_c()._keep)
    line = {
        "metric": METRIC_C1, "value": ms_step / world, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": f"int8 x{args.slices}/x{args.slices_hns} slices, f64 combine",
        "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD_C1, "n": n, "parallelism": f"k-shard x{world}",
                   "l2": "HS output 0.39 GB per k-point exceeds the 126 MB L2"},
        "stage_ms": {k: v for k, v in st.items() if k.startswith("ms_")}, "tuning": tuning,
        "roofline": {"kernel": "k_sph_tc (K-b, tcgen05 int8)", "bound": "tensor",
                     "achieved": sph_tc_ops(p, args.slices) / (st["ms_sph_main"] * 1e-3) / 1e12,
                     "unit": "TOP/s"},
        "e2e": {"value": e2e_ms / world, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": n * n * 16 + n * 16},
        "gpu_launches": launches, "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    kp.free()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--slices", type=int, default=5)
    ap.add_argument("--slices-hns", type=int, default=4,
                    help="int8 slices of HNS (the non-spherical part is 1-2 orders smaller than the spherical one)")
    ap.add_argument("--force-slices", type=int, nargs=2, default=[6, 4], metavar=("RHO", "PROJ"),
                    help="int8 slices of the adjoint's density matrices and of its HNS projections (the "
                         "density matrices carry the force error; 4-slice projections leave it unchanged at c4)")
    ap.add_argument("--force-projection", type=int, nargs=2, default=[-1, 1024], metavar=("SLICES", "BLOCK"),
                    help="the adjoint's spherical pairs of different BLOCK-row blocks as int8 slice projections "
                         "(lapw1gpu_set_force_projection; -1: 6 slices from 6 blocks, 0: the FP64 pair kernel)")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["c4", "c1"], default="c4")
    ap.add_argument("--fd-components", type=int, default=3,
                    help="c3 force components checked against central differences in the default line")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the c3 accuracy and c1 sections")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the library's default tuning (profiling runs: timings under a profiler mislead the autotuner)")
    ap.add_argument("--fd-report", action="store_true",
                    help="instead: central differences of all 300 c3 force components against the adjoint")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.fd_report:
        return fd_report(args)
    if args.workload == "c1":
        return single_c1(args)
    return c4_step_line(args)


if __name__ == "__main__":
    sys.exit(main())
