"""Benchmark of the even-odd clover Dirac operator and the FP64 / mixed-precision solves.

Workload (the configuration the headline metric is quoted on): SU(3)
fundamental, clover csw = 1.0, m0 = -0.2, lattice 16^3 x 32, smooth synthetic
links U = exp(i 0.3 H) (seed 7, plaquette about 0.79), antiperiodic in time, a
Gaussian FP64 source on the even sites.

One step = one application of the even-odd preconditioned clover operator
Cphi_eopre (= D_ee - D_eo D_oo^-1 D_oe), i.e. two launches of the fused hopping
kernel.  value = GB/s under HiRep's own byte model
(TestProgram/DiracOperator/speed_test_diracoperator.c:77-82: 36 vectors + 8
links per site and hop) plus the clover blocks and the (4+m)^2 input read:
    V * 2880 + V/2 * 192 + V/2 * (672 + 576) bytes per application.
The roofline fraction is taken on the bytes the kernels must move at least
(every link once per hop, read as two rows where the links are rebuilt, the
fields in and out, the packed clover blocks once), not on HiRep's model, which
counts each neighbour spinor eight times.  Each application touches about 240
MB, one launch about 130 MB, close to the 126 MB L2, so L2 is flushed between
timed steps: a 512 MB buffer is written and then another 512 MB buffer is read,
which leaves L2 holding clean lines of unrelated data.  Times are CUDA events
on the library's stream.

Besides the step the run reports the time to |r|/|b| < 1e-12 (err2 = 1e-24) of
the plain FP64 CG and of the FP32-inner defect-correction CG on g5Cphi_eopre^2,
the end-to-end rate through the C ABI with host buffers, the roofline of the
hopping kernel against the measured HBM copy bandwidth, the single-field
even-odd operator of the other workloads (16^4 SU(4) antisymmetric, 24^3x48
sextet clover, 32^3x64 SU(2) adjoint) with their rooflines, and HiRep's own
OpenMP build on the host cores as a reported baseline.

--impl reference times HiRep itself: the reference's library built from its
sources (oracle/ref/Makefile into oracle/_ref/), its Cphi_eopre on the same
fields, on all host cores (OMP_PROC_BIND=close), median of the timed
applications as TestProgram/DiracOperator/speed_test_diracoperator.c times
its operator.
With --gpus N (torchrun) every rank runs an independent replica on its own GPU
(the single-GPU scope has no halo exchange); value is the sum over ranks and
the time the max over ranks.
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

DIMS = (32, 16, 16, 16)  # T, X, Y, Z
NG, MASS, CSW, EPS, SEED = 3, -0.2, 1.0, 0.3, 7
SITE_BYTES = 2880  # 36 * sizeof(suNf_vector) + 8 * sizeof(suNf), SU(3) fundamental, double
SPINOR_BYTES = 192
CLOVER_BYTES = 672 + 576  # sizeof(ldl_t) + 4 * sizeof(suNfc), NF = 3
ERR2 = 1e-24
METRIC = "eopre Dslash GB/s (%HBM peak); time to |r|/|b|<1e-12, mixed vs FP64 solve"


def eopre_bytes(V):
    return V * SITE_BYTES + (V // 2) * SPINOR_BYTES + (V // 2) * CLOVER_BYTES


def unique_bytes(V, nf, real, link_rows, clover, link_bytes=None):
    """Bytes one FP64 even-odd application must move at least: every link once
    per hop (link_rows of its NF rows, real or complex; or link_bytes per link
    when the kernels build the links from the fundamental ones), the even input
    twice (hop 1 and the diagonal term of hop 2), the odd temporary written and
    read, the even output written, and the packed clover blocks (D^-1 on the
    odd sites, D on the even ones) once."""
    esz = 8 if real else 16
    links = 2 * 4 * V * (link_bytes if link_bytes else link_rows * nf * esz)
    spinors = 5 * (V // 2) * 4 * nf * 16
    blocks = V * (2 * 2 * nf * 8 + 2 * nf * (2 * nf - 1) * 16) if clover else 0
    return links + spinors + blocks


def workload_config():
    T, X, Y, Z = DIMS
    return {"workload": "clover eopre Dslash + solve, SU(3) fund, 16^3x32, csw=1.0, m0=-0.2, U=exp(i0.3H) seed 7",
            "lattice": f"{X}x{Y}x{Z}x{T}", "ng": NG, "repr": "fundamental", "nf": 3, "csw": CSW, "m0": MASS,
            "l2": "flushed between timed steps (512 MB written, then 512 MB read)", "bytes_model": "HiRep speed_test byte model + clover blocks"}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per launch of the hopping kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "hop_clover_su3_16x16x16x32.txt")
    try:
        for line in open(p):
            if line.startswith("traffic_bytes_per_eopre:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        import datetime

        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                if hasattr(self, "t0") and not (self.t0 - 0.05 <= ts <= self.t1 + 0.05):
                    continue
                sm.append(float(f[2]))
                mx = float(f[3])
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, f[6:10]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_port_arm(seconds):
    """The CPU restatement of HiRep's operator (oracle/hr_oracle.c) on all host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from hirep_b200 import fields as F

    threads = os.cpu_count() or 1
    o = O.Oracle(*DIMS, NG, O.FUND, threads=threads)
    u = F.smooth_gauge(SEED, o.V, NG, EPS)
    o.set_gauge(o.represent_gauge_field(u, True))
    o.clover_init(CSW)
    o.compute_clover_term()
    src = F.gaussian_spinor(SEED, o.VH, o.nf)
    o.Cphi_eopre(MASS, src)  # builds the LDL cache
    times = []
    t_end = time.perf_counter() + seconds
    while len(times) < 3 or (time.perf_counter() < t_end and len(times) < 200):
        t0 = time.perf_counter()
        o.Cphi_eopre(MASS, src)
        times.append(time.perf_counter() - t0)
    t = float(np.median(times))
    return {"value": eopre_bytes(o.V) / t / 1e9, "unit": "GB/s", "cores": threads, "kind": "port",
            "sample": f"{len(times)} Cphi_eopre applications on 16^3x32 (median {t * 1e3:.1f} ms), OpenMP"}


def cpu_reference_arm(args):
    """HiRep's own Cphi_eopre (LibHR/Update/Dphi.c:1240-1255) from the reference's
    library built from its sources, on all host cores, timed as its speed test
    times its operator (warm-up, then the median of >= 20 applications).  Falls
    back to the CPU restatement where the HiRep build is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import hirep_ref as H
    from hirep_b200 import fields as F

    if not H.available("su3_fund_clover"):
        base = cpu_port_arm(args.cpu_seconds)
        return base, eopre_bytes(DIMS[0] * DIMS[1] * DIMS[2] * DIMS[3]) / base["value"] / 1e9
    threads = os.cpu_count() or 1
    V = DIMS[0] * DIMS[1] * DIMS[2] * DIMS[3]
    u = F.smooth_gauge(SEED, V, NG, EPS)
    src = F.gaussian_spinor(SEED, V // 2, 3)
    with H.HiRep("su3_fund_clover", *DIMS, threads=threads) as h:
        h.set_gauge(u)
        h.set_csw(CSW)
        # one probe decides the count: 20..200 applications, about args.cpu_seconds
        probe, _, _ = h.time_op("Cphi_eopre", MASS, H.EVEN, warmup=args.warmup, reps=3, inp=src)
        reps = int(max(20, min(args.steps, args.cpu_seconds / (probe * 1e-6))))
        med, mn, thr = h.time_op("Cphi_eopre", MASS, H.EVEN, warmup=1, reps=reps, inp=src)
    t = med * 1e-6
    base = {"value": eopre_bytes(V) / t / 1e9, "unit": "GB/s", "cores": thr, "kind": "reference",
            "sample": f"HiRep's own Cphi_eopre (libhr built from the reference sources, gcc -O3 -fopenmp, "
                      f"OMP_PROC_BIND=close) on 16^3x32: median of {reps} applications after warm-up, "
                      f"{med / 1e3:.2f} ms (min {mn / 1e3:.2f} ms)",
            "note": "HiRep's Cphi_ (Dphi.c:1092-1146) shares its site temporaries between OpenMP threads, so "
                    "with more than one thread its clover result is not reliable; the time is HiRep's"}
    return base, t


def reference_main(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    base, t = cpu_reference_arm(args)
    if base["kind"] == "reference":
        base["port"] = cpu_port_arm(min(5.0, args.cpu_seconds))
    line = {"impl": "reference", "metric": METRIC, "value": base["value"],
            "unit": "GB/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": workload_config(), "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-solve", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched 22-system solve (24^3x48 sextet)")
    ap.add_argument("--no-force", action="store_true", help="skip the force check (16^4 SU(4) antisymmetric)")
    ap.add_argument("--no-hmc", action="store_true", help="skip the HMC trajectory (32^3x64 SU(2) adjoint)")
    ap.add_argument("--no-g5qmr", action="store_true", help="skip the HMC trajectory with HiRep's g5QMR force solves")
    ap.add_argument("--no-configs", action="store_true", help="skip the single-field operator at the other workloads")
    ap.add_argument("--hmc-only", action="store_true", help="only the HMC trajectories (32^3x64 SU(2) adjoint)")
    ap.add_argument("--force-only", action="store_true",
                    help="only the force leg, without finite differences (for profiling its kernels)")
    ap.add_argument("--dslash-config", type=int, default=None, metavar="K",
                    help="only the single-field operator leg of workload K of the other configurations "
                         "(0: 16^4 SU(4) antisymmetric, 1: 24^3x48 sextet clover, 2: 32^3x64 SU(2) adjoint)")
    ap.add_argument("--batch-op", default=None, metavar="TxXxYxZ",
                    help="only time the batched g5Cphi_eopre of the batched workload on this lattice")
    ap.add_argument("--nb", type=int, default=12, help="fields per batch for --batch-op")
    ap.add_argument("--prec", default="f", choices=["f", "d"], help="precision for --batch-op")
    ap.add_argument("--batch-variant", type=int, default=-1, help="batch kernel variant (-1: autotune)")
    ap.add_argument("--hop-variant", type=int, default=-1, help="hopping-kernel variant (-1: autotune)")
    ap.add_argument("--host-chunks", type=int, default=10, help="chunks of the host-field pipeline (e2e)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return reference_main(args)

    import torch

    from hirep_b200 import fields as F
    from hirep_b200 import hrgpu as G
    from hirep_b200.replicas import max_over_ranks, replica_rate

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if args.batch_op:
        return batch_op_main(args, torch, G, F)
    if args.dslash_config is not None:
        stream = torch.cuda.current_stream()
        flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
        peak, _ = measured_peak()
        out = run_dslash_configs(torch, stream, G, F, flush.zero_, peak, only=args.dslash_config)
        print(json.dumps({"dslash_configs": out}), flush=True)
        return
    if args.force_only:
        print(json.dumps({"force": run_force_check(torch, torch.cuda.current_stream(), G, F, fd=())}), flush=True)
        return
    if args.hmc_only:
        print(json.dumps({"hmc": run_hmc_check(torch, G, F, g5qmr=not args.no_g5qmr)}), flush=True)
        return
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    lat = G.Lattice(*DIMS, NG, G.FUND, device=local)
    G._check(lat.L.hrgpu_set_hop_variant(args.hop_variant), "set_hop_variant")
    u = F.smooth_gauge(SEED, lat.V, NG, EPS)
    lat.set_gauge(u)
    lat.represent_gauge_field(True)
    lat.clover_init(CSW)
    src = F.gaussian_spinor(SEED, lat.VH, lat.nf)
    fin, fout = lat.field(G.EVEN, host=src), lat.field(G.EVEN)
    nbytes = eopre_bytes(lat.V)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    flush_rd = torch.ones(64 << 20, dtype=torch.float64, device="cuda")  # 512 MB, read after the write

    def flush_l2():
        # write 512 MB, then read 512 MB: L2 ends up holding clean lines of an
        # unrelated buffer, so neither our data nor dirty flush data is left in it
        flush.zero_()
        flush_rd.sum()

    stream = torch.cuda.current_stream()

    for _ in range(args.warmup):
        lat.Cphi_eopre(MASS, fout, fin)
    torch.cuda.synchronize()
    lat.getMVM()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        time.sleep(0.3)  # let the sampler start
        # one more second of untimed steps right before the timed ones: the clock
        # record then covers the load the timed steps run under even when they
        # last only milliseconds (the record's window is this second + the timed region)
        clk.t0 = time.time()
        while time.time() - clk.t0 < 1.0:
            for _ in range(50):
                flush_l2()
                lat.Cphi_eopre(MASS, fout, fin)
            torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for a, b in evs:
            flush_l2()
            a.record(stream)
            lat.Cphi_eopre(MASS, fout, fin)
            b.record(stream)
        torch.cuda.synchronize()
        clk.t1 = time.time()
    launches = 2 * args.steps
    step_ms = sum(a.elapsed_time(b) for a, b in evs) / args.steps
    t_max = max_over_ranks(step_ms, dist, "cuda")
    value = replica_rate(nbytes, t_max, world) / 1e9

    # end to end through the C ABI with host (pinned) fields in HiRep's layout:
    # hrgpu_apply_op_host overlaps the chunked copies with the hops; the plain
    # sequence upload + operator + download is timed beside it
    h_in = torch.from_numpy(src.view(np.float64)).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    h2d = d2h = lat.VH * SPINOR_BYTES
    p_in, p_out = G.ctypes.c_void_p(h_in.data_ptr()), G.ctypes.c_void_p(h_out.data_ptr())

    def e2e_pipelined():
        G._check(lat.L.hrgpu_apply_op_host(G.OP_CPHI_EOPRE, G.D(MASS), p_out, p_in, G.DOUBLE), "apply_op_host")

    def e2e_sequential():
        G._check(lat.L.hrgpu_spinor_upload(fin.ptr, p_in, G.EVEN, G.DOUBLE), "upload")
        lat.Cphi_eopre(MASS, fout, fin)
        G._check(lat.L.hrgpu_spinor_download(p_out, fout.ptr, G.EVEN, G.DOUBLE), "download")

    def time_e2e(fn, extra_warmup=0):
        ts = []
        warm = args.warmup + extra_warmup
        for k in range(warm + min(args.steps, 200)):
            flush_l2()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            if k >= warm:
                ts.append(a.elapsed_time(b))
        return max_over_ranks(float(np.mean(ts)), dist, "cuda")

    lat.set_host_chunks(args.host_chunks)
    e2e_ms = time_e2e(e2e_pipelined, extra_warmup=32)  # the first 32 calls choose the form
    e2e_seq_ms = time_e2e(e2e_sequential)
    form, ms_pipe, ms_seq = G.ctypes.c_int(), G.ctypes.c_float(), G.ctypes.c_float()
    G._check(lat.L.hrgpu_host_form(G.ctypes.byref(form), G.ctypes.byref(ms_pipe), G.ctypes.byref(ms_seq)),
             "host_form")

    solve = None
    if not args.no_solve:
        solve = run_solves(lat, fin, torch, stream, G, dist)

    peak, peak_kind = measured_peak()
    ubytes = unique_bytes(lat.V, lat.nf, False, 2 if lat.link_recon() else 3, True)
    line = {
        "metric": METRIC,
        "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "config": workload_config(),
        "roofline": {"bound": "hbm", "achieved": ubytes / (t_max * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": ubytes / (t_max * 1e-3) / 1e9 / peak, "peak_kind": peak_kind,
                     "kernel": "k_hop (2 launches per Cphi_eopre)", "algorithmic_bytes_per_step": ubytes,
                     "algorithmic_bytes": "links once per hop (two rows when rebuilt), even input x2, odd "
                                          "temporary x2, even output, packed clover blocks once",
                     "hirep_model_bytes_per_step": nbytes, "traffic": profile_traffic()},
        "e2e": {"value": replica_rate(nbytes, e2e_ms, world) / 1e9, "unit": "GB/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "call": "hrgpu_apply_op_host(Cphi_eopre), pinned HiRep-layout fields",
                "form": {1: f"pipelined, {args.host_chunks} chunks", 2: "plain sequence"}.get(form.value, "eager"),
                "form_timing_ms": {"pipelined": ms_pipe.value, "sequential": ms_seq.value},
                "sequential_ms": e2e_seq_ms,
                "sequential_value": replica_rate(nbytes, e2e_seq_ms, world) / 1e9},
        "gpu_launches": launches,
        "hop_tuning": hop_tuning(lat, G),
        "clocks": clk.summary(),
    }
    if solve:
        line["solve"] = solve
    if world == 1 and not args.no_configs:
        line["dslash_configs"] = run_dslash_configs(torch, stream, G, F, flush_l2, peak)
    if world == 1 and not args.no_batch:
        line["solve_batch"] = run_batch_solves(torch, stream, G, F)
    if world == 1 and not args.no_force:
        line["force"] = run_force_check(torch, stream, G, F)
    if world == 1 and not args.no_hmc:
        line["hmc"] = run_hmc_check(torch, G, F, g5qmr=not args.no_g5qmr)
    if rank == 0 and world == 1 and not args.no_cpu:
        base, _ = cpu_reference_arm(args)
        line["cpu_baseline"] = base
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


# the single-field even-odd operator at the other workloads' sizes:
# (name, dims T,X,Y,Z, NG, representation, nf, real links, clover csw, m0, eps, seed)
DSLASH_CONFIGS = [
    ("SU(4) antisymmetric (NF=6), Wilson Dphi_eopre, 16^4, U=exp(i0.25H) seed 11", (16, 16, 16, 16), 4, "ASYM",
     None, -0.1, 0.25, 11),
    ("SU(3) symmetric (NF=6), clover csw=1.0 Cphi_eopre, 24^3x48, U=exp(i0.3H) seed 21", (48, 24, 24, 24), 3, "SYM",
     1.0, -0.3, 0.3, 21),
    ("SU(2) adjoint (NF=3, real), Wilson Dphi_eopre, 32^3x64, U=exp(i0.2H) seed 99", (64, 32, 32, 32), 2, "ADJ",
     None, -1.0, 0.2, 99),
]


def run_dslash_configs(torch, stream, G, F, flush_l2, peak, steps=50, only=None):
    """FP64 even-odd operator per workload: device time per application (L2
    flushed between steps, CUDA events), HiRep-model GB/s and the fraction of
    the measured HBM peak on the bytes it must move at least."""
    out = []
    for k, (name, dims, ng, rep, csw, m, eps, seed) in enumerate(DSLASH_CONFIGS):
        if only is not None and k != only:
            continue
        lat = G.Lattice(*dims, ng, getattr(G, rep))
        lat.set_gauge(F.smooth_gauge(seed, lat.V, ng, eps))
        lat.represent_gauge_field(True)
        if csw is not None:
            lat.clover_init(csw)
        real = rep == "ADJ"
        nf = lat.nf
        fin, fout = lat.field(G.EVEN, host=F.gaussian_spinor(seed, lat.VH, nf)), lat.field(G.EVEN)
        op = lat.Cphi_eopre if csw is not None else lat.Dphi_eopre
        for _ in range(5):
            op(m, fout, fin)
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            flush_l2()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            op(m, fout, fin)
            b.record(stream)
            ts.append((a, b))
        torch.cuda.synchronize()
        ms = float(np.mean([a.elapsed_time(b) for a, b in ts]))
        # HiRep's model (speed_test_diracoperator.c:82) + the clover blocks and the rho^2 input read
        vec, link = nf * 16, nf * nf * (8 if real else 16)
        model = lat.V * (36 * vec + 8 * link) + (lat.VH) * 4 * vec
        if csw is not None:
            model += lat.VH * (2 * nf * (2 * nf + 1) * 16 + 4 * nf * nf * 16)
        # the links the tuned kernels read: rows 0 and 1 (modes 1, 2), the
        # fundamental links (modes 3, 4, where the tuner chose variant 6), or all
        mode, tun = lat.link_recon(), hop_tuning(lat, G)
        used = ["f64_clover_inv", "f64_clover"] if csw is not None else ["f64_axpy"]
        fund = mode >= 3 and all(tun.get(k, {}).get("variant") == 6 for k in used)
        rows = 2 if mode in (1, 2) else nf
        ub = unique_bytes(lat.V, nf, real, rows, csw is not None, link_bytes=ng * ng * 16 if fund else None)
        extra = {}
        # the FP32 operator (the inner solves of the mixed-precision CG), same workload
        f32in = lat.field(G.EVEN, G.FLOAT, host=F.gaussian_spinor(seed, lat.VH, nf).astype(np.complex64))
        f32out = lat.field(G.EVEN, G.FLOAT)
        op32 = lat.g5Cphi_eopre_flt if csw is not None else lat.Dphi_eopre_flt
        for _ in range(5):
            op32(m, f32out, f32in)
        torch.cuda.synchronize()
        ts32 = []
        for _ in range(steps):
            flush_l2()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            op32(m, f32out, f32in)
            b.record(stream)
            ts32.append((a, b))
        torch.cuda.synchronize()
        extra["fp32_ms_per_application"] = float(np.mean([a.elapsed_time(b) for a, b in ts32]))
        t32 = hop_tuning(lat, G)
        extra["fp32_hop_tuning"] = {k: t32.get(k) for k in ("f32_axpy", "f32_clover_inv", "f32_clover") if k in t32}
        if csw is not None:
            # compute_clover_term (the clover term from the links; once per gauge field)
            ev = []
            for _ in range(5):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                lat.compute_clover_term()
                b.record(stream)
                ev.append((a, b))
            torch.cuda.synchronize()
            extra["compute_clover_term_ms"] = float(np.median([a.elapsed_time(b) for a, b in ev]))
        out.append({"workload": name, "ms_per_application": ms, "hirep_model_GBps": model / (ms * 1e-3) / 1e9, **extra,
                    "algorithmic_bytes": ub, "achieved_GBps": ub / (ms * 1e-3) / 1e9,
                    "frac_of_measured_hbm": ub / (ms * 1e-3) / 1e9 / peak,
                    "links_read": "fundamental" if fund else f"{rows} of {nf} rows",
                    "link_mode": mode, "hop_tuning": {k: tun.get(k) for k in used}})
    return out


def hop_tuning(lat, G):
    """Variant the autotuner picked for each tuned (precision, epilogue), with its timings."""
    out = {}
    names = {0: "axpy", 1: "clover_inv", 2: "clover"}
    for prec in (G.DOUBLE, G.FLOAT):
        for ep in range(3):
            chosen = G.ctypes.c_int(-1)
            ms = (G.ctypes.c_float * 7)()
            G._check(lat.L.hrgpu_hop_tuning(prec, ep, G.ctypes.byref(chosen), ms), "hop_tuning")
            if chosen.value >= 0:
                out[("f64" if prec == G.DOUBLE else "f32") + "_" + names[ep]] = {
                    "variant": chosen.value, "us_per_launch": [round(1e3 * x, 2) for x in ms]}
    return out


def run_solves(lat, fin, torch, stream, G, dist):
    """Plain FP64 CG vs FP32-inner defect correction on g5Cphi_eopre^2, |r|/|b| < 1e-12."""
    x64, x32 = lat.field(G.EVEN), lat.field(G.EVEN)
    out = {}
    for name, flt, x in (("fp64", False, x64), ("mixed", True, x32)):
        times, iters = [], None
        for rep in range(3):
            lat.la("zero", x)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            it, ok = lat.cg_mshift(G.OP_G5CPHI_EOPRE_SQ, MASS, [0.0], ERR2, fin, [x], flt=flt)
            b.record(stream)
            torch.cuda.synchronize()
            if rep > 0:
                times.append(a.elapsed_time(b))
            iters = it
        out[name + "_ms"] = float(np.median(times))
        out[name + "_mvm"] = iters
    # the same mixed solve with the FP32 operator reading BF16 links
    x16 = lat.field(G.EVEN)
    G._check(lat.L.hrgpu_set_flt_link_storage(G.LINKS_BF16), "set_flt_link_storage")
    try:
        times = []
        for rep in range(3):
            lat.la("zero", x16)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            it, ok = lat.cg_mshift(G.OP_G5CPHI_EOPRE_SQ, MASS, [0.0], ERR2, fin, [x16], flt=True)
            b.record(stream)
            torch.cuda.synchronize()
            if rep > 0:
                times.append(a.elapsed_time(b))
        out["mixed_bf16_links_ms"], out["mixed_bf16_links_mvm"], out["mixed_bf16_links_ok"] = (
            float(np.median(times)), it, bool(ok))
    finally:
        G._check(lat.L.hrgpu_set_flt_link_storage(G.LINKS_F32), "set_flt_link_storage")
    r = lat.field(G.EVEN)
    lat.g5Cphi_eopre_sq(MASS, r, x16)
    lat.la("sub_assign", r, fin)
    out["mixed_bf16_links_true_rel_residual"] = float(np.sqrt(lat.sqnorm(r) / lat.sqnorm(fin)))
    lat.g5Cphi_eopre_sq(MASS, r, x32)
    lat.la("sub_assign", r, fin)
    out["mixed_true_rel_residual"] = float(np.sqrt(lat.sqnorm(r) / lat.sqnorm(fin)))
    lat.la("sub_assign", x32, x64)
    out["mixed_vs_fp64_rel_error"] = float(np.sqrt(lat.sqnorm(x32) / lat.sqnorm(x64)))
    out["speedup_mixed_vs_fp64"] = out["fp64_ms"] / out["mixed_ms"]
    out["err2"] = ERR2
    return out


# batched workload: SU(3) two-index symmetric (NF = 6), clover csw = 1.0, m0 = -0.3,
# 24^3 x 48, U = exp(i 0.3 H) seed 21; the 12 spin-colour point sources at the
# origin (colours 0-2 x 4 spins), source 0 also for 10 shifts sigma log-spaced
# 1e-4 .. 10 (HiRep's shift = -sigma): 22 systems, |r|/|b| < 1e-12
B_DIMS, B_NG, B_MASS, B_CSW, B_EPS, B_SEED = (48, 24, 24, 24), 3, -0.3, 1.0, 0.3, 21


# force workload: SU(4) two-index antisymmetric (NF = 6), Wilson m0 = -0.1, 16^4,
# U = exp(i 0.25 H) seed 11, phi = D^+ eta (eta Gaussian, seed 11),
# S = phi^+ (H^2)^-1 phi with H = g5 D_eopre
F_DIMS, F_NG, F_MASS, F_EPS, F_SEED = (16, 16, 16, 16), 4, -0.1, 0.25, 11


def run_force_check(torch, stream, G, F, fd=((4, 1e-3), (4, 1e-4), (32, 1e-5))):
    """Pseudofermion force: kernel time, its roofline, and its error against
    central differences of S (fourth-order stencil) along random su(4)
    directions on every link, for each (number of directions, step) of fd; FP64
    solves to err2 = 1e-28.  S is about 8e5 here and a solve leaves it about
    1e-8 uncertain, so the error at small steps measures the solver, at large
    ones the stencil's truncation (~ step^4 / 30): the steps are reported side
    by side.  The links are moved on the device (U <- exp(eps i w.T) U with the
    direction w as momenta, update_gauge_field).  Also the force from an X
    solved by the FP32-inner defect-correction CG, against the FP64 force."""
    lat = G.Lattice(*F_DIMS, F_NG, G.ASYM)
    u0 = F.smooth_gauge(F_SEED, lat.V, F_NG, F_EPS)
    lat.set_gauge(u0)
    lat.represent_gauge_field(True)
    nf, V, VH = lat.nf, lat.V, lat.VH
    dimg = F_NG * F_NG - 1
    g5 = np.array([1, 1, -1, -1])[None, :, None]
    eta = F.gaussian_spinor(F_SEED, VH, nf)
    fe, tmp = lat.field(G.EVEN, host=g5 * eta), lat.field(G.EVEN)
    lat.Dphi_eopre(F_MASS, tmp, fe)
    phi = lat.field(G.EVEN, host=g5 * tmp.download())
    x, y = lat.field(G.EVEN), lat.field(G.EVEN)
    op = G.OP_G5DPHI_EOPRE_SQ

    def solve(flt=False, err2=1e-28):
        lat.la("zero", x)
        _, ok = lat.cg_mshift(op, F_MASS, [0.0], err2, phi, [x], flt=flt)
        assert ok
        return lat.prod_re(phi, x)

    Xs = np.zeros((V, 4, nf), complex)
    Ys = np.zeros_like(Xs)
    fX, fY = lat.field(G.FULL), lat.field(G.FULL)

    def force():
        lat.g5Dphi_eopre(F_MASS, y, x)
        Xs[:VH], Ys[:VH] = y.download(), x.download()
        fX.upload(Xs)
        fY.upload(Ys)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        lat.fermion_force_begin()
        a.record(stream)
        lat.force_fermion_core(fX, fY, 1, 1.0, 1.0)
        b.record(stream)
        f = lat.fermion_force_end(1.0, np.zeros((V, 4, dimg)))
        return f, a.elapsed_time(b)

    torch.cuda.synchronize()
    t0 = time.time()
    solve()
    solve_s = time.time() - t0
    f64, _ = force()
    core_ms = float(np.median([force()[1] for _ in range(5)]))
    by_variant = {}
    for v in (1, 2, 3, 4, 5, 6):  # the kernels of the hopping force (hrgpu_set_force_variant)
        G._check(lat.L.hrgpu_set_force_variant(v), "set_force_variant")
        fv, _ = force()
        by_variant[str(v)] = {"ms": float(np.median([force()[1] for _ in range(5)])),
                              "max_rel_diff_vs_default": float(np.abs(fv - f64).max() / np.abs(f64).max())}
    G._check(lat.L.hrgpu_set_force_variant(0), "set_force_variant")
    solve(flt=True, err2=1e-26)
    f32, _ = force()
    rng = np.random.default_rng(32)
    fd_out = []
    for ndir, step in fd:
        worst = 0.0
        for _ in range(ndir):
            w = rng.standard_normal((V, 4, dimg))

            def action(eps):
                lat.set_gauge(u0)
                lat.momenta_set(w)
                lat.update_gauge_field(eps)  # U <- exp(eps i w.T) U, represented again
                return solve()

            s1 = action(step) - action(-step)
            s2 = action(2 * step) - action(-2 * step)
            fd_val = (8 * s1 - s2) / (12 * step)
            an = float(-0.5 * np.sum(w * f64))
            worst = max(worst, abs(fd_val - an) / abs(an))
        fd_out.append({"directions": ndir, "step": step, "max_rel_err_fp64": worst})
    lat.set_gauge(u0)
    lat.represent_gauge_field(True)
    # the bytes the force must move at least: X and Y (full lattice), every
    # link once, the force planes read and written; plus the two odd-site fill
    # hops (links once each, the even half read, the odd half written)
    spin = 4 * nf * 16
    core_bytes = 2 * V * spin + 4 * V * nf * nf * 16 + 2 * 4 * V * dimg * 8
    # the fill hops read the fundamental links where the tuned hop kernel builds them
    fill_fund = lat.link_recon() >= 3 and hop_tuning(lat, G).get("f64_axpy", {}).get("variant") == 6
    fill_link = F_NG * F_NG * 16 if fill_fund else nf * nf * 16
    fill_bytes = 2 * (4 * V * fill_link + 2 * VH * spin)
    peak, _ = measured_peak()
    return {"workload": "SU(4) antisymmetric (NF=6), Wilson m0=-0.1, 16^4, U=exp(i0.25H) seed 11, "
                        "phi = D^+ eta; S = phi^+ (H^2)^-1 phi",
            "force_fermion_core_ms": core_ms, "fp64_solve_s": solve_s,
            "force_fermion_core_ms_by_variant": by_variant,
            "variants": "1: one thread per link; 2: two threads per link in two warps, projection table in "
                        "constant memory; 3: 2 with L2 prefetches of the link and the spinor at x; "
                        "4: 2 with the links built from the fundamental ones; 5: 2 with the link staged in "
                        "shared memory by cp.async (default); 6: 5 with the spinor at x staged too",
            "algorithmic_bytes": core_bytes + fill_bytes,
            "algorithmic_bytes_note": "X, Y, links and force planes (read + write) of the core, plus the two "
                                      "odd-site fill hops" + (" (fundamental links)" if fill_fund else ""),
            "achieved_GBps": (core_bytes + fill_bytes) / (core_ms * 1e-3) / 1e9,
            "frac_of_measured_hbm": (core_bytes + fill_bytes) / (core_ms * 1e-3) / 1e9 / peak,
            "fd": fd_out,
            "fd_method": "random su(4) directions on all links, 4th-order central differences",
            "fd_max_rel_err_fp64": max((r["max_rel_err_fp64"] for r in fd_out), default=None),
            "mixed_vs_fp64_force_rel_err": float(np.abs(f32 - f64).max() / np.abs(f64).max())}


# HMC workload: SU(2) adjoint (NF = 3, real), Nf = 2 Wilson m0 = -1.0, plaquette
# action beta = 2.25, 32^3 x 64, U = exp(i 0.2 H) seed 99; one trajectory of length 1,
# O2MN with 20 steps; force solves at |r|/|b| < 1e-10, accept/reject at 1e-14
H_DIMS, H_NG, H_BETA, H_MASS, H_EPS, H_SEED = (64, 32, 32, 32), 2, 2.25, -1.0, 0.2, 99


def run_hmc_check(torch, G, F, g5qmr=True):
    """One trajectory with mixed-precision force solves against the same trajectory
    (same random numbers) with plain FP64 force solves.  Each form first runs an
    untimed 2-step warm-up trajectory (kernel autotuning, CUDA-graph capture,
    work buffers), as every other timed leg has warm-up steps."""
    from hirep_b200.hmc import HMC

    lat = G.Lattice(*H_DIMS, H_NG, G.ADJ)
    u0 = F.smooth_gauge(H_SEED, lat.V, H_NG, H_EPS)
    out = {"workload": "SU(2) adjoint Nf=2 Wilson m0=-1.0 + plaquette beta=2.25, 32^3x64, U=exp(i0.2H) seed 99; "
                       "O2MN tau=1, 20 steps; force solves 1e-10, accept/reject 1e-14",
           "draws": "momenta and pseudofermion source drawn on the device (gaussian_momenta, "
                    "gaussian_spinor_field: Philox4x32-10, Box-Muller), inside the timed trajectory",
           "accept_reject": "correct_la_pf as FP64 CG on H^2 then H (accept_reject_mvm counts H^2 applications)"}
    for name, solver in (("mixed", "cg_mixed"), ("fp64", "cg")):
        lat.set_gauge(u0)
        lat.represent_gauge_field(True)
        HMC(lat, H_BETA, H_MASS, tau=0.1, nsteps=2, force_err2=1e-20, mt_err2=1e-28,
            force_solver=solver, draws="device").trajectory(np.random.default_rng(H_SEED + 1), metropolis=False)
        lat.set_gauge(u0)
        lat.represent_gauge_field(True)
        plaq0 = lat.avr_plaquette()
        hmc = HMC(lat, H_BETA, H_MASS, tau=1.0, nsteps=20, force_err2=1e-20, mt_err2=1e-28, force_solver=solver,
                  draws="device")
        torch.cuda.synchronize()
        r = hmc.trajectory(np.random.default_rng(H_SEED), metropolis=False)
        out[name] = {"seconds": r["seconds"], "dH": r["dH"], "force_solve_mvm": r["force_solve_iters"],
                     "force_evaluations": r["force_evaluations"], "accept_reject_mvm": r["mt_iters"],
                     "plaquette_start": plaq0, "plaquette_end": lat.avr_plaquette()}
    out["speedup_mixed_vs_fp64"] = out["fp64"]["seconds"] / out["mixed"]["seconds"]
    out["dH_difference"] = out["mixed"]["dH"] - out["fp64"]["dH"]
    if g5qmr:
        # HiRep's own formulation of the same force solves (force_hmc.c:122-155): two
        # g5QMR solves on D per force from the chronological MRE guess over 4 past
        # solutions, and HiRep's g5QMR accept/reject solve on D
        lat.set_gauge(u0)
        lat.represent_gauge_field(True)
        hmc = HMC(lat, H_BETA, H_MASS, tau=1.0, nsteps=20, force_err2=1e-20, mt_err2=1e-28, force_solver="g5qmr",
                  draws="device", mre_past=4, mt_solver="g5qmr")
        torch.cuda.synchronize()
        r = hmc.trajectory(np.random.default_rng(H_SEED), metropolis=False)
        out["g5qmr_mre4"] = {"seconds": r["seconds"], "dH": r["dH"], "force_solve_mvm": r["force_solve_iters"],
                             "accept_reject_mvm": r["mt_iters"],
                             "note": "HiRep's own force formulation: two g5QMR solves on D from the MRE guess; "
                                     "MVM = D applications"}
    return out


def batch_op_main(args, torch, G, F):
    """Time the batched g5Cphi_eopre alone (the batched workload's operator) on one lattice."""
    T, X, Y, Z = (int(v) for v in args.batch_op.split("x"))
    lat = G.Lattice(T, X, Y, Z, B_NG, G.SYM)
    lat.set_gauge(F.smooth_gauge(B_SEED, lat.V, B_NG, B_EPS))
    lat.represent_gauge_field(True)
    lat.clover_init(B_CSW)
    G._check(lat.L.hrgpu_set_batch_variant(args.batch_variant), "set_batch_variant")
    prec = G.FLOAT if args.prec == "f" else G.DOUBLE
    dt = np.complex64 if prec == G.FLOAT else np.complex128
    fs = [lat.field(G.EVEN, prec, host=F.gaussian_spinor(i, lat.VH, lat.nf).astype(dt)) for i in range(args.nb)]
    bi, bo = lat.batch(args.nb, prec, fields=fs), lat.batch(args.nb, prec)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        lat.apply_op_batch(G.OP_G5CPHI_EOPRE, B_MASS, bo, bi)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(args.steps):
        lat.apply_op_batch(G.OP_G5CPHI_EOPRE, B_MASS, bo, bi)
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / args.steps
    # bytes that must move per application: links and clover blocks once per hop,
    # the fields in and out of each hop (and the aux read of the second)
    esz = 8 if prec == G.FLOAT else 16
    nf = lat.nf
    links = 2 * lat.V * 4 * nf * nf * esz  # both hops read every link
    clover = lat.V * 2 * (2 * nf * esz // 2 + nf * (2 * nf - 1) * esz)  # one packed block pair per site and hop
    fields = args.nb * lat.VH * 4 * nf * esz * 5  # hop 1: in, out; hop 2: in, aux, out
    nbytes = links + clover + fields
    print(json.dumps({"batch_op": args.batch_op, "nb": args.nb, "prec": args.prec, "variant": args.batch_variant,
                      "ms_per_application": ms, "ms_per_field": ms / args.nb, "bytes_per_application": nbytes,
                      "GBps": nbytes / (ms * 1e-3) / 1e9}), flush=True)


def run_batch_solves(torch, stream, G, F):
    """22 systems in one batched mixed-precision solve vs 22 sequential FP64 solves."""
    lat = G.Lattice(*B_DIMS, B_NG, G.SYM)
    u = F.smooth_gauge(B_SEED, lat.V, B_NG, B_EPS)
    lat.set_gauge(u)
    lat.represent_gauge_field(True)
    lat.clover_init(B_CSW)
    sig = np.logspace(-4, 1, 10)
    shifts = [[0.0] + list(-sig)] + [[0.0] for _ in range(11)]
    srcs = [lat.field(G.EVEN, host=F.point_source(lat.VH, lat.nf, spin=b, col=c)) for c in range(3) for b in range(4)]
    xb = [lat.field(G.EVEN) for sh in shifts for _ in sh]
    xs = [lat.field(G.EVEN) for sh in shifts for _ in sh]
    op = G.OP_G5CPHI_EOPRE_SQ

    def timed(fn):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        r = fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b), r

    out = {"workload": "SU(3) sym (NF=6), clover csw=1.0, m0=-0.3, 24^3x48, U=exp(i0.3H) seed 21; "
                       "12 point sources + 10 shifts 1e-4..10 on source 0 = 22 systems",
           "err2": ERR2}
    # warm-up: kernel tuning and graph captures happen on first use
    lat.cg_mshift_batch(op, B_MASS, srcs, shifts, ERR2, xb, flt=True)
    ms, (its, ok) = timed(lambda: lat.cg_mshift_batch(op, B_MASS, srcs, shifts, ERR2, xb, flt=True))
    out["batch_mixed_ms"], out["batch_mixed_ok"] = ms, bool(ok)
    out["batch_mixed_iters_per_source"] = [int(i) for i in its]
    lat.cg_mshift_batch(op, B_MASS, srcs, shifts, ERR2, xs, flt=False)
    ms, (its, ok) = timed(lambda: lat.cg_mshift_batch(op, B_MASS, srcs, shifts, ERR2, xs, flt=False))
    out["batch_fp64_ms"], out["batch_fp64_ok"] = ms, bool(ok)
    # sequential FP64: HiRep's cg_mshift one system at a time (zero start)
    tmp = lat.field(G.EVEN)
    lat.g5Cphi_eopre_sq(B_MASS, tmp, srcs[0])  # tunes the single-field kernels

    def sequential():
        j, n_it, all_ok = 0, 0, True
        for s, sh in enumerate(shifts):
            for sg in sh:
                lat.la("zero", xs[j])
                it, ok = lat.cg_mshift(op, B_MASS, [sg], ERR2, srcs[s], [xs[j]])
                n_it += it
                all_ok = all_ok and ok
                j += 1
        return n_it, all_ok

    ms, (n_it, ok) = timed(sequential)
    out["sequential_fp64_ms"], out["sequential_fp64_ok"], out["sequential_fp64_mvm"] = ms, bool(ok), int(n_it)
    # errors of the batched mixed solutions: against the sequential FP64 ones, and
    # true residuals with the FP64 single-field operator
    j, err, res = 0, 0.0, 0.0
    for s, sh in enumerate(shifts):
        for sg in sh:
            lat.g5Cphi_eopre_sq(B_MASS, tmp, xb[j])
            lat.la("mul_add_assign", tmp, -sg, xb[j])
            lat.la("sub_assign", tmp, srcs[s])
            res = max(res, float(np.sqrt(lat.sqnorm(tmp) / lat.sqnorm(srcs[s]))))
            lat.la("copy", tmp, xb[j])
            lat.la("sub_assign", tmp, xs[j])
            err = max(err, float(np.sqrt(lat.sqnorm(tmp) / lat.sqnorm(xs[j]))))
            j += 1
    out["batch_mixed_max_true_rel_residual"] = res
    out["batch_mixed_max_rel_error_vs_fp64"] = err
    out["speedup_batch_mixed_vs_sequential_fp64"] = out["sequential_fp64_ms"] / out["batch_mixed_ms"]
    out["speedup_batch_fp64_vs_sequential_fp64"] = out["sequential_fp64_ms"] / out["batch_fp64_ms"]
    for q in (G.DOUBLE, G.FLOAT):
        for ep in (1, 2):
            ch, tms = G.ctypes.c_int(), (G.ctypes.c_float * 6)()
            lat.L.hrgpu_batch_tuning(q, ep, 12, G.ctypes.byref(ch), tms)
            out[f"tuning_{'f64' if q == G.DOUBLE else 'f32'}_ep{ep}_nb12"] = [ch.value] + [round(t, 4) for t in tms]
    return out


if __name__ == "__main__":
    main()
