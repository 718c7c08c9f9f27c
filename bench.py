"""Benchmark: chi0 + Sigma_c on one B200 (GFLOP/s), plain FP64 vs split FP16.

One step = the hot path over one batch of synthetic input:
  * chi0(q, iw) of the GaAs-like configuration (N=600, nk=216, nocc=9,
    nunocc U{100..300} per k, 24 imaginary frequencies), all k and all iw in
    one call (qsgw_chi0_lorentz_d), and
  * the Sigma_c band sum of 64 tasks (one per q of W_c), each N=600,
    40 target x 400 intermediate states, 24 iw + w=0 and the real-axis pole
    part on a 50-point mesh (qsgw_sxcf_correlation_d per task).
Inputs are seeded synthetic data with the configurations' shapes and value
distributions; W_c(q, iw) is built by this library's own chi0 -> W path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision split-i8|split-f16|fp64] [--slices 3]
    python bench.py --impl reference ...   # the reference's CPU path (oracle)

N > 1 runs N independent replicas (the path needs no collective; the
reference's q/k partitions are independent), timed as the max over ranks.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "chi0+Sigma_c time & GFLOP/s on 1 B200, mixed vs FP64 plain, at QP err <=1 meV"


# ----------------------------------------------------------------------------- helpers
# DRAM bytes (read + write) of one split-precision Sigma_c task launch
# (N=600, 40 x 400 states, 25 imaginary slots + real-axis pole columns),
# measured with ncu on that launch, per kernel of the path.
# split-i8: the 3-slice launch (base-256 digits), the count the automatic choice makes on
# this workload: both launches of the task (full row tiles 1.284e9 B, paired last row tile 0.087e9 B).
SIGC_TC_TRAFFIC = {"split-f16": 3.315e9, "split-i8": 1.371e9}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


from ecalj_b200.replicas import max_over_ranks  # noqa: E402


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ----------------------------------------------------------------------------- workload
def chi0_config(nk=None):
    from ecalj_b200 import synth
    c = dict(synth.CONFIGS["chi0_n600"])
    if nk:
        c["nk"] = nk
    rng = np.random.default_rng(c["seed"])
    nocc, nun, eocc, eun = synth.chi0_spectrum(rng, c["nk"], c["nocc"], c["nun"])
    mesh = synth.imag_mesh(c["niw"])
    npair = int(np.sum(nocc * nun))
    return dict(N=c["N"], nk=c["nk"], niw=c["niw"], nocc=nocc, nun=nun,
                eocc_h=np.concatenate(eocc) * 0.5, eun_h=np.concatenate(eun) * 0.5,
                npair=npair, seed=c["seed"], **mesh)


def sigc_config():
    from ecalj_b200 import synth
    return dict(synth.CONFIGS["sigc_n600"])


def device_normal_c128(n, seed, scale):
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    t = torch.empty(2 * n, dtype=torch.float64, device="cuda")
    t.normal_(0.0, scale, generator=g)
    return t.view(torch.complex128)


def build_sigc_inputs(lib, c, log):
    """W_c(q, iw) for every q from this library's chi0 -> W path (the N=260
    pair model scaled to N=600, iw = 0 plus the 24 Gauss-Legendre points), a real-axis
    model on the 50-point mesh, and zmel per task.  All device-resident."""
    import torch
    from ecalj_b200 import synth
    from ecalj_b200 import sched
    N, niw, ntq, nm = c["N"], c["niw"], c["ntq"], c["nm"]
    mesh = synth.imag_mesh(niw)
    fr = synth.freq_r_mesh(c["nreal"])
    freqs = np.concatenate([[0.0], mesh["freq_i"]])            # slot 0 = w = 0
    nf = niw + 1
    vsq, q = synth.coulomb(N, c["seed"] + 1)
    m2e = lib.to_device(q)
    tasks = []
    t0 = time.time()
    for iq in range(c["nq"]):
        rng = np.random.default_rng(c["seed"] * 1000 + iq)
        nocc_a, nun_a, eocc, eun = synth.chi0_spectrum(rng, c["chi_nk"], c["chi_nocc"], c["chi_nun"])
        npair = int(np.sum(nocc_a * nun_a))
        z = device_normal_c128(N * npair, c["seed"] * 7919 + iq, 1.0 / math.sqrt(N))
        chi = torch.zeros(N * N * nf, dtype=torch.complex128, device="cuda")
        lib.chi0_lorentz_d(chi, N, nf, freqs, c["chi_nk"], nocc_a, nun_a,
                           np.concatenate(eocc) * 0.5, np.concatenate(eun) * 0.5, z)
        del z
        wi = torch.zeros(N * N * nf, dtype=torch.complex128, device="cuda")
        lib.wvi_llw(chi, 2, vsq, m2e, True, True, 2, zw=wi, device=True, ngb=N, niw=nf)
        del chi
        g = torch.tensor(1.0 / (1.0 + (fr / 0.5) ** 2), dtype=torch.float64, device="cuda")
        wr = (wi[:N * N].view(1, N * N) * g.view(-1, 1)).reshape(-1).contiguous()
        trng = np.random.default_rng(c["seed"] * 31 + iq)
        omega = np.sort(trng.uniform(-1.0, 1.0, ntq))
        ekc = np.sort(trng.uniform(-1.0, 4.0, nm))
        zmel = device_normal_c128(N * nm * ntq, c["seed"] * 104729 + iq, 1.0 / math.sqrt(N))
        ef, esmr = 0.0, 0.01
        nwxi, nwx, ntmax = sched.get_nwx(omega, ekc, fr, ef, esmr)
        ns2r = min(nm, ntmax)
        tasks.append(dict(wi=wi, wr=wr, zmel=zmel, omega=omega, ekc=ekc, ef=ef, esmr=esmr,
                          nwxi=nwxi, nwx=nwx, ns2r=ns2r))
    lib.synchronize()
    log(f"sigc inputs: {c['nq']} W stacks built on the GPU in {time.time() - t0:.1f}s")
    return dict(tasks=tasks, mesh=mesh, fr=fr, N=N, niw=niw, ntq=ntq, nm=nm, wkkr=1.0 / c["nq"])


def sigc_flops(lib, s):
    """Algorithmic FLOPs of the Sigma_c step, counted as the reference's GEMMs
    execute them: 8 N^2 (nm ntq) per iw (0..niw), 8 N^2 per pole column and
    real bin, 8 ntq^2 N nm for the final contraction."""
    from ecalj_b200 import sched
    N, nm, ntq, niw = s["N"], s["nm"], s["ntq"], s["niw"]
    f_imag = 8.0 * N * N * nm * ntq * (niw + 1)
    f_fin = 8.0 * ntq * ntq * N * nm
    tot_pole = 0.0
    for t in s["tasks"]:
        ent, _ = sched.pole_bins(t["omega"], t["ekc"], s["fr"], t["ef"], t["esmr"], t["nwxi"], t["nwx"],
                                 t["ns2r"], nm, ntq)
        nb = sum(1 for _, x in ent for j in range(3) if t["nwxi"] <= x - 1 + j <= t["nwx"])
        tot_pole += 8.0 * N * N * nb
    return len(s["tasks"]) * (f_imag + f_fin) + tot_pole, len(s["tasks"]) * f_imag + tot_pole


def run_sigc(lib, s, host=None):
    """Every Sigma_c task of the step: device arrays through one qsgw_sxcf_correlation_batch_d call,
    host arrays (the end-to-end run) through qsgw_sxcf_correlation task by task."""
    m = s["mesh"]

    def kw(t, src):
        return dict(zsec=src["zsec"], zmel=src["zmel"], ns1=1, ns2=s["nm"], ns2r=t["ns2r"], nwxi=t["nwxi"],
                    nwx=t["nwx"], ntqxx=s["ntq"], wc_imag=src["wi"], wc_real=src["wr"], omega=t["omega"],
                    ekc=t["ekc"], nctot=0, ef=t["ef"], esmr=t["esmr"], wkkr=s["wkkr"], ua=m["ua"], freqx=m["x"],
                    wwx=m["wx"], expa=m["expa"], freq_r=s["fr"], nblochpmx=s["N"], ngb=s["N"], ntq=s["ntq"])

    if host is None:
        lib.sxcf_correlation_batch_d([kw(t, t) for t in s["tasks"]])
        return
    for i, t in enumerate(s["tasks"]):
        lib.sxcf_correlation(**kw(t, host["tasks"][i]), keepwv=host.get("keepwv", False))


_PACK_IDX = {}


def pack_upper_device(torch, w, n, nrec, hermitize):
    """W records (n x n, column-major, nrec of them, device) in ecalj's keepwv layout: the upper
    triangle of each record in column order (j, i <= j); real-axis records symmetrised first,
    (W(i,j) + conj(W(j,i)))/2, as the keepwv mode stores them (m_sxcf_gemm.f90:327-358)."""
    m = w.view(nrec, n, n)                               # [record][column j][row i]
    if hermitize:
        m = 0.5 * (m + m.transpose(1, 2).conj())
    key = (n, str(w.device))
    if key not in _PACK_IDX:
        j = torch.arange(n, device=w.device)
        cols = torch.repeat_interleave(j, j + 1)         # j of each packed entry
        rows = torch.arange(cols.numel(), device=w.device) - (cols * (cols + 1)) // 2
        _PACK_IDX[key] = (cols, rows)
    cols, rows = _PACK_IDX[key]
    return m[:, cols, rows].reshape(-1).contiguous()


# ----------------------------------------------------------------------------- reference arm
def reference_arm(args, ws, rank):
    """The reference's CPU path (the oracle restatement on numpy/OpenBLAS with
    every host thread) on a bounded sample of the same workload."""
    if rank != 0:
        return
    from threadpoolctl import threadpool_info
    from oracle import sxcf as osx
    from ecalj_b200 import synth
    cfg_chi = chi0_config()
    N, niw = cfg_chi["N"], cfg_chi["niw"]
    rng = np.random.default_rng(1)
    P_s = 3000
    z = synth.zmel_columns(rng, N, P_s)
    de = rng.uniform(0.025, 2.0, P_s)
    w = -2.0 * de[:, None] / (de[:, None] ** 2 + cfg_chi["freq_i"][None, :] ** 2) / cfg_chi["nk"]
    cfg_sig = sigc_config()
    nm_s = 100
    t = synth.sigc_task(cfg_sig["N"], cfg_sig["ntq"], nm_s, cfg_sig["niw"], cfg_sig["nreal"], seed=5, esmr=0.01, ef=0.0)
    wi = synth.zmel_columns(rng, N, N * (cfg_sig["niw"] + 1)).reshape(N, N, cfg_sig["niw"] + 1, order="F") * 0.01
    wr = synth.real_axis_model(wi[:, :, 0], t["freq_r"])
    nt0p, nt0m = osx.nt0pm(t["ekc"], t["ef"], t["esmr"])
    nwxi, nwx, ntmax = osx.get_nwx(t["omega"], cfg_sig["ntq"], nt0p, nt0m, nm_s, t["freq_r"], t["esmr"], t["ef"],
                                   t["ekc"], 0)
    fl_chi = 8.0 * N * N * P_s * niw
    npole = len(osx.pole_table(t["omega"], t["ekc"], 0, 1, min(nm_s, ntmax), cfg_sig["ntq"], t["ef"], t["esmr"],
                               1.0, t["freq_r"]))
    fl_sig = 8.0 * N * N * nm_s * cfg_sig["ntq"] * (cfg_sig["niw"] + 1) + 8.0 * N * N * 3 * npole \
        + 8.0 * cfg_sig["ntq"] ** 2 * N * nm_s

    def step():
        acc = np.zeros((N, N), complex)
        zh = z.conj().T.copy()
        for iw in range(niw):                       # x0gemm: one ZGEMM per bin
            acc += zh.T @ (z.T * w[:, iw:iw + 1])
        zs = np.zeros((cfg_sig["ntq"], cfg_sig["ntq"]), complex, order="F")
        osx.correlation_block(zs, t["zmel"], 1, nm_s, min(nm_s, ntmax), nwxi, nwx, cfg_sig["ntq"], wi, wr, t["omega"],
                              t["ekc"], 0, t["ef"], t["esmr"], 1.0, t["ua"], t["x"], t["wx"], t["expa"], t["freq_r"])
        return acc, zs

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    gf = (fl_chi + fl_sig) / dt / 1e9
    threads = max([d.get("num_threads", 1) for d in threadpool_info()] + [1])
    sample = (f"chi0 {P_s} of {cfg_chi['npair']} pairs x {niw} iw at N={N}; Sigma_c 1 task with {nm_s} of "
              f"{cfg_sig['nm']} intermediate states x {cfg_sig['ntq']} targets, {cfg_sig['niw']}+1 iw, "
              f"{npole} pole columns")
    cpu = {"value": round(gf, 3), "unit": "GFLOP/s", "cores": threads, "kind": "port", "sample": sample}
    line = {"metric": METRIC, "value": round(gf, 3), "unit": "GFLOP/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": "chi0 N=600 + Sigma_c N=600 (bounded CPU sample)", "sample": sample},
            "impl": "reference", "cpu_baseline": cpu,
            "e2e": {"value": round(gf, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="split-i8", choices=["split-i8", "split-f16", "fp64"],
                    help="headline precision; a split mode also times the FP64 path for the comparison")
    ap.add_argument("--slices", type=int, default=0,
                    help="int8 slices per operand of split-i8 (2..4); 0 = chosen per contraction by the "
                         "library's accuracy targets (QP 1 meV for Sigma_c, 2e-5 relative for chi0)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the W_c frequency-interpolator study")
    ap.add_argument("--no-c4", action="store_true", help="skip the N=1500 all-in study (configuration c4)")
    ap.add_argument("--c4-k", type=int, default=16, help="k points of the 512 timed in the c4 study")
    ap.add_argument("--no-graph", action="store_true", help="time eager calls instead of CUDA-graph replays")
    ap.add_argument("--no-autotune", action="store_true", help="heuristic launch parameters only")
    ap.add_argument("--nq", type=int, default=None, help="Sigma_c tasks (default: the configuration's 64)")
    ap.add_argument("--nk", type=int, default=None, help="k-points of the chi0 part (profiling only)")
    ap.add_argument("--case", choices=["sigc", "chi0"], default=None,
                    help="kernel case for ncu: three calls of one contraction of the workload (one Sigma_c "
                         "task, or chi0 with --nk k points) in the chosen precision, no timing, no JSON line")
    args = ap.parse_args()
    ws, rank, local = dist_setup()
    log = (lambda m: print(f"[bench] {m}", file=sys.stderr, flush=True)) if rank == 0 else (lambda m: None)
    if args.impl == "reference":
        reference_arm(args, ws, rank)
        return
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    from ecalj_b200 import lib
    lib.load()
    lib.init(local)
    lib.share_torch_stream()
    if not args.no_autotune:
        lib.set_autotune(1, None)          # the first (untimed) call of each shape picks its split-K
    prec = args.precision
    split = prec != "fp64"
    modes = {"fp64": (lib.PREC_FP64, 1), "split-f16": (lib.PREC_SPLIT_F16, 2),
             "split-i8": (lib.PREC_SPLIT_I8, args.slices)}
    peaks, peak_src = load_peaks()
    if args.case:
        kernel_case(lib, torch, args, modes[prec], log)
        return

    # ---- workload set-up (untimed)
    lib.set_precision(lib.PREC_FP64)
    cfg_chi = chi0_config(args.nk)
    N, niw = cfg_chi["N"], cfg_chi["niw"]
    zc = device_normal_c128(N * cfg_chi["npair"], cfg_chi["seed"], 1.0 / math.sqrt(N))
    chi = torch.zeros(N * N * niw, dtype=torch.complex128, device="cuda")
    cfg_sig = sigc_config()
    if args.nq:
        cfg_sig["nq"] = args.nq
    s = build_sigc_inputs(lib, cfg_sig, log)
    for t in s["tasks"]:
        t["zsec"] = torch.zeros(s["ntq"] * s["ntq"], dtype=torch.complex128, device="cuda")
    fl_chi = 8.0 * N * N * cfg_chi["npair"] * niw
    fl_sig, fl_sig_seg = sigc_flops(lib, s)
    flops = fl_chi + fl_sig

    def step():
        lib.chi0_lorentz_d(chi, N, niw, cfg_chi["freq_i"], cfg_chi["nk"], cfg_chi["nocc"], cfg_chi["nun"],
                           cfg_chi["eocc_h"],
                           cfg_chi["eun_h"], zc)
        for t in s["tasks"]:
            t["zsec"].zero_()
        run_sigc(lib, s)

    def timed(mode, steps, warmup, sample_clocks, graph=False):
        """Warm-up steps, then `steps` timed steps: eager calls, or replays of
        one step recorded as a CUDA graph (launch count and per-kernel times of
        a replay are those recorded, scaled by the number of replays)."""
        lib.set_precision(*modes[mode])
        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        lib.profile(True)
        per_step = None
        if graph:
            l0 = lib.launch_count()
            lib.graph_begin()
            step()
            lib.graph_end()
            per_step = lib.launch_count() - l0
            lib.graph_launch()                           # one untimed replay
            torch.cuda.synchronize()
        run = lib.graph_launch if graph else step
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.start()
        l0 = lib.launch_count()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(steps):
            run()
        ev1.record()
        torch.cuda.synchronize()
        launches = per_step * steps if graph else lib.launch_count() - l0
        ms = ev0.elapsed_time(ev1) / steps
        kt = {tag: lib.profile_get(tag) for tag in ("chi0_dmma", "sigc_seg_dmma", "gemm_dmma", "chi0_tc",
                                                   "sigc_seg_tc", "chi0_slice_i8", "sigc_slice_i8")}
        if graph:                                        # the latest replay's times, for every replay
            kt = {k: (v[0] * steps, v[1] * steps) for k, v in kt.items()}
            lib.graph_destroy()
        lib.profile(False)
        clocks = sampler.stop() if sampler else None
        if ws > 1:
            ms = max_over_ranks(ms, dist, "cuda")
            dist.barrier()
        return ms, kt, launches, clocks

    # ---- headline run: one step recorded as a CUDA graph and replayed (eager timing beside it)
    ms_eager = None
    if not args.no_graph:
        ms_eager, _, _, _ = timed(prec, max(1, min(args.steps, 3)), args.warmup, False)
    ms, kt, launches, clocks = timed(prec, args.steps, args.warmup, True, graph=not args.no_graph)
    value = ws * flops / (ms * 1e-3) / 1e9
    chi_main = chi.clone()
    zsec_main = [t["zsec"].clone() for t in s["tasks"]]

    # ---- the other precision, same workload, same run (the metric compares them)
    compare = None
    if split and not args.no_compare:
        ms64, kt64, _, _ = timed("fp64", args.steps, 1, False, graph=not args.no_graph)
        d_chi = float(torch.linalg.vector_norm(chi_main - chi) / torch.linalg.vector_norm(chi))
        num = sum(float(torch.linalg.vector_norm(a - t["zsec"]) ** 2) for a, t in zip(zsec_main, s["tasks"]))
        den = sum(float(torch.linalg.vector_norm(t["zsec"]) ** 2) for t in s["tasks"])
        qp = max(float(torch.max(torch.abs(torch.real(a - t["zsec"]).view(s["ntq"], s["ntq"]).diagonal())))
                 for a, t in zip(zsec_main, s["tasks"])) * 27211.386245988
        compare = {"fp64_ms_per_step": round(ms64, 3), "fp64_value": round(ws * flops / (ms64 * 1e-3) / 1e9, 3),
                   "speedup_split_vs_fp64": round(ms64 / ms, 3),
                   "fp64_steps": args.steps,
                   "fp64_kernel_ms": {k: round(v[0] / args.steps, 3) for k, v in kt64.items() if v[1]},
                   "chi0_rel_err_vs_fp64": d_chi, "sigc_rel_err_vs_fp64": math.sqrt(num / den),
                   "qp_err_mev_max": qp}
        # The configurations fix W but not the normalisation of zmel; with
        # re, im ~ N(0, 1/N) the Sigma_c diagonal is hundreds of Hartree.  The
        # error scales linearly with |Sigma_c|, so it is also quoted with
        # Sigma_c rescaled to a mean |Re Sigma_c,nn| of 5 eV (Si/GaAs-like).
        dmean = float(np.mean([float(torch.mean(torch.abs(torch.real(t["zsec"]).view(s["ntq"], s["ntq"]).diagonal())))
                               for t in s["tasks"]])) * 27.211386245988
        compare.update({"sigc_diag_mean_abs_ev": dmean, "qp_err_mev_max_at_5ev_sigma": qp * 5.0 / dmean,
                        "qp_gate_1mev_met": qp <= 1.0})
        lib.set_precision(*modes[prec])

    # ---- roofline of the dominant kernel
    if split:
        dom_tag, dom_flops = "sigc_seg_tc", fl_sig_seg
    else:
        dom_tag, dom_flops = "sigc_seg_dmma", fl_sig_seg
    k_ms, k_n = kt[dom_tag]
    per_launch_ms = k_ms / max(k_n, 1)
    achieved = (dom_flops * args.steps / max(k_n, 1)) / (per_launch_ms * 1e-3) / 1e12 if k_n else None
    fp64_peak = measure_fp64_peak()
    i8_peak = None
    slices_used = chosen_slices(lib, args.slices, (f"={N} ", f"niw={niw}")) if prec == "split-i8" else None
    if prec == "split-i8":
        i8_peak = measure_int8_peak()
        ns_sig = slices_used["sigc"]
        nprod = ns_sig * (ns_sig + 1) // 2
        peak = i8_peak["sustained_tops"] / nprod
        peak_note = (f"int8 tensor peak measured in this run (torch._int_mm, 8192^3, sustained "
                     f"{i8_peak['sustained_tops']:.1f} TOP/s) / {nprod} (int8 slice products per "
                     f"FP64-equivalent product at {ns_sig} slices)")
    elif prec == "split-f16":
        peak = peaks["bf16_tflops_sustained"] / 3.0
        peak_note = (f"{peak_src} bf16 sustained {peaks['bf16_tflops_sustained']} TFLOP/s / 3 "
                     f"(3 FP16 slice products per FP64-equivalent product)")
    else:
        peak = fp64_peak
        peak_note = "cuBLAS ZGEMM (complex128, 4096^3) measured in this run; MEASURED_PEAKS.json has no FP64 figure"
    # Sigma_c tasks per launch of the dominant kernel (the int8 path batches the step's tasks; a batch is
    # a launch over the full row tiles plus one over the paired last row tile): the per-launch figures
    # below are averages over the step's launches of the kernel
    tasks_per_launch = len(s["tasks"]) * args.steps / max(k_n, 1)
    traffic = SIGC_TC_TRAFFIC.get(prec)
    roof = {"bound": "tensor", "achieved": round(achieved, 3) if achieved else None, "peak": round(peak, 3),
            "unit": "TFLOP/s", "frac": round(achieved / peak, 4) if achieved else None,
            "traffic": traffic * tasks_per_launch if traffic else None,
            "traffic_source": (f"dram__bytes_read.sum + dram__bytes_write.sum of the kernel's launches on one "
                               f"Sigma_c task of the same shape from ncu ({traffic:.4g} B), times the "
                               f"{tasks_per_launch:g} tasks a launch runs on average" if traffic else "not captured"),
            "tasks_per_launch": tasks_per_launch,
            "kernel": dom_tag, "launch_ms": round(per_launch_ms, 4), "peak_source": peak_note,
            "algorithmic_flops_per_launch": dom_flops * args.steps / max(k_n, 1)}

    # ---- end-to-end through the host-pointer entry points (pinned host buffers)
    e2e = None
    if not args.no_e2e:
        lib.set_precision(*modes[prec])
        # the full-record run first: its pinned buffers are the larger, and the keepwv run's fit in them
        full = run_e2e(lib, torch, cfg_chi, zc, s, args, flops, ws, dist, keepwv=False)
        release_pinned(torch)
        e2e = run_e2e(lib, torch, cfg_chi, zc, s, args, flops, ws, dist, keepwv=True)
        release_pinned(torch)
        e2e["full_w_records"] = {k: full[k] for k in ("value", "ms_per_step", "h2d_bytes_per_step")}
        # the copy bound of the step: its host -> device bytes at this box's pinned copy rate
        gbs = measure_h2d_gbs()
        e2e["h2d_pinned_gbs"] = round(gbs, 2)
        e2e["h2d_bound_ms"] = round(e2e["h2d_bytes_per_step"] / (gbs * 1e9) * 1e3, 1)
        e2e["full_w_records"]["h2d_bound_ms"] = round(full["h2d_bytes_per_step"] / (gbs * 1e9) * 1e3, 1)
        log(f"e2e: {e2e['ms_per_step']} ms/step (keepwv), copy bound {e2e['h2d_bound_ms']} ms at {gbs:.1f} GB/s "
            f"pinned host -> device; full records {full['ms_per_step']} ms, bound "
            f"{e2e['full_w_records']['h2d_bound_ms']} ms")
    sur = None
    if not args.no_surrogate:
        lib.set_autotune(0, None)          # no tuning trials inside the study's timed calls
        sur = surrogate_summary(lib, log, precision=prec if split else "fp64", nslices=args.slices)
        lib.set_precision(*modes[prec])
    c4 = None
    if split and not args.no_c4:
        lib.set_autotune(0, None)
        c4 = c4_study(lib, torch, log, modes, prec, args.c4_k)
        lib.set_precision(*modes[prec])
    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = cpu_baseline()
    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": {"fp64": "c128", "split-f16": "c128 via 2 FP16 slices, 3 products",
                                               "split-i8": "c128 via int8 slices (Ozaki), exact INT32 accumulation"
                                               }[prec],
                "data": "synthetic",
                "config": {"workload": f"chi0 (N=600, nk={cfg_chi['nk']}, nocc=9, nunocc U{{100..300}}, 24 iw, "
                                       f"{cfg_chi['npair']} pairs) + Sigma_c ({len(s['tasks'])} tasks, N=600, "
                                       "40x400 states, 24+1 iw, 50-point real mesh)",
                           "precision": prec, "slices": slices_used, "parallelism": f"replicas x{ws}",
                           "execution": "CUDA graph replay" if not args.no_graph else "eager calls",
                           "eager_ms_per_step": round(ms_eager, 3) if ms_eager else None,
                           "l2": "inputs exceed L2 (zmel columns 3.73 GB)",
                           "flops_per_step": flops, "flops_chi0": fl_chi, "flops_sigc": fl_sig},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clocks, "kernel_ms": {k: round(v[0] / args.steps, 3) for k, v in kt.items() if v[1]},
                "fp64_peak_tflops": round(fp64_peak, 3), "int8_peak": i8_peak, "compare": compare, "surrogate": sur,
                "c4": c4,
                "autotune": lib.autotune_report()}
        if compare and cpu and cpu.get("value"):
            # both FP64: this library's plain GPU path over the CPU restatement (same flop count)
            compare["fp64_gpu_over_fp64_cpu"] = round(compare["fp64_value"] / cpu["value"], 3)
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


def kernel_case(lib, torch, args, mode, log):
    """Three calls of one contraction of the workload, for a profiler: the third
    launch of the contraction's kernel is the one to capture (-s 2 -c 1)."""
    lib.set_autotune(0, None)
    if args.case == "chi0":
        lib.set_precision(lib.PREC_FP64)
        cfg = chi0_config(args.nk)
        N, niw = cfg["N"], cfg["niw"]
        zc = device_normal_c128(N * cfg["npair"], cfg["seed"], 1.0 / math.sqrt(N))
        chi = torch.zeros(N * N * niw, dtype=torch.complex128, device="cuda")
        lib.set_precision(*mode)
        for _ in range(3):
            lib.chi0_lorentz_d(chi, N, niw, cfg["freq_i"], cfg["nk"], cfg["nocc"], cfg["nun"], cfg["eocc_h"],
                               cfg["eun_h"], zc)
        log(f"chi0 case: N={N}, nk={cfg['nk']}, {cfg['npair']} pairs, {niw} iw")
    else:
        lib.set_precision(lib.PREC_FP64)
        c = sigc_config()
        c["nq"] = 1
        s = build_sigc_inputs(lib, c, log)
        for t in s["tasks"]:
            t["zsec"] = torch.zeros(s["ntq"] * s["ntq"], dtype=torch.complex128, device="cuda")
        lib.set_precision(*mode)
        for _ in range(3):
            run_sigc(lib, s)
        log("Sigma_c case: one task of the workload")
    lib.synchronize()


def c4_study(lib, torch, log, modes, prec, nk_timed=16):
    """Configuration c4, all in, at N = 1500 (nk = 512, nocc = 40, nunocc U{300..1200}, 32 iw):
    chi0 streamed k by k through qsgw_chi0_lorentz_acc_d (zmel of each k generated on the device,
    720 MB per k) on the first nk_timed of the 512 k with the weights of the whole mesh, the time
    extrapolated linearly in k; W = (1 - v chi0)^-1 v on all 33 slots (iw = 0 and the 32 points);
    one Sigma_c task of 400 x 40 states on that W.  The split path (its chi0 -> W -> Sigma_c chain)
    against the FP64 path (its own chain): times, speed-up and the QP error of the whole chain.
    The oracle checks chi0 of k = 0 on 2 seeded frequencies."""
    from ecalj_b200 import synth, sched
    from oracle import x0
    c = synth.CONFIGS["chi0_n1500_streamed"]
    N, nk, niw = c["N"], c["nk"], c["niw"]
    rng = np.random.default_rng(c["seed"])
    nocc, nun, eocc, eun = synth.chi0_spectrum(rng, nk, c["nocc"], c["nun"])
    mesh = synth.imag_mesh(niw)
    freqs = np.concatenate([[0.0], mesh["freq_i"]])
    nf = niw + 1
    ks = list(range(nk_timed))
    npair_k = [int(nocc[k] * nun[k]) for k in ks]
    p_timed, p_all = sum(npair_k), int(np.sum(nocc * nun))
    zs = [device_normal_c128(N * npair_k[k], c["seed"] * 7919 + k, 1.0 / math.sqrt(N)) for k in ks]
    vsq, q = synth.coulomb(N, c["seed"] + 1)
    m2e = lib.to_device(q)
    trng = np.random.default_rng(c["seed"] + 3)
    ntq, nm = 40, 400
    omega = np.sort(trng.uniform(-1.0, 1.0, ntq))
    ekc = np.sort(trng.uniform(-1.0, 4.0, nm))
    zmel = device_normal_c128(N * nm * ntq, c["seed"] * 31 + 1, 1.0 / math.sqrt(N))
    fr = synth.freq_r_mesh(50)
    ef, esmr, wkkr = 0.0, 0.01, 1.0 / 64
    nwxi, nwx, ntmax = sched.get_nwx(omega, ekc, fr, ef, esmr)
    ns2r = min(nm, ntmax)
    ev = lambda: torch.cuda.Event(enable_timing=True)
    out = {}
    for name in (prec, "fp64"):
        lib.set_precision(*modes[name])
        chi = torch.zeros(N * N * nf, dtype=torch.complex128, device="cuda")
        # untimed first call: scratch allocation (the accumulating calls run no trials)
        lib.chi0_lorentz_acc_d(chi, N, nf, freqs, nk, nocc[:1], nun[:1], eocc[0] * 0.5, eun[0] * 0.5, zs[0])
        chi.zero_()
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record()
        for k in ks:
            lib.chi0_lorentz_acc_d(chi, N, nf, freqs, nk, nocc[k:k + 1], nun[k:k + 1], eocc[k] * 0.5, eun[k] * 0.5,
                                   zs[k])
        e1.record()
        torch.cuda.synchronize()
        t_chi = e0.elapsed_time(e1)
        wi = torch.zeros(N * N * nf, dtype=torch.complex128, device="cuda")
        e0, e1 = ev(), ev()
        e0.record()
        lib.wvi_llw(chi, 2, vsq, m2e, True, True, 2, zw=wi, device=True, ngb=N, niw=nf)
        e1.record()
        torch.cuda.synchronize()
        t_w = e0.elapsed_time(e1)
        g = torch.tensor(1.0 / (1.0 + (fr / 0.5) ** 2), dtype=torch.float64, device="cuda")
        wr = (wi[:N * N].view(1, N * N) * g.view(-1, 1)).reshape(-1).contiguous()
        zsec = torch.zeros(ntq * ntq, dtype=torch.complex128, device="cuda")
        sargs = (1, nm, ns2r, nwxi, nwx, ntq, wi, wr, omega, ekc, 0, ef, esmr, wkkr, mesh["ua"], mesh["x"],
                 mesh["wx"], mesh["expa"], fr)
        lib.sxcf_correlation(zsec, zmel, *sargs, device=True, ngb=N, ntq=ntq)   # untimed: slice trials, scratch
        zsec.zero_()
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record()
        lib.sxcf_correlation(zsec, zmel, *sargs, device=True, ngb=N, ntq=ntq)
        e1.record()
        torch.cuda.synchronize()
        out[name] = dict(chi=chi, wi=wi, zsec=zsec.view(ntq, ntq), t_chi=t_chi, t_w=t_w,
                         t_sig=e0.elapsed_time(e1))
        del wr
        log(f"c4 {name}: chi0 {t_chi:.1f} ms on {nk_timed} k, W {t_w:.1f} ms, Sigma_c {out[name]['t_sig']:.1f} ms")
    a, b = out[prec], out["fp64"]
    rel = lambda x, y: float(torch.linalg.vector_norm(x - y) / torch.linalg.vector_norm(y))
    qp = float(torch.max(torch.abs(torch.real(a["zsec"].diagonal() - b["zsec"].diagonal())))) * 27211.386245988
    fl_chi = 8.0 * N * N * p_timed * nf
    scale = p_all / p_timed
    tot = {n: out[n]["t_chi"] * scale + out[n]["t_w"] + out[n]["t_sig"] for n in out}
    # the oracle on a seeded subset: chi0 of k = 0 on 2 of the frequencies
    sel = np.sort(np.random.default_rng(c["seed"] + 9).choice(nf, 2, replace=False))
    z0 = zs[0].cpu().numpy().reshape(N, int(nocc[0]), int(nun[0]), order="F")
    ref = x0.chi0_direct([z0], x0.lorentz_pair_tables([eocc[0] * 0.5], [eun[0] * 0.5], 2, freqs[sel], nk), N, 2)[:, :, 1:]
    oracle_err = {}
    for name in (prec, "fp64"):
        lib.set_precision(*modes[name])
        ch = torch.zeros(N * N * 2, dtype=torch.complex128, device="cuda")
        lib.chi0_lorentz_acc_d(ch, N, 2, freqs[sel], nk, nocc[:1], nun[:1], eocc[0] * 0.5, eun[0] * 0.5, zs[0])
        lib.synchronize()
        got = ch.cpu().numpy().reshape(N, N, 2, order="F")
        oracle_err[name] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    res = {"workload": f"N=1500, nk=512 (chi0 timed on {nk_timed} k streamed, {p_timed} of {p_all} pairs, "
                       "extrapolated linearly), nocc=40, nunocc U{300..1200}, 32 iw + w=0; W on 33 slots; "
                       "one Sigma_c task of 400 x 40 states, 50-point real mesh",
           "precision": prec,
           "chi0_ms_timed": {n: round(out[n]["t_chi"], 2) for n in out},
           "chi0_gflops_timed": {n: round(fl_chi / (out[n]["t_chi"] * 1e-3) / 1e9, 1) for n in out},
           "chi0_s_per_q_extrapolated": {n: round(out[n]["t_chi"] * scale * 1e-3, 3) for n in out},
           "w_ms": {n: round(out[n]["t_w"], 2) for n in out},
           "sigc_ms": {n: round(out[n]["t_sig"], 2) for n in out},
           "total_s_per_q_extrapolated": {n: round(tot[n] * 1e-3, 3) for n in out},
           "speedup_vs_fp64": round(tot["fp64"] / tot[prec], 3),
           "chi0_rel_err_vs_fp64": rel(a["chi"], b["chi"]), "w_rel_err_vs_fp64": rel(a["wi"], b["wi"]),
           "sigc_rel_err_vs_fp64_chain": rel(a["zsec"], b["zsec"]),
           "qp_err_mev_max_chain": qp, "qp_gate_1mev_met": qp <= 1.0,
           "oracle_chi0_k0_2iw_rel_err": oracle_err, "oracle_frequencies": [int(i) for i in sel],
           "slices": chosen_slices(lib, modes[prec][1], (f"={N} ",)) if prec == "split-i8" else None}
    del out, zs
    torch.cuda.empty_cache()
    return res


def surrogate_summary(lib, log, nq_test=8, precision="split-i8", nslices=3):
    """W_c(q, iw) on the 48-point imaginary grid (N=600, Sigma_c configuration
    generator): the plain method (every frequency exact, FP64 and split) against
    the split path with the learned frequency interpolator (17 of 49 slots
    exact, validated, fallback above 1 meV), on q points not trained on."""
    from ecalj_b200 import surrogate
    res = surrogate.study(N=600, nq_train=48, nq_test=nq_test, precision=precision, log=log, nslices=nslices)
    rows = res["rows"]
    mean = lambda k: float(np.mean([r[k] for r in rows]))
    out = {"workload": "W_c interpolation: exact W_c on 48 iw x 48 training q at N=600, 8 anchors, 8 held-out, "
                       "32 predicted; "
                       f"{nq_test} test q",
           "ms_w_plain_fp64": round(mean("ms_plain_fp64"), 3), "ms_w_plain_split": round(mean("ms_plain"), 3),
           "ms_w_surrogate": round(mean("ms_surrogate"), 3),
           "speedup_vs_plain_fp64": round(mean("ms_plain_fp64") / mean("ms_surrogate"), 3),
           "speedup_vs_plain_split": round(mean("ms_plain") / mean("ms_surrogate"), 3),
           "phases_ms": {k: round(mean(k), 3) for k in ("exact_ms", "predict_ms", "validate_ms", "fallback_ms")},
           "fallbacks": int(sum(r["fallback"] for r in rows)),
           "qp_err_mev_max_vs_fp64_plain": max(r["qp_mev_final_vs_fp64"] for r in rows),
           "qp_err_mev_max_prediction": max(r["trained"]["qp_mev"] for r in rows),
           "qp_err_mev_max_linear_interp": max(r["linear"]["qp_mev"] for r in rows),
           "qp_err_mev_max_least_squares": max(r["lsq"]["qp_mev"] for r in rows),
           "w_rel_err": {k: mean_d(rows, k) for k in ("linear", "lsq", "trained")},
           "est_over_true": [round(r["est_mev"] / max(r["trained"]["qp_mev"], 1e-12), 2) for r in rows],
           "train_seconds": round(res["train_seconds"], 3), "train_samples": res["train_samples"],
           "qp_scale": "Sigma_c normalised to a mean |Re Sigma_c,nn| of 5 eV"}
    return out


def mean_d(rows, k):
    return {"full": float(np.mean([r[k]["w_rel"] for r in rows])),
            "dominant_block": float(np.mean([r[k]["w_rel_block"] for r in rows]))}


def chosen_slices(lib, requested, match=()):
    """int8 slices per operand of the chi0 and Sigma_c contractions: the requested
    count, or the automatic choices the library recorded for the shapes whose keys hold
    every string of match (e.g. "=600 " for npr / ngb = 600, "niw=24").  A chi0 shape with
    no record ran only accumulating calls, which take 3 slices when no choice was made."""
    if requested:
        return {"chi0": requested, "sigc": requested, "products": {"chi0": requested * (requested + 1) // 2,
                                                                   "sigc": requested * (requested + 1) // 2}}
    rep = lib.autotune_report()
    mine = lambda k: all(m in k for m in match)
    pick = lambda pre, dflt: max((v for k, v in rep.items() if k.startswith(pre) and "err@" not in k and mine(k)),
                                 default=dflt)
    ns = {"chi0": pick("chi0_i8 slices", 3), "sigc": pick("sigc_i8 slices", 4)}
    ns["products"] = {k: v * (v + 1) // 2 for k, v in list(ns.items())}
    ns["estimates"] = {k: v for k, v in rep.items() if "err@" in k and mine(k)}
    return ns


def measure_int8_peak():
    """int8 tensor throughput of a library GEMM (torch._int_mm, int8 x int8 -> int32,
    8192^3, 2 n^3 ops): best of 5 (burst) and back to back for 2 s (sustained) --
    the denominator of the int8 Ozaki path (a measurement only)."""
    import torch
    n = 8192
    a = torch.randint(-64, 65, (n, n), dtype=torch.int8, device="cuda")
    b = torch.randint(-64, 65, (n, n), dtype=torch.int8, device="cuda")
    torch._int_mm(a, b)
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(); torch._int_mm(a, b); e1.record(); torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    reps = max(1, int(2.0 / (2.0 * n ** 3 / (best * 1e12))))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        torch._int_mm(a, b)
    e1.record(); torch.cuda.synchronize()
    sus = reps * 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12
    del a, b
    return {"burst_tops": round(best, 1), "sustained_tops": round(sus, 1), "reps": reps}


def measure_h2d_gbs():
    """Pinned host -> device copy rate of this box (1 GiB, cudaMemcpyAsync through torch,
    best of 5): the bound of the end-to-end step's input copies (a measurement only)."""
    import torch
    n = 1 << 30
    h = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    d = torch.empty(n, dtype=torch.uint8, device="cuda")
    d.copy_(h, non_blocking=True)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(); d.copy_(h, non_blocking=True); e1.record(); torch.cuda.synchronize()
        best = max(best, n / (e0.elapsed_time(e1) * 1e-3) / 1e9)
    del h, d
    release_pinned(torch)
    return best


def measure_fp64_peak():
    """cuBLAS complex128 GEMM throughput (8 n^3 flops), best of 3 -- the FP64
    tensor-pipe denominator (a measurement only)."""
    import torch
    n = 4096
    a = torch.randn(n, n, dtype=torch.complex128, device="cuda")
    b = torch.randn(n, n, dtype=torch.complex128, device="cuda")
    torch.matmul(a, b)
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(); torch.matmul(a, b); e1.record(); torch.cuda.synchronize()
        best = max(best, 8.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    return best


def run_e2e(lib, torch, cfg_chi, zc, s, args, flops, ws, dist, keepwv=True):
    """Same step through the host-pointer C-ABI entry points: every step copies
    its inputs from pinned host memory and reads the results back.  The calls
    run in the library's asynchronous host mode (each returns once enqueued,
    so one call's copies overlap the previous call's kernels) and every step
    ends with qsgw_synchronize, after which its outputs are on the host.
    keepwv: the W records are held on the host in ecalj's keepwv layout (packed
    upper triangles, half the bytes of the full records); else as full records."""
    N, niw = cfg_chi["N"], cfg_chi["niw"]
    zc_h = torch.empty(zc.numel(), dtype=torch.complex128, pin_memory=True)
    zc_h.copy_(zc)
    chi_h = torch.empty(N * N * niw, dtype=torch.complex128, pin_memory=True)
    host = {"tasks": [], "keepwv": keepwv}
    h2d = zc_h.numel() * 16
    rec = N * (N + 1) // 2 if keepwv else N * N              # complex elements per W record
    for t in s["tasks"]:
        d = {}
        src = {"zmel": t["zmel"]}
        if keepwv:
            src["wi"] = pack_upper_device(torch, t["wi"], N, s["niw"] + 1, False)
            src["wr"] = pack_upper_device(torch, t["wr"], N, len(s["fr"]), True)
        else:
            src["wi"], src["wr"] = t["wi"], t["wr"]
        for k in ("zmel", "wi", "wr"):
            d[k] = torch.empty(src[k].numel(), dtype=torch.complex128, pin_memory=True)
            d[k].copy_(src[k])
        del src
        d["zsec"] = torch.zeros(s["ntq"] * s["ntq"], dtype=torch.complex128, pin_memory=True)
        for k in ("zmel", "wi", "wr", "zsec"):
            d[k] = d[k].numpy().reshape(-1)
        d["zmel"] = d["zmel"].reshape((s["N"], s["nm"], s["ntq"]), order="F")
        d["wi"] = d["wi"].reshape((rec, s["niw"] + 1), order="F")
        d["wr"] = d["wr"].reshape((rec, len(s["fr"])), order="F")
        d["zsec"] = d["zsec"].reshape((s["ntq"], s["ntq"]), order="F")
        host["tasks"].append(d)
        h2d += t["zmel"].numel() * 16 + 16 * rec * (s["niw"] + 1) + 16 * s["ntq"] ** 2
        h2d += 16 * rec * n_real_records(t, s)
    d2h = chi_h.numel() * 16 + len(s["tasks"]) * 16 * s["ntq"] ** 2
    zc_np = zc_h.numpy()
    chi_np = chi_h.numpy()

    def chi0():
        lib.chi0_lorentz_d(chi_np, N, niw, cfg_chi["freq_i"], cfg_chi["nk"], cfg_chi["nocc"], cfg_chi["nun"],
                           cfg_chi["eocc_h"], cfg_chi["eun_h"], zc_np, host=True)

    def step():
        # chi0 first: the step is bound by its host -> device copies (the device work is shorter),
        # so chi0's 67 ms of kernels run under the Sigma_c copies instead of after the last copy
        for d in host["tasks"]:
            d["zsec"][:] = 0
        chi0()
        run_sigc(lib, s, host=host)
        lib.synchronize()

    lib.set_host_async(True)
    step()
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    t0 = time.perf_counter()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    nst = args.steps
    for _ in range(nst):
        step()
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / nst
    lib.set_host_async(False)
    if ws > 1:
        ms = max_over_ranks(ms, dist, "cuda")
    del host
    return {"value": round(ws * flops / (ms * 1e-3) / 1e9, 3), "unit": "GFLOP/s",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "ms_per_step": round(ms, 3),
            "steps": nst, "api": "qsgw_chi0_lorentz + qsgw_sxcf_correlation (host pointers, "
                                 "qsgw_set_host_async(1), one qsgw_synchronize per step)",
            "w_layout": ("keepwv: W records as packed upper triangles (ecalj --keepwv layout, half the bytes)"
                         if keepwv else "full W records")}


def release_pinned(torch):
    """Return the pinned host blocks torch keeps cached (tens of GB after an end-to-end run)."""
    import gc
    gc.collect()
    fn = getattr(torch._C, "_host_emptyCache", None)
    if fn is not None:
        fn()


def n_real_records(t, s):
    from ecalj_b200 import sched
    return len(sched.pole_bins(t["omega"], t["ekc"], s["fr"], t["ef"], t["esmr"], t["nwxi"], t["nwx"],
                               t["ns2r"], s["nm"], s["ntq"])[1])


def cpu_baseline():
    """The oracle (numpy/OpenBLAS, all host threads) on a bounded sample,
    run in a child process so its threads do not share this process."""
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], capture_output=True, text=True, env={**os.environ, "WORLD_SIZE": "1",
                                                                              "RANK": "0"})
    for ln in r.stdout.splitlines():
        if ln.startswith("{"):
            return json.loads(ln)["cpu_baseline"]
    return {"value": None, "unit": "GFLOP/s", "cores": None, "kind": "port", "sample": r.stderr[-300:]}


if __name__ == "__main__":
    main()
