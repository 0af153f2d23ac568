"""Benchmark: GW self-consistency iterations per second on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config c2] [--slices 5]

One step is one iteration of the self-consistency loop of mbpt.exe on the
c2 workload (nk = 125 (5x5x5), nao = 40, naux = 250, ns = 1, ntau = 120,
nw = 120, beta = 200, eps ~ U[-5,5] Ha): HF Fock build, GW self-energy
(P0 -> W -> Sigma, split-precision contractions with 5 INT8 slices of balanced
rounded digits), chemical-potential search and Dyson step, energies.  Inputs are seeded synthetic data with the shapes and
distributions of that configuration (no public dataset exists for it).

Timing: W untimed warm-up steps, then K timed steps bracketed by a barrier and
cudaDeviceSynchronize, CUDA events on the library's stream, max over ranks.
`value` times the iteration with G already in HBM; `e2e` adds, every step, the
copy of G from pinned host memory and the copy of the new G back.  G (384 MB)
and V (100 GB) are larger than L2, so no flush is needed.

With N > 1 (torchrun) the q loop is sharded across ranks and the partial
self-energies are summed with an NCCL all-reduce before the Dyson step.

--impl reference times the CPU oracle (numpy/BLAS restatement of the
reference's gw_cpu_kernel, hf_cpu_kernels and dyson) on a bounded sample of the
same workload on the host cores and extrapolates to one iteration.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "green-mbpt_b200"))

import numpy as np  # noqa: E402

METRIC = "GW iterations/s at nk=125,nao=40: split-prec vs FP64 on B200, max|ΔΣ|≤1e-8"
# DRAM bytes (read + write) per FP64-equivalent flop of the tensor-core contraction kernel, from
# one ncu capture of its six launch shapes on the c2-shaped profiling case (c2k2) with the current
# kernel (profiles/split_gemm_tc_c2k2.md): 8.25 GB for 3.80e11 flops.  Each shape's traffic scales
# with its k-point batch as its flops do, so the roofline traffic per launch is this ratio times
# the step's flops per launch.
TC_DRAM_BYTES_PER_FLOP = 8.25e9 / 3.80e11
UNIT = "iterations/s"
WORKLOADS = {
    "c2": "c2: nk=125 (5x5x5), nao=40, naux=250, ns=1, ntau=120, nw=120, beta=200, eps~U[-5,5]",
    "c1": "c1: nk=64 (4x4x4), nao=26, naux=150, ns=2, ntau=100, beta=100, eps~U[-2,2]",
    "c0": "c0: nk=8 (2x2x2), nao=10, naux=40, ns=1, ntau=60, beta=100, eps~U[-2,2]",
    "c2k2": "c2k2: c2's shapes (nao=40, naux=250, ntau=120, nw=120) on a 2x1x1 mesh (nk=2): profiling case",
    "c4": "c4: nk=27 (3x3x3), nao=20, naux=100, ns=1, ntau=80, beta=100, eps~U[-2,2]: differentiable step",
}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
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
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return d.get("bf16_tflops_sustained", 1412.1), d.get("hbm_gbs", 6546.2), "measured"
    return 1400.0, 6650.0, "fallback"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_baseline(cfg: str, seed: int, nks: int = 3):
    """Time the CPU oracle on a bounded sample and extrapolate to one iteration (seconds).

    Sample: q = 0 with `nks` k-points for the polarization and the self-energy (work per
    (q,k) is uniform, so the full cost is nk*nq/nks times it), the screened-interaction
    solve of that q (times nq), the HF exchange row of one k (times nk*ns) and the Dyson
    step and eigen-spectra of one k (times nk).
    """
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import gw_oracle as O
    from gb200 import synth

    s = synth.make_config(cfg, seed=seed, with_integrals=False)
    g = s.grid
    rng = np.random.default_rng(seed + 1)
    nk, ns, NQ, nts, nao = s.nk, s.ns, s.NQ, s.nts, s.nao
    bz = O.NoSymBZ(s.mesh)
    q = 0
    ks = list(range(min(nks, nk)))
    Vp = {k: synth.random_pair(rng, NQ, nao, hermitian=(bz.k1_from_k2q(k, q) == k)) for k in ks}
    Vm = {k: synth.random_pair(rng, NQ, nao, hermitian=(bz.k2_from_k1q(k, q) == k)) for k in ks}
    t0 = time.perf_counter()
    P0 = np.zeros((nts, NQ, NQ), dtype=np.complex128)
    for k in ks:
        O.eval_P0_tilde(s.G, Vp[k], k, bz.k1_from_k2q(k, q), P0, ns)
    t1 = time.perf_counter()
    O.symmetrize_P0(P0, nk)
    P = O.eval_P_tilde(P0, g.Tnt_b, g.Ttn_b)
    t2 = time.perf_counter()
    Sig = np.zeros_like(s.G)
    for k in ks:
        O.eval_selfenergy(s.G, Vm[k], k, bz.k2_from_k1q(k, q), P, Sig, ns)
    t3 = time.perf_counter()
    # HF exchange row of k = 0 over all k' (the dominant HF term)
    dm = O.hf_density(s.G, ns)
    th0 = time.perf_counter()
    pref = 1.0 if ns == 2 else 0.5
    Frow = np.zeros((nao, nao), dtype=np.complex128)
    for kp in range(nk):
        v = synth.random_pair(rng, NQ, nao)
        vmm = v.reshape(NQ * nao, nao)
        Y = (vmm @ dm[0, kp]).reshape(NQ, nao * nao)
        Frow -= pref * (Y.T.copy().reshape(nao, nao * NQ) @ np.conj(vmm).T.copy().reshape(nao * NQ, nao)) / nk
    th1 = time.perf_counter()
    # Dyson step and eigen-spectra of one k
    one = slice(0, 1)
    F1 = np.zeros((ns, 1, nao, nao), dtype=np.complex128)
    td0 = time.perf_counter()
    O.selfenergy_eigenspectra(F1, Sig[:, :, one], s.F[:, one], s.S[:, one], g.Tnt_f)
    O.compute_G(F1, Sig[:, :, one], s.F[:, one], s.S[:, one], 0.0, g.Tnt_f, g.Ttn_f, g.wsample_f)
    td1 = time.perf_counter()
    per_qk = ((t1 - t0) + (t3 - t2)) / len(ks)
    est = per_qk * nk * nk + (t2 - t1) * nk + (th1 - th0) * nk * ns + (td1 - td0) * nk
    sample_s = (t3 - t0) + (th1 - th0) + (td1 - td0)
    desc = (f"q=0 with {len(ks)} of {nk} k for P0 and Sigma, W solve of that q, HF exchange row of one k, "
            f"Dyson + eigen-spectra of one k; {sample_s:.1f} s measured, scaled by the uniform per-(q,k) work")
    return est, desc, sample_s


def blas_threads():
    try:
        from threadpoolctl import threadpool_info
        n = [i.get("num_threads", 0) for i in threadpool_info() if i.get("user_api") == "blas"]
        return max(n) if n else os.cpu_count()
    except Exception:
        return os.cpu_count()


def setup_context(cfg, seed, slices, device, ws, rank, contraction_slices=None, engine=0):
    from gb200 import lib, shard, solvers, synth

    s = synth.make_config(cfg, seed=seed, with_integrals=False)
    g = s.grid
    ctx = lib.Context(s.nk, s.nao, s.ns, s.NQ, g.nts, g.nw, g.nw_b, s.beta, device=device)
    kp, km = solvers.kq_maps(s.mesh)
    ctx.set_kq_maps(kp, km)
    ctx.set_grid(g.Tnt_f, g.Ttn_f, g.Tnt_b, g.Ttn_b, g.wsample_f)
    if ws > 1:
        # q-sharded: this rank keeps only the integral pairs of its q range
        q0, q1 = shard.q_shard(s.nk, ws, rank)
        synth.upload_device_integral_pairs(ctx, s.nk, s.NQ, s.nao, shard.pairs_for_q_range(kp, q0, q1), seed=seed,
                                           device=device)
        ctx.set_q_range(q0, q1)
    else:
        synth.upload_device_integrals(ctx, s.nk, s.NQ, s.nao, seed=seed, device=device)
    ctx.set_hamiltonian(s.F, s.S)
    ctx.set_precision(lib.PREC_SPLIT, slices)
    ctx.set_split_engine(engine)
    if contraction_slices:
        ctx.set_contraction_slices(contraction_slices)
    return s, ctx


def run_ours(args):
    import torch

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(minutes=15))
    from gb200 import lib, shard

    s, ctx = setup_context(args.config, args.seed, args.slices, local, ws, rank, args.contraction_slices,
                           args.engine)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    # the library runs on torch's stream, so its work is ordered with the copies around it; a null
    # handle would select the context's own non-blocking stream, so the default stream is passed
    # by its legacy handle
    sptr = stream.cuda_stream or 0x1
    G0 = torch.from_numpy(s.G).pin_memory()
    Gout = torch.empty_like(G0).pin_memory()
    G = torch.empty(s.G.shape, dtype=torch.complex128, device=dev)
    S1 = torch.zeros((s.ns, s.nk, s.nao, s.nao), dtype=torch.complex128, device=dev)
    St = torch.zeros(s.G.shape, dtype=torch.complex128, device=dev)
    Sdev = torch.from_numpy(s.S).to(dev)
    dm = torch.empty_like(S1)
    nel = s.nel_from_G0()
    tol, mad = 1e-9, 0.0
    state = {"mu": 0.0, "E": None}

    def iteration():
        if ws == 1:
            # the chemical-potential search starts from the previous iteration's mu, as the
            # reference's dyson object does (its _mu persists across iterations, dyson.cpp:101-174)
            state["mu"], state["E"] = ctx.iteration_device(G.data_ptr(), S1.data_ptr(), St.data_ptr(), mad, nel, tol,
                                                           state["mu"], stream=sptr)
            return
        # q-sharded GW and HF exchange (each rank holds the integral pairs of its q range): the
        # partial Fock matrices and self-energies are summed before the Dyson step
        dm.copy_(G[-1] * (-1.0 if s.ns == 2 else -2.0))
        ctx.hf_fock_device(dm.data_ptr(), Sdev.data_ptr(), mad, S1.data_ptr(), stream=sptr)
        ctx.gw_sigma_device(G.data_ptr(), St.data_ptr(), stream=sptr)
        shard.reduce_partial_sigma(S1, dist)
        shard.reduce_partial_sigma(St, dist)
        state["mu"] = ctx.dyson_solve_device(S1.data_ptr(), St.data_ptr(), nel, tol, state["mu"], G.data_ptr(),
                                             stream=sptr)
        state["E"] = ctx.energy_device(G.data_ptr(), S1.data_ptr(), St.data_ptr(), stream=sptr)

    def step(ev=None):
        if ev:
            ev[0].record(stream)
        G.copy_(G0, non_blocking=True)
        if ev:
            ev[1].record(stream)
        iteration()
        if ev:
            ev[2].record(stream)
        Gout.copy_(G, non_blocking=True)
        if ev:
            ev[3].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ctx.stats_enable(True)
    launches0 = ctx.stats_read()[0]
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    torch.cuda.profiler.start()  # a profiler started with capture off records the timed steps only
    for k in range(args.steps):
        step(evs[k])
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches1, tc_n, tc_ms, tc_fl = ctx.stats_read()
    ctx.stats_enable(False)
    comp_ms = sum(e[1].elapsed_time(e[2]) for e in evs)
    tot_ms = sum(e[0].elapsed_time(e[3]) for e in evs)
    gw_ms = ctx.last_timings()["total"]
    if dist:
        t = torch.tensor([comp_ms, tot_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        comp_ms, tot_ms = float(t[0]), float(t[1])
    return s, ctx, dict(comp_ms=comp_ms, tot_ms=tot_ms, gw_ms=gw_ms, clocks=clk, launches=launches1 - launches0,
                        tc_n=tc_n, tc_ms=tc_ms, tc_fl=tc_fl, E=state["E"], mu=state["mu"],
                        bytes_io=G0.numel() * 16, ws=ws, rank=rank, dist=dist, G0=G0, G=G, St=St, S1=S1,
                        sptr=sptr, Gout=Gout, nel=nel)


def fp64_peak_tflops(n=8192, reps=5):
    """Dense float64 GEMM (torch.matmul, n x n x n) timed with CUDA events, best of `reps`: the FP64
    peak the FP64 path is measured against (no clock changes)."""
    import torch
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = None
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best / 1e3) / 1e12


def gw_contraction_flops(s):
    """Algorithmic flops of the P0 and Sigma contractions of one iteration, counted in the reference's
    contraction order (8 real flops per complex multiply-add)."""
    per = 2 * s.nao ** 3 * s.NQ + s.nao ** 2 * s.NQ ** 2
    return 8.0 * s.nk * s.nk * (s.nts // 2 + s.nts) * s.ns * per


def fp64_full_iteration(s, ctx, r):
    """One whole iteration in split precision and one in FP64, both from the same G0 (the generator's
    non-interacting G, mu searched from 0): the FP64 iteration's device time (CUDA events on the library's
    stream) and the full-size differences of Sigma, the new G, the chemical potential and the energies."""
    import torch
    from gb200 import lib

    dev = r["G"].device
    out = {}
    for name, mode in (("split", lib.PREC_SPLIT), ("fp64", lib.PREC_FP64)):
        ctx.set_precision(mode, r["slices"])
        G = torch.empty_like(r["G"])
        G.copy_(r["G0"])
        S1 = torch.empty_like(r["S1"])
        St = torch.empty_like(r["St"])
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        a.record()
        mu, E = ctx.iteration_device(G.data_ptr(), S1.data_ptr(), St.data_ptr(), 0.0, r["nel"], 1e-9, 0.0,
                                     stream=r["sptr"])
        b.record()
        torch.cuda.synchronize(dev)
        out[name] = dict(G=G, S1=S1, St=St, mu=mu, E=E, ms=a.elapsed_time(b))
    ctx.set_precision(lib.PREC_SPLIT, r["slices"])
    sp, fp = out["split"], out["fp64"]
    acc = {
        "max_abs_dSigma_full": float((sp["St"] - fp["St"]).abs().max()),
        "max_abs_Sigma_full": float(fp["St"].abs().max()),
        "max_abs_dG_full": float((sp["G"] - fp["G"]).abs().max()),
        "max_abs_G_full": float(fp["G"].abs().max()),
        "max_abs_dF_full": float((sp["S1"] - fp["S1"]).abs().max()),
        "d_mu": abs(sp["mu"] - fp["mu"]),
        "dE_HF": abs(sp["E"][1] - fp["E"][1]), "dE_GM": abs(sp["E"][2] - fp["E"][2]),
        "measured": "one whole c2 iteration in each precision from the same G0 (HF, GW, mu search, Dyson, "
                    "energies), full-size tensors compared on the device",
    }
    return fp["ms"], sp["ms"], acc


def full_sigma_accuracy(slices, contraction_slices):
    """Split vs FP64 over one whole iteration from the same G0 on a system with the workload's shapes
    (nao=40, naux=250, ns=1, ntau=120, nw=120, beta=200, eps ~ U[-5,5]) on a 2x1x1 mesh: the full
    self-energy, the new G and the correlation energy, with the FP64 path cheap enough to run whole."""
    import torch
    from gb200 import lib, solvers, synth

    try:
        s = synth.make_system(mesh=(2, 1, 1), nao=40, naux=250, ns=1, beta=200.0, nts=120, nw=120,
                              eps_range=5.0, seed=0)
        res = {}
        for name, prec in (("fp64", lib.PREC_FP64), ("split", lib.PREC_SPLIT)):
            with solvers.make_context(s, precision=prec, slices=slices) as c:
                if contraction_slices:
                    c.set_contraction_slices(contraction_slices)
                G = torch.tensor(s.G, dtype=torch.complex128, device="cuda")
                d = c.dims
                S1 = torch.empty((d.ns, d.nk, d.nso, d.nso), dtype=torch.complex128, device="cuda")
                Sig = torch.empty_like(G)
                torch.cuda.synchronize()
                _, e = c.iteration_device(G.data_ptr(), S1.data_ptr(), Sig.data_ptr(), 0.0, s.nel_from_G0(), 1e-9,
                                          0.0, stream=0x1, energies=True)
                torch.cuda.synchronize()
                res[name] = (G.cpu().numpy(), Sig.cpu().numpy(), e)
        (Ga, Sa, ea), (Gb, Sb, eb) = res["fp64"], res["split"]
        return {"mesh": "2x1x1", "max_abs_dSigma": float(np.abs(Sa - Sb).max()),
                "max_abs_Sigma": float(np.abs(Sa).max()), "max_abs_dG": float(np.abs(Ga - Gb).max()),
                "dE_GM": abs(ea[2] - eb[2])}
    except Exception as ex:  # a report, not the measurement: never let it end the run
        return {"mesh": "2x1x1", "error": f"{type(ex).__name__}: {ex}"}


def main_ours(args):
    s, ctx, r = run_ours(args)
    r["slices"] = args.slices
    ws, rank = r["ws"], r["rank"]
    K = args.steps
    comp_s = r["comp_ms"] / 1e3 / K
    tot_s = r["tot_ms"] / 1e3 / K
    line = None
    if rank == 0:
        bf16_peak, hbm_peak, peak_src = measured_peaks()
        achieved = (r["tc_fl"] / (r["tc_ms"] / 1e3) / 1e12) if r["tc_ms"] > 0 else None
        fp64_iter, acc = None, None
        if ws == 1 and not args.no_fp64:
            fp64_ms, split_ms, acc = fp64_full_iteration(s, ctx, r)
            fp64_iter = fp64_ms / 1e3
            acc["split_iteration_from_G0_ms"] = split_ms
        cpu_est, cpu_desc, _ = cpu_baseline(args.config, args.seed)
        line = {
            "metric": METRIC, "value": 1.0 / comp_s, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": args.warmup,
            "ms_per_step": comp_s * 1e3, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": (f"int8 ({args.slices} balanced base-128 slices per FP64 operand, int32 tensor-core "
                      "accumulate, f64 recombination; f64 aux-basis solve, transforms, Dyson)"),
            "data": "synthetic (seeded generator; V generated on the GPU)",
            "config": {"workload": WORKLOADS[args.config],
                       "precision": f"split, {args.slices} INT8 slices" + (
                           f" (per contraction a-f: {args.contraction_slices})" if args.contraction_slices else ""),
                       "parallelism": f"q-sharded over {ws} GPU(s), NCCL all-reduce of Sigma" if ws > 1 else "1 GPU",
                       "l2": "inputs larger than L2 (G 384 MB, V 100 GB): no flush"},
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": bf16_peak, "unit": "TFLOP/s",
                         "frac": (achieved / bf16_peak) if achieved else None,
                         "traffic": (TC_DRAM_BYTES_PER_FLOP * args.slices / 5 * r["tc_fl"] / r["tc_n"])
                         if r["tc_n"] else None,
                         "traffic_unit": "bytes per launch (scaled from the c2k2 ncu capture at 5 slices, "
                                         "by the launch's flops and by slices / 5 for the digit planes)",
                         "kernel": "split_gemm_tc_kernel (tcgen05 kind::i8)", "launches": r["tc_n"],
                         "peak_source": f"{peak_src} bf16 dense sustained; achieved counts FP64-equivalent complex flops",
                         # the INT8 work behind those flops: S(S+1)/2 digit-plane products, each 4MKN
                         # multiply-adds over the real embedding, per complex product (8MKN flops)
                         "int8_tops": (achieved * args.slices * (args.slices + 1) / 2) if achieved else None,
                         "int8_frac_of_2x_bf16": (achieved * args.slices * (args.slices + 1) / 2 / (2 * bf16_peak))
                         if achieved else None},
            "cpu_baseline": {"value": 1.0 / cpu_est, "unit": UNIT, "cores": blas_threads(), "kind": "port",
                             "sample": cpu_desc, "extrapolated": True},
            "e2e": {"value": 1.0 / tot_s, "unit": UNIT, "h2d_bytes_per_step": r["bytes_io"],
                    "d2h_bytes_per_step": r["bytes_io"]},
            "clocks": r["clocks"], "gpu_launches": r["launches"],
            "energies": {"E_1b": r["E"][0], "E_HF": r["E"][1], "E_corr": r["E"][2], "mu": r["mu"]} if r["E"] else None,
        }
        # size-independent properties of the full-size result: the new G(tau, k) is Hermitian (nothing
        # enforces it: the Dyson step hermitizes Sigma, dyson.cpp:196-198, not G) and G, Sigma are finite
        try:
            def herm_dev(x):
                return float((x - x.conj().transpose(-1, -2)).abs().max() / x.abs().max().clamp_min(1e-300))
            Gnew = r["Gout"]  # the new G of the last timed step (the device copy is reused by the FP64 sample)
            line["properties"] = {"G_hermiticity_rel": herm_dev(Gnew),
                                  "finite": bool(r["St"].isfinite().all() and Gnew.isfinite().all())}
        except Exception as ex:  # a report, not the measurement
            line["properties"] = {"error": f"{type(ex).__name__}: {ex}"}
        # Chebyshev resolution of the new G (transformer_t::check_chebyshev's diagnostic): the
        # grid is the same for the GPU path and the oracle, so this does not affect parity
        try:
            line["chebyshev_leakage_G"] = float(s.grid.leakage(r["Gout"].numpy()))
        except Exception:
            line["chebyshev_leakage_G"] = None
        if fp64_iter is not None:
            try:
                peak64 = fp64_peak_tflops()
            except Exception:  # a report, not the measurement
                peak64 = None
            eff64 = gw_contraction_flops(s) / fp64_iter / 1e12
            line["fp64_gpu"] = {"value": 1.0 / fp64_iter, "unit": UNIT, "ms_per_iteration": fp64_iter * 1e3,
                                "measured": "one whole FP64 iteration at the same workload (CUDA events)",
                                "contraction_tflops_effective": eff64,
                                "fp64_peak_tflops_measured": peak64,
                                "frac_of_fp64_peak": (eff64 / peak64) if peak64 else None,
                                "peak_source": "torch.matmul float64 8192^3, best of 5, CUDA events"}
            line["split_vs_fp64"] = fp64_iter / comp_s
            acc["bound_max_abs_dSigma"] = 1e-8
            acc["within_bound"] = bool(acc["max_abs_dSigma_full"] <= 1e-8)
            acc["full_sigma_same_shapes_2x1x1"] = full_sigma_accuracy(args.slices, args.contraction_slices)
            line["accuracy"] = acc
        print(json.dumps(line), flush=True)
    if r["dist"]:
        r["dist"].barrier()
        r["dist"].destroy_process_group()
    ctx.close()
    return line


def main_gw_profile(args):
    """--gw-q Q: only the GW self-energy over q-points [0, Q), W warm-up calls then K timed ones.

    The kernel-profiling case (ncu captures of the contraction kernels): prints the
    per-stage device times of the last call, not the headline metric.
    """
    import torch

    torch.cuda.set_device(0)
    s, ctx = setup_context(args.config, args.seed, args.slices, 0, 1, 0, args.contraction_slices, args.engine)
    if args.profile_fp64:
        from gb200 import lib
        ctx.set_precision(lib.PREC_FP64, args.slices)
    if args.tile_width:
        ctx.set_tile_width(args.tile_width)
    G = torch.from_numpy(s.G).cuda()
    Sig = torch.empty_like(G)
    ctx.set_q_range(0, min(args.gw_q, s.nk))
    for _ in range(args.warmup):
        ctx.gw_sigma_device(G.data_ptr(), Sig.data_ptr())
    torch.cuda.synchronize()
    out = []
    torch.cuda.profiler.start()  # a profiler started with capture off records the timed calls only
    for _ in range(args.steps):
        ctx.gw_sigma_device(G.data_ptr(), Sig.data_ptr())
        out.append(ctx.last_timings())
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"profile_case": WORKLOADS[args.config], "q_points": min(args.gw_q, s.nk),
                      "precision": "FP64" if args.profile_fp64 else f"split, {args.slices} INT8 slices",
                      "stage_ms": out[-1]}), flush=True)
    ctx.close()


def main_newton(args):
    """--newton N: the differentiable GW step (FP64).  Times the self-energy, its vector-Jacobian
    product with respect to G and to G and V (CUDA events), then runs N plain iterations and N
    Newton-Krylov steps from the same start (the non-interacting G, mu searched every iteration) and
    prints their residual histories |Phi(G) - G|, map evaluations and device-synchronised times."""
    import torch

    from gb200 import newton, solvers, synth

    torch.cuda.set_device(0)
    s = synth.make_config(args.config, seed=args.seed)
    ctx = solvers.make_context(s)
    G = torch.from_numpy(s.G).cuda()
    Sig, Sb = torch.empty_like(G), torch.randn_like(G)
    Gb = torch.empty_like(G)
    Vb = torch.empty((s.V_half.shape), dtype=torch.complex128, device="cuda")

    def timed(fn, n):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(n):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / n

    leg = 0x1  # the library call shares torch's default stream
    t_fwd = timed(lambda: ctx.gw_sigma_device(G.data_ptr(), Sig.data_ptr(), stream=leg), 3)
    t_vjp = timed(lambda: ctx.gw_sigma_vjp_device(G.data_ptr(), Sb.data_ptr(), Gb.data_ptr(), 0, stream=leg), 2)
    t_vjp_v = timed(lambda: ctx.gw_sigma_vjp_device(G.data_ptr(), Sb.data_ptr(), Gb.data_ptr(), Vb.data_ptr(),
                                                   stream=leg), 2)
    it = newton.DeviceIteration(ctx, G, nel=s.nel_from_G0(), mu=0.0, tol=1e-12)
    atol = 1e-11 * (1.0 + float(torch.linalg.norm(G)))  # about the FP64 floor of |Phi(G) - G|
    out = {"workload": WORKLOADS[args.config], "precision": "FP64", "gw_sigma_ms": t_fwd,
           "vjp_G_ms": t_vjp, "vjp_G_V_ms": t_vjp_v}
    for name, run in (("plain", lambda: newton.plain_iteration(it, G, args.newton)),
                      ("plain_g_mixing_0.5", lambda: newton.plain_iteration(it, G, args.newton, mixing=0.5)),
                      ("newton_krylov", lambda: newton.newton_krylov(it, G, args.newton, maxiter=30,
                                                                      atol=atol))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        calls0 = it.calls
        _, h = run()
        torch.cuda.synchronize()
        out[name] = {"steps": args.newton, "residual": h.residual, "map_evaluations": it.calls - calls0,
                     "krylov_matvecs": h.krylov, "seconds": time.perf_counter() - t0, "mu": it.last_mu}
        print(json.dumps(out), flush=True)  # one line per stage, the last one complete
    ctx.close()


def main_batch(args):
    """--batch N: N independent systems of uneven sizes (gb200.batch.uneven_systems: nk from {8, 27, 64},
    nao ~ U{8..48}, naux ~ U{4 nao..6 nao}, ntau = 80, beta = 100), integrals generated on the device,
    one context per system with memory budgets in proportion to their intermediates, tile widths from
    the autotuner's table (gb200/tile_table.json), split precision.  The timed call is
    gb200_gw_sigma_batch_device: the systems' q-points in step, every contraction stage one grouped
    persistent tensor-core launch over the tiles of all systems (CUDA events).  The same batch issued
    from a thread pool of per-system calls is timed beside it.  Prints the aggregate self-energy
    evaluations per second and each system's max|dSigma| against its own FP64 self-energy."""
    import torch

    from gb200 import batch, lib, solvers, synth

    torch.cuda.set_device(0)
    systems = batch.uneven_systems(count=args.batch, seed=args.seed, with_integrals=False)
    ctxs = []
    for i, s in enumerate(systems):
        g = s.grid
        c = lib.Context(s.nk, s.nao, s.ns, s.NQ, g.nts, g.nw, g.nw_b, s.beta, device=0)
        kp, km = solvers.kq_maps(s.mesh)
        c.set_kq_maps(kp, km)
        c.set_grid(g.Tnt_f, g.Ttn_f, g.Tnt_b, g.Ttn_b, g.wsample_f)
        synth.upload_device_integrals(c, s.nk, s.NQ, s.nao, seed=args.seed * 1000 + i, device=0)
        c.set_hamiltonian(s.F, s.S)
        c.set_precision(lib.PREC_SPLIT, args.slices)
        ctxs.append(c)
    b = batch.SystemBatch(ctxs)
    widths = b.apply_tiles()
    # budgets cover the k-block intermediates; their INT8 planes take about 2S/16 of that again
    free_b, _ = torch.cuda.mem_get_info(0)
    b.share_memory(0.4 * free_b)
    G = [torch.from_numpy(s.G).cuda() for s in systems]
    Sig = [torch.empty_like(x) for x in G]
    gp, sp = [x.data_ptr() for x in G], [x.data_ptr() for x in Sig]

    def timed(run):
        for _ in range(args.warmup):
            run()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        t0 = time.perf_counter()
        ev[0].record()
        for _ in range(args.steps):
            run()
        ev[1].record()
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / 1e3 / args.steps, (time.perf_counter() - t0) / args.steps

    grouped_s, grouped_wall = timed(lambda: b.run_gw_grouped(gp, sp))
    grouped = [x.clone() for x in Sig]
    _, pool_wall = timed(lambda: b.run_gw(gp, sp))
    rows = []
    for c, s, g_, x, y in zip(ctxs, systems, G, grouped, Sig):
        c.set_precision(lib.PREC_FP64, args.slices)
        ref = torch.empty_like(x)
        c.gw_sigma_device(g_.data_ptr(), ref.data_ptr())
        torch.cuda.synchronize()
        rows.append({"nk": s.nk, "nao": s.nao, "naux": s.NQ, "tile": c_width(widths, len(rows)),
                     "max_abs_dSigma": float((x - ref).abs().max()), "max_abs_Sigma": float(ref.abs().max()),
                     "grouped_equals_individual": bool(torch.equal(x, y))})
        del ref
    print(json.dumps({"workload": f"{args.batch} uneven systems (nk from {{8, 27, 64}}, nao ~ U{{8..48}}, "
                                  f"naux ~ U{{4 nao..6 nao}}, ntau = 80, beta = 100), seed {args.seed}",
                      "precision": f"split, {args.slices} INT8 slices", "sigma_evals_per_s": args.batch / grouped_s,
                      "seconds_per_batch": grouped_s,
                      "timing": "CUDA events around gb200_gw_sigma_batch_device (grouped launches), "
                                f"mean of {args.steps} after {args.warmup} warm-up",
                      "wall_seconds_per_batch": grouped_wall,
                      "thread_pool_seconds_per_batch": pool_wall,
                      "tile_widths": "gb200/tile_table.json (0: widest)",
                      "systems": rows}), flush=True)
    b.close()


def c_width(widths, i):
    return int(widths[i]) if i < len(widths) else 0


def main_reference(args):
    """The CPU arm: the oracle (numpy/BLAS restatement of gw_cpu_kernel, hf_cpu_kernels and dyson) on the host
    cores.  A whole c2 iteration takes hours on a CPU, so every step runs a bounded sample of it (cpu_baseline's
    sample) and the iteration time is extrapolated from it by the uniform per-(q, k) work; `ms_per_step` is the
    measured wall time of one sample step, `value` the extrapolated iterations per second."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return None  # the CPU reference runs on rank 0 only
    for _ in range(args.warmup):
        cpu_baseline(args.config, args.seed)
    ests, samples, walls, desc = [], [], [], ""
    for _ in range(args.steps):
        t0 = time.perf_counter()
        est, desc, sample_s = cpu_baseline(args.config, args.seed)
        walls.append(time.perf_counter() - t0)
        ests.append(est)
        samples.append(sample_s)
    v = 1.0 / statistics.mean(ests)
    frac = statistics.mean(samples) / statistics.mean(ests)
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * statistics.mean(walls), "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)", "impl": "reference",
        "config": {"workload": WORKLOADS[args.config], "precision": "FP64 (CPU oracle restating the reference kernels)"},
        "extrapolated": True,
        "iteration_ms_extrapolated": 1e3 * statistics.mean(ests),
        "sample_fraction_of_iteration": frac,
        "step": "one bounded sample of the iteration (timed kernels of the sample, plus its set-up); "
                "value = 1 / (iteration time extrapolated from the sample)",
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": blas_threads(), "kind": "port", "sample": desc,
                         "extrapolated": True, "sample_s": statistics.mean(samples)},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return line


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)  # one c2 iteration is about a minute on a B200
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=sorted(WORKLOADS), default="c2")
    ap.add_argument("--slices", type=int, default=5)
    ap.add_argument("--contraction-slices", dest="contraction_slices", default=None,
                    type=lambda x: [int(v) for v in x.split(",")],
                    help="slices of the six contractions P0 (a)-(c), Sigma (d)-(f), comma-separated; "
                         "0 keeps --slices")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--engine", type=int, default=0, choices=[0, 1],
                    help="split engine: 0 tcgen05 tensor cores (default), 1 the CUDA-core validation engine")
    ap.add_argument("--no-fp64", dest="no_fp64", action="store_true",
                    help="skip the whole FP64 iteration (its time and the full-size split-vs-FP64 accuracy)")
    ap.add_argument("--gw-q", dest="gw_q", type=int, default=0,
                    help="profiling case: time only the GW self-energy over q-points [0, GW_Q)")
    ap.add_argument("--profile-fp64", dest="profile_fp64", action="store_true",
                    help="profiling case in FP64 instead of split precision")
    ap.add_argument("--tile-width", dest="tile_width", type=int, default=0,
                    help="profiling case: column tile of the tensor-core contractions (0: the default)")
    ap.add_argument("--newton", type=int, default=0,
                    help="differentiable-step case (--config c4): adjoint timings, then N plain and N "
                         "Newton-Krylov self-consistency steps from the same start")
    ap.add_argument("--batch", type=int, default=0,
                    help="batched case: N systems of uneven sizes evaluated together (aggregate rate, per-system "
                         "error against FP64)")
    a = ap.parse_args(argv)
    if a.warmup < 3 and not (a.gw_q or a.newton or a.batch):
        ap.error("at least 3 warm-up steps")
    return a


if __name__ == "__main__":
    args = parse()
    if args.impl == "reference":
        main_reference(args)
    elif args.gw_q:
        main_gw_profile(args)
    elif args.newton:
        main_newton(args)
    elif args.batch:
        main_batch(args)
    else:
        main_ours(args)
