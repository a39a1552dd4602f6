"""Benchmark: Fock builds/s on a 192x192 k-mesh, nb=8, layer-resolved V (1 GPU per rank).

Workload: ``build_fock`` on a 192x192 mesh with nb=8 band channels, layer-
resolved V_ab(q) = 2 pi tanh(|q| d_ab)/|q| (d_ab = 1 + |a-b|/2, V(0)=0), h from
the seeded |R|<=3 Fourier model, P(k) = U diag(f) U^H with Haar U and
f ~ U(0,1), complex128.  A step is STEP_BUILDS builds; before every build the
L2 cache is flushed by writing a 256 MiB buffer (outside the timed interval)
and each build is bracketed by CUDA events on the launching stream.

``value``  = builds/s with inputs resident in HBM (sum of per-build device time).
``e2e``    = builds/s through the public API with host buffers: H2D of P from
             pinned memory, the build, D2H of Sigma and F, per step; steps are
             pipelined over copy-in / build / copy-out streams with two buffer sets.
``roofline`` = algorithmic bytes of one build / average build time against the
             measured HBM copy bandwidth (MEASURED_PEAKS.json).
``--impl reference`` times the CPU oracle (NumPy/SciPy restatement of the
reference path, all host cores) on the same workload.
Multi-GPU: independent replicas (the path has no exchange step); value = all
ranks' builds / max-over-ranks device time.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Fock builds/s & batched HF solves/s at |dE/E|<=1e-9, mixed vs plain FP64 (1 GPU)"
UNIT = "builds/s"
NK, NB = 192, 8
STEP_BUILDS = 64
WORKLOAD = "build_fock 192x192 mesh, nb=8, layer-resolved V, Haar density, complex128"


def alg_bytes(nk1, nk2, nb, elem=16):
    """Read P, h (complex) and VR (real), write Sigma and F: (4*16 + 8) nk^2 nb^2 B for complex128."""
    return (4 * elem + elem // 2) * nk1 * nk2 * nb * nb


def peaks():
    try:
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """Samples nvidia-smi during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.p = None
        self.gpu = gpu_index
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={gpu_index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except Exception:
            self.p.kill()
            out = ""
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def setup_dist(args):
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return ws, rank, local


def make_inputs(seed, dtype=np.complex128):
    from jax_hf_b200 import synthetic as S
    prob, P = S.fock_build_192(seed)
    return prob, P.astype(dtype)


def run_ours(args, ws, rank, local):
    import torch
    import jax_hf_b200 as G
    from jax_hf_b200 import _lib

    dev = torch.device("cuda", torch.cuda.current_device())
    prob, P_np = make_inputs(1 + rank)
    K = G.HartreeFockKernel(prob.weights, prob.hamiltonian, prob.coulomb_q, prob.T)
    a = K.as_args()
    P = torch.as_tensor(P_np, device=dev)
    kw = dict(h=a["h"], VR=a["VR"], refP=a["refP"], HH=a["HH"], w2d=K.w2d, include_exchange=True,
              include_hartree=False, exchange_hermitian_channel_packing=a["exchange_hermitian_channel_packing"],
              contact_g=a["contact_g"], contact_Oi=a["contact_Oi"], contact_Oj=a["contact_Oj"])
    Sg = torch.empty_like(P)
    F = torch.empty_like(P)
    H = torch.empty((1, 1, NB, NB), dtype=P.dtype, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()

    flush_words = flush.view(torch.float32)

    def timed_builds(n, fn, read_flush=False):
        # L2 flush before every build: a 256 MiB write (the headline), or a 256 MiB read, which
        # leaves no dirty lines whose write-back would land inside the timed build
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
        for i in range(n):
            if read_flush:
                flush_words.sum()
            else:
                flush.fill_(i & 0xFF)
            ev[i][0].record(stream)
            fn()
            ev[i][1].record(stream)
        return ev

    def build():
        G.build_fock(P, out=(Sg, H, F), **kw)

    # warm-up
    for _ in range(args.warmup):
        timed_builds(args.builds_per_step, build)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clk = Clocks(local) if rank == 0 else None
    t_wall = time.perf_counter()
    evs = []
    for _ in range(args.steps):
        evs.append(timed_builds(args.builds_per_step, build))
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall
    clocks = clk.stop() if clk else None
    if ws > 1:
        torch.distributed.barrier()
    per_build = [s.elapsed_time(e) for step in evs for (s, e) in step]   # ms
    dev_ms = float(sum(per_build))
    if ws > 1:
        t = torch.tensor([dev_ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        dev_ms = float(t.item())
    n_builds = args.steps * args.builds_per_step
    value = ws * n_builds / (dev_ms / 1e3)
    avg_us = 1e3 * float(np.mean(per_build))

    # variants: complex64 storage and FP32 exchange FFT with complex128 storage
    variants = {}
    if not args.extras:
        return _finish(args, ws, rank, value, dev_ms, avg_us, n_builds, t_wall, clocks, variants, None, None,
                       P_np, prob)
    P64 = P.to(torch.complex64)
    K64 = G.HartreeFockKernel(prob.weights, prob.hamiltonian.astype(np.complex64), prob.coulomb_q, prob.T)
    a64 = K64.as_args()
    kw64 = dict(kw, h=a64["h"], VR=a64["VR"], refP=a64["refP"], HH=a64["HH"], w2d=K64.w2d,
                contact_g=a64["contact_g"], contact_Oi=a64["contact_Oi"], contact_Oj=a64["contact_Oj"])
    S64, F64 = torch.empty_like(P64), torch.empty_like(P64)
    H64 = torch.empty((1, 1, NB, NB), dtype=P64.dtype, device=dev)
    for name, fn, nbytes, rf in (
        ("c64", lambda: G.build_fock(P64, out=(S64, H64, F64), **kw64), alg_bytes(NK, NK, NB, 8), False),
        ("c128_fp32fft", lambda: G.build_fock(P, out=(Sg, H, F), fft_precision="fp32", **kw), alg_bytes(NK, NK, NB),
         False),
        ("c128_read_flush", build, alg_bytes(NK, NK, NB), True),
        ("c128_pipe_engine", lambda: G.build_fock(P, out=(Sg, H, F), engine="pipe", **kw), alg_bytes(NK, NK, NB),
         False),
    ):
        timed_builds(8, fn, rf)
        ev = timed_builds(STEP_BUILDS, fn, rf)
        torch.cuda.synchronize()
        t = [s.elapsed_time(e) for (s, e) in ev]
        us = 1e3 * float(np.mean(t))
        variants[name] = {"builds_per_s": round(1e6 / us, 1), "us_per_build": round(us, 2),
                          "achieved_gbs": round(nbytes / (us * 1e-6) / 1e9, 1)}

    # a batch of independent densities through build_fock_batch: 12 distinct densities (k-shifted
    # copies of the seeded density) and output sets cycled over the 64 builds of a step (1.4 GB,
    # larger than L2; build i uses set i % 12 and stream i % streams, so a set is reused only 12
    # builds later and on the same stream), h and V-hat shared by the batch as in a scan with one
    # kernel; no flush.  The same batch on one stream isolates the gain
    # of running builds on three streams.
    bP = [torch.roll(P, shifts=(7 * r, 13 * r), dims=(0, 1)).contiguous() for r in range(12)]
    bout = [(torch.empty_like(P), torch.empty_like(H), torch.empty_like(P)) for _ in range(12)]

    def batch_rate(nstreams):
        n = STEP_BUILDS
        call = lambda: G.build_fock_batch([bP[i % 12] for i in range(n)], outs=[bout[i % 12] for i in range(n)],
                                          streams=nstreams, **kw)
        call()
        torch.cuda.synchronize()
        eb0, eb1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        eb0.record(stream)
        call()
        eb1.record(stream)
        torch.cuda.synchronize()
        us_b = 1e3 * eb0.elapsed_time(eb1) / n
        return {"builds_per_s": round(1e6 / us_b, 1), "us_per_build": round(us_b, 2),
                "achieved_gbs": round(alg_bytes(NK, NK, NB) / (us_b * 1e-6) / 1e9, 1)}

    variants["c128_batch_1stream"] = batch_rate(1)
    variants["c128_batch_3streams"] = batch_rate(3)

    # block-diagonal exchange (build_fock with exchange_block_specs) against the full build,
    # both timed the same way: the 12 density sets built back to back inside one CUDA graph
    # (captured once, replayed), so host overhead is out of the comparison; densities made
    # block-diagonal for the checked runs
    blk = np.zeros((NB, NB), bool)
    blk[:NB // 2, :NB // 2] = blk[NB // 2:, NB // 2:] = True
    bPb = [x * torch.as_tensor(blk, device=dev) for x in bP]

    def graph_rate(build_i, reps=4):
        side = torch.cuda.Stream()
        side.wait_stream(stream)
        with torch.cuda.stream(side):
            for i in range(12):
                build_i(i)  # workspaces for this stream, before capture
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=side):
            for i in range(12):
                build_i(i)
        graph.replay()
        torch.cuda.synchronize()
        eb0, eb1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        eb0.record(stream)
        for _ in range(reps):
            graph.replay()
        eb1.record(stream)
        torch.cuda.synchronize()
        del graph
        return 1e3 * eb0.elapsed_time(eb1) / (12 * reps)

    us_full = graph_rate(lambda i: G.build_fock(bP[i], out=bout[i], **kw))
    variants["c128_graph_full"] = {"builds_per_s": round(1e6 / us_full, 1), "us_per_build": round(us_full, 2)}
    half = [{"block_sizes": [NB // 2, NB // 2]}]
    quarter = [{"block_sizes": [NB // 4] * 4}]
    for name, dens, spec, check in (("c128_graph_blocks_2x4_forced", bP, half, False),
                                    ("c128_graph_blocks_4x2_forced", bP, quarter, False),
                                    ("c128_graph_blocks_2x4_checked_blockdiag", bPb, half, True),
                                    ("c128_graph_blocks_2x4_checked_coupled", bP, half, True)):
        us_b = graph_rate(lambda i: G.build_fock(dens[i], out=bout[i], exchange_block_specs=spec,
                                                 exchange_check_offdiag=check, exchange_offdiag_atol=1e-9, **kw))
        variants[name] = {"builds_per_s": round(1e6 / us_b, 1), "us_per_build": round(us_b, 2),
                          "vs_full_build": round(us_b / us_full, 3)}
    del bP, bout, bPb

    solves = run_solves(dev) if args.solves else None
    variants["solves"] = solves

    # e2e: public API with host buffers (H2D P from pinned memory, D2H Sigma and F), pipelined the
    # way a caller streaming many builds would run it: copy-in, build and copy-out on three streams
    # with two device buffer sets, so step i's D2H overlaps step i+1's H2D (PCIe is full duplex).
    # Every step still moves its own inputs in and its own results out inside the timed region.
    hP = torch.from_numpy(P_np).pin_memory()
    nset = 2
    dPs = [torch.empty_like(P) for _ in range(nset)]
    outs = [(torch.empty_like(P), torch.empty_like(H), torch.empty_like(P)) for _ in range(nset)]
    hSs = [torch.empty(P.shape, dtype=P.dtype).pin_memory() for _ in range(nset)]
    hFs = [torch.empty(P.shape, dtype=P.dtype).pin_memory() for _ in range(nset)]
    s_in, s_c, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    ev_c = [torch.cuda.Event() for _ in range(nset)]
    ev_out = [torch.cuda.Event() for _ in range(nset)]
    ev_in = [torch.cuda.Event() for _ in range(nset)]
    for e in ev_c + ev_out:
        e.record(s_c)

    def e2e_step(i):
        b = i % nset
        s_in.wait_event(ev_c[b])            # the build two steps back has read dPs[b]
        with torch.cuda.stream(s_in):
            dPs[b].copy_(hP, non_blocking=True)
        ev_in[b].record(s_in)
        s_c.wait_event(ev_in[b])
        s_c.wait_event(ev_out[b])           # the copy-out two steps back has read outs[b]
        with torch.cuda.stream(s_c):
            G.build_fock(dPs[b], out=outs[b], **kw)
        ev_c[b].record(s_c)
        s_out.wait_event(ev_c[b])
        with torch.cuda.stream(s_out):
            hSs[b].copy_(outs[b][0], non_blocking=True)
            hFs[b].copy_(outs[b][2], non_blocking=True)
        ev_out[b].record(s_out)

    for i in range(3):
        e2e_step(i)
    torch.cuda.synchronize()
    n_e2e = max(8, args.steps)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s_in)
    for i in range(n_e2e):
        e2e_step(i)
    s_out.wait_stream(s_in)
    s_out.wait_stream(s_c)
    e1.record(s_out)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if ws > 1:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_val = ws * n_e2e / (e2e_ms / 1e3)
    nbytes_state = P.numel() * P.element_size()
    return _finish(args, ws, rank, value, dev_ms, avg_us, n_builds, t_wall, clocks, variants, e2e_val,
                   nbytes_state, P_np, prob)


def run_solves(dev):
    """Whole-solve throughput on the solver workloads (device time, CUDA events) and the
    error of every solve against the FP64 oracle.

    The FP64 oracle energy is the self-consistent fixed point computed by the CPU oracle
    (tests/golden/scan64_oracle.json, tests/golden/baseline_oracle.json); the reference
    CG's plateau stop ends 1e-9 .. 4e-6 above it, which the lines report as
    rel_dE_vs_oracle_fixed_point next to the agreement with the oracle's own CG result.

    scf_diis_24x24_nb4: solve_scf (DIIS), FP64.  cg_144x144_nb8: CG at tol_E=1e-9 in
    FP64 (the reference algorithm) against the mixed solve (FP32-exchange CG to a coarse
    plateau, then the FP64 SCF-DIIS polish to the fixed point).  density_scan_64: the 64
    solves of the scan (meshes 36..120, nb 4/6/8): the reference CG solve by solve and
    batched, the FP64 SCF-DIIS with the reference's steps solve by solve (the plain FP64
    path that reaches |dE/E| <= 1e-9), and the mixed solvers batched.
    """
    import time as _time_mod
    import torch
    import jax_hf_b200 as G
    from jax_hf_b200 import synthetic as S
    from jax_hf_b200.reference_scf import SCFConfig, solve_scf, solve_scf_batch
    from jax_hf_b200.solver import SolverConfig, solve, solve_batch

    stream = torch.cuda.current_stream()
    gold = ROOT / "tests" / "golden"
    base = json.loads((gold / "baseline_oracle.json").read_text())
    fx = json.loads((gold / "scan64_oracle.json").read_text())["rows"]

    def ev_time(fn, reps=1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        out = None
        for _ in range(reps):
            out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) / reps

    def median_run(fn, n):
        # median time of n calls; only the last result is kept, so the caching allocator can reuse
        # the previous call's output blocks
        ts, res = [], None
        for _ in range(n):
            res = None
            res, t = ev_time(fn)
            ts.append(t)
        return res, float(statistics.median(ts))

    def rel(E, Eo):
        return abs(float(E) - Eo) / abs(Eo)

    out = {}
    # SCF-DIIS 24x24 nb=4 (reference steps)
    p0 = S.scf_diis_24()
    K0 = G.HartreeFockKernel(**p0.kernel_kwargs())
    P00 = torch.zeros((24, 24, 4, 4), dtype=torch.complex128, device=dev)
    scfg = SCFConfig(acceleration="diis")
    for _ in range(3):  # first calls load kernels
        solve_scf(K0, P00, p0.n_electrons, config=scfg)
    r0, ms0 = median_run(lambda: solve_scf(K0, P00, p0.n_electrons, config=scfg), 7)
    o0 = base["scf_diis_24x24_nb4"]
    out["scf_diis_24x24_nb4_fp64"] = {
        "solves_per_s": round(1e3 / ms0, 2), "ms_per_solve": round(ms0, 2), "iterations": int(r0.iterations),
        "converged": bool(r0.converged), "energy": float(r0.energy),
        "rel_dE_vs_oracle_same_algorithm": rel(r0.energy, o0["reference_algorithm"]["energy"]),
        "rel_dE_vs_oracle_fixed_point": rel(r0.energy, o0["fixed_point_energy"])}
    # CG 144x144 nb=8: FP64 reference algorithm vs the mixed solve
    p2 = S.cg_144()
    K2 = G.HartreeFockKernel(**p2.kernel_kwargs())
    P02 = torch.zeros((144, 144, 8, 8), dtype=torch.complex128, device=dev)
    o2 = base["cg_144x144_nb8"]
    cfgs = (("fp64", SolverConfig(max_iter=400, tol_E=1e-9)),
            ("mixed", SolverConfig(max_iter=400, tol_E=1e-6, fp32_exchange=True, fp32_switch_rel=1e-6,
                                   polish="scf")))
    cg2 = {}
    for name, cfg in cfgs:
        for _ in range(3):
            solve(K2, P02, p2.n_electrons, config=cfg)
        r, ms = median_run(lambda: solve(K2, P02, p2.n_electrons, config=cfg), 7)
        cg2[name] = {"solves_per_s": round(1e3 / ms, 2), "ms_per_solve": round(ms, 2), "n_iter": int(r.n_iter),
                     "converged": bool(r.converged), "energy": float(r.energy),
                     "rel_dE_vs_oracle_fixed_point": rel(r.energy, o2["fixed_point_energy"]),
                     "rel_dE_vs_oracle_reference_cg": rel(r.energy, o2["reference_algorithm"]["energy"])}
        if name == "mixed":
            cg2[name]["polish_iterations"] = int(r.history["polish_iterations"])
    # the same problem through SCF-DIIS (Newton mu, warm eigh), FP64 and mixed: both end at the
    # self-consistent fixed point, which the CG's plateau stop misses by 1.5e-8
    fast2 = dict(acceleration="diis", density_tol=1e-8, comm_tol=1e-7, max_iter=300, mu_method="newton",
                 warm_eigh=True)
    for name, cfg in (("fp64_scf", SCFConfig(**fast2)), ("mixed_scf", SCFConfig(**fast2, fp32_exchange=True))):
        for _ in range(3):
            solve_scf(K2, P02, p2.n_electrons, config=cfg)
        r, ms = median_run(lambda: solve_scf(K2, P02, p2.n_electrons, config=cfg), 7)
        cg2[name] = {"solves_per_s": round(1e3 / ms, 2), "ms_per_solve": round(ms, 2),
                     "iterations": int(r.iterations), "converged": bool(r.converged), "energy": float(r.energy),
                     "rel_dE_vs_oracle_fixed_point": rel(r.energy, o2["fixed_point_energy"])}
    out["cg_144x144_nb8"] = cg2
    # density scan: 64 solves
    probs = S.density_scan(64)
    Ks = [G.HartreeFockKernel(**p.kernel_kwargs()) for p in probs]
    P0s = [torch.zeros((p.nk, p.nk, p.nb, p.nb), dtype=torch.complex128, device=dev) for p in probs]
    nes = [p.n_electrons for p in probs]
    Efp = np.array([r["energy"] for r in fx])
    Ecg = np.array([r["cg_energy"] for r in fx])
    c64 = SolverConfig(max_iter=400, tol_E=1e-9)
    ref_scf = SCFConfig(acceleration="diis", density_tol=1e-8, comm_tol=1e-7, max_iter=300)
    fast = dict(acceleration="diis", density_tol=1e-8, comm_tol=1e-7, max_iter=300, mu_method="newton",
                warm_eigh=True)
    mixed_scf = SCFConfig(**fast, fp32_exchange=True)
    mixed_cg = SolverConfig(max_iter=400, tol_E=1e-6, fp32_exchange=True, fp32_switch_rel=1e-6, polish="scf")

    def errors(Es):
        r_fp = np.abs(np.asarray(Es) - Efp) / np.abs(Efp)
        return {"max_rel_dE_vs_oracle_fixed_point": float(r_fp.max()),
                "n_rel_dE_above_1e-9": int((r_fp > 1e-9).sum())}

    def one_by_one(fn):
        ts, Es = [], []
        for K, P0, ne in zip(Ks, P0s, nes):
            r, ms = ev_time(lambda: fn(K, P0, ne))
            ts.append(ms)
            Es.append(float(r.energy))
        return ts, Es

    # warm-ups (kernel loads, graph instantiation, workspaces)
    for K, P0, ne in zip(Ks[:4], P0s[:4], nes[:4]):
        solve(K, P0, ne, config=c64)
        solve_scf(K, P0, ne, config=ref_scf)
    solve_batch(Ks, P0s, nes, config=c64, lanes=16)
    solve_scf_batch(Ks, P0s, nes, config=mixed_scf, workers=8)
    solve_scf_batch(Ks, P0s, nes, config=SCFConfig(**fast), workers=8)
    solve_batch(Ks[:16], P0s[:16], nes[:16], config=mixed_cg, lanes=16)
    scan = {"n_solves": len(probs), "oracle": "tests/golden/scan64_oracle.json (fixed point: oracle SCF-DIIS to 1e-11)"}
    t_cg, E_cg = one_by_one(lambda K, P0, ne: solve(K, P0, ne, config=c64))
    scan["fp64_solve_by_solve"] = {
        "solver": "CG, tol_E 1e-9 (reference algorithm)", "solves_per_s": round(64 / (sum(t_cg) / 1e3), 2),
        "total_ms": round(sum(t_cg), 2), "p50_ms": round(float(np.percentile(t_cg, 50)), 2),
        "p99_ms": round(float(np.percentile(t_cg, 99)), 2),
        "max_abs_dE_vs_oracle_reference_cg": float(np.abs(np.asarray(E_cg) - Ecg).max()), **errors(E_cg)}
    t_scf, E_scf = one_by_one(lambda K, P0, ne: solve_scf(K, P0, ne, config=ref_scf))
    scan["fp64_scf_solve_by_solve"] = {
        "solver": "SCF-DIIS with the reference's steps (bisection mu, Jacobi eigh), density_tol 1e-8",
        "solves_per_s": round(64 / (sum(t_scf) / 1e3), 2), "total_ms": round(sum(t_scf), 2),
        "p50_ms": round(float(np.percentile(t_scf, 50)), 2), "p99_ms": round(float(np.percentile(t_scf, 99)), 2),
        **errors(E_scf)}
    fp64_fast = SCFConfig(**fast)
    t_fs, E_fs = one_by_one(lambda K, P0, ne: solve_scf(K, P0, ne, config=fp64_fast))
    scan["fp64_fast_scf_solve_by_solve"] = {
        "solver": "SCF-DIIS, FP64 throughout, the mixed solver's steps (Newton mu, warm eigh), density_tol 1e-8",
        "solves_per_s": round(64 / (sum(t_fs) / 1e3), 2), "total_ms": round(sum(t_fs), 2),
        "p50_ms": round(float(np.percentile(t_fs, 50)), 2), "p99_ms": round(float(np.percentile(t_fs, 99)), 2),
        **errors(E_fs)}
    legs = (("fp64_batched", "CG, tol_E 1e-9, 16 streams",
             lambda: solve_batch(Ks, P0s, nes, config=c64, lanes=16, return_times=True)),
            ("mixed_batched", "SCF-DIIS, FP32 exchange until density residual 1e-5 then FP64, Newton mu, warm eigh, "
             "the whole batch as one CUDA graph (loops and DIIS solve on the device), captured once, launched per run",
             lambda: mixed_graph.run(return_times=True)),
            ("mixed_batched_host_threads", "the same mixed SCF-DIIS, 8 host threads with a stream each",
             lambda: solve_scf_batch(Ks, P0s, nes, config=mixed_scf, workers=8, return_times=True)),
            ("fp64_fast_scf_batched", "SCF-DIIS, FP64 throughout, Newton mu, warm eigh, one CUDA graph as above",
             lambda: fp64_graph.run(return_times=True)),
            ("mixed_cg_polish_batched", "FP32-exchange CG to tol_E 1e-6, then FP64 SCF-DIIS polish, 16 streams",
             lambda: solve_batch(Ks, P0s, nes, config=mixed_cg, lanes=16, return_times=True)))
    # the SCF batches as CUDA graphs (built once, outside the timed runs)
    from jax_hf_b200.reference_scf import ScfScanGraph
    t_b = _time_mod.perf_counter()
    mixed_graph = ScfScanGraph(Ks, P0s, nes, config=mixed_scf)
    scf_build_ms = (_time_mod.perf_counter() - t_b) * 1e3
    fp64_graph = ScfScanGraph(Ks, P0s, nes, config=fp64_fast)
    mixed_graph.run()
    fp64_graph.run()
    scan["scf_graph_build_ms_host_once"] = round(scf_build_ms, 1)
    # the FP64 CG batch as one CUDA graph (device-side loops), captured once and launched
    from jax_hf_b200.solver import ScanGraph
    import time as _time
    t_b = _time.perf_counter()
    sg = ScanGraph(Ks, P0s, nes, config=c64)
    build_ms = (_time.perf_counter() - t_b) * 1e3
    sg.run()
    (rg, tg), ms_g = median_run(lambda: sg.run(return_times=True), 3)
    scan["fp64_graph_batched"] = {
        "solver": "CG, tol_E 1e-9, the whole batch as one CUDA graph (conditional WHILE node per solve), "
                  "captured once, launched per run", "solves_per_s": round(64 / (ms_g / 1e3), 2),
        "total_ms": round(ms_g, 2), "graph_build_ms_host_once": round(build_ms, 1),
        "p50_ms": round(float(np.percentile(tg, 50)), 2), "p99_ms": round(float(np.percentile(tg, 99)), 2),
        "all_converged": bool(all(bool(r.converged) for r in rg)),
        "speedup_vs_fp64_solve_by_solve": round(sum(t_cg) / ms_g, 3),
        "max_abs_dE_vs_oracle_reference_cg": float(np.abs(np.asarray([float(r.energy) for r in rg]) - Ecg).max()),
        **errors([float(r.energy) for r in rg])}
    sg.close()
    del rg
    for name, desc, fn in legs:
        (rb, tb), ms = median_run(fn, 3)
        scan[name] = {"solver": desc, "solves_per_s": round(64 / (ms / 1e3), 2), "total_ms": round(ms, 2),
                      "p50_ms": round(float(np.percentile(tb, 50)), 2), "p99_ms": round(float(np.percentile(tb, 99)), 2),
                      "all_converged": bool(all(bool(r.converged) for r in rb)),
                      "speedup_vs_fp64_solve_by_solve": round(sum(t_cg) / ms, 3),
                      "speedup_vs_fp64_scf_solve_by_solve": round(sum(t_scf) / ms, 3),
                      "speedup_vs_fp64_fast_scf_solve_by_solve": round(sum(t_fs) / ms, 3),
                      **errors([float(r.energy) for r in rb])}
    mixed_graph.close()
    fp64_graph.close()
    out["density_scan_64"] = scan
    out["gradients_96x96_nb4"] = run_gradients(dev, median_run, base["newton_96x96_nb4"])
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        # the 64 solves sharded over the ranks (greedy longest-first), FP64, batched per rank
        from jax_hf_b200.scan import batched_runner, scan_shapes, solve_scan
        run_local = batched_runner(probs, c64, lanes=16, device=dev)
        dist.barrier()
        res, ms = ev_time(lambda: solve_scan(scan_shapes(probs), run_local))
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        Es = np.array([r["energy"] for r in res])
        scan["fp64_sharded_over_ranks"] = {
            "ranks": dist.get_world_size(), "solves_per_s": round(len(probs) / (float(t) / 1e3), 2),
            "total_ms_max_over_ranks": round(float(t), 2),
            "max_abs_dE_vs_oracle_reference_cg": float(np.abs(Es - Ecg).max())}
    return out


def run_gradients(dev, median_run, oracle=None):
    """96x96 nb=4 scalar-V model: trust-region Newton (tol_grad 1e-6) and SCF-DIIS solves, then
    d Omega*/d(U, d, h_R) through the hand-written adjoint at the converged density, with a
    central difference of Omega in U at that density (step 1e-6) beside it.  ``oracle``: the
    oracle's record for this problem (its own Newton result and the fixed point)."""
    import torch
    import jax_hf_b200 as G
    from jax_hf_b200 import adjoint as A
    from jax_hf_b200 import synthetic as S
    from jax_hf_b200.reference_scf import SCFConfig, solve_scf
    from jax_hf_b200.solver import SolverConfig, solve

    p3 = S.newton_96()
    K = G.HartreeFockKernel(**p3.kernel_kwargs())
    P0 = torch.zeros((96, 96, 4, 4), dtype=torch.complex128, device=dev)
    out = {}
    ncfg = SolverConfig(optimizer="newton", tol_grad=1e-6, max_iter=200)
    # one untimed call first (first launches of each kernel, workspace allocation), then the
    # median of three
    solve(K, P0, p3.n_electrons, config=ncfg)
    rn, ms_n = median_run(lambda: solve(K, P0, p3.n_electrons, config=ncfg), 3)
    out["newton"] = {"ms_per_solve": round(ms_n, 2), "n_iter": int(rn.n_iter), "converged": bool(rn.converged),
                     "energy": float(rn.energy)}
    if oracle is not None:
        ra = oracle["reference_algorithm"]
        out["newton"].update(oracle_n_iter=ra["n_iter"], oracle_converged=ra["converged"],
                             rel_dE_vs_oracle_newton=abs(float(rn.energy) - ra["energy"]) / abs(ra["energy"]))
    scfg = SCFConfig(acceleration="diis", density_tol=1e-10, comm_tol=1e-9, max_iter=300)
    solve_scf(K, P0, p3.n_electrons, config=scfg)
    rs, ms_s = median_run(lambda: solve_scf(K, P0, p3.n_electrons, config=scfg), 3)
    out["scf_diis"] = {"ms_per_solve": round(ms_s, 2), "iterations": int(rs.iterations),
                       "converged": bool(rs.converged), "energy": float(rs.energy)}
    if oracle is not None:
        Ef = oracle["fixed_point_energy"]
        out["scf_diis"]["rel_dE_vs_oracle_fixed_point"] = abs(float(rs.energy) - Ef) / abs(Ef)
    dens = rs.density_matrix if bool(rs.converged) else rn.density
    dV = S.coulomb_scalar_derivatives(96, 1.0, 2.0)
    R = S.lattice_vectors(2.0)
    A.parameter_gradients(K, dens, coupling_derivatives=dV, lattice_vectors=R)
    A.parameter_gradients(K, dens, coupling_derivatives=dV, lattice_vectors=R)
    g, ms_g = median_run(lambda: A.parameter_gradients(K, dens, coupling_derivatives=dV, lattice_vectors=R), 3)
    step = 1e-6

    def e_at(U):
        Kx = G.HartreeFockKernel(**dict(p3.kernel_kwargs(), coulomb_q=S.coulomb_scalar(96, U, 2.0)))
        return float(A.objective(dens, torch.full((96, 96, 4), 0.5, dtype=torch.float64, device=dev), Kx))

    fd_U = (e_at(1.0 + step) - e_at(1.0 - step)) / (2 * step)
    out["gradients"] = {"ms": round(ms_g, 3), "n_params": 2 + len(R) * 16, "dOmega_dU": g["U"],
                        "dOmega_dd": g["d"], "fd_dOmega_dU_fixed_density": fd_U,
                        "rel_err_vs_fd": abs(fd_U - g["U"]) / max(abs(fd_U), 1e-300)}
    return out


def _finish(args, ws, rank, value, dev_ms, avg_us, n_builds, t_wall, clocks, variants, e2e_val,
            nbytes_state, P_np, prob):
    if rank != 0:
        return None
    peak, peak_kind = peaks()
    ab = alg_bytes(NK, NK, NB)
    achieved = ab / (avg_us * 1e-6) / 1e9
    traffic = None
    tf = ROOT / "profiles" / "fock_build_192x192_nb8_c128_fast_passes.md"
    if tf.exists():
        for ln in tf.read_text().splitlines():
            if ln.strip().startswith("traffic_bytes_per_build:"):
                traffic = int(ln.split(":")[1])
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(dev_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "mesh": [NK, NK], "nb": NB,
                   "l2": "flushed (256 MiB write) before every build", "parallelism": f"replicas x{ws}"},
        "builds_per_step": args.builds_per_step,
        "us_per_build": round(avg_us, 3),
        "wall_s_timed": round(t_wall, 3),
        "variants": variants,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one build's passes, "
                                       "from the committed capture profiles/fock_build_192x192_nb8_c128_fast_passes.md "
                                       "(not measured in this run)",
                     "algorithmic_bytes_per_build": ab, "peak_source": peak_kind},
        "e2e": None if e2e_val is None else {
            "value": round(e2e_val, 1), "unit": UNIT, "h2d_bytes_per_step": nbytes_state,
            "d2h_bytes_per_step": 2 * nbytes_state},
        "gpu_launches": 3 * n_builds,
        "clocks": clocks,
    }
    solves = variants.pop("solves", None)
    if solves is not None:
        line["solves"] = solves
    if args.cpu_baseline and ws == 1:
        line["cpu_baseline"] = cpu_baseline(P_np, prob)
    return line


def oracle_build(prob, P, workers):
    from oracle import hf_oracle as O
    O.FFT_WORKERS = workers
    Ko = O.Kernel(prob.weights, prob.hamiltonian, prob.coulomb_q, prob.T)
    a = Ko.as_args()

    def fn():
        return O.build_fock(P, h=a["h"], VR=a["VR"], refP=a["refP"], HH=a["HH"], w2d=Ko.w2d,
                            include_exchange=True, include_hartree=False,
                            exchange_hermitian_channel_packing=a["exchange_hermitian_channel_packing"],
                            contact_g=a["contact_g"], contact_Oi=a["contact_Oi"], contact_Oj=a["contact_Oj"])
    return fn


def cpu_baseline(P, prob, n=3):
    cores = os.cpu_count() or 1
    fn = oracle_build(prob, P, cores)
    fn()
    t = time.perf_counter()
    for _ in range(n):
        fn()
    dt = (time.perf_counter() - t) / n
    return {"value": round(1.0 / dt, 4), "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{n} oracle build_fock calls (NumPy/SciPy restatement, scipy.fft workers={cores}) "
                      f"on the same 192x192 nb=8 input; {dt:.3f} s per build"}


def jax_probe() -> str:
    """What importing the reference's dependency (JAX) gives on this machine."""
    try:
        import jax  # noqa: F401
        return f"jax {jax.__version__} importable"
    except Exception as exc:  # the reference cannot run without it
        return f"import jax failed: {type(exc).__name__}: {exc}"


def run_reference(args, ws, rank):
    if rank != 0:
        return None
    prob, P = make_inputs(1)
    cores = os.cpu_count() or 1
    fn = oracle_build(prob, P, cores)
    for _ in range(max(0, min(args.warmup, 1))):
        fn()
    t = time.perf_counter()
    for _ in range(args.steps):
        fn()
    dt = time.perf_counter() - t
    val = args.steps / dt
    sample = (f"each step = 1 oracle build_fock (NumPy/SciPy restatement of jax_hf's path; jax_hf itself cannot "
              f"run here: {jax_probe()}) on the 192x192 nb=8 complex128 input, scipy.fft workers={cores}")
    return {
        "impl": "reference", "metric": METRIC, "value": round(val, 4), "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * dt / args.steps, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic (seeded)", "config": {"workload": WORKLOAD, "mesh": [NK, NK], "nb": NB},
        "cpu_baseline": {"value": round(val, 4), "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": round(val, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--builds-per-step", type=int, default=STEP_BUILDS)
    ap.add_argument("--no-solves", dest="solves", action="store_false",
                    help="skip the whole-solve legs (SCF 24x24, CG 144x144, 64-solve density scan)")
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="skip the c64 / FP32-FFT variants and the e2e leg (short runs for profiling)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        ws = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        line = run_reference(args, ws, rank)
    else:
        ws, rank, local = setup_dist(args)
        line = run_ours(args, ws, rank, local)
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
