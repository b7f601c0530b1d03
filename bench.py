"""Benchmark of the recursion hot path: batched energy-dependent chains on the site-class operator.

Workload (the batched, uneven-depth configuration): fcc ternary Fe0.66Ni0.14Cr0.20-like random alloy, one site class,
spd 9 orbitals, NN + NNN Slater-Koster blocks (18 slots), 5^3-cell periodic cluster, closure to 3 levels, rank 1, D2h
reduction (all 9 orbitals one dimensional); 2 spins x 3 central species x 9 start orbitals = 54 chain groups with depths
drawn from U{16..28} (seed 1); energies: 48-point Gauss-Legendre semicircle plus 4096 real-axis energies (Im z = 0.005).
Seeded synthetic inputs stand in for the reference's LMTO potential parameters and structure constants.

One step = every chain group over a slice of 192 consecutive energies of that list (10368 chains); successive steps walk
through the list.  value = chain-steps / s (one Lanczos step of one chain at one energy), whole job, inputs resident in
HBM; e2e = the same through the host C-ABI call with host buffers (copies inside the timed region).
``--impl reference`` times the CPU restatement of the reference (oracle, OpenMP over chain tasks as chain_worker does).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NZ_SLICE = 192
# DRAM bytes (read + write) per launch of the step kernel from one ncu capture (64-energy slice of this workload), the
# algorithmic bytes of that launch and what was captured, per (precision, link-gather variant); traffic is scaled to the
# bench's mean launch
_TAB = 18 * 5 + 3 * 5 + 20
NCU_STEP_TRAFFIC = {
    ("fp64", "fixed-offset"): (3.171e9, 16 * 20969 * (2 * 4608.0 + _TAB),
                               "ncu capture of k_smul<double,1,1,1> (fixed-offset link gathers, a_k epilogue) at 16 tiles"),
    ("fp32", "fixed-offset"): (0.762e9, 8 * 20969 * (2 * 2304.0 + _TAB),
                               "ncu capture of k_smul<float,1,1,1> (fixed-offset link gathers, a_k epilogue, paired FMAs) at "
                               "8 tiles"),
    ("fp64", "general"): (3.30e9, 16 * 20969 * (2 * 4608.0 + _TAB),
                          "ncu capture of the general-link k_smul<double,1,1,0> at 16 tiles (before the a_k epilogue)"),
}


def roof(st, hbm_peak, pipe_peak=None):
    """Roofline entry of one kernel kind from its CUDA-event statistics: achieved algorithmic GB/s per launch and its
    fraction of the HBM peak, TFLOP/s and its fraction of the matching measured pipe peak."""
    if not st or st["launches"] == 0:
        return None
    per = st["ms"] / st["launches"]
    gbs = st["bytes"] / st["launches"] / (per / 1e3) / 1e9
    tf = st["flops"] / st["launches"] / (per / 1e3) / 1e12
    return {"launches": st["launches"], "per_launch_ms": per, "achieved_gbs": gbs, "hbm_frac": gbs / hbm_peak,
            "tflops": tf, "pipe_frac": (tf / pipe_peak) if pipe_peak else None}


def hbm_peak_of():
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        peaks = {}
    if "hbm_gbs" in peaks:
        return float(peaks["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured)"
    return 6650.0, "fallback 6650 GB/s (an earlier B200 copy measurement; no MEASURED_PEAKS.json)"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    p.add_argument("--nz-slice", type=int, default=NZ_SLICE)
    p.add_argument("--cpu-sample", type=int, default=1, help="run the bounded CPU baseline sample (1) or skip it (0)")
    p.add_argument("--e2e", type=int, default=1, help="time the host-buffer C-ABI path too (1) or skip it (0)")
    p.add_argument("--scf", type=int, default=1,
                   help="SCF leg: 0 none, 1 two timed iterations of each scheme at full size, 2 also the convergence on a "
                        "small cluster, 3 converged at full size")
    p.add_argument("--autotune", type=int, default=1, help="choose the batch shape by timing first (1) or use the defaults (0)")
    p.add_argument("--legs", default="1",
                   help="1: measure every leg (mixed precision with its DOS error, adjoint, general operator form, KPM, "
                        "plain, example, spectral, EPI), 0: none, or a comma list of leg names")
    p.add_argument("--lanes", type=int, default=0,
                   help="1: run the multi-GPU step (task split, lane chains, all-reduce of the shares) also on one GPU")
    p.add_argument("--adj-groups", type=int, default=0, help="adjoint leg: the first N chain groups (0: all 54)")
    p.add_argument("--adj-energies", type=int, default=48, help="adjoint leg: the first N of the 48 contour energies")
    p.add_argument("--adj-depth", type=int, default=0, help="adjoint leg: every chain this deep (0: the drawn depths)")
    p.add_argument("--link", default="auto", choices=["auto", "general", "fixed"],
                   help="step-kernel link gathers: the autotuner's choice (auto; general without --autotune), or pinned")
    return p.parse_args()


def workload():
    """Synthetic inputs of the configuration (host arrays only)."""
    from asr_b200 import synthetic as S
    return S.batched_ternary_workload()


def specs_of(groups):
    import asr_b200 as A
    return [A.ChainSpec(c=g["ed"]["c"], d=g["ed"]["d"], o=g["ed"]["o"], e=g["ed"]["e"], pa=g["ed"]["pa"], pb=g["ed"]["pb"],
                        frozen_sp=g["cen"], start_orb=g["l0"], nlev=g["nlev"]) for g in groups]


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(case, fl, groups, z, oop=None):
    """The oracle (CPU restatement of chain_greens / edc_green_blk) on a bounded sample with every host thread: the chain
    groups of start orbital 1 (2 spins x 3 central species), each over ceil(threads / 6) blocks of 4 energies, one task per
    thread and block as chain_worker schedules them (src/asr_class_scf.f90:1071-1160)."""
    from oracle import oracle as O
    nthr = os.cpu_count() or 1
    if oop is None:
        oop = O.OracleOp(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, 3, 1, fl)
    sel = [g for g in groups if g["l0"] == 1]
    nbe = 4
    nblk = max(1, -(-nthr // len(sel)))
    gps = [dict(c=g["ed"]["c"], d=g["ed"]["d"], o=g["ed"]["o"], e=g["ed"]["e"], dc=g["ed"]["dc"], dl=g["ed"]["dl"],
                enu=g["ed"]["enu"]) for g in sel]
    nlevq = np.array([[g["nlev"] for g in sel]], np.int32).T.copy()
    t0 = time.perf_counter()
    gz, steps = oop.chain_greens(gps, [g["cen"] for g in sel], [1], nlevq, z[: nbe * nblk], nbe, nthreads=nthr)
    t = time.perf_counter() - t0
    return {"value": steps / t, "unit": "chain-steps/s", "cores": nthr, "kind": "port", "wall_ms": 1000.0 * t,
            "sample": f"{len(sel)} chain groups x {nbe * nblk} energies in {len(sel) * nblk} tasks ({steps} chain-steps, "
                      f"{t:.1f} s), nn={oop.nn}, oracle edc_green_blk, {nthr} threads"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    case, fl, groups, z = workload()
    oop = O.OracleOp(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, 3, 1, fl)
    vals, walls = [], []
    for it in range(min(args.warmup, 1) + args.steps):
        r = cpu_baseline(case, fl, groups, z, oop)
        if it >= min(args.warmup, 1):
            vals.append(r["value"])
            walls.append(r["wall_ms"])
    v = float(np.mean(vals))
    line = {"metric": "chain-steps/s (batched energy-dependent chains, fcc ternary, 54 groups, depths 16-28)", "value": v,
            "unit": "chain-steps/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": float(np.mean(walls)), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": "fcc ternary Fe0.66Ni0.14Cr0.20, levels 3, rank 1, D2h, 54 chain groups, depth U{16..28}, "
                                   "48-pt contour + 4096 real energies", "sample": "bounded CPU sample per step"},
            "cpu_baseline": {"kind": r["kind"], "cores": r["cores"], "sample": r["sample"], "value": v, "unit": "chain-steps/s"},
            "e2e": {"value": v, "unit": "chain-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def fp32_peak_tflops(torch):
    """Measured FP32 matrix throughput (cuBLAS SGEMM 8192^3 without TF32, best of 3), the denominator of the FP32 pipe
    fractions."""
    torch.backends.cuda.matmul.allow_tf32 = False
    return fp64_peak_tflops(torch, torch.float32)


def fp64_peak_tflops(torch, dtype=None):
    """Measured FP64 matrix throughput of this GPU (cuBLAS DGEMM 8192^3, best of 3), the denominator of the FP64
    fraction of the chain step."""
    n = 8192
    dtype = dtype or torch.float64
    a = torch.randn(n, n, dtype=dtype, device="cuda")
    b = torch.randn(n, n, dtype=dtype, device="cuda")
    c = a @ b
    best = 1e30
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        c = a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b, c
    return 2.0 * n ** 3 / (best / 1000.0) / 1e12


def kpm_leg(torch):
    """KPM on the explicit supercell: fcc 40^3 conventional cells (256,000 sites, 12 NN + 6 NNN slots), species
    Fe/Ni/Cr-like 0.66 / 0.14 / 0.20 placed by seeded Metropolis swaps towards alpha_1 = -0.10, h = c + d S d; 2048
    Chebyshev moments over 64 Rademacher vectors (two moments per matvec), FP32 matvec and vectors with FP64 moments,
    timed, against the FP64 run (moment and Jackson-DOS error)."""
    from asr_b200 import kpm, synthetic as S
    t0 = time.perf_counter()
    nbr, spc, bvec, aout = kpm.fcc_supercell(40, [0.66, 0.14, 0.20], -0.10, seed=4, sweeps=4)
    block, block0 = S.sk_blocks(bvec, 4)
    c, d, o, e = S.plain_params(S.draw_species(3, 4))
    sc = kpm.Supercell(nbr, spc, c, d, o, e, block, block0)
    setup_s = time.perf_counter() - t0
    # spectral bound: |H| <= max|c| + max d^2 sum_slots |B_k|_inf + |B_0|_inf
    bn = sum(np.max(np.sum(np.abs(block[:, :, k]), axis=1)) for k in range(block.shape[2]))
    bound = np.max(np.abs(c)) + np.max(d) ** 2 * (bn + np.max(np.sum(np.abs(block0), axis=1)))
    cen, scl = 0.0, 1.05 * bound
    nmom, nvec = 2048, 64
    out = {"sites": int(sc.n), "rows": int(sc.dim), "moments": nmom, "vectors": nvec, "setup_s": setup_s,
           "alpha1_achieved": float(aout[0, 1])}
    sc.kpm_moments(cen, scl, 64, nvec, seed=5, precision="fp32")
    torch.cuda.synchronize()
    stats = {}
    for prec in ("fp32", "fp64"):
        sc.ctx.profile(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        mu = sc.kpm_moments(cen, scl, nmom, nvec, seed=5, precision=prec)
        e1.record()
        torch.cuda.synchronize()
        sc.ctx.profile(False)
        stats[prec] = sc.ctx.kernel_stats("kpm")
        ms = e0.elapsed_time(e1)
        out[prec] = {"ms": ms, "matvec_rows_per_s": (nmom // 2) * nvec * sc.dim / (ms / 1000.0),
                     "tflops": (nmom // 2) * nvec * sc.n * 2.0 * 81 * (1 + sc.ns) / (ms / 1000.0) / 1e12}
        out["mu_" + prec] = mu
    out["kernel_stats"] = stats
    m32, m64 = out.pop("mu_fp32"), out.pop("mu_fp64")
    egrid = np.linspace(cen - 0.99 * scl, cen + 0.99 * scl, 2000)
    r32, r64 = kpm.kpm_dos(m32, cen, scl, egrid), kpm.kpm_dos(m64, cen, scl, egrid)
    out["moment_error"] = float(np.max(np.abs(m32 - m64)))
    out["dos_error"] = float(np.max(np.abs(r32 - r64)) / np.max(np.abs(r64)))
    # algorithmic bytes per vector and Chebyshev step: 3 FP32 streams x 36 B + 1 B species per site
    out["fp32"]["hbm_gbs_algorithmic"] = (nmom // 2) * nvec * sc.n * (3 * 36 + 1) / (out["fp32"]["ms"] / 1000.0) / 1e9
    sc.free()
    out["asr_comparison"] = kpm_vs_asr(egrid, r64, c, d, o, e)
    return out


def kpm_vs_asr(egrid, dos_kpm, c, d, o, e, eta=0.02):
    """The KPM DOS of the supercell against the configuration-averaged ASR DOS of the same alloy: the site-class operator
    of the fcc ternary (0.66 / 0.14 / 0.20, the same NN + NNN blocks and species parameters, 5^3-cell cluster, levels 3,
    rank 1, D2h), plain real chains of depth 40 from every orbital of the start site frozen to each species, Beer-Pettifor
    tail, DOS per state sum_s x_s sum_l -Im G / (9 pi) at E + i eta; the Jackson-kernel KPM DOS convolved with the same
    Lorentzian of width eta.  The supercell carries short-range order (alpha_1 = -0.10), the single-site ASR configuration
    average does not, so the difference is the physics of the two models plus both methods' truncations."""
    import asr_b200 as A
    from asr_b200 import synthetic as S
    conc = [0.66, 0.14, 0.20]
    case = S.cubic_case("fcc", 5, 3, conc, seed=4, group="d2h")
    fl = np.ones(case["graph"].n, np.int32)
    fl[0] = 0
    op = A.build_augcls_operator(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, 3, maxrank=1,
                                 flippable=fl)
    specs = [A.ChainSpec(c=c, d=d, o=o, e=e, frozen_sp=s, start_orb=l0, nlev=40) for s in (1, 2, 3) for l0 in range(1, 10)]
    sel = np.arange(0, egrid.shape[0], 5)
    eg = egrid[sel]
    g = A.chains_run(op, specs, eg + 1j * eta, mode="plain", tail="bp")["g"].reshape(eg.shape[0], 3, 9)
    dos_asr = np.einsum("s,jsl->j", np.asarray(conc), -g.imag / np.pi) / 9.0
    de = egrid[1] - egrid[0]
    lor = eta / np.pi / ((eg[:, None] - egrid[None, :]) ** 2 + eta ** 2)
    dos_k = lor @ dos_kpm * de
    diff = np.abs(dos_k - dos_asr)
    return {"asr_nodes": int(op.nn), "energies": int(eg.shape[0]), "eta": eta,
            "max_abs_difference_over_max_dos": float(np.max(diff) / np.max(dos_asr)),
            "l1_difference_over_l1_dos": float(np.sum(diff) / np.sum(dos_asr)),
            "kpm_weight_in_window": float(np.sum(dos_k) * (eg[1] - eg[0])),
            "asr_weight_in_window": float(np.sum(dos_asr) * (eg[1] - eg[0]))}


def plain_leg(torch):
    """The CPU-runnable plain configuration: bcc A0.5B0.5 on one site class, D2h, levels 4, rank 1, 9 real chains of
    depth 12 (one per start orbital), Beer-Pettifor tail, G at 2000 real energies (Im z = 0.005): device time of the
    whole call and its DOS against the oracle's lanczos + terminated_green on the same operator."""
    import asr_b200 as A
    from asr_b200 import synthetic as S
    from oracle import oracle as O
    case = S.cubic_case("bcc", 4, 2, [0.5, 0.5], seed=0, group="d2h")
    fl = np.ones(case["graph"].n, np.int32)
    op = A.build_augcls_operator(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, 4, maxrank=1,
                                 flippable=fl)
    c, d, o, e = S.plain_params(S.draw_species(2, 0))
    specs = [A.ChainSpec(c=c, d=d, o=o, e=e, start_orb=l0, nlev=12) for l0 in range(1, 10)]
    z = np.linspace(-1.5, 1.0, 2000) + 0.005j
    A.chains_run(op, specs, z, mode="plain", tail="bp")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g = A.chains_run(op, specs, z, mode="plain", tail="bp")["g"]
    ms = (time.perf_counter() - t0) * 1000.0
    oop = O.OracleOp(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, 4, 1, fl)
    oop.set_params(c, d, o, e)
    t0 = time.perf_counter()
    err = 0.0
    for l0 in range(1, 10):
        oop.set_start(l0)
        v0 = np.zeros(oop.dim)
        v0[l0 - 1] = 1.0
        ao, bo, no = oop.lanczos(v0, 12)
        go, _ = O.terminated_green(ao, bo, no, z, "beer-pettifor")
        err = max(err, float(np.max(np.abs(g[:, l0 - 1].imag - go.imag)) / np.pi))
    ms_cpu = (time.perf_counter() - t0) * 1000.0
    return {"nodes": int(op.nn), "chains": 9, "depth": 12, "energies": 2000, "ms": ms, "oracle_ms_1thread": ms_cpu,
            "dos_abs_error_vs_oracle": err}


def example_leg(torch):
    """Chain throughput on the node set of the reference's bcc Cu0.5Zn0.5 example (levels 4, 17,515 nodes; the count
    of example/reference/cuzn_alloy/asr.out:105): 2 central species x start orbitals s, p_z, d_xy, d_3z2-r2 (one
    dimensional under the class group), depth 24 with the depth test at 1e-5, 8 contours of 77 energies each.
    chain-steps counts the levels each chain actually used; the whole host call (copies included) is timed, the way the
    reference's wall-clock chain count is."""
    import asr_b200 as A
    from asr_b200 import contour as CT
    from asr_b200 import synthetic as S
    c = S.example_case("cuzn_alloy", 1)
    op = A.build_augcls_operator(c["graph"], c["model"], c["cls"], c["perm"], c["dmat"], 1, c["maxlevel"],
                                 maxrank=c["maxrank"], flippable=c["flippable"])
    sp = S.draw_species(2, 7)
    specs = []
    for cen in (1, 2):
        ed = S.edc_params(sp, cen)
        for l0 in (1, 3, 5, 7):
            specs.append(A.ChainSpec(c=ed["c"], d=ed["d"], o=ed["o"], e=ed["e"], pa=ed["pa"], pb=ed["pb"], frozen_sp=cen,
                                     start_orb=l0, nlev=24))
    z = np.concatenate([CT.contour_nodes(-1.2 - 0.02 * k, 0.2 + 0.01 * k, 77)[0] for k in range(8)])
    A.chains_run(op, specs, z[:77], "edc", 1e-5, "hull", "fp64")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = A.chains_run(op, specs, z, "edc", 1e-5, "hull", "fp64")
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    steps = int(np.sum(r["m"]))
    chains = int(r["m"].size)
    val = steps / sec
    return {"nodes": int(op.nn), "chains": chains, "mean_depth_used": steps / chains, "seconds": sec,
            "chain_steps_per_s": val, "chains_per_s": chains / sec,
            "published_chain_steps_per_s": 1.40e3, "ratio_to_published": val / 1.40e3,
            "published_basis": "67 chains/s x 20.86 mean depth, 2 x 48 CPU threads (example/reference/cuzn_alloy/asr.out)"}


def spectral_leg(torch):
    """Projected chains (edc_green_proj) for the Bloch spectral function on the workload's operator: fcc ternary, D2h,
    targets = the sites within 1.5 alat of the origin (minimum image), 3 central species x 9 start orbitals x 64 real
    energies, depth 24.  Chain-steps/s with the projections against the same chains without them."""
    import asr_b200 as A
    from asr_b200 import spectral as SP
    from asr_b200 import synthetic as S
    case, fl, _, _ = workload()
    coord = case["coord"]
    m = 10
    h = (coord + m // 2) % m - m // 2
    sel = np.nonzero(np.sum(h * h, axis=0) <= int(4 * 1.5 ** 2 + 1e-9))[0]
    tsite = (sel + 1).astype(np.int32)
    op, tnode, tgop = A.build_augcls_operator(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, 3,
                                              maxrank=1, flippable=fl, tsite=tsite)
    sp = S.draw_species(3, seed=1)
    conc = [0.66, 0.14, 0.20]
    z = np.linspace(-1.2, 0.6, 64) + 0.01j
    t0 = int(np.nonzero(tsite == 1)[0][0])
    specs, tws = [], []
    for cen in (1, 2, 3):
        ed = S.edc_params(sp, cen)
        tw = np.zeros((9, op.nsmax, len(tsite)))
        for t in range(len(tsite)):
            tw[:, :, t] = SP.spectral_dressing(ed["dc"], ed["dl"], [1, 2, 3], conc, t == t0, op.nsmax)
        for l0 in range(1, 10):
            specs.append(A.ChainSpec(c=ed["c"], d=ed["d"], o=ed["o"], e=ed["e"], pa=ed["pa"], pb=ed["pb"], frozen_sp=cen,
                                     start_orb=l0, nlev=24))
            tws.append(tw)
    tw = np.stack(tws, axis=3)
    A.chains_proj(op, specs[:1], z[:4], tnode, tgop, tw[..., :1])
    torch.cuda.synchronize()
    t = time.perf_counter()
    r = A.chains_proj(op, specs, z, tnode, tgop, tw)
    torch.cuda.synchronize()
    sec_p = time.perf_counter() - t
    t = time.perf_counter()
    A.chains_run(op, specs, z, "edc", 0.0, "hull", "fp64")
    torch.cuda.synchronize()
    sec = time.perf_counter() - t
    steps = int(np.sum(r["m"]))
    return {"nodes": int(op.nn), "targets": int(len(tsite)), "chains": int(r["m"].size), "chain_steps_per_s": steps / sec_p,
            "without_projections": steps / sec, "projection_overhead": sec_p / sec - 1.0}


def epi_leg(torch):
    """EPI block chains (two projected chains per symmetry-adapted start vector) for a first-shell pair of a bcc binary:
    levels 4, rank 1, the pair group, the origin on the path 1 -> 2 at lambda = 0.5 and the partner at (1, 1, 1) frozen
    to species 2, 32 contour energies, depth 24."""
    import asr_b200 as A
    from asr_b200 import contour as CT
    from asr_b200 import epi as EP
    from asr_b200 import lattices as lat
    from asr_b200 import synthetic as S
    l = 8
    g, coord, bvec = lat.periodic_graph_shells("bcc", l, 4)
    block, block0 = S.sk_blocks(bvec, 2)
    jp = int(np.nonzero(np.all(coord == np.array([1, 1, 1])[:, None], axis=0))[0][0]) + 1
    cls = np.ones(g.n, np.int32)
    cls[jp - 1] = 2
    spc = np.asfortranarray(np.array([[1, 1], [2, 0]], np.int32))
    conc = np.asfortranarray(np.array([[0.5, 1.0], [0.5, 0.0]]))
    mdl = S.ClassModel(nsp=3, nsc=np.array([2, 1], np.int32), spc=spc, conc=conc,
                       block=np.asfortranarray(block.reshape(9, 9, -1, 1)), block0=np.asfortranarray(block0.reshape(9, 9, 1)))
    perm, mats = EP.epi_pair_ops(coord, 2 * l, cls)
    dmat = lat.orbital_rep(mats)
    fl = (cls == 1).astype(np.int32)
    fl[0] = 0
    op = A.build_augcls_operator(g, mdl, cls, perm, dmat, 1, 4, maxrank=1, flippable=fl)
    ll = S.ORB_L.astype(float)
    par = [EP.EpiPar(e=0.10 * ll, c=0.30 - 0.15 * ll, d=0.30 - 0.07 * ll, o=0.0 * ll),
           EP.EpiPar(e=0.05 * ll, c=0.45 - 0.10 * ll, d=0.27 - 0.06 * ll, o=0.0 * ll)]
    pt = EP.epi_path(par[0], par[1], 0.5)
    params, ed = EP.epi_setup(par, pt)
    vec, chi, lo = EP.epi_adapted(dmat)
    op.set_params(*params)
    op.freeze_any(1, 3)
    op.freeze_any(jp, 2)
    z, _ = CT.contour_nodes(-1.2, 0.3, 32)
    EP.epi_blocks(op, params, ed, vec[:, :1], chi[:, :1], lo[:1], z[:2], 24)
    torch.cuda.synchronize()
    t = time.perf_counter()
    x, m = EP.epi_blocks(op, params, ed, vec, chi, lo, z, 24)
    torch.cuda.synchronize()
    sec = time.perf_counter() - t
    steps = int(np.sum(m))
    return {"nodes": int(op.nn), "pair_group": int(perm.shape[1]), "chains": int(m.size), "chain_steps_per_s": steps / sec,
            "seconds": sec, "x1_mismatch_max": float(np.max(np.abs(x[3]) / np.abs(x[1])))}


def scf_model(l, maxlevel, precision):
    """The large batched SCF configuration: equiatomic 5-component fcc random alloy (Fe, Co, Ni, Cr, Mn-like parameters
    drawn from seed 4), spd 9 orbitals, spin-polarised (2 x 5 x 9 = 90 chain groups), depths U{20..32}, 64-point
    contour; model potential update (screened on-site response 0.08 Ry/e, exchange splitting 0.06 Ry per unit moment)."""
    import asr_b200 as A
    from asr_b200 import scf as SC, synthetic as S
    case = S.cubic_case("fcc", l, 5, [0.2] * 5, seed=4, group="d2h")
    fl = np.ones(case["graph"].n, np.int32)
    fl[0] = 0
    op = A.build_augcls_operator(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, maxlevel, maxrank=1,
                                 flippable=fl)
    sp = S.draw_species(5, 4)
    depths = np.random.default_rng(4).integers(20, 33, size=(2, 5, 9))
    return SC.ScfModel(op=op, x=np.full(5, 0.2), c0=sp.c, d=sp.d, delta=sp.delta, z=np.array([8.0, 9.0, 10.0, 6.0, 7.0]),
                       u=np.full(5, 0.08), stoner=np.full(5, 0.06), depths=depths, ebot=-2.0, ncont=64, precision=precision)


def scf_leg(torch, mode: int):
    """The large batched SCF configuration at full size (5^3-cell cluster, levels 3): time per SCF iteration of the
    reference's scheme (FP64 forward, E_F search, Anderson) against the mixed one (FP32 forward, E_F search, adjoint
    Jacobian, quasi-Newton step).  mode 1: two iterations of each; 2: also the iterations to a 1e-6 charge residual on a
    3^3-cell cluster at levels 2; 3: converged at full size."""
    from asr_b200 import scf as SC
    out = {}
    for prec, mixer in (("fp64", "anderson"), ("fp32", "broyden")):
        m = scf_model(5, 3, prec)
        q0 = np.vstack([m.z / 2 + 0.3, m.z / 2 - 0.3])
        torch.cuda.synchronize()
        r = SC.scf_run(m, q0, 0.0, mixer=mixer, tol=1e-6, maxit=40 if mode == 3 else 2)
        out[f"{prec}_{mixer}"] = {"seconds_per_iteration": r["seconds"] / r["iterations"], "iterations_run": r["iterations"],
                                 "converged": r["converged"], "forward_runs": r["stats"]["forward"],
                                 "adjoint_runs": r["stats"]["adjoint"], "nodes": int(m.op.nn),
                                 "residuals": [h["residual"] for h in r["history"]]}
    if mode == 2:
        for prec, mixer in (("fp64", "anderson"), ("fp32", "broyden")):
            m = scf_model(3, 2, prec)
            q0 = np.vstack([m.z / 2 + 0.3, m.z / 2 - 0.3])
            r = SC.scf_run(m, q0, 0.0, mixer=mixer, tol=1e-6, maxit=60)
            out[f"{prec}_{mixer}"]["iterations_to_1e-6_small_cluster"] = r["iterations"] if r["converged"] else None
            out[f"{prec}_{mixer}"]["small_cluster_nodes"] = int(m.op.nn)
    return out


def heusler_leg(torch):
    """The adjoint configuration itself: L2_1 four-sublattice bcc cell (one sublattice Cr0.6Fe0.4-like), depth 20, 32-point
    contour, edc_setup's o (o_l D_s / D_c), the Jacobian of the band energy and the four sublattice charges with respect to
    the 45 species parameters through torch.autograd and the device adjoint: time of the forward and of the Jacobian."""
    from asr_b200 import classes as CL
    from asr_b200 import contour as CT
    from asr_b200 import synthetic as S
    cases = [S.heusler_case(4, 3, k) for k in (1, 2, 3, 4)]
    sc = CL.SublatticeChains(cases, 20)
    sp = S.draw_species(5, 3)
    ol = torch.tensor(S.draw_o(5, 3), dtype=torch.float64)
    enu = torch.zeros(5, 3, dtype=torch.float64)
    z, w = CT.contour_nodes(-1.2, 0.2, 32)
    params = [torch.tensor(x, dtype=torch.float64, requires_grad=True) for x in (sp.c, sp.d, sp.delta)]
    sc.energy_and_charges(*params, enu, z, w, ol)   # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with torch.no_grad():
        sc.energy_and_charges(*params, enu, z, w, ol)
    torch.cuda.synchronize()
    t_fwd = time.perf_counter() - t0
    t0 = time.perf_counter()
    e_band, q = sc.energy_and_charges(*params, enu, z, w, ol)
    jac = []
    for o in [e_band] + [q[k] for k in range(4)]:
        gr = torch.autograd.grad(o, params, retain_graph=True)
        jac.append(np.concatenate([g.numpy().ravel() for g in gr]))
    torch.cuda.synchronize()
    t_jac = time.perf_counter() - t0
    nodes = [int(op.nn) for op in sc.ops]
    chains = sum(len(sc.groups(k)[0]) for k in range(4)) * len(z)
    return {"nodes": nodes, "chains": chains, "depth": 20, "energies": len(z), "parameters": 45, "outputs": 5,
            "forward_s": t_fwd, "jacobian_s": t_jac, "jacobian_over_forward": t_jac / t_fwd,
            "forward_chain_steps_per_s": chains * 20 / t_fwd, "jacobian_norm": float(np.linalg.norm(np.array(jac)))}


def general_leg(args, A, op, groups, z_all, stream):
    """The reference's whole operator form on the workload: edc_setup's o (o_l D_s / D_c, src/asr_edc.f90:66, with o_l
    drawn per spin from the spin's seed) in every group, so each chain step applies H = E_nu + h - h o h + X(z) as the
    unfused kernel sequence with two S applications.  FP64 chain-steps/s over one slice of real-axis energies next to the
    fused o = 0 step on the same slice, and the device time of the step's kernels per launch."""
    import torch
    from asr_b200 import synthetic as S
    nzs = args.nz_slice
    zs = z_all[48: 48 + nzs]
    specs_o = []
    for g in groups:
        sp = S.draw_species(3, seed=1 + g["spin"])
        ed = S.edc_params_o(sp, S.draw_o(3, 1 + g["spin"]), g["cen"])
        specs_o.append(A.ChainSpec(c=ed["c"], d=ed["d"], o=ed["o"], e=ed["e"], pa=ed["pa"], pb=ed["pb"], frozen_sp=g["cen"],
                                   start_orb=g["l0"], nlev=g["nlev"]))
    steps = int(sum(g["nlev"] for g in groups)) * nzs
    out = {"energies": nzs, "groups": len(groups), "precision": "fp64",
           "o": "edc_setup's o = o_l D_s / D_c, o_l = synthetic.draw_o(3, 1 + spin)"}
    op.ctx.hold_workspace(True)
    try:
        for name, sp_ in (("o_edc_setup", specs_o), ("o_zero", specs_of(groups))):
            A.chains_run(op, sp_, zs[:32], "edc", 0.0, "hull", "fp64")   # kernels loaded, workspace sized
            torch.cuda.synchronize()
            op.ctx.profile(True)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            A.chains_run(op, sp_, zs, "edc", 0.0, "hull", "fp64")
            e1.record(stream)
            torch.cuda.synchronize()
            op.ctx.profile(False)
            ms = e0.elapsed_time(e1)
            st = op.ctx.kernel_stats("step")
            out[name] = {"chain_steps_per_s": steps / (ms / 1000.0), "ms": ms, "operator_ms": st["ms"],
                         "operator_launches": st["launches"],
                         "operator_ms_per_launch": st["ms"] / max(st["launches"], 1)}
    finally:
        op.ctx.hold_workspace(False)
    out["o_zero_over_o_edc_setup"] = out["o_zero"]["chain_steps_per_s"] / out["o_edc_setup"]["chain_steps_per_s"]
    return out


def guarded(fn, *a):
    """A leg that raises is reported in the line (its error message) instead of ending the run."""
    try:
        return fn(*a)
    except Exception as e:
        return {"error": f"{type(e).__name__}: {e}"}


LEGS = ("mixed", "adjoint", "general", "heusler", "kpm", "plain", "example", "spectral", "epi")


def contour_weights(z_all):
    """dz weights of the 48-point semicircle (the first 48 energies of the workload) for the contour charge M_0."""
    ebot, ef = -1.2, 0.3
    x, wgl = np.polynomial.legendre.leggauss(48)
    th = 0.5 * np.pi * (1.0 - x)
    return z_all[:48], 0.5 * np.pi * wgl * 0.5j * (ef - ebot) * np.exp(1j * th)


def mixed_leg(args, A, op, specs, groups, z_all, step, stream, world):
    """The mixed-precision form (FP32 vectors and matvec, FP64 coefficients and fractions): chain-steps/s on the timed
    slices, and its DOS error against the FP64 run over the whole real axis (all 4096 energies, all 54 groups) and the
    error of the contour charge M_0 per group."""
    import torch
    nzs = args.nz_slice
    depth = np.array([g["nlev"] for g in groups])
    out = {"fp32_batch_shape": A.autotune(op, specs, z_all[:nzs], "fp32")}
    step(0, "fp32")
    torch.cuda.synchronize()
    nsteps = max(1, min(args.steps, 3))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for it in range(nsteps):
        step(args.warmup + it, "fp32")
    e1.record(stream)
    torch.cuda.synchronize()
    ms32 = e0.elapsed_time(e1)
    mixed = {"value": int(depth.sum()) * nzs * nsteps * world / (ms32 / 1000.0), "unit": "chain-steps/s", "steps": nsteps}
    zr = z_all[48:]
    g64 = A.chains_run(op, specs, zr, "edc", 0.0, "hull", "fp64")["g"]
    g32 = A.chains_run(op, specs, zr, "edc", 0.0, "hull", "fp32")["g"]
    dos64, dos32 = -g64.imag / np.pi, -g32.imag / np.pi
    mixed["dos_error"] = float(np.max(np.abs(dos32 - dos64)) / np.max(np.abs(dos64)))
    zc, wc = contour_weights(z_all)
    c64 = A.chains_run(op, specs, zc, "edc", 0.0, "hull", "fp64")["g"]
    c32 = A.chains_run(op, specs, zc, "edc", 0.0, "hull", "fp32")["g"]
    q64 = -np.imag(np.sum(wc[:, None] * c64, axis=0)) / np.pi
    q32 = -np.imag(np.sum(wc[:, None] * c32, axis=0)) / np.pi
    mixed["charge_error"] = float(np.max(np.abs(q32 - q64)))
    mixed["error_basis"] = ("max |DOS32 - DOS64| / max DOS64 over 54 groups x all 4096 real-axis energies (the whole band); "
                            "max |M0_32 - M0_64| of the 48-node contour charge per group")
    out["mixed"] = mixed
    return out


def adjoint_leg(args, A, op, specs, groups, z_all, stream):
    """Forward plus reverse sweep of all 54 groups over the 48 contour energies (seeds: the contour charge weights), in
    FP64 and in the mixed form, against the forward alone on the same energies; the mixed gradient's error against FP64."""
    import torch
    if args.adj_groups > 0 or args.adj_depth > 0:   # a smaller case of the same operator (profiling captures)
        groups = [dict(g, nlev=args.adj_depth or g["nlev"]) for g in groups[: args.adj_groups or len(groups)]]
        specs = specs_of(groups)
    depth = np.array([g["nlev"] for g in groups])
    zc, wc = contour_weights(z_all)
    zc, wc = zc[: args.adj_energies], wc[: args.adj_energies]
    w = np.repeat(wc[:, None], len(specs), axis=1)
    steps_adj = int(depth.sum()) * zc.shape[0]
    out, grads = {}, {}
    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return r, e0.elapsed_time(e1)

    for prec in ("fp64", "fp32"):
        # repeated gradients keep the vector memory in the context (asr_ctx_hold_workspace); the cold call allocates and
        # frees it (about 80 GB in FP64, 0.15-0.5 s of the call)
        op.ctx.hold_workspace(True)
        A.chains_adjoint(op, specs, zc[:8], w[:8], "hull", prec, True)
        A.chains_run(op, specs, zc[:8], "edc", 0.0, "hull", prec)   # the forward's kernels loaded before its timing
        torch.cuda.synchronize()
        (_, grads[prec]), msa = timed(lambda: A.chains_adjoint(op, specs, zc, w, "hull", prec, True))
        _, msf = timed(lambda: A.chains_run(op, specs, zc, "edc", 0.0, "hull", prec))
        op.ctx.hold_workspace(False)
        (_, gcold), msc = timed(lambda: A.chains_adjoint(op, specs, zc, w, "hull", prec, True))
        op.ctx.hold_workspace(True)
        # vectors kept only every ceil(sqrt(depth)) levels and recomputed between (the memory-lean mode); its gradient and
        # the allocating call's are compared with the held-workspace gradient
        stride = int(np.ceil(np.sqrt(depth.max())))
        A.chains_adjoint(op, specs, zc[:8], w[:8], "hull", prec, True, stride)
        (_, gck), msk = timed(lambda: A.chains_adjoint(op, specs, zc, w, "hull", prec, True, stride))
        # the reverse levels' device time from a separate profiled call (the timed call above records no events)
        op.ctx.profile(True)
        A.chains_adjoint(op, specs, zc, w, "hull", prec, True)
        torch.cuda.synchronize()
        op.ctx.profile(False)
        kst = op.ctx.kernel_stats("adjoint")
        fst = [op.ctx.kernel_stats(k) for k in ("step", "lanczos")]
        parts = {k: op.ctx.kernel_stats(k) for k in ("adj_step", "adj_vec", "adj_grad", "adj_scal")}
        op.ctx.hold_workspace(False)
        out[prec] = {"value": steps_adj / (msa / 1000.0), "forward_same_energies": steps_adj / (msf / 1000.0),
                     "adjoint_over_forward_time": msa / msf, "gradient_norm": float(np.linalg.norm(grads[prec])),
                     "cold_value": steps_adj / (msc / 1000.0), "cold_adjoint_over_forward_time": msc / msf,
                     "sqrt_checkpoint_stride": stride, "sqrt_checkpoint_value": steps_adj / (msk / 1000.0),
                     "sqrt_checkpoint_adjoint_over_forward_time": msk / msf,
                     "same_bits_cold_and_sqrt_checkpoint": bool(np.array_equal(gcold, grads[prec]) and
                                                                np.array_equal(gck, grads[prec])),
                     "max_rel_diff_cold": float(np.max(np.abs(gcold - grads[prec])) / np.max(np.abs(grads[prec]))),
                     "max_rel_diff_sqrt_checkpoint": float(np.max(np.abs(gck - grads[prec])) / np.max(np.abs(grads[prec]))),
                     "reverse_level_stats": kst, "reverse_share": kst["ms"] / msa,
                     "forward_step_stats": fst[0], "forward_lanczos_stats": fst[1],
                     "forward_kernel_share": (fst[0]["ms"] + fst[1]["ms"]) / msa,
                     "reverse_parts_ms": {k: v["ms"] for k, v in parts.items()}}
    out["unit"] = ("chain-steps/s (forward + reverse sweep; every level's vectors kept where a batch fits in half the free "
                   "device memory, else checkpoints every sqrt(depth) levels)")
    out["energies"], out["groups"] = int(zc.shape[0]), len(specs)
    out["fp32_gradient_error"] = float(np.max(np.abs(grads["fp32"] - grads["fp64"])) / np.max(np.abs(grads["fp64"])))
    # the FP64 entries under their former names
    out["value"], out["forward_same_energies"] = out["fp64"]["value"], out["fp64"]["forward_same_energies"]
    out["adjoint_over_forward_time"] = out["fp64"]["adjoint_over_forward_time"]
    return out


def run_legs(args, A, op, specs, groups, z_all, step, stream, world):
    """The legs chosen by --legs (all by default), each a dict in the JSON line's ``legs``."""
    import torch
    want = set(LEGS) if args.legs == "1" else set(x.strip() for x in args.legs.split(",") if x.strip())
    out = {}
    if "mixed" in want:
        out.update(mixed_leg(args, A, op, specs, groups, z_all, step, stream, world))
    if "adjoint" in want:
        out["adjoint"] = adjoint_leg(args, A, op, specs, groups, z_all, stream)
    if "general" in want:
        out["general"] = guarded(general_leg, args, A, op, groups, z_all, stream)
    out["fp64_peak_tflops"] = fp64_peak_tflops(torch)
    out["fp32_peak_tflops"] = fp32_peak_tflops(torch)
    if "kpm" in want:
        out["kpm"] = kpm_leg(torch)
    if "plain" in want:
        out["plain"] = plain_leg(torch)
    if "example" in want:
        out["example_cuzn"] = example_leg(torch)
    if "spectral" in want:
        out["spectral"] = spectral_leg(torch)
    if "epi" in want:
        out["epi"] = epi_leg(torch)
    if "heusler" in want:
        out["heusler"] = heusler_leg(torch)
    if args.scf and (args.legs == "1" or "scf" in want):
        out["scf"] = scf_leg(torch, args.scf)
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    split = world > 1 or args.lanes == 1
    if split:
        from datetime import timedelta
        if world == 1:
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            os.environ.setdefault("MASTER_PORT", "29517")
            dist.init_process_group("nccl", rank=0, world_size=1, timeout=timedelta(seconds=300))
        else:
            dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    import asr_b200 as A

    case, fl, groups, z_all = workload()
    ctx = A.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    t0 = time.perf_counter()
    op = A.build_augcls_operator(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, 3, maxrank=1,
                                 flippable=fl, ctx=ctx)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    specs = specs_of(groups)
    nzs = args.nz_slice
    nall = z_all.shape[0]
    z_dev = torch.from_numpy(z_all).to("cuda")
    g_dev = torch.zeros(len(specs) * nzs, dtype=torch.complex128, device="cuda")
    depth_per_group = np.array([g["nlev"] for g in groups])
    chain_steps_per_step = int(depth_per_group.sum()) * nzs

    # batch shape (tiles per batch, nodes per warp) chosen by timing on this operator (asr_autotune), outside the timed region
    tune = (A.autotune(op, specs, z_all[:nzs], args.precision) if args.autotune else
            {"tiles_per_batch": 16 if args.precision == "fp64" else 8, "nodes_per_warp": 4, "ms_tiles": None, "ms_npw": None,
             "link_gather": "general", "ms_link": None})
    if args.link != "auto":
        tune["link_gather"] = "fixed-offset" if args.link == "fixed" else "general"
        A.set_tuning(op, args.precision, tune["tiles_per_batch"], tune["nodes_per_warp"], tune["link_gather"])

    def slice_of(it):
        # one GPU: step it covers the it-th slice of nzs energies; N GPUs: step it covers N consecutive slices (weak
        # scaling), split over the ranks by the reference's task rule below
        return (it * world * nzs) % (nall - world * nzs + 1)

    # N > 1: the step's tasks are (group, block of 32 energies) as chain_greens numbers them, dealt to the ranks by the
    # cyclic rule with energy rotation (src/asr_class_scf.f90:1095-1097); each rank runs its lanes and one all-reduce of
    # the disjoint shares (par_sum_z) leaves the step's whole G on every rank
    from asr_b200 import distributed as D
    nzw = world * nzs
    lane_q, lane_j = D.rank_lanes(len(specs), nzw, 32, world, rank)
    lane_q_dev = torch.from_numpy(lane_q).to("cuda")
    lane_j_dev = torch.from_numpy(lane_j).to("cuda")
    gl_dev = torch.zeros(max(lane_q.size, 1), dtype=torch.complex128, device="cuda")
    zl_dev = torch.zeros_like(gl_dev)
    gz_dev = torch.zeros((len(specs), nzw), dtype=torch.complex128, device="cuda")

    def step(it, precision=args.precision):
        s0 = slice_of(it)
        if not split:
            A.chains_run_device(op, specs, z_dev[s0:s0 + nzs].data_ptr(), g_dev.data_ptr(), nzs, "edc", 0.0, "hull", precision)
            return
        zl_dev[: lane_j.size] = z_dev[s0 + lane_j_dev]
        A.chains_run_lanes_device(op, specs, lane_q, zl_dev.data_ptr(), gl_dev.data_ptr(), "edc" and 0.0, "hull", precision)
        gz_dev.zero_()
        gz_dev[lane_q_dev, lane_j_dev] = gl_dev[: lane_j.size]
        dist.all_reduce(torch.view_as_real(gz_dev), op=dist.ReduceOp.SUM)

    # repeated runs keep their vector memory in the context (asr_ctx_hold_workspace) instead of allocating and freeing
    # about 11 GB per call (FP64, 16 tiles)
    ctx.hold_workspace(True)
    for it in range(args.warmup):
        step(it)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk = Clocks(local)
    clk.start()
    ctx.profile(True)
    launches0 = ctx.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for it in range(args.steps):
        step(args.warmup + it)
    e1.record(stream)
    torch.cuda.synchronize()
    ctx.profile(False)
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    launches = ctx.launches() - launches0
    ks = ctx.kernel_stats("step")
    kl = ctx.kernel_stats("lanczos")
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    clocks = clk.stop()
    total_steps = chain_steps_per_step * args.steps * world
    value = total_steps / (ms / 1000.0)
    # e2e through the host C-ABI call (host z in pinned memory, host g; copies inside the timed region)
    # (N > 1: each rank its lanes of the step, then the disjoint-share sum of the host results)
    z_pinned = []
    for it in range(args.steps):
        s0 = slice_of(args.warmup + it)
        zs = z_all[s0 + lane_j] if split else z_all[s0: s0 + nzs]
        zt = torch.empty(zs.shape[0], dtype=torch.complex128).pin_memory()
        zt.numpy()[:] = zs
        z_pinned.append(zt)
    z_host = [zt.numpy() for zt in z_pinned]
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for it in range(args.steps if args.e2e else 0):
        if not split:
            r = A.chains_run(op, specs, z_host[it], "edc", 0.0, "hull", args.precision)
            _ = r["g"]
        else:
            gl, _ = A.chains_run_lanes(op, specs, lane_q, z_host[it], 0.0, "hull", args.precision)
            gz = np.zeros((len(specs), nzw), np.complex128)
            gz[lane_q, lane_j] = gl
            D.sum_disjoint(gz, dist, "cuda")
    e3.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e2.elapsed_time(e3) if args.e2e else float("nan")
    if world > 1:
        t = torch.tensor([ms_e2e], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e = total_steps / (ms_e2e / 1000.0)
    ctx.hold_workspace(False)
    # the legs measure single-GPU kernels and configurations: one GPU only (every rank skips them alike)
    legs = run_legs(args, A, op, specs, groups, z_all, step, stream, world) if args.legs != "0" and world == 1 else None
    nsp = 3
    h2d = nzs * 16 + len(specs) * 6 * 9 * nsp * 8
    d2h = len(specs) * nzs * (16 + 4)
    if split:   # lane energies in, lane results and depths out, and the step's G array through the all-reduce
        h2d = lane_j.size * 16 + len(specs) * 6 * 9 * nsp * 8 + len(specs) * nzw * 16
        d2h = lane_j.size * (16 + 4) + len(specs) * nzw * 16

    if rank == 0:
        hbm_peak, peak_source = hbm_peak_of()
        per_launch_ms = ks["ms"] / max(ks["launches"], 1)
        achieved = (ks["bytes"] / max(ks["launches"], 1)) / (per_launch_ms / 1000.0) / 1e9
        tflops = (ks["flops"] / max(ks["launches"], 1)) / (per_launch_ms / 1000.0) / 1e12
        cpu = cpu_baseline(case, fl, groups, z_all) if args.cpu_sample else None
        traffic, traffic_source = None, None
        if (args.precision, tune["link_gather"]) in NCU_STEP_TRAFFIC:
            meas, alg, traffic_source = NCU_STEP_TRAFFIC[(args.precision, tune["link_gather"])]
            traffic = meas * (ks["bytes"] / max(ks["launches"], 1)) / alg
            traffic_source += ", scaled to the mean launch"
        # every timed kernel kind: the chain step and the Lanczos update of the timed region, the KPM Chebyshev step and
        # the adjoint's reverse level of the legs
        pipe = None
        if legs:
            pipe = legs["fp64_peak_tflops"] if args.precision == "fp64" else legs["fp32_peak_tflops"]
        rooflines = {"step": roof(ks, hbm_peak, pipe), "lanczos": roof(kl, hbm_peak, pipe)}
        if legs and "kpm" in legs:
            for prec, st in legs["kpm"]["kernel_stats"].items():
                rooflines["kpm_" + prec] = roof(st, hbm_peak, legs[prec + "_peak_tflops"])
        if legs and "adjoint" in legs:
            for prec in ("fp64", "fp32"):
                rooflines["adjoint_level_" + prec] = roof(legs["adjoint"][prec]["reverse_level_stats"], hbm_peak,
                                                          legs[prec + "_peak_tflops"])
        line = {
            "metric": "chain-steps/s (batched energy-dependent chains, fcc ternary, 54 groups, depths 16-28)",
            "value": value, "unit": "chain-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32-matvec/f64-coefficients", "data": "synthetic",
            "config": {"workload": "fcc ternary Fe0.66Ni0.14Cr0.20, 5^3-cell cluster, levels 3, rank 1, D2h, 54 chain groups "
                                   "(2 spins x 3 species x 9 orbitals), depth U{16..28} seed 1, 48-pt contour + 4096 real "
                                   "energies", "nodes": op.nn, "slots": op.nslot, "energies_per_step": nzs,
                       "chains_per_step": len(specs) * nzs, "chain_steps_per_step": chain_steps_per_step,
                       "l2": "inputs larger than L2 (one 32-lane vector is %.0f MB)" % (op.nn * 9 * 32 * 16 / 1e6),
                       "parallelism": (f"chain tasks (group, 32-energy block) over {world} GPU(s) by the cyclic rule with "
                                       f"energy rotation, all-reduce of the disjoint G shares" if split else "one GPU"),
                       "energies_per_step_all_gpus": nzs * world, "operator_build_s": build_s,
                       "batch_shape": {"tiles_per_batch": tune["tiles_per_batch"], "nodes_per_warp": tune["nodes_per_warp"],
                                       "autotune_ms_tiles_4_8_16_32": tune["ms_tiles"], "autotune_ms_npw_1_2_4_8": tune["ms_npw"],
                                       "link_gather": tune["link_gather"], "autotune_ms_link_general_fixed": tune["ms_link"]},
                       "precision": args.precision,
                       "workspace": "vector memory held in the context across steps (asr_ctx_hold_workspace)"},
            "e2e": {"value": e2e, "unit": "chain-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                         "traffic": traffic, "traffic_source": traffic_source,
                         "kernel": "chain step operator (k_smul, fused S + diagonal + dot; %s link gathers)" % tune["link_gather"],
                         "per_launch_ms": per_launch_ms, "launches": ks["launches"], "fp64_tflops": tflops,
                         "share_of_step": ks["ms"] / ms, "peak_source": peak_source,
                         "fp64_frac": (tflops / legs["fp64_peak_tflops"]) if legs else None,
                         "fp64_peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                         "kernels": rooflines,
                         "kernels_basis": "CUDA events around every launch of each kind in its timed region; achieved = "
                                          "algorithmic bytes / time, hbm_frac against the HBM peak above, pipe_frac "
                                          "against the cuBLAS GEMM of the kernel's precision measured in this run"},
            "cpu_baseline": cpu,
            "legs": legs,
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        print(json.dumps(line))
    if split:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
