#!/usr/bin/env python
"""XC-build benchmark: grid points per second of one exchange-correlation build.

Workload (the metric's configuration): a seeded 60-atom C/H cluster (30 C,
30 H in a 12 Angstrom cube, d_min 1.1 Angstrom), C 4s3p1d / H 2s1p spherical
Gaussians (690 functions, exponents log-uniform in [0.05, 1e4]), 75 radial x
300 angular points per atom, PBE, 210 doubly occupied orbitals.  One step is
one full XC build (basis, density, functional, V_xc) over the whole grid.

  value : grid points/s with C already resident in HBM (pgxc_build_device)
  e2e   : grid points/s through pgxc_build with host buffers: C/occ copied
          host->device and the packed V_xc + E_xc/N_el read back every step

`--impl reference` times the CPU path of the reference algorithm instead
(the FP64 oracle port, all host threads, bounded sample per step).
With torchrun (N > 1) the grid is split into spatially compact blocks (Morton
order, whole 128-point tiles), one per GPU, and [packed V_xc, E_xc, N_el] is
summed with one NCCL all-reduce per build: the reduction ParaGauss does with
MPI_Reduce in xc_sndrcv.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "paragauss-gpl_b200"))

METRIC = "XC-build grid pts/s (mixed vs FP64 on B200 at |dExc|<1e-6 Eh; CPU ref beside)"
UNIT = "grid_points/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="pgxc", choices=["pgxc", "reference"])
    p.add_argument("--precision", default=None, help="fp64 | mixed (default: the headline path)")
    p.add_argument("--config", type=int, default=2)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-gradient", action="store_true", help="skip the XC nuclear gradient leg")
    p.add_argument("--profile-gradient", action="store_true",
                   help="create the raw-grid context of the workload and run one XC nuclear gradient (for ncu)")
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--max-chunk-points", type=int, default=0,
                   help="cap on grid points per device chunk (0: sized from free HBM)")
    p.add_argument("--screen", type=float, default=1e-10,
                   help="per-tile basis screening threshold (0: exact cutoff only, <0: dense layout)")
    p.add_argument("--profile", action="store_true",
                   help="one build only (for ncu): no warm-up loop, e2e, CPU baseline or peak probe")
    return p.parse_args()


def headline_precision():
    return "mixed"


# INT8 dense tensor-core rate relative to BF16 on sm_100 (4.5 vs 2.25 PFLOP/s nominal)
INT8_PER_BF16 = 2.0
# INT8 MMAs issued per FP64-equivalent product in the Ozaki split (digit pairs s + t <= 4 of 5 x 5)
OZAKI_PAIRS = 15


# ---------------------------------------------------------------------------
def workload_desc(case):
    return (f"{case.name}: {len(case.coords)} atoms, {case.nbas} spherical fns (l<=3), "
            f"{case.npts} grid pts ({case.meta['nrad']} radial x {case.meta['nang']}-class angular per atom), "
            f"nocc={case.nocc}, {case.functional}")


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        try:
            for line in open(self.f.name):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = np.array([float(r[1]) for r in rows])
        mx = float(rows[0][2])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        busy = sm[sm > 0.5 * mx] if np.any(sm > 0.5 * mx) else sm
        return {"sm_mhz": float(np.median(busy)), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


def cuda_timer(torch, fn, steps):
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(steps):
        fn()
    t1.record()
    torch.cuda.synchronize()
    return t0.elapsed_time(t1)


def fp64_peak_tflops(torch):
    """cuBLAS DGEMM throughput measured now: the FP64 tensor-pipe reference."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = 1e30
    for _ in range(3):
        best = min(best, cuda_timer(torch, lambda: torch.matmul(a, b), 1))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def shard(case, rank, world):
    """This rank's spatially compact block of the grid (pgxc.dist)."""
    if world == 1:
        return case
    from pgxc import dist as D
    return D.shard_case(case, D.spatial_shards(case.grid_xyz, world)[rank])


def algorithmic_flops(case):
    from pgxc import abi
    n, N = case.nbas, case.npts
    x = 2.0 * N * n * n
    v = 2.0 * N * n * n if abi.is_gga(case.functional) else 1.0 * N * n * n
    return x, v


def cpu_baseline(case, weights, seconds, threads=0):
    """Oracle port on host cores over a bounded sample of the workload: whole
    builds (or a contiguous prefix of the grid) repeated to ~`seconds`;
    threads = 0: all host threads."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    c = case
    c.grid_w = weights
    threads = threads or O.max_threads()
    pilot = min(c.npts, 65536 if threads > 1 else 8192)
    O.xc_build(c, pt_range=(0, min(c.npts, 4096)), nthreads=threads)  # thread start-up
    t = time.perf_counter()
    O.xc_build(c, pt_range=(0, pilot), nthreads=threads)
    rate = pilot / max(time.perf_counter() - t, 1e-6)
    n = int(min(c.npts, max(pilot, rate * seconds)))
    n = max(128, n // 128 * 128)
    reps = max(1, int(round(seconds / (n / rate))))
    t = time.perf_counter()
    for _ in range(reps):
        O.xc_build(c, pt_range=(0, n), nthreads=threads)
    dt = time.perf_counter() - t
    what = "the whole grid" if n == c.npts else f"the first {n} of {c.npts} grid points"
    return {"value": reps * n / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{reps} build(s) over {what} (128-point batches), {threads} OpenMP thread(s), "
                      f"OpenBLAS DGEMM; FP64 oracle restating the reference CPU path",
            "seconds": dt}


def fp64_comparison(torch, case, sub, local, args):
    """The plain FP64 build (the drop-in path, parity-checked against the
    oracle at 1e-10) on the same GPU: its throughput and its V_xc, E_xc, N_el
    as the accuracy reference of the headline path."""
    from pgxc import lib
    ctx = lib.Context(sub, precision="fp64", weighted=False, device=local, max_chunk_points=args.max_chunk_points,
                      screen_threshold=args.screen)
    dC = torch.from_numpy(case.c_fortran()).cuda()
    docc = torch.from_numpy(case.occ_fortran()).cuda()
    dham = torch.zeros(case.xc_length, dtype=torch.float64, device="cuda")
    dsum = torch.zeros(2, dtype=torch.float64, device="cuda")

    tm = {}

    def step():
        dham.zero_()
        dsum.zero_()
        tm.update(ctx.build_device(dC.data_ptr(), docc.data_ptr(), dham.data_ptr(), dsum.data_ptr()))

    for _ in range(2):
        step()
    steps = max(1, min(args.steps, 3))
    ms = cuda_timer(torch, step, steps) / steps
    out = {"ham": dham.cpu().numpy(), "exc": float(dsum[0]), "nel": float(dsum[1]), "ms": ms,
           "value": case.npts / (ms * 1e-3), "timings": dict(tm)}
    ctx.close()
    # the unscreened build costs 4 N nbas^2 flop: time it only where that is seconds
    if args.screen >= 0 and 4.0 * case.npts * case.nbas ** 2 < 2e14:
        ctx = lib.Context(sub, precision="fp64", weighted=False, device=local,
                          max_chunk_points=args.max_chunk_points, screen_threshold=-1.0)
        step()
        out["dense_ms"] = cuda_timer(torch, step, 2) / 2
        ctx.close()
    del dC, docc, dham, dsum
    torch.cuda.empty_cache()
    return out


def becke_leg(torch, case):
    """Becke partition weights of the workload's grid on the device (the
    allocation-free entry: device inputs, events around the kernels)."""
    import ctypes as ct
    from pgxc import lib
    natm = len(case.coords)
    if natm > 512:
        return None
    L = lib.lib()
    L.pgxc_becke_weights_noalloc.argtypes = [ct.c_int32, ct.c_void_p, ct.c_int64, ct.c_void_p, ct.c_void_p,
                                             ct.c_void_p, ct.c_void_p]
    coords = torch.from_numpy(np.ascontiguousarray(case.coords)).cuda()
    pts = torch.from_numpy(np.ascontiguousarray(case.grid_xyz.T).reshape(-1).copy()).cuda()
    own = torch.from_numpy(case.point_atom.astype(np.int32)).cuda()
    w = torch.zeros(case.npts, dtype=torch.float64, device="cuda")

    def run():
        st = L.pgxc_becke_weights_noalloc(natm, coords.data_ptr(), case.npts, pts.data_ptr(), own.data_ptr(),
                                          w.data_ptr(), None)
        if st != 0:
            raise RuntimeError(L.pgxc_last_error(None))

    run()
    ms = cuda_timer(torch, run, 3) / 3
    pairs = case.npts * natm * (natm - 1) / 2
    byts = case.npts * (3 * 8 + 4 + 8)  # point coordinates and host atom in, weight out
    return {"ms": ms, "points_per_s": case.npts / (ms * 1e-3), "pair_evals_per_s": pairs / (ms * 1e-3),
            "achieved_gbs": byts / (ms * 1e-3) / 1e9,
            "note": "FP64-ALU bound (natm^2/2 pair terms per point in the reference form); GB/s is secondary"}


def kernel_table(case, screen, tm, prec, mp, tpeak, args):
    """Per-kernel algorithmic work, measured time and roofline fraction of one
    build (library CUDA events around each kernel)."""
    from pgxc import abi
    gga = abi.is_gga(case.functional)
    arrays = 4 if gga else 1
    hbm = mp["hbm_gbs"]
    out = {}
    mixed = prec != "fp64"
    # bytes of one basis value and its gradient: phi in FP64; grad phi in FP32 in
    # the screened INT8 build, FP64 otherwise
    eb = 8.0 + ((12.0 if (mixed and screen is not None) else 24.0) if gga else 0.0)
    if screen is not None:
        nslots, sum_n2, ntl = screen["nslots"], screen["sum_n2"], screen["ntiles"]
        npts_t = 128.0 * ntl
        flops_x = 2.0 * 128 * sum_n2
        flops_v = flops_x if gga else 0.5 * flops_x
        # density: phi (+ grad phi) of every slot read once, rho (+ grad rho) written once
        bytes_x = eb * 128 * nslots + 8.0 * arrays * 128 * ntl
        # potential: phi (+ grad phi) of every slot read once, A (+ B) per point
        bytes_v = eb * 128 * nslots + 8.0 * arrays * npts_t
        bytes_b = eb * 128 * nslots  # basis: phi (+ grad phi) written
    else:
        flops_x = 2.0 * case.npts * case.nbas ** 2
        flops_v = flops_x if gga else 0.5 * flops_x
        bytes_x = 8.0 * arrays * case.npts * (case.nbas + 1)
        bytes_v = 8.0 * arrays * case.npts * (case.nbas + 1)
        bytes_b = 8.0 * arrays * case.npts * case.nbas
    issued = OZAKI_PAIRS if mixed else 1
    names = {"density": "k_sm_density" if mixed else ("k_sdensity" if screen is not None else "k_density"),
             "potential": "k_sm_vpot" if mixed else ("k_svpot" if screen is not None else "k_vpot")}
    if mixed and screen is not None:
        # the potential contraction reads the digits of phi and Z (5 B each per slot-point)
        bytes_v = 10.0 * 128 * nslots
    for key, ms, byts, fl in (("density", tm["xgemm_ms"], bytes_x, flops_x),
                              ("potential", tm["vgemm_ms"], bytes_v, flops_v)):
        gbs = byts / (ms * 1e-3) / 1e9
        tf = fl / (ms * 1e-3) / 1e12
        out[names[key]] = {"ms": ms, "algorithmic_bytes": byts, "achieved_gbs": gbs, "hbm_frac": gbs / hbm,
                           "algorithmic_tflops": tf, "issued_tops": tf * issued, "tensor_frac": tf * issued / tpeak}
    if mixed and screen is not None:
        # Z = A phi (+ B . grad phi) and the digits of Z and phi: the rest of the potential phase
        zms = tm["potential_ms"] - tm["vgemm_ms"]
        zb = eb * 128 * nslots + 8.0 * arrays * npts_t + 10.0 * 128 * nslots
        out["k_sm_zquant"] = {"ms": zms, "algorithmic_bytes": zb, "achieved_gbs": zb / (zms * 1e-3) / 1e9,
                              "hbm_frac": zb / (zms * 1e-3) / 1e9 / hbm,
                              "note": "phase time less the contraction kernel (includes the packing kernel)"}
    fb = 72.0 if gga else 32.0
    fms = tm["functional_ms"]
    out["k_functional"] = {"ms": fms, "algorithmic_bytes": fb * case.npts,
                           "achieved_gbs": fb * case.npts / (fms * 1e-3) / 1e9,
                           "hbm_frac": fb * case.npts / (fms * 1e-3) / 1e9 / hbm,
                           "note": "phase time: the functional kernel and its block-sum reduction"}
    bms = tm["basis_ms"]
    out["k_basis_items"] = {"ms": bms, "algorithmic_bytes": bytes_b, "achieved_gbs": bytes_b / (bms * 1e-3) / 1e9,
                            "hbm_frac": bytes_b / (bms * 1e-3) / 1e9 / hbm,
                            "note": "phase time: one launch per angular momentum and the padding kernel; "
                                    "FP64 ALU + exp bound with the stores of phi (and grad phi)"}
    return out


def keep_orbitals_leg(torch, case, sub, local, args):
    """Builds of one geometry with the basis values kept on the device
    (keep_orbitals, the reference's orbitals_in_memory): the first build
    evaluates and stores them, the timed builds reuse them.  Reported beside
    the headline, whose every step evaluates the basis."""
    from pgxc import lib
    ms = {}
    for prec in ("mixed", "fp64"):
        try:
            ctx = lib.Context(sub, precision=prec, weighted=False, device=local,
                              max_chunk_points=args.max_chunk_points, screen_threshold=args.screen, keep_orbitals=True)
        except lib.PgxcError as e:
            return {"unavailable": str(e)}
        dC = torch.from_numpy(case.c_fortran()).cuda()
        docc = torch.from_numpy(case.occ_fortran()).cuda()
        dham = torch.zeros(case.xc_length, dtype=torch.float64, device="cuda")
        dsum = torch.zeros(2, dtype=torch.float64, device="cuda")

        def step():
            ctx.build_device(dC.data_ptr(), docc.data_ptr(), dham.data_ptr(), dsum.data_ptr())

        for _ in range(3):
            step()
        ms[prec] = cuda_timer(torch, step, args.steps) / args.steps
        ctx.close()
        del dC, docc, dham, dsum
        torch.cuda.empty_cache()
    return {"ms_per_step": ms["mixed"], "value": case.npts / (ms["mixed"] * 1e-3), "unit": UNIT,
            "fp64_ms_per_step": ms["fp64"], "speedup_vs_fp64_kept": ms["fp64"] / ms["mixed"],
            "note": "basis values evaluated by the first build and reused by the timed ones (same geometry); "
                    "the headline value evaluates them in every build"}


def gradient_leg(torch, sub, local):
    """One post-SCF XC nuclear gradient of the geometry (pgxc_xc_gradient:
    moving grid, Becke weight derivatives; FP64), timed once after one
    untimed call.  Reported beside the headline; not a step of it."""
    from pgxc import lib
    try:
        ctx = lib.Context(sub, precision="fp64", weighted=False, device=local, screen_threshold=0.0)
    except lib.PgxcError as e:
        return {"unavailable": str(e)}
    try:
        ctx.xc_gradient()
        torch.cuda.synchronize()
        times = []
        for _ in range(2):
            t0 = time.perf_counter()
            g, e = ctx.xc_gradient()
            times.append((time.perf_counter() - t0) * 1e3)
    finally:
        ctx.close()
    return {"ms": min(times), "ms_calls": times, "E_xc": e, "max_abs_component": float(abs(g).max()), "sum_over_atoms": float(abs(g.sum(0)).max()),
            "note": "dE_xc/dR of every atom with the grid moving with its atoms and the Becke weights differentiated; "
                    "host wall clock around one synchronous call (inputs from host memory), the faster of two calls"}


# ---------------------------------------------------------------------------
def run_batch(args):
    """The batched workload: 256 seeded molecules of 3-40 atoms (LDA and PBE
    alternating), one screened INT8 context each, all device builds replayed
    as one CUDA graph.  Beside it, the same contexts built one by one and the
    plain FP64 path built one by one (pgxc_build_device per molecule)."""
    import torch
    from pgxc import cases, lib

    from pgxc import tune
    torch.cuda.set_device(0)
    mols = cases.molecule_set()
    npts = sum(m.npts for m in mols)
    # chunk sizes from the committed tuning table (pgxc/tune.py): the set's
    # chunk of concatenated tiles, and the FP64 contexts' own chunks
    table = tune.load()
    set_chunk = args.max_chunk_points or tune.choose_set(mols, table)
    chunk = args.max_chunk_points or 32768

    def operands():
        dC = [torch.from_numpy(m.c_fortran()).cuda() for m in mols]
        docc = [torch.from_numpy(m.occ_fortran()).cuda() for m in mols]
        dham = [torch.zeros(m.xc_length, dtype=torch.float64, device="cuda") for m in mols]
        dsum = [torch.zeros(2, dtype=torch.float64, device="cuda") for m in mols]
        return dC, docc, dham, dsum

    def one_by_one(ctxs, ops, steps):
        dC, docc, dham, dsum = ops

        def step():
            for c, a, o, h, s in zip(ctxs, dC, docc, dham, dsum):
                c.build_device(a.data_ptr(), o.data_ptr(), h.data_ptr(), s.data_ptr())
        step()
        return cuda_timer(torch, step, steps) / steps

    # plain FP64 path, one molecule after another
    ops64 = operands()
    ctx64 = [lib.Context(m, precision="fp64", weighted=False, max_chunk_points=chunk, screen_threshold=args.screen)
             for m in mols]
    ms64 = one_by_one(ctx64, ops64, max(1, min(args.steps, 2)))
    e64 = np.array([float(s[0]) for s in ops64[3]])
    # the FP64 builds as one graph (concurrent branches)
    b64 = lib.Batch(ctx64, *[[t.data_ptr() for t in x] for x in ops64])
    b64.run()
    ms64_batch = cuda_timer(torch, b64.run, max(1, min(args.steps, 2))) / max(1, min(args.steps, 2))
    b64.close()
    for c in ctx64:
        c.close()
    del ctx64
    torch.cuda.empty_cache()

    # INT8, one molecule after another, with the same per-context chunks as the FP64 path
    ctx8 = [lib.Context(m, precision="mixed", weighted=False, max_chunk_points=chunk, screen_threshold=args.screen)
            for m in mols]
    ms_seq = one_by_one(ctx8, ops64, max(1, min(args.steps, 2)))
    for c in ctx8:
        c.close()
    del ctx8, ops64
    torch.cuda.empty_cache()

    # the set: the contexts' own chunk buffers stay small (the set does not use them); the set has its own
    ctxs = [lib.Context(m, precision="mixed", weighted=False, max_chunk_points=4096, screen_threshold=args.screen)
            for m in mols]
    ops = operands()
    dC, docc, dham, dsum = ops
    batch = lib.Batch(ctxs, [t.data_ptr() for t in dC], [t.data_ptr() for t in docc], [t.data_ptr() for t in dham],
                      [t.data_ptr() for t in dsum], max_chunk_points=set_chunk)
    gstats = batch.stats()
    batch_is_set = batch.is_set()
    for _ in range(max(args.warmup, 3)):
        batch.run()
    torch.cuda.synchronize()
    with Clocks(0) as clk:
        ms = cuda_timer(torch, batch.run, args.steps) / args.steps
    clocks = clk.summary()
    e8 = np.array([float(s[0]) for s in dsum])
    n8 = np.array([float(s[1]) for s in dsum])

    # end to end: pinned host C / occ in, packed V and {E, N} out, every step
    hC = [torch.from_numpy(m.c_fortran()).pin_memory() for m in mols]
    hocc = [torch.from_numpy(m.occ_fortran()).pin_memory() for m in mols]
    hham = [torch.zeros(m.xc_length, dtype=torch.float64).pin_memory() for m in mols]
    hsum = [torch.zeros(2, dtype=torch.float64).pin_memory() for m in mols]

    def e2e_step():
        for a, b in zip(dC, hC):
            a.copy_(b, non_blocking=True)
        for a, b in zip(docc, hocc):
            a.copy_(b, non_blocking=True)
        torch.cuda.synchronize()
        batch.run()
        for a, b in zip(hham, dham):
            a.copy_(b, non_blocking=True)
        for a, b in zip(hsum, dsum):
            a.copy_(b, non_blocking=True)
        torch.cuda.synchronize()

    e2e_step()
    ms_e = cuda_timer(torch, e2e_step, args.steps) / args.steps
    batch.close()
    for c in ctxs:
        c.close()
    h2d = sum((m.nbas * m.nocc + m.nocc) * 8 for m in mols)
    d2h = sum((m.xc_length + 2) * 8 for m in mols)
    out = {
        "metric": METRIC, "value": npts / (ms * 1e-3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "s8 x s8 -> s32 tensor (5-digit Ozaki split of f64) + f64",
        "data": "synthetic",
        "config": {"workload": f"{len(mols)} molecules of 3-40 C/H/O atoms, {min(m.nbas for m in mols)}-"
                               f"{max(m.nbas for m in mols)} functions, {npts} grid pts in total, VWN and PBE "
                               f"alternating", "precision": "mixed",
                   "screening": f"per 128-point tile, threshold {args.screen:g}",
                   "batching": f"one context per molecule; the INT8 builds of all molecules run as one set: "
                               f"per chunk of their concatenated 128-point tiles ("
                               f"{'at most ' + str(set_chunk) + ' points' if set_chunk else 'sized from free memory'}"
                               f", from the tuning table) one launch of each kernel walking tiles of many "
                               f"molecules, captured with the per-molecule P preparation in one CUDA graph, "
                               f"one replay per step",
                   "tuning": {"key": tune.set_key(npts), "max_chunk_points": set_chunk,
                              "table": "paragauss-gpl_b200/pgxc/tune_b200.json" if table else None},
                   "l2": "no flush: each step streams several GB of basis data (inputs larger than L2)"},
        "molecules_per_s": len(mols) / (ms * 1e-3),
        "one_by_one": {"mixed_ms_per_set": ms_seq, "fp64_ms_per_set": ms64,
                       "fp64_batch_ms_per_set": ms64_batch,
                       "batch_speedup_vs_mixed_one_by_one": ms_seq / ms,
                       "batch_speedup_vs_fp64_one_by_one": ms64 / ms,
                       "max_abs_dE_xc_vs_fp64": float(np.max(np.abs(e8 - e64))),
                       "note": "the same molecules through pgxc_build_device one after another"},
        "N_el_total": float(n8.sum()),
        "roofline": None,
        "roofline_note": "builds of many molecules share one graph; per-kernel rooflines are reported by the "
                         "single-system workloads",
        "e2e": {"value": npts / (ms_e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": ms_e},
        "gpu_launches": gstats["kernel_nodes"] * args.steps, "graph_nodes": gstats["nodes"], "clocks": clocks,
        "set": batch_is_set,
    }
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
def run_reference(args):
    from pgxc import cases
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    case = cases.config(args.config)
    threads = O.max_threads()
    # bounded sample per step: ~10 s of CPU work
    n_probe = min(case.npts, 2048)
    sub = shard(case, 0, 1)
    sub.grid_w = None
    probe = cases.Case(**{**case.__dict__})
    probe.grid_xyz = case.grid_xyz[:n_probe]
    probe.grid_wraw = case.grid_wraw[:n_probe]
    probe.point_atom = case.point_atom[:n_probe]
    O.weight_case(probe)
    t = time.perf_counter()
    O.xc_build(probe)
    rate = n_probe / max(time.perf_counter() - t, 1e-6)
    total_budget = 150.0
    per_step = max(2.0, min(12.0, total_budget / max(1, args.steps + args.warmup)))
    n = int(min(case.npts, max(n_probe, rate * per_step)))
    n = max(128, n // 128 * 128)
    samp = cases.Case(**{**case.__dict__})
    samp.grid_xyz = case.grid_xyz[:n]
    samp.grid_wraw = case.grid_wraw[:n]
    samp.point_atom = case.point_atom[:n]
    O.weight_case(samp)
    for _ in range(args.warmup):
        O.xc_build(samp)
    t = time.perf_counter()
    for _ in range(args.steps):
        O.xc_build(samp)
    dt = (time.perf_counter() - t) / args.steps
    value = n / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_desc(case), "precision": "fp64", "path": "CPU"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"first {n} of {case.npts} grid points per step (contiguous 128-point "
                                   f"batches), {threads} OpenMP threads, OpenBLAS DGEMM; the Fortran reference "
                                   f"cannot be compiled here, so the FP64 oracle port restating it is timed"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return
    if args.config == 4:
        if rank == 0:
            run_batch(args)
        return
    import torch
    import torch.distributed as dist
    from pgxc import cases, lib

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    prec = args.precision or headline_precision()
    case = cases.config(args.config)
    sub = shard(case, rank, world)
    if args.profile_gradient:
        g = gradient_leg(torch, sub, local)
        print(json.dumps({"profile_gradient": True, **g}), flush=True)
        return
    fp64_leg = None
    if prec != "fp64" and world == 1 and not args.profile:
        fp64_leg = fp64_comparison(torch, case, sub, local, args)
    ctx = lib.Context(sub, precision=prec, weighted=False, device=local, max_chunk_points=args.max_chunk_points,
                      screen_threshold=args.screen)
    screen = ctx.screen_stats() if args.screen >= 0 else None
    if args.profile:
        d = ctx.build(timings=True)
        print(json.dumps({"profile": True, "precision": prec, "E_xc": d[1], "N_el": d[2], "timings": d[3]}),
              flush=True)
        ctx.close()
        return
    weights = ctx.grid_weights()
    nb, nocc = case.nbas, case.nocc
    dC = torch.from_numpy(case.c_fortran()).cuda()
    docc = torch.from_numpy(case.occ_fortran()).cuda()
    # [packed V, E_xc, N_el]: one all-reduce per build over NCCL (xc_sndrcv)
    dbuf = torch.zeros(case.xc_length + 2, dtype=torch.float64, device="cuda")
    dham, dsum = dbuf[:-2], dbuf[-2:]
    last_tm = {}

    def step():
        last_tm.update(ctx.build_device(dC.data_ptr(), docc.data_ptr(), dham.data_ptr(), dsum.data_ptr()))
        if world > 1:
            dist.all_reduce(dbuf)

    for _ in range(max(args.warmup, 3)):
        step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        ms = cuda_timer(torch, step, args.steps)
    clocks = clk.summary()
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    per_step = ms / args.steps
    value = case.npts / (per_step * 1e-3)
    exc, nel = dsum.tolist()

    # end to end through the host-buffer C ABI call
    C_host = torch.from_numpy(case.c_fortran()).pin_memory()
    occ_host = torch.from_numpy(case.occ_fortran()).pin_memory()
    ham_host = np.zeros(case.xc_length)

    def e2e_step():
        ham_host[:] = 0.0
        h, e, q = ctx.build(C=C_host.numpy(), occ=occ_host.numpy(), ham=ham_host)
        if world > 1:
            tb = torch.from_numpy(np.concatenate([h, [e, q]])).cuda()
            dist.all_reduce(tb)
            h[:] = tb[:-2].cpu().numpy()
        return e

    for _ in range(2):
        e2e_step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ms_e = cuda_timer(torch, e2e_step, args.steps)
    t = torch.tensor([ms_e], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_e = float(t.item())
    e2e_value = case.npts / (ms_e / args.steps * 1e-3)
    h2d = (nb * nocc + nocc) * 8
    d2h = (case.xc_length + 2) * 8

    # roofline of the dominant kernel of the build (the larger of the two
    # contraction kernels; per launch from the library's CUDA events around it)
    roof = None
    kernels = None
    if rank == 0:
        mp = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        dgemm_peak = fp64_peak_tflops(torch)
        if prec == "fp64":
            tpeak = dgemm_peak
            tsrc = "cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor pipe)"
        else:
            tpeak = mp["bf16_tflops"] * INT8_PER_BF16
            tsrc = "INT8 dense rate taken as 2 x MEASURED_PEAKS.json bf16_tflops (burst), of measured"
        kernels = kernel_table(case, screen, last_tm, prec, mp, tpeak, args)
        single = [k for k in kernels if k in ("k_sm_density", "k_sm_vpot", "k_sm_zquant", "k_sdensity", "k_svpot",
                                              "k_density", "k_vpot")]
        dom = max(single, key=lambda k: kernels[k]["ms"])
        kd = kernels[dom]
        traffic = None
        tf = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tf):
            traffic = json.load(open(tf)).get(f"{case.name}:{prec}:{args.screen:g}:{dom}")
        # the roof the kernel is nearest to: DRAM for the streaming kernels, the
        # tensor pipe (INT8 ops issued, or FP64 DMMA) for a contraction whose
        # operand bytes are small beside its MMA work
        tensor_bound = kd.get("tensor_frac", 0.0) > kd["hbm_frac"]
        roof = {"bound": "tensor" if tensor_bound else "hbm", "kernel": dom,
                "achieved": kd["issued_tops"] if tensor_bound else kd["achieved_gbs"],
                "peak": tpeak if tensor_bound else mp["hbm_gbs"],
                "unit": ("TOP/s" if prec != "fp64" else "TFLOP/s") if tensor_bound else "GB/s",
                "frac": kd["tensor_frac"] if tensor_bound else kd["hbm_frac"], "traffic": traffic,
                "hbm": {"achieved": kd["achieved_gbs"], "peak": mp["hbm_gbs"], "unit": "GB/s", "frac": kd["hbm_frac"]},
                "peak_source": tsrc if tensor_bound else "MEASURED_PEAKS.json hbm_gbs, of measured",
                "algorithmic_bytes": kd["algorithmic_bytes"], "kernel_ms_per_build": kd["ms"],
                "tensor": None if "tensor_frac" not in kd else {
                    "algorithmic_tflops": kd["algorithmic_tflops"], "issued_tflops_or_tops": kd["issued_tops"],
                    "peak": tpeak, "frac_issued": kd["tensor_frac"], "peak_source": tsrc},
                "phase_ms": {k: last_tm[k] for k in ("basis_ms", "density_ms", "functional_ms", "potential_ms",
                                                     "xgemm_ms", "vgemm_ms")}}
        if fp64_leg is not None:
            k64 = kernel_table(case, screen, fp64_leg["timings"], "fp64", mp, dgemm_peak, args)
            kernels["fp64_build"] = {k: v for k, v in k64.items() if k in ("k_sdensity", "k_svpot", "k_density",
                                                                          "k_vpot")}
            kernels["fp64_build"]["fp64_tensor_peak_tflops"] = dgemm_peak
            kernels["fp64_build"]["note"] = ("FP64 DMMA contractions of the drop-in build: algorithmic TFLOP/s "
                                             "against cuBLAS DGEMM measured in this run")
        if world == 1 and not args.profile:
            kernels["k_becke"] = becke_leg(torch, case)

    out = None
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": per_step, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64" if prec == "fp64" else "s8 x s8 -> s32 tensor (5-digit Ozaki split of f64) + f64", "data": "synthetic",
            "config": {"workload": workload_desc(case), "precision": prec,
                       "screening": ("none (dense)" if screen is None else
                                     f"per 128-point tile, threshold {args.screen:g}: "
                                     f"{screen['nlisted'] / screen['ntiles']:.1f} listed functions per tile "
                                     f"of {case.nbas}, {screen['sum_n2'] / (screen['ntiles'] * case.nbas ** 2):.3f} "
                                     f"of the dense n^2 work"),
                       "parallelism": (f"grid split over {world} GPU(s) in Morton blocks of 128-point tiles, "
                                       "one NCCL all-reduce of [packed V_xc, E_xc, N_el] per build"),
                       "l2": "no flush: each build streams several GB of basis/Z data (inputs larger than L2)"},
            "xc_builds_per_s": 1e3 / per_step, "E_xc": exc, "N_el": nel,
            "vs_fp64": None if fp64_leg is None else {
                "fp64_phase_ms": {k: fp64_leg["timings"][k] for k in ("basis_ms", "density_ms", "functional_ms",
                                                                      "potential_ms")},
                "fp64_value": fp64_leg["value"], "fp64_ms_per_step": fp64_leg["ms"],
                "speedup": fp64_leg["ms"] / per_step,
                "dE_xc": exc - fp64_leg["exc"], "dN_el": nel - fp64_leg["nel"],
                "max_dV_xc": float(np.max(np.abs(dham.cpu().numpy() - fp64_leg["ham"]))),
                "fp64_dense_ms_per_step": fp64_leg.get("dense_ms"),
                "note": "FP64 GPU build, same screening, same GPU, this run (matches the FP64 oracle to 1e-10); "
                        "fp64_dense: the unscreened FP64 build"},
            "roofline": roof,
            "kernels": kernels,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": ms_e / args.steps},
            "gpu_launches": int(last_tm["kernel_launches"]) * args.steps,
            "clocks": clocks,
        }
    if world > 1:
        dist.barrier()
    ctx.close()
    if rank == 0 and world == 1 and args.screen >= 0:
        del dC, docc, dbuf, dham, dsum
        torch.cuda.empty_cache()
        out["keep_orbitals"] = keep_orbitals_leg(torch, case, sub, local, args)
        if not args.no_gradient:
            out["xc_gradient"] = gradient_leg(torch, sub, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(case, weights, args.cpu_seconds)
        out["cpu_baseline_1thread"] = cpu_baseline(case, weights, min(args.cpu_seconds, 6.0), threads=1)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
