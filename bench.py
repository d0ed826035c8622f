"""Throughput of the B200 force-and-integration engine on the 200k-atom butane
NPT workload (flexible butane, 14,286 molecules = 200,004 atoms, 130 A box,
anisotropic MTK barostat at 1 atm + NHC thermostat at 250 K, rc 12 A, SPME
128^3 order 5, dt 1 fs, mixed precision, RATTLE on the X-H bonds).

A step is one outer MD step (dt_long) of moldyn_mtk, pair-list rebuilds
included at their natural interval (nstep_book = 50).  Synthetic, seeded
inputs of that shape (no dataset).  The working set (pair list ~0.6 GB) is
larger than L2, so no explicit flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (one per GPU, no collective on the data
path: the reference path does not shard); value = all ranks' atom-steps / max
rank time.  --impl reference times the CPU restatement of the reference
algorithm (the Fortran reference cannot be compiled in this image) on the
host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-steps/s (200k-atom butane NPT, mixed precision)"
UNIT = "atom-steps/s"
WORKLOAD = "butane_200004_npt_mtk_aniso_nhc_spme128_o5_rc12_dt1fs"
NSTEP_BOOK = 50


def make_system(precision):
    from thrid_b200 import systems as S
    s = S.butane_box(precision=precision)
    s.params["nstep_book"] = NSTEP_BOOK
    return s


def md_params(s, nstep_short=1):
    from thrid_b200 import abi
    from thrid_b200 import systems as S
    T = S.kelvin_to_reduced(250.0)
    return abi.md_struct(S.fs_to_reduced(1.0), nstep_short=nstep_short, mchain=3, text=T,
                         tfreq=1.0e13 * S.TIMEREF, vfreq=0.2e12 * S.TIMEREF, pext=S.pa_to_reduced(1.01325e5),
                         pcont_axis=abi.PCONT_ANISO, degfree=s.degfree_all, ifrattle=1, eps_rattle=1e-7,
                         outinterval=0)


def ns_per_day(steps_per_s, dt_fs=1.0):
    return steps_per_s * dt_fs * 86400.0 * 1e-6


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def profiled_traffic(name="k_pair_mixed_butane200k.md"):
    """DRAM bytes (read + write) per launch of one kernel from its committed
    ncu summary under profiles/ (line 'traffic_bytes_per_launch: X')."""
    p = os.path.join(ROOT, "profiles", name)
    try:
        for ln in open(p):
            if ln.startswith("traffic_bytes_per_launch:"):
                return float(ln.split(":", 1)[1])
    except (OSError, ValueError):
        pass
    return None


def period_window(warmup, steps, nb):
    """Timed window of whole pair-list periods: the first step after the
    warm-up that opens a period (step % nb == 1) and a length of at least
    `steps` rounded up to a multiple of nb, so the window holds its list
    rebuilds (steps % nb == 0) at exactly their natural rate."""
    n = max(steps, nb)
    n = -(-n // nb) * nb
    s0 = warmup + 1
    s0 += (1 - s0) % nb
    return s0, n


def run_ours(args, rank, world, local_rank):
    import torch
    from thrid_b200 import abi
    from thrid_b200.pgk import PgkEngine

    torch.cuda.set_device(local_rank)
    s = make_system(abi.PREC_MIXED)
    md = md_params(s)
    eng = PgkEngine(s)
    stream = torch.cuda.ExternalStream(eng.stream)
    eng.set_chain(abi.chain_init(s.box))
    step0, nsteps = period_window(args.warmup, args.steps, NSTEP_BOOK)
    # ---- warm-up: step 0 (initial forces), the W warm-up steps and the rest
    #      of their list period ----
    eng.moldyn_mtk(0, step0 - 1, md)
    eng.sync()
    dist_barrier(world)
    launches0 = eng.kernel_launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize()
        dist_barrier(world)
        e0.record(stream)
        ene = eng.moldyn_mtk(step0, step0 + nsteps - 1, md)
        e1.record(stream)
        torch.cuda.synchronize()
        dist_barrier(world)
    ms = e0.elapsed_time(e1)
    launches = eng.kernel_launches - launches0
    ms_max = dist_max(ms, world)
    nxt = step0 + nsteps
    # ---- end to end through the public API with host buffers ----
    e2e = None if args.no_e2e else e2e_leg(eng, s, md, nxt, nsteps, world)
    # ---- the all-FP64 device path on the same state (the mixed-vs-FP64 comparison) ----
    fp64 = None if args.no_fp64 else fp64_leg(eng, s, md, stream)
    # ---- rooflines of the dominant kernel and the HBM-bound kernels, measured
    #      live (last: the kick/drift launches move the atoms) ----
    roof, roof_hbm = roofline(eng, s)
    eng.close()
    natom = s.natom
    value = world * natom * nsteps / (ms_max / 1e3)
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": nsteps,
        "warmup": args.warmup, "ms_per_step": ms_max / nsteps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32+int64 (pair/SPME/bonded), fp64 (x, v, RATTLE, MTK)",
        "data": "synthetic (seeded butane lattice, OPLS-like parameters)",
        "config": {"workload": WORKLOAD, "natom": natom, "replicas": world, "global_batch": world * natom,
                   "parallelism": f"replicas{world}", "nstep_book": NSTEP_BOOK,
                   "steps_requested": args.steps,
                   "timed_window": f"steps {step0}..{step0 + nsteps - 1}: whole pair-list periods, "
                                   f"{nsteps // NSTEP_BOOK} list rebuilds inside (1 per {NSTEP_BOOK} steps)",
                   "l2": "working set > L2 (pair list ~0.6 GB), no flush"},
        "ns_per_day": ns_per_day(nsteps / (ms_max / 1e3)),
        "e2e": e2e, "gpu_launches": launches, "roofline": roof, "roofline_hbm": roof_hbm, "fp64_path": fp64,
        "energies_last": {k: ene[k] for k in ("pot_tot", "pot_vdw", "pot_elc", "pot_ewk")} if ene else None,
    }
    out["clocks"] = clk.summary()
    from thrid_b200.pgk import tuning_table
    out["autotune"] = tuning_table().splitlines()
    if rank == 0 and not args.no_configs:
        out["other_configs"] = other_configs(args)
    if rank == 0 and world == 1 and not args.no_serve:
        # the replica-serving workload in a bounded form: 32 seeded
        # replicas x 2,000 NVE steps, against this line's single large system
        sa = argparse.Namespace(**vars(args))
        sa.serve_replicas, sa.serve_steps, sa.serve_hf = 32, 2000, False
        sv = run_serve(sa, single={"value": value, "unit": UNIT, "steps": nsteps, "workload": WORKLOAD,
                                   "note": "this line's own timed window"})
        sv.pop("autotune", None)
        out["serving"] = sv
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args)
    return out


def fp64_leg(eng, s, md, stream):
    """The FP64 device path (the parity path) on the mixed run's current state:
    force RMS relative error of the mixed path against it (both MTS groups,
    same positions) and its own MD throughput on the same workload, timed
    over one whole pair-list period (its list rebuild included)."""
    import torch
    from thrid_b200 import abi
    from thrid_b200.pgk import PgkEngine
    cor, vel, box = eng.download_state()
    ch = eng.get_chain()
    fm = eng.calforce(abi.MTS_LONG)[0] + eng.calforce(abi.MTS_SHORT)[0]
    e64 = PgkEngine(s, dict(s.params, precision=abi.PREC_FP64), upload=False)
    try:
        e64.upload_state(cor, vel, box)
        e64.set_chain(ch)
        f64 = e64.calforce(abi.MTS_LONG)[0] + e64.calforce(abi.MTS_SHORT)[0]
        err = float(np.sqrt(((fm - f64) ** 2).sum() / (f64 ** 2).sum()))
        st64 = torch.cuda.ExternalStream(e64.stream)
        s0, nsteps = period_window(3, NSTEP_BOOK, NSTEP_BOOK)
        e64.moldyn_mtk(0, s0 - 1, md)
        e64.sync()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(st64)
        e64.moldyn_mtk(s0, s0 + nsteps - 1, md)
        b.record(st64)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / nsteps
    finally:
        e64.close()
    return {"value": s.natom / (ms / 1e3), "unit": UNIT, "ms_per_step": ms, "steps": nsteps,
            "timed_window": f"steps {s0}..{s0 + nsteps - 1} (one list period, its rebuild inside)",
            "force_rel_rms_mixed_vs_fp64": err}


def e2e_leg(eng, s, md, start, nsteps, world):
    """Host-driver ownership of the state (like the Fortran module arrays):
    every step uploads x, v from pinned host memory, runs one outer step
    through pgk_moldyn_mtk and reads x, v (the step's result) back into
    pinned host memory.  The window covers whole pair-list periods, like the
    device-timed one; energies are not read (no output step, as between the
    reference's outinterval steps)."""
    import torch
    from thrid_b200 import abi
    n = s.natom
    md_e2e = abi.MdParamsStruct.from_buffer_copy(md)
    md_e2e.outinterval = 1 << 30                     # no output step inside the window
    cor = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    vel = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    cn, vn = cor.numpy(), vel.numpy()
    eng.download_state(cn, vn)
    s0 = start + (1 - start) % NSTEP_BOOK
    eng.moldyn_mtk(start, s0 - 1, md_e2e)            # reach a period start; capture the step graph
    eng.download_state(cn, vn)
    torch.cuda.synchronize()
    dist_barrier(world)
    t0 = time.perf_counter()
    for k in range(nsteps):
        eng.upload_state(cn, vn)
        eng.moldyn_mtk(s0 + k, s0 + k, md_e2e)
        eng.download_state(cn, vn)
    torch.cuda.synchronize()
    dt = dist_max(time.perf_counter() - t0, world)
    return {"value": world * n * nsteps / dt, "unit": UNIT, "steps": nsteps, "ms_per_step": 1e3 * dt / nsteps,
            "h2d_bytes_per_step": 2 * 24 * n, "d2h_bytes_per_step": 2 * 24 * n,
            "path": "pgk_upload_state (pinned x, v) -> pgk_moldyn_mtk (1 step) -> pgk_download_state (pinned x, v)"}


# algorithmic bytes per unit of the HBM-bound kernels (formula beside each entry)
HBM_KERNELS = (
    # (bench id, name, profile summary, unit, bytes(natom, K3, entries))
    (1, "k_spread_rows<5> (fill_charge_grid)", "k_spread_rows_butane200k.md",
     "N*16 + K^3*16", lambda n, k3, e: n * 16 + k3 * 16),
    (2, "k_gather_rows<5> (grad_sum)", "k_gather_rows_butane200k.md",
     "N*16 + K^3*4 + N*24", lambda n, k3, e: n * 16 + k3 * 4 + n * 24),
    (5, "k_kick_drift (long kick + drift)", "k_kick_drift_butane200k.md",
     "N*(48 + 48 + 24 + 8)", lambda n, k3, e: n * 128),
    (4, "list build chain (k_cell_* + k_build_clist)", "k_build_clist_butane200k.md",
     "N*(24 + 16) + 4 * list entries", lambda n, k3, e: n * 40 + 4 * e),
)


def roofline(eng, s):
    """Pair kernel against the FP32 pipe; spread, gather, kick/drift and the
    list build against the measured HBM copy bandwidth.  Each kernel is timed
    with CUDA events on the context's stream (pgk_bench_kernel, 20 launches
    after one warm-up launch)."""
    import ctypes as C
    ms = C.c_double(); units = C.c_double(); entries = C.c_double()
    st = eng.L.pgk_bench_kernel(eng.h, 0, 20, C.byref(ms), C.byref(units), C.byref(entries))
    if st != 0:
        return {"error": f"pgk_bench_kernel status {st}"}, None
    flop = 61.0 * units.value                       # algorithmic flop per interacting pair
    achieved = flop / (ms.value * 1e-3) / 1e12       # TFLOP/s
    peaks = measured_peaks()
    clk = peaks.get("sm_max_mhz", 1965.0)
    peak = 148 * 128 * 2 * clk * 1e6 / 1e12           # FP32 CUDA-core FMA peak at the max SM clock
    traffic = profiled_traffic()
    pair = {"kernel": "k_pair_mixed<PM_TENS> (regular instance on the pruned rows)", "bound": "fp32",
            "achieved": achieved, "peak": peak,
            "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
            "peak_source": f"nominal FP32 FMA peak 148 SM x 128 lanes x 2 x {clk:.0f} MHz "
                           "(MEASURED_PEAKS.json has no FP32 CUDA-core figure)",
            "ms_per_launch": ms.value, "pairs_per_launch": units.value, "list_entries": entries.value,
            "hbm_gbs_index_stream": entries.value * 4 / (ms.value * 1e-3) / 1e9,
            "hbm_peak_gbs": peaks.get("hbm_gbs")}
    hbm_peak = peaks.get("hbm_gbs")
    k3 = float(s.params["nfft1"] * s.params["nfft2"] * s.params["nfft3"])
    rows = []
    for kid, name, prof, formula, fbytes in HBM_KERNELS:
        km = C.c_double()
        st = eng.L.pgk_bench_kernel(eng.h, kid, 20, C.byref(km), None, None)
        if st != 0:
            rows.append({"kernel": name, "error": f"pgk_bench_kernel status {st}"})
            continue
        b = float(fbytes(s.natom, k3, entries.value))
        gbs = b / (km.value * 1e-3) / 1e9
        rows.append({"kernel": name, "bound": "hbm", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s",
                     "frac": gbs / hbm_peak if hbm_peak else None, "traffic": profiled_traffic(prof),
                     "algorithmic_bytes": b, "bytes_formula": formula, "ms_per_launch": km.value,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if hbm_peak else None})
    return pair, rows


def cpu_baseline(args, nsteps=None, threads=None):
    """The oracle (C++ FP64 restatement of the reference loops) on the host
    cores, on a bounded sample of the same workload: `nsteps` outer MTK steps
    timed after step 0, plus the share 1/nstep_book of one timed list build
    (the reference rebuilds its list every nstep_book steps)."""
    from oracle import oracle as orc
    from thrid_b200 import abi
    threads = threads or os.cpu_count() or 1
    s = make_system(abi.PREC_FP64)
    md = md_params(s)
    o = orc.Oracle(s, threads=threads)
    o.set_chain(abi.chain_init(s.box))
    t0 = time.perf_counter()
    st, _ = o.moldyn(2, 0, 0, md)              # list build + initial forces (not timed)
    t_init = time.perf_counter() - t0
    nsteps = nsteps or 3
    t0 = time.perf_counter()
    st2, _ = o.moldyn(2, 1, nsteps, md)        # steps 1..nsteps: no list build falls inside
    dt = time.perf_counter() - t0
    t0 = time.perf_counter()
    o.mklist()
    t_list = time.perf_counter() - t0
    per_step = dt / nsteps + t_list / NSTEP_BOOK
    return {"value": s.natom / per_step, "unit": UNIT, "cores": threads, "kind": "port",
            "steps": nsteps, "ms_per_step": 1e3 * per_step,
            "sample": f"{nsteps} outer MTK steps of the 200,004-atom butane system after step 0 "
                      f"({1e3 * dt / nsteps:.0f} ms each) plus 1/{NSTEP_BOOK} of one list build "
                      f"({1e3 * t_list:.0f} ms); step 0 (list + forces, {t_init:.1f} s) untimed",
            "status": int(st2)}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    cb = cpu_baseline(args, nsteps=max(1, min(args.steps, 3)))
    natom = 200004
    return {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": world, "steps": cb["steps"],
            "warmup": args.warmup, "ms_per_step": cb["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp64", "data": "synthetic (seeded butane lattice)",
            "config": {"workload": WORKLOAD, "natom": natom, "replicas": 1, "global_batch": natom,
                       "parallelism": "host threads", "nstep_book": NSTEP_BOOK, "steps_requested": args.steps,
                       "timed_window": cb["sample"], "l2": "host run"},
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference Fortran cannot be compiled here (no gfortran); its C++ restatement runs instead; "
                    "each step of the run is a bounded sample (steps = the steps actually timed)"}


def _timed_md(eng, kind, s0, n, md, stream):
    """CUDA-event time (ms) of moldyn steps s0..s0+n-1 on the context's stream."""
    import torch
    fn = {"nve": eng.moldyn_nve, "nhc": eng.moldyn_nhc, "mtk": eng.moldyn_mtk}[kind]
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    fn(s0, s0 + n - 1, md)
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b)


def nve_drift(s, prec, nchunk=10, chunk=200):
    """NVE drift of the total energy (pot_tot + KE) over nchunk*chunk steps at
    1 fs: least-squares slope per ns, with its standard error, in units of
    eref per atom and of the mean kinetic energy."""
    from thrid_b200 import abi
    from thrid_b200 import systems as S
    from thrid_b200.pgk import PgkEngine
    eng = PgkEngine(s, dict(s.params, precision=prec))
    md = abi.md_struct(S.fs_to_reduced(1.0), ifrattle=1, outinterval=0)
    eng.moldyn_nve(0, 0, md)
    t, E, K = [], [], []
    for k in range(nchunk):
        e = eng.moldyn_nve(k * chunk + 1, (k + 1) * chunk, md)
        kint, _, _ = eng.calpress()
        t.append((k + 1) * chunk * 1e-6)                    # ns
        E.append(e["pot_tot"] + 0.5 * kint)
        K.append(0.5 * kint)
    eng.close()
    t, E = np.asarray(t), np.asarray(E)
    (slope, icpt), cov = np.polyfit(t, E, 1, cov=True)
    se = float(np.sqrt(cov[0, 0]))
    return {"per_atom_eref_per_ns": slope / s.natom, "stderr_per_atom_eref_per_ns": se / s.natom,
            "per_mean_ke_per_ns": slope / np.mean(K), "steps": nchunk * chunk}


def _md_leg(s, kind, md, prec, warm, n, hf=False):
    """Throughput of one configuration on its own context: atom-steps/s over
    steps warm+1..warm+n (whole list periods when n is a multiple of 50)."""
    import torch
    from thrid_b200 import abi
    from thrid_b200.pgk import PgkEngine
    eng = PgkEngine(s, dict(s.params, precision=prec))
    st = torch.cuda.ExternalStream(eng.stream)
    if kind in ("nhc", "mtk"):
        eng.set_chain(abi.chain_init(s.box))
    if hf:
        eng.set_hf(s.regions["hf"])
        eng.moldyn_hf(0, warm, md, cap=1)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(st)
        _, rec = eng.moldyn_hf(warm + 1, warm + n, md, cap=n)
        b.record(st)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        cor, vel, _ = eng.download_state()
        eng.close()
        return ms, rec, cor, vel
    {"nve": eng.moldyn_nve, "nhc": eng.moldyn_nhc, "mtk": eng.moldyn_mtk}[kind](0, warm, md)
    ms = _timed_md(eng, kind, warm + 1, n, md, st)
    eng.close()
    return ms, None, None, None


def _zprofile(s, cor, vel, nbin):
    """z-resolved kinetic temperature (reduced) per slab of the box height."""
    m = s.atmmass
    z = np.mod(cor[:, 2], s.box[2])
    b = np.minimum((z / s.box[2] * nbin).astype(int), nbin - 1)
    ke = 0.5 * m * (vel ** 2).sum(1)
    cnt = np.bincount(b, minlength=nbin)
    kes = np.bincount(b, weights=ke, minlength=nbin)
    return np.where(cnt > 0, 2.0 * kes / (3.0 * np.maximum(cnt, 1)), 0.0), cnt


def other_configs(args):
    """The other named shapes at 1 GPU, mixed precision (each on its own
    context, CUDA-event timed, list rebuilds inside the window):
      C1 rigid water 1536 atoms NVE (+ NVE drift per ns, FP64 and mixed),
      C2 flexible propanol 12,000 atoms NHC,
      C3 alcohol/water slab 43,200 atoms, NVE + region Langevin + per-atom
         heat flux every step (+ J(t) and z temperature profile of the mixed
         path against the FP64 path over the same steps)."""
    from thrid_b200 import abi
    from thrid_b200 import systems as S
    out = {}
    dt = S.fs_to_reduced(1.0)
    c1 = S.water_box(precision=abi.PREC_MIXED)
    md = abi.md_struct(dt, ifrattle=1, outinterval=0)
    ms, *_ = _md_leg(c1, "nve", md, abi.PREC_MIXED, 49, 1000)
    d64 = nve_drift(c1, abi.PREC_FP64)
    dmx = nve_drift(c1, abi.PREC_MIXED)
    out["C1_water_1536_nve"] = {"value": c1.natom * 1000 / (ms / 1e3), "unit": UNIT, "steps": 1000,
                                "ms_per_step": ms / 1000, "ns_per_day": ns_per_day(1000 / (ms / 1e3)),
                                "nve_drift_fp64": d64, "nve_drift_mixed": dmx}
    c2 = S.propanol_box(precision=abi.PREC_MIXED)
    T = S.kelvin_to_reduced(300.0)
    md2 = abi.md_struct(dt, mchain=3, text=T, tfreq=1.0e13 * S.TIMEREF, degfree=c2.degfree_all, ifrattle=1,
                        outinterval=0)
    ms, *_ = _md_leg(c2, "nhc", md2, abi.PREC_MIXED, 49, 200)
    out["C2_propanol_12000_nhc"] = {"value": c2.natom * 200 / (ms / 1e3), "unit": UNIT, "steps": 200,
                                    "ms_per_step": ms / 200, "ns_per_day": ns_per_day(200 / (ms / 1e3))}
    res = {}
    for prec in (abi.PREC_MIXED, abi.PREC_FP64):
        c3 = S.slab_box(precision=prec)
        md3 = abi.md_struct(dt, ifrattle=1, outinterval=0)
        res[prec] = (c3,) + _md_leg(c3, "nve", md3, prec, 49, 100, hf=True)
    c3, ms, rec, cor, vel = res[abi.PREC_MIXED]
    _, ms64, rec64, cor64, vel64 = res[abi.PREC_FP64]
    vols = np.array([(b - a) for a, b in c3.regions["hf"]["regions"]]) * c3.box[0] * c3.box[1]
    jt = (rec[:, :, 17] * vols).sum(1)                 # total J_z(t) of the slab, per step
    jt64 = (rec64[:, :, 17] * vols).sum(1)
    nbin = len(c3.regions["hf"]["regions"])
    tp, cnt = _zprofile(c3, cor, vel, nbin)
    tp64, _ = _zprofile(c3, cor64, vel64, nbin)
    occ = cnt > 0
    out["C3_slab_43200_hf_langevin"] = {
        "value": c3.natom * 100 / (ms / 1e3), "unit": UNIT, "steps": 100, "ms_per_step": ms / 100,
        "ns_per_day": ns_per_day(100 / (ms / 1e3)), "fp64_ms_per_step": ms64 / 100,
        "hf_records": int(rec.shape[0]), "regions": nbin,
        "jz_rel_rms_mixed_vs_fp64": float(np.sqrt(((jt - jt64) ** 2).mean() / (jt64 ** 2).mean())),
        "tprofile_max_rel_err_mixed_vs_fp64": float(np.max(np.abs(tp[occ] - tp64[occ]) / tp64[occ])),
        "note": "same seeded start and Langevin stream; 100 steps after a 49-step warm-up"}
    return out


# ---- torch.distributed plumbing (replicas; barrier + max over ranks only) ----
_pg = None


def dist_init():
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE): NCCL
    on GPUs, gloo on a host without CUDA (the multi-process tests).  The
    ranks run independent replicas; the process group only carries the
    barriers around the timed window and the max over ranks of its time."""
    global _pg
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        cuda = torch.cuda.is_available()
        if cuda:
            torch.cuda.set_device(local)
        dist.init_process_group("nccl" if cuda else "gloo", timeout=datetime.timedelta(seconds=600))
        _pg = dist
    return rank, world, local


def dist_barrier(world):
    if world > 1 and _pg is not None:
        _pg.barrier()


def dist_max(x, world):
    """Max of x over the ranks (the job's time is its slowest rank's)."""
    if world > 1 and _pg is not None:
        import torch
        dev = "cuda" if _pg.get_backend() == "nccl" else "cpu"
        t = torch.tensor([float(x)], device=dev)
        _pg.all_reduce(t, op=_pg.ReduceOp.MAX)
        return float(t.item())
    return float(x)


def dist_close(world):
    if world > 1 and _pg is not None:
        _pg.barrier()
        _pg.destroy_process_group()


def min_intermolecular_distance(s, atoms_per_molecule):
    """Smallest distance (minimum image) between atoms of different molecules
    of a one-species box whose molecules are consecutive atom blocks."""
    from scipy.spatial import cKDTree
    L = float(s.box[0])
    x = np.mod(np.asarray(s.atmcor, float).reshape(-1, 3), L)
    mol = np.arange(len(x)) // atoms_per_molecule
    pairs = cKDTree(x, boxsize=L).query_pairs(2.5, output_type="ndarray")
    pairs = pairs[mol[pairs[:, 0]] != mol[pairs[:, 1]]]
    if len(pairs) == 0:
        return 2.5
    d = (x[pairs[:, 0]] - x[pairs[:, 1]] + 0.5 * L) % L - 0.5 * L
    return float(np.sqrt((d * d).sum(axis=1)).min())


def serve_replica(rng, k, precision):
    """One replica of the serving workload: a water or propanol box of 1.5k-30k
    atoms (log-uniform), rc <= 10 A, SPME at ~1 A grid spacing.  A propanol
    box whose random orientations put atoms of two molecules closer than
    1.5 A is drawn again with the next seed: such a hot start (one of the
    first 32 seeds) heats the box until it fails within a few hundred steps
    in either precision."""
    from thrid_b200 import systems as S
    natom = float(np.exp(rng.uniform(np.log(1500.0), np.log(30000.0))))
    if rng.random() < 0.5:
        nside = max(6, int(round((natom / 3.0) ** (1.0 / 3.0))))
        s = S.small_box("water", nside=nside, spacing=3.1, precision=precision, seed=100 + k,
                        nfft=_nfft(nside * 3.1), order=4, rcut=min(10.0, nside * 3.1 / 2.0 - 2.2))
    else:
        nside = max(3, int(round((natom / 12.0) ** (1.0 / 3.0))))
        for t in range(16):
            s = S.small_box("propanol", nside=nside, spacing=5.2, precision=precision, seed=100 + k + 10000 * t,
                            nfft=_nfft(nside * 5.2), order=4, rcut=min(10.0, nside * 5.2 / 2.0 - 2.2))
            if min_intermolecular_distance(s, 12) >= 1.5:
                break
    return s


def _nfft(L):
    for k in (16, 20, 24, 32, 40, 48, 64, 80, 96, 128):
        if k >= L:
            return k
    return 128


def run_serve(args, single=None):
    """Continuous batching of independent replicas (the serving configuration):
    Poisson arrivals, admission by slots and memory, per-replica latency.
    `single`: the single large system's rate measured in the same run (else
    measured here)."""
    import torch
    from thrid_b200 import abi
    from thrid_b200 import systems as S
    from thrid_b200.pgk import tuning_table
    from thrid_b200.serve import ReplicaServer
    torch.cuda.set_device(0)
    rng = np.random.default_rng(args.serve_seed)
    reps = [serve_replica(rng, k, abi.PREC_MIXED) for k in range(args.serve_replicas)]
    md = abi.md_struct(S.fs_to_reduced(1.0), ifrattle=1, outinterval=0)
    work = sum(s.natom for s in reps) * args.serve_steps
    # --serve-hf: the heat flux of the whole box every step, streamed back as
    # J_z(t) records for Green-Kubo (one region spanning the box, no thermostat)
    kind = 3 if args.serve_hf else 0
    hfs = [dict(regions=[(0.0, float(s.box[2]))], heatfinterval=1) if args.serve_hf else None for s in reps]

    def run(slots, arrivals):
        srv = ReplicaServer(max_slots=slots)
        t0 = time.perf_counter()
        ids = []
        for s, h, ta in zip(reps, hfs, arrivals):
            dt = ta - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            ids.append(srv.submit(s, md, kind=kind, nsteps=args.serve_steps, hf=h))
        res = [srv.result(i) for i in ids]
        if args.serve_hf:
            assert all(r[4].shape[0] == args.serve_steps and np.isfinite(r[4]).all() for r in res)
        srv.close()
        t = np.array([r[5] for r in res])
        lat = t[:, 2] - t[:, 0]
        span = t[:, 2].max() - t[:, 0].min()
        return lat, span

    # warm-up (library load, first context)
    srv = ReplicaServer(max_slots=1)
    srv.result(srv.submit(reps[0], md, kind=kind, nsteps=5, hf=hfs[0]))
    srv.close()
    seq_lat, seq_span = run(1, [0.0] * len(reps))               # one at a time, all queued at t=0
    mean_service = seq_span / len(reps)
    gaps = rng.exponential(mean_service / args.serve_load * 1.0, size=len(reps))
    arrivals = np.cumsum(gaps) - gaps[0]
    lat, span = run(args.serve_slots, arrivals)
    if single is None:
        single = single_system_rate()
    return {
        "metric": "replica serving: aggregate atom-steps/s and p50/p99 latency (mixed precision)",
        "value": work / span, "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
        "config": {"workload": "poisson_replicas_water_or_propanol_1.5k-30k_nve" + ("_jz_every_step" if args.serve_hf
                                                                                        else ""), "replicas": len(reps),
                   "steps_per_replica": args.serve_steps, "slots": args.serve_slots,
                   "offered_load": args.serve_load, "natom_total": int(sum(s.natom for s in reps))},
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "max": float(lat.max())},
        "one_at_a_time": {"value": work / seq_span, "unit": UNIT,
                          "latency_p50_s": float(np.percentile(seq_lat, 50)),
                          "latency_p99_s": float(np.percentile(seq_lat, 99))},
        "single_large_system": single,
        "fraction_of_single_large_system": (work / span) / single["value"],
        "autotune": tuning_table().splitlines(),
        "data": "synthetic (seeded lattices)",
    }


def single_system_rate(nsteps=100):
    """atom-steps/s of the 200k-atom butane NPT system alone (the single large
    system the serving target is quoted against), one list period after a
    warm-up, CUDA-event timed."""
    import torch
    from thrid_b200 import abi
    from thrid_b200.pgk import PgkEngine
    s = make_system(abi.PREC_MIXED)
    md = md_params(s)
    eng = PgkEngine(s)
    eng.set_chain(abi.chain_init(s.box))
    st = torch.cuda.ExternalStream(eng.stream)
    s0, n = period_window(5, nsteps, NSTEP_BOOK)
    eng.moldyn_mtk(0, s0 - 1, md)
    ms = _timed_md(eng, "mtk", s0, n, md, st)
    eng.close()
    return {"value": s.natom * n / (ms / 1e3), "unit": UNIT, "steps": n, "workload": WORKLOAD}


EWK_WORKLOAD = "water_12288_box49.66_alpha0.32_ewaldkp_hf"
EWK_FLOPS = {"k_ewk_sfac": 16, "k_ewk_atom": 34}   # FP64 flops per (atom, wave)
EWK_FLOPS_PER_PAIR = sum(EWK_FLOPS.values())
FP64_NOMINAL_TFLOPS = 37.0   # B200 (HGX) datasheet FP64; no FP64 peak is measured on this pool


def run_ewk(args):
    """ewaldkp_hf (per-atom standard-Ewald k-space term of the bulk heat flux)
    on 4,096 rigid waters (12,288 atoms, 49.66 A cube, alpha 0.32) at
    kmax = --ewk-hf: device time of the whole kernel chain per evaluation;
    the same end to end through the C ABI (positions up from host memory,
    force, per-atom energy and tensor down); the oracle on one host core at a
    smaller kmax, per (atom, wave) pair."""
    import ctypes as C
    from oracle import oracle as orc
    from thrid_b200 import abi
    from thrid_b200 import systems as S
    from thrid_b200.pgk import PgkEngine
    kmax = args.ewk_hf
    s = S.water_box(nside=16, box=49.66)
    eng = PgkEngine(s, dict(s.params, precision=abi.PREC_FP64))
    ms, units = C.c_double(0.0), C.c_double(0.0)
    launches0 = eng.kernel_launches
    r = eng.ewaldkp_hf(kmax)
    launches = eng.kernel_launches - launches0       # kernels of one evaluation
    with ClockSampler(0) as clk:
        st = eng.L.pgk_bench_kernel(eng.h, 256 + kmax, args.steps, C.byref(ms), C.byref(units), None)
    if st:
        raise RuntimeError(f"pgk_bench_kernel status {st}: {eng.L.pgk_last_error(eng.h)}")
    pairs = units.value
    kern = {}
    for name, base in (("k_ewk_sfac", 512), ("k_ewk_atom", 768)):
        km = C.c_double(0.0)
        st = eng.L.pgk_bench_kernel(eng.h, base + kmax, args.steps, C.byref(km), None, None)
        if st:
            raise RuntimeError(f"pgk_bench_kernel status {st}: {eng.L.pgk_last_error(eng.h)}")
        kern[name] = {"ms": km.value, "share": km.value / ms.value,
                      "fp64_tflops": EWK_FLOPS[name] * pairs / (km.value * 1e-3) * 1e-12}
    top = max(kern, key=lambda k: kern[k]["ms"])
    for _ in range(args.warmup):
        eng.upload_state(s.atmcor)
        r = eng.ewaldkp_hf(kmax)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.upload_state(s.atmcor)
        r = eng.ewaldkp_hf(kmax)
    e2e = (time.perf_counter() - t0) / args.steps
    n = s.natom
    kc = max(2, kmax // 2)
    o = orc.Oracle(s)
    t0 = time.perf_counter()
    rc = o.ewaldkp_hf(kc)
    tc = time.perf_counter() - t0
    dev = ms.value * 1e-3
    return {
        "metric": "ewaldkp_hf (atom, wave) pairs/s", "value": pairs / dev, "unit": "pairs/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms.value, "higher_is_better": True,
        "dtype": "f64", "data": "synthetic (seeded water lattice)",
        "config": {"workload": EWK_WORKLOAD, "natom": n, "kmax": kmax, "nwave": r["nwave"],
                   "l2": "working set (tables 12 MB) inside L2; device timing back to back"},
        "fp64_tflops": EWK_FLOPS_PER_PAIR * pairs / dev * 1e-12,
        "kernels": kern,
        "roofline": {"bound": "fp64", "kernel": top, "achieved": kern[top]["fp64_tflops"],
                     "peak": FP64_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                     "frac": kern[top]["fp64_tflops"] / FP64_NOMINAL_TFLOPS, "peak_kind": "nominal (datasheet)",
                     "traffic": None},
        "e2e": {"value": pairs / e2e, "unit": "pairs/s", "h2d_bytes_per_step": 24 * n,
                "d2h_bytes_per_step": 8 * 13 * n + 8 * 11},
        "cpu_baseline": {"value": n * (rc["nwave"] - 1) / tc, "unit": "pairs/s", "cores": 1, "kind": "port",
                         "sample": f"one oracle evaluation of the same system at kmax {kc} ({rc['nwave']} waves)"},
        "gpu_launches": launches, "clocks": clk.summary(),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the host-core baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64-path comparison leg")
    ap.add_argument("--no-configs", action="store_true", help="skip the other named shapes (C1-C3, drift)")
    ap.add_argument("--no-serve", action="store_true", help="skip the bounded serving leg of the main line")
    ap.add_argument("--serve", action="store_true", help="replica-serving benchmark instead of the main line")
    ap.add_argument("--serve-replicas", type=int, default=32)
    ap.add_argument("--serve-steps", type=int, default=2000)
    ap.add_argument("--serve-slots", type=int, default=8)
    ap.add_argument("--serve-load", type=float, default=4.0, help="arrival rate / one-at-a-time service rate")
    ap.add_argument("--serve-seed", type=int, default=2025)
    ap.add_argument("--serve-hf", action="store_true", help="replicas stream the box heat flux J_z(t) every step")
    ap.add_argument("--ewk-hf", type=int, default=0, metavar="KMAX",
                    help="ewaldkp_hf benchmark at this kmax instead of the main line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.ewk_hf:
        print(json.dumps(run_ewk(args)))
        return
    if args.serve:
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")   # before CUDA starts (see thrid_b200/serve.py)
        print(json.dumps(run_serve(args)))
        return
    if args.impl == "ours" and not args.no_serve:
        # the serving leg runs after the main line in the same process: give
        # its replicas' streams their own hardware queues before CUDA starts
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    rank, world, local = dist_init()
    if args.impl == "reference":
        out = run_reference(args, rank, world)
    else:
        out = run_ours(args, rank, world, local)
    if rank == 0 and out is not None:
        print(json.dumps(out))
    dist_close(world)


if __name__ == "__main__":
    main()
