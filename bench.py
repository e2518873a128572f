"""Benchmark of the IP-Glasma hot path on B200.

Headline workload (one step = one whole batch): 64 O+O events at 256^2
(L = 20 fm) and 16 Pb+Pb events at 512^2 (L = 40 fm), impact parameters
uniform in [0, 2R], Ny = 50, tau up to 0.4 fm (52 leapfrog steps for both
sizes). Per step every event draws fresh colour-charge noise (device Philox,
a new key per event and step), then colour charges -> Poisson solve -> Wilson
lines -> tau = 0 Newton links for all events side by side, one persistent
leapfrog launch per step over all 80 lattices (a replayed CUDA graph, tile
shape from the autotuner), then T^{mu nu} + Landau matching + eccentricities
of every event. The g^2 mu^2 maps (seeded Woods-Saxon nuclei) stay resident.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Reported (one JSON line, rank 0):
  value        events/s of the batched FP32-bulk form (whole job, all ranks)
  fp64         the same batch in the plain FP64 form
  error        FP32 bulk vs FP64 on every event of the batch
  e2e          the batch through the C ABI with host buffers: g^2 mu^2 maps in
               and e, u, pi, T^{mu nu} of every event out, every step
  roofline     the batched leapfrog kernel against measured HBM
  large        8 Pb+Pb at 1024^2, Ny 100, tau 1.0 fm, dtau 0.05 a: FP32 and
               FP64 batches, per-kernel GB/s, error
  single_event one 512^2 Pb+Pb event (tau 0.6 fm) per form: the tile kernels
  adjoint      gradient of E_T + eps2 for a 256^2 Au+Au event, 400 steps
  multiplicity Coulomb gauge fixing and the gluon spectrum of a 512^2 Pb+Pb
               event after its first step (the computeGluonMultiplicity
               schedule's it = 1 call)
  cpu_baseline the reference (oracle/_ref, OpenMP, all host cores) on one event
               of each size class of the same workload, combined in the
               batch's proportions
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# One 512^2 Pb+Pb event (the single-event form: TMA tile kernels)
WORKLOAD = dict(name="PbPb_512", N=512, L=40.0, nucleus="Pb", b=6.0, Ny=50,
                maxtime=0.6, g=2.0, m=0.2)
# Batched workloads: event classes (nucleus, N, L, count, impact parameter
# range) evolved together on one time grid (same lattice spacing and dtau)
HEADLINE = dict(name="OO256x64_PbPb512x16", Ny=50, maxtime=0.4, dtau=0.0, g=2.0, m=0.2,
                classes=[dict(nucleus="O", N=256, L=20.0, count=64, bmax=2 * 2.61),
                         dict(nucleus="Pb", N=512, L=40.0, count=16, bmax=2 * 6.62)])
LARGE = dict(name="PbPb1024x8", Ny=100, maxtime=1.0, dtau=0.05, g=2.0, m=0.2,
             classes=[dict(nucleus="Pb", N=1024, L=40.0, count=8, bmax=14.0)])
METRIC = "site-updates/s & events/s: FP32-batched vs plain FP64 at stated err; adjoint/fwd"
# algorithmic bytes per site-update of the fused leapfrog: every state word read
# once and written once (links 2 x 18, E 2 x 8, phi 9, pi 9 = 70 reals)
# Algorithmic bytes of one site advanced one full step (each state word read
# once and written once):
#   FP32 bulk form: the compact count, two links of 18 reals and four su(3)
#     fields of 8 reals, 2 x 68 x 4 B = 544 B;
#   FP64 plain form: the reference's layout, six full 3x3 complex matrices
#     (Ux, Uy, E1, E2, phi, pi), 2 x 108 x 8 B = 1728 B.
# The kernels store 70 reals per site (E traceless in 8 reals, phi and pi
# Hermitian in 9), so they move 560 B (FP32) and 1120 B (FP64) per update;
# both figures are reported beside the roofline.
BYTES_PER_SITE_UPDATE = {"fp32": 2 * 68 * 4, "fp64": 2 * 108 * 8}
BYTES_STORED_PER_SITE_UPDATE = {"fp32": 2 * 70 * 4, "fp64": 2 * 70 * 8}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self._proc = None
        self._t = None

    def _read(self):
        # one streaming nvidia-smi (a line every 50 ms) for the whole region
        for line in self._proc.stdout:
            parts = [p.strip() for p in line.strip().split(",")]
            if len(parts) == 7:
                self.samples.append(parts)

    def __enter__(self):
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            time.sleep(0.1)  # the first line before the timed work starts
        except Exception:
            self._proc = None
        return self

    def __exit__(self, *exc):
        if self._proc is not None:
            time.sleep(0.06)  # one more line after the timed work
            self._proc.terminate()  # this process only, by its handle
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
            if self._t:
                self._t.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4)
                          if s[3 + k].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# ranks: events shard across ranks (no data-path collective); each rank draws
# its own events, the timed region ends with a barrier on every rank and the
# whole-job figure uses the slowest rank's time
# ---------------------------------------------------------------------------
def rank_seed_base(rank: int) -> int:
    """Seeds of rank r's events start at 1000 (r + 1): disjoint event sets for
    up to 1000 events per rank."""
    return 1000 * (rank + 1)


def max_over_ranks(dist, values, device):
    """Element-wise max of per-rank timings (identity without a process group)."""
    if not dist:
        return list(values)
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def whole_job_rate(world: int, per_rank: int, ms_max: float) -> float:
    """Events per second of the whole job: all ranks' events over the slowest
    rank's time."""
    return world * per_rank / (ms_max * 1e-3)


def make_inputs():
    from ipglasma_b200.synthetic import make_event
    w = WORKLOAD
    A, B, _, _ = make_event(w["N"], w["L"], w["nucleus"], w["b"], seed=11, g=w["g"])
    return A, B


def newton_kw(precision: int) -> dict:
    """tau = 0 Newton solve per form: the FP32 bulk form uses Newton on the
    group (exact Jacobian, the reference's criterion sum |F_a| < 1e-6), the
    plain FP64 form the reference's own iteration (numeric Jacobian), bit
    for bit."""
    return {"newton_mode": 1} if precision == 1 else {}


NEWTON_NOTE = {"fp32": "Newton on the group, exact Jacobian, to sum|F_a| < 1e-6",
               "fp64": "the reference's iteration (numeric Jacobian, 1e-6), bit for bit"}


def cfg_for(precision: int, seed: int):
    import ipglasma_b200 as ipg
    w = WORKLOAD
    return ipg.Config(size=w["N"], L=w["L"], Ny=w["Ny"], g=w["g"], m=w["m"],
                      maxtime=w["maxtime"], precision=precision, seed=seed,
                      **newton_kw(precision))


def flush_l2(torch, buf):
    buf.fill_(1.0)  # 256 MB > 126 MB L2


def run_events(torch, ev, d_A, d_B, K, seed0, l2buf, host=None):
    """K events on one context; returns (device ms per event list, leapfrog ms)."""
    import ctypes as ct
    lib = ev._lib
    times, lf = [], []
    for k in range(K):
        flush_l2(torch, l2buf)
        torch.cuda.synchronize()
        st = torch.cuda.Event(enable_timing=True)
        en = torch.cuda.Event(enable_timing=True)
        st.record()
        ev_reset(ev, seed0 + k)
        ev.set_g2mu_device(d_A.data_ptr(), d_B.data_ptr())
        ev.use_device_noise()
        ev.init_fields(allow_nonconverged=True)
        ev.run()
        en.record()
        torch.cuda.synchronize()
        times.append(st.elapsed_time(en))
        lf.append(ev.last_leapfrog_ms()[0])
    return times, lf


def ev_reset(ev, seed):
    """Re-key the device noise of an existing context (no reallocation)."""
    ev.reseed(seed)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-large", action="store_true",
                    help="skip the 8 x 1024^2 Pb+Pb production batch")
    ap.add_argument("--no-single", action="store_true",
                    help="skip the single 512^2 event (tile kernels) measurement")
    ap.add_argument("--no-multiplicity", action="store_true",
                    help="skip the gauge-fixing and gluon-spectrum leg")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint (forward/backward) measurement")
    ap.add_argument("--profile", choices=["fp32", "fp64", "both", "adjoint", "batch32",
                                          "batch64", "gaugefix"], default=None,
                    help="run one warm-up and one timed event per form and exit "
                         "(the command profiled under ncu)")
    ap.add_argument("--profile-n", type=int, default=512,
                    help="lattice size of the profiled events (L = 40 fm)")
    args = ap.parse_args()
    world, rank, local = dist_env()
    if args.profile:
        if args.profile_n != WORKLOAD["N"]:
            WORKLOAD["N"] = args.profile_n
        return run_profile(args.profile, local)
    if args.impl == "reference":
        return run_reference(args, world, rank)
    return run_ours(args, world, rank, local)


def run_profile(which, local):
    import torch
    import ipglasma_b200 as ipg

    torch.cuda.set_device(local)
    if which in ("batch32", "batch64"):
        # the headline batch (64 O+O 256^2 + 16 Pb+Pb 512^2) on the TMA tile
        # variant, no tuner: initial conditions, then two batched runs
        prec = ipg.FP32 if which == "batch32" else ipg.FP64
        w = HEADLINE
        specs = job_events(w, 1)
        evs, _, b = build_batch(ipg, w, specs, prec, 900)
        b.set_shape(3 if prec == ipg.FP32 else 2, 1)
        for k in range(2):
            batch_step(evs, b, 900 + 1000 * k)
        print(f"batch {which}: evolution ms {b.stats()[0]:.2f}")
        b.close()
        for ev in evs:
            ev.close()
        return
    if which == "gaugefix":
        # Coulomb gauge fixing of a Pb+Pb 512^2 event (L 40 fm, Ny 10) after 20
        # leapfrog steps, then the gluon spectrum
        from ipglasma_b200.synthetic import make_event
        A, B, _, _ = make_event(512, 40.0, "Pb", 6.0, seed=5)
        with ipg.Event(ipg.Config(size=512, L=40.0, Ny=10, maxtime=1.0, seed=4)) as ev:
            ev.set_g2mu(A, B)
            ev.use_device_noise()
            ev.init_fields()
            ev.evolve(20)
            rep = ev.gauge_fix(4000)
            m = ev.multiplicity()
        print(f"gauge fixing: {rep['iterations']} iterations in {rep['ms']:.3f} ms, "
              f"dN/dy {m['dNdy']:.6g}")
        return
    if which == "adjoint":
        # the adjoint workload's event (Au+Au 256^2, Ny 50) over 40 steps, every
        # state kept (1.5 GB): one forward and one backward
        from ipglasma_b200.synthetic import make_event
        w = ADJ
        a = w["L"] / w["N"]
        A, B, _, _ = make_event(w["N"], w["L"], w["nucleus"], w["b"], 8000)
        ev = ipg.Event(ipg.Config(size=w["N"], L=w["L"], Ny=w["Ny"], maxtime=40 * w["dtau"] * a,
                                  dtau=w["dtau"], precision=ipg.FP64, seed=8100,
                                  newton_tolerance=1e-12))
        ev.set_g2mu(A, B)
        ev.use_device_noise()
        ev.init_fields(allow_nonconverged=True)
        et, e2 = ev.forward(1)
        ev.backward(1.0, 1.0, inputs=True)
        f, b = ev.adjoint_stats()
        print(f"adjoint steps={ev.itmax} E_T={et} forward_ms={f} backward_ms={b}")
        ev.close()
        return
    A, B = make_inputs()
    d_A = torch.tensor(A, dtype=torch.float64, device="cuda")
    d_B = torch.tensor(B, dtype=torch.float64, device="cuda")
    l2buf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    forms = {"fp32": [ipg.FP32], "fp64": [ipg.FP64], "both": [ipg.FP32, ipg.FP64]}[which]
    for prec in forms:
        ev = ipg.Event(cfg_for(prec, 77))
        t, lf = run_events(torch, ev, d_A, d_B, 2, 77, l2buf)
        print(f"precision={prec} event_ms={t} leapfrog_ms={lf}")
        ev.close()


# ---------------------------------------------------------------------------
# batched workloads: the whole job's events, LPT-sharded over the ranks
# ---------------------------------------------------------------------------
def steps_of(w: dict, cls: dict) -> int:
    """Leapfrog steps of an event class (the reference's itmax rule,
    Evolution.cpp:396, with dtau derived as main.cpp:531-534 unless set)."""
    a = cls["L"] / cls["N"]
    if w.get("dtau", 0) > 0:
        dtau = w["dtau"]
    else:
        dtau = w["maxtime"] / ((int(10 * w["maxtime"] / a) + 1) * a)
    return int(w["maxtime"] / (a * dtau) + 0.1)


def job_events(w: dict, world: int) -> list[dict]:
    """Every event of the whole job: `world` copies of the workload's class
    mix (per-GPU work fixed: weak scaling), each event with its own seed and
    impact parameter, and its cost N^2 x steps."""
    rng = np.random.default_rng(20260 + len(w["name"]))
    out = []
    for r in range(world):
        for ci, cls in enumerate(w["classes"]):
            for k in range(cls["count"]):
                out.append(dict(nucleus=cls["nucleus"], N=cls["N"], L=cls["L"],
                                b=float(rng.uniform(0.0, cls["bmax"])),
                                seed=7000 + 1000 * r + 100 * ci + k, cls=ci,
                                cost=cls["N"] ** 2 * steps_of(w, cls)))
    return out


def lpt_assign(costs: list[float], world: int) -> list[list[int]]:
    """Longest-processing-time-first: events in decreasing cost (ties by
    index) each go to the rank with the least cost assigned so far (ties to
    the lowest rank). Returns every rank's event indices, ascending."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(x) for x in out]


def build_batch(ipg, w: dict, specs: list[dict], precision: int, seed_base: int):
    """Contexts of the given events (g2mu maps set from the host once) and
    their batch."""
    from ipglasma_b200.synthetic import make_event
    evs, maps = [], []
    for k, e in enumerate(specs):
        A, B, _, _ = make_event(e["N"], e["L"], e["nucleus"], e["b"], e["seed"], g=w["g"])
        ev = ipg.Event(ipg.Config(size=e["N"], L=e["L"], Ny=w["Ny"], g=w["g"], m=w["m"],
                                  maxtime=w["maxtime"], dtau=w.get("dtau", 0.0),
                                  precision=precision, seed=seed_base + k,
                                  **newton_kw(precision)))
        ev.set_g2mu(A, B)
        ev.use_device_noise()
        evs.append(ev)
        maps.append((A, B))
    return evs, maps, ipg.Batch(evs)


def batch_step(evs, batch, key0: int):
    """One step of a batched workload: new noise keys, the initial conditions
    of every event, the batched evolution and every event's observables."""
    for k, ev in enumerate(evs):
        ev.reseed(key0 + k)
        ev.use_device_noise()
    batch.init_fields(allow_nonconverged=True)
    return batch.run()


def timed_batch_steps(torch, evs, batch, K: int, key0: int):
    """K batch steps: the device ms of each (CUDA events on torch's stream
    around library calls that wait for their own streams) and the batch's
    evolution ms of each (CUDA events around the replayed step graph)."""
    times, evo = [], []
    for k in range(K):
        torch.cuda.synchronize()
        st = torch.cuda.Event(enable_timing=True)
        en = torch.cuda.Event(enable_timing=True)
        st.record()
        batch_step(evs, batch, key0 + 1000 * k)
        en.record()
        torch.cuda.synchronize()
        times.append(st.elapsed_time(en))
        evo.append(batch.stats()[0])
    return times, evo


def launches_of(evs, batch) -> int:
    return sum(ev.kernel_launches() for ev in evs) + batch.stats()[2]


def cell_errors(eps32, eps64) -> dict:
    """Relative error of e per cell over the cells above 1% and 0.1% of the
    maximum: max and rms, and for 0.1% also the 99.9th percentile and the
    number of cells off by more than 10%. The Landau matching is not
    continuous: a cell whose time-like eigenvector is not found takes a
    neighbour's values (MyEigen.cpp:137-216), so a single cell near that
    branch can differ by O(1) between two forms and set the max alone."""
    out = {}
    for frac in (1e-2, 1e-3):
        m = eps64 > frac * eps64.max()
        rel = np.abs(eps32[m] - eps64[m]) / np.abs(eps64[m])
        out[f"e_rel_max_gt{frac:g}max"] = float(rel.max())
        out[f"e_rel_rms_gt{frac:g}max"] = float(np.sqrt(np.mean(rel ** 2)))
        if frac == 1e-3:
            out["e_rel_p999_gt0.001max"] = float(np.percentile(rel, 99.9))
            out["cells_rel_gt0.1_gt0.001max"] = int((rel > 0.1).sum())
    return out


def batch_errors(evs32, evs64, specs, r32, r64) -> dict:
    """FP32 bulk against FP64 on every event of a batch (same noise keys, so
    the same FP64 initial conditions): per size class the median and the
    worst event of each figure (e per cell over cells above 1% / 0.1% of the
    event's max e, eps_2 and E_T relative), and the worst Gauss violation
    and unitarity of each form."""
    per = []
    for e32, e64, spec, a, b in zip(evs32, evs64, specs, r32, r64):
        eps32, eps64 = e32.observables()[0], e64.observables()[0]
        row = {"cls": f"{spec['nucleus']}{spec['N']}", "b": spec["b"]}
        row.update(cell_errors(eps32, eps64))
        row["eps2_rel"] = abs(a.eccentricity[1] - b.eccentricity[1]) / abs(b.eccentricity[1])
        row["eps2_abs"] = abs(a.eccentricity[1] - b.eccentricity[1])
        row["E_T_rel"] = abs(a.E_T - b.E_T) / abs(b.E_T)
        row["gauss_fp32"], row["gauss_fp64"] = a.gauss_violation, b.gauss_violation
        row["unitarity_fp32"], row["unitarity_fp64"] = a.unitarity_max, b.unitarity_max
        per.append(row)
    keys = ["e_rel_rms_gt0.01max", "e_rel_max_gt0.01max", "e_rel_rms_gt0.001max",
            "e_rel_max_gt0.001max", "e_rel_p999_gt0.001max", "cells_rel_gt0.1_gt0.001max",
            "eps2_rel", "eps2_abs", "E_T_rel"]
    out = {}
    for cls in sorted({r["cls"] for r in per}):
        rows = [r for r in per if r["cls"] == cls]
        out[cls] = {"events": len(rows),
                    "median": {k: float(np.median([r[k] for r in rows])) for k in keys},
                    "worst": {k: float(max(r[k] for r in rows)) for k in keys},
                    "b_of_worst_eps2": float(max(rows, key=lambda r: r["eps2_rel"])["b"])}
    for k in ("gauss_fp32", "gauss_fp64", "unitarity_fp32", "unitarity_fp64"):
        out[k] = float(max(r[k] for r in per))
    out["events_compared"] = len(per)
    return out


def site_updates(w: dict, specs: list[dict]) -> int:
    return sum(e["N"] ** 2 * steps_of(w, w["classes"][e["cls"]]) for e in specs)


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def measure_workload(torch, ipg, w, specs, K, W, key0, dist, clocks=None, e2e_steps=0,
                     fp64_steps=None):
    """FP32 and FP64 batches of one rank's events: W warm-up and K timed
    steps of each, the error of FP32 against FP64 on every event, the
    initial-condition stage rates, and optionally the e2e figure. Times are
    maxed over ranks."""
    out = {}
    evs32, maps, b32 = build_batch(ipg, w, specs, ipg.FP32, key0)
    b32.init_fields(allow_nonconverged=True)
    out["tune"] = b32.tune()  # on freshly initialised events
    b32.run()
    for k in range(W):
        batch_step(evs32, b32, key0 + 100 + k)
    l0 = launches_of(evs32, b32)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with (clocks if clocks is not None else _Null()):
        t32, evo32 = timed_batch_steps(torch, evs32, b32, K, key0 + 10000)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
    out["launches"] = launches_of(evs32, b32) - l0
    e2e = None
    if e2e_steps:
        e2e = measure_batch_e2e(torch, evs32, maps, b32, e2e_steps, key0 + 50000, dist)
    r32 = batch_step(evs32, b32, key0 + 99999)  # the comparison's noise keys
    evs64, _, b64 = build_batch(ipg, w, specs, ipg.FP64, key0)
    b64.init_fields(allow_nonconverged=True)
    b64.tune()
    b64.run()
    for k in range(min(W, 2)):
        batch_step(evs64, b64, key0 + 100 + k)
    K64 = K if fp64_steps is None else fp64_steps
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t64, evo64 = timed_batch_steps(torch, evs64, b64, K64, key0 + 10000)
    if dist:
        dist.barrier()
    r64 = batch_step(evs64, b64, key0 + 99999)
    err = batch_errors(evs32, evs64, specs, r32, r64)
    # the FP64 form's stages, and the FP32 form's (FP32 Poisson transforms,
    # FP64 exponentials and products; Newton on the group)
    stages = {"fp64": stage_rates(w, specs, evs64, key0),
              "fp32": stage_rates(w, specs, evs32, key0)}
    b32.close()
    b64.close()
    for ev in evs32 + evs64:
        ev.close()
    ms32, ms64, mevo32, mevo64 = max_over_ranks(
        dist, [float(np.sum(t32)), float(np.sum(t64)), float(np.mean(evo32)),
               float(np.mean(evo64))], "cuda")
    out.update(ms32=ms32, ms64=ms64, K=K, K64=K64, evo32=mevo32, evo64=mevo64, err=err,
               e2e=e2e, stages=stages)
    return out


def measure_batch_e2e(torch, evs, maps, batch, K, key0, dist):
    """The batch through the C ABI with host buffers: every step copies each
    event's g2mu maps from page-locked host memory, runs the batch, and
    starts the copies of each event's e, u, pi and T^{mu nu} into one of two
    page-locked host sets (ipg_get_observables_async, the library's copy
    streams), as a pipeline would: step k's copies run while step k + 1's
    initial conditions and evolution are computed (its observables stage
    waits for them), and a caller reads set k mod 2 meanwhile. Wall clock
    around K steps, the last copies waited for inside it."""
    def pinned(shape):
        return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()

    host_in = []
    for A, B in maps:
        hA, hB = pinned(A.shape), pinned(B.shape)
        hA[...] = A
        hB[...] = B
        host_in.append((hA, hB))
    host_out = [[(pinned((ev.n,)), pinned((4, ev.n)), pinned((10, ev.n)), pinned((10, ev.n)))
                 for ev in evs] for _ in range(2)]

    def one(k):
        for ev, (hA, hB) in zip(evs, host_in):
            ev.set_g2mu(hA, hB)
        batch_step(evs, batch, key0 + 1000 * k)
        for ev, o in zip(evs, host_out[k % 2]):
            ev.observables_async(*o)
    one(0)
    for ev in evs:
        ev.wait_observables()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(K):
        one(k + 1)
    for ev in evs:
        ev.wait_observables()
    torch.cuda.synchronize()
    total = time.perf_counter() - t0
    h2d = sum(2 * ev.n * 8 for ev in evs)
    d2h = sum(25 * ev.n * 8 for ev in evs)
    return {"ms": total * 1e3, "h2d": h2d, "d2h": d2h}


def stage_rates(w, specs, evs, key0):
    """Device time of the initial-condition stages of one event per size
    class, run alone (ipg_init_report: CUDA events in the library), with
    their algorithmic bytes: the Wilson-line stage reads and writes V once
    per (site, sheet, nucleus), 2 x 18 x 8 = 288 B; Newton reads U1, U2 (36
    doubles) and writes U (18) per link, 432 B. The Wilson-line stage's FFT
    rate uses the conventional count, 2 x 8 x 5 N^2 log2(N^2) flops per
    (sheet, nucleus): eight colours, forward and inverse (the kernels pack
    two real colours into one complex transform, so they execute half)."""
    out = {}
    seen = set()
    for e, ev in zip(specs, evs):
        if e["cls"] in seen:
            continue
        seen.add(e["cls"])
        ev.reseed(key0 + 7)
        ev.use_device_noise()
        rep = ev.init_fields(allow_nonconverged=True)
        n = e["N"] ** 2
        wil = n * w["Ny"] * 2 * 288
        newt = 2 * n * 432
        fft = 2 * 8 * 5 * n * np.log2(n) * w["Ny"] * 2
        out[f"{e['nucleus']}{e['N']}"] = {
            "ms_wilson": round(rep.ms_wilson, 3),
            "wilson_GBs_at_288B": round(wil / (rep.ms_wilson * 1e-3) / 1e9, 1),
            "wilson_fft_TFLOPs_conventional": round(fft / (rep.ms_wilson * 1e-3) / 1e12, 2),
            "ms_newton": round(rep.ms_newton, 3),
            "newton_GBs_at_432B": round(newt / (rep.ms_newton * 1e-3) / 1e9, 1),
            "newton_mean_iterations": round(rep.newton_mean_iterations, 2),
            "ms_fields": round(rep.ms_fields, 3)}
    return out


def workload_config(w: dict, world: int) -> dict:
    return {"workload": w["name"],
            "events_per_step": sum(c["count"] for c in w["classes"]) * world,
            "classes": [{"nucleus": c["nucleus"], "N": c["N"], "L_fm": c["L"],
                         "count_per_gpu": c["count"], "b_max_fm": round(c["bmax"], 2),
                         "leapfrog_steps": steps_of(w, c)} for c in w["classes"]],
            "Ny": w["Ny"], "tau_fm": w["maxtime"],
            "dtau": (f"{w['dtau']} a" if w.get("dtau") else "derived (main.cpp:531-534)"),
            "l2": "no flush: a step's state (over 1 GB) is larger than the 126 MB L2",
            "parallelism": f"events LPT-sharded (cost N^2 x steps) over {world} GPU(s), "
                           "no collective",
            "newton": NEWTON_NOTE}


def run_ours(args, world, rank, local):
    import torch
    import ipglasma_b200 as ipg

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta
        dist_mod.init_process_group("nccl", timeout=timedelta(seconds=300))
        dist = dist_mod
    K, W = args.steps, max(3, args.warmup)
    peaks = load_peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)

    # --- headline: the batched uneven-events workload ------------------------
    w = HEADLINE
    allev = job_events(w, world)
    mine = [allev[i] for i in lpt_assign([e["cost"] for e in allev], world)[rank]]
    clk = ClockSampler(local)
    res = measure_workload(torch, ipg, w, mine, K, W, rank_seed_base(rank) * 100, dist,
                           clocks=clk, e2e_steps=K)
    n_ev = len(allev)
    su = site_updates(w, allev)
    ev32 = n_ev * K / (res["ms32"] * 1e-3)
    ev64 = n_ev * res["K64"] / (res["ms64"] * 1e-3)
    su32 = su / (res["evo32"] * 1e-3)
    su64 = su / (res["evo64"] * 1e-3)
    e2e = res["e2e"]
    e2e_ms = max_over_ranks(dist, [e2e["ms"]], "cuda")[0]
    achieved = su32 * BYTES_PER_SITE_UPDATE["fp32"] / 1e9
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
            "frac": round(achieved / hbm, 4), "traffic": load_traffic(),
            "kernel": "k_leapfrog_batch<float> (FP32 bulk: all events of the batch in one "
                      "persistent launch per step)",
            "bytes_per_site_update": BYTES_PER_SITE_UPDATE["fp32"],
            "bytes_stored_per_site_update": BYTES_STORED_PER_SITE_UPDATE["fp32"],
            "stored_frac": round(su32 * BYTES_STORED_PER_SITE_UPDATE["fp32"] / 1e9 / hbm, 4),
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
            "timing": "CUDA events on the batch's stream around the replayed step graph (all "
                      "leapfrog launches of the batch), mean over the timed steps",
            "fp64_kernel": {"kernel": "k_leapfrog_batch<double>",
                            "achieved": round(su64 * BYTES_PER_SITE_UPDATE["fp64"] / 1e9, 1),
                            "frac": round(su64 * BYTES_PER_SITE_UPDATE["fp64"] / 1e9 / hbm, 4),
                            "bytes_per_site_update": BYTES_PER_SITE_UPDATE["fp64"],
                            "stored_frac": round(su64 * BYTES_STORED_PER_SITE_UPDATE["fp64"]
                                                 / 1e9 / hbm, 4)}}
    tune = res["tune"]

    large = None if args.no_large else measure_large(torch, ipg, rank, world, dist, hbm)
    single = None if args.no_single else measure_single(torch, ipg, K, W, rank, world, dist,
                                                        hbm)
    adjoint = None if args.no_adjoint else measure_adjoint(torch, ipg, rank)
    mult = None if args.no_multiplicity else measure_multiplicity(ipg, rank, hbm)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample()

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": round(ev32, 3),
            "unit": "events/s",
            "n_gpus": world,
            "steps": K,
            "warmup": W,
            "ms_per_step": round(res["ms32"] / K, 3),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 (FP64 Newton, Wilson lines, observables, reductions)",
            "data": "synthetic (seeded Woods-Saxon nuclei, g2mu ~ sqrt(T_A), device Philox "
                    "noise)",
            "config": workload_config(w, world),
            "site_updates_per_s": round(su32, 1),
            "fp64": {"events_per_s": round(ev64, 3),
                     "ms_per_step": round(res["ms64"] / res["K64"], 3),
                     "site_updates_per_s": round(su64, 1), "steps": res["K64"]},
            "fp32_over_fp64_events": round(ev32 / ev64, 3),
            "fp32_over_fp64_site_updates": round(su32 / su64, 3),
            "error": res["err"],
            "evolution_ms_per_step": {"fp32": round(res["evo32"], 3),
                                      "fp64": round(res["evo64"], 3)},
            "initial_condition_stages": res["stages"],
            "e2e": {"value": round(n_ev * K / (e2e_ms * 1e-3), 3), "unit": "events/s",
                    "h2d_bytes_per_step": e2e["h2d"] * world,
                    "d2h_bytes_per_step": e2e["d2h"] * world, "form": "fp32",
                    "host_buffers": "pinned",
                    "copies": "every event's g2mu maps in and e, u, pi, T^munu out, every "
                              "step, inside the wall-clock region; a step's copies out run "
                              "while the next step computes (two host sets)"},
            "roofline": roof,
            "tuned_shape": {"tile_rows": tune.tile_rows, "threads": tune.threads_per_block,
                            "blocks_per_sm": tune.blocks_per_sm, "grid": tune.grid,
                            "candidates": tune.candidates},
            "large": large,
            "single_event": single,
            "adjoint": adjoint,
            "multiplicity": mult,
            "cpu_baseline": cpu,
            "gpu_launches": int(res["launches"]),
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# bytes a site moves in one gauge-fixing iteration: the links read for the
# divergence (2 x 144), the packed g through the FFT passes (64 written, then
# 3 passes of 64 read + 64 written), the exponential (64 read, 144 written),
# the transformation (G 144 read, the state's 70 reals read and written)
GAUGE_BYTES_PER_SITE_ITERATION = 288 + 64 + 3 * 128 + 64 + 144 + 144 + 2 * 560


def measure_multiplicity(ipg, rank, hbm):
    """Evolution::multiplicity on one Pb+Pb 512^2 event (L = 40 fm, Ny = 50,
    b = 6 fm) after its first step, as the computeGluonMultiplicity schedule
    runs it at it = 1: Coulomb gauge fixing (device time, iterations, and the
    HBM rate at GAUGE_BYTES_PER_SITE_ITERATION a site and iteration), then the
    spectrum."""
    if rank != 0:
        return None
    from ipglasma_b200.synthetic import make_event

    N, L = 512, 40.0
    A, B, _, _ = make_event(N, L, "Pb", 6.0, seed=606)
    out = {}
    with ipg.Event(ipg.Config(size=N, L=L, Ny=50, maxtime=0.6, seed=606)) as ev:
        for rep_ in range(2):  # the first pass warms up
            ev.set_g2mu(A, B)
            ev.use_device_noise()
            ev.init_fields()
            ev.evolve(1)
            m = ev.multiplicity()
        g = m["gauge"]
        per_it = g["ms"] / max(1, g["residual_checks"])
        gbs = N * N * GAUGE_BYTES_PER_SITE_ITERATION / (per_it * 1e-3) / 1e9
        out = {"workload": "Pb+Pb 512^2 (L 40 fm, Ny 50, b 6 fm), fields after the first step",
               "gauge_iterations": g["iterations"], "gauge_residual": g["residual"],
               "gauge_ms": round(g["ms"], 3), "us_per_iteration": round(1e3 * per_it, 2),
               "gauge_GBs": round(gbs, 1), "gauge_frac": round(gbs / hbm, 4),
               "bytes_per_site_iteration": GAUGE_BYTES_PER_SITE_ITERATION,
               "spectrum_ms": round(m["ms_spectrum"], 3), "dNdy": m["dNdy"],
               "dNdy_binned": m["dNdy_binned"], "mean_pt": m["mean_pt"],
               "timing": "device time (CUDA events) of the gauge fixing, its iterations "
                         "enqueued in chunks of 16 with one flag read per chunk; the "
                         "iterations after a stopping rule return at once"}
    return out


def measure_large(torch, ipg, rank, world, dist, hbm):
    """8 Pb+Pb events at 1024^2 (L = 40 fm, Ny = 100, b uniform in [0, 14] fm)
    to tau = 1.0 fm at dtau = 0.05 a (512 steps): the FP32 batch and the FP64
    batch, 2 timed steps each after one warm-up, the error of FP32 against
    FP64 on every event, and the per-kernel rates."""
    w = LARGE
    allev = job_events(w, world)
    mine = [allev[i] for i in lpt_assign([e["cost"] for e in allev], world)[rank]]
    res = measure_workload(torch, ipg, w, mine, 2, 1, rank_seed_base(rank) * 100 + 50000,
                           dist)
    n_ev = len(allev)
    su = site_updates(w, allev)
    su32 = su / (res["evo32"] * 1e-3)
    su64 = su / (res["evo64"] * 1e-3)
    g32 = su32 * BYTES_PER_SITE_UPDATE["fp32"] / 1e9
    g64 = su64 * BYTES_PER_SITE_UPDATE["fp64"] / 1e9
    adj = measure_large_adjoint(torch, ipg, w, mine[0])
    return {"config": workload_config(w, world),
            "adjoint_eps2": adj,
            "events_per_s": {"fp32": round(n_ev * 2 / (res["ms32"] * 1e-3), 3),
                             "fp64": round(n_ev * 2 / (res["ms64"] * 1e-3), 3)},
            "ms_per_step": {"fp32": round(res["ms32"] / 2, 1), "fp64": round(res["ms64"] / 2, 1)},
            "fp32_over_fp64_events": round(res["ms64"] / res["ms32"], 3),
            "leapfrog": {"fp32": {"kernel": "k_leapfrog_batch<float>",
                                  "ms_per_batch": round(res["evo32"], 2),
                                  "site_updates_per_s": round(su32, 1),
                                  "GBs_at_544B": round(g32, 1), "frac": round(g32 / hbm, 4)},
                         "fp64": {"kernel": "k_leapfrog_batch<double>",
                                  "ms_per_batch": round(res["evo64"], 2),
                                  "site_updates_per_s": round(su64, 1),
                                  "GBs_at_1728B": round(g64, 1), "frac": round(g64 / hbm, 4)}},
            "initial_condition_stages": res["stages"],
            "error": res["err"],
            "timing": "2 timed batch steps per form after 1 warm-up; CUDA events"}


def measure_large_adjoint(torch, ipg, w, spec):
    """The gradient of eps2 for one event of the large workload (1024^2,
    Ny 100, 512 steps) with the FP32 adjoint (an FP32 context) and the FP64
    adjoint, both with a checkpoint every 23 steps and time reversal between
    them; the same noise (device Philox, same key), Newton to 1e-12.
    Forward = initial conditions + evolution storing checkpoints + T^tautau;
    backward = reverse sweep + initial-condition adjoint (device times)."""
    from ipglasma_b200.synthetic import make_event
    A, B, _, _ = make_event(spec["N"], spec["L"], spec["nucleus"], spec["b"], spec["seed"],
                            g=w["g"])
    out, grads = {}, {}
    for name, prec in (("fp32", ipg.FP32), ("fp64", ipg.FP64)):
        ev = ipg.Event(ipg.Config(size=spec["N"], L=spec["L"], Ny=w["Ny"], g=w["g"], m=w["m"],
                                  maxtime=w["maxtime"], dtau=w["dtau"], precision=prec,
                                  seed=4242, newton_tolerance=1e-12))
        ev.set_g2mu(A, B)
        ev.use_device_noise()
        rep = ev.init_fields(allow_nonconverged=True)
        _, e2 = ev.forward(23)
        g = ev.backward(0.0, 1.0, inputs=True)
        f_ms, b_ms = ev.adjoint_stats()
        init_ms = rep.ms_wilson + rep.ms_newton + rep.ms_fields
        out[name] = {"eps2": e2, "device_ms_forward": round(init_ms + f_ms, 1),
                     "device_ms_backward": round(b_ms, 1),
                     "adjoint_over_forward": round(b_ms / (init_ms + f_ms), 3)}
        grads[name] = (np.array(g["g2mu"]), np.array(g[ipg.UX]))
        ev.close()
    # d/d(g^2 mu^2) goes through sqrt(g^2 mu^2) and grows without bound where
    # the map vanishes: compare on the cells above 1e-6 of the maximum
    support = np.stack([A, B]) > 1e-6 * max(A.max(), B.max())
    for k, key in enumerate(("grad_g2mu", "grad_Ux_tau0")):
        a, b = grads["fp32"][k], grads["fp64"][k]
        if k == 0:
            a, b = a.reshape(support.shape)[support], b.reshape(support.shape)[support]
        out[f"{key}_rel_diff_fp32_vs_fp64"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    out["workload"] = (f"one {spec['nucleus']}+{spec['nucleus']} {spec['N']}^2 event of the "
                       f"batch (b = {spec['b']:.2f} fm), Ny {w['Ny']}, {steps_of(w, w['classes'][0])} "
                       "steps, loss eps2, checkpoint every 23 steps")
    return out


def measure_single(torch, ipg, K, W, rank, world, dist, hbm):
    """One 512^2 Pb+Pb event per step (tau 0.6 fm, 77 steps) in each form:
    the single-event TMA tile kernels."""
    A, B = make_inputs()
    d_A = torch.tensor(A, dtype=torch.float64, device="cuda")
    d_B = torch.tensor(B, dtype=torch.float64, device="cuda")
    l2buf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    N = WORKLOAD["N"]
    Ks = min(K, 10)
    seed_base = rank_seed_base(rank)
    out = {}
    evs = {}
    for name, prec in (("fp32", ipg.FP32), ("fp64", ipg.FP64)):
        ev = ipg.Event(cfg_for(prec, seed_base))
        run_events(torch, ev, d_A, d_B, min(W, 3), seed_base, l2buf)
        if dist:
            dist.barrier()
        t, lf = run_events(torch, ev, d_A, d_B, Ks, seed_base + 100, l2buf)
        ms, mlf = max_over_ranks(dist, [float(np.sum(t)), float(np.mean(lf))], "cuda")
        su = N * N * ev.itmax / (mlf * 1e-3)
        g = su * BYTES_PER_SITE_UPDATE[name] / 1e9
        out[name] = {"events_per_s": round(world * Ks / (ms * 1e-3), 3),
                     "ms_per_event": round(ms / Ks, 3), "leapfrog_ms": round(mlf, 3),
                     "site_updates_per_s": round(su, 1),
                     "kernel": ("k_leapfrog_tile" if name == "fp32" else "k_leapfrog_tile64"),
                     "GBs": round(g, 1), "frac": round(g / hbm, 4),
                     "bytes_per_site_update": BYTES_PER_SITE_UPDATE[name],
                     "stored_frac": round(su * BYTES_STORED_PER_SITE_UPDATE[name] / 1e9 / hbm,
                                          4)}
        evs[name] = ev
    out["fp32_over_fp64_events"] = round(out["fp32"]["events_per_s"]
                                         / out["fp64"]["events_per_s"], 3)
    out["error"] = compare_forms(evs["fp32"], evs["fp64"], d_A, d_B, seed_base + 7)
    if rank == 0:
        ev = evs["fp32"]
        eps, u4, pi10, T10 = ev.observables()
        out["writers"] = measure_writers(ipg, ev, eps, u4, pi10, T10, ev.itmax, ev.dtau)
    out["workload"] = "Pb+Pb 512^2, L 40 fm, b 6 fm, Ny 50, tau 0.6 fm (77 steps)"
    out["l2"] = "flushed (256 MB write) before every event"
    for ev in evs.values():
        ev.close()
    return out


ADJ = dict(N=256, L=30.0, nucleus="Au", b=2.0, Ny=50, steps=400, dtau=0.1, checkpoint=20)
# checkpoint 1 keeps all 401 states (14.7 GB of HBM) and needs no time reversal


def measure_adjoint(torch, ipg, rank):
    """Adjoint of one Au+Au event at 256^2 (L = 30 fm, b = 2 fm, Ny = 50),
    400 leapfrog steps at dtau = 0.1 a, every state kept (the headline) and,
    reported beside it, a checkpoint every 20 steps with time reversal: the
    gradient of E_T + eps2 with respect to the g2mu maps (2 x 256^2) and rho
    (2 x 50 x 8 x 256^2). Forward = initial conditions (Newton to 1e-12) +
    ipg_forward; adjoint = ipg_backward through the evolution and the initial
    conditions."""
    from ipglasma_b200.synthetic import make_event
    w = ADJ
    a = w["L"] / w["N"]
    maxtime = w["steps"] * w["dtau"] * a
    A, B, _, _ = make_event(w["N"], w["L"], w["nucleus"], w["b"], 8000 + rank)
    ev = ipg.Event(ipg.Config(size=w["N"], L=w["L"], Ny=w["Ny"], maxtime=maxtime,
                              dtau=w["dtau"], precision=ipg.FP64, seed=8100 + rank,
                              newton_tolerance=1e-12))
    ev.set_g2mu(A, B)
    ev.use_device_noise()

    def timed(fn):
        torch.cuda.synchronize()
        st = torch.cuda.Event(enable_timing=True)
        en = torch.cuda.Event(enable_timing=True)
        st.record()
        out = fn()
        en.record()
        torch.cuda.synchronize()
        return out, st.elapsed_time(en)

    init_ms = [0.0]
    kcp = [1]
    # page-locked gradient buffers (torch's pinned allocator, seen as numpy)
    pin = lambda k: torch.empty(k, dtype=torch.float64, pin_memory=True).numpy()  # noqa: E731
    n = w["N"] * w["N"]
    outs = {"state": pin(6 * 18 * n), "g2mu": pin(2 * n), "rho": pin(16 * w["Ny"] * n)}

    def forward():
        rep = ev.init_fields(allow_nonconverged=True)
        init_ms[0] = rep.ms_wilson + rep.ms_newton + rep.ms_fields
        return ev.forward(kcp[0])

    ckpt = {}
    for k in (w["checkpoint"], 1):
        kcp[0] = k
        forward()
        ev.backward(1.0, 1.0, inputs=True, rho=True, out=outs)  # warm-up
        (et, e2), ms_f = timed(forward)
        g, ms_b = timed(lambda: ev.backward(1.0, 1.0, inputs=True, rho=True, out=outs))
        dev_f, dev_b = ev.adjoint_stats()
        dev_init = init_ms[0]
        if k != 1:
            ckpt = {"checkpoint_every": k, "device_ms_forward_evolution": round(dev_f, 2),
                    "device_ms_backward": round(dev_b, 2),
                    "adjoint_over_forward": round(dev_b / (dev_init + dev_f), 3),
                    "E_T": et, "eps2": e2,
                    "grad_rho_norm": float(np.linalg.norm(g["rho"]))}
    _, ms_plain = timed(lambda: (ev.init_fields(allow_nonconverged=True), ev.run()))
    steps = ev.itmax
    support = np.concatenate([A, B]) > 1e-6 * max(A.max(), B.max())
    ev.close()
    return {"workload": f"Au+Au 256^2, L 30 fm, Ny 50, {steps} steps, every state kept, FP64",
            "loss": "E_T + eps2 (T^tautau-weighted)", "E_T": et, "eps2": e2,
            "device_ms_forward_init": round(dev_init, 2),
            "device_ms_forward_evolution": round(dev_f, 2),
            "device_ms_backward": round(dev_b, 2),
            "adjoint_over_forward": round(dev_b / (dev_init + dev_f), 3),
            "adjoint_over_forward_evolution_only": round(dev_b / dev_f, 3),
            "e2e_ms_forward": round(ms_f, 2), "e2e_ms_backward": round(ms_b, 2),
            "e2e_adjoint_over_forward": round(ms_b / ms_f, 3),
            "ms_plain_event": round(ms_plain, 2),
            "grad_g2mu_norm_on_support": float(np.linalg.norm(g["g2mu"].ravel()[support])),
            "grad_rho_norm": float(np.linalg.norm(g["rho"])),
            "checkpointed": ckpt,
            "timing": "device: CUDA events inside the library; forward = initial conditions "
                      "(Wilson lines, Newton to 1e-12, fields) + evolution storing states + "
                      "T^tautau, backward = reverse sweep + initial-condition adjoint, so both "
                      "sides cover the same chain. e2e: CUDA events around the API calls, "
                      "backward including the copies of the state, g2mu and rho gradients "
                      "(476 MB) into page-locked host arrays"}


def compare_forms(ev32, ev64, d_A, d_B, seed):
    outs = {}
    for name, ev in (("fp32", ev32), ("fp64", ev64)):
        ev_reset(ev, seed)
        ev.set_g2mu_device(d_A.data_ptr(), d_B.data_ptr())
        ev.use_device_noise()
        ev.init_fields(allow_nonconverged=True)
        res = ev.run()
        eps = ev.observables()[0]
        outs[name] = (eps, res)
    e32, r32 = outs["fp32"]
    e64, r64 = outs["fp64"]
    out = cell_errors(e32, e64)
    out["eps2_rel"] = abs(r32.eccentricity[1] - r64.eccentricity[1]) / abs(r64.eccentricity[1])
    out["E_T_rel"] = abs(r32.E_T - r64.E_T) / abs(r64.E_T)
    out["gauss_fp32"] = r32.gauss_violation
    out["gauss_fp64"] = r64.gauss_violation
    out["unitarity_fp32"] = r32.unitarity_max
    out["unitarity_fp64"] = r64.unitarity_max
    return out


def measure_writers(ipg, ev, eps, u4, pi10, T10, itmax, dtau):
    """Output files, timed apart from the event rate: the reference's hydro
    and T^munu files of the last event (sizeOutput = N over the lattice, one
    eta slice) written into a scratch directory that is removed afterwards,
    by the host writers from its observables and by the GPU writer
    (ipg_write_outputs) from the device copy; the two must be byte-identical."""
    import ctypes as ct
    import shutil
    import tempfile
    N, L = WORKLOAD["N"], WORKLOAD["L"]
    lib = ipg.lib()
    D = ct.c_double
    V = lambda a: ct.c_void_p(a.ctypes.data)  # noqa: E731
    d = tempfile.mkdtemp(prefix="ipg_writers_")
    try:
        hydro, tmunu = os.path.join(d, "hydro.dat"), os.path.join(d, "tmunu.dat")
        t0 = time.perf_counter()
        st = lib.ipg_write_hydro(hydro.encode(), N, D(L), N, D(L), 1, D(0.0), itmax, D(dtau),
                                 V(eps), V(u4), V(pi10), D(1.0), None)
        t1 = time.perf_counter()
        st2 = lib.ipg_write_tmunu(tmunu.encode(), N, D(L), N, D(L), 1, D(0.0), itmax, D(dtau),
                                  V(T10), D(1.0))
        t2 = time.perf_counter()
        sizes = os.path.getsize(hydro) + os.path.getsize(tmunu)
        gh, gt = os.path.join(d, "hydro_gpu.dat"), os.path.join(d, "tmunu_gpu.dat")
        ev.write_outputs(gh, gt)  # warm-up: buffers, first launch
        gpu_ms = []
        for path_h, path_t in ((gh, None), (None, gt)):
            t3 = time.perf_counter()
            ev.write_outputs(path_h, path_t)
            gpu_ms.append((time.perf_counter() - t3) * 1e3)
        same = all(open(a, "rb").read() == open(b, "rb").read()
                   for a, b in ((hydro, gh), (tmunu, gt)))
    finally:
        shutil.rmtree(d, ignore_errors=True)
    threads = os.environ.get("IPG_WRITER_THREADS") or str(os.cpu_count())
    return {"ms_hydro": round((t1 - t0) * 1e3, 1), "ms_tmunu": round((t2 - t1) * 1e3, 1),
            "bytes": int(sizes), "threads": int(threads), "status": [int(st), int(st2)],
            "gpu_ms_hydro": round(gpu_ms[0], 1), "gpu_ms_tmunu": round(gpu_ms[1], 1),
            "gpu_files_identical": bool(same),
            "timing": "wall clock, once per bench run, file write included; not part of the "
                      "event rate. ms_*: host writers from host observables; gpu_ms_*: "
                      "ipg_write_outputs from the device observables"}


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            return {}
    return {}


def load_traffic():
    """DRAM bytes per launch of the batched FP32 leapfrog kernel on this
    workload from the committed ncu summary (profiles/leapfrog_batch_fp32.json),
    or None."""
    p = ROOT / "profiles" / "leapfrog_batch_fp32.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get("dram_bytes_per_launch")
        except Exception:
            return None
    return None


# ---------------------------------------------------------------------------
# CPU baseline and reference arm: the reference itself (oracle/_ref), built
# with the reference's own -Ofast flags (finite-math off, which the reference
# needs), OpenMP over all host cores, one event at a time as the reference's
# executable runs them
# ---------------------------------------------------------------------------
FFT_NOTE = ("shim FFT, not FFTW: the reference's FFTW calls run on this project's "
            "single-threaded radix-2 stand-in (FFTW is absent from the image)")


def reference_event(spec: dict, w: dict, threads: int) -> dict:
    """One event of a workload through the reference harness: seconds of the
    hot path (setV, tau = 0 solve, Evolution::run with T^munu and Landau
    matching, eccentricity) timed inside the harness, dumps off."""
    sys.path.insert(0, str(ROOT / "tests"))
    from refcase import HARNESS_OFAST, run_harness
    from ipglasma_b200.synthetic import make_event
    A, B, _, _ = make_event(spec["N"], spec["L"], spec["nucleus"], spec["b"], spec["seed"],
                            g=w["g"])
    with tempfile.TemporaryDirectory() as tmp:
        r = run_harness(Path(tmp) / "ref", A, B, spec["N"], spec["L"], w["Ny"], w["g"], w["m"],
                        spec["seed"], w["maxtime"], threads=threads, binary=HARNESS_OFAST,
                        dtau=w.get("dtau") or -1.0, dumps=False)
    phases = {k: round(r.meta[k], 3) for k in ("t_setV", "t_tau0", "t_evolution",
                                                "t_eccentricity")}
    return {"seconds": float(sum(phases.values())), "phases_s": phases,
            "itmax": r.meta["itmax"]}


def reference_available() -> str | None:
    sys.path.insert(0, str(ROOT / "tests"))
    from refcase import HARNESS_OFAST
    if not HARNESS_OFAST.exists():
        return "oracle/_ref/ipg_ref_harness_ofast is not built (reference sources absent)"
    return None


def cpu_baseline_sample(threads: int | None = None):
    """The reference on a bounded sample of the headline workload: the first
    event of each size class (one O+O 256^2 and one Pb+Pb 512^2 event, 52
    steps each), combined in the batch's proportions (64 : 16) into the
    batch's events/s."""
    why = reference_available()
    if why:
        return {"value": None, "unit": "events/s", "cores": 0, "kind": "reference",
                "sample": why}
    threads = threads or os.cpu_count() or 1
    w = HEADLINE
    evs = job_events(w, 1)
    per_class = {}
    for e in evs:
        if e["cls"] not in per_class:
            per_class[e["cls"]] = reference_event(e, w, threads)
    t_batch = sum(c["count"] * per_class[i]["seconds"] for i, c in enumerate(w["classes"]))
    n = sum(c["count"] for c in w["classes"])
    return {"value": round(n / t_batch, 6), "unit": "events/s", "cores": threads,
            "kind": "reference",
            "sample": "; ".join(f"one {c['nucleus']}+{c['nucleus']} {c['N']}^2 event in "
                                f"{per_class[i]['seconds']:.1f} s x {c['count']}"
                                for i, c in enumerate(w["classes"]))
                      + f" -> {t_batch:.0f} s per {n}-event batch (reference -Ofast build, "
                        f"OpenMP {threads} threads)",
            "fft": FFT_NOTE,
            "phases_s": {w["classes"][i]["nucleus"]: v["phases_s"]
                         for i, v in per_class.items()}}


def run_reference(args, world, rank):
    """The reference arm: whole events of the headline workload on the host
    cores, in the batch's class proportions (4 O+O then 1 Pb+Pb, repeating),
    one event per step, at most 5 steps (one full rotation, the batch's mix
    exactly) so the run stays within a few minutes. No warm-up: every event
    is a fresh process, as in the reference's own executable."""
    if rank != 0:
        return
    why = reference_available()
    if why:
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return
    threads = os.cpu_count() or 1
    w = HEADLINE
    evs = job_events(w, 1)
    by_class = [[e for e in evs if e["cls"] == i] for i in range(len(w["classes"]))]
    ratio = [c["count"] for c in w["classes"]]
    unit = min(ratio)
    order = []
    idx = [0] * len(ratio)
    while len(order) < sum(ratio):
        for i, r in enumerate(ratio):
            for _ in range(r // unit):
                order.append(by_class[i][idx[i] % len(by_class[i])])
                idx[i] += 1
    K = max(1, min(args.steps, sum(r // unit for r in ratio)))
    done = [reference_event(order[k], w, threads) for k in range(K)]
    total = sum(d["seconds"] for d in done)
    v = K / total
    mix = {}
    for k in range(K):
        key = f"{order[k]['nucleus']}{order[k]['N']}"
        mix[key] = mix.get(key, 0) + 1
    sample = (f"{K} whole events of the workload ("
              + ", ".join(f"{n} x {k}" for k, n in mix.items())
              + f") in {total:.1f} s, reference -Ofast build, OpenMP {threads} threads")
    line = {"metric": METRIC, "value": round(v, 6), "unit": "events/s", "n_gpus": world,
            "steps": K, "warmup": 0, "ms_per_step": round(1e3 * total / K, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (same generator and events as the GPU arm)",
            "config": workload_config(w, world),
            "impl": "reference",
            "fft": FFT_NOTE,
            "per_event_s": [round(d["seconds"], 2) for d in done],
            "phases_s": [d["phases_s"] for d in done],
            "cpu_baseline": {"value": round(v, 6), "unit": "events/s", "cores": threads,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": round(v, 6), "unit": "events/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
