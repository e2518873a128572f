"""Benchmark of the IP-Glasma hot path on B200.

One step = one Pb+Pb event of the 512^2 workload (L = 40 fm, b = 6 fm,
Ny = 50, tau up to 0.6 fm/c, 77 leapfrog steps): colour-charge noise ->
Poisson solve -> Wilson lines -> tau = 0 Newton links -> leapfrog ->
T^{mu nu} + Landau matching + eccentricities. Each step draws fresh noise
(device Philox, new key per event) on the same g^2 mu^2 maps, which stay
resident in HBM.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Reported (one JSON line, rank 0):
  value       events/s of the FP32-bulk form (whole job, all ranks)
  fp64        the plain FP64 form on the same events
  error       FP32-bulk vs FP64 on the same event: per-cell e, epsilon_2, E_T
  e2e         the same events through the C ABI with host buffers: g^2 mu^2
              maps copied in and e, u, pi, T^{mu nu} copied out every event
  roofline    the fused leapfrog kernel of the FP32 form against measured HBM
  cpu_baseline the reference (oracle/_ref, OpenMP, all host cores) on a
              bounded sample of the same event, scaled to one event
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

WORKLOAD = dict(name="PbPb_512", N=512, L=40.0, nucleus="Pb", b=6.0, Ny=50,
                maxtime=0.6, g=2.0, m=0.2)
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


def cfg_for(precision: int, seed: int):
    import ipglasma_b200 as ipg
    w = WORKLOAD
    return ipg.Config(size=w["N"], L=w["L"], Ny=w["Ny"], g=w["g"], m=w["m"],
                      maxtime=w["maxtime"], precision=precision, seed=seed)


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
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched uneven-events measurement")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint (forward/backward) measurement")
    ap.add_argument("--profile", choices=["fp32", "fp64", "both", "adjoint"], default=None,
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
    A, B = make_inputs()
    d_A = torch.tensor(A, dtype=torch.float64, device="cuda")
    d_B = torch.tensor(B, dtype=torch.float64, device="cuda")
    l2buf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    N = WORKLOAD["N"]
    seed_base = rank_seed_base(rank)

    ev32 = ipg.Event(cfg_for(ipg.FP32, seed_base))
    ev64 = ipg.Event(cfg_for(ipg.FP64, seed_base))
    itmax = ev32.itmax
    launches0 = ev32.kernel_launches()

    # warm-up (untimed)
    run_events(torch, ev32, d_A, d_B, W, seed_base, l2buf)
    run_events(torch, ev64, d_A, d_B, min(W, 3), seed_base, l2buf)

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # --- timed: FP32-bulk form (the headline) -------------------------------
    launches_before = ev32.kernel_launches()
    with ClockSampler(local) as clk:
        barrier()
        t32, lf32 = run_events(torch, ev32, d_A, d_B, K, seed_base + 100, l2buf)
        barrier()
    launches_timed = ev32.kernel_launches() - launches_before
    # --- timed: plain FP64 form ----------------------------------------------
    barrier()
    t64, lf64 = run_events(torch, ev64, d_A, d_B, K, seed_base + 100, l2buf)
    barrier()

    ms32, ms64 = max_over_ranks(dist, [float(np.sum(t32)), float(np.sum(t64))], "cuda")
    ev_per_s32 = whole_job_rate(world, K, ms32)
    ev_per_s64 = whole_job_rate(world, K, ms64)
    su32 = N * N * itmax / (np.mean(lf32) * 1e-3)
    su64 = N * N * itmax / (np.mean(lf64) * 1e-3)

    # --- error of the FP32 form against FP64 on one event -------------------
    err = compare_forms(ev32, ev64, d_A, d_B, seed_base + 7)

    # --- end to end through the C ABI with host buffers ---------------------
    e2e = measure_e2e(torch, ipg, A, B, K, seed_base + 500, l2buf, dist)
    e2e["ms"] = max_over_ranks(dist, [e2e["ms"]], "cuda")[0]

    peaks = load_peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)
    achieved = su32 * BYTES_PER_SITE_UPDATE["fp32"] / 1e9
    traffic = load_traffic()
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
            "frac": round(achieved / hbm, 4), "traffic": traffic,
            "kernel": "k_leapfrog_tile (FP32 bulk: TMA-staged 8x32 tiles, both directions in packed f32x2 lanes)",
            "bytes_per_site_update": BYTES_PER_SITE_UPDATE["fp32"],
            "bytes_stored_per_site_update": BYTES_STORED_PER_SITE_UPDATE["fp32"],
            "stored_frac": round(su32 * BYTES_STORED_PER_SITE_UPDATE["fp32"] / 1e9 / hbm, 4),
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
            "fp64_kernel": {"kernel": "k_leapfrog_tile64 (FP64 plain form: TMA-staged 4x32 tiles)", "achieved": round(su64 * BYTES_PER_SITE_UPDATE["fp64"] / 1e9, 1),
                            "frac": round(su64 * BYTES_PER_SITE_UPDATE["fp64"] / 1e9 / hbm, 4),
                            "bytes_per_site_update": BYTES_PER_SITE_UPDATE["fp64"],
                            "bytes_stored_per_site_update": BYTES_STORED_PER_SITE_UPDATE["fp64"],
                            "stored_frac": round(su64 * BYTES_STORED_PER_SITE_UPDATE["fp64"] / 1e9 / hbm, 4)}}

    batched = None if args.no_batched else measure_batched(torch, ipg, rank, dist)
    adjoint = None if args.no_adjoint else measure_adjoint(torch, ipg, rank)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample()

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": round(ev_per_s32, 3),
            "unit": "events/s",
            "n_gpus": world,
            "steps": K,
            "warmup": W,
            "ms_per_step": round(ms32 / K, 3),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 (FP64 Newton, Wilson lines, observables, reductions)",
            "data": "synthetic (seeded Woods-Saxon Pb+Pb, g2mu ~ sqrt(T_A), device Philox noise)",
            "config": {"workload": WORKLOAD["name"], "N": N, "L_fm": WORKLOAD["L"],
                       "Ny": WORKLOAD["Ny"], "b_fm": WORKLOAD["b"], "tau_fm": WORKLOAD["maxtime"],
                       "leapfrog_steps": itmax, "events_per_gpu": K,
                       "l2": "flushed (256 MB write) before every event",
                       "parallelism": f"events sharded over {world} GPU(s), no collective"},
            "site_updates_per_s": round(world * su32, 1),
            "fp64": {"events_per_s": round(ev_per_s64, 3), "ms_per_event": round(ms64 / K, 3),
                     "site_updates_per_s": round(world * su64, 1)},
            "fp32_over_fp64_events": round(ev_per_s32 / ev_per_s64, 3),
            "error": err,
            "e2e": {"value": round(whole_job_rate(world, K, e2e["ms"]), 3), "unit": "events/s",
                    "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"],
                    "form": "fp32", "host_buffers": e2e["host_buffers"],
                    "copies": e2e["copies"]},
            "writers": e2e["writers"] if rank == 0 else None,
            "roofline": roof,
            "batched": batched,
            "adjoint": adjoint,
            "cpu_baseline": cpu,
            "gpu_launches": int(launches_timed),
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    ev32.close()
    ev64.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


BATCH = dict(oo=64, pb=16, maxtime=0.4, reps=2)


def measure_batched(torch, ipg, rank, dist):
    """Batched uneven events: 64 O+O at 256^2 (L = 20 fm) and 16 Pb+Pb at 512^2
    (L = 40 fm), impact parameters uniform in [0, 2R], Ny = 50, FP32 bulk, to
    tau = 0.4 fm (52 steps for both sizes, a = 0.078125 fm). Per batch: the
    initial conditions of every event, then one persistent leapfrog launch per
    step over all 80 lattices (a replayed CUDA graph, launch shape from the
    autotuner), then the observables of every event."""
    from ipglasma_b200.synthetic import make_event
    rng = np.random.default_rng(5 + rank)
    evs = []
    for k in range(BATCH["oo"] + BATCH["pb"]):
        oo = k < BATCH["oo"]
        N, L, nuc, R = (256, 20.0, "O", 2.61) if oo else (512, 40.0, "Pb", 6.62)
        A, B, _, _ = make_event(N, L, nuc, rng.uniform(0.0, 2.0 * R), 7000 + 100 * rank + k)
        ev = ipg.Event(ipg.Config(size=N, L=L, Ny=50, maxtime=BATCH["maxtime"],
                                  precision=ipg.FP32, seed=rank_seed_base(rank) + 600 + k))
        ev.set_g2mu(A, B)
        ev.use_device_noise()
        evs.append(ev)

    batch = ipg.Batch(evs)

    def init_all():
        batch.init_fields(allow_nonconverged=True)

    init_all()
    tune = batch.tune()
    batch.run()  # warm-up: captures the graph
    times, evo = [], []
    for r in range(BATCH["reps"]):
        torch.cuda.synchronize()
        st = torch.cuda.Event(enable_timing=True)
        en = torch.cuda.Event(enable_timing=True)
        st.record()
        init_all()
        batch.run()
        en.record()
        torch.cuda.synchronize()
        times.append(st.elapsed_time(en))
        evo.append(batch.stats()[0])
    launches = batch.stats()[2]
    batch.close()
    for ev in evs:
        ev.close()
    ms = max_over_ranks(dist, [float(np.mean(times))], "cuda")[0]
    n_ev = len(evs)
    world = dist.get_world_size() if dist else 1
    sites = BATCH["oo"] * 256 ** 2 + BATCH["pb"] * 512 ** 2
    steps = evs[0].itmax
    return {"workload": f"{BATCH['oo']} O+O 256^2 + {BATCH['pb']} Pb+Pb 512^2, "
                        f"Ny 50, tau {BATCH['maxtime']} fm, FP32 bulk",
            "events_per_s": round(whole_job_rate(world, n_ev, ms), 2),
            "ms_per_batch": round(ms, 2),
            "evolution_ms": round(float(np.mean(evo)), 2),
            "leapfrog_steps": steps,
            "site_updates_per_s_evolution": round(sites * steps / (np.mean(evo) * 1e-3), 1),
            "launches_per_batch_evolution": steps,
            "cuda_graph": True,
            "tuned_shape": {"tile_rows": tune.tile_rows, "threads": tune.threads_per_block,
                            "blocks_per_sm": tune.blocks_per_sm, "grid": tune.grid,
                            "candidates": tune.candidates},
            "timing": "CUDA events around init of all events + batched run, mean of "
                      f"{BATCH['reps']}; total batched launches {launches}"}


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
    out = {}
    for frac in (1e-2, 1e-3):
        m = e64 > frac * e64.max()
        rel = np.abs(e32[m] - e64[m]) / np.abs(e64[m])
        out[f"e_rel_max_gt{frac:g}max"] = float(rel.max())
        out[f"e_rel_rms_gt{frac:g}max"] = float(np.sqrt(np.mean(rel ** 2)))
    out["eps2_rel"] = abs(r32.eccentricity[1] - r64.eccentricity[1]) / abs(r64.eccentricity[1])
    out["E_T_rel"] = abs(r32.E_T - r64.E_T) / abs(r64.E_T)
    out["gauss_fp32"] = r32.gauss_violation
    out["gauss_fp64"] = r64.gauss_violation
    out["unitarity_fp32"] = r32.unitarity_max
    out["unitarity_fp64"] = r64.unitarity_max
    return out


def measure_e2e(torch, ipg, A, B, K, seed0, l2buf, dist):
    """Events through the C ABI with host buffers: g2mu maps in, observables
    out. Each event's observables are copied back on the library's copy
    stream (ipg_get_observables_async) while the next event starts; the K
    events, the L2 flush before each, and the last copy are one timed region."""
    ev = ipg.Event(cfg_for(ipg.FP32, seed0))
    n = ev.n

    def pinned(shape):
        # page-locked host memory (torch's pinned allocator), seen as numpy
        return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()

    hA, hB = pinned(A.shape), pinned(B.shape)
    hA[...] = A
    hB[...] = B
    # two sets of page-locked observable arrays, alternating between events
    sets = [(pinned((n,)), pinned((4, n)), pinned((10, n)), pinned((10, n))) for _ in range(2)]
    cur = torch.cuda.current_stream()

    def one(seed, k):
        flush_l2(torch, l2buf)
        cur.synchronize()  # torch's stream only: the previous copy keeps running
        ev_reset(ev, seed)
        ev.set_g2mu(hA, hB)
        ev.use_device_noise()
        ev.init_fields(allow_nonconverged=True)
        ev.run()
        ev.observables_async(*sets[k % 2])
    for k in range(3):
        one(seed0 + k, k)
    ev.wait_observables()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(K):
        one(seed0 + 10 + k, k)
    ev.wait_observables()
    torch.cuda.synchronize()
    total = time.perf_counter() - t0
    itmax = ev.itmax
    dtau = ev.dtau
    eps, u4, pi10, T10 = sets[(K - 1) % 2]
    writers = measure_writers(ipg, ev, eps, u4, pi10, T10, itmax, dtau)
    ev.close()
    return {"ms": total * 1e3, "h2d": int(2 * n * 8), "d2h": int(25 * n * 8),
            "host_buffers": "pinned", "writers": writers,
            "copies": "observables back on a copy stream, overlapping the next event; "
                      "L2 flush before each event and the last copy inside the timed region"}


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
    """DRAM bytes per launch of the FP32 leapfrog kernel from the committed ncu
    summary (profiles/leapfrog_fp32_PbPb512.json), or None."""
    p = ROOT / "profiles" / "leapfrog_fp32_PbPb512.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get("dram_bytes_per_launch")
        except Exception:
            return None
    return None


# ---------------------------------------------------------------------------
# CPU baseline: the reference itself (oracle/_ref), all host cores
# ---------------------------------------------------------------------------
SAMPLE = dict(N=128, L=10.0, Ny=50)  # same lattice spacing as the 512^2 event


def cpu_baseline_sample(threads: int | None = None):
    """Time the reference on a bounded sample of the workload: the same lattice
    spacing (a = 0.078125 fm), Ny, tau and schedule on a 128^2 patch centred on
    a Pb+Pb collision; scaled by the site count (512^2 / 128^2 = 16) to one
    event, which is how every stage of the reference scales (the FFTs by a
    further log factor, ignored here in the reference's favour)."""
    sys.path.insert(0, str(ROOT / "tests"))
    from refcase import HARNESS, run_harness
    from ipglasma_b200.synthetic import make_event
    if not HARNESS.exists():
        return {"value": None, "unit": "events/s", "cores": 0, "kind": "reference",
                "sample": "oracle/_ref/ipg_ref_harness not built"}
    threads = threads or os.cpu_count() or 1
    s = SAMPLE
    A, B, _, _ = make_event(s["N"], s["L"], WORKLOAD["nucleus"], WORKLOAD["b"], seed=11)
    with tempfile.TemporaryDirectory() as tmp:
        t0 = time.perf_counter()
        r = run_harness(Path(tmp) / "ref", A, B, s["N"], s["L"], s["Ny"], WORKLOAD["g"],
                        WORKLOAD["m"], 5, WORKLOAD["maxtime"], threads=threads)
        wall = time.perf_counter() - t0
    scale = (WORKLOAD["N"] / s["N"]) ** 2
    t_event = wall * scale
    return {"value": round(1.0 / t_event, 6), "unit": "events/s", "cores": threads,
            "kind": "reference",
            "sample": (f"reference -O2 OpenMP harness, one event at N={s['N']} L={s['L']} fm "
                       f"(same a, Ny={s['Ny']}, tau={WORKLOAD['maxtime']} fm) in {wall:.1f} s, "
                       f"x{scale:.0f} sites -> {t_event:.1f} s per 512^2 event"),
            "phases_s": {k: r.meta[k] for k in ("t_setV", "t_tau0", "t_evolution")}}


def run_reference(args, world, rank):
    if rank != 0:
        return
    K, W = args.steps, args.warmup
    threads = os.cpu_count() or 1
    vals = []
    for k in range(max(1, min(K, 3))):
        cb = cpu_baseline_sample(threads)
        if cb["value"] is None:
            print(json.dumps({"impl": "reference", "unavailable": cb["sample"]}))
            return
        vals.append(cb["value"])
    v = float(np.mean(vals))
    line = {"metric": METRIC, "value": round(v, 6), "unit": "events/s", "n_gpus": world,
            "steps": len(vals), "warmup": 0, "ms_per_step": round(1e3 / v, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (same generator as the GPU arm)",
            "config": {"workload": WORKLOAD["name"], "N": WORKLOAD["N"]},
            "impl": "reference",
            "cpu_baseline": dict(cb, value=round(v, 6)),
            "e2e": {"value": round(v, 6), "unit": "events/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
