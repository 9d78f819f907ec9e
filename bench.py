"""Benchmark: pGM rigid-water MD on the B200 engine, ns/day and CG iterations per step, with the
learned initial guess against plain CG.

Headline workload (one GPU): 32,768 pGM3P-25 waters (98,304 atoms) on a seeded jittered 32^3
lattice in a 9.93 nm cubic box, cutoff 0.9 nm, Ewald 4.0 / nm, PME 192^3 order 6, mixed precision
(FP32 pair / PME / CG vectors, FP64 reductions), Langevin NVT 298 K with gamma 2 / ps, dt 1 fs, CG to
max|alpha r| / mean|alpha b| <= 1e-6 with the reference's local preconditioner (one inner CG
iteration on the row entries inside 0.3 nm; `--local-niter 0` for Jacobi, the reference's default).
A step is one captured CUDA graph: rigid-body kick/drift/Langevin, the force call (rows, PME, CG
as a device-side while loop, energy / forces / virial), closing kick.  `--workload water4096` runs the same line on 4,096 waters (4.966 nm, PME 96^3).

The headline run starts every solve from the learned guess, the 2-layer message-passing model on the
0.5 nm graph: plain-solver MD on the 4,096-water box writes the training frames, the model trains on
the GPU (outside the timed region), then the timed MD uses it.  Beside it, the same MD with plain CG
from the previous step's dipoles (mu1) and from the reference's default mu4 predictor, and with the
per-atom MLP guess (`--model mlp` makes the MLP the headline and measures the network beside it).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload NAME]

With N > 1 (torchrun, one process per GPU) every rank runs its own independent replica (the path
has no exchange step: replicas only); value = total ns/day over the ranks, time = max over ranks.
--impl reference times the CPU restatement of the reference's algorithm (the FP64 oracle, all host
threads) on the same workload, on rank 0 only.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DT_FS, GAMMA, TEMP, TOL = 1.0, 2.0, 298.0, 1e-6
METRIC = "ns/day & CG iters/step on 1 B200: NN-guess vs plain CG at residual≤1e-6"

# water boxes of the MD line: lattice side, box edge [nm], PME mesh
BOXES = {
    "water32768": {"n_side": 32, "edge": 9.93, "grid": 192, "atoms": 98304,
                   "equil_steps": 500, "published": None},
    "water4096": {"n_side": 16, "edge": 4.966, "grid": 96, "atoms": 12288, "equil_steps": 1000,
                  "published": "44 ns/day, 4096 waters, mixed, tol 1e-5, 1x RTX PRO 6000 Blackwell (README.md:448)"},
}
W = dict(BOXES["water32768"], name="water32768")  # the workload of this run (set from --workload)
TRAIN_BOX = "water4096"  # the learned guess trains on pairs written by the plain solver on this box
MODEL = ["mpnn"]  # the headline's learned guess (set from --model)


def config() -> dict:
    n_w = W["atoms"] // 3
    K = W["grid"]
    return {
        "workload": f"{n_w} rigid pGM3P-25 waters, {W['edge']} nm box, PME {K}^3 o6, rc 0.9 nm, beta 4.0/nm, Langevin "
        "298 K gamma 2/ps, dt 1 fs, mixed precision, CG tol 1e-6 from the learned guess "
        f"({'2-layer message-passing model' if MODEL[0] == 'mpnn' else 'per-atom MLP'}, trained on 4096-water frames)",
        "atoms": W["atoms"],
        "pme_grid": [K, K, K],
        "cutoff_nm": 0.9,
        "dt_fs": DT_FS,
        "cg_tol": TOL,
        "solver": "CG from mu4 + the learned correction (fused start); plain CG from mu1 and mu4 beside it",
        "l2": f"working set larger than L2: pair rows 8 x 4 B x {W['atoms']} x capacity "
        f"= {8 * 4 * W['atoms'] * 416 / 1e6:.0f} MB (126 MB L2)",
        "seeds": {"positions": 0, "velocities_thermostat": 1},
        "equilibration": f"{W['equil_steps']} steps of 1 fs at gamma 20/ps from the lattice start, before timing",
        **({"split_rows": f"electrostatics {SPLIT['elec_cutoff']} nm, beta {SPLIT['ewald_beta']:.4f}/nm, LJ 0.9 nm"}
           if SPLIT else {}),
        "preconditioner": (f"local: {LOCAL['local_niter']} inner CG iterations on the row entries inside 0.3 nm "
                           "(forcefield.py:1766-1792), every arm" if LOCAL["local_niter"] else "Jacobi (the reference's default)"),
    }


EQUIL_GAMMA = 20.0  # relaxation of the lattice start before any data or timing


def equilibrate(md, steps: int | None = None) -> None:
    """Relax the lattice start (random orientations) with direct steps under a strong thermostat
    (gamma 20 / ps, then back to the run's gamma), outside any timed region."""
    g = md.gamma
    md.gamma = EQUIL_GAMMA
    for _ in range(W["equil_steps"] if steps is None else steps):
        md.step()
    md.gamma = g
    md.stream.synchronize()


# DRAM bytes of one k_rowfield<float, 0, 1> launch (read + write) from an ncu capture of this
# workload (profiles/k_rowfield_water4096.txt), with the pair count it had; scaled by pairs.
ROWFIELD_NCU_DRAM_BYTES, ROWFIELD_NCU_PAIRS = 93.654784e6 + 3.39328e6, 3.745e6


SPLIT: dict = {}  # --elec-cutoff: split rows (elec_cutoff, ewald_beta for it; the meshes fit its spacing)


LOCAL = {"local_niter": 1}  # --local-niter: the local preconditioner in every arm (0: Jacobi, the reference's default)


def settings(precision="mixed", predictor="mu4", grid=None):
    from pgm_jax_b200.forcefield import MDSettings

    K = W["grid"] if grid is None else grid
    return MDSettings(precision=precision, cutoff=0.9, ewald_beta=SPLIT.get("ewald_beta", 4.0), pme_grid=(K, K, K),
                      pme_order=6, dipole_tol=TOL, max_iter=100, predictor=predictor, elec_cutoff=SPLIT.get("elec_cutoff"),
                      local_cut=0.3, local_niter=LOCAL["local_niter"])


def headline_box(seed: int = 0):
    from pgm_jax_b200.systems import water_box

    return water_box(W["n_side"], W["edge"], seed=seed)


def ns_per_day(ms_per_step: float) -> float:
    return 86.4 * DT_FS / ms_per_step


def bytes_per_step(n_atoms: int, pairs: float, n_it: float, K: int) -> float:
    """Algorithmic bytes of one MD step: row build 32 B/pair, (n_it + 1) CG sweeps of 24 B/pair, the
    force pass 40 B/pair, (n_it + 2) PME passes of 24 K^3 + 288 N bytes, 400 B/atom of state."""
    return pairs * (32 + 24 * (n_it + 1) + 40) + (n_it + 2) * (24 * K**3 + 288 * n_atoms) + 400 * n_atoms


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    def __init__(self, index: int) -> None:
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        self.window = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def mark(self, t0: float, t1: float) -> None:
        """The timed region's wall-clock window (samples outside it are dropped when some fall inside)."""
        self.window = (t0, t1)

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [[c.strip() for c in r.split(",")] for r in self.f.read().strip().splitlines() if r.count(",") >= 9]
        os.unlink(self.f.name)
        if self.window and rows:
            import datetime

            def when(r):
                try:
                    return datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                except ValueError:
                    return None

            inside = [r for r in rows if when(r) is not None and self.window[0] <= when(r) <= self.window[1]]
            if inside:
                rows = inside
        rows = [r[1:] for r in rows]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def drift_frames(s, pos, seed: int = 1):
    """Frames of a smooth trajectory for the CPU leg: every molecule translated at a Maxwell velocity
    (298 K) by 1 fs per frame, so that the predictor extrapolates a smooth history as in MD."""
    rng = np.random.default_rng(seed)
    mw = float(s.masses[s.mol == 0].sum())  # every molecule of the box is a water
    v = rng.normal(scale=np.sqrt(0.0083144626 * TEMP / mw), size=(s.nmol, 3))[s.mol]  # nm/ps
    return lambda k: pos + v * (k * DT_FS * 1e-3)


def cpu_reference(steps: int, warmup: int, budget_s: float = 120.0):
    """The FP64 CPU oracle (restatement of the reference's algorithm) on the same workload: the
    first four frames of a smooth trajectory fill the predictor's history untimed, then up to
    `steps` force steps are timed, time-boxed to `budget_s`."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # noqa: E402  (the checker; this is the reference arm / CPU baseline)

    s, pos, H = headline_box()
    K = W["grid"]
    st = dict(cutoff=0.9, ewald_beta=4.0, pme_grid=(K, K, K), pme_order=6, dipole_tol=TOL, max_iter=100,
              local_cut=0.3, local_niter=LOCAL["local_niter"])
    cores = os.cpu_count() or 1
    o = O.Oracle(s, st, nthreads=cores)
    ind = o.init_induction()
    frame = drift_frames(s, pos)
    n_fill = 4  # mu4 extrapolates once the history holds four steps (forcefield.py:1917-2008)
    times, iters = [], []
    t_start = time.perf_counter()
    k = 0
    while len(times) < max(1, steps):
        t0 = time.perf_counter()
        r = o.compute(frame(k), H, ind)
        dt = time.perf_counter() - t0
        ind = r["induction"]
        k += 1
        if k > n_fill:
            times.append(dt)
            iters.append(r["iterations"])
        if time.perf_counter() - t_start > budget_s and times:
            break
    ms = 1e3 * float(np.mean(times))
    return {
        "value": ns_per_day(ms), "ms_per_step": ms, "cores": cores, "steps_timed": len(times),
        "cg_iters_per_step": float(np.mean(iters)),
        "sample": f"{len(times)} force steps of the {W['atoms'] // 3}-water workload (FP64 oracle, {cores} threads, "
        f"mu4 predictor, CG 1e-6, local preconditioner {LOCAL['local_niter']} inner iterations) on a smooth drift "
        f"trajectory, after {n_fill} untimed steps that fill the history; "
        "the rigid-body integrator's cost (<1%) is not included",
    }


def run_reference(args) -> None:
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    r = cpu_reference(args.steps, args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": "ns/day", "n_gpus": args.gpus,
        "steps": r["steps_timed"], "warmup": 4, "ms_per_step": r["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config(), "cg_iters_per_step": r["cg_iters_per_step"],
        "cpu_baseline": {"value": r["value"], "unit": "ns/day", "cores": r["cores"], "kind": "port", "sample": r["sample"]},
        "e2e": {"value": r["value"], "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference (JAX) is not installable here (no jax/jax_md wheels, no network); its algorithm is "
        "timed through the project's FP64 C restatement (oracle/)",
    }
    print(json.dumps(line), flush=True)


def train_guess(rank: int, torch, kind: str) -> tuple:
    """Plain-solver MD on the 4,096-water box writes (features, mu* - mu4 guess) pairs -- frame by
    frame with the graph for the message-passing model; the model trains on the GPU.  Returns the
    model and what was trained."""
    from pgm_jax_b200.forcefield import PGMForceField
    from pgm_jax_b200.learned import GuessModel, MPNNModel, collect, collect_frames
    from pgm_jax_b200.md import RigidMD
    from pgm_jax_b200.systems import water_box

    t0 = time.perf_counter()
    B = BOXES[TRAIN_BOX]
    s, pos, H = water_box(B["n_side"], B["edge"], seed=0)
    ff = PGMForceField(s, H, settings(predictor="nn", grid=B["grid"]), device=torch.cuda.current_device())
    md = RigidMD(ff, pos, H, temperature=TEMP, dt_fs=DT_FS, gamma_ps=GAMMA, seed=1 + rank)
    equilibrate(md, B["equil_steps"])
    frames = 64
    if kind == "mpnn":
        iters = 2000
        train = collect_frames(md, frames)
        model = MPNNModel(seed=0, device=torch.cuda.current_device())
        model.train(train, iters=iters, lr=2e-3)
        pairs = sum(int(f["inv"].shape[0]) for f in train)
        what = ("2-layer message-passing model on the 0.5 nm graph (64 hidden; continuous-filter convolutions: 16 "
                "message features, filters over 8 radial functions; edge sums as BF16 warp MMAs, dense layers as fused "
                "tcgen05 tiles, FP32 accumulation), one frame per Adam step")
    else:
        iters = 2000
        train = collect(md, frames)
        model = GuessModel(seed=0, device=torch.cuda.current_device())
        model.train(train, iters=iters, batch=32768, lr=2e-3)
        pairs = int(train["inv"].shape[0])
        what = "per-atom MLP 16 -> 64 -> 64 -> 32 on radial-basis features of the 0.5 nm graph (WMMA BF16)"
    info = {"model": what, "train_box": f"{B['atoms'] // 3} waters, {B['edge']} nm, PME {B['grid']}^3",
            "train_frames": frames, "train_pairs": pairs, "adam_steps": iters, "seconds": time.perf_counter() - t0}
    del md, ff, train
    return model, info


def run_engine(args) -> None:
    import torch
    import torch.distributed as dist

    from pgm_jax_b200 import _lib
    from pgm_jax_b200.forcefield import PGMForceField
    from pgm_jax_b200.learned import collect, guess_errors
    from pgm_jax_b200.md import RigidMD

    ws, rank, local = dist_env()
    if ws > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    model, train_info = train_guess(rank, torch, args.model) if args.nn else (None, None)
    s, pos, H = headline_box()
    ff = PGMForceField(s, H, settings(predictor="nn" if args.nn else "mu4"), device=local)
    md = RigidMD(ff, pos, H, temperature=TEMP, dt_fs=DT_FS, gamma_ps=GAMMA, seed=1 + rank)
    lib = ff._lib
    equilibrate(md)
    if args.nn:  # held-out frames of this box (plain solver: the model is not installed yet)
        if args.model == "mpnn":
            from pgm_jax_b200.learned import collect_frames, frame_errors

            held = collect_frames(md, 6)
            train_info["guess_rms_e_nm_held_out"] = frame_errors(model, held)
        else:
            held = collect(md, 6)
            train_info["guess_rms_e_nm_held_out"] = guess_errors(model, held)
        train_info["start"] = "x0 = mu4 + the model's correction, fused start (one field sweep, as mu4)"
        del held
        model.install(ff)
    # warm-up: direct steps (rows sized), then capture and replay
    for _ in range(max(1, args.warmup)):
        md.step()
    md.stream.synchronize()
    md.capture()
    md.run(3)
    md.stream.synchronize()
    it0 = int(md.result.iterations[0])
    builds0 = int(lib.pgm_list_rebuilds(ff._h))
    # the clock sampler starts while warm-up replays keep the GPU busy, so that the timed region
    # begins on a loaded GPU at its running clocks (not after an idle gap)
    clk = Clocks(local)
    n_pre = max(3, args.warmup) + 50
    md.run(n_pre)
    # timed region: K graph replays between CUDA events on the MD stream; clocks sampled meanwhile
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    t_wall = time.time()
    ms, n_it = timed_replays(md, args.steps, torch, label="timed_md")
    clk.mark(t_wall, time.time())
    clocks = clk.stop()
    rebuilds = int(lib.pgm_list_rebuilds(ff._h)) - builds0  # over the last warm-up replays and the timed ones
    rebuilds_steps = args.steps + n_pre
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if ws > 1:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    status = int(md.result.status[0])
    launches = args.steps * (md.launches_outside_loop + max(n_it, md.unrolled_iterations) * md.launches_per_iteration)
    # the dominant kernel: the CG matvec, timed alone with CUDA events on the MD stream
    pairs = int(lib.pgm_row_pairs(ff._h))
    kt = {}
    for which, name in ((0, "cg_matvec_fused"), (1, "spread"), (2, "fft_chain"), (3, "forces"), (4, "rows"),
                        (5, "fft_x_fwd_alone"), (6, "spread_then_fft_x_fwd"), (7, "row_field"), (8, "pme_gather"),
                        (9, "cg_sweep")) + (((10, "nn_chan"), (11, "nn_features"), (12, "nn_model")) if args.nn else ()):
        v = C_double()
        _lib.check(lib.pgm_profile_kernel(ff._h, C_void_p(md.stream.cuda_stream), which, 20, byref(v)))
        kt[name] = v.value
    peak, peak_kind = peaks()
    mv_bytes = 24.0 * pairs + 32.0 * ff.n  # rows (k, x, y, z, G1, G2) + the dipole vector in and out
    mv_gbs = mv_bytes / (kt["row_field"] * 1e-3) / 1e9
    step_bytes = bytes_per_step(ff.n, pairs, n_it, W["grid"])
    # three MD steps launched directly (the CG loop driven from the host), untimed, in their own
    # NVTX range: a profiler cannot see the kernels of graphs with conditional nodes
    with torch.cuda.stream(md.stream):
        torch.cuda.nvtx.range_push("direct_md")
        for _ in range(3):
            md.step()
        md.stream.synchronize()
        torch.cuda.nvtx.range_pop()
    # end to end: the force call through the C ABI with host buffers (positions in, forces out; the
    # induction state on the device, or copied in and out every step), the integrator on the GPU
    e2e = run_e2e(md, ff, args.steps, torch, lib, _lib)
    e2e_host_state = run_e2e(md, ff, args.steps, torch, lib, _lib, state_on_device=False)
    tuning = ff.tuning()
    if args.nn:
        train_info["fallbacks_in_run"] = int(ff.nn_fallback_stats()["fallbacks"][0])
    final = {"pos": md.pos.cpu().numpy(), "box": md.box[0].cpu().numpy(),
             "ind": {k: getattr(md.ind, k).cpu().numpy() for k in ("mu", "hist", "count", "norm")}}
    del md
    # plain CG on the same workload: from the previous step's dipoles and from mu4
    plain = {p: run_plain(s, pos, H, rank, p, args, torch) for p in (("mu1", "mu4") if args.nn else ())}
    other = "mlp" if args.model == "mpnn" else "mpnn"
    alt = run_learned(s, pos, H, rank, other, args, torch) if (args.nn and args.other_model) else None
    acc = accuracy_vs_oracle(s, final, torch) if (rank == 0 and args.cpu_baseline) else None
    value = ws * ns_per_day(ms_max)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "ns/day", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic", "config": config(), "cg_iters_per_step": n_it, "cg_iters_first_step": it0,
            "status": status, "gpu_launches": int(round(launches)), "list_rebuilds_per_step": rebuilds / rebuilds_steps,
            "clocks": clocks,
            "roofline": {
                "bound": "hbm", "kernel": "k_rowfield (CG matvec row stream: k, x, y, z, G1, G2 per pair)",
                "achieved": mv_gbs, "peak": peak, "unit": "GB/s", "frac": mv_gbs / peak, "peak_kind": peak_kind,
                "traffic": ROWFIELD_NCU_DRAM_BYTES * pairs / ROWFIELD_NCU_PAIRS, "traffic_unit": "bytes per launch (ncu)",
                "bytes_per_launch": mv_bytes, "ms_per_launch": kt["row_field"],
                "step_bytes": step_bytes, "step_gbs": step_bytes / (ms_max * 1e-3) / 1e9,
                "step_frac": step_bytes / (ms_max * 1e-3) / 1e9 / peak,
            },
            "kernel_ms": kt, "pairs": pairs, "row_capacity": ff.capacity, "accuracy_vs_oracle": acc,
            "tuning": tuning,
            "e2e": e2e,
            "e2e_host_state": {k: e2e_host_state[k] for k in ("value", "unit", "ms_per_step", "h2d_bytes_per_step",
                                                              "d2h_bytes_per_step", "path")},
            "published_reference": W["published"],
        }
        if args.nn:
            line["learned_guess"] = train_info
            line["plain_cg"] = plain
            line["nn_over_plain_cg"] = {p: ns_per_day(ms_max) / v["value"] for p, v in plain.items()}
            if alt:
                alt["over_plain_cg"] = {p: alt["value"] / v["value"] for p, v in plain.items()}
                line["learned_guess_" + other] = alt
        if args.cpu_baseline:
            r = cpu_reference(2, 1, budget_s=30.0)
            line["cpu_baseline"] = {"value": r["value"], "unit": "ns/day", "cores": r["cores"], "kind": "port",
                                    "sample": r["sample"]}
        print(json.dumps(line), flush=True)
    del ff
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


def accuracy_vs_oracle(s, final: dict, torch, grid=None, label: str = "the final MD frame") -> dict:
    """Mixed precision (the timed path: FP32 kernels, FP64 reductions, CG 1e-6) and the FP64 engine
    (CG 1e-8) against the FP64 oracle (CG 1e-8) at the same coordinates, all three started from the
    MD's induction state at that frame (mu4 from its history)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # noqa: E402  (the checker)

    from pgm_jax_b200.forcefield import InductionState, MDSettings, PGMForceField

    pos, H, ind = final["pos"], final["box"], final["ind"]
    dev = torch.cuda.current_device()
    st = settings(grid=grid)
    K = st.pme_grid
    t0 = time.perf_counter()
    o = O.Oracle(s, dict(cutoff=0.9, ewald_beta=4.0, pme_grid=K, pme_order=6, dipole_tol=1e-8, max_iter=100),
                 nthreads=os.cpu_count() or 1)
    ref = o.compute(pos, H, {k: (np.array(v) if k in ("mu", "hist") else (int(v[0]) if k == "count" else float(v[0])))
                             for k, v in ind.items()})
    t_oracle = time.perf_counter() - t0

    def engine(prec, tol):
        ff = PGMForceField(s, H, MDSettings(**{**st.__dict__, "predictor": "mu4", "precision": prec, "dipole_tol": tol}),
                           device=dev)
        st_in = InductionState(*(torch.as_tensor(ind[k], device=ff.device) for k in ("mu", "hist", "count", "norm")))
        return ff.compute(pos, H, None, st_in)

    rms = lambda a, b: float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b**2)))  # noqa: E731
    out = {"frame": label, "oracle_energy_kjmol": ref["energy"]["total"], "oracle_iterations": ref["iterations"],
           "oracle_seconds": t_oracle}
    for name, prec, tol in (("mixed_tol1e-6", "mixed", TOL), ("fp64_tol1e-8", "double", 1e-8)):
        r = engine(prec, tol)
        e = float(r.energy["total"][0])
        out[name] = {"energy_rel": abs(e - ref["energy"]["total"]) / abs(ref["energy"]["total"]),
                     "forces_rms_rel": rms(r.forces.cpu().numpy(), ref["forces"]),
                     "mu_rms_rel": rms(r.induction.mu.cpu().numpy(), ref["mu"]), "iterations": int(r.iterations[0])}
        del r
    return out


def timed_replays(md, steps: int, torch, label: str | None = None) -> tuple:
    """(ms per step, mean CG iterations) of `steps` graph replays, CUDA events on the MD stream;
    `label` names an NVTX range around them (a profiler can restrict its capture to it)."""
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    it_sum = torch.zeros((), dtype=torch.int64, device=md.ff.device)
    if label:
        torch.cuda.nvtx.range_push(label)
    ev0.record(md.stream)
    for _ in range(steps):
        md.run(1)
        with torch.cuda.stream(md.stream):
            it_sum += md.result.iterations[0].to(torch.int64)
    ev1.record(md.stream)
    if label:
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize(md.ff.device)
    return ev0.elapsed_time(ev1) / steps, float(it_sum.item()) / steps


def run_plain(s, pos, H, rank, predictor, args, torch) -> dict:
    """The same MD with plain CG from `predictor`, graph-replayed and timed like the headline."""
    from pgm_jax_b200.forcefield import PGMForceField
    from pgm_jax_b200.md import RigidMD

    ff = PGMForceField(s, H, settings(predictor=predictor), device=torch.cuda.current_device())
    md = RigidMD(ff, pos, H, temperature=TEMP, dt_fs=DT_FS, gamma_ps=GAMMA, seed=1 + rank)
    equilibrate(md)
    for _ in range(max(1, args.warmup) + 4):
        md.step()
    md.capture()
    md.run(3)
    md.stream.synchronize()
    steps = max(10, min(args.steps, 300))
    ms, n_it = timed_replays(md, steps, torch)
    del md, ff
    return {"value": ns_per_day(ms), "unit": "ns/day", "ms_per_step": ms, "cg_iters_per_step": n_it, "steps": steps,
            "predictor": {"mu1": "previous step's dipoles", "mu4": "4 mu1 - 6 mu2 + 4 mu3 - mu4 (the reference's default)"}[
                predictor]}


def run_learned(s, pos, H, rank, kind, args, torch) -> dict:
    """The same MD with the other learned guess (trained the same way), timed like the headline."""
    from pgm_jax_b200.forcefield import PGMForceField
    from pgm_jax_b200.md import RigidMD

    model, info = train_guess(rank, torch, kind)
    ff = PGMForceField(s, H, settings(predictor="nn"), device=torch.cuda.current_device())
    md = RigidMD(ff, pos, H, temperature=TEMP, dt_fs=DT_FS, gamma_ps=GAMMA, seed=1 + rank)
    equilibrate(md)
    model.install(ff)
    for _ in range(max(1, args.warmup) + 4):
        md.step()
    md.capture()
    md.run(3)
    md.stream.synchronize()
    steps = max(10, min(args.steps, 300))
    ms, n_it = timed_replays(md, steps, torch)
    fb = int(ff.nn_fallback_stats()["fallbacks"][0])
    del md, ff, model
    return {"value": ns_per_day(ms), "unit": "ns/day", "ms_per_step": ms, "cg_iters_per_step": n_it, "steps": steps,
            "model": info["model"], "train_seconds": info["seconds"], "fallbacks_in_run": fb}


def run_e2e(md, ff, steps, torch, lib, _lib, state_on_device: bool = True) -> dict:
    """MD with the force call through pgm_compute_host: host positions in, host forces out, per step;
    the induction state kept on the device in the handle (ind = NULL), or with state_on_device=False
    copied in and out with every call."""
    import ctypes as C

    n = ff.n
    S = ff.nsys
    pin = lambda *shape, dt=torch.float64: torch.empty(shape, dtype=dt, pin_memory=True)  # noqa: E731
    h_pos, h_F, h_box = pin(n, 3), pin(n, 3), pin(S, 3, 3)
    h_mu, h_hist = pin(n, 3), pin(4, n, 3)
    h_cnt, h_norm = pin(S, dt=torch.int32), pin(S)
    h_E, h_V, h_it, h_res, h_st = pin(S, 3), pin(S, 3, 3), pin(S, dt=torch.int32), pin(S), pin(S, dt=torch.int32)
    md.stream.synchronize()
    h_box.copy_(md.box.cpu())
    h_mu.copy_(md.ind.mu.cpu()); h_hist.copy_(md.ind.hist.cpu()); h_cnt.copy_(md.ind.count.cpu()); h_norm.copy_(md.ind.norm.cpu())
    ind = _lib.PgmInduction(h_mu.data_ptr(), h_hist.data_ptr(), h_cnt.data_ptr(), h_norm.data_ptr())
    out = _lib.PgmOutputs(h_E.data_ptr(), h_F.data_ptr(), h_V.data_ptr(), h_it.data_ptr(), h_res.data_ptr(), h_st.data_ptr())
    st = C.c_void_p(md.stream.cuda_stream)
    steps = max(3, min(steps, 200))

    def one(load_state=False):
        _lib.check(lib.pgm_rigid_begin_step(md._h, st, md.dt, md.gamma, C.c_void_p(md.kT.data_ptr()), md.seed,
                                            C.c_void_p(md.forces.data_ptr()), C.c_void_p(md.com.data_ptr()),
                                            C.c_void_p(md.quat.data_ptr()), C.c_void_p(md.mom.data_ptr()),
                                            C.c_void_p(md.angmom.data_ptr()), C.c_void_p(md.pos.data_ptr()),
                                            C.c_void_p(md.box.data_ptr())))
        h_pos.copy_(md.pos, non_blocking=True)
        md.stream.synchronize()
        _lib.check(lib.pgm_compute_host(ff._h, C.c_void_p(h_pos.data_ptr()), C.c_void_p(h_box.data_ptr()),
                                        None if state_on_device and not load_state else C.byref(ind), C.byref(out)))
        md.forces.copy_(h_F, non_blocking=True)
        _lib.check(lib.pgm_rigid_end_step(md._h, st, md.dt, C.c_void_p(md.forces.data_ptr()), C.c_void_p(md.quat.data_ptr()),
                                          C.c_void_p(md.mom.data_ptr()), C.c_void_p(md.angmom.data_ptr())))

    with torch.cuda.stream(md.stream):
        # warm-up: the first call loads the MD's induction state (into the handle when it stays on
        # the device), then five more steps refresh the history with this leg's own steps
        for k in range(6):
            one(load_state=k == 0)
        md.stream.synchronize()
        builds0 = int(lib.pgm_list_rebuilds(ff._h))
        torch.cuda.nvtx.range_push("e2e_md")
        t0 = time.perf_counter()
        for _ in range(steps):
            one()
        md.stream.synchronize()
        ms = (time.perf_counter() - t0) * 1e3 / steps
        torch.cuda.nvtx.range_pop()
        rebuilds = (int(lib.pgm_list_rebuilds(ff._h)) - builds0) / steps
    b = 8 * n * 3
    st_b = 0 if state_on_device else 5 * b + 4 * S + 8 * S  # mu + hist, count, norm
    h2d = b + 9 * 8 * S + st_b + b  # positions, box, (state); forces back to the integrator
    d2h = b + b + st_b + 8 * (3 + 9 + 1) * S + 8 * S  # positions out of the integrator; forces, (state), energy, virial...
    what = ("the induction state kept on the device in the handle (ind = NULL)" if state_on_device
            else "the induction state copied in and out every call")
    return {"value": ns_per_day(ms), "unit": "ns/day", "ms_per_step": ms, "steps": steps, "list_rebuilds_per_step": rebuilds,
            "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h,
            "path": "pgm_compute_host (C ABI, pinned host buffers: positions in; forces, energies, virial out; " + what
            + ") with the rigid-body kernels on the GPU; wall clock around the loop"}


from ctypes import byref, c_double as C_double, c_void_p as C_void_p  # noqa: E402


# ----------------------------------------------------------------------------- other workloads
def batch_workload():
    """16 boxes of uneven sizes (4 each of 216 / 512 / 1000 / 2197 waters, edges 1.86 / 2.48 / 3.10 /
    4.04 nm, PME 32^3 / 48^3 / 64^3 / 72^3) at 298 K plus 32 REMD replicas of 512 waters (2.483 nm,
    48^3) on a geometric 280-400 K ladder, all in one engine."""
    from pgm_jax_b200.remd import geometric_ladder
    from pgm_jax_b200.systems import water_box

    boxes, grids, temps = [], [], []
    for k, (n, L, K) in enumerate([(6, 1.86, 32), (8, 2.48, 48), (10, 3.10, 64), (13, 4.04, 72)]):
        for r in range(4):
            boxes.append(water_box(n, L, seed=100 + 4 * k + r))
            grids.append((K, K, K))
            temps.append(TEMP)
    ladder = geometric_ladder(280.0, 400.0, 32)
    for r in range(32):
        boxes.append(water_box(8, 2.483, seed=200 + r))
        grids.append((48, 48, 48))
    temps += list(ladder)
    return boxes, grids, np.array(temps), ladder


def system_frame(md, k: int) -> dict:
    """Positions, box and induction state of system k of a batched MD (host arrays)."""
    md.stream.synchronize()
    o = md.ff.offsets
    sl = slice(int(o[k]), int(o[k + 1]))
    return {"pos": md.pos[sl].cpu().numpy(), "box": md.box[k].cpu().numpy(),
            "ind": {"mu": md.ind.mu[sl].cpu().numpy(), "hist": md.ind.hist[:, sl].cpu().numpy(),
                    "count": md.ind.count[k:k + 1].cpu().numpy(), "norm": md.ind.norm[k:k + 1].cpu().numpy()}}


def make_md(boxes, grids, temps, predictor, rank, torch, gamma=GAMMA):
    from pgm_jax_b200.forcefield import PGMForceField
    from pgm_jax_b200.md import RigidMD

    ff = PGMForceField([b[0] for b in boxes], [b[2] for b in boxes], settings(predictor=predictor), pme_grids=grids,
                       device=torch.cuda.current_device())
    md = RigidMD(ff, np.concatenate([b[1] for b in boxes]), np.stack([b[2] for b in boxes]), temperature=temps, dt_fs=DT_FS,
                 gamma_ps=gamma, seed=1 + rank)
    return ff, md


def run_workload(args) -> None:
    """--workload batch: the uneven boxes + REMD replicas in one launch, exchanges every 100 steps
    inside the timed region.  --workload npt: the 4,096-water MD with Monte Carlo volume moves.
    --workload pimd: 32 beads x 1,024 flexible waters."""
    import torch

    from pgm_jax_b200 import _lib
    from pgm_jax_b200.remd import ReplicaExchange, RigidReplicas
    from pgm_jax_b200.systems import water_box

    torch.cuda.set_device(0)
    line = {"metric": METRIC, "unit": "ns/day", "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
            "dtype": "f32+f64", "workload": args.workload}
    if args.workload == "batch":
        boxes, grids, temps, ladder = batch_workload()
        ff, md = make_md(boxes, grids, temps, "mu4", 0, torch)
        equilibrate(md, 500)
        rex = ReplicaExchange(RigidReplicas(md, systems=range(16, 48)), ladder, seed=1)
        md.step()
        md.capture()
        md.run(5)
        md.stream.synchronize()
        blocks = max(1, args.steps // 100)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        it_sum = torch.zeros(ff.nsys, dtype=torch.int64, device=ff.device)
        clk = Clocks(0)
        md.run(50)  # the GPU stays loaded while the sampler starts
        torch.cuda.synchronize()
        t_wall = time.time()
        ev0.record(md.stream)
        for _ in range(blocks):
            for _ in range(100):
                md.run(1)
                with torch.cuda.stream(md.stream):
                    it_sum += md.result.iterations.to(torch.int64)
            rex.exchange()  # host: energies of the replicas, Metropolis, temperatures, momenta
        ev1.record(md.stream)
        torch.cuda.synchronize()
        clk.mark(t_wall, time.time())
        clocks = clk.stop()
        steps = 100 * blocks
        ms = ev0.elapsed_time(ev1) / steps
        its = it_sum.cpu().numpy() / steps
        line.update({
            "value": ns_per_day(ms), "ms_per_step": ms, "steps": steps, "systems": ff.nsys, "atoms": ff.n,
            "system_ns_per_day": ns_per_day(ms) * ff.nsys, "atom_steps_per_s": ff.n * 1e3 / ms,
            "cg_iters_per_step_mean": float(its.mean()), "cg_iters_per_step_max": float(its.max()),
            "exchange_acceptance": rex.stats.neighbour_acceptance().tolist(), "exchanges": rex.stats.n_exchanges,
            "status_any": int(md.result.status.max()), "clocks": clocks, "row_capacity": ff.capacity,
            "accuracy_vs_oracle": accuracy_vs_oracle(boxes[12][0], system_frame(md, 12), torch, grid=72,
                                                     label="the final frame of the first 2197-water box (72^3)"),
            "config": {"workload": "4 x (216 @ 1.86 nm, 32^3; 512 @ 2.48 nm, 48^3; 1000 @ 3.10 nm, 64^3; 2197 @ 4.04 nm, "
                       "72^3) at 298 K + 32 x 512 waters REMD 280-400 K (geometric), one engine, mixed, CG 1e-6 from mu4, "
                       "Langevin 2/ps, dt 1 fs, exchanges every 100 steps (timed)", "equilibration": "500 steps at 20/ps"},
        })
    elif args.workload == "npt":
        from pgm_jax_b200.barostat import MonteCarloBarostat
        from pgm_jax_b200.forcefield import PGMForceField
        from pgm_jax_b200.md import RigidMD

        B = BOXES["water4096"]
        s, pos, H = water_box(B["n_side"], B["edge"], seed=0)
        ff = PGMForceField(s, H, settings(predictor="mu4", grid=B["grid"]), device=0)
        md = RigidMD(ff, pos, H, temperature=TEMP, dt_fs=DT_FS, gamma_ps=GAMMA, seed=1)
        equilibrate(md, B["equil_steps"])
        for _ in range(4):
            md.step()
        md.capture()
        baro = MonteCarloBarostat(md, pressure=1.0, every=100, seed=1)
        baro.run(400)  # warm-up: the step size adapts, the first moves are made
        md.stream.synchronize()
        V0 = float(baro.volumes()[0])
        tries0, acc0 = int(baro.total_tries[0]), int(baro.total_accepted[0])
        steps = max(200, (min(args.steps, 2000) // 100) * 100)
        clk = Clocks(0)
        md.run(50)  # the GPU stays loaded while the sampler starts
        torch.cuda.synchronize()
        # wall clock: the volume moves return to the host (the accept decision), so events on the
        # MD stream alone would miss the host's part
        t0 = time.perf_counter()
        baro.run(steps)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        clk.mark(t0, t1)
        clocks = clk.stop()
        ms = (t1 - t0) * 1e3 / steps
        line.update({
            "value": ns_per_day(ms), "ms_per_step": ms, "steps": steps, "clocks": clocks,
            "volume_moves": int(baro.total_tries[0]) - tries0, "accepted": int(baro.total_accepted[0]) - acc0,
            "volume_nm3": [V0, float(baro.volumes()[0])], "dv_nm3": float(baro.dv[0]),
            "status_any": int(md.ff._status.max()),
            "config": {"workload": "4096 rigid pGM3P-25 waters, NPT 1 bar / 298 K: the bench MD (mu4 start, mixed, CG 1e-6) "
                       "with an isotropic Monte Carlo volume move every 100 steps", "timing": "wall clock over the steps "
                       "and the moves (each move: one trial energy, and the forces again when accepted)"},
        })
    elif args.workload == "pimd":
        from pgm_jax_b200.forcefield import MDSettings
        from pgm_jax_b200.pimd import PIMD

        s, pos, H = water_box(11, 3.13, seed=0, n_water=1024)
        st = MDSettings(precision="mixed", cutoff=0.9, ewald_beta=4.0, pme_grid=(64, 64, 64), pme_order=6, dipole_tol=TOL,
                        max_iter=100, predictor="mu4")
        pm = PIMD(s, pos, H, st, beads=32, temperature=300.0, dt_fs=0.5, mode="pimd", seed=1)
        for _ in range(5):
            pm.step()
        pm.capture()
        pm.run(800)  # relaxation of the lattice start (captured steps)
        pm.stream.synchronize()
        steps = max(10, min(args.steps, 200))
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        it_sum = torch.zeros(32, dtype=torch.int64, device=pm.dev)
        clk = Clocks(0)
        pm.run(30)  # the GPU stays loaded while the sampler starts
        torch.cuda.synchronize()
        t_wall = time.time()
        ev0.record(pm.stream)
        for _ in range(steps):
            pm.run(1)
            with torch.cuda.stream(pm.stream):
                it_sum += pm.result.iterations.to(torch.int64)
        ev1.record(pm.stream)
        torch.cuda.synchronize()
        clk.mark(t_wall, time.time())
        clocks = clk.stop()
        ms = ev0.elapsed_time(ev1) / steps
        est = pm.estimators()
        bead0 = {"pos": pm.q[: pm.n].cpu().numpy(), "box": pm.box[0].cpu().numpy(),
                 "ind": {"mu": pm.ind.mu[: pm.n].cpu().numpy(), "hist": pm.ind.hist[:, : pm.n].cpu().numpy(),
                         "count": pm.ind.count[:1].cpu().numpy(), "norm": pm.ind.norm[:1].cpu().numpy()}}
        line["accuracy_vs_oracle"] = accuracy_vs_oracle(s, bead0, torch, grid=64, label="bead 0 of the final frame")
        line.update({
            "value": 86.4 * 0.5 / ms, "ms_per_step": ms, "steps": steps, "beads": 32, "atoms": 3072, "bead_atoms": 98304,
            "cg_iters_per_step_mean": float(it_sum.float().mean().item()) / steps, "clocks": clocks,
            "t_centroid_K": est["t_centroid"], "t_internal_modes_K": float(np.mean(est["t_modes"][1:])),
            "kinetic_prim_per_atom_kjmol": est["prim"] / 3072, "kinetic_cv_per_atom_kjmol": est["cv"] / 3072,
            "status_any": int(pm.result.status.max()),
            "config": {"workload": "PIMD 32 beads x 1024 flexible pGM waters (q-TIP4P/F intramolecular), 3.13 nm, PME 64^3 o6, "
                       "rc 0.9 nm, 300 K PILE-L (tau_centroid 0.2 ps), dt 0.5 fs, mixed, CG 1e-6 from mu4 per bead, "
                       "all beads in one engine", "equilibration": "805 steps from the lattice + free ring polymer start"},
        })
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-nn", dest="nn", action="store_false", help="plain mu4 CG only, without the learned guess")
    ap.add_argument("--model", default="mpnn", choices=["mpnn", "mlp"],
                    help="the learned guess of the headline: the 2-layer message-passing model (default) or the "
                    "per-atom MLP on the graph's features; the other one is measured beside it")
    ap.add_argument("--no-other-model", dest="other_model", action="store_false",
                    help="skip the MD with the other learned guess")
    ap.add_argument("--workload", default="water32768", choices=["water32768", "water4096", "batch", "pimd", "npt"],
                    help="water32768: the headline; water4096 the same line on the smaller box; the others print "
                    "their own line (one GPU)")
    ap.add_argument("--equil-steps", type=int, default=None,
                    help="relaxation steps of the lattice start before timing (default: the workload's)")
    ap.add_argument("--local-niter", type=int, default=1,
                    help="the reference's local preconditioner in every arm: inner CG iterations on the row entries "
                    "inside 0.3 nm (default 1; 0: Jacobi, the reference's default)")
    ap.add_argument("--elec-cutoff", type=float, default=None,
                    help="split rows: electrostatics cutoff [nm] below the 0.9 nm LJ cutoff (Ewald coefficient for it)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    MODEL[0] = args.model
    LOCAL["local_niter"] = args.local_niter
    if args.elec_cutoff:
        from pgm_jax_b200.forcefield import elec_cutoff_settings

        SPLIT.update(elec_cutoff_settings(args.elec_cutoff))
    if args.workload in BOXES:
        W.clear()
        W.update(BOXES[args.workload], name=args.workload)
        if args.equil_steps is not None:
            W["equil_steps"] = args.equil_steps
    if args.impl == "reference":
        run_reference(args)
    elif args.workload not in BOXES:
        run_workload(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
