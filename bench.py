"""Benchmark of the B200-native Boussinesq RBC step (one JSON line on rank 0).

Workload (the config the headline metric is quoted on that fits one GPU): plain FP64
step, 256 x 256 grid, Lx = Ly = 32, Nz = 8 Galerkin modes, Pr = 0.9, Ra = 5000,
dt = 5e-4, 65,536 passive tracers, seeded synthetic initial state (theta N(0, 1e-3^2)
on |k| <= 8 of the lowest mode, tracers uniform). A "step" is one IMEX step plus one
tracer advance. Timing: W untimed warm-up steps, then K steps bracketed by a barrier and
a synchronize, CUDA events on the solver's stream, max over ranks. N > 1 runs N
independent replicas (weak scaling; no collective on the data path).

--impl reference times the reference method's CPU implementation (the FP64 oracle
port, all host cores) on the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Sim-time/s per GPU: mixed/batched/surrogate vs plain FP64 at ≤1e-3 Nu error"
WORK = dict(nx=256, ny=256, nz=8, lx=32.0, ly=32.0, ra=5000.0, pr=0.9, dt=5e-4)
NTRACERS = 65536
SEED = 2
# the workload string both arms print (the same workload, so the lines are comparable)
WORKLOAD = ("plain FP64 RBC step 256x256x8, Lx=Ly=32, Ra=5000, Pr=0.9, dt=5e-4, Nz=8 Galerkin modes, "
            "+65536 tracers, 1000-2000-step run length sampled by the timed steps")


def bytes_alg(nx, ny, L, ntr):
    """Algorithmic bytes of one plain FP64 step (step + tracers)."""
    S = (nx // 2 + 1) * ny
    P = nx * ny
    step = L * (12 * S * 16 + 44 * P * 8) + 40 * L * L * S
    tr = 5 * L * P * 8 + 816 * ntr
    return step, tr


def contract_fmas_per_point(L):
    """FP64 FMAs of the Galerkin contraction per grid point: 20 units of L x ceil(L/2)
    coefficients per output mode and 38 edges of L + 1 FMAs, for each of the L modes."""
    return L * (20 * L * ((L + 1) // 2) + 38 * (L + 1))


def stage_bytes(nx, ny, L, ckeep, nkept, ntr):
    """Algorithmic bytes per launch of each kernel (read + write of its compulsory data)."""
    P = nx * ny
    C = 16  # complex double
    kept = nkept  # kept wavenumbers (c < ckeep, rows of the 2/3 rule)
    col = ckeep * ny
    return {
        "synth_columns": 3 * L * kept * C + 8 * L * col * C,
        "rows_c2r": 8 * L * col * C + 8 * L * P * 8,
        "tracers": 5 * L * P * 8 + 48 * ntr,
        "contract": 8 * L * P * 8 + 13 * L * P * 8,
        "rows_r2c": 13 * L * P * 8 + 13 * L * col * C,
        "columns_combine": 13 * L * col * C + 3 * L * col * C,
        # N, state and history read, state and history written, operator table rows (the
        # same-parity half of each row of the five L x L matrices)
        "update": kept * L * C * (3 + 3 + 3 + 3 + 3) + kept * 5 * L * ((L + 1) // 2) * 8,
    }


def dist_env():
    """(world, rank, local_rank) from the torchrun environment (1, 0, 0 without it)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(value, world, device=None):
    """The largest of every rank's `value` (all ranks get it); identity for one rank."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_value(world, steps, dt, ms_max):
    """Whole-job sim time per second: every replica advances `steps` steps of dt."""
    return world * steps * dt / (ms_max / 1000.0)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def profile_traffic(kernel):
    """DRAM bytes per launch from a committed ncu summary (profiles/traffic.json)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    v = d.get(kernel)
    return None if v is None else v.get("dram_bytes_per_launch")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, device):
        self.proc = None
        self.out = os.path.join("/tmp", f"rbc_clocks_{os.getpid()}.csv")
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.out, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # the timed region starts once the sampler has produced its first line
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < 5.0 and self.proc.poll() is None:
            self.f.flush()
            if os.path.getsize(self.out) > 0:
                break
            time.sleep(0.05)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.out) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        os.unlink(self.out)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(steps_hint):
    """Oracle port on the host cores: bounded sample of the same workload."""
    import oracle
    threads = os.cpu_count() or 1
    o = oracle.Oracle(WORK["nx"], WORK["ny"], WORK["nz"], WORK["lx"], WORK["ly"], WORK["ra"], WORK["pr"],
                      WORK["dt"], threads=threads)
    o.init_theta(SEED, 1e-3, 8.0)
    o.tracers_set(oracle.tracer_positions(SEED, NTRACERS, WORK["lx"], WORK["ly"]))
    t = time.perf_counter()
    o.step(1)
    first = time.perf_counter() - t
    n = max(2, min(steps_hint, int(20.0 / max(first, 1e-3))))
    t = time.perf_counter()
    o.step(n)
    el = time.perf_counter() - t
    return {"value": n * WORK["dt"] / el, "unit": "sim-time/s", "cores": threads, "kind": "port",
            "sample": f"{n} oracle steps (after 1 warm-up) of the 256x256x8 + 65536-tracer workload, "
                      f"{el / n:.3f} s/step", "steps_per_s": n / el}


def run_reference(args, rank):
    if rank != 0:
        return
    import oracle  # noqa: F401  (checker library; the reference method's CPU port)
    cb = cpu_baseline(args.steps)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "sim-time/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 / cb["steps_per_s"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "form": "fp64", "impl": "oracle port of the reference method"},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": "sim-time/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def mixed_form(s64, stream, args, local, world, form="mixed"):
    """Mixed form (FP32 synthesis, products and FFTs; FP64 implicit solve and reductions),
    or the collocation form (form="colloc": the same, with the nonlinear products on 2 Nz
    Gauss-Legendre levels and the mode -> level products on the tensor cores), on the same
    workload: sim-time/s over the same timed step count from the given state, and the
    relative error of Nu_wall, Nu_vol and KE against the FP64 form after 2000 steps from that
    state (equal sim time)."""
    import torch
    import sdc_b200
    state = s64.get_state()
    tr = s64.tracers_get()
    m = sdc_b200.Solver(**WORK, form=form, n_tracers=NTRACERS, device=local, tune=bool(args.tune))
    m.set_stream(stream.cuda_stream)
    m.set_state(*state)
    m.tracers_set(tr)
    m.step(args.warmup)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    m.step_async(args.steps)
    e1.record(stream)
    m.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world, device="cuda")
    value = weak_scaling_value(world, args.steps, WORK["dt"], ms)
    # accuracy at equal sim time
    n_cmp = 2000
    for sv in (s64, m):
        sv.set_state(*state)
        sv.tracers_set(tr)
        sv.step(n_cmp)
    d64, dm = s64.diagnostics(), m.diagnostics()
    err = {k: abs(dm[k] - d64[k]) / abs(d64[k]) for k in ("nu_wall", "nu_vol", "ke")}
    m.close()
    dtype = ("f32 synthesis/products/FFTs + f64 implicit solve, mean flow, diagnostics" if form == "mixed" else
             "f32 FFTs; mode -> level products tcgen05 kind::tf32 with split operands (3xTF32), level products and "
             "level -> mode sums f32 on 2 Nz Gauss-Legendre levels; f64 implicit solve, mean flow, diagnostics")
    return {"value": value, "unit": "sim-time/s", "ms_per_step": ms / args.steps, "dtype": dtype,
            "rel_err_vs_fp64": err, "compared_after_steps": n_cmp,
            "fp64_nu_wall": d64["nu_wall"], "nu_err_le_1e-3": bool(err["nu_wall"] <= 1e-3)}


SDC = dict(nx=512, ny=512, nz=12, lx=64.0, ly=64.0, ra=6000.0, pr=1.0, dt=2.5e-4)
# the surrogate's spectrum judge: relative L2 error of the z = 0 theta spectrum over 32
# shells, against the plain step's, above which the plain step takes over
SPEC_TOL = 0.05


def mixed_sdc_form(stream, local, steps=4000):
    """The mixed-precision configuration: 512 x 512 grid, Lx = Ly = 64, Nz = 12, Ra = 6000,
    Pr = 1, dt = 2.5e-4, 4000 steps from the seeded perturbation (seed 3, |k| <= 8). The
    mixed form (FP32 synthesis, products and transforms; FP64 implicit solve, mean flow and
    reductions) and the FP64 form run the same steps from the same state; reported: both
    forms' sim-time/s (CUDA events) and the error of Nu (wall and volume), kinetic energy
    and the radial spectrum of theta at z = 0 against the FP64 run."""
    import numpy as np
    import torch
    import sdc_b200
    res = {}
    diag = {}
    for form in ("fp64", "mixed", "colloc"):
        s = sdc_b200.Solver(**SDC, form=form, device=local, tune=True)
        s.set_stream(stream.cuda_stream)
        s.init_fields(3, 1e-3, 8.0)
        s.step(3)
        s.init_fields(3, 1e-3, 8.0)  # warm-up steps discarded: both forms start from the seed
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.step_async(steps)
        e1.record(stream)
        s.synchronize()
        ms = e0.elapsed_time(e1)
        res[form] = {"sim_time_per_s": steps * SDC["dt"] / (ms * 1e-3), "ms_per_step": ms / steps}
        d = s.diagnostics()
        diag[form] = (d, s.spectrum(64, 0.0))
        s.close()
    d64, sp64 = diag["fp64"]

    def errors(form):
        dm, spm = diag[form]
        err = {k: abs(dm[k] - d64[k]) / abs(d64[k]) for k in ("nu_wall", "nu_vol", "ke")}
        err["spectrum_rel_l2"] = float(np.linalg.norm(spm - sp64) / np.linalg.norm(sp64))
        return err

    err = errors("mixed")
    cerr = errors("colloc")
    return {"config": "512x512x12, Lx=Ly=64, Ra=6000, Pr=1, dt=2.5e-4, %d steps, seed 3 |k|<=8" % steps,
            "value": res["mixed"]["sim_time_per_s"], "unit": "sim-time/s",
            "fp64_value": res["fp64"]["sim_time_per_s"],
            "speedup_vs_fp64": res["mixed"]["sim_time_per_s"] / res["fp64"]["sim_time_per_s"],
            "ms_per_step": res["mixed"]["ms_per_step"], "fp64_ms_per_step": res["fp64"]["ms_per_step"],
            "rel_err_vs_fp64": err, "fp64_nu_wall": d64["nu_wall"], "fp64_ke": d64["ke"],
            "nu_err_le_1e-3": bool(err["nu_wall"] <= 1e-3),
            "dtype": "f32 synthesis/products/FFTs + f64 implicit solve, mean flow, diagnostics",
            "colloc": {"value": res["colloc"]["sim_time_per_s"], "ms_per_step": res["colloc"]["ms_per_step"],
                       "speedup_vs_fp64": res["colloc"]["sim_time_per_s"] / res["fp64"]["sim_time_per_s"],
                       "levels": 24, "rel_err_vs_fp64": cerr, "nu_err_le_1e-3": bool(cerr["nu_wall"] <= 1e-3),
                       "dtype": "mode -> level products on tcgen05 (kind::tf32, split operands), FP32 level "
                                "products and sums, FP64 implicit solve"}}


def optional_physics_forms(s64, stream, local, steps=2000):
    """The reference's optional physics on the same workload and state: the penalized
    operator (PENALIZED build, circle mask, eta = 0.01) as plain steps, and the iteration
    loop with the freeze (circle 0.8) and the heating (frame 0.1, +1.5/100) before every
    step, as main.cu:569-616 runs them. ms per iteration against the plain step."""
    import torch
    import sdc_b200
    state = s64.get_state()
    tr = s64.tracers_get()
    out = {}

    def timed(run):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        run()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    s64.set_state(*state)
    s64.tracers_set(tr)
    s64.step(10)
    plain = timed(lambda: s64.step_async(steps))
    p = sdc_b200.Solver(**WORK, n_tracers=NTRACERS, device=local, penalization=(0.01, "circle"))
    p.set_stream(stream.cuda_stream)
    p.set_state(*state)
    p.tracers_set(tr)
    p.step(10)
    pen = timed(lambda: p.step_async(steps))
    dp = p.diagnostics()
    p.close()
    out["penalized"] = {"ms_per_step": pen, "plain_ms_per_step": plain, "overhead": pen / plain - 1.0,
                        "mask": "circle", "eta": 0.01, "nu_wall_after": dp["nu_wall"], "steps": steps}
    f = sdc_b200.Solver(**WORK, n_tracers=NTRACERS, device=local, field_ops=("freeze", "heat"))
    f.set_stream(stream.cuda_stream)
    f.set_state(*state)
    f.tracers_set(tr)
    f.step(10)
    f.freeze_mask("circle", 0.8)
    f.heat_mask("rectangle", 0.1, 1.5 / 100)

    def loop():
        for _ in range(steps):
            f.freeze_apply()
            f.heat_apply()
            f.step_async(1)

    it = timed(loop)
    df = f.diagnostics()
    f.close()
    out["freeze_heat"] = {"ms_per_iteration": it, "plain_ms_per_step": plain, "overhead": it / plain - 1.0,
                          "freeze": "circle 0.8", "heat": "frame 0.1, +0.015", "nu_wall_after": df["nu_wall"],
                          "steps": steps}
    return out


# Learned surrogate (the fourth form): Fourier neural operator on (theta, u, v, w) at
# 12 Gauss-Legendre levels of the 128 x 128 x 6 grid (Lx = Ly = 16), one surrogate
# interval = 40 plain steps of dt = 5e-4 (0.02 time units).
SURR = dict(nx=128, ny=128, nz=6, lx=16.0, ly=16.0, pr=1.0, dt=5e-4)
SURR_NET = dict(nq=12, width=32, modes=16, layers=4, hidden=128)
SURR_INTERVAL = 40
# The same surrogate on the plain step's own 256 x 256 x 8 grid (Lx = Ly = 32, Pr = 0.9,
# rollout at its Ra = 5000; without tracers): 16 collocation levels, fewer runs.
SURR_C2 = dict(nx=256, ny=256, nz=8, lx=32.0, ly=32.0, pr=0.9, dt=5e-4)
SURR_C2_NET = dict(nq=16, width=32, modes=16, layers=4, hidden=128)


def nu_wall_of(state):
    """Nu_wall = 1 - sum_k (k+1) pi Re theta_k(q = 0) of a host state."""
    import numpy as np
    th = state[0]
    return 1.0 - sum((k + 1) * np.pi * th[k, 0, 0].real for k in range(th.shape[0]))


def spun_up_states(ras, seeds, local, t_spin=10.0, dt_spin=1e-3, c=SURR):
    """States of the surrogate grid c after t_spin time units from seeded perturbations, one
    per (Ra, seed), advanced together as one ensemble (concurrent CUDA-graph branches)."""
    import sdc_b200
    cfg = [(c["nx"], c["ny"], c["nz"], c["lx"], c["ly"], float(ra), c["pr"], dt_spin) for ra in ras]
    e = sdc_b200.Ensemble(cfg, nstreams=16, device=local)
    for m, sd in zip(e.members, seeds):
        m.init_fields(int(sd), 1e-2, 8.0)
    e.step(int(round(t_spin / dt_spin)))
    out = [m.get_state() for m in e.members]
    e.close()
    return out


def snapshot_pairs(f, ras, starts, nsnap, local, slot0=0, c=SURR):
    """Captures nsnap snapshots, SURR_INTERVAL plain steps apart, of one run per (Ra, start
    state) on grid c into the surrogate's store from slot0 on; the runs advance together
    as one ensemble. Returns the (src, dst) slot pairs of consecutive snapshots."""
    import sdc_b200
    cfg = [(c["nx"], c["ny"], c["nz"], c["lx"], c["ly"], float(ra), c["pr"], c["dt"]) for ra in ras]
    e = sdc_b200.Ensemble(cfg, nstreams=16, device=local)
    for m, st in zip(e.members, starts):
        m.set_state(*st)
    src, dst = [], []
    n = len(ras)
    for k in range(nsnap):
        for j, m in enumerate(e.members):
            f.capture(m, slot0 + k * n + j)
            if k:
                src.append(slot0 + (k - 1) * n + j)
                dst.append(slot0 + k * n + j)
        if k + 1 < nsnap:
            e.step(SURR_INTERVAL)
    e.close()
    return src, dst


def surrogate_form(local, epochs=80, ntraj=50, nsnap=41, n_intervals=200, judge_every=10, augment=2,
                   noise_rel=0.0, physics_mean=True, c=SURR, net=SURR_NET, batch=16, ra=4500.0):
    """Trains the surrogate on ntraj * (nsnap - 1) snapshot pairs of the plain solver on
    grid c at Ra ~ U[2500, 6000] (runs spun up for 10 time units from seeded perturbations),
    then times a rollout at Ra = ra from a held-out state: the surrogate with the plain
    step judging every judge_every-th interval (Nu_wall tolerance 1e-3) against the plain
    step alone over the same sim time."""
    import numpy as np
    import torch
    import sdc_b200
    f = sdc_b200.FNO(c["nx"], c["ny"], c["nz"], max_batch=batch, device=local, seed=7, interval_steps=SURR_INTERVAL,
                     physics_mean=physics_mean, **net)
    f.reserve(ntraj * nsnap)
    ras = np.random.default_rng(11).uniform(2500.0, 6000.0, ntraj)
    t0 = time.perf_counter()
    starts = spun_up_states(ras, 100 + np.arange(ntraj), local, c=c)
    src, dst = snapshot_pairs(f, ras, starts, nsnap, local, c=c)
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    f.set_train_options(augment=augment if c["nx"] == c["ny"] and c["lx"] == c["ly"] else min(augment, 1),
                        noise_rel=noise_rel)
    losses = f.train(src, dst, epochs=epochs, batch=batch, lr=1e-3, seed=3)
    train_s = time.perf_counter() - t0

    st0 = spun_up_states([ra], [999], local, c=c)[0]
    stream = torch.cuda.Stream()
    nsteps = n_intervals * SURR_INTERVAL
    mk = lambda: sdc_b200.Solver(c["nx"], c["ny"], c["nz"], c["lx"], c["ly"], ra, c["pr"], c["dt"], device=local,
                                 diag_capacity=nsteps + 16)
    plain = mk()
    plain.set_stream(stream.cuda_stream)
    plain.set_state(*st0)
    plain.step(SURR_INTERVAL)  # warm-up (graph capture)
    plain.set_state(*st0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    plain.step_async(nsteps)
    e1.record(stream)
    plain.synchronize()
    ms_plain = e0.elapsed_time(e1)
    hist = plain.diag_history(nsteps)
    nu_plain_trace = hist[-nsteps:, 0][SURR_INTERVAL - 1::SURR_INTERVAL]
    nu_plain = float(nu_plain_trace[-1])
    sim_t = nsteps * c["dt"]

    def rollout(model):
        s = mk()
        s.set_stream(stream.cuda_stream)
        s.set_state(*st0)
        rep = model.run(s, intervals=n_intervals, judge_every=judge_every,
                        nu_tol=1e-3, spec_tol=SPEC_TOL, spec_bins=32, fallback_intervals=judge_every, trace=True)
        s.close()
        tr = rep.pop("nu_trace")
        rep["nu_wall"] = float(tr[-1])
        rep["nu_err_vs_plain"] = float(abs(tr[-1] - nu_plain) / abs(nu_plain))
        rep["nu_mean_err_vs_plain"] = float(abs(tr.mean() - nu_plain_trace.mean()) / abs(nu_plain_trace.mean()))
        rep["nu_trace_max_err_vs_plain"] = float(np.max(np.abs(tr - nu_plain_trace)) / abs(nu_plain_trace.mean()))
        rep["sim_time_per_s"] = sim_t / (rep["ms"] * 1e-3)
        return rep

    rollout(f)  # warm-up
    rep = rollout(f)
    # one-interval accuracy on held-out states of this run (collocation-field error of the
    # prediction relative to the true increment; persistence scores 1)
    s = mk()
    s.set_state(*st0)
    num = den = 0.0
    for i in range(10):
        s.step(SURR_INTERVAL * 5)
        x0 = s.get_state()
        c0 = f.colloc_get(s)
        s.step(SURR_INTERVAL)
        c1 = f.colloc_get(s)
        x1 = s.get_state()
        s.set_state(*x0)
        f.advance(s, 1)
        cp = f.colloc_get(s)
        num += float(np.sum((cp - c1) ** 2))
        den += float(np.sum((c1 - c0) ** 2))
        s.set_state(*x1)
    s.close()
    one_interval_err = (num / den) ** 0.5
    # the same rollout without the learned part: zero increment from the network (the
    # fluctuations persist), mean modes still advanced by the plain recursion
    g = sdc_b200.FNO(c["nx"], c["ny"], c["nz"], max_batch=1, device=local, seed=7, interval_steps=SURR_INTERVAL,
                     physics_mean=physics_mean, **net)
    g.set_params(np.zeros(g.num_params, np.float32))
    C = g.C
    g.set_norm(np.stack([np.zeros(C), np.ones(C), np.zeros(C), np.ones(C)]).astype(np.float32))
    rep0 = rollout(g)
    g.close()
    plain.close()
    f.close()
    return {"config": "FNO %d layers x width %d, %d modes, (theta,u,v,w) at %d levels of %dx%dx%d, "
                      "Lx=Ly=%g, Pr=%g; interval 40 steps of dt=%g; %d pairs from %d runs at Ra U[2500,6000]; "
                      "rollout Ra=%g without tracers, judge every %d intervals (Nu tol 1e-3, fallback %d "
                      "intervals)" % (net["layers"], net["width"], net["modes"], net["nq"], c["nx"], c["ny"],
                                      c["nz"], c["lx"], c["pr"], c["dt"], len(src), ntraj, ra, judge_every,
                                      judge_every),
            "value": rep["sim_time_per_s"], "unit": "sim-time/s",
            "plain_value": sim_t / (ms_plain * 1e-3), "speedup_vs_plain": ms_plain / rep["ms"],
            "sim_time": sim_t, "nu_wall_plain": nu_plain, "nu_err_vs_plain": rep["nu_err_vs_plain"],
            "nu_mean_err_vs_plain": rep["nu_mean_err_vs_plain"],
            "nu_mean_err_le_1e-3": bool(rep["nu_mean_err_vs_plain"] <= 1e-3), "report": rep,
            "one_interval_err_vs_increment": one_interval_err, "zero_increment_report": rep0,
            "train": {"pairs": len(src), "runs": ntraj, "epochs": epochs, "batch": batch, "augment": augment,
                      "noise_rel": noise_rel, "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
                      "seconds": train_s, "data_seconds": gen_s},
            "dtype": "bf16 GEMMs, f32 accumulate/loss/Adam; f64 state and judge"}


def profile_surrogate(local):
    """Small surrogate workload for kernel profiling, on the C5 network and grid. First the
    inference kernels, driven directly rather than from the rollout's CUDA graph so that a
    profiler sees every launch: the collocation encode, 3 batch-1 network passes, and the
    decode of an increment into the state. Then 32 snapshot pairs of one run and 2
    training epochs (batch 16)."""
    import numpy as np
    import sdc_b200
    c = SURR
    s = sdc_b200.Solver(c["nx"], c["ny"], c["nz"], c["lx"], c["ly"], 4500.0, c["pr"], c["dt"], device=local)
    s.init_fields(3, 1e-2, 8.0)
    s.step(400)
    f = sdc_b200.FNO(c["nx"], c["ny"], c["nz"], max_batch=16, device=local, seed=7, interval_steps=SURR_INTERVAL,
                     **SURR_NET)
    x = f.colloc_get(s)
    for _ in range(3):
        y = f.forward(x[None])
    f.colloc_add(s, 1e-3 * y[0])
    f.reserve(33)
    for k in range(33):
        f.capture(s, k)
        s.step(SURR_INTERVAL)
    f.set_train_options(2, 0.0)
    f.train(np.arange(32), np.arange(1, 33), epochs=2, batch=16, lr=1e-3)
    f.advance(s, 3)
    print(json.dumps({"profile_surrogate": "done", "nu_wall": s.diagnostics()["nu_wall"]}))


def profile_field_ops(local, iters=5):
    """Small workload for kernel profiling of the optional physics on the plain step's
    256 x 256 x 8 grid without tracers: `iters` iterations of freeze (circle 0.8) + heating
    (frame 0.1) + one step, then `iters` penalized nonlinear operators (circle mask,
    eta = 0.01; the standalone operator launches its kernels outside CUDA graphs)."""
    import sdc_b200
    s = sdc_b200.Solver(**WORK, device=local, field_ops=("freeze", "heat"))
    s.init_fields(SEED, 1e-3, 8.0)
    s.step(20)
    s.freeze_mask("circle", 0.8)
    s.heat_mask("rectangle", 0.1, 1.5 / 100)
    for _ in range(iters):
        s.freeze_apply()
        s.heat_apply()
        s.step(1)
    p = sdc_b200.Solver(**WORK, device=local, penalization=(0.01, "circle"))
    state = s.get_state()
    for _ in range(iters):
        n = p.nonlinear(*state)
    print(json.dumps({"profile_field_ops": "done", "nu_wall": s.diagnostics()["nu_wall"],
                      "n_theta_00": abs(n[0][0, 0, 0])}))


def profile_diagnostics(local, iters=3):
    """Small workload for kernel profiling of the diagnostics and loop extras on the plain
    step's 256 x 256 x 8 grid without tracers: `iters` radial spectra of theta at z = 0 (64
    shells), structure functions of theta and u_1 along x (32 displacements each), and steps
    with the mean-flow forcing (-mean_F 0.01, one forcing kernel per step)."""
    import sdc_b200
    s = sdc_b200.Solver(**WORK, device=local, mean_F=0.01)
    s.init_fields(SEED, 1e-3, 8.0)
    s.step(5)
    for _ in range(iters):
        sp = s.spectrum(64, 0.0)
        s.structure_function("theta", "x", 0.1, 8.0, 32)
        s.structure_function("u1", "x", 0.1, 8.0, 32)
        s.step(1)
    print(json.dumps({"profile_diagnostics": "done", "spectrum_0": float(sp[0]),
                      "nu_wall": s.diagnostics()["nu_wall"]}))


def profile_sdc(local, form="mixed", steps=6):
    """Small workload for kernel profiling on the spiral-defect-chaos grid (512 x 512 x 12,
    Lx = Ly = 64, Ra 6000, Pr 1, dt 2.5e-4): `steps` steps of the given form from the seeded
    state (its transforms run on the Stockham kernels: 512 has no two-pass form)."""
    import sdc_b200
    s = sdc_b200.Solver(**SDC, form=form, device=local, tune=True)
    s.init_fields(3, 1e-3, 8.0)
    s.step(steps)
    print(json.dumps({"profile_sdc": form, "nu_wall": s.diagnostics()["nu_wall"],
                      "stages_us": {k: round(v[0] * 1000, 1) for k, v in s.stage_times(10).items()}}))


def profile_stockham(local, steps=6):
    """Small workload for kernel profiling of the shared-memory Stockham FFT kernels (the
    lengths without a register form): `steps` FP64 steps of a 384 x 384 x 8 grid (Lx = Ly = 48,
    Ra 5000, Pr 0.9, dt 5e-4) from a seeded state, launch tiling not autotuned."""
    import sdc_b200
    s = sdc_b200.Solver(384, 384, 8, 48.0, 48.0, 5000.0, 0.9, 5e-4, device=local, tune=False)
    s.init_fields(3, 1e-3, 8.0)
    s.step(steps)
    print(json.dumps({"profile_stockham": "384x384x8", "nu_wall": s.diagnostics()["nu_wall"],
                      "stages_us": {k: round(v[0] * 1000, 1) for k, v in s.stage_times(10).items()}}))


def ensemble_configs(n=64, seed=4):
    """The uneven ensemble: per member a grid from {64, 128, 192, 256}^2, Nz from {4, 6, 8},
    Ra ~ U[2000, 8000], Pr from {0.7, 1, 7}, Lx = Ly = grid / 8, dt = 5e-4 (drawn by seed)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        g = int(rng.choice([64, 128, 192, 256]))
        out.append((g, g, int(rng.choice([4, 6, 8])), g / 8.0, g / 8.0, float(rng.uniform(2000.0, 8000.0)),
                    float(rng.choice([0.7, 1.0, 7.0])), 5e-4))
    return out


def batched_form(local, steps=1000, n=64):
    """64 uneven runs advanced together (one CUDA graph per step: each member's step
    kernels as concurrent branches, members balanced over 32 streams) against the same
    runs advanced one after another with the plain step; results are compared. Both are
    timed with CUDA events on the stream the work ends on (the ensemble's root stream, each
    solver's stream), synchronized on both sides."""
    import numpy as np
    import torch
    import sdc_b200
    cfg = ensemble_configs(n)
    dt = 5e-4
    e = sdc_b200.Ensemble(cfg, nstreams=32, device=local, tune=True)
    for i, m in enumerate(e.members):
        m.init_fields(100 + i, 1e-3, 8.0)
    e.step(3)
    torch.cuda.synchronize()
    t_ens = e.timed_step(steps) * 1e-3
    nu_ens = [m.diagnostics()["nu_wall"] for m in e.members]
    e.close()
    t_seq = 0.0
    nu_seq = []
    for i, c in enumerate(cfg):
        s = sdc_b200.Solver(*c, device=local, tune=True)
        s.init_fields(100 + i, 1e-3, 8.0)
        stream = torch.cuda.Stream()
        s.set_stream(stream.cuda_stream)
        s.step(3)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.step_async(steps)
        e1.record(stream)
        s.synchronize()
        t_seq += e0.elapsed_time(e1) * 1e-3
        nu_seq.append(s.diagnostics()["nu_wall"])
        s.close()
    same = bool(np.array_equal(np.array(nu_ens), np.array(nu_seq)))
    return {"config": "%d runs: grids {64,128,192,256}^2, Nz {4,6,8}, Ra U[2000,8000], Pr {0.7,1,7}, "
                      "Lx=Ly=grid/8, dt=5e-4, %d steps each (seeded draw)" % (n, steps),
            "value": n * steps * dt / t_ens, "unit": "sim-time/s (aggregate)",
            "sequential_value": n * steps * dt / t_seq, "speedup_vs_sequential": t_seq / t_ens,
            "seconds": t_ens, "sequential_seconds": t_seq, "nu_identical_to_sequential": same,
            "timing": "CUDA events: the ensemble's root stream around rbc_ensemble_step, each solver's stream "
                      "around its queued steps",
            "dtype": "f64"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--form", default="fp64", choices=["fp64", "mixed", "colloc"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tune", type=int, default=1, help="1: autotune the FFT launch tiling at creation")
    ap.add_argument("--no-forms", action="store_true", help="skip the mixed-form and surrogate legs")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the surrogate leg")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-ensemble leg")
    ap.add_argument("--surrogate-epochs", type=int, default=80)
    ap.add_argument("--profile-surrogate", action="store_true",
                    help="run only a small surrogate workload (for kernel profiling) and exit")
    ap.add_argument("--profile-field-ops", action="store_true",
                    help="run only a small freeze/heating/penalization workload (for kernel profiling) and exit")
    ap.add_argument("--profile-diagnostics", action="store_true",
                    help="run only a small spectrum/structure-function/mean-forcing workload (for kernel profiling) and exit")
    ap.add_argument("--profile-stockham", action="store_true",
                    help="run only a few FP64 steps on a 384x384x8 grid (Stockham FFT kernels, for kernel profiling) and exit")
    ap.add_argument("--profile-sdc", default=None, choices=["fp64", "mixed", "colloc"],
                    help="run only a few steps of the given form on the 512x512x12 grid (for kernel profiling) and exit")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.profile_surrogate:
        profile_surrogate(int(os.environ.get("LOCAL_RANK", "0")))
        return
    if args.profile_field_ops:
        profile_field_ops(int(os.environ.get("LOCAL_RANK", "0")))
        return
    if args.profile_diagnostics:
        profile_diagnostics(int(os.environ.get("LOCAL_RANK", "0")))
        return
    if args.profile_stockham:
        profile_stockham(int(os.environ.get("LOCAL_RANK", "0")))
        return
    if args.profile_sdc:
        profile_sdc(int(os.environ.get("LOCAL_RANK", "0")), form=args.profile_sdc)
        return

    world, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    import numpy as np
    import sdc_b200

    s = sdc_b200.Solver(**WORK, form=args.form, n_tracers=NTRACERS, device=local, tune=bool(args.tune))
    W, NP = s.launch_config
    # one dedicated stream for the library and the timing events
    stream = torch.cuda.Stream()
    s.set_stream(stream.cuda_stream)
    s.init_fields(SEED, 1e-3, 8.0)
    s.tracers_seed(SEED)
    s.step(args.warmup)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident throughput
    clk = ClockSampler(local)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.step_async(args.steps)
    e1.record(stream)
    s.synchronize()
    launches = s.kernel_launches
    barrier()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, world, device="cuda")
    value = weak_scaling_value(world, args.steps, WORK["dt"], ms_max)

    # ---- per-kernel timing (roofline of the dominant kernel)
    stages = s.stage_times(max(5, min(50, args.steps // 10)))
    nx, ny, L = WORK["nx"], WORK["ny"], WORK["nz"]
    mox = nx // 2 + 1
    ck = 0
    while ck < mox and not (mox - ck <= (1.0 / 3.0) * mox):
        ck += 1
    nrow = sum(1 for r in range(ny) if not (abs(0.5 * ny - r) <= (1.0 / 3.0) * 0.5 * ny))
    sb = stage_bytes(nx, ny, L, ck, ck * nrow, NTRACERS)
    per_step = {k: v[0] * v[1] for k, v in stages.items()}
    dom = max(per_step, key=per_step.get)
    peak, peak_kind = measured_peaks()
    ach = sb[dom] / (stages[dom][0] * 1e-3) / 1e9
    roof = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
            "frac": ach / peak, "traffic": profile_traffic(dom), "peak_source": peak_kind,
            "alg_bytes_per_launch": sb[dom], "ms_per_launch": stages[dom][0],
            "stages_ms": {k: round(v[0], 5) for k, v in stages.items()}}
    if dom == "contract" and args.form == "fp64":
        # the contraction is bound by the FP64 FMA pipe: its FLOP rate against the FP64
        # FMA throughput measured on this device (no FP64 figure in the measured peaks)
        flops = 2.0 * contract_fmas_per_point(L) * nx * ny
        fp64_peak = sdc_b200.fp64_peak_tflops(local)
        hbm = {k: roof.pop(k) for k in ("achieved", "peak", "unit", "frac", "peak_source")}
        tf = flops / (stages[dom][0] * 1e-3) / 1e12
        roof.update({"bound": "fp64", "achieved": tf, "peak": fp64_peak, "unit": "TFLOP/s",
                     "frac": tf / fp64_peak, "flops_per_launch": flops,
                     "peak_source": "measured on this device (FP64 FMA loop; no FP64 figure in the measured peaks)",
                     "hbm": hbm})
    step_b, tr_b = bytes_alg(nx, ny, L, NTRACERS)

    # ---- end to end through the C ABI with host buffers (pinned, as a caller that streams
    # states in and out would hold them)
    pins = []

    def pinned(a):
        t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
        pins.append(t)
        v = t.numpy().view(a.dtype).reshape(a.shape)
        v[...] = a
        return v

    host_state = [pinned(a) for a in s.get_state()]
    host_tr = pinned(s.tracers_get())
    out_state = [pinned(a) for a in host_state]
    out_tr = pinned(host_tr)
    barrier()
    t0 = time.perf_counter()
    s.set_state(*host_state)
    s.tracers_set(host_tr)
    # steps are enqueued in chunks of 8 (the library's multi-step graph), the newest
    # diagnostics of each chunk read back while the next chunk is already queued, and at
    # the end every step's Nu_wall, Nu_vol and KE from the diagnostics ring
    prev = None
    done = nchunks = 0
    while done < args.steps:
        n = 8 if args.steps - done >= 8 else 1
        s.step_async(n)
        done += n
        nchunks += 1
        t = s.diagnostics_async()
        if prev is not None:
            s.diagnostics_get(prev)  # waits for that chunk only; reports a non-finite state
        prev = t
    s.diagnostics_get(prev)
    hist = s.diag_history(args.steps)
    s.get_state(out_state)
    s.tracers_get(out_tr)
    el = max_over_ranks(time.perf_counter() - t0, world, device="cuda")
    assert hist.shape[0] == args.steps and np.all(np.isfinite(hist))
    state_bytes = sum(a.nbytes for a in host_state)
    tr_bytes = host_tr.nbytes
    e2e = {"value": world * args.steps * WORK["dt"] / el, "unit": "sim-time/s",
           "h2d_bytes_per_step": (state_bytes + tr_bytes) / args.steps,
           "d2h_bytes_per_step": (state_bytes + tr_bytes + 36 * nchunks + 32 * args.steps) / args.steps,
           "host_buffers": "pinned (cudaHostAlloc through torch)",
           "includes": "set_state + tracers_set, rbc_step_async in chunks of 8 steps (1 for the rest) each "
                       "followed by rbc_diagnostics_async and rbc_diagnostics_get of the chunk before, "
                       "rbc_diag_history of every step, get_state + tracers_get"}
    d = s.diagnostics()
    assert np.isfinite(d["ke"]) and np.all(np.isfinite(out_tr)) and all(np.all(np.isfinite(a)) for a in out_state)

    # ---- the mixed form on the same workload (the first form): throughput from the
    # convective FP64 state reached above, and its diagnostics error against the FP64 form
    # over the same 2000 steps from that state
    forms = None
    if args.form == "fp64" and not args.no_forms and world == 1:
        forms = {"mixed": mixed_form(s, stream, args, local, world),
                 "colloc": mixed_form(s, stream, args, local, world, form="colloc"),
                 "mixed_512x512x12": mixed_sdc_form(stream, local)}
        forms.update(optional_physics_forms(s, stream, local))
        if not args.no_batched:
            forms["batched"] = batched_form(local)
        if not args.no_surrogate:
            forms["surrogate"] = surrogate_form(local, epochs=args.surrogate_epochs)
            forms["surrogate_256x256x8"] = surrogate_form(local, epochs=60, ntraj=20, nsnap=41, c=SURR_C2,
                                                          net=SURR_C2_NET, batch=8, ra=WORK["ra"])

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(8)
        cb = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "sim-time/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "steps_per_s": 1000.0 * args.steps / ms_max, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if args.form == "fp64" else "f32+f64", "data": "synthetic",
                "config": {"workload": WORKLOAD if args.form == "fp64" else WORKLOAD.replace("FP64", args.form.upper()),
                           "form": args.form, "parallelism": f"replicas x{world}",
                           "launch": {"autotuned": bool(args.tune), "column_block": W, "row_pairs": NP},
                           "l2": "working set > 126 MB L2 (state, history, scratch ~300 MB); no flush",
                           "alg_bytes_per_step": step_b + tr_b},
                "roofline": roof, "gpu_launches": launches,
                "hbm_gbs_step_alg": (step_b + tr_b) / (ms_max / args.steps * 1e-3) / 1e9,
                "clocks": clocks, "e2e": e2e, "cpu_baseline": cb, "forms": forms,
                "diag": {"nu_wall": d["nu_wall"], "ke": d["ke"], "step": d["step"]}}
        print(json.dumps(line), flush=True)
    s.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
