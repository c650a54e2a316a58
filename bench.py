"""Benchmark: node-steps/s of the monodomain split step on the ~2M-node shell.

    python bench.py [--gpus N] [--steps K] [--warmup W]
                    [--form surrogate|plain_fp32|fp64] [--impl ours|reference]
                    [--workload shell_c2|slab_c0|slab_c1|batch_c3] [--t-start MS]
                    [--no-tune] [--no-compare] [--no-cpu] [--accuracy MS]

One step = one global dt (0.1 ms) of EP_CrankNicholson::Solve over the whole
shell: half diffusion step (SpMV + Jacobi-PCG to 1e-7), the ionic phase (ten
Tusscher, endo/M/epi, PMJ stimuli; by default the learned form, with the
plain FP32 form timed over the same window for the ratio), half diffusion
step, and the pseudo-ECG every 10 steps.  The timed window starts at
--t-start (40 ms) after an untimed advance, and each form's launch shape is
picked by the autotuner first.  Inputs (the operators and all cell states)
are resident in HBM; they total > 126 MB, so no L2 flush is needed between
steps.  Multi-GPU: independent replicas (the path does not shard), weak
scaling, timing = max over ranks of the device (CUDA-event) time.

--accuracy MS runs the workload that long in FP64, FP32 and the learned form
in lockstep and prints the errors against FP64 instead of timing.

--impl reference times the reference's own CPU implementation on the host
cores: the reference cell-model sources compiled unmodified (oracle/_ref)
inside the C restatement of the CN/PCG split step, on a bounded sample of the
same workload (a coarser shell), all host threads.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "node-steps/s at 2M-node shell: surrogate vs plain FP32, act-time err ≤0.5 ms"
WORKLOAD_TEXT = {
    "shell_c2": "shell_c2: truncated prolate-ellipsoid shell, {n} nodes, {m} tets, ten Tusscher endo/M/epi "
                "40/30/30, G_Ks 0.8->1.2 apex->base, 200 PMJ stimuli t~U(0,30) ms, 10 electrodes",
    "slab_c0": "slab_c0: 1.0x1.0x0.2 cm slab, {n} nodes, {m} tets, ten Tusscher epi, corner stimulus, dt 0.02 ms",
    "slab_c1": "slab_c1: 4.0x4.0x0.4 cm slab, {n} nodes, {m} tets, Mahajan, edge-strip stimulus, dt 0.01 ms",
}
UNIT = "node-steps/s"


def max_over_ranks(ms, dist):
    """The slowest rank's device time (replicas: the job ends with it)."""
    if dist is None:
        return ms
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(ms)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(n_nodes, steps, world, ms):
    """Whole-job node-steps/s: every rank advances its own copy of the
    workload, so the job does world x n x steps node-steps in max-rank time."""
    return n_nodes * steps * world / (ms * 1e-3)


def _env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.lines = []
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.p = None

    def _read(self):
        for line in self.p.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        import statistics
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), for the CPU baseline."""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic(kernel, form, cg_iters, cg_predict=0):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/traffic.json); the CG launch's bytes grow with its
    iteration count, so they are stored as prologue + per iteration, plus the
    predictor's own passes when one is on (None if that was not captured)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            t = json.load(f)
    except Exception:
        return None
    if kernel == "cg" and "cg" in t:
        extra = 0
        if cg_predict:
            extra = t["cg"].get("predict_extra_bytes", {}).get(str(cg_predict))
            if extra is None:
                return None
        return t["cg"]["prologue_bytes"] + extra + cg_iters * t["cg"]["per_iteration_bytes"]
    if kernel == "ionic":
        return t.get("surrogate" if form == "surrogate" else "ionic_plain_fp32" if form == "plain_fp32" else "-")
    return None


def algorithmic_bytes(kernel, n, nnz, cg_iters_per_solve, rbytes, nstate=19, ne=10, ecg_every=10, cg_predict=0):
    """Bytes one launch must move at minimum.

    cg (one half diffusion step, SELL values + int32 columns):
      prologue  nnz*(A + B + col) + n*(x + dinv read + r, z, p write)
      iteration nnz*(A + col) + n*(z, p_old read + p_new, q write)         [phase A]
                + n*(p_new, x, r, q, dinv read + x, r, z write)             [phase B]
      predictor (cg_predict k = 1, 2): n*(k corrections read + V saved) in the
                prologue, n*(x, V, k corrections read + x, k corrections
                written) after the iterations
    ionic: the V + stored states read and written once, the activation
      record read (16 B), node type (1 B), G_Ks scale and stimulus head (4 B each).
    ecg: V and the ne weight rows read once per sample.
    """
    if kernel == "cg":
        pro = nnz * (2 * rbytes + 4) + n * 5 * rbytes
        if cg_predict:
            pro += n * rbytes * ((cg_predict + 1) + (2 + cg_predict + 1 + cg_predict))
        it = nnz * (rbytes + 4) + n * 4 * rbytes + n * 8 * rbytes
        return pro + cg_iters_per_solve * it
    if kernel == "ionic":
        return n * (2 * nstate * rbytes + 16 + 1 + rbytes + 4)
    if kernel == "ecg":
        return n * (1 + ne) * rbytes
    raise ValueError(kernel)


def node_step_bytes(n, nnz, cg_iters_per_solve, rbytes, nstate=19, ne=10, ecg_every=10, cg_predict=0):
    """Algorithmic bytes of one node-step: the ionic phase, the two CN half
    steps and the ECG sample share, per node (the whole-step roofline: these
    bytes x node-steps/s against the copy bandwidth)."""
    tot = (algorithmic_bytes("ionic", n, nnz, cg_iters_per_solve, rbytes, nstate=nstate)
           + 2 * algorithmic_bytes("cg", n, nnz, cg_iters_per_solve, rbytes, cg_predict=cg_predict)
           + algorithmic_bytes("ecg", n, nnz, cg_iters_per_solve, rbytes, ne=ne) / max(1, ecg_every))
    return tot / n


def cpu_sample(kind, h, steps, threads):
    """Time the CPU path on a coarser shell (same model, dt, stimuli).
    kind 'reference': the reference cell objects (oracle/_ref) in the C
    restatement of the CN split step with AztecOO's 3-step Jacobi;
    kind 'port': the C restatement throughout."""
    from oracle import oracle as O
    from ucla_cmg_b200 import workloads as W
    O.set_threads(threads)
    wl = W.shell_c2(h=h)
    m = wl.mesh
    csr = O.Csr(m.xyz, m.tets, m.fibers, wl.D, 1.0, wl.dt)
    if kind == "reference" and O.ref_lib() is not None:
        cells = O.RefCells(O.TUSSCHER, m.n)        # the reference has the epicardial set only
    else:
        kind = "port"
        cells = O.Cells(O.TUSSCHER, m.n, types=wl.node_type, type_consts=wl.type_consts,
                        gks_scale=wl.gks_scale, tt_jac_true=1, newton_cap=100)
    sim = O.Sim(csr, cells, wl.dt, wl.ionic_dt, cg_tol=1e-7, cg_maxit=1000, jacobi_steps=3)
    sim.V[:] = wl.V0
    on = (wl.stim_on / wl.dt).astype(int)
    off = (wl.stim_off / wl.dt).astype(int)
    times = []
    for k in range(steps):
        sim.istim[:] = 0.0
        act = (on <= k) & (k < off)
        sim.istim[wl.stim_ids[act]] = wl.stim_amp[act]
        t0 = time.perf_counter()
        sim.step()
        times.append(time.perf_counter() - t0)
    return m.n, times, kind


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    h = float(os.environ.get("EP_REF_SAMPLE_H", "0.2"))
    n, times, kind = cpu_sample("reference", h, args.warmup + args.steps, threads)
    timed = times[args.warmup:]
    tot = sum(timed)
    v = n * len(timed) / tot
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(timed), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": f"shell_c2 sample: truncated ellipsoid shell h={h} cm ({n} nodes), "
                                   "ten Tusscher, dt 0.1 / ionic 0.02 ms, 200 PMJ stimuli",
                       "form": "reference CPU (FP64)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"{len(timed)} steps of a {n}-node shell (h={h} cm) from t=0",
                             "cpu": cpu_model()},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local):
    import numpy as np
    import torch
    from ucla_cmg_b200 import capi, workloads as W

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    prec = {"fp64": capi.FP64, "plain_fp32": capi.FP32, "surrogate": capi.SURROGATE}[args.form]
    if args.workload == "batch_c3":
        return run_batch(args, rank, world, local, dist, prec)
    wl = {"shell_c2": W.shell_c2, "slab_c0": W.slab_c0, "slab_c1": W.slab_c1}[args.workload]()
    g = wl.create(prec, device=local)
    if prec == capi.SURROGATE:
        from ucla_cmg_b200.surrogate import Surrogate, DEFAULT_PATH
        Surrogate.load(os.environ.get("EP_SURROGATE_PATH", DEFAULT_PATH)).deploy(g)
    n = wl.mesh.n
    # the timed window starts at t_start (advanced untimed), inside the
    # activation of the wall, so that the window holds wavefronts, plateau
    # and rest rather than the quiet first milliseconds
    pre = int(round(args.t_start / wl.dt))
    if args.launch:
        g.set_launch_config(**json.loads(args.launch))
    for k in range(0, pre, 500):
        g.step(min(500, pre - k))
    # the project's autotuner picks the launch shape (state is restored)
    tuned = g.autotune(20) if not args.no_tune else None
    if args.launch and tuned:
        g.set_launch_config(**json.loads(args.launch))
    g.set_profiling(True)
    g.step(args.warmup)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = Clocks(local)
    clk.start()
    st = g.step(args.steps)
    clocks = clk.stop()
    torch.cuda.synchronize()
    ms = max_over_ranks(st["device_ms"], dist)
    if dist:
        dist.barrier()
    value = replica_value(n, args.steps, world, ms)
    # ---- end to end through the public API with host buffers ----
    states = g.states()
    V = g.voltage()
    k_e2e = max(3, args.steps)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g.set_states(states)
    g.set_voltage(V)
    for _ in range(k_e2e):
        g.step(1)
        V = g.voltage()
    e2e_s = time.perf_counter() - t0
    rb = 8 if prec == capi.FP64 else 4
    e2e = {"value": n * k_e2e / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": int((states.nbytes + V.nbytes) / k_e2e),
           "d2h_bytes_per_step": int(V.nbytes)}
    # ---- roofline of the dominant kernel ----
    nnz = int(wl.mesh.n + 2 * _edge_count(wl.mesh))
    cg_per_solve = st["cg_iters"] / max(1, 2 * args.steps)
    kms = {"cg": st["cg_ms"], "ionic": st["ionic_ms"], "ecg": st["ecg_ms"]}
    ecg_every = max(1, int(round(1.0 / wl.dt)))
    launches = {"cg": 2 * args.steps, "ionic": args.steps, "ecg": max(1, args.steps // ecg_every)}
    dom = max(kms, key=kms.get)
    per_launch_ms = kms[dom] / max(1, launches[dom])
    nstate = capi.model_nstate(wl.model)
    alg = algorithmic_bytes(dom, n, nnz, cg_per_solve, rb, nstate=nstate, ne=len(wl.electrodes),
                            ecg_every=ecg_every, cg_predict=g.launch_config()["cg_predict"])
    peak, peak_kind = _peaks()
    achieved = alg / (per_launch_ms * 1e-3) / 1e9
    roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind, "traffic": _traffic(dom, args.form, cg_per_solve, g.launch_config()["cg_predict"]) if wl.name == "shell_c2" else None,
            "algorithmic_bytes_per_launch": alg, "ms_per_launch": per_launch_ms,
            "kernel_ms": kms}
    b_ns = node_step_bytes(n, nnz, cg_per_solve, rb, nstate=nstate, ne=len(wl.electrodes), ecg_every=ecg_every,
                           cg_predict=g.launch_config()["cg_predict"])
    roof["step"] = {"bytes_per_node_step": b_ns, "achieved": b_ns * value / 1e9, "frac": b_ns * value / 1e9 / peak}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == capi.FP64 else ("bf16+f32" if prec == capi.SURROGATE else "f32"),
            "data": "synthetic",
            "config": {"workload": WORKLOAD_TEXT[wl.name].format(n=n, m=wl.mesh.m),
                       "form": args.form, "dt_ms": wl.dt, "ionic_dt_ms": wl.ionic_dt,
                       "t_window_ms": [round((pre + args.warmup) * wl.dt, 3),
                                       round((pre + args.warmup + args.steps) * wl.dt, 3)],
                       "l2": "inputs > L2 (operators + states ~ 0.5 GB), no flush",
                       "cg_iters_per_solve": cg_per_solve, "newton_iters": st["newton_iters"],
                       "launch_config": tuned[0] if tuned else g.launch_config(),
                       "fallback_fraction": st["fallback_nodes"] / float(n * args.steps),
                       "parallelism": f"replicas x{world}"},
            "gpu_launches": int(st["launches"]),
            "clocks": clocks, "roofline": roof, "e2e": e2e}
    if prec == capi.SURROGATE and not args.no_compare:
        # the plain FP32 form over the same simulated window, for the ratio
        # the metric is about (same handle set-up, same steps)
        gp = wl.create(capi.FP32, device=local)
        for k in range(0, pre, 500):
            gp.step(min(500, pre - k))
        if not args.no_tune:
            gp.autotune(20)
        gp.step(args.warmup)
        torch.cuda.synchronize()
        stp = gp.step(args.steps)
        vp = replica_value(n, args.steps, world, max_over_ranks(stp["device_ms"], dist))
        line["config"]["plain_fp32"] = {"value": vp, "ms_per_step": stp["device_ms"] / args.steps,
                                        "launch_config": gp.launch_config(),
                                        "cg_iters_per_solve": stp["cg_iters"] / max(1, 2 * args.steps)}
        line["config"]["speedup_vs_plain_fp32"] = value / vp
        gp.close()
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        h = float(os.environ.get("EP_CPU_SAMPLE_H", "0.12"))
        ncpu, times, kind = cpu_sample("reference", h, 6, threads)
        v = ncpu * 5 / sum(times[1:])
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": kind,
                                "sample": f"5 steps (after 1 untimed) of a {ncpu}-node shell "
                                          f"(h={h} cm) from t=0, same model, dt and stimuli",
                                "cpu": cpu_model()}
        # the same path on one host thread (the reference runs one MPI rank
        # per core; this is one rank's speed), on a coarser sample
        n1, t1, _ = cpu_sample("reference", 0.2, 3, 1)
        line["cpu_baseline"]["value_1_thread"] = n1 * 2 / sum(t1[1:])
        line["cpu_baseline"]["sample_1_thread"] = f"2 steps (after 1 untimed) of a {n1}-node shell (h=0.2 cm)"
    g.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_batch(args, rank, world, local, dist, prec):
    """64 independent slabs (uneven sizes and parameters) stepped together."""
    import torch
    from ucla_cmg_b200 import capi, workloads as W
    wl = W.batch_c3()
    b = wl.create(prec, device=local)
    n = wl.n_nodes
    tuned = b.autotune(trial_steps=20)
    b.set_profiling(False)
    b.step(args.warmup)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = Clocks(local)
    clk.start()
    st = b.step(args.steps)
    clocks = clk.stop()
    torch.cuda.synchronize()
    ms = max_over_ranks(st["device_ms"], dist)
    if dist:
        dist.barrier()
    line = {"metric": "node-steps/s, 64 independent slabs in one batch", "value": replica_value(n, args.steps, world, ms),
            "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == capi.FP64 else "f32", "data": "synthetic",
            "config": {"workload": f"batch_c3: 64 ten Tusscher slabs, 21x21x6..101x101x11 nodes, {n} nodes "
                                   "in all, G_Ks/G_to/G_CaL x U(0.5,1.5), corner stimuli, dt 0.02 ms",
                       "form": args.form, "launch_config": tuned[0], "tuned_ms_per_step": tuned[1],
                       "untuned_ms_per_step": tuned[2], "configs_tried": tuned[3],
                       "cg_iters_per_solve": st["cg_iters"] / max(1, 2 * 64 * args.steps),
                       "l2": "inputs > L2, no flush", "parallelism": f"replicas x{world}"},
            "gpu_launches": int(st["launches"]), "clocks": clocks}
    b.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_accuracy(args, local):
    """The workload run for args.accuracy ms in the FP64, plain FP32 and (ten
    Tusscher at dt = 0.1 ms, the step the network was trained for) learned
    forms; errors against FP64: activation time, APD90, Vm L-infinity over
    1 ms snapshots, pseudo-ECG relative L2."""
    import numpy as np
    import torch
    from ucla_cmg_b200 import capi, workloads as W
    from ucla_cmg_b200.surrogate import Surrogate, DEFAULT_PATH
    torch.cuda.set_device(local)
    wl = {"shell_c2": W.shell_c2, "slab_c0": W.slab_c0, "slab_c1": W.slab_c1}[args.workload]()
    steps = int(round(args.accuracy / wl.dt))
    per_ms = max(1, int(round(1.0 / wl.dt)))
    forms = [("fp64", capi.FP64), ("plain_fp32", capi.FP32)]
    if wl.model == capi.TUSSCHER and abs(wl.dt - 0.1) < 1e-12:
        forms.append(("surrogate", capi.SURROGATE))
    hs = {}
    tuned = {}
    for name, prec in forms:
        hs[name] = wl.create(prec, device=local)
        if prec == capi.SURROGATE:
            Surrogate.load(os.environ.get("EP_SURROGATE_PATH", DEFAULT_PATH)).deploy(hs[name])
        if not args.no_tune:
            tuned[name] = hs[name].autotune(20)[0]      # the state is put back afterwards
    res = {name: dict(ms=0.0, fb=0, vinf=0.0) for name, _ in forms}
    # the three runs advance in lockstep; Vm is compared every 1 ms
    for k in range(0, steps, per_ms):
        V = {}
        for name, _ in forms:
            st = hs[name].step(min(per_ms, steps - k))
            res[name]["ms"] += st["device_ms"]
            res[name]["fb"] += st["fallback_nodes"]
            V[name] = hs[name].voltage()
        for name, _ in forms[1:]:
            res[name]["vinf"] = max(res[name]["vinf"], float(np.abs(V[name] - V["fp64"]).max()))
    for name, _ in forms:
        r = res[name]
        r["ta"], r["apd"] = hs[name].activation()
        r["ecg"] = hs[name].ecg()[1]
        r["fb"] /= float(wl.mesh.n * steps)
        hs[name].close()
    ref = res["fp64"]
    out = {"workload": wl.name, "t_ms": args.accuracy, "n_nodes": int(wl.mesh.n), "dt_ms": wl.dt}
    for name, _ in forms:
        r = res[name]
        e = {"node_steps_per_s": wl.mesh.n * steps / (r["ms"] * 1e-3), "fallback_fraction": r["fb"],
             "launch_config": tuned.get(name)}
        if name != "fp64":
            both = (ref["ta"] >= 0) & (r["ta"] >= 0)
            da = np.abs(r["ta"] - ref["ta"])[both]
            ab = (ref["apd"] > 0) & (r["apd"] > 0)
            dp = np.abs(r["apd"] - ref["apd"])[ab]
            e.update({"activated": float((r["ta"] >= 0).mean()), "activated_fp64": float((ref["ta"] >= 0).mean()),
                      "act_err_ms": {"mean": float(da.mean()), "p99": float(np.percentile(da, 99)), "max": float(da.max())},
                      "apd90_err_ms": {"n": int(ab.sum()), "mean": float(dp.mean()) if ab.any() else None,
                                       "p99": float(np.percentile(dp, 99)) if ab.any() else None,
                                       "max": float(dp.max()) if ab.any() else None,
                                       "repolarised": float((r["apd"] > 0).mean()),
                                       "repolarised_fp64": float((ref["apd"] > 0).mean())},
                      "vm_linf_mv": r["vinf"],
                      "ecg_rel_l2": float(np.linalg.norm(r["ecg"] - ref["ecg"]) / np.linalg.norm(ref["ecg"]))})
        out[name] = e
    print(json.dumps(out), flush=True)


def _edge_count(m):
    import numpy as np
    e = np.concatenate([m.tets[:, [a, b]] for a in range(4) for b in range(a + 1, 4)])
    e.sort(axis=1)
    key = e[:, 0].astype(np.int64) * m.n + e[:, 1]
    return len(np.unique(key))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="surrogate", choices=["plain_fp32", "fp64", "surrogate"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", default="shell_c2", choices=["shell_c2", "batch_c3", "slab_c0", "slab_c1"])
    ap.add_argument("--no-tune", action="store_true", help="skip the launch-shape autotuner")
    ap.add_argument("--launch", default="", help='launch-shape fields set after tuning, JSON ({"cg_predict": 2})')
    ap.add_argument("--no-compare", action="store_true",
                    help="surrogate form: skip the plain FP32 run over the same window")
    ap.add_argument("--t-start", type=float, default=40.0,
                    help="simulated ms advanced (untimed) before the warm-up")
    ap.add_argument("--accuracy", type=float, default=0.0,
                    help="instead of timing: run the shell this many ms in FP64, FP32 and the "
                         "learned form and print the errors against FP64")
    args = ap.parse_args()
    rank, world, local = _env()
    if args.accuracy > 0:
        if rank == 0:
            run_accuracy(args, local)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
