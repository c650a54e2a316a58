"""Benchmark: node-steps/s of the monodomain split step on the ~2M-node shell.

    python bench.py [--gpus N] [--steps K] [--warmup W]
                    [--form surrogate|plain_fp32|fp64] [--impl ours|reference]
                    [--workload shell_c2|slab_c0|slab_c1|batch_c3]
                    [--no-tune] [--no-run] [--no-cpu] [--accuracy MS]

One step = one global dt (0.1 ms) of EP_CrankNicholson::Solve over the whole
shell: half diffusion step (SpMV + Jacobi-PCG to 1e-7), the ionic phase (ten
Tusscher, endo/M/epi, PMJ stimuli), half diffusion step, and the pseudo-ECG
every 10 steps.

What one default run prints (one JSON line):

* ``value`` -- the learned form (surrogate) over the common window: W
  untimed warm-up steps from t = 0, then exactly K timed steps.  The
  reference arm (``--impl reference``) times the same K steps after the same
  W warm-up steps of the same 2,004,051-node shell on the host cores, so the
  two arms share one ``config``.
* ``forms`` -- the plain FP32 form over the same window, and the ratio.
* ``run_500ms`` -- the metric's whole run: the shell for 500 ms in the
  FP64, plain FP32 and learned forms in lockstep, every step timed on the
  device; node-steps/s of each form, the learned/plain FP32 ratio
  (``speedup_vs_plain_fp32``, also at the top level), and the errors of the
  FP32 and learned forms against FP64 (activation time, APD90, Vm L-inf,
  pseudo-ECG relative L2), with a per-50-ms throughput profile.
* ``roofline`` (the dominant kernel, from per-kernel CUDA events over the
  timed window), ``e2e`` (the same window through the public API with host
  buffers), ``cpu_baseline`` (the CPU port on the same shell, a 2-step
  sample), ``clocks``.

Inputs are resident in HBM and exceed the L2 (operators + states >= 0.5 GB),
so no flush is needed.  Multi-GPU: independent replicas (the path does not
shard), weak scaling, timing = max over ranks of the device time; the
whole 500-ms run and the CPU sample run at N = 1 only.

--accuracy MS runs --workload that long in FP64, FP32 (and, for the shell,
the learned form) in lockstep and prints the errors against FP64.

--impl reference times the CPU implementation on all host cores: the C
restatement of the reference's split step (oracle/) with the same cell
set-up as the GPU arm (endo/M/epi, G_Ks scale, the true-Jacobian Newton),
never loading this project's GPU library.
"""
import argparse
import json
import math
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


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def shared_config(name, n, m, dt, ionic_dt, warmup, steps):
    """The workload and the timed window, identical in both arms."""
    return {"workload": WORKLOAD_TEXT[name].format(n=n, m=m), "dt_ms": dt, "ionic_dt_ms": ionic_dt,
            "window": f"{warmup} untimed warm-up steps from t = 0, then {steps} timed steps "
                      f"(t = {warmup * dt:.2f}-{(warmup + steps) * dt:.2f} ms)",
            "l2": "inputs > L2 (operators + cell states >= 0.5 GB), no flush"}


def _finite(x):
    """JSON has no NaN/inf: map them to None."""
    if isinstance(x, float) and not math.isfinite(x):
        return None
    if isinstance(x, dict):
        return {k: _finite(v) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [_finite(v) for v in x]
    return x


class Clocks:
    """nvidia-smi sampler; reports the median SM clock over the samples taken
    while the GPU was busy (utilization >= 50 %) and every throttle reason
    seen in them."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.lines = []
        self.p = None

    def start(self, wait_first=True):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.p = None
            return
        t0 = time.time()
        while wait_first and not self.lines and time.time() - t0 < 3.0:
            time.sleep(0.02)

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
        return self.summary(self.lines)

    @staticmethod
    def summary(lines):
        import statistics
        sm, busy, smax, reasons = [], [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 10:
                continue
            try:
                mhz, smax, util = float(f[1]), float(f[2]), float(f[4])
            except ValueError:
                continue
            sm.append(mhz)
            if util >= 50.0:
                busy.append(mhz)
                for nm, v in zip(names, f[6:10]):
                    if v.lower() == "active":
                        reasons.add(nm)
        use = busy or sm
        return {"sm_mhz": statistics.median(use) if use else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "samples_under_load": len(busy)}


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


def _traffic(kernel, form, cg_iters, cg_predict=0, cg_batch=8):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/traffic.json); the CG launch's bytes grow with its
    iteration count, so they are stored as prologue + per iteration, plus the
    predictor's own passes when one is on (None if that was not captured).
    The staged CG kernel (cg_batch 32) has its own entry: its evict-first
    matrix stream leaves the vectors in L2."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            t = json.load(f)
    except Exception:
        return None
    key = "cg_staged" if cg_batch == 32 else "cg"
    if kernel == "cg" and key in t:
        c = t[key]
        if "predict2_bytes" in c:               # measured with predictor 2 only
            if cg_predict != 2:
                return None
            return c["predict2_bytes"]["prologue_bytes"] + cg_iters * c["predict2_bytes"]["per_iteration_bytes"]
        extra = 0
        if cg_predict:
            extra = c.get("predict_extra_bytes", {}).get(str(cg_predict))
            if extra is None:
                return None
        return c["prologue_bytes"] + extra + cg_iters * c["per_iteration_bytes"]
    if kernel == "ionic":
        return t.get("surrogate" if form == "surrogate" else "ionic_plain_fp32" if form == "plain_fp32" else "-")
    return None


def algorithmic_bytes(kernel, n, nnz, cg_iters_per_solve, rbytes, nstate=19, ne=10, ecg_every=10, cg_predict=0):
    """Bytes one launch must move at minimum.

    cg (one half diffusion step, SELL values + int32 columns):
      prologue  nnz*(A + B + col) + n*(x + dinv read + r, z, p write)
      iteration nnz*(A + col) + n*(z, p_old read + p_new, q write)         [phase A]
                + n*(p_new, x, r, q, dinv read + x, r, z write)             [phase B]
      predictor (cg_predict k = 1, 2): n*(the start correction read + V saved)
                in the prologue (k = 2: the extrapolation the previous solve
                stored), n*(x, V, k corrections read + x, k corrections
                written) after the iterations
    ionic: the V + stored states read and written once, the activation
      record read (16 B), node type (1 B), G_Ks scale and stimulus head (4 B each).
    ecg: V and the ne weight rows read once per sample.
    """
    if kernel == "cg":
        pro = nnz * (2 * rbytes + 4) + n * 5 * rbytes
        if cg_predict:
            pro += n * rbytes * (2 + (2 + cg_predict + 1 + cg_predict))
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


# --------------------------------------------------------------------------
# CPU side (the oracle; never the GPU library)
# --------------------------------------------------------------------------

def cpu_sim(wl, kind="port"):
    """The CPU split step on the workload's mesh: the C restatement of
    EP_CrankNicholson::Solve with AztecOO's 3-step Jacobi PCG, and as cells
    either the restatement with the GPU arm's set-up (kind 'port': endo/M/epi
    sets, the G_Ks scale, the true-Jacobian Newton capped at 100) or the
    reference's own cell objects compiled from its sources (kind 'reference':
    epicardial constants everywhere, the reference's transposed-Jacobian
    Newton -- the only set-up those objects have)."""
    from oracle import oracle as O
    m = wl.mesh
    csr = O.Csr(m.xyz, m.tets, m.fibers, wl.D, 1.0, wl.dt)
    if kind == "reference":
        cells = O.RefCells(O.TUSSCHER, m.n)
    else:
        cells = O.Cells(O.TUSSCHER, m.n, types=wl.node_type, type_consts=wl.type_consts,
                        gks_scale=wl.gks_scale, tt_jac_true=1, newton_cap=100)
    sim = O.Sim(csr, cells, wl.dt, wl.ionic_dt, cg_tol=1e-7, cg_maxit=1000, jacobi_steps=3)
    sim.V[:] = wl.V0
    return sim, (csr, cells)


def cpu_steps(sim, wl, k0, k1):
    """Steps k0..k1-1 with the stimulus windows [long(t_on/dt), long(t_off/dt));
    wall time of each step."""
    on = (wl.stim_on / wl.dt).astype(int)
    off = (wl.stim_off / wl.dt).astype(int)
    times = []
    for k in range(k0, k1):
        sim.istim[:] = 0.0
        act = (on <= k) & (k < off)
        sim.istim[wl.stim_ids[act]] = wl.stim_amp[act]
        t0 = time.perf_counter()
        sim.step()
        times.append(time.perf_counter() - t0)
    return times


def run_reference(args, rank, world):
    """The CPU arm: rank 0 alone (the other ranks exit without work)."""
    if rank != 0:
        return
    from oracle import oracle as O
    from ucla_cmg_b200 import workloads as W
    threads = host_threads()
    O.set_threads(threads)
    wl = W.shell_c2(epi=O.tt_constants())          # constants from the oracle, not the GPU library
    n = wl.mesh.n
    sim, keep = cpu_sim(wl, "port")
    times = cpu_steps(sim, wl, 0, args.warmup + args.steps)
    timed = times[args.warmup:]
    tot = sum(timed)
    v = n * len(timed) / tot
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(timed), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "form": "CPU split step (FP64)",
            "config": shared_config("shell_c2", n, wl.mesh.m, wl.dt, wl.ionic_dt, args.warmup, args.steps),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"the whole {n}-node shell, steps {args.warmup}..{args.warmup + args.steps - 1} "
                                       f"from t = 0 after {args.warmup} untimed steps, same cell set-up as the GPU arm",
                             "why_port": "the reference's cell objects carry the epicardial constants only and "
                                         "their transposed-Jacobian Newton diverges at ionic dt 0.02 ms in tissue; "
                                         "the port runs the GPU arm's endo/M/epi set-up with the true Jacobian",
                             "cpu": cpu_model()},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    del sim, keep
    if not getattr(args, "no_ref_objects", False):
        # the reference's own cell objects on the same mesh and the same
        # first step, for scale (epicardial everywhere: their only set-up)
        rs, rkeep = cpu_sim(wl, "reference")
        t1 = cpu_steps(rs, wl, 0, 1)
        line["cpu_baseline"]["reference_objects"] = {
            "value": n / t1[0], "unit": UNIT, "cores": threads,
            "sample": "step 0 of the same shell with the reference's unmodified cell objects "
                      "(oracle/_ref), epicardial constants everywhere"}
        del rs, rkeep
    print(json.dumps(_finite(line)), flush=True)


# --------------------------------------------------------------------------
# GPU side
# --------------------------------------------------------------------------

def _deploy(h, prec):
    from ucla_cmg_b200 import capi
    if prec == capi.SURROGATE:
        from ucla_cmg_b200.surrogate import Surrogate, DEFAULT_PATH
        Surrogate.load(os.environ.get("EP_SURROGATE_PATH", DEFAULT_PATH)).deploy(h)
    return h


def whole_run(wl, forms, shapes, local, T=None, bin_ms=50.0, tune=True):
    """The workload for T ms in the given forms, in lockstep: every step
    timed on the device (the handle's CUDA events), Vm compared with the
    first form (FP64) every 1 ms; at the end activation time, APD90 and the
    pseudo-ECG against it."""
    import numpy as np
    T = wl.T if T is None else T
    steps = int(round(T / wl.dt))
    per_ms = max(1, int(round(1.0 / wl.dt)))
    nbin = max(1, int(math.ceil(T / bin_ms)))
    hs = {}
    for name, prec in forms:
        h = _deploy(wl.create(prec, device=local), prec)
        if name in shapes and shapes[name]:
            h.set_launch_config(**shapes[name])
        elif tune:
            shapes[name] = h.autotune(20)[0]          # the state is put back afterwards
        h.set_profiling(False)
        hs[name] = h
    ref = forms[0][0]
    res = {name: dict(ms=0.0, fb=0, cg=0, vinf=0.0, bins=[0.0] * nbin) for name, _ in forms}
    for k in range(0, steps, per_ms):
        kk = min(per_ms, steps - k)
        b = min(nbin - 1, int(k * wl.dt / bin_ms))
        V = {}
        for name, _ in forms:
            st = hs[name].step(kk)
            r = res[name]
            r["ms"] += st["device_ms"]
            r["bins"][b] += st["device_ms"]
            r["fb"] += st["fallback_nodes"]
            r["cg"] += st["cg_iters"]
            V[name] = hs[name].voltage()
        for name, _ in forms[1:]:
            res[name]["vinf"] = max(res[name]["vinf"], float(np.abs(V[name] - V[ref]).max()))
    n = wl.mesh.n
    for name, _ in forms:
        r = res[name]
        r["ta"], r["apd"] = hs[name].activation()
        r["ecg"] = hs[name].ecg()[1]
        hs[name].close()
    bin_steps = [min(steps, int(round((i + 1) * bin_ms / wl.dt))) - min(steps, int(round(i * bin_ms / wl.dt)))
                 for i in range(nbin)]
    out = {"t_ms": T, "steps": steps, "n_nodes": int(n),
           "timed": "every step of the run, device time (CUDA events on each handle's stream)"}
    R = res[ref]
    for name, _ in forms:
        r = res[name]
        e = {"node_steps_per_s": n * steps / (r["ms"] * 1e-3), "ms_per_step": r["ms"] / steps,
             "fallback_fraction": r["fb"] / float(n * steps), "cg_iters_per_solve": r["cg"] / (2.0 * steps),
             "launch_config": shapes.get(name),
             "node_steps_per_s_per_bin": [n * s / (ms * 1e-3) if ms > 0 else None
                                          for s, ms in zip(bin_steps, r["bins"])]}
        if name != ref:
            e["vs_" + ref] = accuracy(R, r, n)
        out[name] = e
    out["bin_ms"] = bin_ms
    return out


def accuracy(R, r, n):
    """Errors of one form's run (r) against the reference form's (R)."""
    import numpy as np
    both = (R["ta"] >= 0) & (r["ta"] >= 0)
    da = np.abs(r["ta"] - R["ta"])[both]
    ab = (R["apd"] > 0) & (r["apd"] > 0)
    dp = np.abs(r["apd"] - R["apd"])[ab]
    e = {"activated": float((r["ta"] >= 0).mean()), "activated_ref": float((R["ta"] >= 0).mean()),
         "act_err_ms": {"mean": float(da.mean()) if both.any() else None,
                        "p99": float(np.percentile(da, 99)) if both.any() else None,
                        "max": float(da.max()) if both.any() else None},
         "apd90_err_ms": {"n": int(ab.sum()),
                          "mean": float(dp.mean()) if ab.any() else None,
                          "p99": float(np.percentile(dp, 99)) if ab.any() else None,
                          "p9999": float(np.percentile(dp, 99.99)) if ab.any() else None,
                          "max": float(dp.max()) if ab.any() else None,
                          "nodes_over_1ms": int((dp > 1.0).sum()), "nodes_over_5ms": int((dp > 5.0).sum()),
                          "repolarised": float((r["apd"] > 0).mean()),
                          "repolarised_ref": float((R["apd"] > 0).mean())},
         "vm_linf_mv": r["vinf"],
         "ecg_rel_l2": float(np.linalg.norm(r["ecg"] - R["ecg"]) / np.linalg.norm(R["ecg"]))}
    if ab.any():
        idx = np.where(ab)[0]
        w = int(idx[int(np.argmax(dp))])
        e["apd90_err_ms"]["worst_node"] = {"node": w, "apd90_ref": float(R["apd"][w]), "apd90": float(r["apd"][w]),
                                           "t_act_ref": float(R["ta"][w]), "t_act": float(r["ta"][w])}
    return e


def _timed_window(h, warmup, steps, dist, clk=None):
    """W untimed steps, then K steps timed on the device (per-kernel events on)."""
    import torch
    h.set_profiling(True)
    h.step(warmup)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    st = h.step(steps)
    torch.cuda.synchronize()
    return st, max_over_ranks(st["device_ms"], dist)


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
    n = wl.mesh.n
    K, Wu = args.steps, args.warmup
    clk = Clocks(local)
    clk.start()
    # ---- the primary form over the common window ----
    g = _deploy(wl.create(prec, device=local), prec)
    if args.launch:
        g.set_launch_config(**json.loads(args.launch))
    tuned = g.autotune(20) if not args.no_tune else None    # the state is put back afterwards
    if args.launch and tuned:
        g.set_launch_config(**json.loads(args.launch))
    shape = g.launch_config()
    st, ms = _timed_window(g, Wu, K, dist)
    value = replica_value(n, K, world, ms)
    rb = 8 if prec == capi.FP64 else 4
    # roofline of the dominant kernel, from the per-kernel events of the window
    nnz = int(wl.mesh.n + 2 * _edge_count(wl.mesh))
    cg_per_solve = st["cg_iters"] / max(1, 2 * K)
    kms = {"cg": st["cg_ms"], "ionic": st["ionic_ms"], "ecg": st["ecg_ms"]}
    ecg_every = max(1, int(round(1.0 / wl.dt)))
    launches = {"cg": 2 * K, "ionic": K, "ecg": max(1, K // ecg_every)}
    dom = max(kms, key=kms.get)
    per_launch_ms = kms[dom] / max(1, launches[dom])
    nstate = capi.model_nstate(wl.model)
    alg = algorithmic_bytes(dom, n, nnz, cg_per_solve, rb, nstate=nstate, ne=len(wl.electrodes),
                            ecg_every=ecg_every, cg_predict=shape["cg_predict"])
    peak, peak_kind = _peaks()
    achieved = alg / (per_launch_ms * 1e-3) / 1e9
    roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind,
            "traffic": _traffic(dom, args.form, cg_per_solve, shape["cg_predict"], shape["cg_batch"])
            if wl.name == "shell_c2" else None,
            "algorithmic_bytes_per_launch": alg, "ms_per_launch": per_launch_ms, "kernel_ms": kms}
    b_ns = node_step_bytes(n, nnz, cg_per_solve, rb, nstate=nstate, ne=len(wl.electrodes), ecg_every=ecg_every,
                           cg_predict=shape["cg_predict"])
    roof["step"] = {"bytes_per_node_step": b_ns, "achieved": b_ns * value / 1e9, "frac": b_ns * value / 1e9 / peak}
    forms = {args.form: {"value": value, "ms_per_step": ms / K, "cg_iters_per_solve": cg_per_solve,
                         "newton_iters": st["newton_iters"], "fallback_fraction": st["fallback_nodes"] / float(n * K),
                         "launch_config": shape}}
    gpu_launches = int(st["launches"])
    g.close()
    # ---- the plain FP32 form over the same window (the metric's ratio) ----
    if prec == capi.SURROGATE and not args.no_compare:
        gp = wl.create(capi.FP32, device=local)
        tp = gp.autotune(20) if not args.no_tune else None
        stp, msp = _timed_window(gp, Wu, K, dist)
        vp = replica_value(n, K, world, msp)
        forms["plain_fp32"] = {"value": vp, "ms_per_step": msp / K,
                               "cg_iters_per_solve": stp["cg_iters"] / max(1, 2 * K),
                               "newton_iters": stp["newton_iters"], "launch_config": gp.launch_config()}
        forms["speedup_vs_plain_fp32"] = value / vp
        gp.close()
    # ---- end to end through the public API with host buffers, same window ----
    ge = _deploy(wl.create(prec, device=local), prec)
    ge.set_launch_config(**shape)
    ge.step(Wu)
    S_host, V_host = ge.states(), ge.voltage()      # the window's inputs, in host memory
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ge.set_states(S_host)
    ge.set_voltage(V_host)
    for _ in range(K):
        ge.step(1)
        V_out = ge.voltage()
    e2e_s = time.perf_counter() - t0
    if dist:
        e2e_s = max_over_ranks(e2e_s * 1e3, dist) * 1e-3
    e2e = {"value": replica_value(n, K, world, e2e_s * 1e3), "unit": UNIT,
           "h2d_bytes_per_step": int((S_host.nbytes + V_host.nbytes) / K),
           "d2h_bytes_per_step": int(V_out.nbytes),
           "copies": "the window's inputs (V and all cell states, FP64 host arrays) uploaded once at the "
                     "start of the timed region, V read back after every step; wall clock, synchronised"}
    ge.close()
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": Wu, "ms_per_step": ms / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == capi.FP64 else ("bf16+f32" if prec == capi.SURROGATE else "f32"),
            "data": "synthetic", "form": args.form,
            "config": shared_config(wl.name, n, wl.mesh.m, wl.dt, wl.ionic_dt, Wu, K)
            if wl.name in WORKLOAD_TEXT else {"workload": wl.name},
            "forms": forms, "parallelism": f"replicas x{world}", "gpu_launches": gpu_launches,
            "roofline": roof, "e2e": e2e}
    # ---- the metric's whole run (500 ms), three forms in lockstep ----
    if world == 1 and not args.no_run and wl.name == "shell_c2" and prec == capi.SURROGATE:
        shapes = {"surrogate": shape}
        if "plain_fp32" in forms:
            shapes["plain_fp32"] = forms["plain_fp32"]["launch_config"]
        run = whole_run(wl, [("fp64", capi.FP64), ("plain_fp32", capi.FP32), ("surrogate", capi.SURROGATE)],
                        shapes, local, T=args.run_ms, tune=not args.no_tune)
        run["speedup_vs_plain_fp32"] = run["surrogate"]["node_steps_per_s"] / run["plain_fp32"]["node_steps_per_s"]
        run["speedup_vs_fp64"] = run["surrogate"]["node_steps_per_s"] / run["fp64"]["node_steps_per_s"]
        line["run_500ms" if abs(args.run_ms - 500.0) < 1e-9 else f"run_{args.run_ms:g}ms"] = run
        line["speedup_vs_plain_fp32"] = run["speedup_vs_plain_fp32"]
    line["clocks"] = clk.stop()
    # ---- CPU baseline: the port on the same shell (bounded sample) ----
    if rank == 0 and world == 1 and not args.no_cpu and wl.name == "shell_c2":
        from oracle import oracle as O
        threads = host_threads()
        O.set_threads(threads)
        sim, keep = cpu_sim(wl, "port")
        t = cpu_steps(sim, wl, 0, 2)
        line["cpu_baseline"] = {"value": n * len(t) / sum(t), "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"steps 0-1 of the same {n}-node shell from t = 0 (the CPU restatement "
                                          "of the split step with the GPU arm's cell set-up)",
                                "cpu": cpu_model()}
        del sim, keep
    if rank == 0:
        print(json.dumps(_finite(line)), flush=True)
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
    import torch
    from ucla_cmg_b200 import capi, workloads as W
    torch.cuda.set_device(local)
    wl = {"shell_c2": W.shell_c2, "slab_c0": W.slab_c0, "slab_c1": W.slab_c1}[args.workload]()
    forms = [("fp64", capi.FP64), ("plain_fp32", capi.FP32)]
    if wl.model == capi.TUSSCHER and abs(wl.dt - 0.1) < 1e-12:
        forms.append(("surrogate", capi.SURROGATE))
    out = whole_run(wl, forms, {}, local, T=args.accuracy, tune=not args.no_tune)
    out["workload"] = wl.name
    print(json.dumps(_finite(out)), flush=True)


def _edge_count(m):
    import numpy as np
    e = np.concatenate([m.tets[:, [a, b]] for a in range(4) for b in range(a + 1, 4)])
    e.sort(axis=1)
    key = e[:, 0].astype(np.int64) * m.n + e[:, 1]
    return len(np.unique(key))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="surrogate", choices=["plain_fp32", "fp64", "surrogate"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--no-run", action="store_true", help="skip the whole 500-ms run of the three forms")
    ap.add_argument("--run-ms", type=float, default=500.0, help="length of the whole run (ms)")
    ap.add_argument("--no-ref-objects", action="store_true",
                    help="reference arm: skip the one-step sample of the reference's own cell objects")
    ap.add_argument("--workload", default="shell_c2", choices=["shell_c2", "batch_c3", "slab_c0", "slab_c1"])
    ap.add_argument("--no-tune", action="store_true", help="skip the launch-shape autotuner")
    ap.add_argument("--launch", default="", help='launch-shape fields set after tuning, JSON ({"cg_predict": 2})')
    ap.add_argument("--no-compare", action="store_true",
                    help="surrogate form: skip the plain FP32 run over the same window")
    ap.add_argument("--accuracy", type=float, default=0.0,
                    help="instead of timing: run --workload this many ms in FP64, FP32 (and the "
                         "learned form) and print the errors against FP64")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours" and args.accuracy <= 0:
        ap.error("--warmup must be >= 3")
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
