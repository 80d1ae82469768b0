"""Benchmark: jerk-search throughput (spectra/hour) on one B200 per rank.

Workload (the paper-scale configuration): 2^25-sample spectra (2^24 complex
bins, dt = 54.6 us, T ~ 1832 s) of seeded Gaussian noise plus four injected
pulsars, searched with -zmax 200 -wmax 300 -numharm 16 -sigma 3.0
(23,364 rsteps of 718 bins per spectrum).  Data are synthetic (no dataset is
available offline); the reference's published runs used real GBT data.

A step is one full search of one spectrum.  value: spectra/hour over K timed
steps with the spectra already resident in HBM.  e2e: the same through the
public C ABI with the spectrum in pinned host memory (host-to-device copy and
the hit/candidate read-back inside the timed region).  Each spectrum (128 MiB)
and the per-batch ffdot volumes (163 MB per rstep, GBs per batch) exceed the
126 MB L2, so no flush is needed between steps.  The rsteps per batch are
autotuned (cached per geometry) unless --batch is given.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun every rank searches its own spectra (weak scaling, no data-path
collective); the time is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "spectra/hr (2^25 bins, z200 w300 h16) batched+served vs plain on B200; p50/p99"
UNIT = "spectra/hour"
N_SAMPLES = 1 << 25
DT = 54.6e-6
ZMAX, WMAX, NUMHARM, SIGMA = 200, 300, 16, 3.0
WORKLOAD = "jerk search, 2^25-sample spectra, -zmax 200 -wmax 300 -numharm 16 -sigma 3.0"


# FP32 CUDA-core peak of one B200 at its maximum SM clock (148 SMs x 128 FP32
# lanes x 2 flops per FMA x 1965 MHz); the correlation kernels are bound by it.
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12

# DRAM traffic of one fftlen-2048 correlation launch (corr_fold_kernel) at 16
# rsteps per batch, from an ncu capture (dram__bytes_read.sum /
# dram__bytes_write.sum) of
#   python bench.py --rsteps 128 --steps 1 --warmup 1 --no-cpu-baseline --no-ref-gpu
#                   --e2e-steps 1 --batch 16 --no-extras
# The read side (folded kernel rows + data rows) is paid once per launch; the
# write side (the volumes) grows with the rsteps per batch.
CORR2048_TRAFFIC = {"read": 491.168256e6, "write": 2241.328e6, "batch": 16}


def corr2048_traffic(batch: int) -> float:
    t = CORR2048_TRAFFIC
    return t["read"] + t["write"] * batch / t["batch"]


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
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
        except subprocess.TimeoutExpired:
            self.proc.kill()
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
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def paper_setup():
    from prestozl_b200 import jerk

    obs, fftlen, _ = jerk.obs_from_params(N_SAMPLES // 2, N_SAMPLES, DT, ZMAX, WMAX, NUMHARM,
                                          SIGMA)
    subs = jerk.subharm_sizes(obs, fftlen)
    return obs, fftlen, subs


def make_spectrum(seed: int, device):
    from prestozl_b200 import synth

    rng = np.random.default_rng(seed)
    pulsars = synth.random_pulsars(rng, 4)
    ts = synth.timeseries_torch(N_SAMPLES, DT, pulsars, seed, device=device)
    return synth.presto_fft_torch(ts)


# --------------------------------------------------------------------------
# CPU reference: the reference's own accelsearch (compiled from its sources
# into oracle/_ref), run as the reference recommends for throughput: one
# single-threaded search per core (its README's `xargs -P cores` with
# -ncpus 1).  Its OpenMP form is not used: at many hits its threads call
# candidate_sigma (dcdflib's cdfchi, which keeps static state) at once
# (src/accel_utils.c:1518-1535), which aborts at 32 harmonics.  Nothing of
# this project's engine is loaded on this path: the workers load only the
# reference build, and the geometry is the reference's own create_accelobs.

SEARCH_ARGS = ["-zmax", str(ZMAX), "-wmax", str(WMAX), "-numharm", str(NUMHARM),
               "-sigma", str(SIGMA)]


def _ref_worker(conn, fftpath, search_args):
    """One reference search process: opens the .fft, builds the reference's
    kernel bank, then times ref.search(max_steps=n) on request."""
    from oracle import bindings as ob

    ob.set_threads(1)
    ob.quiet_wisdom()
    ref = ob.RefSearch(fftpath, search_args)
    ref.make_bank()
    conn.send("ready")
    while True:
        msg = conn.recv()
        if msg[0] == "search":
            t0 = time.perf_counter()
            ref.search(max_steps=msg[1])
            conn.send(time.perf_counter() - t0)
        elif msg[0] == "polish":
            done, t_pol = 0, 0.0
            for nh, r, z, w in msg[1]:
                t0 = time.perf_counter()
                ref.polish(nh, r - ref.obs.lobin, z, w)
                t_pol += time.perf_counter() - t0
                done += 1
                if t_pol > msg[2]:
                    break
            conn.send((done, t_pol))
        else:
            break
    ref.close()
    conn.close()


class RefPool:
    """procs reference searches in spawned processes, all on one .fft file
    (memory-mapped, so its pages are shared).  step(n) runs the first n
    rsteps in every process at once and returns the wall seconds until the
    last one finished."""

    def __init__(self, spec_np, procs: int):
        import multiprocessing as mp

        self.tmp = tempfile.TemporaryDirectory()
        root = os.path.join(self.tmp.name, "paper")
        from oracle import bindings as ob  # noqa: F401  (reference build present)
        from prestozl_b200 import synth  # data generator only (numpy)
        synth.write_fft(root, spec_np, N_SAMPLES, DT)
        self.fft = root + ".fft"
        ctx = mp.get_context("spawn")
        self.conns, self.procs = [], []
        for _ in range(procs):
            a, b = ctx.Pipe()
            p = ctx.Process(target=_ref_worker, args=(b, self.fft, SEARCH_ARGS), daemon=True)
            p.start()
            self.conns.append(a)
            self.procs.append(p)
        for c in self.conns:
            if c.recv() != "ready":
                raise RuntimeError("reference worker failed to start")

    def step(self, n: int) -> float:
        t0 = time.perf_counter()
        for c in self.conns:
            c.send(("search", n))
        for c in self.conns:
            c.recv()
        return time.perf_counter() - t0

    def polish(self, cands, budget_s: float):
        """The reference's candidate polishing (one core, as its CPU2 runs
        it) on up to budget_s seconds of the given candidates."""
        self.conns[0].send(("polish", [(int(c["numharm"]), float(c["r"]), float(c["z"]),
                                        float(c["w"])) for c in cands], budget_s))
        done, t = self.conns[0].recv()
        return {"candidates": done, "s_per_candidate": t / max(done, 1), "cores": 1}

    def close(self):
        for c in self.conns:
            try:
                c.send(("quit",))
            except (OSError, BrokenPipeError):
                pass
        for p in self.procs:
            p.join(timeout=30)
        self.tmp.cleanup()


def ref_processes() -> int:
    """One process per core, bounded by host memory (about 0.8 GB each at the
    paper configuration: the kernel bank and the correlation buffers)."""
    cores = os.cpu_count() or 1
    try:
        import psutil

        avail = psutil.virtual_memory().available
        cores = min(cores, max(1, int(avail // (1.2 * 2 ** 30))))
    except ImportError:
        pass
    return max(1, min(cores, 64))


def ref_geometry(spec_np):
    """(rsteps per spectrum, obs) from the reference's own create_accelobs."""
    from oracle import bindings as ob
    from prestozl_b200 import synth

    with tempfile.TemporaryDirectory() as tmp:
        root = os.path.join(tmp, "paper")
        synth.write_fft(root, spec_np, N_SAMPLES, DT)
        ref = ob.RefSearch(root + ".fft", SEARCH_ARGS)
        obs = ref.obs
        n = _count_rsteps(obs)
        ref.close()
    return n


def reference_sample(spec_np, procs: int, target_s: float, steps: int = 1, warmup: int = 0,
                     polish_cands=None, polish_s: float = 10.0):
    """The reference CPU search as a process pool: calibrates the rsteps per
    step on one rstep so that a step takes about target_s, then times warmup +
    steps steps.  Returns (step seconds of the timed steps, rsteps per process
    per step, polishing or None)."""
    pool = RefPool(spec_np, procs)
    try:
        t1 = pool.step(1)
        n = max(1, min(int(target_s / max(t1, 1e-3)), 400))
        times = [pool.step(n) for _ in range(warmup + steps)][warmup:]
        pol = pool.polish(polish_cands, polish_s) if polish_cands is not None and len(
            polish_cands) else None
    finally:
        pool.close()
    return times, n, pol


def workload_config(world: int, nrsteps: int, nsearch: int = 0) -> dict:
    """The config both arms report (the same dict, so the arms compare)."""
    return {"workload": WORKLOAD if not nsearch else
            f"{WORKLOAD} (PARTIAL: first {nsearch} rsteps per spectrum)",
            "numbins": N_SAMPLES // 2, "rsteps_per_spectrum": nrsteps,
            "l2": "inputs larger than L2 (128 MiB spectra, GB-sized volumes), no flush",
            "parallelism": f"replicas x{world}"}


def input_prep_leg(device, reps: int = 5):
    """The .dat preparation on the GPU (jerk_spectrum_from_timeseries: realfft,
    deredden, bin 0) of one N_SAMPLES float32 series already in HBM."""
    import torch

    from prestozl_b200 import jerk

    g = torch.Generator(device=device)
    g.manual_seed(11)
    ts = torch.randn(N_SAMPLES, device=device, generator=g)
    out = torch.empty(N_SAMPLES // 2, dtype=torch.complex64, device=device)
    for _ in range(2):
        jerk.spectrum_from_timeseries(ts, out)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        jerk.spectrum_from_timeseries(ts, out)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    alg = 8.0 * N_SAMPLES  # the series read once, the spectrum written once
    return {"samples": N_SAMPLES, "ms_per_series": ms, "algorithmic_bytes": alg,
            "achieved_gbs": alg / ms / 1e6, "kernels": "rf_twiddle x2, rf_column, rf_row, "
            "rf_post, dr_level, dr_scale", "launches": 7,
            "note": "three FFT passes and two red-noise passes move about 5x the algorithmic "
                    "bytes; one-off per series (about 0.02 % of its search)"}


def dedisp_leg(device, reps: int = 5, worklen: int = 65536, nsub: int = 64,
               numdms: int = 512, bs: int = 4):
    """prepsubband_cu's GPU steps on one block (jerk_downsample_subbands of
    bs x worklen samples, then jerk_dedisp_subbands into numdms series),
    inputs in HBM, CUDA events on torch's current stream; beside them the
    reference's own DownsampDataArray / getDedisp (src/prepsubband_kernels.cu,
    compiled for sm_100a into oracle/_ref) on the same buffers when present.
    Offsets follow the cold-plasma law over 1200-1600 MHz for DMs 0..255.5 at
    dt = 256 us (the largest under a block)."""
    import ctypes as C

    import torch

    from prestozl_b200 import jerk

    f = 1200.0 + (np.arange(nsub) + 0.5) * 400.0 / nsub
    dms = 0.5 * np.arange(numdms)
    off = np.rint(4.148808e3 * dms[:, None] * (f[None, :] ** -2 - f[-1] ** -2) / 256e-6)
    off = np.minimum(off, worklen).astype(np.int32)
    g = torch.Generator(device=device)
    g.manual_seed(12)
    raw = torch.randn((worklen * bs, nsub), device=device, generator=g)
    cur = torch.randn((worklen, nsub), device=device, generator=g)
    last = torch.randn((worklen, nsub), device=device, generator=g)
    ds = torch.empty((worklen, nsub), device=device)
    out = torch.empty((numdms, worklen), device=device)
    dd = jerk.Dedisperser(worklen, nsub, off)

    def timed(fn):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    ms_ds = timed(lambda: jerk.downsample_subbands(raw, bs, out=ds))
    ms_dd = timed(lambda: dd(cur, last, out=out))
    shape = dd.shape
    dd.close()
    adds = float(numdms) * worklen * nsub
    dd_bytes = 4.0 * (2 * worklen * nsub + numdms * worklen)
    ds_bytes = 4.0 * (worklen * bs * nsub + worklen * nsub)
    res = {"worklen": worklen, "nsub": nsub, "numdms": numdms, "downsamp": bs,
           "tiling_dms_x_samples": list(shape),
           "dedisp_ms": ms_dd, "dedisp_gadds_per_s": adds / ms_dd / 1e6,
           "dedisp_algorithmic_bytes": dd_bytes, "dedisp_achieved_gbs": dd_bytes / ms_dd / 1e6,
           "downsample_ms": ms_ds, "downsample_achieved_gbs": ds_bytes / ms_ds / 1e6,
           "bound": "dedisp: shared-memory load wavefronts (about 1.03 per 32 adds in the "
                    "sums, plus the window staging); downsample: HBM"}
    try:
        from oracle import bindings as ob

        path = getattr(ob, "REF_DEDISP_GPU_LIB", "")
        if os.path.exists(path):
            lib = C.CDLL(path)
            lib.DownsampDataArray.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
            lib.getDedisp.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                      C.c_int, C.c_void_p]
            doff = torch.from_numpy(off).to(device)
            ref = torch.empty_like(out)
            res["reference_downsample_ms"] = timed(lambda: lib.DownsampDataArray(
                ds.data_ptr(), raw.data_ptr(), worklen, bs, nsub))
            res["reference_dedisp_ms"] = timed(lambda: lib.getDedisp(
                cur.data_ptr(), last.data_ptr(), ref.data_ptr(), worklen, nsub, numdms,
                doff.data_ptr()))
            torch.cuda.synchronize()
            res["equal_to_reference"] = bool(torch.equal(ref, out))
    except OSError as e:
        res["reference"] = f"not loaded: {e}"
    return res


def polish_leg(spec_np, cands, max_cands: int = 64):
    """GPU polishing (jerk_polish_rzw) of a search's final candidates.  The
    local powers only scale the per-harmonic sums, so 1.0 is passed: the
    device work is the same."""
    from prestozl_b200 import jerk

    sel = list(cands[:max_cands])
    if not sel:
        return None
    pol = jerk.Polisher()
    args = [(int(c["numharm"]), float(c["r"]), float(c["z"]), float(c["w"])) for c in sel]
    nh, r, z, w = args[0]
    pol.polish(spec_np, nh, r, z, w, np.ones(nh, np.float32))  # buffers, modules
    t0 = time.perf_counter()
    for nh, r, z, w in args:
        pol.polish(spec_np, nh, r, z, w, np.ones(nh, np.float32))
    dt = time.perf_counter() - t0
    pol.close()
    counts = {}
    for nh, _, _, _ in args:
        counts[str(nh)] = counts.get(str(nh), 0) + 1
    return {"candidates": len(args), "ms_per_candidate": dt * 1000.0 / len(args),
            "numharm_counts": counts,
            "timing": "host wall clock around each synchronous call (upload, 6 kernel kinds, "
                      "result copy)",
            "launches_per_candidate": "2 + 3 per distinct kernel FFT length + 1 per w-response "
                                      "FFT length + 1"}


def run_extras(args):
    """--extras-only: the input-preparation and polishing legs alone, on one
    paper-scale spectrum with candidates on the search's grid (a few hundred
    MB on the device; the form profiled with ncu).  Polishing runs first."""
    import torch

    from prestozl_b200 import build

    build.build()
    torch.cuda.set_device(0)
    spec_np = make_spectrum(7, "cuda").cpu().numpy()
    rng = np.random.default_rng(5)
    cands = []
    for nh in (16, 8, 4, 2):
        for _ in range(args.extras_cands):
            r = float(rng.integers(40000 * nh, (1 << 24) - 40000)) / (2 * nh) * 2
            cands.append({"numharm": nh, "r": r,
                          "z": float(rng.integers(-ZMAX // 2, ZMAX // 2 + 1)) * 2 / nh,
                          "w": float(rng.integers(-WMAX // 20, WMAX // 20 + 1)) * 20 / nh})
    pol = polish_leg(spec_np, cands, max_cands=len(cands))
    prep = input_prep_leg("cuda", reps=args.extras_reps)
    prep["frac_of_hbm"] = prep["achieved_gbs"] / peaks()[0]
    dedisp = dedisp_leg("cuda", reps=args.extras_reps)
    print(json.dumps({"impl": "ours", "mode": "extras-only", "input_prep": prep, "polish": pol,
                      "dedisp": dedisp}))


def reference_gpu(spec_np):
    """The reference's own GPU search stage (accelsearch_cu: accel_kernels.cu +
    cuFFT, compiled for sm_100a from its sources into oracle/_ref) on one
    spectrum on this GPU, -batchsize 8: the plain reference on B200."""
    from oracle import bindings as ob
    from prestozl_b200 import synth

    if not os.path.exists(getattr(ob, "REFGPU_CLI", "")):
        return None
    with tempfile.TemporaryDirectory() as tmp:
        synth.write_fft(os.path.join(tmp, "paper"), spec_np, N_SAMPLES, DT)
        ob.quiet_wisdom()
        try:
            out = subprocess.run([ob.REFGPU_CLI, "-zmax", str(ZMAX), "-wmax", str(WMAX),
                                  "-numharm", str(NUMHARM), "-sigma", str(SIGMA),
                                  "-batchsize", "8", "paper.fft"],
                                 cwd=tmp, capture_output=True, text=True, timeout=900)
            rec = json.loads([x for x in out.stderr.splitlines() if "refgpu_search_s" in x][-1])
        except Exception as exc:  # reported, never required
            return {"value": None, "error": str(exc)[:200]}
    return {"value": 3600.0 / rec["refgpu_search_s"], "unit": UNIT,
            "search_s": rec["refgpu_search_s"], "candidates": rec["ncands"], "batchsize": 8,
            "what": "the reference's accelsearch_cu GPU stage (cuFFT), built for sm_100a, "
                    "wall time of accelsearch_GPU on the same spectrum and GPU"}


def run_reference(args):
    """--impl reference: the reference CPU search on this host's cores, one
    single-threaded search process per core.  A step is one bounded sample:
    every process searches the first n rsteps of the paper-scale spectrum
    (n calibrated so that a step takes about --ref-step-seconds);
    ms_per_step is that step's wall time, and value counts the spectra the
    step covered (processes x n / rsteps per spectrum)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import bindings as ob

    if not ob.have_reference():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref not built (reference sources absent)"}))
        return
    spec = make_spectrum(7, "cpu").numpy()
    nrsteps = ref_geometry(spec)
    procs = ref_processes()
    times, n, _ = reference_sample(spec, procs, args.ref_step_seconds, steps=args.steps,
                                   warmup=args.warmup)
    t = statistics.mean(times)
    spectra_per_step = procs * n / nrsteps
    value = spectra_per_step / t * 3600.0
    sample = (f"{procs} single-threaded reference searches at once (one per core, the "
              f"reference's xargs -P mode), each over the first {n} rsteps of the same "
              f"spectrum: {spectra_per_step:.4f} spectra per step of {nrsteps} rsteps; "
              f"FFT = project FFTW stand-in (scalar double precision)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1000.0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": workload_config(args.gpus, nrsteps),
        "sample": sample,
        "step_ms": [x * 1000.0 for x in times],
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def _count_rsteps(obs) -> int:
    rstep = obs.corr_uselen // 2
    n, startr = 0, obs.rlo
    while startr + rstep < obs.highestbin:
        n += 1
        startr += rstep
    return n


# --------------------------------------------------------------------------
# The batched workload: 48 spectra of uneven length and geometry.

MIX_LENGTHS = (1 << 22, 1 << 24, 1 << 25)
MIX_GEOMS = ((50, 160), (200, 300), (100, 0))
MIX_SIGMA = 3.0


def mix_workload(n: int = 48):
    """(N, zmax, wmax, numharm, seed) per spectrum: lengths 2^22 / 2^24 /
    2^25 in turn, the three (zmax, wmax) pairs and numharm 8 / 16 spread over
    them (16 spectra of each length; every combination occurs)."""
    return [(MIX_LENGTHS[i % 3], *MIX_GEOMS[(i // 3) % 3], (8, 16)[(i // 9) % 2], 7000 + i)
            for i in range(n)]


def mix_spectrum(N: int, zmax: int, wmax: int, seed: int, device):
    """Seeded Gaussian noise with 0-2 pulsars (up to 5 harmonics, SNR 8-20)
    inside the geometry's f-dot / f-dot-dot range."""
    from prestozl_b200 import synth

    rng = np.random.default_rng(seed)
    ps = synth.random_pulsars(rng, int(rng.integers(0, 3)), zmax=0.9 * zmax,
                              wmax=0.9 * wmax if wmax else 0.0, snr=(8.0, 20.0), maxharm=5)
    return synth.presto_fft_torch(synth.timeseries_torch(N, DT, ps, seed, device=device))


def mix_leg(args, local: int):
    """The batched workload three ways, on resident kernel banks:
    plain drop-in -- what accelsearch_GPU does per spectrum: a plan at
    -batchsize 8, the host spectrum copied in, the search, the plan freed;
    sequential -- one search at a time at args.mix_batch rsteps per batch,
    spectra and plans resident; batched -- the request loop, every spectrum
    submitted at once, args.mix_active searches in flight advanced in waves
    of merged launches.  Each mode's lists must equal the plain drop-in's."""
    import torch

    from prestozl_b200 import jerk

    work = mix_workload(args.mix_spectra)
    specs = [mix_spectrum(N, z, w, seed, "cuda") for N, z, w, nh, seed in work]
    torch.cuda.synchronize()
    geo, banks = [], {}
    for (N, z, w, nh, seed), sp in zip(work, specs):
        obs, fftlen, _ = jerk.obs_from_params(N // 2, N, DT, z, w, nh, MIX_SIGMA)
        subs = jerk.subharm_sizes(obs, fftlen)
        key = (z, w, nh)
        if key not in banks:
            banks[key] = jerk.DeviceBank(subs)
        geo.append((obs, subs, key))
    torch.cuda.synchronize()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1000.0, out

    host = [sp.cpu().numpy() for sp in specs]

    def plain_dropin():
        res = []
        for (obs, subs, key), hs in zip(geo, host):
            p = jerk.JerkPlan(obs, subs, batch=8, device_bank=banks[key].ptr.value)
            res.append(p.search(hs))
            p.close()
        return res

    def sequential():
        plans, res = {}, []
        for (obs, subs, key), sp in zip(geo, specs):
            k = (key, obs.numbins)
            if k not in plans:
                plans[k] = jerk.JerkPlan(obs, subs, batch=args.mix_batch,
                                         device_bank=banks[key].ptr.value)
            res.append(plans[k].search(sp))
        for p in plans.values():
            p.close()
        return res

    srv = jerk.JerkServer(max_active=args.mix_active, batch=args.mix_batch, device=local)
    # warm: one request per geometry builds the server's resident banks
    seen = {}
    for i, (N, z, w, nh, seed) in enumerate(work):
        seen.setdefault((z, w, nh), i)
    for i in seen.values():
        N, z, w, nh, _ = work[i]
        srv.submit(specs[i], N, DT, z, w, nh, MIX_SIGMA, tag=10 ** 6 + i)
    for _ in seen:
        srv.poll(600000)

    def batched():
        for i, ((N, z, w, nh, seed), sp) in enumerate(zip(work, specs)):
            srv.submit(sp, N, DT, z, w, nh, MIX_SIGMA, tag=i)
        res = [None] * len(work)
        for _ in work:
            r = srv.poll(600000)
            if r is None:
                raise RuntimeError("batched workload stalled")
            res[r[0]] = r[1]
        return res

    t_drop, r_drop = timed(plain_dropin)
    t_seq, r_seq = timed(sequential)
    t_bat, r_bat = timed(batched)
    srv.close()
    for b in banks.values():
        b.close()

    def same(a, b):
        return len(a) == len(b) and all(np.array_equal(a[f], b[f]) for f in a.dtype.names)

    equal = all(same(a, b) and same(a, c) for a, b, c in zip(r_drop, r_seq, r_bat))
    n = len(work)
    return {"workload": f"{n} spectra: 16 each of 2^22 / 2^24 / 2^25 samples (dt 54.6 us), "
                        "(zmax, wmax) in (50, 160), (200, 300), (100, 0), numharm 8 / 16, "
                        f"sigma {MIX_SIGMA}",
            "plain_dropin": {"value": n / t_drop * 3600.0, "s": t_drop, "batch_rsteps": 8},
            "sequential": {"value": n / t_seq * 3600.0, "s": t_seq,
                           "batch_rsteps": args.mix_batch},
            "batched": {"value": n / t_bat * 3600.0, "s": t_bat, "batch_rsteps": args.mix_batch,
                        "in_flight": args.mix_active,
                        "form": "request loop, all spectra submitted at once, waves of merged "
                                "launches"},
            "speedup_vs_plain_dropin": t_drop / t_bat,
            "speedup_vs_sequential": t_seq / t_bat,
            "candidates": int(sum(len(r) for r in r_drop)),
            "equal_results": bool(equal),
            "timing": "CUDA events around each whole mode"}


# --------------------------------------------------------------------------
# The served stream: dedispersion trials arriving at 40 per second, with a
# memory-heavy spectrum mixed in.

HEAVY_TAG = 999999


def stream_leg(args, local: int):
    """A bounded sample of the served stream: args.stream_trials consecutive
    dedispersion trials (2^24 samples each, zmax 200, wmax 300, numharm 16)
    around the DM index where a pulsar peaks (it is in 6 of them, SNR
    falling as a Gaussian of sigma 3 trials), arriving as a Poisson process
    at 40 per second, plus one memory-heavy request (a 2^25-sample red-noise
    time series with 20 birdies, prepared, zapped and searched at zmax 300,
    wmax 600, numharm 32, sigma 4) arriving mid-stream, under a 150 GB
    device budget.  Latencies are from submission to result (queue and
    service) and from admission to result (service)."""
    import torch

    from prestozl_b200 import jerk, synth

    Nt, peak, sig_trials = 1 << 24, 288, 3.0
    first = peak - args.stream_trials // 2
    trials = list(range(first, first + args.stream_trials))
    rng = np.random.default_rng(4040)
    base = synth.random_pulsars(np.random.default_rng(88), 1, zmax=150.0, wmax=250.0,
                                snr=(20.0, 20.0), maxharm=4)[0]
    specs = []
    for t in trials:
        ps = []
        if abs(t - peak) <= 2 or t == peak + 3:  # the 6 trials that carry it
            snr = 20.0 * float(np.exp(-0.5 * ((t - peak) / sig_trials) ** 2))
            ps = [synth.Pulsar(base.f, base.z, base.w, snr, base.nharm, base.phase)]
        specs.append(synth.presto_fft_torch(synth.timeseries_torch(Nt, DT, ps, 9000 + t,
                                                                   device="cuda")))
    Nh = 1 << 25
    birds = synth.memory_heavy_birdies()
    heavy = torch.from_numpy(synth.red_noise_timeseries(Nh, DT, 505, birdies=birds)).cuda()
    Th = Nh * DT
    lob = sorted((f - 0.0015) * Th for f in birds)
    hib = sorted((f + 0.0015) * Th for f in birds)
    small_heavy = torch.from_numpy(synth.red_noise_timeseries(1 << 20, DT, 506)).cuda()
    torch.cuda.synchronize()

    srv = jerk.JerkServer(hbm_budget_bytes=150 * 10 ** 9, max_active=args.stream_active,
                          batch=args.stream_batch, device=local)
    # warm: the two geometries' banks (a short series of the heavy one)
    srv.submit(specs[0], Nt, DT, 200, 300, 16, 3.0, tag=10 ** 6)
    srv.submit(small_heavy, 1 << 20, DT, 300, 600, 32, 4.0, tag=10 ** 6 + 1, timeseries=True)
    for _ in range(2):
        srv.poll(600000)
    s0 = srv.stats()

    arrivals = np.cumsum(rng.exponential(1.0 / 40.0, len(trials) + 1))
    heavy_at = len(trials) // 2
    order = list(range(len(trials)))
    order.insert(heavy_at, -1)
    t0 = time.perf_counter()
    submitted, results, best = 0, {}, {}
    t_sub = {}
    while len(results) < len(order):
        now = time.perf_counter() - t0
        while submitted < len(order) and arrivals[submitted] <= now:
            k = order[submitted]
            if k < 0:
                srv.submit(heavy, Nh, DT, 300, 600, 32, 4.0, tag=HEAVY_TAG, timeseries=True,
                           birdies=(lob, hib))
            else:
                srv.submit(specs[k], Nt, DT, 200, 300, 16, 3.0, tag=k)
            submitted += 1
        wait_ms = 1 if submitted < len(order) else 1000
        r = srv.poll(wait_ms)
        if r is not None:
            tag, cands, t = r
            results[tag] = t
            if tag < len(trials):
                best[trials[tag]] = float(cands["sigma"].max()) if len(cands) else 0.0
    t_end = time.perf_counter() - t0
    s1 = srv.stats()
    srv.close()
    tl = [results[k] for k in range(len(trials))]
    total = [(t["done"] - t["submit"]) * 1000.0 for t in tl]
    service = [(t["done"] - t["start"]) * 1000.0 for t in tl]
    h = results[HEAVY_TAG]
    n = len(order)
    return {"workload": f"{len(trials)} dedispersion trials (2^24 samples, zmax 200 wmax 300 "
                        "numharm 16 sigma 3) around the DM of a pulsar that is in 6 of them, "
                        "Poisson arrivals at 40/s, plus one memory-heavy time series "
                        "(2^25 samples, red noise + 20 birdies zapped, zmax 300 wmax 600 "
                        "numharm 32 sigma 4) arriving mid-stream; 150 GB device budget",
            "value": n / t_end * 3600.0, "unit": UNIT, "wall_s": t_end,
            "arrival_span_s": float(arrivals[len(order) - 1]),
            "latency_ms": {"p50": float(np.percentile(total, 50)),
                           "p99": float(np.percentile(total, 99)),
                           "service_p50": float(np.percentile(service, 50)),
                           "service_p99": float(np.percentile(service, 99)),
                           "heavy": (h["done"] - h["submit"]) * 1000.0},
            "peak_device_bytes": s1["peak_bytes"], "budget_bytes": s1["budget"],
            "max_in_flight": args.stream_active, "batch_rsteps": args.stream_batch,
            "h2d_bytes": s1["h2d_bytes"] - s0["h2d_bytes"],
            "d2h_bytes": s1["d2h_bytes"] - s0["d2h_bytes"],
            "best_sigma_by_trial": best,
            "timing": "host wall clock from the first arrival to the last result; latencies "
                      "from the server's own submit / start / done times"}


# --------------------------------------------------------------------------

def run_served(srv, spectra, dev: bool, device_events: bool = True):
    """Submit every spectrum at once to the server and wait for all results.
    Returns (job seconds on the device timeline, per-request service and
    queueing latencies in ms, candidates per spectrum)."""
    import torch

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for i, sp in enumerate(spectra):
        srv.submit(sp, N_SAMPLES, DT, ZMAX, WMAX, NUMHARM, SIGMA, tag=i)
    service, total, ncand = [], [], []
    for _ in spectra:
        r = srv.poll(600000)
        if r is None:
            raise RuntimeError("served search stalled")
        tag, cands, t = r
        service.append((t["done"] - t["start"]) * 1000.0)
        total.append((t["done"] - t["submit"]) * 1000.0)
        ncand.append(len(cands))
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1000.0, service, total, ncand


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4,
                    help="spectra per timed job (plain: sequential searches; served: one burst)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=0,
                    help="rsteps per batch (0: autotuned per geometry, cached)")
    ap.add_argument("--max-active", type=int, default=3, help="served: searches in flight")
    ap.add_argument("--ref-step-seconds", type=float, default=5.0,
                    help="--impl reference: wall seconds per timed step (rsteps calibrated)")
    ap.add_argument("--ref-seconds", type=float, default=10.0,
                    help="cpu_baseline of the GPU arm: wall seconds of its one timed step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the input-preparation and candidate-polishing legs")
    ap.add_argument("--extras-only", action="store_true",
                    help="only the input-preparation and polishing legs (small footprint)")
    ap.add_argument("--dedisp-only", action="store_true",
                    help="only the subband-dedispersion leg (one block; the form profiled "
                         "with ncu)")
    ap.add_argument("--extras-cands", type=int, default=4,
                    help="--extras-only: candidates per harmonic count (16, 8, 4, 2)")
    ap.add_argument("--extras-reps", type=int, default=5,
                    help="--extras-only: timed input preparations")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--no-mix", action="store_true",
                    help="skip the batched workload of uneven spectra")
    ap.add_argument("--mix-only", action="store_true",
                    help="only the batched workload and the served stream")
    ap.add_argument("--mix-spectra", type=int, default=48)
    ap.add_argument("--mix-batch", type=int, default=32)
    ap.add_argument("--mix-active", type=int, default=12)
    ap.add_argument("--no-stream", action="store_true", help="skip the served stream")
    ap.add_argument("--stream-trials", type=int, default=16)
    ap.add_argument("--stream-active", type=int, default=16,
                    help="served stream: searches in flight at most (the 150 GB budget "
                         "binds first at the default batch)")
    ap.add_argument("--stream-batch", type=int, default=64)
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip timing the reference's own GPU search on this GPU")
    ap.add_argument("--e2e-steps", type=int, default=0)
    ap.add_argument("--rsteps", type=int, default=0,
                    help="search only the first R rsteps of each spectrum (profiling runs; "
                         "the line is then marked partial and the served legs are skipped)")
    args = ap.parse_args()

    if args.impl == "reference":
        run_reference(args)
        return
    if args.dedisp_only:
        import torch

        from prestozl_b200 import build

        build.build()
        torch.cuda.set_device(0)
        print(json.dumps({"impl": "ours", "mode": "dedisp-only",
                          "dedisp": dedisp_leg("cuda", reps=args.extras_reps)}))
        return
    if args.extras_only:
        run_extras(args)
        return
    if args.mix_only:
        import torch

        from prestozl_b200 import build

        build.build()
        torch.cuda.set_device(0)
        out = {"impl": "ours", "mode": "mix-only"}
        if not args.no_mix:
            out["batched_mix"] = mix_leg(args, 0)
        if not args.no_stream:
            out["served_stream"] = stream_leg(args, 0)
        print(json.dumps(out))
        return

    import torch

    from prestozl_b200 import replicas

    env = replicas.rank_env()
    rank, world, local = env.rank, env.world, env.local
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    from prestozl_b200 import build, jerk
    build.build()

    obs, fftlen, subs = paper_setup()
    bank = jerk.DeviceBank(subs)

    # this rank's spectra, resident in HBM (each larger than L2)
    nspec = max(2, args.steps)
    specs = [make_spectrum(1000 * rank + i, "cuda") for i in range(nspec)]
    torch.cuda.synchronize()

    tuned = None
    harm_mode = 0
    if args.batch <= 0:
        from prestozl_b200 import autotune
        tuned = autotune.tune(obs, subs, bank.ptr.value, specs[0])
        args.batch = tuned["batch_rsteps"]
        harm_mode = tuned.get("harm_mode", 0)
    plan = jerk.JerkPlan(obs, subs, batch=args.batch, device_bank=bank.ptr.value,
                         harm_mode=harm_mode)
    nrsteps = plan.num_rsteps
    nsearch = args.rsteps if args.rsteps > 0 else 0
    served = not args.no_served and not nsearch

    def barrier():
        if dist is not None:
            dist.barrier()

    for i in range(args.warmup):
        plan.search(specs[i % nspec], 0, nsearch)
    torch.cuda.synchronize()

    # ---- plain: one spectrum per search call, sequentially
    sampler = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    step_ms, ncands = [], []
    t_all0 = time.perf_counter()
    for i in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        c = plan.search(specs[i % nspec], 0, nsearch)
        e1.record()
        torch.cuda.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        ncands.append(len(c))
        if i == 0:
            cands0 = c
    torch.cuda.synchronize()
    barrier()
    plain_wall = time.perf_counter() - t_all0
    plain_s = replicas.max_over_ranks(sum(step_ms) / 1000.0, dist, "cuda")
    plain_value = world * args.steps / plain_s * 3600.0

    # ---- batched under a captured CUDA graph: the same searches, each pass
    # replayed from one graph (captured on the warm-up call)
    graph_info = None
    if not nsearch:
        gplan = jerk.JerkPlan(obs, subs, batch=args.batch, device_bank=bank.ptr.value,
                              harm_mode=harm_mode, use_graph=True)
        gplan.search(specs[0], 0, nsearch)
        torch.cuda.synchronize()
        barrier()
        g_ms = []
        for i in range(min(args.steps, 4)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            gplan.search(specs[i % nspec], 0, nsearch)
            e1.record()
            torch.cuda.synchronize()
            g_ms.append(e0.elapsed_time(e1))
        gplan.close()
        g_s = replicas.max_over_ranks(sum(g_ms) / 1000.0, dist, "cuda")
        graph_info = {"value": world * len(g_ms) / g_s * 3600.0,
                      "ms_per_spectrum": statistics.mean(g_ms)}

    # ---- plain drop-in: what accelsearch_GPU does per spectrum -- allocate a
    # plan (-batchsize 8, the reference's default) over the kernel bank it keeps
    # resident between calls of one geometry, copy the host spectrum, search,
    # build the list, free the plan
    dropin = None
    if served:
        hspec = [specs[i % nspec].cpu().numpy() for i in range(2)]
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for hs in hspec:
            p1 = jerk.JerkPlan(obs, subs, batch=8, device_bank=bank.ptr.value)
            p1.search(hs)
            p1.close()
        e1.record()
        torch.cuda.synchronize()
        dropin_s = replicas.max_over_ranks(e0.elapsed_time(e1) / 1000.0, dist, "cuda")
        dropin = {"value": world * len(hspec) / dropin_s * 3600.0,
                  "ms_per_spectrum": dropin_s * 1000.0 / len(hspec), "batch_rsteps": 8,
                  "bank": "resident on the device, as the drop-in keeps it"}

    # ---- served: the request loop, every spectrum of the job submitted at once
    served_info = None
    if served:
        srv = jerk.JerkServer(max_active=args.max_active, batch=args.batch, device=local,
                              harm_mode=harm_mode)
        run_served(srv, specs[:1], True)  # warm: bank + plans
        barrier()
        job_s, service, total, ncand_s = run_served(srv, specs[: args.steps], True)
        barrier()
        srv.close()
        job_s = replicas.max_over_ranks(job_s, dist, "cuda")
        served_info = {"value": world * args.steps / job_s * 3600.0, "job_s": job_s,
                       "service_ms": service, "queue_and_service_ms": total,
                       "candidates": ncand_s}
    clocks = sampler.stop()

    # ---- e2e: spectra in pinned host memory through the public API
    e2e_steps = args.e2e_steps or (args.steps if served else max(1, min(args.steps, 2)))
    host = [specs[i % nspec].cpu().pin_memory() for i in range(e2e_steps)]
    hnp = [h.numpy() for h in host]
    barrier()
    if served:
        srv = jerk.JerkServer(max_active=args.max_active, batch=args.batch, device=local,
                              harm_mode=harm_mode)
        run_served(srv, hnp[:1], False)
        st0 = srv.stats()
        e2e_s, _, _, _ = run_served(srv, hnp, False)
        st1 = srv.stats()
        srv.close()
        # the served path's own copies: host spectra in, hit counts and lists out
        h2d = st1["h2d_bytes"] - st0["h2d_bytes"]
        d2h = st1["d2h_bytes"] - st0["d2h_bytes"]
    else:
        plan.reset_stats()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for i in range(e2e_steps):
            plan.search(hnp[i], 0, nsearch)
        e1.record()
        torch.cuda.synchronize()
        e2e_s = e0.elapsed_time(e1) / 1000.0
        h2d, d2h = plan.transfer_stats()
    e2e_s = replicas.max_over_ranks(e2e_s, dist, "cuda")
    e2e_value = world * e2e_steps / e2e_s * 3600.0

    # ---- roofline: one profiled search (CUDA events around every launch)
    plan.reset_stats()
    plan.set_profiling(True)
    plan.search(specs[0], 0, nsearch)
    torch.cuda.synchronize()
    plan.set_profiling(False)
    kstats = plan.kernel_stats()
    dom = max(kstats.items(), key=lambda kv: kv[1]["ms"])
    dname, d = dom
    launches = max(d["launches"], 1)
    per_launch_s = d["ms"] / 1000.0 / launches
    achieved = d["bytes"] / launches / per_launch_s / 1e9
    fp32_achieved = d["flops"] / launches / per_launch_s / 1e12
    traffic = corr2048_traffic(args.batch) if dname == "corr_2048" else None
    peak, peak_kind = peaks()
    hs = kstats.get("harmsum")
    harmsum_roofline = None
    if hs and hs["ms"] > 0:
        hs_gbs = hs["bytes"] / (hs["ms"] / 1000.0) / 1e9
        harmsum_roofline = {"bound": "hbm", "kernel": "harmsum", "achieved": hs_gbs,
                            "peak": peak, "unit": "GB/s", "frac": hs_gbs / peak,
                            "peak_source": peak_kind,
                            "algorithmic": "every volume of the batch read once"}
    launches_per_spectrum = sum(v["launches"] for v in kstats.values())

    # ---- next to the search: input preparation and candidate polishing
    extras = {}
    if not args.no_extras:
        extras["input_prep"] = input_prep_leg("cuda")
        extras["input_prep"]["frac_of_hbm"] = extras["input_prep"]["achieved_gbs"] / peaks()[0]
        try:
            extras["dedisp"] = dedisp_leg("cuda")
        except Exception as e:  # a side leg: report it, keep the search's line
            extras["dedisp"] = {"error": f"{type(e).__name__}: {e}"}
        spec0_np = specs[0].cpu().numpy()
        extras["polish"] = polish_leg(spec0_np, cands0)
    if not nsearch and world == 1:
        # the other workloads of the batched and served forms (1 GPU)
        for name, skip, fn in (("batched_mix", args.no_mix, mix_leg),
                               ("served_stream", args.no_stream, stream_leg)):
            if skip:
                continue
            try:
                extras[name] = fn(args, local)
            except Exception as e:  # a side leg: report it, keep the headline line
                extras[name] = {"error": f"{type(e).__name__}: {e}"}
    timed_spectra = args.steps * (2 if served else 1)

    value = served_info["value"] if served else plain_value
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": (served_info["job_s"] * 1000.0 / args.steps) if served
            else statistics.mean(step_ms),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": workload_config(world, nrsteps, nsearch),
            "run": {"batch_rsteps": args.batch, "batch_autotune": tuned,
                    "form": ("served: one request loop per GPU, all step spectra submitted "
                             f"at once, {args.max_active} in flight, shared resident bank")
                    if served else "plain: one spectrum per search call",
                    "timing": "CUDA events on the device timeline around the whole job "
                              "(served) or each search (plain); max over ranks"},
            "batched_graph": graph_info,
            "plain": {"value": plain_value, "ms_per_spectrum": statistics.mean(step_ms),
                      "p50_ms": float(np.percentile(step_ms, 50)),
                      "p99_ms": float(np.percentile(step_ms, 99))},
            "latency_ms": ({"p50": float(np.percentile(served_info["service_ms"], 50)),
                            "p99": float(np.percentile(served_info["service_ms"], 99)),
                            "p50_with_queue": float(np.percentile(
                                served_info["queue_and_service_ms"], 50)),
                            "p99_with_queue": float(np.percentile(
                                served_info["queue_and_service_ms"], 99))}
                           if served else
                           {"p50": float(np.percentile(step_ms, 50)),
                            "p99": float(np.percentile(step_ms, 99))}),
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": int(h2d // e2e_steps),
                    "d2h_bytes_per_step": int(d2h // e2e_steps)},
            "roofline": {"bound": "hbm", "kernel": dname, "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind, "traffic": traffic,
                         "traffic_source": "ncu capture of corr_fold_kernel at 16 rsteps per "
                                           "batch, write side scaled by rsteps per batch"
                                           if traffic else None,
                         "fp32": {"achieved": fp32_achieved, "peak": FP32_PEAK_TFLOPS,
                                  "unit": "TFLOP/s", "frac": fp32_achieved / FP32_PEAK_TFLOPS,
                                  "peak_source": "nominal (148 SMs x 128 lanes x 2 x 1965 MHz)"},
                         "note": "the correlation kernels are FP32-issue bound: the HBM "
                                 "fraction is what they leave of the memory roofline"},
            "roofline_harmsum": harmsum_roofline,
            "kernels": {k: {"launches": v["launches"], "ms": v["ms"],
                            "share": v["ms"] / max(sum(x["ms"] for x in kstats.values()), 1e-9),
                            "gbs": v["bytes"] / max(v["ms"], 1e-9) / 1e6,
                            "tflops": v["flops"] / max(v["ms"], 1e-9) / 1e9}
                        for k, v in kstats.items()},
            "gpu_launches": launches_per_spectrum * timed_spectra,
            "clocks": clocks,
            "wall_s": plain_wall,
            "candidates_per_spectrum": ncands,
        }
        line.update(extras)
        if served:
            line["plain_dropin"] = dropin
            line["speedup_vs_plain"] = value / plain_value
            line["speedup_vs_plain_dropin"] = value / dropin["value"]
        if world == 1 and not args.no_cpu_baseline and not nsearch:
            try:
                from oracle import bindings as ob
                if ob.have_reference():
                    spec_np = specs[0].cpu().numpy()
                    procs = ref_processes()
                    times, n, pol = reference_sample(
                        spec_np, procs, args.ref_seconds,
                        polish_cands=cands0 if line.get("polish") else None)
                    cpu_val = procs * n / nrsteps / times[0] * 3600.0
                    line["cpu_baseline"] = {
                        "value": cpu_val, "unit": UNIT, "cores": procs, "kind": "reference",
                        "sample": f"{procs} single-threaded reference searches at once (one "
                                  f"per core), each over the first {n} rsteps of one spectrum "
                                  f"({times[0]:.1f} s); FFT = project FFTW stand-in"}
                    if pol:
                        line["cpu_baseline"]["polish"] = pol
                        line["polish"]["speedup_vs_reference_cpu"] = (
                            pol["s_per_candidate"] * 1000.0 / line["polish"]["ms_per_candidate"])
            except Exception as exc:  # the baseline is reported, never required
                line["cpu_baseline"] = {"value": None, "unit": UNIT, "error": str(exc)}
        if world == 1 and not args.no_ref_gpu and not nsearch:
            ref_gpu = reference_gpu(specs[0].cpu().numpy())
            if ref_gpu:
                line["reference_gpu"] = ref_gpu
                if ref_gpu.get("value"):
                    line["speedup_vs_reference_gpu"] = value / ref_gpu["value"]
        print(json.dumps(line))

    plan.close()
    bank.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
