"""Benchmark of the displacement hot path: atoms/s with all loops and images.

Default workload: fcc_random (FCC a0 3.615 A, 150^3 cells = 13.5 M atoms, 64
glide loops = 1696 segments, images +-2 = 125, nu 0.34), FP64 line method, one
GPU.  A step is one full displacement sum over all atoms.

  value   device-resident: positions and displacements already in HBM, one
          plan execute per step (CUDA events on the launching stream, max over
          ranks).  Inputs (324 MB of positions) are larger than L2.
  e2e     the public host call (kroupa_gpu, the kroupaGPU drop-in) on pinned
          host arrays: table build, allocation, H2D of positions and
          displacements, kernel, D2H of the displacements, per step.
  roofline  W = 128 flop per segment-image evaluation (66 per loopon-image)
          against the FP64 peak measured here with a DGEMM (the driver's peak
          file has no FP64 figure); traffic from the committed ncu summary.
  cpu_baseline  the oracle (CPU restatement, the reference's flags) on a
          seeded atom sample, all host threads, rank 0 only.

--impl reference times the reference's CPU implementation on the same
workload: its own kroupaCPU compiled from its sources (oracle/_ref) where the
workload has the reference's fixed images +-1, else the oracle restatement of
it (images and nu are compile-time constants in the reference).

Multi-GPU (torchrun): every rank runs the same workload on its own GPU
(replicas, weak scaling, no collective on the data path); value = all ranks'
atoms / max-over-ranks time.
"""
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

METRIC = "atoms/s with all loops+images; learned/FP32 vs plain FP64 at max |Δu|≤1e-3 Å"
W_LINE = 128.0     # flop per segment-image evaluation
W_LOOPON = 66.0    # flop per loopon-image evaluation


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", default="fcc_random")
    p.add_argument("--precision", default=None, choices=["fp64", "fp32c"],
                   help="default: fp64, fp32c for the batch workload")
    p.add_argument("--e2e-steps", type=int, default=None)
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--image-split", type=int, default=0)
    p.add_argument("--samples", type=int, default=256, help="batch workload: number of samples")
    p.add_argument("--images", type=int, default=None,
                   help="override the workload's image range (profiling of small cases)")
    p.add_argument("--retrain", action="store_true", help="learned: train the network even if cached")
    p.add_argument("--epochs", type=int, default=32, help="learned: training epochs over 2^22 samples")
    p.add_argument("--no-fp64", action="store_true", help="learned: skip the plain FP64 comparison run")
    p.add_argument("--no-output", action="store_true", help="skip the output-writer measurement")
    p.add_argument("--no-forms", action="store_true",
                   help="default workload: skip the fp32c, learned and bcc_prismatic keys")
    p.add_argument("--kernel-only", action="store_true",
                   help="time the device-resident steps only (no e2e, output, forms, CPU): for profiling")
    return p.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), \
        int(os.environ.get("LOCAL_RANK", 0))


L2_BYTES = 126 * 2 ** 20


class L2Flush:
    """Rewrites a 256 MB buffer (twice the L2) between timed steps when a
    workload's inputs would fit in L2; a no-op otherwise."""

    def __init__(self, torch, input_bytes):
        self.on = input_bytes < L2_BYTES
        self.buf = torch.empty(256 * 2 ** 20, dtype=torch.uint8, device="cuda") if self.on else None

    def __call__(self):
        if self.on:
            self.buf.fill_(1)

    def note(self, input_bytes):
        return l2_note(input_bytes)


def l2_note(input_bytes):
    return (f"L2 flushed between timed steps (inputs {input_bytes / 1e6:.0f} MB < L2)" if input_bytes < L2_BYTES
            else f"inputs larger than L2 ({input_bytes / 1e6:.0f} MB)")


def timed_steps(torch, step, steps, stream, flush):
    """Device seconds of `steps` calls of step() (CUDA events on the launching
    stream); with an active flush, L2 is rewritten before each step outside
    the events."""
    if not flush.on:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) * 1e-3
    total = 0.0
    for _ in range(steps):
        flush()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1) * 1e-3
    return total


def measured_peaks():
    """The pool's measured peaks (HBM copy GB/s, BF16 TFLOP/s) from
    MEASURED_PEAKS.json beside this file, or None."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return json.load(open(path))
    except (OSError, ValueError):
        return None


def max_over_ranks(value, world, device="cuda"):
    """The largest of the ranks' values (every rank gets it); value itself when
    world == 1.  Timings of a multi-GPU run are the slowest rank's."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def build_workload(name, images=None, geom=None):
    from disco_b200 import workloads as W
    w = W.FULL[name](geom=geom)
    if images is not None:
        w.images = images
    return w


def arm_config(args, w, precision, n_segments, n_loopons, image_min=0):
    """The `config` of a bench line, the same for both arms."""
    W_ = 2 * w.images + 1
    inner = 2 * image_min - 1 if image_min > 0 else 0
    return {"workload": args.config, "atoms": w.n, "loops": len(w.loops), "segments": int(n_segments),
            "loopons": int(n_loopons), "images": W_ ** 3 - inner ** 3, "nu": w.nu, "method": w.method,
            "precision": precision, "l2": l2_note(48 * w.n), "parallelism": f"replicas x{args.gpus}"}


def flop_per_eval(w):
    return W_LINE if w.method == "line" else W_LOOPON


class Clocks:
    """nvidia-smi samples during the timed region (every 200 ms)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def fp64_peak_tflops(torch):
    """Dense FP64 throughput of this GPU, measured with a DGEMM (best of 5)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def fp32_peak_tflops(torch):
    """Dense FP32 CUDA-core throughput, measured with an SGEMM without TF32
    (best of 5): the denominator of the FP32 kernels' roofline."""
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        n = 8192
        a = torch.randn(n, n, dtype=torch.float32, device="cuda")
        b = torch.randn(n, n, dtype=torch.float32, device="cuda")
        for _ in range(2):
            torch.matmul(a, b)
        torch.cuda.synchronize()
        best = 1e9
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1) * 1e-3)
        del a, b
        torch.cuda.empty_cache()
        return 2.0 * n ** 3 / best / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = old


def pipe_peak_tflops(torch, clk, fp64=True):
    """Peak of the CUDA-core FMA pipe a field kernel runs on: SMs x FMA lanes
    per SM per clock (64 FP64, 128 FP32 on B200) x 2 flop x the median SM
    clock sampled during the timed region (clocks.max.sm without samples).
    Returns (TFLOP/s, how it was derived)."""
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz, src = (clk or {}).get("sm_mhz"), "median SM clock sampled in the timed region"
    if not mhz:
        try:
            out = subprocess.run(["nvidia-smi", "-i", str(torch.cuda.current_device()),
                                  "--query-gpu=clocks.max.sm", "--format=csv,noheader,nounits"],
                                 capture_output=True, text=True, timeout=20).stdout
            mhz, src = float(out.strip().splitlines()[0]), "clocks.max.sm (no samples)"
        except Exception:
            mhz, src = 1965.0, "1965 MHz nominal (no clock reading)"
    lanes = 64 if fp64 else 128
    tf = sms * lanes * 2 * mhz * 1e6 / 1e12
    return tf, (f"{'FP64' if fp64 else 'FP32'} FMA pipe: {sms} SMs x {lanes} lanes x 2 flop x "
                f"{mhz:.0f} MHz ({src})")


def traffic_from_profiles(kernel_key):
    """DRAM bytes per launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"{kernel_key}.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.strip().startswith("traffic_per_launch_bytes:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


class quiet_stdout:
    """Sends file descriptor 1 to /dev/null for the duration (the reference's
    backends print progress lines with std::cout; the bench prints one JSON
    line)."""

    def __enter__(self):
        import ctypes
        sys.stdout.flush()
        self.libc = ctypes.CDLL(None)
        self.libc.fflush(None)
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *exc):
        self.libc.fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)
        return False


def reference_gpu(w, x, y, z, ours_u=None, reps=3):
    """The reference's own CUDA backend (Code/backend_cuda.cu, built for
    sm_100a in oracle/_ref) on the same GPU and atoms: kroupaGPU per call
    (allocation, upload, one launch and one device wait per loop, download,
    free: its host-buffer drop-in, like this library's e2e) and its own
    kernel time (host clock around the per-loop launches and waits), FP64 and
    --fp32, best of `reps`.  Images +-1 and nu 0.35 are fixed there; the
    cost does not depend on nu.  max_abs_du: against this library's FP64
    result on the same atoms when given (ours_u, shape (3, n))."""
    import oracle as O
    if not O.have_ref_cuda():
        return {"unavailable": "the reference's CUDA backend is not built here (oracle/_ref)"}
    if w.images != 1:
        return {"unavailable": "the reference's kernels fix the images at +-1"}
    n = len(x)
    evals = w.evals_per_atom() * n
    out = {"what": "kroupaGPU of Code/backend_cuda.cu built for sm_100a (nvcc -O3, its Makefile flags)",
           "atoms": n, "images": 27, "nu": 0.35}
    with quiet_stdout():
        O.ref_displace_gpu(x[:256], y[:256], z[:256], w.loops, w.box)          # context, module load
    for fp32 in (False, True):
        best_call, best_k, u = 1e30, 1e30, None
        for _ in range(reps):
            with quiet_stdout():
                t0 = time.perf_counter()
                u, t = O.ref_displace_gpu(x, y, z, w.loops, w.box, fp32=fp32)
                call = time.perf_counter() - t0
            best_call, best_k = min(best_call, call), min(best_k, float(t[1]))
        r = {"call_s": best_call, "kernels_s": best_k, "atoms_per_s": n / best_call,
             "kernel_atoms_per_s": n / best_k, "kernel_evals_per_s": evals / best_k}
        if ours_u is not None and not fp32:
            r["max_abs_du_vs_ours_fp64"] = float(max(np.abs(u[k] - ours_u[k]).max() for k in range(3)))
        out["fp32" if fp32 else "fp64"] = r
    return out


def cpu_baseline(w, seconds, use_reference):
    """Atoms/s of a CPU implementation on a seeded atom sample (all threads)."""
    import oracle as O
    rng = np.random.default_rng(1234)
    threads = os.cpu_count() or 1
    ref_ok = use_reference and w.images == 1 and O.have_ref()

    def run(idx):
        x, y, z = w.x[idx], w.y[idx], w.z[idx]
        t0 = time.perf_counter()
        if ref_ok:
            with quiet_stdout():
                u = O.ref_displace(x, y, z, w.loops, w.box)
        else:
            u = O.displace(x, y, z, w.loops, w.box, images=w.images, nu=w.nu, threads=threads)
        return time.perf_counter() - t0, u

    # calibrate: a small probe, then samples scaled to the target time (at most 3 runs)
    k = min(w.n, 4 * threads)
    idx = np.sort(rng.choice(w.n, size=k, replace=False))
    dt, u = run(idx)
    for _ in range(3):
        if dt >= 0.5 * seconds or k >= w.n:
            break
        k = int(min(w.n, max(2 * k, k * seconds / max(dt, 1e-3))))
        idx = np.sort(rng.choice(w.n, size=k, replace=False))
        dt, u = run(idx)
    kind = "reference" if ref_ok else "port"
    what = ("the reference's kroupaCPU compiled from its sources (oracle/_ref), nu fixed at 0.35 "
            "in the reference, same operation count") if ref_ok else \
        ("oracle restatement of kroupaCPU (Code/backend_cpu.cpp:28-99) with the workload's nu and "
         "image range, built with the reference's flags")
    return {"value": k / dt, "unit": "atoms/s", "cores": threads, "kind": kind,
            "sample": f"{k} seeded random atoms of {w.n}, all {len(w.loops)} loops x "
                      f"{(2 * w.images + 1) ** 3} images, {dt:.1f} s; {what}",
            "seconds": dt}, idx, u


def run_reference_batch(args):
    """Reference arm of the batch workload: the oracle restatement of kroupaCPU
    (the reference has no batched form: it runs samples one after another) on
    bounded samples of random batch samples, all host threads; the rate in
    evaluations/s is converted to atoms/s of the whole batch."""
    from disco_b200 import workloads as W
    import oracle as O
    threads = os.cpu_count() or 1
    batch = W.batch(nsamples=args.samples, geom=O.RefGeometry if O.have_ref() else None)
    n = sum(w.n for w in batch)
    evals = sum(w.n * w.evals_per_atom() for w in batch)
    rng = np.random.default_rng(99)
    per_step = max(8.0, min(25.0, 150.0 / max(1, args.steps + args.warmup)))
    times, done = [], []
    for s in range(args.warmup + args.steps):
        t_used, e_done = 0.0, 0.0
        while t_used < per_step:
            w = batch[rng.integers(len(batch))]
            k = min(w.n, max(8, int(2e8 / max(1.0, w.evals_per_atom()))))
            idx = np.sort(rng.choice(w.n, size=k, replace=False))
            t0 = time.perf_counter()
            O.displace(w.x[idx], w.y[idx], w.z[idx], w.loops, w.box, images=w.images, nu=w.nu, threads=threads)
            t_used += time.perf_counter() - t0
            e_done += k * w.evals_per_atom()
        if s >= args.warmup:
            times.append(t_used)
            done.append(e_done)
    rate = sum(done) / sum(times)
    value = rate * n / evals
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "atoms/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * n / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "batch", "samples": len(batch), "atoms": n, "evals_per_step": evals},
        "cpu_baseline": {"value": value, "unit": "atoms/s", "cores": threads, "kind": "port",
                         "sample": f"random atoms of random samples, {per_step:.0f} s per step; evaluations/s "
                                   "converted to the whole batch's atoms"},
        "e2e": {"value": value, "unit": "atoms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    if args.config == "batch":
        return run_reference_batch(args)
    import oracle as O
    # inputs built by the reference's own geometry code where it is compiled
    # here (lattice, mid-plane snap, loop class, polylines, loopon grids), so
    # that this arm runs nothing of this library
    geom = O.RefGeometry if O.have_ref() else None
    # the learned workload's reference is the exact sum over all 729 images (+-4)
    w = build_workload("fcc_random", 4, geom) if args.config == "learned" else \
        build_workload(args.config, args.images, geom)
    threads = os.cpu_count() or 1
    ref_ok = w.images == 1 and O.have_ref()
    rng = np.random.default_rng(99)

    def run(idx):
        t0 = time.perf_counter()
        if ref_ok:
            with quiet_stdout():
                O.ref_displace(w.x[idx], w.y[idx], w.z[idx], w.loops, w.box)
        else:
            O.displace(w.x[idx], w.y[idx], w.z[idx], w.loops, w.box, images=w.images, nu=w.nu,
                       threads=threads)
        return time.perf_counter() - t0

    # bounded sample per step so that warmup + steps stay within a few minutes:
    # a small probe, then samples scaled to the per-step target (at most 3 runs)
    per_step = max(8.0, min(25.0, 150.0 / max(1, args.steps + args.warmup)))
    k = min(w.n, 4 * threads)
    dt = run(np.sort(rng.choice(w.n, size=k, replace=False)))
    for _ in range(3):
        if dt >= 0.25 * per_step or k >= w.n:
            break
        k = int(min(w.n, max(2 * k, 0.5 * k * per_step / max(dt, 1e-3))))
        dt = run(np.sort(rng.choice(w.n, size=k, replace=False)))
    k = int(min(w.n, max(k, k * per_step / max(dt, 1e-3))))
    times = []
    for s in range(args.warmup + args.steps):
        dt = run(np.sort(rng.choice(w.n, size=k, replace=False)))
        if s >= args.warmup:
            times.append(dt)
    T = sum(times)
    value = k * args.steps / T
    kind = "reference" if ref_ok else "port"
    sample = (f"{k} seeded random atoms of {w.n} per step, all loops and images; inputs from "
              f"{'the reference geometry code (oracle/_ref)' if geom else 'this library geometry'}")
    nseg = sum(len(lp.vx) for lp in w.loops if lp.line)
    nlp = sum(len(lp.x) for lp in w.loops if not lp.line)
    if args.config == "learned":
        cfg = {"workload": "fcc_random_learned", "atoms": w.n, "loops": len(w.loops), "segments": nseg,
               "images": 729, "nu": w.nu}
    else:
        cfg = arm_config(args, w, args.precision, nseg, nlp)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "atoms/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * T / args.steps * (w.n / k), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": cfg,
        "extrapolated": {"sampled_atoms_per_step": k, "atoms": w.n, "timed_seconds": T,
                         "note": "each step times a seeded sample of the workload's atoms with all loops "
                                 "and images; value is the sample's atoms/s and ms_per_step that rate "
                                 "scaled to every atom (per-atom cost is uniform)"},
        "cpu_baseline": {"value": value, "unit": "atoms/s", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "atoms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


ELEMENTS = {("fcc", 3.615): "Cu", ("bcc", 2.855): "Fe", ("bcc", 3.165): "W"}


def write_output(w, pos, u, stream):
    """The output epilogue after the field, outside the timed step: final
    positions (disco_b200_finalize_resident: add u, wrap, shift) and the XYZ
    atom lines (disco_b200_format_atoms) on the device, then the text to
    pinned host memory; checked byte for byte against the oracle's stream
    formatting on the first 200 000 atoms, and the oracle's formatting rate on
    one host thread (the reference writes with one ofstream) for comparison."""
    import ctypes
    import torch
    import oracle as O
    from disco_b200 import _capi as C
    from disco_b200 import geometry as G
    lib = C.cuda_lib()
    n = pos.shape[1]
    elem = ELEMENTS.get(("fcc" if w.lattice == G.FCC else "bcc", round(w.a0, 3)), "X")
    fin = torch.empty((3, n), dtype=torch.float64, device="cuda")
    cap = 72 * n + 64
    text = torch.empty(cap, dtype=torch.uint8, device="cuda")
    host = torch.empty(cap, dtype=torch.uint8, pin_memory=True)
    box = (ctypes.c_double * 3)(*w.box)
    sp = ctypes.c_void_p(stream.cuda_stream)
    nbytes = ctypes.c_int64()

    def once():
        C.check(lib.disco_b200_finalize_resident(pos[0].data_ptr(), pos[1].data_ptr(), pos[2].data_ptr(),
                                                 u[0].data_ptr(), u[1].data_ptr(), u[2].data_ptr(), n, None, 0,
                                                 box, fin[0].data_ptr(), fin[1].data_ptr(), fin[2].data_ptr(),
                                                 None, None, None, sp), lib)
        C.check(lib.disco_b200_format_atoms(0, elem.encode(), fin[0].data_ptr(), fin[1].data_ptr(),
                                            fin[2].data_ptr(), n, text.data_ptr(), cap, ctypes.byref(nbytes), sp),
                lib)
        host[:nbytes.value].copy_(text[:nbytes.value], non_blocking=True)

    once()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    once()
    e1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    m = min(n, 200000)
    f = fin[:, :m].cpu().numpy()
    t1 = time.perf_counter()
    ref = O.format_atoms(0, elem, f[0], f[1], f[2])
    cpu_rate = m / (time.perf_counter() - t1)
    ok = bytes(host[:len(ref)].numpy()) == ref
    return {"what": "finalize + XYZ atom lines on the device + text to pinned host memory",
            "atoms": n, "bytes": int(nbytes.value), "ms": e0.elapsed_time(e1), "wall_ms": 1e3 * wall,
            "atoms_per_s": n / (e0.elapsed_time(e1) * 1e-3), "bytes_match_oracle_first_atoms": m if ok else 0,
            "cpu_oracle_atoms_per_s_1_thread": cpu_rate}


def fp32c_form(args, w, pos, u64, idx, uref):
    """The FP32 compensated form on the default workload's atoms: device-resident
    step time, roofline against the FP32 FMA pipe, max and RMS |du| against the
    plain FP64 result on every atom and against the oracle on the parity
    sample (idx, uref)."""
    import torch
    from disco_b200 import backend as B
    from disco_b200 import _capi as C
    stream = torch.cuda.current_stream()
    n = w.n
    plan = B.Plan(w.loops, w.box, precision=C.DISCO_FP32C, images=w.images, nu=w.nu, max_atoms=n)
    st = plan.stats()
    u = torch.zeros_like(pos)
    for _ in range(args.warmup):
        plan.execute(pos, u)
    plan.sync(stream.cuda_stream)
    flush = L2Flush(torch, 48 * n)
    clocks = Clocks(torch.cuda.current_device())
    torch.cuda.synchronize()
    clocks.start()
    el = timed_steps(torch, lambda: plan.execute(pos, u), args.steps, stream, flush)
    clk = clocks.stop()
    plan.sync(stream.cuda_stream)
    per = el / args.steps
    u.zero_()
    plan.execute(pos, u)
    plan.sync(stream.cuda_stream)
    plan.close()
    uf = u.cpu().numpy()
    del u
    d = uf - u64
    evals = st["evals_per_atom"] * n
    achieved = evals * W_LINE / per / 1e12
    peak, src = pipe_peak_tflops(torch, clk, fp64=False)
    gemm = fp32_peak_tflops(torch)
    out = {"value": n / per, "unit": "atoms/s", "ms_per_step": 1e3 * per, "steps": args.steps,
           "speedup_vs_fp64": None, "evals_per_s": evals / per,
           "max_abs_du": float(np.abs(d).max()), "rms_du": float(np.sqrt(np.mean(d * d))),
           "against": "plain FP64 result (this run, every atom; itself within 1e-9 A of the oracle)",
           "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                        "frac": achieved / peak, "peak_source": src, "peak_gemm": gemm,
                        "frac_of_gemm": achieved / gemm, "flop_per_eval": W_LINE, "evals_per_launch": evals},
           "clocks": clk, "gpu_launches": 2 * args.steps}
    if idx is not None:
        out["max_abs_du_vs_oracle_sample"] = float(np.abs(uf[:, idx] - np.stack(uref)).max())
        out["oracle_sample_atoms"] = int(len(idx))
    return out


def north_star_forms(args, w, pos, u64, idx, uref):
    """The forms the target names beside the plain FP64 path, each timed on its
    own (CUDA events, its own clock samples) after the headline measurement:
      fp32c          the FP32 compensated form on the same atoms;
      learned        images +-4 with the network's far shells: speed-up over the
                     plain FP64 path on the same workload, max/RMS |du| on every
                     atom, per-loop fallbacks, training time;
      bcc_prismatic  the matter step + loopon field + epilogue: step time,
                     bit-exact atom sets, compaction rate."""
    import argparse as ap
    import torch
    sub = ap.Namespace(**{**vars(args), "steps": 3, "warmup": 1, "e2e_steps": 1, "no_cpu": True,
                          "no_output": True, "image_split": 0, "images": None, "retrain": False,
                          "no_fp64": False, "precision": "fp64"})
    out = {}
    f = fp32c_form(sub, w, pos, u64, idx, uref)
    out["fp32c"] = f
    torch.cuda.empty_cache()
    ln = run_learned(sub, embedded=(w, pos))
    L = ln["learned"]
    out["learned"] = {
        "value": ln["value"], "unit": "atoms/s", "ms_per_step": ln["ms_per_step"], "steps": ln["steps"],
        "speedup_vs_fp64": L["speedup_vs_fp64"], "fp64_ms_per_step": (ln["fp64_exact"] or {}).get("ms_per_step"),
        "max_abs_du": (L["accuracy"] or {}).get("max_abs_du"), "rms_du": (L["accuracy"] or {}).get("rms_du"),
        "truncated_max_abs_du": (L["accuracy"] or {}).get("truncated_max_abs_du"),
        "against": (L["accuracy"] or {}).get("against"), "n_fallback": L["n_fallback"],
        "check_max": L["check_max"], "phase_seconds": L["phase_seconds"],
        "training_seconds": L["training"].get("train_seconds"), "training": L["training"],
        "config": {k: ln["config"][k] for k in ("images", "near_images", "far_images", "near", "far", "check")},
        "roofline_near_shell": ln["roofline"], "clocks": ln["clocks"], "gpu_launches": ln["gpu_launches"]}
    torch.cuda.empty_cache()
    pr = run_prismatic(sub, embedded=True)
    out["bcc_prismatic"] = {
        "value": pr["value"], "unit": "atoms/s", "ms_per_step": pr["ms_per_step"], "steps": pr["steps"],
        "config": pr["config"], "parity": pr["parity"], "compaction": pr["compaction"],
        "compaction_13m": pr.get("compaction_13m"),
        "roofline_loopon_field": pr["roofline"], "clocks": pr["clocks"], "gpu_launches": pr["gpu_launches"]}
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist
    from disco_b200 import backend as B
    from disco_b200 import _capi as C
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    w = build_workload(args.config, args.images)
    prec = C.DISCO_FP32C if args.precision == "fp32c" else C.DISCO_FP64
    n = w.n
    plan = B.Plan(w.loops, w.box, precision=prec, images=w.images, nu=w.nu,
                  image_split=args.image_split, max_atoms=n)
    st = plan.stats()
    evals_atom = st["evals_per_atom"]
    stream = torch.cuda.current_stream()
    pos = torch.tensor(np.stack([w.x, w.y, w.z]), dtype=torch.float64, device="cuda")
    u = torch.zeros_like(pos)
    launches_per_step = int(st["n_line_loops"] > 0) + int(st["n_loopon_loops"] > 0)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        plan.execute(pos, u)
    plan.sync(stream.cuda_stream)
    flush = L2Flush(torch, 48 * n)
    clocks = Clocks(local)
    barrier()
    clocks.start()
    elapsed = timed_steps(torch, lambda: plan.execute(pos, u), args.steps, stream, flush)
    barrier()
    clk = clocks.stop()
    plan.sync(stream.cuda_stream)
    elapsed = max_over_ranks(elapsed, world)
    per_launch = elapsed / args.steps
    value = n * world * args.steps / elapsed

    # parity on a seeded sample (fresh sum) while the CPU baseline runs on it
    u1d = torch.zeros_like(pos)
    plan.execute(pos, u1d)
    plan.sync(stream.cuda_stream)
    u1 = u1d.cpu().numpy()
    output = write_output(w, pos, u1d, stream) if (rank == 0 and not args.no_output) else None
    del u1d

    if args.kernel_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "atoms/s", "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * per_launch,
                              "config": arm_config(args, w, args.precision, st["n_segments"], st["n_loopons"]),
                              "note": "--kernel-only: device-resident steps alone"}), flush=True)
        plan.close()
        return

    # e2e: the public host call on pinned host memory
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else max(1, min(args.steps, 3))
    hp = torch.empty((6, n), dtype=torch.float64, pin_memory=True)
    hv = hp.numpy()
    hv[0], hv[1], hv[2] = w.x, w.y, w.z
    atoms = B.AtomArrays(hv[0], hv[1], hv[2], hv[3], hv[4], hv[5])
    hv[3:] = 0.0
    B.kroupa_gpu(atoms, w.loops, *w.box, B.GpuOptions(fp32=prec == C.DISCO_FP32C), images=w.images,
                 nu=w.nu, image_split=args.image_split)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        hv[3:] = 0.0
        B.kroupa_gpu(atoms, w.loops, *w.box, B.GpuOptions(fp32=prec == C.DISCO_FP32C),
                     images=w.images, nu=w.nu, image_split=args.image_split)
    barrier()
    e2e_t = time.perf_counter() - t0
    e2e_t = max_over_ranks(e2e_t, world)
    e2e = {"value": n * world * e2e_steps / e2e_t, "unit": "atoms/s",
           "h2d_bytes_per_step": 6 * 8 * n, "d2h_bytes_per_step": 3 * 8 * n, "steps": e2e_steps}
    del hp, hv, atoms
    # the same from the device lattice: sites built on the GPU (generateLattice
    # order, bit-identical), loop tables from the host loops, the field, the
    # displacements read back; nothing but the tables crosses to the device
    e2e_lat = None
    if w.cells[0] > 0:
        import ctypes
        lib = C.cuda_lib()
        from disco_b200 import geometry as G
        dl = torch.empty((3, n), dtype=torch.float64, device="cuda")
        ul = torch.empty((3, n), dtype=torch.float64, device="cuda")
        hu = torch.empty((3, n), dtype=torch.float64, pin_memory=True)

        def lat_step():
            C.check(lib.disco_b200_lattice(w.lattice, w.cells[0], w.cells[1], w.cells[2], w.a0,
                                           dl[0].data_ptr(), dl[1].data_ptr(), dl[2].data_ptr(),
                                           ctypes.c_void_p(stream.cuda_stream)), lib)
            ul.zero_()
            pl = B.Plan(w.loops, w.box, precision=prec, images=w.images, nu=w.nu, max_atoms=n)
            pl.execute(dl, ul)
            hu.copy_(ul, non_blocking=True)
            pl.sync(stream.cuda_stream)
            pl.close()
        lat_step()
        same = bool(torch.equal(dl, pos))
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            lat_step()
        barrier()
        tl = max_over_ranks(time.perf_counter() - t0, world)
        e2e_lat = {"value": n * world * e2e_steps / tl, "unit": "atoms/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 3 * 8 * n, "steps": e2e_steps,
                   "device_lattice_equals_host_lattice": same,
                   "what": "disco_b200_lattice + plan (tables from the host loops) + field + displacements "
                           "to pinned host memory, per step"}
        del dl, ul, hu

    if rank == 0:
        fp64 = prec == C.DISCO_FP64
        gemm = fp64_peak_tflops(torch) if fp64 else fp32_peak_tflops(torch)
        peak, peak_src = pipe_peak_tflops(torch, clk, fp64)
        flops = evals_atom * n * flop_per_eval(w)
        achieved = flops / per_launch / 1e12
        key = f"{'line' if w.method == 'line' else 'loopon'}_{args.precision}_{args.config}"
        traffic = traffic_from_profiles(key)
        roof = {"bound": "fp64" if fp64 else "fp32", "achieved": achieved,
                "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
                "peak_source": peak_src + "; MEASURED_PEAKS.json has no FP64 or FP32 CUDA-core figure",
                "peak_gemm": gemm, "frac_of_gemm": achieved / gemm if gemm else None,
                "peak_gemm_source": ("torch DGEMM 8192^3, best of 5: it runs on the FP64 tensor-core path, "
                                     "not on the DFMA pipe this kernel uses") if fp64 else
                                    "torch SGEMM 8192^3 without TF32, best of 5",
                "flop_per_eval": flop_per_eval(w), "evals_per_launch": evals_atom * n}
        cpu = None
        parity = None
        if not args.no_cpu:
            cpu, idx, ucpu = cpu_baseline(w, args.cpu_seconds, use_reference=False)
            du = np.abs(u1[:, idx] - np.stack(ucpu)).max()
            parity = {"max_abs_du": float(du), "atoms": int(len(idx)), "against": "oracle"}
            cpu.pop("seconds", None)
        refgpu = None
        if world == 1 and args.config == "quadrupole" and fp64:
            p35 = B.Plan(w.loops, w.box, precision=C.DISCO_FP64, images=1, nu=0.35, max_atoms=n)
            u35 = torch.zeros_like(pos)
            p35.execute(pos, u35)
            p35.sync(stream.cuda_stream)
            p35.close()
            refgpu = reference_gpu(w, w.x, w.y, w.z, ours_u=u35.cpu().numpy())
            del u35
            refgpu["ours"] = {"kernel_atoms_per_s": value, "e2e_atoms_per_s": e2e["value"],
                              "note": "this library on the same atoms (nu 0.29: same operation count)"}
        forms = {}
        if world == 1 and not args.no_forms and args.config == "fcc_random" and fp64:
            forms = north_star_forms(args, w, pos, u1, idx if parity else None, ucpu if parity else None)
        line = {
            "metric": METRIC, "value": value, "unit": "atoms/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * per_launch,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == C.DISCO_FP64 else "f32c", "data": "synthetic",
            "config": arm_config(args, w, args.precision, st["n_segments"], st["n_loopons"]),
            "evals_per_s": evals_atom * n * world * args.steps / elapsed,
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "e2e_device_lattice": e2e_lat, "clocks": clk,
            "gpu_launches": launches_per_step * args.steps, "parity": parity, "output": output,
            **({"reference_gpu": refgpu} if refgpu else {}), **forms,
        }
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_batch(args):
    """The batch workload: 256 independent BCC samples in one persistent, graph-captured
    launch (FP32 compensated by default), knobs from the autotuner."""
    import torch
    import torch.distributed as dist
    from disco_b200 import autotune as A
    from disco_b200 import backend as B
    from disco_b200 import _capi as C
    from disco_b200 import workloads as W
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    prec = C.DISCO_FP64 if args.precision == "fp64" else C.DISCO_FP32C
    batch = W.batch(nsamples=args.samples)
    tune = A.tune(batch, prec, log=(lambda m: print(m, file=sys.stderr)) if rank == 0 else None)
    n = sum(w.n for w in batch)
    evals = sum(w.n * w.evals_per_atom() for w in batch)
    pos = [torch.tensor(np.stack([w.x, w.y, w.z]), dtype=torch.float64, device="cuda") for w in batch]
    u = [torch.zeros_like(p) for p in pos]
    ptrs = [(p[0].data_ptr(), p[1].data_ptr(), p[2].data_ptr(), q[0].data_ptr(), q[1].data_ptr(),
             q[2].data_ptr()) for p, q in zip(pos, u)]
    plan = B.BatchPlan(batch, ptrs, precision=prec, image_split=tune["image_split"],
                       stage_kb=tune["stage_kb"], stages=tune["stages"])
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        plan.execute(stream.cuda_stream)
    plan.sync(stream.cuda_stream)
    flush = L2Flush(torch, 48 * n)
    clocks = Clocks(local)
    barrier()
    clocks.start()
    elapsed = timed_steps(torch, lambda: plan.execute(stream.cuda_stream), args.steps, stream, flush)
    barrier()
    clk = clocks.stop()
    plan.sync(stream.cuda_stream)
    elapsed = max_over_ranks(elapsed, world)
    per = elapsed / args.steps
    # parity: a fresh sum on a few samples against the oracle
    for q in u:
        q.zero_()
    plan.execute(stream.cuda_stream)
    plan.sync(stream.cuda_stream)
    parity = None
    cpu = None
    if rank == 0 and not args.no_cpu:
        import oracle as O
        rng = np.random.default_rng(7)
        pick = rng.choice(len(batch), size=min(4, len(batch)), replace=False)
        worst, t_cpu, ev_cpu, at_cpu = 0.0, 0.0, 0.0, 0
        threads = os.cpu_count() or 1
        for i in pick:
            w = batch[i]
            k = min(w.n, max(8, int(args.cpu_seconds * 2e8 / max(1.0, w.evals_per_atom()) / len(pick))))
            idx = np.sort(rng.choice(w.n, size=k, replace=False))
            t0 = time.perf_counter()
            ref = O.displace(w.x[idx], w.y[idx], w.z[idx], w.loops, w.box, images=w.images, nu=w.nu,
                             threads=threads)
            t_cpu += time.perf_counter() - t0
            ev_cpu += k * w.evals_per_atom()
            at_cpu += k
            g = u[i].cpu().numpy()[:, idx]
            worst = max(worst, float(np.abs(g - np.stack(ref)).max()))
        parity = {"max_abs_du": worst, "atoms": at_cpu, "against": "oracle (FP64)"}
        cpu = {"value": ev_cpu / t_cpu * n / evals, "unit": "atoms/s", "cores": threads, "kind": "port",
               "sample": f"{at_cpu} random atoms of {len(pick)} samples, all their loops and images, "
                         f"{t_cpu:.1f} s; rate converted to the whole batch's atoms via its "
                         "evaluations per atom"}
    # e2e: the public batched call on pinned host memory
    e2e = None
    if args.e2e_steps != 0:
        hp = [torch.empty((6, w.n), dtype=torch.float64, pin_memory=True) for w in batch]
        for w, h in zip(batch, hp):
            hv = h.numpy()
            hv[0], hv[1], hv[2] = w.x, w.y, w.z
            hv[3:] = 0.0
        arr, keep = B.sample_array(batch, us=[h.numpy()[3:] for h in hp])
        for i, h in enumerate(hp):
            hv = h.numpy()
            arr[i].atoms = C.DiscoAtoms(*(hv[k].ctypes.data for k in range(6)), batch[i].n)
        o = B.options(prec, 1, batch[0].nu, tune["image_split"])
        o.stage_kb = tune["stage_kb"]
        o.stages = tune["stages"]
        tm = C.DiscoTiming(0.0, 0.0, 0.0, None)
        barrier()
        t0 = time.perf_counter()
        C.check(C.cuda_lib().disco_b200_batch(arr, len(batch), ctypes_byref(o), ctypes_byref(tm)))
        barrier()
        e2e_t = time.perf_counter() - t0
        e2e = {"value": n * world / e2e_t, "unit": "atoms/s", "h2d_bytes_per_step": 48 * n,
               "d2h_bytes_per_step": 24 * n, "steps": 1}
    if rank == 0:
        gemm = fp64_peak_tflops(torch) if prec == C.DISCO_FP64 else fp32_peak_tflops(torch)
        peak, peak_src = pipe_peak_tflops(torch, clk, prec == C.DISCO_FP64)
        achieved = evals * W_LINE / per / 1e12
        roof = {"bound": "fp32" if prec != C.DISCO_FP64 else "fp64", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None, "flop_per_eval": W_LINE,
                "evals_per_launch": evals, "peak_source": peak_src, "peak_gemm": gemm,
                "frac_of_gemm": achieved / gemm,
                "peak_gemm_source": "measured here: torch " + ("DGEMM" if prec == C.DISCO_FP64 else
                                                               "SGEMM without TF32") + " 8192^3, best of 5"}
        line = {
            "metric": METRIC, "value": n * world / per, "unit": "atoms/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * per,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == C.DISCO_FP64 else "f32c", "data": "synthetic",
            "config": {"workload": "batch", "samples": len(batch), "atoms": n,
                       "loops": sum(len(w.loops) for w in batch), "evals_per_step": evals,
                       "images": "+-1..+-3 per sample", "nu": batch[0].nu,
                       "precision": "fp64" if prec == C.DISCO_FP64 else "fp32c",
                       "tuning": {"image_split": tune["image_split"], "stage_kb": tune["stage_kb"],
                                  "stages": tune["stages"]},
                       "graph": "one CUDA graph replay per step",
                       "l2": flush.note(48 * n),
                       "parallelism": f"replicas x{world}"},
            "evals_per_s": evals * world / per,
            "roofline": roof,
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "gpu_launches": args.steps * (2 if prec == C.DISCO_FP32C else 1), "parity": parity,
        }
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_learned(args, embedded=None):
    """Learned form on the fcc_random geometry with images +-4 (729 images):
    exact near images +-1 (27, FP32 compensated), the network's far shells
    2 <= max|n| <= 4 (702 images), the exact FP64 far-shell sum re-checked on a
    1 % stratified random atom subsample every step with per-loop fallback.
    The plain FP64 path on the same workload (all 729 images exact) is timed
    once and is the reference for the learned result on every atom.
    embedded = (fcc_random workload, its positions on the device): one GPU,
    returns the line instead of printing it."""
    import torch
    from disco_b200 import backend as B
    from disco_b200 import _capi as C
    from disco_b200 import learned as Ln
    rank, world, local = dist_env()
    if embedded is not None:
        rank, world = 0, 1
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    if embedded is not None:
        import copy
        w = copy.copy(embedded[0])
        w.images = 4
    else:
        w = build_workload("fcc_random", 4)
    n = w.n
    log = (lambda m: print(m, file=sys.stderr, flush=True)) if rank == 0 else None
    path = os.environ.get("DISCO_B200_FAR_NET",
                          os.path.join(ROOT, "disco_b200", "_lib", f"far_fcc_random_nu{w.nu:.2f}.npz"))
    if args.retrain and os.path.exists(path) and rank == 0:
        os.remove(path)
    if world > 1:
        dist.barrier()
    m, norm, info = Ln.cached_or_train(path if rank == 0 else None, log=log, nloops=4096, atoms=1024, seed=5,
                                       nu=w.nu, epochs=args.epochs)
    stream = torch.cuda.current_stream()
    pos = embedded[1] if embedded is not None else \
        torch.tensor(np.stack([w.x, w.y, w.z]), dtype=torch.float64, device="cuda")
    u = torch.zeros_like(pos)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for s in range(args.warmup):
        Ln.learned_displace(m, norm, pos, u, w.loops, w.box, w.nu, seed=s)
    clocks = Clocks(local)
    barrier()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = []
    e0.record(stream)
    for s in range(args.steps):
        reps.append(Ln.learned_displace(m, norm, pos, u, w.loops, w.box, w.nu, seed=100 + s))
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    elapsed = e0.elapsed_time(e1) * 1e-3
    elapsed = max_over_ranks(elapsed, world)
    per = elapsed / args.steps

    # accuracy on every atom against the plain FP64 path (+-4, all images exact)
    ul = torch.zeros_like(pos)
    rep = Ln.learned_displace(m, norm, pos, ul, w.loops, w.box, w.nu, seed=777)
    acc, fp64 = None, None
    if not args.no_fp64:
        ux = torch.zeros_like(pos)
        plan = B.Plan(w.loops, w.box, precision=C.DISCO_FP64, images=4, nu=w.nu, max_atoms=n)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        plan.execute(pos, ux)
        f1.record(stream)
        plan.sync(stream.cuda_stream)
        t64 = f0.elapsed_time(f1) * 1e-3
        st64 = plan.stats()
        plan.close()
        un = torch.zeros_like(pos)
        pn = B.Plan(w.loops, w.box, precision=C.DISCO_FP32C, images=1, nu=w.nu, max_atoms=n)
        pn.execute(pos, un)
        pn.sync(stream.cuda_stream)
        pn.close()
        d = ul - ux
        acc = {"max_abs_du": float(d.abs().max()), "rms_du": float(d.pow(2).mean().sqrt()),
               "truncated_max_abs_du": float((un - ux).abs().max()),
               "against": "plain FP64 path, images +-4, every atom"}
        fp64 = {"value": n / t64, "unit": "atoms/s", "ms_per_step": 1e3 * t64, "steps": 1,
                "evals_per_s": st64["evals_per_atom"] * n / t64}
        del ux, un
    # e2e: host positions in, host displacements out, every step
    hp = torch.empty((6, n), dtype=torch.float64, pin_memory=True)
    hv = hp.numpy()
    hv[0], hv[1], hv[2] = w.x, w.y, w.z
    hv[3:] = 0.0
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else 2
    dpos = torch.empty_like(pos)
    du_ = torch.empty_like(pos)
    barrier()
    t0 = time.perf_counter()
    for s in range(e2e_steps):
        dpos.copy_(hp[:3], non_blocking=True)
        du_.copy_(hp[3:], non_blocking=True)
        Ln.learned_displace(m, norm, dpos, du_, w.loops, w.box, w.nu, seed=500 + s)
        hp[3:].copy_(du_, non_blocking=True)
        torch.cuda.synchronize()
    e2e_t = time.perf_counter() - t0
    e2e_t = max_over_ranks(e2e_t, world)
    e2e = {"value": n * world * e2e_steps / e2e_t, "unit": "atoms/s", "h2d_bytes_per_step": 48 * n,
           "d2h_bytes_per_step": 24 * n, "steps": e2e_steps}
    if rank == 0:
        segs = sum(len(lp.vx) for lp in w.loops)
        near_evals = segs * 27 * n
        t_near = statistics.median(r["t_near"] for r in reps)
        peak, peak_src = pipe_peak_tflops(torch, clk, fp64=False)
        gemm = fp32_peak_tflops(torch)
        achieved = near_evals * W_LINE / t_near / 1e12
        cpu = None
        if not args.no_cpu:
            cpu, idx, ucpu = cpu_baseline(w, args.cpu_seconds, use_reference=False)
            cpu.pop("seconds", None)
        mean = lambda k: statistics.mean(r[k] for r in reps)
        line = {
            "metric": METRIC, "value": n * world / per, "unit": "atoms/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * per,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32c+bf16",
            "data": "synthetic",
            "config": {"workload": "fcc_random_learned", "atoms": n, "loops": len(w.loops), "segments": segs,
                       "images": 729, "near_images": 27, "far_images": 702, "nu": w.nu,
                       "near": "exact, FP32 compensated", "far": "MLP 14-128-128-128-3, BF16 tcgen05",
                       "check": "exact FP64 far shells on 1% of the atoms per step, per-loop fallback above "
                                "1e-3 A", "l2": f"inputs larger than L2 (positions {24 * n / 1e6:.0f} MB)",
                       "parallelism": f"replicas x{world}"},
            "learned": {"speedup_vs_fp64": (fp64["ms_per_step"] / (1e3 * per)) if fp64 else None,
                        "accuracy": acc, "n_fallback": [r["n_fallback"] for r in reps],
                        "check_max": max(r["check_max"] for r in reps),
                        "worst_loop": max(r["worst_loop"] for r in reps),
                        "phase_seconds": {k: mean(k) for k in ("t_check", "t_near", "t_far", "t_fallback")},
                        "training": {k: v for k, v in info.items() if k != "loss"}},
            "fp64_exact": fp64,
            "roofline": {"bound": "fp32", "kernel": "near-shell FP32 line kernel", "achieved": achieved,
                         "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                         "peak_source": peak_src, "peak_gemm": gemm, "frac_of_gemm": achieved / gemm,
                         "peak_gemm_source": "torch SGEMM 8192^3 without TF32, best of 5",
                         "flop_per_eval": W_LINE, "evals_per_launch": near_evals},
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "gpu_launches": sum(r["launches"] for r in reps),
        }
        if embedded is not None:
            return line
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def compaction_rate(lib, C, torch, stream, cells=128):
    """The matter step alone (disco_b200_prismatic_noalloc: slab membership,
    stable compaction, new-index map, slab entries, copies) on a BCC box of
    cells^3 (2 cells^3 atoms; 128: 4 194 304) with 16 loops of the bcc_prismatic
    distribution: achieved GB/s of the algorithmic bytes (52 B per atom:
    positions read once, survivors written, 4 B new index; the slab entries
    and copies add a few hundred KB) against the measured HBM peak.  Timed per
    call with CUDA events around the whole call, which ends with one
    device-to-host read of the totals (its only host wait)."""
    import ctypes
    from disco_b200 import workloads as W
    w = W.bcc_prismatic(cells=cells)
    n = w.n
    pos = torch.tensor(np.stack([w.x, w.y, w.z]), dtype=torch.float64, device="cuda")
    out = torch.empty((3, n), dtype=torch.float64, device="cuda")
    new_index = torch.empty(n, dtype=torch.int32, device="cuda")
    cap = 1 << 21
    slab_atoms = torch.empty(cap, dtype=torch.int32, device="cuda")
    slab_side = torch.empty(cap, dtype=torch.int8, device="cuda")
    copies = torch.empty((cap, 4), dtype=torch.float64, device="cuda")
    nl = len(w.slab_loops)
    sl = (C.DiscoSlabLoop * nl)(*w.slab_loops)
    info = (C.DiscoSlabInfo * nl)()
    counts = (ctypes.c_int64 * 3)()
    box = (ctypes.c_double * 3)(*w.box)
    sp = ctypes.c_void_p(stream.cuda_stream)

    def call():
        C.check(lib.disco_b200_prismatic_noalloc(
            pos[0].data_ptr(), pos[1].data_ptr(), pos[2].data_ptr(), n, sl, nl, box,
            out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), new_index.data_ptr(), info,
            slab_atoms.data_ptr(), slab_side.data_ptr(), cap, copies.data_ptr(), cap, counts, sp), lib)

    for _ in range(3):
        call()
    torch.cuda.synchronize()
    reps = 20
    flush = L2Flush(torch, 0)                     # always: 100 MB of positions < L2
    t = timed_steps(torch, call, reps, stream, flush) / reps
    pk = measured_peaks()
    peak = pk["hbm_gbs"] if pk else 6650.0
    gbs = 52.0 * n / t / 1e9
    return {"atoms": n, "survivors": int(counts[0]), "slab_atoms": int(counts[1]), "copies": int(counts[2]),
            "ms": 1e3 * t, "atoms_per_s": n / t, "algorithmic_bytes": 52 * n, "achieved_gbs": gbs,
            "peak_gbs": peak, "frac": gbs / peak, "l2": "flushed before each timed call",
            "traffic": traffic_from_profiles("compaction_bcc128") if cells == 128 else None,
            "traffic_what": "DRAM bytes read + written by one matter_kernel launch on this box (one ncu capture)",
            "timed": "whole call (loop upload, matter kernel, totals read back) with CUDA events",
            "peak_source": "MEASURED_PEAKS.json hbm_gbs" if pk else "fallback 6650 GB/s"}


def run_prismatic(args, embedded=False):
    """The bcc_prismatic workload: one step = the prismatic matter step (slab selection, vacancy
    removal, interstitial copies; disco_b200_prismatic_noalloc on device
    arrays), the loopon field of all 16 loops over the surviving atoms (plan),
    and the fused copy/add-u/wrap epilogue (disco_b200_finalize_resident).
    value = input atoms / step time.  Parity: atom sets, order, copies bit-exact
    against the oracle; the field on a seeded survivor sample within 1e-9 A
    (FP64); the final positions of that sample against the oracle's epilogue.
    embedded: one GPU, returns the line instead of printing it."""
    import ctypes
    import torch
    from disco_b200 import backend as B
    from disco_b200 import _capi as C
    from disco_b200 import prismatic as P
    rank, world, local = dist_env()
    if embedded:
        rank, world = 0, 1
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    lib = C.cuda_lib()
    w = build_workload("bcc_prismatic", args.images)
    prec = C.DISCO_FP32C if args.precision == "fp32c" else C.DISCO_FP64
    n = w.n
    first = P.prismatic(w.x, w.y, w.z, w.slab_loops, w.box)       # capacities for the device arrays
    ns0, nc0 = len(first["slab_atoms"]), len(first["copy_atom"])
    scap, ccap = ns0 + 1024, nc0 + 1024
    plan = B.Plan(w.loops, w.box, precision=prec, images=w.images, nu=w.nu, image_split=args.image_split,
                  max_atoms=n)
    st_plan = plan.stats()
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    pos = torch.tensor(np.stack([w.x, w.y, w.z]), dtype=torch.float64, device="cuda")
    out = torch.empty((3, n), dtype=torch.float64, device="cuda")
    new_index = torch.empty(n, dtype=torch.int32, device="cuda")
    slab_atoms = torch.empty(scap, dtype=torch.int32, device="cuda")
    slab_side = torch.empty(scap, dtype=torch.int8, device="cuda")
    copies = torch.empty((ccap, 4), dtype=torch.float64, device="cuda")
    u = torch.zeros((3, n), dtype=torch.float64, device="cuda")
    fin = torch.empty((6, n + ccap), dtype=torch.float64, device="cuda")
    nl = len(w.slab_loops)
    sl = (C.DiscoSlabLoop * nl)(*w.slab_loops)
    info = (C.DiscoSlabInfo * nl)()
    counts = (ctypes.c_int64 * 3)()
    box = (ctypes.c_double * 3)(*w.box)

    def step():
        C.check(lib.disco_b200_prismatic_noalloc(
            pos[0].data_ptr(), pos[1].data_ptr(), pos[2].data_ptr(), n, sl, nl, box,
            out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), new_index.data_ptr(), info,
            slab_atoms.data_ptr(), slab_side.data_ptr(), scap, copies.data_ptr(), ccap, counts, sp), lib)
        k, nc = int(counts[0]), int(counts[2])
        u[:, :k].zero_()
        plan.execute_ptrs(out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), u[0].data_ptr(),
                          u[1].data_ptr(), u[2].data_ptr(), k, stream.cuda_stream)
        tot = k + nc
        C.check(lib.disco_b200_finalize_resident(
            out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), u[0].data_ptr(), u[1].data_ptr(),
            u[2].data_ptr(), k, copies.data_ptr(), nc, box, fin[0].data_ptr(), fin[1].data_ptr(),
            fin[2].data_ptr(), fin[3].data_ptr(), fin[4].data_ptr(), fin[5].data_ptr(), sp), lib)
        return k, nc

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    plan.sync(stream.cuda_stream)
    flush = L2Flush(torch, 48 * n)
    kn = [0, 0]

    def timed_step():
        kn[0], kn[1] = step()

    clocks = Clocks(local)
    barrier()
    clocks.start()
    elapsed = timed_steps(torch, timed_step, args.steps, stream, flush)
    barrier()
    clk = clocks.stop()
    plan.sync(stream.cuda_stream)
    k, nc = kn
    elapsed = max_over_ranks(elapsed, world)
    per = elapsed / args.steps
    evals = st_plan["evals_per_atom"] * k

    # e2e: the host entry points (matter step, kroupa_gpu drop-in, epilogue) on host arrays
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else 2
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        r = P.prismatic(w.x, w.y, w.z, w.slab_loops, w.box)
        sx, sy, sz = r["survivors"]
        atoms = B.AtomArrays.zeros_like_positions(sx, sy, sz)
        B.kroupa_gpu(atoms, w.loops, *w.box, B.GpuOptions(fp32=prec == C.DISCO_FP32C), images=w.images,
                     nu=w.nu)
        final = P.finalize(sx, sy, sz, atoms.ux, atoms.uy, atoms.uz, r["copy_atom"], r["copy_shift"], w.box)
    e2e_t = max_over_ranks(time.perf_counter() - t0, world)

    compaction = compaction_rate(lib, C, torch, stream) if rank == 0 else None
    compaction_13m = compaction_rate(lib, C, torch, stream, cells=189) if rank == 0 else None
    if compaction_13m is not None:
        compaction_13m["workload"] = "bcc_prismatic 189^3 (13 502 538 atoms, 16 loops)"
    parity = None
    cpu = None
    if rank == 0:
        import oracle as O
        ref = O.prismatic(w.x, w.y, w.z, w.slab_loops, w.box)
        o = out.cpu().numpy()
        sets = (int(counts[0]) == len(ref["survivors"][0]) and
                all(np.array_equal(o[d, :k], ref["survivors"][d]) for d in range(3)) and
                np.array_equal(new_index.cpu().numpy(), ref["new_index"]) and
                np.array_equal(slab_atoms.cpu().numpy()[:int(counts[1])], ref["slab_atoms"]) and
                np.array_equal(copies.cpu().numpy()[:nc, 1:], ref["copy_shift"]))
        rng = np.random.default_rng(5)
        idx = np.sort(rng.choice(k, size=min(k, 2000), replace=False))
        ug = u.cpu().numpy()[:, idx]
        uo = np.stack(O.displace(o[0, idx], o[1, idx], o[2, idx], w.loops, w.box, images=w.images, nu=w.nu))
        f = fin.cpu().numpy()[:3, idx]
        fo = np.stack(O.finalize(o[0, idx], o[1, idx], o[2, idx], ug[0], ug[1], ug[2],
                                 np.zeros(0, np.int32), np.zeros((0, 3)), w.box)[:3])
        parity = {"atom_sets_bit_exact": bool(sets), "max_abs_du": float(np.abs(ug - uo).max()),
                  "final_positions_bit_exact_on_sample": bool(np.array_equal(f, fo)),
                  "atoms": int(len(idx)), "survivors": k, "copies": nc, "against": "oracle"}
        if not args.no_cpu:
            cpu, _, _ = cpu_baseline(w, args.cpu_seconds, use_reference=False)
            cpu.pop("seconds", None)
            cpu["sample"] += "; the matter step is not in the CPU figure (host serial in the reference, ms)"
        refgpu = None
        if not embedded and prec == C.DISCO_FP64:
            # the loopon field over the survivors, the reference's kernels against ours at its nu
            p35 = B.Plan(w.loops, w.box, precision=C.DISCO_FP64, images=1, nu=0.35, max_atoms=k)
            u35 = torch.zeros((3, k), dtype=torch.float64, device="cuda")
            p35.execute_ptrs(out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), u35[0].data_ptr(),
                             u35[1].data_ptr(), u35[2].data_ptr(), k, stream.cuda_stream)
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            u35.zero_()
            f0.record(stream)
            p35.execute_ptrs(out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), u35[0].data_ptr(),
                             u35[1].data_ptr(), u35[2].data_ptr(), k, stream.cuda_stream)
            f1.record(stream)
            p35.sync(stream.cuda_stream)
            p35.close()
            refgpu = reference_gpu(w, o[0, :k].copy(), o[1, :k].copy(), o[2, :k].copy(),
                                   ours_u=u35.cpu().numpy(), reps=1)
            refgpu["ours"] = {"kernel_s": f0.elapsed_time(f1) * 1e-3,
                              "note": "this library's loopon field over the same survivors, nu 0.35"}
            del u35
        gemm = fp64_peak_tflops(torch) if prec == C.DISCO_FP64 else fp32_peak_tflops(torch)
        peak, peak_src = pipe_peak_tflops(torch, clk, prec == C.DISCO_FP64)
        achieved = evals * W_LOOPON / per / 1e12
        line = {
            "metric": METRIC, "value": n * world / per, "unit": "atoms/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * per,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == C.DISCO_FP64 else "f32c", "data": "synthetic",
            "config": {"workload": "bcc_prismatic", "atoms": n, "survivors": k, "copies": nc,
                       "loops": len(w.loops), "loopons": st_plan["n_loopons"], "images": st_plan["n_images"],
                       "nu": w.nu, "method": "loopons", "precision": args.precision,
                       "step": "matter step + loopon field + copy/add-u/wrap epilogue, all on device",
                       "l2": flush.note(48 * n), "parallelism": f"replicas x{world}"},
            "evals_per_s": evals * world / per,
            "roofline": {"bound": "fp64" if prec == C.DISCO_FP64 else "fp32", "kernel": "loopon field",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "peak_source": peak_src + " (the step also holds the matter step and epilogue)",
                         "peak_gemm": gemm, "frac_of_gemm": achieved / gemm,
                         "traffic": None, "flop_per_eval": W_LOOPON, "evals_per_launch": evals},
            "cpu_baseline": cpu,
            "e2e": {"value": n * world * e2e_steps / e2e_t, "unit": "atoms/s",
                    "h2d_bytes_per_step": 24 * n + 48 * k + 48 * k,
                    "d2h_bytes_per_step": 28 * n + 24 * k + 48 * (k + nc), "steps": e2e_steps},
            "clocks": clk, "gpu_launches": args.steps * 3,     # matter kernel, field kernel, epilogue
            "parity": parity, "compaction": compaction, "compaction_13m": compaction_13m,
            **({"reference_gpu": refgpu} if refgpu else {}),
        }
        if embedded:
            plan.close()
            return line
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def ctypes_byref(x):
    import ctypes
    return ctypes.byref(x)


def run_matter(args):
    """--config matter: the matter step alone (compaction_rate) on BCC 128^3
    (4 194 304 atoms) and BCC 189^3 (13 502 538 atoms), for profiling; one line."""
    import torch
    from disco_b200 import _capi as C
    torch.cuda.set_device(dist_env()[2])
    r = compaction_rate(C.cuda_lib(), C, torch, torch.cuda.current_stream())
    big = compaction_rate(C.cuda_lib(), C, torch, torch.cuda.current_stream(), cells=189)
    print(json.dumps({"metric": "matter step atoms/s", "value": r["atoms_per_s"], "unit": "atoms/s",
                      "config": {"workload": "bcc_prismatic 128^3 (4 194 304 atoms, 16 loops)"},
                      "compaction": r,
                      "compaction_13m": dict(big, workload="bcc_prismatic 189^3 (13 502 538 atoms, 16 loops)")}),
          flush=True)


def main():
    args = parse()
    if args.precision is None:
        args.precision = "fp32c" if args.config == "batch" else "fp64"
    if args.config == "matter":
        return run_matter(args)
    if args.impl == "reference":
        run_reference(args)
    elif args.config == "batch":
        run_batch(args)
    elif args.config == "learned":
        run_learned(args)
    elif args.config == "bcc_prismatic":
        run_prismatic(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
