"""Energy + force throughput of the n2p2 prediction path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --profile-case [--molecules M] [--potential P]
                    [--precision fp64|mixed|bf16] [--evaluations E]
                    [--autotune]

Workload (the FP64 plain form at scale): a periodic water box of 8,192
molecules = 24,576 atoms at 1.0 g/cm^3 (cubic, L = 118.26 bohr), seeded
uniform O positions with O-O >= 4.7 bohr, seeded orientations, then 100
frames with Gaussian position noise sigma = 0.1 bohr.  Potential: 52 symmetry
functions per element (radial + narrow angular, cos cutoff 12 bohr), NN
52-25-25-1 (tanh), seeded Nguyen-Widrow weights (tests/golden/potentials/
h2o_52).  One step = one frame through neighbor list, symmetry functions +
dG/dr, atomic NNs + dE/dG, energy and forces, all in FP64.

Metric: E+F atoms/s (higher is better).
  value : device-resident frames (HBM), K steps between CUDA events on the
          library's stream, max over ranks; frames cycle through 100
          distinct coordinate sets and the per-frame working set (dG/dr,
          2 GB) is far larger than L2.
  e2e   : the same through the C-ABI with HOST buffers -- every step copies
          the frame's positions host->device (pinned) and reads back energy
          and forces (n2p2b_set_positions / n2p2b_evaluate /
          n2p2b_get_forces / n2p2b_get_energy), wall clock around K steps.
Further entries of the same line (one GPU):
  forms   : the mixed-precision forms (FP32 symmetry functions, tensor-core
            BF16 networks) and the gated student, on the same frames, for
            this potential and the wider 92-SF / 64-64-64 one; speed-up over
            FP64 and energy-per-atom / force RMSE against the FP64 form, and
            whether each meets the stated targets; the gated student also on
            compressed, noisier frames where it gates atoms to the teacher;
  config4 : the precision form as specified: 98,304 atoms (32,768
            molecules, L = 187.7 bohr), 92-SF / 64-64-64 softplus potential,
            FP64 vs mixed atoms/s, RMSE against the FP64 form and against
            the reference CPU library on one frame;
  batch   : 4,096 structures of 33-513 atoms as one CUDA-graph launch, the
            one-structure-per-call loop, and the largest per-structure
            energy / force errors against the reference on a sample;
  roofline: the dominant kernel (symmetry functions) against the FP64 pipe
            (the bound: DGEMM peak measured in this run) with the HBM figure
            beside it;
  cpu_baseline: the reference library (OpenMP, all host cores) on 5 frames.

Multi-GPU: one process per GPU (torchrun); each rank evaluates its own
frames (independent replicas, weak scaling, no data-path collective); the
time is the max over ranks.

--impl reference times the reference n2p2 CPU path (oracle/_ref, OpenMP on
all host cores) on the same workload; each step is one full frame.

--profile-case runs a small fixed evaluation (seed-77 water box, default
4,096 molecules) and prints its per-stage device times; it is the command
the ncu captures under profiles/ run.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

POT_DIR = os.path.join(ROOT, "tests", "golden", "potentials")
POT = os.path.join(POT_DIR, "h2o_52")
STAGES = ("neighbor_list", "symmetry_functions", "neural_networks", "energy",
          "forces")
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one FP64
# symmetry-function launch on this workload, per kernel family, from the
# ncu captures summarized under profiles/ (12,288-atom box), scaled to the
# 24,576-atom frame by its neighbor entries (x 2.002): the staged-triplet
# kernel (variants 6, 7; the default) and the per-owner kernel (0-5).
SF_TRAFFIC = {
    "staged": (2.669e9, "ncu dram__bytes_read.sum + dram__bytes_write.sum of "
                        "the FP64 sfStagedKernel on the 12,288-atom box "
                        "(1.333 GB), x 2.002 neighbor entries for 24,576 "
                        "atoms (profiles/sfStagedKernel_fp64_fp32_"
                        "water12288.md)"),
    "owner": (4.184e9, "ncu dram__bytes_read.sum + dram__bytes_write.sum of "
                       "the FP64 per-owner sfKernel on the 12,288-atom box "
                       "(2.090 GB), x 2.002 neighbor entries for 24,576 "
                       "atoms (profiles/sfKernel_fp64_fp32_water12288.md)"),
}


def sf_family(tune: str) -> str:
    """Kernel family of the autotuner's choice ("... sf variant N ...")."""
    import re
    m = re.search(r"sf variant (\d+)", tune or "")
    return "staged" if m and int(m.group(1)) >= 6 else "owner"


N_MOL = 8192
SEED = 2026
N_FRAMES = 100
SIGMA = 0.1
METRIC = ("E+F atoms/s on 1 B200: plain FP64 vs BF16 / gated student at "
          "stated force RMSE")
TARGETS = {"energy_per_atom_rmse": 1e-4, "force_rmse": 5e-3}


def args():
    a = argparse.ArgumentParser()
    a.add_argument("--gpus", type=int, default=1)
    a.add_argument("--steps", type=int, default=200)
    a.add_argument("--warmup", type=int, default=5)
    a.add_argument("--impl", choices=["ours", "reference"], default="ours")
    a.add_argument("--frames", type=int, default=N_FRAMES)
    a.add_argument("--cpu-frames", type=int, default=5,
                   help="frames of the in-line CPU baseline")
    a.add_argument("--no-cpu-baseline", action="store_true")
    a.add_argument("--no-forms", action="store_true",
                   help="skip the mixed-precision / student comparison")
    a.add_argument("--no-config4", action="store_true",
                   help="skip the 98,304-atom precision-form configuration")
    a.add_argument("--no-batch", action="store_true",
                   help="skip the 4,096-structure batching form")
    # --profile-case
    a.add_argument("--profile-case", action="store_true")
    a.add_argument("--molecules", type=int, default=4096)
    a.add_argument("--potential", default="h2o_52")
    a.add_argument("--precision", default="fp64",
                   choices=["fp64", "mixed", "bf16"])
    a.add_argument("--evaluations", type=int, default=5)
    a.add_argument("--autotune", action="store_true")
    a.add_argument("--student-steps", type=int, default=0,
                   help="--profile-case: that many training steps of the "
                        "distilled student (h2o_92_student) instead")
    return a.parse_args()


def workload(rank: int, n_frames: int):
    from n2p2_b200 import synth
    box, pos, elem = synth.water_box(N_MOL, SEED)
    boxes, frames = synth.noisy_frames(pos, n_frames, SIGMA,
                                       seed=SEED + 1 + 1000 * rank, box=box)
    return box, frames, elem


def config(n_gpus: int, steps_note: str = ""):
    return {
        "workload": "water box, 8,192 molecules = 24,576 atoms, 1.0 g/cm^3, "
                    "L = 118.26 bohr, 100 noisy frames (sigma 0.1 bohr)",
        "potential": "h2o_52: 52 SFs/element (16 radial G2 + 36 narrow "
                     "angular G3, cos cutoff rc = 12 bohr), NN 52-25-25-1 tanh",
        "form": "plain FP64",
        "atoms_per_step_per_gpu": 3 * N_MOL,
        "l2": "per-frame working set > L2 (dG/dr buffer ~2 GB; frames cycle)",
        "parallelism": f"replicas x{n_gpus}",
        **({"note": steps_note} if steps_note else {}),
    }


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for name, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [],
                    "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# algorithmic work model (FLOPs and bytes per frame)
# ---------------------------------------------------------------------------
def potential_shape(p):
    """Counting-model parameters of a set-up Prediction: angular members per
    group M_a, radial members per group M_r, dG/dr slots per neighbor S,
    SFs per element and NN multiply-adds per atom (first element)."""
    M_a, M_r = 0, 0
    for e in range(p.num_elements):
        for g in p.symmetry_function_groups(e):
            t = int(p.symmetry_function_params(e, g[0])[0])
            if t == 2:
                M_r = max(M_r, len(g))
            else:
                M_a = max(M_a, len(g))
    S = max(p.num_slots(e, f) for e in range(p.num_elements)
            for f in range(p.num_elements))
    n_sf = max(p.num_symmetry_functions(e) for e in range(p.num_elements))
    return M_a, M_r, S, n_sf


def work_model(cnt, dr, d, shape, mac, rc=12.0):
    """Exact neighbor (n) and valid-triplet (T) counts of one frame and the
    FLOP / byte model: per triplet 40 + 60 M_a, per (pair, radial member)
    20, NN 3*2*MAC, chain rule 6 per stored Vec3D slot; bytes of the SF
    kernel = neighbor data read + dG/dr, G and dG/dr(self) written."""
    import torch
    M_a, M_r, S, n_sf = shape
    dev = torch.device("cuda")
    N = len(cnt)
    off = np.concatenate([[0], np.cumsum(cnt)])
    mx = int(cnt.max())
    # padded [atom, neighbor, xyz]; padding sits far outside the cutoff
    pad = np.full((N, mx, 3), 1e6)
    valid = np.zeros((N, mx), dtype=bool)
    for i in range(N):
        k = int(cnt[i])
        pad[i, :k] = dr[off[i]:off[i + 1]]
        valid[i, :k] = d[off[i]:off[i + 1]] < rc
    pad[~valid] = 1e6
    T = 0
    rc2 = rc * rc
    tri = torch.triu(torch.ones(mx, mx, dtype=torch.bool, device=dev), 1)
    for b in range(0, N, 1024):
        v = torch.tensor(pad[b:b + 1024], device=dev)
        ok = torch.tensor(valid[b:b + 1024], device=dev)
        dd = ((v[:, :, None, :] - v[:, None, :, :]) ** 2).sum(-1)
        m = (dd < rc2) & ok[:, :, None] & ok[:, None, :] & tri
        T += int(m.sum())
    n = int(cnt.sum())
    flops_sf = T * (40 + 60 * M_a) + n * M_r * 20
    flops_all = flops_sf + N * 3 * 2 * mac + 6 * (n * S + N * n_sf)
    bytes_sf = n * 32 + n * S * 3 * 8 + N * n_sf * 8 * 4 + N * 8 * 2
    return {"atoms": N, "neighbors": n, "triplets": T,
            "neighbors_per_atom": n / N, "triplets_per_atom": T / N,
            "M_a": M_a, "M_r": M_r, "S": S, "n_sf": n_sf, "mac_nn": mac,
            "flops_sf": flops_sf, "flops_total": flops_all,
            "bytes_sf": bytes_sf}


def fp64_peak_tflops():
    """Dense FP64 peak measured here: cuBLAS DGEMM 8192^3 via torch (best
    of 5).  The plain FP64 kernels run on the FP64 pipe."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            j = json.load(fh)
        return j.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def rmse_vs(acc, ref, n):
    de = [(e - e0) / n for (e, _), (e0, _) in zip(acc, ref)]
    df = np.concatenate([(f - f0).ravel() for (_, f), (_, f0) in zip(acc, ref)])
    return (float(np.sqrt(np.mean(np.square(de)))),
            float(np.sqrt(np.mean(np.square(df)))))


def meets(entry, ref):
    e = entry.get(f"energy_per_atom_rmse_vs_{ref}")
    f = entry.get(f"force_rmse_vs_{ref}")
    if e is None or f is None:
        return None
    return bool(e <= TARGETS["energy_per_atom_rmse"]
                and f <= TARGETS["force_rmse"])


# ---------------------------------------------------------------------------
# CPU baseline (reference library, OpenMP) -- rank 0, N = 1 only
# ---------------------------------------------------------------------------
def cpu_baseline(frames, box, elem, n_frames=5):
    from oracle import ref as oref
    lib = os.path.join(ROOT, "oracle", "_ref", "libn2p2ref_perf.so")
    if not os.path.exists(lib):
        return {"value": None, "unit": "atoms/s", "cores": 0,
                "kind": "reference", "sample": "unavailable: oracle/_ref "
                "not built"}
    oref.REF_LIB = lib
    threads = os.cpu_count() or 1
    m = oref.RefModel(POT)
    m.setup_statistics()
    t = np.zeros(5)
    k = min(n_frames, len(frames))
    for f in range(k):
        m.set_structure(frames[f], elem, box)
        t += m.time_stages(threads=threads, reps=1)
    total = float(t.sum())
    natoms = len(elem) * k
    return {"value": natoms / total, "unit": "atoms/s", "cores": threads,
            "kind": "reference",
            "sample": f"{k} frames of the 24,576-atom box, full path "
                      "(neighbor list + SF + NN + E + F); stage seconds "
                      f"NL {t[0]:.2f}, SF {t[1]:.2f}, NN {t[2]:.2f}, "
                      f"E {t[3]:.4f}, F {t[4]:.2f}; without the O(N^2) "
                      f"neighbor list: {natoms / (total - t[0]):.0f} atoms/s"}


def run_reference(a):
    """--impl reference: the reference CPU path on the same workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ref as oref
    lib = os.path.join(ROOT, "oracle", "_ref", "libn2p2ref_perf.so")
    if not os.path.exists(lib):
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref not built here"}))
        return
    oref.REF_LIB = lib
    box, frames, elem = workload(0, min(a.frames, max(a.steps, 1) + 1))
    threads = os.cpu_count() or 1
    m = oref.RefModel(POT)
    m.setup_statistics()   # no extrapolation-warning output, as our arm
    # one warm-up frame (a CPU path has no device warm-up to amortize)
    m.set_structure(frames[0], elem, box)
    t0 = time.perf_counter()
    m.time_stages(threads=threads, reps=1)
    per = time.perf_counter() - t0
    budget = 150.0
    k = max(1, min(a.steps, int(budget / max(per, 1e-3))))
    tot = np.zeros(5)
    for s in range(k):
        m.set_structure(frames[(s + 1) % len(frames)], elem, box)
        tot += m.time_stages(threads=threads, reps=1)
    secs = float(tot.sum())
    val = len(elem) * k / secs
    note = "" if k == a.steps else (f"timed {k} of {a.steps} requested steps "
                                    "(150 s budget; one frame per step)")
    line = {
        "metric": METRIC, "value": val, "unit": "atoms/s", "impl": "reference",
        "n_gpus": a.gpus, "steps": k, "warmup": 1,
        "ms_per_step": 1e3 * secs / k, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config(a.gpus, note),
        "cpu_baseline": {"value": val, "unit": "atoms/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"{k} full frame(s) per run, stage "
                                   f"seconds NL {tot[0]:.2f} SF {tot[1]:.2f} "
                                   f"NN {tot[2]:.2f} E {tot[3]:.4f} "
                                   f"F {tot[4]:.2f}"},
        "e2e": {"value": val, "unit": "atoms/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def _time_steps(p, frames_dev, steps, stream, lib):
    """Device time of `steps` evaluations on device-resident frames (CUDA
    events on the library's stream) and the number of launches."""
    import torch
    F = len(frames_dev)
    l0 = lib.n2p2b_kernel_launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for s in range(steps):
        p.set_positions(frames_dev[s % F])
        p.evaluate_async(True)
    ev1.record(stream)
    p.finish()
    return ev0.elapsed_time(ev1) / 1e3, int(lib.n2p2b_kernel_launch_count()
                                            - l0)


def _stage_ms(p, frames_dev, steps):
    F = len(frames_dev)
    p.set_profiling(True)
    p.stage_times(reset=True)
    for s in range(steps):
        p.set_positions(frames_dev[s % F])
        p.evaluate_async(True)
    p.finish()
    ms, runs = p.stage_times(reset=True)
    p.set_profiling(False)
    return [x / max(runs, 1) for x in ms]


def _eval_frames(p, frames, box=None, elem=None):
    """(energy, forces) of each frame (host arrays); a new box sets the
    structure, otherwise only positions change."""
    out = []
    for x in frames:
        if box is not None:
            p.set_structure(x, elem, box)
        else:
            p.set_positions(x)
        p.evaluate_nnp(True)
        out.append((p.energy, p.forces().copy()))
    return out


def measure_forms(box, frames, elem, dev_frames, stream, lib, steps, local):
    """Plain FP64 vs the mixed forms on the same 24,576-atom frames, for the
    52-SF potential and the wider 92-SF / 64-64-64 softplus potential, and
    for the latter the distilled 92-32-1 student (gated by its training
    range; atoms outside it are re-evaluated by the teacher on the tensor
    cores).  Accuracy is measured against the FP64 form on three frames (the
    FP64 form equals the reference to 1e-10 on this very workload,
    tests/test_gpu_bench_parity.py) and, for the student, also against the
    mixed-precision teacher."""
    from n2p2_b200.mode import Prediction
    n = len(elem)
    out = {}
    for pot in ("h2o_52", "h2o_92"):
        p = Prediction(os.path.join(POT_DIR, pot), device=local)
        p.setup()
        p.setup_symmetry_function_statistics(False, False, False, False)
        p.set_stream(stream.cuda_stream)
        p.set_structure(frames[0], elem, box)
        forms = [("fp64", "fp64", None), ("mixed", "mixed", None),
                 ("bf16", "bf16", None)]
        sdir = os.path.join(POT_DIR, pot + "_student")
        has_student = os.path.exists(os.path.join(sdir,
                                                  "training_range.data"))
        if has_student:
            p.setup_student(sdir)
            forms += [("student_gated", "mixed", "gated"),
                      ("student_only", "mixed", "only")]
        refs = {}
        tunes = {}
        for name, prec, smode in forms:
            p.set_precision(prec)
            if has_student:
                p.set_student_mode(smode if smode else "off")
            p.set_positions(frames[0])
            p.evaluate_nnp(True)
            if prec not in tunes:
                tunes[prec] = p.autotune(True, 1)
            for s in range(3):
                p.set_positions(dev_frames[s])
                p.evaluate_async(True)
            p.finish()
            t, launches = _time_steps(p, dev_frames, steps, stream, lib)
            stage = _stage_ms(p, dev_frames, min(steps, 10))
            acc = _eval_frames(p, frames[:3])
            gated = []
            if smode == "gated":
                for s in range(3):
                    p.set_positions(frames[s])
                    p.evaluate_nnp(True)
                    gated.append(p.student_gated_count() / n)
            entry = {"value": n * steps / t, "unit": "atoms/s",
                     "ms_per_step": 1e3 * t / steps, "steps": steps,
                     "gpu_launches_per_step": launches / steps,
                     "stage_ms_per_step": dict(zip(STAGES, stage)),
                     "autotune": tunes[prec]}
            refs[name] = acc
            for rname in (("fp64", "mixed") if smode else ("fp64",)):
                if name == rname:
                    continue
                e_r, f_r = rmse_vs(acc, refs[rname], n)
                entry[f"energy_per_atom_rmse_vs_{rname}"] = e_r
                entry[f"force_rmse_vs_{rname}"] = f_r
            if name != "fp64":
                entry["speedup_vs_fp64"] = (
                    entry["value"] / out[pot]["fp64"]["value"])
                entry["meets_targets"] = meets(entry, "fp64")
            if gated:
                entry["gated_fraction"] = float(np.mean(gated))
            out.setdefault(pot, {})[name] = entry
        out[pot]["force_rms"] = float(
            np.sqrt(np.mean(np.square(refs["fp64"][0][1]))))
        if has_student:
            out[pot]["student_gated_compressed"] = measure_gated_compressed(
                p, box, elem, stream, lib, steps)
        p.close()
    out["targets"] = dict(TARGETS, units="potential energy units; energy / "
                                         "bohr")
    out["forms"] = {
        "fp64": "plain form, everything FP64",
        "mixed": "FP32 symmetry functions + dG/dr; NN on tcgen05 with BF16 "
                 "hi/lo operand pairs (3 MMAs per step), FP32 accumulation; "
                 "FP64 displacements, energy sum, force accumulation",
        "bf16": "as mixed, except single BF16 deltas against hi/lo "
                "weights in the backward GEMMs of the hidden layers above "
                "the first (2 MMAs per step there); meets_targets says "
                "whether its RMSE is inside the targets",
        "student_gated": "FP32 symmetry functions; distilled 92-32-1 FP32 "
                         "student for atoms inside its training range, the "
                         "mixed-precision teacher for the others",
        "student_only": "the student for every atom (no gate)",
        "student_gated_compressed": "the gated student on frames outside "
                                    "its training distribution (box and "
                                    "positions compressed by 5 %, noise "
                                    "sigma 0.25 bohr), where the gate hands "
                                    "atoms to the teacher"}
    return out


def measure_gated_compressed(p, box, elem, stream, lib, steps):
    """The gated student (its Prediction already set up) on frames the
    student was not trained for -- compressed by 5 % with sigma = 0.25 bohr
    noise (its training used +-3 % and sigma <= 0.2) -- so that a part of the
    atoms falls outside its training range and goes to the teacher.  Speed
    with that gated fraction, and accuracy against the FP64 form."""
    import torch
    from n2p2_b200 import synth
    n = len(elem)
    s = 0.95
    bx = box * s
    _, pos0, _ = synth.water_box(N_MOL, SEED)
    _, fr = synth.noisy_frames(pos0 * s, 12, 0.25, seed=SEED + 77)
    dev = torch.tensor(fr, dtype=torch.float64, device="cuda")
    p.set_precision("fp64")
    p.set_student_mode("off")
    ref = _eval_frames(p, fr[:3], bx, elem)
    p.set_precision("mixed")
    p.set_student_mode("gated")
    p.set_structure(fr[0], elem, bx)
    p.evaluate_nnp(True)
    for k in range(3):
        p.set_positions(dev[k])
        p.evaluate_async(True)
    p.finish()
    t, launches = _time_steps(p, dev, steps, stream, lib)
    acc, gated = [], []
    for k in range(3):
        p.set_positions(fr[k])
        p.evaluate_nnp(True)
        acc.append((p.energy, p.forces().copy()))
        gated.append(p.student_gated_count() / n)
    e_r, f_r = rmse_vs(acc, ref, n)
    entry = {"value": n * steps / t, "unit": "atoms/s",
             "ms_per_step": 1e3 * t / steps, "steps": steps,
             "gated_fraction": float(np.mean(gated)),
             "energy_per_atom_rmse_vs_fp64": e_r, "force_rmse_vs_fp64": f_r,
             "frames": "box x0.95, sigma 0.25 bohr, 12 frames"}
    entry["meets_targets"] = meets(entry, "fp64")
    p.set_student_mode("off")
    return entry


def measure_config4(stream, lib, local, steps=10):
    """The precision form as specified: 32,768 water molecules = 98,304
    atoms (L = 187.7 bohr at 1.0 g/cm^3), the 92-SF / 64-64-64 softplus
    potential (h2o_92), three noisy frames (sigma 0.1 bohr).  FP64 vs mixed
    atoms/s (device-resident frames), per-atom energy and force RMSE of the
    mixed form against the FP64 form (3 frames) and of both against the
    reference CPU library on the first frame."""
    import torch
    from n2p2_b200 import synth
    from n2p2_b200.mode import Prediction
    pot = os.path.join(POT_DIR, "h2o_92")
    t0 = time.perf_counter()
    box, pos, elem = synth.water_box(32768, 2030)
    _, fr = synth.noisy_frames(pos, 3, SIGMA, seed=2031, box=box)
    gen = time.perf_counter() - t0
    n = len(elem)
    dev = torch.tensor(fr, dtype=torch.float64, device="cuda")
    p = Prediction(pot, device=local)
    p.setup()
    p.setup_symmetry_function_statistics(False, False, False, False)
    p.set_stream(stream.cuda_stream)
    out = {"atoms": n, "box_bohr": float(box[0, 0]),
           "potential": "h2o_92: 92 SFs/element, NN 92-64-64-64-1 softplus",
           "generation_s": gen}
    res = {}
    for prec in ("fp64", "mixed"):
        p.set_precision(prec)
        p.set_structure(fr[0], elem, box)
        p.evaluate_nnp(True)
        tune = p.autotune(True, 1)
        for k in range(3):
            p.set_positions(dev[k])
            p.evaluate_async(True)
        p.finish()
        t, _ = _time_steps(p, dev, steps, stream, lib)
        stage = _stage_ms(p, dev, 3)
        res[prec] = _eval_frames(p, fr)
        out[prec] = {"value": n * steps / t, "unit": "atoms/s",
                     "ms_per_step": 1e3 * t / steps, "steps": steps,
                     "stage_ms_per_step": dict(zip(STAGES, stage)),
                     "autotune": tune}
    p.close()
    e_r, f_r = rmse_vs(res["mixed"], res["fp64"], n)
    out["mixed"]["energy_per_atom_rmse_vs_fp64"] = e_r
    out["mixed"]["force_rmse_vs_fp64"] = f_r
    out["mixed"]["speedup_vs_fp64"] = (out["mixed"]["value"]
                                       / out["fp64"]["value"])
    out["mixed"]["meets_targets"] = meets(out["mixed"], "fp64")
    from oracle import ref as oref
    if oref.ref_available():
        t0 = time.perf_counter()
        ref = oref.RefModel(pot)
        ref.setup_statistics()
        ref.set_structure(fr[0], elem, box)
        e0, f0 = ref.predict()
        out["reference_frame_s"] = time.perf_counter() - t0
        for prec in ("fp64", "mixed"):
            e_r, f_r = rmse_vs(res[prec][:1], [(e0, f0)], n)
            out[prec]["energy_per_atom_rmse_vs_reference"] = e_r
            out[prec]["force_rmse_vs_reference"] = f_r
        e, f = res["fp64"][0]
        scale = np.maximum(np.abs(f0), np.sqrt(np.mean(f0 ** 2)))
        out["fp64"]["relative_energy_error_vs_reference"] = abs(e - e0) / abs(
            e0)
        out["fp64"]["max_force_error_vs_reference"] = float(
            (np.abs(f - f0) / scale).max())
        del ref
    return out


def measure_batch(stream, lib, local, n_structures=4096, steps=5,
                  check=64):
    """Batching form: 4,096 independent water boxes of 11-171 molecules
    (33-513 atoms, density 1.0 g/cm^3), evaluated together as one CUDA-graph
    launch after the autotuner picked the launch configuration for their
    size bucket (tuned on a 256-structure sample of the same distribution).
    Compared with a loop that evaluates one structure per call.  The FP64
    batch result of `check` structures (the largest and smallest included)
    is compared with the reference library, structure by structure."""
    import torch
    from n2p2_b200 import synth
    from n2p2_b200.mode import Prediction
    t0 = time.perf_counter()
    structs = synth.batch_structures(n_structures, 2027, device=f"cuda:{local}")
    sample = synth.batch_structures(256, 2028, device=f"cuda:{local}")
    gen_s = time.perf_counter() - t0
    natoms = sum(len(s[2]) for s in structs)
    sizes = np.array([len(s[2]) for s in structs])
    out = {"structures": n_structures, "atoms": natoms,
           "atoms_per_structure": [int(sizes.min()), int(sizes.max())],
           "generation_s": gen_s}
    p = Prediction(POT, device=local)
    p.setup()
    p.setup_symmetry_function_statistics(False, False, False, False)
    p.set_stream(stream.cuda_stream)
    for prec in ("fp64", "mixed"):
        p.set_precision(prec)
        p.set_structures(sample)
        p.evaluate_nnp(True)
        tune = p.autotune(True, 1)
        p.set_structures(structs)
        p.evaluate_nnp(True)
        if prec == "fp64":
            E = p.structure_energies()
            F = p.forces()
        p.capture_graph(True)
        p.launch_graph()
        p.finish()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        l0 = lib.n2p2b_kernel_launch_count()
        ev0.record(stream)
        for _ in range(steps):
            p.launch_graph()
        ev1.record(stream)
        p.finish()
        t = ev0.elapsed_time(ev1) / 1e3
        out[prec] = {"value": natoms * steps / t, "unit": "atoms/s",
                     "ms_per_batch": 1e3 * t / steps, "steps": steps,
                     "graph_launches_per_batch": 1,
                     "kernels_per_graph": "the evaluation pipeline "
                                          "(captured once; replays are not "
                                          "counted as launches)",
                     "autotune": tune}
    # Per-structure errors of the FP64 batch against the reference.
    from oracle import ref as oref
    if oref.ref_available():
        ref = oref.RefModel(POT)
        ref.setup_statistics()
        off = np.concatenate([[0], np.cumsum(sizes)])
        pick = sorted(set([int(sizes.argmax()), int(sizes.argmin())]
                          + list(np.random.default_rng(5).choice(
                              n_structures, check - 2, replace=False))))
        we, wf = 0.0, 0.0
        for s in pick:
            box, x, el = structs[s]
            ref.set_structure(x, el, box)
            e0, f0 = ref.predict()
            f = F[off[s]:off[s + 1]]
            scale = np.maximum(np.abs(f0), np.sqrt(np.mean(f0 ** 2)))
            we = max(we, abs(E[s] - e0) / abs(e0))
            wf = max(wf, float((np.abs(f - f0) / scale).max()))
        out["fp64"]["reference_check"] = {
            "structures": len(pick),
            "atoms_range": [int(sizes[pick].min()), int(sizes[pick].max())],
            "max_relative_energy_error": we,
            "max_force_error": wf,
            "force_error_measure": "|dF| / max(|F|, rms F) per component"}
    # One structure per call (set_structure + evaluate), on a sample.
    p.set_precision("fp64")
    k = 512
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    na = 0
    for box, x, el in structs[:k]:
        p.set_structure(x, el, box)
        p.evaluate_nnp(True)
        na += len(el)
    p.finish()
    t = time.perf_counter() - t0
    out["loop_fp64"] = {"value": na / t, "unit": "atoms/s",
                        "sample": f"first {k} structures, one "
                                  "set_structure + evaluate per structure"}
    out["speedup_fp64_vs_loop"] = out["fp64"]["value"] / out["loop_fp64"][
        "value"]
    p.close()
    return out


def run_ours(a):
    import torch
    from n2p2_b200.replicas import Replicas
    # One process per GPU, each on its own frames (weak scaling); NCCL only
    # for the barrier and the maximum of the ranks' times.
    rep = Replicas("nccl")
    world, rank, local = rep.world, rep.rank, rep.local

    from n2p2_b200 import _capi
    from n2p2_b200.mode import Prediction

    box, frames, elem = workload(rank, a.frames)
    n = len(elem)
    F = len(frames)
    dev_frames = torch.tensor(frames, dtype=torch.float64, device="cuda")
    host_frames = torch.tensor(frames, dtype=torch.float64).pin_memory()
    host_forces = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    stream = torch.cuda.Stream()

    p = Prediction(POT, device=local)
    p.setup()
    # Hot path only: no extrapolation-warning output (the reference arm runs
    # with the same setting).
    p.setup_symmetry_function_statistics(False, False, False, False)
    p.set_stream(stream.cuda_stream)
    p.set_structure(host_frames[0].numpy(), elem, box)
    p.evaluate_nnp(True)          # sizes all buffers (capacity known)
    # Launch configuration for this size bucket (Prediction.autotune, the
    # library's own tuner; part of setup, outside the timed region).
    tune = p.autotune(True, 1)
    lib = _capi.load()

    # ---- warm-up ---------------------------------------------------------
    for s in range(max(a.warmup, 3)):
        p.set_positions(dev_frames[s % F])
        p.evaluate_async(True)
    p.finish()

    with ClockSampler(local) as clocks:
        # ---- value: device-resident frames -------------------------------
        rep.barrier()
        t_dev, launches = _time_steps(p, dev_frames, a.steps, stream, lib)
        rep.barrier()
        t_dev = rep.max(t_dev)

        # ---- e2e: host buffers through the C-ABI -------------------------
        rep.barrier()
        t0 = time.perf_counter()
        energy = 0.0
        for s in range(a.steps):
            p.set_positions(host_frames[s % F].numpy())
            p.evaluate_nnp(True)
            p._check(lib.n2p2b_get_forces(p._h, host_forces.data_ptr(),
                                          _capi.HOST))
            energy = p.energy
        rep.barrier()
        t_e2e = rep.max(time.perf_counter() - t0)

        # ---- profiled pass: per-stage device time -------------------------
        per = _stage_ms(p, dev_frames, a.steps)
    clock_summary = clocks.summary()

    # ---- the other forms and configurations (one GPU only) ----------------
    forms = config4 = batch = None
    if world == 1 and not a.no_forms:
        forms = measure_forms(box, frames, elem, dev_frames, stream, lib,
                              min(a.steps, 50), local)
    if world == 1 and not a.no_config4:
        config4 = measure_config4(stream, lib, local)
    if world == 1 and not a.no_batch:
        batch = measure_batch(stream, lib, local)

    rep.barrier()

    atoms_total = n * a.steps * world
    value = atoms_total / t_dev
    e2e = atoms_total / t_e2e
    if rank != 0:
        rep.close()
        return

    # ---- roofline of the dominant kernel (symmetry functions) -------------
    p.set_positions(dev_frames[0])
    p.evaluate_nnp(True)
    cnt, index, dr, d = p.neighbor_list()
    mac = 52 * 25 + 25 * 25 + 25
    wm = work_model(cnt, dr, d, potential_shape(p), mac)
    sf_s = per[1] / 1e3
    hbm_peak, peak_kind = measured_peaks()
    gbs = wm["bytes_sf"] / sf_s / 1e9
    fp64_peak = fp64_peak_tflops()
    sf_tflops = wm["flops_sf"] / sf_s / 1e12

    line = {
        "metric": METRIC,
        "value": value, "unit": "atoms/s",
        "n_gpus": world, "steps": a.steps, "warmup": max(a.warmup, 3),
        "ms_per_step": 1e3 * t_dev / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "config": config(world),
        "e2e": {"value": e2e, "unit": "atoms/s",
                "h2d_bytes_per_step": n * 3 * 8,
                "d2h_bytes_per_step": n * 3 * 8 + 8,
                "path": "n2p2b_set_positions(host) + n2p2b_evaluate + "
                        "n2p2b_get_forces(host) + n2p2b_get_energy"},
        "gpu_launches": launches,
        "stage_ms_per_step": dict(zip(STAGES, per)),
        "autotune": tune,
        "roofline": {
            "kernel": ("sfStagedKernel<double>" if sf_family(tune) == "staged"
                       else "sfKernel<double>")
                      + " (symmetry functions + dG/dr)",
            "bound": "fp64",
            "achieved": sf_tflops, "peak": fp64_peak, "unit": "TFLOP/s",
            "frac": sf_tflops / fp64_peak,
            "peak_source": "cuBLAS DGEMM 8192^3 timed in this run "
                           "(builder-measured: the driver's peaks file has "
                           "no FP64 figure)",
            "achieved_source": "counting-model FLOPs of the frame (exact "
                               "triplet and neighbor counts, see work) / "
                               "the SF stage's CUDA-event time",
            "algorithmic_flops_per_launch": wm["flops_sf"],
            "traffic": SF_TRAFFIC[sf_family(tune)][0],
            "traffic_source": SF_TRAFFIC[sf_family(tune)][1],
            "hbm": {"achieved": gbs, "peak": hbm_peak, "unit": "GB/s",
                    "frac": gbs / hbm_peak,
                    "peak_source": f"{peak_kind} (MEASURED_PEAKS.json "
                                   "hbm_gbs)",
                    "algorithmic_bytes_per_launch": wm["bytes_sf"]}},
        "work": wm,
        "energy_last_frame": energy,
        "clocks": clock_summary,
    }
    if forms is not None:
        line["forms"] = forms
    if config4 is not None:
        line["config4"] = config4
    if batch is not None:
        line["batch"] = batch
    if not a.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(frames, box, elem, a.cpu_frames)
    print(json.dumps(line))
    rep.close()


def profile_case(a):
    """A small fixed evaluation for profilers and quick timings: a seed-77
    water box of --molecules molecules on one of the test potentials,
    --evaluations evaluations (energy + forces); prints the per-stage
    device times of the last three.  The symmetry-function kernel of
    evaluation k is that kernel's launch k (the first evaluation's sizing
    pass launches the neighbor list only).  --autotune runs the library's
    tuner first and prints its choice; a capture that should see launch k
    passes that choice through N2P2B_SF_VARIANT / N2P2B_SF_SORT instead,
    because the tuner launches every configuration."""
    from n2p2_b200 import synth
    from n2p2_b200.mode import Prediction
    box, pos, elem = synth.water_box(a.molecules, 77)
    if a.student_steps:
        return profile_student(a, box, pos, elem)
    p = Prediction(os.path.join(POT_DIR, a.potential))
    p.setup()
    p.setup_symmetry_function_statistics(False, False, False, False)
    p.set_precision(a.precision)
    p.set_structure(pos, elem, box)
    if a.autotune:
        p.evaluate_nnp(True)
        print("autotune", p.autotune(True, 3))
    for _ in range(max(a.evaluations - 3, 1)):
        p.evaluate_nnp(True)
    p.set_profiling(True)
    p.stage_times(True)
    for _ in range(3):
        p.evaluate_nnp(True)
    ms, runs = p.stage_times(True)
    print(a.potential, a.precision, len(elem), "atoms; stage ms "
          "(NL, SF, NN, E, F):", [round(x / runs, 3) for x in ms],
          "energy", p.energy)


def profile_student(a, box, pos, elem):
    """--profile-case --student-steps K: K Adam steps of the distilled
    92-32-1 student (tests/golden/potentials/h2o_92_student, in memory
    only) on batches of 4,096 atoms of one frame labelled by its FP64
    teacher; prints the device time per step."""
    import torch
    from n2p2_b200.mode import Prediction
    teacher = os.path.join(POT_DIR, "h2o_92")
    t = Prediction(teacher)
    t.setup()
    t.setup_symmetry_function_statistics(False, False, False, False)
    t.set_structure(pos, elem, box)
    t.evaluate_nnp(True)
    E = torch.tensor(t.atomic_energies(), dtype=torch.float64, device="cuda")
    F = torch.tensor(t.forces(), dtype=torch.float64, device="cuda")
    t.close()
    p = Prediction(teacher)
    p.setup()
    p.setup_symmetry_function_statistics(False, False, False, False)
    p.set_precision("mixed")
    p.setup_student(os.path.join(POT_DIR, "h2o_92_student"))
    p.set_structure(pos, elem, box)
    p.calculate_neighbor_list()
    p.calculate_symmetry_function_groups(True)
    n = len(elem)
    idx = torch.arange(min(4096, n), dtype=torch.int32, device="cuda")
    for _ in range(3):
        p.student_train_step(E, F, idx, 1.0, 1.0, 1e-6)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.student_steps):
        p.student_train_step(E, F, idx, 1.0, 1.0, 1e-6)
    e1.record()
    torch.cuda.synchronize()
    print(f"student training: {a.student_steps} steps of {int(idx.numel())} "
          f"atoms, {e0.elapsed_time(e1) / a.student_steps:.3f} ms per step")
    p.close()


def main():
    a = args()
    if a.profile_case:
        profile_case(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
