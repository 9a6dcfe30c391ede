#!/usr/bin/env python
"""Benchmark of the sinc-DVR orbital right-hand side on B200.

Metric: orbital-RHS evaluations per second.  One evaluation (one "step") is a
mean-field build -- 1-RDM, its regularised inverse and the 2-RDM from the
A-vector over the walk tables, pair densities, Toeplitz/FFT Coulomb solves,
twoematel, reducedpot -- followed by one actreduced00 on the same orbitals
(MCTDH.SRC/derivs.f90:629-852 with the SINCDVR project operators).

Workload B (default): two Z=1 nuclei at z=+-0.75 bohr, 41^3 grid, spacing 0.25,
10 orbitals, 2 electrons (full M_s=0 CI, 100 configurations), complex128,
seeded synthetic orbitals and A-vector.

  python bench.py [--gpus N --steps K --warmup W]      # this implementation
  python bench.py --impl reference [...]               # CPU reference restatement

Multi-GPU: independent replicas (the path has no exchange step); value is the
sum over ranks, timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "v1-1_b200"))

import numpy as np  # noqa: E402

METRIC = "orbital-RHS evals/s"
UNIT = "evals/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="C", choices=["A", "B", "C"])
    ap.add_argument("--no-workload-b", action="store_true",
                    help="skip the 41^3 / 10-orbital workload measured beside the headline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="only the warm-up and timed evaluations (profiling runs)")
    ap.add_argument("--profile-precision-form", action="store_true",
                    help="with --no-extras: time the precision form (FP32 Coulomb passes, 3xTF32 "
                         "tensor-core reducedpot) instead of the FP64 form")
    ap.add_argument("--precision-trajectory", type=int, default=0, metavar="STEPS",
                    help="instead of the benchmark: STEPS field-free CMF steps of the workload in the FP64 form, "
                         "the precision form and the precision form with FP64 final mean fields; per-quantity "
                         "errors against the FP64 form")
    ap.add_argument("--only", choices=["served", "batched", "propagation"], default=None,
                    help="run only the served or the batched form, or the CMF steps of the workload, and print "
                         "its object")
    ap.add_argument("--stages", action="store_true",
                    help="with --no-extras: also time each stage on one stream (per-stage CUDA events)")
    ap.add_argument("--e2e", action="store_true",
                    help="with --no-extras: also time the end-to-end host-array entry")
    ap.add_argument("--option", action="append", default=[], metavar="NAME=VALUE",
                    help="context option for the measured workloads (sincgpu_set_option), e.g. coul_fused=1")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--batched-count", type=int, default=64)
    ap.add_argument("--served-count", type=int, default=24)
    ap.add_argument("--served-steps", type=int, default=10)
    ap.add_argument("--served-full", action="store_true",
                    help="served stream at the stated sizes (31^3-81^3 grids, 2-6 electrons, 4-16 orbitals); "
                         "use with --served-steps 200")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload_config(w, l2="flushed (256 MiB write between timed steps)"):
    return {
        "workload": f"{w.name}: {w.note}, {w.numpoints}^3 grid, spacing {w.spacing}, "
                    f"{w.nspf} orbitals, nuclei Z={list(w.nuccharges)} at centershift {list(map(list, w.centershift))}",
        "numpoints": w.numpoints, "nspf": w.nspf, "pairs": w.nspf * (w.nspf + 1) // 2,
        "l2": l2, "parallelism": "replicas",
    }


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
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
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU reference (oracle restatement), used for --impl reference and cpu_baseline
# ---------------------------------------------------------------------------
def oracle_walks(w):
    """The oracle's CI object for workload `w`.  Up to a few hundred determinants
    the oracle builds its own walk tables; above that (the 14400-determinant
    workload, where its pure-Python builder needs minutes) the tables come from
    the library's host builder, which equals the oracle's bit for bit
    (tests/test_walks.py, frozen digests of the 4-electron / 16-orbital tables),
    and the oracle's numpy RDM routines run on them.  Set-up, not timed."""
    from oracle.walks_oracle import CIWalks
    from sincgpu import WalkTables
    from sincgpu.inputs import ci_size
    if ci_size(w.numelec, w.nspf) <= 1000:
        return CIWalks(w.numelec, w.nspf, 0), "oracle"
    wt = WalkTables(w.numelec, w.nspf, 0)
    ow = object.__new__(CIWalks)
    ow.numelec = ow.numpart = w.numelec
    ow.nspf, ow.restrictms, ow.numconfig = w.nspf, 0, wt.numconfig
    for name in ("configlist", "numsinglewalks", "numdoublewalks", "singlewalk", "singlewalkdirphase",
                 "singlewalkopspf", "doublewalk", "doublewalkdirphase", "doublewalkdirspf"):
        setattr(ow, name, wt.table(name))
    ow.scol = np.concatenate([[0], np.cumsum(ow.numsinglewalks)]).astype(np.int64)
    ow.dcol = np.concatenate([[0], np.cumsum(ow.numdoublewalks)]).astype(np.int64)
    wt.close()
    return ow, "library host builder (bit-identical to the oracle's)"


def cpu_reference_eval(w, threads, want_outputs=False):
    """Seconds for one orbital-RHS evaluation with the CPU restatement of the
    reference (1-RDM + regularised inverse + 2-RDM from the A-vector, pair
    Coulomb solves and twoematel, reducedpot, actreduced00), a description of
    what was timed, and, for a complete evaluation with `want_outputs`, its RHS
    and twoematel.

    Grids up to 41^3 run the whole evaluation.  Larger workloads time a
    bounded sample: the Coulomb solves of
    4 of the reference's n op_tinv batches (one batch = the n densities of one
    orbital b, coreproject.f90:1042-1081) and the twoematel contractions of n of
    its n^2 (a1, b1) rows (coreproject.f90:1089-1099), each scaled to the full
    count, plus the complete RDMs, reducedpot and actreduced00."""
    sys.path.insert(0, str(REPO))
    from oracle import sinc_oracle as orc
    from sincgpu.inputs import seeded_avector, seeded_orbitals
    sysm = orc.SincSystem(w.numpoints, w.spacing, w.centershift, w.nuccharges)
    ow, tables = oracle_walks(w)
    phi = seeded_orbitals(w.numpoints, w.spacing, w.nspf, seed=1)
    a = seeded_avector(ow.numconfig, seed=2)
    n, G = w.nspf, w.G
    full = w.numpoints <= 41
    t0 = time.perf_counter()
    den = ow.getdenmat00(a)
    inv = orc.invmatsmooth(den)
    tally = ow.get_tworeducedx(a)
    t_ci = time.perf_counter() - t0
    if full:
        t0 = time.perf_counter()
        mat, red = sysm.call_twoe_matel00(phi, phi, workers=threads)
        rp = orc.get_reducedpot(red, tally)
        rhs = orc.actreduced00(sysm, phi, phi, den, inv, rp)
        t = t_ci + time.perf_counter() - t0
        sample = (f"1 complete orbital-RHS evaluation, numpy/scipy restatement of the reference on {threads} host "
                  f"threads (walk tables: {tables}, set-up)")
        return t, sample, ({"rhs": rhs, "twoematel": mat} if want_outputs else None)
    nb = 4
    red = np.empty((G, n, n), dtype=np.complex128, order="F")
    t0 = time.perf_counter()
    for b in range(nb):                                   # coreproject.f90:1042-1081
        den_b = phi * np.conj(phi[:, b])[:, None]
        red[:, :, b] = sysm.op_tinv(den_b, workers=threads)
    t_coul = (time.perf_counter() - t0) * n / nb
    for b in range(nb, n):                                # values for the timed GEMMs below (not timed)
        red[:, :, b] = red[:, :, b % nb]
    R = red.reshape(G, n * n, order="F")
    mat = np.zeros((n, n, n, n), dtype=np.complex128, order="F")
    t0 = time.perf_counter()
    for a1 in range(n):                                   # coreproject.f90:1089-1099, row b1 = 0
        myden = phi[:, a1] * np.conj(phi[:, 0])
        mat[a1, 0, :, :] = (R.T @ myden).reshape(n, n, order="F")
    t_twoe = (time.perf_counter() - t0) * n
    t0 = time.perf_counter()
    rp = orc.get_reducedpot(red, tally)
    orc.actreduced00(sysm, phi, phi, den, inv, rp)
    t_rest = time.perf_counter() - t0
    t = t_ci + t_coul + t_twoe + t_rest
    sample = (f"bounded sample of one orbital-RHS evaluation, numpy/scipy restatement of the reference on {threads} "
              f"host threads: RDMs {t_ci:.2f} s, Coulomb solves {nb} of {n} op_tinv batches x {n / nb:g} = "
              f"{t_coul:.2f} s, twoematel {n} of {n * n} rows x {n} = {t_twoe:.2f} s, reducedpot + actreduced00 "
              f"{t_rest:.2f} s (walk tables: {tables}, set-up)")
    return t, sample, None


def parity_report(w, outputs, ref):
    """GPU outputs of the timed evaluation (rank 0's seeded inputs) against the
    oracle: the live CPU evaluation where it ran completely, else the oracle's
    results frozen in tests/golden/workload_C.npz (same seeds) for that workload."""
    def rel(x, y):
        return float(np.abs(x - y).max() / np.abs(y).max())
    if ref is not None:
        return {"against": "oracle (numpy/scipy restatement), same seeded inputs, this run",
                "rhs_rel_err": rel(outputs["rhs"], ref["rhs"]),
                "twoematel_rel_err": rel(outputs["twoematel"], ref["twoematel"]), "tolerance": 1e-11}
    gold_path = REPO / "tests" / "golden" / f"workload_{w.name}.npz"
    if not gold_path.exists():
        return None
    gold = np.load(gold_path)
    pts = gold["points"]
    return {"against": f"oracle results frozen in tests/golden/{gold_path.name} (same seeded inputs)",
            "rhs_rel_err": float(np.abs(outputs["rhs"][pts] - gold["rhs_pts"]).max() / gold["rhs_absmax"]),
            "rhs_points_compared": int(pts.size) * w.nspf,
            "twoematel_rel_err": rel(outputs["twoematel"], gold["twoematel"]), "tolerance": 1e-11}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from sincgpu.inputs import WORKLOADS
    w = WORKLOADS[args.config]
    threads = os.cpu_count() or 1
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_reference_eval(w, threads)
    runs = [cpu_reference_eval(w, threads) for _ in range(max(1, min(args.steps, 3)))]
    ts = [r[0] for r in runs]
    t = float(np.median(ts))
    v = 1.0 / t
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0,
        "steps": len(ts), "warmup": min(args.warmup, 1), "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
        "data": "synthetic", "config": workload_config(w, l2="n/a (CPU)"),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"median of {len(ts)}: {runs[-1][1]}; the Fortran reference has no compiler "
                                   f"in this image"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# this implementation
# ---------------------------------------------------------------------------
def measure(w, args, rank, world, local, dist, extras=True, e2e=True, propagation=True):
    """Device-timed evaluations of workload `w` (inputs resident, L2 flushed
    between steps), then, with `extras`, the secondary rates, the precision form,
    the per-stage profile and roofline, CMF steps/s and the end-to-end rate
    through the host-array entry.  Returns the numbers and rank 0's outputs."""
    import torch
    from sincgpu import SincProject, WalkTables
    from sincgpu.inputs import seeded_avector, seeded_orbitals

    n, G = w.nspf, w.G
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    proj = SincProject(w.numpoints, w.spacing, w.centershift, w.nuccharges, n, device=local)
    proj.set_stream(stream.cuda_stream)
    for opt in args.option:
        name, value = opt.split("=")
        proj.set_option(name, int(value))
    walks = WalkTables(w.numelec, n, 0)
    proj.ci_attach(walks)
    nc = walks.numconfig

    phi_h = seeded_orbitals(w.numpoints, w.spacing, n, seed=1 + rank)
    a_h = seeded_avector(nc, seed=2 + rank)

    def dev_from_fortran(x):
        return torch.from_numpy(np.ascontiguousarray(np.asarray(x).T)).to(dev)

    phi = dev_from_fortran(phi_h)
    avec = dev_from_fortran(a_h)
    cplx = dict(dtype=torch.complex128, device=dev)
    den = torch.empty((n, n), **cplx)
    inv = torch.empty((n, n), **cplx)
    tally = torch.empty((n, n, n, n), **cplx)
    mat = torch.empty((n, n, n, n), **cplx)
    red = torch.empty((n, n, G), **cplx)
    out = torch.empty((n, G), **cplx)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step():
        proj.orbital_rhs_avec_dev(phi, avec, den, inv, tally, mat, red, out)

    if args.profile_precision_form:
        proj.set_option("coulomb_fp32", 1)
        proj.set_option("contract_tf32", 1)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- timed region (device events per step, L2 flushed between steps) ----
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = SincProject.launch_count()
    for a, b in evs:
        flush.zero_()
        a.record(stream)
        step()
        b.record(stream)
    torch.cuda.synchronize()
    launches = SincProject.launch_count() - l0
    total_ms = sum(a.elapsed_time(b) for a, b in evs)
    clk = clocks.stop()
    t_local = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(t_local, op=dist.ReduceOp.MAX)
    total_ms = float(t_local.item())
    ms_step = total_ms / args.steps
    res = {"value": world * args.steps / (total_ms / 1e3), "ms_per_step": ms_step, "clocks": clk,
           "gpu_launches": int(launches), "launches_per_step": launches / args.steps,
           "fft_length": proj.fft_length, "numconfig": nc}
    if rank == 0 and not args.profile_precision_form:
        res["outputs"] = {"rhs": out.cpu().numpy().T, "twoematel": mat.cpu().numpy().T.reshape((n,) * 4, order="F"),
                          "phi": phi_h, "avector": a_h}
    if not extras:
        if args.stages:
            proj.set_option("rhs_overlap", 0)
            proj.profile(True)
            for _ in range(3):
                flush.zero_()
                step()
            prof = proj.profile_read()
            proj.profile(False)
            proj.set_option("rhs_overlap", 1)
            res["stage_ms_per_step"] = {k: v[0] / 3 for k, v in prof.items()}
        if args.e2e:
            res["e2e"] = run_e2e(proj, w, phi_h, a_h, args, stream, world, dist)
        proj.close()
        return res

    # ---- secondary rates: orbital-RHS matvec alone, CI sigma alone ----
    res["secondary"] = secondary_rates(proj, torch, stream, flush, phi, den, inv, red, out, mat, avec, n, G)

    # ---- precision form: Coulomb passes in FP32, reducedpot 3xTF32 ----
    res["precision_forms"] = precision_form(proj, torch, stream, flush, step, out, mat, max(3, args.steps), world,
                                            dist, dev)

    # ---- per-kernel times (profiled pass, one stream) for the roofline ----
    # the timed evaluations overlap the CI part, the kinetic contraction and
    # twoematel with the Coulomb passes on a second stream; the per-stage events
    # are taken with that overlap off so that each stage is timed alone
    proj.set_option("rhs_overlap", 0)
    proj.profile(True)
    nprof = max(3, min(20, args.steps))
    for _ in range(nprof):
        flush.zero_()
        step()
    prof = proj.profile_read()
    proj.profile(False)
    proj.set_option("rhs_overlap", 1)
    res["roofline"] = make_roofline(w, prof, nprof, dev, proj.fft_length)
    res["evaluation_roofline"] = eval_roofline(w, prof, nprof, dev, proj.fft_length, ms_step)
    res["stage_ms_per_step"] = {k: v[0] / nprof for k, v in prof.items()}
    res["stage_timing"] = "CUDA events per stage on one stream (rhs_overlap 0); the timed value overlaps them"

    # ---- CMF propagation steps/s on the same workload ----
    if propagation:
        res["propagation"] = cmf_rate(proj, w, phi, avec, torch, local)

    # ---- end to end through the host-array C entry (pinned host buffers) ----
    if e2e and not args.no_e2e:
        res["e2e"] = run_e2e(proj, w, phi_h, a_h, args, stream, world, dist)
    proj.close()
    return res


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_precision_form and not args.no_extras:
        raise SystemExit("--profile-precision-form is a profiling mode: use it with --no-extras")
    rank, world, local = dist_env()
    import torch
    from sincgpu import SincProject  # noqa: F401  (fails loudly without the CUDA library)
    from sincgpu.inputs import WORKLOADS

    torch.cuda.set_device(local)
    if args.only:
        out = {}
        if args.only == "served":
            out["served"] = {f: served_form(local, f == "mixed_fp32_coulomb", args.served_count, args.served_steps,
                                            args.served_full)
                             for f in ("plain_fp64", "mixed_fp32_coulomb")}
            pl, mx = out["served"]["plain_fp64"], out["served"]["mixed_fp32_coulomb"]
            out["served"]["mixed_vs_plain_steps_per_s"] = mx["steps_per_s"] / max(pl["steps_per_s"], 1e-30)
        elif args.only == "propagation":
            out["propagation"] = propagation_only(WORKLOADS[args.config], local, args.steps)
        else:
            out["batched"] = batched_form(torch, local, torch.cuda.current_stream(), args.batched_count)
        if rank == 0:
            print(json.dumps(out), flush=True)
        return 0
    if args.precision_trajectory:
        if rank == 0:
            print(json.dumps(precision_trajectory(WORKLOADS[args.config], args.precision_trajectory, local)),
                  flush=True)
        return 0
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    w = WORKLOADS[args.config]
    head = measure(w, args, rank, world, local, dist, extras=not args.no_extras)
    outputs = head.pop("outputs", None)

    if args.no_extras:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_step"],
                              "higher_is_better": True, "gpu_launches": head["gpu_launches"],
                              "config": workload_config(w), "stage_ms_per_step": head.get("stage_ms_per_step"),
                              "e2e": head.get("e2e"), "note": "profiling run (--no-extras)"}), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    line = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "complex128",
        "data": "synthetic (seeded Gaussian-envelope orbitals, seeded normalised A-vector)",
        "config": workload_config(w), **{k: v for k, v in head.items() if k not in ("value", "ms_per_step")},
    }
    # the 41^3 / 10-orbital workload beside the headline (BASELINE's plain FP64 GPU drop-in)
    sub_outputs = None
    if args.config != "B" and not args.no_workload_b:
        wb = WORKLOADS["B"]
        sub = measure(wb, args, rank, world, local, dist, extras=True, propagation=True)
        sub_outputs = sub.pop("outputs", None)
        line["workload_B"] = {"config": workload_config(wb), **sub}
    if not args.no_batched:
        line["batched"] = batched_form(torch, local, torch.cuda.current_stream(), args.batched_count)
    if not args.no_served:
        line["served"] = {f: served_form(local, f == "mixed_fp32_coulomb", args.served_count, args.served_steps,
                                         args.served_full)
                          for f in ("plain_fp64", "mixed_fp32_coulomb")}
        pl, mx = line["served"]["plain_fp64"], line["served"]["mixed_fp32_coulomb"]
        line["served"]["mixed_vs_plain_steps_per_s"] = mx["steps_per_s"] / max(pl["steps_per_s"], 1e-30)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        t, sample, ref = cpu_reference_eval(w, threads, want_outputs=outputs is not None)
        line["cpu_baseline"] = {"value": 1.0 / t, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample}
        if outputs is not None:
            line["parity"] = parity_report(w, outputs, ref)
        if sub_outputs is not None:
            tb, sample_b, ref_b = cpu_reference_eval(WORKLOADS["B"], threads, want_outputs=True)
            line["workload_B"]["cpu_baseline"] = {"value": 1.0 / tb, "unit": UNIT, "cores": threads, "kind": "port",
                                                  "sample": sample_b}
            line["workload_B"]["parity"] = parity_report(WORKLOADS["B"], sub_outputs, ref_b)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def precision_form(proj, torch, stream, flush, step, out, mat, steps, world, dist, dev):
    """Same step with the Coulomb passes in FP32 (context option coulomb_fp32):
    throughput and the relative errors of the orbital RHS and twoematel against
    the FP64 form's results of the same inputs (the FP64 form is the one pinned
    to the oracle at 1e-11)."""
    step()
    torch.cuda.synchronize()
    out64, mat64 = out.clone(), mat.clone()
    proj.set_option("coulomb_fp32", 1)
    proj.set_option("contract_tf32", 1)
    try:
        for _ in range(3):
            step()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(steps)]
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for a, b in evs:
            flush.zero_()
            a.record(stream)
            step()
            b.record(stream)
        torch.cuda.synchronize()
        total_ms = sum(a.elapsed_time(b) for a, b in evs)
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())

        def rel(x, y):
            return float((x - y).abs().max() / y.abs().max())
        res = {"plain": {"coulomb": "fp64", "rhs_rel_err": 0.0},
               "mixed_fp32_coulomb": {
                   "value": world * steps / (total_ms / 1e3), "unit": UNIT,
                   "ms_per_step": total_ms / steps,
                   "coulomb": "fp32 (complex64 FFT passes; pair products formed in fp64)",
                   "contractions": "reducedpot on the tensor cores (tcgen05 kind::tf32, 3xTF32, fp32 "
                                   "accumulation); twoematel fp64",
                   "rhs_rel_err_vs_fp64": rel(out, out64), "twoematel_rel_err_vs_fp64": rel(mat, mat64)}}
    finally:
        proj.set_option("coulomb_fp32", 0)
        proj.set_option("contract_tf32", 0)
    return res


def precision_trajectory(w, nsteps, local, dt=0.05):
    """The precision form along a trajectory: `nsteps` field-free CMF steps of
    workload `w` from the seeded state, run three ways -- FP64 (the plain form,
    pinned to the oracle), mixed (FP32 Coulomb passes, 3xTF32 reducedpot) and
    mixed with the last mean-field build of each step in FP64 (cmf_fp64_last) --
    with the energy and z dipole of every step; then one orbital-RHS evaluation
    of the FP64 run's final state in each precision.  Errors are against the
    FP64 run."""
    import torch
    from sincgpu import SincProject, WalkTables
    from sincgpu.inputs import seeded_avector, seeded_orbitals
    n, G = w.nspf, w.G
    dev = torch.device("cuda", local)
    phi_h = seeded_orbitals(w.numpoints, w.spacing, n, seed=1)
    variants = {"fp64": {}, "mixed": {"coulomb_fp32": 1, "contract_tf32": 1},
                "mixed_fp64_last": {"coulomb_fp32": 1, "contract_tf32": 1, "cmf_fp64_last": 1}}
    runs, final = {}, None
    for name, opts in variants.items():
        with SincProject(w.numpoints, w.spacing, w.centershift, w.nuccharges, n, device=local) as p:
            wt = WalkTables(w.numelec, n, 0).build_spin()
            p.ci_attach(wt)
            for k, v in opts.items():
                p.set_option(k, v)
            p.cmf_setup(par_timestep=dt)
            p.cmf_pulses([])
            a_h = seeded_avector(wt.numconfig, seed=2)
            e0 = p.cmf_init_dev(torch.from_numpy(np.ascontiguousarray(phi_h.T)).to(dev), torch.from_numpy(a_h).to(dev))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            en, dip = [e0], []
            for k in range(nsteps):
                en.append(p.cmf_step(dt * k, dt * (k + 1))["energy"])
                d, nn = p.cmf_dipole_z()
                dip.append(d.real / nn)
            wall = time.perf_counter() - t0
            runs[name] = {"energy": np.array(en), "dipole": np.array(dip), "ms_per_step": 1e3 * wall / nsteps}
            if name == "fp64":
                ph = torch.empty((n, G), dtype=torch.complex128, device=dev)
                av = torch.empty(wt.numconfig, dtype=torch.complex128, device=dev)
                p.cmf_state_dev(ph, av)
                final = (ph, av)
    # one evaluation of the FP64 run's final state in each precision
    evals = {}
    with SincProject(w.numpoints, w.spacing, w.centershift, w.nuccharges, n, device=local) as p:
        wt = WalkTables(w.numelec, n, 0)
        p.ci_attach(wt)
        cx = dict(dtype=torch.complex128, device=dev)
        bufs = [torch.empty((n, n), **cx), torch.empty((n, n), **cx), torch.empty((n,) * 4, **cx),
                torch.empty((n,) * 4, **cx), torch.empty((n, n, G), **cx), torch.empty((n, G), **cx)]
        for name, opts in (("fp64", {}), ("mixed", {"coulomb_fp32": 1, "contract_tf32": 1})):
            for k in ("coulomb_fp32", "contract_tf32"):
                p.set_option(k, opts.get(k, 0))
            p.orbital_rhs_avec_dev(final[0], final[1], *bufs)
            torch.cuda.synchronize()
            evals[name] = {"twoematel": bufs[3].clone(), "reducedpot": bufs[4].clone(), "rhs": bufs[5].clone()}
    ref, mix = evals["fp64"], evals["mixed"]
    rp_err = ((mix["reducedpot"] - ref["reducedpot"]).abs().amax(dim=2) /
              ref["reducedpot"].abs().amax(dim=2).clamp_min(1e-300)).cpu().numpy()
    rhs_err = ((mix["rhs"] - ref["rhs"]).abs().amax(dim=1) / ref["rhs"].abs().amax(dim=1)).cpu().numpy()
    twoe = float((mix["twoematel"] - ref["twoematel"]).abs().max() / ref["twoematel"].abs().max())
    e_ref, d_ref = runs["fp64"]["energy"], runs["fp64"]["dipole"]
    out = {"workload": workload_config(w, l2="n/a")["workload"], "steps": nsteps, "dt_au": dt,
           "timing": "host wall clock over the steps (each CMF step ends in a device synchronisation)",
           "fp64_ms_per_step": runs["fp64"]["ms_per_step"], "fp64_energy_first_last": [e_ref[0], e_ref[-1]]}
    for name in ("mixed", "mixed_fp64_last"):
        r = runs[name]
        out[name] = {"ms_per_step": r["ms_per_step"],
                     "speedup_vs_fp64": runs["fp64"]["ms_per_step"] / r["ms_per_step"],
                     "energy_dev_max_hartree": float(np.abs(r["energy"] - e_ref).max()),
                     "energy_dev_last_hartree": float(abs(r["energy"][-1] - e_ref[-1])),
                     "dipole_z_dev_max_au": float(np.abs(r["dipole"] - d_ref).max()),
                     "energy_dev_at_steps": {str(k): float(abs(r["energy"][k] - e_ref[k]))
                                             for k in (1, 10, 50, 100, 200) if k <= nsteps}}
    out["evaluation_at_final_state"] = {
        "reduced_potentials_rel_err": {"max": float(rp_err.max()), "median": float(np.median(rp_err)),
                                       "count": int(rp_err.size),
                                       "per_potential": "reducedpot(:, k, i): max |mixed - fp64| / max |fp64|"},
        "rhs_rel_err_per_orbital_max": float(rhs_err.max()), "twoematel_rel_err": twoe}
    return out


def cmf_rate(proj, w, phi, avec, torch, local, nsteps=6):
    """Constant-mean-field steps/s (cmf_prop_wfn, dt = 0.05, field free, spin
    projected) on the bench workload, device-resident state."""
    from sincgpu import WalkTables
    wt = WalkTables(w.numelec, w.nspf, 0).build_spin()
    proj.ci_attach(wt)
    proj.cmf_setup(par_timestep=0.05)
    proj.cmf_pulses([])
    e0 = proj.cmf_init_dev(phi, avec)
    proj.cmf_step(0.0, 0.05)                     # warm-up step (sizes the Krylov workspaces)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = [proj.cmf_step(0.05 * k, 0.05 * (k + 1)) for k in range(1, nsteps + 1)]
    dt = time.perf_counter() - t0
    ms = [r["ms"] for r in res] if "ms" in res[0] else None
    return {"steps_per_s": nsteps / dt, "ms_per_step": 1e3 * dt / nsteps, "steps": nsteps, "dt_au": 0.05,
            "energy0": e0, "energy_last": res[-1]["energy"], "orb_jacobian_products_per_step":
            float(np.mean([r["orb_iters"] for r in res])), "sigma_products_per_step":
            float(np.mean([r["avec_iters"] for r in res])), "per_step_ms": ms,
            "timing": "host wall clock around each step (each step ends in a device synchronisation)"}


def propagation_only(w, local, nsteps):
    """CMF steps of workload `w` alone (rank 0's seeded inputs; `nsteps` timed steps
    after one warm-up step), for profiling the propagation."""
    import torch
    from sincgpu import SincProject
    from sincgpu.inputs import ci_size, seeded_avector, seeded_orbitals
    phi_h = seeded_orbitals(w.numpoints, w.spacing, w.nspf, seed=1)
    a_h = seeded_avector(ci_size(w.numelec, w.nspf), seed=2)
    proj = SincProject(w.numpoints, w.spacing, w.centershift, w.nuccharges, w.nspf, device=local)
    try:
        phi = torch.from_numpy(np.ascontiguousarray(phi_h.T)).cuda(local)
        avec = torch.from_numpy(np.ascontiguousarray(a_h)).cuda(local)
        return cmf_rate(proj, w, phi, avec, torch, local, nsteps=nsteps)
    finally:
        proj.close()


def batched_form(torch, local, stream, count):
    """Batched form: `count` uneven instances (inputs.batched_instances).  Plain
    FP64 evaluated one after another through the direct entry point, against
    the captured graphs of all instances launched as one parent graph, in FP64
    and with the Coulomb passes in FP32 (pair chunks from the autotuner).  Rates
    are instance evaluations per second; errors are the mixed results against
    the plain FP64 ones."""
    from sincgpu import Batch, SincProject, WalkTables
    from sincgpu.inputs import batched_instances, seeded_orbitals
    dev = torch.device("cuda", local)
    cx = dict(dtype=torch.complex128, device=dev)
    inst = batched_instances(count)
    t_setup = time.perf_counter()
    made = []
    for i, s in enumerate(inst):
        n, N = s["nspf"], s["numpoints"]
        G = N ** 3
        p = SincProject(N, s["spacing"], s["centershift"], s["nuccharges"], n, device=local)
        p.set_stream(stream.cuda_stream)
        wt = WalkTables(s["numelec"], n, s["restrictms"])
        p.ci_attach(wt)
        phi = seeded_orbitals(N, s["spacing"], n, seed=100 + i)
        rng = np.random.default_rng(200 + i)
        a = rng.standard_normal(wt.numconfig) + 1j * rng.standard_normal(wt.numconfig)
        a /= np.linalg.norm(a)
        b = dict(phi=torch.from_numpy(np.ascontiguousarray(phi.T)).to(dev), a=torch.from_numpy(a).to(dev),
                 den=torch.empty((n, n), **cx), inv=torch.empty((n, n), **cx), tally=torch.empty((n,) * 4, **cx),
                 mat=torch.empty((n,) * 4, **cx), rp=torch.empty((n, n, G), **cx), out=torch.empty((n, G), **cx))
        made.append((p, wt, b))
    setup_s = time.perf_counter() - t_setup

    def args_of(b):
        return (b["phi"], b["a"], b["den"], b["inv"], b["tally"], b["mat"], b["rp"], b["out"])

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def sequential():
        for p, _, b in made:
            p.orbital_rhs_avec_dev(*args_of(b))

    plain_ms = timed(sequential, 3)
    ref_out = [b["out"].clone() for _, _, b in made]
    ref_mat = [b["mat"].clone() for _, _, b in made]
    for p, _, b in made:
        p.rhs_graph_capture(*args_of(b))
    batch = Batch([m[0] for m in made])
    batched_plain_ms = timed(lambda: batch.launch(stream.cuda_stream), 3)
    batch.close()
    t_tune = time.perf_counter()
    tuned = {}
    for p, _, b in made:
        p.set_option("coulomb_fp32", 1)
        p.set_option("contract_tf32", 1)
        key = (p.N, p.nspf)
        if key in tuned:
            for name, v in tuned[key].items():
                p.set_option(name, v)
        else:
            p.autotune_rhs(*args_of(b))
            tuned[key] = {name: p.get_option(name) for name in ("coul_chunk", "twoe_tile", "coul_tma")}
        p.rhs_graph_capture(*args_of(b))
    tune_s = time.perf_counter() - t_tune
    batch = Batch([m[0] for m in made])
    mixed_ms = timed(lambda: batch.launch(stream.cuda_stream), 3)
    torch.cuda.synchronize()
    rhs_err = max(float((b["out"] - r).abs().max() / r.abs().max()) for (_, _, b), r in zip(made, ref_out))
    de = max(abs(0.5 * complex(((b["mat"] - r) * b["tally"]).sum().item())) for (_, _, b), r in zip(made, ref_mat))
    batch.close()
    for p, _, _ in made:
        p.close()
    return {
        "instances": count, "workload": "inputs.batched_instances: odd 21^3-61^3 grids, spacing 0.25-0.4, 1-2 "
        "nuclei Z=1-3 within +-2 bohr, 2-6 electrons, 4-12 orbitals, full M_s=0 CI (up to 48400 "
        "determinants), seeded",
        "grid_points_total": int(sum(s["numpoints"] ** 3 for s in inst)),
        "plain_fp64_sequential": {"value": count / (plain_ms / 1e3), "unit": "evals/s", "ms_per_round": plain_ms},
        "batched_fp64_graph": {"value": count / (batched_plain_ms / 1e3), "unit": "evals/s",
                               "ms_per_round": batched_plain_ms},
        "batched_mixed_graph": {"value": count / (mixed_ms / 1e3), "unit": "evals/s", "ms_per_round": mixed_ms,
                                "coulomb": "fp32 passes, fp64 pair products",
                                "contractions": "reducedpot 3xTF32 on the tensor cores, twoematel fp64",
                                "rhs_rel_err_max_vs_fp64": rhs_err,
                                "two_electron_energy_dev_max_hartree": de},
        "mixed_batched_vs_plain_sequential": plain_ms / mixed_ms,
        "setup_s": setup_s, "autotune_s": tune_s, "autotuned_shapes": len(tuned),
        "autotuned": {f"{k[0]}^3/{k[1]}": v for k, v in sorted(tuned.items())},
        "timing": "CUDA events on the launching stream, 3 rounds after one warm-up round; each round touches "
                  "several GB (inputs larger than L2)",
    }


SERVED_FULL = dict(nmin=31, nmax=81, omax=16, emax=6, max_configs=20000)


def served_form(local, fp32, count, nsteps, full=False):
    """Served form: requests (inputs.served_requests) submitted at their Poisson
    arrival offsets to the device-resident request loop; per-step latency
    percentiles and steps/s over the run.  `full`: the stated stream's sizes
    (31^3-81^3 grids, 2-6 electrons, 4-16 orbitals, full CI up to 20000
    determinants) instead of the bounded default (21^3-41^3, 2-4, 4-8, 1000).
    One untimed single-step request of the first system runs before the stream
    (its time is reported as `warmup_request_ms`)."""
    from types import SimpleNamespace
    from sincgpu.inputs import ci_size, seeded_orbitals, served_requests
    from sincgpu.serve import Server
    reqs = served_requests(count, **(SERVED_FULL if full else {}))
    states = []
    for i, r in enumerate(reqs):
        phi = seeded_orbitals(r["numpoints"], r["spacing"], r["nspf"], seed=300 + i)
        rng = np.random.default_rng(400 + i)
        nc = ci_size(r["numelec"], r["nspf"])
        a = rng.standard_normal(nc) + 1j * rng.standard_normal(nc)
        states.append((phi, a / np.linalg.norm(a)))
    pulses = [[SimpleNamespace(pulsestart=0.0, phaseshift=0.0, longstep=1.0, pulsetheta=0.0, **r["pulse"])]
              for r in reqs]
    with Server(device=local, max_active=8) as srv:
        # one untimed request first: the process's first request loads the
        # library's kernels and sizes the worker slots' workspaces
        r, (phi, a), pl = reqs[0], states[0], pulses[0]
        tw = time.perf_counter()
        srv.wait(srv.submit(r["numpoints"], r["spacing"], r["centershift"], r["nuccharges"], r["nspf"],
                            r["numelec"], r["restrictms"], phi, a, 1, dt=0.05, pulses=pl, coulomb_fp32=fp32))
        warm_ms = (time.perf_counter() - tw) * 1e3
        t0 = time.perf_counter()
        ids = []
        for r, (phi, a), pl in zip(reqs, states, pulses):
            delay = t0 + r["arrival"] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            ids.append(srv.submit(r["numpoints"], r["spacing"], r["centershift"], r["nuccharges"], r["nspf"],
                                  r["numelec"], r["restrictms"], phi, a, nsteps, dt=0.05, pulses=pl,
                                  coulomb_fp32=fp32))
        res = [srv.wait(i) for i in ids]
        wall = time.perf_counter() - t0
        st = srv.stats()
    # percentiles and rate over the timed requests (the server's own stats also
    # count the warm-up request); the percentile rule is the server's
    steps = np.sort(np.concatenate([r["step_ms"] for r in res]))

    def pct(p):
        return float(steps[min(steps.size - 1, max(0, int(np.ceil(p * steps.size)) - 1))])
    span = max(r["timeline_ms"]["finished"] for r in res) - min(r["timeline_ms"]["admitted"] for r in res)
    later = np.concatenate([r["step_ms"][1:] for r in res if len(r["step_ms"]) > 1])
    setup = np.array([r["timeline_ms"]["ready"] - r["timeline_ms"]["admitted"] for r in res])
    queued = np.array([r["timeline_ms"]["admitted"] - r["timeline_ms"]["submitted"] for r in res])
    return {"requests": count, "steps_per_request": nsteps, "dt_au": 0.05, "arrival_rate_per_s": 20.0,
            "p50_step_ms": pct(0.50), "p99_step_ms": pct(0.99), "steps_per_s": steps.size / (span / 1e3),
            "p99_step_ms_after_first_step": float(np.percentile(later, 99)) if later.size else None,
            "setup_ms_p50": float(np.median(setup)), "setup_ms_max": float(setup.max()),
            "queue_wait_ms_p50": float(np.median(queued)), "warmup_request_ms": warm_ms,
            "peak_concurrent": st["peak_active"], "completed": st["completed"] - 1, "wall_s": wall,
            "mean_request_s": float(np.mean([len(r["step_ms"]) and r["step_ms"].sum() / 1e3 for r in res])),
            "workload": ("inputs.served_requests: odd 31^3-81^3 grids, 2-6 electrons, 4-16 orbitals, <= 20000 "
                         "determinants" if full else "inputs.served_requests: odd 21^3-41^3 grids, 2-4 electrons, "
                         "4-8 orbitals, <= 1000 determinants") + ", one sin^2 pulse each (type 2), seeded; the "
                        "request loop uses 8 worker slots",
            "requests_detail": [[r["numpoints"], r["nspf"], r["numelec"]] for r in reqs],
            "slowest_steps_ms": sorted(([round(float(ms), 2), i, k] for i, q in enumerate(res)
                                        for k, ms in enumerate(q["step_ms"])), reverse=True)[:6],
            "slowest_setups_ms": sorted(([round(float(v), 2), i] for i, v in enumerate(setup)), reverse=True)[:4]}


def secondary_rates(proj, torch, stream, flush, phi, den, inv, red, out, mat, avec, n, G):
    """Krylov-matvec rate (actreduced00 alone on resident mean fields) and CI
    sigma rate (sparseconfigmult on assembled matrices)."""
    res = {}
    mats = torch.empty((3, n, n), dtype=torch.complex128, device=phi.device)
    proj.onebody_matel_dev(phi, mats)
    proj.assemble_sparsemats_dev(mat, mats)
    sig = torch.empty_like(avec)
    for name, fn, reps in (
            ("rhs_matvecs_per_s", lambda: proj.actreduced_dev(phi, phi, den, inv, red, out), 50),
            ("sigma_per_s", lambda: proj.sparseconfigmult_dev(avec, sig), 200)):
        for _ in range(3):
            fn()
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        res[name] = reps / (e0.elapsed_time(e1) / 1e3)
    return res


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) from one
# ncu capture of workload B (41^3 grid, 10 orbitals; one Coulomb launch per pass
# covers all 55 pairs), keyed by (stage, N, nspf).  ncu flushes L2 before each
# captured launch, so these are cold-cache figures.
TRAFFIC = {
    ("coul_fwd_x", 41, 10): 70590000, ("coul_fwd_y", 41, 10): 300490000, ("coul_z", 41, 10): 426130000,
    ("coul_inv_y", 41, 10): 323310000, ("coul_inv_x", 41, 10): 143240000, ("twoe_gemm", 41, 10): 72000000,
    ("rp_gemm", 41, 10): 169050000, ("rhs_redpot", 41, 10): 136340000, ("ke_xy", 41, 10): 12170000,
    ("ke_z", 41, 10): 22090000,
}

# DRAM bytes per pair of a Coulomb z launch on the 81^3 grid (P = 162), from one
# ncu capture of an 8-pair launch (coul_chunk=8; the full 40-pair launches hold
# more than the capture size allows): (360.6 + 226.2) MB / 8 pairs.  The W2 slab
# read and written grows with the pairs (the real spectrum stays in L2), so a
# launch's traffic is this times its pairs.
TRAFFIC_PER_PAIR = {("coul_z", 81, 16): 73350000}

_DGEMM = {}


def _dgemm_tflops(dev):
    """FP64 ceiling of this GPU: cuBLAS DGEMM 8192^3, measured once per run."""
    import torch
    if "v" not in _DGEMM:
        a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
        torch.matmul(a, a)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(5):
            torch.matmul(a, a)
        e1.record()
        torch.cuda.synchronize()
        _DGEMM["v"] = 5 * 2 * 8192 ** 3 / (e0.elapsed_time(e1) / 1e3) / 1e12
        del a
    return _DGEMM["v"]


def measured_peaks():
    """HBM bandwidth (GB/s) of this GPU pool from MEASURED_PEAKS.json when the
    file is present, else the pool's earlier STREAM-copy measurement."""
    try:
        peaks = json.loads((REPO / "MEASURED_PEAKS.json").read_text())
        return float(peaks["hbm_gbs"]), "of measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "of fallback (6.65 TB/s STREAM copy measured earlier on this pool; MEASURED_PEAKS.json absent)"


def coulomb_pass_work(name, N, P, U):
    """Algorithmic bytes and FP64 flops of one Coulomb pass over U pair densities.
    Bytes: each pass reads its input slab and writes its output slab once (16-byte
    complex values; the z pass reads the real kernel spectrum, 8 P^3 bytes, once
    per launch).  Flops: 5 L log2 L per transformed line of length L = P (the
    pruned lines only), the pair products (6 per point) in the x pass and the
    spectrum multiply (2 per value) in the z pass."""
    fl = 5.0 * P * math.log2(P)
    by = {"coul_fwd_x": 16.0 * (2 * N ** 3 + N * N * P) * U,   # phi_a, phi_b in; W1 out
          "coul_fwd_y": 16.0 * (N * N * P + N * P * P) * U,
          "coul_z": 32.0 * N * P * P * U + 8.0 * P ** 3,
          "coul_inv_y": 16.0 * (N * P * P + N * N * P) * U,
          "coul_inv_x": 16.0 * (N * N * P + N ** 3) * U}[name]
    lines = {"coul_fwd_x": N * N, "coul_fwd_y": N * P, "coul_z": 2 * P * P, "coul_inv_y": N * P,
             "coul_inv_x": N * N}[name]
    extra = {"coul_fwd_x": 6.0 * N ** 3, "coul_z": 2.0 * P ** 3}.get(name, 0.0)
    return by, (lines * fl + extra) * U


def make_roofline(w, prof, nprof, dev, proj_fft_length=None):
    """Dominant kernel of the step (largest summed time in the per-stage profile)
    with its algorithmic bytes or flops per launch.  Coulomb passes and the
    element-wise RHS kernels are booked against HBM; the FP64 GEMMs (twoematel,
    reducedpot, the kinetic contraction: FP64 tensor cores, mma.sync f64) against
    a cuBLAS DGEMM measured in this run."""
    if not prof:
        return None
    name, (ms, nl) = max(prof.items(), key=lambda kv: kv[1][0])
    per_launch_ms = ms / nl
    n, G, N = w.nspf, w.G, w.numpoints
    U = n * (n + 1) // 2
    hbm, hbm_src = measured_peaks()
    launches_per_step = nl / nprof
    traffic, src = TRAFFIC.get((name, N, n)), None
    if traffic:
        src = "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, profiles/"
    elif TRAFFIC_PER_PAIR.get((name, N, n)):
        # the average launch: the U pair solves over the launches of one evaluation
        traffic = TRAFFIC_PER_PAIR[(name, N, n)] * U / launches_per_step
        src = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of an 8-pair launch, scaled to the average "
               "launch's pairs, profiles/")
    base = {"kernel": name, "launch_ms": per_launch_ms, "launches_per_step": launches_per_step,
            "traffic": traffic, "traffic_source": src}
    if name in ("rp_gemm", "twoe_gemm", "ke_xy", "ke_z"):
        dgemm = _dgemm_tflops(dev)
        flops = {"rp_gemm": 2.0 * G * 2 * U * n * (n + 1), "twoe_gemm": 2.0 * G * (2 * U) ** 2,
                 "ke_xy": 2 * 2 * 2.0 * N ** 3 * N * n, "ke_z": 2 * 2.0 * N ** 3 * N * n}[name] / launches_per_step
        ach = flops / (per_launch_ms / 1e3) / 1e12
        return {**base, "bound": "tensor", "precision": "fp64 (mma.sync f64)", "achieved": ach, "peak": dgemm,
                "unit": "TFLOP/s", "frac": ach / dgemm,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor cores; "
                               "MEASURED_PEAKS.json holds no FP64 figure)"}
    P = proj_fft_length
    if name.startswith("coul_"):
        by, flops = coulomb_pass_work(name, N, P, U)
        by /= launches_per_step
        flops /= launches_per_step
        ach = by / (per_launch_ms / 1e3) / 1e9
        dgemm = _dgemm_tflops(dev)
        fp64 = flops / (per_launch_ms / 1e3) / 1e12
        return {**base, "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                "peak_source": hbm_src, "algorithmic_bytes_per_launch": by,
                "fp64": {"bound": "fp64", "achieved": fp64, "peak": dgemm, "unit": "TFLOP/s",
                         "frac": fp64 / dgemm, "flops_per_launch": flops,
                         "peak_source": "cuBLAS DGEMM 8192^3 in this run (FFT butterflies run on the FP64 "
                                        "CUDA-core pipe, whose peak equals it on B200)"}}
    if name == "rhs_redpot":
        by = 16.0 * G * (n * n + 3 * n)
    else:
        by = 16.0 * G * n * 2
    ach = by / (per_launch_ms / 1e3) / 1e9
    return {**base, "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
            "peak_source": hbm_src, "algorithmic_bytes_per_launch": by}


def eval_roofline(w, prof, nprof, dev, P, ms_step):
    """Whole-evaluation roofline: per stage the larger of its algorithmic bytes over
    the measured HBM bandwidth and its algorithmic FP64 flops over the in-run DGEMM
    rate; their sum against the measured (overlapped) evaluation time."""
    if not prof:
        return None
    n, G, N = w.nspf, w.G, w.numpoints
    U = n * (n + 1) // 2
    hbm = measured_peaks()[0] * 1e9
    fp64 = _dgemm_tflops(dev) * 1e12
    stages = {
        # name: (algorithmic bytes, algorithmic flops) per evaluation
        **{k: coulomb_pass_work(k, N, P, U) for k in ("coul_fwd_x", "coul_fwd_y", "coul_z", "coul_inv_y",
                                                      "coul_inv_x")},
        "twoe_gemm": (16.0 * G * (n + 2 * U), 2.0 * G * (2 * U) ** 2),
        "rp_gemm": (8.0 * G * 2 * U + 16.0 * G * n * n, 2.0 * G * 2 * U * n * (n + 1)),
        "ke_xy": (16.0 * G * n * 2, 2 * 2 * 2.0 * N ** 3 * N * n),
        "ke_z": (16.0 * G * n * 3, 2 * 2.0 * N ** 3 * N * n),
        "rhs_mix": (16.0 * G * n * 2, 8.0 * G * n * n),
        "rhs_redpot": (16.0 * G * (n * n + 3 * n), 8.0 * G * n * n * 2),
        "rhs_proj": (16.0 * G * n * 5, 8.0 * G * n * n * 2),
    }
    out, total = {}, 0.0
    for name, (by, fp) in stages.items():
        if name not in prof:
            continue
        t_roof = max(by / hbm, fp / fp64) * 1e3
        total += t_roof
        out[name] = {"roof_ms": t_roof, "measured_ms": prof[name][0] / nprof,
                     "bound": "hbm" if by / hbm >= fp / fp64 else "fp64"}
    return {"sum_roofline_ms": total, "measured_ms": ms_step, "frac": total / ms_step,
            "peaks": {"hbm_gbs": hbm / 1e9, "fp64_tflops": fp64 / 1e12},
            "note": "stages timed one at a time on one stream (measured_ms); the evaluation overlaps "
                    "them on two streams; small stages (CI, split-K reduce, W build) not counted",
            "stages": out}


def run_e2e(proj, w, phi_h, a_h, args, stream, world, dist):
    import torch
    from sincgpu.capi import _call, _ptr
    n, G = w.nspf, w.G
    phi_p = torch.from_numpy(np.ascontiguousarray(phi_h.T)).pin_memory()
    a_p = torch.from_numpy(np.ascontiguousarray(a_h)).pin_memory()
    out_p = torch.empty((n, G), dtype=torch.complex128).pin_memory()

    def call():
        _call("sincgpu_orbital_rhs_avec", proj._h, _ptr(phi_p), _ptr(a_p), 0.0, -1.0, 0.0, _ptr(out_p))

    for _ in range(3):
        call()
    steps = max(10, args.steps // 3)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        call()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    h2d = 16 * (G * n + len(a_h))
    d2h = 16 * (G * n)
    return {"value": world * steps / (ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "steps": steps, "ms_per_step": ms / steps,
            "upload_groups": proj.get_option("rhs_upload_groups"),
            "path": "sincgpu_orbital_rhs_avec (host orbitals + A-vector in, host RHS out; pinned) through the C ABI; "
                    "orbitals up in groups under the Coulomb pair loop, RHS down under twoematel"}


if __name__ == "__main__":
    sys.exit(main())
