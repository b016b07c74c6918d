#!/usr/bin/env python
"""NNP energy+force throughput (atoms/s) on B200.

Workload (per GPU, weak scaling): the batched-inference configuration --
4096 periodic structures with 16-512 atoms (uniform), 3 elements with
Dirichlet(1,1,1) fractions, triclinic cells at 0.05 atoms/A^3 with +-10%
shear, cutoff 6 A, per element 24 radial + 32 angular symmetry functions
and a 56-32-32-1 tanh network.  Synthetic, seeded (no public dataset exists).

One step = one full energy+force evaluation of the batch: neighbour list,
symmetry functions, networks, forces, per-structure energies.

  value : device-resident inputs, CUDA-event time of the step (L2 flushed
          between steps, flush not timed), max over ranks.
  e2e   : the same step through the C ABI with pinned host buffers, the
          host->device copy of the inputs and the device->host copy of the
          energies and forces inside the timed region (wall clock).

--impl reference times the reference's CPU implementation of the path on
this host's cores (the reference's own code compiled in oracle/_ref, else
the FP64 restatement in oracle/), on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "NNP energy+force atoms/s on 1 B200, plain vs batched+BF16, at stated force error"
UNIT = "atoms/s"
WORKLOAD = "batched inference: 4096 structures x U{16..512} atoms, 3 elements, 56-32-32-1 tanh, rc 6 A"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--structures", type=int, default=4096)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


# ---------------------------------------------------------------- workload

def workload(rank: int, n_struct: int):
    from ace_b200 import synth
    return synth.config2(seed=11 + 1000 * rank, n_struct=n_struct)


def conditioning_sample():
    from ace_b200 import synth
    return synth.config2(seed=999, n_struct=16)


def build_potential(path: str):
    """Config-2 potential; input bias/scale from G statistics of a 16-structure
    sample computed by the GPU path (nnptefr's PREBIAS MEAN / PRESCALE DEV)."""
    from ace_b200 import NNP, potential, synth
    pot = synth.potential_config(2)
    potential.write(path, pot)
    nn = NNP.read(path)
    s = conditioning_sample()
    _, _, G = nn.compute_batch(s.atom_off, s.pos, s.type, s.cell, symm=True)
    nn.close()
    synth.condition(pot, G, s.type)
    potential.write(path, pot)
    return pot


def flops_per_stage(pot, types: np.ndarray, counts: np.ndarray):
    """Algorithmic FLOPs (FMA = 2) of the symmetry-function and force kernels
    and the networks, from the per-atom neighbour counts by type: the per-atom
    count P(20 + 20 nR) + T(57 + 24 nA) + 4 sum n_{l-1} n_l, split as
    symm P(10 + 8 nR) + T(25 + 10 nA), force P(10 + 12 nR) + T(32 + 14 nA)."""
    from ace_b200.potential import tt_index
    Tn = pot.ntypes
    f_symm = f_force = f_nn = 0.0
    pairs = trip = 0.0
    for II in range(Tn):
        sel = types == II
        c = counts[sel].astype(np.float64)          # [n_II, T]
        if len(c) == 0:
            continue
        for J in range(Tn):
            nR = pot.basis_r[II][J].size
            P = c[:, J].sum()
            pairs += P
            f_symm += P * (10 + 8 * nR)
            f_force += P * (10 + 12 * nR)
        for J in range(Tn):
            for K in range(J, Tn):
                nA = pot.basis_a[II][tt_index(J, K)].size
                t = (c[:, J] * (c[:, J] - 1) / 2).sum() if J == K else (c[:, J] * c[:, K]).sum()
                trip += t
                f_symm += t * (25 + 10 * nA)
                f_force += t * (32 + 14 * nA)
        nodes = pot.nets[II].nodes
        f_nn += len(c) * 4 * sum(nodes[l] * nodes[l + 1] for l in range(len(nodes) - 1))
    return {"symm": f_symm, "forces": f_force, "networks": f_nn, "pairs": pairs, "triplets": trip}


# ---------------------------------------------------------------- clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None
        self.gpu = gpu_index

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for k, n in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        load = [x for x in sm if x > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- CPU reference

def _ref_worker(args):
    """NeighborList::build + compute_symm + compute_force per structure: the
    reference's own code (oracle/_ref) when built, else the FP64 port."""
    path, chunk, kind = args
    sys.path.insert(0, ROOT)
    out = []
    if kind == "reference":
        from oracle import ref
        rp = ref.RefNNP(path)
        for (p, t, c) in chunk:
            e, f, _, _ = rp.compute(p, t, c)
            out.append((e, f))
        rp.close()
        return out
    from oracle import oracle as orc
    op = orc.OraclePot.from_file(path)
    for (p, t, c) in chunk:
        e, f, _ = orc.compute(op, p, t, c)
        out.append((e, f))
    return out


def cpu_reference(path: str, batch, n_sample: int, procs: int):
    """Times the reference path (NeighborList::build + compute_symm +
    compute_force per structure, FP64) on n_sample structures with `procs`
    worker processes.  Returns (atoms/s, seconds, atoms, results)."""
    import multiprocessing as mp
    structs = [batch.structure(s) for s in range(min(n_sample, batch.n_struct))]
    chunks = [structs[k::procs] for k in range(procs)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        kind = ref_kind()
        pool.map(_ref_worker, [(path, [structs[0]], kind)] * procs)       # import / warm-up
        t0 = time.perf_counter()
        res = pool.map(_ref_worker, [(path, ch, kind) for ch in chunks])
        dt = time.perf_counter() - t0
    ordered = [None] * len(structs)
    for k in range(procs):
        for q, r in enumerate(res[k]):
            ordered[k + q * procs] = r
    atoms = sum(len(s[0]) for s in structs)
    return atoms / dt, dt, atoms, ordered


# DRAM bytes per atom of one launch, from the ncu capture of the 512-structure
# case of this workload (dram__bytes_read.sum + dram__bytes_write.sum / atoms)
DRAM_BYTES_PER_ATOM = {"k_force_jit": 145.647616e6 / 134400, "k_symm_jit": 118.50496e6 / 134400}


def traffic_bytes(kernel: str, atoms: int):
    b = DRAM_BYTES_PER_ATOM.get(kernel)
    return None if b is None else round(b * atoms)


def ref_kind():
    """"reference" when the reference's own code is built in oracle/_ref."""
    from oracle import ref
    return "reference" if ref.available() else "port"


# ---------------------------------------------------------------- main

def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        run_reference(args, world)
        return 0

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    from ace_b200 import NNP
    tmp = tempfile.mkdtemp()
    ppath = os.path.join(tmp, "config2.nnp")
    pot = build_potential(ppath)
    nn = NNP.read(ppath)
    stream = torch.cuda.current_stream(dev)
    nn.set_stream(stream.cuda_stream)

    b = workload(rank, args.structures)
    N, S = b.n_atoms, b.n_struct
    off = torch.tensor(b.atom_off, device=dev)
    pos = torch.tensor(b.pos, device=dev)
    typ = torch.tensor(b.type, device=dev)
    cell = torch.tensor(b.cell.reshape(-1, 9), device=dev)
    E = torch.zeros(S, dtype=torch.float64, device=dev)
    F = torch.zeros(3 * N, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        nn.compute_device(off.data_ptr(), pos.data_ptr(), typ.data_ptr(), cell.data_ptr(), S, E.data_ptr(),
                          F.data_ptr())

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    counts = nn.neighbor_counts(N)
    fl = flops_per_stage(pot, b.type, counts)

    # ---- device-resident timing
    nn.set_timing(True)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stage_ms = {k: 0.0 for k in NNP.STAGES}
    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = nn.launch_count()
    clocks.start()
    for k in range(args.steps):
        flush.zero_()
        starts[k].record(stream)
        step()
        ends[k].record(stream)
        st = nn.stage_times()
        for key in stage_ms:
            stage_ms[key] += st[key]
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = nn.launch_count() - launches0
    if world > 1:
        dist.barrier()
    total_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    atoms = torch.tensor([float(N)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(atoms, op=dist.ReduceOp.SUM)
    t_max = float(t.item())
    all_atoms = float(atoms.item())
    value = all_atoms * args.steps / (t_max / 1e3)
    nn.set_timing(False)

    # ---- end to end through the C ABI with pinned host buffers
    def pinned(a, dtype):
        t_ = torch.empty(a.shape, dtype=dtype, pin_memory=True)
        t_.numpy()[...] = a
        return t_
    h_off = pinned(b.atom_off, torch.int64)
    h_pos = pinned(b.pos, torch.float64)
    h_typ = pinned(b.type, torch.int32)
    h_cell = pinned(b.cell.reshape(-1, 9), torch.float64)
    h_E = torch.empty(S, dtype=torch.float64, pin_memory=True)
    h_F = torch.empty((N, 3), dtype=torch.float64, pin_memory=True)
    for _ in range(max(1, args.warmup)):
        nn.compute_batch(h_off.numpy(), h_pos.numpy(), h_typ.numpy(), h_cell.numpy(), out_e=h_E.numpy(),
                         out_f=h_F.numpy())
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        nn.compute_batch(h_off.numpy(), h_pos.numpy(), h_typ.numpy(), h_cell.numpy(), out_e=h_E.numpy(),
                         out_f=h_F.numpy())
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = all_atoms * args.steps / float(te.item())
    h2d = b.atom_off.nbytes + b.pos.nbytes + b.type.nbytes + b.cell.nbytes
    d2h = S * 8 + N * 3 * 8

    # ---- roofline of the dominant kernel (FP32 CUDA cores)
    per_step = {k: v / args.steps for k, v in stage_ms.items()}
    kern = max(("symm", "forces"), key=lambda k: per_step[k])
    flo = fl[kern]
    sm_mhz = (clk or {}).get("sm_mhz") or 1965.0
    n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
    peak_fp32 = n_sm * 128 * 2 * sm_mhz * 1e6 / 1e12
    achieved = flo / (per_step[kern] / 1e3) / 1e12
    jit = bool(nn.specialization()[0])
    kname = ("k_symm" if kern == "symm" else "k_force") + ("_jit" if jit else "")
    roofline = {"bound": "fp32", "kernel": kname,
                "achieved": round(achieved, 3), "peak": round(peak_fp32, 2), "unit": "TFLOP/s",
                "frac": round(achieved / peak_fp32, 4),
                "peak_source": "%d SMs x 128 FP32 FMA/clk x 2 x measured %.0f MHz (no FP32 figure in MEASURED_PEAKS.json)"
                               % (n_sm, sm_mhz),
                "traffic": traffic_bytes(kname, N)}
    if roofline["traffic"] is not None:
        roofline["traffic_source"] = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one %s launch on the "
                                      "first 512 structures (134,400 atoms), scaled by atoms" % kname)

    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t_max / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "structures_per_gpu": S, "atoms_per_gpu": N,
                   "pairs_per_atom": round(fl["pairs"] / N, 2), "triplets_per_atom": round(fl["triplets"] / N, 1),
                   "l2": "flushed between timed steps (256 MB write, not timed)", "parallelism": "dp%d" % world},
        "stage_ms": {k: round(v, 4) for k, v in per_step.items()},
        "roofline": roofline,
        "e2e": {"value": round(e2e_value, 1), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "clocks": clk,
    }

    # ---- CPU baseline (rank 0, one GPU only) and error against the FP64 oracle
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        procs = os.cpu_count() or 1
        sample = b.subset(range(128))
        v1, dt, at, res = cpu_reference(ppath, sample, 128, procs)
        err_e, err_f = 0.0, 0.0
        Eh = E.cpu().numpy()
        Fh = F.cpu().numpy().reshape(-1, 3)
        for s_ in range(sample.n_struct):
            e_ref, f_ref = res[s_]
            a0, a1 = int(b.atom_off[s_]), int(b.atom_off[s_ + 1])
            err_e = max(err_e, abs(Eh[s_] - e_ref) / (a1 - a0))
            err_f = max(err_f, float(np.abs(Fh[a0:a1] - f_ref).max()))
        line["cpu_baseline"] = {"value": round(v1, 1), "unit": UNIT, "cores": procs, "kind": ref_kind(),
                                "sample": "first 128 structures (%d atoms) of the rank-0 batch, %.1f s wall" % (at, dt)}
        line["error_vs_fp64"] = {"energy_eV_per_atom_max": err_e, "force_eV_per_A_max": err_f,
                                 "sample": "same 128 structures"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    nn.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_reference(args, world):
    """CPU reference arm: each step evaluates a bounded sample of the workload."""
    from ace_b200 import potential, synth
    tmp = tempfile.mkdtemp()
    ppath = os.path.join(tmp, "config2.nnp")
    pot = synth.potential_config(2)
    potential.write(ppath, pot)
    b = workload(0, args.structures)
    procs = os.cpu_count() or 1
    sample_structs = 64
    times, atoms = [], 0
    for k in range(args.warmup + args.steps):
        sub = b.subset(range((k * sample_structs) % b.n_struct, (k * sample_structs) % b.n_struct + sample_structs))
        v, dt, at, _ = cpu_reference(ppath, sub, sample_structs, procs)
        if k >= args.warmup:
            times.append(dt)
            atoms += at
    value = atoms / sum(times)
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * sum(times) / len(times), 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "sample_per_step": "%d structures" % sample_structs,
                       "parallelism": "%d host processes" % procs},
            "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": procs, "kind": ref_kind(),
                             "sample": "%d structures per step" % sample_structs},
            "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    sys.exit(main())
