#!/usr/bin/env python
"""NNP energy+force throughput (atoms/s) on B200.

Default workload (per GPU, weak scaling): batched inference -- 4096
periodic structures with 16-512 atoms (uniform), 3 elements with
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

Other workloads (--workload): small (one 64-atom cell), train (energy+force
loss gradient of 256 structures), large (one 131,072-atom FCC cell), stream
(20,000 structures of 8-2048 atoms in batches of 1000, with per-batch
latency percentiles).

--impl reference times the reference's CPU implementation of the path on
this host's cores (the reference's own code compiled in oracle/_ref, else
the FP64 restatement in oracle/), on a bounded sample of the same workload.
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

METRIC = "NNP energy+force atoms/s on 1 B200, plain vs batched+BF16, at stated force error"
UNIT = "atoms/s"

WORKLOADS = {
    "batched": (2, "batched inference: 4096 structures x U{16..512} atoms, 3 elements, 56-32-32-1 tanh, rc 6 A"),
    "small": (1, "one 64-atom single-element cubic cell (8.5 A), 16+16 functions, 32-20-20-1 tanh, rc 6 A"),
    "train": (3, "training step: 256 structures x U{64..256} atoms, 2 elements, 48-32-32-1 tanh, "
                 "energy+force MSE loss gradient (w_f 1, norm LINEAR)"),
    "large": (4, "one 131,072-atom jittered FCC cell (a 4.05 A, 32^3 cells), 2 elements, 80-64-64-1 tanh, rc 6.5 A"),
    "stream": (5, "20,000 structures, log-uniform 8..2048 atoms, 4 elements, 64-48-48-1 tanh, batches of 1000 "
                  "structures"),
}
STREAM_BATCH = 1000


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched", choices=sorted(WORKLOADS))
    ap.add_argument("--structures", type=int, default=4096, help="structures per GPU (batched workload)")
    ap.add_argument("--precision", default="bf16x3", choices=["fp32", "bf16", "bf16x3"],
                    help="network layers: FP32 CUDA cores, or BF16 / split-BF16 tensor cores")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch and tile choices")
    return ap.parse_args()


PRECISION = {"fp32": 0, "bf16": 1, "bf16x3": 2}


# ---------------------------------------------------------------- workloads

def make_batch(name: str, rank: int, n_struct: int = 4096):
    from ace_b200 import synth
    if name == "batched":
        return synth.config2(seed=11 + 1000 * rank, n_struct=n_struct)
    if name == "small":
        return synth.config1(seed=7 + 1000 * rank)
    if name == "train":
        return synth.config3(seed=13 + 1000 * rank)
    if name == "large":
        return synth.config4(seed=17 + 1000 * rank)
    return synth.config5(seed=19 + 1000 * rank)


def conditioning_sample(name: str):
    """Structures whose symmetry-function statistics set each network's input
    bias/scale (nnptefr's PREBIAS MEAN / PRESCALE DEV)."""
    from ace_b200 import synth
    if name == "batched":
        return synth.config2(seed=999, n_struct=16)
    if name == "small":
        return synth.config1()
    if name == "train":
        return synth.config3(seed=998, n_struct=16)
    if name == "large":
        return synth.config4(seed=997, ncell=8)
    return synth.config5(seed=996, n_struct=32)


def build_potential(name: str, path: str, seed: int = 1234):
    """The workload's potential, conditioned on G computed by the GPU path."""
    from ace_b200 import NNP, potential, synth
    pot = synth.potential_config(WORKLOADS[name][0], seed=seed)
    potential.write(path, pot)
    nn = NNP.read(path)
    s = conditioning_sample(name)
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


# DRAM bytes per atom of one launch, from the ncu capture of the 512-structure
# case of the batched workload (dram__bytes_read.sum + dram__bytes_write.sum / atoms)
DRAM_BYTES_PER_ATOM = {"k_force_jit": 146.598144e6 / 134400, "k_symm_jit": 119.099648e6 / 134400}


def traffic_bytes(kernel: str, atoms: int):
    b = DRAM_BYTES_PER_ATOM.get(kernel)
    return None if b is None else round(b * atoms)


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
        lines = open(self.path).read().splitlines() if os.path.exists(self.path) else []
        if not lines:
            # a region shorter than the sampling period: one reading at its end
            try:
                r = subprocess.run(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                    "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=10)
                lines = r.stdout.splitlines()
            except Exception:
                lines = []
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        lines += [x for x in open(self.path).read().splitlines() if x not in lines]
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in lines:
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


def ref_kind():
    """"reference" when the reference's own code is built in oracle/_ref."""
    from oracle import ref
    return "reference" if ref.available() else "port"


def cpu_reference(path: str, batch, n_sample: int, procs: int):
    """Times the reference path (NeighborList::build + compute_symm +
    compute_force per structure, FP64) on n_sample structures with `procs`
    worker processes.  Returns (atoms/s, seconds, atoms, results)."""
    import multiprocessing as mp
    structs = [batch.structure(s) for s in range(min(n_sample, batch.n_struct))]
    procs = max(1, min(procs, len(structs)))
    chunks = [structs[k::procs] for k in range(procs)]
    ctx = mp.get_context("spawn")
    kind = ref_kind()
    with ctx.Pool(procs) as pool:
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


def cpu_sample(name: str, b):
    """Bounded CPU sample of the workload (about 10-30 s of CPU work) and its
    description.  The large cell is replaced by a 4000-atom FCC cell of the
    same density and basis: the reference's neighbour search is O(N^2) per
    structure, its per-atom cost of the rest does not depend on N."""
    from ace_b200 import synth
    if name == "large":
        return synth.config4(seed=17, ncell=10), "a 4000-atom FCC cell (10^3 cells) of the same density and basis"
    if name == "small":
        return b, "the 64-atom cell"
    n = {"batched": 128, "stream": 64}[name]
    s = b.subset(range(min(n, b.n_struct)))
    return s, "first %d structures (%d atoms) of the rank-0 batch" % (s.n_struct, s.n_atoms)


# ---------------------------------------------------------------- timing helpers

def device_views(b, dev):
    import torch
    return (torch.tensor(b.atom_off, device=dev), torch.tensor(b.pos, device=dev),
            torch.tensor(b.type, device=dev), torch.tensor(b.cell.reshape(-1, 9), device=dev))


def pinned(a, dtype):
    import torch
    t_ = torch.empty(a.shape, dtype=dtype, pin_memory=True)
    t_.numpy()[...] = a
    return t_


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
    name = args.workload
    tmp = tempfile.mkdtemp()
    ppath = os.path.join(tmp, "potential.nnp")
    pot = build_potential(name, ppath)
    nn = NNP.read(ppath)
    nn.set_precision(PRECISION[args.precision])
    # launch and tile choices tuned on the first call of this batch (cached on disk)
    nn.set_autotune(not args.no_autotune)
    # a stream of our own: the library can capture and replay its step as a
    # CUDA graph on it (not on the legacy default stream)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    nn.set_stream(stream.cuda_stream)
    b = make_batch(name, rank, args.structures)
    clocks = ClockSampler(local)
    if name == "train":
        line = time_train(args, nn, b, ppath, world, dist, clocks, dev)
    else:
        line, E_chk, F_chk = time_inference(args, name, nn, pot, b, world, dist, clocks, dev, stream)
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            add_cpu_baseline(line, name, nn, b, ppath, E_chk, F_chk)
    if rank == 0:
        print(json.dumps(line), flush=True)
    nn.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def time_inference(args, name, nn, pot, b, world, dist, clocks, dev, stream):
    import torch
    from ace_b200 import NNP
    N, S = b.n_atoms, b.n_struct
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    # calls: the whole batch, or the stream in pieces of STREAM_BATCH structures
    pieces = [(0, S)] if name != "stream" else [(s, min(S, s + STREAM_BATCH)) for s in range(0, S, STREAM_BATCH)]
    subs = [b.subset(range(s0, s1)) for s0, s1 in pieces] if len(pieces) > 1 else [b]
    dviews = [device_views(sb, dev) for sb in subs]
    outs = [(torch.zeros(sb.n_struct, dtype=torch.float64, device=dev),
             torch.zeros(3 * sb.n_atoms, dtype=torch.float64, device=dev)) for sb in subs]

    def run_piece(k):
        off, pos, typ, cell = dviews[k]
        Eo, Fo = outs[k]
        nn.compute_device(off.data_ptr(), pos.data_ptr(), typ.data_ptr(), cell.data_ptr(), subs[k].n_struct,
                          Eo.data_ptr(), Fo.data_ptr())

    for _ in range(args.warmup):
        for k in range(len(subs)):
            run_piece(k)
    torch.cuda.synchronize()
    cl = []
    for k in range(len(subs)):          # neighbour counts of the whole workload
        run_piece(k)
        cl.append(nn.neighbor_counts(subs[k].n_atoms))
    counts = np.concatenate(cl)

    # ---- device-resident timing (stage timers off: the library replays its
    # CUDA graph of the step when the shape repeats)
    starts = [[torch.cuda.Event(enable_timing=True) for _ in subs] for _ in range(args.steps)]
    ends = [[torch.cuda.Event(enable_timing=True) for _ in subs] for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = nn.launch_count()
    clocks.start()
    for i in range(args.steps):
        for k in range(len(subs)):
            flush.zero_()
            starts[i][k].record(stream)
            run_piece(k)
            ends[i][k].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = nn.launch_count() - launches0
    if world > 1:
        dist.barrier()
    per_call = [s.elapsed_time(e) for i in range(args.steps) for s, e in zip(starts[i], ends[i])]
    t = torch.tensor([sum(per_call)], dtype=torch.float64, device=dev)
    atoms = torch.tensor([float(N)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(atoms, op=dist.ReduceOp.SUM)
    t_max = float(t.item())
    all_atoms = float(atoms.item())
    value = all_atoms * args.steps / (t_max / 1e3)
    # ---- the plain FP32 GPU path on the same batch and the same handle: the
    # prebuilt generic kernels (no run-time specialisation), FP32 CUDA-core
    # networks, eager launches (no CUDA graph); device-resident inputs, L2
    # flushed, CUDA events, max over ranks, as for `value`
    plain = time_plain(args, nn, subs, run_piece, flush, stream, world, dist, dev, all_atoms)

    # ---- stage times: a separate pass with the stage timers on (eager launches)
    nn.set_timing(True)
    stage_ms = {k: 0.0 for k in NNP.STAGES}
    stage_steps = min(args.steps, 10)
    for i in range(stage_steps):
        for k in range(len(subs)):
            flush.zero_()
            run_piece(k)
            st = nn.stage_times()
            for key in stage_ms:
                stage_ms[key] += st[key]
    nn.set_timing(False)

    # ---- end to end through the C ABI with pinned host buffers
    hsubs = [(pinned(sb.atom_off, torch.int64), pinned(sb.pos, torch.float64), pinned(sb.type, torch.int32),
              pinned(sb.cell.reshape(-1, 9), torch.float64),
              torch.empty(sb.n_struct, dtype=torch.float64, pin_memory=True),
              torch.empty((sb.n_atoms, 3), dtype=torch.float64, pin_memory=True)) for sb in subs]

    def run_host(k):
        h_off, h_pos, h_typ, h_cell, h_E, h_F = hsubs[k]
        nn.compute_batch(h_off.numpy(), h_pos.numpy(), h_typ.numpy(), h_cell.numpy(), out_e=h_E.numpy(),
                         out_f=h_F.numpy())

    for _ in range(max(1, args.warmup)):
        for k in range(len(subs)):
            run_host(k)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for k in range(len(subs)):
            run_host(k)
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = all_atoms * args.steps / float(te.item())
    h2d = b.atom_off.nbytes + b.pos.nbytes + b.type.nbytes + b.cell.nbytes
    d2h = S * 8 + N * 3 * 8
    E_chk = np.concatenate([o[0].cpu().numpy() for o in outs])
    F_chk = np.concatenate([o[1].cpu().numpy() for o in outs]).reshape(-1, 3)

    # ---- roofline of the dominant kernel (FP32 CUDA cores)
    fl = flops_per_stage(pot, b.type, counts)
    per_step = {k: v / stage_steps for k, v in stage_ms.items()}
    kern = max(("symm", "forces"), key=lambda k: per_step[k])
    sm_mhz = (clk or {}).get("sm_mhz") or 1965.0
    n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
    peak_fp32 = n_sm * 128 * 2 * sm_mhz * 1e6 / 1e12
    achieved = fl[kern] / (per_step[kern] / 1e3) / 1e12
    jit = bool(nn.specialization()[0])
    kname = ("k_symm" if kern == "symm" else "k_force") + ("_jit" if jit else "")
    roofline = {"bound": "fp32", "kernel": kname, "achieved": round(achieved, 3), "peak": round(peak_fp32, 2),
                "unit": "TFLOP/s", "frac": round(achieved / peak_fp32, 4),
                "peak_source": "%d SMs x 128 FP32 FMA/clk x 2 x measured %.0f MHz (no FP32 figure in "
                               "MEASURED_PEAKS.json)" % (n_sm, sm_mhz),
                "traffic": traffic_bytes(kname, N) if name == "batched" else None}
    if roofline["traffic"] is not None:
        roofline["traffic_source"] = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one %s launch on the "
                                      "first 512 structures (134,400 atoms), scaled by atoms" % kname)
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t_max / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32" if args.precision == "fp32" else "fp32 basis + %s networks" % args.precision,
        "data": "synthetic (seeded)",
        "config": {"workload": WORKLOADS[name][1], "structures_per_gpu": S, "atoms_per_gpu": N,
                   "network_precision": args.precision,
                   "pairs_per_atom": round(fl["pairs"] / max(N, 1), 2),
                   "triplets_per_atom": round(fl["triplets"] / max(N, 1), 1),
                   "l2": "flushed before every timed call (256 MB write, not timed)",
                   "parallelism": "dp%d" % world},
        "plain": dict(plain, ratio=round(value / plain["value"], 3)),
        "stage_ms": {k: round(v, 4) for k, v in per_step.items()},
        "roofline": roofline,
        "e2e": {"value": round(e2e_value, 1), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "clocks": clk,
        "tuning": tuning_summary(nn),
    }
    if name == "stream":
        line["batch_latency_ms"] = {"p50": round(float(np.percentile(per_call, 50)), 4),
                                    "p99": round(float(np.percentile(per_call, 99)), 4),
                                    "batches_per_step": len(subs), "structures_per_batch": STREAM_BATCH}
    return line, E_chk, F_chk


def tuning_summary(nn):
    """The kernels' launch and tile choices and where they came from."""
    choices, source, log = nn.tune_params()
    return {"choices": choices, "source": source, "log": log}


def time_plain(args, nn, subs, run_piece, flush, stream, world, dist, dev, all_atoms):
    """The plain FP32 GPU path: generic kernels, FP32 networks, no graph.
    The handle's settings are restored afterwards."""
    import torch
    jit = bool(nn.specialization()[0])
    prec = nn.precision
    nn.set_specialization(False)
    nn.set_precision(0)
    nn.set_graphs(False)
    for _ in range(args.warmup):
        for k in range(len(subs)):
            run_piece(k)
    steps = max(1, min(args.steps, 10))
    ev = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in subs]
          for _ in range(steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    for i in range(steps):
        for k in range(len(subs)):
            flush.zero_()
            ev[i][k][0].record(stream)
            run_piece(k)
            ev[i][k][1].record(stream)
    torch.cuda.synchronize()
    t = torch.tensor([sum(a.elapsed_time(b_) for row in ev for a, b_ in row)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    nn.set_specialization(jit)
    nn.set_precision(prec)
    nn.set_graphs(True)
    ms = float(t.item()) / steps
    return {"value": round(all_atoms / (ms / 1e3), 1), "ms_per_step": round(ms, 4), "steps": steps,
            "definition": "same batch and handle: prebuilt generic kernels, FP32 CUDA-core networks, eager "
                          "launches (no CUDA graph)"}


def add_cpu_baseline(line, name, nn, b, ppath, E_chk, F_chk):
    """CPU baseline (rank 0, one GPU) and the error against the reference."""
    procs = os.cpu_count() or 1
    sample, desc = cpu_sample(name, b)
    if name == "large":
        Es, Fs = nn.compute_batch(sample.atom_off, sample.pos, sample.type, sample.cell)
        Fs = Fs.reshape(-1, 3)
    else:
        Es, Fs = E_chk[:sample.n_struct], F_chk[:sample.n_atoms]
    v1, dt, at, res = cpu_reference(ppath, sample, sample.n_struct, procs)
    err_e, err_f = 0.0, 0.0
    for s_ in range(sample.n_struct):
        e_ref, f_ref = res[s_]
        a0, a1 = int(sample.atom_off[s_]), int(sample.atom_off[s_ + 1])
        err_e = max(err_e, abs(Es[s_] - e_ref) / (a1 - a0))
        err_f = max(err_f, float(np.abs(Fs[a0:a1] - f_ref).max()))
    line["cpu_baseline"] = {"value": round(v1, 1), "unit": UNIT, "cores": min(procs, sample.n_struct),
                            "kind": ref_kind(), "sample": "%s, %.1f s wall" % (desc, dt)}
    # the bound this precision is held to: the FP32 path's parity tolerances,
    # or 1 meV/atom and 10 meV/A for the tensor-core networks
    fp32 = line["config"]["network_precision"] == "fp32"
    e_tol, f_tol = (2e-6, 1e-4) if fp32 else (1e-3, 1e-2)
    ok = err_e <= e_tol and err_f <= f_tol
    line["error_vs_fp64"] = {"energy_eV_per_atom_max": err_e, "force_eV_per_A_max": err_f, "sample": desc,
                             "against": ref_kind(), "bound": {"energy_eV_per_atom": e_tol, "force_eV_per_A": f_tol},
                             "within_bound": ok}
    if not ok:
        print("bench.py: results differ from the reference beyond the bound (energy %.3g eV/atom, force %.3g eV/A)"
              % (err_e, err_f), file=sys.stderr)


def time_train(args, nn, b, ppath, world, dist, clocks, dev):
    """Training step of configuration 3: the energy+force loss gradient of the
    batch (nnp_train_grad) and the optimiser step on it (nnp_opt_step, ADAM),
    labels from a teacher potential plus noise (1 meV/atom, 20 meV/A).

    value: every array resident on the device, CUDA events around each step,
           L2 flushed between steps.
    e2e:   the same step through host buffers (batch and labels copied in,
           loss and gradient copied out), wall clock.
    plain: the device-resident step with the prebuilt generic kernels."""
    import torch
    from ace_b200 import NNP
    tpath = os.path.join(os.path.dirname(ppath), "teacher.nnp")
    build_potential("train", tpath, seed=4321)
    teacher = NNP.read(tpath)
    Et, Ft = teacher.compute_batch(b.atom_off, b.pos, b.type, b.cell)
    teacher.close()
    rng = np.random.default_rng(5)
    nat = np.diff(b.atom_off)
    e_ref = Et + rng.normal(0, 1e-3, size=b.n_struct) * nat
    f_ref = Ft + rng.normal(0, 0.02, size=Ft.shape)
    w_f = 1.0
    gamma = 1e-4
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    off, pos, typ, cell = device_views(b, dev)
    er = torch.tensor(e_ref, device=dev)
    fr = torch.tensor(f_ref.reshape(-1), device=dev)
    loss = torch.zeros(1, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def dev_step(t):
        nn.train_grad_device(off.data_ptr(), pos.data_ptr(), typ.data_ptr(), cell.data_ptr(), b.n_struct,
                             er.data_ptr(), fr.data_ptr(), w_f, loss.data_ptr(), 0, norm_mode=1)
        nn.opt_step(gamma, t)

    def timed(steps):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for t in range(steps):
            flush.zero_()
            ev[t][0].record(stream)
            dev_step(t + 1)
            ev[t][1].record(stream)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(c) for a, c in ev)

    for t in range(args.warmup):
        dev_step(t + 1)
    torch.cuda.synchronize()
    launches0 = nn.launch_count()
    if world > 1:
        dist.barrier()
    clocks.start()
    ms = timed(args.steps)
    clk = clocks.stop()
    launches = nn.launch_count() - launches0
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    atoms = torch.tensor([float(b.n_atoms)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(atoms, op=dist.ReduceOp.SUM)
    value = float(atoms.item()) * args.steps / (float(t.item()) / 1e3)
    L = float(loss.item())
    # end to end through host buffers
    for _ in range(max(1, args.warmup)):
        Lh, g, eo, fo = nn.train_grad(b.atom_off, b.pos, b.type, b.cell, e_ref, f_ref, w_f, norm_mode=1)
        nn.opt_step(gamma, 1)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        Lh, g, eo, fo = nn.train_grad(b.atom_off, b.pos, b.type, b.cell, e_ref, f_ref, w_f, norm_mode=1)
        nn.opt_step(gamma, k + 1)
    te = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e = float(atoms.item()) * args.steps / float(te.item())
    # the plain FP32 GPU path: the same device-resident step, prebuilt generic kernels
    nn.set_specialization(False)
    for t_ in range(args.warmup):
        dev_step(t_ + 1)
    torch.cuda.synchronize()
    psteps = max(1, min(args.steps, 10))
    tp = torch.tensor([timed(psteps)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tp, op=dist.ReduceOp.MAX)
    nn.set_specialization(True)
    plain_ms = float(tp.item()) / psteps
    plain_value = float(atoms.item()) / (plain_ms / 1e3)
    line = {"metric": METRIC + " (training step)", "value": round(value, 1), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(float(t.item()) / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic (seeded teacher labels + noise)",
            "config": {"workload": WORKLOADS["train"][1], "structures_per_gpu": b.n_struct,
                       "atoms_per_gpu": b.n_atoms, "parallelism": "dp%d" % world,
                       "step": "nnp_train_grad (energy+force loss gradient, w_f 1, norm LINEAR) + nnp_opt_step (ADAM)",
                       "l2": "flushed before every timed step (256 MB write, not timed)"},
            "loss": L,
            "plain": {"value": round(plain_value, 1), "ms_per_step": round(plain_ms, 4), "steps": psteps,
                      "definition": "the same device-resident step with the prebuilt generic kernels",
                      "ratio": round(value / plain_value, 3)},
            "e2e": {"value": round(e2e, 1), "unit": UNIT,
                    "h2d_bytes_per_step": int(b.atom_off.nbytes + b.pos.nbytes + b.type.nbytes + b.cell.nbytes
                                              + e_ref.nbytes + f_ref.nbytes),
                    "d2h_bytes_per_step": int(8 + 8 * b.n_struct + 24 * b.n_atoms + 8 * len(g))},
            "gpu_launches": int(launches), "clocks": clk}
    if not args.no_cpu_baseline and world == 1:
        import multiprocessing as mp
        n = 16
        sub = b.subset(range(n))
        procs = max(1, min(os.cpu_count() or 1, n))
        parts = [list(range(k, n, procs)) for k in range(procs)]
        ctx = mp.get_context("spawn")
        with ctx.Pool(procs) as pool:
            pool.map(_train_worker, [(ppath, sub, e_ref[:n], f_ref[:sub.n_atoms], [0])] * procs)
            t0 = time.perf_counter()
            pool.map(_train_worker, [(ppath, sub, e_ref[:n], f_ref[:sub.n_atoms], p) for p in parts])
            dtc = time.perf_counter() - t0
        line["cpu_baseline"] = {
            "value": round(sub.n_atoms / dtc, 1), "unit": UNIT, "cores": procs, "kind": "port",
            "sample": ("FP64 restatement of the same energy+force loss gradient (orc_ef_loss_grad; the reference "
                       "has no force-loss gradient), first %d structures (%d atoms), %.1f s wall"
                       % (n, sub.n_atoms, dtc))}
    return line


def _train_worker(args):
    path, sub, e_ref, f_ref, idx = args
    sys.path.insert(0, ROOT)
    from oracle import oracle as orc
    op = orc.OraclePot.from_file(path)
    for s in idx:
        one = sub.subset([s])
        a0, a1 = int(sub.atom_off[s]), int(sub.atom_off[s + 1])
        orc.ef_loss_grad(op, one, e_ref[s:s + 1], f_ref[a0:a1], 1.0, norm_mode=1)
    return True


def run_reference(args, world):
    """CPU reference arm: each step evaluates a bounded sample of the workload."""
    from ace_b200 import potential, synth
    name = args.workload
    tmp = tempfile.mkdtemp()
    ppath = os.path.join(tmp, "potential.nnp")
    pot = synth.potential_config(WORKLOADS[name][0])
    potential.write(ppath, pot)
    b = make_batch(name, 0, args.structures)
    if name == "large":
        b = synth.config4(seed=17, ncell=10)
    procs = os.cpu_count() or 1
    per_step = {"batched": 64, "small": 1, "train": 16, "large": 1, "stream": 32}[name]
    times, atoms = [], 0
    for k in range(args.warmup + args.steps):
        s0 = (k * per_step) % b.n_struct
        sub = b.subset(range(s0, min(b.n_struct, s0 + per_step)))
        v, dt, at, _ = cpu_reference(ppath, sub, sub.n_struct, procs)
        if k >= args.warmup:
            times.append(dt)
            atoms += at
    value = atoms / sum(times)
    desc = ("%d structures per step" % per_step) if name != "large" else "a 4000-atom FCC cell per step"
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * sum(times) / len(times), 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": WORKLOADS[name][1], "sample_per_step": desc,
                       "parallelism": "%d host processes" % procs},
            "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": procs, "kind": ref_kind(),
                             "sample": desc},
            "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    sys.exit(main())
