"""Benchmark: MC trial moves/s and full-energy evaluations/s of the periodic DMK
energy path on one B200 (FP64 path, 1e-8 accuracy setting: 9 digits).

Workload (one GPU): N = 1e5 point charges, uniform in a periodic cube of
side L = 46.4 (density ~1), alternating +1/-1 charges (net neutral), 9-digit
DMK (PSWF tolerance 1e-9), n_per_leaf = 200. One step = one full energy
evaluation from raw positions resident in HBM (tree build, outgoing and
incoming plane waves, window + difference + residual energies) followed by
10^4 sequential Metropolis moves (displacement uniform in [-0.3, 0.3]^3,
beta = 1) with accept-and-update. Inputs are seeded synthetic data; no
dataset is involved.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

With --gpus N > 1 (torchrun) every rank runs an independent replica of the
workload (the method does not shard: replicas only) and the whole-job value
is the sum over ranks of moves over the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MC trial moves/s & full-energy evals/s, mixed vs FP64 GPU at 1e-8 rel err"
WORKLOAD = dict(workload="uniform periodic cube, Metropolis MC + full energy", N=100000, L=46.4, digits=9,
                n_per_leaf=200, moves_per_step=10000, step=0.3, beta=1.0, charges="alternating +1/-1")
WORKLOAD_N1E5 = WORKLOAD


def make_system(seed, n, L):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.0, L, 3 * n)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    return r, q


def make_moves(seed, n, m, step):
    rng = np.random.default_rng(seed + 1000)
    idx = rng.integers(0, n, m)
    disp = rng.uniform(-step, step, (m, 3))
    u = rng.uniform(0.0, 1.0, m)
    return idx, disp, u


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, path):
        self.path = path
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self, device_index=0):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        try:
            rows = [l.strip().split(",") for l in open(self.path) if l.strip()]
        except OSError:
            return out
        rows = [[c.strip() for c in r] for r in rows if len(r) >= 9]
        rows = [r for r in rows if r[0] == str(device_index)] or rows
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        out["sm_mhz"] = float(np.median(sm)) if sm else None
        out["sm_max_mhz"] = max(mx) if mx else None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, nm in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        out["reasons"] = sorted(reasons)
        out["samples"] = len(rows)
        return out


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if ws > 1:
        import torch.distributed as dist
        import datetime
        backend = "nccl"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return rank, ws


def all_max(x, ws):
    """Max over ranks (device timings are reported as the slowest rank's)."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_baseline_sample(W):
    """The oracle port (CPU restatement of the reference algorithm) on a bounded sample."""
    from oracle import oracle as O
    n, L = W["N"], W["L"]
    r, q = make_system(7, n, L)
    ncores = os.cpu_count() or 1
    t0 = time.perf_counter()
    T = O.OracleTree(L, W["n_per_leaf"], W["digits"], r, q, nthreads=ncores)
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    T.form_outgoing_pw()
    T.form_incoming_pw()
    E = T.eval_energy()
    t_energy = time.perf_counter() - t0
    m = 40
    idx, disp, u = make_moves(7, n, m, W["step"])
    T.nthreads = 1
    t0 = time.perf_counter()
    acc = 0
    for c in range(m):
        dE = T.eval_shift_energy(idx[c], *disp[c])
        if u[c] < np.exp(-W["beta"] * dE):
            T.update_shift(idx[c], *disp[c])
            acc += 1
    t_moves = time.perf_counter() - t0
    return dict(moves_per_s=m / t_moves, energy_evals_per_s=1.0 / t_energy, t_build_s=t_build, energy=E,
                cores=ncores, moves=m, accepted=acc)


def run_reference(args, rank, ws):
    if rank != 0:
        return
    W = dict(WORKLOAD)
    vals = []
    ee = []
    for s in range(args.warmup + args.steps):
        res = cpu_baseline_sample(W)
        if s >= args.warmup:
            vals.append(res["moves_per_s"])
            ee.append(res["energy_evals_per_s"])
    v = float(np.mean(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "moves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * W["moves_per_step"] / v,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(W, parallelism="replicas" if ws > 1 else "single"),
        "full_energy_evals_per_s": float(np.mean(ee)),
        "cpu_baseline": {"value": v, "unit": "moves/s", "cores": 1, "kind": "port",
                         "sample": f"{res['moves']} sequential Metropolis moves (1 thread, as the reference's "
                                   f"timing driver) + 1 full energy on {res['cores']} threads, per step"},
        "e2e": {"value": v, "unit": "moves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_b200(args, rank, ws):
    import torch
    import pdmk4mc_b200 as P

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    W = dict(WORKLOAD)
    W["moves_per_step"] = args.moves_per_step
    n, L, M = W["N"], W["L"], W["moves_per_step"]
    params = P.HPDMKParams(n_per_leaf=W["n_per_leaf"], digits=W["digits"], L=L, init=P.DIRECT)
    r, q = make_system(1 + rank, n, L)
    # inputs resident in HBM for the device-timed value
    idx, disp, u = make_moves(1 + rank, n, M * (args.steps + args.warmup), W["step"])
    d_idx = torch.tensor(idx, dtype=torch.int32, device="cuda")
    d_disp = torch.tensor(disp.reshape(-1), dtype=torch.float64, device="cuda")
    d_u = torch.tensor(u, dtype=torch.float64, device="cuda")
    d_dE = torch.zeros(M, dtype=torch.float64, device="cuda")
    d_acc = torch.zeros(M, dtype=torch.int32, device="cuda")
    d_r = torch.tensor(r, dtype=torch.float64, device="cuda")
    d_q = torch.tensor(q, dtype=torch.float64, device="cuda")
    # MC tree (slack for moves); its stream carries every kernel
    tree = P.HPDMKPtTree(params, r, q, leaf_slack=8)
    tree.set_mc_mode(P.MC_GRAPH if args.mc_mode == "graph" else P.MC_PERSISTENT)
    stream = torch.cuda.ExternalStream(tree.stream_ptr())
    tree.form_outgoing_pw()
    tree.form_incoming_pw()
    tree.eval_energy()
    estream = torch.cuda.Stream()

    t_moves = []
    t_energy = []
    work = np.zeros(3)
    launches = 0
    l2_flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    clk_path = os.path.join(ROOT, "gpurun_out", f"clocks_rank{rank}.csv") if os.path.isdir(
        os.path.join(ROOT, "gpurun_out")) else "/tmp/pdmk_clocks.csv"
    with Clocks(clk_path) as clk:
        for s in range(args.warmup + args.steps):
            timed = s >= args.warmup
            if timed and s == args.warmup:
                tree.get_timing(reset=True)
                tree.set_timing(True)
            barrier(ws)
            l2_flush.zero_()
            torch.cuda.synchronize()
            # energy phase: tree build + outgoing + incoming + energy from HBM-resident inputs
            ee0 = torch.cuda.Event(enable_timing=True)
            ee1 = torch.cuda.Event(enable_timing=True)
            ee0.record(estream)
            if timed:
                launches0 = P.launch_count()
            ef = P.HPDMKPtTree(params, None, None, leaf_slack=0, stream=estream.cuda_stream,
                               device_inputs=(d_r.data_ptr(), d_q.data_ptr(), n))
            ef.form_outgoing_pw()
            ef.form_incoming_pw()
            e_dmk = ef.eval_energy()
            ee1.record(estream)
            torch.cuda.synchronize()
            ef.close()
            # move phase, device-resident proposals
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            off = s * M
            ev0.record(stream)
            tree.mc_run_device(M, d_idx[off:].data_ptr(), d_disp[3 * off:].data_ptr(), d_u[off:].data_ptr(),
                               W["beta"], d_dE.data_ptr(), d_acc.data_ptr())
            ev1.record(stream)
            torch.cuda.synchronize()
            barrier(ws)
            if timed:
                launches += P.launch_count() - launches0
                t_moves.append(ev0.elapsed_time(ev1) / 1e3)
                t_energy.append(ee0.elapsed_time(ee1) / 1e3)
                work += tree.update_work()
        timing = tree.get_timing()
        tree.set_timing(False)
    tm = all_max(float(np.sum(t_moves)), ws)
    te = all_max(float(np.sum(t_energy)), ws)
    moves_per_s = ws * M * args.steps / tm
    energy_per_s = ws * args.steps / te
    # roofline of the dominant MC kernel, HBM bound. Persistent mode: k_mc,
    # one launch per step, bytes = dE reads + update read-modify-writes of all
    # timed moves. Graph mode: k_update, bytes over every timed move, duration
    # from the event-bracketed sample of launches inside the timed region.
    hbm, peak_kind = peaks()
    if args.mc_mode == "graph":
        upd_ms, upd_n = timing["update"]
        kernel = "k_update (accept-and-update; bytes averaged over all launches, rejected moves move none)"
        bytes_per_launch = work[1] / (M * args.steps)
    else:
        upd_ms, upd_n = timing["mc"]
        kernel = ("k_mc (persistent Metropolis: dE reads + accept-and-update read-modify-writes, "
                  f"{M} moves per launch)")
        bytes_per_launch = (work[1] + work[2]) / max(upd_n, 1)
    achieved = bytes_per_launch / (upd_ms / upd_n / 1e3) / 1e9 if upd_n else None
    # DRAM traffic of k_mc from one ncu capture of a 256-move launch on this
    # workload (966 MB read + 1 322 MB written), scaled to a launch by moves
    traffic = None if args.mc_mode == "graph" else (966.42e6 + 1321.68e6) / 256 * M

    # end to end through the C-ABI with host buffers (copies inside the timed region)
    e2e_t = []
    h2d = M * (8 + 24 + 8)
    d2h = M * (8 + 4)
    hidx, hdisp, hu = make_moves(99 + rank, n, M * args.steps, W["step"])
    for s in range(args.steps):
        barrier(ws)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tree.mc_run(hidx[s * M:(s + 1) * M], hdisp[s * M:(s + 1) * M], hu[s * M:(s + 1) * M], W["beta"])
        e2e_t.append(time.perf_counter() - t0)
    te2e = all_max(float(np.sum(e2e_t)), ws)
    e2e_val = ws * M * args.steps / te2e

    # accuracy of the timed energy against the stored FP64 Ewald energy of
    # this workload (tests/golden/bench_ewald.json, made by the oracle)
    accuracy = None
    gp = os.path.join(ROOT, "tests", "golden", "bench_ewald.json")
    if rank == 0 and os.path.exists(gp):
        g = json.load(open(gp))
        if g["workload"]["N"] == n and g["workload"]["L"] == L and g["workload"]["seed"] == 1:
            ew = g["ewald"]["energy"]
            accuracy = {"energy_dmk": e_dmk, "energy_ewald_fp64": ew, "rel_err": abs(e_dmk - ew) / abs(ew),
                        "ewald": "oracle FP64 Ewald, s = 5, stored"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        res = cpu_baseline_sample(W)
        cpu = {"value": res["moves_per_s"], "unit": "moves/s", "cores": 1, "kind": "port",
               "sample": f"{res['moves']} sequential Metropolis moves of the oracle port (1 thread, as the "
                         f"reference times moves) on the same workload; its full energy "
                         f"{res['energy_evals_per_s']:.4g} evals/s on {res['cores']} threads",
               "full_energy_evals_per_s": res["energy_evals_per_s"]}
    if rank == 0:
        c = clk.summary(dev)
        line = {
            "metric": METRIC, "value": moves_per_s, "unit": "moves/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * (tm + te) / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(W, parallelism="replicas" if ws > 1 else "single", mc_mode=args.mc_mode,
                           l2="256 MB written before each step; the 0.56 GB of expansions exceed the 126 MB L2"),
            "full_energy_evals_per_s": energy_per_s,
            "accept_rate": work[0] / (M * args.steps),
            "accuracy": accuracy,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of a 256-move k_mc "
                                           "launch, scaled by moves per launch" if traffic else None,
                         "kernel": kernel,
                         "timed_launches": int(upd_n),
                         "peak_source": peak_kind},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": "moves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "clocks": c,
        }
        print(json.dumps(line), flush=True)
    tree.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mc-mode", default="persistent", choices=["persistent", "graph"])
    ap.add_argument("--moves-per-step", type=int, default=WORKLOAD["moves_per_step"],
                    help="smaller values only for profiler runs; the reported workload uses the default")
    args = ap.parse_args()
    rank, ws = dist_init()
    try:
        if args.impl == "reference":
            run_reference(args, rank, ws)
        else:
            run_b200(args, rank, ws)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
