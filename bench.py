#!/usr/bin/env python
"""GAP energy + forces throughput (atoms/s) on many uneven small molecules.

Workload (one step = one pass of the hot path over one batch): 10 000
non-periodic random-walk clusters of 3..29 atoms (Z in {1,6,7,8,9}, half H),
SOAP power spectrum with r_c = 5 A, smooth width 0.5 A, n_max = 8,
l_max = 6, sigma = 0.4 A, GTO spline, normalised; sparse GAP with 4000
sparse environments (proportional to the species counts), zeta = 2,
weights ~ N(0, 1). Each step builds the neighbour list, the expansion, the
power spectrum, the GAP energies and the forces of every atom.

  value  device-resident inputs (uploaded once), outputs left on the device;
  e2e    through the C ABI with host buffers: the step's structures are
         copied host->device and the energies and forces device->host
         inside the timed region.

`--impl reference` times the CPU restatement of the reference algorithm (the
oracle; the reference itself cannot be built here) on a bounded sample of
the same workload, with all host threads.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HYPERS = dict(interaction_cutoff=5.0, cutoff_smooth_width=0.5, max_radial=8, max_angular=6,
              gaussian_sigma_type="Constant", gaussian_sigma_constant=0.4,
              optimization=dict(Spline=dict(accuracy=1e-8)))
METRIC = "GAP E+F atoms/s on 1 B200: adjoint+FP32 vs plain FP64 GPU, force err <=1e-4"
WORKLOAD = ("molecule_clusters: 10000 non-periodic clusters of 3-29 atoms, Z in {1,6,7,8,9} (H 0.5), "
            "rc 5.0, n 8, l 6, sigma 0.4, GTO spline, 4000 sparse points, zeta 2")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    p.add_argument("--n-struct", type=int, default=10000)
    p.add_argument("--n-sparse", type=int, default=4000)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--cpu-sample", type=int, default=40, help="clusters in the CPU baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--workload", default="gap", choices=["gap", "training", "md"],
                   help="gap: E+F prediction (the headline); training: sparse-kernel K_NM energy and "
                        "gradient rows for GAP fitting; md: MD steps of the reference's fitted methane "
                        "model (rgpu_md_step)")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def sparse_selection(rb, calc, batch, n_sparse, seed):
    """4000 sparse environments, per species in proportion to its atom count,
    picked at random (seeded) from features of the first 1000 clusters."""
    from librascal_b200 import synthetic
    off = batch["atom_offsets"]
    n_pick = min(1000, len(off) - 1)
    sub = {k: v for k, v in batch.items() if k != "atom_offsets"}
    a1 = off[n_pick]
    sub = dict(atom_offsets=off[:n_pick + 1], positions=batch["positions"][:a1], numbers=batch["numbers"][:a1],
               cells=batch["cells"][:n_pick], pbc=batch["pbc"][:n_pick])
    species = sorted(set(int(z) for z in batch["numbers"]))
    al = calc.transform(rb.AtomsList(rb.StructureSet(sub)))
    keys = calc.get_keys(species)
    X = al.get_features(calc, keys=keys)
    info = al.get_representation_info()
    counts = {s: int(np.sum(batch["numbers"] == s)) for s in species}
    tot = sum(counts.values())
    per = {s: int(round(n_sparse * c / tot)) for s, c in counts.items()}
    per[species[0]] += n_sparse - sum(per.values())
    idx = synthetic.select_sparse_points(X, info[:, 2], per, seed=seed)
    rng = np.random.default_rng(seed + 1)
    alpha = rng.normal(size=len(idx))
    sp = rb.SparsePoints(calc)
    sp.add_dense(info[idx, 2], X[idx], keys)
    return sp, alpha, species, X[idx], info[idx, 2]


def oracle_sample(batch, n_clusters, species, T, sps, alpha, threads=1):
    """Time the CPU restatement (reference algorithm, FP64) on the first
    n_clusters structures; returns (seconds, atoms)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O
    calc = O.Calculator(HYPERS["interaction_cutoff"], HYPERS["cutoff_smooth_width"], HYPERS["max_radial"],
                        HYPERS["max_angular"], HYPERS["gaussian_sigma_constant"], spline=True, accuracy=1e-8)
    off = batch["atom_offsets"]

    def one(i):
        a0, a1 = off[i], off[i + 1]
        b = dict(atom_offsets=np.array([0, a1 - a0]), positions=batch["positions"][a0:a1],
                 numbers=batch["numbers"][a0:a1], cells=batch["cells"][i:i + 1], pbc=batch["pbc"][i:i + 1])
        r = O.Run(calc, b, species, gradients=True)
        r.gap(sps, T, alpha, 2)
        return int(a1 - a0)

    t = time.perf_counter()
    if threads <= 1:
        atoms = sum(one(i) for i in range(n_clusters))
    else:
        with ThreadPoolExecutor(threads) as ex:
            atoms = sum(ex.map(one, range(n_clusters)))
    return time.perf_counter() - t, atoms


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.out = []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.out.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return dict(sm_mhz=float(np.median(sm)), sm_max_mhz=float(max(mx)), reasons=sorted(reasons),
                    samples=len(sm))


def peaks():
    """Dense BF16 TFLOP/s and HBM GB/s. The GEMMs run inside a long, power-capped
    step, so the sustained BF16 figure is the denominator."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        bf = d.get("bf16_tflops_sustained", d.get("bf16_tflops", 1400.0))
        kind = "measured sustained" if "bf16_tflops_sustained" in d else "measured burst"
        return bf, d.get("hbm_gbs", 6650.0), kind
    return 1400.0, 6650.0, "fallback sustained"


# DRAM bytes (read + write) per grouped GEMM launch at the benchmark workload:
# the average of the forward and backward launches of one capture of the
# 2 000-cluster case (32 505 atoms), scaled by atoms to 160 449 atoms
# (profiles/gemm_tc_bf16x3_clusters2000.md).
GEMM_TRAFFIC_PER_LAUNCH = 0.5 * (1.498e9 + 1.766e9) * 160449 / 32505


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from librascal_b200 import synthetic
    # the first clusters of the same seeded batch as the GPU arm; the sparse
    # points come from the oracle features of the first 1 000 of them (enough
    # centres of every species for the 4 000-point model)
    n_pool = 1000
    batch = synthetic.molecule_clusters(n_struct=max(args.cpu_sample * (args.steps + args.warmup), n_pool),
                                        seed=args.seed)
    species = sorted(set(int(z) for z in batch["numbers"]))
    from oracle import oracle as O
    calc = O.Calculator(HYPERS["interaction_cutoff"], HYPERS["cutoff_smooth_width"], HYPERS["max_radial"],
                        HYPERS["max_angular"], HYPERS["gaussian_sigma_constant"], spline=True, accuracy=1e-8)
    off = batch["atom_offsets"]
    k = min(n_pool, len(off) - 1)
    sub = dict(atom_offsets=off[:k + 1], positions=batch["positions"][:off[k]], numbers=batch["numbers"][:off[k]],
               cells=batch["cells"][:k], pbc=batch["pbc"][:k])
    r = O.Run(calc, sub, species)
    X = r.power_spectrum()
    ca, _, _ = r.centers()
    rowsp = sub["numbers"][ca]
    counts = {s: int(np.sum(batch["numbers"] == s)) for s in species}
    tot = sum(counts.values())
    per = {s: int(round(args.n_sparse * c / tot)) for s, c in counts.items()}
    idx = synthetic.select_sparse_points(X, rowsp, per, seed=args.seed)
    T, sps = X[idx], rowsp[idx]
    alpha = np.random.default_rng(args.seed + 1).normal(size=len(idx))
    threads = os.cpu_count() or 1
    rates, secs_timed = [], []
    for step in range(args.warmup + args.steps):
        lo = step * args.cpu_sample
        b = dict(atom_offsets=off[lo:lo + args.cpu_sample + 1] - off[lo],
                 positions=batch["positions"][off[lo]:off[lo + args.cpu_sample]],
                 numbers=batch["numbers"][off[lo]:off[lo + args.cpu_sample]],
                 cells=batch["cells"][lo:lo + args.cpu_sample], pbc=batch["pbc"][lo:lo + args.cpu_sample])
        secs, atoms = oracle_sample(b, args.cpu_sample, species, T, sps, alpha, threads)
        if step >= args.warmup:
            rates.append(atoms / secs)
            secs_timed.append(secs)
    v = float(np.mean(rates))
    line = dict(metric=METRIC, value=v, unit="atoms/s", n_gpus=args.gpus, steps=args.steps, warmup=args.warmup,
                ms_per_step=1e3 * float(np.mean(secs_timed)), higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="f64",
                data="synthetic", impl="reference",
                config=dict(workload=WORKLOAD, sample="%d clusters per step, %d sparse points" %
                            (args.cpu_sample, len(idx))),
                cpu_baseline=dict(value=v, unit="atoms/s", cores=threads, kind="port",
                                  sample="%d clusters (%d sparse points) per step, CPU FP64 restatement, "
                                         "%d threads" % (args.cpu_sample, len(idx), threads)),
                e2e=dict(value=v, unit="atoms/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)
    return 0


TRAINING_METRIC = "GAP training K_NM rows (energy + position gradients) atoms/s on 1 B200, FP64"
FP64_NOMINAL_TFLOPS = 37.0  # no measured FP64 peak on this pool; B200 nominal FP64 (CUDA cores)


def run_training(args):
    """One step = the K_NM energy rows and gradient rows of compute_KNM for a
    batch of clusters against 4 000 sparse points, FP64, through the C ABI."""
    import torch
    import librascal_b200 as rb
    from librascal_b200 import _native as N, synthetic
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    n_struct = min(args.n_struct, 1000)
    batch = synthetic.molecule_clusters(n_struct=n_struct, seed=args.seed + rank)
    n_atoms = int(batch["atom_offsets"][-1])
    calc = rb.SphericalInvariants(**HYPERS)
    sp, alpha, species, T_sel, sps_sel = sparse_selection(rb, calc, batch, args.n_sparse, args.seed)
    kern = rb.Kernel(calc, name="GAP", zeta=2, target_type="Structure", kernel_type="Sparse")
    model = kern._model(sp)
    st = rb.StructureSet(batch)
    lib = rb.lib()
    M = sp.size()
    K_e = np.zeros((n_struct, M))
    K_g = np.zeros((3 * n_atoms, M))

    def step():
        st.invalidate()
        N.check(lib.rgpu_sparse_kernel(model.handle, st.handle, 0, N.ptr(K_e, N.c_dbl_p)))
        N.check(lib.rgpu_sparse_kernel_derivative(model.handle, st.handle, 0, N.ptr(K_g, N.c_dbl_p)))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    l0 = lib.rgpu_kernel_launches(0)
    dev_ms, wall = [], []
    with Clocks(torch.cuda.current_device()) as clk:
        for _ in range(args.steps):
            t = time.perf_counter()
            step()
            wall.append(time.perf_counter() - t)
            dev_ms.append(st.stage_times()[0])
    launches = int(lib.rgpu_kernel_launches(0) - l0)
    # FP64 flops of the gradient block's GEMM: 2 * 3 * pairs_s * D * M_s per species
    nl = st.neighbour_list()
    npc = np.diff(nl["pair_offsets"])
    zc = batch["numbers"][nl["center_atom"]]
    D = T_sel.shape[1]
    msp = {int(z): int(np.sum(np.asarray(sp.species) == z)) for z in set(sp.species)}
    flops = sum(2.0 * 3 * float(npc[zc == z].sum()) * D * m for z, m in msp.items())
    ms = float(np.mean(dev_ms))
    achieved = flops / (ms * 1e-3) / 1e12
    value = n_atoms / (ms * 1e-3)
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        ns = 10
        off = batch["atom_offsets"]
        sub = dict(atom_offsets=off[:ns + 1], positions=batch["positions"][:off[ns]],
                   numbers=batch["numbers"][:off[ns]], cells=batch["cells"][:ns], pbc=batch["pbc"][:ns])
        oc = O.Calculator(HYPERS["interaction_cutoff"], HYPERS["cutoff_smooth_width"], HYPERS["max_radial"],
                          HYPERS["max_angular"], HYPERS["gaussian_sigma_constant"], spline=True, accuracy=1e-8)
        t = time.perf_counter()
        r = O.Run(oc, sub, species, gradients=True)
        r.kernel_nm(sps_sel, T_sel, 2)
        r.kernel_nm_derivative(sps_sel, T_sel, 2)
        secs = time.perf_counter() - t
        cpu = dict(value=float(off[ns]) / secs, unit="atoms/s", cores=1, kind="port",
                   sample="first %d clusters (%d atoms), K_NM energy + gradient rows, CPU FP64 restatement, "
                          "1 thread, %.1f s" % (ns, int(off[ns]), secs))
    line = dict(metric=TRAINING_METRIC, value=value, unit="atoms/s", n_gpus=1, steps=args.steps,
                warmup=args.warmup, ms_per_step=ms, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f64", data="synthetic",
                config=dict(workload="molecule_clusters: first %d of the seeded 3-29 atom clusters, rc 5.0, n 8, "
                                     "l 6, GTO spline, %d sparse points, zeta 2; K_NM energy rows + 3 gradient "
                                     "rows per atom" % (n_struct, M),
                            n_atoms=n_atoms, output_gb=K_g.nbytes / 1e9,
                            l2="inputs larger than L2: dX/dr chunks of up to 24 GB"),
                roofline=dict(bound="fp64", kernel="gathered FP64 tile GEMM of the gradient block (dgemm.cuh), "
                              "with the materialised dX/dr chunks in the same timed stage",
                              achieved=achieved, peak=FP64_NOMINAL_TFLOPS, unit="TFLOP/s",
                              frac=achieved / FP64_NOMINAL_TFLOPS, traffic=None,
                              peak_kind="nominal FP64 (no measured FP64 peak on this pool)",
                              flops_per_step=flops),
                cpu_baseline=cpu,
                e2e=dict(value=n_atoms / float(np.mean(wall)), unit="atoms/s", h2d_bytes_per_step=0,
                         d2h_bytes_per_step=int(K_e.nbytes + K_g.nbytes), ms_per_step=1e3 * float(np.mean(wall))),
                gpu_launches=launches, clocks=clk.summary())
    print(json.dumps(line), flush=True)
    return 0


MD_METRIC = "GAP MD steps/s on 1 B200 (energy, forces, stress per step; FP32 path, recorded step)"


def run_md(args):
    """One step = rgpu_md_step on the 10-atom methane dimer with the
    reference's fitted GAP model (tests/golden/simple_gap_model.json):
    positions in from host memory, energy, forces and stress out to host
    memory, each step replaying the recorded CUDA graph."""
    import torch
    import librascal_b200 as rb
    from librascal_b200 import io
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    golden = os.path.join(ROOT, "tests", "golden")
    krr = io.load_obj(os.path.join(golden, "simple_gap_model.json"))
    frame = io.read_extxyz(os.path.join(golden, "methane_dimer_sample.xyz"), 0)
    cell = frame["cell"]
    pos0 = frame["positions"] + np.diag(cell) / 2.0
    st = rb.StructureSet(rb.frames_to_batch([dict(frame, positions=pos0)]))
    model = krr._gap()
    ext = torch.cuda.ExternalStream(st.stream())
    rng = np.random.default_rng(args.seed)
    steps = [pos0 + 0.01 * rng.normal(size=pos0.shape) for _ in range(args.warmup + args.steps)]
    for p in steps[:args.warmup]:
        model.md_step(st, p, stress=True)
    lib = rb.lib()
    l0 = lib.rgpu_kernel_launches(0)
    with Clocks(torch.cuda.current_device()) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        for p in steps[args.warmup:]:
            model.md_step(st, p, stress=True)
        e1.record(ext)
        e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    recorded, caps, replays, _ = st.md_step_info()
    # kernels replayed from the graph do not pass the library's launch
    # counter: count the graph's kernel nodes per replayed step
    launches = int(lib.rgpu_kernel_launches(0) - l0) + st.md_graph_kernels * min(replays, args.steps)
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        h = krr.get_representation_calculator()._get_init_params()
        oc = O.Calculator(h["interaction_cutoff"], h["cutoff_smooth_width"], h["max_radial"], h["max_angular"],
                          h["gaussian_sigma_constant"], spline=False, normalize=h["normalize"],
                          radial_scaling=h["cutoff_function_parameters"])
        species = krr.X_train.get_species()
        T = krr.X_train.dense(species)
        sps = np.asarray(krr.X_train.species)
        n_cpu = 20
        t = time.perf_counter()
        for p in steps[:n_cpu]:
            b = rb.frames_to_batch([dict(frame, positions=p)])
            O.Run(oc, b, species, gradients=True).gap_stress(sps, T, krr.weights, krr.kernel.zeta)
        secs = time.perf_counter() - t
        cpu = dict(value=n_cpu / secs, unit="steps/s", cores=1, kind="port",
                   sample="%d steps of the same structure, CPU FP64 restatement (direct GTO as the model "
                          "asks), 1 thread, %.2f s" % (n_cpu, secs))
    n_atoms = len(frame["numbers"])
    line = dict(metric=MD_METRIC, value=1e3 / ms, unit="steps/s", n_gpus=1, steps=args.steps,
                warmup=args.warmup, ms_per_step=ms, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f32", data="the reference's methane-dimer structure with 0.01 A random displacements",
                config=dict(workload="methane dimer (10 atoms, periodic 30 A cell), simple_gap_model.json "
                                     "(rc 7.5, n 4, l 2, RadialScaling, 30 sparse points, zeta 2)",
                            recorded_graph=bool(recorded), replays=replays, capacities=caps,
                            l2="inputs far below L2; a latency measurement"),
                roofline=dict(bound="hbm", kernel="latency-bound step (about 40 small launches)",
                              achieved=None, peak=None, unit="GB/s", frac=None, traffic=None,
                              note="a 10-atom step moves a few hundred KB; the measure is latency"),
                cpu_baseline=cpu,
                e2e=dict(value=1e3 / ms, unit="steps/s", h2d_bytes_per_step=int(8 * 3 * n_atoms),
                         d2h_bytes_per_step=int(8 * (1 + 3 * n_atoms + 6))),
                gpu_launches=launches, clocks=clk.summary())
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "training":
        return run_training(args)
    if args.workload == "md":
        return run_md(args)
    import torch
    import librascal_b200 as rb
    from librascal_b200 import sharding, synthetic
    pg = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()

    batch = synthetic.molecule_clusters(n_struct=args.n_struct, seed=args.seed + rank)
    n_atoms = int(batch["atom_offsets"][-1])
    calc = rb.SphericalInvariants(**HYPERS)
    sp, alpha, species, T_sel, sps_sel = sparse_selection(rb, calc, batch, args.n_sparse, args.seed)
    model = rb.GAPModel(calc, sp, alpha, zeta=2)
    st = rb.StructureSet(batch)
    ext = torch.cuda.ExternalStream(st.stream())
    lib = rb.lib()

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return sharding.max_over_ranks(x, device="cuda") if pg is not None else x

    # ---- value: inputs resident, outputs on the device
    def step_resident():
        st.invalidate()
        model.predict(st, args.precision, energies=False, forces=False)

    for _ in range(args.warmup):
        step_resident()
    barrier()
    l0 = lib.rgpu_kernel_launches(0)
    with Clocks(dev) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        for _ in range(args.steps):
            step_resident()
        e1.record(ext)
        e1.synchronize()
    barrier()
    launches = int(lib.rgpu_kernel_launches(0) - l0)
    ms = max_over_ranks(e0.elapsed_time(e1)) / args.steps
    value = n_atoms * world / (ms * 1e-3)

    # ---- stage breakdown (untimed extra passes)
    stages = np.zeros(8)
    for _ in range(3):
        step_resident()
        stages += st.stage_times()
    stages /= 3
    off = batch["atom_offsets"]
    counts = np.array([np.sum(batch["numbers"] == s) for s in species])
    msp = np.array([int(np.sum(np.asarray(sp.species) == s)) for s in species])
    D = len(species) * (len(species) + 1) // 2 * HYPERS["max_radial"] ** 2 * (HYPERS["max_angular"] + 1)
    gemm_flops = 4.0 * float(np.sum(counts * msp)) * D  # forward + backward
    gemm_ms = stages[4] + stages[5]
    bf16_peak, hbm_peak, peak_kind = peaks()
    achieved = gemm_flops / (gemm_ms * 1e-3) / 1e12 if gemm_ms > 0 else None

    # ---- e2e: host buffers through the C ABI
    e2e = None
    if not args.no_e2e:
        E = np.zeros(len(off) - 1)
        F = np.zeros((n_atoms, 3))
        off64 = np.ascontiguousarray(off, np.int64)
        pos = np.ascontiguousarray(batch["positions"], np.float64)
        num = np.ascontiguousarray(batch["numbers"], np.int32)
        cel = np.ascontiguousarray(batch["cells"], np.float64)
        pbc = np.ascontiguousarray(batch["pbc"], np.int32)
        from librascal_b200 import _native as N

        def step_e2e():
            N.check(lib.rgpu_structures_set(st.handle, len(off64) - 1, N.ptr(off64, N.c_i64_p),
                                            N.ptr(pos, N.c_dbl_p), N.ptr(num, N.c_int_p), N.ptr(cel, N.c_dbl_p),
                                            N.ptr(pbc, N.c_int_p), None))
            N.check(lib.rgpu_gap_predict(model.handle, st.handle, N.PRECISION_FP32 if args.precision == "fp32"
                                         else N.PRECISION_FP64, N.ptr(E, N.c_dbl_p), N.ptr(F, N.c_dbl_p)))

        for _ in range(args.warmup):
            step_e2e()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        for _ in range(args.steps):
            step_e2e()
        e1.record(ext)
        e1.synchronize()
        barrier()
        ms_e2e = max_over_ranks(e0.elapsed_time(e1)) / args.steps
        h2d = off64.nbytes + pos.nbytes + num.nbytes + cel.nbytes + pbc.nbytes
        h2d += 4 * (len(off64) - 1) + 8 * len(off64) + 4 * n_atoms  # centre counts, offsets, atom->structure
        d2h = E.nbytes + F.nbytes
        e2e = dict(value=n_atoms * world / (ms_e2e * 1e-3), unit="atoms/s", h2d_bytes_per_step=int(h2d),
                   d2h_bytes_per_step=int(d2h), ms_per_step=ms_e2e)

    # ---- CPU baseline (rank 0, N = 1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        T = sp.dense(species)
        secs, atoms = oracle_sample(batch, args.cpu_sample, species, T, np.asarray(sp.species), alpha, 1)
        cpu = dict(value=atoms / secs, unit="atoms/s", cores=1, kind="port",
                   sample="first %d clusters (%d atoms), E+F, CPU FP64 restatement of the reference algorithm, "
                          "1 thread, %.1f s" % (args.cpu_sample, atoms, secs))

    if rank == 0:
        line = dict(
            metric=METRIC, value=value, unit="atoms/s", n_gpus=world, steps=args.steps, warmup=args.warmup,
            ms_per_step=ms, higher_is_better=True, scaling="weak", vs_baseline=None,
            dtype="f32" if args.precision == "fp32" else "f64", data="synthetic",
            config=dict(workload=WORKLOAD, n_structures=int(len(off) - 1), n_atoms=n_atoms,
                        sparse_points=int(sp.size()), precision=args.precision,
                        parallelism="dp%d (independent structures per rank)" % world,
                        l2="inputs larger than L2: X and dE/dX are %.1f GB each" %
                           (n_atoms * D * 4 / 1e9),
                        stage_ms=dict(zip(["total", "neighbour_list", "expansion", "power_spectrum",
                                           "gemm_fwd", "gemm_bwd", "ps_backward", "pair_adjoint"],
                                          [round(float(x), 4) for x in stages]))),
            roofline=dict(bound="tensor", kernel="tcgen05 BF16x3 GEMMs (forward + backward)",
                          achieved=achieved, peak=bf16_peak, unit="TFLOP/s",
                          frac=(achieved / bf16_peak) if achieved else None,
                          traffic=GEMM_TRAFFIC_PER_LAUNCH if args.n_struct == 10000 else None,
                          peak_kind="%s dense bf16; achieved counts algorithmic 2MNK flops, the "
                                    "3-term split issues 3x that on the tensor pipe" % peak_kind,
                          issued_frac=(3 * achieved / bf16_peak) if achieved else None,
                          flops_per_step=gemm_flops),
            cpu_baseline=cpu, e2e=e2e, gpu_launches=launches, clocks=clk.summary())
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
