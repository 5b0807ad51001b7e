#!/usr/bin/env python
"""GAP energy + forces throughput (atoms/s) on one B200, FP32 adjoint path
against the plain FP64 GPU path, with the force error of the fast path.

Workloads (one step = one pass of the hot path over one batch: neighbour
list, spherical expansion, power spectrum, GAP energies, forces of every
atom):

  gap        (default) 10 000 non-periodic random-walk clusters of 3..29
             atoms (Z in {1,6,7,8,9}, half H); r_c 5 A, smooth width 0.5 A,
             n_max 8, l_max 6, sigma 0.4 A, GTO spline, normalised; 4 000
             sparse environments in proportion to the species counts,
             zeta 2, weights ~ N(0, 1)
  bulk       one periodic cubic box of 100 000 atoms at 0.05 atoms/A^3,
             Z in {14, 8} 1:2; r_c 6, n_max 12, l_max 9, sigma 0.5; 4 000
             sparse points in proportion to the species counts
  triclinic  256 sheared periodic cells of 32..512 atoms at 0.1 atoms/A^3,
             Z in {1,6,7,8}; r_c 5, n_max 8, l_max 6, sigma 0.4; 2 000
             sparse points per species
  training   K_NM energy and gradient rows for GAP fitting (FP64)
  md         MD steps of the reference's fitted methane model

Reported for the gap-like workloads:
  value     FP32 path, device-resident inputs (uploaded once), outputs left
            on the device;
  e2e       the same through the C ABI with host buffers: the step's
            structures are copied host->device and the energies and forces
            device->host inside the timed region;
  plain_fp64_ms_per_step, speedup_vs_plain_fp64
            the plain FP64 GPU path (the reference's algorithm with the
            materialised dX/dr) on the same batch, timed the same way;
  force_err, energy_err
            max|F32 - F64| / max|F64| and max|E32 - E64| / max|E64| over the
            whole batch, and both GPU paths against the CPU oracle on the
            CPU-baseline sample (oracle_errors);
  roofline  the tensor-core GEMMs against the measured sustained BF16 rate;
            stage_roofline gives every per-centre kernel against HBM and the
            measured FP32 FMA rate.

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

METRIC = "GAP E+F atoms/s on 1 B200: adjoint+FP32 vs plain FP64 GPU, force err <=1e-4"
FORCE_ERR_BAR = 1e-4
TARGET_SPEEDUP = 5.0


def _hypers(rc, n, l, sigma):
    return dict(interaction_cutoff=rc, cutoff_smooth_width=0.5, max_radial=n, max_angular=l,
                gaussian_sigma_type="Constant", gaussian_sigma_constant=sigma,
                optimization=dict(Spline=dict(accuracy=1e-8)))


def workload_spec(name, seed, bulk_atoms=100000):
    """Hypers, batch maker, sparse-point rule, the batch the sparse points
    are picked from and the CPU sample of one gap-like workload."""
    from librascal_b200 import synthetic
    if name == "gap":
        return dict(
            name=name, hypers=_hypers(5.0, 8, 6, 0.4), n_sparse=4000, per_species=None,
            desc=("molecule_clusters: 10000 non-periodic clusters of 3-29 atoms, Z in {1,6,7,8,9} (H 0.5), "
                  "rc 5.0, n 8, l 6, sigma 0.4, GTO spline, 4000 sparse points, zeta 2"),
            make=lambda n_struct, s: synthetic.molecule_clusters(n_struct=n_struct, seed=s),
            default_struct=10000, shardable=True,
            # sparse points: picked from the features of the first 1 000 clusters
            selection=lambda batch: _first(batch, 1000),
            # CPU sample: the first clusters of the batch
            sample=lambda batch, k: _first(batch, k), sample_default=40,
            sample_desc="first %d clusters")
    if name == "bulk":
        return dict(
            name=name, hypers=_hypers(6.0, 12, 9, 0.5), n_sparse=4000, per_species=None,
            desc=("bulk_box: one periodic cubic box of 100000 atoms at 0.05 atoms/A^3, Z in {14,8} 1:2, "
                  "min distance 1.2 A, rc 6.0, n 12, l 9, sigma 0.5, GTO spline, 4000 sparse points, zeta 2"),
            make=lambda n_struct, s: synthetic.bulk_box(n_atoms=bulk_atoms, seed=s),
            default_struct=1, shardable=False,
            # a box of 8 000 atoms with the same density and composition
            selection=lambda batch: synthetic.bulk_box(n_atoms=8000, seed=seed + 17),
            # a 300-atom box of the same density and composition (side 18.2 A)
            sample=lambda batch, k: synthetic.bulk_box(n_atoms=300, seed=seed + 23), sample_default=1,
            sample_desc="one 300-atom box of the same density and composition (%d)")
    if name == "triclinic":
        return dict(
            name=name, hypers=_hypers(5.0, 8, 6, 0.4), n_sparse=None, per_species=2000,
            desc=("triclinic_cells: 256 periodic cells with +-10% shear, 32-512 atoms at 0.1 atoms/A^3, "
                  "Z in {1,6,7,8}, rc 5.0, n 8, l 6, sigma 0.4, GTO spline, 2000 sparse points per species, "
                  "zeta 2"),
            make=lambda n_struct, s: synthetic.triclinic_cells(n_struct=n_struct, seed=s),
            default_struct=256, shardable=True,
            selection=lambda batch: _first(batch, 64),
            sample=lambda batch, k: _first(batch, k), sample_default=2,
            sample_desc="first %d cells")
    raise ValueError(name)


def _first(batch, k):
    from librascal_b200 import sharding
    k = min(k, len(batch["atom_offsets"]) - 1)
    return sharding.shard_batch(batch, 0, k)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    p.add_argument("--n-struct", type=int, default=None, help="structures per GPU (default: the workload's)")
    p.add_argument("--n-sparse", type=int, default=None)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--cpu-sample", type=int, default=None, help="structures in the CPU baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison")
    p.add_argument("--plain-steps", type=int, default=2)
    p.add_argument("--bulk-atoms", type=int, default=100000, help="atoms of the bulk box")
    p.add_argument("--profile", action="store_true",
                   help="run the warm-up steps, then one step between cudaProfilerStart and cudaProfilerStop "
                        "(for ncu --profile-from-start off), and exit")
    p.add_argument("--workload", default="gap", choices=["gap", "bulk", "triclinic", "training", "md"],
                   help="gap: E+F prediction on 10 000 molecule clusters (the headline); bulk: one periodic "
                        "100 000-atom box (n 12, l 9); triclinic: 256 sheared periodic cells, 2 000 sparse "
                        "points per species; training: sparse-kernel K_NM energy and gradient rows for GAP "
                        "fitting; md: MD steps of the reference's fitted methane model (rgpu_md_step)")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def sparse_counts(numbers, species, n_sparse, per_species):
    """Sparse points per species: a fixed number each, or n_sparse split in
    proportion to the species' atom counts."""
    if per_species is not None:
        return {s: int(per_species) for s in species}
    counts = {s: int(np.sum(numbers == s)) for s in species}
    tot = sum(counts.values())
    per = {s: int(round(n_sparse * c / tot)) for s, c in counts.items()}
    per[species[0]] += n_sparse - sum(per.values())
    return per


def sparse_selection(rb, calc, sel_batch, numbers, n_sparse, per_species, seed):
    """Sparse environments picked at random (seeded) from the features of
    sel_batch, per species as sparse_counts gives them; weights ~ N(0, 1)."""
    from librascal_b200 import synthetic
    species = sorted(set(int(z) for z in numbers) | set(int(z) for z in sel_batch["numbers"]))
    al = calc.transform(rb.AtomsList(rb.StructureSet(sel_batch)))
    keys = calc.get_keys(species)
    X = al.get_features(calc, keys=keys)
    info = al.get_representation_info()
    per = sparse_counts(numbers, species, n_sparse, per_species)
    idx = synthetic.select_sparse_points(X, info[:, 2], per, seed=seed)
    rng = np.random.default_rng(seed + 1)
    alpha = rng.normal(size=len(idx))
    sp = rb.SparsePoints(calc)
    sp.add_dense(info[idx, 2], X[idx], keys)
    return sp, alpha, species, X[idx], info[idx, 2]


def oracle_calc(hypers):
    from oracle import oracle as O
    return O.Calculator(hypers["interaction_cutoff"], hypers["cutoff_smooth_width"], hypers["max_radial"],
                        hypers["max_angular"], hypers["gaussian_sigma_constant"], spline=True, accuracy=1e-8)


def oracle_run(hypers, batch, species, T, sps, alpha, threads=1):
    """The CPU restatement (reference algorithm, FP64) on every structure of
    `batch`, one structure per task; returns (seconds, atoms, E, F)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O
    calc = oracle_calc(hypers)
    off = batch["atom_offsets"]
    n = len(off) - 1

    def one(i):
        a0, a1 = off[i], off[i + 1]
        b = dict(atom_offsets=np.array([0, a1 - a0]), positions=batch["positions"][a0:a1],
                 numbers=batch["numbers"][a0:a1], cells=batch["cells"][i:i + 1], pbc=batch["pbc"][i:i + 1])
        r = O.Run(calc, b, species, gradients=True)
        return r.gap(sps, T, alpha, 2)

    t = time.perf_counter()
    if threads <= 1:
        res = [one(i) for i in range(n)]
    else:
        with ThreadPoolExecutor(threads) as ex:
            res = list(ex.map(one, range(n)))
    secs = time.perf_counter() - t
    E = np.concatenate([r[0] for r in res])
    F = np.concatenate([r[1] for r in res])
    return secs, int(off[-1]), E, F


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


def fma_peaks(lib):
    """FP32 and FP64 FMA TFLOP/s of this GPU, measured by the library's
    microbenchmark (rgpu_measure_fma_peak)."""
    import ctypes
    out = {}
    for name, prec in (("fp32", 1), ("fp64", 0)):
        v = ctypes.c_double()
        rc = lib.rgpu_measure_fma_peak(prec, ctypes.byref(v))
        out[name] = v.value if rc == 0 else None
    return out


# DRAM bytes (read + write) per grouped GEMM launch at the molecule-cluster
# workload: the average of the forward and backward launches of one ncu
# capture of the 2 000-cluster case (32 505 atoms), scaled by atoms to
# 160 449 atoms.
GEMM_TRAFFIC_PER_LAUNCH = 0.5 * (1.280e9 + 1.925e9) * 160449 / 32505


def row_stride(L):
    """Floats between consecutive (species, radial) rows of the FP32
    expansion coefficients: l-blocks padded to 4 floats, the stride an odd
    multiple of 4."""
    s = sum((2 * l + 1 + 3) // 4 * 4 for l in range(L + 1))
    return s if (s // 4) % 2 == 1 else s + 4


def stage_roofline(stages, nc, n_pairs, n_atoms, S, n, L, Dg, hbm, fp32):
    """Per-centre kernels of the FP32 path against HBM: algorithmic bytes each
    kernel must move in its layout (pair data read once, per-centre arrays
    read or written once; feature rows of Dg packed columns) over its
    CUDA-event time."""
    K = (L + 1) ** 2
    C = 4.0 * nc * S * n * row_stride(L)   # FP32 expansion coefficients
    dC = 4.0 * nc * S * n * K              # dE/dC
    X2 = 4.0 * nc * Dg                     # BF16 hi + lo rows
    pair = 36.0 * n_pairs                  # distance, direction, neighbour index
    rows = {
        "expansion": (2, pair + C),
        "power_spectrum": (3, C + X2 + 4.0 * nc),
        "ps_backward": (6, C + X2 + 4.0 * nc * Dg + dC + 4.0 * nc),
        "pair_adjoint": (7, pair + 4.0 * n_pairs + dC + 24.0 * n_atoms),
    }
    out = {}
    for k, (i, b) in rows.items():
        ms = float(stages[i])
        gbs = b / (ms * 1e-3) / 1e9 if ms > 0 else None
        out[k] = dict(ms=round(ms, 4), algorithmic_gb=round(b / 1e9, 4), achieved_gbs=gbs,
                      frac_hbm=(gbs / hbm) if gbs else None)
    out["peaks"] = dict(hbm_gbs=hbm, fp32_tflops_measured=fp32)
    return out
def gemm_flops_algorithmic(st, batch, species, msp, n, L):
    """Flops the two GAP contractions need (forward k = x . t and backward
    dE/dx = W T, 2 flops per multiply-add each): per row, the sparse points
    of its species times the power-spectrum entries it can hold, the
    upper triangles of the per-l Gram blocks of the species pairs present
    among its neighbours (n(n+1)/2 per l for a same-species pair, n^2 for
    two species). The GEMMs skip what no row of a 128-row tile holds, so
    they issue at least this."""
    nl = st.neighbour_list()
    sidx = {int(z): i for i, z in enumerate(species)}
    lut = np.zeros(int(max(species)) + 1, np.int64)
    for z, i in sidx.items():
        lut[z] = i
    po = nl["pair_offsets"]
    bits = np.left_shift(1, lut[batch["numbers"][nl["j"]]])
    mask = np.bitwise_or.reduceat(bits, po[:-1])
    present = np.array([[(m >> a) & 1 for a in range(len(species))] for m in range(1 << len(species))], bool)
    L1 = L + 1
    per_mask = np.zeros(1 << len(species))
    for m in range(1 << len(species)):
        k = present[m].sum()
        per_mask[m] = L1 * (k * n * (n + 1) // 2 + k * (k - 1) // 2 * n * n)
    centre_species = lut[batch["numbers"][nl["center_atom"]]]
    m_row = np.asarray(msp)[centre_species]
    return float(4.0 * np.sum(m_row * per_mask[mask]))


TRAINING_METRIC = "GAP training K_NM rows (energy + position gradients) atoms/s on 1 B200, FP64"
FP64_NOMINAL_TFLOPS = 37.0  # B200 nominal FP64 (CUDA cores), used only if the measurement fails


def run_training(args):
    """One step = the K_NM energy rows and gradient rows of compute_KNM for a
    batch of clusters against 4 000 sparse points, FP64, through the C ABI."""
    import torch
    import librascal_b200 as rb
    from librascal_b200 import _native as N, synthetic
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    spec = workload_spec("gap", args.seed)
    hypers = spec["hypers"]
    n_struct = min(args.n_struct or 1000, 1000)
    batch = synthetic.molecule_clusters(n_struct=n_struct, seed=args.seed + rank)
    n_atoms = int(batch["atom_offsets"][-1])
    calc = rb.SphericalInvariants(**hypers)
    sp, alpha, species, T_sel, sps_sel = sparse_selection(rb, calc, batch, batch["numbers"],
                                                          args.n_sparse or spec["n_sparse"], None, args.seed)
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
        oc = oracle_calc(hypers)
        t = time.perf_counter()
        r = O.Run(oc, sub, species, gradients=True)
        r.kernel_nm(sps_sel, T_sel, 2)
        r.kernel_nm_derivative(sps_sel, T_sel, 2)
        secs = time.perf_counter() - t
        cpu = dict(value=float(off[ns]) / secs, unit="atoms/s", cores=1, kind="port",
                   sample="first %d clusters (%d atoms), K_NM energy + gradient rows, CPU FP64 restatement, "
                          "1 thread, %.1f s" % (ns, int(off[ns]), secs))
    fp64_peak = fma_peaks(lib)["fp64"]
    fp64_kind = "measured FP64 FMA rate of this GPU (rgpu_measure_fma_peak)"
    if not fp64_peak:
        fp64_peak, fp64_kind = FP64_NOMINAL_TFLOPS, "nominal FP64 (the measurement failed)"
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
                              achieved=achieved, peak=fp64_peak, unit="TFLOP/s",
                              frac=achieved / fp64_peak, traffic=None, peak_kind=fp64_kind,
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


def run_reference_arm(args):
    """The reference algorithm (CPU restatement, FP64) on a bounded sample of
    the workload per step, with all host threads; rank 0 only."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import oracle as O
    spec = workload_spec(args.workload if args.workload in ("gap", "bulk", "triclinic") else "gap", args.seed)
    hypers = spec["hypers"]
    k = args.cpu_sample or spec["sample_default"]
    n_struct = args.n_struct or spec["default_struct"]
    if spec["shardable"]:
        # the first structures of the same seeded batch as the GPU arm, a
        # new sample for every step
        batch = spec["make"](max(k * (args.steps + args.warmup), min(n_struct, 1000)), args.seed)
        samples = [_slice(batch, step * k, (step + 1) * k) for step in range(args.warmup + args.steps)]
    else:
        samples = [spec["sample"](None, k)] * (args.warmup + args.steps)
        batch = spec["make"](1, args.seed)
    sel = spec["selection"](batch)
    species = sorted(set(int(z) for z in batch["numbers"]) | set(int(z) for z in sel["numbers"]))
    # sparse points from the oracle's features of the selection batch
    r = O.Run(oracle_calc(hypers), sel, species)
    X = r.power_spectrum()
    ca, _, _ = r.centers()
    rowsp = sel["numbers"][ca]
    from librascal_b200 import synthetic
    per = sparse_counts(batch["numbers"], species, args.n_sparse or spec["n_sparse"], spec["per_species"])
    idx = synthetic.select_sparse_points(X, rowsp, per, seed=args.seed)
    T, sps = X[idx], rowsp[idx]
    alpha = np.random.default_rng(args.seed + 1).normal(size=len(idx))
    threads = os.cpu_count() or 1
    rates, secs_timed = [], []
    for step, b in enumerate(samples):
        secs, atoms, _, _ = oracle_run(hypers, b, species, T, sps, alpha, threads)
        if step >= args.warmup:
            rates.append(atoms / secs)
            secs_timed.append(secs)
    v = float(np.mean(rates))
    desc = spec["sample_desc"] % k
    line = dict(metric=METRIC, value=v, unit="atoms/s", n_gpus=args.gpus, steps=args.steps, warmup=args.warmup,
                ms_per_step=1e3 * float(np.mean(secs_timed)), higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="f64", data="synthetic", impl="reference",
                config=dict(workload=spec["desc"], sample="%s per step, %d sparse points" % (desc, len(idx))),
                cpu_baseline=dict(value=v, unit="atoms/s", cores=threads, kind="port",
                                  sample="%s (%d sparse points) per step, CPU FP64 restatement, %d threads"
                                         % (desc, len(idx), threads)),
                e2e=dict(value=v, unit="atoms/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)
    return 0


def _slice(batch, a, b):
    from librascal_b200 import sharding
    n = len(batch["atom_offsets"]) - 1
    return sharding.shard_batch(batch, min(a, n), min(b, n))


def rel_err(a, b):
    """max|a - b| / max|b| (0 for an all-zero reference)."""
    d = float(np.abs(np.asarray(a) - np.asarray(b)).max()) if np.size(b) else 0.0
    s = float(np.abs(np.asarray(b)).max()) if np.size(b) else 0.0
    return d / s if s > 0 else d


def run_gap(args):
    """The gap-like workloads: FP32 adjoint path timed with device-resident
    inputs (value) and through the C ABI with host buffers (e2e), the plain
    FP64 GPU path on the same batch, the accuracy of both, and the CPU
    baseline."""
    import torch
    import librascal_b200 as rb
    from librascal_b200 import _native as N, sharding
    rank, world, local = dist_env()
    spec = workload_spec(args.workload, args.seed, args.bulk_atoms)
    hypers = spec["hypers"]
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()

    n_struct = args.n_struct or spec["default_struct"]
    if spec["shardable"]:
        # one seeded batch of world x n_struct structures, cut into per-rank
        # shards of nearly equal cost: every GPU has about n_struct
        # structures' work (weak scaling) and no two ranks share a structure
        full = spec["make"](n_struct * world, args.seed)
        parts = sharding.partition(sharding.structure_costs(full), world)
        batch = sharding.shard_batch(full, *parts[rank])
        parallelism = "dp%d: structures sharded across ranks by cost (sharding.partition)" % world
    else:
        full = spec["make"](1, args.seed + rank)  # one box per rank: replicas
        batch = full
        parallelism = "dp%d: one box per rank (replicas)" % world
    n_atoms = int(batch["atom_offsets"][-1])
    calc = rb.SphericalInvariants(**hypers)
    sp, alpha, species, T_sel, sps_sel = sparse_selection(rb, calc, spec["selection"](full), full["numbers"],
                                                          args.n_sparse or spec["n_sparse"], spec["per_species"],
                                                          args.seed)
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

    def timed(step, steps, warmup):
        for _ in range(warmup):
            step()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        for _ in range(steps):
            step()
        e1.record(ext)
        e1.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1)) / steps

    # ---- value: inputs resident, outputs on the device
    def step_resident(precision=args.precision):
        st.invalidate()
        model.predict(st, precision, energies=False, forces=False)

    for _ in range(args.warmup):
        step_resident()
    barrier()
    if args.profile:
        # one step of the timed kind (the recorded graph of this bucket) in a
        # profiler range, for a launch list or a per-kernel capture
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        step_resident()
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        if pg is not None:
            pg.destroy_process_group()
        return 0
    l0 = lib.rgpu_kernel_launches(0)
    g0 = st.graph_info()
    with Clocks(dev) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        for _ in range(args.steps):
            step_resident()
        e1.record(ext)
        e1.synchronize()
    barrier()
    g1 = st.graph_info()
    # kernels replayed from a recorded graph do not pass the library's launch
    # counter: count the graph's kernel nodes per replay
    launches = int(lib.rgpu_kernel_launches(0) - l0) + (g1[1] - g0[1]) * g1[3]
    ms = max_over_ranks(e0.elapsed_time(e1)) / args.steps
    value = n_atoms * world / (ms * 1e-3)

    # ---- the same steps without the recorded graphs (the ordinary path,
    # which sizes its buffers through host synchronisations), and the stage
    # breakdown, which only the ordinary path records
    st.use_graphs(False)
    ms_ordinary = timed(step_resident, max(args.steps // 2, 3), 1)
    stages = np.zeros(8)
    for _ in range(3):
        step_resident()
        stages += st.stage_times()
    stages /= 3
    # the launch shapes in use (the autotuner's table, librascal_b200/tune.py)
    # against the hand-picked defaults, stage by stage
    from librascal_b200 import tune
    shape = (len(species), hypers["max_radial"], hypers["max_angular"])
    tiles_cfg = tune.get_config(shape)
    tiles = dict(shape=list(shape), config=tiles_cfg, tuned=tiles_cfg != tune.DEFAULT)
    if tiles["tuned"]:
        tune.set_config(shape, None)
        dstages = np.zeros(8)
        for _ in range(3):
            step_resident()
            dstages += st.stage_times()
        tune.set_config(shape, tiles_cfg)
        tiles["default_stage_ms"] = [round(float(x) / 3, 4) for x in dstages]
        tiles["tuned_stage_ms"] = [round(float(x), 4) for x in stages]
    st.use_graphs(True)
    # a small batch of the same workload (launch- and synchronisation-bound),
    # recorded against ordinary
    small = None
    if spec["shardable"]:
        sb = _first(batch, 100)
        ss = rb.StructureSet(sb)
        ext_s = torch.cuda.ExternalStream(ss.stream())

        def step_small():
            ss.invalidate()
            model.predict(ss, args.precision, energies=False, forces=False)

        small = dict(n_structures=int(len(sb["atom_offsets"]) - 1), n_atoms=int(sb["atom_offsets"][-1]))
        for g in (True, False):
            ss.use_graphs(g)
            for _ in range(3):
                step_small()
            torch.cuda.synchronize()
            a0 = torch.cuda.Event(enable_timing=True)
            a1 = torch.cuda.Event(enable_timing=True)
            a0.record(ext_s)
            for _ in range(20):
                step_small()
            a1.record(ext_s)
            a1.synchronize()
            small["ms_per_step_graph" if g else "ms_per_step_ordinary"] = a0.elapsed_time(a1) / 20
        del ss
    import ctypes
    nc_, np_ = ctypes.c_int64(), ctypes.c_int64()
    N.check(lib.rgpu_neighbour_list_size(st.handle, ctypes.byref(nc_), ctypes.byref(np_)))
    n_centers, n_pairs = nc_.value, np_.value
    counts = np.array([np.sum(batch["numbers"] == s) for s in species])
    msp = np.array([int(np.sum(np.asarray(sp.species) == s)) for s in species])
    S, n, L = len(species), hypers["max_radial"], hypers["max_angular"]
    # the FP32 path's rows: the upper triangles of the per-l Gram matrices in
    # 2 x 2 tiles grouped into species-pair segments of 32-column multiples,
    # Dg columns in all
    Sn = S * n
    G, npg = (S, n // 2) if n % 2 == 0 else (1, (Sn + 1) // 2)
    lenD = (4 * (L + 1) * npg * (npg + 1) // 2 + 31) // 32 * 32
    lenO = (4 * (L + 1) * npg * npg + 31) // 32 * 32
    Dg = G * lenD + G * (G - 1) // 2 * lenO
    gemm_flops = gemm_flops_algorithmic(st, batch, species, msp, n, L)  # forward + backward
    gemm_ms = stages[4] + stages[5]
    bf16_peak, hbm_peak, peak_kind = peaks()
    achieved = gemm_flops / (gemm_ms * 1e-3) / 1e12 if gemm_ms > 0 else None

    # ---- e2e: host buffers through the C ABI
    e2e = None
    off = batch["atom_offsets"]
    if not args.no_e2e:
        E = np.zeros(len(off) - 1)
        F = np.zeros((n_atoms, 3))
        off64 = np.ascontiguousarray(off, np.int64)
        pos = np.ascontiguousarray(batch["positions"], np.float64)
        num = np.ascontiguousarray(batch["numbers"], np.int32)
        cel = np.ascontiguousarray(batch["cells"], np.float64)
        pbc = np.ascontiguousarray(batch["pbc"], np.int32)
        prec = N.PRECISION_FP32 if args.precision == "fp32" else N.PRECISION_FP64

        def step_e2e():
            N.check(lib.rgpu_structures_set(st.handle, len(off64) - 1, N.ptr(off64, N.c_i64_p),
                                            N.ptr(pos, N.c_dbl_p), N.ptr(num, N.c_int_p), N.ptr(cel, N.c_dbl_p),
                                            N.ptr(pbc, N.c_int_p), None))
            N.check(lib.rgpu_gap_predict(model.handle, st.handle, prec, N.ptr(E, N.c_dbl_p), N.ptr(F, N.c_dbl_p)))

        ms_e2e = timed(step_e2e, args.steps, args.warmup)
        h2d = off64.nbytes + pos.nbytes + num.nbytes + cel.nbytes + pbc.nbytes
        h2d += 4 * (len(off64) - 1) + 8 * len(off64) + 4 * n_atoms  # centre counts, offsets, atom->structure
        d2h = E.nbytes + F.nbytes
        e2e = dict(value=n_atoms * world / (ms_e2e * 1e-3), unit="atoms/s", h2d_bytes_per_step=int(h2d),
                   d2h_bytes_per_step=int(d2h), ms_per_step=ms_e2e)

    # ---- the metric's comparison: the plain FP64 GPU path, same batch
    plain = None
    acc = None
    if not args.no_plain and args.precision == "fp32":
        plain_ms = timed(lambda: step_resident("fp64"), max(args.plain_steps, 1), 1)
        plain_stages = st.stage_times()
        st.invalidate()
        E32, F32 = model.predict(st, "fp32")
        st.invalidate()
        E64, F64 = model.predict(st, "fp64")
        st.invalidate()
        acc = dict(force_err=max_over_ranks(rel_err(F32, F64)), energy_err=max_over_ranks(rel_err(E32, E64)))
        plain = dict(ms=plain_ms, stage_ms=[round(float(x), 3) for x in plain_stages])

    # ---- CPU baseline and the accuracy of both GPU paths against the oracle
    # on the same sample (rank 0, N = 1)
    cpu = None
    oracle_errors = None
    fma = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        k = args.cpu_sample or spec["sample_default"]
        sample = spec["sample"](batch, k)
        T = sp.dense(species)
        secs, atoms, E_o, F_o = oracle_run(hypers, sample, species, T, np.asarray(sp.species), alpha, 1)
        cpu = dict(value=atoms / secs, unit="atoms/s", cores=1, kind="port",
                   sample="%s (%d atoms), E+F, CPU FP64 restatement of the reference algorithm, 1 thread, "
                          "%.1f s" % (spec["sample_desc"] % k, atoms, secs))
        ss = rb.StructureSet(sample)
        oracle_errors = dict(sample=spec["sample_desc"] % k, atoms=atoms)
        for prec in ("fp64", "fp32"):
            Eg, Fg = model.predict(ss, prec)
            ss.invalidate()
            oracle_errors[prec] = dict(force_err=rel_err(Fg, F_o), energy_err=rel_err(Eg, E_o))
        del ss
    if rank == 0:
        fma = fma_peaks(lib)

    if rank == 0:
        speedup = (plain["ms"] / ms) if plain else None
        line = dict(
            metric=METRIC, value=value, unit="atoms/s", n_gpus=world, steps=args.steps, warmup=args.warmup,
            ms_per_step=ms, higher_is_better=True, scaling="weak", vs_baseline=None,
            dtype="f32" if args.precision == "fp32" else "f64", data="synthetic",
            config=dict(workload=spec["desc"], n_structures=int(len(off) - 1), n_atoms=n_atoms,
                        n_pairs=int(n_pairs), sparse_points=int(sp.size()), precision=args.precision,
                        parallelism=parallelism,
                        l2="inputs larger than L2: X and dE/dX are %.1f GB each" % (n_atoms * Dg * 4 / 1e9),
                        stage_ms=dict(zip(["total", "neighbour_list", "expansion", "power_spectrum",
                                           "gemm_fwd", "gemm_bwd", "ps_backward", "pair_adjoint"],
                                          [round(float(x), 4) for x in stages]))),
            graphs=dict(ms_per_step_ordinary_path=ms_ordinary, buckets=g1[0], replays_timed=g1[1] - g0[1],
                        kernels_per_replay=g1[3], small_batch=small,
                        note="value is timed with the recorded CUDA graph of this size bucket; the ordinary "
                             "path runs the same kernels with host synchronisations that size its buffers"),
            tiles=tiles,
            plain_fp64_ms_per_step=plain["ms"] if plain else None,
            plain_fp64_atoms_per_s=(n_atoms * world / (plain["ms"] * 1e-3)) if plain else None,
            plain_fp64_stage_ms=plain["stage_ms"] if plain else None,
            speedup_vs_plain_fp64=speedup,
            force_err=acc["force_err"] if acc else None,
            energy_err=acc["energy_err"] if acc else None,
            force_err_bar=FORCE_ERR_BAR,
            meets_target=(bool(speedup >= TARGET_SPEEDUP and acc["force_err"] <= FORCE_ERR_BAR)
                          if plain else None),
            oracle_errors=oracle_errors,
            roofline=dict(bound="tensor", kernel="tcgen05 BF16x3 GEMMs (forward + backward)",
                          achieved=achieved, peak=bf16_peak, unit="TFLOP/s",
                          frac=(achieved / bf16_peak) if achieved else None,
                          traffic=(GEMM_TRAFFIC_PER_LAUNCH if (args.workload == "gap" and n_struct == 10000)
                                   else None),
                          peak_kind="%s dense bf16; achieved counts algorithmic 2MNK flops, the "
                                    "3-term split issues 3x that on the tensor pipe" % peak_kind,
                          issued_frac=(3 * achieved / bf16_peak) if achieved else None,
                          flops_per_step=gemm_flops),
            stage_roofline=stage_roofline(stages, n_centers, n_pairs, n_atoms, S, n, L, Dg, hbm_peak,
                                          fma["fp32"] if fma else None),
            measured_fma_tflops=fma,
            cpu_baseline=cpu, e2e=e2e, gpu_launches=launches, clocks=clk.summary())
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "training":
        return run_training(args)
    if args.workload == "md":
        return run_md(args)
    return run_gap(args)


if __name__ == "__main__":
    sys.exit(main())
