"""Benchmark of the fused FP64 mass operator_apply (GDoF/s) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (one GPU): the order-sweep mesh of ~64M DoFs -- a perturbed 3D hex
box of 100^3 elements on [0,1]^3, P=5 GLL nodes and Q=6 Gauss points per
direction, num_comp=1, FP64, u ~ U[-1,1] (seeded), qdata = det(J) w built on
the device.  A step is one operator apply v = M u over the whole mesh (v
zeroed, then the fused gather/interp/qfunction/interp^T/scatter-add kernel).
Inputs (3.3 GB per apply) exceed the 126 MB L2, so no flush is needed between
steps.  With N ranks (torchrun) each GPU applies its own copy of the mesh
(independent meshes, no collective on the data path): weak scaling, value =
all ranks' DoFs / max-over-ranks time.

--impl reference times the reference CPU implementation (fe-demo-cpp's own
operator_apply, compiled from its sources into oracle/_ref) with all host
threads, on a bounded sample of the same workload; rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GDoF/s operator_apply"
UNIT = "GDoF/s"
SHAPE, P, Q, NC, SEED = (100, 100, 100), 5, 6, 1, 1
WORKLOAD = ("mass operator_apply, FP64 3D hex box 100^3 elements on [0,1]^3 (interior vertices "
            "perturbed U[-0.1h,0.1h], seed 1), P=5 GLL nodes, Q=6 Gauss points, num_comp=1, "
            "~64.5M DoFs, qdata = det(J)*w, u ~ U[-1,1]")


def algorithmic_bytes(num_elem, num_nodes, P, Q, nc=1, dim=3):
    """Compulsory HBM bytes of one fused apply: offsets (int32) and qdata (FP64)
    per element, u read + v write per DoF."""
    return num_elem * (4 * P**dim + 8 * Q**dim) + 16 * nc * num_nodes


def algorithmic_flops(num_elem, P, Q, nc=1, dim=3):
    """Sum-factorised flops of one apply: interp + interp^T + pointwise."""
    if dim == 2:
        return num_elem * nc * (4 * (P**2 * Q + P * Q**2) + Q**2)
    return num_elem * nc * (4 * (P**3 * Q + P**2 * Q**2 + P * Q**3) + Q**3)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


TRAFFIC_PROFILE = os.path.join("profiles", "mass3d_apply_P5Q6_64M.md")


def ncu_traffic(variant):
    """DRAM bytes per launch of the fused kernel as captured by ncu and
    summarised in profiles/mass3d_apply_P5Q6_64M.md (line
    'dram_bytes_per_launch: <n> (<variant>)'), labelled as that profile's
    figure: it is not measured in this run.  None when the profile covers
    another kernel variant than the one this run times."""
    path = os.path.join(ROOT, TRAFFIC_PROFILE)
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.strip().startswith("dram_bytes_per_launch:"):
            rest = line.split(":", 1)[1].strip()
            try:
                val = float(rest.split()[0])
            except ValueError:
                return None
            tag = rest[rest.find("(") + 1: rest.find(")")] if "(" in rest else ""
            if tag and tag != variant:
                return None
            return {"value": val, "source": f"ncu capture of the same workload, {TRAFFIC_PROFILE} "
                                          "(not measured in this run)"}
    return None


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# reference CPU path on a bounded sample
# ---------------------------------------------------------------------------
class RefSample:
    """The first `n_slabs` z-layers of elements of the workload mesh as a
    self-contained mesh, applied by the reference's operator_apply on element
    chunks in parallel threads (oracle.RefPlan)."""

    def __init__(self, mesh, target_s=2.0, threads=None):
        import oracle
        self.oracle = oracle
        oracle.build(with_ref=None)
        self.ref = oracle.ref()
        self.mesh = mesh
        self.threads = threads or host_threads()
        slab = mesh.shape[0] * mesh.shape[1]
        # calibrate on one slab, then size the sample to ~target_s per apply
        self._make(1)
        self._time_once()
        t = self._time_once()
        self.close()
        slabs = int(max(1, min(mesh.shape[2], round(target_s / max(t, 1e-3)))))
        self.n_slabs = slabs
        self.ne = self._make(slabs)
        self.frac = self.ne / mesh.num_elem

    def _make(self, slabs):
        m = self.mesh
        ne = slabs * m.shape[0] * m.shape[1]
        local, n_loc, _, coords = self.oracle.compact_submesh(m.offsets, P**3, ne, m.coords, 3, m.num_nodes)
        # qdata through the reference build operator, per chunk in parallel
        self.plan = self.oracle.RefPlan(self.ref, 3, ne, P, Q, n_loc, local, None, self.threads, coords=coords)
        self.u = np.random.default_rng([SEED, 1]).uniform(-1, 1, n_loc)
        self.v = np.zeros(n_loc)
        self.local, self.n_loc, self.coords = local, n_loc, coords
        return ne

    def device_parity(self, fem, dev):
        """Parity guard at the workload's own mesh: the sample's submesh
        through the device path (fused build, then the fused apply) against
        the reference's build + operator_apply output of the last timed
        apply; returns max |v_dev - v_ref| / max |v_ref|."""
        import torch
        rx = fem.Restriction(self.ne, P**3, 3, self.n_loc, 3 * self.n_loc, self.local)
        qd = torch.empty(Q**3 * self.ne, dtype=torch.float64, device=dev)
        fem.mass_build(rx, fem.Basis(3, 3, P, Q), torch.from_numpy(self.coords).to(dev), qd)
        op = fem.MassOperator(fem.Restriction(self.ne, P**3, 1, self.n_loc, self.n_loc, self.local),
                              fem.Basis(3, 1, P, Q), qd, fem.QF.apply_mass)
        v = torch.empty(self.n_loc, dtype=torch.float64, device=dev)
        op.apply(torch.from_numpy(self.u).to(dev), v)
        got = v.cpu().numpy()
        return float(np.abs(got - self.v).max() / np.abs(self.v).max())

    def _time_once(self):
        t0 = time.perf_counter()
        self.plan.apply(self.u, self.v)
        return time.perf_counter() - t0

    def gdofs(self, seconds):
        # scaled to the whole workload by the element fraction of the sample
        return self.mesh.num_nodes * self.frac / seconds / 1e9

    def describe(self):
        return (f"first {self.n_slabs} of {self.mesh.shape[2]} z-slabs ({self.ne} of {self.mesh.num_elem} elements, "
                f"{self.frac:.1%}) through the reference operator_apply, {self.threads} threads, element-chunked; "
                f"GDoF/s scaled by the element fraction")

    def close(self):
        if getattr(self, "plan", None) is not None:
            self.plan.close()
            self.plan = None


def run_reference(args, rank):
    from fe_demo_cpp_b200.mesh import box_mesh
    if rank != 0:
        return None
    mesh = box_mesh(SHAPE, P, seed=SEED)
    # each step is a sample sized so that warm-up + steps take about two minutes
    s = RefSample(mesh, target_s=min(2.0, 120.0 / (args.steps + args.warmup)))
    for _ in range(args.warmup):
        s._time_once()
    times = [s._time_once() for _ in range(args.steps)]
    s.close()
    t = statistics.median(times)
    value = s.gdofs(t)
    single = single_core_baseline(mesh)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "mesh": "x".join(map(str, SHAPE)), "P": P, "Q": Q, "num_comp": NC,
                   "dofs": mesh.num_nodes, "parallelism": "host threads over element chunks"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": s.threads, "kind": "reference",
                         "sample": s.describe(), "single_core": single},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def single_core_baseline(mesh, target_s=3.0):
    """The reference operator_apply on one host thread (it is single-threaded,
    src/operator.cpp:148), on a bounded sample of whole z-slabs: median of 3
    after 1 warm-up, GDoF/s scaled to the workload by the element fraction."""
    s = RefSample(mesh, target_s=target_s, threads=1)
    s._time_once()
    ts = [s._time_once() for _ in range(3)]
    s.close()
    return {"value": s.gdofs(statistics.median(ts)), "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": s.describe() + ", median of 3 after 1 warm-up"}


# ---------------------------------------------------------------------------
# the device path
# ---------------------------------------------------------------------------
def run_b200(args, rank, world, local_rank):
    import torch
    import fe_demo_cpp_b200 as fem
    from fe_demo_cpp_b200.build import build
    from fe_demo_cpp_b200.mesh import box_mesh
    from fe_demo_cpp_b200.telemetry import ClockSampler

    build()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    stream = torch.cuda.current_stream()

    mesh = box_mesh(SHAPE, P, seed=SEED)
    N, ne = mesh.num_nodes, mesh.num_elem
    x = torch.from_numpy(mesh.coords).to(dev)
    rx = fem.Restriction(ne, P**3, 3, N, 3 * N, mesh.offsets)
    bx = fem.Basis(3, 3, P, Q)
    qdata = torch.empty(Q**3 * ne, dtype=torch.float64, device=dev)
    fem.mass_build(rx, bx, x, qdata)
    ru = fem.Restriction(ne, P**3, 1, N, N, mesh.offsets)
    bu = fem.Basis(3, 1, P, Q)
    op = fem.MassOperator(ru, bu, qdata)
    op.set_kernel(fem.KernelVariant[args.kernel])
    info = op.info()
    launches = info["launches_per_apply"]
    del x, rx, bx, qdata
    torch.cuda.synchronize()
    torch.cuda.empty_cache()

    g = torch.Generator(device=dev).manual_seed(SEED + rank)
    u = torch.rand(N, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    v = torch.empty(N, dtype=torch.float64, device=dev)
    w = torch.zeros(N, dtype=torch.float64, device=dev)

    tuned = None
    if args.kernel == "auto":  # set-up, untimed: pick the fastest variant on this device
        tuned = op.autotune(u, v, reps=10)
        info = op.info()
    for _ in range(max(3, args.warmup)):
        op.apply(u, v)
        op.apply_add(u, w)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()

    K = args.steps
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(K + 1)] for _ in range(2)]
    sampler = ClockSampler(local_rank).start()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    # timed region 1: the public apply (zero v + fused kernel), per step
    for i in range(K):
        ev[0][i].record(stream)
        op.apply(u, v)
    ev[0][K].record(stream)
    # timed region 2: the fused kernel alone (apply_add: no zeroing)
    for i in range(K):
        ev[1][i].record(stream)
        op.apply_add(u, w)
    ev[1][K].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    step_ms = [ev[0][i].elapsed_time(ev[0][i + 1]) for i in range(K)]
    kern_ms = [ev[1][i].elapsed_time(ev[1][i + 1]) for i in range(K)]
    t_step = sum(step_ms) / K
    t_kern = sum(kern_ms) / K
    if dist:
        t = torch.tensor([t_step, t_kern], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_step, t_kern = t.tolist()
    value = world * N / (t_step * 1e-3) / 1e9

    # end to end through the host-memory entry point: pinned u in, v out
    u_h = torch.empty(N, dtype=torch.float64, pin_memory=True)
    v_h = torch.empty(N, dtype=torch.float64, pin_memory=True)
    u_h.copy_(u.cpu())
    for _ in range(2):
        op.apply_host(u_h.numpy(), v_h.numpy())
    e2e_steps = max(3, min(K, 20))
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        op.apply_host(u_h.numpy(), v_h.numpy())
    t_e2e = (time.perf_counter() - t0) / e2e_steps
    if dist:
        t = torch.tensor([t_e2e], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_e2e = t.item()
    e2e_value = world * N / t_e2e / 1e9
    # e2e parity guard: the host path returns the device result
    assert np.array_equal(v_h.numpy(), v.cpu().numpy()) or np.abs(v_h.numpy() - v.cpu().numpy()).max() <= 1e-13 * np.abs(v.cpu().numpy()).max()

    peak, peak_kind = measured_peaks()
    abytes = algorithmic_bytes(ne, N, P, Q)
    achieved = abytes / (t_kern * 1e-3) / 1e9
    traffic = ncu_traffic(info["kernel"]) if (SHAPE, P) == ((100, 100, 100), 5) else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": t_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "mesh": "x".join(map(str, SHAPE)), "P": P, "Q": Q, "num_comp": NC,
                   "dofs": N, "elements": ne, "scatter": "atomic", "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (3.3 GB per apply); no flush",
                   "kernel": "mass3d_apply_{}kernel<{},{}>".format(
                       {"pipelined": "pipe_", "paired": "x2_", "prefetch": "prefetch_", "occupancy": "occ_", "narrow": "narrow_", "element": "element_"}.get(info["kernel"], ""), P, Q),
                   "kernel_variant": info["kernel"], "autotuned": tuned is not None, "kernel_ms": t_kern,
                   "algorithmic_bytes_per_apply": abytes,
                   "algorithmic_flops_per_apply": algorithmic_flops(ne, P, Q)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                     if peak_kind == "measured" else "fallback 6650 GB/s"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * N, "d2h_bytes_per_step": 8 * N,
                "path": "fem_b200_mass_apply_host (pinned host u in, v out, synchronous; copies pipelined against element chunks)"},
        "clocks": clocks,
        "gpu_launches": 2 * K * launches,
    }
    # full-size property after the timed region: 1^T M 1 = the volume of the unit box
    u.fill_(1.0)
    op.apply(u, v)
    vol = float(v.sum())
    line["parity"] = {"full_size_1tM1": vol, "full_size_1tM1_err": abs(vol - 1.0)}
    assert abs(vol - 1.0) <= 1e-11, f"1^T M 1 = {vol!r}, not the unit box's volume"
    if rank == 0 and world == 1 and not args.no_orders:
        # after the timed region and the e2e run; the workload's buffers are released first
        del u, v, w, op, ru, bu
        torch.cuda.empty_cache()
        line["orders"] = {"note": "P = 2..4 (Q = P+1), ~64M DoFs, FP64, atomic scatter, autotuned kernel; "
                                  "kernel_ms = the fused kernel alone (apply_add), apply_ms = the public apply "
                                  "(v zeroed + kernel); frac = algorithmic bytes / kernel_ms / measured HBM peak; "
                                  f"{args.orders_steps} launches each, CUDA events",
                          "entries": measure_orders(dev, peak, args.orders_steps)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        s = RefSample(mesh, target_s=args.cpu_sample_s / 4)
        s._time_once()
        ts = [s._time_once() for _ in range(3)]
        s.close()
        line["cpu_baseline"] = {"value": s.gdofs(statistics.median(ts)), "unit": UNIT, "cores": s.threads,
                                "kind": "reference", "sample": s.describe() + ", median of 3 after 1 warm-up",
                                "single_core": single_core_baseline(mesh)}
        # parity guard on the same sample of the workload mesh (outside every timed region)
        err = s.device_parity(fem, dev)
        line["parity"].update({"sample": f"first {s.n_slabs} z-slabs of the workload mesh ({s.ne} elements)",
                               "against": "reference build + operator_apply (oracle/_ref), element-chunked",
                               "max_rel_err": err, "tol": 1e-12})
        assert err <= 1e-12, f"device apply differs from the reference on the workload sample: {err:.3e}"
    return line


# ---------------------------------------------------------------------------
# low orders in the same run: P = 2, 3, 4 (Q = P+1) at ~64M DoFs, one and three
# components (the vector mass), the plan's autotuned kernel; the fused FP64
# apply's HBM roofline fraction at each
# ---------------------------------------------------------------------------
ORDERS = [(2, 1), (2, 3), (3, 1), (3, 3), (4, 1), (4, 3)]


def measure_orders(dev, peak, steps):
    import torch
    import fe_demo_cpp_b200 as fem
    from fe_demo_cpp_b200.mesh import mesh_for_dofs
    from fe_demo_cpp_b200.mesh_gpu import box_mesh_device

    out = []
    for Pp, nc in ORDERS:
        Qq = Pp + 1
        shape = mesh_for_dofs(64_000_000 // nc, Pp, 3)
        m = box_mesh_device(shape, Pp, seed=SEED, device=dev)
        N, ne = m.num_nodes, m.num_elem
        offs = m.offsets.cpu().numpy()
        rx = fem.Restriction(ne, Pp**3, 3, N, 3 * N, offs)
        qd = torch.empty(Qq**3 * ne, dtype=torch.float64, device=dev)
        fem.mass_build(rx, fem.Basis(3, 3, Pp, Qq), m.coords, qd)
        del rx
        m.coords = None
        op = fem.MassOperator(fem.Restriction(ne, Pp**3, nc, N, nc * N, offs), fem.Basis(3, nc, Pp, Qq), qd,
                              fem.QF.apply_mass_vector if nc > 1 else fem.QF.apply_mass)
        del qd
        g = torch.Generator(device=dev).manual_seed(SEED)
        u = torch.rand(nc * N, dtype=torch.float64, device=dev, generator=g) * 2 - 1
        v = torch.empty_like(u)
        op.autotune(u, v, reps=5)
        variant = op.info()["kernel"]
        for _ in range(3):
            op.apply(u, v)
        res = {}
        for name, fn in (("apply", op.apply), ("kernel", op.apply_add)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(steps):
                fn(u, v)
            e1.record()
            torch.cuda.synchronize()
            res[name] = e0.elapsed_time(e1) / steps
        ab = algorithmic_bytes(ne, N, Pp, Qq, nc)
        out.append({"P": Pp, "Q": Qq, "num_comp": nc, "mesh": "x".join(map(str, shape)), "dofs": nc * N,
                    "kernel_variant": variant, "apply_ms": res["apply"], "kernel_ms": res["kernel"],
                    "gdofs": nc * N / res["apply"] / 1e6, "algorithmic_bytes": ab,
                    "frac": ab / (res["kernel"] * 1e-3) / 1e9 / peak,
                    "frac_apply": ab / (res["apply"] * 1e-3) / 1e9 / peak})
        del op, u, v, m
        torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------
# order sweep: P = 2..8 (Q = P+1), num_comp 1 and 3, ~64M DoFs, every kernel
# variant, plus the standalone interp / grad basis applies (extra JSON lines)
# ---------------------------------------------------------------------------
def run_sweep(args):
    import torch
    import fe_demo_cpp_b200 as fem
    from fe_demo_cpp_b200.build import build
    from fe_demo_cpp_b200.mesh import mesh_for_dofs
    from fe_demo_cpp_b200.mesh_gpu import box_mesh_device

    build()
    dev = torch.device("cuda", 0)
    peak, _ = measured_peaks()
    Ps = [int(p) for p in args.sweep_P.split(",")]
    for dim, Pp in [(d, p) for d in (int(x) for x in args.sweep_dim.split(",")) for p in Ps]:
        Qq = Pp + 1
        for nc in (1, 3):
            shape = mesh_for_dofs(args.sweep_dofs // nc, Pp, dim)
            m = box_mesh_device(shape, Pp, seed=SEED, device=dev)
            N, ne = m.num_nodes, m.num_elem
            offs = m.offsets.cpu().numpy()
            rx = fem.Restriction(ne, Pp**dim, dim, N, dim * N, offs)
            bx = fem.Basis(dim, dim, Pp, Qq)
            qd = torch.empty(Qq**dim * ne, dtype=torch.float64, device=dev)
            fem.mass_build(rx, bx, m.coords, qd)
            del rx, bx
            m.coords = None
            ru = fem.Restriction(ne, Pp**dim, nc, N, nc * N, offs)
            bu = fem.Basis(dim, nc, Pp, Qq)
            op = fem.MassOperator(ru, bu, qd, fem.QF.apply_mass_vector if nc > 1 else fem.QF.apply_mass)
            u = torch.rand(nc * N, dtype=torch.float64, device=dev) * 2 - 1
            v = torch.empty_like(u)
            abytes = algorithmic_bytes(ne, N, Pp, Qq, nc, dim)
            for variant in fem.KernelVariant:
                if variant == fem.KernelVariant.auto or args.sweep_storage_only:
                    continue
                try:
                    op.set_kernel(variant)
                except fem.FemUnsupported:
                    continue
                for _ in range(3):
                    op.apply_add(u, v)
                torch.cuda.synchronize()
                t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                t0.record()
                for _ in range(args.sweep_steps):
                    op.apply_add(u, v)
                t1.record()
                torch.cuda.synchronize()
                kms = t0.elapsed_time(t1) / args.sweep_steps
                print(json.dumps({"sweep": "mass_apply", "dim": dim, "P": Pp, "Q": Qq, "num_comp": nc,
                                  "mesh": list(shape),
                                  "dofs": nc * N, "kernel": variant.name, "kernel_ms": kms,
                                  "gdofs_kernel": nc * N / kms / 1e6,
                                  "roofline_frac": abytes / (kms * 1e-3) / 1e9 / peak,
                                  "fp64_tflops": algorithmic_flops(ne, Pp, Qq, nc, dim) / (kms * 1e-3) / 1e12}),
                      flush=True)
            # reduced storage: FP32 (u, v, qdata) and BF16 (u, qdata; FP32 v), public applies;
            # in 3D at P >= 6, Q <= 8 also the tensor-core forms (3xTF32, one TF32 part, BF16)
            ab32 = ne * (4 * Pp**dim + 4 * Qq**dim) + 8 * nc * N
            ab16 = ne * (4 * Pp**dim + 2 * Qq**dim) + 6 * nc * N
            forms = [("fp32", "f32", op.apply_f32, ab32), ("bf16", "bf16", op.apply_bf16, ab16)]
            if dim == 3 and 6 <= Pp <= 8 and Qq <= 8:
                forms += [("fp32_tc_3xtf32", "f32", lambda a, b: op.apply_f32_tc(a, b, split=True), ab32),
                          ("fp32_tc_tf32", "f32", lambda a, b: op.apply_f32_tc(a, b, split=False), ab32),
                          ("bf16_tc", "bf16", op.apply_bf16_tc, ab16)]
            for name, st, fn, ab in forms:
                uu = u.float() if st == "f32" else u.to(torch.bfloat16)
                vv = torch.empty(nc * N, dtype=torch.float32, device=dev)
                for _ in range(3):
                    fn(uu, vv)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(args.sweep_steps):
                    fn(uu, vv)
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / args.sweep_steps
                print(json.dumps({"sweep": "mass_apply_storage", "storage": name, "dim": dim, "P": Pp, "Q": Qq,
                                  "num_comp": nc,
                                  "dofs": nc * N, "ms_per_apply": ms, "gdofs": nc * N / ms / 1e6,
                                  "algorithmic_bytes": ab, "roofline_frac": ab / (ms * 1e-3) / 1e9 / peak}),
                      flush=True)
                del uu, vv
            if args.sweep_storage_only:
                del op, ru, qd, u, v
                torch.cuda.empty_cache()
                continue
            op.set_kernel(fem.KernelVariant.auto)
            ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev[0].record()
            for _ in range(args.sweep_steps):
                op.apply(u, v)
            ev[1].record()
            torch.cuda.synchronize()
            ams = ev[0].elapsed_time(ev[1]) / args.sweep_steps
            print(json.dumps({"sweep": "mass_apply_auto", "dim": dim, "P": Pp, "Q": Qq, "num_comp": nc,
                              "dofs": nc * N,
                              "kernel": op.info()["kernel"], "ms_per_apply": ams,
                              "gdofs": nc * N / ams / 1e6}), flush=True)
            del op, ru, qd, u, v
            # standalone basis applies on E-vector / Q-vector sized arrays
            pn, qn = nc * Pp**3 * ne, nc * Qq**3 * ne
            if nc == 1 and dim == 3:
                b = fem.Basis(3, nc, Pp, Qq)
                for name, t_mode, ev_mode, n_in, n_out, flop_mult in [
                        ("interp", 0, 1, pn, qn, 1), ("interpT", 1, 1, qn, pn, 1),
                        ("grad", 0, 2, pn, 3 * qn, 3), ("gradT", 1, 2, 3 * qn, pn, 3)]:
                    x = torch.rand(n_in, dtype=torch.float64, device=dev)
                    y = torch.empty(n_out, dtype=torch.float64, device=dev)
                    b.apply(ne, t_mode, ev_mode, x, y)
                    torch.cuda.synchronize()
                    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    t0.record()
                    steps = max(2, args.sweep_steps // 4)
                    for _ in range(steps):
                        b.apply(ne, t_mode, ev_mode, x, y)
                    t1.record()
                    torch.cuda.synchronize()
                    ms = t0.elapsed_time(t1) / steps
                    flops = flop_mult * ne * 2 * (Pp**3 * Qq + Pp**2 * Qq**2 + Pp * Qq**3)
                    print(json.dumps({"sweep": "basis_apply", "op": name, "P": Pp, "Q": Qq, "elements": ne,
                                      "ms": ms, "io_gbs": 8 * (n_in + n_out) / (ms * 1e-3) / 1e9,
                                      "fp64_tflops": flops / (ms * 1e-3) / 1e12}), flush=True)
                    del x, y
                b.close()
            torch.cuda.empty_cache()
    return 0


# ---------------------------------------------------------------------------
# mixed-precision mass solve M u = f: 64^3 hexes, P=5, Q=6, num_comp=3 (vector
# mass), f ~ U[-1,1], rtol 1e-10; FP64 PCG against FP32 PCG inside FP64
# iterative refinement (extra JSON lines)
# ---------------------------------------------------------------------------
def cg_iteration_bytes(ne, n, P, Q, prec, nc):
    """Compulsory HBM bytes of one Chronopoulos-Gear PCG iteration: k-byte
    r, p, s and qdata, f-byte x, w and dinv (fp64: 8/8, fp32_ir: 4/4,
    bf16_ir: 2/4).  The vector update reads dinv, r, p, s, w, x and writes
    p, s, w, x, r (6 k + 5 f per entry); the apply reads offsets and qdata
    per element, gathers r (k) and one dinv per node (f / nc) and adds into
    w (2 f)."""
    k, f = {"fp64": (8, 8), "fp32_ir": (4, 4), "bf16_ir": (2, 4)}[prec]
    return n * (6 * k + 5 * f) + n * (k + 2 * f) + n * f // nc + ne * (4 * P**3 + k * Q**3)


def run_solve(args):
    import torch
    import fe_demo_cpp_b200 as fem
    from fe_demo_cpp_b200.build import build
    from fe_demo_cpp_b200.mesh_gpu import box_mesh_device
    from fe_demo_cpp_b200.telemetry import ClockSampler

    build()
    dev = torch.device("cuda", 0)
    shape = tuple(int(x) for x in args.solve_shape.split(","))
    Pp, nc = args.solve_P, 3
    Qq = Pp + 1
    m = box_mesh_device(shape, Pp, seed=SEED, device=dev)
    N, ne = m.num_nodes, m.num_elem
    offs = m.offsets.cpu().numpy()
    rx = fem.Restriction(ne, Pp**3, 3, N, 3 * N, offs)
    qd = torch.empty(Qq**3 * ne, dtype=torch.float64, device=dev)
    fem.mass_build(rx, fem.Basis(3, 3, Pp, Qq), m.coords, qd)
    del rx
    m.coords = None
    n = nc * N
    op = fem.MassOperator(fem.Restriction(ne, Pp**3, nc, N, n, offs, args.solve_scatter), fem.Basis(3, nc, Pp, Qq),
                          qd, fem.QF.apply_mass_vector)
    del qd
    g = torch.Generator(device=dev).manual_seed(SEED)
    f = torch.rand(n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    results, sols = {}, {}
    sampler = ClockSampler(0).start()
    for prec in ("fp64", "fp32_ir", "bf16_ir"):
        u = torch.empty_like(f)
        for _ in range(max(1, args.warmup // 3)):
            info = op.solve(f, u, rtol=args.solve_rtol, max_iter=2000, precision=prec)
        torch.cuda.synchronize()
        wall, dev_ms = [], []
        for _ in range(args.solve_steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record()
            info = op.solve(f, u, rtol=args.solve_rtol, max_iter=2000, precision=prec)
            e1.record()
            e1.synchronize()
            wall.append((time.perf_counter() - t0) * 1e3)
            dev_ms.append(e0.elapsed_time(e1))
        sols[prec] = u
        results[prec] = (info, wall, dev_ms)
    clocks = sampler.stop()
    ref = sols["fp64"]
    peak, _ = measured_peaks()
    base = None
    for prec, (info, wall, dev_ms) in results.items():
        wall_s = sorted(wall)
        p50 = statistics.median(wall_s)
        p99 = wall_s[min(len(wall_s) - 1, int(round(0.99 * (len(wall_s) - 1))))]
        mean_dev = sum(dev_ms) / len(dev_ms)
        sps = 1e3 / (sum(wall) / len(wall))
        base = sps if prec == "fp64" else base
        err = float((sols[prec] - ref).norm() / ref.norm())
        it_bytes = cg_iteration_bytes(ne, n, Pp, Qq, prec, nc)
        print(json.dumps({
            "solve": "mass", "precision": prec, "metric": "solves/s", "value": sps, "unit": "solves/s",
            "p50_ms": p50, "p99_ms": p99, "device_ms_mean": mean_dev, "steps": len(wall),
            "iterations": info["iterations"], "refinements": info["refinements"],
            "rel_residual": info["rel_residual"], "rel_err_vs_fp64": err,
            "speedup_vs_fp64": sps / base,
            "config": {"mesh": list(shape), "P": Pp, "Q": Qq, "num_comp": nc, "dofs": n, "elements": ne,
                       "rtol": args.solve_rtol, "scatter": "deterministic" if args.solve_scatter else "atomic",
                       "f": "U[-1,1] seed 1", "preconditioner": "Jacobi (assembled diagonal)",
                       "krylov": "Chronopoulos-Gear PCG, device-resident scalars"},
            "iteration_roofline": {"bytes_per_iteration": it_bytes,
                                   "achieved_gbs": it_bytes * info["iterations"] / (mean_dev * 1e-3) / 1e9,
                                   "peak_gbs": peak},
            "clocks": clocks}), flush=True)
    return 0


# ---------------------------------------------------------------------------
# batched uneven meshes: 512 independent 2D/3D boxes (d = 2 or 3 at 50/50,
# elements log-uniform in [4^d, 48^d], P uniform in 2..6, Q = P+1, num_comp
# uniform in 1..3), one graph launch per step, FP64 and FP32 (extra lines)
# ---------------------------------------------------------------------------
def batch_specs(n, seed):
    rng = np.random.default_rng([seed, 4])
    specs = []
    for _ in range(n):
        d = 2 if rng.random() < 0.5 else 3
        side = int(round(float(np.exp(rng.uniform(np.log(4), np.log(48))))))
        P = int(rng.integers(2, 7))
        nc = int(rng.integers(1, 4))
        specs.append((d, (side,) * d, P, nc))
    return specs


def make_batch_ops(n_meshes, dev):
    """The batch workload's operators and inputs: (specs, ops, us, dofs,
    algorithmic bytes in FP64, in FP32)."""
    import torch
    import fe_demo_cpp_b200 as fem
    from fe_demo_cpp_b200.mesh import box_mesh
    from fe_demo_cpp_b200.mesh_gpu import box_mesh_device
    specs = batch_specs(n_meshes, SEED)
    ops, us, abytes64, abytes32, dofs = [], [], 0, 0, 0
    for i, (d, shape, Pp, nc) in enumerate(specs):
        Qq = Pp + 1
        if d == 3:
            m = box_mesh_device(shape, Pp, seed=SEED + i, device=dev)
            offs, coords = m.offsets.cpu().numpy(), m.coords
        else:
            m = box_mesh(shape, Pp, seed=SEED + i)
            offs, coords = m.offsets, torch.from_numpy(m.coords).to(dev)
        N, ne = m.num_nodes, m.num_elem
        rx = fem.Restriction(ne, Pp**d, d, N, d * N, offs)
        qd = torch.empty(Qq**d * ne, dtype=torch.float64, device=dev)
        fem.mass_build(rx, fem.Basis(d, d, Pp, Qq), coords, qd)
        del rx, coords
        op = fem.MassOperator(fem.Restriction(ne, Pp**d, nc, N, nc * N, offs), fem.Basis(d, nc, Pp, Qq), qd,
                              fem.QF.apply_mass_vector)
        del qd
        ops.append(op)
        g = torch.Generator(device=dev).manual_seed(SEED * 1000 + i)
        us.append(torch.rand(nc * N, dtype=torch.float64, device=dev, generator=g) * 2 - 1)
        dofs += nc * N
        abytes64 += ne * (4 * Pp**d + 8 * Qq**d) + 16 * nc * N
        abytes32 += ne * (4 * Pp**d + 4 * Qq**d) + 8 * nc * N
    return specs, ops, us, dofs, abytes64, abytes32


def run_batch(args):
    import torch
    import fe_demo_cpp_b200 as fem
    from fe_demo_cpp_b200.build import build
    from fe_demo_cpp_b200.telemetry import ClockSampler

    build()
    dev = torch.device("cuda", 0)
    specs, ops, us, dofs, abytes64, abytes32 = make_batch_ops(args.batch_meshes, dev)
    torch.cuda.synchronize()
    peak, _ = measured_peaks()
    n3 = sum(1 for sp in specs if sp[0] == 3)
    cfg = {"meshes": len(specs), "meshes_3d": n3, "meshes_2d": len(specs) - n3, "dofs": dofs,
           "elements": int(sum(int(np.prod(sp[1])) for sp in specs)),
           "spec": "d in {2,3} 50/50, elements log-uniform in [4^d, 48^d] (cubic/square boxes), P uniform 2..6, "
                   "Q=P+1, num_comp uniform 1..3 (vector mass), seeded perturbation, u ~ U[-1,1]",
           "l2": "inputs larger than L2; no flush"}
    K = args.batch_steps
    sampler = ClockSampler(0).start()

    def timed(fn, steps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    results = []
    # per-operator loop (the unbatched path: one public apply per mesh)
    vs = [torch.empty_like(u) for u in us]

    def loop():
        for op, u, v in zip(ops, us, vs):
            op.apply(u, v)
    results.append(("fp64", "per-operator loop", timed(loop, max(2, K // 4)), None))
    for prec in ("fp64", "fp32"):
        uu = us if prec == "fp64" else [u.float() for u in us]
        vv = [torch.empty_like(u) for u in uu]
        b = fem.Batch(ops, prec)
        b.bind(uu, vv)
        # the per-class form: a zeroing kernel and one kernel per class
        b.set_mode("classes")
        results.append((prec, "per-class kernels launched directly", timed(lambda: b.apply(graph=False), K),
                        b.info()))
        b.autotune(reps=3)
        results.append((prec, "per-class kernels, one graph launch, autotuned", timed(lambda: b.apply(graph=True), K),
                        b.info()))
        # the one-launch form: a single persistent kernel for the whole batch
        b.set_mode("persistent")
        results.append((prec, "one persistent kernel launch", timed(lambda: b.apply(graph=False), K), b.info()))
        results.append((prec, "one persistent kernel launch, in a graph", timed(lambda: b.apply(graph=True), K),
                        b.info()))
        b.check()
        # auto: the faster of the two after autotuning
        b.set_mode("auto")
        b.autotune(reps=3)
        results.append((prec, "auto (autotuned choice), one graph launch", timed(lambda: b.apply(graph=True), K),
                        b.info()))
        if prec == "fp64":
            # parity guard: the batch result against each operator's own apply
            worst = 0.0
            for op, u, v in list(zip(ops, uu, vv))[:: max(1, len(ops) // 32)]:
                w = torch.empty_like(u)
                op.apply(u, w)
                worst = max(worst, float((v - w).abs().max() / w.abs().max()))
            assert worst <= 1e-13, worst
        del b, uu, vv
    clocks = sampler.stop()
    for prec, mode, ms, info in results:
        ab = abytes64 if prec == "fp64" else abytes32
        print(json.dumps({"batch": "mass_apply", "precision": prec, "mode": mode, "metric": "GDoF/s batched apply",
                          "value": dofs / (ms * 1e-3) / 1e9, "unit": "GDoF/s", "ms_per_step": ms, "steps": K,
                          "roofline": {"bound": "hbm", "achieved_gbs": ab / (ms * 1e-3) / 1e9, "peak_gbs": peak,
                                       "frac": ab / (ms * 1e-3) / 1e9 / peak, "algorithmic_bytes": ab},
                          "batch_info": info, "config": cfg, "clocks": clocks}), flush=True)
    return 0


# ---------------------------------------------------------------------------
# served mass solves: Poisson arrivals at swept rates; each request a 3D box
# with elements log-uniform in [8^3, 64^3], P uniform in 2..6, num_comp 1 or 3,
# f ~ U[-1,1], rtol 1e-10; admitted by a 120 GB device budget; mixed precision
# against the plain FP64 path (extra lines)
# ---------------------------------------------------------------------------
def serve_requests(n, seed):
    rng = np.random.default_rng([seed, 5])
    out = []
    for i in range(n):
        side = int(round(float(np.exp(rng.uniform(np.log(8), np.log(64))))))
        out.append(((side,) * 3, int(rng.integers(2, 7)), 1 if rng.random() < 0.5 else 3, 1000 + i))
    return out


def run_serve(args):
    import threading
    import torch
    import fe_demo_cpp_b200 as fem
    from fe_demo_cpp_b200.build import build
    from fe_demo_cpp_b200.telemetry import ClockSampler

    build()
    torch.cuda.set_device(0)
    rates = [float(r) for r in args.serve_rates.split(",")]
    reqs = serve_requests(args.serve_requests, SEED)
    budget = int(args.serve_budget_gb * (1 << 30))
    sampler = ClockSampler(0).start()
    lines = []
    for prec in ("fp32_ir", "fp64"):
        with fem.Server(slots=args.serve_slots, hbm_budget=budget) as srv:
            # warm-up: one request of each order and component count the stream
            # draws (kernels loaded on first use, kernel attributes, pool)
            for Pw in range(2, 7):
                for ncw in (1, 3):
                    srv.wait(srv.submit_box(3, (8, 8, 8), Pw, num_comp=ncw, seed=1, precision=prec))
            for rate in rates:
                rng = np.random.default_rng([SEED, int(rate)])
                gaps = rng.exponential(1.0 / rate, len(reqs))
                ids = [None] * len(reqs)

                def client():
                    t = time.perf_counter()
                    for k, (shape, Pp, nc, seed) in enumerate(reqs):
                        t += gaps[k]
                        delay = t - time.perf_counter()
                        if delay > 0:
                            time.sleep(delay)
                        ids[k] = srv.submit_box(3, shape, Pp, num_comp=nc, seed=seed, rtol=1e-10, precision=prec)
                th = threading.Thread(target=client)
                th.start()
                res = []
                for k in range(len(reqs)):
                    while ids[k] is None:
                        time.sleep(0.0005)
                    res.append(srv.wait(ids[k]))
                th.join()
                st = srv.stats()
                bad = [r for r in res if r["status"] != 0]
                assert not bad, bad[0]["message"]
                lat = sorted((r["t_end"] - r["t_submit"]) * 1e3 for r in res)
                span = max(r["t_end"] for r in res) - min(r["t_submit"] for r in res)
                lines.append({
                    "serve": "mass_solve", "precision": prec, "rate_rps": rate, "requests": len(res),
                    "metric": "solves/s", "value": len(res) / span, "unit": "solves/s",
                    "p50_ms": lat[len(lat) // 2], "p99_ms": lat[min(len(lat) - 1, int(round(0.99 * (len(lat) - 1))))],
                    "mean_queue_ms": float(np.mean([(r["t_start"] - r["t_submit"]) * 1e3 for r in res])),
                    "mean_service_ms": float(np.mean([(r["t_end"] - r["t_start"]) * 1e3 for r in res])),
                    "gdofs_solved_per_s": sum(r["dofs"] for r in res) / span / 1e9,
                    "mean_dofs": float(np.mean([r["dofs"] for r in res])),
                    "mean_iterations": float(np.mean([r["iterations"] for r in res])),
                    "max_rel_residual": max(r["rel_residual"] for r in res),
                    "bytes_peak": st["bytes_peak"],
                    "config": {"slots": args.serve_slots, "budget_bytes": budget,
                               "requests": "3D boxes, elements log-uniform in [8^3, 64^3] (cubes), P uniform 2..6, "
                                           "Q=P+1, num_comp 1 or 3, f ~ U[-1,1], rtol 1e-10, Poisson arrivals",
                               "mesh": "generated on the device per request; set-up (mesh, qdata, plan) inside "
                                       "each request's latency"}})
                print(json.dumps(lines[-1]), flush=True)
    clocks = sampler.stop()
    print(json.dumps({"serve": "clocks", "clocks": clocks}), flush=True)
    return 0


# ---------------------------------------------------------------------------
# the restriction stages against the reference's own CUDA kernels
# (src/cuda/cuda-elem-restriction.cu built for sm_100a, oracle/_ref) on the
# bench mesh: gather, atomic and deterministic scatter (extra lines)
# ---------------------------------------------------------------------------
def run_restriction(args):
    import torch
    import fe_demo_cpp_b200 as fem
    import oracle
    from fe_demo_cpp_b200.build import build
    from fe_demo_cpp_b200.mesh import box_mesh

    build()
    if not oracle.refcuda_available():
        print(json.dumps({"restriction": "reference-cuda", "unavailable": "oracle/_ref/libfemrefcuda.so not built"}))
        return 0
    dev = torch.device("cuda", 0)
    mesh = box_mesh(SHAPE, P, seed=SEED)
    N, ne, es = mesh.num_nodes, mesh.num_elem, P**3
    n_e = ne * es
    peak, _ = measured_peaks()
    rng = np.random.default_rng([SEED, 9])
    l_host = rng.uniform(-1, 1, N)
    e_host = rng.uniform(-1, 1, n_e)
    K = args.restriction_steps
    results = {}

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(K):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / K

    # algorithmic bytes: offsets, the L-vector once, the E-vector once (scatter: L read + written)
    bytes_gather = 4 * n_e + 8 * N + 8 * n_e
    bytes_scatter = 4 * n_e + 8 * n_e + 16 * N
    l_dev = torch.from_numpy(l_host).to(dev)
    e_dev = torch.from_numpy(e_host).to(dev)
    for det in (False, True):
        ours = fem.Restriction(ne, es, 1, N, N, mesh.offsets, 1 if det else 0)
        ref = oracle.RefCudaRestriction(ne, es, 1, N, N, mesh.offsets, det)
        ref.set_l(l_host)
        ref.set_e(e_host)
        e_out = torch.empty(n_e, dtype=torch.float64, device=dev)
        l_out = torch.zeros(N, dtype=torch.float64, device=dev)
        if not det:
            results[("gather", "b200")] = timed(lambda: ours.apply(0, l_dev, e_out))
            results[("gather", "reference-cuda")] = timed(lambda: ref.apply(False))
            assert np.array_equal(e_out.cpu().numpy(), ref.get_e())  # parity guard
        mode = "scatter_deterministic" if det else "scatter_atomic"
        results[(mode, "b200")] = timed(lambda: ours.apply(1, e_dev, l_out))
        results[(mode, "reference-cuda")] = timed(lambda: ref.apply(True))
        ref.close()
        del ours, e_out, l_out
    del l_dev, e_dev
    # the fused operator apply with each scatter (zero v + kernel [+ the
    # deterministic E-vector reduction]): the deterministic mode's cost
    x = torch.from_numpy(mesh.coords).to(dev)
    qd = torch.empty(Q**3 * ne, dtype=torch.float64, device=dev)
    fem.mass_build(fem.Restriction(ne, es, 3, N, 3 * N, mesh.offsets), fem.Basis(3, 3, P, Q), x, qd)
    del x
    u = torch.from_numpy(l_host).to(dev)
    v = torch.empty_like(u)
    apply_ms = {}
    for det in (0, 1):
        op = fem.MassOperator(fem.Restriction(ne, es, 1, N, N, mesh.offsets, det), fem.Basis(3, 1, P, Q), qd)
        apply_ms[det] = timed(lambda: op.apply(u, v))
        del op
    print(json.dumps({"apply": "mass", "scatter_atomic_ms": apply_ms[0], "scatter_deterministic_ms": apply_ms[1],
                      "deterministic_over_atomic": apply_ms[1] / apply_ms[0],
                      "config": {"mesh": "x".join(map(str, SHAPE)), "P": P, "Q": Q, "num_comp": 1, "dofs": N,
                                 "note": "public apply: v zeroed + fused kernel (+ E-vector transpose-map "
                                         "reduction in the deterministic mode)"}}), flush=True)
    for (mode, impl), ms in results.items():
        ab = bytes_gather if mode == "gather" else bytes_scatter
        other = results[(mode, "reference-cuda" if impl == "b200" else "b200")]
        print(json.dumps({"restriction": mode, "impl": impl, "ms": ms, "algorithmic_bytes": ab,
                          "achieved_gbs": ab / (ms * 1e-3) / 1e9, "roofline_frac": ab / (ms * 1e-3) / 1e9 / peak,
                          "speedup_vs_other": other / ms,
                          "config": {"mesh": "x".join(map(str, SHAPE)), "P": P, "num_comp": 1, "dofs": N,
                                     "e_size": n_e}}), flush=True)
    return 0


# ---------------------------------------------------------------------------
# end-to-end (host vectors) apply: the PCIe ceilings and the copy pipeline's
# chunk count, on the bench workload (extra lines)
# ---------------------------------------------------------------------------
# ---------------------------------------------------------------------------
# one mesh over the ranks (--split): the 100^3 P=5 mesh split into contiguous
# element ranges (fem_b200_shard_*), each rank applying its elements, then one
# interface exchange per apply: device pack, NCCL send/recv of the shared
# values only, rank-ordered unpack-add (extra line; strong scaling: the mesh
# is fixed as N grows)
# ---------------------------------------------------------------------------
def run_split(args, rank, world, local_rank):
    import torch
    import fe_demo_cpp_b200 as fem
    from fe_demo_cpp_b200.build import build
    from fe_demo_cpp_b200.mesh import box_mesh

    build()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    mesh = box_mesh(SHAPE, P, seed=SEED)
    N = mesh.num_nodes
    plan = fem.ShardPlan(mesh.offsets, P**3, world, rank)
    n = plan.num_nodes
    coords = np.concatenate([mesh.coords[k * N + plan.l2g] for k in range(3)])
    rx = fem.Restriction(plan.num_elem, P**3, 3, n, 3 * n, plan.offsets)
    qd = torch.empty(Q**3 * plan.num_elem, dtype=torch.float64, device=dev)
    fem.mass_build(rx, fem.Basis(3, 3, P, Q), torch.from_numpy(coords).to(dev), qd)
    op = fem.MassOperator(fem.Restriction(plan.num_elem, P**3, 1, n, n, plan.offsets), fem.Basis(3, 1, P, Q), qd)
    del rx, coords
    g = torch.Generator(device=dev).manual_seed(SEED)
    u = torch.rand(n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    v = torch.empty_like(u)
    send = torch.empty(max(1, plan.shared_total), dtype=torch.float64, device=dev)
    recv = torch.empty_like(send)
    segs, s0 = [], 0
    for q, idx in plan.peers:
        segs.append((q, s0, len(idx)))
        s0 += len(idx)

    def exchange():
        if not segs:
            return
        plan.pack(v, send[:plan.shared_total])
        ops = []
        for q, a, c in segs:
            ops.append(dist.P2POp(dist.isend, send[a:a + c], q))
            ops.append(dist.P2POp(dist.irecv, recv[a:a + c], q))
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        plan.unpack_add(recv[:plan.shared_total], v)

    stream = torch.cuda.current_stream()
    for _ in range(max(3, args.warmup)):
        op.apply(u, v)
        exchange()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    K = args.steps
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3 * K)]
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for i in range(K):
        e[3 * i].record(stream)
        op.apply(u, v)
        e[3 * i + 1].record(stream)
        exchange()
        e[3 * i + 2].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    wall = (time.perf_counter() - t0) / K * 1e3
    apply_ms = sum(e[3 * i].elapsed_time(e[3 * i + 1]) for i in range(K)) / K
    exch_ms = sum(e[3 * i + 1].elapsed_time(e[3 * i + 2]) for i in range(K)) / K
    step_ms = apply_ms + exch_ms
    t = torch.tensor([step_ms, apply_ms, exch_ms, wall], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    step_ms, apply_max, exch_max, wall = t.tolist()
    xbytes = torch.tensor([8.0 * plan.shared_total], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(xbytes)
    line = {"split": "mass_apply", "metric": "GDoF/s operator_apply, one mesh over the ranks",
            "value": N / (step_ms * 1e-3) / 1e9, "unit": "GDoF/s", "n_gpus": world, "steps": K,
            "ms_per_step": step_ms, "scaling": "strong", "higher_is_better": True,
            "per_rank_max": {"apply_ms": apply_max, "exchange_ms": exch_max, "wall_ms": wall},
            "exchange_bytes_per_step_all_ranks": xbytes.item(),
            "config": {"workload": WORKLOAD, "mesh": "x".join(map(str, SHAPE)), "P": P, "Q": Q, "dofs": N,
                       "partition": "contiguous element ranges (fem_b200_shard_*)",
                       "exchange": "device pack, NCCL batch_isend_irecv of the shared values, rank-ordered "
                                   "unpack-add (same bits on every rank)"}}
    return line


def run_e2e_sweep(args):
    import torch
    import fe_demo_cpp_b200 as fem
    from fe_demo_cpp_b200.build import build
    from fe_demo_cpp_b200.mesh import box_mesh

    build()
    dev = torch.device("cuda", 0)
    mesh = box_mesh(SHAPE, P, seed=SEED)
    N, ne = mesh.num_nodes, mesh.num_elem
    rx = fem.Restriction(ne, P**3, 3, N, 3 * N, mesh.offsets)
    qdata = torch.empty(Q**3 * ne, dtype=torch.float64, device=dev)
    fem.mass_build(rx, fem.Basis(3, 3, P, Q), torch.from_numpy(mesh.coords).to(dev), qdata)
    op = fem.MassOperator(fem.Restriction(ne, P**3, 1, N, N, mesh.offsets), fem.Basis(3, 1, P, Q), qdata)
    del rx
    gen = torch.Generator(device=dev).manual_seed(SEED)
    u = torch.rand(N, dtype=torch.float64, device=dev, generator=gen) * 2 - 1
    v = torch.empty_like(u)
    op.autotune(u, v, reps=5)
    u_h = u.cpu().pin_memory()
    v_h = torch.empty(N, dtype=torch.float64).pin_memory()
    nbytes = 8 * N
    reps = args.e2e_steps

    # the link: u in alone, v out alone, both at once (page-locked, one copy each)
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    cur = torch.cuda.current_stream()

    def copies(do_in, do_out):
        s_in.wait_stream(cur)
        s_out.wait_stream(cur)
        if do_in:
            with torch.cuda.stream(s_in):
                u.copy_(u_h, non_blocking=True)
        if do_out:
            with torch.cuda.stream(s_out):
                v_h.copy_(v, non_blocking=True)
        cur.wait_stream(s_in)
        cur.wait_stream(s_out)

    def device_ms(fn):
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

    link = {"in_ms": device_ms(lambda: copies(True, False)), "out_ms": device_ms(lambda: copies(False, True)),
            "both_ms": device_ms(lambda: copies(True, True))}
    link.update({"in_gbs": nbytes / link["in_ms"] / 1e6, "out_gbs": nbytes / link["out_ms"] / 1e6,
                 "both_gbs_each": nbytes / link["both_ms"] / 1e6})
    cfg = {"mesh": "x".join(map(str, SHAPE)), "P": P, "Q": Q, "dofs": N, "bytes_each_way": nbytes}
    print(json.dumps({"e2e": "pcie", **link, "config": cfg}), flush=True)

    want = None
    u_np, v_np = u_h.numpy(), v_h.numpy()
    for pinned in (True, False):
        uu, vv = (u_np, v_np) if pinned else (u_np.copy(), np.empty(N))
        for chunks in ((1, 8, 16, 24, 32, 64) if pinned else (1, 0)):
            op.set_host_chunks(chunks)
            for _ in range(2):
                op.apply_host(uu, vv)
            ts = []
            for _ in range(reps):
                t0 = time.perf_counter()
                op.apply_host(uu, vv)
                ts.append(time.perf_counter() - t0)
            if want is None:
                want = vv.copy()
            assert np.abs(vv - want).max() <= 1e-13 * np.abs(want).max()  # parity guard
            t = statistics.median(ts)
            print(json.dumps({"e2e": "apply_host", "host_memory": "page-locked" if pinned else "pageable",
                              "chunks": chunks or "default", "ms": t * 1e3, "gdofs": N / t / 1e9,
                              "vs_both_directions_at_once": link["both_ms"] / (t * 1e3), "config": cfg}),
                  flush=True)
    op.set_host_chunks(0)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-orders", action="store_true", help="skip the P = 2..4 roofline fractions")
    ap.add_argument("--split", action="store_true",
                    help="one mesh over the ranks: element ranges, interface exchange over NCCL (extra line)")
    ap.add_argument("--orders-steps", type=int, default=20)
    ap.add_argument("--cpu-sample-s", type=float, default=12.0, help="approximate CPU seconds of the baseline")
    ap.add_argument("--shape", default=None, help="elements per direction nx,ny,nz (default 100,100,100)")
    ap.add_argument("--P", type=int, default=None, help="nodes per direction (Q = P+1)")
    ap.add_argument("--kernel", choices=["auto", "simple", "pipelined", "paired", "prefetch", "occupancy", "narrow", "element"], default="auto")
    ap.add_argument("--sweep", action="store_true", help="order sweep P=2..8, num_comp 1 and 3 (extra lines)")
    ap.add_argument("--sweep-P", default="2,3,4,5,6,7,8")
    ap.add_argument("--sweep-dim", default="3", help="dimensions of the order sweep, e.g. 2,3")
    ap.add_argument("--sweep-steps", type=int, default=20)
    ap.add_argument("--sweep-dofs", type=int, default=64_000_000, help="DoFs of each sweep mesh")
    ap.add_argument("--sweep-storage-only", action="store_true",
                    help="sweep only the reduced-storage and tensor-core applies (no FP64 variants, no basis)")
    ap.add_argument("--solve", action="store_true", help="mixed-precision mass solve, FP64 vs FP32+IR (extra lines)")
    ap.add_argument("--solve-shape", default="64,64,64")
    ap.add_argument("--solve-P", type=int, default=5)
    ap.add_argument("--solve-rtol", type=float, default=1e-10)
    ap.add_argument("--solve-steps", type=int, default=20)
    ap.add_argument("--solve-scatter", type=int, default=0, help="0 atomic, 1 deterministic")
    ap.add_argument("--batch", action="store_true", help="512 uneven meshes in one graph, FP64 and FP32 (extra lines)")
    ap.add_argument("--batch-meshes", type=int, default=512)
    ap.add_argument("--batch-steps", type=int, default=20)
    ap.add_argument("--serve", action="store_true", help="served solve stream at swept Poisson rates (extra lines)")
    ap.add_argument("--serve-rates", default="50,200,1000,2000")
    ap.add_argument("--serve-requests", type=int, default=64)
    ap.add_argument("--serve-slots", type=int, default=8)
    ap.add_argument("--serve-budget-gb", type=float, default=120.0)
    ap.add_argument("--restriction", action="store_true",
                    help="restriction stages vs the reference's CUDA kernels (extra lines)")
    ap.add_argument("--restriction-steps", type=int, default=20)
    ap.add_argument("--e2e-sweep", action="store_true",
                    help="host-vector apply: PCIe ceilings and copy-pipeline chunk counts (extra lines)")
    ap.add_argument("--e2e-steps", type=int, default=10)
    args = ap.parse_args()
    if args.e2e_sweep:
        return run_e2e_sweep(args)
    if args.restriction:
        return run_restriction(args)
    if args.serve:
        return run_serve(args)
    if args.batch:
        return run_batch(args)
    if args.sweep:
        return run_sweep(args)
    if args.solve:
        return run_solve(args)
    global SHAPE, P, Q, WORKLOAD
    if args.shape or args.P:
        SHAPE = tuple(int(s) for s in args.shape.split(",")) if args.shape else SHAPE
        P = args.P or P
        Q = P + 1
        WORKLOAD = (f"mass operator_apply, FP64 3D hex box {'x'.join(map(str, SHAPE))} elements (perturbed, "
                    f"seed 1), P={P}, Q={Q}, num_comp=1 (non-default size)")
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        line = run_reference(args, rank)
        if rank == 0:
            print(json.dumps(line), flush=True)
        return 0
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    line = run_split(args, rank, world, local_rank) if args.split else run_b200(args, rank, world, local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
