"""Benchmark of the XaNSoNS histogram hot path on B200.

Workload (one "step"): the DebyePDF scenario of calcPDFandDebye on a seeded synthetic rock-salt
nanocube -- 30^3 unit cells, a = 5.64 A, 10 % vacancies, Gaussian displacement 0.07 A (~1.94e5 atoms,
two species with neutron lengths 3.63 / 9.58 fm): the per-element-pair u64 pair-distance histogram at
0.001 A bins (bit-identical to the reference), the rPDF on those bins, and I(q) on 4096 q points in
[0.1, 25) A^-1.  Metric: atom pairs per second (N(N-1)/2 pairs per step).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Ours: `value` times the device-resident path (xns_pdf_and_debye_device: coordinates already in HBM),
`e2e` the host-buffer C-ABI call (xns_calc_pdf_and_debye) from pinned host memory, H2D and D2H inside
the timed region.  L2 (126 MB) is flushed by writing a 512 MB buffer before every timed step (the
inputs, 4.7 MB, would otherwise stay L2-resident).  With N ranks each rank computes its own structure
(seed = rank): weak scaling, no collective on the data path; the time is the max over ranks.

Reference: the reference's own CPU calc functions (CalcFunctions.cpp compiled from its sources into
oracle/_ref/libxnsref.so; the FP64 oracle port if that build is absent) on all host cores, on a bounded
sample of the same workload (a smaller cube of the same lattice), rank 0 only.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "softx-d-16-00083_b200"))

METRIC = "atom-pairs/s"
CELLS, A, VAC, SIGMA = 30, 5.64, 0.1, 0.07
BIN, NQ, QMIN, QMAX = 0.001, 4096, 0.1, 25.0
SL = [3.63, 9.58]
HIST_FLOPS_PER_PAIR = 10  # the reference's per-pair FP64 arithmetic: 3 sub, 3 mul, 2 add, sqrt, divide
# DRAM bytes (read + write) of one hist_window_kernel launch on the 30^3-cell cube, from an ncu capture
# of this benchmark (dram__bytes_read.sum + dram__bytes_write.sum); re-measure when the kernel changes
HIST_TRAFFIC_30 = 108_363_520 + 4_282_112  # bytes per hist_window_kernel launch, rock-salt 30^3 cube (ncu, 1 pass)


def workload(seed, cells=CELLS):
    from xns_b200 import synth
    els = synth.rocksalt_cube(cells=cells, a=A, vacancy=VAC, sigma=SIGMA, seed=seed)
    nh = synth.hist_size(els, BIN)
    q = synth.q_mesh(QMIN, QMAX, NQ)
    p0 = atomic_density(els)
    return els, nh, q, p0


def atomic_density(els):
    """GetAtomicDensity (CalcFunctions.cpp:204-223) restated in numpy: atoms within a third of the
    ensemble size of the centre, divided by that sphere's volume."""
    xyz = np.concatenate(els)
    c = xyz.mean(axis=0)
    d2 = ((xyz - c) ** 2).sum(axis=1)
    r2 = (0.33333 * 2 * np.sqrt(d2.max())) ** 2
    return float((d2 < r2).sum() / (4 / 3 * np.pi * np.sqrt(r2) ** 3))


def npairs(els):
    n = sum(len(e) for e in els)
    return n * (n - 1) // 2


def config_block(els, nh, cells=CELLS):
    """The workload's description, the same dict in both arms (seed 0)."""
    return {"workload": "DebyePDF rock-salt nanocube %d^3 cells a=%.2f A, %d atoms, hist bin %.3f A (%d bins x 3 pairs), "
                        "rPDF, I(q) %d q in [%.1f,%.1f)" % (cells, A, sum(len(e) for e in els), BIN, nh, NQ, QMIN, QMAX),
            "atoms": int(sum(len(e) for e in els)), "pairs_per_step": int(npairs(els)), "nhist": int(nh), "nq": NQ,
            "seed": 0, "l2": "flushed (512 MB write) before every timed step"}


def hist_sha256(h):
    """SHA-256 of u64 counts (little-endian): both arms print it for the full-size histogram."""
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(h, dtype="<u8").tobytes()).hexdigest()


# ---- ranks ------------------------------------------------------------------------------------------
def rank_max(x, device=None):
    """The largest x over the ranks of the default process group (x itself without one): every rank
    reports the slowest rank's time, so the whole job's rate is the units all ranks processed divided by
    it."""
    import torch
    import torch.distributed as tdist
    if not (tdist.is_available() and tdist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, units_per_rank, ms_max):
    """Whole-job throughput of weak-scaling replicas: world ranks of units_per_rank each, in the slowest
    rank's time."""
    return world * units_per_rank / (ms_max * 1e-3)


# ---- clocks -----------------------------------------------------------------------------------------
class Clocks:
    """SM clock and throttle reasons during a timed region: NVML polled every 10 ms from a thread (the
    CUDA device found by its PCI address), else nvidia-smi -lms 200 in a child process."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    # NVML clocks-event reason bits (nvml.h nvmlClocksEventReason*)
    REASON_BITS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
                   ("sw_power_cap", 0x4))
    PERIOD_S = 0.01

    def __init__(self, device, pci_bus_id=None):
        self.device = device
        self.pci_bus_id = pci_bus_id
        self.proc = None
        self.path = None
        self.nvml = None
        self.thread = None
        self.out = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        bus = self.pci_bus_id
        if bus is None:
            try:
                import torch
                if not torch.cuda.is_initialized():  # never the first CUDA call of a process (workers may fork)
                    raise RuntimeError("CUDA not initialised")
                pr = torch.cuda.get_device_properties(self.device)
                bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            except Exception:
                bus = None
        h = None
        if bus is not None:
            try:
                h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                h = None
        if h is None:
            h = pynvml.nvmlDeviceGetHandleByIndex(self.device)
        return pynvml, h

    def _poll(self, nv, h, stop, rows):
        reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while True:
            try:
                rows.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), int(reasons(h))))
            except Exception:
                pass
            if stop.wait(self.PERIOD_S):
                return

    def start(self):
        """Starts both samplers; stop() reports NVML's when it took samples, else nvidia-smi's."""
        try:
            import threading
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.nvml = (nv, h, threading.Event(), [])
            self.thread = threading.Thread(target=self._poll, args=self.nvml, daemon=True)
            self.thread.start()
        except Exception:
            self.nvml = None
            self.thread = None
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            if self.out is not None:
                self.out.close()
            if self.path is not None:
                os.unlink(self.path)

    def stop(self):
        if self.nvml is not None:
            self.nvml[2].set()
            self.thread.join()
        smi = self._stop_smi()
        if self.nvml is not None:
            nv, h, stop, rows = self.nvml
            try:
                nv.nvmlShutdown()
            except Exception:
                pass
            if rows:
                reasons = sorted({n for _, r in rows for n, bit in self.REASON_BITS if r & bit})
                return {"sm_mhz": float(np.median([c for c, _ in rows])), "sm_max_mhz": self.max_mhz,
                        "reasons": reasons, "samples": len(rows), "source": "nvml, 10 ms",
                        "nvidia_smi": smi}
        return smi

    def _stop_smi(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.out.close()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "source": "nvidia-smi, 200 ms"}


# ---- CPU baseline ---------------------------------------------------------------------------------
def cpu_reference_sample(target_s=12.0, max_cells=CELLS):
    """Times the reference's calcPDFandDebye (DebyePDF, rPDF, the same bin and q mesh) on the seed-0
    cube, grown from 6^3 cells until one pass takes about target_s (the full 30^3 cells where the host
    is fast enough).  Returns (pairs/s, kind, cores, sample, (cells, seconds))."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    cores = os.cpu_count() or 1
    try:
        R = orc.Reference(threads=cores)
        kind, O = "reference", None
    except FileNotFoundError:
        R, kind, O = None, "port", orc.Oracle()

    def run(cells):
        els, nh, q, p0 = workload(0, cells)
        t = time.perf_counter()
        if R is not None:
            R.pdf_and_debye(els, nh, BIN, 4, 2, p0, q, 0, sl=SL)
        else:
            h = O.hist(els, nh, BIN)
            O.pdf(h, [len(e) for e in els], nh, BIN, 2, p0, SL)
            O.int_1d_hist(h, [len(e) for e in els], nh, BIN, q, 0, sl=SL)
        return time.perf_counter() - t, els

    cells = min(6, max_cells)
    dt, els = run(cells)
    while dt < target_s / 4 and cells < max_cells:
        # pairs grow as cells^6, the transform as cells: step the size by the measured time
        grow = min(max((target_s / max(dt, 1e-3)) ** (1 / 6), 1.15), 1.8)
        cells = min(max_cells, max(cells + 1, int(cells * grow)))
        dt, els = run(cells)
    pairs = npairs(els)
    sample = ("one calcPDFandDebye pass (histogram + rPDF + I(q), %d q) on the seed-0 cube of %d^3 cells, %d atoms, "
              "%.3g pairs, %.2f s" % (NQ, cells, sum(len(e) for e in els), pairs, dt))
    return pairs / dt, kind, cores, sample, (cells, dt)


# ---- reference arm --------------------------------------------------------------------------------
def reference_arm(args, rank, world):
    if rank != 0:
        return 0
    v, kind, cores, sample, (cells, dt0) = cpu_reference_sample(max_cells=args.cells)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    els, nh, q, p0 = workload(0, cells)
    if kind == "reference":
        R = orc.Reference(threads=cores)
        step = lambda: R.pdf_and_debye(els, nh, BIN, 4, 2, p0, q, 0, sl=SL)  # noqa: E731
    else:
        O = orc.Oracle()

        def step():
            h = O.hist(els, nh, BIN)
            O.pdf(h, [len(e) for e in els], nh, BIN, 2, p0, SL)
            O.int_1d_hist(h, [len(e) for e in els], nh, BIN, q, 0, sl=SL)
    for _ in range(args.warmup):
        step()
    t = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t) / args.steps
    value = npairs(els) / dt
    full, nh_full = workload(0, args.cells)[:2]
    sample = sample if cells == args.cells else sample + " (a bounded sample of the full cube)"
    line = {"metric": METRIC, "value": value, "unit": "pairs/s", "impl": "reference", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": config_block(full, nh_full, args.cells),
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    # the reference's histogram of the full cube (calcHist, untimed), hashed: our line prints the hash of
    # ours for the same cube
    R = orc.Reference(threads=cores) if kind == "reference" else orc.Oracle()
    line["histogram_sha256"] = hist_sha256(R.hist(full, nh_full, BIN))
    line["histogram_sha256_of"] = ("calcHist of the reference on the full %d-atom cube" % sum(len(e) for e in full)
                                   if kind == "reference" else "the oracle port's histogram of the full cube")
    print(json.dumps(line))
    return 0


def reference_workload_arm(args, rank):
    """--impl reference for the one-GPU workloads: the reference's own CPU code for that workload's
    path (oracle/_ref, else the oracle port) on a bounded sample of the workload, all host cores where
    the reference is parallel; metric and unit of our line for that workload."""
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "softx-d-16-00083_b200"))
    import oracle as orc
    from xns_b200 import synth
    cores = os.cpu_count() or 1
    try:
        R, kind = orc.Reference(threads=cores), "reference"
    except FileNotFoundError:
        R, kind = orc.Oracle(), "port"
    w = args.workload
    if w == "debye":
        els = synth.fcc_sphere(n=5000, a=4.078, sigma=0.05, seed=0)
        q = synth.q_mesh(0.1, 10.0, 1024)
        m = 1500
        sub = [els[0][:m]]
        units = m * (m - 1) // 2
        step = lambda: R.int_debye(sub, q, 0, sl=[7.63])  # noqa: E731
        metric, unit = "atom-pairs/s", "pairs/s"
        sample = "calcIntDebye on the first %d atoms of the 5000-atom sphere, 1024 q, %d threads" % (m, cores)
    elif w == "2d":
        els = synth.fcc_crystallite(cells=args.cells2d, a=3.61, subst=0.05, seed=0)
        n = sum(len(e) for e in els)
        q = synth.q_mesh(0.05, 8.0, args.mesh2d)
        ff = synth.ff_on_mesh(synth.ff_coefficients(2, seed=3), q)
        rows, nfi = cores, 64
        units = n * rows * nfi
        step = lambda: R.int_2d(els, q[:rows], nfi, [0, 0, 0], [0, 0, 0], [1, 1, 1], 5, 0.01, 1,  # noqa: E731
                                ff=ff[:, :rows])
        metric, unit = "terms/s", "(atom, q-point) terms/s"
        sample = "calcInt2D on %d q rows x %d phi, all %d atoms, %d threads" % (rows, nfi, n, cores)
    elif w == "batch":
        structs, ns, _ = synth.sphere_ensemble(count=args.batch_count, seed=0)
        small = [s for s, n in zip(structs, ns) if n < 6000][:4]
        q = synth.q_mesh(0.1, 25.0, 4096)

        def step():
            for st in small:
                nh = synth.hist_size(st, 0.001)
                R.pdf_and_debye(st, nh, 0.001, 2, 2, 0.0, q, 0, sl=[7.63])
        units = len(small)
        metric, unit = "patterns/s", "patterns/s"
        sample = ("calcPDFandDebye (Debye_hist) on the %d smallest-index spheres under 6000 atoms of the ensemble "
                  "(%s atoms), 4096 q, %d threads" % (len(small), ",".join(str(sum(len(e) for e in st)) for st in small),
                                                      cores))
    elif w == "build":
        m = 20000
        blk = synth.atom_file_block(m)
        units = m * (m - 1) // 2
        step = (lambda: R.calc_atoms([blk], 2)) if kind == "reference" else (lambda: R.build_atoms([blk], 2, 1))
        metric, unit, cores = "site pairs/s (structure build)", "pairs/s", 1
        sample = "block::calcAtoms on an atom-list block of %d sites (single-threaded in the reference)" % m
    elif w == "learned":
        print(json.dumps({"impl": "reference", "unavailable": "the learned binning correction has no counterpart in the "
                          "reference; its exact path, calcIntDebye, is timed by --workload debye"}))
        return 0
    else:
        raise ValueError(w)
    for _ in range(args.warmup):
        step()
    t = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t) / args.steps
    value = units / dt
    line = {"metric": metric, "value": value, "unit": unit, "impl": "reference", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": w, "sample": sample},
            "cpu_baseline": {"value": value, "unit": unit, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---- our arm --------------------------------------------------------------------------------------
def ours(args, rank, world, local_rank):
    import ctypes as C

    import torch
    import xns_b200
    from xns_b200 import lib

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ctx = xns_b200.Context(local_rank)
    stream = torch.cuda.current_stream(dev)
    ctx.set_stream(stream.cuda_stream)

    # replicas: one structure per rank (seeded by the rank); --shard: one structure split over the ranks
    els, nh, q, p0 = workload(0 if args.shard else rank, args.cells)
    n_el = np.array([len(e) for e in els], dtype=np.uint32)
    P = 3
    pairs = npairs(els)
    sl = np.array(SL)
    xyz = np.ascontiguousarray(np.concatenate(els))
    d_xyz = torch.from_numpy(xyz).to(dev)
    d_hist = torch.zeros(P * nh, dtype=torch.int64, device=dev)
    d_I = torch.zeros(NQ, dtype=torch.float64, device=dev)
    d_pdf = torch.zeros((1 + P) * nh, dtype=torch.float64, device=dev)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    p = C.c_void_p

    def step_device():
        if args.shard:
            from xns_b200 import shard
            shard.pdf_and_debye(ctx, d_xyz, n_el, nh, BIN, 4, 2, p0, q, 0, sl, d_hist, d_I, d_pdf, rank, world)
            return
        st = lib.xns_pdf_and_debye_device(ctx.handle, p(d_xyz.data_ptr()), n_el.ctypes.data_as(p), len(n_el), nh, BIN, 4, 2,
                                          p0, q.ctypes.data_as(p), NQ, 0, None, sl.ctypes.data_as(p), 0, 0.0,
                                          p(d_I.data_ptr()), p(d_pdf.data_ptr()), p(d_hist.data_ptr()))
        if st:
            raise xns_b200.XnsError(st, lib.xns_last_error(ctx.handle).decode())

    lib.xns_pdf_and_debye_device.argtypes = [p, p, p, C.c_uint32, C.c_uint32, C.c_double, C.c_int, C.c_int, C.c_double, p,
                                             C.c_uint32, C.c_int, p, p, C.c_int, C.c_double, p, p, p]
    lib.xns_last_stage_ms.argtypes = [p, C.c_int]
    lib.xns_last_stage_ms.restype = C.c_double
    lib.xns_measure_fma_peak.argtypes = [p, C.c_int, C.POINTER(C.c_double)]

    dist = world > 1
    if dist:
        import torch.distributed as tdist

    def barrier():
        if dist:
            tdist.barrier()

    # warm-up
    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()

    clocks = Clocks(local_rank)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = ctx.kernel_launches
    total_ms, hist_ms, iq_ms, pdf_ms = 0.0, 0.0, 0.0, 0.0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(args.steps):
        flush.fill_(1.0)
        ev0.record(stream)
        step_device()
        ev1.record(stream)
        ev1.synchronize()
        total_ms += ev0.elapsed_time(ev1)
        hist_ms += lib.xns_last_stage_ms(ctx.handle, 0)
        pdf_ms += lib.xns_last_stage_ms(ctx.handle, 1)
        iq_ms += lib.xns_last_stage_ms(ctx.handle, 2)
    torch.cuda.synchronize()
    barrier()
    launches = ctx.kernel_launches - launches0
    clk = clocks.stop()
    ms_step = rank_max(total_ms / args.steps, dev)

    # end-to-end through the host-buffer C ABI from pinned host memory
    pin_xyz = [torch.from_numpy(np.ascontiguousarray(e)).pin_memory() for e in els]
    table = (C.c_void_p * len(els))(*[t.data_ptr() for t in pin_xyz])
    pin_I = torch.zeros(NQ, dtype=torch.float64).pin_memory()
    pin_pdf = torch.zeros((1 + P) * nh, dtype=torch.float64).pin_memory()
    lib.xns_calc_pdf_and_debye.argtypes = [p, p, p, C.c_uint32, C.c_uint32, C.c_double, C.c_int, C.c_int, C.c_double, p,
                                           C.c_uint32, C.c_int, p, p, C.c_int, C.c_double, p, p, p]

    pin_all = torch.from_numpy(xyz).pin_memory()

    def step_e2e():
        if args.shard:  # host coordinates in, the whole I(q) and PDF out on every rank
            d_xyz.copy_(pin_all, non_blocking=True)
            step_device()
            pin_I.copy_(d_I, non_blocking=True)
            pin_pdf.copy_(d_pdf, non_blocking=True)
            return
        st = lib.xns_calc_pdf_and_debye(ctx.handle, table, n_el.ctypes.data_as(p), len(n_el), nh, BIN, 4, 2, p0,
                                        q.ctypes.data_as(p), NQ, 0, None, sl.ctypes.data_as(p), 0, 0.0,
                                        p(pin_I.data_ptr()), p(pin_pdf.data_ptr()), None)
        if st:
            raise xns_b200.XnsError(st, lib.xns_last_error(ctx.handle).decode())

    for _ in range(max(1, args.warmup // 2)):
        step_e2e()
    e2e_ms = 0.0
    barrier()
    for _ in range(args.steps):
        flush.fill_(1.0)
        ev0.record(stream)
        step_e2e()
        ev1.record(stream)
        ev1.synchronize()
        e2e_ms += ev0.elapsed_time(ev1)
    e2e_ms = rank_max(e2e_ms / args.steps, dev)
    h2d = int(xyz.nbytes + q.nbytes + sl.nbytes)
    d2h = int(NQ * 8 + (1 + P) * nh * 8)

    if rank != 0:
        return 0
    # roofline of the dominant kernel, the histogram: one shared-memory atomic increment per counted pair
    # against the measured conflict-free increment rate (DRAM is idle: coordinates and counts stay in
    # shared memory and L2); the FP64 view (the reference's 10 flops per pair) beside it
    lib.xns_measure_smem_atomic_peak.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    atom_peak = C.c_double(0)
    lib.xns_measure_smem_atomic_peak(ctx.handle, C.byref(atom_peak))
    peak = C.c_double(0)
    lib.xns_measure_fma_peak(ctx.handle, 1, C.byref(peak))
    hist_avg = hist_ms / args.steps
    inc = pairs / (hist_avg * 1e-3) / 1e9
    # pairs of the job: every rank's structure (replicas) or the one shared structure (--shard)
    units = 1 if args.shard else world
    par = ("one structure over %d ranks (histogram shards + NCCL all-reduce of the counts)" % world if args.shard
           else "replicas x%d (one structure per rank)" % world)
    line = {"metric": METRIC, "value": job_rate(units, pairs, ms_step), "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "strong" if args.shard else "weak", "vs_baseline": None,
            "dtype": "f32 distance estimate + f64 exact re-binning near bin edges, u64 counts (histogram); f64 "
                     "angle-split transform (I(q)); f64 (PDF)",
            "data": "synthetic (seeded)",
            "patterns_per_s": units / (ms_step * 1e-3),
            "config": config_block(els, nh, args.cells), "parallelism": par,
            "stages_ms": {"histogram": hist_avg, "pdf": pdf_ms / args.steps, "iq": iq_ms / args.steps},
            "roofline": {"kernel": "hist_window_kernel", "bound": "smem_atomic", "achieved": inc, "peak": atom_peak.value,
                         "unit": "1e9 shared-memory increments/s", "frac": inc / atom_peak.value if atom_peak.value else None,
                         "traffic": HIST_TRAFFIC_30 if args.cells == CELLS else None,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one hist_window_kernel "
                                           "launch of this workload (108.4 MB + 4.3 MB; 1-pass capture)",
                         "peak_source": "measured in-process (conflict-free atomicAdd loop, xns_measure_smem_atomic_peak)",
                         "fp64_view": {"flops_per_pair": HIST_FLOPS_PER_PAIR, "peak_tflops": peak.value,
                                       "frac": HIST_FLOPS_PER_PAIR * pairs / (hist_avg * 1e-3) / 1e12 / peak.value}},
            "e2e": {"value": job_rate(units, pairs, e2e_ms), "unit": "pairs/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches), "clocks": clk}
    # the full-size histogram, hashed (the reference arm prints the hash of the reference's calcHist for the
    # same cube; tests/golden holds the one the reference's own code produced)
    step_device()
    torch.cuda.synchronize()
    h_last = d_hist.cpu().numpy().view(np.uint64)
    line["histogram_sha256"] = hist_sha256(h_last)
    gpath = os.path.join(ROOT, "tests", "golden", "histhash__rocksalt30_seed0_b0.001.npz")
    if args.cells == CELLS and rank == 0 and not args.shard and os.path.exists(gpath):
        with np.load(gpath) as g:
            line["histogram_matches_reference"] = {"equal": line["histogram_sha256"] == str(g["sha256"]),
                                                   "reference_sha256": str(g["sha256"]),
                                                   "source": "tests/golden/histhash__rocksalt30_seed0_b0.001.npz "
                                                             "(calcHist of the reference, tests/golden/make_golden.py)"}
    if world == 1 and not args.no_extra:
        line.update(extra_rows(args))
    if world == 1 and not args.no_cpu_baseline:
        v, kind, cores, sample, _ = cpu_reference_sample()
        line["cpu_baseline"] = {"value": v, "unit": "pairs/s", "cores": cores, "kind": kind, "sample": sample}
        # the full-size pattern against FP64: I(q) against the reference's calcInt1DHist of the same
        # histogram, the rPDF against the oracle's PDF of it (bit for bit), every pair counted once
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        step_device()
        torch.cuda.synchronize()
        h = d_hist.cpu().numpy().view(np.uint64)
        I_ours, pdf_ours = d_I.cpu().numpy(), d_pdf.cpu().numpy()
        try:
            R, rk = orc.Reference(threads=cores), "reference calcInt1DHist"
        except FileNotFoundError:
            R, rk = orc.Oracle(), "oracle port of calcInt1DHist"
        I_ref = R.int_1d_hist(h, n_el, nh, BIN, q, 0, sl=SL)
        rel = np.abs(I_ours - I_ref) / np.abs(I_ref)
        pdf_ref = orc.Oracle().pdf(h, n_el, nh, BIN, 2, p0, SL)
        line["max_rel_err_vs_reference"] = {
            "iq": float(rel.max()), "iq_q_at_max": float(q[int(rel.argmax())]), "iq_checker": rk,
            "iq_points_above_1e-5": int((rel > 1e-5).sum()), "iq_points": int(len(q)),
            "rpdf_identical_to_oracle": bool(np.array_equal(pdf_ours, pdf_ref)),
            "histogram_counts_every_pair_once": bool(int(h.sum()) == pairs)}
    print(json.dumps(line))
    ctx.close()
    return 0


# ---- secondary workloads (one GPU): the other measurement rows of the hot path -------------------
def _measure(ctx, call, steps, warmup, stage):
    """Runs call() warmup + steps times; returns (mean event time of the whole call in ms, mean
    kernel-only stage time in ms, kernels launched in the timed calls, clocks)."""
    import torch
    from xns_b200 import lib
    lib.xns_last_stage_ms.argtypes = [__import__("ctypes").c_void_p, __import__("ctypes").c_int]
    lib.xns_last_stage_ms.restype = __import__("ctypes").c_double
    for _ in range(warmup):
        call()
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    clocks = Clocks(0)
    clocks.start()
    l0 = ctx.kernel_launches
    tot = kern = 0.0
    for _ in range(steps):
        flush.fill_(1.0)
        ev0.record(stream)
        call()
        ev1.record(stream)
        ev1.synchronize()
        tot += ev0.elapsed_time(ev1)
        kern += lib.xns_last_stage_ms(ctx.handle, stage)
    return tot / steps, kern / steps, ctx.kernel_launches - l0, clocks.stop()


def _fma_peaks(ctx):
    import ctypes as C
    from xns_b200 import lib
    lib.xns_measure_fma_peak.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
    p64, p32 = C.c_double(0), C.c_double(0)
    lib.xns_measure_fma_peak(ctx.handle, 1, C.byref(p64))
    lib.xns_measure_fma_peak(ctx.handle, 0, C.byref(p32))
    return p64.value, p32.value


def _ctx0():
    import torch
    import xns_b200
    torch.cuda.set_device(0)
    ctx = xns_b200.Context(0)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    return ctx


DEBYE_GOLDEN = os.path.join(ROOT, "tests", "golden", "debye__fcc5000_neutron.npz")


def debye_measure(ctx, steps, warmup):
    """Exact Debye double sum (calcIntDebye), fcc sphere a = 4.078 A cropped to 5000 atoms, Gaussian
    displacement 0.05 A, neutron b = 7.63 fm, 1024 q in [0.1, 10).  `value` = atom pairs / call time of
    the host-buffer C-ABI call (coordinates in, I(q) out).  The sum runs on the integer tensor cores
    (debye_tc_kernel, the default on a uniform mesh); its roofline is stated as the FP32 sine recurrence's
    was, 4 flops per (pair, q) term over the kernel-only stage time against the FP32 peak, so that the two
    paths compare on one scale.  The error is against the reference's own
    calcIntDebye of the same input (tests/golden, made by tests/golden/make_golden.py)."""
    import xns_b200
    from xns_b200 import synth
    els = synth.fcc_sphere(n=5000, a=4.078, sigma=0.05, seed=0)
    q = synth.q_mesh(0.1, 10.0, 1024)
    n = 5000
    pairs = n * (n - 1) // 2
    ms, kms, launches, clk = _measure(ctx, lambda: ctx.calc_int_debye(els, q, xns_b200.NEUTRON, sl=[7.63]), steps,
                                      warmup, 3)
    p64, p32 = _fma_peaks(ctx)
    achieved = 4.0 * pairs * len(q) / (kms * 1e-3) / 1e12
    line = {"metric": "atom-pairs/s", "value": pairs / (ms * 1e-3), "unit": "pairs/s", "n_gpus": 1, "steps": steps,
            "warmup": warmup, "ms_per_step": ms, "kernel_ms": kms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "data": "synthetic (seeded)",
            "dtype": "int8 digit products on the tensor cores (sin/cos of coarse q: 3 digits; offsets x r_min/r: 4), "
                     "exact int32 sums, f64 reductions",
            "patterns_per_s": 1e3 / ms,
            "config": {"workload": "exact Debye, fcc sphere 5000 atoms a=4.078 A sigma=0.05 A, neutron, 1024 q in [0.1,10)",
                       "pairs_per_step": pairs, "nq": len(q), "l2": "flushed (512 MB write) before every timed step"},
            "roofline": {"kernel": "debye_tc_kernel (tcgen05 kind::i8)", "bound": "fp32-equivalent: 4 flops per (pair, q) "
                         "term against the FP32 peak, the measure of the FP32 sine recurrence it replaces",
                         "achieved": achieved, "peak": p32,
                         "unit": "TFLOP/s", "frac": achieved / p32, "traffic": None, "flops_per_term": 4,
                         "time": "kernel-only stage (closest-pair pass, tensor-core kernel, +1e-8 kernel, epilogue)",
                         "peak_source": "measured in-process (FFMA loop, xns_measure_fma_peak)"},
            "e2e": {"value": pairs / (ms * 1e-3), "unit": "pairs/s", "ms_per_step": ms, "h2d_bytes_per_step": n * 24 + 8 * 1024,
                    "d2h_bytes_per_step": 8 * 1024},
            "gpu_launches": int(launches), "clocks": clk}
    if os.path.exists(DEBYE_GOLDEN):
        with np.load(DEBYE_GOLDEN) as g:
            gx, Iref = g["xyz"], g["I"]
        if np.array_equal(gx, np.concatenate(els)):
            I = ctx.calc_int_debye(els, q, xns_b200.NEUTRON, sl=[7.63])
            rel = np.abs(I - Iref) / np.abs(Iref)
            line["max_rel_err_vs_reference"] = {
                "atoms": n, "max": float(rel.max()), "q_at_max": float(q[int(rel.argmax())]),
                "I_at_max_over_max_I": float(abs(Iref[int(rel.argmax())]) / np.abs(Iref).max()),
                "points_above_1e-5": int((rel > 1e-5).sum()), "points": len(q),
                "reference": "calcIntDebye of the reference on the same 5000 atoms (tests/golden/debye__fcc5000_neutron.npz)"}
    return line


def debye_workload(args):
    ctx = _ctx0()
    line = debye_measure(ctx, args.steps, args.warmup)
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        from xns_b200 import synth
        cores = os.cpu_count() or 1
        try:
            R, kind = orc.Reference(threads=cores), "reference"
        except FileNotFoundError:
            R, kind = orc.Oracle(), "port"
        els = synth.fcc_sphere(n=5000, a=4.078, sigma=0.05, seed=0)
        q = synth.q_mesh(0.1, 10.0, 1024)
        m = 1500
        while True:
            sub = [els[0][:m]]
            t = time.perf_counter()
            R.int_debye(sub, q, 0, sl=[7.63])
            dt = time.perf_counter() - t
            if dt > 3.0 or m >= 5000:
                break
            m = min(5000, int(m * min(2.0, max(1.2, (8.0 / max(dt, 1e-3)) ** 0.5))))
        line["cpu_baseline"] = {"value": m * (m - 1) // 2 / dt, "unit": "pairs/s", "cores": cores, "kind": kind,
                                "sample": "calcIntDebye on the first %d atoms of the sphere, 1024 q, %.2f s" % (m, dt)}
    print(json.dumps(line))
    ctx.close()
    return 0


def batch_measure(ctx, steps, warmup, count=256, errors=True):
    """An ensemble of fcc spheres (a = 4.078 A), atom counts log-uniform in [1e3, 2e5], each with its own
    Gaussian displacement sigma in [0.02, 0.1] A; 0.001 A bins, 4096 q in [0.1, 25), neutron b = 7.63 fm.
    Metric: patterns (I(q) of one structure) per second of the batched pass (one plan, one persistent
    histogram launch, one exact tensor-core transform), next to the plain path (one Debye_hist call
    per structure)."""
    import xns_b200
    from xns_b200 import synth
    structs, ns, sig = synth.sphere_ensemble(count=count, seed=0)
    bin = 0.001
    nh = max(synth.hist_size(s, bin) for s in structs)
    q = synth.q_mesh(0.1, 25.0, 4096)
    sl = [[7.63]] * len(structs)
    pairs = int(sum(int(n) * (int(n) - 1) // 2 for n in ns))
    chosen = lambda: ctx.calc_batch_debye_hist(structs, nh, bin, q, xns_b200.NEUTRON, sl=sl)  # noqa: E731
    ms_c, kms_c, launches_c, clk = _measure(ctx, chosen, steps, warmup, 0)

    def plain():  # the common bin count keeps the transform's sinc planes cached between structures
        for s in structs:
            ctx.calc_pdf_and_debye(s, nh, bin, xns_b200.DEBYE_HIST, 0, 0.0, q, xns_b200.NEUTRON, sl=[7.63])

    ms_p, _, launches_p, _ = _measure(ctx, plain, max(1, steps // 2), 1, 0)
    b = ctx.batch(structs, nh, bin, q, xns_b200.NEUTRON, sl=sl, autotune=True)
    I, h = b.run(want_hist=True)
    reps = []
    for _ in range(3):
        b.run()
        reps.append(b.last_ms)
    ct, wb, tms = b.tuning()
    b.close()
    # per-pattern error for the smallest, a median and the largest structure: against the reference's
    # FP64 transform (calcInt1DHist, its summation order) on the same histograms, and against an
    # extended-precision (x87 80-bit) sum on 128 q points that include the deepest minima -- at those
    # minima the sequential FP64 sum itself is off by up to ~1e-5 for 2e5-atom particles
    errs = {}
    if errors:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        O = orc.Oracle()
        for s in sorted({int(np.argmin(ns)), int(np.argsort(ns)[len(ns) // 2]), int(np.argmax(ns))}):
            hs = h[s * nh:(s + 1) * nh]
            Io = O.int_1d_hist(hs, [int(ns[s])], nh, bin, q, 0, sl=[7.63])
            sel = np.unique(np.concatenate([np.argsort(np.abs(Io))[:64], np.linspace(0, len(q) - 1, 64).astype(int)]))
            k = np.nonzero(hs)[0]
            r = (k.astype(np.longdouble) + 0.5) * np.longdouble(bin)
            hk = hs[k].astype(np.longdouble)
            G = np.zeros(len(sel), dtype=np.longdouble)
            for c in range(0, len(sel), 8):
                x = np.outer(q[sel[c:c + 8]].astype(np.longdouble), r)
                G[c:c + 8] = (np.sin(x) / (x + np.longdouble(1e-8))) @ hk
            Ix = np.asarray((int(ns[s]) * np.longdouble(7.63) ** 2 + 2 * np.longdouble(7.63) ** 2 * G) / int(ns[s]),
                            dtype=np.float64)
            errs["%d atoms" % ns[s]] = {"vs_reference_fp64": float(np.max(np.abs(I[s] - Io) / np.abs(Io))),
                                        "vs_extended_128q": float(np.max(np.abs(I[s][sel] - Ix) / np.abs(Ix))),
                                        "reference_fp64_vs_extended_128q": float(np.max(np.abs(Io[sel] - Ix) / np.abs(Ix)))}
    line = {"metric": "patterns/s", "value": len(structs) / (ms_c * 1e-3), "unit": "patterns/s", "n_gpus": 1,
            "steps": steps, "warmup": warmup, "ms_per_step": ms_c, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 distances + u64 counts (histogram), integer-digit tensor-core transform",
            "data": "synthetic (seeded)",
            "config": {"workload": "%d fcc spheres a=4.078 A, %d-%d atoms (log-uniform), sigma 0.02-0.1 A, bin 0.001 A "
                                   "(%d bins), 4096 q in [0.1,25), neutron" % (len(structs), ns.min(), ns.max(), nh),
                       "structures": len(structs), "atoms": int(ns.sum()), "pairs_per_step": pairs,
                       "l2": "flushed (512 MB write) before every timed step"},
            "pairs_per_s": pairs / (ms_c * 1e-3),
            "plain": {"patterns_per_s": len(structs) / (ms_p * 1e-3), "ms_per_step": ms_p,
                      "path": "one xns_calc_pdf_and_debye (Debye_hist) call per structure"},
            "speedup_vs_plain": ms_p / ms_c,
            "graph_replay_ms": min(reps), "autotune": {"cell_target": ct, "window_bins": wb, "hist_ms": tms},
            "max_rel_err_vs_fp64": errs,
            "e2e": {"value": len(structs) / (ms_c * 1e-3), "unit": "patterns/s", "ms_per_step": ms_c,
                    "h2d_bytes_per_step": int(ns.sum()) * 24 + 8 * len(q), "d2h_bytes_per_step": 8 * len(q) * len(structs)},
            "gpu_launches": int(launches_c), "clocks": clk}
    return line


def batch_workload(args):
    ctx = _ctx0()
    print(json.dumps(batch_measure(ctx, args.steps, args.warmup, args.batch_count, not args.no_cpu_baseline)))
    ctx.close()
    return 0


def plane_measure(ctx, steps, warmup, cells2d=63, mesh2d=1024, polar=True, errors=True):
    """2D intensity of a 1,000,188-atom fcc crystallite (a = 3.61 A, 63^3 cells, 5 % second
    species, seeded random orientation), X-ray form factors from seeded 4-Gaussian coefficients, one
    orientation, on two meshes:
      * the Cartesian q plane normal to the beam, 1024 x 1024 points over [-8, 8)^2 A^-1 (the
        configuration's mesh): xns_calc_amp_plane, a complex digit product on the tensor cores -- the
        line's `value` (call time of the host-buffer C-ABI call);
      * the reference's polar mesh of 1024 q in [0.05, 8) x 1024 phi with lambda = 0.01 A (nearly flat):
        xns_calc_int_2d, the drop-in path (FP64 phase, FP32 sincos) -- reported beside it.
    Metric (atom, mesh point) terms per second."""
    import xns_b200
    from xns_b200 import synth
    els = synth.fcc_crystallite(cells=cells2d, a=3.61, subst=0.05, seed=0)
    n = sum(len(e) for e in els)
    nq = nfi = mesh2d
    coef = synth.ff_coefficients(2, seed=3)
    dq = 16.0 / nq
    plane = lambda: ctx.calc_amp_plane(els, -8.0, dq, nq, -8.0, dq, nq, xns_b200.XRAY, coef=coef)  # noqa: E731
    ms, kms, launches, clk = _measure(ctx, plane, steps, warmup, 4)
    q = synth.q_mesh(0.05, 8.0, nq)
    ff = synth.ff_on_mesh(coef, q)
    terms = n * nq * nfi
    p64, p32 = _fma_peaks(ctx)
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {"bf16_tflops": 1590.0}
    bf16 = float(peaks["bf16_tflops"])
    line = {"metric": "terms/s", "value": terms / (ms * 1e-3), "unit": "(atom, q-point) terms/s", "n_gpus": 1,
            "steps": steps, "warmup": warmup, "ms_per_step": ms, "kernel_ms": kms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 sines, 4 integer digits per value on the bf16 tensor cores, exact sums, f64 totals",
            "data": "synthetic (seeded)", "patterns_per_s": 1e3 / ms,
            "config": {"workload": "2D Cartesian q plane %dx%d over [-8,8)^2, fcc crystallite %d atoms, X-ray" % (nq, nfi, n),
                       "atoms": n, "terms_per_step": terms},
            "roofline": {"kernel": "sinc_exact_kernel<PlaneScheme> (digit GEMM)", "bound": "tensor",
                         "achieved": 8.0 * terms / (kms * 1e-3) / 1e12, "peak": bf16, "unit": "TFLOP/s",
                         "frac": 8.0 * terms / (kms * 1e-3) / 1e12 / bf16, "traffic": None,
                         "time": "kernel-only stage",
                         "flops_per_term": "8 (one complex multiply-add), counted once: the 10 digit products "
                                           "per term are not credited",
                         "peak_source": "MEASURED_PEAKS.json bf16_tflops (cuBLAS bf16, burst)"},
            "e2e": {"value": terms / (ms * 1e-3), "unit": "(atom, q-point) terms/s", "ms_per_step": ms,
                    "h2d_bytes_per_step": n * 24, "d2h_bytes_per_step": nq * nfi * 8},
            "gpu_launches": int(launches), "clocks": clk}
    if polar:
        pol = lambda: ctx.calc_int_2d(els, q, nfi, [0, 0, 0], [0, 0, 0], [1, 1, 1], 5, 0.01, xns_b200.XRAY, ff=ff)  # noqa
        ms_p, kms_p, _, _ = _measure(ctx, pol, 1, 1, 4)
        line["polar_mesh"] = {"ms_per_step": ms_p, "terms_per_s": terms / (ms_p * 1e-3),
                              "roofline_fp64_frac": 10.0 * terms / (kms_p * 1e-3) / 1e12 / p64,
                              "path": "xns_calc_int_2d (drop-in), 1024 q x 1024 phi, lambda 0.01 A"}
    if errors:
        # sampled points of the full-size plane against the FP64 sum over all atoms (the oracle's restatement of
        # the reference's amplitude sum at q_z = 0): 64 columns of two rows
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        Ip = ctx.calc_amp_plane(els, -8.0, dq, nq, -8.0, dq, nq, xns_b200.XRAY, coef=coef).reshape(nq, nq)
        O = orc.Oracle()
        errs = []
        for iy in (nq // 3, nq // 2 + 7):
            cols = slice(nq // 4, nq // 4 + 64)
            ref = O.amp_plane(els, -8.0 + (nq // 4) * dq, dq, 64, -8.0 + iy * dq, dq, 1, xns_b200.XRAY, coef=coef).ravel()
            got = Ip[iy, cols]
            floor = 1e-2 * float(np.median(np.abs(ref)))
            errs.append(float(np.max(np.abs(got - ref) / np.maximum(np.abs(ref), floor))))
        line["max_rel_err_vs_fp64"] = {"plane_sampled_points": 128, "max": max(errs),
                                       "note": "relative, denominator floored at 1 % of the sampled median"}
    return line, (els, q, ff, n, nfi)


def twod_workload(args):
    import xns_b200
    ctx = _ctx0()
    line, (els, q, ff, n, nfi) = plane_measure(ctx, args.steps, args.warmup, args.cells2d, args.mesh2d, True,
                                               not args.no_cpu_baseline)
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        cores = os.cpu_count() or 1
        try:
            R, kind = orc.Reference(threads=cores), "reference"
        except FileNotFoundError:
            R, kind = orc.Oracle(), "port"
        # the reference parallelises over q rows: one row per core, a 64-point phi mesh (the work per term
        # does not depend on the mesh)
        rows, nfi_s = cores, 64
        t = time.perf_counter()
        R.int_2d(els, q[:rows], nfi_s, [0, 0, 0], [0, 0, 0], [1, 1, 1], 5, 0.01, xns_b200.XRAY, ff=ff[:, :rows])
        dt = time.perf_counter() - t
        line["cpu_baseline"] = {"value": n * rows * nfi_s / dt, "unit": "(atom, q-point) terms/s", "cores": cores,
                                "kind": kind, "sample": "calcInt2D on %d q rows x %d phi, all %d atoms, %.2f s"
                                                        % (rows, nfi_s, n, dt)}
    print(json.dumps(line))
    ctx.close()
    return 0


def extra_rows(args):
    """The other configurations of the hot path, measured in the default run's process on the same GPU
    (each with its own clock record): the exact Debye sum (5000-atom sphere), the Cartesian 2D plane
    (1e6 atoms, 1024^2) and the batched ensemble against the plain per-structure path (256 spheres)."""
    ctx = _ctx0()
    out = {}
    keep = ("metric", "value", "unit", "ms_per_step", "kernel_ms", "steps", "warmup", "config", "roofline", "e2e",
            "clocks", "gpu_launches", "max_rel_err_vs_reference", "max_rel_err_vs_fp64", "patterns_per_s", "plain",
            "speedup_vs_plain", "pairs_per_s", "graph_replay_ms", "autotune", "dtype")
    d = debye_measure(ctx, 20, 5)
    out["debye_sphere5000"] = {k: v for k, v in d.items() if k in keep}
    p, _ = plane_measure(ctx, 5, 3, polar=False, errors=True)
    out["plane2d_crystallite1e6"] = {k: v for k, v in p.items() if k in keep}
    b = batch_measure(ctx, 3, 3, errors=False)
    out["batch_spheres256"] = {k: v for k, v in b.items() if k in keep}
    ctx.close()
    return out


def build_workload(args):
    """Structure builder (block::calcAtoms, CalcFunctions.cpp:251-392): an atom-list block of 200,000
    sites, where the O(sites^2) merge of sites closer than 0.5 A dominates.  Metric site pairs/s (one
    build examines S(S-1)/2 site pairs); roofline: the merge kernel's FP32 prefilter, 9 flops per pair
    (3 subtractions and the 3 FMAs of d^2 - thr), on the FP32 pipe."""
    import ctypes as C

    import torch
    import xns_b200
    from xns_b200 import lib, synth
    torch.cuda.set_device(0)
    lib.xns_last_stage_ms.argtypes = [C.c_void_p, C.c_int]
    lib.xns_last_stage_ms.restype = C.c_double
    ctx = xns_b200.Context(0)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    n = args.build_sites
    blk = synth.atom_file_block(n)
    S = n
    pairs = S * (S - 1) // 2
    for w in range(args.warmup):
        ctx.build_atoms([blk], 2, w)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    clocks = Clocks(0)
    clocks.start()
    l0 = ctx.kernel_launches
    call = merge = fill = e2e = 0.0
    atoms = 0
    for k in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dev, n_el, _ = ctx.build_atoms([blk], 2, 100 + k)
        call += ctx.last_kernel_ms
        merge += lib.xns_last_stage_ms(ctx.handle, 5)
        fill += lib.xns_last_stage_ms(ctx.handle, 6)
        xs = ctx.copy_atoms(n_el)  # the atoms to the host, as the reference's ra[] vectors
        e2e += (time.perf_counter() - t0) * 1e3
        atoms = int(n_el.sum())
    launches = ctx.kernel_launches - l0
    clk = clocks.stop()
    call, merge, fill, e2e = call / args.steps, merge / args.steps, fill / args.steps, e2e / args.steps
    p64, p32 = _fma_peaks(ctx)
    achieved = 9.0 * pairs / (merge * 1e-3) / 1e12
    # the crystal case and the 1e7-atom scale case, timed the same way (device events of the call)
    extra = {}
    for name, b, nel in (("rock-salt 30^3 cells, 10% vacancies, sigma 0.07 A", synth.rocksalt_block(30), 2),):
        for w in range(2):
            ctx.build_atoms([b], nel, w)
        ms = []
        for k in range(3):
            _, ne, _ = ctx.build_atoms([b], nel, 10 + k)
            ms.append(ctx.last_kernel_ms)
        extra[name] = {"atoms": int(ne.sum()), "ms": float(np.median(ms)), "atoms_per_s": float(ne.sum() / np.median(ms) * 1e3)}
    line = {"metric": "site pairs/s (structure build)", "value": pairs / (call * 1e-3), "unit": "pairs/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": call, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 prefilter, f64 exact test and coordinates", "data": "synthetic (seeded)",
            "config": {"workload": "structure builder: atom-list block of %d sites (density 0.05 A^-3, 2%% planted "
                                   "within 0.1 A, occupancy 0.6 on every third site) -> %d atoms" % (n, atoms),
                       "site_pairs_per_step": pairs, "merge_ms": merge, "write_ms": fill,
                       "l2": "flushed (512 MB write) before every timed step", "also": extra},
            "roofline": {"kernel": "merge_kernel", "bound": "fp32", "achieved": achieved, "peak": p32, "unit": "TFLOP/s",
                         "frac": achieved / p32, "traffic": None, "flops_per_pair": 9,
                         "peak_source": "measured in-process (FFMA loop, xns_measure_fma_peak)"},
            "e2e": {"value": pairs / (e2e * 1e-3), "unit": "pairs/s", "ms_per_step": e2e, "h2d_bytes_per_step": S * 40,
                    "d2h_bytes_per_step": atoms * 24},
            "gpu_launches": int(launches), "clocks": clk}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        try:
            R, kind = orc.Reference(), "reference"
            run = lambda b: R.calc_atoms([b], 2)  # noqa: E731
        except FileNotFoundError:
            R, kind = orc.Oracle(), "port"
            run = lambda b: R.build_atoms([b], 2, 1)  # noqa: E731
        m = 10000
        while True:
            b = synth.atom_file_block(m)
            t = time.perf_counter()
            run(b)
            dt = time.perf_counter() - t
            if dt > 4.0 or m >= n:
                break
            m = min(n, int(m * min(2.0, max(1.2, (12.0 / max(dt, 1e-3)) ** 0.5))))
        line["cpu_baseline"] = {"value": m * (m - 1) // 2 / dt, "unit": "pairs/s", "cores": 1, "kind": kind,
                                "sample": "block::calcAtoms on an atom-list block of %d sites of the same generator, "
                                          "%.2f s (the reference's builder is single-threaded)" % (m, dt)}
        # the crystal case through the reference's builder as well
        for name, b, nel in (("rock-salt 30^3 cells, 10% vacancies, sigma 0.07 A", synth.rocksalt_block(30), 2),):
            t = time.perf_counter()
            (R.calc_atoms([b], nel) if kind == "reference" else R.build_atoms([b], nel, 1))
            extra[name]["reference_ms"] = (time.perf_counter() - t) * 1e3
    print(json.dumps(line))
    ctx.close()
    return 0


def learned_workload(args):
    """Config 5, the learned binning correction, at the sizes one bench call can run: training structures
    from the config-3 generator (fcc crystallites, 5 % substitution, Gaussian displacements) plus 10 %
    random-packed amorphous clusters with atom counts log-uniform in [--learned-nmin, --learned-nmax]
    (5k-50k by default; config 5 names 5k-2M), coarse 0.02 A histograms, the MLP trained on the GPU to
    predict each coarse bin's moments, 2048 q in [0.1, 20); the exact double sum of the held-out
    structures is the arbiter (tolerance 1e-4, else the exact path is used).  Then the scale case: one
    fcc sphere of --scale-atoms atoms (1e7 by default), coarse histogram -> I(q) with and without the
    correction, against the 0.001 A histogram's I(q) (binning error below (q 0.001)^2 / 24 = 1.7e-5 at
    q = 20): the exact double sum of 5e13 pairs is out of reach (its per-pair +1e-8 histogram updates
    alone take hours).  Progress on stderr; one JSON line on stdout."""
    import time

    import xns_b200
    from xns_b200 import learned, synth
    T0 = time.perf_counter()

    def say(msg):
        print("[%7.1f s] %s" % (time.perf_counter() - T0, msg), file=sys.stderr, flush=True)

    ctx = _ctx0()
    sync = __import__("torch").cuda.synchronize
    q = synth.q_mesh(0.1, 20.0, 2048)
    structs, sls = learned.training_structures(args.learned_count, seed=0, nmin=args.learned_nmin,
                                               nmax=args.learned_nmax)
    ns = [sum(len(e) for e in st) for st in structs]
    say("%d training structures, %d-%d atoms" % (len(structs), min(ns), max(ns)))
    lc = learned.LearnedCorrector(ctx, q, tol=1e-4)
    t0 = time.perf_counter()
    lc.fit(structs, sls)
    fit_s = time.perf_counter() - t0
    say("fit done: %s" % json.dumps(lc.validation))
    # throughput of both paths on the same structures (the first 32 of the set)
    sub, subl = structs[:32], sls[:32]
    sync()
    t0 = time.perf_counter()
    I_c, hs, s0, _ = learned.hist_pass(ctx, sub, subl, q, learned.COARSE_BIN)
    I_l = lc.corrected(I_c, hs, s0)
    sync()
    t_learned = time.perf_counter() - t0
    t0 = time.perf_counter()
    I_x = learned.exact_pass(ctx, sub, subl, q)
    sync()
    t_exact = time.perf_counter() - t0
    say("throughput: learned %.3f s, exact %.3f s for %d structures" % (t_learned, t_exact, len(sub)))
    line = {"metric": "patterns/s", "value": len(sub) / t_learned, "unit": "patterns/s", "n_gpus": 1,
            "higher_is_better": True, "workload": "learned binning correction (config 5, scaled)",
            "config": {"structures": len(structs), "atoms_min": int(min(ns)), "atoms_max": int(max(ns)),
                       "q": "2048 in [0.1, 20)", "coarse_bin": learned.COARSE_BIN, "mlp": "3 layers, width 256, GELU, "
                       "BF16 weights, FP32 accumulation", "holdout": "12.5 %", "tolerance": 1e-4},
            "exact_patterns_per_s": len(sub) / t_exact, "learned_vs_exact_speed": t_exact / t_learned,
            "fit_s": fit_s, "validation": lc.validation, "trusted": bool(lc.trusted),
            "path_chosen": "learned" if lc.trusted else "exact (the validated error exceeds the tolerance)",
            "throughput_sample": "%d structures, %d-%d atoms" % (len(sub), min(ns[:32]), max(ns[:32])),
            "max_rel_err_learned_vs_exact_on_sample": float(learned.max_rel_err(I_l, I_x).max())}
    if args.scale_atoms > 0:
        els = synth.fcc_sphere(n=args.scale_atoms, a=3.61, sigma=0.05, seed=5)
        n = len(els[0])
        say("scale case: %d atoms" % n)

        def hist_iq(bin):
            sync()
            t0 = time.perf_counter()
            nh = synth.hist_size(els, bin)
            h = ctx.calc_hist(els, nh, bin)
            I = ctx.calc_int_1d_hist(h, [n], nh, bin, q, xns_b200.NEUTRON, sl=[1.0])
            sync()
            return I, h, nh, time.perf_counter() - t0

        I_c, hc, nh, t_c = hist_iq(learned.COARSE_BIN)
        say("coarse histogram and I(q): %.1f s" % t_c)
        h = learned.weighted_hist(els, [1.0], hc, nh)
        s0 = learned.self_term(els, [1.0])
        t0 = time.perf_counter()
        I_lc = I_c + learned.correction(ctx, h, lc._moments_pred(h), q, s0)
        t_corr = time.perf_counter() - t0
        unif = np.tile(np.array([[0.0, 1.0 / 12.0]], np.float32), (nh, 1))
        I_u = I_c + learned.correction(ctx, h, unif, q, s0)
        I_f, _, _, t_f = hist_iq(0.001)
        say("0.001 A histogram and I(q): %.1f s" % t_f)
        line["scale_case"] = {"atoms": n, "pairs": n * (n - 1) // 2, "q_points": len(q),
                              "coarse_path_s": t_c + t_corr, "fine_path_s": t_f,
                              "reference": "I(q) from the 0.001 A histogram (binning error < 1.7e-5 at q = 20)",
                              "max_rel_err_vs_fine": {"coarse": float(learned.max_rel_err(I_c, I_f)),
                                                      "uniform_bins": float(learned.max_rel_err(I_u, I_f)),
                                                      "learned": float(learned.max_rel_err(I_lc, I_f))}}
    lc.close()
    ctx.close()
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="histogram workload: skip the other configurations' keys (Debye, 2D plane, batch)")
    ap.add_argument("--cells", type=int, default=CELLS,
                    help="cube edge in unit cells (default 30, the benchmark; smaller only for profiler captures)")
    ap.add_argument("--workload", default="histogram", choices=["histogram", "debye", "2d", "batch", "build",
                                                                "learned"],
                    help="histogram (default, the headline: rock-salt cube histogram + rPDF + I(q)); debye (fcc "
                         "sphere exact Debye sum), 2d (q plane), batch (ensemble of spheres) and build (structure "
                         "builder on an atom-list block) and learned (config 5: the learned binning correction, "
                         "scaled) run on one GPU")
    ap.add_argument("--batch-count", type=int, default=256, help="batch workload: structures in the ensemble")
    ap.add_argument("--cells2d", type=int, default=63, help="2d workload: crystallite edge in fcc cells (63: 1e6 atoms)")
    ap.add_argument("--mesh2d", type=int, default=1024, help="2d workload: q and phi points")
    ap.add_argument("--build-sites", type=int, default=200000, help="build workload: sites of the atom-list block")
    ap.add_argument("--learned-count", type=int, default=256, help="learned workload: training structures")
    ap.add_argument("--learned-nmin", type=int, default=5000, help="learned workload: smallest structure (atoms)")
    ap.add_argument("--learned-nmax", type=int, default=50000, help="learned workload: largest structure (atoms)")
    ap.add_argument("--scale-atoms", type=int, default=10000000,
                    help="learned workload: atoms of the scale case's fcc sphere (0: no scale case)")
    ap.add_argument("--shard", action="store_true",
                    help="histogram workload with N ranks: split one structure over the ranks (strong scaling) "
                         "instead of one structure per rank")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "debye" and args.impl == "ours":
        return debye_workload(args)
    if args.workload == "2d" and args.impl == "ours":
        return twod_workload(args)
    if args.workload == "batch" and args.impl == "ours":
        return batch_workload(args)
    if args.workload == "build" and args.impl == "ours":
        return build_workload(args)
    if args.workload == "learned" and args.impl == "ours":
        return learned_workload(args)
    if args.impl == "reference":
        if args.workload != "histogram":
            return reference_workload_arm(args, rank)
        return reference_arm(args, rank, world)
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local_rank))
    try:
        return ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as tdist
            tdist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
