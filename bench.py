"""Benchmark: D3Q19 collide-stream MLUPS on B200 (one JSON line on rank 0).

Workload (default): D3Q19 TRT (Lambda = 1/4), 256^3 periodic box, Taylor-Green
vortex (u0 = 0.05, rho = 1) plus seeded Gaussian velocity noise (sigma 1e-3),
tau = 0.55, FP32 populations. One step = one fused pull collide-stream launch
over the whole box. Inputs (1.27 GB per population buffer) are larger than L2,
so no flush is needed between steps.

value   MLUPS with the populations resident in HBM (CUDA events, max over ranks)
e2e     MLUPS through the reference-facing C ABI (lbm_launch_step_gpu_*) with
        host buffers: the pinned host field is copied in, K steps run, the
        field is copied back, all inside the timed region
roofline achieved HBM GB/s of the step kernel = 152 B/LU x cells / mean launch
        time, against the measured copy bandwidth (MEASURED_PEAKS.json)

`--impl reference` times LB-Cube's own CPU step (oracle/_ref, or the oracle
restatement when the reference build is absent) on a bounded sample of the
same workload and prints the same metric.

Multi-GPU (torchrun, N ranks): one periodic 256 x 256 x 256N box cut into
z-slabs of 256^3, one per GPU (weak scaling); every step exchanges the face
populations with the two neighbours over NCCL point-to-point, overlapped with
the interior planes (lb-cube_b200/slab.py). value = cells of all ranks x
steps / the max over ranks of the timed region.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "lb-cube_b200"))

METRIC = "D3Q19 MLUPS, %HBM peak: FP32 vs FP16-store @L2err<=1e-3; adjoint cost/fwd"
UNIT = "MLUPS"
NX = NY = NZ = 256
TAU = 0.55
U0 = 0.05
NOISE = 1e-3
SEED = 20261203
OP = "TRT"  # operator of the timed run
BYTES_PER_LU = 2 * 19 * 4  # read Q + write Q FP32 populations


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-variants", action="store_true",
                    help="skip the other storage/lattice variants and the 2000-step accuracy run")
    ap.add_argument("--storage", choices=["fp32", "f16s", "bf16s", "e3m12s", "q15s"], default="fp32",
                    help="population storage of the timed run (16-bit ones are shifted)")
    ap.add_argument("--size", type=int, default=256,
                    help="cube edge; smaller sizes are for profiling captures only")
    ap.add_argument("--collision", choices=["TRT", "BGK", "MRT"], default="TRT",
                    help="operator of the timed run (TRT is the headline; others for profiling captures)")
    ap.add_argument("--kernel-survey", action="store_true",
                    help="launch every kernel family a few times at 128^3 (1024^2 for 2-D), time each with "
                         "CUDA events and print one JSON line; the command the per-kernel ncu summary captures")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="run only the adjoint cost measurements (KE: D3Q19 BGK FP32; reactive: D3Q19 TRT "
                         "+ 2 D3Q7 with --storage in the forward; --size cube, --steps steps, checkpoint "
                         "every min(100, steps)) and print them; for profiling captures")
    a = ap.parse_args()
    global NX, NY, NZ, OP
    NX = NY = NZ = a.size
    OP = a.collision
    return a


def config_dict():
    return {
        "workload": f"D3Q19 {OP}{' (Lambda 1/4)' if OP == 'TRT' else ''} {NX}^3 periodic, Taylor-Green u0 0.05 "
                    "+ N(0, 1e-3) velocity noise, tau 0.55, FP32 populations",
        "lattice": "D3Q19", "collision": OP, "storage": "fp32",
        "nx": NX, "ny": NY, "nz": NZ, "tau": TAU,
        "l2": f"inputs larger than L2 ({19 * 4 * NX * NY * NZ / 1e9:.2f} GB per population buffer); no flush",
    }


# ----------------------------------------------------------------------------
# clocks sampled during the timed region
# ----------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def committed_traffic(kernel_key):
    """Per-launch DRAM bytes from a committed ncu summary, scaled to the bench box."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as fh:
            return json.load(fh).get(kernel_key)
    except (OSError, ValueError):
        return None


# ----------------------------------------------------------------------------
# engine arm
# ----------------------------------------------------------------------------
C_D3Q19 = [[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
           [1, 1, 0], [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1], [1, 0, -1],
           [-1, 0, -1], [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1]]
FORMAT_NOTE = {"q15s": "Q15 shifted (16-bit fixed point, |f/w - rho0| < 1)",
               "e3m12s": "E3M12 shifted (sign, 3-bit exponent, 12-bit mantissa)",
               "f16s": "IEEE FP16 shifted (x 4096)", "bf16s": "BF16 shifted"}
FORMATS16 = ("q15s", "e3m12s", "f16s", "bf16s")
def make_initial_state(torch, E, dev):
    """Taylor-Green + seeded noise, rho = 1, built on the device and turned into
    equilibrium populations by the engine's own init kernel."""
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED)
    k = 2 * math.pi / NX
    ax = torch.arange(NX, device=dev, dtype=torch.float64) * k
    z, y, x = torch.meshgrid(ax, ax, ax, indexing="ij")
    u = torch.empty((3, NZ, NY, NX), device=dev, dtype=torch.float64)
    u[0] = U0 * torch.sin(x) * torch.cos(y) * torch.cos(z)
    u[1] = -U0 * torch.cos(x) * torch.sin(y) * torch.cos(z)
    u[2] = 0.0
    u += NOISE * torch.randn(u.shape, generator=gen, device=dev, dtype=torch.float64)
    del x, y, z
    rho = torch.ones((NZ, NY, NX), device=dev, dtype=torch.float32)
    u32 = u.to(torch.float32).contiguous()
    del u
    f = torch.empty((19, NZ, NY, NX), device=dev, dtype=torch.float32)
    E.check(E.init_equilibrium_async("D3Q19", "float", rho, u32, f, NX, NY, NZ))
    torch.cuda.synchronize()
    return f


def _time_steps(torch, launch, a, b, steps, warmup):
    """Mean ms per step of `launch(cur, nxt)` with ping-pong buffers (CUDA events)."""
    import lbcube as E

    for _ in range(warmup):
        E.check(launch(a, b))
        a, b = b, a
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.current_stream()
    t0.record(stream)
    for _ in range(steps):
        rc = launch(a, b)
        a, b = b, a
    t1.record(stream)
    torch.cuda.synchronize()
    E.check(rc)
    return t0.elapsed_time(t1) / steps


def run_variants(torch, E, dev, f32, peak, fp32_ms):
    """Single-GPU characterisation at the same size: every operator in FP32 and
    FP64 for D3Q19 and D3Q27, and 16-bit shifted storage. 10 warm-up + 200 timed
    steps each (5 + 50 for the slower FP64 / D3Q27 operators)."""
    omega = 1.0 / TAU
    cells = NX * NY * NZ
    out = []

    def rec(name, ms, bytes_per_lu, **kw):
        gbs = bytes_per_lu * cells / (ms * 1e-3) / 1e9
        d = {"variant": name, "mlups": round(cells / (ms * 1e-3) / 1e6, 1), "ms_per_step": round(ms, 5),
             "bytes_per_lu": bytes_per_lu, "achieved_gbs": round(gbs, 1), "hbm_frac": round(gbs / peak, 4)}
        d.update(kw)
        out.append(d)
        return d

    g = torch.empty_like(f32)
    for op in ("MRT", "BGK", "RLBM"):
        ms = _time_steps(torch, lambda a, b, op=op: E.launch_step_gpu("D3Q19", "float", op, a, b, NX, NY, NZ, omega),
                         f32.clone(), g, 200, 10)
        rec(f"D3Q19 {op} fp32", ms, 152)
    # every step also reduces mass, kinetic energy, max |u| and the blow-up flag
    nb = E.diagnostics_partials_bytes("D3Q19", NX, NY, NZ)
    part = torch.empty(nb, dtype=torch.uint8, device=dev)
    diag = torch.empty(5, dtype=torch.float64, device=dev)
    ms = _time_steps(torch, lambda a, b: E.step_diagnostics_async("D3Q19", "float", "TRT", a, b, NX, NY, NZ, omega,
                                                                    part, nb, diag, speed_limit=0.2),
                     f32.clone(), g, 200, 10)
    rec("D3Q19 TRT fp32 + diagnostics every step", ms, 152, vs_plain_step=round(fp32_ms / ms, 3))
    count = [0]

    def every10(a, b):  # the drivers' usual cadence: diagnostics on every 10th step
        count[0] += 1
        if count[0] % 10 == 0:
            return E.step_diagnostics_async("D3Q19", "float", "TRT", a, b, NX, NY, NZ, omega, part, nb, diag,
                                            speed_limit=0.2)
        return E.launch_step_gpu("D3Q19", "float", "TRT", a, b, NX, NY, NZ, omega)

    ms = _time_steps(torch, every10, f32.clone(), g, 200, 10)
    rec("D3Q19 TRT fp32 + diagnostics every 10th step", ms, 152, vs_plain_step=round(fp32_ms / ms, 3))
    del part, diag
    h = torch.empty(f32.shape, dtype=torch.int16, device=dev)
    hg = torch.empty_like(h)
    for fmt in FORMATS16:
        E.check(E.encode_shifted_async("D3Q19", fmt, "float", f32, h, NX, NY, NZ, 1.0))
        for op in ("TRT", "MRT"):
            ms = _time_steps(torch, lambda a, b, op=op, fmt=fmt: E.step_shifted_async("D3Q19", fmt, op, a, b, NX, NY, NZ, omega, 1.0),
                             h, hg, 200, 10)
            ref = fp32_ms if op == "TRT" else out[0]["ms_per_step"]
            rec(f"D3Q19 {op} {fmt}", ms, 76, format=FORMAT_NOTE[fmt], speedup_vs_fp32=round(ref / ms, 3))
    del h, hg, g
    # FP64 (the reference drivers' precision) and the 27-velocity bandwidth case
    f64 = f32.double()
    g64 = torch.empty_like(f64)
    for op in ("BGK", "TRT", "MRT", "RLBM"):
        ms = _time_steps(torch, lambda a, b, op=op: E.launch_step_gpu("D3Q19", "double", op, a, b, NX, NY, NZ, omega),
                         f64.clone(), g64, 200 if op == "BGK" else 50, 5)
        rec(f"D3Q19 {op} fp64", ms, 304)
    del f64, g64
    f27 = torch.empty((27, NZ, NY, NX), dtype=torch.float32, device=dev)
    rho = torch.ones((NZ, NY, NX), dtype=torch.float32, device=dev)
    u = torch.zeros((3, NZ, NY, NX), dtype=torch.float32, device=dev)
    E.check(E.init_equilibrium_async("D3Q27", "float", rho, u, f27, NX, NY, NZ))
    g27 = torch.empty_like(f27)
    for op in ("BGK", "TRT", "MRT", "RLBM"):
        ms = _time_steps(torch, lambda a, b, op=op: E.launch_step_gpu("D3Q27", "float", op, a, b, NX, NY, NZ, omega),
                         f27.clone(), g27, 200 if op == "BGK" else 50, 5)
        rec(f"D3Q27 {op} fp32", ms, 216)
    f27d = f27.double()
    del f27, g27
    g27d = torch.empty_like(f27d)
    for op in ("BGK", "MRT"):
        ms = _time_steps(torch, lambda a, b, op=op: E.launch_step_gpu("D3Q27", "double", op, a, b, NX, NY, NZ, omega),
                         f27d.clone(), g27d, 50, 5)
        rec(f"D3Q27 {op} fp64", ms, 432)
    del f27d, g27d, rho, u
    torch.cuda.empty_cache()
    return out


def run_accuracy(torch, E, dev, steps=2000):
    """Velocity rel-L2 after `steps` steps of the benchmark case against the FP64
    run (the FP64 kernel is bit-identical to the reference CPU path)."""
    omega = 1.0 / TAU
    c = torch.tensor(C_D3Q19, dtype=torch.float64, device=dev)

    def vel(f):
        f = f.double()
        return torch.einsum("qd,q...->d...", c, f) / f.sum(0)

    res = {}
    for op in ("TRT", "MRT"):
        f32 = make_initial_state(torch, E, dev)
        f64 = f32.double()  # same initial bits in both precisions
        runs = {"fp64": [f64, torch.empty_like(f64)], "fp32": [f32, torch.empty_like(f32)]}
        for fmt in FORMATS16:
            h = torch.empty(f32.shape, dtype=torch.int16, device=dev)
            E.check(E.encode_shifted_async("D3Q19", fmt, "float", f32, h, NX, NY, NZ, 1.0))
            runs[fmt] = [h, torch.empty_like(h)]
        for _ in range(steps):
            for k, (a, b) in runs.items():
                if k == "fp64":
                    rc = E.launch_step_gpu("D3Q19", "double", op, a, b, NX, NY, NZ, omega)
                elif k == "fp32":
                    rc = E.launch_step_gpu("D3Q19", "float", op, a, b, NX, NY, NZ, omega)
                else:
                    rc = E.step_shifted_async("D3Q19", k, op, a, b, NX, NY, NZ, omega, 1.0)
                E.check(rc)
                runs[k] = [b, a]
        u_ref = vel(runs["fp64"][0])
        nref = torch.linalg.vector_norm(u_ref)
        errs = {}
        for k, (a, _) in runs.items():
            if k == "fp64":
                continue
            if k == "fp32":
                fk = a
            else:
                fk = torch.empty((19, NZ, NY, NX), dtype=torch.float64, device=dev)
                E.check(E.decode_shifted_async("D3Q19", k, "double", a, fk, NX, NY, NZ, 1.0))
            errs[k] = float(torch.linalg.vector_norm(vel(fk) - u_ref) / nref)
            del fk
        res[op] = {k: float(f"{v:.4g}") for k, v in errs.items()}
        del runs, u_ref
        torch.cuda.empty_cache()
    return {"steps": steps, "quantity": "velocity relative L2 vs the FP64 run", "tau": TAU, "by_collision": res}


def solenoidal_field(torch, dev, n, amp, k_peak, seed):
    """Seeded random solenoidal velocity: curl of a random-phase vector potential
    whose spectrum peaks at |k| = k_peak, rescaled to max |u| = amp."""
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    k1 = torch.fft.fftfreq(n, d=1.0 / n, device=dev)
    kz, ky, kx = torch.meshgrid(k1, k1, k1, indexing="ij")
    kk = torch.sqrt(kx * kx + ky * ky + kz * kz)
    env = (kk / k_peak) ** 2 * torch.exp(-(kk / k_peak) ** 2)
    A = [torch.fft.fftn(torch.randn((n, n, n), generator=gen, device=dev, dtype=torch.float64)) * env
         for _ in range(3)]
    Ax, Ay, Az = A
    uh = [1j * (ky * Az - kz * Ay), 1j * (kz * Ax - kx * Az), 1j * (kx * Ay - ky * Ax)]
    u = torch.stack([torch.fft.ifftn(c).real for c in uh])
    return (u * (amp / u.abs().max())).contiguous()


def run_adjoint_cost(torch, E, dev, n=128, steps=2000, interval=100, tau=0.56):
    """Adjoint cost: full gradient (forward with checkpoints, segment
    recomputation, adjoint sweep) over one forward run, D3Q19 BGK FP32."""
    u0 = solenoidal_field(torch, dev, n, 0.03, 4.0, SEED).float()
    rho0 = torch.ones((n, n, n), dtype=torch.float32, device=dev)
    f = torch.empty((19, n, n, n), dtype=torch.float32, device=dev)
    g = torch.empty_like(f)
    omega = 1.0 / tau

    def forward():
        E.check(E.init_equilibrium_async("D3Q19", "float", rho0, u0, f, n, n, n))
        a, b = f, g
        for _ in range(steps):
            E.check(E.launch_step_gpu("D3Q19", "float", "BGK", a, b, n, n, n, omega))
            a, b = b, a

    nbytes = E.ke_gradient_workspace_bytes("D3Q19", "float", n, n, n, steps, interval)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    out = torch.zeros(2, dtype=torch.float64, device=dev)
    grad = torch.empty_like(u0)

    def gradient():
        E.check(E.ke_gradient_async("D3Q19", "float", "BGK", rho0, u0, n, n, n, tau, steps, interval,
                                    ws, nbytes, out, grad))

    def timed(fn):
        fn()  # warm-up
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        fn()
        t1.record()
        torch.cuda.synchronize()
        return t0.elapsed_time(t1)

    fwd_ms = timed(forward)
    grad_ms = timed(gradient)
    res = {"config": f"D3Q19 BGK FP32 {n}^3, tau {tau}, {steps} steps, solenoidal u0 (amplitude 0.03, "
                     f"spectrum peak |k| = 4), objective final total kinetic energy, checkpoint every {interval}",
           "forward_ms": round(fwd_ms, 2), "gradient_ms": round(grad_ms, 2),
           "cost_ratio": round(grad_ms / fwd_ms, 3), "objective": float(out[0]), "dJ_dtau": float(out[1]),
           "workspace_gb": round(nbytes / 1e9, 2)}
    del ws, f, g, grad
    torch.cuda.empty_cache()
    return res


def blob_fields(torch, dev, n, block, seed):
    """A and B in {0, 1} on interleaved block^3 cubes (a 3-D checkerboard) with a
    seeded random phase per axis; B = 1 - A."""
    gen = torch.Generator().manual_seed(seed)
    off = torch.randint(0, block, (3,), generator=gen).tolist()
    ax = torch.arange(n, device=dev)
    z, y, x = torch.meshgrid(ax, ax, ax, indexing="ij")
    parity = ((x + off[2]) // block + (y + off[1]) // block + (z + off[0]) // block) % 2
    a = (parity == 0).float()
    return a.contiguous(), (1.0 - a).contiguous()


def run_slab_gradient(torch, E, dev, n=160, steps=600, interval=100, world=2, tau=0.56, tau_c=0.55,
                      k=0.03 / 16, storage="f16s", c0=0.5):
    """The reactive gradient of run_reactive_adjoint_cost decomposed into `world`
    z-slabs (slab.ReactiveSlabGradient), all ranks in this process on this GPU
    (slab.run_local: faces exchanged by device copies, all-reduces as sums),
    against the same gradient of the whole box (lbm_reactive_gradient_async).
    Both timed by CUDA events around the whole call, host sequencing included;
    the slab path issues every rank's launches from this one process and runs
    them one after the other on this GPU, so the ratio is the cost of the
    decomposition (exchanges, unpacks, twice the launches from one host
    thread), not a multi-GPU speed-up. The slab's initial-state gradients
    must equal the whole box's bit for bit."""
    import slab

    u0 = solenoidal_field(torch, dev, n, 0.03, 4.0, SEED).float()
    rho0 = torch.ones((n, n, n), dtype=torch.float32, device=dev)
    a0, b0 = blob_fields(torch, dev, n, 16, SEED)
    nbytes = E.reactive_gradient_workspace_bytes("D3Q19", "float", n, n, n, steps, interval, storage=storage)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    res = torch.zeros(4, dtype=torch.float64, device=dev)
    ga, gb, gu = torch.empty_like(a0), torch.empty_like(b0), torch.empty_like(u0)
    grads = [slab.ReactiveSlabGradient(torch, "D3Q19", "float", "TRT", "mean_product", n, n, n, tau, tau_c, k,
                                       steps, interval, r, world, dev, storage=storage, c0=c0)
             for r in range(world)]
    inputs = [(rho0[g.z0:g.z0 + g.nz].contiguous(), u0[:, g.z0:g.z0 + g.nz].contiguous(),
               a0[g.z0:g.z0 + g.nz].contiguous(), b0[g.z0:g.z0 + g.nz].contiguous()) for g in grads]

    def whole():
        E.check(E.reactive_gradient_async("D3Q19", "float", "TRT", "mean_product", rho0, u0, a0, b0, n, n, n,
                                          tau, tau_c, k, steps, interval, ws, nbytes, res, ga, gb, gu,
                                          storage=storage, c0=c0))

    def timed(fn):
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        fn()
        t1.record()
        torch.cuda.synchronize()
        return t0.elapsed_time(t1)

    whole()  # warm-up
    slab.run_local(grads, inputs)
    whole_ms = timed(whole)
    slab_ms = timed(lambda: slab.run_local(grads, inputs))
    same = all(bool(torch.equal(torch.cat([getattr(g, name) for g in grads], dim=axis).view(torch.int32),
                                want.view(torch.int32)))
               for name, axis, want in (("grad_a0", 0, ga), ("grad_b0", 0, gb), ("grad_u0", 1, gu)))
    rel = max(abs(float(x) - float(y)) / max(abs(float(y)), 1e-300)
              for x, y in zip(grads[0].result.tolist(), res.tolist()))
    store = "FP32" if storage is None else f"{FORMAT_NOTE[storage]} populations (scalars shifted by {c0})"
    return {"config": f"the reactive gradient of adjoint_reactive at {n}^3, {steps} steps, checkpoint every "
                      f"{interval}, {store}, as {world} z-slabs of {n // world} planes stepped in one process",
            "whole_box_ms": round(whole_ms, 2), "slabs_ms": round(slab_ms, 2),
            "slabs_over_whole_box": round(slab_ms / whole_ms, 3),
            "gradient_fields_bit_identical": same, "scalars_max_rel_diff": rel}


def run_reactive_adjoint_cost(torch, E, dev, n=192, steps=3000, interval=100, tau=0.56, tau_c=0.55,
                              k=0.03 / 16, storage=None, c0=0.5):
    """Reactive adjoint cost: D3Q19 TRT + two D3Q7 scalars (A + B -> C), FP32
    (storage None) or 16-bit shifted population storage in the forward
    (storage a format; fluid shifted by 1, scalars by c0) with the FP32 adjoint;
    objective final mean C; gradient w.r.t. k, tau, tau_c and the initial A and
    B fields, over one forward run of the same coupled step."""
    u0 = solenoidal_field(torch, dev, n, 0.03, 4.0, SEED).float()
    rho0 = torch.ones((n, n, n), dtype=torch.float32, device=dev)
    a0, b0 = blob_fields(torch, dev, n, 16, SEED)
    nbytes = E.reactive_gradient_workspace_bytes("D3Q19", "float", n, n, n, steps, interval, storage=storage)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    res = torch.zeros(4, dtype=torch.float64, device=dev)
    ga, gb = torch.empty_like(a0), torch.empty_like(b0)
    omega, omega_c = 1.0 / tau, 1.0 / tau_c
    # forward-only run of the same coupled step, in buffers of the workspace
    elem = torch.float32 if storage is None else torch.int16
    es = 4 if storage is None else 2
    f = [ws[i * 19 * n ** 3 * es:(i + 1) * 19 * n ** 3 * es].view(elem).view(19, n, n, n) for i in range(2)]
    base = 38 * n ** 3 * es
    sc = [ws[base + i * 7 * n ** 3 * es: base + (i + 1) * 7 * n ** 3 * es].view(elem).view(7, n, n, n)
          for i in range(4)]
    if storage is not None:  # FP32 initial fields, encoded into the 16-bit buffers
        tf = torch.empty((19, n, n, n), dtype=torch.float32, device=dev)
        ts = torch.empty((7, n, n, n), dtype=torch.float32, device=dev)

    def forward(nsteps):
        if storage is None:
            E.check(E.init_equilibrium_async("D3Q19", "float", rho0, u0, f[0], n, n, n))
            E.check(E.init_equilibrium_async("D3Q7", "float", a0, u0, sc[0], n, n, n))
            E.check(E.init_equilibrium_async("D3Q7", "float", b0, u0, sc[2], n, n, n))
        else:
            E.check(E.init_equilibrium_async("D3Q19", "float", rho0, u0, tf, n, n, n))
            E.check(E.encode_shifted_async("D3Q19", storage, "float", tf, f[0], n, n, n, 1.0))
            for src, dst in ((a0, sc[0]), (b0, sc[2])):
                E.check(E.init_equilibrium_async("D3Q7", "float", src, u0, ts, n, n, n))
                E.check(E.encode_shifted_async("D3Q7", storage, "float", ts, dst, n, n, n, c0))
        for s_ in range(nsteps):
            i, j = s_ % 2, (s_ + 1) % 2
            if storage is None:
                E.check(E.fluid_reaction_ab_async("D3Q19", "float", "TRT", f[i], f[j], sc[i], sc[j], sc[2 + i],
                                                  sc[2 + j], n, n, n, omega, omega_c, k))
            else:
                E.check(E.fluid_reaction_ab_shifted_async("D3Q19", storage, "TRT", f[i], f[j], sc[i], sc[j],
                                                          sc[2 + i], sc[2 + j], n, n, n, omega, omega_c, k,
                                                          1.0, c0))

    def gradient(nsteps, nint):
        E.check(E.reactive_gradient_async("D3Q19", "float", "TRT", "mean_product", rho0, u0, a0, b0, n, n, n,
                                          tau, tau_c, k, nsteps, nint, ws, nbytes, res, ga, gb, storage=storage,
                                          c0=c0))

    def timed(fn):
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        fn()
        t1.record()
        torch.cuda.synchronize()
        return t0.elapsed_time(t1)

    forward(4)  # warm-up (kernels, clocks)
    gradient(4, 2)
    fwd_ms = timed(lambda: forward(steps))
    grad_ms = timed(lambda: gradient(steps, interval))
    r = res.tolist()
    store = "FP32" if storage is None else f"{FORMAT_NOTE[storage]} populations (scalars shifted by {c0})"
    out = {"config": f"D3Q19 TRT + 2 x D3Q7 (A + B -> C) {n}^3, {store} in the forward, FP32 adjoint, "
                     f"tau {tau}, tau_c {tau_c}, k {k:.6g}, {steps} steps, solenoidal u0 (amplitude 0.03, "
                     f"spectrum peak |k| = 4), A, B in {{0, 1}} on interleaved 16^3 blocks, objective final mean "
                     f"C, checkpoint every {interval}",
           "forward_ms": round(fwd_ms, 2), "gradient_ms": round(grad_ms, 2),
           "cost_ratio": round(grad_ms / fwd_ms, 3), "objective": r[0], "dJ_dk": r[1], "dJ_dtau": r[2],
           "dJ_dtau_c": r[3], "grad_a0_l2": float(torch.linalg.vector_norm(ga.double())),
           "workspace_gb": round(nbytes / 1e9, 2)}
    del ws, ga, gb, f, sc
    torch.cuda.empty_cache()
    return out


def run_reactive_mixing(torch, E, dev, n=1024, steps=20000, every=10):
    """2-D reactive mixing: D2Q9 MRT double shear layer coupled to two D2Q5
    scalars reacting A + B -> C (workloads.reactive_shear_layer: u = 0.04 tanh
    with delta = 8 cells, the periodic form of turbulent_shear_layer.cpp:61-63,
    seeded transverse perturbation; A = 1 in the top half, B = 1 in the bottom
    half; Pe = 1000, Da = 1 for L = n; tau 0.6). Every step is one fused fluid +
    reaction launch; every `every` steps that launch also writes the statistics
    partials and lbm_reactive_stats_append_async writes the eight
    ReactiveDiagnostics fields to the next row of a device table. The `every`
    steps plus the append are captured once in a CUDA graph and replayed
    steps / every times: no host work and no synchronisation in the loop.
    The same workload and sequence is held to the reference CPU run in
    tests/test_gpu_c3.py."""
    import workloads as W

    w = W.reactive_shear_layer(n)
    tau, tau_c, k = w["tau"], w["tau_c"], w["k"]
    rho = torch.from_numpy(w["rho"]).to(dev)
    u = torch.from_numpy(w["u"]).to(dev)
    a0 = torch.from_numpy(w["a0"]).to(dev)
    b0 = torch.from_numpy(w["b0"]).to(dev)
    f = [torch.empty((9, n, n), device=dev, dtype=torch.float32) for _ in range(2)]
    A = [torch.empty((5, n, n), device=dev, dtype=torch.float32) for _ in range(2)]
    B = [torch.empty((5, n, n), device=dev, dtype=torch.float32) for _ in range(2)]
    pb = E.stats_partials_bytes("D2Q9", n, n, 1)
    part = torch.empty(pb, dtype=torch.uint8, device=dev)
    rows = steps // every
    table = torch.zeros((rows, 8), dtype=torch.float64, device=dev)
    row = torch.zeros(1, dtype=torch.int64, device=dev)
    assert every % 2 == 0  # a chunk returns the ping-pong buffers to their places

    def init():
        E.check(E.init_equilibrium_async("D2Q9", "float", rho, u, f[0], n, n, 1))
        E.check(E.init_equilibrium_async("D2Q5", "float", a0, u, A[0], n, n, 1))
        E.check(E.init_equilibrium_async("D2Q5", "float", b0, u, B[0], n, n, 1))
        row.zero_()

    def chunk(stream):
        for s_ in range(every):
            i, j = s_ % 2, (s_ + 1) % 2
            last = s_ == every - 1
            E.check(E.fluid_reaction_ab_async("D2Q9", "float", "MRT", f[i], f[j], A[i], A[j], B[i], B[j], n, n, 1,
                                              1.0 / tau, 1.0 / tau_c, k, part if last else None, pb if last else 0,
                                              stream=stream))
        E.check(E.reactive_stats_append_async("D2Q9", "float", n, n, 1, k, part, pb, table, rows, row,
                                              stream=stream))

    s = torch.cuda.Stream(device=dev)
    init()
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        chunk(s)  # warm-up outside the graph
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        chunk(s)
    init()
    for _ in range(2):  # warm-up replays
        graph.replay()
    init()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(s)
    with torch.cuda.stream(s):
        for _ in range(rows):
            graph.replay()
    t1.record(s)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    assert int(row.item()) == rows
    cells = n * n
    mlups = cells * steps / (ms * 1e-3) / 1e6
    last = table[-1].tolist()
    out = {"config": f"D2Q9 MRT + 2 x D2Q5 (A + B -> C) FP32 {n}^2 double shear layer (u0 0.04, delta 8), "
                     f"tau {tau}, tau_c {tau_c:.5f} (Pe 1000), k {k:.6g} (Da 1), {steps} steps, statistics "
                     f"every {every} steps in FP64 on the device; {every}-step chunks replayed as one CUDA graph",
           "ms_total": round(ms, 2), "mlups": round(mlups, 1), "bytes_per_lu": 152,
           "achieved_gbs": round(152 * cells * steps / (ms * 1e-3) / 1e9, 1),
           "stats_rows": int(table.shape[0]), "final_mean_a": last[0], "final_mean_b": last[1],
           "final_segregation_intensity": last[5], "final_true_rate": last[6], "final_mixed_rate": last[7]}
    del graph, f, A, B, part, table
    torch.cuda.empty_cache()
    return out


def run_kernel_survey(torch, E, dev, n=128, reps=10):
    """Every kernel family once per rep at n^3 (D2Q9 at (8n)^2), timed with CUDA
    events; algorithmic bytes per launch give the achieved GB/s."""
    import slab

    f32, f64 = torch.float32, torch.float64
    cells = n ** 3
    om, omc, k = 1.0 / TAU, 1.0 / 0.55, 0.002
    out = []

    def timed(name, bytes_per_launch, launch):
        for _ in range(2):
            E.check(launch())
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(reps):
            E.check(launch())
        t1.record()
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1) / reps
        out.append({"kernel": name, "ms": round(ms, 4), "bytes": int(bytes_per_launch),
                    "gbs": round(bytes_per_launch / (ms * 1e-3) / 1e9, 1)})

    rho = torch.ones((n, n, n), dtype=f32, device=dev)
    u = 0.02 * torch.randn((3, n, n, n), dtype=f32, device=dev, generator=torch.Generator(device=dev).manual_seed(1))
    f = torch.empty((19, n, n, n), dtype=f32, device=dev)
    g = torch.empty_like(f)
    timed("init_equilibrium D3Q19 f32", cells * (4 * 4 + 76), lambda: E.init_equilibrium_async("D3Q19", "float", rho, u, f, n, n, n))
    for op in ("TRT", "BGK", "MRT", "RLBM"):
        timed(f"step D3Q19 f32 {op}", cells * 152, lambda op=op: E.step_async("D3Q19", "float", op, f, g, n, n, n, om))
    fd, gd = f.double(), torch.empty((19, n, n, n), dtype=f64, device=dev)
    timed("step D3Q19 f64 BGK", cells * 304, lambda: E.step_async("D3Q19", "double", "BGK", fd, gd, n, n, n, om))
    del fd, gd
    f27 = torch.empty((27, n, n, n), dtype=f32, device=dev)
    E.check(E.init_equilibrium_async("D3Q27", "float", rho, u, f27, n, n, n))
    g27 = torch.empty_like(f27)
    for op in ("BGK", "TRT", "MRT", "RLBM"):
        timed(f"step D3Q27 f32 {op}", cells * 216, lambda op=op: E.step_async("D3Q27", "float", op, f27, g27, n, n, n, om))
    d27 = slab.SlabDomain(torch, "D3Q27", "float", "BGK", n, n, n, om, 0, 1, dev)
    d27.pack(f27)
    ex27 = slab.LocalExchange([d27])
    ex27.exchange_all()

    def slab_step27():
        d27.compute(f27, g27)
        ex27.exchange_all()
        return 0
    timed("slab step D3Q27 f32 BGK (interior + faces + face copies)", cells * 216, slab_step27)
    del d27, ex27, f27, g27
    h = torch.empty((19, n, n, n), dtype=torch.int16, device=dev)
    hg = torch.empty_like(h)
    timed("encode_shifted D3Q19 q15s", cells * (76 + 38), lambda: E.encode_shifted_async("D3Q19", "q15s", "float", f, h, n, n, n))
    for fmt, op in (("q15s", "TRT"), ("f16s", "TRT"), ("f16s", "MRT"), ("e3m12s", "TRT")):
        E.check(E.encode_shifted_async("D3Q19", fmt, "float", f, h, n, n, n))
        timed(f"step_shifted D3Q19 {fmt} {op}", cells * 76,
              lambda fmt=fmt, op=op: E.step_shifted_async("D3Q19", fmt, op, h, hg, n, n, n, om))
    timed("decode_shifted D3Q19 f16s", cells * (38 + 76), lambda: E.decode_shifted_async("D3Q19", "f16s", "float", h, g, n, n, n))
    del h, hg
    # scalars and the coupled step
    a = torch.empty((7, n, n, n), dtype=f32, device=dev)
    b = torch.empty_like(a)
    E.check(E.init_equilibrium_async("D3Q7", "float", rho, u, a, n, n, n))
    E.check(E.init_equilibrium_async("D3Q7", "float", rho * 0.5, u, b, n, n, n))
    a2, b2 = torch.empty_like(a), torch.empty_like(b)
    timed("scalar_step D3Q19/D3Q7 f32", cells * (56 + 76), lambda: E.scalar_step_async("D3Q19", "float", a, a2, f, n, n, n, omc))
    timed("reaction_ab D3Q19/D3Q7 f32", cells * (112 + 76), lambda: E.reaction_ab_async("D3Q19", "float", a, a2, b, b2, f, n, n, n, omc, k))
    pb = E.stats_partials_bytes("D3Q19", n, n, n)
    part = torch.empty(pb, dtype=torch.uint8, device=dev)
    st = torch.empty(8, dtype=f64, device=dev)
    timed("fluid_reaction D3Q19 f32 TRT", cells * 264,
          lambda: E.fluid_reaction_ab_async("D3Q19", "float", "TRT", f, g, a, a2, b, b2, n, n, n, om, omc, k))
    timed("fluid_reaction D3Q19 f32 TRT + stats", cells * 264,
          lambda: E.fluid_reaction_ab_async("D3Q19", "float", "TRT", f, g, a, a2, b, b2, n, n, n, om, omc, k, part, pb))
    h19 = [torch.empty((19, n, n, n), dtype=torch.int16, device=dev) for _ in range(2)]
    h7 = [torch.empty((7, n, n, n), dtype=torch.int16, device=dev) for _ in range(4)]
    E.check(E.encode_shifted_async("D3Q19", "f16s", "float", f, h19[0], n, n, n, 1.0))
    E.check(E.encode_shifted_async("D3Q7", "f16s", "float", a, h7[0], n, n, n, 0.5))
    E.check(E.encode_shifted_async("D3Q7", "f16s", "float", b, h7[2], n, n, n, 0.5))
    timed("fluid_reaction_shifted D3Q19 f16s TRT", cells * 132,
          lambda: E.fluid_reaction_ab_shifted_async("D3Q19", "f16s", "TRT", h19[0], h19[1], h7[0], h7[1], h7[2],
                                                    h7[3], n, n, n, om, omc, k, 1.0, 0.5))
    del h19, h7
    timed("reactive_stats D3Q7 f32 (2 passes)", cells * 56,
          lambda: E.reactive_stats_async("D3Q7", "float", a, b, n, n, n, k, part, pb, st))
    dpb = E.diagnostics_partials_bytes("D3Q19", n, n, n)
    dpart = torch.empty(dpb, dtype=torch.uint8, device=dev)
    dg = torch.empty(5, dtype=f64, device=dev)
    timed("fluid_diagnostics D3Q19 f32 (2 passes)", cells * 76,
          lambda: E.fluid_diagnostics_async("D3Q19", "float", f, n, n, n, dpart, dpb, dg))
    timed("step_diagnostics D3Q19 f32 TRT", cells * 152,
          lambda: E.step_diagnostics_async("D3Q19", "float", "TRT", f, g, n, n, n, om, dpart, dpb, dg))
    mr, mu, ms = torch.empty(cells, dtype=f32, device=dev), torch.empty((3, cells), dtype=f32, device=dev), \
        torch.empty(cells, dtype=f32, device=dev)
    timed("macro_fields D3Q19 f32", cells * (76 + 20), lambda: E.macro_fields_async("D3Q19", "float", f, n, n, n, mr, mu, ms))
    # adjoint steps
    lam, lam2 = torch.zeros_like(f), torch.zeros_like(f)
    timed("adjoint_step D3Q19 f32 TRT", cells * 228,
          lambda: E.adjoint_step_async("D3Q19", "float", "TRT", f, lam, lam2, n, n, n, TAU))
    del lam, lam2
    # the slab step: one rank, faces exchanged locally
    d = slab.SlabDomain(torch, "D3Q19", "float", "TRT", n, n, n, om, 0, 1, dev)
    d.pack(f)
    ex = slab.LocalExchange([d])
    ex.exchange_all()

    def slab_step():
        d.compute(f, g)
        ex.exchange_all()
        return 0
    timed("slab step D3Q19 f32 TRT (interior + faces + face copies)", cells * 152, slab_step)
    del a, b, a2, b2, part, dpart, mr, mu, ms
    # 2-D: D2Q9 MRT + two D2Q5 at (8n)^2
    m2 = 8 * n
    c2 = m2 * m2
    rho2 = torch.ones((m2, m2), dtype=f32, device=dev)
    u2 = 0.02 * torch.randn((2, m2, m2), dtype=f32, device=dev, generator=torch.Generator(device=dev).manual_seed(2))
    q = torch.empty((9, m2, m2), dtype=f32, device=dev)
    q2 = torch.empty_like(q)
    E.check(E.init_equilibrium_async("D2Q9", "float", rho2, u2, q, m2, m2, 1))
    timed("step D2Q9 f32 MRT", c2 * 72, lambda: E.step_async("D2Q9", "float", "MRT", q, q2, m2, m2, 1, om))
    s5 = [torch.empty((5, m2, m2), dtype=f32, device=dev) for _ in range(4)]
    for t in s5:
        E.check(E.init_equilibrium_async("D2Q5", "float", rho2 * 0.5, u2, t, m2, m2, 1))
    timed("fluid_reaction D2Q9 f32 MRT", c2 * 152,
          lambda: E.fluid_reaction_ab_async("D2Q9", "float", "MRT", q, q2, s5[0], s5[1], s5[2], s5[3], m2, m2, 1, om, omc, k))
    torch.cuda.synchronize()
    return {"kernel_survey": out, "size": f"{n}^3 (2-D: {m2}^2)", "reps": reps,
            "note": "ms = CUDA-event mean over reps after 2 warm-ups; bytes = algorithmic bytes per launch"}


def run_engine(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    import lbcube as E

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    E.load()
    omega = 1.0 / TAU
    cells = NX * NY * NZ

    f = make_initial_state(torch, E, dev)
    storage = args.storage
    bytes_per_lu = BYTES_PER_LU if storage == "fp32" else BYTES_PER_LU // 2
    slabs = None
    launches_per_step = 1
    if storage != "fp32":  # 16-bit codes of the initial state
        h = torch.empty(f.shape, dtype=torch.int16, device=dev)
        E.check(E.encode_shifted_async("D3Q19", storage, "float", f, h, NX, NY, NZ, 1.0))
        torch.cuda.synchronize()
        f = h
    if world > 1:
        # one periodic NX x NY x (NZ * world) box cut into z-slabs, one per rank;
        # the face populations (or their 16-bit codes) cross NVLink (NCCL
        # point-to-point) every step
        import slab

        slabs = slab.SlabDomain(torch, "D3Q19", "float", OP, NX, NY, NZ * world, omega, rank, world, dev,
                                storage=None if storage == "fp32" else storage)
        exchange = slab.DistributedExchange(dist)
        slabs.prime(f, exchange)
        launches_per_step = len(sum(slabs.ranges(), []))

        def step(cur, nxt):
            slabs.step(cur, nxt, exchange)
            return 0
    elif storage == "fp32":
        def step(cur, nxt):
            return E.launch_step_gpu("D3Q19", "float", OP, cur, nxt, NX, NY, NZ, omega)
    else:
        def step(cur, nxt):
            return E.step_shifted_async("D3Q19", storage, OP, cur, nxt, NX, NY, NZ, omega, 1.0)
    g = torch.empty_like(f)

    for _ in range(args.warmup):
        E.check(step(f, g))
        f, g = g, f
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()

    sampler = ClockSampler(local_rank) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    stream = torch.cuda.current_stream()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        rc = step(f, g)
        f, g = g, f
    if slabs is not None:
        slabs.finish()
    t1.record(stream)
    torch.cuda.synchronize()
    E.check(rc)
    clocks = sampler.stop() if sampler else None
    ms = t0.elapsed_time(t1)
    if world > 1:
        dist.barrier()
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps
    value = cells * world * args.steps / (ms * 1e-3) / 1e6
    achieved_gbs = bytes_per_lu * cells / (ms_per_step * 1e-3) / 1e9

    # end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        host = torch.empty(f.shape, dtype=f.dtype, pin_memory=True)
        host.copy_(f)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        f.copy_(host, non_blocking=True)
        for _ in range(args.steps):
            rc = step(f, g)
            f, g = g, f
        if slabs is not None:
            slabs.finish()
        host.copy_(f, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        E.check(rc)
        ems = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ems], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        nbytes = f.numel() * f.element_size()
        e2e = {"value": round(cells * world * args.steps / (ems * 1e-3) / 1e6, 1), "unit": UNIT,
               "h2d_bytes_per_step": nbytes / args.steps, "d2h_bytes_per_step": nbytes / args.steps,
               "note": "pinned host field copied in, K steps via lbm_launch_step_gpu_d3q19_float_trt, "
                       "field copied back; copies amortised over K"}
        if slabs is not None:
            e2e["note"] = e2e["note"].replace(
                "lbm_launch_step_gpu_d3q19_float_trt",
                ("lbm_step_slab_async" if storage == "fp32" else "lbm_step_slab_shifted_async") +
                " + NCCL face exchange")
        elif storage != "fp32":
            e2e["note"] = e2e["note"].replace("lbm_launch_step_gpu_d3q19_float_trt", "lbm_step_shifted_async")
        del host

    if rank != 0:
        return None
    if world == 1:
        parallelism = "single GPU"
    else:
        parallelism = (f"z-slab decomposition of one {NX}x{NY}x{NZ * world} periodic box over {world} GPUs "
                       f"({NZ} planes each), NCCL point-to-point face exchange every step, overlapped with "
                       f"the interior planes")
    peak, peak_kind = measured_hbm_peak()
    traffic = committed_traffic(f"d3q19_float_trt_{NX}") if storage == "fp32" and OP == "TRT" else None
    variants = accuracy = fp16_store = adjoint = adjoint_reactive = adjoint_reactive_16 = mixing = None
    slab_gradient = None
    if world == 1 and not args.no_variants and storage == "fp32" and OP == "TRT":
        variants = run_variants(torch, E, dev, f, peak, ms_per_step)
        del f, g
        torch.cuda.empty_cache()
        accuracy = run_accuracy(torch, E, dev)
        adjoint = run_adjoint_cost(torch, E, dev)
        adjoint_reactive = run_reactive_adjoint_cost(torch, E, dev)
        adjoint_reactive_16 = run_reactive_adjoint_cost(torch, E, dev, storage="f16s")
        adjoint_reactive_16["vs_fp32"] = {
            key: round(adjoint_reactive_16[key] / adjoint_reactive[key] - 1.0, 6)
            for key in ("objective", "dJ_dk", "dJ_dtau_c", "grad_a0_l2")}
        adjoint_reactive_16["forward_speedup_vs_fp32"] = round(adjoint_reactive["forward_ms"] /
                                                               adjoint_reactive_16["forward_ms"], 3)
        # the same gradient against the FP32 forward run of the configuration
        adjoint_reactive_16["cost_ratio_vs_fp32_forward"] = round(adjoint_reactive_16["gradient_ms"] /
                                                                  adjoint_reactive["forward_ms"], 3)
        slab_gradient = run_slab_gradient(torch, E, dev)
        mixing = run_reactive_mixing(torch, E, dev)
        # per operator: the fastest 16-bit format meeting the 1e-3 velocity error
        # bar, with its speed-up over FP32 storage of the same operator
        fp16_store = {"bar": "velocity rel-L2 <= 1e-3 after 2000 steps vs the FP64 run", "by_collision": {}}
        for op in ("TRT", "MRT"):
            pre = f"D3Q19 {op} "
            ok = [v for v in variants if v["variant"].startswith(pre) and v["variant"][len(pre):] in FORMATS16
                  and accuracy["by_collision"][op][v["variant"][len(pre):]] <= 1e-3]
            if ok:
                best = max(ok, key=lambda v: v["mlups"])
                fmt = best["variant"][len(pre):]
                fp16_store["by_collision"][op] = {
                    "format": FORMAT_NOTE[fmt], "mlups": best["mlups"], "hbm_frac": best["hbm_frac"],
                    "speedup_vs_fp32": best["speedup_vs_fp32"],
                    "velocity_rel_l2_2000_steps": accuracy["by_collision"][op][fmt]}
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if storage == "fp32" else f"{storage} storage, f32 compute",
        "data": "synthetic", "config": dict(config_dict(), storage=storage, parallelism=parallelism),
        "roofline": {"bound": "hbm", "achieved": round(achieved_gbs, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved_gbs / peak, 4),
                     "traffic": traffic, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": bytes_per_lu * cells},
        "e2e": e2e, "clocks": clocks, "gpu_launches": args.steps * launches_per_step,
        "fp16_store": fp16_store, "adjoint": adjoint, "adjoint_reactive": adjoint_reactive,
        "adjoint_reactive_f16s": adjoint_reactive_16, "slab_gradient": slab_gradient,
        "reactive_mixing": mixing,
        "variants": variants, "accuracy": accuracy,
    }
    return line


# ----------------------------------------------------------------------------
# CPU baseline (reference CPU path) and the reference arm
# ----------------------------------------------------------------------------
def _reference_lib():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    if O.REF.available:
        return O, O.REF, "reference"
    return O, O.ORACLE, "port"


def workload_slab(O, nz_sample):
    """FP32 equilibrium populations of planes 0 .. nz_sample-1 of the benchmark
    field (Taylor-Green u0 = 0.05 with wavenumber 2 pi / 256 in each axis plus
    seeded N(0, 1e-3) velocity noise, rho = 1), as a periodic slab."""
    import numpy as np

    n = NX * NY * nz_sample
    rng = np.random.default_rng(SEED)
    k = 2 * math.pi / NX
    ax = np.arange(NX) * k
    z, y, x = np.meshgrid(np.arange(nz_sample) * k, ax, ax, indexing="ij")
    u = np.stack([U0 * np.sin(x) * np.cos(y) * np.cos(z), -U0 * np.cos(x) * np.sin(y) * np.cos(z),
                  np.zeros_like(x)]).reshape(3, -1) + NOISE * rng.standard_normal((3, n))
    return O.init_equilibrium("D3Q19", np.ones(n), u, NX, NY, nz_sample, np.float32)


def cpu_sample(nz_sample, steps):
    """Time `steps` serial step_cpu<D3Q19, float, TRT> calls on a 256 x 256 x
    nz_sample periodic slab of the benchmark state (same per-cell work)."""
    O, lib, kind = _reference_lib()
    n = NX * NY * nz_sample
    f = workload_slab(O, nz_sample)
    t = time.perf_counter()
    O.step(f, "D3Q19", "TRT", NX, NY, nz_sample, 1 / TAU, steps=steps, lib=lib)
    dt = time.perf_counter() - t
    return n * steps / dt / 1e6, kind, dt


def cpu_baseline():
    nz_sample, steps = 128, 2
    mlups, kind, dt = cpu_sample(nz_sample, steps)
    return {"value": round(mlups, 3), "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"{steps} steps of step_cpu<D3Q19,float,TRT> on a 256x256x{nz_sample} periodic slab "
                      f"({dt:.1f} s); serial, as the reference is", "host_threads": os.cpu_count()}


def run_reference(args):
    # calibrate: one sample step, then size the per-step slab so the run stays within ~3 min
    rate, kind, _ = cpu_sample(4, 1)
    budget_s = 150.0
    total = max(1, args.steps + args.warmup)
    nz_s = int(max(1, min(64, budget_s * rate * 1e6 / total / (NX * NY))))
    O, lib, kind = _reference_lib()
    n = NX * NY * nz_s
    f = workload_slab(O, nz_s)
    for _ in range(args.warmup):
        f = O.step(f, "D3Q19", "TRT", NX, NY, nz_s, 1 / TAU, steps=1, lib=lib)
    t = time.perf_counter()
    for _ in range(args.steps):
        f = O.step(f, "D3Q19", "TRT", NX, NY, nz_s, 1 / TAU, steps=1, lib=lib)
    dt = time.perf_counter() - t
    value = n * args.steps / dt / 1e6
    sample = (f"each step: step_cpu<D3Q19,float,TRT> on planes 0..{nz_s - 1} of the 256^3 workload field as "
              f"a 256x256x{nz_s} periodic slab (serial reference CPU path, 1 thread of {os.cpu_count()})")
    return {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": dict(config_dict(), slab=f"{NX}x{NY}x{nz_s} (planes 0..{nz_s - 1})"),
            "impl": "reference",
            "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": 1, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if args.kernel_survey:
        import torch

        import lbcube as E

        dev = torch.device("cuda", local_rank)
        torch.cuda.set_device(dev)
        E.load()
        print(json.dumps(run_kernel_survey(torch, E, dev, n=args.size if args.size != 256 else 128)), flush=True)
        return
    if args.adjoint_only:
        import torch

        import lbcube as E

        dev = torch.device("cuda", local_rank)
        torch.cuda.set_device(dev)
        E.load()
        res = run_adjoint_cost(torch, E, dev, n=args.size, steps=args.steps, interval=min(100, args.steps))
        rres = run_reactive_adjoint_cost(torch, E, dev, n=args.size, steps=args.steps,
                                         interval=min(100, args.steps),
                                         storage=None if args.storage == "fp32" else args.storage)
        print(json.dumps({"adjoint": res, "adjoint_reactive": rres}), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        line = run_engine(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
    if rank == 0:
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline()
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
